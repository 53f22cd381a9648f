/*
 * adtlert_b200 -- C ABI of the B200 (sm_100a) forward-and-sensitivity path of AD-TLERT's
 * 2.5D and 3D DC-resistivity operators.
 *
 * One plan per discretization (mesh + survey + wavenumber quadrature; a 3D operator is one
 * system per model: a single wavenumber 0 of weight 1). Geometry, element
 * templates, the sparse pattern, its assembly routing and the block elimination schedule of
 * the direct solver are host arrays copied into the plan once; the plan owns that device
 * memory. Every other array crossing this boundary is a caller-owned DEVICE pointer (for
 * example a PyTorch CUDA tensor); work is enqueued on the caller's stream and the entry points
 * return without synchronizing unless stated. Entry points are not thread-safe per plan, and
 * the work of one plan must be ordered on the GPU (one stream, or streams the caller
 * synchronizes): factorizations share the plan's solver workspaces (split-depth partial tiles,
 * diagonal-tile inverses) whatever their slot.
 *
 * Layouts (row-major, C order):
 *   sigma      [S][model_cells]                       float32 (conductivity, S models)
 *   fields     [S][W][dofs][E]                        float32 (total potentials; the dof axis
 *                                                      is the plan's solver order, see
 *                                                      adt_plan_dof_order)
 *   normal, reciprocal   [S][D]                       float64 (transfer resistances)
 *   jacobian   [rows][columns]                        float32
 *
 * ABMN rows use electrode slots; slot E is the remote electrode, whose potential is zero.
 *
 * Status codes map onto the reference's Python exceptions: INVALID_ARG -> ValueError,
 * NONFINITE -> FloatingPointError, SOLVER_FAIL -> FloatingPointError (non-positive pivot),
 * OOM -> MemoryError, CUDA_ERROR / TIMEOUT -> RuntimeError.
 */
#ifndef ADTLERT_B200_H
#define ADTLERT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  ADT_OK = 0,
  ADT_INVALID_ARG = 1,
  ADT_NONFINITE = 2,
  ADT_SOLVER_FAIL = 3,
  ADT_OOM = 4,
  ADT_TIMEOUT = 5,
  ADT_CUDA_ERROR = 6
} adt_status;

typedef struct adt_plan adt_plan;
typedef void* adt_stream; /* a cudaStream_t; NULL is the legacy default stream */

/* Discretization of one operator (host arrays, copied by adt_plan_create).
 * Mirrors adtlert/forward/discretization.py:128-156 (Discretization) plus the quadrature of
 * adtlert/forward/integration.py:32-49 and the survey slots of adtlert/survey/core.py:77-85;
 * for 3D, the tetrahedral templates, Robin faces and Dirichlet dofs of
 * adtlert/forward/ert3d.py:224-351. */
typedef struct {
  int32_t dof_count;              /* N */
  int32_t dim;                    /* coordinate dimension of dof_coordinates (2 or 3) */
  const double* dof_coordinates;  /* N*dim, used to choose the elimination order */
  int32_t cell_count;             /* C: discretization cells */
  int32_t local_dofs;             /* K: dofs per cell (3 P1 triangle, 4 Q1 quad, ...) */
  const int32_t* cell_dofs;       /* C*K */
  const double* stiffness;        /* C*K*K unit-conductivity stiffness templates */
  const double* mass;             /* C*K*K unit mass templates */
  const int32_t* parent_cells;    /* C: model cell of each discretization cell, NULL = identity */
  int32_t model_cell_count;       /* number of model (conductivity) cells */
  int32_t boundary_count;         /* Nb Robin boundary elements */
  int32_t boundary_local;         /* dofs per boundary element */
  const int32_t* boundary_dofs;   /* Nb*boundary_local */
  const int32_t* boundary_cells;  /* Nb: owning discretization cell */
  const double* boundary_mass;    /* Nb*boundary_local^2 unit boundary-mass templates */
  const double* boundary_coefficients; /* W*Nb mixed-boundary geometry per wavenumber */
  int32_t wavenumber_count;       /* W */
  const double* wavenumbers;      /* W */
  const double* weights;          /* W inverse cosine-transform weights */
  int32_t electrode_count;        /* E: source electrodes == field rows per wavenumber */
  int32_t receiver_width;         /* nonzeros per electrode interpolation row */
  const int32_t* receiver_dofs;   /* E*receiver_width (-1 pads) */
  const double* receiver_weights; /* E*receiver_width */
  int32_t measurement_count;      /* D */
  const int32_t* abmn;            /* D*4 electrode slots, E = remote */
  const int32_t* source_cell_ptr; /* E+1: model cells averaged for each source resistivity */
  const int32_t* source_cells;    /* source_cell_ptr[E] model cell ids */
  int32_t fixed_count;            /* Dirichlet dofs: identity rows, no couplings, zero fields */
  const int32_t* fixed_dofs;      /* fixed_count dof ids (NULL when fixed_count is 0) */
} adt_problem;

/* Summary of a plan (sizes, elimination schedule). */
typedef struct {
  int32_t dof_count, nnz, block_count, max_block, levels;
  int32_t features;                  /* Gram features per cell and wavenumber */
  int64_t factor_doubles_per_system; /* dense factor storage of one system */
  int64_t contributions;             /* routed assembly contributions */
} adt_plan_info;

/* Replaces: ERTForward2p5D.from_mesh_survey geometry set-up (adtlert/forward/ert2p5d.py:133-216),
 * sparse_pattern (adtlert/forward/discretization.py:100-125), the GroupSum routing of
 * _assemble (ert2p5d.py:275-314) and the cuDSS analysis/plan (adtlert/forward/cudss.py:24-45). */
adt_status adt_plan_create(const adt_problem* problem, adt_plan** plan);
adt_status adt_plan_destroy(adt_plan* plan);
adt_status adt_plan_get_info(const adt_plan* plan, adt_plan_info* info);
/* Copies the solver dof order (N int32: position -> original dof) to host memory. */
adt_status adt_plan_dof_order(const adt_plan* plan, int32_t* order);
/* Copies the last error message of the plan (or of a failed create, when plan is NULL). */
adt_status adt_last_error(const adt_plan* plan, char* buffer, size_t size);

/* Unit-resistivity primary field, host array [W][E][N] in original dof order; computes the
 * conductivity-independent right-hand side A(1) u_p on the device.
 * Replaces: _unit_primary / _reference_rhs (adtlert/forward/ert2p5d.py:418-478). */
adt_status adt_set_primary(adt_plan* plan, const double* primary, adt_stream stream);

/* Conductivity-independent right-hand sides of fields solved without a primary-field
 * correction (the 3D operator): rhs = A(1) unit_primary + direct, zeroed on the fixed dofs;
 * both host arrays are [W][E][N] in original dof order and either may be NULL. Afterwards
 * adt_solve_fields solves A(sigma) u = rhs and writes u (sigma only selects the factorization).
 * Replaces: _build_unit_operator, _build_source_rhs and _build_receiver_rhs
 * (adtlert/forward/ert3d.py:353-413). */
adt_status adt_set_static_rhs(adt_plan* plan, const double* unit_primary, const double* direct,
                              adt_stream stream);

/* Assembles A_w(sigma_s) for S models (S*W systems) into factor slot `slot` and factorizes
 * them. Replaces: _assemble (ert2p5d.py:275-314) + BatchedSolver.solve factorization
 * (adtlert/forward/cudss.py:63-122). */
adt_status adt_factorize(adt_plan* plan, int32_t slot, const float* sigma, int32_t models,
                         adt_stream stream);

/* adt_factorize plus the field right-hand sides of the same models: forms
 * A(1) u_p - rho A(sigma) u_p and forward-reduces it during the factorization (each level's
 * forward updates run in that level's Schur-update launch), keeping it in the slot. The next
 * adt_solve_fields on this slot with the same sigma pointer and model count then runs only the
 * backward substitution and the total field; any other call factorizing into the slot drops the
 * reduced right-hand sides. Plans where this does not apply (3D static right-hand sides, the
 * tiled solver, more electrodes than the solver's block width) factorize as adt_factorize.
 * Replaces: the factorization + solve phases of _solve_fields (adtlert/forward/ert2p5d.py:532-553,
 * cudss.py:63-122) when called back to back. */
adt_status adt_factorize_fields(adt_plan* plan, int32_t slot, const float* sigma, int32_t models,
                                adt_stream stream);

/* Secondary-field solve with the slot's factorization of the same models, writing total
 * fields u = u_s + rho_src u_p. Replaces: _solve_fields (ert2p5d.py:532-553). */
adt_status adt_solve_fields(adt_plan* plan, int32_t slot, const float* sigma, int32_t models,
                            float* fields, adt_stream stream);

/* Assembles and factorizes the operators of wavenumbers [w_begin, w_begin + w_count) of one
 * model into `slot` (system i is wavenumber w_begin + i), so that large discretizations can be
 * factorized a few wavenumbers at a time. Replaces the per-batch assembly and factorization of
 * _unit_potentials (adtlert/forward/ert2p5d.py:404-416). */
adt_status adt_factorize_wavenumbers(adt_plan* plan, int32_t slot, const float* sigma,
                                     int32_t w_begin, int32_t w_count, adt_stream stream);

/* Solves A_s X = B in place with the factorization held in `slot` for its first `systems`
 * systems (system s = model * W + w): rhs [systems][N][nrhs] float64 in solver dof order.
 * Replaces the solve phase of BatchedSolver.solve (adtlert/forward/cudss.py:63-122), e.g. for
 * the unit potentials of a terrain operator's auxiliary discretizations
 * (adtlert/forward/ert2p5d.py:404-416). */
adt_status adt_solve(adt_plan* plan, int32_t slot, int32_t systems, int32_t nrhs, double* rhs,
                     adt_stream stream);

/* One call for the forward of S models: adt_factorize_fields + adt_solve_fields into `fields`
 * [S][W][N][E] + adt_measure (normal and reciprocal resistances [S][D], float64). The slot keeps
 * the factorization, so adt_vjp / adt_jvp / adt_adjoint_jacobian may follow. Replaces: the
 * field and measurement phases of solve() / resistance() (adtlert/forward/ert2p5d.py:532-589). */
adt_status adt_forward(adt_plan* plan, int32_t slot, const float* sigma, int32_t models, float* fields,
                       double* normal, double* reciprocal, adt_stream stream);

/* One call for the normal Jacobian of one model: adt_factorize_fields + adt_solve_fields into
 * `fields` [W][N][E] + adt_normal_jacobian of rows [row_begin, row_begin+row_count) into
 * jacobian [row_count][C]. Replaces: jacobian(conductivity) with the default normal sensitivity
 * (adtlert/forward/ert2p5d.py:971-1010) up to the host copy. */
adt_status adt_jacobian(adt_plan* plan, int32_t slot, const float* sigma, float* fields, int32_t row_begin,
                        int32_t row_count, float* jacobian, adt_stream stream);

/* Normal and reciprocal transfer resistances of S models (and, if not NULL, the E*E electrode
 * potentials per model). Replaces: _integrate + _normal_reciprocal (ert2p5d.py:560-589). */
adt_status adt_measure(adt_plan* plan, const float* fields, int32_t models, double* normal,
                       double* reciprocal, double* potentials, adt_stream stream);

/* Integrated potentials [E][N] in original dof order of one model (ForwardResponse field). */
adt_status adt_integrated_potentials(adt_plan* plan, const float* fields, float* integrated,
                                     adt_stream stream);

/* Normal-quadrupole sensitivity rows [row_begin, row_begin+row_count) of one model,
 * out[d][c] = -sum_w w_w (u_M - u_N)^T (K_c + k_w^2 M_c) (u_A - u_B) over discretization cells.
 * Replaces: normal_sensitivity (adtlert/forward/kernels.py:132-268) as called by
 * _normal_jacobian (ert2p5d.py:984-1010). Single-wavenumber (3D) operators compute every entry
 * directly from per-cell features (no electrode Gram); otherwise the electrode Grams run on the
 * tensor cores (tcgen05, TF32 with a hi/lo split) for up to 64 field columns, else on FP32 FMA.
 * The environment variable ADTLERT_B200_JACOBIAN, read at plan creation, overrides the choice:
 * "fma" takes the FP32 Gram kernel everywhere, "tc" the tensor cores wherever they apply. A
 * tensor-core launch whose MMAs do not complete within its bounded wait writes NaN into its
 * cells' columns, and the plan's next adt_normal_jacobian call returns ADT_TIMEOUT. */
adt_status adt_normal_jacobian(adt_plan* plan, const float* fields, int32_t row_begin,
                               int32_t row_count, float* jacobian, adt_stream stream);

/* Failure detection of the tensor-core Jacobian: with polls > 0 each block waits for its MMA
 * chain with at most `polls` non-blocking polls before it gives up (NaN columns, ADT_TIMEOUT on
 * the plan's next adt_normal_jacobian), while the wait that guards the release of its tensor
 * memory keeps the full limit; polls = 0 restores the default wait. Synchronizes the device and
 * clears the plan's timeout flag. No counterpart in the reference (its kernel has no wait). */
adt_status adt_set_jacobian_wait_limit(adt_plan* plan, uint32_t polls);

/* The whole normal Jacobian of one model (the adt_normal_jacobian product for rows 0 .. D-1)
 * into host_jacobian [D][C] float32, which must be page-locked (cudaHostAlloc / pinned), through
 * device_jacobian (same layout, on the device). J is computed on `stream` in `chunks` column
 * ranges (at most C/64), and each finished range is copied to the host on a stream of the plan
 * while the next range is computed; `stream` then waits for the last copy, so synchronizing
 * `stream` makes host_jacobian complete. Replaces: the device Jacobian and its copy to the host
 * in jacobian() (adtlert/forward/ert2p5d.py:984-1010 and its torch .cpu()). */
adt_status adt_normal_jacobian_to_host(adt_plan* plan, const float* fields, float* device_jacobian,
                                       float* host_jacobian, int32_t chunks, adt_stream stream);

/* Sums the `in_columns` columns of values [rows][in_columns] into `columns` outputs:
 * column_ptr[columns+1] / column_cells[] list the input columns of every output column in
 * summation order (host arrays, cached in the plan under `key`; inputs listed nowhere are
 * dropped). Replaces CellAggregation.columns (adtlert/forward/kernels.py:88-113). */
adt_status adt_aggregate_columns(adt_plan* plan, int32_t key, int32_t columns,
                                 const int32_t* column_ptr, const int32_t* column_cells,
                                 const float* values, int32_t rows, int32_t in_columns,
                                 float* out, adt_stream stream);

/* Exact VJP of the reciprocity-averaged resistance for S models factorized in `slot`:
 * cotangents [S][D] (float64) -> gradients [S][model_cells] (float32). With `robin` the mixed
 * boundary derivative is included. Replaces: vjp_series (ert2p5d.py:835-871) with
 * _pair_cotangent/_adjoint_rhs/_cell_gradient (591-639, 765-825). */
adt_status adt_vjp(adt_plan* plan, int32_t slot, const float* fields, const double* normal,
                   const double* reciprocal, const double* cotangents, int32_t models,
                   float* gradient, adt_stream stream);

/* Exact-derivative Jacobian rows of one model factorized in `slot` (model 0 of the slot),
 * rows [row_begin, row_begin+row_count), each the VJP of a unit cotangent; with
 * `normal_only` the cotangent acts on the normal reading only (the normal-quadrupole
 * convention) and `robin` adds the boundary term. Replaces _adjoint_jacobian
 * (ert2p5d.py:1012-1050). */
adt_status adt_adjoint_jacobian(adt_plan* plan, int32_t slot, const float* fields,
                                const double* normal, const double* reciprocal,
                                int32_t row_begin, int32_t row_count, int32_t robin,
                                int32_t normal_only, float* jacobian, adt_stream stream);

/* JVP of one model factorized in `slot`: direction [model_cells] -> [D] resistance tangent.
 * Replaces: jvp (ert2p5d.py:873-890). */
adt_status adt_jvp(adt_plan* plan, int32_t slot, const float* fields, const double* normal,
                   const double* reciprocal, const float* direction, double* out,
                   adt_stream stream);

/* Normal-convention products without a solve. normal_vjp: cotangent [D] -> [model_cells]
 * (before parameter aggregation); normal_jvp: direction [model_cells] -> [D]. With `robin`
 * the operator derivative includes the mixed-boundary terms: for a 3D operator, whose
 * receiver fields are field columns of their own, these are the exact vjp and jvp.
 * Replaces: normal_vjp / normal_jvp (ert2p5d.py:892-943); vjp, jvp, normal_vjp and
 * normal_jvp of ERTForward3D (adtlert/forward/ert3d.py:736-865). */
adt_status adt_normal_vjp(adt_plan* plan, const float* fields, const double* cotangent,
                          int32_t robin, float* gradient, adt_stream stream);
adt_status adt_normal_jvp(adt_plan* plan, const float* fields, const float* direction,
                          int32_t robin, double* out, adt_stream stream);

/* Adds the mixed-boundary derivative to Jacobian rows [row_begin, row_begin+row_count) of one
 * model written by adt_normal_jacobian (same layout, discretization-cell columns):
 * J[d][c] += -sum_w w_w sum_{b owned by c} alpha_wb (u_M - u_N)_b^T Mb_b (u_A - u_B)_b.
 * Replaces: the Robin templates of ERTForward3D.jacobian(include_robin_boundary_derivative=True)
 * (adtlert/forward/ert3d.py:867-927). */
adt_status adt_boundary_jacobian(adt_plan* plan, const float* fields, int32_t row_begin,
                                 int32_t row_count, float* jacobian, adt_stream stream);

/* adt_measure without any device allocation: no counterpart in the reference. For callers that
 * may not call cudaMalloc while running (GPU memory fully reserved by another allocator, or
 * loops that must not block on the driver's allocator); adt_measure grows a plan-owned table
 * with cudaMalloc instead. The potential table lives in a fixed array compiled into the library:
 * 65,536 doubles (512 KiB) per device, held until exit, so models * (E+1)^2 must not exceed
 * 65,536 (larger requests return ADT_INVALID_ARG). All calls share that array: calls that overlap
 * on the GPU race and must be ordered by the caller. The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress), so make it before any stream capture; the address
 * is cached, so a device reset after that first call is not supported. */
adt_status adt_measure_static(adt_plan* plan, const float* fields, int32_t models, double* normal,
                              double* reciprocal, adt_stream stream);

/* values[r][c] *= row_scale[r] * column_scale[c] for a rows x columns float32 device array
 * (row_scale, column_scale: float64 device arrays; either may be NULL for ones). Used for the
 * log-space Jacobian d log(rhoa) / d log(rho) = k J_R (-sigma) / rhoa without moving J off the
 * device. Replaces the chain rule of log_response_and_jacobian
 * (adtlert/forward/modeling.py:137-162). */
adt_status adt_scale_rows_columns(float* values, int32_t rows, int32_t columns,
                                  const double* row_scale, const double* column_scale,
                                  adt_stream stream);

/* Content fingerprints of `models` consecutive models of bytes_per_model bytes each (a multiple
 * of 4, the data 4-byte aligned): two uint64 per model, the keys of the operators' field caches
 * (two 64-bit sums of a mixed word stream; identical for identical bytes, different models
 * collide with probability about 2^-128). adt_fingerprint reads device memory and writes the
 * device array `fingerprints` [models][2] on `stream`; adt_fingerprint_host computes the same
 * bits from host memory on the calling thread. Replaces the blake2b digest of FieldCache.key
 * (adtlert/forward/field_cache.py:54-59), which first copies a device model to the host. */
adt_status adt_fingerprint(adt_plan* plan, const void* models_data, int64_t bytes_per_model, int32_t models,
                           uint64_t* fingerprints, adt_stream stream);
adt_status adt_fingerprint_host(const void* models_data, int64_t bytes_per_model, int32_t models,
                                uint64_t* fingerprints);

/* Gauss-Newton step of a time-lapse window of `steps` models (rows x columns log Jacobians each):
 * solves min ||A x - b|| by `iterations` CGLS iterations on the device (stopping early, with the
 * rest of the launched iterations doing nothing, once gamma / gamma_0 < tolerance), where
 *   A = [ W J_t (per model) ; sqrt(spatial) R (per model) ; sqrt(temporal) D_t ],
 *   b = [ data_rhs ; -sqrt(spatial) R m ; -sqrt(temporal) D_t m ],
 * W = diag(data_weights), R the first-order neighbour differences given as symmetric neighbour
 * lists (neighbour_ptr[columns+1], neighbour_cells, neighbour_weights = squared row weights; each
 * neighbouring pair listed from both cells), D_t the first difference between consecutive models.
 * Device arrays: jacobian [steps][rows][columns] float32 (16-byte aligned; columns a multiple of
 * 4, at most 16384), data_weights and data_rhs [steps][rows] float64, models and step
 * [steps][columns] float64. The caller provides `workspace` (256-byte aligned, the size that
 * adt_gn_workspace_bytes gives for the same sizes and `multiprocessors`); nothing is allocated.
 * Replaces: the gauss_newton_cgls linearized step with gpu_cgls of
 * adtlert/inversion/core.py:204-216 (_data_system, objective.py:56-80; RegularizationTerms.blocks,
 * terms.py:75-186; _gpu_cgls, optimizers.py:314-360), without forming the stacked sparse matrix. */
adt_status adt_gn_workspace_bytes(int32_t steps, int32_t rows, int32_t columns, int32_t multiprocessors,
                                  size_t* bytes);
adt_status adt_gn_step(adt_plan* plan, const float* jacobian, int32_t steps, int32_t rows, int32_t columns,
                       const double* data_weights, const double* data_rhs, const double* models,
                       const int32_t* neighbour_ptr, const int32_t* neighbour_cells,
                       const double* neighbour_weights, double spatial, double temporal, int32_t iterations,
                       double tolerance, double* step, void* workspace, size_t workspace_bytes,
                       int32_t multiprocessors, adt_stream stream);
/* out = (spatial R^T R + temporal D_t^T D_t) models for [steps][columns] float64 device arrays
 * (the regularization part of A^T A; the line search of the Gauss-Newton iteration evaluates its
 * quadratic from it). Replaces the regularization rows of _line_search_tau
 * (adtlert/inversion/objective.py:168-192). */
adt_status adt_gn_regularize(adt_plan* plan, int32_t steps, int32_t columns, const int32_t* neighbour_ptr,
                             const int32_t* neighbour_cells, const double* neighbour_weights, double spatial,
                             double temporal, const double* models, double* out, adt_stream stream);

/* Kernels of the learned apparent-resistivity surrogate (BF16 operands, FP32 accumulation). No
 * counterpart in the reference, whose inversion evaluates every line-search and window candidate
 * with the FEM (adtlert/inversion/core.py:224-257, objective.py:168-192); the surrogate screens
 * those candidates and the FEM still judges every accepted model. Device pointers; BF16 arrays
 * are passed as void*.
 * adt_mlp_gemm: partial[s][m][n] = sum over split s's K range of a[m][k] b[n][k] (a: m x k, b:
 *   n x k, row-major BF16, 16-byte aligned; m, n multiples of 128, k of 64), on tcgen05 tensor
 *   cores; `splits` must be the value adt_mlp_gemm_splits returns for these sizes (it fills the
 *   multiprocessors and gives every split at least one 64-wide K chunk); partial holds at least
 *   splits*m*n floats; *error is set to 1 when a bounded wait inside the kernel ran out.
 * adt_mlp_epilogue: sums the splits in order and applies mode 0 (z = sum + bias -> z_out; y =
 *   gelu(z) -> row_out and, if not NULL, col_out[n][m]), 1 (f32_out = sum + bias), 2 (g = sum *
 *   gelu'(z_in) -> row_out, col_out) or 3 (f32_out = sum); gelu is the tanh form.
 * adt_mlp_loss: g = 2 (pred - target) / (m n_valid) on columns < n_valid (0 beyond) -> g_row,
 *   g_col (transposed); sums[(m / 32) (n / 32)] receives per-tile squared-error sums.
 * adt_mlp_bias_grad: db[n] = sum_m g_col[n][m]. adt_mlp_adam: one Adam step on FP32 parameters
 *   (correction1 = 1 / (1 - beta1^t), correction2 = 1 / (1 - beta2^t)), writing the BF16 copy if
 *   params_bf16 is not NULL. adt_mlp_transpose: out[c][r] = in[r][c] (BF16, sides multiples of
 *   32). adt_mlp_to_bf16: FP32 -> BF16 (round to nearest even). */
int32_t adt_mlp_gemm_splits(int32_t m, int32_t n, int32_t k, int32_t multiprocessors);
adt_status adt_mlp_gemm(const void* a, const void* b, int32_t m, int32_t n, int32_t k, int32_t splits,
                        float* partial, size_t partial_floats, int32_t* error, adt_stream stream);
adt_status adt_mlp_epilogue(int32_t mode, const float* partial, int32_t splits, int32_t m, int32_t n,
                            const float* bias, const void* z_in, void* z_out, void* row_out, void* col_out,
                            float* f32_out, adt_stream stream);
adt_status adt_mlp_loss(const float* pred, const float* target, int32_t m, int32_t n, int32_t n_valid,
                        void* g_row, void* g_col, float* sums, adt_stream stream);
adt_status adt_mlp_bias_grad(const void* g_col, int32_t n, int32_t m, float* db, adt_stream stream);
adt_status adt_mlp_adam(float* params, const float* grads, float* first, float* second, int64_t count, float lr,
                        float beta1, float beta2, float eps, float correction1, float correction2,
                        void* params_bf16, adt_stream stream);
adt_status adt_mlp_transpose(const void* in, int32_t rows, int32_t cols, void* out, adt_stream stream);
adt_status adt_mlp_to_bf16(const float* in, int64_t count, void* out, adt_stream stream);

/* Number of kernels this library has launched since the plan was created. */
int64_t adt_kernel_launches(const adt_plan* plan);

/* Launch shapes of one plan, chosen by measurement. No counterpart in the reference (cuDSS and
 * its NVRTC kernel choose their own launch shapes). The settings change which blocks compute
 * what; a narrower strip or a different split depth can also split a block's float64 reductions
 * differently, so results of two settings agree to rounding, and each setting is bitwise
 * repeatable.
 *   strip_fill       substitution launches (forward, backward, tiled strips) narrow their
 *                    right-hand-side strips while blocks x strips < strip_fill x SMs: 1, 2, 4 or 8
 *   split_fill       tiled panel launches split their reduction depth while
 *                    tiles x systems x splits x 2 <= split_fill x SMs: 0 (never), 1 or 2
 *   jacobian_kernel  ADT_JACOBIAN_* below; a kernel that does not apply to the plan's shapes
 *                    falls through to the next one in that order
 *   fields_ms, jacobian_ms  (adt_autotune only) the fastest time of the chosen setting */
enum {
  ADT_JACOBIAN_DIRECT = 0,      /* direct form, one wavenumber (3D) */
  ADT_JACOBIAN_TC_PIPELINED = 1,/* tensor-core Gram with producer / MMA / epilogue warp roles */
  ADT_JACOBIAN_TC = 2,          /* tensor-core Gram, one block chain per cell group */
  ADT_JACOBIAN_FMA = 3          /* FP32 CUDA-core Gram */
};
typedef struct {
  int32_t strip_fill;
  int32_t split_fill;
  int32_t jacobian_kernel;
  float fields_ms;
  float jacobian_ms;
} adt_tuning;

/* Autotuner of the plan's launch shapes: times adt_factorize_fields + adt_solve_fields of
 * `models` models `sigma` in slot `slot` for every strip_fill (and, on tiled plans, split_fill),
 * then adt_normal_jacobian of all rows for every Jacobian kernel that applies, each candidate
 * once untimed and `repeats` (1..32) times timed with CUDA events on `stream`; keeps the fastest
 * of each and writes the choice to `out` (may be NULL). On return `fields` ([models][W][dofs][E])
 * and `jacobian` ([D][cells of the discretization], of the first model; NULL skips the Jacobian)
 * hold the results of the chosen settings. Synchronizes the stream; allocates what the timed entry points
 * allocate on first use. Beside the reference's fixed launch geometry (kernels.py:222-268). */
adt_status adt_autotune(adt_plan* plan, int32_t slot, const float* sigma, int32_t models, float* fields,
                        float* jacobian, int32_t repeats, adt_tuning* out, adt_stream stream);
/* CUDA graph of one fresh-model Jacobian: adt_factorize_fields, adt_solve_fields (one model),
 * adt_measure and adt_normal_jacobian of all rows (skipped when `jacobian` is NULL), captured
 * once from a private stream after one uncaptured run on `stream` (which allocates what the
 * chain grows on first use and synchronizes), then replayed by adt_graph_launch on any stream.
 * Every launch reads `sigma` ([model_cells]) and writes `fields`, `normal`, `reciprocal` and
 * `jacobian` at the addresses given here; the caller refreshes `sigma` before a launch. A launch
 * is refused (ADT_INVALID_ARG) once the plan has reallocated a workspace the graph holds (for
 * example a later call on the same slot with more models): create the graph again. Destroy
 * graphs before their plan, after their last launch has completed. Replaces the per-call launch
 * sequence of jacobian() (adtlert/forward/ert2p5d.py:945-1010) for repeated fresh models. */
typedef struct adt_graph adt_graph;
adt_status adt_jacobian_graph_create(adt_plan* plan, int32_t slot, const float* sigma, float* fields,
                                     double* normal, double* reciprocal, float* jacobian, adt_stream stream,
                                     adt_graph** graph);
adt_status adt_graph_launch(adt_graph* graph, adt_stream stream);
/* Library kernels one launch of the graph runs. */
int64_t adt_graph_kernels(const adt_graph* graph);
adt_status adt_graph_destroy(adt_graph* graph);

/* The plan's current launch shapes (timing fields zero). */
adt_status adt_get_tuning(const adt_plan* plan, adt_tuning* out);
/* Apply saved launch shapes (for example an earlier adt_autotune result on the same device);
 * out-of-range values are rejected. */
adt_status adt_set_tuning(adt_plan* plan, const adt_tuning* tuning);

#ifdef __cplusplus
}
#endif

#endif /* ADTLERT_B200_H */
