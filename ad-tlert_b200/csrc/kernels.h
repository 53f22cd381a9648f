// Kernel argument blocks and declarations (device side of adtlert_b200).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace adt {

struct AssembleArgs {
  const float* sigma;  // [models][Cm]
  const int* parent;   // [C] or null
  const int* contrib_ptr;
  const int* contrib;
  const double* stiffness;
  const double* mass;
  const double* bmass;
  const double* bcoef;
  const int* bcells;
  const double* k2;
  double* values;  // [systems][nnz]
  int systems, nnz, W, C, Cm, K2, BL2, Nb, robin;
  int identity;    // add the unit diagonal of fixed dofs (system matrices, not derivatives)
  int w0;          // wavenumber of system 0 (systems cover wavenumbers w0 .. w0 + W - 1)
  // optional: source resistivities rho[s][e] of the models, computed by the same launch
  double* rho = nullptr;
  const int* src_ptr = nullptr;
  const int* src_cells = nullptr;
  int models = 0, E = 0;
};

struct SpmmArgs {
  const double* values;  // [systems or W][nnz]
  const int* csr_ptr;
  const int* csr_col;
  const void* x;         // [systems or W][N][E], float64 if x_double else float32
  int x_double;
  const double* rho;     // [models][E] or null
  const double* base;    // [W][N][E] or null
  double* out;           // [systems][N][E]
  double scale;
  int systems, N, E, W, nnz, x_per_system, values_per_wavenumber;
};

struct MeasureArgs {
  const void* fields;  // [models][W][N][E], float64 if f_double else float32
  int f_double;
  const double* weights;
  const int* rcv_dofs;
  const double* rcv_w;
  const int* abmn;
  double* normal;
  double* reciprocal;
  double* potentials;  // [models][E][E] or null
  const double* base_normal;  // combine mode: the model's normal / reciprocal readings
  const double* base_recip;
  int W, N, E, RW, D, combine;
};

struct PairArgs {
  const int* pair_ptr;   // [(E+1)^2 + 1]
  const int* pair_list;  // d * 4 + kind
  const double* cot;     // [count][D] (unless unit)
  const double* normal;  // [models][D]
  const double* recip;
  double* pairs;         // [count][E][E]
  int count, E, D, normal_only, unit, row_begin, model_of_count;
};

struct AdjointRhsArgs {
  const double* pairs;  // [models*q_per_model][E][E]
  const int* rdof_ptr;  // receiver dof routing
  const int* rdof_rcv;
  const double* rdof_w;
  const int* rdof_dof;
  const double* weights;
  double* rhs;          // [systems][N][q_per_model*E]
  int systems, rdofs, q_per_model, E, W, N;
};

struct JacobianArgs {
  const float* fields;    // [W][N][E] one model
  const float* features;  // [C][R][K]
  const int* cell_dofs;   // [C][K]
  const float* fscale;    // [W][R] per-wavenumber feature scales
  const int* abmn;        // [D][4]
  float* out;             // row d, cell c at out[d * ldo + c]
  int W, N, E, C, K, R, row_begin, rows, cells_per_block;
  int c_begin, c_end;     // cells computed: [c_begin, c_end)
  int64_t ldo;            // row stride of out
  unsigned first_wait_polls = 0;  // tensor-core kernel: 0 = the default bounded wait for each MMA
                                  // chain; n > 0 = give up after n non-blocking polls (tests)
};

struct CellGradientArgs {
  const void* x;          // first field set [systems][N][ncol] (lambda or current)
  const void* y;          // second field set [models][W][N][E] (phi)
  int x_double, y_double;
  const double* x_scale;  // [W] or null: multiplies x (weights)
  const double* y_scale;  // [W] or null
  const double* stiffness, *mass, *bmass, *bcoef;
  const double* k2;
  const int* cell_dofs;
  const int* cell_bptr;
  const int* cell_blist;
  const int* bdofs;
  double* out;            // [count][C] (before parent aggregation)
  int models, W, N, E, C, K, BL, Nb, robin, x_cols, q_per_model;
};

struct BoundaryJacobianArgs {
  const float* fields;     // [W][N][E] one model
  const double* weights;   // [W]
  const double* bcoef;     // [W][Nb]
  const double* bmass;     // [Nb][BL][BL]
  const int* bdofs;        // [Nb][BL] solver order
  const int* cell_bptr;    // [C+1]
  const int* cell_blist;
  const int* owners;       // cells owning boundary elements
  const int* abmn;         // [D][4]
  float* out;              // [rows][C]
  int W, N, E, C, Nb, BL, owner_count, row_begin, rows;
};

__global__ void assemble_kernel(AssembleArgs a);
__global__ void source_rho_kernel(const float* sigma, int Cm, int E, int models, const int* ptr,
                                  const int* cells, double* rho);
__global__ void spmm_kernel(SpmmArgs a);
__global__ void total_kernel(const double* x, const double* primary, const double* rho, int W,
                             int N, int E, int systems, float* fields);
__global__ void potentials_kernel(MeasureArgs a, int models, double* pot);
__global__ void transfers_kernel(MeasureArgs a, int models, const double* pot);
__global__ void pair_kernel(PairArgs a);
__global__ void adjoint_rhs_kernel(AdjointRhsArgs a);
__global__ void gram_partial_kernel(const float* phi, const double* y, const double* weights,
                                    int W, int N, int E, int chunk, int sub, double* partial);
__global__ void gram_reduce_kernel(const double* partial, int blocks, int E, double* gram);
__global__ void gram_gather_kernel(const double* gram, int E, int D, const int* abmn, double* out);
__global__ void integrated_kernel(const float* fields, const double* weights, const int* iperm,
                                  int W, int N, int E, float* integrated);
constexpr int kMixTileRows = 64;  // field rows per block of mix_tiled_kernel
__global__ void mix_tiled_kernel(const double* pairs, const float* phi, int64_t rows, int E, double* current);
size_t mix_tiled_smem(int E);
__global__ void mix_kernel(const double* pairs, const float* phi, int W, int N, int E,
                           double* current);
cudaError_t launch_jacobian(const JacobianArgs& a, size_t smem, cudaStream_t s);
int jacobian_direct_cells(int R, int E, int K);
cudaError_t launch_jacobian_direct(const JacobianArgs& a, const int2* rows, cudaStream_t s);
bool jacobian_tc_supported(int E, int W, int R, int K, int rows);
cudaError_t launch_jacobian_tc(const JacobianArgs& a, int* error, int sms, cudaStream_t s);
// Pipelined tensor-core kernel (warp roles): the Gram batch (pairs per row store) it would use
// for these sizes, 0 when it does not apply.
int jacobian_tcpipe_batch(int E, int W, int R, int K, int rows);
cudaError_t launch_jacobian_tcpipe(const JacobianArgs& a, int batch, int* error, int sms, cudaStream_t s);
cudaError_t launch_cell_gradient(const CellGradientArgs& a, int blocks, cudaStream_t s);
__global__ void boundary_jacobian_kernel(BoundaryJacobianArgs a);
__global__ void add_kernel(double* y, const double* x, int64_t count);
__global__ void scale_rows_columns_kernel(float* values, int rows, int columns, const double* row_scale,
                                          const double* column_scale);
__global__ void zero_rows_kernel(double* x, const int* rows, int count, int W, int N, int E);
__global__ void aggregate_kernel(const double* in, int rows, int C, int columns, const int* ptr,
                                 const int* cells, float* out, int64_t in_stride);
__global__ void aggregate_float_kernel(const float* in, int rows, int C, int columns,
                                       const int* ptr, const int* cells, float* out);

}  // namespace adt
