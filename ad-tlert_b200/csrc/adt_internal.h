// Internal declarations shared by the adtlert_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "adtlert_b200.h"
#include "plan_host.h"

namespace adt {

// Threads of the solver kernels.
constexpr int kSolverThreads = 256;

// The library's kernels run as one dependent chain per stream. Each kernel's first statement
// waits for the grid before it in the stream (griddepcontrol.wait: that grid has completed and
// its memory is visible) and then lets the next grid be scheduled; every launch allows
// programmatic stream serialization, so a grid's launch overlaps the drain of the one before.
// A kernel launched without the attribute, or after a foreign kernel, waits as usual.
__device__ __forceinline__ void chain_wait() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename... P, typename... A>
inline cudaError_t launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  A&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

struct Slot {
  int systems = 0;          // systems currently factorized (models * W)
  size_t capacity = 0;      // systems allocated
  double* values = nullptr; // [systems][nnz]
  double* factors = nullptr;// [systems][factor_stride]
  // field right-hand sides forward-reduced by adt_factorize_fields, consumed by the next
  // adt_solve_fields of the same sigma and model count
  double* rhs = nullptr;    // [systems][N][E]
  double* rho = nullptr;    // [models][E] source resistivities
  size_t rhs_capacity = 0;  // systems allocated for rhs
  bool rhs_ready = false;
  const float* rhs_sigma = nullptr;
  int rhs_models = 0;
};

struct Aggregation {
  int key = -1, columns = 0;
  int* ptr = nullptr;
  int* cells = nullptr;
};

}  // namespace adt

struct adt_plan {
  // sizes
  int N = 0, dim = 2, C = 0, K = 0, Cm = 0, Nb = 0, BL = 0, W = 0, E = 0, D = 0, RW = 0;
  int nnz = 0, nb = 0, max_m = 0, levels = 0;
  int max_width = 0;  // widest augmented row [D_j | A_jp | A_qj^T] of the level blocks
  int64_t contributions = 0;
  int64_t factor_stride = 0;
  int RS = 0;  // stiffness features per wavenumber
  int R = 0;   // all features per wavenumber (stiffness + mass)
  std::vector<int> perm;  // position -> original dof
  std::vector<int> iperm; // original dof -> position
  std::vector<int> level_begin;  // task ranges per level (root is the last level)
  // device geometry
  int* csr_ptr = nullptr;
  int* csr_col = nullptr;
  int* csr_row = nullptr;
  int* contrib_ptr = nullptr;
  int* contrib = nullptr;
  double* stiffness = nullptr;  // [C][K*K]
  double* mass = nullptr;       // [C][K*K]
  double* bmass = nullptr;      // [Nb][BL*BL]
  double* bcoef = nullptr;      // [W][Nb]
  int* cell_dofs = nullptr;     // [C][K] solver order
  int* parent = nullptr;        // [C] or null
  int* bcells = nullptr;        // [Nb]
  int* bdofs = nullptr;         // [Nb][BL] solver order
  int* cell_bptr = nullptr;     // [C+1] boundary elements of each cell
  int* cell_blist = nullptr;
  double* k2 = nullptr;         // [W]
  double* weights = nullptr;    // [W]
  int* abmn = nullptr;          // [D][4]
  double* partials = nullptr;   // tiled solver: split-depth partial tiles (2 x SMs tiles of 64 x 64)
  double* inverses = nullptr;   // tiled solver: L_kk^-1 per task of a level and system (grown on use)
  size_t inverses_capacity = 0; // doubles
  int2* row_entries = nullptr;  // [2][D] (A | B << 8 | M << 16 | N << 24, d): sorted by (A, B, M, N), then in row order
  int* rcv_dofs = nullptr;      // [E][RW] solver order
  double* rcv_w = nullptr;      // [E][RW]
  int* src_ptr = nullptr;       // [E+1]
  int* src_cells = nullptr;
  float* features = nullptr;    // [C][R][K]
  float* fscale = nullptr;      // [W][R]
  int* model_ptr = nullptr;     // [Cm+1] discretization cells of each model cell
  int* model_list = nullptr;
  int* pair_ptr = nullptr;      // [(E+1)^2+1] routed pair-cotangent scatter
  int* pair_list = nullptr;
  int* rdof_ptr = nullptr;      // receiver dofs of the adjoint right-hand side
  int* rdof_rcv = nullptr;
  double* rdof_w = nullptr;
  int* rdof_dof = nullptr;
  int rdofs = 0;
  int64_t* tasks = nullptr;
  int64_t* pulls = nullptr;
  int* fixed = nullptr;         // fixed (Dirichlet) dofs, solver order
  int nfixed = 0;
  int* owners = nullptr;        // cells owning boundary elements
  int nowners = 0;
  int* update_items = nullptr;  // eager Schur update items (task, pull begin, pull end)
  std::vector<int> update_begin;
  // tiled solver (blocks wider than kMaxBlock): device work items, host ranges
  bool tiled = false;
  int* titems = nullptr;
  std::vector<int> tranges, panel_ptr;
  std::vector<int> panel_width;  // per tiled item range: widest column panel of its items (0: not a panel)
  // primary field
  double* primary = nullptr;    // [W][N][E] solver order
  double* refrhs = nullptr;     // [W][N][E]
  bool has_primary = false;
  bool static_rhs = false;      // refrhs is the whole right-hand side (no primary correction)
  // slots and workspace
  std::vector<adt::Slot> slots;
  std::vector<adt::Aggregation> aggregations;
  double* pot = nullptr;        // potential tables of the measurement kernels
  size_t pot_count = 0;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  std::string error;
  int64_t launches = 0;
  int device = 0;
  int sms = 148;                // multiprocessors of the device
  // launch-shape rules of the solver (chosen by adt_autotune, else these defaults):
  int strip_fill = 2;           // substitution strips narrow while blocks x strips < strip_fill x SMs
  int split_fill = 2;           // tiled panels split while tiles x systems x splits x 2 <= split_fill x SMs
  bool jacobian_tc = true;      // tensor-core Jacobian where it applies
  bool jacobian_pipe = true;    // its warp-role pipelined form where that applies
  bool jacobian_direct = true;  // direct-form Jacobian for single-wavenumber operators
  bool cgls_ring = true;        // shared-memory ring data pass of adt_gn_step where p and its rows fit
  unsigned tc_first_wait_polls = 0;  // 0: default MMA wait of the tensor-core Jacobian; n: n polls
  int* tc_error = nullptr;      // device flag raised by a tensor-core block that timed out
  int* tc_error_host = nullptr; // pinned copy, refreshed after each tensor-core launch
  cudaStream_t copy_stream = nullptr;        // device-to-host copies of Jacobian column chunks
  std::vector<cudaEvent_t> chunk_events;     // chunk done (compute stream), copies done (copy stream)
};

namespace adt {

// Record an error on the plan and return `status`.
adt_status fail(adt_plan* plan, adt_status status, const std::string& message);
// Check the launch status of the last kernel.
adt_status check_launch(adt_plan* plan, const char* what);
// Grow the plan's scratch to `bytes`; returns nullptr on failure.
void* scratch(adt_plan* plan, size_t bytes);

}  // namespace adt
