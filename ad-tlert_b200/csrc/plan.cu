// Plan construction (host) and the C-ABI entry points of adtlert_b200.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include <cstdlib>
#include <cstring>

#include "adt_internal.h"
#include "kernels.h"
#include "plan_host.h"

namespace adt {

adt_status factorize_systems(adt_plan* p, int systems, const double* values, double* factors,
                             cudaStream_t s);
adt_status solve_systems(adt_plan* p, int systems, int nrhs, const double* factors,
                         double* rhs, cudaStream_t s);
bool fused_rhs_supported(const adt_plan* p, int nrhs);
adt_status factorize_systems_rhs(adt_plan* p, int systems, const double* values, double* factors, double* rhs,
                                 int nrhs, cudaStream_t s);
adt_status backward_systems(adt_plan* p, int systems, int nrhs, const double* factors, double* rhs, cudaStream_t s);
void configure_solver_kernels();
size_t jacobian_smem(int cells, int R, int E, int K);

namespace {

thread_local std::string g_create_error;

template <typename T>
adt_status upload(adt_plan* p, T** dst, const T* src, size_t count) {
  *dst = nullptr;
  if (count == 0) return ADT_OK;
  if (cudaMalloc(dst, count * sizeof(T)) != cudaSuccess)
    return fail(p, ADT_OOM, "device allocation failed");
  if (cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(p, ADT_CUDA_ERROR, "host-to-device copy failed");
  return ADT_OK;
}

template <typename T>
adt_status upload(adt_plan* p, T** dst, const std::vector<T>& src) {
  return upload(p, dst, src.data(), src.size());
}

}  // namespace

adt_status fail(adt_plan* plan, adt_status status, const std::string& message) {
  if (plan) plan->error = message;
  else g_create_error = message;
  return status;
}

adt_status check_launch(adt_plan* plan, const char* what) {
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess)
    return fail(plan, ADT_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(err));
  return ADT_OK;
}

void* scratch(adt_plan* p, size_t bytes) {
  if (bytes <= p->scratch_bytes) return p->scratch;
  if (p->scratch) cudaFree(p->scratch);
  p->scratch = nullptr;
  p->scratch_bytes = 0;
  if (cudaMalloc(&p->scratch, bytes) != cudaSuccess) return nullptr;
  p->scratch_bytes = bytes;
  return p->scratch;
}

// Carves aligned sub-buffers out of the plan scratch.
struct Carve {
  size_t total = 0;
  std::vector<size_t> offsets;
  size_t add(size_t bytes) {
    offsets.push_back(total);
    total += (bytes + 255) & ~size_t(255);
    return offsets.size() - 1;
  }
};

inline int grid_for(int64_t work, int threads = 256) {
  int64_t blocks = (work + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, 148 * 32));
}

// Systems over y (grid-stride beyond 65535), a system's `per_system` entries over x.
inline dim3 system_grid(int systems, int64_t per_system) {
  return dim3(grid_for(per_system), (unsigned)std::max(1, std::min(systems, 65535)));
}

adt_status ensure_slot(adt_plan* p, int slot, int systems) {
  if (slot < 0) return fail(p, ADT_INVALID_ARG, "slot must be non-negative");
  if ((int)p->slots.size() <= slot) p->slots.resize(slot + 1);
  Slot& s = p->slots[slot];
  if (s.capacity < (size_t)systems) {
    if (s.values) cudaFree(s.values);
    if (s.factors) cudaFree(s.factors);
    s.values = nullptr;
    s.factors = nullptr;
    s.capacity = 0;
    if (cudaMalloc(&s.values, (size_t)systems * p->nnz * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&s.factors, (size_t)systems * p->factor_stride * sizeof(double)) != cudaSuccess)
      return fail(p, ADT_OOM, "factor slot allocation failed");
    s.capacity = systems;
  }
  return ADT_OK;
}

AssembleArgs assemble_args(adt_plan* p, const float* sigma, int systems, double* values,
                           bool robin, bool identity) {
  AssembleArgs a;
  a.sigma = sigma;
  a.parent = p->parent;
  a.contrib_ptr = p->contrib_ptr;
  a.contrib = p->contrib;
  a.stiffness = p->stiffness;
  a.mass = p->mass;
  a.bmass = p->bmass;
  a.bcoef = p->bcoef;
  a.bcells = p->bcells;
  a.k2 = p->k2;
  a.values = values;
  a.systems = systems;
  a.nnz = p->nnz;
  a.W = p->W;
  a.C = p->C;
  a.Cm = p->Cm;
  a.K2 = p->K * p->K;
  a.BL2 = p->BL * p->BL;
  a.Nb = p->Nb;
  a.robin = robin ? 1 : 0;
  a.identity = identity ? 1 : 0;
  a.w0 = 0;
  return a;
}

// System matrices (identity = true: unit diagonals on fixed dofs) or their sigma-derivatives;
// with `rho`, the same launch also writes the source resistivities of the `models` models.
void launch_assemble(adt_plan* p, const float* sigma, int systems, double* values, bool robin,
                     bool identity, cudaStream_t s, double* rho = nullptr, int models = 0) {
  AssembleArgs a = assemble_args(p, sigma, systems, values, robin, identity);
  if (rho) {
    a.rho = rho;
    a.src_ptr = p->src_ptr;
    a.src_cells = p->src_cells;
    a.models = models;
    a.E = p->E;
  }
  launch_chained(assemble_kernel, grid_for((int64_t)systems * p->nnz), 256, 0, s, a);
  p->launches++;
}

template <typename TX>
void launch_spmm(adt_plan* p, const double* values, bool values_per_wavenumber, const TX* x,
                 bool x_per_system, const double* rho, const double* base, double scale,
                 int systems, double* out, cudaStream_t s) {
  SpmmArgs a;
  a.values = values;
  a.csr_ptr = p->csr_ptr;
  a.csr_col = p->csr_col;
  a.x = x;
  a.x_double = sizeof(TX) == sizeof(double);
  a.rho = rho;
  a.base = base;
  a.out = out;
  a.scale = scale;
  a.systems = systems;
  a.N = p->N;
  a.E = p->E;
  a.W = p->W;
  a.nnz = p->nnz;
  a.x_per_system = x_per_system ? 1 : 0;
  a.values_per_wavenumber = values_per_wavenumber ? 1 : 0;
  launch_chained(spmm_kernel, system_grid(systems, (int64_t)p->N * p->E), 256, 0, s, a);
  p->launches++;
}

template <typename TF>
void launch_measure(adt_plan* p, const TF* fields, int models, double* normal, double* recip,
                    double* potentials, const double* base_n, const double* base_r,
                    cudaStream_t s) {
  MeasureArgs a;
  a.fields = fields;
  a.f_double = sizeof(TF) == sizeof(double);
  a.weights = p->weights;
  a.rcv_dofs = p->rcv_dofs;
  a.rcv_w = p->rcv_w;
  a.abmn = p->abmn;
  a.normal = normal;
  a.reciprocal = recip;
  a.potentials = potentials;
  a.base_normal = base_n;
  a.base_recip = base_r;
  a.W = p->W;
  a.N = p->N;
  a.E = p->E;
  a.RW = p->RW;
  a.D = p->D;
  a.combine = base_n ? 1 : 0;
  const size_t need = (size_t)models * (p->E + 1) * (p->E + 1);
  if (need > p->pot_count) {
    if (p->pot) cudaFree(p->pot);
    p->pot = nullptr;
    p->pot_count = 0;
    if (cudaMalloc(&p->pot, need * sizeof(double)) != cudaSuccess) return;
    p->pot_count = need;
  }
  launch_chained(potentials_kernel, grid_for((int64_t)need * 32), 256, 0, s, a, models, p->pot);  // warp per entry
  launch_chained(transfers_kernel, grid_for((int64_t)models * p->D), 256, 0, s, a, models, p->pot);
  p->launches += 2;
}

void launch_pairs(adt_plan* p, const double* cot, const double* normal, const double* recip,
                  int count, bool normal_only, bool unit, int row_begin, bool model_of_count,
                  double* pairs, cudaStream_t s) {
  PairArgs a;
  a.pair_ptr = p->pair_ptr;
  a.pair_list = p->pair_list;
  a.cot = cot;
  a.normal = normal;
  a.recip = recip;
  a.pairs = pairs;
  a.count = count;
  a.E = p->E;
  a.D = p->D;
  a.normal_only = normal_only ? 1 : 0;
  a.unit = unit ? 1 : 0;
  a.row_begin = row_begin;
  a.model_of_count = model_of_count ? 1 : 0;
  launch_chained(pair_kernel, grid_for((int64_t)count * p->E * p->E), 256, 0, s, a);
  p->launches++;
}

void launch_adjoint_rhs(adt_plan* p, const double* pairs, int systems, int q_per_model,
                        double* rhs, cudaStream_t s) {
  cudaMemsetAsync(rhs, 0, (size_t)systems * p->N * q_per_model * p->E * sizeof(double), s);
  AdjointRhsArgs a;
  a.pairs = pairs;
  a.rdof_ptr = p->rdof_ptr;
  a.rdof_rcv = p->rdof_rcv;
  a.rdof_w = p->rdof_w;
  a.rdof_dof = p->rdof_dof;
  a.weights = p->weights;
  a.rhs = rhs;
  a.systems = systems;
  a.rdofs = p->rdofs;
  a.q_per_model = q_per_model;
  a.E = p->E;
  a.W = p->W;
  a.N = p->N;
  launch_chained(adjoint_rhs_kernel, grid_for((int64_t)systems * p->rdofs * q_per_model * p->E), 256, 0, s, a);
  p->launches++;
}

void launch_cell_gradient(adt_plan* p, const void* x, bool x_double, int x_cols,
                          const double* x_scale, const void* y, bool y_double,
                          const double* y_scale, int models, int q_per_model, bool robin,
                          double* out, cudaStream_t s) {
  CellGradientArgs a;
  a.x = x;
  a.y = y;
  a.x_double = x_double;
  a.y_double = y_double;
  a.x_scale = x_scale;
  a.y_scale = y_scale;
  a.stiffness = p->stiffness;
  a.mass = p->mass;
  a.bmass = p->bmass;
  a.bcoef = p->bcoef;
  a.k2 = p->k2;
  a.cell_dofs = p->cell_dofs;
  a.cell_bptr = p->cell_bptr;
  a.cell_blist = p->cell_blist;
  a.bdofs = p->bdofs;
  a.out = out;
  a.models = models;
  a.W = p->W;
  a.N = p->N;
  a.E = p->E;
  a.C = p->C;
  a.K = p->K;
  a.BL = p->BL;
  a.Nb = p->Nb;
  a.robin = robin ? 1 : 0;
  a.x_cols = x_cols;
  a.q_per_model = q_per_model;
  const int64_t warps = (int64_t)models * q_per_model * p->C;
  launch_cell_gradient(a, (int)((warps + 7) / 8), s);
  p->launches++;
}

// Sum discretization-cell values [rows][C] (double) into model cells [rows][Cm] (float).
void launch_to_model_cells(adt_plan* p, const double* in, int rows, float* out, cudaStream_t s) {
  launch_chained(aggregate_kernel, grid_for((int64_t)rows * p->Cm), 256, 0, s, 
      in, rows, p->C, p->Cm, p->model_ptr, p->model_list, out, p->C);
  p->launches++;
}

}  // namespace adt

using namespace adt;

extern "C" {

adt_status adt_plan_create(const adt_problem* pr, adt_plan** out) {
  g_create_error.clear();
  if (!pr || !out) return fail(nullptr, ADT_INVALID_ARG, "null argument");
  *out = nullptr;
  HostPlan hp;
  std::string err;
  const adt_status built = build_host_plan(pr, hp, err);
  if (built != ADT_OK) return fail(nullptr, built, err);
  adt_plan* p = new adt_plan();
  cudaGetDevice(&p->device);
  cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device);
  if (const char* choice = std::getenv("ADTLERT_B200_JACOBIAN")) {
    // "fma": the CUDA-core Gram kernel everywhere; "tc": tensor cores wherever they apply
    // "tc1": the tensor-core kernel without warp roles (for comparison)
    p->jacobian_tc = std::strcmp(choice, "fma") != 0;
    p->jacobian_direct = std::strcmp(choice, "fma") != 0 && std::strcmp(choice, "tc") != 0 &&
                         std::strcmp(choice, "tc1") != 0;
    p->jacobian_pipe = std::strcmp(choice, "tc1") != 0;
  }
  if (const char* choice = std::getenv("ADTLERT_B200_CGLS")) {
    // "registers": the register data pass of the Gauss-Newton step at every size (for comparison)
    p->cgls_ring = std::strcmp(choice, "registers") != 0;
  }
  configure_solver_kernels();
  auto bail = [&](adt_status st) {
    g_create_error = p->error;
    adt_plan_destroy(p);
    return st;
  };
  p->N = hp.N; p->dim = hp.dim; p->C = hp.C; p->K = hp.K; p->Cm = hp.Cm; p->Nb = hp.Nb;
  p->BL = hp.BL; p->W = hp.W; p->E = hp.E; p->D = hp.D; p->RW = hp.RW;
  p->nnz = hp.nnz; p->nb = hp.nb; p->max_m = hp.max_m; p->levels = hp.levels;
  for (size_t t = 0; t + T_FIELDS <= hp.task_rows.size(); t += T_FIELDS) {
    const int64_t* row = hp.task_rows.data() + t;
    const int width = (int)(row[T_MJ] + (row[T_P] >= 0 ? row[T_MP] : 0) + (row[T_Q] >= 0 ? row[T_MQ] : 0));
    p->max_width = std::max(p->max_width, width);
  }
  p->RS = hp.RS; p->R = hp.R; p->rdofs = hp.rdofs;
  p->contributions = hp.contributions; p->factor_stride = hp.factor_stride;
  p->perm = hp.perm; p->iperm = hp.iperm; p->level_begin = hp.level_begin;
  const int C = hp.C, K = hp.K, Nb = hp.Nb, BL = hp.BL, W = hp.W, D = hp.D, E = hp.E;
  // ---- upload ----
  adt_status st = ADT_OK;
#define ADT_UP(dst, ...) if ((st = upload(p, dst, __VA_ARGS__)) != ADT_OK) return bail(st)
  ADT_UP(&p->csr_ptr, hp.csr_ptr);
  ADT_UP(&p->csr_col, hp.csr_col);
  ADT_UP(&p->csr_row, hp.csr_row);
  ADT_UP(&p->contrib_ptr, hp.contrib_ptr);
  ADT_UP(&p->contrib, hp.contrib);
  ADT_UP(&p->stiffness, pr->stiffness, (size_t)C * K * K);
  ADT_UP(&p->mass, pr->mass, (size_t)C * K * K);
  if (Nb > 0) {
    ADT_UP(&p->bmass, pr->boundary_mass, (size_t)Nb * BL * BL);
    ADT_UP(&p->bcoef, pr->boundary_coefficients, (size_t)W * Nb);
    ADT_UP(&p->bcells, pr->boundary_cells, (size_t)Nb);
    ADT_UP(&p->bdofs, hp.bd);
  }
  ADT_UP(&p->cell_dofs, hp.cdofs);
  if (pr->parent_cells) ADT_UP(&p->parent, pr->parent_cells, (size_t)C);
  ADT_UP(&p->cell_bptr, hp.cell_bptr);
  ADT_UP(&p->cell_blist, hp.cell_blist);
  ADT_UP(&p->k2, hp.k2);
  ADT_UP(&p->weights, pr->weights, (size_t)W);
  ADT_UP(&p->abmn, pr->abmn, (size_t)D * 4);
  if (E <= 255) {  // packed measurement rows of the direct-form Jacobian
    std::vector<int> order(D);
    std::iota(order.begin(), order.end(), 0);
    const int32_t* q = pr->abmn;
    std::stable_sort(order.begin(), order.end(), [q](int x, int y) {
      return std::lexicographical_compare(q + 4 * x, q + 4 * x + 4, q + 4 * y, q + 4 * y + 4);
    });
    auto pack = [q](int d) {
      return make_int2((int)((uint32_t)q[4 * d] | (uint32_t)q[4 * d + 1] << 8 | (uint32_t)q[4 * d + 2] << 16 |
                             (uint32_t)q[4 * d + 3] << 24), d);
    };
    std::vector<int2> entries(2 * (size_t)D);
    for (int i = 0; i < D; ++i) {
      entries[i] = pack(order[i]);
      entries[(size_t)D + i] = pack(i);
    }
    ADT_UP(&p->row_entries, entries);
  }
  ADT_UP(&p->rcv_dofs, hp.rcv_dofs);
  ADT_UP(&p->rcv_w, hp.rcv_w);
  ADT_UP(&p->src_ptr, pr->source_cell_ptr, (size_t)E + 1);
  ADT_UP(&p->src_cells, pr->source_cells, (size_t)pr->source_cell_ptr[E]);
  ADT_UP(&p->features, hp.features);
  ADT_UP(&p->fscale, hp.fscale);
  ADT_UP(&p->model_ptr, hp.model_ptr);
  ADT_UP(&p->model_list, hp.model_list);
  ADT_UP(&p->tasks, hp.task_rows);
  ADT_UP(&p->pulls, hp.pulls);
  ADT_UP(&p->pair_ptr, hp.pair_ptr);
  ADT_UP(&p->pair_list, hp.pair_list);
  ADT_UP(&p->rdof_ptr, hp.rdof_ptr);
  ADT_UP(&p->rdof_rcv, hp.rdof_rcv);
  ADT_UP(&p->rdof_w, hp.rdof_w);
  ADT_UP(&p->rdof_dof, hp.rdof_dof);
  ADT_UP(&p->fixed, hp.fixed);
  ADT_UP(&p->titems, hp.titems);
  ADT_UP(&p->update_items, hp.update_items);
  p->update_begin = hp.update_begin;
  p->tiled = hp.tiled;
  p->tranges = hp.tranges;
  p->panel_ptr = hp.panel_ptr;
  // the column width of every panel range: min(64, m_j - 64 k) over its items' tasks
  p->panel_width.assign(hp.tranges.size() / 2, 0);
  for (int level = 0; hp.tiled && level < hp.levels; ++level)
    for (int k = 0; k < hp.panel_ptr[level + 1] - hp.panel_ptr[level]; ++k) {
      const int r = 3 * hp.levels + hp.panel_ptr[level] + k;
      for (int it = hp.tranges[2 * r]; it < hp.tranges[2 * r + 1]; ++it) {
        const int64_t mj = hp.task_rows[(size_t)hp.titems[4 * (size_t)it] * T_FIELDS + T_MJ];
        p->panel_width[r] = std::max<int>(p->panel_width[r], (int)std::min<int64_t>(kTile, mj - (int64_t)kTile * k));
      }
    }
  ADT_UP(&p->owners, hp.bowners);
  p->nfixed = (int)hp.fixed.size();
  if (p->tiled && cudaMalloc(&p->partials, sizeof(double) * 2 * (size_t)p->sms * kTile * kTile) != cudaSuccess)
    return bail(fail(p, ADT_OOM, "split workspace allocation failed"));
  if (cudaMalloc(&p->tc_error, sizeof(int)) != cudaSuccess || cudaMemset(p->tc_error, 0, sizeof(int)) != cudaSuccess ||
      cudaHostAlloc(&p->tc_error_host, sizeof(int), cudaHostAllocDefault) != cudaSuccess)
    return bail(fail(p, ADT_OOM, "error flag allocation failed"));
  *p->tc_error_host = 0;
  p->nowners = (int)hp.bowners.size();
#undef ADT_UP
  *out = p;
  return ADT_OK;
}

adt_status adt_plan_destroy(adt_plan* p) {
  if (!p) return ADT_OK;
  void* ptrs[] = {p->csr_ptr, p->csr_col, p->csr_row, p->contrib_ptr, p->contrib, p->stiffness,
                  p->mass, p->bmass, p->bcoef, p->cell_dofs, p->parent, p->bcells, p->bdofs,
                  p->cell_bptr, p->cell_blist, p->k2, p->weights, p->abmn, p->row_entries, p->rcv_dofs,
                  p->rcv_w, p->src_ptr, p->src_cells, p->features, p->fscale, p->model_ptr,
                  p->model_list, p->tasks, p->pulls, p->pair_ptr, p->pair_list, p->rdof_ptr,
                  p->rdof_rcv, p->rdof_w, p->rdof_dof, p->primary, p->refrhs, p->scratch, p->pot,
                  p->fixed, p->owners, p->titems, p->update_items, p->tc_error, p->partials, p->inverses};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (p->tc_error_host) cudaFreeHost(p->tc_error_host);
  for (cudaEvent_t e : p->chunk_events) cudaEventDestroy(e);
  if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
  for (auto& s : p->slots) {
    if (s.values) cudaFree(s.values);
    if (s.factors) cudaFree(s.factors);
    if (s.rhs) cudaFree(s.rhs);
    if (s.rho) cudaFree(s.rho);
  }
  for (auto& a : p->aggregations) {
    if (a.ptr) cudaFree(a.ptr);
    if (a.cells) cudaFree(a.cells);
  }
  delete p;
  return ADT_OK;
}

adt_status adt_plan_get_info(const adt_plan* p, adt_plan_info* info) {
  if (!p || !info) return ADT_INVALID_ARG;
  info->dof_count = p->N;
  info->nnz = p->nnz;
  info->block_count = p->nb;
  info->max_block = p->max_m;
  info->levels = p->levels;
  info->features = p->R;
  info->factor_doubles_per_system = p->factor_stride;
  info->contributions = p->contributions;
  return ADT_OK;
}

adt_status adt_plan_dof_order(const adt_plan* p, int32_t* order) {
  if (!p || !order) return ADT_INVALID_ARG;
  std::memcpy(order, p->perm.data(), sizeof(int32_t) * p->N);
  return ADT_OK;
}

adt_status adt_last_error(const adt_plan* p, char* buffer, size_t size) {
  if (!buffer || size == 0) return ADT_INVALID_ARG;
  const std::string& msg = p ? p->error : g_create_error;
  std::snprintf(buffer, size, "%s", msg.c_str());
  return ADT_OK;
}

adt_status adt_set_primary(adt_plan* p, const double* primary, adt_stream stream) {
  if (!p || !primary) return ADT_INVALID_ARG;
  if (p->static_rhs) return fail(p, ADT_INVALID_ARG, "the plan already holds a static right-hand side");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t count = (size_t)p->W * p->N * p->E;
  std::vector<double> host(count);
  for (int w = 0; w < p->W; ++w)
    for (int e = 0; e < p->E; ++e)
      for (int n = 0; n < p->N; ++n)
        host[((size_t)w * p->N + p->iperm[n]) * p->E + e] = primary[((size_t)w * p->E + e) * p->N + n];
  if (!p->primary && (cudaMalloc(&p->primary, count * sizeof(double)) != cudaSuccess ||
                      cudaMalloc(&p->refrhs, count * sizeof(double)) != cudaSuccess))
    return fail(p, ADT_OOM, "primary field allocation failed");
  if (cudaMemcpy(p->primary, host.data(), count * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(p, ADT_CUDA_ERROR, "primary field copy failed");
  Carve cv;
  const size_t iv = cv.add((size_t)p->W * p->nnz * sizeof(double));
  const size_t is = cv.add((size_t)p->Cm * sizeof(float));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* values = (double*)(base + cv.offsets[iv]);
  float* ones = (float*)(base + cv.offsets[is]);
  std::vector<float> h1(p->Cm, 1.0f);
  cudaMemcpyAsync(ones, h1.data(), h1.size() * sizeof(float), cudaMemcpyHostToDevice, s);
  launch_assemble(p, ones, p->W, values, true, true, s);
  // A(1) u_p for every wavenumber
  launch_spmm<double>(p, values, false, p->primary, false, nullptr, nullptr, 1.0, p->W, p->refrhs, s);
  cudaStreamSynchronize(s);
  p->has_primary = true;
  return check_launch(p, "reference right-hand side");
}

adt_status adt_set_static_rhs(adt_plan* p, const double* unit_primary, const double* direct,
                              adt_stream stream) {
  if (!p) return ADT_INVALID_ARG;
  if (p->primary) return fail(p, ADT_INVALID_ARG, "the plan already holds a primary field");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t count = (size_t)p->W * p->N * p->E;
  // host [W][E][N] original order -> [W][N][E] solver order
  auto permuted = [&](const double* src) {
    std::vector<double> host(count);
    for (int w = 0; w < p->W; ++w)
      for (int e = 0; e < p->E; ++e)
        for (int n = 0; n < p->N; ++n)
          host[((size_t)w * p->N + p->iperm[n]) * p->E + e] = src[((size_t)w * p->E + e) * p->N + n];
    return host;
  };
  if (!p->refrhs && cudaMalloc(&p->refrhs, count * sizeof(double)) != cudaSuccess)
    return fail(p, ADT_OOM, "right-hand side allocation failed");
  Carve cv;
  const size_t iv = cv.add((size_t)p->W * p->nnz * sizeof(double));
  const size_t is = cv.add((size_t)p->Cm * sizeof(float));
  const size_t ix = cv.add(count * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* values = (double*)(base + cv.offsets[iv]);
  float* ones = (float*)(base + cv.offsets[is]);
  double* x = (double*)(base + cv.offsets[ix]);
  cudaMemsetAsync(p->refrhs, 0, count * sizeof(double), s);
  if (unit_primary) {
    const std::vector<double> host = permuted(unit_primary);
    cudaMemcpyAsync(x, host.data(), count * sizeof(double), cudaMemcpyHostToDevice, s);
    std::vector<float> h1(p->Cm, 1.0f);
    cudaMemcpyAsync(ones, h1.data(), h1.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    launch_assemble(p, ones, p->W, values, true, true, s);
    launch_spmm<double>(p, values, false, x, false, nullptr, nullptr, 1.0, p->W, p->refrhs, s);
    cudaStreamSynchronize(s);  // the host staging buffers go out of scope
  }
  if (direct) {
    const std::vector<double> host = permuted(direct);
    cudaMemcpyAsync(x, host.data(), count * sizeof(double), cudaMemcpyHostToDevice, s);
    launch_chained(add_kernel, grid_for((int64_t)count), 256, 0, s, p->refrhs, x, (int64_t)count);
    p->launches++;
    cudaStreamSynchronize(s);
  }
  if (p->nfixed > 0) {
    launch_chained(zero_rows_kernel, grid_for((int64_t)p->W * p->nfixed * p->E), 256, 0, s, 
        p->refrhs, p->fixed, p->nfixed, p->W, p->N, p->E);
    p->launches++;
  }
  cudaStreamSynchronize(s);
  p->has_primary = true;
  p->static_rhs = true;
  return check_launch(p, "static right-hand side");
}

adt_status adt_factorize(adt_plan* p, int32_t slot, const float* sigma, int32_t models,
                         adt_stream stream) {
  if (!p || !sigma || models <= 0) return fail(p, ADT_INVALID_ARG, "invalid factorize arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int systems = models * p->W;
  adt_status st = ensure_slot(p, slot, systems);
  if (st != ADT_OK) return st;
  Slot& sl = p->slots[slot];
  sl.rhs_ready = false;
  launch_assemble(p, sigma, systems, sl.values, true, true, s);
  st = factorize_systems(p, systems, sl.values, sl.factors, s);
  sl.systems = systems;
  return st;
}

adt_status adt_factorize_fields(adt_plan* p, int32_t slot, const float* sigma, int32_t models,
                                adt_stream stream) {
  if (!p || !sigma || models <= 0) return fail(p, ADT_INVALID_ARG, "invalid factorize arguments");
  if (!p->has_primary || p->static_rhs || !fused_rhs_supported(p, p->E))
    return adt_factorize(p, slot, sigma, models, stream);
  cudaStream_t s = (cudaStream_t)stream;
  const int systems = models * p->W;
  adt_status st = ensure_slot(p, slot, systems);
  if (st != ADT_OK) return st;
  Slot& sl = p->slots[slot];
  sl.rhs_ready = false;
  if (sl.rhs_capacity < (size_t)systems) {
    if (sl.rhs) cudaFree(sl.rhs);
    if (sl.rho) cudaFree(sl.rho);
    sl.rhs = sl.rho = nullptr;
    sl.rhs_capacity = 0;
    if (cudaMalloc(&sl.rhs, (size_t)systems * p->N * p->E * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&sl.rho, (size_t)systems * p->E * sizeof(double)) != cudaSuccess)
      return fail(p, ADT_OOM, "field right-hand side allocation failed");
    sl.rhs_capacity = systems;
  }
  launch_assemble(p, sigma, systems, sl.values, true, true, s, sl.rho, models);  // + source resistivities
  // rhs = A(1) u_p - rho A(sigma) u_p, forward-reduced level by level with the factorization
  launch_spmm<double>(p, sl.values, false, p->primary, false, sl.rho, p->refrhs, -1.0, systems, sl.rhs, s);
  st = factorize_systems_rhs(p, systems, sl.values, sl.factors, sl.rhs, p->E, s);
  sl.systems = systems;
  if (st != ADT_OK) return st;
  sl.rhs_ready = true;
  sl.rhs_sigma = sigma;
  sl.rhs_models = models;
  return ADT_OK;
}

adt_status adt_solve_fields(adt_plan* p, int32_t slot, const float* sigma, int32_t models,
                            float* fields, adt_stream stream) {
  if (!p || !sigma || !fields || models <= 0) return fail(p, ADT_INVALID_ARG, "invalid solve arguments");
  if (!p->has_primary)
    return fail(p, ADT_INVALID_ARG, "adt_set_primary or adt_set_static_rhs must be called first");
  if (slot < 0 || slot >= (int)p->slots.size() || p->slots[slot].systems < models * p->W)
    return fail(p, ADT_INVALID_ARG, "slot does not hold a factorization of these models");
  cudaStream_t s = (cudaStream_t)stream;
  const int systems = models * p->W;
  Slot& fs = p->slots[slot];
  if (fs.rhs_ready && fs.rhs_sigma == sigma && fs.rhs_models == models && fs.systems == systems) {
    // right-hand sides formed and forward-reduced by adt_factorize_fields: backward levels only
    fs.rhs_ready = false;  // solved in place
    adt_status st = backward_systems(p, systems, p->E, fs.factors, fs.rhs, s);
    if (st != ADT_OK) return st;
    launch_chained(total_kernel, system_grid(systems, (int64_t)p->N * p->E), 256, 0, s, fs.rhs, p->primary, fs.rho,
                   p->W, p->N, p->E, systems, fields);
    p->launches++;
    return check_launch(p, "field solve");
  }
  Carve cv;
  const size_t ir = cv.add((size_t)models * p->E * sizeof(double));
  const size_t ix = cv.add((size_t)systems * p->N * p->E * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* rho = (double*)(base + cv.offsets[ir]);
  double* x = (double*)(base + cv.offsets[ix]);
  if (p->static_rhs) {
    const size_t per_model = (size_t)p->W * p->N * p->E;
    for (int m = 0; m < models; ++m)
      cudaMemcpyAsync(x + m * per_model, p->refrhs, per_model * sizeof(double),
                      cudaMemcpyDeviceToDevice, s);
    adt_status st = solve_systems(p, systems, p->E, p->slots[slot].factors, x, s);
    if (st != ADT_OK) return st;
    launch_chained(total_kernel, system_grid(systems, (int64_t)p->N * p->E), 256, 0, s, x, nullptr, nullptr, p->W,
                                                                           p->N, p->E, systems, fields);
    p->launches++;
    return check_launch(p, "field solve");
  }
  launch_chained(source_rho_kernel, grid_for((int64_t)models * p->E), 256, 0, s, sigma, p->Cm, p->E, models,
                                                                      p->src_ptr, p->src_cells, rho);
  p->launches++;
  const Slot& sl = p->slots[slot];
  // rhs = A(1) u_p - rho A(sigma) u_p
  launch_spmm<double>(p, sl.values, false, p->primary, false, rho, p->refrhs, -1.0, systems, x, s);
  adt_status st = solve_systems(p, systems, p->E, sl.factors, x, s);
  if (st != ADT_OK) return st;
  launch_chained(total_kernel, system_grid(systems, (int64_t)p->N * p->E), 256, 0, s, x, p->primary, rho, p->W,
                                                                         p->N, p->E, systems, fields);
  p->launches++;
  return check_launch(p, "field solve");
}

adt_status adt_factorize_wavenumbers(adt_plan* p, int32_t slot, const float* sigma, int32_t w_begin,
                                     int32_t w_count, adt_stream stream) {
  if (!p || !sigma || w_begin < 0 || w_count <= 0 || w_begin + w_count > p->W)
    return fail(p, ADT_INVALID_ARG, "invalid wavenumber range");
  cudaStream_t s = (cudaStream_t)stream;
  adt_status st = ensure_slot(p, slot, w_count);
  if (st != ADT_OK) return st;
  Slot& sl = p->slots[slot];
  sl.rhs_ready = false;
  AssembleArgs a = assemble_args(p, sigma, w_count, sl.values, true, true);
  a.W = w_count;
  a.w0 = w_begin;
  launch_chained(assemble_kernel, grid_for((int64_t)w_count * p->nnz), 256, 0, s, a);
  p->launches++;
  st = factorize_systems(p, w_count, sl.values, sl.factors, s);
  sl.systems = w_count;
  return st;
}

adt_status adt_solve(adt_plan* p, int32_t slot, int32_t systems, int32_t nrhs, double* rhs,
                     adt_stream stream) {
  if (!p || !rhs || systems <= 0 || nrhs <= 0) return fail(p, ADT_INVALID_ARG, "invalid solve arguments");
  if (slot < 0 || slot >= (int)p->slots.size() || p->slots[slot].systems < systems)
    return fail(p, ADT_INVALID_ARG, "slot does not hold that many factorized systems");
  const adt_status st = solve_systems(p, systems, nrhs, p->slots[slot].factors, rhs, (cudaStream_t)stream);
  if (st != ADT_OK) return st;
  return check_launch(p, "solve");
}

adt_status adt_forward(adt_plan* p, int32_t slot, const float* sigma, int32_t models, float* fields,
                       double* normal, double* reciprocal, adt_stream stream) {
  if (adt_status st = adt_factorize_fields(p, slot, sigma, models, stream)) return st;
  if (adt_status st = adt_solve_fields(p, slot, sigma, models, fields, stream)) return st;
  return adt_measure(p, fields, models, normal, reciprocal, nullptr, stream);
}

adt_status adt_jacobian(adt_plan* p, int32_t slot, const float* sigma, float* fields, int32_t row_begin,
                        int32_t row_count, float* jacobian, adt_stream stream) {
  if (adt_status st = adt_factorize_fields(p, slot, sigma, 1, stream)) return st;
  if (adt_status st = adt_solve_fields(p, slot, sigma, 1, fields, stream)) return st;
  return adt_normal_jacobian(p, fields, row_begin, row_count, jacobian, stream);
}

adt_status adt_measure(adt_plan* p, const float* fields, int32_t models, double* normal,
                       double* reciprocal, double* potentials, adt_stream stream) {
  if (!p || !fields || !normal || !reciprocal || models <= 0)
    return fail(p, ADT_INVALID_ARG, "invalid measure arguments");
  launch_measure<float>(p, fields, models, normal, reciprocal, potentials, nullptr, nullptr,
                        (cudaStream_t)stream);
  return check_launch(p, "measure");
}

adt_status adt_integrated_potentials(adt_plan* p, const float* fields, float* integrated,
                                     adt_stream stream) {
  if (!p || !fields || !integrated) return ADT_INVALID_ARG;
  int* iperm = nullptr;
  Carve cv;
  const size_t ii = cv.add((size_t)p->N * sizeof(int));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  iperm = (int*)(base + cv.offsets[ii]);
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemcpyAsync(iperm, p->iperm.data(), p->N * sizeof(int), cudaMemcpyHostToDevice, s);
  launch_chained(integrated_kernel, grid_for((int64_t)p->N * p->E), 256, 0, s, fields, p->weights, iperm, p->W,
                                                                    p->N, p->E, integrated);
  p->launches++;
  cudaStreamSynchronize(s);
  return check_launch(p, "integrated potentials");
}

namespace {

// Jacobian rows [row_begin, row_begin + row_count) for cells [c_begin, c_end) into
// out[d * ldo + c] (d relative to row_begin); the tensor-core kernel when it applies.
adt_status launch_normal_jacobian(adt_plan* p, const float* fields, int row_begin, int row_count, int c_begin,
                                  int c_end, float* out, int64_t ldo, cudaStream_t s) {
  JacobianArgs a;
  a.fields = fields;
  a.features = p->features;
  a.cell_dofs = p->cell_dofs;
  a.fscale = p->fscale;
  a.abmn = p->abmn;
  a.out = out;
  a.W = p->W;
  a.N = p->N;
  a.E = p->E;
  a.C = p->C;
  a.K = p->K;
  a.R = p->R;
  a.row_begin = row_begin;
  a.rows = row_count;
  a.c_begin = c_begin;
  a.c_end = c_end;
  a.ldo = ldo;
  if (p->jacobian_direct && p->W == 1 && p->row_entries) {
    if (const int cells = jacobian_direct_cells(p->R, p->E, p->K)) {
      a.cells_per_block = cells;
      // all rows: sorted by current pair; a row range: in row order
      const bool all_rows = row_begin == 0 && row_count == p->D;
      const int2* rows = all_rows ? p->row_entries : p->row_entries + p->D + row_begin;
      const cudaError_t err = launch_jacobian_direct(a, rows, s);
      p->launches++;
      if (err != cudaSuccess) return fail(p, ADT_CUDA_ERROR, std::string("direct jacobian: ") + cudaGetErrorString(err));
      return ADT_OK;
    }
  }
  if (p->jacobian_tc && jacobian_tc_supported(p->E, p->W, p->R, p->K, row_count)) {
    a.cells_per_block = 0;
    a.first_wait_polls = p->tc_first_wait_polls;
    const int batch = p->jacobian_pipe ? jacobian_tcpipe_batch(p->E, p->W, p->R, p->K, row_count) : 0;
    const cudaError_t err = batch > 0 ? launch_jacobian_tcpipe(a, batch, p->tc_error, p->sms, s)
                                      : launch_jacobian_tc(a, p->tc_error, p->sms, s);
    p->launches++;
    if (err != cudaSuccess)
      return fail(p, ADT_CUDA_ERROR, std::string("tensor-core jacobian: ") + cudaGetErrorString(err));
    return ADT_OK;
  }
  const int E4 = (p->E + 3) & ~3;
  const int nt4 = E4 / 4, NT = nt4 * (nt4 + 1) / 2;
  // cells per block: a power of two (threads split evenly over cells), at most 5 Gram tiles and
  // 4 feature items per thread, and shared memory for two blocks per SM
  int cells = 32;
  while (cells > 1 && (cells * NT > 256 * 5 || cells * E4 > 256 * 4 ||
                       jacobian_smem(cells, p->R, p->E, p->K) > 110 * 1024))
    cells /= 2;
  const size_t smem = jacobian_smem(cells, p->R, p->E, p->K);
  if (smem > 220 * 1024 || cells * NT > 256 * 5 || cells * E4 > 256 * 4)
    return fail(p, ADT_INVALID_ARG, "too many electrodes for the sensitivity kernel");
  a.cells_per_block = cells;
  launch_jacobian(a, smem, s);
  p->launches++;
  return ADT_OK;
}

adt_status jacobian_timeout_status(adt_plan* p) {
  if (p->tc_error_host && *p->tc_error_host != 0)
    return fail(p, ADT_TIMEOUT, "a tensor-core Jacobian launch of this plan timed out waiting for its MMAs");
  return ADT_OK;
}

// After tensor-core launches: the error flag to the pinned host word read by the next call.
void fetch_jacobian_error(adt_plan* p, cudaStream_t s) {
  if (p->jacobian_tc && jacobian_tc_supported(p->E, p->W, p->R, p->K, p->D))
    cudaMemcpyAsync(p->tc_error_host, p->tc_error, sizeof(int), cudaMemcpyDeviceToHost, s);
}

}  // namespace

adt_status adt_normal_jacobian(adt_plan* p, const float* fields, int32_t row_begin,
                               int32_t row_count, float* jacobian, adt_stream stream) {
  if (!p || !fields || !jacobian || row_begin < 0 || row_count < 0 || row_begin + row_count > p->D)
    return fail(p, ADT_INVALID_ARG, "invalid jacobian arguments");
  if (row_count == 0) return ADT_OK;
  if (adt_status st = jacobian_timeout_status(p)) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if (adt_status st = launch_normal_jacobian(p, fields, row_begin, row_count, 0, p->C, jacobian, p->C, s)) return st;
  if (p->jacobian_tc && jacobian_tc_supported(p->E, p->W, p->R, p->K, row_count))
    cudaMemcpyAsync(p->tc_error_host, p->tc_error, sizeof(int), cudaMemcpyDeviceToHost, s);
  return check_launch(p, "normal jacobian");
}

adt_status adt_normal_jacobian_to_host(adt_plan* p, const float* fields, float* device_jacobian,
                                       float* host_jacobian, int32_t chunks, adt_stream stream) {
  if (!p || !fields || !device_jacobian || !host_jacobian || chunks < 1)
    return fail(p, ADT_INVALID_ARG, "invalid jacobian arguments");
  if (p->D == 0) return ADT_OK;
  if (adt_status st = jacobian_timeout_status(p)) return st;
  cudaStream_t s = (cudaStream_t)stream;
  chunks = std::min<int32_t>(chunks, std::max(1, p->C / 64));
  if (!p->copy_stream) {
    if (cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(p, ADT_CUDA_ERROR, "could not create the copy stream");
  }
  while ((int)p->chunk_events.size() < chunks + 1) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      return fail(p, ADT_CUDA_ERROR, "could not create a chunk event");
    p->chunk_events.push_back(e);
  }
  const size_t pitch = (size_t)p->C * sizeof(float);
  for (int k = 0; k < chunks; ++k) {
    // even cell boundaries keep the paired stores of a row aligned
    const int c0 = k == 0 ? 0 : (int)(((int64_t)p->C * k / chunks) & ~int64_t(1));
    const int c1 = k == chunks - 1 ? p->C : (int)(((int64_t)p->C * (k + 1) / chunks) & ~int64_t(1));
    if (c1 <= c0) continue;
    if (adt_status st = launch_normal_jacobian(p, fields, 0, p->D, c0, c1, device_jacobian, p->C, s)) return st;
    cudaEventRecord(p->chunk_events[k], s);
    cudaStreamWaitEvent(p->copy_stream, p->chunk_events[k], 0);
    cudaMemcpy2DAsync(host_jacobian + c0, pitch, device_jacobian + c0, pitch, (size_t)(c1 - c0) * sizeof(float),
                      p->D, cudaMemcpyDeviceToHost, p->copy_stream);
  }
  cudaEventRecord(p->chunk_events[chunks], p->copy_stream);
  cudaStreamWaitEvent(s, p->chunk_events[chunks], 0);
  fetch_jacobian_error(p, s);
  return check_launch(p, "normal jacobian to host");
}

adt_status adt_aggregate_columns(adt_plan* p, int32_t key, int32_t columns,
                                 const int32_t* column_ptr, const int32_t* column_cells,
                                 const float* values, int32_t rows, int32_t in_columns,
                                 float* out, adt_stream stream) {
  if (!p || !column_ptr || !column_cells || !values || !out || columns <= 0 || rows < 0 ||
      in_columns <= 0)
    return fail(p, ADT_INVALID_ARG, "invalid aggregation arguments");
  Aggregation* agg = nullptr;
  for (auto& a : p->aggregations)
    if (a.key == key && a.columns == columns) agg = &a;
  if (!agg) {
    for (int i = 0; i < column_ptr[columns]; ++i)
      if (column_cells[i] < 0 || column_cells[i] >= in_columns)
        return fail(p, ADT_INVALID_ARG, "aggregation cell out of range");
    Aggregation a;
    a.key = key;
    a.columns = columns;
    adt_status st;
    if ((st = upload(p, &a.ptr, column_ptr, (size_t)columns + 1)) != ADT_OK) return st;
    if ((st = upload(p, &a.cells, column_cells, (size_t)std::max(column_ptr[columns], 1))) != ADT_OK) return st;
    p->aggregations.push_back(a);
    agg = &p->aggregations.back();
  }
  if (rows == 0) return ADT_OK;
  launch_chained(aggregate_float_kernel, grid_for((int64_t)rows * columns), 256, 0, (cudaStream_t)stream, 
      values, rows, in_columns, columns, agg->ptr, agg->cells, out);
  p->launches++;
  return check_launch(p, "aggregation");
}

adt_status adt_vjp(adt_plan* p, int32_t slot, const float* fields, const double* normal,
                   const double* reciprocal, const double* cotangents, int32_t models,
                   float* gradient, adt_stream stream) {
  if (!p || !fields || !normal || !reciprocal || !cotangents || !gradient || models <= 0)
    return fail(p, ADT_INVALID_ARG, "invalid vjp arguments");
  if (slot < 0 || slot >= (int)p->slots.size() || p->slots[slot].systems < models * p->W)
    return fail(p, ADT_INVALID_ARG, "slot does not hold a factorization of these models");
  cudaStream_t s = (cudaStream_t)stream;
  const int systems = models * p->W;
  Carve cv;
  const size_t ip = cv.add((size_t)models * p->E * p->E * sizeof(double));
  const size_t ix = cv.add((size_t)systems * p->N * p->E * sizeof(double));
  const size_t ig = cv.add((size_t)models * p->C * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* pairs = (double*)(base + cv.offsets[ip]);
  double* lam = (double*)(base + cv.offsets[ix]);
  double* g = (double*)(base + cv.offsets[ig]);
  launch_pairs(p, cotangents, normal, reciprocal, models, false, false, 0, true, pairs, s);
  launch_adjoint_rhs(p, pairs, systems, 1, lam, s);
  adt_status st = solve_systems(p, systems, p->E, p->slots[slot].factors, lam, s);
  if (st != ADT_OK) return st;
  launch_cell_gradient(p, lam, true, p->E, nullptr, fields, false, nullptr, models, 1, true, g, s);
  launch_to_model_cells(p, g, models, gradient, s);
  return check_launch(p, "vjp");
}

adt_status adt_adjoint_jacobian(adt_plan* p, int32_t slot, const float* fields,
                                const double* normal, const double* reciprocal,
                                int32_t row_begin, int32_t row_count, int32_t robin,
                                int32_t normal_only, float* jacobian, adt_stream stream) {
  if (!p || !fields || !normal || !reciprocal || !jacobian || row_begin < 0 || row_count <= 0 ||
      row_begin + row_count > p->D)
    return fail(p, ADT_INVALID_ARG, "invalid adjoint jacobian arguments");
  if (slot < 0 || slot >= (int)p->slots.size() || p->slots[slot].systems < p->W)
    return fail(p, ADT_INVALID_ARG, "slot does not hold a factorization");
  cudaStream_t s = (cudaStream_t)stream;
  const int Q = row_count;
  Carve cv;
  const size_t ip = cv.add((size_t)Q * p->E * p->E * sizeof(double));
  const size_t ix = cv.add((size_t)p->W * p->N * Q * p->E * sizeof(double));
  const size_t ig = cv.add((size_t)Q * p->C * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* pairs = (double*)(base + cv.offsets[ip]);
  double* lam = (double*)(base + cv.offsets[ix]);
  double* g = (double*)(base + cv.offsets[ig]);
  launch_pairs(p, nullptr, normal, reciprocal, Q, normal_only != 0, true, row_begin, false, pairs, s);
  launch_adjoint_rhs(p, pairs, p->W, Q, lam, s);
  adt_status st = solve_systems(p, p->W, Q * p->E, p->slots[slot].factors, lam, s);
  if (st != ADT_OK) return st;
  launch_cell_gradient(p, lam, true, Q * p->E, nullptr, fields, false, nullptr, 1, Q, robin != 0, g, s);
  launch_to_model_cells(p, g, Q, jacobian, s);
  return check_launch(p, "adjoint jacobian");
}

adt_status adt_jvp(adt_plan* p, int32_t slot, const float* fields, const double* normal,
                   const double* reciprocal, const float* direction, double* out,
                   adt_stream stream) {
  if (!p || !fields || !normal || !reciprocal || !direction || !out)
    return fail(p, ADT_INVALID_ARG, "invalid jvp arguments");
  if (slot < 0 || slot >= (int)p->slots.size() || p->slots[slot].systems < p->W)
    return fail(p, ADT_INVALID_ARG, "slot does not hold a factorization");
  cudaStream_t s = (cudaStream_t)stream;
  Carve cv;
  const size_t iv = cv.add((size_t)p->W * p->nnz * sizeof(double));
  const size_t ix = cv.add((size_t)p->W * p->N * p->E * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* values = (double*)(base + cv.offsets[iv]);
  double* x = (double*)(base + cv.offsets[ix]);
  launch_assemble(p, direction, p->W, values, true, false, s);
  launch_spmm<float>(p, values, false, fields, true, nullptr, nullptr, -1.0, p->W, x, s);
  adt_status st = solve_systems(p, p->W, p->E, p->slots[slot].factors, x, s);
  if (st != ADT_OK) return st;
  launch_measure<double>(p, x, 1, out, nullptr, nullptr, normal, reciprocal, s);
  return check_launch(p, "jvp");
}

adt_status adt_normal_vjp(adt_plan* p, const float* fields, const double* cotangent,
                          int32_t robin, float* gradient, adt_stream stream) {
  if (!p || !fields || !cotangent || !gradient) return fail(p, ADT_INVALID_ARG, "invalid normal_vjp arguments");
  cudaStream_t s = (cudaStream_t)stream;
  Carve cv;
  const size_t ip = cv.add((size_t)p->E * p->E * sizeof(double));
  const size_t ix = cv.add((size_t)p->W * p->N * p->E * sizeof(double));
  const size_t ig = cv.add((size_t)p->C * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* pairs = (double*)(base + cv.offsets[ip]);
  double* current = (double*)(base + cv.offsets[ix]);
  double* g = (double*)(base + cv.offsets[ig]);
  launch_pairs(p, cotangent, nullptr, nullptr, 1, true, false, 0, false, pairs, s);
  if (mix_tiled_smem(p->E) <= 48 * 1024) {
    const int64_t rows = (int64_t)p->W * p->N;
    launch_chained(mix_tiled_kernel, (int)((rows + kMixTileRows - 1) / kMixTileRows), 256, mix_tiled_smem(p->E), s,
                   pairs, fields, rows, p->E, current);
  } else {
    launch_chained(mix_kernel, grid_for((int64_t)p->W * p->N * p->E), 256, 0, s, pairs, fields, p->W, p->N, p->E,
                   current);
  }
  p->launches++;
  launch_cell_gradient(p, current, true, p->E, nullptr, fields, false, p->weights, 1, 1, robin != 0, g, s);
  launch_to_model_cells(p, g, 1, gradient, s);
  return check_launch(p, "normal vjp");
}

adt_status adt_normal_jvp(adt_plan* p, const float* fields, const float* direction,
                          int32_t robin, double* out, adt_stream stream) {
  if (!p || !fields || !direction || !out) return fail(p, ADT_INVALID_ARG, "invalid normal_jvp arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t rows = (int64_t)p->W * p->N;
  const int chunk = 256;
  const int blocks = (int)((rows + chunk - 1) / chunk);
  // rows staged per pass: two float64 row blocks of the padded width within 48 KB, at most N
  const int Ep = (p->E + 3) / 4 * 4;
  const int sub = std::max(1, std::min({64, p->N, 48 * 1024 / (16 * Ep)}));
  Carve cv;
  const size_t iv = cv.add((size_t)p->W * p->nnz * sizeof(double));
  const size_t iy = cv.add((size_t)p->W * p->N * p->E * sizeof(double));
  const size_t ip = cv.add((size_t)blocks * p->E * p->E * sizeof(double));
  const size_t ig = cv.add((size_t)p->E * p->E * sizeof(double));
  char* base = (char*)scratch(p, cv.total);
  if (!base) return fail(p, ADT_OOM, "scratch allocation failed");
  double* values = (double*)(base + cv.offsets[iv]);
  double* y = (double*)(base + cv.offsets[iy]);
  double* partial = (double*)(base + cv.offsets[ip]);
  double* gram = (double*)(base + cv.offsets[ig]);
  launch_assemble(p, direction, p->W, values, robin != 0, false, s);
  launch_spmm<float>(p, values, false, fields, true, nullptr, nullptr, 1.0, p->W, y, s);
  launch_chained(gram_partial_kernel, blocks, 256, (size_t)2 * sub * Ep * sizeof(double), s, fields, y, p->weights,
                 p->W, p->N, p->E, chunk, sub, partial);
  p->launches++;
  launch_chained(gram_reduce_kernel, (p->E * p->E + 255) / 256, 256, 0, s, partial, blocks, p->E, gram);
  p->launches++;
  launch_chained(gram_gather_kernel, (p->D + 255) / 256, 256, 0, s, gram, p->E, p->D, p->abmn, out);
  p->launches++;
  return check_launch(p, "normal jvp");
}

adt_status adt_boundary_jacobian(adt_plan* p, const float* fields, int32_t row_begin,
                                 int32_t row_count, float* jacobian, adt_stream stream) {
  if (!p || !fields || !jacobian || row_begin < 0 || row_count < 0 || row_begin + row_count > p->D)
    return fail(p, ADT_INVALID_ARG, "invalid boundary jacobian arguments");
  if (row_count == 0 || p->nowners == 0) return ADT_OK;
  BoundaryJacobianArgs a;
  a.fields = fields;
  a.weights = p->weights;
  a.bcoef = p->bcoef;
  a.bmass = p->bmass;
  a.bdofs = p->bdofs;
  a.cell_bptr = p->cell_bptr;
  a.cell_blist = p->cell_blist;
  a.owners = p->owners;
  a.abmn = p->abmn;
  a.out = jacobian;
  a.W = p->W;
  a.N = p->N;
  a.E = p->E;
  a.C = p->C;
  a.Nb = p->Nb;
  a.BL = p->BL;
  a.owner_count = p->nowners;
  a.row_begin = row_begin;
  a.rows = row_count;
  launch_chained(boundary_jacobian_kernel, grid_for((int64_t)row_count * p->nowners), 256, 0, (cudaStream_t)stream, a);
  p->launches++;
  return check_launch(p, "boundary jacobian");
}

adt_status adt_scale_rows_columns(float* values, int32_t rows, int32_t columns,
                                  const double* row_scale, const double* column_scale,
                                  adt_stream stream) {
  if (!values || rows < 0 || columns < 0) return fail(nullptr, ADT_INVALID_ARG, "invalid scaling arguments");
  if ((int64_t)rows * columns == 0) return ADT_OK;
  launch_chained(scale_rows_columns_kernel, grid_for((int64_t)rows * columns), 256, 0, (cudaStream_t)stream, 
      values, rows, columns, row_scale, column_scale);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess)
    return fail(nullptr, ADT_CUDA_ERROR, std::string("scaling: ") + cudaGetErrorString(err));
  return ADT_OK;
}

int64_t adt_kernel_launches(const adt_plan* p) { return p ? p->launches : 0; }

}  // extern "C"

extern "C" adt_status adt_set_jacobian_wait_limit(adt_plan* p, uint32_t polls) {
  if (!p) return ADT_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(p, ADT_CUDA_ERROR, "cudaDeviceSynchronize failed");
  p->tc_first_wait_polls = polls;
  if (p->tc_error && cudaMemset(p->tc_error, 0, sizeof(int)) != cudaSuccess)
    return fail(p, ADT_CUDA_ERROR, "resetting the tensor-core error flag failed");
  if (p->tc_error_host) *p->tc_error_host = 0;
  return ADT_OK;
}
