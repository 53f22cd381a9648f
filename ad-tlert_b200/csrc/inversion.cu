// Gauss-Newton model step of the windowed time-lapse inversion, on the device.
//
// One window holds T models of C cells and T x D log-apparent-resistivity data. Its linearized
// system (adtlert/inversion/core.py:81-300 with the weighted log L2 data term of
// adtlert/inversion/misfit.py:75-115, first-order spatial smoothness and first-order temporal
// smoothness of adtlert/inversion/regularization.py:97-357) is
//
//   A = [ W J (block-diagonal over t) ; sqrt(ls) R (per t) ; sqrt(lt) (first difference in t) ],
//   b = [ -W (pred - obs) ; -sqrt(ls) R m ; -sqrt(lt) T m ],
//
// and the step solves min ||A x - b|| by CGLS (adtlert/inversion/optimizers.py:314-360): x = 0,
// s = A^T b, p = s, gamma = s.s; per iteration alpha = gamma / ||A p||^2, x += alpha p,
// s -= alpha A^T A p, gamma' = s.s, stop when gamma' / gamma_0 < tolerance, p = s + (gamma' /
// gamma) p. The reference keeps r = b - A x and recomputes s = A^T r; here s follows its own
// recurrence, which is the same sequence in exact arithmetic and lets one pass over J per
// iteration produce both ||A p||^2 = p.(A^T A p) and A^T A p.
//
// Kernels of one iteration (all chained on the caller's stream; a device flag set when the
// iteration stops turns the rest of the launched iterations into no-ops, so the host never waits
// inside the loop):
//   normal_data_kernel   per block, a range of rows of one model: q_d = w_d (J_d . p_t), then
//                        partial += J_d w_d q_d, in float64 registers; written once per block.
//   normal_reduce_kernel u = sum of the block partials (fixed order) + ls L p_t + lt T^T T p,
//                        with L = R^T R from neighbour lists; block partials of p.u.
//   cgls_update_kernel   one block: alpha, x, s, gamma', beta, p.
// Every reduction runs in a fixed order, so a step is bitwise repeatable.
#include "adt_internal.h"

namespace {

constexpr int kPassThreads = 512;
constexpr int kReduceThreads = 256;
constexpr int kUpdateThreads = 1024;
constexpr int kMaxVec = 8;  // float4 per thread of the data pass: C <= 4 * 512 * 8 = 16384 columns

struct CglsState {
  double gamma;
  double gamma0;
  int done;
  int iterations;
};

struct Workspace {
  CglsState* state;
  double* s;
  double* p;
  double* u;
  double* partial;
  double* dots;
  int ctas_per_model;
  int reduce_blocks;
};

size_t align256(size_t bytes) { return (bytes + 255) & ~size_t(255); }

int data_ctas_per_model(int steps, int sms) {
  const int per = (sms + steps - 1) / steps;
  return per < 1 ? 1 : per;
}

size_t workspace_layout(int T, int D, int C, int sms, Workspace* w, char* base) {
  const size_t n = (size_t)T * C;
  const int per = data_ctas_per_model(T, sms);
  const int reduce_blocks = (int)((n + kReduceThreads - 1) / kReduceThreads);
  size_t offset = 0;
  auto take = [&](size_t bytes) {
    char* at = base ? base + offset : nullptr;
    offset += align256(bytes);
    return at;
  };
  char* state = take(sizeof(CglsState));
  char* s = take(n * sizeof(double));
  char* p = take(n * sizeof(double));
  char* u = take(n * sizeof(double));
  char* partial = take((size_t)T * per * C * sizeof(double));
  char* dots = take((size_t)reduce_blocks * sizeof(double));
  (void)D;
  if (w) {
    w->state = reinterpret_cast<CglsState*>(state);
    w->s = reinterpret_cast<double*>(s);
    w->p = reinterpret_cast<double*>(p);
    w->u = reinterpret_cast<double*>(u);
    w->partial = reinterpret_cast<double*>(partial);
    w->dots = reinterpret_cast<double*>(dots);
    w->ctas_per_model = per;
    w->reduce_blocks = reduce_blocks;
  }
  return offset;
}

// Data pass. `given` (T x D) replaces the row products q_d when not null (A^T b: q = b_data).
// J is read as float32 (streamed once), every product and sum is float64: CGLS truncated at
// tens of iterations is sensitive to rounding in A^T A p (float32 rounding of it alone moves the
// least-squares residual after 60 iterations by ~6e-4), so only the matrix is float32.
template <int VEC>
__global__ void __launch_bounds__(kPassThreads) normal_data_kernel(
    const float* __restrict__ J, int D, int C, const double* __restrict__ weights, const double* __restrict__ vec,
    const double* __restrict__ given, int ctas_per_model, double* __restrict__ partial,
    const CglsState* __restrict__ state) {
  adt::chain_wait();
  if (state != nullptr && state->done) return;
  extern __shared__ double pvec[];  // p_t (C doubles) when the rows' products are formed here
  const int t = blockIdx.x / ctas_per_model, k = blockIdx.x % ctas_per_model;
  const int rows_per = (D + ctas_per_model - 1) / ctas_per_model;
  const int d0 = k * rows_per, d1 = min(D, d0 + rows_per);
  const int C4 = C >> 2;
  if (given == nullptr)
    for (int c = threadIdx.x; c < C; c += kPassThreads) pvec[c] = vec[(size_t)t * C + c];
  __syncthreads();
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  double acc[VEC][4];
#pragma unroll
  for (int v = 0; v < VEC; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.0;
  __shared__ double red[2][kPassThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int parity = 0;
  for (int d = d0; d < d1; ++d) {
    const float4* row = reinterpret_cast<const float4*>(J + ((size_t)t * D + d) * C);
    float4 r[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const int idx = threadIdx.x + v * kPassThreads;
      r[v] = idx < C4 ? __ldcs(row + idx) : zero;
    }
    const double w = weights[(size_t)t * D + d];
    double q;
    if (given != nullptr) {
      q = given[(size_t)t * D + d];
    } else {
      double dot = 0.0;
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        const int idx = threadIdx.x + v * kPassThreads;
        if (idx < C4) {
          const double* pc = pvec + 4 * idx;
          dot = fma((double)r[v].x, pc[0], dot);
          dot = fma((double)r[v].y, pc[1], dot);
          dot = fma((double)r[v].z, pc[2], dot);
          dot = fma((double)r[v].w, pc[3], dot);
        }
      }
#pragma unroll
      for (int offset = 16; offset > 0; offset >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, offset);
      if (lane == 0) red[parity][warp] = dot;
      __syncthreads();
      dot = 0.0;
#pragma unroll
      for (int i = 0; i < kPassThreads / 32; ++i) dot += red[parity][i];
      parity ^= 1;
      q = w * dot;
    }
    const double wq = w * q;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      acc[v][0] = fma((double)r[v].x, wq, acc[v][0]);
      acc[v][1] = fma((double)r[v].y, wq, acc[v][1]);
      acc[v][2] = fma((double)r[v].z, wq, acc[v][2]);
      acc[v][3] = fma((double)r[v].w, wq, acc[v][3]);
    }
  }
  double* out = partial + (size_t)blockIdx.x * C;
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    const int idx = threadIdx.x + v * kPassThreads;
    if (idx < C4) {
      double2* pair = reinterpret_cast<double2*>(out + 4 * idx);
      pair[0] = make_double2(acc[v][0], acc[v][1]);
      pair[1] = make_double2(acc[v][2], acc[v][3]);
    }
  }
}

// Block sum of one double per thread, in a fixed order (shuffle tree, then warp 0 over the
// warps in order). The result is valid in thread 0.
template <int THREADS>
__device__ __forceinline__ double block_sum(double value, double* shared) {
  for (int offset = 16; offset > 0; offset >>= 1) value += __shfl_xor_sync(0xffffffffu, value, offset);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) shared[warp] = value;
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < THREADS / 32; ++i) total += shared[i];
  __syncthreads();
  return total;
}

// u = (sum of the data partials) + spatial L v_t + temporal T^T T v, element (t, c) per thread;
// with `dot_with`, per-block partials of dot_with . u. `partial` may be null (regularizer only).
__global__ void __launch_bounds__(kReduceThreads) normal_reduce_kernel(
    const double* __restrict__ partial, int ctas_per_model, int T, int C, const double* __restrict__ v,
    const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_cell, const double* __restrict__ nbr_w2,
    double spatial, double temporal, const double* __restrict__ dot_with, double* __restrict__ u,
    double* __restrict__ dots, const CglsState* __restrict__ state) {
  adt::chain_wait();
  if (state != nullptr && state->done) return;
  __shared__ double shared[kReduceThreads / 32];
  const int64_t n = (int64_t)T * C;
  const int64_t i = (int64_t)blockIdx.x * kReduceThreads + threadIdx.x;
  double product = 0.0;
  if (i < n) {
    const int t = (int)(i / C), c = (int)(i % C);
    double sum = 0.0;
    if (partial != nullptr)
      for (int k = 0; k < ctas_per_model; ++k) sum += partial[((size_t)t * ctas_per_model + k) * C + c];
    const double* vt = v + (size_t)t * C;
    const double vc = vt[c];
    double lap = 0.0;
    for (int j = nbr_ptr[c]; j < nbr_ptr[c + 1]; ++j) lap += nbr_w2[j] * (vc - vt[nbr_cell[j]]);
    double tt = 0.0;
    if (t > 0) tt += vc - v[i - C];
    if (t < T - 1) tt += vc - v[i + C];
    const double value = sum + spatial * lap + temporal * tt;
    u[i] = value;
    if (dot_with != nullptr) product = dot_with[i] * value;
  }
  if (dot_with != nullptr) {
    const double total = block_sum<kReduceThreads>(product, shared);
    if (threadIdx.x == 0) dots[blockIdx.x] = total;
  }
}

// x = 0, s = p = A^T b (in u), gamma = gamma_0 = s.s.
__global__ void __launch_bounds__(kUpdateThreads) cgls_start_kernel(CglsState* st, int64_t n, const double* __restrict__ u,
                                                                    double* __restrict__ x, double* __restrict__ s,
                                                                    double* __restrict__ p) {
  adt::chain_wait();
  __shared__ double shared[kUpdateThreads / 32];
  double ss = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kUpdateThreads) {
    const double value = u[i];
    x[i] = 0.0;
    s[i] = value;
    p[i] = value;
    ss += value * value;
  }
  const double gamma = block_sum<kUpdateThreads>(ss, shared);
  if (threadIdx.x == 0) {
    st->gamma = gamma;
    st->gamma0 = gamma;
    st->done = gamma > 0.0 ? 0 : 1;
    st->iterations = 0;
  }
}

__global__ void __launch_bounds__(kUpdateThreads) cgls_update_kernel(CglsState* st, int64_t n,
                                                                     const double* __restrict__ dots, int blocks,
                                                                     double* __restrict__ x, double* __restrict__ s,
                                                                     double* __restrict__ p,
                                                                     const double* __restrict__ u, double tolerance) {
  adt::chain_wait();
  __shared__ double shared[kUpdateThreads / 32];
  __shared__ double alpha_s, beta_s;
  __shared__ int stop_s;
  if (threadIdx.x == 0) {  // only thread 0 reads or writes the flag in this kernel
    if (st->done) {
      stop_s = 1;
    } else {
      double pu = 0.0;
      for (int b = 0; b < blocks; ++b) pu += dots[b];
      stop_s = pu > 0.0 ? 0 : 1;
      alpha_s = stop_s ? 0.0 : st->gamma / pu;
      if (stop_s) st->done = 1;
    }
  }
  __syncthreads();
  if (stop_s) return;
  const double alpha = alpha_s;
  double ss = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kUpdateThreads) {
    x[i] += alpha * p[i];
    const double si = s[i] - alpha * u[i];
    s[i] = si;
    ss += si * si;
  }
  const double gamma_new = block_sum<kUpdateThreads>(ss, shared);
  if (threadIdx.x == 0) {
    st->iterations += 1;
    if (!(gamma_new > 0.0) || gamma_new / st->gamma0 < tolerance) {
      stop_s = 1;
      st->done = 1;
    } else {
      beta_s = gamma_new / st->gamma;
      st->gamma = gamma_new;
    }
  }
  __syncthreads();
  if (stop_s) return;
  const double beta = beta_s;
  for (int64_t i = threadIdx.x; i < n; i += kUpdateThreads) {
    const double value = s[i] + beta * p[i];
    p[i] = value;
  }
}

template <int VEC>
void launch_data(const float* J, int T, int D, int C, const double* weights, const double* vec, const double* given,
                 const Workspace& w, const CglsState* state, cudaStream_t s) {
  const size_t smem = given == nullptr ? (size_t)C * sizeof(double) : 0;
  static bool raised = false;  // the dynamic shared-memory limit, raised once per instantiation
  if (!raised) {
    cudaFuncSetAttribute(normal_data_kernel<VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         4 * kPassThreads * VEC * (int)sizeof(double));
    raised = true;
  }
  adt::launch_chained(normal_data_kernel<VEC>, dim3(T * w.ctas_per_model), dim3(kPassThreads), smem, s, J, D, C,
                      weights, vec, given, w.ctas_per_model, w.partial, state);
}

bool data_pass(const float* J, int T, int D, int C, const double* weights, const double* vec, const double* given,
               const Workspace& w, const CglsState* state, cudaStream_t s) {
  const int vec_per_thread = ((C >> 2) + kPassThreads - 1) / kPassThreads;
  switch (vec_per_thread) {
    case 0:
    case 1: launch_data<1>(J, T, D, C, weights, vec, given, w, state, s); return true;
    case 2: launch_data<2>(J, T, D, C, weights, vec, given, w, state, s); return true;
    case 3: launch_data<3>(J, T, D, C, weights, vec, given, w, state, s); return true;
    case 4: launch_data<4>(J, T, D, C, weights, vec, given, w, state, s); return true;
    case 5: launch_data<5>(J, T, D, C, weights, vec, given, w, state, s); return true;
    case 6: launch_data<6>(J, T, D, C, weights, vec, given, w, state, s); return true;
    case 7:
    case 8: launch_data<8>(J, T, D, C, weights, vec, given, w, state, s); return true;
    default: return false;
  }
}

}  // namespace

extern "C" adt_status adt_gn_workspace_bytes(int32_t steps, int32_t rows, int32_t columns, int32_t multiprocessors,
                                             size_t* bytes) {
  if (steps <= 0 || rows <= 0 || columns <= 0 || multiprocessors <= 0 || !bytes) return ADT_INVALID_ARG;
  *bytes = workspace_layout(steps, rows, columns, multiprocessors, nullptr, nullptr);
  return ADT_OK;
}

extern "C" adt_status adt_gn_step(adt_plan* p, const float* jacobian, int32_t steps, int32_t rows, int32_t columns,
                                  const double* data_weights, const double* data_rhs, const double* models,
                                  const int32_t* neighbour_ptr, const int32_t* neighbour_cells,
                                  const double* neighbour_weights, double spatial, double temporal,
                                  int32_t iterations, double tolerance, double* step, void* workspace,
                                  size_t workspace_bytes, int32_t multiprocessors, adt_stream stream) {
  if (!p) return ADT_INVALID_ARG;
  if (!jacobian || !data_weights || !data_rhs || !models || !neighbour_ptr || !step || !workspace || steps <= 0 ||
      rows <= 0 || columns <= 0 || iterations < 0 || multiprocessors <= 0 || spatial < 0.0 || temporal < 0.0)
    return adt::fail(p, ADT_INVALID_ARG, "adt_gn_step: invalid arguments");
  if (columns % 4 != 0 || columns > 4 * kPassThreads * kMaxVec)
    return adt::fail(p, ADT_INVALID_ARG,
                     "adt_gn_step: the column count must be a multiple of 4 and at most " +
                         std::to_string(4 * kPassThreads * kMaxVec));
  if ((reinterpret_cast<uintptr_t>(jacobian) & 15) != 0)
    return adt::fail(p, ADT_INVALID_ARG, "adt_gn_step: the Jacobian must be 16-byte aligned");
  Workspace w;
  const size_t need = workspace_layout(steps, rows, columns, multiprocessors, &w, static_cast<char*>(workspace));
  if (workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return adt::fail(p, ADT_INVALID_ARG, "adt_gn_step: workspace too small or not 256-byte aligned (need " +
                                             std::to_string(need) + " bytes)");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = (int64_t)steps * columns;
  // s_0 = A^T b = J^T W b_data - ls L m - lt T^T T m
  data_pass(jacobian, steps, rows, columns, data_weights, w.p, data_rhs, w, nullptr, s);
  adt::launch_chained(normal_reduce_kernel, dim3(w.reduce_blocks), dim3(kReduceThreads), 0, s, (const double*)w.partial,
                      w.ctas_per_model, (int)steps, (int)columns, models, neighbour_ptr, neighbour_cells,
                      neighbour_weights, -spatial, -temporal, (const double*)nullptr, w.u, w.dots,
                      (const CglsState*)nullptr);
  adt::launch_chained(cgls_start_kernel, dim3(1), dim3(kUpdateThreads), 0, s, w.state, n, (const double*)w.u, step,
                      w.s, w.p);
  p->launches += 3;
  for (int it = 0; it < iterations; ++it) {
    data_pass(jacobian, steps, rows, columns, data_weights, w.p, nullptr, w, w.state, s);
    adt::launch_chained(normal_reduce_kernel, dim3(w.reduce_blocks), dim3(kReduceThreads), 0, s,
                        (const double*)w.partial, w.ctas_per_model, (int)steps, (int)columns, (const double*)w.p,
                        neighbour_ptr, neighbour_cells, neighbour_weights, spatial, temporal, (const double*)w.p, w.u,
                        w.dots, (const CglsState*)w.state);
    adt::launch_chained(cgls_update_kernel, dim3(1), dim3(kUpdateThreads), 0, s, w.state, n, (const double*)w.dots,
                        w.reduce_blocks, step, w.s, w.p, (const double*)w.u, tolerance);
    p->launches += 3;
  }
  return adt::check_launch(p, "gauss-newton step");
}

extern "C" adt_status adt_gn_regularize(adt_plan* p, int32_t steps, int32_t columns, const int32_t* neighbour_ptr,
                                        const int32_t* neighbour_cells, const double* neighbour_weights,
                                        double spatial, double temporal, const double* models, double* out,
                                        adt_stream stream) {
  if (!p) return ADT_INVALID_ARG;
  if (steps <= 0 || columns <= 0 || !neighbour_ptr || !models || !out)
    return adt::fail(p, ADT_INVALID_ARG, "adt_gn_regularize: invalid arguments");
  const int64_t n = (int64_t)steps * columns;
  adt::launch_chained(normal_reduce_kernel, dim3((unsigned)((n + kReduceThreads - 1) / kReduceThreads)),
                      dim3(kReduceThreads), 0, (cudaStream_t)stream, (const double*)nullptr, 0, (int)steps,
                      (int)columns, models, neighbour_ptr, neighbour_cells, neighbour_weights, spatial, temporal,
                      (const double*)nullptr, out, (double*)nullptr, (const CglsState*)nullptr);
  p->launches += 1;
  return adt::check_launch(p, "gauss-newton regularizer");
}
