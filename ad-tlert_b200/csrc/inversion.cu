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
// iteration produce both ||A p||^2 = p.(A^T A p) and A^T A p. With u = A^T A p, the new
// gamma' = (s - alpha u).(s - alpha u) = s.s - 2 alpha s.u + alpha^2 u.u comes from dot products
// of the iteration's own s and u (no recurrence over iterations), so one update kernel finishes
// the iteration.
//
// Kernels of one iteration (all chained on the caller's stream; a device flag set when the
// iteration stops turns the rest of the launched iterations into no-ops, so the host never waits
// inside the loop):
//   normal_ring_kernel   per block, a range of rows of one model, streamed through a shared-memory
//                        ring by bulk copies: q_d = w_d (J_d . p_t), then partial += J_d w_d q_d,
//                        in float64 registers; written once per block (normal_data_kernel: the
//                        same with register loads, where p_t and the ring exceed shared memory).
//   normal_reduce_kernel u = sum of the block partials (fixed order) + ls L p_t + lt T^T T p,
//                        with L = R^T R from neighbour lists; block partials of p.u, s.u, u.u
//                        and s.s.
//   cgls_update_kernel   gamma = s.s, alpha = gamma / p.u, gamma' from the sums above, the stop
//                        test; x += alpha p, s -= alpha u, p = s + (gamma' / gamma) p. Every
//                        block sums the partials itself, in one order.
// Every reduction runs in a fixed order, so a step is bitwise repeatable.
#include <algorithm>

#include "adt_internal.h"
#include "tcgen05.h"

namespace {

constexpr int kPassThreads = 512;
constexpr int kReduceColumns = 64;  // reduce kernel: 64 elements per block ...
constexpr int kReduceGroups = 4;    // ... with the data partials of each split over 4 threads
constexpr int kReduceThreads = kReduceColumns * kReduceGroups;
constexpr int kUpdateThreads = 256;  // alpha and beta kernels: one element per thread
constexpr int kStartThreads = 1024;  // start kernel: one block
constexpr int kMaxVec = 8;  // float4 per thread of the data pass: C <= 4 * 512 * 8 = 16384 columns
constexpr int kRingSlots = 4;  // most rows of J in the shared-memory ring of one data-pass block
constexpr uint32_t kRingWaitLimit = 1u << 22;  // mbarrier polls before a ring wait gives up
constexpr size_t kL2ResidentBytes = 96u << 20;  // J bytes loaded evict-last (kept in L2 between passes)
constexpr int kDots = 4;  // dot products per reduce block: p.u, s.u, u.u, s.s

// Per-step device state. The host clears it before a step; `error` is raised by a data pass that
// gave up waiting for its row copies (the step is then NaN). `done` is 0 while the iterations
// run, else 1 + the first iteration that must not run: the update kernel of the stopping
// iteration sets it while its own other blocks still finish that iteration, and every later
// kernel returns at once. gamma0 is s.s of the start (the stop test's reference); gamma[it & 1]
// records iteration it's gamma' (nothing on the device reads it back).
struct CglsState {
  int done;
  int iterations;
  int error;
  int reserved;
  double gamma0;
  double gamma[2];
};

struct Workspace {
  CglsState* state;
  double* s;
  double* p;
  double* u;
  double* partial;
  double* dots;     // per-block partials of p.u, s.u, u.u and s.s (reduce kernel), kDots arrays
  int ctas_per_model;
  int reduce_blocks;
  int update_blocks;
};

size_t align256(size_t bytes) { return (bytes + 255) & ~size_t(255); }

// Blocks per model of a data pass: both data kernels hold one block per multiprocessor, so the
// grid is at most one wave (rounding up would leave a second wave of a few blocks that doubles
// the pass).
int data_ctas_per_model(int steps, int sms) {
  const int per = sms / steps;
  return per < 1 ? 1 : per;
}

int reduce_grid(int64_t n) { return (int)((n + kReduceColumns - 1) / kReduceColumns); }
int update_grid(int64_t n) { return (int)((n + kUpdateThreads - 1) / kUpdateThreads); }

size_t workspace_layout(int T, int D, int C, int sms, Workspace* w, char* base) {
  const size_t n = (size_t)T * C;
  const int per = data_ctas_per_model(T, sms);
  const int reduce_blocks = reduce_grid((int64_t)n), update_blocks = update_grid((int64_t)n);
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
  char* dots = take((size_t)kDots * reduce_blocks * sizeof(double));
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
    w->update_blocks = update_blocks;
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

// Shared-memory ring data pass, the default wherever p_t and three rows fit in shared memory:
// the sums of normal_data_kernel, but the rows of J arrive by bulk asynchronous copies
// (cp.async.bulk, one row per copy, completion counted on one mbarrier per slot) into a ring of
// 4 slots (3 where 4 do not fit), issued that many rows ahead, so they stream while the block
// forms a row's dot product, reduces it and accumulates. Thread 0 issues the copies; a slot is
// refilled after the barrier that ends every thread's reads of it (each thread keeps its slice of
// the row in registers for the accumulation). p_t is held as two planes of double2, (p0, p1) and
// (p2, p3) of each group of four columns, so a warp's reads are conflict-free. Rows of models
// t < l2_resident_models are loaded evict-last and the others evict-first: with three 47 MB
// Jacobians per window, two stay in the 126 MB L2 from one CGLS iteration to the next instead of
// all three thrashing it.
struct RingLayout {
  size_t rows, bars, total;
};

__host__ __device__ inline RingLayout ring_layout(int C, int slots) {
  RingLayout l;
  l.rows = (size_t)C * sizeof(double);  // p_t first, then the slots
  l.bars = l.rows + (size_t)slots * C * sizeof(float);
  l.total = l.bars + (size_t)slots * sizeof(uint64_t);
  return l;
}

constexpr size_t kRingSmemLimit = 227 * 1024 - 1024;  // dynamic bytes; the rest is the static reduction buffer

// Ring slots for C columns: 4 where they fit, else 3, else 0 (the register pass).
inline int ring_slots(int C) {
  for (int slots = kRingSlots; slots >= 3; --slots)
    if (ring_layout(C, slots).total <= kRingSmemLimit) return slots;
  return 0;
}

__device__ __forceinline__ uint64_t l2_policy(bool keep) {
  uint64_t policy;
  if (keep)
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(policy));
  else
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(policy));
  return policy;
}

__device__ __forceinline__ void ring_copy(uint64_t* bar, void* dst, const void* src, uint32_t bytes,
                                          uint64_t policy) {
  const uint32_t b = adt::tc::smem_addr(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;\n" ::
          "r"(adt::tc::smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(b), "l"(policy)
      : "memory");
}

__device__ __forceinline__ bool ring_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t b = adt::tc::smem_addr(bar);
  for (uint32_t polls = 0; polls < kRingWaitLimit; ++polls)
    if (adt::tc::mbar_try_wait(b, parity)) return true;
  return false;
}

template <int VEC>
__global__ void __launch_bounds__(kPassThreads, 1) normal_ring_kernel(
    const float* __restrict__ J, int D, int C, const double* __restrict__ weights, const double* __restrict__ vec,
    const double* __restrict__ given, int ctas_per_model, double* __restrict__ partial, CglsState* state,
    int l2_resident_models, int slots) {
  adt::chain_wait();
  if (given == nullptr && state->done) return;
  extern __shared__ __align__(16) unsigned char ring[];
  const RingLayout lay = ring_layout(C, slots);
  const int C4 = C >> 2;
  double2* pa = reinterpret_cast<double2*>(ring);
  double2* pb = pa + C4;
  float* ring_rows = reinterpret_cast<float*>(ring + lay.rows);
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + lay.bars);
  const int t = blockIdx.x / ctas_per_model, k = blockIdx.x % ctas_per_model;
  const int rows_per = (D + ctas_per_model - 1) / ctas_per_model;
  const int d0 = k * rows_per, n = max(0, min(D, d0 + rows_per) - d0);
  const uint32_t row_bytes = (uint32_t)C * sizeof(float);
  const float* rows0 = J + ((size_t)t * D + d0) * C;
  const uint64_t policy = l2_policy(t < l2_resident_models);
  if (threadIdx.x == 0) {
    for (int slot = 0; slot < slots; ++slot)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(adt::tc::smem_addr(full + slot)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    for (int i = 0; i < min(slots, n); ++i)
      ring_copy(full + i, ring_rows + (size_t)i * C, rows0 + (size_t)i * C, row_bytes, policy);
  }
  if (given == nullptr)
    for (int i = threadIdx.x; i < C4; i += kPassThreads) {
      const double* src = vec + (size_t)t * C + 4 * i;
      pa[i] = make_double2(src[0], src[1]);
      pb[i] = make_double2(src[2], src[3]);
    }
  __syncthreads();
  auto wait_row = [&](int i) { return ring_wait(full + i % slots, (uint32_t)((i / slots) & 1)); };
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  double acc[VEC][4];
#pragma unroll
  for (int v = 0; v < VEC; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = 0.0;
  __shared__ double red[2][kPassThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int stalled = -1;  // the row whose copy did not arrive within the wait limit
  int issued = min(slots, n);
  for (int i = 0; i < n; ++i) {
    const int slot = i % slots;
    const double w = weights[(size_t)t * D + d0 + i];
    const double given_q = given != nullptr ? given[(size_t)t * D + d0 + i] : 0.0;
    const bool ready = wait_row(i);
    const float4* row = reinterpret_cast<const float4*>(ring_rows + (size_t)slot * C);
    float4 r[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const int idx = threadIdx.x + v * kPassThreads;
      r[v] = (ready && idx < C4) ? row[idx] : zero;
    }
    if (given == nullptr) {
      double part[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        const int idx = threadIdx.x + v * kPassThreads;
        if (idx < C4) {
          const double2 a = pa[idx], b = pb[idx];
          part[0] = fma((double)r[v].x, a.x, part[0]);
          part[1] = fma((double)r[v].y, a.y, part[1]);
          part[2] = fma((double)r[v].z, b.x, part[2]);
          part[3] = fma((double)r[v].w, b.y, part[3]);
        }
      }
      double dot = (part[0] + part[1]) + (part[2] + part[3]);
#pragma unroll
      for (int offset = 16; offset > 0; offset >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, offset);
      if (lane == 0) red[i & 1][warp] = dot;
    }
    // one barrier per row: the block's dot product is complete and every thread holds its slice of
    // the row in registers, so the slot can take the row `slots` further on
    if (__syncthreads_or(!ready)) {
      stalled = i;
      break;
    }
    if (i + slots < n) {
      if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        ring_copy(full + slot, ring_rows + (size_t)slot * C, rows0 + (size_t)(i + slots) * C, row_bytes, policy);
      }
      issued = i + slots + 1;
    }
    double q = given_q;
    if (given == nullptr) {
      double dot = 0.0;
#pragma unroll
      for (int j = 0; j < kPassThreads / 32; ++j) dot += red[i & 1][j];
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
  if (stalled >= 0) {
    // a copy did not complete within the wait limit: wait (bounded) for the copies still in flight
    // into this block's shared memory, mark the step and leave NaN in this block's partial
    if (threadIdx.x == 0) {
      for (int j = stalled; j < issued; ++j) wait_row(j);
      atomicExch(&state->error, 1);
    }
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v][0] = acc[v][1] = acc[v][2] = acc[v][3] = nan;
  }
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    const int idx = threadIdx.x + v * kPassThreads;
    if (idx < C4) {
      double2* pair = reinterpret_cast<double2*>(out + 4 * idx);
      pair[0] = make_double2(acc[v][0], acc[v][1]);
      pair[1] = make_double2(acc[v][2], acc[v][3]);
    }
  }
  __syncthreads();  // thread 0's waits for in-flight copies end before the block's shared memory is released
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

// u = (sum of the data partials) + spatial L v_t + temporal T^T T v, kReduceColumns elements (t, c)
// per block, the data partials of each summed by kReduceGroups threads (every kReduceGroups-th
// partial) and the group sums added in group order; with `dot_with` (v = p) and `s_vec`, the
// block's partials of p.u, s.u, u.u and s.s into dots[k * gridDim.x + block], k = 0 .. 3.
// `partial` may be null (regularizer only).
__global__ void __launch_bounds__(kReduceThreads) normal_reduce_kernel(
    const double* __restrict__ partial, int ctas_per_model, int T, int C, const double* __restrict__ v,
    const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_cell, const double* __restrict__ nbr_w2,
    double spatial, double temporal, const double* __restrict__ dot_with, const double* __restrict__ s_vec,
    double* __restrict__ u, double* __restrict__ dots, const CglsState* __restrict__ state) {
  adt::chain_wait();
  if (state != nullptr && state->done) return;
  __shared__ double group_sum[kReduceGroups - 1][kReduceColumns];
  __shared__ double shared[kDots][kReduceColumns / 32];
  const int64_t n = (int64_t)T * C;
  const int column = threadIdx.x % kReduceColumns, group = threadIdx.x / kReduceColumns;
  const int64_t i = (int64_t)blockIdx.x * kReduceColumns + column;
  const int t = i < n ? (int)(i / C) : 0, c = i < n ? (int)(i % C) : 0;
  double sum = 0.0;
  if (partial != nullptr && i < n)
    for (int k = group; k < ctas_per_model; k += kReduceGroups)
      sum += partial[((size_t)t * ctas_per_model + k) * C + c];
  if (group > 0) group_sum[group - 1][column] = sum;
  __syncthreads();
  if (group > 0) return;
#pragma unroll
  for (int g = 0; g < kReduceGroups - 1; ++g) sum += group_sum[g][column];
  double product[kDots] = {0.0, 0.0, 0.0, 0.0};
  if (i < n) {
    const double* vt = v + (size_t)t * C;
    const double vc = vt[c];
    double lap = 0.0;
    for (int j = nbr_ptr[c]; j < nbr_ptr[c + 1]; ++j) lap += nbr_w2[j] * (vc - vt[nbr_cell[j]]);
    double tt = 0.0;
    if (t > 0) tt += vc - v[i - C];
    if (t < T - 1) tt += vc - v[i + C];
    const double value = sum + spatial * lap + temporal * tt;
    u[i] = value;
    if (dot_with != nullptr) {
      const double si = s_vec[i];
      product[0] = dot_with[i] * value;
      product[1] = si * value;
      product[2] = value * value;
      product[3] = si * si;
    }
  }
  if (dot_with != nullptr) {  // the first kReduceColumns threads (the other groups have left): named barrier
#pragma unroll
    for (int k = 0; k < kDots; ++k) {
#pragma unroll
      for (int offset = 16; offset > 0; offset >>= 1) product[k] += __shfl_xor_sync(0xffffffffu, product[k], offset);
      if ((threadIdx.x & 31) == 0) shared[k][threadIdx.x >> 5] = product[k];
    }
    asm volatile("bar.sync 1, %0;\n" ::"n"(kReduceColumns) : "memory");
    if (threadIdx.x < kDots) {
      double total = 0.0;
#pragma unroll
      for (int w = 0; w < kReduceColumns / 32; ++w) total += shared[threadIdx.x][w];
      dots[threadIdx.x * gridDim.x + blockIdx.x] = total;
    }
  }
}

// x = 0, s = p = A^T b (in u), gamma = gamma_0 = s.s.
__global__ void __launch_bounds__(kStartThreads) cgls_start_kernel(CglsState* st, int64_t n, const double* __restrict__ u,
                                                                   double* __restrict__ x, double* __restrict__ s,
                                                                   double* __restrict__ p) {
  adt::chain_wait();
  __shared__ double shared[kStartThreads / 32];
  double ss = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kStartThreads) {
    const double value = u[i];
    x[i] = 0.0;
    s[i] = value;
    p[i] = value;
    ss += value * value;
  }
  const double gamma = block_sum<kStartThreads>(ss, shared);
  if (threadIdx.x == 0) {
    st->gamma[0] = gamma;
    st->gamma0 = gamma;
    st->done = gamma > 0.0 ? 0 : 1;  // 1: iteration 0 must not run
    st->iterations = 0;
  }
}

// Iteration `it`: gamma = s.s, alpha = gamma / p.u, gamma' = s.s - 2 alpha s.u + alpha^2 u.u
// (every block sums the reduce partials in the same order), x += alpha p, s -= alpha u; unless
// the stop test holds (gamma' / gamma_0 < tolerance, or gamma' <= 0), p = s + (gamma' / gamma) p.
// p.u <= 0 stops before the update, as the reference's `denominator <= 0` does.
__global__ void __launch_bounds__(kUpdateThreads) cgls_update_kernel(CglsState* st, int it, int64_t n,
                                                                     const double* __restrict__ dots, int dot_count,
                                                                     double* __restrict__ x, double* __restrict__ s,
                                                                     double* __restrict__ p,
                                                                     const double* __restrict__ u, double tolerance) {
  adt::chain_wait();
  const int done = st->done;
  if (done != 0 && done - 1 <= it) return;  // an earlier iteration stopped
  __shared__ double totals[kDots];
  // warp k sums the partials of product k in one fixed order (lane l adds partials l, l + 32, ...,
  // then a butterfly), the same in every block
  if (threadIdx.x < 32 * kDots) {
    const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
    const double* values = dots + (size_t)k * dot_count;
    double v = 0.0;
    for (int j = lane; j < dot_count; j += 32) v += values[j];
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_xor_sync(0xffffffffu, v, offset);
    if (lane == 0) totals[k] = v;
  }
  __syncthreads();
  const double pu = totals[0], su = totals[1], uu = totals[2], gamma = totals[3];
  if (!(pu > 0.0)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st->done = it + 1;
    return;
  }
  const double alpha = gamma / pu;
  const double gamma_new = gamma - 2.0 * alpha * su + alpha * alpha * uu;
  const bool stop = !(gamma_new > 0.0) || gamma_new / st->gamma0 < tolerance;
  const double beta = gamma_new / gamma;
  const int64_t i = (int64_t)blockIdx.x * kUpdateThreads + threadIdx.x;
  if (i < n) {
    x[i] += alpha * p[i];
    const double si = s[i] - alpha * u[i];
    s[i] = si;
    if (!stop) p[i] = si + beta * p[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iterations += 1;
    st->gamma[it & 1] = gamma_new;
    if (stop) st->done = it + 2;
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

template <int VEC>
void launch_ring(const float* J, int T, int D, int C, const double* weights, const double* vec, const double* given,
                 const Workspace& w, int slots, cudaStream_t s) {
  static bool raised = false;
  if (!raised) {
    cudaFuncSetAttribute(normal_ring_kernel<VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRingSmemLimit);
    raised = true;
  }
  const size_t model_bytes = (size_t)D * C * sizeof(float);
  const int resident = (int)std::min<size_t>((size_t)T, kL2ResidentBytes / model_bytes);
  adt::launch_chained(normal_ring_kernel<VEC>, dim3(T * w.ctas_per_model), dim3(kPassThreads),
                      ring_layout(C, slots).total, s, J, D, C, weights, vec, given, w.ctas_per_model, w.partial,
                      w.state, resident, slots);
}

// One pass over J: A^T b (given = b_data, `iteration` false) or the product of a CGLS iteration.
bool data_pass(const adt_plan* p, const float* J, int T, int D, int C, const double* weights, const double* vec,
               const double* given, const Workspace& w, bool iteration, cudaStream_t s) {
  const int vec_per_thread = std::max(1, ((C >> 2) + kPassThreads - 1) / kPassThreads);
  const int slots = p->cgls_ring ? ring_slots(C) : 0;
  if (slots > 0) {
    switch (vec_per_thread) {
      case 1: launch_ring<1>(J, T, D, C, weights, vec, given, w, slots, s); return true;
      case 2: launch_ring<2>(J, T, D, C, weights, vec, given, w, slots, s); return true;
      case 3: launch_ring<3>(J, T, D, C, weights, vec, given, w, slots, s); return true;
      case 4: launch_ring<4>(J, T, D, C, weights, vec, given, w, slots, s); return true;
      case 5: launch_ring<5>(J, T, D, C, weights, vec, given, w, slots, s); return true;
      case 6: launch_ring<6>(J, T, D, C, weights, vec, given, w, slots, s); return true;
      default: break;  // p_t and the ring above the shared-memory limit: the register pass below
    }
  }
  const CglsState* state = iteration ? w.state : nullptr;
  switch (vec_per_thread) {
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
  cudaMemsetAsync(w.state, 0, sizeof(CglsState), s);
  data_pass(p, jacobian, steps, rows, columns, data_weights, w.p, data_rhs, w, false, s);
  adt::launch_chained(normal_reduce_kernel, dim3(w.reduce_blocks), dim3(kReduceThreads), 0, s, (const double*)w.partial,
                      w.ctas_per_model, (int)steps, (int)columns, models, neighbour_ptr, neighbour_cells,
                      neighbour_weights, -spatial, -temporal, (const double*)nullptr, (const double*)nullptr, w.u,
                      w.dots, (const CglsState*)nullptr);
  adt::launch_chained(cgls_start_kernel, dim3(1), dim3(kStartThreads), 0, s, w.state, n, (const double*)w.u, step,
                      w.s, w.p);
  p->launches += 3;
  for (int it = 0; it < iterations; ++it) {
    data_pass(p, jacobian, steps, rows, columns, data_weights, w.p, nullptr, w, true, s);
    adt::launch_chained(normal_reduce_kernel, dim3(w.reduce_blocks), dim3(kReduceThreads), 0, s,
                        (const double*)w.partial, w.ctas_per_model, (int)steps, (int)columns, (const double*)w.p,
                        neighbour_ptr, neighbour_cells, neighbour_weights, spatial, temporal, (const double*)w.p,
                        (const double*)w.s, w.u, w.dots, (const CglsState*)w.state);
    adt::launch_chained(cgls_update_kernel, dim3(w.update_blocks), dim3(kUpdateThreads), 0, s, w.state, it, n,
                        (const double*)w.dots, w.reduce_blocks, step, w.s, w.p, (const double*)w.u, tolerance);
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
  adt::launch_chained(normal_reduce_kernel, dim3((unsigned)reduce_grid(n)), dim3(kReduceThreads), 0,
                      (cudaStream_t)stream, (const double*)nullptr, 0, (int)steps, (int)columns, models, neighbour_ptr, neighbour_cells, neighbour_weights, spatial, temporal,
                      (const double*)nullptr, (const double*)nullptr, out, (double*)nullptr, (const CglsState*)nullptr);
  p->launches += 1;
  return adt::check_launch(p, "gauss-newton regularizer");
}
