// Batched sparse direct solver: block cyclic reduction over level-set blocks.
//
// The plan orders the dofs in breadth-first level sets, so every operator is block tridiagonal
// (a level only couples to its neighbours). Eliminating the odd blocks of the chain, then the
// odd blocks of the surviving chain, and so on, is a block Cholesky factorization in a nested
// (odd-even) order: every level is one launch in which all eliminated blocks of all systems
// factor in parallel. An eliminated block "pulls" the Schur-complement updates of the blocks
// eliminated next to it at earlier levels, so a level needs no second update pass and every
// reduction has a fixed order (bitwise repeatable).
//
// Storage of one system (doubles): L_j for every block, and per elimination of j with chain
// neighbours p (left) and q (right): U_p = L_j^-1 A[j,p] (m_j x m_p), V_q = A[q,j] L_j^-T
// (m_q x m_j) and the fill A[q,p] = -V_q U_p (m_q x m_p) consumed at the next level.
// Forward: y_j = L_j^-1 (b_j - sum pulls); backward: x_j = L_j^-T (y_j - U_p x_p - V_q^T x_q).
#include "adt_internal.h"

namespace adt {
namespace {

constexpr int kLd = kMaxBlock + 1;  // shared-memory leading dimension (odd: no bank conflicts)

__device__ __forceinline__ void zero_tile(double* a, int rows, int cols) {
  for (int i = threadIdx.x; i < rows * kLd; i += blockDim.x) a[i] = 0.0;
}

__device__ __forceinline__ void load_tile(double* dst, const double* src, int rows, int cols) {
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    const int r = i / cols, c = i - r * cols;
    dst[r * kLd + c] = src[i];
  }
}

__device__ __forceinline__ void store_tile(double* dst, const double* src, int rows, int cols) {
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    const int r = i / cols, c = i - r * cols;
    dst[i] = src[r * kLd + c];
  }
}

// In-place lower Cholesky of an m x m tile; non-positive pivots become NaN so the failure
// propagates to every result of the system (the host reports non-finite output).
__device__ void cholesky_tile(double* a, int m) {
  const int tid = threadIdx.x;
  for (int k = 0; k < m; ++k) {
    if (tid == 0) {
      const double d = a[k * kLd + k];
      a[k * kLd + k] = d > 0.0 ? sqrt(d) : __longlong_as_double(0x7ff8000000000000ULL);
    }
    __syncthreads();
    const double inv = 1.0 / a[k * kLd + k];
    for (int i = k + 1 + tid; i < m; i += blockDim.x) a[i * kLd + k] *= inv;
    __syncthreads();
    const int n = m - k - 1;
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
      const int i = k + 1 + idx / n, j = k + 1 + idx % n;
      if (j <= i) a[i * kLd + j] -= a[i * kLd + k] * a[j * kLd + k];
    }
    __syncthreads();
  }
  for (int idx = tid; idx < m * m; idx += blockDim.x) {
    const int i = idx / m, j = idx % m;
    if (j > i) a[i * kLd + j] = 0.0;
  }
  __syncthreads();
}

// Solve L X = B in place (L m x m lower, B m x n), columns in parallel.
__device__ void lower_solve_tile(const double* l, double* b, int m, int n) {
  for (int k = 0; k < m; ++k) {
    const double inv = 1.0 / l[k * kLd + k];
    for (int c = threadIdx.x; c < n; c += blockDim.x) b[k * kLd + c] *= inv;
    __syncthreads();
    const int rows = m - k - 1;
    for (int idx = threadIdx.x; idx < rows * n; idx += blockDim.x) {
      const int i = k + 1 + idx / n, c = idx % n;
      b[i * kLd + c] -= l[i * kLd + k] * b[k * kLd + c];
    }
    __syncthreads();
  }
}

// Solve L^T X = B in place.
__device__ void upper_solve_tile(const double* l, double* b, int m, int n) {
  for (int k = m - 1; k >= 0; --k) {
    const double inv = 1.0 / l[k * kLd + k];
    for (int c = threadIdx.x; c < n; c += blockDim.x) b[k * kLd + c] *= inv;
    __syncthreads();
    for (int idx = threadIdx.x; idx < k * n; idx += blockDim.x) {
      const int i = idx / n, c = idx % n;
      b[i * kLd + c] -= l[k * kLd + i] * b[k * kLd + c];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSolverThreads)
factor_level_kernel(const int64_t* __restrict__ tasks, const int64_t* __restrict__ pulls,
                    int task_begin, const int* __restrict__ csr_ptr,
                    const int* __restrict__ csr_row, const int* __restrict__ csr_col, int nnz,
                    const double* __restrict__ values, double* __restrict__ factors,
                    int64_t stride) {
  extern __shared__ double sm[];
  double* dm = sm;                    // D_j -> L_j
  double* ap = dm + kMaxBlock * kLd;  // A[j,p] -> U_p
  double* aq = ap + kMaxBlock * kLd;  // A[q,j] -> V_q
  double* ws = aq + kMaxBlock * kLd;  // pull staging / fill
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* val = values + (int64_t)blockIdx.y * nnz;
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  const int p = (int)t[T_P], mp = (int)t[T_MP], offp = (int)t[T_OFFP];
  const int q = (int)t[T_Q], mq = (int)t[T_MQ], offq = (int)t[T_OFFQ];
  const bool p_csr = p >= 0 && t[T_LINKP] < 0, q_csr = q >= 0 && t[T_LINKQ] < 0;

  zero_tile(dm, mj, mj);
  if (p >= 0) zero_tile(ap, mj, mp);
  if (q >= 0) zero_tile(aq, mq, mj);
  __syncthreads();
  // Original couplings of block j's rows, straight from the assembled CSR values.
  const int s0 = csr_ptr[offj], s1 = csr_ptr[offj + mj];
  for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
    const int r = csr_row[s] - offj, c = csr_col[s];
    const double v = val[s];
    if (c >= offj && c < offj + mj) dm[r * kLd + (c - offj)] = v;
    else if (p_csr && c >= offp && c < offp + mp) ap[r * kLd + (c - offp)] = v;
    else if (q_csr && c >= offq && c < offq + mq) aq[(c - offq) * kLd + r] = v;
  }
  if (p >= 0 && !p_csr) load_tile(ap, f + t[T_LINKP], mj, mp);
  if (q >= 0 && !q_csr) load_tile(aq, f + t[T_LINKQ], mq, mj);
  __syncthreads();

  // Schur-complement updates from blocks eliminated next to j at earlier levels.
  for (int64_t u = t[T_PULL0]; u < t[T_PULL1]; ++u) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int type = (int)pl[P_TYPE], me = (int)pl[P_ME];
    if (type == 0) load_tile(ws, f + pl[P_OFF], me, mj);  // U (me x mj): D -= U^T U
    else load_tile(ws, f + pl[P_OFF], mj, me);            // V (mj x me): D -= V V^T
    __syncthreads();
    for (int idx = threadIdx.x; idx < mj * mj; idx += blockDim.x) {
      const int r = idx / mj, c = idx % mj;
      if (c > r) continue;
      double acc = 0.0;
      if (type == 0)
        for (int k = 0; k < me; ++k) acc += ws[k * kLd + r] * ws[k * kLd + c];
      else
        for (int k = 0; k < me; ++k) acc += ws[r * kLd + k] * ws[c * kLd + k];
      dm[r * kLd + c] -= acc;
    }
    __syncthreads();
  }
  cholesky_tile(dm, mj);
  store_tile(f + t[T_LOFF], dm, mj, mj);

  if (p >= 0) {  // U_p = L^-1 A[j,p]
    lower_solve_tile(dm, ap, mj, mp);
    store_tile(f + t[T_UOFF], ap, mj, mp);
  }
  if (q >= 0) {  // V_q = A[q,j] L^-T, row r: solve L v = a_r
    for (int r = threadIdx.x; r < mq; r += blockDim.x) {
      double* v = aq + r * kLd;
      for (int k = 0; k < mj; ++k) {
        double acc = v[k];
        for (int i = 0; i < k; ++i) acc -= v[i] * dm[k * kLd + i];
        v[k] = acc / dm[k * kLd + k];
      }
    }
    __syncthreads();
    store_tile(f + t[T_VOFF], aq, mq, mj);
  }
  if (p >= 0 && q >= 0) {  // fill A[q,p] = -V_q U_p
    double* out = f + t[T_FILL];
    for (int idx = threadIdx.x; idx < mq * mp; idx += blockDim.x) {
      const int r = idx / mp, c = idx % mp;
      double acc = 0.0;
      for (int k = 0; k < mj; ++k) acc += aq[r * kLd + k] * ap[k * kLd + c];
      out[idx] = -acc;
    }
  }
}

// Forward level: y_j = L_j^-1 (b_j - pulls); the root also back-substitutes.
__global__ void __launch_bounds__(kSolverThreads)
forward_level_kernel(const int64_t* __restrict__ tasks, const int64_t* __restrict__ pulls,
                     int task_begin, const double* __restrict__ factors, int64_t stride,
                     double* __restrict__ rhs, int64_t rhs_stride, int nrhs, int root) {
  extern __shared__ double sm[];
  double* lt = sm;
  double* bt = lt + kMaxBlock * kLd;
  double* mt = bt + kMaxBlock * kLd;
  double* yt = mt + kMaxBlock * kLd;
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * kMaxBlock;
  const int nc = min(kMaxBlock, nrhs - c0);
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];

  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i % nc;
    bt[r * kLd + c] = x[(int64_t)(offj + r) * nrhs + c0 + c];
  }
  for (int64_t u = t[T_PULL0]; u < t[T_PULL1]; ++u) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int type = (int)pl[P_TYPE], me = (int)pl[P_ME], eoff = (int)pl[P_EOFF];
    if (type == 0) load_tile(mt, f + pl[P_OFF], me, mj);
    else load_tile(mt, f + pl[P_OFF], mj, me);
    for (int i = threadIdx.x; i < me * nc; i += blockDim.x) {
      const int r = i / nc, c = i % nc;
      yt[r * kLd + c] = x[(int64_t)(eoff + r) * nrhs + c0 + c];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < mj * nc; idx += blockDim.x) {
      const int r = idx / nc, c = idx % nc;
      double acc = 0.0;
      if (type == 0)
        for (int k = 0; k < me; ++k) acc += mt[k * kLd + r] * yt[k * kLd + c];
      else
        for (int k = 0; k < me; ++k) acc += mt[r * kLd + k] * yt[k * kLd + c];
      bt[r * kLd + c] -= acc;
    }
    __syncthreads();
  }
  load_tile(lt, f + t[T_LOFF], mj, mj);
  __syncthreads();
  lower_solve_tile(lt, bt, mj, nc);
  if (root) upper_solve_tile(lt, bt, mj, nc);
  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i % nc;
    x[(int64_t)(offj + r) * nrhs + c0 + c] = bt[r * kLd + c];
  }
}

// Backward level: x_j = L_j^-T (y_j - U_p x_p - V_q^T x_q).
__global__ void __launch_bounds__(kSolverThreads)
backward_level_kernel(const int64_t* __restrict__ tasks, int task_begin,
                      const double* __restrict__ factors, int64_t stride,
                      double* __restrict__ rhs, int64_t rhs_stride, int nrhs) {
  extern __shared__ double sm[];
  double* lt = sm;
  double* bt = lt + kMaxBlock * kLd;
  double* mt = bt + kMaxBlock * kLd;
  double* yt = mt + kMaxBlock * kLd;
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * kMaxBlock;
  const int nc = min(kMaxBlock, nrhs - c0);
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];

  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i % nc;
    bt[r * kLd + c] = x[(int64_t)(offj + r) * nrhs + c0 + c];
  }
  for (int side = 0; side < 2; ++side) {
    const int nb = side == 0 ? (int)t[T_P] : (int)t[T_Q];
    if (nb < 0) continue;
    const int me = side == 0 ? (int)t[T_MP] : (int)t[T_MQ];
    const int eoff = side == 0 ? (int)t[T_OFFP] : (int)t[T_OFFQ];
    if (side == 0) load_tile(mt, f + t[T_UOFF], mj, me);  // U_p (mj x mp)
    else load_tile(mt, f + t[T_VOFF], me, mj);            // V_q (mq x mj)
    for (int i = threadIdx.x; i < me * nc; i += blockDim.x) {
      const int r = i / nc, c = i % nc;
      yt[r * kLd + c] = x[(int64_t)(eoff + r) * nrhs + c0 + c];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < mj * nc; idx += blockDim.x) {
      const int r = idx / nc, c = idx % nc;
      double acc = 0.0;
      if (side == 0)
        for (int k = 0; k < me; ++k) acc += mt[r * kLd + k] * yt[k * kLd + c];
      else
        for (int k = 0; k < me; ++k) acc += mt[k * kLd + r] * yt[k * kLd + c];
      bt[r * kLd + c] -= acc;
    }
    __syncthreads();
  }
  load_tile(lt, f + t[T_LOFF], mj, mj);
  __syncthreads();
  upper_solve_tile(lt, bt, mj, nc);
  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i % nc;
    x[(int64_t)(offj + r) * nrhs + c0 + c] = bt[r * kLd + c];
  }
}

constexpr size_t kSolverSmem = 4 * kMaxBlock * kLd * sizeof(double);

}  // namespace

// Opt the solver kernels in to their dynamic shared memory on the current device.
void configure_solver_kernels() {
  cudaFuncSetAttribute(factor_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kSolverSmem);
  cudaFuncSetAttribute(forward_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kSolverSmem);
  cudaFuncSetAttribute(backward_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kSolverSmem);
}

adt_status factorize_systems(adt_plan* p, int systems, const double* values, double* factors,
                             cudaStream_t s) {
  for (int level = 0; level < p->levels; ++level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    dim3 grid(t1 - t0, systems);
    factor_level_kernel<<<grid, kSolverThreads, kSolverSmem, s>>>(
        p->tasks, p->pulls, t0, p->csr_ptr, p->csr_row, p->csr_col, p->nnz, values, factors,
        p->factor_stride);
    p->launches++;
  }
  return check_launch(p, "factorization");
}

adt_status solve_systems(adt_plan* p, int systems, int nrhs, const double* factors,
                         double* rhs, cudaStream_t s) {
  const int64_t rhs_stride = (int64_t)p->N * nrhs;
  const int tiles = (nrhs + kMaxBlock - 1) / kMaxBlock;
  for (int level = 0; level < p->levels; ++level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    dim3 grid(t1 - t0, systems, tiles);
    forward_level_kernel<<<grid, kSolverThreads, kSolverSmem, s>>>(
        p->tasks, p->pulls, t0, factors, p->factor_stride, rhs, rhs_stride, nrhs,
        level == p->levels - 1);
    p->launches++;
  }
  for (int level = p->levels - 2; level >= 0; --level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    dim3 grid(t1 - t0, systems, tiles);
    backward_level_kernel<<<grid, kSolverThreads, kSolverSmem, s>>>(
        p->tasks, t0, factors, p->factor_stride, rhs, rhs_stride, nrhs);
    p->launches++;
  }
  return check_launch(p, "solve");
}

}  // namespace adt
