// Batched sparse direct solver: block cyclic reduction over level-set blocks (float64).
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
//
// Dense block work runs on shared-memory tiles of MAXM rows (32, 48 or 64, chosen from the
// plan's widest level): Cholesky and triangular solves are blocked by 8 (the 8x8 diagonal part in
// registers, the rest as register-tiled updates), so a block of m rows needs about 3 m/8
// barriers instead of 2-3 per row.
#include "adt_internal.h"

namespace adt {
namespace {

constexpr int kB = 8;  // diagonal block of the blocked Cholesky / triangular solves

__device__ __forceinline__ double quiet_nan() { return __longlong_as_double(0x7ff8000000000000ULL); }

// C[i][j] += alpha * sum_p opA(i,p) opB(p,j) for i < m, j < n, p < k, where
// opA(i,p) = A_T ? A[p*lda+i] : A[i*lda+p] and opB(p,j) = B_T ? B[j*ldb+p] : B[p*ldb+j].
// Every operand tile is zero beyond its logical size up to a multiple of 4, so the 4x4
// micro-tiles (rows ti + r*mt, columns tj + s*nt: conflict-free, broadcast-friendly) read
// without bounds checks; only the stores are predicated.
template <bool A_T, bool B_T>
__device__ void tile_gemm(double* C, int ldc, const double* A, int lda, const double* B, int ldb,
                          int m, int n, int k, double alpha) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const int mt = (m + 3) >> 2, nt = (n + 3) >> 2;
  for (int t = threadIdx.x; t < mt * nt; t += blockDim.x) {
    const int ti = t / nt, tj = t - ti * nt;
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int s = 0; s < 4; ++s) acc[r][s] = 0.0;
    for (int p = 0; p < k; ++p) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = ti + r * mt;
        a[r] = A_T ? A[p * lda + i] : A[i * lda + p];
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int j = tj + s * nt;
        b[s] = B_T ? B[j * ldb + p] : B[p * ldb + j];
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int s = 0; s < 4; ++s) acc[r][s] = fma(a[r], b[s], acc[r][s]);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = ti + r * mt;
      if (i >= m) continue;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int j = tj + s * nt;
        if (j < n) C[i * ldc + j] += alpha * acc[r][s];
      }
    }
  }
}

template <int LD>
__device__ void zero(double* a, int rows) {
  for (int i = threadIdx.x; i < rows * LD; i += blockDim.x) a[i] = 0.0;
}

// In-place lower Cholesky of the m x m tile `a` (leading dimension LD, zero-padded). A
// non-positive pivot becomes NaN, which propagates to every result of the system.
template <int LD>
__device__ void cholesky(double* a, int m) {
  for (int kb = 0; kb < m; kb += kB) {
    const int nb = min(kB, m - kb);
    if (threadIdx.x < 32) {  // diagonal block in registers: lane r owns row r
      const int r = threadIdx.x;
      double row[kB];
#pragma unroll
      for (int c = 0; c < kB; ++c) row[c] = (r < nb && c <= r) ? a[(kb + r) * LD + kb + c] : 0.0;
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        if (k < nb) {
          const double pivot = __shfl_sync(0xffffffffu, row[k], k);
          const double d = pivot > 0.0 ? sqrt(pivot) : quiet_nan();
          if (r == k) row[k] = d;
          else if (r > k) row[k] /= d;
#pragma unroll
          for (int c = k + 1; c < kB; ++c) {
            const double lck = __shfl_sync(0xffffffffu, row[k], c);
            if (c < nb && r >= c) row[c] = fma(-row[k], lck, row[c]);
          }
        }
      }
      if (r < nb)
#pragma unroll
        for (int c = 0; c < kB; ++c)
          if (c <= r) a[(kb + r) * LD + kb + c] = row[c];
    }
    __syncthreads();
    // panel below the diagonal block: x L_bb^T = a_i for every row i
    for (int i = kb + nb + threadIdx.x; i < m; i += blockDim.x) {
      double x[kB];
#pragma unroll
      for (int c = 0; c < kB; ++c) {
        if (c < nb) {
          double v = a[i * LD + kb + c];
#pragma unroll
          for (int s = 0; s < c; ++s) v = fma(-x[s], a[(kb + c) * LD + kb + s], v);
          x[c] = v / a[(kb + c) * LD + kb + c];
          a[i * LD + kb + c] = x[c];
        }
      }
    }
    __syncthreads();
    const int rest = m - kb - nb;
    if (rest > 0) {
      double* panel = a + (kb + nb) * LD + kb;
      tile_gemm<false, true>(a + (kb + nb) * LD + kb + nb, LD, panel, LD, panel, LD, rest, rest, nb, -1.0);
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    const int i = idx / m, j = idx - i * m;
    if (j > i) a[i * LD + j] = 0.0;
  }
  __syncthreads();
}

// Solve L X = B in place (L: m x m lower, leading dimension LDL; B: m x n, leading dimension LDB).
template <int LDL, int LDB>
__device__ void lower_solve(const double* l, double* b, int m, int n) {
  for (int kb = 0; kb < m; kb += kB) {
    const int nb = min(kB, m - kb);
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      double x[kB];
#pragma unroll
      for (int r = 0; r < kB; ++r) {
        if (r < nb) {
          double v = b[(kb + r) * LDB + c];
#pragma unroll
          for (int s = 0; s < r; ++s) v = fma(-l[(kb + r) * LDL + kb + s], x[s], v);
          x[r] = v / l[(kb + r) * LDL + kb + r];
          b[(kb + r) * LDB + c] = x[r];
        }
      }
    }
    __syncthreads();
    const int rest = m - kb - nb;
    if (rest > 0)
      tile_gemm<false, false>(b + (kb + nb) * LDB, LDB, l + (kb + nb) * LDL + kb, LDL, b + kb * LDB, LDB,
                              rest, n, nb, -1.0);
    __syncthreads();
  }
}

// Solve L^T X = B in place.
template <int LDL, int LDB>
__device__ void upper_solve(const double* l, double* b, int m, int n) {
  const int last = ((m - 1) / kB) * kB;
  for (int kb = last; kb >= 0; kb -= kB) {
    const int nb = min(kB, m - kb);
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      double x[kB];
#pragma unroll
      for (int r = kB - 1; r >= 0; --r) {
        if (r < nb) {
          double v = b[(kb + r) * LDB + c];
#pragma unroll
          for (int s = r + 1; s < kB; ++s)
            if (s < nb) v = fma(-l[(kb + s) * LDL + kb + r], x[s], v);
          x[r] = v / l[(kb + r) * LDL + kb + r];
          b[(kb + r) * LDB + c] = x[r];
        }
      }
    }
    __syncthreads();
    if (kb > 0)
      tile_gemm<true, false>(b, LDB, l + kb * LDL, LDL, b + kb * LDB, LDB, kb, n, nb, -1.0);
    __syncthreads();
  }
}

template <int LD>
__device__ void load_tile(double* dst, const double* src, int rows, int cols) {
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    const int r = i / cols, c = i - r * cols;
    dst[r * LD + c] = src[i];
  }
}

template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, MAXM <= 48 ? 3 : 1)
factor_level_kernel(const int64_t* __restrict__ tasks, const int64_t* __restrict__ pulls,
                    int task_begin, const int* __restrict__ csr_ptr,
                    const int* __restrict__ csr_row, const int* __restrict__ csr_col, int nnz,
                    const double* __restrict__ values, double* __restrict__ factors,
                    int64_t stride) {
  constexpr int LD = MAXM + 1, LDB = 2 * MAXM + 1;
  extern __shared__ double sm[];
  double* dm = sm;                 // D_j -> L_j                       (MAXM x LD)
  double* bt = dm + MAXM * LD;     // [A[j,p] | A[q,j]^T] -> [U_p | V_q^T]  (MAXM x LDB)
  double* ws = bt + MAXM * LDB;    // pull staging / fill              (MAXM x LD)
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* val = values + (int64_t)blockIdx.y * nnz;
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  const int p = (int)t[T_P], mp = p >= 0 ? (int)t[T_MP] : 0, offp = (int)t[T_OFFP];
  const int q = (int)t[T_Q], mq = q >= 0 ? (int)t[T_MQ] : 0, offq = (int)t[T_OFFQ];
  const bool p_csr = p >= 0 && t[T_LINKP] < 0, q_csr = q >= 0 && t[T_LINKQ] < 0;

  zero<LD>(dm, MAXM);
  zero<LDB>(bt, MAXM);
  __syncthreads();
  // original couplings of block j's rows, straight from the assembled CSR values
  const int s0 = csr_ptr[offj], s1 = csr_ptr[offj + mj];
  for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
    const int r = csr_row[s] - offj, c = csr_col[s];
    const double v = val[s];
    if (c >= offj && c < offj + mj) dm[r * LD + (c - offj)] = v;
    else if (p_csr && c >= offp && c < offp + mp) bt[r * LDB + (c - offp)] = v;
    else if (q_csr && c >= offq && c < offq + mq) bt[r * LDB + mp + (c - offq)] = v;
  }
  if (p >= 0 && !p_csr) {  // A[j,p] (mj x mp) from the previous level's fill
    const double* src = f + t[T_LINKP];
    for (int i = threadIdx.x; i < mj * mp; i += blockDim.x) {
      const int r = i / mp, c = i - r * mp;
      bt[r * LDB + c] = src[i];
    }
  }
  if (q >= 0 && !q_csr) {  // A[q,j] (mq x mj), stored transposed next to A[j,p]
    const double* src = f + t[T_LINKQ];
    for (int i = threadIdx.x; i < mq * mj; i += blockDim.x) {
      const int r = i / mj, k = i - r * mj;
      bt[k * LDB + mp + r] = src[i];
    }
  }
  __syncthreads();

  // Schur-complement updates from blocks eliminated next to j at earlier levels
  for (int64_t u = t[T_PULL0]; u < t[T_PULL1]; ++u) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int type = (int)pl[P_TYPE], me = (int)pl[P_ME];
    zero<LD>(ws, MAXM);
    __syncthreads();
    if (type == 0) load_tile<LD>(ws, f + pl[P_OFF], me, mj);  // U (me x mj): D -= U^T U
    else load_tile<LD>(ws, f + pl[P_OFF], mj, me);            // V (mj x me): D -= V V^T
    __syncthreads();
    if (type == 0) tile_gemm<true, false>(dm, LD, ws, LD, ws, LD, mj, mj, me, -1.0);
    else tile_gemm<false, true>(dm, LD, ws, LD, ws, LD, mj, mj, me, -1.0);
    __syncthreads();
  }
  cholesky<LD>(dm, mj);
  {
    double* out = f + t[T_LOFF];
    for (int i = threadIdx.x; i < mj * mj; i += blockDim.x) {
      const int r = i / mj, c = i - r * mj;
      out[i] = dm[r * LD + c];
    }
  }
  if (mp + mq > 0) {
    lower_solve<LD, LDB>(dm, bt, mj, mp + mq);  // [U_p | V_q^T]
    double* up = f + t[T_UOFF];
    for (int i = threadIdx.x; i < mj * mp; i += blockDim.x) {
      const int r = i / mp, c = i - r * mp;
      up[i] = bt[r * LDB + c];
    }
    if (q >= 0) {
      double* vq = f + t[T_VOFF];
      for (int i = threadIdx.x; i < mq * mj; i += blockDim.x) {
        const int r = i / mj, k = i - r * mj;
        vq[i] = bt[k * LDB + mp + r];
      }
    }
    if (p >= 0 && q >= 0) {  // fill A[q,p] = -V_q U_p = -(V_q^T)^T U_p
      zero<LD>(ws, MAXM);
      __syncthreads();
      tile_gemm<true, false>(ws, LD, bt + mp, LDB, bt, LDB, mq, mp, mj, -1.0);
      __syncthreads();
      double* out = f + t[T_FILL];
      for (int i = threadIdx.x; i < mq * mp; i += blockDim.x) {
        const int r = i / mp, c = i - r * mp;
        out[i] = ws[r * LD + c];
      }
    }
  }
}

// Forward level: y_j = L_j^-1 (b_j - pulls); the root also back-substitutes.
template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, MAXM <= 48 ? 3 : 1)
forward_level_kernel(const int64_t* __restrict__ tasks, const int64_t* __restrict__ pulls,
                     int task_begin, const double* __restrict__ factors, int64_t stride,
                     double* __restrict__ rhs, int64_t rhs_stride, int nrhs, int root) {
  constexpr int LD = MAXM + 1;
  extern __shared__ double sm[];
  double* lt = sm;
  double* bt = lt + MAXM * LD;
  double* mt = bt + MAXM * LD;
  double* yt = mt + MAXM * LD;
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * MAXM;
  const int nc = min(MAXM, nrhs - c0);
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];

  zero<LD>(bt, MAXM);
  zero<LD>(lt, MAXM);
  __syncthreads();
  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i - r * nc;
    bt[r * LD + c] = x[(int64_t)(offj + r) * nrhs + c0 + c];
  }
  for (int64_t u = t[T_PULL0]; u < t[T_PULL1]; ++u) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int type = (int)pl[P_TYPE], me = (int)pl[P_ME], eoff = (int)pl[P_EOFF];
    zero<LD>(mt, MAXM);
    zero<LD>(yt, MAXM);
    __syncthreads();
    if (type == 0) load_tile<LD>(mt, f + pl[P_OFF], me, mj);
    else load_tile<LD>(mt, f + pl[P_OFF], mj, me);
    for (int i = threadIdx.x; i < me * nc; i += blockDim.x) {
      const int r = i / nc, c = i - r * nc;
      yt[r * LD + c] = x[(int64_t)(eoff + r) * nrhs + c0 + c];
    }
    __syncthreads();
    if (type == 0) tile_gemm<true, false>(bt, LD, mt, LD, yt, LD, mj, nc, me, -1.0);
    else tile_gemm<false, false>(bt, LD, mt, LD, yt, LD, mj, nc, me, -1.0);
    __syncthreads();
  }
  load_tile<LD>(lt, f + t[T_LOFF], mj, mj);
  __syncthreads();
  lower_solve<LD, LD>(lt, bt, mj, nc);
  if (root) upper_solve<LD, LD>(lt, bt, mj, nc);
  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i - r * nc;
    x[(int64_t)(offj + r) * nrhs + c0 + c] = bt[r * LD + c];
  }
}

// Backward level: x_j = L_j^-T (y_j - U_p x_p - V_q^T x_q).
template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, MAXM <= 48 ? 3 : 1)
backward_level_kernel(const int64_t* __restrict__ tasks, int task_begin,
                      const double* __restrict__ factors, int64_t stride,
                      double* __restrict__ rhs, int64_t rhs_stride, int nrhs) {
  constexpr int LD = MAXM + 1;
  extern __shared__ double sm[];
  double* lt = sm;
  double* bt = lt + MAXM * LD;
  double* mt = bt + MAXM * LD;
  double* yt = mt + MAXM * LD;
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * MAXM;
  const int nc = min(MAXM, nrhs - c0);
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];

  zero<LD>(bt, MAXM);
  zero<LD>(lt, MAXM);
  __syncthreads();
  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i - r * nc;
    bt[r * LD + c] = x[(int64_t)(offj + r) * nrhs + c0 + c];
  }
  for (int side = 0; side < 2; ++side) {
    const int nb = side == 0 ? (int)t[T_P] : (int)t[T_Q];
    if (nb < 0) continue;
    const int me = side == 0 ? (int)t[T_MP] : (int)t[T_MQ];
    const int eoff = side == 0 ? (int)t[T_OFFP] : (int)t[T_OFFQ];
    zero<LD>(mt, MAXM);
    zero<LD>(yt, MAXM);
    __syncthreads();
    if (side == 0) load_tile<LD>(mt, f + t[T_UOFF], mj, me);  // U_p (mj x mp)
    else load_tile<LD>(mt, f + t[T_VOFF], me, mj);            // V_q (mq x mj)
    for (int i = threadIdx.x; i < me * nc; i += blockDim.x) {
      const int r = i / nc, c = i - r * nc;
      yt[r * LD + c] = x[(int64_t)(eoff + r) * nrhs + c0 + c];
    }
    __syncthreads();
    if (side == 0) tile_gemm<false, false>(bt, LD, mt, LD, yt, LD, mj, nc, me, -1.0);
    else tile_gemm<true, false>(bt, LD, mt, LD, yt, LD, mj, nc, me, -1.0);
    __syncthreads();
  }
  load_tile<LD>(lt, f + t[T_LOFF], mj, mj);
  __syncthreads();
  upper_solve<LD, LD>(lt, bt, mj, nc);
  for (int i = threadIdx.x; i < mj * nc; i += blockDim.x) {
    const int r = i / nc, c = i - r * nc;
    x[(int64_t)(offj + r) * nrhs + c0 + c] = bt[r * LD + c];
  }
}

template <int MAXM>
constexpr size_t factor_smem() { return sizeof(double) * ((size_t)MAXM * (MAXM + 1) * 2 + (size_t)MAXM * (2 * MAXM + 1)); }
template <int MAXM>
constexpr size_t solve_smem() { return sizeof(double) * 4 * (size_t)MAXM * (MAXM + 1); }

template <int MAXM>
void configure() {
  cudaFuncSetAttribute(factor_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)factor_smem<MAXM>());
  cudaFuncSetAttribute(forward_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<MAXM>());
  cudaFuncSetAttribute(backward_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem<MAXM>());
}

template <int MAXM>
void factor_levels(adt_plan* p, int systems, const double* values, double* factors, cudaStream_t s) {
  for (int level = 0; level < p->levels; ++level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    dim3 grid(t1 - t0, systems);
    factor_level_kernel<MAXM><<<grid, kSolverThreads, factor_smem<MAXM>(), s>>>(
        p->tasks, p->pulls, t0, p->csr_ptr, p->csr_row, p->csr_col, p->nnz, values, factors,
        p->factor_stride);
    p->launches++;
  }
}

template <int MAXM>
void solve_levels(adt_plan* p, int systems, int nrhs, const double* factors, double* rhs, cudaStream_t s) {
  const int64_t rhs_stride = (int64_t)p->N * nrhs;
  const int tiles = (nrhs + MAXM - 1) / MAXM;
  for (int level = 0; level < p->levels; ++level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    dim3 grid(t1 - t0, systems, tiles);
    forward_level_kernel<MAXM><<<grid, kSolverThreads, solve_smem<MAXM>(), s>>>(
        p->tasks, p->pulls, t0, factors, p->factor_stride, rhs, rhs_stride, nrhs, level == p->levels - 1);
    p->launches++;
  }
  for (int level = p->levels - 2; level >= 0; --level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    dim3 grid(t1 - t0, systems, tiles);
    backward_level_kernel<MAXM><<<grid, kSolverThreads, solve_smem<MAXM>(), s>>>(
        p->tasks, t0, factors, p->factor_stride, rhs, rhs_stride, nrhs);
    p->launches++;
  }
}

}  // namespace

// Opt the solver kernels in to their dynamic shared memory on the current device.
void configure_solver_kernels() {
  configure<32>();
  configure<48>();
  configure<64>();
}

adt_status factorize_systems(adt_plan* p, int systems, const double* values, double* factors,
                             cudaStream_t s) {
  if (p->max_m <= 32) factor_levels<32>(p, systems, values, factors, s);
  else if (p->max_m <= 48) factor_levels<48>(p, systems, values, factors, s);
  else factor_levels<64>(p, systems, values, factors, s);
  return check_launch(p, "factorization");
}

adt_status solve_systems(adt_plan* p, int systems, int nrhs, const double* factors,
                         double* rhs, cudaStream_t s) {
  if (p->max_m <= 32) solve_levels<32>(p, systems, nrhs, factors, rhs, s);
  else if (p->max_m <= 48) solve_levels<48>(p, systems, nrhs, factors, rhs, s);
  else solve_levels<64>(p, systems, nrhs, factors, rhs, s);
  return check_launch(p, "solve");
}

}  // namespace adt
