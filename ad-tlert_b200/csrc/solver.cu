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
// plan's widest level). The pulled updates of a block accumulate in per-thread 4x4 register
// tiles while the next pull's operands stream into shared memory with cp.async (one barrier per
// pull); Cholesky and triangular solves are blocked by 8 (the diagonal part in registers, the
// rest as register-tiled updates) and multiply by reciprocal diagonals.
#include <type_traits>

#include "adt_internal.h"

namespace adt {
namespace {

constexpr int kB = 8;  // diagonal block of the blocked Cholesky / triangular solves

__device__ __forceinline__ double quiet_nan() { return __longlong_as_double(0x7ff8000000000000ULL); }

// ---- asynchronous global -> shared copies (8-byte cp.async) --------------------------------
__device__ __forceinline__ void async_copy8(double* dst, const double* src) {
  const unsigned addr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(addr), "l"(src));
}
__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// f(r, c, i) for every entry i = r * cols + c of a rows x cols block that falls to this thread
// (i = threadIdx.x, threadIdx.x + blockDim.x, ...): the row and column advance by the stride's
// quotient and remainder, so a call divides twice instead of once per entry.
template <typename F>
__device__ __forceinline__ void for_each_entry(int rows, int cols, F&& f) {
  if (rows <= 0 || cols <= 0) return;
  const int stride = blockDim.x, dr = stride / cols, dc = stride - dr * cols;
  int r = threadIdx.x / cols, c = threadIdx.x - r * cols, i = threadIdx.x;
  while (r < rows) {
    f(r, c, i);
    i += stride;
    r += dr;
    c += dc;
    if (c >= cols) {
      c -= cols;
      ++r;
    }
  }
}

// rows x cols dense block at src -> tile with leading dimension ld
__device__ __forceinline__ void async_tile(double* dst, int ld, const double* src, int rows, int cols) {
  for_each_entry(rows, cols, [&](int r, int c, int i) { async_copy8(dst + r * ld + c, src + i); });
}

// rows x cols slice of a right-hand-side array (row stride `stride`) -> tile
__device__ __forceinline__ void async_rows(double* dst, int ld, const double* src, int64_t stride, int rows, int cols) {
  for_each_entry(rows, cols, [&](int r, int c, int) { async_copy8(dst + r * ld + c, src + r * stride + c); });
}

// ---- register-tiled products ---------------------------------------------------------------
// Output m x n is covered by 4x4 micro-tiles with rows ti + r*mt and columns tj + s*nt
// (conflict-free, broadcast-friendly shared-memory reads). Rows/columns past m/n read whatever
// the tile holds there and only feed accumulators that are never stored; the reduction index p
// is always exact.
struct Micro {
  int mt, nt, tile, part, nsplit, ti, tj;
  bool active;
  __device__ Micro(int m, int n) {
    mt = (m + 3) >> 2;
    nt = (n + 3) >> 2;
    const int tiles = mt * nt;
    nsplit = tiles <= (int)blockDim.x / 2 ? 2 : 1;  // small outputs: two threads split the reduction
    const int per = blockDim.x / nsplit;
    tile = threadIdx.x % per;
    part = threadIdx.x / per;
    active = tile < tiles;
    ti = active ? tile / nt : 0;
    tj = active ? tile - ti * nt : 0;
  }
};

template <bool A_T, bool B_T>
__device__ __forceinline__ void accumulate(double (&acc)[4][4], const Micro& u, const double* A, int lda,
                                           const double* B, int ldb, int k) {
  if (!u.active) return;
  for (int p = u.part; p < k; p += u.nsplit) {
    double a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = u.ti + r * u.mt;
      a[r] = A_T ? A[p * lda + i] : A[i * lda + p];
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int j = u.tj + s * u.nt;
      b[s] = B_T ? B[j * ldb + p] : B[p * ldb + j];
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int s = 0; s < 4; ++s) acc[r][s] = fma(a[r], b[s], acc[r][s]);
  }
}

// Combine the split halves (through `scratch`, >= 128 x 16 doubles) and subtract from C (m x n).
// Must be entered by all threads after the operands' last use; ends with a barrier.
__device__ void subtract_tile(double (&acc)[4][4], const Micro& u, double* C, int ldc, int m, int n,
                              double* scratch) {
  if (u.nsplit == 2) {
    if (u.part == 1 && u.active)
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int s = 0; s < 4; ++s) scratch[u.tile * 16 + r * 4 + s] = acc[r][s];
    __syncthreads();
  }
  if (u.part == 0 && u.active) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = u.ti + r * u.mt;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int j = u.tj + s * u.nt;
        double v = acc[r][s];
        if (u.nsplit == 2) v += scratch[u.tile * 16 + r * 4 + s];
        if (i < m && j < n) C[i * ldc + j] -= v;
      }
    }
  }
  __syncthreads();
}

// C[i][j] += alpha * sum_p opA(i,p) opB(p,j) for i < m, j < n, p < k (one call, no split).
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

// ---- FP64 tensor-core tiles (mma.sync m8n8k4 f64) for the fill GEMM of the level kernel.
// An m x n output is a grid of 8 x 8 tiles; warp w of the block owns tiles w, w + 8, w + 16, ...
// (row-major over the grid), at most MAXT of them, and lane (g, t) = (lane / 4, lane % 4) holds
// entries (8 ti + g, 8 tj + 2 t + {0, 1}) of each. Operands are read from shared memory straight
// into fragments: A's (row g, column p + t) and B's (row p + t, column g) of each k-step of 4.
// Rows and columns past m / n read whatever the operand tiles hold there and only feed entries
// that are never stored; the reduction index is exact (the last partial k-step is masked).
constexpr int kSolverWarps = kSolverThreads / 32;

template <int MAXM>
constexpr int mma_tiles() { return ((MAXM / 8) * (MAXM / 8) + kSolverWarps - 1) / kSolverWarps; }

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// acc = -A B (A: m x k row-major, lda; B: k x n row-major, ldb) for the warp's tiles.
template <int MAXT>
__device__ __forceinline__ void mma_negated_product(double (&acc)[MAXT][2], int m, int n, const double* A,
                                                    int lda, const double* B, int ldb, int k) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int tn = (n + 7) >> 3, tiles = ((m + 7) >> 3) * tn;
  const double* ap[MAXT];
  const double* bp[MAXT];
#pragma unroll
  for (int x = 0; x < MAXT; ++x) {
    acc[x][0] = acc[x][1] = 0.0;
    const int tile = min(warp + kSolverWarps * x, tiles - 1);
    const int ti = tile / tn, tj = tile - ti * tn;
    ap[x] = A + (8 * ti + g) * lda + t;
    bp[x] = B + t * ldb + 8 * tj + g;
  }
  int p0 = 0;
  for (; p0 + 4 <= k; p0 += 4) {
#pragma unroll
    for (int x = 0; x < MAXT; ++x) {
      if (warp + kSolverWarps * x >= tiles) break;
      dmma(acc[x], -*ap[x], *bp[x]);
      ap[x] += 4;
      bp[x] += 4 * ldb;
    }
  }
  if (p0 < k) {
    const bool ok = p0 + t < k;
#pragma unroll
    for (int x = 0; x < MAXT; ++x) {
      if (warp + kSolverWarps * x >= tiles) break;
      dmma(acc[x], ok ? -*ap[x] : 0.0, ok ? *bp[x] : 0.0);
    }
  }
}

// For each held entry (i, j) of an m x n output with i < m, j < n: f(i, j, value).
template <int MAXT, typename F>
__device__ __forceinline__ void mma_for_each(const double (&acc)[MAXT][2], int m, int n, F&& f) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int tn = (n + 7) >> 3, tiles = ((m + 7) >> 3) * tn;
#pragma unroll
  for (int x = 0; x < MAXT; ++x) {
    const int tile = warp + kSolverWarps * x;
    if (tile >= tiles) break;
    const int ti = tile / tn, tj = tile - ti * tn;
    const int i = 8 * ti + g, j = 8 * tj + 2 * t;
    if (i < m) {
      if (j < n) f(i, j, acc[x][0]);
      if (j + 1 < n) f(i, j + 1, acc[x][1]);
    }
  }
}

// In-place lower Cholesky of the m x m tile `a` (leading dimension LD); rinv[i] = 1 / L[i][i].
// A non-positive pivot becomes NaN, which propagates to every result of the system. Only the
// lower triangle is read; the strict upper triangle is zeroed on exit.
template <int LD>
__device__ void cholesky(double* a, int m, double* rinv) {
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
          const double inv = 1.0 / d;
          if (r == k) row[k] = d;
          else if (r > k) row[k] *= inv;
          if (r == 0) rinv[kb + k] = inv;
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
          x[c] = v * rinv[kb + c];
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

// rinv[i] = 1 / l[i][i] for a loaded factor tile; ends with a barrier.
__device__ void reciprocal_diagonal(const double* l, int ldl, int m, double* rinv) {
  for (int i = threadIdx.x; i < m; i += blockDim.x) rinv[i] = 1.0 / l[i * ldl + i];
  __syncthreads();
}

// Solve L X = B in place (L: m x m lower; B: m x n).
__device__ void lower_solve(const double* l, int ldl, const double* rinv, double* b, int ldb, int m, int n) {
  for (int kb = 0; kb < m; kb += kB) {
    const int nb = min(kB, m - kb);
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      double x[kB];
#pragma unroll
      for (int r = 0; r < kB; ++r) {
        if (r < nb) {
          double v = b[(kb + r) * ldb + c];
#pragma unroll
          for (int s = 0; s < r; ++s) v = fma(-l[(kb + r) * ldl + kb + s], x[s], v);
          x[r] = v * rinv[kb + r];
          b[(kb + r) * ldb + c] = x[r];
        }
      }
    }
    __syncthreads();
    const int rest = m - kb - nb;
    if (rest > 0)
      tile_gemm<false, false>(b + (kb + nb) * ldb, ldb, l + (kb + nb) * ldl + kb, ldl, b + kb * ldb, ldb,
                              rest, n, nb, -1.0);
    __syncthreads();
  }
}

// Solve L^T X = B in place.
__device__ void upper_solve(const double* l, int ldl, const double* rinv, double* b, int ldb, int m, int n) {
  const int last = ((m - 1) / kB) * kB;
  for (int kb = last; kb >= 0; kb -= kB) {
    const int nb = min(kB, m - kb);
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      double x[kB];
#pragma unroll
      for (int r = kB - 1; r >= 0; --r) {
        if (r < nb) {
          double v = b[(kb + r) * ldb + c];
#pragma unroll
          for (int s = r + 1; s < kB; ++s)
            if (s < nb) v = fma(-l[(kb + s) * ldl + kb + r], x[s], v);
          x[r] = v * rinv[kb + r];
          b[(kb + r) * ldb + c] = x[r];
        }
      }
    }
    __syncthreads();
    if (kb > 0)
      tile_gemm<true, false>(b, ldb, l + kb * ldl, ldl, b + kb * ldb, ldb, kb, n, nb, -1.0);
    __syncthreads();
  }
}

// Column capacity of the level kernel: 3 MAXM, or 128 when every augmented row fits in it.
constexpr int kNarrowColumns = 128;
// Augmented matrix (MAXM x WCOL + 1), two buffers of panel rows (8 x WCOL) and panel columns
// (MAXM x 9), and per warp the pivot-block inverse (8 x 8) and its own rows of L P^-1 (MAXM / 8 x 8).
template <int MAXM, int WCOL = 3 * MAXM>
constexpr size_t invert_smem() {
  return sizeof(double) * ((size_t)MAXM * (WCOL + 1) + 2 * 8 * (size_t)WCOL + 2 * (size_t)MAXM * 9 +
                           8 * 64 + 8 * (size_t)MAXM);
}

// 1 / x for x > 0 (NaN otherwise): the hardware approximation refined by two Newton-Raphson steps
// y <- y + y (1 - x y), each of which squares the relative error.
__device__ __forceinline__ double positive_reciprocal(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  return x > 0.0 ? y : quiet_nan();
}
template <int MAXM>
constexpr size_t update_smem() { return sizeof(double) * (5 * (size_t)MAXM * (MAXM + 1)); }
template <int MAXM>
constexpr size_t forward_update_smem() { return sizeof(double) * (5 * (size_t)MAXM * (MAXM + 1)); }
template <int MAXM>
constexpr size_t backward_smem() { return sizeof(double) * (6 * (size_t)MAXM * (MAXM + 1)); }

// D_j of every block from the assembled CSR values, into the block's G_j storage (the eager
// Schur updates then subtract from it level by level).
__global__ void __launch_bounds__(kSolverThreads)
scatter_diagonal_kernel(const int64_t* __restrict__ tasks, const int* __restrict__ csr_ptr,
                        const int* __restrict__ csr_row, const int* __restrict__ csr_col, int nnz,
                        const double* __restrict__ values, double* __restrict__ factors, int64_t stride) {
  chain_wait();
  const int64_t* t = tasks + (int64_t)blockIdx.x * T_FIELDS;
  const double* val = values + (int64_t)blockIdx.y * nnz;
  double* d = factors + (int64_t)blockIdx.y * stride + t[T_LOFF];
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  for (int i = threadIdx.x; i < mj * mj; i += blockDim.x) d[i] = 0.0;
  __syncthreads();
  for (int s = csr_ptr[offj] + threadIdx.x; s < csr_ptr[offj + mj]; s += blockDim.x) {
    const int c = csr_col[s];
    if (c >= offj && c < offj + mj) d[(csr_row[s] - offj) * mj + (c - offj)] = val[s];
  }
}

// C (m x n, leading dimension ldc, may be global memory) = acc, combining split halves through
// `scratch` (>= 128 x 16 doubles). Entered by all threads; ends with a barrier.
__device__ void store_tile(double (&acc)[4][4], const Micro& u, double* C, int64_t ldc, int m, int n,
                           double* scratch) {
  if (u.nsplit == 2) {
    if (u.part == 1 && u.active)
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int s = 0; s < 4; ++s) scratch[u.tile * 16 + r * 4 + s] = acc[r][s];
    __syncthreads();
  }
  if (u.part == 0 && u.active) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = u.ti + r * u.mt;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int j = u.tj + s * u.nt;
        double v = acc[r][s];
        if (u.nsplit == 2) v += scratch[u.tile * 16 + r * 4 + s];
        if (i < m && j < n) C[i * ldc + j] = v;
      }
    }
  }
  __syncthreads();
}

// One BCR level, inverse form. For the eliminated block j with chain neighbours p and q, the
// augmented matrix [D_j | A[j,p] | A[q,j]^T] (D_j with every earlier Schur update applied) is
// reduced by block Gauss-Jordan elimination without pivoting (D_j is SPD) to
// [G_j | Z_p | Z_q], G_j = D_j^-1, Z_p = G_j A[j,p], Z_q = G_j A[q,j]^T. Pivots go in panels of
// 8: with the panel P (8 x 8), its rows R, its columns L and the rest S, one step is
// P <- P^-1, R <- P^-1 R, L <- -L P^-1, S <- S - L P^-1 R. Every thread holds a fixed set of
// augmented entries in registers (rows tr + 8 r, columns tc + 32 c; a panel's rows are pass
// r = k0 / 8 of the 8 row groups). A step publishes the panel rows (with the identity in the
// panel columns) and columns to one of two buffers, then a barrier; warp 0 inverts P, then a
// second barrier; every warp forms C = L P^-1 for its own rows (C = -P^-1 on the panel rows,
// which start from zero), and updates its entries by a <- a - C R. Stored: G_j, Z_p,
// V_q = Z_q^T, copies of the couplings (for the Schur updates) and the fill A[q,p] = -A[q,j] Z_p.
// A non-positive pivot becomes NaN, which reaches every result of the system.
template <int MAXM, int WCOL = 3 * MAXM>
__global__ void __launch_bounds__(kSolverThreads, MAXM <= 48 ? 2 : 1)
invert_level_kernel(const int64_t* __restrict__ tasks, int task_begin, const int* __restrict__ csr_ptr,
                    const int* __restrict__ csr_row, const int* __restrict__ csr_col, int nnz,
                    const double* __restrict__ values, double* __restrict__ factors, int64_t stride) {
  chain_wait();
  constexpr int LDA = WCOL + 1;
  constexpr int W3 = WCOL;                      // column capacity (>= every mj + mp + mq)
  constexpr int RP = MAXM / 8;                  // rows per thread
  constexpr int CP = (W3 + 31) / 32;            // columns per thread
  constexpr int PB = 8;                         // pivot panel
  extern __shared__ double sm[];
  double* aug = sm;                             // [MAXM][LDA]
  double* rbuf = aug + MAXM * LDA;              // panel rows      [2][PB][W3]
  double* lbuf = rbuf + 2 * PB * W3;            // panel columns   [2][MAXM][PB + 1]
  double* pinv_all = lbuf + 2 * MAXM * (PB + 1);  // P^-1 [PB][PB] (room for 8)
  double* c_all = pinv_all + 8 * PB * PB;       // per warp C      [8][RP][PB]
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* val = values + (int64_t)blockIdx.y * nnz;
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  const int p = (int)t[T_P], mp = p >= 0 ? (int)t[T_MP] : 0, offp = (int)t[T_OFFP];
  const int q = (int)t[T_Q], mq = q >= 0 ? (int)t[T_MQ] : 0, offq = (int)t[T_OFFQ];
  const bool p_csr = p >= 0 && t[T_LINKP] < 0, q_csr = q >= 0 && t[T_LINKQ] < 0;
  const int width = mj + mp + mq;
  const int s0 = csr_ptr[offj], s1 = csr_ptr[offj + mj];

  // 1. [D_j | A[j,p] | A[q,j]^T] in shared memory
  async_tile(aug, LDA, f + t[T_LOFF], mj, mj);
  if (p >= 0 && !p_csr) async_tile(aug + mj, LDA, f + t[T_LINKP], mj, mp);  // A[j,p]: the previous level's fill
  async_commit();
  for_each_entry(mj, mp + mq, [&](int r, int c, int) {
    if (p_csr || c >= mp) aug[r * LDA + mj + c] = 0.0;
  });
  __syncthreads();
  for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
    const int r = csr_row[s] - offj, c = csr_col[s];
    if (p_csr && c >= offp && c < offp + mp) aug[r * LDA + mj + (c - offp)] = val[s];
    else if (q_csr && c >= offq && c < offq + mq) aug[r * LDA + mj + mp + (c - offq)] = val[s];
  }
  if (q >= 0 && !q_csr) {  // A[q,j] (mq x mj), stored transposed after A[j,p]
    const double* src = f + t[T_LINKQ];
    for_each_entry(mq, mj, [&](int r, int k, int i) { aug[k * LDA + mj + mp + r] = src[i]; });
  }
  async_wait_all();
  __syncthreads();

  // 2. copies of the couplings (read by the Schur updates and the fill)
  if (p >= 0) {
    double* ru = f + t[T_RUOFF];
    for_each_entry(mj, mp, [&](int r, int c, int i) { ru[i] = aug[r * LDA + mj + c]; });
  }
  if (q >= 0) {
    double* rv = f + t[T_RVOFF];
    for_each_entry(mq, mj, [&](int r, int k, int i) { rv[i] = aug[k * LDA + mj + mp + r]; });
  }

  // 3. block Gauss-Jordan in registers
  const int tc = threadIdx.x & 31, tr = threadIdx.x >> 5;
  double* pinv = pinv_all;  // P^-1 of the current panel (written by warp 0)
  double* cw = c_all + tr * RP * PB;
  double a[RP][CP];
#pragma unroll
  for (int r = 0; r < RP; ++r)
#pragma unroll
    for (int c = 0; c < CP; ++c) {
      const int i = tr + 8 * r, j = tc + 32 * c;
      a[r][c] = (i < mj && j < width) ? aug[i * LDA + j] : 0.0;
    }
  // the panel loop is unrolled over the register row rb that holds the panel's rows, so the
  // panel's row, column group and buffer are compile-time in each copy
#pragma unroll
  for (int rb = 0; rb < RP; ++rb) {
    const int k0 = rb * PB;
    if (k0 >= mj) break;
    const int nb = min(PB, mj - k0);
    double* rows = rbuf + (rb & 1) * PB * W3;
    double* cols = lbuf + (rb & 1) * MAXM * (PB + 1);
    const int cg = k0 >> 5;                                  // column group of the panel columns
    const unsigned s = (unsigned)(tc - (k0 & 31));           // this lane's panel column, if < PB
    // (a) publish the panel rows (row k0 + tr from register row rb; identity in the panel
    //     columns) and the panel columns (P itself in rows k0 .. k0 + 7); no warp still reads
    //     this buffer, since every warp has passed the previous step's barrier
#pragma unroll
    for (int c = 0; c < CP; ++c) {
      const int j = tc + 32 * c;
      const unsigned sj = (unsigned)(j - k0);
      if (j < W3)
        rows[tr * W3 + j] = tr >= nb ? 0.0 : sj < (unsigned)nb ? (sj == (unsigned)tr ? 1.0 : 0.0)
                                                                : (j < width ? a[rb][c] : 0.0);
    }
    if (s < (unsigned)PB)
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (c == cg)
#pragma unroll
          for (int r = 0; r < RP; ++r) {
            const int i = tr + 8 * r;
            cols[i * (PB + 1) + s] = (s < (unsigned)nb && i < mj) ? a[r][c] : 0.0;
          }
    __syncthreads();
    // (b) P^-1 by warp 0 (the other warps wait at the barrier below instead of repeating it):
    //     lane 4 v + h holds row v, columns 2 h and 2 h + 1 (the padding beyond nb is the identity)
    if (tr == 0) {
      const int v = tc >> 2, h = tc & 3;
      double x0 = (v < nb && 2 * h < nb) ? cols[(k0 + v) * (PB + 1) + 2 * h] : (v == 2 * h ? 1.0 : 0.0);
      double x1 = (v < nb && 2 * h + 1 < nb) ? cols[(k0 + v) * (PB + 1) + 2 * h + 1] : (v == 2 * h + 1 ? 1.0 : 0.0);
#pragma unroll
      for (int k = 0; k < PB; ++k) {
        const double r0 = __shfl_sync(0xffffffffu, x0, 4 * k + h);   // row k, columns 2h, 2h + 1
        const double r1 = __shfl_sync(0xffffffffu, x1, 4 * k + h);
        const double pivot = __shfl_sync(0xffffffffu, (k & 1) ? x1 : x0, 4 * k + (k >> 1));
        const double mk = __shfl_sync(0xffffffffu, (k & 1) ? x1 : x0, 4 * v + (k >> 1));  // row v, column k
        const double inv = positive_reciprocal(pivot);
        const double lik = mk * inv;
        const bool c0k = 2 * h == k, c1k = 2 * h + 1 == k;
        if (v == k) {
          x0 = c0k ? inv : x0 * inv;
          x1 = c1k ? inv : x1 * inv;
        } else {
          x0 = c0k ? -lik : fma(-lik, r0, x0);
          x1 = c1k ? -lik : fma(-lik, r1, x1);
        }
      }
      *reinterpret_cast<double2*>(pinv + v * PB + 2 * h) = make_double2(x0, x1);
    }
    __syncthreads();
    // (c) C for this warp's rows: L P^-1, or -P^-1 on the panel row
    for (int e = tc; e < RP * PB; e += 32) {
      const int r = e / PB, u = e - r * PB, i = tr + 8 * r;
      double v = 0.0;
      if (r == rb && tr < nb) {
        v = -pinv[tr * PB + u];
      } else {
#pragma unroll
        for (int w = 0; w < PB; ++w) v = fma(cols[i * (PB + 1) + w], pinv[w * PB + u], v);
      }
      cw[e] = v;
    }
    __syncwarp();
    // (d) a <- keep a - C R: the panel columns and the panel row start from zero
    if (s < (unsigned)nb)
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (c == cg)
#pragma unroll
          for (int r = 0; r < RP; ++r) a[r][c] = 0.0;
    if (tr < nb)
#pragma unroll
      for (int c = 0; c < CP; ++c) a[rb][c] = 0.0;
#pragma unroll
    for (int u = 0; u < PB; u += 2) {
      double2 lu[RP];
      double ru0[CP], ru1[CP];
#pragma unroll
      for (int r = 0; r < RP; ++r) lu[r] = *reinterpret_cast<const double2*>(cw + r * PB + u);
#pragma unroll
      for (int c = 0; c < CP; ++c) {
        const int j = tc + 32 * c;
        ru0[c] = j < W3 ? rows[u * W3 + j] : 0.0;
        ru1[c] = j < W3 ? rows[(u + 1) * W3 + j] : 0.0;
      }
#pragma unroll
      for (int r = 0; r < RP; ++r)
#pragma unroll
        for (int c = 0; c < CP; ++c) a[r][c] = fma(-lu[r].y, ru1[c], fma(-lu[r].x, ru0[c], a[r][c]));
    }
  }

  // 4. G_j, Z_p, V_q to the factor storage; Z_p back to shared memory for the fill
#pragma unroll
  for (int r = 0; r < RP; ++r)
#pragma unroll
    for (int c = 0; c < CP; ++c) {
      const int i = tr + 8 * r, j = tc + 32 * c;
      if (i >= mj || j >= width) continue;
      const double v = a[r][c];
      aug[i * LDA + j] = v;
      if (j < mj) f[t[T_LOFF] + i * mj + j] = v;
      else if (j < mj + mp) f[t[T_UOFF] + i * mp + (j - mj)] = v;
      else f[t[T_VOFF] + (j - mj - mp) * mj + i] = v;
    }
  if (p < 0 || q < 0) return;
  __syncthreads();
  // 5. fill A[q,p] = -A[q,j] Z_p: the coupling copy (written by this block above) replaces G_j
  //    in shared memory
  {
    const double* rv = f + t[T_RVOFF];
    for_each_entry(mq, mj, [&](int r, int k, int i) { aug[r * LDA + k] = rv[i]; });
  }
  double* fill = f + t[T_FILL];
  __syncthreads();
  double acc[mma_tiles<MAXM>()][2];
  mma_negated_product(acc, mq, mp, aug, LDA, aug + mj, LDA, mj);
  mma_for_each(acc, mq, mp, [&](int i, int j, double v) { fill[i * mp + j] = v; });
}

// Eager Schur updates after a level: block j of every item subtracts the pulls [u0, u1) of that
// level from D_j, in place in its G_j storage: A[e,j]^T Z_j for the elimination e on its right,
// V_j A[j,e]^T for the one on its left (operands stream in with cp.async, products accumulate in
// registers).
template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, 2)
update_level_kernel(const int* __restrict__ items, int item_begin, const int64_t* __restrict__ tasks,
                    const int64_t* __restrict__ pulls, double* __restrict__ factors, int64_t stride) {
  chain_wait();
  constexpr int LD = MAXM + 1;
  extern __shared__ double sm[];
  auto tile = [&](int i) { return sm + i * MAXM * LD; };
  double* dm = tile(4);
  const int* it = items + 3 * (item_begin + blockIdx.x);
  const int64_t* t = tasks + (int64_t)it[0] * T_FIELDS;
  const int64_t u0 = it[1], u1 = it[2];
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int mj = (int)t[T_MJ];
  double* d = f + t[T_LOFF];
  auto issue = [&](int64_t u, int pair) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int me = (int)pl[P_ME];
    if (pl[P_TYPE] == 0) {  // coupling A[e,j] and Z_j, both me x mj
      async_tile(tile(2 * pair), LD, f + pl[P_AOFF], me, mj);
      async_tile(tile(2 * pair + 1), LD, f + pl[P_OFF], me, mj);
    } else {                // V_j and coupling A[j,e], both mj x me
      async_tile(tile(2 * pair), LD, f + pl[P_OFF], mj, me);
      async_tile(tile(2 * pair + 1), LD, f + pl[P_AOFF], mj, me);
    }
  };
  async_tile(dm, LD, d, mj, mj);
  issue(u0, 0);
  async_commit();
  const Micro mu(mj, mj);
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int s = 0; s < 4; ++s) acc[r][s] = 0.0;
  for (int64_t u = u0; u < u1; ++u) {
    async_wait_all();
    __syncthreads();
    const int cur = (int)((u - u0) & 1);
    if (u + 1 < u1) {
      issue(u + 1, cur ^ 1);
      async_commit();
    }
    const double* X = tile(2 * cur);
    const double* Y = tile(2 * cur + 1);
    const int me = (int)pulls[u * P_FIELDS + P_ME];
    if (pulls[u * P_FIELDS + P_TYPE] == 0) accumulate<true, false>(acc, mu, X, LD, Y, LD, me);
    else accumulate<false, true>(acc, mu, X, LD, Y, LD, me);
  }
  __syncthreads();
  subtract_tile(acc, mu, dm, LD, mj, mj, tile(0));
  for_each_entry(mj, mj, [&](int r, int c, int i) { d[i] = dm[r * LD + c]; });
}

// The Schur updates of one level with the forward substitution of the same level fused in: block
// j of every item subtracts, for each of its pulls, A[e,j]^T Z_j (or V_j A[j,e]^T) from D_j and
// Z_j^T b_e (or V_j b_e) from b_j, all nrhs (<= MAXM) columns of the right-hand side. Operands
// of one pull at a time (coupling, Z_j or V_j, b_e) plus D_j and b_j in shared memory; products
// accumulate in registers; D_j and b_j are written back once.
template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, 2)
update_rhs_level_kernel(const int* __restrict__ items, int item_begin, const int64_t* __restrict__ tasks,
                        const int64_t* __restrict__ pulls, double* __restrict__ factors, int64_t stride,
                        double* __restrict__ rhs, int64_t rhs_stride, int nrhs) {
  chain_wait();
  constexpr int LD = MAXM + 1;
  extern __shared__ double sm[];
  auto tile = [&](int i) { return sm + i * MAXM * LD; };
  double* X = tile(0);   // A[e,j] (type 0) or V_j (type 1)
  double* Y = tile(1);   // Z_j (type 0) or A[j,e] (type 1)
  double* be = tile(2);  // b_e (me x nrhs)
  double* dm = tile(3);  // D_j
  double* bt = tile(4);  // b_j
  const int* it = items + 3 * (item_begin + blockIdx.x);
  const int64_t* t = tasks + (int64_t)it[0] * T_FIELDS;
  const int64_t u0 = it[1], u1 = it[2];
  double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  double* d = f + t[T_LOFF];
  async_tile(dm, LD, d, mj, mj);
  async_rows(bt, LD, x + (int64_t)offj * nrhs, nrhs, mj, nrhs);
  const Micro md(mj, mj), mb(mj, nrhs);
  double accd[4][4], accb[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) accd[r][c] = accb[r][c] = 0.0;
  for (int64_t u = u0; u < u1; ++u) {
    if (u > u0) __syncthreads();  // the previous pull's operands have been read
    const int64_t* pl = pulls + u * P_FIELDS;
    const int me = (int)pl[P_ME];
    const bool right = pl[P_TYPE] == 0;
    if (right) {
      async_tile(X, LD, f + pl[P_AOFF], me, mj);
      async_tile(Y, LD, f + pl[P_OFF], me, mj);
    } else {
      async_tile(X, LD, f + pl[P_OFF], mj, me);
      async_tile(Y, LD, f + pl[P_AOFF], mj, me);
    }
    async_rows(be, LD, x + (int64_t)pl[P_EOFF] * nrhs, nrhs, me, nrhs);
    async_commit();
    async_wait_all();
    __syncthreads();
    if (right) {
      accumulate<true, false>(accd, md, X, LD, Y, LD, me);   // A[e,j]^T Z_j
      accumulate<true, false>(accb, mb, Y, LD, be, LD, me);  // Z_j^T b_e
    } else {
      accumulate<false, true>(accd, md, X, LD, Y, LD, me);   // V_j A[j,e]^T
      accumulate<false, false>(accb, mb, X, LD, be, LD, me); // V_j b_e
    }
  }
  __syncthreads();
  subtract_tile(accd, md, dm, LD, mj, mj, tile(0));
  subtract_tile(accb, mb, bt, LD, mj, nrhs, tile(0));
  for_each_entry(mj, mj, [&](int r, int c, int i) { d[i] = dm[r * LD + c]; });
  for_each_entry(mj, nrhs, [&](int r, int c, int) { x[(int64_t)(offj + r) * nrhs + c] = bt[r * LD + c]; });
}

// Eager forward updates after a level: b_j -= Z_j^T b_e / V_j b_e for the pulls [u0, u1) of the
// item, right-hand-side columns [c0, c0 + strip).
template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, 2)
forward_update_kernel(const int* __restrict__ items, int item_begin, const int64_t* __restrict__ tasks,
                      const int64_t* __restrict__ pulls, const double* __restrict__ factors,
                      int64_t stride, double* __restrict__ rhs, int64_t rhs_stride, int nrhs, int strip) {
  chain_wait();
  constexpr int LD = MAXM + 1;
  extern __shared__ double sm[];
  auto tile = [&](int i) { return sm + i * MAXM * LD; };
  double* bt = tile(4);
  const int* it = items + 3 * (item_begin + blockIdx.x);
  const int64_t* t = tasks + (int64_t)it[0] * T_FIELDS;
  const int64_t u0 = it[1], u1 = it[2];
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * strip;
  const int nc = min(strip, nrhs - c0);
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  auto issue = [&](int64_t u, int pair) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int me = (int)pl[P_ME];
    if (pl[P_TYPE] == 0) async_tile(tile(2 * pair), LD, f + pl[P_OFF], me, mj);
    else async_tile(tile(2 * pair), LD, f + pl[P_OFF], mj, me);
    async_rows(tile(2 * pair + 1), LD, x + (int64_t)pl[P_EOFF] * nrhs + c0, nrhs, me, nc);
  };
  async_rows(bt, LD, x + (int64_t)offj * nrhs + c0, nrhs, mj, nc);
  issue(u0, 0);
  async_commit();
  const Micro mu(mj, nc);
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int s = 0; s < 4; ++s) acc[r][s] = 0.0;
  for (int64_t u = u0; u < u1; ++u) {
    async_wait_all();
    __syncthreads();
    const int cur = (int)((u - u0) & 1);
    if (u + 1 < u1) {
      issue(u + 1, cur ^ 1);
      async_commit();
    }
    const double* M = tile(2 * cur);
    const double* Y = tile(2 * cur + 1);
    const int me = (int)pulls[u * P_FIELDS + P_ME];
    if (pulls[u * P_FIELDS + P_TYPE] == 0) accumulate<true, false>(acc, mu, M, LD, Y, LD, me);   // Z^T b
    else accumulate<false, false>(acc, mu, M, LD, Y, LD, me);                                     // V b
  }
  __syncthreads();
  subtract_tile(acc, mu, bt, LD, mj, nc, tile(0));
  for_each_entry(mj, nc, [&](int r, int c, int) { x[(int64_t)(offj + r) * nrhs + c0 + c] = bt[r * LD + c]; });
}

// Backward level: x_j = G_j b_j - Z_p x_p - V_q^T x_q (the root: x = G b), every operand
// prefetched at once; columns [c0, c0 + strip).
template <int MAXM>
__global__ void __launch_bounds__(kSolverThreads, 2)
backward_level_kernel(const int64_t* __restrict__ tasks, int task_begin,
                      const double* __restrict__ factors, int64_t stride,
                      double* __restrict__ rhs, int64_t rhs_stride, int nrhs, int strip) {
  chain_wait();
  constexpr int LD = MAXM + 1;
  extern __shared__ double sm[];
  double* ut = sm;                 // Z_p (mj x mp)
  double* xp = ut + MAXM * LD;     // -x_p (mp x nc)
  double* vt = xp + MAXM * LD;     // V_q (mq x mj)
  double* xq = vt + MAXM * LD;     // -x_q (mq x nc)
  double* bt = xq + MAXM * LD;     // b_j
  double* gt = bt + MAXM * LD;     // G_j
  const int64_t* t = tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS;
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * strip;
  const int nc = min(strip, nrhs - c0);
  const int mj = (int)t[T_MJ], offj = (int)t[T_OFFJ];
  const int p = (int)t[T_P], q = (int)t[T_Q];
  const int mp = p >= 0 ? (int)t[T_MP] : 0, mq = q >= 0 ? (int)t[T_MQ] : 0;
  if (p >= 0) {
    async_tile(ut, LD, f + t[T_UOFF], mj, mp);
    async_rows(xp, LD, x + t[T_OFFP] * nrhs + c0, nrhs, mp, nc);
  }
  if (q >= 0) {
    async_tile(vt, LD, f + t[T_VOFF], mq, mj);
    async_rows(xq, LD, x + t[T_OFFQ] * nrhs + c0, nrhs, mq, nc);
  }
  async_rows(bt, LD, x + (int64_t)offj * nrhs + c0, nrhs, mj, nc);
  async_tile(gt, LD, f + t[T_LOFF], mj, mj);
  async_commit();
  async_wait_all();
  __syncthreads();
  for_each_entry(mp, nc, [&](int r, int c, int) { xp[r * LD + c] *= -1.0; });
  for_each_entry(mq, nc, [&](int r, int c, int) { xq[r * LD + c] *= -1.0; });
  __syncthreads();
  const Micro mu(mj, nc);
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int s = 0; s < 4; ++s) acc[r][s] = 0.0;
  accumulate<false, false>(acc, mu, gt, LD, bt, LD, mj);
  if (p >= 0) accumulate<false, false>(acc, mu, ut, LD, xp, LD, mp);
  if (q >= 0) accumulate<true, false>(acc, mu, vt, LD, xq, LD, mq);
  __syncthreads();
  store_tile(acc, mu, x + (int64_t)offj * nrhs + c0, nrhs, mj, nc, ut);
}

// ============================================================================================
// Tiled solver for blocks wider than kMaxBlock. The same elimination (same storage of L_j, U_p,
// V_q and fills) runs on 64 x 64 tiles in global memory, several launches per level:
//   scatter   D_j (lower), [A[j,p]] -> U_p, [A[q,j]] -> V_q from the CSR values or earlier fills
//   panel k   (a) update: tile (i, k) of the stacked rows [j; p; q] -= sum_{c < 64k} row_i(c)
//                 row_k(c) (and, for rows of j, the Schur pulls of earlier eliminations); the
//                 item of the diagonal tile (k, k) then factors it (no other item of the launch
//                 reads it: they read columns < 64k and write their own tiles);
//             (b) triangular solve of every tile below the diagonal with L_kk. Rows p and q of
//                 the stacked factor are U_p^T and V_q.
//   fill      A[q,p] = -V_q U_p
// A block's pulls and its own left-looking columns are summed in fixed order (bitwise
// repeatable). Solves: forward = pull update of b_j, then a left-looking substitution per
// (task, 64-column strip); backward = coupling update, then the transposed substitution.
// ============================================================================================
constexpr int kTT = kSolverThreads;  // threads of the tiled kernels (16 x 16 micro-tile grid)
constexpr int kKC = 16;              // reduction depth staged per step
constexpr int kTLD = kTile + 1;      // leading dimension of the shared tiles
constexpr int kSLD = kTile + 4;      // leading dimension of the GEMM staging tiles (== 4 mod 16)
constexpr int kStage = 4 * kKC * kSLD;  // doubles of GEMM staging (two buffers of A and B chunks)

// Element (a, c) of a strided operand: base[a * rs + c * cs].
struct Operand {
  const double* base;
  int64_t rs, cs;
};

__device__ __forceinline__ Operand operand(const double* base, int64_t rs, int64_t cs) {
  Operand o;
  o.base = base;
  o.rs = rs;
  o.cs = cs;
  return o;
}

template <int N>
__device__ __forceinline__ void async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The elements one thread copies for every depth chunk of an operand: rows a < SPAN of the
// chunk, kKC depths each, kTT threads. Addresses are formed once per GEMM call; a chunk only adds
// its depth offset.
template <int SPAN>
struct StagePlan {
  static constexpr int kPer = (kKC * SPAN + kTT - 1) / kTT;
  const double* src[kPer];
  int dst[kPer];
  int depth_of[kPer];  // the element's depth within a chunk; -1: row past the operand or unused
  int64_t step;        // source advance per chunk
  __device__ StagePlan(const Operand& op, int rows, int d0) {
    const bool depth_fast = op.cs == 1;
    step = (int64_t)kKC * op.cs;
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
      const int idx = threadIdx.x + e * kTT;
      const int a = depth_fast ? idx / kKC : idx % SPAN;
      const int c = depth_fast ? idx % kKC : idx / SPAN;
      const bool used = idx < kKC * SPAN;
      dst[e] = c * kSLD + a;  // see gemm_nt
      depth_of[e] = used && a < rows ? c : -1;
      src[e] = op.base + (int64_t)a * op.rs + (int64_t)(d0 + c) * op.cs;
    }
  }
  // chunk ch (depths d0 + ch * kKC + [0, kKC)) into tile; zero outside the operand or depth
  __device__ __forceinline__ void copy(double* tile, int ch, int limit) const {
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
      if (threadIdx.x + e * kTT >= kKC * SPAN) continue;
      if (depth_of[e] >= 0 && depth_of[e] + ch * kKC < limit) async_copy8(tile + dst[e], src[e] + ch * step);
      else tile[dst[e]] = 0.0;
    }
  }
};

// acc[r][s] += sum_{d0 <= c < depth} A(ty + 16 r, c) B(tx + 16 s, c) for A rows < ra, B rows
// < rb (d0 a multiple of kKC); the output has 64 rows and 16 NQ columns. The products run on
// the FP64 tensor cores (mma.sync m8n8k4): warp w owns rows 16 (w & 3) + [0, 16) and columns
// 8 NQ (w >> 2) + [0, 8 NQ) as 2 x NQ tiles of 8 x 8; the fragments are added to `acc` through
// shared memory at the end. Operand chunks are staged depth-major with cp.async,
// double-buffered: element (a, c) at tile[c * 68 + a]. 8-byte accesses are served per half-warp,
// and with a leading dimension of 4 mod 16 doubles the 4 depths x 4 rows of a half-warp's
// fragment load hit 16 distinct banks. (The leading dimension 72, with 2-way conflicted
// fragment loads, was 10 % slower on the terrain section; an XOR swizzle of the rows by depth,
// which spreads the staging writes of depth-contiguous operands, was slower again there and
// gained 1 ms at the 3D box.) `sm` holds kStage doubles; entered and left by all threads (ends
// with a barrier).
template <int NQ>
__device__ void gemm_nt(double (&acc)[4][NQ], const Operand& A, int ra, const Operand& B, int rb,
                        int depth, double* sm, int d0 = 0) {
  if (depth <= d0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = 16 * (warp & 3), n0 = 8 * NQ * (warp >> 2);
  const int chunks = (depth - d0 + kKC - 1) / kKC;
  const int limit = depth - d0;  // depths past it read as zero
  auto a_tile = [&](int b) { return sm + b * 2 * kKC * kSLD; };
  auto b_tile = [&](int b) { return sm + b * 2 * kKC * kSLD + kKC * kSLD; };
  const StagePlan<kTile> pa(A, ra, d0);
  const StagePlan<16 * NQ> pb(B, rb, d0);
  double frag[2][NQ][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NQ; ++j) frag[i][j][0] = frag[i][j][1] = 0.0;
  pa.copy(a_tile(0), 0, limit);
  pb.copy(b_tile(0), 0, limit);
  async_commit();
  for (int ch = 0; ch < chunks; ++ch) {
    if (ch + 1 < chunks) {
      pa.copy(a_tile((ch + 1) & 1), ch + 1, limit);
      pb.copy(b_tile((ch + 1) & 1), ch + 1, limit);
      async_commit();
      async_wait<1>();
    } else {
      async_wait<0>();
    }
    __syncthreads();
    const double* at = a_tile(ch & 1) + t * kSLD + m0;
    const double* bt = b_tile(ch & 1) + t * kSLD + n0;
#pragma unroll
    for (int k = 0; k < kKC; k += 4) {
      const int row = k * kSLD + g;
      double a[2], b[NQ];
#pragma unroll
      for (int i = 0; i < 2; ++i) a[i] = at[row + 8 * i];
#pragma unroll
      for (int j = 0; j < NQ; ++j) b[j] = bt[row + 8 * j];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NQ; ++j) dmma(frag[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  // fragments -> the block's accumulator layout, through the (now idle) staging buffer
  double* out = sm;  // [64][kTLD]
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      double* row = out + (m0 + 8 * i + g) * kTLD + n0 + 8 * j + 2 * t;
      row[0] = frag[i][j][0];
      row[1] = frag[i][j][1];
    }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[r][q] += out[(ty + 16 * r) * kTLD + tx + 16 * q];
  __syncthreads();
}

template <int NQ>
__device__ __forceinline__ void zero_acc(double (&acc)[4][NQ]) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[r][q] = 0.0;
}

// C(a, b) = C(a, b) - acc (subtract) or -acc (store) for a < rows, b < cols (and b <= a when
// `lower`), C(a, b) at c[a * rs + b * cs].
template <int NQ>
__device__ __forceinline__ void put_acc(const double (&acc)[4][NQ], double* c, int64_t rs, int64_t cs,
                                        int rows, int cols, bool subtract, bool lower) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int a = ty + 16 * r;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int b = tx + 16 * q;
      if (a < rows && b < cols && (!lower || b <= a)) {
        double* dst = c + a * rs + b * cs;
        *dst = subtract ? *dst - acc[r][q] : -acc[r][q];
      }
    }
  }
}

struct TaskView {
  int mj, offj, p, mp, offp, q, mq, offq;
  int64_t loff, uoff, voff, fill, linkp, linkq, pull0, pull1;
  __device__ explicit TaskView(const int64_t* t) {
    mj = (int)t[T_MJ];
    offj = (int)t[T_OFFJ];
    loff = t[T_LOFF];
    p = (int)t[T_P];
    mp = p >= 0 ? (int)t[T_MP] : 0;
    offp = (int)t[T_OFFP];
    uoff = t[T_UOFF];
    linkp = t[T_LINKP];
    q = (int)t[T_Q];
    mq = q >= 0 ? (int)t[T_MQ] : 0;
    offq = (int)t[T_OFFQ];
    voff = t[T_VOFF];
    linkq = t[T_LINKQ];
    fill = t[T_FILL];
    pull0 = t[T_PULL0];
    pull1 = t[T_PULL1];
  }
  // element (r, c) of segment `seg` of the stacked factor: rows of L_j, U_p^T or V_q
  __device__ Operand segment(double* f, int seg, int r, int c) const {
    if (seg == SEG_J) return operand(f + loff + (int64_t)r * mj + c, mj, 1);
    if (seg == SEG_P) return operand(f + uoff + (int64_t)c * mp + r, 1, mp);
    return operand(f + voff + (int64_t)r * mj + c, mj, 1);
  }
  __device__ int rows(int seg) const { return seg == SEG_J ? mj : (seg == SEG_P ? mp : mq); }
};

__global__ void __launch_bounds__(kTT)
tiled_scatter_kernel(const int* __restrict__ items, int begin, const int64_t* __restrict__ tasks,
                     const int* __restrict__ csr_ptr, const int* __restrict__ csr_row,
                     const int* __restrict__ csr_col, int nnz, const double* __restrict__ values,
                     double* __restrict__ factors, int64_t stride) {
  chain_wait();
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  const int r0 = it[1], rows = it[2];
  const double* val = values + (int64_t)blockIdx.y * nnz;
  double* f = factors + (int64_t)blockIdx.y * stride;
  const bool p_csr = v.p >= 0 && v.linkp < 0, q_csr = v.q >= 0 && v.linkq < 0;
  for (int64_t i = threadIdx.x; i < (int64_t)rows * v.mj; i += blockDim.x)
    f[v.loff + (int64_t)r0 * v.mj + i] = 0.0;
  for (int64_t i = threadIdx.x; i < (int64_t)rows * v.mp; i += blockDim.x)
    f[v.uoff + (int64_t)r0 * v.mp + i] = p_csr ? 0.0 : f[v.linkp + (int64_t)r0 * v.mp + i];
  for (int64_t i = threadIdx.x; i < (int64_t)rows * v.mq; i += blockDim.x) {
    const int qr = (int)(i / rows), r = r0 + (int)(i - (int64_t)qr * rows);
    f[v.voff + (int64_t)qr * v.mj + r] = q_csr ? 0.0 : f[v.linkq + (int64_t)qr * v.mj + r];
  }
  __syncthreads();
  const int s0 = csr_ptr[v.offj + r0], s1 = csr_ptr[v.offj + r0 + rows];
  for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
    const int r = csr_row[s] - v.offj, c = csr_col[s];
    if (c >= v.offj && c < v.offj + v.mj) {
      if (c - v.offj <= r) f[v.loff + (int64_t)r * v.mj + (c - v.offj)] = val[s];
    } else if (p_csr && c >= v.offp && c < v.offp + v.mp) {
      f[v.uoff + (int64_t)r * v.mp + (c - v.offp)] = val[s];
    } else if (q_csr && c >= v.offq && c < v.offq + v.mq) {
      f[v.voff + (int64_t)(c - v.offq) * v.mj + r] = val[s];
    }
  }
}

// L^-1 of the factored m x m diagonal tile in `dm` (rinv = 1 / diagonal) through the scratch
// tile `x` (64 x kTLD), stored 64 x 64 row-major at `out` (zero above the diagonal and past m):
// the triangular-solve launch of the panel applies it as a GEMM. Entered by all threads; ends
// with a barrier.
__device__ void store_inverse(const double* dm, const double* rinv, double* x, int m, double* out) {
  for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
    const int r = idx / kTile, c = idx - r * kTile;
    x[r * kTLD + c] = (r == c && r < m) ? 1.0 : 0.0;
  }
  __syncthreads();
  lower_solve(dm, kTLD, rinv, x, kTLD, m, m);  // columns of the identity: exact zeros above
  for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
    const int r = idx / kTile, c = idx - r * kTile;
    out[idx] = (r < m && c < m) ? x[r * kTLD + c] : 0.0;
  }
  __syncthreads();
}

// Depth chunks (of kKC) of one update item: its own columns [0, 64k), then each pull's depth.
__device__ __forceinline__ int update_chunks(const TaskView& v, int seg, int k, const int64_t* pulls) {
  int n = (kTile * k) / kKC;
  if (seg == SEG_J)
    for (int64_t u = v.pull0; u < v.pull1; ++u) n += ((int)pulls[u * P_FIELDS + P_ME] + kKC - 1) / kKC;
  return n;
}

// Panel k update of tile (i, k) of segment seg: acc = row_i(c < 64k) row_k^T (+ the Schur pulls
// for rows of j), 64 rows by the panel's 16 NQ columns. With `splits` == 1 the block subtracts acc from the tile and, for the diagonal
// item, factors it. With splits > 1 the item's depth chunks are divided evenly over blockIdx.z
// and each block stores its partial acc in `partials` (tile (item, z) of the launch: rows < ni,
// columns < mk at [((system * items + item) * splits + z) * 4096 + a * 64 + b]); the diagonal
// and triangular-solve launches sum them.
template <int NQ>
__global__ void __launch_bounds__(kTT)
tiled_update_kernel(const int* __restrict__ items, int begin, int k, const int64_t* __restrict__ tasks,
                    const int64_t* __restrict__ pulls, double* __restrict__ factors, int64_t stride,
                    int splits, double* __restrict__ partials, double* __restrict__ inverses, int t0,
                    int level_tasks) {
  chain_wait();
  extern __shared__ double sm[];
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  const int seg = it[1], i = it[2];
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int ni = min(kTile, v.rows(seg) - kTile * i), mk = min(kTile, v.mj - kTile * k);
  double acc[4][NQ];  // columns of the panel: 16 NQ >= its width
  zero_acc(acc);
  // this block's chunk range [lo, hi) of the item's depth chunks (all of them when unsplit)
  int lo = 0, hi = 1 << 30;
  if (splits > 1) {
    const int n = update_chunks(v, seg, k, pulls), z = blockIdx.z;
    lo = (int)((int64_t)n * z / splits);
    hi = (int)((int64_t)n * (z + 1) / splits);
  }
  // sum over one depth segment of `chunks` chunks starting at chunk `base` of the item
  auto segment = [&](const Operand& A, const Operand& B, int depth, int base) {
    const int chunks = (depth + kKC - 1) / kKC;
    const int c0 = max(lo - base, 0), c1 = min(hi - base, chunks);
    if (c1 > c0) gemm_nt(acc, A, ni, B, mk, min(depth, c1 * kKC), sm, c0 * kKC);
    return base + chunks;
  };
  int base = 0;
  if (k > 0)
    base = segment(v.segment(f, seg, kTile * i, 0), v.segment(f, SEG_J, kTile * k, 0), kTile * k, base);
  if (seg == SEG_J) {
    for (int64_t u = v.pull0; u < v.pull1; ++u) {
      const int64_t* pl = pulls + u * P_FIELDS;
      const int me = (int)pl[P_ME];
      const double* x = f + pl[P_OFF];
      if (pl[P_TYPE] == 0)  // U_e (me x mj): (U^T U)[a][b] = sum_r U[r][a] U[r][b]
        base = segment(operand(x + kTile * i, 1, v.mj), operand(x + kTile * k, 1, v.mj), me, base);
      else  // V_e (mj x me): (V V^T)[a][b] = sum_r V[a][r] V[b][r]
        base = segment(operand(x + (int64_t)kTile * i * me, me, 1), operand(x + (int64_t)kTile * k * me, me, 1),
                       me, base);
    }
  }
  if (splits > 1) {
    double* out = partials + ((int64_t)(blockIdx.y * gridDim.x + blockIdx.x) * splits + blockIdx.z) * kTile * kTile;
    put_acc(acc, out, kTile, 1, ni, mk, false, false);  // stores -acc
    return;
  }
  const Operand c = v.segment(f, seg, kTile * i, kTile * k);
  const bool diagonal = seg == SEG_J && i == k;
  put_acc(acc, const_cast<double*>(c.base), c.rs, c.cs, ni, mk, true, diagonal);
  if (!diagonal) return;
  // factor the updated diagonal tile in shared memory (after the staging buffers' last use)
  double* dm = sm + kStage;
  double* rinv = dm + kTile * kTLD;
  double* diag = const_cast<double*>(c.base);
  __syncthreads();
  for (int idx = threadIdx.x; idx < mk * mk; idx += blockDim.x) {
    const int r = idx / mk, col = idx - r * mk;
    dm[r * kTLD + col] = diag[(int64_t)r * v.mj + col];
  }
  __syncthreads();
  cholesky<kTLD>(dm, mk, rinv);
  for (int idx = threadIdx.x; idx < mk * mk; idx += blockDim.x) {
    const int r = idx / mk, col = idx - r * mk;
    diag[(int64_t)r * v.mj + col] = dm[r * kTLD + col];
  }
  store_inverse(dm, rinv, sm, mk,
                inverses + ((int64_t)blockIdx.y * level_tasks + (it[0] - t0)) * kTile * kTile);
}

// Split panels: the diagonal item adds its partials (stored negated, summed in split order) to
// the lower triangle of the diagonal tile and factors it; the launch's other items return. (The
// tiles below solve with L_kk by substitution: a split panel has few of them, and forming
// L_kk^-1 here would lengthen the panel's critical path.)
__global__ void __launch_bounds__(kTT)
tiled_diagonal_kernel(const int* __restrict__ items, int begin, int k, const int64_t* __restrict__ tasks,
                      double* __restrict__ factors, int64_t stride, int splits,
                      const double* __restrict__ partials) {
  chain_wait();
  extern __shared__ double sm[];
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  if (it[1] != SEG_J || it[2] != k) return;
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int mk = min(kTile, v.mj - kTile * k);
  double* dm = sm;
  double* rinv = dm + kTile * kTLD;
  double* diag = f + v.loff + (int64_t)kTile * k * v.mj + kTile * k;
  const double* part = partials + (int64_t)(blockIdx.y * gridDim.x + blockIdx.x) * splits * kTile * kTile;
  for (int idx = threadIdx.x; idx < mk * mk; idx += blockDim.x) {
    const int r = idx / mk, col = idx - r * mk;
    double x = diag[(int64_t)r * v.mj + col];
    if (col <= r)
      for (int z = 0; z < splits; ++z) x += part[(int64_t)z * kTile * kTile + r * kTile + col];
    dm[r * kTLD + col] = x;
  }
  __syncthreads();
  cholesky<kTLD>(dm, mk, rinv);
  for (int idx = threadIdx.x; idx < mk * mk; idx += blockDim.x) {
    const int r = idx / mk, col = idx - r * mk;
    diag[(int64_t)r * v.mj + col] = dm[r * kTLD + col];
  }
}

// Tile (i, k) below the diagonal: X = T L_kk^-T, with T = the updated tile (plus the panel
// update's partials when split). Unsplit panels (many tiles) apply L_kk^-1 from the panel's
// diagonal step as one shared-memory GEMM; split panels (few tiles) solve with L_kk by blocked
// substitution. Rows of U_p^T / V_q and of L_j alike.
__global__ void __launch_bounds__(kTT)
tiled_factor_kernel(const int* __restrict__ items, int begin, int k, const int64_t* __restrict__ tasks,
                    double* __restrict__ factors, int64_t stride, int splits,
                    const double* __restrict__ partials, const double* __restrict__ inverses, int t0,
                    int level_tasks) {
  chain_wait();
  extern __shared__ double sm[];
  double* li = sm;                 // L_kk^-1 (unsplit) or L_kk (split)
  double* tt = li + kTile * kTLD;  // transposed tile
  double* xo = tt + kTile * kTLD;  // result (unsplit) or 1 / diag(L_kk) (split)
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  const int seg = it[1], i = it[2];
  if (seg == SEG_J && i == k) return;  // factored by the diagonal step
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int mk = min(kTile, v.mj - kTile * k);
  if (splits == 1) {
    const double* inv = inverses + ((int64_t)blockIdx.y * level_tasks + (it[0] - t0)) * kTile * kTile;
    for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
      const int r = idx / kTile, c = idx - r * kTile;
      li[r * kTLD + c] = inv[idx];
      xo[r * kTLD + c] = 0.0;
    }
  } else {
    const double* diag = f + v.loff + (int64_t)kTile * k * v.mj + kTile * k;
    for (int idx = threadIdx.x; idx < mk * mk; idx += blockDim.x) {
      const int r = idx / mk, c = idx - r * mk;
      li[r * kTLD + c] = diag[(int64_t)r * v.mj + c];
    }
  }
  const int ni = min(kTile, v.rows(seg) - kTile * i);
  const Operand t = v.segment(f, seg, kTile * i, kTile * k);
  double* tb = const_cast<double*>(t.base);
  const double* part = partials + (int64_t)(blockIdx.y * gridDim.x + blockIdx.x) * splits * kTile * kTile;
  for (int idx = threadIdx.x; idx < ni * mk; idx += blockDim.x) {
    const int a = idx / mk, c = idx - a * mk;
    double x = tb[a * t.rs + c * t.cs];
    if (splits > 1)  // the panel update's partials (stored negated), in split order
      for (int z = 0; z < splits; ++z) x += part[(int64_t)z * kTile * kTile + a * kTile + c];
    tt[c * kTLD + a] = x;
  }
  __syncthreads();
  if (splits == 1) {
    tile_gemm<true, true>(xo, kTLD, tt, kTLD, li, kTLD, ni, mk, mk, 1.0);  // X[a][b] = sum_c T[a][c] Linv[b][c]
    __syncthreads();
    for (int idx = threadIdx.x; idx < ni * mk; idx += blockDim.x) {
      const int a = idx / mk, c = idx - a * mk;
      tb[a * t.rs + c * t.cs] = xo[a * kTLD + c];
    }
  } else {
    reciprocal_diagonal(li, kTLD, mk, xo);
    lower_solve(li, kTLD, xo, tt, kTLD, mk, ni);  // L_kk X^T = T^T
    for (int idx = threadIdx.x; idx < ni * mk; idx += blockDim.x) {
      const int a = idx / mk, c = idx - a * mk;
      tb[a * t.rs + c * t.cs] = tt[c * kTLD + a];
    }
  }
}

__global__ void __launch_bounds__(kTT)
tiled_fill_kernel(const int* __restrict__ items, int begin, const int64_t* __restrict__ tasks,
                  double* __restrict__ factors, int64_t stride) {
  chain_wait();
  extern __shared__ double sm[];
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  const int qi = it[1], pi = it[2];
  double* f = factors + (int64_t)blockIdx.y * stride;
  const int nq = min(kTile, v.mq - kTile * qi), np = min(kTile, v.mp - kTile * pi);
  double acc[4][4];
  zero_acc(acc);
  // A[q,p] = -V_q U_p: sum_c V[a][c] U[c][b]
  gemm_nt(acc, operand(f + v.voff + (int64_t)kTile * qi * v.mj, v.mj, 1), nq,
          operand(f + v.uoff + kTile * pi, 1, v.mp), np, v.mj, sm);
  put_acc(acc, f + v.fill + (int64_t)kTile * qi * v.mp + kTile * pi, v.mp, 1, nq, np, false, false);
}

// b_j -= sum of the pulls (U_e^T y_e or V_e y_e) on tile rows i of j, columns [c0, c0 + 16 NQ).
template <int NQ>
__global__ void __launch_bounds__(kTT, 2)
tiled_forward_update_kernel(const int* __restrict__ items, int begin, const int64_t* __restrict__ tasks,
                            const int64_t* __restrict__ pulls, const double* __restrict__ factors,
                            int64_t stride, double* __restrict__ rhs, int64_t rhs_stride, int nrhs) {
  chain_wait();
  extern __shared__ double sm[];
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  if (v.pull0 == v.pull1) return;
  const int i = it[1];
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * 16 * NQ, nc = min(16 * NQ, nrhs - c0);
  const int ni = min(kTile, v.mj - kTile * i);
  double acc[4][NQ];
  zero_acc(acc);
  for (int64_t u = v.pull0; u < v.pull1; ++u) {
    const int64_t* pl = pulls + u * P_FIELDS;
    const int me = (int)pl[P_ME];
    const double* m = f + pl[P_OFF];
    const Operand y = operand(x + pl[P_EOFF] * nrhs + c0, 1, nrhs);
    if (pl[P_TYPE] == 0) gemm_nt(acc, operand(m + kTile * i, 1, v.mj), ni, y, nc, me, sm);
    else gemm_nt(acc, operand(m + (int64_t)kTile * i * me, me, 1), ni, y, nc, me, sm);
  }
  put_acc(acc, x + (int64_t)(v.offj + kTile * i) * nrhs + c0, nrhs, 1, ni, nc, true, false);
}

// y_j -= U_p x_p + V_q^T x_q on tile rows i of j, columns [c0, c0 + 16 NQ).
template <int NQ>
__global__ void __launch_bounds__(kTT, 2)
tiled_backward_update_kernel(const int* __restrict__ items, int begin, const int64_t* __restrict__ tasks,
                             const double* __restrict__ factors, int64_t stride,
                             double* __restrict__ rhs, int64_t rhs_stride, int nrhs) {
  chain_wait();
  extern __shared__ double sm[];
  const int* it = items + 4 * (begin + blockIdx.x);
  const TaskView v(tasks + (int64_t)it[0] * T_FIELDS);
  if (v.p < 0 && v.q < 0) return;
  const int i = it[1];
  const double* f = factors + (int64_t)blockIdx.y * stride;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride;
  const int c0 = blockIdx.z * 16 * NQ, nc = min(16 * NQ, nrhs - c0);
  const int ni = min(kTile, v.mj - kTile * i);
  double acc[4][NQ];
  zero_acc(acc);
  if (v.p >= 0)
    gemm_nt(acc, operand(f + v.uoff + (int64_t)kTile * i * v.mp, v.mp, 1), ni,
            operand(x + (int64_t)v.offp * nrhs + c0, 1, nrhs), nc, v.mp, sm);
  if (v.q >= 0)
    gemm_nt(acc, operand(f + v.voff + kTile * i, 1, v.mj), ni,
            operand(x + (int64_t)v.offq * nrhs + c0, 1, nrhs), nc, v.mq, sm);
  put_acc(acc, x + (int64_t)(v.offj + kTile * i) * nrhs + c0, nrhs, 1, ni, nc, true, false);
}

// Substitutions with L_j on columns [c0, c0 + 16 NQ) of one task: forward (L y = b,
// left-looking over tile rows), and backward (L^T x = y) when `backward`; `forward` may be off.
template <int NQ>
__global__ void __launch_bounds__(kTT)
tiled_substitute_kernel(int task_begin, const int64_t* __restrict__ tasks,
                        const double* __restrict__ factors, int64_t stride, double* __restrict__ rhs,
                        int64_t rhs_stride, int nrhs, int forward, int backward) {
  chain_wait();
  extern __shared__ double sm[];
  double* dm = sm;                 // L_rr
  double* bt = dm + kTile * kTLD;  // right-hand-side rows of tile r
  double* rinv = bt + kTile * kTLD;
  double* gs = rinv + kTile;       // gemm staging
  const TaskView v(tasks + (int64_t)(task_begin + blockIdx.x) * T_FIELDS);
  const double* f = factors + (int64_t)blockIdx.y * stride;
  const double* l = f + v.loff;
  double* x = rhs + (int64_t)blockIdx.y * rhs_stride + (int64_t)v.offj * nrhs;
  const int c0 = blockIdx.z * 16 * NQ, nc = min(16 * NQ, nrhs - c0);
  const int tiles = (v.mj + kTile - 1) / kTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  auto load_diag = [&](int r, int nr) {
    for (int idx = threadIdx.x; idx < nr * nr; idx += blockDim.x) {
      const int a = idx / nr, b = idx - a * nr;
      dm[a * kTLD + b] = l[(int64_t)(kTile * r + a) * v.mj + kTile * r + b];
    }
  };
  // bt = x rows of tile r minus acc
  auto load_rows = [&](int r, int nr, const double (&acc)[4][NQ]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int a = ty + 16 * i;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int b = tx + 16 * q;
        if (a < nr && b < nc) bt[a * kTLD + b] = x[(int64_t)(kTile * r + a) * nrhs + c0 + b] - acc[i][q];
      }
    }
  };
  auto store_rows = [&](int r, int nr) {
    for (int idx = threadIdx.x; idx < nr * nc; idx += blockDim.x) {
      const int a = idx / nc, b = idx - a * nc;
      x[(int64_t)(kTile * r + a) * nrhs + c0 + b] = bt[a * kTLD + b];
    }
  };
  double acc[4][NQ];
  if (forward) {
    for (int r = 0; r < tiles; ++r) {
      const int nr = min(kTile, v.mj - kTile * r);
      zero_acc(acc);
      gemm_nt(acc, operand(l + (int64_t)kTile * r * v.mj, v.mj, 1), nr, operand(x + c0, 1, nrhs), nc,
              kTile * r, gs);
      load_diag(r, nr);
      load_rows(r, nr, acc);
      __syncthreads();
      reciprocal_diagonal(dm, kTLD, nr, rinv);
      lower_solve(dm, kTLD, rinv, bt, kTLD, nr, nc);
      store_rows(r, nr);
      __syncthreads();
    }
  }
  if (backward) {
    for (int r = tiles - 1; r >= 0; --r) {
      const int nr = min(kTile, v.mj - kTile * r);
      const int below = kTile * (r + 1);
      zero_acc(acc);
      if (below < v.mj)  // sum_c L[below + c][64 r + a] x[below + c]
        gemm_nt(acc, operand(l + (int64_t)below * v.mj + kTile * r, 1, v.mj), nr,
                operand(x + (int64_t)below * nrhs + c0, 1, nrhs), nc, v.mj - below, gs);
      load_diag(r, nr);
      load_rows(r, nr, acc);
      __syncthreads();
      reciprocal_diagonal(dm, kTLD, nr, rinv);
      upper_solve(dm, kTLD, rinv, bt, kTLD, nr, nc);
      store_rows(r, nr);
      __syncthreads();
    }
  }
}

constexpr size_t kGemmSmem = sizeof(double) * kStage;
static_assert(kStage >= kTile * kTLD, "the GEMM staging buffer holds the accumulator exchange");
constexpr size_t kUpdateSmem = kGemmSmem + sizeof(double) * (kTile * kTLD + kTile);
constexpr size_t kFactorSmem = sizeof(double) * (2 * kTile * kTLD + kTile);
constexpr size_t kTileSolveSmem = sizeof(double) * 3 * kTile * kTLD;
constexpr size_t kSubstituteSmem = sizeof(double) * (2 * kTile * kTLD + kTile) + kGemmSmem;

void configure_tiled() {
  for (auto kernel : {tiled_update_kernel<4>, tiled_update_kernel<2>, tiled_update_kernel<1>})
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdateSmem);
  cudaFuncSetAttribute(tiled_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSolveSmem);
  cudaFuncSetAttribute(tiled_diagonal_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFactorSmem);
  for (auto kernel : {tiled_substitute_kernel<4>, tiled_substitute_kernel<2>, tiled_substitute_kernel<1>})
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSubstituteSmem);
}

template <typename F>
void with_strip(int nq, F&& f) {
  if (nq == 4) f(std::integral_constant<int, 4>());
  else if (nq == 2) f(std::integral_constant<int, 2>());
  else f(std::integral_constant<int, 1>());
}

// Depth splits of a panel launch of `tiles` items x `systems`: 1 when the launch fills `target`
// block slots (2 x SMs by default: two blocks per SM; 0 never splits), else the largest of 2, 4,
// 8 that keeps it within that. `target` is at most 2 x SMs, so the partials of a split launch
// (tiles x systems x splits <= SMs) fit the plan's workspace of 2 x SMs tiles.
int panel_splits(int tiles, int systems, int64_t target) {
  int splits = 1;
  while (splits < 8 && (int64_t)tiles * systems * splits * 2 <= target) splits *= 2;
  return splits;
}

void factor_tiled(adt_plan* p, int systems, const double* values, double* factors, cudaStream_t s) {
  const int L = p->levels;
  auto range = [&](int r) { return std::make_pair(p->tranges[2 * r], p->tranges[2 * r + 1]); };
  for (int level = 0; level < L; ++level) {
    auto [b, e] = range(level);
    launch_chained(tiled_scatter_kernel, dim3(e - b, systems), kTT, 0, s, p->titems, b, p->tasks, p->csr_ptr, p->csr_row,
                                                             p->csr_col, p->nnz, values, factors, p->factor_stride);
    p->launches++;
    const int t0 = p->level_begin[level], level_tasks = p->level_begin[level + 1] - t0;
    for (int k = 0; k < p->panel_ptr[level + 1] - p->panel_ptr[level]; ++k) {
      const auto [rb, re] = range(3 * L + p->panel_ptr[level] + k);
      const int pb = rb, pe = re;
      if (pe == pb) continue;
      const int splits = panel_splits(pe - pb, systems, (int64_t)p->split_fill * p->sms);
      const int width = p->panel_width[3 * L + p->panel_ptr[level] + k];
      with_strip(width <= 16 ? 1 : width <= 32 ? 2 : 4, [&](auto nq) {
        launch_chained(tiled_update_kernel<nq()>, dim3(pe - pb, systems, splits), kTT, kUpdateSmem, s, p->titems, pb, k,
                       p->tasks, p->pulls, factors, p->factor_stride, splits, p->partials, p->inverses, t0,
                       level_tasks);
      });
      if (splits > 1) {
        launch_chained(tiled_diagonal_kernel, dim3(pe - pb, systems), kTT, kFactorSmem, s, p->titems, pb, k, p->tasks,
                       factors, p->factor_stride, splits, (const double*)p->partials);
        p->launches++;
      }
      launch_chained(tiled_factor_kernel, dim3(pe - pb, systems), kTT, kTileSolveSmem, s, p->titems, pb, k, p->tasks,
                     factors, p->factor_stride, splits, (const double*)p->partials, (const double*)p->inverses, t0,
                     level_tasks);
      p->launches += 2;
    }
    auto [fb, fe] = range(L + level);
    if (fe > fb) {
      launch_chained(tiled_fill_kernel, dim3(fe - fb, systems), kTT, kGemmSmem, s, p->titems, fb, p->tasks, factors,
                                                                       p->factor_stride);
      p->launches++;
    }
  }
}

// Column strip of the tiled solve launches, in units of 16 columns (4: a full tile), narrowed
// while the launch would leave most SMs idle. (Narrowing a launch that fills the GPU to pad
// fewer columns, e.g. 96 as three strips of 32, was measured slower: 32.8 -> 36.8 ms at the
// terrain section.)
int tiled_strip(int blocks, int nrhs, int64_t target) {
  int nq = 4;
  while (nq > 1 && (int64_t)blocks * ((nrhs + 16 * nq - 1) / (16 * nq)) < target) nq /= 2;
  return nq;
}


void solve_tiled(adt_plan* p, int systems, int nrhs, const double* factors, double* rhs, cudaStream_t s) {
  const int L = p->levels;
  const int64_t rhs_stride = (int64_t)p->N * nrhs;
  auto range = [&](int r) { return std::make_pair(p->tranges[2 * r], p->tranges[2 * r + 1]); };
  auto strips = [&](int nq) { return (nrhs + 16 * nq - 1) / (16 * nq); };
  for (int level = 0; level < L; ++level) {
    const auto [rb, re] = range(2 * L + level);
    const int b = rb, e = re;
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    with_strip(tiled_strip((e - b) * systems, nrhs, (int64_t)p->strip_fill * p->sms), [&](auto nq) {
      launch_chained(tiled_forward_update_kernel<nq()>, dim3(e - b, systems, strips(nq())), kTT, kGemmSmem, s,
                     p->titems, b, p->tasks, p->pulls, factors, p->factor_stride, rhs, rhs_stride, nrhs);
    });
    with_strip(tiled_strip((t1 - t0) * systems, nrhs, (int64_t)p->strip_fill * p->sms), [&](auto nq) {
      launch_chained(tiled_substitute_kernel<nq()>, dim3(t1 - t0, systems, strips(nq())), kTT, kSubstituteSmem, s,
                     t0, p->tasks, factors, p->factor_stride, rhs, rhs_stride, nrhs, 1, level == L - 1);
    });
    p->launches += 2;
  }
  for (int level = L - 2; level >= 0; --level) {
    const auto [rb, re] = range(2 * L + level);
    const int b = rb, e = re;
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    with_strip(tiled_strip((e - b) * systems, nrhs, (int64_t)p->strip_fill * p->sms), [&](auto nq) {
      launch_chained(tiled_backward_update_kernel<nq()>, dim3(e - b, systems, strips(nq())), kTT, kGemmSmem, s,
                     p->titems, b, p->tasks, factors, p->factor_stride, rhs, rhs_stride, nrhs);
    });
    with_strip(tiled_strip((t1 - t0) * systems, nrhs, (int64_t)p->strip_fill * p->sms), [&](auto nq) {
      launch_chained(tiled_substitute_kernel<nq()>, dim3(t1 - t0, systems, strips(nq())), kTT, kSubstituteSmem, s,
                     t0, p->tasks, factors, p->factor_stride, rhs, rhs_stride, nrhs, 0, 1);
    });
    p->launches += 2;
  }
}

template <int MAXM>
void configure() {
  cudaFuncSetAttribute(invert_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)invert_smem<MAXM>());
  if constexpr (3 * MAXM > kNarrowColumns)
    cudaFuncSetAttribute(invert_level_kernel<MAXM, kNarrowColumns>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)invert_smem<MAXM, kNarrowColumns>());
  cudaFuncSetAttribute(update_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)update_smem<MAXM>());
  cudaFuncSetAttribute(forward_update_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)forward_update_smem<MAXM>());
  cudaFuncSetAttribute(backward_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)backward_smem<MAXM>());
  cudaFuncSetAttribute(update_rhs_level_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)update_smem<MAXM>());
}

// One level of inversions: the narrow column capacity when every augmented row fits in it.
template <int MAXM>
void launch_invert(adt_plan* p, int t0, int t1, int systems, const double* values, double* factors, cudaStream_t s) {
  if constexpr (3 * MAXM > kNarrowColumns) {
    if (p->max_width <= kNarrowColumns) {
      launch_chained(invert_level_kernel<MAXM, kNarrowColumns>, dim3(t1 - t0, systems), kSolverThreads,
                     invert_smem<MAXM, kNarrowColumns>(), s, p->tasks, t0, p->csr_ptr, p->csr_row, p->csr_col,
                     p->nnz, values, factors, p->factor_stride);
      return;
    }
  }
  launch_chained(invert_level_kernel<MAXM>, dim3(t1 - t0, systems), kSolverThreads, invert_smem<MAXM>(), s,
                 p->tasks, t0, p->csr_ptr, p->csr_row, p->csr_col, p->nnz, values, factors, p->factor_stride);
}

template <int MAXM>
void factor_levels(adt_plan* p, int systems, const double* values, double* factors, cudaStream_t s) {
  const int tasks = p->level_begin[p->levels];
  launch_chained(scatter_diagonal_kernel, dim3(tasks, systems), kSolverThreads, 0, s, 
      p->tasks, p->csr_ptr, p->csr_row, p->csr_col, p->nnz, values, factors, p->factor_stride);
  p->launches++;
  for (int level = 0; level < p->levels; ++level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    launch_invert<MAXM>(p, t0, t1, systems, values, factors, s);
    p->launches++;
    const int i0 = p->update_begin[level], i1 = p->update_begin[level + 1];
    if (i1 > i0) {
      launch_chained(update_level_kernel<MAXM>, dim3(i1 - i0, systems), kSolverThreads, update_smem<MAXM>(), s, 
          p->update_items, i0, p->tasks, p->pulls, factors, p->factor_stride);
      p->launches++;
    }
  }
}

// factor_levels with the forward substitution of `rhs` (nrhs <= MAXM columns per system) fused
// into the Schur-update launches.
template <int MAXM>
void factor_levels_rhs(adt_plan* p, int systems, const double* values, double* factors, double* rhs, int nrhs,
                       cudaStream_t s) {
  const int tasks = p->level_begin[p->levels];
  const int64_t rhs_stride = (int64_t)p->N * nrhs;
  launch_chained(scatter_diagonal_kernel, dim3(tasks, systems), kSolverThreads, 0, s,
      p->tasks, p->csr_ptr, p->csr_row, p->csr_col, p->nnz, values, factors, p->factor_stride);
  p->launches++;
  for (int level = 0; level < p->levels; ++level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    launch_invert<MAXM>(p, t0, t1, systems, values, factors, s);
    p->launches++;
    const int i0 = p->update_begin[level], i1 = p->update_begin[level + 1];
    if (i1 > i0) {
      launch_chained(update_rhs_level_kernel<MAXM>, dim3(i1 - i0, systems), kSolverThreads, update_smem<MAXM>(), s,
          p->update_items, i0, p->tasks, p->pulls, factors, p->factor_stride, rhs, rhs_stride, nrhs);
      p->launches++;
    }
  }
}

// Column strip of the substitution kernels: the full tile unless the launch would have fewer
// than `target` blocks (2 x SMs by default).
template <int MAXM>
int strip_for(int blocks, int nrhs, int64_t target) {
  int strip = MAXM;
  while (strip > 16 && (int64_t)blocks * ((nrhs + strip - 1) / strip) < target) strip /= 2;
  return strip;
}

// The backward levels alone (the right-hand side already forward-reduced).
template <int MAXM>
void backward_levels(adt_plan* p, int systems, int nrhs, const double* factors, double* rhs, cudaStream_t s) {
  const int64_t rhs_stride = (int64_t)p->N * nrhs;
  for (int level = p->levels - 1; level >= 0; --level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    const int strip = strip_for<MAXM>((t1 - t0) * systems, nrhs, (int64_t)p->strip_fill * p->sms);
    launch_chained(backward_level_kernel<MAXM>, dim3(t1 - t0, systems, (nrhs + strip - 1) / strip), kSolverThreads,
                   backward_smem<MAXM>(), s, p->tasks, t0, factors, p->factor_stride, rhs, rhs_stride, nrhs, strip);
    p->launches++;
  }
}

template <int MAXM>
void solve_levels(adt_plan* p, int systems, int nrhs, const double* factors, double* rhs, cudaStream_t s) {
  const int64_t rhs_stride = (int64_t)p->N * nrhs;
  for (int level = 0; level < p->levels; ++level) {  // forward: eager updates only
    const int i0 = p->update_begin[level], i1 = p->update_begin[level + 1];
    if (i1 <= i0) continue;
    const int strip = strip_for<MAXM>((i1 - i0) * systems, nrhs, (int64_t)p->strip_fill * p->sms);
    launch_chained(forward_update_kernel<MAXM>, dim3(i1 - i0, systems, (nrhs + strip - 1) / strip), kSolverThreads, forward_update_smem<MAXM>(), s, 
        p->update_items, i0, p->tasks, p->pulls, factors, p->factor_stride, rhs, rhs_stride, nrhs, strip);
    p->launches++;
  }
  for (int level = p->levels - 1; level >= 0; --level) {
    const int t0 = p->level_begin[level], t1 = p->level_begin[level + 1];
    const int strip = strip_for<MAXM>((t1 - t0) * systems, nrhs, (int64_t)p->strip_fill * p->sms);
    launch_chained(backward_level_kernel<MAXM>, dim3(t1 - t0, systems, (nrhs + strip - 1) / strip), kSolverThreads,
                   backward_smem<MAXM>(), s, p->tasks, t0, factors, p->factor_stride, rhs, rhs_stride, nrhs, strip);
    p->launches++;
  }
}

}  // namespace

// Opt the solver kernels in to their dynamic shared memory on the current device.
void configure_solver_kernels() {
  configure_tiled();
  configure<32>();
  configure<48>();
  configure<64>();
}

adt_status factorize_systems(adt_plan* p, int systems, const double* values, double* factors,
                             cudaStream_t s) {
  if (p->tiled) {
    // L_kk^-1 of every task of a level and system, for the panels' triangular solves
    int widest = 0;
    for (int level = 0; level < p->levels; ++level)
      widest = std::max(widest, p->level_begin[level + 1] - p->level_begin[level]);
    const size_t need = (size_t)widest * systems * kTile * kTile;
    if (p->inverses_capacity < need) {
      if (p->inverses) cudaFree(p->inverses);
      p->inverses = nullptr;
      p->inverses_capacity = 0;
      if (cudaMalloc(&p->inverses, need * sizeof(double)) != cudaSuccess)
        return fail(p, ADT_OOM, "tiled solver workspace allocation failed");
      p->inverses_capacity = need;
    }
    factor_tiled(p, systems, values, factors, s);
  }
  else if (p->max_m <= 32) factor_levels<32>(p, systems, values, factors, s);
  else if (p->max_m <= 48) factor_levels<48>(p, systems, values, factors, s);
  else factor_levels<64>(p, systems, values, factors, s);
  return check_launch(p, "factorization");
}

adt_status solve_systems(adt_plan* p, int systems, int nrhs, const double* factors,
                         double* rhs, cudaStream_t s) {
  if (p->tiled) solve_tiled(p, systems, nrhs, factors, rhs, s);
  else if (p->max_m <= 32) solve_levels<32>(p, systems, nrhs, factors, rhs, s);
  else if (p->max_m <= 48) solve_levels<48>(p, systems, nrhs, factors, rhs, s);
  else solve_levels<64>(p, systems, nrhs, factors, rhs, s);
  return check_launch(p, "solve");
}

// Whether the field right-hand side can be forward-reduced during the factorization: the
// shared-memory solver, and nrhs within its block width.
bool fused_rhs_supported(const adt_plan* p, int nrhs) {
  const int width = p->max_m <= 32 ? 32 : p->max_m <= 48 ? 48 : 64;
  return !p->tiled && nrhs <= width;
}

adt_status factorize_systems_rhs(adt_plan* p, int systems, const double* values, double* factors, double* rhs,
                                 int nrhs, cudaStream_t s) {
  if (!fused_rhs_supported(p, nrhs)) return fail(p, ADT_INVALID_ARG, "fused right-hand side not supported");
  if (p->max_m <= 32) factor_levels_rhs<32>(p, systems, values, factors, rhs, nrhs, s);
  else if (p->max_m <= 48) factor_levels_rhs<48>(p, systems, values, factors, rhs, nrhs, s);
  else factor_levels_rhs<64>(p, systems, values, factors, rhs, nrhs, s);
  return check_launch(p, "factorization with right-hand side");
}

adt_status backward_systems(adt_plan* p, int systems, int nrhs, const double* factors, double* rhs, cudaStream_t s) {
  if (!fused_rhs_supported(p, nrhs)) return fail(p, ADT_INVALID_ARG, "fused right-hand side not supported");
  if (p->max_m <= 32) backward_levels<32>(p, systems, nrhs, factors, rhs, s);
  else if (p->max_m <= 48) backward_levels<48>(p, systems, nrhs, factors, rhs, s);
  else backward_levels<64>(p, systems, nrhs, factors, rhs, s);
  return check_launch(p, "backward substitution");
}

}  // namespace adt
