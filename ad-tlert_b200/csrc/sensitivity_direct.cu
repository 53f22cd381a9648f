// Normal-quadrupole Jacobian of single-wavenumber operators (3D), in direct form.
//
// With one wavenumber the per-cell features F[e] = s * Ls x_e (x_e = fields[dofs(c)][e], R
// features per cell) give every row without an electrode Gram:
//   J[d][c] = -sum_f (F[M] - F[N])_f (F[A] - F[B])_f      (column E = remote = 0),
// R products per entry against the Gram's E(E+1)/2 * R per cell. The Gram kernel stays the
// choice for the 17-wavenumber 2.5D operator, where the Gram's products are shared by all rows.
//
// A block owns CB consecutive cells (CB = 32, 16, 8 or 4). It forms the features of all E
// columns of its cells in shared memory, column-major by cell ([col][f][cell], odd column
// stride), so that a group of CB lanes reading one (column, feature) reads CB consecutive words.
// Each warp holds 32/CB row slots; a slot walks a contiguous range of the rows sorted by current
// pair (A, B) (the plan's packed row entries: ABMN bytes and the output row, one 8-byte load per
// row), keeping F[A] - F[B] in registers while the pair repeats, and its CB lanes store
// CB consecutive floats of the row: every store covers whole 32-byte sectors, so a Jacobian much
// larger than L2 is written once to DRAM instead of read-modified-written sector by sector.
// Equals the reference's per-entry contraction (adtlert/forward/kernels.py:132-178, called by
// adtlert/forward/ert3d.py:867-927) up to rounding.
#include "adt_internal.h"
#include "kernels.h"

namespace adt {

constexpr int kDirectThreads = 512;
constexpr int kDirectMaxR = 16;

// Shared memory of jacobian_direct_kernel for CB cells per block.
size_t jacobian_direct_smem(int cells, int R, int E, int K) {
  const size_t stride = (size_t)R * cells + 1;
  return sizeof(float) * ((size_t)(E + 1) * stride + (size_t)cells * R * K) + sizeof(int) * (size_t)cells * K;
}

template <int KC, int RC, int CBC>
__global__ void __launch_bounds__(kDirectThreads, 2)
    jacobian_direct_kernel(JacobianArgs a, const int2* rows) {
  chain_wait();
  extern __shared__ float dsm[];
  const int K = KC > 0 ? KC : a.K;
  const int R = RC > 0 ? RC : a.R;
  constexpr int KMAX = KC > 0 ? KC : 16;
  constexpr int RMAX = RC > 0 ? RC : kDirectMaxR;
  const int CB = CBC > 0 ? CBC : a.cells_per_block, E = a.E;
  const int S = R * CB + 1;  // column stride (odd)
  float* feat = dsm;                         // [E + 1][S]
  float* coef = feat + (size_t)(E + 1) * S;  // [CB][R][K]
  int* dofs = reinterpret_cast<int*>(coef + CB * R * K);  // [CB][K]
  const int c0 = a.c_begin + blockIdx.x * CB;
  const int ncells = min(CB, a.c_end - c0);
  const int tid = threadIdx.x;

  for (int i = tid; i < CB * R * K; i += kDirectThreads) {
    const int c = min(c0 + i / (R * K), a.c_end - 1);
    coef[i] = a.features[(int64_t)c * R * K + i % (R * K)];
  }
  for (int i = tid; i < CB * K; i += kDirectThreads) {
    const int c = c0 + i / K;
    dofs[i] = c < a.c_end ? a.cell_dofs[(int64_t)c * K + i % K] : -1;
  }
  for (int i = tid; i < R * CB; i += kDirectThreads) feat[E * S + i] = 0.f;  // remote column
  __syncthreads();

  // features: item (cell, column), columns fastest so the field loads of a dof are coalesced
  for (int item = tid; item < CB * E; item += kDirectThreads) {
    const int cell = item / E, col = item - cell * E;
    float x[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      float v = 0.f;
      if (KC > 0 || k < K) {
        const int dof = dofs[cell * K + k];
        if (dof >= 0) v = __ldg(a.fields + (int64_t)dof * E + col);
      }
      x[k] = v;
    }
    const float* cf = coef + cell * R * K;
#pragma unroll
    for (int f = 0; f < RMAX; ++f) {
      if (RC == 0 && f >= R) break;
      float v = 0.f;
#pragma unroll
      for (int k = 0; k < KMAX; ++k)
        if (KC > 0 || k < K) v = fmaf(cf[f * K + k], x[k], v);
      feat[col * S + f * CB + cell] = v * __ldg(a.fscale + f);
    }
  }
  __syncthreads();

  // rows: slot = (warp, lane / CB), cell = lane % CB; a row entry is (A | B << 8 | M << 16 |
  // N << 24, measurement row d), stored at out[(d - row_begin) * ldo]
  const int lane = tid & 31, per_warp = 32 / CB;
  const int slots = (kDirectThreads / 32) * per_warp;
  const int slot = (tid >> 5) * per_warp + lane / CB;
  const int cell = lane % CB;
  const int begin = (int)((int64_t)a.rows * slot / slots), end = (int)((int64_t)a.rows * (slot + 1) / slots);
  const float* fc = feat + cell;
  float* out = a.out + c0 + cell;
  const bool store = cell < ncells;
  int pair = -1;
  float dab[RMAX];
#pragma unroll
  for (int f = 0; f < RMAX; ++f) dab[f] = 0.f;
  auto entry = [&](const int2 r) {
    if ((r.x & 0xffff) != pair) {
      pair = r.x & 0xffff;
      const float* pa = fc + (r.x & 0xff) * S;
      const float* pb = fc + ((r.x >> 8) & 0xff) * S;
#pragma unroll
      for (int f = 0; f < RMAX; ++f) {
        if (RC == 0 && f >= R) break;
        dab[f] = pa[f * CB] - pb[f * CB];
      }
    }
    const float* pm = fc + ((r.x >> 16) & 0xff) * S;
    const float* pn = fc + ((unsigned)r.x >> 24) * S;
    float v = 0.f;
#pragma unroll
    for (int f = 0; f < RMAX; ++f) {
      if (RC == 0 && f >= R) break;
      v = fmaf(pm[f * CB] - pn[f * CB], dab[f], v);
    }
    return -v;
  };
  int i = begin;
  for (; i + 1 < end; i += 2) {
    const int2 r0 = __ldg(rows + i), r1 = __ldg(rows + i + 1);
    const float v0 = entry(r0), v1 = entry(r1);
    if (store) {
      out[(int64_t)(r0.y - a.row_begin) * a.ldo] = v0;
      out[(int64_t)(r1.y - a.row_begin) * a.ldo] = v1;
    }
  }
  if (i < end) {
    const int2 r0 = __ldg(rows + i);
    const float v0 = entry(r0);
    if (store) out[(int64_t)(r0.y - a.row_begin) * a.ldo] = v0;
  }
}

// Largest cells-per-block (32, 16, 8, 4) whose shared memory fits two blocks per SM; 0 if none
// (or if a column index does not fit the 8-bit fields of a packed row entry).
int jacobian_direct_cells(int R, int E, int K) {
  if (R > kDirectMaxR || K > 16 || E > 255) return 0;
  for (int cells = 32; cells >= 4; cells /= 2)
    if (jacobian_direct_smem(cells, R, E, K) <= 110 * 1024) return cells;
  return 0;
}

cudaError_t launch_jacobian_direct(const JacobianArgs& a, const int2* rows, cudaStream_t s) {
  const size_t smem = jacobian_direct_smem(a.cells_per_block, a.R, a.E, a.K);
  const int blocks = (a.c_end - a.c_begin + a.cells_per_block - 1) / a.cells_per_block;
  auto go = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_chained(kernel, blocks, kDirectThreads, smem, s, a, rows);
    return cudaGetLastError();
  };
  if (a.K == 4 && a.R == 3 && a.cells_per_block == 32) return go(jacobian_direct_kernel<4, 3, 32>);
  if (a.K == 10 && a.R == 9 && a.cells_per_block == 8) return go(jacobian_direct_kernel<10, 9, 8>);
  return go(jacobian_direct_kernel<0, 0, 0>);
}

}  // namespace adt
