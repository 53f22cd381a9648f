// Sensitivity contractions: the normal-quadrupole Jacobian and the per-cell adjoint gradients.
//
// Jacobian. For every discretization cell c, the unit templates factor as K_c = Ls^T Ls and
// M_c = Lm^T Lm (computed once on the host), so with per-wavenumber features
//   F_w[e] = ( sqrt(w_w) Ls x_we ; sqrt(w_w) k_w Lm x_we ),   x_we = fields_w[dofs(c)][e],
// the electrode Gram G_c[e][f] = sum_w F_w[e] . F_w[f] = sum_w w_w x_we^T (K_c + k_w^2 M_c) x_wf,
// and every ABMN row is four Gram entries:
//   J[d][c] = -(G[M][A] - G[M][B] - G[N][A] + G[N][B])      (slot E = remote = 0).
// A block owns `cells_per_block` cells; each thread accumulates 4x4 tiles of the upper triangle
// of some cells' Grams in registers (fixed wavenumber/feature order: bitwise repeatable), the
// packed Grams go to shared memory, and the rows are gathered so that a warp writes contiguous
// cells of one row. This replaces the per-entry serial contraction of the reference kernel
// (adtlert/forward/kernels.py:132-178), whose result it equals up to rounding.
#include "adt_internal.h"
#include "kernels.h"

namespace adt {

constexpr int kJacThreads = 256;
constexpr int kJacJobs = 5;   // 4x4 Gram tiles per thread
constexpr int kJacItems = 4;  // feature items (cell, electrode) per thread and wavenumber

// Dynamic shared memory of jacobian_kernel for `cells` cells per block: two feature buffers
// (wavenumbers w and w+1) and the packed upper-triangular Grams.
size_t jacobian_smem(int cells, int R, int E, int K) {
  const int E4 = (E + 3) & ~3;
  const size_t gram = (size_t)(E * (E + 1) / 2) | 1;  // odd stride: conflict-free across cells
  return sizeof(float) * (2 * (size_t)cells * R * E4 + (size_t)cells * gram +
                          (size_t)cells * R * K + (size_t)cells * K);
}

__device__ __forceinline__ int packed_index(int i, int j, int E) {
  // i <= j < E, row-major upper triangle
  return i * E - (i * (i - 1)) / 2 + (j - i);
}

// K local dofs and R features per cell and wavenumber are compile-time (K = R = 0: runtime).
template <int KC, int RC>
__global__ void __launch_bounds__(kJacThreads, 2) jacobian_kernel(JacobianArgs a) {
  chain_wait();
  extern __shared__ float jsm[];
  const int K = KC > 0 ? KC : a.K;
  const int R = RC > 0 ? RC : a.R;
  constexpr int KMAX = KC > 0 ? KC : 16;
  const int CT = a.cells_per_block;
  const int E = a.E, E4 = (E + 3) & ~3;
  const int nt4 = E4 / 4;
  const int NT = nt4 * (nt4 + 1) / 2;
  const int P = (E * (E + 1) / 2) | 1;  // packed Gram stride (odd: cells hit distinct banks)
  const int fsize = CT * R * E4;
  float* gram = jsm + 2 * fsize;  // [CT][P]
  const int c0 = a.c_begin + blockIdx.x * CT;
  const int tid = threadIdx.x;

  // this thread's Gram tiles: smem offsets of the two 4-electrode strips they multiply (-1: none)
  int off_u[kJacJobs], off_v[kJacJobs];
#pragma unroll
  for (int j = 0; j < kJacJobs; ++j) {
    const int job = tid + j * kJacThreads;
    off_u[j] = off_v[j] = -1;
    if (job < CT * NT) {
      const int cell = job / NT;
      int t = job - cell * NT, ti = 0, len = nt4;
      while (t >= len) { t -= len; ++ti; --len; }
      off_u[j] = cell * R * E4 + 4 * ti;
      off_v[j] = cell * R * E4 + 4 * (ti + t);
    }
  }
  // feature stage: threads are cell-major (TPC threads per cell, strided electrodes); the block's
  // template factors and cell dofs are staged in shared memory once
  float* coef = gram + CT * P;                           // [CT][R][K]
  int* dofs = reinterpret_cast<int*>(coef + CT * R * K);  // [CT][K]
  for (int i = tid; i < CT * R * K; i += kJacThreads) {
    const int c = min(c0 + i / (R * K), a.c_end - 1);
    coef[i] = a.features[(int64_t)c * R * K + i % (R * K)];
  }
  for (int i = tid; i < CT * K; i += kJacThreads) {
    const int c = c0 + i / K;
    dofs[i] = c < a.c_end ? a.cell_dofs[(int64_t)c * K + i % K] : -1;
  }
  const int TPC = kJacThreads / CT;
  const int my_cell = tid / TPC, my_eg = tid - my_cell * TPC;
  float acc[kJacJobs][16];
#pragma unroll
  for (int j = 0; j < kJacJobs; ++j)
#pragma unroll
    for (int r = 0; r < 16; ++r) acc[j][r] = 0.f;
  __syncthreads();

  float xv[kJacItems][KMAX];
  auto fetch = [&](int w) {
    const float* fw = a.fields + (int64_t)w * a.N * E;
#pragma unroll
    for (int it = 0; it < kJacItems; ++it) {
      const int e = my_eg + it * TPC;
#pragma unroll
      for (int k = 0; k < KMAX; ++k) {
        float v = 0.f;
        if (KC > 0 || k < K) {
          const int dof = dofs[my_cell * K + k];
          if (dof >= 0 && e < E) v = __ldg(fw + (int64_t)dof * E + e);
        }
        xv[it][k] = v;
      }
    }
  };
  auto features = [&](int w, float* buf) {
    const float* cf = coef + my_cell * R * K;
    const float* sc = a.fscale + w * R;
#pragma unroll
    for (int it = 0; it < kJacItems; ++it) {
      const int e = my_eg + it * TPC;
      if (e >= E4) continue;
#pragma unroll
      for (int f = 0; f < (RC > 0 ? RC : 32); ++f) {
        if (RC == 0 && f >= R) break;
        float v = 0.f;
#pragma unroll
        for (int k = 0; k < KMAX; ++k)
          if (KC > 0 || k < K) v = fmaf(cf[f * K + k], xv[it][k], v);
        buf[(my_cell * R + f) * E4 + e] = v * __ldg(sc + f);
      }
    }
  };

  fetch(0);
  features(0, jsm);
  __syncthreads();
  for (int w = 0; w < a.W; ++w) {
    const float* cur = jsm + (w & 1) * fsize;
    if (w + 1 < a.W) fetch(w + 1);  // loads in flight during the tile products
#pragma unroll
    for (int j = 0; j < kJacJobs; ++j) {
      if (off_u[j] < 0) continue;
      const float* pu = cur + off_u[j];
      const float* pv = cur + off_v[j];
#pragma unroll
      for (int f = 0; f < (RC > 0 ? RC : 32); ++f) {
        if (RC == 0 && f >= R) break;
        const float4 u = *reinterpret_cast<const float4*>(pu + f * E4);
        const float4 v = *reinterpret_cast<const float4*>(pv + f * E4);
        const float ua[4] = {u.x, u.y, u.z, u.w};
        const float va[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[j][r * 4 + s] = fmaf(ua[r], va[s], acc[j][r * 4 + s]);
      }
    }
    if (w + 1 < a.W) features(w + 1, jsm + ((w + 1) & 1) * fsize);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < kJacJobs; ++j) {
    if (off_u[j] < 0) continue;
    const int job = tid + j * kJacThreads;
    const int cell = job / NT;
    int t = job - cell * NT, ti = 0, len = nt4;
    while (t >= len) { t -= len; ++ti; --len; }
    float* g = gram + cell * P;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int i = 4 * ti + r, k = 4 * (ti + t) + s;
        if (i <= k && k < E) g[packed_index(i, k, E)] = acc[j][r * 4 + s];
      }
  }
  __syncthreads();
  // rows go to groups of CT threads (CT is a power of two <= 32); thread ci of a group reads cell
  // ci's four Gram entries, so a group stores CT contiguous floats of one row
  const int ncells = min(CT, a.c_end - c0);
  const int ci = tid % CT;
  for (int dl = tid / CT; dl < a.rows; dl += kJacThreads / CT) {
    const int4 q = *reinterpret_cast<const int4*>(a.abmn + 4 * (a.row_begin + dl));
    auto index = [&](int i, int k) -> int {
      if (i >= E || k >= E) return -1;
      return i <= k ? packed_index(i, k, E) : packed_index(k, i, E);
    };
    const int ima = index(q.z, q.x), imb = index(q.z, q.y), ina = index(q.w, q.x), inb = index(q.w, q.y);
    if (ci < ncells) {
      const float* g = gram + ci * P;
      const float ma = ima >= 0 ? g[ima] : 0.f, mb = imb >= 0 ? g[imb] : 0.f;
      const float na = ina >= 0 ? g[ina] : 0.f, nb = inb >= 0 ? g[inb] : 0.f;
      a.out[(int64_t)dl * a.ldo + c0 + ci] = -((ma - mb) - (na - nb));
    }
  }
}

template __global__ void jacobian_kernel<3, 5>(JacobianArgs);
template __global__ void jacobian_kernel<4, 3>(JacobianArgs);
template __global__ void jacobian_kernel<3, 6>(JacobianArgs);
template __global__ void jacobian_kernel<4, 7>(JacobianArgs);
template __global__ void jacobian_kernel<4, 8>(JacobianArgs);
template __global__ void jacobian_kernel<0, 0>(JacobianArgs);

// Launch the instantiation matching the plan's (K, R).
cudaError_t launch_jacobian(const JacobianArgs& a, size_t smem, cudaStream_t s) {
  const int blocks = (a.c_end - a.c_begin + a.cells_per_block - 1) / a.cells_per_block;
  auto go = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_chained(kernel, blocks, kJacThreads, smem, s, a);
    return cudaGetLastError();
  };
  if (a.K == 3 && a.R == 5) return go(jacobian_kernel<3, 5>);
  if (a.K == 4 && a.R == 3) return go(jacobian_kernel<4, 3>);
  if (a.K == 3 && a.R == 6) return go(jacobian_kernel<3, 6>);
  if (a.K == 4 && a.R == 7) return go(jacobian_kernel<4, 7>);
  if (a.K == 4 && a.R == 8) return go(jacobian_kernel<4, 8>);
  return go(jacobian_kernel<0, 0>);
}

// One warp per (cotangent q, cell): g[q][c] = -sum_w sum_e x_we^T (K + k_w^2 M) y_we over the
// cell's dofs (x scaled by x_scale[w], y by y_scale[w]), plus the mixed-boundary term
// -sum_w sum_e x^T (alpha_w[b] Mb) y over the cell's boundary elements when `robin`.
// Lanes own electrodes; the lane sums are combined by a fixed shuffle tree. KT > 0 fixes the
// element's dof count at compile time (P1 triangles and tetrahedra, Q1 quads: the dof values
// stay in registers); KT = 0 takes a.K.
// Replaces _cell_gradient (adtlert/forward/ert2p5d.py:765-825).
template <int KT>
__global__ void __launch_bounds__(256, 3) cell_gradient_kernel_t(CellGradientArgs a) {
  chain_wait();
  const int warps = blockDim.x / 32;
  const int64_t warp_id = (int64_t)blockIdx.x * warps + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  const int64_t count = (int64_t)a.models * a.q_per_model;
  if (warp_id >= count * a.C) return;
  const int q = (int)(warp_id / a.C), c = (int)(warp_id % a.C);
  const int s = q / a.q_per_model, ql = q % a.q_per_model;
  const int K = KT > 0 ? KT : a.K, K2 = K * K;
  constexpr int KA = KT > 0 ? KT : 16;
  const int* dofs = a.cell_dofs + (int64_t)c * K;
  double acc = 0.0;
  for (int w = 0; w < a.W; ++w) {
    const int64_t t = (int64_t)s * a.W + w;
    const double xs = a.x_scale ? a.x_scale[w] : 1.0;
    const double ys = a.y_scale ? a.y_scale[w] : 1.0;
    const double k2 = a.k2[w];
    for (int e = lane; e < a.E; e += 32) {
      double xv[KA], yv[KA];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int64_t xi = (t * a.N + dofs[k]) * a.x_cols + (int64_t)ql * a.E + e;
        const int64_t yi = (t * a.N + dofs[k]) * a.E + e;
        xv[k] = xs * (a.x_double ? ((const double*)a.x)[xi] : (double)((const float*)a.x)[xi]);
        yv[k] = ys * (a.y_double ? ((const double*)a.y)[yi] : (double)((const float*)a.y)[yi]);
      }
      const double* st = a.stiffness + (int64_t)c * K2;
      const double* ms = a.mass + (int64_t)c * K2;
      double sum = 0.0;
#pragma unroll
      for (int i = 0; i < K; ++i) {
        double row = 0.0;
#pragma unroll
        for (int j = 0; j < K; ++j) row += (st[i * K + j] + k2 * ms[i * K + j]) * yv[j];
        sum += xv[i] * row;
      }
      if (a.robin) {
        for (int bi = a.cell_bptr[c]; bi < a.cell_bptr[c + 1]; ++bi) {
          const int b = a.cell_blist[bi];
          const double alpha = a.bcoef[(int64_t)w * a.Nb + b];
          const int* bd = a.bdofs + (int64_t)b * a.BL;
          const double* bm = a.bmass + (int64_t)b * a.BL * a.BL;
          for (int i = 0; i < a.BL; ++i) {
            const int64_t xi = (t * a.N + bd[i]) * a.x_cols + (int64_t)ql * a.E + e;
            const double xb = xs * (a.x_double ? ((const double*)a.x)[xi] : (double)((const float*)a.x)[xi]);
            double row = 0.0;
            for (int j = 0; j < a.BL; ++j) {
              const int64_t yi = (t * a.N + bd[j]) * a.E + e;
              const double yb = ys * (a.y_double ? ((const double*)a.y)[yi] : (double)((const float*)a.y)[yi]);
              row += alpha * bm[i * a.BL + j] * yb;
            }
            sum += xb * row;
          }
        }
      }
      acc += sum;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (lane == 0) a.out[(int64_t)q * a.C + c] = -acc;
}

cudaError_t launch_cell_gradient(const CellGradientArgs& a, int blocks, cudaStream_t s) {
  switch (a.K) {
    case 3: return launch_chained(cell_gradient_kernel_t<3>, blocks, 256, 0, s, a);
    case 4: return launch_chained(cell_gradient_kernel_t<4>, blocks, 256, 0, s, a);
    default: return launch_chained(cell_gradient_kernel_t<0>, blocks, 256, 0, s, a);
  }
}

// Mixed-boundary part of the Jacobian, added to rows already holding the volume part: one thread
// per (row, boundary-owning cell) sums, over the cell's boundary elements in list order,
//   sum_w weight_w alpha_w[b] (u_M - u_N)_b^T Mb[b] (u_A - u_B)_b          (slot E = remote = 0)
// and subtracts it from out[row][cell]. This is the Robin template of the reference's cell
// templates (adtlert/forward/ert3d.py:224-256, used by jacobian at 867-927).
__global__ void boundary_jacobian_kernel(BoundaryJacobianArgs a) {
  chain_wait();
  const int64_t total = (int64_t)a.rows * a.owner_count;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int dl = (int)(idx / a.owner_count), c = a.owners[idx % a.owner_count];
    const int* q = a.abmn + 4 * (a.row_begin + dl);
    const int A = q[0], B = q[1], M = q[2], Nn = q[3];
    double acc = 0.0;
    for (int w = 0; w < a.W; ++w) {
      const float* f = a.fields + (int64_t)w * a.N * a.E;
      auto at = [&](int dof, int e) -> double { return e < a.E ? (double)f[(int64_t)dof * a.E + e] : 0.0; };
      for (int bi = a.cell_bptr[c]; bi < a.cell_bptr[c + 1]; ++bi) {
        const int b = a.cell_blist[bi];
        const int* bd = a.bdofs + (int64_t)b * a.BL;
        const double* bm = a.bmass + (int64_t)b * a.BL * a.BL;
        double sum = 0.0;
        for (int i = 0; i < a.BL; ++i) {
          const double v = at(bd[i], M) - at(bd[i], Nn);
          double row = 0.0;
          for (int j = 0; j < a.BL; ++j) row += bm[i * a.BL + j] * (at(bd[j], A) - at(bd[j], B));
          sum += v * row;
        }
        acc += a.weights[w] * a.bcoef[(int64_t)w * a.Nb + b] * sum;
      }
    }
    float* o = a.out + (int64_t)dl * a.C + c;
    *o = (float)((double)*o - acc);
  }
}

// values[r][c] *= row_scale[r] * column_scale[c] (null scales are ones).
__global__ void scale_rows_columns_kernel(float* values, int rows, int columns, const double* row_scale,
                                          const double* column_scale) {
  chain_wait();
  const int64_t total = (int64_t)rows * columns;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / columns), c = (int)(idx - (int64_t)r * columns);
    double v = values[idx];
    if (row_scale) v *= row_scale[r];
    if (column_scale) v *= column_scale[c];
    values[idx] = (float)v;
  }
}

// y += x elementwise.
__global__ void add_kernel(double* y, const double* x, int64_t count) {
  chain_wait();
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < count;
       idx += (int64_t)gridDim.x * blockDim.x)
    y[idx] += x[idx];
}

// x[w][row][e] = 0 for the listed rows (the fixed dofs of a Dirichlet boundary).
__global__ void zero_rows_kernel(double* x, const int* rows, int count, int W, int N, int E) {
  chain_wait();
  const int64_t total = (int64_t)W * count * E;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx % E);
    const int64_t rest = idx / E;
    const int i = (int)(rest % count), w = (int)(rest / count);
    x[((int64_t)w * N + rows[i]) * E + e] = 0.0;
  }
}

// current[w][n][e] = sum_f pairs[f][e] phi[w][n][f] (the "current" fields of normal_vjp,
// adtlert/forward/ert2p5d.py:907-908).
__global__ void mix_kernel(const double* pairs, const float* phi, int W, int N, int E,
                           double* current) {
  chain_wait();
  const int64_t total = (int64_t)W * N * E;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx % E);
    const int64_t row = idx / E;
    const float* x = phi + row * E;
    double acc = 0.0;
    for (int f = 0; f < E; ++f) acc += pairs[f * E + e] * (double)x[f];
    current[idx] = acc;
  }
}

// mix_kernel for E <= 64 as register-tiled products: a block takes 64 rows of the (W N) x E field
// matrix, stages them (as float64) and the E x E pair matrix in shared memory, and every thread
// forms a 4 x 4 tile of current = rows x pairs, summing f = 0 .. E-1 in order with fused
// multiply-adds -- the same operations in the same order as mix_kernel.
__global__ void __launch_bounds__(256) mix_tiled_kernel(const double* pairs, const float* phi, int64_t rows, int E,
                                                        double* current) {
  chain_wait();
  extern __shared__ double mix_sm[];
  const int Et = (E + 3) / 4, Ep = 4 * Et;
  double* pm = mix_sm;                 // [E][Ep] pairs, zero-padded columns
  double* xs = mix_sm + E * Ep;        // [kMixTileRows][E] rows
  const int64_t r0 = (int64_t)blockIdx.x * kMixTileRows;
  const int nr = (int)(rows - r0 < kMixTileRows ? rows - r0 : kMixTileRows);
  for (int i = threadIdx.x; i < E * Ep; i += blockDim.x) {
    const int f = i / Ep, e = i - f * Ep;
    pm[i] = e < E ? pairs[f * E + e] : 0.0;
  }
  for (int i = threadIdx.x; i < kMixTileRows * E; i += blockDim.x) {
    const int r = i / E;
    xs[i] = r < nr ? (double)phi[r0 * E + i] : 0.0;
  }
  __syncthreads();
  const int tiles = (kMixTileRows / 4) * Et;
  for (int t = threadIdx.x; t < tiles; t += blockDim.x) {
    const int tr = t / Et, te = t - tr * Et;
    double acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
    for (int f = 0; f < E; ++f) {
      double x[4], y[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = xs[(4 * tr + u) * E + f];
#pragma unroll
      for (int v = 0; v < 4; ++v) y[v] = pm[f * Ep + 4 * te + v];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(y[v], x[u], acc[u][v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = 4 * tr + u;
      if (r >= nr) continue;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int e = 4 * te + v;
        if (e < E) current[(r0 + r) * E + e] = acc[u][v];
      }
    }
  }
}

size_t mix_tiled_smem(int E) { return sizeof(double) * ((size_t)E * ((E + 3) / 4 * 4) + (size_t)kMixTileRows * E); }

// out[r][col] = sum over the column's cells (fixed order) of in[r][cell].
__global__ void aggregate_kernel(const double* in, int rows, int C, int columns, const int* ptr,
                                 const int* cells, float* out, int64_t in_stride) {
  chain_wait();
  const int64_t total = (int64_t)rows * columns;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / columns), col = (int)(idx % columns);
    double acc = 0.0;
    for (int i = ptr[col]; i < ptr[col + 1]; ++i) acc += in[(int64_t)r * in_stride + cells[i]];
    out[idx] = (float)acc;
  }
}

__global__ void aggregate_float_kernel(const float* in, int rows, int C, int columns,
                                       const int* ptr, const int* cells, float* out) {
  chain_wait();
  const int64_t total = (int64_t)rows * columns;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / columns), col = (int)(idx % columns);
    float acc = 0.f;
    for (int i = ptr[col]; i < ptr[col + 1]; ++i) acc += in[(int64_t)r * C + cells[i]];
    out[idx] = acc;
  }
}

}  // namespace adt
