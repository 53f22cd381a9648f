// Assembly, right-hand sides, total fields and measurement gathers of the 2.5D operator.
//
// All reductions run over precomputed lists in a fixed order (no atomics), so every result is
// bitwise repeatable. Fields are node-major, [system][dof][electrode], with dofs in the plan's
// solver order: the electrode axis is contiguous, so a warp reading one dof row of all
// electrodes is one coalesced transaction.
#include "adt_internal.h"
#include "kernels.h"

namespace adt {

// values[t][slot] = sum over the slot's routed contributions of
//   sigma_parent(cell) * (K + k_w^2 M)[cell][ij]        (volume)
//   sigma_parent(cell(b)) * alpha_w[b] * Mb[b][ij]       (mixed boundary, if robin)
// for systems t = model * W + w. Replaces _assemble + GroupSum (adtlert/forward/ert2p5d.py:275-314,
// adtlert/forward/kernels.py:30-85).
__device__ __forceinline__ double source_resistivity(const float* sigma, int Cm, int E, int idx, const int* ptr,
                                                     const int* cells) {
  const int s = idx / E, e = idx % E;
  double acc = 0.0;
  for (int i = ptr[e]; i < ptr[e + 1]; ++i) acc -= log((double)sigma[(int64_t)s * Cm + cells[i]]);
  const int n = ptr[e + 1] - ptr[e];
  return n > 0 ? exp(acc / n) : 1.0;
}

__global__ void assemble_kernel(AssembleArgs a) {
  chain_wait();
  if (a.rho)  // the source resistivities ride along with the assembly (one launch fewer)
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < a.models * a.E; idx += gridDim.x * blockDim.x)
      a.rho[idx] = source_resistivity(a.sigma, a.Cm, a.E, idx, a.src_ptr, a.src_cells);
  const int64_t total = (int64_t)a.systems * a.nnz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(idx / a.nnz), slot = (int)(idx - (int64_t)t * a.nnz);
    const int w = a.w0 + t % a.W, s = t / a.W;
    const float* sig = a.sigma + (int64_t)s * a.Cm;
    const double k2 = a.k2[w];
    const int volume = a.C * a.K2;
    double acc = 0.0;
    for (int c = a.contrib_ptr[slot]; c < a.contrib_ptr[slot + 1]; ++c) {
      const int code = a.contrib[c];
      if (code < 0) {
        if (a.identity) acc += 1.0;
      } else if (code < volume) {
        const int cell = code / a.K2;
        const double sigma = sig[a.parent ? a.parent[cell] : cell];
        acc += sigma * (a.stiffness[code] + k2 * a.mass[code]);
      } else if (a.robin) {
        const int bc = code - volume, b = bc / a.BL2;
        const int cell = a.bcells[b];
        const double sigma = sig[a.parent ? a.parent[cell] : cell];
        acc += sigma * a.bcoef[(int64_t)w * a.Nb + b] * a.bmass[bc];
      }
    }
    a.values[idx] = acc;
  }
}

// rho[s][e] = exp(-(1/n) sum log sigma) over the cells around electrode e's node, or 1/sigma of its
// cell (a list of one). Replaces _source_resistivities (ert2p5d.py:480-511).
__global__ void source_rho_kernel(const float* sigma, int Cm, int E, int models,
                                  const int* ptr, const int* cells, double* rho) {
  chain_wait();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= models * E) return;
  rho[idx] = source_resistivity(sigma, Cm, E, idx, ptr, cells);
}

// out[t][n][e] = base[w][n][e] + coef(t,e) * sum_{slot in row n} values[t][slot] x[src(t)][col][e]
// where coef(t,e) = scale * (rho ? rho[model(t)][e] : 1). `x_per_model` selects whether x is indexed
// by system (fields of each system) or by wavenumber (the primary field shared by all models).
__global__ void spmm_kernel(SpmmArgs a) {
  chain_wait();
  // systems over blockIdx.y, the (dof, electrode) entries of a system over blockIdx.x
  const int NE = a.N * a.E;
  for (int t = blockIdx.y; t < a.systems; t += gridDim.y) {
    const int w = t % a.W, s = t / a.W;
    const double* v = a.values + (int64_t)(a.values_per_wavenumber ? w : t) * a.nnz;
    const int64_t xo = (int64_t)(a.x_per_system ? t : w) * NE;
    const double* rho = a.rho ? a.rho + (int64_t)s * a.E : nullptr;
    const double* base = a.base ? a.base + (int64_t)w * NE : nullptr;
    double* out = a.out + (int64_t)t * NE;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NE; i += gridDim.x * blockDim.x) {
      const int n = i / a.E, e = i - n * a.E;
      double acc = 0.0;
      if (a.x_double) {
        const double* x = (const double*)a.x + xo;
        for (int slot = a.csr_ptr[n]; slot < a.csr_ptr[n + 1]; ++slot)
          acc += v[slot] * x[(int64_t)a.csr_col[slot] * a.E + e];
      } else {
        const float* x = (const float*)a.x + xo;
        for (int slot = a.csr_ptr[n]; slot < a.csr_ptr[n + 1]; ++slot)
          acc += v[slot] * (double)x[(int64_t)a.csr_col[slot] * a.E + e];
      }
      double coef = a.scale;
      if (rho) coef *= rho[e];
      double o = coef * acc;
      if (base) o += base[i];
      out[i] = o;
    }
  }
}

// fields[t][n][e] = x[t][n][e] + rho[s][e] * primary[w][n][e]
__global__ void total_kernel(const double* x, const double* primary, const double* rho, int W,
                             int N, int E, int systems, float* fields) {
  chain_wait();
  // systems over blockIdx.y, the (dof, electrode) entries of a system over blockIdx.x; with E a
  // multiple of 4, four consecutive electrodes of one dof per thread (vector loads and store)
  const int NE = N * E;
  const bool quad = (E & 3) == 0;
  for (int t = blockIdx.y; t < systems; t += gridDim.y) {
    const int w = t % W, s = t / W;
    const double* xs = x + (int64_t)t * NE;
    const double* up = primary ? primary + (int64_t)w * NE : nullptr;
    const double* rs = rho ? rho + (int64_t)s * E : nullptr;
    float* out = fields + (int64_t)t * NE;
    if (quad) {
      for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < NE / 4; q += gridDim.x * blockDim.x) {
        const int i = 4 * q, e = i % E;
        const double2 x0 = *reinterpret_cast<const double2*>(xs + i), x1 = *reinterpret_cast<const double2*>(xs + i + 2);
        double v[4] = {x0.x, x0.y, x1.x, x1.y};
        if (up) {
          const double2 u0 = *reinterpret_cast<const double2*>(up + i), u1 = *reinterpret_cast<const double2*>(up + i + 2);
          const double u[4] = {u0.x, u0.y, u1.x, u1.y};
#pragma unroll
          for (int k = 0; k < 4; ++k) v[k] = v[k] + rs[e + k] * u[k];
        }
        *reinterpret_cast<float4*>(out + i) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
      }
    } else {
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NE; i += gridDim.x * blockDim.x)
        out[i] = up ? (float)(xs[i] + rs[i % E] * up[i]) : (float)xs[i];
    }
  }
}

// Electrode potentials pot[s][e][r] = sum_k wr_k sum_w weight_w u_w[dof_rk][e] of every model into
// a padded (E+1) x (E+1) table (slot E: the zero remote row and column), one warp per entry: its
// lanes take the (k, w) terms, summed by a fixed shuffle tree (repeatable).
// Replaces _integrate + the electrode product of _normal_reciprocal (ert2p5d.py:560-582).
__global__ void potentials_kernel(MeasureArgs a, int models, double* pot) {
  chain_wait();
  const int E1 = a.E + 1, lane = threadIdx.x & 31;
  const int64_t total = (int64_t)models * E1 * E1;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int terms = a.RW * a.W;
  for (int64_t idx = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); idx < total; idx += warps) {
    const int s = (int)(idx / (E1 * E1));
    const int rem = (int)(idx - (int64_t)s * E1 * E1);
    const int r = rem / E1, e = rem - r * E1;  // pot[s][e][r] stored at [s][r][e]: e fastest
    double acc = 0.0;
    if (r < a.E && e < a.E) {
      const int64_t fo = (int64_t)s * a.W * a.N * a.E;
      for (int item = lane; item < terms; item += 32) {
        const int k = item / a.W, w = item - k * a.W;
        const int dof = a.rcv_dofs[r * a.RW + k];
        if (dof < 0) continue;
        const int64_t i = fo + ((int64_t)w * a.N + dof) * a.E + e;
        const double f = a.f_double ? ((const double*)a.fields)[i] : (double)((const float*)a.fields)[i];
        acc += a.rcv_w[r * a.RW + k] * (a.weights[w] * f);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    }
    if (lane == 0) {
      if (a.potentials && r < a.E && e < a.E) a.potentials[((int64_t)s * a.E + e) * a.E + r] = acc;
      pot[idx] = acc;
    }
  }
}

// Normal and reciprocal transfers of every (model, row) from the potential table; in combine
// mode the tangent of sign(n) sqrt|n r| instead (ert2p5d.py:584-589, 647-655, 886-890).
__global__ void transfers_kernel(MeasureArgs a, int models, const double* pot) {
  chain_wait();
  const int E1 = a.E + 1;
  const int64_t total = (int64_t)models * a.D;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(idx / a.D), d = (int)(idx - (int64_t)s * a.D);
    const double* P = pot + (int64_t)s * E1 * E1;
    auto at = [&](int src, int rcv) { return P[rcv * E1 + src]; };
    const int A = a.abmn[4 * d], B = a.abmn[4 * d + 1], M = a.abmn[4 * d + 2], N = a.abmn[4 * d + 3];
    const double n = (at(A, M) - at(A, N)) - (at(B, M) - at(B, N));
    const double r = (at(M, A) - at(M, B)) - (at(N, A) - at(N, B));
    if (a.combine) {
      const double n0 = a.base_normal[idx], r0 = a.base_recip[idx];
      const double scale = fmax(sqrt(fabs(n0 * r0)), 1e-30);
      const double sign = (r0 > 0.0) - (r0 < 0.0);
      a.normal[idx] = 0.5 * sign * (n * r0 + n0 * r) / scale;
    } else {
      a.normal[idx] = n;
      a.reciprocal[idx] = r;
    }
  }
}

// pairs[q][e][f] (e, f < E) = sum over the (e, f) entry's routed list of +-coef, where each entry
// names a row d and whether it carries the normal or the reciprocal cotangent.
// Replaces _pair_cotangent (ert2p5d.py:591-629).
__global__ void pair_kernel(PairArgs a) {
  chain_wait();
  const int64_t total = (int64_t)a.count * a.E * a.E;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(idx / (a.E * a.E));
    const int ef = (int)(idx - (int64_t)q * a.E * a.E);
    const int e = ef / a.E, f = ef % a.E;
    const int slot = e * (a.E + 1) + f;
    double acc = 0.0;
    for (int i = a.pair_ptr[slot]; i < a.pair_ptr[slot + 1]; ++i) {
      const int code = a.pair_list[i];
      const int d = code >> 2, kind = code & 3;
      if (kind >= 2 && a.normal_only) continue;
      double coef;
      if (a.unit) {
        coef = (d == a.row_begin + q) ? 1.0 : 0.0;
        if (coef == 0.0) continue;
      } else {
        coef = a.cot[(int64_t)q * a.D + d];
      }
      if (!a.normal_only) {
        // exact derivative of sign(n) sqrt|n r|: common * r for normal, common * n for reciprocal
        const int64_t md = (int64_t)(a.model_of_count ? q : 0) * a.D + d;
        const double n0 = a.normal[md], r0 = a.recip[md];
        const double scale = fmax(sqrt(fabs(n0 * r0)), 1e-30);
        const double sign = (r0 > 0.0) - (r0 < 0.0);
        coef *= 0.5 * sign / scale * (kind < 2 ? r0 : n0);
      }
      acc += (kind & 1) ? -coef : coef;
    }
    a.pairs[idx] = acc;
  }
}

// Adjoint right-hand sides rhs[t][n][col] with t = model * W + w, col = q_local * E + e:
// weight_w * sum_r pairs[q][e][r] Pel[r][n], nonzero only at receiver dofs (routed list).
// Replaces _adjoint_rhs (ert2p5d.py:631-639).
__global__ void adjoint_rhs_kernel(AdjointRhsArgs a) {
  chain_wait();
  const int ncol = a.q_per_model * a.E;
  const int64_t total = (int64_t)a.systems * a.rdofs * ncol;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int col = (int)(idx % ncol);
    const int64_t rest = idx / ncol;
    const int i = (int)(rest % a.rdofs), t = (int)(rest / a.rdofs);
    const int w = t % a.W, s = t / a.W;
    const int ql = col / a.E, e = col % a.E;
    const int q = s * a.q_per_model + ql;
    const double* pr = a.pairs + ((int64_t)q * a.E + e) * a.E;
    double acc = 0.0;
    for (int j = a.rdof_ptr[i]; j < a.rdof_ptr[i + 1]; ++j) acc += pr[a.rdof_rcv[j]] * a.rdof_w[j];
    a.rhs[((int64_t)t * a.N + a.rdof_dof[i]) * ncol + col] = a.weights[w] * acc;
  }
}

// Partial Gram sums for normal_jvp: partial[b][e][f] = sum over this block's slice of (w, n) of
// weight_w * phi[w][n][e] * y[w][n][f]; a second pass sums the partials in block order.
// partial[b] = sum over the rows r of chunk b (rows of the W x N row space, in order) of
// weight_{w(r)} phi[r]^T y[r] (E x E, float64). Rows stream through shared memory `sub` at a
// time (weighted phi and y, row stride padded to a multiple of 4 with zeros); each thread owns
// 4 x 4 output tiles and sums its rows in order, so every partial is bitwise repeatable.
__global__ void gram_partial_kernel(const float* phi, const double* y, const double* weights,
                                    int W, int N, int E, int chunk, int sub, double* partial) {
  chain_wait();
  extern __shared__ double rows_sm[];
  const int Et = (E + 3) / 4, Ep = 4 * Et, tiles = Et * Et;
  double* ps = rows_sm;            // [sub][Ep]
  double* ys = rows_sm + sub * Ep; // [sub][Ep]
  const int64_t total = (int64_t)W * N;
  const int64_t begin = (int64_t)blockIdx.x * chunk;
  const int64_t end = begin + chunk < total ? begin + chunk : total;
  double* out = partial + (int64_t)blockIdx.x * E * E;
  for (int t0 = 0; t0 < tiles; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const bool active = t < tiles;
    const int ti = active ? t / Et : 0, tj = active ? t - ti * Et : 0;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int64_t r0 = begin; r0 < end; r0 += sub) {
      const int rows = (int)(end - r0 < sub ? end - r0 : sub);
      const int w0 = (int)(r0 / N);
      const int64_t boundary = (int64_t)(w0 + 1) * N;  // rows at or past it belong to w0 + 1 (sub <= N)
      __syncthreads();  // the previous rows have been read
      for (int i = threadIdx.x; i < sub * Ep; i += blockDim.x) {
        const int r = i / Ep, c = i - r * Ep;
        const int64_t row = r0 + r;
        double pv = 0.0, yv = 0.0;
        if (r < rows && c < E) {
          const int w = row >= boundary ? w0 + 1 : w0;
          pv = weights[w] * (double)phi[row * E + c];
          yv = y[row * E + c];
        }
        ps[i] = pv;
        ys[i] = yv;
      }
      __syncthreads();
      if (active)
        for (int r = 0; r < rows; ++r) {
          const double* pr = ps + r * Ep + 4 * ti;
          const double* yr = ys + r * Ep + 4 * tj;
          double a[4], b[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            a[k] = pr[k];
            b[k] = yr[k];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
    }
    if (active)
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int i = 4 * ti + u, j = 4 * tj + v;
          if (i < E && j < E) out[i * E + j] = acc[u][v];
        }
  }
}

// gram[ef] = sum over the blocks' partials in block order (fixed order: repeatable).
__global__ void gram_reduce_kernel(const double* partial, int blocks, int E, double* gram) {
  chain_wait();
  const int ef = blockIdx.x * blockDim.x + threadIdx.x;
  if (ef >= E * E) return;
  double acc = 0.0;
  for (int b = 0; b < blocks; ++b) acc += partial[(int64_t)b * E * E + ef];
  gram[ef] = acc;
}

// out[d] = -(G[M][A] - G[M][B] - G[N][A] + G[N][B]), slot E (the remote electrode) contributing 0.
__global__ void gram_gather_kernel(const double* gram, int E, int D, const int* abmn, double* out) {
  chain_wait();
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= D) return;
  const int A = abmn[4 * d], B = abmn[4 * d + 1], M = abmn[4 * d + 2], N = abmn[4 * d + 3];
  auto g = [&](int i, int j) -> double { return (i >= E || j >= E) ? 0.0 : gram[(int64_t)i * E + j]; };
  out[d] = -(g(M, A) - g(M, B) - g(N, A) + g(N, B));
}

// integrated[e][orig] = sum_w weight_w fields[w][pos(orig)][e]
__global__ void integrated_kernel(const float* fields, const double* weights, const int* iperm,
                                  int W, int N, int E, float* integrated) {
  chain_wait();
  const int64_t total = (int64_t)N * E;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / N), orig = (int)(idx % N);
    const int n = iperm[orig];
    double acc = 0.0;
    for (int w = 0; w < W; ++w) acc += weights[w] * (double)fields[((int64_t)w * N + n) * E + e];
    integrated[idx] = (float)acc;
  }
}


}  // namespace adt
