// Normal-quadrupole Jacobian on the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
// Same contraction as jacobian_kernel: for every cell c the electrode Gram
//   G_c = F_c^T F_c,   F_c[w R + f][e] = sqrt(w_w) (k_w) L_c[f] . x_we   (R features per wavenumber),
// and each ABMN row takes four Gram entries, J[d][c] = -(G[M][A] - G[M][B] - G[N][A] + G[N][B]).
// Here the Grams of a pair of cells are one tcgen05.mma chain: the two cells' feature matrices
// are stacked as rows (electrode e of cell i at row i Ep + e, Ep = E rounded up to 8) of one
// K-major operand S in shared memory, and A = S (M = 128 rows; rows past 2 Ep read whatever
// follows and only feed rows of D that are never read), B = S (N = 2 Ep), so D = S S^T (fp32, in
// tensor memory) holds both Grams as its diagonal blocks. K = 8 features per instruction.
// Float32 accuracy comes from a hi/lo split of every feature (hi = TF32 rounding, lo = the
// remainder): G = hi.hi + hi.lo + lo.hi, three MMAs per K-step accumulating in fp32.
//
// Persistent blocks (two per SM; 256 threads each) loop over the cell pairs: (1) all threads
// compute the features of the pair into shared memory (thread e of a 64-thread lane group
// handles electrode e of (cell, four consecutive wavenumbers) work pairs and stores whole 16-byte
// chunks; generic proxy, then fence.proxy.async); (2) one
// thread issues the MMAs and commits them to an mbarrier; (3) all threads wait on it (bounded: on
// timeout the block raises the error flag, writes NaN for its rows and stops); (4) warps read
// their TMEM lanes back (tcgen05.ld; warps 0-3 the first cell's columns, 4-7 the second's),
// stage the Grams in shared memory and write two consecutive floats per row. Shared-memory
// operand layout (no swizzle, K-major canonical layout): chunk q of row r at
// (part*KC + q)*2Ep*16 + r*16, so one 8-row core matrix is 128 contiguous bytes (stride byte
// offset 128) and the two 16-byte K halves of one MMA are 2Ep*16 bytes apart (leading byte
// offset).
#include "adt_internal.h"
#include "kernels.h"
#include "tcgen05.h"

namespace adt {
namespace {

using namespace tc;

constexpr int kTcThreads = 256;
constexpr int kTcCells = 2;      // cells per group (stacked in one MMA operand)
constexpr int kTcM = 128;        // MMA M (rows of the stacked operand)
constexpr uint32_t kTcWaitLimit = 1u << 20;  // mbarrier polls before the block gives up
constexpr int kTcRowTable = 4096;            // rows whose Gram offsets stay in shared memory
constexpr int kTcStaticW = 17;  // the 2.5D quadrature's wavenumber count: a compile-time variant

}  // namespace

// Shared memory of jacobian_tc_kernel for E electrodes, W wavenumbers, R features, K dofs.
size_t jacobian_tc_smem(int E, int W, int R, int K, int rows) {
  const int Ep = (E + 7) & ~7, RW = kTcCells * Ep;
  const int KC = (W * R + 7) / 8 * 2;  // 16-byte feature chunks per row and part (K padded to 8)
  const size_t feat = (size_t)2 * KC * RW * 16 + (size_t)kTcM * 16;  // + rows read past the end
  const size_t gram = (size_t)kTcCells * (E * (E + 1) + 1) * 4;
  const size_t tables = (size_t)kTcCells * (R * K + K) * 4 + (size_t)W * R * 4;
  // per row: Gram offsets of (M,A) (M,B) (N,A) (N,B); at most kTcRowTable rows resident
  const size_t offsets = (size_t)(rows < kTcRowTable ? rows : kTcRowTable) * 8;
  return (feat + gram + tables + offsets + 64 + 31) / 16 * 16;
}

// KT dofs and RT features per cell are compile-time; WT > 0 makes the wavenumber count
// compile-time too (the feature stage then indexes registers and chunks statically).
template <int KT, int RT, int WT = 0>
__global__ void __launch_bounds__(kTcThreads, 2) jacobian_tc_kernel(JacobianArgs a, int* error) {
  chain_wait();
  extern __shared__ __align__(128) unsigned char tc_sm[];
  constexpr int K = KT, R = RT;
  const int E = a.E, W = a.W;
  const int Ep = (E + 7) & ~7, RW = kTcCells * Ep;           // rows of the stacked operand
  const int KF = W * R, KC = (KF + 7) / 8 * 2, KS = KC / 2;  // features, 16B chunks, MMA K-steps
  const size_t part_bytes = (size_t)KC * RW * 16;
  unsigned char* feat = tc_sm;                                         // [2][KC][RW][4] fp32
  float* gram = reinterpret_cast<float*>(feat + 2 * part_bytes + kTcM * 16);  // [kTcCells][E(E+1)+1]
  const int GLD = E + 1, GS = E * GLD + 1;                            // entry GS-1 is the remote zero
  float* coef = gram + (size_t)kTcCells * GS;                          // [kTcCells][R][K]
  float* scale = coef + kTcCells * R * K;                              // [W][R]
  int* dofs = reinterpret_cast<int*>(scale + W * R);                   // [kTcCells][K]
  const int table_rows = min(a.rows, kTcRowTable);
  short4* offs = reinterpret_cast<short4*>(
      (reinterpret_cast<uintptr_t>(dofs + kTcCells * K) + 7) & ~uintptr_t(7));  // [table_rows]
  uint64_t* bar = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(offs + table_rows) + 15) & ~uintptr_t(15));
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int groups = (a.c_end - a.c_begin + kTcCells - 1) / kTcCells;
  uint32_t tmem_cols = 32;
  while (tmem_cols < (uint32_t)RW) tmem_cols <<= 1;

  // set-up: mbarrier (one arrival per group) and the tensor-memory columns of the block
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(smem_addr(tmem_slot)), "r"(tmem_cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = tf32_idesc(kTcM, RW);
  bool failed = false;
  uint32_t phase = 0;
  // per-block tables: feature scales, Gram offsets of every row (remote slot: the zero entry)
  for (int i = tid; i < W * R; i += kTcThreads) scale[i] = a.fscale[i];
  auto fill_offsets = [&](int r0, int n) {
    for (int d = tid; d < n; d += kTcThreads) {
      const int4 q = *reinterpret_cast<const int4*>(a.abmn + 4 * (a.row_begin + r0 + d));
      auto at = [&](int i, int k) -> short {
        return (short)(((unsigned)i < (unsigned)E && (unsigned)k < (unsigned)E) ? i * GLD + k : GS - 1);
      };
      offs[d] = make_short4(at(q.z, q.x), at(q.z, q.y), at(q.w, q.x), at(q.w, q.y));
    }
  };
  const bool resident = a.rows <= kTcRowTable;
  if (resident) fill_offsets(0, a.rows);
  for (int ci = tid; ci < kTcCells; ci += kTcThreads) gram[(size_t)ci * GS + GS - 1] = 0.f;
  // chunks past the ones the feature stage writes (R ceil(W / 4), or the two halves' 2R +
  // ceil((WT - 8) R / 4), .. KC - 1) are K padding: zero for every group, written once
  constexpr int WT_CHUNKS = WT > 0 ? 2 * R + ((WT - 8) * R + 3) / 4 : 0;
  const int written = WT > 0 ? WT_CHUNKS : R * ((W + 3) >> 2);
  for (int item = tid, q0 = min(written, KC); item < (KC - q0) * RW * 4; item += kTcThreads) {
    const size_t off = ((size_t)q0 * RW) * 16 + (size_t)item * 4;
    *reinterpret_cast<float*>(feat + off) = 0.f;
    *reinterpret_cast<float*>(feat + part_bytes + off) = 0.f;
  }

  for (int group = blockIdx.x; group < groups && !failed; group += gridDim.x) {
    const int c0 = a.c_begin + group * kTcCells;
    // (1) cell tables, then features (hi part 0, lo part 1)
    for (int i = tid; i < kTcCells * R * K; i += kTcThreads) {
      const int c = min(c0 + i / (R * K), a.c_end - 1);
      coef[i] = a.features[(int64_t)c * R * K + i % (R * K)];
    }
    for (int i = tid; i < kTcCells * K; i += kTcThreads) {
      const int c = c0 + i / K;
      dofs[i] = c < a.c_end ? a.cell_dofs[(int64_t)c * K + i % K] : -1;
    }
    __syncthreads();
    if constexpr (WT > 0) {
      // thread (cell ci, half h, electrode e): wavenumbers 0 .. 7 (h = 0: chunks 0 .. 2R - 1) or
      // 8 .. WT - 1 (h = 1: chunks 2R .. KC - 1, the tail padded with zeros); its field loads
      // are issued first, then whole 16-byte chunks are stored
      constexpr int WH = 8, WB = WT - WH, CH0 = WH * R / 4;
      static_assert(WB >= WH && WB <= 16, "two halves of at most 16 wavenumbers");
      const int e = tid & 63, h = (tid >> 6) & 1, ci = tid >> 7;
      if (e < E) {
        int dof[K];
#pragma unroll
        for (int k = 0; k < K; ++k) dof[k] = dofs[ci * K + k];
        const int w0 = h * WH, wn = h ? WB : WH;
        float x[WB][K];
#pragma unroll
        for (int j = 0; j < WB; ++j)
#pragma unroll
          for (int k = 0; k < K; ++k)
            x[j][k] = (j < wn && dof[k] >= 0) ? __ldg(a.fields + ((int64_t)(w0 + j) * a.N + dof[k]) * E + e) : 0.f;
        float cf[R][K];
#pragma unroll
        for (int f = 0; f < R; ++f)
#pragma unroll
          for (int k = 0; k < K; ++k) cf[f][k] = coef[(ci * R + f) * K + k];
        const int nch = h ? KC - CH0 : CH0;
        unsigned char* row_feat = feat + ((size_t)(h * CH0) * RW + ci * Ep + e) * 16;
        float hi[4] = {0.f, 0.f, 0.f, 0.f}, lo[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int j = 0; j < WB; ++j) {
#pragma unroll
          for (int f = 0; f < R; ++f) {
            const int kl = j * R + f;  // compile-time: chunk kl / 4, lane kl % 4
            float v = 0.f;
            if (j < wn) {
#pragma unroll
              for (int k = 0; k < K; ++k) v = fmaf(cf[f][k], x[j][k], v);
              v *= scale[(w0 + j) * R + f];
            }
            hi[kl & 3] = tf32_round(v);
            lo[kl & 3] = v - hi[kl & 3];
            if ((kl & 3) == 3 && (kl >> 2) < nch) {
              const size_t off = (size_t)(kl >> 2) * RW * 16;
              *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
              *reinterpret_cast<float4*>(row_feat + part_bytes + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            }
          }
        }
        constexpr int last = WB * R;  // a partial last chunk: its remaining lanes are padding
        if constexpr (last % 4 != 0) {
#pragma unroll
          for (int i = last % 4; i < 4; ++i) hi[i] = lo[i] = 0.f;
          if ((last >> 2) < nch) {
            const size_t off = (size_t)(last >> 2) * RW * 16;
            *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(row_feat + part_bytes + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
      }
    } else {
      // work pairs (cell ci, wavenumber quad m): features of wavenumbers 4m .. 4m + 3 are the R
      // whole chunks R m .. R m + R - 1. Thread e of lane group lg takes electrode e of pairs
      // lg, lg + 4, ..., two at a time with all their field loads issued first, and stores whole
      // 16-byte chunks (consecutive lanes: consecutive rows); chunks past KC hold only padding
      {
        const int lg = tid >> 6, e = tid & 63;
        const int NQ = (W + 3) >> 2, pairs = kTcCells * NQ;
        if (e < E) {
          for (int p0 = lg; p0 < pairs; p0 += 8) {
            float x[2][4][K];
  #pragma unroll
            for (int pp = 0; pp < 2; ++pp) {
              const int p = p0 + 4 * pp;
              const int ci = p / NQ, m = p - ci * NQ;
  #pragma unroll
              for (int k = 0; k < K; ++k) {
                const int dof = p < pairs ? dofs[ci * K + k] : -1;
  #pragma unroll
                for (int wq = 0; wq < 4; ++wq) {
                  const int w = 4 * m + wq;
                  x[pp][wq][k] = (dof >= 0 && w < W) ? __ldg(a.fields + ((int64_t)w * a.N + dof) * E + e) : 0.f;
                }
              }
            }
  #pragma unroll
            for (int pp = 0; pp < 2; ++pp) {
              const int p = p0 + 4 * pp;
              if (p >= pairs) break;
              const int ci = p / NQ, m = p - ci * NQ;
              float cf[R][K];
  #pragma unroll
              for (int f = 0; f < R; ++f)
  #pragma unroll
                for (int k = 0; k < K; ++k) cf[f][k] = coef[(ci * R + f) * K + k];
              unsigned char* row_feat = feat + ((size_t)R * m * RW + ci * Ep + e) * 16;
              float hi[4], lo[4];
  #pragma unroll
              for (int wq = 0; wq < 4; ++wq) {
                const int w = min(4 * m + wq, W - 1);
  #pragma unroll
                for (int f = 0; f < R; ++f) {
                  float v = 0.f;
  #pragma unroll
                  for (int k = 0; k < K; ++k) v = fmaf(cf[f][k], x[pp][wq][k], v);
                  v *= scale[w * R + f];
                  const int kl = wq * R + f;  // compile-time: chunk kl / 4, lane kl % 4
                  hi[kl & 3] = tf32_round(v);
                  lo[kl & 3] = v - hi[kl & 3];
                  if ((kl & 3) == 3 && R * m + (kl >> 2) < KC) {
                    const size_t off = (size_t)(kl >> 2) * RW * 16;
                    *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
                    *reinterpret_cast<float4*>(row_feat + part_bytes + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
                  }
                }
              }
            }
          }
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

    // (2) one thread issues every MMA of the pair and commits them to the mbarrier; a K-step
    //     advances both descriptors by two chunks
    if (tid == 0) {
      const uint32_t base = smem_addr(feat);
      uint64_t dh = operand_desc(base, (uint32_t)RW * 16, 128);
      uint64_t dl = operand_desc(base + (uint32_t)part_bytes, (uint32_t)RW * 16, 128);
      const uint64_t step = (uint64_t)(2 * RW * 16) >> 4;
      for (int s = 0; s < KS; ++s) {
        mma_tf32(tmem, dh, dh, idesc, s > 0 ? 1u : 0u);
        mma_tf32(tmem, dh, dl, idesc, 1u);
        mma_tf32(tmem, dl, dh, idesc, 1u);
        dh += step;
        dl += step;
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                   ::"r"(smem_addr(bar)) : "memory");
    }

    // (3) bounded wait for the MMAs (a plan option may shorten it to a few non-blocking polls,
    //     so that a test can make it run out; the drain below keeps the full limit)
    uint32_t polls = 0;
    if (a.first_wait_polls == 0) {
      while (!mbar_try_wait(smem_addr(bar), phase)) {
        if (++polls >= kTcWaitLimit) { failed = true; break; }
      }
    } else {
      while (!mbar_test_wait(smem_addr(bar), phase)) {
        if (++polls >= a.first_wait_polls) { failed = true; break; }
      }
    }
    phase ^= 1u;
    failed = __syncthreads_or(failed);
    if (failed) break;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

    // (4) tensor memory -> staged Grams: warp w reads TMEM lanes 32 (w % 4) .. + 31 (= rows of D)
    //     in the columns of cell h = w / 4; a lane keeps the entries of its row when the row
    //     belongs to cell h
    {
      const int h = warp >> 2, row = 32 * (warp & 3) + lane;
      const int lr = row - h * Ep;
      const bool mine = lr >= 0 && lr < E;
      float* g = gram + (size_t)h * GS + (size_t)(mine ? lr : 0) * GLD;
      // warp-uniform: whether any row of this warp's lane quarter belongs to cell h
      const int first = 32 * (warp & 3) - h * Ep;
      const bool any = first < E && first + 32 > 0;
      for (int cc = 0; any && cc < Ep; cc += 8) {
        uint32_t v[8];
        tmem_load8(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(h * Ep + cc), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (mine) {
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (cc + j < E) g[cc + j] = __uint_as_float(v[j]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    // (5) rows: one thread per row, both cells of the group (adjacent floats of J); with more
    //     rows than the table holds, the table is refilled chunk by chunk
    const int ncells = min(kTcCells, a.c_end - c0);
    for (int r0 = 0; r0 < a.rows; r0 += kTcRowTable) {
      const int n = min(kTcRowTable, a.rows - r0);
      if (!resident) {
        if (r0 > 0) __syncthreads();
        fill_offsets(r0, n);
        __syncthreads();
      }
      for (int d = tid; d < n; d += kTcThreads) {
        const int dl = r0 + d;
        const short4 o = offs[d];
        float v[kTcCells];
#pragma unroll
        for (int ci = 0; ci < kTcCells; ++ci) {
          const float* gc = gram + (size_t)ci * GS;
          v[ci] = -((gc[o.x] - gc[o.y]) - (gc[o.z] - gc[o.w]));
        }
        float* out = a.out + (int64_t)dl * a.ldo + c0;
        if (ncells == kTcCells && (((uintptr_t)out & 7) == 0)) {
          *reinterpret_cast<float2*>(out) = make_float2(v[0], v[1]);
        } else {
          for (int ci = 0; ci < ncells; ++ci) out[ci] = v[ci];
        }
      }
    }
    __syncthreads();
  }

  if (failed) {
    if (tid == 0) atomicOr(error, 1);
    // NaN in every row of this block's remaining cells
    for (int group = blockIdx.x; group < groups; group += gridDim.x)
      for (int idx = tid; idx < a.rows * kTcCells; idx += kTcThreads) {
        const int c = a.c_begin + group * kTcCells + idx % kTcCells;
        if (c < a.c_end) a.out[(int64_t)(idx / kTcCells) * a.ldo + c] = __int_as_float(0x7fc00000);
      }
    // the last commit may still be pending: give it a bounded second chance before freeing
    uint32_t polls = 0;
    while (!mbar_try_wait(smem_addr(bar), phase ^ 1u) && ++polls < kTcWaitLimit) {
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols) : "memory");
}

template __global__ void jacobian_tc_kernel<3, 5>(JacobianArgs, int*);
template __global__ void jacobian_tc_kernel<3, 6>(JacobianArgs, int*);
template __global__ void jacobian_tc_kernel<4, 3>(JacobianArgs, int*);
template __global__ void jacobian_tc_kernel<4, 7>(JacobianArgs, int*);
template __global__ void jacobian_tc_kernel<4, 8>(JacobianArgs, int*);

namespace {
bool tc_shape(int K, int R) {
  return (K == 3 && (R == 5 || R == 6)) || (K == 4 && (R == 3 || R == 7 || R == 8));
}
}  // namespace

// Whether the tensor-core kernel applies: E <= 64 electrode slots (two cells stack into the
// 128 rows of one MMA), an instantiated (K, R), and two blocks' shared memory per SM.
bool jacobian_tc_supported(int E, int W, int R, int K, int rows) {
  return E <= kTcM / kTcCells && tc_shape(K, R) && jacobian_tc_smem(E, W, R, K, rows) <= 110 * 1024;
}

cudaError_t launch_jacobian_tc(const JacobianArgs& a, int* error, int sms, cudaStream_t s) {
  const size_t smem = jacobian_tc_smem(a.E, a.W, a.R, a.K, a.rows);
  const int groups = (a.c_end - a.c_begin + kTcCells - 1) / kTcCells;
  const int blocks = groups < 2 * sms ? groups : 2 * sms;
  auto go = [&](auto kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_chained(kernel, blocks, kTcThreads, smem, s, a, error);
    return cudaGetLastError();
  };
  if (a.W == kTcStaticW) {
    if (a.K == 3 && a.R == 5) return go(jacobian_tc_kernel<3, 5, kTcStaticW>);
    if (a.K == 3 && a.R == 6) return go(jacobian_tc_kernel<3, 6, kTcStaticW>);
    if (a.K == 4 && a.R == 3) return go(jacobian_tc_kernel<4, 3, kTcStaticW>);
    if (a.K == 4 && a.R == 7) return go(jacobian_tc_kernel<4, 7, kTcStaticW>);
    return go(jacobian_tc_kernel<4, 8, kTcStaticW>);
  }
  if (a.K == 3 && a.R == 5) return go(jacobian_tc_kernel<3, 5>);
  if (a.K == 3 && a.R == 6) return go(jacobian_tc_kernel<3, 6>);
  if (a.K == 4 && a.R == 3) return go(jacobian_tc_kernel<4, 3>);
  if (a.K == 4 && a.R == 7) return go(jacobian_tc_kernel<4, 7>);
  return go(jacobian_tc_kernel<4, 8>);
}

}  // namespace adt
