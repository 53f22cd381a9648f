// Normal-quadrupole Jacobian on tcgen05 with warp roles and a two-deep pipeline.
//
// Same contraction and operand layout as jacobian_tc_kernel (sensitivity_tc.cu): the features of
// a pair of cells (hi/lo TF32 split) are stacked as the rows of one K-major operand S, and D =
// S S^T in tensor memory holds both electrode Grams; J[d][c] = -(G[M][A] - G[M][B] - G[N][A] +
// G[N][B]). What changes is how the per-pair chain overlaps. One persistent block per SM:
//
//   producer warps 0-7   two teams: warps 0-3 build the even pairs into operand stage 0, warps
//                        4-7 the odd pairs into stage 1 (thread: one electrode row of one cell,
//                        all wavenumbers; the team's next cell dofs loaded a pair ahead), so one
//                        team's field loads are in flight while the other computes; each thread
//                        arrives on stage_full[j % 2].
//   MMA warp 15          one thread issues pair j's MMAs into accumulator j % 4 (TMEM columns
//                        128 (j % 4)) and commits them to stage_free[j % 2] and acc_full[j % 4].
//   epilogue warps 8-14  wait for acc_full[j % 4], read the Grams back (warp 8 + w: TMEM lanes
//                        32 (w % 4) .., the columns of cell w / 4; 16-column loads, one wait),
//                        release the accumulator (acc_free[j % 4]), and after `batch` pairs
//                        write every row of the batch's 2 batch consecutive cells at once (32
//                        bytes per row for 4 pairs). The batch's Grams are stored entry-major
//                        with the cells interleaved, so a row's four entries for all 8 cells
//                        are eight 16-byte shared-memory loads.
//
// So the features of pair j + 1, the MMAs of pair j and the readback and rows of up to three
// earlier pairs run at the same time. A stage is rebuilt only after the MMAs that read it
// completed, an accumulator rewritten only after its readback. Every wait is bounded: a role that gives up
// raises the block's abort flag (the other role stops at its next wait), the block writes NaN
// into its columns and raises the caller's error flag, and before tensor memory is freed it
// waits (again bounded) for the last MMAs it issued.
#include "adt_internal.h"
#include "kernels.h"
#include "tcgen05.h"

namespace adt {
namespace {

using namespace tc;

constexpr int kPipeThreads = 512;       // 8 producer warps, 7 epilogue warps, 1 MMA warp
constexpr int kProducerThreads = 256;
constexpr int kTeamThreads = 128;     // producers per operand stage
constexpr int kEpilogueThreads = 224;
constexpr int kMmaWarp = 15;
constexpr int kAccumulators = 4;        // TMEM accumulators of 128 columns
constexpr int kPipeM = 128;
constexpr int kPipeRowTable = 4096;     // rows whose Gram offsets stay in shared memory
constexpr uint32_t kPipeWaitLimit = 1u << 20;
constexpr int kPipeStaticW = 17;

struct PipeLayout {
  int Ep, RW, KC, KS, GLD, GS;
  size_t part, stage, feat, gram, offs, total;
};

__host__ __device__ inline PipeLayout pipe_layout(int E, int W, int R, int batch, int rows) {
  PipeLayout l;
  l.Ep = (E + 7) & ~7;
  l.RW = 2 * l.Ep;
  l.KC = (W * R + 7) / 8 * 2;
  l.KS = l.KC / 2;
  l.GLD = E + 1;
  l.GS = E * l.GLD + 1;
  l.part = (size_t)l.KC * l.RW * 16;
  l.stage = 2 * l.part;
  l.feat = 2 * l.stage + (size_t)kPipeM * 16;  // + the rows the M = 128 MMA reads past the end
  l.gram = (size_t)batch * 2 * l.GS * 4;
  l.offs = (size_t)rows * 8;
  const size_t tail = 12 * 8 + 16 + (size_t)W * R * 4 + 64;  // barriers, TMEM slot, flags, scales
  l.total = ((l.feat + l.gram + 15) / 16 * 16) + l.offs + tail;
  return l;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 state;\n\tmbarrier.arrive.shared::cta.b64 state, [%0];\n\t}\n" ::"r"(smem_addr(bar))
               : "memory");
}

// Bounded wait; also gives up when the block's abort flag is raised.
__device__ __forceinline__ bool pipe_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t polls = 0; polls < kPipeWaitLimit; ++polls) {
    if (mbar_try_wait(smem_addr(bar), parity)) return true;
    if ((polls & 63) == 63 && *abort) return false;
  }
  return false;
}

__device__ __forceinline__ void tmem_load16(uint32_t addr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
}

__device__ __forceinline__ void commit_to(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(threads) : "memory");
}

}  // namespace

template <int K, int R, int WT>
__global__ void __launch_bounds__(kPipeThreads, 1) jacobian_tcpipe_kernel(JacobianArgs a, int batch, int* error) {
  chain_wait();
  extern __shared__ __align__(128) unsigned char pipe_sm[];
  const int E = a.E;
  const PipeLayout L = pipe_layout(E, WT, R, batch, a.rows);
  unsigned char* feat = pipe_sm;
  float* gram = reinterpret_cast<float*>(pipe_sm + L.feat);  // [GS][2 batch]: cells interleaved per entry
  const int NC = 2 * batch;
  short4* offs = reinterpret_cast<short4*>(pipe_sm + (L.feat + L.gram + 15) / 16 * 16);
  uint64_t* bars = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(offs + a.rows) + 15) & ~uintptr_t(15));
  uint64_t* stage_free = bars;      // [2]  MMAs of the pair in stage s completed
  uint64_t* stage_full = bars + 2;  // [2]  features of the pair in stage s written
  uint64_t* acc_full = bars + 4;    // [4]  MMAs of the pair in accumulator k completed
  uint64_t* acc_free = bars + 8;    // [4]  accumulator k read back
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 12);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* epilogue_flag = reinterpret_cast<int*>(tmem_slot + 3);
  float* scale = reinterpret_cast<float*>(tmem_slot + 4);   // [WT][R]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int pairs_total = (a.c_end - a.c_begin + 1) / 2;
  const int supers = (pairs_total + batch - 1) / batch;
  const int my_supers = blockIdx.x < supers ? (supers - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int pairs = my_supers * batch;  // pairs of this block, including empty ones at the end

  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(stage_free + i, 1);
      mbar_init(stage_full + i, kTeamThreads);
    }
    for (int i = 0; i < kAccumulators; ++i) {
      mbar_init(acc_full + i, 1);
      mbar_init(acc_free + i, kEpilogueThreads);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *abort = 0;
    *epilogue_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(tmem_slot)),
                 "r"(128u * kAccumulators)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  for (int i = tid; i < WT * R; i += kPipeThreads) scale[i] = a.fscale[i];
  for (int d = tid; d < a.rows; d += kPipeThreads) {
    const int4 q = *reinterpret_cast<const int4*>(a.abmn + 4 * (a.row_begin + d));
    auto at = [&](int i, int k) -> short {
      return (short)(((unsigned)i < (unsigned)E && (unsigned)k < (unsigned)E) ? i * L.GLD + k : L.GS - 1);
    };
    offs[d] = make_short4(at(q.z, q.x), at(q.z, q.y), at(q.w, q.x), at(q.w, q.y));
  }
  for (int i = tid; i < NC; i += kPipeThreads) gram[(size_t)(L.GS - 1) * NC + i] = 0.f;  // remote entry
  // chunks the producers never write (K padding) are zero in both stages
  constexpr int kWritten = (WT * R + 3) / 4;
  for (int item = tid; item < (L.KC - kWritten) * L.RW * 4 * 4; item += kPipeThreads) {
    const int per_part = (L.KC - kWritten) * L.RW * 4;
    const int which = item / per_part, rest = item % per_part;  // (stage, part) and float index
    const size_t off = (size_t)(which >> 1) * L.stage + (size_t)(which & 1) * L.part + (size_t)kWritten * L.RW * 16;
    reinterpret_cast<float*>(feat + off)[rest] = 0.f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  int issued = 0;  // MMA thread: pairs whose MMAs were committed

  if (warp < kProducerThreads / 32) {
    // ---------------------------------------------------------------- producers
    // two teams: warps 0-3 build the even pairs (stage 0), warps 4-7 the odd pairs (stage 1), so
    // one team's field loads are in flight while the other computes. Thread (cell ci, electrode
    // e) builds its row of the operand for all wavenumbers: chunks 0 .. KC - 1 of row ci Ep + e.
    static_assert(WT * R <= 88, "the features of a row fit 22 chunks");
    const int team = warp >> 2, tt = tid & (kTeamThreads - 1), ci = tt >> 6, e = tt & 63;
    const bool on = e < E;
    auto cell_of = [&](int j) {
      return a.c_begin + 2 * ((blockIdx.x + (j / batch) * gridDim.x) * batch + j % batch) + ci;
    };
    auto load_dofs = [&](int j, int (&d)[K]) {
      const int c = cell_of(j);
      const bool valid = on && j < pairs && c < a.c_end;
#pragma unroll
      for (int k = 0; k < K; ++k) d[k] = valid ? __ldg(a.cell_dofs + (int64_t)c * K + k) : -1;
    };
    int dnext[K];
    load_dofs(team, dnext);
    for (int j = team; j < pairs; j += 2) {
      const int s = team;  // == j & 1
      int dof[K];
#pragma unroll
      for (int k = 0; k < K; ++k) dof[k] = dnext[k];
      load_dofs(j + 2, dnext);  // the team's next pair
      const int c = cell_of(j);
      const bool valid = on && c < a.c_end;
      float cf[R][K], x[WT][K];
#pragma unroll
      for (int f = 0; f < R; ++f)
#pragma unroll
        for (int k = 0; k < K; ++k) cf[f][k] = valid ? __ldg(a.features + ((int64_t)c * R + f) * K + k) : 0.f;
      const float* column = a.fields + e;
#pragma unroll
      for (int w = 0; w < WT; ++w)
#pragma unroll
        for (int k = 0; k < K; ++k)
          x[w][k] = dof[k] >= 0 ? __ldg(column + ((int64_t)w * a.N + dof[k]) * E) : 0.f;
      // stage s is free once pair j - 2's MMAs completed
      if ((j >= 2 && !pipe_wait(stage_free + s, ((j >> 1) & 1) ^ 1u, abort)) || *abort) {
        *abort = 1;
        break;
      }
      if (on) {
        unsigned char* row_feat = feat + (size_t)s * L.stage + (size_t)(ci * L.Ep + e) * 16;
        float hi[4], lo[4];
#pragma unroll
        for (int w = 0; w < WT; ++w) {
#pragma unroll
          for (int f = 0; f < R; ++f) {
            const int kl = w * R + f;  // compile-time: chunk kl / 4, lane kl % 4
            float v = 0.f;
#pragma unroll
            for (int k = 0; k < K; ++k) v = fmaf(cf[f][k], x[w][k], v);
            v *= scale[w * R + f];
            hi[kl & 3] = tf32_round(v);
            lo[kl & 3] = v - hi[kl & 3];
            if ((kl & 3) == 3) {
              const size_t off = (size_t)(kl >> 2) * L.RW * 16;
              *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
              *reinterpret_cast<float4*>(row_feat + L.part + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            }
          }
        }
        constexpr int last = WT * R;
        if constexpr (last % 4 != 0) {  // a partial last chunk: its remaining lanes are padding
#pragma unroll
          for (int i = last % 4; i < 4; ++i) hi[i] = lo[i] = 0.f;
          const size_t off = (size_t)(last >> 2) * L.RW * 16;
          *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
          *reinterpret_cast<float4*>(row_feat + L.part + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_arrive(stage_full + s);
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA issue (one thread)
    if (lane == 0) {
      for (int j = 0; j < pairs; ++j) {
        const int s = j & 1, acc_index = j % kAccumulators;
        if (!pipe_wait(stage_full + s, (j >> 1) & 1, abort) ||
            (j >= kAccumulators && !pipe_wait(acc_free + acc_index, ((j >> 2) & 1) ^ 1u, abort))) {
          *abort = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t base = smem_addr(feat + (size_t)s * L.stage);
        uint64_t dh = operand_desc(base, (uint32_t)L.RW * 16, 128);
        uint64_t dl = operand_desc(base + (uint32_t)L.part, (uint32_t)L.RW * 16, 128);
        const uint64_t step = (uint64_t)(2 * L.RW * 16) >> 4;
        const uint32_t idesc = tf32_idesc(kPipeM, L.RW);
        const uint32_t acc = tmem + (uint32_t)(acc_index * 128);
        for (int ks = 0; ks < L.KS; ++ks) {
          mma_tf32(acc, dh, dh, idesc, ks > 0 ? 1u : 0u);
          mma_tf32(acc, dh, dl, idesc, 1u);
          mma_tf32(acc, dl, dh, idesc, 1u);
          dh += step;
          dl += step;
        }
        commit_to(stage_free + s);
        commit_to(acc_full + acc_index);
        issued = j + 1;
      }
    }
  } else {
    // ---------------------------------------------------------------- epilogue
    const int et = tid - kProducerThreads, ew = warp - kProducerThreads / 32;  // warps 8 .. 14
    const int lq = ew & 3, hh = ew >> 2;  // TMEM lane quarter lq, columns of cell hh
    const int first = 32 * lq - hh * L.Ep;  // lane 0's row within cell hh
    const bool busy = first < E && first + 32 > 0;  // warp-uniform: some rows of cell hh here
    const int lr = first + lane;
    const bool mine = lr >= 0 && lr < E;
    for (int j = 0; j < pairs; ++j) {
      const int acc_index = j % kAccumulators, q = j % batch;
      if (et == 0) {
        bool done;
        if (a.first_wait_polls == 0) {
          done = pipe_wait(acc_full + acc_index, (j >> 2) & 1, abort);
        } else {  // failure-detection tests: a few non-blocking polls
          done = false;
          for (unsigned polls = 0; !done && polls < a.first_wait_polls; ++polls)
            done = mbar_test_wait(smem_addr(acc_full + acc_index), (j >> 2) & 1);
        }
        if (!done) *abort = 1;
        *epilogue_flag = *abort;
      }
      named_sync(2, kEpilogueThreads);
      if (*epilogue_flag) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      if (busy) {
        const uint32_t base = tmem + ((uint32_t)(32 * lq) << 16) + (uint32_t)(acc_index * 128 + hh * L.Ep);
        float* g = gram + (size_t)(mine ? lr : 0) * L.GLD * NC + (2 * q + hh);  // entry (lr, col) of cell 2q + hh
        uint32_t v[4][16];
#pragma unroll
        for (int b = 0; b < 4; ++b)
          if (16 * b < L.Ep) tmem_load16(base + 16 * b, v[b]);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (mine) {
#pragma unroll
          for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int jj = 0; jj < 16; ++jj)
              if (16 * b + jj < E) g[(size_t)(16 * b + jj) * NC] = __uint_as_float(v[b][jj]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      mbar_arrive(acc_free + acc_index);
      if (q == batch - 1 || j == pairs - 1) {
        named_sync(2, kEpilogueThreads);  // every Gram of the batch is staged
        const int cfirst = a.c_begin + 2 * (blockIdx.x + (j / batch) * gridDim.x) * batch;
        const int ncells = min(2 * (q + 1), a.c_end - cfirst);
        for (int d = et; ncells > 0 && d < a.rows; d += kEpilogueThreads) {
          const short4 o = offs[d];
          float v[8];
          if (NC == 8) {  // the 8 cells of an entry are 32 contiguous bytes: two float4 loads each
            const float4* gx = reinterpret_cast<const float4*>(gram + (size_t)o.x * 8);
            const float4* gy = reinterpret_cast<const float4*>(gram + (size_t)o.y * 8);
            const float4* gz = reinterpret_cast<const float4*>(gram + (size_t)o.z * 8);
            const float4* gw = reinterpret_cast<const float4*>(gram + (size_t)o.w * 8);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const float4 X = gx[h], Y = gy[h], Z = gz[h], W = gw[h];
              v[4 * h + 0] = -((X.x - Y.x) - (Z.x - W.x));
              v[4 * h + 1] = -((X.y - Y.y) - (Z.y - W.y));
              v[4 * h + 2] = -((X.z - Y.z) - (Z.z - W.z));
              v[4 * h + 3] = -((X.w - Y.w) - (Z.w - W.w));
            }
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i)
              v[i] = i < ncells ? -((gram[(size_t)o.x * NC + i] - gram[(size_t)o.y * NC + i]) -
                                    (gram[(size_t)o.z * NC + i] - gram[(size_t)o.w * NC + i]))
                                : 0.f;
          }
          float* out = a.out + (int64_t)d * a.ldo + cfirst;
          if (ncells == 8 && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
            reinterpret_cast<float4*>(out)[0] = make_float4(v[0], v[1], v[2], v[3]);
            reinterpret_cast<float4*>(out)[1] = make_float4(v[4], v[5], v[6], v[7]);
          } else {
            for (int i = 0; i < ncells; ++i) out[i] = v[i];
          }
        }
        named_sync(2, kEpilogueThreads);  // before the next batch overwrites the Grams
      }
    }
  }

  // ---------------------------------------------------------------- teardown
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (*abort) {
    if (warp == kMmaWarp && lane == 0) {
      atomicExch(error, 1);
      if (issued > 0) {  // the last commit covers every MMA issued; full bounded wait
        const int last = issued - 1;
        for (uint32_t polls = 0; polls < kPipeWaitLimit; ++polls)
          if (mbar_try_wait(smem_addr(stage_free + (last & 1)), (uint32_t)((last >> 1) & 1))) break;
      }
    }
    for (int sg = 0; sg < my_supers; ++sg) {  // NaN in every column of this block
      const int cfirst = a.c_begin + 2 * (blockIdx.x + sg * gridDim.x) * batch;
      const int ncells = min(2 * batch, a.c_end - cfirst);
      for (int idx = tid; ncells > 0 && idx < a.rows * ncells; idx += kPipeThreads)
        a.out[(int64_t)(idx / ncells) * a.ldo + cfirst + idx % ncells] = __int_as_float(0x7fc00000);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(128u * kAccumulators)
                 : "memory");
}

template __global__ void jacobian_tcpipe_kernel<3, 5, kPipeStaticW>(JacobianArgs, int, int*);

// The pipelined kernel applies to the flat 2.5D operator's shape (P1 triangles: K = 3, R = 5,
// the 17-wavenumber quadrature) with at most 48 electrodes (so TMEM lanes 96-127, whose warp
// issues the MMAs, hold no Gram row) and 4096 rows; the Gram batch is
// the largest of 4, 2, 1 pairs whose shared memory fits one block per SM.
int jacobian_tcpipe_batch(int E, int W, int R, int K, int rows) {
  if (K != 3 || R != 5 || W != kPipeStaticW || E > 48 || rows > kPipeRowTable) return 0;
  for (int batch = 4; batch >= 1; batch >>= 1)
    if (pipe_layout(E, W, R, batch, rows).total <= 227 * 1024) return batch;
  return 0;
}

cudaError_t launch_jacobian_tcpipe(const JacobianArgs& a, int batch, int* error, int sms, cudaStream_t s) {
  const size_t smem = pipe_layout(a.E, a.W, a.R, batch, a.rows).total;
  const int pairs = (a.c_end - a.c_begin + 1) / 2;
  const int supers = (pairs + batch - 1) / batch;
  const int blocks = supers < sms ? supers : sms;
  auto kernel = jacobian_tcpipe_kernel<3, 5, kPipeStaticW>;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  launch_chained(kernel, blocks, kPipeThreads, smem, s, a, batch, error);
  return cudaGetLastError();
}

}  // namespace adt
