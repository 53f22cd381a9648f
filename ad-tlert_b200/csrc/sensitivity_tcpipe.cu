// Normal-quadrupole Jacobian on tcgen05 with warp roles and a two-deep pipeline.
//
// Same contraction and operand layout as jacobian_tc_kernel (sensitivity_tc.cu): the features of
// a pair of cells (hi/lo TF32 split) are stacked as the rows of one K-major operand S, and D =
// S S^T in tensor memory holds both electrode Grams; J[d][c] = -(G[M][A] - G[M][B] - G[N][A] +
// G[N][B]). What changes is how the per-pair chain overlaps. One persistent block per SM:
//
//   producer warps 0-7   build the features of pair j into operand stage j % 2 (thread: cell,
//                        half of the wavenumbers, electrode), from registers loaded one pair
//                        ahead (cell dofs two pairs ahead, so the dependent field loads are
//                        issued a whole pair early), and arrive on stage_full[j % 2].
//   MMA warp 15          one thread issues pair j's MMAs into accumulator j % 4 (TMEM columns
//                        128 (j % 4)) and commits them to stage_free[j % 2] and acc_full[j % 4].
//   epilogue warps 8-14  wait for acc_full[j % 4], read the Grams back (warp 8 + w: TMEM lanes
//                        32 (w % 4) .., the columns of cell w / 4; 16-column loads, one wait),
//                        release the accumulator (acc_free[j % 4]), and after `batch` pairs
//                        write every row of the batch's 2 batch consecutive cells at once (32
//                        bytes per row for 4 pairs).
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
  float* gram = reinterpret_cast<float*>(pipe_sm + L.feat);  // [batch][2][GS]
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
      mbar_init(stage_full + i, 4 * E);  // the active producers (4 E <= 192)
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
  for (int i = tid; i < batch * 2; i += kPipeThreads) gram[(size_t)i * L.GS + L.GS - 1] = 0.f;
  // chunks the producers never write (K padding) are zero in both stages
  constexpr int kWritten = 2 * R + ((WT - 8) * R + 3) / 4;
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
    // thread tid < 4 E: (cell ci, half hf, electrode e), packed so that whole warps work and the
    // rest (warps past 4 E threads) leave the role at once; wavenumbers 0 .. 7 (hf = 0: chunks
    // 0 .. 2R - 1) or 8 .. WT - 1 (hf = 1: chunks 2R .. KC - 1); whole 16-byte chunks stored
    constexpr int WH = 8, WB = WT - WH, CH0 = WH * R / 4;
    static_assert(WB >= WH && WB <= 16 && (WH * R) % 4 == 0, "two halves of at most 16 wavenumbers");
    const int ci = tid / (2 * E), hf = (tid / E) & 1, e = tid % E;
    const bool on = tid < 4 * E;
    const int w0 = hf * WH, wn = hf ? WB : WH;
    auto cell_of = [&](int j) {
      return a.c_begin + 2 * ((blockIdx.x + (j / batch) * gridDim.x) * batch + j % batch) + ci;
    };
    auto load_dofs = [&](int j, int (&d)[K]) {
      const int c = cell_of(j);
      const bool valid = on && j < pairs && c < a.c_end;
#pragma unroll
      for (int k = 0; k < K; ++k) d[k] = valid ? __ldg(a.cell_dofs + (int64_t)c * K + k) : -1;
    };
    float x[WB][K], cf[R][K];
    int dnext[K];
    auto load_pair = [&](int j, const int (&d)[K]) {  // fields and template factors of pair j
      const int c = cell_of(j);
      const bool valid = on && j < pairs && c < a.c_end;
#pragma unroll
      for (int f = 0; f < R; ++f)
#pragma unroll
        for (int k = 0; k < K; ++k) cf[f][k] = valid ? __ldg(a.features + ((int64_t)c * R + f) * K + k) : 0.f;
#pragma unroll
      for (int jj = 0; jj < WB; ++jj)
#pragma unroll
        for (int k = 0; k < K; ++k)
          x[jj][k] = (jj < wn && d[k] >= 0) ? __ldg(a.fields + ((int64_t)(w0 + jj) * a.N + d[k]) * E + e) : 0.f;
    };
    {
      int d0[K];
      load_dofs(0, d0);
      load_pair(0, d0);
      load_dofs(1, dnext);
    }
    for (int j = 0; on && j < pairs; ++j) {  // idle producer threads leave at once
      const int s = j & 1;
      // stage s is free once pair j - 2's MMAs completed (each thread waits: producers need no
      // barrier among themselves)
      if ((j >= 2 && !pipe_wait(stage_free + s, ((j >> 1) & 1) ^ 1u, abort)) || *abort) {
        *abort = 1;
        break;
      }
      if (on) {
        const int nch = hf ? L.KC - CH0 : CH0;
        unsigned char* row_feat = feat + (size_t)s * L.stage + ((size_t)(hf * CH0) * L.RW + ci * L.Ep + e) * 16;
        float hi[4] = {0.f, 0.f, 0.f, 0.f}, lo[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int jj = 0; jj < WB; ++jj) {
#pragma unroll
          for (int f = 0; f < R; ++f) {
            const int kl = jj * R + f;  // compile-time: chunk kl / 4, lane kl % 4
            float v = 0.f;
            if (jj < wn) {
#pragma unroll
              for (int k = 0; k < K; ++k) v = fmaf(cf[f][k], x[jj][k], v);
              v *= scale[(w0 + jj) * R + f];
            }
            hi[kl & 3] = tf32_round(v);
            lo[kl & 3] = v - hi[kl & 3];
            if ((kl & 3) == 3 && (kl >> 2) < nch) {
              const size_t off = (size_t)(kl >> 2) * L.RW * 16;
              *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
              *reinterpret_cast<float4*>(row_feat + L.part + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            }
          }
        }
        constexpr int last = WB * R;
        if constexpr (last % 4 != 0) {
#pragma unroll
          for (int i = last % 4; i < 4; ++i) hi[i] = lo[i] = 0.f;
          if ((last >> 2) < nch) {
            const size_t off = (size_t)(last >> 2) * L.RW * 16;
            *reinterpret_cast<float4*>(row_feat + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(row_feat + L.part + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_arrive(stage_full + s);
      // prefetch: fields of pair j + 1 (its dofs arrived during pair j), dofs of pair j + 2
      load_pair(j + 1, dnext);
      load_dofs(j + 2, dnext);
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
        float* g = gram + ((size_t)q * 2 + hh) * L.GS + (size_t)(mine ? lr : 0) * L.GLD;
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
              if (16 * b + jj < E) g[16 * b + jj] = __uint_as_float(v[b][jj]);
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
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float* gc = gram + (size_t)i * L.GS;
            v[i] = i < ncells ? -((gc[o.x] - gc[o.y]) - (gc[o.z] - gc[o.w])) : 0.f;
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
