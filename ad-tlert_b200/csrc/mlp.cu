// BF16 training and inference kernels of the learned apparent-resistivity surrogate.
//
// The surrogate is a multilayer perceptron; every layer is a GEMM C = A B^T of row-major BF16
// operands (A: M x K, B: N x K, both K contiguous) accumulated in FP32:
//   forward   Z_l = Y_{l-1} W_l^T + b_l,  Y_l = gelu(Z_l)      (A = activations, B = weights)
//   backward  G_l = (G_{l+1} W_{l+1}) * gelu'(Z_l)             (A = G_{l+1}, B = W_{l+1}^T)
//             dW_l = G_l^T Y_{l-1}                             (A = G_l^T, B = Y_{l-1}^T)
// M, N are multiples of 128 and K of 64 (the caller pads).
//
// gemm_bf16_kernel: one CTA (128 threads) per 128 x 128 output tile and K range (split-K fills the
// multiprocessors when the tile grid is small). Operands stream through a 4-stage ring in shared
// memory (cp.async, 16-byte chunks, canonical K-major no-swizzle layout: core matrices of 8 rows
// x 16 bytes, chunk kc of row r at kc * 2048 + (r / 8) * 128 + (r % 8) * 16). Thread 0 issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = 128, K = 16 per instruction; 4 per 64-wide
// chunk) into a 128-column FP32 accumulator in tensor memory and commits each chunk to that
// stage's mbarrier, which frees the stage for the chunk STAGES - 1 later. The accumulator is read
// back with tcgen05.ld (warp w owns lanes 32 w .. 32 w + 31 = tile rows) and written as an FP32
// partial tile; mlp_epilogue_kernel sums the splits in fixed order and applies the layer's
// epilogue, so results are bitwise repeatable.
//
// Every mbarrier wait is bounded: a CTA that gives up raises the caller's error flag, waits
// (again bounded) for its own MMAs, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "adt_internal.h"

namespace {

constexpr int kGemmThreads = 128;
constexpr int kTile = 128;         // M and N of a tile (one MMA: M = 128, N = 128)
constexpr int kChunk = 64;         // K per pipeline stage (four K = 16 MMAs)
constexpr int kStages = 4;
constexpr int kStageBytes = 2 * kTile * kChunk * 2;  // A and B tiles, BF16
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 format: version 1 at bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulate (bit 4), BF16 A (bits 7-9 = 1) and B
// (bits 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t bf16_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void tmem_load8(uint32_t addr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(addr));
}

// Copies K-chunk `chunk` of the A and B tiles into stage `stage` (thread t: rows t % 128 ...,
// chunks in order; 16 copies per thread).
__device__ __forceinline__ void load_stage(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
                                           int K, int m0, int n0, int k0, unsigned char* stage_base) {
  const uint32_t base = smem_u32(stage_base);
  const int r = threadIdx.x;  // one row of A and one row of B per thread
  const __nv_bfloat16* a_row = A + (size_t)(m0 + r) * K + k0;
  const __nv_bfloat16* b_row = B + (size_t)(n0 + r) * K + k0;
  const uint32_t row_off = (uint32_t)((r >> 3) * 128 + (r & 7) * 16);
#pragma unroll
  for (int kc = 0; kc < kChunk / 8; ++kc) {
    cp_async16(base + kc * 2048 + row_off, a_row + kc * 8);
    cp_async16(base + kTile * kChunk * 2 + kc * 2048 + row_off, b_row + kc * 8);
  }
}

}  // namespace

namespace {

// Partial tile of C = A B^T over the K range of split blockIdx.z into partial[split][M][N].
__global__ void __launch_bounds__(kGemmThreads, 1) gemm_bf16_kernel(const __nv_bfloat16* __restrict__ A,
                                                                    const __nv_bfloat16* __restrict__ B, int M, int N,
                                                                    int K, int chunks_per_split,
                                                                    float* __restrict__ partial, int* error) {
  adt::chain_wait();
  extern __shared__ __align__(1024) unsigned char gemm_sm[];
  unsigned char* stages = gemm_sm;
  uint64_t* bars = reinterpret_cast<uint64_t*>(gemm_sm + kStages * kStageBytes);  // [kStages]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kStages);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.x * kTile, m0 = blockIdx.y * kTile;
  const int total_chunks = K / kChunk;
  const int c0 = blockIdx.z * chunks_per_split;
  const int chunks = min(chunks_per_split, total_chunks - c0);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + s)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(128u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t idesc = bf16_idesc(kTile, kTile);
  bool failed = false;
  int issued = 0;  // chunks whose MMAs have been committed

  // prologue: chunks 0 .. kStages - 2
  for (int j = 0; j < kStages - 1; ++j) {
    if (j < chunks) load_stage(A, B, K, m0, n0, (c0 + j) * kChunk, stages + j * kStageBytes);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int j = 0; j < chunks && !failed; ++j) {
    const int stage = j % kStages;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a_base = smem_u32(stages + stage * kStageBytes);
      const uint32_t b_base = a_base + kTile * kChunk * 2;
#pragma unroll
      for (int ks = 0; ks < kChunk / 16; ++ks) {
        // K = 16 BF16 = two 16-byte chunks, 2048 bytes apart (leading byte offset); 8-row core
        // matrices 128 bytes apart (stride byte offset)
        const uint64_t a = smem_desc(a_base + ks * 2 * 2048, 2048, 128);
        const uint64_t b = smem_desc(b_base + ks * 2 * 2048, 2048, 128);
        mma_bf16(tmem, a, b, idesc, (j > 0 || ks > 0) ? 1u : 0u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(bars + stage))
                   : "memory");
    }
    issued = j + 1;
    // refill the stage chunk j - 1 used, once its MMAs have read it
    const int next = j + kStages - 1;
    if (next < chunks) {
      const int ns = next % kStages;
      if (j >= 1 && !mbar_wait(smem_u32(bars + ns), (uint32_t)(((j - 1) / kStages) & 1))) failed = true;
      if (!failed) load_stage(A, B, K, m0, n0, (c0 + next) * kChunk, stages + ns * kStageBytes);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    failed = __syncthreads_or(failed);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  // the last commit covers every MMA this thread issued
  if (!failed && chunks > 0) {
    const int last = chunks - 1;
    if (!mbar_wait(smem_u32(bars + last % kStages), (uint32_t)((last / kStages) & 1))) failed = true;
  }
  failed = __syncthreads_or(failed);
  if (failed) {
    if (tid == 0) atomicExch(error, 1);
    // drain: the latest commit covers every MMA issued; bounded again, before TMEM is freed
    if (issued > 0) mbar_wait(smem_u32(bars + (issued - 1) % kStages), (uint32_t)(((issued - 1) / kStages) & 1));
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    float* out = partial + ((size_t)blockIdx.z * M + m0 + warp * 32 + lane) * N + n0;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c = 0; c < kTile; c += 8) {
      uint32_t v[8];
      tmem_load8(lane_base + c, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      float4* dst = reinterpret_cast<float4*>(out + c);
      dst[0] = make_float4(__uint_as_float(v[0]), __uint_as_float(v[1]), __uint_as_float(v[2]), __uint_as_float(v[3]));
      dst[1] = make_float4(__uint_as_float(v[4]), __uint_as_float(v[5]), __uint_as_float(v[6]), __uint_as_float(v[7]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(128u) : "memory");
}

}  // namespace

namespace {

constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;

// GELU, tanh form: 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), and its derivative.
__device__ __forceinline__ float gelu(float z) {
  const float u = kGeluC * (z + kGeluA * z * z * z);
  return 0.5f * z * (1.f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad(float z) {
  const float u = kGeluC * (z + kGeluA * z * z * z);
  const float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * kGeluC * (1.f + 3.f * kGeluA * z * z);
}

enum EpilogueMode { kForwardGelu = 0, kForwardLinear = 1, kBackwardGelu = 2, kPlain = 3 };

// One 32 x 32 tile of the M x N output per block (32 x 8 threads, four rows each): sums the
// split partials in order, applies the mode, writes row-major outputs and, through shared
// memory, the transposed BF16 copy (col_out[n][m]).
__global__ void __launch_bounds__(256) mlp_epilogue_kernel(int mode, const float* __restrict__ partial, int splits,
                                                           int M, int N, const float* __restrict__ bias,
                                                           const __nv_bfloat16* __restrict__ z_in,
                                                           __nv_bfloat16* __restrict__ z_out,
                                                           __nv_bfloat16* __restrict__ row_out,
                                                           __nv_bfloat16* __restrict__ col_out,
                                                           float* __restrict__ f32_out) {
  adt::chain_wait();
  __shared__ float tile[32][33];
  const int n = blockIdx.x * 32 + threadIdx.x;
  const int mb = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int m = mb + i;
    const size_t at = (size_t)m * N + n;
    float sum = 0.f;
    for (int s = 0; s < splits; ++s) sum += partial[(size_t)s * M * N + at];
    float value;
    if (mode == kForwardGelu) {
      const float z = sum + bias[n];
      z_out[at] = __float2bfloat16(z);
      value = gelu(z);
      row_out[at] = __float2bfloat16(value);
    } else if (mode == kForwardLinear) {
      value = sum + bias[n];
      f32_out[at] = value;
    } else if (mode == kBackwardGelu) {
      value = sum * gelu_grad(__bfloat162float(z_in[at]));
      row_out[at] = __float2bfloat16(value);
    } else {
      value = sum;
      f32_out[at] = value;
    }
    tile[i][threadIdx.x] = value;
  }
  if (col_out == nullptr) return;
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int nn = blockIdx.x * 32 + i;
    col_out[(size_t)nn * M + mb + threadIdx.x] = __float2bfloat16(tile[threadIdx.x][i]);
  }
}

// Gradient of the mean squared error over the first n_valid columns: g = 2 (pred - target) /
// (M n_valid) (0 in padding columns), row-major and transposed BF16; per-block squared-error sums.
__global__ void __launch_bounds__(256) mlp_loss_kernel(const float* __restrict__ pred, const float* __restrict__ target,
                                                       int M, int N, int n_valid, __nv_bfloat16* __restrict__ g_row,
                                                       __nv_bfloat16* __restrict__ g_col, float* __restrict__ sums) {
  adt::chain_wait();
  __shared__ float tile[32][33];
  __shared__ float warp_sums[8];
  const int n = blockIdx.x * 32 + threadIdx.x;
  const int mb = blockIdx.y * 32;
  const float scale = 2.f / ((float)M * (float)n_valid);
  float squared = 0.f;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const size_t at = (size_t)(mb + i) * N + n;
    const float diff = n < n_valid ? pred[at] - target[at] : 0.f;
    squared += diff * diff;
    const float g = scale * diff;
    g_row[at] = __float2bfloat16(g);
    tile[i][threadIdx.x] = g;
  }
  for (int offset = 16; offset > 0; offset >>= 1) squared += __shfl_xor_sync(0xffffffffu, squared, offset);
  if (threadIdx.x == 0) warp_sums[threadIdx.y] = squared;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    float total = 0.f;
    for (int w = 0; w < 8; ++w) total += warp_sums[w];
    sums[blockIdx.y * gridDim.x + blockIdx.x] = total;
  }
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int nn = blockIdx.x * 32 + i;
    g_col[(size_t)nn * M + mb + threadIdx.x] = __float2bfloat16(tile[threadIdx.x][i]);
  }
}

// db[n] = sum_m g_col[n][m]: one warp per n, fixed order.
__global__ void __launch_bounds__(256) mlp_bias_grad_kernel(const __nv_bfloat16* __restrict__ g_col, int N, int M,
                                                            float* __restrict__ db) {
  adt::chain_wait();
  const int n = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (n >= N) return;
  float sum = 0.f;
  for (int m = lane; m < M; m += 32) sum += __bfloat162float(g_col[(size_t)n * M + m]);
  for (int offset = 16; offset > 0; offset >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, offset);
  if (lane == 0) db[n] = sum;
}

// Adam on FP32 master parameters (Kingma and Ba 2015); c1 = 1 / (1 - b1^t), c2 = 1 / (1 - b2^t).
// Writes the BF16 copy the GEMMs read.
__global__ void __launch_bounds__(256) mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                                                       float* __restrict__ m, float* __restrict__ v, int64_t n,
                                                       float lr, float b1, float b2, float eps, float c1, float c2,
                                                       __nv_bfloat16* __restrict__ p_bf16) {
  adt::chain_wait();
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    p[i] = pi;
    if (p_bf16 != nullptr) p_bf16[i] = __float2bfloat16(pi);
  }
}

// out[c][r] = in[r][c] for a rows x cols BF16 matrix (both multiples of 32).
__global__ void __launch_bounds__(256) mlp_transpose_kernel(const __nv_bfloat16* __restrict__ in, int rows, int cols,
                                                            __nv_bfloat16* __restrict__ out) {
  adt::chain_wait();
  __shared__ __nv_bfloat16 tile[32][34];
  const int c = blockIdx.x * 32 + threadIdx.x, rb = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) tile[i][threadIdx.x] = in[(size_t)(rb + i) * cols + c];
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8)
    out[(size_t)(blockIdx.x * 32 + i) * rows + rb + threadIdx.x] = tile[threadIdx.x][i];
}

__global__ void __launch_bounds__(256) mlp_to_bf16_kernel(const float* __restrict__ in, int64_t n,
                                                          __nv_bfloat16* __restrict__ out) {
  adt::chain_wait();
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
    out[i] = __float2bfloat16(in[i]);
}

int stride_blocks(int64_t n) {
  const int64_t blocks = (n + 255) / 256;
  return (int)(blocks < 1 ? 1 : (blocks > 148 * 16 ? 148 * 16 : blocks));
}

}  // namespace

// ------------------------------------------------------------------------------------ C ABI

extern "C" int32_t adt_mlp_gemm_splits(int32_t m, int32_t n, int32_t k, int32_t multiprocessors) {
  if (m <= 0 || n <= 0 || k <= 0 || m % kTile || n % kTile || k % kChunk || multiprocessors <= 0) return 0;
  const int tiles = (m / kTile) * (n / kTile), chunks = k / kChunk;
  int splits = (multiprocessors + tiles - 1) / tiles;
  splits = splits < 1 ? 1 : (splits > chunks ? chunks : splits);
  if (splits > 16) splits = 16;
  const int per = (chunks + splits - 1) / splits;
  return (chunks + per - 1) / per;  // every split gets at least one chunk
}

extern "C" adt_status adt_mlp_gemm(const void* a, const void* b, int32_t m, int32_t n, int32_t k, int32_t splits,
                                   float* partial, size_t partial_floats, int32_t* error, adt_stream stream) {
  if (!a || !b || !partial || !error || m <= 0 || n <= 0 || k <= 0 || m % kTile || n % kTile || k % kChunk ||
      splits <= 0 || splits > k / kChunk)
    return ADT_INVALID_ARG;
  const int chunks = k / kChunk, per = (chunks + splits - 1) / splits;
  if ((chunks + per - 1) / per != splits) return ADT_INVALID_ARG;  // a split would have no chunk
  if (partial_floats < (size_t)splits * m * n) return ADT_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) return ADT_INVALID_ARG;
  const size_t smem = (size_t)kStages * kStageBytes + kStages * sizeof(uint64_t) + 16;
  static bool raised = false;
  if (!raised) {
    if (cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return ADT_CUDA_ERROR;
    raised = true;
  }
  const cudaError_t err = adt::launch_chained(gemm_bf16_kernel, dim3(n / kTile, m / kTile, splits), dim3(kGemmThreads),
                                              smem, (cudaStream_t)stream, (const __nv_bfloat16*)a,
                                              (const __nv_bfloat16*)b, (int)m, (int)n, (int)k, per, partial,
                                              (int*)error);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}

extern "C" adt_status adt_mlp_epilogue(int32_t mode, const float* partial, int32_t splits, int32_t m, int32_t n,
                                       const float* bias, const void* z_in, void* z_out, void* row_out, void* col_out,
                                       float* f32_out, adt_stream stream) {
  if (!partial || splits <= 0 || m <= 0 || n <= 0 || m % 32 || n % 32 || mode < 0 || mode > 3) return ADT_INVALID_ARG;
  if ((mode == kForwardGelu && (!bias || !z_out || !row_out)) || (mode == kForwardLinear && (!bias || !f32_out)) ||
      (mode == kBackwardGelu && (!z_in || !row_out)) || (mode == kPlain && !f32_out))
    return ADT_INVALID_ARG;
  const cudaError_t err = adt::launch_chained(
      mlp_epilogue_kernel, dim3(n / 32, m / 32), dim3(32, 8), 0, (cudaStream_t)stream, (int)mode, partial,
      (int)splits, (int)m, (int)n, bias, (const __nv_bfloat16*)z_in, (__nv_bfloat16*)z_out, (__nv_bfloat16*)row_out,
      (__nv_bfloat16*)col_out, f32_out);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}

extern "C" adt_status adt_mlp_loss(const float* pred, const float* target, int32_t m, int32_t n, int32_t n_valid,
                                   void* g_row, void* g_col, float* sums, adt_stream stream) {
  if (!pred || !target || !g_row || !g_col || !sums || m <= 0 || n <= 0 || m % 32 || n % 32 || n_valid <= 0 ||
      n_valid > n)
    return ADT_INVALID_ARG;
  const cudaError_t err = adt::launch_chained(mlp_loss_kernel, dim3(n / 32, m / 32), dim3(32, 8), 0,
                                              (cudaStream_t)stream, pred, target, (int)m, (int)n, (int)n_valid,
                                              (__nv_bfloat16*)g_row, (__nv_bfloat16*)g_col, sums);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}

extern "C" adt_status adt_mlp_bias_grad(const void* g_col, int32_t n, int32_t m, float* db, adt_stream stream) {
  if (!g_col || !db || n <= 0 || m <= 0) return ADT_INVALID_ARG;
  const cudaError_t err = adt::launch_chained(mlp_bias_grad_kernel, dim3((n + 7) / 8), dim3(256), 0,
                                              (cudaStream_t)stream, (const __nv_bfloat16*)g_col, (int)n, (int)m, db);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}

extern "C" adt_status adt_mlp_adam(float* params, const float* grads, float* first, float* second, int64_t count,
                                   float lr, float beta1, float beta2, float eps, float correction1, float correction2,
                                   void* params_bf16, adt_stream stream) {
  if (!params || !grads || !first || !second || count <= 0) return ADT_INVALID_ARG;
  const cudaError_t err = adt::launch_chained(mlp_adam_kernel, dim3(stride_blocks(count)), dim3(256), 0,
                                              (cudaStream_t)stream, params, grads, first, second, count, lr, beta1,
                                              beta2, eps, correction1, correction2, (__nv_bfloat16*)params_bf16);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}

extern "C" adt_status adt_mlp_transpose(const void* in, int32_t rows, int32_t cols, void* out, adt_stream stream) {
  if (!in || !out || rows <= 0 || cols <= 0 || rows % 32 || cols % 32) return ADT_INVALID_ARG;
  const cudaError_t err = adt::launch_chained(mlp_transpose_kernel, dim3(cols / 32, rows / 32), dim3(32, 8), 0,
                                              (cudaStream_t)stream, (const __nv_bfloat16*)in, (int)rows, (int)cols,
                                              (__nv_bfloat16*)out);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}

extern "C" adt_status adt_mlp_to_bf16(const float* in, int64_t count, void* out, adt_stream stream) {
  if (!in || !out || count <= 0) return ADT_INVALID_ARG;
  const cudaError_t err = adt::launch_chained(mlp_to_bf16_kernel, dim3(stride_blocks(count)), dim3(256), 0,
                                              (cudaStream_t)stream, in, count, (__nv_bfloat16*)out);
  return err == cudaSuccess ? ADT_OK : ADT_CUDA_ERROR;
}
