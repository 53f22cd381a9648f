// Content fingerprints of conductivity models: the keys of the operators' field caches.
//
// A model's bytes are read as 32-bit words x_i (i = 0 .. n-1) and summed in two independent
// 64-bit lanes,
//
//   h_0 = sum_i mix(x_i + (i + 1) * P_0),   h_1 = sum_i mix((x_i * 2^32 + x_i) ^ ((i + 1) * P_1))
//
// modulo 2^64, where mix is the splitmix64 output function (S. Vigna, "Further scramblings of
// Marsaglia's xorshift generators", 2017) and P_0, P_1 are odd constants. Integer addition is
// exact and commutative, so any reduction order gives the same 128 bits: the device kernel (one
// block per model, for models already in GPU memory) and the host loop (for models in host
// memory) agree bit for bit, and only 16 bytes per model cross the bus for a device model.
// Accidental collisions of two different models have probability about 2^-128; the fingerprint
// is not meant to resist deliberately constructed inputs.
#include "adt_internal.h"

namespace {

constexpr uint64_t kLane0 = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kLane1 = 0xD1B54A32D192ED03ull;
constexpr int kFingerprintThreads = 512;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 27;
  z *= 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z;
}

__host__ __device__ __forceinline__ void accumulate(uint64_t word, uint64_t position, uint64_t& h0, uint64_t& h1) {
  h0 += mix64(word + position * kLane0);
  h1 += mix64(((word << 32) | word) ^ (position * kLane1));
}

__global__ void __launch_bounds__(kFingerprintThreads) fingerprint_kernel(const uint32_t* __restrict__ words,
                                                                          int64_t per_model,
                                                                          uint64_t* __restrict__ out) {
  adt::chain_wait();
  const uint32_t* x = words + (int64_t)blockIdx.x * per_model;
  uint64_t h0 = 0, h1 = 0;
  for (int64_t i = threadIdx.x; i < per_model; i += kFingerprintThreads)
    accumulate(__ldg(x + i), (uint64_t)(i + 1), h0, h1);
  for (int offset = 16; offset > 0; offset >>= 1) {
    h0 += __shfl_xor_sync(0xffffffffu, h0, offset);
    h1 += __shfl_xor_sync(0xffffffffu, h1, offset);
  }
  __shared__ uint64_t partial[2][kFingerprintThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    partial[0][warp] = h0;
    partial[1][warp] = h1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t s0 = 0, s1 = 0;
    for (int w = 0; w < kFingerprintThreads / 32; ++w) {
      s0 += partial[0][w];
      s1 += partial[1][w];
    }
    out[2 * blockIdx.x] = s0;
    out[2 * blockIdx.x + 1] = s1;
  }
}

bool bad_shape(int64_t bytes_per_model, int32_t models) {
  return models <= 0 || bytes_per_model <= 0 || bytes_per_model % 4 != 0 || models > 65535;
}

}  // namespace

extern "C" adt_status adt_fingerprint(adt_plan* p, const void* models_data, int64_t bytes_per_model, int32_t models,
                                      uint64_t* fingerprints, adt_stream stream) {
  if (!p || !models_data || !fingerprints || bad_shape(bytes_per_model, models))
    return adt::fail(p, ADT_INVALID_ARG, "adt_fingerprint: invalid arguments");
  if ((reinterpret_cast<uintptr_t>(models_data) & 3) != 0)
    return adt::fail(p, ADT_INVALID_ARG, "adt_fingerprint: models must be 4-byte aligned");
  adt::launch_chained(fingerprint_kernel, dim3(models), dim3(kFingerprintThreads), 0, (cudaStream_t)stream,
                      static_cast<const uint32_t*>(models_data), bytes_per_model / 4, fingerprints);
  p->launches++;
  return adt::check_launch(p, "fingerprint");
}

extern "C" adt_status adt_fingerprint_host(const void* models_data, int64_t bytes_per_model, int32_t models,
                                           uint64_t* fingerprints) {
  if (!models_data || !fingerprints || bad_shape(bytes_per_model, models)) return ADT_INVALID_ARG;
  const int64_t per_model = bytes_per_model / 4;
  for (int32_t m = 0; m < models; ++m) {
    const unsigned char* base = static_cast<const unsigned char*>(models_data) + (int64_t)m * bytes_per_model;
    uint64_t h0 = 0, h1 = 0;
    for (int64_t i = 0; i < per_model; ++i) {
      uint32_t word;
      __builtin_memcpy(&word, base + 4 * i, 4);
      accumulate(word, (uint64_t)(i + 1), h0, h1);
    }
    fingerprints[2 * m] = h0;
    fingerprints[2 * m + 1] = h1;
  }
  return ADT_OK;
}
