// adt_measure_static: the measurement (integrated electrode potentials -> normal and reciprocal
// transfer resistances) without any device allocation.
//
// Who needs it: callers that may not call cudaMalloc once they are running -- code whose GPU
// memory is fully reserved up front by another allocator (a framework's memory pool, a
// fixed-budget service process), or real-time loops that must not block on the driver's
// allocator. adt_measure keeps its potential table in plan memory that it grows with cudaMalloc
// on first use and whenever more models arrive; this variant keeps the table in a fixed array
// compiled into the library instead.
//
// The table is a file-scope __device__ array of kStaticPotentials doubles (512 KiB). Every GPU
// that loads this library holds one copy of it until the process exits, and every call shares
// that copy: two calls that overlap on the GPU (different streams, or different host threads on
// the same device) race on it, so callers must order them. The array keeps the previous call's
// contents; nothing needs clearing, because the potentials kernel writes every entry it later
// reads (the zero remote row and column included).
//
// In host code the array's name is only a host-side stand-in, not a device address, so the device
// address is fetched with cudaGetSymbolAddress once per device (with that device current) and
// cached. That happens during the first call on each device, so make that first call before any
// stream capture. The cached address belongs to the device's primary context as it was then: a
// cudaDeviceReset (or any teardown of that context) after the first call is not supported, since
// the reloaded module may place the array elsewhere.
//
// Both kernels are launched like the rest of the library (adt::launch_chained: programmatic
// stream serialization; each kernel waits on the grid before it as its first statement).
#include <mutex>

#include "adt_internal.h"
#include "kernels.h"

namespace {

constexpr size_t kStaticPotentials = 65536;  // models * (E+1)^2 doubles, 512 KiB

static __device__ __align__(256) double g_static_potentials[kStaticPotentials];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_address[kMaxDevices] = {};

// Device address of the table on `device` (fetched once, with that device current).
adt_status static_table(adt_plan* p, int device, double** out) {
  if (device < 0 || device >= kMaxDevices)
    return adt::fail(p, ADT_INVALID_ARG, "device ordinal out of range for the static measurement table");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_address[device]) {
    int previous = 0;
    if (cudaGetDevice(&previous) != cudaSuccess)
      return adt::fail(p, ADT_CUDA_ERROR, "cudaGetDevice failed");
    if (previous != device && cudaSetDevice(device) != cudaSuccess)
      return adt::fail(p, ADT_CUDA_ERROR, "cudaSetDevice failed");
    void* address = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&address, g_static_potentials);
    if (previous != device) cudaSetDevice(previous);
    if (err != cudaSuccess || !address)
      return adt::fail(p, ADT_CUDA_ERROR,
                       std::string("cudaGetSymbolAddress of the static measurement table failed: ") +
                           cudaGetErrorString(err));
    g_address[device] = static_cast<double*>(address);
  }
  *out = g_address[device];
  return ADT_OK;
}

// Blocks of 256 threads for `work` grid-stride items: at most 32 per multiprocessor.
inline int grid_for(int64_t work, int sms) {
  const int64_t blocks = (work + 255) / 256;
  const int64_t cap = (int64_t)sms * 32;
  return (int)(blocks < 1 ? 1 : (blocks > cap ? cap : blocks));
}

}  // namespace

extern "C" adt_status adt_measure_static(adt_plan* p, const float* fields, int32_t models,
                                         double* normal, double* reciprocal, adt_stream stream) {
  if (!p || !fields || !normal || !reciprocal || models <= 0)
    return adt::fail(p, ADT_INVALID_ARG, "invalid measure arguments");
  const size_t need = (size_t)models * (p->E + 1) * (p->E + 1);
  if (need > kStaticPotentials)
    return adt::fail(p, ADT_INVALID_ARG,
                     "adt_measure_static: models * (electrodes + 1)^2 = " + std::to_string(need) +
                         " exceeds the static table of " + std::to_string(kStaticPotentials) +
                         " entries; measure fewer models per call");
  double* table = nullptr;
  const adt_status st = static_table(p, p->device, &table);
  if (st != ADT_OK) return st;
  adt::MeasureArgs a;
  a.fields = fields;
  a.f_double = 0;
  a.weights = p->weights;
  a.rcv_dofs = p->rcv_dofs;
  a.rcv_w = p->rcv_w;
  a.abmn = p->abmn;
  a.normal = normal;
  a.reciprocal = reciprocal;
  a.potentials = nullptr;
  a.base_normal = nullptr;
  a.base_recip = nullptr;
  a.W = p->W;
  a.N = p->N;
  a.E = p->E;
  a.RW = p->RW;
  a.D = p->D;
  a.combine = 0;
  cudaStream_t s = (cudaStream_t)stream;
  adt::launch_chained(adt::potentials_kernel, grid_for((int64_t)need * 32, p->sms), 256, 0, s, a, models,
                      table);  // a warp per entry
  adt::launch_chained(adt::transfers_kernel, grid_for((int64_t)models * p->D, p->sms), 256, 0, s, a, models, table);
  p->launches += 2;
  return adt::check_launch(p, "static measure");
}
