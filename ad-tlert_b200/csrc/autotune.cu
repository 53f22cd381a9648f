// Autotuner of a plan's launch shapes: the substitution strip rule, the tiled solver's split
// rule and the Jacobian kernel, each chosen by timing the real entry points on the caller's
// data (CUDA events on the caller's stream). Host code only: it calls the same entry points a
// user calls, with the plan's settings switched between candidates.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "adt_internal.h"
#include "kernels.h"

using namespace adt;

namespace {

struct JacobianFlags {
  bool direct, tc, pipe;
};

JacobianFlags flags_for(int kernel) {
  switch (kernel) {
    case ADT_JACOBIAN_DIRECT: return {true, true, true};
    case ADT_JACOBIAN_TC_PIPELINED: return {false, true, true};
    case ADT_JACOBIAN_TC: return {false, true, false};
    default: return {false, false, false};
  }
}

bool applies(const adt_plan* p, int kernel);

// The kernel adt_normal_jacobian launches for all rows under the plan's current flags.
int kernel_of(const adt_plan* p) {
  if (p->jacobian_direct && applies(p, ADT_JACOBIAN_DIRECT)) return ADT_JACOBIAN_DIRECT;
  if (p->jacobian_tc && p->jacobian_pipe && applies(p, ADT_JACOBIAN_TC_PIPELINED)) return ADT_JACOBIAN_TC_PIPELINED;
  if (p->jacobian_tc && applies(p, ADT_JACOBIAN_TC)) return ADT_JACOBIAN_TC;
  return ADT_JACOBIAN_FMA;
}

void apply(adt_plan* p, int kernel) {
  const JacobianFlags f = flags_for(kernel);
  p->jacobian_direct = f.direct;
  p->jacobian_tc = f.tc;
  p->jacobian_pipe = f.pipe;
}

// Whether `kernel` is the one adt_normal_jacobian launches for all rows (not a fall-through).
bool applies(const adt_plan* p, int kernel) {
  switch (kernel) {
    case ADT_JACOBIAN_DIRECT:
      return p->W == 1 && p->row_entries && jacobian_direct_cells(p->R, p->E, p->K) > 0;
    case ADT_JACOBIAN_TC_PIPELINED:
      return jacobian_tc_supported(p->E, p->W, p->R, p->K, p->D) &&
             jacobian_tcpipe_batch(p->E, p->W, p->R, p->K, p->D) > 0;
    case ADT_JACOBIAN_TC: return jacobian_tc_supported(p->E, p->W, p->R, p->K, p->D);
    default: return true;
  }
}

// Fastest of `repeats` timed runs of `run` after one untimed run; FLT_MAX if any run fails.
template <typename F>
float fastest(adt_plan* p, cudaStream_t s, int repeats, cudaEvent_t start, cudaEvent_t stop, F&& run,
              adt_status& status) {
  status = run();
  if (status != ADT_OK) return FLT_MAX;
  float best = FLT_MAX;
  for (int r = 0; r < repeats; ++r) {
    cudaEventRecord(start, s);
    status = run();
    cudaEventRecord(stop, s);
    if (status != ADT_OK) return FLT_MAX;
    if (cudaEventSynchronize(stop) != cudaSuccess) {
      status = fail(p, ADT_CUDA_ERROR, "autotune: a timed run failed");
      return FLT_MAX;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, start, stop);
    best = std::min(best, ms);
  }
  return best;
}

}  // namespace

extern "C" {

adt_status adt_get_tuning(const adt_plan* p, adt_tuning* out) {
  if (!p || !out) return ADT_INVALID_ARG;
  out->strip_fill = p->strip_fill;
  out->split_fill = p->split_fill;
  out->jacobian_kernel = kernel_of(p);
  out->fields_ms = 0.0f;
  out->jacobian_ms = 0.0f;
  return ADT_OK;
}

adt_status adt_set_tuning(adt_plan* p, const adt_tuning* t) {
  if (!p || !t) return fail(p, ADT_INVALID_ARG, "null tuning");
  const int strip = t->strip_fill;
  if ((strip != 1 && strip != 2 && strip != 4 && strip != 8) || t->split_fill < 0 || t->split_fill > 2 ||
      t->jacobian_kernel < ADT_JACOBIAN_DIRECT || t->jacobian_kernel > ADT_JACOBIAN_FMA)
    return fail(p, ADT_INVALID_ARG, "tuning out of range (strip_fill 1, 2, 4 or 8; split_fill 0..2; kernel 0..3)");
  p->strip_fill = strip;
  p->split_fill = t->split_fill;
  apply(p, t->jacobian_kernel);
  return ADT_OK;
}

adt_status adt_autotune(adt_plan* p, int32_t slot, const float* sigma, int32_t models, float* fields,
                        float* jacobian, int32_t repeats, adt_tuning* out, adt_stream stream) {
  if (!p || !sigma || !fields || models <= 0 || slot < 0 || repeats < 1 || repeats > 32)
    return fail(p, ADT_INVALID_ARG, "invalid autotune arguments");
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t start, stop;
  if (cudaEventCreate(&start) != cudaSuccess) return fail(p, ADT_CUDA_ERROR, "autotune: event creation failed");
  if (cudaEventCreate(&stop) != cudaSuccess) {
    cudaEventDestroy(start);
    return fail(p, ADT_CUDA_ERROR, "autotune: event creation failed");
  }
  adt_status status = ADT_OK;
  auto fields_run = [&]() -> adt_status {
    if (adt_status st = adt_factorize_fields(p, slot, sigma, models, stream)) return st;
    return adt_solve_fields(p, slot, sigma, models, fields, stream);
  };
  // 1. solver launch shapes
  const int strips[] = {1, 2, 4, 8};
  std::vector<int> splits = {p->split_fill};
  if (p->tiled) splits = {0, 1, 2};
  float best_fields = FLT_MAX;
  int best_strip = p->strip_fill, best_split = p->split_fill;
  for (int split : splits) {
    for (int strip : strips) {
      p->strip_fill = strip;
      p->split_fill = split;
      const float ms = fastest(p, s, repeats, start, stop, fields_run, status);
      if (status != ADT_OK) break;
      if (ms < best_fields) {
        best_fields = ms;
        best_strip = strip;
        best_split = split;
      }
    }
    if (status != ADT_OK) break;
  }
  p->strip_fill = best_strip;
  p->split_fill = best_split;
  if (status == ADT_OK) status = fields_run();  // the fields of the chosen shapes
  // 2. Jacobian kernel
  const int kernel_before = kernel_of(p);
  int best_kernel = kernel_before;
  float best_jacobian = 0.0f;
  if (status == ADT_OK && jacobian) {
    best_jacobian = FLT_MAX;
    for (int kernel = ADT_JACOBIAN_DIRECT; kernel <= ADT_JACOBIAN_FMA; ++kernel) {
      if (!applies(p, kernel)) continue;
      apply(p, kernel);
      adt_status st = ADT_OK;
      const float ms = fastest(p, s, repeats, start, stop,
                               [&]() { return adt_normal_jacobian(p, fields, 0, p->D, jacobian, stream); }, st);
      if (st == ADT_TIMEOUT || st == ADT_CUDA_ERROR) {
        status = st;
        break;
      }
      if (st == ADT_OK && ms < best_jacobian) {  // a kernel refusing these shapes is skipped
        best_jacobian = ms;
        best_kernel = kernel;
      }
    }
    apply(p, best_kernel);
    if (status == ADT_OK) status = adt_normal_jacobian(p, fields, 0, p->D, jacobian, stream);
  }
  if (status == ADT_OK && cudaStreamSynchronize(s) != cudaSuccess)
    status = fail(p, ADT_CUDA_ERROR, "autotune: synchronization failed");
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (status != ADT_OK) return status;
  p->error.clear();
  if (out) {
    out->strip_fill = p->strip_fill;
    out->split_fill = p->split_fill;
    out->jacobian_kernel = kernel_of(p);
    out->fields_ms = best_fields;
    out->jacobian_ms = best_jacobian;
  }
  return ADT_OK;
}

}  // extern "C"
