// CUDA graph of one fresh-model Jacobian: the whole launch chain of adt_factorize_fields,
// adt_solve_fields, adt_measure and adt_normal_jacobian (about 35 dependent kernels with their
// programmatic launch edges) captured once and replayed with one cudaGraphLaunch per model.
// The graph reads the model from, and writes fields, transfers and J to, the buffers given at
// capture; the caller refreshes the model buffer before each launch. It also holds the addresses
// of the plan's workspaces at capture (the slot's values, factors and right-hand sides, the
// potential table, the scratch and tiled-solver buffers): a launch after any of them was
// reallocated (a later call on the same slot with more models, for example) is refused.
#include <array>

#include "adt_internal.h"

using namespace adt;

namespace {

using Workspaces = std::array<const void*, 8>;

Workspaces workspaces(const adt_plan* p, int slot) {
  const Slot& s = p->slots[slot];
  return {s.values, s.factors, s.rhs, s.rho, p->pot, p->scratch, p->inverses, p->partials};
}

}  // namespace

struct adt_graph {
  adt_plan* plan = nullptr;
  int slot = 0;
  Workspaces buffers{};
  cudaStream_t capture = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;  // library kernels per replay
};

namespace {

adt_status chain(adt_plan* p, int32_t slot, const float* sigma, float* fields, double* normal, double* reciprocal,
                 float* jacobian, cudaStream_t s) {
  if (adt_status st = adt_factorize_fields(p, slot, sigma, 1, s)) return st;
  if (adt_status st = adt_solve_fields(p, slot, sigma, 1, fields, s)) return st;
  if (adt_status st = adt_measure(p, fields, 1, normal, reciprocal, nullptr, s)) return st;
  if (jacobian) return adt_normal_jacobian(p, fields, 0, p->D, jacobian, s);
  return ADT_OK;
}

void release(adt_graph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->capture) cudaStreamDestroy(g->capture);
  delete g;
}

}  // namespace

extern "C" {

adt_status adt_jacobian_graph_create(adt_plan* p, int32_t slot, const float* sigma, float* fields, double* normal,
                                     double* reciprocal, float* jacobian, adt_stream stream, adt_graph** out) {
  if (!p || !sigma || !fields || !normal || !reciprocal || !out || slot < 0)
    return fail(p, ADT_INVALID_ARG, "invalid graph arguments");
  *out = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  // one uncaptured run: workspaces the chain grows on first use are allocated outside the capture
  if (adt_status st = chain(p, slot, sigma, fields, normal, reciprocal, jacobian, s)) return st;
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(p, ADT_CUDA_ERROR, "graph: warm-up run failed");
  adt_graph* g = new adt_graph();
  g->plan = p;
  if (cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking) != cudaSuccess) {
    release(g);
    return fail(p, ADT_CUDA_ERROR, "graph: could not create the capture stream");
  }
  if (cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    release(g);
    return fail(p, ADT_CUDA_ERROR, "graph: could not begin the capture");
  }
  const int64_t before = p->launches;
  const adt_status st = chain(p, slot, sigma, fields, normal, reciprocal, jacobian, g->capture);
  const cudaError_t end = cudaStreamEndCapture(g->capture, &g->graph);
  g->kernels = p->launches - before;
  p->launches = before;
  if (st != ADT_OK || end != cudaSuccess) {
    release(g);
    if (st != ADT_OK) return st;
    return fail(p, ADT_CUDA_ERROR, std::string("graph: capture failed: ") + cudaGetErrorString(end));
  }
  const cudaError_t made = cudaGraphInstantiateWithFlags(&g->exec, g->graph, 0);
  if (made != cudaSuccess) {
    release(g);
    return fail(p, ADT_CUDA_ERROR, std::string("graph: instantiation failed: ") + cudaGetErrorString(made));
  }
  g->slot = slot;
  g->buffers = workspaces(p, slot);
  *out = g;
  return ADT_OK;
}

adt_status adt_graph_launch(adt_graph* g, adt_stream stream) {
  if (!g) return ADT_INVALID_ARG;
  adt_plan* p = g->plan;
  if (workspaces(p, g->slot) != g->buffers)
    return fail(p, ADT_INVALID_ARG, "graph: the plan's workspaces were reallocated since the capture; create it again");
  if (p->tc_error_host && *p->tc_error_host != 0)
    return fail(p, ADT_TIMEOUT, "a tensor-core Jacobian launch of this plan timed out waiting for its MMAs");
  const cudaError_t err = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  if (err != cudaSuccess) return fail(p, ADT_CUDA_ERROR, std::string("graph launch: ") + cudaGetErrorString(err));
  p->launches += g->kernels;
  return ADT_OK;
}

int64_t adt_graph_kernels(const adt_graph* g) { return g ? g->kernels : 0; }

adt_status adt_graph_destroy(adt_graph* g) {
  if (g) release(g);
  return ADT_OK;
}

}  // extern "C"
