// CPU-only test shim: runs the plan builder of adtlert_b200 (ad-tlert_b200/csrc/plan_host.cpp)
// without CUDA and exposes its tables, so the tests can check the elimination schedule,
// routings and template factors against SciPy before any GPU run.
#include <cstring>
#include <string>

#include "plan_host.h"

namespace {
struct Shim {
  adt::HostPlan hp;
  std::string err;
};

template <typename T>
bool copy_out(const std::vector<T>& v, void* dst, long long* size) {
  *size = (long long)v.size();
  if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(T));
  return true;
}
}  // namespace

extern "C" {

void* shim_build(const adt_problem* pr, int* status) {
  Shim* s = new Shim();
  *status = adt::build_host_plan(pr, s->hp, s->err);
  return s;
}

const char* shim_error(void* h) { return ((Shim*)h)->err.c_str(); }

void shim_free(void* h) { delete (Shim*)h; }

long long shim_scalar(void* h, const char* name) {
  const adt::HostPlan& p = ((Shim*)h)->hp;
  const std::string n(name);
  if (n == "N") return p.N;
  if (n == "nnz") return p.nnz;
  if (n == "nb") return p.nb;
  if (n == "max_m") return p.max_m;
  if (n == "levels") return p.levels;
  if (n == "RS") return p.RS;
  if (n == "R") return p.R;
  if (n == "rdofs") return p.rdofs;
  if (n == "factor_stride") return p.factor_stride;
  if (n == "contributions") return p.contributions;
  if (n == "tiled") return p.tiled ? 1 : 0;
  return -1;
}

// Copies the named table into dst (if not null) and returns its length; element types:
// int32 for index tables, int64 for task_rows/pulls, float32 for features/fscale, float64
// for rcv_w/rdof_w/k2.
long long shim_table(void* h, const char* name, void* dst) {
  const adt::HostPlan& p = ((Shim*)h)->hp;
  const std::string n(name);
  long long size = -1;
#define T(field) if (n == #field) { copy_out(p.field, dst, &size); return size; }
  T(perm) T(iperm) T(level_begin) T(csr_ptr) T(csr_col) T(csr_row) T(contrib_ptr) T(contrib)
  T(task_rows) T(pulls) T(features) T(fscale) T(pair_ptr) T(pair_list) T(rcv_dofs) T(rcv_w)
  T(rdof_ptr) T(rdof_rcv) T(rdof_dof) T(rdof_w) T(cdofs) T(bd) T(cell_bptr) T(cell_blist)
  T(model_ptr) T(model_list) T(k2) T(bowners) T(fixed) T(titems) T(tranges) T(panel_ptr) T(update_items) T(update_begin)
#undef T
  return size;
}
}
