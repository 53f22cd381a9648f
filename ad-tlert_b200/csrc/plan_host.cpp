// Host-side plan construction (see plan_host.h). Plain C++: also compiled on its own by the
// CPU tests, which check the tables against a SciPy factorization.
#include "plan_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <numeric>
#include <string>
#include <vector>

namespace adt {
namespace {

// Cyclic Jacobi eigen-decomposition of a small symmetric matrix (row-major n x n).
void symmetric_eigen(std::vector<double> a, int n, std::vector<double>& values,
                     std::vector<double>& vectors) {
  vectors.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i) vectors[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0, norm = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        norm += a[i * n + j] * a[i * n + j];
        if (i != j) off += a[i * n + j] * a[i * n + j];
      }
    if (off <= 1e-30 * norm || norm == 0.0) break;
    for (int pi = 0; pi < n; ++pi)
      for (int qi = pi + 1; qi < n; ++qi) {
        const double apq = a[pi * n + qi];
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (a[qi * n + qi] - a[pi * n + pi]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a[k * n + pi], akq = a[k * n + qi];
          a[k * n + pi] = c * akp - s * akq;
          a[k * n + qi] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[pi * n + k], aqk = a[qi * n + k];
          a[pi * n + k] = c * apk - s * aqk;
          a[qi * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = vectors[k * n + pi], vkq = vectors[k * n + qi];
          vectors[k * n + pi] = c * vkp - s * vkq;
          vectors[k * n + qi] = s * vkp + c * vkq;
        }
      }
  }
  values.resize(n);
  for (int i = 0; i < n; ++i) values[i] = a[i * n + i];
}

// Breadth-first level sets from `roots` (unreached components continue as further levels).
std::vector<std::vector<int>> level_sets(const std::vector<int>& ptr, const std::vector<int>& adj,
                                         int n, const std::vector<int>& roots) {
  std::vector<int> level(n, -1);
  std::vector<std::vector<int>> out;
  std::vector<int> frontier;
  for (int r : roots)
    if (level[r] < 0) { level[r] = 0; frontier.push_back(r); }
  int next_unreached = 0;
  while (true) {
    if (frontier.empty()) {
      while (next_unreached < n && level[next_unreached] >= 0) ++next_unreached;
      if (next_unreached >= n) break;
      level[next_unreached] = (int)out.size();
      frontier.push_back(next_unreached);
    }
    std::sort(frontier.begin(), frontier.end());
    out.push_back(frontier);
    std::vector<int> nxt;
    for (int v : frontier)
      for (int i = ptr[v]; i < ptr[v + 1]; ++i) {
        const int u = adj[i];
        if (level[u] < 0) { level[u] = (int)out.size(); nxt.push_back(u); }
      }
    frontier.swap(nxt);
  }
  return out;
}

int pseudo_peripheral(const std::vector<int>& ptr, const std::vector<int>& adj, int n) {
  int root = 0, ecc = -1;
  for (int it = 0; it < 8; ++it) {
    auto levels = level_sets(ptr, adj, n, {root});
    if ((int)levels.size() <= ecc) break;
    ecc = (int)levels.size();
    int best = levels.back()[0];
    for (int v : levels.back())
      if (ptr[v + 1] - ptr[v] < ptr[best + 1] - ptr[best]) best = v;
    root = best;
  }
  return root;
}

int tiles_of(int64_t m) { return (int)((m + kTile - 1) / kTile); }

// Work items of the tiled solver from the task table (see HostPlan).
void build_tile_items(HostPlan& hp, const std::vector<int64_t>& task_rows) {
  const int L = hp.levels;
  std::vector<std::vector<int>> groups(3 * L);
  std::vector<std::vector<std::vector<int>>> panels(L);
  for (int l = 0; l < L; ++l) {
    int max_panels = 0;
    for (int t = hp.level_begin[l]; t < hp.level_begin[l + 1]; ++t)
      max_panels = std::max(max_panels, tiles_of(task_rows[(int64_t)t * T_FIELDS + T_MJ]));
    panels[l].assign(max_panels, {});
    for (int t = hp.level_begin[l]; t < hp.level_begin[l + 1]; ++t) {
      const int64_t* row = &task_rows[(int64_t)t * T_FIELDS];
      const int mj = (int)row[T_MJ];
      const int tj = tiles_of(mj);
      const int tp = row[T_P] >= 0 ? tiles_of(row[T_MP]) : 0;
      const int tq = row[T_Q] >= 0 ? tiles_of(row[T_MQ]) : 0;
      for (int r0 = 0; r0 < mj; r0 += kScatterRows)
        groups[l].insert(groups[l].end(), {t, r0, std::min(kScatterRows, mj - r0), 0});
      for (int qi = 0; qi < tq && tp > 0; ++qi)
        for (int pi = 0; pi < tp; ++pi) groups[L + l].insert(groups[L + l].end(), {t, qi, pi, 0});
      for (int i = 0; i < tj; ++i) groups[2 * L + l].insert(groups[2 * L + l].end(), {t, i, 0, 0});
      for (int k = 0; k < tj; ++k) {
        auto& g = panels[l][k];
        for (int i = k; i < tj; ++i) g.insert(g.end(), {t, SEG_J, i, 0});
        for (int i = 0; i < tp; ++i) g.insert(g.end(), {t, SEG_P, i, 0});
        for (int i = 0; i < tq; ++i) g.insert(g.end(), {t, SEG_Q, i, 0});
      }
    }
  }
  hp.titems.clear();
  hp.tranges.clear();
  auto add_range = [&](const std::vector<int>& items) {
    hp.tranges.push_back((int)(hp.titems.size() / 4));
    hp.titems.insert(hp.titems.end(), items.begin(), items.end());
    hp.tranges.push_back((int)(hp.titems.size() / 4));
  };
  for (auto& g : groups) add_range(g);
  hp.panel_ptr.assign(1, 0);
  for (int l = 0; l < L; ++l) {
    for (auto& g : panels[l]) add_range(g);
    hp.panel_ptr.push_back(hp.panel_ptr.back() + (int)panels[l].size());
  }
}

}  // namespace

adt_status build_host_plan(const adt_problem* pr, HostPlan& hp, std::string& err) {
  if (!pr) { err = "null argument"; return ADT_INVALID_ARG; }
  const int N = pr->dof_count, C = pr->cell_count, K = pr->local_dofs;
  const int Nb = pr->boundary_count, BL = pr->boundary_local, W = pr->wavenumber_count;
  const int E = pr->electrode_count, D = pr->measurement_count, RW = pr->receiver_width;
  if (N <= 0 || C <= 0 || K <= 0 || K > 16 || W <= 0 || E <= 0 || E > kMaxColumns || D < 0 || RW <= 0 ||
      (Nb > 0 && (BL <= 0 || BL > 16)) || pr->model_cell_count <= 0 || !pr->cell_dofs ||
      !pr->stiffness || !pr->mass || !pr->dof_coordinates || pr->dim < 1 || pr->dim > 3)
    { err = "invalid problem sizes or missing arrays"; return ADT_INVALID_ARG; }
  if (!pr->receiver_dofs || !pr->receiver_weights || !pr->abmn || !pr->source_cell_ptr ||
      !pr->weights || !pr->wavenumbers || (Nb > 0 && (!pr->boundary_dofs || !pr->boundary_cells ||
      !pr->boundary_mass || !pr->boundary_coefficients)))
    { err = "missing problem arrays"; return ADT_INVALID_ARG; }
  for (int64_t i = 0; i < (int64_t)C * K; ++i)
    if (pr->cell_dofs[i] < 0 || pr->cell_dofs[i] >= N)
      { err = "cell dofs out of range"; return ADT_INVALID_ARG; }
  for (int64_t i = 0; i < (int64_t)Nb * BL; ++i)
    if (pr->boundary_dofs[i] < 0 || pr->boundary_dofs[i] >= N)
      { err = "boundary dofs out of range"; return ADT_INVALID_ARG; }
  for (int64_t i = 0; i < (int64_t)D * 4; ++i)
    if (pr->abmn[i] < 0 || pr->abmn[i] > E)
      { err = "measurement slots out of range"; return ADT_INVALID_ARG; }
  if (pr->parent_cells)
    for (int c = 0; c < C; ++c)
      if (pr->parent_cells[c] < 0 || pr->parent_cells[c] >= pr->model_cell_count)
        { err = "parent cells out of range"; return ADT_INVALID_ARG; }
  for (int64_t i = 0; i < (int64_t)E * RW; ++i)
    if (pr->receiver_dofs[i] < -1 || pr->receiver_dofs[i] >= N)
      { err = "receiver dofs out of range"; return ADT_INVALID_ARG; }
  if (pr->source_cell_ptr[0] != 0) { err = "source_cell_ptr must start at 0"; return ADT_INVALID_ARG; }
  for (int e = 0; e < E; ++e)
    if (pr->source_cell_ptr[e + 1] < pr->source_cell_ptr[e])
      { err = "source_cell_ptr must be non-decreasing"; return ADT_INVALID_ARG; }
  for (int i = 0; i < pr->source_cell_ptr[E]; ++i)
    if (pr->source_cells[i] < 0 || pr->source_cells[i] >= pr->model_cell_count)
      { err = "source cells out of range"; return ADT_INVALID_ARG; }
  for (int b = 0; b < Nb; ++b)
    if (pr->boundary_cells[b] < 0 || pr->boundary_cells[b] >= C)
      { err = "boundary cells out of range"; return ADT_INVALID_ARG; }
  if (!pr->parent_cells && pr->model_cell_count != C)
    { err = "model_cell_count must equal cell_count without parents"; return ADT_INVALID_ARG; }
  if (pr->fixed_count < 0 || pr->fixed_count > N || (pr->fixed_count > 0 && !pr->fixed_dofs))
    { err = "invalid fixed dofs"; return ADT_INVALID_ARG; }
  std::vector<char> fixed(N, 0);
  for (int i = 0; i < pr->fixed_count; ++i) {
    if (pr->fixed_dofs[i] < 0 || pr->fixed_dofs[i] >= N)
      { err = "fixed dofs out of range"; return ADT_INVALID_ARG; }
    fixed[pr->fixed_dofs[i]] = 1;
  }

  hp.N = N; hp.dim = pr->dim; hp.C = C; hp.K = K; hp.Cm = pr->model_cell_count;
  hp.Nb = Nb; hp.BL = BL; hp.W = W; hp.E = E; hp.D = D; hp.RW = RW;

  // ---- sparse pattern in original numbering: unique (row, col) of all local pairs ----
  std::vector<int64_t> keys;
  keys.reserve((size_t)C * K * K + (size_t)Nb * BL * BL);
  for (int c = 0; c < C; ++c)
    for (int i = 0; i < K; ++i)
      for (int j = 0; j < K; ++j)
        keys.push_back((int64_t)pr->cell_dofs[c * K + i] * N + pr->cell_dofs[c * K + j]);
  for (int b = 0; b < Nb; ++b)
    for (int i = 0; i < BL; ++i)
      for (int j = 0; j < BL; ++j)
        keys.push_back((int64_t)pr->boundary_dofs[b * BL + i] * N + pr->boundary_dofs[b * BL + j]);
  std::vector<int64_t> uniq(keys);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  std::vector<int> aptr(N + 1, 0), adj;
  for (int64_t k : uniq)
    if (k / N != k % N) aptr[k / N + 1]++;
  for (int i = 0; i < N; ++i) aptr[i + 1] += aptr[i];
  adj.resize(aptr[N]);
  {
    std::vector<int> fill(aptr.begin(), aptr.end() - 1);
    for (int64_t k : uniq)
      if (k / N != k % N) adj[fill[k / N]++] = (int)(k % N);
  }

  // ---- elimination order: breadth-first level sets from the best root set ----
  std::vector<std::vector<int>> roots;
  roots.push_back({pseudo_peripheral(aptr, adj, N)});
  for (int axis = 0; axis < pr->dim; ++axis) {
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < N; ++i) {
      lo = std::min(lo, pr->dof_coordinates[i * pr->dim + axis]);
      hi = std::max(hi, pr->dof_coordinates[i * pr->dim + axis]);
    }
    const double tol = 1e-6 * std::max(hi - lo, 1e-300);
    for (int side = 0; side < 2; ++side) {
      std::vector<int> set;
      for (int i = 0; i < N; ++i) {
        const double x = pr->dof_coordinates[i * pr->dim + axis];
        if (std::fabs(x - (side ? hi : lo)) <= tol) set.push_back(i);
      }
      if (!set.empty()) roots.push_back(set);
    }
  }
  std::vector<std::vector<int>> best;
  double best_cost = 1e300;
  int best_width = 0;
  for (auto& r : roots) {
    auto lv = level_sets(aptr, adj, N, r);
    int width = 0;
    double cost = 0.0;
    for (auto& l : lv) {
      width = std::max(width, (int)l.size());
      cost += std::pow((double)l.size(), 3.0);
    }
    const bool ok = width <= kMaxBlock;
    const bool best_ok = best_width > 0 && best_width <= kMaxBlock;
    if (best.empty() || (ok && !best_ok) || (ok == best_ok && cost < best_cost)) {
      best = lv;
      best_cost = cost;
      best_width = width;
    }
  }
  if (best_width > kMaxTiledBlock) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "the narrowest level-set ordering has %d dofs per level; the solver accepts at most %d",
                  best_width, kMaxTiledBlock);
    err = msg;
    return ADT_INVALID_ARG;
  }
  hp.tiled = best_width > kMaxBlock;
  hp.nb = (int)best.size();
  hp.max_m = best_width;
  std::vector<int> bm(hp.nb), boff(hp.nb + 1, 0);
  hp.perm.clear();
  for (int b = 0; b < hp.nb; ++b) {
    bm[b] = (int)best[b].size();
    boff[b + 1] = boff[b] + bm[b];
    for (int v : best[b]) hp.perm.push_back(v);
  }
  hp.iperm.assign(N, 0);
  for (int i = 0; i < N; ++i) hp.iperm[hp.perm[i]] = i;

  // ---- CSR in solver order and the assembly routing ----
  std::vector<int64_t> pkeys(uniq.size());
  for (size_t i = 0; i < uniq.size(); ++i)
    pkeys[i] = (int64_t)hp.iperm[uniq[i] / N] * N + hp.iperm[uniq[i] % N];
  std::sort(pkeys.begin(), pkeys.end());
  hp.nnz = (int)pkeys.size();
  std::vector<int> csr_ptr(N + 1, 0), csr_col(hp.nnz), csr_row(hp.nnz);
  for (int s = 0; s < hp.nnz; ++s) {
    csr_row[s] = (int)(pkeys[s] / N);
    csr_col[s] = (int)(pkeys[s] % N);
    csr_ptr[csr_row[s] + 1]++;
  }
  for (int i = 0; i < N; ++i) csr_ptr[i + 1] += csr_ptr[i];
  auto slot_of = [&](int r, int c) -> int {
    const int64_t key = (int64_t)hp.iperm[r] * N + hp.iperm[c];
    return (int)(std::lower_bound(pkeys.begin(), pkeys.end(), key) - pkeys.begin());
  };
  std::vector<int> ccount(hp.nnz + 1, 0);
  std::vector<std::pair<int, int>> routed;  // (slot, code)
  routed.reserve(keys.size());
  // pairs touching a fixed dof are not routed (they stay explicit zeros of the pattern, so the
  // elimination order does not depend on the boundary mode); a fixed diagonal gets the unit code
  for (int c = 0; c < C; ++c)
    for (int i = 0; i < K; ++i)
      for (int j = 0; j < K; ++j) {
        const int r = pr->cell_dofs[c * K + i], q = pr->cell_dofs[c * K + j];
        if (!fixed[r] && !fixed[q]) routed.push_back({slot_of(r, q), c * K * K + i * K + j});
      }
  for (int b = 0; b < Nb; ++b)
    for (int i = 0; i < BL; ++i)
      for (int j = 0; j < BL; ++j) {
        const int r = pr->boundary_dofs[b * BL + i], q = pr->boundary_dofs[b * BL + j];
        if (!fixed[r] && !fixed[q]) routed.push_back({slot_of(r, q), C * K * K + b * BL * BL + i * BL + j});
      }
  for (int n = 0; n < N; ++n)
    if (fixed[n]) routed.push_back({slot_of(n, n), kUnitCode});
  std::stable_sort(routed.begin(), routed.end());
  std::vector<int> contrib_ptr(hp.nnz + 1, 0), contrib(routed.size());
  for (size_t i = 0; i < routed.size(); ++i) {
    contrib_ptr[routed[i].first + 1]++;
    contrib[i] = routed[i].second;
  }
  for (int s = 0; s < hp.nnz; ++s) contrib_ptr[s + 1] += contrib_ptr[s];
  hp.contributions = (int64_t)routed.size();

  // ---- block cyclic reduction schedule ----
  std::vector<int64_t> loff(hp.nb);
  int64_t cursor = 0;
  for (int b = 0; b < hp.nb; ++b) { loff[b] = cursor; cursor += (int64_t)bm[b] * bm[b]; }
  struct Elim { int j, p, q; int64_t u, v, ru = -1, rv = -1; };
  std::vector<Elim> elims;
  std::vector<int64_t> task_rows;
  std::vector<int> elim_level;
  std::map<std::pair<int, int>, int64_t> link;  // (left, right) -> fill offset, -1 = CSR
  std::vector<int> chain(hp.nb);
  std::iota(chain.begin(), chain.end(), 0);
  for (int b = 0; b + 1 < hp.nb; ++b) link[{b, b + 1}] = -1;
  std::vector<int> level_of_task;
  std::vector<Elim> task_elim;  // per task
  hp.level_begin.assign(1, 0);
  int level = 0;
  while (chain.size() > 1) {
    std::vector<int> next;
    for (size_t pos = 0; pos < chain.size(); ++pos) {
      if (pos % 2 == 0) { next.push_back(chain[pos]); continue; }
      Elim e;
      e.j = chain[pos];
      e.p = chain[pos - 1];
      e.q = pos + 1 < chain.size() ? chain[pos + 1] : -1;
      e.u = cursor; cursor += (int64_t)bm[e.j] * bm[e.p];
      e.v = -1;
      if (e.q >= 0) { e.v = cursor; cursor += (int64_t)bm[e.q] * bm[e.j]; }
      if (!hp.tiled) {  // the inverse-based kernels keep the couplings for the Schur updates
        e.ru = cursor; cursor += (int64_t)bm[e.j] * bm[e.p];
        if (e.q >= 0) { e.rv = cursor; cursor += (int64_t)bm[e.q] * bm[e.j]; }
      }
      task_elim.push_back(e);
      level_of_task.push_back(level);
    }
    // fills of this level become the links of the next
    std::map<std::pair<int, int>, int64_t> next_link;
    std::vector<int64_t> fills;
    for (size_t t = hp.level_begin.back(); t < task_elim.size(); ++t) {
      const Elim& e = task_elim[t];
      if (e.q >= 0) {
        next_link[{e.p, e.q}] = cursor;
        fills.push_back(cursor);
        cursor += (int64_t)bm[e.q] * bm[e.p];
      } else {
        fills.push_back(-1);
      }
    }
    for (size_t t = hp.level_begin.back(), k = 0; t < task_elim.size(); ++t, ++k) {
      const Elim& e = task_elim[t];
      std::vector<int64_t> row(T_FIELDS, -1);
      row[T_J] = e.j; row[T_MJ] = bm[e.j]; row[T_OFFJ] = boff[e.j]; row[T_LOFF] = loff[e.j];
      row[T_P] = e.p; row[T_MP] = bm[e.p]; row[T_OFFP] = boff[e.p]; row[T_UOFF] = e.u;
      row[T_LINKP] = link.at({e.p, e.j});
      if (e.q >= 0) {
        row[T_Q] = e.q; row[T_MQ] = bm[e.q]; row[T_OFFQ] = boff[e.q]; row[T_VOFF] = e.v;
        row[T_LINKQ] = link.at({e.j, e.q});
      } else {
        row[T_Q] = -1; row[T_MQ] = 0; row[T_OFFQ] = 0;
      }
      row[T_FILL] = fills[k];
      row[T_RUOFF] = e.ru;
      row[T_RVOFF] = e.rv;
      task_rows.insert(task_rows.end(), row.begin(), row.end());
    }
    link = next_link;
    chain = next;
    hp.level_begin.push_back((int)task_elim.size());
    ++level;
  }
  {  // root
    Elim e{chain[0], -1, -1, -1, -1};
    task_elim.push_back(e);
    level_of_task.push_back(level);
    std::vector<int64_t> row(T_FIELDS, -1);
    row[T_J] = e.j; row[T_MJ] = bm[e.j]; row[T_OFFJ] = boff[e.j]; row[T_LOFF] = loff[e.j];
    row[T_MP] = 0; row[T_OFFP] = 0; row[T_MQ] = 0; row[T_OFFQ] = 0;
    task_rows.insert(task_rows.end(), row.begin(), row.end());
    hp.level_begin.push_back((int)task_elim.size());
    ++level;
  }
  hp.levels = level;
  hp.factor_stride = cursor;
  // pulls: for task j, every earlier elimination next to j (left one first, per level)
  std::vector<int64_t> pulls;
  std::vector<int> pull_level;
  std::vector<std::vector<int>> by_block_q(hp.nb), by_block_p(hp.nb);
  for (size_t t = 0; t + 1 < task_elim.size(); ++t) {
    if (task_elim[t].q >= 0) by_block_q[task_elim[t].q].push_back((int)t);
    by_block_p[task_elim[t].p].push_back((int)t);
  }
  for (size_t t = 0; t < task_elim.size(); ++t) {
    const int j = task_elim[t].j;
    std::vector<std::pair<int, int>> list;  // (task index, type)
    for (int e : by_block_q[j]) list.push_back({e, 1});
    for (int e : by_block_p[j]) list.push_back({e, 0});
    std::sort(list.begin(), list.end(), [&](auto a, auto b) {
      if (level_of_task[a.first] != level_of_task[b.first])
        return level_of_task[a.first] < level_of_task[b.first];
      return a.second > b.second;  // left neighbour (V type) first
    });
    task_rows[t * T_FIELDS + T_PULL0] = (int64_t)pulls.size() / P_FIELDS;
    for (auto& [e, type] : list) {
      const Elim& el = task_elim[e];
      pulls.push_back(type);
      pulls.push_back(type == 0 ? el.u : el.v);
      pulls.push_back(bm[el.j]);
      pulls.push_back(boff[el.j]);
      pulls.push_back(type == 0 ? el.ru : el.rv);
      pull_level.push_back(level_of_task[e]);
    }
    task_rows[t * T_FIELDS + T_PULL1] = (int64_t)pulls.size() / P_FIELDS;
  }
  // eager updates: after level l, every block next to an elimination of level l applies the
  // pulls of that level (a contiguous run of its pull list, which is sorted by level)
  hp.update_begin.assign(1, 0);
  hp.update_items.clear();
  for (int l = 0; l < hp.levels; ++l) {
    for (size_t t = 0; t < task_elim.size(); ++t) {
      const int64_t u0 = task_rows[t * T_FIELDS + T_PULL0], u1 = task_rows[t * T_FIELDS + T_PULL1];
      int64_t b = u0;
      while (b < u1 && pull_level[b] < l) ++b;
      int64_t e = b;
      while (e < u1 && pull_level[e] == l) ++e;
      if (e > b) hp.update_items.insert(hp.update_items.end(), {(int)t, (int)b, (int)e});
    }
    hp.update_begin.push_back((int)(hp.update_items.size() / 3));
  }

  if (hp.tiled) build_tile_items(hp, task_rows);

  // ---- per-cell template factors (features of the sensitivity Gram) ----
  std::vector<std::vector<double>> svals(C), svecs(C), mvals(C), mvecs(C);
  int rs = K - 1;
  for (int c = 0; c < C; ++c) {
    std::vector<double> s(pr->stiffness + (size_t)c * K * K, pr->stiffness + (size_t)(c + 1) * K * K);
    std::vector<double> m(pr->mass + (size_t)c * K * K, pr->mass + (size_t)(c + 1) * K * K);
    symmetric_eigen(s, K, svals[c], svecs[c]);
    symmetric_eigen(m, K, mvals[c], mvecs[c]);
    double lo = 1e300, hi = 0.0;
    for (double v : svals[c]) { lo = std::min(lo, v); hi = std::max(hi, std::fabs(v)); }
    if (lo > 1e-9 * hi) rs = K;
  }
  // mass features only when some wavenumber is non-zero (a 3D operator has none)
  bool any_mass = false;
  for (int w = 0; w < W; ++w) any_mass = any_mass || pr->wavenumbers[w] != 0.0;
  hp.RS = rs;
  hp.R = rs + (any_mass ? K : 0);
  std::vector<float> features((size_t)C * hp.R * K);
  for (int c = 0; c < C; ++c) {
    std::vector<int> order(K);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return svals[c][a] > svals[c][b]; });
    for (int f = 0; f < hp.R; ++f) {
      const bool stiff = f < rs;
      const int col = stiff ? order[f] : f - rs;
      const double lam = std::max(stiff ? svals[c][col] : mvals[c][col], 0.0);
      const std::vector<double>& vec = stiff ? svecs[c] : mvecs[c];
      for (int k = 0; k < K; ++k)
        features[((size_t)c * hp.R + f) * K + k] = (float)(std::sqrt(lam) * vec[k * K + col]);
    }
  }
  std::vector<float> fscale((size_t)W * hp.R);
  for (int w = 0; w < W; ++w)
    for (int f = 0; f < hp.R; ++f)
      fscale[w * hp.R + f] = (float)(std::sqrt(pr->weights[w]) * (f < rs ? 1.0 : std::fabs(pr->wavenumbers[w])));

  // ---- measurement routing ----
  std::vector<std::vector<int>> pair_entries((size_t)(E + 1) * (E + 1));
  for (int d = 0; d < D; ++d) {
    const int a = pr->abmn[4 * d], b = pr->abmn[4 * d + 1], m = pr->abmn[4 * d + 2], n = pr->abmn[4 * d + 3];
    const int normal[4][3] = {{a, m, 0}, {a, n, 1}, {b, m, 1}, {b, n, 0}};
    const int recip[4][3] = {{m, a, 2}, {m, b, 3}, {n, a, 3}, {n, b, 2}};
    for (auto& e : normal) pair_entries[e[0] * (E + 1) + e[1]].push_back(d * 4 + e[2]);
    for (auto& e : recip) pair_entries[e[0] * (E + 1) + e[1]].push_back(d * 4 + e[2]);
  }
  std::vector<int> pair_ptr(1, 0), pair_list;
  for (auto& v : pair_entries) {
    std::sort(v.begin(), v.end());
    pair_list.insert(pair_list.end(), v.begin(), v.end());
    pair_ptr.push_back((int)pair_list.size());
  }
  std::vector<int> rcv_dofs((size_t)E * RW);
  std::vector<double> rcv_w((size_t)E * RW);
  std::map<int, std::vector<std::pair<int, double>>> by_dof;
  for (int r = 0; r < E; ++r)
    for (int k = 0; k < RW; ++k) {
      const int dof = pr->receiver_dofs[r * RW + k];
      rcv_dofs[r * RW + k] = dof < 0 ? -1 : hp.iperm[dof];
      rcv_w[r * RW + k] = pr->receiver_weights[r * RW + k];
      if (dof >= 0 && pr->receiver_weights[r * RW + k] != 0.0)
        by_dof[hp.iperm[dof]].push_back({r, pr->receiver_weights[r * RW + k]});
    }
  std::vector<int> rdof_ptr(1, 0), rdof_rcv, rdof_dof;
  std::vector<double> rdof_w;
  for (auto& [dof, list] : by_dof) {
    rdof_dof.push_back(dof);
    for (auto& [r, wv] : list) { rdof_rcv.push_back(r); rdof_w.push_back(wv); }
    rdof_ptr.push_back((int)rdof_rcv.size());
  }
  hp.rdofs = (int)rdof_dof.size();

  // ---- cells in solver order, boundary lists, model-cell lists ----
  std::vector<int> cdofs((size_t)C * K), bd((size_t)Nb * BL);
  for (int64_t i = 0; i < (int64_t)C * K; ++i) cdofs[i] = hp.iperm[pr->cell_dofs[i]];
  for (int64_t i = 0; i < (int64_t)Nb * BL; ++i) bd[i] = hp.iperm[pr->boundary_dofs[i]];
  std::vector<int> cell_bptr(C + 1, 0), cell_blist(Nb);
  for (int b = 0; b < Nb; ++b) cell_bptr[pr->boundary_cells[b] + 1]++;
  for (int c = 0; c < C; ++c) cell_bptr[c + 1] += cell_bptr[c];
  {
    std::vector<int> fill(cell_bptr.begin(), cell_bptr.end() - 1);
    for (int b = 0; b < Nb; ++b) cell_blist[fill[pr->boundary_cells[b]]++] = b;
  }
  std::vector<int> model_ptr(hp.Cm + 1, 0), model_list(C);
  for (int c = 0; c < C; ++c) model_ptr[(pr->parent_cells ? pr->parent_cells[c] : c) + 1]++;
  for (int m = 0; m < hp.Cm; ++m) model_ptr[m + 1] += model_ptr[m];
  {
    std::vector<int> fill(model_ptr.begin(), model_ptr.end() - 1);
    for (int c = 0; c < C; ++c) model_list[fill[pr->parent_cells ? pr->parent_cells[c] : c]++] = c;
  }
  std::vector<double> k2(W);
  for (int w = 0; w < W; ++w) k2[w] = pr->wavenumbers[w] * pr->wavenumbers[w];
  std::vector<int> bowners, fixed_solver;
  for (int c = 0; c < C; ++c)
    if (cell_bptr[c + 1] > cell_bptr[c]) bowners.push_back(c);
  for (int n = 0; n < N; ++n)
    if (fixed[hp.perm[n]]) fixed_solver.push_back(n);

  hp.csr_ptr = std::move(csr_ptr);
  hp.csr_col = std::move(csr_col);
  hp.csr_row = std::move(csr_row);
  hp.contrib_ptr = std::move(contrib_ptr);
  hp.contrib = std::move(contrib);
  hp.task_rows = std::move(task_rows);
  hp.pulls = std::move(pulls);
  hp.features = std::move(features);
  hp.fscale = std::move(fscale);
  hp.pair_ptr = std::move(pair_ptr);
  hp.pair_list = std::move(pair_list);
  hp.rcv_dofs = std::move(rcv_dofs);
  hp.rcv_w = std::move(rcv_w);
  hp.rdof_ptr = std::move(rdof_ptr);
  hp.rdof_rcv = std::move(rdof_rcv);
  hp.rdof_w = std::move(rdof_w);
  hp.rdof_dof = std::move(rdof_dof);
  hp.cdofs = std::move(cdofs);
  hp.bd = std::move(bd);
  hp.cell_bptr = std::move(cell_bptr);
  hp.cell_blist = std::move(cell_blist);
  hp.model_ptr = std::move(model_ptr);
  hp.model_list = std::move(model_list);
  hp.k2 = std::move(k2);
  hp.bowners = std::move(bowners);
  hp.fixed = std::move(fixed_solver);
  return ADT_OK;
}

}  // namespace adt
