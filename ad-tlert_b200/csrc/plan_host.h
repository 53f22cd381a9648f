// Host-side plan construction of adtlert_b200 (no CUDA): sparse pattern, level-set elimination
// order, assembly routing, block cyclic reduction schedule, per-cell template factors and the
// measurement routings. The device plan uploads these arrays unchanged.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "adtlert_b200.h"

namespace adt {

constexpr int kMaxBlock = 64;  // largest block of the shared-memory solver kernels
constexpr int kMaxTiledBlock = 4096;  // largest block of the tiled (global-memory) solver
// Most field columns (electrodes in 2.5D; current + receiver columns in 3D): the FP32 Gram kernel
// holds one cell's packed E x E Gram as at most 1280 4 x 4 tiles of a 256-thread block.
constexpr int kMaxColumns = 200;
constexpr int kTile = 64;       // tile edge of the tiled solver
constexpr int kScatterRows = 32;  // block rows per scatter item of the tiled solver
constexpr int kUnitCode = -1;  // assembly contribution of constant 1 (a fixed dof's diagonal)

// Fields of one elimination task (one row of the int64 task table).
enum TaskField : int {
  T_J = 0, T_MJ, T_OFFJ, T_LOFF,
  T_P, T_MP, T_OFFP, T_UOFF, T_LINKP,
  T_Q, T_MQ, T_OFFQ, T_VOFF, T_LINKQ,
  T_FILL, T_PULL0, T_PULL1,
  T_RUOFF, T_RVOFF,  // shared-memory solver: copies of the couplings A[j,p] and A[q,j]
  T_FIELDS
};
// Row segments of a tiled elimination: the eliminated block j and its chain neighbours p, q.
enum TileSegment : int { SEG_J = 0, SEG_P = 1, SEG_Q = 2 };

// Fields of one pull (a Schur-complement contribution of an earlier elimination).
enum PullField : int { P_TYPE = 0, P_OFF, P_ME, P_EOFF, P_AOFF, P_FIELDS };

struct HostPlan {
  int N = 0, dim = 2, C = 0, K = 0, Cm = 0, Nb = 0, BL = 0, W = 0, E = 0, D = 0, RW = 0;
  int nnz = 0, nb = 0, max_m = 0, levels = 0, RS = 0, R = 0, rdofs = 0;
  int64_t contributions = 0, factor_stride = 0;
  std::vector<int> perm, iperm, level_begin;
  std::vector<int> csr_ptr, csr_col, csr_row, contrib_ptr, contrib;
  std::vector<int64_t> task_rows, pulls;
  std::vector<float> features, fscale;
  std::vector<int> pair_ptr, pair_list, rcv_dofs;
  std::vector<double> rcv_w;
  std::vector<int> rdof_ptr, rdof_rcv, rdof_dof;
  std::vector<double> rdof_w;
  std::vector<int> cdofs, bd, cell_bptr, cell_blist, model_ptr, model_list;
  std::vector<double> k2;
  std::vector<int> bowners;  // cells owning at least one boundary element, ascending
  std::vector<int> fixed;    // fixed dofs in solver order, ascending
  // tiled solver (blocks wider than kMaxBlock): work items of 4 ints and [begin, end) ranges.
  // Range r: scatter items of level r (task, row0, rows, -); r = L + l: fill tiles of level l
  // (task, qi, pi, -); r = 2L + l: row tiles of the eliminated blocks of level l (task, i, -, -);
  // r = 3L + panel_ptr[l] + k: panel k of level l (task, segment, tile row, -).
  // eager Schur updates of the shared-memory solver: items (task, pull begin, pull end) of
  // the blocks that apply level l's pulls right after level l, range update_begin[l] ..
  std::vector<int> update_items, update_begin;
  bool tiled = false;
  std::vector<int> titems, tranges, panel_ptr;
};

// Validates `pr` and builds every host array of its plan; on failure returns the status and
// sets `err`.
adt_status build_host_plan(const adt_problem* pr, HostPlan& hp, std::string& err);

}  // namespace adt
