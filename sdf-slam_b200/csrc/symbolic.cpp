// Symbolic analysis of the LM normal equations for the multifrontal LDL^T.
//
// Ordering: every grid is split by geometric nested dissection (a one-node
// wide grid line separates the 9-point stencil of the map block), leaves of
// at most kLeafNodes active nodes; the 3(N-1) pose parameters of an instance
// form the last supernode (the dense pose root). This replaces Eigen's AMD
// ordering inside SimplicialLDLT::analyzePattern
// (src/solvers/parallel_ldlt.hpp:38-41).
//
// Pattern: a superset of the reference's structural J^T J
// (src/solvers/lm_solver.cpp:312-320): the full 9-point stencil among active
// nodes (every point row couples the 4 nodes of its cell, every Eikonal row
// three nodes of one cell), for each pose the nodes of the cells its points
// touch dilated by a margin (point rows couple a pose to its cell's nodes),
// same-frame pose blocks and the pose pairs linked by odometry / relation
// rows. When a point leaves its pose's dilated cell set the engine re-runs
// this analysis.
//
// Supernodes are contiguous ranges of the permuted order. The row structure
// of supernode s is the union of the pattern below its columns and of its
// children's structures; its parent is the supernode owning the first row of
// that structure. Any contiguous partition gives a valid assembly tree this
// way.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <numeric>

#include "host_pool.h"
#include "internal.h"
#include "schur_tc.h"

namespace sdfgpu {

namespace {

constexpr int kLeafNodes = 64;

struct LocalSym {
  std::vector<int> sn_begin;               // S + 1 boundaries (local permuted columns)
  std::vector<std::vector<int>> rows;      // R_s, sorted, local permuted
  std::vector<int> parent;
  std::vector<std::vector<int>> children;
};

/// Per-thread map from a column to a value, valid while the column's stamp
/// equals the current generation: starting a new map costs nothing. Pool
/// workers keep theirs from one problem to the next.
struct ColumnMap {
  std::vector<uint32_t> stamp;
  std::vector<int32_t> value;
  uint32_t gen = 0;
  void Begin(size_t n) {
    if (stamp.size() < n) {
      stamp.resize(n, 0u);
      value.resize(n, 0);
    }
    if (++gen == 0u) {
      std::fill(stamp.begin(), stamp.end(), 0u);
      gen = 1u;
    }
  }
  bool Has(int i) const { return stamp[static_cast<size_t>(i)] == gen; }
  void Set(int i, int32_t v) {
    stamp[static_cast<size_t>(i)] = gen;
    value[static_cast<size_t>(i)] = v;
  }
  int32_t Get(int i) const { return value[static_cast<size_t>(i)]; }
};

ColumnMap& ThreadColumnMap() {
  thread_local ColumnMap map;
  return map;
}

/// Generic supernodal symbolic factorization over a partition of the
/// permuted columns. lower(col, out) appends the pattern rows > col.
///
/// `subtrees` lists ranges [begin, end) of supernodes that are closed under
/// the assembly tree below them (every child of a member is a member, as
/// for the groups of one nested-dissection region): those ranges run in
/// parallel, the remaining supernodes afterwards in order. Children lists
/// ascend, so the result equals the plain sequential pass.
LocalSym SupernodalSymbolic(int n, const std::function<void(int, std::vector<int>&)>& lower,
                            const std::vector<int>& sn_begin,
                            const std::vector<std::pair<int, int>>& subtrees = {}) {
  LocalSym L;
  L.sn_begin = sn_begin;
  const int S = static_cast<int>(sn_begin.size()) - 1;
  L.rows.resize(static_cast<size_t>(S));
  L.parent.assign(static_cast<size_t>(S), -1);
  L.children.resize(static_cast<size_t>(S));
  std::vector<int> owner(static_cast<size_t>(n), -1);
  for (int s = 0; s < S; ++s) {
    for (int c = sn_begin[static_cast<size_t>(s)]; c < sn_begin[static_cast<size_t>(s) + 1]; ++c) {
      owner[static_cast<size_t>(c)] = s;
    }
  }
  // range of the subtree holding each supernode (-1: none)
  std::vector<int> in_range(static_cast<size_t>(S), -1);
  for (size_t t = 0; t < subtrees.size(); ++t) {
    for (int s = subtrees[t].first; s < subtrees[t].second; ++s) {
      in_range[static_cast<size_t>(s)] = static_cast<int>(t);
    }
  }
  // Structure of supernode s. It joins its parent's children list here when
  // link_all is set or the parent lies in the same subtree range; the other
  // links are made after the parallel part.
  auto structure = [&](int s, std::vector<int>& tmp, ColumnMap& mark, bool link_all, int range) {
    const int b = sn_begin[static_cast<size_t>(s)];
    const int e = sn_begin[static_cast<size_t>(s) + 1];
    std::vector<int>& R = L.rows[static_cast<size_t>(s)];
    mark.Begin(static_cast<size_t>(n));
    for (int c = b; c < e; ++c) {
      tmp.clear();
      lower(c, tmp);
      for (const int r : tmp) {
        if (r >= e && !mark.Has(r)) {
          mark.Set(r, 0);
          R.push_back(r);
        }
      }
    }
    for (const int ch : L.children[static_cast<size_t>(s)]) {
      for (const int r : L.rows[static_cast<size_t>(ch)]) {
        if (r >= e && !mark.Has(r)) {
          mark.Set(r, 0);
          R.push_back(r);
        }
      }
    }
    std::sort(R.begin(), R.end());
    if (!R.empty()) {
      const int p = owner[static_cast<size_t>(R.front())];
      L.parent[static_cast<size_t>(s)] = p;
      if (link_all || in_range[static_cast<size_t>(p)] == range) {
        L.children[static_cast<size_t>(p)].push_back(s);
      }
    }
  };
  PoolRun(static_cast<int>(subtrees.size()), [&](int t) {
    std::vector<int> tmp;
    ColumnMap& mark = ThreadColumnMap();
    for (int s = subtrees[static_cast<size_t>(t)].first; s < subtrees[static_cast<size_t>(t)].second; ++s) {
      structure(s, tmp, mark, false, t);
    }
  });
  // links from the subtrees to the supernodes above them, ascending
  for (int s = 0; s < S; ++s) {
    const int p = L.parent[static_cast<size_t>(s)];
    if (in_range[static_cast<size_t>(s)] >= 0 && p >= 0 &&
        in_range[static_cast<size_t>(p)] != in_range[static_cast<size_t>(s)]) {
      L.children[static_cast<size_t>(p)].push_back(s);
    }
  }
  {
    std::vector<int> tmp;
    ColumnMap& mark = ThreadColumnMap();
    for (int s = 0; s < S; ++s) {
      if (in_range[static_cast<size_t>(s)] < 0) {
        structure(s, tmp, mark, true, -1);
      }
    }
  }
  for (std::vector<int>& ch : L.children) {
    std::sort(ch.begin(), ch.end());
  }
  return L;
}

/// Geometric nested dissection of the active nodes of a grid. Appends groups
/// of local natural columns in postorder (halves, then separator). The
/// regions `split` levels down each record their range of groups in
/// `subtrees` (none when split < 0).
void Dissect(const HostProblem& hp, int w0, int w1, int h0, int h1, std::vector<std::vector<int>>& groups,
             int depth, int split, std::vector<std::pair<int, int>>& subtrees) {
  if (depth == split) {
    // the groups of this region form one subtree of the assembly tree
    const int begin = static_cast<int>(groups.size());
    Dissect(hp, w0, w1, h0, h1, groups, depth + 1, split, subtrees);
    if (static_cast<int>(groups.size()) > begin) {
      subtrees.emplace_back(begin, static_cast<int>(groups.size()));
    }
    return;
  }
  const int width = w1 - w0;
  const int height = h1 - h0;
  if (width <= 0 || height <= 0) {
    return;
  }
  int active = 0;
  for (int h = h0; h < h1; ++h) {
    for (int w = w0; w < w1; ++w) {
      active += hp.node_to_active[static_cast<size_t>(h) * hp.nx + w] >= 0 ? 1 : 0;
    }
  }
  if (active == 0) {
    return;
  }
  if (active <= kLeafNodes || (width <= 2 && height <= 2)) {
    std::vector<int> g;
    for (int h = h0; h < h1; ++h) {
      for (int w = w0; w < w1; ++w) {
        const int c = hp.node_to_active[static_cast<size_t>(h) * hp.nx + w];
        if (c >= 0) {
          g.push_back(c);
        }
      }
    }
    groups.push_back(std::move(g));
    return;
  }
  std::vector<int> sep;
  if (width >= height) {
    const int mid = w0 + width / 2;
    Dissect(hp, w0, mid, h0, h1, groups, depth + 1, split, subtrees);
    Dissect(hp, mid + 1, w1, h0, h1, groups, depth + 1, split, subtrees);
    for (int h = h0; h < h1; ++h) {
      const int c = hp.node_to_active[static_cast<size_t>(h) * hp.nx + mid];
      if (c >= 0) {
        sep.push_back(c);
      }
    }
  } else {
    const int mid = h0 + height / 2;
    Dissect(hp, w0, w1, h0, mid, groups, depth + 1, split, subtrees);
    Dissect(hp, w0, w1, mid + 1, h1, groups, depth + 1, split, subtrees);
    for (int w = w0; w < w1; ++w) {
      const int c = hp.node_to_active[static_cast<size_t>(mid) * hp.nx + w];
      if (c >= 0) {
        sep.push_back(c);
      }
    }
  }
  if (!sep.empty()) {
    groups.push_back(std::move(sep));
  }
}

/// Position of permuted row r inside the front index list of supernode s.
inline int LocalIndex(const SupernodeRec& s, const int32_t* rows, int r) {
  if (r < s.first_col + s.ncols) {
    return r - s.first_col;
  }
  const int32_t* it = std::lower_bound(rows, rows + s.nrows, r);
  return s.ncols + static_cast<int>(it - rows);
}

void AppendInstance(Symbolic& S, const LocalSym& L, int col_off, int instance, std::vector<int>& height) {
  const int S0 = static_cast<int>(S.sn.size());
  const int Sn = static_cast<int>(L.rows.size());
  for (int s = 0; s < Sn; ++s) {
    SupernodeRec r{};
    r.first_col = col_off + L.sn_begin[static_cast<size_t>(s)];
    r.ncols = L.sn_begin[static_cast<size_t>(s) + 1] - L.sn_begin[static_cast<size_t>(s)];
    r.nrows = static_cast<int>(L.rows[static_cast<size_t>(s)].size());
    r.F = r.ncols + r.nrows;
    r.parent = L.parent[static_cast<size_t>(s)] >= 0 ? S0 + L.parent[static_cast<size_t>(s)] : -1;
    r.instance = instance;
    r.rows_off = static_cast<int64_t>(S.sn_rows.size());
    for (const int row : L.rows[static_cast<size_t>(s)]) {
      S.sn_rows.push_back(col_off + row);
    }
    r.child_begin = static_cast<int>(S.child_list.size());
    r.child_count = static_cast<int>(L.children[static_cast<size_t>(s)].size());
    for (const int c : L.children[static_cast<size_t>(s)]) {
      S.child_list.push_back(S0 + c);
    }
    r.front_off = S.front_doubles;
    const int64_t size = static_cast<int64_t>(r.F) * r.F;
    S.front_doubles += (size + 31) / 32 * 32;
    r.upd_off = S.update_doubles;
    S.update_doubles += r.nrows;
    S.sn.push_back(r);
    int hgt = 0;
    for (const int c : L.children[static_cast<size_t>(s)]) {
      hgt = std::max(hgt, height[static_cast<size_t>(S0 + c)] + 1);
    }
    height.push_back(hgt);
    for (int c = r.first_col; c < r.first_col + r.ncols; ++c) {
      S.col_owner[static_cast<size_t>(c)] = S0 + s;
    }
    // useful flops of the partial factorization: sum over pivots of the
    // (F - j - 1)^2 multiply-adds of the rank-1 update plus the divisions
    for (int j = 0; j < r.ncols; ++j) {
      const int64_t rem = r.F - j - 1;
      S.total_flops += rem * rem + rem;
    }
  }
}

/// Relative indices, level lists and task lists once all supernodes exist.
/// Position of every front row in its parent's front (extend-add map).
void ComputeRel(Symbolic& S) {
  const int Sn = static_cast<int>(S.sn.size());
  S.sn_rel.assign(S.sn_rows.size(), 0);
  for (int s = 0; s < Sn; ++s) {
    const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    if (r.parent < 0) {
      continue;
    }
    const SupernodeRec& p = S.sn[static_cast<size_t>(r.parent)];
    // both row lists ascend: one merge walk
    const int32_t* prow = S.sn_rows.data() + p.rows_off;
    int j = 0;
    for (int q = 0; q < r.nrows; ++q) {
      const int32_t row = S.sn_rows[static_cast<size_t>(r.rows_off + q)];
      if (row < p.first_col + p.ncols) {
        S.sn_rel[static_cast<size_t>(r.rows_off + q)] = row - p.first_col;
        continue;
      }
      while (j < p.nrows && prow[j] < row) {
        ++j;
      }
      S.sn_rel[static_cast<size_t>(r.rows_off + q)] = p.ncols + j;
    }
  }
}

/// Level lists and task lists once all supernodes exist.
void Finalize(Symbolic& S, const std::vector<int>& height, int panel_width, int tile) {
  S.panel_width = panel_width;
  S.tile = tile;
  S.height = height;
  const int Sn = static_cast<int>(S.sn.size());
  int levels = 0;
  for (const int h : height) {
    levels = std::max(levels, h + 1);
  }
  S.num_levels = levels;
  S.level_begin.assign(static_cast<size_t>(levels) + 1, 0);
  for (const int h : height) {
    ++S.level_begin[static_cast<size_t>(h) + 1];
  }
  for (int l = 0; l < levels; ++l) {
    S.level_begin[static_cast<size_t>(l) + 1] += S.level_begin[static_cast<size_t>(l)];
  }
  S.level_sn.assign(static_cast<size_t>(Sn), 0);
  {
    std::vector<int> fill(S.level_begin.begin(), S.level_begin.end() - 1);
    for (int s = 0; s < Sn; ++s) {
      S.level_sn[static_cast<size_t>(fill[static_cast<size_t>(height[static_cast<size_t>(s)])]++)] = s;
    }
  }
  const int B = panel_width;
  const int T = tile;
  constexpr int kEaCols = 16;
  const int kFrontRows = S.front_rows;
  // launch slots of the wide fronts: one per outer block when whole outer
  // blocks are factored at once (panel_rows 0), else one per panel
  const bool block_mode = S.panel_rows == 0;
  const int slot_width = block_mode ? kOuterPanels * B : B;
  // dense pose roots take the tiled launch instead of panels
  auto tiled = [&S](const SupernodeRec& r) { return r.pose_root != 0 && r.nrows == 0 && r.ncols > S.small_pivots; };
  // fronts factored by the single-kernel path keep the pivot block's lower
  // triangle (read by every task of the front) and store L11 transposed
  for (SupernodeRec& r : S.sn) {
    r.upper_l11 = r.ncols <= S.small_pivots ? 1 : 0;
  }
  S.inv_tasks.clear();
  for (int s = 0; s < Sn; ++s) {
    SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    r.panel_base = static_cast<int32_t>(S.inv_tasks.size() / 2);
    for (int p = 0; p * B < r.ncols; ++p) {
      S.inv_tasks.push_back(s);
      S.inv_tasks.push_back(p);
    }
  }
  // blocks that keep every SM of a B200 (148) busy
  constexpr int64_t kFillBlocks = 148;
  const int small = S.small_pivots;
  S.level_panels.assign(static_cast<size_t>(levels), 0);
  S.panel_index_base.assign(static_cast<size_t>(levels) + 1, 0);
  S.small_range.assign(static_cast<size_t>(levels), {});
  S.small_max_k.assign(static_cast<size_t>(levels), 0);
  S.small_threads.assign(static_cast<size_t>(levels), S.front_rows);
  S.small_tasks.clear();
  for (int l = 0; l < levels; ++l) {
    int maxp = 0;
    S.small_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.small_tasks.size() / 3);
    // Rows per single-kernel task: the schedule's front_rows, or fewer where
    // the level would not fill the GPU (every task repeats the pivot block,
    // so small chunks shorten the level when SMs would otherwise idle).
    int chunk = kFrontRows;
    int threads = kFrontRows;
    int fronts = 0;
    for (int q = S.level_begin[static_cast<size_t>(l)]; q < S.level_begin[static_cast<size_t>(l) + 1]; ++q) {
      fronts += S.sn[static_cast<size_t>(S.level_sn[static_cast<size_t>(q)])].ncols <= small ? 1 : 0;
    }
    // more fronts than SMs: blocks of 128 threads (two per SM by registers)
    // and chunks of 128 rows keep the level in about one wave
    const bool many = fronts > kFillBlocks && kFrontRows > 128;
    for (const int cand : {many ? 128 : kFrontRows, 64, 32}) {
      chunk = cand;
      int64_t blocks = 0;
      for (int q = S.level_begin[static_cast<size_t>(l)]; q < S.level_begin[static_cast<size_t>(l) + 1]; ++q) {
        const SupernodeRec& r = S.sn[static_cast<size_t>(S.level_sn[static_cast<size_t>(q)])];
        if (r.ncols <= small) {
          blocks += std::max(1, (r.nrows + cand - 1) / cand);
        }
      }
      if (blocks >= kFillBlocks) {
        break;
      }
    }
    if (many) {
      threads = 128;
    }
    S.small_threads[static_cast<size_t>(l)] = threads;
    for (int q = S.level_begin[static_cast<size_t>(l)]; q < S.level_begin[static_cast<size_t>(l) + 1]; ++q) {
      const int sid = S.level_sn[static_cast<size_t>(q)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(sid)];
      if (r.ncols <= small) {
        const int chunks = std::max(1, (r.nrows + chunk - 1) / chunk);
        for (int ch = 0; ch < chunks; ++ch) {
          S.small_tasks.push_back(sid);
          S.small_tasks.push_back(r.ncols + ch * chunk);
          S.small_tasks.push_back(chunk);
        }
        S.small_max_k[static_cast<size_t>(l)] = std::max(S.small_max_k[static_cast<size_t>(l)], r.ncols);
        continue;
      }
      if (!tiled(r)) {
        maxp = std::max(maxp, (r.ncols + slot_width - 1) / slot_width);
      }
    }
    S.small_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.small_tasks.size() / 3) - S.small_range[static_cast<size_t>(l)].begin;
    S.level_panels[static_cast<size_t>(l)] = maxp;
    S.panel_index_base[static_cast<size_t>(l) + 1] = S.panel_index_base[static_cast<size_t>(l)] + maxp;
  }
  const int slots = S.panel_index_base.back();
  S.panel_range.assign(static_cast<size_t>(slots), {});
  S.update_range.assign(static_cast<size_t>(slots), {});
  S.ea_range.assign(static_cast<size_t>(levels), {});
  S.ea_stage.assign(static_cast<size_t>(levels), 0);
  // sibling slots (see the Schur tasks below)
  std::vector<int32_t> sibling_slot(static_cast<size_t>(Sn), 0);
  {
    std::vector<int32_t> per_level(static_cast<size_t>(levels), 0);
    for (int p = 0; p < Sn; ++p) {
      const SupernodeRec& r = S.sn[static_cast<size_t>(p)];
      for (int ci = 0; ci < r.child_count; ++ci) {
        const int c = S.child_list[static_cast<size_t>(r.child_begin + ci)];
        sibling_slot[static_cast<size_t>(c)] = per_level[static_cast<size_t>(height[static_cast<size_t>(c)])]++;
      }
      for (int ci = 0; ci < r.child_count; ++ci) {
        const int c = S.child_list[static_cast<size_t>(r.child_begin + ci)];
        per_level[static_cast<size_t>(height[static_cast<size_t>(c)])] = 0;
      }
    }
  }
  S.schur_range.clear();
  S.schur_base.assign(static_cast<size_t>(levels) + 1, 0);
  for (int l = 0; l < levels; ++l) {
    const int qb = S.level_begin[static_cast<size_t>(l)];
    const int qe = S.level_begin[static_cast<size_t>(l) + 1];
    // extend-add: parent columns in chunks, only for supernodes with children
    S.ea_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.ea_tasks.size() / 4);
    // narrower column ranges on levels that would not fill the GPU
    int ea_cols = kEaCols;
    {
      int64_t tasks = 0;
      for (int q = qb; q < qe; ++q) {
        const SupernodeRec& r = S.sn[static_cast<size_t>(S.level_sn[static_cast<size_t>(q)])];
        if (r.child_count > 0) {
          tasks += (r.F + kEaCols - 1) / kEaCols;
        }
      }
      if (tasks < 2 * kFillBlocks) {
        ea_cols = 4;
      }
    }
    std::vector<int32_t> cursor;
    int32_t stage = 0;
    for (int q = qb; q < qe; ++q) {
      const int s = S.level_sn[static_cast<size_t>(q)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      if (r.child_count == 0) {
        continue;
      }
      // a task of a front up to kEaStageMaxF wide stages its columns' lower
      // part in shared memory (narrower ranges where they would not fit)
      const bool staged = r.F <= kEaStageMaxF;
      const int cols = staged ? std::max(1, std::min(ea_cols, kEaStageDoubles / r.F)) : ea_cols;
      // per child: the range of its update columns that land in [c, chi);
      // the positions ascend, so one cursor per child walks them once
      cursor.assign(static_cast<size_t>(r.child_count), 0);
      for (int c = 0; c < r.F; c += cols) {
        const int chi = std::min(r.F, c + cols);
        if (staged) {
          stage = std::max(stage, (chi - c) * (r.F - c));
        }
        S.ea_tasks.push_back(s);
        S.ea_tasks.push_back(c);
        S.ea_tasks.push_back(chi);
        S.ea_tasks.push_back(static_cast<int32_t>(S.ea_child.size()));
        for (int ci = 0; ci < r.child_count; ++ci) {
          const SupernodeRec& ch = S.sn[static_cast<size_t>(S.child_list[static_cast<size_t>(r.child_begin + ci)])];
          const int32_t* rel = S.sn_rel.data() + ch.rows_off;
          int32_t& k = cursor[static_cast<size_t>(ci)];
          S.ea_child.push_back(k);
          while (k < ch.nrows && rel[k] < chi) {
            ++k;
          }
          S.ea_child.push_back(k);
        }
      }
    }
    S.ea_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.ea_tasks.size() / 4) - S.ea_range[static_cast<size_t>(l)].begin;
    S.ea_stage[static_cast<size_t>(l)] = stage;
    for (int t = 0; t < S.level_panels[static_cast<size_t>(l)]; ++t) {
      const size_t slot = static_cast<size_t>(S.panel_index_base[static_cast<size_t>(l)] + t);
      S.panel_range[slot].begin = static_cast<int64_t>(S.panel_tasks.size() / 3);
      S.update_range[slot].begin = static_cast<int64_t>(S.update_tasks.size() / 4);
      for (int q = qb; q < qe; ++q) {
        const int s = S.level_sn[static_cast<size_t>(q)];
        const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
        if (tiled(r)) {
          continue;
        }
        const int outer = kOuterPanels * B;
        auto tiles = [&S, s, T](int32_t code, int nr, int nc) {
          for (int tj = 0; tj * T < nc; ++tj) {
            for (int ti = 0; ti * T < nr; ++ti) {
              // lower part only: the tile must reach at or below the diagonal
              if ((ti + 1) * T - 1 < tj * T) {
                continue;
              }
              S.update_tasks.push_back(s);
              S.update_tasks.push_back(code);
              S.update_tasks.push_back(ti);
              S.update_tasks.push_back(tj);
            }
          }
        };
        if (block_mode) {
          // slot t: outer block t, factored with the rows below it by block
          // tasks (sn, t, first row of a kBlockRows chunk; the first chunk
          // writes the block), then the block's update of the pivot columns
          // [c1, k), rows [c1, F)
          const int c0 = t * outer;
          if (c0 >= r.ncols || r.ncols <= small) {
            continue;
          }
          const int c1 = std::min(r.ncols, c0 + outer);
          const int chunks = std::max(1, (r.F - c1 + kBlockRows - 1) / kBlockRows);
          for (int ch = 0; ch < chunks; ++ch) {
            S.panel_tasks.push_back(s);
            S.panel_tasks.push_back(t);
            S.panel_tasks.push_back(c1 + ch * kBlockRows);
          }
          tiles(UpdateCodeOuter(t), r.F - c1, r.ncols - c1);
          continue;
        }
        // slot t: panel t (sn, t, first row of a panel_rows chunk; chunk 0
        // also owns the diagonal block), then the panel's update of the
        // pivot columns [c1, cend) left in its outer block, rows [c1, F); the
        // outer block's last panel is followed by the block's update of the
        // pivot columns [cend, k), rows [cend, F)
        const int c0 = t * B;
        if (c0 >= r.ncols || r.ncols <= small) {
          continue;
        }
        const int c1 = std::min(r.ncols, c0 + B);
        const int chunks = std::max(1, (r.F - c1 + S.panel_rows - 1) / S.panel_rows);
        for (int ch = 0; ch < chunks; ++ch) {
          S.panel_tasks.push_back(s);
          S.panel_tasks.push_back(t);
          S.panel_tasks.push_back(c1 + ch * S.panel_rows);
        }
        const int cend = std::min(r.ncols, (c0 / outer + 1) * outer);
        if (c1 < cend) {
          tiles(UpdateCodeInner(t), r.F - c1, cend - c1);
        } else if (cend < r.ncols) {
          tiles(UpdateCodeOuter(c0 / outer), r.F - cend, r.ncols - cend);
        }
      }
      S.panel_range[slot].count = static_cast<int64_t>(S.panel_tasks.size() / 3) - S.panel_range[slot].begin;
      S.update_range[slot].count = static_cast<int64_t>(S.update_tasks.size() / 4) - S.update_range[slot].begin;
    }
    // Schur complements, added straight into the parents' fronts: fronts of
    // the level that share a parent go in separate launches, one per sibling
    // slot (the front's rank among its parent's children of this level, in
    // child-list order), so no two blocks of a launch add into one entry
    // and each parent entry takes its children's terms in a fixed order
    S.schur_base[static_cast<size_t>(l)] = static_cast<int32_t>(S.schur_range.size());
    for (int slot = 0;; ++slot) {
      TaskRange range;
      range.begin = static_cast<int64_t>(S.update_tasks.size() / 4);
      bool any = false;
      for (int q = qb; q < qe; ++q) {
        const int s = S.level_sn[static_cast<size_t>(q)];
        if (sibling_slot[static_cast<size_t>(s)] != slot) {
          continue;
        }
        any = true;
        const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
        const int m = r.nrows;
        for (int tj = 0; tj * T < m; ++tj) {
          for (int ti = tj; ti * T < m; ++ti) {
            S.update_tasks.push_back(s);
            S.update_tasks.push_back(-1);
            S.update_tasks.push_back(ti);
            S.update_tasks.push_back(tj);
          }
        }
      }
      if (!any) {
        break;
      }
      range.count = static_cast<int64_t>(S.update_tasks.size() / 4) - range.begin;
      S.schur_range.push_back(range);
    }
  }
  S.schur_base[static_cast<size_t>(levels)] = static_cast<int32_t>(S.schur_range.size());
  // one-launch solve tasks
  S.solve_tasks.clear();
  S.solve_parts.assign(2 * static_cast<size_t>(Sn), 1);
  S.zpart_off.assign(static_cast<size_t>(Sn), -1);
  S.zpart_doubles = 0;
  auto push_task = [&S](int32_t type, int32_t sn, int32_t part) {
    S.solve_tasks.push_back(type);
    S.solve_tasks.push_back(sn);
    S.solve_tasks.push_back(part);
    S.solve_tasks.push_back(0);
  };
  auto root_split = [&S](const SupernodeRec& r) { return r.nrows == 0 && r.ncols >= kSolveRootSplit &&
                                                         r.ncols > S.small_pivots; };
  for (int q = 0; q < Sn; ++q) {
    const int s = S.level_sn[static_cast<size_t>(q)];
    const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    if (root_split(r)) {
      // a tiled dense root solves by 64-row panels with its tile inverses
      const int pw = tiled(r) ? kDenseTileCols : B;
      const int np = (r.ncols + pw - 1) / pw;
      push_task(kTaskRootGather, s, 0);
      for (int p = 0; p < np; ++p) {
        push_task(kTaskRootForward, s, p);
      }
      S.solve_parts[2 * static_cast<size_t>(s)] = np;
      S.solve_parts[2 * static_cast<size_t>(s) + 1] = np;
    } else if (r.nrows >= kSolveWideRows) {
      const int chunks = (r.nrows + kSolveRowChunk - 1) / kSolveRowChunk;
      push_task(kTaskForward, s, 0);
      for (int p = 0; p < chunks; ++p) {
        push_task(kTaskForwardRows, s, p);
      }
      S.solve_parts[2 * static_cast<size_t>(s)] = 1 + chunks;
      S.zpart_off[static_cast<size_t>(s)] = S.zpart_doubles;
      S.zpart_doubles += static_cast<int64_t>(chunks) * r.ncols;
    } else {
      push_task(kTaskForward, s, 0);
    }
  }
  for (int q = Sn - 1; q >= 0; --q) {
    const int s = S.level_sn[static_cast<size_t>(q)];
    const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    if (root_split(r)) {
      const int pw = tiled(r) ? kDenseTileCols : B;
      for (int p = (r.ncols + pw - 1) / pw - 1; p >= 0; --p) {
        push_task(kTaskRootBackward, s, p);
      }
    } else if (r.nrows >= kSolveWideRows) {
      const int chunks = (r.nrows + kSolveRowChunk - 1) / kSolveRowChunk;
      for (int p = 0; p < chunks; ++p) {
        push_task(kTaskBackwardRows, s, p);
      }
      push_task(kTaskBackward, s, 0);
    } else {
      push_task(kTaskBackward, s, 0);
    }
  }
  // tensor-core Schur tasks of the wide grid fronts (used by mixed solves)
  S.pack_tasks.clear();
  S.tc_tasks.clear();
  S.pack_range.assign(static_cast<size_t>(levels), {});
  S.tc_range.assign(static_cast<size_t>(levels), {});
  S.tc_pack_rows = 0;
  for (SupernodeRec& r : S.sn) {
    r.tc_pack = -1;
  }
  for (int l = 0; l < levels; ++l) {
    const int qb = S.level_begin[static_cast<size_t>(l)];
    const int qe = S.level_begin[static_cast<size_t>(l) + 1];
    int64_t rows = 0;
    S.pack_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.pack_tasks.size() / 3);
    S.tc_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.tc_tasks.size() / 3);
    for (int q = qb; q < qe; ++q) {
      const int s = S.level_sn[static_cast<size_t>(q)];
      SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      if (r.pose_root != 0 || S.tc_min_rows <= 0 || r.nrows < S.tc_min_rows || r.ncols < 1) {
        continue;
      }
      r.tc_pack = rows;
      rows += TcPackRows(r.ncols, r.nrows);
      const int nT = (r.nrows + kTcTile - 1) / kTcTile;
      const int nC = (r.ncols + kTcChunk - 1) / kTcChunk;
      for (int t = 0; t < nT; ++t) {
        for (int c = 0; c < nC; ++c) {
          S.pack_tasks.push_back(s);
          S.pack_tasks.push_back(t);
          S.pack_tasks.push_back(c);
        }
      }
      for (int tj = 0; tj < nT; ++tj) {
        for (int ti = tj; ti < nT; ++ti) {
          S.tc_tasks.push_back(s);
          S.tc_tasks.push_back(ti);
          S.tc_tasks.push_back(tj);
        }
      }
    }
    S.pack_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.pack_tasks.size() / 3) - S.pack_range[static_cast<size_t>(l)].begin;
    S.tc_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.tc_tasks.size() / 3) - S.tc_range[static_cast<size_t>(l)].begin;
    S.tc_pack_rows = std::max(S.tc_pack_rows, rows);
  }
  // front clearing tasks
  S.zero_tasks.clear();
  for (int pass = 0; pass < 2; ++pass) {
    for (int s = 0; s < Sn; ++s) {
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      const int split = r.child_count == 0 ? r.ncols : r.F;
      for (int c = 0; c < r.F; c += kZeroCols) {
        if ((c < split) == (pass == 0)) {
          S.zero_tasks.push_back(s);
          S.zero_tasks.push_back(c);
        }
      }
    }
    if (pass == 0) {
      S.zero_main = static_cast<int64_t>(S.zero_tasks.size() / 2);
    }
  }
  // tiled dense roots: counters, inverse workspace and task lists per level
  S.dense_tasks.clear();
  S.dense_range.assign(static_cast<size_t>(levels), {});
  S.dense_cnt_words = 0;
  S.dense_inv_doubles = 0;
  for (SupernodeRec& r : S.sn) {
    r.dense_cnt = -1;
    r.dense_inv = 0;
    if (tiled(r)) {
      const int64_t nt = (r.ncols + kDenseTileCols - 1) / kDenseTileCols;
      r.dense_cnt = S.dense_cnt_words;
      r.dense_inv = S.dense_inv_doubles;
      S.dense_cnt_words += nt * nt;
      S.dense_inv_doubles += nt * kDenseTileCols * kDenseTileCols;
    }
  }
  std::vector<DenseTileTask> level_tasks;
  for (int l = 0; l < levels; ++l) {
    level_tasks.clear();
    for (int q = S.level_begin[static_cast<size_t>(l)]; q < S.level_begin[static_cast<size_t>(l) + 1]; ++q) {
      const int s = S.level_sn[static_cast<size_t>(q)];
      if (S.sn[static_cast<size_t>(s)].dense_cnt >= 0) {
        AppendDenseTileTasks(s, S.sn[static_cast<size_t>(s)].ncols, &level_tasks);
      }
    }
    OrderDenseTileTasks(&level_tasks);
    S.dense_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.dense_tasks.size() / 4);
    for (const DenseTileTask& t : level_tasks) {
      S.dense_tasks.push_back(t.sn);
      S.dense_tasks.push_back(t.i);
      S.dense_tasks.push_back(t.j);
      S.dense_tasks.push_back(t.k);
    }
    S.dense_range[static_cast<size_t>(l)].count = static_cast<int64_t>(level_tasks.size());
  }
}

}  // namespace

/// Appends the tasks of an n-column dense root's tiled LDL^T with their
/// bottom levels: the longest path of task weights (about their relative
/// durations) from the task to the end of the graph, so that sorting by it
/// descending lists each task after the tasks it waits for. Tasks: FACTOR(k)
/// (with SOLVE(k, k - 1) and UPDATE(k, k, k - 1) folded in for k >= 1),
/// SOLVE(i, k) for i >= k + 2, UPDATE(i, j, k) for k < j <= i except
/// (k + 1, k + 1, k). Successors:
///   FACTOR(k)     -> FACTOR(k + 1), SOLVE(i, k), UPDATE(i, k, k - 1) (it
///                    produces L(k, k - 1));
///   SOLVE(i, k)   -> UPDATE(i, j, k), UPDATE(i', i, k);
///   UPDATE(i,j,k) -> the next step's task on tile (i, j): UPDATE(i, j, k + 1)
///                    or, folded into them, FACTOR(j) (i == j == k + 2) and
///                    FACTOR(j + 1) (i == j + 1 == k + 2); SOLVE(i, j) when
///                    j == k + 1 and i >= j + 2.
/// A topological order is tau = 4k (FACTOR), 4k + 1 (SOLVE), 4k + 2 (UPDATE,
/// j >= k + 2), 4k + 4.5 (UPDATE, j == k + 1); the bottom levels are
/// computed in decreasing tau.
void AppendDenseTileTasks(int32_t sn, int n, std::vector<DenseTileTask>* out) {
  const int nt = (n + kDenseTileCols - 1) / kDenseTileCols;
  constexpr double kWFactor = 6.0;     // FACTOR(0) alone
  constexpr double kWFolded = 14.0;    // FACTOR(k >= 1) with its SOLVE and UPDATE
  constexpr double kWSolve = 4.0;
  constexpr double kWUpdate = 4.0;
  struct Item {
    double tau;
    int32_t i, j, k;
  };
  std::vector<Item> items;
  for (int k = 0; k < nt; ++k) {
    items.push_back({4.0 * k, k, k, k});
    for (int i = k + 2; i < nt; ++i) {
      items.push_back({4.0 * k + 1.0, i, k, k});
    }
    for (int j = k + 1; j < nt; ++j) {
      for (int i = j; i < nt; ++i) {
        if (i == k + 1 && j == k + 1) {
          continue;
        }
        items.push_back({j == k + 1 ? 4.0 * k + 4.5 : 4.0 * k + 2.0, i, j, k});
      }
    }
  }
  std::sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.tau > b.tau; });
  const size_t nn = static_cast<size_t>(nt) * nt;
  // bottom levels: FACTOR per k, SOLVE per (i, k), UPDATE per (i, j) of the
  // step being computed and of the step after it (tau orders steps so that
  // both are all that is read)
  std::vector<double> bf(static_cast<size_t>(nt), 0.0);
  std::vector<double> bs(nn, 0.0);
  std::vector<std::vector<double>> bu(static_cast<size_t>(nt) + 1);
  auto ub = [&](int i, int j, int k) -> double {
    if (k >= nt || bu[static_cast<size_t>(k)].empty()) {
      return 0.0;
    }
    return bu[static_cast<size_t>(k)][static_cast<size_t>(i) * nt + j];
  };
  auto uset = [&](int i, int j, int k, double v) {
    std::vector<double>& b = bu[static_cast<size_t>(k)];
    if (b.empty()) {
      b.assign(nn, 0.0);
    }
    b[static_cast<size_t>(i) * nt + j] = v;
  };
  auto next_on_tile = [&](int i, int j, int k) -> double {
    // the task that next reads or writes tile (i, j) after UPDATE(i, j, k)
    if (k + 1 < j) {
      if (i == j && j == k + 2) {
        return bf[static_cast<size_t>(j)];
      }
      if (i == j + 1 && j == k + 1) {
        return bf[static_cast<size_t>(i)];
      }
      return ub(i, j, k + 1);
    }
    // j == k + 1: the tile is complete
    if (i == j + 1) {
      return bf[static_cast<size_t>(i)];
    }
    return bs[static_cast<size_t>(i) * nt + j];
  };
  std::vector<DenseTileTask> local;
  local.reserve(items.size());
  for (const Item& it : items) {
    const int i = it.i;
    const int j = it.j;
    const int k = it.k;
    double b;
    if (i == k && j == k) {
      double m = k + 1 < nt ? bf[static_cast<size_t>(k) + 1] : 0.0;
      for (int r = k + 2; r < nt; ++r) {
        m = std::max(m, bs[static_cast<size_t>(r) * nt + k]);
      }
      if (k >= 1) {
        for (int r = k + 1; r < nt; ++r) {
          m = std::max(m, ub(r, k, k - 1));
        }
      }
      b = (k == 0 ? kWFactor : kWFolded) + m;
      bf[static_cast<size_t>(k)] = b;
    } else if (j == k) {
      double m = 0.0;
      for (int c = k + 1; c <= i; ++c) {
        m = std::max(m, ub(i, c, k));
      }
      for (int r = i; r < nt; ++r) {
        m = std::max(m, ub(r, i, k));
      }
      b = kWSolve + m;
      bs[static_cast<size_t>(i) * nt + k] = b;
    } else {
      b = kWUpdate + next_on_tile(i, j, k);
      uset(i, j, k, b);
    }
    local.push_back({b, sn, i, j, k});
    // steps two behind the one being computed are no longer read
    if (k + 3 <= nt && !bu[static_cast<size_t>(k) + 2].empty() && i == k && j == k) {
      std::vector<double>().swap(bu[static_cast<size_t>(k) + 2]);
    }
  }
  out->insert(out->end(), local.begin(), local.end());
}

void OrderDenseTileTasks(std::vector<DenseTileTask>* tasks) {
  std::sort(tasks->begin(), tasks->end(), [](const DenseTileTask& a, const DenseTileTask& b) {
    if (a.prio != b.prio) {
      return a.prio > b.prio;
    }
    if (a.k != b.k) {
      return a.k < b.k;
    }
    if (a.i != b.i) {
      return a.i < b.i;
    }
    if (a.j != b.j) {
      return a.j < b.j;
    }
    return a.sn < b.sn;
  });
}

SymPiece AnalyzeInstance(const HostProblem& hp, int margin, int threads, const std::vector<double>* poses) {
  if (threads <= 0) {
    threads = PoolThreads();
  }
  if (margin < 0) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "negative coupling margin");
  }
  const std::vector<double>& state = poses != nullptr ? *poses : hp.poses;
  if (state.size() != hp.poses.size()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "analysed poses do not match the problem's frames");
  }
  // The per-pose coupling sets are derived from the current cells of every
  // point row, dilated by `margin` cells.
  SymPiece piece;
  piece.margin = margin;
  Symbolic& S = piece.s;
  std::vector<int>& height = piece.height;
  const int n = hp.num_params();
  S.n = n;
  S.perm.assign(static_cast<size_t>(n), 0);
  S.pinv.assign(static_cast<size_t>(n), 0);
  S.col_owner.assign(static_cast<size_t>(n), -1);
  S.mm_off.assign(static_cast<size_t>(n) * 9, -1);
  S.mp_ptr.assign(static_cast<size_t>(n) + 1, 0);
  S.allow_off.assign(1, 0);
  S.allow_words.assign(1, 0);
  S.pp_base.assign(1, -1);
  S.pp_ld.assign(1, 0);
  S.pp_first.assign(1, 0);
  const int A = hp.num_active();
  const int Fr = hp.num_frames();
  const int np = hp.num_params();
  const int col_off = 0;
  // 1. partition and permutation (local); the regions a few levels down the
  // dissection are subtrees of the assembly tree, analysed in parallel
  std::vector<std::vector<int>> groups;
  std::vector<std::pair<int, int>> subtrees;
  int split = 0;
  while (split < 4 && (1 << split) < threads) {
    ++split;
  }
  Dissect(hp, 0, hp.nx, 0, hp.ny, groups, 0, threads > 1 ? split : -1, subtrees);
  std::vector<int> lperm;
  std::vector<int> sn_begin{0};
  for (const auto& g : groups) {
    lperm.insert(lperm.end(), g.begin(), g.end());
    sn_begin.push_back(static_cast<int>(lperm.size()));
  }
  if (static_cast<int>(lperm.size()) != A) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "nested dissection lost active nodes");
  }
  if (Fr > 1) {
    for (int c = A; c < np; ++c) {
      lperm.push_back(c);
    }
    sn_begin.push_back(np);
  }
  std::vector<int> lpinv(static_cast<size_t>(np));
  for (int k = 0; k < np; ++k) {
    lpinv[static_cast<size_t>(lperm[static_cast<size_t>(k)])] = k;
    S.perm[static_cast<size_t>(col_off + k)] = col_off + lperm[static_cast<size_t>(k)];
    S.pinv[static_cast<size_t>(col_off + lperm[static_cast<size_t>(k)])] = col_off + k;
  }
  // 2. pose coupling: frames coupled to each active node (ascending). The
  // points of each frame (in any order in the caller's specs) give the cells
  // they occupy; that set dilated by `margin` cells (clipped to the grid) is
  // the frame's allowed set (one bitmap row per frame), and the corner nodes
  // of the allowed cells are coupled to the frame. Frames run in parallel on
  // row-major 64-bit bitmaps of the cell grid.
  // frame-major lists: the coupled columns of frame f, ascending, at
  // fmp_ptr[f]..fmp_ptr[f + 1] of fmp_col
  std::vector<std::vector<int32_t>> frame_cols(static_cast<size_t>(std::max(Fr, 1)));
  {
    const int cw = hp.nx - 1;
    const int chh = hp.ny - 1;
    const int words = (cw * chh + 31) / 32;
    S.allow_off[0] = 0;
    S.allow_words[0] = words;
    S.allow_bits.assign(static_cast<size_t>(words) * Fr, 0u);
    // the rows of each frame; rows ordered by frame (as the builders emit
    // them) index themselves and their frame ranges come from binary
    // searches, other rows are counting-sorted
    const bool by_frame = std::is_sorted(hp.pt_frame.begin(), hp.pt_frame.end());
    std::vector<int> fptr(static_cast<size_t>(Fr) + 1, 0);
    if (by_frame) {
      for (int f = 0; f <= Fr; ++f) {
        fptr[static_cast<size_t>(f)] = static_cast<int>(
            std::lower_bound(hp.pt_frame.begin(), hp.pt_frame.end(), f) - hp.pt_frame.begin());
      }
    } else {
      for (const int32_t f : hp.pt_frame) {
        ++fptr[static_cast<size_t>(f) + 1];
      }
      for (int f = 0; f < Fr; ++f) {
        fptr[static_cast<size_t>(f) + 1] += fptr[static_cast<size_t>(f)];
      }
    }
    std::vector<int> fpts(by_frame ? 0 : hp.pt_frame.size());
    if (!by_frame) {
      std::vector<int> fill(fptr.begin(), fptr.end() - 1);
      for (size_t q = 0; q < hp.pt_frame.size(); ++q) {
        fpts[static_cast<size_t>(fill[static_cast<size_t>(hp.pt_frame[q])]++)] = static_cast<int>(q);
      }
    }
    const double dxg = hp.dx();
    const double dyg = hp.dy();
    // 64-bit words per bitmap row, wide enough for a row of nodes (cw + 1)
    const int rw = (hp.nx + 63) / 64;
    std::vector<uint64_t> row_mask(static_cast<size_t>(rw), 0);
    for (int w = 0; w < cw; ++w) {
      row_mask[static_cast<size_t>(w >> 6)] |= uint64_t{1} << (w & 63);
    }
    auto frame_work = [&](int f0, int f1) {
      const size_t cells = static_cast<size_t>(rw) * static_cast<size_t>(std::max(chh, 0));
      std::vector<uint64_t> occ(cells);
      std::vector<uint64_t> horiz(cells);
      std::vector<uint64_t> allowed(cells);
      std::vector<uint64_t> tmp(static_cast<size_t>(rw));
      std::vector<uint64_t> nodes(static_cast<size_t>(rw));
      for (int f = std::max(f0, 1); f < f1; ++f) {
        const double* pose = &state[3 * static_cast<size_t>(f)];
        const double c = std::cos(pose[2]);
        const double sn = std::sin(pose[2]);
        std::fill(occ.begin(), occ.end(), uint64_t{0});
        for (int q = fptr[static_cast<size_t>(f)]; q < fptr[static_cast<size_t>(f) + 1]; ++q) {
          const size_t pt = static_cast<size_t>(by_frame ? q : fpts[static_cast<size_t>(q)]);
          const double px = hp.pt_xy[2 * pt];
          const double py = hp.pt_xy[2 * pt + 1];
          const double gx = (c * px + (-sn) * py) + pose[0];
          const double gy = (sn * px + c * py) + pose[1];
          const double fx = (gx - hp.min_x) / dxg;
          const double fy = (gy - hp.min_y) / dyg;
          if (!(fx >= -margin) || !(fy >= -margin) || !(fx <= hp.nx - 1 + margin) || !(fy <= hp.ny - 1 + margin)) {
            continue;
          }
          // clamp(floor(f), 0, cells - 1) for the bounded f above: truncation
          // equals floor for f >= 0, and every f < 0 maps to cell 0
          const int w = fx > 0.0 ? std::min(static_cast<int>(fx), cw - 1) : 0;
          const int h = fy > 0.0 ? std::min(static_cast<int>(fy), chh - 1) : 0;
          occ[static_cast<size_t>(h) * rw + static_cast<size_t>(w >> 6)] |= uint64_t{1} << (w & 63);
        }
        // horizontal dilation: `margin` passes of a one-cell shift both ways;
        // bits past the last cell only regenerate cells already reached
        for (int h = 0; h < chh; ++h) {
          uint64_t* row = &horiz[static_cast<size_t>(h) * rw];
          std::copy(&occ[static_cast<size_t>(h) * rw], &occ[static_cast<size_t>(h) * rw] + rw, row);
          for (int pass = 0; pass < margin; ++pass) {
            for (int k = 0; k < rw; ++k) {
              const uint64_t up = (row[k] << 1) | (k > 0 ? row[k - 1] >> 63 : 0);
              const uint64_t down = (row[k] >> 1) | (k + 1 < rw ? row[k + 1] << 63 : 0);
              tmp[static_cast<size_t>(k)] = row[k] | up | down;
            }
            std::copy(tmp.begin(), tmp.end(), row);
          }
          for (int k = 0; k < rw; ++k) {
            row[k] &= row_mask[static_cast<size_t>(k)];
          }
        }
        // vertical dilation, clipped to the grid
        uint32_t* allow = S.allow_bits.data() + static_cast<size_t>(f) * words;
        for (int h = 0; h < chh; ++h) {
          uint64_t* row = &allowed[static_cast<size_t>(h) * rw];
          std::fill(row, row + rw, uint64_t{0});
          for (int hh = std::max(0, h - margin); hh <= std::min(chh - 1, h + margin); ++hh) {
            const uint64_t* src = &horiz[static_cast<size_t>(hh) * rw];
            for (int k = 0; k < rw; ++k) {
              row[k] |= src[k];
            }
          }
          for (int k = 0; k < rw; ++k) {
            for (uint64_t bits = row[k]; bits != 0; bits &= bits - 1) {
              const int d = h * cw + k * 64 + __builtin_ctzll(bits);
              allow[d >> 5] |= 1u << (d & 31);
            }
          }
        }
        // active corner nodes of the allowed cells, in node order (active
        // columns ascend with the node)
        std::vector<int32_t>& cols = frame_cols[static_cast<size_t>(f)];
        cols.clear();
        for (int y = 0; y < hp.ny; ++y) {
          std::fill(nodes.begin(), nodes.end(), uint64_t{0});
          for (const int h : {y - 1, y}) {
            if (h < 0 || h >= chh) {
              continue;
            }
            const uint64_t* a = &allowed[static_cast<size_t>(h) * rw];
            for (int k = 0; k < rw; ++k) {
              nodes[static_cast<size_t>(k)] |= a[k] | (a[k] << 1) | (k > 0 ? a[k - 1] >> 63 : 0);
            }
          }
          for (int k = 0; k < rw; ++k) {
            for (uint64_t bits = nodes[static_cast<size_t>(k)]; bits != 0; bits &= bits - 1) {
              const int x = k * 64 + __builtin_ctzll(bits);
              const int col = hp.node_to_active[static_cast<size_t>(y) * hp.nx + x];
              if (col >= 0) {
                cols.push_back(col);
              }
            }
          }
        }
      }
    };
    ParallelRanges(threads, Fr, 4, [&](int64_t f0, int64_t f1) {
      frame_work(static_cast<int>(f0), static_cast<int>(f1));
    });
  }
  // frame-major index of the coupling entries
  S.fmp_ptr.assign(static_cast<size_t>(Fr) + 1, 0);
  for (int f = 0; f < Fr; ++f) {
    S.fmp_ptr[static_cast<size_t>(f) + 1] =
        S.fmp_ptr[static_cast<size_t>(f)] + static_cast<int64_t>(frame_cols[static_cast<size_t>(f)].size());
  }
  const int64_t entries = Fr > 0 ? S.fmp_ptr[static_cast<size_t>(Fr)] : 0;
  // node-major CSR (nf_ptr, nf): the frames of each active column, ascending.
  // The frame lists ascend, so a thread owning a range of columns finds its
  // part of every list by binary search.
  std::vector<int64_t> nf_ptr(static_cast<size_t>(A) + 1, 0);
  FillVector<int32_t> nf(static_cast<size_t>(entries));
  S.fmp_col.resize(static_cast<size_t>(entries));
  const int csr_threads = entries > (int64_t{1} << 14) ? threads : 1;
  auto frame_part = [&](int f, int64_t c0, int64_t c1) {
    const std::vector<int32_t>& cols = frame_cols[static_cast<size_t>(f)];
    const auto lo = std::lower_bound(cols.begin(), cols.end(), static_cast<int32_t>(c0));
    const auto hi = std::lower_bound(lo, cols.end(), static_cast<int32_t>(c1));
    return std::make_pair(lo, hi);
  };
  ParallelRanges(csr_threads, A, 256, [&](int64_t c0, int64_t c1) {
    for (int f = 1; f < Fr; ++f) {
      const auto [lo, hi] = frame_part(f, c0, c1);
      for (auto it = lo; it != hi; ++it) {
        ++nf_ptr[static_cast<size_t>(*it) + 1];
      }
    }
  });
  for (int c = 0; c < A; ++c) {
    nf_ptr[static_cast<size_t>(c) + 1] += nf_ptr[static_cast<size_t>(c)];
  }
  // emap[j]: the node-major entry of frame-major entry j (each thread writes
  // contiguous runs of every frame's list, not one entry per frame per node)
  FillVector<int64_t> emap(static_cast<size_t>(entries));
  ParallelRanges(csr_threads, A, 256, [&](int64_t c0, int64_t c1) {
    std::vector<int64_t> fill(nf_ptr.begin() + c0, nf_ptr.begin() + c1);
    for (int f = 1; f < Fr; ++f) {
      const auto [lo, hi] = frame_part(f, c0, c1);
      const auto begin = frame_cols[static_cast<size_t>(f)].begin();
      for (auto it = lo; it != hi; ++it) {
        const int64_t e = fill[static_cast<size_t>(*it - c0)]++;
        nf[static_cast<size_t>(e)] = f;
        emap[static_cast<size_t>(S.fmp_ptr[static_cast<size_t>(f)] + (it - begin))] = e;
      }
    }
  });
  ParallelRanges(csr_threads, Fr, 4, [&](int64_t f0, int64_t f1) {
    for (int64_t f = f0; f < f1; ++f) {
      const std::vector<int32_t>& cols = frame_cols[static_cast<size_t>(f)];
      int32_t* out = S.fmp_col.data() + S.fmp_ptr[static_cast<size_t>(f)];
      for (size_t k = 0; k < cols.size(); ++k) {
        out[k] = col_off + cols[k];
      }
    }
  });
  // pose pairs linked by odometry / relation rows
  std::vector<std::vector<int>> frame_links(static_cast<size_t>(Fr));
  for (int o = 0; o < hp.num_odom(); ++o) {
    const int fi = hp.odom_ij[2 * static_cast<size_t>(o)];
    const int fj = hp.odom_ij[2 * static_cast<size_t>(o) + 1];
    if (fi >= 1 && fj >= 1) {
      frame_links[static_cast<size_t>(std::min(fi, fj))].push_back(std::max(fi, fj));
    }
  }
  // 3. lower pattern in local permuted order
  auto lower = [&](int pc, std::vector<int>& out) {
    const int c = lperm[static_cast<size_t>(pc)];
    if (c < A) {
      const int node = hp.active_to_node[static_cast<size_t>(c)];
      const int w = node % hp.nx;
      const int h = node / hp.nx;
      for (int dh = -1; dh <= 1; ++dh) {
        for (int dw = -1; dw <= 1; ++dw) {
          const int ww = w + dw;
          const int hh = h + dh;
          if (ww < 0 || hh < 0 || ww >= hp.nx || hh >= hp.ny) {
            continue;
          }
          const int c2 = hp.node_to_active[static_cast<size_t>(hh) * hp.nx + ww];
          if (c2 >= 0 && lpinv[static_cast<size_t>(c2)] > pc) {
            out.push_back(lpinv[static_cast<size_t>(c2)]);
          }
        }
      }
      for (int64_t e = nf_ptr[static_cast<size_t>(c)]; e < nf_ptr[static_cast<size_t>(c) + 1]; ++e) {
        const int f = nf[static_cast<size_t>(e)];
        for (int a = 0; a < 3; ++a) {
          out.push_back(A + 3 * (f - 1) + a);
        }
      }
    } else {
      const int f = (c - A) / 3 + 1;
      for (int a = (c - A) % 3 + 1; a < 3; ++a) {
        out.push_back(A + 3 * (f - 1) + a);
      }
      for (const int g : frame_links[static_cast<size_t>(f)]) {
        for (int a = 0; a < 3; ++a) {
          out.push_back(A + 3 * (g - 1) + a);
        }
      }
    }
  };
  const LocalSym L = SupernodalSymbolic(np, lower, sn_begin, subtrees);
  AppendInstance(S, L, col_off, 0, height);
  // 4. assembly offsets for this instance: 9 stencil slots per node column
  // and one (node, frame) entry per coupled frame (stored node-major in
  // mp_off and frame-major in fmp_off), looked up in a map from the front's
  // rows to their positions. Supernodes are independent: each
  // writes the slots and entries of its own columns.
  for (int c = 0; c < n; ++c) {
    S.mp_ptr[static_cast<size_t>(c) + 1] = nf_ptr[static_cast<size_t>(std::min(c + 1, A))];
  }
  S.mp_off.resize(static_cast<size_t>(entries));
  S.fmp_off.resize(static_cast<size_t>(entries));
  const int Sn = static_cast<int>(S.sn.size());
  // tasks of at most kOffsetCols pivot columns of one supernode, taken from
  // a shared counter (wide separators hold most of the coupled entries)
  constexpr int kOffsetCols = 16;
  std::vector<std::pair<int32_t, int32_t>> offset_tasks;
  for (int s = 0; s < Sn; ++s) {
    const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    if (r.first_col >= col_off + A) {
      continue;  // the pose root holds no node columns
    }
    for (int j = 0; j < r.ncols; j += kOffsetCols) {
      offset_tasks.emplace_back(s, j);
    }
  }
  std::atomic<int64_t> next_offset_task{0};
  const int offset_parts = threads > 1 ? std::min<int>(static_cast<int>(offset_tasks.size()), threads) : 1;
  PoolRun(std::max(1, offset_parts), [&](int) {
    ColumnMap& pos = ThreadColumnMap();
    for (;;) {
      const int64_t task = next_offset_task.fetch_add(1);
      if (task >= static_cast<int64_t>(offset_tasks.size())) {
        break;
      }
      const int s = offset_tasks[static_cast<size_t>(task)].first;
      const int j0 = offset_tasks[static_cast<size_t>(task)].second;
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      const int32_t* rows = S.sn_rows.data() + r.rows_off;
      pos.Begin(static_cast<size_t>(col_off + n));
      for (int j = 0; j < r.ncols; ++j) {
        pos.Set(r.first_col + j, j);
      }
      for (int q = 0; q < r.nrows; ++q) {
        pos.Set(rows[q], r.ncols + q);
      }
      const int pc_end = r.first_col - col_off + std::min(r.ncols, j0 + kOffsetCols);
      for (int pc = r.first_col - col_off + j0; pc < pc_end; ++pc) {
        const int c = lperm[static_cast<size_t>(pc)];
        const int node = hp.active_to_node[static_cast<size_t>(c)];
        const int w = node % hp.nx;
        const int h = node / hp.nx;
        const int64_t col_base = r.front_off + static_cast<int64_t>(col_off + pc - r.first_col) * r.F;
        for (int dh = -1; dh <= 1; ++dh) {
          for (int dw = -1; dw <= 1; ++dw) {
            const int slot = (dh + 1) * 3 + (dw + 1);
            const int ww = w + dw;
            const int hh = h + dh;
            if (ww < 0 || hh < 0 || ww >= hp.nx || hh >= hp.ny) {
              continue;
            }
            const int c2 = hp.node_to_active[static_cast<size_t>(hh) * hp.nx + ww];
            if (c2 < 0) {
              continue;
            }
            const int pc2 = lpinv[static_cast<size_t>(c2)];
            if (pc2 < pc) {
              continue;  // stored in the neighbour's column
            }
            if (!pos.Has(col_off + pc2)) {
              Fail(SDFGPU_ERR_CUDA, "stencil row missing from a node's front");
            }
            S.mm_off[static_cast<size_t>(col_off + c) * 9 + static_cast<size_t>(slot)] = col_base + pos.Get(col_off + pc2);
          }
        }
        // pose rows lie below the pivot block of a grid supernode
        for (int64_t e = nf_ptr[static_cast<size_t>(c)]; e < nf_ptr[static_cast<size_t>(c) + 1]; ++e) {
          const int32_t target = col_off + A + 3 * (nf[static_cast<size_t>(e)] - 1);
          if (!pos.Has(target)) {
            Fail(SDFGPU_ERR_CUDA, "pose row missing from a node's front");
          }
          const int64_t off = col_base + pos.Get(target);
          S.mp_off[static_cast<size_t>(e)] = off;
        }
      }
    }
  });
  // the frame-major copy of the offsets: a gather, frame by frame
  ParallelRanges(csr_threads, entries, 1 << 14, [&](int64_t j0, int64_t j1) {
    for (int64_t j = j0; j < j1; ++j) {
      S.fmp_off[static_cast<size_t>(j)] = S.mp_off[static_cast<size_t>(emap[static_cast<size_t>(j)])];
    }
  });
  S.mp_frame = std::move(nf);
  // pose root
  if (Fr > 1) {
    const int s = S.col_owner[static_cast<size_t>(col_off + A)];
    const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    S.sn[static_cast<size_t>(s)].pose_root = 1;
    S.pp_base[0] = r.front_off;
    S.pp_ld[0] = r.F;
    S.pp_first[0] = col_off + A - r.first_col;
  }
  ComputeRel(S);
  return piece;
}

namespace {

/// Sizes a recycled array for n elements that are all written afterwards:
/// one too small is replaced (its contents are not copied) by one with half
/// again the room, so that the next growth fits.
template <typename Vec>
void Regrow(Vec& v, size_t n) {
  if (v.capacity() < n) {
    Vec fresh;
    fresh.reserve(n + n / 2);
    v.swap(fresh);
  }
  v.resize(n);
}

}  // namespace

Symbolic Concatenate(const std::vector<SymPiece>& pieces, const std::vector<InstanceLayout>& layout,
                     int panel_width, int tile, const Schedule& sched, Symbolic recycle) {
  Symbolic S;
  // every element of these arrays is written below; resizing a recycled
  // array initializes only growth
  S.perm = std::move(recycle.perm);
  S.pinv = std::move(recycle.pinv);
  S.col_owner = std::move(recycle.col_owner);
  S.sn = std::move(recycle.sn);
  S.sn_rows = std::move(recycle.sn_rows);
  S.sn_rel = std::move(recycle.sn_rel);
  S.child_list = std::move(recycle.child_list);
  S.mm_off = std::move(recycle.mm_off);
  S.mp_frame = std::move(recycle.mp_frame);
  S.mp_off = std::move(recycle.mp_off);
  S.allow_bits = std::move(recycle.allow_bits);
  S.fmp_col = std::move(recycle.fmp_col);
  S.fmp_off = std::move(recycle.fmp_off);
  S.small_pivots = sched.small_pivots;
  S.front_rows = sched.front_rows;
  S.panel_rows = sched.panel_rows;
  S.tc_min_rows = sched.tc_min_rows;
  const size_t I = pieces.size();
  // where each instance's part starts in every global array (a prefix pass),
  // then the parts are copied and rebased in parallel
  struct Base {
    int32_t sn;
    int64_t rows;
    int32_t child;
    int64_t front;
    int64_t upd;
    int64_t mp;
    int64_t allow;
    int64_t fmp;
  };
  std::vector<Base> base(I);
  Base t{0, 0, 0, 0, 0, 0, 0, 0};
  int n = 0;
  int frames = 0;
  S.allow_off.assign(I, 0);
  S.allow_words.assign(I, 0);
  S.pp_base.assign(I, -1);
  S.pp_ld.assign(I, 0);
  S.pp_first.assign(I, 0);
  for (size_t i = 0; i < I; ++i) {
    const Symbolic& L = pieces[i].s;
    base[i] = t;
    t.sn += static_cast<int32_t>(L.sn.size());
    t.rows += static_cast<int64_t>(L.sn_rows.size());
    t.child += static_cast<int32_t>(L.child_list.size());
    t.front += L.front_doubles;
    t.upd += L.update_doubles;
    t.mp += static_cast<int64_t>(L.mp_frame.size());
    t.allow += static_cast<int64_t>(L.allow_bits.size());
    t.fmp += static_cast<int64_t>(L.fmp_col.size());
    n += L.n;
    frames = std::max(frames, layout[i].frame_off + static_cast<int>(L.fmp_ptr.size()) - 1);
    S.total_flops += L.total_flops;
    S.allow_off[i] = base[i].allow;
    S.allow_words[i] = L.allow_words[0];
    S.pp_base[i] = L.pp_base[0] >= 0 ? L.pp_base[0] + base[i].front : -1;
    S.pp_ld[i] = L.pp_ld[0];
    S.pp_first[i] = L.pp_first[0];
  }
  S.n = n;
  S.front_doubles = t.front;
  S.update_doubles = t.upd;
  Regrow(S.perm, static_cast<size_t>(n));
  Regrow(S.pinv, static_cast<size_t>(n));
  Regrow(S.col_owner, static_cast<size_t>(n));
  Regrow(S.sn, static_cast<size_t>(t.sn));
  Regrow(S.sn_rows, static_cast<size_t>(t.rows));
  Regrow(S.sn_rel, static_cast<size_t>(t.rows));
  Regrow(S.child_list, static_cast<size_t>(t.child));
  Regrow(S.mm_off, static_cast<size_t>(n) * 9);
  S.mp_ptr.assign(static_cast<size_t>(n) + 1, 0);
  Regrow(S.mp_frame, static_cast<size_t>(t.mp));
  Regrow(S.mp_off, static_cast<size_t>(t.mp));
  Regrow(S.allow_bits, static_cast<size_t>(t.allow));
  S.fmp_ptr.assign(static_cast<size_t>(frames) + 1, 0);
  Regrow(S.fmp_col, static_cast<size_t>(t.fmp));
  Regrow(S.fmp_off, static_cast<size_t>(t.fmp));
  std::vector<int> height(static_cast<size_t>(t.sn));
  PoolRun(static_cast<int>(I), [&](int part) {
    const auto i = static_cast<size_t>(part);
    const Symbolic& L = pieces[i].s;
    const Base& B = base[i];
    const int col_off = layout[i].col_off;
    for (int k = 0; k < L.n; ++k) {
      S.perm[static_cast<size_t>(col_off + k)] = col_off + L.perm[static_cast<size_t>(k)];
      S.pinv[static_cast<size_t>(col_off + k)] = col_off + L.pinv[static_cast<size_t>(k)];
      S.col_owner[static_cast<size_t>(col_off + k)] = B.sn + L.col_owner[static_cast<size_t>(k)];
    }
    for (size_t q = 0; q < L.sn.size(); ++q) {
      SupernodeRec r = L.sn[q];
      r.front_off += B.front;
      r.rows_off += B.rows;
      r.upd_off += B.upd;
      r.first_col += col_off;
      r.child_begin += B.child;
      r.parent = r.parent >= 0 ? r.parent + B.sn : -1;
      r.instance = static_cast<int32_t>(i);
      S.sn[static_cast<size_t>(B.sn) + q] = r;
      height[static_cast<size_t>(B.sn) + q] = pieces[i].height[q];
    }
    for (size_t q = 0; q < L.sn_rows.size(); ++q) {
      S.sn_rows[static_cast<size_t>(B.rows) + q] = col_off + L.sn_rows[q];
    }
    std::copy(L.sn_rel.begin(), L.sn_rel.end(), S.sn_rel.begin() + B.rows);
    for (size_t q = 0; q < L.child_list.size(); ++q) {
      S.child_list[static_cast<size_t>(B.child) + q] = B.sn + L.child_list[q];
    }
    for (size_t q = 0; q < L.mm_off.size(); ++q) {
      const int64_t v = L.mm_off[q];
      S.mm_off[static_cast<size_t>(col_off) * 9 + q] = v >= 0 ? v + B.front : -1;
    }
    for (int k = 0; k < L.n; ++k) {
      S.mp_ptr[static_cast<size_t>(col_off + k) + 1] = B.mp + L.mp_ptr[static_cast<size_t>(k) + 1];
    }
    std::copy(L.mp_frame.begin(), L.mp_frame.end(), S.mp_frame.begin() + B.mp);
    for (size_t q = 0; q < L.mp_off.size(); ++q) {
      S.mp_off[static_cast<size_t>(B.mp) + q] = L.mp_off[q] + B.front;
    }
    std::copy(L.allow_bits.begin(), L.allow_bits.end(), S.allow_bits.begin() + B.allow);
    // instances are laid out in frame order, so their frame ranges are
    // disjoint
    const int fr = static_cast<int>(L.fmp_ptr.size()) - 1;
    for (int f = 0; f < fr; ++f) {
      S.fmp_ptr[static_cast<size_t>(layout[i].frame_off + f) + 1] = B.fmp + L.fmp_ptr[static_cast<size_t>(f) + 1];
    }
    for (size_t q = 0; q < L.fmp_col.size(); ++q) {
      S.fmp_col[static_cast<size_t>(B.fmp) + q] = col_off + L.fmp_col[q];
      S.fmp_off[static_cast<size_t>(B.fmp) + q] = L.fmp_off[q] + B.front;
    }
  });
  Finalize(S, height, panel_width, tile);
  return S;
}

Symbolic ConcatenateOne(SymPiece&& piece, int panel_width, int tile, const Schedule& sched) {
  // a lone piece is already numbered from column, frame and front 0
  Symbolic S = std::move(piece.s);
  const std::vector<int> height = std::move(piece.height);
  piece = SymPiece{};
  S.small_pivots = sched.small_pivots;
  S.front_rows = sched.front_rows;
  S.panel_rows = sched.panel_rows;
  S.tc_min_rows = sched.tc_min_rows;
  for (SupernodeRec& r : S.sn) {
    r.instance = 0;
  }
  Finalize(S, height, panel_width, tile);
  return S;
}

void Reschedule(Symbolic& S, const Schedule& sched) {
  S.small_pivots = sched.small_pivots;
  S.front_rows = sched.front_rows;
  S.panel_rows = sched.panel_rows;
  S.tc_min_rows = sched.tc_min_rows;
  S.ea_tasks.clear();
  S.ea_child.clear();
  S.panel_tasks.clear();
  S.update_tasks.clear();
  S.small_tasks.clear();
  S.ea_range.clear();
  S.ea_stage.clear();
  S.panel_range.clear();
  S.update_range.clear();
  S.small_range.clear();
  S.small_max_k.clear();
  S.small_threads.clear();
  S.level_panels.clear();
  S.panel_index_base.clear();
  const std::vector<int> height = S.height;
  Finalize(S, height, S.panel_width, S.tile);
}

Symbolic Analyze(const std::vector<HostProblem>& problems, const std::vector<InstanceLayout>& layout,
                 int panel_width, int tile) {
  std::vector<SymPiece> pieces(problems.size());
  AnalyzeInstances(problems, std::vector<int>(problems.size(), kDefaultMargin), pieces, nullptr);
  return Concatenate(pieces, layout, panel_width, tile);
}

void AnalyzeInstances(const std::vector<HostProblem>& problems, const std::vector<int>& margin,
                      std::vector<SymPiece>& pieces, const std::vector<int>* which) {
  std::vector<int> todo;
  if (which != nullptr) {
    todo = *which;
  } else {
    todo.resize(problems.size());
    std::iota(todo.begin(), todo.end(), 0);
  }
  // Many instances: one instance per part, each analysed on one thread.
  // Few: one after another, each on all threads.
  if (static_cast<int>(todo.size()) < PoolThreads()) {
    for (const int i : todo) {
      pieces[static_cast<size_t>(i)] =
          AnalyzeInstance(problems[static_cast<size_t>(i)], margin[static_cast<size_t>(i)], 0);
    }
    return;
  }
  PoolRun(static_cast<int>(todo.size()), [&](int q) {
    const int i = todo[static_cast<size_t>(q)];
    pieces[static_cast<size_t>(i)] =
        AnalyzeInstance(problems[static_cast<size_t>(i)], margin[static_cast<size_t>(i)], 1);
  });
}

Symbolic AnalyzeGeneral(int n, const int32_t* outer, const int32_t* inner, const std::vector<int32_t>& perm_in,
                        int panel_width, int tile, std::vector<int64_t>& value_offsets) {
  Symbolic S;
  S.n = n;
  S.perm.resize(static_cast<size_t>(n));
  if (perm_in.empty()) {
    std::iota(S.perm.begin(), S.perm.end(), 0);
  } else {
    S.perm = perm_in;
  }
  S.pinv.assign(static_cast<size_t>(n), -1);
  for (int k = 0; k < n; ++k) {
    const int old = S.perm[static_cast<size_t>(k)];
    if (old < 0 || old >= n || S.pinv[static_cast<size_t>(old)] != -1) {
      Fail(SDFGPU_ERR_INVALID_ARGUMENT, "perm is not a permutation");
    }
    S.pinv[static_cast<size_t>(old)] = k;
  }
  S.col_owner.assign(static_cast<size_t>(n), -1);
  // lower pattern by permuted column
  std::vector<std::vector<int>> low(static_cast<size_t>(n));
  for (int j = 0; j < n; ++j) {
    for (int p = outer[j]; p < outer[j + 1]; ++p) {
      const int i = inner[p];
      const int pi = S.pinv[static_cast<size_t>(i)];
      const int pj = S.pinv[static_cast<size_t>(j)];
      if (pi > pj) {
        low[static_cast<size_t>(pj)].push_back(pi);
      }
    }
  }
  // Fundamental-ish partition: consecutive columns j, j+1 share a supernode
  // while j+1 is j's only-child chain link (first below-diagonal row of j is
  // j+1), capped at 2 panels.
  std::vector<int> sn_begin{0};
  {
    int start = 0;
    for (int j = 0; j < n; ++j) {
      auto& v = low[static_cast<size_t>(j)];
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    for (int j = 0; j + 1 < n; ++j) {
      const auto& v = low[static_cast<size_t>(j)];
      const bool chain = !v.empty() && v.front() == j + 1;
      if (!chain || j + 1 - start >= 2 * panel_width) {
        sn_begin.push_back(j + 1);
        start = j + 1;
      }
    }
    if (n > 0) {
      sn_begin.push_back(n);
    }
  }
  auto lower = [&](int pc, std::vector<int>& out) {
    const auto& v = low[static_cast<size_t>(pc)];
    out.insert(out.end(), v.begin(), v.end());
  };
  const LocalSym L = SupernodalSymbolic(n, lower, sn_begin);
  std::vector<int> height;
  AppendInstance(S, L, 0, 0, height);
  ComputeRel(S);
  value_offsets.assign(static_cast<size_t>(outer[n]), -1);
  for (int j = 0; j < n; ++j) {
    for (int p = outer[j]; p < outer[j + 1]; ++p) {
      const int pi = S.pinv[static_cast<size_t>(inner[p])];
      const int pj = S.pinv[static_cast<size_t>(j)];
      if (pi < pj) {
        continue;
      }
      const int s = S.col_owner[static_cast<size_t>(pj)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      value_offsets[static_cast<size_t>(p)] = r.front_off + static_cast<int64_t>(pj - r.first_col) * r.F +
                                              LocalIndex(r, S.sn_rows.data() + r.rows_off, pi);
    }
  }
  Finalize(S, height, panel_width, tile);
  return S;
}

}  // namespace sdfgpu
