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
#include <cmath>
#include <functional>
#include <numeric>

#include "internal.h"

namespace sdfgpu {

namespace {

constexpr int kLeafNodes = 64;

struct LocalSym {
  std::vector<int> sn_begin;               // S + 1 boundaries (local permuted columns)
  std::vector<std::vector<int>> rows;      // R_s, sorted, local permuted
  std::vector<int> parent;
  std::vector<std::vector<int>> children;
};

/// Generic supernodal symbolic factorization over a partition of the
/// permuted columns. lower(col, out) appends the pattern rows > col.
LocalSym SupernodalSymbolic(int n, const std::function<void(int, std::vector<int>&)>& lower,
                            const std::vector<int>& sn_begin) {
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
  std::vector<int> mark(static_cast<size_t>(n), -1);
  std::vector<int> tmp;
  for (int s = 0; s < S; ++s) {
    const int b = sn_begin[static_cast<size_t>(s)];
    const int e = sn_begin[static_cast<size_t>(s) + 1];
    std::vector<int>& R = L.rows[static_cast<size_t>(s)];
    for (int c = b; c < e; ++c) {
      tmp.clear();
      lower(c, tmp);
      for (const int r : tmp) {
        if (r >= e && mark[static_cast<size_t>(r)] != s) {
          mark[static_cast<size_t>(r)] = s;
          R.push_back(r);
        }
      }
    }
    for (const int ch : L.children[static_cast<size_t>(s)]) {
      for (const int r : L.rows[static_cast<size_t>(ch)]) {
        if (r >= e && mark[static_cast<size_t>(r)] != s) {
          mark[static_cast<size_t>(r)] = s;
          R.push_back(r);
        }
      }
    }
    std::sort(R.begin(), R.end());
    if (!R.empty()) {
      const int p = owner[static_cast<size_t>(R.front())];
      L.parent[static_cast<size_t>(s)] = p;
      L.children[static_cast<size_t>(p)].push_back(s);
    }
  }
  return L;
}

/// Geometric nested dissection of the active nodes of a grid. Appends groups
/// of local natural columns in postorder (halves, then separator).
void Dissect(const HostProblem& hp, int w0, int w1, int h0, int h1, std::vector<std::vector<int>>& groups) {
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
    Dissect(hp, w0, mid, h0, h1, groups);
    Dissect(hp, mid + 1, w1, h0, h1, groups);
    for (int h = h0; h < h1; ++h) {
      const int c = hp.node_to_active[static_cast<size_t>(h) * hp.nx + mid];
      if (c >= 0) {
        sep.push_back(c);
      }
    }
  } else {
    const int mid = h0 + height / 2;
    Dissect(hp, w0, w1, h0, mid, groups);
    Dissect(hp, w0, w1, mid + 1, h1, groups);
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
void Finalize(Symbolic& S, const std::vector<int>& height, int panel_width, int tile) {
  S.panel_width = panel_width;
  S.tile = tile;
  const int Sn = static_cast<int>(S.sn.size());
  S.sn_rel.assign(S.sn_rows.size(), 0);
  for (int s = 0; s < Sn; ++s) {
    const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
    if (r.parent < 0) {
      continue;
    }
    const SupernodeRec& p = S.sn[static_cast<size_t>(r.parent)];
    for (int q = 0; q < r.nrows; ++q) {
      S.sn_rel[static_cast<size_t>(r.rows_off + q)] =
          LocalIndex(p, S.sn_rows.data() + p.rows_off, S.sn_rows[static_cast<size_t>(r.rows_off + q)]);
    }
  }
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
  constexpr int kPanelRows = 128;
  constexpr int kEaCols = 16;
  constexpr int kFrontRows = 256;
  const int small = S.small_pivots;
  S.level_panels.assign(static_cast<size_t>(levels), 0);
  S.panel_index_base.assign(static_cast<size_t>(levels) + 1, 0);
  S.small_range.assign(static_cast<size_t>(levels), {});
  S.small_max_k.assign(static_cast<size_t>(levels), 0);
  S.small_tasks.clear();
  for (int l = 0; l < levels; ++l) {
    int maxp = 0;
    S.small_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.small_tasks.size() / 2);
    for (int q = S.level_begin[static_cast<size_t>(l)]; q < S.level_begin[static_cast<size_t>(l) + 1]; ++q) {
      const int sid = S.level_sn[static_cast<size_t>(q)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(sid)];
      if (r.ncols <= small) {
        const int chunks = std::max(1, (r.nrows + kFrontRows - 1) / kFrontRows);
        for (int ch = 0; ch < chunks; ++ch) {
          S.small_tasks.push_back(sid);
          S.small_tasks.push_back(r.ncols + ch * kFrontRows);
        }
        S.small_max_k[static_cast<size_t>(l)] = std::max(S.small_max_k[static_cast<size_t>(l)], r.ncols);
        continue;
      }
      maxp = std::max(maxp, (r.ncols + B - 1) / B);
    }
    S.small_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.small_tasks.size() / 2) - S.small_range[static_cast<size_t>(l)].begin;
    S.level_panels[static_cast<size_t>(l)] = maxp;
    S.panel_index_base[static_cast<size_t>(l) + 1] = S.panel_index_base[static_cast<size_t>(l)] + maxp;
  }
  const int slots = S.panel_index_base.back();
  S.panel_range.assign(static_cast<size_t>(slots), {});
  S.update_range.assign(static_cast<size_t>(slots), {});
  S.ea_range.assign(static_cast<size_t>(levels), {});
  // Schur complement tasks (rank-k update of the trailing block) are stored
  // as update tasks with panel = -1 after the per-panel ones of each level;
  // update_range has one extra slot per level for them.
  std::vector<TaskRange> schur_range(static_cast<size_t>(levels));
  for (int l = 0; l < levels; ++l) {
    const int qb = S.level_begin[static_cast<size_t>(l)];
    const int qe = S.level_begin[static_cast<size_t>(l) + 1];
    // extend-add: parent columns in chunks, only for supernodes with children
    S.ea_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.ea_tasks.size() / 3);
    for (int q = qb; q < qe; ++q) {
      const int s = S.level_sn[static_cast<size_t>(q)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      if (r.child_count == 0) {
        continue;
      }
      for (int c = 0; c < r.F; c += kEaCols) {
        S.ea_tasks.push_back(s);
        S.ea_tasks.push_back(c);
        S.ea_tasks.push_back(std::min(r.F, c + kEaCols));
      }
    }
    S.ea_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.ea_tasks.size() / 3) - S.ea_range[static_cast<size_t>(l)].begin;
    for (int t = 0; t < S.level_panels[static_cast<size_t>(l)]; ++t) {
      const size_t slot = static_cast<size_t>(S.panel_index_base[static_cast<size_t>(l)] + t);
      S.panel_range[slot].begin = static_cast<int64_t>(S.panel_tasks.size() / 3);
      S.update_range[slot].begin = static_cast<int64_t>(S.update_tasks.size() / 4);
      for (int q = qb; q < qe; ++q) {
        const int s = S.level_sn[static_cast<size_t>(q)];
        const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
        const int c0 = t * B;
        if (c0 >= r.ncols || r.ncols <= small) {
          continue;
        }
        const int c1 = std::min(r.ncols, c0 + B);
        // panel tasks: chunk 0 also owns the diagonal block
        const int below = r.F - c1;
        const int chunks = std::max(1, (below + kPanelRows - 1) / kPanelRows);
        for (int ch = 0; ch < chunks; ++ch) {
          S.panel_tasks.push_back(s);
          S.panel_tasks.push_back(t);
          S.panel_tasks.push_back(c1 + ch * kPanelRows);
        }
        // update of the remaining pivot columns [c1, k) for rows [c1, F)
        if (c1 < r.ncols) {
          const int nr = r.F - c1;
          const int nc = r.ncols - c1;
          for (int tj = 0; tj * T < nc; ++tj) {
            for (int ti = 0; ti * T < nr; ++ti) {
              // lower part only: the tile must reach at or below the diagonal
              if ((ti + 1) * T - 1 < tj * T) {
                continue;
              }
              S.update_tasks.push_back(s);
              S.update_tasks.push_back(t);
              S.update_tasks.push_back(ti);
              S.update_tasks.push_back(tj);
            }
          }
        }
      }
      S.panel_range[slot].count = static_cast<int64_t>(S.panel_tasks.size() / 3) - S.panel_range[slot].begin;
      S.update_range[slot].count = static_cast<int64_t>(S.update_tasks.size() / 4) - S.update_range[slot].begin;
    }
    schur_range[static_cast<size_t>(l)].begin = static_cast<int64_t>(S.update_tasks.size() / 4);
    for (int q = qb; q < qe; ++q) {
      const int s = S.level_sn[static_cast<size_t>(q)];
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
    schur_range[static_cast<size_t>(l)].count =
        static_cast<int64_t>(S.update_tasks.size() / 4) - schur_range[static_cast<size_t>(l)].begin;
  }
  for (int l = 0; l < levels; ++l) {
    S.update_range.push_back(schur_range[static_cast<size_t>(l)]);
  }
}

}  // namespace

Symbolic Analyze(const std::vector<HostProblem>& problems, const std::vector<InstanceLayout>& layout,
                 int panel_width, int tile) {
  // The per-pose coupling sets are derived from the current cells of every
  // point row, dilated by the margin below (in cells).
  constexpr int kMargin = 2;
  Symbolic S;
  int n = 0;
  for (const HostProblem& hp : problems) {
    n += hp.num_params();
  }
  S.n = n;
  S.perm.assign(static_cast<size_t>(n), 0);
  S.pinv.assign(static_cast<size_t>(n), 0);
  S.col_owner.assign(static_cast<size_t>(n), -1);
  std::vector<int> height;
  S.mm_off.assign(static_cast<size_t>(n) * 9, -1);
  S.mp_ptr.assign(static_cast<size_t>(n) + 1, 0);
  S.mp_frame.clear();
  S.mp_off.clear();
  S.allow_off.assign(problems.size(), 0);
  S.allow_words.assign(problems.size(), 0);
  std::vector<std::vector<int>> mp_frames_by_col(static_cast<size_t>(n));
  std::vector<std::vector<int64_t>> mp_offs_by_col(static_cast<size_t>(n));
  S.pp_base.assign(problems.size(), -1);
  S.pp_ld.assign(problems.size(), 0);
  S.pp_first.assign(problems.size(), 0);
  for (size_t i = 0; i < problems.size(); ++i) {
    (void)layout;
    const HostProblem& hp = problems[i];
    const int A = hp.num_active();
    const int Fr = hp.num_frames();
    const int np = hp.num_params();
    const int col_off = layout[i].col_off;
    // 1. partition and permutation (local)
    std::vector<std::vector<int>> groups;
    Dissect(hp, 0, hp.nx, 0, hp.ny, groups);
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
    // 2. pose coupling: frames coupled to each active node (sorted)
    std::vector<std::vector<int>> node_frames(static_cast<size_t>(A));
    {
      const int cw = hp.nx - 1;
      const int chh = hp.ny - 1;
      const int words = (cw * chh + 31) / 32;
      S.allow_off[i] = static_cast<int64_t>(S.allow_bits.size());
      S.allow_words[i] = words;
      S.allow_bits.resize(S.allow_bits.size() + static_cast<size_t>(words) * Fr, 0u);
      uint32_t* allow = S.allow_bits.data() + S.allow_off[i];
      std::vector<int> stamp(static_cast<size_t>(cw) * chh, -1);
      std::vector<int> cells;
      const double dxg = hp.dx();
      const double dyg = hp.dy();
      int s = 0;
      for (int f = 0; f < Fr; ++f) {
        cells.clear();
        const double* pose = &hp.poses[3 * static_cast<size_t>(f)];
        const double c = std::cos(pose[2]);
        const double sn = std::sin(pose[2]);
        for (; s < hp.num_points() && hp.pt_frame[static_cast<size_t>(s)] == f; ++s) {
          const double px = hp.pt_xy[2 * static_cast<size_t>(s)];
          const double py = hp.pt_xy[2 * static_cast<size_t>(s) + 1];
          const double gx = (c * px + (-sn) * py) + pose[0];
          const double gy = (sn * px + c * py) + pose[1];
          const double fx = (gx - hp.min_x) / dxg;
          const double fy = (gy - hp.min_y) / dyg;
          if (!(fx >= -kMargin) || !(fy >= -kMargin) || !(fx <= hp.nx - 1 + kMargin) || !(fy <= hp.ny - 1 + kMargin)) {
            continue;
          }
          const int w = std::clamp(static_cast<int>(std::floor(fx)), 0, cw - 1);
          const int h = std::clamp(static_cast<int>(std::floor(fy)), 0, chh - 1);
          for (int hh = std::max(0, h - kMargin); hh <= std::min(chh - 1, h + kMargin); ++hh) {
            for (int ww = std::max(0, w - kMargin); ww <= std::min(cw - 1, w + kMargin); ++ww) {
              const int cell = hh * cw + ww;
              if (stamp[static_cast<size_t>(cell)] != f) {
                stamp[static_cast<size_t>(cell)] = f;
                cells.push_back(cell);
              }
            }
          }
        }
        if (f == 0) {
          continue;
        }
        for (const int cell : cells) {
          allow[static_cast<size_t>(f) * words + static_cast<size_t>(cell >> 5)] |= 1u << (cell & 31);
        }
        // nodes of the coupled cells
        for (const int cell : cells) {
          const int ww = cell % cw;
          const int hh = cell / cw;
          for (int q = 0; q < 4; ++q) {
            const int node = (hh + (q >> 1)) * hp.nx + ww + (q & 1);
            const int col = hp.node_to_active[static_cast<size_t>(node)];
            if (col >= 0) {
              auto& v = node_frames[static_cast<size_t>(col)];
              if (v.empty() || v.back() != f) {
                v.push_back(f);
              }
            }
          }
        }
      }
      // the point specs of a frame need not be contiguous in a caller's desc
      for (auto& v : node_frames) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
      }
    }
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
        for (const int f : node_frames[static_cast<size_t>(c)]) {
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
    const LocalSym L = SupernodalSymbolic(np, lower, sn_begin);
    const int S0 = static_cast<int>(S.sn.size());
    AppendInstance(S, L, col_off, static_cast<int>(i), height);
    // 4. assembly offsets for this instance
    for (int c = 0; c < A; ++c) {
      const int pc = lpinv[static_cast<size_t>(c)];
      const int s = S.col_owner[static_cast<size_t>(col_off + pc)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      const int32_t* rows = S.sn_rows.data() + r.rows_off;
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
          S.mm_off[static_cast<size_t>(col_off + c) * 9 + static_cast<size_t>(slot)] =
              col_base + LocalIndex(r, rows, col_off + pc2);
        }
      }
      for (const int f : node_frames[static_cast<size_t>(c)]) {
        mp_frames_by_col[static_cast<size_t>(col_off + c)].push_back(f);
        mp_offs_by_col[static_cast<size_t>(col_off + c)].push_back(
            col_base + LocalIndex(r, rows, col_off + A + 3 * (f - 1)));
      }
    }
    (void)S0;
    // pose root
    if (Fr > 1) {
      const int s = S.col_owner[static_cast<size_t>(col_off + A)];
      const SupernodeRec& r = S.sn[static_cast<size_t>(s)];
      S.pp_base[i] = r.front_off;
      S.pp_ld[i] = r.F;
      S.pp_first[i] = col_off + A - r.first_col;
    }
  }
  for (int c = 0; c < n; ++c) {
    S.mp_ptr[static_cast<size_t>(c) + 1] =
        S.mp_ptr[static_cast<size_t>(c)] + static_cast<int64_t>(mp_frames_by_col[static_cast<size_t>(c)].size());
    S.mp_frame.insert(S.mp_frame.end(), mp_frames_by_col[static_cast<size_t>(c)].begin(),
                      mp_frames_by_col[static_cast<size_t>(c)].end());
    S.mp_off.insert(S.mp_off.end(), mp_offs_by_col[static_cast<size_t>(c)].begin(),
                    mp_offs_by_col[static_cast<size_t>(c)].end());
  }
  Finalize(S, height, panel_width, tile);
  return S;
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
