// Internal host-side types of the sdfgpu library (not part of the C ABI).
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/sdfgpu.h"

namespace sdfgpu {

/// Exception carrying a C-ABI status code; converted at the boundary.
class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  [[nodiscard]] int code() const { return code_; }

 private:
  int code_;
};

[[noreturn]] inline void Fail(int code, const std::string& msg) { throw Error(code, msg); }

/// Allocator whose value-less construct() default-initializes: resizing a
/// vector of plain numbers leaves the new elements unwritten, so that the
/// threads that then fill a large array in parallel also take its first-touch
/// page faults (a serial resize of the coupling-offset arrays of a 910-pose
/// office spent 12 ms of a 27 ms analysis in page faults).
template <typename T>
struct UninitAllocator : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = UninitAllocator<U>;
  };
  UninitAllocator() = default;
  template <typename U>
  UninitAllocator(const UninitAllocator<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
};
/// A vector whose growth writes nothing: every element must be written
/// before it is read.
template <typename T>
using FillVector = std::vector<T, UninitAllocator<T>>;

/// One problem's spec arrays in host memory: the fields of sdf_slam::Problem
/// the LM path reads (src/problem/problem.hpp:104-142), flattened.
struct HostProblem {
  int nx{2};
  int ny{2};
  double min_x{0.0};
  double min_y{0.0};
  double max_x{1.0};
  double max_y{1.0};
  std::vector<double> map_values;
  std::vector<double> poses;  // 3 per frame
  std::vector<int32_t> pt_frame;
  std::vector<double> pt_xy;
  std::vector<double> pt_expected;
  std::vector<double> pt_sqrtw;
  std::vector<int32_t> eik_wh;
  std::vector<double> eik_n;
  std::vector<double> eik_sqrtw;
  std::vector<int32_t> odom_ij;
  std::vector<double> odom_meas;
  std::vector<double> odom_sqrtw;
  std::vector<int32_t> node_to_active;
  std::vector<int32_t> active_to_node;
  double huber_delta{0.0};
  bool smooth_gradient{true};
  double smooth_gradient_step{0.0};

  [[nodiscard]] int num_frames() const { return static_cast<int>(poses.size() / 3); }
  [[nodiscard]] int num_points() const { return static_cast<int>(pt_frame.size()); }
  [[nodiscard]] int num_eikonal() const { return static_cast<int>(eik_sqrtw.size()); }
  [[nodiscard]] int num_odom() const { return static_cast<int>(odom_sqrtw.size()); }
  [[nodiscard]] int num_active() const { return static_cast<int>(active_to_node.size()); }
  [[nodiscard]] int num_pose_params() const { return 3 * (num_frames() - 1); }
  [[nodiscard]] int num_params() const { return num_active() + num_pose_params(); }
  [[nodiscard]] int num_rows() const { return num_points() + num_eikonal() + 3 * num_odom(); }
  [[nodiscard]] double dx() const { return (max_x - min_x) / (nx - 1); }
  [[nodiscard]] double dy() const { return (max_y - min_y) / (ny - 1); }
};

/// Validates a C-ABI problem description and copies it (throws Error with
/// SDFGPU_ERR_INVALID_ARGUMENT).
HostProblem FromDesc(const sdfgpu_problem_desc& desc);

/// How BuildProblem computes a problem: device_stages runs the point rows,
/// active maps, normals and Eikonal specs as CUDA kernels (the same values);
/// pattern_only (host only) stops after what a symbolic analysis reads (no
/// normals, no Eikonal specs); without rows, the device stages leave the
/// point rows out of the result (the caller supplies them: they depend on
/// the scans alone).
struct BuildMode {
  bool device_stages{false};
  bool pattern_only{false};
  bool rows{true};
};

/// Problem::Problem (src/problem/problem.cpp:11-115).
HostProblem BuildProblem(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                         const double* map_values, int num_frames, const double* poses,
                         const int32_t* scan_offsets, const double* scan_xy,
                         const double* odometry, int num_odometry, int num_relations,
                         const int32_t* relation_ij, const double* relation_meas,
                         const double* relation_sqrt_weight, const sdfgpu_problem_options& options,
                         const BuildMode& mode = BuildMode{});

/// A bucket grid over a point set for exact k-nearest-neighbour search: the
/// bucket of a point is its clamped cell (floor((p - origin) / cell) per
/// axis, row-major over gx * gy); start holds gx * gy + 1 offsets into items,
/// the point indices bucket by bucket.
struct KnnBuckets {
  double ox{0.0};
  double oy{0.0};
  double cell{1.0};
  int gx{1};
  int gy{1};
  std::vector<int> start;
  std::vector<int> items;
};

/// The host part of the on-device normals (src/core/normals.cpp:102-220):
/// every scan point in world coordinates at its frame's pose (2 values per
/// point, frame by frame), the bucket grid over those world points (for the
/// per-node nearest point, and for the scan normals unless per_scan), and
/// with per_scan one grid per frame over its sensor-frame points. The
/// grids are the host builder's, so a device search over them finds the
/// host's neighbours in the host's order.
struct NormalGrids {
  std::vector<double> world;
  KnnBuckets world_grid;
  std::vector<KnnBuckets> frame_grids;
};
void PrepareNormalGrids(const HostProblem& hp, int num_frames, const int32_t* scan_offsets, const double* scan_xy,
                        bool per_scan, NormalGrids* out);

/// The device stages of BuildProblem (device_stages = true): the point specs
/// (scan rows, then hallucinated rows, frame by frame), the active-region
/// maps, the scan-point and per-node normals and the Eikonal spec list,
/// computed by CUDA kernels on the current device from the scans and the
/// poses, then copied into hp. Same values, bit for bit, as the host stages.
void DeviceBuildSpecs(HostProblem& hp, int num_frames, const int32_t* scan_offsets, const double* scan_xy,
                      const sdfgpu_problem_options& options, bool download_rows = true);

// -------------------------------------------------------------- writers --
// run_slam's output files and metrics (src/pipeline/runner.cpp:82-192).
void WritePoses(const char* path, const double* poses, int num_frames);
void WriteMap(const char* path, int nx, int ny, double min_x, double min_y, double max_x, double max_y,
              const double* values);
void WriteScanPoints(const char* path, int num_frames, const double* poses, const int32_t* offsets,
                     const double* xy);
void PointsOutsideMap(int nx, int ny, double min_x, double min_y, double max_x, double max_y, int num_frames,
                      const double* poses, const int32_t* offsets, const double* xy, int64_t* outside,
                      int64_t* total);
void EvaluateTrajectory(const double* est, const double* gt, int num_frames, double* metrics);
void WriteMetrics(const char* path, const sdfgpu_solve_result& result, const double* metrics);

// ------------------------------------------------------------- symbolic --

/// Per-supernode record uploaded to the device.
struct SupernodeRec {
  int64_t front_off;  // first double of the dense front (column major, ld = F)
  int64_t rows_off;   // first entry in the row / relative-index arrays
  int64_t upd_off;    // first entry of the forward-solve update vector
  int32_t first_col;  // global permuted column of the first pivot
  int32_t ncols;      // k: pivots
  int32_t nrows;      // m: rows below the pivot block
  int32_t F;          // k + m
  int32_t child_begin;
  int32_t child_count;
  int32_t parent;     // -1 for a root
  int32_t instance;
  int32_t pose_root;  // 1: the dense pose block of its instance
  int32_t upper_l11;  // 1: L of the pivot block is stored transposed in its upper triangle
  int32_t panel_base; // first of its ceil(ncols / 32) inverted diagonal blocks
  int64_t tc_pack;    // first packed operand row of its tensor-core Schur update (within its level), or -1
  int64_t dense_cnt;  // a tiled dense root: first of its tile counters, else -1
  int64_t dense_inv;  // a tiled dense root: first double of its diagonal-tile inverses
};

/// Task types of the one-launch solve.
enum SolveTask : int32_t {
  kTaskForward = 0,      // gather, pivot block solve, (narrow fronts) u = v_m - L21 y
  kTaskForwardRows = 1,  // u for one chunk of rows of a wide front
  kTaskRootGather = 2,   // right-hand side of a panel-split root
  kTaskRootForward = 3,  // one 32-row panel of a panel-split root, forward
  kTaskRootBackward = 4, // one 32-row panel of a panel-split root, backward
  kTaskBackwardRows = 5, // L21^T x_R over one chunk of rows of a wide front
  kTaskBackward = 6,     // z = x_k - L21^T x_R, pivot block back-substitution
};
/// Fronts with more than small_pivots pivots factor their pivot block in
/// outer blocks of kOuterPanels 32-column panels, one of two ways (the
/// schedule's panel_rows picks it): panel_rows > 0, panel by panel (KPanel,
/// panel_rows rows below per task), each panel updating the rest of its outer
/// block; panel_rows == 0, the whole outer block with its rows below at once
/// (KPanelBlock). Either way the finished outer block updates every later
/// pivot column with one rank-128 update. Update task codes (the task's
/// panel field): -2 - 2 p for panel p's update within its outer block,
/// -3 - 2 b for outer block b's update of the pivot columns past it, -1 a
/// front's Schur complement, p >= 0 panel p's update of every later pivot
/// column (the allocation-free dense solve's panel path).
constexpr int kOuterPanels = 4;
constexpr int32_t UpdateCodeInner(int panel) { return -2 - 2 * panel; }
constexpr int32_t UpdateCodeOuter(int block) { return -3 - 2 * block; }
/// Columns per task of the front clearing (one warp each).
constexpr int kZeroCols = 8;
/// Fronts with at least this many rows below the pivot block take the
/// tensor-core Schur update in a mixed solve unless the autotuner measured
/// the SIMT tiles faster (Schedule::tc_min_rows).
constexpr int kTcMinRowsDefault = 256;
/// Tile edge of the tiled dense-root factorization.
constexpr int kDenseTileCols = 64;
/// One task of the tiled factorization of a dense root: FACTOR (i == j ==
/// k), SOLVE (j == k < i) or UPDATE (k < j <= i), with its bottom level.
struct DenseTileTask {
  double prio;
  int32_t sn;
  int32_t i;
  int32_t j;
  int32_t k;
};

/// Appends the tasks of an n-column dense root's tiled LDL^T (kDenseTileCols
/// tiles) with their bottom levels: the longest path of task weights
/// (FACTOR 8, SOLVE 2, UPDATE 2) from the task to the end of the graph.
/// Sorted by it descending, every task follows the tasks it waits for.
void AppendDenseTileTasks(int32_t sn, int n, std::vector<DenseTileTask>* out);
/// The order blocks take the tasks in: bottom level descending (ties by k,
/// i, j, supernode).
void OrderDenseTileTasks(std::vector<DenseTileTask>* tasks);
/// Rows below an outer block that one block-factorization task takes.
constexpr int kBlockRows = 64;
constexpr int kSolveWideRows = 512;
constexpr int kSolveRowChunk = 256;
constexpr int kSolveRootSplit = 256;

/// A contiguous block of work items of one kernel launch in the level
/// schedule.
struct TaskRange {
  int64_t begin{0};
  int64_t count{0};
};

/// Supernodal multifrontal structure of the normal equations of all
/// instances of a handle (nested dissection of each grid, pose block last).
struct Symbolic {
  int n{0};                                  // total columns, all instances
  std::vector<int32_t> perm;                 // permuted -> natural (global)
  std::vector<int32_t> pinv;                 // natural -> permuted (global)
  std::vector<SupernodeRec> sn;
  std::vector<int32_t> sn_rows;              // concatenated R_s (global permuted rows)
  std::vector<int32_t> sn_rel;               // position of each R_s row in the parent front
  std::vector<int32_t> child_list;
  std::vector<int32_t> col_owner;            // permuted column -> supernode
  int64_t front_doubles{0};
  int64_t update_doubles{0};
  int num_levels{0};
  int panel_width{32};
  int tile{64};
  // Level schedule. For level L: supernodes level_sn[level_begin[L]..]. For
  // each (level, panel t) a range of panel tasks (supernode, row chunk) and of
  // update tasks (supernode, tile i, tile j); extend-add tasks per level.
  std::vector<int32_t> level_begin;
  std::vector<int32_t> level_sn;
  std::vector<int32_t> level_panels;         // max panel count per level
  std::vector<int32_t> ea_tasks;             // (sn, col_lo, col_hi, ea_child offset) quads
  std::vector<int32_t> ea_child;             // per task and child: update column range [begin, end)
  std::vector<TaskRange> ea_range;           // per level
  std::vector<int32_t> ea_stage;             // per level: values a task stages in shared memory
  std::vector<int32_t> panel_tasks;          // (sn, panel, row_begin) triples
  std::vector<TaskRange> panel_range;        // per (level, panel) flattened
  std::vector<int32_t> update_tasks;         // (sn, panel, ti, tj) quads
  std::vector<TaskRange> update_range;       // per (level, panel) flattened
  std::vector<int32_t> panel_index_base;     // level -> first (level,panel) slot
  // Schur complement tasks (update tasks with panel -1), per (level, sibling
  // slot): schur_range[schur_base[l] + slot]; a task adds its tile of the
  // front's Schur complement into the parent front
  std::vector<TaskRange> schur_range;
  std::vector<int32_t> schur_base;           // levels + 1 entries
  // Tensor-core Schur complements of a mixed solve's FP32 fronts with at
  // least kTcMinRows rows below the pivot block (their SIMT Schur tasks are
  // skipped then): per level, operand packing tasks (sn, row tile, K chunk)
  // and output tile tasks (sn, tile i, tile j), i >= j; the packed operand
  // buffer is reused level after level (tc_pack_rows rows of the widest).
  // Task list of the one-launch solve, in the order blocks take them: the
  // forward tasks of every supernode in level order, then the backward
  // tasks in reverse. (type, sn, part, 0) quads, SolveTask types. A front
  // with at least kSolveWideRows rows below its pivots splits its forward
  // update u = v_m - L21 y and its backward product L21^T x_R into chunks of
  // kSolveRowChunk rows; a front without rows below and with more than
  // small_pivots pivots (a dense pose root) solves its pivot block by
  // 32-row panels, one task per panel, each waiting for the panels before
  // it. solve_parts: per supernode, the forward and backward tasks whose
  // completion its dependents wait for; zpart_off: per supernode the first
  // double of its backward partial products (-1 when not split).
  std::vector<int32_t> solve_tasks;
  std::vector<int32_t> solve_parts;
  std::vector<int64_t> zpart_off;
  int64_t zpart_doubles{0};
  std::vector<int32_t> pack_tasks;
  std::vector<TaskRange> pack_range;
  std::vector<int32_t> tc_tasks;
  std::vector<TaskRange> tc_range;
  int64_t tc_pack_rows{0};
  // Dense pose roots (no rows below, more than small_pivots pivots) are
  // factored by one persistent launch per level over 64 x 64 tiles instead
  // of panels: (sn, i, j, k) task quads (FACTOR i == j == k, SOLVE j == k <
  // i, UPDATE k < j <= i) in descending bottom level, dense_range per level,
  // the tile counters (nt x nt per front) and the diagonal-tile inverses
  // (64 x 64 doubles per tile) they use.
  // (sn, first column) pairs of kZeroCols columns: the fronts' lower
  // triangles cleared before every assembly. The first zero_main pairs are
  // what an FP64 assembly needs; the rest are the trailing columns of the
  // leaf fronts (no child adds into them, and their Schur update reads them
  // as zero without loading them), cleared only for the tensor-core Schur
  // complement of a mixed solve, which accumulates into them in place.
  std::vector<int32_t> zero_tasks;
  int64_t zero_main{0};
  std::vector<int32_t> dense_tasks;
  std::vector<TaskRange> dense_range;
  int64_t dense_cnt_words{0};
  int64_t dense_inv_doubles{0};
  // fronts with at most small_pivots pivots: one factorization kernel per
  // level, tasks (sn, first row of the chunk below the pivot block, rows in
  // the chunk) with front_rows threads per block (rows per chunk shrink to
  // 64 or 32 on levels that would not fill the GPU); larger fronts: panel
  // tasks of panel_rows rows (0: whole outer blocks, KPanelBlock). The three
  // are the schedule an autotuner picks.
  int small_pivots{128};
  int front_rows{256};
  int panel_rows{128};
  // mixed solves: fronts with at least tc_min_rows rows below the pivot
  // block take the tensor-core Schur update (0: none does)
  int tc_min_rows{kTcMinRowsDefault};
  std::vector<int> height;                   // per supernode: height in the assembly tree
  // (sn, panel) of every 32-column diagonal block, in panel_base order: the
  // inverted unit triangles the solve multiplies by
  std::vector<int32_t> inv_tasks;
  std::vector<int32_t> small_tasks;
  std::vector<TaskRange> small_range;        // per level
  std::vector<int32_t> small_max_k;          // per level
  std::vector<int32_t> small_threads;        // per level: threads per single-kernel block
  // Assembly offsets of J^T J entries into the front buffer, indexed by the
  // global natural column of a node.
  std::vector<int64_t> mm_off;               // 9 stencil slots per column (-1: stored elsewhere)
  std::vector<int64_t> mp_ptr;               // per column + 1: range in mp_frame / mp_off
  FillVector<int32_t> mp_frame;             // coupled frame (instance-local, >= 1), ascending
  FillVector<int64_t> mp_off;                // offset of (pose var (frame, x), node column)
  // Cells each frame's points may occupy without leaving the pattern:
  // bitmap over the instance's cells, one row of words per frame.
  std::vector<uint32_t> allow_bits;
  std::vector<int64_t> allow_off;            // per instance: first word
  std::vector<int32_t> allow_words;          // per instance: words per frame
  std::vector<int64_t> pp_base;              // per instance: root front offset (pose block)
  std::vector<int32_t> pp_ld;                // per instance: root front leading dimension
  std::vector<int32_t> pp_first;             // per instance: local index of pose var 0 in the root front
  // Map-pose entries grouped by frame (global frames in a concatenation,
  // local frames >= 1 in a piece): node columns and offsets of (pose var 0, node).
  std::vector<int64_t> fmp_ptr;
  FillVector<int32_t> fmp_col;
  FillVector<int64_t> fmp_off;
  int64_t total_flops{0};                    // dense front flops (useful)
};

/// Per-instance layout inside a handle's concatenated arrays.
struct InstanceLayout {
  int nx, ny;
  double min_x, min_y, dx, dy;
  int64_t node_off;   // first global node
  int64_t cell_off;   // first global cell ((nx-1)*(ny-1) per instance)
  int32_t col_off;    // first global (natural and permuted) column
  int32_t num_active;
  int32_t num_frames;
  int32_t frame_off;
  int64_t pt_off;
  int32_t num_points;
  int64_t eik_off;
  int32_t num_eik;
  int64_t odom_off;
  int32_t num_odom;
  double huber_delta;
  int32_t smooth_gradient;
  double smooth_gradient_step;
};

/// Symbolic analysis of one grid instance in instance-local numbering
/// (columns, supernodes, rows and front offsets start at 0; relative
/// extend-add indices filled); Concatenate places pieces one after another.
struct SymPiece {
  Symbolic s;
  std::vector<int> height;  // per supernode: height in the assembly tree
  int margin{0};            // coupling dilation (cells) the piece was built with
};

/// Coupling dilation (cells) of a first analysis. 7: a re-analysis holds the
/// GPU for the host analysis and the structure upload (about 30 ms for the
/// 910-pose office on B200, more for a batch, whose every instance's
/// structure is re-concatenated), and the first LM iterations from
/// odometry poses move points by several cells; the wider pattern makes the
/// office's factorization about 5 % slower per iteration than at 5 cells but
/// saves most re-analyses (64 uneven instances: 1 re-analysis in 20
/// iterations at 7 against 4 at 5 and 11 at 3). The same for one instance as
/// for a batch, so that a problem follows the same steps alone and in a
/// batch.
constexpr int kDefaultMargin = 7;
/// Default refine_tolerance of mixed solves (sdfgpu_solver_options).
constexpr double kDefaultRefineTol = 1e-13;
/// Growth of the dilation at each re-analysis, and its cap.
constexpr int kMarginStep = 2;
constexpr int kMaxMargin = 9;
/// A point farther than margin - kNearCells cells from the cells of its
/// pose's points at the analysed state (probed kNearCells cells around it)
/// marks its instance near the pattern's edge.
constexpr int kNearCells = 2;
/// Such an instance is re-analysed in the background (same margin, from the
/// state that marked it) once its pattern has held kSpeculateAfter
/// iterations (the first iterations from odometry poses move points by
/// several cells each; a pattern they leave is re-analysed at once, with a
/// wider margin), and the analysis replaces the pattern kSpeculationDelay
/// iterations after it started.
constexpr int64_t kSpeculateAfter = 20;
constexpr int64_t kSpeculationDelay = 6;

/// Analyses one instance at its current state on up to `threads` host
/// threads (0: all hardware threads); `poses` (3 per frame), when given,
/// replaces the problem's own poses as the state analysed.
SymPiece AnalyzeInstance(const HostProblem& hp, int margin, int threads = 0,
                         const std::vector<double>* poses = nullptr);

/// Analyses the instances listed in `which` (all when null) into
/// pieces[i] on the host pool: one instance per thread when there are at
/// least as many instances as threads, else one after another on all.
void AnalyzeInstances(const std::vector<HostProblem>& problems, const std::vector<int>& margin,
                      std::vector<SymPiece>& pieces, const std::vector<int>* which);

/// Values (doubles) of a parent front's column range that one extend-add
/// task stages in shared memory at most (96 KB).
constexpr int kEaStageDoubles = 12288;
/// Widest parent front whose extend-add is staged in shared memory; wider
/// fronts (whose children touch a small part of each column) are added in
/// place.
constexpr int kEaStageMaxF = 384;

/// Schedule parameters of the factorization (see Symbolic).
struct Schedule {
  int small_pivots{128};
  int front_rows{256};
  int panel_rows{128};
  int tc_min_rows{kTcMinRowsDefault};
};

/// Global structure (task lists, level schedule) of pieces laid out by
/// `layout`. `recycle` (a previous result, may be empty) lends its large
/// arrays, so that a re-concatenation writes into memory already mapped.
Symbolic Concatenate(const std::vector<SymPiece>& pieces, const std::vector<InstanceLayout>& layout,
                     int panel_width, int tile, const Schedule& sched = Schedule{}, Symbolic recycle = Symbolic{});

/// Concatenate for a single instance: takes the piece's arrays over instead
/// of copying them (the piece is left empty).
Symbolic ConcatenateOne(SymPiece&& piece, int panel_width, int tile, const Schedule& sched = Schedule{});

/// Rebuilds the level schedule and task lists of S for another schedule.
void Reschedule(Symbolic& S, const Schedule& sched);

/// Builds the supernodal symbolic factorization for a set of instances.
Symbolic Analyze(const std::vector<HostProblem>& problems, const std::vector<InstanceLayout>& layout,
                 int panel_width, int tile);

/// Symbolic analysis of a general symmetric pattern (factor-only API): full
/// CSC pattern, perm new->old (empty: natural order).
Symbolic AnalyzeGeneral(int n, const int32_t* outer, const int32_t* inner,
                        const std::vector<int32_t>& perm, int panel_width, int tile,
                        std::vector<int64_t>& value_offsets);

}  // namespace sdfgpu
