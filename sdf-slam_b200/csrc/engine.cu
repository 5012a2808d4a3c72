// Engine: uploads problems, runs the symbolic analysis, and drives the LM
// iterations of SolveLm (src/solvers/lm_solver.cpp:201-434) on the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <future>
#include <map>
#include <utility>

#include "engine.h"
#include "host_pool.h"

namespace sdfgpu {

__global__ void KPointRows(DeviceView V);
__global__ void KEikonalRows(DeviceView V);
__global__ void KOdomRows(DeviceView V);
__global__ void KCellStart(const int32_t* keys, int64_t n, int64_t num_cells, int32_t* cell_start);
__global__ void KCellPass(DeviceView V, const int64_t* cells, int64_t count);
__global__ void KPoseFrames(DeviceView V);
__global__ void KFinalizeNormal(DeviceView V);
__global__ void KZeroFronts(DeviceView V, const int32_t* tasks);
__global__ void KPosePairs(DeviceView V);
__global__ void KBackup(DeviceView V, int dir, const int32_t* revert_mask);
__global__ void KApplyStep(DeviceView V);
__global__ void KCommitPoses(DeviceView V);
__global__ void KCostTerms(DeviceView V, double* terms);
__global__ void KStepTerms(DeviceView V, double* sq, double* pred);
__global__ void KSegmentPartial(const double* x, const int64_t* seg_begin, const int64_t* seg_end, double* partial);
__global__ void KSegmentFinal(const double* partial, int num_segments, double* out);
__global__ void KConvertFronts(DeviceView V, const int32_t* tasks);
__global__ void KNormalMatVecMap(DeviceView V, const double* x, double* y);
__global__ void KNormalMatVecPose(DeviceView V, const double* x, double* y);
__global__ void KRefineResidual(DeviceView V, const double* y, double* r);
__global__ void KAddCorrection(DeviceView V, const double* corr);
__global__ void KRefineReset(DeviceView V);
__global__ void KRefineCheck(DeviceView V);
void LaunchCellSort(const int32_t* pt_cell, int64_t n, int64_t num_cells, int32_t* keys_a, int32_t* vals_a,
                    int32_t* keys_b, int32_t* vals_b, int32_t* hist, cudaStream_t stream, bool* result_in_a);

void ThrowCuda(cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? SDFGPU_ERR_OUT_OF_MEMORY : SDFGPU_ERR_CUDA;
  Fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

inline unsigned Blocks(int64_t n, int threads) {
  return static_cast<unsigned>((n + threads - 1) / threads);
}

/// Position of permuted row r in the front index list of supernode s.
int FrontIndex(const Symbolic& S, const SupernodeRec& s, int r) {
  if (r < s.first_col + s.ncols) {
    return r - s.first_col;
  }
  const int32_t* rows = S.sn_rows.data() + s.rows_off;
  const int32_t* it = std::lower_bound(rows, rows + s.nrows, r);
  if (it == rows + s.nrows || *it != r) {
    return -1;
  }
  return s.ncols + static_cast<int>(it - rows);
}

}  // namespace

Engine::Engine(std::vector<HostProblem> problems) : host_(std::move(problems)) { Init(nullptr); }

Engine::Engine(HostProblem problem, SymPiece piece) {
  host_.push_back(std::move(problem));
  std::vector<SymPiece> pieces;
  pieces.push_back(std::move(piece));
  Init(&pieces);
}

Engine::Engine(std::vector<HostProblem> problems, std::vector<SymPiece> pieces) : host_(std::move(problems)) {
  if (pieces.size() != host_.size()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "one analysis per problem is required");
  }
  Init(&pieces);
}

void Engine::Init(std::vector<SymPiece>* pieces) {
  if (host_.empty()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "no problems");
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    Fail(SDFGPU_ERR_CUDA, "no CUDA device available (the GPU backend has no CPU fallback)");
  }
  CudaCheck(cudaGetDevice(&device_), "cudaGetDevice");
  CudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  for (auto& e : ev_) {
    CudaCheck(cudaEventCreate(&e), "cudaEventCreate");
  }
  for (auto& e : span_) {
    CudaCheck(cudaEventCreate(&e), "cudaEventCreate");
  }
  const char* ng = std::getenv("SDFGPU_NO_GRAPH");
  use_graph_ = !(ng != nullptr && ng[0] == '1');
  BuildLayout();
  h_active_.Alloc(host_.size());
  h_marq_.Alloc(host_.size());
  h_lam_.Alloc(host_.size());
  h_seg_.Alloc(5 * host_.size());
  h_status_.Alloc(host_.size());
  mixed_.assign(host_.size(), 0);  // plain FP64 until a solve asks otherwise
  refine_tol_.assign(host_.size(), kDefaultRefineTol);
  AnalyzeAndUpload(pieces, 0);
}

void Engine::AnalyzeAndUpload(std::vector<SymPiece>* pieces, int64_t keep_rows) {
  // the symbolic analysis (host only) runs while the problem is uploaded;
  // given analyses (one per instance) only need their global structure
  std::future<void> analysis = std::async(std::launch::async, [this, pieces] {
    if (pieces == nullptr) {
      AnalyzeHost();
      return;
    }
    margin_.clear();
    for (const SymPiece& p : *pieces) {
      margin_.push_back(p.margin);
    }
    pieces_ = std::move(*pieces);
    pending_.clear();
    sym_ = GlobalStructure();
  });
  try {
    UploadProblem(keep_rows);
  } catch (...) {
    analysis.wait();
    throw;
  }
  analysis.get();
  iters_.assign(host_.size(), 0);
  analysed_at_.assign(host_.size(), 0);
  near_.clear();
  UploadSymbolic();
}

bool Engine::CanReplace(const HostProblem& next) const {
  if (host_.size() != 1) {
    return false;
  }
  const HostProblem& cur = host_[0];
  return next.nx == cur.nx && next.ny == cur.ny && next.min_x == cur.min_x && next.min_y == cur.min_y &&
         next.max_x == cur.max_x && next.max_y == cur.max_y && next.node_to_active == cur.node_to_active;
}

void Engine::Replace(HostProblem next, SymPiece* piece, int64_t keep_rows) {
  if (!CanReplace(next)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "replacement problem has another grid or other active columns");
  }
  keep_rows = std::max<int64_t>(0, std::min<int64_t>({keep_rows, host_[0].num_points(), next.num_points()}));
  // no background analysis may still read the current problem
  DropSpeculations(nullptr);
  // nothing enqueued may still read the current problem's buffers
  CudaCheck(cudaStreamSynchronize(stream_), "replace sync");
  DropGraph();
  host_[0] = std::move(next);
  BuildLayout();
  if (piece == nullptr) {
    AnalyzeAndUpload(nullptr, keep_rows);
  } else {
    std::vector<SymPiece> pieces;
    pieces.push_back(std::move(*piece));
    AnalyzeAndUpload(&pieces, keep_rows);
  }
}

void Engine::DropGraph() {
  for (auto& g : graph_exec_) {
    if (g != nullptr) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  }
}

Engine::~Engine() {
  try {
    DropSpeculations(nullptr);
  } catch (...) {
  }
  DropGraph();
  if (stream_ != nullptr) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
  for (auto& e : ev_) {
    if (e != nullptr) {
      cudaEventDestroy(e);
    }
  }
  for (auto& e : span_) {
    if (e != nullptr) {
      cudaEventDestroy(e);
    }
  }
}

void Engine::BuildLayout() {
  layout_.clear();
  int64_t node = 0;
  int64_t cell = 0;
  int col = 0;
  int frame = 0;
  int64_t pt = 0;
  int64_t eik = 0;
  int64_t odom = 0;
  for (const HostProblem& hp : host_) {
    InstanceLayout L{};
    L.nx = hp.nx;
    L.ny = hp.ny;
    L.min_x = hp.min_x;
    L.min_y = hp.min_y;
    L.dx = hp.dx();
    L.dy = hp.dy();
    L.node_off = node;
    L.cell_off = cell;
    L.col_off = col;
    L.num_active = hp.num_active();
    L.num_frames = hp.num_frames();
    L.frame_off = frame;
    L.pt_off = pt;
    L.num_points = hp.num_points();
    L.eik_off = eik;
    L.num_eik = hp.num_eikonal();
    L.odom_off = odom;
    L.num_odom = hp.num_odom();
    L.huber_delta = hp.huber_delta;
    L.smooth_gradient = hp.smooth_gradient ? 1 : 0;
    L.smooth_gradient_step = hp.smooth_gradient_step;
    layout_.push_back(L);
    node += static_cast<int64_t>(hp.nx) * hp.ny;
    cell += static_cast<int64_t>(hp.nx - 1) * (hp.ny - 1);
    col += hp.num_params();
    frame += hp.num_frames();
    pt += hp.num_points();
    eik += hp.num_eikonal();
    odom += hp.num_odom();
  }
  if (pt > (int64_t{1} << 31) - 1 || col > (1 << 30)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "problem too large for 32-bit row / column indices");
  }
  total_nodes_ = node;
  total_cells_ = cell;
  n_ = col;
  total_frames_ = frame;
  total_points_ = pt;
  total_eik_ = eik;
  total_odom_ = odom;
}

void Engine::UploadProblem(int64_t keep_rows) {
  const size_t I = host_.size();
  // One instance: its point rows go up from its own arrays (rows before
  // keep_rows are on the device already) and only the frame index of the
  // rows is built here; several: every array is gathered first.
  const bool direct = I == 1;
  if (!direct) {
    keep_rows = 0;
  }
  std::vector<int32_t> node_col(static_cast<size_t>(total_nodes_), -1);
  std::vector<int32_t> col_node(static_cast<size_t>(n_), -1);
  std::vector<int32_t> col_inst(static_cast<size_t>(n_), 0);
  std::vector<int32_t> frame_inst(static_cast<size_t>(total_frames_), 0);
  std::vector<int32_t> frame_col(static_cast<size_t>(total_frames_), -1);
  const size_t gathered = direct ? 0 : static_cast<size_t>(total_points_);
  std::vector<int32_t> pt_frame(gathered);
  std::vector<double2> pt_xy(gathered);
  std::vector<double> pt_exp(gathered);
  std::vector<double> pt_sw(gathered);
  std::vector<int32_t> eik_node(static_cast<size_t>(total_eik_));
  std::vector<int32_t> eik_index(static_cast<size_t>(total_nodes_), -1);
  std::vector<double2> eik_n(static_cast<size_t>(total_eik_));
  std::vector<double> eik_sw(static_cast<size_t>(total_eik_));
  std::vector<int32_t> odom_fi(static_cast<size_t>(total_odom_));
  std::vector<int32_t> odom_fj(static_cast<size_t>(total_odom_));
  std::vector<double> odom_meas(3 * static_cast<size_t>(total_odom_));
  std::vector<double> odom_sw(static_cast<size_t>(total_odom_));
  std::vector<int64_t> frame_rows_ptr(static_cast<size_t>(total_frames_) + 1, 0);
  std::vector<int32_t> frame_rows(static_cast<size_t>(total_points_));
  std::vector<int64_t> frame_odom_ptr(static_cast<size_t>(total_frames_) + 1, 0);
  std::vector<int32_t> frame_odom(2 * static_cast<size_t>(total_odom_));
  std::vector<int32_t> pair_f;
  std::vector<int32_t> pair_g;
  std::vector<int64_t> pair_ptr{0};
  std::vector<int32_t> pair_spec;
  std::vector<double> map;
  std::vector<double> poses;
  for (size_t i = 0; i < I; ++i) {
    const HostProblem& hp = host_[i];
    const InstanceLayout& L = layout_[i];
    map.insert(map.end(), hp.map_values.begin(), hp.map_values.end());
    poses.insert(poses.end(), hp.poses.begin(), hp.poses.end());
    for (int a = 0; a < hp.num_active(); ++a) {
      const int64_t node = L.node_off + hp.active_to_node[static_cast<size_t>(a)];
      node_col[static_cast<size_t>(node)] = L.col_off + a;
      col_node[static_cast<size_t>(L.col_off + a)] = static_cast<int32_t>(node);
    }
    for (int c = 0; c < hp.num_params(); ++c) {
      col_inst[static_cast<size_t>(L.col_off + c)] = static_cast<int32_t>(i);
    }
    for (int f = 0; f < hp.num_frames(); ++f) {
      frame_inst[static_cast<size_t>(L.frame_off + f)] = static_cast<int32_t>(i);
      frame_col[static_cast<size_t>(L.frame_off + f)] = f >= 1 ? L.col_off + hp.num_active() + 3 * (f - 1) : -1;
    }
    if (direct) {
      // rows ordered by frame (as the builders emit them): the frame ranges
      // by binary search, else counted
      if (std::is_sorted(hp.pt_frame.begin(), hp.pt_frame.end())) {
        for (int f = 0; f < hp.num_frames(); ++f) {
          frame_rows_ptr[static_cast<size_t>(f) + 1] = static_cast<int64_t>(
              std::upper_bound(hp.pt_frame.begin(), hp.pt_frame.end(), f) -
              std::lower_bound(hp.pt_frame.begin(), hp.pt_frame.end(), f));
        }
      } else {
        for (const int32_t f : hp.pt_frame) {
          ++frame_rows_ptr[static_cast<size_t>(f) + 1];
        }
      }
    } else {
      for (int k = 0; k < hp.num_points(); ++k) {
        const size_t g = static_cast<size_t>(L.pt_off + k);
        pt_frame[g] = L.frame_off + hp.pt_frame[static_cast<size_t>(k)];
        pt_xy[g] = make_double2(hp.pt_xy[2 * static_cast<size_t>(k)], hp.pt_xy[2 * static_cast<size_t>(k) + 1]);
        pt_exp[g] = hp.pt_expected[static_cast<size_t>(k)];
        pt_sw[g] = hp.pt_sqrtw[static_cast<size_t>(k)];
        ++frame_rows_ptr[static_cast<size_t>(pt_frame[g]) + 1];
      }
    }
    for (int e = 0; e < hp.num_eikonal(); ++e) {
      const size_t g = static_cast<size_t>(L.eik_off + e);
      const int64_t node = L.node_off + static_cast<int64_t>(hp.eik_wh[2 * static_cast<size_t>(e) + 1]) * hp.nx +
                           hp.eik_wh[2 * static_cast<size_t>(e)];
      eik_node[g] = static_cast<int32_t>(node);
      eik_index[static_cast<size_t>(node)] = static_cast<int32_t>(g);
      eik_n[g] = make_double2(hp.eik_n[2 * static_cast<size_t>(e)], hp.eik_n[2 * static_cast<size_t>(e) + 1]);
      eik_sw[g] = hp.eik_sqrtw[static_cast<size_t>(e)];
    }
    std::map<std::pair<int, int>, std::vector<int32_t>> pairs;
    for (int o = 0; o < hp.num_odom(); ++o) {
      const size_t g = static_cast<size_t>(L.odom_off + o);
      const int fi = hp.odom_ij[2 * static_cast<size_t>(o)];
      const int fj = hp.odom_ij[2 * static_cast<size_t>(o) + 1];
      odom_fi[g] = L.frame_off + fi;
      odom_fj[g] = L.frame_off + fj;
      for (int q = 0; q < 3; ++q) {
        odom_meas[3 * g + static_cast<size_t>(q)] = hp.odom_meas[3 * static_cast<size_t>(o) + static_cast<size_t>(q)];
      }
      odom_sw[g] = hp.odom_sqrtw[static_cast<size_t>(o)];
      ++frame_odom_ptr[static_cast<size_t>(odom_fi[g]) + 1];
      ++frame_odom_ptr[static_cast<size_t>(odom_fj[g]) + 1];
      if (fi >= 1 && fj >= 1) {
        const int lo = std::min(fi, fj);
        const int hi = std::max(fi, fj);
        pairs[{lo, hi}].push_back(static_cast<int32_t>(2 * g + (fi > fj ? 1 : 0)));
      }
    }
    for (const auto& kv : pairs) {
      pair_f.push_back(L.frame_off + kv.first.first);
      pair_g.push_back(L.frame_off + kv.first.second);
      pair_spec.insert(pair_spec.end(), kv.second.begin(), kv.second.end());
      pair_ptr.push_back(static_cast<int64_t>(pair_spec.size()));
    }
  }
  for (int f = 0; f < total_frames_; ++f) {
    frame_rows_ptr[static_cast<size_t>(f) + 1] += frame_rows_ptr[static_cast<size_t>(f)];
    frame_odom_ptr[static_cast<size_t>(f) + 1] += frame_odom_ptr[static_cast<size_t>(f)];
  }
  const std::vector<int32_t>& row_frame = direct ? host_[0].pt_frame : pt_frame;
  // rows ordered by frame (as the builders emit them) make the frame index
  // the identity, of which a kept prefix is on the device already
  const bool identity = std::is_sorted(row_frame.begin(), row_frame.end());
  {
    if (identity) {
      for (int64_t k = frame_rows_identity_ ? keep_rows : 0; k < total_points_; ++k) {
        frame_rows[static_cast<size_t>(k)] = static_cast<int32_t>(k);
      }
    } else {
      std::vector<int64_t> fill(frame_rows_ptr.begin(), frame_rows_ptr.end() - 1);
      for (int64_t k = 0; k < total_points_; ++k) {
        frame_rows[static_cast<size_t>(fill[static_cast<size_t>(row_frame[static_cast<size_t>(k)])]++)] =
            static_cast<int32_t>(k);
      }
    }
    std::vector<int64_t> ofill(frame_odom_ptr.begin(), frame_odom_ptr.end() - 1);
    for (int64_t o = 0; o < total_odom_; ++o) {
      frame_odom[static_cast<size_t>(ofill[static_cast<size_t>(odom_fi[static_cast<size_t>(o)])]++)] =
          static_cast<int32_t>(2 * o);
      frame_odom[static_cast<size_t>(ofill[static_cast<size_t>(odom_fj[static_cast<size_t>(o)])]++)] =
          static_cast<int32_t>(2 * o + 1);
    }
  }
  num_pairs_ = static_cast<int>(pair_f.size());
  cudaStream_t s = stream_;
  node_col_.Upload(node_col, s);
  col_node_.Upload(col_node, s);
  col_inst_.Upload(col_inst, s);
  frame_inst_.Upload(frame_inst, s);
  frame_inst_host_ = frame_inst;
  frame_col_.Upload(frame_col, s);
  if (direct) {
    const HostProblem& hp = host_[0];
    const auto rows = static_cast<size_t>(total_points_);
    const auto keep = static_cast<size_t>(keep_rows);
    static_assert(sizeof(double2) == 2 * sizeof(double));
    pt_frame_.UploadKeep(hp.pt_frame.data(), rows, keep, s);
    pt_xy_.UploadKeep(reinterpret_cast<const double2*>(hp.pt_xy.data()), rows, keep, s);
    pt_exp_.UploadKeep(hp.pt_expected.data(), rows, keep, s);
    pt_sw_.UploadKeep(hp.pt_sqrtw.data(), rows, keep, s);
  } else {
    pt_frame_.Upload(pt_frame, s);
    pt_xy_.Upload(pt_xy, s);
    pt_exp_.Upload(pt_exp, s);
    pt_sw_.Upload(pt_sw, s);
  }
  eik_node_.Upload(eik_node, s);
  eik_index_.Upload(eik_index, s);
  eik_n_.Upload(eik_n, s);
  eik_sw_.Upload(eik_sw, s);
  odom_fi_.Upload(odom_fi, s);
  odom_fj_.Upload(odom_fj, s);
  odom_meas_.Upload(odom_meas, s);
  odom_sw_.Upload(odom_sw, s);
  frame_rows_ptr_.Upload(frame_rows_ptr, s);
  frame_rows_.UploadKeep(frame_rows.data(), frame_rows.size(),
                         identity && frame_rows_identity_ ? static_cast<size_t>(keep_rows) : 0, s);
  frame_rows_identity_ = identity;
  frame_odom_ptr_.Upload(frame_odom_ptr, s);
  frame_odom_.Upload(frame_odom, s);
  pair_f_.Upload(pair_f, s);
  pair_g_.Upload(pair_g, s);
  pair_ptr_.Upload(pair_ptr, s);
  pair_spec_.Upload(pair_spec, s);
  map_.Upload(map, s);
  poses_.Upload(poses, s);
  map_backup_.Alloc(map.size());
  poses_backup_.Alloc(poses.size());
  {
    const size_t F = static_cast<size_t>(total_frames_);
    pose_cs_.Alloc(F);
    pose_cs_backup_.Alloc(F);
    theta_pre_.Alloc(F);
    theta_upd_.Alloc(F);
    theta_out_.Alloc(4 * F);
    h_theta_pre_.Alloc(F);
    h_theta_upd_.Alloc(F);
    h_theta_out_.Alloc(4 * F);
    UploadPoseTrig(poses.data(), 0, total_frames_);
  }
  pt_rec_.Alloc(static_cast<size_t>(total_points_) * kPointRec);
  pt_poff_.Alloc(static_cast<size_t>(total_points_) * 4);
  pt_cell_.Alloc(static_cast<size_t>(total_points_));
  eik_rec_.Alloc(static_cast<size_t>(total_eik_) * kEikRec);
  odom_rec_.Alloc(static_cast<size_t>(total_odom_) * kOdomRec);
  cell_start_.Alloc(static_cast<size_t>(total_cells_) + 2);
  {
    // the cells of each colour class (cx % 2, cy % 2) = (pass & 1, pass >> 1)
    std::vector<int64_t> cells;
    cells.reserve(static_cast<size_t>(total_cells_));
    for (int pass = 0; pass < 4; ++pass) {
      pass_begin_[pass] = static_cast<int64_t>(cells.size());
      for (const InstanceLayout& L : layout_) {
        const int cw = L.nx - 1;
        const int ch = L.ny - 1;
        for (int cy = pass >> 1; cy < ch; cy += 2) {
          for (int cx = pass & 1; cx < cw; cx += 2) {
            cells.push_back(L.cell_off + static_cast<int64_t>(cy) * cw + cx);
          }
        }
      }
    }
    pass_begin_[4] = static_cast<int64_t>(cells.size());
    pass_cells_.Upload(cells, stream_);
  }
  sort_keys_a_.Alloc(static_cast<size_t>(total_points_));
  sort_vals_a_.Alloc(static_cast<size_t>(total_points_));
  sort_keys_b_.Alloc(static_cast<size_t>(total_points_));
  sort_vals_b_.Alloc(static_cast<size_t>(total_points_));
  sort_hist_.Alloc(256 * static_cast<size_t>((total_points_ + 2047) / 2048 + 1));
  rhs_.Alloc(static_cast<size_t>(n_));
  step_.Alloc(static_cast<size_t>(n_));
  xs_.Alloc(static_cast<size_t>(n_));
  dvec_.Alloc(static_cast<size_t>(n_));
  lam_.Alloc(I);
  marq_.Alloc(I);
  status_.Alloc(I);
  active_.Alloc(I);
  revert_.Alloc(I);
  terms_.Alloc(static_cast<size_t>(total_points_ + total_eik_ + total_odom_));
  sq_terms_.Alloc(static_cast<size_t>(n_));
  pred_terms_.Alloc(static_cast<size_t>(n_));
  seg_out_.Alloc(5 * I);
  seg_partial_.Alloc(32 * 3 * I);
  std::vector<int64_t> sb;
  std::vector<int64_t> se;
  for (size_t i = 0; i < I; ++i) {
    const InstanceLayout& L = layout_[i];
    sb.push_back(L.pt_off);
    se.push_back(L.pt_off + L.num_points);
    sb.push_back(total_points_ + L.eik_off);
    se.push_back(total_points_ + L.eik_off + L.num_eik);
    sb.push_back(total_points_ + total_eik_ + L.odom_off);
    se.push_back(total_points_ + total_eik_ + L.odom_off + L.num_odom);
  }
  seg_begin_.Upload(sb, s);
  seg_end_.Upload(se, s);
  std::vector<int64_t> ssb;
  std::vector<int64_t> sse;
  for (size_t i = 0; i < I; ++i) {
    ssb.push_back(layout_[i].col_off);
    sse.push_back(layout_[i].col_off + host_[i].num_params());
  }
  step_seg_begin_.Upload(ssb, s);
  step_seg_end_.Upload(sse, s);
  std::vector<int32_t> ones(I, 1);
  active_.Upload(ones, s);
  std::vector<int32_t> zeros(I, 0);
  status_.Upload(zeros, s);
  marq_.Upload(zeros, s);
  std::vector<double> lam(I, 1.0);
  lam_.Upload(lam, s);
  CudaCheck(cudaStreamSynchronize(s), "upload");
}

void Engine::AnalyzeHost() {
  margin_.assign(host_.size(), kDefaultMargin);
  pieces_.assign(host_.size(), SymPiece{});
  pending_.clear();
  AnalyzeInstances(host_, margin_, pieces_, nullptr);
  sym_ = GlobalStructure();
}

Symbolic Engine::GlobalStructure() {
  // a single instance's piece is re-analysed whenever its structure changes,
  // so it is not kept
  if (pieces_.size() == 1) {
    return ConcatenateOne(std::move(pieces_[0]), 32, 64, sched_);
  }
  return Concatenate(pieces_, layout_, 32, 64, sched_, std::move(sym_));
}

void Engine::UploadSymbolic() {
  DropGraph();
  // the previous structure may still be read by enqueued work
  CudaCheck(cudaStreamSynchronize(stream_), "analysis sync");
  cudaStream_t s = stream_;
  perm_.Upload(sym_.perm, s);
  pinv_.Upload(sym_.pinv, s);
  sn_.Upload(sym_.sn, s);
  sn_rows_.Upload(sym_.sn_rows, s);
  sn_rel_.Upload(sym_.sn_rel, s);
  child_list_.Upload(sym_.child_list, s);
  level_sn_.Upload(sym_.level_sn, s);
  mm_off_.Upload(sym_.mm_off, s);
  mp_ptr_.Upload(sym_.mp_ptr, s);
  mp_off_.Upload(sym_.mp_off, s);
  mp_frame_.Upload(sym_.mp_frame, s);
  allow_bits_.Upload(sym_.allow_bits, s);
  ea_tasks_.Upload(sym_.ea_tasks, s);
  ea_child_.Upload(sym_.ea_child, s);
  panel_tasks_.Upload(sym_.panel_tasks, s);
  update_tasks_.Upload(sym_.update_tasks, s);
  small_tasks_.Upload(sym_.small_tasks, s);
  pack_tasks_.Upload(sym_.pack_tasks, s);
  tc_tasks_.Upload(sym_.tc_tasks, s);
  fronts_.AllocGrowable(static_cast<size_t>(sym_.front_doubles));
  upd_.Alloc(static_cast<size_t>(std::max<int64_t>(1, sym_.update_doubles)));
  max_front_ = 1;
  for (const SupernodeRec& r : sym_.sn) {
    max_front_ = std::max(max_front_, r.F);
  }
  ConfigureSolveKernels(max_front_);
  solve_sync_.Alloc(SolveSyncWords(static_cast<int>(sym_.sn.size()), static_cast<int>(sym_.inv_tasks.size() / 2)));
  UploadSolveTasks(s);
  inv_tasks_.Upload(sym_.inv_tasks, s);
  inv_.Alloc(std::max<size_t>(1, sym_.inv_tasks.size() / 2) * kInvBlockDoubles);
  std::vector<InstDev> inst(host_.size());
  for (size_t i = 0; i < host_.size(); ++i) {
    const InstanceLayout& L = layout_[i];
    InstDev& d = inst[i];
    d.nx = L.nx;
    d.ny = L.ny;
    d.min_x = L.min_x;
    d.min_y = L.min_y;
    d.dx = L.dx;
    d.dy = L.dy;
    d.node_off = L.node_off;
    d.cell_off = L.cell_off;
    d.col_off = L.col_off;
    d.num_active = L.num_active;
    d.num_frames = L.num_frames;
    d.frame_off = L.frame_off;
    d.pt_off = L.pt_off;
    d.num_points = L.num_points;
    d.eik_off = L.eik_off;
    d.num_eik = L.num_eik;
    d.odom_off = L.odom_off;
    d.num_odom = L.num_odom;
    d.smooth_gradient = L.smooth_gradient;
    d.smooth_gradient_step = L.smooth_gradient_step;
    d.huber_delta = L.huber_delta;
    d.allow_off = sym_.allow_off[i];
    d.allow_words = sym_.allow_words[i];
    d.pp_base = sym_.pp_base[i];
    d.pp_ld = sym_.pp_ld[i];
    d.pp_first = sym_.pp_first[i];
    d.num_params = host_[i].num_params();
    d.mixed = i < mixed_.size() ? mixed_[i] : 0;
    d.refine_tol = i < refine_tol_.size() ? refine_tol_[i] : kDefaultRefineTol;
    d.near_cells = i < margin_.size() ? std::max(0, std::min(kNearCells, margin_[i] - 1)) : 0;
  }
  inst_host_ = inst;
  inst_.Upload(inst, s);
  fmp_ptr_.Upload(sym_.fmp_ptr, s);
  fmp_col_.Upload(sym_.fmp_col, s);
  fmp_off_.Upload(sym_.fmp_off, s);
  if (any_mixed_) {
    AllocMixed();
  }
  device_bytes_ = 0;
  device_bytes_ += static_cast<int64_t>(fronts_.size()) * 8 + static_cast<int64_t>(pt_rec_.size()) * 8 +
                   static_cast<int64_t>(mp_off_.size()) * 12 + static_cast<int64_t>(mm_off_.size()) * 8 +
                   static_cast<int64_t>(total_points_) * 80;
  RefreshView();
  CudaCheck(cudaStreamSynchronize(s), "analyze upload");
}

void Engine::RefreshView() {
  DeviceView& V = V_;
  V.inst = inst_.get();
  V.num_inst = count();
  V.total_nodes = total_nodes_;
  V.total_cells = total_cells_;
  V.total_frames = total_frames_;
  V.total_points = total_points_;
  V.total_eik = total_eik_;
  V.total_odom = total_odom_;
  V.n = n_;
  V.node_col = node_col_.get();
  V.col_node = col_node_.get();
  V.col_inst = col_inst_.get();
  V.frame_inst = frame_inst_.get();
  V.frame_col = frame_col_.get();
  V.pt_frame = pt_frame_.get();
  V.pt_xy = pt_xy_.get();
  V.pt_exp = pt_exp_.get();
  V.pt_sw = pt_sw_.get();
  V.eik_node = eik_node_.get();
  V.eik_n = eik_n_.get();
  V.eik_sw = eik_sw_.get();
  V.eik_index = eik_index_.get();
  V.odom_fi = odom_fi_.get();
  V.odom_fj = odom_fj_.get();
  V.odom_meas = odom_meas_.get();
  V.odom_sw = odom_sw_.get();
  V.frame_rows_ptr = frame_rows_ptr_.get();
  V.frame_rows = frame_rows_.get();
  V.frame_odom_ptr = frame_odom_ptr_.get();
  V.frame_odom = frame_odom_.get();
  V.num_pairs = num_pairs_;
  V.pair_f = pair_f_.get();
  V.pair_g = pair_g_.get();
  V.pair_ptr = pair_ptr_.get();
  V.pair_spec = pair_spec_.get();
  V.map = map_.get();
  V.poses = poses_.get();
  V.map_backup = map_backup_.get();
  V.poses_backup = poses_backup_.get();
  V.pose_cs = pose_cs_.get();
  V.pose_cs_backup = pose_cs_backup_.get();
  V.theta_pre = theta_pre_.get();
  V.theta_upd = theta_upd_.get();
  V.theta_out = theta_out_.get();
  V.pt_rec = pt_rec_.get();
  V.pt_poff = pt_poff_.get();
  V.pt_cell = pt_cell_.get();
  V.eik_rec = eik_rec_.get();
  V.odom_rec = odom_rec_.get();
  V.cell_start = cell_start_.get();
  V.cell_rows = cell_rows_ptr_;
  V.rhs = rhs_.get();
  V.step = step_.get();
  V.xs = xs_.get();
  V.lam = lam_.get();
  V.marquardt = marq_.get();
  V.status = status_.get();
  V.active = active_.get();
  V.perm = perm_.get();
  V.pinv = pinv_.get();
  V.sn = sn_.get();
  V.sn_rows = sn_rows_.get();
  V.sn_rel = sn_rel_.get();
  V.child_list = child_list_.get();
  V.mm_off = mm_off_.get();
  V.mp_ptr = mp_ptr_.get();
  V.mp_frame = mp_frame_.get();
  V.mp_off = mp_off_.get();
  V.allow_bits = allow_bits_.get();
  V.fronts = fronts_.get();
  V.fronts32 = any_mixed_ ? fronts32_.get() : nullptr;
  V.asm_fronts = any_mixed_ ? amat_.get() : fronts_.get();
  V.upd = upd_.get();
  V.tc_schur = (any_mixed_ && sym_.tc_pack_rows > 0 && tc_map_base_ != nullptr) ? 1 : 0;
  V.fmp_ptr = fmp_ptr_.get();
  V.fmp_col = fmp_col_.get();
  V.fmp_off = fmp_off_.get();
}

void Engine::AllocMixed() {
  amat_.AllocGrowable(static_cast<size_t>(sym_.front_doubles));
  fronts32_.AllocGrowable(static_cast<size_t>(sym_.front_doubles));
  res_.Alloc(static_cast<size_t>(std::max(n_, 1)));
  ax_.Alloc(static_cast<size_t>(std::max(n_, 1)));
  corr_.Alloc(static_cast<size_t>(std::max(n_, 1)));
  refine_done_.Alloc(host_.size());
  refine_max_.Alloc(2 * host_.size());
  refine_left_.Alloc(1);
  if (sym_.tc_pack_rows > 0) {
    pack_.Alloc(static_cast<size_t>(sym_.tc_pack_rows) * kTcChunk);
    const int64_t rows = static_cast<int64_t>(pack_.size() / kTcChunk);
    if (pack_.get() != tc_map_base_ || rows != tc_map_rows_) {
      EncodePackMap(&tc_map_, pack_.get(), rows);
      tc_map_base_ = pack_.get();
      tc_map_rows_ = rows;
    }
  }
}

void Engine::SetMode(const std::vector<int32_t>& mixed, int refine_steps, const std::vector<double>& refine_tol) {
  std::vector<double> tol = refine_tol;
  tol.resize(mixed.size(), kDefaultRefineTol);
  if (mixed == mixed_ && refine_steps == refine_steps_ && tol == refine_tol_) {
    return;
  }
  CudaCheck(cudaStreamSynchronize(stream_), "mode sync");
  mixed_ = mixed;
  refine_steps_ = refine_steps;
  refine_tol_ = tol;
  any_mixed_ = std::any_of(mixed_.begin(), mixed_.end(), [](int32_t v) { return v != 0; });
  for (size_t i = 0; i < inst_host_.size(); ++i) {
    inst_host_[i].mixed = mixed_[i];
    inst_host_[i].refine_tol = refine_tol_[i];
  }
  inst_.Upload(inst_host_, stream_);
  if (any_mixed_) {
    AllocMixed();
  }
  RefreshView();
  DropGraph();
  CudaCheck(cudaStreamSynchronize(stream_), "mode upload");
}

void Engine::SetActive(const std::vector<int32_t>& active) {
  // the pinned buffer may still feed an enqueued copy
  CudaCheck(cudaStreamSynchronize(stream_), "active sync");
  std::copy(active.begin(), active.end(), h_active_.get());
  CudaCheck(cudaMemcpyAsync(active_.get(), h_active_.get(), active.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            stream_),
            "active");
}

void Engine::SetLambda(const std::vector<double>& lam, const std::vector<int32_t>& marquardt) {
  CudaCheck(cudaStreamSynchronize(stream_), "lambda sync");
  std::copy(lam.begin(), lam.end(), h_lam_.get());
  std::copy(marquardt.begin(), marquardt.end(), h_marq_.get());
  CudaCheck(cudaMemcpyAsync(lam_.get(), h_lam_.get(), lam.size() * sizeof(double), cudaMemcpyHostToDevice, stream_),
            "lambda");
  CudaCheck(cudaMemcpyAsync(marq_.get(), h_marq_.get(), marquardt.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            stream_),
            "marquardt");
}

void Engine::ClearStatus() {
  CudaCheck(cudaMemsetAsync(status_.get(), 0, sizeof(int32_t) * host_.size(), stream_), "status");
}

namespace {

/// A wait of the one-launch solve that ran out of its limit leaves no valid
/// result behind: the call fails.
void CheckWaits(const int32_t* st, size_t count) {
  for (size_t i = 0; i < count; ++i) {
    if ((st[i] & kStatusWaitTimeout) != 0) {
      Fail(SDFGPU_ERR_TIMEOUT, "a wait of the solve kernel ran out of its limit");
    }
  }
}

}  // namespace

std::vector<int32_t> Engine::DownloadStatus() {
  std::vector<int32_t> st(host_.size());
  CudaCheck(cudaMemcpyAsync(st.data(), status_.get(), st.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_),
            "status");
  CudaCheck(cudaStreamSynchronize(stream_), "status sync");
  CheckWaits(st.data(), st.size());
  return st;
}

void Engine::LaunchRows() {
  if (total_points_ > 0) {
    KPointRows<<<Blocks(total_points_, 256), 256, 0, stream_>>>(V_);
  }
  if (total_eik_ > 0) {
    KEikonalRows<<<Blocks(total_eik_, 256), 256, 0, stream_>>>(V_);
  }
  if (total_odom_ > 0) {
    KOdomRows<<<Blocks(total_odom_, 128), 128, 0, stream_>>>(V_);
  }
  bool in_a = true;
  if (total_points_ > 0) {
    LaunchCellSort(pt_cell_.get(), total_points_, total_cells_, sort_keys_a_.get(), sort_vals_a_.get(),
                   sort_keys_b_.get(), sort_vals_b_.get(), sort_hist_.get(), stream_, &in_a);
  }
  const int32_t* keys = in_a ? sort_keys_a_.get() : sort_keys_b_.get();
  cell_rows_ptr_ = in_a ? sort_vals_a_.get() : sort_vals_b_.get();
  V_.cell_rows = cell_rows_ptr_;
  KCellStart<<<Blocks(total_cells_ + 1, 256), 256, 0, stream_>>>(keys, total_points_, total_cells_,
                                                                   cell_start_.get());
  CudaCheck(cudaGetLastError(), "row kernels");
  int bits = 1;
  while ((int64_t{1} << bits) <= total_cells_) {
    ++bits;
  }
  times_.launches += (total_points_ > 0 ? 1 + 1 + 3 * ((bits + 7) / 8) : 0) + (total_eik_ > 0 ? 1 : 0) +
                     (total_odom_ > 0 ? 1 : 0) + 1;
}

int64_t Engine::ZeroTaskCount() const {
  // the leaf fronts' trailing columns only for an in-place tensor-core
  // Schur complement
  return V_.tc_schur != 0 ? static_cast<int64_t>(sym_.zero_tasks.size() / 2) : sym_.zero_main;
}

void Engine::LaunchNormal() {
  const int64_t zero_count = ZeroTaskCount();
  if (zero_count > 0) {
    KZeroFronts<<<static_cast<unsigned>(zero_count), 32 * kZeroCols, 0, stream_>>>(V_, zero_tasks_.get());
    CudaCheck(cudaGetLastError(), "front zeroing");
    ++times_.launches;
  }
  CudaCheck(cudaMemsetAsync(rhs_.get(), 0, static_cast<size_t>(n_) * sizeof(double), stream_), "rhs memset");
  if (total_cells_ > 0) {
    // as many blocks as are resident at once
    static const int64_t resident = [] {
      int dev = 0;
      int sms = 0;
      int per_sm = 0;
      CudaCheck(cudaGetDevice(&dev), "device");
      CudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
      CudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, KCellPass, 256, 0), "occupancy");
      return static_cast<int64_t>(std::max(1, per_sm)) * sms;
    }();
    for (int pass = 0; pass < 4; ++pass) {
      const int64_t count = pass_begin_[pass + 1] - pass_begin_[pass];
      if (count > 0) {
        const int64_t blocks = std::min<int64_t>(Blocks(count * 32, 256), resident);
        KCellPass<<<static_cast<unsigned>(blocks), 256, 0, stream_>>>(V_, pass_cells_.get() + pass_begin_[pass],
                                                                      count);
      }
    }
  }
  KPoseFrames<<<static_cast<unsigned>(total_frames_), 256, 0, stream_>>>(V_);
  if (num_pairs_ > 0) {
    KPosePairs<<<Blocks(static_cast<int64_t>(num_pairs_) * 9, 128), 128, 0, stream_>>>(V_);
  }
  if (n_ > 0) {
    KFinalizeNormal<<<Blocks(n_, 256), 256, 0, stream_>>>(V_);
  }
  CudaCheck(cudaGetLastError(), "normal kernels");
  times_.launches += (total_cells_ > 0 ? 4 : 0) + 1 + (num_pairs_ > 0 ? 1 : 0) + (n_ > 0 ? 1 : 0);
}

void Engine::SegmentSum(const double* x, const int64_t* seg_begin, const int64_t* seg_end, int segments,
                        double* out) {
  KSegmentPartial<<<static_cast<unsigned>(segments * 32), 256, 0, stream_>>>(x, seg_begin, seg_end,
                                                                            seg_partial_.get());
  KSegmentFinal<<<Blocks(static_cast<int64_t>(segments) * 32, 128), 128, 0, stream_>>>(seg_partial_.get(), segments,
                                                                                      out);
  times_.launches += 2;
}

FactorPlan Engine::Plan() {
  FactorPlan P;
  P.small_tasks = small_tasks_.get();
  P.ea_tasks = ea_tasks_.get();
  P.ea_child = ea_child_.get();
  P.panel_tasks = panel_tasks_.get();
  P.update_tasks = update_tasks_.get();
  P.level_sn = level_sn_.get();
  P.dvec = dvec_.get();
  P.max_front = max_front_;
  P.solve_sync = solve_sync_.get();
  P.solve_tasks = solve_tasks_.get();
  P.num_solve_tasks = static_cast<int>(sym_.solve_tasks.size() / 4);
  P.solve_parts = solve_parts_.get();
  P.zpart_off = zpart_off_.get();
  P.ys = ys_.get();
  P.zpart = zpart_.get();
  P.inv_tasks = inv_tasks_.get();
  P.num_inv = static_cast<int>(sym_.inv_tasks.size() / 2);
  P.inv = inv_.get();
  P.fp32_fronts = any_mixed_;
  P.dense_tasks = dense_tasks_.get();
  P.dense_sync = dense_sync_.get();
  P.dense_inv = dense_inv_.get();
  P.solve_withhold = solve_withhold_;
  P.solve_wait_polls = solve_wait_polls_;
  // only the iteration's own factor and solve phases are timed
  P.timer = timing_phase_ ? &timer_ : nullptr;
  if (any_mixed_ && sym_.tc_pack_rows > 0 && tc_map_base_ != nullptr) {
    P.tc_map = &tc_map_;
    P.pack_tasks = pack_tasks_.get();
    P.tc_tasks = tc_tasks_.get();
    P.tc = TcArgs{sn_.get(), fronts32_.get(), dvec_.get(), active_.get(), inst_.get(), status_.get(), pack_.get()};
  }
  return P;
}

void Engine::LaunchFactor() {
  const int64_t conv_count = ZeroTaskCount();
  if (any_mixed_ && conv_count > 0) {
    // work copies of the assembled fronts (FP32 for mixed grid supernodes),
    // over the region the zeroing cleared
    KConvertFronts<<<static_cast<unsigned>(conv_count), 32 * kZeroCols, 0, stream_>>>(V_, zero_tasks_.get());
    CudaCheck(cudaGetLastError(), "convert fronts");
    ++times_.launches;
  }
  times_.launches += LaunchFactorLevels(sym_, V_, Plan(), stream_);
}

void Engine::LaunchSolve() {
  times_.launches += LaunchSolveLevels(sym_, V_, Plan(), stream_);
  if (!any_mixed_ || n_ == 0) {
    return;
  }
  // iterative refinement of the mixed instances' steps against the FP64
  // normal matrix: r = rhs - A delta, delta += (LDL^T)^-1 r
  // A round stops counting for an instance once its largest correction is
  // below its refine_tol times its largest step entry: each round shrinks
  // the error by about cond(A) * 2^-24, so the next one would move the step
  // by a small fraction of that (the default, 1e-13, by far less than the
  // FP64 path's own rounding differences).
  DeviceView Vm = V_;
  Vm.refine_done = refine_done_.get();
  Vm.refine_max = refine_max_.get();
  Vm.refine_left = refine_left_.get();
  DeviceView Vr = Vm;
  Vr.rhs = res_.get();
  Vr.step = corr_.get();
  if (refine_steps_ > 0) {
    KRefineReset<<<1, 128, 0, stream_>>>(Vm);
    ++times_.launches;
  }
  for (int round = 0; round < refine_steps_; ++round) {
    KNormalMatVecMap<<<Blocks(32 * static_cast<int64_t>(n_), 256), 256, 0, stream_>>>(Vm, step_.get(), ax_.get());
    KNormalMatVecPose<<<Blocks(3 * static_cast<int64_t>(total_frames_) * 32, 256), 256, 0, stream_>>>(
        Vm, step_.get(), ax_.get());
    KRefineResidual<<<Blocks(n_, 256), 256, 0, stream_>>>(Vm, ax_.get(), res_.get());
    times_.launches += 3 + LaunchSolveLevels(sym_, Vr, Plan(), stream_);
    KAddCorrection<<<Blocks(n_, 256), 256, 0, stream_>>>(Vm, corr_.get());
    KRefineCheck<<<1, 256, 0, stream_>>>(Vm);
    times_.launches += 2;
  }
  CudaCheck(cudaGetLastError(), "refinement kernels");
}

void Engine::LaunchCost(std::vector<double>& cost) {
  const int64_t terms = total_points_ + total_eik_ + total_odom_;
  ClearStatus();
  if (terms > 0) {
    KCostTerms<<<Blocks(terms, 128), 128, 0, stream_>>>(V_, terms_.get());
  }
  const size_t I = host_.size();
  SegmentSum(terms_.get(), seg_begin_.get(), seg_end_.get(), static_cast<int>(3 * I), seg_out_.get());
  std::vector<double> out(3 * I);
  CudaCheck(cudaMemcpyAsync(out.data(), seg_out_.get(), out.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_),
            "cost");
  std::vector<int32_t> st(I);
  CudaCheck(cudaMemcpyAsync(st.data(), status_.get(), I * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_),
            "status");
  CudaCheck(cudaStreamSynchronize(stream_), "cost sync");
  cost.resize(I);
  for (size_t i = 0; i < I; ++i) {
    cost[i] = (out[3 * i] + out[3 * i + 1]) + out[3 * i + 2];
    if ((st[i] & kStatusNextOverflow) != 0) {
      pending_.push_back(static_cast<int>(i));
    }
  }
}

void Engine::LaunchStepAndCost(bool backup) {
  const int64_t big = std::max<int64_t>(total_nodes_, 3 * static_cast<int64_t>(total_frames_));
  if (backup) {
    KBackup<<<Blocks(big, 256), 256, 0, stream_>>>(V_, 0, revert_.get());
  }
  if (n_ > 0) {
    LaunchApplyStep();
    KStepTerms<<<Blocks(n_, 256), 256, 0, stream_>>>(V_, sq_terms_.get(), pred_terms_.get());
  }
  const size_t I = host_.size();
  SegmentSum(sq_terms_.get(), step_seg_begin_.get(), step_seg_end_.get(), static_cast<int>(I), seg_out_.get() + 3 * I);
  SegmentSum(pred_terms_.get(), step_seg_begin_.get(), step_seg_end_.get(), static_cast<int>(I),
             seg_out_.get() + 4 * I);
  const int64_t terms = total_points_ + total_eik_ + total_odom_;
  if (terms > 0) {
    KCostTerms<<<Blocks(terms, 128), 128, 0, stream_>>>(V_, terms_.get());
  }
  SegmentSum(terms_.get(), seg_begin_.get(), seg_end_.get(), static_cast<int>(3 * I), seg_out_.get());
  times_.launches += (backup ? 1 : 0) + (n_ > 0 ? 1 : 0) + (terms > 0 ? 1 : 0);
  CudaCheck(cudaMemcpyAsync(h_seg_.get(), seg_out_.get(), 5 * I * sizeof(double), cudaMemcpyDeviceToHost, stream_),
            "step terms");
  CudaCheck(cudaMemcpyAsync(h_status_.get(), status_.get(), I * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_),
            "status");
  CudaCheck(cudaGetLastError(), "step kernels");
}

void Engine::Reanalyze(const std::vector<int>& which) {
  const auto t0 = std::chrono::steady_clock::now();
  // a background analysis of these instances is superseded by this one
  DropSpeculations(&which);
  std::vector<double> poses(3 * static_cast<size_t>(total_frames_));
  CudaCheck(cudaMemcpyAsync(poses.data(), poses_.get(), poses.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_),
            "poses");
  CudaCheck(cudaStreamSynchronize(stream_), "reanalyze sync");
  for (const int i : which) {
    const InstanceLayout& L = layout_[static_cast<size_t>(i)];
    std::copy(poses.begin() + 3 * L.frame_off, poses.begin() + 3 * (L.frame_off + L.num_frames),
              host_[static_cast<size_t>(i)].poses.begin());
    // a pattern that was left once is widened so that it is left less often
    margin_[static_cast<size_t>(i)] = std::min(margin_[static_cast<size_t>(i)] + kMarginStep, kMaxMargin);
  }
  AnalyzeInstances(host_, margin_, pieces_, &which);
  for (const int i : which) {
    analysed_at_[static_cast<size_t>(i)] = iters_[static_cast<size_t>(i)];
  }
  sym_ = GlobalStructure();
  UploadSymbolic();
  ++times_.reanalyses;
  times_.reanalysis_host += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void Engine::SetKernelTiming(uint32_t mask) {
  CudaCheck(cudaStreamSynchronize(stream_), "timing sync");
  timer_.SetMask(mask);
  DropGraph();  // the captured phases carry the previous event nodes
}

void Engine::SetSolveFault(int withhold, uint32_t wait_polls) {
  if (withhold < -1 || withhold >= static_cast<int>(sym_.sn.size())) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "supernode index out of range");
  }
  solve_withhold_ = withhold;
  solve_wait_polls_ = wait_polls;
  DropGraph();  // the captured solve holds the previous parameters
}

void Engine::UploadSolveTasks(cudaStream_t s) {
  zero_tasks_.Upload(sym_.zero_tasks, s);
  dense_tasks_.Upload(sym_.dense_tasks, s);
  dense_sync_.Alloc(DenseSyncWords(sym_));
  dense_inv_.Alloc(static_cast<size_t>(std::max<int64_t>(1, sym_.dense_inv_doubles)));
  solve_tasks_.Upload(sym_.solve_tasks, s);
  solve_parts_.Upload(sym_.solve_parts, s);
  zpart_off_.Upload(sym_.zpart_off, s);
  ys_.Alloc(static_cast<size_t>(std::max(n_, 1)));
  zpart_.Alloc(static_cast<size_t>(std::max<int64_t>(1, sym_.zpart_doubles)));
}

void Engine::UploadSchedule() {
  DropGraph();
  CudaCheck(cudaStreamSynchronize(stream_), "schedule sync");
  ea_tasks_.Upload(sym_.ea_tasks, stream_);
  ea_child_.Upload(sym_.ea_child, stream_);
  panel_tasks_.Upload(sym_.panel_tasks, stream_);
  update_tasks_.Upload(sym_.update_tasks, stream_);
  small_tasks_.Upload(sym_.small_tasks, stream_);
  pack_tasks_.Upload(sym_.pack_tasks, stream_);
  tc_tasks_.Upload(sym_.tc_tasks, stream_);
  level_sn_.Upload(sym_.level_sn, stream_);
  sn_.Upload(sym_.sn, stream_);
  UploadSolveTasks(stream_);
  CudaCheck(cudaStreamSynchronize(stream_), "schedule upload");
}

double Engine::Autotune(std::vector<std::pair<Schedule, double>>* trials) {
  // Candidate schedules: the pivot count below which a front is factored by
  // one kernel, that kernel's rows per block, and the rows per panel task
  // (0: wider fronts by whole outer blocks of 128 pivots, KPanelBlock).
  const std::vector<Schedule> candidates = {{128, 256, 128}, {128, 128, 128}, {96, 256, 128}, {64, 256, 128},
                                            {64, 128, 64},   {128, 256, 64},  {64, 128, 0},   {128, 256, 0}};
  const size_t I = host_.size();
  // the precision of the last solve: a mixed one also decides whether the
  // wide FP32 fronts' Schur complements run on the tensor cores
  const std::vector<int32_t> last_mixed = mixed_;
  const int last_refine = refine_steps_;
  const std::vector<double> last_tol = refine_tol_;
  const bool tune_tc = any_mixed_;
  SetMode(std::vector<int32_t>(I, 0), 0);
  SetActive(std::vector<int32_t>(I, 1));
  SetLambda(std::vector<double>(I, 1.0), std::vector<int32_t>(I, 0));
  double best = 0.0;
  Schedule best_sched = sched_;
  for (Schedule c : candidates) {
    c.tc_min_rows = sched_.tc_min_rows;
    Reschedule(sym_, c);
    UploadSchedule();
    double ms_min = 0.0;
    for (int rep = 0; rep < 3; ++rep) {
      // factor the current state's normal matrix (reassembled each time:
      // the factorization overwrites it)
      ClearStatus();
      LaunchRows();
      LaunchNormal();
      CudaCheck(cudaEventRecord(ev_[0], stream_), "event");
      LaunchFactor();
      CudaCheck(cudaEventRecord(ev_[1], stream_), "event");
      CudaCheck(cudaStreamSynchronize(stream_), "autotune");
      float ms = 0.0f;
      CudaCheck(cudaEventElapsedTime(&ms, ev_[0], ev_[1]), "autotune timing");
      ms_min = rep == 0 ? ms : std::min(ms_min, static_cast<double>(ms));
    }
    if (trials != nullptr) {
      trials->emplace_back(c, ms_min);
    }
    if (best == 0.0 || ms_min < best) {
      best = ms_min;
      best_sched = c;
    }
  }
  if (tune_tc) {
    // factor + solve (with the refinement rounds the step needs: a less
    // accurate factor costs rounds) of the last solve's mixed instances,
    // with and without the tensor-core Schur complements; every front
    // eligible for them is wide, so one threshold decides
    SetMode(last_mixed, last_refine, last_tol);
    double best_mixed = 0.0;
    tc_trial_ms_[0] = tc_trial_ms_[1] = 0.0;
    for (const int rows : {kTcMinRowsDefault, 0}) {
      sched_ = best_sched;
      sched_.tc_min_rows = rows;
      InstallSchedule();
      if (rows > 0 && sym_.tc_pack_rows == 0) {
        continue;  // no front is wide enough
      }
      const double ms = TimeMixedFactorSolve();
      tc_trial_ms_[rows > 0 ? 0 : 1] = ms;
      if (best_mixed == 0.0 || ms < best_mixed) {
        best_mixed = ms;
        best_sched.tc_min_rows = rows;
      }
    }
  }
  sched_ = best_sched;
  InstallSchedule();
  return best;
}

void Engine::SetSchedule(const Schedule& sched) {
  if (sched.small_pivots < 32 || sched.small_pivots > 128 || sched.front_rows < 128 || sched.front_rows > 256 ||
      (sched.panel_rows != 0 && (sched.panel_rows < 16 || sched.panel_rows > 128))) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT,
         "schedule out of range (small_pivots 32..128, front_rows 128..256, panel_rows 0 or 16..128)");
  }
  sched_ = sched;
  InstallSchedule();
}

void Engine::InstallSchedule() {
  Reschedule(sym_, sched_);
  UploadSchedule();
  // the tensor-core task lists and their operand buffer follow tc_min_rows
  if (any_mixed_) {
    AllocMixed();
  }
  RefreshView();
}

double Engine::TimeMixedFactorSolve() {
  double ms_min = 0.0;
  for (int rep = 0; rep < 3; ++rep) {
    ClearStatus();
    LaunchRows();
    LaunchNormal();
    CudaCheck(cudaEventRecord(ev_[0], stream_), "event");
    LaunchFactor();
    LaunchSolve();
    CudaCheck(cudaEventRecord(ev_[1], stream_), "event");
    CudaCheck(cudaStreamSynchronize(stream_), "autotune");
    float ms = 0.0f;
    CudaCheck(cudaEventElapsedTime(&ms, ev_[0], ev_[1]), "autotune timing");
    ms_min = rep == 0 ? ms : std::min(ms_min, static_cast<double>(ms));
  }
  return ms_min;
}

void Engine::ReanalyzePending() {
  if (pending_.empty()) {
    return;
  }
  std::sort(pending_.begin(), pending_.end());
  pending_.erase(std::unique(pending_.begin(), pending_.end()), pending_.end());
  const std::vector<int> which = std::move(pending_);
  pending_.clear();
  Reanalyze(which);
}

void Engine::StartSpeculation(int i, const std::vector<double>& poses) {
  auto sp = std::make_unique<Speculation>();
  const InstanceLayout& L = layout_[static_cast<size_t>(i)];
  sp->inst = i;
  sp->margin = margin_[static_cast<size_t>(i)];
  sp->poses.assign(poses.begin() + 3 * static_cast<int64_t>(L.frame_off),
                   poses.begin() + 3 * static_cast<int64_t>(L.frame_off + L.num_frames));
  sp->adopt_at = iters_[static_cast<size_t>(i)] + kSpeculationDelay;
  sp->has_structure = host_.size() == 1;
  sp->sched = sched_;
  // the thread reads only this instance's problem, which stays unchanged
  // until the speculation is installed or dropped
  Speculation* raw = sp.get();
  sp->done = std::async(std::launch::async, [this, raw] {
    raw->piece = AnalyzeInstance(host_[static_cast<size_t>(raw->inst)], raw->margin, 0, &raw->poses);
    if (raw->has_structure) {
      raw->structure = ConcatenateOne(std::move(raw->piece), 32, 64, raw->sched);
    }
  });
  specs_.push_back(std::move(sp));
}

void Engine::DropSpeculations(const std::vector<int>* which) {
  for (auto it = specs_.begin(); it != specs_.end();) {
    if (which != nullptr && std::find(which->begin(), which->end(), (*it)->inst) == which->end()) {
      ++it;
      continue;
    }
    if ((*it)->done.valid()) {
      (*it)->done.wait();  // an exception it stored is discarded with it
    }
    it = specs_.erase(it);
  }
}

void Engine::StepSpeculations() {
  // instances about to be re-analysed from their current state
  if (!pending_.empty() && !specs_.empty()) {
    DropSpeculations(&pending_);
  }
  std::vector<std::unique_ptr<Speculation>> due;
  for (auto it = specs_.begin(); it != specs_.end();) {
    if ((*it)->adopt_at <= iters_[static_cast<size_t>((*it)->inst)]) {
      due.push_back(std::move(*it));
      it = specs_.erase(it);
    } else {
      ++it;
    }
  }
  if (!due.empty()) {
    const auto t0 = std::chrono::steady_clock::now();
    bool built = false;
    for (auto& sp : due) {
      sp->done.get();
      const auto i = static_cast<size_t>(sp->inst);
      host_[i].poses = std::move(sp->poses);
      analysed_at_[i] = iters_[i];
      if (sp->has_structure) {
        // a single instance (never pending here: its pending state dropped
        // the speculation); the schedule may have changed since
        sym_ = std::move(sp->structure);
        const Schedule& now = sched_;
        if (now.small_pivots != sp->sched.small_pivots || now.front_rows != sp->sched.front_rows ||
            now.panel_rows != sp->sched.panel_rows || now.tc_min_rows != sp->sched.tc_min_rows) {
          Reschedule(sym_, sched_);
        }
        built = true;
      } else {
        pieces_[i] = std::move(sp->piece);
      }
    }
    // a synchronous re-analysis (pending_) rebuilds the structure anyway
    if (pending_.empty()) {
      if (!built) {
        sym_ = GlobalStructure();
      }
      UploadSymbolic();
    }
    ++times_.reanalyses;
    times_.reanalysis_host += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  std::vector<int> start;
  for (const int i : near_) {
    const auto u = static_cast<size_t>(i);
    if (iters_[u] - analysed_at_[u] < kSpeculateAfter ||
        std::find(pending_.begin(), pending_.end(), i) != pending_.end() ||
        std::find(start.begin(), start.end(), i) != start.end()) {
      continue;
    }
    bool busy = false;
    for (const auto& sp : specs_) {
      busy = busy || sp->inst == i;
    }
    if (!busy) {
      start.push_back(i);
    }
  }
  near_.clear();
  if (!start.empty()) {
    // the accepted states (a revert of other instances may still be queued)
    std::vector<double> poses(3 * static_cast<size_t>(total_frames_));
    CudaCheck(cudaMemcpyAsync(poses.data(), poses_.get(), poses.size() * sizeof(double), cudaMemcpyDeviceToHost,
                              stream_),
              "poses");
    CudaCheck(cudaStreamSynchronize(stream_), "speculation sync");
    for (const int i : start) {
      StartSpeculation(i, poses);
    }
  }
}

/// Rows + normal equations; re-runs the symbolic analysis (once) when a point
/// left its pose's analysed cell set. Returns the per-instance status OR.
int Engine::AssembleWithPattern() {
  for (int attempt = 0; attempt < 2; ++attempt) {
    ClearStatus();
    CudaCheck(cudaEventRecord(ev_[0], stream_), "event");
    LaunchRows();
    CudaCheck(cudaEventRecord(ev_[1], stream_), "event");
    LaunchNormal();
    CudaCheck(cudaEventRecord(ev_[2], stream_), "event");
    const std::vector<int32_t> st = DownloadStatus();
    std::vector<int> overflow;
    for (size_t i = 0; i < st.size(); ++i) {
      if ((st[i] & kStatusPatternOverflow) != 0) {
        overflow.push_back(static_cast<int>(i));
      }
    }
    if (overflow.empty()) {
      float ms = 0.0f;
      CudaCheck(cudaEventElapsedTime(&ms, ev_[0], ev_[1]), "phase timing");
      times_.assemble += ms * 1e-3;
      CudaCheck(cudaEventElapsedTime(&ms, ev_[1], ev_[2]), "phase timing");
      times_.normal += ms * 1e-3;
      return 0;
    }
    Reanalyze(overflow);
  }
  Fail(SDFGPU_ERR_CUDA, "sparsity pattern still overflows after re-analysis");
}

void Engine::GetState(int i, double* map_values, double* poses) {
  const InstanceLayout& L = layout_[static_cast<size_t>(i)];
  if (map_values != nullptr) {
    CudaCheck(cudaMemcpyAsync(map_values, map_.get() + L.node_off,
                              sizeof(double) * static_cast<size_t>(L.nx) * L.ny, cudaMemcpyDeviceToHost, stream_),
              "get map");
  }
  if (poses != nullptr) {
    CudaCheck(cudaMemcpyAsync(poses, poses_.get() + 3 * L.frame_off, sizeof(double) * 3 * L.num_frames,
                              cudaMemcpyDeviceToHost, stream_),
              "get poses");
  }
  CudaCheck(cudaStreamSynchronize(stream_), "get state");
}

void Engine::SetState(int i, const double* map_values, const double* poses) {
  const InstanceLayout& L = layout_[static_cast<size_t>(i)];
  if (map_values != nullptr) {
    CudaCheck(cudaMemcpyAsync(map_.get() + L.node_off, map_values,
                              sizeof(double) * static_cast<size_t>(L.nx) * L.ny, cudaMemcpyHostToDevice, stream_),
              "set map");
  }
  if (poses != nullptr) {
    CudaCheck(cudaMemcpyAsync(poses_.get() + 3 * L.frame_off, poses, sizeof(double) * 3 * L.num_frames,
                              cudaMemcpyHostToDevice, stream_),
              "set poses");
    UploadPoseTrig(poses, L.frame_off, L.num_frames);
  }
  CudaCheck(cudaStreamSynchronize(stream_), "set state");
}

void Engine::UploadPoseTrig(const double* poses, int frame_off, int frames) {
  if (frames <= 0) {
    return;
  }
  // the reference's rotation (pose.hpp:19-25) with the platform's cos and sin
  std::vector<double2> cs(static_cast<size_t>(frames));
  for (int f = 0; f < frames; ++f) {
    const double th = poses[3 * static_cast<size_t>(f) + 2];
    cs[static_cast<size_t>(f)] = make_double2(std::cos(th), std::sin(th));
  }
  CudaCheck(cudaMemcpyAsync(pose_cs_.get() + frame_off, cs.data(), cs.size() * sizeof(double2),
                            cudaMemcpyHostToDevice, stream_),
            "pose trig");
  // the pageable source must outlive the copy
  CudaCheck(cudaStreamSynchronize(stream_), "pose trig");
}

void Engine::LaunchApplyStep() {
  if (n_ <= 0) {
    return;
  }
  const size_t F = static_cast<size_t>(total_frames_);
  CudaCheck(cudaMemsetAsync(theta_upd_.get(), 0, F * sizeof(int32_t), stream_), "angle flags");
  KApplyStep<<<Blocks(n_, 256), 256, 0, stream_>>>(V_);
  // the moved frames' angles for the host's exact wrap (CommitAngles)
  CudaCheck(cudaMemcpyAsync(h_theta_pre_.get(), theta_pre_.get(), F * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_),
            "angles");
  CudaCheck(cudaMemcpyAsync(h_theta_upd_.get(), theta_upd_.get(), F * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            stream_),
            "angle flags");
  CudaCheck(cudaGetLastError(), "apply step");
  times_.launches += 1;
}

void Engine::CommitAngles(const std::vector<int32_t>* revert) {
  // the stream has drained: h_theta_pre_ / h_theta_upd_ hold the last step's
  // angles, and the previous commit's upload has read h_theta_out_
  const int F = total_frames_;
  if (F <= 0 || n_ <= 0) {
    return;
  }
  const int32_t* upd = h_theta_upd_.get();
  const double* pre = h_theta_pre_.get();
  double* out = h_theta_out_.get();
  bool any = false;
  for (int f = 0; f < F; ++f) {
    any = any || (upd[f] != 0 && (revert == nullptr || (*revert)[static_cast<size_t>(frame_inst_host_[f])] == 0));
  }
  if (!any) {
    return;
  }
  // WrapAngle (pose.hpp:9) and the new angle's cos and sin with the
  // platform's libm, as the reference computes them (problem.cpp:117-130);
  // on the host pool's threads when there are many frames
  ParallelRanges(PoolThreads(), F, 256, [&](int64_t b, int64_t e) {
    for (int64_t f = b; f < e; ++f) {
      const bool commit = upd[f] != 0 &&
                          (revert == nullptr || (*revert)[static_cast<size_t>(frame_inst_host_[f])] == 0);
      out[4 * f + 3] = commit ? 1.0 : 0.0;
      if (commit) {
        const double t = pre[f];
        const double th = std::atan2(std::sin(t), std::cos(t));
        out[4 * f] = th;
        out[4 * f + 1] = std::cos(th);
        out[4 * f + 2] = std::sin(th);
      }
    }
  });
  CudaCheck(cudaMemcpyAsync(theta_out_.get(), out, 4 * static_cast<size_t>(F) * sizeof(double), cudaMemcpyHostToDevice,
                            stream_),
            "wrapped angles");
  KCommitPoses<<<Blocks(F, 128), 128, 0, stream_>>>(V_);
  CudaCheck(cudaGetLastError(), "commit angles");
  ++times_.launches;
}

double Engine::Cost(int i) {
  std::vector<double> cost;
  LaunchCost(cost);
  return cost[static_cast<size_t>(i)];
}

void Engine::ApplyStep(int i, const double* step) {
  const InstanceLayout& L = layout_[static_cast<size_t>(i)];
  std::vector<int32_t> active(host_.size(), 0);
  active[static_cast<size_t>(i)] = 1;
  SetActive(active);
  ClearStatus();
  CudaCheck(cudaMemcpyAsync(step_.get() + L.col_off, step, sizeof(double) * host_[static_cast<size_t>(i)].num_params(),
                            cudaMemcpyHostToDevice, stream_),
            "step");
  LaunchApplyStep();
  CudaCheck(cudaStreamSynchronize(stream_), "apply step sync");
  CommitAngles(nullptr);
  std::vector<int32_t> ones(host_.size(), 1);
  SetActive(ones);
  CudaCheck(cudaStreamSynchronize(stream_), "apply step sync");
}

void Engine::Linearize(int i, double lambda, bool marquardt, bool compute_step) {
  const size_t I = host_.size();
  SetMode(std::vector<int32_t>(I, 0), 0);
  const HostProblem& hp = host_[static_cast<size_t>(i)];
  const InstanceLayout& L = layout_[static_cast<size_t>(i)];
  std::vector<int32_t> active(I, 0);
  active[static_cast<size_t>(i)] = 1;
  SetActive(active);
  std::vector<double> lam(I, lambda);
  std::vector<int32_t> marq(I, marquardt ? 1 : 0);
  SetLambda(lam, marq);
  AssembleWithPattern();
  const int P = hp.num_points();
  const int E = hp.num_eikonal();
  const int O = hp.num_odom();
  std::vector<double> prec(static_cast<size_t>(P) * kPointRec);
  std::vector<double> erec(static_cast<size_t>(E) * kEikRec);
  std::vector<double> orec(static_cast<size_t>(O) * kOdomRec);
  std::vector<int32_t> cells(static_cast<size_t>(P));
  std::vector<double> rhs(static_cast<size_t>(hp.num_params()));
  std::vector<double> fronts(static_cast<size_t>(sym_.front_doubles));
  cudaStream_t s = stream_;
  CudaCheck(cudaMemcpyAsync(prec.data(), pt_rec_.get() + L.pt_off * kPointRec, prec.size() * 8, cudaMemcpyDeviceToHost, s), "lin");
  CudaCheck(cudaMemcpyAsync(erec.data(), eik_rec_.get() + L.eik_off * kEikRec, erec.size() * 8, cudaMemcpyDeviceToHost, s), "lin");
  CudaCheck(cudaMemcpyAsync(orec.data(), odom_rec_.get() + L.odom_off * kOdomRec, orec.size() * 8, cudaMemcpyDeviceToHost, s), "lin");
  CudaCheck(cudaMemcpyAsync(cells.data(), pt_cell_.get() + L.pt_off, cells.size() * 4, cudaMemcpyDeviceToHost, s), "lin");
  CudaCheck(cudaMemcpyAsync(rhs.data(), rhs_.get() + L.col_off, rhs.size() * 8, cudaMemcpyDeviceToHost, s), "lin");
  CudaCheck(cudaMemcpyAsync(fronts.data(), fronts_.get(), fronts.size() * 8, cudaMemcpyDeviceToHost, s), "lin");
  CudaCheck(cudaStreamSynchronize(s), "lin sync");
  Lin out;
  out.instance = i;
  const int nrows = hp.num_rows();
  const int np = hp.num_params();
  out.residuals.resize(static_cast<size_t>(nrows));
  out.point_cell.resize(static_cast<size_t>(P));
  // rows in the reference's order with their (column, value) entries
  std::vector<int32_t> row_ptr(static_cast<size_t>(nrows) + 1, 0);
  std::vector<int32_t> rcols;
  std::vector<double> rvals;
  const int A = hp.num_active();
  const int cw = hp.nx - 1;
  for (int k = 0; k < P; ++k) {
    const double* rec = prec.data() + static_cast<size_t>(k) * kPointRec;
    out.residuals[static_cast<size_t>(k)] = rec[7];
    const int cell = cells[static_cast<size_t>(k)];
    if (cell >= 0) {
      const int local_cell = static_cast<int>(cell - L.cell_off);
      const int w = local_cell % cw;
      const int h = local_cell / cw;
      out.point_cell[static_cast<size_t>(k)] = h * hp.nx + w;
      for (int q = 0; q < 4; ++q) {
        const int node = (h + (q >> 1)) * hp.nx + w + (q & 1);
        const int col = hp.node_to_active[static_cast<size_t>(node)];
        if (col >= 0) {
          rcols.push_back(col);
          rvals.push_back(rec[q]);
        }
      }
      const int f = hp.pt_frame[static_cast<size_t>(k)];
      if (f >= 1) {
        for (int c = 0; c < 3; ++c) {
          rcols.push_back(A + 3 * (f - 1) + c);
          rvals.push_back(rec[4 + c]);
        }
      }
    } else {
      out.point_cell[static_cast<size_t>(k)] = -1;
    }
    row_ptr[static_cast<size_t>(k) + 1] = static_cast<int32_t>(rcols.size());
  }
  for (int e = 0; e < E; ++e) {
    const double* rec = erec.data() + static_cast<size_t>(e) * kEikRec;
    out.residuals[static_cast<size_t>(P + e)] = rec[3];
    const int w = hp.eik_wh[2 * static_cast<size_t>(e)];
    const int h = hp.eik_wh[2 * static_cast<size_t>(e) + 1];
    const int nodes[3] = {h * hp.nx + w, h * hp.nx + w + 1, (h + 1) * hp.nx + w};
    for (int q = 0; q < 3; ++q) {
      rcols.push_back(hp.node_to_active[static_cast<size_t>(nodes[q])]);
      rvals.push_back(rec[q]);
    }
    row_ptr[static_cast<size_t>(P + e) + 1] = static_cast<int32_t>(rcols.size());
  }
  for (int o = 0; o < O; ++o) {
    const double* rec = orec.data() + static_cast<size_t>(o) * kOdomRec;
    const int fi = hp.odom_ij[2 * static_cast<size_t>(o)];
    const int fj = hp.odom_ij[2 * static_cast<size_t>(o) + 1];
    for (int r = 0; r < 3; ++r) {
      const int row = P + E + 3 * o + r;
      out.residuals[static_cast<size_t>(row)] = rec[r];
      std::vector<std::pair<int, double>> ent;
      if (fi >= 1) {
        for (int c = 0; c < 3; ++c) {
          ent.emplace_back(A + 3 * (fi - 1) + c, rec[3 + 3 * r + c]);
        }
      }
      for (int c = 0; c < 3; ++c) {
        ent.emplace_back(A + 3 * (fj - 1) + c, rec[12 + 3 * r + c]);
      }
      std::sort(ent.begin(), ent.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      for (const auto& pr : ent) {
        rcols.push_back(pr.first);
        rvals.push_back(pr.second);
      }
      row_ptr[static_cast<size_t>(row) + 1] = static_cast<int32_t>(rcols.size());
    }
  }
  // J as CSC (rows ascending per column)
  out.j_outer.assign(static_cast<size_t>(np) + 1, 0);
  for (const int c : rcols) {
    ++out.j_outer[static_cast<size_t>(c) + 1];
  }
  for (int c = 0; c < np; ++c) {
    out.j_outer[static_cast<size_t>(c) + 1] += out.j_outer[static_cast<size_t>(c)];
  }
  out.j_inner.resize(rcols.size());
  out.j_values.resize(rcols.size());
  {
    std::vector<int32_t> fill(out.j_outer.begin(), out.j_outer.end() - 1);
    for (int r = 0; r < nrows; ++r) {
      for (int p = row_ptr[static_cast<size_t>(r)]; p < row_ptr[static_cast<size_t>(r) + 1]; ++p) {
        const int c = rcols[static_cast<size_t>(p)];
        const int dst = fill[static_cast<size_t>(c)]++;
        out.j_inner[static_cast<size_t>(dst)] = r;
        out.j_values[static_cast<size_t>(dst)] = rvals[static_cast<size_t>(p)];
      }
    }
  }
  // structural J^T J (+ inserted diagonal) with values read from the fronts
  out.n_outer.assign(static_cast<size_t>(np) + 1, 0);
  std::vector<char> mark(static_cast<size_t>(np), 0);
  std::vector<int32_t> idx;
  for (int j = 0; j < np; ++j) {
    idx.clear();
    for (int q = out.j_outer[static_cast<size_t>(j)]; q < out.j_outer[static_cast<size_t>(j) + 1]; ++q) {
      const int r = out.j_inner[static_cast<size_t>(q)];
      for (int p = row_ptr[static_cast<size_t>(r)]; p < row_ptr[static_cast<size_t>(r) + 1]; ++p) {
        const int c = rcols[static_cast<size_t>(p)];
        if (mark[static_cast<size_t>(c)] == 0) {
          mark[static_cast<size_t>(c)] = 1;
          idx.push_back(c);
        }
      }
    }
    if (mark[static_cast<size_t>(j)] == 0) {
      mark[static_cast<size_t>(j)] = 1;
      idx.push_back(j);
    }
    std::sort(idx.begin(), idx.end());
    for (const int c : idx) {
      mark[static_cast<size_t>(c)] = 0;
      const int pa = sym_.pinv[static_cast<size_t>(L.col_off + c)];
      const int pb = sym_.pinv[static_cast<size_t>(L.col_off + j)];
      const int hi = std::max(pa, pb);
      const int lo = std::min(pa, pb);
      const SupernodeRec& rec = sym_.sn[static_cast<size_t>(sym_.col_owner[static_cast<size_t>(lo)])];
      const int li = FrontIndex(sym_, rec, hi);
      double v = 0.0;
      if (li >= 0) {
        v = fronts[static_cast<size_t>(rec.front_off + static_cast<int64_t>(lo - rec.first_col) * rec.F + li)];
      }
      out.n_inner.push_back(c);
      out.n_values.push_back(v);
    }
    out.n_outer[static_cast<size_t>(j) + 1] = static_cast<int32_t>(out.n_inner.size());
  }
  out.rhs = rhs;
  if (compute_step) {
    LaunchFactor();
    LaunchSolve();
    const std::vector<int32_t> st = DownloadStatus();
    if ((st[static_cast<size_t>(i)] & kStatusZeroPivot) != 0) {
      std::vector<int32_t> ones(I, 1);
      SetActive(ones);
      Fail(SDFGPU_ERR_NUMERICAL, "sparse Cholesky factorization failed");
    }
    out.step.resize(static_cast<size_t>(np));
    CudaCheck(cudaMemcpyAsync(out.step.data(), step_.get() + L.col_off, out.step.size() * 8, cudaMemcpyDeviceToHost, s),
              "step");
    CudaCheck(cudaStreamSynchronize(s), "step sync");
  }
  std::vector<int32_t> ones(I, 1);
  SetActive(ones);
  CudaCheck(cudaStreamSynchronize(s), "lin done");
  lin_ = std::move(out);
}

void Engine::LinearizationSizes(int64_t* sizes) const {
  if (lin_.instance < 0) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "no linearization computed");
  }
  sizes[0] = static_cast<int64_t>(lin_.residuals.size());
  sizes[1] = static_cast<int64_t>(lin_.rhs.size());
  sizes[2] = static_cast<int64_t>(lin_.j_inner.size());
  sizes[3] = static_cast<int64_t>(lin_.n_inner.size());
}

void Engine::LinearizationGet(double* residuals, int32_t* point_cell, int32_t* j_outer, int32_t* j_inner,
                              double* j_values, int32_t* n_outer, int32_t* n_inner, double* n_values,
                              double* rhs, double* step) const {
  if (lin_.instance < 0) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "no linearization computed");
  }
  auto cp = [](auto* dst, const auto& v) {
    if (dst != nullptr && !v.empty()) {
      std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    }
  };
  cp(residuals, lin_.residuals);
  cp(point_cell, lin_.point_cell);
  cp(j_outer, lin_.j_outer);
  cp(j_inner, lin_.j_inner);
  cp(j_values, lin_.j_values);
  cp(n_outer, lin_.n_outer);
  cp(n_inner, lin_.n_inner);
  cp(n_values, lin_.n_values);
  cp(rhs, lin_.rhs);
  if (step != nullptr && lin_.step.empty()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "step was not computed");
  }
  cp(step, lin_.step);
}

void Engine::BeginSolve(const std::vector<sdfgpu_solver_options>& options) {
  const size_t I = host_.size();
  {
    std::vector<int32_t> mixed(I, 0);
    std::vector<double> tol(I, kDefaultRefineTol);
    int refine = 0;
    for (size_t i = 0; i < I; ++i) {
      if (options[i].precision == SDFGPU_PRECISION_MIXED) {
        mixed[i] = 1;
        refine = std::max(refine, options[i].refine_steps);
        tol[i] = options[i].refine_tolerance;
      }
    }
    SetMode(mixed, refine, tol);
  }
  t_start_ = std::chrono::steady_clock::now();
  times_ = IterTimes{};
  lm_.assign(I, LmInst{});
  span_started_ = false;
  need_backup_ = false;
  iter_ = 0;
  h_seg_.Alloc(5 * I);
  h_status_.Alloc(I);
  SetActive(std::vector<int32_t>(I, 1));
  std::vector<double> cost0;
  LaunchCost(cost0);
  for (size_t i = 0; i < I; ++i) {
    LmInst& L = lm_[i];
    L.opt = options[i];
    L.lam = L.opt.lambda_init;
    L.prev = cost0[i];
    L.nu = 2.0;
    L.active = L.opt.max_iterations > 0 ? 1 : 0;
    L.res = sdfgpu_solve_result{};
    L.res.initial_cost = cost0[i];
    L.hist.assign(1, cost0[i]);
    need_backup_ = need_backup_ || L.opt.reject_worse_steps != 0 || L.opt.trust_region != 0;
  }
}

bool Engine::SolveDone() const {
  for (const LmInst& L : lm_) {
    if (L.active != 0 && iter_ < L.opt.max_iterations) {
      return false;
    }
  }
  return true;
}

void Engine::EnqueuePhase(int phase) {
  switch (phase) {
    case 0: {
      const size_t I = host_.size();
      CudaCheck(cudaMemcpyAsync(active_.get(), h_active_.get(), I * sizeof(int32_t), cudaMemcpyHostToDevice, stream_),
                "active");
      CudaCheck(cudaMemcpyAsync(lam_.get(), h_lam_.get(), I * sizeof(double), cudaMemcpyHostToDevice, stream_),
                "lambda");
      CudaCheck(cudaMemcpyAsync(marq_.get(), h_marq_.get(), I * sizeof(int32_t), cudaMemcpyHostToDevice, stream_),
                "marquardt");
      ClearStatus();
      LaunchRows();
      break;
    }
    case 1:
      LaunchNormal();
      break;
    case 2:
      // the timed launches of phases 2 and 3 are recorded afresh
      timer_.NewSequence();
      timing_phase_ = true;
      LaunchFactor();
      timing_phase_ = false;
      break;
    case 3:
      timing_phase_ = true;
      LaunchSolve();
      timing_phase_ = false;
      break;
    default:
      LaunchStepAndCost(need_backup_);
      break;
  }
}

void Engine::LaunchIteration() {
  const size_t I = host_.size();
  // the previous iteration (and any copy reading the pinned parameters) has
  // finished: FinishIteration synchronised the stream
  for (size_t i = 0; i < I; ++i) {
    LmInst& L = lm_[i];
    if (L.active != 0 && iter_ >= L.opt.max_iterations) {
      L.active = 0;
    }
    h_active_[i] = L.active;
    h_lam_[i] = L.lam;
    h_marq_[i] = L.opt.marquardt_scaling != 0 ? 1 : 0;
  }
  if (!span_started_) {
    CudaCheck(cudaEventRecord(span_[0], stream_), "event");
    span_started_ = true;
  }
  for (size_t i = 0; i < I; ++i) {
    iters_[i] += h_active_[i] != 0 ? 1 : 0;
  }
  StepSpeculations();
  // a state that left its pattern is re-analysed before it is linearized
  ReanalyzePending();
  EnqueueIteration();
}

void Engine::EnqueueIteration() {
  if (use_graph_ && (graph_exec_[0] == nullptr || graph_backup_ != need_backup_)) {
    const auto t0 = std::chrono::steady_clock::now();
    DropGraph();
    const int64_t before = times_.launches;
    for (int phase = 0; phase < 5; ++phase) {
      cudaGraph_t graph = nullptr;
      CudaCheck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
      try {
        EnqueuePhase(phase);
      } catch (...) {
        cudaStreamEndCapture(stream_, &graph);
        if (graph != nullptr) {
          cudaGraphDestroy(graph);
        }
        DropGraph();
        throw;
      }
      CudaCheck(cudaStreamEndCapture(stream_, &graph), "end capture");
      const cudaError_t e = cudaGraphInstantiate(&graph_exec_[phase], graph, 0);
      cudaGraphDestroy(graph);
      CudaCheck(e, "graph instantiate");
    }
    graph_launches_ = times_.launches - before;
    times_.launches = before;
    graph_backup_ = need_backup_;
    times_.capture_host += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  for (int phase = 0; phase < 5; ++phase) {
    CudaCheck(cudaEventRecord(ev_[phase], stream_), "event");
    if (use_graph_) {
      CudaCheck(cudaGraphLaunch(graph_exec_[phase], stream_), "graph launch");
    } else {
      EnqueuePhase(phase);
    }
  }
  CudaCheck(cudaEventRecord(ev_[5], stream_), "event");
  if (use_graph_) {
    times_.launches += graph_launches_;
  }
}

bool Engine::IterationReady() const {
  const cudaError_t e = cudaEventQuery(ev_[5]);
  if (e == cudaErrorNotReady) {
    return false;
  }
  CudaCheck(e, "iteration event");
  return true;
}

void Engine::FinishIteration() {
  const size_t I = host_.size();
  CudaCheck(cudaStreamSynchronize(stream_), "iteration");
  CheckWaits(h_status_.get(), I);
  std::vector<int> overflow;
  for (size_t i = 0; i < I; ++i) {
    if (lm_[i].active != 0 && (h_status_[i] & kStatusPatternOverflow) != 0) {
      overflow.push_back(static_cast<int>(i));
    }
  }
  if (!overflow.empty()) {
    // A point left its pose's analysed cell set (a state the look-ahead of
    // the cost kernel did not see, e.g. one set by the caller): the step
    // kernel skipped these instances. Re-analyse them at the current state
    // and run the iteration again for them alone; the other instances keep
    // the results (and the applied steps) of the first run.
    std::vector<double> seg(h_seg_.get(), h_seg_.get() + 5 * I);
    std::vector<int32_t> st(h_status_.get(), h_status_.get() + I);
    const size_t F = static_cast<size_t>(total_frames_);
    std::vector<double> pre(h_theta_pre_.get(), h_theta_pre_.get() + F);
    std::vector<int32_t> upd(h_theta_upd_.get(), h_theta_upd_.get() + F);
    Reanalyze(overflow);
    std::fill(h_active_.get(), h_active_.get() + I, 0);
    for (const int i : overflow) {
      h_active_[i] = 1;
    }
    EnqueueIteration();
    CudaCheck(cudaStreamSynchronize(stream_), "iteration");
    CheckWaits(h_status_.get(), I);
    std::vector<char> rerun(I, 0);
    for (const int i : overflow) {
      rerun[static_cast<size_t>(i)] = 1;
      if ((h_status_[i] & kStatusPatternOverflow) != 0) {
        Fail(SDFGPU_ERR_CUDA, "sparsity pattern still overflows after re-analysis");
      }
    }
    for (size_t f = 0; f < F; ++f) {
      if (rerun[static_cast<size_t>(frame_inst_host_[f])] == 0) {
        // the first run's moved angles of the instances it kept
        h_theta_pre_[f] = pre[f];
        h_theta_upd_[f] = upd[f];
      }
    }
    for (size_t i = 0; i < I; ++i) {
      if (rerun[i] == 0) {
        h_seg_[3 * i] = seg[3 * i];
        h_seg_[3 * i + 1] = seg[3 * i + 1];
        h_seg_[3 * i + 2] = seg[3 * i + 2];
        h_seg_[3 * I + i] = seg[3 * I + i];
        h_seg_[4 * I + i] = seg[4 * I + i];
        h_status_[i] = st[i];
      }
    }
  }
  float ms = 0.0f;
  double* acc[5] = {&times_.assemble, &times_.normal, &times_.factor, &times_.solve, &times_.update};
  for (int q = 0; q < 5; ++q) {
    CudaCheck(cudaEventElapsedTime(&ms, ev_[q], ev_[q + 1]), "phase timing");
    *acc[q] += ms * 1e-3;
  }
  timer_.Accumulate();
  ++times_.iterations;
  bool any_revert = false;
  std::vector<int32_t> revert(I, 0);
  for (size_t i = 0; i < I; ++i) {
    LmInst& L = lm_[i];
    if (L.active == 0) {
      continue;
    }
    const double cost = (h_seg_[3 * i] + h_seg_[3 * i + 1]) + h_seg_[3 * i + 2];
    const double sq = h_seg_[3 * I + i];
    const double pred = h_seg_[4 * I + i];
    if ((h_status_[i] & kStatusZeroPivot) != 0) {
      // lm_solver.cpp:354-362: the factorization failure ends the solve
      // before ApplyStep (the step kernel skipped this instance).
      L.res.status = SDFGPU_ERR_NUMERICAL;
      L.active = 0;
      continue;
    }
    L.res.iterations = iter_ + 1;
    if (std::sqrt(sq) < L.opt.step_tolerance) {
      L.hist.push_back(cost);
      L.res.final_cost = cost;
      L.res.converged = 1;
      L.active = 0;
      continue;
    }
    double current = cost;
    if (L.opt.trust_region != 0) {
      const double rho = pred > 0.0 ? (L.prev - cost) / pred : -1.0;
      if (rho > 0.0) {
        L.prev = cost;
        const double shrink = 1.0 - std::pow(2.0 * rho - 1.0, 3);
        L.lam = std::max(L.lam * std::max(1.0 / 3.0, shrink), 1e-7);
        L.nu = 2.0;
      } else {
        revert[i] = 1;
        any_revert = true;
        current = L.prev;
        L.lam *= L.nu;
        L.nu *= 2.0;
      }
    } else if (cost < L.prev) {
      L.lam /= L.opt.lambda_factor;
      L.prev = cost;
    } else {
      L.lam *= L.opt.lambda_factor;
      if (L.opt.reject_worse_steps != 0) {
        revert[i] = 1;
        any_revert = true;
        current = L.prev;
      } else {
        L.prev = cost;
      }
    }
    L.hist.push_back(current);
    L.res.final_cost = current;
  }
  for (size_t i = 0; i < I; ++i) {
    // the accepted state lies outside the pattern: analyse before the next
    // linearization (a reverted state is the one just linearized)
    if (h_active_[i] != 0 && (h_status_[i] & kStatusNextOverflow) != 0 && revert[i] == 0 &&
        (h_status_[i] & kStatusZeroPivot) == 0) {
      pending_.push_back(static_cast<int>(i));
    } else if (h_active_[i] != 0 && (h_status_[i] & kStatusNearEdge) != 0 && revert[i] == 0 &&
               (h_status_[i] & kStatusZeroPivot) == 0) {
      near_.push_back(static_cast<int>(i));
    }
  }
  if (any_revert) {
    CudaCheck(cudaMemcpyAsync(revert_.get(), revert.data(), revert.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                              stream_),
              "revert mask");
    const int64_t big = std::max<int64_t>(total_nodes_, 3 * static_cast<int64_t>(total_frames_));
    KBackup<<<Blocks(big, 256), 256, 0, stream_>>>(V_, 1, revert_.get());
    CudaCheck(cudaGetLastError(), "restore");
    // the revert mask is read by the kernel; keep the host copy alive
    CudaCheck(cudaStreamSynchronize(stream_), "restore");
  }
  // the accepted steps' angles with the reference's bits
  CommitAngles(&revert);
  ++iter_;
}

bool Engine::InstanceDone(int i) const {
  const LmInst& L = lm_[static_cast<size_t>(i)];
  return L.active == 0 || iter_ >= L.opt.max_iterations;
}

sdfgpu_solve_result Engine::InstanceResult(int i) const {
  const LmInst& L = lm_[static_cast<size_t>(i)];
  sdfgpu_solve_result r = L.res;
  if (r.iterations == 0) {
    r.final_cost = r.initial_cost;
  }
  r.duration_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start_).count();
  r.cost_history_length = static_cast<int32_t>(L.hist.size());
  return r;
}

void Engine::EndSolve(sdfgpu_solve_result* results, double* cost_history, int capacity) {
  const size_t I = host_.size();
  if (span_started_) {
    CudaCheck(cudaEventRecord(span_[1], stream_), "event");
  }
  SetActive(std::vector<int32_t>(I, 1));
  CudaCheck(cudaStreamSynchronize(stream_), "solve done");
  if (span_started_) {
    float ms = 0.0f;
    CudaCheck(cudaEventElapsedTime(&ms, span_[0], span_[1]), "span");
    times_.span = ms * 1e-3;
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start_).count();
  for (size_t i = 0; i < I; ++i) {
    LmInst& L = lm_[i];
    if (L.res.iterations == 0) {
      L.res.final_cost = L.res.initial_cost;
    }
    L.res.duration_seconds = secs;
    const int len = static_cast<int>(L.hist.size());
    L.res.cost_history_length = std::min(len, capacity);
    if (cost_history != nullptr) {
      for (int q = 0; q < L.res.cost_history_length; ++q) {
        cost_history[i * static_cast<size_t>(capacity) + static_cast<size_t>(q)] = L.hist[static_cast<size_t>(q)];
      }
    }
    results[i] = L.res;
  }
}

void Engine::Solve(const std::vector<sdfgpu_solver_options>& options, sdfgpu_solve_result* results,
                   double* cost_history, int capacity) {
  BeginSolve(options);
  while (!SolveDone()) {
    LaunchIteration();
    FinishIteration();
  }
  EndSolve(results, cost_history, capacity);
}

}  // namespace sdfgpu
