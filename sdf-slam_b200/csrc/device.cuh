// Device-side data view shared by the assembly, factorization and solve
// kernels of the sdfgpu library.
#pragma once

#include <cstdint>

#include "internal.h"

namespace sdfgpu {

/// Per-instance constants (device copy of InstanceLayout plus schedule data).
struct InstDev {
  int32_t nx, ny;
  double min_x, min_y, dx, dy;
  int64_t node_off;
  int64_t cell_off;
  int32_t col_off;
  int32_t num_active;
  int32_t num_frames;
  int32_t frame_off;
  int64_t pt_off;
  int32_t num_points;
  int64_t eik_off;
  int32_t num_eik;
  int64_t odom_off;
  int32_t num_odom;
  int32_t smooth_gradient;
  double smooth_gradient_step;
  double huber_delta;
  int64_t allow_off;
  int32_t allow_words;
  int32_t pp_ld;
  int64_t pp_base;
  int32_t pp_first;
  int32_t num_params;
  int32_t mixed;  // 1: this solve factors the grid supernodes in FP32
  // mixed: refinement of the step stops once its largest correction is at
  // most this fraction of its largest entry
  double refine_tol;
  // cells probed around each point by the cost kernel for kStatusNearEdge
  // (0: no probe)
  int32_t near_cells;
};

/// Status bits per instance.
constexpr int kStatusZeroPivot = 1;
constexpr int kStatusPatternOverflow = 2;
// set by the cost kernel: at the state it evaluated, a point lies outside its
// pose's analysed cell set (the next linearization would overflow)
constexpr int kStatusNextOverflow = 4;
/// A wait on another block's flag ran out of its limit (the results of the
/// launch are not valid).
constexpr int kStatusWaitTimeout = 8;
// set by the cost kernel: at the state it evaluated, a point lies within
// near_cells cells of its pose's analysed cell set's edge (the pattern is
// re-centred ahead of time, in the background)
constexpr int kStatusNearEdge = 16;

/// Per point row record: 4 node Jacobian entries, 3 pose entries, residual.
constexpr int kPointRec = 8;
/// Per Eikonal row record: 3 node entries, residual.
constexpr int kEikRec = 4;
/// Per odometry spec: residual[3], d_pose_i[3][3], d_pose_j[3][3] (scaled).
constexpr int kOdomRec = 24;

struct DeviceView {
  // problem (static between uploads)
  const InstDev* inst;
  int32_t num_inst;
  int64_t total_nodes;
  int64_t total_cells;
  int32_t total_frames;
  int64_t total_points;
  int64_t total_eik;
  int64_t total_odom;
  int32_t n;  // total columns
  const int32_t* node_col;       // global node -> global natural column or -1
  const int32_t* col_node;       // global natural column -> global node, or -1 for poses
  const int32_t* col_inst;       // global natural column -> instance
  const int32_t* frame_inst;     // global frame -> instance
  const int32_t* frame_col;      // global frame -> global natural column of x (or -1, frame 0)
  const int32_t* pt_frame;       // global frame id
  const double2* pt_xy;
  const double* pt_exp;
  const double* pt_sw;
  const int32_t* eik_node;       // global node of (w, h)
  const double2* eik_n;
  const double* eik_sw;
  const int32_t* eik_index;      // global node -> Eikonal spec whose (w,h) it is, or -1
  const int32_t* odom_fi;        // global frames
  const int32_t* odom_fj;
  const double* odom_meas;       // 3 per spec
  const double* odom_sw;
  const int64_t* frame_rows_ptr; // per global frame + 1
  const int32_t* frame_rows;     // point rows of each frame, ascending
  const int64_t* frame_odom_ptr; // per global frame + 1
  const int32_t* frame_odom;     // 2*spec + role (0: frame is i, 1: frame is j)
  int32_t num_pairs;
  const int32_t* pair_f;         // smaller frame (global)
  const int32_t* pair_g;         // larger frame (global)
  const int64_t* pair_ptr;
  const int32_t* pair_spec;      // 2*spec + (1 if frame_i of the spec is the larger frame)
  // state
  double* map;
  double* poses;
  double* map_backup;
  double* poses_backup;
  // (cos, sin) of every frame's angle, computed on the host with the
  // platform's libm whenever a state is set or a step accepted (upload,
  // SetState, Engine::CommitAngles), so that every linearization rotates the
  // scan points with the reference's bits; a candidate state whose cost
  // decides the step holds correctly rounded device values until then
  double2* pose_cs;
  double2* pose_cs_backup;
  // ApplyStep hand-off: the unwrapped angle theta + delta of each frame the
  // step moved (theta_upd 1), and the host's wrapped angle, cos, sin and a
  // commit flag per frame
  double* theta_pre;
  int32_t* theta_upd;
  const double* theta_out;  // 4 per frame
  // per iteration
  double* pt_rec;                // kPointRec per point row
  int64_t* pt_poff;              // 4 per point row: front offsets of its (pose, corner node) blocks
  int32_t* pt_cell;              // global cell or -1
  double* eik_rec;
  double* odom_rec;
  int32_t* cell_start;           // total_cells + 1
  int32_t* cell_rows;            // point rows sorted by cell
  double* rhs;                   // natural order, -J^T r
  double* step;                  // natural order
  double* xs;                    // permuted solve vector
  double* lam;                   // per instance
  int32_t* marquardt;            // per instance
  int32_t* status;               // per instance
  int32_t* active;               // per instance: 1 while the instance is iterating
  // symbolic
  const int32_t* perm;
  const int32_t* pinv;
  const SupernodeRec* sn;
  const int32_t* sn_rows;
  const int32_t* sn_rel;
  const int32_t* child_list;
  const int64_t* mm_off;
  const int64_t* mp_ptr;
  const int32_t* mp_frame;
  const int64_t* mp_off;
  const uint32_t* allow_bits;
  double* fronts;     // factorization work fronts (FP64 supernodes)
  float* fronts32;    // factorization work fronts of FP32 supernodes (mixed solves), else null
  double* asm_fronts; // assembly target: the FP64 normal matrix (== fronts when no solve is mixed)
  double* upd;
  int32_t tc_schur;   // 1: the wide FP32 fronts' Schur complements run on the tensor cores
  // adaptive refinement of mixed steps: per instance 1 once its corrections
  // became negligible (null outside the refinement rounds), per instance the
  // largest |correction| and |step| of the round (bits of non-negative
  // doubles, ordered like the values), and whether any instance still refines
  int32_t* refine_done;
  unsigned long long* refine_max;
  int32_t* refine_left;
  // map-pose entries grouped by frame (transpose of mp_*): per global frame
  // the node columns coupled to it and the front offset of (pose var 0, node)
  const int64_t* fmp_ptr;
  const int32_t* fmp_col;
  const int64_t* fmp_off;
};

/// True when supernode S is factored in FP32 (a mixed solve's grid supernode).
__device__ __forceinline__ bool Fp32Front(const DeviceView& V, const SupernodeRec& S) {
  return V.fronts32 != nullptr && S.pose_root == 0 && V.inst[S.instance].mixed != 0;
}

}  // namespace sdfgpu
