/*
 * sdfgpu -- B200 (sm_100a) backend for the joint Levenberg-Marquardt path of
 * sdf-slam: point / hallucination / Eikonal / odometry residuals and
 * Jacobians, J^T J and -J^T r accumulation, damping, a supernodal LDL^T
 * factorization of the normal equations, the step, the state update and the
 * cost, driven by the reference's LM control logic.
 *
 * Plain C ABI: opaque handles, plain pointers and sizes, int status codes.
 * Every function returns SDFGPU_OK (0) or an SDFGPU_ERR_* code; the message of
 * the last failure on the calling thread is sdfgpu_last_error_message().
 * No exception crosses this boundary. Paths in the comments are files of the
 * reference repository (RobinJehn/sdf-slam) that each entry point replaces.
 *
 * Threading: a handle is used by one thread at a time; distinct handles may be
 * used from distinct threads. Calls are synchronous (they return after the
 * GPU work they start has finished), except for the serving queue, which has
 * its own worker thread.
 */
#ifndef SDFGPU_H_
#define SDFGPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDFGPU_OK 0
#define SDFGPU_ERR_INVALID_ARGUMENT 1 /* std::invalid_argument, problem.cpp:19-24,108-110,118-120 */
#define SDFGPU_ERR_NUMERICAL 2        /* "sparse Cholesky factorization failed", lm_solver.cpp:354-362 */
#define SDFGPU_ERR_OUT_OF_MEMORY 3    /* device allocation or admission budget exceeded */
#define SDFGPU_ERR_TIMEOUT 4          /* a bounded wait ran out */
#define SDFGPU_ERR_CUDA 5             /* any other CUDA runtime failure */
#define SDFGPU_ERR_NOT_READY 6        /* serving: the request has not finished yet */

/* Precision of a solve. FP64 runs every step in double precision (the plain
 * path that matches the reference). MIXED factors the grid supernodes in
 * FP32 (the dense pose-block root stays FP64) and recovers the FP64 step by
 * up to refine_steps rounds of iterative refinement against the FP64 normal
 * matrix, stopping once a round's correction falls below refine_tolerance;
 * residuals, J^T J, cost, gain ratio and acceptance stay FP64. */
#define SDFGPU_PRECISION_FP64 0
#define SDFGPU_PRECISION_MIXED 1

typedef struct sdfgpu_problem sdfgpu_problem; /* one or more independent problems */
typedef struct sdfgpu_ldlt sdfgpu_ldlt;       /* factor-only sparse LDL^T */
typedef struct sdfgpu_server sdfgpu_server;   /* serving queue */

/* Message of the last failure on this thread ("" when none). */
const char* sdfgpu_last_error_message(void);

/* Library version string. */
const char* sdfgpu_version(void);

/* Number of CUDA devices visible to the library (0 when none; never fails). */
int32_t sdfgpu_device_count(void);

/* --------------------------------------------------------------- problem --
 * Flat arrays of everything the LM path reads from sdf_slam::Problem: the
 * public getters map(), poses(), point_specs(), eikonal_specs(), odom_specs(),
 * NodeColumn(), huber_delta(), smooth_gradient(), smooth_gradient_step()
 * (src/problem/problem.hpp:104-142). The grid follows GridMap
 * (src/core/grid_map.hpp:13-23): node (w, h) has id h*nx + w, spacing
 * (max - min) / (n - 1). Arrays are copied; the caller keeps ownership. */
typedef struct sdfgpu_problem_desc {
  int32_t nx;
  int32_t ny;
  double min_x;
  double min_y;
  double max_x;
  double max_y;
  const double* map_values;          /* nx*ny */
  int32_t num_frames;
  const double* poses;               /* num_frames*3: x, y, theta; frame 0 is fixed */
  int32_t num_points;                /* PointSpec, problem.hpp:28-33 */
  const int32_t* point_frame;        /* num_points */
  const double* point_xy;            /* num_points*2, sensor frame */
  const double* point_expected;      /* num_points: expected SDF (0 for scan points) */
  const double* point_sqrt_weight;   /* num_points */
  int32_t num_eikonal;               /* EikonalSpec, problem.hpp:36-41 */
  const int32_t* eikonal_wh;         /* num_eikonal*2 */
  const double* eikonal_normal;      /* num_eikonal*2 */
  const double* eikonal_sqrt_weight; /* num_eikonal */
  int32_t num_odom;                  /* OdomSpec, problem.hpp:45-50 (odometry then relations) */
  const int32_t* odom_ij;            /* num_odom*2: frame_i, frame_j */
  const double* odom_meas;           /* num_odom*3: x, y, theta */
  const double* odom_sqrt_weight;    /* num_odom */
  const int32_t* node_to_active;     /* nx*ny: state column of each node or -1 (NodeColumn) */
  double huber_delta;                /* 0 disables */
  int32_t smooth_gradient;
  double smooth_gradient_step;
} sdfgpu_problem_desc;

/* ProblemOptions (src/problem/problem.hpp:63-87, with Weights :16-25,
 * HallucinationOptions src/core/hallucination.hpp:17-23 and NormalOptions
 * src/core/normals.hpp:44-57). normals_method: 0 pca, 1 hybrid, 2 weighted. */
typedef struct sdfgpu_problem_options {
  double weight_scan;
  double weight_hallucination;
  double weight_eikonal;
  double weight_odometry;
  double weight_relation;
  int32_t hallucination_points_per_scan_point;
  double hallucination_step_size;
  int32_t hallucination_both_directions;
  int32_t normals_method;
  int32_t normals_k_neighbors;
  int32_t normals_per_scan;
  double normals_corner_threshold;
  double huber_delta;
  int32_t smooth_gradient;
  double smooth_gradient_step;
  int32_t active_region;
  int32_t active_margin;
} sdfgpu_problem_options;

/* Reference defaults of ProblemOptions. */
void sdfgpu_problem_options_default(sdfgpu_problem_options* options);

/* Problem::Problem (src/problem/problem.cpp:11-115): builds the point specs
 * (scan points, then hallucinated points, frame by frame), the active-region
 * index maps, the Eikonal specs from k-NN PCA normals and the odometry and
 * relation specs, then uploads the problem. scan_offsets has num_frames + 1
 * entries into scan_xy (2 doubles per point). odometry holds num_odometry
 * relative poses (0 or num_frames - 1). Relations whose frame_j is not below
 * num_frames are skipped; frames must satisfy 0 <= i < j. */
int sdfgpu_problem_build(int32_t nx, int32_t ny, double min_x, double min_y, double max_x,
                         double max_y, const double* map_values, int32_t num_frames,
                         const double* poses, const int32_t* scan_offsets, const double* scan_xy,
                         const double* odometry, int32_t num_odometry, int32_t num_relations,
                         const int32_t* relation_ij, const double* relation_meas,
                         const double* relation_sqrt_weight, const sdfgpu_problem_options* options,
                         sdfgpu_problem** out);

/* sdfgpu_problem_build with the point specs (scan rows, then hallucinated
 * rows, frame by frame; src/core/hallucination.cpp:5-28), the active-region
 * maps (problem.cpp:39-70), the k-NN PCA scan normals and per-node normals
 * (normals.cpp:70-220) and the Eikonal spec list (problem.cpp:79-94)
 * computed by CUDA kernels on the current device (the k-NN bucket grids are
 * built on the host). The resulting problem is the one sdfgpu_problem_build
 * returns, bit for bit. Fails with SDFGPU_ERR_CUDA when no device is usable
 * and with SDFGPU_ERR_INVALID_ARGUMENT for normals.k_neighbors above 64 or
 * non-finite poses or scan points. */
int sdfgpu_problem_build_device(int32_t nx, int32_t ny, double min_x, double min_y, double max_x,
                                double max_y, const double* map_values, int32_t num_frames,
                                const double* poses, const int32_t* scan_offsets,
                                const double* scan_xy, const double* odometry,
                                int32_t num_odometry, int32_t num_relations,
                                const int32_t* relation_ij, const double* relation_meas,
                                const double* relation_sqrt_weight,
                                const sdfgpu_problem_options* options, sdfgpu_problem** out);

/* Copies a problem given by its spec arrays (the drop-in path: the caller's
 * own Problem is marshalled into a desc). Validation and spec queries run on
 * the host; the first call that needs the GPU (cost, step, solve, state,
 * linearization) uploads the problem to the current CUDA device and fails
 * with SDFGPU_ERR_CUDA when there is none. */
int sdfgpu_problem_create(const sdfgpu_problem_desc* desc, sdfgpu_problem** out);

/* Several independent problems solved together: every kernel of an LM
 * iteration covers all of them in one launch (persistent level schedule of
 * the factorization, one graph per iteration). */
int sdfgpu_problem_create_batch(const sdfgpu_problem_desc* descs, int32_t count,
                                sdfgpu_problem** out);

/* Frees the handle and its device memory. Accepts NULL. */
int sdfgpu_problem_destroy(sdfgpu_problem* problem);

/* No counterpart in the reference (whose solver allocates through Eigen and
 * CHOLMOD on the host). Device blocks released by handles stay cached in the
 * library (by size class, up to 8 GB) and in its own memory pool on the
 * current device, so that the next handle allocates without cudaMalloc.
 * This returns both to the driver; call it with no handle's work in flight
 * on the current device when the host application needs the memory. */
int sdfgpu_release_cached_memory(void);

/* No counterpart in the reference. Measures the current device's FP64
 * fused-multiply-add throughput (TFLOP/s, best of five timed launches of
 * independent FMA chains on every SM); the roofline denominator for the FP64
 * factorization kernels. Synchronous. */
int sdfgpu_measure_fp64_peak(double* tflops);

/* No counterpart in the reference: a test hook for the failure path of the
 * one-launch triangular solve, whose blocks wait on flags that other blocks
 * publish. From the next solve on, supernode `withhold_front` (an index into
 * the handle's current symbolic structure) never publishes its forward flag
 * and every wait gives up after `wait_polls` polls (0: the default of about
 * a second); the wait that runs out ends the solve with SDFGPU_ERR_TIMEOUT,
 * the state is not moved and the device stays usable. withhold_front = -1
 * restores normal solves. */
int sdfgpu_debug_solve_fault(sdfgpu_problem* problem, int32_t withhold_front, uint32_t wait_polls);
/* Supernodes of the handle's current symbolic structure (0 before its first
 * device use). */
int32_t sdfgpu_debug_supernode_count(sdfgpu_problem* problem);

/* No counterpart in the reference: device time per kernel class of the
 * handle's LM iterations. From the next iteration on, CUDA events on the
 * handle's stream bracket every launch of the factorization and solve kernel
 * classes in `class_mask` (bit c for class c, named by
 * sdfgpu_kernel_class_name(c)); the totals restart at zero. 0 stops the
 * timing. sdfgpu_kernel_times returns, per class since then, the device
 * milliseconds, the launches and the algorithmic work of those launches
 * (useful flops, 2 per multiply-add; bytes for the classes for which
 * sdfgpu_kernel_class_is_memory_bound is 1); count <= SDFGPU_KERNEL_CLASSES,
 * any output may be NULL. */
#define SDFGPU_KERNEL_CLASSES 10
int sdfgpu_kernel_timing(sdfgpu_problem* problem, uint32_t class_mask);
int sdfgpu_kernel_times(sdfgpu_problem* problem, double* ms, int64_t* launches, double* work, int32_t count);
const char* sdfgpu_kernel_class_name(int32_t kernel_class);
int32_t sdfgpu_kernel_class_is_memory_bound(int32_t kernel_class);

/* Number of instances in the handle (1 unless created as a batch). */
int32_t sdfgpu_problem_count(const sdfgpu_problem* problem);

/* sizes[0..8] of instance `index`: num_points, num_eikonal, num_odom,
 * num_active_nodes, num_parameters, num_residuals, num_frames, nx, ny. */
int sdfgpu_problem_sizes(const sdfgpu_problem* problem, int32_t index, int32_t* sizes);

/* Copies the spec arrays of instance `index` out (any pointer may be NULL). */
int sdfgpu_problem_get_specs(const sdfgpu_problem* problem, int32_t index, int32_t* point_frame,
                             double* point_xy, double* point_expected, double* point_sqrt_weight,
                             int32_t* eikonal_wh, double* eikonal_normal,
                             double* eikonal_sqrt_weight, int32_t* odom_ij, double* odom_meas,
                             double* odom_sqrt_weight, int32_t* node_to_active);

/* problem.map().values() and problem.poses() of instance `index`. */
int sdfgpu_get_state(sdfgpu_problem* problem, int32_t index, double* map_values, double* poses);
int sdfgpu_set_state(sdfgpu_problem* problem, int32_t index, const double* map_values,
                     const double* poses);

/* Problem::Cost (src/problem/problem.cpp:132-156) at the current state. */
int sdfgpu_cost(sdfgpu_problem* problem, int32_t index, double* cost);

/* Problem::ApplyStep (src/problem/problem.cpp:117-130); step has
 * num_parameters entries (active node values, then x, y, theta of frames
 * 1..N-1). */
int sdfgpu_apply_step(sdfgpu_problem* problem, int32_t index, const double* step);

/* ------------------------------------------------------------------- LM ---
 * SolverOptions / SolveResult (src/solvers/solver.hpp:29-64). */
typedef struct sdfgpu_solver_options {
  int32_t max_iterations;
  double step_tolerance;
  double lambda_init;
  double lambda_factor;
  int32_t reject_worse_steps;
  int32_t marquardt_scaling;
  int32_t trust_region;
  int32_t num_threads; /* accepted for interface parity; unused on the GPU */
  int32_t precision;   /* SDFGPU_PRECISION_* */
  int32_t refine_steps; /* MIXED: refinement rounds per LM step (0..16) */
  /* MIXED: a step's refinement stops once its largest correction is at
   * most this fraction of its largest entry ([0, 1); default 1e-13, where
   * the refined step agrees with the FP64 path's to its own rounding). The
   * step's error after the last round is about this fraction times the
   * error reduction of one round (cond(A) * 2^-24). */
  double refine_tolerance;
} sdfgpu_solver_options;

typedef struct sdfgpu_solve_result {
  int32_t converged;
  int32_t iterations;
  double initial_cost;
  double final_cost;
  double duration_seconds;
  int32_t cost_history_length; /* entries written to cost_history (<= capacity) */
  int32_t status;              /* SDFGPU_OK or the instance's own error code */
} sdfgpu_solve_result;

/* Reference defaults of SolverOptions. */
void sdfgpu_solver_options_default(sdfgpu_solver_options* options);

/* SolveLm (src/solvers/lm_solver.cpp:201-434) behind Solve's dispatch
 * (:436-444) as SolverBackend::kGpuLm. Mutates the state in place. options,
 * results and cost_history are per instance: options and results have
 * sdfgpu_problem_count() entries (options may be NULL for the defaults);
 * cost_history holds that many rows of `capacity` doubles (NULL to skip).
 * Returns the first non-OK instance status (SDFGPU_ERR_NUMERICAL when a
 * factorization failed; that instance stops before applying the step). */
int sdfgpu_solve(sdfgpu_problem* problem, const sdfgpu_solver_options* options,
                 sdfgpu_solve_result* results, double* cost_history, int32_t capacity);

/* --------------------------------------------------------- linearization --
 * One LM iteration's quantities at the current state, without moving it:
 * residuals and Jacobian (lm_solver.cpp:304-385), J^T J with damping
 * (:391-402), -J^T r (:403) and the step delta (:423-436). Sizes first, then
 * the copies; pattern buffers use the reference's layout (CSC of the full
 * symmetric normal matrix with sorted row indices; Jacobian as CSC). */
int sdfgpu_linearize(sdfgpu_problem* problem, int32_t index, double lambda, int32_t marquardt,
                     int32_t compute_step);

/* sizes[0..3]: num_rows, num_parameters, nnz(J), nnz(J^T J + damping). */
int sdfgpu_linearization_sizes(sdfgpu_problem* problem, int64_t* sizes);

/* Any pointer may be NULL. point_cell: per point row h*(nx)+w of its cell or
 * -1 outside the domain. */
int sdfgpu_linearization_get(sdfgpu_problem* problem, double* residuals, int32_t* point_cell,
                             int32_t* j_outer, int32_t* j_inner, double* j_values,
                             int32_t* n_outer, int32_t* n_inner, double* n_values, double* rhs,
                             double* step);

/* Timing breakdown of the last solve on this handle, measured with CUDA
 * events on the handle's stream, in seconds of GPU time per phase summed over
 * its iterations: [0] residuals + Jacobian + cell sort, [1] J^T J + J^T r,
 * [2] factorization, [3] triangular solves, [4] step + cost; [5] iterations;
 * [6] device time from the first iteration's start to the last one's end;
 * [7] kernels launched by the iterations; [8] useful FP64 flops of one
 * factorization; [9] symbolic re-analyses during the solve (a state left
 * the analysed sparsity pattern); [10] host seconds spent in those
 * re-analyses; [11] host seconds capturing the iteration's CUDA graphs.
 * phases must hold 12 doubles. */
int sdfgpu_last_profile(sdfgpu_problem* problem, double* phases);

/* Autotuner (no counterpart in the reference): times the factorization of
 * the handle's current normal matrix under each candidate schedule (the
 * pivot count up to which a front is factored by one kernel, that kernel's
 * rows per block, the rows per panel block of the wide fronts, 0 meaning
 * that each 128-column outer block is factored whole by one kernel) and
 * keeps the fastest for the
 * handle's later solves, also across pattern re-analyses. schedule (3
 * int32, may be NULL) receives the chosen one, factor_ms (may be NULL) its
 * factorization time; trials (may be NULL) receives up to max_trials rows
 * of 4 doubles (small_pivots, front_rows, panel_rows, ms). Returns the
 * number of candidates timed in *num_trials when not NULL. When the
 * handle's last solve was MIXED, the autotuner then times that solve's
 * factorization and refined triangular solves under the chosen schedule
 * with and without the tensor-core Schur complements of the wide FP32
 * fronts and keeps the faster (sdfgpu_tensor_core_choice). */
int sdfgpu_autotune(sdfgpu_problem* problem, int32_t* schedule, double* factor_ms, double* trials,
                    int32_t max_trials, int32_t* num_trials);

/* Installs the factorization schedule (small_pivots, front_rows,
 * panel_rows) for the handle's later solves, also across pattern
 * re-analyses (no counterpart in the reference; the autotuner's choice made
 * by hand). small_pivots 32..128, front_rows 128..256, panel_rows 0 (whole
 * outer blocks) or 16..128; SDFGPU_ERR_INVALID_ARGUMENT otherwise. */
int sdfgpu_set_schedule(sdfgpu_problem* problem, const int32_t* schedule);

/* The autotuner's tensor-core choice for mixed solves (no counterpart in
 * the reference): *min_rows receives the number of rows below the pivot
 * block from which a FP32 front's Schur complement runs on the tensor cores
 * (0: none does; 256 until an autotune of a mixed handle decides), ms_with
 * and ms_without (may be NULL) the mixed factor + solve times the last such
 * autotune measured (0 when it did not time that variant). */
int sdfgpu_tensor_core_choice(sdfgpu_problem* problem, int32_t* min_rows, double* ms_with, double* ms_without);

/* Installs that choice by hand (no counterpart in the reference): min_rows
 * 0 (no tensor-core Schur complements) or 128..65536; kept across pattern
 * re-analyses and schedule changes; SDFGPU_ERR_INVALID_ARGUMENT otherwise. */
int sdfgpu_set_tensor_core_choice(sdfgpu_problem* problem, int32_t min_rows);

/* ----------------------------------------------------------- incremental --
 * Run in incremental mode (src/pipeline/runner.cpp:226-285, without its file
 * output): the dataset's odometry is poses[i].RelativeTo(poses[i + 1]); frame
 * 0 starts at its dataset pose; each step appends increment_size frames,
 * composing each new pose from the previous one and the odometry, rebuilds
 * the problem over the frames so far from the current map and poses (as
 * sdfgpu_problem_build, or sdfgpu_problem_build_device when build_on_device
 * is set) and runs SolveLm with max_iterations = iterations_per_increment.
 * The step results are summed as the runner does: the first step's initial
 * cost, the last step's final cost and convergence, the iterations and
 * durations summed, the cost histories concatenated. With warm_analysis set,
 * the next step's symbolic analysis runs on a host thread during the
 * current step's GPU iterations, from the poses the step started with; the
 * iterations re-analyse if the solved poses leave that pattern. */
typedef void (*sdfgpu_snapshot_fn)(void* user, int32_t num_frames, const double* map_values,
                                   const double* poses);

typedef struct sdfgpu_incremental_desc {
  int32_t nx;
  int32_t ny;
  double min_x;
  double min_y;
  double max_x;
  double max_y;
  const double* map_values;      /* nx * ny initial SDF values, NULL: zeros */
  int32_t num_frames;            /* >= 2 */
  const double* poses;           /* dataset poses, 3 per frame */
  const int32_t* scan_offsets;   /* num_frames + 1 */
  const double* scan_xy;         /* sensor-frame points, 2 per point */
  int32_t num_relations;
  const int32_t* relation_ij;
  const double* relation_meas;
  const double* relation_sqrt_weight; /* NULL: 1 */
  int32_t increment_size;        /* frames appended per step, >= 1 */
  int32_t iterations_per_increment;
  int32_t snapshot_every;        /* call snapshot every N steps and after the last; 0: never */
  sdfgpu_snapshot_fn snapshot;   /* may be NULL */
  void* snapshot_user;
  int32_t build_on_device;
  int32_t warm_analysis;
} sdfgpu_incremental_desc;

/* Runs the incremental driver on the current device. map_out (nx * ny) and
 * poses_out (3 * num_frames) receive the final state, total the summed
 * result; cost_history (may be NULL) receives the first `capacity` entries
 * of the concatenated histories (total->cost_history_length of them).
 * phases (12 doubles, may be NULL): host seconds spent building problems,
 * waiting for overlapped analyses, setting the engine up, iterating, reading
 * state back and releasing the engine, the run's wall time, the number of
 * steps, the number of steps whose analysis overlapped the previous step,
 * the pattern re-analyses inside the iterations, their host seconds and the
 * host seconds spent capturing iteration graphs (both part of iterating).
 * Fails with the step's
 * status (SDFGPU_ERR_NUMERICAL for a failed factorization) and stops there. */
int sdfgpu_run_incremental(const sdfgpu_incremental_desc* desc, const sdfgpu_problem_options* problem_options,
                           const sdfgpu_solver_options* solver_options, double* map_out, double* poses_out,
                           sdfgpu_solve_result* total, double* cost_history, int32_t capacity,
                           double* phases);

/* -------------------------------------------------------------- outputs --
 * run_slam's output files (src/pipeline/runner.cpp:82-192), same formats:
 * poses as "x,y,theta" CSV with 17 significant digits (WritePoses :82-88);
 * the map as a "nx ny min_x min_y dx dy" line and ny lines of nx values
 * (WriteMap :90-99); every scan point at its frame's pose as "x,y" CSV with
 * 9 digits (WriteGlobalScanPoints :101-114); the result and, when metrics is
 * not NULL, the four trajectory errors as JSON (WriteJson :172-192). No GPU
 * is needed. */
int sdfgpu_write_poses(const char* path, const double* poses, int32_t num_frames);
int sdfgpu_write_map(const char* path, int32_t nx, int32_t ny, double min_x, double min_y, double max_x,
                     double max_y, const double* map_values);
int sdfgpu_write_scan_points(const char* path, int32_t num_frames, const double* poses,
                             const int32_t* scan_offsets, const double* scan_xy);
int sdfgpu_write_metrics(const char* path, const sdfgpu_solve_result* result, const double* metrics);

/* Evaluate (runner.cpp:145-170): metrics[0..3] = mean translation error, mean
 * |rotation error|, and the same two over consecutive relative poses, of the
 * estimated poses against ground truth (num_frames >= 2 each). */
int sdfgpu_evaluate_trajectory(const double* estimated, const double* ground_truth, int32_t num_frames,
                               double* metrics);

/* The scan points WarnIfPointsOutsideMap (runner.cpp:116-137) counts: those
 * whose global position lies outside the grid's domain, and all of them. */
int sdfgpu_points_outside_map(int32_t nx, int32_t ny, double min_x, double min_y, double max_x, double max_y,
                              int32_t num_frames, const double* poses, const int32_t* scan_offsets,
                              const double* scan_xy, int64_t* outside, int64_t* total);

/* ------------------------------------------------------------ factor only --
 * LinearSolver::kGpu: ParallelSimplicialLdlt's interface
 * (src/solvers/parallel_ldlt.hpp:38-51 and Eigen's solve) for any symmetric
 * matrix given as a full CSC pattern (both triangles, sorted rows). perm
 * (new -> old, may be NULL for the natural order) fixes the elimination
 * order. */
int sdfgpu_ldlt_create(int32_t n, const int32_t* outer, const int32_t* inner, const int32_t* perm,
                       sdfgpu_ldlt** out);
/* Numeric factorization with new values on the same pattern; returns
 * SDFGPU_ERR_NUMERICAL on a zero pivot (Eigen::NumericalIssue). */
int sdfgpu_ldlt_factorize(sdfgpu_ldlt* ldlt, const double* values);
int sdfgpu_ldlt_solve(sdfgpu_ldlt* ldlt, const double* b, double* x);
int sdfgpu_ldlt_destroy(sdfgpu_ldlt* ldlt);

/* ---------------------------------------------------------------- serving --
 * A request loop with continuous batching: submitted problems are admitted
 * while their device footprint (state, symbolic analysis, factors) fits the
 * budget, run LM iterations together with every other admitted request, and
 * retire individually. */
int sdfgpu_server_create(int64_t memory_budget_bytes, int32_t max_batch, sdfgpu_server** out);
/* Copies the request; returns its id. options as for sdfgpu_solve. Fails with
 * SDFGPU_ERR_OUT_OF_MEMORY when the request alone exceeds the budget. */
int sdfgpu_server_submit(sdfgpu_server* server, const sdfgpu_problem_desc* desc,
                         const sdfgpu_solver_options* options, int64_t* request_id);
/* SDFGPU_ERR_NOT_READY until the request has finished; then fills result and
 * copies the final state (pointers may be NULL) and forgets the request. */
int sdfgpu_server_poll(sdfgpu_server* server, int64_t request_id, sdfgpu_solve_result* result,
                       double* map_values, double* poses);
/* Cancels a queued or running request. */
int sdfgpu_server_cancel(sdfgpu_server* server, int64_t request_id);
/* stats[0..7]: submitted, completed, queued, running, p50 ms, p99 ms,
 * throughput requests/s, LM iterations/s since creation. */
int sdfgpu_server_stats(sdfgpu_server* server, double* stats);
/* Waits up to timeout_ms for every submitted request to finish;
 * SDFGPU_ERR_TIMEOUT otherwise. */
int sdfgpu_server_drain(sdfgpu_server* server, int64_t timeout_ms);
int sdfgpu_server_destroy(sdfgpu_server* server);

/* ------------------------------------------------- allocation-free solve --
 * No counterpart in the reference. For callers that cannot allocate device
 * memory when they need a solve -- a host framework whose caching allocator
 * already holds the device's free memory, or a real-time loop that allows no
 * allocation after start-up: solves A x = b for a dense symmetric n x n
 * matrix A (host arrays; A column major, only its lower triangle is read)
 * with the library's LDL^T panel, update and triangular-solve kernels,
 * keeping every intermediate in one file-scope device array of about 8.6 MB
 * that each GPU loading the library holds until the process exits. Calls no
 * cudaMalloc / cudaFree and creates no stream: its copies and kernels run on
 * the calling thread's per-thread default stream (cudaStreamPerThread), which
 * does not wait for the host application's other streams (it does order with
 * the legacy default stream, if the application uses that one). n above
 * SDFGPU_NOALLOC_MAX_N gives SDFGPU_ERR_INVALID_ARGUMENT; a zero pivot
 * SDFGPU_ERR_NUMERICAL. The first call on a device looks the array's address
 * up with that device current, and under CUDA's lazy module loading (the
 * default) that first lookup is also when the driver loads the code holding
 * the array and reserves its ~8.6 MB: make that first call (a call with
 * n = 1 will do) at start-up, before the host framework's allocator takes
 * the device's free memory and before any stream capture. All calls share
 * the array and it keeps the last call's contents; calls whose GPU work
 * overlaps (from several host threads, for example) race and must be
 * serialised. */
#define SDFGPU_NOALLOC_MAX_N 1024
int sdfgpu_dense_ldlt_solve_noalloc(int32_t n, const double* a, const double* b, double* x);

#ifdef __cplusplus
}
#endif

#endif /* SDFGPU_H_ */
