"""sdf_slam_b200: B200 backend for the joint LM path of sdf-slam.

Python mirror of the reference's solver / problem API (the host side used by
the tests, the benchmark and scripting callers) over the C ABI of
lib/libsdfgpu.so:

* ``ProblemOptions``, ``Problem`` -- src/problem/problem.hpp:63-161
* ``SolverOptions``, ``SolveResult``, ``solve`` -- src/solvers/solver.hpp:10-70,
  with ``backend="gpu"`` (SolverBackend::kGpuLm)
* ``LdltSolver`` -- the factor-only interface of ParallelSimplicialLdlt
  (src/solvers/parallel_ldlt.hpp:38-51) on the GPU
* ``Server`` -- the continuous-batching request loop.

Errors follow the reference: shape and argument errors raise ``ValueError``
(std::invalid_argument), a failed factorization raises ``RuntimeError`` with
"sparse Cholesky factorization failed" (lm_solver.cpp:354-362). There is no
CPU fallback: without the built library or a GPU every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import (SDFGPU_ERR_INVALID_ARGUMENT, SDFGPU_ERR_NOT_READY, SDFGPU_ERR_NUMERICAL,
                    SDFGPU_ERR_OUT_OF_MEMORY, SDFGPU_ERR_TIMEOUT, SDFGPU_OK)

__all__ = ["ProblemOptions", "SolverOptions", "SolveResult", "Problem", "Specs", "solve",
           "run_incremental", "run_incremental_scene", "IncrementalResult", "write_run_outputs",
           "evaluate_trajectory",
           "LdltSolver", "Server", "GpuError", "NotReady", "device_count", "lib", "measure_fp64_peak",
           "release_cached_memory"]

NORMAL_METHODS = {"pca": 0, "hybrid": 1, "weighted": 2}


class GpuError(RuntimeError):
    """A CUDA runtime failure inside the library."""


class NotReady(Exception):
    """A serving request has not finished yet."""


def lib():
    return _capi.load()


def _check(rc: int):
    if rc == SDFGPU_OK:
        return
    msg = (lib().sdfgpu_last_error_message() or b"").decode()
    if rc == SDFGPU_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == SDFGPU_ERR_NUMERICAL:
        raise RuntimeError(msg or "sparse Cholesky factorization failed")
    if rc == SDFGPU_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    if rc == SDFGPU_ERR_TIMEOUT:
        raise TimeoutError(msg)
    if rc == SDFGPU_ERR_NOT_READY:
        raise NotReady(msg)
    raise GpuError(msg)


def device_count() -> int:
    return int(lib().sdfgpu_device_count())


def _d(a):
    return a.ctypes.data_as(_capi.c_dbl_p)


def _i(a):
    return a.ctypes.data_as(_capi.c_int_p)


@dataclass
class ProblemOptions:
    """ProblemOptions with Weights, HallucinationOptions and NormalOptions
    (problem.hpp:16-87, hallucination.hpp:17-23, normals.hpp:44-57)."""
    weights_scan: float = 1.0
    weights_hallucination: float = 1.0
    weights_eikonal: float = 1.0
    weights_odometry: float = 1.0
    weights_relation: float = 1.0
    hallucination_points: int = 6
    hallucination_step: float = 0.1
    hallucination_both: bool = True
    normal_method: int = 2
    k_neighbors: int = 10
    normals_per_scan: bool = False
    corner_threshold: float = 0.2
    huber_delta: float = 0.0
    smooth_gradient: bool = True
    smooth_gradient_step: float = 0.0
    active_region: bool = False
    active_margin: int = 2

    def to_c(self) -> _capi.ProblemOptionsC:
        m = self.normal_method
        if isinstance(m, str):
            m = NORMAL_METHODS[m]
        return _capi.ProblemOptionsC(
            self.weights_scan, self.weights_hallucination, self.weights_eikonal,
            self.weights_odometry, self.weights_relation, int(self.hallucination_points),
            self.hallucination_step, int(self.hallucination_both), int(m), int(self.k_neighbors),
            int(self.normals_per_scan), self.corner_threshold, self.huber_delta,
            int(self.smooth_gradient), self.smooth_gradient_step, int(self.active_region),
            int(self.active_margin))


@dataclass
class SolverOptions:
    """SolverOptions (solver.hpp:29-55) with backend "gpu" and a precision
    ("fp64" or "mixed")."""
    backend: str = "gpu"
    max_iterations: int = 100
    step_tolerance: float = 1e-6
    lambda_init: float = 1.0
    lambda_factor: float = 1.0
    reject_worse_steps: bool = False
    marquardt_scaling: bool = False
    trust_region: bool = False
    num_threads: int = 0
    precision: str = "fp64"
    refine_steps: int = 3
    refine_tolerance: float = 1e-13

    def to_c(self) -> _capi.SolverOptionsC:
        if self.backend != "gpu":
            raise ValueError(f"unknown solver.backend '{self.backend}' for this library")
        prec = {"fp64": 0, "mixed": 1}.get(self.precision)
        if prec is None:
            raise ValueError(f"unknown precision '{self.precision}'")
        return _capi.SolverOptionsC(int(self.max_iterations), self.step_tolerance, self.lambda_init,
                                    self.lambda_factor, int(self.reject_worse_steps),
                                    int(self.marquardt_scaling), int(self.trust_region),
                                    int(self.num_threads), prec, int(self.refine_steps),
                                    float(self.refine_tolerance))


@dataclass
class SolveResult:
    """SolveResult (solver.hpp:57-64)."""
    converged: bool = False
    iterations: int = 0
    initial_cost: float = 0.0
    final_cost: float = 0.0
    duration_seconds: float = 0.0
    cost_history: list = field(default_factory=list)
    status: int = 0


@dataclass
class Specs:
    """Flat spec arrays of one problem (what the C ABI's desc points at)."""
    nx: int
    ny: int
    min_corner: tuple
    max_corner: tuple
    map_values: np.ndarray
    poses: np.ndarray
    pt_frame: np.ndarray
    pt_xy: np.ndarray
    pt_expected: np.ndarray
    pt_sqrtw: np.ndarray
    eik_wh: np.ndarray
    eik_n: np.ndarray
    eik_sqrtw: np.ndarray
    odom_ij: np.ndarray
    odom_meas: np.ndarray
    odom_sqrtw: np.ndarray
    node_to_active: np.ndarray
    huber_delta: float = 0.0
    smooth_gradient: bool = True
    smooth_gradient_step: float = 0.0

    def desc(self):
        """A C desc plus the arrays it points into (keep both alive)."""
        keep = dict(
            map_values=np.ascontiguousarray(self.map_values, np.float64),
            poses=np.ascontiguousarray(self.poses, np.float64).reshape(-1),
            pt_frame=np.ascontiguousarray(self.pt_frame, np.int32),
            pt_xy=np.ascontiguousarray(self.pt_xy, np.float64).reshape(-1),
            pt_expected=np.ascontiguousarray(self.pt_expected, np.float64),
            pt_sqrtw=np.ascontiguousarray(self.pt_sqrtw, np.float64),
            eik_wh=np.ascontiguousarray(self.eik_wh, np.int32).reshape(-1),
            eik_n=np.ascontiguousarray(self.eik_n, np.float64).reshape(-1),
            eik_sqrtw=np.ascontiguousarray(self.eik_sqrtw, np.float64),
            odom_ij=np.ascontiguousarray(self.odom_ij, np.int32).reshape(-1),
            odom_meas=np.ascontiguousarray(self.odom_meas, np.float64).reshape(-1),
            odom_sqrtw=np.ascontiguousarray(self.odom_sqrtw, np.float64),
            node_to_active=np.ascontiguousarray(self.node_to_active, np.int32))
        k = keep
        d = _capi.ProblemDesc(
            int(self.nx), int(self.ny), float(self.min_corner[0]), float(self.min_corner[1]),
            float(self.max_corner[0]), float(self.max_corner[1]), _d(k["map_values"]),
            len(k["poses"]) // 3, _d(k["poses"]), len(k["pt_frame"]), _i(k["pt_frame"]),
            _d(k["pt_xy"]), _d(k["pt_expected"]), _d(k["pt_sqrtw"]), len(k["eik_sqrtw"]),
            _i(k["eik_wh"]), _d(k["eik_n"]), _d(k["eik_sqrtw"]), len(k["odom_sqrtw"]),
            _i(k["odom_ij"]), _d(k["odom_meas"]), _d(k["odom_sqrtw"]), _i(k["node_to_active"]),
            float(self.huber_delta), int(self.smooth_gradient), float(self.smooth_gradient_step))
        return d, keep

    def host_bytes(self) -> int:
        return sum(np.asarray(getattr(self, f)).nbytes for f in (
            "map_values", "poses", "pt_frame", "pt_xy", "pt_expected", "pt_sqrtw", "eik_wh",
            "eik_n", "eik_sqrtw", "odom_ij", "odom_meas", "odom_sqrtw", "node_to_active"))


class Problem:
    """The joint SLAM problem on the device (Problem, problem.hpp:92-161).

    ``Problem(grid, poses, scans, odometry, options, relations)`` builds the
    specs like the reference constructor (``on_device=True``: the point rows,
    active maps and Eikonal spec list by CUDA kernels, with the same
    result); ``Problem.from_specs`` uploads an
    existing problem's spec arrays; ``Problem.batch`` uploads several
    independent problems that are solved together."""

    def __init__(self, nx, ny, min_corner, max_corner, poses, scans, odometry=(), options=None,
                 relations=(), map_values=None, _handle=None, on_device=False):
        L = lib()
        if _handle is not None:
            self._h = _handle
            return
        options = options or ProblemOptions()
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 3)
        offsets = np.zeros(len(scans) + 1, np.int32)
        for f, s in enumerate(scans):
            offsets[f + 1] = offsets[f] + len(s)
        xy = (np.ascontiguousarray(np.concatenate([np.asarray(s, np.float64).reshape(-1, 2) for s in scans]))
              if len(scans) else np.zeros((0, 2)))
        if len(scans) != len(poses):
            raise ValueError("scan count != pose count")
        odo = np.ascontiguousarray(odometry, np.float64).reshape(-1, 3)
        rel_ij = np.ascontiguousarray([[r[0], r[1]] for r in relations], np.int32).reshape(-1, 2)
        rel_meas = np.ascontiguousarray([r[2] for r in relations], np.float64).reshape(-1, 3)
        rel_w = np.ascontiguousarray([r[3] if len(r) > 3 else 1.0 for r in relations], np.float64)
        mv = None if map_values is None else np.ascontiguousarray(map_values, np.float64)
        opts = options.to_c()
        h = ctypes.c_void_p()
        build = L.sdfgpu_problem_build_device if on_device else L.sdfgpu_problem_build
        _check(build(
            int(nx), int(ny), float(min_corner[0]), float(min_corner[1]), float(max_corner[0]),
            float(max_corner[1]), _d(mv) if mv is not None else None, len(poses), _d(poses),
            _i(offsets), _d(xy), _d(odo) if len(odo) else None, len(odo), len(rel_ij),
            _i(rel_ij) if len(rel_ij) else None, _d(rel_meas) if len(rel_meas) else None,
            _d(rel_w) if len(rel_w) else None, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h

    @classmethod
    def from_scene(cls, scene, options: ProblemOptions | None = None, on_device: bool = False):
        opts = options or ProblemOptions()
        for k, v in scene.options.items():
            if k != "active_region" or options is None:
                setattr(opts, k, v)
        return cls(scene.nx, scene.ny, scene.min_corner, scene.max_corner, scene.poses, scene.scans,
                   scene.odometry, opts, on_device=on_device)

    @classmethod
    def from_specs(cls, specs: Specs):
        d, keep = specs.desc()
        h = ctypes.c_void_p()
        _check(lib().sdfgpu_problem_create(ctypes.byref(d), ctypes.byref(h)))
        del keep
        return cls(0, 0, (0, 0), (0, 0), None, None, _handle=h)

    @classmethod
    def batch(cls, specs_list):
        descs = (_capi.ProblemDesc * len(specs_list))()
        keeps = []
        for q, s in enumerate(specs_list):
            d, keep = s.desc()
            descs[q] = d
            keeps.append(keep)
        h = ctypes.c_void_p()
        _check(lib().sdfgpu_problem_create_batch(descs, len(specs_list), ctypes.byref(h)))
        del keeps
        return cls(0, 0, (0, 0), (0, 0), None, None, _handle=h)

    def close(self):
        if getattr(self, "_h", None) and _capi._lib is not None:
            _capi._lib.sdfgpu_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def count(self) -> int:
        return int(lib().sdfgpu_problem_count(self._h))

    def sizes(self, index=0) -> dict:
        out = np.zeros(9, np.int32)
        _check(lib().sdfgpu_problem_sizes(self._h, index, _i(out)))
        keys = ["num_points", "num_eikonal", "num_odom", "num_active", "num_parameters",
                "num_residuals", "num_frames", "nx", "ny"]
        return dict(zip(keys, (int(v) for v in out)))

    def num_parameters(self, index=0) -> int:
        return self.sizes(index)["num_parameters"]

    def specs(self, index=0, min_corner=None, max_corner=None, huber_delta=0.0,
              smooth_gradient=True, smooth_gradient_step=0.0) -> Specs:
        z = self.sizes(index)
        P, E, O = z["num_points"], z["num_eikonal"], z["num_odom"]
        nx, ny = z["nx"], z["ny"]
        a = dict(pt_frame=np.zeros(P, np.int32), pt_xy=np.zeros((P, 2)), pt_expected=np.zeros(P),
                 pt_sqrtw=np.zeros(P), eik_wh=np.zeros((E, 2), np.int32), eik_n=np.zeros((E, 2)),
                 eik_sqrtw=np.zeros(E), odom_ij=np.zeros((O, 2), np.int32),
                 odom_meas=np.zeros((O, 3)), odom_sqrtw=np.zeros(O),
                 node_to_active=np.zeros(nx * ny, np.int32))
        _check(lib().sdfgpu_problem_get_specs(
            self._h, index, _i(a["pt_frame"]), _d(a["pt_xy"]), _d(a["pt_expected"]),
            _d(a["pt_sqrtw"]), _i(a["eik_wh"]), _d(a["eik_n"]), _d(a["eik_sqrtw"]),
            _i(a["odom_ij"]), _d(a["odom_meas"]), _d(a["odom_sqrtw"]), _i(a["node_to_active"])))
        m, p = self.state(index)
        return Specs(nx=nx, ny=ny, min_corner=tuple(min_corner or (0.0, 0.0)),
                     max_corner=tuple(max_corner or (1.0, 1.0)), map_values=m, poses=p,
                     huber_delta=huber_delta, smooth_gradient=smooth_gradient,
                     smooth_gradient_step=smooth_gradient_step, **a)

    def state(self, index=0):
        """(map().values(), poses()) of instance `index`."""
        z = self.sizes(index)
        m = np.zeros(z["nx"] * z["ny"])
        p = np.zeros((z["num_frames"], 3))
        _check(lib().sdfgpu_get_state(self._h, index, _d(m), _d(p)))
        return m, p

    def set_state(self, map_values, poses, index=0):
        m = np.ascontiguousarray(map_values, np.float64)
        p = np.ascontiguousarray(poses, np.float64)
        _check(lib().sdfgpu_set_state(self._h, index, _d(m), _d(p)))

    def cost(self, index=0) -> float:
        """Problem::Cost (problem.cpp:132-156)."""
        c = ctypes.c_double()
        _check(lib().sdfgpu_cost(self._h, index, ctypes.byref(c)))
        return c.value

    def apply_step(self, step, index=0):
        """Problem::ApplyStep (problem.cpp:117-130)."""
        s = np.ascontiguousarray(step, np.float64)
        if len(s) != self.num_parameters(index):
            raise ValueError("step size != parameter count")
        _check(lib().sdfgpu_apply_step(self._h, index, _d(s)))

    def linearize(self, lam=1.0, marquardt=False, compute_step=True, index=0) -> dict:
        """One LM iteration's residuals, Jacobian (CSC), damped J^T J (CSC,
        full symmetric, the reference's structural pattern), -J^T r and step."""
        L = lib()
        _check(L.sdfgpu_linearize(self._h, index, float(lam), int(marquardt), int(compute_step)))
        sz = np.zeros(4, np.int64)
        _check(L.sdfgpu_linearization_sizes(self._h, sz.ctypes.data_as(_capi.c_i64_p)))
        rows, n, nnz_j, nnz_n = (int(v) for v in sz)
        P = self.sizes(index)["num_points"]
        out = dict(residuals=np.zeros(rows), point_cell=np.zeros(P, np.int32),
                   j_outer=np.zeros(n + 1, np.int32), j_inner=np.zeros(nnz_j, np.int32),
                   j_values=np.zeros(nnz_j), n_outer=np.zeros(n + 1, np.int32),
                   n_inner=np.zeros(nnz_n, np.int32), n_values=np.zeros(nnz_n), rhs=np.zeros(n),
                   step=np.zeros(n) if compute_step else None)
        _check(L.sdfgpu_linearization_get(
            self._h, _d(out["residuals"]), _i(out["point_cell"]), _i(out["j_outer"]),
            _i(out["j_inner"]), _d(out["j_values"]), _i(out["n_outer"]), _i(out["n_inner"]),
            _d(out["n_values"]), _d(out["rhs"]), _d(out["step"]) if compute_step else None))
        return out

    def autotune(self) -> dict:
        """Picks the fastest factorization schedule for this handle (kept for
        its later solves): {"schedule": (small_pivots, front_rows,
        panel_rows), "factor_ms": ..., "trials": [(s, f, p, ms), ...]}."""
        sched = (ctypes.c_int32 * 3)()
        best = ctypes.c_double()
        trials = np.zeros((16, 4))
        n = ctypes.c_int32()
        _check(lib().sdfgpu_autotune(self._h, sched, ctypes.byref(best), _d(trials), 16, ctypes.byref(n)))
        return {"schedule": tuple(int(v) for v in sched), "factor_ms": best.value,
                "trials": [tuple(r) for r in trials[:n.value]]}

    def tensor_core_choice(self) -> dict:
        """The autotuner's tensor-core choice for mixed solves
        (sdfgpu_tensor_core_choice): {"min_rows": rows below the pivot block
        from which a FP32 front's Schur complement runs on the tensor cores
        (0: none), "ms_with": ..., "ms_without": ...} (mixed factor + solve
        times of the last autotune of a mixed handle, 0 when not timed)."""
        rows = ctypes.c_int32()
        w = ctypes.c_double()
        wo = ctypes.c_double()
        _check(lib().sdfgpu_tensor_core_choice(self._h, ctypes.byref(rows), ctypes.byref(w), ctypes.byref(wo)))
        return {"min_rows": rows.value, "ms_with": w.value, "ms_without": wo.value}

    def set_tensor_core_choice(self, min_rows: int):
        """Installs the tensor-core choice of mixed solves by hand
        (sdfgpu_set_tensor_core_choice): 0 for none, else the rows below the
        pivot block from which a FP32 front's Schur complement runs on the
        tensor cores."""
        _check(lib().sdfgpu_set_tensor_core_choice(self._h, int(min_rows)))

    def set_schedule(self, small_pivots: int, front_rows: int, panel_rows: int):
        """Installs a factorization schedule for this handle's later solves
        (sdfgpu_set_schedule): fronts with up to small_pivots pivots are
        factored by one kernel of front_rows rows per block, wider ones panel
        by panel with panel_rows rows per task, or by whole 128-column outer
        blocks when panel_rows is 0."""
        sched = (ctypes.c_int32 * 3)(int(small_pivots), int(front_rows), int(panel_rows))
        _check(lib().sdfgpu_set_schedule(self._h, sched))

    def debug_solve_fault(self, withhold_front: int, wait_polls: int = 0):
        """Test hook (sdfgpu_debug_solve_fault): from the next solve on, the
        one-launch triangular solve never publishes supernode
        `withhold_front`'s forward flag and a wait gives up after `wait_polls`
        polls, so the solve ends with TimeoutError; -1 restores it."""
        _check(lib().sdfgpu_debug_solve_fault(self._h, int(withhold_front), int(wait_polls)))

    def kernel_timing(self, classes=None):
        """Times the launches of the named kernel classes (all when None, none
        for an empty list) from the next iteration on (sdfgpu_kernel_timing);
        totals restart at zero."""
        names = kernel_class_names()
        mask = (1 << len(names)) - 1 if classes is None else sum(1 << names.index(c) for c in classes)
        _check(lib().sdfgpu_kernel_timing(self._h, mask))

    def kernel_times(self) -> dict:
        """{class name: {"ms", "launches", "work", "work_unit"}} since
        kernel_timing: device milliseconds, launches and their algorithmic
        work (useful flops, or bytes for the memory-bound classes)."""
        names = kernel_class_names()
        ms = np.zeros(len(names))
        n = np.zeros(len(names), np.int64)
        w = np.zeros(len(names))
        _check(lib().sdfgpu_kernel_times(self._h, _d(ms), n.ctypes.data_as(_capi.c_i64_p), _d(w), len(names)))
        return {k: {"ms": float(ms[c]), "launches": int(n[c]), "work": float(w[c]),
                    "work_unit": "bytes" if lib().sdfgpu_kernel_class_is_memory_bound(c) else "flop"}
                for c, k in enumerate(names)}

    def debug_supernode_count(self) -> int:
        return int(lib().sdfgpu_debug_supernode_count(self._h))

    def last_profile(self) -> dict:
        ph = np.zeros(12)
        _check(lib().sdfgpu_last_profile(self._h, _d(ph)))
        return dict(assemble=ph[0], normal=ph[1], factor=ph[2], solve=ph[3], update=ph[4],
                    iterations=int(ph[5]), span=ph[6], launches=int(ph[7]), factor_flops=ph[8],
                    reanalyses=int(ph[9]), reanalysis_host=ph[10], capture_host=ph[11])


def solve(problem: Problem, options: SolverOptions | list | None = None):
    """Solve (solver.hpp:67) with SolverBackend::kGpuLm. Mutates the problem's
    state in place. Returns a SolveResult (a list for batch handles)."""
    L = lib()
    count = problem.count
    if options is None:
        options = SolverOptions()
    if isinstance(options, (list, tuple)):
        if len(options) != count:
            raise ValueError("one SolverOptions per instance")
        opts = options
    else:
        opts = [options] * count
    c_opts = (_capi.SolverOptionsC * count)(*[o.to_c() for o in opts])
    cap = max(o.max_iterations for o in opts) + 2
    results = (_capi.SolveResultC * count)()
    hist = np.zeros((count, cap))
    if count == 1:
        rc = L.sdfgpu_solve(problem._h, c_opts, results, _d(hist), cap)
    else:
        rc = _solve_batch(problem, c_opts, results, hist, cap)
    out = []
    for i in range(count):
        r = results[i]
        out.append(SolveResult(bool(r.converged), int(r.iterations), r.initial_cost, r.final_cost,
                               r.duration_seconds, hist[i, : r.cost_history_length].tolist(),
                               int(r.status)))
    if count == 1:
        _check(rc)
        return out[0]
    if rc not in (SDFGPU_OK, SDFGPU_ERR_NUMERICAL):
        _check(rc)
    return out


@dataclass
class IncrementalResult:
    """Final state and summed result of an incremental run."""
    map_values: np.ndarray
    poses: np.ndarray
    result: SolveResult
    phases: dict


def run_incremental(nx, ny, min_corner, max_corner, poses, scans, options: ProblemOptions | None = None,
                    solver: SolverOptions | None = None, relations=(), map_values=None, increment_size=1,
                    iterations_per_increment=10, snapshot_every=0, snapshot=None, on_device=True,
                    warm_analysis=True) -> IncrementalResult:
    """Run in incremental mode (runner.cpp:226-285) on the GPU: `poses` are
    the dataset poses (their consecutive RelativeTo is the odometry), each
    step appends `increment_size` frames and runs `iterations_per_increment`
    LM iterations over all frames so far. snapshot(frames, map_values, poses)
    is called every `snapshot_every` steps and after the last."""
    L = lib()
    options = options or ProblemOptions()
    solver = solver or SolverOptions()
    poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 3)
    if len(scans) != len(poses):
        raise ValueError("scan count != pose count")
    offsets = np.zeros(len(scans) + 1, np.int32)
    for f, s in enumerate(scans):
        offsets[f + 1] = offsets[f] + len(s)
    xy = (np.ascontiguousarray(np.concatenate([np.asarray(s, np.float64).reshape(-1, 2) for s in scans]))
          if len(scans) else np.zeros((0, 2)))
    rel_ij = np.ascontiguousarray([[r[0], r[1]] for r in relations], np.int32).reshape(-1, 2)
    rel_meas = np.ascontiguousarray([r[2] for r in relations], np.float64).reshape(-1, 3)
    rel_w = np.ascontiguousarray([r[3] if len(r) > 3 else 1.0 for r in relations], np.float64)
    mv = None if map_values is None else np.ascontiguousarray(map_values, np.float64).reshape(-1)

    def _snap(_user, frames, m, p):
        snapshot(int(frames), np.ctypeslib.as_array(m, (int(nx) * int(ny),)).copy(),
                 np.ctypeslib.as_array(p, (int(frames) * 3,)).reshape(-1, 3).copy())

    cb = _capi.SnapshotFn(_snap) if snapshot is not None else _capi.SnapshotFn()
    d = _capi.IncrementalDesc(
        int(nx), int(ny), float(min_corner[0]), float(min_corner[1]), float(max_corner[0]),
        float(max_corner[1]), _d(mv) if mv is not None else None, len(poses), _d(poses), _i(offsets),
        _d(xy), len(rel_ij), _i(rel_ij) if len(rel_ij) else None,
        _d(rel_meas) if len(rel_meas) else None, _d(rel_w) if len(rel_w) else None,
        int(increment_size), int(iterations_per_increment), int(snapshot_every), cb, None,
        int(bool(on_device)), int(bool(warm_analysis)))
    po = options.to_c()
    so = solver.to_c()
    map_out = np.zeros(int(nx) * int(ny))
    poses_out = np.zeros_like(poses)
    total = _capi.SolveResultC()
    steps = -(-max(len(poses) - 1, 0) // max(int(increment_size), 1))
    cap = steps * (max(int(iterations_per_increment), 0) + 2)
    hist = np.zeros(max(cap, 1))
    ph = np.zeros(12)
    _check(L.sdfgpu_run_incremental(ctypes.byref(d), ctypes.byref(po), ctypes.byref(so), _d(map_out),
                                    _d(poses_out), ctypes.byref(total), _d(hist), cap, _d(ph)))
    res = SolveResult(bool(total.converged), int(total.iterations), total.initial_cost, total.final_cost,
                      total.duration_seconds, hist[: total.cost_history_length].tolist(), int(total.status))
    keys = ["build", "wait_analysis", "setup", "solve", "readback", "teardown", "wall"]
    phases = dict(zip(keys, ph[:7].tolist()))
    phases["increments"] = int(ph[7])
    phases["warm_analyses"] = int(ph[8])
    phases["reanalyses"] = int(ph[9])
    phases["reanalysis"] = float(ph[10])
    phases["capture"] = float(ph[11])
    return IncrementalResult(map_out, poses_out, res, phases)


def run_incremental_scene(scene, options: ProblemOptions | None = None, **kwargs) -> IncrementalResult:
    """run_incremental over a synthetic scene (its options applied as
    Problem.from_scene does)."""
    opts = options or ProblemOptions()
    for k, v in scene.options.items():
        if k != "active_region" or options is None:
            setattr(opts, k, v)
    return run_incremental(scene.nx, scene.ny, scene.min_corner, scene.max_corner, scene.poses, scene.scans,
                           opts, **kwargs)


def _scan_arrays(scans):
    offsets = np.zeros(len(scans) + 1, np.int32)
    for f, s in enumerate(scans):
        offsets[f + 1] = offsets[f] + len(s)
    xy = (np.ascontiguousarray(np.concatenate([np.asarray(s, np.float64).reshape(-1, 2) for s in scans]))
          if len(scans) else np.zeros((0, 2)))
    return offsets, xy


def evaluate_trajectory(estimated, ground_truth) -> dict:
    """Evaluate (runner.cpp:145-170): the four mean trajectory errors."""
    est = np.ascontiguousarray(estimated, np.float64).reshape(-1, 3)
    gt = np.ascontiguousarray(ground_truth, np.float64).reshape(-1, 3)
    if len(est) != len(gt):
        raise ValueError("pose count mismatch between estimate and ground truth")
    m = np.zeros(4)
    _check(lib().sdfgpu_evaluate_trajectory(_d(est), _d(gt), len(est), _d(m)))
    return dict(zip(["mean_translation_error", "mean_rotation_error", "mean_relative_translation_error",
                     "mean_relative_rotation_error"], m.tolist()))


def write_run_outputs(output_dir, nx, ny, min_corner, max_corner, dataset_poses, scans, estimated, map_values,
                      result: SolveResult, ground_truth=None):
    """The output section of Run (runner.cpp:288-303): poses_odometry.csv,
    poses_estimated.csv, map.txt, scan_points_global.csv, the out-of-domain
    warning on stderr, and metrics.json (with the trajectory errors and
    poses_ground_truth.csv when ground truth is given). Returns the metrics
    (None without ground truth)."""
    import sys
    L = lib()
    os.makedirs(output_dir, exist_ok=True)

    def path(name):
        return os.path.join(os.fspath(output_dir), name).encode()

    dp = np.ascontiguousarray(dataset_poses, np.float64).reshape(-1, 3)
    est = np.ascontiguousarray(estimated, np.float64).reshape(-1, 3)
    mv = np.ascontiguousarray(map_values, np.float64).reshape(-1)
    offsets, xy = _scan_arrays(scans)
    mn, mx = (float(min_corner[0]), float(min_corner[1])), (float(max_corner[0]), float(max_corner[1]))
    _check(L.sdfgpu_write_poses(path("poses_odometry.csv"), _d(dp), len(dp)))
    _check(L.sdfgpu_write_poses(path("poses_estimated.csv"), _d(est), len(est)))
    _check(L.sdfgpu_write_map(path("map.txt"), int(nx), int(ny), *mn, *mx, _d(mv)))
    _check(L.sdfgpu_write_scan_points(path("scan_points_global.csv"), len(est), _d(est), _i(offsets), _d(xy)))
    outside = ctypes.c_int64()
    total = ctypes.c_int64()
    _check(L.sdfgpu_points_outside_map(int(nx), int(ny), *mn, *mx, len(est), _d(est), _i(offsets), _d(xy),
                                       ctypes.byref(outside), ctypes.byref(total)))
    if outside.value > 0:
        print(f"WARNING: {outside.value} of {total.value} scan points "
              f"({100.0 * outside.value / total.value:g}%) fall outside the map domain and are unanchored "
              "(SDF 0, no gradient). Widen the map domain or disable auto_domain with explicit corners.",
              file=sys.stderr)
    r = _capi.SolveResultC(int(result.converged), int(result.iterations), float(result.initial_cost),
                           float(result.final_cost), float(result.duration_seconds), 0, 0)
    metrics = None
    m = None
    if ground_truth is not None:
        gt = np.ascontiguousarray(ground_truth, np.float64).reshape(-1, 3)
        _check(L.sdfgpu_write_poses(path("poses_ground_truth.csv"), _d(gt), len(gt)))
        metrics = evaluate_trajectory(est, gt)
        m = np.array(list(metrics.values()))
    _check(L.sdfgpu_write_metrics(path("metrics.json"), ctypes.byref(r), _d(m) if m is not None else None))
    return metrics


def _solve_batch(problem, c_opts, results, hist, cap):
    # per-instance options: the C ABI reads `count` entries when given an array
    return lib().sdfgpu_solve(problem._h, c_opts, results, _d(hist), cap)


class LdltSolver:
    """Factor-only sparse LDL^T (ParallelSimplicialLdlt's interface):
    analyze_pattern(csc) / factorize(values) / solve(b)."""

    def __init__(self, n, outer, inner, perm=None):
        self._outer = np.ascontiguousarray(outer, np.int32)
        self._inner = np.ascontiguousarray(inner, np.int32)
        p = None if perm is None else np.ascontiguousarray(perm, np.int32)
        h = ctypes.c_void_p()
        _check(lib().sdfgpu_ldlt_create(int(n), _i(self._outer), _i(self._inner),
                                        _i(p) if p is not None else None, ctypes.byref(h)))
        self._h = h
        self.n = int(n)

    def factorize(self, values):
        v = np.ascontiguousarray(values, np.float64)
        _check(lib().sdfgpu_ldlt_factorize(self._h, _d(v)))

    def solve(self, b):
        bb = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n)
        _check(lib().sdfgpu_ldlt_solve(self._h, _d(bb), _d(x)))
        return x

    def close(self):
        if getattr(self, "_h", None) and _capi._lib is not None:
            _capi._lib.sdfgpu_ldlt_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Server:
    """Serving loop: submit / poll / cancel / stats / drain."""

    def __init__(self, memory_budget_bytes: int, max_batch: int = 64):
        h = ctypes.c_void_p()
        _check(lib().sdfgpu_server_create(int(memory_budget_bytes), int(max_batch), ctypes.byref(h)))
        self._h = h

    def submit(self, specs: Specs, options: SolverOptions | None = None) -> int:
        d, keep = specs.desc()
        o = (options or SolverOptions()).to_c()
        rid = ctypes.c_int64()
        _check(lib().sdfgpu_server_submit(self._h, ctypes.byref(d), ctypes.byref(o), ctypes.byref(rid)))
        del keep
        return rid.value

    def poll(self, request_id: int, nx_ny=None, num_frames=None):
        """Returns (SolveResult, map_values, poses) once finished; raises
        NotReady before."""
        r = _capi.SolveResultC()
        m = np.zeros(nx_ny) if nx_ny else None
        p = np.zeros((num_frames, 3)) if num_frames else None
        _check(lib().sdfgpu_server_poll(self._h, int(request_id), ctypes.byref(r),
                                        _d(m) if m is not None else None,
                                        _d(p) if p is not None else None))
        res = SolveResult(bool(r.converged), int(r.iterations), r.initial_cost, r.final_cost,
                          r.duration_seconds, [], int(r.status))
        return res, m, p

    def cancel(self, request_id: int):
        _check(lib().sdfgpu_server_cancel(self._h, int(request_id)))

    def stats(self) -> dict:
        s = np.zeros(8)
        _check(lib().sdfgpu_server_stats(self._h, _d(s)))
        keys = ["submitted", "completed", "queued", "running", "p50_ms", "p99_ms",
                "requests_per_s", "iterations_per_s"]
        return dict(zip(keys, s.tolist()))

    def drain(self, timeout_ms: int = 600000):
        _check(lib().sdfgpu_server_drain(self._h, int(timeout_ms)))

    def close(self):
        if getattr(self, "_h", None) and _capi._lib is not None:
            _capi._lib.sdfgpu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def release_cached_memory() -> None:
    """Returns the device blocks that released handles left cached, and the
    library's memory pool reserve on the current device, to the driver
    (sdfgpu_release_cached_memory). No handle's work may be in flight."""
    _check(lib().sdfgpu_release_cached_memory())


def measure_fp64_peak() -> float:
    """The current device's measured FP64 FMA throughput in TFLOP/s
    (sdfgpu_measure_fp64_peak), the denominator of the FP64 kernels'
    roofline."""
    v = ctypes.c_double()
    _check(lib().sdfgpu_measure_fp64_peak(ctypes.byref(v)))
    return v.value


KERNEL_CLASSES = 10


def kernel_class_names() -> list:
    """Names of the kernel classes sdfgpu_kernel_timing can time."""
    return [lib().sdfgpu_kernel_class_name(c).decode() for c in range(KERNEL_CLASSES)]
