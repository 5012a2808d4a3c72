"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline / reference leg of ``bench.py``. The product library
never loads it. The oracle restates the reference's FP64 arithmetic for the
joint LM path (src/problem/residual_math.hpp, src/problem/problem.cpp,
src/solvers/lm_solver.cpp, src/solvers/parallel_ldlt.hpp); see oracle.hpp for
what is pinned by the reference's own tests and what is not.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_i64_p = ctypes.POINTER(ctypes.c_int64)


def build() -> str:
    """Compile the oracle with its Makefile (g++ -O2 -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    vp = ctypes.c_void_p
    L.oracle_problem_build.restype = vp
    L.oracle_problem_build.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [
        c_dbl_p, ctypes.c_int, c_dbl_p, c_int_p, c_dbl_p, c_dbl_p, ctypes.c_int, ctypes.c_int,
        c_int_p, c_dbl_p, c_dbl_p, c_dbl_p, c_int_p, ctypes.c_char_p, ctypes.c_int]
    L.oracle_problem_from_specs.restype = vp
    L.oracle_problem_from_specs.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [
        c_dbl_p, ctypes.c_int, c_dbl_p, ctypes.c_int, c_int_p, c_dbl_p, c_dbl_p, c_dbl_p,
        ctypes.c_int, c_int_p, c_dbl_p, c_dbl_p, ctypes.c_int, c_int_p, c_dbl_p, c_dbl_p, c_int_p,
        ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]
    L.oracle_problem_free.argtypes = [vp]
    L.oracle_problem_sizes.argtypes = [vp, c_int_p]
    L.oracle_problem_get_specs.argtypes = [vp, c_int_p, c_dbl_p, c_dbl_p, c_dbl_p, c_int_p, c_dbl_p,
                                           c_dbl_p, c_int_p, c_dbl_p, c_dbl_p, c_int_p]
    L.oracle_problem_get_state.argtypes = [vp, c_dbl_p, c_dbl_p]
    L.oracle_problem_set_state.argtypes = [vp, c_dbl_p, c_dbl_p]
    L.oracle_problem_cost.restype = ctypes.c_double
    L.oracle_problem_cost.argtypes = [vp]
    L.oracle_problem_apply_step.argtypes = [vp, c_dbl_p]
    L.oracle_nd_ordering.argtypes = [vp, c_int_p]
    L.oracle_linearize.restype = vp
    L.oracle_linearize.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.oracle_lin_sizes.argtypes = [vp, c_i64_p]
    L.oracle_lin_get.argtypes = [vp, c_dbl_p, c_int_p, c_int_p, c_int_p, c_dbl_p, c_int_p, c_int_p,
                                 c_dbl_p, c_dbl_p, c_dbl_p]
    L.oracle_lin_free.argtypes = [vp]
    L.oracle_solve.argtypes = [vp, c_dbl_p, c_int_p, c_dbl_p, c_int_p, c_dbl_p, ctypes.c_int,
                               ctypes.c_char_p, ctypes.c_int]
    L.oracle_ldlt_solve.argtypes = [ctypes.c_int, c_int_p, c_int_p, c_dbl_p, c_int_p, ctypes.c_int,
                                    c_dbl_p, c_dbl_p, c_dbl_p]
    L.oracle_locate.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [
        c_dbl_p, ctypes.c_double, ctypes.c_double, c_int_p, c_dbl_p, c_dbl_p, c_dbl_p]
    L.oracle_eval_point.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [
        c_dbl_p, c_dbl_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
        ctypes.c_double, c_dbl_p, c_int_p]
    L.oracle_eval_odom.argtypes = [c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p]
    L.oracle_eval_eikonal.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [
        c_dbl_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, c_dbl_p, c_int_p]
    L.oracle_hallucinate.argtypes = [c_dbl_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_int, c_dbl_p, c_dbl_p]
    L.oracle_pose_op.argtypes = [ctypes.c_int, c_dbl_p, c_dbl_p, c_dbl_p]
    L.oracle_normals.argtypes = [ctypes.c_int, c_dbl_p, c_int_p, c_dbl_p, ctypes.c_int, ctypes.c_int,
                                 c_dbl_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [
                                     ctypes.c_int, ctypes.c_double, c_dbl_p]
    L.oracle_random_map.argtypes = [ctypes.c_uint32, c_dbl_p]
    L.oracle_random_map.restype = None
    L.oracle_selftest_jacobians.argtypes = [c_int_p]
    L.oracle_selftest_jacobians.restype = ctypes.c_int


def _d(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.ctypes.data_as(c_dbl_p)


def _i(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a.ctypes.data_as(c_int_p)


class _Keep(list):
    """Holds numpy buffers alive for the duration of a ctypes call."""

    def d(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.append(a)
        return a.ctypes.data_as(c_dbl_p)

    def i(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.int32)
        self.append(a)
        return a.ctypes.data_as(c_int_p)


@dataclass
class Specs:
    """Flat spec arrays of a Problem (problem.hpp:28-50, 135-142)."""
    nx: int
    ny: int
    min_corner: tuple
    max_corner: tuple
    map_values: np.ndarray
    poses: np.ndarray            # (F, 3)
    pt_frame: np.ndarray         # (P,)
    pt_xy: np.ndarray            # (P, 2)
    pt_expected: np.ndarray
    pt_sqrtw: np.ndarray
    eik_wh: np.ndarray           # (E, 2)
    eik_n: np.ndarray            # (E, 2)
    eik_sqrtw: np.ndarray
    odom_ij: np.ndarray          # (O, 2)
    odom_meas: np.ndarray        # (O, 3)
    odom_sqrtw: np.ndarray
    node_to_active: np.ndarray   # (nx*ny,)
    huber_delta: float = 0.0
    smooth_gradient: bool = True
    smooth_gradient_step: float = 0.0


@dataclass
class OracleOptions:
    """ProblemOptions with its Weights, HallucinationOptions and NormalOptions
    at the reference's defaults (src/problem/problem.hpp:16-87,
    src/core/hallucination.hpp:17-23, src/core/normals.hpp:44-57)."""
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


class OracleProblem:
    """The oracle's Problem (src/problem/problem.hpp:92-161)."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("oracle problem construction failed")
        self._h = ctypes.c_void_p(handle)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_problem_free(self._h)
            self._h = None

    @classmethod
    def build(cls, nx, ny, min_corner, max_corner, poses, scans, odometry, options,
              relations=(), map_values=None):
        """Problem::Problem(map, poses, scans, odometry, options, relations)."""
        L = lib()
        k = _Keep()
        poses = np.asarray(poses, dtype=np.float64).reshape(-1, 3)
        offsets = np.zeros(len(scans) + 1, dtype=np.int32)
        for f, s in enumerate(scans):
            offsets[f + 1] = offsets[f] + len(s)
        xy = np.concatenate([np.asarray(s, dtype=np.float64).reshape(-1, 2) for s in scans]) \
            if len(scans) else np.zeros((0, 2))
        odo = np.asarray(odometry, dtype=np.float64).reshape(-1, 3)
        rel_ij = np.array([[r[0], r[1]] for r in relations], dtype=np.int32).reshape(-1, 2)
        rel_meas = np.array([r[2] for r in relations], dtype=np.float64).reshape(-1, 3)
        rel_w = np.array([r[3] if len(r) > 3 else 1.0 for r in relations], dtype=np.float64)
        o = options
        od = [o.weights_scan, o.weights_hallucination, o.weights_eikonal, o.weights_odometry,
              o.weights_relation, o.hallucination_step, o.huber_delta, o.smooth_gradient_step,
              o.corner_threshold]
        oi = [o.hallucination_points, int(o.hallucination_both), o.normal_method, o.k_neighbors,
              int(o.normals_per_scan), int(o.smooth_gradient), int(o.active_region), o.active_margin]
        err = ctypes.create_string_buffer(512)
        h = L.oracle_problem_build(int(nx), int(ny), float(min_corner[0]), float(min_corner[1]),
                                   float(max_corner[0]), float(max_corner[1]), k.d(map_values),
                                   len(poses), k.d(poses), k.i(offsets), k.d(xy), k.d(odo),
                                   len(odo), len(rel_ij), k.i(rel_ij), k.d(rel_meas), k.d(rel_w),
                                   k.d(od), k.i(oi), err, 512)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    @classmethod
    def from_specs(cls, s: Specs):
        L = lib()
        k = _Keep()
        err = ctypes.create_string_buffer(512)
        h = L.oracle_problem_from_specs(
            s.nx, s.ny, float(s.min_corner[0]), float(s.min_corner[1]), float(s.max_corner[0]),
            float(s.max_corner[1]), k.d(s.map_values), len(s.poses), k.d(s.poses), len(s.pt_frame),
            k.i(s.pt_frame), k.d(s.pt_xy), k.d(s.pt_expected), k.d(s.pt_sqrtw), len(s.eik_wh),
            k.i(s.eik_wh), k.d(s.eik_n), k.d(s.eik_sqrtw), len(s.odom_ij), k.i(s.odom_ij),
            k.d(s.odom_meas), k.d(s.odom_sqrtw), k.i(s.node_to_active), float(s.huber_delta),
            int(s.smooth_gradient), float(s.smooth_gradient_step), err, 512)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    def sizes(self):
        out = np.zeros(9, dtype=np.int32)
        lib().oracle_problem_sizes(self._h, out.ctypes.data_as(c_int_p))
        keys = ["num_points", "num_eikonal", "num_odom", "num_active", "num_params",
                "num_residuals", "num_frames", "nx", "ny"]
        return dict(zip(keys, out.tolist()))

    def specs(self, nx, ny, min_corner, max_corner, huber_delta=0.0, smooth_gradient=True,
              smooth_gradient_step=0.0) -> Specs:
        z = self.sizes()
        P, E, O, F = z["num_points"], z["num_eikonal"], z["num_odom"], z["num_frames"]
        a = dict(pt_frame=np.zeros(P, np.int32), pt_xy=np.zeros((P, 2)), pt_expected=np.zeros(P),
                 pt_sqrtw=np.zeros(P), eik_wh=np.zeros((E, 2), np.int32), eik_n=np.zeros((E, 2)),
                 eik_sqrtw=np.zeros(E), odom_ij=np.zeros((O, 2), np.int32),
                 odom_meas=np.zeros((O, 3)), odom_sqrtw=np.zeros(O),
                 node_to_active=np.zeros(nx * ny, np.int32))
        lib().oracle_problem_get_specs(
            self._h, _i(a["pt_frame"]), a["pt_xy"].ctypes.data_as(c_dbl_p),
            a["pt_expected"].ctypes.data_as(c_dbl_p), a["pt_sqrtw"].ctypes.data_as(c_dbl_p),
            a["eik_wh"].ctypes.data_as(c_int_p), a["eik_n"].ctypes.data_as(c_dbl_p),
            a["eik_sqrtw"].ctypes.data_as(c_dbl_p), a["odom_ij"].ctypes.data_as(c_int_p),
            a["odom_meas"].ctypes.data_as(c_dbl_p), a["odom_sqrtw"].ctypes.data_as(c_dbl_p),
            a["node_to_active"].ctypes.data_as(c_int_p))
        a["pt_frame"] = a["pt_frame"]
        m, p = self.state(nx * ny, F)
        return Specs(nx=nx, ny=ny, min_corner=tuple(min_corner), max_corner=tuple(max_corner),
                     map_values=m, poses=p, huber_delta=huber_delta,
                     smooth_gradient=smooth_gradient, smooth_gradient_step=smooth_gradient_step, **a)

    def state(self, num_nodes=None, num_frames=None):
        z = self.sizes()
        m = np.zeros(z["nx"] * z["ny"])
        p = np.zeros((z["num_frames"], 3))
        lib().oracle_problem_get_state(self._h, m.ctypes.data_as(c_dbl_p), p.ctypes.data_as(c_dbl_p))
        return m, p

    def set_state(self, map_values, poses):
        k = _Keep()
        lib().oracle_problem_set_state(self._h, k.d(map_values), k.d(poses))

    def cost(self) -> float:
        return lib().oracle_problem_cost(self._h)

    def apply_step(self, step):
        k = _Keep()
        lib().oracle_problem_apply_step(self._h, k.d(step))

    def nd_ordering(self):
        z = self.sizes()
        perm = np.zeros(z["num_params"], np.int32)
        lib().oracle_nd_ordering(self._h, perm.ctypes.data_as(c_int_p))
        return perm

    def linearize(self, lam=1.0, marquardt=False, num_threads=0, compute_step=True):
        """One LM iteration's quantities from the current state
        (lm_solver.cpp:304-436) without applying the step."""
        L = lib()
        h = L.oracle_linearize(self._h, float(lam), int(marquardt), int(num_threads), int(compute_step))
        sz = np.zeros(7, np.int64)
        L.oracle_lin_sizes(h, sz.ctypes.data_as(c_i64_p))
        rows, n, nnz_j, nnz_n, ok, nnz_l, has_step = (int(v) for v in sz)
        P = self.sizes()["num_points"]
        out = dict(residuals=np.zeros(rows), point_cell=np.zeros(P, np.int32),
                   j_outer=np.zeros(n + 1, np.int32), j_inner=np.zeros(nnz_j, np.int32),
                   j_values=np.zeros(nnz_j), n_outer=np.zeros(n + 1, np.int32),
                   n_inner=np.zeros(nnz_n, np.int32), n_values=np.zeros(nnz_n), rhs=np.zeros(n),
                   step=np.zeros(n) if has_step else None)
        L.oracle_lin_get(h, out["residuals"].ctypes.data_as(c_dbl_p),
                         out["point_cell"].ctypes.data_as(c_int_p),
                         out["j_outer"].ctypes.data_as(c_int_p), out["j_inner"].ctypes.data_as(c_int_p),
                         out["j_values"].ctypes.data_as(c_dbl_p), out["n_outer"].ctypes.data_as(c_int_p),
                         out["n_inner"].ctypes.data_as(c_int_p), out["n_values"].ctypes.data_as(c_dbl_p),
                         out["rhs"].ctypes.data_as(c_dbl_p),
                         out["step"].ctypes.data_as(c_dbl_p) if has_step else None)
        L.oracle_lin_free(h)
        out["factor_ok"] = bool(ok)
        out["nnz_l"] = nnz_l
        return out

    def solve(self, max_iterations=100, step_tolerance=1e-6, lambda_init=1.0, lambda_factor=1.0,
              reject_worse_steps=False, marquardt_scaling=False, trust_region=False, num_threads=0):
        """SolveLm (lm_solver.cpp:201-434). Mutates the state in place."""
        od = np.array([step_tolerance, lambda_init, lambda_factor], np.float64)
        oi = np.array([max_iterations, int(reject_worse_steps), int(marquardt_scaling),
                       int(trust_region), num_threads], np.int32)
        rd = np.zeros(8)
        ri = np.zeros(3, np.int32)
        hist = np.zeros(max_iterations + 2)
        err = ctypes.create_string_buffer(512)
        rc = lib().oracle_solve(self._h, od.ctypes.data_as(c_dbl_p), oi.ctypes.data_as(c_int_p),
                                rd.ctypes.data_as(c_dbl_p), ri.ctypes.data_as(c_int_p),
                                hist.ctypes.data_as(c_dbl_p), len(hist), err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return dict(converged=bool(ri[0]), iterations=int(ri[1]), initial_cost=rd[0],
                    final_cost=rd[1], duration_seconds=rd[2], phase_seconds=rd[3:8].copy(),
                    cost_history=hist[: ri[2]].copy())


def run_incremental(nx, ny, min_corner, max_corner, poses, scans, options, relations=(),
                    map_values=None, increment_size=1, iterations_per_increment=10,
                    solver=None, num_threads=0):
    """Run in incremental mode (src/pipeline/runner.cpp:226-285) on the
    oracle: odometry = RelativeTo of consecutive dataset poses (:52-59); each
    step appends frames composed from the last optimized pose, rebuilds the
    Problem over the frames so far from the current map and poses (:247-258)
    and solves it for iterations_per_increment iterations (:259), summing the
    step results as :264-272 do. Returns (map, poses, summed result dict)."""
    poses = np.asarray(poses, dtype=np.float64).reshape(-1, 3)
    F = len(poses)
    odometry = [pose_op(2, poses[i], poses[i + 1]) for i in range(F - 1)]
    m = np.zeros(nx * ny) if map_values is None else np.asarray(map_values, np.float64).reshape(-1).copy()
    est = [poses[0].copy()]
    solver = dict(solver or {})
    solver["max_iterations"] = iterations_per_increment
    total = dict(converged=False, iterations=0, initial_cost=-1.0, final_cost=0.0, cost_history=[])
    next_frame = 1
    while next_frame < F:
        last = min(F, next_frame + increment_size)
        for i in range(next_frame, last):
            est.append(pose_op(1, est[-1], odometry[i - 1]))
        next_frame = last
        prob = OracleProblem.build(nx, ny, min_corner, max_corner, np.array(est), scans[:next_frame],
                                   np.array(odometry[: next_frame - 1]), options, relations, m)
        r = prob.solve(num_threads=num_threads, **solver)
        m, p = prob.state()
        est = [row.copy() for row in p]
        if total["initial_cost"] < 0.0:
            total["initial_cost"] = r["initial_cost"]
        total["iterations"] += r["iterations"]
        total["final_cost"] = r["final_cost"]
        total["converged"] = r["converged"]
        total["cost_history"].extend(r["cost_history"].tolist())
    return m, np.array(est), total


def ldlt_solve(n, outer, inner, values, b, perm=None, num_threads=1):
    """Factor + solve of a full symmetric CSC matrix; returns (x, diag) or
    raises on a zero pivot (parallel_ldlt.hpp NumericalIssue)."""
    k = _Keep()
    x = np.zeros(n)
    d = np.zeros(n)
    rc = lib().oracle_ldlt_solve(int(n), k.i(outer), k.i(inner), k.d(values), k.i(perm),
                                 int(num_threads), k.d(b), x.ctypes.data_as(c_dbl_p),
                                 d.ctypes.data_as(c_dbl_p))
    if rc != 0:
        raise ArithmeticError("sparse LDLT: zero pivot")
    return x, d


def locate(nx, ny, mn, mx, values, p):
    k = _Keep()
    wh = np.zeros(2, np.int32)
    ab = np.zeros(2)
    val = ctypes.c_double()
    g = np.zeros(2)
    ok = lib().oracle_locate(nx, ny, mn[0], mn[1], mx[0], mx[1], k.d(values), float(p[0]),
                             float(p[1]), wh.ctypes.data_as(c_int_p), ab.ctypes.data_as(c_dbl_p),
                             ctypes.byref(val), g.ctypes.data_as(c_dbl_p))
    if not ok:
        return None
    return dict(w=int(wh[0]), h=int(wh[1]), alpha=ab[0], beta=ab[1], value=val.value, grad=g)


def eval_point(nx, ny, mn, mx, values, pose, p, delta, smooth=False, smooth_step=0.0):
    k = _Keep()
    od = np.zeros(8)
    oi = np.zeros(5, np.int32)
    lib().oracle_eval_point(nx, ny, mn[0], mn[1], mx[0], mx[1], k.d(values), k.d(pose),
                            float(p[0]), float(p[1]), float(delta), int(smooth), float(smooth_step),
                            od.ctypes.data_as(c_dbl_p), oi.ctypes.data_as(c_int_p))
    return dict(valid=bool(oi[0]), residual=od[0], d_nodes=od[1:5].copy(), node_ids=oi[1:5].copy(),
                d_pose=od[5:8].copy())


def random_map(seed):
    """RandomMap(std::mt19937(seed)) of tests/test_jacobians.cpp:13-20: the
    node values of a 6 x 5 grid over [-3, 3] x [-2, 2]."""
    out = np.zeros(30)
    lib().oracle_random_map(int(seed), out.ctypes.data_as(c_dbl_p))
    return out


def eval_odom(pi, pj, meas):
    k = _Keep()
    out = np.zeros(21)
    lib().oracle_eval_odom(k.d(pi), k.d(pj), k.d(meas), out.ctypes.data_as(c_dbl_p))
    return out[:3].copy(), out[3:12].reshape(3, 3).copy(), out[12:21].reshape(3, 3).copy()


def eval_eikonal(nx, ny, mn, mx, values, w, h, normal):
    k = _Keep()
    out = np.zeros(4)
    ids = np.zeros(3, np.int32)
    lib().oracle_eval_eikonal(nx, ny, mn[0], mn[1], mx[0], mx[1], k.d(values), int(w), int(h),
                              float(normal[0]), float(normal[1]), out.ctypes.data_as(c_dbl_p),
                              ids.ctypes.data_as(c_int_p))
    return out[0], out[1:].copy(), ids


def hallucinate(points, per_point=6, step=0.1, both=True):
    k = _Keep()
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 2)
    n = lib().oracle_hallucinate(k.d(pts), len(pts), per_point, step, int(both), None, None)
    xy = np.zeros((n, 2))
    ex = np.zeros(n)
    lib().oracle_hallucinate(k.d(pts), len(pts), per_point, step, int(both),
                             xy.ctypes.data_as(c_dbl_p), ex.ctypes.data_as(c_dbl_p))
    return xy, ex


def pose_op(mode, a, b=(0.0, 0.0, 0.0)):
    k = _Keep()
    out = np.zeros(3)
    lib().oracle_pose_op(int(mode), k.d(np.asarray(a, float)), k.d(np.asarray(b, float)),
                         out.ctypes.data_as(c_dbl_p))
    return out


def normals(poses, scans, k_neighbors=10, per_scan=False, grid=None, method=2,
            corner_threshold=0.2):
    k = _Keep()
    poses = np.asarray(poses, dtype=np.float64).reshape(-1, 3)
    offsets = np.zeros(len(scans) + 1, dtype=np.int32)
    for f, s in enumerate(scans):
        offsets[f + 1] = offsets[f] + len(s)
    xy = np.concatenate([np.asarray(s, dtype=np.float64).reshape(-1, 2) for s in scans])
    out_pts = np.zeros((offsets[-1], 3))
    if grid is not None:
        nx, ny, mn, mx = grid
        out_nodes = np.zeros((nx * ny, 3))
    else:
        nx, ny, mn, mx = 2, 2, (0.0, 0.0), (1.0, 1.0)
        out_nodes = None
    lib().oracle_normals(len(poses), k.d(poses), k.i(offsets), k.d(xy), int(k_neighbors),
                         int(per_scan), out_pts.ctypes.data_as(c_dbl_p), nx, ny, mn[0], mn[1],
                         mx[0], mx[1], int(method), float(corner_threshold),
                         out_nodes.ctypes.data_as(c_dbl_p) if out_nodes is not None else None)
    return out_pts, out_nodes


def selftest_jacobians():
    checked = ctypes.c_int()
    failures = lib().oracle_selftest_jacobians(ctypes.byref(checked))
    return failures, checked.value
