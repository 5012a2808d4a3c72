"""CPU tests of the product's host side: the C ABI library loads and exports
every entry point declared in include/sdfgpu.h, the host problem builder
(Problem::Problem mirror) produces the oracle's specs bit for bit, and
malformed inputs are rejected before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
import sdf_slam_b200 as P
import sdf_slam_b200.scenes as scenes
from sdf_slam_b200 import _capi
from helpers import corner_setup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sdfgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sdfgpu_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = P.lib()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in _capi.SIGNATURES, n
    assert lib.sdfgpu_version().startswith(b"sdfgpu")


def test_defaults_match_reference_structs():
    so = _capi.SolverOptionsC()
    P.lib().sdfgpu_solver_options_default(ctypes.byref(so))
    assert (so.max_iterations, so.step_tolerance, so.lambda_init, so.lambda_factor) == (100, 1e-6, 1.0, 1.0)
    assert (so.reject_worse_steps, so.marquardt_scaling, so.trust_region) == (0, 0, 0)
    po = _capi.ProblemOptionsC()
    P.lib().sdfgpu_problem_options_default(ctypes.byref(po))
    assert po.hallucination_points_per_scan_point == 6 and po.hallucination_step_size == 0.1
    assert po.normals_method == 2 and po.normals_k_neighbors == 10 and po.smooth_gradient == 1
    assert po.active_margin == 2 and po.huber_delta == 0.0


def _oracle_build(scene, opts):
    return O.OracleProblem.build(scene.nx, scene.ny, scene.min_corner, scene.max_corner, scene.poses,
                                 scene.scans, scene.odometry, opts)


@pytest.mark.parametrize("active", [False, True])
@pytest.mark.parametrize("method", [0, 1, 2])
def test_builder_specs_equal_oracle_bitwise(active, method):
    sc = scenes.room_scene(seed=5)
    opts = P.ProblemOptions(hallucination_points=4, active_region=active, normal_method=method)
    prob = P.Problem(sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, sc.odometry, opts)
    mine = prob.specs(min_corner=sc.min_corner, max_corner=sc.max_corner)
    ref = _oracle_build(sc, opts).specs(sc.nx, sc.ny, sc.min_corner, sc.max_corner)
    for f in ["pt_frame", "pt_xy", "pt_expected", "pt_sqrtw", "eik_wh", "eik_n", "eik_sqrtw", "odom_ij",
              "odom_meas", "odom_sqrtw", "node_to_active", "poses"]:
        a, b = getattr(mine, f), getattr(ref, f)
        assert a.shape == b.shape, f
        assert np.array_equal(a.view(np.uint8), np.ascontiguousarray(b).view(np.uint8)), f


def test_builder_relations_and_errors():
    s = corner_setup()
    nx, ny, mn, mx = s["grid"]
    p = P.Problem(nx, ny, mn, mx, s["init"], s["scans"], [s["odo"]], s["opts"], [(0, 5, s["odo"], 1.0)])
    assert p.sizes()["num_odom"] == 1
    p = P.Problem(nx, ny, mn, mx, s["init"], s["scans"], [], s["opts"], [(0, 1, s["odo"], 2.0)])
    assert p.specs().odom_sqrtw[0] == 2.0
    with pytest.raises(ValueError, match="relation frames"):
        P.Problem(nx, ny, mn, mx, s["init"], s["scans"], [s["odo"]], s["opts"], [(1, 1, s["odo"], 1.0)])
    with pytest.raises(ValueError, match="odometry count"):
        P.Problem(nx, ny, mn, mx, s["init"], s["scans"], [s["odo"], s["odo"]], s["opts"])
    with pytest.raises(ValueError):
        P.Problem(1, ny, mn, mx, s["init"], s["scans"], [s["odo"]], s["opts"])


def _room_specs():
    sc = scenes.room_scene(seed=1, frames=4, beams=60)
    prob = P.Problem.from_scene(sc)
    return prob.specs(min_corner=sc.min_corner, max_corner=sc.max_corner)


@pytest.mark.parametrize("mutate,msg", [
    (lambda s: setattr(s, "pt_frame", np.full_like(s.pt_frame, 99)), "frame out of range"),
    (lambda s: setattr(s, "odom_ij", np.array([[0, 0]] * len(s.odom_ij), np.int32)), "odometry"),
    (lambda s: setattr(s, "node_to_active", np.where(s.node_to_active == 3, 7, s.node_to_active)), "node_to_active"),
    (lambda s: setattr(s, "eik_wh", s.eik_wh[::-1].copy()), "ordered"),
    (lambda s: setattr(s, "nx", 1), "nx"),
])
def test_desc_validation_rejects_malformed_specs(mutate, msg):
    s = _room_specs()
    mutate(s)
    with pytest.raises(ValueError, match=msg):
        P.Problem.from_specs(s)


def test_state_roundtrip_on_host_before_upload():
    s = _room_specs()
    prob = P.Problem.from_specs(s)
    m, p = prob.state()
    assert np.array_equal(m, s.map_values) and np.array_equal(p, s.poses)
    prob.set_state(m + 1.0, p)
    m2, _ = prob.state()
    assert np.array_equal(m2, m + 1.0)


def test_compute_without_gpu_fails_loudly():
    if P.device_count() > 0:
        pytest.skip("a GPU is present")
    prob = P.Problem.from_specs(_room_specs())
    with pytest.raises(P.GpuError, match="no CUDA device"):
        prob.cost()
    with pytest.raises(P.GpuError):
        P.solve(prob, P.SolverOptions(max_iterations=1))


def test_oracle_reproduces_committed_fixture():
    """The oracle build on this machine reproduces the committed golden
    outputs of the seeded room scene bit for bit."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "room_oracle.npz"))
    sc = scenes.room_scene(seed=0)
    opts = P.ProblemOptions(hallucination_points=4)
    p = _oracle_build(sc, opts)
    spec = p.specs(sc.nx, sc.ny, sc.min_corner, sc.max_corner)
    assert np.array_equal(spec.pt_xy, g["pt_xy"]) and np.array_equal(spec.eik_n, g["eik_n"])
    lin = p.linearize(1.0, False, 1, True)
    assert np.array_equal(lin["residuals"], g["residuals"])
    assert np.array_equal(lin["point_cell"], g["point_cell"])
    assert np.array_equal(lin["rhs"], g["rhs"])
    assert np.array_equal(lin["step"], g["step"])
    res = p.solve(max_iterations=10, num_threads=1)
    assert np.array_equal(np.array(res["cost_history"]), g["cost_history"])


def test_set_schedule_rejects_out_of_range_values():
    """sdfgpu_set_schedule checks its ranges before touching the handle (a
    NULL handle fails as an invalid argument without a device)."""
    import ctypes
    from sdf_slam_b200 import _capi
    L = _capi.load()
    sched = (ctypes.c_int32 * 3)(128, 256, 128)
    assert L.sdfgpu_set_schedule(None, sched) == 1
    assert L.sdfgpu_set_schedule(None, None) == 1


def test_tensor_core_choice_rejects_bad_arguments_without_a_device():
    """sdfgpu_set_tensor_core_choice checks min_rows (0, or 128..65536)
    before it touches the handle; both entry points refuse a NULL handle
    with SDFGPU_ERR_INVALID_ARGUMENT and say why."""
    import ctypes
    from sdf_slam_b200 import _capi
    L = _capi.load()
    for rows in (5, 127, 65537, -1):
        assert L.sdfgpu_set_tensor_core_choice(None, rows) == 1
        assert b"min_rows" in L.sdfgpu_last_error_message()
    assert L.sdfgpu_set_tensor_core_choice(None, 0) == 1
    assert b"problem" in L.sdfgpu_last_error_message()
    rows = ctypes.c_int32()
    assert L.sdfgpu_tensor_core_choice(None, ctypes.byref(rows), None, None) == 1
    assert L.sdfgpu_tensor_core_choice(None, None, None, None) == 1


def test_solver_options_default_refine_tolerance():
    """The C default of refine_tolerance is the Python mirror's (1e-13), and
    the options struct carries it after refine_steps."""
    from sdf_slam_b200 import _capi
    import sdf_slam_b200 as P
    L = _capi.load()
    o = _capi.SolverOptionsC()
    L.sdfgpu_solver_options_default(o)
    assert o.refine_tolerance == 1e-13 == P.SolverOptions().refine_tolerance
    assert o.refine_steps == 3
    c = P.SolverOptions(precision="mixed", refine_tolerance=1e-6).to_c()
    assert c.refine_tolerance == 1e-6 and c.precision == 1
