"""On-device problem construction (sdfgpu_problem_build_device): the point
rows (scan rows, then hallucinated rows, frame by frame;
hallucination.cpp:5-28), the active-region maps (problem.cpp:39-70), the
k-NN PCA scan normals and per-node normals (normals.cpp:70-220) and the
Eikonal spec list (problem.cpp:79-94) computed by CUDA kernels must equal
the host builder's (sdfgpu_problem_build) bit for bit, and so must a solve
started from either problem.
"""
import numpy as np
import pytest

import sdf_slam_b200 as P
import sdf_slam_b200.scenes as scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pt_frame", "pt_xy", "pt_expected", "pt_sqrtw", "eik_wh", "eik_n", "eik_sqrtw", "odom_ij",
          "odom_meas", "odom_sqrtw", "node_to_active", "map_values", "poses")


def _both(scene, options=None):
    host = P.Problem.from_scene(scene, options)
    dev = P.Problem.from_scene(scene, options, on_device=True)
    return host, dev


def _assert_same_specs(host, dev):
    assert host.sizes() == dev.sizes()
    a = host.specs()
    b = dev.specs()
    for f in FIELDS:
        x = np.asarray(getattr(a, f))
        y = np.asarray(getattr(b, f))
        assert x.shape == y.shape, f
        assert x.tobytes() == y.tobytes(), f"{f} differs"


@pytest.mark.parametrize("active_region", [False, True])
@pytest.mark.parametrize("points,both", [(4, True), (6, True), (3, False), (0, True)])
def test_device_build_equals_host_build(active_region, points, both):
    sc = scenes.room_scene(seed=3, frames=6, beams=120, active_region=active_region)
    sc.options = {}  # the options below decide
    opts = P.ProblemOptions(hallucination_points=points, hallucination_both=both, active_region=active_region,
                            active_margin=2)
    host, dev = _both(sc, opts)
    _assert_same_specs(host, dev)


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("per_scan", [False, True])
@pytest.mark.parametrize("k", [2, 10, 17, 64])
def test_device_normals_equal_host_normals(method, per_scan, k):
    # the Eikonal normals and weights carry every node's normal and scale
    sc = scenes.room_scene(seed=7, frames=5, beams=90)
    sc.options = {}
    opts = P.ProblemOptions(normal_method=method, normals_per_scan=per_scan, k_neighbors=k,
                            corner_threshold=0.05 if method == 2 else 0.2)
    host, dev = _both(sc, opts)
    _assert_same_specs(host, dev)


def test_device_normals_with_duplicate_and_collinear_points():
    # equal distances (ties broken by index), zero covariance and a scan with
    # fewer points than k
    sc = scenes.room_scene(seed=9, frames=4, beams=40)
    sc.options = {}
    sc.scans[0] = np.vstack([np.asarray(sc.scans[0]), np.asarray(sc.scans[0])[:5]])
    sc.scans[1] = np.array([[1.0, 0.0], [2.0, 0.0], [3.0, 0.0], [1.0, 0.0]])
    sc.scans[2] = np.array([[1.5, 0.5]])
    for per_scan in (False, True):
        opts = P.ProblemOptions(normal_method=1, normals_per_scan=per_scan, k_neighbors=8)
        host, dev = _both(sc, opts)
        _assert_same_specs(host, dev)


def test_device_normals_reject_more_than_64_neighbours():
    sc = scenes.room_scene(seed=7, frames=2, beams=40)
    sc.options = {}
    with pytest.raises(ValueError, match="k_neighbors up to 64"):
        P.Problem.from_scene(sc, P.ProblemOptions(k_neighbors=65), on_device=True)


def test_device_build_skips_points_at_the_origin():
    # a scan point at the sensor origin gets a scan row but no hallucinated rows
    sc = scenes.room_scene(seed=5, frames=3, beams=60)
    sc.scans[1] = np.vstack([np.asarray(sc.scans[1]), [[0.0, 0.0], [1e-12, 0.0]]])
    host, dev = _both(sc)
    _assert_same_specs(host, dev)


def test_device_build_floor_plan_and_solve():
    sc = scenes.WORKLOADS["floorplan"]()
    host, dev = _both(sc)
    _assert_same_specs(host, dev)
    opts = P.SolverOptions(max_iterations=3, step_tolerance=0.0)
    ra = P.solve(host, opts)
    rb = P.solve(dev, opts)
    assert ra.cost_history == rb.cost_history
    ma, pa = host.state()
    mb, pb = dev.state()
    assert ma.tobytes() == mb.tobytes() and pa.tobytes() == pb.tobytes()
