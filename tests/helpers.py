"""Test helpers shared by the CPU and GPU suites: reference fixtures
(CornerScan of tests/test_e2e.cpp:18-61), option conversion between the
product's and the oracle's problem options, and comparison utilities."""
import math

import numpy as np

import oracle as O
import sdf_slam_b200 as P


def rot(t):
    c, s = math.cos(t), math.sin(t)
    return np.array([[c, -s], [s, c]])


def corner_scan(pose):
    """Two perpendicular walls x = 0 and y = 0 seen from `pose`
    (tests/test_e2e.cpp:18-29)."""
    R = rot(pose[2]).T
    pts = []
    s = 0.25
    while s <= 10.0:
        for w in ([0.0, s], [s, 0.0]):
            pts.append(R @ (np.array(w) - np.array(pose[:2])))
        s += 0.25
    return np.array(pts)


def corner_setup():
    """MakeSetup / MakeProblemOptions / MakeE2eMap (test_e2e.cpp:38-61)."""
    pose0 = np.array([4.0, 4.0, 0.2])
    gt1 = np.array([5.0, 5.0, -0.1])
    scans = [corner_scan(pose0), corner_scan(gt1)]
    init = np.array([pose0, [5.4, 4.7, 0.05]])
    odo = O.pose_op(2, pose0, gt1)
    opts = P.ProblemOptions(hallucination_points=4, hallucination_step=0.2, k_neighbors=8,
                            normal_method=0)
    return dict(scans=scans, init=init, odo=odo, gt1=gt1, opts=opts, grid=(40, 40, (-2.0, -2.0), (12.0, 12.0)))


def expect_recovered(map_values, poses, setup, initial_cost, final_cost, grid):
    """ExpectRecovered (test_e2e.cpp:63-88)."""
    nx, ny, mn, mx = grid
    assert final_cost < 0.05 * initial_cost
    est = poses[1]
    gt1 = setup["gt1"]
    terr = np.linalg.norm(est[:2] - gt1[:2])
    ierr = np.linalg.norm(setup["init"][1, :2] - gt1[:2])
    assert terr < 0.1
    assert terr < ierr
    assert abs(math.atan2(math.sin(est[2] - gt1[2]), math.cos(est[2] - gt1[2]))) < 0.05
    tot = 0.0
    cnt = 0
    c, s = math.cos(poses[0, 2]), math.sin(poses[0, 2])
    for p in setup["scans"][0]:
        g = (c * p[0] - s * p[1] + poses[0, 0], s * p[0] + c * p[1] + poses[0, 1])
        loc = O.locate(nx, ny, mn, mx, map_values, g)
        if loc is not None:
            tot += abs(loc["value"])
            cnt += 1
    assert cnt > 0
    assert tot / cnt < 0.1


def oracle_options(opts: "P.ProblemOptions"):
    """The oracle wrapper reads the same field names."""
    return opts


def oracle_from_specs(specs: "P.Specs"):
    s = O.Specs(**{k: getattr(specs, k) for k in O.Specs.__dataclass_fields__})
    return O.OracleProblem.from_specs(s)


def scene_specs(scene, options=None):
    """Builds the problem with the product's host builder and returns its
    specs (the identical input state both sides start from)."""
    prob = P.Problem.from_scene(scene, options)
    o = options or P.ProblemOptions()
    return prob.specs(min_corner=scene.min_corner, max_corner=scene.max_corner,
                      huber_delta=o.huber_delta, smooth_gradient=o.smooth_gradient,
                      smooth_gradient_step=o.smooth_gradient_step), prob


def csc_to_dense(n_rows, n_cols, outer, inner, values):
    m = np.zeros((n_rows, n_cols))
    for j in range(n_cols):
        for p in range(outer[j], outer[j + 1]):
            m[inner[p], j] = values[p]
    return m


def rel_err(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    den = max(np.linalg.norm(b), 1e-300)
    return float(np.linalg.norm(a - b) / den)
