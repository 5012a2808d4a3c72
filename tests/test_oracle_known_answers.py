"""Pins the CPU oracle to the reference's own tests for the LM path.

Each test restates one of RobinJehn/sdf-slam's known-answer, finite-difference
or end-to-end tests (file:line in tests/golden/known_answers.json) against the
oracle, so that the oracle the GPU parity tests compare with follows the
reference's behaviour.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle as O
from helpers import corner_setup, expect_recovered

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def _grid_values():
    return np.array([w + 10.0 * h for h in range(3) for w in range(3)])


def test_grid_interpolation_matches_manual_bilinear():
    g = KA["grid_map"]
    r = O.locate(3, 3, g["min"], g["max"], _grid_values(), g["interpolation"]["p"])
    assert r is not None
    assert abs(r["value"] - g["interpolation"]["value"]) < g["interpolation"]["tol"]


def test_grid_gradient_matches_finite_difference():
    g = KA["grid_map"]
    p = np.array(g["gradient_fd"]["p"])
    eps = g["gradient_fd"]["eps"]
    v = _grid_values()
    grad = O.locate(3, 3, g["min"], g["max"], v, p)["grad"]
    for axis in range(2):
        d = np.zeros(2)
        d[axis] = eps
        fd = (O.locate(3, 3, g["min"], g["max"], v, p + d)["value"] -
              O.locate(3, 3, g["min"], g["max"], v, p - d)["value"]) / (2 * eps)
        assert abs(grad[axis] - fd) < g["gradient_fd"]["tol"]


@pytest.mark.parametrize("case", ["grid_line", "upper_boundary"])
def test_grid_cell_assignment_rules(case):
    g = KA["grid_map"]
    c = g[case]
    r = O.locate(3, 3, g["min"], g["max"], _grid_values(), c["p"])
    assert (r["w"], r["h"]) == (c["w"], c["h"])
    assert abs(r["alpha"] - c["alpha"]) < 1e-12 and abs(r["beta"] - c["beta"]) < 1e-12


def test_grid_outside_domain():
    g = KA["grid_map"]
    for p in g["outside"]:
        assert O.locate(3, 3, g["min"], g["max"], _grid_values(), p) is None


def test_hallucination_both_directions():
    c = KA["hallucination"]["both"]
    xy, ex = O.hallucinate([c["point"]], c["per_point"], c["step"], True)
    assert len(xy) == c["count"]
    for k, v in c["x"].items():
        assert abs(xy[int(k), 0] - v) < 1e-12
    for k, v in c["expected"].items():
        assert abs(ex[int(k)] - v) < 1e-12
    assert np.all(np.abs(xy[:, 1]) < 1e-12)


def test_hallucination_one_direction_and_zero_beam():
    c = KA["hallucination"]["one_direction"]
    xy, ex = O.hallucinate([c["point"]], c["per_point"], c["step"], False)
    assert len(xy) == c["count"]
    assert np.all(ex > 0) and np.all(xy[:, 1] < 2.0)
    xy, ex = O.hallucinate([KA["hallucination"]["zero_beam"]["point"]], 6, 0.1, True)
    assert len(xy) == 0


def test_pose_apply_roundtrip_wrap():
    c = KA["pose"]
    out = O.pose_op(0, c["apply"]["pose"], c["apply"]["p"])
    assert np.allclose(out[:2], c["apply"]["out"], atol=1e-12)
    a, b = c["roundtrip"]["a"], c["roundtrip"]["b"]
    rel = O.pose_op(2, a, b)
    back = O.pose_op(1, a, rel)
    assert abs(back[0] - b[0]) < 1e-12 and abs(back[1] - b[1]) < 1e-12
    assert abs(O.pose_op(3, [back[2] - b[2]])[0]) < 1e-12
    for x, want, mode in c["wrap"]:
        got = O.pose_op(3, [x])[0]
        assert abs((abs(got) if mode == "abs" else got) - want) < 1e-12


def test_jacobians_match_finite_differences():
    failures, checked = O.selftest_jacobians()
    assert checked > 50
    assert failures == 0


def test_normals_wall_and_corner():
    """tests/test_normals.cpp:8-70 (setup code the Eikonal specs come from)."""
    wall = np.array([[0.2 * i, 5.0] for i in range(-20, 21)])
    pts, _ = O.normals([[0.0, 0.0, 0.0]], [wall], k_neighbors=8)
    assert np.all(np.abs(pts[:, 0]) < 1e-9) and np.allclose(pts[:, 1], -1.0, atol=1e-9)
    assert np.all(pts[:, 2] < 1e-6)
    corner = []
    for i in range(21):
        corner += [[5.0 - 0.2 * i, 5.0], [5.0, 5.0 - 0.2 * i]]
    corner = np.array(corner)
    pts, nodes = O.normals([[0.0, 0.0, 0.0]], [corner], k_neighbors=10,
                           grid=(11, 11, (0.0, 0.0), (10.0, 10.0)), method=2, corner_threshold=0.2)
    near = np.linalg.norm(corner - [5.0, 5.0], axis=1) < 0.3
    assert pts[near, 2].max() > 0.1
    assert nodes[5 * 11 + 5, 2] < nodes[5 * 11 + 2, 2]
    assert abs(nodes[5 * 11 + 2, 2] - 1.0) < 1e-6
    _, hyb = O.normals([[0.0, 0.0, 0.0]], [corner], k_neighbors=10,
                       grid=(11, 11, (0.0, 0.0), (10.0, 10.0)), method=1)
    assert np.allclose(np.linalg.norm(hyb[:, :2], axis=1), 1.0, atol=1e-9)


def random_spd(n, width, seed):
    """Banded grid-like SPD fixture (tests/test_parallel_ldlt.cpp:32-54) with a
    seeded generator."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        rows.append(i), cols.append(i), vals.append(30.0 + abs(rng.uniform(-1, 1)))
        if i + 1 < n:
            v = rng.uniform(-1, 1)
            rows += [i, i + 1]
            cols += [i + 1, i]
            vals += [v, v]
        if i + width < n:
            v = rng.uniform(-1, 1)
            rows += [i, i + width]
            cols += [i + width, i]
            vals += [v, v]
    order = np.lexsort((rows, cols))
    rows = np.array(rows)[order]
    cols = np.array(cols)[order]
    vals = np.array(vals)[order]
    outer = np.zeros(n + 1, np.int32)
    np.add.at(outer, cols + 1, 1)
    outer = np.cumsum(outer).astype(np.int32)
    return outer, rows.astype(np.int32), vals


def dense(n, outer, inner, vals):
    a = np.zeros((n, n))
    for j in range(n):
        a[inner[outer[j]:outer[j + 1]], j] = vals[outer[j]:outer[j + 1]]
    return a


@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_ldlt_solves_random_spd(seed):
    n = 600 + 100 * seed  # reduced from 3000 + 500 seed to keep the dense check fast
    outer, inner, vals = random_spd(n, 57, seed)
    b = np.random.default_rng(seed).uniform(-1, 1, n)
    x, d = O.ldlt_solve(n, outer, inner, vals, b, num_threads=4)
    ref = np.linalg.solve(dense(n, outer, inner, vals), b)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-13
    x1, _ = O.ldlt_solve(n, outer, inner, vals, b, num_threads=1)
    assert np.array_equal(x, x1), "thread count must not change the bits"


def test_oracle_ldlt_reports_singular():
    n = 600
    outer = np.arange(n + 1, dtype=np.int32)
    inner = np.arange(n, dtype=np.int32)
    vals = np.where(np.arange(n) == n // 2, 0.0, 2.0)
    with pytest.raises(ArithmeticError):
        O.ldlt_solve(n, outer, inner, vals, np.ones(n), num_threads=4)


@pytest.mark.parametrize("variant", ["lm", "relation", "trust_region", "huber", "active_region"])
def test_oracle_e2e_corner_scan(variant):
    s = corner_setup()
    o = s["opts"]
    if variant == "huber":
        o.huber_delta = 0.5
    if variant == "active_region":
        o.active_region = True
    rel, odo = [], [s["odo"]]
    if variant == "relation":
        rel, odo = [(0, 1, s["odo"], 1.0)], []
    nx, ny, mn, mx = s["grid"]
    p = O.OracleProblem.build(nx, ny, mn, mx, s["init"], s["scans"], odo, o, rel)
    r = p.solve(max_iterations=40, trust_region=(variant == "trust_region"))
    m, poses = p.state()
    expect_recovered(m, poses, s, r["initial_cost"], r["final_cost"], s["grid"])
    if variant == "trust_region":
        h = r["cost_history"]
        assert all(h[i] <= h[i - 1] + 1e-9 for i in range(1, len(h)))
    if variant == "active_region":
        assert p.sizes()["num_active"] < nx * ny


def test_relation_beyond_frame_count_is_skipped():
    s = corner_setup()
    nx, ny, mn, mx = s["grid"]
    p = O.OracleProblem.build(nx, ny, mn, mx, s["init"], s["scans"], [s["odo"]], s["opts"],
                              [(0, 5, s["odo"], 1.0)])
    assert p.sizes()["num_odom"] == 1
    p2 = O.OracleProblem.build(nx, ny, mn, mx, s["init"], s["scans"], [], s["opts"], [(0, 1, s["odo"], 2.0)])
    spec = p2.specs(nx, ny, mn, mx)
    assert spec.odom_sqrtw[0] == math.sqrt(1.0) * 2.0
