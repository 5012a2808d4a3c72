"""The Ceres-parity comparison harness on the CPU: the restatement of the
reference's Ceres backend (oracle/ceres_formulation.py) pinned by the
reference's own tests of it, and compared with the LM backend as the
reference compares its backends (the same end-to-end recovery bounds).

Ceres is absent from this image, so parity with Ceres's iterates is unpinned;
the GPU side of the harness is `test_gpu_parity.py::test_ceres_parity_harness_corner_scan`.
"""
import math

import numpy as np
import pytest

import oracle as O
from ceres_formulation import CeresFormulation, compare, frozen_cell_point, observed_nodes, solve_ceres
from helpers import corner_setup, expect_recovered

RANDOM_MAP = (6, 5, (-3.0, -2.0), (3.0, 2.0))


def test_frozen_cell_matches_regular_eval_inside_cell():
    """tests/test_jacobians.cpp:78-102: RandomMap(mt19937(7)), pose (0.1,
    -0.2, 0.3), point (0.4, 0.5), delta 0.25: inside its cell the frozen-cell
    residual, node weights and pose partials equal the regular evaluation's
    to 1e-12."""
    nx, ny, mn, mx = RANDOM_MAP
    values = O.random_map(7)
    pose = np.array([0.1, -0.2, 0.3])
    p = (0.4, 0.5)
    regular = O.eval_point(nx, ny, mn, mx, values, pose, p, 0.25)
    assert regular["valid"]
    c, s = math.cos(pose[2]), math.sin(pose[2])
    g = (c * p[0] - s * p[1] + pose[0], s * p[0] + c * p[1] + pose[1])
    cell = O.locate(nx, ny, mn, mx, values, g)
    assert cell is not None
    ids = [cell["h"] * nx + cell["w"], cell["h"] * nx + cell["w"] + 1, (cell["h"] + 1) * nx + cell["w"],
           (cell["h"] + 1) * nx + cell["w"] + 1]
    r, dn, nid, dp = frozen_cell_point(nx, ny, mn, mx, cell["w"], cell["h"], pose, p, 0.25, values[ids])
    assert abs(r - regular["residual"]) <= 1e-12
    assert np.array_equal(nid, regular["node_ids"])
    assert np.max(np.abs(dn - regular["d_nodes"])) <= 1e-12
    assert np.max(np.abs(dp - regular["d_pose"])) <= 1e-12


@pytest.mark.parametrize("seed", [42, 7, 43])
def test_frozen_cell_jacobian_matches_finite_differences(seed):
    """The frozen-cell partials against central differences (eps 1e-6,
    tolerance 1e-5, as tests/test_jacobians.cpp checks the regular ones),
    also for a pose that moves the point out of its frozen cell."""
    nx, ny, mn, mx = RANDOM_MAP
    values = O.random_map(seed)
    rng = np.random.default_rng(seed)
    eps, tol = 1e-6, 1e-5
    for _ in range(10):
        pose = rng.uniform(-0.5, 0.5, 3)
        p = rng.uniform(-1.0, 1.0, 2)
        cw, ch = int(rng.integers(0, nx - 1)), int(rng.integers(0, ny - 1))
        ids = [ch * nx + cw, ch * nx + cw + 1, (ch + 1) * nx + cw, (ch + 1) * nx + cw + 1]
        v = values[ids]
        _, dn, _, dp = frozen_cell_point(nx, ny, mn, mx, cw, ch, pose, p, 0.3, v)
        for k in range(4):
            vp, vm = v.copy(), v.copy()
            vp[k] += eps
            vm[k] -= eps
            fd = (frozen_cell_point(nx, ny, mn, mx, cw, ch, pose, p, 0.3, vp)[0] -
                  frozen_cell_point(nx, ny, mn, mx, cw, ch, pose, p, 0.3, vm)[0]) / (2 * eps)
            assert abs(fd - dn[k]) <= tol
        for k in range(3):
            pp, pm = pose.copy(), pose.copy()
            pp[k] += eps
            pm[k] -= eps
            fd = (frozen_cell_point(nx, ny, mn, mx, cw, ch, pp, p, 0.3, v)[0] -
                  frozen_cell_point(nx, ny, mn, mx, cw, ch, pm, p, 0.3, v)[0]) / (2 * eps)
            assert abs(fd - dp[k]) <= tol


def _corner_specs(variant="ceres"):
    s = corner_setup()
    o = s["opts"]
    if variant == "huber":
        o.huber_delta = 0.5
    if variant == "active_region":
        o.active_region = True
    nx, ny, mn, mx = s["grid"]
    orc = O.OracleProblem.build(nx, ny, mn, mx, s["init"], s["scans"], [s["odo"]], o)
    return s, orc, orc.specs(nx, ny, mn, mx, huber_delta=o.huber_delta)


def test_ceres_formulation_blocks_follow_solve_ceres():
    """The residual blocks SolveCeres adds (ceres_solver.cpp:161-193): every
    point spec located in the grid at the start with four active nodes, every
    Eikonal spec with three active nodes, every odometry spec; frame 0 holds
    no parameters. Its cost at the start is half the problem's Cost()
    (no loss, every block present in both)."""
    s, orc, specs = _corner_specs()
    f = CeresFormulation(specs)
    assert f.n == f.num_active + 3 * (len(specs.poses) - 1)
    assert len(f.eikonal) == len(specs.eik_sqrtw)
    assert 0 < len(f.points) <= len(specs.pt_frame)
    cost, r, J = f.evaluate(f.pack(specs.map_values, specs.poses))
    assert J.shape == (len(r), f.n)
    if len(f.points) == len(specs.pt_frame):
        assert abs(cost - 0.5 * orc.cost()) <= 1e-12 * orc.cost()


@pytest.mark.parametrize("variant", ["ceres", "huber", "active_region"])
def test_ceres_formulation_recovers_corner_scan(variant):
    """tests/test_e2e.cpp:155-166 (backend kCeres, 60 iterations) through the
    restated Ceres backend: ExpectRecovered's bounds (final cost below 5 %
    of the initial, frame 1 within 0.1 m and 0.05 rad of the truth and
    closer than it started, mean |SDF| on the surface below 0.1); with a
    Huber loss and with the active region as well."""
    s, orc, specs = _corner_specs(variant)
    m, poses, res = solve_ceres(specs, max_iterations=60)
    expect_recovered(m, poses, s, res["initial_cost"], res["final_cost"], s["grid"])
    assert res["iterations"] <= 61


def test_ceres_parity_harness_against_the_lm_backend_on_the_cpu():
    """The comparison harness on the CPU, as the reference compares its
    backends (tests/test_e2e.cpp:90-101 and :155-166): the LM backend (the
    oracle's SolveLm, 40 iterations) and the Ceres backend (60 iterations)
    from the same CornerScan problem both pass ExpectRecovered. The frozen
    cells make the two formulations different problems, so their final
    states differ by less than the recovery bounds: poses by at most 0.1 m
    and 0.05 rad."""
    s, orc, specs = _corner_specs()
    rl = orc.solve(max_iterations=40, num_threads=1)
    lm_state = orc.state()
    m, poses, rc = solve_ceres(specs, max_iterations=60)
    expect_recovered(lm_state[0], lm_state[1], s, rl["initial_cost"], rl["final_cost"], s["grid"])
    expect_recovered(m, poses, s, rc["initial_cost"], rc["final_cost"], s["grid"])
    cmp = compare(lm_state, rl, (m, poses), rc, observed_nodes(specs))
    print("LM vs Ceres formulation:", cmp)
    assert cmp["max_pose_diff_m"] <= 0.1
    assert cmp["max_angle_diff_rad"] <= 0.05
