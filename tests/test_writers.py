"""run_slam's output files through the library's writers (runner.cpp:82-192):
the text of every file equals the reference format written out here with
Python's %g formatting (the same conversion as a C++ stream at that
precision), and the trajectory metrics equal a restatement of Evaluate
(runner.cpp:145-170) over the oracle's RelativeTo."""
import json
import math

import numpy as np
import pytest

import oracle as O
import sdf_slam_b200 as P
import sdf_slam_b200.scenes as scenes


def _wrap(a):
    return math.atan2(math.sin(a), math.cos(a))


def _scene():
    sc = scenes.room_scene(seed=11, frames=4, beams=30)
    rng = np.random.default_rng(3)
    est = np.asarray(sc.poses, float) + rng.normal(0, 0.05, (len(sc.poses), 3))
    m = rng.normal(0, 1, sc.nx * sc.ny)
    m[5] = -0.0
    m[6] = 1e-300
    m[7] = 123456789.125
    return sc, est, m


def _expected_files(sc, est, m, result, gt):
    g = lambda v, p=17: format(v, f".{p}g")
    poses = lambda arr: "x,y,theta\n" + "".join(f"{g(a)},{g(b)},{g(c)}\n" for a, b, c in arr)
    nx, ny = sc.nx, sc.ny
    dx = (sc.max_corner[0] - sc.min_corner[0]) / (nx - 1)
    dy = (sc.max_corner[1] - sc.min_corner[1]) / (ny - 1)
    mp = f"{nx} {ny} {g(sc.min_corner[0])} {g(sc.min_corner[1])} {g(dx)} {g(dy)}\n"
    for h in range(ny):
        mp += " ".join(g(v) for v in m[h * nx:(h + 1) * nx]) + "\n"
    pts = "x,y\n"
    for f, s in enumerate(sc.scans):
        c, sn = math.cos(est[f, 2]), math.sin(est[f, 2])
        for px, py in np.asarray(s, float):
            pts += f"{g((c * px + (-sn) * py) + est[f, 0], 9)},{g((sn * px + c * py) + est[f, 1], 9)}\n"
    return {"poses_odometry.csv": poses(sc.poses), "poses_estimated.csv": poses(est), "map.txt": mp,
            "scan_points_global.csv": pts, "poses_ground_truth.csv": poses(gt)}


def _evaluate(est, gt):
    n = len(est)
    t = sum(math.hypot(*(est[i, :2] - gt[i, :2])) for i in range(n)) / n
    r = sum(abs(_wrap(est[i, 2] - gt[i, 2])) for i in range(n)) / n
    rt = rr = 0.0
    for i in range(n - 1):
        a = O.pose_op(2, est[i], est[i + 1])
        b = O.pose_op(2, gt[i], gt[i + 1])
        d = a[:2] - b[:2]
        rt += math.sqrt(d[0] * d[0] + d[1] * d[1])
        rr += abs(_wrap(a[2] - b[2]))
    return [t, r, rt / (n - 1), rr / (n - 1)]


def test_output_files_match_reference_format(tmp_path):
    sc, est, m = _scene()
    gt = np.asarray(sc.gt_poses, float)
    res = P.SolveResult(True, 7, 1234.5, 0.1, 0.25)
    metrics = P.write_run_outputs(tmp_path, sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, est,
                                  m, res, ground_truth=gt)
    for name, text in _expected_files(sc, est, m, res, gt).items():
        assert (tmp_path / name).read_text() == text, name
    assert list(metrics.values()) == _evaluate(est, gt)
    js = (tmp_path / "metrics.json").read_text()
    assert js.startswith('{\n  "converged": true,\n  "iterations": 7,\n  "initial_cost": 1234.5,\n')
    assert json.loads(js) == {"converged": True, "iterations": 7, "initial_cost": 1234.5, "final_cost": 0.1,
                              "duration_seconds": 0.25, **metrics}
    # the loaders of the reference's plotting tools read them back
    assert np.loadtxt(tmp_path / "map.txt", skiprows=1).shape == (sc.ny, sc.nx)
    assert np.array_equal(np.loadtxt(tmp_path / "poses_estimated.csv", delimiter=",", skiprows=1), est)


def test_metrics_without_ground_truth(tmp_path):
    sc, est, m = _scene()
    out = P.write_run_outputs(tmp_path, sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, est, m,
                              P.SolveResult(False, 0, 2.0, 2.0, 0.0))
    assert out is None
    assert (tmp_path / "metrics.json").read_text() == (
        '{\n  "converged": false,\n  "iterations": 0,\n  "initial_cost": 2,\n  "final_cost": 2,\n'
        '  "duration_seconds": 0\n}\n')
    assert not (tmp_path / "poses_ground_truth.csv").exists()


def test_points_outside_warning(tmp_path, capsys):
    sc, est, m = _scene()
    est = est.copy()
    est[1, :2] += 100.0  # frame 1 leaves the domain
    P.write_run_outputs(tmp_path, sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, est, m,
                        P.SolveResult())
    # GridMap::Locate's domain test (grid_map.hpp:58-63) on every global point
    dx = (sc.max_corner[0] - sc.min_corner[0]) / (sc.nx - 1)
    dy = (sc.max_corner[1] - sc.min_corner[1]) / (sc.ny - 1)
    outside = 0
    for f, s in enumerate(sc.scans):
        c, sn = math.cos(est[f, 2]), math.sin(est[f, 2])
        for px, py in np.asarray(s, float):
            fx = ((c * px + (-sn) * py) + est[f, 0] - sc.min_corner[0]) / dx
            fy = ((sn * px + c * py) + est[f, 1] - sc.min_corner[1]) / dy
            outside += fx < 0.0 or fy < 0.0 or fx > sc.nx - 1 or fy > sc.ny - 1
    total = sum(len(s) for s in sc.scans)
    assert outside >= len(sc.scans[1])
    err = capsys.readouterr().err
    assert err.startswith(f"WARNING: {outside} of {total} scan points ({100.0 * outside / total:g}%) fall outside")


def test_writer_errors():
    with pytest.raises(ValueError, match="pose count mismatch"):
        P.evaluate_trajectory(np.zeros((1, 3)), np.zeros((1, 3)))
    with pytest.raises(ValueError, match="cannot open output file"):
        P.lib().sdfgpu_write_poses(b"/nonexistent-dir/x.csv", None, 0) and P._check(
            P.lib().sdfgpu_write_poses(b"/nonexistent-dir/x.csv", None, 0))
