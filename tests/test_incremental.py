"""The incremental driver (Run in incremental mode,
src/pipeline/runner.cpp:226-285) behind sdfgpu_run_incremental: argument
checks on the host, the oracle's restatement of the loop, and GPU runs
against the oracle's (same tolerances as a single solve: cost history
1e-8 relative, poses and map 1e-4)."""
import numpy as np
import pytest

import oracle as O
import sdf_slam_b200 as P
import sdf_slam_b200.scenes as scenes


def _room(frames=6, beams=90, seed=4, **kw):
    sc = scenes.room_scene(seed=seed, frames=frames, beams=beams, **kw)
    sc.options = {}
    return sc


def _oracle_run(sc, opts, relations=(), **kw):
    return O.run_incremental(sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, opts,
                             relations=relations, num_threads=4, **kw)


def _gpu_run(sc, opts, relations=(), **kw):
    return P.run_incremental(sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, opts,
                             relations=relations, **kw)


def _assert_close(gpu, orc):
    om, op, ot = orc
    assert gpu.result.iterations == ot["iterations"]
    hg = np.array(gpu.result.cost_history)
    ho = np.array(ot["cost_history"])
    assert hg.shape == ho.shape
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8
    assert abs(gpu.result.initial_cost - ot["initial_cost"]) <= 1e-8 * abs(ot["initial_cost"])
    assert abs(gpu.result.final_cost - ot["final_cost"]) <= 1e-8 * abs(ot["final_cost"])
    assert np.max(np.abs(gpu.poses[:, :2] - op[:, :2])) <= 1e-4
    assert np.max(np.abs(gpu.map_values - om)) <= 1e-4


def test_incremental_rejects_bad_arguments():
    sc = _room(frames=3, beams=20)
    with pytest.raises(ValueError, match="increment_size"):
        _gpu_run(sc, P.ProblemOptions(), increment_size=0)
    with pytest.raises(ValueError, match="iterations_per_increment"):
        _gpu_run(sc, P.ProblemOptions(), iterations_per_increment=-1)
    with pytest.raises(ValueError, match="two scans"):
        P.run_incremental(sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses[:1], sc.scans[:1])


def test_oracle_incremental_without_iterations_integrates_odometry():
    # with no iterations the poses are the dataset poses re-integrated from
    # their own odometry, and each step records its initial cost only
    sc = _room(frames=5, beams=30)
    m, p, t = _oracle_run(sc, P.ProblemOptions(hallucination_points=2), increment_size=2,
                          iterations_per_increment=0)
    chain = [np.asarray(sc.poses[0], float)]
    for i in range(1, len(sc.poses)):
        chain.append(O.pose_op(1, chain[-1], O.pose_op(2, sc.poses[i - 1], sc.poses[i])))
    assert np.array_equal(p, np.array(chain))
    assert t["iterations"] == 0
    assert len(t["cost_history"]) == 2  # steps of frames 1-2 and 3-4
    assert np.array_equal(m, np.zeros(sc.nx * sc.ny))


@pytest.mark.gpu
@pytest.mark.parametrize("increment_size", [1, 2])
@pytest.mark.parametrize("warm", [False, True])
def test_incremental_matches_oracle(increment_size, warm):
    sc = _room()
    opts = P.ProblemOptions(hallucination_points=4)
    orc = _oracle_run(sc, opts, increment_size=increment_size, iterations_per_increment=3)
    gpu = _gpu_run(sc, opts, increment_size=increment_size, iterations_per_increment=3, warm_analysis=warm)
    _assert_close(gpu, orc)
    steps = -(-(len(sc.poses) - 1) // increment_size)
    assert gpu.phases["increments"] == steps
    if warm:
        assert gpu.phases["warm_analyses"] >= 1


@pytest.mark.gpu
def test_incremental_with_relations_and_active_region_matches_oracle():
    sc = _room(frames=7, seed=6)
    opts = P.ProblemOptions(hallucination_points=4, active_region=True, active_margin=2)
    rel = O.pose_op(2, sc.gt_poses[0], sc.gt_poses[5])
    relations = [(0, 5, rel, 4.0), (1, 6, O.pose_op(2, sc.gt_poses[1], sc.gt_poses[6]))]
    orc = _oracle_run(sc, opts, relations=relations, increment_size=2, iterations_per_increment=4)
    gpu = _gpu_run(sc, opts, relations=relations, increment_size=2, iterations_per_increment=4)
    _assert_close(gpu, orc)


@pytest.mark.gpu
def test_incremental_device_build_equals_host_build():
    sc = _room(frames=5)
    opts = P.ProblemOptions(hallucination_points=4)
    a = _gpu_run(sc, opts, iterations_per_increment=3, on_device=False)
    b = _gpu_run(sc, opts, iterations_per_increment=3, on_device=True)
    assert a.result.cost_history == b.result.cost_history
    assert a.poses.tobytes() == b.poses.tobytes() and a.map_values.tobytes() == b.map_values.tobytes()


@pytest.mark.gpu
def test_incremental_snapshots():
    sc = _room(frames=7, beams=40)
    seen = []
    out = _gpu_run(sc, P.ProblemOptions(hallucination_points=2), iterations_per_increment=2, snapshot_every=2,
                   snapshot=lambda frames, m, p: seen.append((frames, m, p)))
    assert [s[0] for s in seen] == [3, 5, 7]
    assert all(s[2].shape == (s[0], 3) for s in seen)
    assert np.array_equal(seen[-1][1], out.map_values) and np.array_equal(seen[-1][2], out.poses)
