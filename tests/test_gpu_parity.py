"""GPU parity tests: the CUDA LM path through the C ABI against the CPU oracle
on the same input state.

Tolerances (the contract of the FP64 path):
* point-to-cell assignment, the Jacobian's and the normal matrix's sparsity
  patterns: bit-exact;
* Jacobian entries, residuals, J^T J, -J^T r: <= 1e-12 relative (the kernels
  evaluate the reference's expressions unfused in its association order,
  with every pose's cos / sin from the platform's libm);
* the LM step delta: <= 1e-10 norm-wise relative (an independent FP64
  factorization with a different elimination order);
* full solves: cost history <= 1e-8 relative, poses <= 1e-4 m.
"""
import math

import numpy as np
import pytest

import oracle as O
import sdf_slam_b200 as P
import sdf_slam_b200.scenes as scenes
from helpers import corner_setup, expect_recovered, oracle_from_specs, rel_err, scene_specs

pytestmark = pytest.mark.gpu

TOL_EVAL = 1e-12
TOL_STEP = 1e-10


def _warm_state(specs, iterations=3):
    """A nontrivial identical input state: the oracle's state after a few
    iterations from the scene's start."""
    o = oracle_from_specs(specs)
    o.solve(max_iterations=iterations, num_threads=4)
    return o.state()


def _compare_linearization(g, o):
    assert np.array_equal(g["point_cell"], o["point_cell"]), "point-to-cell assignment"
    assert np.array_equal(g["j_outer"], o["j_outer"]) and np.array_equal(g["j_inner"], o["j_inner"])
    assert np.array_equal(g["n_outer"], o["n_outer"]) and np.array_equal(g["n_inner"], o["n_inner"])
    assert rel_err(g["residuals"], o["residuals"]) <= TOL_EVAL
    assert rel_err(g["j_values"], o["j_values"]) <= TOL_EVAL
    assert rel_err(g["n_values"], o["n_values"]) <= TOL_EVAL
    assert rel_err(g["rhs"], o["rhs"]) <= TOL_EVAL
    assert rel_err(g["step"], o["step"]) <= TOL_STEP


VARIANTS = {
    "smooth_node": dict(),
    "exact_gradient": dict(smooth_gradient=False),
    "smooth_meters": dict(smooth_gradient_step=0.3),
    "huber": dict(huber_delta=0.05),
    "active_region": dict(active_region=True),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_linearization_parity_room(variant):
    sc = scenes.room_scene(seed=0)
    opts = P.ProblemOptions(hallucination_points=4, **VARIANTS[variant])
    specs, _ = scene_specs(sc, opts)
    m, p = _warm_state(specs)
    gpu = P.Problem.from_specs(specs)
    gpu.set_state(m, p)
    orc = oracle_from_specs(specs)
    orc.set_state(m, p)
    for lam, marq in [(1.0, False), (0.5, True)]:
        g = gpu.linearize(lam, marq)
        o = orc.linearize(lam, marq, 4, True)
        _compare_linearization(g, o)


def test_cost_and_apply_step_parity():
    sc = scenes.room_scene(seed=3)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    m, p = _warm_state(specs, 2)
    gpu = P.Problem.from_specs(specs)
    orc = oracle_from_specs(specs)
    gpu.set_state(m, p)
    orc.set_state(m, p)
    assert abs(gpu.cost() - orc.cost()) <= 1e-12 * orc.cost()
    step = np.random.default_rng(0).normal(0, 1e-2, gpu.num_parameters())
    gpu.apply_step(step)
    orc.apply_step(step)
    gm, gp = gpu.state()
    om, op = orc.state()
    # map and poses bit for bit: the angles are wrapped (atan2(sin, cos))
    # with the platform's libm on the host side of ApplyStep
    assert np.array_equal(gm, om)
    assert np.array_equal(gp, op)
    # the cost at the stepped state again from cells that agree bit for bit
    assert abs(gpu.cost() - orc.cost()) <= 1e-12 * orc.cost()


@pytest.mark.parametrize("options", [
    dict(),
    dict(trust_region=True),
    dict(lambda_factor=2.0, reject_worse_steps=True),
    dict(marquardt_scaling=True, lambda_init=0.1),
])
def test_solve_parity_room(options):
    sc = scenes.room_scene(seed=0)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    gpu = P.Problem.from_specs(specs)
    orc = oracle_from_specs(specs)
    rg = P.solve(gpu, P.SolverOptions(max_iterations=10, **options))
    ro = orc.solve(max_iterations=10, num_threads=4, **options)
    assert rg.iterations == ro["iterations"]
    assert rg.converged == ro["converged"]
    hg = np.array(rg.cost_history)
    ho = np.array(ro["cost_history"])
    assert hg.shape == ho.shape
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8
    gm, gp = gpu.state()
    om, op = orc.state()
    assert np.max(np.abs(gp[:, :2] - op[:, :2])) <= 1e-4
    assert np.max(np.abs(gm - om)) <= 1e-4


def test_solve_is_deterministic():
    sc = scenes.room_scene(seed=2)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    outs = []
    for _ in range(2):
        gpu = P.Problem.from_specs(specs)
        r = P.solve(gpu, P.SolverOptions(max_iterations=5))
        outs.append((np.array(r.cost_history), *gpu.state()))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


def test_solve_after_releasing_cached_memory_is_unchanged():
    """sdfgpu_release_cached_memory hands the cached blocks and the pool's
    reserve back to the driver; the next handle allocates afresh and solves
    to the same bits."""
    sc = scenes.room_scene(seed=2)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    outs = []
    for _ in range(2):
        gpu = P.Problem.from_specs(specs)
        r = P.solve(gpu, P.SolverOptions(max_iterations=5))
        outs.append((np.array(r.cost_history), *gpu.state()))
        gpu.close()
        P.release_cached_memory()
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("variant", ["lm", "relation", "trust_region", "huber", "active_region"])
def test_e2e_corner_scan_gpu(variant):
    """tests/test_e2e.cpp:90-218 with the GPU backend."""
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
    prob = P.Problem(nx, ny, mn, mx, s["init"], s["scans"], odo, o, rel)
    r = P.solve(prob, P.SolverOptions(max_iterations=40, trust_region=(variant == "trust_region")))
    m, poses = prob.state()
    expect_recovered(m, poses, s, r.initial_cost, r.final_cost, s["grid"])
    if variant == "trust_region":
        h = r.cost_history
        assert all(h[i] <= h[i - 1] + 1e-9 for i in range(1, len(h)))


def test_ceres_parity_harness_corner_scan():
    """The Ceres-parity comparison harness with the GPU backend, as the
    reference compares its backends (tests/test_e2e.cpp:90-101, :155-166):
    the GPU LM (40 iterations) and the restated Ceres backend
    (oracle/ceres_formulation.py, 60 iterations) from the same CornerScan
    problem both pass ExpectRecovered, and their final poses differ by at
    most 0.1 m and 0.05 rad (the frozen cells make them different problems;
    Ceres is absent here, so its own iterates are not compared)."""
    from ceres_formulation import compare, observed_nodes, solve_ceres
    s = corner_setup()
    nx, ny, mn, mx = s["grid"]
    prob = P.Problem(nx, ny, mn, mx, s["init"], s["scans"], [s["odo"]], s["opts"])
    gspecs = prob.specs(min_corner=mn, max_corner=mx)
    ospecs = O.Specs(**{k: getattr(gspecs, k) for k in O.Specs.__dataclass_fields__})
    r = P.solve(prob, P.SolverOptions(max_iterations=40))
    gm, gp = prob.state()
    expect_recovered(gm, gp, s, r.initial_cost, r.final_cost, s["grid"])
    m, poses, rc = solve_ceres(ospecs, max_iterations=60)
    expect_recovered(m, poses, s, rc["initial_cost"], rc["final_cost"], s["grid"])
    cmp = compare((gm, gp), {"final_cost": r.final_cost}, (m, poses), rc, observed_nodes(ospecs))
    print("GPU LM vs Ceres formulation:", cmp)
    assert cmp["max_pose_diff_m"] <= 0.1 and cmp["max_angle_diff_rad"] <= 0.05
    prob.close()


def test_zero_pivot_raises_and_keeps_state():
    """lambda = 0 leaves map nodes without residual rows with a zero pivot:
    the reference throws "sparse Cholesky factorization failed" before it
    applies the step (lm_solver.cpp:354-362)."""
    sc = scenes.room_scene(seed=0)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4, weights_eikonal=0.0))
    gpu = P.Problem.from_specs(specs)
    before = gpu.state()
    with pytest.raises(RuntimeError, match="sparse Cholesky factorization failed"):
        P.solve(gpu, P.SolverOptions(max_iterations=3, lambda_init=0.0))
    after = gpu.state()
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])


def test_floorplan_full_size_linearization():
    """The 76-pose / 100x100 workload at full size: bit-exact cells and
    patterns, values and step within tolerance."""
    sc = scenes.floorplan_scene(seed=1)
    specs, _ = scene_specs(sc)
    m, p = _warm_state(specs, 2)
    gpu = P.Problem.from_specs(specs)
    gpu.set_state(m, p)
    orc = oracle_from_specs(specs)
    orc.set_state(m, p)
    _compare_linearization(gpu.linearize(1.0, False), orc.linearize(1.0, False, 0, True))


def test_batch_matches_individual_solves():
    scs = [scenes.room_scene(seed=s, grid=g, frames=f, beams=b, active_region=a)
           for s, g, f, b, a in [(10, 40, 10, 180, False), (11, 56, 14, 120, True), (12, 48, 7, 90, False)]]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=4, active_region=sc.options["active_region"]))[0]
             for sc in scs]
    batch = P.Problem.batch(specs)
    opts = [P.SolverOptions(max_iterations=6), P.SolverOptions(max_iterations=4, trust_region=True),
            P.SolverOptions(max_iterations=5)]
    rb = P.solve(batch, opts)
    for i, s in enumerate(specs):
        single = P.Problem.from_specs(s)
        r1 = P.solve(single, opts[i])
        assert rb[i].cost_history == r1.cost_history
        bm, bp = batch.state(i)
        sm, sp = single.state()
        assert np.array_equal(bm, sm) and np.array_equal(bp, sp)


def test_batch_instances_follow_the_oracle():
    """Every instance of an uneven batch (grids 40-56, 7-14 poses, 90-180
    beams, one with the active region, one with the trust region) against
    the CPU oracle's own solve of that instance: cost history within 1e-8,
    poses within 1e-4 m, iterations and convergence equal."""
    scs = [scenes.room_scene(seed=s, grid=g, frames=f, beams=b, active_region=a)
           for s, g, f, b, a in [(40, 40, 10, 180, False), (41, 56, 14, 120, True), (42, 48, 7, 90, False)]]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=4, active_region=sc.options["active_region"]))[0]
             for sc in scs]
    kw = [dict(max_iterations=6), dict(max_iterations=4, trust_region=True), dict(max_iterations=5)]
    batch = P.Problem.batch(specs)
    rb = P.solve(batch, [P.SolverOptions(**k) for k in kw])
    for i, s in enumerate(specs):
        orc = oracle_from_specs(s)
        ro = orc.solve(num_threads=4, **kw[i])
        hb = np.array(rb[i].cost_history)
        ho = np.array(ro["cost_history"])
        assert hb.shape == ho.shape
        assert np.max(np.abs(hb - ho) / np.abs(ho)) <= 1e-8
        assert rb[i].iterations == ro["iterations"] and bool(rb[i].converged) == bool(ro["converged"])
        bm, bp = batch.state(i)
        om, op = orc.state()
        assert np.max(np.abs(bp[:, :2] - op[:, :2])) <= 1e-4
        assert np.max(np.abs(bm - om)) <= 1e-4
    batch.close()


def test_state_outside_pattern_reanalyses_only_that_instance():
    # Poses moved by set_state leave the analysed coupling pattern: the cost
    # evaluation that opens the solve sees it and that instance alone is
    # re-analysed (with a wider margin) before its first linearization.
    scs = [scenes.room_scene(seed=s, grid=g, frames=f, beams=b)
           for s, g, f, b in [(20, 44, 9, 120), (21, 48, 11, 150), (22, 40, 8, 90)]]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=3))[0] for sc in scs]
    batch = P.Problem.batch(specs)
    batch.cost(0)  # the device problem and its analysis at the scenes' poses
    m1, p1 = batch.state(1)
    moved = p1.copy()
    moved[1:, 0] += 2.5  # beyond the 7-cell coupling margin of 0.25 m cells
    moved[1:, 2] += 0.05
    batch.set_state(m1, moved, index=1)
    opts = P.SolverOptions(max_iterations=4)
    rb = P.solve(batch, [opts] * 3)
    assert batch.last_profile()["reanalyses"] >= 1
    for i, s in enumerate(specs):
        single = P.Problem.from_specs(s)
        if i == 1:
            single.cost()
            single.set_state(m1, moved)
        r1 = P.solve(single, opts)
        assert rb[i].cost_history == r1.cost_history
        bm, bp = batch.state(i)
        sm, sp = single.state()
        assert np.array_equal(bm, sm) and np.array_equal(bp, sp)
    # the re-analysed solve still follows the oracle
    orc = oracle_from_specs(specs[1])
    orc.set_state(m1, moved)
    ro = orc.solve(max_iterations=4, num_threads=4)
    hg = np.array(rb[1].cost_history)
    ho = np.array(ro["cost_history"])
    assert hg.shape == ho.shape and np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8


def _recentring_run(prob, index, moved, one_step, n):
    """20 iterations, instance `index`'s poses replaced by `moved` (its map
    kept), then n one-iteration solves; the re-analyses of each solve."""
    P.solve(prob, [P.SolverOptions(max_iterations=20, step_tolerance=0.0)] * prob.count
            if prob.count > 1 else P.SolverOptions(max_iterations=20, step_tolerance=0.0))
    m, _ = prob.state(index)
    prob.set_state(m, moved, index=index)
    counts = []
    for _ in range(n):
        P.solve(prob, [one_step] * prob.count if prob.count > 1 else one_step)
        counts.append(prob.last_profile()["reanalyses"])
    return counts


def test_pattern_recentred_ahead_of_time_follows_oracle():
    # An instance whose pattern has held 20 of its iterations and whose
    # accepted state brings points within two cells of the pattern's edge
    # (here: poses moved by 1.5 m, six of the seven 0.25 m cells of the
    # coupling margin) is analysed again on a host thread and the analysis
    # replaces its pattern six of its iterations later. The results depend
    # neither on host timing nor on the batch, and follow the oracle.
    scs = [scenes.room_scene(seed=s, grid=g, frames=f, beams=b)
           for s, g, f, b in [(20, 44, 9, 120), (21, 48, 11, 150)]]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=3))[0] for sc in scs]
    probe = P.Problem.from_specs(specs[1])
    P.solve(probe, P.SolverOptions(max_iterations=20, step_tolerance=0.0))
    _, p20 = probe.state()
    moved = p20.copy()
    moved[1:, 0] += 1.5
    one = P.SolverOptions(max_iterations=1, step_tolerance=0.0)
    n = 10
    runs = []
    for _ in range(2):
        single = P.Problem.from_specs(specs[1])
        counts = _recentring_run(single, 0, moved, one, n)
        runs.append((counts, single.state()))
    counts, (sm, sp) = runs[0]
    assert sum(counts) >= 1
    # not the re-analysis a pattern overflow forces before the next iteration
    assert next(k for k, c in enumerate(counts) if c) >= 6
    assert runs[1][0] == counts
    assert np.array_equal(runs[1][1][0], sm) and np.array_equal(runs[1][1][1], sp)
    batch = P.Problem.batch(specs)
    bcounts = _recentring_run(batch, 1, moved, one, n)
    assert sum(bcounts) >= 1
    bm, bp = batch.state(1)
    assert np.array_equal(bm, sm) and np.array_equal(bp, sp)
    lone = P.Problem.from_specs(specs[0])
    P.solve(lone, P.SolverOptions(max_iterations=20, step_tolerance=0.0))
    for _ in range(n):
        P.solve(lone, one)
    lm, lp = lone.state()
    bm0, bp0 = batch.state(0)
    assert np.array_equal(bm0, lm) and np.array_equal(bp0, lp)
    # the oracle from the moved state, one-iteration solves as well
    orc = oracle_from_specs(specs[1])
    orc.solve(max_iterations=20, step_tolerance=0.0, num_threads=4)
    om, _ = orc.state()
    orc.set_state(om, moved)
    for _ in range(n):
        orc.solve(max_iterations=1, step_tolerance=0.0, num_threads=4)
    om, op = orc.state()
    assert np.max(np.abs(sp[:, :2] - op[:, :2])) <= 1e-6
    assert np.max(np.abs(sm - om)) <= 1e-6
    assert rel_err(single.cost(), orc.cost()) <= 1e-8


def test_mixed_precision_solve_follows_fp64_oracle():
    # Mixed: FP32 grid fronts, FP64 pose root, FP64 refinement. With three
    # refinement rounds the LM trajectory stays on the FP64 oracle's within
    # the contract (final cost 1e-8 relative, poses 1e-4 m); without
    # refinement the FP32 factors show.
    sc = scenes.room_scene(seed=0)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    orc = oracle_from_specs(specs)
    ro = orc.solve(max_iterations=10, num_threads=4)
    ho = np.array(ro["cost_history"])
    om, op = orc.state()
    gpu = P.Problem.from_specs(specs)
    rg = P.solve(gpu, P.SolverOptions(max_iterations=10, precision="mixed", refine_steps=3))
    hg = np.array(rg.cost_history)
    assert hg.shape == ho.shape
    assert abs(hg[-1] - ho[-1]) <= 1e-8 * abs(ho[-1])
    gm, gp = gpu.state()
    assert np.max(np.abs(gp[:, :2] - op[:, :2])) <= 1e-4
    assert np.max(np.abs(gm - om)) <= 1e-4
    raw = P.Problem.from_specs(specs)
    r0 = P.solve(raw, P.SolverOptions(max_iterations=10, precision="mixed", refine_steps=0))
    h0 = np.array(r0.cost_history)
    assert np.max(np.abs(h0 - ho) / np.abs(ho)) > 1e-12


def test_mixed_and_plain_instances_in_one_batch():
    scs = [scenes.room_scene(seed=s, grid=g, frames=f, beams=b)
           for s, g, f, b in [(30, 44, 9, 120), (31, 48, 11, 150)]]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=3))[0] for sc in scs]
    batch = P.Problem.batch(specs)
    opts = [P.SolverOptions(max_iterations=5), P.SolverOptions(max_iterations=5, precision="mixed")]
    rb = P.solve(batch, opts)
    # the plain instance is bitwise its own plain solve
    single = P.Problem.from_specs(specs[0])
    r1 = P.solve(single, opts[0])
    assert rb[0].cost_history == r1.cost_history
    assert all(np.array_equal(a, b) for a, b in zip(batch.state(0), single.state()))
    # the mixed one follows its FP64 solve within the contract
    plain = P.Problem.from_specs(specs[1])
    rp = P.solve(plain, P.SolverOptions(max_iterations=5))
    hb = np.array(rb[1].cost_history)
    hp = np.array(rp.cost_history)
    assert hb.shape == hp.shape and np.max(np.abs(hb - hp) / np.abs(hp)) <= 1e-8
    bm, bp = batch.state(1)
    pm, pp = plain.state()
    assert np.max(np.abs(bp[:, :2] - pp[:, :2])) <= 1e-4


def test_mixed_instances_with_their_own_refinement_tolerances_in_one_batch():
    """Each mixed instance of a batch refines to its own refine_tolerance and
    ends bitwise where it ends alone; the looser tolerance still keeps the
    FP64 solve's cost history within 1e-8."""
    scs = [scenes.room_scene(seed=s, grid=g, frames=f, beams=b)
           for s, g, f, b in [(32, 44, 9, 120), (33, 48, 11, 150)]]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=3))[0] for sc in scs]
    opts = [P.SolverOptions(max_iterations=5, precision="mixed"),
            P.SolverOptions(max_iterations=5, precision="mixed", refine_tolerance=1e-6)]
    batch = P.Problem.batch(specs)
    rb = P.solve(batch, opts)
    for i in range(2):
        alone = P.Problem.from_specs(specs[i])
        ra = P.solve(alone, opts[i])
        assert rb[i].cost_history == ra.cost_history
        assert all(np.array_equal(a, b) for a, b in zip(batch.state(i), alone.state()))
        alone.close()
    plain = P.Problem.from_specs(specs[1])
    rp = P.solve(plain, P.SolverOptions(max_iterations=5))
    hb = np.array(rb[1].cost_history)
    hp = np.array(rp.cost_history)
    assert hb.shape == hp.shape and np.max(np.abs(hb - hp) / np.abs(hp)) <= 1e-8
    plain.close()
    batch.close()


def test_autotuned_schedule_keeps_parity():
    sc = scenes.room_scene(seed=0)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    gpu = P.Problem.from_specs(specs)
    tune = gpu.autotune()
    assert len(tune["trials"]) >= 2 and tune["factor_ms"] > 0
    assert tune["schedule"] in [tuple(int(v) for v in t[:3]) for t in tune["trials"]]
    assert tune["factor_ms"] == min(t[3] for t in tune["trials"])
    rg = P.solve(gpu, P.SolverOptions(max_iterations=10))
    ro = oracle_from_specs(specs).solve(max_iterations=10, num_threads=4)
    hg = np.array(rg.cost_history)
    ho = np.array(ro["cost_history"])
    assert hg.shape == ho.shape and np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8


def test_server_results_equal_alone_and_in_mix():
    """Requests merged into batched cohorts while others run give, each,
    bitwise the result of their solve alone, and follow the CPU oracle's
    solve of the same request (final cost within 1e-8, poses 1e-4 m)."""
    scs = [scenes.request_scene(seed=100 + i, grid_range=(40, 70), pose_range=(8, 24), iterations=6)
           for i in range(5)]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=4))[0] for sc in scs]
    server = P.Server(memory_budget_bytes=8 << 30, max_batch=3)
    ids = [server.submit(s, P.SolverOptions(max_iterations=6)) for s in specs]
    server.drain(300000)
    for s, rid in zip(specs, ids):
        res, m, p = server.poll(rid, nx_ny=s.nx * s.ny, num_frames=len(s.poses))
        alone = P.Problem.from_specs(s)
        ra = P.solve(alone, P.SolverOptions(max_iterations=6))
        am, ap = alone.state()
        assert res.status == 0
        assert res.final_cost == ra.final_cost and res.iterations == ra.iterations
        assert np.array_equal(m, am) and np.array_equal(p, ap)
        # and the oracle's own solve of the request
        orc = oracle_from_specs(s)
        ro = orc.solve(max_iterations=6, num_threads=4)
        assert rel_err(res.final_cost, ro["final_cost"]) <= 1e-8
        _, op = orc.state()
        assert np.max(np.abs(p[:, :2] - op[:, :2])) <= 1e-4
    st = server.stats()
    assert st["completed"] == 5 and st["p99_ms"] >= st["p50_ms"] > 0
    server.close()


def _random_spd(n, width, seed):
    from test_oracle_known_answers import random_spd
    return random_spd(n, width, seed)


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_ldlt_factor_only_matches_oracle(seed):
    n = 3000 + 500 * seed // 11
    outer, inner, vals = _random_spd(n, 57, seed)
    b = np.random.default_rng(seed).uniform(-1, 1, n)
    solver = P.LdltSolver(n, outer, inner)
    solver.factorize(vals)
    x = solver.solve(b)
    xo, _ = O.ldlt_solve(n, outer, inner, vals, b, num_threads=4)
    assert rel_err(x, xo) <= 1e-13
    # refactorization with new values on the same pattern
    diag = np.array([inner[p] == j for j in range(n) for p in range(outer[j], outer[j + 1])])
    vals2 = vals + 2.5 * diag
    solver.factorize(vals2)
    x2 = solver.solve(b)
    xo2, _ = O.ldlt_solve(n, outer, inner, vals2, b, num_threads=4)
    assert rel_err(x2, xo2) <= 1e-13


def test_ldlt_factor_only_singular():
    n = 600
    outer = np.arange(n + 1, dtype=np.int32)
    inner = np.arange(n, dtype=np.int32)
    vals = np.where(np.arange(n) == n // 2, 0.0, 2.0)
    solver = P.LdltSolver(n, outer, inner)
    with pytest.raises(RuntimeError, match="factorization failed"):
        solver.factorize(vals)


def test_solve_wait_that_runs_out_reports_timeout_and_keeps_state():
    """The one-launch solve's blocks wait on flags other blocks publish, each
    wait bounded. With a flag that is never published (test hook) and a
    short limit the wait runs out: the solve fails with SDFGPU_ERR_TIMEOUT
    (TimeoutError), the state is not moved, and the device keeps working."""
    sc = scenes.room_scene(seed=1)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    gpu = P.Problem.from_specs(specs)
    P.solve(gpu, P.SolverOptions(max_iterations=1))
    assert gpu.debug_supernode_count() > 1
    before = gpu.state()
    gpu.debug_solve_fault(0, 4096)
    with pytest.raises(TimeoutError):
        P.solve(gpu, P.SolverOptions(max_iterations=2))
    after = gpu.state()
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
    gpu.debug_solve_fault(-1, 0)
    r = P.solve(gpu, P.SolverOptions(max_iterations=2))
    assert r.status == 0 and r.iterations == 2
    # two fresh handles still solve to the same bits
    a = P.Problem.from_specs(specs)
    b = P.Problem.from_specs(specs)
    ra = P.solve(a, P.SolverOptions(max_iterations=3))
    rb = P.solve(b, P.SolverOptions(max_iterations=3))
    assert ra.cost_history == rb.cost_history


def test_server_refuses_a_request_over_the_budget():
    """Admission by device footprint: a request whose own footprint exceeds
    the budget is refused at submit with SDFGPU_ERR_OUT_OF_MEMORY."""
    sc = scenes.request_scene(seed=7, grid_range=(120, 120), pose_range=(60, 60), iterations=5)
    specs, _ = scene_specs(sc, P.ProblemOptions(hallucination_points=4))
    server = P.Server(memory_budget_bytes=1 << 20, max_batch=4)
    with pytest.raises(MemoryError, match="exceeds the budget"):
        server.submit(specs, P.SolverOptions(max_iterations=5))
    assert server.stats()["submitted"] == 0
    server.close()


def test_server_cancels_a_queued_request():
    """With one request running at a time the later ones queue; a queued
    request that is cancelled is never run and polls with
    SDFGPU_ERR_INVALID_ARGUMENT, the others complete normally."""
    scs = [scenes.request_scene(seed=200 + i, grid_range=g, pose_range=f, iterations=40)
           for i, (g, f) in enumerate([((150, 150), (200, 200)), ((50, 50), (12, 12)), ((50, 50), (12, 12))])]
    specs = [scene_specs(sc, P.ProblemOptions(hallucination_points=4))[0] for sc in scs]
    server = P.Server(memory_budget_bytes=16 << 30, max_batch=1)
    ids = [server.submit(s, P.SolverOptions(max_iterations=40, step_tolerance=0.0)) for s in specs]
    server.cancel(ids[2])
    server.drain(300000)
    results = [server.poll(rid)[0] for rid in ids]
    assert results[0].status == 0 and results[1].status == 0
    assert results[0].iterations == 40 and results[1].iterations == 40
    assert results[2].status == P.SDFGPU_ERR_INVALID_ARGUMENT
    assert server.stats()["completed"] == 2
    server.close()
