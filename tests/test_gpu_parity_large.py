"""GPU parity at the full benchmark sizes: the 910-pose office (200x200 grid
at 0.15 m, 1,146,600 point rows, 42,727 unknowns) and the 76-pose floor plan
(100x100 at 0.2 m, 191,520 point rows), through the C ABI against the CPU
oracle from the same input state.

Contract (the FP64 path):
* point-to-cell assignment and the sparsity patterns of J and J^T J:
  bit-exact (every rotated point uses the cos / sin of the platform's libm,
  as the reference does; the number of rows whose cell differs is counted
  and must be 0);
* residuals, Jacobian entries, J^T J, -J^T r: <= 1e-12 relative;
* the LM step delta: <= 1e-10 norm-wise relative;
* LM solves: cost history <= 1e-8 relative, poses <= 1e-4 m.
"""
import numpy as np
import pytest

import sdf_slam_b200 as P
import sdf_slam_b200.scenes as scenes
from helpers import oracle_from_specs, rel_err, scene_specs

pytestmark = pytest.mark.gpu

TOL_EVAL = 1e-12
TOL_STEP = 1e-10


@pytest.fixture(scope="module")
def office_specs():
    specs, _ = scene_specs(scenes.office_scene(seed=2))
    return specs


def _linearization_report(g, o):
    flips = int(np.count_nonzero(g["point_cell"] != o["point_cell"]))
    return {
        "cell_flips": flips,
        "residuals": rel_err(g["residuals"], o["residuals"]),
        "j_values": rel_err(g["j_values"], o["j_values"]),
        "n_values": rel_err(g["n_values"], o["n_values"]),
        "rhs": rel_err(g["rhs"], o["rhs"]),
        "step": rel_err(g["step"], o["step"]),
    }


def test_office_linearization_parity(office_specs):
    """One LM linearization of the office from a state two FP64 GPU
    iterations away from the scene's start (the same state is set on both
    sides)."""
    specs = office_specs
    gpu = P.Problem.from_specs(specs)
    P.solve(gpu, P.SolverOptions(max_iterations=2, step_tolerance=0.0))
    m, p = gpu.state()
    orc = oracle_from_specs(specs)
    orc.set_state(m, p)
    g = gpu.linearize(1.0, False)
    o = orc.linearize(1.0, False, 0, True)
    rep = _linearization_report(g, o)
    print("office linearization vs oracle:", rep)
    assert rep["cell_flips"] == 0
    assert np.array_equal(g["j_outer"], o["j_outer"]) and np.array_equal(g["j_inner"], o["j_inner"])
    assert np.array_equal(g["n_outer"], o["n_outer"]) and np.array_equal(g["n_inner"], o["n_inner"])
    for key in ("residuals", "j_values", "n_values", "rhs"):
        assert rep[key] <= TOL_EVAL, key
    assert rep["step"] <= TOL_STEP


def test_office_three_iteration_solve_parity(office_specs):
    """Three LM iterations of the office from the scene's start (odometry
    poses, zero map): cost history, poses and map against the oracle's
    SolveLm."""
    specs = office_specs
    gpu = P.Problem.from_specs(specs)
    rg = P.solve(gpu, P.SolverOptions(max_iterations=3, step_tolerance=0.0))
    orc = oracle_from_specs(specs)
    ro = orc.solve(max_iterations=3, step_tolerance=0.0, num_threads=0)
    hg = np.array(rg.cost_history)
    ho = np.array(ro["cost_history"])
    assert hg.shape == ho.shape
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8
    gm, gp = gpu.state()
    om, op = orc.state()
    assert np.max(np.abs(gp[:, :2] - op[:, :2])) <= 1e-4
    assert np.max(np.abs(gm - om)) <= 1e-4


def test_floorplan_ten_iteration_solve_parity():
    """Ten LM iterations of the 76-pose floor plan from the scene's start:
    every iteration's cost, the final poses and the map against the
    oracle."""
    specs, _ = scene_specs(scenes.floorplan_scene(seed=1))
    gpu = P.Problem.from_specs(specs)
    rg = P.solve(gpu, P.SolverOptions(max_iterations=10, step_tolerance=0.0))
    orc = oracle_from_specs(specs)
    ro = orc.solve(max_iterations=10, step_tolerance=0.0, num_threads=0)
    hg = np.array(rg.cost_history)
    ho = np.array(ro["cost_history"])
    assert hg.shape == ho.shape == (11,)
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8
    gm, gp = gpu.state()
    om, op = orc.state()
    assert np.max(np.abs(gp[:, :2] - op[:, :2])) <= 1e-4
    assert np.max(np.abs(gm - om)) <= 1e-4


def test_floorplan_cells_bit_exact_after_steps():
    """After GPU steps (the angles wrapped and rotated with the platform's
    libm on the host side of ApplyStep) the state's cells still agree bit
    for bit with the oracle evaluated at that same state."""
    specs, _ = scene_specs(scenes.floorplan_scene(seed=1))
    gpu = P.Problem.from_specs(specs)
    P.solve(gpu, P.SolverOptions(max_iterations=4, step_tolerance=0.0))
    m, p = gpu.state()
    orc = oracle_from_specs(specs)
    orc.set_state(m, p)
    rep = _linearization_report(gpu.linearize(1.0, False), orc.linearize(1.0, False, 0, True))
    assert rep["cell_flips"] == 0
    assert rep["j_values"] <= TOL_EVAL and rep["step"] <= TOL_STEP


@pytest.mark.parametrize("workload", ["floorplan", "office"])
def test_mixed_step_tensor_core_fronts(workload, office_specs):
    """Mixed precision factors the wide grid fronts in FP32 with their Schur
    complements on the tensor cores (split TF32). One LM iteration from the
    same state: without refinement the state differs from the FP64 path's by
    an FP32-level fraction of the step; with three FP64 refinement rounds by
    less than 1e-9 of it."""
    specs = office_specs if workload == "office" else scene_specs(scenes.floorplan_scene(seed=1))[0]
    base = P.Problem.from_specs(specs)
    m0, p0 = base.state()
    P.solve(base, P.SolverOptions(max_iterations=1, step_tolerance=0.0))
    m64, p64 = base.state()
    step = max(np.max(np.abs(m64 - m0)), np.max(np.abs(p64 - p0)))
    for refine, bound in [(0, 1e-3), (3, 1e-9)]:
        g = P.Problem.from_specs(specs)
        r = P.solve(g, P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision="mixed",
                                       refine_steps=refine))
        assert r.status == 0
        gm, gp = g.state()
        dev = max(np.max(np.abs(gm - m64)), np.max(np.abs(gp - p64)))
        print(f"{workload} mixed refine={refine}: max state difference {dev:.3e} of step {step:.3e}")
        assert dev <= bound * step
        g.close()


@pytest.mark.parametrize("schedule", [(128, 256, 128), (64, 128, 64), (64, 128, 0), (128, 256, 0), (32, 256, 32)])
def test_floorplan_every_factor_schedule(schedule):
    """Each factorization schedule (single-kernel fronts up to small_pivots,
    wider pivot blocks panel by panel or, with panel_rows 0, by whole outer
    blocks) gives the oracle's three-iteration solve of the floor plan."""
    specs, _ = scene_specs(scenes.floorplan_scene(seed=1))
    gpu = P.Problem.from_specs(specs)
    gpu.set_schedule(*schedule)
    rg = P.solve(gpu, P.SolverOptions(max_iterations=3, step_tolerance=0.0))
    ro = _floorplan_oracle_three()
    hg = np.array(rg.cost_history)
    ho = np.array(ro["cost_history"])
    assert hg.shape == ho.shape
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8
    gm, gp = gpu.state()
    assert np.max(np.abs(gp[:, :2] - ro["poses"][:, :2])) <= 1e-4
    assert np.max(np.abs(gm - ro["map"])) <= 1e-4


_ORACLE_CACHE = {}


def _floorplan_oracle_three():
    if "floorplan3" not in _ORACLE_CACHE:
        specs, _ = scene_specs(scenes.floorplan_scene(seed=1))
        orc = oracle_from_specs(specs)
        ro = orc.solve(max_iterations=3, step_tolerance=0.0, num_threads=0)
        om, op = orc.state()
        _ORACLE_CACHE["floorplan3"] = {"cost_history": ro["cost_history"], "poses": op, "map": om}
    return _ORACLE_CACHE["floorplan3"]


@pytest.fixture(scope="module")
def floorplan_oracle10():
    specs = scene_specs(scenes.floorplan_scene(seed=1))[0]
    orc = oracle_from_specs(specs)
    ro = orc.solve(max_iterations=10, step_tolerance=0.0, num_threads=0)
    return specs, np.array(ro["cost_history"]), orc.state()


@pytest.mark.parametrize("tc_rows", [256, 0])
def test_floorplan_mixed_follows_oracle_with_and_without_tensor_cores(tc_rows, floorplan_oracle10):
    """Ten mixed LM iterations of the floor plan from the scene's start,
    with the wide FP32 fronts' Schur complements on the tensor cores (256)
    and on the SIMT tiles (0), refinement stopped once a round corrects
    less than 1e-6 of the step: the cost history stays within 1e-8 of the
    FP64 oracle's and the poses within 1e-4 m (the mixed path's contract)."""
    specs, ho, (om, op) = floorplan_oracle10
    gpu = P.Problem.from_specs(specs)
    gpu.set_tensor_core_choice(tc_rows)
    assert gpu.tensor_core_choice()["min_rows"] == tc_rows
    rg = P.solve(gpu, P.SolverOptions(max_iterations=10, step_tolerance=0.0, precision="mixed",
                                      refine_tolerance=1e-6))
    assert rg.status == 0
    hg = np.array(rg.cost_history)
    assert hg.shape == ho.shape
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 1e-8
    gm, gp = gpu.state()
    print(f"floor plan mixed tc_rows={tc_rows}: cost history {np.max(np.abs(hg - ho) / np.abs(ho)):.3e}, "
          f"poses {np.max(np.abs(gp[:, :2] - op[:, :2])):.3e} m")
    assert np.max(np.abs(gp[:, :2] - op[:, :2])) <= 1e-4
    assert np.max(np.abs(gm - om)) <= 1e-4
    gpu.close()


def test_autotune_after_mixed_solve_picks_tensor_core_choice(floorplan_oracle10):
    """An autotune after a mixed solve times the mixed factor + refined solve
    with and without the tensor-core Schur complements and keeps the faster;
    the next mixed iteration from a saved state still agrees with the FP64
    iteration from that state to 1e-9 of the step."""
    specs = floorplan_oracle10[0]
    gpu = P.Problem.from_specs(specs)
    P.solve(gpu, P.SolverOptions(max_iterations=2, step_tolerance=0.0, precision="mixed"))
    gpu.autotune()
    choice = gpu.tensor_core_choice()
    assert choice["min_rows"] in (0, 256)
    assert choice["ms_with"] > 0.0 and choice["ms_without"] > 0.0
    assert choice["min_rows"] == (256 if choice["ms_with"] <= choice["ms_without"] else 0)
    m0, p0 = gpu.state()
    ref = P.Problem.from_specs(specs)
    ref.set_state(m0, p0)
    P.solve(ref, P.SolverOptions(max_iterations=1, step_tolerance=0.0))
    m64, p64 = ref.state()
    step = max(np.max(np.abs(m64 - m0)), np.max(np.abs(p64 - p0)))
    P.solve(gpu, P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision="mixed"))
    gm, gp = gpu.state()
    assert max(np.max(np.abs(gm - m64)), np.max(np.abs(gp - p64))) <= 1e-9 * step
    # the choice stays when the schedule is set by hand
    gpu.set_schedule(64, 128, 64)
    assert gpu.tensor_core_choice()["min_rows"] == choice["min_rows"]
    gpu.close()
    ref.close()


def test_mixed_option_ranges():
    """refine_tolerance outside [0, 1) and a tensor-core row threshold
    outside {0} and [128, 65536] are refused with the reason."""
    specs = scene_specs(scenes.room_scene(seed=0))[0]
    gpu = P.Problem.from_specs(specs)
    for tol in (-1e-3, 1.0, float("nan")):
        with pytest.raises(ValueError, match="refine_tolerance"):
            P.solve(gpu, P.SolverOptions(max_iterations=1, precision="mixed", refine_tolerance=tol))
    for rows in (5, 127, 70000):
        with pytest.raises(ValueError, match="min_rows"):
            gpu.set_tensor_core_choice(rows)
    gpu.close()
