#!/usr/bin/env python
"""LM iterations/s of the joint Levenberg-Marquardt path on one B200.

Workload (default, `--workload office`): the 910-pose, 3-lap trajectory
through a 30 m x 30 m office (corridors 1.5-2 m, 20-30 rooms), 180 beams over
180 deg, max range 30 m, range noise N(0, 0.01 m), 200x200 SDF grid at
0.15 m, 6 hallucinated points per beam: 1,146,600 point rows, 42,727
unknowns. Seeded synthetic data (sdf-slam_b200/scenes.py) stands in for the
reference's datasets. `--workload floorplan` is the 76-pose floor plan (100x100
at 0.2 m, 360 beams).

A step is one LM iteration (residuals and Jacobian, cell sort, J^T J and
-J^T r, supernodal LDL^T, triangular solves, step, cost) of the plain FP64
path. Each timed step is a one-iteration solve call; an L2 flush (a write of
2x the 126 MB L2) runs between steps outside the timed events. `value` is
steps over the device time of the steps (CUDA events on the library's
stream, max over ranks); `e2e` times complete solves through the public API
from host buffers (problem upload, analysis, iterations, state download).

Beside the headline the line carries, on one GPU: the FP64 path's and the
mixed path's final cost, pose and map differences from the CPU oracle after
the same iterations from the same state (the oracle's time is the
`cpu_baseline`); mixed precision (`mixed`); 64 uneven instances in one engine
(`batched`); the office's incremental run (`incremental`); the serving loop
at several request rates (`served`).

Multi-GPU: replicas only. Every rank solves its own independent problem of
the same size (a different seed) on its own GPU; no data crosses GPUs; rank 0
reports the aggregate (weak scaling).

--impl reference times the CPU restatement of the reference's LM (oracle/),
built from the scene by the oracle's own Problem constructor, on the host
cores with all threads; it loads no library of this package.

--profile N runs N one-iteration solves of the workload and prints the
per-phase device times (the command the committed ncu summaries capture).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))


def _load_package():
    if "sdf_slam_b200" in sys.modules:
        return sys.modules["sdf_slam_b200"]
    pkg_dir = os.path.join(ROOT, "sdf-slam_b200")
    spec = importlib.util.spec_from_file_location("sdf_slam_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sdf_slam_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _load_scenes():
    """The scene generator alone (pure numpy), without the package and its
    library."""
    name = "sdf_slam_b200_scenes"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "sdf-slam_b200", "scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


METRIC = "LM iters/s plain FP64 vs mixed+batched at equal final cost; served p50/p99 ms"
WORKLOADS = {
    "office": "910-pose 3-lap office, 200x200 grid @0.15 m, 180 beams/180 deg, 6 hallucinated/beam",
    "floorplan": "76-pose floor-plan loop, 100x100 grid @0.2 m, 360 beams, 6 hallucinated/beam",
    "room": "10-pose room loop, 40x40 grid @0.25 m, 180 beams, 4 hallucinated/beam",
}
SEEDS = {"office": 2, "floorplan": 1, "room": 0}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except (OSError, ValueError):
            self.proc = None
            return
        # nvidia-smi needs a moment before its first sample: wait for it so
        # that the samples cover the timed region
        deadline = time.perf_counter() + 5.0
        while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
            time.sleep(0.01)

    def mark(self):
        """Start of the timed region: earlier samples are dropped (the last
        one before it is kept, as the clock the region started at)."""
        self.first = max(0, len(self.lines) - 1)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines[self.first:]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _init_dist(world):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    # replicas only: no data-path collective, the process group carries the
    # barrier and the max-over-ranks reduction of the timings
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return dist


def _reduce(dist, value, op):
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op))
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def make_scene(scenes, workload, seed):
    return scenes.WORKLOADS[workload](seed=seed)


def scene_specs(P, scene, options=None):
    """The product's host builder (Problem::Problem) -> flat specs."""
    prob = P.Problem.from_scene(scene, options)
    out = prob.specs(min_corner=scene.min_corner, max_corner=scene.max_corner)
    prob.close()
    return out


def _oracle_problem(specs):
    O = _oracle()
    s = O.Specs(**{k: getattr(specs, k) for k in O.Specs.__dataclass_fields__})
    return O.OracleProblem.from_specs(s)


def _oracle_scene_problem(scene, options=None):
    """The oracle's own Problem constructor on the scene (hallucination,
    normals, Eikonal and odometry specs restated from the reference)."""
    O = _oracle()
    opts = O.OracleOptions()
    for k, v in scene.options.items():
        setattr(opts, k, v)
    for k, v in (options or {}).items():
        setattr(opts, k, v)
    return O.OracleProblem.build(scene.nx, scene.ny, scene.min_corner, scene.max_corner, scene.poses,
                                 scene.scans, scene.odometry, opts)


def _state_errors(cost_a, state_a, cost_b, state_b):
    import numpy as np
    return {"final_cost_rel_err": abs(cost_a - cost_b) / abs(cost_b),
            "max_pose_err_m": float(np.max(np.abs(state_a[1][:, :2] - state_b[1][:, :2]))),
            "max_angle_err_rad": float(np.max(np.abs(state_a[1][:, 2] - state_b[1][:, 2]))),
            "max_map_err": float(np.max(np.abs(state_a[0] - state_b[0])))}


class L2Flusher:
    """Writes 2x the 126 MB L2 between timed steps (cuda-python runtime; no
    torch in the process, so that ncu sees the library's kernels)."""

    BYTES = 2 * 126 * 1000 * 1000

    def __init__(self):
        from cuda.bindings import runtime as rt
        self.rt = rt
        err, self.ptr = rt.cudaMalloc(self.BYTES)
        if err != rt.cudaError_t.cudaSuccess:
            raise RuntimeError(f"cudaMalloc for the L2 flush failed: {err}")
        self.value = 0

    def flush(self):
        self.value = (self.value + 1) & 0xFF
        self.rt.cudaMemset(self.ptr, self.value, self.BYTES)
        self.sync()

    def sync(self):
        self.rt.cudaDeviceSynchronize()

    def close(self):
        self.rt.cudaFree(self.ptr)


def run_reference(args, dist, rank):
    """The reference's CPU LM (the oracle port, all host threads) on the
    same workload: one untimed iteration, then a bounded sample of the K
    timed iterations (as many as fit args.ref_budget_s at the warm-up
    iteration's pace, at least one)."""
    if rank != 0:
        return 0
    scenes = _load_scenes()
    scene = make_scene(scenes, args.workload, args.seed if args.seed is not None else SEEDS[args.workload])
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    _oracle_scene_problem(scene).solve(max_iterations=1, step_tolerance=0.0, num_threads=threads)
    per_iter = time.perf_counter() - t0
    timed = max(1, min(args.steps, int(args.ref_budget_s / max(per_iter, 1e-9))))
    orc = _oracle_scene_problem(scene)
    t0 = time.perf_counter()
    res = orc.solve(max_iterations=timed, step_tolerance=0.0, num_threads=threads)
    wall = time.perf_counter() - t0
    rate = res["iterations"] / wall
    sample = (f"{res['iterations']} of the {args.steps} LM iterations from the scene's start "
              f"({wall:.1f} s), after 1 untimed iteration")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "LM iters/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / max(1, res["iterations"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic (seeded {args.workload}, scenes.py)",
        "config": {"workload": WORKLOADS[args.workload], "threads": threads,
                   "problem": "built by the oracle's Problem constructor"},
        "cpu_baseline": {"value": rate, "unit": "LM iters/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "LM iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phase_s": dict(zip(["assemble", "normal", "factor", "solve", "cost"],
                            [float(v) for v in res["phase_seconds"]])),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_profile(args):
    """One-iteration solves printing the per-phase device times; the process
    loads no CUDA library but the package's (for ncu captures)."""
    P = _load_package()
    import sdf_slam_b200.scenes as scenes
    scene = make_scene(scenes, args.workload, args.seed if args.seed is not None else SEEDS[args.workload])
    specs = scene_specs(P, scene)
    gpu = P.Problem.from_specs(specs)
    if args.tensor_core_min_rows is not None:
        gpu.set_tensor_core_choice(args.tensor_core_min_rows)
    opts = P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision=args.precision,
                           refine_steps=args.refine_steps, refine_tolerance=args.refine_tolerance)
    for it in range(args.profile):
        if it == 1:
            gpu.kernel_timing()  # every kernel class, from the second iteration on
        r = P.solve(gpu, opts)
        prof = gpu.last_profile()
        print(f"iteration {it}: cost {r.final_cost:.9e} " +
              " ".join(f"{k}={v * 1e3:.3f}ms" if isinstance(v, float) and k != "factor_flops" else f"{k}={v}"
                       for k, v in prof.items()), flush=True)
    if args.profile > 1:
        n = args.profile - 1
        for name, t in gpu.kernel_times().items():
            if t["launches"]:
                rate = t["work"] / (t["ms"] * 1e-3) / (1e9 if t["work_unit"] == "bytes" else 1e12)
                unit = "GB/s" if t["work_unit"] == "bytes" else "TFLOP/s"
                print(f"kernel {name}: {t['ms'] / n:.3f} ms/iteration, {t['launches'] / n:.1f} launches/iteration, "
                      f"{rate:.2f} {unit}", flush=True)
    gpu.close()
    return 0


def _timed_solves(P, prob, opts1, steps, flusher, spans=None):
    """One-iteration solves, L2 flushed before each; device span of each
    (the library's events), launches and phase times summed. `spans`
    (a dict, optional) receives every step's span and the pattern
    re-analyses that ran inside the timed steps."""
    import numpy as np
    device = 0.0
    launches = 0
    phases = np.zeros(5)
    each = []
    reanalyses = 0
    for _ in range(steps):
        flusher.flush()
        P.solve(prob, opts1)
        prof = prob.last_profile()
        device += prof["span"]
        each.append(prof["span"])
        reanalyses += int(prof["reanalyses"])
        launches += prof["launches"]
        phases += [prof["assemble"], prof["normal"], prof["factor"], prof["solve"], prof["update"]]
    if spans is not None:
        spans["spans"] = each
        spans["reanalyses"] = reanalyses
    return device, launches, phases


def _span_summary(spans):
    """Median step and the timed steps' pattern re-analyses: a step whose
    state left the analysed pattern pays a host re-analysis inside it."""
    import numpy as np
    return {"median_ms_per_step": 1000.0 * float(np.median(spans["spans"])),
            "reanalyses_in_timed_steps": spans["reanalyses"]}


PHASES = ["assemble", "normal", "factor", "solve", "update"]


def run_oracle_comparison(P, args, specs):
    """The FP64 and mixed GPU paths against the CPU oracle after the same
    iterations from the same state (the scene's start); the oracle's run is
    the CPU baseline."""
    threads = os.cpu_count() or 1
    iters = args.cpu_iterations
    orc = _oracle_problem(specs)
    t0 = time.perf_counter()
    ro = orc.solve(max_iterations=iters, step_tolerance=0.0, num_threads=threads)
    dt = time.perf_counter() - t0
    ostate = orc.state()
    out = {"iterations": iters}
    for precision in ("fp64", "mixed"):
        g = P.Problem.from_specs(specs)
        r = P.solve(g, P.SolverOptions(max_iterations=iters, step_tolerance=0.0, precision=precision,
                                       refine_steps=args.refine_steps, refine_tolerance=args.refine_tolerance))
        out[precision] = _state_errors(r.final_cost, g.state(), ro["final_cost"], ostate)
        out[precision]["final_cost"] = r.final_cost
        g.close()
    out["oracle_final_cost"] = ro["final_cost"]
    cpu = {"value": ro["iterations"] / dt, "unit": "LM iters/s", "cores": threads, "kind": "port",
           "sample": f"{ro['iterations']} LM iterations of the same workload from its start ({dt:.1f} s)"}
    return out, cpu


def run_mixed(P, args, specs, flusher, state0):
    """The same workload with precision "mixed": LM iterations/s
    (one-iteration solves, L2 flushed between them), timed from `state0`,
    the state the plain FP64 timed steps started from (so that both meet
    the same pattern re-analyses)."""
    prob = P.Problem.from_specs(specs)
    opts1 = P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision="mixed",
                            refine_steps=args.refine_steps, refine_tolerance=args.refine_tolerance)
    prob.set_state(*state0)
    for _ in range(args.warmup):
        P.solve(prob, opts1)
    if not args.no_autotune:
        prob.autotune()
    # whether the autotuner kept the tensor-core Schur complements, with the
    # mixed factor + solve times it measured both ways
    tc_choice = prob.tensor_core_choice()
    prob.set_state(*state0)
    P.solve(prob, opts1)
    prob.set_state(*state0)
    steps = args.steps
    spans = {}
    device, launches, phases = _timed_solves(P, prob, opts1, steps, flusher, spans)
    kernels = kernel_profile(P, prob, opts1, flusher)
    prob.close()
    out = {"value": steps / device, "unit": "LM iters/s", "refine_steps": args.refine_steps,
           "refine_tolerance": args.refine_tolerance, "tensor_core_choice": tc_choice, "steps": steps,
           **_span_summary(spans),
           "phase_ms_per_step": {k: 1000.0 * v / steps for k, v in zip(PHASES, phases)}, "kernels": kernels}
    tc = kernels.get("KSchurTc")
    if tc:
        # split TF32 runs three tensor-core products per useful one; the
        # TF32 dense rate of B200 is half its BF16 rate
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except OSError:
            pass
        bf16 = peaks.get("bf16_tflops")
        tf32 = bf16 / 2 if bf16 else 1590.0 / 2
        out["roofline_tensor_core"] = {
            "kernel": "KSchurTc", "bound": "tensor", "unit": "TFLOP/s",
            "achieved_useful": tc["achieved"], "achieved_executed": 3 * tc["achieved"], "peak": tf32,
            "frac": 3 * tc["achieved"] / tf32,
            "peak_source": ("half the measured BF16 burst rate (MEASURED_PEAKS.json bf16_tflops): TF32 dense "
                            "runs at half the BF16 rate" if bf16 else "half the fallback BF16 1590 TFLOP/s")}
    return out


def run_batch(P, args, flusher):
    """Uneven independent instances solved together in one engine (every
    kernel of an iteration covers all of them): aggregate LM iterations/s,
    plain FP64 and mixed, and the per-instance final cost against the CPU
    oracle after the same iterations (on a sample of the instances)."""
    import numpy as np
    import sdf_slam_b200.scenes as scenes
    scs = scenes.batch_scenes(seed=3, count=args.batch_count)
    specs = [scene_specs(P, sc, P.ProblemOptions(hallucination_points=4, active_region=sc.options["active_region"]))
             for sc in scs]
    count = len(specs)
    steps = max(3, min(20, args.steps // 5))
    out = {"instances": count, "unit": "LM iters/s (all instances)",
           "point_rows": sum(len(s.pt_frame) for s in specs),
           "workload": "uneven room-style instances, grid 40-150 @0.25 m, 10-200 poses, 90-360 beams, "
                       "every other one active-region", "steps": steps}
    for precision in ("fp64", "mixed"):
        batch = P.Problem.batch(specs)
        opts1 = [P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision=precision)] * count
        for _ in range(2):
            P.solve(batch, opts1)
        if not args.no_autotune:
            out.setdefault("schedule", {})[precision] = batch.autotune()["schedule"]
        device = 0.0
        reanalyses = 0
        for _ in range(steps):
            flusher.flush()
            P.solve(batch, opts1)
            device += batch.last_profile()["span"]
            reanalyses += int(batch.last_profile()["reanalyses"])
        out[precision] = {"value": count * steps / device, "ms_per_batched_iteration": 1000.0 * device / steps,
                          "reanalyses_in_timed_steps": reanalyses}
        batch.close()
    # final cost after `iters` iterations from the scenes' start, against the
    # oracle's, on every `stride`-th instance
    iters, stride = 5, max(1, count // 8)
    sample = list(range(0, count, stride))
    errs = {"fp64": [], "mixed": []}
    finals = {}
    for precision in ("fp64", "mixed"):
        batch = P.Problem.batch(specs)
        res = P.solve(batch, [P.SolverOptions(max_iterations=iters, step_tolerance=0.0, precision=precision)] * count)
        finals[precision] = [res[i].final_cost for i in range(count)]
        batch.close()
    for i in sample:
        ro = _oracle_problem(specs[i]).solve(max_iterations=iters, step_tolerance=0.0, num_threads=0)
        for precision in ("fp64", "mixed"):
            errs[precision].append(abs(finals[precision][i] - ro["final_cost"]) / abs(ro["final_cost"]))
    out["vs_oracle"] = {"iterations": iters, "instances": sample,
                        "max_final_cost_rel_err": {k: float(np.max(v)) for k, v in errs.items()}}
    out["value"] = out["fp64"]["value"]
    return out


def run_batch_office(P, args, flusher, plain_value):
    """`office_batch` independent 910-pose offices (different seeds) in one
    engine: every kernel of an iteration covers all of them. Aggregate LM
    iterations/s with plain FP64 and mixed precision (one-iteration solves,
    L2 flushed between them), against the single office's plain FP64
    iterations/s, and each mixed instance's final cost against its FP64
    solve after the same iterations from the same start."""
    import numpy as np
    import sdf_slam_b200.scenes as scenes
    count = args.office_batch
    specs = [scene_specs(P, scenes.office_scene(seed=100 + q)) for q in range(count)]
    steps = max(3, min(10, args.steps // 4))
    out = {"instances": count, "unit": "LM iters/s (all instances)", "steps": steps,
           "workload": "910-pose offices (seeds 100..), 200x200 @0.15 m, 180 beams, 6 hallucinated/beam"}
    for precision in ("fp64", "mixed"):
        batch = P.Problem.batch(specs)
        opts1 = [P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision=precision,
                                 refine_steps=args.refine_steps, refine_tolerance=args.refine_tolerance)] * count
        # past the first iterations, whose large pose moves re-analyse the
        # patterns of most instances (the single office is timed as far in)
        for _ in range(args.office_batch_warmup):
            P.solve(batch, opts1)
        device = 0.0
        phases = np.zeros(5)
        reanalyses = 0
        for _ in range(steps):
            flusher.flush()
            P.solve(batch, opts1)
            prof = batch.last_profile()
            device += prof["span"]
            reanalyses += int(prof["reanalyses"])
            phases += [prof["assemble"], prof["normal"], prof["factor"], prof["solve"], prof["update"]]
        out[precision] = {"value": count * steps / device, "ms_per_batched_iteration": 1000.0 * device / steps,
                          "reanalyses_in_timed_steps": reanalyses, "warmup_iterations": args.office_batch_warmup,
                          "phase_ms": {k: 1000.0 * v / steps for k, v in zip(PHASES, phases)},
                          "over_single_plain": count * steps / device / plain_value}
        batch.close()
    iters = 3
    finals = {}
    for precision in ("fp64", "mixed"):
        batch = P.Problem.batch(specs)
        res = P.solve(batch, [P.SolverOptions(max_iterations=iters, step_tolerance=0.0, precision=precision,
                                              refine_steps=args.refine_steps, refine_tolerance=args.refine_tolerance)] * count)
        finals[precision] = np.array([r.final_cost for r in res])
        batch.close()
    out["mixed"]["max_final_cost_rel_err_vs_fp64"] = float(
        np.max(np.abs(finals["mixed"] - finals["fp64"]) / np.abs(finals["fp64"])))
    out["mixed"]["iterations_compared"] = iters
    return out


def run_incremental(P, args, scene):
    """The office's incremental run (runner.cpp:226-285): 909 steps of
    `incremental_iterations` LM iterations over the frames so far, then a
    100-iteration batch polish of the result, on the GPU."""
    t0 = time.perf_counter()
    inc = P.run_incremental_scene(scene, solver=P.SolverOptions(step_tolerance=0.0),
                                  iterations_per_increment=args.incremental_iterations)
    t_inc = time.perf_counter() - t0
    prob = P.Problem.from_scene(scene)
    prob.set_state(inc.map_values, inc.poses)
    t0 = time.perf_counter()
    pol = P.solve(prob, P.SolverOptions(max_iterations=100, step_tolerance=1e-3))
    t_pol = time.perf_counter() - t0
    prob.close()
    return {"steps": inc.phases["increments"], "iterations_per_step": args.incremental_iterations,
            "seconds": t_inc, "lm_iterations": inc.result.iterations,
            "lm_iters_s": inc.result.iterations / t_inc, "final_cost": inc.result.final_cost,
            "phases_s": {k: inc.phases[k] for k in ("build", "setup", "solve", "reanalysis", "capture")},
            "reanalyses": inc.phases["reanalyses"],
            "polish": {"iterations": pol.iterations, "seconds": t_pol, "final_cost": pol.final_cost,
                       "converged": pol.converged, "step_tolerance": 1e-3}}


def run_serve(P, args):
    """Poisson streams of solve requests through the serving loop at each
    rate of args.serve_rates: throughput and p50/p99 latency of a warm
    server (two untimed passes over other requests of the same distribution
    come first), and the final cost of a sample of requests against the CPU
    oracle's 20-iteration solve of the same problem."""
    cold = None
    for warm_seed in (1500, 2500):
        r = _serve_pass(P, args, warm_seed, args.serve_rates[0])
        cold = cold or {k: r[k] for k in ("p50_ms", "p99_ms", "throughput_req_s")}
    rates = {}
    for q, rate in enumerate(args.serve_rates):
        rates[str(rate)] = _serve_pass(P, args, 500 + 100 * q, rate, check_oracle=(q == 0))
    return {"rates": rates, "cold_first_pass": cold, "warmup_passes": 2,
            "iterations_per_request": args.serve_iterations,
            "workload": "room-style requests, grid log-U[40,200] @0.25 m, 10-400 poses, 180 beams"}


def _serve_pass(P, args, seed0, rate, check_oracle=False):
    """One pass of args.serve_requests requests (scene seeds seed0, seed0+1,
    ...) with Poisson arrivals at `rate`, on a fresh server."""
    import numpy as np
    import sdf_slam_b200.scenes as scenes
    rng = np.random.default_rng(seed0 + 7)
    reqs = []
    for i in range(args.serve_requests):
        sc = scenes.request_scene(seed=seed0 + i, iterations=args.serve_iterations)
        reqs.append(scene_specs(P, sc, P.ProblemOptions(hallucination_points=4)))
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    server = P.Server(memory_budget_bytes=int(args.serve_budget_gb * (1 << 30)), max_batch=args.serve_batch)
    opts = P.SolverOptions(max_iterations=args.serve_iterations, step_tolerance=0.0, precision=args.precision)
    t0 = time.perf_counter()
    ids = []
    due = t0
    for spec, gap in zip(reqs, gaps):
        due += gap
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        ids.append(server.submit(spec, opts))
    last_arrival = time.perf_counter() - t0
    server.drain(600000)
    wall = time.perf_counter() - t0
    st = server.stats()
    ok = 0
    finals = []
    for spec, rid in zip(reqs, ids):
        res, _, _ = server.poll(rid)
        ok += int(res.status == 0)
        finals.append(res.final_cost)
    server.close()
    out = {"requests": len(reqs), "completed_ok": ok, "rate_req_s": rate,
           "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "throughput_req_s": len(reqs) / wall,
           # throughput counts the arrival window and the drain after it: a
           # server that keeps up drains in about one request's latency
           "arrival_window_s": last_arrival, "drain_after_last_arrival_s": wall - last_arrival,
           "lm_iters_s": st["iterations_per_s"]}
    if check_oracle:
        # the oracle on the smallest requests of the pass, as many as fit
        # args.serve_oracle_budget_s
        order = sorted(range(len(reqs)), key=lambda i: len(reqs[i].pt_frame))
        errs, idx = [], []
        t0 = time.perf_counter()
        for i in order:
            if time.perf_counter() - t0 > args.serve_oracle_budget_s:
                break
            ro = _oracle_problem(reqs[i]).solve(max_iterations=args.serve_iterations, step_tolerance=0.0,
                                                num_threads=0)
            errs.append(abs(finals[i] - ro["final_cost"]) / abs(ro["final_cost"]))
            idx.append(i)
        out["vs_oracle"] = {"requests": idx, "max_final_cost_rel_err": float(max(errs)) if errs else None}
    return out


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of a
# kernel class on a workload, from the committed one-kernel ncu captures
# named beside each entry (L2 flushed before the captured step, as here).
# DRAM bytes (read + written) per launch of a kernel class, averaged over its
# launches in one iteration of the workload, from one-kernel ncu captures
# (-k <kernel>, one iteration's launches; dram__bytes_read / _write)
# summarised in profiles/launch_list_office.md
KERNEL_TRAFFIC_BYTES = {
    ("office", "KSchur"): 3054.4e6 / 20,   # the 20 Schur launches of the iteration
    ("office", "KDenseRoot"): 33.4e6,
    ("office", "KSolveTree"): 275.2e6,
    ("office", "KFactorFront"): 137.0e6 / 10,
}


def kernel_profile(P, prob, opts1, flusher, iterations=3):
    """Device time, launches and achieved rate per kernel class over
    `iterations` one-iteration solves with every class timed."""
    prob.kernel_timing()
    for _ in range(iterations):
        flusher.flush()
        P.solve(prob, opts1)
    times = prob.kernel_times()
    prob.kernel_timing([])
    out = {}
    for name, t in times.items():
        if t["launches"] == 0:
            continue
        rate = t["work"] / (t["ms"] * 1e-3) if t["ms"] > 0 else 0.0
        out[name] = {"ms_per_iteration": t["ms"] / iterations, "launches_per_iteration": t["launches"] / iterations,
                     "achieved": rate / (1e9 if t["work_unit"] == "bytes" else 1e12),
                     "achieved_unit": "GB/s" if t["work_unit"] == "bytes" else "TFLOP/s"}
    return out


def run_gpu(args, dist, world, rank, local):
    import numpy as np
    P = _load_package()
    import sdf_slam_b200.scenes as scenes
    seed = (args.seed if args.seed is not None else SEEDS[args.workload]) + rank
    scene = make_scene(scenes, args.workload, seed)
    specs = scene_specs(P, scene)
    flusher = L2Flusher()
    opts1 = P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision=args.precision)
    prob = P.Problem.from_specs(specs)
    # warm-up: upload, symbolic analysis, first iterations; then the
    # autotuner picks the factorization schedule
    for _ in range(args.warmup):
        P.solve(prob, opts1)
    tune = prob.autotune() if not args.no_autotune else None
    P.solve(prob, opts1)
    # per-kernel device times of three iterations (every kernel class timed),
    # then the timed region times the dominant class alone
    kernels = kernel_profile(P, prob, opts1, flusher)
    dominant_kernel = max(kernels, key=lambda k: kernels[k]["ms_per_iteration"])
    prob.kernel_timing([dominant_kernel])
    flusher.sync()
    _barrier(dist)
    sampler = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)) \
        if rank == 0 else None
    if sampler:
        sampler.start()
    flusher.sync()
    _barrier(dist)
    if sampler:
        sampler.mark()
    wall0 = time.perf_counter()
    state0 = prob.state()
    spans = {}
    device_s, launches, phases = _timed_solves(P, prob, opts1, args.steps, flusher, spans)
    flusher.sync()
    _barrier(dist)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop() if sampler else None
    dom = prob.kernel_times()[dominant_kernel]
    prob.kernel_timing([])
    prof_last = prob.last_profile()
    flops = prof_last["factor_flops"]
    device_max = _reduce(dist, device_s, "MAX")
    wall_max = _reduce(dist, wall, "MAX")
    total_steps = _reduce(dist, args.steps, "SUM")
    # end to end through the public API from host buffers
    e2e_iters = args.e2e_iterations
    h2d = specs.host_bytes()
    e2e_t = 0.0
    d2h = 0
    if args.e2e_steps > 0:
        # one untimed call: the first in a process pays one-time costs (the
        # caching allocators' first device and pinned blocks for a second
        # resident problem), as the warm-up steps do for the device loop
        w2 = P.Problem.from_specs(specs)
        P.solve(w2, P.SolverOptions(max_iterations=e2e_iters, step_tolerance=0.0, precision=args.precision))
        w2.state()
        w2.close()
    for _ in range(args.e2e_steps):
        flusher.sync()
        t0 = time.perf_counter()
        p2 = P.Problem.from_specs(specs)
        r = P.solve(p2, P.SolverOptions(max_iterations=e2e_iters, step_tolerance=0.0, precision=args.precision))
        m, poses = p2.state()
        e2e_t += time.perf_counter() - t0
        d2h = m.nbytes + poses.nbytes + 8 * len(r.cost_history)
        p2.close()
    e2e_t = _reduce(dist, e2e_t, "MAX")
    e2e_value = world * args.e2e_steps * e2e_iters / e2e_t if e2e_t > 0 else 0.0
    single = world == 1
    mixed = run_mixed(P, args, specs, flusher, state0) if (single and not args.no_mixed) else None
    batched = run_batch(P, args, flusher) if (args.batch_count > 0 and single) else None
    plain_value = total_steps / device_max
    batched_office = (run_batch_office(P, args, flusher, plain_value)
                      if (args.office_batch > 0 and single and args.workload == "office") else None)
    flusher.close()
    fp64_peak = P.measure_fp64_peak() if rank == 0 else None
    vs_oracle, cpu = (None, None)
    if single and not args.no_cpu_baseline:
        vs_oracle, cpu = run_oracle_comparison(P, args, specs)
    incremental = run_incremental(P, args, scene) if (single and args.workload == "office"
                                                      and not args.no_incremental) else None
    served = run_serve(P, args) if (args.serve_requests > 0 and single) else None
    if rank != 0:
        return 0
    z = prob.sizes()
    per_step = phases / args.steps
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs")
    hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if hbm else "fallback 6650 GB/s"
    hbm = hbm or 6650.0
    # algorithmic bytes of the assembly phase per iteration (row kernels + sort)
    P_rows = z["num_points"]
    assemble_bytes = P_rows * (40 + 64 + 4) + P_rows * 4 * 2 * 2 * 2
    # the dominant kernel, timed live over the timed region (CUDA events on
    # the library's stream around each of its launches)
    launches_dom = max(1, dom["launches"])
    avg_ms = dom["ms"] / launches_dom
    work_per_launch = dom["work"] / launches_dom
    if dom["work_unit"] == "bytes":
        achieved = work_per_launch / (avg_ms * 1e-3) / 1e9
        peak, unit, bound, src = hbm, "GB/s", "hbm", hbm_src
    else:
        achieved = work_per_launch / (avg_ms * 1e-3) / 1e12
        peak, unit, bound = fp64_peak, "TFLOP/s", "tensor"
        src = "measured FP64 FMA throughput of this GPU (sdfgpu_measure_fp64_peak): the FP64 pipe bounds it"
    roofline = {
        "bound": bound, "achieved": achieved, "peak": peak, "unit": unit, "frac": achieved / peak,
        "traffic": KERNEL_TRAFFIC_BYTES.get((args.workload, dominant_kernel)),
        "traffic_source": "one-kernel ncu capture, DRAM bytes per launch (profiles/launch_list_office.md)",
        "kernel": dominant_kernel, "peak_source": src, "launches_timed": dom["launches"],
        "avg_launch_ms": avg_ms, "work_per_launch": work_per_launch, "work_unit": dom["work_unit"]}
    roofline_factor = {
        "bound": "tensor", "achieved": flops / per_step[2] / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
        "frac": flops / per_step[2] / 1e12 / fp64_peak,
        "kernel": "factor phase (every factorization kernel), FP64",
        "peak_source": "measured FP64 FMA throughput of this GPU (sdfgpu_measure_fp64_peak)",
        "useful_flop_per_iteration": flops}
    roofline_assemble = {
        "bound": "hbm", "achieved": assemble_bytes / per_step[0] / 1e9, "peak": hbm, "unit": "GB/s",
        "frac": assemble_bytes / per_step[0] / 1e9 / hbm, "traffic": None,
        "kernel": "assembly phase (point rows + cell sort)", "peak_source": hbm_src}
    line = {
        "metric": METRIC, "value": total_steps / device_max, "unit": "LM iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * device_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic (seeded {args.workload}, scenes.py)",
        "config": {"workload": WORKLOADS[args.workload], "seed": seed, "precision": args.precision,
                   "unknowns": z["num_parameters"], "point_rows": z["num_points"],
                   "l2": "flushed between steps (2x126 MB write)", "parallelism": f"replicas x{world}"},
        "wall_ms_per_step": 1000.0 * wall_max / args.steps,
        **_span_summary(spans),
        "phase_ms_per_step": {k: 1000.0 * v for k, v in zip(PHASES, per_step)},
        "factor_gflop_per_step": flops / 1e9,
        "gpu_launches": int(launches),
        "roofline": roofline,
        "roofline_phases": {"factor": roofline_factor, "assemble": roofline_assemble},
        "kernels": kernels,
        "cpu_baseline": cpu,
        "vs_oracle": vs_oracle,
        "e2e": {"value": e2e_value, "unit": "LM iters/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "iterations_per_step": e2e_iters},
        "clocks": clocks,
        "schedule": {"small_pivots": tune["schedule"][0], "front_rows": tune["schedule"][1],
                     "panel_rows": tune["schedule"][2], "factor_ms": tune["factor_ms"],
                     "trials": len(tune["trials"])} if tune else None,
        "mixed": mixed,
        "mixed_over_fp64": mixed["value"] / (total_steps / device_max) if mixed else None,
        "batched": batched,
        "batched_office": batched_office,
        "incremental": incremental,
        "served": served,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="office", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--profile", type=int, default=0, help="print per-phase times of N one-iteration solves")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--e2e-iterations", type=int, default=10)
    ap.add_argument("--cpu-iterations", type=int, default=3)
    ap.add_argument("--ref-budget-s", type=float, default=90.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-incremental", action="store_true")
    ap.add_argument("--incremental-iterations", type=int, default=5)
    ap.add_argument("--refine-steps", type=int, default=3)
    ap.add_argument("--tensor-core-min-rows", type=int, default=None,
                    help="--profile runs: the tensor-core Schur choice of mixed solves (0: none)")
    ap.add_argument("--refine-tolerance", type=float, default=1e-6,
                    help="mixed solves: refinement stops once a round's largest correction is this fraction "
                         "of the step's largest entry (the library's default is 1e-13)")
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--office-batch", type=int, default=8)
    ap.add_argument("--office-batch-warmup", type=int, default=8)
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[50.0, 100.0, 200.0, 500.0])
    ap.add_argument("--serve-iterations", type=int, default=20)
    ap.add_argument("--serve-batch", type=int, default=16)
    ap.add_argument("--serve-budget-gb", type=float, default=32.0)
    ap.add_argument("--serve-oracle-budget-s", type=float, default=20.0)
    args = ap.parse_args()
    if args.profile > 0:
        return run_profile(args)
    world, rank, local = _dist()
    if world > 1 and args.impl == "b200":
        # one GPU per rank
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    dist = _init_dist(world)
    try:
        if args.impl == "reference":
            rc = run_reference(args, dist, rank)
        else:
            rc = run_gpu(args, dist, world, rank, local)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
