#!/usr/bin/env python
"""LM iterations/s of the joint Levenberg-Marquardt path (plain FP64 GPU).

Workload (default): the 76-pose indoor loop through a 20 m x 20 m floor plan
with 6-10 rooms, 360 beams over 360 deg, range noise N(0, 0.02 m), odometry
noise 0.02 m / 0.01 rad, 100x100 SDF grid at 0.2 m, 6 hallucinated points per
beam: 191,520 point rows, ~5,000 Eikonal rows, 75 odometry rows, 10,225
unknowns. Seeded synthetic data (sdf-slam_b200/scenes.py) stands in for the
reference's datasets.

A step is one LM iteration (residuals and Jacobian, cell sort, J^T J and
-J^T r, supernodal LDL^T, triangular solves, step, cost). Each timed step is a
one-iteration solve call; an L2 flush (a write of 2x the 126 MB L2) runs
between steps outside the timed events. `value` is steps over the device time
of the steps (CUDA events on the library's stream, max over ranks); `e2e`
times complete solves through the public API from host buffers (problem
upload, iterations, state download).

Multi-GPU: replicas only. Every rank solves its own independent problem of
the same size (a different seed) on its own GPU; no data crosses GPUs; rank 0
reports the aggregate (weak scaling).

--impl reference times the CPU restatement of the reference's LM (oracle/) on
the host cores with all threads, on the same workload.
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


METRIC = "LM iters/s plain FP64 vs mixed+batched at equal final cost; served p50/p99 ms"
WORKLOADS = {
    "floorplan": "76-pose floor-plan loop, 100x100 grid @0.2 m, 360 beams, 6 hallucinated/beam",
    "room": "10-pose room loop, 40x40 grid @0.25 m, 180 beams, 4 hallucinated/beam",
    "office": "910-pose 3-lap office, 200x200 grid @0.15 m, 180 beams/180 deg, 6 hallucinated/beam",
}


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
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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


def _reduce_max(dist, value):
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _reduce_sum(dist, value):
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def make_scene(workload, seed):
    import sdf_slam_b200.scenes as scenes
    if workload == "floorplan":
        return scenes.floorplan_scene(seed=seed)
    if workload == "room":
        return scenes.room_scene(seed=seed)
    if workload == "office":
        return scenes.office_scene(seed=seed)
    raise ValueError(workload)


def scene_specs(P, scene):
    prob = P.Problem.from_scene(scene)
    return prob.specs(min_corner=scene.min_corner, max_corner=scene.max_corner)


def _oracle_problem(specs):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    s = O.Specs(**{k: getattr(specs, k) for k in O.Specs.__dataclass_fields__})
    return O.OracleProblem.from_specs(s)


def cpu_reference_rate(specs, iterations, threads):
    """The oracle's LM (CPU restatement of the reference) on the same problem:
    iterations/s with `threads` host threads."""
    orc = _oracle_problem(specs)
    t0 = time.perf_counter()
    res = orc.solve(max_iterations=iterations, step_tolerance=0.0, num_threads=threads)
    dt = time.perf_counter() - t0
    return res["iterations"] / dt, res, dt


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
    if rank != 0:
        return 0
    P = _load_package()
    scene = make_scene(args.workload, args.seed)
    specs = scene_specs(P, scene)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference_rate(specs, 1, threads)
    t0 = time.perf_counter()
    rate, res, dt = cpu_reference_rate(specs, args.steps, threads)
    wall = time.perf_counter() - t0
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "LM iters/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / max(1, res["iterations"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded floor plan, scenes.py)",
        "config": {"workload": WORKLOADS[args.workload], "seed": args.seed, "threads": threads},
        "cpu_baseline": {"value": rate, "unit": "LM iters/s", "cores": threads, "kind": "port",
                         "sample": f"{res['iterations']} LM iterations of the workload"},
        "e2e": {"value": rate, "unit": "LM iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch(P, args, flusher):
    """Uneven independent instances solved together in one engine (every
    kernel of an iteration covers all of them): aggregate LM iterations/s,
    plain FP64 and mixed, and the mixed instances' final-cost error against
    their FP64 solves after the same iterations."""
    import numpy as np
    import sdf_slam_b200.scenes as scenes
    scs = scenes.batch_scenes(seed=3, count=args.batch_count)
    specs = []
    for sc in scs:
        opts = P.ProblemOptions(hallucination_points=4, active_region=sc.options["active_region"])
        prob = P.Problem.from_scene(sc, opts)
        specs.append(prob.specs(min_corner=sc.min_corner, max_corner=sc.max_corner))
    count = len(specs)
    steps = max(3, min(20, args.steps // 5))
    out = {"instances": count, "unit": "LM iters/s (all instances)",
           "point_rows": sum(len(s.pt_frame) for s in specs),
           "workload": "uneven room-style instances, grid 40-150 @0.25 m, 10-200 poses, 90-360 beams, "
                       "every other one active-region", "steps": steps}
    final = {}
    for precision in ("fp64", "mixed"):
        batch = P.Problem.batch(specs)
        opts1 = [P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision=precision)] * count
        for _ in range(2):
            P.solve(batch, opts1)
        if not args.no_autotune:
            out.setdefault("schedule", {})[precision] = batch.autotune()["schedule"]
        device = 0.0
        for _ in range(steps):
            flusher.flush()
            P.solve(batch, opts1)
            device += batch.last_profile()["span"]
        final[precision] = np.array([batch.cost(i) for i in range(count)])
        out[precision] = {"value": count * steps / device, "ms_per_batched_iteration": 1000.0 * device / steps}
        batch.close()
    out["value"] = out["fp64"]["value"]
    out["mixed"]["max_final_cost_rel_err_vs_fp64"] = float(
        np.max(np.abs(final["mixed"] - final["fp64"]) / np.abs(final["fp64"])))
    return out


def run_mixed(P, args, specs, flusher):
    """The same workload with precision "mixed": LM iterations/s (one-iteration
    solves, L2 flushed between them) and, after 10 iterations from the same
    start, the final-cost and pose differences against the FP64 path."""
    import numpy as np
    prob = P.Problem.from_specs(specs)
    opts1 = P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision="mixed",
                            refine_steps=args.refine_steps)
    for _ in range(args.warmup):
        P.solve(prob, opts1)
    if not args.no_autotune:
        prob.autotune()
    steps = max(3, args.steps // 2)
    device = 0.0
    phases = np.zeros(5)
    for _ in range(steps):
        flusher.flush()
        P.solve(prob, opts1)
        prof = prob.last_profile()
        device += prof["span"]
        phases += [prof["assemble"], prof["normal"], prof["factor"], prof["solve"], prof["update"]]
    prob.close()
    res = {}
    for precision in ("fp64", "mixed"):
        p = P.Problem.from_specs(specs)
        r = P.solve(p, P.SolverOptions(max_iterations=10, step_tolerance=0.0, precision=precision,
                                       refine_steps=args.refine_steps))
        res[precision] = (r.final_cost, *p.state())
        p.close()
    names = ["assemble", "normal", "factor", "solve", "update"]
    return {"value": steps / device, "unit": "LM iters/s", "refine_steps": args.refine_steps,
            "phase_ms_per_step": {k: 1000.0 * v / steps for k, v in zip(names, phases)},
            "final_cost_rel_err_vs_fp64_10_iters": abs(res["mixed"][0] - res["fp64"][0]) / abs(res["fp64"][0]),
            "max_pose_err_m_vs_fp64_10_iters": float(np.max(np.abs(res["mixed"][2][:, :2] - res["fp64"][2][:, :2]))),
            "max_map_err_vs_fp64_10_iters": float(np.max(np.abs(res["mixed"][1] - res["fp64"][1])))}


def run_serve(P, args):
    """Poisson stream of solve requests through the serving loop: p50/p99
    latency and throughput of a warm server. Two untimed passes over other
    requests of the same distribution (other seeds) come first: the first
    requests of a process take their device and pinned blocks from the
    driver and load kernels, which measured 916 ms p50 on the first pass,
    692 ms on the second and 220 ms from the third on. The first pass's
    figures are reported as `cold_first_pass`."""
    cold = None
    for warm_seed in (1500, 2500):
        r = _serve_pass(P, args, warm_seed)
        cold = cold or {k: r[k] for k in ("p50_ms", "p99_ms", "throughput_req_s")}
    out = _serve_pass(P, args, 500)
    out["cold_first_pass"] = cold
    out["warmup_passes"] = 2
    return out


def _serve_pass(P, args, seed0):
    """One pass of args.serve_requests requests (scene seeds seed0, seed0+1,
    ...) with Poisson arrivals, on a fresh server."""
    import numpy as np
    import sdf_slam_b200.scenes as scenes
    rng = np.random.default_rng(7 if seed0 == 500 else seed0)
    reqs = []
    for i in range(args.serve_requests):
        sc = scenes.request_scene(seed=seed0 + i, iterations=args.serve_iterations)
        prob = P.Problem.from_scene(sc, P.ProblemOptions(hallucination_points=4))
        reqs.append(prob.specs(min_corner=sc.min_corner, max_corner=sc.max_corner))
    gaps = rng.exponential(1.0 / args.serve_rate, size=len(reqs))
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
    server.drain(600000)
    wall = time.perf_counter() - t0
    st = server.stats()
    ok = 0
    for spec, rid in zip(reqs, ids):
        res, _, _ = server.poll(rid)
        ok += int(res.status == 0)
    server.close()
    return {"requests": len(reqs), "completed_ok": ok, "rate_req_s": args.serve_rate,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "throughput_req_s": len(reqs) / wall,
            "lm_iters_s": st["iterations_per_s"], "iterations_per_request": args.serve_iterations,
            "workload": "room-style requests, grid log-U[40,200] @0.25 m, 10-400 poses, 180 beams"}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the
# factor-phase kernels (KFactorFront, KUpdate, KPanel, KExtendAdd,
# KInvertDiagonal) in one LM iteration, from one ncu capture of
# `profile_run.py floorplan 2` (default schedule); L2 is not flushed inside
# that capture, so writes that stay in L2 are not counted.
FACTOR_TRAFFIC_BYTES = {"floorplan": 126.3e6}


def run_gpu(args, dist, world, rank, local):
    import numpy as np
    P = _load_package()
    scene = make_scene(args.workload, args.seed + rank)
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
    device_s = 0.0
    launches = 0
    phases = np.zeros(5)
    for _ in range(args.steps):
        flusher.flush()
        P.solve(prob, opts1)
        prof = prob.last_profile()
        device_s += prof["span"]
        launches += prof["launches"]
        phases += [prof["assemble"], prof["normal"], prof["factor"], prof["solve"], prof["update"]]
    flusher.sync()
    _barrier(dist)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop() if sampler else None
    flops = prob.last_profile()["factor_flops"]
    device_max = _reduce_max(dist, device_s)
    wall_max = _reduce_max(dist, wall)
    total_steps = _reduce_sum(dist, args.steps)
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
    mixed = run_mixed(P, args, specs, flusher) if (world == 1 and not args.no_mixed) else None
    batched = run_batch(P, args, flusher) if (args.batch_count > 0 and world == 1) else None
    flusher.close()
    served = run_serve(P, args) if (args.serve_requests > 0 and world == 1) else None
    e2e_t = _reduce_max(dist, e2e_t)
    e2e_value = world * args.e2e_steps * e2e_iters / e2e_t if e2e_t > 0 else 0.0
    if rank != 0:
        return 0
    z = prob.sizes()
    per_step = phases / args.steps
    names = ["assemble", "normal", "factor", "solve", "update"]
    dominant = names[int(np.argmax(per_step))]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    fp64_peak = float(os.environ.get("SDFGPU_FP64_PEAK_TFLOPS", "37.0"))
    # algorithmic bytes of the assembly phase per iteration (row kernels + sort)
    P_rows = z["num_points"]
    assemble_bytes = P_rows * (40 + 64 + 4) + P_rows * 4 * 2 * 2 * 2
    roofline_factor = {
        "bound": "tensor", "achieved": flops / per_step[2] / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
        "frac": flops / per_step[2] / 1e12 / fp64_peak,
        "traffic": FACTOR_TRAFFIC_BYTES.get(args.workload),
        "kernel": "multifrontal LDL^T (KFactorFront + KPanel + KUpdate + KExtendAdd + KInvertDiagonal), FP64",
        "peak_source": "nominal B200 FP64 (no measured FP64 peak on this pool)"}
    roofline_assemble = {
        "bound": "hbm", "achieved": assemble_bytes / per_step[0] / 1e9, "peak": hbm, "unit": "GB/s",
        "frac": assemble_bytes / per_step[0] / 1e9 / hbm, "traffic": None,
        "kernel": "point rows + cell sort", "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)"}
    roofline = roofline_factor if dominant in ("factor",) else roofline_assemble
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, res, dt = cpu_reference_rate(specs, args.cpu_iterations, threads)
        cpu = {"value": rate, "unit": "LM iters/s", "cores": threads, "kind": "port",
               "sample": f"{res['iterations']} LM iterations of the same workload ({dt:.1f} s)"}
    line = {
        "metric": METRIC, "value": total_steps / device_max, "unit": "LM iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * device_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded floor plan, scenes.py)",
        "config": {"workload": WORKLOADS[args.workload], "seed": args.seed, "precision": args.precision,
                   "unknowns": z["num_parameters"], "point_rows": z["num_points"],
                   "l2": "flushed between steps (2x126 MB write)", "parallelism": f"replicas x{world}"},
        "wall_ms_per_step": 1000.0 * wall_max / args.steps,
        "phase_ms_per_step": {k: 1000.0 * v for k, v in zip(names, per_step)},
        "factor_gflop_per_step": flops / 1e9,
        "gpu_launches": int(launches),
        "roofline": roofline,
        "roofline_other": roofline_assemble if roofline is roofline_factor else roofline_factor,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "LM iters/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "iterations_per_step": e2e_iters},
        "clocks": clocks,
        "schedule": {"small_pivots": tune["schedule"][0], "front_rows": tune["schedule"][1],
                     "panel_rows": tune["schedule"][2], "factor_ms": tune["factor_ms"],
                     "trials": len(tune["trials"])} if tune else None,
        "mixed": mixed,
        "batched": batched,
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
    ap.add_argument("--workload", default="floorplan", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--e2e-iterations", type=int, default=10)
    ap.add_argument("--cpu-iterations", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--refine-steps", type=int, default=3)
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-rate", type=float, default=100.0)
    ap.add_argument("--serve-iterations", type=int, default=20)
    ap.add_argument("--serve-batch", type=int, default=16)
    ap.add_argument("--serve-budget-gb", type=float, default=32.0)
    args = ap.parse_args()
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
