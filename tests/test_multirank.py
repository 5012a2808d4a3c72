"""Multi-process (N > 1) paths of bench.py on CPU: gloo process groups of two
ranks on 127.0.0.1. The GPU path shards nothing (replicas only), so what N > 1
adds is the barrier, the max-over-ranks timing reduction, the sum of steps,
per-rank problem seeds and rank-0-only output; these run here without a GPU.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench._init_dist(world)
    try:
        bench._barrier(dist)
        mx = bench._reduce(dist, 1.5 + rank, "MAX")
        sm = bench._reduce(dist, 10 * (rank + 1), "SUM")
        w, r, lr = bench._dist()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": mx, "sum": sm, "world": w, "rank": r, "local": lr}, f)
    finally:
        dist.destroy_process_group()


def test_replica_reductions_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r, g in enumerate(got):
        assert g["max"] == 2.5
        assert g["sum"] == 30.0
        assert (g["world"], g["rank"], g["local"]) == (2, r, r)


def test_replicas_solve_distinct_problems():
    # each rank solves its own problem of the same size (seed + rank)
    sys.path.insert(0, ROOT)
    import bench
    scenes = bench._load_scenes()
    a = bench.make_scene(scenes, "room", 1)
    b = bench.make_scene(scenes, "room", 2)
    assert (a.nx, a.ny, len(a.poses)) == (b.nx, b.ny, len(b.poses))
    assert any(pa.shape != pb.shape or (pa != pb).any() for pa, pb in zip(a.scans, b.scans))


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--workload", "room"]
    res = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_maps_no_library_of_the_package():
    """The reference arm builds its problem with the oracle's own Problem
    constructor and times the oracle's LM: the process maps the oracle's
    library and none of this package's."""
    code = (
        "import sys, json, types; sys.path.insert(0, %r); import bench;"
        "args = types.SimpleNamespace(workload='room', seed=None, steps=2, warmup=0, gpus=1, ref_budget_s=5.0);"
        "bench.run_reference(args, None, 0);"
        "maps = open('/proc/self/maps').read();"
        "print(json.dumps({'sdfgpu': 'libsdfgpu' in maps, 'oracle': 'liboracle' in maps}))" % ROOT)
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(ln) for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert lines[0]["impl"] == "reference" and lines[0]["value"] > 0
    assert lines[-1] == {"sdfgpu": False, "oracle": True}
