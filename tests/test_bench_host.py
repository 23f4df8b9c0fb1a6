"""bench.py's multi-process host logic on the CPU: two gloo ranks (the GPU run uses NCCL with the
same calls). The replicas meet only at the barrier and the max over ranks of their timed region;
the reference arm runs on rank 0 alone and the other ranks exit without work."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import io, json, sys, contextlib
sys.path.insert(0, sys.argv[1])
import bench
rank, world, local = bench.dist_init(2, timeout_s=60)
bench.barrier(world)
m = bench.max_over_ranks(10.0 * (rank + 1) + 0.5, world)
out = io.StringIO()
if rank != 0:
    class A: gpus = 2; steps = 1; warmup = 0
    with contextlib.redirect_stdout(out):
        bench.run_reference(A, rank, world)
bench.barrier(world)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({"rank": rank, "world": world, "max": m, "reference_output": out.getvalue()}))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_max_and_only_rank0_runs_the_reference_arm():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    results = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        results.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(r["rank"] for r in results) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 20.5 for r in results)
    assert all(r["reference_output"] == "" for r in results)


def test_bench_launches_its_own_ranks_when_torchrun_did_not():
    """`python bench.py --gpus 2` with no torchrun environment starts two gloo ranks itself; the
    reference arm runs on rank 0 alone, whose line reports both ranks, and rank 1 prints nothing."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
                        "--raster", "128,64,10000,4", "--steps", "2", "--warmup", "1", "--inputs", "1"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["steps"] == 2 and line["warmup"] == 1
    assert "@128x64" in line["metric"] and line["value"] > 0
    assert abs(line["ms_per_step"] * line["steps"] / 1e3 - 2 / line["value"]) < 1e-9
