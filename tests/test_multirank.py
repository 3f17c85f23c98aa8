"""Host logic of multi-GPU runs, as two gloo ranks on the CPU.

bench.py gives each rank its own replica of the workload (no exchange step
on one domain) and reports the time as the max over ranks; the reference arm
runs on rank 0 only.  Here the same helpers run under world size 2."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import torch
import bench
world, rank, local = bench.dist_setup()
dev = torch.device("cpu")
bench.barrier(world, dev)
m = bench.max_over_ranks(float(10 + rank), world, dev)
out = dict(rank=rank, world=world, max=m)
import torch.distributed as dist
dist.barrier()
dist.destroy_process_group()
print(json.dumps(out))
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def run_ranks(code, world=2, extra_env=None, timeout=120):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), MPLB_BENCH_BACKEND="gloo", CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_max_over_ranks_gloo():
    import json
    outs = run_ranks(WORKER.format(root=ROOT))
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 11.0 for r in res)


def test_reference_arm_prints_on_rank0_only():
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); sys.argv=['bench.py','--impl','reference','--gpus','2',"
            "'--cpu-steps','2','--cpu-procs','1','--warmup','3']; import bench; bench.main()")
    outs = run_ranks(code)
    printed = [o for o in outs if o.strip()]
    assert len(printed) == 1 and '"impl": "reference"' in printed[0]


def test_reference_arm_ranks_mode():
    """--ref-mode ranks: the reference's own multi-rank step on host threads
    prints one line on the arm's metric, unit and config."""
    import json
    import subprocess
    import sys
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--ref-mode", "ranks",
                        "--cpu-procs", "3", "--steps", "2", "--warmup", "3"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "GLUPS" and line["value"] > 0
    assert line["cpu_baseline"]["cores"] == 3 and "3 reference ranks" in line["config"]["parallelism"]
