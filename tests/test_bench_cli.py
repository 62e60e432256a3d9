"""The bench.py contract on the CPU: the reference arm's JSON line (one line
from rank 0 under torchrun, the other rank silent), the rank logic of the
replicated run (barrier, max over ranks) over gloo with two processes, and
no CPU fallback for the GPU arm."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _torchrun(args, nproc=2, port=29541, timeout=300):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", f"--master-port={port}"] + args
    env = dict(os.environ, OMP_NUM_THREADS="2")
    return subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout, env=env)


def test_reference_arm_two_ranks():
    r = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
                   "--ref-pixels", "256"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "1024^2 MRPNN frames/s" and d["unit"] == "frames/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


RANKS = r"""
import sys
sys.path.insert(0, ".")
import bench
rank, world, local = bench.dist_setup(2)
assert world == 2
bench.barrier(world)
m = bench.max_over_ranks(float(rank + 1) * 1.5, world)
assert m == 3.0, m
import torch.distributed as dist
dist.destroy_process_group()
sys.stdout.write(f"rank {rank} ok\n")   # one write: the ranks share the pipe
sys.stdout.flush()
"""


def test_max_over_ranks_gloo(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(RANKS)
    r = _torchrun([str(script)], port=29542, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert sorted(ln for ln in r.stdout.splitlines() if ln.endswith(" ok")) == ["rank 0 ok", "rank 1 ok"]


def test_gpu_arm_has_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    r = subprocess.run([sys.executable, "bench.py", "--steps", "1", "--warmup", "1"], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode != 0
    assert not any(ln.startswith("{") for ln in r.stdout.splitlines())
