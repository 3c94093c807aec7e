"""bench.py's multi-rank path (torchrun, one image slab per rank, barrier and
max over ranks) run with two ranks on one GPU through gloo
(SARBP_BENCH_BACKEND=gloo): the ranks' kernels are independent (no
data-path collective), the ranks meet only in host-side gloo collectives, so
this exercises the path an 8-GPU run takes without a second GPU.  Rank 0
must print exactly one JSON line, for two GPUs' worth of slabs."""
import json
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bench_world_two_prints_one_line():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    env = dict(os.environ, SARBP_BENCH_BACKEND="gloo", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--gpus", "2", "--steps", "3", "--warmup", "3", "--config", "point_targets"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    line = lines[0]
    assert line["n_gpus"] == 2 and line["scaling"] == "weak"
    assert line["value"] > 0 and line["e2e"]["value"] > 0
    assert line["mixed_vs_fp64_gpu"]["rel_l2"] < 1e-4
    assert line["config"]["parallelism"].startswith("2 image slab")
