"""Multi-GPU runs are replicas: each rank runs its own step, and the job
reports units of all ranks over the slowest rank's time.  These CPU tests
run the same code with two gloo ranks: the max-over-ranks reduction, the
barrier, the whole-job rate, and bench.py's reference arm under torchrun
(rank 0 alone measures and prints; the other rank exits cleanly)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

from oracle import bindings as B

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    from moonlab_b200 import replicas
    w, r, _ = replicas.init("gloo", timeout_s=60)
    m = replicas.max_over_ranks(1.5 + r, w)
    replicas.barrier(w)
    v = replicas.job_throughput(1.0, w, m)
    replicas.done(w)
    q.put((r, w, m, v))


def test_two_gloo_ranks_reduce_and_rate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    for _, w, m, v in res:
        assert w == 2 and m == 2.5 and abs(v - 2 / 2.5) < 1e-15


@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--qubits", "14", "--depth", "4", "--ref-budget", "0.2"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 only
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
