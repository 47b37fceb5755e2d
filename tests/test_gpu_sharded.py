"""Sharded states on the device: every shard an engine state (tile passes on
the GPU), the whole state split over 2^g shards held by one process on one
GPU, half-shards exchanged in bounded chunks by device-to-device copies
(moonlab_b200.sharded.LocalShards).  Checked against the whole state run by
the engine (1e-12 per amplitude) and, at the smallest size, by the oracle.

The torch.distributed path (ShardedState: one shard per rank, NCCL send/recv
through the same bounded staging) runs here with one rank (g = 0), which
exercises the engine executor under a real NCCL group; its exchanges are
tested with gloo ranks on the CPU (tests/test_sharded.py)."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from moonlab_b200 import StateVector
from moonlab_b200 import sharded as S
from moonlab_b200.circuits import brickwork, qaoa_circuit
from oracle import bindings as B
from test_tile_plan import random_gates

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
TOL = 1e-12

CIRCUITS = {
    "brickwork": lambda n: brickwork(n, 12, 0x6A, zz_every=3),
    "qaoa": lambda n: qaoa_circuit(n, 2, 0x6B),
    "random": lambda n: random_gates(n, 400, 0x6C + n),
}


@pytest.mark.parametrize("n,g,name,chunk", [(12, 1, "brickwork", 1 << 6), (16, 1, "random", 1 << 20),
                                            (16, 2, "qaoa", 1 << 9), (18, 2, "random", 1 << 11),
                                            (20, 3, "brickwork", 1 << 14)])
def test_engine_shards_match_the_whole_state(gpu, n, g, name, chunk):
    gates = CIRCUITS[name](n)
    exs = [S.EngineExecutor(n - g, 0) for _ in range(1 << g)]
    try:
        st = S.LocalShards(n, exs, chunk=chunk)
        half = len(gates) // 2
        st.run(gates[:half])  # the second call starts from a permuted layout
        st.run(gates[half:])
        got = st.gather()
        exchanges = st.exchanges
        staged = st.staging.send.numel()
    finally:
        for e in exs:
            e.close()
    with StateVector(n) as sv:
        sv.run(gates)
        want = sv.amplitudes()
    assert np.abs(got - want).max() < TOL
    assert exchanges > 0
    assert staged == min(chunk, 1 << (n - g - 1))  # the only extra device memory of an exchange
    if n <= 12:
        assert np.abs(got - B.port_run(n, gates)).max() < TOL


_ONE_RANK = r"""
import datetime, os, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import torch, torch.distributed as dist
from moonlab_b200 import StateVector, sharded as S
from moonlab_b200.circuits import brickwork
torch.cuda.set_device(0)
dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
try:
    n = 14
    gates = brickwork(n, 8, 0x6D, zz_every=4)
    ex = S.EngineExecutor(n, 0)
    st = S.ShardedState(n, ex)
    st.run(gates)
    got = st.gather()
    ex.close()
    with StateVector(n) as sv:
        sv.run(gates)
        want = sv.amplitudes()
    err = float(np.abs(got - want).max())
    print("ERR", err)
    assert err < 1e-12
finally:
    dist.destroy_process_group()
"""


def test_nccl_group_of_one_rank(gpu):
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(29700 + os.getpid() % 200), RANK="0",
               WORLD_SIZE="1", NCCL_NVLS_ENABLE="0")
    code = _ONE_RANK.format(root=str(ROOT), tests=str(ROOT / "tests"))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ERR" in r.stdout
