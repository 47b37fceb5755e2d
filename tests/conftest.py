"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on a
CPU-only machine."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _ensure_built():
    lib = ROOT / "moonlab_b200" / "libmoonlab_b200.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(ROOT / "moonlab_b200" / "csrc"), "-j8"], check=True,
                       stdout=subprocess.DEVNULL)
    port = ROOT / "oracle" / "libsv_oracle.so"
    if not port.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "port"], check=True, stdout=subprocess.DEVNULL)


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN, allow_pickle=False)


def corpus_case(g, k):
    """(n, gates, amplitudes) of corpus circuit k from the golden fixture."""
    n = int(g["corpus_n"][k])
    go = g["corpus_gate_offsets"]
    ao = g["corpus_amp_offsets"]
    return n, g["corpus_gates"][go[k]:go[k + 1]], g["corpus_amps"][ao[k]:ao[k + 1]]


@pytest.fixture(scope="session")
def gpu():
    """Fail loudly (not skip) when a GPU test runs without a usable device."""
    from moonlab_b200 import _lib
    import ctypes as C
    lib = _lib.load()
    cnt = C.c_int()
    rc = lib.mlb_device_count(C.byref(cnt))
    assert rc == 0 and cnt.value > 0, "GPU test run without a CUDA device"
    return lib
