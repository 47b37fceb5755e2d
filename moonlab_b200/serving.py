"""Serving: the engine's continuous-batching request loop (mlb_server_*).

`Server.submit` queues a circuit and returns a ticket at once; the library's
worker threads admit requests as worker slots and HBM budget free up, so
requests that arrive while others run overlap with them on the device.
`run_load` replays a Poisson request stream (circuits.config_c5) against a
server in real time and reports throughput and latency percentiles.
`ControlFrontEnd` puts the reference control server's request frames
(HEALTH / CIRCUIT / SHOTS) onto the same loop.  `Mailbox` is the persistent
request loop for small circuits (mlb_mailbox_*): one long-running launch
serves posted requests without a launch per request.
"""
from __future__ import annotations

import ctypes as C
import threading
import time

import numpy as np

from . import _lib
from ._lib import check
from .circuits import GATE_DTYPE, brickwork

DTYPES = {"c128": _lib.MLB_C128, "c64": _lib.MLB_C64}


class MlbRequest(C.Structure):
    _fields_ = [("num_qubits", C.c_uint32), ("dtype", C.c_int32), ("gates", C.c_void_p),
                ("num_gates", C.c_size_t), ("num_shots", C.c_uint32), ("reserved", C.c_uint32),
                ("rng_seed", C.c_uint64)]


class MlbRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("num_qubits", C.c_uint32), ("dtype", C.c_int32),
                ("num_shots", C.c_uint32), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("done_s", C.c_double)]


class MlbServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "failed", "pending", "running",
                                          "peak_running", "reserved_bytes", "peak_reserved_bytes",
                                          "budget_bytes", "small_batches", "small_requests",
                                          "plan_cache_hits")]


class MlbMailboxConfig(C.Structure):
    _fields_ = [("dtype", C.c_int32), ("device", C.c_int32), ("ctas", C.c_int32), ("slots", C.c_uint32),
                ("max_ops", C.c_uint32), ("max_shots", C.c_uint32), ("idle_ms", C.c_double)]


class MlbMailboxStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "launches", "idle_exits", "running")]


_SIGS = {
    "mlb_mailbox_create": (C.c_int, [C.POINTER(MlbMailboxConfig), C.POINTER(C.c_void_p)]),
    "mlb_mailbox_submit": (C.c_int, [C.c_void_p, C.POINTER(MlbRequest), C.POINTER(C.c_uint64)]),
    "mlb_mailbox_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_uint64), C.c_size_t]),
    "mlb_mailbox_get_stats": (C.c_int, [C.c_void_p, C.POINTER(MlbMailboxStats)]),
    "mlb_mailbox_free": (C.c_int, [C.c_void_p]),
    "mlb_server_create": (C.c_int, [C.c_int, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]),
    "mlb_server_submit": (C.c_int, [C.c_void_p, C.POINTER(MlbRequest), C.POINTER(C.c_uint64)]),
    "mlb_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_uint64), C.c_size_t,
                                  C.POINTER(MlbRequestInfo)]),
    "mlb_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(MlbServerStats)]),
    "mlb_server_destroy": (None, [C.c_void_p]),
}


def _bind():
    lib = _lib.load()
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


class Server:
    """One GPU's request loop.  hbm_budget: bytes of device memory the
    server may hold in states (0 = 80 % of free memory); workers: requests
    in flight at once."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, workers: int = 8):
        self._lib = _bind()
        h = C.c_void_p()
        check(self._lib.mlb_server_create(device, hbm_budget, workers, C.byref(h)), "mlb_server_create")
        self._h = h
        self._shots = {}

    def submit(self, num_qubits: int, gates: np.ndarray, shots: int, seed: int, dtype: str = "c128") -> int:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        req = MlbRequest(num_qubits, DTYPES[dtype], g.ctypes.data, len(g), shots, 0, seed)
        t = C.c_uint64()
        check(self._lib.mlb_server_submit(self._h, C.byref(req), C.byref(t)), "mlb_server_submit")
        self._shots[t.value] = shots
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(outcomes uint64[shots], info dict); raises MlbError on failure."""
        shots = self._shots[ticket]
        out = np.empty(max(shots, 1), dtype=np.uint64)
        info = MlbRequestInfo()
        rc = self._lib.mlb_server_wait(self._h, ticket, timeout_ms,
                                       out.ctypes.data_as(C.POINTER(C.c_uint64)), len(out), C.byref(info))
        if rc == -7:
            raise TimeoutError(f"request {ticket} not done after {timeout_ms} ms")
        del self._shots[ticket]
        check(rc, "request")
        return out[:shots], {"status": info.status, "num_qubits": info.num_qubits, "dtype": info.dtype,
                             "shots": info.num_shots, "submit_s": info.submit_s, "admit_s": info.admit_s,
                             "done_s": info.done_s, "latency_s": info.done_s - info.submit_s}

    def stats(self) -> dict:
        s = MlbServerStats()
        check(self._lib.mlb_server_get_stats(self._h, C.byref(s)), "mlb_server_get_stats")
        return {k: int(getattr(s, k)) for k, _ in MlbServerStats._fields_}

    def close(self) -> None:
        if self._h:
            self._lib.mlb_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Mailbox:
    """The persistent request loop for small circuits (<= 12 qubits
    complex128, <= 13 complex64; one dtype per mailbox): `ctas` thread blocks
    of one long-running launch serve requests as they are posted.  The loop
    ends itself after idle_ms without work (a bounded wait; counted in
    stats()["idle_exits"]) and is relaunched by the next submit.  submit
    raises MlbError(MLB_ERR_BUSY) when every slot holds an unwaited ticket."""

    def __init__(self, dtype: str = "c128", device: int = 0, ctas: int = 0, slots: int = 0,
                 max_ops: int = 0, max_shots: int = 0, idle_ms: float = 0.0):
        self._lib = _bind()
        cfg = MlbMailboxConfig(DTYPES[dtype], device, ctas, slots, max_ops, max_shots, idle_ms)
        h = C.c_void_p()
        check(self._lib.mlb_mailbox_create(C.byref(cfg), C.byref(h)), "mlb_mailbox_create")
        self._h, self._dtype = h, DTYPES[dtype]
        self._shots = {}

    def submit(self, num_qubits: int, gates: np.ndarray, shots: int, seed: int) -> int:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        req = MlbRequest(num_qubits, self._dtype, g.ctypes.data, len(g), shots, 0, seed)
        t = C.c_uint64()
        check(self._lib.mlb_mailbox_submit(self._h, C.byref(req), C.byref(t)), "mlb_mailbox_submit")
        self._shots[t.value] = shots
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> np.ndarray:
        """Outcomes uint64[shots]; TimeoutError if not done in time (the
        ticket stays valid)."""
        shots = self._shots[ticket]
        out = np.empty(max(shots, 1), dtype=np.uint64)
        rc = self._lib.mlb_mailbox_wait(self._h, ticket, timeout_ms, out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                        len(out))
        if rc == -7:
            raise TimeoutError(f"request {ticket} not done after {timeout_ms} ms")
        check(rc, "mlb_mailbox_wait")
        del self._shots[ticket]
        return out[:shots]

    def stats(self) -> dict:
        s = MlbMailboxStats()
        check(self._lib.mlb_mailbox_get_stats(self._h, C.byref(s)), "mlb_mailbox_get_stats")
        return {k: int(getattr(s, k)) for k, _ in MlbMailboxStats._fields_}

    def close(self) -> None:
        if self._h:
            rc = self._lib.mlb_mailbox_free(self._h)
            self._h = None
            check(rc, "mlb_mailbox_free")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_mailbox_load(mb: "Mailbox", requests, time_scale: float = 1.0, circuits=None):
    """run_load for the persistent loop: submit at the arrival times from one
    thread, collect in order in another.  A request's latency is submit to
    the return of its wait on the host clock.  A submit refused because every
    slot holds a ticket is retried after 50 us."""
    circuits = circuits if circuits is not None else [request_circuit(r) for r in requests]
    tickets = [None] * len(requests)
    t_sub = [0.0] * len(requests)
    ready = [threading.Event() for _ in requests]
    errors = []

    def producer():
        t0 = time.perf_counter()
        for i, r in enumerate(requests):
            delay = r.arrival * time_scale - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            while True:
                try:
                    t_sub[i] = time.perf_counter()
                    tickets[i] = mb.submit(r.n, circuits[i], r.shots, r.seed)
                    break
                except _lib.MlbError as e:
                    if e.status != -8:  # MLB_ERR_BUSY: retry
                        errors.append((i, e))
                        break
                    time.sleep(50e-6)
            ready[i].set()

    t_done = [0.0] * len(requests)
    th = threading.Thread(target=producer)
    th.start()
    for i in range(len(requests)):
        ready[i].wait()
        if tickets[i] is not None:
            mb.wait(tickets[i])
            t_done[i] = time.perf_counter()
    th.join()
    if errors:
        raise RuntimeError(f"{len(errors)} submissions failed; first: {errors[0]}")
    lat = np.array([d - s for s, d in zip(t_sub, t_done)])
    span = max(t_done) - min(t_sub)
    return {"circuits_per_s": len(requests) / span, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "span_s": span,
            "stats": mb.stats()}


class ControlFrontEnd:
    """The control server's request execution on the device loop
    (mlb_control_*): `handle(frame)` takes one request frame of the
    reference's wire protocol (src/control/control_plane.h:8-33: HEALTH,
    CIRCUIT <N>, SHOTS <k> <N> with a "moonlab-circuit v1" body) and returns
    its response frame (OK / SAMPLES / ERR).  SHOTS requests share one
    continuous-batching server; `set_seed` fixes the shot seed (default: the
    clock, as the reference's server)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, workers: int = 8, max_qubits: int = 0):
        self._lib = _lib.load()
        self._h = C.c_void_p()
        check(self._lib.mlb_control_create(device, budget_bytes, workers, max_qubits, C.byref(self._h)),
              "mlb_control_create")

    def set_seed(self, seed: int) -> None:
        check(self._lib.mlb_control_set_seed(self._h, seed), "mlb_control_set_seed")

    def handle(self, frame: bytes) -> bytes:
        out, n = C.c_void_p(), C.c_size_t()
        check(self._lib.mlb_control_handle(self._h, frame, len(frame), C.byref(out), C.byref(n)),
              "mlb_control_handle")
        try:
            return C.string_at(out, n.value)
        finally:
            self._lib.mlb_control_free(out)

    def close(self) -> None:
        if self._h:
            self._lib.mlb_control_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def request_circuit(r) -> np.ndarray:
    """The circuit of a config_c5 request: brickwork of its width and depth."""
    return brickwork(r.n, r.depth, r.seed)


def run_load(server: Server, requests, time_scale: float = 1.0, circuits=None):
    """Submit requests at their Poisson arrival times (scaled by time_scale)
    from one thread while another collects results.  Returns a summary with
    circuits/s, p50/p99 latency, and per-request (latency, outcomes)."""
    circuits = circuits if circuits is not None else [request_circuit(r) for r in requests]
    tickets = [None] * len(requests)
    ready = [threading.Event() for _ in requests]
    errors = []

    def producer():
        t0 = time.perf_counter()
        for i, r in enumerate(requests):
            delay = r.arrival * time_scale - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            try:
                tickets[i] = server.submit(r.n, circuits[i], r.shots, r.seed, "c64" if r.dtype else "c128")
            except Exception as e:  # reported below
                errors.append((i, e))
            ready[i].set()

    results = [None] * len(requests)
    th = threading.Thread(target=producer)
    th.start()
    for i in range(len(requests)):
        ready[i].wait()
        if tickets[i] is not None:
            results[i] = server.wait(tickets[i])
    th.join()
    if errors:
        raise RuntimeError(f"{len(errors)} submissions failed; first: {errors[0]}")
    lat = np.array([info["latency_s"] for _, info in results])
    first = min(info["submit_s"] for _, info in results)
    last = max(info["done_s"] for _, info in results)
    return {"circuits_per_s": len(results) / (last - first), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "span_s": last - first,
            "results": results, "stats": server.stats()}
