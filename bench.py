#!/usr/bin/env python3
"""Benchmark: the 30-qubit depth-40 random circuit (brickwork RX/RY/RZ +
CNOT, a ZZ layer every 4 layers) on the B200 engine.

One step = prepare |0...0> and run the whole 4470-gate circuit (4180 one-
and two-qubit gates + 290 ZZ) on a complex128 state (16 GiB), the plain
drop-in path; the same circuit on a complex64 state (8 GiB) is reported
beside it.  `value` is circuits/s over all ranks, device-timed with CUDA
events on the engine's stream; `e2e` is the same metric through the public
C ABI from host gate records to host results (<Z_i> for every qubit and
1024 sampled outcomes read back) each step.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref/liboracle.so, built from its sources; all host threads) on a
bounded, stratified sample of the same circuit and extrapolates per gate.

Multi-GPU: one process per GPU (torchrun); each rank runs its own circuit
replica (the workload does not shard below 34 qubits), timing is the max
over ranks, and value = circuits of all ranks / that time ("weak").
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "30q circuit time & HBM GB/s (fused c64 vs plain c128); circuits/s, p99 at load"
def workload(n: int, depth: int, gates: int) -> str:
    """The circuit workload's name ("30q depth-40 ... (4470 gates)" by default)."""
    return f"{n}q depth-{depth} brickwork RX/RY/RZ+CNOT, ZZ(theta) layer every 4 layers ({gates} gates)"


def l2_note(n: int) -> str:
    """Whether a complex128 state of n qubits is larger than the 126 MB L2."""
    size = 16 << n
    human = f"{size >> 30} GiB" if size >= 1 << 30 else f"{size >> 20} MiB"
    return f"state ({human}) {'larger than' if size > 126 * 10**6 else 'fits in'} L2"


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# FP64 tensor-core (mma.sync m8n8k4 f64) peak: measured live on the bench's
# GPU by mlb_fp64_tensor_peak (register-only probe, 8 accumulator chains per
# warp as the dense segments run them); this earlier measurement on the same
# kind of GPU (63.5 multiply-adds per clock per SM x 148 SMs x 2 x 1.965 GHz)
# stands in only if the probe fails.
DMMA_PEAK_TFLOPS = 36.9


def fp64_tensor_peak(local: int):
    from moonlab_b200 import _lib
    v = C.c_double()
    if _lib.load().mlb_fp64_tensor_peak(local, C.byref(v)) == 0 and v.value > 0:
        return v.value, "measured live (mlb_fp64_tensor_peak)"
    return DMMA_PEAK_TFLOPS, "earlier measurement (probe failed)"


def profiled_traffic(n: int):
    """DRAM bytes of one k_tile<double> pass at n qubits: the ncu figure of
    bytes per amplitude (profiles/k_tile_c128_traffic.json: dram read + write
    of a 26-qubit pass, the capture command inside the file) times 2^n.  A
    pass moves every amplitude once each way, so its traffic grows in
    proportion to 2^n.  None if the file is gone."""
    p = ROOT / "profiles" / "k_tile_c128_traffic.json"
    if not p.exists():
        return None
    return float(json.loads(p.read_text())["dram_bytes_per_amplitude_per_pass"]) * (1 << n)


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference CPU path: per-gate samples of the circuit, every target covered
# ---------------------------------------------------------------------------
class ReferenceSampler:
    """Times the reference library's gate_* calls at n qubits and
    extrapolates the whole circuit from the circuit's own histogram of
    (gate type, target) pairs: RX / RY / RZ at every target 0..n-1 and
    CNOT(q, q+1) at every q (ZZ = CNOT.RZ.CNOT, qaoa.c:745-753).  The
    reference threads a gate only when the state has >= 2^18 amplitudes and
    >= 32 blocks above the target (gates.c:121, 137-140), so per-target times
    differ and every target is sampled: each step times the next pairs of a
    fixed rotation until its time budget is spent, and a pair's time is the
    mean of all its samples so far (a pair not yet sampled takes its gate
    type's mean)."""

    def __init__(self, n: int, gates):
        cores = os.cpu_count() or 1
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
        self.cores = int(os.environ.get("OMP_NUM_THREADS", cores))
        from oracle import bindings as B
        if not B.have_ref():
            raise RuntimeError("reference library oracle/_ref/liboracle.so not built")
        self.kind = "reference"
        self.r = B.RefStateVector(n)
        L, p = self.r.lib, C.byref(self.r.s)
        self.n = n
        self.call = {"rx": lambda q: L.gate_rx(p, q, 0.3), "ry": lambda q: L.gate_ry(p, q, 0.4),
                     "rz": lambda q: L.gate_rz(p, q, 0.5), "cnot": lambda q: L.gate_cnot(p, q, q + 1)}
        # the circuit's (type, target) histogram; CNOT keyed by its control q (target q + 1)
        self.count = {}
        for g in gates:
            t, tgt, ctl = int(g["type"]), int(g["target"]), int(g["control"])
            keys = {7: [("rx", tgt)], 8: [("ry", tgt)], 9: [("rz", tgt)], 10: [("cnot", ctl)],
                    27: [("cnot", ctl), ("rz", tgt), ("cnot", ctl)]}[t]
            for k in keys:
                self.count[k] = self.count.get(k, 0) + 1
        # targets in bit-reversed order, so every prefix of the rotation spreads
        # over low, middle and high targets (and the threaded / serial regimes)
        nb = max(1, (n - 1).bit_length())
        spread = sorted(range(n), key=lambda q: int(format(q, f"0{nb}b")[::-1], 2))
        self.pairs = [(k, q) for q in spread for k in ("rx", "ry", "rz", "cnot") if k != "cnot" or q < n - 1]
        self.samples = {}
        self.next = 0
        self.calls = 0

    def step(self, budget_s: float) -> float:
        t_start = time.perf_counter()
        done = 0
        while done < 4 or time.perf_counter() - t_start < budget_s:
            k, q = self.pairs[self.next % len(self.pairs)]
            self.next += 1
            t0 = time.perf_counter()
            self.call[k](q)
            self.samples.setdefault((k, q), []).append(time.perf_counter() - t0)
            done += 1
        self.calls += done
        by_kind = {}
        for (k, _), v in self.samples.items():
            by_kind.setdefault(k, []).extend(v)
        kind_mean = {k: sum(v) / len(v) for k, v in by_kind.items()}
        total = 0.0
        for (k, q), c in self.count.items():
            v = self.samples.get((k, q))
            total += c * (sum(v) / len(v) if v else kind_mean.get(k, max(kind_mean.values())))
        return total

    def describe(self) -> str:
        covered = sum(1 for pq in self.pairs if pq in self.samples)
        return (f"{self.calls} gate_* calls at {self.n} qubits so far, rotating over all {len(self.pairs)} "
                f"(type, target) pairs of the circuit (RX/RY/RZ at every target, CNOT(q, q+1) at every q; "
                f"{covered} covered); circuit time = sum over the circuit's {sum(self.count.values())} "
                f"gate calls (ZZ = CNOT.RZ.CNOT) of its pair's mean time")

    def close(self):
        self.r.close()


def reference_sample(n: int, budget_s: float, gates, rounds: int = 1):
    """Circuit seconds from `rounds` sampler steps (the CPU baseline of the
    B200 line); returns (seconds, sample, cores, kind)."""
    smp = ReferenceSampler(n, gates)
    try:
        for _ in range(rounds):
            secs = smp.step(budget_s)
        return secs, smp.describe(), smp.cores, smp.kind
    finally:
        smp.close()


# ---------------------------------------------------------------------------
# replicas over several GPUs (moonlab_b200.replicas)
# ---------------------------------------------------------------------------
def dist_init():
    from moonlab_b200 import replicas
    return replicas.init()


def dist_max(x: float, ws: int) -> float:
    from moonlab_b200 import replicas
    return replicas.max_over_ranks(x, ws)


def dist_barrier(ws: int):
    from moonlab_b200 import replicas
    replicas.barrier(ws)


def dist_done(ws: int):
    from moonlab_b200 import replicas
    replicas.done(ws)


# ---------------------------------------------------------------------------
def run_reference(args, ws, rank):
    from moonlab_b200.circuits import config_c2
    if rank != 0:
        return
    gates, _ = config_c2(args.qubits, args.depth)
    smp = ReferenceSampler(args.qubits, gates)
    step_vals = []
    for i in range(args.warmup + args.steps):
        secs = smp.step(args.ref_budget)
        if i >= args.warmup:
            step_vals.append(secs)
    sample, cores, kind = smp.describe(), smp.cores, smp.kind
    smp.close()
    secs = statistics.median(step_vals)
    val = 1.0 / secs
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "circuits/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic seeded circuit (splitmix64 0xC2)",
            "config": {"workload": workload(args.qubits, args.depth, int(len(gates))),
                       "qubits": args.qubits, "depth": args.depth},
            "cpu_baseline": {"value": val, "unit": "circuits/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": val, "unit": "circuits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args, ws, rank, local):
    import torch
    from moonlab_b200 import replicas
    from moonlab_b200 import StateVector, _lib, kernel_launches
    from moonlab_b200.circuits import config_c2

    torch.cuda.set_device(local)
    gates, shots = config_c2(args.qubits, args.depth)
    n = args.qubits
    sv = StateVector(n, "c128", device=local)
    sv.set_timing(True)
    stream = torch.cuda.ExternalStream(sv.stream(), device=torch.device("cuda", local))

    def step():
        sv.reset()
        sv.run(gates)
        sv.flush()

    dmma_peak, dmma_src = fp64_tensor_peak(local)

    # warm-up
    for _ in range(args.warmup):
        step()
        sv.synchronize()
    dist_barrier(ws)
    torch.cuda.synchronize()
    launches0 = kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_gbs = []  # HBM bytes the step's launches moved / the step's device time
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
            st = sv.flush_stats()  # waits for this step's kernels (device events)
            step_gbs.append(st["bytes_moved"] / max(1e-9, st["gpu_ms"] / 1e3) / 1e9)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    dist_barrier(ws)
    launches = kernel_launches() - launches0
    t = ev0.elapsed_time(ev1) / 1e3 / args.steps
    t_max = dist_max(t, ws)
    st = sv.flush_stats()
    passes = int(st["passes"])
    dense_segments = int(st["dense_blocks"])
    per_pass_bytes = 2 * 16 * (1 << n)
    # After the reset that starts every step, the first passes run only over
    # the tiles that can be nonzero; the engine counts the bytes its launches
    # moved, and the roofline is taken over those bytes.
    moved = int(st["bytes_moved"])
    peak, peak_kind = measured_peaks()
    achieved = statistics.median(step_gbs)
    # the dense segments' FP64 tensor-core work: a 16x16 complex matrix on
    # every 16 amplitudes as three real 16x16 products (Gauss) = 48 real
    # multiply-adds (96 flops) per amplitude
    dense_flops = 96.0 * int(st["dense_amps"])  # over the tiles the launches ran over

    # the same c128 path with dense segments off: every register segment runs
    # gate by gate on the CUDA cores (no gate matrices multiplied together
    # beyond runs of 1-qubit gates on one qubit)
    sv.set_dense(False)
    gbg = []
    for i in range(1 + max(1, min(args.steps, 2))):
        step()
        st_g = sv.flush_stats()
        if i > 0:
            gbg.append(st_g["gpu_ms"] / 1e3)
    sv.set_dense(True)
    gbg_s = statistics.median(gbg)

    # end to end through the C ABI: host gate records in, <Z_i> + 1024 shots out
    e2e_t = []
    for i in range(max(2, min(args.steps, 3)) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sv.reset()
        sv.run(gates)
        ez = sv.expectation_z_all()
        outs = sv.sample(shots)
        t1 = time.perf_counter()
        if i > 0:
            e2e_t.append(t1 - t0)
    e2e_s = dist_max(statistics.median(e2e_t), ws)
    h2d = gates.nbytes + shots.nbytes
    d2h = ez.nbytes + outs.nbytes

    # complex64 on the same circuit (plain tile passes, and the fused
    # tensor-core path), each against the complex128 result
    sv.reset()
    sv.run(gates)
    sv.synchronize()
    ref128 = torch.as_tensor(_DeviceView(sv.device_ptr(), 1 << n, "<c16"), device=f"cuda:{local}")

    def c64_leg(mode):
        s64 = StateVector(n, "c64", device=local)
        s64.set_exec_mode(mode)
        s64.set_timing(True)
        t64, st64 = [], None
        for i in range(args.warmup + max(1, min(args.steps, 3))):
            s64.reset()
            s64.run(gates)
            s64.flush()
            st64 = s64.flush_stats()
            if i >= args.warmup:
                t64.append(st64["gpu_ms"] / 1e3)
        b = torch.as_tensor(_DeviceView(s64.device_ptr(), 1 << n, "<c8"), device=f"cuda:{local}")
        ip = torch.zeros((), dtype=torch.complex128, device=f"cuda:{local}")
        nb, maxerr = 0.0, 0.0
        chunk = 1 << 26
        for off in range(0, 1 << n, chunk):
            bb = b[off:off + chunk].to(torch.complex128)
            aa = ref128[off:off + chunk]
            ip += torch.vdot(aa, bb)
            nb += float(torch.vdot(bb, bb).real.item())
            maxerr = max(maxerr, float((aa - bb).abs().max().item()))
        s64.close()
        secs = statistics.median(t64)
        gbs = st64["bytes_moved"] / secs / 1e9  # the bytes the launches moved (all-zero tiles skipped)
        return {"circuit_ms": secs * 1e3, "speedup_vs_c128": t_max / secs,
                "speedup_vs_c128_gate_by_gate": gbg_s / secs,
                "fidelity": float(ip.abs().item() ** 2) / nb, "norm": nb, "max_amp_err": maxerr,
                "passes": int(st64["passes"]), "dense_blocks": int(st64["dense_blocks"]),
                "hbm_gbs_per_pass": gbs, "hbm_frac": gbs / peak}

    c64 = c64_leg("tiled")
    c64["path"] = "c64 tiled (CUDA cores)"
    fused = c64_leg("fused")
    fused["path"] = ("c64 fused: <=5-qubit dense blocks on tcgen05 tensor cores, split-bf16 products, "
                     "FP32 accumulation; fidelity = |<psi128|psi64>|^2 / <psi64|psi64>")
    fused["kernel"] = "k_fused"

    sv.close()
    # the serving, per-gate and VQE legs describe one GPU: run at N = 1 only
    one = ws == 1
    serving = None if args.no_serving or not one else serving_leg(args, local, not args.no_cpu_baseline)
    sweep = None if args.no_sweep or not one else gate_sweep_leg(local, peak)
    vqe = None if args.no_vqe or not one else vqe_leg(local, not args.no_cpu_baseline)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            secs, sample, cores, kind = reference_sample(n, args.ref_budget, gates)
            cpu = {"value": 1.0 / secs, "unit": "circuits/s", "cores": cores, "kind": kind, "sample": sample}
        except Exception as e:  # reported, never silently replaced
            cpu = {"value": None, "unit": "circuits/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": replicas.job_throughput(1.0, ws, t_max), "unit": "circuits/s",
            "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic seeded circuit (splitmix64 0xC2)",
            "config": {"workload": workload(n, args.depth, int(len(gates))), "qubits": n, "depth": args.depth,
                       "path": "plain c128 tiled", "parallelism": f"replicas x{ws}", "l2": l2_note(n),
                       "tile_passes_per_circuit": passes, "gates": int(len(gates))},
            "hbm_gbs_per_pass": achieved,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic(n),
                         "kernel": "k_tile<double>", "peak_source": peak_kind,
                         "algorithmic_bytes_per_pass": per_pass_bytes,
                         "bytes_moved_per_circuit": moved,
                         "all_zero_tile_bytes_skipped": passes * per_pass_bytes - moved},
            # what bounds the c128 pass now: the FP64 tensor pipe (mma.sync f64)
            # running the dense segments; peak measured live (fp64_tensor_peak)
            "fp64_tensor": {"dense_segments": dense_segments, "segments": int(st["segments"]),
                            "flops_per_circuit": dense_flops,
                            "achieved_tflops": dense_flops / t_max / 1e12,
                            "peak_tflops": dmma_peak, "peak_source": dmma_src,
                            "frac_of_circuit_time": dense_flops / t_max / 1e12 / dmma_peak},
            "c128_gate_by_gate": {"circuit_ms": gbg_s * 1e3, "passes": int(st_g["passes"]),
                                  "path": "c128 tile passes, dense segments off"},
            "c64": c64,
            "fused_c64": fused,
            "e2e": {"value": replicas.job_throughput(1.0, ws, e2e_s), "unit": "circuits/s",
                    "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        if serving is not None:
            line["serving"] = serving
        if sweep is not None:
            line["gate_sweep"] = sweep
        if vqe is not None:
            line["vqe_gradient"] = vqe
        print(json.dumps(line), flush=True)


def serving_leg(args, local, with_cpu: bool):
    """The request stream of the serving workload (Poisson arrivals; qubits
    U{10..28}, depth U{10..100}, shots U{1..4096}, dtype 50/50), all
    --serve-requests of it (10,000 by default) paced at --serve-rate through
    the continuous-batching server on this rank's GPU: circuits/s and p50/p99
    latency at that load.  Beside it: the capacity (the first
    --serve-capacity requests submitted at once) and a short arrival-rate
    sweep (100 requests per rate) with the highest rate whose p99 meets the
    stated target.  Latency = submit to result on the host clock; circuits/s
    = requests / (last result - first submit).  With with_cpu, the
    reference's moonlab_qgtl_execute (the control server's per-request path,
    control_plane.c:688-716) is timed on the host on up to 12 requests of <=
    16 qubits beside the engine's time for the same requests run one at a
    time."""
    from moonlab_b200.circuits import config_c5
    from moonlab_b200.serving import Server, request_circuit, run_load
    reqs = config_c5(num=args.serve_requests, rate=args.serve_rate)
    circ = [request_circuit(r) for r in reqs]
    workers = 8
    p99_target_ms = 2000.0
    sweep = []
    ncap = min(args.serve_capacity, len(reqs))
    with Server(device=local, workers=workers) as srv:
        sat = run_load(srv, reqs[:ncap], time_scale=0.0, circuits=circ[:ncap])
        paced = run_load(srv, reqs, time_scale=1.0, circuits=circ)
        # arrival-rate sweep: 100 requests of the stream re-timed at each rate
        for lam in (10.0, 20.0, 30.0, 40.0):
            sub = config_c5(num=100, rate=lam, seed=0xC5)
            sr = run_load(srv, sub, time_scale=1.0)
            sweep.append({"rate_per_s": lam, "circuits_per_s": sr["circuits_per_s"], "p50_ms": sr["p50_s"] * 1e3,
                          "p99_ms": sr["p99_s"] * 1e3})
        # per-request service time of small requests alone (for the CPU comparison)
        small = [i for i, r in enumerate(reqs) if r.n <= 16][:12]
        gpu_alone = []
        for i in small:
            r = reqs[i]
            _, info = srv.wait(srv.submit(r.n, circ[i], r.shots, r.seed, "c64" if r.dtype else "c128"))
            gpu_alone.append(info["done_s"] - info["submit_s"])
    meets = [x["rate_per_s"] for x in sweep if x["p99_ms"] <= p99_target_ms]
    small_leg = small_requests_leg(local)
    cpu = None
    if with_cpu:
        try:  # the reference's moonlab_qgtl_execute on the same small requests (all host threads)
            from oracle import bindings as B
            t_cpu = []
            for i in small:
                r = reqs[i]
                t0 = time.perf_counter()
                B.ref_qgtl_execute(r.n, circ[i], r.shots, r.seed, want_probs=False)
                t_cpu.append(time.perf_counter() - t0)
            cpu = {"kind": "reference", "cores": os.cpu_count(),
                   "sample": f"{len(small)} requests with <= 16 qubits through moonlab_qgtl_execute",
                   "mean_service_ms": 1e3 * sum(t_cpu) / len(t_cpu),
                   "b200_mean_service_ms": 1e3 * sum(gpu_alone) / len(gpu_alone)}
        except Exception as e:  # reported, never replaced
            cpu = {"kind": "reference", "sample": f"unavailable: {e}"}
    lat = np.array([info["latency_s"] for _, info in paced["results"]])
    return {
        "workload": (f"{len(reqs):,} requests of the Poisson stream (seed 0xC5) at {args.serve_rate:g}/s: "
                     "qubits U{10..28}, depth U{10..100} brickwork, shots U{1..4096}, c128/c64 50/50"),
        "rate_per_s": args.serve_rate, "workers": workers, "requests": len(reqs),
        "circuits_per_s": paced["circuits_per_s"], "p50_ms": paced["p50_s"] * 1e3,
        "p99_ms": paced["p99_s"] * 1e3, "mean_ms": paced["mean_s"] * 1e3,
        "p999_ms": float(np.percentile(lat, 99.9)) * 1e3, "span_s": paced["span_s"],
        "capacity": {"requests": ncap, "circuits_per_s": sat["circuits_per_s"], "p99_ms": sat["p99_s"] * 1e3,
                     "how": f"the first {ncap} requests of the stream submitted at once"},
        "peak_running": paced["stats"]["peak_running"],
        "peak_reserved_gib": paced["stats"]["peak_reserved_bytes"] / 2**30,
        "p99_target_ms": p99_target_ms, "rate_sweep": sweep,
        "max_rate_meeting_p99_per_s": max(meets) if meets else None,
        "small_batches": paced["stats"]["small_batches"], "plan_cache_hits": paced["stats"]["plan_cache_hits"],
        "cpu_reference": cpu,
        "small_requests": small_leg,
    }


def small_requests_leg(local, num: int = 1000, rate: float = 200.0):
    """Small requests alone (8..12 qubits complex128, depth U{10..100}
    brickwork, shots U{1..4096}, Poisson at `rate`/s): the batch launches of
    mlb_server_* against the persistent loop (mlb_mailbox_*), p50/p99
    latency from submit to result on the host clock."""
    from moonlab_b200.circuits import Request
    from moonlab_b200.serving import Mailbox, Server, request_circuit, run_load, run_mailbox_load
    rng = np.random.default_rng(0x5A11)
    gaps = rng.exponential(1.0 / rate, num)
    reqs = [Request(i, float(t), int(rng.integers(8, 13)), int(rng.integers(10, 101)), int(rng.integers(1, 4097)),
                    0, int(rng.integers(1, 2**62))) for i, t in enumerate(np.cumsum(gaps))]
    circ = [request_circuit(r) for r in reqs]
    with Server(device=local, workers=8) as srv:
        run_load(srv, reqs[:50], time_scale=0.0, circuits=circ[:50])  # warm-up
        batch = run_load(srv, reqs, time_scale=1.0, circuits=circ)
    with Mailbox("c128", device=local, ctas=8) as mb:
        run_mailbox_load(mb, reqs[:50], time_scale=0.0, circuits=circ[:50])
        loop = run_mailbox_load(mb, reqs, time_scale=1.0, circuits=circ)
    pick = lambda d: {"circuits_per_s": d["circuits_per_s"], "p50_ms": d["p50_s"] * 1e3, "p99_ms": d["p99_s"] * 1e3,
                      "mean_ms": d["mean_s"] * 1e3}
    return {"workload": f"{num} requests of 8..12 qubits (c128), depth U{{10..100}} brickwork, shots U{{1..4096}}, "
                        f"Poisson at {rate:g}/s",
            "batch_launches": pick(batch), "persistent_loop": dict(pick(loop), ctas=8,
                                                                    launches=loop["stats"]["launches"])}


def gate_sweep_leg(local, peak):
    """Per-gate HBM throughput on the per-gate kernels (one full sweep over
    the amplitudes a gate touches), depth-20-circuit sizes 26..33 qubits in
    complex128 and 26..34 in complex64: RX on low (0, 1, 2), middle (n/2) and
    high (n-3 .. n-1) targets, CNOT and CRZ with the control below / above
    the target.  GB/s = 2 x (bytes of the touched amplitudes) / device time
    of the gate's kernel (CUDA events on the engine's stream), median of 3."""
    from moonlab_b200 import StateVector
    c, sn = math.cos(0.15), math.sin(0.15)
    rx = np.array([[c, -1j * sn], [-1j * sn, c]])
    xm = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    rz = np.diag([np.exp(-0.15j), np.exp(0.15j)])
    out = {}
    for dtype, ns in (("c128", (26, 28, 30, 32, 33)), ("c64", (26, 28, 30, 32, 34))):
        out[dtype] = {}
        for n in ns:
            sv = StateVector(n, dtype, device=local)
            sv.set_exec_mode("eager")
            sv.set_timing(True)
            mid = n // 2
            cases = [("rx_low", [(lambda q=q: sv.apply_1q(q, rx)) for q in (0, 1, 2)]),
                     ("rx_mid", [lambda: sv.apply_1q(mid, rx)]),
                     ("rx_high", [(lambda q=q: sv.apply_1q(q, rx)) for q in (n - 3, n - 2, n - 1)]),
                     ("cnot_ctrl_below", [lambda: sv.apply_controlled_1q([1], mid, xm)]),
                     ("cnot_ctrl_above", [lambda: sv.apply_controlled_1q([n - 2], mid, xm)]),
                     ("crz_ctrl_below", [lambda: sv.apply_controlled_1q([1], mid, rz)]),
                     ("crz_ctrl_above", [lambda: sv.apply_controlled_1q([n - 2], mid, rz)])]
            row = {}
            for name, fns in cases:
                rates = []
                for f in fns:
                    ts = []
                    for rep in range(4):
                        f()
                        sv.flush()
                        st = sv.flush_stats()
                        if rep:
                            ts.append(st["bytes_moved"] / (st["gpu_ms"] / 1e3) / 1e9)
                    rates.append(statistics.median(ts))
                row[name] = round(statistics.median(rates), 1)
            row["frac_of_peak_rx_mid"] = round(row["rx_mid"] / peak, 3)
            out[dtype][str(n)] = row
            sv.close()
    return out


def vqe_leg(local, with_cpu: bool):
    """VQE adjoint gradient: hardware-efficient ansatz N = 20, L = 8 (320
    parameters), 80 random 2-local Pauli terms, a batch of 256 parameter
    vectors in one call, complex128 and complex64; host parameters in,
    host energies and gradients out (timed end to end)."""
    from moonlab_b200.circuits import config_c4
    from moonlab_b200.vqe import HEAProblem
    prob = config_c4(n=20, layers=8, batch=256, seed=0xC4)
    res = {"workload": "HEA N=20 L=8 (320 parameters), 80 2-local Pauli terms, batch 256"}
    grads = {}
    peak, peak_kind = measured_peaks()
    for dt in ("c128", "c64", "c64_cuda_core_forward"):
        p = HEAProblem(20, 8, prob.coeffs, xmasks=prob.xmasks, zmasks=prob.zmasks,
                       dtype="c128" if dt == "c128" else "c64", device=local)
        if dt == "c64_cuda_core_forward":
            p.set_fused_forward("off")
        p.evaluate(prob.params)  # warm-up at the full batch: workspaces are sized by the first call
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            E, G = p.evaluate(prob.params)
            times.append(time.perf_counter() - t0)
        t = statistics.median(times)
        grads[dt] = G
        # algorithmic bytes of one batch (per vector, S = one state's bytes):
        # forward passes read + write psi (2 S each), the first lambda pass
        # reads psi and writes lambda (2 S), later ones also read lambda (3 S),
        # backward passes read + write psi and lambda (4 S each), and each
        # checkpoint is saved and restored once (2 S + 2 S)
        ps, ev = p.plan_stats(), p.last_eval_stats()
        S = (16 if dt == "c128" else 8) << 20
        ck = 0
        if ev["checkpoints"]:
            ck = -(-8 // ev["segment_layers"]) - 1  # segments - 1
        fwd = ev["fused_forward_passes"] if ev["fused_forward"] else ps["forward_passes"]
        per_vec = S * (2 * fwd + 2 + 3 * (ps["lambda_passes"] - 1) + 4 * ps["backward_passes"] + 4 * ck)
        achieved = per_vec * len(prob.params) / t / 1e9
        path = ("complex128 adjoint tile passes on the CUDA cores" if dt == "c128" else
                "complex64: forward sweep on the tensor cores (fused <= 5-qubit blocks, per-vector operand "
                "images built on the device), lambda and backward passes on the CUDA cores"
                if ev["fused_forward"] else "complex64 adjoint tile passes on the CUDA cores")
        res[dt] = {"vectors_per_s": len(prob.params) / t, "batch_ms": t * 1e3, "path": path,
                   "timing": "median of 3 calls after a full-batch warm-up (host parameters in, host "
                             "energies and gradients out)",
                   "passes": ps, "checkpoints": ev,
                   "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                "frac": achieved / peak, "peak_source": peak_kind,
                                "algorithmic_bytes_per_vector": per_vec,
                                "kernel": "k_adj_gates / k_adj_pauli (whole evaluation)"}}
        p.close()
    res["c64_max_rel_grad_err"] = float(np.abs(grads["c64"] - grads["c128"]).max() /
                                        max(1e-300, np.abs(grads["c128"]).max()))
    res["c64_cuda_core_forward_max_rel_grad_err"] = float(
        np.abs(grads["c64_cuda_core_forward"] - grads["c128"]).max() / max(1e-300, np.abs(grads["c128"]).max()))
    if with_cpu:  # the reference's moonlab_vqe_gradient at N = 12 (minutes per vector at N = 20)
        try:
            from oracle import bindings as B
            small = config_c4(n=12, layers=8, batch=64, seed=0xC4)
            p12 = HEAProblem(12, 8, small.coeffs, xmasks=small.xmasks, zmasks=small.zmasks, device=local)
            p12.evaluate(small.params[:4])
            t0 = time.perf_counter()
            p12.evaluate(small.params)
            gpu12 = len(small.params) / (time.perf_counter() - t0)
            p12.close()
            solver = B.RefSolver(12, 8, small.paulis, small.coeffs)
            t0 = time.perf_counter()
            for k in range(2):
                solver.gradient(small.params[k])
            cpu12 = 2 / (time.perf_counter() - t0)
            solver.close()
            res["cpu_reference"] = {"kind": "reference", "cores": os.cpu_count(),
                                    "sample": "moonlab_vqe_gradient, N=12 L=8, 48 terms, 2 vectors",
                                    "vectors_per_s": cpu12, "b200_c128_vectors_per_s_same_problem": gpu12}
        except Exception as e:  # reported, never replaced
            res["cpu_reference"] = {"kind": "reference", "sample": f"unavailable: {e}"}
    return res


class _DeviceView:
    """__cuda_array_interface__ over an engine-owned device buffer (for torch)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--ref-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=10000)
    ap.add_argument("--serve-rate", type=float, default=25.0)
    ap.add_argument("--serve-capacity", type=int, default=1000)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the per-gate GB/s sweep")
    ap.add_argument("--no-vqe", action="store_true", help="skip the VQE adjoint-gradient leg")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_b200(args, ws, rank, local)
    finally:
        dist_done(ws)


if __name__ == "__main__":
    main()
