"""Generate the committed golden fixtures from the reference itself.

Run where the reference tree is (the script reads its circuit corpus,
tests/oracle/corpus/circuit_corpus.json) and the reference library is built
from its sources (oracle/Makefile -> oracle/_ref/liboracle.so); the tree is
given by --reference or the MOONLAB_REFERENCE environment variable:

    make -C oracle ref REF=<tree> && python tests/golden/gen_golden.py --reference <tree>

(`python tests/golden/gen_golden.py circuit_text` writes only
circuit_text.json.)  Every expected value below is produced by calling the
reference's own public C functions (gate_*, measurement_*,
moonlab_qgtl_execute, moonlab_scheduler_run, moonlab_vqe_gradient,
moonlab_qgtl_circuit_serialize / _deserialize) through ctypes.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

from moonlab_b200.circuits import GATE_DTYPE, SplitMix64, brickwork, config_c4  # noqa: E402
from oracle import bindings as B  # noqa: E402

def reference_tree() -> Path:
    """The reference tree: --reference PATH, else $MOONLAB_REFERENCE."""
    args = sys.argv[1:]
    if "--reference" in args:
        return Path(args[args.index("--reference") + 1])
    env = os.environ.get("MOONLAB_REFERENCE")
    if not env:
        raise SystemExit("give the reference tree: --reference PATH or MOONLAB_REFERENCE=PATH")
    return Path(env)


CORPUS_REL = Path("tests/oracle/corpus/circuit_corpus.json")
OUT = Path(__file__).resolve().parent / "reference_golden.npz"
NAME2TYPE = dict(x=1, y=2, z=3, h=4, s=5, t=6, rx=7, ry=8, rz=9, cnot=10, cz=12, swap=13,
                 sdg=20, tdg=21)


def corpus_gates(c) -> np.ndarray:
    recs = []
    for g in c["gates"]:
        t, q = NAME2TYPE[g["g"]], g["q"]
        if len(q) == 2:
            recs.append((t, q[1], q[0], 0, float(g["p"])))  # (control q[0], target q[1])
        else:
            recs.append((t, q[0], -1, 0, float(g["p"])))
    return np.array(recs, dtype=GATE_DTYPE)


def main() -> None:
    L = B.ref()
    out = {}
    circuits = json.loads((reference_tree() / CORPUS_REL).read_text())["circuits"]
    ids, ns, offs, gates_all, amp_offs, amps_all = [], [], [0], [], [0], []
    samp_u = SplitMix64(0x601DE11).uniforms(256)
    samp_all, mall_all, ez_all, ex0, ey0, zz01 = [], [], [], [], [], []
    for c in circuits:
        n = c["num_qubits"]
        g = corpus_gates(c)
        r = B.RefStateVector(n)
        r.run(g)
        a = r.amplitudes()
        ids.append(c["id"])
        ns.append(n)
        gates_all.append(g)
        offs.append(offs[-1] + len(g))
        amps_all.append(a)
        amp_offs.append(amp_offs[-1] + a.size)
        samp_all.append(r.sample(samp_u))
        # measurement_all_qubits collapses: run it on clones, one uniform each
        mo = []
        for u in samp_u[:64]:
            cl = B.RefState()
            L.quantum_state_clone(C.byref(cl), C.byref(r.s))
            mo.append(L.measurement_all_qubits(C.byref(cl), float(u)))
            L.quantum_state_free(C.byref(cl))
        mall_all.append(np.array(mo, dtype=np.uint64))
        ez_all.append(np.array([L.measurement_expectation_z(C.byref(r.s), q) for q in range(n)]))
        ex0.append(L.measurement_expectation_x(C.byref(r.s), 0))
        ey0.append(L.measurement_expectation_y(C.byref(r.s), 0))
        zz01.append(L.measurement_correlation_zz(C.byref(r.s), 0, 1))
        r.close()
    out.update(corpus_ids=np.array(ids), corpus_n=np.array(ns), corpus_gate_offsets=np.array(offs),
               corpus_gates=np.concatenate(gates_all), corpus_amp_offsets=np.array(amp_offs),
               corpus_amps=np.concatenate(amps_all), sample_uniforms=samp_u,
               corpus_sample=np.stack(samp_all), corpus_measure_all=np.stack(mall_all),
               corpus_ez=np.concatenate(ez_all), corpus_ex0=np.array(ex0), corpus_ey0=np.array(ey0),
               corpus_zz01=np.array(zz01))

    # 12-qubit brickwork (the 20-qubit workload's structure at oracle-cheap size)
    g12 = brickwork(12, 20, 0xC1)
    r = B.RefStateVector(12)
    r.run(g12)
    out.update(bw12_gates=g12, bw12_amps=r.amplitudes(), bw12_probs=r.probabilities())
    r.close()
    outs, probs = B.ref_qgtl_execute(12, g12[[t in (7, 8, 9, 10) for t in g12["type"]]], 1024, 0xABCDEF)
    out.update(bw12_qgtl_outcomes=outs, bw12_qgtl_probs=probs, bw12_qgtl_seed=np.uint64(0xABCDEF))

    # scheduler simulator backend: 10 qubits, 1000 shots over 4 workers
    g10 = brickwork(10, 8, 0x5C4ED)
    job = L.moonlab_job_create(10)
    for gr in g10:
        par = C.c_double(float(gr["theta"]))
        L.moonlab_job_add_gate(job, int(gr["type"]), int(gr["target"]), int(gr["control"]),
                               C.byref(par) if int(gr["type"]) in (7, 8, 9) else None)
    L.moonlab_job_set_num_shots(job, 1000)
    L.moonlab_job_set_num_workers(job, 4)
    L.moonlab_job_set_rng_seed(job, 0x1234ABCD)
    res = B.JobResults()
    rc = L.moonlab_scheduler_run(job, C.byref(res))
    assert rc == 0, rc
    out.update(sched_gates=g10, sched_outcomes=np.ctypeslib.as_array(res.outcomes, shape=(1000,)).copy(),
               sched_seed=np.uint64(0x1234ABCD), sched_workers=np.int32(4))
    buf = C.create_string_buffer(1 << 20)
    L.moonlab_job_to_json(job, buf, len(buf))
    out.update(sched_json=np.array(buf.value.decode()))
    L.moonlab_job_results_free(C.byref(res))
    L.moonlab_job_free(job)

    # VQE adjoint gradient (moonlab_vqe_gradient) on small HEA problems
    for tag, n, layers, terms, batch in (("vqe4", 4, 2, 16, 3), ("vqe6", 6, 3, 24, 2)):
        prob = config_c4(n=n, layers=layers, batch=batch, num_terms=terms, seed=0xC4 ^ n)
        grads = np.stack([B.ref_vqe_gradient(n, layers, prob.paulis, prob.coeffs, p) for p in prob.params])
        out.update({f"{tag}_paulis": np.array(prob.paulis), f"{tag}_coeffs": prob.coeffs,
                    f"{tag}_params": prob.params, f"{tag}_grads": grads,
                    f"{tag}_shape": np.array([n, layers])})

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    circuit_text()


# Edge cases of the "moonlab-circuit v1" reader: the reference's verdict on
# each (moonlab_qgtl_circuit_deserialize with the text's length).
TEXT_CASES = [
    "NUM_QUBITS 4\nH 0\nCNOT 1 0\n",
    "  # lead comment\n\n\t\nNUM_QUBITS 4\n   # indented comment\nX 3\n\n",
    "NUM_QUBITS 4\r\nRX 1 0.5\r\nCZ 2 3\r\n",
    "NUM_QUBITS 4\nRY 0 -1e-300\nRZ 1 1e308\nRX 2 0x1.8p1\nRY 3 +.5\nRZ 0 -0\n",
    "NUM_QUBITS 4\nRX 0 1e\nRY 1 1e+\nRZ 2 0x1p\n",
    "NUM_QUBITS 4\nRX 0 inf\nRY 1 -infinity\nRZ 2 nan\n",
    "NUM_QUBITS 4\nRX 0 0x\n",
    "NUM_QUBITS 4\nRX 0 infin\n",
    "NUM_QUBITS 4\nRX 0\n",
    "NUM_QUBITS 4\nRX 0 .\n",
    "NUM_QUBITS 4\nH 0 junk after\nCNOT 1 2 3 4\nRX 3 0.25rad\n",
    "NUM_QUBITS 4\nCNOT 1 1\n",
    "NUM_QUBITS 4\nCNOT 4 0\n",
    "NUM_QUBITS 4\nCNOT 0 -1\n",
    "NUM_QUBITS 4\nCNOT 0\n",
    "NUM_QUBITS 4\nH 4\n",
    "NUM_QUBITS 4\nH -1\n",
    "NUM_QUBITS 4\nH +2\n",
    "NUM_QUBITS 4\nH 01\n",
    "NUM_QUBITS 4\nH\n",
    "NUM_QUBITS 4\nh 0\n",
    "NUM_QUBITS 4\nCX 0 1\n",
    "NUM_QUBITS 4\nHADAMARD 0\n",
    "NUM_QUBITS 4\nH0\n",
    "NUM_QUBITS 4\nSWAP 3 2\nCY 0 3\nI 1\nS 2\nT 3\nY 0\nZ 1\n",
    "NUM_QUBITS 4\nCNOT 1+2\n",
    "NUM_QUBITS 4\nCNOT 1,2\n",
    "NUM_QUBITS4\nH 0\n",
    "NUM_QUBITS 4 trailing\nH 0\n",
    "NUM_QUBITS 0\n",
    "NUM_QUBITS 32\nH 31\n",
    "NUM_QUBITS 33\nH 0\n",
    "NUM_QUBITS -3\n",
    "NUM_QUBITS\n",
    "num_qubits 4\nH 0\n",
    "H 0\nNUM_QUBITS 4\n",
    "# only a comment\n",
    "",
    "NUM_QUBITS 4\nNUM_QUBITS 4\n",
    "NUM_QUBITS 4",
    "NUM_QUBITS 4\nRX 3 0.125",
    "NUM_QUBITS 4\nRX 0 " + "1" * 240 + "\n",
    "NUM_QUBITS 4\nRX 0 " + "1" * 260 + "\n",
    "NUM_QUBITS 4\n" + " " * 300 + "\nH 0\n",
    "NUM_QUBITS 4\n" + " " * 300 + "H 0\n",
]


def circuit_text() -> None:
    """tests/golden/circuit_text.json: the reference serializer's text for a
    circuit of every gate type, and its deserializer's verdict on TEXT_CASES."""
    gates = brickwork(10, 6, 0x7E47)
    extra = np.zeros(14 + 6, dtype=GATE_DTYPE)
    extra["type"] = list(range(14)) + [7, 8, 9, 7, 8, 9]
    extra["target"] = [q % 10 for q in range(3, 23)]
    extra["control"] = [(q + 4) % 10 for q in range(3, 23)]
    extra["theta"] = [0.0] * 7 + [1.0 / 3, -2.5, 1e-300] + [0.0] * 4 + [-0.0, 6.283185307179586, 1e300,
                                                                        float.fromhex("0x1.fffffffffffffp+1"),
                                                                        5e-324, -12345.678901234567]
    gates = np.concatenate([gates, extra])
    text = B.ref_circuit_text(10, gates)
    cases = []
    for t in TEXT_CASES:
        st, back = B.ref_circuit_roundtrip(t.encode())
        cases.append({"text": t, "status": st, "reserialized": back})
    out = Path(__file__).resolve().parent / "circuit_text.json"
    out.write_text(json.dumps({"num_qubits": 10, "gates": [[int(g["type"]), int(g["target"]), int(g["control"]),
                                                            float(g["theta"]).hex()] for g in gates],
                               "text": text, "cases": cases}, indent=0))
    print(f"wrote {out} ({out.stat().st_size} bytes)")


if __name__ == "__main__":
    if "circuit_text" in sys.argv[1:]:
        circuit_text()
        sys.exit(0)
    main()
