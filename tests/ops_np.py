"""Dense numpy application of the engine's op kinds, the reference for the
random-op GPU tests.  tests/test_oracle_pin.py pins it to the oracle's
kernels (oracle/sv_oracle.c: svo_apply_1q_matrix, svo_apply_2q_matrix,
svo_apply_mcx, svo_apply_mcz and the SWAP / Fredkin / ZZ / CRX / CRY / CRZ
gates), so the GPU tests that use it compare against the pinned oracle."""
from __future__ import annotations

import numpy as np


def np_apply(a, n, kind, t, t2, cmask, m):
    idx = np.arange(1 << n, dtype=np.uint64)
    sel = (idx & np.uint64(cmask)) == np.uint64(cmask)
    out = a.copy()
    if kind in ("1q", "x"):
        tb = np.uint64(1 << t)
        i0 = idx[sel & ((idx & tb) == 0)]
        i1 = i0 | tb
        if kind == "x":
            out[i0], out[i1] = a[i1], a[i0]
        else:
            M = m.reshape(2, 2)
            out[i0] = M[0, 0] * a[i0] + M[0, 1] * a[i1]
            out[i1] = M[1, 0] * a[i0] + M[1, 1] * a[i1]
    elif kind in ("2q", "swap"):
        b0, b1 = np.uint64(1 << t), np.uint64(1 << t2)
        base = idx[sel & ((idx & (b0 | b1)) == 0)]
        ii = [base, base | b0, base | b1, base | b0 | b1]
        if kind == "swap":
            out[ii[1]], out[ii[2]] = a[ii[2]], a[ii[1]]
        else:
            M = m.reshape(4, 4)
            for r in range(4):
                out[ii[r]] = sum(M[r, c] * a[ii[c]] for c in range(4))
    elif kind == "zz":
        par = ((idx >> np.uint64(t)) ^ (idx >> np.uint64(t2))) & np.uint64(1)
        out = np.where(par == 0, m[0], m[1]) * a
    elif kind == "phase":
        out = np.where(sel, m[0] * a, a)
    return out


def rand_unitary(rng, d):
    z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))
