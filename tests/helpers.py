"""Shared helpers for the test-suite (random states, unitaries, circuits)."""
from __future__ import annotations

import math

import numpy as np


def rand_state(n: int, seed: int, dtype=np.complex64) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    v /= np.linalg.norm(v)
    return v.astype(dtype)


def haar_u2(rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def random_invertible_rows(n: int, rng: np.random.Generator):
    """Uniform random n-bit rows, resampled until invertible over GF(2)."""
    while True:
        rows = [int(x) for x in rng.integers(0, 1 << n, size=n, dtype=np.uint64)]
        # rank via elimination
        basis = []
        for r in rows:
            for b in basis:
                r = min(r, r ^ b)
            if r:
                basis.append(r)
        if len(basis) == n:
            return rows


def oracle_apply_terms(o, terms) -> None:
    """Apply fused diagonal terms (kind, a, b, params) with the oracle's
    per-gate routines (kinds as in mettleq_b200.fusion.DIAG_*)."""
    from mettleq_b200 import fusion as F
    for kind, a, b, p in terms:
        t = p[0] if p else 0.0
        if kind == F.DIAG_ZZ:
            o.apply_zz_phase(t, a, b)
        elif kind == F.DIAG_CPHASE:
            o.apply_diagonal([1, 1, 1, np.exp(1j * t)], [a, b])
        elif kind == F.DIAG_CRZ:
            o.apply_diagonal([1, 1, np.exp(-0.5j * t), np.exp(0.5j * t)], [a, b])
        elif kind == F.DIAG_RZ:
            o.apply_diagonal([np.exp(-0.5j * t), np.exp(0.5j * t)], [a])
        elif kind == F.DIAG_PHASE:
            o.apply_diagonal([1, np.exp(1j * t)], [a])
        elif kind == F.DIAG_1Q:
            o.apply_diagonal([p[0] + 1j * p[1], p[2] + 1j * p[3]], [a])
        elif kind == F.DIAG_2Q:
            o.apply_diagonal([p[2 * i] + 1j * p[2 * i + 1] for i in range(4)], [a, b])
        elif kind == F.DIAG_GLOBAL:
            o.apply_global_phase(t)
        else:
            raise AssertionError(kind)
