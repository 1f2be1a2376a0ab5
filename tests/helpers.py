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
