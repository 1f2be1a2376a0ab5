"""Seeded synthetic circuits for the benchmark configurations.

There is no public dataset on this path: every workload is generated here
from a fixed seed with the shapes of the benchmark configurations.

plain / scale layer (one "layer"):
  * a Haar-random U(2) on every qubit: QR of a complex Ginibre 2x2 with the
    phase fix of Mezzadri (2007); draw order layer -> qubit;
  * RZZ(t) = exp(-i t/2 Z Z) on (i, i+1), i = 0..n-2, t ~ U[0, 2pi) (passed
    to the native ZZPHASE as t/2, integrations/qiskit.py:572-575);
  * a CNOT ladder CNOT(0,1), CNOT(1,2), ..., CNOT(n-2,n-1), applied in order.
The scale workload inserts a full QFT (no swaps) after every 10th layer,
followed by a random GF(2) permutation layer (uniform random n-bit rows,
resampled until invertible, plus a random n-bit flip).
"""
from __future__ import annotations

import cmath
import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np


def haar_u2(rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def u3_params(u: np.ndarray) -> Tuple[float, float, float, float]:
    """(theta, phi, lam, alpha) with u = e^{i alpha} U3(theta, phi, lam)
    and U3 = RZ(phi) RY(theta) RZ(lam) (gates.py:85-87)."""
    alpha = cmath.phase(np.linalg.det(u)) / 2.0
    v = u * cmath.exp(-1j * alpha)
    a, b = v[0, 0], v[1, 0]
    theta = 2.0 * math.atan2(abs(b), abs(a))
    pa = cmath.phase(a) if abs(a) > 1e-300 else 0.0
    pb = cmath.phase(b) if abs(b) > 1e-300 else 0.0
    phi = pb - pa
    lam = -pa - pb
    return theta, phi, lam, alpha


def invertible_rows(n: int, rng: np.random.Generator) -> List[int]:
    while True:
        rows = [int(x) for x in rng.integers(0, 1 << n, size=n, dtype=np.uint64)]
        basis: List[int] = []
        for r in rows:
            for b in basis:
                r = min(r, r ^ b)
            if r:
                basis.append(r)
        if len(basis) == n:
            return rows


@dataclass
class Layer:
    mats: np.ndarray                   # (n, 4) complex128 Haar U(2)
    thetas: np.ndarray                 # (n-1,) RZZ angles t (exp(-i t/2 ZZ))
    qft_after: bool = False
    xor: Optional[Tuple[List[int], int]] = None


@dataclass
class Circuit:
    n: int
    layers: List[Layer] = field(default_factory=list)

    # -- kernel-level counts --------------------------------------------
    def logical_layers(self) -> int:
        """U(2) layer + RZZ layer + CNOT ladder per layer, plus each QFT and
        each permutation layer."""
        k = 3 * len(self.layers)
        k += sum(1 for L in self.layers if L.qft_after)
        k += sum(1 for L in self.layers if L.xor is not None)
        return k

    def ops(self) -> Tuple[List[dict], float]:
        """Canonical op dicts (U3 + ZZPHASE + CNOT, QFT as H/CPHASE stages,
        permutation layers as explicit rows) and the accumulated global phase."""
        n = self.n
        out: List[dict] = []
        gphase = 0.0
        for L in self.layers:
            for q in range(n):
                th, ph, lam, al = u3_params(L.mats[q].reshape(2, 2))
                out.append({"name": "U3", "wires": [q], "parameters": [th, ph, lam]})
                gphase += al
            for i in range(n - 1):
                out.append({"name": "ZZPHASE", "wires": [i, i + 1], "parameters": [float(L.thetas[i]) / 2.0]})
            for i in range(n - 1):
                out.append({"name": "CNOT", "wires": [i, i + 1], "parameters": []})
            if L.qft_after:
                out.extend(qft_ops(n))
            if L.xor is not None:
                out.extend(affine_gates(list(L.xor[0]), int(L.xor[1]), n))
        return out, gphase


def qft_ops(n: int, wires: Optional[List[int]] = None) -> List[dict]:
    """Gate-decomposed QFT without swaps: H(j) then CPHASE(k -> j, pi/2^(k-j))."""
    w = list(range(n)) if wires is None else list(wires)
    ops = []
    for j in range(len(w)):
        ops.append({"name": "H", "wires": [w[j]], "parameters": []})
        for k in range(j + 1, len(w)):
            ops.append({"name": "CPHASE", "wires": [w[k], w[j]], "parameters": [math.pi / (1 << (k - j))]})
    return ops


def plain_circuit(n: int = 20, layers: int = 20, seed: int = 0) -> Circuit:
    rng = np.random.default_rng(seed)
    c = Circuit(n)
    for _ in range(layers):
        mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
        thetas = rng.uniform(0.0, 2.0 * math.pi, n - 1)
        c.layers.append(Layer(mats, thetas))
    return c


def scale_circuit(n: int = 30, layers: int = 40, seed: int = 0, qft_every: int = 10) -> Circuit:
    rng = np.random.default_rng(seed)
    c = Circuit(n)
    for i in range(layers):
        mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
        thetas = rng.uniform(0.0, 2.0 * math.pi, n - 1)
        L = Layer(mats, thetas)
        if (i + 1) % qft_every == 0:
            L.qft_after = True
            L.xor = (invertible_rows(n, rng), int(rng.integers(0, 1 << n)))
        c.layers.append(L)
    return c


def cnot_ladder_rows(n: int) -> Tuple[List[int], int]:
    """Inverse rows of CNOT(0,1), ..., CNOT(n-2,n-1) (xor_affine.py:46-76)."""
    rows = [1 << (n - 1 - k) for k in range(n)]
    for a in reversed(range(n - 1)):
        rows[a + 1] ^= rows[a]
    return rows, 0


def affine_gates(rows: List[int], c: int, n: int) -> List[dict]:
    """CNOT/SWAP/X sequence whose permutation is out[y] = in[src(y)] with
    src qubit-k bit = parity(rows[k] & y) ^ bit_k(c) (xor_affine.py:22-32).

    The forward basis map is f = src^{-1}: f(x) = M x ^ d with M = A^{-1},
    d = A^{-1} c.  Gauss-Jordan elimination writes M = E_1 E_2 ... E_k with
    elementary row operations E (CNOT: row_t += row_c; SWAP: exchange), so
    the gates run E_k first and E_1 last, followed by X on the bits of d."""
    # A as index-bit rows: A[b] = mask of y bits feeding src bit b
    A = [0] * n
    for k, r in enumerate(rows):
        A[n - 1 - k] = r
    # M = A^{-1} by Gauss-Jordan on [A | I]
    work = list(A)
    inv = [1 << b for b in range(n)]
    for col in range(n):
        piv = next((r for r in range(col, n) if (work[r] >> col) & 1), None)
        if piv is None:
            raise ValueError("affine map is not invertible over GF(2)")
        work[col], work[piv] = work[piv], work[col]
        inv[col], inv[piv] = inv[piv], inv[col]
        for r in range(n):
            if r != col and (work[r] >> col) & 1:
                work[r] ^= work[col]
                inv[r] ^= inv[col]
    M = inv
    d = 0
    for b in range(n):
        d |= (bin(M[b] & c).count("1") & 1) << b
    # eliminate M to I with recorded row operations
    E: List[Tuple[str, int, int]] = []
    work = list(M)
    for col in range(n):
        piv = next(r for r in range(col, n) if (work[r] >> col) & 1)
        if piv != col:
            work[col], work[piv] = work[piv], work[col]
            E.append(("SWAP", col, piv))
        for r in range(n):
            if r != col and (work[r] >> col) & 1:
                work[r] ^= work[col]
                E.append(("CNOT", col, r))
    gates = []
    for kind, a, b in reversed(E):
        gates.append({"name": kind, "wires": [n - 1 - a, n - 1 - b], "parameters": []})
    for b in range(n):
        if (d >> b) & 1:
            gates.append({"name": "X", "wires": [n - 1 - b], "parameters": []})
    return gates


def run_circuit_layers(sv, circuit: Circuit, on_layer=None, fused: bool = True) -> None:
    """Apply a circuit at the kernel level.  Each config layer (U(2) layer,
    RZZ diagonal, CNOT-ladder permutation) is one fused ``apply_layer`` call
    (``fused=False``: the three layer calls), then the QFT / permutation
    layers.  ``on_layer(kind, edge)`` brackets every call (edge 0 before,
    1 after) with kind "layer" (or "u2" / "diag" / "xor"), "qft" or "xor"."""
    n = circuit.n
    bonds = [(i, i + 1) for i in range(n - 1)]
    ladder = cnot_ladder_rows(n)

    def run(kind, fn):
        if on_layer:
            on_layer(kind, 0)
        fn()
        if on_layer:
            on_layer(kind, 1)

    from .fusion import DIAG_ZZ
    for L in circuit.layers:
        if fused:
            terms = [(DIAG_ZZ, i, i + 1, [t / 2.0]) for i, t in enumerate(L.thetas)]
            run("layer", lambda: sv.apply_layer(L.mats, None, terms, *ladder))
        else:
            run("u2", lambda: sv.apply_u2_layer(L.mats))
            run("diag", lambda: sv.apply_zz_weighted(bonds, [t / 2.0 for t in L.thetas]))
            run("xor", lambda: sv.apply_xor_affine(*ladder))
        if L.qft_after:
            run("qft", lambda: sv.apply_qft(None))
        if L.xor is not None:
            run("xor", lambda: sv.apply_xor_affine(*L.xor))
