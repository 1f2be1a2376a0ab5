"""numpy restatement of the reference's CPU statevector algorithm.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Every routine below
cites the reference function whose semantics it restates (paths relative to
the MettleQ source tree).  The oracle applies one full-state numpy pass per
gate, exactly as the reference's pure-MLX path does (device.py:1138-1290), in
complex64 (the reference's only amplitude type, execution.py:21-22) or in
complex128 (the FP64 oracle).

Conventions (reference): qubit ``q`` is state-index bit ``n-1-q`` (MSB-first,
sim.py:10-14); the initial state is |0...0> (sim.py:32-45).
"""
from __future__ import annotations

import math
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

_SQ = 1.0 / math.sqrt(2.0)


# --------------------------------------------------------------------------
# Gate matrices -- gates.py:5-234
# --------------------------------------------------------------------------
def _rz(theta: float) -> np.ndarray:
    ht = theta / 2.0
    return np.array([[complex(math.cos(-ht), math.sin(-ht)), 0], [0, complex(math.cos(ht), math.sin(ht))]],
                    dtype=np.complex128)


def _ry(theta: float) -> np.ndarray:
    c, s = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def gate_matrix(name: str, params: Sequence[float] = ()) -> np.ndarray:
    """Single-qubit 2x2 matrix in complex128 (gates.py:5-87).

    U2(phi, lam) = RZ(phi) RY(pi/2) RZ(lam) and U3(theta, phi, lam) =
    RZ(phi) RY(theta) RZ(lam) (gates.py:80-87); RZ(t) = diag(e^{-it/2},
    e^{+it/2}) (gates.py:64-68).
    """
    name = name.upper()
    name = {"SDAG": "SDG", "TDAG": "TDG", "S†": "SDG", "T†": "TDG"}.get(name, name)
    p = list(params)
    if name == "I":
        return np.eye(2, dtype=np.complex128)
    if name == "X":
        return np.array([[0, 1], [1, 0]], dtype=np.complex128)
    if name == "Y":
        return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    if name == "Z":
        return np.array([[1, 0], [0, -1]], dtype=np.complex128)
    if name == "H":
        return np.array([[_SQ, _SQ], [_SQ, -_SQ]], dtype=np.complex128)
    if name == "S":
        return np.array([[1, 0], [0, 1j]], dtype=np.complex128)
    if name == "SDG":
        return np.array([[1, 0], [0, -1j]], dtype=np.complex128)
    if name in ("T", "TDG"):
        ang = math.pi / 4.0 if name == "T" else -math.pi / 4.0
        return np.array([[1, 0], [0, complex(math.cos(ang), math.sin(ang))]], dtype=np.complex128)
    if name == "SX":
        a, b = complex(0.5, 0.5), complex(0.5, -0.5)
        return np.array([[a, b], [b, a]], dtype=np.complex128)
    if name == "RX":
        c, s = math.cos(p[0] / 2.0), math.sin(p[0] / 2.0)
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)
    if name == "RY":
        return _ry(p[0])
    if name == "RZ":
        return _rz(p[0])
    if name in ("U1", "PHASESHIFT"):
        return np.array([[1, 0], [0, complex(math.cos(p[0]), math.sin(p[0]))]], dtype=np.complex128)
    if name == "U2":
        return _rz(p[0]) @ _ry(math.pi / 2.0) @ _rz(p[1])
    if name == "U3":
        return _rz(p[1]) @ _ry(p[0]) @ _rz(p[2])
    raise ValueError(f"Unsupported single-qubit op: {name}")


def qft_matrix_without_swaps(m: int) -> np.ndarray:
    """Dense QFT on m qubits without the final bit-reversal swaps, the
    independent golden of src/tests/mlxQQmlQftSubsetTest.py:41-46:
    rows of the DFT matrix e^{+2 pi i x k / 2^m} / sqrt(2^m) taken in
    bit-reversed order."""
    size = 1 << m
    idx = np.arange(size)
    fourier = np.exp(2j * np.pi * np.outer(idx, idx) / size) / math.sqrt(size)
    rev = [int(format(i, f"0{m}b")[::-1], 2) if m > 0 else 0 for i in range(size)]
    return fourier[rev, :]


# --------------------------------------------------------------------------
# GF(2) affine composition -- shaders/xor_affine.py:46-76
# --------------------------------------------------------------------------
def compose_inverse_affine(ops: Iterable[dict], n: int) -> Tuple[List[int], int]:
    """Compose a CNOT/X/SWAP run into inverse rows (qubit k = row k) and a
    packed flip ``c`` such that the source of output index y has qubit-k bit
    parity(rows[k] & y) XOR bit_k(c); replays the run in reverse onto the
    identity map (xor_affine.py:46-76)."""
    rows = [1 << (n - 1 - k) for k in range(n)]
    c = 0
    for op in reversed(list(ops)):
        name = str(op.get("name", "")).upper()
        w = list(op.get("wires", []))
        if name == "X":
            c ^= 1 << (n - 1 - w[0])
        elif name in ("CNOT", "CX"):
            a, b = w
            rows[b] ^= rows[a]
            if (c >> (n - 1 - a)) & 1:
                c ^= 1 << (n - 1 - b)
        elif name == "SWAP":
            a, b = w
            rows[a], rows[b] = rows[b], rows[a]
            if ((c >> (n - 1 - a)) & 1) != ((c >> (n - 1 - b)) & 1):
                c ^= (1 << (n - 1 - a)) | (1 << (n - 1 - b))
        else:
            raise ValueError(f"Not a GF(2) affine gate: {name}")
    return rows, c


def affine_sources(n: int, rows: Sequence[int], c: int) -> np.ndarray:
    """src[y] = sum_k parity(rows[k] & y) << (n-1-k) XOR c for every y
    (the index map of xor_affine.py:22-32), vectorised with uint64."""
    y = np.arange(1 << n, dtype=np.uint64)
    src = np.zeros_like(y)
    for k, r in enumerate(rows):
        par = np.bitwise_and(y, np.uint64(r))
        # parity by folding
        for sh in (32, 16, 8, 4, 2, 1):
            par ^= par >> np.uint64(sh)
        src |= (par & np.uint64(1)) << np.uint64(n - 1 - k)
    return src ^ np.uint64(c)


# --------------------------------------------------------------------------
# State engine -- sim.py:17-343, 466-563
# --------------------------------------------------------------------------
class OracleSim:
    """Per-gate statevector simulator with the reference's semantics."""

    def __init__(self, n: int, dtype=np.complex64):
        if int(n) <= 0:
            raise ValueError("n_qubits must be positive")
        self.n = int(n)
        self.dtype = np.dtype(dtype)
        self.rdtype = np.float32 if self.dtype == np.complex64 else np.float64
        self.reset()

    # sim.py:32-45
    def reset(self) -> None:
        self.state = np.zeros(1 << self.n, dtype=self.dtype)
        self.state[0] = 1.0

    def set_state(self, vec) -> None:
        v = np.asarray(vec, dtype=self.dtype).reshape(-1)
        if v.size != (1 << self.n):
            raise ValueError("state has the wrong length")
        self.state = v.copy()

    def _check(self, q: int) -> int:
        if not (0 <= q < self.n):
            raise ValueError("Qubit index out of range")
        return q

    # sim.py:75-87
    def apply_single(self, u: np.ndarray, q: int) -> None:
        q = self._check(q)
        u = np.asarray(u).astype(self.dtype)
        t = self.state.reshape(1 << q, 2, 1 << (self.n - q - 1))
        s0, s1 = t[:, 0, :], t[:, 1, :]
        n0 = u[0, 0] * s0 + u[0, 1] * s1
        n1 = u[1, 0] * s0 + u[1, 1] * s1
        self.state = np.stack([n0, n1], axis=1).reshape(-1)

    # sim.py:94-138 (general-k broadcast form)
    def apply_diagonal(self, diag, qubits: Sequence[int]) -> None:
        qs = [self._check(q) for q in qubits]
        k = len(qs)
        if k == 0:
            return
        if len(set(qs)) != k:
            raise ValueError("Duplicate qubit indices")
        d = np.asarray(diag).astype(self.dtype).reshape([2] * k)
        order = sorted(range(k), key=lambda i: qs[i])
        d = np.transpose(d, order)
        shape = [1] * self.n
        for q in qs:
            shape[q] = 2
        self.state = (self.state.reshape([2] * self.n) * d.reshape(shape)).reshape(-1)

    # sim.py:47-73
    def apply_dense_gate(self, gate: np.ndarray, qubits: Sequence[int]) -> None:
        qs = [self._check(q) for q in qubits]
        k = len(qs)
        gate = np.asarray(gate).astype(self.dtype)
        if gate.shape != (1 << k, 1 << k):
            raise ValueError("Gate dimension does not match target qubits")
        perm = [i for i in range(self.n) if i not in qs] + qs
        inv = np.argsort(perm)
        t = self.state.reshape([2] * self.n).transpose(perm).reshape(-1, 1 << k)
        t = (t @ gate.T).reshape([2] * self.n).transpose(inv)
        self.state = np.ascontiguousarray(t).reshape(-1)

    # sim.py:140-173
    def apply_controlled_single(self, u: np.ndarray, c: int, t: int) -> None:
        if c == t:
            raise ValueError("Control and target must differ")
        self._check(c), self._check(t)
        u = np.asarray(u).astype(self.dtype)
        ten = self.state.reshape([2] * self.n).copy()
        sel0 = [slice(None)] * self.n
        sel1 = [slice(None)] * self.n
        sel0[c] = 1
        sel1[c] = 1
        sel0[t] = 0
        sel1[t] = 1
        a0 = ten[tuple(sel0)].copy()
        a1 = ten[tuple(sel1)].copy()
        ten[tuple(sel0)] = u[0, 0] * a0 + u[0, 1] * a1
        ten[tuple(sel1)] = u[1, 0] * a0 + u[1, 1] * a1
        self.state = ten.reshape(-1)

    # sim.py:185-213
    def apply_multi_controlled_single(self, u, controls: Sequence[int], target: int) -> None:
        cs = list(controls)
        if target in cs or len(set(cs)) != len(cs):
            raise ValueError("Control/target wires must be distinct")
        u = np.asarray(u).astype(self.dtype)
        ten = self.state.reshape([2] * self.n).copy()
        sel0 = [slice(None)] * self.n
        for c in cs:
            sel0[c] = 1
        sel1 = list(sel0)
        sel0[target] = 0
        sel1[target] = 1
        a0 = ten[tuple(sel0)].copy()
        a1 = ten[tuple(sel1)].copy()
        ten[tuple(sel0)] = u[0, 0] * a0 + u[0, 1] * a1
        ten[tuple(sel1)] = u[1, 0] * a0 + u[1, 1] * a1
        self.state = ten.reshape(-1)

    # sim.py:215-224
    def apply_swap_wires(self, a: int, b: int) -> None:
        if a == b:
            return
        perm = list(range(self.n))
        perm[a], perm[b] = perm[b], perm[a]
        self.state = np.ascontiguousarray(self.state.reshape([2] * self.n).transpose(perm)).reshape(-1)

    # sim.py:203-213
    def apply_controlled_swap(self, c: int, a: int, b: int) -> None:
        if len({c, a, b}) != 3:
            raise ValueError("Control/target wires must be distinct")
        ten = self.state.reshape([2] * self.n).copy()
        s01 = [slice(None)] * self.n
        s10 = [slice(None)] * self.n
        s01[c] = s10[c] = 1
        s01[a], s01[b] = 0, 1
        s10[a], s10[b] = 1, 0
        x = ten[tuple(s01)].copy()
        ten[tuple(s01)] = ten[tuple(s10)]
        ten[tuple(s10)] = x
        self.state = ten.reshape(-1)

    # sim.py:226-258: exp(-i theta P(x)P) for P in {X, Y}
    def _antidiag_phase(self, theta: float, a: int, b: int, signs) -> None:
        cth = math.cos(theta)
        msth = complex(0.0, -math.sin(theta))
        ten = self.state.reshape([2] * self.n)
        out = np.empty_like(ten)
        g = dict(zip(((0, 0), (0, 1), (1, 0), (1, 1)), signs))
        for (ba, bb) in g:
            dst = [slice(None)] * self.n
            src = [slice(None)] * self.n
            dst[a], dst[b] = ba, bb
            src[a], src[b] = 1 - ba, 1 - bb
            out[tuple(dst)] = cth * ten[tuple(dst)] + msth * g[(ba, bb)] * ten[tuple(src)]
        self.state = out.reshape(-1)

    def apply_xx_phase(self, theta: float, a: int, b: int) -> None:
        self._antidiag_phase(theta, a, b, (1.0, 1.0, 1.0, 1.0))

    def apply_yy_phase(self, theta: float, a: int, b: int) -> None:
        self._antidiag_phase(theta, a, b, (-1.0, 1.0, 1.0, -1.0))

    # sim.py:260-264: exp(-i theta Z(x)Z), no factor 1/2
    def apply_zz_phase(self, theta: float, a: int, b: int) -> None:
        em = complex(math.cos(theta), -math.sin(theta))
        ep = complex(math.cos(theta), math.sin(theta))
        self.apply_diagonal([em, ep, ep, em], [a, b])

    def apply_global_phase(self, phase: float) -> None:
        """integrations/_common.py:231-238: scalar multiply."""
        if phase:
            self.state = self.state * self.dtype.type(complex(math.cos(phase), math.sin(phase)))

    def apply_affine(self, rows: Sequence[int], c: int) -> None:
        """out[y] = state[src(y)] (xor_affine.py:22-32)."""
        src = affine_sources(self.n, rows, c)
        self.state = self.state[src.astype(np.int64)]

    # sim.py:485-510 / 522-563
    def _phase_ladder(self, wires: List[int], j: int, sign: float) -> None:
        m = len(wires)
        if j + 1 >= m:
            return
        ten = self.state.reshape([2] * self.n)
        factor = np.ones([1] * self.n, dtype=self.dtype)
        for k in range(j + 1, m):
            phi = sign * math.pi / (2 ** (k - j))
            v = np.array([1.0, complex(math.cos(phi), math.sin(phi))], dtype=self.dtype)
            shape = [1] * self.n
            shape[wires[k]] = 2
            factor = factor * v.reshape(shape)
        shape = [1] * self.n
        shape[wires[j]] = 2
        bit_j = np.array([0, 1], dtype=self.dtype).reshape(shape)
        one_j = np.array([1, 0], dtype=self.dtype).reshape(shape)
        self.state = (ten * (one_j + bit_j * factor)).reshape(-1)

    def _qft_wires(self, wires) -> List[int]:
        w = list(wires)
        if len(set(w)) != len(w):
            raise ValueError("Duplicate QFT wire indices")
        for q in w:
            self._check(q)
        return w

    def qft(self, wires: Optional[Sequence[int]] = None) -> None:
        """Ordered-wire QFT without terminal swaps (sim.py:522-546)."""
        w = self._qft_wires(range(self.n) if wires is None else wires)
        h = gate_matrix("H")
        for j in range(len(w)):
            self.apply_single(h, w[j])
            self._phase_ladder(w, j, 1.0)

    def iqft(self, wires: Optional[Sequence[int]] = None) -> None:
        """Exact inverse of :meth:`qft` (sim.py:549-563)."""
        w = self._qft_wires(range(self.n) if wires is None else wires)
        h = gate_matrix("H")
        for j in reversed(range(len(w))):
            self._phase_ladder(w, j, -1.0)
            self.apply_single(h, w[j])

    # sim.py:322-343
    def probabilities(self, wires: Optional[Sequence[int]] = None) -> np.ndarray:
        amp2 = (np.abs(self.state) ** 2).astype(self.rdtype)
        if wires is None:
            return amp2
        sel = list(wires)
        if len(set(sel)) != len(sel):
            raise ValueError("Duplicate qubit indices")
        for q in sel:
            self._check(q)
        rest = [q for q in range(self.n) if q not in sel]
        perm = sel + rest
        t = amp2.reshape([2] * self.n).transpose(perm).reshape(1 << len(sel), -1)
        return t.sum(axis=1)

    # integrations/_common.py:351-381: <psi| P |psi> for one Pauli word
    def pauli_expectation(self, word: dict) -> complex:
        paulis = {"X": gate_matrix("X"), "Y": gate_matrix("Y"), "Z": gate_matrix("Z")}
        acted = OracleSim.__new__(OracleSim)
        acted.n, acted.dtype, acted.rdtype = self.n, self.dtype, self.rdtype
        acted.state = self.state.copy()
        for w, p in word.items():
            p = str(p).upper()
            if p == "I":
                continue
            acted.apply_single(paulis[p], int(w))
        return complex(np.sum(np.conj(self.state).astype(np.complex128) * acted.state.astype(np.complex128)))

    # ------------------------------------------------------------------
    # device.py:1138-1290 (per-gate dispatch of the pure-MLX path)
    # ------------------------------------------------------------------
    def apply_op(self, op: dict) -> None:
        name = str(op.get("name", "")).upper()
        wires = [int(w) for w in op.get("wires", [])]
        params = [float(p) for p in op.get("parameters", []) or []]
        name = {"SDAG": "SDG", "TDAG": "TDG", "CX": "CNOT", "CP": "CPHASE",
                "CCX": "TOFFOLI", "CSWAP": "FREDKIN"}.get(name, name)
        if len(wires) == 1:
            q = wires[0]
            if name in ("Z", "S", "SDG", "T", "TDG", "RZ", "U1"):
                u = gate_matrix(name, params)
                self.apply_diagonal([u[0, 0], u[1, 1]], [q])
                return
            self.apply_single(gate_matrix(name, params), q)
            return
        if len(wires) == 2:
            c, t = wires
            if name == "CZ":
                self.apply_diagonal([1, 1, 1, -1], [c, t])
            elif name == "CPHASE":
                self.apply_diagonal([1, 1, 1, complex(math.cos(params[0]), math.sin(params[0]))], [c, t])
            elif name == "CRZ":
                rz = gate_matrix("RZ", params)
                self.apply_diagonal([1, 1, rz[0, 0], rz[1, 1]], [c, t])
            elif name == "CNOT":
                self.apply_controlled_single(gate_matrix("X"), c, t)
            elif name == "CH":
                self.apply_controlled_single(gate_matrix("H"), c, t)
            elif name == "CRX":
                self.apply_controlled_single(gate_matrix("RX", params), c, t)
            elif name == "CRY":
                self.apply_controlled_single(gate_matrix("RY", params), c, t)
            elif name == "SWAP":
                self.apply_swap_wires(c, t)
            elif name == "ISWAP":
                self.apply_diagonal([1, 1j, 1j, 1], [c, t])
                self.apply_swap_wires(c, t)
            elif name == "ZZPHASE":
                self.apply_zz_phase(params[0], c, t)
            elif name == "XXPHASE":
                self.apply_xx_phase(params[0], c, t)
            elif name == "YYPHASE":
                self.apply_yy_phase(params[0], c, t)
            else:
                raise ValueError(f"Unsupported two-qubit op: {name}")
            return
        if len(wires) == 3:
            if name == "TOFFOLI":
                self.apply_multi_controlled_single(gate_matrix("X"), wires[:2], wires[2])
            elif name == "FREDKIN":
                self.apply_controlled_swap(*wires)
            else:
                raise ValueError(f"Unsupported three-qubit op: {name}")
            return
        raise ValueError(f"Unsupported operation arity for: {name}")

    def execute(self, ops: Iterable[dict]) -> np.ndarray:
        for op in ops:
            self.apply_op(op)
        return self.state
