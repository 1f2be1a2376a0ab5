"""Adjoint-method gradients of Pauli-sum energies (differentiation direction).

The reference differentiates circuits by parameter shift, running the circuit
twice per parameter (integrations/qml.py:308-332; bench.py:1831-1841 times it
on the hardware-efficient ansatz).  Here one forward run prepares
``psi = U|0>``, one pass builds ``lam = H psi`` and the energy
``E = Re <psi|lam>``, and one backward run un-applies the circuit layer by
layer from the final state, so no intermediate state is stored:

    for each layer, last to first:
        psi, lam <- P^dag psi, P^dag lam               (the CNOT ladder)
        for the rotations of every qubit, last to first (exp(-i t G / 2)):
            dE/dt = Im <lam|G|psi>;  psi, lam <- R^dag psi, R^dag lam

The per-layer work is ``mq_adjoint_layer_xor_async`` (tile sweeps over both
states, mq_adjoint.cu; the ladder's un-apply is gathered by the layer's first
sweep as it loads its tiles), or ``mq_adjoint_layer`` after a separate
permutation pass when the gradients are read back per layer;
``AdjointEnergy`` exposes it as a ``torch.autograd.Function``.

Circuits: ``LayeredAnsatz`` = layers of per-qubit rotation sequences (RX / RY /
RZ, e.g. the RY+RZ hardware-efficient ansatz) followed by a CNOT ladder
0->1->...->n-1 (optional).  Observables: ``PauliSum`` = Z words plus
single-qubit X terms (Ising / transverse-field Hamiltonians such as
H = sum_i Z_i Z_{i+1} + 0.5 sum_i X_i).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .engine import StateVector
from .workloads import cnot_ladder_rows

GEN = {"RX": 1, "RY": 2, "RZ": 3}
_PAULI = {"RX": np.array([[0, 1], [1, 0]], dtype=np.complex128),
          "RY": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
          "RZ": np.array([[1, 0], [0, -1]], dtype=np.complex128)}


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def rotation(name: str, t: float) -> np.ndarray:
    """exp(-i t G / 2) for G = X, Y, Z (gates.py RX / RY / RZ)."""
    c, s = math.cos(t / 2.0), math.sin(t / 2.0)
    if name == "RX":
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)
    if name == "RY":
        return np.array([[c, -s], [s, c]], dtype=np.complex128)
    if name == "RZ":
        return np.array([[np.exp(-0.5j * t), 0], [0, np.exp(0.5j * t)]], dtype=np.complex128)
    raise ValueError(f"rotation must be RX, RY or RZ, not {name}")


def rotations(name: str, t: np.ndarray) -> np.ndarray:
    """exp(-i t G / 2) for an array of angles: (len(t), 4) [u00, u01, u10, u11]."""
    t = np.asarray(t, dtype=np.float64)
    c, s = np.cos(t / 2.0), np.sin(t / 2.0)
    out = np.zeros((t.size, 4), dtype=np.complex128)
    if name == "RX":
        out[:, 0] = out[:, 3] = c
        out[:, 1] = out[:, 2] = -1j * s
    elif name == "RY":
        out[:, 0] = out[:, 3] = c
        out[:, 1], out[:, 2] = -s, s
    elif name == "RZ":
        out[:, 0], out[:, 3] = np.exp(-0.5j * t), np.exp(0.5j * t)
    else:
        raise ValueError(f"rotation must be RX, RY or RZ, not {name}")
    return out


def _dagger(m: np.ndarray) -> np.ndarray:
    """Conjugate transpose of (k, 4) row-major 2x2 matrices."""
    return np.conj(m[:, [0, 2, 1, 3]])


@dataclass
class PauliSum:
    """H = sum_w c_w prod_{q in w} Z_q + sum_q x_q X_q."""
    n: int
    zwords: List[Tuple[Tuple[int, ...], float]] = field(default_factory=list)
    xcoef: Optional[np.ndarray] = None

    @staticmethod
    def ising_chain(n: int, j: float = 1.0, h: float = 0.5) -> "PauliSum":
        """sum_{i<n-1} j Z_i Z_{i+1} + sum_i h X_i (the differentiation
        benchmark's observable)."""
        return PauliSum(n, [((i, i + 1), j) for i in range(n - 1)], np.full(n, h, dtype=np.float64))

    def arrays(self):
        zm = np.array([sum(1 << (self.n - 1 - q) for q in w) for w, _ in self.zwords], dtype=np.uint64)
        zc = np.array([c for _, c in self.zwords], dtype=np.float64)
        xc = None if self.xcoef is None else np.ascontiguousarray(self.xcoef, dtype=np.float64)
        return zm, zc, xc

    def words(self) -> List[Tuple[Dict[int, str], float]]:
        """(Pauli word, coefficient) pairs, for expectation-value checks."""
        out = [({q: "Z" for q in w}, c) for w, c in self.zwords]
        if self.xcoef is not None:
            out += [({q: "X"}, float(c)) for q, c in enumerate(self.xcoef) if c != 0.0]
        return out


@dataclass
class LayeredAnsatz:
    """``layers`` repetitions of: rotations ``rots`` (applied in that order) on
    every qubit, then a CNOT ladder 0->1->...->n-1 when ``ladder``.
    Parameters have shape (layers, n, len(rots))."""
    n: int
    layers: int
    rots: Tuple[str, ...] = ("RY", "RZ")
    ladder: bool = True

    @property
    def shape(self) -> Tuple[int, int, int]:
        return (self.layers, self.n, len(self.rots))

    def layer_mats(self, p: np.ndarray) -> np.ndarray:
        """(n, 4) products R_last ... R_first of one layer's rotations."""
        u = np.tile(np.eye(2, dtype=np.complex128).reshape(1, 2, 2), (self.n, 1, 1))
        for k, name in enumerate(self.rots):
            u = rotations(name, p[:, k]).reshape(self.n, 2, 2) @ u
        return u.reshape(self.n, 4)

    def generator_coefficients(self, p: np.ndarray) -> np.ndarray:
        """(n, K, 3): for rotation k of every qubit, the real (a, b, c) with
        V G_k V^dag = aX + bY + cZ, V = R_{K-1} ... R_{k+1} (the rotations
        after it in the layer), so that dE/dt_k = a Im<lam|X|psi> +
        b Im<lam|Y|psi> + c Im<lam|Z|psi> at the point after the layer's
        rotations."""
        K = len(self.rots)
        out = np.zeros((self.n, K, 3), dtype=np.float64)
        V = np.tile(np.eye(2, dtype=np.complex128).reshape(1, 2, 2), (self.n, 1, 1))
        for k in reversed(range(K)):
            G = _PAULI[self.rots[k]]
            Gp = V @ G @ np.conj(np.transpose(V, (0, 2, 1)))
            for j, P in enumerate((_PAULI["RX"], _PAULI["RY"], _PAULI["RZ"])):
                out[:, k, j] = 0.5 * np.real(np.einsum("qab,ba->q", Gp, P))
            V = V @ rotations(self.rots[k], p[:, k]).reshape(self.n, 2, 2)
        return out

    def ops(self, params: np.ndarray) -> List[dict]:
        """The circuit as op dicts (for the oracle and the parameter-shift
        reference)."""
        params = np.asarray(params, dtype=np.float64).reshape(self.shape)
        out = []
        for l in range(self.layers):
            for k, name in enumerate(self.rots):
                for q in range(self.n):
                    out.append({"name": name, "wires": [q], "parameters": [float(params[l, q, k])]})
            if self.ladder:
                for q in range(self.n - 1):
                    out.append({"name": "CNOT", "wires": [q, q + 1], "parameters": []})
        return out

    def forward(self, sv: StateVector, params: np.ndarray) -> None:
        """|0> -> U(params)|0> on ``sv``: one fused layer call per layer (the
        rotation product on every qubit, with the ladder on its last sweep)."""
        params = np.asarray(params, dtype=np.float64).reshape(self.shape)
        sv.reset()
        rows, c = cnot_ladder_rows(self.n) if self.ladder else (None, 0)
        for l in range(self.layers):
            sv.apply_layer(self.layer_mats(params[l]), None, [], rows, c)


def _ladder_inverse_rows(n: int) -> Tuple[List[int], int]:
    """Inverse rows of the inverse ladder CNOT(n-2,n-1), ..., CNOT(0,1):
    out[y] = in[f(y)] with f the ladder's forward map (bit k of f(y) = XOR of
    qubits 0..k)."""
    rows = [0] * n
    acc = 0
    for k in range(n):
        acc |= 1 << (n - 1 - k)
        rows[k] = acc
    return rows, 0


class AdjointEngine:
    """Owns the two device states (psi, lam) of one (ansatz, observable)."""

    def __init__(self, ansatz: LayeredAnsatz, ham: PauliSum, dtype="complex64", device: int = 0,
                 stream: Optional[int] = None):
        if ham.n != ansatz.n:
            raise ValueError("observable and ansatz act on different qubit counts")
        for name in ansatz.rots:
            if name not in GEN:
                raise ValueError(f"rotation must be RX, RY or RZ, not {name}")
        self.ansatz, self.ham = ansatz, ham
        self.psi = StateVector(ansatz.n, dtype=dtype, device=device, stream=stream)
        self.lam = StateVector(ansatz.n, dtype=dtype, device=device, stream=self.psi.stream)
        self._lib = N.lib()
        self._zm, self._zc, self._xc = ham.arrays()

    def close(self) -> None:
        # lam borrows psi's stream: release it first
        self.lam.close()
        self.psi.close()

    def _pauli_sum(self) -> float:
        e = C.c_double()
        zm, zc, xc = self._zm, self._zc, self._xc
        N.check(self._lib.mq_apply_pauli_sum(self.psi.handle, self.lam.handle, int(zm.size),
                                             _ptr(zm) if zm.size else None, _ptr(zc) if zc.size else None,
                                             _ptr(xc) if xc is not None else None, C.byref(e)))
        return float(e.value)

    def energy(self, params: np.ndarray) -> float:
        """E = <psi|H|psi> (forward run + observable; leaves psi, lam = H psi)."""
        self.ansatz.forward(self.psi, params)
        return self._pauli_sum()

    def energy_and_grad(self, params: np.ndarray) -> Tuple[float, np.ndarray]:
        e = self.energy(params)
        return e, self.backward(params)

    def backward(self, params: np.ndarray) -> np.ndarray:
        """dE/dparams by the adjoint sweeps; psi and lam must be the states
        that ``energy(params)`` left (psi = U|0>, lam = H psi).  Un-applies
        the circuit from both states, one ``mq_adjoint_layer`` call per layer
        (the per-qubit rotation product at once); the transition values of
        every layer go to one device buffer, read back once."""
        A = self.ansatz
        params = np.asarray(params, dtype=np.float64).reshape(A.shape)
        n, L = A.n, A.layers
        inv_rows, inv_c = _ladder_inverse_rows(n)
        rows = np.ascontiguousarray(np.asarray(inv_rows, dtype=np.uint64))
        qubits = np.arange(n, dtype=np.int32)
        dev = self._grad_buffer(L * 3 * n)
        trans = np.zeros((L, n, 3), dtype=np.float64)
        for i, l in enumerate(reversed(range(L))):
            m = np.ascontiguousarray(_dagger(A.layer_mats(params[l]))).view(np.float64)
            if dev is not None:
                # the ladder's un-apply rides on the layer's first sweep
                out = C.c_void_p(dev.data_ptr() + i * 3 * n * 8)
                if A.ladder:
                    N.check(self._lib.mq_adjoint_layer_xor_async(self.psi.handle, self.lam.handle, _ptr(rows),
                                                                 int(inv_c), n, _ptr(qubits), _ptr(m), out))
                else:
                    N.check(self._lib.mq_adjoint_layer_async(self.psi.handle, self.lam.handle, n, _ptr(qubits),
                                                             _ptr(m), out))
            else:
                if A.ladder:
                    self.psi.apply_xor_affine(inv_rows, inv_c)
                    self.lam.apply_xor_affine(inv_rows, inv_c)
                t = np.zeros(3 * n, dtype=np.float64)
                N.check(self._lib.mq_adjoint_layer(self.psi.handle, self.lam.handle, n, _ptr(qubits), _ptr(m),
                                                   _ptr(t)))
                trans[i] = t.reshape(n, 3)
        if dev is not None:
            self.psi.synchronize()
            trans = dev[: L * 3 * n].cpu().numpy().reshape(L, n, 3)
        grad = np.zeros(A.shape, dtype=np.float64)
        for i, l in enumerate(reversed(range(L))):
            coef = A.generator_coefficients(params[l])          # (n, K, 3)
            grad[l] = np.einsum("qkp,qp->qk", coef, trans[i])
        return grad

    def _grad_buffer(self, count: int):
        """Device buffer of ``count`` doubles (torch plumbing), or None."""
        try:
            import torch
        except ImportError:  # pragma: no cover
            return None
        buf = getattr(self, "_gbuf", None)
        if buf is None or buf.numel() < count:
            buf = torch.empty(count, dtype=torch.float64, device=f"cuda:{self.psi.device}")
            self._gbuf = buf
        return buf


def parameter_shift_grad(energy_fn, params: np.ndarray) -> np.ndarray:
    """The reference's gradient rule for exp(-i t G/2) rotations:
    dE/dt = (E(t + pi/2) - E(t - pi/2)) / 2 per parameter (qml.py:308-332)."""
    p = np.array(params, dtype=np.float64)
    flat = p.reshape(-1)
    g = np.zeros_like(flat)
    for i in range(flat.size):
        old = flat[i]
        flat[i] = old + math.pi / 2
        ep = energy_fn(p)
        flat[i] = old - math.pi / 2
        em = energy_fn(p)
        flat[i] = old
        g[i] = 0.5 * (ep - em)
    return g.reshape(p.shape)


try:  # torch is plumbing here: the autograd binding only
    import torch

    class AdjointEnergy(torch.autograd.Function):
        """E(params) with its adjoint-method gradient: ``forward`` runs the
        circuit and the observable on the device, ``backward`` the adjoint
        sweeps.  Use as ``AdjointEnergy.apply(params, engine)``."""

        @staticmethod
        def forward(ctx, params, engine: AdjointEngine):
            p = params.detach().to("cpu", torch.float64).numpy().copy()
            e = engine.energy(p)
            engine._forward_params = p
            ctx.engine, ctx.p = engine, p
            ctx.dtype, ctx.device = params.dtype, params.device
            return params.new_tensor(e)

        @staticmethod
        def backward(ctx, grad_out):
            engine, p = ctx.engine, ctx.p
            # another forward may have moved the device states since
            if getattr(engine, "_forward_params", None) is not p:
                engine.energy(p)
            engine._forward_params = None
            g = engine.backward(p)
            return grad_out * torch.as_tensor(g, dtype=ctx.dtype, device=ctx.device), None
except ImportError:  # pragma: no cover
    AdjointEnergy = None
