"""Kernel-level statevector API over libmq (the layer calls of the hot path).

``StateVector`` owns one device state (a C-ABI ``mq_state`` handle).  Its
methods are the B200 counterparts of the reference's Metal layer API
(shaders/__init__.py:26-56: u2_list_layer_all, diag_weighted_layer,
zz_weighted_layer, qft_stage_all / qft_stage_sub, xor_affine_gather) and of
``StateVectorSimulator.probabilities_array`` / ``sample_array``
(sim.py:322-419).  Every call goes to CUDA; nothing here computes on the host
beyond argument packing.

Conventions: qubit q is index bit n-1-q (MSB-first, sim.py:10-14).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N

_DTYPES = {"complex64": N.MQ_C64, "complex128": N.MQ_C128, np.complex64: N.MQ_C64, np.complex128: N.MQ_C128}


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _mats_array(n: int, mats) -> np.ndarray:
    m = np.asarray(mats, dtype=np.complex128).reshape(n, 4)
    out = np.empty((n, 8), dtype=np.float64)
    out[:, 0::2] = m.real
    out[:, 1::2] = m.imag
    return np.ascontiguousarray(out)


def _pack_terms(terms):
    """Diagonal terms (kind, wire_a, wire_b, params) as the C arrays
    kinds[k], wires[2k], params[8k]; (None, None, None) when empty."""
    k = len(terms)
    if k == 0:
        return None, None, None
    kinds = np.empty(k, dtype=np.int32)
    wires = np.empty(2 * k, dtype=np.int32)
    params = np.zeros((k, 8), dtype=np.float64)
    for i, (kind, a, b, p) in enumerate(terms):
        kinds[i] = int(kind)
        wires[2 * i] = int(a)
        wires[2 * i + 1] = int(b)
        pp = list(p)
        params[i, :len(pp)] = pp
    return kinds, wires, params


def pauli_masks(n: int, word: Dict[int, str]) -> Tuple[int, int, int]:
    """(xmask, zmask, ny) over index bits for a Pauli word {wire: 'X'|'Y'|'Z'|'I'}."""
    x = z = ny = 0
    for w, p in word.items():
        w = int(w)
        p = str(p).upper()
        if not (0 <= w < n):
            raise ValueError("Observable wire is outside the device")
        bit = 1 << (n - 1 - w)
        if p == "I":
            continue
        if p == "X":
            x |= bit
        elif p == "Z":
            z |= bit
        elif p == "Y":
            x |= bit
            z |= bit
            ny += 1
        else:
            raise ValueError("Pauli products support only I, X, Y, and Z")
    return x, z, ny


class DeviceState:
    """The ``state`` attribute of a ``StateVector``: a handle on the resident
    device state, standing where the reference keeps its MLX array
    (``StateVectorSimulator.state``, sim.py:32-45).

    It supports exactly what the reference's SDK helpers do with that array
    (integrations/_common.py:231-253): ``np.asarray(state, dtype)`` reads the
    amplitudes back to the host, and ``sim.state = sim.state * factor``
    multiplies the resident state by a complex scalar on the GPU (the
    product is a deferred ``ScaledState`` that the setter applies), so
    ``apply_global_phase`` never moves the state to the host."""

    __array_priority__ = 1000  # numpy scalars on the left defer to __rmul__

    def __init__(self, sv: "StateVector"):
        self._sv = sv

    @property
    def shape(self) -> Tuple[int]:
        return (1 << self._sv.n,)

    @property
    def dtype(self) -> np.dtype:
        return self._sv.dtype

    def __len__(self) -> int:
        return 1 << self._sv.n

    def __array__(self, dtype=None, copy=None):
        out = self._sv.get()
        return out if dtype is None else out.astype(dtype, copy=False)

    def __mul__(self, factor) -> "ScaledState":
        return ScaledState(self._sv, complex(factor))

    __rmul__ = __mul__


class ScaledState:
    """``factor`` times a resident state, not yet applied: assigning it to
    the same simulator's ``state`` multiplies the state on the GPU; reading
    it with ``np.asarray`` gives the scaled amplitudes without changing the
    resident state."""

    __array_priority__ = 1000

    def __init__(self, sv: "StateVector", factor: complex):
        self._sv = sv
        self.factor = complex(factor)

    def __mul__(self, other) -> "ScaledState":
        return ScaledState(self._sv, self.factor * complex(other))

    __rmul__ = __mul__

    def __array__(self, dtype=None, copy=None):
        out = (self._sv.get() * self._sv.dtype.type(self.factor)).astype(self._sv.dtype)
        return out if dtype is None else out.astype(dtype, copy=False)


class StateVector:
    """One statevector resident in device memory (one CUDA stream)."""

    def __init__(self, n: int, dtype="complex64", device: int = 0, stream: Optional[int] = None):
        self.n = int(n)
        if self.n <= 0:
            raise ValueError("n_qubits must be positive")
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.complex64, np.complex128):
            raise ValueError("dtype must be complex64 or complex128")
        self._dt = N.MQ_C64 if self.dtype == np.complex64 else N.MQ_C128
        self.device = int(device)
        lib = N.lib()
        h = C.c_void_p()
        N.check(lib.mq_state_create(self.n, self._dt, self.device, C.c_void_p(stream or 0), C.byref(h)))
        self._h = h
        self._lib = lib
        # host->device parameter bytes handed to kernels (end-to-end accounting)
        self.param_bytes = 0

    # -- lifetime -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mq_state_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- state ----------------------------------------------------------
    def reset(self) -> None:
        N.check(self._lib.mq_state_reset(self._h))

    def set(self, vec) -> None:
        v = np.ascontiguousarray(np.asarray(vec, dtype=self.dtype).reshape(-1))
        if v.size != (1 << self.n):
            raise ValueError("state has the wrong length")
        N.check(self._lib.mq_state_set(self._h, _ptr(v)))

    def get(self) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=self.dtype)
        N.check(self._lib.mq_state_get(self._h, _ptr(out)))
        return out

    def copy_from(self, other: "StateVector") -> None:
        N.check(self._lib.mq_state_copy(self._h, other._h))

    # -- the reference simulator's state attribute (sim.py:32-45) -------------
    @property
    def state(self) -> DeviceState:
        """The resident state (see ``DeviceState``)."""
        return DeviceState(self)

    @state.setter
    def state(self, value) -> None:
        if isinstance(value, ScaledState) and value._sv is self:
            self.scale(value.factor)
        elif isinstance(value, DeviceState) and value._sv is self:
            return
        elif isinstance(value, (DeviceState, ScaledState)):
            if value._sv.n != self.n or value._sv.dtype != self.dtype:
                raise ValueError("state has the wrong length or dtype")
            self.copy_from(value._sv)
            if isinstance(value, ScaledState):
                self.scale(value.factor)
        else:
            self.set(value)

    def scale(self, factor: complex) -> None:
        """Multiply the resident state by a complex scalar (one diagonal pass,
        the same factor on both values of qubit 0)."""
        f = complex(factor)
        if f == 1.0:
            return
        self.apply_diag_terms([(N.MQ_DIAG_1Q, 0, -1, [f.real, f.imag, f.real, f.imag])])

    @property
    def stream(self) -> int:
        """cudaStream_t (as an integer) the handle launches on."""
        out = C.c_void_p()
        N.check(self._lib.mq_state_stream(self._h, C.byref(out)))
        return int(out.value or 0)

    def set_sm_limit(self, sms: int) -> None:
        """Launch grids for at most ``sms`` SMs (<= 0: all of them)."""
        N.check(self._lib.mq_state_set_sm_limit(self._h, int(sms)))

    def set_stream(self, stream: Optional[int]) -> None:
        N.check(self._lib.mq_state_set_stream(self._h, C.c_void_p(stream or 0)))

    def device_ptr(self) -> int:
        p = C.c_void_p()
        N.check(self._lib.mq_state_device_ptr(self._h, C.byref(p)))
        return int(p.value or 0)

    def synchronize(self) -> None:
        N.check(self._lib.mq_sync(self._h))

    def counters(self) -> Tuple[int, int]:
        a, b = C.c_uint64(), C.c_uint64()
        N.check(self._lib.mq_state_counters(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    # -- (a) single-qubit layers -------------------------------------
    def apply_u2_layer(self, mats, active: Optional[Iterable[int]] = None) -> None:
        """Per-qubit 2x2 unitaries (u2_list_layer_all, single_qubit.py:512-615).
        ``mats`` is (n, 4) [u00, u01, u10, u11]; ``active`` lists the qubits
        whose matrices are applied (None = all)."""
        m = _mats_array(self.n, mats)
        act = None
        if active is not None:
            act = np.zeros(self.n, dtype=np.uint8)
            for q in active:
                if not (0 <= int(q) < self.n):
                    raise ValueError("Qubit index out of range")
                act[int(q)] = 1
        self.param_bytes += m.nbytes + (act.nbytes if act is not None else 0)
        N.check(self._lib.mq_apply_u2_layer(self._h, _ptr(m), _ptr(act) if act is not None else None))

    def apply_u2_uniform(self, u2x2) -> None:
        """The same 2x2 on every qubit (u2_layer_all, single_qubit.py:422-509)."""
        m = _mats_array(1, u2x2).reshape(8)
        N.check(self._lib.mq_apply_u2_uniform(self._h, _ptr(m)))

    def apply_single(self, u, q: int) -> None:
        mats = np.tile(np.eye(2, dtype=np.complex128).reshape(1, 4), (self.n, 1))
        mats[int(q)] = np.asarray(u, dtype=np.complex128).reshape(4)
        self.apply_u2_layer(mats, [int(q)])

    def apply_controlled(self, gates: Sequence[Tuple[Sequence[int], int, np.ndarray]]) -> None:
        """Controlled 2x2 gates in order: (controls, target, matrix)."""
        if not gates:
            return
        targets = np.array([int(t) for _, t, _ in gates], dtype=np.int32)
        coff = np.zeros(len(gates) + 1, dtype=np.int32)
        ctl: List[int] = []
        for i, (cs, _, _) in enumerate(gates):
            ctl.extend(int(c) for c in cs)
            coff[i + 1] = len(ctl)
        controls = np.array(ctl if ctl else [0], dtype=np.int32)
        mats = _mats_array(len(gates), [np.asarray(u).reshape(4) for _, _, u in gates])
        self.param_bytes += targets.nbytes + coff.nbytes + controls.nbytes + mats.nbytes
        N.check(self._lib.mq_apply_controlled_u2(self._h, len(gates), _ptr(targets), _ptr(coff), _ptr(controls),
                                                 _ptr(mats)))

    # -- (b) diagonal layers -------------------------------------------
    def apply_diag_terms(self, terms: Sequence[Tuple[int, int, int, Sequence[float]]]) -> None:
        """Terms (kind, wire_a, wire_b, params) with kinds MQ_DIAG_*; all
        commute and are applied in one pass."""
        k = len(terms)
        if k == 0:
            return
        kinds, wires, params = _pack_terms(terms)
        self.param_bytes += kinds.nbytes + wires.nbytes + params.nbytes
        N.check(self._lib.mq_apply_diag_terms(self._h, k, _ptr(kinds), _ptr(wires), _ptr(params)))

    def apply_zz_weighted(self, bonds: Sequence[Tuple[int, int]], thetas: Sequence[float]) -> None:
        """exp(-i sum_b theta_b Z_a Z_b) (zz_weighted_layer, zz.py:99-140)."""
        self._diag_layer(N.MQ_DIAG_ZZ, bonds, thetas)

    def apply_cphase_weighted(self, bonds: Sequence[Tuple[int, int]], thetas: Sequence[float]) -> None:
        """CPHASE(theta_b) per bond, CZ = pi (diag_weighted_layer, diag.py:123-167)."""
        self._diag_layer(N.MQ_DIAG_CPHASE, bonds, thetas)

    def apply_pauli_pair_layer(self, kind: str, bonds: Sequence[Tuple[int, int]], thetas: Sequence[float]) -> None:
        """exp(-i sum_b theta_b P_a P_b) for P = X (kind "XX") or Y ("YY"),
        the native XXPHASE / YYPHASE without the 1/2 (xx_layer / yy_layer,
        shaders/pauli_pair.py:32-64).  The terms of one family commute, so
        with U = H (X = H Z H) or U = S H (Y = U Z U^+) the layer is U on the
        bonds' wires after the ZZ layer after U^+: one fused layer (the U^+
        sweeps carry the ZZ terms in their last register phase) and one U(2)
        layer."""
        bonds = [(int(a), int(b)) for a, b in bonds]
        thetas = [float(t) for t in thetas]
        if len(bonds) != len(thetas):
            raise ValueError("bonds/thetas length mismatch")
        if not bonds:
            return
        h = np.array([[1, 1], [1, -1]], dtype=np.complex128) / math.sqrt(2.0)
        if kind == "XX":
            u = h
        elif kind == "YY":
            u = np.array([[1, 0], [0, 1j]], dtype=np.complex128) @ h
        else:
            raise ValueError("kind must be 'XX' or 'YY'")
        wires = sorted({w for b in bonds for w in b})
        pre = np.tile(np.eye(2, dtype=np.complex128).reshape(1, 4), (self.n, 1))
        post = pre.copy()
        for w in wires:
            if not (0 <= w < self.n):
                raise ValueError("Qubit index out of range")
            pre[w] = u.conj().T.reshape(4)
            post[w] = u.reshape(4)
        self.apply_layer(pre, wires, [(N.MQ_DIAG_ZZ, a, b, [t]) for (a, b), t in zip(bonds, thetas)])
        self.apply_u2_layer(post, wires)

    def _diag_layer(self, kind: int, bonds, thetas) -> None:
        bonds = list(bonds)
        thetas = list(thetas)
        if len(bonds) != len(thetas):
            raise ValueError("bonds/thetas length mismatch")
        if not bonds:
            return
        b = np.ascontiguousarray(np.asarray(bonds, dtype=np.int32).reshape(-1))
        t = np.ascontiguousarray(np.asarray(thetas, dtype=np.float64))
        self.param_bytes += b.nbytes + t.nbytes
        N.check(self._lib.mq_apply_diag_layer(self._h, int(kind), len(bonds), _ptr(b), _ptr(t)))

    # -- (c) QFT ------------------------------------------------------------
    def apply_qft(self, wires: Optional[Sequence[int]] = None, inverse: bool = False) -> None:
        """Ordered-wire QFT without final swaps (sim.py:522-563)."""
        w = np.ascontiguousarray(np.asarray(list(range(self.n)) if wires is None else list(wires), dtype=np.int32))
        N.check(self._lib.mq_apply_qft(self._h, _ptr(w), int(w.size), 1 if inverse else 0))

    def apply_qft_stages(self, q0: int, k: int, j_begin: int, j_end: int, inverse: bool = False) -> None:
        N.check(self._lib.mq_apply_qft_stages(self._h, int(q0), int(k), int(j_begin), int(j_end), 1 if inverse else 0))

    # -- (d) GF(2) affine permutation ------------------------------------
    def apply_xor_affine(self, rows: Sequence[int], c: int) -> None:
        """out[y] = in[f^{-1}(y)] with inverse rows/c (xor_affine.py:79-116)."""
        r = np.ascontiguousarray(np.asarray([int(x) for x in rows], dtype=np.uint64))
        if r.size != self.n:
            raise ValueError("rows must have one mask per qubit")
        self.param_bytes += r.nbytes + 8
        N.check(self._lib.mq_apply_xor_affine(self._h, _ptr(r), int(c)))

    # -- fused layer ----------------------------------------------------------
    def pack_layer(self, mats=None, active: Optional[Iterable[int]] = None,
                   terms: Sequence[Tuple[int, int, int, Sequence[float]]] = (),
                   rows: Optional[Sequence[int]] = None, c: int = 0) -> tuple:
        """The C arrays of ``apply_layer`` (validated), for layers applied
        more than once or issued from a latency-sensitive loop."""
        m = act = None
        if mats is not None:
            m = _mats_array(self.n, mats)
            if active is not None:
                act = np.zeros(self.n, dtype=np.uint8)
                for q in active:
                    if not (0 <= int(q) < self.n):
                        raise ValueError("Qubit index out of range")
                    act[int(q)] = 1
        kinds, wires, params = _pack_terms(terms)
        r = None
        if rows is not None:
            r = np.ascontiguousarray(np.asarray([int(x) for x in rows], dtype=np.uint64))
            if r.size != self.n:
                raise ValueError("rows must have one mask per qubit")
        return (m, act, kinds, wires, params, r, int(c))

    def apply_packed_layer(self, packed: tuple) -> None:
        """``apply_layer`` from the arrays of ``pack_layer``."""
        m, act, kinds, wires, params, r, c = packed
        for a in (m, act, kinds, wires, params, r):
            if a is not None:
                self.param_bytes += a.nbytes
        N.check(self._lib.mq_apply_layer(
            self._h, _ptr(m) if m is not None else None, _ptr(act) if act is not None else None,
            0 if kinds is None else int(kinds.size), _ptr(kinds) if kinds is not None else None,
            _ptr(wires) if wires is not None else None, _ptr(params) if params is not None else None,
            _ptr(r) if r is not None else None, c))

    def apply_layer(self, mats=None, active: Optional[Iterable[int]] = None,
                    terms: Sequence[Tuple[int, int, int, Sequence[float]]] = (),
                    rows: Optional[Sequence[int]] = None, c: int = 0) -> None:
        """U(2) on the active qubits, then the commuting diagonal ``terms``,
        then the permutation out[y] = in[f^{-1}(y)] (inverse ``rows``/``c``),
        in the sweeps of the U(2) layer alone where the diagonal and the
        permutation allow it (one config-0 layer: u2_list_layer_all +
        zz_weighted_layer + xor_affine_gather, device.py:1089-1097)."""
        self.apply_packed_layer(self.pack_layer(mats, active, terms, rows, c))

    # -- (e) probabilities, sampling, expectations ------------------------
    def probabilities(self, wires: Optional[Sequence[int]] = None, dtype=np.float64) -> np.ndarray:
        """Full (wires=None) or marginal probabilities, first wire = MSB."""
        dt = np.dtype(dtype)
        if dt not in (np.float32, np.float64):
            raise ValueError("probabilities dtype must be float32 or float64")
        code = 0 if dt == np.float32 else 1
        if wires is None:
            out = np.empty(1 << self.n, dtype=dt)
            N.check(self._lib.mq_probabilities(self._h, None, -1, code, _ptr(out)))
            return out
        w = np.ascontiguousarray(np.asarray(list(wires), dtype=np.int32))
        out = np.empty(1 << w.size, dtype=dt)
        N.check(self._lib.mq_probabilities(self._h, _ptr(w) if w.size else _ptr(np.zeros(1, np.int32)),
                                           int(w.size), code, _ptr(out)))
        return out

    def probabilities_to_device(self, out_ptr: int, dtype=np.float32) -> None:
        """The full probability vector into device memory at ``out_ptr``
        (2^n entries of float32 or float64), asynchronously on the stream."""
        dt = np.dtype(dtype)
        if dt not in (np.float32, np.float64):
            raise ValueError("probabilities dtype must be float32 or float64")
        N.check(self._lib.mq_probabilities_device(self._h, 0 if dt == np.float32 else 1, C.c_void_p(int(out_ptr))))

    def sample_indices(self, shots: int, wires: Optional[Sequence[int]] = None, *, seed: int = 0,
                       stream_offset: int = 0) -> np.ndarray:
        shots = int(shots)
        if shots < 0:
            raise ValueError("shots must be non-negative")
        out = np.empty(max(shots, 1), dtype=np.int64)
        if wires is None:
            N.check(self._lib.mq_sample(self._h, None, -1, int(seed) & 0xFFFFFFFFFFFFFFFF, int(stream_offset),
                                        shots, _ptr(out)))
        else:
            w = np.ascontiguousarray(np.asarray(list(wires), dtype=np.int32))
            N.check(self._lib.mq_sample(self._h, _ptr(w) if w.size else _ptr(np.zeros(1, np.int32)), int(w.size),
                                        int(seed) & 0xFFFFFFFFFFFFFFFF, int(stream_offset), shots, _ptr(out)))
        return out[:shots]

    def sample_bits(self, shots: int, wires: Optional[Sequence[int]] = None, *, seed: int = 0,
                    stream_offset: int = 0) -> np.ndarray:
        """Shot bits (shots, k), first requested wire = MSB (sim.py:414-419)."""
        k = self.n if wires is None else len(list(wires))
        idx = self.sample_indices(shots, wires, seed=seed, stream_offset=stream_offset)
        shifts = np.arange(k - 1, -1, -1, dtype=np.int64)
        return ((idx[:, None] >> shifts) & 1).astype(np.int64)

    # -- the reference simulator's measurement surface (sim.py:322-430) ------
    def probabilities_array(self, wires: Optional[Sequence[int]] = None) -> np.ndarray:
        """Full (None) or marginal probabilities in the requested wire order,
        first wire = most significant bit, as float32 like the reference's
        |amplitude|^2 of a complex64 state (sim.py:322-343); an empty list
        gives [total probability].  Reduced on the GPU in float64."""
        if wires is not None:
            wires = [int(w) for w in wires]
        return self.probabilities(wires, dtype=np.float32)

    def sample_array(self, shots: int, wires: Optional[Sequence[int]] = None, *, rng=None) -> np.ndarray:
        """``shots`` samples of ``wires`` (None = all) as int64 bit rows, first
        wire = most significant (sim.py:383-419).  Draws one uint32 from
        ``rng`` (``np.random.default_rng()`` when None) exactly as the
        reference does (sim.py:405-408) and uses it as the key of the
        engine's Philox4x32-10 stream, so one generator state fixes the
        shots."""
        shots = int(shots)
        if shots < 0:
            raise ValueError("shots must be non-negative")
        rng = np.random.default_rng() if rng is None else rng
        seed = int(rng.integers(0, np.iinfo(np.uint32).max, dtype=np.uint32))
        return self.sample_bits(shots, None if wires is None else [int(w) for w in wires], seed=seed)

    def sample(self, shots: int, wires: Optional[Sequence[int]] = None, *, rng=None) -> List[List[int]]:
        """sim.py:421-422."""
        return self.sample_array(shots, wires, rng=rng).tolist()

    def sample_counts(self, shots: int, wires: Optional[Sequence[int]] = None, *, rng=None) -> Dict[str, int]:
        """Bit-string counts, first wire leftmost (sim.py:424-430)."""
        counts: Dict[str, int] = {}
        for bits in self.sample_array(shots, wires, rng=rng):
            key = "".join(str(int(b)) for b in bits)
            counts[key] = counts.get(key, 0) + 1
        return counts

    def expval_pauli(self, words: Sequence[Dict[int, str]]) -> np.ndarray:
        """<psi|P|psi> per Pauli word (pauli_product_expectations,
        integrations/_common.py:384-427), complex128 array."""
        k = len(words)
        if k == 0:
            return np.zeros(0, dtype=np.complex128)
        xs = np.empty(k, dtype=np.uint64)
        zs = np.empty(k, dtype=np.uint64)
        ny = np.empty(k, dtype=np.int32)
        for i, wd in enumerate(words):
            x, z, y = pauli_masks(self.n, wd)
            xs[i], zs[i], ny[i] = x, z, y
        out = np.empty(2 * k, dtype=np.float64)
        N.check(self._lib.mq_expval_pauli(self._h, k, _ptr(xs), _ptr(zs), _ptr(ny), _ptr(out)))
        return out[0::2] + 1j * out[1::2]
