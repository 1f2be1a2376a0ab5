"""Shared execution and measurement helpers for the SDK adapters.

Same surface as the reference's integrations/_common.py:86-479 for
method="statevector": ``core_operation`` validation, ``execute_operations``
with a per-width Device cache, global phase, state / marginal read-back,
seeded sampling, and Pauli expectations.  Every reduction runs on the GPU;
only results cross to the host.

Sampling consumes one uint32 from the caller's ``np.random.Generator``
exactly as the reference does (sim.py:405-408), and uses it as the key of the
engine's Philox4x32-10 stream, so one SDK seed fixes the counts.
"""
from __future__ import annotations

import math
from collections import Counter
from typing import Iterable, Optional, Sequence

import numpy as np

from ..device import Device
from ..fusion import ARITIES as _ARITIES, PARAMS as _PARAMETER_COUNTS

_ALIASES = {"CX": "CNOT", "CP": "CPHASE", "CCX": "TOFFOLI", "CSWAP": "FREDKIN"}

_PAULI = {
    "X": np.array([[0, 1], [1, 0]], dtype=np.complex128),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    "Z": np.array([[1, 0], [0, -1]], dtype=np.complex128),
    "I": np.eye(2, dtype=np.complex128),
}


def core_operation(name: str, wires: Iterable[int], parameters: Sequence[float] = ()) -> dict:
    """Build and validate one canonical operation (_common.py:86-115)."""
    cname = _ALIASES.get(str(name).upper(), str(name).upper())
    cw = [int(w) for w in wires]
    cp = [float(v) for v in parameters]
    if cname == "I":
        return {"name": "I", "wires": cw, "parameters": []}
    if cname not in _ARITIES:
        raise ValueError(f"Unsupported operation: {name}")
    if len(cw) != _ARITIES[cname]:
        raise ValueError(f"{cname} expects {_ARITIES[cname]} wire(s), got {len(cw)}")
    expected = _PARAMETER_COUNTS.get(cname, 0)
    if len(cp) != expected:
        raise ValueError(f"{cname} expects {expected} parameter(s), got {len(cp)}")
    return {"name": cname, "wires": cw, "parameters": cp}


def normalize_method(method: str) -> str:
    m = str(method).strip().lower().replace("-", "_")
    if m in ("automatic", "auto", "statevector", "sv"):
        return "statevector"
    if m in ("matrix_product_state", "mps"):
        raise NotImplementedError("method='matrix_product_state' stays on the reference's CPU path")
    raise ValueError(f"Unknown simulation method: {method}")


def execute_operations(
    n_qubits: int,
    operations: Sequence[dict],
    *,
    shots: int = 1000,
    report: bool = False,
    allow_unsafe_statevector: Optional[bool] = None,
    method: str = "automatic",
    execution_device: str = "auto",
    execution_cache: Optional[dict] = None,
    dtype: str = "complex64",
    **_ignored,
) -> Device:
    """Execute canonical operations on a (cached) Device (_common.py:118-228)."""
    normalize_method(method)
    key = (int(n_qubits), "sv", dtype)
    device = execution_cache.get(key) if execution_cache is not None else None
    if device is None:
        device = Device(int(n_qubits), shots=shots, allow_unsafe_statevector=allow_unsafe_statevector,
                        execution_device=None if execution_device in (None, "auto") else execution_device,
                        dtype=dtype)
        if execution_cache is not None:
            execution_cache[key] = device
    else:
        device.shots = int(shots)
        device.reset()
    device.execute(list(operations), report=report)
    device.execution_selection = {"selected_method": "statevector", "selected_device": "gpu",
                                  "reason": "explicit_statevector_request; cuda"}
    if device.last_execution_plan is not None:
        device.last_execution_plan["sdk_execution_selection"] = device.execution_selection
    return device


def apply_global_phase(device: Device, phase: float) -> None:
    """Scalar e^{i phase} on the resident state (_common.py:231-238)."""
    if phase:
        device.sim.apply_diag_terms([(5, -1, -1, [float(phase)])])


def statevector_numpy(device: Device) -> np.ndarray:
    device.synchronize()
    return device.sim.get()


def marginal_probabilities(device: Device, wires: Sequence[int]) -> np.ndarray:
    """Marginal over ``wires`` renormalised in float64 (_common.py:256-266)."""
    result = device.sim.probabilities(list(wires), dtype=np.float64)
    total = float(result.sum())
    if total <= 0.0:
        raise RuntimeError("Simulator returned a zero-probability state")
    return result / total


def draw_seed(rng: np.random.Generator) -> int:
    """One uint32 from the caller's generator (sim.py:405-408)."""
    return int(rng.integers(0, np.iinfo(np.uint32).max, dtype=np.uint32))


def sample_bits(device: Device, shots: int, wires: Sequence[int], rng: np.random.Generator) -> np.ndarray:
    """MSB-first bit rows for ``shots`` samples of ``wires`` (_common.py:269-288)."""
    wires = list(wires)
    if not wires:
        return np.empty((int(shots), 0), dtype=np.int64)
    seed = draw_seed(rng)
    return device.sim.sample_bits(int(shots), wires, seed=seed)


def bit_counts(samples: np.ndarray) -> dict:
    return dict(Counter("".join(str(int(b)) for b in row) for row in samples))


def pauli_product_expectations(device: Device, words: Sequence[dict]) -> list:
    """<psi|P|psi> per Pauli word, one GPU pass per X/Y support
    (_common.py:384-427)."""
    normalized = [{int(w): str(p).upper() for w, p in word.items() if str(p).upper() != "I"} for word in words]
    for word in normalized:
        if any(p not in ("X", "Y", "Z") for p in word.values()):
            raise ValueError("Pauli products support only I, X, Y, and Z")
    vals = device.sim.expval_pauli(normalized)
    return [complex(v) for v in vals]


def pauli_product_expectation(device: Device, paulis: dict) -> complex:
    return pauli_product_expectations(device, [paulis])[0]


def _pauli_decomposition(matrix: np.ndarray, k: int):
    """Coefficients c_P = tr(P M) / 2^k over the 4^k Pauli words on k wires."""
    import itertools
    coeffs = []
    for labels in itertools.product("IXYZ", repeat=k):
        p = np.array([[1.0 + 0j]])
        for lab in labels:
            p = np.kron(p, _PAULI[lab])
        c = np.trace(p @ matrix) / (1 << k)
        if abs(c) > 1e-14:
            coeffs.append((labels, c))
    return coeffs


def local_expectation(device: Device, wires: Sequence[int], matrix: np.ndarray) -> complex:
    """<psi| M_wires |psi> for a small dense M (_common.py:336-348), via its
    Pauli decomposition so the state stays on the GPU."""
    wires = [int(w) for w in wires]
    m = np.asarray(matrix, dtype=np.complex128)
    k = len(wires)
    if not wires:
        return complex(m.reshape(-1)[0])
    if len(set(wires)) != k:
        raise ValueError("Observable wires must be unique")
    if m.shape != (1 << k, 1 << k):
        raise ValueError(f"Observable matrix must have shape {(1 << k, 1 << k)}, got {m.shape}")
    terms = _pauli_decomposition(m, k)
    words = [{w: lab for w, lab in zip(wires, labels)} for labels, _ in terms]
    vals = pauli_product_expectations(device, words)
    return complex(sum(c * v for (_, c), v in zip(terms, vals)))
