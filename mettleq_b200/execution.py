"""Admission policy, memory estimates and execution reports.

Counterpart of the reference's execution.py for the B200 engine:
``state_memory_estimate`` / ``statevector_preflight`` /
``require_statevector_preflight`` (execution.py:195-407) refuse a state
before allocation when it cannot fit, with the same override variable
(``METTLEQ_ALLOW_UNSAFE_STATEVECTOR``, explicit argument wins), and
``build_execution_plan`` records the fused layers with their expected
full-state sweeps and predicted I/O bytes (the reference's
``out_of_place_bytes_per_custom_launch`` = 2 x state bytes,
execution.py:783-1131).
"""
from __future__ import annotations

import math
import os
from typing import Any, Dict, List, Optional, Sequence

from . import fusion
from ._native import StatevectorMemoryError

STATEVECTOR_UNSAFE_OVERRIDE_ENV = "METTLEQ_ALLOW_UNSAFE_STATEVECTOR"
# 2^n amplitudes are counted in 32 bits, so 31 qubits at most (the
# reference's METAL_INDEX_QUBIT_LIMIT, execution.py:23-25)
INDEX_QUBIT_LIMIT = 31
_TRUE = {"1", "true", "on", "yes", "enabled"}
_FALSE = {"0", "false", "off", "no", "disabled", ""}


def bytes_per_amplitude(dtype: str) -> int:
    if dtype == "complex64":
        return 8
    if dtype == "complex128":
        return 16
    raise ValueError("dtype must be complex64 or complex128")


def state_memory_estimate(n_qubits: int, dtype: str = "complex64") -> Dict[str, Any]:
    n = int(n_qubits)
    if n < 0:
        raise ValueError("n_qubits must be non-negative")
    b = bytes_per_amplitude(dtype)
    state = (1 << n) * b
    return {
        "dtype": dtype,
        "amplitudes": 1 << n,
        "bytes_per_amplitude": b,
        "state_bytes": state,
        "state_mib": state / 2 ** 20,
        # tile sweeps and diagonal layers run in place; the permutation layer
        # and the full probability read-back use a second buffer
        "minimum_input_plus_output_bytes": 2 * state,
        "bytes_per_sweep": 2 * state,
    }


def _device_memory(device_index: int = 0) -> Dict[str, Optional[int]]:
    try:
        import torch
        if torch.cuda.is_available():
            free, total = torch.cuda.mem_get_info(device_index)
            return {"free": int(free), "total": int(total)}
    except Exception:
        pass
    return {"free": None, "total": None}


def unsafe_override(allow_unsafe: Optional[bool]) -> Dict[str, Any]:
    raw = os.environ.get(STATEVECTOR_UNSAFE_OVERRIDE_ENV)
    if allow_unsafe is not None:
        if not isinstance(allow_unsafe, bool):
            raise TypeError("allow_unsafe_statevector must be a boolean or None")
        return {"enabled": allow_unsafe, "source": "constructor_argument"}
    if raw is None:
        return {"enabled": False, "source": "default_disabled"}
    v = raw.strip().lower()
    if v in _TRUE:
        return {"enabled": True, "source": "environment"}
    if v in _FALSE:
        return {"enabled": False, "source": "environment"}
    raise ValueError(f"{STATEVECTOR_UNSAFE_OVERRIDE_ENV} must be a boolean value")


def statevector_preflight(n_qubits: int, *, dtype: str = "complex64", allow_unsafe: Optional[bool] = None,
                          device_index: int = 0, memory: Optional[Dict[str, Optional[int]]] = None) -> Dict[str, Any]:
    n = int(n_qubits)
    est = state_memory_estimate(n, dtype)
    override = unsafe_override(allow_unsafe)
    mem = memory if memory is not None else _device_memory(device_index)
    failures: List[str] = []
    if n > INDEX_QUBIT_LIMIT:
        failures.append("exceeds_32_bit_index_limit")
    if mem.get("total") is not None and est["state_bytes"] > mem["total"]:
        failures.append("single_state_exceeds_device_memory")
    if mem.get("free") is not None and est["minimum_input_plus_output_bytes"] > mem["free"]:
        failures.append("two_state_lower_bound_exceeds_free_memory")
    hard = "exceeds_32_bit_index_limit" in failures
    refused = bool(failures)
    allowed = (not refused) or (override["enabled"] and not hard)
    return {
        "schema_version": 1,
        "allowed": allowed,
        "decision": ("refused" if not allowed else
                     "allowed_with_unsafe_override" if refused else "allowed_within_reported_lower_bounds"),
        "failure_reasons": failures,
        "qubits": n,
        "dtype": dtype,
        "device_memory": mem,
        "cost_model": est,
        "override": override,
    }


def require_statevector_preflight(n_qubits: int, *, dtype: str = "complex64", allow_unsafe: Optional[bool] = None,
                                  device_index: int = 0,
                                  memory: Optional[Dict[str, Optional[int]]] = None) -> Dict[str, Any]:
    report = statevector_preflight(n_qubits, dtype=dtype, allow_unsafe=allow_unsafe, device_index=device_index,
                                   memory=memory)
    if report["allowed"]:
        return report
    est = report["cost_model"]
    gib = 1024.0 ** 3
    raise StatevectorMemoryError(
        f"Refusing {n_qubits}-qubit {dtype} statevector before allocation: one state is "
        f"{est['state_bytes'] / gib:.2f} GiB and the two-buffer lower bound is "
        f"{est['minimum_input_plus_output_bytes'] / gib:.2f} GiB ({', '.join(report['failure_reasons'])}). "
        f"Reduce qubits or set {STATEVECTOR_UNSAFE_OVERRIDE_ENV}=1 to bypass this preflight.",
        report)


def build_execution_plan(n_qubits: int, dtype: str, operations: Sequence[dict], layers: Sequence[dict]) -> Dict[str, Any]:
    est = state_memory_estimate(n_qubits, dtype)
    entries = []
    total_sweeps = 0
    for i, layer in enumerate(layers):
        sweeps = fusion.expected_sweeps(layer, n_qubits, dtype)
        total_sweeps += sweeps
        entries.append({
            "index": i,
            "kernel_family": layer["name"],
            "expected_sweeps": sweeps,
            "predicted_io_bytes": sweeps * est["bytes_per_sweep"],
        })
    return {
        "schema_version": 1,
        "n_qubits": int(n_qubits),
        "dtype": dtype,
        "input_operations": len(operations),
        "fused_layers": entries,
        "expected_sweeps": total_sweeps,
        "predicted_io_bytes": total_sweeps * est["bytes_per_sweep"],
        "cost_model": est,
    }
