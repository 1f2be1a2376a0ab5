"""``Device``: the op-dict runtime of the statevector path.

Mirrors the reference's ``mettleq.device.Device`` (device.py:73-156, 541-554,
1089-1097) for ``backend="sv"``: it owns one statevector, fuses the gate
stream (``fusion.fuse``, the counterpart of ``_fuse_zz_layers``) and
dispatches every fused layer to a CUDA kernel through the C ABI.  The
bounded-MPS backend is out of scope for this engine and is refused.

Differences by design: the state lives on a B200 and is mutated in place
(double-buffered inside libmq); ``execute`` returns the ``StateVector``
handle instead of an MLX array; there is no CPU execution device.
"""
from __future__ import annotations

import os
from typing import Any, Dict, List, Optional

import numpy as np

from . import fusion
from .engine import StateVector
from .execution import build_execution_plan, require_statevector_preflight


class Device:
    def __init__(
        self,
        wires: int,
        shots: int = 1000,
        backend: Optional[str] = None,
        mps_opts=None,
        *,
        metal_checkpoint_budget_bytes: Optional[int] = None,
        allow_unsafe_statevector: Optional[bool] = None,
        execution_device: Optional[str] = None,
        dtype: str = "complex64",
        device_index: int = 0,
        stream: Optional[int] = None,
    ):
        self.wires = int(wires)
        self.shots = int(shots)
        backend = str(backend or os.environ.get("METTLEQ_BACKEND", "sv")).strip().lower()
        if backend != "sv":
            raise NotImplementedError(
                "The B200 engine implements method='statevector' only; the MPS backend stays on the "
                "reference's CPU path")
        self.backend = "sv"
        if execution_device is not None:
            dev = str(execution_device).strip().lower()
            if dev not in ("gpu", "cuda", "auto"):
                raise ValueError("execution_device must be 'gpu' (CUDA) or None; this engine has no CPU path")
        self.execution_device = "gpu"
        self.dtype = str(np.dtype(dtype))
        self._allow_unsafe_statevector = allow_unsafe_statevector
        self.statevector_preflight = require_statevector_preflight(
            self.wires, dtype=self.dtype, allow_unsafe=allow_unsafe_statevector, device_index=device_index)
        self.sim = StateVector(self.wires, dtype=self.dtype, device=device_index, stream=stream)
        self.last_execution_plan: Optional[Dict[str, Any]] = None
        self.execution_selection: Optional[Dict[str, Any]] = None

    # reference: device.py:148-152
    def reset(self) -> None:
        self.sim.reset()

    def close(self) -> None:
        self.sim.close()

    # reference: device.py:154-431
    def execute(self, operations: List[Dict[str, Any]], *, report: Optional[bool] = None) -> StateVector:
        layers = fusion.fuse(operations, self.wires)
        if report is None:
            report = os.environ.get("METTLEQ_EXECUTION_REPORT", "0") == "1"
        before = self.sim.counters() if report else None
        for layer in layers:
            self.apply_layer(layer)
        if report:
            self.last_execution_plan = build_execution_plan(self.wires, self.dtype, operations, layers)
            after = self.sim.counters()
            self.last_execution_plan["observed"] = {
                "launches": after[0] - before[0],
                "sweeps": after[1] - before[1],
            }
        else:
            self.last_execution_plan = None
        return self.sim

    def explain(self, operations: List[Dict[str, Any]]) -> Dict[str, Any]:
        """Execution report without applying anything (device.py:520-539)."""
        layers = fusion.fuse(operations, self.wires)
        return build_execution_plan(self.wires, self.dtype, operations, layers)

    def apply_layer(self, layer: Dict[str, Any]) -> None:
        name = layer["name"]
        sim = self.sim
        if name == "_U2LISTLAYER":
            sim.apply_u2_layer(layer["mats"], layer["active"])
        elif name == "_LAYER":
            sim.apply_layer(layer["mats"], layer["active"], layer["terms"], layer["rows"], layer["c"])
        elif name == "_DIAG":
            sim.apply_diag_terms(layer["terms"])
        elif name == "_XORLAYER":
            sim.apply_xor_affine(layer["rows"], layer["c"])
        elif name == "_QFTSTAGES":
            sim.apply_qft_stages(layer["q0"], layer["k"], layer["j_begin"], layer["j_end"], layer["inverse"])
        elif name == "_QFTWIRES":
            sim.apply_qft(layer["wires"], inverse=layer.get("inverse", False))
        elif name == "_CULIST":
            sim.apply_controlled(layer["gates"])
        elif name == "_PAIRLAYER":
            sim.apply_pauli_pair_layer(layer["kind"], layer["bonds"], layer["thetas"])
        else:
            raise ValueError(f"Unknown fused layer: {name}")

    # reference: device.py:541-554 (returns the simulator's state, which
    # ``np.asarray(state, dtype=np.complex64)`` reads back like the MLX array
    # the reference returns)
    def synchronize(self):
        self.sim.synchronize()
        return self.sim.state

    def statevector(self) -> np.ndarray:
        return self.sim.get()

    # reference: device.py:1089-1097 (seeded here: the project's Philox stream)
    def sample(self, shots: Optional[int] = None, wires: Optional[List[int]] = None, *, seed: Optional[int] = None):
        shots = self.shots if shots is None else int(shots)
        if seed is None:
            seed = int(np.random.default_rng().integers(0, np.iinfo(np.uint32).max, dtype=np.uint32))
        return self.sim.sample_bits(shots, wires, seed=seed).tolist()

    def counts(self, shots: Optional[int] = None, wires: Optional[List[int]] = None, *, seed: Optional[int] = None):
        counts: Dict[str, int] = {}
        for bits in self.sample(shots, wires, seed=seed):
            key = "".join(str(b) for b in bits)
            counts[key] = counts.get(key, 0) + 1
        return counts
