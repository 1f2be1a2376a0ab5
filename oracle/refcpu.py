"""Timing of the reference's own CPU statevector code (the reference arm).

MEASUREMENT INFRASTRUCTURE, like the rest of ``oracle/``: only ``bench.py``'s
reference and CPU-baseline legs call this module, and nothing in
``mettleq_b200`` imports it.

The reference (MettleQ, installed without dependencies into a directory such
as ``baseline/_ref``) runs its ``method="statevector"`` circuits on a host
CPU through ``Device(n, execution_device="cpu").execute(ops)``: one MLX pass
per gate (device.py:1138-1290 -> sim.py).  MLX exists only for Apple
silicon, so ``oracle/mlx_shim`` stands in for ``mlx.core`` with numpy; the
reference's Python code itself runs unchanged.

A full 30-qubit circuit of thousands of gates takes hours on host cores, so
the arm times a bounded sample: every gate name of the circuit once, at
``n_cpu`` qubits, and extrapolates by the circuit's own gate counts.  To use
every host thread, the n_cpu-qubit state is split into 2^k independent
chunk devices of n_cpu - k qubits, one thread each (numpy releases the GIL
inside its array loops); a gate on a chunk's own qubits is the same gate on
the full state, so the timed work is that of one n_cpu-qubit gate pass.
"""
from __future__ import annotations

import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "mlx_shim")


def load_reference_device(path: Optional[str]):
    """The reference's ``mettleq.device.Device`` from ``path`` (an installed
    tree holding the ``mettleq`` package) under the numpy ``mlx.core``
    stand-in, or None when it is not there."""
    if not path or not os.path.isdir(os.path.join(path, "mettleq")):
        return None
    for p in (path, SHIM):
        if p not in sys.path:
            sys.path.insert(0, p)
    try:
        from mettleq.device import Device  # the reference's own runtime
    except Exception:
        return None
    return Device


def _sample_op(name: str, nl: int, rng: np.random.Generator) -> dict:
    """One op of ``name`` on middle qubits of an nl-qubit chunk."""
    a, b = nl // 2, nl // 2 + 1
    if name == "U3":
        return {"name": "U3", "wires": [a], "parameters": [float(x) for x in rng.uniform(-np.pi, np.pi, 3)]}
    if name in ("ZZPHASE", "CPHASE", "CRZ", "CRX", "CRY", "XXPHASE", "YYPHASE"):
        return {"name": name, "wires": [b, a], "parameters": [float(rng.uniform(-np.pi, np.pi))]}
    if name in ("RX", "RY", "RZ", "U1"):
        return {"name": name, "wires": [a], "parameters": [float(rng.uniform(-np.pi, np.pi))]}
    if name in ("CNOT", "CZ", "SWAP", "CH", "ISWAP"):
        return {"name": name, "wires": [a, b], "parameters": []}
    return {"name": name, "wires": [a], "parameters": []}


class PortDevice:
    """The oracle's restatement of the same per-gate CPU path
    (``oracle.sv.OracleSim``, device.py:1138-1290) behind the two calls the
    timing uses; the fallback when the reference is not installed."""

    def __init__(self, n: int, execution_device: str = "cpu"):
        from .sv import OracleSim
        self.sim = OracleSim(n, np.complex64)

    def set_state(self, v: np.ndarray) -> None:
        self.sim.set_state(v)

    def execute(self, ops) -> None:
        self.sim.execute(ops)


def _set_state(d, v: np.ndarray) -> None:
    if isinstance(d, PortDevice):
        d.set_state(v)
    else:
        import mlx.core as mx  # the stand-in, put on sys.path by load_reference_device
        d.sim.state = mx.array(v)


_CHUNKS: Dict[tuple, list] = {}  # chunk devices kept across timed steps


def time_reference_gates(Device, names: Sequence[str], n_cpu: int, threads: int,
                         repeats: int = 2) -> Tuple[Dict[str, float], int, int]:
    """Seconds of one ``Device.execute([op])`` of each gate name over a
    2^n_cpu-amplitude state split into chunk devices on ``threads`` threads
    (best of ``repeats``; the first call of a name on new devices is run
    once untimed).  The chunk devices are kept for later calls with the same
    shape, so repeated steps time the gates, not the set-up.  Returns
    (times, chunks, qubits per chunk)."""
    k = 0
    while (2 << k) <= max(1, threads) and n_cpu - (k + 1) >= 8:
        k += 1
    T = 1 << k
    nl = n_cpu - k
    rng = np.random.default_rng(1)
    key = (Device, n_cpu, T)
    fresh = key not in _CHUNKS
    if fresh:
        _CHUNKS.clear()  # one set of chunk devices at a time (host memory)
        devs = []
        for _ in range(T):
            d = Device(nl, execution_device="cpu")
            v = (rng.standard_normal(1 << nl) + 1j * rng.standard_normal(1 << nl)).astype(np.complex64)
            _set_state(d, (v / np.linalg.norm(v)).astype(np.complex64))
            devs.append(d)
            del v
        _CHUNKS[key] = devs
    devs = _CHUNKS[key]
    pool = ThreadPoolExecutor(T) if T > 1 else None

    def run(op):
        if pool is None:
            devs[0].execute([op])
        else:
            list(pool.map(lambda d: d.execute([op]), devs))

    times: Dict[str, float] = {}
    try:
        for name in names:
            op = _sample_op(name, nl, rng)
            if fresh:
                run(op)  # first call on new devices: code paths and allocator warm
            best = float("inf")
            for _ in range(max(1, repeats)):
                t0 = time.perf_counter()
                run(op)
                best = min(best, time.perf_counter() - t0)
            times[name] = best
    finally:
        if pool is not None:
            pool.shutdown()
    return times, T, nl


def extrapolate(counts: Dict[str, int], times: Dict[str, float], n_target: int, n_cpu: int) -> float:
    """Seconds of the whole circuit at n_target qubits: per-gate time x
    2^(n_target - n_cpu) (one pass over a state twice as large takes twice
    as long) x the circuit's count of that gate."""
    scale = 2.0 ** (n_target - n_cpu)
    return sum(c * times[name] * scale for name, c in counts.items())
