"""Batched circuits in one CUDA-graph launch (the batching direction).

The reference runs a batch as a loop over circuits, one launch sequence per
circuit (integrations/qiskit.py:505-514).  ``CircuitBatch`` hands a whole
batch of layered circuits (per layer: a 2x2 on every qubit, then optionally
the CNOT ladder) to ``mq_batch_*``: circuits of <= 13 qubits run whole in
shared memory inside one persistent kernel, larger ones run tile sweeps on
parallel streams, and the first run captures everything as one CUDA graph
that later runs replay with new parameters (the matrices are read from device
memory).  Outputs stay on the device: every circuit's probability vector
(float32) and <Z_0> (float64).

``autotune`` picks the batch's launch shape (threads per block of the
shared-memory kernel, number of parallel lanes) and then the tile shape of
the large circuits' sweeps (largest tile, passenger bits, smallest tile) by
timing the candidates on the batch itself.

``hea_batch`` generates the benchmark's batches: hardware-efficient ansatz
circuits, RY and RZ angles U[-pi, pi] on every qubit per layer, then a CNOT
ladder, n ~ U{10..24}, depth ~ U{4..16}.
"""
from __future__ import annotations

import ctypes as C
import itertools
import math
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def hea_mats(params: np.ndarray) -> np.ndarray:
    """(depth, n, 2) angles (RY theta, RZ phi) -> (depth, n, 4) matrices
    RZ(phi) RY(theta) (the RY then RZ of one layer, gates.py RY / RZ)."""
    p = np.asarray(params, dtype=np.float64)
    th, ph = p[..., 0], p[..., 1]
    c, s = np.cos(th / 2.0), np.sin(th / 2.0)
    em, ep = np.exp(-0.5j * ph), np.exp(0.5j * ph)
    out = np.empty(p.shape[:-1] + (4,), dtype=np.complex128)
    out[..., 0] = em * c
    out[..., 1] = -em * s
    out[..., 2] = ep * s
    out[..., 3] = ep * c
    return out


def hea_ops(params: np.ndarray, ladder: bool = True) -> List[dict]:
    """The same circuit as op dicts (for the plain path and the oracle)."""
    p = np.asarray(params, dtype=np.float64)
    depth, n = p.shape[0], p.shape[1]
    ops = []
    for d in range(depth):
        for q in range(n):
            ops.append({"name": "RY", "wires": [q], "parameters": [float(p[d, q, 0])]})
        for q in range(n):
            ops.append({"name": "RZ", "wires": [q], "parameters": [float(p[d, q, 1])]})
        if ladder:
            for q in range(n - 1):
                ops.append({"name": "CNOT", "wires": [q, q + 1], "parameters": []})
    return ops


def hea_batch(count: int, seed: int = 0, n_range: Tuple[int, int] = (10, 24),
              depth_range: Tuple[int, int] = (4, 16)) -> Tuple[List[int], List[int], List[np.ndarray]]:
    """(qubit counts, depths, angle arrays (depth, n, 2)) of ``count``
    seeded hardware-efficient-ansatz circuits."""
    rng = np.random.default_rng(seed)
    ns = [int(x) for x in rng.integers(n_range[0], n_range[1] + 1, size=count)]
    depths = [int(x) for x in rng.integers(depth_range[0], depth_range[1] + 1, size=count)]
    params = [rng.uniform(-math.pi, math.pi, size=(d, n, 2)) for n, d in zip(ns, depths)]
    return ns, depths, params


class CircuitBatch:
    """A planned batch; ``run(mats)`` is one host-to-device copy and one graph
    launch (the first run also captures the graph)."""

    def __init__(self, n_qubits: Sequence[int], depths: Sequence[int], ladder=True, device: int = 0,
                 lanes: int = 8, small_threads: int = 256, stream: Optional[int] = None,
                 tiles: Optional[Tuple[int, int, int]] = None):
        import torch  # device memory for the outputs (plumbing)
        self.n = [int(x) for x in n_qubits]
        self.depths = [int(x) for x in depths]
        if len(self.n) != len(self.depths):
            raise ValueError("n_qubits and depths differ in length")
        lad = np.array([1 if (ladder if isinstance(ladder, bool) else ladder[i]) else 0
                        for i in range(len(self.n))], dtype=np.uint8)
        self.device = int(device)
        self._lib = N.lib()
        ns = np.asarray(self.n, dtype=np.int32)
        ds = np.asarray(self.depths, dtype=np.int32)
        h = C.c_void_p()
        N.check(self._lib.mq_batch_create(self.device, C.c_void_p(stream or 0), len(self.n), _ptr(ns), _ptr(ds),
                                          _ptr(lad), int(lanes), int(small_threads), C.byref(h)))
        self._h = h
        self.tiles = tuple(int(x) for x in tiles) if tiles is not None else (0, -1, 0)
        if tiles is not None:
            N.check(self._lib.mq_batch_set_tiles(h, *self.tiles))
        mc, pc = C.c_uint64(), C.c_uint64()
        nsm, nlg = C.c_int(), C.c_int()
        N.check(self._lib.mq_batch_info(h, C.byref(mc), C.byref(pc), C.byref(nsm), C.byref(nlg)))
        self.mats_count, self.probs_count = int(mc.value), int(pc.value)
        self.n_small, self.n_large = int(nsm.value), int(nlg.value)
        dev = f"cuda:{self.device}"
        self.probs_dev = torch.empty(max(1, self.probs_count), dtype=torch.float32, device=dev)
        self.z0_dev = torch.empty(max(1, len(self.n)), dtype=torch.float64, device=dev)
        self.offsets = np.concatenate([[0], np.cumsum([1 << n for n in self.n])]).astype(np.int64)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mq_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack(self, mats: Sequence[np.ndarray]) -> np.ndarray:
        """Per-circuit (depth, n, 4) complex matrices -> the flat float64
        array of mq_batch_run."""
        if len(mats) != len(self.n):
            raise ValueError("one matrix array per circuit")
        parts = []
        for m, n, d in zip(mats, self.n, self.depths):
            m = np.asarray(m, dtype=np.complex128)
            if m.shape != (d, n, 4):
                raise ValueError(f"matrices of a {n}-qubit depth-{d} circuit must have shape {(d, n, 4)}")
            parts.append(np.ascontiguousarray(m).view(np.float64).reshape(-1))
        flat = np.concatenate(parts) if parts else np.zeros(1)
        assert flat.size == max(self.mats_count, 0) or self.mats_count == 0
        return np.ascontiguousarray(flat)

    def run(self, mats: Sequence[np.ndarray] = None, packed: Optional[np.ndarray] = None) -> None:
        flat = packed if packed is not None else self.pack(mats)
        N.check(self._lib.mq_batch_run(self._h, _ptr(flat), C.c_void_p(self.probs_dev.data_ptr()),
                                       C.c_void_p(self.z0_dev.data_ptr())))

    def synchronize(self) -> None:
        N.check(self._lib.mq_batch_sync(self._h))

    def z0(self) -> np.ndarray:
        self.synchronize()
        return self.z0_dev[: len(self.n)].cpu().numpy()

    def probabilities(self, c: int) -> np.ndarray:
        self.synchronize()
        return self.probs_dev[int(self.offsets[c]):int(self.offsets[c + 1])].cpu().numpy()


# Tile shapes (largest tile, low passenger bits, smallest tile) the autotuner
# tries for the large circuits: the library default first, then smaller and
# larger tiles and fewer / more passengers (shorter / longer contiguous runs).
TILE_CANDIDATES = ((0, -1, 0), (11, 4, 0), (10, 4, 0), (12, 3, 0), (12, 5, 0), (12, 4, 12))


def _time_batch(n_qubits, depths, packed, device, repeats, **kw) -> float:
    import torch
    b = CircuitBatch(n_qubits, depths, device=device, **kw)
    try:
        b.run(packed=packed)  # captures the graph (untimed)
        b.synchronize()
        ts = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            b.run(packed=packed)
            b.synchronize()
            ts.append(time.perf_counter() - t0)
        return min(ts)
    finally:
        b.close()
        torch.cuda.synchronize(device)


def autotune(n_qubits: Sequence[int], depths: Sequence[int], packed: np.ndarray, device: int = 0,
             lanes=(4, 8, 16), small_threads=(128, 256, 512), tiles=TILE_CANDIDATES, repeats: int = 2,
             cache: Optional[Dict] = None) -> Dict:
    """Choose the batch's launch shape and tile shape by timing them on this
    batch (graph capture excluded: each candidate runs once untimed):
    first every (lanes, small_threads) pair with the default tiles, then
    every tile shape of ``tiles`` (largest tile, passengers, smallest tile)
    for the large circuits' sweeps with the best pair.  Returns the choice
    with the time of every tile candidate.  ``cache`` (a dict) memoises the
    choice per batch signature."""
    key = (tuple(sorted(set(int(n) for n in n_qubits))), len(n_qubits), int(sum(depths)))
    if cache is not None and key in cache:
        return cache[key]
    best, best_t = None, float("inf")
    for nl, nt in itertools.product(lanes, small_threads):
        t = _time_batch(n_qubits, depths, packed, device, repeats, lanes=nl, small_threads=nt)
        if t < best_t:
            best, best_t = {"lanes": nl, "small_threads": nt}, t
    tried = {}
    best_tiles, best_tt = None, float("inf")
    if any(int(n) > 13 for n in n_qubits):
        for tl in tiles:
            t = _time_batch(n_qubits, depths, packed, device, repeats, lanes=best["lanes"],
                            small_threads=best["small_threads"], tiles=tl)
            tried["%d/%d/%d" % tl] = t
            if t < best_tt:
                best_tiles, best_tt = tl, t
    best = dict(best, tiles=best_tiles, tile_times_s=tried)
    if cache is not None:
        cache[key] = best
    return best
