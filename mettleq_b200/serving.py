"""Request serving with continuous batching (the serving direction).

The reference serves circuits one ``MettleQBackend.run`` call at a time
(integrations/qiskit.py:461-528): a request waits for every request before
it.  ``Server`` runs a request loop over one GPU instead:

  * admission: a request is admitted when its device footprint (both state
    buffers, 2 x 2^n x 8 B for complex64: permutation layers are
    out-of-place) fits the memory budget and an execution slot is free;
    waiting requests are taken smallest work (layers x 2^n) first, except
    that the oldest one is not passed any more once it has waited longer
    than ``max_bypass_s``;
  * every admitted request keeps its statevector resident on its own CUDA
    stream (higher priority for fewer qubits) for all its layers and shots;
    at most ``max_large`` requests with more than ``small_work`` amplitude-
    layers are on the device at once, and their launch grids leave
    ``sm_reserve`` SMs free, so short requests never wait for a sweep that
    holds the whole GPU;
    each round the loop issues work to the active requests with the least
    remaining work first, within a few milliseconds of host time: a request
    whose remaining work is small (up to 100 layers of 22 qubits) gets all
    of it at once, larger ones a few layers per round; short requests thus
    overtake long ones while the work of several requests overlaps on the
    device, and the loop polls CUDA events to notice completion;
  * finished requests draw their shots (mq_sample, seeded Philox stream) and
    give their state back to a pool, so steady-state serving allocates and
    frees no device memory (a cudaFree would stall every stream).

Each request's result depends only on its own circuit and seed: the same
kernels run on the same data whether it is served alone or in a mix.

``poisson_requests`` generates the serving benchmark's stream: Poisson
arrivals, qubit counts log-uniform in [12, 30], depth U{10..100} layers of
the config-0 structure (Haar U(2) on every qubit, RZZ chain, CNOT ladder),
each layer followed by a QFT with probability 0.1 and a random GF(2)
permutation with probability 0.1, 1000 shots.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from .engine import StateVector
from .fusion import DIAG_ZZ
from .workloads import cnot_ladder_rows, invertible_rows


@dataclass
class RequestLayer:
    mats: np.ndarray                       # (n, 4) U(2) per qubit
    thetas: np.ndarray                     # (n-1,) RZZ angles
    qft: bool = False
    xor: Optional[Tuple[List[int], int]] = None


@dataclass
class Request:
    rid: int
    arrival: float                         # seconds from the start of the stream
    n: int
    layers: List[RequestLayer]
    shots: int = 1000
    seed: int = 0
    # filled in by the server
    admitted: float = -1.0
    finished: float = -1.0
    samples: Optional[np.ndarray] = None
    state: Optional[np.ndarray] = None

    @property
    def footprint(self) -> int:
        return 2 * (1 << self.n) * 8

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def work(self) -> int:
        """Device work in amplitude-layers (layers x 2^n)."""
        return len(self.layers) << self.n


def haar_u2_batch(rng: np.random.Generator, k: int) -> np.ndarray:
    """k Haar-random 2x2 unitaries (QR of complex Ginibre matrices with the
    phase fix of Mezzadri 2007), as (k, 4)."""
    z = (rng.standard_normal((k, 2, 2)) + 1j * rng.standard_normal((k, 2, 2))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=1, axis2=2)
    return (q * (d / np.abs(d))[:, None, :]).reshape(k, 4)


def random_layer(n: int, rng: np.random.Generator, p_qft: float = 0.1, p_xor: float = 0.1) -> RequestLayer:
    mats = haar_u2_batch(rng, n)
    thetas = rng.uniform(0.0, 2.0 * math.pi, n - 1)
    L = RequestLayer(mats, thetas)
    if rng.random() < p_qft:
        L.qft = True
    if rng.random() < p_xor:
        L.xor = (invertible_rows(n, rng), int(rng.integers(0, 1 << n)))
    return L


def poisson_requests(count: int, rate: float = 200.0, seed: int = 0, n_range: Tuple[int, int] = (12, 30),
                     depth_range: Tuple[int, int] = (10, 100), shots: int = 1000) -> List[Request]:
    """``count`` seeded requests with exponential inter-arrival times (rate in
    requests/s), log-uniform qubit counts and uniform depths."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    lo, hi = math.log(n_range[0]), math.log(n_range[1] + 1)
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        n = min(n_range[1], int(math.exp(rng.uniform(lo, hi))))
        depth = int(rng.integers(depth_range[0], depth_range[1] + 1))
        layers = [random_layer(n, rng) for _ in range(depth)]
        reqs.append(Request(i, t, n, layers, shots, seed=int(rng.integers(0, 2 ** 62))))
    return reqs


def apply_request_layer(sv: StateVector, L: RequestLayer, ladder) -> None:
    """One layer: fused U(2) + RZZ chain + CNOT ladder, then the optional QFT
    and permutation.  The layer's C arrays are packed on first use."""
    packed = getattr(L, "_packed", None)
    if packed is None:
        terms = [(DIAG_ZZ, i, i + 1, [float(t) / 2.0]) for i, t in enumerate(L.thetas)]
        packed = sv.pack_layer(L.mats, None, terms, *ladder)
        L._packed = packed
    sv.apply_packed_layer(packed)
    if L.qft:
        sv.apply_qft(None)
    if L.xor is not None:
        sv.apply_xor_affine(*L.xor)


class StatePool:
    """Device states by qubit count, reused across requests."""

    def __init__(self, device: int):
        self.device = device
        self.free: Dict[int, List[Tuple[StateVector, object]]] = {}
        self.bytes_free = 0

    def get(self, n: int):
        lst = self.free.get(n)
        if lst:
            self.bytes_free -= 2 * (1 << n) * 8
            return lst.pop()
        import torch
        # fewer qubits -> higher stream priority (lower numbers are higher)
        prio = -1 if n <= 22 else 0
        stream = torch.cuda.Stream(device=self.device, priority=prio)
        sv = StateVector(n, "complex64", device=self.device, stream=stream.cuda_stream)
        return sv, stream

    def put(self, n: int, item) -> None:
        self.free.setdefault(n, []).append(item)
        self.bytes_free += 2 * (1 << n) * 8

    def evict(self, need: int) -> int:
        """Free pooled states (largest first) until ``need`` bytes are
        released or the pool is empty; returns the bytes released."""
        released = 0
        for n in sorted(self.free, reverse=True):
            while self.free[n] and released < need:
                sv, _ = self.free[n].pop()
                sv.close()
                released += 2 * (1 << n) * 8
                self.bytes_free -= 2 * (1 << n) * 8
        return released

    def close(self) -> None:
        self.evict(1 << 62)


class Server:
    """Continuous-batching request loop (see the module docstring)."""

    def __init__(self, budget_bytes: int = 150 * 10 ** 9, max_active: int = 64, layers_per_round: int = 4,
                 max_bypass_s: float = 30.0, device: int = 0, keep_states: bool = False,
                 round_budget_s: float = 0.004, small_work: int = 100 << 22, max_large: int = 8,
                 sm_reserve: int = 20, devices: Optional[List[int]] = None):
        # budget_bytes, max_large and sm_reserve hold per device; with several
        # devices every request goes to the device with the least footprint
        # admitted that has room for it (one queue per device)
        self.budget = int(budget_bytes)
        self.max_active = int(max_active)
        self.k = int(layers_per_round)
        self.round_budget_s = float(round_budget_s)    # host time spent issuing per round
        self.small_work = int(small_work)              # layers x 2^n issued in one go
        self.max_large = int(max_large)                # large requests on the device at once
        self.sm_reserve = int(sm_reserve)              # SMs large requests leave to the others
        self.max_bypass_s = float(max_bypass_s)
        self.devices = [int(d) for d in devices] if devices else [int(device)]
        self.device = self.devices[0]
        self.keep_states = keep_states
        self.pools = {d: StatePool(d) for d in self.devices}
        self.pool = self.pools[self.device]
        self.served_on: Dict[int, int] = {d: 0 for d in self.devices}  # requests admitted per device
        self._ladders: Dict[int, Tuple[List[int], int]] = {}
        self.peak_used = 0      # most footprint bytes admitted at once on one device
        self.peak_active = 0    # most requests on the device at once
        self.peak_large = 0     # most large requests on the device at once
        self.partial_issues = 0  # issues of a chunk shorter than the request's remaining work

    def _ladder(self, n: int):
        if n not in self._ladders:
            self._ladders[n] = cnot_ladder_rows(n)
        return self._ladders[n]

    def serve(self, requests: List[Request], realtime: bool = True,
              clock: Callable[[], float] = time.perf_counter) -> Dict[str, float]:
        """Serve ``requests``.  With ``realtime`` the arrivals follow the wall
        clock from now; otherwise every request is available at once.  Fills
        admitted / finished / samples of each request and returns summary
        statistics (latency = finished - arrival)."""
        import torch
        sms = {d: torch.cuda.get_device_properties(d).multi_processor_count for d in self.devices}
        for r in requests:
            if r.footprint > self.budget:
                raise MemoryError(f"request {r.rid}: {r.n} qubits need {r.footprint} bytes, budget {self.budget}")
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: List[Request] = []
        active: List[dict] = []
        used = {d: 0 for d in self.devices}
        done = 0
        while done < len(requests):
            t = now()
            while pending and (not realtime or pending[0].arrival <= t):
                waiting.append(pending.popleft())
            # admission: smallest work first; the oldest request may not be
            # passed once it has waited max_bypass_s
            if waiting:
                head = min(waiting, key=lambda r: r.arrival)
                if now() - head.arrival > self.max_bypass_s:
                    waiting.sort(key=lambda r: (r is not head, r.work))
                else:
                    waiting.sort(key=lambda r: r.work)
            i = 0
            n_large = {d: sum(1 for a in active if a["large"] and a["dev"] == d) for d in self.devices}
            while i < len(waiting) and len(active) < self.max_active:
                r = waiting[i]
                large = r.work > self.small_work
                # the device with the least footprint admitted among those
                # with room (and a free large-request slot when it is large)
                fits = [d for d in self.devices if used[d] + r.footprint <= self.budget
                        and not (large and n_large[d] >= self.max_large)]
                if fits:
                    dev = min(fits, key=lambda d: (used[d], d))
                    pool = self.pools[dev]
                    reuse = bool(pool.free.get(r.n))
                    if not reuse:
                        over = used[dev] + r.footprint + pool.bytes_free - self.budget
                        if over > 0:
                            pool.evict(over)
                    sv, stream = pool.get(r.n)
                    sv.reset()
                    # large requests leave SMs free, so the kernels of short
                    # requests start without waiting for a whole-GPU sweep
                    sv.set_sm_limit(sms[dev] - self.sm_reserve if large else 0)
                    n_large[dev] += 1 if large else 0
                    self.peak_large = max(self.peak_large, n_large[dev])
                    r.admitted = now()
                    active.append({"req": r, "sv": sv, "stream": stream, "next": 0, "events": deque(),
                                   "large": large, "dev": dev})
                    used[dev] += r.footprint
                    self.served_on[dev] += 1
                    self.peak_used = max(self.peak_used, used[dev])
                    self.peak_active = max(self.peak_active, len(active))
                    waiting.pop(i)
                    continue
                if i == 0 and now() - r.arrival > self.max_bypass_s:
                    break  # the overdue head waits for room; nothing passes it
                i += 1
            # issue: smallest remaining work first within a host-time budget
            # per round; a request whose whole remaining work is small gets
            # all of it at once, larger ones a chunk of layers, with at most
            # two chunks queued per request
            progressed = False
            order = sorted(active, key=lambda a: (len(a["req"].layers) - a["next"]) << a["req"].n)
            round_end = clock() + self.round_budget_s
            for a in order:
                if clock() > round_end:
                    break
                r = a["req"]
                ev = a["events"]
                while ev and ev[0].query():
                    ev.popleft()
                if a["next"] >= len(r.layers) or len(ev) >= 2:
                    continue
                left = len(r.layers) - a["next"]
                chunk = left if (left << r.n) <= self.small_work else self.k
                stop = min(len(r.layers), a["next"] + chunk)
                if stop < len(r.layers):
                    self.partial_issues += 1
                for j in range(a["next"], stop):
                    apply_request_layer(a["sv"], r.layers[j], self._ladder(r.n))
                a["next"] = stop
                e = torch.cuda.Event()
                e.record(a["stream"])
                ev.append(e)
                progressed = True
            # completions: shots, then the state goes back to the pool
            still = []
            for a in active:
                r = a["req"]
                ev = a["events"]
                while ev and ev[0].query():
                    ev.popleft()
                if a["next"] >= len(r.layers) and not ev:
                    r.samples = a["sv"].sample_indices(r.shots, seed=r.seed)
                    if self.keep_states:
                        r.state = a["sv"].get()
                    r.finished = now()
                    used[a["dev"]] -= r.footprint
                    self.pools[a["dev"]].put(r.n, (a["sv"], a["stream"]))
                    done += 1
                    progressed = True
                else:
                    still.append(a)
            active = still
            if not progressed:
                if not active and not waiting and pending and realtime:
                    time.sleep(max(0.0, min(0.001, pending[0].arrival - now())))
                else:
                    time.sleep(0.0001)
        makespan = now()
        lat = np.array([r.latency for r in requests])
        return {"requests": len(requests), "makespan_s": makespan, "circuits_per_s": len(requests) / makespan,
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(lat.mean())}

    def close(self) -> None:
        for p in self.pools.values():
            p.close()


def assign_by_work(requests: List[Request], n_devices: int) -> List[List[int]]:
    """One queue per device for a request stream split over processes (one
    per GPU): in arrival order, each request goes to the device with the
    least work (layers x 2^n) assigned so far (ties to the lowest device).
    Only earlier arrivals decide a request's device, so the rule can run
    online, and every process computes the same split.  Returns request
    positions per device."""
    if n_devices < 1:
        raise ValueError("n_devices must be >= 1")
    load = [0] * n_devices
    out: List[List[int]] = [[] for _ in range(n_devices)]
    for i in sorted(range(len(requests)), key=lambda k: (requests[k].arrival, k)):
        d = min(range(n_devices), key=lambda k: (load[k], k))
        out[d].append(i)
        load[d] += requests[i].work
    return out


def device_work(requests: List[Request], device: int = 0, host_s_per_layer: float = 5e-4) -> List[float]:
    """Device time of each request's layers run alone (seconds, CUDA events):
    the GPU first spins for longer than the host needs to issue all of the
    request's layers, so the events bracket back-to-back kernels only and
    their sum is a lower bound on any schedule's busy time (shots excluded:
    one read of the state).  Spins are bounded (torch's clock-cycle sleep);
    a request whose issue outlasted its spin is measured again with twice
    the spin."""
    import torch
    pool = StatePool(device)
    ladders: Dict[int, Tuple[List[int], int]] = {}
    rate = 2.0e9  # spin cycles per second: at or above the SM clock, so a spin lasts at least its time
    out = []
    try:
        for r in requests:
            ladder = ladders.setdefault(r.n, cnot_ladder_rows(r.n))
            sv, stream = pool.get(r.n)
            spin = host_s_per_layer * max(1, len(r.layers))
            for _ in range(6):
                sv.reset()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    torch.cuda._sleep(int(spin * rate))
                    e0.record(stream)
                    for L in r.layers:
                        apply_request_layer(sv, L, ladder)
                    late = e0.query()  # the spin ended before the last layer was issued
                    e1.record(stream)
                e1.synchronize()
                if not late:
                    break
                spin *= 2.0
            out.append(e0.elapsed_time(e1) / 1e3)
            pool.put(r.n, (sv, stream))
    finally:
        pool.close()
    return out


def serve_plain(requests: List[Request], realtime: bool = True, device: int = 0,
                clock: Callable[[], float] = time.perf_counter, cache: Optional[dict] = None) -> Dict[str, float]:
    """The reference's serving model: one request at a time in arrival order,
    each through the op-dict runtime (Device.execute, integrations/_common.py
    :118-228) and a seeded sample.  Devices are cached per width like the
    reference's ``execution_cache`` (_common.py:166-195): a width seen before
    reuses its state, reset to |0...0>."""
    from .device import Device
    from .workloads import affine_gates, qft_ops, u3_params
    own = cache is None
    cache = {} if own else cache
    t0 = clock()
    now = lambda: clock() - t0  # noqa: E731
    for r in sorted(requests, key=lambda x: x.arrival):
        if realtime and r.arrival > now():
            time.sleep(r.arrival - now())
        ops = []
        n = r.n
        for L in r.layers:
            for q in range(n):
                th, ph, lam, _ = u3_params(L.mats[q].reshape(2, 2))  # global phase: no effect on shots
                ops.append({"name": "U3", "wires": [q], "parameters": [th, ph, lam]})
            for i, th in enumerate(L.thetas):
                ops.append({"name": "ZZPHASE", "wires": [i, i + 1], "parameters": [float(th) / 2.0]})
            for i in range(n - 1):
                ops.append({"name": "CNOT", "wires": [i, i + 1], "parameters": []})
            if L.qft:
                ops.extend(qft_ops(n))
            if L.xor is not None:
                ops.extend(affine_gates(list(L.xor[0]), int(L.xor[1]), n))
        dev = cache.get(n)
        if dev is None:
            dev = cache[n] = Device(n, device_index=device)
        else:
            dev.reset()
        dev.execute(ops)
        r.samples = dev.sim.sample_indices(r.shots, seed=r.seed)
        r.finished = now()
    makespan = now()
    if own:
        for d in cache.values():
            d.close()
    lat = np.array([r.latency for r in requests])
    return {"requests": len(requests), "makespan_s": makespan, "circuits_per_s": len(requests) / makespan,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean())}
