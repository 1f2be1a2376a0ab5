#!/usr/bin/env python
"""Headline benchmark: 30-qubit complex64 layer throughput on B200.

Workload (the scale configuration): n = 30 qubits, complex64 (8 GiB state),
40 layers of [Haar U(2) on every qubit, RZZ(i, i+1) with random angles, CNOT
ladder 0->1->...->29], a full 30-qubit QFT after every 10th layer followed by a
random GF(2) permutation layer.  Seeded synthetic inputs (no dataset exists
for this path).

One step = one pass of the whole circuit from |0...0>.  Metric "30q layer
GB/s" = (logical layers x 2 x 2^n x 8 bytes) / step time: every logical layer
(a U(2) layer, an RZZ layer, a CNOT ladder, a QFT, a permutation layer) is
credited with one read and one write of the state, so fusing sweeps shows up
as a higher number.  The 8 GiB state is far larger than L2 (126 MB).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 (torchrun, one rank per GPU) every rank runs its own replica
(weak scaling, no data-path collective); value sums all ranks' bytes over the
max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["scale", "batch", "adjoint", "serve", "sharded"], default="scale",
                    help="scale (the headline line), batch (4096 mixed circuits in one graph), adjoint "
                         "(24-qubit gradient of 384 parameters), serve (Poisson request stream), sharded "
                         "(one state of qubits + log2 N qubits over the N GPUs)")
    ap.add_argument("--count", type=int, default=None, help="circuits (batch) or requests (serve)")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--layers", type=int, default=40)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--shots", type=int, default=1000)
    ap.add_argument("--cpu-qubits", type=int, default=int(os.environ.get("MQ_BENCH_CPU_QUBITS", "28")))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-infidelity", action="store_true",
                    help="skip the complex128 run of the scale circuit (1 - |<psi64|psi128>|^2)")
    ap.add_argument("--no-extras", action="store_true",
                    help="scale workload: skip the batch / adjoint / serve sub-results of the headline line")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s, p in zip(sm, power) if p > 200.0] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "samples": len(sm),
                "power_w_max": max(power), "reasons": sorted(reasons)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- CPU side
def cpu_threads() -> int:
    """Host threads the CPU baseline may use: the process's CPU affinity."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return max(1, os.cpu_count() or 1)


REFERENCE_TREE = os.environ.get("MQ_REFERENCE_TREE", os.path.join(ROOT, "baseline", "_ref"))


def cpu_baseline_sample(n_target: int, n_cpu: int, circuit, threads: int = 1, repeats: int = 2):
    """Time the reference's own CPU statevector path on a bounded sample and
    extrapolate it to the full circuit.

    The circuit is the op-dict stream a user hands the reference
    (``circuit.ops()``: U3, ZZPHASE, CNOT, the QFTs as H + CPHASE ladders,
    each GF(2) layer as its Gauss-Jordan CNOT / SWAP / X synthesis).  The
    reference runs it one full-state pass per gate on a CPU
    (``Device(n, execution_device="cpu").execute``, device.py:1138-1290), so
    every gate name of the stream is executed once at n_cpu qubits (split
    into independent chunk devices, one per host thread) and the circuit's
    time is the sum over its gates of that name's time x 2^(n_target -
    n_cpu).  The reference's installed tree (``baseline/_ref``, or
    MQ_REFERENCE_TREE) runs under the numpy ``mlx.core`` stand-in; without
    it, the oracle's restatement of the same path is timed instead
    (kind "port").  Returns (seconds, sample description, threads, kind)."""
    from collections import Counter
    from oracle import refcpu
    ops, _ = circuit.ops()
    counts = Counter(op["name"] for op in ops)
    dev_cls = refcpu.load_reference_device(REFERENCE_TREE)
    kind = "reference" if dev_cls is not None else "port"
    if dev_cls is None:
        dev_cls = refcpu.PortDevice
    times, T, nl = refcpu.time_reference_gates(dev_cls, sorted(counts), n_cpu, threads, repeats)
    total = refcpu.extrapolate(counts, times, n_target, n_cpu)
    who = ("the reference's Device(n, execution_device='cpu').execute (MettleQ 0.3.1 under the numpy mlx.core "
           "stand-in)" if kind == "reference" else "the oracle's restatement of the reference's per-gate CPU path")
    split = f" as {T} chunks of {nl} qubits on {T} threads" if T > 1 else " on one thread"
    sample = (f"{who}: one gate of each name at n={n_cpu}{split}, best of {repeats}; x2^{n_target - n_cpu} per gate "
              f"to n={n_target}, summed over the circuit's {len(ops)} gates "
              f"({', '.join(f'{k} {v}' for k, v in sorted(counts.items()))}; the GF(2) layers by their "
              "Gauss-Jordan CNOT/SWAP/X synthesis)")
    return total, sample, T, kind


def scale_config(n: int, layers: int, logical: int, world: int) -> dict:
    """The workload description both arms print (identical for one N)."""
    return {"workload": f"scale: {n} qubits complex64, {layers} layers of U(2)+RZZ chain+CNOT ladder, "
                        f"QFT + random GF(2) layer after every 10th",
            "qubits": n, "layers": layers, "logical_layers_per_step": logical,
            "state_bytes": (1 << n) * 8, "l2": f"inputs larger than L2 ({(1 << n) * 8 / 2 ** 30:g} GiB state vs 126 MB L2)",
            "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------- fidelity
class _DeviceArray:
    """A device buffer of n complex amplitudes as a __cuda_array_interface__
    object (torch.as_tensor wraps it without a copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "strides": None, "version": 3}


def infidelity_vs_c128(sv64, sv128, device) -> float:
    """1 - |<psi64|psi128>|^2 / (<psi64|psi64> <psi128|psi128>) of two device
    states, summed in complex128 on the GPU in chunks of 2^26 amplitudes."""
    import torch
    n = 1 << sv64.n
    a = torch.as_tensor(_DeviceArray(sv64.device_ptr(), n, "<c8"), device=device)
    b = torch.as_tensor(_DeviceArray(sv128.device_ptr(), n, "<c16"), device=device)
    ov = torch.zeros((), dtype=torch.complex128, device=device)
    na = torch.zeros((), dtype=torch.float64, device=device)
    nb = torch.zeros((), dtype=torch.float64, device=device)
    step = 1 << 26
    for s in range(0, n, step):
        x = a[s:s + step].to(torch.complex128)
        y = b[s:s + step]
        ov += torch.vdot(x, y)
        na += torch.vdot(x, x).real
        nb += torch.vdot(y, y).real
    f = (ov.abs() ** 2 / (na * nb)).item()
    return max(0.0, 1.0 - f)


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank, dist):
    import torch
    from mettleq_b200 import workloads as W
    from mettleq_b200.engine import StateVector
    from mettleq_b200.device import Device
    from mettleq_b200.replicas import max_over_ranks

    torch.cuda.set_device(local_rank)
    # a dedicated (non-default) stream: libmq launches on it and the CUDA
    # events that time the kernels are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    n = args.qubits
    circuit = W.scale_circuit(n, args.layers, seed=args.seed)
    logical = circuit.logical_layers()
    state_bytes = (1 << n) * 8
    layer_bytes = 2 * state_bytes

    sv = StateVector(n, "complex64", device=local_rank, stream=stream.cuda_stream)

    # how many k_tile launches one fused config layer takes (planner output)
    from mettleq_b200.fusion import DIAG_ZZ
    L0 = circuit.layers[0]
    l0, s0 = sv.counters()
    sv.apply_layer(L0.mats, None, [(DIAG_ZZ, i, i + 1, [t / 2.0]) for i, t in enumerate(L0.thetas)],
                   *W.cnot_ladder_rows(n))
    l1, s1 = sv.counters()
    layer_launches = l1 - l0
    sv.synchronize()

    def step(record=None):
        sv.reset()
        W.run_circuit_layers(sv, circuit, on_layer=record)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    # timed region: per-layer-type events on the launching stream
    kinds = ("layer", "xor", "qft")
    spans = {k: [] for k in kinds}
    pending = {}

    def record(kind, edge):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        if edge == 0:
            pending[kind] = ev
        else:
            spans[kind].append((pending.pop(kind), ev))

    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    c0 = sv.counters()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step(record)
    end.record(stream)
    torch.cuda.synchronize()
    c1 = sv.counters()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    elapsed = max_over_ranks(start.elapsed_time(end) / 1000.0, dist, device="cuda")
    per_kind = {k: sum(a.elapsed_time(b) for a, b in v) / 1000.0 for k, v in spans.items()}
    counts = {k: len(v) for k, v in spans.items()}
    launches = c1[0] - c0[0]
    sweeps = c1[1] - c0[1]

    # accuracy of the timed result (untimed): the same circuit in complex128
    infid = None
    if not args.no_infidelity:
        sv128 = StateVector(n, "complex128", device=local_rank, stream=stream.cuda_stream)
        W.run_circuit_layers(sv128, circuit)
        torch.cuda.synchronize()
        infid = infidelity_vs_c128(sv, sv128, f"cuda:{local_rank}")
        sv128.close()

    value = world * args.steps * logical * layer_bytes / elapsed / 1e9
    peak, peak_kind = measured_peaks()
    # dominant kernel: the tile sweep of the fused config layers (every launch
    # of a layer is a k_tile sweep: U(2) groups, the last one carrying the
    # RZZ diagonal and the CNOT-ladder permutation)
    layer_total = per_kind["layer"]
    n_layer_launch = counts["layer"] * layer_launches
    avg_launch = layer_total / max(1, n_layer_launch)
    achieved = layer_bytes / avg_launch / 1e9
    breakdown = {}
    for k in kinds:
        if counts[k]:
            breakdown[k] = {
                "layers": counts[k] // args.steps,
                "ms_per_layer": per_kind[k] / counts[k] * 1e3,
                "layer_GBps": (3 if k == "layer" else 1) * layer_bytes * counts[k] / per_kind[k] / 1e9,
            }
    breakdown["layer"]["sweeps_per_layer"] = layer_launches
    breakdown["layer"]["logical_layers_each"] = 3
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                traffic = json.load(f).get("k_tile_bytes_per_launch")
        except Exception:
            traffic = None

    out = {
        "metric": "30q layer GB/s",
        "value": value,
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(3, args.warmup),
        "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64",
        "data": "synthetic (seeded Haar U(2), RZZ angles, random GF(2) layers)",
        "config": scale_config(n, args.layers, logical, world),
        "layer_breakdown": breakdown,
        "sweeps_per_step": sweeps / args.steps,
        "infidelity_vs_c128": infid,
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_tile (sweep of the fused U(2)+RZZ+CNOT-ladder layer)",
                     "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                     else "fallback 6650 GB/s",
                     "algorithmic_bytes_per_launch": layer_bytes,
                     "avg_launch_ms": avg_launch * 1e3},
        "clocks": clk,
    }

    # end to end through the public API: op dicts -> Device.execute (fusion +
    # kernels) -> global phase -> 1000 seeded shots read back to the host
    if not args.no_e2e:
        ops, gphase = circuit.ops()
        dev = Device(n, shots=args.shots, stream=stream.cuda_stream)
        from mettleq_b200.integrations import _common as C

        def e2e_step(i):
            dev.reset()
            dev.execute(ops)
            C.apply_global_phase(dev, gphase)
            return dev.sim.sample_indices(args.shots, seed=1234 + i)

        e2e_step(0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        k = max(1, args.steps)  # as many steps as the device-resident timing
        p0 = dev.sim.param_bytes
        e0.record(stream)
        for i in range(k):
            e2e_step(i + 1)
        e1.record(stream)
        torch.cuda.synchronize()
        te = max_over_ranks(e0.elapsed_time(e1) / 1000.0, dist, device="cuda")
        h2d = (dev.sim.param_bytes - p0) / k
        out["e2e"] = {"value": world * k * logical * layer_bytes / te / 1e9, "unit": "GB/s",
                      "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(args.shots * 8 + 16),
                      "ms_per_step": te / k * 1e3,
                      "path": "integrations._common.execute_operations-equivalent: Device.execute(op dicts) + "
                              "apply_global_phase + seeded sample of all qubits"}
        dev.close()
    sv.close()

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_cpu = min(args.cpu_qubits, n)
        t_cpu, sample, used, kind = cpu_baseline_sample(n, n_cpu, circuit, threads=cpu_threads())
        out["cpu_baseline"] = {"value": logical * layer_bytes / t_cpu / 1e9, "unit": "GB/s", "cores": used,
                               "kind": kind, "sample": sample, "extrapolated_circuit_s": t_cpu}
    return out


# ---------------------------------------------------------------- other workloads
def _timed_clocks(fn, index: int = 0):
    clocks = ClockSampler(index)
    clocks.start()
    try:
        r = fn()
    finally:
        clk = clocks.stop()
    return r, clk


def run_batch(args, count=None, steps=None, device: int = 0, indices=None, plain: bool = True):
    """Hardware-efficient-ansatz circuits (n ~ U{10..24}, depth ~ U{4..16},
    RY/RZ angles U[-pi, pi], CNOT ladder), complex64, in one CUDA-graph launch
    per batch; beside it the plain path (one circuit at a time through
    Device.execute) on a sample of the same circuits.  Both produce the same
    outputs: every probability vector in device memory, <Z_0> read back to
    the host.  ``indices`` selects this process's circuits of the batch (one
    rank's share)."""
    import torch
    from mettleq_b200.batch import CircuitBatch, autotune, hea_batch, hea_mats, hea_ops
    from mettleq_b200.device import Device
    count = count or args.count or 4096
    steps = steps or args.steps
    ns, ds, ps = hea_batch(count, seed=args.seed)
    if indices is not None:
        ns, ds, ps = [ns[i] for i in indices], [ds[i] for i in indices], [ps[i] for i in indices]
    mine = len(ns)
    mats = [hea_mats(p) for p in ps]
    sub = list(range(0, mine, max(1, mine // 512)))
    b0 = CircuitBatch([ns[i] for i in sub], [ds[i] for i in sub], device=device)
    packed_sub = b0.pack([mats[i] for i in sub])
    b0.close()
    t0 = time.perf_counter()
    tune = autotune([ns[i] for i in sub], [ds[i] for i in sub], packed_sub, device=device)
    tune_s = time.perf_counter() - t0
    b = CircuitBatch(ns, ds, lanes=tune["lanes"], small_threads=tune["small_threads"], device=device,
                     tiles=tune.get("tiles"))
    packed = b.pack(mats)
    t0 = time.perf_counter()
    b.run(packed=packed)
    b.synchronize()
    capture_s = time.perf_counter() - t0
    for _ in range(max(0, args.warmup - 1)):
        b.run(packed=packed)
    b.synchronize()

    def timed():
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            b.run(packed=packed)   # host copy of the matrices + graph launch
            z = b.z0()             # <Z_0> of every circuit to the host
            ts.append(time.perf_counter() - t0)
        return ts, z

    (ts, z0), clk = _timed_clocks(timed, device)
    t_run = statistics.median(ts)
    # plain path on a sample: Device.execute, the probability vector into
    # device memory, <Z_0> to the host
    sample = list(range(0, mine, max(1, mine // 256))) if plain else []
    devs = {}
    buf = torch.empty(1 << max([ns[i] for i in sample] + [1]), dtype=torch.float32, device=f"cuda:{device}")
    err = 0.0
    t0 = time.perf_counter()
    for i in sample:
        n = ns[i]
        d = devs.get(n)
        if d is None:
            d = devs[n] = Device(n, device_index=device)
        else:
            d.reset()
        d.execute(hea_ops(ps[i]))
        d.sim.probabilities_to_device(buf.data_ptr())
        z = float(d.sim.expval_pauli([{0: "Z"}])[0].real)
        err = max(err, abs(z - z0[i]))
    t_plain = time.perf_counter() - t0
    for d in devs.values():
        d.close()
    n_small, n_large = b.n_small, b.n_large
    b.close()
    plain_cps = len(sample) / t_plain if sample else None
    value = mine / t_run
    return {
        "metric": "batched circuits/s", "value": value, "unit": "circuits/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t_run * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded hardware-efficient ansatz)",
        "config": {"workload": f"batch: {count} circuits, n ~ U{{10..24}}, depth ~ U{{4..16}}, RY+RZ on every qubit "
                               "then CNOT ladder; outputs <Z_0> (to host) and full probabilities (float32, on device)",
                   "circuits": mine, "sum_state_GB": sum((1 << n) * 8 for n in ns) / 1e9, "small_circuits": n_small,
                   "large_circuits": n_large},
        "step": "host copy of all matrices + one CUDA-graph launch + <Z_0> of every circuit to the host "
                "(graph captured once, untimed)",
        "capture_first_run_s": capture_s, "autotune": dict(tune, seconds=tune_s),
        "plain": {"circuits_per_s": plain_cps, "sample": len(sample),
                  "path": "one circuit at a time: Device.execute(op dicts) + probabilities into device memory "
                          "+ <Z_0> to the host; Devices cached per width"},
        "speedup_vs_plain": value / plain_cps if plain_cps else None, "z0_max_diff_vs_plain": err, "clocks": clk,
    }


def run_adjoint(args, steps=None):
    """Adjoint gradient of E = <H>, H = sum Z_i Z_{i+1} + 0.5 sum X_i, for 8
    layers of RY+RZ on 24 qubits + CNOT ladder (384 parameters), complex64,
    against one forward pass (circuit + energy)."""
    import torch
    from mettleq_b200.adjoint import AdjointEngine, LayeredAnsatz, PauliSum
    steps = steps or args.steps
    n = 24 if args.qubits == 30 else args.qubits
    A = LayeredAnsatz(n, 8)
    H = PauliSum.ising_chain(n)
    p = np.random.default_rng(args.seed).uniform(-math.pi, math.pi, A.shape)
    stream = torch.cuda.Stream()
    eng = AdjointEngine(A, H, dtype="complex64", stream=stream.cuda_stream)

    def t(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts)

    def measure():
        return t(lambda: eng.energy(p)), t(lambda: eng.energy_and_grad(p))

    (tf, tg), clk = _timed_clocks(measure)
    e, g = eng.energy_and_grad(p)
    # spot check against the parameter-shift rule on the same engine
    flat = p.reshape(-1)
    idx = [0, 100, 200, 383]
    ps_err = 0.0
    for i in idx:
        q = flat.copy()
        q[i] += math.pi / 2
        ep = eng.energy(q.reshape(A.shape))
        q[i] -= math.pi
        em = eng.energy(q.reshape(A.shape))
        ps_err = max(ps_err, abs(0.5 * (ep - em) - g.reshape(-1)[i]))
    eng.close()
    return {
        "metric": "adjoint gradient time / forward time", "value": (tg - tf) / tf, "unit": "x",
        "n_gpus": 1, "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": tg * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
        "config": {"workload": f"adjoint: {n} qubits, 8 layers RY+RZ + CNOT ladder ({p.size} parameters), "
                               "H = sum Z_i Z_i+1 + 0.5 sum X_i"},
        "forward_ms": tf * 1e3, "forward_plus_gradient_ms": tg * 1e3, "gradient_only_ms": (tg - tf) * 1e3,
        "total_over_forward": tg / tf, "energy": e, "param_shift_max_diff": ps_err, "clocks": clk,
    }


def run_serve(args, count=None):
    """Poisson stream at 200 requests/s, n log-uniform in [12, 30], depth
    U{10..100} config-0 layers (QFT and GF(2) layer each with p = 0.1), 1000
    shots, complex64, 150 GB admission budget; beside it the plain path (one
    request at a time through Device.execute, Devices cached per width) on
    the same stream, and the device time of every request run alone (the
    lower bound of any schedule's busy time)."""
    from mettleq_b200.serving import Server, device_work, poisson_requests, serve_plain
    count = count or args.count or 200
    reqs = poisson_requests(count, rate=200.0, seed=args.seed)
    srv = Server(budget_bytes=150 * 10 ** 9)
    srv.serve(poisson_requests(8, seed=99, n_range=(12, 16), depth_range=(2, 3)), realtime=False)
    stats, clk = _timed_clocks(lambda: srv.serve(reqs, realtime=True))
    peak, active = srv.peak_used, srv.peak_active
    srv.close()
    work = device_work(reqs)
    busy = float(sum(work))
    plain = serve_plain(poisson_requests(count, rate=200.0, seed=args.seed), realtime=True)
    last_arrival = max(r.arrival for r in reqs)
    return {
        "metric": "serve p50 latency", "value": stats["p50_s"], "unit": "s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": stats["makespan_s"] * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded Poisson request stream)",
        "config": {"workload": f"serve: {count} requests, Poisson 200 req/s, n log-uniform 12..30, depth U{{10..100}}, "
                               "QFT/XOR p=0.1, 1000 shots, 150 GB budget"},
        "p99_s": stats["p99_s"], "mean_s": stats["mean_s"], "circuits_per_s": stats["circuits_per_s"],
        "makespan_s": stats["makespan_s"], "peak_admitted_GB": peak / 1e9, "peak_active": active,
        "device_work_alone_s": busy,
        "device_busy_fraction": busy / stats["makespan_s"],
        "makespan_floor_s": max(busy, last_arrival),
        "plain": dict(plain, path="one request at a time: Device.execute(op dicts) + seeded shots, Devices cached "
                                  "per width"),
        "throughput_vs_plain": stats["circuits_per_s"] / plain["circuits_per_s"],
        "throughput_ceiling_vs_plain": plain["makespan_s"] / max(busy, last_arrival),
        "clocks": clk,
    }


def compact(d: dict, keys) -> dict:
    return {k: d[k] for k in keys if k in d}


def run_batch_ranks(args, rank, world, local_rank, dist):
    """The batch over N GPUs: each rank runs its share (longest-processing-
    time split by depth x 2^n) as its own captured graph; value = all
    circuits over the slowest rank's median step."""
    from mettleq_b200.batch import hea_batch
    from mettleq_b200.replicas import gather_objects, max_over_ranks, partition_by_cost
    count = args.count or 4096
    ns, ds, _ = hea_batch(count, seed=args.seed)
    mine = partition_by_cost([d << n for n, d in zip(ns, ds)], world)[rank]
    dist.barrier()
    r = run_batch(args, count=count, indices=mine, device=local_rank, plain=False)
    t = max_over_ranks(r["ms_per_step"] / 1e3, dist, device=f"cuda:{local_rank}")
    shares = gather_objects(len(mine), dist)
    r.update({"value": count / t, "n_gpus": world, "ms_per_step": t * 1e3, "scaling": "strong",
              "circuits_per_rank": shares, "parallelism": f"replicas x{world}"})
    r["config"]["circuits"] = count
    return r


def run_serve_ranks(args, rank, world, local_rank, dist):
    """The request stream over N GPUs at N x 200 requests/s (weak scaling):
    one queue per GPU (``assign_by_work``: each arrival to the GPU with the
    least work so far), a Server per rank, latencies gathered to rank 0."""
    from mettleq_b200.replicas import gather_objects, max_over_ranks
    from mettleq_b200.serving import Server, assign_by_work, poisson_requests
    count = (args.count or 200) * world
    reqs = poisson_requests(count, rate=200.0 * world, seed=args.seed)
    mine = [reqs[i] for i in assign_by_work(reqs, world)[rank]]
    srv = Server(budget_bytes=150 * 10 ** 9, device=local_rank)
    srv.serve(poisson_requests(8, seed=99, n_range=(12, 16), depth_range=(2, 3)), realtime=False)
    dist.barrier()
    stats, clk = _timed_clocks(lambda: srv.serve(mine, realtime=True), local_rank)
    srv.close()
    makespan = max_over_ranks(stats["makespan_s"], dist, device=f"cuda:{local_rank}")
    lat = np.concatenate([np.asarray(x) for x in gather_objects([r.latency for r in mine], dist)])
    return {
        "metric": "serve p50 latency", "value": float(np.percentile(lat, 50)), "unit": "s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": makespan * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded Poisson request stream)",
        "config": {"workload": f"serve: {count} requests, Poisson {200 * world} req/s over {world} GPUs (one queue "
                               "each), n log-uniform 12..30, depth U{10..100}, QFT/XOR p=0.1, 1000 shots, "
                               "150 GB budget per GPU"},
        "p99_s": float(np.percentile(lat, 99)), "circuits_per_s": count / makespan, "makespan_s": makespan,
        "requests_per_rank": gather_objects(len(mine), dist), "clocks": clk,
    }


def run_sharded(args, rank, world, local_rank, dist):
    """One state sharded over the N ranks: n = qubits-per-GPU + log2 N
    (8 GiB of complex64 per GPU at 30), layers of the scale structure (Haar
    U(2) on every qubit, RZZ chain, CNOT ladder); a layer touching global
    qubits swaps them with local ones by one all-to-all, the ladder remaps
    whole shards between ranks.  Time: CUDA events on each rank's shard
    stream, max over ranks."""
    import torch
    from mettleq_b200 import workloads as W
    from mettleq_b200.fusion import DIAG_ZZ
    from mettleq_b200.replicas import gather_objects, max_over_ranks
    from mettleq_b200.sharded import GpuShard, ShardedState
    g = int(round(math.log2(world)))
    n = args.qubits + g
    layers = min(args.layers, 10)
    circuit = W.plain_circuit(n, layers, seed=args.seed)
    shard = GpuShard(n - g, "complex64", device=local_rank)
    st = ShardedState(n, shard, dist if world > 1 else None)
    ladder = W.cnot_ladder_rows(n)
    terms = [[(DIAG_ZZ, i, i + 1, [float(t) / 2.0]) for i, t in enumerate(L.thetas)] for L in circuit.layers]

    def step():
        st.reset()
        for L, tm in zip(circuit.layers, terms):
            st.apply_layer(L.mats, None, tm, *ladder)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ex0, rm0, by0 = st.exchanges, st.remaps, st.bytes_sent
    l0 = shard.sv.counters()[0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0.record(shard.stream)
    for _ in range(args.steps):
        step()
    e1.record(shard.stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist is not None:
        dist.barrier()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, device=f"cuda:{local_rank}")
    sent = gather_objects((st.bytes_sent - by0) / args.steps, dist)
    launches = shard.sv.counters()[0] - l0
    logical = 3 * layers
    total_bytes = (1 << n) * 8
    shard.close()
    return {
        "metric": "sharded layer GB/s", "value": args.steps * logical * 2 * total_bytes / t / 1e9, "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (seeded Haar U(2), RZZ angles)",
        "config": {"workload": f"sharded: {n} qubits complex64 over {world} GPU(s) ({n - g} local qubits each), "
                               f"{layers} layers of U(2)+RZZ chain+CNOT ladder",
                   "qubits": n, "global_qubits": g, "layers": layers, "logical_layers_per_step": logical,
                   "state_bytes": total_bytes, "parallelism": f"sharded x{world}"},
        "exchanges_per_step": (st.exchanges - ex0) / args.steps, "remaps_per_step": (st.remaps - rm0) / args.steps,
        "bytes_sent_per_rank_per_step": sent, "gpu_launches": launches, "clocks": clk,
    }


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    from mettleq_b200 import workloads as W
    n = args.qubits
    circuit = W.scale_circuit(n, args.layers, seed=args.seed)
    logical = circuit.logical_layers()
    layer_bytes = 2 * (1 << n) * 8
    n_cpu = min(args.cpu_qubits, n)
    threads = cpu_threads()
    # warm-up: builds the chunk devices and runs every gate once; the timed
    # steps reuse them
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_baseline_sample(n, n_cpu, circuit, threads=threads)
    times, walls = [], []
    used, kind, sample = 1, "port", ""
    for _ in range(max(1, args.steps)):
        w0 = time.perf_counter()
        t_cpu, sample, used, kind = cpu_baseline_sample(n, n_cpu, circuit, threads=threads)
        walls.append(time.perf_counter() - w0)
        times.append(t_cpu)
    t = statistics.median(times)
    value = logical * layer_bytes / t / 1e9
    return {
        "metric": "30q layer GB/s", "value": value, "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded Haar U(2), RZZ angles, random GF(2) layers)",
        "config": scale_config(n, args.layers, logical, world=1),
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": used, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        # one step = one timed sample (its wall time); the metric is the
        # full circuit's time extrapolated from it
        "ms_per_step": statistics.median(walls) * 1e3, "extrapolated_circuit_ms": t * 1e3,
    }


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0
    if world == 1 and args.workload in ("batch", "adjoint", "serve"):
        fn = {"batch": run_batch, "adjoint": run_adjoint, "serve": run_serve}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return 0
    if args.workload == "adjoint":
        # one gradient job: rank 0 alone
        if rank == 0:
            import torch
            torch.cuda.set_device(local_rank)
            print(json.dumps(run_adjoint(args)), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = td
    try:
        if args.workload != "scale":
            fn = {"batch": run_batch_ranks, "serve": run_serve_ranks, "sharded": run_sharded}[args.workload]
            out = fn(args, rank, world, local_rank, dist)
            if rank == 0:
                print(json.dumps(out), flush=True)
            return 0
        out = run_ours(args, rank, world, local_rank, dist)
        if rank == 0 and world == 1 and not args.no_extras:
            # the metric's other two parts on the same GPU, bounded in size:
            # batched circuits/s and serve p50/p99 against their plain paths,
            # and the adjoint gradient against one forward pass
            import torch
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            bt = run_batch(args, count=1024, steps=5)
            out["batch"] = compact(bt, ("value", "unit", "ms_per_step", "speedup_vs_plain", "plain", "autotune",
                                        "z0_max_diff_vs_plain", "config", "clocks"))
            torch.cuda.empty_cache()
            ad = run_adjoint(args, steps=5)
            out["adjoint"] = compact(ad, ("value", "unit", "forward_ms", "forward_plus_gradient_ms",
                                          "gradient_only_ms", "param_shift_max_diff", "config", "clocks"))
            torch.cuda.empty_cache()
            sv = run_serve(args, count=200)
            out["serve"] = compact(sv, ("value", "unit", "p99_s", "circuits_per_s", "makespan_s", "plain",
                                        "throughput_vs_plain", "device_work_alone_s", "device_busy_fraction",
                                        "makespan_floor_s", "throughput_ceiling_vs_plain", "peak_admitted_GB",
                                        "peak_active", "config", "clocks"))
            out["serve"]["p50_s"] = sv["value"]
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
