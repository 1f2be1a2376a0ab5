"""The runtime-level drop-in on the GPU.

* The reference's own golden gate streams (tests/golden/cases.json, recorded
  by running ``Device(n, execution_device="cpu")`` of the reference) go
  through ``mettleq_b200.device.Device.execute`` on CUDA in complex64 and
  complex128: every fused-layer family the fusion emits for them runs
  (_LAYER, _U2LISTLAYER, _DIAG with DIAG_2Q from ISWAP, _XORLAYER, _CULIST
  with two controls from TOFFOLI / FREDKIN, the XX/YY basis-change windows,
  CH/CRX/CRY), as do probabilities on wire subsets, Pauli words and QFTs on
  ordered wire subsets.  Tolerances: 5e-6 against the reference's complex64
  outputs (its own Metal-vs-MLX budget, src/tests/mlxQMetalKernelsTest.py),
  1e-5 (complex64) / 1e-12 (complex128) against the complex128 oracle.
* A 16-qubit stream with every one of the 30 gate names plus a forward and
  an inverse QFT spelled as H + CPHASE ladders, against the oracle.
* The reference's SDK measurement helpers (src/mettleq/integrations/
  _common.py:231-288), restated below as the contract of the swap, run
  unchanged against this Device; the package's own helpers
  (mettleq_b200/integrations/_common.py) are checked against the oracle.

This mirrors the reference's two-path parity tests
(src/tests/mlxQMetalKernelsTest.py:26-566): the same ops on both paths.
"""
import json
import math
import os
from collections import Counter

import numpy as np
import pytest

from oracle import OracleSim
from oracle import sampler as S

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
TOL = {"complex64": 1e-5, "complex128": 1e-12}


def _cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ref():
    return np.load(os.path.join(GOLDEN, "reference_outputs.npz"))


def _err(a, b):
    return float(np.max(np.abs(np.asarray(a, np.complex128) - np.asarray(b, np.complex128))))


def _oracle(n, ops, phase=0.0):
    o = OracleSim(n, np.complex128)
    o.execute(ops)
    o.apply_global_phase(phase)
    return o


# ------------------------------------------------------------ golden streams
@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
def test_reference_golden_streams_on_cuda(ref, dtype):
    from mettleq_b200.device import Device
    from mettleq_b200.integrations import _common as C
    seen = Counter()
    for c in _cases():
        if c["kind"] != "device":
            continue
        n = c["n"]
        dev = Device(n, dtype=dtype)
        try:
            from mettleq_b200 import fusion
            for L in fusion.fuse(c["ops"], n):
                seen[L["name"]] += 1
            dev.execute(c["ops"])
            C.apply_global_phase(dev, c["global_phase"])
            got = dev.statevector()
        finally:
            dev.close()
        assert _err(got, ref[c["tag"]]) < 5e-6, c["tag"]
        assert _err(got, _oracle(n, c["ops"], c["global_phase"]).state) <= TOL[dtype], c["tag"]
    # the streams reach every layer family of the runtime
    for name in ("_LAYER", "_U2LISTLAYER", "_DIAG", "_XORLAYER", "_CULIST"):
        assert seen[name] > 0, name


@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
def test_reference_golden_probabilities_and_pauli_words(ref, dtype):
    from mettleq_b200.device import Device
    from mettleq_b200.integrations import _common as C
    cases = {c["tag"]: c for c in _cases()}
    src = cases["layers_uniform"]
    dev = Device(src["n"], dtype=dtype)
    try:
        dev.execute(src["ops"])
        C.apply_global_phase(dev, src["global_phase"])
        for c in cases.values():
            if c["kind"] == "probs":
                got = dev.sim.probabilities_array(c["wires"])
                assert got.dtype == np.float32
                assert np.max(np.abs(got.astype(np.float64) - ref[c["tag"]])) < 5e-6, c["tag"]
            elif c["kind"] == "pauli":
                words = [{int(k): v for k, v in w.items()} for w in c["words"]]
                got = np.array(C.pauli_product_expectations(dev, words))
                assert np.max(np.abs(got - ref[c["tag"]])) < 5e-6, c["tag"]
    finally:
        dev.close()


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_reference_golden_qft_on_ordered_wire_subsets(ref, dtype):
    from mettleq_b200.engine import StateVector
    for c in _cases():
        if c["kind"] != "qft":
            continue
        with StateVector(c["n"], dtype=dtype) as sv:
            sv.set(ref[c["tag"] + "_in"])
            sv.apply_qft(c["wires"], inverse=c["inverse"])
            got = sv.get()
        assert _err(got, ref[c["tag"] + "_out"]) < 5e-6, c["tag"]


# ------------------------------------------------------------ every gate name
def _every_gate_stream(n, rng, count):
    from mettleq_b200.fusion import ARITIES, PARAMS
    names = sorted(ARITIES)
    assert len(names) == 30
    ops = []

    def one(name):
        w = [int(x) for x in rng.choice(n, ARITIES[name], replace=False)]
        p = [float(x) for x in rng.uniform(-math.pi, math.pi, PARAMS.get(name, 0))]
        ops.append({"name": name, "wires": w, "parameters": p})

    for name in names:          # every name at least once, in random order
        one(name)
    rng.shuffle(ops)
    for _ in range(count):
        one(str(rng.choice(names)))
    # a forward QFT on wires 3..8 and an inverse one on wires 9..14, spelled
    # as the SDKs emit them (H + CPHASE ladder; descending negative ladder + H)
    for j in range(3, 9):
        ops.append({"name": "H", "wires": [j], "parameters": []})
        for k in range(j + 1, 9):
            ops.append({"name": "CPHASE", "wires": [k, j], "parameters": [math.pi / (1 << (k - j))]})
    for j in range(14, 8, -1):
        for k in range(14, j, -1):
            ops.append({"name": "CPHASE", "wires": [k, j], "parameters": [-math.pi / (1 << (k - j))]})
        ops.append({"name": "H", "wires": [j], "parameters": []})
    for _ in range(count // 2):
        one(str(rng.choice(names)))
    return ops


@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
def test_every_gate_name_stream_16_qubits(dtype):
    from mettleq_b200 import fusion
    from mettleq_b200.device import Device
    n = 16
    ops = _every_gate_stream(n, np.random.default_rng(31), 240)
    kinds = Counter(L["name"] for L in fusion.fuse(ops, n))
    assert kinds["_QFTSTAGES"] >= 2 and kinds["_CULIST"] > 0 and kinds["_DIAG"] + kinds["_LAYER"] > 0
    dev = Device(n, dtype=dtype)
    try:
        dev.execute(ops)
        got = dev.statevector()
    finally:
        dev.close()
    assert _err(got, _oracle(n, ops).state) <= TOL[dtype]


# ------------------------------------------------------------ the reference's helpers, unchanged
# Restated from src/mettleq/integrations/_common.py:231-288 (statevector
# branches; the MLX type test in marginal_probabilities is left out, there is
# no MLX here).  These are the calls the reference's Qiskit and PennyLane
# adapters make on the Device that execute_operations returns.
def ref_apply_global_phase(device, phase):
    if phase:
        factor = complex(np.cos(float(phase)), np.sin(float(phase)))
        if hasattr(device.sim, "state"):
            device.sim.state = device.sim.state * factor
        else:
            device.sim.A[0] = device.sim.A[0] * factor


def ref_statevector_numpy(device):
    state = device.synchronize()
    if state is not None:
        return np.asarray(state, dtype=np.complex64)
    raise AssertionError("the statevector branch returns the state")


def ref_marginal_probabilities(device, wires):
    device.synchronize()
    probabilities = device.sim.probabilities_array(list(wires))
    result = np.asarray(probabilities, dtype=np.float64)
    total = float(result.sum())
    if total <= 0.0:
        raise RuntimeError("Simulator returned a zero-probability state")
    return result / total


def ref_sample_bits(device, shots, wires, rng):
    wires = list(wires)
    if not wires:
        return np.empty((int(shots), 0), dtype=np.int64)
    device.synchronize()
    if hasattr(device.sim, "sample_array"):
        return np.asarray(device.sim.sample_array(int(shots), wires, rng=rng), dtype=np.int64)
    raise AssertionError("the engine has sample_array")


def ref_bit_counts(samples):
    return dict(Counter("".join(str(int(bit)) for bit in row) for row in samples))


def test_reference_sdk_helpers_run_unchanged_on_the_cuda_device():
    from mettleq_b200.device import Device
    from mettleq_b200 import workloads as W
    n = 12
    circ = W.scale_circuit(n, 3, seed=5, qft_every=2)
    ops, gphase = circ.ops()
    dev = Device(n)
    try:
        dev.execute(ops)
        ref_apply_global_phase(dev, gphase)
        o = _oracle(n, ops, gphase)
        # the phase was applied on the device (one diagonal pass), and the
        # state read back through the reference's conversion
        got = ref_statevector_numpy(dev)
        assert got.dtype == np.complex64 and got.shape == (1 << n,)
        assert _err(got, o.state) <= 1e-5
        for wires in ([0], [5, 2], [11, 0, 7], list(range(n))[::-1], []):
            m = ref_marginal_probabilities(dev, wires)
            want = o.probabilities(wires) if wires else np.array([1.0])
            assert np.max(np.abs(m - want / want.sum())) < 1e-6, wires
        # one uint32 drawn from the caller's generator keys the shot stream
        wires = [3, 9, 1]
        bits = ref_sample_bits(dev, 700, wires, np.random.default_rng(42))
        again = ref_sample_bits(dev, 700, wires, np.random.default_rng(42))
        assert bits.dtype == np.int64 and bits.shape == (700, 3)
        assert np.array_equal(bits, again)
        key = int(np.random.default_rng(42).integers(0, np.iinfo(np.uint32).max, dtype=np.uint32))
        p = S.marginal_probabilities(S.amp2(got), n, wires)
        idx = S.sample_indices(p, key, 700)
        want_bits = (idx[:, None] >> np.arange(2, -1, -1)) & 1
        assert np.array_equal(bits, want_bits)
        counts = ref_bit_counts(bits)
        assert sum(counts.values()) == 700 and all(len(k) == 3 for k in counts)
        assert ref_sample_bits(dev, 5, [], np.random.default_rng(0)).shape == (5, 0)
        # a general complex scalar through the state attribute
        dev.sim.state = dev.sim.state * (0.5 - 0.25j)
        assert _err(np.asarray(dev.synchronize(), dtype=np.complex64), got * (0.5 - 0.25j)) <= 1e-5
        # reading a product leaves the resident state alone
        scaled = np.asarray(dev.sim.state * 2.0)
        assert _err(scaled, 2.0 * dev.statevector()) <= 1e-5
    finally:
        dev.close()


# ------------------------------------------------------------ the package's helpers
def test_execute_operations_cache_across_widths_and_reset():
    from mettleq_b200.integrations import _common as C
    cache = {}
    results = {}
    for n in (5, 9, 5, 9, 7):
        ops = [{"name": "H", "wires": [q], "parameters": []} for q in range(n)]
        ops += [{"name": "RZ", "wires": [n - 1], "parameters": [0.3 * n]}, {"name": "CNOT", "wires": [0, n - 1]}]
        dev = C.execute_operations(n, ops, shots=64, execution_cache=cache)
        # a cached device is reset before it runs again
        got = C.statevector_numpy(dev)
        assert _err(got, _oracle(n, ops).state) <= 1e-5
        if n in results:
            assert dev is results[n]
        results[n] = dev
        assert dev.shots == 64 and dev.execution_selection["selected_method"] == "statevector"
    assert sorted(k[0] for k in cache) == [5, 7, 9]
    for d in cache.values():
        d.close()


def test_package_helpers_against_the_oracle():
    from mettleq_b200.integrations import _common as C
    n = 15
    ops = _every_gate_stream(n, np.random.default_rng(8), 60)
    dev = C.execute_operations(n, ops)
    try:
        o = _oracle(n, ops)
        got = C.statevector_numpy(dev)
        assert _err(got, o.state) <= 1e-5
        # marginals renormalised in float64
        for wires in ([2], [7, 0, 4], [9, 8, 7, 6]):
            m = C.marginal_probabilities(dev, wires)
            assert abs(m.sum() - 1.0) < 1e-12
            want = o.probabilities(wires)
            assert np.max(np.abs(m - want / want.sum())) < 1e-6
        # sample_bits: one uint32 from the caller's generator, bit-exact
        # against the oracle's stream for that key
        wires = [6, 1]
        b1 = C.sample_bits(dev, 1000, wires, np.random.default_rng(11))
        b2 = C.sample_bits(dev, 1000, wires, np.random.default_rng(11))
        assert np.array_equal(b1, b2)
        key = C.draw_seed(np.random.default_rng(11))
        idx = S.sample_indices(S.marginal_probabilities(S.amp2(got), n, wires), key, 1000)
        assert np.array_equal(b1, (idx[:, None] >> np.array([1, 0])) & 1)
        counts = C.bit_counts(b1)
        assert sum(counts.values()) == 1000 and set(counts) <= {"00", "01", "10", "11"}
        # local_expectation of a random 2-qubit Hermitian M (through its
        # Pauli decomposition on the GPU) against <psi|M|psi> on the host
        rng = np.random.default_rng(19)
        a = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
        M = a + a.conj().T
        for wires in ([3, 8], [8, 3], [0, 9]):
            val = C.local_expectation(dev, wires, M)
            psi = o.state.reshape([2] * n)
            rest = [q for q in range(n) if q not in wires]
            t = np.transpose(psi, wires + rest).reshape(4, -1)
            want = np.vdot(t, M @ t)
            assert abs(val - want) < 2e-5, wires
        # Pauli words (the complex64 state after ~130 gates keeps its norm to
        # ~2e-6, so expectations are held to the amplitude bar, 1e-5)
        words = [{0: "Z"}, {1: "X", 4: "Y"}, {2: "Y", 3: "Y", 9: "Z"}, {}]
        vals = C.pauli_product_expectations(dev, words)
        for w, v in zip(words, vals):
            assert abs(v - o.pauli_expectation(w)) < 1e-5, w
    finally:
        dev.close()
