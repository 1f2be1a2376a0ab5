"""The CPU oracle pinned against the reference (CPU only).

* tests/golden/reference_outputs.npz + cases.json were produced by running
  the reference's own ``Device(n, execution_device="cpu")`` code
  (device.py:1138-1290, sim.py) through a numpy ``mlx.core`` stand-in; see
  tests/golden/make_golden.py.  Tolerance 5e-6 is the reference's own
  Metal-vs-MLX parity budget (src/tests/mlxQMetalKernelsTest.py).
* The independent QFT matrix without final swaps
  (src/tests/mlxQQmlQftSubsetTest.py:41-66), the affine-inverse property test
  (src/tests/mlxQMetalKernelsTest.py:293-323) and core identities
  (src/tests/mlxQCoreTest.py) are restated here against the oracle.
* Philox4x32-10 against the Random123 known-answer vectors.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import OracleSim, compose_inverse_affine, gate_matrix, qft_matrix_without_swaps
from oracle import sampler as S

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ref():
    return np.load(os.path.join(GOLDEN, "reference_outputs.npz"))


@pytest.fixture(scope="module")
def device_states(ref):
    out = {}
    for c in _cases():
        if c["kind"] == "device":
            o = OracleSim(c["n"], np.complex128)
            o.execute(c["ops"])
            o.apply_global_phase(c["global_phase"])
            out[c["tag"]] = o
    return out


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_device_streams_match_reference(ref, dtype):
    for c in _cases():
        if c["kind"] != "device":
            continue
        o = OracleSim(c["n"], dtype)
        o.execute(c["ops"])
        o.apply_global_phase(c["global_phase"])
        assert np.max(np.abs(o.state - ref[c["tag"]])) < 5e-6, c["tag"]


def test_probabilities_match_reference(ref, device_states):
    for c in _cases():
        if c["kind"] == "probs":
            got = device_states[c["source"]].probabilities(c["wires"])
            assert np.max(np.abs(got - ref[c["tag"]])) < 5e-6, c["tag"]


def test_pauli_expectations_match_reference(ref, device_states):
    for c in _cases():
        if c["kind"] == "pauli":
            o = device_states[c["source"]]
            got = np.array([o.pauli_expectation({int(k): v for k, v in w.items()}) for w in c["words"]])
            assert np.max(np.abs(got - ref[c["tag"]])) < 5e-6


def test_qft_matches_reference_runs(ref):
    for c in _cases():
        if c["kind"] == "qft":
            o = OracleSim(c["n"], np.complex128)
            o.set_state(ref[c["tag"] + "_in"])
            (o.iqft if c["inverse"] else o.qft)(c["wires"])
            assert np.max(np.abs(o.state - ref[c["tag"] + "_out"])) < 5e-6


def test_affine_composition_matches_reference():
    for c in _cases():
        if c["kind"] == "affine":
            assert compose_inverse_affine(c["ops"], c["n"]) == (c["rows"], c["c"])


def _apply_reference_qft(vec, n, wires, inverse=False):
    gate = qft_matrix_without_swaps(len(wires))
    if inverse:
        gate = gate.conj().T
    rest = [w for w in range(n) if w not in wires]
    perm = rest + list(wires)
    m = vec.reshape([2] * n).transpose(perm).reshape(1 << (n - len(wires)), 1 << len(wires))
    out = (m @ gate.T).reshape([2] * n).transpose(np.argsort(perm))
    return out.reshape(-1)


@pytest.mark.parametrize("wires", [(0, 1, 2, 3), (2, 0), (3, 1, 0)])
def test_qft_independent_matrix_golden(wires):
    # src/tests/mlxQQmlQftSubsetTest.py:75-94
    n = 4
    rng = np.random.default_rng(208)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    o = OracleSim(n, np.complex128)
    o.set_state(v)
    o.qft(list(wires))
    assert np.max(np.abs(o.state - _apply_reference_qft(v, n, wires))) < 2e-12
    o.iqft(list(wires))
    assert np.max(np.abs(o.state - v)) < 2e-12


def test_affine_inverse_property():
    # src/tests/mlxQMetalKernelsTest.py:293-323 (seeded default_rng(4))
    n = 6
    ops = ([{"name": "CNOT", "wires": [q, q + 1]} for q in range(n - 1)]
           + [{"name": "X", "wires": [3]}, {"name": "SWAP", "wires": [0, 5]}, {"name": "CNOT", "wires": [4, 1]}])
    rows, c = compose_inverse_affine(ops, n)

    def forward(x):
        bits = [(x >> (n - 1 - q)) & 1 for q in range(n)]
        for op in ops:
            w = op["wires"]
            if op["name"] == "X":
                bits[w[0]] ^= 1
            elif op["name"] == "CNOT":
                bits[w[1]] ^= bits[w[0]]
            else:
                bits[w[0]], bits[w[1]] = bits[w[1]], bits[w[0]]
        return sum(b << (n - 1 - q) for q, b in enumerate(bits))

    def inverse(y):
        src = 0
        for k in range(n):
            src |= (bin(rows[k] & y).count("1") & 1) << (n - 1 - k)
        return src ^ c

    rng = np.random.default_rng(4)
    for x in rng.integers(0, 1 << n, size=32):
        assert inverse(forward(int(x))) == int(x)


def test_core_identities():
    # mlxQCoreTest.py: CPHASE(pi) = CZ, U3/U2 decompositions, RZ(2pi) = -I
    s1, s2 = OracleSim(2), OracleSim(2)
    for s in (s1, s2):
        s.apply_single(gate_matrix("H"), 0)
        s.apply_single(gate_matrix("H"), 1)
    s1.apply_op({"name": "CPHASE", "wires": [0, 1], "parameters": [math.pi]})
    s2.apply_op({"name": "CZ", "wires": [0, 1], "parameters": []})
    assert np.max(np.abs(s1.state - s2.state)) < 1e-6
    assert np.allclose(gate_matrix("U2", [0.3, -0.7]), gate_matrix("U3", [math.pi / 2, 0.3, -0.7]))
    assert np.allclose(gate_matrix("RZ", [2 * math.pi]), -np.eye(2))
    # Bell state expectations (mlxQCoreTest.py:817-835)
    b = OracleSim(2, np.complex128)
    b.apply_single(gate_matrix("H"), 0)
    b.apply_op({"name": "CNOT", "wires": [0, 1], "parameters": []})
    assert abs(b.pauli_expectation({0: "Z", 1: "Z"}) - 1) < 1e-12
    assert abs(b.pauli_expectation({0: "X", 1: "X"}) - 1) < 1e-12
    assert abs(b.pauli_expectation({0: "Y", 1: "Y"}) + 1) < 1e-12
    assert abs(b.pauli_expectation({0: "Z"})) < 1e-12


def test_parameter_shift_gradient_kat():
    # mlxQSdkIntegrationsTest.py:182-192: d<Z>/dtheta of RX(0.4) = -sin(0.4)
    def f(t):
        o = OracleSim(1, np.complex128)
        o.apply_single(gate_matrix("RX", [t]), 0)
        return o.pauli_expectation({0: "Z"}).real
    g = 0.5 * (f(0.4 + math.pi / 2) - f(0.4 - math.pi / 2))
    assert abs(g + math.sin(0.4)) < 2e-12


def test_philox_known_answers():
    # Random123 kat_vectors, philox4x32_10
    def run(ctr, key):
        r = S.philox4x32_10(np.array([ctr], dtype=np.uint32), np.array([key], dtype=np.uint32))[0]
        return [int(x) for x in r]
    assert run([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert run([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert run([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_sampler_distribution_matches_probabilities():
    rng = np.random.default_rng(5)
    p = rng.random(64)
    idx = S.sample_indices(p, seed=3, shots=20000)
    freq = np.bincount(idx, minlength=64) / 20000
    assert np.max(np.abs(freq - p / p.sum())) < 0.01
    # zero-probability entries are never drawn
    p[::2] = 0.0
    idx = S.sample_indices(p, seed=4, shots=5000)
    assert np.all(idx % 2 == 1)
    # deterministic per (seed, offset), shots are a prefix-stable stream
    a = S.sample_indices(p, seed=9, shots=100, stream_offset=0)
    b = S.sample_indices(p, seed=9, shots=50, stream_offset=50)
    assert np.array_equal(a[50:], b)


def test_marginal_order_first_wire_msb():
    o = OracleSim(3, np.complex128)
    o.apply_single(gate_matrix("X"), 0)  # |100>
    p = S.amp2(o.state)
    m = S.marginal_probabilities(p, 3, [2, 0])
    assert np.allclose(m, [0, 1, 0, 0])


def _chi2_pvalue(counts, probs):
    from scipy.stats import chi2
    shots = counts.sum()
    keep = probs * shots >= 5.0          # pool the sparse tail into one bin
    obs = np.append(counts[keep], counts[~keep].sum())
    exp = np.append(probs[keep] * shots, probs[~keep].sum() * shots)
    m = exp > 0
    stat = float(np.sum((obs[m] - exp[m]) ** 2 / exp[m]))
    return float(chi2.sf(stat, int(m.sum()) - 1))


def test_sampled_counts_agree_with_reference_probabilities(ref):
    """MLX's generator cannot run here, so counts are compared in distribution:
    1000 shots of the project's seeded stream on the reference's own state
    (layers_uniform) against the reference's exact probabilities (chi-square
    over bins with >= 5 expected counts, the tail pooled)."""
    probs = np.asarray(ref["probs_0_1_2_3_4_5_6_7"], dtype=np.float64)
    probs = probs / probs.sum()
    state = np.asarray(ref["layers_uniform"], dtype=np.complex128)
    for seed in (1, 2, 3):
        idx = S.sample_indices(S.amp2(state), seed, 1000)
        counts = np.bincount(idx, minlength=probs.size).astype(np.float64)
        assert _chi2_pvalue(counts, probs) > 1e-3, seed
