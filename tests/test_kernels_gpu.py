"""CUDA kernels vs the CPU oracle, through the C ABI (kernel-level API).

Tolerances: max |amplitude error| <= 1e-5 in complex64 and <= 1e-12 in
complex128; the permutation layer and sampling are bit-exact.  The reference
asserts 5e-6 between its Metal and MLX paths (src/tests/mlxQMetalKernelsTest.py).
"""
import math

import numpy as np
import pytest

from oracle import OracleSim, compose_inverse_affine
from oracle import sampler as osamp
from tests.helpers import haar_u2, oracle_apply_terms, rand_state, random_invertible_rows

pytestmark = pytest.mark.gpu

TOL = {np.complex64: 1e-5, np.complex128: 1e-12}


def _sv(n, dtype, vec=None):
    from mettleq_b200.engine import StateVector
    sv = StateVector(n, dtype=dtype)
    if vec is not None:
        sv.set(vec)
    return sv


def _oracle(n, dtype, vec):
    o = OracleSim(n, dtype)
    o.set_state(vec)
    return o


def _err(a, b):
    return float(np.max(np.abs(a.astype(np.complex128) - b.astype(np.complex128))))


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 9, 12, 13, 14, 17, 20, 23])
def test_u2_layer_all_qubits(n, dtype):
    rng = np.random.default_rng(100 + n)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    vec = rand_state(n, n, dtype)
    sv = _sv(n, dtype, vec)
    sv.apply_u2_layer(mats)
    o = _oracle(n, dtype if dtype == np.complex128 else np.complex128, vec)
    for q in range(n):
        o.apply_single(mats[q].reshape(2, 2), q)
    assert _err(sv.get(), o.state) <= TOL[dtype]


@pytest.mark.parametrize("n", [6, 15, 21])
def test_u2_layer_active_subset(n):
    rng = np.random.default_rng(7)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    active = sorted(rng.choice(n, size=max(1, n // 3), replace=False).tolist())
    vec = rand_state(n, 3)
    sv = _sv(n, np.complex64, vec)
    sv.apply_u2_layer(mats, active)
    o = _oracle(n, np.complex128, vec)
    for q in active:
        o.apply_single(mats[q].reshape(2, 2), q)
    assert _err(sv.get(), o.state) <= 1e-5


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("n", [2, 5, 11, 16, 22])
def test_diag_terms_mixed(n, dtype):
    from mettleq_b200 import _native as N
    rng = np.random.default_rng(200 + n)
    terms = []
    for a in range(n - 1):
        terms.append((N.MQ_DIAG_ZZ, a, a + 1, [rng.uniform(0, 2 * math.pi)]))
    for _ in range(n):
        a, b = rng.choice(n, 2, replace=False)
        kind = int(rng.choice([N.MQ_DIAG_CPHASE, N.MQ_DIAG_CRZ, N.MQ_DIAG_ZZ]))
        terms.append((kind, int(a), int(b), [rng.uniform(-math.pi, math.pi)]))
    for q in range(n):
        kind = int(rng.choice([N.MQ_DIAG_RZ, N.MQ_DIAG_PHASE]))
        terms.append((kind, q, -1, [rng.uniform(-math.pi, math.pi)]))
    terms.append((N.MQ_DIAG_CPHASE, 0, n - 1, [math.pi]))  # CZ on the ring wrap
    d0, d1 = np.exp(1j * rng.uniform(0, 6, 2))
    terms.append((N.MQ_DIAG_1Q, n // 2, -1, [d0.real, d0.imag, d1.real, d1.imag]))
    d = np.exp(1j * rng.uniform(0, 6, 4))
    terms.append((N.MQ_DIAG_2Q, 0, n - 1, [x for v in d for x in (v.real, v.imag)]))
    terms.append((N.MQ_DIAG_GLOBAL, -1, -1, [0.37]))
    vec = rand_state(n, 11, dtype)
    sv = _sv(n, dtype, vec)
    sv.apply_diag_terms(terms)
    o = _oracle(n, np.complex128, vec)
    for kind, a, b, p in terms:
        t = p[0]
        if kind == N.MQ_DIAG_ZZ:
            o.apply_zz_phase(t, a, b)
        elif kind == N.MQ_DIAG_CPHASE:
            o.apply_diagonal([1, 1, 1, np.exp(1j * t)], [a, b])
        elif kind == N.MQ_DIAG_CRZ:
            o.apply_diagonal([1, 1, np.exp(-0.5j * t), np.exp(0.5j * t)], [a, b])
        elif kind == N.MQ_DIAG_RZ:
            o.apply_diagonal([np.exp(-0.5j * t), np.exp(0.5j * t)], [a])
        elif kind == N.MQ_DIAG_PHASE:
            o.apply_diagonal([1, np.exp(1j * t)], [a])
        elif kind == N.MQ_DIAG_1Q:
            o.apply_diagonal([p[0] + 1j * p[1], p[2] + 1j * p[3]], [a])
        elif kind == N.MQ_DIAG_2Q:
            o.apply_diagonal([p[2 * i] + 1j * p[2 * i + 1] for i in range(4)], [a, b])
        elif kind == N.MQ_DIAG_GLOBAL:
            o.apply_global_phase(t)
    assert _err(sv.get(), o.state) <= TOL[dtype] * (10 if dtype == np.complex64 else 1)


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("n", [1, 2, 3, 6, 9, 13, 14, 19, 22])
@pytest.mark.parametrize("inverse", [False, True])
def test_qft_full_register(n, dtype, inverse):
    vec = rand_state(n, 31 + n, dtype)
    sv = _sv(n, dtype, vec)
    sv.apply_qft(None, inverse=inverse)
    o = _oracle(n, np.complex128, vec)
    (o.iqft if inverse else o.qft)()
    assert _err(sv.get(), o.state) <= TOL[dtype]


@pytest.mark.parametrize("wires,inverse", [((2, 0), False), ((3, 1, 0), True), ((1, 2, 3, 4), False),
                                           ((5, 9, 0, 7, 2), False), ((4, 5, 6, 7, 8, 9), True)])
def test_qft_wire_subsets(wires, inverse):
    n = 10
    vec = rand_state(n, 5)
    sv = _sv(n, np.complex64, vec)
    sv.apply_qft(wires, inverse=inverse)
    o = _oracle(n, np.complex128, vec)
    (o.iqft if inverse else o.qft)(list(wires))
    assert _err(sv.get(), o.state) <= 1e-5


def test_qft_stage_ranges_compose():
    n = 16
    vec = rand_state(n, 8)
    sv = _sv(n, np.complex64, vec)
    for j0, j1 in ((0, 3), (3, 11), (11, 16)):
        sv.apply_qft_stages(0, n, j0, j1)
    o = _oracle(n, np.complex128, vec)
    o.qft()
    assert _err(sv.get(), o.state) <= 1e-5


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 10, 11, 13, 18, 21])
def test_xor_affine_random_invertible_bit_exact(n, dtype):
    rng = np.random.default_rng(300 + n)
    rows = random_invertible_rows(n, rng)
    c = int(rng.integers(0, 1 << n))
    vec = rand_state(n, 9, dtype)
    sv = _sv(n, dtype, vec)
    sv.apply_xor_affine(rows, c)
    o = _oracle(n, dtype, vec)
    o.apply_affine(rows, c)
    assert np.array_equal(sv.get(), o.state)


@pytest.mark.parametrize("n", [4, 12, 20])
def test_xor_cnot_ladder_and_flips_bit_exact(n):
    ops = [{"name": "CNOT", "wires": [q, q + 1]} for q in range(n - 1)] + [{"name": "X", "wires": [n // 2]},
                                                                          {"name": "SWAP", "wires": [0, n - 1]}]
    rows, c = compose_inverse_affine(ops, n)
    vec = rand_state(n, 4)
    sv = _sv(n, np.complex64, vec)
    sv.apply_xor_affine(rows, c)
    o = _oracle(n, np.complex64, vec)
    o.execute([dict(op, parameters=[]) for op in ops])
    assert np.array_equal(sv.get(), o.state)
    # pure flips (identity rows)
    sv.apply_xor_affine([1 << (n - 1 - k) for k in range(n)], (1 << n) - 1)
    o.apply_affine([1 << (n - 1 - k) for k in range(n)], (1 << n) - 1)
    assert np.array_equal(sv.get(), o.state)


def test_xor_singular_rows_rejected():
    sv = _sv(4, np.complex64)
    with pytest.raises(ValueError):
        sv.apply_xor_affine([0b1000, 0b1000, 0b0010, 0b0001], 0)


@pytest.mark.parametrize("n", [3, 9, 17])
def test_controlled_gates(n):
    from oracle import gate_matrix
    rng = np.random.default_rng(n)
    gates = []
    for _ in range(2 * n):
        k = int(rng.integers(1, 3)) if n >= 3 else 1
        w = rng.choice(n, k + 1, replace=False)
        u = haar_u2(rng)
        gates.append(([int(x) for x in w[:k]], int(w[k]), u))
    gates.append(([0, 1], 2, gate_matrix("X")))
    vec = rand_state(n, 12)
    sv = _sv(n, np.complex64, vec)
    sv.apply_controlled(gates)
    o = _oracle(n, np.complex128, vec)
    for cs, t, u in gates:
        o.apply_multi_controlled_single(u, cs, t)
    assert _err(sv.get(), o.state) <= 1e-5


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("n,wires", [(5, None), (5, [4, 0]), (12, [3, 1]), (12, [11]), (12, []),
                                     (12, list(range(12))[::-1]), (16, [0, 5, 9, 15, 2])])
def test_probabilities_match_oracle_bit_exact(n, wires, dtype):
    vec = rand_state(n, 21, dtype)
    sv = _sv(n, dtype, vec)
    got = sv.probabilities(wires)
    p = osamp.amp2(vec)
    ref = osamp.marginal_probabilities(p, n, wires)
    assert np.array_equal(got, ref)
    o = _oracle(n, np.complex128, vec)
    assert np.max(np.abs(got - o.probabilities(wires))) < 1e-12


@pytest.mark.parametrize("n,wires,shots,seed", [(4, None, 1000, 0), (13, None, 1000, 12345),
                                                (13, [2, 7], 500, 7), (18, None, 257, 2**40 + 3),
                                                (11, list(range(11))[::-1], 300, 9)])
def test_sampling_bit_exact(n, wires, shots, seed):
    vec = rand_state(n, 77, np.complex64)
    sv = _sv(n, np.complex64, vec)
    got = sv.sample_indices(shots, wires, seed=seed, stream_offset=5)
    p = osamp.marginal_probabilities(osamp.amp2(vec), n, wires)
    ref = osamp.sample_indices(p, seed, shots, stream_offset=5)
    assert np.array_equal(got, ref)


def test_sampling_sparse_state_hits_support_only():
    n = 14
    vec = np.zeros(1 << n, dtype=np.complex64)
    vec[[3, 1000, 9999]] = [0.6, 0.0, 0.8]
    sv = _sv(n, np.complex64, vec)
    idx = sv.sample_indices(4000, seed=1)
    assert set(np.unique(idx).tolist()) <= {3, 9999}
    frac = np.mean(idx == 9999)
    assert abs(frac - 0.64) < 0.05


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_expval_pauli_words(dtype):
    n = 9
    vec = rand_state(n, 5, dtype)
    sv = _sv(n, dtype, vec)
    words = [{0: "Z"}, {0: "Z", 1: "Z"}, {3: "X"}, {2: "Y", 5: "Z"}, {1: "X", 4: "Y", 8: "Z"}, {}, {7: "Y"},
             {i: "Z" for i in range(n)}, {0: "X", 8: "X"}]
    got = sv.expval_pauli(words)
    o = _oracle(n, np.complex128, vec)
    ref = np.array([o.pauli_expectation(w) for w in words])
    tol = 1e-6 if dtype == np.complex64 else 1e-12
    assert np.max(np.abs(got - ref)) < tol


def _layer_reference(n, vec, mats, active, terms, rows, c):
    o = _oracle(n, np.complex128, vec)
    if mats is not None:
        for q in (range(n) if active is None else active):
            o.apply_single(mats[q].reshape(2, 2), q)
    oracle_apply_terms(o, terms)
    if rows is not None:
        o.apply_affine(rows, c)
    return o.state


def _ladder(n):
    from mettleq_b200.workloads import cnot_ladder_rows
    return cnot_ladder_rows(n)


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 12, 13, 17, 22])
def test_fused_config_layer(n, dtype):
    """U(2) on every qubit + RZZ chain + CNOT ladder in one apply_layer call
    (diagonal and ladder on the last U(2) sweep) equals the three layers."""
    from mettleq_b200 import fusion as F
    rng = np.random.default_rng(300 + n)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, math.pi))]) for i in range(n - 1)]
    rows, c = _ladder(n)
    vec = rand_state(n, n + 1, dtype)
    sv = _sv(n, dtype, vec)
    s0 = sv.counters()[1]
    sv.apply_layer(mats, None, terms, rows, c)
    sweeps = sv.counters()[1] - s0
    assert _err(sv.get(), _layer_reference(n, vec, mats, None, terms, rows, c)) <= TOL[dtype]
    # as many sweeps as the U(2) layer alone
    s1 = sv.counters()[1]
    sv.apply_u2_layer(mats)
    assert sweeps == sv.counters()[1] - s1


@pytest.mark.parametrize("case", ["far_bond", "random_perm", "high_only", "no_u2", "perm_only", "mixed_terms",
                                  "no_perm", "flip_ladder"])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_fused_layer_variants(case, dtype):
    """Every combination, including the ones that fall back to separate
    diagonal / permutation passes, equals the sequential reference."""
    from mettleq_b200 import fusion as F
    n = 17
    rng = np.random.default_rng(11)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    active = None
    terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, math.pi))]) for i in range(n - 1)]
    rows, c = _ladder(n)
    if case == "far_bond":
        terms = terms + [(F.DIAG_ZZ, 0, n - 1, [0.37])]
    elif case == "random_perm":
        rows = random_invertible_rows(n, rng)
        c = int(rng.integers(0, 1 << n))
    elif case == "high_only":
        active = [0, 1, 2, 5]
    elif case == "no_u2":
        mats = None
    elif case == "perm_only":
        mats, terms = None, []
    elif case == "mixed_terms":
        terms = [(F.DIAG_CPHASE, 3, 4, [0.7]), (F.DIAG_RZ, 16, -1, [1.1]), (F.DIAG_GLOBAL, 0, -1, [0.3]),
                 (F.DIAG_CRZ, 9, 7, [-0.4]), (F.DIAG_PHASE, 0, -1, [2.0])]
    elif case == "no_perm":
        rows = None
    elif case == "flip_ladder":
        c = int(rng.integers(0, 1 << n))
    vec = rand_state(n, 5, dtype)
    sv = _sv(n, dtype, vec)
    sv.apply_layer(mats, active, terms, rows, c)
    assert _err(sv.get(), _layer_reference(n, vec, mats, active, terms, rows, c)) <= TOL[dtype]


def test_fused_layer_rejects_singular_rows_before_any_work():
    n = 6
    vec = rand_state(n, 2)
    sv = _sv(n, np.complex64, vec)
    mats = np.stack([np.eye(2).reshape(4) * 1j for _ in range(n)])
    with pytest.raises(ValueError):
        sv.apply_layer(mats, None, [], [1, 1, 4, 8, 16, 32], 0)
    assert _err(sv.get(), vec) == 0.0


def test_errors_map_to_python_exceptions():
    from mettleq_b200.engine import StateVector
    with pytest.raises(ValueError):
        StateVector(0)
    with pytest.raises(ValueError):
        StateVector(33)
    sv = _sv(3, np.complex64)
    with pytest.raises(ValueError):
        sv.apply_qft([0, 0])
    with pytest.raises(ValueError):
        sv.probabilities([5])
    with pytest.raises(ValueError):
        sv.apply_diag_layer if False else sv.apply_zz_weighted([(0, 0)], [0.1])


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_euler_split_layer_equals_complex_sweeps(dtype, monkeypatch):
    """From 20 qubits a fused layer with a diagonal runs its U(2) gates as real
    RY sweeps between two diagonals (the RZ factors); the result equals the
    complex 2x2 sweeps."""
    from mettleq_b200 import fusion as F
    n = 21
    rng = np.random.default_rng(77)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, math.pi))]) for i in range(n - 1)]
    rows, c = _ladder(n)
    vec = rand_state(n, 4, dtype)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("MQ_EULER", flag)
        sv = _sv(n, dtype, vec)
        sv.apply_layer(mats, None, terms, rows, c)
        sv.apply_u2_layer(mats)
        out[flag] = sv.get()
        sv.close()
    ref = _oracle(n, np.complex128, vec)
    for q in range(n):
        ref.apply_single(mats[q].reshape(2, 2), q)
    oracle_apply_terms(ref, terms)
    ref.apply_affine(rows, c)
    for q in range(n):
        ref.apply_single(mats[q].reshape(2, 2), q)
    for flag in ("1", "0"):
        assert _err(out[flag], ref.state) <= TOL[dtype], flag


@pytest.mark.parametrize("dtype,n", [(d, n) for d in (np.complex64, np.complex128) for n in (4, 9, 12, 13, 17, 21)]
                         + [(np.complex64, 24)])
def test_euler_tangent_rotations(n, dtype, monkeypatch):
    """The Euler split's RY gates in tangent form (one FMA per output
    component, the cos / sin factors multiplied into the low sweep's
    diagonal) equal the oracle's gate-by-gate layer, with the edge angles
    that select each form: identity, X and Z (c or s exactly 0), Hadamard,
    RY(pi/2) (|c| = |s|), and Haar U(2)s on the other qubits."""
    from mettleq_b200 import fusion as F
    monkeypatch.setenv("MQ_EULER_MIN_QUBITS", "1")
    rng = np.random.default_rng(500 + n)
    special = [np.eye(2), np.array([[0, 1], [1, 0]]), np.diag([1, -1]),
               np.array([[1, 1], [1, -1]]) / math.sqrt(2.0),
               np.array([[1, -1], [1, 1]]) / math.sqrt(2.0)]
    mats = np.stack([(special[q].astype(np.complex128) if q < len(special) else haar_u2(rng)).reshape(4)
                     for q in range(n)])
    terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, math.pi))]) for i in range(n - 1)]
    rows, c = _ladder(n)
    vec = rand_state(n, 11 + n, dtype)
    ref = _layer_reference(n, vec, mats, None, terms, rows, c)
    ref = _layer_reference(n, ref, mats[::-1].copy(), None, terms, rows, c)
    for flag in ("1", "0"):
        monkeypatch.setenv("MQ_ROT", flag)
        sv = _sv(n, dtype, vec)
        sv.apply_layer(mats, None, terms, rows, c)
        sv.apply_layer(mats[::-1].copy(), None, terms, rows, c)
        got = sv.get()
        sv.close()
        assert _err(got, ref) <= 2 * TOL[dtype], flag


def test_fused_layer_full_active_list_takes_the_whole_layer_path():
    """The gate-stream fusion passes the list of active qubits even when it
    holds every qubit; such a layer runs exactly as one with no list (the
    Euler split included, from 20 qubits): bit-identical states."""
    from mettleq_b200 import fusion as F
    n = 21
    rng = np.random.default_rng(91)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, math.pi))]) for i in range(n - 1)]
    rows, c = _ladder(n)
    vec = rand_state(n, 5)
    out = []
    for active in (None, list(range(n))):
        sv = _sv(n, np.complex64, vec)
        sv.apply_layer(mats, active, terms, rows, c)
        out.append(sv.get())
        sv.close()
    assert np.array_equal(out[0], out[1])
    assert _err(out[1], _layer_reference(n, vec, mats, None, terms, rows, c)) <= 1e-5


@pytest.mark.gpu
def test_device_shots_agree_with_reference_probabilities():
    """1000 device shots from the reference's own 8-qubit state, against the
    reference's exact probabilities (chi-square, tail pooled): the sampled
    counts agree in distribution, as the reference's MLX stream is not
    reproducible off Apple hardware."""
    import os
    from scipy.stats import chi2
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz"))
    probs = np.asarray(g["probs_0_1_2_3_4_5_6_7"], dtype=np.float64)
    probs /= probs.sum()
    sv = _sv(8, np.complex64, np.asarray(g["layers_uniform"], dtype=np.complex64))
    for seed in (11, 12):
        idx = sv.sample_indices(1000, seed=seed)
        counts = np.bincount(idx, minlength=256).astype(np.float64)
        keep = probs * 1000 >= 5.0
        obs = np.append(counts[keep], counts[~keep].sum())
        exp = np.append(probs[keep] * 1000, probs[~keep].sum() * 1000)
        stat = float(np.sum((obs - exp) ** 2 / exp))
        assert chi2.sf(stat, obs.size - 1) > 1e-3, seed


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("kind", ["XX", "YY"])
@pytest.mark.parametrize("n", [6, 16, 22])
def test_pauli_pair_layer(n, kind, dtype):
    """exp(-i sum_b t_b P_a P_b) (xx_layer / yy_layer, shaders/pauli_pair.py
    :32-64) over a chain and long-range bonds, against the oracle's per-bond
    anti-diagonal passes (sim.py:226-258); also through Device.execute."""
    from mettleq_b200.device import Device
    rng = np.random.default_rng(300 + n)
    bonds = [(i, i + 1) for i in range(n - 1)] + [(0, n - 1), (1, n // 2)]
    thetas = rng.uniform(-math.pi, math.pi, len(bonds))
    vec = rand_state(n, 9, dtype)
    sv = _sv(n, dtype, vec)
    sv.apply_pauli_pair_layer(kind, bonds, thetas)
    o = _oracle(n, np.complex128, vec)
    for (a, b), t in zip(bonds, thetas):
        (o.apply_xx_phase if kind == "XX" else o.apply_yy_phase)(float(t), a, b)
    assert _err(sv.get(), o.state) <= TOL[dtype]
    sv.close()
    ops = [{"name": kind + "PHASE", "wires": [a, b], "parameters": [float(t)]} for (a, b), t in zip(bonds, thetas)]
    dev = Device(n, dtype=np.dtype(dtype).name)
    try:
        dev.sim.set(vec)
        dev.execute(ops)
        assert _err(dev.statevector(), o.state) <= TOL[dtype]
    finally:
        dev.close()
