"""Adjoint-method gradients (differentiation direction).

CPU tests pin the host logic with the oracle: the inverse-ladder rows, the
op-dict form of the ansatz, and the parameter-shift rule against central
finite differences in complex128.  GPU tests check the adjoint gradients
against both (complex128 central differences with h = 1e-4, and the
reference's parameter-shift rule, integrations/qml.py:308-332), and the
torch.autograd binding.

Tolerances: complex128 adjoint vs parameter shift 1e-9, vs central
differences 1e-7 (their own O(h^2) error); complex64 adjoint 5e-5.
"""
import math
from typing import List, Tuple

import numpy as np
import pytest

from mettleq_b200.adjoint import LayeredAnsatz, PauliSum, _ladder_inverse_rows, parameter_shift_grad
from mettleq_b200.workloads import cnot_ladder_rows
from oracle import OracleSim
from tests.helpers import rand_state


def oracle_energy(ansatz, ham, params):
    o = OracleSim(ansatz.n, np.complex128)
    o.execute(ansatz.ops(params))
    return float(sum(c * o.pauli_expectation(w).real for w, c in ham.words()))


def fd_grad(fn, params, h=1e-4):
    p = np.array(params, dtype=np.float64)
    flat = p.reshape(-1)
    g = np.zeros_like(flat)
    for i in range(flat.size):
        old = flat[i]
        flat[i] = old + h
        ep = fn(p)
        flat[i] = old - h
        em = fn(p)
        flat[i] = old
        g[i] = (ep - em) / (2 * h)
    return g.reshape(p.shape)


def test_inverse_ladder_rows_undo_the_ladder():
    n = 7
    vec = rand_state(n, 1, np.complex128)
    o = OracleSim(n, np.complex128)
    o.set_state(vec)
    o.apply_affine(*cnot_ladder_rows(n))
    o.apply_affine(*_ladder_inverse_rows(n))
    assert np.max(np.abs(o.state - vec)) < 1e-15


def test_ansatz_ops_match_layer_matrices():
    A = LayeredAnsatz(4, 2, ("RY", "RZ", "RX"))
    rng = np.random.default_rng(0)
    p = rng.uniform(-math.pi, math.pi, A.shape)
    o1 = OracleSim(4, np.complex128)
    o1.execute(A.ops(p))
    o2 = OracleSim(4, np.complex128)
    for l in range(A.layers):
        mats = A.layer_mats(p[l])
        for q in range(4):
            o2.apply_single(mats[q].reshape(2, 2), q)
        o2.apply_affine(*cnot_ladder_rows(4))
    assert np.max(np.abs(o1.state - o2.state)) < 1e-13


def test_parameter_shift_equals_finite_differences_on_the_oracle():
    A = LayeredAnsatz(4, 2)
    H = PauliSum.ising_chain(4)
    p = np.random.default_rng(3).uniform(-math.pi, math.pi, A.shape)
    f = lambda x: oracle_energy(A, H, x)  # noqa: E731
    assert np.max(np.abs(parameter_shift_grad(f, p) - fd_grad(f, p))) < 1e-7


# ------------------------------------------------------------------ GPU
def _engine(A, H, dtype):
    from mettleq_b200.adjoint import AdjointEngine
    return AdjointEngine(A, H, dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,tol", [("complex128", 1e-9), ("complex64", 5e-5)])
@pytest.mark.parametrize("n,layers,rots", [(3, 2, ("RY", "RZ")), (6, 3, ("RY", "RZ")), (9, 2, ("RX", "RY", "RZ")),
                                           (13, 2, ("RY", "RZ")), (16, 1, ("RZ", "RY"))])
def test_adjoint_matches_parameter_shift(n, layers, rots, dtype, tol):
    A = LayeredAnsatz(n, layers, rots)
    H = PauliSum.ising_chain(n)
    p = np.random.default_rng(n).uniform(-math.pi, math.pi, A.shape)
    eng = _engine(A, H, dtype)
    try:
        e, g = eng.energy_and_grad(p)
        e_ref = oracle_energy(A, H, p)
        assert abs(e - e_ref) < tol
        # parameter shift on the oracle for a subset of parameters (all when small)
        f = lambda x: oracle_energy(A, H, x)  # noqa: E731
        flat_idx = np.arange(p.size) if p.size <= 40 else np.random.default_rng(1).choice(p.size, 24, replace=False)
        for i in flat_idx:
            pp = p.copy().reshape(-1)
            pp[i] += math.pi / 2
            ep = f(pp.reshape(A.shape))
            pp[i] -= math.pi
            em = f(pp.reshape(A.shape))
            assert abs(g.reshape(-1)[i] - 0.5 * (ep - em)) < tol, i
    finally:
        eng.close()


@pytest.mark.gpu
def test_adjoint_complex128_matches_central_differences():
    A = LayeredAnsatz(6, 3)
    H = PauliSum.ising_chain(6)
    p = np.random.default_rng(5).uniform(-math.pi, math.pi, A.shape)
    eng = _engine(A, H, "complex128")
    try:
        _, g = eng.energy_and_grad(p)
    finally:
        eng.close()
    fd = fd_grad(lambda x: oracle_energy(A, H, x), p, h=1e-4)
    assert np.max(np.abs(g - fd)) < 1e-7


@pytest.mark.gpu
def test_adjoint_restores_the_initial_state():
    """The backward run un-applies the whole circuit: psi returns to |0>."""
    A = LayeredAnsatz(11, 3)
    H = PauliSum.ising_chain(11)
    p = np.random.default_rng(2).uniform(-math.pi, math.pi, A.shape)
    eng = _engine(A, H, "complex128")
    try:
        eng.energy_and_grad(p)
        psi = eng.psi.get()
    finally:
        eng.close()
    ref = np.zeros(1 << 11, dtype=np.complex128)
    ref[0] = 1.0
    assert np.max(np.abs(psi - ref)) < 1e-12


@pytest.mark.gpu
def test_torch_autograd_binding():
    import torch
    from mettleq_b200.adjoint import AdjointEnergy
    A = LayeredAnsatz(8, 2)
    H = PauliSum.ising_chain(8)
    p0 = np.random.default_rng(4).uniform(-math.pi, math.pi, A.shape)
    eng = _engine(A, H, "complex128")
    try:
        x = torch.tensor(p0, dtype=torch.float64, requires_grad=True)
        e = AdjointEnergy.apply(x, eng)
        # an unrelated forward in between: backward recomputes its own state
        AdjointEnergy.apply(torch.zeros_like(x), eng)
        (2.0 * e).backward()
        _, g = eng.energy_and_grad(p0)
    finally:
        eng.close()
    assert abs(float(e) - oracle_energy(A, H, p0)) < 1e-10
    assert np.max(np.abs(x.grad.numpy() - 2.0 * g)) < 1e-12


@pytest.mark.gpu
def test_pauli_sum_energy_and_lambda():
    """lam = H psi and E = <psi|H|psi> for Z words and X terms."""
    from mettleq_b200.adjoint import AdjointEngine
    n = 12
    H = PauliSum(n, [((0, 1), 0.7), ((3,), -0.2), ((2, 5, 11), 1.3)], np.linspace(-0.5, 0.5, n))
    A = LayeredAnsatz(n, 1)
    eng = AdjointEngine(A, H, dtype="complex128")
    try:
        vec = rand_state(n, 9, np.complex128)
        eng.psi.set(vec)
        e = eng._pauli_sum()
        lam = eng.lam.get()
    finally:
        eng.close()
    o = OracleSim(n, np.complex128)
    o.set_state(vec)
    ref_e = sum(c * o.pauli_expectation(w).real for w, c in H.words())
    # H psi by dense Pauli application on the oracle
    out = np.zeros_like(vec)
    for w, c in H.words():
        o2 = OracleSim(n, np.complex128)
        o2.set_state(vec)
        for q, p in w.items():
            o2.apply_single(np.array([[0, 1], [1, 0]]) if p == "X" else np.diag([1, -1]), q)
        out += c * o2.state
    assert abs(e - ref_e) < 1e-12
    assert np.max(np.abs(lam - out)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2])
def test_pauli_sum_window_tables_and_wide_words(seed):
    """lam = H psi for random Z words of every width (one to all qubits), a
    constant word and a chain: the words within 8 index bits go through the
    window tables, the wider ones one by one."""
    from mettleq_b200.adjoint import AdjointEngine
    n = 16
    rng = np.random.default_rng(seed)
    words = [((i, i + 1), float(rng.uniform(-1, 1))) for i in range(n - 1)]
    for k in (1, 2, 3, 5, 9, 16):
        for _ in range(3):
            words.append((tuple(sorted(int(q) for q in rng.choice(n, k, replace=False))), float(rng.uniform(-1, 1))))
    words.append(((), 0.25))
    H = PauliSum(n, words, None)
    eng = AdjointEngine(LayeredAnsatz(n, 1), H, dtype="complex128")
    try:
        vec = rand_state(n, seed, np.complex128)
        eng.psi.set(vec)
        e = eng._pauli_sum()
        lam = eng.lam.get()
    finally:
        eng.close()
    idx = np.arange(1 << n)
    d = np.zeros(1 << n)
    for w, c in words:
        z = 0
        for q in w:
            z |= 1 << (n - 1 - q)
        par = np.array([bin(int(x)).count("1") & 1 for x in (idx & z)])
        d += c * (1 - 2 * par)
    assert np.max(np.abs(lam - d * vec)) < 1e-12
    assert abs(e - float(np.real(np.vdot(vec, d * vec)))) < 1e-12


@pytest.mark.gpu
def test_host_and_device_gradient_readback_agree(monkeypatch):
    """mq_adjoint_layer (host gradients, one wait per layer) and
    mq_adjoint_layer_async (device gradients, one read at the end) give the
    same bits."""
    from mettleq_b200.adjoint import AdjointEngine
    A = LayeredAnsatz(14, 3, ("RX", "RY", "RZ"))
    H = PauliSum.ising_chain(14, 0.8, -0.3)
    p = np.random.default_rng(8).uniform(-math.pi, math.pi, A.shape)
    eng = AdjointEngine(A, H, dtype="complex64")
    try:
        _, g_dev = eng.energy_and_grad(p)
        monkeypatch.setattr(eng, "_grad_buffer", lambda count: None)
        _, g_host = eng.energy_and_grad(p)
    finally:
        eng.close()
    assert np.array_equal(g_dev, g_host)


def _gf2_map(n: int, m: int, rng, mixing: bool) -> Tuple[List[int], int]:
    """Rows (qubit k = row k, as mq_apply_xor_affine) and flip of a random
    invertible map out[x] = in[A x ^ c].  Column operations on the identity:
    with ``mixing`` False, A maps the low tile [0, m) onto itself and keeps
    e_0; with ``mixing`` True a high column is added into a low one."""
    cols = [1 << j for j in range(n)]
    for _ in range(6 * n):
        j = int(rng.integers(1, n))
        i = int(rng.integers(0, n))
        if i == j or (j < m and i >= m):
            continue
        cols[j] ^= cols[i]
    if mixing:
        cols[int(rng.integers(1, m))] ^= cols[int(rng.integers(m, n))]
    rows = [sum(((cols[j] >> (n - 1 - k)) & 1) << j for j in range(n)) for k in range(n)]
    return rows, int(rng.integers(0, 1 << n))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["complex64", "complex128"])
@pytest.mark.parametrize("kind", ["low", "mixing", "map_only"])
def test_adjoint_layer_with_map_equals_separate_pass(dtype, kind):
    """mq_adjoint_layer_xor_async gives the bits of mq_apply_xor_affine on
    both states followed by mq_adjoint_layer_async.  That holds for maps that
    the layer's first sweep gathers on load (they keep its low tile [0, 10)
    and bit 0), for maps that mix that tile with high bits (a separate pass
    runs), and for a map with no layer (n_q = 0)."""
    import ctypes as C
    import torch
    from mettleq_b200 import _native as N
    from mettleq_b200.engine import StateVector
    n = 16
    rng = np.random.default_rng({"low": 1, "mixing": 2, "map_only": 3}[kind])
    rows, c = _gf2_map(n, 10, rng, kind == "mixing")
    rows_a = np.ascontiguousarray(np.asarray(rows, dtype=np.uint64))
    n_q = 0 if kind == "map_only" else n
    qubits = np.arange(n, dtype=np.int32)
    mats = np.empty((n, 2, 2), dtype=np.complex128)
    for q in range(n):
        z = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        mats[q] = np.linalg.qr(z)[0]
    m = np.ascontiguousarray(mats).view(np.float64)
    p0, l0 = rand_state(n, 11, np.dtype(dtype)), rand_state(n, 12, np.dtype(dtype))
    lib = N.lib()
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    states = []
    for _ in range(2):
        psi = StateVector(n, dtype=dtype)
        states.append((psi, StateVector(n, dtype=dtype, stream=psi.stream)))  # one stream per pair
    grads = [torch.zeros(3 * n, dtype=torch.float64, device="cuda") for _ in range(2)]
    try:
        for psi, lam in states:
            psi.set(p0)
            lam.set(l0)
        (psi, lam), g = states[0], grads[0]
        N.check(lib.mq_adjoint_layer_xor_async(psi.handle, lam.handle, ptr(rows_a), c, n_q, ptr(qubits), ptr(m),
                                               C.c_void_p(g.data_ptr())))
        (psi2, lam2), g2 = states[1], grads[1]
        psi2.apply_xor_affine(rows, c)
        lam2.apply_xor_affine(rows, c)
        if n_q:
            N.check(lib.mq_adjoint_layer_async(psi2.handle, lam2.handle, n_q, ptr(qubits), ptr(m),
                                               C.c_void_p(g2.data_ptr())))
        out = []
        for (p, l_), gg in zip(states, grads):
            p.synchronize()
            l_.synchronize()
            out.append((p.get(), l_.get(), gg.cpu().numpy()))
    finally:
        for p, l_ in states:
            l_.close()
            p.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    if kind != "map_only":
        assert np.any(out[0][2] != 0)
    # the map itself against the oracle
    o = OracleSim(n, np.complex128)
    o.set_state(p0.astype(np.complex128))
    o.apply_affine(rows, c)
    if kind == "map_only":
        tol = 1e-6 if dtype == "complex64" else 1e-15
        assert np.max(np.abs(out[0][0] - o.state)) < tol
