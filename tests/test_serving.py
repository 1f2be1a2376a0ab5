"""Serving with continuous batching: admission under the memory budget,
every result the same alone and in the mix (states bit-identical, identical
counts under the same seed), and equal to the oracle."""
import math

import numpy as np
import pytest

from mettleq_b200.serving import Request, RequestLayer, haar_u2_batch, poisson_requests


def test_poisson_stream_shape():
    reqs = poisson_requests(300, rate=200.0, seed=4, depth_range=(1, 2))
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert 0.8 < len(reqs) / arr[-1] / 200.0 < 1.25
    ns = np.array([r.n for r in reqs])
    assert ns.min() >= 12 and ns.max() <= 30
    # log-uniform: about as many requests in [12, 19) as in [19, 30]
    assert 0.6 < np.sum(ns < 19) / np.sum(ns >= 19) < 1.7
    assert all(r.footprint == 2 * (1 << r.n) * 8 for r in reqs)


def test_haar_batch_is_unitary():
    u = haar_u2_batch(np.random.default_rng(0), 64).reshape(64, 2, 2)
    eye = np.einsum("kab,kcb->kac", u, u.conj())
    assert np.max(np.abs(eye - np.eye(2))) < 1e-12


def _small_requests(count, seed):
    rng = np.random.default_rng(seed)
    from mettleq_b200.serving import random_layer
    reqs = []
    for i in range(count):
        n = int(rng.integers(6, 15))
        layers = [random_layer(n, rng, p_qft=0.3, p_xor=0.3) for _ in range(int(rng.integers(2, 7)))]
        reqs.append(Request(i, 0.0005 * i, n, layers, shots=500, seed=1000 + i))
    return reqs


def _oracle_state(r):
    from mettleq_b200.workloads import cnot_ladder_rows
    from oracle import OracleSim
    o = OracleSim(r.n, np.complex128)
    for L in r.layers:
        for q in range(r.n):
            o.apply_single(L.mats[q].reshape(2, 2), q)
        for i, t in enumerate(L.thetas):
            o.apply_zz_phase(float(t) / 2.0, i, i + 1)
        o.apply_affine(*cnot_ladder_rows(r.n))
        if L.qft:
            o.qft(list(range(r.n)))
        if L.xor is not None:
            o.apply_affine(*L.xor)
    return o.state


@pytest.mark.gpu
def test_each_result_is_the_same_alone_and_in_the_mix():
    from mettleq_b200.serving import Server
    mix = _small_requests(14, seed=1)
    srv = Server(max_active=8, layers_per_round=2, keep_states=True)
    try:
        stats = srv.serve(mix, realtime=False)
        assert stats["requests"] == 14 and srv.peak_active > 1
        for r in mix:
            alone = _small_requests(14, seed=1)[r.rid]
            srv.serve([alone], realtime=False)
            assert np.array_equal(alone.state, r.state), r.rid
            assert np.array_equal(alone.samples, r.samples), r.rid
            assert np.max(np.abs(r.state - _oracle_state(r))) < 1e-5
    finally:
        srv.close()


def _mixed_with_large(seed):
    """Ten small requests (6-14 qubits) and three large ones (22-24 qubits,
    QFT and GF(2) layers likely) in one stream."""
    from mettleq_b200.serving import random_layer
    rng = np.random.default_rng(seed)
    reqs = _small_requests(10, seed)
    for j, n in enumerate((22, 23, 24)):
        layers = [random_layer(n, rng, p_qft=0.5, p_xor=0.5) for _ in range(3)]
        reqs.append(Request(10 + j, 0.0002 * j, n, layers, shots=1000, seed=77 + j))
    return reqs


@pytest.mark.gpu
def test_large_requests_are_the_same_alone_and_in_the_mix():
    """The branches the 30-qubit serving numbers depend on: large requests
    (work above ``small_work``) run with an SM limit, at most ``max_large``
    of them at once, and get their layers in chunks over several rounds.
    Each result is bit-identical to the same request served alone; the
    22-qubit one (and every small one) is within 1e-5 of the oracle."""
    from mettleq_b200.serving import Server
    mix = _mixed_with_large(5)
    kw = dict(max_active=16, layers_per_round=1, keep_states=True, small_work=1 << 20, max_large=2,
              sm_reserve=20)
    srv = Server(**kw)
    try:
        stats = srv.serve(mix, realtime=False)
        assert stats["requests"] == len(mix)
        assert srv.peak_large == 2            # the cap engaged: three large requests, two at a time
        assert srv.partial_issues > 0         # large requests were issued in chunks
        assert srv.peak_active > 2
        for r in mix:
            alone = _mixed_with_large(5)[r.rid]
            srv.serve([alone], realtime=False)
            assert np.array_equal(alone.state, r.state), r.rid
            assert np.array_equal(alone.samples, r.samples), r.rid
            if r.n <= 22:
                assert np.max(np.abs(r.state - _oracle_state(r))) < 1e-5, r.rid
    finally:
        srv.close()


@pytest.mark.gpu
def test_one_server_over_a_device_list():
    """The multi-device Server with one device: every request is admitted on
    it and each result equals the single-device Server's."""
    from mettleq_b200.serving import Server
    a = _small_requests(8, seed=7)
    b = _small_requests(8, seed=7)
    s1 = Server(max_active=8, keep_states=True)
    s2 = Server(max_active=8, keep_states=True, devices=[0])
    try:
        s1.serve(a, realtime=False)
        s2.serve(b, realtime=False)
        assert s2.served_on == {0: 8}
        for x, y in zip(a, b):
            assert np.array_equal(x.state, y.state) and np.array_equal(x.samples, y.samples)
    finally:
        s1.close()
        s2.close()


@pytest.mark.gpu
def test_admission_stays_within_the_budget():
    from mettleq_b200.serving import Server
    reqs = _small_requests(20, seed=2)
    budget = 3 * 2 * (1 << 14) * 8  # three of the largest requests at a time
    srv = Server(budget_bytes=budget, max_active=16)
    try:
        stats = srv.serve(reqs, realtime=False)
    finally:
        srv.close()
    assert stats["requests"] == 20
    assert 0 < srv.peak_used <= budget
    assert all(r.finished >= r.admitted >= 0 for r in reqs)


@pytest.mark.gpu
def test_oversized_request_is_refused():
    from mettleq_b200.serving import Server
    r = _small_requests(1, seed=3)[0]
    srv = Server(budget_bytes=r.footprint - 1)
    with pytest.raises(MemoryError):
        srv.serve([r], realtime=False)
    srv.close()
