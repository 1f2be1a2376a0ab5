"""Batched circuits (mq_batch_*): every circuit of a mixed-width batch equals
the oracle run of the same circuit, the captured graph stays valid when the
parameters change, and the plain per-circuit path agrees.

Tolerances: probabilities (float32 outputs of complex64 states) 2e-6
absolute, <Z_0> 1e-5.
"""
import math

import numpy as np
import pytest

from mettleq_b200.batch import hea_batch, hea_mats, hea_ops
from oracle import OracleSim


def oracle_run(params, ladder=True):
    n = params.shape[1]
    o = OracleSim(n, np.complex128)
    o.execute(hea_ops(params, ladder))
    p = np.abs(o.state) ** 2
    z0 = float(np.sum(p[: len(p) // 2]) - np.sum(p[len(p) // 2:]))
    return p, z0


def test_hea_mats_equal_the_gate_products():
    rng = np.random.default_rng(0)
    params = rng.uniform(-math.pi, math.pi, size=(2, 3, 2))
    m = hea_mats(params)
    for d in range(2):
        for q in range(3):
            th, ph = params[d, q]
            ry = np.array([[math.cos(th / 2), -math.sin(th / 2)], [math.sin(th / 2), math.cos(th / 2)]])
            rz = np.diag([np.exp(-0.5j * ph), np.exp(0.5j * ph)])
            assert np.max(np.abs(m[d, q].reshape(2, 2) - rz @ ry)) < 1e-15


def test_hea_batch_shapes_and_ranges():
    ns, ds, ps = hea_batch(64, seed=3)
    assert all(10 <= n <= 24 for n in ns) and all(4 <= d <= 16 for d in ds)
    assert all(p.shape == (d, n, 2) for n, d, p in zip(ns, ds, ps))
    assert all(np.all(np.abs(p) <= math.pi) for p in ps)


@pytest.mark.gpu
@pytest.mark.parametrize("lanes,threads", [(1, 256), (4, 128), (8, 512)])
def test_mixed_batch_matches_oracle(lanes, threads):
    from mettleq_b200.batch import CircuitBatch
    rng = np.random.default_rng(lanes)
    ns = [1, 2, 3, 5, 9, 12, 13, 14, 15, 16, 13, 4, 11, 17, 10, 14]
    ds = [int(x) for x in rng.integers(0, 6, size=len(ns))]
    params = [rng.uniform(-math.pi, math.pi, size=(d, n, 2)) for n, d in zip(ns, ds)]
    b = CircuitBatch(ns, ds, lanes=lanes, small_threads=threads)
    try:
        assert b.n_small == sum(1 for n in ns if n <= 13) and b.n_large == sum(1 for n in ns if n > 13)
        for it in range(2):  # the second run replays the graph with new matrices
            if it:
                params = [rng.uniform(-math.pi, math.pi, size=p.shape) for p in params]
            b.run([hea_mats(p) for p in params])
            z0 = b.z0()
            for c, p in enumerate(params):
                ref_p, ref_z = oracle_run(p)
                got = b.probabilities(c)
                assert np.max(np.abs(got - ref_p)) < 2e-6, (it, c, ns[c])
                assert abs(z0[c] - ref_z) < 1e-5, (it, c, ns[c])
    finally:
        b.close()


@pytest.mark.gpu
def test_batch_without_ladder_and_plain_path_agree():
    from mettleq_b200.batch import CircuitBatch
    from mettleq_b200.device import Device
    rng = np.random.default_rng(9)
    ns = [6, 13, 15, 18]
    ds = [3, 2, 4, 2]
    params = [rng.uniform(-math.pi, math.pi, size=(d, n, 2)) for n, d in zip(ns, ds)]
    ladder = [False, True, False, True]
    b = CircuitBatch(ns, ds, ladder=ladder, lanes=2)
    try:
        b.run([hea_mats(p) for p in params])
        z0 = b.z0()
        for c, p in enumerate(params):
            ref_p, ref_z = oracle_run(p, ladder[c])
            assert np.max(np.abs(b.probabilities(c) - ref_p)) < 2e-6
            assert abs(z0[c] - ref_z) < 1e-5
            dev = Device(ns[c])
            dev.execute(hea_ops(p, ladder[c]))
            plain = dev.sim.probabilities(dtype=np.float32)
            dev.close()
            assert np.max(np.abs(b.probabilities(c) - plain)) < 2e-6
    finally:
        b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("tiles", [(11, 4, 0), (10, 4, 0), (12, 3, 0), (12, 5, 0), (12, 4, 12), (8, 2, 6)])
def test_batch_tile_shapes_match_oracle(tiles):
    """Every tile shape the autotuner may choose gives the oracle's results
    (the large circuits' sweeps re-planned with that shape)."""
    from mettleq_b200.batch import CircuitBatch
    rng = np.random.default_rng(sum(tiles))
    ns = [14, 15, 17, 19, 20, 9]
    ds = [3, 2, 2, 3, 2, 2]
    params = [rng.uniform(-math.pi, math.pi, size=(d, n, 2)) for n, d in zip(ns, ds)]
    b = CircuitBatch(ns, ds, lanes=2, tiles=tiles)
    try:
        b.run([hea_mats(p) for p in params])
        z0 = b.z0()
        for c, p in enumerate(params):
            ref_p, ref_z = oracle_run(p)
            assert np.max(np.abs(b.probabilities(c) - ref_p)) < 2e-6, (tiles, ns[c])
            assert abs(z0[c] - ref_z) < 1e-5
    finally:
        b.close()


@pytest.mark.gpu
def test_autotune_chooses_a_launch_and_tile_shape():
    from mettleq_b200.batch import TILE_CANDIDATES, CircuitBatch, autotune
    ns, ds, ps = hea_batch(24, seed=4)
    b = CircuitBatch(ns, ds)
    packed = b.pack([hea_mats(p) for p in ps])
    b.close()
    choice = autotune(ns, ds, packed, lanes=(2, 4), small_threads=(256,), repeats=1)
    assert choice["lanes"] in (2, 4) and choice["small_threads"] == 256
    assert tuple(choice["tiles"]) in TILE_CANDIDATES
    assert len(choice["tile_times_s"]) == len(TILE_CANDIDATES)
    b2 = CircuitBatch(ns, ds, lanes=choice["lanes"], tiles=choice["tiles"])
    try:
        b2.run(packed=packed)
        z0 = b2.z0()
        for c in (0, len(ns) - 1):
            assert abs(z0[c] - oracle_run(ps[c])[1]) < 1e-5
    finally:
        b2.close()