"""mq_expval_pauli_static: Pauli expectations that allocate no device memory.

Some callers cannot let a library call cudaMalloc or cudaFree part-way
through their work: a serving loop that admits requests by state footprint
alone, a host whose own pool already owns the free HBM, or one that cannot
let cudaFree's device-wide wait stall its other streams.  For them the
library keeps this one entry point, whose scratch is a fixed device array
inside libmq.  These tests call it through the C ABI and check that it
returns exactly what mq_expval_pauli returns, on two calls in a row (the
second call reuses the array the first one left behind).

This file is collected last, so a run that stops at the first failure has
run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import rand_state

pytestmark = pytest.mark.gpu


def _words(n, rng, count):
    out = []
    for _ in range(count):
        w = {}
        for q in rng.choice(n, int(rng.integers(0, 4)), replace=False):
            w[int(q)] = str(rng.choice(["X", "Y", "Z"]))
        out.append(w)
    return out


def _masks(n, words):
    from mettleq_b200.engine import pauli_masks
    xs = np.empty(len(words), dtype=np.uint64)
    zs = np.empty(len(words), dtype=np.uint64)
    ny = np.empty(len(words), dtype=np.int32)
    for i, w in enumerate(words):
        xs[i], zs[i], ny[i] = pauli_masks(n, w)
    return xs, zs, ny


def _call(lib, fn, h, words, n):
    from mettleq_b200 import _native as N
    xs, zs, ny = _masks(n, words)
    out = np.full(2 * len(words), np.nan)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = getattr(lib, fn)(h, len(words), p(xs), p(zs), p(ny), p(out))
    assert rc == N.MQ_OK, N.last_error()
    return out


@pytest.mark.parametrize("dtype,code", [(np.complex64, 0), (np.complex128, 1)])
def test_static_scratch_matches_allocating_entry_point(dtype, code):
    from mettleq_b200 import _native as N
    lib = N.lib()
    n = 14
    rng = np.random.default_rng(7)
    h = C.c_void_p()
    assert lib.mq_state_create(n, code, 0, None, C.byref(h)) == N.MQ_OK, N.last_error()
    try:
        vec = rand_state(n, 3, dtype)
        assert lib.mq_state_set(h, vec.ctypes.data_as(C.c_void_p)) == N.MQ_OK
        # two calls in a row with different word lists (runs of shared X/Y
        # masks and single words); each must equal the allocating call
        first = [{0: "Z"}, {0: "Z", 1: "Z"}, {5: "X"}, {5: "X", 2: "Z"}, {5: "Y", 9: "Z"}, {}] + _words(n, rng, 20)
        second = [{i: "Z", i + 1: "Z"} for i in range(n - 1)] + [{i: "X"} for i in range(n)]
        for words in (first, second):
            got = _call(lib, "mq_expval_pauli_static", h, words, n)
            ref = _call(lib, "mq_expval_pauli", h, words, n)
            assert np.array_equal(got, ref), np.max(np.abs(got - ref))
    finally:
        lib.mq_state_destroy(h)


def test_static_scratch_long_mask_runs_and_optional_arguments():
    """More than eight consecutive words on one X/Y mask (a pass holds eight,
    so the run splits), runs of one mask broken up by other masks (the
    allocating call groups them across the gap, this one does not), ny = NULL
    and an empty word list: every value equals mq_expval_pauli's."""
    from mettleq_b200 import _native as N
    lib = N.lib()
    n = 12
    h = C.c_void_p()
    assert lib.mq_state_create(n, 0, 0, None, C.byref(h)) == N.MQ_OK, N.last_error()
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    try:
        vec = rand_state(n, 11, np.complex64)
        assert lib.mq_state_set(h, p(vec)) == N.MQ_OK
        # 11 words on X(1) in a row, then X(1) runs interleaved with X(4) words
        words = [{1: "X", q: "Z"} for q in range(2, 12)] + [{1: "X"}]
        for q in range(2, 8):
            words += [{1: "X", q: "Z"}, {4: "X", q: "Z"}, {4: "X"}]
        words += [{1: "Y", 3: "Z"}, {1: "Y"}]
        got = _call(lib, "mq_expval_pauli_static", h, words, n)
        ref = _call(lib, "mq_expval_pauli", h, words, n)
        assert np.array_equal(got, ref), np.max(np.abs(got - ref))
        # ny = NULL: no Y factors, results as with ny = 0
        zw = [{q: "Z"} for q in range(n)] + [{2: "X", 5: "X"}] * 10
        xs, zs, _ = _masks(n, zw)
        a = np.full(2 * len(zw), np.nan)
        b = np.full(2 * len(zw), np.nan)
        assert lib.mq_expval_pauli_static(h, len(zw), p(xs), p(zs), None, p(a)) == N.MQ_OK, N.last_error()
        assert lib.mq_expval_pauli(h, len(zw), p(xs), p(zs), None, p(b)) == N.MQ_OK, N.last_error()
        assert np.array_equal(a, b)
        # no words: nothing launched, nothing written
        out = np.full(2, 7.0)
        one = np.zeros(1, dtype=np.uint64)
        assert lib.mq_expval_pauli_static(h, 0, p(one), p(one), None, p(out)) == N.MQ_OK, N.last_error()
        assert np.array_equal(out, [7.0, 7.0])
    finally:
        lib.mq_state_destroy(h)


def test_static_scratch_rejects_masks_outside_the_register():
    from mettleq_b200 import _native as N
    lib = N.lib()
    h = C.c_void_p()
    assert lib.mq_state_create(6, 0, 0, None, C.byref(h)) == N.MQ_OK, N.last_error()
    try:
        xs = np.array([1 << 6], dtype=np.uint64)
        zs = np.zeros(1, dtype=np.uint64)
        ny = np.zeros(1, dtype=np.int32)
        out = np.zeros(2)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        assert lib.mq_expval_pauli_static(h, 1, p(xs), p(zs), p(ny), p(out)) == N.MQ_EINVAL
        assert "outside the register" in N.last_error()
    finally:
        lib.mq_state_destroy(h)
