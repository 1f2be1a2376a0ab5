"""numpy-backed stand-in for the subset of ``mlx.core`` the reference's CPU
statevector path calls.

Test and measurement infrastructure only: ``tests/golden/make_golden.py`` and
``bench.py --impl reference`` put this package on ``sys.path`` so that the
reference's own ``Device(n, execution_device="cpu")`` (device.py:73-431 ->
sim.py per-gate routines) runs unchanged on a host without MLX, to record its
outputs as golden vectors or to time it.  ``metal.is_available``
answers False and ``fast.metal_kernel`` is absent, so the reference never
selects its Metal shaders (execution.py:123-125, 156-183).

Arithmetic is numpy's complex64/float32, not MLX's, so goldens are compared at
the reference's own Metal-vs-MLX parity tolerance (5e-6) or looser.
"""
from __future__ import annotations

import contextlib
import types

import numpy as np

complex64 = np.complex64
float32 = np.float32
float64 = np.float64
int32 = np.int32
uint32 = np.uint32
int64 = np.int64
uint64 = np.uint64
bool_ = np.bool_


class array(np.ndarray):
    """``mx.array`` is both a constructor and a type; an ndarray subclass
    keeps ``isinstance(x, mx.array)`` true for every array this module
    returns."""

    def __new__(cls, data, dtype=None):
        return np.asarray(data, dtype=dtype).view(cls)

    def item(self, *args):  # noqa: D401 - numpy semantics
        return np.ndarray.item(self, *args)


def _wrap(x):
    return np.asarray(x).view(array)


def reshape(a, shape):
    return _wrap(np.reshape(np.asarray(a), tuple(shape) if not isinstance(shape, int) else shape))


def transpose(a, axes=None):
    return _wrap(np.ascontiguousarray(np.transpose(np.asarray(a), axes)))


def matmul(a, b):
    return _wrap(np.matmul(np.asarray(a), np.asarray(b)))


def stack(arrays, axis=0):
    return _wrap(np.stack([np.asarray(x) for x in arrays], axis=axis))


def concatenate(arrays, axis=0):
    return _wrap(np.concatenate([np.asarray(x) for x in arrays], axis=axis))


def zeros(shape, dtype=float32):
    return _wrap(np.zeros(shape, dtype=dtype))


def ones(shape, dtype=float32):
    return _wrap(np.ones(shape, dtype=dtype))


def eye(n, dtype=float32):
    return _wrap(np.eye(n, dtype=dtype))


def take(a, indices, axis=None):
    return _wrap(np.take(np.asarray(a), np.asarray(indices), axis=axis))


def abs(a):  # noqa: A001 - mirrors mlx name
    return _wrap(np.abs(np.asarray(a)))


def sum(a, axis=None):  # noqa: A001
    return _wrap(np.sum(np.asarray(a), axis=axis))


def max(a, axis=None):  # noqa: A001
    return _wrap(np.max(np.asarray(a), axis=axis))


def maximum(a, b):
    return _wrap(np.maximum(np.asarray(a), b))


def log(a):
    return _wrap(np.log(np.asarray(a)))


def cos(a):
    return _wrap(np.cos(np.asarray(a)))


def sin(a):
    return _wrap(np.sin(np.asarray(a)))


def sqrt(a):
    return _wrap(np.sqrt(np.asarray(a)))


def arange(*args, dtype=None):
    return _wrap(np.arange(*args, dtype=dtype))


def conj(a):
    return _wrap(np.conj(np.asarray(a)))


conjugate = conj


def diagonal(a, *args, **kwargs):
    return _wrap(np.diagonal(np.asarray(a), *args, **kwargs))


def eval(*args):  # noqa: A001 - lazy-graph boundary is a no-op here
    return None


class _Device:
    def __init__(self, name):
        self.name = name

    def __repr__(self):
        return f"Device({self.name}, 0)"

    __str__ = __repr__


cpu = _Device("cpu")
gpu = _Device("gpu")
_default = [cpu]


def default_device():
    return _default[0]


def set_default_device(device):
    _default[0] = device


@contextlib.contextmanager
def stream(device):
    yield


metal = types.SimpleNamespace(is_available=lambda: False)
fast = types.SimpleNamespace()  # no metal_kernel attribute: Metal path stays off
fft = types.SimpleNamespace(ifft=lambda a: _wrap(np.fft.ifft(np.asarray(a)).astype(np.complex64)))


def _no_mlx_rng(*args, **kwargs):
    raise RuntimeError("MLX's random stream is not reproducible outside MLX")


random = types.SimpleNamespace(key=_no_mlx_rng, categorical=_no_mlx_rng)
