"""ctypes binding of libmq.so (the C ABI declared in include/mq.h).

The shared library is built in-tree by ``mettleq_b200.build``.  There is no
CPU fallback: if the library cannot be loaded, every engine entry point
raises.  Status codes map to the reference's exception types
(execution.py:33-38 StatevectorMemoryError, ValueError for bad arguments,
RuntimeError for device failures).
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libmq.so")

MQ_OK, MQ_EINVAL, MQ_ENOMEM, MQ_EDEVICE, MQ_ETIMEOUT, MQ_EUNSUPPORTED = range(6)
MQ_C64, MQ_C128 = 0, 1
(MQ_DIAG_ZZ, MQ_DIAG_CPHASE, MQ_DIAG_RZ, MQ_DIAG_PHASE, MQ_DIAG_CRZ,
 MQ_DIAG_GLOBAL, MQ_DIAG_1Q, MQ_DIAG_2Q) = range(8)

# Every exported symbol of include/mq.h with its ctypes signature.
_P = C.c_void_p
_I = C.c_int
_U64 = C.c_uint64
_I64 = C.c_int64
SIGNATURES = {
    "mq_last_error": (C.c_char_p, []),
    "mq_version": (_I, []),
    "mq_device_count": (_I, [C.POINTER(_I)]),
    "mq_state_footprint": (_I, [_I, _I, _I, C.POINTER(_U64)]),
    "mq_state_create": (_I, [_I, _I, _I, _P, C.POINTER(_P)]),
    "mq_state_destroy": (_I, [_P]),
    "mq_state_info": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    "mq_state_set_stream": (_I, [_P, _P]),
    "mq_state_stream": (_I, [_P, C.POINTER(_P)]),
    "mq_state_set_sm_limit": (_I, [_P, _I]),
    "mq_state_reset": (_I, [_P]),
    "mq_state_set": (_I, [_P, _P]),
    "mq_state_get": (_I, [_P, _P]),
    "mq_state_copy": (_I, [_P, _P]),
    "mq_state_device_ptr": (_I, [_P, C.POINTER(_P)]),
    "mq_sync": (_I, [_P]),
    "mq_state_counters": (_I, [_P, C.POINTER(_U64), C.POINTER(_U64)]),
    "mq_apply_u2_layer": (_I, [_P, _P, _P]),
    "mq_apply_u2_uniform": (_I, [_P, _P]),
    "mq_apply_controlled_u2": (_I, [_P, _I, _P, _P, _P, _P]),
    "mq_apply_diag_terms": (_I, [_P, _I, _P, _P, _P]),
    "mq_apply_diag_layer": (_I, [_P, _I, _I, _P, _P]),
    "mq_apply_qft": (_I, [_P, _P, _I, _I]),
    "mq_apply_qft_stages": (_I, [_P, _I, _I, _I, _I, _I]),
    "mq_apply_xor_affine": (_I, [_P, _P, _U64]),
    "mq_apply_layer": (_I, [_P, _P, _P, _I, _P, _P, _P, _P, _U64]),
    "mq_probabilities": (_I, [_P, _P, _I, _I, _P]),
    "mq_probabilities_device": (_I, [_P, _I, _P]),
    "mq_sample": (_I, [_P, _P, _I, _U64, _U64, _I64, _P]),
    "mq_expval_pauli": (_I, [_P, _I, _P, _P, _P, _P]),
    "mq_expval_pauli_static": (_I, [_P, _I, _P, _P, _P, _P]),
    "mq_batch_create": (_I, [_I, _P, _I, _P, _P, _P, _I, _I, C.POINTER(_P)]),
    "mq_batch_info": (_I, [_P, C.POINTER(_U64), C.POINTER(_U64), C.POINTER(_I), C.POINTER(_I)]),
    "mq_batch_run": (_I, [_P, _P, _P, _P]),
    "mq_batch_set_tiles": (_I, [_P, _I, _I, _I]),
    "mq_batch_sync": (_I, [_P]),
    "mq_batch_destroy": (_I, [_P]),
    "mq_apply_pauli_sum": (_I, [_P, _P, _I, _P, _P, _P, _P]),
    "mq_adjoint_layer": (_I, [_P, _P, _I, _P, _P, _P]),
    "mq_adjoint_layer_async": (_I, [_P, _P, _I, _P, _P, _P]),
    "mq_adjoint_layer_xor_async": (_I, [_P, _P, _P, _U64, _I, _P, _P, _P]),
}


class StatevectorMemoryError(MemoryError):
    """Raised before allocation when the device cannot hold the state
    (mirrors execution.py:33-38)."""

    def __init__(self, message: str, report: Optional[dict] = None):
        super().__init__(message)
        self.report = report or {}


class DeviceTimeoutError(RuntimeError):
    """A bounded device wait gave up (MQ_ETIMEOUT)."""


_lib = None
_lock = threading.Lock()


def lib():
    """Load libmq.so once; raise loudly if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libmq.so not found at {LIB_PATH}; build it with `python -m mettleq_b200.build` "
                "(the engine has no CPU fallback)")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().mq_last_error()
    return msg.decode(errors="replace") if msg else ""


def check(rc: int, what: str = "") -> None:
    if rc == MQ_OK:
        return
    msg = last_error() or what
    if rc == MQ_EINVAL:
        raise ValueError(msg)
    if rc == MQ_ENOMEM:
        raise StatevectorMemoryError(msg)
    if rc == MQ_ETIMEOUT:
        raise DeviceTimeoutError(msg)
    if rc == MQ_EUNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)


def device_count() -> int:
    out = C.c_int(0)
    check(lib().mq_device_count(C.byref(out)))
    return int(out.value)


def footprint(n: int, dtype: int = MQ_C64, double_buffered: bool = True) -> int:
    out = C.c_uint64(0)
    check(lib().mq_state_footprint(int(n), int(dtype), 1 if double_buffered else 0, C.byref(out)))
    return int(out.value)
