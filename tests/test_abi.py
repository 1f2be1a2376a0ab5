"""The C-ABI library: it loads and exports every symbol include/mq.h declares
(CPU only: no compute calls), and the host-side argument checks that run
before any device work."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    with open(os.path.join(ROOT, "include", "mq.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mq_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    from mettleq_b200 import build as B
    B.build()
    from mettleq_b200 import _native as N
    lib = N.lib()
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(N.SIGNATURES), "ctypes signatures and header disagree"


def test_library_reports_version_and_errors_without_device():
    from mettleq_b200 import _native as N
    assert N.lib().mq_version() == 1
    n = N.device_count()
    assert n >= 0
    if n == 0:
        import ctypes as C
        h = C.c_void_p()
        rc = N.lib().mq_state_create(4, 0, 0, None, C.byref(h))
        assert rc == N.MQ_EDEVICE
        assert "device" in N.last_error().lower()


def test_footprint_and_argument_validation():
    from mettleq_b200 import _native as N
    assert N.footprint(30, N.MQ_C64, True) == 2 * (1 << 30) * 8
    assert N.footprint(10, N.MQ_C128, False) == (1 << 10) * 16
    with pytest.raises(ValueError):
        N.footprint(0)
    with pytest.raises(ValueError):
        N.footprint(33)
    with pytest.raises(ValueError):
        N.footprint(10, dtype=7)


def test_preflight_refuses_before_allocation():
    from mettleq_b200.execution import require_statevector_preflight, statevector_preflight
    from mettleq_b200._native import StatevectorMemoryError
    mem = {"free": 10 * 2 ** 30, "total": 16 * 2 ** 30}
    assert statevector_preflight(28, memory=mem)["allowed"]
    with pytest.raises(StatevectorMemoryError) as ei:
        require_statevector_preflight(31, memory=mem)
    assert ei.value.report["failure_reasons"]
    r = statevector_preflight(31, memory=mem, allow_unsafe=True)
    assert r["allowed"] and r["decision"] == "allowed_with_unsafe_override"
    assert not statevector_preflight(33, memory=mem, allow_unsafe=True)["allowed"]


def test_preflight_env_override(monkeypatch):
    from mettleq_b200.execution import statevector_preflight
    mem = {"free": 2 ** 30, "total": 2 ** 30}
    monkeypatch.setenv("METTLEQ_ALLOW_UNSAFE_STATEVECTOR", "1")
    assert statevector_preflight(30, memory=mem)["allowed"]
    monkeypatch.setenv("METTLEQ_ALLOW_UNSAFE_STATEVECTOR", "maybe")
    with pytest.raises(ValueError):
        statevector_preflight(30, memory=mem)
