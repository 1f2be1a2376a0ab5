"""Gate-stream fusion (host logic) checked on the CPU.

The fused layers are interpreted with the oracle's per-gate routines and
compared with the oracle running the original gate stream, in complex128.
Also pins the fused layer shapes the reference's launch-count tests assert
(src/tests/mlxQMetalKernelsTest.py:153-192, 502-552).
"""
import math

import numpy as np
import pytest

from mettleq_b200 import fusion as F
from mettleq_b200 import workloads as W
from oracle import OracleSim, compose_inverse_affine
from tests.helpers import oracle_apply_terms, rand_state


def interpret(layers, n, vec):
    o = OracleSim(n, np.complex128)
    o.set_state(vec)
    for L in layers:
        name = L["name"]
        if name == "_U2LISTLAYER":
            for q in L["active"]:
                o.apply_single(L["mats"][q].reshape(2, 2), q)
        elif name == "_DIAG":
            oracle_apply_terms(o, L["terms"])
        elif name == "_LAYER":
            if L["mats"] is not None:
                for q in L["active"]:
                    o.apply_single(L["mats"][q].reshape(2, 2), q)
            oracle_apply_terms(o, L["terms"])
            if L["rows"] is not None:
                o.apply_affine(L["rows"], L["c"])
        elif name == "_XORLAYER":
            o.apply_affine(L["rows"], L["c"])
        elif name == "_QFTSTAGES":
            wires = list(range(L["q0"], L["q0"] + L["k"]))
            h = np.array([[1, 1], [1, -1]]) / math.sqrt(2)
            js = range(L["j_begin"], L["j_end"])
            if not L["inverse"]:
                for j in js:
                    o.apply_single(h, wires[j])
                    o._phase_ladder(wires, j, 1.0)
            else:
                for j in reversed(js):
                    o._phase_ladder(wires, j, -1.0)
                    o.apply_single(h, wires[j])
        elif name == "_CULIST":
            for cs, t, u in L["gates"]:
                o.apply_multi_controlled_single(u, cs, t)
        elif name == "_PAIRLAYER":
            for (a, b), t in zip(L["bonds"], L["thetas"]):
                (o.apply_xx_phase if L["kind"] == "XX" else o.apply_yy_phase)(t, a, b)
        else:
            raise AssertionError(name)
    return o.state


def test_pair_terms_fuse_into_one_layer_per_family_run():
    """Runs of XXPHASE (YYPHASE) terms, even on overlapping bonds, become one
    _PAIRLAYER; the two families are not merged (X and Y on one qubit do not
    commute), and the result equals the gate stream's."""
    n = 7
    rng = np.random.default_rng(3)
    ops = [{"name": "XXPHASE", "wires": [i, i + 1], "parameters": [float(rng.uniform(-1, 1))]} for i in range(n - 1)]
    ops += [{"name": "XXPHASE", "wires": [0, 5], "parameters": [0.3]}]
    ops += [{"name": "YYPHASE", "wires": [i, (i + 2) % n], "parameters": [float(rng.uniform(-1, 1))]}
            for i in range(n)]
    ops += [{"name": "RX", "wires": [2], "parameters": [0.4]}]
    ops += [{"name": "XXPHASE", "wires": [1, 3], "parameters": [0.2]}]
    layers = F.fuse(ops, n)
    pairs = [L for L in layers if L["name"] == "_PAIRLAYER"]
    assert [p["kind"] for p in pairs] == ["XX", "YY", "XX"]
    assert len(pairs[0]["bonds"]) == n and len(pairs[1]["bonds"]) == n
    vec = rand_state(n, 4, np.complex128)
    assert np.max(np.abs(interpret(layers, n, vec) - reference(ops, n, vec))) < 1e-12
    # at 30 qubits a chain over every qubit is two U(2) layers: 2 x 3 sweeps
    # (13-bit tiles: index bits 0-11, 12-20, 21-29; 12-bit tiles would need 4)
    chain = {"name": "_PAIRLAYER", "kind": "XX", "bonds": [(i, i + 1) for i in range(29)], "thetas": [0.1] * 29}
    assert F.expected_sweeps(chain, 30) == 6
    assert F.expected_sweeps(pairs[0], 30) == 2  # wires 0..6: the top bit group only
    chain28 = {"name": "_PAIRLAYER", "kind": "XX", "bonds": [(i, i + 1) for i in range(27)], "thetas": [0.1] * 27}
    assert F.expected_sweeps(chain28, 28) == 6  # 12-bit tiles: bits 0-11, 12-19, 20-27


def reference(ops, n, vec):
    o = OracleSim(n, np.complex128)
    o.set_state(vec)
    o.execute([op for op in ops])
    return o.state


def _mixed_ops(n, rng, count):
    names1 = ["H", "X", "Y", "Z", "S", "SDG", "T", "TDG", "SX", "I"]
    p1 = {"RX": 1, "RY": 1, "RZ": 1, "U1": 1, "U2": 2, "U3": 3}
    two = ["CNOT", "CZ", "SWAP", "CH", "ISWAP"]
    two_p = ["CPHASE", "CRX", "CRY", "CRZ", "XXPHASE", "YYPHASE", "ZZPHASE"]
    ops = []
    for _ in range(count):
        k = rng.integers(0, 5)
        if k == 0:
            ops.append({"name": str(rng.choice(names1)), "wires": [int(rng.integers(0, n))], "parameters": []})
        elif k == 1:
            nm = str(rng.choice(sorted(p1)))
            ops.append({"name": nm, "wires": [int(rng.integers(0, n))],
                        "parameters": [float(x) for x in rng.uniform(-3, 3, p1[nm])]})
        elif k == 2:
            w = rng.choice(n, 2, replace=False)
            ops.append({"name": str(rng.choice(two)), "wires": [int(x) for x in w], "parameters": []})
        elif k == 3:
            w = rng.choice(n, 2, replace=False)
            ops.append({"name": str(rng.choice(two_p)), "wires": [int(x) for x in w],
                        "parameters": [float(rng.uniform(-3, 3))]})
        else:
            w = rng.choice(n, 3, replace=False)
            ops.append({"name": str(rng.choice(["TOFFOLI", "FREDKIN"])), "wires": [int(x) for x in w],
                        "parameters": []})
    return ops


@pytest.mark.parametrize("seed", range(8))
def test_mixed_streams_fuse_exactly(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 8))
    ops = _mixed_ops(n, rng, 80)
    vec = rand_state(n, seed, np.complex128)
    got = interpret(F.fuse(ops, n), n, vec)
    assert np.max(np.abs(got - reference(ops, n, vec))) < 1e-10


@pytest.mark.parametrize("n", [3, 6, 9])
def test_qft_streams_collapse_to_stage_ranges(n):
    vec = rand_state(n, n, np.complex128)
    ops = W.qft_ops(n)
    layers = F.fuse(ops, n)
    assert [L["name"] for L in layers] == ["_QFTSTAGES"]
    assert (layers[0]["q0"], layers[0]["k"], layers[0]["j_begin"], layers[0]["j_end"]) == (0, n, 0, n)
    assert np.max(np.abs(interpret(layers, n, vec) - reference(ops, n, vec))) < 1e-10


def _iqft_ops(wires):
    ops = []
    m = len(wires)
    for j in reversed(range(m)):
        for k in reversed(range(j + 1, m)):
            ops.append({"name": "CPHASE", "wires": [wires[k], wires[j]], "parameters": [-math.pi / (1 << (k - j))]})
        ops.append({"name": "H", "wires": [wires[j]], "parameters": []})
    return ops


@pytest.mark.parametrize("lo,hi", [(0, 5), (2, 7), (1, 3)])
def test_inverse_and_subregister_qft_streams(lo, hi):
    n = 8
    vec = rand_state(n, 3, np.complex128)
    wires = list(range(lo, hi))
    for ops in (W.qft_ops(n, wires), _iqft_ops(wires)):
        layers = F.fuse(ops, n)
        assert len(layers) == 1 and layers[0]["name"] == "_QFTSTAGES"
        assert np.max(np.abs(interpret(layers, n, vec) - reference(ops, n, vec))) < 1e-10


def test_config_layer_structure_fuses_to_three_layers():
    c = W.plain_circuit(8, 3, seed=1)
    ops, gphase = c.ops()
    layers = F.fuse(ops, 8)
    assert [L["name"] for L in layers] == ["_LAYER"] * 3
    assert all(L["mats"] is not None and L["terms"] and L["rows"] is not None for L in layers)
    vec = rand_state(8, 1, np.complex128)
    got = interpret(layers, 8, vec) * np.exp(1j * gphase)
    o = OracleSim(8, np.complex128)
    o.set_state(vec)
    for L in c.layers:
        for q in range(8):
            o.apply_single(L.mats[q].reshape(2, 2), q)
        for i in range(7):
            o.apply_zz_phase(L.thetas[i] / 2.0, i, i + 1)
        for i in range(7):
            o.apply_controlled_single(np.array([[0, 1], [1, 0]]), i, i + 1)
    assert np.max(np.abs(got - o.state)) < 1e-10


def test_scale_circuit_fuses_to_logical_layers():
    c = W.scale_circuit(12, 20, seed=2)
    ops, gphase = c.ops()
    layers = F.fuse(ops, 12)
    # one fused layer per config layer, plus each QFT and permutation layer
    n_extra = sum(1 for L in c.layers if L.qft_after) + sum(1 for L in c.layers if L.xor is not None)
    assert len(layers) == len(c.layers) + n_extra
    vec = rand_state(12, 5, np.complex128)
    got = interpret(layers, 12, vec)
    assert np.max(np.abs(got - reference(ops, 12, vec))) < 1e-9


def test_asap_interleaved_stream_is_rescheduled():
    # Qiskit-style ASAP order: single-qubit gates interleaved with the ladder
    n = 6
    rng = np.random.default_rng(0)
    ops = []
    for q in range(n):
        ops.append({"name": "U3", "wires": [q], "parameters": [float(x) for x in rng.uniform(-3, 3, 3)]})
        if q:
            ops.append({"name": "CNOT", "wires": [q - 1, q], "parameters": []})
    layers = F.fuse(ops, n)
    vec = rand_state(n, 2, np.complex128)
    assert np.max(np.abs(interpret(layers, n, vec) - reference(ops, n, vec))) < 1e-10
    assert len(layers) <= 2 * n


def test_small_angle_rz_is_not_dropped():
    # mlxQMetalKernelsTest.py:369-390: RZ(1e-6) must survive window collapse
    ops = [{"name": "H", "wires": [0], "parameters": []}, {"name": "RZ", "wires": [0], "parameters": [1e-6]},
           {"name": "H", "wires": [0], "parameters": []}]
    layers = F.fuse(ops, 2)
    assert layers and layers[0]["name"] == "_U2LISTLAYER"
    vec = rand_state(2, 0, np.complex128)
    assert np.max(np.abs(interpret(layers, 2, vec) - reference(ops, 2, vec))) < 1e-14


def test_identity_window_emits_nothing():
    ops = [{"name": "H", "wires": [1], "parameters": []}, {"name": "H", "wires": [1], "parameters": []},
           {"name": "X", "wires": [0], "parameters": []}, {"name": "X", "wires": [0], "parameters": []}]
    assert F.fuse(ops, 3) == []


def test_all_x_window_is_a_flip_permutation():
    ops = [{"name": "X", "wires": [q], "parameters": []} for q in range(5)]
    layers = F.fuse(ops, 5)
    assert [L["name"] for L in layers] == ["_XORLAYER"]
    assert layers[0]["c"] == 31


def test_affine_run_matches_reference_composition():
    n = 6
    ops = ([{"name": "CNOT", "wires": [q, q + 1]} for q in range(n - 1)]
           + [{"name": "X", "wires": [3]}, {"name": "SWAP", "wires": [0, 5]}, {"name": "CNOT", "wires": [4, 1]}])
    rows, c = F.affine_of([dict(o, parameters=[]) for o in ops], n)
    assert (rows, c) == compose_inverse_affine(ops, n)


def test_affine_gate_synthesis_round_trip():
    rng = np.random.default_rng(11)
    for n in (1, 3, 7, 16):
        rows = W.invertible_rows(n, rng)
        c = int(rng.integers(0, 1 << n))
        gates = W.affine_gates(rows, c, n)
        assert F.affine_of(gates, n) == (rows, c)


def test_validation_errors():
    with pytest.raises(ValueError):
        F.fuse([{"name": "RX", "wires": [0], "parameters": []}], 2)
    with pytest.raises(ValueError):
        F.fuse([{"name": "CNOT", "wires": [0, 0], "parameters": []}], 2)
    with pytest.raises(ValueError):
        F.fuse([{"name": "H", "wires": [3], "parameters": []}], 2)
    with pytest.raises(ValueError):
        F.fuse([{"name": "FOO", "wires": [0], "parameters": []}], 2)


def test_fuse_layers_combinations():
    u = {"name": "_U2LISTLAYER", "mats": np.zeros((3, 4)), "active": [0]}
    d = {"name": "_DIAG", "terms": [(F.DIAG_RZ, 0, -1, [0.1])]}
    x = {"name": "_XORLAYER", "rows": [4, 2, 1], "c": 1}
    q = {"name": "_QFTSTAGES", "q0": 0, "k": 3, "j_begin": 0, "j_end": 3, "inverse": False}
    names = lambda ls: [L["name"] for L in ls]  # noqa: E731
    assert names(F.fuse_layers([u, d, x])) == ["_LAYER"]
    assert names(F.fuse_layers([u, x, q])) == ["_LAYER", "_QFTSTAGES"]
    assert names(F.fuse_layers([d, x, u])) == ["_LAYER", "_U2LISTLAYER"]
    assert names(F.fuse_layers([x, u, q, d])) == ["_XORLAYER", "_U2LISTLAYER", "_QFTSTAGES", "_DIAG"]
    L = F.fuse_layers([d, x])[0]
    assert L["mats"] is None and L["rows"] == [4, 2, 1] and L["c"] == 1


def test_expected_sweeps_of_fused_config_layer():
    c = W.plain_circuit(30, 1, seed=0)
    ops, _ = c.ops()
    layers = F.fuse(ops, 30)
    assert [L["name"] for L in layers] == ["_LAYER"]
    # 30 index bits in three tile groups (13-bit tiles); diagonal and ladder
    # ride on the low sweep
    assert F.expected_sweeps(layers[0], 30) == 3
