"""Generate golden vectors by running the reference's own CPU statevector code.

Run in a container that has the MettleQ source tree (it is not needed, and
not read, anywhere else):

    python tests/golden/make_golden.py /path/to/MettleQ/src

The reference imports ``mlx.core`` everywhere; ``oracle/mlx_shim``
supplies a numpy-backed stand-in, with ``metal.is_available() == False`` so
that ``Device(n, execution_device="cpu")`` takes its pure per-gate path
(device.py:1138-1290, sim.py).  Outputs land in ``tests/golden/*.npz`` and
``tests/golden/cases.json``; the tests read only those files.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _ops_mixed(n: int, rng: np.random.Generator, count: int):
    one = ["H", "X", "Y", "Z", "S", "SDG", "T", "TDG", "SX", "I"]
    one_p = {"RX": 1, "RY": 1, "RZ": 1, "U1": 1, "U2": 2, "U3": 3}
    two = ["CNOT", "CZ", "SWAP", "CH", "ISWAP"]
    two_p = ["CPHASE", "CRX", "CRY", "CRZ", "XXPHASE", "YYPHASE", "ZZPHASE"]
    three = ["TOFFOLI", "FREDKIN"]
    ops = []
    for _ in range(count):
        kind = rng.integers(0, 5)
        if kind == 0:
            ops.append({"name": str(rng.choice(one)), "wires": [int(rng.integers(0, n))], "parameters": []})
        elif kind == 1:
            name = str(rng.choice(sorted(one_p)))
            ops.append({"name": name, "wires": [int(rng.integers(0, n))],
                        "parameters": [float(x) for x in rng.uniform(-math.pi, math.pi, one_p[name])]})
        elif kind == 2:
            w = rng.choice(n, 2, replace=False)
            ops.append({"name": str(rng.choice(two)), "wires": [int(x) for x in w], "parameters": []})
        elif kind == 3:
            w = rng.choice(n, 2, replace=False)
            ops.append({"name": str(rng.choice(two_p)), "wires": [int(x) for x in w],
                        "parameters": [float(rng.uniform(-math.pi, math.pi))]})
        else:
            w = rng.choice(n, 3, replace=False)
            ops.append({"name": str(rng.choice(three)), "wires": [int(x) for x in w], "parameters": []})
    return ops


def _ops_layers(n: int, rng: np.random.Generator, layers: int, uniform_zz: bool):
    """Config-0 structure with U3 single-qubit gates: U3 on every qubit,
    ZZPHASE on (i, i+1), CNOT ladder 0->1->...->n-1."""
    ops = []
    for _ in range(layers):
        for q in range(n):
            ops.append({"name": "U3", "wires": [q],
                        "parameters": [float(x) for x in rng.uniform(-math.pi, math.pi, 3)]})
        th = float(rng.uniform(0, 2 * math.pi))
        for q in range(n - 1):
            t = th if uniform_zz else float(rng.uniform(0, 2 * math.pi))
            ops.append({"name": "ZZPHASE", "wires": [q, q + 1], "parameters": [t / 2.0]})
        for q in range(n - 1):
            ops.append({"name": "CNOT", "wires": [q, q + 1], "parameters": []})
    return ops


def main(src_root: str) -> None:
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "mlx_shim"))
    sys.path.insert(0, src_root)
    import mlx.core as mx  # the shim
    from mettleq.device import Device
    from mettleq.sim import StateVectorSimulator, qft, iqft
    from mettleq.shaders.xor_affine import compose_inverse_affine
    from mettleq.integrations import _common

    rng = np.random.default_rng(20261203)
    cases = []
    arrays = {}

    def run_device(tag, n, ops, phase=0.0):
        dev = Device(n, execution_device="cpu")
        dev.execute(ops)
        if phase:
            _common.apply_global_phase(dev, phase)
        arrays[tag] = np.asarray(dev.sim.state, dtype=np.complex64)
        cases.append({"tag": tag, "kind": "device", "n": n, "ops": ops, "global_phase": phase})
        return dev

    # 1. mixed gate streams through Device.execute (all arities, all names)
    for i, n in enumerate((3, 5, 7)):
        run_device(f"mixed_{i}", n, _ops_mixed(n, rng, 60))
    # 2. config-0-shaped layers (distinct and uniform ZZ angles)
    run_device("layers_distinct", 8, _ops_layers(8, rng, 4, False))
    dev = run_device("layers_uniform", 8, _ops_layers(8, rng, 4, True), phase=0.7)
    # 3. probabilities on wire subsets (sim.py:322-343)
    for wires in ([0], [7], [3, 1], [2, 5, 0], list(range(8)), [7, 6, 5, 4, 3, 2, 1, 0]):
        tag = "probs_" + "_".join(map(str, wires))
        arrays[tag] = np.asarray(dev.sim.probabilities_array(wires), dtype=np.float32)
        cases.append({"tag": tag, "kind": "probs", "source": "layers_uniform", "wires": wires})
    # 4. Pauli words (integrations/_common.py:384-427)
    words = [{0: "Z"}, {0: "Z", 1: "Z"}, {3: "X"}, {2: "Y", 5: "Z"}, {1: "X", 4: "Y", 7: "Z"}, {}]
    vals = _common.pauli_product_expectations(dev, words)
    arrays["pauli_layers_uniform"] = np.asarray(vals, dtype=np.complex128)
    cases.append({"tag": "pauli_layers_uniform", "kind": "pauli", "source": "layers_uniform",
                  "words": [{str(k): v for k, v in w.items()} for w in words]})
    # 5. QFT / iQFT on random states and ordered subsets (sim.py:522-563)
    for i, (n, wires, inverse) in enumerate(((5, list(range(5)), False), (5, [3, 0, 4], False),
                                             (6, [5, 1, 2, 0], True), (6, list(range(6)), True))):
        v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        v = (v / np.linalg.norm(v)).astype(np.complex64)
        sim = StateVectorSimulator(n)
        sim.state = mx.array(v)
        (iqft if inverse else qft)(sim, wires)
        arrays[f"qft_{i}_in"] = v
        arrays[f"qft_{i}_out"] = np.asarray(sim.state, dtype=np.complex64)
        cases.append({"tag": f"qft_{i}", "kind": "qft", "n": n, "wires": wires, "inverse": inverse})
    # 6. affine composition of CNOT/X/SWAP runs (xor_affine.py:46-76)
    for i, n in enumerate((6, 9, 12)):
        ops = []
        for _ in range(3 * n):
            k = rng.integers(0, 3)
            if k == 0:
                ops.append({"name": "X", "wires": [int(rng.integers(0, n))]})
            else:
                w = rng.choice(n, 2, replace=False)
                ops.append({"name": "CNOT" if k == 1 else "SWAP", "wires": [int(x) for x in w]})
        rows, c = compose_inverse_affine(ops, n)
        cases.append({"tag": f"affine_{i}", "kind": "affine", "n": n, "ops": ops, "rows": rows, "c": c})

    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **arrays)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(cases, f, indent=1)
    print(f"wrote {len(cases)} cases, {len(arrays)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the MettleQ src directory>")
    main(sys.argv[1])
