"""Gate-stream -> layer fusion (host side of the runtime).

Turns a list of canonical op dicts ``{"name", "wires", "parameters"}``
(integrations/_common.py:86-115) into the fused layer ops that the kernels
execute, with the detection semantics of the reference's
``Device._fuse_zz_layers`` (device.py:608-1087) and its dependency scheduler
(device.py:557-606):

* single-qubit windows collapse per wire into one 2x2 product in complex128,
  with rtol=0 / atol=1e-12 identity tests so small angles survive
  (device.py:683-755); an all-diagonal window becomes diagonal terms, an
  all-X window a bit-flip permutation, anything else one U(2) layer;
* runs of diagonal gates (Z/S/T/RZ/U1, CZ/CPHASE/CRZ, ZZPHASE, with any
  angles) commute and become one diagonal layer (device.py:895-965);
* runs of X/CNOT/SWAP become one GF(2) affine permutation
  (device.py:807-834, xor_affine.py:46-76);
* forward and inverse QFT stage patterns (H + CPHASE ladder, or the
  descending negative ladder + H) become QFT stage ranges
  (device.py:835-894, 992-1028);
* CH/CRX/CRY/Toffoli runs become controlled-U(2) lists (device.py:756-806).

Composite gates are rewritten first: ISWAP = diag(1,i,i,1) then SWAP
(device.py:1233-1236); FREDKIN = CNOT(b,a) TOFFOLI(c,a,b) CNOT(b,a).  Runs
of XXPHASE (or of YYPHASE) terms become one ``_PAIRLAYER``: the basis change
H (or V = S H) on their wires around one ZZ layer (the conjugation of
shaders/pauli_pair.py:32-64), which the engine runs as one fused layer (the
basis change's sweeps carrying the ZZ terms) and one U(2) layer.
"""
from __future__ import annotations

import math
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import gates as G

# kinds shared with the C ABI (include/mq.h)
DIAG_ZZ, DIAG_CPHASE, DIAG_RZ, DIAG_PHASE, DIAG_CRZ, DIAG_GLOBAL, DIAG_1Q, DIAG_2Q = range(8)

ARITIES = {"H": 1, "I": 1, "X": 1, "Y": 1, "Z": 1, "S": 1, "SDG": 1, "T": 1, "TDG": 1, "SX": 1,
           "RX": 1, "RY": 1, "RZ": 1, "U1": 1, "U2": 1, "U3": 1,
           "CNOT": 2, "CH": 2, "CZ": 2, "CPHASE": 2, "CRX": 2, "CRY": 2, "CRZ": 2, "SWAP": 2, "ISWAP": 2,
           "XXPHASE": 2, "YYPHASE": 2, "ZZPHASE": 2, "TOFFOLI": 3, "FREDKIN": 3}
PARAMS = {"RX": 1, "RY": 1, "RZ": 1, "U1": 1, "U2": 2, "U3": 3, "CPHASE": 1, "CRX": 1, "CRY": 1, "CRZ": 1,
          "XXPHASE": 1, "YYPHASE": 1, "ZZPHASE": 1}

_EYE = np.eye(2, dtype=np.complex128)
_X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
_V = np.array([[1, 0], [0, 1j]], dtype=np.complex128) @ G.single_qubit_matrix("H")  # S H: V Z V^+ = Y


def _is(m: np.ndarray, ref: np.ndarray) -> bool:
    """Every entry within 1e-12 of ``ref`` (allclose with rtol=0, without its
    per-call overhead: this runs once per fused window)."""
    return float(np.abs(m - ref).max()) <= 1e-12


def normalize(ops: Sequence[dict], n: int) -> List[dict]:
    """Canonical names, validated arity/wires/parameter counts."""
    out = []
    append = out.append
    names: Dict[Any, str] = {}  # raw name -> canonical name, per call
    for op in ops:
        raw = op.get("name", "")
        name = names.get(raw)
        if name is None:
            name = names[raw] = G.canonical_name(raw)
        wires = [int(w) for w in op.get("wires", ())]
        params = [float(p) for p in (op.get("parameters") or ())]
        if name[:1] == "_":
            append(dict(op))
            continue
        arity = ARITIES.get(name)
        if arity is None:
            raise ValueError(f"Unsupported operation: {raw}")
        if len(wires) != arity:
            raise ValueError(f"{name} expects {arity} wire(s), got {len(wires)}")
        if len(params) < PARAMS.get(name, 0):
            raise ValueError(f"{name} expects {PARAMS.get(name, 0)} parameter(s), got {len(params)}")
        for w in wires:
            if not (0 <= w < n):
                raise ValueError("Qubit index out of range")
        if arity > 1 and len(set(wires)) != arity:
            raise ValueError("Control/target wires must be distinct")
        append({"name": name, "wires": wires, "parameters": params})
    return out


def decompose(ops: Sequence[dict]) -> List[dict]:
    out: List[dict] = []
    for op in ops:
        name, w, p = op["name"], op.get("wires", []), op.get("parameters", [])
        if name == "ISWAP":
            out.append({"name": "_D2", "wires": list(w), "diag": [1, 1j, 1j, 1]})
            out.append({"name": "SWAP", "wires": list(w), "parameters": []})
        elif name in ("XXPHASE", "YYPHASE"):
            # a pair term; runs of one family become one _PAIRLAYER
            out.append({"name": "_XXPAIR" if name == "XXPHASE" else "_YYPAIR", "wires": list(w),
                        "parameters": [p[0]]})
        elif name == "FREDKIN":
            c, a, b = w
            out.append({"name": "CNOT", "wires": [b, a], "parameters": []})
            out.append({"name": "TOFFOLI", "wires": [c, a, b], "parameters": []})
            out.append({"name": "CNOT", "wires": [b, a], "parameters": []})
        else:
            out.append(op)
    return out


def _category(op: dict) -> str:
    name = op["name"]
    if len(op.get("wires", [])) == 1 and name != "_QFTSTAGE":
        return "single"
    if name in DIAG_TWO:
        return "diag"
    if name in AFFINE:
        return "affine"
    if name in CONTROLLED:
        return "controlled"
    return "other:" + name


def dependency_schedule(ops: Sequence[dict]) -> List[dict]:
    """Topological re-order of the per-wire dependency DAG that exposes
    fusable layers (device.py:557-606 hoists ready single-qubit ops).

    Ops on the same wire keep their order; only ops on disjoint wires move.
    Policy: keep extending the current multi-qubit run while ops of its
    category are ready (so a CNOT ladder or a ZZ chain is not interrupted by
    hoisted one-qubit gates), otherwise emit every ready one-qubit op,
    otherwise start the category of the earliest ready op."""
    import heapq
    count = len(ops)
    if count < 2:
        return list(ops)
    indeg = [0] * count
    succ: List[List[int]] = [[] for _ in range(count)]
    last: Dict[int, int] = {}
    for i, op in enumerate(ops):
        wires = op.get("wires", ())
        if len(wires) == 1:
            p = last.get(wires[0])
            if p is not None:
                indeg[i] = 1
                succ[p].append(i)
            last[wires[0]] = i
            continue
        preds = {last[w] for w in wires if w in last}
        indeg[i] = len(preds)
        for p in preds:
            succ[p].append(i)
        for w in wires:
            last[w] = i
    cats = [_category(op) for op in ops]
    ready: Dict[str, list] = {}
    for i in range(count):
        if indeg[i] == 0:
            heapq.heappush(ready.setdefault(cats[i], []), i)
    out: List[dict] = []
    current: Optional[str] = None

    def emit(i):
        out.append(ops[i])
        for s_ in succ[i]:
            indeg[s_] -= 1
            if indeg[s_] == 0:
                heapq.heappush(ready.setdefault(cats[s_], []), s_)

    while len(out) < count:
        if current is not None and ready.get(current):
            batch = [heapq.heappop(ready[current]) for _ in range(len(ready[current]))]
            for i in batch:
                emit(i)
            continue
        if ready.get("single"):
            batch = [heapq.heappop(ready["single"]) for _ in range(len(ready["single"]))]
            for i in batch:
                emit(i)
            current = None
            continue
        nonempty = [(h[0], c) for c, h in ready.items() if h]
        if not nonempty:
            raise RuntimeError("operation dependency graph contains a cycle")
        current = min(nonempty)[1]
    return out


# ---------------------------------------------------------------- GF(2)
def affine_of(ops: Sequence[dict], n: int) -> Tuple[List[int], int]:
    """Inverse-map rows and flip of an X/CNOT/SWAP run (xor_affine.py:46-76)."""
    rows = [1 << (n - 1 - k) for k in range(n)]
    c = 0
    for op in reversed(list(ops)):
        name, w = op["name"], op["wires"]
        if name == "X":
            c ^= 1 << (n - 1 - w[0])
        elif name == "CNOT":
            a, b = w
            rows[b] ^= rows[a]
            if (c >> (n - 1 - a)) & 1:
                c ^= 1 << (n - 1 - b)
        elif name == "SWAP":
            a, b = w
            rows[a], rows[b] = rows[b], rows[a]
            if ((c >> (n - 1 - a)) & 1) != ((c >> (n - 1 - b)) & 1):
                c ^= (1 << (n - 1 - a)) | (1 << (n - 1 - b))
        else:
            raise ValueError(f"Not a GF(2) affine gate: {name}")
    return rows, c


def _src(rows: Sequence[int], c: int, n: int, y: int) -> int:
    s = 0
    for k, r in enumerate(rows):
        s |= (bin(r & y).count("1") & 1) << (n - 1 - k)
    return s ^ c


def compose_affine(first: Tuple[List[int], int], second: Tuple[List[int], int], n: int) -> Tuple[List[int], int]:
    """Rows/flip of applying ``first`` then ``second`` (both as out[y]=in[src(y)])."""
    r1, c1 = first
    r2, c2 = second
    # total src(y) = src1(src2(y)); linear part column j = L1(L2 e_j)
    c = _src(r1, c1, n, _src(r2, c2, n, 0))
    cols = [_src(r1, c1, n, _src(r2, c2, n, 1 << j)) ^ c for j in range(n)]
    rows = []
    for k in range(n):
        bit = n - 1 - k
        rows.append(sum(((cols[j] >> bit) & 1) << j for j in range(n)))
    return rows, c


# ---------------------------------------------------------------- diagonals
def diag_terms_of(op: dict, n: int) -> List[tuple]:
    name, w, p = op["name"], op.get("wires", []), op.get("parameters", [])
    if name == "Z":
        return [(DIAG_PHASE, w[0], -1, [math.pi])]
    if name in ("S", "SDG", "T", "TDG", "RZ", "U1"):
        m = G.single_qubit_matrix(name, p)
        d0, d1 = m[0, 0], m[1, 1]
        return [(DIAG_1Q, w[0], -1, [d0.real, d0.imag, d1.real, d1.imag])]
    if name == "CZ":
        return [(DIAG_CPHASE, w[0], w[1], [math.pi])]
    if name == "CPHASE":
        return [(DIAG_CPHASE, w[0], w[1], [p[0]])]
    if name == "CRZ":
        return [(DIAG_CRZ, w[0], w[1], [p[0]])]
    if name == "ZZPHASE":
        return [(DIAG_ZZ, w[0], w[1], [p[0]])]
    if name == "_D2":
        d = [complex(x) for x in op["diag"]]
        return [(DIAG_2Q, w[0], w[1], [v for z in d for v in (z.real, z.imag)])]
    raise ValueError(f"not diagonal: {name}")


DIAG_TWO = {"CZ", "CPHASE", "CRZ", "ZZPHASE", "_D2"}
AFFINE = {"X", "CNOT", "SWAP"}
CONTROLLED = {"CH", "CRX", "CRY", "TOFFOLI"}


def _single_matrix(op: dict) -> np.ndarray:
    if op["name"] == "_M1":
        return np.asarray(op["matrix"], dtype=np.complex128)
    return G.single_qubit_matrix(op["name"], op.get("parameters", []))


def _cphase_of(op: dict):
    if op["name"] != "CPHASE":
        return None
    return list(op["wires"]), float(op["parameters"][0])


def _qft_forward_stage(ops, i):
    """H(j) + CPHASE([k, j], pi/2^(k-j)) for k = j+1.. (device.py:854-871)."""
    op = ops[i]
    if op["name"] != "H":
        return None
    jq = op["wires"][0]
    j2, kk = i + 1, jq + 1
    while j2 < len(ops):
        cp = _cphase_of(ops[j2])
        if cp is not None and cp[0] == [kk, jq] and cp[1] == math.pi / (1 << (kk - jq)):
            kk += 1
            j2 += 1
        else:
            break
    if kk > jq + 1:
        return (jq, kk, j2)  # stage j on subregister [j, m=kk), next index
    return None


def _qft_inverse_stage(ops, i):
    """Descending CPHASE([k, j], -pi/2^(k-j)) then H(j) (device.py:872-894)."""
    cp0 = _cphase_of(ops[i])
    if cp0 is None or cp0[1] >= 0:
        return None
    (k0, jq), _ = cp0
    kk, j2 = k0, i
    while kk > jq:
        cp = _cphase_of(ops[j2]) if j2 < len(ops) else None
        if cp is not None and cp[0] == [kk, jq] and cp[1] == -math.pi / (1 << (kk - jq)):
            kk -= 1
            j2 += 1
        else:
            return None
    if j2 < len(ops) and ops[j2]["name"] == "H" and ops[j2]["wires"] == [jq]:
        return (jq, k0 + 1, j2 + 1)
    return None


def _mark_qft_stages(ops: List[dict]) -> List[dict]:
    """Replace forward / inverse QFT stage patterns by _QFTSTAGE pseudo-ops
    (wires = the stage's subregister) before any re-ordering."""
    out: List[dict] = []
    i, N = 0, len(ops)
    while i < N:
        st = _qft_forward_stage(ops, i)
        inv = False
        if st is None:
            st = _qft_inverse_stage(ops, i)
            inv = st is not None
        if st is not None:
            j, m, nxt = st
            out.append({"name": "_QFTSTAGE", "j": j, "m": m, "inverse": inv, "wires": list(range(j, m))})
            i = nxt
            continue
        out.append(ops[i])
        i += 1
    return out


def fuse(operations: Sequence[dict], n: int, *, schedule: bool = True) -> List[Dict[str, Any]]:
    ops = _mark_qft_stages(decompose(normalize(operations, n)))
    if schedule:
        ops = dependency_schedule(ops)
    fused: List[Dict[str, Any]] = []
    i = 0
    N = len(ops)
    while i < N:
        op = ops[i]
        name = op["name"]
        if name == "_QFTSTAGE":
            fused.append({k: op[k] for k in ("name", "j", "m", "inverse")})
            i += 1
            continue
        if len(op.get("wires", [])) == 1:
            j = i
            per_wire: Dict[int, np.ndarray] = {}
            while j < N and len(ops[j].get("wires", [])) == 1 and ops[j]["name"] != "_QFTSTAGE":
                q = ops[j]["wires"][0]
                per_wire[q] = _single_matrix(ops[j]) @ per_wire.get(q, _EYE)
                j += 1
            fused.extend(_window_layer(per_wire, n))
            i = j
            continue
        if name in DIAG_TWO:
            terms = []
            j = i
            while j < N and (ops[j]["name"] in DIAG_TWO):
                terms.extend(diag_terms_of(ops[j], n))
                j += 1
            fused.append({"name": "_DIAG", "terms": terms})
            i = j
            continue
        if name in AFFINE:
            j = i
            while j < N and ops[j]["name"] in AFFINE:
                j += 1
            rows, c = affine_of(ops[i:j], n)
            fused.append({"name": "_XORLAYER", "rows": rows, "c": c})
            i = j
            continue
        if name in ("_XXPAIR", "_YYPAIR"):
            # exp(-i sum_b t_b P_a P_b), P = X or Y: the terms of one family
            # commute, so the run is one basis change around one ZZ layer
            # (shaders/pauli_pair.py:32-64)
            bonds, thetas = [], []
            j = i
            while j < N and ops[j]["name"] == name:
                bonds.append(tuple(ops[j]["wires"]))
                thetas.append(float(ops[j]["parameters"][0]))
                j += 1
            fused.append({"name": "_PAIRLAYER", "kind": "XX" if name == "_XXPAIR" else "YY",
                          "bonds": bonds, "thetas": thetas})
            i = j
            continue
        if name in CONTROLLED:
            gates = []
            j = i
            while j < N and ops[j]["name"] in CONTROLLED:
                w = ops[j]["wires"]
                gates.append((list(w[:-1]), w[-1], G.controlled_target_matrix(ops[j]["name"], ops[j]["parameters"])))
                j += 1
            fused.append({"name": "_CULIST", "gates": gates})
            i = j
            continue
        if name.startswith("_"):
            fused.append(op)
            i += 1
            continue
        raise ValueError(f"Unsupported operation for the statevector engine: {name}")
    return fuse_layers(_merge(fused, n))


def fuse_layers(layers: List[dict]) -> List[dict]:
    """Combine a U(2) layer with the diagonal layer and / or permutation
    that follow it (in that order), or a diagonal with the permutation after
    it, into one ``_LAYER``: the engine applies the three in the sweeps of
    the U(2) layer alone (one config-0 layer is u2_list_layer_all +
    zz_weighted_layer + xor_affine_gather in the reference,
    device.py:1089-1097)."""
    out: List[dict] = []
    i, N = 0, len(layers)
    while i < N:
        L = layers[i]
        if L["name"] not in ("_U2LISTLAYER", "_DIAG"):
            out.append(L)
            i += 1
            continue
        fusedl = {"name": "_LAYER", "mats": None, "active": None, "terms": [], "rows": None, "c": 0}
        j = i
        if layers[j]["name"] == "_U2LISTLAYER":
            fusedl["mats"], fusedl["active"] = layers[j]["mats"], layers[j]["active"]
            j += 1
        if j < N and layers[j]["name"] == "_DIAG":
            fusedl["terms"] = layers[j]["terms"]
            j += 1
        if j < N and layers[j]["name"] == "_XORLAYER":
            fusedl["rows"], fusedl["c"] = layers[j]["rows"], layers[j]["c"]
            j += 1
        if j - i >= 2:
            out.append(fusedl)
        else:
            out.append(L)
        i = max(j, i + 1)
    return out


def _window_layer(per_wire: Dict[int, np.ndarray], n: int) -> List[dict]:
    active = {q: m for q, m in per_wire.items() if not _is(m, _EYE)}
    if not active:
        return []
    if all(abs(m[0, 1]) <= 1e-15 and abs(m[1, 0]) <= 1e-15 for m in active.values()):
        terms = []
        for q in sorted(active):
            d0, d1 = active[q][0, 0], active[q][1, 1]
            terms.append((DIAG_1Q, q, -1, [d0.real, d0.imag, d1.real, d1.imag]))
        return [{"name": "_DIAG", "terms": terms}]
    if all(_is(m, _X) for m in active.values()):
        c = 0
        for q in active:
            c ^= 1 << (n - 1 - q)
        return [{"name": "_XORLAYER", "rows": [1 << (n - 1 - k) for k in range(n)], "c": c}]
    mats = np.tile(_EYE.reshape(1, 4), (n, 1))
    for q, m in active.items():
        mats[q] = m.reshape(4)
    return [{"name": "_U2LISTLAYER", "mats": mats, "active": sorted(active)}]


def _merge(fused: List[dict], n: int) -> List[dict]:
    out: List[dict] = []
    for op in fused:
        prev = out[-1] if out else None
        if prev is not None and prev["name"] == "_DIAG" and op["name"] == "_DIAG":
            prev["terms"] = prev["terms"] + op["terms"]
            continue
        if prev is not None and prev["name"] == "_XORLAYER" and op["name"] == "_XORLAYER":
            rows, c = compose_affine((prev["rows"], prev["c"]), (op["rows"], op["c"]), n)
            prev["rows"], prev["c"] = rows, c
            continue
        if prev is not None and prev["name"] == "_QFTSTAGES" and op["name"] == "_QFTSTAGE":
            q0, k, jb, je, inv = prev["q0"], prev["k"], prev["j_begin"], prev["j_end"], prev["inverse"]
            if op["m"] == q0 + k and op["inverse"] == inv:
                if not inv and op["j"] == q0 + je:
                    prev["j_end"] += 1
                    continue
                if inv and op["j"] == q0 + jb - 1 and jb > 0:
                    prev["j_begin"] -= 1
                    continue
                if inv and op["j"] == q0 - 1 and jb == 0:
                    # extend the subregister downward: stage j of [j, m)
                    prev["q0"], prev["k"] = op["j"], k + 1
                    prev["j_end"] = je + 1
                    continue
        if op["name"] == "_QFTSTAGE":
            j, m, inv = op["j"], op["m"], op["inverse"]
            # an inverse transform opens with a bare H(m-1): its stage of width 0
            if (inv and m == j + 2 and prev is not None and prev["name"] == "_U2LISTLAYER"
                    and prev["active"] == [m - 1]
                    and _is(prev["mats"][m - 1].reshape(2, 2), G.single_qubit_matrix("H"))):
                out[-1] = {"name": "_QFTSTAGES", "q0": j, "k": 2, "j_begin": 0, "j_end": 2, "inverse": True}
                continue
            out.append({"name": "_QFTSTAGES", "q0": j, "k": m - j, "j_begin": 0, "j_end": 1, "inverse": inv})
            continue
        # a bare H(m-1) right after forward stages ending at m-2 is the last stage
        if (prev is not None and prev["name"] == "_QFTSTAGES" and not prev["inverse"]
                and op["name"] == "_U2LISTLAYER" and op["active"] == [prev["q0"] + prev["k"] - 1]
                and prev["q0"] + prev["j_end"] == prev["q0"] + prev["k"] - 1
                and _is(op["mats"][op["active"][0]].reshape(2, 2), G.single_qubit_matrix("H"))):
            prev["j_end"] += 1
            continue
        out.append(op)
    return out


def _split_bits(n: int, tmax: int, pas: int) -> List[Tuple[int, int]]:
    """Index-bit groups of the tile sweeps (mq_tile.cu split_bits)."""
    if n <= tmax:
        return [(0, n)]
    hi_cap = tmax - pas
    n_hi = -(-(n - tmax) // hi_cap)
    low = max(n - n_hi * hi_cap, min(tmax, (n + n_hi) // (n_hi + 1)))
    groups, start, rest = [(0, low)], low, n - low
    for i in range(n_hi):
        cnt = rest // n_hi + (1 if i < rest % n_hi else 0)
        groups.append((start, cnt))
        start += cnt
    return groups


def expected_sweeps(layer: dict, n: int, dtype: str = "complex64") -> int:
    """Full-state passes a fused layer launches (for execution reports), from
    the engine's default tile plan: complex64 tiles of 13 bits from 29 qubits
    and of 12 bits below (mq_tile.cu tile_max), complex128 tiles of 11 bits,
    4 low passenger bits."""
    tmax = (13 if n >= 29 else 12) if dtype == "complex64" else 11
    pas = 4
    name = layer["name"]
    groups = _split_bits(n, tmax, pas)

    def u2_sweeps(active):
        bits = {n - 1 - q for q in active}
        return sum(1 for st, cnt in groups if any(st <= b < st + cnt for b in bits))

    if name == "_U2LISTLAYER":
        return u2_sweeps(layer["active"])
    if name == "_LAYER":
        hi = u2_sweeps(layer["active"]) if layer["mats"] is not None else 0
        low_bits = {n - 1 - q for q in (layer["active"] or [])}
        m = min(n, max(groups[0][1], 10))
        if layer["mats"] is not None and any(b < groups[0][1] for b in low_bits):
            hi -= 1  # the low sweep is counted below
        terms = layer["terms"]
        far = any(b >= 0 and abs(a - b) >= 10 for _, a, b, _ in terms)
        extra = 1 if far and terms else 0
        perm_low = True
        if layer["rows"] is not None:
            rows = layer["rows"]
            # columns A e_j for index bits j < m must stay below bit m
            for j in range(m):
                col = 0
                for k, r in enumerate(rows):
                    if (r >> j) & 1:
                        col |= 1 << (n - 1 - k)
                if col >> m:
                    perm_low = False
            if not perm_low or extra:
                extra += 1
        return hi + 1 + extra
    if name in ("_DIAG", "_XORLAYER"):
        return 1
    if name == "_PAIRLAYER":
        wires = sorted({w for b in layer["bonds"] for w in b})
        return 2 * u2_sweeps(wires)
    if name == "_QFTSTAGES":
        cnt = layer["j_end"] - layer["j_begin"]
        return 1 if cnt + pas <= tmax else -(-cnt // (tmax - pas))
    if name == "_CULIST":
        return max(1, len(layer["gates"]))
    return 1
