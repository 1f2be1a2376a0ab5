"""Gate matrices (complex128 numpy) with the reference's definitions.

Same matrices as MettleQ gates.py:5-234: RX(t) = [[c, -is], [-is, c]],
RY(t) = [[c, -s], [s, c]], RZ(t) = diag(e^{-it/2}, e^{+it/2}),
U1(l) = diag(1, e^{il}), U2(p, l) = RZ(p) RY(pi/2) RZ(l),
U3(t, p, l) = RZ(p) RY(t) RZ(l).  Built in double precision on the host and
handed to the kernels as doubles.
"""
from __future__ import annotations

import math
from typing import Sequence

import numpy as np

_SQ = 1.0 / math.sqrt(2.0)

ALIASES = {"CX": "CNOT", "CP": "CPHASE", "CCX": "TOFFOLI", "CSWAP": "FREDKIN",
           "SDAG": "SDG", "TDAG": "TDG", "S†": "SDG", "T†": "TDG", "P": "U1", "PHASESHIFT": "U1"}


def canonical_name(name: str) -> str:
    n = str(name).upper()
    return ALIASES.get(n, n)


def rz(theta: float) -> np.ndarray:
    h = theta / 2.0
    return np.array([[complex(math.cos(h), -math.sin(h)), 0], [0, complex(math.cos(h), math.sin(h))]],
                    dtype=np.complex128)


def ry(theta: float) -> np.ndarray:
    c, s = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def rx(theta: float) -> np.ndarray:
    c, s = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)


def phase(lam: float) -> np.ndarray:
    return np.array([[1, 0], [0, complex(math.cos(lam), math.sin(lam))]], dtype=np.complex128)


_CONST = {
    "I": np.eye(2, dtype=np.complex128),
    "X": np.array([[0, 1], [1, 0]], dtype=np.complex128),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    "Z": np.array([[1, 0], [0, -1]], dtype=np.complex128),
    "H": np.array([[_SQ, _SQ], [_SQ, -_SQ]], dtype=np.complex128),
    "S": np.array([[1, 0], [0, 1j]], dtype=np.complex128),
    "SDG": np.array([[1, 0], [0, -1j]], dtype=np.complex128),
    "T": np.array([[1, 0], [0, complex(math.cos(math.pi / 4), math.sin(math.pi / 4))]], dtype=np.complex128),
    "TDG": np.array([[1, 0], [0, complex(math.cos(math.pi / 4), -math.sin(math.pi / 4))]], dtype=np.complex128),
    "SX": np.array([[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]], dtype=np.complex128),
}

SINGLE_PARAMS = {"RX": 1, "RY": 1, "RZ": 1, "U1": 1, "U2": 2, "U3": 3}
DIAG_SINGLE = {"Z", "S", "SDG", "T", "TDG", "RZ", "U1"}


def single_qubit_matrix(name: str, params: Sequence[float] = ()) -> np.ndarray:
    name = canonical_name(name)
    p = [float(x) for x in params]
    if name in _CONST:
        return _CONST[name].copy()
    if name == "RX":
        return rx(p[0])
    if name == "RY":
        return ry(p[0])
    if name == "RZ":
        return rz(p[0])
    if name == "U1":
        return phase(p[0])
    if name == "U2":
        return _u3(math.pi / 2.0, p[0], p[1])
    if name == "U3":
        return _u3(p[0], p[1], p[2])
    raise ValueError(f"Unsupported single-qubit op: {name}")


def _u3(theta: float, phi: float, lam: float) -> np.ndarray:
    """RZ(phi) RY(theta) RZ(lam) multiplied out:
    [[e^{-i(phi+lam)/2} c, -e^{-i(phi-lam)/2} s], [e^{i(phi-lam)/2} s, e^{i(phi+lam)/2} c]]."""
    c, s = math.cos(theta / 2.0), math.sin(theta / 2.0)
    a, b = (phi + lam) / 2.0, (phi - lam) / 2.0
    ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
    return np.array([[complex(ca * c, -sa * c), complex(-cb * s, sb * s)],
                     [complex(cb * s, sb * s), complex(ca * c, sa * c)]], dtype=np.complex128)


def controlled_target_matrix(name: str, params: Sequence[float] = ()) -> np.ndarray:
    """Target matrix of CH / CRX / CRY (gates.py:141-177)."""
    name = canonical_name(name)
    if name == "CH":
        return _CONST["H"].copy()
    if name == "CRX":
        return rx(float(params[0]))
    if name == "CRY":
        return ry(float(params[0]))
    if name == "TOFFOLI":
        return _CONST["X"].copy()
    raise ValueError(f"Unsupported controlled op: {name}")
