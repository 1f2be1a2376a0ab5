"""One statevector sharded over P = 2^g processes (one per GPU).

The reference holds a state on one device (sim.py:17-45); past one GPU's
memory (33 qubits and up in complex64 on B200s) the state is split by its top
g index bits: process r holds the 2^(n-g) amplitudes whose top bits equal r,
as an (n-g)-qubit local state (a ``StateVector`` on its GPU, or any object
with the same layer methods).

Qubits live at *positions*: position p < g is a global bit (bit g-1-p of the
rank), position p >= g is local qubit p-g of the shard; a map ``pos[q]``
tracks where logical qubit q sits, so a SWAP is a relabelling.  Operations:

* U(2) layer: gates on local qubits run on the shard; if the layer touches
  global qubits, one exchange swaps all g global positions with the top g
  local positions (an all-to-all of equal slabs: slab k of rank r goes to
  rank k and lands at slab r) and the rest of the layer runs locally.
* diagonal terms: no data moves; each rank substitutes its own values of the
  global bits (a ZZ term on a global and a local qubit becomes a one-qubit
  diagonal on the local one, a term on global qubits only a scalar).
* GF(2) affine permutation: synthesised as CNOT / SWAP / X (Gauss-Jordan);
  runs of gates whose targets are local, or whose control and target are
  both global, compose into one map that is block lower triangular over
  (global, local) bits: one local permutation sweep (its constant depends on
  the rank) and one rank remap (a whole shard sent to one other rank).  A
  CNOT with a global target and a local control first takes an exchange.
* marginal probabilities: local marginals placed at their global bits, then
  one all-reduce (sum); sampling: the rank totals by all-gather, shots split
  over ranks multinomially with the caller's seed, each rank samples its
  share from its shard, and the shots are gathered (all-gather) and put in a
  seeded random order.

Collectives go through ``torch.distributed`` (NCCL between GPUs, gloo on
CPUs); data moves between whole shards in local memory (no peer pointer is
handed to any kernel, no multicast).
"""
from __future__ import annotations

import cmath
import contextlib
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .fusion import DIAG_1Q, DIAG_2Q, DIAG_CPHASE, DIAG_CRZ, DIAG_GLOBAL, DIAG_PHASE, DIAG_RZ, DIAG_ZZ
from .workloads import affine_gates


def _entries(kind: int, params: Sequence[float]) -> List[complex]:
    """Diagonal entries of a term: 2 for one-wire kinds, 4 for two-wire
    kinds (first wire = most significant)."""
    p = list(params) + [0.0] * 8
    t = float(p[0])
    if kind == DIAG_ZZ:
        a, b = cmath.exp(-1j * t), cmath.exp(1j * t)
        return [a, b, b, a]
    if kind == DIAG_CPHASE:
        return [1, 1, 1, cmath.exp(1j * t)]
    if kind == DIAG_CRZ:
        return [1, 1, cmath.exp(-0.5j * t), cmath.exp(0.5j * t)]
    if kind == DIAG_2Q:
        return [complex(p[2 * i], p[2 * i + 1]) for i in range(4)]
    if kind == DIAG_RZ:
        return [cmath.exp(-0.5j * t), cmath.exp(0.5j * t)]
    if kind == DIAG_PHASE:
        return [1, cmath.exp(1j * t)]
    if kind == DIAG_1Q:
        return [complex(p[0], p[1]), complex(p[2], p[3])]
    raise ValueError(f"unknown diagonal kind {kind}")


def _one(q: int, d0: complex, d1: complex) -> tuple:
    return (DIAG_1Q, q, -1, [d0.real, d0.imag, d1.real, d1.imag])


def _parity(x: int) -> int:
    return bin(x).count("1") & 1


def _gf2_inverse_rows(cols: List[int], m: int) -> List[int]:
    """Rows (bit masks) of the inverse of the m x m GF(2) matrix whose
    column j is cols[j]: Gauss-Jordan on the rows, the same row operations
    applied to the identity."""
    work = [0] * m
    for j, c in enumerate(cols):
        for i in range(m):
            if (c >> i) & 1:
                work[i] |= 1 << j
    inv = [1 << i for i in range(m)]
    for col in range(m):
        piv = next((r for r in range(col, m) if (work[r] >> col) & 1), None)
        if piv is None:
            raise ValueError("local permutation is not invertible")
        work[col], work[piv] = work[piv], work[col]
        inv[col], inv[piv] = inv[piv], inv[col]
        for r in range(m):
            if r != col and (work[r] >> col) & 1:
                work[r] ^= work[col]
                inv[r] ^= inv[col]
    return inv


class GpuShard:
    """The local part of a sharded state on one GPU: a ``StateVector`` on its
    own CUDA stream, viewed as a torch tensor (no copy) for the exchanges."""

    def __init__(self, n_local: int, dtype: str = "complex64", device: int = 0):
        import torch
        from .engine import StateVector
        self.device = int(device)
        self.stream = torch.cuda.Stream(device=self.device)
        self.sv = StateVector(n_local, dtype, device=self.device, stream=self.stream.cuda_stream)
        self.n = n_local
        self.dtype = np.dtype(dtype)
        self._scratch = None

    # layer calls go straight to the engine
    def apply_u2_layer(self, mats, active):
        self.sv.apply_u2_layer(mats, active)

    def apply_diag_terms(self, terms):
        self.sv.apply_diag_terms(terms)

    def apply_xor_affine(self, rows, c):
        self.sv.apply_xor_affine(rows, c)

    def probabilities(self, wires):
        return self.sv.probabilities(wires, dtype=np.float64)

    def sample_indices(self, shots, seed):
        return self.sv.sample_indices(shots, seed=seed)

    def reset(self, first: bool):
        self.sv.reset()
        if not first:
            self.sv.scale(0.0)

    def get(self):
        return self.sv.get()

    def set(self, vec):
        self.sv.set(vec)

    def context(self):
        import torch
        return torch.cuda.stream(self.stream)

    def view(self):
        """The current amplitude buffer as a torch tensor (it changes after
        out-of-place kernels, so it is looked up at every exchange)."""
        import torch

        class _A:
            pass
        a = _A()
        a.__cuda_array_interface__ = {"shape": (1 << self.n,), "typestr": "<c8" if self.dtype == np.complex64 else "<c16",
                                      "data": (self.sv.device_ptr(), False), "strides": None, "version": 3}
        return torch.as_tensor(a, device=f"cuda:{self.device}")

    def scratch(self):
        import torch
        if self._scratch is None:
            self._scratch = torch.empty(1 << self.n, dtype=torch.complex64 if self.dtype == np.complex64
                                        else torch.complex128, device=f"cuda:{self.device}")
        return self._scratch

    def collective_device(self) -> str:
        return f"cuda:{self.device}"

    def close(self):
        self.sv.close()
        self._scratch = None


class ShardedState:
    """An n-qubit state over the ranks of ``dist`` (a power of two of them),
    this rank's part held by ``shard`` (n - g local qubits, g = log2 ranks).
    Every rank makes the same calls in the same order."""

    def __init__(self, n: int, shard, dist=None, group=None):
        self.dist = dist
        self.group = group
        self.P = dist.get_world_size(group) if dist is not None else 1
        self.rank = dist.get_rank(group) if dist is not None else 0
        g = int(round(math.log2(self.P)))
        if (1 << g) != self.P:
            raise ValueError("the number of ranks must be a power of two")
        self.n, self.g, self.nl = int(n), g, int(n) - g
        if shard.n != self.nl:
            raise ValueError(f"the shard must hold {self.nl} qubits")
        if self.nl < max(1, g):
            raise ValueError("each rank must hold at least as many qubits as there are global ones")
        self.shard = shard
        self.pos = list(range(self.n))
        self.exchanges = 0       # all-to-all swaps of the global and top local positions
        self.remaps = 0          # whole-shard moves between ranks
        self.bytes_sent = 0      # bytes this rank sent over the interconnect

    # ------------------------------------------------------------ state
    def reset(self) -> None:
        """|0...0>: rank 0 holds the 1, the others zeros; the qubit map is the
        identity again."""
        self.pos = list(range(self.n))
        self.shard.reset(self.rank == 0)

    def _ctx(self):
        ctx = getattr(self.shard, "context", None)
        return ctx() if ctx is not None else contextlib.nullcontext()

    def _bit(self, p: int) -> int:
        """This rank's value of the global bit at position p < g."""
        return (self.rank >> (self.g - 1 - p)) & 1

    # ------------------------------------------------------------ exchange
    def exchange(self) -> None:
        """Swap the g global positions with local positions g .. 2g-1: with
        the local index as (slab k = its top g bits, rest), slab k of rank r
        goes to rank k and lands at slab r of it (one all-to-all of 2^g equal
        slabs)."""
        if self.P == 1:
            return
        with self._ctx():
            t = self.shard.view()
            recv = self.shard.scratch()
            self.dist.all_to_all_single(recv, t, group=self.group)
            t.copy_(recv)
        self.exchanges += 1
        self.bytes_sent += t.numel() * t.element_size() * (self.P - 1) // self.P
        g = self.g
        for q in range(self.n):
            p = self.pos[q]
            if p < g:
                self.pos[q] = p + g
            elif p < 2 * g:
                self.pos[q] = p - g

    def _remap_ranks(self, dest: List[int]) -> None:
        """Rank r's shard moves whole to rank dest[r] (a permutation): one
        all-to-all in which every rank sends everything to one rank (itself
        when it keeps its shard), so all ranks take part in the same
        collective."""
        me = self.rank
        src = dest.index(me)
        with self._ctx():
            t = self.shard.view()
            recv = self.shard.scratch()
            size = t.numel()
            send_splits = [size if r == dest[me] else 0 for r in range(self.P)]
            recv_splits = [size if r == src else 0 for r in range(self.P)]
            self.dist.all_to_all_single(recv, t, output_split_sizes=recv_splits, input_split_sizes=send_splits,
                                        group=self.group)
            t.copy_(recv)
        if dest[me] != me:
            self.bytes_sent += t.numel() * t.element_size()

    # ------------------------------------------------------------ layers
    def _local_u2(self, mats: np.ndarray, qubits: List[int]) -> None:
        if not qubits:
            return
        m = np.tile(np.eye(2, dtype=np.complex128).reshape(1, 4), (self.nl, 1))
        act = []
        for q in qubits:
            lq = self.pos[q] - self.g
            m[lq] = mats[q]
            act.append(lq)
        self.shard.apply_u2_layer(m, sorted(act))

    def apply_u2_layer(self, mats, active: Optional[Sequence[int]] = None) -> None:
        """A 2x2 on each active logical qubit (all when None)."""
        mats = np.asarray(mats, dtype=np.complex128).reshape(self.n, 4)
        act = list(range(self.n)) if active is None else [int(q) for q in active]
        self._local_u2(mats, [q for q in act if self.pos[q] >= self.g])
        rest = [q for q in act if self.pos[q] < self.g]
        if rest:
            # the top local positions hold qubits that are done (or idle)
            self.exchange()
            self._local_u2(mats, rest)

    def apply_diag_terms(self, terms: Sequence[tuple]) -> None:
        """Commuting diagonal terms (kind, wire_a, wire_b, params) on logical
        wires, with this rank's global bits substituted."""
        g = self.g
        out = []
        scalar = 1.0 + 0j
        for kind, a, b, p in terms:
            kind = int(kind)
            if kind == DIAG_GLOBAL:
                scalar *= cmath.exp(1j * float(list(p)[0]))
                continue
            d = _entries(kind, p)
            pa = self.pos[int(a)]
            if len(d) == 2:
                if pa < g:
                    scalar *= d[self._bit(pa)]
                else:
                    out.append((kind, pa - g, -1, list(p)))
                continue
            pb = self.pos[int(b)]
            if pa < g and pb < g:
                scalar *= d[2 * self._bit(pa) + self._bit(pb)]
            elif pa < g:
                va = self._bit(pa)
                out.append(_one(pb - g, d[2 * va], d[2 * va + 1]))
            elif pb < g:
                vb = self._bit(pb)
                out.append(_one(pa - g, d[vb], d[2 + vb]))
            else:
                out.append((kind, pa - g, pb - g, list(p)))
        if scalar != 1.0:
            out.append(_one(0, scalar, scalar))
        if out:
            self.shard.apply_diag_terms(out)

    def apply_zz_weighted(self, bonds, thetas) -> None:
        self.apply_diag_terms([(DIAG_ZZ, int(a), int(b), [float(t)]) for (a, b), t in zip(bonds, thetas)])

    def apply_xor_affine(self, rows: Sequence[int], c: int) -> None:
        """out[y] = in[src(y)], src qubit-k bit = parity(rows[k] & y) ^ bit_k(c)
        on logical qubits (xor_affine.py:22-32): Gauss-Jordan CNOT / SWAP / X
        synthesis, SWAPs as relabellings, the rest in block-lower-triangular
        runs (see the module docstring)."""
        pending: List[tuple] = []
        for op in affine_gates([int(r) for r in rows], int(c), self.n):
            name, w = op["name"], op["wires"]
            if name == "SWAP":
                a, b = w
                self.pos[a], self.pos[b] = self.pos[b], self.pos[a]
            elif name == "X":
                pending.append(("X", self.pos[w[0]]))
            else:  # CNOT
                cq, tq = w
                if self.pos[tq] < self.g and self.pos[cq] >= self.g:
                    self._flush_affine(pending)
                    pending = []
                    self.exchange()
                pending.append(("CNOT", self.pos[cq], self.pos[tq]))
        self._flush_affine(pending)

    def apply_qft(self, wires=None, inverse: bool = False) -> None:
        raise NotImplementedError(
            "QFT layers on a sharded state are not supported: their stages on global qubits need a global/local "
            "swap before the stage sweeps, which is not built")

    def apply_layer(self, mats=None, active=None, terms=(), rows=None, c: int = 0) -> None:
        """U(2) layer, then diagonal terms, then permutation (the order of
        ``StateVector.apply_layer``)."""
        if mats is not None:
            self.apply_u2_layer(mats, active)
        if terms:
            self.apply_diag_terms(terms)
        if rows is not None:
            self.apply_xor_affine(rows, c)

    def _flush_affine(self, pending: List[tuple]) -> None:
        """Apply pending X / CNOT gates (physical positions) whose composition
        keeps global output bits functions of global input bits: a local
        permutation x -> M x ^ k_r on every rank, then the rank remap."""
        if not pending:
            return
        n, g, nl = self.n, self.g, self.nl

        def fwd(i: int) -> int:
            for op in pending:
                if op[0] == "X":
                    i ^= 1 << (n - 1 - op[1])
                elif (i >> (n - 1 - op[1])) & 1:
                    i ^= 1 << (n - 1 - op[2])
            return i

        d = fwd(0)
        cols = [fwd(1 << b) ^ d for b in range(n)]
        lmask = (1 << nl) - 1
        if any(cols[b] >> nl for b in range(nl)):
            raise AssertionError("a pending run moves local bits into global ones")
        dest = [fwd(r << nl) >> nl for r in range(self.P)]
        k = fwd(self.rank << nl) & lmask
        mcols = [cols[b] & lmask for b in range(nl)]
        if k or any(mcols[b] != 1 << b for b in range(nl)):
            inv = _gf2_inverse_rows(mcols, nl)
            cpack = 0
            for b in range(nl):
                if _parity(inv[b] & k):
                    cpack |= 1 << b
            self.shard.apply_xor_affine([inv[nl - 1 - q] for q in range(nl)], cpack)
        if any(dest[r] != r for r in range(self.P)):
            self._remap_ranks(dest)
            self.remaps += 1

    # ------------------------------------------------------------ measurement
    def _coll_device(self) -> str:
        f = getattr(self.shard, "collective_device", None)
        return f() if f is not None else "cpu"

    def _allreduce_f64(self, a: np.ndarray) -> np.ndarray:
        if self.P == 1:
            return a
        import torch
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self._coll_device())
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def _allgather(self, a: np.ndarray, counts: Optional[Sequence[int]] = None) -> List[np.ndarray]:
        """Every rank's array (counts[r] entries from rank r; equal sizes when
        counts is None)."""
        if self.P == 1:
            return [a]
        import torch
        size = len(a) if counts is None else max(int(c) for c in counts)
        buf = np.zeros(max(size, 1), dtype=a.dtype)
        buf[:len(a)] = a
        t = torch.from_numpy(buf)
        if t.is_complex():
            t = torch.view_as_real(t)
        t = t.contiguous().to(self._coll_device())
        parts = [torch.empty_like(t) for _ in range(self.P)]
        self.dist.all_gather(parts, t, group=self.group)
        out = []
        for r, p in enumerate(parts):
            p = p.cpu()
            if np.iscomplexobj(a):
                p = torch.view_as_complex(p)
            arr = p.numpy()
            out.append(arr[: (len(a) if counts is None else int(counts[r]))])
        return out

    def _logical(self, phys: np.ndarray) -> np.ndarray:
        """Logical basis indices of physical indices (the qubit map)."""
        phys = np.asarray(phys, dtype=np.int64)
        out = np.zeros_like(phys)
        n = self.n
        for q in range(n):
            out |= ((phys >> (n - 1 - self.pos[q])) & 1) << (n - 1 - q)
        return out

    def probabilities(self, wires: Optional[Sequence[int]] = None) -> np.ndarray:
        """Marginal probabilities of logical ``wires`` (first = most
        significant; None = all, for states small enough to gather), the
        same on every rank: local marginals at their global bits, then one
        all-reduce."""
        W = list(range(self.n)) if wires is None else [int(w) for w in wires]
        k = len(W)
        if k > 28:
            raise ValueError("marginals over more than 28 wires are not gathered")
        g = self.g
        locw = [(i, q) for i, q in enumerate(W) if self.pos[q] >= g]
        base = 0
        for i, q in enumerate(W):
            if self.pos[q] < g:
                base |= self._bit(self.pos[q]) << (k - 1 - i)
        lm = np.asarray(self.shard.probabilities([self.pos[q] - g for _, q in locw]), dtype=np.float64)
        j = np.arange(lm.size, dtype=np.int64)
        idx = np.full(lm.size, base, dtype=np.int64)
        L = len(locw)
        for t, (i, _) in enumerate(locw):
            idx |= ((j >> (L - 1 - t)) & 1) << (k - 1 - i)
        out = np.zeros(1 << k, dtype=np.float64)
        out[idx] = lm
        return self._allreduce_f64(out)

    def sample_indices(self, shots: int, seed: int = 0) -> np.ndarray:
        """``shots`` logical basis indices, the same array on every rank: the
        ranks' probability totals (all-gather) split the shots multinomially
        (generator seeded with ``seed``), each rank samples its share from
        its shard (seed, rank), and the gathered shots are put in a seeded
        random order."""
        shots = int(shots)
        tot = np.array([float(np.asarray(self.shard.probabilities([]))[0])])
        totals = np.concatenate(self._allgather(tot))
        if not totals.sum() > 0.0:
            raise RuntimeError("Simulator returned a zero-probability state")
        rng = np.random.default_rng(int(seed))
        counts = rng.multinomial(shots, totals / totals.sum())
        mine = np.asarray(self.shard.sample_indices(int(counts[self.rank]),
                                                    (int(seed) * 1000003 + self.rank) & 0x7FFFFFFFFFFFFFFF),
                          dtype=np.int64)
        logical = self._logical((np.int64(self.rank) << self.nl) | mine)
        allv = np.concatenate(self._allgather(logical, counts))
        return allv[rng.permutation(shots)]

    def get(self) -> np.ndarray:
        """The whole state in logical order, on every rank (gathers every
        shard: for states that fit one host)."""
        parts = self._allgather(np.asarray(self.shard.get()))
        phys = np.concatenate(parts)
        out = np.empty_like(phys)
        out[self._logical(np.arange(phys.size, dtype=np.int64))] = phys
        return out
