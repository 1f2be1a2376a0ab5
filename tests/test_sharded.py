"""The sharded statevector (mettleq_b200/sharded.py) on CPU: 2 and 4 gloo
ranks, each holding its part of a 12-qubit state in a numpy shard (the
oracle), run the exchange schedule the GPU ranks run (all-to-all swaps of
global and local qubits, rank remaps, per-rank diagonals, all-reduced
marginals, gathered samples), checked against the oracle on the whole state.
One-GPU runs of the same class with the engine's shard are in the gpu test
at the end."""
import math
import os
import socket

import numpy as np
import pytest

from tests.helpers import haar_u2, oracle_apply_terms, random_invertible_rows

N_QUBITS = 12


class NumpyShard:
    """A local part held by the oracle (complex128), with the calls
    ShardedState makes of a shard."""

    def __init__(self, n):
        from oracle import OracleSim
        self.n = n
        self.sim = OracleSim(n, np.complex128)
        self._scratch = None

    def apply_u2_layer(self, mats, active):
        for q in active:
            self.sim.apply_single(np.asarray(mats[q]).reshape(2, 2), q)

    def apply_diag_terms(self, terms):
        oracle_apply_terms(self.sim, terms)

    def apply_xor_affine(self, rows, c):
        self.sim.apply_affine(rows, c)

    def probabilities(self, wires):
        return self.sim.probabilities(list(wires))

    def sample_indices(self, shots, seed):
        from oracle import sampler as S
        if shots == 0:
            return np.zeros(0, dtype=np.int64)
        return S.sample_indices(S.amp2(self.sim.state), seed, shots)

    def reset(self, first):
        self.sim.reset()
        if not first:
            self.sim.state[:] = 0

    def get(self):
        return self.sim.state.copy()

    def view(self):
        import torch
        return torch.from_numpy(self.sim.state)

    def scratch(self):
        import torch
        if self._scratch is None:
            self._scratch = torch.empty(1 << self.n, dtype=torch.complex128)
        return self._scratch


def _program(n, seed):
    """Layers touching global and local qubits: U(2) on all or some qubits,
    diagonal terms of every kind on random wires, a CNOT ladder and a random
    GF(2) layer."""
    from mettleq_b200 import fusion as F
    from mettleq_b200.workloads import cnot_ladder_rows
    rng = np.random.default_rng(seed)
    prog = []
    for layer in range(4):
        mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
        active = None if layer % 2 == 0 else sorted(rng.choice(n, n // 2, replace=False).tolist())
        prog.append(("u2", mats, active))
        terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, 2 * math.pi))]) for i in range(n - 1)]
        for _ in range(6):
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            kind = int(rng.choice([F.DIAG_CPHASE, F.DIAG_CRZ, F.DIAG_ZZ]))
            terms.append((kind, a, b, [float(rng.uniform(-math.pi, math.pi))]))
        for q in rng.choice(n, 4, replace=False):
            kind = int(rng.choice([F.DIAG_RZ, F.DIAG_PHASE]))
            terms.append((kind, int(q), -1, [float(rng.uniform(-math.pi, math.pi))]))
        d = np.exp(1j * rng.uniform(0, 2 * math.pi, 4))
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        terms.append((F.DIAG_2Q, a, b, [v for z in d for v in (z.real, z.imag)]))
        terms.append((F.DIAG_GLOBAL, 0, -1, [0.37]))
        prog.append(("diag", terms))
        prog.append(("affine",) + tuple(cnot_ladder_rows(n)))
        if layer in (1, 3):
            prog.append(("affine", random_invertible_rows(n, rng), int(rng.integers(0, 1 << n))))
    return prog


def _run(target, prog):
    for step in prog:
        if step[0] == "u2":
            target.apply_u2_layer(step[1], step[2])
        elif step[0] == "diag":
            target.apply_diag_terms(step[1])
        else:
            target.apply_xor_affine(step[1], step[2])


class _OracleTarget:
    def __init__(self, n):
        from oracle import OracleSim
        self.o = OracleSim(n, np.complex128)
        self.n = n

    def apply_u2_layer(self, mats, active):
        for q in (range(self.n) if active is None else active):
            self.o.apply_single(mats[q].reshape(2, 2), q)

    def apply_diag_terms(self, terms):
        oracle_apply_terms(self.o, terms)

    def apply_xor_affine(self, rows, c):
        self.o.apply_affine(rows, c)


WIRES = ([0], [11, 0, 5], [1, 2, 3, 9], [])


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    from mettleq_b200.sharded import ShardedState
    torch.set_num_threads(1)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g = int(math.log2(world))
        st = ShardedState(N_QUBITS, NumpyShard(N_QUBITS - g), dist)
        st.reset()
        _run(st, _program(N_QUBITS, 9))
        state = st.get()
        probs = [st.probabilities(w) for w in WIRES]
        s1 = st.sample_indices(4000, seed=21)
        s2 = st.sample_indices(4000, seed=21)
        q.put((rank, state, probs, s1, s2, st.exchanges, st.remaps))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_state_over_gloo_ranks_matches_the_oracle(world):
    import torch.multiprocessing as mp
    from oracle import sampler as S
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got.sort(key=lambda x: x[0])
    ref = _OracleTarget(N_QUBITS)
    _run(ref, _program(N_QUBITS, 9))
    want = ref.o.state
    for rank, state, probs, s1, s2, exchanges, remaps in got:
        assert np.max(np.abs(state - want)) < 1e-12, rank
        for w, pr in zip(WIRES, probs):
            exp = ref.o.probabilities(w)
            assert np.max(np.abs(pr - exp)) < 1e-12, (rank, w)
        # the same shots on every rank, and again for the same seed
        assert np.array_equal(s1, got[0][3]) and np.array_equal(s1, s2)
        # the schedule moved data: U(2) layers on global qubits, the ladder
        assert exchanges >= 4 and remaps >= 1
    # the shots follow the state's distribution: chi-square over the top
    # three qubits (8 bins, 4000 shots; 26.1 is the 0.9995 quantile, 7 dof)
    s1 = got[0][3]
    p3 = S.marginal_probabilities(np.abs(want) ** 2, N_QUBITS, [0, 1, 2])
    obs = np.bincount(s1 >> (N_QUBITS - 3), minlength=8)
    expct = p3 / p3.sum() * len(s1)
    chi2 = float(np.sum((obs - expct) ** 2 / np.maximum(expct, 1e-12)))
    assert chi2 < 26.1, chi2


def test_sharded_rewrite_of_diagonal_terms_on_one_rank():
    """With one rank there are no global qubits: the state equals the
    oracle's after the same program (the single-process path)."""
    from mettleq_b200.sharded import ShardedState
    st = ShardedState(8, NumpyShard(8), None)
    st.reset()
    prog = _program(8, 4)
    _run(st, prog)
    ref = _OracleTarget(8)
    _run(ref, prog)
    assert np.max(np.abs(st.get() - ref.o.state)) < 1e-12
    assert st.exchanges == 0 and st.remaps == 0


@pytest.mark.gpu
def test_sharded_state_with_the_engine_shard_on_one_gpu():
    """The GPU shard adapter (engine StateVector behind the shard calls) on
    one rank, complex128, against the oracle."""
    from mettleq_b200.sharded import GpuShard, ShardedState
    shard = GpuShard(14, "complex128", device=0)
    try:
        st = ShardedState(14, shard, None)
        st.reset()
        prog = _program(14, 6)
        _run(st, prog)
        ref = _OracleTarget(14)
        _run(ref, prog)
        assert np.max(np.abs(st.get() - ref.o.state)) < 1e-12
        pr = st.probabilities([3, 0])
        assert np.max(np.abs(pr - ref.o.probabilities([3, 0]))) < 1e-12
        t = shard.view()
        assert t.numel() == 1 << 14 and str(t.device) == "cuda:0"
        # rank 0 of one: |0...0> after reset, a zero shard otherwise
        shard.reset(False)
        assert np.max(np.abs(shard.get())) == 0.0
    finally:
        shard.close()
