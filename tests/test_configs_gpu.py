"""The workload configurations as parity cases, through the public API.

* Plain statevector, 20 qubits, complex64, seed 0: 20 layers of [Haar U(2)
  on every qubit, RZZ(i, i+1) with angles U[0, 2pi), CNOT ladder], the full
  probability vector and 1000 seeded shots.  The CPU oracle (the reference's
  per-gate algorithm, complex128) runs it in full: amplitudes within 1e-5,
  probabilities within 1e-6, shots bit-exact with the oracle's stream on the
  device's own probabilities.
* Plain statevector at scale, 30 qubits: too large for the oracle, so a
  size-independent property checks it: the complex64 state against the same
  circuit run in complex128 on the GPU (infidelity <= 1e-9) and its norm.
  At 31 qubits (the largest register) the 13-bit and 12-bit tile plans
  against each other the same way.
* Its random GF(2) layer at 28 qubits, bit-exact against the oracle's source
  map evaluated on the GPU; its fused config layer at 28 qubits against the
  same layer as separate passes on other kernels; its QFT at 28 qubits on
  basis states against the closed form.
* Batching at full size (4096 circuits in one graph) against the per-circuit
  path on 48 circuits and the oracle on the smallest.
* Differentiation at full size (24 qubits, 384 parameters): complex64 vs
  complex128 adjoint gradients, and the parameter-shift rule and central
  differences on a spread of parameters.
"""
import numpy as np
import pytest

from oracle import OracleSim
from oracle import sampler as osamp

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _release_torch_cache():
    """The full-size checks build references with torch on the device; hand
    its cached blocks back after each test, so that later tests (which
    allocate through libmq) find the memory free."""
    yield
    import torch
    if torch.cuda.is_initialized():
        torch.cuda.synchronize()
        torch.cuda.empty_cache()


def test_plain_config_20_qubits_against_the_oracle():
    from mettleq_b200 import workloads as W
    from mettleq_b200.device import Device
    from mettleq_b200.integrations import _common as C
    n = 20
    circ = W.plain_circuit(n, 20, seed=0)
    ops, gphase = circ.ops()
    dev = Device(n)
    dev.execute(ops)
    C.apply_global_phase(dev, gphase)
    got = dev.statevector()
    o = OracleSim(n, np.complex128)
    o.execute(ops)
    o.apply_global_phase(gphase)
    assert float(np.max(np.abs(got.astype(np.complex128) - o.state))) <= 1e-5
    probs = dev.sim.probabilities()
    assert float(np.max(np.abs(probs - np.abs(o.state) ** 2))) <= 1e-6
    idx = dev.sim.sample_indices(1000, seed=0)
    assert np.array_equal(idx, osamp.sample_indices(osamp.amp2(got), 0, 1000))
    dev.close()


def _device_infidelity(sv64, sv128, b_typestr="<c16"):
    """(1 - |<a|b>|^2 / (<a|a><b|b>), <a|a>) of two device states (a complex64,
    b of b_typestr), summed on the GPU in complex128 (the 30-qubit states stay
    in device memory)."""
    import torch

    class _Dev:
        def __init__(self, ptr, n, typestr):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                             "strides": None, "version": 3}

    n = 1 << sv64.n
    sv64.synchronize()
    sv128.synchronize()
    a = torch.as_tensor(_Dev(sv64.device_ptr(), n, "<c8"), device="cuda:0")
    b = torch.as_tensor(_Dev(sv128.device_ptr(), n, b_typestr), device="cuda:0")
    ov = torch.zeros((), dtype=torch.complex128, device="cuda:0")
    na = torch.zeros((), dtype=torch.float64, device="cuda:0")
    nb = torch.zeros((), dtype=torch.float64, device="cuda:0")
    for s in range(0, n, 1 << 26):
        x = a[s:s + (1 << 26)].to(torch.complex128)
        y = b[s:s + (1 << 26)].to(torch.complex128)
        ov += torch.vdot(x, y)
        na += torch.vdot(x, x).real
        nb += torch.vdot(y, y).real
    torch.cuda.synchronize()
    return 1.0 - (ov.abs() ** 2 / (na * nb)).item(), na.item()


def test_31_qubits_tile_plans_agree(monkeypatch):
    """The largest register: at 31 qubits the 13-bit tile plan runs a fused
    layer as three sweeps whose low sweep is a 13-bit tile of 13 targets, and
    a QFT as three sweeps; the 12-bit plan (MQ_TILE_MAX=12) runs four.  Both
    give the same state of 3 config layers, a QFT and a GF(2) layer to within
    complex64 rounding (infidelity on the GPU in complex128, norm 1)."""
    from mettleq_b200 import workloads as W
    from mettleq_b200.engine import StateVector
    n = 31
    circ = W.scale_circuit(n, 3, seed=0, qft_every=3)
    monkeypatch.delenv("MQ_TILE_MAX", raising=False)
    sv13 = StateVector(n, "complex64")
    W.run_circuit_layers(sv13, circ)
    sweeps13 = sv13.counters()[1]
    monkeypatch.setenv("MQ_TILE_MAX", "12")
    sv12 = StateVector(n, "complex64")
    W.run_circuit_layers(sv12, circ)
    sweeps12 = sv12.counters()[1]
    monkeypatch.delenv("MQ_TILE_MAX", raising=False)
    try:
        infid, norm = _device_infidelity(sv13, sv12, "<c8")
    finally:
        sv12.close()
        sv13.close()
    assert sweeps13 < sweeps12
    assert abs(1.0 - norm) <= 1e-5
    assert infid <= 1e-9


def test_scale_config_30_qubits_against_complex128():
    from mettleq_b200 import workloads as W
    from mettleq_b200.engine import StateVector
    n = 30
    circ = W.scale_circuit(n, 6, seed=0, qft_every=3)  # 6 config layers, 2 QFT + 2 GF(2) layers
    sv64 = StateVector(n, "complex64")
    sv128 = StateVector(n, "complex128")
    W.run_circuit_layers(sv64, circ)
    W.run_circuit_layers(sv128, circ)
    infid, norm64 = _device_infidelity(sv64, sv128)
    sv64.close()
    sv128.close()
    assert abs(1.0 - norm64) <= 1e-5
    assert infid <= 1e-9


def test_random_gf2_layer_28_qubits_bit_exact():
    """A random invertible GF(2) layer at 28 qubits (2^18 cosets: every byte
    table of the coset offsets in use) against an independent gather: the
    oracle's source map src[y] = sum_k parity(rows[k] & y) << (n-1-k) ^ c
    (oracle.affine_sources) evaluated on the GPU with torch, bit-exact."""
    import torch
    from mettleq_b200.engine import StateVector
    from tests.helpers import random_invertible_rows
    n = 28
    rng = np.random.default_rng(2028)
    rows = random_invertible_rows(n, rng)
    c = int(rng.integers(0, 1 << n))
    dev = torch.device("cuda:0")
    gen = torch.Generator(device=dev).manual_seed(5)
    vec = torch.complex(torch.randn(1 << n, generator=gen, device=dev),
                        torch.randn(1 << n, generator=gen, device=dev)).to(torch.complex64)
    sv = StateVector(n, "complex64")
    sv.set(vec.cpu().numpy())
    sv.apply_xor_affine(rows, c)
    got = torch.from_numpy(sv.get()).to(dev)
    sv.close()
    y = torch.arange(1 << n, dtype=torch.int64, device=dev)
    src = torch.zeros_like(y)
    for k, r in enumerate(rows):
        par = y & r
        for sh in (16, 8, 4, 2, 1):
            par = par ^ (par >> sh)
        src |= (par & 1) << (n - 1 - k)
    src ^= c
    assert torch.equal(got, vec[src])


def test_fused_layer_28_qubits_against_separate_layers():
    """One config layer at 28 qubits through the fused path (Euler split: RY
    sweeps in tangent form, register diagonals, the CNOT ladder on the low
    sweep's write-back) against the same layer as three separate passes on
    other kernels (complex U(2) sweeps, the diagonal pass, the GF(2) layer):
    amplitudes within 1e-5."""
    import math
    import torch
    from mettleq_b200 import fusion as F
    from mettleq_b200 import workloads as W
    from mettleq_b200.engine import StateVector
    from tests.helpers import haar_u2
    n = 28
    rng = np.random.default_rng(28)
    mats = np.stack([haar_u2(rng).reshape(4) for _ in range(n)])
    terms = [(F.DIAG_ZZ, i, i + 1, [float(rng.uniform(0, math.pi))]) for i in range(n - 1)]
    rows, c = W.cnot_ladder_rows(n)
    dev = torch.device("cuda:0")
    gen = torch.Generator(device=dev).manual_seed(28)
    vec = torch.complex(torch.randn(1 << n, generator=gen, device=dev),
                        torch.randn(1 << n, generator=gen, device=dev)).to(torch.complex64)
    vec = (vec / torch.linalg.vector_norm(vec)).cpu().numpy()
    fused = StateVector(n, "complex64")
    fused.set(vec)
    fused.apply_layer(mats, None, terms, rows, c)
    a = fused.get()
    fused.close()
    sep = StateVector(n, "complex64")
    sep.set(vec)
    sep.apply_u2_layer(mats)
    sep.apply_diag_terms(terms)
    sep.apply_xor_affine(rows, c)
    b = sep.get()
    sep.close()
    assert float(np.max(np.abs(a - b))) <= 1e-5


def _bit_reverse(k, n):
    r = k & 0
    for i in range(n):
        r = r | (((k >> i) & 1) << (n - 1 - i))
    return r


def test_qft_28_qubits_on_basis_states_closed_form():
    """The 28-qubit QFT (no final swaps) of a basis state |x> against its
    closed form out[k] = e^{2 pi i x rev(k) / 2^n} / 2^{n/2} (rev: n-bit
    reversal), evaluated on the GPU in float64 from exact integer phases.
    The closed form is first checked against the oracle's gate-by-gate QFT at
    6 qubits.  Amplitudes within 2e-5 of their magnitude 2^{-n/2}."""
    import torch
    from mettleq_b200.engine import StateVector
    m = 6
    for x in (0, 1, 13, 63):
        v = np.zeros(1 << m, np.complex128)
        v[x] = 1.0
        o = OracleSim(m, np.complex128)
        o.set_state(v)
        o.qft()
        k = np.arange(1 << m)
        ref = np.exp(2j * np.pi * x * _bit_reverse(k, m) / (1 << m)) / np.sqrt(1 << m)
        assert float(np.max(np.abs(o.state - ref))) <= 1e-12
    n = 28
    dev = torch.device("cuda:0")
    sv = StateVector(n, "complex64")
    for x in (0x9E3779B & ((1 << n) - 1), (1 << n) - 1):
        v = np.zeros(1 << n, np.complex64)
        v[x] = 1.0
        sv.set(v)
        sv.apply_qft()
        got = torch.from_numpy(sv.get()).to(dev)
        k = torch.arange(1 << n, dtype=torch.int64, device=dev)
        ph = (x * _bit_reverse(k, n)) % (1 << n)  # exact: x, rev(k) < 2^28
        ang = ph.to(torch.float64) * (2.0 * np.pi / (1 << n))
        ref = torch.polar(torch.full_like(ang, 2.0 ** (-n / 2)), ang)
        err = (got.to(torch.complex128) - ref).abs().max().item()
        assert err <= 2e-5 * 2.0 ** (-n / 2), err
    sv.close()


def test_adjoint_config_24_qubits_384_parameters():
    """The differentiation configuration at full size: 24 qubits, 8 layers of
    RY+RZ on every qubit + CNOT ladder (384 parameters, U[-pi, pi]),
    H = sum Z_i Z_{i+1} + 0.5 sum X_i.  The complex64 adjoint gradient within
    5e-5 of the complex128 one; the complex128 gradient against the parameter-
    shift rule (1e-9) and central differences with h = 1e-4 (1e-7) on 12
    parameters spread over the layers, all energies from the complex128
    engine on the GPU."""
    import math
    from mettleq_b200.adjoint import AdjointEngine, LayeredAnsatz, PauliSum
    n = 24
    A = LayeredAnsatz(n, 8)
    H = PauliSum.ising_chain(n)
    p = np.random.default_rng(0).uniform(-math.pi, math.pi, A.shape)
    assert p.size == 384
    e64 = AdjointEngine(A, H, dtype="complex64")
    e128 = AdjointEngine(A, H, dtype="complex128")
    try:
        _, g64 = e64.energy_and_grad(p)
        _, g128 = e128.energy_and_grad(p)
        assert float(np.max(np.abs(g64 - g128))) <= 5e-5
        flat = p.reshape(-1)
        for i in np.linspace(0, p.size - 1, 12).astype(int):
            def energy_at(delta):
                q = flat.copy()
                q[i] += delta
                return e128.energy(q.reshape(A.shape))
            shift = 0.5 * (energy_at(math.pi / 2) - energy_at(-math.pi / 2))
            central = (energy_at(1e-4) - energy_at(-1e-4)) / 2e-4
            assert abs(g128.reshape(-1)[i] - shift) <= 1e-9, i
            assert abs(g128.reshape(-1)[i] - central) <= 1e-7, i
    finally:
        e64.close()
        e128.close()


def test_batch_config_4096_circuits():
    """The batching configuration at full size: 4096 hardware-efficient
    circuits (n ~ U{10..24}, depth ~ U{4..16}) in one captured graph.  Every
    circuit's <Z_0> and probabilities are produced; 48 circuits spread over
    the batch (small ones from the shared-memory kernel and large ones from
    the fused-layer lanes) are checked against the per-circuit Device path
    (probabilities within 2e-6, <Z_0> within 1e-5), and the four smallest
    against the oracle."""
    from mettleq_b200.batch import CircuitBatch, hea_batch, hea_mats, hea_ops
    from mettleq_b200.device import Device
    ns, ds, ps = hea_batch(4096, seed=0)
    b = CircuitBatch(ns, ds, lanes=16, small_threads=256)
    try:
        b.run([hea_mats(p) for p in ps])
        z0 = b.z0()
        assert z0.shape == (4096,) and np.all(np.abs(z0) <= 1.0 + 1e-6)
        order = np.argsort(np.asarray(ns), kind="stable")
        picks = sorted(set(order[np.linspace(0, 4095, 48).astype(int)].tolist()))
        for c in picks:
            dev = Device(ns[c])
            dev.execute(hea_ops(ps[c], True))
            plain = dev.sim.probabilities(dtype=np.float64)
            dev.close()
            got = b.probabilities(c)
            assert np.max(np.abs(got - plain)) < 2e-6, (c, ns[c])
            half = len(plain) // 2
            assert abs(z0[c] - (plain[:half].sum() - plain[half:].sum())) < 1e-5, (c, ns[c])
        for c in order[:4].tolist():
            o = OracleSim(ns[c], np.complex128)
            o.execute(hea_ops(ps[c], True))
            assert np.max(np.abs(b.probabilities(c) - np.abs(o.state) ** 2)) < 2e-6, (c, ns[c])
    finally:
        b.close()
