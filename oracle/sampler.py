"""Seeded sampling stream and deterministic reductions (CPU restatement).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference samples with ``mx.random.categorical`` keyed by one uint32 drawn
from ``np.random.default_rng(seed)`` (sim.py:383-419).  MLX's generator cannot
run outside MLX, so counts are pinned to the project's own stream instead, and
this module restates it bit for bit so the CUDA sampler can be compared
exactly:

* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11; Random123), key = the 64-bit
  seed, counter = (shot + stream_offset) as a 64-bit integer in words 0-1.
  u = (((x1 << 32) | x0) >> 11) * 2^-53, a double in [0, 1).
* p_i = re_i^2 + im_i^2 evaluated in float64 (exact products for complex64).
* Block sums over blocks of BS = min(1024, M) entries: 32 lanes each add
  entries lane, lane+32, ... sequentially, then lanes combine by an XOR
  butterfly (offsets 16, 8, 4, 2, 1); the block sum is lane 0's value.
* Exclusive block offsets, two-level: within a super-block of 1024 blocks a
  sequential running sum; the super-block totals summed sequentially; offset
  C_b = E_superblock + L_b.
* Shot: t = u * total; b = largest block with C_b <= t, clamped to the last
  block with a positive sum; then a sequential running sum r = C_b + p_i
  inside the block returns the first i with r > t, or the block's last
  positive entry when rounding leaves r <= t.
* Marginals over k < n wires: bucket index has the first requested wire as
  its MSB (sim.py:322-343); each bucket's 2^(n-k) entries (remaining index
  bits in ascending order) are reduced with the same block sum, and the block
  sums are added sequentially in two levels (1024 per super-chunk).
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
_MASK32 = np.uint64(0xFFFFFFFF)

BLOCK = 1024
LANES = 32
SUPER = 1024


def philox4x32_10(ctr: np.ndarray, key: np.ndarray) -> np.ndarray:
    """Philox4x32-10 on arrays: ctr (..., 4) uint32, key (..., 2) uint32."""
    c = [np.asarray(ctr[..., i], dtype=np.uint64) for i in range(4)]
    k0 = np.asarray(key[..., 0], dtype=np.uint32).copy()
    k1 = np.asarray(key[..., 1], dtype=np.uint32).copy()
    for r in range(10):
        if r:
            k0 = (k0 + W0).astype(np.uint32)
            k1 = (k1 + W1).astype(np.uint32)
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK32
        c = [hi1 ^ c[1] ^ k0.astype(np.uint64), lo1, hi0 ^ c[3] ^ k1.astype(np.uint64), lo0]
    return np.stack([x.astype(np.uint32) for x in c], axis=-1)


def uniforms(seed: int, shots: int, stream_offset: int = 0) -> np.ndarray:
    """Doubles in [0, 1), one per shot, from the Philox stream."""
    s = np.arange(shots, dtype=np.uint64) + np.uint64(stream_offset)
    ctr = np.zeros((shots, 4), dtype=np.uint32)
    ctr[:, 0] = (s & _MASK32).astype(np.uint32)
    ctr[:, 1] = (s >> np.uint64(32)).astype(np.uint32)
    key = np.empty((shots, 2), dtype=np.uint32)
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    key[:, 0] = seed & 0xFFFFFFFF
    key[:, 1] = seed >> 32
    x = philox4x32_10(ctr, key).astype(np.uint64)
    bits = ((x[:, 1] << np.uint64(32)) | x[:, 0]) >> np.uint64(11)
    return bits.astype(np.float64) * (2.0 ** -53)


def amp2(state: np.ndarray) -> np.ndarray:
    """p_i = re^2 + im^2 in float64 (no fused multiply-add)."""
    re = state.real.astype(np.float64)
    im = state.imag.astype(np.float64)
    return re * re + im * im


def block_sums(p: np.ndarray) -> np.ndarray:
    """Per-block deterministic sums (lane-strided, then XOR butterfly)."""
    m = p.size
    bs = min(BLOCK, m)
    nb = m // bs
    per_lane = -(-bs // LANES)
    padded = np.zeros((nb, per_lane * LANES), dtype=np.float64)
    padded[:, :bs] = p.reshape(nb, bs)
    v = padded.reshape(nb, per_lane, LANES)
    acc = np.zeros((nb, LANES), dtype=np.float64)
    for j in range(per_lane):
        acc = acc + v[:, j, :]
    lane = np.arange(LANES)
    for off in (16, 8, 4, 2, 1):
        acc = acc + acc[:, lane ^ off]
    return acc[:, 0].copy()


def _two_level_exclusive(s: np.ndarray):
    """Exclusive offsets C, total, with the two-level sequential order."""
    nb = s.size
    ng = -(-nb // SUPER)
    local = np.zeros(nb, dtype=np.float64)
    totals = np.zeros(ng, dtype=np.float64)
    for g in range(ng):
        seg = s[g * SUPER:(g + 1) * SUPER]
        inc = np.cumsum(seg)  # sequential, starts with 0.0 + s0 = s0
        local[g * SUPER:g * SUPER + seg.size] = np.concatenate(([0.0], inc[:-1]))
        totals[g] = inc[-1]
    einc = np.cumsum(totals)
    e = np.concatenate(([0.0], einc[:-1]))
    offsets = e[np.arange(nb) // SUPER] + local
    return offsets, float(einc[-1])


def _two_level_sum(d: np.ndarray) -> float:
    ng = -(-d.size // SUPER)
    parts = np.array([np.cumsum(d[g * SUPER:(g + 1) * SUPER])[-1] for g in range(ng)])
    return float(np.cumsum(parts)[-1])


def marginal_probabilities(p: np.ndarray, n: int, wires: Optional[Sequence[int]]) -> np.ndarray:
    """Deterministic float64 marginal over ``wires`` (first wire = MSB)."""
    if wires is None or list(wires) == list(range(n)):
        return p.copy()
    sel = list(wires)
    k = len(sel)
    rest = [q for q in range(n) if q not in sel]
    # bucket-major order: selected wires (in request order) then the rest in
    # qubit order (= descending index bit, so ascending u runs over the
    # remaining index bits from the lowest)
    t = p.reshape([2] * n).transpose(sel + rest).reshape(1 << k, 1 << (n - k))
    out = np.empty(1 << k, dtype=np.float64)
    for b in range(1 << k):
        d = block_sums(t[b])
        out[b] = _two_level_sum(d)
    return out


def sample_indices(p: np.ndarray, seed: int, shots: int, stream_offset: int = 0) -> np.ndarray:
    """Inverse-CDF sampling of ``shots`` indices from unnormalised p."""
    m = p.size
    bs = min(BLOCK, m)
    s = block_sums(p)
    offs, total = _two_level_exclusive(s)
    if not total > 0.0:
        raise RuntimeError("Simulator returned a zero-probability state")
    positive = np.nonzero(s > 0.0)[0]
    last_block = int(positive[-1])
    u = uniforms(seed, shots, stream_offset)
    t = u * total
    out = np.empty(shots, dtype=np.int64)
    for j in range(shots):
        b = int(np.searchsorted(offs, t[j], side="right")) - 1
        b = min(max(b, 0), last_block)
        blk = p[b * bs:(b + 1) * bs]
        # sequential running sum r_i = (...((C_b + p_0) + p_1) ...) + p_i
        r = np.cumsum(np.concatenate(([offs[b]], blk)))[1:]
        hit = np.nonzero(r > t[j])[0]
        if hit.size:
            found = int(hit[0])
        else:
            found = int(np.nonzero(blk > 0.0)[0][-1])
        out[j] = b * bs + found
    return out
