// Tile sweeps: the fused single-qubit layer (a), QFT stages (c) and
// controlled single-qubit gates.
//
// Replaces the reference's one-thread-per-2^r-amplitudes Metal passes
// (shaders/single_qubit.py:165-210 radix-16 and :422-615 drivers;
// shaders/qft.py:61-137 radix-4 / pair stages and :144-236 drivers;
// shaders/controlled_single.py:18-134).  One sweep here applies the gates of
// up to 12 index bits:
//
//   * a tile is 2^M amplitudes whose "tile bits" are the swept target bits
//     plus low passenger bits, so every global access is a run of >= 8
//     contiguous amplitudes;
//   * persistent CTAs stream tiles through two shared-memory buffers: while
//     tile t is processed, cp.async brings tile t+grid into the other buffer;
//   * the tile is processed in place in shared memory by "phases": each
//     thread loads 2^LR amplitudes that differ in LR tile bits into
//     registers, applies the gates of those bits, and writes them back;
//   * global memory moves in 16-byte chunks, loaded with cp.async and stored
//     with vector stores; shared memory holds the tile in a chunk-swizzled
//     layout (see k_tile) so register phases over the lowest bits stay free
//     of bank conflicts;
//   * the finished tile is written back with coalesced stores.
//
// QFT stages (sim.py:522-563, no final swaps): stage j on index bit s is a
// butterfly on bit s, then on the bit-s = 1 half the phase e^{+i pi L / 2^w}
// with L the integer value of the ladder bits below s (the closed form of
// qft.py:18-59); the inverse applies the conjugate phase first.  Stages run
// in the required order (high bit first forward, low bit first inverse); the
// 1/sqrt(2) of every butterfly is applied once per sweep as 2^{-stages/2}.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "mq_internal.cuh"

namespace mq {

enum : uint8_t { OP_U2 = 0, OP_QFT_FWD = 1, OP_QFT_INV = 2, OP_CU2 = 3 };

constexpr int kMaxPhases = 6;
// Tile buffers in shared memory: two (the next tile is prefetched while one
// is processed), or one for 13-bit tiles at 256 threads, where three CTAs per
// SM overlap one another's loads instead.
__host__ __device__ constexpr int tile_nbuf(int m, int lt) { return (m >= 13 && lt <= 8) ? 1 : 2; }
constexpr int kMaxOps = 16;
// Per register phase, the shared-memory and global offsets of a group's
// thread bits as two XOR tables each: thread bits 0-3 (16 entries) and 4-8
// (32 entries); words per phase: 2 x (16 + 32).
constexpr int kThreadTabWords = 96;
constexpr int kMaxTileBits = 13;

struct TileOp {
  uint8_t kind, phase, rk, lad_shift, width, pad[3];
  uint32_t cmask;  // OP_CU2: global index bits that must all be set
  int32_t qubit;   // OP_U2 with device-resident matrices: row of mats_dev
  double u[8];     // 2x2 matrix (re, im interleaved)
};

// One register phase: which tile bits sit in registers, the shared-memory
// (tile-local) and global offsets of every register / group bit, and for
// U(2) sweeps one matrix slot per register bit.
struct __align__(16) PhaseDesc {
  uint32_t s_reg[5];
  uint32_t s_grp[kMaxTileBits];
  uint32_t g_reg[5];
  uint32_t g_grp[kMaxTileBits];
  uint32_t cmask[5];     // controls of the slot's gate (0 = none)
  uint8_t active;        // slots carrying a gate
  uint8_t any_ctl;       // some slot is controlled
  uint8_t real;          // slots whose matrix is real (RY-type: 2 FMA per output component)
  // slots holding a rotation [[c, -s], [s, c]] as one tangent t in uf/ud[k][0]:
  // c (x0 - t x1, t x0 + x1) with t = s / c, or (rotB) s (t x0 - x1, x0 + t x1)
  // with t = c / s; the factor c or s is left to the caller (one FMA per
  // output component)
  uint8_t rot, rotB;
  alignas(16) float uf[5][8];   // rows read as two 16-byte vectors
  alignas(16) double ud[5][8];
};
static_assert(offsetof(PhaseDesc, uf) % 16 == 0, "matrix rows must be 16-byte aligned");
static_assert(sizeof(PhaseDesc) % 16 == 0, "PhaseDesc array stride must keep rows aligned");

// set when a sweep was abandoned (read and cleared by mq_sync)
__device__ unsigned int g_tile_fault;

struct TileParams {
  TmaDesc tma;
  uint32_t n_tiles;
  uint8_t n, m, n_phases, n_ops;
  uint8_t tile_bit[16];
  uint8_t need_tw, has_scale, hi_contig, hi_shift;
  uint32_t pad2;
  BaseRuns runs;  // tile index -> base index (deposit_runs)
  double scale;
  uint8_t ph_op[kMaxPhases + 2];     // QFT: ops of phase p are [ph_op[p], ph_op[p+1])
  uint8_t qchain[kMaxPhases];        // QFT: 1 + the largest width when the phase's stages chain (else 0)
  // QFT: ns (3 or 4) when a chained phase holds ns stages on register slots
  // 0 .. ns-1 in the order of their direction (top slot first forward, slot
  // 0 first inverse): its register factors are then compile-time constants
  // (apply_qft_chain); 0 otherwise
  uint8_t qfull[kMaxPhases];
  // U(2) matrices read from device memory at launch (mats_dev[8 q ..]):
  // slot k of phase p takes row mat_q[p][k] - 1 (0 = the matrix in ph)
  int16_t mat_q[kMaxPhases][5];
  const double* mats_dev;
  PhaseDesc ph[kMaxPhases];
  TileOp ops[kMaxOps];
};

// Epilogue of the fused layer's low sweep (tile = index bits [0, M)): after
// the U(2) phases, every amplitude x of the tile is multiplied by the
// diagonal phase(x) = prod_w lut[off[w] + ((x >> shift[w]) & (2^nbits[w]-1))]
// and, with a permutation out[y] = in[A y ^ c] whose matrix maps the low
// space span(e_0..e_{M-1}) onto itself, written to its output position.
// Windows [0, n_var) overlap the tile bits; [n_var, n_win) are constant
// over a tile and multiplied once per tile.
constexpr int kEpiWin = 8;
constexpr int kEpiLutBytes = 16384;
// Register-phase diagonals first try tables of at most this many entries
// (narrower windows, one more lookup per 16-amplitude group), which keeps
// the sweep at the occupancy of a plain one.
constexpr int kRegDiagSmall = 1024;
// A diagonal applied to a 4-bit register phase: windows [0, n_win) taken at
// the group base, times T[c][r] at lut[toff + 17c + r] (c = index bits
// cbit[0..nc); rows padded to 17 entries against bank conflicts).
struct RegDiag {
  uint8_t on, nc, cbit[3], n_win, pad[2];
  uint8_t shift[kEpiWin];
  uint8_t nbits[kEpiWin];
  uint16_t off[kEpiWin];
  uint16_t toff, pad1;
};
struct EpiDesc {
  RegDiag pre;  // applied in the first register phase, before its gates
  uint8_t diag, perm, n_win, n_var;
  // dreg: the diagonal is applied in the last register phase instead:
  // windows [0, n_win) at the group base times T[c][r] at lut[toff + 17c + r]
  // (c = index bits cbit[0..nc))
  uint8_t dreg, nc, cbit[3], pad0;
  uint16_t toff, pad1;
  uint8_t shift[kEpiWin];
  uint8_t nbits[kEpiWin];
  uint16_t off[kEpiWin];
  uint32_t n_entries;  // table entries (complex values of the state's type)
  uint32_t c;          // permutation flip constant
  uint32_t cols[32];   // permutation columns A e_j
  // A (t << M) for tile index t = XOR of htab[256 k + byte k of t], k < 3
  // (A is linear); read at a CTA-uniform index from the parameter space
  uint32_t htab[768];
  alignas(16) unsigned char lut[kEpiLutBytes];
};
struct FusedParams : TileParams {
  EpiDesc epi;
};
// QFT sweeps: per stage op, the phase factor of each register pattern r
// (e^{i pi Lr(r) / 2^width}, see apply_qft).
struct QftParams : TileParams {
  alignas(16) float2 twf[kMaxOps][32];
  alignas(16) double2 twd[kMaxOps][32];
};
static_assert(sizeof(QftParams) <= 32000, "kernel parameter block too large");
static_assert(sizeof(FusedParams) <= 32000, "kernel parameter block too large");

// Twiddle tables of the complex64 QFT sweeps: entry j of table w (j < 1024)
// is e^{i pi j 2^{-10(w+1)}}.  One copy per device in global memory (read
// through L1), uploaded by the first QFT sweep on the device; keeping them
// out of shared memory leaves the sweep at the occupancy of a U(2) sweep.
__device__ float2 g_qft_twiddles[3072];

// e^{i pi L / 2^width}, 1 <= width <= 31, L < 2^width.
template <typename R> struct Twiddle;
template <> struct Twiddle<float> {
  static __device__ __forceinline__ float2 get(const float2* tw, uint32_t L, int width) {
    const uint32_t F = L << (32 - width);
    float2 t = tw[F >> 22];
    t = cmul(t, tw[1024 + ((F >> 12) & 1023u)]);
    t = cmul(t, tw[2048 + ((F >> 2) & 1023u)]);
    return t;
  }
};
template <> struct Twiddle<double> {
  static __device__ __forceinline__ double2 get(const float2*, uint32_t L, int width) {
    double s, c;
    sincospi(ldexp((double)L, -width), &s, &c);
    return make_double2(c, s);
  }
};

template <int LR>
__device__ __forceinline__ uint32_t osel(int r, const uint32_t* g) {
  uint32_t o = 0;
#pragma unroll
  for (int k = 0; k < LR; ++k)
    if (r & (1 << k)) o ^= g[k];
  return o;
}

// out = u0 * x0 + u1 * x1 as explicit fused multiply-adds (4 per component).
template <typename T>
__device__ __forceinline__ T cmac2(T u0, T x0, T u1, T x1) {
  T r;
  r.x = fma(u0.x, x0.x, fma(-u0.y, x0.y, fma(u1.x, x1.x, -u1.y * x1.y)));
  r.y = fma(u0.x, x0.y, fma(u0.y, x0.x, fma(u1.x, x1.y, u1.y * x1.x)));
  return r;
}

// 2x2 gate on register bit K; CTL: only where all cmask bits are set.
// REAL: real matrices take the real path (else the complex one; the sweeps
// with register diagonals leave it out for registers).
template <typename R, int LR, int K, bool CTL, bool REAL>
__device__ __forceinline__ void apply_u2(V2<R> (&a)[1 << LR], const PhaseDesc& D, uint32_t gq, const uint32_t* greg) {
  using T = V2<R>;
  constexpr int NR = 1 << LR;
  T u00, u01, u10, u11;
  if constexpr (sizeof(R) == 4) {
    const float4 m0 = *reinterpret_cast<const float4*>(&D.uf[K][0]);
    const float4 m1 = *reinterpret_cast<const float4*>(&D.uf[K][4]);
    u00 = make_float2(m0.x, m0.y); u01 = make_float2(m0.z, m0.w);
    u10 = make_float2(m1.x, m1.y); u11 = make_float2(m1.z, m1.w);
  } else {
    u00 = mk<R>(D.ud[K][0], D.ud[K][1]); u01 = mk<R>(D.ud[K][2], D.ud[K][3]);
    u10 = mk<R>(D.ud[K][4], D.ud[K][5]); u11 = mk<R>(D.ud[K][6], D.ud[K][7]);
  }
  const uint32_t cm = D.cmask[K];
  if (!CTL && ((D.rot >> K) & 1u)) {
    const R t = u00.x;
    if ((D.rotB >> K) & 1u) {
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (r & (1 << K)) continue;
        const T x0 = a[r], x1 = a[r | (1 << K)];
        a[r] = caxmy(t, x0, x1);
        a[r | (1 << K)] = caxpy(t, x1, x0);
      }
    } else {
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (r & (1 << K)) continue;
        const T x0 = a[r], x1 = a[r | (1 << K)];
        a[r] = caxpy(-t, x1, x0);
        a[r | (1 << K)] = caxpy(t, x0, x1);
      }
    }
    return;
  }
  if (REAL && !CTL && ((D.real >> K) & 1u)) {
    // real matrix: each output component is two products
    const R c00 = u00.x, c01 = u01.x, c10 = u10.x, c11 = u11.x;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (r & (1 << K)) continue;
      const T x0 = a[r], x1 = a[r | (1 << K)];
      a[r] = caxpy(c00, x0, cscale(x1, c01));
      a[r | (1 << K)] = caxpy(c10, x0, cscale(x1, c11));
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    if (r & (1 << K)) continue;
    if (CTL && (((gq | osel<LR>(r, greg)) & cm) != cm)) continue;
    const T x0 = a[r], x1 = a[r | (1 << K)];
    a[r] = cmac2(u00, x0, u01, x1);
    a[r | (1 << K)] = cmac2(u10, x0, u11, x1);
  }
}

template <typename R, int LR, bool CTL, bool REAL>
__device__ __forceinline__ void apply_u2_phase(V2<R> (&a)[1 << LR], const PhaseDesc& D, uint32_t gq,
                                               const uint32_t* greg) {
  const uint32_t act = D.active;
  if (act & 1u) apply_u2<R, LR, 0, CTL, REAL>(a, D, gq, greg);
  if constexpr (LR > 1) if (act & 2u) apply_u2<R, LR, 1, CTL, REAL>(a, D, gq, greg);
  if constexpr (LR > 2) if (act & 4u) apply_u2<R, LR, 2, CTL, REAL>(a, D, gq, greg);
  if constexpr (LR > 3) if (act & 8u) apply_u2<R, LR, 3, CTL, REAL>(a, D, gq, greg);
  if constexpr (LR > 4) if (act & 16u) apply_u2<R, LR, 4, CTL, REAL>(a, D, gq, greg);
}

// One QFT stage on register bit K (forward: butterfly then phase; inverse:
// conjugate phase then butterfly).  The phase of the bit-1 half is
// e^{i pi L / 2^w} with L = Lg + Lr: Lg from the group's index bits (one
// Twiddle per group), Lr from the register bits, whose factor treg[r] the
// host tabulates per stage, so a pair costs one complex product for its
// phase.
template <typename R, int LR, int K, bool FWD>
__device__ __forceinline__ void apply_qft(V2<R> (&a)[1 << LR], const TileOp& op, V2<R> tg, const V2<R>* treg) {
  using T = V2<R>;
  constexpr int NR = 1 << LR;
  const int width = op.width;
  if (width == 0) {  // the first stage of a register: no ladder bits, no phase
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (r & (1 << K)) continue;
      const T x0 = a[r], x1 = a[r | (1 << K)];
      a[r] = cadd(x0, x1);
      a[r | (1 << K)] = csub(x0, x1);
    }
    return;
  }
  // a pair's register factor depends only on the register bits below K (the
  // bits above the stage's bit are not ladder bits): for K < 3 the 2^K
  // distinct products are formed once
  constexpr int NW = K < 3 ? (1 << K) : 1;
  T wk[NW];
  if constexpr (K < 3) {
#pragma unroll
    for (int j = 0; j < NW; ++j) wk[j] = cmul(tg, treg[j | (1 << K)]);
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    if (r & (1 << K)) continue;
    const int r1 = r | (1 << K);
    T x0 = a[r], x1 = a[r1];
    T w;
    if constexpr (K < 3) w = wk[r & (NW - 1)];
    else w = cmul(tg, treg[r1]);
    if constexpr (FWD) {
      a[r] = cadd(x0, x1);
      a[r1] = cmul(csub(x0, x1), w);
    } else {
      x1 = cmulc(x1, w);
      a[r] = cadd(x0, x1);
      a[r1] = csub(x0, x1);
    }
  }
}

template <typename R, int LR, bool FWD>
__device__ __forceinline__ void apply_qft_dir(V2<R> (&a)[1 << LR], const TileOp& op, V2<R> tg, const V2<R>* treg) {
  switch (op.rk) {
    case 0: apply_qft<R, LR, 0, FWD>(a, op, tg, treg); break;
    case 1: if constexpr (LR > 1) apply_qft<R, LR, 1, FWD>(a, op, tg, treg); break;
    case 2: if constexpr (LR > 2) apply_qft<R, LR, 2, FWD>(a, op, tg, treg); break;
    case 3: if constexpr (LR > 3) apply_qft<R, LR, 3, FWD>(a, op, tg, treg); break;
    case 4: if constexpr (LR > 4) apply_qft<R, LR, 4, FWD>(a, op, tg, treg); break;
    default: break;
  }
}

// tg: the group factor e^{i pi Lg / 2^width} of the stage (1 for width 0)
template <typename R, int LR>
__device__ __forceinline__ void apply_qft_op(V2<R> (&a)[1 << LR], const TileOp& op, V2<R> tg, const V2<R>* treg) {
  if (op.kind == OP_QFT_FWD) apply_qft_dir<R, LR, true>(a, op, tg, treg);
  else apply_qft_dir<R, LR, false>(a, op, tg, treg);
}

// A phase of chained QFT stages, one per register slot of a 16-amplitude
// group, on consecutive ladder bits.  The stage on slot K has width
// wmax - (top - K); its pair (r, r | 2^K) takes the factor
//   e^{i pi Lg / 2^{width}} e^{i pi rho / 2^K},  rho = r mod 2^K,
// the first the group factor p^(2^(top-K)) (p the top stage's), the second a
// compile-time constant: a multiple of pi/8, formed from the group factor by
// a quarter turn (free), the pi/4 rotation (two adds, two products) or one
// complex product with cos/sin(pi/8).
template <typename R, int K, int RHO>
__device__ __forceinline__ V2<R> qft_wk(V2<R> tg, const V2<R>* wk) {
  constexpr int N = 1 << K;       // angle pi RHO / N, RHO < N
  constexpr int E = RHO * (8 / N);  // the same angle in units of pi/8
  constexpr R kC8 = (R)0.92387953251128675613, kS8 = (R)0.38268343236508977173;
  constexpr R kH = (R)0.70710678118654752440;
  if constexpr (E == 0) {
    return tg;
  } else if constexpr (E >= 4) {  // a quarter turn after the factor of angle - pi/2
    const V2<R> b = wk[RHO - N / 2];
    return mk<R>(-b.y, b.x);
  } else if constexpr (E == 2) {
    return mk<R>((tg.x - tg.y) * kH, (tg.x + tg.y) * kH);
  } else if constexpr (E == 1) {
    return cmul(tg, mk<R>(kC8, kS8));
  } else {
    return cmul(tg, mk<R>(kS8, kC8));
  }
}

template <typename R, int K, bool FWD>
__device__ __forceinline__ void qft_slot(V2<R> (&a)[16], V2<R> tg) {
  using T = V2<R>;
  constexpr int NW = 1 << K;
  T wk[NW];
  wk[0] = tg;
  if constexpr (NW > 1) wk[1] = qft_wk<R, K, 1>(tg, wk);
  if constexpr (NW > 2) {
    wk[2] = qft_wk<R, K, 2>(tg, wk);
    wk[3] = qft_wk<R, K, 3>(tg, wk);
  }
  if constexpr (NW > 4) {
    wk[4] = qft_wk<R, K, 4>(tg, wk);
    wk[5] = qft_wk<R, K, 5>(tg, wk);
    wk[6] = qft_wk<R, K, 6>(tg, wk);
    wk[7] = qft_wk<R, K, 7>(tg, wk);
  }
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    if (r & (1 << K)) continue;
    const int r1 = r | (1 << K);
    const T w = wk[r & (NW - 1)];
    T x0 = a[r], x1 = a[r1];
    if constexpr (FWD) {
      a[r] = cadd(x0, x1);
      a[r1] = cmul(csub(x0, x1), w);
    } else {
      x1 = cmulc(x1, w);
      a[r] = cadd(x0, x1);
      a[r1] = csub(x0, x1);
    }
  }
}

// NS chained stages (3 or 4) on register slots 0 .. NS-1 (a fourth slot
// above them carries no stage).  p: the group factor of the top stage (slot
// NS-1, width wmax); slot K takes p^(2^(NS-1-K)).  Forward stages run from
// the top slot down, inverse ones from slot 0 up (conjugate factors), as
// apply_qft does one stage at a time.
template <typename R, bool FWD, int NS>
__device__ __forceinline__ void apply_qft_chain(V2<R> (&a)[16], V2<R> p) {
  using T = V2<R>;
  T pw[NS];
  pw[0] = p;
#pragma unroll
  for (int d = 1; d < NS; ++d) pw[d] = cmul(pw[d - 1], pw[d - 1]);
  if constexpr (FWD) {
    if constexpr (NS == 4) qft_slot<R, 3, true>(a, pw[NS - 4]);
    qft_slot<R, 2, true>(a, pw[NS - 3]);
    qft_slot<R, 1, true>(a, pw[NS - 2]);
    qft_slot<R, 0, true>(a, pw[NS - 1]);
  } else {
    qft_slot<R, 0, false>(a, pw[NS - 1]);
    qft_slot<R, 1, false>(a, pw[NS - 2]);
    qft_slot<R, 2, false>(a, pw[NS - 3]);
    if constexpr (NS == 4) qft_slot<R, 3, false>(a, pw[NS - 4]);
  }
}

// The group factor of a stage from the twiddle tables (Lg = 0 reads entry 0
// of every table, exactly 1).
template <typename R>
__device__ __forceinline__ V2<R> qft_group_factor(const TileOp& op, uint32_t gq, const float2* tw) {
  const int width = op.width;
  if (width == 0) return mk<R>(1, 0);
  const uint32_t mask = (width >= 32) ? 0xffffffffu : ((1u << width) - 1u);
  return Twiddle<R>::get(tw, (gq >> op.lad_shift) & mask, width);
}

// Shared-memory slot of tile-local amplitude i (the chunk swizzle of k_tile
// at amplitude granularity).
template <typename R>
__device__ __forceinline__ uint32_t amp_slot(uint32_t i) {
  return sizeof(R) == 4 ? (i ^ ((i >> 3) & 0xEu)) : (i ^ ((i >> 3) & 7u));
}

template <typename R>
__device__ __forceinline__ V2<R> epi_phase(const EpiDesc& D, const V2<R>* lut, uint32_t x, V2<R> f) {
#pragma unroll
  for (int w = 0; w < kEpiWin; ++w) {
    if (w >= D.n_var) break;
    f = cmul(f, lut[D.off[w] + ((x >> D.shift[w]) & ((1u << D.nbits[w]) - 1u))]);
  }
  return f;
}

constexpr int ilog2_c(int x) { return x <= 1 ? 0 : 1 + ilog2_c(x >> 1); }

// A applied to the chunk-index bits of k*NT (chunk c = tid + k*NT, amplitude
// c << CB): the XOR of the permutation columns of k's set bits
template <int LT, int LCH, int CB>
__device__ __forceinline__ uint32_t chunk_cols(int k, const uint32_t* cols) {
  uint32_t a = 0;
#pragma unroll
  for (int b = 0; b < LCH; ++b)
    if ((k >> b) & 1) a ^= cols[CB + LT + b];
  return a;
}

// MODE 2 write-back: output chunk c = tid + k*NT of output tile bo holds
// amplitudes y = c << CB (and y | 1 for complex64); their values are the
// processed input amplitudes l = cl ^ A y (identity without a permutation)
// of input tile ib, times phase(ib | l).
template <typename R, int M, int LT, int CPT>
__device__ __forceinline__ void epilogue_store(const EpiDesc& D, const V2<R>* cur, const uint32_t* cols,
                                               const V2<R>* lut, V2<R>* dst, uint32_t bo, uint32_t ib, uint32_t cl,
                                               int tid, uint32_t at) {
  using T = V2<R>;
  constexpr int NT = 1 << LT;
  constexpr int CB = sizeof(T) == 8 ? 1 : 0;
  constexpr int LCH = ilog2_c(CPT);
  const bool perm = D.perm, diag = D.diag;
  T hc = mk<R>(1, 0);
  if (diag) {
    for (int w = D.n_var; w < D.n_win; ++w)
      hc = cmul(hc, lut[D.off[w] + ((ib >> D.shift[w]) & ((1u << D.nbits[w]) - 1u))]);
  }
  // a permutation that keeps index bit 0 (A e_0 = e_0, CNOT ladders) moves
  // amplitude pairs: the output pair (y, y|1) is one 16-byte chunk of the
  // input, swapped when l0 is odd
  if constexpr (CB == 1) {
    if (perm && !diag && cols[0] == 1u) {
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        const uint32_t y = ((uint32_t)tid + (uint32_t)(k * NT)) << 1;
        const uint32_t l0 = cl ^ at ^ chunk_cols<LT, LCH, CB>(k, cols);
        const float4 v = *reinterpret_cast<const float4*>(cur + amp_slot<R>(l0 & ~1u));
        *reinterpret_cast<float4*>(dst + (bo | y)) = (l0 & 1u) ? make_float4(v.z, v.w, v.x, v.y) : v;
      }
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const uint32_t y = ((uint32_t)tid + (uint32_t)(k * NT)) << CB;
    const uint32_t l0 = perm ? (cl ^ at ^ chunk_cols<LT, LCH, CB>(k, cols)) : y;
    T v0 = cur[amp_slot<R>(l0)];
    if (diag) v0 = cmul(v0, epi_phase<R>(D, lut, ib | l0, hc));
    if constexpr (CB == 1) {
      const uint32_t l1 = perm ? (l0 ^ cols[0]) : (y | 1u);
      T v1 = cur[amp_slot<R>(l1)];
      if (diag) v1 = cmul(v1, epi_phase<R>(D, lut, ib | l1, hc));
      *reinterpret_cast<float4*>(dst + (bo | y)) = make_float4((float)v0.x, (float)v0.y, (float)v1.x, (float)v1.y);
    } else {
      dst[bo | y] = v0;
    }
  }
}

template <typename R>
__device__ __forceinline__ void apply_regdiag(V2<R> (&a)[16], const V2<R>* lut, const RegDiag& D, uint32_t gq) {
  using T = V2<R>;
  T f = mk<R>(1, 0);
#pragma unroll
  for (int w = 0; w < kEpiWin; ++w) {
    if (w >= D.n_win) break;
    f = cmul(f, lut[D.off[w] + ((gq >> D.shift[w]) & ((1u << D.nbits[w]) - 1u))]);
  }
  uint32_t cc = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (j < D.nc) cc |= ((gq >> D.cbit[j]) & 1u) << j;
  const T* tr = lut + D.toff + cc * 17u;
#pragma unroll
  for (int r = 0; r < 16; ++r) a[r] = cmul(a[r], cmul(f, tr[r]));
}

// Build-time choices kept for comparison builds (-D...): resident CTAs per SM
// of the 256-thread MODE 2 sweep (3: 80 registers a thread, the fused layer's
// low sweep 0.5 ms faster at 30 qubits than with 2), and the late request of
// the next tile (see k_tile; 0 requests it before waiting for the current one).
#ifndef MQ_MODE2_CTAS
#define MQ_MODE2_CTAS 3
#endif
#ifndef MQ_LATE_PREFETCH
#define MQ_LATE_PREFETCH 1
#endif
// Tile of 2^M amplitudes, 2^LT threads, 2^LR amplitudes per register
// group.  Global traffic moves in 16-byte chunks (two complex64 or one
// complex128 amplitude): chunk c covers tile-local element c << CB.
//
// Shared-memory layout: chunk c sits at chunk slot swz(c) = c ^ ((c >> 3) & 7),
// i.e. the chunk's position inside its 128-byte row is XORed with the next
// three chunk-index bits.  swz is linear over GF(2), so the slot of an
// amplitude is the XOR of the slots of its index bits; the host stores those
// per-bit slots (PhaseDesc s_reg / s_grp) and the kernel combines them with
// XOR.  Without it, a register phase over tile bits 0-3 (the low sweep) has
// the 16 threads of a half-warp 128 bytes apart, all in one bank pair.
//
// MODE 0: U(2) / controlled U(2) phases; MODE 1: QFT stages; MODE 2: U(2)
// phases plus the fused-layer epilogue (PT = FusedParams; a permuted or
// window-diagonal write-back needs the tile bits [0, M)); MODE 3: U(2) phases
// with register-phase diagonals only and the plain write-back.
//
// TMA: tiles arrive by one tensor-map load per tile (P.tma), issued by
// thread 0 and completed on an mbarrier per tile buffer; the plain write-back
// leaves as one tensor-map store.  Every wait for a tile is bounded
// (kTmaWaitNs); a CTA whose tile does not arrive in time records the fault
// in g_tile_fault and returns as a whole.
template <typename R, int M, int LR, int LT, int MODE, typename PT, bool TMA>
__global__ void __launch_bounds__(1 << LT, (LT >= 9 ? 1 : (LT >= 8 ? (MODE == 2 ? MQ_MODE2_CTAS : 3) : (LT >= 7 ? (sizeof(R) == 4 && LR == 4 ? 6 : 3) : (LT >= 6 && sizeof(R) == 4 ? 8 : 1)))))
k_tile(const V2<R>* src, V2<R>* dst, const __grid_constant__ PT P) {
  using T = V2<R>;
  constexpr bool QFT = MODE == 1;
  constexpr bool EPI = MODE >= 2;
  constexpr bool STORE_EPI = MODE == 2;  // MODE 3: register diagonals only, plain write-back
  constexpr int NT = 1 << LT;
  constexpr int NR = 1 << LR;
  constexpr int E = 1 << M;
  constexpr int GPT = (E / NR) / NT;
  constexpr int CB = sizeof(T) == 8 ? 1 : 0;          // log2 amplitudes per 16-byte chunk
  constexpr int NCH = E >> CB;                         // chunks per tile
  constexpr int CPT = NCH / NT;                        // chunks per thread
  constexpr int LCH = (M - CB) - LT;                   // chunk-index bits above the thread bits
  constexpr int NBUF = tile_nbuf(M, LT);
  static_assert(GPT >= 1 && CPT >= 1, "bad tile configuration");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // TMA tiles start on a 1024-byte boundary (the 128-byte swizzle repeats
  // every 8 rows of 128 bytes, counted from the address), followed by one
  // 8-byte mbarrier per tile buffer in a 64-byte slot; the host adds the
  // slack for both
  unsigned char* smem = smem_raw;
  if constexpr (TMA) smem += (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  T* bufs = reinterpret_cast<T*>(smem);
  constexpr size_t kBarBytes = TMA ? 64 : 0;
  const uint32_t bar0 = smem_u32(smem + NBUF * sizeof(T) * E);
  PhaseDesc* phs = reinterpret_cast<PhaseDesc*>(smem + NBUF * sizeof(T) * E + kBarBytes);
  const float2* tw = nullptr;
  // shared memory: tile buffers, (TMA) the mbarriers, the launch's phase
  // descriptors, then (MODE >= 2) the permutation columns and the diagonal
  // tables
  uint32_t* ttab = reinterpret_cast<uint32_t*>(smem + NBUF * sizeof(T) * E + kBarBytes + sizeof(PhaseDesc) * P.n_phases);
  const size_t ph_end = NBUF * sizeof(T) * E + kBarBytes + sizeof(PhaseDesc) * P.n_phases +
                        sizeof(uint32_t) * kThreadTabWords * P.n_phases;
  uint32_t* ecols = reinterpret_cast<uint32_t*>(smem + ph_end);
  T* qreg = reinterpret_cast<T*>(smem + ph_end);  // MODE 1: per op, the register factors treg[32]
  T* elut = reinterpret_cast<T*>(smem + ph_end + 128);
  const int tid = threadIdx.x;
  const uint32_t t_lo = (uint32_t)tid & 15u, t_hi = (uint32_t)tid >> 4;
  if constexpr (TMA) {
    if (tid == 0) {
      for (int b = 0; b < NBUF; ++b) mbar_init(bar0 + 8u * b, 1);
      mbar_init_fence();
    }
  }
  {
    const uint32_t words = (uint32_t)(sizeof(PhaseDesc) * P.n_phases / 4);
    const uint32_t* srcw = reinterpret_cast<const uint32_t*>(&P.ph[0]);
    uint32_t* dstw = reinterpret_cast<uint32_t*>(phs);
    for (uint32_t w = tid; w < words; w += NT) dstw[w] = srcw[w];
  }
  // the thread tables of every phase: a group's offsets over the thread's
  // bits of its index q (q's bits below LT are the thread id's) are then two
  // table reads, the same for every tile of the sweep
  constexpr int TLO = LT < 4 ? LT : 4;
  static_assert(LT - TLO <= 5, "thread tables hold 5 high thread bits");
  for (int w = tid; w < P.n_phases * kThreadTabWords; w += NT) {
    const int p = w / kThreadTabWords, r = w % kThreadTabWords;
    const uint32_t* grp = (r >= 48) ? P.ph[p].g_grp : P.ph[p].s_grp;
    const int e = r % 48;
    const bool hi = e >= 16;
    const uint32_t bits = hi ? (uint32_t)(e - 16) : (uint32_t)e;
    const int j0 = hi ? TLO : 0, nb = hi ? LT - TLO : TLO;
    uint32_t v = 0;
    for (int j = 0; j < nb; ++j)
      if ((bits >> j) & 1u) v ^= grp[j0 + j];
    ttab[w] = v;
  }
  if constexpr (!QFT) {
    if (P.mats_dev) {
      __syncthreads();
      for (int j = tid; j < P.n_phases * 40; j += NT) {
        const int p = j / 40, k = (j / 8) % 5, e = j % 8;
        const int q = P.mat_q[p][k] - 1;
        if (q >= 0) {
          const double v = P.mats_dev[(size_t)q * 8 + e];
          phs[p].ud[k][e] = v;
          phs[p].uf[k][e] = (float)v;
        }
      }
    }
  }
  if constexpr (QFT) {
    const uint32_t words = (uint32_t)P.n_ops * 32u * (uint32_t)(sizeof(T) / 4);
    const uint32_t* srcw;
    if constexpr (sizeof(R) == 4) srcw = reinterpret_cast<const uint32_t*>(&P.twf[0][0]);
    else srcw = reinterpret_cast<const uint32_t*>(&P.twd[0][0]);
    uint32_t* dstw = reinterpret_cast<uint32_t*>(qreg);
    for (uint32_t w = tid; w < words; w += NT) dstw[w] = srcw[w];
  }
  if constexpr (EPI) {
    for (int w = tid; w < 32; w += NT) ecols[w] = P.epi.cols[w];
    const uint32_t words = P.epi.n_entries * (uint32_t)(sizeof(T) / 4);
    const uint32_t* srcw = reinterpret_cast<const uint32_t*>(P.epi.lut);
    uint32_t* dstw = reinterpret_cast<uint32_t*>(elut);
    for (uint32_t w = tid; w < words; w += NT) dstw[w] = srcw[w];
  }
  __syncthreads();

  if constexpr (QFT) tw = g_qft_twiddles;
  // MODE 2 with a permutation: A applied to the thread part of this
  // thread's output chunks (c = tid + k*NT -> amplitude c << CB), computed
  // once; the part of k*NT comes from the columns at the write-back (one
  // register held through the sweep instead of CPT)
  uint32_t epi_at = 0;
  if constexpr (STORE_EPI) {
    if (P.epi.perm) {
#pragma unroll
      for (int b = 0; b < LT; ++b)
        if ((tid >> b) & 1) epi_at ^= ecols[CB + b];
    }
  }

  // chunk c = tid + k*NT: global part of the thread bits, computed once
  uint32_t g_t = 0;
#pragma unroll
  for (int b = 0; b < LT; ++b)
    if ((tid >> b) & 1) g_t |= 1u << P.tile_bit[CB + b];
  // swz(tid + k*NT) = swz(tid) ^ swz(k*NT) (tid < NT, swz linear); the
  // second term is a compile-time value once the k loops are unrolled
  const uint32_t s_t = (uint32_t)tid ^ (((uint32_t)tid >> 3) & 7u);
  auto slot = [&](int k) -> uint32_t {
    const uint32_t kk = (uint32_t)(k * NT);
    return s_t ^ (kk ^ ((kk >> 3) & 7u));
  };
  const bool hi_contig = P.hi_contig;
  const int hi_shift = P.hi_shift;
  auto g_k = [&](int k) -> uint32_t {
    if (hi_contig) return (uint32_t)k << hi_shift;
    uint32_t g = 0;
#pragma unroll
    for (int b = 0; b < LCH; ++b)
      if ((k >> b) & 1) g |= 1u << P.tile_bit[CB + LT + b];
    return g;
  };

  // Source tile of output tile t.  MODE 2 with a permutation: the output
  // tile t << M reads A (t << M) ^ c, a whole input tile plus a low offset
  // (returned in cl) because A maps the low space onto itself.
  auto src_base = [&](uint32_t t, uint32_t& cl) -> uint32_t {
    cl = 0;
    if constexpr (STORE_EPI) {
      if (!P.epi.perm) return deposit_runs(t, P.runs);
      const uint32_t b =
          P.epi.c ^ P.epi.htab[t & 255u] ^ P.epi.htab[256 + ((t >> 8) & 255u)] ^ P.epi.htab[512 + ((t >> 16) & 255u)];
      cl = b & (uint32_t)(E - 1);
      return b & ~(uint32_t)(E - 1);
    } else {
      return deposit_runs(t, P.runs);
    }
  };
  uint32_t tile = blockIdx.x;
  auto load_tile = [&](uint32_t t, T* buf) {
    uint32_t cl;
    const uint32_t gb = src_base(t, cl) | g_t;
    const uint32_t sb = smem_u32(buf);
#pragma unroll
    for (int k = 0; k < CPT; ++k) cp_async<16>(sb + 16u * slot(k), src + (gb | g_k(k)));
  };
  // TMA: the box coordinates of the tile whose base index is `base` (free
  // dimensions take base's bits of their run, tile dimensions 0)
  auto tma_coords = [&](uint32_t base, int32_t (&c)[5]) {
#pragma unroll
    for (int d = 0; d < 5; ++d) c[d] = (int32_t)((base >> P.tma.start[d]) & P.tma.mask[d]);
  };
  // TMA (thread 0): tile t into buffer b
  auto tma_load_tile = [&](uint32_t t, int b) {
    uint32_t cl;
    int32_t c[5];
    tma_coords(src_base(t, cl), c);
    const uint32_t bar = bar0 + 8u * (uint32_t)b;
    mbar_expect_tx(bar, P.tma.bytes);
    tma_load_5d(smem_u32(bufs + b * E), &P.tma.src, c, bar);
  };
  if constexpr (TMA) {
    if (tid == 0 && tile < P.n_tiles) tma_load_tile(tile, 0);
  } else if constexpr (NBUF == 2) {
    if (tile < P.n_tiles) load_tile(tile, bufs);
    cp_async_commit();
  }
  // two buffers: the next tile is requested after the barrier that follows
  // this tile's arrival; every thread has then finished the previous tile's
  // write-back from the buffer it goes into, so the write-back needs no
  // barrier of its own (three barriers per tile of two phases, not four)
  constexpr bool LATE = NBUF == 2 && MQ_LATE_PREFETCH;
  T a[NR];
  for (int it = 0; tile < P.n_tiles; tile += gridDim.x, ++it) {
    const int cb = NBUF == 2 ? (it & 1) : 0;
    T* cur = bufs + cb * E;
    if constexpr (TMA) {
      // every thread waits for the tile itself (acquiring the TMA's writes);
      // if any wait gives up, the whole CTA records it and returns together
      const uint32_t bar = bar0 + 8u * (uint32_t)cb;
      const uint32_t parity = (uint32_t)((NBUF == 2 ? (it >> 1) : it) & 1);
      const bool ok = mbar_wait_bounded(bar, parity, kTmaWaitNs);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(&g_tile_fault, 1u);
          mbar_wait_bounded(bar, parity, kTmaWaitNs);  // the load in flight, once more
          bulk_wait_all();
        }
        return;
      }
    } else if constexpr (LATE) {
      cp_async_wait<0>();
      __syncthreads();
      const uint32_t next = tile + gridDim.x;
      if (next < P.n_tiles) load_tile(next, bufs + ((it + 1) & 1) * E);
      cp_async_commit();
    } else if constexpr (NBUF == 2) {
      const uint32_t next = tile + gridDim.x;
      if (next < P.n_tiles) load_tile(next, bufs + ((it + 1) & 1) * E);
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
    } else {
      // the buffer is free: the previous tile's write-back ended with a barrier
      load_tile(tile, bufs);
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
    }
    uint32_t cl_in;
    const uint32_t base = src_base(tile, cl_in);
    for (int ph = 0; ph < P.n_phases; ++ph) {
      const PhaseDesc& D = phs[ph];
      uint32_t greg[LR], sreg[LR];
#pragma unroll
      for (int k = 0; k < LR; ++k) { greg[k] = D.g_reg[k]; sreg[k] = D.s_reg[k]; }
      // the group's global index is read only by controlled gates, QFT
      // twiddles and register-phase diagonals
      bool need_g = QFT || D.any_ctl;
      if constexpr (EPI && LR == 4)
        need_g = need_g || (ph == 0 && P.epi.pre.on) || (ph == P.n_phases - 1 && P.epi.dreg);
#pragma unroll
      for (int g = 0; g < GPT; ++g) {
        const uint32_t q = (uint32_t)tid + (uint32_t)g * NT;
        // thread bits from the phase's tables, the bits of g (above LT) from
        // the descriptor (compile-time selected)
        const uint32_t* tt = ttab + ph * kThreadTabWords;
        uint32_t sq = tt[t_lo] ^ tt[16 + t_hi], gq = base;
#pragma unroll
        for (int j = LT; j < M - LR; ++j)
          if ((q >> j) & 1) sq ^= D.s_grp[j];
        if (need_g) {
          gq |= tt[48 + t_lo] | tt[64 + t_hi];
#pragma unroll
          for (int j = LT; j < M - LR; ++j)
            if ((q >> j) & 1) gq |= D.g_grp[j];
        }
        // complex64 with tile bit 0 in register slot 0: amplitudes r, r+1 share
        // one 16-byte chunk, read as one vector (a quarter-warp then covers
        // all eight chunk slots of a row)
        const bool pair = sizeof(R) == 4 && sreg[0] == 1u;
        if (pair) {
#pragma unroll
          for (int r = 0; r < NR; r += 2) {
            const float4 v = *reinterpret_cast<const float4*>(cur + (sq ^ osel<LR>(r, sreg)));
            a[r] = mk<R>((R)v.x, (R)v.y);
            a[r + 1] = mk<R>((R)v.z, (R)v.w);
          }
        } else {
#pragma unroll
          for (int r = 0; r < NR; ++r) a[r] = cur[sq ^ osel<LR>(r, sreg)];
        }
        if constexpr (EPI && LR == 4) {
          if (P.epi.pre.on && ph == 0) apply_regdiag<R>(a, elut, P.epi.pre, gq);
        }
        if constexpr (QFT) {
          const int o0 = P.ph_op[ph], o1 = P.ph_op[ph + 1];
          if (P.qchain[ph]) {
            // the phase's stages sit on consecutive bits over one ladder, so
            // they share Lg (the ladder bits below the phase) and differ in
            // width by one: the factor of width w - d is p^(2^d), p the factor
            // at the largest width w (squarings instead of table lookups)
            const int wmax = P.qchain[ph] - 1;
            T pw[LR];
            pw[0] = mk<R>(1, 0);
            if (wmax) {
              const uint32_t mask = (wmax >= 32) ? 0xffffffffu : ((1u << wmax) - 1u);
              pw[0] = Twiddle<R>::get(tw, (gq >> P.ops[o0].lad_shift) & mask, wmax);
            }
            bool done = false;
            if constexpr (LR == 4) {
              const int ns = P.qfull[ph];
              if (ns) {
                const bool fwd = P.ops[o0].kind == OP_QFT_FWD;
                if (ns == 4) {
                  if (fwd) apply_qft_chain<R, true, 4>(a, pw[0]);
                  else apply_qft_chain<R, false, 4>(a, pw[0]);
                } else {
                  if (fwd) apply_qft_chain<R, true, 3>(a, pw[0]);
                  else apply_qft_chain<R, false, 3>(a, pw[0]);
                }
                done = true;
              }
            }
            if (!done) {
#pragma unroll
              for (int d = 1; d < LR; ++d) pw[d] = cmul(pw[d - 1], pw[d - 1]);
              for (int o = o0; o < o1; ++o) {
                const int d = wmax - P.ops[o].width;
                T tg = pw[0];
#pragma unroll
                for (int e = 1; e < LR; ++e)
                  if (d == e) tg = pw[e];
                apply_qft_op<R, LR>(a, P.ops[o], tg, qreg + 32 * o);
              }
            }
          } else {
            for (int o = o0; o < o1; ++o)
              apply_qft_op<R, LR>(a, P.ops[o], qft_group_factor<R>(P.ops[o], gq, tw), qreg + 32 * o);
          }
        } else {
          if (D.any_ctl) apply_u2_phase<R, LR, true, (MODE < 2)>(a, D, gq, greg);
          else apply_u2_phase<R, LR, false, (MODE < 2)>(a, D, gq, greg);
        }
        if constexpr (EPI && LR == 4) {
          if (P.epi.dreg && ph == P.n_phases - 1) {
            T f = mk<R>(1, 0);
#pragma unroll
            for (int w = 0; w < kEpiWin; ++w) {
              if (w >= P.epi.n_win) break;
              f = cmul(f, elut[P.epi.off[w] + ((gq >> P.epi.shift[w]) & ((1u << P.epi.nbits[w]) - 1u))]);
            }
            uint32_t cc = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j)
              if (j < P.epi.nc) cc |= ((gq >> P.epi.cbit[j]) & 1u) << j;
            const T* tr = elut + P.epi.toff + cc * 17u;
#pragma unroll
            for (int r = 0; r < NR; ++r) a[r] = cmul(a[r], cmul(f, tr[r]));
          }
        }
        if constexpr (QFT && TMA) {
          // a TMA store writes the tile as it stands: the sweep's 2^{-stages/2}
          // is applied here instead of in the write-back (the same product)
          if (ph == P.n_phases - 1) {
#pragma unroll
            for (int r = 0; r < NR; ++r) a[r] = cscale(a[r], (R)P.scale);
          }
        }
        if (pair) {
#pragma unroll
          for (int r = 0; r < NR; r += 2)
            *reinterpret_cast<float4*>(cur + (sq ^ osel<LR>(r, sreg))) =
                make_float4((float)a[r].x, (float)a[r].y, (float)a[r + 1].x, (float)a[r + 1].y);
        } else {
#pragma unroll
          for (int r = 0; r < NR; ++r) cur[sq ^ osel<LR>(r, sreg)] = a[r];
        }
      }
      // TMA: the tile's last shared-memory writes become visible to the
      // async proxy (the TMA store that reads them, the TMA load that will
      // overwrite them) before the barrier
      if constexpr (TMA)
        if (ph == P.n_phases - 1) fence_proxy_async_smem();
      __syncthreads();
      if constexpr (TMA && NBUF == 2) {
        // after the first barrier of this tile every thread has finished the
        // previous tile, so its buffer takes this CTA's next tile (once a TMA
        // store from it has read it out)
        if (ph == 0 && tid == 0) {
          const uint32_t next = tile + gridDim.x;
          if (next < P.n_tiles) {
            if (P.tma.store) bulk_wait_read();
            tma_load_tile(next, cb ^ 1);
          }
        }
      }
    }
    if constexpr (STORE_EPI && TMA && CB == 1) {
      if (P.tma.store == 2) {
        // permutation keeping index bit 0: output chunk c = tid + k*NT is the
        // input pair at l0 = cl ^ A(c << 1) (swapped when l0 is odd).  Every
        // thread reads its chunks, the barrier ends all reads of the tile,
        // the chunks go to their output slots, and the tile leaves as one
        // TMA store to output tile `tile`
        float4 v[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
          const uint32_t l0 = cl_in ^ epi_at ^ chunk_cols<LT, LCH, CB>(k, ecols);
          const float4 w = *reinterpret_cast<const float4*>(cur + amp_slot<R>(l0 & ~1u));
          v[k] = (l0 & 1u) ? make_float4(w.z, w.w, w.x, w.y) : w;
        }
        __syncthreads();
        float4* c4w = reinterpret_cast<float4*>(cur);
#pragma unroll
        for (int k = 0; k < CPT; ++k) c4w[slot(k)] = v[k];
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
          int32_t c[5];
          tma_coords(tile << M, c);
          tma_store_5d(&P.tma.dst, c, smem_u32(cur));
          bulk_commit();
          if constexpr (NBUF == 1) {
            const uint32_t next = tile + gridDim.x;
            if (next < P.n_tiles) {
              bulk_wait_read();
              tma_load_tile(next, 0);
            }
          }
        }
        continue;
      }
    }
    if constexpr (STORE_EPI) {
      if (P.epi.perm || P.epi.diag) {
        epilogue_store<R, M, LT, CPT>(P.epi, cur, ecols, elut, dst, tile << M, base, cl_in, tid, epi_at);
        if constexpr (TMA && NBUF == 1) {
          __syncthreads();
          const uint32_t next = tile + gridDim.x;
          if (tid == 0 && next < P.n_tiles) tma_load_tile(next, 0);
        } else if constexpr (!LATE && !TMA) {
          __syncthreads();
        }
        continue;
      }
    }
    if constexpr (TMA) {
      if (P.tma.store) {
        // in place: the tile goes back where it came from
        if (tid == 0) {
          int32_t c[5];
          tma_coords(base, c);
          tma_store_5d(&P.tma.dst, c, smem_u32(cur));
          bulk_commit();
          if constexpr (NBUF == 1) {
            const uint32_t next = tile + gridDim.x;
            if (next < P.n_tiles) {
              bulk_wait_read();
              tma_load_tile(next, 0);
            }
          }
        }
        continue;
      }
    }
    const uint32_t gb = base | g_t;
    const float4* c4 = reinterpret_cast<const float4*>(cur);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      float4 v = c4[slot(k)];
      if (QFT) {
        if constexpr (sizeof(R) == 4) {
          const float sc = (float)P.scale;
          v.x *= sc; v.y *= sc; v.z *= sc; v.w *= sc;
        } else {
          double2 d = *reinterpret_cast<double2*>(&v);
          d.x *= P.scale; d.y *= P.scale;
          v = *reinterpret_cast<float4*>(&d);
        }
      }
      *reinterpret_cast<float4*>(dst + (gb | g_k(k))) = v;
    }
    if constexpr (TMA && NBUF == 1) {
      __syncthreads();
      const uint32_t next = tile + gridDim.x;
      if (tid == 0 && next < P.n_tiles) tma_load_tile(next, 0);
    } else if constexpr (!LATE && !TMA) {
      __syncthreads();
    }
  }
  if constexpr (TMA) {
    if (tid == 0) bulk_wait_all();  // the last TMA stores have written global memory
  } else {
    cp_async_wait<0>();
  }
}

// ---------------------------------------------------------------- host side
struct Sweep {
  const double* mats_dev = nullptr;        // U(2) matrices in device memory (rows by qubit)
  std::vector<int> tile_bits;              // ascending global bits
  std::vector<std::vector<int>> phases;    // register bits (tile-local) per phase
  std::vector<TileOp> ops;
  bool need_tw = false;
  double scale = 1.0;
  bool has_scale = false;
  // rotation matrices may run in tangent form (PhaseDesc::rot); the caller
  // multiplies the product of their factors (rot_factor) into a diagonal
  bool rot = false;
};

static bool rot_enabled() {
  const char* v = std::getenv("MQ_ROT");
  return !(v && v[0] == '0');
}
// The factor a rotation row pair keeps out of its tangent form: c when
// |c| >= |s| (then |t| <= 1), else s.
static double rot_factor(double c, double s) { return std::fabs(c) >= std::fabs(s) ? c : s; }

static int env_int(const char* name, int dflt, int lo, int hi) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  int x = std::atoi(v);
  return std::min(hi, std::max(lo, x));
}

static int reg_bits(int dtype, int m) {
  const int lr = dtype == MQ_C64 ? env_int("MQ_TILE_LR", 4, 4, 5) : 4;
  return std::min(m, lr);
}
// Largest tile of the general sweeps.  complex64 from 29 qubits: 13 bits,
// where 12-bit tiles (8 targets beside 4 passengers) would need a fourth
// sweep per layer.  A 30-qubit layer is then 3 sweeps (12 + 9 + 9 targets)
// and a QFT 3 sweeps.  They moved 25 % less data, held the SM clock at its
// maximum under the power cap, and measured 3776-3780 against 3620-3630 GB/s
// with 12-bit tiles.  Smaller states keep 12 (their layers fit 3 sweeps, and
// more tiles fill the SMs).
static int tile_max(int dtype, int n) {
  if (dtype != MQ_C64) return 11;
  const int lim = reg_bits(MQ_C64, 13) == 4 ? 13 : 12;
  return env_int("MQ_TILE_MAX", n >= env_int("MQ_TILE13_MIN_QUBITS", 29, 1, 32) ? lim : 12, 6, lim);
}
static int passengers() { return env_int("MQ_TILE_PASSENGERS", 4, 0, 5); }
static bool euler_enabled(const mq_state* h) {
  const char* v = std::getenv("MQ_EULER");
  if (v && v[0] == '0') return false;
  return h->n >= env_int("MQ_EULER_MIN_QUBITS", 20, 1, 32);
}
static int min_tile() { return env_int("MQ_TILE_MIN", 10, 1, 12); }
// The sweep plan of one handle: its own tile shape (mq_batch_set_tiles sets
// one on a batch's states) or the process-wide defaults above.
static int plan_tile_max(const mq_state* h) {
  if (h->tile_max > 0) return std::min(h->tile_max, h->dtype == MQ_C64 ? 12 : 11);
  // a state held to fewer SMs than the device has shares the GPU (a server's
  // large requests beside small ones): it keeps 12-bit tiles, whose CTAs
  // leave more room on each SM (served p50 0.04-0.06 s against 0.10-0.57 s
  // with 13-bit tiles for the 29-30-qubit requests)
  return tile_max(h->dtype, h->num_sms < h->device_sms ? 0 : h->n);
}
static int plan_passengers(const mq_state* h) { return h->tile_pas >= 0 ? h->tile_pas : passengers(); }
static int plan_min_tile(const mq_state* h) { return h->tile_min > 0 ? h->tile_min : min_tile(); }
// The Euler layer's sweeps fill their tiles to 12 bits with low passengers:
// a 7-bit sweep then moves 256-byte runs (fused config layer at 30 qubits
// 17.9 -> 16.3 ms); the complex sweeps measured slower that way.
static int euler_min_tile() { return env_int("MQ_EULER_TILE_MIN", 12, 1, 12); }
// ... and the low sweep's tile (its bits are contiguous: any size moves long runs)
static int euler_low_tile() { return env_int("MQ_EULER_LOW_TILE", 12, 1, 12); }
// Threads of a 13-bit complex64 tile: 2^9 with two tile buffers, or 2^8
// with one (three CTAs per SM).
static int tile13_lt() { return env_int("MQ_TILE13_LT", 8, 8, 9); }
// Euler layers: a high sweep of 8 target bits as a 13-bit tile with five
// passengers (256-byte runs, one tile buffer) instead of a 12-bit one.  With
// per-thread copies that paid (fused config layer at 30 qubits 15.6 -> 15.5
// ms); with TMA tiles the 12-bit tile and its second buffer win (30 qubits
// 14.07 -> 13.76 ms), so the default follows the tile movement.
static bool euler_hi13() { return env_int("MQ_EULER_HI13", tma_enabled() ? 0 : 1, 0, 1) == 1; }
// U(2) layers without diagonal terms through the Euler split as well.
static bool euler_plain() { return env_int("MQ_EULER_PLAIN", 1, 0, 1) == 1; }
// Euler layers: the high bit group (1 = the lowest) whose sweep carries the
// pre diagonal.  Default: the lowest with 12-bit tiles (30 qubits, four
// sweeps: 15.35 against 15.8 ms per layer for the others); the top one with
// 13-bit tiles (three sweeps: 12.32 against 12.47 ms)
static int euler_pre_group(int dflt) { return env_int("MQ_EULER_PRE_GROUP", dflt, 1, 8); }

// Register phases: targets (tile-local) chunked in the given order into
// groups of LR; the short group (the last, or with pad_first the first) is
// padded with the highest tile bits it does not hold (targets of other phases
// included: a slot without a gate is left alone), which keeps tile bits 0-3
// as thread bits and shared-memory access free of bank conflicts.  Records
// the phase index and register slot of every target.
static void make_phases(int m, int lr, const std::vector<int>& order, Sweep& sw, std::vector<int>& op_phase,
                        std::vector<int>& op_rk, bool pad_first = false) {
  sw.phases.clear();
  op_phase.assign(order.size(), 0);
  op_rk.assign(order.size(), 0);
  // pad_first: the first group takes the remainder, so that targets given
  // from the highest bit down fill the lower groups whole (a low sweep's
  // groups then sit on 4-bit boundaries, where register phases are free of
  // bank conflicts)
  const size_t rem = order.size() % (size_t)lr;
  const size_t first = (pad_first && rem) ? rem : (size_t)lr;
  for (size_t i = 0; i < order.size(); i += (i == 0 ? first : (size_t)lr)) {
    const size_t cnt = i == 0 ? first : (size_t)lr;
    std::vector<int> regs;
    for (size_t j = i; j < std::min(order.size(), i + cnt); ++j) {
      op_phase[j] = (int)sw.phases.size();
      regs.push_back(order[j]);
    }
    for (int b = m - 1; (int)regs.size() < lr && b >= 0; --b)
      if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
    std::vector<int> sorted = regs;
    std::sort(sorted.begin(), sorted.end());
    for (size_t j = i; j < std::min(order.size(), i + cnt); ++j)
      op_rk[j] = (int)(std::find(sorted.begin(), sorted.end(), order[j]) - sorted.begin());
    sw.phases.push_back(sorted);
  }
}

// cuTensorMapEncodeTiled from the driver, looked up once (the runtime hands
// out driver entry points, so the library needs no link against libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

void prepare_tile_maps() { (void)tensor_map_encoder(); }

// The tensor maps of a TMA sweep over the buffers it reads and writes.
int encode_tile_maps(TmaDesc& D, void* src, void* dst) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(MQ_EDEVICE, "cuTensorMapEncodeTiled is not available from the CUDA driver");
  const cuuint32_t estride[5] = {1, 1, 1, 1, 1};
  for (int k = 0; k < 2; ++k) {
    const CUresult r = enc(k ? &D.dst : &D.src, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, k ? dst : src, D.gdim, D.gstride,
                           D.box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MQ_EDEVICE, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
  }
  return MQ_OK;
}

template <typename R, int M, int LR, int LT, int MODE, typename PT, bool TMA>
static int launch_tile_t(mq_state* h, PT& P, size_t smem, bool out_of_place) {
  auto kern = k_tile<R, M, LR, LT, MODE, PT, TMA>;
  // the caller sized shared memory for two tile buffers
  if (tile_nbuf(M, LT) == 1) smem -= sizeof(V2<R>) << M;
  if constexpr (TMA) {
    smem += 1024 + 64;  // 1024-byte alignment of the tiles, the mbarriers
    int rc = encode_tile_maps(P.tma, h->buf[h->cur], out_of_place ? h->buf[1 - h->cur] : h->buf[h->cur]);
    if (rc) return rc;
  }
  // the opt-in shared-memory limit only grows; resident CTAs per SM depend on
  // this launch's shared memory (rounded up to 1 KiB), looked up per size
  static std::mutex mu;
  static int configured_smem = -1;
  static std::map<size_t, int> occupancy;
  int blocks_per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    const size_t key = (smem + 1023) & ~size_t(1023);
    if ((int)key > configured_smem) {
      MQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(key, 48 * 1024)));
      configured_smem = (int)std::max<size_t>(key, 48 * 1024);
    }
    auto it = occupancy.find(key);
    if (it == occupancy.end()) {
      MQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, 1 << LT, key));
      occupancy[key] = blocks_per_sm;
    } else {
      blocks_per_sm = it->second;
    }
  }
  const uint32_t grid = (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>(P.n_tiles, (uint64_t)h->num_sms * std::max(1, blocks_per_sm)));
  const V2<R>* s = reinterpret_cast<const V2<R>*>(h->buf[h->cur]);
  V2<R>* d = reinterpret_cast<V2<R>*>(out_of_place ? h->buf[1 - h->cur] : h->buf[h->cur]);
  kern<<<grid, 1 << LT, smem, h->stream>>>(s, d, P);
  MQ_LAUNCHED("k_tile");
  if (out_of_place) h->cur = 1 - h->cur;
  h->launches += 1;
  h->sweeps += 1;
  return MQ_OK;
}

// TMA form for the tiles of 10 bits and more (the sweeps of large states);
// smaller tiles, and sweeps whose tile the TMA form cannot describe, keep the
// per-thread asynchronous copies.
template <typename R, int M, int LR, int LT, int MODE, typename PT>
static int launch_tile_sel(mq_state* h, PT& P, size_t smem, bool oop) {
  if constexpr (M >= 10 && LR == 4) {
    if (P.tma.ndim) return launch_tile_t<R, M, LR, LT, MODE, PT, true>(h, P, smem, oop);
  }
  return launch_tile_t<R, M, LR, LT, MODE, PT, false>(h, P, smem, oop);
}

template <typename R, int MODE, int LR, typename PT>
static int dispatch_tile_lr(mq_state* h, PT& P, size_t smem, bool oop) {
  switch (P.m) {
#define MQ_TILE_CASE(MM)                                                        \
    case MM: {                                                                  \
      constexpr int L = (MM) < LR ? (MM) : LR;                                  \
      constexpr int LT = ((MM) - L) < 8 ? ((MM) - L) : 8;                       \
      return launch_tile_sel<R, MM, L, LT, MODE, PT>(h, P, smem, oop);          \
    }
    MQ_TILE_CASE(1) MQ_TILE_CASE(2) MQ_TILE_CASE(3) MQ_TILE_CASE(4) MQ_TILE_CASE(5) MQ_TILE_CASE(6)
    MQ_TILE_CASE(7) MQ_TILE_CASE(8) MQ_TILE_CASE(9) MQ_TILE_CASE(10) MQ_TILE_CASE(11)
#undef MQ_TILE_CASE
    case 12:
      if constexpr (sizeof(R) == 4) {
        constexpr int LT = LR == 5 ? 7 : 8;
        return launch_tile_sel<R, 12, LR, LT, MODE, PT>(h, P, smem, oop);
      }
      break;
    case 13:
      if constexpr (sizeof(R) == 4 && LR == 4) {
        if (tile13_lt() == 8) return launch_tile_sel<R, 13, 4, 8, MODE, PT>(h, P, smem, oop);
        return launch_tile_sel<R, 13, 4, 9, MODE, PT>(h, P, smem, oop);
      }
      break;
    default: break;
  }
  return fail(MQ_EUNSUPPORTED, "tile size not instantiated");
}

template <typename R, int MODE, typename PT>
static int dispatch_tile(mq_state* h, PT& P, size_t smem, bool oop) {
  if constexpr (MODE >= 2) {
    return dispatch_tile_lr<R, MODE, 4>(h, P, smem, oop);
  } else {
    if constexpr (sizeof(R) == 4) {
      if (reg_bits(MQ_C64, 12) == 4) return dispatch_tile_lr<R, MODE, 4>(h, P, smem, oop);
      return dispatch_tile_lr<R, MODE, 5>(h, P, smem, oop);
    }
    return dispatch_tile_lr<R, MODE, 4>(h, P, smem, oop);
  }
}

// Uploads g_qft_twiddles to the handle's device once (values formed in double
// on the host) and waits for the copy, so every stream of the device may read
// the table afterwards.
static int ensure_qft_twiddles(mq_state* h) {
  static std::mutex mu;
  static bool done[64] = {};
  if (h->device < 0 || h->device >= 64) return fail(MQ_EUNSUPPORTED, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(mu);
  if (done[h->device]) return MQ_OK;
  std::vector<float2> t(3072);
  for (int w = 0; w < 3; ++w)
    for (int j = 0; j < 1024; ++j) {
      const double a = M_PI * std::ldexp((double)j, -10 * (w + 1));
      t[w * 1024 + j] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  MQ_CUDA(cudaMemcpyToSymbolAsync(g_qft_twiddles, t.data(), t.size() * sizeof(float2), 0, cudaMemcpyHostToDevice,
                                  h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  done[h->device] = true;
  return MQ_OK;
}

// Fused-layer epilogue of a low sweep (see EpiDesc).
struct EpiPlan {
  bool diag = false, perm = false, dreg = false, pre = false;
  DiagWindows win;
  DiagRegister reg;      // dreg: after the last register phase's gates
  DiagRegister pre_reg;  // pre: before the first register phase's gates
  uint32_t cols[32] = {};
  uint32_t c = 0;
};

// Copies a register-phase diagonal's tables to vals[base..] and its
// descriptor into RD (offsets relative to the whole table array).
template <typename R>
static uint32_t fill_regdiag(RegDiag& RD, const DiagRegister& G, R* vals, uint32_t base) {
  RD.on = 1;
  RD.n_win = (uint8_t)G.win.n;
  RD.nc = (uint8_t)G.nc;
  for (int j = 0; j < G.nc; ++j) RD.cbit[j] = (uint8_t)G.cbit[j];
  for (int w = 0; w < G.win.n; ++w) {
    RD.shift[w] = (uint8_t)G.win.shift[w];
    RD.nbits[w] = (uint8_t)G.win.nbits[w];
    RD.off[w] = (uint16_t)(base + G.win.off[w]);
  }
  RD.toff = (uint16_t)(base + G.t_off);
  const size_t cnt = G.win.vals.size() / 2;
  for (size_t j = 0; j < 2 * cnt; ++j) vals[2 * base + j] = (R)G.win.vals[j];
  return base + (uint32_t)cnt;
}

template <typename R>
static void fill_epi(EpiDesc& D, const EpiPlan& e, int m, int n) {
  D.diag = e.diag ? 1 : 0;
  D.perm = e.perm ? 1 : 0;
  if (e.perm) {
    for (int j = 0; j < n; ++j) D.cols[j] = e.cols[j];
    D.c = e.c;
    for (int x = 0; x < 768; ++x) {
      uint32_t v = 0;
      for (int bit = 0; bit < 8; ++bit) {
        const int j = m + 8 * (x >> 8) + bit;
        if (((x >> bit) & 1) && j < n) v ^= e.cols[j];
      }
      D.htab[x] = v;
    }
  }
  uint32_t used = 0;
  if (e.pre) {
    // after the post tables when both are present
    const uint32_t base = e.dreg ? (uint32_t)(e.reg.win.vals.size() / 2) : 0u;
    used = fill_regdiag<R>(D.pre, e.pre_reg, reinterpret_cast<R*>(D.lut), base);
    D.n_entries = used;
  }
  if (e.dreg) {
    const DiagRegister& G = e.reg;
    D.dreg = 1;
    D.n_win = (uint8_t)G.win.n;
    D.nc = (uint8_t)G.nc;
    for (int j = 0; j < G.nc; ++j) D.cbit[j] = (uint8_t)G.cbit[j];
    for (int w = 0; w < G.win.n; ++w) {
      D.shift[w] = (uint8_t)G.win.shift[w];
      D.nbits[w] = (uint8_t)G.win.nbits[w];
      D.off[w] = (uint16_t)G.win.off[w];
    }
    D.toff = (uint16_t)G.t_off;
    R* vals = reinterpret_cast<R*>(D.lut);
    const size_t cnt = G.win.vals.size() / 2;
    for (size_t j = 0; j < 2 * cnt; ++j) vals[j] = (R)G.win.vals[j];
    D.n_entries = std::max<uint32_t>(used, (uint32_t)cnt);
    return;
  }
  if (e.pre) return;
  if (!e.diag) return;
  // windows overlapping the tile bits [0, m) first
  std::vector<int> order;
  for (int w = 0; w < e.win.n; ++w)
    if (e.win.shift[w] < m) order.push_back(w);
  D.n_var = (uint8_t)order.size();
  for (int w = 0; w < e.win.n; ++w)
    if (e.win.shift[w] >= m) order.push_back(w);
  D.n_win = (uint8_t)order.size();
  R* vals = reinterpret_cast<R*>(D.lut);
  uint32_t off = 0;
  for (size_t i = 0; i < order.size(); ++i) {
    const int w = order[i];
    D.shift[i] = (uint8_t)e.win.shift[w];
    D.nbits[i] = (uint8_t)e.win.nbits[w];
    D.off[i] = (uint16_t)off;
    const uint32_t cnt = 1u << e.win.nbits[w];
    for (uint32_t j = 0; j < cnt; ++j) {
      vals[2 * (off + j)] = (R)e.win.vals[2 * (e.win.off[w] + j)];
      vals[2 * (off + j) + 1] = (R)e.win.vals[2 * (e.win.off[w] + j) + 1];
    }
    off += cnt;
  }
  D.n_entries = off;
}

// Tile movement by TMA (MQ_TMA=0: per-thread asynchronous copies throughout).
bool tma_enabled() { return env_int("MQ_TMA", 1, 0, 1) == 1; }
// The fused layer's permuted write-back gathered in shared memory and
// TMA-stored (1) or stored per thread (0).
static bool tma_perm_store() { return env_int("MQ_TMA_PERM_STORE", 1, 0, 1) == 1; }
// QFT phases of four chained stages on compile-time register factors (1) or
// through the per-stage path (0).
static bool qft_full_phases() { return env_int("MQ_QFT_FULL", 1, 0, 1) == 1; }

int check_tile_fault(mq_state* h) {
  unsigned int v = 0;
  MQ_CUDA(cudaMemcpyFromSymbolAsync(&v, g_tile_fault, sizeof(v), 0, cudaMemcpyDeviceToHost, h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  bool adj = false;
  int rc = take_adj_fault(h, &adj);
  if (rc) return rc;
  if (!v && !adj) return MQ_OK;
  const unsigned int zero = 0;
  MQ_CUDA(cudaMemcpyToSymbolAsync(g_tile_fault, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  return fail(MQ_ETIMEOUT, "a tile sweep on this device abandoned its work: a tile load did not arrive within 2 s");
}

// The TMA shape of a sweep's tiles (see TmaDesc): false when it needs more
// than five dimensions or the tile lacks the low 128 bytes of its rows.
// Dimensions of size 1 above the state pad the maps to five.
bool plan_tma(int n, size_t amp_bytes, const std::vector<int>& tile_bits, TmaDesc& D) {
  const int s = amp_bytes == 16 ? 1 : 0;  // word bits below the amplitude bits (real / imaginary part)
  const int nw = n + s;
  if (nw < 4) return false;
  std::vector<bool> tb(nw, false);
  for (int w = 0; w < s; ++w) tb[w] = true;
  for (int b : tile_bits) tb[b + s] = true;
  for (int w = 0; w < 4; ++w)
    if (!tb[w]) return false;
  int nd = 0;
  auto add = [&](int w0, int len, bool tile) -> bool {
    if (nd == 5) return false;
    D.gdim[nd] = cuuint64_t(1) << len;
    D.box[nd] = tile ? (cuuint32_t(1) << len) : 1u;
    if (nd > 0) D.gstride[nd - 1] = cuuint64_t(8) << w0;
    D.start[nd] = (uint8_t)(tile ? 0 : w0 - s);
    D.mask[nd] = tile ? 0u : (uint32_t)((uint64_t(1) << len) - 1u);
    ++nd;
    return true;
  };
  add(0, 4, true);
  for (int w = 4; w < nw;) {
    const bool t = tb[w];
    int e = w;
    while (e < nw && tb[e] == t) ++e;
    if (t) {
      for (int a = w; a < e; a += 8)
        if (!add(a, std::min(8, e - a), true)) return false;
    } else if (!add(w, e - w, false)) {
      return false;
    }
    w = e;
  }
  const cuuint64_t total = cuuint64_t(8) << nw;
  while (nd < 5) {
    D.gdim[nd] = 1;
    D.box[nd] = 1;
    D.gstride[nd - 1] = total;
    D.start[nd] = 0;
    D.mask[nd] = 0;
    ++nd;
  }
  D.ndim = 5;
  D.bytes = (uint32_t)(amp_bytes << tile_bits.size());
  return true;
}

static int run_sweep(mq_state* h, Sweep& sw, const std::vector<int>& op_phase, const std::vector<int>& op_rk,
                     const EpiPlan* epi = nullptr) {
  const int m = (int)sw.tile_bits.size();
  const int lr = epi ? std::min(m, 4) : reg_bits(h->dtype, m);
  if (m < 1 || m > std::max(plan_tile_max(h), h->dtype == MQ_C64 && lr == 4 ? kTileMaxC64 : 0) || m > h->n)
    return fail(MQ_EINVAL, "bad tile size");
  if (sw.tile_bits[0] != 0) return fail(MQ_EINVAL, "tile must contain index bit 0");
  if ((int)sw.ops.size() > kMaxOps || (int)sw.phases.size() > kMaxPhases) return fail(MQ_EINVAL, "tile plan too large");
  if (epi && (epi->perm || epi->diag))
    for (int k = 0; k < m; ++k)
      if (sw.tile_bits[k] != k) return fail(MQ_EINVAL, "fused epilogue needs the low tile [0, m)");
  const bool qft = !sw.ops.empty() && (sw.ops[0].kind == OP_QFT_FWD || sw.ops[0].kind == OP_QFT_INV);
  FusedParams F;
  std::memset(&F, 0, sizeof(F));
  TileParams& P = F;
  P.n_tiles = (uint32_t)(uint64_t(1) << (h->n - m));
  P.n = (uint8_t)h->n;
  P.m = (uint8_t)m;
  P.n_phases = (uint8_t)sw.phases.size();
  P.n_ops = (uint8_t)sw.ops.size();
  for (int k = 0; k < m; ++k) P.tile_bit[k] = (uint8_t)sw.tile_bits[k];
  make_base_runs(P.runs, h->n, P.tile_bit, m);
  // TMA form for tiles of 10 bits and more whose shape it can describe.
  // Write-back: a TMA store of the tile in place (1); for a permutation that
  // keeps index bit 0 (complex64, no window diagonal), the output tile is
  // gathered in shared memory and then TMA-stored (2); otherwise per-thread
  // stores (0)
  if (tma_enabled() && m >= 10 && !sw.phases.empty() && plan_tma(h->n, h->amp_bytes(), sw.tile_bits, P.tma)) {
    if (!epi || (!epi->perm && !epi->diag)) P.tma.store = 1;
    else if (epi->perm && !epi->diag && epi->cols[0] == 1u && h->dtype == MQ_C64 && tma_perm_store()) P.tma.store = 2;
    else P.tma.store = 0;
  }
  // chunk-index bits above the thread bits: contiguous global bits?
  {
    const int cb = h->dtype == MQ_C64 ? 1 : 0;
    const int lt = (m == 12 && lr == 5) ? 7 : (m == 13 ? tile13_lt() : std::min(8, m - lr));
    const int first = cb + lt;
    bool contig = true;
    for (int b = first + 1; b < m; ++b)
      if (sw.tile_bits[b] != sw.tile_bits[b - 1] + 1) contig = false;
    P.hi_contig = (first < m && contig) ? 1 : 0;
    P.hi_shift = (uint8_t)(first < m ? sw.tile_bits[first] : 0);
  }
  // shared-memory slot of tile-local amplitude index i (the chunk swizzle
  // of k_tile applied at amplitude granularity)
  const bool c64 = h->dtype == MQ_C64;
  auto phys = [c64](uint32_t i) -> uint32_t { return c64 ? (i ^ ((i >> 3) & 0xEu)) : (i ^ ((i >> 3) & 7u)); };
  for (size_t p = 0; p < sw.phases.size(); ++p) {
    const auto& regs = sw.phases[p];
    PhaseDesc& D = P.ph[p];
    for (int k = 0; k < lr; ++k) {
      D.s_reg[k] = phys(1u << regs[k]);
      D.g_reg[k] = 1u << sw.tile_bits[regs[k]];
    }
    int j = 0;
    for (int b = 0; b < m; ++b) {
      if (std::find(regs.begin(), regs.end(), b) != regs.end()) continue;
      D.s_grp[j] = phys(1u << b);
      D.g_grp[j] = 1u << sw.tile_bits[b];
      ++j;
    }
  }
  if (qft) {
    int w = 0;
    for (size_t p = 0; p < sw.phases.size(); ++p) {
      P.ph_op[p] = (uint8_t)w;
      for (size_t o = 0; o < sw.ops.size(); ++o) {
        if (op_phase[o] != (int)p) continue;
        P.ops[w] = sw.ops[o];
        P.ops[w].phase = (uint8_t)p;
        P.ops[w].rk = (uint8_t)op_rk[o];
        ++w;
      }
    }
    P.ph_op[sw.phases.size()] = (uint8_t)w;
    // chained phases: every stage's ladder is the bits from one lad_shift up
    // to its own bit, and the stage bits are consecutive
    for (size_t p = 0; p < sw.phases.size(); ++p) {
      const int o0 = P.ph_op[p], o1 = P.ph_op[p + 1];
      if (o1 <= o0) continue;
      bool chain = true;
      int wmax = 0, gmin = 64, gmax = -1;
      for (int o = o0; o < o1 && chain; ++o) {
        const TileOp& op = P.ops[o];
        const int g = sw.tile_bits[sw.phases[p][op.rk]];
        chain = op.lad_shift == P.ops[o0].lad_shift && op.width == g - (int)op.lad_shift;
        wmax = std::max(wmax, (int)op.width);
        gmin = std::min(gmin, g);
        gmax = std::max(gmax, g);
      }
      if (chain && gmax - gmin == o1 - o0 - 1 && wmax <= 31) P.qchain[p] = (uint8_t)(wmax + 1);
      // ns = 3 or 4 stages on register slots 0 .. ns-1 of a 16-amplitude
      // phase, in the order of the direction
      const int ns = o1 - o0;
      if (P.qchain[p] && lr == 4 && (ns == 4 || ns == 3) && wmax >= ns - 1 && qft_full_phases()) {
        const bool fwd = P.ops[o0].kind == OP_QFT_FWD;
        bool full = true;
        for (int i = 0; i < ns; ++i) {
          const TileOp& op = P.ops[o0 + i];
          full = full && op.kind == P.ops[o0].kind && op.rk == (fwd ? ns - 1 - i : i) &&
                 op.width == (fwd ? wmax - i : wmax - (ns - 1) + i);
        }
        P.qfull[p] = full ? (uint8_t)ns : 0;
      }
    }
  } else {
    for (size_t o = 0; o < sw.ops.size(); ++o) {
      PhaseDesc& D = P.ph[op_phase[o]];
      const int k = op_rk[o];
      if (D.active & (1u << k)) return fail(MQ_EINVAL, "two gates on one register slot");
      D.active |= (uint8_t)(1u << k);
      if (sw.mats_dev && sw.ops[o].kind == OP_U2) P.mat_q[op_phase[o]][k] = (int16_t)(sw.ops[o].qubit + 1);
      else if (sw.ops[o].kind == OP_U2 && sw.ops[o].u[1] == 0.0 && sw.ops[o].u[3] == 0.0 && sw.ops[o].u[5] == 0.0 &&
               sw.ops[o].u[7] == 0.0)
        D.real |= (uint8_t)(1u << k);
      D.cmask[k] = sw.ops[o].kind == OP_CU2 ? sw.ops[o].cmask : 0u;
      if (D.cmask[k]) D.any_ctl = 1;
      for (int j = 0; j < 8; ++j) {
        D.ud[k][j] = sw.ops[o].u[j];
        D.uf[k][j] = (float)sw.ops[o].u[j];
      }
      const double* u = sw.ops[o].u;
      if (sw.rot && !sw.mats_dev && ((D.real >> k) & 1u) && u[0] == u[6] && u[2] == -u[4] &&
          (u[0] != 0.0 || u[4] != 0.0)) {
        const double c = u[0], sn = u[4];
        const bool b = rot_factor(c, sn) != c;
        const double t = b ? c / sn : sn / c;
        D.rot |= (uint8_t)(1u << k);
        if (b) D.rotB |= (uint8_t)(1u << k);
        D.ud[k][0] = t;
        D.uf[k][0] = (float)t;
      }
    }
  }
  if (!qft) P.mats_dev = sw.mats_dev;
  P.need_tw = (qft && sw.need_tw && h->dtype == MQ_C64) ? 1 : 0;
  P.has_scale = sw.has_scale ? 1 : 0;
  P.scale = sw.has_scale ? sw.scale : 1.0;
  size_t smem = 2 * (h->amp_bytes() << m) + (sizeof(PhaseDesc) + sizeof(uint32_t) * kThreadTabWords) * sw.phases.size();
  if (P.need_tw) {
    int rc = ensure_qft_twiddles(h);
    if (rc) return rc;
  }
  if (epi) {
    if (qft) return fail(MQ_EINVAL, "fused epilogue on a QFT sweep");
    if (h->dtype == MQ_C64) fill_epi<float>(F.epi, *epi, m, h->n);
    else fill_epi<double>(F.epi, *epi, m, h->n);
    smem += 128 + (size_t)((F.epi.n_entries + 1u) & ~1u) * h->amp_bytes();
    if (epi->perm || epi->diag) {
      if (h->dtype == MQ_C64) return dispatch_tile<float, 2>(h, F, smem, epi->perm);
      return dispatch_tile<double, 2>(h, F, smem, epi->perm);
    }
    if (h->dtype == MQ_C64) return dispatch_tile<float, 3>(h, F, smem, false);
    return dispatch_tile<double, 3>(h, F, smem, false);
  }
  if (qft) {
    QftParams Q;
    std::memset(&Q, 0, sizeof(Q));
    static_cast<TileParams&>(Q) = P;
    for (int w = 0; w < P.n_ops; ++w) {
      const TileOp& op = P.ops[w];
      const PhaseDesc& D = P.ph[op.phase];
      const uint32_t mask = op.width >= 32 ? 0xffffffffu : ((1u << op.width) - 1u);
      for (int r = 0; r < (1 << lr); ++r) {
        uint64_t Lr = 0;
        for (int k = 0; k < lr; ++k)
          if ((r >> k) & 1) Lr += (D.g_reg[k] >> op.lad_shift) & mask;
        const double ang = op.width ? M_PI * std::ldexp((double)Lr, -op.width) : 0.0;
        const double c = std::cos(ang), sn = std::sin(ang);
        Q.twf[w][r] = make_float2((float)c, (float)sn);
        Q.twd[w][r] = make_double2(c, sn);
      }
      // the kernel forms a pair's factor from its register bits below the
      // stage's slot only
      const int K = op.rk;
      for (int r = 0; r < (1 << lr); ++r) {
        const int r0 = (r & ((1 << K) - 1)) | (1 << K);
        if (((r >> K) & 1) && (Q.twd[w][r].x != Q.twd[w][r0].x || Q.twd[w][r].y != Q.twd[w][r0].y))
          return fail(MQ_EINVAL, "QFT stage with a ladder bit above its own bit");
      }
    }
    smem += (size_t)P.n_ops * 32 * h->amp_bytes();  // the register factors, staged in shared memory
    if (h->dtype == MQ_C64) return dispatch_tile<float, 1>(h, Q, smem, false);
    return dispatch_tile<double, 1>(h, Q, smem, false);
  }
  if (h->dtype == MQ_C64) return dispatch_tile<float, 0>(h, P, smem, false);
  return dispatch_tile<double, 0>(h, P, smem, false);
}

static int tile_local(const std::vector<int>& bits, int gbit) {
  for (size_t k = 0; k < bits.size(); ++k)
    if (bits[k] == gbit) return (int)k;
  return -1;
}

// Tile bits for a set of target bits: the targets, the low passengers, and
// further low bits until the tile has at least min(n, MQ_TILE_MIN) bits.
static std::vector<int> tile_for(int n, const std::vector<int>& targets, int pas, int tmax, int tmin) {
  std::vector<int> bits = targets;
  const int lowest = *std::min_element(targets.begin(), targets.end());
  for (int b = 0; b < std::min(std::max(pas, 1), lowest); ++b) bits.push_back(b);
  std::sort(bits.begin(), bits.end());
  bits.erase(std::unique(bits.begin(), bits.end()), bits.end());
  const int want = std::min({n, tmin, tmax});
  for (int b = 0; (int)bits.size() < want && b < n; ++b)
    if (std::find(bits.begin(), bits.end(), b) == bits.end()) bits.push_back(b);
  std::sort(bits.begin(), bits.end());
  return bits;
}

// Split index bits [0, n) into sweeps: the lowest group is a contiguous tile
// of up to tmax bits, every other group carries `pas` passengers and at most
// tmax - pas target bits.
static std::vector<std::pair<int, int>> split_bits(int n, int tmax, int pas) {
  std::vector<std::pair<int, int>> groups;
  if (n <= tmax) { groups.push_back({0, n}); return groups; }
  const int hi_cap = tmax - pas;
  int n_hi = (n - tmax + hi_cap - 1) / hi_cap;
  int low = std::max(n - n_hi * hi_cap, std::min(tmax, (n + n_hi) / (n_hi + 1)));
  const int want_low = env_int("MQ_SPLIT_LOW", 0, 0, tmax);
  if (want_low > 0) {
    low = want_low;
    n_hi = (n - low + hi_cap - 1) / hi_cap;
  }
  groups.push_back({0, low});
  int start = low;
  const int rest = n - low;
  for (int i = 0; i < n_hi; ++i) {
    const int cnt = rest / n_hi + (i < rest % n_hi ? 1 : 0);
    groups.push_back({start, cnt});
    start += cnt;
  }
  return groups;
}

// The U(2) sweep of index bits [start, start+cnt): targets are the active
// qubits among them.  Returns false when none is active.
static bool build_u2_sweep(mq_state* h, const double* mats, const uint8_t* active, int start, int cnt, Sweep& sw,
                           std::vector<int>& op_phase, std::vector<int>& op_rk, const double* mats_dev = nullptr,
                           int tmin = -1) {
  const int n = h->n;
  std::vector<int> gbits, qubits;
  for (int b = start + cnt - 1; b >= start; --b) {
    const int q = n - 1 - b;
    if (active && !active[q]) continue;
    gbits.push_back(b);
    qubits.push_back(q);
  }
  if (gbits.empty()) return false;
  // a caller's minimum above the planner's maximum (13-bit complex64 tiles)
  // raises the maximum with it
  const int tmax = (h->dtype == MQ_C64 && tmin > plan_tile_max(h)) ? std::min(tmin, kTileMaxC64) : plan_tile_max(h);
  sw.tile_bits = tile_for(n, gbits, plan_passengers(h), tmax, tmin > 0 ? tmin : plan_min_tile(h));
  const int m = (int)sw.tile_bits.size();
  const int lr = reg_bits(h->dtype, m);
  std::vector<int> order;
  for (int b : gbits) order.push_back(tile_local(sw.tile_bits, b));
  make_phases(m, lr, order, sw, op_phase, op_rk, env_int("MQ_PAD_FIRST", 1, 0, 1) == 1);
  for (size_t i = 0; i < order.size(); ++i) {
    TileOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = OP_U2;
    op.qubit = qubits[i];
    if (mats)
      for (int j = 0; j < 8; ++j) op.u[j] = mats[(size_t)qubits[i] * 8 + j];
    sw.ops.push_back(op);
  }
  sw.mats_dev = mats ? nullptr : mats_dev;
  return true;
}

int launch_u2_layer(mq_state* h, const double* mats, const uint8_t* active) {
  // a U(2) on every qubit takes the Euler split too (RY sweeps in tangent
  // form between the two RZ diagonals)
  if (euler_plain() && euler_enabled(h)) {
    bool all = true;
    if (active)
      for (int q = 0; q < h->n; ++q) all = all && active[q];
    if (all) return launch_layer(h, mats, nullptr, 0, nullptr, nullptr, nullptr, nullptr, 0);
  }
  for (auto [start, cnt] : split_bits(h->n, plan_tile_max(h), plan_passengers(h))) {
    Sweep sw;
    std::vector<int> op_phase, op_rk;
    if (!build_u2_sweep(h, mats, active, start, cnt, sw, op_phase, op_rk)) continue;
    int rc = run_sweep(h, sw, op_phase, op_rk);
    if (rc) return rc;
  }
  return MQ_OK;
}

// One layer of the config-0 structure in as few sweeps as the U(2) layer
// alone: U(2) on every active qubit, then the diagonal terms, then the GF(2)
// permutation (the reference runs u2_list_layer_all, zz_weighted_layer and
// xor_affine_gather as three kernels, device.py:1089-1097).  The high bit
// groups run first as plain sweeps; the low group [0, m) runs last and, as
// every other U(2) gate is applied by then, multiplies the diagonal into its
// tile and writes through the permutation when A maps span(e_0..e_{m-1})
// onto itself (CNOT ladders do).  A diagonal that does not factor into
// contiguous windows, or a permutation that mixes the low bits with high
// ones, runs as its own pass after the sweep.
// U = e^{i alpha} RZ(phi) RY(theta) RZ(lam) for a 2x2 unitary u (8 doubles).
static void zyz(const double* u, double& alpha, double& phi, double& theta, double& lam) {
  const std::complex<double> u00(u[0], u[1]), u01(u[2], u[3]), u10(u[4], u[5]), u11(u[6], u[7]);
  alpha = 0.5 * std::arg(u00 * u11 - u01 * u10);
  const std::complex<double> ph = std::polar(1.0, -alpha);
  const std::complex<double> x = u00 * ph, y = u10 * ph;  // V = e^{-i alpha} U in SU(2)
  theta = 2.0 * std::atan2(std::abs(y), std::abs(x));
  const double pa = std::abs(x) > 1e-300 ? std::arg(x) : 0.0;
  const double pb = std::abs(y) > 1e-300 ? std::arg(y) : 0.0;
  phi = pb - pa;
  lam = -pa - pb;
}


// launch_layer with every qubit's U(2) split as e^{i alpha} RZ(phi) RY(theta)
// (measured at 30 qubits: fused config layer 20.7 ms against 21.7 ms with
// complex 2x2 sweeps)
// RZ(lam): the sweeps apply only the real RY matrices (half the arithmetic of
// a complex 2x2), the product of all RZ(lam) is a diagonal applied in the
// first register phase of the first sweep (before any RY), and the product of
// all RZ(phi), the global phase and the layer's own diagonal terms ride on the
// last register phase of the low sweep.  Sets *done = false (nothing
// launched) when a diagonal does not fit the register-phase tables.
static int launch_layer_euler(mq_state* h, const double* mats, int n_terms, const int32_t* kinds,
                              const int32_t* wires, const double* params, const uint32_t* cols, uint32_t c,
                              bool* done) {
  *done = false;
  const int n = h->n;
  std::vector<double> ry((size_t)n * 8, 0.0);
  std::vector<int32_t> pre_k, pre_w, post_k(kinds, kinds + n_terms), post_w(wires, wires + 2 * n_terms);
  std::vector<double> pre_p, post_p(params, params + 8 * (size_t)n_terms);
  double alpha_sum = 0.0;
  for (int q = 0; q < n; ++q) {
    double al, ph, th, la;
    zyz(mats + (size_t)q * 8, al, ph, th, la);
    const double cs = std::cos(0.5 * th), sn = std::sin(0.5 * th);
    double* r = ry.data() + (size_t)q * 8;
    r[0] = cs; r[2] = -sn; r[4] = sn; r[6] = cs;
    alpha_sum += al;
    pre_k.push_back(MQ_DIAG_RZ); pre_w.push_back(q); pre_w.push_back(-1);
    pre_p.push_back(la); pre_p.insert(pre_p.end(), 7, 0.0);
    post_k.push_back(MQ_DIAG_RZ); post_w.push_back(q); post_w.push_back(-1);
    post_p.push_back(ph); post_p.insert(post_p.end(), 7, 0.0);
  }
  post_k.push_back(MQ_DIAG_GLOBAL); post_w.push_back(0); post_w.push_back(-1);
  post_p.push_back(alpha_sum); post_p.insert(post_p.end(), 7, 0.0);
  const auto groups = split_bits(n, plan_tile_max(h), plan_passengers(h));
  const int max_entries = kEpiLutBytes / (int)h->amp_bytes();
  // RY sweeps in tangent form: the product of the factors they leave out
  // rides on the low sweep's register diagonal
  const bool rot = rot_enabled();
  double rot_scale = 1.0;
  if (rot)
    for (int q = 0; q < n; ++q) rot_scale *= rot_factor(ry[(size_t)q * 8], ry[(size_t)q * 8 + 4]);
  Sweep low;
  std::vector<int> low_phase, low_rk;
  const int tmin = euler_min_tile();
  const bool hi13 = h->dtype == MQ_C64 && euler_hi13() && reg_bits(MQ_C64, 13) == 4;
  auto hi_tmin = [&](int cnt) { return (hi13 && cnt + 5 > tmin) ? kTileMaxC64 : tmin; };
  if (!build_u2_sweep(h, ry.data(), nullptr, groups[0].first, groups[0].second, low, low_phase, low_rk, nullptr,
                      euler_low_tile()))
    return MQ_OK;
  low.rot = rot;
  const int m = (int)low.tile_bits.size();
  if (low.phases.empty() || low.phases.back().size() != 4 || low.phases.front().size() != 4) return MQ_OK;
  EpiPlan e;
  {
    const auto& regs = low.phases.back();
    const int rb[4] = {regs[0], regs[1], regs[2], regs[3]};
    // small tables first: they share the SM's shared memory with the tile
    for (int budget : {kRegDiagSmall, max_entries}) {
      int rc = plan_diag_register(h, (int)post_k.size(), post_k.data(), post_w.data(), post_p.data(), rb, budget,
                                  e.reg);
      if (rc) return rc;
      if (e.reg.win.n >= 0) break;
    }
    if (e.reg.win.n < 0) return MQ_OK;
    e.dreg = true;
    // every amplitude takes exactly one entry of T (entries [t_off, end))
    for (size_t j = 2 * (size_t)e.reg.t_off; j < e.reg.win.vals.size(); ++j) e.reg.win.vals[j] *= rot_scale;
  }
  // the first sweep executed carries the pre diagonal
  Sweep first;
  std::vector<int> first_phase, first_rk;
  EpiPlan e_first;
  // the high sweeps commute (disjoint qubits): the one that carries the pre
  // diagonal runs first, the others follow in order
  const int pre_dflt = plan_tile_max(h) >= 13 ? (int)groups.size() - 1 : 1;
  const size_t pre_g =
      groups.size() > 1 ? (size_t)std::min<int>(euler_pre_group(std::max(1, pre_dflt)), (int)groups.size() - 1) : 0;
  const bool has_high = groups.size() > 1 &&
                        build_u2_sweep(h, ry.data(), nullptr, groups[pre_g].first, groups[pre_g].second, first,
                                       first_phase, first_rk, nullptr, hi_tmin(groups[pre_g].second));
  first.rot = rot;
  {
    const Sweep& fs = has_high ? first : low;
    if (fs.phases.empty() || fs.phases.front().size() != 4) return MQ_OK;
    int rb[4];
    for (int k = 0; k < 4; ++k) rb[k] = fs.tile_bits[fs.phases.front()[k]];
    DiagRegister& pr = has_high ? e_first.pre_reg : e.pre_reg;
    const int room = has_high ? max_entries : max_entries - (int)(e.reg.win.vals.size() / 2);
    for (int budget : {std::min(room, kRegDiagSmall / 2), room}) {
      int rc = plan_diag_register(h, (int)pre_k.size(), pre_k.data(), pre_w.data(), pre_p.data(), rb, budget, pr);
      if (rc) return rc;
      if (pr.win.n >= 0) break;
    }
    if (pr.win.n < 0) return MQ_OK;
    (has_high ? e_first.pre : e.pre) = true;
  }
  if (cols) {
    e.perm = true;
    for (int j = 0; j < m; ++j)
      if (cols[j] >> m) e.perm = false;
    if (e.perm) {
      for (int j = 0; j < n; ++j) e.cols[j] = cols[j];
      e.c = c;
      int rc = ensure_alt(h);
      if (rc) return rc;
    }
  }
  *done = true;
  if (has_high) {
    int rc = run_sweep(h, first, first_phase, first_rk, &e_first);
    if (rc) return rc;
  }
  for (size_t g = 1; g < groups.size(); ++g) {
    if (g == pre_g) continue;
    Sweep sw;
    std::vector<int> op_phase, op_rk;
    if (!build_u2_sweep(h, ry.data(), nullptr, groups[g].first, groups[g].second, sw, op_phase, op_rk, nullptr,
                        hi_tmin(groups[g].second)))
      continue;
    sw.rot = rot;
    int rc = run_sweep(h, sw, op_phase, op_rk);
    if (rc) return rc;
  }
  int rc = run_sweep(h, low, low_phase, low_rk, &e);
  if (rc) return rc;
  if (cols && !e.perm) return launch_affine_cols(h, cols, c);
  return MQ_OK;
}

int launch_layer(mq_state* h, const double* mats, const uint8_t* active, int n_terms, const int32_t* kinds,
                 const int32_t* wires, const double* params, const uint32_t* cols, uint32_t c,
                 const double* mats_dev) {
  const bool u2 = mats || mats_dev;
  const int n = h->n;
  if (cols) {
    uint32_t inv[32];
    if (!gf2_invert(n, cols, inv)) return fail(MQ_EINVAL, "affine map is not invertible over GF(2)");
  }
  // a mask with every qubit set is the whole layer (the gate-stream fusion
  // lists the active qubits even when all of them are)
  if (active) {
    bool all = true;
    for (int q = 0; q < n; ++q) all = all && active[q];
    if (all) active = nullptr;
  }
  // the split pays when the layer carries a diagonal of its own, which the
  // RZ(phi) factors join at no extra cost; with RY sweeps in tangent form it
  // pays for a bare U(2) layer as well (MQ_EULER_PLAIN)
  if (mats && !mats_dev && !active && (n_terms > 0 || euler_plain()) && euler_enabled(h)) {
    // validate the layer's own terms before anything is launched
    if (n_terms > 0) {
      DiagWindows probe;
      int rc = plan_diag_windows(h, n_terms, kinds, wires, params, 1, probe);
      if (rc) return rc;
    }
    bool done = false;
    int rc = launch_layer_euler(h, mats, n_terms, kinds, wires, params, cols, c, &done);
    if (rc || done) return rc;
  }
  const auto groups = split_bits(n, plan_tile_max(h), plan_passengers(h));
  // low sweep plan first, so that argument errors surface before any launch
  Sweep low;
  std::vector<int> low_phase, low_rk;
  const bool low_u2 = u2 && build_u2_sweep(h, mats, active, groups[0].first, groups[0].second, low, low_phase, low_rk,
                                           mats_dev);
  if (!low_u2) low.tile_bits = tile_for(n, {0}, plan_passengers(h), plan_tile_max(h), plan_min_tile(h));
  const int m = (int)low.tile_bits.size();
  EpiPlan e;
  if (n_terms > 0) {
    const int max_entries = kEpiLutBytes / (int)h->amp_bytes();
    // preferred: the diagonal in the last register phase of the low sweep
    if (low_u2 && !low.phases.empty() && low.phases.back().size() == 4 && m >= 4) {
      const auto& regs = low.phases.back();
      const int rb[4] = {regs[0], regs[1], regs[2], regs[3]};
      for (int budget : {kRegDiagSmall, max_entries}) {
        int rc = plan_diag_register(h, n_terms, kinds, wires, params, rb, budget, e.reg);
        if (rc) return rc;
        if (e.reg.win.n >= 0) break;
      }
      e.dreg = e.reg.win.n >= 0;
    }
    if (!e.dreg) {
      int rc = plan_diag_windows(h, n_terms, kinds, wires, params, max_entries, e.win);
      if (rc) return rc;
      e.diag = e.win.n > 0;
    }
  }
  const bool diag_separate = n_terms > 0 && !e.diag && !e.dreg;
  if (cols && !diag_separate) {
    e.perm = true;
    for (int j = 0; j < m; ++j)
      if (cols[j] >> m) e.perm = false;
    if (e.perm) {
      for (int j = 0; j < n; ++j) e.cols[j] = cols[j];
      e.c = c;
      int rc = ensure_alt(h);
      if (rc) return rc;
    }
  }
  if (u2) {
    for (size_t g = 1; g < groups.size(); ++g) {
      Sweep sw;
      std::vector<int> op_phase, op_rk;
      if (!build_u2_sweep(h, mats, active, groups[g].first, groups[g].second, sw, op_phase, op_rk, mats_dev)) continue;
      int rc = run_sweep(h, sw, op_phase, op_rk);
      if (rc) return rc;
    }
  }
  if (low_u2 || e.diag || e.perm || e.dreg) {
    int rc = run_sweep(h, low, low_phase, low_rk, (e.diag || e.perm || e.dreg) ? &e : nullptr);
    if (rc) return rc;
  }
  if (diag_separate) {
    int rc = launch_diag_terms(h, n_terms, kinds, wires, params);
    if (rc) return rc;
  }
  if (cols && !e.perm) return launch_affine_cols(h, cols, c);
  return MQ_OK;
}

// Stages [j_begin, j_end) of the QFT on qubits [q0, q0+k), first qubit = most
// significant logical bit (sim.py:522-563 with wires = range(q0, q0+k); a
// single stage is qft_stage_sub of qft.py:144-181).  Forward stages run in
// increasing j (descending index bit), inverse stages in decreasing j.
int launch_qft_stages(mq_state* h, int q0, int k, int j_begin, int j_end, int inverse) {
  const int n = h->n;
  if (k <= 0 || j_begin >= j_end) return MQ_OK;
  if (q0 < 0 || q0 + k > n || j_begin < 0 || j_end > k) return fail(MQ_EINVAL, "invalid QFT stage range");
  const int tmax = plan_tile_max(h);
  const int pas = plan_passengers(h);
  const int lad_shift = n - q0 - k;  // index bit of the last wire
  // stage j acts on bit b_j = n-1-q0-j.  Groups of consecutive stages: the
  // lowest group may reach bit 0 (tmax bits), the others hold tmax - pas.
  const int count = j_end - j_begin;
  const int blo_all = n - 1 - q0 - (j_end - 1);
  std::vector<std::pair<int, int>> groups;  // [j0, cnt)
  {
    const int cap_hi = std::max(1, tmax - pas);
    const int cap_lo = (blo_all < pas) ? std::max(1, tmax - blo_all) : cap_hi;
    int n_groups = 1;
    while (cap_lo + (n_groups - 1) * cap_hi < count) ++n_groups;
    int remaining = count;
    int j0 = j_begin;
    for (int g = 0; g < n_groups; ++g) {
      const int left = n_groups - g;
      int cnt = remaining;
      if (left > 1) {
        cnt = std::min(cap_hi, (remaining + left - 1) / left);
        // what stays must still fit the remaining groups
        cnt = std::max(cnt, remaining - (cap_lo + (left - 2) * cap_hi));
      }
      groups.push_back({j0, cnt});
      j0 += cnt;
      remaining -= cnt;
    }
  }
  if (inverse) std::reverse(groups.begin(), groups.end());
  for (auto [j0, cnt] : groups) {
    std::vector<int> stages;
    if (!inverse) for (int j = j0; j < j0 + cnt; ++j) stages.push_back(j);
    else for (int j = j0 + cnt - 1; j >= j0; --j) stages.push_back(j);
    std::vector<int> gbits;
    for (int j : stages) gbits.push_back(n - 1 - q0 - j);
    Sweep sw;
    sw.tile_bits = tile_for(n, gbits, pas, tmax, plan_min_tile(h));
    const int m = (int)sw.tile_bits.size();
    if (m > tmax) return fail(MQ_EINVAL, "qft tile too large");
    const int lr = reg_bits(h->dtype, m);
    std::vector<int> order;
    for (int b : gbits) order.push_back(tile_local(sw.tile_bits, b));
    std::vector<int> op_phase, op_rk;
    make_phases(m, lr, order, sw, op_phase, op_rk);
    for (size_t i = 0; i < order.size(); ++i) {
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = inverse ? OP_QFT_INV : OP_QFT_FWD;
      op.lad_shift = (uint8_t)lad_shift;
      op.width = (uint8_t)(k - 1 - stages[i]);
      if (op.width) sw.need_tw = true;
      sw.ops.push_back(op);
    }
    // 2^{-cnt/2}: exact power of two for even counts
    sw.scale = std::ldexp(1.0, -(cnt / 2)) * ((cnt & 1) ? 0.70710678118654752440 : 1.0);
    sw.has_scale = true;
    int rc = run_sweep(h, sw, op_phase, op_rk);
    if (rc) return rc;
  }
  return MQ_OK;
}

int launch_qft_contiguous(mq_state* h, int q0, int k, int inverse) {
  return launch_qft_stages(h, q0, k, 0, k, inverse);
}

// Controlled single-qubit gates (CH/CRX/CRY, Toffoli as doubly controlled X;
// controlled_single.py:18-134, sim.py:140-213).  Consecutive gates whose wire
// sets are pairwise disjoint commute and share one sweep; any other gate
// starts a new sweep, so the list order is respected.
int launch_cu2_list(mq_state* h, int n_gates, const int32_t* targets, const uint32_t* cmasks, const double* mats) {
  const int n = h->n;
  const int tmax = plan_tile_max(h);
  const int pas = plan_passengers(h);
  int g = 0;
  while (g < n_gates) {
    std::vector<int> members;
    uint32_t used = 0;
    while (g < n_gates && (int)members.size() < std::max(1, tmax - pas)) {
      const int tb = n - 1 - targets[g];
      const uint32_t sup = cmasks[g] | (1u << tb);
      if (used & sup) break;
      used |= sup;
      members.push_back(g);
      ++g;
    }
    std::vector<int> gbits;
    for (int i : members) gbits.push_back(n - 1 - targets[i]);
    Sweep sw;
    sw.tile_bits = tile_for(n, gbits, pas, tmax, plan_min_tile(h));
    const int m = (int)sw.tile_bits.size();
    if (m > tmax) return fail(MQ_EINVAL, "controlled-gate tile too large");
    const int lr = reg_bits(h->dtype, m);
    std::vector<int> order;
    for (int b : gbits) order.push_back(tile_local(sw.tile_bits, b));
    std::vector<int> op_phase, op_rk;
    make_phases(m, lr, order, sw, op_phase, op_rk);
    for (size_t i = 0; i < members.size(); ++i) {
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = OP_CU2;
      op.cmask = cmasks[members[i]];
      for (int j = 0; j < 8; ++j) op.u[j] = mats[(size_t)members[i] * 8 + j];
      sw.ops.push_back(op);
    }
    int rc = run_sweep(h, sw, op_phase, op_rk);
    if (rc) return rc;
  }
  return MQ_OK;
}

}  // namespace mq
