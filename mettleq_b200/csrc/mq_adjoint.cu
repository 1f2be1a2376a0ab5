// Adjoint-method gradients (the differentiation direction of the engine).
//
// The reference differentiates by parameter shift: two full circuit runs per
// parameter (integrations/qml.py:308-332).  The adjoint method needs one
// forward run, one application of the observable and one backward run that
// un-applies the circuit from the final state, so no intermediate states are
// stored:
//
//   psi = U_L ... U_1 |0>,  lam = H psi,  E = Re <psi|lam>
//   backward, for every gate U = exp(-i t G / 2) from the last to the first:
//     dE/dt = Im <lam|G|psi>       (psi, lam taken right after U)
//     psi <- U^dag psi,  lam <- U^dag lam
//
// Gates of one layer act on different qubits and commute, and a unitary
// applied to both psi and lam leaves <lam|G_q|psi> unchanged when it acts on
// other qubits, so a whole layer is handled by tile sweeps over index-bit
// groups (as the U(2) layer): k_adj streams tiles of psi and lam through
// shared memory together and, for every target qubit, accumulates the three
// transition values Im <lam|P_q|psi> (P = X, Y, Z) and then un-applies the
// qubit's whole rotation product U_q in one 2x2 step.  The gradient of any
// rotation inside U_q is a real combination of the three: for
// U_q = R_{K-1} ... R_0 and R_k = exp(-i t G / 2), taken at the point after
// U_q, dE/dt_k = Im <lam| V G V^dag |psi> with V = R_{K-1} ... R_{k+1}, and
// V G V^dag = a X + b Y + c Z (the host forms a, b, c).
//
//   k_hdiag: lam = D psi for the Z-word part of H (one pass)
//   k_adj (build mode): lam += sum_q c_q X_q psi (tile sweeps)
//   k_dot:   E = Re <psi|lam> (one pass)
//   k_adj (backward mode): gradients + un-apply, per layer
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

enum : uint8_t { SLOT_NONE = 0, SLOT_MEASURE = 1, SLOT_XADD = 2 };

constexpr int kAdjLR = 4;           // register bits per phase, complex64 (complex128: 3)
constexpr int kAdjMaxPhases = 4;    // up to 12 target bits per sweep
constexpr int kAdjTileMax = 11;     // psi and lam tiles, double-buffered: 4 * 2^11 * 8 B (complex64)
constexpr int kAdjSlots = kAdjMaxPhases * kAdjLR;
constexpr int kAdjPartials = 3 * kAdjSlots;  // per block: Im <lam|X,Y,Z|psi> per slot
constexpr int kAdjMaxTargets = 12;

struct AdjSlot {
  uint8_t mode;        // SLOT_MEASURE: transition values, then un-apply u
  uint8_t has_u;       // u is not the identity
  uint8_t pad[6];
  alignas(16) float uf[8];
  alignas(16) double ud[8];  // SLOT_XADD: ud[0] = coefficient of X_q
};

struct AdjPhase {
  uint32_t s_reg[kAdjLR];
  uint32_t s_grp[16];
  AdjSlot slot[kAdjLR];
};

struct AdjParams {
  TmaDesc tma;  // TMA form: src = psi, dst = lam (both swept in place)
  uint32_t n_tiles;
  uint8_t n, m, n_phases, store_psi;
  uint8_t tile_bit[16];
  uint8_t hi_contig, hi_shift, pad[6];
  BaseRuns runs;  // tile index -> base index (deposit_runs)
  AdjPhase ph[kAdjMaxPhases];
  // A GF(2) map un-applied on load (TMA form, low tile [0, M)): output
  // amplitude x of both states is input amplitude perm_c ^ A x, A given by
  // its columns; A maps the low tile onto itself, so output tile t reads the
  // input tile of A (t << M) ^ perm_c whole (htab: A of the tile index's
  // bytes, as EpiDesc).  The outputs go to the states' second buffers
  // (out[0]: psi, out[1]: lam).
  uint8_t perm, pad2[3];
  uint32_t perm_c;
  uint32_t cols[32];
  uint32_t htab[768];
  CUtensorMap out[2];
};

template <typename R>
__device__ __forceinline__ V2<R> slot_u(const AdjSlot& S, int j) {
  if constexpr (sizeof(R) == 4) return make_float2(S.uf[2 * j], S.uf[2 * j + 1]);
  else return make_double2(S.ud[2 * j], S.ud[2 * j + 1]);
}

template <typename T>
__device__ __forceinline__ T cmac(T u0, T x0, T u1, T x1) {
  T r;
  r.x = fma(u0.x, x0.x, fma(-u0.y, x0.y, fma(u1.x, x1.x, -u1.y * x1.y)));
  r.y = fma(u0.x, x0.y, fma(u0.y, x0.x, fma(u1.x, x1.y, u1.y * x1.x)));
  return r;
}

// complex64 form of the SLOT_MEASURE step on the paired FP32 instructions.
// With s = (x.y, x.x) the swapped amplitude (formed once per pair and shared
// by both parts), the products of both components of a pair sit in one
// paired FMA:
//   Im conj(l) x = (l (.) s).x - (l (.) s).y,  Re conj(l) x = (l (.) x).x + (l (.) x).y,
// so gx, gy, gz are paired partial sums folded at the end.  The un-apply
// u0 x0 + u1 x1 is x0 (.) (u0.x, u0.x) + s0 (.) (-u0.y, u0.y) + x1 (.) (u1.x, u1.x)
// + s1 (.) (-u1.y, u1.y), chained in the order of cmac, so each lane takes
// the rounding steps of the scalar form.
template <int LR, int K>
__device__ __forceinline__ void adj_slot_c64(float2 (&a)[1 << LR], float2 (&b)[1 << LR], const AdjSlot& S,
                                             float (&acc)[3]) {
  auto swp = [](float2 v) { return make_float2(v.y, v.x); };
  auto neg = [](float2 v) { return make_float2(-v.x, -v.y); };
  float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax;
  const bool has_u = S.has_u;
  float2 U[4][2];  // per matrix entry: (u.x, u.x), (-u.y, u.y)
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float ux = S.uf[2 * j], uy = S.uf[2 * j + 1];
    U[j][0] = make_float2(ux, ux);
    U[j][1] = make_float2(-uy, uy);
  }
  auto apply = [&](float2 x0, float2 s0, float2 x1, float2 s1, int row) {
    const float2* u0 = U[2 * row];
    const float2* u1 = U[2 * row + 1];
    return __ffma2_rn(x0, u0[0], __ffma2_rn(s0, u0[1], __ffma2_rn(x1, u1[0], __fmul2_rn(s1, u1[1]))));
  };
#pragma unroll
  for (int r = 0; r < (1 << LR); ++r) {
    if (r & (1 << K)) continue;
    const int r1 = r | (1 << K);
    const float2 x0 = a[r], x1 = a[r1], l0 = b[r], l1 = b[r1];
    const float2 s0 = swp(x0), s1 = swp(x1);
    az = __ffma2_rn(l0, s0, az);
    az = __ffma2_rn(neg(l1), s1, az);
    ay = __ffma2_rn(l1, x0, ay);
    ay = __ffma2_rn(neg(l0), x1, ay);
    ax = __ffma2_rn(l0, s1, ax);
    ax = __ffma2_rn(l1, s0, ax);
    if (has_u) {
      a[r] = apply(x0, s0, x1, s1, 0);
      a[r1] = apply(x0, s0, x1, s1, 1);
      const float2 t0 = swp(l0), t1 = swp(l1);
      b[r] = apply(l0, t0, l1, t1, 0);
      b[r1] = apply(l0, t0, l1, t1, 1);
    }
  }
  acc[0] += ax.x - ax.y;
  acc[1] += ay.x + ay.y;
  acc[2] += az.x - az.y;
}

// Register bit K: transition values Im <lam|P|psi> for P = X, Y, Z over the
// thread's pairs (SLOT_MEASURE), then the 2x2 un-apply on both register
// sets; SLOT_XADD adds c X_q psi to lam instead.
template <typename R, int LR, int K>
__device__ __forceinline__ void adj_slot(V2<R> (&a)[1 << LR], V2<R> (&b)[1 << LR], const AdjSlot& S,
                                         R (&acc)[3]) {
  using T = V2<R>;
  if constexpr (sizeof(R) == 4) {
    if (S.mode == SLOT_MEASURE) {
      adj_slot_c64<LR, K>(a, b, S, acc);
      return;
    }
  }
  if (S.mode == SLOT_MEASURE) {
    R gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int r = 0; r < (1 << LR); ++r) {
      if (r & (1 << K)) continue;
      const T x0 = a[r], x1 = a[r | (1 << K)], l0 = b[r], l1 = b[r | (1 << K)];
      gz += (l0.x * x0.y - l0.y * x0.x) - (l1.x * x1.y - l1.y * x1.x);
      gy += (l1.x * x0.x + l1.y * x0.y) - (l0.x * x1.x + l0.y * x1.y);
      gx += (l0.x * x1.y - l0.y * x1.x) + (l1.x * x0.y - l1.y * x0.x);
    }
    acc[0] += gx;
    acc[1] += gy;
    acc[2] += gz;
    if (S.has_u) {
      const T u00 = slot_u<R>(S, 0), u01 = slot_u<R>(S, 1), u10 = slot_u<R>(S, 2), u11 = slot_u<R>(S, 3);
#pragma unroll
      for (int r = 0; r < (1 << LR); ++r) {
        if (r & (1 << K)) continue;
        const int r1 = r | (1 << K);
        const T x0 = a[r], x1 = a[r1];
        a[r] = cmac(u00, x0, u01, x1);
        a[r1] = cmac(u10, x0, u11, x1);
        const T y0 = b[r], y1 = b[r1];
        b[r] = cmac(u00, y0, u01, y1);
        b[r1] = cmac(u10, y0, u11, y1);
      }
    }
  } else if (S.mode == SLOT_XADD) {
    const R c = (R)S.ud[0];
#pragma unroll
    for (int r = 0; r < (1 << LR); ++r) {
      if (r & (1 << K)) continue;
      const T x0 = a[r], x1 = a[r | (1 << K)];
      b[r] = caxpy(c, x1, b[r]);
      b[r | (1 << K)] = caxpy(c, x0, b[r | (1 << K)]);
    }
  }
}

template <int LR>
__device__ __forceinline__ uint32_t xsel(int r, const uint32_t* g) {
  uint32_t o = 0;
#pragma unroll
  for (int k = 0; k < LR; ++k)
    if (r & (1 << k)) o ^= g[k];
  return o;
}

// set when an adjoint sweep was abandoned (read and cleared by mq_sync)
__device__ unsigned int g_adj_fault;

// Tiles of 2^M amplitudes of psi and lam, 2^LT threads, shared-memory layout
// as k_tile (chunk c at slot c ^ ((c >> 3) & 7)); per-block gradient partials
// (one double per phase slot and step) go to `partials`.  TMA: thread 0 loads
// a tile of both states as two boxes completing on one mbarrier per buffer
// pair, and writes them back as two TMA stores; every wait is bounded
// (kTmaWaitNs), and a CTA whose tile does not arrive sets g_adj_fault and
// returns as a whole.
template <typename R, int M, int LR, int LT, bool TMA>
__global__ void __launch_bounds__(1 << LT)
k_adj(V2<R>* psi, V2<R>* lam, const __grid_constant__ AdjParams P, double* __restrict__ partials) {
  using T = V2<R>;
  constexpr int NT = 1 << LT;
  constexpr int NR = 1 << LR;
  constexpr int E = 1 << M;
  constexpr int GPT = (E / NR) / NT;
  constexpr int CB = sizeof(T) == 8 ? 1 : 0;
  constexpr int NCH = E >> CB;
  constexpr int CPT = NCH / NT;
  constexpr int LCH = (M - CB) - LT;
  static_assert(GPT >= 1 && CPT >= 1, "bad tile configuration");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // TMA: buffers on a 1024-byte boundary (the 128-byte swizzle), then the two
  // mbarriers (the host adds the slack)
  unsigned char* smem = smem_raw;
  if constexpr (TMA) smem += (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  T* bufs = reinterpret_cast<T*>(smem);  // [psi0, psi1, lam0, lam1]
  const uint32_t bar0 = smem_u32(smem + 4 * sizeof(T) * E);
  constexpr int WS = NT < 32 ? NT : 32;  // lanes per warp in use
  constexpr unsigned WMASK = WS == 32 ? 0xffffffffu : ((1u << WS) - 1u);
  __shared__ double red[(NT + 31) / 32][kAdjPartials];
  const int tid = threadIdx.x;
  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(bar0, 1);
      mbar_init(bar0 + 8u, 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  uint32_t g_t = 0;
#pragma unroll
  for (int b = 0; b < LT; ++b)
    if ((tid >> b) & 1) g_t |= 1u << P.tile_bit[CB + b];
  const uint32_t s_t = (uint32_t)tid ^ (((uint32_t)tid >> 3) & 7u);
  auto slot = [&](int k) -> uint32_t {
    const uint32_t kk = (uint32_t)(k * NT);
    return s_t ^ (kk ^ ((kk >> 3) & 7u));
  };
  auto g_k = [&](int k) -> uint32_t {
    if (P.hi_contig) return (uint32_t)k << P.hi_shift;
    uint32_t g = 0;
#pragma unroll
    for (int b = 0; b < LCH; ++b)
      if ((k >> b) & 1) g |= 1u << P.tile_bit[CB + LT + b];
    return g;
  };
  auto base_of = [&](uint32_t tile) -> uint32_t { return deposit_runs(tile, P.runs); };
  // GF(2) map on load: the input tile of output tile t (its base) and the
  // low offset perm_c ^ A (t << M) leaves inside it; A applied to the thread
  // part of this thread's chunks (c = tid + k*NT -> amplitude c << CB)
  auto src_base = [&](uint32_t t, uint32_t& lo) -> uint32_t {
    lo = 0;
    if (!P.perm) return base_of(t);
    const uint32_t b = P.perm_c ^ P.htab[t & 255u] ^ P.htab[256 + ((t >> 8) & 255u)] ^ P.htab[512 + ((t >> 16) & 255u)];
    lo = b & (uint32_t)(E - 1);
    return b & ~(uint32_t)(E - 1);
  };
  uint32_t perm_at = 0;
  if (P.perm) {
#pragma unroll
    for (int b = 0; b < LT; ++b)
      if ((tid >> b) & 1) perm_at ^= P.cols[CB + b];
  }
  // one state's tile gathered in place: chunk c takes input amplitudes
  // lo ^ A (c << CB) (complex64: the pair there, swapped when A flips bit 0;
  // A e_0 = e_0 keeps pairs whole)
  auto gather = [&](T* buf, uint32_t lo) {
    float4* c4 = reinterpret_cast<float4*>(buf);
    float4 v[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      uint32_t l = lo ^ perm_at;
#pragma unroll
      for (int b = 0; b < LCH; ++b)
        if ((k >> b) & 1) l ^= P.cols[CB + LT + b];
      const uint32_t ch = l >> CB;
      const float4 w = c4[ch ^ ((ch >> 3) & 7u)];
      v[k] = (CB == 1 && (l & 1u)) ? make_float4(w.z, w.w, w.x, w.y) : w;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < CPT; ++k) c4[slot(k)] = v[k];
  };
  auto issue = [&](uint32_t tile, int which) {
    const uint32_t gb = base_of(tile) | g_t;
    const uint32_t sp = smem_u32(bufs + which * E), sl = smem_u32(bufs + (2 + which) * E);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      cp_async<16>(sp + 16u * slot(k), psi + (gb | g_k(k)));
      cp_async<16>(sl + 16u * slot(k), lam + (gb | g_k(k)));
    }
  };
  // per-thread gradient sums over this thread's tiles, in the state's type
  // (a few dozen terms each); blocks reduce them in double
  constexpr int MAXPH = (12 + LR - 1) / LR < kAdjMaxPhases ? (12 + LR - 1) / LR : kAdjMaxPhases;
  static_assert(MAXPH <= kAdjMaxPhases, "too many phases");
  R acc[MAXPH][LR][3];
#pragma unroll
  for (int p = 0; p < MAXPH; ++p)
#pragma unroll
    for (int k = 0; k < LR; ++k) acc[p][k][0] = acc[p][k][1] = acc[p][k][2] = 0;

  // TMA (thread 0): the tile's psi and lam boxes into buffer pair `which`
  auto tma_coords = [&](uint32_t base, int32_t (&c)[5]) {
#pragma unroll
    for (int d = 0; d < 5; ++d) c[d] = (int32_t)((base >> P.tma.start[d]) & P.tma.mask[d]);
  };
  auto tma_issue = [&](uint32_t tile, int which) {
    int32_t c[5];
    uint32_t lo;
    tma_coords(src_base(tile, lo), c);
    const uint32_t bar = bar0 + 8u * (uint32_t)which;
    mbar_expect_tx(bar, 2u * P.tma.bytes);
    tma_load_5d(smem_u32(bufs + which * E), &P.tma.src, c, bar);
    tma_load_5d(smem_u32(bufs + (2 + which) * E), &P.tma.dst, c, bar);
  };

  uint32_t tile = blockIdx.x;
  if constexpr (TMA) {
    if (tid == 0 && tile < P.n_tiles) tma_issue(tile, 0);
  } else {
    if (tile < P.n_tiles) issue(tile, 0);
    cp_async_commit();
  }
  T a[NR], b[NR];
  for (int it = 0; tile < P.n_tiles; tile += gridDim.x, ++it) {
    const int cb = it & 1;
    T* cp = bufs + cb * E;
    T* cl = bufs + (2 + cb) * E;
    const uint32_t next = tile + gridDim.x;
    if constexpr (TMA) {
      const uint32_t bar = bar0 + 8u * (uint32_t)cb;
      const uint32_t parity = (uint32_t)((it >> 1) & 1);
      const bool ok = mbar_wait_bounded(bar, parity, kTmaWaitNs);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicOr(&g_adj_fault, 1u);
          mbar_wait_bounded(bar, parity, kTmaWaitNs);  // the load in flight, once more
          bulk_wait_all();
        }
        return;
      }
      if (P.perm) {
        uint32_t lo;
        (void)src_base(tile, lo);
        gather(cp, lo);  // each gather reads its buffer, waits, then writes it
        gather(cl, lo);
        __syncthreads();
      }
    } else {
      if (next < P.n_tiles) issue(next, cb ^ 1);
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
    }
#pragma unroll
    for (int ph = 0; ph < MAXPH; ++ph) {
      if (ph >= P.n_phases) break;
      const AdjPhase& D = P.ph[ph];
      uint32_t sreg[LR];
#pragma unroll
      for (int k = 0; k < LR; ++k) sreg[k] = D.s_reg[k];
#pragma unroll
      for (int g = 0; g < GPT; ++g) {
        const uint32_t q = (uint32_t)tid + (uint32_t)g * NT;
        uint32_t sq = 0;
#pragma unroll
        for (int j = 0; j < M - LR; ++j)
          if ((q >> j) & 1) sq ^= D.s_grp[j];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          a[r] = cp[sq ^ xsel<LR>(r, sreg)];
          b[r] = cl[sq ^ xsel<LR>(r, sreg)];
        }
        adj_slot<R, LR, 0>(a, b, D.slot[0], acc[ph][0]);
        if constexpr (LR > 1) adj_slot<R, LR, 1>(a, b, D.slot[1], acc[ph][1]);
        if constexpr (LR > 2) adj_slot<R, LR, 2>(a, b, D.slot[2], acc[ph][2]);
        if constexpr (LR > 3) adj_slot<R, LR, 3>(a, b, D.slot[3], acc[ph][3]);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          if (P.store_psi) cp[sq ^ xsel<LR>(r, sreg)] = a[r];
          cl[sq ^ xsel<LR>(r, sreg)] = b[r];
        }
      }
      // TMA: the tile's last shared-memory writes become visible to the
      // async proxy (the stores that read them, the load that overwrites)
      if constexpr (TMA)
        if (ph == P.n_phases - 1) fence_proxy_async_smem();
      __syncthreads();
      if constexpr (TMA) {
        // every thread has finished the previous tile: its buffer pair takes
        // this CTA's next tile once the stores from it have read it out
        if (ph == 0 && tid == 0 && next < P.n_tiles) {
          bulk_wait_read();
          tma_issue(next, cb ^ 1);
        }
      }
    }
    if constexpr (TMA) {
      if (tid == 0) {
        int32_t c[5];
        tma_coords(base_of(tile), c);
        if (P.perm) {
          tma_store_5d(&P.out[0], c, smem_u32(cp));
          tma_store_5d(&P.out[1], c, smem_u32(cl));
        } else {
          if (P.store_psi) tma_store_5d(&P.tma.src, c, smem_u32(cp));
          tma_store_5d(&P.tma.dst, c, smem_u32(cl));
        }
        bulk_commit();
      }
      continue;
    }
    const uint32_t gb = base_of(tile) | g_t;
    const float4* p4 = reinterpret_cast<const float4*>(cp);
    const float4* l4 = reinterpret_cast<const float4*>(cl);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      if (P.store_psi) *reinterpret_cast<float4*>(psi + (gb | g_k(k))) = p4[slot(k)];
      *reinterpret_cast<float4*>(lam + (gb | g_k(k))) = l4[slot(k)];
    }
    __syncthreads();
  }
  if constexpr (TMA) {
    if (tid == 0) bulk_wait_all();  // the last stores have written global memory
  } else {
    cp_async_wait<0>();
  }
  // deterministic block reduction: lanes (xor tree), then warps in order
  const int lane = tid & 31, warp = tid >> 5;
  for (int j = tid; j < (NT + 31) / 32 * kAdjPartials; j += NT) (&red[0][0])[j] = 0.0;
  __syncthreads();
#pragma unroll
  for (int p = 0; p < MAXPH; ++p)
#pragma unroll
    for (int k = 0; k < LR; ++k)
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        double v = (double)acc[p][k][s];
#pragma unroll
        for (int off = WS / 2; off; off >>= 1) v = __dadd_rn(v, __shfl_xor_sync(WMASK, v, off));
        if (lane == 0) red[warp][(p * kAdjLR + k) * 3 + s] = v;
      }
  __syncthreads();
  for (int j = tid; j < kAdjPartials; j += NT) {
    double v = 0.0;
    for (int w = 0; w < (NT + 31) / 32; ++w) v = __dadd_rn(v, red[w][j]);
    partials[(size_t)j * gridDim.x + blockIdx.x] = v;  // value-major: the collect reads runs
  }
}

// lam_x = d(x) psi_x with d(x) = sum_w c_w (-1)^popcount(x & z_w).
// Words whose support lies within 8 consecutive index bits are summed on the
// host into window tables: tab[k][v] = sum over the window's words of
// c_w (-1)^popcount(v & (z_w >> shift_k)), so d(x) = base + sum_k
// tab[k][(x >> shift_k) & 255] + the remaining (wider) words one by one.  An
// Ising chain's ZZ terms then cost one shared-memory read per window instead
// of a popcount per term, and the pass runs at memory speed.
constexpr int kHZWords = 64;
constexpr int kHTab = 8;  // window tables of 256 entries
struct HDiagParams {
  uint32_t dim;
  int32_t nz;          // words evaluated one by one
  uint32_t z[kHZWords];
  double c[kHZWords];
  int32_t ntab;        // window tables
  uint8_t shift[kHTab];
  double base;         // words without a Z factor
  double tab[kHTab][256];
};

template <typename R>
__global__ void __launch_bounds__(256) k_hdiag(const V2<R>* __restrict__ psi, V2<R>* __restrict__ lam,
                                               const __grid_constant__ HDiagParams P) {
  __shared__ R tab[kHTab * 256];
  for (int j = threadIdx.x; j < P.ntab * 256; j += blockDim.x) tab[j] = (R)P.tab[j >> 8][j & 255];
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.dim; i += stride) {
    R d = (R)P.base;
    for (int k = 0; k < P.ntab; ++k) d += tab[k * 256 + ((i >> P.shift[k]) & 255u)];
    for (int w = 0; w < P.nz; ++w) d += (__popc(i & P.z[w]) & 1) ? -(R)P.c[w] : (R)P.c[w];
    const V2<R> v = psi[i];
    lam[i] = mk<R>(d * v.x, d * v.y);
  }
}

// per-block partial sums of Re <psi|lam> (fixed order)
template <typename R>
__global__ void __launch_bounds__(256) k_dot(const V2<R>* __restrict__ psi, const V2<R>* __restrict__ lam,
                                             uint32_t dim, double* __restrict__ partials) {
  __shared__ double red[8];
  double acc = 0.0;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
    const V2<R> p = psi[i], l = lam[i];
    acc = __dadd_rn(acc, __dadd_rn(__dmul_rn((double)p.x, (double)l.x), __dmul_rn((double)p.y, (double)l.y)));
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = __dadd_rn(v, red[w]);
    partials[blockIdx.x] = v;
  }
}

// out[index[j/3]*3 + j%3] = sum over blocks b of partials[j][b] (a fixed
// order) for every (slot, Pauli) j whose slot carries a target.
struct AdjCollect {
  int32_t index[kAdjSlots];
};
// One block per value j (partials[j * nblocks + b]): each thread sums a
// strided set of blocks in increasing b, then a fixed halving tree; the
// order depends only on nblocks, so results are reproducible.
constexpr int kCollectThreads = 128;
__global__ void __launch_bounds__(kCollectThreads)
k_adj_collect(const double* __restrict__ partials, uint32_t nblocks, const __grid_constant__ AdjCollect C,
              double* __restrict__ out) {
  const int j = blockIdx.x;
  const int t = C.index[j / 3];
  if (t < 0) return;  // the whole block: j is uniform
  __shared__ double red[kCollectThreads];
  double v = 0.0;
  const double* p = partials + (size_t)j * nblocks;
  for (uint32_t b = threadIdx.x; b < nblocks; b += kCollectThreads) v = __dadd_rn(v, p[b]);
  red[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = kCollectThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[t * 3 + j % 3] = red[0];
}

// ================================================================ host side
static uint32_t adj_phys(bool c64, uint32_t i) { return c64 ? (i ^ ((i >> 3) & 0xEu)) : (i ^ ((i >> 3) & 7u)); }

// One sweep: tile bits and, for each target (global index bit), its two steps.
struct AdjTarget {
  int bit;
  uint8_t mode, has_u;
  double u[8];
};

int take_adj_fault(mq_state* h, bool* fault) {
  unsigned int v = 0;
  MQ_CUDA(cudaMemcpyFromSymbolAsync(&v, g_adj_fault, sizeof(v), 0, cudaMemcpyDeviceToHost, h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  *fault = v != 0;
  if (v) {
    const unsigned int zero = 0;
    MQ_CUDA(cudaMemcpyToSymbolAsync(g_adj_fault, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
  }
  return MQ_OK;
}

template <typename R, int M, int LR, int LT, bool TMA>
static int launch_adj_t(mq_state* psi, mq_state* lam, const AdjParams& P0, double* partials, uint32_t* grid_out) {
  auto kern = k_adj<R, M, LR, LT, TMA>;
  size_t smem = 4 * sizeof(V2<R>) * (size_t(1) << M);
  AdjParams P = P0;
  if constexpr (TMA) {
    smem += 1024 + 64;  // 1024-byte alignment of the buffers, the mbarriers
    int rc = encode_tile_maps(P.tma, psi->cur_buf(), lam->cur_buf());
    if (rc) return rc;
    if (P.perm) {  // the outputs: both states' second buffers
      TmaDesc o = P.tma;
      rc = encode_tile_maps(o, psi->buf[1 - psi->cur], lam->buf[1 - lam->cur]);
      if (rc) return rc;
      P.out[0] = o.src;
      P.out[1] = o.dst;
    }
  }
  // one shared-memory size per instance: configure it once
  static std::mutex mu;
  static int configured = -1, bps_cached = 0;
  int bps = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    if ((int)smem > configured) {
      MQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
      configured = (int)std::max<size_t>(smem, 48 * 1024);
      MQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_cached, kern, 1 << LT, smem));
    }
    bps = bps_cached;
  }
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(P.n_tiles, (uint64_t)psi->num_sms * std::max(1, bps)));
  kern<<<grid, 1 << LT, smem, psi->stream>>>(reinterpret_cast<V2<R>*>(psi->cur_buf()),
                                             reinterpret_cast<V2<R>*>(lam->cur_buf()), P, partials);
  MQ_LAUNCHED("k_adj");
  psi->launches += 1;
  psi->sweeps += 2;
  *grid_out = grid;
  return MQ_OK;
}

// Register bits per phase.  complex64: 4 (one phase fewer per sweep; with
// the paired-FP32 slot a 16-amplitude phase fits 3 CTAs of 128 threads per
// SM, and the 24-qubit gradient measured 5.55 against 5.66 ms with 3);
// MQ_ADJ_LR=3 selects 3.  complex128: 3.
static int adj_lr(int dtype) {
  if (dtype != MQ_C64) return 3;
  const char* v = std::getenv("MQ_ADJ_LR");
  return (v && std::atoi(v) == 3) ? 3 : 4;
}

template <typename R, int LRT>
static int dispatch_adj_lr(mq_state* psi, mq_state* lam, const AdjParams& P, double* partials, uint32_t* grid) {
  switch (P.m) {
#define MQ_ADJ_CASE(MM)                                                              \
    case MM: {                                                                       \
      constexpr int L = (MM) < LRT ? (MM) : LRT;                                     \
      constexpr int LTMAX = LRT == 3 ? 8 : 7;                                        \
      constexpr int LT = ((MM) - L) < LTMAX ? ((MM) - L) : LTMAX;                    \
      if constexpr ((MM) >= 10) {                                                    \
        if (P.tma.ndim) return launch_adj_t<R, MM, L, LT, true>(psi, lam, P, partials, grid); \
      }                                                                              \
      return launch_adj_t<R, MM, L, LT, false>(psi, lam, P, partials, grid);         \
    }
    MQ_ADJ_CASE(1) MQ_ADJ_CASE(2) MQ_ADJ_CASE(3) MQ_ADJ_CASE(4) MQ_ADJ_CASE(5) MQ_ADJ_CASE(6)
    MQ_ADJ_CASE(7) MQ_ADJ_CASE(8) MQ_ADJ_CASE(9) MQ_ADJ_CASE(10) MQ_ADJ_CASE(11)
#undef MQ_ADJ_CASE
    default: break;
  }
  return fail(MQ_EUNSUPPORTED, "adjoint tile size not instantiated");
}

template <typename R>
static int dispatch_adj(mq_state* psi, mq_state* lam, const AdjParams& P, double* partials, uint32_t* grid) {
  if constexpr (sizeof(R) == 4) {
    if (adj_lr(MQ_C64) == 3) return dispatch_adj_lr<R, 3>(psi, lam, P, partials, grid);
    return dispatch_adj_lr<R, 4>(psi, lam, P, partials, grid);
  }
  return dispatch_adj_lr<R, 3>(psi, lam, P, partials, grid);
}

// Run one sweep over `targets` (all within one tile).  With grads_dev, the
// gradient of target t, step s is written to grads_dev[index[t]*2+s]
// (device memory) on the stream.
static int run_adj_sweep(mq_state* psi, mq_state* lam, const std::vector<AdjTarget>& targets,
                         const std::vector<int>& tile_bits, bool store_psi, const std::vector<int>& index,
                         double* grads_dev, const uint32_t* perm_cols = nullptr, uint32_t perm_c = 0) {
  const int n = psi->n;
  const int m = (int)tile_bits.size();
  const bool c64 = psi->dtype == MQ_C64;
  const int lrt = adj_lr(psi->dtype);
  const int lr = std::min(m, lrt);
  const int maxph = std::min(kAdjMaxPhases, (12 + lrt - 1) / lrt);
  if ((int)targets.size() > maxph * lr) return fail(MQ_EINVAL, "too many targets for one adjoint sweep");
  AdjParams P;
  std::memset(&P, 0, sizeof(P));
  P.n_tiles = (uint32_t)(uint64_t(1) << (n - m));
  P.n = (uint8_t)n;
  P.m = (uint8_t)m;
  P.store_psi = store_psi ? 1 : 0;
  for (int k = 0; k < m; ++k) P.tile_bit[k] = (uint8_t)tile_bits[k];
  make_base_runs(P.runs, n, P.tile_bit, m);
  // TMA form for tiles of 10 bits and more (both states move by TMA boxes)
  if (tma_enabled() && m >= 10) {
    if (plan_tma(n, psi->amp_bytes(), tile_bits, P.tma)) P.tma.store = 1;
  }
  // a GF(2) map to un-apply first: on load when the sweep is the TMA form of
  // the low tile [0, m) and the map keeps that tile (complex64: and bit 0),
  // else as a permutation pass over both states before the sweep
  if (perm_cols) {
    bool fuse = store_psi && P.tma.store;
    for (int k = 0; k < m && fuse; ++k) fuse = tile_bits[k] == k;
    for (int j = 0; j < m && fuse; ++j) fuse = (perm_cols[j] >> m) == 0;
    if (fuse && c64) fuse = perm_cols[0] == 1u;
    if (fuse) {
      int rc = ensure_alt(psi);
      if (!rc) rc = ensure_alt(lam);
      if (rc) return rc;
      P.perm = 1;
      P.perm_c = perm_c;
      for (int j = 0; j < n; ++j) P.cols[j] = perm_cols[j];
      for (int x = 0; x < 768; ++x) {
        uint32_t v = 0;
        for (int bit = 0; bit < 8; ++bit) {
          const int j = m + 8 * (x >> 8) + bit;
          if (((x >> bit) & 1) && j < n) v ^= perm_cols[j];
        }
        P.htab[x] = v;
      }
    } else {
      int rc = launch_affine_cols(psi, perm_cols, perm_c);
      if (!rc) rc = launch_affine_cols(lam, perm_cols, perm_c);
      if (rc) return rc;
    }
  }
  {
    const int cb = c64 ? 1 : 0;
    const int lt = std::min(lrt == 3 ? 8 : 7, m - lr);
    const int first = cb + lt;
    bool contig = true;
    for (int b = first + 1; b < m; ++b)
      if (tile_bits[b] != tile_bits[b - 1] + 1) contig = false;
    P.hi_contig = (first < m && contig) ? 1 : 0;
    P.hi_shift = (uint8_t)(first < m ? tile_bits[first] : 0);
  }
  // phases: targets in groups of lr, padded with the highest free tile bits
  std::vector<int> local;
  for (const auto& t : targets)
    local.push_back((int)(std::find(tile_bits.begin(), tile_bits.end(), t.bit) - tile_bits.begin()));
  std::vector<int> slot_target(kAdjMaxPhases * kAdjLR, -1);
  int np = 0;
  for (size_t i = 0; i < local.size(); i += lr, ++np) {
    std::vector<int> regs(local.begin() + i, local.begin() + std::min(local.size(), i + lr));
    for (int b = m - 1; (int)regs.size() < lr && b >= 0; --b)
      if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
    std::vector<int> sorted = regs;
    std::sort(sorted.begin(), sorted.end());
    AdjPhase& D = P.ph[np];
    for (int k = 0; k < lr; ++k) D.s_reg[k] = adj_phys(c64, 1u << sorted[k]);
    int j = 0;
    for (int b = 0; b < m; ++b)
      if (std::find(sorted.begin(), sorted.end(), b) == sorted.end()) D.s_grp[j++] = adj_phys(c64, 1u << b);
    for (size_t t = i; t < std::min(local.size(), i + lr); ++t) {
      const int k = (int)(std::find(sorted.begin(), sorted.end(), local[t]) - sorted.begin());
      AdjSlot& S = D.slot[k];
      S.mode = targets[t].mode;
      S.has_u = targets[t].has_u;
      for (int e = 0; e < 8; ++e) {
        S.ud[e] = targets[t].u[e];
        S.uf[e] = (float)targets[t].u[e];
      }
      slot_target[np * kAdjLR + k] = (int)t;
    }
  }
  P.n_phases = (uint8_t)np;
  const uint32_t max_grid = (uint32_t)psi->num_sms * 32;
  const size_t need = (size_t)max_grid * kAdjPartials * sizeof(double);
  int rc = ensure_scratch(psi, need);
  if (rc) return rc;
  double* partials = reinterpret_cast<double*>(psi->scratch);
  uint32_t grid = 0;
  rc = c64 ? dispatch_adj<float>(psi, lam, P, partials, &grid) : dispatch_adj<double>(psi, lam, P, partials, &grid);
  if (rc) return rc;
  if (P.perm) {  // both states now live in their second buffers
    psi->cur ^= 1;
    lam->cur ^= 1;
  }
  if (!grads_dev) return MQ_OK;
  AdjCollect C;
  for (int sl = 0; sl < kAdjSlots; ++sl) C.index[sl] = slot_target[sl] < 0 ? -1 : index[slot_target[sl]];
  k_adj_collect<<<kAdjPartials, kCollectThreads, 0, psi->stream>>>(partials, grid, C, grads_dev);
  MQ_LAUNCHED("k_adj_collect");
  psi->launches += 1;
  return MQ_OK;
}

// Tile groups: index bits split as the U(2) layer does, with tiles of at
// most kAdjTileMax bits (psi and lam share shared memory).
static int run_adj_layer(mq_state* psi, mq_state* lam, const std::vector<AdjTarget>& all, bool store_psi,
                         double* grads_dev, const uint32_t* perm_cols = nullptr, uint32_t perm_c = 0) {
  const int n = psi->n;
  const int tmax = std::min(kAdjTileMax, n);
  const int pas = 4;
  const int lrt = adj_lr(psi->dtype);
  std::vector<std::pair<int, int>> groups;
  if (n <= tmax) {
    groups.push_back({0, n});
  } else {
    const int hi_cap = std::min(tmax - pas, kAdjMaxTargets);
    const int n_hi = (n - tmax + hi_cap - 1) / hi_cap;
    const int low = std::max(n - n_hi * hi_cap, std::min(tmax, (n + n_hi) / (n_hi + 1)));
    groups.push_back({0, low});
    int start = low;
    const int rest = n - low;
    for (int i = 0; i < n_hi; ++i) {
      const int cnt = rest / n_hi + (i < rest % n_hi ? 1 : 0);
      groups.push_back({start, cnt});
      start += cnt;
    }
  }
  const size_t per = (size_t)std::min(kAdjMaxPhases, (12 + lrt - 1) / lrt) * (size_t)std::min(lrt, tmax);
  for (auto [start, cnt] : groups) {
    std::vector<AdjTarget> tg;
    std::vector<int> idx;
    for (size_t i = 0; i < all.size(); ++i)
      if (all[i].bit >= start && all[i].bit < start + cnt) { tg.push_back(all[i]); idx.push_back((int)i); }
    // split further if a group holds more targets than one sweep's phases
    for (size_t i0 = 0; i0 < tg.size(); i0 += per) {
      const size_t i1 = std::min(tg.size(), i0 + per);
      std::vector<AdjTarget> part(tg.begin() + i0, tg.begin() + i1);
      std::vector<int> pidx(idx.begin() + i0, idx.begin() + i1);
      std::vector<int> bits;
      for (auto& t : part) bits.push_back(t.bit);
      const int lowest = *std::min_element(bits.begin(), bits.end());
      for (int b = 0; b < std::min(pas, lowest); ++b) bits.push_back(b);
      std::sort(bits.begin(), bits.end());
      bits.erase(std::unique(bits.begin(), bits.end()), bits.end());
      for (int b = 0; (int)bits.size() < std::min(n, 10) && b < n; ++b)
        if (std::find(bits.begin(), bits.end(), b) == bits.end()) bits.push_back(b);
      std::sort(bits.begin(), bits.end());
      if ((int)bits.size() > kAdjTileMax) return fail(MQ_EINVAL, "adjoint tile too large");
      // a GF(2) map goes with the first sweep (the low group, [0, low))
      int rc = run_adj_sweep(psi, lam, part, bits, store_psi, pidx, grads_dev, perm_cols, perm_c);
      if (rc) return rc;
      perm_cols = nullptr;
    }
  }
  if (perm_cols) {  // no sweep ran: the map on its own
    int rc = launch_affine_cols(psi, perm_cols, perm_c);
    if (!rc) rc = launch_affine_cols(lam, perm_cols, perm_c);
    if (rc) return rc;
  }
  return MQ_OK;
}

int adjoint_sweep(mq_state* psi, mq_state* lam, int n_q, const int32_t* qubits, const double* mats, double* out,
                  bool out_on_device, const uint32_t* perm_cols, uint32_t perm_c) {
  const int n = psi->n;
  std::vector<AdjTarget> all;
  std::vector<bool> seen(n, false);
  for (int i = 0; i < n_q; ++i) {
    const int q = qubits[i];
    if (q < 0 || q >= n) return fail(MQ_EINVAL, "Qubit index out of range");
    if (seen[q]) return fail(MQ_EINVAL, "Duplicate qubit indices");
    seen[q] = true;
    AdjTarget t;
    std::memset(&t, 0, sizeof(t));
    t.bit = n - 1 - q;
    t.mode = SLOT_MEASURE;
    const double* u = mats + (size_t)i * 8;
    const bool ident = u[0] == 1.0 && u[1] == 0.0 && u[2] == 0.0 && u[3] == 0.0 && u[4] == 0.0 && u[5] == 0.0 &&
                       u[6] == 1.0 && u[7] == 0.0;
    t.has_u = ident ? 0 : 1;
    for (int e = 0; e < 8; ++e) t.u[e] = u[e];
    all.push_back(t);
  }
  double* grads = out;
  const bool grads_on_device = out_on_device;
  // scratch: per-block partials, then (host output) the layer's gradients
  const size_t part_bytes = (size_t)psi->num_sms * 32 * kAdjPartials * sizeof(double);
  int rc = ensure_scratch(psi, part_bytes + (size_t)3 * n_q * sizeof(double) + 256);
  if (rc) return rc;
  double* dev = grads_on_device ? grads : (grads ? reinterpret_cast<double*>(static_cast<char*>(psi->scratch) + part_bytes) : nullptr);
  if (dev) MQ_CUDA(cudaMemsetAsync(dev, 0, (size_t)3 * n_q * sizeof(double), psi->stream));
  rc = run_adj_layer(psi, lam, all, true, dev, perm_cols, perm_c);
  if (rc) return rc;
  if (grads && !grads_on_device) {
    MQ_CUDA(cudaMemcpyAsync(grads, dev, (size_t)3 * n_q * sizeof(double), cudaMemcpyDeviceToHost, psi->stream));
    MQ_CUDA(cudaStreamSynchronize(psi->stream));
  }
  return MQ_OK;
}

int apply_hamiltonian(mq_state* psi, mq_state* lam, int n_z, const uint64_t* zmasks, const double* zcoef,
                      const double* xcoef, double* energy) {
  const int n = psi->n;
  const uint64_t lim = psi->dim() - 1;
  if (n_z > kHZWords) return fail(MQ_EUNSUPPORTED, "at most 64 Z words");
  HDiagParams H;
  std::memset(&H, 0, sizeof(H));
  H.dim = (uint32_t)psi->dim();
  for (int w = 0; w < n_z; ++w)
    if (zmasks[w] & ~lim) return fail(MQ_EINVAL, "Pauli mask outside the register");
  // window tables: from the lowest remaining word, every word whose support
  // fits in the 8 bits [lo, lo + 8) joins the table of that window
  std::vector<bool> done(n_z, false);
  for (int w = 0; w < n_z; ++w)
    if (zmasks[w] == 0) { H.base += zcoef[w]; done[w] = true; }
  auto lowbit = [](uint64_t z) { return __builtin_ctzll(z); };
  auto highbit = [](uint64_t z) { return 63 - __builtin_clzll(z); };
  while (H.ntab < kHTab) {
    int first = -1;
    for (int w = 0; w < n_z; ++w)
      if (!done[w] && highbit(zmasks[w]) - lowbit(zmasks[w]) < 8 &&
          (first < 0 || lowbit(zmasks[w]) < lowbit(zmasks[first])))
        first = w;
    if (first < 0) break;
    const int lo = lowbit(zmasks[first]);
    double* t = H.tab[H.ntab];
    for (int w = 0; w < n_z; ++w) {
      if (done[w] || lowbit(zmasks[w]) < lo || highbit(zmasks[w]) >= lo + 8) continue;
      const uint32_t zl = (uint32_t)(zmasks[w] >> lo);
      for (int v = 0; v < 256; ++v) t[v] += (__builtin_popcount((uint32_t)v & zl) & 1) ? -zcoef[w] : zcoef[w];
      done[w] = true;
    }
    H.shift[H.ntab] = (uint8_t)lo;
    ++H.ntab;
  }
  for (int w = 0; w < n_z; ++w) {
    if (done[w]) continue;
    H.z[H.nz] = (uint32_t)zmasks[w];
    H.c[H.nz] = zcoef[w];
    ++H.nz;
  }
  const uint32_t dim = (uint32_t)psi->dim();
  const uint32_t grid = (uint32_t)std::min<uint64_t>((dim + 255) / 256, (uint64_t)psi->num_sms * 8);
  if (psi->dtype == MQ_C64)
    k_hdiag<float><<<grid, 256, 0, psi->stream>>>((const float2*)psi->cur_buf(), (float2*)lam->cur_buf(), H);
  else
    k_hdiag<double><<<grid, 256, 0, psi->stream>>>((const double2*)psi->cur_buf(), (double2*)lam->cur_buf(), H);
  MQ_LAUNCHED("k_hdiag");
  psi->launches += 1;
  psi->sweeps += 1;
  // X part through the tile sweeps (psi read-only)
  std::vector<AdjTarget> xs;
  for (int q = 0; q < n; ++q) {
    if (!xcoef || xcoef[q] == 0.0) continue;
    AdjTarget t;
    std::memset(&t, 0, sizeof(t));
    t.bit = n - 1 - q;
    t.mode = SLOT_XADD;
    t.u[0] = xcoef[q];
    xs.push_back(t);
  }
  if (!xs.empty()) {
    int rc = run_adj_layer(psi, lam, xs, false, nullptr);
    if (rc) return rc;
  }
  if (!energy) return MQ_OK;
  const uint32_t g2 = (uint32_t)psi->num_sms * 4;
  int rc = ensure_scratch(psi, (size_t)g2 * sizeof(double));
  if (rc) return rc;
  double* partials = reinterpret_cast<double*>(psi->scratch);
  if (psi->dtype == MQ_C64)
    k_dot<float><<<g2, 256, 0, psi->stream>>>((const float2*)psi->cur_buf(), (const float2*)lam->cur_buf(), dim, partials);
  else
    k_dot<double><<<g2, 256, 0, psi->stream>>>((const double2*)psi->cur_buf(), (const double2*)lam->cur_buf(), dim, partials);
  MQ_LAUNCHED("k_dot");
  psi->launches += 1;
  psi->sweeps += 1;
  std::vector<double> host(g2);
  MQ_CUDA(cudaMemcpyAsync(host.data(), partials, host.size() * sizeof(double), cudaMemcpyDeviceToHost, psi->stream));
  MQ_CUDA(cudaStreamSynchronize(psi->stream));
  double e = 0.0;
  for (uint32_t b = 0; b < g2; ++b) e += host[b];
  *energy = e;
  return MQ_OK;
}

}  // namespace mq
