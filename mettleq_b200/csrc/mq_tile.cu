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
//   * shared-memory addresses are XOR-swizzled with a per-sweep linear map
//     chosen on the host so that every phase's accesses are free of bank
//     conflicts;
//   * the finished tile is written back with coalesced stores.
//
// QFT stages (sim.py:522-563, no final swaps): stage j on index bit s is a
// butterfly on bit s, then on the bit-s = 1 half the phase e^{+i pi L / 2^w}
// with L the integer value of the ladder bits below s (the closed form of
// qft.py:18-59); the inverse applies the conjugate phase first.  Stages run
// in the required order (high bit first forward, low bit first inverse); the
// 1/sqrt(2) of every butterfly is applied once per sweep as 2^{-stages/2}.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

enum : uint8_t { OP_U2 = 0, OP_QFT_FWD = 1, OP_QFT_INV = 2, OP_CU2 = 3 };

constexpr int kMaxPhases = 6;
constexpr int kMaxOps = 16;
constexpr int kMaxTileBits = 12;

struct TileOp {
  uint8_t kind, phase, rk, lad_shift, width, pad[3];
  uint32_t cmask;  // OP_CU2: global index bits that must all be set
  uint32_t pad2;
  double u[8];     // 2x2 matrix (re, im interleaved)
  float uf[8];     // the same matrix rounded to float for complex64 sweeps
};

struct PhaseDesc {
  uint16_t swz_reg[5];               // swizzled smem offset of each register bit
  uint16_t swz_grp[kMaxTileBits];    // ... of each group (thread/loop) bit
  uint32_t g_reg[5];                 // global index bit of each register bit
  uint32_t g_grp[kMaxTileBits];
};

struct TileParams {
  uint32_t n_tiles;
  uint8_t n, m, n_phases, n_ops;
  uint8_t tile_bit[16];
  uint8_t need_tw, has_scale, pad[6];
  double scale;
  uint16_t swz_tile[16];             // swizzled smem offset of tile bit k
  uint8_t ph_op[kMaxPhases + 2];     // ops of phase p are [ph_op[p], ph_op[p+1])
  PhaseDesc ph[kMaxPhases];
  TileOp ops[kMaxOps];
};

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
__device__ __forceinline__ uint32_t gsel(int r, const uint32_t* g) {
  uint32_t o = 0;
#pragma unroll
  for (int k = 0; k < LR; ++k)
    if (r & (1 << k)) o |= g[k];
  return o;
}

// XOR of the swizzled shared-memory offsets of the set register bits
// (swizzled offsets are multi-bit, so they combine with XOR, not OR).
template <int LR>
__device__ __forceinline__ uint32_t xsel(int r, const uint32_t* s) {
  uint32_t o = 0;
#pragma unroll
  for (int k = 0; k < LR; ++k)
    if (r & (1 << k)) o ^= s[k];
  return o;
}

template <typename R, int LR, int K, bool QFT>
__device__ __forceinline__ void apply_op_k(V2<R> (&a)[1 << LR], const TileOp& op, uint32_t gq, const uint32_t* greg,
                                           const float2* tw) {
  using T = V2<R>;
  constexpr int NR = 1 << LR;
  if constexpr (!QFT) {
    T u00, u01, u10, u11;
    if constexpr (sizeof(R) == 4) {
      u00 = mk<R>(op.uf[0], op.uf[1]); u01 = mk<R>(op.uf[2], op.uf[3]);
      u10 = mk<R>(op.uf[4], op.uf[5]); u11 = mk<R>(op.uf[6], op.uf[7]);
    } else {
      u00 = mk<R>(op.u[0], op.u[1]); u01 = mk<R>(op.u[2], op.u[3]);
      u10 = mk<R>(op.u[4], op.u[5]); u11 = mk<R>(op.u[6], op.u[7]);
    }
    const uint32_t cm = op.cmask;
    const bool ctl = op.kind == OP_CU2;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (r & (1 << K)) continue;
      if (ctl && (((gq | gsel<LR>(r, greg)) & cm) != cm)) continue;
      const T x0 = a[r], x1 = a[r | (1 << K)];
      a[r] = cadd(cmul(u00, x0), cmul(u01, x1));
      a[r | (1 << K)] = cadd(cmul(u10, x0), cmul(u11, x1));
    }
  } else {
    const int width = op.width;
    const int shift = op.lad_shift;
    const uint32_t mask = width ? ((width >= 32) ? 0xffffffffu : ((1u << width) - 1u)) : 0u;
    const bool fwd = op.kind == OP_QFT_FWD;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (r & (1 << K)) continue;
      const int r1 = r | (1 << K);
      T x0 = a[r], x1 = a[r1];
      uint32_t L = 0;
      if (width) L = ((gq | gsel<LR>(r1, greg)) >> shift) & mask;
      if (fwd) {
        T d = csub(x0, x1);
        a[r] = cadd(x0, x1);
        if (L) d = cmul(d, Twiddle<R>::get(tw, L, width));
        a[r1] = d;
      } else {
        if (L) x1 = cmulc(x1, Twiddle<R>::get(tw, L, width));
        a[r] = cadd(x0, x1);
        a[r1] = csub(x0, x1);
      }
    }
  }
}

template <typename R, int LR, bool QFT>
__device__ __forceinline__ void apply_op(V2<R> (&a)[1 << LR], const TileOp& op, uint32_t gq, const uint32_t* greg,
                                         const float2* tw) {
  switch (op.rk) {
    case 0: apply_op_k<R, LR, 0, QFT>(a, op, gq, greg, tw); break;
    case 1: if constexpr (LR > 1) apply_op_k<R, LR, 1, QFT>(a, op, gq, greg, tw); break;
    case 2: if constexpr (LR > 2) apply_op_k<R, LR, 2, QFT>(a, op, gq, greg, tw); break;
    case 3: if constexpr (LR > 3) apply_op_k<R, LR, 3, QFT>(a, op, gq, greg, tw); break;
    case 4: if constexpr (LR > 4) apply_op_k<R, LR, 4, QFT>(a, op, gq, greg, tw); break;
    default: break;
  }
}

// Tile of 2^M amplitudes, 2^LT threads, 2^LR amplitudes in registers per
// group, 2^(M-LR-LT) groups per thread per phase.  QFT selects the op family
// (QFT stages vs U(2) / controlled U(2)) so each instance carries only the
// code it runs.
template <typename R, int M, int LR, int LT>
__device__ __forceinline__ uint32_t tile_base_of(uint32_t tile, const TileParams& P) {
  uint64_t x = tile;
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const int pb = P.tile_bit[k];
    x = ((x >> pb) << (pb + 1)) | (x & ((uint64_t(1) << pb) - 1));
  }
  return (uint32_t)x;
}

template <typename R, int M, int LR, int LT, bool QFT>
__global__ void __launch_bounds__(1 << LT, (LT >= 7 ? 3 : 1))
k_tile(const V2<R>* src, V2<R>* dst, const __grid_constant__ TileParams P) {
  using T = V2<R>;
  constexpr int NT = 1 << LT;
  constexpr int NR = 1 << LR;
  constexpr int E = 1 << M;
  constexpr int GPT = (E / NR) / NT;
  constexpr int LPT = E / NT;            // elements per thread in load / store
  constexpr int LHI = M - LT;            // element-index bits above the thread bits
  constexpr int CPB = sizeof(T);         // bytes per cp.async
  static_assert(GPT >= 1 && LPT >= 1, "bad tile configuration");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* bufs = reinterpret_cast<T*>(smem_raw);
  float2* tw = reinterpret_cast<float2*>(smem_raw + 2 * sizeof(T) * E);
  const int tid = threadIdx.x;

  if (QFT && P.need_tw) {
    for (int j = tid; j < 3072; j += NT) {
      const int which = j >> 10;
      const float x = (float)(j & 1023);
      const float arg = x * (which == 0 ? 0x1p-10f : (which == 1 ? 0x1p-20f : 0x1p-30f));
      float s, c;
      sincospif(arg, &s, &c);
      tw[j] = make_float2(c, s);
    }
  }

  // per-thread part of the load/store mapping (element e = tid + k*NT)
  uint32_t g_t = 0, s_t = 0;
#pragma unroll
  for (int b = 0; b < LT; ++b)
    if ((tid >> b) & 1) { g_t |= 1u << P.tile_bit[b]; s_t ^= P.swz_tile[b]; }

  uint32_t tile = blockIdx.x;
  if (tile < P.n_tiles) {
    const uint32_t base = tile_base_of<R, M, LR, LT>(tile, P) | g_t;
    const uint32_t sb = smem_u32(bufs);
#pragma unroll
    for (int k = 0; k < LPT; ++k) {
      uint32_t g = base, s = s_t;
#pragma unroll
      for (int b = 0; b < LHI; ++b)
        if ((k >> b) & 1) { g |= 1u << P.tile_bit[LT + b]; s ^= P.swz_tile[LT + b]; }
      cp_async<CPB>(sb + s * (uint32_t)sizeof(T), src + g);
    }
  }
  cp_async_commit();
  if (QFT && P.need_tw) __syncthreads();
  T a[NR];
  for (int it = 0; tile < P.n_tiles; tile += gridDim.x, ++it) {
    T* cur = bufs + (it & 1) * E;
    const uint32_t next = tile + gridDim.x;
    if (next < P.n_tiles) {
      const uint32_t nbase = tile_base_of<R, M, LR, LT>(next, P) | g_t;
      const uint32_t sb = smem_u32(bufs + ((it + 1) & 1) * E);
#pragma unroll
      for (int k = 0; k < LPT; ++k) {
        uint32_t g = nbase, s = s_t;
#pragma unroll
        for (int b = 0; b < LHI; ++b)
          if ((k >> b) & 1) { g |= 1u << P.tile_bit[LT + b]; s ^= P.swz_tile[LT + b]; }
        cp_async<CPB>(sb + s * (uint32_t)sizeof(T), src + g);
      }
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const uint32_t base = tile_base_of<R, M, LR, LT>(tile, P);
    for (int ph = 0; ph < P.n_phases; ++ph) {
      const PhaseDesc& D = P.ph[ph];
      const int o0 = P.ph_op[ph], o1 = P.ph_op[ph + 1];
      uint32_t greg[LR], sreg[LR];
#pragma unroll
      for (int k = 0; k < LR; ++k) { greg[k] = D.g_reg[k]; sreg[k] = D.swz_reg[k]; }
#pragma unroll
      for (int g = 0; g < GPT; ++g) {
        const uint32_t q = (uint32_t)tid + (uint32_t)g * NT;
        uint32_t sq = 0, gq = base;
#pragma unroll
        for (int j = 0; j < M - LR; ++j)
          if ((q >> j) & 1) { sq ^= D.swz_grp[j]; gq |= D.g_grp[j]; }
#pragma unroll
        for (int r = 0; r < NR; ++r) a[r] = cur[sq ^ xsel<LR>(r, sreg)];
        for (int o = o0; o < o1; ++o) apply_op<R, LR, QFT>(a, P.ops[o], gq, greg, tw);
#pragma unroll
        for (int r = 0; r < NR; ++r) cur[sq ^ xsel<LR>(r, sreg)] = a[r];
      }
      __syncthreads();
    }
    const uint32_t gb = base | g_t;
#pragma unroll
    for (int k = 0; k < LPT; ++k) {
      uint32_t g = gb, s = s_t;
#pragma unroll
      for (int b = 0; b < LHI; ++b)
        if ((k >> b) & 1) { g |= 1u << P.tile_bit[LT + b]; s ^= P.swz_tile[LT + b]; }
      T v = cur[s];
      if (QFT) v = cscale(v, (R)P.scale);
      dst[g] = v;
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------- host side
struct Sweep {
  std::vector<int> tile_bits;              // ascending global bits
  std::vector<std::vector<int>> phases;    // register bits (tile-local) per phase
  std::vector<TileOp> ops;
  bool need_tw = false;
  double scale = 1.0;
  bool has_scale = false;
};

static int env_int(const char* name, int dflt, int lo, int hi) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  int x = std::atoi(v);
  return std::min(hi, std::max(lo, x));
}

static int reg_bits(int dtype, int m) { return std::min(m, dtype == MQ_C64 ? 5 : 4); }
static int tile_max(int dtype) { return dtype == MQ_C64 ? env_int("MQ_TILE_MAX", 12, 6, 12) : 11; }
static int passengers() { return env_int("MQ_TILE_PASSENGERS", 3, 0, 5); }
static int min_tile() { return env_int("MQ_TILE_MIN", 10, 1, 12); }

// Register phases: targets (tile-local) chunked in the given order into
// groups of LR; the last group is padded with non-target bits.  Records the
// phase index and register slot of every target.
static void make_phases(int m, int lr, const std::vector<int>& order, Sweep& sw, std::vector<int>& op_phase,
                        std::vector<int>& op_rk) {
  sw.phases.clear();
  op_phase.assign(order.size(), 0);
  op_rk.assign(order.size(), 0);
  std::vector<bool> is_target(m, false);
  for (int t : order) is_target[t] = true;
  for (size_t i = 0; i < order.size(); i += lr) {
    std::vector<int> regs;
    for (size_t j = i; j < std::min(order.size(), i + lr); ++j) {
      op_phase[j] = (int)sw.phases.size();
      regs.push_back(order[j]);
    }
    for (int b = 0; (int)regs.size() < lr && b < m; ++b)
      if (std::find(regs.begin(), regs.end(), b) == regs.end() && !is_target[b]) regs.push_back(b);
    for (int b = 0; (int)regs.size() < lr && b < m; ++b)
      if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
    std::vector<int> sorted = regs;
    std::sort(sorted.begin(), sorted.end());
    for (size_t j = i; j < std::min(order.size(), i + lr); ++j)
      op_rk[j] = (int)(std::find(sorted.begin(), sorted.end(), order[j]) - sorted.begin());
    sw.phases.push_back(sorted);
  }
}

// Swizzle: the shared-memory offset of tile bit b is (1 << b) ^ S(b) with
// S(b) confined to the low `lb` bits (S(b) = 0 for b < lb).  For every phase,
// the lowest lb group bits (the lanes of one shared-memory wavefront) must
// map to independent low-bit patterns.  Small backtracking search; S = 0
// (correct, possibly conflicted) if none is found.
static bool independent(const std::vector<uint32_t>& v) {
  uint32_t basis[8] = {0};
  for (uint32_t x : v) {
    for (int p = 7; p >= 0; --p) {
      if (!((x >> p) & 1u)) continue;
      if (basis[p]) x ^= basis[p];
      else { basis[p] = x; break; }
    }
    if (!x) return false;
  }
  return true;
}

static std::vector<uint32_t> solve_swizzle(int m, int lb, const std::vector<std::vector<int>>& phases) {
  std::vector<std::vector<int>> lanes;
  for (auto& regs : phases) {
    std::vector<int> grp;
    for (int b = 0; b < m && (int)grp.size() < lb; ++b)
      if (std::find(regs.begin(), regs.end(), b) == regs.end()) grp.push_back(b);
    lanes.push_back(grp);
  }
  std::vector<uint32_t> S(m, 0);
  const uint32_t full = (1u << lb) - 1u;
  auto img = [&](int b) -> uint32_t { return b < lb ? (1u << b) : S[b]; };
  auto ok_upto = [&](int upto) {
    for (auto& grp : lanes) {
      if ((int)grp.size() < lb) continue;
      bool determined = true;
      for (int b : grp)
        if (b >= lb && b > upto) determined = false;
      if (!determined) continue;
      std::vector<uint32_t> v;
      for (int b : grp) v.push_back(img(b));
      if (!independent(v)) return false;
    }
    return true;
  };
  int nodes = 0;
  std::function<bool(int)> rec = [&](int b) -> bool {
    if (b >= m) return true;
    if (++nodes > 100000) return false;
    for (uint32_t c = 1; c <= full; ++c) {
      S[b] = c;
      if (ok_upto(b) && rec(b + 1)) return true;
    }
    S[b] = 0;
    return false;
  };
  if (m <= lb || rec(lb)) return S;
  return std::vector<uint32_t>(m, 0);
}

template <typename R, int M, int LR, int LT, bool QFT>
static int launch_tile_t(mq_state* h, const TileParams& P, size_t smem, bool out_of_place) {
  auto kern = k_tile<R, M, LR, LT, QFT>;
  static int configured_smem = -1;
  static int blocks_per_sm = 0;
  if ((int)smem > configured_smem) {
    MQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
    configured_smem = (int)std::max<size_t>(smem, 48 * 1024);
    MQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, 1 << LT, smem));
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

template <typename R, bool QFT>
static int dispatch_tile(mq_state* h, const TileParams& P, size_t smem) {
  constexpr bool F = sizeof(R) == 4;
  constexpr int LRMAX = F ? 5 : 4;
  switch (P.m) {
#define MQ_TILE_CASE(MM)                                                        \
    case MM: {                                                                  \
      constexpr int LR = (MM) < LRMAX ? (MM) : LRMAX;                           \
      constexpr int LT = ((MM) - LR) < 7 ? ((MM) - LR) : 7;                     \
      return launch_tile_t<R, MM, LR, LT, QFT>(h, P, smem, false);                  \
    }
    MQ_TILE_CASE(1) MQ_TILE_CASE(2) MQ_TILE_CASE(3) MQ_TILE_CASE(4) MQ_TILE_CASE(5) MQ_TILE_CASE(6)
    MQ_TILE_CASE(7) MQ_TILE_CASE(8) MQ_TILE_CASE(9) MQ_TILE_CASE(10) MQ_TILE_CASE(11)
#undef MQ_TILE_CASE
    case 12:
      if constexpr (F) return launch_tile_t<R, 12, 5, 7, QFT>(h, P, smem, false);
      break;
    default: break;
  }
  return fail(MQ_EUNSUPPORTED, "tile size not instantiated");
}

static int run_sweep(mq_state* h, Sweep& sw, const std::vector<int>& op_phase, const std::vector<int>& op_rk) {
  const int m = (int)sw.tile_bits.size();
  const int lr = reg_bits(h->dtype, m);
  if (m < 1 || m > tile_max(h->dtype) || m > h->n) return fail(MQ_EINVAL, "bad tile size");
  if ((int)sw.ops.size() > kMaxOps || (int)sw.phases.size() > kMaxPhases) return fail(MQ_EINVAL, "tile plan too large");
  const int lb = std::min(m, h->dtype == MQ_C64 ? 4 : 3);  // 2^lb lanes per shared-memory wavefront
  std::vector<uint32_t> S = env_int("MQ_TILE_SWIZZLE", 1, 0, 1) ? solve_swizzle(m, lb, sw.phases)
                                                                 : std::vector<uint32_t>(m, 0);
  auto swz_of = [&](int b) -> uint16_t { return (uint16_t)((1u << b) ^ S[b]); };
  TileParams P;
  std::memset(&P, 0, sizeof(P));
  P.n_tiles = (uint32_t)(uint64_t(1) << (h->n - m));
  P.n = (uint8_t)h->n;
  P.m = (uint8_t)m;
  P.n_phases = (uint8_t)sw.phases.size();
  P.n_ops = (uint8_t)sw.ops.size();
  for (int k = 0; k < m; ++k) {
    P.tile_bit[k] = (uint8_t)sw.tile_bits[k];
    P.swz_tile[k] = swz_of(k);
  }
  for (size_t p = 0; p < sw.phases.size(); ++p) {
    const auto& regs = sw.phases[p];
    PhaseDesc& D = P.ph[p];
    for (int k = 0; k < lr; ++k) {
      D.swz_reg[k] = swz_of(regs[k]);
      D.g_reg[k] = 1u << sw.tile_bits[regs[k]];
    }
    int j = 0;
    for (int b = 0; b < m; ++b) {
      if (std::find(regs.begin(), regs.end(), b) != regs.end()) continue;
      D.swz_grp[j] = swz_of(b);
      D.g_grp[j] = 1u << sw.tile_bits[b];
      ++j;
    }
  }
  // ops grouped by phase, original order kept inside each phase
  {
    int w = 0;
    for (size_t p = 0; p < sw.phases.size(); ++p) {
      P.ph_op[p] = (uint8_t)w;
      for (size_t o = 0; o < sw.ops.size(); ++o) {
        if (op_phase[o] != (int)p) continue;
        P.ops[w] = sw.ops[o];
        for (int j = 0; j < 8; ++j) P.ops[w].uf[j] = (float)sw.ops[o].u[j];
        P.ops[w].phase = (uint8_t)p;
        P.ops[w].rk = (uint8_t)op_rk[o];
        ++w;
      }
    }
    P.ph_op[sw.phases.size()] = (uint8_t)w;
  }
  P.need_tw = (sw.need_tw && h->dtype == MQ_C64) ? 1 : 0;
  P.has_scale = sw.has_scale ? 1 : 0;
  P.scale = sw.has_scale ? sw.scale : 1.0;
  size_t smem = 2 * (h->amp_bytes() << m);
  if (P.need_tw) smem += 3072 * sizeof(float2);
  const bool qft = !sw.ops.empty() && (sw.ops[0].kind == OP_QFT_FWD || sw.ops[0].kind == OP_QFT_INV);
  if (h->dtype == MQ_C64) return qft ? dispatch_tile<float, true>(h, P, smem) : dispatch_tile<float, false>(h, P, smem);
  return qft ? dispatch_tile<double, true>(h, P, smem) : dispatch_tile<double, false>(h, P, smem);
}

static int tile_local(const std::vector<int>& bits, int gbit) {
  for (size_t k = 0; k < bits.size(); ++k)
    if (bits[k] == gbit) return (int)k;
  return -1;
}

// Tile bits for a set of target bits: the targets, the low passengers, and
// further low bits until the tile has at least min(n, MQ_TILE_MIN) bits.
static std::vector<int> tile_for(int n, const std::vector<int>& targets, int pas, int tmax) {
  std::vector<int> bits = targets;
  const int lowest = *std::min_element(targets.begin(), targets.end());
  for (int b = 0; b < std::min(pas, lowest); ++b) bits.push_back(b);
  std::sort(bits.begin(), bits.end());
  bits.erase(std::unique(bits.begin(), bits.end()), bits.end());
  const int want = std::min({n, min_tile(), tmax});
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
  return groups;
}

int launch_u2_layer(mq_state* h, const double* mats, const uint8_t* active) {
  const int n = h->n;
  const int tmax = tile_max(h->dtype);
  const int pas = passengers();
  for (auto [start, cnt] : split_bits(n, tmax, pas)) {
    std::vector<int> gbits;
    std::vector<int> qubits;
    for (int b = start + cnt - 1; b >= start; --b) {
      const int q = n - 1 - b;
      if (active && !active[q]) continue;
      gbits.push_back(b);
      qubits.push_back(q);
    }
    if (gbits.empty()) continue;
    Sweep sw;
    sw.tile_bits = tile_for(n, gbits, pas, tmax);
    const int m = (int)sw.tile_bits.size();
    const int lr = reg_bits(h->dtype, m);
    std::vector<int> order;
    for (int b : gbits) order.push_back(tile_local(sw.tile_bits, b));
    std::vector<int> op_phase, op_rk;
    make_phases(m, lr, order, sw, op_phase, op_rk);
    for (size_t i = 0; i < order.size(); ++i) {
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = OP_U2;
      for (int j = 0; j < 8; ++j) op.u[j] = mats[(size_t)qubits[i] * 8 + j];
      sw.ops.push_back(op);
    }
    int rc = run_sweep(h, sw, op_phase, op_rk);
    if (rc) return rc;
  }
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
  const int tmax = tile_max(h->dtype);
  const int pas = passengers();
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
    sw.tile_bits = tile_for(n, gbits, pas, tmax);
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
  const int tmax = tile_max(h->dtype);
  const int pas = passengers();
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
    sw.tile_bits = tile_for(n, gbits, pas, tmax);
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
