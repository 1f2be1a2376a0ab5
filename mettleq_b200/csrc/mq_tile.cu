// Tile sweeps: the fused single-qubit layer (a) and the QFT layer (c).
//
// Replaces the reference's one-thread-per-2^r-amplitudes Metal passes
// (shaders/single_qubit.py:165-210 radix-16, :422-615 layer drivers, and
// shaders/qft.py:61-137 radix-4 / pair stages, :144-236 drivers).  Instead of
// floor(n/4) or ceil(n/2) full-state passes, one sweep here applies the
// gates of up to ~10 index bits:
//
//   * a tile is 2^m amplitudes: its "tile bits" are the swept target bits plus
//     a few low passenger bits, so every global access is a run of >= 8
//     contiguous amplitudes (64 B);
//   * each thread holds 2^LR amplitudes in registers that differ in LR tile
//     bits (a "phase"); the gates of those bits are applied in registers;
//   * between phases the tile is transposed through shared memory (XOR
//     swizzled) so that the next LR bits land in registers;
//   * the sweep is persistent: a grid of resident CTAs strides over tiles.
//
// QFT stages (sim.py:522-563 semantics, no final swaps) fit the same frame:
// stage j on index bit s is a butterfly on bit s followed, on the bit-s = 1
// half, by the phase e^{+i pi L / 2^w} with L the integer value of the ladder
// bits below s (the closed form of qft.py:18-59); the inverse applies the
// conjugate phase first.  Stages within a sweep run in the required order
// (high bit first forward, low bit first inverse); the 1/sqrt(2) of every
// butterfly is applied once per sweep as 2^{-stages/2}.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

enum : uint8_t { OP_U2 = 0, OP_QFT_FWD = 1, OP_QFT_INV = 2, OP_CU2 = 3 };

struct TileOp {
  uint8_t kind, tbit, phase, lad_shift, width, pad[3];
  uint32_t cmask;  // OP_CU2: global index bits that must all be set
  uint32_t pad2;
  double u[8];
};

constexpr int kMaxPhases = 6;
constexpr int kMaxOps = 16;

struct TileParams {
  uint32_t n_tiles;
  uint8_t n, m, n_phases, n_ops;
  uint8_t tile_bit[16];
  uint8_t phase_lo[kMaxPhases];
  uint8_t need_tw, has_scale;
  double scale;
  TileOp ops[kMaxOps];
};

// -------------------------------------------------------------- device side
__device__ __forceinline__ uint32_t swz(uint32_t e) {
  return e ^ (((e >> 4) ^ (e >> 8) ^ (e >> 12)) & 15u);
}

template <int LR>
__device__ __forceinline__ uint32_t roff(int r, const uint32_t (&rb)[LR]) {
  uint32_t o = 0;
#pragma unroll
  for (int k = 0; k < LR; ++k)
    if (r & (1 << k)) o |= rb[k];
  return o;
}

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

template <typename R, int LR, int K>
__device__ __forceinline__ void apply_op_k(V2<R> (&a)[1 << LR], const TileOp& op, uint32_t gt,
                                           const uint32_t (&rb)[LR], const float2* tw) {
  using T = V2<R>;
  constexpr int NR = 1 << LR;
  if (op.kind == OP_U2 || op.kind == OP_CU2) {
    const T u00 = mk<R>((R)op.u[0], (R)op.u[1]), u01 = mk<R>((R)op.u[2], (R)op.u[3]);
    const T u10 = mk<R>((R)op.u[4], (R)op.u[5]), u11 = mk<R>((R)op.u[6], (R)op.u[7]);
    const uint32_t cm = op.cmask;
    const bool ctl = op.kind == OP_CU2;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (r & (1 << K)) continue;
      if (ctl && (((gt | roff<LR>(r, rb)) & cm) != cm)) continue;
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
      if (width) L = ((gt | roff<LR>(r1, rb)) >> shift) & mask;
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

template <typename R, int LR>
__device__ __forceinline__ void apply_op(V2<R> (&a)[1 << LR], const TileOp& op, int k, uint32_t gt,
                                         const uint32_t (&rb)[LR], const float2* tw) {
  switch (k) {
    case 0: apply_op_k<R, LR, 0>(a, op, gt, rb, tw); break;
    case 1: if constexpr (LR > 1) apply_op_k<R, LR, 1>(a, op, gt, rb, tw); break;
    case 2: if constexpr (LR > 2) apply_op_k<R, LR, 2>(a, op, gt, rb, tw); break;
    case 3: if constexpr (LR > 3) apply_op_k<R, LR, 3>(a, op, gt, rb, tw); break;
    case 4: if constexpr (LR > 4) apply_op_k<R, LR, 4>(a, op, gt, rb, tw); break;
    default: break;
  }
}

// Global index of the thread part and of each register bit for layout `lo`
// (register bits = tile-local bits [lo, lo+LR), thread bits = the rest).
template <int LT, int LR>
__device__ __forceinline__ void layout(int lo, int tid, uint32_t base, const TileParams& P,
                                       uint32_t& gt, uint32_t (&rb)[LR], uint32_t& et) {
  gt = base;
  et = 0;
#pragma unroll
  for (int i = 0; i < LT; ++i) {
    const int pos = (i < lo) ? i : i + LR;
    if ((tid >> i) & 1) {
      gt |= 1u << P.tile_bit[pos];
      et |= 1u << pos;
    }
  }
#pragma unroll
  for (int k = 0; k < LR; ++k) rb[k] = 1u << P.tile_bit[lo + k];
}

template <typename R, int LT, int LR>
__global__ void __launch_bounds__(1 << LT)
k_tile(V2<R>* __restrict__ st, const __grid_constant__ TileParams P) {
  using T = V2<R>;
  constexpr int NT = 1 << LT;
  constexpr int NR = 1 << LR;
  constexpr int M = LT + LR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  float2* tw = reinterpret_cast<float2*>(smem_raw + (P.n_phases > 1 ? (sizeof(T) << M) : 0));
  const int tid = threadIdx.x;
  if (P.need_tw) {
    for (int j = tid; j < 3072; j += NT) {
      const int which = j >> 10;
      const float x = (float)(j & 1023);
      const float arg = x * (which == 0 ? 0x1p-10f : (which == 1 ? 0x1p-20f : 0x1p-30f));
      float s, c;
      sincospif(arg, &s, &c);
      tw[j] = make_float2(c, s);
    }
    __syncthreads();
  }
  T a[NR];
  for (uint32_t tile = blockIdx.x; tile < P.n_tiles; tile += gridDim.x) {
    uint64_t b = tile;
#pragma unroll
    for (int k = 0; k < M; ++k) {
      const int pb = P.tile_bit[k];
      b = ((b >> pb) << (pb + 1)) | (b & ((uint64_t(1) << pb) - 1));
    }
    const uint32_t base = (uint32_t)b;
    int lo = P.phase_lo[0];
    uint32_t gt, et, rb[LR];
    layout<LT, LR>(lo, tid, base, P, gt, rb, et);
#pragma unroll
    for (int r = 0; r < NR; ++r) a[r] = st[gt | roff<LR>(r, rb)];
    for (int ph = 0; ph < P.n_phases; ++ph) {
      if (ph > 0) {
        const uint32_t s_prev = swz(et);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NR; ++r) sm[s_prev ^ swz((uint32_t)r << lo)] = a[r];
        lo = P.phase_lo[ph];
        layout<LT, LR>(lo, tid, base, P, gt, rb, et);
        const uint32_t s_now = swz(et);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NR; ++r) a[r] = sm[s_now ^ swz((uint32_t)r << lo)];
      }
      for (int o = 0; o < P.n_ops; ++o) {
        const TileOp& op = P.ops[o];
        if (op.phase != ph) continue;
        apply_op<R, LR>(a, op, (int)op.tbit - lo, gt, rb, tw);
      }
    }
    if (P.has_scale) {
      const R s = (R)P.scale;
#pragma unroll
      for (int r = 0; r < NR; ++r) a[r] = cscale(a[r], s);
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) st[gt | roff<LR>(r, rb)] = a[r];
  }
}

// ---------------------------------------------------------------- host side
struct Sweep {
  std::vector<int> tile_bits;   // ascending global bits
  std::vector<int> phase_lo;
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
static int tile_max(int dtype) { return dtype == MQ_C64 ? kTileMaxC64 : kTileMaxC128; }
static int passengers() { return env_int("MQ_TILE_PASSENGERS", 3, 0, 5); }

// Phases visiting tile-local targets from the top down (U(2) layers and
// forward QFT stages).  The first phase is the coalesced load layout.
static void phases_descending(int m, int lr, const std::vector<int>& targets, Sweep& sw,
                              std::vector<int>& op_phase) {
  sw.phase_lo.clear();
  int lo = m - lr;
  sw.phase_lo.push_back(lo);
  int min_t = targets.empty() ? lo : *std::min_element(targets.begin(), targets.end());
  while (min_t < lo) {
    lo = std::max(lo - lr, min_t);
    sw.phase_lo.push_back(lo);
  }
  op_phase.assign(targets.size(), 0);
  for (size_t i = 0; i < targets.size(); ++i) {
    for (size_t p = 0; p < sw.phase_lo.size(); ++p) {
      if (targets[i] >= sw.phase_lo[p] && targets[i] < sw.phase_lo[p] + lr) { op_phase[i] = (int)p; break; }
    }
  }
  if (sw.phase_lo.back() < 3 && m - lr >= 3) sw.phase_lo.push_back(m - lr);  // coalesced store
}

// Phases visiting targets from the bottom up (inverse QFT stages).
static void phases_ascending(int m, int lr, const std::vector<int>& targets, Sweep& sw,
                             std::vector<int>& op_phase) {
  sw.phase_lo.clear();
  const int top = m - lr;
  int min_t = *std::min_element(targets.begin(), targets.end());
  int max_t = *std::max_element(targets.begin(), targets.end());
  int lo = std::min(min_t, top);
  int first_op_phase = 0;
  if (lo < 3 && top >= 3) { sw.phase_lo.push_back(top); first_op_phase = 1; }  // coalesced load
  sw.phase_lo.push_back(lo);
  while (lo + lr <= max_t) {
    lo = std::min(lo + lr, top);
    sw.phase_lo.push_back(lo);
  }
  op_phase.assign(targets.size(), 0);
  for (size_t i = 0; i < targets.size(); ++i) {
    for (size_t p = first_op_phase; p < sw.phase_lo.size(); ++p) {
      if (targets[i] >= sw.phase_lo[p] && targets[i] < sw.phase_lo[p] + lr) { op_phase[i] = (int)p; break; }
    }
  }
  if (sw.phase_lo.back() < 3 && top >= 3) sw.phase_lo.push_back(top);
}

template <typename R, int LT, int LR>
static int launch_tile_t(mq_state* h, const TileParams& P, size_t smem) {
  auto kern = k_tile<R, LT, LR>;
  static int configured_smem = -1;
  static int blocks_per_sm = 0;
  if ((int)smem > configured_smem) {
    MQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
    configured_smem = (int)std::max<size_t>(smem, 48 * 1024);
    MQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, 1 << LT, smem));
  }
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(P.n_tiles, (uint64_t)h->num_sms * std::max(1, blocks_per_sm)));
  kern<<<grid, 1 << LT, smem, h->stream>>>(reinterpret_cast<V2<R>*>(h->cur_buf()), P);
  MQ_LAUNCHED("k_tile");
  h->launches += 1;
  h->sweeps += 1;
  return MQ_OK;
}

template <typename R, int LR>
static int dispatch_m(mq_state* h, const TileParams& P, size_t smem) {
  switch (P.m - LR) {
    case 0: return launch_tile_t<R, 0, LR>(h, P, smem);
    case 1: return launch_tile_t<R, 1, LR>(h, P, smem);
    case 2: return launch_tile_t<R, 2, LR>(h, P, smem);
    case 3: return launch_tile_t<R, 3, LR>(h, P, smem);
    case 4: return launch_tile_t<R, 4, LR>(h, P, smem);
    case 5: return launch_tile_t<R, 5, LR>(h, P, smem);
    case 6: return launch_tile_t<R, 6, LR>(h, P, smem);
    case 7: return launch_tile_t<R, 7, LR>(h, P, smem);
    case 8: return launch_tile_t<R, 8, LR>(h, P, smem);
    default: break;
  }
  return fail(MQ_EUNSUPPORTED, "tile size not instantiated");
}

static int run_sweep(mq_state* h, const Sweep& sw) {
  const int m = (int)sw.tile_bits.size();
  const int lr = reg_bits(h->dtype, m);
  if (m < 1 || m > tile_max(h->dtype) || m > h->n) return fail(MQ_EINVAL, "bad tile size");
  if ((int)sw.ops.size() > kMaxOps || (int)sw.phase_lo.size() > kMaxPhases)
    return fail(MQ_EINVAL, "tile plan too large");
  TileParams P;
  std::memset(&P, 0, sizeof(P));
  P.n_tiles = (uint32_t)(uint64_t(1) << (h->n - m));
  P.n = (uint8_t)h->n;
  P.m = (uint8_t)m;
  P.n_phases = (uint8_t)sw.phase_lo.size();
  P.n_ops = (uint8_t)sw.ops.size();
  for (int k = 0; k < m; ++k) P.tile_bit[k] = (uint8_t)sw.tile_bits[k];
  for (size_t p = 0; p < sw.phase_lo.size(); ++p) P.phase_lo[p] = (uint8_t)sw.phase_lo[p];
  for (size_t o = 0; o < sw.ops.size(); ++o) P.ops[o] = sw.ops[o];
  P.need_tw = (sw.need_tw && h->dtype == MQ_C64) ? 1 : 0;
  P.has_scale = sw.has_scale ? 1 : 0;
  P.scale = sw.scale;
  size_t smem = 0;
  if (P.n_phases > 1) smem += h->amp_bytes() << m;
  if (P.need_tw) smem += 3072 * sizeof(float2);
  if (h->dtype == MQ_C64) {
    if (lr == 5) return dispatch_m<float, 5>(h, P, smem);
    switch (lr) {
      case 1: return launch_tile_t<float, 0, 1>(h, P, smem);
      case 2: return launch_tile_t<float, 0, 2>(h, P, smem);
      case 3: return launch_tile_t<float, 0, 3>(h, P, smem);
      case 4: return launch_tile_t<float, 0, 4>(h, P, smem);
    }
  } else {
    if (lr == 4) return dispatch_m<double, 4>(h, P, smem);
    switch (lr) {
      case 1: return launch_tile_t<double, 0, 1>(h, P, smem);
      case 2: return launch_tile_t<double, 0, 2>(h, P, smem);
      case 3: return launch_tile_t<double, 0, 3>(h, P, smem);
    }
  }
  return fail(MQ_EUNSUPPORTED, "register tile not instantiated");
}

// Split n index bits into sweeps of at most kmax target bits: the lowest
// group is a contiguous tile, the others carry `pas` low passenger bits.
static std::vector<std::pair<int, int>> split_bits(int n, int kmax) {
  std::vector<std::pair<int, int>> groups;  // [start, count)
  const int s = (n + kmax - 1) / kmax;
  int start = 0;
  for (int i = 0; i < s; ++i) {
    const int cnt = n / s + (i < n % s ? 1 : 0);
    groups.push_back({start, cnt});
    start += cnt;
  }
  return groups;
}

static Sweep make_tile(int n, int start, int cnt, int pas) {
  Sweep sw;
  std::vector<int> bits;
  for (int b = 0; b < std::min(pas, start); ++b) bits.push_back(b);
  for (int b = start; b < start + cnt; ++b) bits.push_back(b);
  std::sort(bits.begin(), bits.end());
  bits.erase(std::unique(bits.begin(), bits.end()), bits.end());
  (void)n;
  sw.tile_bits = bits;
  return sw;
}

static int tile_local(const Sweep& sw, int gbit) {
  for (size_t k = 0; k < sw.tile_bits.size(); ++k)
    if (sw.tile_bits[k] == gbit) return (int)k;
  return -1;
}

int launch_u2_layer(mq_state* h, const double* mats, const uint8_t* active) {
  const int n = h->n;
  const int tmax = tile_max(h->dtype);
  const int pas = passengers();
  const int kdef = h->dtype == MQ_C64 ? 10 : 8;
  const int kmax = std::min(env_int("MQ_U2_BITS", kdef, 1, tmax), tmax - pas);
  std::vector<std::pair<int, int>> groups;
  if (n <= tmax) groups.push_back({0, n});
  else groups = split_bits(n, std::max(1, kmax));
  for (auto [start, cnt] : groups) {
    Sweep sw = (start == 0) ? make_tile(n, 0, cnt, 0) : make_tile(n, start, cnt, pas);
    const int m = (int)sw.tile_bits.size();
    const int lr = reg_bits(h->dtype, m);
    std::vector<int> targets;
    std::vector<int> qubits;
    for (int b = start; b < start + cnt; ++b) {
      const int q = n - 1 - b;
      if (active && !active[q]) continue;
      targets.push_back(tile_local(sw, b));
      qubits.push_back(q);
    }
    if (targets.empty()) continue;
    std::vector<int> op_phase;
    phases_descending(m, lr, targets, sw, op_phase);
    for (size_t i = 0; i < targets.size(); ++i) {
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = OP_U2;
      op.tbit = (uint8_t)targets[i];
      op.phase = (uint8_t)op_phase[i];
      for (int j = 0; j < 8; ++j) op.u[j] = mats[qubits[i] * 8 + j];
      sw.ops.push_back(op);
    }
    int rc = run_sweep(h, sw);
    if (rc) return rc;
  }
  return MQ_OK;
}

// Stages [j_begin, j_end) of the QFT on qubits [q0, q0+k), first qubit = most
// significant logical bit (sim.py:522-563 with wires = range(q0, q0+k); a
// single stage is qft_stage_sub of qft.py:144-181).  Forward stages run in
// increasing j, inverse stages in decreasing j.
int launch_qft_stages(mq_state* h, int q0, int k, int j_begin, int j_end, int inverse) {
  const int n = h->n;
  if (k <= 0 || j_begin >= j_end) return MQ_OK;
  if (q0 < 0 || q0 + k > n || j_begin < 0 || j_end > k) return fail(MQ_EINVAL, "invalid QFT stage range");
  const int tmax = tile_max(h->dtype);
  const int pas = passengers();
  const int kdef = h->dtype == MQ_C64 ? 8 : 6;
  const int kq = std::min(env_int("MQ_QFT_STAGES", kdef, 1, tmax), tmax - pas);
  const int lad_shift = n - q0 - k;  // index bit of the last wire
  const int count = j_end - j_begin;
  // stage j acts on bit b_j = n-1-q0-j with ladder width k-1-j
  std::vector<std::pair<int, int>> groups;  // stage ranges [j0, j0+cnt)
  const int blo_all = n - 1 - q0 - (j_end - 1);
  if (count + std::min(pas, blo_all) <= tmax) {
    groups.push_back({j_begin, count});
  } else {
    const int s = (count + kq - 1) / kq;
    int j0 = j_begin;
    for (int i = 0; i < s; ++i) {
      const int cnt = count / s + (i < count % s ? 1 : 0);
      groups.push_back({j0, cnt});
      j0 += cnt;
    }
  }
  if (inverse) std::reverse(groups.begin(), groups.end());
  for (auto [j0, cnt] : groups) {
    const int bhi = n - 1 - q0 - j0;
    const int blo = bhi - cnt + 1;
    Sweep sw;
    std::vector<int> bits;
    const int pas_here = (blo > 0) ? std::min(pas, blo) : 0;
    for (int b = 0; b < pas_here; ++b) bits.push_back(b);
    for (int b = blo; b <= bhi; ++b) bits.push_back(b);
    sw.tile_bits = bits;
    const int m = (int)bits.size();
    if (m > tmax) return fail(MQ_EINVAL, "qft tile too large");
    const int lr = reg_bits(h->dtype, m);
    std::vector<int> targets, stages;
    if (!inverse) {
      for (int j = j0; j < j0 + cnt; ++j) { stages.push_back(j); targets.push_back(tile_local(sw, n - 1 - q0 - j)); }
    } else {
      for (int j = j0 + cnt - 1; j >= j0; --j) { stages.push_back(j); targets.push_back(tile_local(sw, n - 1 - q0 - j)); }
    }
    std::vector<int> op_phase;
    if (!inverse) phases_descending(m, lr, targets, sw, op_phase);
    else phases_ascending(m, lr, targets, sw, op_phase);
    for (size_t i = 0; i < targets.size(); ++i) {
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = inverse ? OP_QFT_INV : OP_QFT_FWD;
      op.tbit = (uint8_t)targets[i];
      op.phase = (uint8_t)op_phase[i];
      op.lad_shift = (uint8_t)lad_shift;
      op.width = (uint8_t)(k - 1 - stages[i]);
      if (op.width) sw.need_tw = true;
      sw.ops.push_back(op);
    }
    // 2^{-cnt/2}: exact power of two for even counts
    sw.scale = std::ldexp(1.0, -(cnt / 2)) * ((cnt & 1) ? 0.70710678118654752440 : 1.0);
    sw.has_scale = true;
    int rc = run_sweep(h, sw);
    if (rc) return rc;
  }
  return MQ_OK;
}

int launch_qft_contiguous(mq_state* h, int q0, int k, int inverse) {
  return launch_qft_stages(h, q0, k, 0, k, inverse);
}

// Controlled single-qubit gates (CH/CRX/CRY, Toffoli as doubly controlled X;
// controlled_single.py:18-134, sim.py:140-213).  Consecutive gates whose
// wire sets are pairwise disjoint commute and share one sweep; any other
// gate starts a new sweep, so the list order is respected.
int launch_cu2_list(mq_state* h, int n_gates, const int32_t* targets, const uint32_t* cmasks, const double* mats) {
  const int n = h->n;
  const int tmax = tile_max(h->dtype);
  const int pas = passengers();
  const int kdef = h->dtype == MQ_C64 ? 10 : 8;
  const int kmax = std::min(env_int("MQ_U2_BITS", kdef, 1, tmax), tmax - pas);
  int g = 0;
  while (g < n_gates) {
    std::vector<int> members;
    uint32_t used = 0;
    int lowest = n;
    while (g < n_gates && (int)members.size() < kmax) {
      const int tb = n - 1 - targets[g];
      const uint32_t sup = cmasks[g] | (1u << tb);
      if (used & sup) break;
      used |= sup;
      members.push_back(g);
      lowest = std::min(lowest, tb);
      ++g;
      (void)lowest;
    }
    Sweep sw;
    std::vector<int> bits;
    for (int i : members) bits.push_back(n - 1 - targets[i]);
    std::sort(bits.begin(), bits.end());
    const int low_target = bits.front();
    for (int b = 0; b < std::min(pas, low_target); ++b) bits.push_back(b);
    // pad with the lowest unused bits so that the tile has >= 5 bits when possible
    for (int b = 0; (int)bits.size() < std::min(n, 5) && b < n; ++b)
      if (std::find(bits.begin(), bits.end(), b) == bits.end()) bits.push_back(b);
    std::sort(bits.begin(), bits.end());
    bits.erase(std::unique(bits.begin(), bits.end()), bits.end());
    sw.tile_bits = bits;
    const int m = (int)bits.size();
    if (m > tmax) return fail(MQ_EINVAL, "controlled-gate tile too large");
    const int lr = reg_bits(h->dtype, m);
    std::vector<int> tl;
    for (int i : members) tl.push_back(tile_local(sw, n - 1 - targets[i]));
    std::vector<int> op_phase;
    phases_descending(m, lr, tl, sw, op_phase);
    for (size_t i = 0; i < members.size(); ++i) {
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = OP_CU2;
      op.tbit = (uint8_t)tl[i];
      op.phase = (uint8_t)op_phase[i];
      op.cmask = cmasks[members[i]];
      for (int j = 0; j < 8; ++j) op.u[j] = mats[(size_t)members[i] * 8 + j];
      sw.ops.push_back(op);
    }
    int rc = run_sweep(h, sw);
    if (rc) return rc;
  }
  return MQ_OK;
}

}  // namespace mq
