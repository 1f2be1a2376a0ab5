// Diagonal phase layers (b): RZ / U1 / Z / S / T, CZ / CPHASE / CRZ, ZZ and
// any mix of them, in ONE streaming pass.
//
// Replaces diag_pair_layer / diag_weighted_layer (shaders/diag.py:19-217),
// zz_chain_layer / zz_weighted_layer (shaders/zz.py:16-185) and the per-gate
// apply_diagonal passes of the CPU path (sim.py:94-138, device.py:1154-1211).
//
// The reference multiplies one unit phase per equal-angle group inside the
// kernel (zz.py:40-71); here the host factors the whole diagonal into at most
// eight lookup tables, each indexed by a window of <= 10 index bits (or by a
// short list of scattered bits for far-apart pairs).  Every term's phase is
// folded into exactly one table in double precision, so a 29-bond chain with
// all-different angles costs four table reads and four complex products per
// amplitude, independent of the number of bonds.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

struct DiagLut {
  uint16_t off;
  uint8_t nbits;
  uint8_t contig;
  uint8_t shift;
  uint8_t pos[11];
};

constexpr int kMaxLuts = 8;
template <typename R> struct DiagCap;
template <> struct DiagCap<float> { static constexpr int v = 2048; };
template <> struct DiagCap<double> { static constexpr int v = 1024; };

template <typename R>
struct DiagParams {
  uint32_t n_pairs;  // 2^(n-1) element pairs
  int32_t n_luts;
  uint32_t n_entries;
  int32_t n_low;     // tables [0, n_low) read index bit 0
  int32_t pair_lut0; // table 0 is a contiguous window starting at bit 0
  int32_t pad[3];
  DiagLut lut[kMaxLuts];
  V2<R> e[DiagCap<R>::v];
};

__device__ __forceinline__ uint32_t lut_index(const DiagLut& L, uint32_t i) {
  if (L.contig) return (i >> L.shift) & ((1u << L.nbits) - 1u);
  uint32_t x = 0;
  for (int k = 0; k < L.nbits; ++k) x |= ((i >> L.pos[k]) & 1u) << k;
  return x;
}

// Each thread handles amplitude pairs (2p, 2p+1), four independent pairs per
// iteration, with 16-byte (complex64) accesses that are contiguous across the
// warp.  Tables [0, n_low) read index bit 0: when table 0 is a window starting
// at bit 0 (pair_lut0) the pair's two entries are adjacent and read as one
// 16-byte value; the other tables give one factor per pair.
template <typename R>
__global__ void __launch_bounds__(256) k_diag(V2<R>* __restrict__ st, const __grid_constant__ DiagParams<R> P) {
  using T = V2<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* lut = reinterpret_cast<T*>(smem_raw);
  for (uint32_t j = threadIdx.x; j < P.n_entries; j += blockDim.x) lut[j] = P.e[j];
  __syncthreads();
  constexpr int U = 4;
  const uint32_t stride = gridDim.x * blockDim.x;
  const int n_low = P.n_low;
  const bool pair0 = P.pair_lut0;
  for (uint32_t p0 = blockIdx.x * blockDim.x + threadIdx.x; p0 < P.n_pairs; p0 += U * stride) {
    T a0[U], a1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t p = p0 + (uint32_t)u * stride;
      if (p < P.n_pairs) {
        if constexpr (sizeof(R) == 4) {
          const float4 x = reinterpret_cast<const float4*>(st)[p];
          a0[u] = make_float2(x.x, x.y);
          a1[u] = make_float2(x.z, x.w);
        } else {
          a0[u] = st[2 * p];
          a1[u] = st[2 * p + 1];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t p = p0 + (uint32_t)u * stride;
      if (p >= P.n_pairs) continue;
      const uint32_t i0 = 2 * p;
      T hi = mk<R>(1, 0);
      for (int l = n_low; l < P.n_luts; ++l) hi = cmul(hi, lut[P.lut[l].off + lut_index(P.lut[l], i0)]);
      T f0 = hi, f1 = hi;
      int l = 0;
      if (pair0 && n_low > 0) {
        const uint32_t k = P.lut[0].off + lut_index(P.lut[0], i0);
        f0 = cmul(f0, lut[k]);
        f1 = cmul(f1, lut[k + 1]);
        l = 1;
      }
      for (; l < n_low; ++l) {
        f0 = cmul(f0, lut[P.lut[l].off + lut_index(P.lut[l], i0)]);
        f1 = cmul(f1, lut[P.lut[l].off + lut_index(P.lut[l], i0 + 1)]);
      }
      const T b0 = cmul(a0[u], f0), b1 = cmul(a1[u], f1);
      if constexpr (sizeof(R) == 4) {
        reinterpret_cast<float4*>(st)[p] = make_float4(b0.x, b0.y, b1.x, b1.y);
      } else {
        st[i0] = b0;
        st[i0 + 1] = b1;
      }
    }
  }
}

// ---------------------------------------------------------------- planner
struct Term {
  std::vector<int> bits;                   // global index bits, first = MSB of table index
  std::vector<std::complex<double>> tab;   // 2^|bits| values
};

struct PlannedLut {
  std::vector<int> pos;  // index bit k of the table <- global bit pos[k]
  bool contig = false;
  std::vector<const Term*> members;          // terms the table holds
  std::vector<std::complex<double>> vals;    // filled by realize() once a plan is chosen
};
static size_t lut_size(const PlannedLut& L) { return L.vals.empty() ? (size_t(1) << L.pos.size()) : L.vals.size(); }

static std::complex<double> cis(double t) { return {std::cos(t), std::sin(t)}; }

static int build_terms(int n, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params,
                       std::vector<Term>& terms, std::complex<double>& scalar) {
  scalar = 1.0;
  for (int t = 0; t < n_terms; ++t) {
    const int kind = kinds[t];
    const int a = wires[2 * t], b = wires[2 * t + 1];
    const double* p = params + 8 * t;
    const bool two = (kind == MQ_DIAG_ZZ || kind == MQ_DIAG_CPHASE || kind == MQ_DIAG_CRZ || kind == MQ_DIAG_2Q);
    const bool one = (kind == MQ_DIAG_RZ || kind == MQ_DIAG_PHASE || kind == MQ_DIAG_1Q);
    if (kind == MQ_DIAG_GLOBAL) { scalar *= cis(p[0]); continue; }
    if (!one && !two) return fail(MQ_EINVAL, "unknown diagonal term kind " + std::to_string(kind));
    if (a < 0 || a >= n) return fail(MQ_EINVAL, "diagonal term wire out of range");
    if (two && (b < 0 || b >= n || b == a)) return fail(MQ_EINVAL, "invalid bond (" + std::to_string(a) + ", " + std::to_string(b) + ")");
    Term tm;
    const double th = p[0];
    switch (kind) {
      case MQ_DIAG_ZZ: tm.tab = {cis(-th), cis(th), cis(th), cis(-th)}; break;
      case MQ_DIAG_CPHASE: tm.tab = {1.0, 1.0, 1.0, cis(th)}; break;
      case MQ_DIAG_CRZ: tm.tab = {1.0, 1.0, cis(-th / 2), cis(th / 2)}; break;
      case MQ_DIAG_2Q:
        tm.tab = {{p[0], p[1]}, {p[2], p[3]}, {p[4], p[5]}, {p[6], p[7]}};
        break;
      case MQ_DIAG_RZ: tm.tab = {cis(-th / 2), cis(th / 2)}; break;
      case MQ_DIAG_PHASE: tm.tab = {1.0, cis(th)}; break;
      case MQ_DIAG_1Q: tm.tab = {{p[0], p[1]}, {p[2], p[3]}}; break;
    }
    // CZ is CPHASE(pi): use exact -1 (diag.py:89-98 keeps +-1 exact too)
    if (kind == MQ_DIAG_CPHASE && std::fabs(th - M_PI) < 1e-15) tm.tab[3] = -1.0;
    if (kind == MQ_DIAG_PHASE && std::fabs(th - M_PI) < 1e-15) tm.tab[1] = -1.0;
    tm.bits.push_back(n - 1 - a);
    if (two) tm.bits.push_back(n - 1 - b);
    terms.push_back(std::move(tm));
  }
  return MQ_OK;
}

static std::complex<double> term_value(const Term& tm, const std::vector<int>& pos, uint32_t x) {
  uint32_t idx = 0;
  const int k = (int)tm.bits.size();
  for (int j = 0; j < k; ++j) {
    const int gb = tm.bits[j];
    int lp = (int)(std::find(pos.begin(), pos.end(), gb) - pos.begin());
    const uint32_t bit = (x >> lp) & 1u;
    idx |= bit << (k - 1 - j);
  }
  return tm.tab[idx];
}

static void finalize_lut(PlannedLut& L) {
  const uint32_t sz = 1u << L.pos.size();
  // table-local position of every member bit, found once
  struct Local { int k, lp[2]; const std::complex<double>* tab; };
  std::vector<Local> ms;
  for (const Term* tm : L.members) {
    Local m{(int)tm->bits.size(), {0, 0}, tm->tab.data()};
    for (int j = 0; j < m.k; ++j)
      m.lp[j] = (int)(std::find(L.pos.begin(), L.pos.end(), tm->bits[j]) - L.pos.begin());
    ms.push_back(m);
  }
  L.vals.assign(sz, 1.0);
  for (uint32_t x = 0; x < sz; ++x) {
    std::complex<double> v = 1.0;
    for (const Local& m : ms) {
      uint32_t idx = 0;
      for (int j = 0; j < m.k; ++j) idx |= ((x >> m.lp[j]) & 1u) << (m.k - 1 - j);
      v *= m.tab[idx];
    }
    L.vals[x] = v;
  }
}
// Table values of a chosen plan (planning itself only sizes the tables).
static void realize(std::vector<PlannedLut>& luts) {
  for (auto& L : luts)
    if (L.vals.empty()) finalize_lut(L);
}

// Greedy factorisation with windows of width <= W.
static std::vector<PlannedLut> plan_luts(const std::vector<Term>& terms, int W) {
  std::vector<PlannedLut> luts;
  std::vector<int> local, far;
  for (size_t t = 0; t < terms.size(); ++t) {
    auto [mn, mx] = std::minmax_element(terms[t].bits.begin(), terms[t].bits.end());
    ((*mx - *mn) < W ? local : far).push_back((int)t);
  }
  std::vector<bool> done(terms.size(), false);
  while (true) {
    int s = 1 << 30;
    for (int t : local)
      if (!done[t]) s = std::min(s, *std::min_element(terms[t].bits.begin(), terms[t].bits.end()));
    if (s == (1 << 30)) break;
    std::vector<const Term*> members;
    int hi = s;
    for (int t : local) {
      if (done[t]) continue;
      auto [mn, mx] = std::minmax_element(terms[t].bits.begin(), terms[t].bits.end());
      if (*mn >= s && *mx < s + W) { done[t] = true; members.push_back(&terms[t]); hi = std::max(hi, *mx); }
    }
    PlannedLut L;
    for (int b = s; b <= hi; ++b) L.pos.push_back(b);
    L.contig = true;
    L.members = std::move(members);
    luts.push_back(std::move(L));
  }
  // far pairs: scattered-bit tables
  size_t i = 0;
  while (i < far.size()) {
    PlannedLut L;
    std::vector<const Term*> members;
    while (i < far.size()) {
      std::vector<int> pos = L.pos;
      for (int b : terms[far[i]].bits)
        if (std::find(pos.begin(), pos.end(), b) == pos.end()) pos.push_back(b);
      if ((int)pos.size() > W && !members.empty()) break;
      L.pos = pos;
      members.push_back(&terms[far[i]]);
      ++i;
    }
    std::sort(L.pos.begin(), L.pos.end());
    L.contig = true;
    for (size_t k = 1; k < L.pos.size(); ++k)
      if (L.pos[k] != L.pos[0] + (int)k) L.contig = false;
    L.members = std::move(members);
    luts.push_back(std::move(L));
  }
  return luts;
}

template <typename R>
static int launch_diag_pass(mq_state* h, const std::vector<PlannedLut>& in_luts) {
  using T = V2<R>;
  std::vector<PlannedLut> luts;
  auto has0 = [](const PlannedLut& L) { return std::find(L.pos.begin(), L.pos.end(), 0) != L.pos.end(); };
  for (const auto& L : in_luts)
    if (has0(L) && L.contig && L.pos[0] == 0) luts.push_back(L);
  const bool pair0 = !luts.empty();
  for (const auto& L : in_luts)
    if (has0(L) && !(L.contig && L.pos[0] == 0)) luts.push_back(L);
  const int n_low = (int)luts.size();
  for (const auto& L : in_luts)
    if (!has0(L)) luts.push_back(L);
  auto* P = new DiagParams<R>();
  std::memset(P, 0, sizeof(DiagParams<R>));
  P->n_pairs = (uint32_t)(h->dim() >> 1);
  P->n_luts = (int32_t)luts.size();
  P->n_low = n_low;
  P->pair_lut0 = pair0 ? 1 : 0;
  uint32_t off = 0;
  for (size_t l = 0; l < luts.size(); ++l) {
    const PlannedLut& L = luts[l];
    DiagLut& d = P->lut[l];
    d.off = (uint16_t)off;
    d.nbits = (uint8_t)L.pos.size();
    d.contig = L.contig ? 1 : 0;
    d.shift = (uint8_t)(L.pos.empty() ? 0 : L.pos[0]);
    for (size_t k = 0; k < L.pos.size(); ++k) d.pos[k] = (uint8_t)L.pos[k];
    for (auto v : L.vals) P->e[off++] = mk<R>((R)v.real(), (R)v.imag());
  }
  P->n_entries = off;
  const size_t smem = sizeof(T) * std::max<uint32_t>(off, 1);
  const uint32_t pairs = P->n_pairs;
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((pairs + 255) / 256, (uint64_t)h->num_sms * 8));
  k_diag<R><<<grid, 256, smem, h->stream>>>(reinterpret_cast<T*>(h->cur_buf()), *P);
  delete P;
  MQ_LAUNCHED("k_diag");
  h->launches += 1;
  h->sweeps += 1;
  return MQ_OK;
}

// The diagonal as contiguous-window tables for a tile-sweep epilogue (the
// fused layer of mq_tile.cu): same factorisation as launch_diag_terms, with
// the global phase folded into the first table.  out.n = -1 when no plan with
// <= 8 contiguous windows and <= max_entries entries exists.
int plan_diag_windows(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params,
                      int max_entries, DiagWindows& out) {
  std::vector<Term> terms;
  std::complex<double> scalar;
  int rc = build_terms(h->n, n_terms, kinds, wires, params, terms, scalar);
  if (rc) return rc;
  out = DiagWindows();
  out.n = -1;
  for (int W = 10; W >= 1; --W) {
    std::vector<PlannedLut> luts = plan_luts(terms, W);
    size_t entries = 0;
    bool contig = true;
    for (auto& L : luts) {
      entries += lut_size(L);
      contig = contig && L.contig && !L.pos.empty();
    }
    if (!contig || (int)luts.size() > kMaxLuts) continue;
    if (luts.empty()) {
      PlannedLut L;
      L.pos = {0};
      L.contig = true;
      L.vals = {1.0, 1.0};
      luts.push_back(L);
      entries = 2;
    }
    if ((int)entries > max_entries) continue;
    realize(luts);
    for (auto& v : luts[0].vals) v *= scalar;
    out.n = (int)luts.size();
    uint32_t off = 0;
    for (int l = 0; l < out.n; ++l) {
      out.shift[l] = luts[l].pos[0];
      out.nbits[l] = (int)luts[l].pos.size();
      out.off[l] = (int)off;
      for (auto v : luts[l].vals) {
        out.vals.push_back(v.real());
        out.vals.push_back(v.imag());
      }
      off += (uint32_t)luts[l].vals.size();
    }
    break;
  }
  return MQ_OK;
}

// The diagonal split for a register phase whose register bits are rbits[4]
// (ascending): phase(x) = W(x) * T[c(x)][r(x)] (row c at entry 17c) with r(x) the four register
// bits, c(x) the values of the (at most 3) other bits that share a term with
// a register bit, T the product of those terms, and W the remaining terms as
// contiguous windows that do not read the register bits (so W can be taken
// at the register group's base index).  out.n = -1 when this does not fit.
int plan_diag_register(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params,
                       const int* rbits, int max_entries, DiagRegister& out) {
  std::vector<Term> terms;
  std::complex<double> scalar;
  int rc = build_terms(h->n, n_terms, kinds, wires, params, terms, scalar);
  if (rc) return rc;
  out = DiagRegister();
  out.win.n = -1;
  auto is_reg = [&](int b) { return b == rbits[0] || b == rbits[1] || b == rbits[2] || b == rbits[3]; };
  std::vector<Term> group, reg;
  std::vector<int> cross;
  for (const Term& t : terms) {
    bool touches = false;
    for (int b : t.bits) touches = touches || is_reg(b);
    if (!touches) { group.push_back(t); continue; }
    reg.push_back(t);
    for (int b : t.bits)
      if (!is_reg(b) && std::find(cross.begin(), cross.end(), b) == cross.end()) cross.push_back(b);
  }
  if (cross.size() > 3) return MQ_OK;
  std::sort(cross.begin(), cross.end());
  // T[c][r]: value bit k of r = global bit rbits[k], bit j of c = cross[j]
  std::vector<int> pos = {rbits[0], rbits[1], rbits[2], rbits[3]};
  for (int b : cross) pos.push_back(b);
  const uint32_t nt = 1u << pos.size();
  std::vector<std::complex<double>> T(nt, scalar);
  for (uint32_t x = 0; x < nt; ++x)
    for (const Term& t : reg) T[x] *= term_value(t, pos, x);
  // W: contiguous windows over the group terms
  std::vector<PlannedLut> luts;
  bool ok = false;
  for (int W = 10; W >= 1 && !ok; --W) {
    luts = plan_luts(group, W);
    size_t entries = (nt / 16) * 17;
    bool contig = true;
    for (auto& L : luts) {
      entries += lut_size(L);
      contig = contig && L.contig && !L.pos.empty();
    }
    ok = contig && (int)luts.size() <= kMaxLuts && (int)entries <= max_entries;
  }
  if (!ok) return MQ_OK;
  realize(luts);
  out.nc = (int)cross.size();
  for (int j = 0; j < out.nc; ++j) out.cbit[j] = cross[j];
  out.win.n = (int)luts.size();
  uint32_t off = 0;
  for (int l = 0; l < out.win.n; ++l) {
    out.win.shift[l] = luts[l].pos[0];
    out.win.nbits[l] = (int)luts[l].pos.size();
    out.win.off[l] = (int)off;
    for (auto v : luts[l].vals) {
      out.win.vals.push_back(v.real());
      out.win.vals.push_back(v.imag());
    }
    off += (uint32_t)luts[l].vals.size();
  }
  // rows of 16 at a stride of 17 entries: lanes that read rows c and c' of
  // the same register pattern hit different shared-memory banks
  out.t_off = (int)off;
  for (uint32_t c = 0; c < nt / 16; ++c) {
    for (uint32_t r = 0; r < 16; ++r) {
      out.win.vals.push_back(T[c * 16 + r].real());
      out.win.vals.push_back(T[c * 16 + r].imag());
    }
    out.win.vals.push_back(1.0);
    out.win.vals.push_back(0.0);
  }
  return MQ_OK;
}

int launch_diag_terms(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params) {
  std::vector<Term> terms;
  std::complex<double> scalar;
  int rc = build_terms(h->n, n_terms, kinds, wires, params, terms, scalar);
  if (rc) return rc;
  if (terms.empty() && scalar == std::complex<double>(1.0, 0.0)) return MQ_OK;
  const int cap = h->dtype == MQ_C64 ? DiagCap<float>::v : DiagCap<double>::v;
  std::vector<PlannedLut> luts;
  for (int W = 10; W >= 1; --W) {
    luts = plan_luts(terms, W);
    size_t entries = 0;
    for (auto& L : luts) entries += lut_size(L);
    if ((int)luts.size() <= kMaxLuts && (int)entries <= cap) break;
    if (W == 1) break;  // fall through to multi-pass below
  }
  if (luts.empty()) {
    PlannedLut L;
    L.contig = true;
    L.vals = {1.0};
    luts.push_back(L);
  }
  realize(luts);
  for (auto& v : luts[0].vals) v *= scalar;
  // Split into passes that respect the parameter-block capacity.
  size_t i = 0;
  while (i < luts.size()) {
    std::vector<PlannedLut> pass;
    size_t entries = 0;
    while (i < luts.size() && (int)pass.size() < kMaxLuts && (int)(entries + luts[i].vals.size()) <= cap) {
      entries += luts[i].vals.size();
      pass.push_back(luts[i]);
      ++i;
    }
    if (pass.empty()) return fail(MQ_EUNSUPPORTED, "diagonal table exceeds capacity");
    rc = (h->dtype == MQ_C64) ? launch_diag_pass<float>(h, pass) : launch_diag_pass<double>(h, pass);
    if (rc) return rc;
  }
  return MQ_OK;
}

}  // namespace mq
