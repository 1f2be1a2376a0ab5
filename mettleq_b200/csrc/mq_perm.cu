// GF(2) affine permutation layer (d): out[y] = in[A y ^ c].
//
// Replaces xor_affine_gather / the X-only flip fast path
// (shaders/xor_affine.py:22-40, 79-116).  The reference computes one source
// index per thread with n popcount parities and gathers 8-byte amplitudes
// from arbitrary addresses, so a map that mixes high bits reads one 32-byte
// sector per 8 useful bytes.
//
// Here the permutation is done by tiles that are coalesced on BOTH sides.
// With P low passenger bits (32 amplitudes = 256 B by default):
//   S_in  = span(e_0..e_{P-1}, A e_0..A e_{P-1}), padded with unit vectors to
//           dimension D (1024 amplitudes per tile);
//   S_out = A^{-1} S_in, which contains e_0..e_{P-1} by construction.
// Each output coset y in h ^ S_out reads from the input coset A h ^ c ^ S_in:
// both cosets are unions of 2^P-amplitude runs.  A CTA loads the input coset in
// address order into shared memory and writes the output coset in address
// order, mapping slots through the D x D coordinate matrix of A on the tile.
// Any invertible A (CNOT/X/SWAP runs, SWAP-network wire permutations, random
// GF(2) layers) costs exactly one read and one write of the state.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

struct PermParams {
  uint32_t n_tiles;
  uint32_t c;
  uint8_t n, D, n_comp, pad;
  uint32_t comp_out[32];
  uint32_t comp_in[32];
  uint32_t lin_in[16];
  uint32_t lin_out[16];
  uint32_t tab[16];
  // coset offsets of tile t as XORs of byte tables: h_in(t) = c ^ XOR_k
  // hin[k][byte k of t], h_out likewise (read at CTA-uniform indices)
  uint32_t hin[4][256];
  uint32_t hout[4][256];
};

static_assert(sizeof(PermParams) <= 32000, "kernel parameter block too large");

// Persistent CTAs stream cosets through two shared-memory buffers: the input
// coset of tile t+grid is fetched with cp.async while tile t is written out.
// Tile elements e = tid + NT*j.  All index maps are GF(2)-linear in e, so a
// thread's lane/warp part is combined once and each element adds one
// CTA-uniform term.  Only basis vector 0 (= e_0) has index bit 0 set, so
// input pairs (e, e^1) are one aligned 16-byte chunk, stored in shared
// memory with the coset's bit-0 offset `flip` folded into the slot index.
template <typename R, int D>
__global__ void __launch_bounds__(256) k_perm(const V2<R>* __restrict__ in, V2<R>* __restrict__ out,
                                              const __grid_constant__ PermParams P) {
  using T = V2<R>;
  constexpr int E = 1 << D;
  constexpr int NT = E < 256 ? E : 256;
  constexpr int EPT = E / NT;
  constexpr bool PAIRS = (sizeof(T) == 8) && D >= 1;  // 16-byte input chunks
  constexpr int CPT = PAIRS ? (EPT >= 2 ? EPT / 2 : 1) : EPT;
  __shared__ __align__(16) T buf[2][E < 2 ? 2 : E];
  __shared__ uint32_t t_in[E], t_out[E], t_tab[E];
  const int tid = threadIdx.x;
  // full linear tables over the D tile coordinates (E <= 1024 entries)
  for (int e = tid; e < E; e += NT) {
    uint32_t a = 0, b = 0, c = 0;
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (e & (1 << k)) { a ^= P.lin_in[k]; b ^= P.lin_out[k]; c ^= P.tab[k]; }
    t_in[e] = a; t_out[e] = b; t_tab[e] = c;
  }
  __syncthreads();
  auto h_in_of = [&](uint32_t t) -> uint32_t {
    return P.c ^ P.hin[0][t & 255u] ^ P.hin[1][(t >> 8) & 255u] ^ P.hin[2][(t >> 16) & 255u] ^ P.hin[3][t >> 24];
  };
  auto h_out_of = [&](uint32_t t) -> uint32_t {
    return P.hout[0][t & 255u] ^ P.hout[1][(t >> 8) & 255u] ^ P.hout[2][(t >> 16) & 255u] ^ P.hout[3][t >> 24];
  };
  // per-thread parts: input chunks c = tid + NT*j cover elements 2c, 2c+1
  auto issue = [&](uint32_t h_in, int which) {
    const uint32_t sb = smem_u32(&buf[which][0]);
    if constexpr (PAIRS) {
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const uint32_t c = (uint32_t)tid + (uint32_t)(NT * j);
        if (2 * c < (uint32_t)E) {
          const uint32_t src = (h_in ^ t_in[2 * c]) & ~1u;
          cp_async<16>(sb + 16u * c, in + src);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < EPT; ++j) {
        const uint32_t e = (uint32_t)tid + (uint32_t)(NT * j);
        cp_async<sizeof(T)>(sb + (uint32_t)sizeof(T) * e, in + (h_in ^ t_in[e]));
      }
    }
  };
  uint32_t tile = blockIdx.x;
  uint32_t h_cur = tile < P.n_tiles ? h_in_of(tile) : 0u;
  if (tile < P.n_tiles) issue(h_cur, 0);
  cp_async_commit();
  for (int it = 0; tile < P.n_tiles; tile += gridDim.x, ++it) {
    const uint32_t next = tile + gridDim.x;
    const uint32_t h_next = next < P.n_tiles ? h_in_of(next) : 0u;
    if (next < P.n_tiles) issue(h_next, (it + 1) & 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const T* cb = buf[it & 1];
    const uint32_t h_out = h_out_of(tile);
    const uint32_t flip = PAIRS ? (h_cur & 1u) : 0u;
    h_cur = h_next;
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      const uint32_t e = (uint32_t)tid + (uint32_t)(NT * j);
      out[h_out ^ t_out[e]] = cb[t_tab[e] ^ flip];
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

// ------------------------------------------------------------ GF(2) algebra
namespace {
struct Echelon {
  uint32_t vec[32] = {0};
  uint32_t comb[32] = {0};
  int rank = 0;
  // Insert x tagged as basis element `tag`; false if dependent.
  bool add(uint32_t x, int tag) {
    uint32_t c = (tag >= 0) ? (1u << tag) : 0u;
    for (int p = 31; p >= 0; --p) {
      if (!((x >> p) & 1u)) continue;
      if (vec[p]) { x ^= vec[p]; c ^= comb[p]; }
      else { vec[p] = x; comb[p] = c; ++rank; return true; }
    }
    return false;
  }
  bool contains(uint32_t x) const {
    for (int p = 31; p >= 0; --p) {
      if (!((x >> p) & 1u)) continue;
      if (!vec[p]) return false;
      x ^= vec[p];
    }
    return true;
  }
  uint32_t coords(uint32_t x) const {
    uint32_t c = 0;
    for (int p = 31; p >= 0; --p) {
      if (!((x >> p) & 1u)) continue;
      x ^= vec[p];
      c ^= comb[p];
    }
    return c;
  }
};

uint32_t apply_cols(const uint32_t* cols, int n, uint32_t x) {
  uint32_t y = 0;
  for (int j = 0; j < n; ++j)
    if ((x >> j) & 1u) y ^= cols[j];
  return y;
}
}  // namespace

bool gf2_invert(int n, const uint32_t* cols, uint32_t* inv_cols) {
  // Gauss-Jordan on [A | I] with columns as bit masks (row = bit position).
  uint32_t rows[32], inv[32];
  for (int r = 0; r < n; ++r) {
    rows[r] = 0;
    inv[r] = 1u << r;
    for (int j = 0; j < n; ++j) rows[r] |= ((cols[j] >> r) & 1u) << j;
  }
  for (int col = 0; col < n; ++col) {
    int piv = -1;
    for (int r = col; r < n; ++r)
      if ((rows[r] >> col) & 1u) { piv = r; break; }
    if (piv < 0) return false;
    std::swap(rows[col], rows[piv]);
    std::swap(inv[col], inv[piv]);
    for (int r = 0; r < n; ++r)
      if (r != col && ((rows[r] >> col) & 1u)) { rows[r] ^= rows[col]; inv[r] ^= inv[col]; }
  }
  // inv rows are rows of A^{-1}; convert to columns
  for (int j = 0; j < n; ++j) {
    inv_cols[j] = 0;
    for (int r = 0; r < n; ++r) inv_cols[j] |= ((inv[r] >> j) & 1u) << r;
  }
  return true;
}

template <typename R, int D>
static int launch_perm_d(mq_state* h, const PermParams& P) {
  constexpr int E = 1 << D;
  constexpr int NT = E < 256 ? E : 256;
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(P.n_tiles, (uint64_t)h->num_sms * 8));
  const V2<R>* src = reinterpret_cast<const V2<R>*>(h->buf[h->cur]);
  V2<R>* dst = reinterpret_cast<V2<R>*>(h->buf[1 - h->cur]);
  k_perm<R, D><<<grid, NT, 0, h->stream>>>(src, dst, P);
  MQ_LAUNCHED("k_perm");
  return MQ_OK;
}

template <typename R>
static int launch_perm_t(mq_state* h, const PermParams& P) {
  int rc = MQ_EUNSUPPORTED;
  switch (P.D) {
    case 1: rc = launch_perm_d<R, 1>(h, P); break;
    case 2: rc = launch_perm_d<R, 2>(h, P); break;
    case 3: rc = launch_perm_d<R, 3>(h, P); break;
    case 4: rc = launch_perm_d<R, 4>(h, P); break;
    case 5: rc = launch_perm_d<R, 5>(h, P); break;
    case 6: rc = launch_perm_d<R, 6>(h, P); break;
    case 7: rc = launch_perm_d<R, 7>(h, P); break;
    case 8: rc = launch_perm_d<R, 8>(h, P); break;
    case 9: rc = launch_perm_d<R, 9>(h, P); break;
    case 10: rc = launch_perm_d<R, 10>(h, P); break;
    default: return fail(MQ_EUNSUPPORTED, "permutation tile size not instantiated");
  }
  if (rc) return rc;
  h->cur = 1 - h->cur;
  h->launches += 1;
  h->sweeps += 1;
  return MQ_OK;
}

int launch_affine_cols(mq_state* h, const uint32_t* cols, uint32_t c) {
  const int n = h->n;
  uint32_t inv[32];
  if (!gf2_invert(n, cols, inv)) return fail(MQ_EINVAL, "affine map is not invertible over GF(2)");
  int rc = ensure_alt(h);
  if (rc) return rc;
  const int D = std::min(10, n);
  // passenger bits: both cosets are unions of 2^pas-amplitude runs (5: 256
  // bytes, all of D = 10 then spanned by e_j and A e_j, j < 5; the random
  // 30-qubit GF(2) layer measured 3.13 ms against 3.57-3.60 ms with 4, 128
  // bytes); MQ_PERM_PASSENGERS overrides
  const char* pv = std::getenv("MQ_PERM_PASSENGERS");
  const int pas_want = (pv && *pv) ? std::max(1, std::min(5, std::atoi(pv))) : 5;
  const int pas = std::min(pas_want, D / 2);
  // input-side tile basis
  Echelon ein;
  std::vector<uint32_t> vin;
  for (int j = 0; j < pas; ++j) { ein.add(1u << j, (int)vin.size()); vin.push_back(1u << j); }
  for (int j = 0; j < pas && (int)vin.size() < D; ++j) {
    const uint32_t v = cols[j];
    if (ein.add(v, (int)vin.size())) vin.push_back(v);
  }
  for (int j = 0; j < n && (int)vin.size() < D; ++j) {
    if (ein.add(1u << j, (int)vin.size())) vin.push_back(1u << j);
  }
  // output-side tile basis: A^{-1} S_in, listed with e_0..e_{pas-1} first
  Echelon eout;
  std::vector<uint32_t> vout;
  for (int j = 0; j < pas; ++j) { eout.add(1u << j, (int)vout.size()); vout.push_back(1u << j); }
  for (uint32_t v : vin) {
    const uint32_t w = apply_cols(inv, n, v);
    if ((int)vout.size() < D && eout.add(w, (int)vout.size())) vout.push_back(w);
  }
  if ((int)vin.size() != D || (int)vout.size() != D) return fail(MQ_EDEVICE, "affine tile basis construction failed");
  // Clear index bit 0 from every basis vector but the first (which is e_0),
  // so that tile coordinate 0 alone decides the bit-0 parity of an address.
  if (pas >= 1) {
    Echelon e2in, e2out;
    for (int k = 1; k < D; ++k) {
      if (vin[k] & 1u) vin[k] ^= vin[0];
      if (vout[k] & 1u) vout[k] ^= vout[0];
    }
    for (int k = 0; k < D; ++k) { e2in.add(vin[k], k); e2out.add(vout[k], k); }
    ein = e2in;
    eout = e2out;
  }
  PermParams P;
  std::memset(&P, 0, sizeof(P));
  P.n = (uint8_t)n;
  P.D = (uint8_t)D;
  P.c = c;
  for (int k = 0; k < D; ++k) {
    P.lin_in[k] = vin[k];
    P.lin_out[k] = vout[k];
    P.tab[k] = ein.coords(apply_cols(cols, n, vout[k]));
  }
  // complement of S_out enumerates the tiles
  int nc = 0;
  for (int j = 0; j < n && nc < n - D; ++j) {
    if (eout.add(1u << j, -1)) {
      P.comp_out[nc] = 1u << j;
      P.comp_in[nc] = apply_cols(cols, n, 1u << j);
      ++nc;
    }
  }
  if (nc != n - D) return fail(MQ_EDEVICE, "affine coset basis construction failed");
  P.n_comp = (uint8_t)nc;
  P.n_tiles = 1u << nc;
  for (int k = 0; k < 4; ++k)
    for (uint32_t x = 0; x < 256; ++x) {
      uint32_t a = 0, b = 0;
      for (int bit = 0; bit < 8; ++bit)
        if (((x >> bit) & 1u) && 8 * k + bit < nc) { a ^= P.comp_in[8 * k + bit]; b ^= P.comp_out[8 * k + bit]; }
      P.hin[k][x] = a;
      P.hout[k][x] = b;
    }
  return h->dtype == MQ_C64 ? launch_perm_t<float>(h, P) : launch_perm_t<double>(h, P);
}

}  // namespace mq
