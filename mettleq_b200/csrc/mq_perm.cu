// GF(2) affine permutation layer (d): out[y] = in[A y ^ c].
//
// Replaces xor_affine_gather / the X-only flip fast path
// (shaders/xor_affine.py:22-40, 79-116).  The reference computes one source
// index per thread with n popcount parities and gathers 8-byte amplitudes
// from arbitrary addresses, so a map that mixes high bits reads one 32-byte
// sector per 8 useful bytes.
//
// Here the permutation is done by tiles that are coalesced on BOTH sides.
// With P low passenger bits (16 amplitudes = 128 B):
//   S_in  = span(e_0..e_{P-1}, A e_0..A e_{P-1}), padded with unit vectors to
//           dimension D (1024 amplitudes per tile);
//   S_out = A^{-1} S_in, which contains e_0..e_{P-1} by construction.
// Each output coset y in h ^ S_out reads from the input coset A h ^ c ^ S_in:
// both cosets are unions of 128-byte runs.  A CTA loads the input coset in
// address order into shared memory and writes the output coset in address
// order, mapping slots through the D x D coordinate matrix of A on the tile.
// Any invertible A (CNOT/X/SWAP runs, SWAP-network wire permutations, random
// GF(2) layers) costs exactly one read and one write of the state.
#include <algorithm>
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
};

// Persistent CTAs stream cosets through two shared-memory buffers: the input
// coset of tile t+grid is fetched with cp.async while tile t is written out.
template <typename R>
__global__ void __launch_bounds__(256) k_perm(const V2<R>* __restrict__ in, V2<R>* __restrict__ out,
                                              const __grid_constant__ PermParams P) {
  using T = V2<R>;
  __shared__ __align__(16) T buf[2][1024];
  __shared__ uint32_t t_in[2][32], t_out[2][32], t_tab[2][32];
  const int tid = threadIdx.x;
  const int D = P.D;
  const int dlo = D < 5 ? D : 5;
  const int dhi = D - dlo;
  if (tid < 32) {
    uint32_t a = 0, b = 0, c = 0, x = 0, y = 0, z = 0;
    for (int k = 0; k < dlo; ++k)
      if (tid & (1 << k)) { a ^= P.lin_in[k]; b ^= P.lin_out[k]; c ^= P.tab[k]; }
    for (int k = 0; k < dhi; ++k)
      if (tid & (1 << k)) { x ^= P.lin_in[dlo + k]; y ^= P.lin_out[dlo + k]; z ^= P.tab[dlo + k]; }
    t_in[0][tid] = a; t_out[0][tid] = b; t_tab[0][tid] = c;
    t_in[1][tid] = x; t_out[1][tid] = y; t_tab[1][tid] = z;
  }
  __syncthreads();
  const uint32_t E = 1u << D;
  const uint32_t lomask = (1u << dlo) - 1u;
  auto h_of = [&](uint32_t tile, bool input) -> uint32_t {
    uint32_t h = input ? P.c : 0u;
    for (int k = 0; k < P.n_comp; ++k)
      if ((tile >> k) & 1u) h ^= input ? P.comp_in[k] : P.comp_out[k];
    return h;
  };
  uint32_t tile = blockIdx.x;
  if (tile < P.n_tiles) {
    const uint32_t h_in = h_of(tile, true);
    for (uint32_t e = tid; e < E; e += blockDim.x)
      cp_async<sizeof(T)>(smem_u32(&buf[0][e]), in + (h_in ^ t_in[0][e & lomask] ^ t_in[1][e >> dlo]));
  }
  cp_async_commit();
  for (int it = 0; tile < P.n_tiles; tile += gridDim.x, ++it) {
    const uint32_t next = tile + gridDim.x;
    if (next < P.n_tiles) {
      const uint32_t h_in = h_of(next, true);
      T* nb = buf[(it + 1) & 1];
      for (uint32_t e = tid; e < E; e += blockDim.x)
        cp_async<sizeof(T)>(smem_u32(&nb[e]), in + (h_in ^ t_in[0][e & lomask] ^ t_in[1][e >> dlo]));
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const T* cb = buf[it & 1];
    const uint32_t h_out = h_of(tile, false);
    for (uint32_t e = tid; e < E; e += blockDim.x) {
      const uint32_t y = h_out ^ t_out[0][e & lomask] ^ t_out[1][e >> dlo];
      const uint32_t slot = t_tab[0][e & lomask] ^ t_tab[1][e >> dlo];
      out[y] = cb[slot];
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

template <typename R>
static int launch_perm_t(mq_state* h, const PermParams& P) {
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(P.n_tiles, (uint64_t)h->num_sms * 8));
  const V2<R>* src = reinterpret_cast<const V2<R>*>(h->buf[h->cur]);
  V2<R>* dst = reinterpret_cast<V2<R>*>(h->buf[1 - h->cur]);
  k_perm<R><<<grid, 256, 0, h->stream>>>(src, dst, P);
  MQ_LAUNCHED("k_perm");
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
  const int pas = std::min(4, D / 2);
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
  return h->dtype == MQ_C64 ? launch_perm_t<float>(h, P) : launch_perm_t<double>(h, P);
}

}  // namespace mq
