// Probabilities, seeded sampling and Pauli expectations (e).
//
// Replaces the reference's MLX library calls on this path:
//   probabilities_array: |a|^2, transpose, sum           (sim.py:322-343)
//   sample_array: log(max(p,1e-30)) + mx.random.categorical (sim.py:383-419)
//   pauli_product_expectations: one functional copy per word (_common.py:384-427)
//
// Every reduction has a fixed order so results are bit-reproducible run to
// run and can be restated exactly on the CPU:
//   * p_i = re^2 + im^2 in float64 with explicitly rounded operations;
//   * block sums: 32 lanes add entries lane, lane+32, ... sequentially, then
//     an XOR butterfly over the lanes;
//   * longer sums are sequential over <= 1024 partial sums, in two levels.
// Sampling uses Philox4x32-10 (counter = shot + stream_offset, key = seed),
// u = 53 random bits / 2^53, target t = u * total, a binary search over block
// offsets and a sequential running sum inside the chosen block.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

constexpr uint32_t kBlock = 1024;
constexpr uint32_t kSuper = 1024;

template <typename R>
__device__ __forceinline__ double amp2(V2<R> a) {
  const double re = (double)a.x, im = (double)a.y;
  return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}

template <typename R> struct StateSrc {
  const V2<R>* st;
  __device__ __forceinline__ double operator()(uint32_t i) const { return amp2<R>(st[i]); }
};
struct VecSrc {
  const double* q;
  __device__ __forceinline__ double operator()(uint32_t i) const { return q[i]; }
};

// -------------------------------------------------------------- full |a|^2
template <typename R, typename O>
__global__ void k_amp2_out(const V2<R>* __restrict__ st, O* __restrict__ out, uint32_t dim) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) out[i] = (O)amp2<R>(st[i]);
}

// -------------------------------------------------------------- block sums
template <typename Src>
__global__ void k_block_sums(Src src, uint32_t bs, uint32_t nb, double* __restrict__ S) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nb) return;
  const uint32_t base = warp * bs;
  double acc = 0.0;
  for (uint32_t j = lane; j < bs; j += 32) acc = __dadd_rn(acc, src(base + j));
#pragma unroll
  for (int off = 16; off; off >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, off));
  if (lane == 0) S[warp] = acc;
}

// Marginal chunk sums in bucket-major order: j -> global index by three
// deposit tables (the selected/remaining bit permutation is linear).
template <typename R>
__global__ void k_chunk_sums(const V2<R>* __restrict__ st, const uint32_t* __restrict__ dep, uint32_t cs,
                             uint32_t nc, double* __restrict__ D) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nc) return;
  const uint32_t base = warp * cs;
  double acc = 0.0;
  for (uint32_t jj = lane; jj < cs; jj += 32) {
    const uint32_t j = base + jj;
    const uint32_t g = dep[j & 4095u] | dep[4096 + ((j >> 12) & 4095u)] | dep[8192 + (j >> 24)];
    acc = __dadd_rn(acc, amp2<R>(st[g]));
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, off));
  if (lane == 0) D[warp] = acc;
}

// Sequential sums of consecutive runs: out[t] = sum of in[t*len .. t*len+cnt)
// with cnt = min(len, total - t*len) restricted to the run's own group.
__global__ void k_seq_sums(const double* __restrict__ in, uint32_t group_len, uint32_t run_len,
                           uint32_t runs_per_group, uint32_t n_runs, double* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_runs) return;
  const uint32_t g = t / runs_per_group, r = t % runs_per_group;
  const uint32_t start = g * group_len + r * run_len;
  const uint32_t end = min(start + run_len, (g + 1) * group_len);
  double acc = 0.0;
  for (uint32_t i = start; i < end; ++i) acc = __dadd_rn(acc, in[i]);
  out[t] = acc;
}

// Exclusive running sums inside super-blocks of kSuper blocks.
__global__ void k_local_prefix(const double* __restrict__ S, uint32_t nb, double* __restrict__ L,
                               double* __restrict__ T, int32_t* __restrict__ LP) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t start = g * kSuper;
  if (start >= nb) return;
  const uint32_t end = min(nb, start + kSuper);
  double e = 0.0;
  int32_t last = -1;
  for (uint32_t b = start; b < end; ++b) {
    L[b] = e;
    const double s = S[b];
    e = __dadd_rn(e, s);
    if (s > 0.0) last = (int32_t)b;
  }
  T[g] = e;
  LP[g] = last;
}

struct SampleMeta {
  double total;
  int32_t last_block;
  int32_t pad;
};

__global__ void k_super_prefix(const double* __restrict__ T, const int32_t* __restrict__ LP, uint32_t ng,
                               double* __restrict__ E, SampleMeta* __restrict__ meta) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double acc = 0.0;
  int32_t last = -1;
  for (uint32_t g = 0; g < ng; ++g) {
    E[g] = acc;
    acc = __dadd_rn(acc, T[g]);
    last = max(last, LP[g]);
  }
  meta->total = acc;
  meta->last_block = last;
}

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k.x += W0; k.y += W1; }
    const uint32_t lo0 = M0 * c.x, hi0 = __umulhi(M0, c.x);
    const uint32_t lo1 = M1 * c.z, hi1 = __umulhi(M1, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
  }
  return c;
}

template <typename Src>
__global__ void k_draw(Src src, uint32_t bs, uint32_t nb, const double* __restrict__ L, const double* __restrict__ E,
                       const SampleMeta* __restrict__ meta, uint64_t seed, uint64_t offset, int64_t shots,
                       int64_t* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= shots) return;
  const uint64_t ctr = (uint64_t)s + offset;
  const uint4 x = philox4x32_10(make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u),
                                make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  const uint64_t bits = ((((uint64_t)x.y) << 32) | x.x) >> 11;
  const double u = (double)bits * 0x1p-53;
  const double t = __dmul_rn(u, meta->total);
  uint32_t lo = 0, hi = nb - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    const double c = __dadd_rn(E[mid / kSuper], L[mid]);
    if (c <= t) lo = mid; else hi = mid - 1;
  }
  uint32_t b = lo;
  if ((int32_t)b > meta->last_block) b = (uint32_t)max(meta->last_block, 0);
  double r = __dadd_rn(E[b / kSuper], L[b]);
  const uint32_t base = b * bs;
  int64_t found = -1;
  for (uint32_t i = 0; i < bs; ++i) {
    r = __dadd_rn(r, src(base + i));
    if (r > t) { found = i; break; }
  }
  if (found < 0) {
    for (int64_t i = (int64_t)bs - 1; i >= 0; --i)
      if (src(base + (uint32_t)i) > 0.0) { found = i; break; }
    if (found < 0) found = 0;
  }
  out[s] = (int64_t)base + found;
}

// -------------------------------------------------------------- Pauli words
constexpr int kWords = 8;
struct PauliParams {
  uint32_t dim;
  uint32_t x;
  int32_t nw;
  uint32_t z[kWords];
};

template <typename R>
__global__ void __launch_bounds__(256) k_pauli(const V2<R>* __restrict__ st, const __grid_constant__ PauliParams P,
                                               double2* __restrict__ partials) {
  __shared__ double2 red[8][kWords];
  double2 acc[kWords];
#pragma unroll
  for (int w = 0; w < kWords; ++w) acc[w] = make_double2(0.0, 0.0);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.dim; i += stride) {
    const V2<R> a = st[i], b = st[i ^ P.x];
    const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
    const double vr = __dadd_rn(__dmul_rn(br, ar), __dmul_rn(bi, ai));
    const double vi = __dsub_rn(__dmul_rn(br, ai), __dmul_rn(bi, ar));
#pragma unroll
    for (int w = 0; w < kWords; ++w) {
      if (w >= P.nw) break;
      if (__popc(i & P.z[w]) & 1) { acc[w].x = __dsub_rn(acc[w].x, vr); acc[w].y = __dsub_rn(acc[w].y, vi); }
      else { acc[w].x = __dadd_rn(acc[w].x, vr); acc[w].y = __dadd_rn(acc[w].y, vi); }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int w = 0; w < kWords; ++w) {
    double xr = acc[w].x, xi = acc[w].y;
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      xr = __dadd_rn(xr, __shfl_xor_sync(0xffffffffu, xr, off));
      xi = __dadd_rn(xi, __shfl_xor_sync(0xffffffffu, xi, off));
    }
    if (lane == 0) red[warp][w] = make_double2(xr, xi);
  }
  __syncthreads();
  if (threadIdx.x < kWords) {
    const int w = threadIdx.x;
    double xr = 0.0, xi = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { xr = __dadd_rn(xr, red[k][w].x); xi = __dadd_rn(xi, red[k][w].y); }
    partials[blockIdx.x * kWords + w] = make_double2(xr, xi);
  }
}

// ================================================================ host side
static uint32_t grid_for(uint64_t threads, int bs) { return (uint32_t)std::max<uint64_t>(1, (threads + bs - 1) / bs); }

// Deterministic marginal over `wires` (k < n or permuted order) into dev q[2^k].
static int marginal_device(mq_state* h, const int32_t* wires, int k, double* q, double* work, uint32_t* dep) {
  const int n = h->n;
  // deposit tables: bucket-major index j -> global index
  std::vector<int> img(n);  // j bit t -> global bit img[t]
  std::vector<bool> sel(n, false);
  for (int t = 0; t < k; ++t) sel[n - 1 - wires[t]] = true;
  int t = 0;
  for (int b = 0; b < n; ++b)
    if (!sel[b]) img[t++] = b;  // remaining bits ascending = low j bits
  for (int s = k - 1; s >= 0; --s) img[t++] = n - 1 - wires[s];  // first wire = MSB of bucket
  std::vector<uint32_t> tab(8192 + 256, 0);
  for (uint32_t x = 0; x < 4096; ++x) {
    uint32_t a = 0, b = 0;
    for (int bit = 0; bit < 12; ++bit) {
      if (!((x >> bit) & 1u)) continue;
      if (bit < n) a |= 1u << img[bit];
      if (bit + 12 < n) b |= 1u << img[bit + 12];
    }
    tab[x] = a;
    tab[4096 + x] = b;
  }
  for (uint32_t x = 0; x < 256; ++x) {
    uint32_t c = 0;
    for (int bit = 0; bit < 8; ++bit)
      if (((x >> bit) & 1u) && bit + 24 < n) c |= 1u << img[bit + 24];
    tab[8192 + x] = c;
  }
  MQ_CUDA(cudaMemcpyAsync(dep, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, h->stream));
  const uint64_t bucket_len = uint64_t(1) << (n - k);
  const uint32_t cs = (uint32_t)std::min<uint64_t>(kBlock, bucket_len);
  const uint32_t nc = (uint32_t)((uint64_t(1) << n) / cs);
  const uint32_t ncb = (uint32_t)(bucket_len / cs);      // chunks per bucket
  const uint32_t nsb = (ncb + kSuper - 1) / kSuper;       // super-chunks per bucket
  const uint32_t nbk = 1u << k;
  double* D = work;
  double* Pp = work + nc;
  if (h->dtype == MQ_C64)
    k_chunk_sums<float><<<grid_for((uint64_t)nc * 32, 256), 256, 0, h->stream>>>((const float2*)h->cur_buf(), dep, cs, nc, D);
  else
    k_chunk_sums<double><<<grid_for((uint64_t)nc * 32, 256), 256, 0, h->stream>>>((const double2*)h->cur_buf(), dep, cs, nc, D);
  MQ_LAUNCHED("k_chunk_sums");
  k_seq_sums<<<grid_for((uint64_t)nbk * nsb, 128), 128, 0, h->stream>>>(D, ncb, kSuper, nsb, nbk * nsb, Pp);
  MQ_LAUNCHED("k_seq_sums");
  k_seq_sums<<<grid_for(nbk, 128), 128, 0, h->stream>>>(Pp, nsb, nsb, 1, nbk, q);
  MQ_LAUNCHED("k_seq_sums");
  h->launches += 3;
  h->sweeps += 1;
  return MQ_OK;
}

static bool natural_order(int n, const int32_t* wires, int k) {
  if (!wires || k < 0) return true;
  if (k != n) return false;
  for (int i = 0; i < n; ++i)
    if (wires[i] != i) return false;
  return true;
}

static int check_wires(int n, const int32_t* wires, int k) {
  if (!wires || k < 0) return MQ_OK;
  if (k > n) return fail(MQ_EINVAL, "more wires than qubits");
  std::vector<bool> seen(n, false);
  for (int i = 0; i < k; ++i) {
    if (wires[i] < 0 || wires[i] >= n) return fail(MQ_EINVAL, "Qubit index out of range");
    if (seen[wires[i]]) return fail(MQ_EINVAL, "Duplicate qubit indices");
    seen[wires[i]] = true;
  }
  return MQ_OK;
}

// |a|^2 of every amplitude, natural order, into out (device memory of the
// handle's device), asynchronously on the handle's stream.
int run_probabilities_device(mq_state* h, int out_dtype, void* out) {
  const uint32_t dim = (uint32_t)h->dim();
  const uint32_t grid = (uint32_t)std::min<uint64_t>((dim + 255) / 256, (uint64_t)h->num_sms * 16);
  if (h->dtype == MQ_C64) {
    if (out_dtype == 0) k_amp2_out<float, float><<<grid, 256, 0, h->stream>>>((const float2*)h->cur_buf(), (float*)out, dim);
    else k_amp2_out<float, double><<<grid, 256, 0, h->stream>>>((const float2*)h->cur_buf(), (double*)out, dim);
  } else {
    if (out_dtype == 0) k_amp2_out<double, float><<<grid, 256, 0, h->stream>>>((const double2*)h->cur_buf(), (float*)out, dim);
    else k_amp2_out<double, double><<<grid, 256, 0, h->stream>>>((const double2*)h->cur_buf(), (double*)out, dim);
  }
  MQ_LAUNCHED("k_amp2_out");
  h->launches += 1;
  h->sweeps += 1;
  return MQ_OK;
}

int run_probabilities(mq_state* h, const int32_t* wires, int k, int out_dtype, void* out) {
  int rc = check_wires(h->n, wires, k);
  if (rc) return rc;
  const int n = h->n;
  if (natural_order(n, wires, k)) {
    rc = ensure_alt(h);
    if (rc) return rc;
    const uint32_t dim = (uint32_t)h->dim();
    void* stage = h->buf[1 - h->cur];
    const uint32_t grid = (uint32_t)std::min<uint64_t>((dim + 255) / 256, (uint64_t)h->num_sms * 16);
    if (h->dtype == MQ_C64) {
      if (out_dtype == 0) k_amp2_out<float, float><<<grid, 256, 0, h->stream>>>((const float2*)h->cur_buf(), (float*)stage, dim);
      else k_amp2_out<float, double><<<grid, 256, 0, h->stream>>>((const float2*)h->cur_buf(), (double*)stage, dim);
    } else {
      if (out_dtype == 0) k_amp2_out<double, float><<<grid, 256, 0, h->stream>>>((const double2*)h->cur_buf(), (float*)stage, dim);
      else k_amp2_out<double, double><<<grid, 256, 0, h->stream>>>((const double2*)h->cur_buf(), (double*)stage, dim);
    }
    MQ_LAUNCHED("k_amp2_out");
    h->launches += 1;
    h->sweeps += 1;
    MQ_CUDA(cudaMemcpyAsync(out, stage, (size_t)dim * (out_dtype == 0 ? 4 : 8), cudaMemcpyDeviceToHost, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
    return MQ_OK;
  }
  const uint64_t nc = (uint64_t(1) << n) / std::min<uint64_t>(kBlock, uint64_t(1) << (n - k));
  const size_t nbk = size_t(1) << k;
  const size_t need = (nc + nc + nbk) * 8 + (8192 + 256) * 4 + 256;
  rc = ensure_scratch(h, need);
  if (rc) return rc;
  double* work = (double*)h->scratch;
  double* q = work + 2 * nc;
  uint32_t* dep = (uint32_t*)(q + nbk);
  rc = marginal_device(h, wires, k, q, work, dep);
  if (rc) return rc;
  if (out_dtype == 1) {
    MQ_CUDA(cudaMemcpyAsync(out, q, nbk * 8, cudaMemcpyDeviceToHost, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<double> tmp(nbk);
    MQ_CUDA(cudaMemcpyAsync(tmp.data(), q, nbk * 8, cudaMemcpyDeviceToHost, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < nbk; ++i) ((float*)out)[i] = (float)tmp[i];
  }
  return MQ_OK;
}

template <typename Src>
static int sample_from(mq_state* h, Src src, uint32_t m, uint64_t seed, uint64_t offset, int64_t shots,
                       int64_t* out, double* work) {
  const uint32_t bs = std::min<uint32_t>(kBlock, m);
  const uint32_t nb = m / bs;
  const uint32_t ng = (nb + kSuper - 1) / kSuper;
  double* S = work;
  double* L = S + nb;
  double* T = L + nb;
  double* E = T + ng;
  int32_t* LP = (int32_t*)(E + ng);
  SampleMeta* meta = (SampleMeta*)(((uintptr_t)(LP + ng) + 15) & ~(uintptr_t)15);
  int64_t* dout = (int64_t*)(meta + 1);
  k_block_sums<Src><<<grid_for((uint64_t)nb * 32, 256), 256, 0, h->stream>>>(src, bs, nb, S);
  MQ_LAUNCHED("k_block_sums");
  k_local_prefix<<<grid_for(ng, 128), 128, 0, h->stream>>>(S, nb, L, T, LP);
  MQ_LAUNCHED("k_local_prefix");
  k_super_prefix<<<1, 1, 0, h->stream>>>(T, LP, ng, E, meta);
  MQ_LAUNCHED("k_super_prefix");
  SampleMeta hm;
  MQ_CUDA(cudaMemcpyAsync(&hm, meta, sizeof(hm), cudaMemcpyDeviceToHost, h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  if (!(hm.total > 0.0)) return fail(MQ_EINVAL, "Simulator returned a zero-probability state");
  if (shots > 0) {
    k_draw<Src><<<grid_for((uint64_t)shots, 128), 128, 0, h->stream>>>(src, bs, nb, L, E, meta, seed, offset, shots, dout);
    MQ_LAUNCHED("k_draw");
    MQ_CUDA(cudaMemcpyAsync(out, dout, (size_t)shots * 8, cudaMemcpyDeviceToHost, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
  }
  h->launches += 4;
  h->sweeps += 1;
  return MQ_OK;
}

static size_t sample_work_bytes(uint32_t m, int64_t shots) {
  const uint32_t bs = std::min<uint32_t>(kBlock, m);
  const uint32_t nb = m / bs;
  const uint32_t ng = (nb + kSuper - 1) / kSuper;
  return (size_t)(2 * nb + 2 * ng) * 8 + (size_t)ng * 4 + 64 + (size_t)std::max<int64_t>(shots, 1) * 8 + 64;
}

int run_sample(mq_state* h, const int32_t* wires, int k, uint64_t seed, uint64_t offset, int64_t shots, int64_t* out) {
  int rc = check_wires(h->n, wires, k);
  if (rc) return rc;
  if (shots < 0) return fail(MQ_EINVAL, "shots must be non-negative");
  const int n = h->n;
  if (natural_order(n, wires, k)) {
    const uint32_t m = (uint32_t)h->dim();
    rc = ensure_scratch(h, sample_work_bytes(m, shots));
    if (rc) return rc;
    if (h->dtype == MQ_C64) return sample_from(h, StateSrc<float>{(const float2*)h->cur_buf()}, m, seed, offset, shots, out, (double*)h->scratch);
    return sample_from(h, StateSrc<double>{(const double2*)h->cur_buf()}, m, seed, offset, shots, out, (double*)h->scratch);
  }
  if (k == 0) {
    for (int64_t s = 0; s < shots; ++s) out[s] = 0;
    return MQ_OK;
  }
  const uint64_t nc = (uint64_t(1) << n) / std::min<uint64_t>(kBlock, uint64_t(1) << (n - k));
  const size_t nbk = size_t(1) << k;
  const size_t marg = (nc + nc + nbk) * 8 + (8192 + 256) * 4 + 256;
  rc = ensure_scratch(h, marg + sample_work_bytes((uint32_t)nbk, shots) + 64);
  if (rc) return rc;
  double* work = (double*)h->scratch;
  double* q = work + 2 * nc;
  uint32_t* dep = (uint32_t*)(q + nbk);
  rc = marginal_device(h, wires, k, q, work, dep);
  if (rc) return rc;
  double* swork = (double*)((((uintptr_t)h->scratch + marg) + 63) & ~(uintptr_t)63);
  return sample_from(h, VecSrc{q}, (uint32_t)nbk, seed, offset, shots, out, swork);
}

int run_expval_pauli(mq_state* h, int n_words, const uint64_t* xmask, const uint64_t* zmask, const int32_t* ny,
                     double* out) {
  const uint64_t lim = h->dim() - 1;
  for (int w = 0; w < n_words; ++w)
    if ((xmask[w] & ~lim) || (zmask[w] & ~lim)) return fail(MQ_EINVAL, "Pauli mask outside the register");
  const uint32_t grid = (uint32_t)h->num_sms * 4;
  int rc = ensure_scratch(h, (size_t)grid * kWords * sizeof(double2));
  if (rc) return rc;
  double2* partials = (double2*)h->scratch;
  std::vector<double2> host((size_t)grid * kWords);
  std::vector<bool> done(n_words, false);
  for (int w0 = 0; w0 < n_words; ++w0) {
    if (done[w0]) continue;
    PauliParams P;
    std::memset(&P, 0, sizeof(P));
    P.dim = (uint32_t)h->dim();
    P.x = (uint32_t)xmask[w0];
    std::vector<int> members;
    for (int w = w0; w < n_words && (int)members.size() < kWords; ++w)
      if (!done[w] && xmask[w] == xmask[w0]) { members.push_back(w); done[w] = true; }
    P.nw = (int32_t)members.size();
    for (size_t i = 0; i < members.size(); ++i) P.z[i] = (uint32_t)zmask[members[i]];
    if (h->dtype == MQ_C64) k_pauli<float><<<grid, 256, 0, h->stream>>>((const float2*)h->cur_buf(), P, partials);
    else k_pauli<double><<<grid, 256, 0, h->stream>>>((const double2*)h->cur_buf(), P, partials);
    MQ_LAUNCHED("k_pauli");
    h->launches += 1;
    h->sweeps += 1;
    MQ_CUDA(cudaMemcpyAsync(host.data(), partials, host.size() * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < members.size(); ++i) {
      double re = 0.0, im = 0.0;
      for (uint32_t b = 0; b < grid; ++b) { re += host[b * kWords + i].x; im += host[b * kWords + i].y; }
      // multiply by i^ny
      const int w = members[i];
      const int r = ((ny ? ny[w] : 0) % 4 + 4) % 4;
      double fr = re, fi = im;
      if (r == 1) { fr = -im; fi = re; }
      else if (r == 2) { fr = -re; fi = -im; }
      else if (r == 3) { fr = im; fi = -re; }
      out[2 * w] = fr;
      out[2 * w + 1] = fi;
    }
  }
  return MQ_OK;
}

// ================================================ allocation-free expectations
// mq_expval_pauli_static computes the same values as mq_expval_pauli, but
// never allocates device memory.  mq_expval_pauli grows the handle's scratch
// buffer with cudaMalloc (and cudaFree) the first time it needs room for
// its per-block partial sums; cudaFree waits for the whole device.  Callers
// that run under a fixed device-memory budget (a serving loop that admits
// requests by their state footprint alone, or a host whose memory pool owns
// all free HBM) or that cannot stall other streams with that device-wide
// wait use this entry point instead.
//
// Its scratch is a file-scope device array of a fixed size: every GPU that
// loads the library holds these 131,200 bytes until the process exits.  The
// host reaches the array through the address that cudaGetSymbolAddress
// returns for the current device (the array's name in host code is only a
// host-side stand-in); the address is looked up once per device, on the
// first call made on that device, and kept for the life of the process.  A
// cudaDeviceReset (or any teardown of the device's primary context) makes
// the kept address stale: a process that resets a device must not call this
// entry point on it afterwards.
constexpr uint32_t kStaticBlocks = 1024;  // partial-sum blocks the array holds
static __device__ __align__(256) double2 g_pauli_static[kStaticBlocks * kWords + kWords];

constexpr int kStaticMaxDevices = 64;
static std::mutex g_static_mu;
static void* g_static_addr[kStaticMaxDevices] = {};

// Device address of g_pauli_static on `device`, which must be current.
static int pauli_static_scratch(int device, double2** out) {
  if (device < 0 || device >= kStaticMaxDevices) return fail(MQ_EUNSUPPORTED, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_addr[device]) {
    void* p = nullptr;
    MQ_CUDA(cudaGetSymbolAddress(&p, g_pauli_static));
    g_static_addr[device] = p;
  }
  *out = reinterpret_cast<double2*>(g_static_addr[device]);
  return MQ_OK;
}

// res[w] = sum over blocks b of partials[b][w], in increasing b: the order
// and rounding of the host loop in run_expval_pauli, so both entry points
// return the same bits.
__global__ void k_pauli_finish(const double2* __restrict__ partials, uint32_t nblocks, int nw,
                               double2* __restrict__ res) {
  const int w = threadIdx.x;
  if (w >= nw) return;
  double re = 0.0, im = 0.0;
  for (uint32_t b = 0; b < nblocks; ++b) {
    re = __dadd_rn(re, partials[b * kWords + w].x);
    im = __dadd_rn(im, partials[b * kWords + w].y);
  }
  res[w] = make_double2(re, im);
}

int run_expval_pauli_static(mq_state* h, int n_words, const uint64_t* xmask, const uint64_t* zmask,
                            const int32_t* ny, double* out) {
  const uint64_t lim = h->dim() - 1;
  for (int w = 0; w < n_words; ++w)
    if ((xmask[w] & ~lim) || (zmask[w] & ~lim)) return fail(MQ_EINVAL, "Pauli mask outside the register");
  // same grid as run_expval_pauli: the partial sums, and so the result bits,
  // depend on it
  const uint32_t grid = (uint32_t)h->num_sms * 4;
  if (grid > kStaticBlocks)
    return fail(MQ_EUNSUPPORTED, "mq_expval_pauli_static: this GPU needs " + std::to_string(grid) +
                                     " partial-sum blocks; the static scratch holds 1024 (GPUs of up to 256 SMs)");
  double2* partials = nullptr;
  int rc = pauli_static_scratch(h->device, &partials);
  if (rc) return rc;
  double2* res = partials + (size_t)kStaticBlocks * kWords;
  // Every slot read below is written earlier in the same call (k_pauli writes
  // all kWords slots of each of its blocks, k_pauli_finish all nw results it
  // returns), so whatever an earlier call left in the array is never read
  // and nothing has to be cleared.
  int w0 = 0;
  while (w0 < n_words) {
    // consecutive words with one X/Y mask share a pass over the state
    int cnt = 1;
    while (w0 + cnt < n_words && cnt < kWords && xmask[w0 + cnt] == xmask[w0]) ++cnt;
    PauliParams P;
    std::memset(&P, 0, sizeof(P));
    P.dim = (uint32_t)h->dim();
    P.x = (uint32_t)xmask[w0];
    P.nw = cnt;
    for (int i = 0; i < cnt; ++i) P.z[i] = (uint32_t)zmask[w0 + i];
    if (h->dtype == MQ_C64) k_pauli<float><<<grid, 256, 0, h->stream>>>((const float2*)h->cur_buf(), P, partials);
    else k_pauli<double><<<grid, 256, 0, h->stream>>>((const double2*)h->cur_buf(), P, partials);
    MQ_LAUNCHED("k_pauli");
    k_pauli_finish<<<1, 32, 0, h->stream>>>(partials, grid, cnt, res);
    MQ_LAUNCHED("k_pauli_finish");
    h->launches += 2;
    h->sweeps += 1;
    double2 host[kWords];
    MQ_CUDA(cudaMemcpyAsync(host, res, (size_t)cnt * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    MQ_CUDA(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < cnt; ++i) {
      const int w = w0 + i;
      const double re = host[i].x, im = host[i].y;
      const int r = ((ny ? ny[w] : 0) % 4 + 4) % 4;  // multiply by i^ny
      double fr = re, fi = im;
      if (r == 1) { fr = -im; fi = re; }
      else if (r == 2) { fr = -re; fi = -im; }
      else if (r == 3) { fr = im; fi = -re; }
      out[2 * w] = fr;
      out[2 * w + 1] = fi;
    }
    w0 += cnt;
  }
  return MQ_OK;
}

}  // namespace mq
