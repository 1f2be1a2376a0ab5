// Batched circuits (the batching direction): many independent circuits of
// uneven width in one CUDA-graph launch.
//
// The reference runs a batch as a Python loop, one circuit and one launch
// sequence at a time (integrations/qiskit.py:505-514).  Here a batch of
// layered circuits (per layer: a 2x2 on every qubit, optionally followed by
// the CNOT ladder 0->1->...->n-1) is planned once and captured as one graph:
//
//   * circuits of at most kSmallMax qubits run whole inside shared memory:
//     k_batch_small is a persistent kernel whose CTAs take circuits from an
//     atomic counter, start from |0...0>, apply every layer in place (the
//     ladder is a gather between two shared buffers) and write the
//     probabilities and <Z_0>; nothing but the outputs touches HBM;
//   * larger circuits run the fused-layer tile sweeps on per-lane states
//     (one stream per lane, the lanes are parallel branches of the graph, so
//     small sweeps of different circuits overlap on the device), followed by
//     k_probs_z.
//
// Gate matrices live in device memory (read by the kernels when they run),
// so one captured graph serves every later parameter set: a run is one
// host-to-device copy of the matrices and one graph launch.
#include <algorithm>
#include <cstring>
#include <exception>
#include <map>
#include <new>
#include <numeric>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

constexpr int kSmallMax = 13;  // 2 x 2^13 complex64 = 128 KiB of shared memory

struct SmallCircuit {
  uint32_t n, depth, ladder, index;
  uint64_t mats_off;   // doubles: depth * n * 8, layer-major, qubit-major
  uint64_t probs_off;  // floats
};

__device__ __forceinline__ uint32_t bslot(uint32_t i) { return i ^ ((i >> 3) & 0xEu); }

__device__ __forceinline__ float2 cmac2f(float2 u0, float2 x0, float2 u1, float2 x1) {
  float2 r;
  r.x = fmaf(u0.x, x0.x, fmaf(-u0.y, x0.y, fmaf(u1.x, x1.x, -u1.y * x1.y)));
  r.y = fmaf(u0.x, x0.y, fmaf(u0.y, x0.x, fmaf(u1.x, x1.y, u1.y * x1.x)));
  return r;
}

template <int NT>
__global__ void __launch_bounds__(NT) k_batch_small(const SmallCircuit* __restrict__ circ, uint32_t n_circ,
                                                    const double* __restrict__ mats, float* __restrict__ probs,
                                                    double* __restrict__ z0, uint32_t* __restrict__ next) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ float2 um[kSmallMax][4];
  __shared__ uint32_t cid;
  __shared__ double zred[NT / 32];
  const int tid = threadIdx.x;
  for (;;) {
    __syncthreads();
    if (tid == 0) cid = atomicAdd(next, 1u);
    __syncthreads();
    const uint32_t c = cid;
    if (c >= n_circ) break;
    const SmallCircuit C = circ[c];
    const int n = (int)C.n;
    const uint32_t E = 1u << n;
    float2* a = sm;
    float2* b = sm + (1u << kSmallMax);
    for (uint32_t i = tid; i < E; i += NT) a[bslot(i)] = make_float2(i == 0 ? 1.f : 0.f, 0.f);
    for (uint32_t l = 0; l < C.depth; ++l) {
      __syncthreads();
      for (int j = tid; j < n * 4; j += NT) {
        const double* m = mats + C.mats_off + ((size_t)l * n * 4 + j) * 2;
        um[j >> 2][j & 3] = make_float2((float)m[0], (float)m[1]);
      }
      __syncthreads();
      // 2x2 on every qubit, four index bits per register pass; the last pass
      // is shifted down to [n-4, n) and skips the bits already done
      for (int g0 = 0; g0 < n; g0 += 4) {
        const int lo = n >= 4 ? min(g0, n - 4) : 0;
        const int nb = n >= 4 ? 4 : n;
        const uint32_t groups = E >> nb;
        for (uint32_t gi = tid; gi < groups; gi += NT) {
          const uint32_t base = ((gi >> lo) << (lo + nb)) | (gi & ((1u << lo) - 1u));
          float2 v[16];
#pragma unroll
          for (int r = 0; r < 16; ++r)
            if (r < (1 << nb)) v[r] = a[bslot(base | ((uint32_t)r << lo))];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int bit = lo + k;
            if (k >= nb || bit < g0) continue;
            const int q = n - 1 - bit;
            const float2 u00 = um[q][0], u01 = um[q][1], u10 = um[q][2], u11 = um[q][3];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
              if ((r & (1 << k)) || r >= (1 << nb)) continue;
              const float2 x0 = v[r], x1 = v[r | (1 << k)];
              v[r] = cmac2f(u00, x0, u01, x1);
              v[r | (1 << k)] = cmac2f(u10, x0, u11, x1);
            }
          }
#pragma unroll
          for (int r = 0; r < 16; ++r)
            if (r < (1 << nb)) a[bslot(base | ((uint32_t)r << lo))] = v[r];
        }
        __syncthreads();
      }
      if (C.ladder) {
        // CNOT(0,1), ..., CNOT(n-2,n-1): out[y] = in[y ^ (y >> 1)]
        for (uint32_t y = tid; y < E; y += NT) b[bslot(y)] = a[bslot(y ^ (y >> 1))];
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
      }
    }
    double zacc = 0.0;
    for (uint32_t i = tid; i < E; i += NT) {
      const float2 v = a[bslot(i)];
      const double p = (double)v.x * v.x + (double)v.y * v.y;
      probs[C.probs_off + i] = (float)p;
      zacc += ((i >> (n - 1)) & 1u) ? -p : p;
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) zacc += __shfl_xor_sync(0xffffffffu, zacc, off);
    if ((tid & 31) == 0) zred[tid >> 5] = zacc;
    __syncthreads();
    if (tid == 0) {
      double z = 0.0;
      for (int w = 0; w < NT / 32; ++w) z += zred[w];
      z0[C.index] = z;
    }
  }
}

// probabilities of a full state and per-block partial sums of <Z_0>
__global__ void __launch_bounds__(256) k_probs_z(const float2* __restrict__ st, uint32_t dim, int n,
                                                 float* __restrict__ probs, double* __restrict__ zpart) {
  __shared__ double red[8];
  double acc = 0.0;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
    const float2 v = st[i];
    const double p = (double)v.x * v.x + (double)v.y * v.y;
    probs[i] = (float)p;
    acc += ((i >> (n - 1)) & 1u) ? -p : p;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double z = 0.0;
    for (int w = 0; w < 8; ++w) z += red[w];
    zpart[blockIdx.x] = z;
  }
}

__global__ void k_zsum(const double* __restrict__ zpart, uint32_t nb, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double z = 0.0;
  for (uint32_t b = 0; b < nb; ++b) z += zpart[b];
  *out = z;
}

__global__ void k_basis0(float2* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st[0] = make_float2(1.f, 0.f);
}

}  // namespace mq

using namespace mq;

struct mq_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int n_circ = 0;
  std::vector<int32_t> n, depth;
  std::vector<uint8_t> ladder;
  std::vector<uint64_t> mats_off, probs_off;
  uint64_t mats_total = 0, probs_total = 0;
  double* d_mats = nullptr;
  // small circuits
  std::vector<int> small;
  SmallCircuit* d_small = nullptr;
  uint32_t* d_next = nullptr;
  int small_threads = 256;
  // large circuits
  std::vector<int> large;
  int lanes = 1;
  std::vector<std::vector<int>> lane_work;
  std::vector<cudaStream_t> lane_stream;
  std::vector<cudaEvent_t> lane_event;
  cudaEvent_t fork_event = nullptr;
  std::vector<std::map<int, mq_state*>> lane_state;
  double* d_zpart = nullptr;
  uint32_t zblocks = 0;
  int num_sms = 148;
  // sweep plan of the large circuits (mq_batch_set_tiles; 0 / -1 = defaults)
  int tile_max = 0, tile_pas = -1, tile_min = 0;
  cudaGraphExec_t exec = nullptr;
  float* graph_probs = nullptr;
  double* graph_z0 = nullptr;
};

namespace mq {

static void batch_free(mq_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (auto& m : b->lane_state)
    for (auto& kv : m) {
      mq_state* h = kv.second;
      if (h->buf[0]) cudaFree(h->buf[0]);
      if (h->buf[1]) cudaFree(h->buf[1]);
      if (h->scratch) cudaFree(h->scratch);
      delete h;
    }
  for (auto s : b->lane_stream) cudaStreamDestroy(s);
  for (auto e : b->lane_event) cudaEventDestroy(e);
  if (b->fork_event) cudaEventDestroy(b->fork_event);
  if (b->d_mats) cudaFree(b->d_mats);
  if (b->d_small) cudaFree(b->d_small);
  if (b->d_next) cudaFree(b->d_next);
  if (b->d_zpart) cudaFree(b->d_zpart);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// A lane's workspace state for n qubits (both buffers allocated up front:
// nothing may allocate while the graph is being captured).
static int lane_state_for(mq_batch* b, int lane, int n, mq_state** out) {
  auto it = b->lane_state[lane].find(n);
  if (it != b->lane_state[lane].end()) { *out = it->second; return MQ_OK; }
  auto* h = new mq_state();
  h->n = n;
  h->dtype = MQ_C64;
  h->device = b->device;
  h->num_sms = b->num_sms;
  h->device_sms = b->num_sms;
  h->stream = b->lane_stream[lane];
  h->tile_max = b->tile_max;
  h->tile_pas = b->tile_pas;
  h->tile_min = b->tile_min;
  h->state_bytes = (size_t(1) << n) * 8;
  cudaError_t e = cudaMalloc(&h->buf[0], h->state_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&h->buf[1], h->state_bytes);
  if (e != cudaSuccess) {
    if (h->buf[0]) cudaFree(h->buf[0]);
    delete h;
    return cuda_fail(e, "cudaMalloc(batch lane state)");
  }
  b->lane_state[lane][n] = h;
  *out = h;
  return MQ_OK;
}

template <int NT>
static int launch_small(mq_batch* b, float* probs, double* z0, bool configure) {
  const size_t smem = 2 * sizeof(float2) * (size_t(1) << kSmallMax);
  if (configure) {
    MQ_CUDA(cudaFuncSetAttribute(k_batch_small<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return MQ_OK;
  }
  int bps = 0;
  MQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch_small<NT>, NT, smem));
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b->small.size(), (uint64_t)b->num_sms * std::max(1, bps)));
  k_batch_small<NT><<<grid, NT, smem, b->stream>>>(b->d_small, (uint32_t)b->small.size(), b->d_mats, probs, z0, b->d_next);
  MQ_LAUNCHED("k_batch_small");
  return MQ_OK;
}

static int small_dispatch(mq_batch* b, float* probs, double* z0, bool configure) {
  switch (b->small_threads) {
    case 128: return launch_small<128>(b, probs, z0, configure);
    case 512: return launch_small<512>(b, probs, z0, configure);
    default: return launch_small<256>(b, probs, z0, configure);
  }
}

// Record the whole batch on b->stream (being captured).
static int record_batch(mq_batch* b, float* probs, double* z0) {
  if (!b->small.empty()) {
    MQ_CUDA(cudaMemsetAsync(b->d_next, 0, sizeof(uint32_t), b->stream));
    int rc = small_dispatch(b, probs, z0, false);
    if (rc) return rc;
  }
  if (b->large.empty()) return MQ_OK;
  MQ_CUDA(cudaEventRecord(b->fork_event, b->stream));
  for (int l = 0; l < b->lanes; ++l) MQ_CUDA(cudaStreamWaitEvent(b->lane_stream[l], b->fork_event, 0));
  uint32_t cols[32];
  for (int l = 0; l < b->lanes; ++l) {
    cudaStream_t s = b->lane_stream[l];
    double* zpart = b->d_zpart + (size_t)l * b->zblocks;
    for (int c : b->lane_work[l]) {
      const int n = b->n[c];
      mq_state* h = nullptr;
      int rc = lane_state_for(b, l, n, &h);
      if (rc) return rc;
      h->cur = 0;
      MQ_CUDA(cudaMemsetAsync(h->buf[0], 0, h->state_bytes, s));
      k_basis0<<<1, 32, 0, s>>>(reinterpret_cast<float2*>(h->buf[0]));
      MQ_LAUNCHED("k_basis0");
      // CNOT ladder: columns A e_j of out[y] = in[A y], A e_j = e_j + e_{j-1}
      for (int j = 0; j < n; ++j) cols[j] = (1u << j) | (j ? (1u << (j - 1)) : 0u);
      for (int d = 0; d < b->depth[c]; ++d) {
        const double* md = b->d_mats + b->mats_off[c] + (size_t)d * n * 8;
        rc = launch_layer(h, nullptr, nullptr, 0, nullptr, nullptr, nullptr, b->ladder[c] ? cols : nullptr, 0, md);
        if (rc) return rc;
      }
      const uint32_t dim = 1u << n;
      const uint32_t grid = std::min<uint32_t>(b->zblocks, std::max<uint32_t>(1, dim / 256));
      k_probs_z<<<grid, 256, 0, s>>>(reinterpret_cast<const float2*>(h->cur_buf()), dim, n, probs + b->probs_off[c], zpart);
      MQ_LAUNCHED("k_probs_z");
      k_zsum<<<1, 32, 0, s>>>(zpart, grid, z0 + c);
      MQ_LAUNCHED("k_zsum");
    }
    MQ_CUDA(cudaEventRecord(b->lane_event[l], s));
    MQ_CUDA(cudaStreamWaitEvent(b->stream, b->lane_event[l], 0));
  }
  return MQ_OK;
}

}  // namespace mq

#define MQ_TRY_BEGIN try {
#define MQ_TRY_END                                                      \
  }                                                                     \
  catch (const std::bad_alloc&) { return fail(MQ_ENOMEM, "host allocation failed"); } \
  catch (const std::exception& ex) { return fail(MQ_EDEVICE, ex.what()); } \
  catch (...) { return fail(MQ_EDEVICE, "unknown C++ exception"); }

extern "C" {

int mq_batch_create(int device, void* stream, int n_circuits, const int32_t* n_qubits, const int32_t* depth,
                    const uint8_t* ladder, int lanes, int small_threads, mq_batch** out) {
  MQ_TRY_BEGIN
  if (!out) return fail(MQ_EINVAL, "null output handle");
  *out = nullptr;
  if (n_circuits < 0 || (n_circuits > 0 && (!n_qubits || !depth))) return fail(MQ_EINVAL, "invalid circuit arrays");
  if (lanes < 1 || lanes > 64) return fail(MQ_EINVAL, "lanes must be in [1, 64]");
  if (small_threads != 128 && small_threads != 256 && small_threads != 512)
    return fail(MQ_EINVAL, "small_threads must be 128, 256 or 512");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(MQ_EDEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= ndev) return fail(MQ_EINVAL, "device index out of range");
  for (int c = 0; c < n_circuits; ++c) {
    if (n_qubits[c] < 1 || n_qubits[c] > 30) return fail(MQ_EINVAL, "batched circuits take 1 to 30 qubits");
    if (depth[c] < 0) return fail(MQ_EINVAL, "negative depth");
  }
  DeviceGuard g(device);
  auto* b = new mq_batch();
  b->device = device;
  b->n_circ = n_circuits;
  b->lanes = lanes;
  b->small_threads = small_threads;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) b->num_sms = sms;
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete b; return cuda_fail(e, "cudaStreamCreate"); }
    b->own_stream = true;
  }
  b->n.assign(n_qubits, n_qubits + n_circuits);
  b->depth.assign(depth, depth + n_circuits);
  b->ladder.assign(n_circuits, 1);
  if (ladder) b->ladder.assign(ladder, ladder + n_circuits);
  for (int c = 0; c < n_circuits; ++c) {
    b->mats_off.push_back(b->mats_total);
    b->probs_off.push_back(b->probs_total);
    b->mats_total += (uint64_t)b->depth[c] * b->n[c] * 8;
    b->probs_total += uint64_t(1) << b->n[c];
    (b->n[c] <= kSmallMax ? b->small : b->large).push_back(c);
  }
  auto bail = [&](cudaError_t e, const char* where) {
    const int rc = cuda_fail(e, where);
    batch_free(b);
    return rc;
  };
  cudaError_t e = cudaMalloc(&b->d_mats, std::max<uint64_t>(8, b->mats_total * sizeof(double)));
  if (e != cudaSuccess) return bail(e, "cudaMalloc(batch matrices)");
  if (!b->small.empty()) {
    std::vector<SmallCircuit> sc;
    // largest circuits first: the atomic counter hands them out early
    std::vector<int> order = b->small;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      return ((uint64_t)b->depth[x] << b->n[x]) > ((uint64_t)b->depth[y] << b->n[y]);
    });
    for (int c : order)
      sc.push_back({(uint32_t)b->n[c], (uint32_t)b->depth[c], (uint32_t)b->ladder[c], (uint32_t)c, b->mats_off[c],
                    b->probs_off[c]});
    e = cudaMalloc(&b->d_small, sc.size() * sizeof(SmallCircuit));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_next, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_small, sc.data(), sc.size() * sizeof(SmallCircuit), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bail(e, "batch small-circuit setup");
    int rc = small_dispatch(b, nullptr, nullptr, true);
    if (rc) { batch_free(b); return rc; }
  }
  if (!b->large.empty()) {
    b->lanes = std::min<int>(lanes, (int)b->large.size());
    b->lane_work.resize(b->lanes);
    b->lane_state.resize(b->lanes);
    // longest-processing-time assignment of circuits to lanes
    std::vector<int> order = b->large;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      return ((uint64_t)std::max(1, b->depth[x]) << b->n[x]) > ((uint64_t)std::max(1, b->depth[y]) << b->n[y]);
    });
    std::vector<uint64_t> load(b->lanes, 0);
    for (int c : order) {
      const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      b->lane_work[l].push_back(c);
      load[l] += (uint64_t)std::max(1, b->depth[c]) << b->n[c];
    }
    for (int l = 0; l < b->lanes; ++l) {
      cudaStream_t s;
      cudaEvent_t ev;
      e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
      if (e != cudaSuccess) return bail(e, "cudaStreamCreate(lane)");
      b->lane_stream.push_back(s);
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e != cudaSuccess) return bail(e, "cudaEventCreate(lane)");
      b->lane_event.push_back(ev);
      for (int c : b->lane_work[l]) {
        mq_state* h = nullptr;
        int rc = lane_state_for(b, l, b->n[c], &h);
        if (rc) { batch_free(b); return rc; }
      }
    }
    e = cudaEventCreateWithFlags(&b->fork_event, cudaEventDisableTiming);
    if (e != cudaSuccess) return bail(e, "cudaEventCreate(fork)");
    b->zblocks = (uint32_t)b->num_sms * 4;
    e = cudaMalloc(&b->d_zpart, (size_t)b->lanes * b->zblocks * sizeof(double));
    if (e != cudaSuccess) return bail(e, "cudaMalloc(batch partials)");
  }
  *out = b;
  return MQ_OK;
  MQ_TRY_END
}

int mq_batch_info(const mq_batch* b, uint64_t* mats_count, uint64_t* probs_count, int* n_small, int* n_large) {
  if (!b) return fail(MQ_EINVAL, "null batch handle");
  if (mats_count) *mats_count = b->mats_total;
  if (probs_count) *probs_count = b->probs_total;
  if (n_small) *n_small = (int)b->small.size();
  if (n_large) *n_large = (int)b->large.size();
  return MQ_OK;
}

int mq_batch_set_tiles(mq_batch* b, int tile_max, int passengers, int tile_min) {
  if (!b) return fail(MQ_EINVAL, "null batch handle");
  if (b->exec) return fail(MQ_EINVAL, "the tile plan is fixed once the batch has run (its graph is captured)");
  if (tile_max != 0 && (tile_max < 6 || tile_max > 12)) return fail(MQ_EINVAL, "tile_max must be 0 or in [6, 12]");
  if (passengers < -1 || passengers > 5) return fail(MQ_EINVAL, "passengers must be -1 or in [0, 5]");
  if (tile_min < 0 || tile_min > 12) return fail(MQ_EINVAL, "tile_min must be 0 or in [1, 12]");
  if (tile_max && passengers >= tile_max) return fail(MQ_EINVAL, "passengers must leave room for targets in a tile");
  b->tile_max = tile_max;
  b->tile_pas = passengers;
  b->tile_min = tile_min;
  return MQ_OK;
}

int mq_batch_run(mq_batch* b, const double* mats, float* probs_dev, double* z0_dev) {
  MQ_TRY_BEGIN
  if (!b) return fail(MQ_EINVAL, "null batch handle");
  if (b->n_circ == 0) return MQ_OK;
  if ((b->mats_total && !mats) || !probs_dev || !z0_dev) return fail(MQ_EINVAL, "null batch arrays");
  DeviceGuard g(b->device);
  if (b->mats_total)
    MQ_CUDA(cudaMemcpyAsync(b->d_mats, mats, b->mats_total * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  if (!b->exec || b->graph_probs != probs_dev || b->graph_z0 != z0_dev) {
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    MQ_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = record_batch(b, probs_dev, z0_dev);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(batch)");
    e = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate(batch)");
    b->graph_probs = probs_dev;
    b->graph_z0 = z0_dev;
  }
  MQ_CUDA(cudaGraphLaunch(b->exec, b->stream));
  return MQ_OK;
  MQ_TRY_END
}

int mq_batch_sync(mq_batch* b) {
  if (!b) return fail(MQ_EINVAL, "null batch handle");
  DeviceGuard g(b->device);
  MQ_CUDA(cudaStreamSynchronize(b->stream));
  return MQ_OK;
}

int mq_batch_destroy(mq_batch* b) {
  if (!b) return MQ_OK;
  DeviceGuard g(b->device);
  cudaStreamSynchronize(b->stream);
  batch_free(b);
  return MQ_OK;
}

}  // extern "C"
