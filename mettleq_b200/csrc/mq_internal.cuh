// Internal definitions shared by the libmq CUDA sources (not part of the ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/mq.h"

namespace mq {

// ---------------------------------------------------------------- complex
template <typename R> struct V2T;
template <> struct V2T<float> { using T = float2; };
template <> struct V2T<double> { using T = double2; };
template <typename R> using V2 = typename V2T<R>::T;

template <typename R> __host__ __device__ __forceinline__ V2<R> mk(R re, R im) {
  V2<R> v; v.x = re; v.y = im; return v;
}
template <typename T> __device__ __forceinline__ T cadd(T a, T b) { a.x += b.x; a.y += b.y; return a; }
template <typename T> __device__ __forceinline__ T csub(T a, T b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename T> __device__ __forceinline__ T cmul(T a, T b) {
  T r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename T> __device__ __forceinline__ T cmulc(T a, T b) {  // a * conj(b)
  T r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename T, typename R> __device__ __forceinline__ T cscale(T a, R s) { a.x *= s; a.y *= s; return a; }
// x + t y for a real t
template <typename T, typename R> __device__ __forceinline__ T caxpy(R t, T y, T x) {
  x.x = fma(t, y.x, x.x); x.y = fma(t, y.y, x.y); return x;
}
// t y - x for a real t
template <typename T, typename R> __device__ __forceinline__ T caxmy(R t, T y, T x) {
  x.x = fma(t, y.x, -x.x); x.y = fma(t, y.y, -x.y); return x;
}
// complex64 on the paired FP32 instructions of sm_100 (FADD2 / FMUL2 /
// FFMA2): one instruction where the components take the same operation.
// Each lane rounds like the scalar instruction, so the results are the bits
// of the scalar forms above (a - b as a + (-1) b: the product is exact).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ float2 caxpy(float t, float2 y, float2 x) { return __ffma2_rn(make_float2(t, t), y, x); }
__device__ __forceinline__ float2 caxmy(float t, float2 y, float2 x) {
  return __ffma2_rn(make_float2(t, t), y, make_float2(-x.x, -x.y));
}

// ---------------------------------------------------------------- async copies
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void* src) {
  if constexpr (BYTES == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
  } else {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------- TMA + mbarriers
// Tile copies by the tensor memory accelerator: one thread issues a whole
// tile (cp.async.bulk.tensor, up to 5 dimensions) that completes on an
// mbarrier in shared memory; stores go back the same way from shared memory.
// No cluster multicast is used anywhere: every copy moves this GPU's own
// memory into (or out of) the issuing CTA's shared memory.
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits for the phase of parity `parity` of the mbarrier to complete, for at
// most `limit_ns` nanoseconds of the global timer; false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
}
// Load box `coords` of tensor map `map` (a kernel parameter) into shared
// memory at `dst`, completing `bytes` of transactions on `bar`.
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const void* map, const int32_t (&c)[5], uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_store_5d(const void* map, const int32_t (&c)[5], uint32_t src) {
  asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// The bulk stores issued so far have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// ... and finished writing global memory.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// Generic-proxy writes to shared memory become visible to the async proxy
// (a TMA store that reads them, a TMA load that overwrites them).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// ---------------------------------------------------------------- TMA tiles
// TMA form of a sweep's tile movement (k_tile, k_adj).  The state is viewed
// as a tensor of 8-byte words (complex64: one amplitude; complex128: its real
// or imaginary part, word bit 0) whose dimensions are runs of index bits in
// ascending order: dimension 0 is word bits [0, 4) (128 bytes), then
// alternately runs of tile bits (box = the whole run, split at 8 bits) and
// runs of free bits (box 1; coordinate = the tile base's bits there).  A tile
// is then one box, and the tensor map's 128-byte swizzle puts 16-byte chunk j
// of 128-byte row r at chunk j ^ (r & 7): the chunk layout the register
// phases use, so they read TMA-loaded tiles unchanged.
struct alignas(64) TmaDesc {
  CUtensorMap src;     // over the buffer the sweep reads (k_adj: psi)
  CUtensorMap dst;     // over the buffer it writes, the same one in place (k_adj: lam)
  uint32_t bytes;      // one tile: the transaction count of one load
  uint8_t ndim;        // 5 when the sweep runs in TMA form, else 0
  uint8_t store;       // plain write-backs go out as TMA stores
  uint8_t start[5];    // free dimension: first index bit of its run
  uint32_t mask[5];    // free dimension: 2^len - 1 (0: a tile dimension)
  // host side: the maps' shape (words of 8 bytes), encoded at launch
  cuuint64_t gdim[5];
  cuuint64_t gstride[4];
  cuuint32_t box[5];
};
// a tile load that has not arrived after this long abandons the sweep
constexpr uint64_t kTmaWaitNs = 2000000000ull;

// ---------------------------------------------------------------- limits
// 31 qubits at most, the reference's limit (execution.py:23-25): the
// amplitude count 2^n is carried in 32-bit variables (launch sizes, the
// reductions' dimension), which cannot hold 2^32.
constexpr int kMaxQubits = 31;
constexpr int kTileMaxC64 = 13;       // 2^13 complex64 = 64 KiB tile
constexpr int kTileMaxC128 = 12;      // 2^12 complex128 = 64 KiB tile

// ---------------------------------------------------------------- tile bases
// The base index of tile t of a sweep: t's bits deposited, in ascending
// order, into the index bits that are not tile bits.  Those free bits form
// at most (tile bits + 1) contiguous runs; run j takes t's bits
// [src[j], src[j] + len) (mask = 2^len - 1) to index bits [dst[j], ...).
// One shift, mask and shift per run replaces a per-tile-bit insertion loop.
constexpr int kMaxRuns = 14;
struct BaseRuns {
  uint8_t n;
  uint8_t src[kMaxRuns];
  uint8_t dst[kMaxRuns];
  uint8_t pad;
  uint32_t mask[kMaxRuns];
};
__host__ __device__ __forceinline__ uint32_t deposit_runs(uint32_t t, const BaseRuns& R) {
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < kMaxRuns; ++j) {
    if (j >= R.n) break;
    x |= ((t >> R.src[j]) & R.mask[j]) << R.dst[j];
  }
  return x;
}
// tile_bits: the m tile bits of an n-qubit index, ascending, m <= 13.
inline void make_base_runs(BaseRuns& R, int n, const uint8_t* tile_bits, int m) {
  R = BaseRuns{};
  uint32_t tmask = 0;
  for (int k = 0; k < m; ++k) tmask |= 1u << tile_bits[k];
  int src = 0;
  for (int b = 0; b < n;) {
    if ((tmask >> b) & 1u) { ++b; continue; }
    const int start = b;
    while (b < n && !((tmask >> b) & 1u)) ++b;
    const int len = b - start;
    R.src[R.n] = (uint8_t)src;
    R.dst[R.n] = (uint8_t)start;
    R.mask[R.n] = len >= 32 ? 0xffffffffu : ((1u << len) - 1u);
    src += len;
    ++R.n;
  }
}

// ---------------------------------------------------------------- errors
void set_error(int code, const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);

#define MQ_CUDA(call)                                                   \
  do {                                                                  \
    cudaError_t _e = (call);                                            \
    if (_e != cudaSuccess) return ::mq::cuda_fail(_e, #call);           \
  } while (0)

#define MQ_LAUNCHED(where)                                              \
  do {                                                                  \
    cudaError_t _e = cudaGetLastError();                                \
    if (_e != cudaSuccess) return ::mq::cuda_fail(_e, where);           \
  } while (0)

}  // namespace mq

// ---------------------------------------------------------------- handle
struct mq_state {
  int n = 0;
  int dtype = MQ_C64;
  int device = 0;
  int num_sms = 148;         // SMs the launch grids are sized for (mq_state_set_sm_limit)
  int device_sms = 148;      // SMs of the device
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void* buf[2] = {nullptr, nullptr};
  int cur = 0;
  size_t state_bytes = 0;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  uint64_t launches = 0;
  uint64_t sweeps = 0;
  // sweep plan of this handle (0 / -1: the process-wide defaults): largest
  // tile (bits), low passenger bits of a high sweep, smallest tile
  int tile_max = 0;
  int tile_pas = -1;
  int tile_min = 0;

  size_t amp_bytes() const { return dtype == MQ_C64 ? 8 : 16; }
  uint64_t dim() const { return uint64_t(1) << n; }
  void* cur_buf() const { return buf[cur]; }
};

namespace mq {

// Make the handle's device current for the duration of a call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
};

int ensure_scratch(mq_state* h, size_t bytes);
int ensure_alt(mq_state* h);  // allocate the second buffer if absent
// After a synchronisation: MQ_ETIMEOUT (and the flag cleared) when a tile
// sweep on the handle's device abandoned its work because a tile load did not
// arrive in time, else MQ_OK (mq_tile.cu).
int check_tile_fault(mq_state* h);
// Looks up the driver's tensor-map encoder once per process (state creation
// calls it, so that no lookup happens inside a stream capture).
void prepare_tile_maps();
// TMA tiles (mq_tile.cu): on unless MQ_TMA=0; the shape of a sweep's tiles
// (false when the TMA form cannot describe it); the two maps of a launch.
bool tma_enabled();
bool plan_tma(int n, size_t amp_bytes, const std::vector<int>& tile_bits, TmaDesc& D);
int encode_tile_maps(TmaDesc& D, void* src, void* dst);
// The adjoint sweeps' abandoned-work flag, read and cleared (mq_adjoint.cu).
int take_adj_fault(mq_state* h, bool* fault);

// ------------------------------------------------------------ launchers
// Tile sweeps: U(2) layer and QFT (mq_tile.cu)
int launch_u2_layer(mq_state* h, const double* mats, const uint8_t* active);
int launch_qft_contiguous(mq_state* h, int q0, int k, int inverse);
int launch_qft_stages(mq_state* h, int q0, int k, int j_begin, int j_end, int inverse);
int launch_cu2_list(mq_state* h, int n_gates, const int32_t* targets, const uint32_t* cmasks, const double* mats);
// Diagonal layers (mq_diag.cu)
int launch_diag_terms(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires,
                      const double* params);
// A diagonal factored into <= 8 tables indexed by contiguous index windows:
// phase(x) = prod_w vals[off[w] + ((x >> shift[w]) & (2^nbits[w] - 1))]
// (vals: re, im interleaved).  Planned by mq_diag.cu for tile epilogues.
struct DiagWindows {
  int n = 0;  // -1: not representable within the budget
  int shift[8] = {}, nbits[8] = {}, off[8] = {};
  std::vector<double> vals;
};
int plan_diag_windows(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params,
                      int max_entries, DiagWindows& out);
// A diagonal factored for a 4-bit register phase (plan_diag_register):
// window tables (win, evaluated at the register group's base) followed, at
// entry t_off, by T[c][r] (row c at t_off + 17c, 17 << nc entries) indexed by the register bits r
// and the cross bits c = bits cbit[0..nc) of the index.
struct DiagRegister {
  DiagWindows win;
  int nc = 0;
  int cbit[3] = {};
  int t_off = 0;
};
int plan_diag_register(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params,
                       const int* rbits, int max_entries, DiagRegister& out);
// Fused layer: U(2) on every active qubit, then the diagonal terms, then the
// GF(2) permutation out[y] = in[A y ^ c] (cols = A e_j; null = none)
// (mq_tile.cu).
// mats == NULL with mats_dev: the U(2) matrices are read from device memory
// (n rows of 8 doubles) when the sweeps run, so a captured graph of the
// layer stays valid when the matrices change.
int launch_layer(mq_state* h, const double* mats, const uint8_t* active, int n_terms, const int32_t* kinds,
                 const int32_t* wires, const double* params, const uint32_t* cols, uint32_t c,
                 const double* mats_dev = nullptr);
// GF(2) affine permutation, out-of-place into the alternate buffer (mq_perm.cu).
// cols[j] = A e_j (index-bit columns of the source map), c = flip constant.
int launch_affine_cols(mq_state* h, const uint32_t* cols, uint32_t c);
// Reductions (mq_reduce.cu)
int run_probabilities(mq_state* h, const int32_t* wires, int k, int out_dtype, void* out);
int run_probabilities_device(mq_state* h, int out_dtype, void* out_dev);
int run_sample(mq_state* h, const int32_t* wires, int k, uint64_t seed, uint64_t offset,
               int64_t shots, int64_t* out);
int run_expval_pauli(mq_state* h, int n_words, const uint64_t* xmask, const uint64_t* zmask,
                     const int32_t* ny, double* out);
// Same values through a fixed file-scope device array: allocates nothing.
int run_expval_pauli_static(mq_state* h, int n_words, const uint64_t* xmask, const uint64_t* zmask,
                            const int32_t* ny, double* out);

// Adjoint method (mq_adjoint.cu): one backward layer on (psi, lam), and
// lam = H psi for H = sum_w zcoef_w Z-word_w + sum_q xcoef_q X_q.
// perm_cols / perm_c: a GF(2) map out[x] = in[A x ^ c] (A by its columns)
// un-applied from both states before the layer, fused into the layer's first
// sweep where that sweep's form allows
int adjoint_sweep(mq_state* psi, mq_state* lam, int n_q, const int32_t* qubits, const double* mats, double* out,
                  bool out_on_device, const uint32_t* perm_cols = nullptr, uint32_t perm_c = 0);
int apply_hamiltonian(mq_state* psi, mq_state* lam, int n_z, const uint64_t* zmasks, const double* zcoef,
                      const double* xcoef, double* energy);

// GF(2) helpers (host)
bool gf2_invert(int n, const uint32_t* cols, uint32_t* inv_cols);

}  // namespace mq
