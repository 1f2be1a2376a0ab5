// C ABI of libmq: state handles, error reporting and the layer entry points
// declared in include/mq.h.  Each entry point validates its arguments on the
// host, makes the handle's device current and enqueues work on the handle's
// stream; nothing throws across the boundary.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "mq_internal.cuh"

namespace mq {

static thread_local std::string g_last_error;
static thread_local int g_last_code = MQ_OK;

void set_error(int code, const std::string& msg) {
  g_last_code = code;
  g_last_error = msg;
}

int fail(int code, const std::string& msg) {
  set_error(code, msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  const int code = (e == cudaErrorMemoryAllocation) ? MQ_ENOMEM : MQ_EDEVICE;
  return fail(code, std::string(where) + ": " + cudaGetErrorString(e));
}

int ensure_scratch(mq_state* h, size_t bytes) {
  if (h->scratch_bytes >= bytes) return MQ_OK;
  size_t want = std::max(bytes, h->scratch_bytes * 2);
  want = (want + 4095) & ~size_t(4095);
  if (h->scratch) {
    MQ_CUDA(cudaStreamSynchronize(h->stream));
    MQ_CUDA(cudaFree(h->scratch));
    h->scratch = nullptr;
    h->scratch_bytes = 0;
  }
  MQ_CUDA(cudaMalloc(&h->scratch, want));
  h->scratch_bytes = want;
  return MQ_OK;
}

int ensure_alt(mq_state* h) {
  const int alt = 1 - h->cur;
  if (h->buf[alt]) return MQ_OK;
  MQ_CUDA(cudaMalloc(&h->buf[alt], h->state_bytes));
  return MQ_OK;
}

}  // namespace mq

using namespace mq;

#define MQ_TRY_BEGIN try {
#define MQ_TRY_END                                                      \
  }                                                                     \
  catch (const std::bad_alloc&) { return fail(MQ_ENOMEM, "host allocation failed"); } \
  catch (const std::exception& ex) { return fail(MQ_EDEVICE, ex.what()); } \
  catch (...) { return fail(MQ_EDEVICE, "unknown C++ exception"); }

#define MQ_CHECK_HANDLE(h) \
  if (!(h)) return fail(MQ_EINVAL, "null state handle")

extern "C" {

const char* mq_last_error(void) { return g_last_error.c_str(); }

int mq_version(void) { return 1; }

int mq_device_count(int* out) {
  if (!out) return fail(MQ_EINVAL, "null output");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = 0;
    return MQ_OK;
  }
  *out = c;
  return MQ_OK;
}

int mq_state_footprint(int n, int dtype, int double_buffered, uint64_t* out_bytes) {
  if (!out_bytes) return fail(MQ_EINVAL, "null output");
  if (n < 1 || n > kMaxQubits) return fail(MQ_EINVAL, "n_qubits must be in [1, 31]");
  if (dtype != MQ_C64 && dtype != MQ_C128) return fail(MQ_EINVAL, "dtype must be MQ_C64 or MQ_C128");
  const uint64_t amp = dtype == MQ_C64 ? 8 : 16;
  const uint64_t state = (uint64_t(1) << n) * amp;
  *out_bytes = state * (double_buffered ? 2 : 1);
  return MQ_OK;
}

int mq_state_create(int n, int dtype, int device, void* stream, mq_state** out) {
  MQ_TRY_BEGIN
  if (!out) return fail(MQ_EINVAL, "null output handle");
  *out = nullptr;
  if (n < 1 || n > kMaxQubits) return fail(MQ_EINVAL, "n_qubits must be in [1, 31]");
  if (dtype != MQ_C64 && dtype != MQ_C128) return fail(MQ_EINVAL, "dtype must be MQ_C64 or MQ_C128");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(MQ_EDEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= ndev) return fail(MQ_EINVAL, "device index out of range");
  DeviceGuard g(device);
  const uint64_t bytes = (uint64_t(1) << n) * (dtype == MQ_C64 ? 8 : 16);
  size_t free_b = 0, total_b = 0;
  MQ_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes > free_b) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "Refusing %d-qubit statevector before allocation: one state is %.2f GiB and the device has %.2f GiB free",
                  n, bytes / 1073741824.0, free_b / 1073741824.0);
    return fail(MQ_ENOMEM, msg);
  }
  prepare_tile_maps();
  auto* h = new mq_state();
  h->n = n;
  h->dtype = dtype;
  h->device = device;
  h->state_bytes = (size_t)bytes;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) {
    h->num_sms = sms;
    h->device_sms = sms;
  }
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaStreamCreate"); }
    h->own_stream = true;
  }
  cudaError_t e = cudaMalloc(&h->buf[0], h->state_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return cuda_fail(e, "cudaMalloc(state)");
  }
  *out = h;
  return mq_state_reset(h);
  MQ_TRY_END
}

int mq_state_destroy(mq_state* h) {
  if (!h) return MQ_OK;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  for (int i = 0; i < 2; ++i)
    if (h->buf[i]) cudaFree(h->buf[i]);
  if (h->scratch) cudaFree(h->scratch);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  delete h;
  return MQ_OK;
}

int mq_state_info(const mq_state* h, int* n, int* dtype, int* device) {
  MQ_CHECK_HANDLE(h);
  if (n) *n = h->n;
  if (dtype) *dtype = h->dtype;
  if (device) *device = h->device;
  return MQ_OK;
}

int mq_state_set_stream(mq_state* h, void* stream) {
  MQ_CHECK_HANDLE(h);
  DeviceGuard g(h->device);
  if (h->own_stream) {
    MQ_CUDA(cudaStreamSynchronize(h->stream));
    cudaStreamDestroy(h->stream);
    h->own_stream = false;
  }
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    MQ_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return MQ_OK;
}

int mq_state_set_sm_limit(mq_state* h, int sms) {
  MQ_CHECK_HANDLE(h);
  h->num_sms = (sms <= 0 || sms > h->device_sms) ? h->device_sms : sms;
  return MQ_OK;
}

int mq_state_stream(const mq_state* h, void** out) {
  MQ_CHECK_HANDLE(h);
  if (!out) return fail(MQ_EINVAL, "null output");
  *out = (void*)h->stream;
  return MQ_OK;
}

int mq_state_reset(mq_state* h) {
  MQ_CHECK_HANDLE(h);
  DeviceGuard g(h->device);
  MQ_CUDA(cudaMemsetAsync(h->cur_buf(), 0, h->state_bytes, h->stream));
  if (h->dtype == MQ_C64) {
    static const float one[2] = {1.0f, 0.0f};
    MQ_CUDA(cudaMemcpyAsync(h->cur_buf(), one, sizeof(one), cudaMemcpyHostToDevice, h->stream));
  } else {
    static const double one[2] = {1.0, 0.0};
    MQ_CUDA(cudaMemcpyAsync(h->cur_buf(), one, sizeof(one), cudaMemcpyHostToDevice, h->stream));
  }
  return MQ_OK;
}

int mq_state_set(mq_state* h, const void* host_amps) {
  MQ_CHECK_HANDLE(h);
  if (!host_amps) return fail(MQ_EINVAL, "null host buffer");
  DeviceGuard g(h->device);
  MQ_CUDA(cudaMemcpyAsync(h->cur_buf(), host_amps, h->state_bytes, cudaMemcpyHostToDevice, h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  return MQ_OK;
}

int mq_state_get(mq_state* h, void* host_amps) {
  MQ_CHECK_HANDLE(h);
  if (!host_amps) return fail(MQ_EINVAL, "null host buffer");
  DeviceGuard g(h->device);
  MQ_CUDA(cudaMemcpyAsync(host_amps, h->cur_buf(), h->state_bytes, cudaMemcpyDeviceToHost, h->stream));
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  return check_tile_fault(h);
}

int mq_state_copy(mq_state* dst, const mq_state* src) {
  MQ_CHECK_HANDLE(dst);
  MQ_CHECK_HANDLE(src);
  if (dst->n != src->n || dst->dtype != src->dtype) return fail(MQ_EINVAL, "state shapes differ");
  DeviceGuard g(dst->device);
  MQ_CUDA(cudaStreamSynchronize(src->stream));
  MQ_CUDA(cudaMemcpyAsync(dst->cur_buf(), src->cur_buf(), dst->state_bytes, cudaMemcpyDeviceToDevice, dst->stream));
  return MQ_OK;
}

int mq_state_device_ptr(mq_state* h, void** out) {
  MQ_CHECK_HANDLE(h);
  if (!out) return fail(MQ_EINVAL, "null output");
  *out = h->cur_buf();
  return MQ_OK;
}

int mq_sync(mq_state* h) {
  MQ_CHECK_HANDLE(h);
  DeviceGuard g(h->device);
  MQ_CUDA(cudaStreamSynchronize(h->stream));
  return check_tile_fault(h);
}

int mq_state_counters(const mq_state* h, uint64_t* launches, uint64_t* sweeps) {
  MQ_CHECK_HANDLE(h);
  if (launches) *launches = h->launches;
  if (sweeps) *sweeps = h->sweeps;
  return MQ_OK;
}

int mq_apply_u2_layer(mq_state* h, const double* mats, const uint8_t* active) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (!mats) return fail(MQ_EINVAL, "null matrices");
  DeviceGuard g(h->device);
  return launch_u2_layer(h, mats, active);
  MQ_TRY_END
}

int mq_apply_u2_uniform(mq_state* h, const double* mat4) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (!mat4) return fail(MQ_EINVAL, "null matrix");
  std::vector<double> mats((size_t)h->n * 8);
  for (int q = 0; q < h->n; ++q) std::memcpy(&mats[(size_t)q * 8], mat4, 8 * sizeof(double));
  DeviceGuard g(h->device);
  return launch_u2_layer(h, mats.data(), nullptr);
  MQ_TRY_END
}

int mq_apply_controlled_u2(mq_state* h, int n_gates, const int32_t* targets, const int32_t* coff,
                           const int32_t* controls, const double* mats) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (n_gates < 0) return fail(MQ_EINVAL, "negative gate count");
  if (n_gates == 0) return MQ_OK;
  if (!targets || !coff || !mats || (coff[n_gates] > 0 && !controls)) return fail(MQ_EINVAL, "null gate arrays");
  const int n = h->n;
  std::vector<uint32_t> cmasks(n_gates, 0);
  for (int g = 0; g < n_gates; ++g) {
    if (targets[g] < 0 || targets[g] >= n) return fail(MQ_EINVAL, "Qubit index out of range");
    if (coff[g + 1] < coff[g]) return fail(MQ_EINVAL, "bad control offsets");
    for (int c = coff[g]; c < coff[g + 1]; ++c) {
      const int q = controls[c];
      if (q < 0 || q >= n) return fail(MQ_EINVAL, "Qubit index out of range");
      if (q == targets[g]) return fail(MQ_EINVAL, "Control and target must differ");
      const uint32_t bit = 1u << (n - 1 - q);
      if (cmasks[g] & bit) return fail(MQ_EINVAL, "Control/target wires must be distinct");
      cmasks[g] |= bit;
    }
  }
  DeviceGuard g(h->device);
  return launch_cu2_list(h, n_gates, targets, cmasks.data(), mats);
  MQ_TRY_END
}

int mq_apply_qft_stages(mq_state* h, int q0, int k, int j_begin, int j_end, int inverse) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (!(0 <= j_begin && j_begin <= j_end && j_end <= k && q0 >= 0 && q0 + k <= h->n))
    return fail(MQ_EINVAL, "qft_stage_sub: invalid stage range");
  DeviceGuard g(h->device);
  return launch_qft_stages(h, q0, k, j_begin, j_end, inverse);
  MQ_TRY_END
}

int mq_apply_diag_terms(mq_state* h, int n_terms, const int32_t* kinds, const int32_t* wires, const double* params) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (n_terms < 0) return fail(MQ_EINVAL, "negative term count");
  if (n_terms == 0) return MQ_OK;
  if (!kinds || !wires || !params) return fail(MQ_EINVAL, "null term arrays");
  DeviceGuard g(h->device);
  return launch_diag_terms(h, n_terms, kinds, wires, params);
  MQ_TRY_END
}

int mq_apply_diag_layer(mq_state* h, int kind, int n_bonds, const int32_t* bonds, const double* thetas) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (kind != MQ_DIAG_ZZ && kind != MQ_DIAG_CPHASE) return fail(MQ_EINVAL, "diag layer kind must be ZZ or CPHASE");
  if (n_bonds < 0) return fail(MQ_EINVAL, "negative bond count");
  if (n_bonds == 0) return MQ_OK;
  if (!bonds || !thetas) return fail(MQ_EINVAL, "null bond arrays");
  std::vector<int32_t> kinds(n_bonds, kind);
  std::vector<double> params((size_t)n_bonds * 8, 0.0);
  for (int b = 0; b < n_bonds; ++b) params[(size_t)b * 8] = thetas[b];
  DeviceGuard g(h->device);
  return launch_diag_terms(h, n_bonds, kinds.data(), bonds, params.data());
  MQ_TRY_END
}

int mq_apply_qft(mq_state* h, const int32_t* wires, int k, int inverse) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  const int n = h->n;
  if (k < 0 || k > n) return fail(MQ_EINVAL, "bad QFT wire count");
  if (k == 0) return MQ_OK;
  if (!wires) return fail(MQ_EINVAL, "null QFT wires");
  std::vector<bool> seen(n, false);
  for (int i = 0; i < k; ++i) {
    if (wires[i] < 0 || wires[i] >= n) return fail(MQ_EINVAL, "Qubit index out of range");
    if (seen[wires[i]]) return fail(MQ_EINVAL, "Duplicate QFT wire indices");
    seen[wires[i]] = true;
  }
  DeviceGuard g(h->device);
  bool contiguous = true;
  for (int i = 1; i < k; ++i)
    if (wires[i] != wires[0] + i) contiguous = false;
  if (contiguous) return launch_qft_contiguous(h, wires[0], k, inverse);
  // Move wire j to qubit j (others keep their relative order after them),
  // run the contiguous QFT on qubits [0, k), and move back.  Wire
  // permutations are GF(2) linear, so each move is one permutation sweep.
  std::vector<int> sigma(n, -1);  // old qubit -> new qubit
  int next = k;
  for (int j = 0; j < k; ++j) sigma[wires[j]] = j;
  for (int q = 0; q < n; ++q)
    if (sigma[q] < 0) sigma[q] = next++;
  uint32_t fwd[32], back[32];
  for (int q = 0; q < n; ++q) {
    fwd[n - 1 - sigma[q]] = 1u << (n - 1 - q);
    back[n - 1 - q] = 1u << (n - 1 - sigma[q]);
  }
  int rc = launch_affine_cols(h, fwd, 0);
  if (rc) return rc;
  rc = launch_qft_contiguous(h, 0, k, inverse);
  if (rc) return rc;
  return launch_affine_cols(h, back, 0);
  MQ_TRY_END
}

// rows (inverse-map rows, qubit k = row k) -> columns A e_j of the source
// map over index bits; validates the masks.
static int rows_to_cols(const mq_state* h, const uint64_t* rows, uint64_t c, uint32_t* cols) {
  const int n = h->n;
  const uint64_t lim = h->dim() - 1;
  if (c & ~lim) return fail(MQ_EINVAL, "flip constant outside the register");
  for (int j = 0; j < n; ++j) cols[j] = 0;
  for (int k = 0; k < n; ++k) {
    if (rows[k] & ~lim) return fail(MQ_EINVAL, "affine row outside the register");
    for (int j = 0; j < n; ++j)
      if ((rows[k] >> j) & 1u) cols[j] |= 1u << (n - 1 - k);
  }
  return MQ_OK;
}

int mq_apply_layer(mq_state* h, const double* mats, const uint8_t* active, int n_terms, const int32_t* kinds,
                   const int32_t* wires, const double* params, const uint64_t* rows, uint64_t c) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (n_terms < 0) return fail(MQ_EINVAL, "negative term count");
  if (n_terms > 0 && (!kinds || !wires || !params)) return fail(MQ_EINVAL, "null term arrays");
  uint32_t cols[32];
  if (rows) {
    int rc = rows_to_cols(h, rows, c, cols);
    if (rc) return rc;
  }
  DeviceGuard g(h->device);
  return launch_layer(h, mats, active, n_terms, kinds, wires, params, rows ? cols : nullptr, (uint32_t)c);
  MQ_TRY_END
}

int mq_apply_xor_affine(mq_state* h, const uint64_t* rows, uint64_t c) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (!rows) return fail(MQ_EINVAL, "null rows");
  uint32_t cols[32];
  int rc = rows_to_cols(h, rows, c, cols);
  if (rc) return rc;
  DeviceGuard g(h->device);
  return launch_affine_cols(h, cols, (uint32_t)c);
  MQ_TRY_END
}

int mq_probabilities(mq_state* h, const int32_t* wires, int k, int out_dtype, void* out) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (!out) return fail(MQ_EINVAL, "null output");
  if (out_dtype != 0 && out_dtype != 1) return fail(MQ_EINVAL, "out_dtype must be 0 (float32) or 1 (float64)");
  DeviceGuard g(h->device);
  // k == 0 with a wire list is the empty marginal: the total probability
  // ([1] for a normalised state, sim.py:322-328), reduced like any marginal.
  return run_probabilities(h, wires, k, out_dtype, out);
  MQ_TRY_END
}

int mq_probabilities_device(mq_state* h, int out_dtype, void* out_dev) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (!out_dev) return fail(MQ_EINVAL, "null output");
  if (out_dtype != 0 && out_dtype != 1) return fail(MQ_EINVAL, "out_dtype must be 0 (float32) or 1 (float64)");
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, out_dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(MQ_EINVAL, "output is not a device pointer");
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
    return fail(MQ_EINVAL, "output is not device memory");
  if (attr.type == cudaMemoryTypeDevice && attr.device != h->device)
    return fail(MQ_EINVAL, "output lives on another device than the state");
  DeviceGuard g(h->device);
  return run_probabilities_device(h, out_dtype, out_dev);
  MQ_TRY_END
}

int mq_sample(mq_state* h, const int32_t* wires, int k, uint64_t seed, uint64_t stream_offset, int64_t shots,
              int64_t* out) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (shots > 0 && !out) return fail(MQ_EINVAL, "null output");
  DeviceGuard g(h->device);
  return run_sample(h, wires, k, seed, stream_offset, shots, out);
  MQ_TRY_END
}

int mq_expval_pauli(mq_state* h, int n_words, const uint64_t* xmask, const uint64_t* zmask, const int32_t* ny,
                    double* out) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (n_words < 0) return fail(MQ_EINVAL, "negative word count");
  if (n_words == 0) return MQ_OK;
  if (!xmask || !zmask || !out) return fail(MQ_EINVAL, "null Pauli arrays");
  DeviceGuard g(h->device);
  return run_expval_pauli(h, n_words, xmask, zmask, ny, out);
  MQ_TRY_END
}

static int check_pair(const mq_state* a, const mq_state* b) {
  if (!a || !b) return fail(MQ_EINVAL, "null state handle");
  if (a == b) return fail(MQ_EINVAL, "the two states must be different handles");
  if (a->n != b->n || a->dtype != b->dtype || a->device != b->device)
    return fail(MQ_EINVAL, "states differ in qubit count, dtype or device");
  if (a->stream != b->stream) return fail(MQ_EINVAL, "both states must be bound to the same stream");
  return MQ_OK;
}

int mq_apply_pauli_sum(mq_state* psi, mq_state* out, int n_z, const uint64_t* zmasks, const double* zcoef,
                       const double* xcoef, double* energy) {
  MQ_TRY_BEGIN
  int rc = check_pair(psi, out);
  if (rc) return rc;
  if (n_z < 0 || (n_z > 0 && (!zmasks || !zcoef))) return fail(MQ_EINVAL, "invalid Z-word arrays");
  DeviceGuard g(psi->device);
  return apply_hamiltonian(psi, out, n_z, zmasks, zcoef, xcoef, energy);
  MQ_TRY_END
}

int mq_adjoint_layer(mq_state* psi, mq_state* lam, int n_q, const int32_t* qubits, const double* mats,
                     double* out) {
  MQ_TRY_BEGIN
  int rc = check_pair(psi, lam);
  if (rc) return rc;
  if (n_q < 0) return fail(MQ_EINVAL, "negative qubit count");
  if (n_q == 0) return MQ_OK;
  if (!qubits || !mats) return fail(MQ_EINVAL, "null layer arrays");
  DeviceGuard g(psi->device);
  return adjoint_sweep(psi, lam, n_q, qubits, mats, out, false);
  MQ_TRY_END
}

int mq_adjoint_layer_async(mq_state* psi, mq_state* lam, int n_q, const int32_t* qubits, const double* mats,
                           double* out_dev) {
  MQ_TRY_BEGIN
  int rc = check_pair(psi, lam);
  if (rc) return rc;
  if (n_q < 0) return fail(MQ_EINVAL, "negative qubit count");
  if (n_q == 0) return MQ_OK;
  if (!qubits || !mats || !out_dev) return fail(MQ_EINVAL, "null layer arrays");
  DeviceGuard g(psi->device);
  return adjoint_sweep(psi, lam, n_q, qubits, mats, out_dev, true);
  MQ_TRY_END
}

int mq_adjoint_layer_xor_async(mq_state* psi, mq_state* lam, const uint64_t* rows, uint64_t c, int n_q,
                               const int32_t* qubits, const double* mats, double* out_dev) {
  MQ_TRY_BEGIN
  int rc = check_pair(psi, lam);
  if (rc) return rc;
  if (!rows) return fail(MQ_EINVAL, "null rows");
  if (n_q < 0) return fail(MQ_EINVAL, "negative qubit count");
  if (n_q > 0 && (!qubits || !mats || !out_dev)) return fail(MQ_EINVAL, "null layer arrays");
  uint32_t cols[32];
  rc = rows_to_cols(psi, rows, c, cols);
  if (rc) return rc;
  DeviceGuard g(psi->device);
  if (n_q == 0) {
    rc = launch_affine_cols(psi, cols, (uint32_t)c);
    return rc ? rc : launch_affine_cols(lam, cols, (uint32_t)c);
  }
  return adjoint_sweep(psi, lam, n_q, qubits, mats, out_dev, true, cols, (uint32_t)c);
  MQ_TRY_END
}

// Allocation-free variant of mq_expval_pauli; see include/mq.h.
int mq_expval_pauli_static(mq_state* h, int n_words, const uint64_t* xmask, const uint64_t* zmask,
                           const int32_t* ny, double* out) {
  MQ_TRY_BEGIN
  MQ_CHECK_HANDLE(h);
  if (n_words < 0) return fail(MQ_EINVAL, "negative word count");
  if (n_words == 0) return MQ_OK;
  if (!xmask || !zmask || !out) return fail(MQ_EINVAL, "null Pauli arrays");
  DeviceGuard g(h->device);
  return run_expval_pauli_static(h, n_words, xmask, zmask, ny, out);
  MQ_TRY_END
}

}  // extern "C"
