/*
 * mq.h -- C ABI of the B200 statevector engine (libmq.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, integer status codes.
 * No C++ exception and no torch type crosses this boundary.  Every entry
 * point returns MQ_OK (0) or an MQ_E* code; mq_last_error() returns a
 * thread-local message for the last failure on the calling thread.
 *
 * Conventions shared with the reference (MettleQ, method="statevector"):
 *   - amplitudes are complex64 (dtype MQ_C64; interleaved float re, im) or
 *     complex128 (MQ_C128, the FP64 oracle build), execution.py:21-22;
 *   - qubit q is state-index bit n-1-q (MSB-first), sim.py:10-14;
 *   - the initial state is |0...0>, sim.py:32-45;
 *   - layer calls act on the handle's state in place from the caller's
 *     point of view (the reference rebinds a new functional array,
 *     device.py:309-379; here a double buffer is swapped internally).
 *
 * Threading: every handle is bound to one CUDA stream; launches are
 * asynchronous on it.  Calls on one handle must be serialised by the caller;
 * different handles are independent.  mq_sync() is the equivalent of the
 * reference's Device.synchronize() (device.py:541-554).
 */
#ifndef MQ_H
#define MQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum mq_status {
  MQ_OK = 0,
  MQ_EINVAL = 1,      /* bad argument: ValueError in the reference (diag.py:129-131, zz.py:103-106, qft.py:151-152) */
  MQ_ENOMEM = 2,      /* refused or failed allocation: StatevectorMemoryError (execution.py:33-38, 377-407) */
  MQ_EDEVICE = 3,     /* CUDA/device failure: RuntimeError (device.py:97-139) */
  MQ_ETIMEOUT = 4,    /* a bounded device wait gave up */
  MQ_EUNSUPPORTED = 5 /* request outside what the library supports */
};

enum mq_dtype { MQ_C64 = 0, MQ_C128 = 1 };

/* Diagonal term kinds for mq_apply_diag_terms / mq_apply_diag_layer. */
enum mq_diag_kind {
  MQ_DIAG_ZZ = 0,      /* exp(-i t Z_a Z_b), the reference's native ZZPHASE (sim.py:260-264) */
  MQ_DIAG_CPHASE = 1,  /* diag(1,1,1,e^{i t}) on (a,b); CZ is t = pi (gates.py:120-138) */
  MQ_DIAG_RZ = 2,      /* diag(e^{-i t/2}, e^{+i t/2}) on a (gates.py:64-68) */
  MQ_DIAG_PHASE = 3,   /* diag(1, e^{i t}) on a: U1/P, Z=pi, S=pi/2, T=pi/4 (gates.py:71-77) */
  MQ_DIAG_CRZ = 4,     /* controlled RZ(t), control a, target b (device.py:1206-1208) */
  MQ_DIAG_GLOBAL = 5,  /* scalar e^{i t} (integrations/_common.py:231-238) */
  MQ_DIAG_1Q = 6,      /* explicit diag(d0, d1) on a; params p[0..3] = d0.re, d0.im, d1.re, d1.im */
  MQ_DIAG_2Q = 7       /* explicit 4-entry diagonal on (a,b), first wire = MSB; params p[0..7] */
};

typedef struct mq_state mq_state;

/* ---- library ------------------------------------------------------------ */
const char* mq_last_error(void);
int mq_version(void);
int mq_device_count(int* out);
/* Device bytes a state of n qubits holds: buffers (1 or 2) plus scratch. */
int mq_state_footprint(int n, int dtype, int double_buffered, uint64_t* out_bytes);

/* ---- state handles (StateVectorSimulator, sim.py:17-45) ------------------ */
/* stream: a cudaStream_t, or NULL for a stream owned by the handle.
 * Refuses n outside [1, 31] with MQ_EINVAL (the reference's limit,
 * execution.py:23-25: 2^n amplitudes are counted in 32 bits) and
 * allocation failure with MQ_ENOMEM, before touching device memory. */
int mq_state_create(int n, int dtype, int device, void* stream, mq_state** out);
int mq_state_destroy(mq_state* h);
int mq_state_info(const mq_state* h, int* n, int* dtype, int* device);
int mq_state_set_stream(mq_state* h, void* stream);
/* The stream the handle launches on (its own or the caller's). */
int mq_state_stream(const mq_state* h, void** out);
/* Size this handle's launch grids for at most `sms` SMs (<= 0: all), so that
 * kernels of other streams find free SMs while its kernels run (a serving
 * loop keeps a reserve for short requests this way). */
int mq_state_set_sm_limit(mq_state* h, int sms);
int mq_state_reset(mq_state* h);                       /* sim.py:32-45 */
int mq_state_set(mq_state* h, const void* host_amps);  /* 2^n amplitudes */
int mq_state_get(mq_state* h, void* host_amps);
int mq_state_copy(mq_state* dst, const mq_state* src); /* same n and dtype */
int mq_state_device_ptr(mq_state* h, void** out);      /* current buffer */
int mq_sync(mq_state* h);                               /* device.py:541-554 */
/* Launch accounting since creation (the reference's dispatch evidence,
 * execution.py:657-780): kernels launched and full-state sweeps executed. */
int mq_state_counters(const mq_state* h, uint64_t* launches, uint64_t* sweeps);

/* ---- (a) single-qubit layer (shaders/single_qubit.py:422-615) ----------- */
/* mats: n x 4 complex as doubles [q][u00.re,u00.im,u01.re,...,u11.im];
 * active: n bytes (nonzero = apply) or NULL for all qubits. */
int mq_apply_u2_layer(mq_state* h, const double* mats, const uint8_t* active);
/* Replaces u2_layer_all (single_qubit.py:422-509): one matrix on every qubit. */
int mq_apply_u2_uniform(mq_state* h, const double* mat4);

/* Controlled single-qubit gates applied in list order (CH/CRX/CRY and the
 * doubly controlled X of Toffoli; controlled_single.py:18-134, sim.py:140-213):
 * gate g acts on qubit targets[g] when every qubit in controls[coff[g] ..
 * coff[g+1]) is 1; mats as in mq_apply_u2_layer, one 2x2 per gate. */
int mq_apply_controlled_u2(mq_state* h, int n_gates, const int32_t* targets,
                           const int32_t* coff, const int32_t* controls,
                           const double* mats);

/* ---- (b) diagonal layers (shaders/diag.py, shaders/zz.py, sim.py:94-138) - */
/* kinds[t], wires[2t], wires[2t+1] (b = -1 for one-wire kinds), params[8t..8t+7]. */
int mq_apply_diag_terms(mq_state* h, int n_terms, const int32_t* kinds,
                        const int32_t* wires, const double* params);
/* Replaces diag_weighted_layer / zz_weighted_layer (diag.py:123-167,
 * zz.py:99-140): one kind (MQ_DIAG_ZZ or MQ_DIAG_CPHASE) over bonds[2*B]
 * with per-bond angles thetas[B]. */
int mq_apply_diag_layer(mq_state* h, int kind, int n_bonds, const int32_t* bonds,
                        const double* thetas);

/* ---- fused layer (device.py:1089-1097 dispatch of one config-0 layer) ---- */
/* U(2) on every qubit with active[q] != 0 (mats as in mq_apply_u2_layer;
 * mats == NULL: none), then the diagonal terms (as in mq_apply_diag_terms;
 * n_terms may be 0), then the GF(2) permutation of mq_apply_xor_affine
 * (rows == NULL: none).  The result equals the three calls in that order;
 * the diagonal and a permutation that keeps the low index bits among
 * themselves (CNOT ladders) ride on the last U(2) sweep instead of taking
 * sweeps of their own. */
int mq_apply_layer(mq_state* h, const double* mats, const uint8_t* active,
                   int n_terms, const int32_t* kinds, const int32_t* wires,
                   const double* params, const uint64_t* rows, uint64_t c);

/* ---- (c) QFT (shaders/qft.py:144-236, sim.py:522-563) -------------------- */
/* Ordered wire list, first wire = most significant logical bit, no final
 * swaps; inverse != 0 applies iqft.  The first complex64 QFT sweep on a
 * device uploads the library's twiddle table and waits for that copy (once
 * per device and process): make it before any stream capture. */
int mq_apply_qft(mq_state* h, const int32_t* wires, int k, int inverse);
/* Stages [j_begin, j_end) of the QFT on qubits [q0, q0+k): the fused stage
 * passes of qft_stage_sub (qft.py:144-181); j_begin=0, j_end=k is the full
 * transform. */
int mq_apply_qft_stages(mq_state* h, int q0, int k, int j_begin, int j_end, int inverse);

/* ---- (d) GF(2) affine permutation (shaders/xor_affine.py:79-116) -------- */
/* out[y] = in[src(y)], src qubit-k bit = parity(rows[k] & y) ^ bit_k(c);
 * rows are the inverse-map rows of compose_inverse_affine (xor_affine.py:46-76). */
int mq_apply_xor_affine(mq_state* h, const uint64_t* rows, uint64_t c);

/* ---- (e) probabilities and sampling (sim.py:322-430) --------------------- */
/* wires == NULL or k < 0: full register in natural order.  out_dtype 0 =
 * float32, 1 = float64; out has 2^k (or 2^n) entries, first wire = MSB. */
int mq_probabilities(mq_state* h, const int32_t* wires, int k, int out_dtype, void* out);
/* The full probability vector (natural order, 2^n entries of out_dtype) into
 * DEVICE memory of the handle's device, asynchronously on its stream: a
 * caller that keeps results on the GPU (batched or pipelined circuits) reads
 * nothing back.  Same values as mq_probabilities with wires == NULL. */
int mq_probabilities_device(mq_state* h, int out_dtype, void* out_dev);
/* Seeded inverse-CDF sampling over the marginal of wires (NULL/k<0 = all):
 * out[s] = outcome index (first wire = MSB) for s in [0, shots).  Philox4x32-10
 * stream keyed by seed, counter = s + stream_offset. */
int mq_sample(mq_state* h, const int32_t* wires, int k, uint64_t seed,
              uint64_t stream_offset, int64_t shots, int64_t* out);
/* <psi|P_w|psi> for Pauli words P_w given as masks over state-index bits:
 * xmask (X or Y), zmask (Z or Y), ny = number of Y factors.  out[2w] = re,
 * out[2w+1] = im (integrations/_common.py:384-427). */
int mq_expval_pauli(mq_state* h, int n_words, const uint64_t* xmask,
                    const uint64_t* zmask, const int32_t* ny, double* out);
/* ---- differentiation: adjoint method ------------------------------------ */
/* The reference differentiates by parameter shift, two circuit runs per
 * parameter (integrations/qml.py:308-332); these two calls give the adjoint
 * method.  Both handles: same n, dtype, device and stream.
 * out = H psi for H = sum_w zcoef[w] Z(zmasks[w]) + sum_q xcoef[q] X_q
 * (zmasks over index bits; xcoef NULL = no X part); energy (nullable) =
 * Re <psi|H|psi>. */
int mq_apply_pauli_sum(mq_state* psi, mq_state* out, int n_z, const uint64_t* zmasks,
                       const double* zcoef, const double* xcoef, double* energy);
/* One backward layer: for each listed qubit q_i, out[3i+0..2] = Im <lam|P|psi>
 * for P = X, Y, Z on q_i, then psi, lam <- mats[8i ..] (2x2 complex128
 * [u00,u01,u10,u11]) on q_i.  The 2x2s must commute (different qubits).
 * For a qubit whose last forward gate was U = R_{K-1} ... R_0 with
 * R_k = exp(-i t_k G_k / 2), pass U^dag: then dE/dt_k = a X + b Y + c Z
 * read off out, with V G_k V^dag = aX + bY + cZ, V = R_{K-1} ... R_{k+1}.
 * out == NULL: un-apply only. */
int mq_adjoint_layer(mq_state* psi, mq_state* lam, int n_q, const int32_t* qubits,
                     const double* mats, double* out);
/* mq_adjoint_layer with out in DEVICE memory (3*n_q doubles), written on the
 * stream without waiting for the GPU: a backward run of many layers reads
 * its gradients back once. */
int mq_adjoint_layer_async(mq_state* psi, mq_state* lam, int n_q, const int32_t* qubits,
                           const double* mats, double* out_dev);
/* A GF(2) map (rows, c as mq_apply_xor_affine) applied to psi and lam, then
 * mq_adjoint_layer_async: one backward layer of a circuit whose forward layer
 * ended with the map's inverse (the CNOT ladder of the layered ansatz; the
 * reference un-applies it as xor_affine_gather, shaders/xor_affine.py:79-116).
 * When the map keeps the low tile of the layer's first sweep, that sweep
 * gathers its input tiles through the map instead of a separate pass over
 * both states; the results are the same bits either way.  n_q == 0 applies
 * the map only. */
int mq_adjoint_layer_xor_async(mq_state* psi, mq_state* lam, const uint64_t* rows, uint64_t c, int n_q,
                               const int32_t* qubits, const double* mats, double* out_dev);

/* ---- batched circuits (integrations/qiskit.py:505-514 runs them one by one) */
/* A batch of layered circuits: circuit c has n_qubits[c] qubits (1..30) and
 * depth[c] layers, each a 2x2 on every qubit followed (ladder[c] != 0, or
 * ladder == NULL) by CNOT(0,1), ..., CNOT(n-2,n-1).  Circuits of <= 13 qubits
 * run whole in shared memory (small_threads: 128, 256 or 512 threads per
 * block); larger ones run tile sweeps on `lanes` parallel streams.  The
 * first run captures everything as one CUDA graph; later runs with the same
 * output pointers replay it. */
typedef struct mq_batch mq_batch;
int mq_batch_create(int device, void* stream, int n_circuits, const int32_t* n_qubits,
                    const int32_t* depth, const uint8_t* ladder, int lanes, int small_threads,
                    mq_batch** out);
/* mats_count = total doubles of mq_batch_run's mats; probs_count = sum of 2^n. */
int mq_batch_info(const mq_batch* b, uint64_t* mats_count, uint64_t* probs_count,
                  int* n_small, int* n_large);
/* mats (host): for every circuit in order, depth x n x 8 doubles (layer,
 * qubit, [u00,u01,u10,u11] re/im).  probs_dev (device, float32): every
 * circuit's full probability vector in order (first qubit = MSB); z0_dev
 * (device, float64): <Z_0> per circuit.  Asynchronous on the batch stream. */
int mq_batch_run(mq_batch* b, const double* mats, float* probs_dev, double* z0_dev);
/* The tile shape of the large circuits' sweeps (an autotuner's choice):
 * largest tile in bits (0 = default, else 6..12), low passenger bits of a
 * high sweep (-1 = default, else 0..5, fewer than tile_max), smallest tile
 * (0 = default).  Only before the first mq_batch_run. */
int mq_batch_set_tiles(mq_batch* b, int tile_max, int passengers, int tile_min);
int mq_batch_sync(mq_batch* b);
int mq_batch_destroy(mq_batch* b);

/* mq_expval_pauli without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc or cudaFree
 * in the middle of their work -- a serving loop that admits requests by
 * state footprint alone and must not let a measurement grow device memory,
 * a host whose own pool already owns the free HBM, or one that cannot let
 * cudaFree's device-wide wait stall its other streams.
 * Same arguments and the same result bits as mq_expval_pauli.  Its scratch
 * is a fixed 131,200-byte device array inside the library, held by every
 * GPU that loads it until the process exits; it holds the partial sums of
 * up to 1024 blocks, enough for GPUs of up to 256 SMs, and larger GPUs get
 * MQ_EUNSUPPORTED.  The first call on each device looks up the array's
 * device address; make that first call before any stream capture.  The
 * address is kept for the life of the process: after a cudaDeviceReset of a
 * device it is stale, so do not call this entry point on that device
 * again.  All
 * calls on one device share the array: calls that overlap on the GPU (other
 * handles, other streams) race and must be serialised by the caller.  Each
 * call writes every scratch slot it reads, so nothing needs clearing
 * between calls. */
int mq_expval_pauli_static(mq_state* h, int n_words, const uint64_t* xmask,
                           const uint64_t* zmask, const int32_t* ny, double* out);

#ifdef __cplusplus
}
#endif
#endif /* MQ_H */
