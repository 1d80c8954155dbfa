/*
 * snuqs_b200 -- C ABI of the B200 state-vector engine.
 *
 * Drop-in for SnuQS's per-gate state-update path:
 *   functionals::apply   src/braket/snuqs/csrc/functionals/functionals.cc:15-28
 *   cu::applyGate        src/braket/snuqs/csrc/operation/gate_operations_impl_cuda.cu:159-175
 *   initialize_zero / initialize_basis_z   functionals.cc:30-50
 *   StateVector(DeviceType::CUDA, n) / .cpu() / .copy()
 *                        src/braket/snuqs/csrc/result_types/state_vector.cc:21-56
 *   core.cuda.*          src/braket/snuqs/csrc/core/cuda/runtime.cu:4-25
 *
 * Conventions (the reference's):
 *   - a state is 2^n amplitudes, interleaved re/im, complex128 (SQ_C128) or
 *     complex64 (SQ_C64);
 *   - qubit q is index bit n-1-q (big-endian, Braket order);
 *   - a k-qubit matrix is row-major 2^k x 2^k complex128 (interleaved
 *     re/im doubles, whatever the state's precision) and qubits[0] is the
 *     most significant bit of its row/column index.
 *
 * Every entry point returns an sq_status; a nonzero status leaves a message
 * for sq_last_error() (thread-local).  No entry point exits the process.
 * Streams are cudaStream_t passed as void* (NULL = the legacy default stream).
 * Gate application is queued per state and executed, fused, at the next
 * flush; sq_flush, the copies, the reductions and sq_init_* flush first.
 */
#ifndef SNUQS_B200_H
#define SNUQS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sq_state sq_state;

typedef enum {
  SQ_OK = 0,
  SQ_ERR_INVALID = 1,     /* bad argument: qubit out of range, repeated qubit, null pointer */
  SQ_ERR_CUDA = 2,        /* a CUDA runtime call failed (message has the CUDA error) */
  SQ_ERR_OOM = 3,         /* device or pinned-host allocation failed */
  SQ_ERR_UNSUPPORTED = 4, /* a size or option this build does not handle */
  SQ_ERR_TIMEOUT = 5      /* a bounded device-side wait gave up */
} sq_status;

typedef enum { SQ_C128 = 0, SQ_C64 = 1 } sq_dtype;

/* Gate ids: GateOperationType order of
 * src/braket/snuqs/csrc/operation/operation.h:17-52, then the Braket gates the
 * reference lists as removed (src/braket/snuqs/gate_operations.py:238). */
typedef enum {
  SQ_GATE_IDENTITY = 0, SQ_GATE_HADAMARD, SQ_GATE_PAULI_X, SQ_GATE_PAULI_Y,
  SQ_GATE_PAULI_Z, SQ_GATE_CX, SQ_GATE_CY, SQ_GATE_CZ, SQ_GATE_S, SQ_GATE_SI,
  SQ_GATE_T, SQ_GATE_TI, SQ_GATE_V, SQ_GATE_VI, SQ_GATE_PHASE_SHIFT,
  SQ_GATE_CPHASE_SHIFT, SQ_GATE_CPHASE_SHIFT00, SQ_GATE_CPHASE_SHIFT01,
  SQ_GATE_CPHASE_SHIFT10, SQ_GATE_ROT_X, SQ_GATE_ROT_Y, SQ_GATE_ROT_Z,
  SQ_GATE_SWAP, SQ_GATE_ISWAP, SQ_GATE_PSWAP, SQ_GATE_XY, SQ_GATE_XX,
  SQ_GATE_YY, SQ_GATE_ZZ, SQ_GATE_CCNOT, SQ_GATE_CSWAP, SQ_GATE_U,
  SQ_GATE_GPHASE, SQ_GATE_SWAP_A2A, SQ_GATE_ECR, SQ_GATE_CV, SQ_GATE_PRX,
  SQ_GATE_COUNT
} sq_gate;

typedef enum {
  SQ_OPT_FUSION = 0,    /* 1 (default): fused tile sweeps; 0: one unfused kernel per gate */
  SQ_OPT_TILE_BITS = 1, /* log2 amplitudes per shared-memory tile (4..12; default 11 for
                           complex128, 12 for complex64: 32 KiB either way) */
  SQ_OPT_REORDER = 2,   /* 1 (default): the planner may absorb later gates that commute */
  SQ_OPT_TIMING = 3,    /* 1: record a CUDA event pair around every fused-sweep launch */
  SQ_OPT_JIT = 4,       /* -1 (default): JIT-specialised sweep kernels for states of >= 20
                           qubits when NVRTC is present; 1: always; 0: never */
  SQ_OPT_LOW_BITS = 5,  /* contiguous low index bits in every tile (each global access
                           covers runs of 2^value amplitudes); 0 (default): 3 for
                           complex128, 4 for complex64 (128-byte runs) when the state
                           spans several tiles; ignored unless value + 4 <= tile bits */
  SQ_OPT_REMAP = 6      /* 1: JIT-specialised sweeps may store their tiles with index bits
                           permuted so that the next sweeps find their most used qubits
                           on the low bits every tile holds; every flush ends in the
                           original order.  0 (default; SQ_REMAP=1 changes it): never */
} sq_option;

/* ---- library / device ------------------------------------------------ */
const char *sq_version(void);
const char *sq_last_error(void);
/* core.cuda.device_count / get_device / set_device / device_synchronize /
 * mem_info: src/braket/snuqs/csrc/core/cuda/runtime.cu:4-25 */
int sq_device_count(int *count);
int sq_get_device(int *device);
int sq_set_device(int device);
int sq_device_synchronize(void);
int sq_mem_info(size_t *free_bytes, size_t *total_bytes);

/* Stream / Event / pinned host memory, so callers need no CUDA headers:
 * Stream (src/braket/snuqs/csrc/stream/stream.cc:6-34), Event
 * (src/braket/snuqs/csrc/event/event.cc:5-26), BufferPinned host memory. */
int sq_stream_create(void **stream, int nonblocking);
int sq_stream_destroy(void *stream);
int sq_stream_synchronize(void *stream);
int sq_stream_wait_event(void *stream, void *event);
int sq_event_create(void **event);
int sq_event_destroy(void *event);
int sq_event_record(void *event, void *stream);
int sq_event_synchronize(void *event);
/* Milliseconds between two recorded events. */
int sq_event_elapsed(void *start, void *stop, float *ms);
int sq_host_alloc(void **ptr, size_t bytes);
int sq_host_free(void *ptr);

/* ---- gate matrices ------------------------------------------------------
 * Matrix of a named gate (the reference constructors,
 * src/braket/snuqs/csrc/operation/gate_operations.cc:9-734; ECR/CV/PRx from
 * their Braket definitions).  out receives 4^k complex128 (interleaved);
 * *k receives the gate's qubit count. */
int sq_gate_matrix(int gate, const double *angles, uint32_t nangles,
                   double *out, uint32_t *k);
int sq_gate_qubits(int gate);
/* Analytic derivative d/d angles[param] of the named gate's matrix (same
 * layout as sq_gate_matrix).  No counterpart in the reference (it has no
 * gradients); used by the adjoint gradient. */
int sq_gate_matrix_derivative(int gate, const double *angles, uint32_t nangles,
                              uint32_t param, double *out, uint32_t *k);

/* ---- state handle -------------------------------------------------------
 * StateVector(DeviceType::CUDA, n): state_vector.cc:21-25 + buffer_cuda.cc:13-17. */
/* SQ_ERR_OOM when the device cannot hold the state; the library stays usable. */
int sq_state_create(uint32_t num_qubits, int dtype, sq_state **out);
/* Wraps caller-owned device memory of 2^n amplitudes (not freed by destroy). */
int sq_state_wrap(void *device_ptr, uint32_t num_qubits, int dtype,
                  sq_state **out);
int sq_state_destroy(sq_state *s);
void *sq_state_data(const sq_state *s);
uint32_t sq_state_num_qubits(const sq_state *s);
int sq_state_dtype(const sq_state *s);
int sq_set_option(sq_state *s, int option, int64_t value);

/* initialize_zero / initialize_basis_z (functionals.cc:30-50); init_basis
 * writes |index>, so index 0 is the reference's |0...0>. Pending gates are
 * discarded. */
int sq_init_zero(sq_state *s, void *stream);
int sq_init_basis(sq_state *s, uint64_t index, void *stream);

/* functionals::apply (functionals.cc:15-28): queue one k-qubit gate given by
 * its matrix (k = 0 is a global phase: a 1x1 matrix).  k <= 10. */
int sq_apply_matrix(sq_state *s, const double *matrix, const uint32_t *qubits,
                    uint32_t k, void *stream);
/* As sq_apply_matrix with extra control qubits: the matrix acts on `qubits`
 * when every control qubit c[i] has value cv[i] (cv NULL = all ones).  This
 * is the ctrl/negctrl modifier the reference stores but never applies
 * (src/braket/snuqs/openqasm/program_context.py:744-780). */
int sq_apply_controlled_matrix(sq_state *s, const double *matrix,
                               const uint32_t *qubits, uint32_t k,
                               const uint32_t *controls,
                               const uint8_t *control_values, uint32_t nc,
                               void *stream);
/* Queue a named gate (sq_gate id) with its angles. */
int sq_apply_gate(sq_state *s, int gate, const uint32_t *qubits, uint32_t k,
                  const double *angles, uint32_t nangles, void *stream);
/* Execute every queued gate on `stream` (fused sweeps). */
int sq_flush(sq_state *s, void *stream);
int sq_pending(const sq_state *s, uint32_t *count);
/* Kernels launched by all flushes of this state so far. */
int sq_launch_count(const sq_state *s, uint64_t *count);
/* With SQ_OPT_TIMING on: total device time (ms) and number of the fused-sweep
 * launches recorded since the last call (synchronises on the recorded
 * events, then clears them).  The reverse two-state sweeps of
 * sq_adjoint_gradient are recorded on its psi state. */
int sq_sweep_timing(sq_state *s, double *total_ms, uint64_t *launches);
/* JIT-specialised sweeps, process-wide: whether NVRTC could be loaded, and
 * how many sweeps ran a JIT kernel / fell back to the generic kernel. */
int sq_jit_info(int *available, uint64_t *jit_launches, uint64_t *fallbacks);
/* Test hook: compile `source` with NVRTC for sm_100a (no GPU needed).
 * SQ_OK, or SQ_ERR_INVALID with the compiler log in sq_last_error(). */
int sq_jit_compile(const char *source);

/* cu::applyGate (gate_operations_impl_cuda.cu:159-175), unqueued: apply
 * one gate to a raw complex128 device buffer of nelems = 2^nqubits
 * amplitudes, with a device-resident row-major matrix, on `stream`.
 * targets are size_t-sized qubit indices as in the reference. */
int sq_apply_gate_buffer(void *buffer, const void *gate_device,
                         const uint64_t *targets, uint32_t ntargets,
                         uint32_t nqubits, uint64_t nelems, void *stream);

/* ---- copies (StateVector.cpu()/.cuda()/.copy(): state_vector.cc:35-56) --
 * Asynchronous on `stream`; synchronise the stream before reading dst. */
int sq_copy_to_host(sq_state *s, void *dst, void *stream);
int sq_copy_from_host(sq_state *s, const void *src, void *stream);
int sq_copy_state(sq_state *dst, sq_state *src, void *stream);
/* Synchronises `stream` and reports a sweep kernel that gave up one of its
 * bounded waits on this state since the last check (SQ_ERR_TIMEOUT; the
 * state's contents are then invalid).  No counterpart in the reference,
 * whose CUDA errors exit the process (utils_cuda.h:8-16). */
int sq_state_check(sq_state *s, void *stream);

/* ---- results ----------------------------------------------------------- */
/* |psi_i|^2 into a caller-provided DEVICE array of 2^n doubles
 * (simulation.py:208-215 computes this on the host). */
int sq_probabilities(sq_state *s, double *out_device, void *stream);
/* sum_t w_t <psi|P_t|psi> for n_terms Pauli strings, paulis[t*n + q] in
 * {'I','X','Y','Z'} acting on qubit q (observables.py:136-243 semantics).
 * Synchronous: returns the FP64 value in *out. */
int sq_expect_pauli(sq_state *s, const char *paulis, const double *weights,
                    uint32_t n_terms, double *out, void *stream);
/* Squared norm in FP64 (synchronous). */
int sq_norm2(sq_state *s, double *out, void *stream);
/* Variance <H^2> - <H>^2 of H = sum_t w_t P_t (paulis as in sq_expect_pauli;
 * n_terms <= 1024), FP64, synchronous.  H^2 is expanded into Pauli strings on
 * the host (anticommuting pairs cancel) and both moments run on the device.
 * Replaces the Variance result type the reference plugin does not register
 * (src/braket/snuqs/result_types.py:149-151, simulator.py:578-580). */
int sq_variance_pauli(sq_state *s, const char *paulis, const double *weights,
                      uint32_t n_terms, double *out, void *stream);
/* Measurement shots on the device, replacing the host-side
 * np.random.choice over |psi|^2 after a full state copy
 * (src/braket/snuqs/simulation.py:208-220).  uniforms_device: `shots`
 * doubles in [0, 1) (DEVICE memory); out_device: `shots` basis-state indices
 * (DEVICE memory, uint64; bit n-1-q of an index is qubit q).  Index of shot
 * s = the inverse CDF of |psi_i|^2 at uniforms[s] * sum|psi|^2, with the
 * probabilities summed in one fixed binary tree (adjacent pairs first), so
 * the result is reproducible bit for bit.  Asynchronous on `stream`;
 * shots <= 2^31 per call; num_qubits <= 34. */
int sq_sample(sq_state *s, const double *uniforms_device, uint64_t shots,
              uint64_t *out_device, void *stream);
/* sq_sample with HOST buffers (staged through the state's device scratch
 * and a pinned host buffer of 8 x shots bytes that the state keeps until it
 * is destroyed): the uniforms go to the device while the probability tree is
 * built, only the shot indices come back.  Synchronous. */
int sq_sample_host(sq_state *s, const double *uniforms, uint64_t shots,
                   uint64_t *out, void *stream);
/* Amplitudes psi[indices[i]] as complex128 (interleaved doubles) into
 * out_device; indices_device and out_device are DEVICE arrays of `count`
 * entries.  Synchronous; SQ_ERR_INVALID if an index is >= 2^n.  The Braket
 * Amplitude result type (not registered by the reference plugin). */
int sq_amplitudes(sq_state *s, const uint64_t *indices_device, uint64_t count,
                  double *out_device, void *stream);
/* Marginal probabilities of the k target qubits into a DEVICE array of 2^k
 * doubles; qubits[0] is the most significant bit of the output index (the
 * Braket Probability result type with targets).  k <= 30. */
int sq_marginal_probabilities(sq_state *s, const uint32_t *qubits, uint32_t k,
                              double *out_device, void *stream);
/* Precision report of one state against another of the same size (either
 * precision, e.g. a complex64 result against the complex128 one): max_i
 * |a_i - b_i| and 1 - |<a|b>|^2 / (<a|a><b|b>), accumulated in FP64.
 * Synchronous.  No counterpart in the reference (complex128 only). */
int sq_state_distance(sq_state *a, sq_state *b, double *max_abs,
                      double *one_minus_fidelity, void *stream);

/* ---- adjoint gradient ---------------------------------------------------
 * No counterpart in the reference (its plugin forbids the adjoint-gradient
 * result type: src/braket/snuqs/simulator.py:649).
 *
 * One gate of a parametrised circuit.  gate is an sq_gate id, or -1 for a
 * fixed matrix (`matrix`, 4^k complex128).  Angle j of the gate takes the
 * value angles[j]; when param[j] >= 0 it depends on parameter param[j] with
 * d angles[j] / d theta[param[j]] = scale[j] (1 for the angle itself). */
typedef struct {
  int32_t gate;
  uint32_t k;
  uint32_t qubits[3];
  uint32_t nangles;
  double angles[3];
  int32_t param[3];
  double scale[3];
  const double *matrix;
} sq_circuit_op;

/* Test hook: CUDA source of the JIT kernel of fused sweep `sweep_index` of
 * the default plan of a circuit (params ignored).  Writes at most cap bytes (NUL-terminated), the full length to
 * *len and the number of fused sweeps to *nsweeps.  Needs no GPU. */
int sq_jit_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                  uint32_t sweep_index, char *buf, uint64_t cap, uint64_t *len,
                  uint32_t *nsweeps);
/* Test hook: as sq_jit_source, for reverse sweep `sweep_index` of the
 * circuit's adjoint-gradient plan (two-state JIT kernel; *len = 0 when that
 * sweep runs on the generic adjoint kernel).  Needs no GPU. */
int sq_jit_adjoint_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                          uint32_t sweep_index, char *buf, uint64_t cap, uint64_t *len,
                          uint32_t *nsweeps);

/* Energy E = <psi|H|psi> of psi = U(theta)|0...0> for H = sum_t w_t P_t, and
 * dE/dtheta for n_params parameters, by one forward pass and one reverse
 * (adjoint) pass: the reverse pass un-computes the gates on psi and on
 * lambda = H psi together in fused two-state sweeps and accumulates
 * 2 Re <lambda| dU U^dagger |psi> per parametrised angle; no intermediate
 * state is stored.  `psi` and `lam` are two caller-owned work states of the
 * same size and precision (their contents are overwritten).  energy and grad
 * (n_params doubles) are host pointers; the call is synchronous. */
int sq_adjoint_gradient(sq_state *psi, sq_state *lam, const sq_circuit_op *ops,
                        uint32_t nops, const char *paulis, const double *weights,
                        uint32_t n_terms, uint32_t n_params, double *energy,
                        double *grad, void *stream);

/* No counterpart in the reference.  sq_expect_pauli for callers that cannot
 * allocate device memory: code recording a CUDA graph (a cudaMalloc would
 * break the capture), applications whose memory pool owns the whole device,
 * callers holding only a raw device pointer to a state.  `state` is a device
 * array of 2^num_qubits amplitudes of `dtype`; the FP64 result is written
 * to out_device (one double in device memory), asynchronously on `stream`.
 * Nothing is allocated: the reduction's partial sums live in one fixed
 * 16 KiB device array (2048 doubles) inside the library, which each device
 * holds from the moment the library's device code is loaded on it until the
 * process exits.  The first call on each device looks that array up (make
 * it once, before any stream capture); the look-up is repeated only when the
 * device's CUDA context has changed (after cudaDeviceReset).  Every call on a
 * device shares the array, so calls that overlap on the GPU (different
 * streams, no ordering) race; order them.  Limits: n_terms <= 1024 and at
 * most 256 distinct (X/Y mask, Y parity) groups; larger requests return
 * SQ_ERR_UNSUPPORTED.  A call stages the grouped terms on the calling
 * thread's stack (about 45 KiB). */
int sq_expect_pauli_noalloc(const void *state, uint32_t num_qubits, int dtype,
                            const char *paulis, const double *weights,
                            uint32_t n_terms, double *out_device, void *stream);

/* ---- batched circuits ----------------------------------------------------
 * No counterpart in the reference (one circuit per run: simulator.py:152-155).
 * Many small circuits (4..30 qubits each, uneven) and their Pauli-sum
 * energies in ONE persistent kernel launch: CTAs take circuits from an
 * atomic work queue, largest first; a circuit that fits one shared-memory
 * tile (<= 11 qubits complex128, <= 12 complex64) never touches HBM. */
typedef struct sq_batch sq_batch;
typedef enum {
  SQ_BOPT_KEEP_STATES = 0, /* 1: keep every final state for sq_batch_state */
  SQ_BOPT_TILE_BITS = 1,   /* log2 amplitudes per shared-memory tile (10..12; 0 = 11 for
                              complex128, 12 for complex64): the fusion block and, for
                              circuits of at most that many qubits, the resident state */
  SQ_BOPT_LOW_BITS = 2,    /* contiguous low bits of a streamed tile (0 = planner default) */
  SQ_BOPT_MAX_OPS = 3,     /* most gates one fused sweep carries (0 = 64) */
  SQ_BOPT_CTAS_PER_SM = 4  /* persistent CTAs per SM (0 = the occupancy limit) */
} sq_batch_option;
int sq_batch_create(int dtype, sq_batch **out);
int sq_batch_destroy(sq_batch *b);
int sq_batch_set_option(sq_batch *b, int option, int64_t value);
/* Pauli-sum observable on num_qubits qubits (paulis as in sq_expect_pauli). */
int sq_batch_add_hamiltonian(sq_batch *b, uint32_t num_qubits, const char *paulis,
                             const double *weights, uint32_t n_terms, uint32_t *ham_id);
/* One circuit (gates as sq_circuit_op; param/scale are ignored) measured with
 * Hamiltonian ham_id (same qubit count). */
int sq_batch_add_circuit(sq_batch *b, uint32_t num_qubits, const sq_circuit_op *ops,
                         uint32_t nops, uint32_t ham_id, uint32_t *circuit_id);
/* Replace the angles of circuit `circuit` (same gates; nangles per op as
 * given at add time, concatenated). */
int sq_batch_set_angles(sq_batch *b, uint32_t circuit, const double *angles, uint32_t count);
int sq_batch_num_circuits(const sq_batch *b, uint32_t *count);
/* Plan, upload and run every circuit in one launch; energies (host,
 * one double per circuit, in circuit-id order).  Synchronous. */
int sq_batch_run(sq_batch *b, double *energies, void *stream);
/* Launch configuration of the energy kernel, as the autotuner reports it. */
typedef struct {
  uint32_t tile_bits, low_bits, max_ops, ctas_per_sm;
  double kernel_ms; /* best kernel time measured for it */
} sq_batch_config;
/* Autotuner (no counterpart in the reference): runs the batch's energy
 * kernel for every tile size (10..12 bits), low-bit count (default / 3),
 * fusion width (32 / 64 gates per sweep) and CTAs per SM (1 .. occupancy
 * limit, at most 4), `reps` times each, times each run with CUDA events,
 * keeps the fastest configuration on the batch (later sq_batch_run calls use
 * it) and reports it in *best.  Synchronous; runs the circuits many times. */
int sq_batch_autotune(sq_batch *b, uint32_t reps, sq_batch_config *best, void *stream);
/* Energies and adjoint gradients of every circuit in one persistent launch
 * (no counterpart in the reference): per circuit a forward pass, lambda = H psi
 * and a reverse two-state pass, with the circuit's psi and lambda in shared
 * memory when it fits one tile and in a device pool otherwise.  Circuits
 * declare their parametrised angles with sq_circuit_op.param/scale as for
 * sq_adjoint_gradient; grads is a host array of ncircuits x n_params doubles
 * (row = circuit id), energies one double per circuit.  Synchronous. */
int sq_batch_run_gradients(sq_batch *b, uint32_t n_params, double *energies, double *grads,
                           void *stream);
/* Test hook: CUDA source of the JIT batched-gradient kernel that
 * sq_batch_run_gradients uses when every circuit of a batch shares this
 * circuit's plan structure (num_qubits above the batch tile bits); *len = 0
 * when the plan is not covered.  Needs no GPU. */
int sq_jit_batch_adjoint_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                                char *buf, uint64_t cap, uint64_t *len);
/* Final state of a circuit (needs SQ_BOPT_KEEP_STATES before sq_batch_run);
 * host_dst receives 2^n amplitudes of the batch's precision. */
int sq_batch_state(sq_batch *b, uint32_t circuit, void *host_dst, void *stream);
/* Device time of the last sq_batch_run's kernel (ms) and its CTA count. */
int sq_batch_last_timing(const sq_batch *b, double *kernel_ms, uint32_t *ctas);
/* Plan statistics of the last sq_batch_run: circuits streamed through HBM
 * (more qubits than the tile), their fused sweeps, and their algorithmic HBM
 * bytes (per streamed circuit (2 x sweeps + 1) x 2^n x amplitude bytes: every
 * sweep reads and writes the state, the energy pass reads it once; one pass
 * less for a circuit of a structure group whose first sweep starts from
 * |0...0> without reading). */
int sq_batch_stats(const sq_batch *b, uint64_t *streamed, uint64_t *sweeps, uint64_t *hbm_bytes);
/* Structure groups of the last sq_batch_run: streamed circuits whose plans
 * differ only in their angles (the same circuit with other parameters) run
 * as one multi-state JIT launch per sweep over all of their states instead of
 * one CTA per circuit (needs NVRTC; SQ_BATCH_MULTI=0 turns it off).  Writes
 * the number of groups and of the circuits they hold. */
int sq_batch_groups(const sq_batch *b, uint32_t *groups, uint32_t *circuits);
/* Test hook: CUDA source of the multi-state JIT kernel (sq_jit_msweep) of
 * sweep `sweep_index` of a circuit as a batch energy run plans it with the
 * default tile size (num_qubits above it); from_zero = 1: the form that
 * starts every state from |0...0> instead of reading it (*len = 0 when the
 * sweep has none).  Writes at most cap bytes (NUL-terminated), the full
 * length to *len and the number of sweeps to *nsweeps.  Needs no GPU. */
int sq_jit_multi_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                        uint32_t sweep_index, int from_zero, char *buf, uint64_t cap, uint64_t *len,
                        uint32_t *nsweeps);

#ifdef __cplusplus
}
#endif
#endif /* SNUQS_B200_H */
