/*
 * tmfqs_b200 -- C ABI of the B200 dense state-vector engine for TMFQS.
 *
 * One handle = one register's state vector resident in HBM plus the CUDA
 * stream its kernels run on.  The C++ `gpu` storage strategy
 * (GpuStateBackend, an IStateBackend) binds to these entry points; so do the
 * Python tests and the benchmark.  Plain pointers and sizes only; host
 * buffers are caller-owned; every call returns a tmfqs_status and leaves a
 * message for tmfqs_gpu_last_error() on failure.
 *
 * Layout in HBM: 2^n interleaved complex amplitudes [re0, im0, re1, im1, ...]
 * -- complex128 (TMFQS_FP64, the reference's AmplitudesVector layout,
 * include/tmfqs/core/types.h:28) or complex64 (TMFQS_FP32).  Qubit q is bit
 * (n-1-q) of the state index (qubit 0 = most significant, types.h:12-13).
 *
 * Semantics follow the reference Dense backend operation by operation.  In
 * TMFQS_FP64 every gate, diffusion, affine map, total probability and
 * measurement is bit-identical to the reference (same IEEE operations in the
 * same order; sequential sums replayed exactly).  Reference citations below
 * are paths inside the reference project.
 */
#ifndef TMFQS_B200_H
#define TMFQS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TMFQS_API __attribute__((visibility("default")))
#else
#define TMFQS_API
#endif

typedef struct tmfqs_gpu_state tmfqs_gpu_state;

/* Status codes; each maps to the exception class the reference throws. */
typedef enum {
	TMFQS_OK = 0,
	TMFQS_ERR_OUT_OF_RANGE = 1,    /* std::out_of_range   (validation.h:19-41) */
	TMFQS_ERR_INVALID_ARGUMENT = 2, /* std::invalid_argument (validation.h:43-80) */
	TMFQS_ERR_LOGIC = 3,           /* std::logic_error (backend_validation.h:13-18) */
	TMFQS_ERR_RUNTIME = 4,         /* std::runtime_error (dense_state_backend.cpp:186) */
	TMFQS_ERR_CUDA = 5,            /* CUDA failure (mapped to std::runtime_error) */
	TMFQS_ERR_NOMEM = 6            /* device allocation failure (std::runtime_error) */
} tmfqs_status;

typedef enum {
	TMFQS_FP64 = 0, /* complex128 amplitudes, FP64 arithmetic (plain form) */
	TMFQS_FP32 = 1  /* complex64 amplitudes, FP32 gates, FP64 reductions (precision form) */
} tmfqs_precision;

/* Circuit operation: the circuit::Operation variant (circuit/circuit.h:16-61). */
typedef enum {
	TMFQS_OP_H = 0,          /* Hadamard{target}                 */
	TMFQS_OP_X = 1,          /* PauliX{target}                   */
	TMFQS_OP_CNOT = 2,       /* ControlledNot{control, target}   */
	TMFQS_OP_CPHASE = 3,     /* ControlledPhaseShift{c, t, theta} */
	TMFQS_OP_SWAP = 4,       /* Swap{first, second}              */
	TMFQS_OP_GATE = 5,       /* MatrixGate{gate, targets}        */
	TMFQS_OP_PHASE_FLIP = 6, /* PhaseFlipBasisState{state}       */
	TMFQS_OP_INVERSION = 7   /* InversionAboutMean{materialized} */
} tmfqs_op_kind;

typedef struct {
	int kind;               /* tmfqs_op_kind */
	unsigned q0;            /* target (H, X); control (CNOT, CPHASE); first (SWAP) */
	unsigned q1;            /* target (CNOT, CPHASE); second (SWAP) */
	double theta;           /* CPHASE angle in radians */
	uint64_t state;         /* PHASE_FLIP basis state */
	int materialized;       /* INVERSION: 1 materialised, 0 lazy overlay */
	const double *matrix;   /* GATE: row-major 2^k x 2^k interleaved complex (host) */
	const unsigned *qubits; /* GATE: targets, first = most significant block bit */
	unsigned k;             /* GATE: number of targets */
} tmfqs_op;

/* The register-side state that QuantumRegister keeps around its backend:
 * cached logical amplitude sum and lazy affine overlay
 * (register/quantum_register.h:218-224). */
typedef struct {
	int has_sum;
	double sum_re, sum_im;
	int overlay;
	double scale_re, scale_im;
	double bias_re, bias_im;
} tmfqs_register_view;

/* experiment::StateComparison (experiment/comparison.h:19-28), field for field. */
typedef struct {
	int bitwise_equal;
	double max_abs_amplitude_error;
	double max_abs_component_error;
	double rmse_amplitude;
	double rel_l2;
	double max_abs_probability_error;
	double total_probability_diff;
	uint64_t worst_state;
} tmfqs_state_comparison;

/* Counters of the work a handle has issued (for benchmarks and tests). */
typedef struct {
	uint64_t kernel_launches;   /* kernels launched by this handle */
	uint64_t fused_passes;      /* fused multi-gate passes over the state */
	uint64_t gate_passes;       /* single-gate passes over the state */
	uint64_t reduction_passes;  /* passes of the exact reductions */
	uint64_t h2d_bytes, d2h_bytes;
	uint64_t qft_passes;        /* fused passes that ran as the dedicated QFT pass */
} tmfqs_stats;

/* Tunables (tmfqs_gpu_set_option). */
typedef enum {
	TMFQS_OPT_FUSION = 0,        /* 1 (default): apply_ops fuses gates into multi-gate passes */
	TMFQS_OPT_FUSED_QUBITS = 1,  /* target qubits per fused pass (default: tile bits minus the
	                                contiguous low bits kept for coalescing) */
	TMFQS_OPT_GROVER_FUSION = 2, /* 1 (default): Grover runs execute as one temporal pass */
	TMFQS_OPT_KERNEL_TIMING = 3, /* 1: time every pass with CUDA events on the handle's stream */
	TMFQS_OPT_EXACT = 4,         /* FP64 handles: 1 (default) bit-identical controlled-phase chains;
	                                0: each chain as one twiddle per amplitude from FP64 tables
	                                (about 1e-15 relative error per pass).  FP32 handles always
	                                use twiddles. */
	TMFQS_OPT_RADIX = 5,         /* fast forms (FP32 handles, or EXACT=0): 1 (default) passes made only
	                                of Hadamards and controlled phases run as radix-2^k register
	                                stages; 0: the general fused pass */
	TMFQS_OPT_TENSOR = 6,        /* FP32 handles: 1 (default) dense 4- and 5-qubit gates run as
	                                3xTF32 GEMMs on the tensor cores; 0: the CUDA-core gate kernel */
	TMFQS_OPT_QFT_PASS = 7       /* fast forms with RADIX on: 1 (default) passes that are a segment of
	                                the QFT ladder run as the dedicated QFT pass (per-thread twiddle
	                                tables, swizzled stages, three tiles in flight); 0: the general
	                                radix pass */
} tmfqs_option;

/* Kernel classes for tmfqs_gpu_kernel_times. */
typedef enum {
	TMFQS_KT_FUSED = 0,   /* fused multi-gate pass */
	TMFQS_KT_PERMUTE = 1, /* bit-permutation (swap run) pass */
	TMFQS_KT_GATE = 2,    /* single-gate pass (incl. diffusion and affine sweeps) */
	TMFQS_KT_REDUCE = 3,  /* exact reduction (sum, norm, measurement) */
	TMFQS_KT_GROVER = 4,  /* temporal Grover pass */
	TMFQS_KT_ADJOINT = 5, /* adjoint-gradient passes (observable, gradient runs) */
	TMFQS_KT_COUNT = 6
} tmfqs_kernel_class;

/* Accumulated device time of one kernel class since the last reset:
 * launches, milliseconds (CUDA events), and algorithmic HBM bytes
 * (one read + one write of the state per pass; reads only for reductions). */
typedef struct {
	uint64_t launches;
	double ms;
	double bytes;
} tmfqs_kernel_time;

/* ---- lifetime --------------------------------------------------------- */
/* Creates an empty handle on `device` (no state yet). */
TMFQS_API int tmfqs_gpu_create(int precision, int device, tmfqs_gpu_state **out);
TMFQS_API int tmfqs_gpu_destroy(tmfqs_gpu_state *h);
/* Deep copy: IStateBackend::clone, storage/i_state_backend.h:31. */
TMFQS_API int tmfqs_gpu_clone(tmfqs_gpu_state *h, tmfqs_gpu_state **out);
TMFQS_API const char *tmfqs_gpu_last_error(void);
/* Test hook, no counterpart in the reference: after `skip` further device
 * allocations of the library (state, staging, reduction scratch, pass
 * programs) succeed, the next `count` fail as if cudaMalloc had run out of
 * memory -- the call then returns TMFQS_ERR_NOMEM, which the C++ binding maps
 * to std::runtime_error like the reference's other resource failures.  No
 * device memory is touched.  (0, 0) disarms it.  Process-wide. */
TMFQS_API int tmfqs_debug_fail_allocations(unsigned skip, unsigned count);

/* ---- initialisation / IO (storage/i_state_backend.h:37-66) ------------ */
/* initZero, i_state_backend.h:37; dense_state_backend.cpp:77-81. */
TMFQS_API int tmfqs_gpu_init_zero(tmfqs_gpu_state *h, unsigned num_qubits);
/* initBasis, i_state_backend.h:44; dense_state_backend.cpp:84-89. */
TMFQS_API int tmfqs_gpu_init_basis(tmfqs_gpu_state *h, unsigned num_qubits, uint64_t state, double re, double im);
/* initUniformSuperposition, i_state_backend.h:50; dense_state_backend.cpp:92-115
 * (deduplicates, amplitude 1/sqrt(unique count)). */
TMFQS_API int tmfqs_gpu_init_uniform(tmfqs_gpu_state *h, unsigned num_qubits, const uint64_t *states, size_t count);
/* loadAmplitudes, i_state_backend.h:56: 2^(n+1) doubles from host memory. */
TMFQS_API int tmfqs_gpu_load(tmfqs_gpu_state *h, unsigned num_qubits, const double *host_amps);
/* Loads `count` amplitudes starting at `first_state` into an initialised state. */
/* loadAmplitudes followed by a gate batch (tmfqs_gpu_apply_ops), for a caller
 * that holds the whole input on the host -- IStateBackend::loadAmplitudes
 * (i_state_backend.h:56) and the run of Simulator::run that follows it
 * (simulator.cpp:72-82).  Same results and errors as tmfqs_gpu_load then
 * tmfqs_gpu_apply_ops; for an exact complex128 batch that starts with a fused
 * pass the host-to-device copy goes in slabs on a second stream and the first
 * pass runs each slab's tiles as soon as it lands.  `host` must stay valid until
 * the call returns (pinned memory lets the slabs overlap the pass). */
TMFQS_API int tmfqs_gpu_load_apply_ops(tmfqs_gpu_state *h, unsigned num_qubits, const double *host, const tmfqs_op *ops,
                                       size_t count);
TMFQS_API int tmfqs_gpu_load_chunk(tmfqs_gpu_state *h, uint64_t first_state, const double *host_amps, uint64_t count);
/* exportAmplitudes, i_state_backend.h:61. */
TMFQS_API int tmfqs_gpu_export(tmfqs_gpu_state *h, double *host_out);
/* forEachAmplitudeChunk, i_state_backend.h:66: one chunk into a host buffer. */
TMFQS_API int tmfqs_gpu_export_chunk(tmfqs_gpu_state *h, uint64_t first_state, double *host_out, uint64_t count);
/* amplitude / setAmplitude, i_state_backend.h:73,79 (host-cached single reads/writes). */
TMFQS_API int tmfqs_gpu_get_amp(tmfqs_gpu_state *h, uint64_t state, double *re, double *im);
TMFQS_API int tmfqs_gpu_set_amp(tmfqs_gpu_state *h, uint64_t state, double re, double im);
TMFQS_API int tmfqs_gpu_num_qubits(tmfqs_gpu_state *h, unsigned *out);
TMFQS_API int tmfqs_gpu_precision(tmfqs_gpu_state *h, int *out);

/* ---- reductions (bit-identical to the reference's sequential loops) --- */
/* totalProbability, i_state_backend.h:90; dense_state_backend.cpp:161-171. */
TMFQS_API int tmfqs_gpu_total_probability(tmfqs_gpu_state *h, double *out);
/* sampleMeasurement, i_state_backend.h:96; dense_state_backend.cpp:173-188:
 * first state whose running probability reaches rnd; rnd in [0,1). */
TMFQS_API int tmfqs_gpu_sample(tmfqs_gpu_state *h, double rnd, uint64_t *out);
/* Sequential sum of amplitudes (real and imaginary parts), the loop in
 * QuantumRegister::logicalAmplitudeSum, quantum_register.cpp:176-190, and in
 * inversionAboutMean(), dense_state_backend.cpp:213-228. */
TMFQS_API int tmfqs_gpu_amplitude_sum(tmfqs_gpu_state *h, double *re, double *im);
/* The same three reductions over logical amplitudes scale*a+bias
 * (QuantumRegister overlay branches, quantum_register.cpp:160-165,176-211,269-310). */
TMFQS_API int tmfqs_gpu_overlay_sum(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim,
                                    double *re, double *im);
TMFQS_API int tmfqs_gpu_overlay_total_probability(tmfqs_gpu_state *h, double sre, double sim, double bre,
                                                  double bim, double *out);
TMFQS_API int tmfqs_gpu_overlay_sample(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim,
                                       double rnd, uint64_t *out);

/* ---- single operations (storage/i_state_backend.h:104-151) ------------ */
/* phaseFlipBasisState, i_state_backend.h:108; dense_state_backend.cpp:205-211. */
TMFQS_API int tmfqs_gpu_phase_flip(tmfqs_gpu_state *h, uint64_t state);
/* inversionAboutMean(), i_state_backend.h:110; dense_state_backend.cpp:213-228. */
TMFQS_API int tmfqs_gpu_inversion(tmfqs_gpu_state *h);
/* inversionAboutMean(mean), i_state_backend.h:115; dense_state_backend.cpp:230-240. */
TMFQS_API int tmfqs_gpu_inversion_mean(tmfqs_gpu_state *h, double re, double im);
/* applyAffineTransform, i_state_backend.h:121; dense_state_backend.cpp:242-253. */
TMFQS_API int tmfqs_gpu_affine(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim);
/* applyHadamard, i_state_backend.h:126; dense_state_backend.cpp:255-274. */
TMFQS_API int tmfqs_gpu_h(tmfqs_gpu_state *h, unsigned qubit);
/* applyPauliX, i_state_backend.h:131; dense_state_backend.cpp:276-287. */
TMFQS_API int tmfqs_gpu_x(tmfqs_gpu_state *h, unsigned qubit);
/* applyControlledPhaseShift, i_state_backend.h:138; dense_state_backend.cpp:289-304
 * (cos/sin of theta taken on the host with the C library, as the reference does). */
TMFQS_API int tmfqs_gpu_cphase(tmfqs_gpu_state *h, unsigned control, unsigned target, double theta);
/* applyControlledNot, i_state_backend.h:144; dense_state_backend.cpp:306-319. */
TMFQS_API int tmfqs_gpu_cnot(tmfqs_gpu_state *h, unsigned control, unsigned target);
/* applyGate, i_state_backend.h:151; gate_block_apply.h:103-213 (k <= 10). */
TMFQS_API int tmfqs_gpu_gate(tmfqs_gpu_state *h, const double *matrix, const unsigned *qubits, unsigned k);
/* QuantumRegister::applySwap, quantum_register.cpp:518-527, as one pass. */
TMFQS_API int tmfqs_gpu_swap(tmfqs_gpu_state *h, unsigned a, unsigned b);

/* ---- batched execution (sim::Simulator::run, simulator.cpp:54-96) ----- */
/* Applies a run of gate operations (H, X, CNOT, CPHASE, SWAP, GATE,
 * PHASE_FLIP) with register semantics, fusing them into multi-gate passes
 * over HBM.  INVERSION is rejected here: it depends on register state and
 * goes through tmfqs_gpu_grover_run or the single-op entry points. */
TMFQS_API int tmfqs_gpu_apply_ops(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t count);
/* Runs `iterations` Grover iterations -- a phase flip of each sorted, unique
 * marked state, then inversion about the mean, materialised or lazy -- with
 * exactly the register semantics of QuantumRegister::applyPhaseFlipBasisState
 * and applyInversionAboutMean[Materialized] (quantum_register.cpp:405-467),
 * updating *view in place (appendGrover, circuit.cpp:118-141). */
TMFQS_API int tmfqs_gpu_grover_run(tmfqs_gpu_state *h, tmfqs_register_view *view, const uint64_t *marked,
                                   size_t count, uint64_t iterations, int materialized);
/* No counterpart in the reference.  The exact measurement of
 * tmfqs_gpu_sample for callers that cannot let the library allocate device
 * memory -- an application whose own caching allocator already holds nearly
 * all of HBM, or a loop that must not pay the device-wide synchronisation of
 * cudaMalloc/cudaFree.  The caller passes its own device state (2^n
 * interleaved complex amplitudes: complex128 for TMFQS_FP64, complex64 for
 * TMFQS_FP32), the draw, the CUDA stream to run on (NULL = default stream)
 * and a host pointer for the index; the function allocates nothing.  Its
 * working tables live in a fixed 2 MiB device array inside the library, so
 * states are limited to num_qubits <= 24 (larger ones return
 * TMFQS_ERR_INVALID_ARGUMENT).  Every call made outside stream capture looks
 * up that array's device address (cudaGetSymbolAddress), so a context reset
 * (cudaDeviceReset, which may reload the library's module elsewhere) is picked
 * up by the next such call; a call on a capturing stream reuses the address
 * of the last call outside capture on that device, so the first call on each
 * device -- and the first after a reset -- must come before any stream capture
 * (otherwise TMFQS_ERR_LOGIC).  All calls share the array -- calls that overlap
 * on the GPU race -- and each call returns after the result is on the host. */
TMFQS_API int tmfqs_sample_static(const void *device_amps, int precision, unsigned num_qubits, double rnd,
                                  void *stream, uint64_t *index_out);
/* The differentiation form (no reference counterpart; its checks use the
 * reference's Dense forward through the parameter-shift rule).  Runs `ops` on
 * the handle's current state psi_0 (the forward pass: the same fused passes as
 * tmfqs_gpu_apply_ops), and returns the expectation E = <psi|O|psi> of the
 * diagonal observable O = sum_j obs_weights[j] * Z(obs_masks[j]) -- Z(m) is the
 * product of Pauli Z over the qubits whose index bits are set in m (qubit q is
 * bit n-1-q), eigenvalue (-1)^popcount(x & m) -- and dE/dtheta for every
 * TMFQS_OP_CPHASE in `ops`, in op order, in `grads` (one double each).
 * Reverse-mode: lambda = O psi is carried back through the inverse circuit;
 * each run of consecutive diagonal ops (controlled phases, phase flips) gets
 * all its derivatives from one read of lambda and psi.  psi is checkpointed
 * every `checkpoint_every` ops of the forward pass (0: the smallest interval
 * whose checkpoints fit in half the free device memory); the backward pass
 * takes psi of each segment from its checkpoint (un-computing it there, in
 * place, where the segment needs it), which bounds the complex64 drift of psi.
 * Ops: H, X, CNOT, CPHASE, SWAP, PHASE_FLIP, GATE (INVERSION is rejected);
 * 1 <= obs_terms <= 64.  On return the handle holds the final state. */
TMFQS_API int tmfqs_gpu_adjoint_gradient(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t count,
                                         const uint64_t *obs_masks, const double *obs_weights, unsigned obs_terms,
                                         size_t checkpoint_every, double *expectation, double *grads);
/* experiment::compareStates(reference, candidate), comparison.cpp:12-62, on
 * two device states of the same qubit count (either precision, same device):
 * every field equals the reference's, bit for bit -- its left-to-right FP64
 * sums are replayed exactly.  Compares the stored amplitudes (a register's
 * lazy overlay is not applied). */
TMFQS_API int tmfqs_gpu_compare(tmfqs_gpu_state *reference, tmfqs_gpu_state *candidate, tmfqs_state_comparison *out);
/* endOperationBatch, i_state_backend.h:163: waits for all queued work. */
TMFQS_API int tmfqs_gpu_sync(tmfqs_gpu_state *h);

/* ---- host-side inputs and draws (no GPU needed) ------------------------ */
/* QuantumState::randomPhase(n, seed), state/quantum_state.cpp:264-277 (and
 * buildRandomPhaseInput, examples/qftG.cpp:70-81): 2^(n+1) doubles. */
TMFQS_API int tmfqs_random_phase(unsigned num_qubits, uint32_t seed, double *host_out);
/* The first `count` draws of Mt19937RandomSource(seed).nextUnitDouble(),
 * core/random.h:32-58 -- the draws measure() consumes. */
TMFQS_API int tmfqs_mt19937_unit(uint32_t seed, uint64_t count, double *host_out);
/* `count` distinct basis states drawn by std::uniform_int_distribution<uint64_t>(lo, hi)
 * over std::mt19937_64(seed), in draw order (repeats skipped): the marked
 * states of the 30-qubit, 4-marked-state Grover benchmark.  No reference
 * counterpart (its CLIs take the marked states as arguments). */
TMFQS_API int tmfqs_uniform_states(uint64_t seed, uint64_t count, uint64_t lo, uint64_t hi, uint64_t *host_out);

/* ---- instrumentation -------------------------------------------------- */
TMFQS_API int tmfqs_gpu_stats(tmfqs_gpu_state *h, tmfqs_stats *out);
TMFQS_API int tmfqs_gpu_reset_stats(tmfqs_gpu_state *h);
TMFQS_API int tmfqs_gpu_set_option(tmfqs_gpu_state *h, int option, long value);
/* Per-class device times recorded while TMFQS_OPT_KERNEL_TIMING is on
 * (synchronises the stream; `out` has TMFQS_KT_COUNT entries).  Reset with
 * tmfqs_gpu_reset_stats. */
TMFQS_API int tmfqs_gpu_kernel_times(tmfqs_gpu_state *h, tmfqs_kernel_time *out);
/* One timed device pass (recorded while TMFQS_OPT_KERNEL_TIMING is on).  The
 * per-operation trace of sim::Simulator (simulator.cpp:72-82, RunReport of
 * report.cpp:39-93) becomes one entry per pass when operations are fused:
 * a pass of tmfqs_gpu_apply_ops covers ops [first_op, first_op + op_count) of
 * that call; other launches (Grover runs, reductions) have op_count 0. */
typedef struct tmfqs_pass_record {
	int kind;          /* TMFQS_KT_* class */
	unsigned op_count; /* operations of the apply_ops call the pass applied (0: not a gate batch) */
	uint64_t segment;  /* the handle's segment number when the pass was launched (tmfqs_gpu_pass_mark) */
	uint64_t first_op; /* index of its first operation within that tmfqs_gpu_apply_ops call */
	double ms;         /* CUDA-event time on the handle's stream */
	double bytes;      /* algorithmic HBM bytes of the pass */
} tmfqs_pass_record;
/* Starts a new segment of the pass log and returns its number (segments let a
 * caller map passes back to the calls it made).  tmfqs_gpu_reset_stats clears
 * the log and restarts the numbering at 0. */
TMFQS_API int tmfqs_gpu_pass_mark(tmfqs_gpu_state *h, uint64_t *segment_out);
/* Waits for the handle's stream, then copies up to `capacity` records of the
 * log (oldest first) and sets *count to the log's length (out may be NULL to
 * query it). */
TMFQS_API int tmfqs_gpu_pass_log(tmfqs_gpu_state *h, tmfqs_pass_record *out, size_t capacity, size_t *count);
/* The handle's device buffer and CUDA stream (for device-resident benchmarks
 * and interop; the buffer stays owned by the handle). */
TMFQS_API int tmfqs_gpu_device_buffer(tmfqs_gpu_state *h, void **ptr, size_t *bytes);
TMFQS_API int tmfqs_gpu_stream(tmfqs_gpu_state *h, void **stream);

#ifdef __cplusplus
}
#endif

#endif /* TMFQS_B200_H */
