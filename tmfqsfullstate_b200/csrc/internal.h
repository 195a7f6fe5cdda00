// Internal interfaces of libtmfqs_b200: the handle, kernel launchers, and the
// fused-pass program format.  Not part of the public C ABI.
#ifndef TMFQS_B200_INTERNAL_H
#define TMFQS_B200_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/tmfqs_b200.h"

namespace tqb {

// ---------------------------------------------------------------------------
// Errors: launchers throw Error; the C ABI converts it to a status code.
// ---------------------------------------------------------------------------
struct Error {
	int status;
	std::string message;
};

[[noreturn]] void fail(int status, const std::string &message);
void check_cuda(cudaError_t e, const char *what);

// cudaMalloc for the library's device buffers.  While the failure knob of
// tmfqs_debug_fail_allocations is armed it returns cudaErrorMemoryAllocation
// instead (without calling cudaMalloc), so the out-of-memory paths can be
// tested on the host side without exhausting a GPU.
cudaError_t device_alloc(void **p, size_t bytes);
void arm_alloc_failures(unsigned skip, unsigned count);

// ---------------------------------------------------------------------------
// Exact sequential-sum engine (seqsum.cu)
// ---------------------------------------------------------------------------
enum TermKind { kTermProb = 0, kTermReal = 1, kTermImag = 2 };

struct Overlay {
	bool active = false;
	double sre = 1.0, sim = 0.0, bre = 0.0, bim = 0.0;
};

struct SeqScratch {
	void *base = nullptr;  // one device allocation, carved below
	size_t bytes = 0;
	uint64_t tiles = 0, groups = 0;
	void *tile_a = nullptr, *tile_pre = nullptr, *tile_b = nullptr;
	void *group_a = nullptr, *group_pre = nullptr, *group_b = nullptr;
	void *walk_out = nullptr;  // WalkOut
	void *host_out = nullptr;  // pinned WalkOut mirror
};

struct SeqResult {
	uint64_t index;  // first index whose running sum reaches the threshold, or N
	double value;    // running sum at that index (or the full sum)
};

// Computes the reference's left-to-right double sum of term(j), j < N, or
// with stop=true the first j whose running sum reaches rnd.  Synchronises.
SeqResult seq_replay(int precision, const void *amps, uint64_t N, TermKind kind, const Overlay &ov, bool stop,
                     double rnd, SeqScratch &scratch, cudaStream_t stream, int num_sms, uint64_t *launches);
void seq_scratch_free(SeqScratch &scratch);
// The reference's left-to-right sum over j of |got_j - ref_j|^2
// (experiment::compareStates), exactly.  Synchronises.
double seq_diff_norm(int prec_ref, const void *ref, int prec_got, const void *got, uint64_t N, SeqScratch &scratch,
                     cudaStream_t stream, int num_sms, uint64_t *launches);
// sampleMeasurement over a caller-owned device state, using the library's
// fixed device scratch instead of allocating (tmfqs_sample_static).
SeqResult seq_sample_static(int precision, const void *amps, unsigned num_qubits, double rnd, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Single-operation kernels (gates.cu)
// ---------------------------------------------------------------------------
// Pinned staging slots for small host-to-device uploads (pass programs): a
// copy leaves the host at once and a slot is reused only after its copy has
// completed, so the host can plan passes while the GPU runs earlier ones.
struct UploadRing {
	static constexpr unsigned kSlots = 8;
	static constexpr size_t kSlotBytes = size_t(64) << 10;
	unsigned char *host = nullptr;
	cudaEvent_t ev[kSlots] = {};
	bool pending[kSlots] = {};
	unsigned next = 0;
};

struct LaunchCtx {
	cudaStream_t stream;
	int num_sms;
	uint64_t *launches;
	int *err = nullptr;          // device-visible error word of the handle (nonzero: a bounded wait gave up)
	UploadRing *ring = nullptr;  // the handle's upload slots
};

// Copies `bytes` from host memory to `dev` in stream order: through a slot of
// the context's ring when it fits (no host wait), else synchronously.
void upload_async(const LaunchCtx &c, void *dev, const void *src, size_t bytes, const char *what);

void launch_h(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned bit);
void launch_x(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned bit);
void launch_cnot(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned cbit, unsigned tbit);
void launch_cphase(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned cbit, unsigned tbit, double cr,
                   double ci);
void launch_swap(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned abit, unsigned bbit);
void launch_phase_flip(const LaunchCtx &c, int prec, void *a, uint64_t s);
void launch_inversion(const LaunchCtx &c, int prec, void *a, unsigned n, double two_mre, double two_mim);
void launch_affine(const LaunchCtx &c, int prec, void *a, unsigned n, double sre, double sim, double bre,
                   double bim);
// Fast forms: the amplitude sum in FP64, one partial (re, im) per block of
// sum_fast_blocks(c) blocks into `part`, added by the caller in block order.
unsigned sum_fast_blocks(const LaunchCtx &c);
void launch_sum_fast(const LaunchCtx &c, int prec, const void *a, uint64_t N, double2 *part);
void launch_scatter_uniform(const LaunchCtx &c, int prec, void *a, const uint64_t *states, uint64_t count,
                            double amp);
void launch_scatter_values(const LaunchCtx &c, int prec, void *a, const uint64_t *idx, const double *vals,
                           uint64_t count);
// matrix: device, row-major 2^k x 2^k interleaved complex (double);
// tpos: device array of the k target bit positions in block order.
void launch_gate(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned k, const double *matrix,
                 const unsigned *tpos_host);
// complex128 <-> complex64 conversion of `count` amplitudes (device buffers).
void launch_to_c64(const LaunchCtx &c, void *dst, const double *src, uint64_t count);
void launch_from_c64(const LaunchCtx &c, double *dst, const void *src, uint64_t count);

// ---------------------------------------------------------------------------
// Fused multi-gate passes (fused.cu)
// ---------------------------------------------------------------------------
enum FusedOpKind : uint32_t {
	kFH = 0,       // Hadamard on local bit
	kFHChain = 1,  // Hadamard on local bit, then a chain of controlled phases on its |1> half
	kFX = 2,       // Pauli-X on local bit
	kFCnot = 3,    // CNOT: local target bit, global control mask
	kFCP = 4,      // controlled phase, any two bits (diagonal)
	kFFlip = 5,    // phase flip of one basis state (diagonal)
	kFSwap = 6,    // swap of two local bits
	kFHTwiddle = 7 // Hadamard, then its H-chain applied as one twiddle per |1> output
};

struct FusedOp {
	uint32_t kind;
	uint32_t lt;     // local target bit (H, HChain, X, CNOT, Swap first)
	uint32_t lc;     // Swap: second local bit; HChain: number of chain entries
	uint32_t tab;    // HChain: index of its first entry in FusedPass::chain
	uint64_t mask;   // CNOT: control mask; CP: both bit masks
	uint64_t state;  // Flip state
	double cr, ci;   // CP phase
	double theta;    // CP angle (fast forms)
};

// One controlled phase of an H-chain, in circuit order (bit positions
// strictly descending along a chain).
struct ChainEntry {
	double cr, ci;   // cos(theta), sin(theta) from the host C library
	double theta;    // the angle itself (twiddle form)
	int32_t local;   // local bit index of the other qubit, or -1 if it is an outer bit
	uint32_t bit;    // global bit position of the other qubit
};

struct FusedPass {
	unsigned n = 0;
	unsigned K = 0;                 // local bits (tile = 2^K amplitudes)
	unsigned lpos[16] = {0};        // global bit position of local bit i, ascending
	std::vector<FusedOp> ops;
	std::vector<ChainEntry> chain;  // H-chain entries of all chains of the pass
	unsigned gate_count = 0;        // circuit operations folded into this pass
	// Exact fused passes: run only tiles [tile_begin, tile_end) (0, 0: all).
	uint64_t tile_begin = 0, tile_end = 0;
	// The pass's program is already in `dev_prog` (prepare_fused_pass): the
	// launch uploads nothing.
	bool program_ready = false;
};

// Runs one fused pass over the whole state.  `dev_prog` is a device buffer
// the launcher may (re)use for the program.
void launch_fused_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, void *&dev_prog,
                       size_t &dev_prog_bytes);

// Uploads the program of an exact register-stage pass into `dev_prog` ahead
// of its launches (the tile ranges of one pass share it); false when the pass
// runs another kernel (which uploads at launch).
bool prepare_fused_pass(const LaunchCtx &c, int prec, const FusedPass &pass, void *&dev_prog, size_t &dev_prog_bytes);

// Radix-2^RB form of a fused pass for the fast forms (complex64, or complex128
// without exact arithmetic): programs of H, H-chains, twiddles and controlled
// phases.  Returns false (nothing launched) when the pass does not qualify.
// With `mirror` (a state-sized buffer) the pass also writes its result there.
bool launch_radix_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, void *&dev_prog,
                       size_t &dev_prog_bytes, void *mirror = nullptr);

// The dedicated pass for a segment of the QFT ladder (Hadamards on consecutive
// descending bits, each followed by the phases pi/2^(b-c) with every lower bit
// c of the register) in the fast forms.  Returns false (nothing launched) when
// the pass is not such a segment or its layout does not qualify.
// A QFT segment pass (k_qft_pass); with allow_walsh also a pass of Hadamards
// only.  False: the pass is neither (or does not fit the kernel's tiles).
bool launch_qft_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, bool allow_walsh);

// ---------------------------------------------------------------------------
// Adjoint gradient (adjoint.cu)
// ---------------------------------------------------------------------------
constexpr unsigned kMaxObsTerms = 64;  // Z-string terms of a diagonal observable
constexpr unsigned kMaxDiagRun = 32;   // diagonal gates per gradient pass

enum DiagKind : int { kDiagCPhase = 0, kDiagFlip = 1 };

struct DiagEntry {
	int kind;       // DiagKind
	uint64_t mask;  // controlled phase: both bit masks; flip: the basis state
	double cr, ci;  // controlled phase: cos(theta), sin(theta)
};

// Upper bound on the blocks (and so the per-block partial sums) of a launch.
unsigned adjoint_max_blocks(int num_sms);
// lambda = O psi; writes one FP64 partial of <psi|O|psi> per block; returns
// the number of blocks.
unsigned launch_obs_apply(const LaunchCtx &c, int prec, const void *psi, void *lam, unsigned n, const uint64_t *masks,
                          const double *weights, unsigned nterms, double *dev_partials);
// Angle-derivative sums of a diagonal run (partials[block * kMaxDiagRun + k]),
// then the run's inverse on lambda (and on psi if asked); returns the blocks.
// Entries that depend on index bits 0-2 (flips, masks with a bit there) placed
// first, at most 8 of them, let the pass look up one phase table per amplitude.
unsigned launch_grad_run(const LaunchCtx &c, int prec, void *lam, void *psi, unsigned n, const DiagEntry *entries,
                         unsigned count, bool uncompute_psi, double *dev_partials);

// Partial-sum arrays left on the device by the launches above, reduced
// together: array i starts at partials + i * chunk_doubles and holds
// blocks[i] rows of stride[i] (<= kMaxDiagRun) columns.
constexpr unsigned kMaxPendingSums = 64;
struct PartialChunks {
	unsigned count;
	unsigned blocks[kMaxPendingSums];
	unsigned stride[kMaxPendingSums];
};
// out[i * kMaxDiagRun + k] = sum of column k of array i over its rows, in FP64
// and in a fixed order (32 interleaved row-order sums, then a fixed tree), so
// the result does not depend on scheduling.
void launch_sum_partials(const LaunchCtx &c, const double *partials, size_t chunk_doubles, const PartialChunks &t,
                         double *out);

// ---------------------------------------------------------------------------
// Tensor-core dense gates on complex64 states (tc_gate.cu)
// ---------------------------------------------------------------------------
bool tc_gate_supported(int prec, unsigned n, unsigned k);
// matrix_host: row-major 2^k x 2^k interleaved complex (double); tpos: the k
// target bit positions in block order.  dev_buf is the launcher's reusable
// device buffer.  Synchronises.
void launch_tc_gate(const LaunchCtx &c, void *a, unsigned n, unsigned k, const double *matrix_host, const unsigned *tpos,
                    void *&dev_buf, size_t &dev_buf_bytes);

// ---------------------------------------------------------------------------
// Device compareStates (compare.cu): the order-independent fields.
// ---------------------------------------------------------------------------
struct CompareReport {
	bool bitwise_equal;
	double max_abs_amplitude_error, max_abs_component_error, max_abs_probability_error;
	uint64_t worst_state;
};
void launch_compare(const LaunchCtx &c, int prec_ref, const void *ref, int prec_got, const void *got, uint64_t N,
                    CompareReport &out);

// Involutive permutation of bit positions (disjoint transpositions), as one
// in-place pass: amplitude x moves to perm(x).  pairs[i] = (p, q) bit positions.
void launch_bit_permutation(const LaunchCtx &c, int prec, void *a, unsigned n,
                            const std::vector<std::pair<unsigned, unsigned>> &pairs);

// Materialised Grover iterations as one temporal pass: for k in [0,K):
// flip marked states, then a <- two_mean[k] - a (exact per-iteration ops).
// two_mean holds complex values in the storage type (double2 / float2).
// Marked states are flipped from iteration `flip_from` on (the first
// iteration's flips may already have been applied when its mean was taken).
void launch_grover_temporal(const LaunchCtx &c, int prec, void *a, unsigned n, const void *dev_two_means,
                            uint64_t iterations, const uint64_t *dev_marked, unsigned marked_count,
                            uint64_t flip_from);

}  // namespace tqb

// ---------------------------------------------------------------------------
// The handle.
// ---------------------------------------------------------------------------
struct tmfqs_gpu_state {
	int device = 0;
	int precision = TMFQS_FP64;
	int num_sms = 148;
	unsigned n = 0;
	uint64_t N = 0;
	bool initialized = false;
	void *amps = nullptr;
	size_t bytes = 0;
	cudaStream_t stream = nullptr;
	cudaStream_t copy_stream = nullptr;  // tmfqs_gpu_load_apply_ops: host-to-device slabs
	tqb::SeqScratch seq;
	// Host cache of single amplitudes (amplitude / setAmplitude / phase flips
	// of cached states); dirty entries are flushed before any kernel runs.
	std::unordered_map<uint64_t, std::pair<double, double>> cache;
	std::unordered_map<uint64_t, bool> dirty;
	double *pinned = nullptr;  // small pinned staging buffer
	size_t pinned_elems = 0;
	void *dev_small = nullptr;  // small device staging buffer
	size_t dev_small_bytes = 0;
	void *dev_prog = nullptr;
	size_t dev_prog_bytes = 0;
	tmfqs_stats stats{};
	// Kernel timing (TMFQS_OPT_KERNEL_TIMING): event pairs per class, resolved lazily.
	bool opt_timing = false;
	struct TimedLaunch {
		int kind;
		cudaEvent_t start, stop;
		double bytes;
		uint64_t segment, first;
		unsigned count;
	};
	std::vector<TimedLaunch> timed;
	tmfqs_kernel_time times[TMFQS_KT_COUNT] = {};
	// Pass log (tmfqs_gpu_pass_log): the op range of the launch being issued
	// (within the current apply_ops call; count 0 outside gate batches).
	uint64_t segment = 0, cur_first = 0;
	unsigned cur_count = 0;
	std::vector<tmfqs_pass_record> pass_log;
	bool opt_fusion = true;
	int opt_fused_qubits = 0;  // 0 = default by precision
	bool opt_grover_fusion = true;
	bool opt_exact = true;
	bool opt_radix = true;  // fast forms: radix passes where the program allows
	bool opt_tensor = true; // complex64: 4- and 5-qubit gates on the tensor cores
	bool opt_qft_pass = true;  // fast forms: QFT ladder segments on the dedicated QFT pass
	int *err_host = nullptr;   // mapped pinned error word written by bounded device waits
	int *err_dev = nullptr;
	tqb::UploadRing ring;      // pinned staging for pass programs
	void *dev_tc = nullptr; // tensor-core gate operands
	size_t dev_tc_bytes = 0;
	// Adjoint-gradient work buffers, kept for the next call (freed by destroy):
	// psi checkpoints, FP64 partial sums, and the lambda / psi work states.
	void *adj_ckpt = nullptr;
	size_t adj_ckpt_bytes = 0;
	void *adj_part = nullptr;
	tmfqs_gpu_state *adj_lam = nullptr, *adj_psi = nullptr;
};

#endif
