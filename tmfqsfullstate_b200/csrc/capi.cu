// C ABI of libtmfqs_b200 (declared in include/tmfqs_b200.h).
//
// Validation mirrors the reference backend and register contracts
// (core/validation.h:19-80, storage/common/backend_validation.h:13-39,
// dense_state_backend.cpp:31-50) with 64-bit state counts.  Errors become
// status codes plus a thread-local message.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace tqb {

void fail(int status, const std::string &message) { throw Error{status, message}; }

void check_cuda(cudaError_t e, const char *what) {
	if(e != cudaSuccess) {
		cudaGetLastError();
		throw Error{TMFQS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
	}
}

namespace {
std::mutex g_fail_mutex;
unsigned g_fail_skip = 0, g_fail_count = 0;
}  // namespace

void arm_alloc_failures(unsigned skip, unsigned count) {
	std::lock_guard<std::mutex> lock(g_fail_mutex);
	g_fail_skip = skip;
	g_fail_count = count;
}

cudaError_t device_alloc(void **p, size_t bytes) {
	{
		std::lock_guard<std::mutex> lock(g_fail_mutex);
		if(g_fail_count > 0) {
			if(g_fail_skip > 0) {
				--g_fail_skip;
			} else {
				--g_fail_count;
				*p = nullptr;
				return cudaErrorMemoryAllocation;
			}
		}
	}
	return cudaMalloc(p, bytes);
}

}  // namespace tqb

namespace {

using tqb::fail;
using tqb::check_cuda;

thread_local std::string g_last_error;

template <class F>
int guarded(F &&fn) {
	try {
		fn();
		return TMFQS_OK;
	} catch(const tqb::Error &e) {
		g_last_error = e.message;
		return e.status;
	} catch(const std::bad_alloc &) {
		g_last_error = "host allocation failed";
		return TMFQS_ERR_NOMEM;
	} catch(const std::exception &e) {
		g_last_error = e.what();
		return TMFQS_ERR_RUNTIME;
	}
}

constexpr unsigned kMaxQubits = 40;
constexpr size_t kPinnedElems = 3 * 4096;  // idx + 2 doubles per flushed entry

struct DeviceScope {
	explicit DeviceScope(const tmfqs_gpu_state *h) { check_cuda(cudaSetDevice(h->device), "cudaSetDevice"); }
};

tqb::LaunchCtx ctx(tmfqs_gpu_state *h) {
	return tqb::LaunchCtx{h->stream, h->num_sms, &h->stats.kernel_launches, h->err_dev, &h->ring};
}

// Reports (and clears) a failure recorded by a bounded device wait since the
// last check.  Call after the stream has been synchronized.
void check_device_error(tmfqs_gpu_state *h) {
	if(h->err_host && *reinterpret_cast<volatile int *>(h->err_host)) {
		*reinterpret_cast<volatile int *>(h->err_host) = 0;
		fail(TMFQS_ERR_RUNTIME, "a device pass gave up waiting for its tile copies");
	}
}

size_t amp_bytes(const tmfqs_gpu_state *h) { return h->precision == TMFQS_FP64 ? 16 : 8; }

// Records CUDA events around one pass when kernel timing is on.
class PassTimer {
	public:
		PassTimer(tmfqs_gpu_state *h, int kind, double bytes) : h_(h), kind_(kind), bytes_(bytes) {
			if(!h_->opt_timing) return;
			check_cuda(cudaEventCreate(&start_), "timer event");
			check_cuda(cudaEventCreate(&stop_), "timer event");
			check_cuda(cudaEventRecord(start_, h_->stream), "timer record");
		}
		~PassTimer() {
			if(!h_->opt_timing || !start_) return;
			if(cudaEventRecord(stop_, h_->stream) == cudaSuccess) {
				h_->timed.push_back({kind_, start_, stop_, bytes_, h_->segment, h_->cur_first, h_->cur_count});
			} else {
				cudaGetLastError();
				cudaEventDestroy(start_);
				cudaEventDestroy(stop_);
			}
		}
	private:
		tmfqs_gpu_state *h_;
		int kind_;
		double bytes_;
		cudaEvent_t start_ = nullptr, stop_ = nullptr;
};

double sweep_bytes(const tmfqs_gpu_state *h) { return 2.0 * (double)h->N * (double)amp_bytes(h); }

void resolve_timers(tmfqs_gpu_state *h) {
	for(auto &t : h->timed) {
		check_cuda(cudaEventSynchronize(t.stop), "timer sync");
		float ms = 0.f;
		check_cuda(cudaEventElapsedTime(&ms, t.start, t.stop), "timer elapsed");
		h->times[t.kind].launches += 1;
		h->times[t.kind].ms += ms;
		h->times[t.kind].bytes += t.bytes;
		if(h->pass_log.size() < (size_t(1) << 22))
			h->pass_log.push_back(tmfqs_pass_record{t.kind, t.count, t.segment, t.first, (double)ms, t.bytes});
		cudaEventDestroy(t.start);
		cudaEventDestroy(t.stop);
	}
	h->timed.clear();
}

void require_handle(tmfqs_gpu_state *h) {
	if(!h) fail(TMFQS_ERR_INVALID_ARGUMENT, "null handle");
}

void ensure_initialized(tmfqs_gpu_state *h, const char *operation) {
	require_handle(h);
	if(!h->initialized) fail(TMFQS_ERR_LOGIC, std::string("GpuStateBackend is not initialized for ") + operation);
}

void validate_state(tmfqs_gpu_state *h, uint64_t s, const char *scope) {
	if(s >= h->N) fail(TMFQS_ERR_OUT_OF_RANGE, std::string(scope) + " state index out of range");
}

void validate_qubit(tmfqs_gpu_state *h, unsigned q, const char *scope) {
	if(q >= h->n) fail(TMFQS_ERR_OUT_OF_RANGE, std::string(scope) + " qubit index out of range");
}

void validate_two(tmfqs_gpu_state *h, unsigned a, unsigned b, const char *scope) {
	validate_qubit(h, a, scope);
	validate_qubit(h, b, scope);
	if(a == b) fail(TMFQS_ERR_INVALID_ARGUMENT, std::string(scope) + " requires distinct qubits");
}

unsigned bit_of(const tmfqs_gpu_state *h, unsigned q) { return h->n - q - 1u; }

// Allocates (or reuses) the device state for n qubits.
void ensure_state(tmfqs_gpu_state *h, unsigned n) {
	if(n > kMaxQubits) fail(TMFQS_ERR_INVALID_ARGUMENT, "Number of qubits exceeds supported range for this device build");
	const size_t bytes = amp_bytes(h) << n;
	if(h->amps && h->bytes == bytes) {
		h->n = n;
		h->N = 1ull << n;
		return;
	}
	if(h->amps) {
		check_cuda(cudaStreamSynchronize(h->stream), "sync before free");
		cudaFree(h->amps);
		h->amps = nullptr;
		h->bytes = 0;
	}
	tqb::seq_scratch_free(h->seq);
	if(tqb::device_alloc(&h->amps, bytes) != cudaSuccess) {
		cudaGetLastError();
		h->amps = nullptr;
		h->initialized = false;
		fail(TMFQS_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes for the state failed");
	}
	h->bytes = bytes;
	h->n = n;
	h->N = 1ull << n;
}

void ensure_dev_small(tmfqs_gpu_state *h, size_t bytes) {
	if(h->dev_small_bytes >= bytes) return;
	if(h->dev_small) {
		check_cuda(cudaStreamSynchronize(h->stream), "sync before staging free");
		cudaFree(h->dev_small);
	}
	h->dev_small = nullptr;
	h->dev_small_bytes = 0;
	const size_t sz = std::max<size_t>(bytes, 1 << 16);
	if(tqb::device_alloc(&h->dev_small, sz) != cudaSuccess) {
		cudaGetLastError();
		fail(TMFQS_ERR_NOMEM, "device staging allocation failed");
	}
	h->dev_small_bytes = sz;
}

// Writes dirty cached amplitudes to the device (one scatter per 4096).
void flush_dirty(tmfqs_gpu_state *h) {
	if(h->dirty.empty()) return;
	std::vector<uint64_t> idx;
	idx.reserve(h->dirty.size());
	for(const auto &kv : h->dirty) idx.push_back(kv.first);
	std::sort(idx.begin(), idx.end());
	ensure_dev_small(h, 4096 * 24);
	for(size_t off = 0; off < idx.size(); off += 4096) {
		const size_t cnt = std::min<size_t>(4096, idx.size() - off);
		check_cuda(cudaStreamSynchronize(h->stream), "flush sync");
		uint64_t *pi = reinterpret_cast<uint64_t *>(h->pinned);
		double *pv = h->pinned + cnt;
		for(size_t i = 0; i < cnt; ++i) {
			pi[i] = idx[off + i];
			const auto &v = h->cache[idx[off + i]];
			pv[2 * i] = v.first;
			pv[2 * i + 1] = v.second;
		}
		check_cuda(cudaMemcpyAsync(h->dev_small, h->pinned, cnt * 24, cudaMemcpyHostToDevice, h->stream), "flush upload");
		const uint64_t *di = static_cast<const uint64_t *>(h->dev_small);
		const double *dv = reinterpret_cast<const double *>(static_cast<unsigned char *>(h->dev_small) + cnt * 8);
		tqb::launch_scatter_values(ctx(h), h->precision, h->amps, di, dv, cnt);
		h->stats.h2d_bytes += cnt * 24;
	}
	h->dirty.clear();
}

// Before a kernel that mutates the state: push pending writes, drop the cache.
void before_mutation(tmfqs_gpu_state *h) {
	flush_dirty(h);
	h->cache.clear();
}

// Round a value to the storage precision (what the device will hold).
double to_storage(const tmfqs_gpu_state *h, double v) {
	return h->precision == TMFQS_FP64 ? v : (double)(float)v;
}

std::pair<double, double> read_amp(tmfqs_gpu_state *h, uint64_t s) {
	auto it = h->cache.find(s);
	if(it != h->cache.end()) return it->second;
	const size_t ab = amp_bytes(h);
	check_cuda(cudaMemcpyAsync(h->pinned, static_cast<unsigned char *>(h->amps) + s * ab, ab, cudaMemcpyDeviceToHost,
	                           h->stream),
	           "amplitude read");
	check_cuda(cudaStreamSynchronize(h->stream), "amplitude read sync");
	h->stats.d2h_bytes += ab;
	std::pair<double, double> v;
	if(h->precision == TMFQS_FP64) {
		v = {h->pinned[0], h->pinned[1]};
	} else {
		const float *f = reinterpret_cast<const float *>(h->pinned);
		v = {(double)f[0], (double)f[1]};
	}
	h->cache[s] = v;
	return v;
}

void write_amp(tmfqs_gpu_state *h, uint64_t s, double re, double im) {
	h->cache[s] = {to_storage(h, re), to_storage(h, im)};
	h->dirty[s] = true;
}

// Like write_amp, but the cache keeps the FP64 value: a complex64 state then
// rounds it once, when it is flushed to the device, instead of at every
// register update (the lazy Grover flips rewrite the same few amplitudes once
// per iteration).  Identical to write_amp for complex128.
void carry_amp(tmfqs_gpu_state *h, uint64_t s, double re, double im) {
	h->cache[s] = {re, im};
	h->dirty[s] = true;
}

// Host <-> device copies of interleaved complex128 data, converting for
// complex64 states through a device staging buffer.
void copy_in(tmfqs_gpu_state *h, uint64_t first, const double *host, uint64_t count) {
	if(count == 0) return;
	if(h->precision == TMFQS_FP64) {
		check_cuda(cudaMemcpyAsync(static_cast<double2 *>(h->amps) + first, host, count * 16, cudaMemcpyHostToDevice, h->stream), "load");
	} else {
		const uint64_t chunk = 1ull << 22;
		ensure_dev_small(h, chunk * 16);
		for(uint64_t off = 0; off < count; off += chunk) {
			const uint64_t c = std::min<uint64_t>(chunk, count - off);
			check_cuda(cudaMemcpyAsync(h->dev_small, host + 2 * off, c * 16, cudaMemcpyHostToDevice, h->stream), "load");
			tqb::launch_to_c64(ctx(h), static_cast<float2 *>(h->amps) + first + off, static_cast<const double *>(h->dev_small), c);
		}
	}
	h->stats.h2d_bytes += count * 16;
}

void copy_out(tmfqs_gpu_state *h, uint64_t first, double *host, uint64_t count) {
	if(count == 0) return;
	if(h->precision == TMFQS_FP64) {
		check_cuda(cudaMemcpyAsync(host, static_cast<double2 *>(h->amps) + first, count * 16, cudaMemcpyDeviceToHost, h->stream), "export");
	} else {
		const uint64_t chunk = 1ull << 22;
		ensure_dev_small(h, chunk * 16);
		for(uint64_t off = 0; off < count; off += chunk) {
			const uint64_t c = std::min<uint64_t>(chunk, count - off);
			tqb::launch_from_c64(ctx(h), static_cast<double *>(h->dev_small), static_cast<const float2 *>(h->amps) + first + off, c);
			check_cuda(cudaMemcpyAsync(host + 2 * off, h->dev_small, c * 16, cudaMemcpyDeviceToHost, h->stream), "export");
		}
	}
	check_cuda(cudaStreamSynchronize(h->stream), "export sync");
	h->stats.d2h_bytes += count * 16;
}

tqb::SeqResult reduce(tmfqs_gpu_state *h, tqb::TermKind kind, const tqb::Overlay &ov, bool stop, double rnd) {
	flush_dirty(h);
	h->stats.reduction_passes += 2;
	PassTimer timer(h, TMFQS_KT_REDUCE, sweep_bytes(h));  // two read passes = one sweep's bytes
	return tqb::seq_replay(h->precision, h->amps, h->N, kind, ov, stop, rnd, h->seq, h->stream, h->num_sms,
	                       &h->stats.kernel_launches);
}

// ---------------------------------------------------------------------------
// Fusion planner for tmfqs_gpu_apply_ops (the Simulator's gate runs).
// ---------------------------------------------------------------------------
struct Planner {
	tmfqs_gpu_state *h;
	unsigned K;     // local bits of a pass
	unsigned mlow;  // low bits always local (row of >= 128 bytes)
	tqb::FusedPass pass;
	uint64_t tmask = 0;  // bits that must be local (moving bits of ops in the pass)
	int chain_op = -1;   // index of the H-chain op that may still grow
	size_t nontrivial = 0;
	std::vector<const tmfqs_op *> pending;  // circuit ops in the pass (for single-op fallback)
	std::vector<unsigned> msched;  // fast forms: low-bit width of the first multi-op passes
	unsigned mrest = 0;            // ... and of the passes after them
	size_t npass = 0;              // multi-op passes run so far
	void *mirror = nullptr;        // a radix pass launched by the next flush also writes its result here
	bool mirrored = false;         // ... and did
	const tmfqs_op *base = nullptr;  // the apply_ops call's op array (pass-log op indexes)
	// Dry run (tmfqs_gpu_load_apply_ops): the first flushed pass is recorded,
	// not launched.
	bool dry = false, dry_done = false;
	size_t dry_ops = 0;
	tqb::FusedPass dry_pass;

	explicit Planner(tmfqs_gpu_state *hh) : h(hh) {
		// Tiles of 2^12 complex128 / 2^13 complex64 amplitudes (64 KB).  The
		// exact form keeps rows of >= 128 bytes local; the fast forms' radix
		// passes copy 16-byte granules and take rows of 32 (complex128) or 64
		// (complex64) bytes, which leaves more bits per pass for the circuit.
		const unsigned Kmax = h->precision == TMFQS_FP64 ? 12u : 13u;
		const bool fast = !h->opt_exact || h->precision == TMFQS_FP32;
		if(fast && h->opt_radix) {
			// Wider rows (up to four times the narrowest) stream far better when
			// the other local bits are high, so take the widest that still
			// covers all n bits in the fewest passes.
			auto passes = [&](unsigned m) -> unsigned {
				return h->n <= Kmax ? 1u : 1u + (h->n - Kmax + (Kmax - m) - 1u) / (Kmax - m);
			};
			const unsigned mmin = h->precision == TMFQS_FP64 ? 2u : 3u, mmax = mmin + 2u;
			mlow = mmin;
			for(unsigned m = mmin + 1; m <= mmax; ++m)
				if(passes(m) == passes(mmin)) mlow = m;
			mrest = mlow;
			// Per pass: the fewest passes need (P-1)(Kmax-mmin)+Kmax >= n bits; the
			// spare bits widen the rows of the first passes one by one (a QFT's
			// last pass holds the Kmax lowest bits, contiguous whatever its width).
			if(h->opt_fused_qubits == 0 && h->n > Kmax) {
				const unsigned P = passes(mmin);
				unsigned slack = (P - 1) * (Kmax - mmin) + Kmax - h->n;
				for(unsigned i = 0; i + 1 < P; ++i) {
					const unsigned inc = std::min(mmax - mmin, slack);
					msched.push_back(mmin + inc);
					slack -= inc;
				}
				mlow = msched[0];
			}
		} else {
			mlow = h->precision == TMFQS_FP64 ? 3u : 4u;
		}
		const unsigned q = h->opt_fused_qubits > 0 ? (unsigned)h->opt_fused_qubits : Kmax - mlow;
		K = std::min<unsigned>(h->n, std::min<unsigned>(Kmax, q + mlow));
		reset();
	}

	void reset() {
		if(!msched.empty()) mlow = npass < msched.size() ? msched[npass] : mrest;
		pass = tqb::FusedPass{};
		pass.n = h->n;
		tmask = 0;
		chain_op = -1;
		nontrivial = 0;
		pending.clear();
	}

	// Whether bits in `m` can be local together with the current ones.
	bool fits(uint64_t m) const {
		const uint64_t all = tmask | m;
		const uint64_t low = mlow >= 64 ? ~0ull : ((1ull << mlow) - 1ull);
		const unsigned extra = (unsigned)__builtin_popcountll(all & ~low);
		return extra + std::min(mlow, h->n) <= K;
	}

	unsigned local_index(unsigned bit) const {
		for(unsigned i = 0; i < pass.K; ++i)
			if(pass.lpos[i] == bit) return i;
		fail(TMFQS_ERR_LOGIC, "planner: bit not local");
	}

	void finalize_local_set() {
		std::vector<unsigned> L;
		for(unsigned b = 0; b < h->n; ++b)
			if((tmask >> b) & 1ull) L.push_back(b);
		for(unsigned b = 0; b < h->n && L.size() < K; ++b)
			if(!((tmask >> b) & 1ull)) L.push_back(b);
		std::sort(L.begin(), L.end());
		pass.K = (unsigned)L.size();
		for(unsigned i = 0; i < pass.K; ++i) pass.lpos[i] = L[i];
	}

	// A chain becomes a twiddle when its local controls are distinct and fit
	// the two per-tile tables (6 + 5 bits); outer controls are unlimited.
	bool twiddle_ok(const tqb::FusedOp &op) const {
		uint32_t seen = 0;
		unsigned locals = 0;
		for(unsigned e = 0; e < op.lc; ++e) {
			const auto &ce = pass.chain[op.tab + e];
			if(ce.local < 0) continue;
			if(seen & (1u << ce.local)) return false;
			seen |= 1u << ce.local;
			++locals;
		}
		return locals <= 11;
	}

	// Ops are recorded with global bit positions in `lt`/`lc` and converted to
	// local indices once the local set is known.
	void flush() {
		if(pending.empty()) return;
		// The pass is consumed whether or not its launch succeeds: a failed
		// launch must not leave its (already converted) ops pending for the
		// error path's flush of the ops before a failing one.
		struct Consume {
			Planner *p;
			~Consume() { p->reset(); }
		} consume{this};
		if(base) {
			h->cur_first = (uint64_t)(pending.front() - base);
			h->cur_count = (unsigned)pending.size();
		}
		if(dry && pending.size() == 1) {
			dry_done = true;  // a single-gate pass: nothing to overlap with
			dry_ops = 0;
		} else if(pending.size() == 1) {
			run_single(*pending[0]);
		} else {
			finalize_local_set();
			for(auto &e : pass.chain) {
				e.local = -1;
				for(unsigned i = 0; i < pass.K; ++i)
					if(pass.lpos[i] == e.bit) e.local = (int32_t)i;
			}
			const bool twiddle = !h->opt_exact || h->precision == TMFQS_FP32;
			for(auto &op : pass.ops) {
				if(op.kind == tqb::kFHChain && twiddle && twiddle_ok(op)) op.kind = tqb::kFHTwiddle;
				if(op.kind == tqb::kFH || op.kind == tqb::kFHChain || op.kind == tqb::kFHTwiddle || op.kind == tqb::kFX ||
				   op.kind == tqb::kFCnot)
					op.lt = local_index(op.lt);
				if(op.kind == tqb::kFSwap) {
					op.lt = local_index(op.lt);
					op.lc = local_index(op.lc);
				}
			}
			pass.gate_count = (unsigned)pending.size();
			if(dry) {
				dry_done = true;
				dry_ops = pending.size();
				dry_pass = pass;
				return;
			}
			++npass;
			PassTimer timer(h, TMFQS_KT_FUSED, sweep_bytes(h));
			const bool qft = twiddle && h->opt_radix && h->opt_qft_pass &&
			                 tqb::launch_qft_pass(ctx(h), h->precision, h->amps, pass, mirror == nullptr);
			if(qft) ++h->stats.qft_passes;
			const bool done = qft || (twiddle && h->opt_radix &&
			                          tqb::launch_radix_pass(ctx(h), h->precision, h->amps, pass, h->dev_prog, h->dev_prog_bytes,
			                                                 mirror));
			mirrored = !qft && done && mirror;
			if(!done) tqb::launch_fused_pass(ctx(h), h->precision, h->amps, pass, h->dev_prog, h->dev_prog_bytes);
			++h->stats.fused_passes;
		}
	}

	void run_single(const tmfqs_op &op) {
		const auto c = ctx(h);
		PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
		switch(op.kind) {
			case TMFQS_OP_H: tqb::launch_h(c, h->precision, h->amps, h->n, bit_of(h, op.q0)); break;
			case TMFQS_OP_X: tqb::launch_x(c, h->precision, h->amps, h->n, bit_of(h, op.q0)); break;
			case TMFQS_OP_CNOT: tqb::launch_cnot(c, h->precision, h->amps, h->n, bit_of(h, op.q0), bit_of(h, op.q1)); break;
			case TMFQS_OP_CPHASE:
				tqb::launch_cphase(c, h->precision, h->amps, h->n, bit_of(h, op.q0), bit_of(h, op.q1), std::cos(op.theta), std::sin(op.theta));
				break;
			case TMFQS_OP_SWAP: tqb::launch_swap(c, h->precision, h->amps, h->n, bit_of(h, op.q0), bit_of(h, op.q1)); break;
			case TMFQS_OP_PHASE_FLIP: tqb::launch_phase_flip(c, h->precision, h->amps, op.state); break;
			default: fail(TMFQS_ERR_LOGIC, "planner: unexpected single op");
		}
		++h->stats.gate_passes;
	}

	void add_pair_op(const tmfqs_op &op, uint32_t kind, unsigned bit, uint64_t cmask) {
		const uint64_t m = 1ull << bit;
		if(!fits(m)) flush();
		tmask |= m;
		tqb::FusedOp f{};
		f.kind = kind;
		f.lt = bit;
		f.mask = cmask;
		pass.ops.push_back(f);
		pending.push_back(&op);
		++nontrivial;
		chain_op = -1;
		if(kind == tqb::kFH) {
			// A Hadamard may grow into an H-chain with the phases that follow.
			chain_op = (int)pass.ops.size() - 1;
		}
	}

	void add(const tmfqs_op &op) {
		switch(op.kind) {
			case TMFQS_OP_H: add_pair_op(op, tqb::kFH, bit_of(h, op.q0), 0); return;
			case TMFQS_OP_X: add_pair_op(op, tqb::kFX, bit_of(h, op.q0), 0); return;
			case TMFQS_OP_CNOT: add_pair_op(op, tqb::kFCnot, bit_of(h, op.q1), 1ull << bit_of(h, op.q0)); return;
			case TMFQS_OP_SWAP: {
				const unsigned a = bit_of(h, op.q0), b = bit_of(h, op.q1);
				const uint64_t m = (1ull << a) | (1ull << b);
				if(!fits(m)) flush();
				tmask |= m;
				tqb::FusedOp f{};
				f.kind = tqb::kFSwap;
				f.lt = a;
				f.lc = b;
				pass.ops.push_back(f);
				pending.push_back(&op);
				chain_op = -1;
				return;
			}
			case TMFQS_OP_CPHASE: {
				const unsigned bc = bit_of(h, op.q0), bt = bit_of(h, op.q1);
				const double cr = std::cos(op.theta), ci = std::sin(op.theta);  // dense_state_backend.cpp:293-294
				if(chain_op >= 0) {
					tqb::FusedOp &ch = pass.ops[chain_op];
					const unsigned hb = ch.lt;  // global bit of the chain's Hadamard
					const int other = bc == hb ? (int)bt : (bt == hb ? (int)bc : -1);
					// Any controlled phase on the Hadamard's qubit that directly follows
					// it acts only on the butterflies' |1> outputs: append it to the chain.
					if(other >= 0 && ch.lc < 64) {
						if(ch.kind == tqb::kFH) {
							ch.kind = tqb::kFHChain;
							ch.tab = (uint32_t)pass.chain.size();
							ch.lc = 0;
						}
						pass.chain.push_back(tqb::ChainEntry{cr, ci, op.theta, -1, (uint32_t)other});
						++ch.lc;
						pending.push_back(&op);
						return;
					}
				}
				tqb::FusedOp f{};
				f.kind = tqb::kFCP;
				f.mask = (1ull << bc) | (1ull << bt);
				f.cr = cr;
				f.ci = ci;
				f.theta = op.theta;
				pass.ops.push_back(f);
				pending.push_back(&op);
				chain_op = -1;
				return;
			}
			case TMFQS_OP_PHASE_FLIP: {
				tqb::FusedOp f{};
				f.kind = tqb::kFFlip;
				f.state = op.state;
				pass.ops.push_back(f);
				pending.push_back(&op);
				chain_op = -1;
				return;
			}
			default: fail(TMFQS_ERR_LOGIC, "planner: unsupported op in fused pass");
		}
	}
};

// Validates one op in the register's order of checks (QuantumRegister
// methods, quantum_register.cpp:394-527; validateGateTargets,
// validation.h:53-80).
void validate_op(tmfqs_gpu_state *h, const tmfqs_op &op) {
	switch(op.kind) {
		case TMFQS_OP_H: validate_qubit(h, op.q0, "QuantumRegister::applyHadamard"); return;
		case TMFQS_OP_X: validate_qubit(h, op.q0, "QuantumRegister::applyPauliX"); return;
		case TMFQS_OP_CNOT: validate_two(h, op.q0, op.q1, "QuantumRegister::applyControlledNot"); return;
		case TMFQS_OP_CPHASE: validate_two(h, op.q0, op.q1, "QuantumRegister::applyControlledPhaseShift"); return;
		case TMFQS_OP_SWAP: validate_two(h, op.q0, op.q1, "QuantumRegister::applySwap"); return;
		case TMFQS_OP_PHASE_FLIP: validate_state(h, op.state, "QuantumRegister::applyPhaseFlipBasisState"); return;
		case TMFQS_OP_GATE: {
			if(op.k > h->n) fail(TMFQS_ERR_INVALID_ARGUMENT, "QuantumRegister::applyGate gate acts on more qubits than available");
			if(!op.matrix || (op.k && !op.qubits)) fail(TMFQS_ERR_INVALID_ARGUMENT, "QuantumRegister::applyGate null matrix or qubits");
			std::vector<bool> seen(h->n, false);
			for(unsigned i = 0; i < op.k; ++i) {
				validate_qubit(h, op.qubits[i], "QuantumRegister::applyGate");
				if(seen[op.qubits[i]]) fail(TMFQS_ERR_INVALID_ARGUMENT, "QuantumRegister::applyGate duplicate qubit index");
				seen[op.qubits[i]] = true;
			}
			if(op.k > 10) fail(TMFQS_ERR_INVALID_ARGUMENT, "applyGate: this device build applies gates on at most 10 qubits");
			return;
		}
		case TMFQS_OP_INVERSION:
			fail(TMFQS_ERR_INVALID_ARGUMENT, "apply_ops: inversion about the mean needs register state; use tmfqs_gpu_grover_run");
		default: fail(TMFQS_ERR_INVALID_ARGUMENT, "apply_ops: unknown operation kind");
	}
}

void run_gate(tmfqs_gpu_state *h, const double *matrix, const unsigned *qubits, unsigned k) {
	if(h->opt_tensor && tqb::tc_gate_supported(h->precision, h->n, k)) {
		std::vector<unsigned> tpos(k);
		for(unsigned i = 0; i < k; ++i) tpos[i] = bit_of(h, qubits[i]);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_tc_gate(ctx(h), h->amps, h->n, k, matrix, tpos.data(), h->dev_tc, h->dev_tc_bytes);
		}
		++h->stats.gate_passes;
		return;
	}
	const size_t dim = 1ull << k;
	const size_t mbytes = dim * dim * 16;
	ensure_dev_small(h, mbytes);
	check_cuda(cudaStreamSynchronize(h->stream), "gate staging sync");
	check_cuda(cudaMemcpyAsync(h->dev_small, matrix, mbytes, cudaMemcpyHostToDevice, h->stream), "gate matrix upload");
	std::vector<unsigned> tpos(k);
	for(unsigned i = 0; i < k; ++i) tpos[i] = bit_of(h, qubits[i]);
	{
		PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
		tqb::launch_gate(ctx(h), h->precision, h->amps, h->n, k, static_cast<const double *>(h->dev_small), tpos.data());
	}
	check_cuda(cudaStreamSynchronize(h->stream), "gate sync");
	++h->stats.gate_passes;
}

// A maximal run of >= 2 swaps on pairwise-disjoint qubits starting at i.
size_t swap_run(const tmfqs_op *ops, size_t i, size_t count) {
	uint64_t used = 0;
	size_t j = i;
	while(j < count && ops[j].kind == TMFQS_OP_SWAP && ops[j].q0 != ops[j].q1 && ops[j].q0 < 64 && ops[j].q1 < 64) {
		const uint64_t m = (1ull << ops[j].q0) | (1ull << ops[j].q1);
		if(used & m) break;
		used |= m;
		++j;
	}
	return j - i;
}

// ---- QuantumRegister arithmetic on the host (quantum_register.cpp:21-57) ----
struct Cx {
	double re, im;
};
Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
Cx csub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
Cx cneg(Cx a) { return {-a.re, -a.im}; }
Cx cscale(Cx a, double s) { return {a.re * s, a.im * s}; }
Cx cmul(Cx l, Cx r) { return {l.re * r.re - l.im * r.im, l.re * r.im + l.im * r.re}; }
Cx cdiv(Cx n, Cx d) {
	const double q = d.re * d.re + d.im * d.im;
	if(q == 0.0) fail(TMFQS_ERR_LOGIC, "QuantumRegister affine overlay scale is zero");
	return {(n.re * d.re + n.im * d.im) / q, (n.im * d.re - n.re * d.im) / q};
}

Cx overlay_apply(const tmfqs_register_view &v, Cx a) {
	if(!v.overlay) return a;
	return cadd(cmul({v.scale_re, v.scale_im}, a), {v.bias_re, v.bias_im});
}
Cx overlay_remove(const tmfqs_register_view &v, Cx l) {
	if(!v.overlay) return l;
	return cdiv(csub(l, {v.bias_re, v.bias_im}), {v.scale_re, v.scale_im});
}

// Logical amplitude sum for the fast forms (complex64, or complex128 with
// TMFQS_OPT_EXACT off): one FP64 read pass, the overlay applied as
// scale * sum + N * bias.
Cx fast_logical_sum(tmfqs_gpu_state *h, const tmfqs_register_view &v) {
	const unsigned nb = tqb::sum_fast_blocks(ctx(h));
	ensure_dev_small(h, nb * sizeof(double2));
	if(h->pinned_elems < 2 * (size_t)nb) fail(TMFQS_ERR_LOGIC, "fast sum: pinned staging too small");
	tqb::launch_sum_fast(ctx(h), h->precision, h->amps, h->N, static_cast<double2 *>(h->dev_small));
	check_cuda(cudaMemcpyAsync(h->pinned, h->dev_small, nb * sizeof(double2), cudaMemcpyDeviceToHost, h->stream),
	           "fast sum read");
	check_cuda(cudaStreamSynchronize(h->stream), "fast sum sync");
	Cx sum{0.0, 0.0};
	for(unsigned b = 0; b < nb; ++b) {
		sum.re += h->pinned[2 * b];
		sum.im += h->pinned[2 * b + 1];
	}
	if(!v.overlay) return sum;
	return cadd(cmul({v.scale_re, v.scale_im}, sum), cscale({v.bias_re, v.bias_im}, (double)h->N));
}

// Exact logical amplitude sum (quantum_register.cpp:176-190); the fast forms
// take the one-pass FP64 sum.
Cx logical_sum(tmfqs_gpu_state *h, const tmfqs_register_view &v) {
	if(h->precision == TMFQS_FP32 || !h->opt_exact) return fast_logical_sum(h, v);
	tqb::Overlay ov;
	ov.active = v.overlay != 0;
	ov.sre = v.scale_re;
	ov.sim = v.scale_im;
	ov.bre = v.bias_re;
	ov.bim = v.bias_im;
	const double re = reduce(h, tqb::kTermReal, ov, false, 0.0).value;
	const double im = reduce(h, tqb::kTermImag, ov, false, 0.0).value;
	return {re, im};
}

// Device value a float-stored state holds after `tr - v` in float.
template <typename S>
S storage_sub(double t, S v) {
	return (S)t - v;
}

// Materialised Grover iterations with the register's semantics, all at once.
// closed = false (exact form): the means are computed here exactly as the
// register would, and the device replays every iteration per amplitude with
// its rounding (k_grover_temporal).  closed = true (fast forms): an unmarked
// amplitude follows a <- t_k - a, so after K iterations it is
// (-1)^K a_0 + S_K with S_K independent of the amplitude; the run becomes one
// affine sweep, with S_K and the marked amplitudes carried in FP64 and rounded
// once into the state.
template <typename S>
void grover_materialized_fused(tmfqs_gpu_state *h, tmfqs_register_view *view, const std::vector<uint64_t> &marked,
                               uint64_t iters, bool closed) {
	const double N = (double)h->N;
	uint64_t flip_from = 0;
	if(!view->has_sum) {
		// Iteration 0: flips without reads (no cached sum, no overlay), then
		// the exact logical sum of the flipped state.
		before_mutation(h);
		for(uint64_t s : marked) tqb::launch_phase_flip(ctx(h), h->precision, h->amps, s);
		const Cx sum = logical_sum(h, *view);
		view->has_sum = 1;
		view->sum_re = sum.re;
		view->sum_im = sum.im;
		flip_from = 1;
	}
	std::vector<double> vr(marked.size()), vi(marked.size());
	for(size_t q = 0; q < marked.size(); ++q) {
		const auto a = read_amp(h, marked[q]);
		vr[q] = a.first;
		vi[q] = a.second;
	}
	std::vector<double> tm(2 * iters);
	double sr = view->sum_re, si = view->sum_im;
	double bre = 0.0, bim = 0.0, sign = 1.0;  // closed form: a_K = sign * a_0 + b
	for(uint64_t k = 0; k < iters; ++k) {
		if(k >= flip_from) {
			for(size_t q = 0; q < marked.size(); ++q) {
				// applyPhaseFlipBasisState with a cached sum, no overlay (:408-419).
				sr -= 2.0 * (double)vr[q];
				si -= 2.0 * (double)vi[q];
				vr[q] = -vr[q];
				vi[q] = -vi[q];
			}
		}
		// applyInversionAboutMeanMaterialized() (:447-467).
		const double mr = sr / N, mi = si / N;
		sr = 2.0 * mr * N - sr;
		si = 2.0 * mi * N - si;
		tm[2 * k] = 2.0 * mr;
		tm[2 * k + 1] = 2.0 * mi;
		for(size_t q = 0; q < marked.size(); ++q) {
			if(closed) {
				vr[q] = tm[2 * k] - vr[q];
				vi[q] = tm[2 * k + 1] - vi[q];
			} else {
				vr[q] = (double)storage_sub<S>(tm[2 * k], (S)vr[q]);
				vi[q] = (double)storage_sub<S>(tm[2 * k + 1], (S)vi[q]);
			}
		}
		bre = tm[2 * k] - bre;
		bim = tm[2 * k + 1] - bim;
		sign = -sign;
	}
	before_mutation(h);
	if(closed) {
		{
			PassTimer timer(h, TMFQS_KT_GROVER, sweep_bytes(h));
			tqb::launch_affine(ctx(h), h->precision, h->amps, h->n, sign, 0.0, bre, bim);
		}
		++h->stats.fused_passes;
		view->sum_re = sr;
		view->sum_im = si;
		for(size_t q = 0; q < marked.size(); ++q) write_amp(h, marked[q], vr[q], vi[q]);
		return;
	}
	// The means in the storage type: the device rounds them exactly as the
	// per-iteration update `(S)t - v` above does.
	std::vector<S> tms(2 * iters);
	for(size_t i = 0; i < tms.size(); ++i) tms[i] = (S)tm[i];
	const size_t tm_bytes = iters * 2 * sizeof(S), mk_bytes = marked.size() * 8;
	const size_t off = (tm_bytes + 255) & ~size_t(255);
	ensure_dev_small(h, off + mk_bytes);
	check_cuda(cudaStreamSynchronize(h->stream), "grover staging sync");
	check_cuda(cudaMemcpyAsync(h->dev_small, tms.data(), tm_bytes, cudaMemcpyHostToDevice, h->stream), "grover means upload");
	check_cuda(cudaMemcpyAsync(static_cast<unsigned char *>(h->dev_small) + off, marked.data(), mk_bytes, cudaMemcpyHostToDevice, h->stream), "grover marked upload");
	PassTimer timer(h, TMFQS_KT_GROVER, sweep_bytes(h));
	tqb::launch_grover_temporal(ctx(h), h->precision, h->amps, h->n, h->dev_small, iters,
	                            reinterpret_cast<const uint64_t *>(static_cast<unsigned char *>(h->dev_small) + off),
	                            (unsigned)marked.size(), flip_from);
	check_cuda(cudaStreamSynchronize(h->stream), "grover sync");
	++h->stats.fused_passes;
	view->sum_re = sr;
	view->sum_im = si;
	for(size_t q = 0; q < marked.size(); ++q) h->cache[marked[q]] = {vr[q], vi[q]};
}

// One phase flip with register semantics (quantum_register.cpp:405-420).
void register_flip(tmfqs_gpu_state *h, tmfqs_register_view *v, uint64_t s) {
	if(v->has_sum || v->overlay) {
		const auto b = read_amp(h, s);
		const Cx logical = overlay_apply(*v, {b.first, b.second});
		if(v->has_sum) {
			v->sum_re -= 2.0 * logical.re;
			v->sum_im -= 2.0 * logical.im;
		}
		if(v->overlay) {
			const Cx nb = overlay_remove(*v, cneg(logical));
			carry_amp(h, s, nb.re, nb.im);
			return;
		}
	}
	auto it = h->cache.find(s);
	if(it != h->cache.end()) {
		carry_amp(h, s, -it->second.first, -it->second.second);
		return;
	}
	flush_dirty(h);
	tqb::launch_phase_flip(ctx(h), h->precision, h->amps, s);
}

// applyInversionAboutMean[Materialized]() with register semantics (:423-467).
void register_inversion(tmfqs_gpu_state *h, tmfqs_register_view *v, bool materialized) {
	if(!v->has_sum) {
		const Cx s = logical_sum(h, *v);
		v->has_sum = 1;
		v->sum_re = s.re;
		v->sum_im = s.im;
	}
	const double N = (double)h->N;
	const Cx mean{v->sum_re / N, v->sum_im / N};
	v->sum_re = 2.0 * mean.re * N - v->sum_re;
	v->sum_im = 2.0 * mean.im * N - v->sum_im;
	if(materialized) {
		if(v->overlay) {
			before_mutation(h);
			{
				PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
				tqb::launch_affine(ctx(h), h->precision, h->amps, h->n, v->scale_re, v->scale_im, v->bias_re, v->bias_im);
			}
			v->overlay = 0;
			v->scale_re = 1.0;
			v->scale_im = 0.0;
			v->bias_re = 0.0;
			v->bias_im = 0.0;
		}
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_inversion(ctx(h), h->precision, h->amps, h->n, 2.0 * mean.re, 2.0 * mean.im);
		}
		++h->stats.gate_passes;
		return;
	}
	const Cx scale = v->overlay ? Cx{v->scale_re, v->scale_im} : Cx{1.0, 0.0};
	const Cx bias = v->overlay ? Cx{v->bias_re, v->bias_im} : Cx{0.0, 0.0};
	const Cx ns = cneg(scale);
	const Cx nb = csub(cscale(mean, 2.0), bias);
	v->scale_re = ns.re;
	v->scale_im = ns.im;
	v->bias_re = nb.re;
	v->bias_im = nb.im;
	v->overlay = 1;
}

}  // namespace

// ===========================================================================
// Public entry points
// ---- dense-block fusion (complex64 handles, tensor cores) ----
// The qubits an op acts on, in its own order (first = most significant), and
// its matrix (row-major, complex); false for ops that cannot join a block.
bool op_as_matrix(const tmfqs_op &op, std::vector<unsigned> &qs, std::vector<std::complex<double>> &g) {
	typedef std::complex<double> C;
	switch(op.kind) {
		case TMFQS_OP_H: {
			const double inv = 1.0 / std::sqrt(2.0);  // dense_state_backend.cpp:258
			qs = {op.q0};
			g = {C(inv), C(inv), C(inv), C(-inv)};
			return true;
		}
		case TMFQS_OP_X:
			qs = {op.q0};
			g = {C(0), C(1), C(1), C(0)};
			return true;
		case TMFQS_OP_CNOT:
			qs = {op.q0, op.q1};
			g.assign(16, C(0));
			g[0] = g[5] = g[11] = g[14] = C(1);
			return true;
		case TMFQS_OP_CPHASE:
			qs = {op.q0, op.q1};
			g.assign(16, C(0));
			g[0] = g[5] = g[10] = C(1);
			g[15] = C(std::cos(op.theta), std::sin(op.theta));
			return true;
		case TMFQS_OP_SWAP:
			qs = {op.q0, op.q1};
			g.assign(16, C(0));
			g[0] = g[6] = g[9] = g[15] = C(1);
			return true;
		case TMFQS_OP_GATE: {
			if(op.k == 0 || op.k > 5) return false;
			qs.assign(op.qubits, op.qubits + op.k);
			const size_t dim = size_t(1) << op.k;
			g.resize(dim * dim);
			for(size_t e = 0; e < dim * dim; ++e) g[e] = C(op.matrix[2 * e], op.matrix[2 * e + 1]);
			return true;
		}
		default: return false;
	}
}

// Block fusion applies to the fast forms only: the block is multiplied out in
// FP64, which rounds differently from the reference's gate-by-gate products.
bool block_fusion(const tmfqs_gpu_state *h) { return h->precision == TMFQS_FP32 || !h->opt_exact; }

// The run of ops starting at ops[i] that acts within 5 qubits and that a
// block can take: its end (exclusive), and whether it holds a dense gate
// (MatrixGate) -- runs without one are left to the fused passes.
size_t dense_block_extent(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t i, size_t count, bool &has_gate) {
	std::vector<unsigned> Q;
	has_gate = false;
	size_t j = i;
	for(; j < count; ++j) {
		std::vector<unsigned> qs;
		std::vector<std::complex<double>> g;
		if(!op_as_matrix(ops[j], qs, g)) break;
		std::vector<unsigned> U = Q;
		for(unsigned q : qs)
			if(std::find(U.begin(), U.end(), q) == U.end()) U.push_back(q);
		if(U.size() > 5) break;
		Q = U;
		has_gate = has_gate || ops[j].kind == TMFQS_OP_GATE;
	}
	return j;
}

// Starting at ops[i], the longest run of ops acting within 5 qubits (holding
// a dense gate), multiplied in FP64 into one block matrix and applied in one
// sweep: a tensor-core gate for complex64 (padded to 4 qubits), the CUDA-core
// block kernel for the fast complex128 form.  Returns the number of ops
// consumed (0: no block).
size_t run_dense_block(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t i, size_t count) {
	typedef std::complex<double> C;
	if(!block_fusion(h)) return 0;
	bool has_gate = false;
	const size_t jend = dense_block_extent(h, ops, i, count, has_gate);
	if(!has_gate || jend - i < 2) return 0;
	std::vector<unsigned> Q;  // block qubits, block order (first = most significant)
	std::vector<std::pair<std::vector<unsigned>, std::vector<C>>> parts;
	size_t j = i;
	for(; j < jend; ++j) {
		std::vector<unsigned> qs;
		std::vector<C> g;
		op_as_matrix(ops[j], qs, g);
		validate_op(h, ops[j]);
		for(unsigned q : qs)
			if(std::find(Q.begin(), Q.end(), q) == Q.end()) Q.push_back(q);
		parts.push_back({qs, g});
	}
	const bool tensor = h->precision == TMFQS_FP32 && h->opt_tensor;
	if(tensor) {
		// Pad to 4 qubits with the highest-order unused ones (identity on them).
		for(unsigned q = 0; Q.size() < 4 && q < h->n; ++q)
			if(std::find(Q.begin(), Q.end(), q) == Q.end()) Q.push_back(q);
		if(!tqb::tc_gate_supported(h->precision, h->n, (unsigned)Q.size())) return 0;
	}
	const unsigned s = (unsigned)Q.size();
	const size_t d = size_t(1) << s;
	std::vector<C> M(d * d, C(0));
	for(size_t r = 0; r < d; ++r) M[r * d + r] = C(1);
	std::vector<C> T(d * d);
	for(const auto &pg : parts) {
		const std::vector<unsigned> &qs = pg.first;
		const std::vector<C> &g = pg.second;
		const unsigned t = (unsigned)qs.size();
		std::vector<unsigned> bitpos(t);  // block-index bit of each op qubit
		for(unsigned a = 0; a < t; ++a)
			bitpos[a] = s - 1 - (unsigned)(std::find(Q.begin(), Q.end(), qs[a]) - Q.begin());
		auto sub = [&](size_t r) {
			size_t v = 0;
			for(unsigned a = 0; a < t; ++a) v |= ((r >> bitpos[a]) & 1u) << (t - 1 - a);
			return v;
		};
		auto with = [&](size_t r, size_t v) {
			for(unsigned a = 0; a < t; ++a) {
				const size_t b = (v >> (t - 1 - a)) & 1u;
				r = (r & ~(size_t(1) << bitpos[a])) | (b << bitpos[a]);
			}
			return r;
		};
		// T = G (x) I . M
		const size_t td = size_t(1) << t;
		for(size_t r = 0; r < d; ++r) {
			const size_t rv = sub(r);
			for(size_t c = 0; c < d; ++c) {
				C acc(0);
				for(size_t v = 0; v < td; ++v) acc += g[rv * td + v] * M[with(r, v) * d + c];
				T[r * d + c] = acc;
			}
		}
		M.swap(T);
	}
	std::vector<double> mat(2 * d * d);
	for(size_t e = 0; e < d * d; ++e) {
		mat[2 * e] = M[e].real();
		mat[2 * e + 1] = M[e].imag();
	}
	h->cur_first = i;
	h->cur_count = (unsigned)(j - i);
	if(!tensor) {
		run_gate(h, mat.data(), Q.data(), s);
		return j - i;
	}
	std::vector<unsigned> tpos(s);
	for(unsigned a = 0; a < s; ++a) tpos[a] = bit_of(h, Q[a]);
	{
		PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
		tqb::launch_tc_gate(ctx(h), h->amps, h->n, s, mat.data(), tpos.data(), h->dev_tc, h->dev_tc_bytes);
	}
	++h->stats.gate_passes;
	return j - i;
}

// tmfqs_gpu_apply_ops: the Simulator's gate runs through the fusion planner.
// With sync false the passes are left in flight on the handle's stream (the
// caller synchronises and checks the device error word).  With `mirror` (a
// state-sized buffer), returns whether the batch's last launch was a radix
// pass that also wrote the final state there.
bool apply_ops_body(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t count, bool sync = true, void *mirror = nullptr) {
	ensure_initialized(h, "operation batch");
	if(count && !ops) fail(TMFQS_ERR_INVALID_ARGUMENT, "null op list");
	DeviceScope d(h);
	before_mutation(h);
	struct RangeReset {
		tmfqs_gpu_state *h;
		~RangeReset() {
			h->cur_first = 0;
			h->cur_count = 0;
		}
	} range_reset{h};
	if(!h->opt_fusion) {
		for(size_t i = 0; i < count; ++i) {
			validate_op(h, ops[i]);
			h->cur_first = i;
			h->cur_count = 1;
			Planner p(h);
			if(ops[i].kind == TMFQS_OP_GATE) run_gate(h, ops[i].matrix, ops[i].qubits, ops[i].k);
			else p.run_single(ops[i]);
		}
		if(sync) {
			check_cuda(cudaStreamSynchronize(h->stream), "apply_ops sync");
			check_device_error(h);
		}
		return false;
	}
	Planner p(h);
	p.base = ops;
	size_t i = 0;
	try {
		while(i < count) {
			const tmfqs_op &op = ops[i];
			validate_op(h, op);
			if(op.kind == TMFQS_OP_SWAP) {
				const size_t run = swap_run(ops, i, count);
				if(run >= 2) {
					for(size_t j = i; j < i + run; ++j) validate_op(h, ops[j]);
					p.flush();
					std::vector<std::pair<unsigned, unsigned>> pairs;
					for(size_t j = i; j < i + run; ++j) pairs.push_back({bit_of(h, ops[j].q0), bit_of(h, ops[j].q1)});
					h->cur_first = i;
					h->cur_count = (unsigned)run;
					{
						PassTimer timer(h, TMFQS_KT_PERMUTE, sweep_bytes(h));
						tqb::launch_bit_permutation(ctx(h), h->precision, h->amps, h->n, pairs);
					}
					++h->stats.fused_passes;
					i += run;
					continue;
				}
			}
			if(op.kind == TMFQS_OP_GATE) {
				p.flush();
				h->cur_first = i;
				h->cur_count = 1;
				// A dense gate and the ops after it that stay within 5 qubits: one block sweep.
				const size_t used = run_dense_block(h, ops, i, count);
				if(used) {
					i += used;
					continue;
				}
				run_gate(h, op.matrix, op.qubits, op.k);
				++i;
				continue;
			}
			if(block_fusion(h)) {
				// Gates that lead into a dense gate within the same 5 qubits join its block.
				bool has_gate = false;
				const size_t jend = dense_block_extent(h, ops, i, count, has_gate);
				if(has_gate && jend - i >= 2) {
					validate_op(h, op);
					p.flush();
					const size_t used = run_dense_block(h, ops, i, count);
					if(used) {
						i += used;
						continue;
					}
				}
			}
			p.add(op);
			++i;
		}
		p.mirror = mirror;
		p.flush();
		p.mirror = nullptr;
	} catch(const tqb::Error &) {
		// Ops before the failing one are applied, as in the reference's
		// sequential loop (simulator.cpp:72-82).
		p.mirror = nullptr;
		p.flush();
		throw;
	}
	if(sync) {
		check_cuda(cudaStreamSynchronize(h->stream), "apply_ops sync");
		check_device_error(h);
	}
	return p.mirrored;
}

// tmfqs_gpu_load_apply_ops: loadAmplitudes followed by a batch, with the
// host-to-device copy overlapped with the batch's first pass.  The first pass
// is formed as the planner would form it (a dry run); when it is an exact
// complex128 fused pass whose top four outer bits are consecutive, the state
// is copied in 16 slabs -- the slab of value v holds the amplitudes whose top
// outer bits are v: rows of 2^p contiguous amplitudes, one per value of the
// bits above them (one cudaMemcpy2DAsync) -- on a copy stream, and the pass
// runs each slab's tiles as soon as that slab has landed.  The rest of the
// batch runs as tmfqs_gpu_apply_ops.  Anything else (other forms, an invalid
// op, a batch that does not start with a fused pass) takes the plain path:
// load, then apply -- with the same results and errors.
void load_apply_ops_body(tmfqs_gpu_state *h, unsigned n, const double *host, const tmfqs_op *ops, size_t count) {
	require_handle(h);
	if(!host) fail(TMFQS_ERR_INVALID_ARGUMENT, "null amplitude buffer");
	if(count && !ops) fail(TMFQS_ERR_INVALID_ARGUMENT, "null op list");
	DeviceScope d(h);
	auto plain = [&] {
		ensure_state(h, n);
		h->cache.clear();
		h->dirty.clear();
		copy_in(h, 0, host, h->N);
		h->initialized = true;
		apply_ops_body(h, ops, count);
	};
	if(h->precision != TMFQS_FP64 || !h->opt_exact || !h->opt_fusion || count < 2) return plain();
	ensure_state(h, n);
	h->cache.clear();
	h->dirty.clear();
	h->initialized = false;
	try {
		for(size_t i = 0; i < count; ++i) validate_op(h, ops[i]);
	} catch(const tqb::Error &) {
		return plain();  // the plain path applies the ops before the invalid one, then reports it
	}
	Planner p(h);
	p.dry = true;
	for(size_t i = 0; i < count && !p.dry_done; ++i) {
		const tmfqs_op &op = ops[i];
		if(op.kind != TMFQS_OP_H && op.kind != TMFQS_OP_X && op.kind != TMFQS_OP_CNOT && op.kind != TMFQS_OP_CPHASE &&
		   op.kind != TMFQS_OP_PHASE_FLIP)
			break;
		p.add(op);
	}
	if(!p.dry_done) p.flush();
	const size_t k = p.dry_ops;
	tqb::FusedPass fp = p.dry_pass;
	// The pass's outer bits, ascending (tile index bit i is outer bit i).
	std::vector<unsigned> outer;
	for(unsigned b = 0; b < n; ++b)
		if(std::find(fp.lpos, fp.lpos + fp.K, b) == fp.lpos + fp.K) outer.push_back(b);
	constexpr unsigned t = 4;
	const unsigned nout = (unsigned)outer.size();
	if(k < 2 || nout < t + 1 || outer[nout - 1] - outer[nout - t] != t - 1) {
		h->initialized = true;  // state allocated; plain() loads it
		return plain();
	}
	const unsigned pbit = outer[nout - t];
	if(!h->copy_stream) check_cuda(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "copy stream");
	const size_t width = (size_t(16) << pbit), pitch = (size_t(16) << (pbit + t)), height = size_t(1) << (n - pbit - t);
	const unsigned slabs = 1u << t;
	std::vector<cudaEvent_t> ev(slabs, nullptr);
	struct Events {
		std::vector<cudaEvent_t> &e;
		~Events() {
			for(cudaEvent_t x : e)
				if(x) cudaEventDestroy(x);
		}
	} events{ev};
	// The copy stream must not overwrite the state while earlier work on the handle's stream still reads it.
	cudaEvent_t ready = nullptr;
	check_cuda(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event");
	check_cuda(cudaEventRecord(ready, h->stream), "event record");
	check_cuda(cudaStreamWaitEvent(h->copy_stream, ready, 0), "copy stream wait");
	cudaEventDestroy(ready);
	h->initialized = true;
	h->cur_first = 0;
	h->cur_count = (unsigned)k;
	// The slabs' launches share one program: upload it now, ahead of the slab
	// copies (on the same copy engine a later upload would queue behind them).
	fp.program_ready = tqb::prepare_fused_pass(ctx(h), h->precision, fp, h->dev_prog, h->dev_prog_bytes);
	const uint64_t per = (1ull << (nout - t));
	for(unsigned v = 0; v < slabs; ++v) {
		unsigned char *dst = static_cast<unsigned char *>(h->amps) + (size_t(v) << pbit) * 16;
		const unsigned char *src = reinterpret_cast<const unsigned char *>(host) + (size_t(v) << pbit) * 16;
		check_cuda(cudaMemcpy2DAsync(dst, pitch, src, pitch, width, height, cudaMemcpyHostToDevice, h->copy_stream),
		           "slab copy");
		check_cuda(cudaEventCreateWithFlags(&ev[v], cudaEventDisableTiming), "event");
		check_cuda(cudaEventRecord(ev[v], h->copy_stream), "event record");
		check_cuda(cudaStreamWaitEvent(h->stream, ev[v], 0), "slab wait");
		fp.tile_begin = v * per;
		fp.tile_end = (v + 1) * per;
		PassTimer timer(h, TMFQS_KT_FUSED, sweep_bytes(h) / slabs);
		tqb::launch_fused_pass(ctx(h), h->precision, h->amps, fp, h->dev_prog, h->dev_prog_bytes);
	}
	h->stats.h2d_bytes += h->N * 16;
	++h->stats.fused_passes;
	h->cur_count = 0;
	if(k < count) {
		apply_ops_body(h, ops + k, count - k);
	} else {
		check_cuda(cudaStreamSynchronize(h->stream), "load_apply_ops sync");
		check_device_error(h);
	}
}

// ---- adjoint gradient (tmfqs_gpu_adjoint_gradient) ----
// A work handle of `h` (kept in *w between calls) with h's options and a state
// of h->n qubits; without a state buffer of its own when `with_state` is false
// (the caller points it at one).
tmfqs_gpu_state *work_handle(tmfqs_gpu_state *h, tmfqs_gpu_state *&w, bool with_state = true) {
	if(!w) {
		const int rc = tmfqs_gpu_create(h->precision, h->device, &w);
		if(rc) throw tqb::Error{rc, g_last_error};
	}
	w->opt_fusion = h->opt_fusion;
	w->opt_fused_qubits = h->opt_fused_qubits;
	w->opt_exact = h->opt_exact;
	w->opt_radix = h->opt_radix;
	w->opt_qft_pass = h->opt_qft_pass;
	if(with_state) {
		ensure_state(w, h->n);
	} else {
		if(w->amps) {
			check_cuda(cudaStreamSynchronize(w->stream), "sync before free");
			cudaFree(w->amps);
			w->amps = nullptr;
		}
		tqb::seq_scratch_free(w->seq);
		w->bytes = amp_bytes(w) << h->n;
		w->n = h->n;
		w->N = 1ull << h->n;
	}
	w->initialized = true;
	return w;
}

// Releases the adjoint work buffers of a handle.
void free_adjoint_buffers(tmfqs_gpu_state *h) {
	if(h->adj_ckpt) cudaFree(h->adj_ckpt);
	if(h->adj_part) cudaFree(h->adj_part);
	h->adj_ckpt = h->adj_part = nullptr;
	h->adj_ckpt_bytes = 0;
	if(h->adj_lam) tmfqs_gpu_destroy(h->adj_lam);
	if(h->adj_psi) tmfqs_gpu_destroy(h->adj_psi);
	h->adj_lam = h->adj_psi = nullptr;
}

bool is_diagonal_op(const tmfqs_op &op) { return op.kind == TMFQS_OP_CPHASE || op.kind == TMFQS_OP_PHASE_FLIP; }

// The work handles of an adjoint call run on the caller's stream for the
// duration of the call, so one stream orders every pass and no host waits
// are needed between them.  Their own streams and state buffers (psi works
// in place on the checkpoints) come back on exit.
struct StreamBorrow {
	tmfqs_gpu_state *owner;
	tmfqs_gpu_state *w[2];
	cudaStream_t saved[2];
	void *amps[2];
	StreamBorrow(tmfqs_gpu_state *h, tmfqs_gpu_state *a, tmfqs_gpu_state *b)
	    : owner(h), w{a, b}, saved{a->stream, b->stream}, amps{a->amps, b->amps} {
		a->stream = b->stream = h->stream;
	}
	~StreamBorrow() {
		cudaStreamSynchronize(owner->stream);
		for(int i = 0; i < 2; ++i) {
			w[i]->stream = saved[i];
			w[i]->amps = amps[i];
		}
	}
};

// Gradient partial sums kept on the device: each launch writes its own array
// of the handle's scratch, and one reduction and one read serve them all (or
// every kMaxPendingSums arrays, when a circuit has more diagonal runs).
class PendingSums {
public:
	struct Use {
		bool obs;                    // the expectation (column 0)
		std::vector<size_t> col_op;  // gradient pass: the op of each column
	};
	PendingSums(tmfqs_gpu_state *h, double *part, size_t chunk_doubles, double *out, const tmfqs_op *ops,
	            const std::vector<size_t> &param_of, double *expectation, double *grads)
	    : h_(h), part_(part), chunk_(chunk_doubles), out_(out), ops_(ops), param_of_(param_of), expectation_(expectation),
	      grads_(grads) {
		tab_.count = 0;
	}
	// Scratch for the next launch's partials (flushing first when full).
	double *next() {
		if(tab_.count == tqb::kMaxPendingSums) flush();
		return part_ + (size_t)tab_.count * chunk_;
	}
	void add(unsigned blocks, unsigned stride, Use u) {
		tab_.blocks[tab_.count] = blocks;
		tab_.stride[tab_.count] = stride;
		uses_.push_back(std::move(u));
		++tab_.count;
	}
	void flush() {
		if(!tab_.count) return;
		tqb::launch_sum_partials(ctx(h_), part_, chunk_, tab_, out_);
		std::vector<double> host((size_t)tab_.count * tqb::kMaxDiagRun);
		check_cuda(cudaMemcpyAsync(host.data(), out_, host.size() * sizeof(double), cudaMemcpyDeviceToHost, h_->stream),
		           "partials read");
		check_cuda(cudaStreamSynchronize(h_->stream), "partials sync");
		for(unsigned c = 0; c < tab_.count; ++c) {
			const double *g = host.data() + (size_t)c * tqb::kMaxDiagRun;
			const Use &u = uses_[c];
			if(u.obs) *expectation_ = g[0];
			for(size_t col = 0; col < u.col_op.size(); ++col) {
				const size_t k = u.col_op[col];
				if(ops_[k].kind == TMFQS_OP_CPHASE) grads_[param_of_[k]] = 2.0 * g[col];
			}
		}
		tab_.count = 0;
		uses_.clear();
	}

private:
	tmfqs_gpu_state *h_;
	double *part_;
	size_t chunk_;
	double *out_;
	const tmfqs_op *ops_;
	const std::vector<size_t> &param_of_;
	double *expectation_, *grads_;
	tqb::PartialChunks tab_;
	std::vector<Use> uses_;
};

void adjoint_gradient(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t count, const uint64_t *masks,
                      const double *weights, unsigned terms, size_t every, double *expectation, double *grads) {
	ensure_initialized(h, "adjoint gradient");
	if(count && !ops) fail(TMFQS_ERR_INVALID_ARGUMENT, "null op list");
	if(!expectation) fail(TMFQS_ERR_INVALID_ARGUMENT, "null expectation output");
	if(terms == 0 || terms > tqb::kMaxObsTerms) fail(TMFQS_ERR_INVALID_ARGUMENT, "observable: 1 to 64 terms");
	if(!masks || !weights) fail(TMFQS_ERR_INVALID_ARGUMENT, "null observable");
	for(unsigned j = 0; j < terms; ++j)
		if(h->n < 64 && (masks[j] >> h->n) != 0) fail(TMFQS_ERR_OUT_OF_RANGE, "observable mask beyond the register");
	std::vector<size_t> param_of(count, 0);
	size_t nparams = 0;
	for(size_t i = 0; i < count; ++i) {
		if(ops[i].kind == TMFQS_OP_INVERSION) fail(TMFQS_ERR_INVALID_ARGUMENT, "adjoint gradient: inversion about the mean is not supported");
		validate_op(h, ops[i]);
		if(ops[i].kind == TMFQS_OP_CPHASE) param_of[i] = nparams++;
	}
	if(nparams && !grads) fail(TMFQS_ERR_INVALID_ARGUMENT, "null gradient output");
	DeviceScope d(h);
	before_mutation(h);
	const size_t bytes = h->bytes;
	size_t K = every;
	if(K == 0) {
		size_t freeb = 0, totalb = 0;
		check_cuda(cudaMemGetInfo(&freeb, &totalb), "free memory");
		const size_t cap = std::max<size_t>(1, (freeb / 2) / bytes);
		K = std::max<size_t>(1, (count + cap - 1) / cap);
	}
	const size_t nseg = count ? (count + K - 1) / K : 0;
	if(h->adj_ckpt_bytes < nseg * bytes) {
		check_cuda(cudaStreamSynchronize(h->stream), "checkpoint sync");
		if(h->adj_ckpt) cudaFree(h->adj_ckpt);
		h->adj_ckpt = nullptr;
		h->adj_ckpt_bytes = 0;
		if(tqb::device_alloc((void **)&h->adj_ckpt, nseg * bytes) != cudaSuccess) {
			cudaGetLastError();
			h->adj_ckpt = nullptr;
			fail(TMFQS_ERR_NOMEM, "adjoint gradient: checkpoint allocation failed (raise checkpoint_every)");
		}
		h->adj_ckpt_bytes = nseg * bytes;
	}
	// Scratch: kMaxPendingSums partial arrays of the largest launch, then the
	// reduced sums.
	const size_t chunk = (size_t)tqb::adjoint_max_blocks(h->num_sms) * tqb::kMaxDiagRun;
	if(!h->adj_part &&
	   tqb::device_alloc((void **)&h->adj_part, (chunk * tqb::kMaxPendingSums + tqb::kMaxPendingSums * tqb::kMaxDiagRun) * sizeof(double)) !=
	       cudaSuccess) {
		cudaGetLastError();
		h->adj_part = nullptr;
		fail(TMFQS_ERR_NOMEM, "adjoint gradient: scratch allocation failed");
	}
	unsigned char *ckb = static_cast<unsigned char *>(h->adj_ckpt);
	double *part = static_cast<double *>(h->adj_part);
	PendingSums sums(h, part, chunk, part + chunk * tqb::kMaxPendingSums, ops, param_of, expectation, grads);

	struct {
		tmfqs_gpu_state *h;
	} lam{work_handle(h, h->adj_lam)}, psi{work_handle(h, h->adj_psi, false)};
	StreamBorrow borrow(h, lam.h, psi.h);

	// Forward pass, with psi saved after every segment of K ops.
	for(size_t sidx = 0; sidx < nseg; ++sidx) {
		const size_t a0 = sidx * K, len = std::min(K, count - a0);
		// The segment's last pass writes the checkpoint as well when it is a
		// radix pass; otherwise the state is copied.
		if(!apply_ops_body(h, ops + a0, len, false, ckb + sidx * bytes))
			check_cuda(cudaMemcpyAsync(ckb + sidx * bytes, h->amps, bytes, cudaMemcpyDeviceToDevice, h->stream), "checkpoint");
	}

	{
		PassTimer timer(h, TMFQS_KT_ADJOINT, sweep_bytes(h));
		double *dst = sums.next();
		const unsigned blocks =
		    tqb::launch_obs_apply(ctx(h), h->precision, h->amps, lam.h->amps, h->n, masks, weights, terms, dst);
		sums.add(blocks, 1, {true, {}});
	}

	// Backward pass: segment by segment, psi taken from its checkpoint.
	for(size_t sidx = nseg; sidx-- > 0;) {
		const size_t a0 = sidx * K, b0 = std::min(count, a0 + K);
		// cp_before[i - a0]: a controlled phase lies in [a0, i).
		std::vector<char> cp_before(b0 - a0 + 1, 0);
		for(size_t i = a0; i < b0; ++i) cp_before[i - a0 + 1] = cp_before[i - a0] || ops[i].kind == TMFQS_OP_CPHASE;
		// psi = the state after the segment: its checkpoint, used in place (each
		// checkpoint is read by one segment only).
		psi.h->amps = ckb + sidx * bytes;
		size_t i = b0;
		while(i > a0) {
			const bool diag = is_diagonal_op(ops[i - 1]);
			size_t j = i;
			while(j > a0 && is_diagonal_op(ops[j - 1]) == diag) --j;  // the run [j, i)
			if(diag) {
				for(size_t e = i; e > j;) {
					const size_t st = std::max(j, e > tqb::kMaxDiagRun ? e - tqb::kMaxDiagRun : 0);
					// Entries that depend on the three lowest index bits (flips, and
					// phases with a mask bit there) first: the gradient pass then
					// looks up one phase table per amplitude when they fit in 8.
					std::vector<tqb::DiagEntry> ent;
					std::vector<size_t> col_op;
					for(int low = 1; low >= 0; --low)
						for(size_t k = st; k < e; ++k) {
							const tmfqs_op &op = ops[k];
							tqb::DiagEntry d;
							if(op.kind == TMFQS_OP_CPHASE)
								d = {tqb::kDiagCPhase, (1ull << bit_of(h, op.q0)) | (1ull << bit_of(h, op.q1)), std::cos(op.theta),
								     std::sin(op.theta)};
							else
								d = {tqb::kDiagFlip, op.state, 1.0, 0.0};
							if((d.kind == tqb::kDiagFlip || (d.mask & 7u)) != (low == 1)) continue;
							ent.push_back(d);
							col_op.push_back(k);
						}
					const bool need_psi = cp_before[st - a0] != 0;
					{
						PassTimer timer(h, TMFQS_KT_ADJOINT, sweep_bytes(h) * (need_psi ? 2.0 : 1.5));
						double *dst = sums.next();
						const unsigned blocks = tqb::launch_grad_run(ctx(h), h->precision, lam.h->amps, psi.h->amps, h->n,
						                                             ent.data(), (unsigned)ent.size(), need_psi, dst);
						sums.add(blocks, tqb::kMaxDiagRun, {false, std::move(col_op)});
					}
					e = st;
				}
			} else {
				// Inverse of the run, last op first.  A run of Hadamards and X gates
				// on distinct qubits commutes and each op is its own inverse: it is
				// un-applied in circuit order, which the planner packs into the same
				// passes as the forward (a layer's Hadamards from the top qubit down).
				bool commuting = true;
				uint64_t seen = 0;
				for(size_t k = j; k < i && commuting; ++k) {
					const tmfqs_op &op = ops[k];
					const uint64_t q = 1ull << bit_of(h, op.q0);
					commuting = (op.kind == TMFQS_OP_H || op.kind == TMFQS_OP_X) && !(seen & q);
					seen |= q;
				}
				std::vector<tmfqs_op> inv;
				std::vector<std::vector<double>> mats;
				for(size_t s = 0; s < i - j; ++s) {
					const size_t k = commuting ? j + s : i - 1 - s;
					tmfqs_op op = ops[k];
					if(op.kind == TMFQS_OP_GATE) {
						const size_t dim = size_t(1) << op.k;
						std::vector<double> m(2 * dim * dim);
						for(size_t r = 0; r < dim; ++r)
							for(size_t c = 0; c < dim; ++c) {
								m[2 * (r * dim + c)] = op.matrix[2 * (c * dim + r)];
								m[2 * (r * dim + c) + 1] = -op.matrix[2 * (c * dim + r) + 1];
							}
						mats.push_back(std::move(m));
						op.matrix = mats.back().data();
					}
					inv.push_back(op);
				}
				apply_ops_body(lam.h, inv.data(), inv.size(), false);
				if(cp_before[j - a0]) apply_ops_body(psi.h, inv.data(), inv.size(), false);
			}
			i = j;
		}
	}
	sums.flush();
	check_cuda(cudaStreamSynchronize(h->stream), "backward sync");
	check_device_error(h);
	check_device_error(lam.h);
	check_device_error(psi.h);
}

// ===========================================================================
extern "C" {

const char *tmfqs_gpu_last_error(void) { return g_last_error.c_str(); }

int tmfqs_gpu_create(int precision, int device, tmfqs_gpu_state **out) {
	return guarded([&] {
		if(!out) fail(TMFQS_ERR_INVALID_ARGUMENT, "null output handle");
		*out = nullptr;
		if(precision != TMFQS_FP64 && precision != TMFQS_FP32) fail(TMFQS_ERR_INVALID_ARGUMENT, "unknown precision");
		int count = 0;
		const cudaError_t e = cudaGetDeviceCount(&count);
		if(e != cudaSuccess || count == 0) {
			cudaGetLastError();
			fail(TMFQS_ERR_CUDA, "no CUDA device available for the gpu storage strategy");
		}
		if(device < 0 || device >= count) fail(TMFQS_ERR_INVALID_ARGUMENT, "device ordinal out of range");
		auto *h = new tmfqs_gpu_state();
		h->device = device;
		h->precision = precision;
		try {
			check_cuda(cudaSetDevice(device), "cudaSetDevice");
			check_cuda(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device), "SM count");
			check_cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream create");
			if(cudaMallocHost(&h->pinned, kPinnedElems * sizeof(double)) != cudaSuccess) {
				cudaGetLastError();
				fail(TMFQS_ERR_NOMEM, "pinned staging allocation failed");
			}
			h->pinned_elems = kPinnedElems;
			if(cudaHostAlloc(&h->err_host, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
			   cudaHostGetDevicePointer(&h->err_dev, h->err_host, 0) != cudaSuccess) {
				cudaGetLastError();
				fail(TMFQS_ERR_NOMEM, "pinned error word allocation failed");
			}
			*h->err_host = 0;
			if(cudaMallocHost(&h->ring.host, tqb::UploadRing::kSlots * tqb::UploadRing::kSlotBytes) != cudaSuccess) {
				cudaGetLastError();
				h->ring.host = nullptr;  // uploads fall back to synchronous copies
			}
			for(unsigned k = 0; k < tqb::UploadRing::kSlots; ++k)
				check_cuda(cudaEventCreateWithFlags(&h->ring.ev[k], cudaEventDisableTiming), "upload event");
		} catch(...) {
			for(unsigned k = 0; k < tqb::UploadRing::kSlots; ++k)
				if(h->ring.ev[k]) cudaEventDestroy(h->ring.ev[k]);
			if(h->ring.host) cudaFreeHost(h->ring.host);
			if(h->err_host) cudaFreeHost(h->err_host);
			if(h->pinned) cudaFreeHost(h->pinned);
			if(h->stream) cudaStreamDestroy(h->stream);
			delete h;
			throw;
		}
		*out = h;
	});
}

int tmfqs_gpu_destroy(tmfqs_gpu_state *h) {
	if(!h) return TMFQS_OK;
	return guarded([&] {
		cudaSetDevice(h->device);
		if(h->stream) cudaStreamSynchronize(h->stream);
		for(auto &t : h->timed) {
			cudaEventDestroy(t.start);
			cudaEventDestroy(t.stop);
		}
		tqb::seq_scratch_free(h->seq);
		free_adjoint_buffers(h);
		if(h->dev_tc) cudaFree(h->dev_tc);
		if(h->amps) cudaFree(h->amps);
		if(h->dev_small) cudaFree(h->dev_small);
		if(h->dev_prog) cudaFree(h->dev_prog);
		if(h->pinned) cudaFreeHost(h->pinned);
		if(h->err_host) cudaFreeHost(h->err_host);
		for(unsigned k = 0; k < tqb::UploadRing::kSlots; ++k)
			if(h->ring.ev[k]) cudaEventDestroy(h->ring.ev[k]);
		if(h->ring.host) cudaFreeHost(h->ring.host);
		if(h->copy_stream) {
			cudaStreamSynchronize(h->copy_stream);
			cudaStreamDestroy(h->copy_stream);
		}
		if(h->stream) cudaStreamDestroy(h->stream);
		delete h;
	});
}

int tmfqs_gpu_clone(tmfqs_gpu_state *h, tmfqs_gpu_state **out) {
	return guarded([&] {
		require_handle(h);
		if(!out) fail(TMFQS_ERR_INVALID_ARGUMENT, "null output handle");
		tmfqs_gpu_state *c = nullptr;
		const int rc = tmfqs_gpu_create(h->precision, h->device, &c);
		if(rc) throw tqb::Error{rc, g_last_error};
		try {
			DeviceScope d(h);
			c->opt_fusion = h->opt_fusion;
			c->opt_fused_qubits = h->opt_fused_qubits;
			c->opt_grover_fusion = h->opt_grover_fusion;
			c->opt_exact = h->opt_exact;
			c->opt_radix = h->opt_radix;
			c->opt_tensor = h->opt_tensor;
			c->opt_qft_pass = h->opt_qft_pass;
			if(h->initialized) {
				flush_dirty(h);
				ensure_state(c, h->n);
				check_cuda(cudaStreamSynchronize(h->stream), "clone sync");
				check_cuda(cudaMemcpyAsync(c->amps, h->amps, h->bytes, cudaMemcpyDeviceToDevice, c->stream), "clone copy");
				check_cuda(cudaStreamSynchronize(c->stream), "clone copy sync");
				c->initialized = true;
			}
		} catch(...) {
			tmfqs_gpu_destroy(c);
			throw;
		}
		*out = c;
	});
}

int tmfqs_gpu_init_zero(tmfqs_gpu_state *h, unsigned n) {
	return guarded([&] {
		require_handle(h);
		DeviceScope d(h);
		ensure_state(h, n);
		h->cache.clear();
		h->dirty.clear();
		check_cuda(cudaMemsetAsync(h->amps, 0, h->bytes, h->stream), "init zero");
		h->initialized = true;
	});
}

int tmfqs_gpu_init_basis(tmfqs_gpu_state *h, unsigned n, uint64_t s, double re, double im) {
	return guarded([&] {
		require_handle(h);
		if(n <= kMaxQubits && s >= (1ull << n)) fail(TMFQS_ERR_OUT_OF_RANGE, "GpuStateBackend::initBasis state index out of range");
		DeviceScope d(h);
		ensure_state(h, n);
		h->cache.clear();
		h->dirty.clear();
		check_cuda(cudaMemsetAsync(h->amps, 0, h->bytes, h->stream), "init basis");
		h->initialized = true;
		write_amp(h, s, re, im);
		flush_dirty(h);
	});
}

int tmfqs_gpu_init_uniform(tmfqs_gpu_state *h, unsigned n, const uint64_t *states, size_t count) {
	return guarded([&] {
		require_handle(h);
		if(n > kMaxQubits) fail(TMFQS_ERR_INVALID_ARGUMENT, "Number of qubits exceeds supported range for this device build");
		if(count && !states) fail(TMFQS_ERR_INVALID_ARGUMENT, "null state list");
		std::vector<uint64_t> sel(states, states + count);
		for(uint64_t s : sel)
			if(s >= (1ull << n)) fail(TMFQS_ERR_OUT_OF_RANGE, "GpuStateBackend::initUniformSuperposition state index out of range");
		std::sort(sel.begin(), sel.end());
		sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
		if(sel.empty()) fail(TMFQS_ERR_INVALID_ARGUMENT, "GpuStateBackend::initUniformSuperposition requires at least one state");
		DeviceScope d(h);
		ensure_state(h, n);
		h->cache.clear();
		h->dirty.clear();
		check_cuda(cudaMemsetAsync(h->amps, 0, h->bytes, h->stream), "init uniform");
		const double amp = 1.0 / std::sqrt(static_cast<double>(sel.size()));  // dense_state_backend.cpp:110
		const uint64_t chunk = 1ull << 20;
		ensure_dev_small(h, chunk * 8);
		for(uint64_t off = 0; off < sel.size(); off += chunk) {
			const uint64_t c = std::min<uint64_t>(chunk, sel.size() - off);
			check_cuda(cudaStreamSynchronize(h->stream), "uniform staging sync");
			check_cuda(cudaMemcpyAsync(h->dev_small, sel.data() + off, c * 8, cudaMemcpyHostToDevice, h->stream), "uniform upload");
			tqb::launch_scatter_uniform(ctx(h), h->precision, h->amps, static_cast<const uint64_t *>(h->dev_small), c, amp);
		}
		check_cuda(cudaStreamSynchronize(h->stream), "uniform sync");
		h->initialized = true;
	});
}

int tmfqs_gpu_load(tmfqs_gpu_state *h, unsigned n, const double *host) {
	return guarded([&] {
		require_handle(h);
		if(!host) fail(TMFQS_ERR_INVALID_ARGUMENT, "null amplitude buffer");
		DeviceScope d(h);
		ensure_state(h, n);
		h->cache.clear();
		h->dirty.clear();
		copy_in(h, 0, host, h->N);
		check_cuda(cudaStreamSynchronize(h->stream), "load sync");
		h->initialized = true;
	});
}

int tmfqs_gpu_load_chunk(tmfqs_gpu_state *h, uint64_t first, const double *host, uint64_t count) {
	return guarded([&] {
		ensure_initialized(h, "amplitude loading");
		if(!host && count) fail(TMFQS_ERR_INVALID_ARGUMENT, "null amplitude buffer");
		if(first > h->N || count > h->N - first) fail(TMFQS_ERR_OUT_OF_RANGE, "load_chunk range out of range");
		DeviceScope d(h);
		before_mutation(h);
		copy_in(h, first, host, count);
		check_cuda(cudaStreamSynchronize(h->stream), "load sync");
	});
}

int tmfqs_gpu_export(tmfqs_gpu_state *h, double *out) {
	return guarded([&] {
		ensure_initialized(h, "amplitude export");
		if(!out) fail(TMFQS_ERR_INVALID_ARGUMENT, "null output buffer");
		DeviceScope d(h);
		flush_dirty(h);
		copy_out(h, 0, out, h->N);
	});
}

int tmfqs_gpu_export_chunk(tmfqs_gpu_state *h, uint64_t first, double *out, uint64_t count) {
	return guarded([&] {
		ensure_initialized(h, "amplitude chunk iteration");
		if(!out && count) fail(TMFQS_ERR_INVALID_ARGUMENT, "null output buffer");
		if(first > h->N || count > h->N - first) fail(TMFQS_ERR_OUT_OF_RANGE, "export_chunk range out of range");
		DeviceScope d(h);
		flush_dirty(h);
		copy_out(h, first, out, count);
	});
}

int tmfqs_gpu_get_amp(tmfqs_gpu_state *h, uint64_t s, double *re, double *im) {
	return guarded([&] {
		ensure_initialized(h, "amplitude query");
		validate_state(h, s, "GpuStateBackend::amplitude");
		DeviceScope d(h);
		const auto v = read_amp(h, s);
		*re = v.first;
		*im = v.second;
	});
}

int tmfqs_gpu_set_amp(tmfqs_gpu_state *h, uint64_t s, double re, double im) {
	return guarded([&] {
		ensure_initialized(h, "state update");
		validate_state(h, s, "GpuStateBackend::setAmplitude");
		write_amp(h, s, re, im);
	});
}

int tmfqs_gpu_num_qubits(tmfqs_gpu_state *h, unsigned *out) {
	return guarded([&] {
		require_handle(h);
		*out = h->n;
	});
}

int tmfqs_gpu_precision(tmfqs_gpu_state *h, int *out) {
	return guarded([&] {
		require_handle(h);
		*out = h->precision;
	});
}

int tmfqs_gpu_total_probability(tmfqs_gpu_state *h, double *out) {
	return guarded([&] {
		ensure_initialized(h, "total probability query");
		DeviceScope d(h);
		*out = reduce(h, tqb::kTermProb, tqb::Overlay{}, false, 0.0).value;
	});
}

int tmfqs_gpu_sample(tmfqs_gpu_state *h, double rnd, uint64_t *out) {
	return guarded([&] {
		ensure_initialized(h, "measurement");
		if(!(rnd >= 0.0 && rnd < 1.0)) fail(TMFQS_ERR_INVALID_ARGUMENT, "GpuStateBackend::sampleMeasurement requires rnd in [0,1)");
		DeviceScope d(h);
		const tqb::SeqResult r = reduce(h, tqb::kTermProb, tqb::Overlay{}, true, rnd);
		if(r.index >= h->N) fail(TMFQS_ERR_RUNTIME, "GpuStateBackend::sampleMeasurement cumulative probability did not reach sample");
		*out = r.index;
	});
}

int tmfqs_gpu_amplitude_sum(tmfqs_gpu_state *h, double *re, double *im) {
	return guarded([&] {
		ensure_initialized(h, "amplitude sum");
		DeviceScope d(h);
		*re = reduce(h, tqb::kTermReal, tqb::Overlay{}, false, 0.0).value;
		*im = reduce(h, tqb::kTermImag, tqb::Overlay{}, false, 0.0).value;
	});
}

int tmfqs_gpu_overlay_sum(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim, double *re, double *im) {
	return guarded([&] {
		ensure_initialized(h, "amplitude sum");
		DeviceScope d(h);
		const tqb::Overlay ov{true, sre, sim, bre, bim};
		*re = reduce(h, tqb::kTermReal, ov, false, 0.0).value;
		*im = reduce(h, tqb::kTermImag, ov, false, 0.0).value;
	});
}

int tmfqs_gpu_overlay_total_probability(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim, double *out) {
	return guarded([&] {
		ensure_initialized(h, "probability summation");
		DeviceScope d(h);
		*out = reduce(h, tqb::kTermProb, tqb::Overlay{true, sre, sim, bre, bim}, false, 0.0).value;
	});
}

int tmfqs_gpu_overlay_sample(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim, double rnd, uint64_t *out) {
	return guarded([&] {
		ensure_initialized(h, "measurement");
		DeviceScope d(h);
		const tqb::SeqResult r = reduce(h, tqb::kTermProb, tqb::Overlay{true, sre, sim, bre, bim}, true, rnd);
		if(r.index >= h->N) fail(TMFQS_ERR_RUNTIME, "QuantumRegister::measure cumulative probability did not reach sample");
		*out = r.index;
	});
}

int tmfqs_gpu_phase_flip(tmfqs_gpu_state *h, uint64_t s) {
	return guarded([&] {
		ensure_initialized(h, "basis-state phase flip");
		validate_state(h, s, "GpuStateBackend::phaseFlipBasisState");
		DeviceScope d(h);
		auto it = h->cache.find(s);
		if(it != h->cache.end()) {
			write_amp(h, s, -it->second.first, -it->second.second);
			return;
		}
		flush_dirty(h);
		tqb::launch_phase_flip(ctx(h), h->precision, h->amps, s);
	});
}

int tmfqs_gpu_inversion_mean(tmfqs_gpu_state *h, double re, double im) {
	return guarded([&] {
		ensure_initialized(h, "inversion about mean");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_inversion(ctx(h), h->precision, h->amps, h->n, 2.0 * re, 2.0 * im);
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_inversion(tmfqs_gpu_state *h) {
	return guarded([&] {
		ensure_initialized(h, "inversion about mean");
		DeviceScope d(h);
		const double sr = reduce(h, tqb::kTermReal, tqb::Overlay{}, false, 0.0).value;
		const double si = reduce(h, tqb::kTermImag, tqb::Overlay{}, false, 0.0).value;
		const double N = (double)h->N;
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_inversion(ctx(h), h->precision, h->amps, h->n, 2.0 * (sr / N), 2.0 * (si / N));
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_affine(tmfqs_gpu_state *h, double sre, double sim, double bre, double bim) {
	return guarded([&] {
		ensure_initialized(h, "affine transform");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_affine(ctx(h), h->precision, h->amps, h->n, sre, sim, bre, bim);
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_h(tmfqs_gpu_state *h, unsigned q) {
	return guarded([&] {
		ensure_initialized(h, "DenseStateBackend::applyHadamard");
		validate_qubit(h, q, "GpuStateBackend::applyHadamard");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_h(ctx(h), h->precision, h->amps, h->n, bit_of(h, q));
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_x(tmfqs_gpu_state *h, unsigned q) {
	return guarded([&] {
		ensure_initialized(h, "GpuStateBackend::applyPauliX");
		validate_qubit(h, q, "GpuStateBackend::applyPauliX");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_x(ctx(h), h->precision, h->amps, h->n, bit_of(h, q));
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_cphase(tmfqs_gpu_state *h, unsigned c, unsigned t, double theta) {
	return guarded([&] {
		ensure_initialized(h, "GpuStateBackend::applyControlledPhaseShift");
		validate_two(h, c, t, "GpuStateBackend::applyControlledPhaseShift");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_cphase(ctx(h), h->precision, h->amps, h->n, bit_of(h, c), bit_of(h, t), std::cos(theta), std::sin(theta));
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_cnot(tmfqs_gpu_state *h, unsigned c, unsigned t) {
	return guarded([&] {
		ensure_initialized(h, "GpuStateBackend::applyControlledNot");
		validate_two(h, c, t, "GpuStateBackend::applyControlledNot");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_cnot(ctx(h), h->precision, h->amps, h->n, bit_of(h, c), bit_of(h, t));
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_swap(tmfqs_gpu_state *h, unsigned a, unsigned b) {
	return guarded([&] {
		ensure_initialized(h, "swap");
		validate_two(h, a, b, "GpuStateBackend::applySwap");
		DeviceScope d(h);
		before_mutation(h);
		{
			PassTimer timer(h, TMFQS_KT_GATE, sweep_bytes(h));
			tqb::launch_swap(ctx(h), h->precision, h->amps, h->n, bit_of(h, a), bit_of(h, b));
		}
		++h->stats.gate_passes;
	});
}

int tmfqs_gpu_gate(tmfqs_gpu_state *h, const double *matrix, const unsigned *qubits, unsigned k) {
	return guarded([&] {
		ensure_initialized(h, "gate application");
		tmfqs_op op{};
		op.kind = TMFQS_OP_GATE;
		op.matrix = matrix;
		op.qubits = qubits;
		op.k = k;
		validate_op(h, op);
		DeviceScope d(h);
		before_mutation(h);
		run_gate(h, matrix, qubits, k);
	});
}

int tmfqs_gpu_load_apply_ops(tmfqs_gpu_state *h, unsigned n, const double *host, const tmfqs_op *ops, size_t count) {
	return guarded([&] { load_apply_ops_body(h, n, host, ops, count); });
}

int tmfqs_debug_fail_allocations(unsigned skip, unsigned count) {
	tqb::arm_alloc_failures(skip, count);
	return TMFQS_OK;
}

int tmfqs_gpu_apply_ops(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t count) {
	return guarded([&] { apply_ops_body(h, ops, count); });
}

int tmfqs_gpu_grover_run(tmfqs_gpu_state *h, tmfqs_register_view *view, const uint64_t *marked, size_t count,
                         uint64_t iterations, int materialized) {
	return guarded([&] {
		ensure_initialized(h, "grover");
		if(!view) fail(TMFQS_ERR_INVALID_ARGUMENT, "null register view");
		if(count && !marked) fail(TMFQS_ERR_INVALID_ARGUMENT, "null marked list");
		std::vector<uint64_t> mk(marked, marked + count);
		std::sort(mk.begin(), mk.end());
		mk.erase(std::unique(mk.begin(), mk.end()), mk.end());
		for(uint64_t s : mk) validate_state(h, s, "QuantumRegister::applyPhaseFlipBasisState");
		DeviceScope d(h);
		if(iterations == 0) return;
		if(materialized && h->opt_grover_fusion && !view->overlay) {
			const bool closed = h->precision == TMFQS_FP32 || !h->opt_exact;
			if(h->precision == TMFQS_FP64) grover_materialized_fused<double>(h, view, mk, iterations, closed);
			else grover_materialized_fused<float>(h, view, mk, iterations, closed);
			return;
		}
		for(uint64_t k = 0; k < iterations; ++k) {
			for(uint64_t s : mk) register_flip(h, view, s);
			register_inversion(h, view, materialized != 0);
		}
		check_cuda(cudaStreamSynchronize(h->stream), "grover sync");
	});
}

int tmfqs_sample_static(const void *device_amps, int precision, unsigned num_qubits, double rnd, void *stream,
                        uint64_t *index_out) {
	return guarded([&] {
		if(!device_amps || !index_out) fail(TMFQS_ERR_INVALID_ARGUMENT, "tmfqs_sample_static: null pointer");
		if(precision != TMFQS_FP64 && precision != TMFQS_FP32) fail(TMFQS_ERR_INVALID_ARGUMENT, "unknown precision");
		if(!(rnd >= 0.0 && rnd < 1.0)) fail(TMFQS_ERR_INVALID_ARGUMENT, "tmfqs_sample_static requires rnd in [0,1)");
		const tqb::SeqResult r =
			tqb::seq_sample_static(precision, device_amps, num_qubits, rnd, static_cast<cudaStream_t>(stream));
		if(r.index >= (1ull << num_qubits)) fail(TMFQS_ERR_RUNTIME, "tmfqs_sample_static: cumulative probability did not reach sample");
		*index_out = r.index;
	});
}

int tmfqs_gpu_adjoint_gradient(tmfqs_gpu_state *h, const tmfqs_op *ops, size_t count, const uint64_t *obs_masks,
                               const double *obs_weights, unsigned obs_terms, size_t checkpoint_every,
                               double *expectation, double *grads) {
	return guarded([&] {
		require_handle(h);
		adjoint_gradient(h, ops, count, obs_masks, obs_weights, obs_terms, checkpoint_every, expectation, grads);
	});
}

int tmfqs_gpu_compare(tmfqs_gpu_state *ref, tmfqs_gpu_state *got, tmfqs_state_comparison *out) {
	return guarded([&] {
		ensure_initialized(ref, "compare");
		ensure_initialized(got, "compare");
		if(!out) fail(TMFQS_ERR_INVALID_ARGUMENT, "null comparison output");
		if(ref->N != got->N) fail(TMFQS_ERR_INVALID_ARGUMENT, "Compared states must have the same state count");
		if(ref->device != got->device) fail(TMFQS_ERR_INVALID_ARGUMENT, "compare: states on different devices");
		DeviceScope d(ref);
		flush_dirty(got);
		check_cuda(cudaStreamSynchronize(got->stream), "compare sync");
		flush_dirty(ref);
		tqb::CompareReport r{};
		tqb::launch_compare(ctx(ref), ref->precision, ref->amps, got->precision, got->amps, ref->N, r);
		const tqb::Overlay none;
		const double ref_sq = tqb::seq_replay(ref->precision, ref->amps, ref->N, tqb::kTermProb, none, false, 0.0, ref->seq,
		                                      ref->stream, ref->num_sms, &ref->stats.kernel_launches).value;
		const double got_sq = tqb::seq_replay(got->precision, got->amps, got->N, tqb::kTermProb, none, false, 0.0, got->seq,
		                                      got->stream, got->num_sms, &got->stats.kernel_launches).value;
		const double diff_sq = tqb::seq_diff_norm(ref->precision, ref->amps, got->precision, got->amps, ref->N, ref->seq,
		                                          ref->stream, ref->num_sms, &ref->stats.kernel_launches);
		out->bitwise_equal = r.bitwise_equal ? 1 : 0;
		out->max_abs_amplitude_error = r.max_abs_amplitude_error;
		out->max_abs_component_error = r.max_abs_component_error;
		out->rmse_amplitude = std::sqrt(diff_sq / static_cast<double>(ref->N));
		out->rel_l2 = ref_sq == 0.0 ? 0.0 : std::sqrt(diff_sq / ref_sq);
		out->max_abs_probability_error = r.max_abs_probability_error;
		out->total_probability_diff = std::abs(got_sq - ref_sq);
		out->worst_state = r.worst_state;
	});
}

int tmfqs_gpu_sync(tmfqs_gpu_state *h) {
	return guarded([&] {
		require_handle(h);
		DeviceScope d(h);
		flush_dirty(h);
		check_cuda(cudaStreamSynchronize(h->stream), "sync");
	});
}

int tmfqs_gpu_stats(tmfqs_gpu_state *h, tmfqs_stats *out) {
	return guarded([&] {
		require_handle(h);
		*out = h->stats;
	});
}

int tmfqs_gpu_reset_stats(tmfqs_gpu_state *h) {
	return guarded([&] {
		require_handle(h);
		DeviceScope d(h);
		resolve_timers(h);
		h->stats = tmfqs_stats{};
		for(auto &t : h->times) t = tmfqs_kernel_time{};
		h->pass_log.clear();
		h->segment = 0;
	});
}

int tmfqs_gpu_pass_mark(tmfqs_gpu_state *h, uint64_t *segment_out) {
	return guarded([&] {
		require_handle(h);
		++h->segment;
		if(segment_out) *segment_out = h->segment;
	});
}

int tmfqs_gpu_pass_log(tmfqs_gpu_state *h, tmfqs_pass_record *out, size_t capacity, size_t *count) {
	return guarded([&] {
		require_handle(h);
		if(!count) fail(TMFQS_ERR_INVALID_ARGUMENT, "null count");
		DeviceScope d(h);
		resolve_timers(h);
		*count = h->pass_log.size();
		if(out) std::copy(h->pass_log.begin(), h->pass_log.begin() + std::min(capacity, h->pass_log.size()), out);
	});
}

int tmfqs_gpu_kernel_times(tmfqs_gpu_state *h, tmfqs_kernel_time *out) {
	return guarded([&] {
		require_handle(h);
		if(!out) fail(TMFQS_ERR_INVALID_ARGUMENT, "null output");
		DeviceScope d(h);
		resolve_timers(h);
		for(int i = 0; i < TMFQS_KT_COUNT; ++i) out[i] = h->times[i];
	});
}

int tmfqs_gpu_set_option(tmfqs_gpu_state *h, int option, long value) {
	return guarded([&] {
		require_handle(h);
		switch(option) {
			case TMFQS_OPT_FUSION: h->opt_fusion = value != 0; break;
			case TMFQS_OPT_FUSED_QUBITS:
				if(value < 0 || value > 10) fail(TMFQS_ERR_INVALID_ARGUMENT, "fused qubits must be in [0, 10]");
				h->opt_fused_qubits = (int)value;
				break;
			case TMFQS_OPT_GROVER_FUSION: h->opt_grover_fusion = value != 0; break;
			case TMFQS_OPT_KERNEL_TIMING: h->opt_timing = value != 0; break;
			case TMFQS_OPT_EXACT: h->opt_exact = value != 0; break;
			case TMFQS_OPT_RADIX: h->opt_radix = value != 0; break;
			case TMFQS_OPT_TENSOR: h->opt_tensor = value != 0; break;
			case TMFQS_OPT_QFT_PASS: h->opt_qft_pass = value != 0; break;
			default: fail(TMFQS_ERR_INVALID_ARGUMENT, "unknown option");
		}
	});
}

int tmfqs_gpu_device_buffer(tmfqs_gpu_state *h, void **ptr, size_t *bytes) {
	return guarded([&] {
		ensure_initialized(h, "device buffer query");
		flush_dirty(h);
		h->cache.clear();
		*ptr = h->amps;
		*bytes = h->bytes;
	});
}

int tmfqs_gpu_stream(tmfqs_gpu_state *h, void **stream) {
	return guarded([&] {
		require_handle(h);
		*stream = h->stream;
	});
}

}  // extern "C"
