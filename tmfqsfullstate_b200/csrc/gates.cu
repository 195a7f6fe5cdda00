// Single-operation kernels: one pass over HBM per gate, with the arithmetic
// of the reference Dense backend (dense_state_backend.cpp) restated per
// amplitude pair.  All kernels use 128-bit (complex128) or 64-bit (complex64)
// vector loads, 64-bit indices, and grid-stride loops over a grid sized to a
// multiple of the SM count.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cstring>

#include "device_common.cuh"
#include "internal.h"

namespace tqb {

namespace {

constexpr int kThreads = 256;

unsigned grid_for(const LaunchCtx &c, uint64_t work, unsigned per_thread = 1) {
	const uint64_t threads = (work + per_thread - 1) / per_thread;
	const uint64_t blocks = (threads + kThreads - 1) / kThreads;
	const uint64_t cap = (uint64_t)c.num_sms * 8u;
	return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(blocks, cap));
}

void after_launch(const LaunchCtx &c, const char *what) {
	check_cuda(cudaGetLastError(), what);
	if(c.launches) ++*c.launches;
}

}  // namespace

void upload_async(const LaunchCtx &c, void *dev, const void *src, size_t bytes, const char *what) {
	UploadRing *r = c.ring;
	if(!r || !r->host || bytes > UploadRing::kSlotBytes) {
		check_cuda(cudaMemcpyAsync(dev, src, bytes, cudaMemcpyHostToDevice, c.stream), what);
		check_cuda(cudaStreamSynchronize(c.stream), what);
		return;
	}
	const unsigned s = r->next;
	r->next = (s + 1) % UploadRing::kSlots;
	if(r->pending[s]) check_cuda(cudaEventSynchronize(r->ev[s]), what);
	unsigned char *slot = r->host + (size_t)s * UploadRing::kSlotBytes;
	std::memcpy(slot, src, bytes);
	check_cuda(cudaMemcpyAsync(dev, slot, bytes, cudaMemcpyHostToDevice, c.stream), what);
	check_cuda(cudaEventRecord(r->ev[s], c.stream), what);
	r->pending[s] = true;
}

namespace {

// applyHadamard, dense_state_backend.cpp:255-274: pairs (s0, s0|m), skip
// all-zero pairs, a0' = (a0+a1)*inv, a1' = (a0-a1)*inv per component.
template <typename R>
__global__ void k_h(typename Vec2<R>::type *a, uint64_t npairs, unsigned bit, R inv) {
	for(uint64_t i = gtid(); i < npairs; i += gstride()) {
		const uint64_t s0 = insert0(i, bit), s1 = s0 | (1ull << bit);
		const auto x = a[s0];
		const auto y = a[s1];
		if(x.x == R(0) && x.y == R(0) && y.x == R(0) && y.y == R(0)) continue;
		typename Vec2<R>::type o0, o1;
		o0.x = rmul(radd(x.x, y.x), inv);
		o0.y = rmul(radd(x.y, y.y), inv);
		o1.x = rmul(rsub(x.x, y.x), inv);
		o1.y = rmul(rsub(x.y, y.y), inv);
		a[s0] = o0;
		a[s1] = o1;
	}
}

// applyPauliX, dense_state_backend.cpp:276-287: swap every pair.
template <typename R>
__global__ void k_x(typename Vec2<R>::type *a, uint64_t npairs, unsigned bit) {
	for(uint64_t i = gtid(); i < npairs; i += gstride()) {
		const uint64_t s0 = insert0(i, bit), s1 = s0 | (1ull << bit);
		const auto x = a[s0];
		const auto y = a[s1];
		if(x.x == y.x && x.y == y.y) continue;
		a[s0] = y;
		a[s1] = x;
	}
}

// applyControlledNot, dense_state_backend.cpp:306-319: swap pairs on the
// target whose control bit is set.  Iterates the quarter space directly.
template <typename R>
__global__ void k_cnot(typename Vec2<R>::type *a, uint64_t nquads, unsigned cbit, unsigned tbit) {
	const unsigned lo = cbit < tbit ? cbit : tbit, hi = cbit < tbit ? tbit : cbit;
	for(uint64_t i = gtid(); i < nquads; i += gstride()) {
		const uint64_t s0 = insert00(i, lo, hi) | (1ull << cbit);
		const uint64_t s1 = s0 | (1ull << tbit);
		const auto x = a[s0];
		const auto y = a[s1];
		if(x.x == y.x && x.y == y.y) continue;
		a[s0] = y;
		a[s1] = x;
	}
}

// applyControlledPhaseShift, dense_state_backend.cpp:289-304: multiply the
// amplitudes with both bits set by (cos, sin); skip zero amplitudes.
template <typename R>
__global__ void k_cphase(typename Vec2<R>::type *a, uint64_t nquads, unsigned cbit, unsigned tbit, R pr, R pi) {
	const unsigned lo = cbit < tbit ? cbit : tbit, hi = cbit < tbit ? tbit : cbit;
	for(uint64_t i = gtid(); i < nquads; i += gstride()) {
		const uint64_t s = insert00(i, lo, hi) | (1ull << cbit) | (1ull << tbit);
		auto v = a[s];
		if(v.x == R(0) && v.y == R(0)) continue;
		cmul_ref(pr, pi, v.x, v.y);
		a[s] = v;
	}
}

// QuantumRegister::applySwap, quantum_register.cpp:518-527: three CNOTs are
// a pure permutation, exchanging the |..1..0..> and |..0..1..> amplitudes.
template <typename R>
__global__ void k_swap(typename Vec2<R>::type *a, uint64_t nquads, unsigned abit, unsigned bbit) {
	const unsigned lo = abit < bbit ? abit : bbit, hi = abit < bbit ? bbit : abit;
	for(uint64_t i = gtid(); i < nquads; i += gstride()) {
		const uint64_t base = insert00(i, lo, hi);
		const uint64_t s0 = base | (1ull << abit), s1 = base | (1ull << bbit);
		const auto x = a[s0];
		const auto y = a[s1];
		a[s0] = y;
		a[s1] = x;
	}
}

// phaseFlipBasisState, dense_state_backend.cpp:205-211.
template <typename R>
__global__ void k_phase_flip(typename Vec2<R>::type *a, uint64_t s) {
	auto v = a[s];
	v.x = -v.x;
	v.y = -v.y;
	a[s] = v;
}

// inversionAboutMean(mean), dense_state_backend.cpp:230-240:
// a' = 2*mean - a (2*mean is formed on the host; doubling is exact).
template <typename R>
__global__ void k_inversion(typename Vec2<R>::type *a, uint64_t N, R tmr, R tmi) {
	for(uint64_t i = gtid(); i < N; i += gstride()) {
		auto v = a[i];
		v.x = rsub(tmr, v.x);
		v.y = rsub(tmi, v.y);
		a[i] = v;
	}
}

// applyAffineTransform, dense_state_backend.cpp:242-253:
// re' = (sr*re - si*im) + br ; im' = (sr*im + si*re) + bi.
template <typename R>
__global__ void k_affine(typename Vec2<R>::type *a, uint64_t N, R sr, R si, R br, R bi) {
	for(uint64_t i = gtid(); i < N; i += gstride()) {
		auto v = a[i];
		const R re = v.x, im = v.y;
		v.x = radd(rsub(rmul(sr, re), rmul(si, im)), br);
		v.y = radd(radd(rmul(sr, im), rmul(si, re)), bi);
		a[i] = v;
	}
}

// The sum of all amplitudes in FP64 for the fast forms: each thread adds its
// share in a fixed order, the warps and then the block add theirs, and the
// caller adds the block partials in block order (deterministic; one read of
// the state).  The exact forms use the sequential-sum engine instead.
template <typename R>
__global__ void __launch_bounds__(256) k_sum_fast(const typename Vec2<R>::type *a, uint64_t N, double2 *part) {
	double sr = 0.0, si = 0.0;
#pragma unroll 4
	for(uint64_t i = gtid(); i < N; i += gstride()) {
		const auto v = a[i];
		sr += (double)v.x;
		si += (double)v.y;
	}
#pragma unroll
	for(int o = 16; o; o >>= 1) {
		sr += __shfl_xor_sync(0xffffffffu, sr, o);
		si += __shfl_xor_sync(0xffffffffu, si, o);
	}
	__shared__ double2 ws[8];
	if((threadIdx.x & 31u) == 0) ws[threadIdx.x >> 5] = make_double2(sr, si);
	__syncthreads();
	if(threadIdx.x == 0) {
		double2 t = make_double2(0.0, 0.0);
		for(unsigned w = 0; w < (blockDim.x >> 5); ++w) {
			t.x += ws[w].x;
			t.y += ws[w].y;
		}
		part[blockIdx.x] = t;
	}
}

template <typename R>
__global__ void k_scatter_uniform(typename Vec2<R>::type *a, const uint64_t *states, uint64_t count, R amp) {
	for(uint64_t i = gtid(); i < count; i += gstride()) {
		typename Vec2<R>::type v;
		v.x = amp;
		v.y = R(0);
		a[states[i]] = v;
	}
}

template <typename R>
__global__ void k_scatter_values(typename Vec2<R>::type *a, const uint64_t *idx, const double *vals, uint64_t count) {
	for(uint64_t i = gtid(); i < count; i += gstride()) {
		typename Vec2<R>::type v;
		v.x = (R)vals[2 * i];
		v.y = (R)vals[2 * i + 1];
		a[idx[i]] = v;
	}
}

template <typename R>
__global__ void k_convert(typename Vec2<R>::type *dst, const double2 *src, uint64_t count) {
	for(uint64_t i = gtid(); i < count; i += gstride()) {
		const double2 s = src[i];
		typename Vec2<R>::type v;
		v.x = (R)s.x;
		v.y = (R)s.y;
		dst[i] = v;
	}
}

template <typename R>
__global__ void k_convert_back(double2 *dst, const typename Vec2<R>::type *src, uint64_t count) {
	for(uint64_t i = gtid(); i < count; i += gstride()) {
		const auto s = src[i];
		dst[i] = make_double2((double)s.x, (double)s.y);
	}
}

// ---------------------------------------------------------------------------
// Generic k-qubit gate: applyGateByBlocks, gate_block_apply.h:103-213.
// Block index bits fill the non-target positions (composeBaseStateFromBlock,
// :14-22); local index idx has target b at bit (k-1-b) (:87-96).  All-zero
// blocks are skipped.  k == 1 uses the unrolled formula of :117-140; k >= 2
// accumulates row sums term by term (:165-176, :199-210).
// ---------------------------------------------------------------------------
struct GateGeom {
	unsigned n, k;
	unsigned tpos[10];   // target bit positions, block order
	unsigned sorted[10]; // target positions ascending (for base expansion)
};

template <typename R>
__device__ __forceinline__ uint64_t gate_base(uint64_t blk, const GateGeom &g) {
	uint64_t b = blk;
	for(unsigned i = 0; i < g.k; ++i) b = insert0(b, g.sorted[i]);
	return b;
}

__device__ __forceinline__ uint64_t gate_offset(unsigned idx, const GateGeom &g) {
	uint64_t off = 0;
	for(unsigned b = 0; b < g.k; ++b)
		if((idx >> (g.k - b - 1u)) & 1u) off |= 1ull << g.tpos[b];
	return off;
}

// k in {1, 2}: one thread per block.
template <typename R>
__global__ void k_gate_small(typename Vec2<R>::type *a, uint64_t nblocks, GateGeom g, const double *m) {
	for(uint64_t blk = gtid(); blk < nblocks; blk += gstride()) {
		const uint64_t base = gate_base<R>(blk, g);
		if(g.k == 1) {
			const uint64_t s0 = base, s1 = base | (1ull << g.tpos[0]);
			const auto x = a[s0];
			const auto y = a[s1];
			if(x.x == R(0) && x.y == R(0) && y.x == R(0) && y.y == R(0)) continue;
			const R a0r = x.x, a0i = x.y, a1r = y.x, a1i = y.y;
			const R g00r = (R)m[0], g00i = (R)m[1], g01r = (R)m[2], g01i = (R)m[3];
			const R g10r = (R)m[4], g10i = (R)m[5], g11r = (R)m[6], g11i = (R)m[7];
			typename Vec2<R>::type o0, o1;
			o0.x = rsub(radd(rsub(rmul(g00r, a0r), rmul(g00i, a0i)), rmul(g01r, a1r)), rmul(g01i, a1i));
			o0.y = radd(radd(radd(rmul(g00r, a0i), rmul(g00i, a0r)), rmul(g01r, a1i)), rmul(g01i, a1r));
			o1.x = rsub(radd(rsub(rmul(g10r, a0r), rmul(g10i, a0i)), rmul(g11r, a1r)), rmul(g11i, a1i));
			o1.y = radd(radd(radd(rmul(g10r, a0i), rmul(g10i, a0r)), rmul(g11r, a1i)), rmul(g11i, a1r));
			a[s0] = o0;
			a[s1] = o1;
			continue;
		}
		// k == 2
		uint64_t s[4];
		R ar[4], ai[4];
		bool nz = false;
		for(unsigned j = 0; j < 4; ++j) {
			s[j] = base | gate_offset(j, g);
			const auto v = a[s[j]];
			ar[j] = v.x;
			ai[j] = v.y;
			nz = nz || v.x != R(0) || v.y != R(0);
		}
		if(!nz) continue;
		typename Vec2<R>::type o[4];
		for(unsigned r = 0; r < 4; ++r) {
			R nr = R(0), ni = R(0);
			for(unsigned col = 0; col < 4; ++col) {
				const R gr = (R)m[2 * (r * 4 + col)], gi = (R)m[2 * (r * 4 + col) + 1];
				nr = radd(nr, rsub(rmul(gr, ar[col]), rmul(gi, ai[col])));
				ni = radd(ni, radd(rmul(gr, ai[col]), rmul(gi, ar[col])));
			}
			o[r].x = nr;
			o[r].y = ni;
		}
		for(unsigned r = 0; r < 4; ++r) a[s[r]] = o[r];
	}
}

// k == 0 or 3 <= k <= 10: one CTA per block; amplitudes staged in shared memory.
template <typename R>
__global__ void k_gate_block(typename Vec2<R>::type *a, uint64_t nblocks, GateGeom g, const double *m) {
	extern __shared__ unsigned char smem_raw[];
	typedef typename Vec2<R>::type V;
	V *loc = reinterpret_cast<V *>(smem_raw);
	const unsigned bs = 1u << g.k;
	V *out = loc + bs;
	for(uint64_t blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
		const uint64_t base = gate_base<R>(blk, g);
		bool nz = false;
		for(unsigned j = threadIdx.x; j < bs; j += blockDim.x) {
			const V v = a[base | gate_offset(j, g)];
			loc[j] = v;
			nz = nz || v.x != R(0) || v.y != R(0);
		}
		if(!__syncthreads_or(nz)) continue;
		for(unsigned r = threadIdx.x; r < bs; r += blockDim.x) {
			R nr = R(0), ni = R(0);
			const double *row = m + 2ull * r * bs;
			for(unsigned col = 0; col < bs; ++col) {
				const R gr = (R)row[2 * col], gi = (R)row[2 * col + 1];
				nr = radd(nr, rsub(rmul(gr, loc[col].x), rmul(gi, loc[col].y)));
				ni = radd(ni, radd(rmul(gr, loc[col].y), rmul(gi, loc[col].x)));
			}
			out[r].x = nr;
			out[r].y = ni;
		}
		__syncthreads();
		for(unsigned j = threadIdx.x; j < bs; j += blockDim.x) a[base | gate_offset(j, g)] = out[j];
		__syncthreads();
	}
}

template <typename R>
void dispatch_gate(const LaunchCtx &c, void *a, unsigned n, unsigned k, const double *m, const unsigned *tpos) {
	GateGeom g{};
	g.n = n;
	g.k = k;
	std::vector<unsigned> s(tpos, tpos + k);
	std::sort(s.begin(), s.end());
	for(unsigned i = 0; i < k; ++i) {
		g.tpos[i] = tpos[i];
		g.sorted[i] = s[i];
	}
	const uint64_t nblocks = 1ull << (n - k);
	auto *p = static_cast<typename Vec2<R>::type *>(a);
	if(k >= 1 && k <= 2) {
		k_gate_small<R><<<grid_for(c, nblocks), kThreads, 0, c.stream>>>(p, nblocks, g, m);
	} else {
		const size_t sm = 2ull * (1ull << k) * sizeof(typename Vec2<R>::type);
		if(sm > 48 * 1024) check_cuda(cudaFuncSetAttribute(k_gate_block<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), "gate smem");
		const unsigned threads = k <= 6 ? 64 : 256;
		const uint64_t blocks = std::min<uint64_t>(nblocks, (uint64_t)c.num_sms * 16u);
		k_gate_block<R><<<(unsigned)blocks, threads, sm, c.stream>>>(p, nblocks, g, m);
	}
	after_launch(c, "gate");
}

}  // namespace

#define TQB_DISPATCH(prec, ...)                 \
	do {                                        \
		if((prec) == TMFQS_FP64) {              \
			typedef double R;                   \
			__VA_ARGS__;                        \
		} else {                                \
			typedef float R;                    \
			__VA_ARGS__;                        \
		}                                       \
	} while(0)

void launch_h(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned bit) {
	const uint64_t np = 1ull << (n - 1);
	const double inv = 1.0 / std::sqrt(2.0);  // dense_state_backend.cpp:258
	TQB_DISPATCH(prec, k_h<R><<<grid_for(c, np), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), np, bit, (R)inv));
	after_launch(c, "hadamard");
}

void launch_x(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned bit) {
	const uint64_t np = 1ull << (n - 1);
	TQB_DISPATCH(prec, k_x<R><<<grid_for(c, np), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), np, bit));
	after_launch(c, "pauli_x");
}

void launch_cnot(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned cbit, unsigned tbit) {
	const uint64_t nq = 1ull << (n - 2);
	TQB_DISPATCH(prec, k_cnot<R><<<grid_for(c, nq), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), nq, cbit, tbit));
	after_launch(c, "cnot");
}

void launch_cphase(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned cbit, unsigned tbit, double cr, double ci) {
	const uint64_t nq = 1ull << (n - 2);
	TQB_DISPATCH(prec, k_cphase<R><<<grid_for(c, nq), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), nq, cbit, tbit, (R)cr, (R)ci));
	after_launch(c, "cphase");
}

void launch_swap(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned abit, unsigned bbit) {
	const uint64_t nq = 1ull << (n - 2);
	TQB_DISPATCH(prec, k_swap<R><<<grid_for(c, nq), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), nq, abit, bbit));
	after_launch(c, "swap");
}

void launch_phase_flip(const LaunchCtx &c, int prec, void *a, uint64_t s) {
	TQB_DISPATCH(prec, k_phase_flip<R><<<1, 1, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), s));
	after_launch(c, "phase_flip");
}

void launch_inversion(const LaunchCtx &c, int prec, void *a, unsigned n, double tmr, double tmi) {
	const uint64_t N = 1ull << n;
	TQB_DISPATCH(prec, k_inversion<R><<<grid_for(c, N), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), N, (R)tmr, (R)tmi));
	after_launch(c, "inversion");
}

void launch_affine(const LaunchCtx &c, int prec, void *a, unsigned n, double sre, double sim, double bre, double bim) {
	const uint64_t N = 1ull << n;
	TQB_DISPATCH(prec, k_affine<R><<<grid_for(c, N), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), N, (R)sre, (R)sim, (R)bre, (R)bim));
	after_launch(c, "affine");
}

unsigned sum_fast_blocks(const LaunchCtx &c) { return (unsigned)c.num_sms * 8u; }

void launch_sum_fast(const LaunchCtx &c, int prec, const void *a, uint64_t N, double2 *part) {
	TQB_DISPATCH(prec, k_sum_fast<R><<<sum_fast_blocks(c), 256, 0, c.stream>>>(static_cast<const Vec2<R>::type *>(a), N, part));
	after_launch(c, "fast sum");
}

void launch_scatter_uniform(const LaunchCtx &c, int prec, void *a, const uint64_t *states, uint64_t count, double amp) {
	TQB_DISPATCH(prec, k_scatter_uniform<R><<<grid_for(c, count), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), states, count, (R)amp));
	after_launch(c, "init_uniform");
}

void launch_scatter_values(const LaunchCtx &c, int prec, void *a, const uint64_t *idx, const double *vals, uint64_t count) {
	TQB_DISPATCH(prec, k_scatter_values<R><<<grid_for(c, count), kThreads, 0, c.stream>>>(static_cast<Vec2<R>::type *>(a), idx, vals, count));
	after_launch(c, "scatter");
}

void launch_gate(const LaunchCtx &c, int prec, void *a, unsigned n, unsigned k, const double *m, const unsigned *tpos) {
	TQB_DISPATCH(prec, dispatch_gate<R>(c, a, n, k, m, tpos));
}

void launch_to_c64(const LaunchCtx &c, void *dst, const double *src, uint64_t count) {
	k_convert<float><<<grid_for(c, count), kThreads, 0, c.stream>>>(static_cast<float2 *>(dst), reinterpret_cast<const double2 *>(src), count);
	after_launch(c, "to_c64");
}

void launch_from_c64(const LaunchCtx &c, double *dst, const void *src, uint64_t count) {
	k_convert_back<float><<<grid_for(c, count), kThreads, 0, c.stream>>>(reinterpret_cast<double2 *>(dst), static_cast<const float2 *>(src), count);
	after_launch(c, "from_c64");
}

}  // namespace tqb
