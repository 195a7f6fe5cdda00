// Fused passes: many circuit operations per read/write of the state.
//
// 1. k_fused: a tile of 2^K amplitudes -- the K "local" bit positions of a
//    pass, always including the lowest bits so each row is a contiguous run
//    of >= 128 bytes -- is staged in shared memory, and a program of
//    operations is applied to it in circuit order: Hadamards, X, CNOT and
//    swaps whose moving bits are local, and diagonal operations (controlled
//    phases, basis-state phase flips) on any bits.  Every amplitude goes
//    through exactly the IEEE operations of the per-gate path, in the same
//    order, so results are bit-identical to the reference's gate-by-gate
//    Dense backend; only HBM traffic changes (one read + one write per pass
//    instead of per gate).  A Hadamard followed by controlled phases that all
//    share its qubit ("H-chain", the QFT ladder) is applied in one step per
//    amplitude pair: the chain only touches the |1> output of each butterfly.
// 2. k_bit_perm: trailing SWAP runs of disjoint qubit pairs (the QFT's final
//    bit reversal) as one in-place pass over tile pairs.
// 3. k_grover_temporal: materialised Grover iterations applied to each
//    amplitude for all iterations while it sits in registers (the per-
//    iteration scalar means are precomputed exactly on the host).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace tqb {

namespace {

constexpr unsigned kFusedThreads = 256;
constexpr unsigned kMaxLocal = 13;

struct FusedGeom {
	unsigned n, K, m;          // state bits, local bits, contiguous low local bits
	unsigned lpos[kMaxLocal];  // ascending local bit positions
	uint64_t ntiles;
	unsigned nops;
	double inv;                // 1.0 / std::sqrt(2.0), formed on the host (dense_state_backend.cpp:258)
};

__device__ __forceinline__ uint64_t expand_outer(uint64_t o, const FusedGeom &g) {
	for(unsigned i = 0; i < g.K; ++i) o = insert0(o, g.lpos[i]);
	return o;
}

template <typename R>
__device__ __forceinline__ void apply_chain(R &re, R &im, uint64_t gidx, uint64_t mask, const double2 *tab) {
	uint64_t bits = gidx & mask;
	while(bits) {
		const unsigned b = 63u - (unsigned)__clzll((long long)bits);
		bits ^= 1ull << b;
		if(re == R(0) && im == R(0)) continue;
		const double2 ph = tab[b];
		cmul_ref((R)ph.x, (R)ph.y, re, im);
	}
}

template <typename R>
__global__ void __launch_bounds__(kFusedThreads) k_fused(typename Vec2<R>::type *a, FusedGeom g, const FusedOp *ops,
                                                         const double2 *phases) {
	typedef typename Vec2<R>::type V;
	extern __shared__ unsigned char smem_raw[];
	const unsigned T = 1u << g.K;
	V *s = reinterpret_cast<V *>(smem_raw);
	uint64_t *hitab = reinterpret_cast<uint64_t *>(s + T);
	const unsigned nhi = 1u << (g.K - g.m);
	for(unsigned h = threadIdx.x; h < nhi; h += blockDim.x) {
		uint64_t v = 0;
		for(unsigned i = 0; i < g.K - g.m; ++i)
			if((h >> i) & 1u) v |= 1ull << g.lpos[g.m + i];
		hitab[h] = v;
	}
	__syncthreads();
	const unsigned lowmask = (1u << g.m) - 1u;
	auto scatter = [&](unsigned j) -> uint64_t { return (uint64_t)(j & lowmask) | hitab[j >> g.m]; };
	const unsigned half = T >> 1, quarter = T >> 2;
	for(uint64_t o = blockIdx.x; o < g.ntiles; o += gridDim.x) {
		const uint64_t base = expand_outer(o, g);
		for(unsigned j = threadIdx.x; j < T; j += blockDim.x) s[j] = a[base | scatter(j)];
		__syncthreads();
		for(unsigned k = 0; k < g.nops; ++k) {
			const FusedOp op = ops[k];
			switch(op.kind) {
				case kFH:
				case kFHChain: {
					const R inv = (R)g.inv;
					for(unsigned p = threadIdx.x; p < half; p += blockDim.x) {
						const unsigned j0 = (unsigned)insert0(p, op.lt), j1 = j0 | (1u << op.lt);
						const V x = s[j0], y = s[j1];
						if(x.x == R(0) && x.y == R(0) && y.x == R(0) && y.y == R(0)) continue;
						V o0, o1;
						o0.x = rmul(radd(x.x, y.x), inv);
						o0.y = rmul(radd(x.y, y.y), inv);
						o1.x = rmul(rsub(x.x, y.x), inv);
						o1.y = rmul(rsub(x.y, y.y), inv);
						if(op.kind == kFHChain) apply_chain<R>(o1.x, o1.y, base | scatter(j1), op.mask, phases + op.tab);
						s[j0] = o0;
						s[j1] = o1;
					}
					__syncthreads();
					break;
				}
				case kFX:
				case kFCnot: {
					for(unsigned p = threadIdx.x; p < half; p += blockDim.x) {
						const unsigned j0 = (unsigned)insert0(p, op.lt), j1 = j0 | (1u << op.lt);
						if(op.kind == kFCnot && ((base | scatter(j0)) & op.mask) == 0) continue;
						const V x = s[j0], y = s[j1];
						if(x.x == y.x && x.y == y.y) continue;
						s[j0] = y;
						s[j1] = x;
					}
					__syncthreads();
					break;
				}
				case kFSwap: {
					const unsigned lo = op.lt < op.lc ? op.lt : op.lc, hi = op.lt < op.lc ? op.lc : op.lt;
					for(unsigned q = threadIdx.x; q < quarter; q += blockDim.x) {
						const unsigned j = (unsigned)insert00(q, lo, hi);
						const unsigned ja = j | (1u << op.lt), jb = j | (1u << op.lc);
						const V x = s[ja], y = s[jb];
						s[ja] = y;
						s[jb] = x;
					}
					__syncthreads();
					break;
				}
				case kFCP: {
					const R pr = (R)op.cr, pi = (R)op.ci;
					for(unsigned j = threadIdx.x; j < T; j += blockDim.x) {
						if(((base | scatter(j)) & op.mask) != op.mask) continue;
						V v = s[j];
						if(v.x == R(0) && v.y == R(0)) continue;
						cmul_ref(pr, pi, v.x, v.y);
						s[j] = v;
					}
					// Diagonal ops keep the thread->amplitude ownership; a barrier
					// is needed only before the next pair operation.
					if(k + 1 == g.nops || (ops[k + 1].kind != kFCP && ops[k + 1].kind != kFFlip)) __syncthreads();
					break;
				}
				case kFFlip: {
					for(unsigned j = threadIdx.x; j < T; j += blockDim.x) {
						if((base | scatter(j)) != op.state) continue;
						V v = s[j];
						v.x = -v.x;
						v.y = -v.y;
						s[j] = v;
					}
					if(k + 1 == g.nops || (ops[k + 1].kind != kFCP && ops[k + 1].kind != kFFlip)) __syncthreads();
					break;
				}
				default:
					break;
			}
		}
		for(unsigned j = threadIdx.x; j < T; j += blockDim.x) a[base | scatter(j)] = s[j];
		__syncthreads();
	}
}

// ---------------------------------------------------------------------------
// In-place bit permutation for disjoint transpositions of bit positions.
// Local set S = low bits {0..r-1} plus their images; the remaining ("outer")
// bits are permuted among themselves, so tile o maps to tile perm(o).  A CTA
// loads tile o and its partner, then writes each to the other's slot with the
// local bits permuted; tiles fixed by the permutation are permuted alone.
// ---------------------------------------------------------------------------
constexpr unsigned kPermMaxLocal = 12;

struct PermGeom {
	unsigned n, K, m;
	unsigned lpos[kPermMaxLocal];
	unsigned lmap[kPermMaxLocal];  // local bit i -> local bit lmap[i]
	unsigned npairs;
	unsigned pa[32], pb[32];       // all transposed bit-position pairs
	uint64_t ntiles;
};

__device__ __forceinline__ uint64_t perm_global(uint64_t x, const PermGeom &g) {
	for(unsigned i = 0; i < g.npairs; ++i) {
		const uint64_t ba = (x >> g.pa[i]) & 1ull, bb = (x >> g.pb[i]) & 1ull;
		if(ba != bb) x ^= (1ull << g.pa[i]) | (1ull << g.pb[i]);
	}
	return x;
}

__device__ __forceinline__ uint64_t compress_outer(uint64_t x, const PermGeom &g) {
	// Remove local bit positions (descending so lower positions stay valid).
	for(int i = (int)g.K - 1; i >= 0; --i) {
		const unsigned p = g.lpos[i];
		const uint64_t lo = x & ((1ull << p) - 1ull);
		x = ((x >> (p + 1)) << p) | lo;
	}
	return x;
}

__device__ __forceinline__ unsigned perm_local(unsigned j, const PermGeom &g) {
	unsigned r = 0;
	for(unsigned i = 0; i < g.K; ++i)
		if((j >> i) & 1u) r |= 1u << g.lmap[i];
	return r;
}

template <typename R>
__global__ void __launch_bounds__(256) k_bit_perm(typename Vec2<R>::type *a, PermGeom g) {
	typedef typename Vec2<R>::type V;
	extern __shared__ unsigned char smem_raw[];
	const unsigned T = 1u << g.K;
	V *A = reinterpret_cast<V *>(smem_raw);
	V *B = A + T;
	uint64_t *hitab = reinterpret_cast<uint64_t *>(B + T);
	const unsigned nhi = 1u << (g.K - g.m);
	for(unsigned h = threadIdx.x; h < nhi; h += blockDim.x) {
		uint64_t v = 0;
		for(unsigned i = 0; i < g.K - g.m; ++i)
			if((h >> i) & 1u) v |= 1ull << g.lpos[g.m + i];
		hitab[h] = v;
	}
	__syncthreads();
	const unsigned lowmask = (1u << g.m) - 1u;
	auto scatter = [&](unsigned j) -> uint64_t { return (uint64_t)(j & lowmask) | hitab[j >> g.m]; };
	for(uint64_t o = blockIdx.x; o < g.ntiles; o += gridDim.x) {
		uint64_t base = o;
		for(unsigned i = 0; i < g.K; ++i) base = insert0(base, g.lpos[i]);
		const uint64_t pbase = perm_global(base, g);
		const uint64_t po = compress_outer(pbase, g);
		if(po < o) continue;  // handled with its partner
		for(unsigned j = threadIdx.x; j < T; j += blockDim.x) A[j] = a[base | scatter(j)];
		if(po != o)
			for(unsigned j = threadIdx.x; j < T; j += blockDim.x) B[j] = a[pbase | scatter(j)];
		__syncthreads();
		// amplitude (base|scatter(j)) moves to (pbase|scatter(perm_local(j))).
		for(unsigned jw = threadIdx.x; jw < T; jw += blockDim.x) {
			const unsigned js = perm_local(jw, g);  // involution: source of slot jw
			a[pbase | scatter(jw)] = A[js];
			if(po != o) a[base | scatter(jw)] = B[js];
		}
		__syncthreads();
	}
}

// ---------------------------------------------------------------------------
// Temporal Grover pass.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_grover_temporal(typename Vec2<R>::type *a, uint64_t N, const double2 *tm,
                                                        uint64_t iters, uint64_t flip_from, const uint64_t *marked,
                                                        unsigned nm) {
	typedef typename Vec2<R>::type V;
	constexpr unsigned kPer = 4;
	for(uint64_t i0 = gtid() * kPer; i0 < N; i0 += gstride() * kPer) {
		V v[kPer];
		bool mk[kPer];
		bool anymk = false;
#pragma unroll
		for(unsigned u = 0; u < kPer; ++u) {
			const uint64_t i = i0 + u;
			mk[u] = false;
			if(i < N) {
				v[u] = a[i];
				for(unsigned q = 0; q < nm; ++q) mk[u] = mk[u] || marked[q] == i;
			}
			anymk = anymk || mk[u];
		}
		if(!anymk) {
			for(uint64_t k = 0; k < iters; ++k) {
				const double2 t = tm[k];
				const R tr = (R)t.x, ti = (R)t.y;
#pragma unroll
				for(unsigned u = 0; u < kPer; ++u) {
					v[u].x = rsub(tr, v[u].x);
					v[u].y = rsub(ti, v[u].y);
				}
			}
		} else {
			for(uint64_t k = 0; k < iters; ++k) {
				const double2 t = tm[k];
				const R tr = (R)t.x, ti = (R)t.y;
#pragma unroll
				for(unsigned u = 0; u < kPer; ++u) {
					if(mk[u] && k >= flip_from) {
						v[u].x = -v[u].x;
						v[u].y = -v[u].y;
					}
					v[u].x = rsub(tr, v[u].x);
					v[u].y = rsub(ti, v[u].y);
				}
			}
		}
#pragma unroll
		for(unsigned u = 0; u < kPer; ++u)
			if(i0 + u < N) a[i0 + u] = v[u];
	}
}

void after_launch(const LaunchCtx &c, const char *what) {
	check_cuda(cudaGetLastError(), what);
	if(c.launches) ++*c.launches;
}

template <typename R>
void run_fused(const LaunchCtx &c, void *a, const FusedPass &pass, void *&dev_prog, size_t &dev_prog_bytes) {
	FusedGeom g{};
	g.n = pass.n;
	g.K = pass.K;
	g.m = 0;
	while(g.m < pass.K && pass.lpos[g.m] == g.m) ++g.m;
	if(g.m == 0 || pass.K > kMaxLocal) fail(TMFQS_ERR_LOGIC, "fused pass: bad local set");
	for(unsigned i = 0; i < pass.K; ++i) g.lpos[i] = pass.lpos[i];
	g.ntiles = 1ull << (pass.n - pass.K);
	g.nops = (unsigned)pass.ops.size();
	g.inv = 1.0 / std::sqrt(2.0);
	const size_t ops_bytes = pass.ops.size() * sizeof(FusedOp);
	const size_t ph_off = (ops_bytes + 255) & ~size_t(255);
	const size_t need = ph_off + std::max<size_t>(16, pass.phases.size() * sizeof(double));
	if(need > dev_prog_bytes) {
		if(dev_prog) {
			check_cuda(cudaStreamSynchronize(c.stream), "fused program sync");
			cudaFree(dev_prog);
		}
		dev_prog = nullptr;
		dev_prog_bytes = 0;
		if(cudaMalloc(&dev_prog, need * 2) != cudaSuccess) {
			cudaGetLastError();
			fail(TMFQS_ERR_NOMEM, "fused pass program allocation failed");
		}
		dev_prog_bytes = need * 2;
	}
	// The program buffer is reused: make sure the previous pass consumed it.
	std::vector<unsigned char> host(need, 0);
	std::memcpy(host.data(), pass.ops.data(), ops_bytes);
	if(!pass.phases.empty()) std::memcpy(host.data() + ph_off, pass.phases.data(), pass.phases.size() * sizeof(double));
	check_cuda(cudaMemcpyAsync(dev_prog, host.data(), need, cudaMemcpyHostToDevice, c.stream), "fused program upload");
	check_cuda(cudaStreamSynchronize(c.stream), "fused program upload sync");
	const size_t smem = (sizeof(typename Vec2<R>::type) << pass.K) + (sizeof(uint64_t) << (pass.K - g.m));
	check_cuda(cudaFuncSetAttribute(k_fused<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fused smem");
	int per_sm = 1;
	check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<R>, kFusedThreads, smem), "fused occupancy");
	const uint64_t grid = std::min<uint64_t>(g.ntiles, (uint64_t)c.num_sms * std::max(1, per_sm));
	k_fused<R><<<(unsigned)grid, kFusedThreads, smem, c.stream>>>(
		static_cast<typename Vec2<R>::type *>(a), g, static_cast<const FusedOp *>(dev_prog),
		reinterpret_cast<const double2 *>(static_cast<unsigned char *>(dev_prog) + ph_off));
	after_launch(c, "fused pass");
}

template <typename R>
void run_perm(const LaunchCtx &c, void *a, unsigned n, const std::vector<std::pair<unsigned, unsigned>> &pairs) {
	PermGeom g{};
	g.n = n;
	g.npairs = (unsigned)pairs.size();
	if(g.npairs > 32) fail(TMFQS_ERR_LOGIC, "bit permutation: too many pairs");
	std::vector<int> img(n);
	for(unsigned i = 0; i < n; ++i) img[i] = (int)i;
	for(unsigned i = 0; i < g.npairs; ++i) {
		g.pa[i] = pairs[i].first;
		g.pb[i] = pairs[i].second;
		img[pairs[i].first] = (int)pairs[i].second;
		img[pairs[i].second] = (int)pairs[i].first;
	}
	const unsigned maxK = sizeof(R) == 8 ? 10u : 11u;  // two tiles of 16/32 KB
	// Grow the low run r while the closed local set fits.
	std::vector<unsigned> best;
	for(unsigned r = 1; r <= n; ++r) {
		std::vector<bool> in(n, false);
		for(unsigned b = 0; b < r; ++b) {
			in[b] = true;
			in[img[b]] = true;
		}
		std::vector<unsigned> set;
		for(unsigned b = 0; b < n; ++b)
			if(in[b]) set.push_back(b);
		if(set.size() > maxK) break;
		best = set;
	}
	g.K = (unsigned)best.size();
	g.m = 0;
	while(g.m < g.K && best[g.m] == g.m) ++g.m;
	for(unsigned i = 0; i < g.K; ++i) {
		g.lpos[i] = best[i];
		const unsigned target = (unsigned)img[best[i]];
		g.lmap[i] = (unsigned)(std::find(best.begin(), best.end(), target) - best.begin());
	}
	g.ntiles = 1ull << (n - g.K);
	const size_t smem = 2 * (sizeof(typename Vec2<R>::type) << g.K) + (sizeof(uint64_t) << (g.K - g.m));
	check_cuda(cudaFuncSetAttribute(k_bit_perm<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "perm smem");
	int per_sm = 1;
	check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bit_perm<R>, 256, smem), "perm occupancy");
	const uint64_t grid = std::min<uint64_t>(g.ntiles, (uint64_t)c.num_sms * std::max(1, per_sm));
	k_bit_perm<R><<<(unsigned)grid, 256, smem, c.stream>>>(static_cast<typename Vec2<R>::type *>(a), g);
	after_launch(c, "bit permutation");
}

}  // namespace

void launch_fused_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, void *&dev_prog,
                       size_t &dev_prog_bytes) {
	if(prec == TMFQS_FP64) run_fused<double>(c, a, pass, dev_prog, dev_prog_bytes);
	else run_fused<float>(c, a, pass, dev_prog, dev_prog_bytes);
}

void launch_bit_permutation(const LaunchCtx &c, int prec, void *a, unsigned n,
                            const std::vector<std::pair<unsigned, unsigned>> &pairs) {
	if(prec == TMFQS_FP64) run_perm<double>(c, a, n, pairs);
	else run_perm<float>(c, a, n, pairs);
}

void launch_grover_temporal(const LaunchCtx &c, int prec, void *a, unsigned n, const double *dev_two_means,
                            uint64_t iterations, const uint64_t *dev_marked, unsigned marked_count,
                            uint64_t flip_from) {
	const uint64_t N = 1ull << n;
	const uint64_t threads = (N + 3) / 4;
	const uint64_t blocks = std::max<uint64_t>(1, std::min<uint64_t>((threads + 255) / 256, (uint64_t)c.num_sms * 8));
	const double2 *tm = reinterpret_cast<const double2 *>(dev_two_means);
	if(prec == TMFQS_FP64)
		k_grover_temporal<double><<<(unsigned)blocks, 256, 0, c.stream>>>(static_cast<double2 *>(a), N, tm, iterations, flip_from, dev_marked, marked_count);
	else
		k_grover_temporal<float><<<(unsigned)blocks, 256, 0, c.stream>>>(static_cast<float2 *>(a), N, tm, iterations, flip_from, dev_marked, marked_count);
	after_launch(c, "grover temporal");
}

}  // namespace tqb
