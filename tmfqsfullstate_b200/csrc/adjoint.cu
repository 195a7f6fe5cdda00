// Kernels of the adjoint (reverse-mode) gradient of a diagonal observable
// with respect to controlled-phase angles (tmfqs_gpu_adjoint_gradient).
//
// k_obs_apply: lambda = O psi for a diagonal observable
//   O = sum_j w_j Z^{m_j}  (Z^{m} = product of Z over the qubits of bit mask m:
//   eigenvalue (-1)^popcount(x & m) on basis state x), with the expectation
//   <psi|O|psi> accumulated in FP64.
// k_grad_run: for a run of consecutive diagonal gates (controlled phases and
//   phase flips), all their angle derivatives in one read of lambda and psi,
//   then the run's inverse applied to lambda (and psi when asked).  Within a
//   run the gates commute and have unit-modulus phases, so for every gate the
//   derivative 2 Re <lambda_k| dU_k/dtheta |psi_{k-1}> equals
//       2 * sum_{x: both bits set} (Im(lambda_x) Re(psi_x) - Re(lambda_x) Im(psi_x))
//   with lambda and psi taken at the end of the run (the phases of the later
//   gates of the run cancel in conj(lambda_x) psi_x).
// Per-block FP64 partial sums stay on the device and are added in a fixed
// order (k_sum_partials), so the results do not depend on scheduling.
#include <algorithm>
#include <cmath>

#include "device_common.cuh"
#include "internal.h"

namespace tqb {

namespace {

constexpr unsigned kAdjThreads = 256;
constexpr unsigned kBatch = 4;      // amplitudes per thread per loop trip (observable)
constexpr unsigned kGradBatch = 8;  // consecutive amplitudes per thread per loop trip (gradient runs)

struct ObsParams {
	uint64_t mask[kMaxObsTerms];
	double weight[kMaxObsTerms];
	unsigned nterms;
};

struct RunParams {
	uint64_t mask[kMaxDiagRun];  // controlled phase: both bit masks; flip: the basis state
	double cr[kMaxDiagRun], ci[kMaxDiagRun];
	int kind[kMaxDiagRun];       // DiagEntry kind
	unsigned count;
	unsigned nvary;              // leading entries that depend on index bits 0-2 (flips included)
};

__device__ __forceinline__ double block_sum(double v, double *red) {
#pragma unroll
	for(int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
	__syncthreads();
	if(lane == 0) red[warp] = v;
	__syncthreads();
	double s = 0.0;
	if(threadIdx.x == 0)
		for(unsigned w = 0; w < blockDim.x / 32; ++w) s += red[w];
	return s;
}

// O(x) = sum_j w_j (-1)^parity(x & m_j).  The parities of all terms form one
// 64-bit word, the XOR over the index bytes of x of a per-byte table word
// (bit j: parity of that byte of x & m_j); O(x) is then the sum over the
// word's bytes of a table of signed weight sums (256 per byte of terms, FP64).
template <typename R>
__global__ void __launch_bounds__(kAdjThreads) k_obs_apply(const typename Vec2<R>::type *psi, typename Vec2<R>::type *lam,
                                                          uint64_t N, ObsParams p, unsigned nbytes, double *partials) {
	typedef typename Vec2<R>::type V;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	uint64_t *par = reinterpret_cast<uint64_t *>(smem_raw);     // [nbytes][256]; byte 0 as [v & 3][v >> 2]
	double *wsum = reinterpret_cast<double *>(par + nbytes * 256);  // [ceil(nterms / 8)][256]
	__shared__ double red[kAdjThreads / 32];
	const unsigned nt = (p.nterms + 7) / 8;
	for(unsigned e = threadIdx.x; e < nbytes * 256; e += blockDim.x) {
		const unsigned j = e >> 8, v = e & 255u;
		uint64_t w = 0;
		for(unsigned t = 0; t < p.nterms; ++t) w |= (uint64_t)(__popc(v & ((unsigned)(p.mask[t] >> (8 * j)) & 255u)) & 1) << t;
		par[j ? e : (((v & 3u) << 6) | (v >> 2))] = w;
	}
	for(unsigned e = threadIdx.x; e < nt * 256; e += blockDim.x) {
		const unsigned k = e >> 8, v = e & 255u;
		double o = 0.0;
		for(unsigned b = 0; b < 8 && 8 * k + b < p.nterms; ++b) o += ((v >> b) & 1u) ? -p.weight[8 * k + b] : p.weight[8 * k + b];
		wsum[e] = o;
	}
	__syncthreads();
	double acc = 0.0;
	// kBatch consecutive amplitudes per thread, loads issued together.
	for(uint64_t x0 = gtid() * kBatch; x0 < N; x0 += gstride() * kBatch) {
		V v[kBatch];
#pragma unroll
		for(unsigned u = 0; u < kBatch; ++u)
			if(x0 + u < N) v[u] = psi[x0 + u];
		uint64_t hi = 0;
		for(unsigned j = 1; j < nbytes; ++j) hi ^= par[(j << 8) | ((unsigned)(x0 >> (8 * j)) & 255u)];
		const unsigned b0s = ((unsigned)x0 & 255u) >> 2;
#pragma unroll
		for(unsigned u = 0; u < kBatch; ++u) {
			const uint64_t x = x0 + u;
			if(x >= N) break;
			const uint64_t w = hi ^ par[(u << 6) | b0s];
			double o = wsum[w & 255u];
			for(unsigned k = 1; k < nt; ++k) o += wsum[(k << 8) | ((unsigned)(w >> (8 * k)) & 255u)];
			const double re = (double)v[u].x, im = (double)v[u].y;
			acc += o * (re * re + im * im);
			V l;
			l.x = (R)(o * re);
			l.y = (R)(o * im);
			lam[x] = l;
		}
	}
	const double s = block_sum(acc, red);
	if(threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Which entries of a run act on basis state x: an entry's condition (x
// contains its mask, or x equals the flipped state) holds exactly when it
// holds byte by byte, so the set of entries hitting x is the AND of one
// 32-bit table word per index byte ("hit" word, bit k for entry k).
//
// The inverse of the run multiplies amplitude x by the product of the
// conjugate phases of its hit entries (-1 for a flip).  The gates commute, so
// the product is taken byte by byte over the hit word: up to four tables of
// 256 products (formed in FP64, rounded once to the storage type).  When the
// caller put the entries that depend on index bits 0-2 first and there are at
// most 8 of them, bytes 1-3 of the hit word are the same for a thread's eight
// amplitudes: their product is formed once per batch, and each amplitude takes
// one lookup and one complex product for its phase.
//
// Gradients: a thread owns kGradBatch = 8 consecutive amplitudes x0 + u, so
// for a controlled phase with mask m the condition splits into its low part
// c = m & 7 (on u) and the rest (on x0, the same for all eight).  Every
// entry whose rest holds (the hit word of x0 | 7, flips removed) receives the
// superset sum S[c] = sum over u containing c of v(x0 + u), once per batch.
// Each lane adds these into its own shared-memory column (entry-major, no
// bank conflicts).  A: FP32 columns for complex64, FP64 for complex128; block
// and grid sums are FP64.
template <typename V, typename R>
__device__ __forceinline__ V cmul(V a, V b) {
	V r;
	r.x = fma(a.x, b.x, -(a.y * b.y));
	r.y = fma(a.x, b.y, a.y * b.x);
	return r;
}

template <typename R, typename A>
__global__ void __launch_bounds__(kAdjThreads, 2) k_grad_run(typename Vec2<R>::type *lam, typename Vec2<R>::type *psi,
                                                            uint64_t N, RunParams rp, unsigned nbytes, int uncompute_psi,
                                                            double *partials) {
	typedef typename Vec2<R>::type V;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	A *accs = reinterpret_cast<A *>(smem_raw);                                              // [warps][entries][32]
	V *qtab = reinterpret_cast<V *>(accs + (kAdjThreads / 32) * kMaxDiagRun * 32);           // [4][256]
	uint32_t *tab = reinterpret_cast<uint32_t *>(qtab + 4 * 256);                           // [nbytes][256]
	__shared__ double red[kAdjThreads / 32];
	__shared__ uint32_t cls[kGradBatch];
	const unsigned count = rp.count;
	const unsigned nq = (count + 7) / 8;  // phase tables in use
	uint32_t flips = 0;
	for(unsigned k = 0; k < count; ++k)
		if(rp.kind[k] == kDiagFlip) flips |= 1u << k;
	if(threadIdx.x < kGradBatch) {
		uint32_t m = 0;
		for(unsigned k = 0; k < count; ++k)
			if(!((flips >> k) & 1u) && (unsigned)(rp.mask[k] & (kGradBatch - 1)) == threadIdx.x) m |= 1u << k;
		cls[threadIdx.x] = m;
	}
	for(unsigned e = threadIdx.x; e < nq * 256; e += blockDim.x) {
		const unsigned j = e >> 8, v = e & 255u;
		double pr = 1.0, pi = 0.0;
		for(unsigned b = 0; b < 8; ++b) {
			const unsigned k = 8 * j + b;
			if(k >= count || !((v >> b) & 1u)) continue;
			const double c = ((flips >> k) & 1u) ? -1.0 : rp.cr[k], sn = ((flips >> k) & 1u) ? 0.0 : -rp.ci[k];
			const double tr = pr * c - pi * sn;
			pi = pr * sn + pi * c;
			pr = tr;
		}
		V q;
		q.x = (R)pr;
		q.y = (R)pi;
		qtab[e] = q;
	}
	// Byte 0 is stored transposed, [v & 7][v >> 3]: a warp's lanes look up
	// b0 | u with b0 = 8 * lane, on 32 consecutive words.
	for(unsigned e = threadIdx.x; e < nbytes * 256; e += blockDim.x) {
		const unsigned j = e >> 8, v = e & 255u;
		uint32_t bits = 0;
		for(unsigned k = 0; k < count; ++k) {
			const unsigned mb = (unsigned)(rp.mask[k] >> (8 * j)) & 255u;
			const bool ok = ((flips >> k) & 1u) ? v == mb : (v & mb) == mb;
			bits |= (ok ? 1u : 0u) << k;
		}
		tab[j ? e : (((v & 7u) << 5) | (v >> 3))] = bits;
	}
	for(unsigned e = threadIdx.x; e < (kAdjThreads / 32) * kMaxDiagRun * 32; e += blockDim.x) accs[e] = A(0);
	__syncthreads();
	const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	A *col = accs + warp * kMaxDiagRun * 32 + lane;
	const uint32_t all = count >= 32 ? ~0u : ((1u << count) - 1u);
	uint32_t cm[kGradBatch];
#pragma unroll
	for(unsigned c = 0; c < kGradBatch; ++c) cm[c] = cls[c];
	// A register of fewer than kGradBatch amplitudes (n < 3) fills the batch
	// with zero terms.
	const unsigned lim = N < kGradBatch ? (unsigned)N : kGradBatch;
	// The entries that depend on the three lowest index bits come first and
	// number at most 8: bytes 1-3 of the hit word are the same for the batch.
	const bool split = nq > 1 && rp.nvary <= 8;
	for(uint64_t x0 = gtid() * kGradBatch; x0 < N; x0 += gstride() * kGradBatch) {
		V lb[kGradBatch], pb[kGradBatch];
		if constexpr(sizeof(V) == 8) {
			if(lim == kGradBatch) {
				// Eight complex64 values: two 32-byte loads each (x0 is a multiple of 8).
#pragma unroll
				for(unsigned q = 0; q < kGradBatch / 4; ++q) {
					float a[8], b[8];
					ld_global_v8f(reinterpret_cast<const float *>(lam + x0 + 4 * q), a);
					ld_global_v8f(reinterpret_cast<const float *>(psi + x0 + 4 * q), b);
#pragma unroll
					for(unsigned u = 0; u < 4; ++u) {
						lb[4 * q + u] = V{a[2 * u], a[2 * u + 1]};
						pb[4 * q + u] = V{b[2 * u], b[2 * u + 1]};
					}
				}
			}
		}
#pragma unroll
		for(unsigned u = 0; u < kGradBatch; ++u)
			if(u < lim && (sizeof(V) != 8 || lim < kGradBatch)) {
				lb[u] = lam[x0 + u];
				pb[u] = psi[x0 + u];
			}
		uint32_t hh = all;
		for(unsigned j = 1; j < nbytes; ++j) hh &= tab[(j << 8) | ((unsigned)(x0 >> (8 * j)) & 255u)];
		const unsigned b0s = ((unsigned)x0 & 255u) >> 3;  // byte 0 of x0, transposed index
		// Entries 8 and up hit all eight amplitudes alike (split runs): their
		// phase product once per batch.
		V Prest;
		if(split) {
			const uint32_t h7 = hh & tab[((kGradBatch - 1) << 5) | b0s];
			Prest = qtab[256 | ((h7 >> 8) & 255u)];
			if(nq > 2) Prest = cmul<V, R>(Prest, qtab[512 | ((h7 >> 16) & 255u)]);
			if(nq > 3) Prest = cmul<V, R>(Prest, qtab[768 | (h7 >> 24)]);
		}
		A S[kGradBatch];
		// complex64: the results wait in registers for 16-byte stores.
		V lo[sizeof(V) == 8 ? kGradBatch : 1], po[sizeof(V) == 8 ? kGradBatch : 1];
#pragma unroll
		for(unsigned u = 0; u < kGradBatch; ++u) {
			S[u] = A(0);
			if(u >= lim) continue;
			V l = lb[u], p = pb[u];
			S[u] = (A)l.y * (A)p.x - (A)l.x * (A)p.y;
			// Table entry 0 is the empty product 1, which leaves a value unchanged.
			const uint32_t hit = hh & tab[(u << 5) | b0s];
			V P = qtab[hit & 255u];
			if(split) {
				P = cmul<V, R>(P, Prest);
			} else {
				if(nq > 1) P = cmul<V, R>(P, qtab[256 | ((hit >> 8) & 255u)]);
				if(nq > 2) P = cmul<V, R>(P, qtab[512 | ((hit >> 16) & 255u)]);
				if(nq > 3) P = cmul<V, R>(P, qtab[768 | (hit >> 24)]);
			}
			if(sizeof(V) == 8 && lim == kGradBatch) {
				lo[sizeof(V) == 8 ? u : 0] = cmul<V, R>(l, P);
				po[sizeof(V) == 8 ? u : 0] = cmul<V, R>(p, P);
			} else {
				lam[x0 + u] = cmul<V, R>(l, P);
				if(uncompute_psi) psi[x0 + u] = cmul<V, R>(p, P);
			}
		}
		if constexpr(sizeof(V) == 8) {
			if(lim == kGradBatch) {
#pragma unroll
				for(unsigned q = 0; q < kGradBatch / 4; ++q) {
					float a[8], b[8];
#pragma unroll
					for(unsigned u = 0; u < 4; ++u) {
						a[2 * u] = lo[4 * q + u].x;
						a[2 * u + 1] = lo[4 * q + u].y;
						b[2 * u] = po[4 * q + u].x;
						b[2 * u + 1] = po[4 * q + u].y;
					}
					st_global_v8f(reinterpret_cast<float *>(lam + x0 + 4 * q), a);
					if(uncompute_psi) st_global_v8f(reinterpret_cast<float *>(psi + x0 + 4 * q), b);
				}
			}
		}
		// Superset sums over the three low bits.
#pragma unroll
		for(unsigned b = 0; b < 3; ++b)
#pragma unroll
			for(unsigned u = 0; u < kGradBatch; ++u)
				if(!((u >> b) & 1u)) S[u] += S[u | (1u << b)];
		const uint32_t rest = hh & tab[((kGradBatch - 1) << 5) | b0s] & ~flips;
		if(rest) {
			// Columns of distinct entries never alias: the next column is read
			// before the current one is written, so the reads overlap.
#pragma unroll
			for(unsigned c = 0; c < kGradBatch; ++c) {
				uint32_t m = rest & cm[c];
				if(!m) continue;
				A *p = col + (__ffs(m) - 1) * 32;
				A cur = *p;
				for(m &= m - 1u; m; m &= m - 1u) {
					A *q = col + (__ffs(m) - 1) * 32;
					const A nxt = *q;
					*p = cur + S[c];
					p = q;
					cur = nxt;
				}
				*p = cur + S[c];
			}
		}
	}
	__syncthreads();
	// Entry k: sum its column of every warp (fixed order), then the block.
	for(unsigned k = 0; k < count; ++k) {
		double t = 0.0;
		const A *ck = accs + k * 32 + lane;
		for(unsigned w = 0; w < kAdjThreads / 32; ++w) t += (double)ck[w * kMaxDiagRun * 32];
		// Each warp holds the same t per lane; block_sum adds the lanes of every warp.
		const double s = block_sum(warp == 0 ? t : 0.0, red);
		if(threadIdx.x == 0) partials[blockIdx.x * kMaxDiagRun + k] = s;
	}
}

// One block per partial-sum array, one warp per column: lane l adds rows
// l, l + 32, ... in row order, then the warp adds its lanes in a fixed tree.
__global__ void k_sum_partials(const double *partials, size_t chunk_doubles, const __grid_constant__ PartialChunks t,
                               double *out) {
	const unsigned i = blockIdx.x, k = threadIdx.y, lane = threadIdx.x;
	const unsigned stride = t.stride[i];
	double s = 0.0;
	if(k < stride) {
		const double *p = partials + (size_t)i * chunk_doubles + k;
		for(unsigned b = lane; b < t.blocks[i]; b += 32) s += p[(size_t)b * stride];
	}
#pragma unroll
	for(int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
	if(lane == 0) out[i * kMaxDiagRun + k] = s;
}

size_t grad_smem(size_t acc_bytes, size_t vec_bytes, unsigned nbytes) {
	return acc_bytes * (kAdjThreads / 32) * kMaxDiagRun * 32 + vec_bytes * 4 * 256 + sizeof(uint32_t) * 256 * nbytes;
}

unsigned adj_blocks(const LaunchCtx &c, uint64_t N) {
	const uint64_t per_block = (uint64_t)kAdjThreads * kGradBatch;
	return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((N + per_block - 1) / per_block, (uint64_t)c.num_sms * 4));
}

}  // namespace

unsigned adjoint_max_blocks(int num_sms) { return (unsigned)num_sms * 4; }

unsigned launch_obs_apply(const LaunchCtx &c, int prec, const void *psi, void *lam, unsigned n, const uint64_t *masks,
                          const double *weights, unsigned nterms, double *dev_partials) {
	if(nterms == 0 || nterms > kMaxObsTerms) fail(TMFQS_ERR_INVALID_ARGUMENT, "observable: 1 to 64 terms");
	ObsParams p{};
	for(unsigned j = 0; j < nterms; ++j) {
		p.mask[j] = masks[j];
		p.weight[j] = weights[j];
	}
	p.nterms = nterms;
	const uint64_t N = 1ull << n;
	const unsigned blocks = adj_blocks(c, N);
	const unsigned nbytes = (n + 7) / 8;
	const size_t smem = sizeof(uint64_t) * 256 * nbytes + sizeof(double) * 256 * ((nterms + 7) / 8);
	if(prec == TMFQS_FP64) {
		check_cuda(cudaFuncSetAttribute(k_obs_apply<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "observable smem");
		k_obs_apply<double><<<blocks, kAdjThreads, smem, c.stream>>>(static_cast<const double2 *>(psi), static_cast<double2 *>(lam), N, p,
		                                                              nbytes, dev_partials);
	} else {
		check_cuda(cudaFuncSetAttribute(k_obs_apply<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "observable smem");
		k_obs_apply<float><<<blocks, kAdjThreads, smem, c.stream>>>(static_cast<const float2 *>(psi), static_cast<float2 *>(lam), N, p,
		                                                             nbytes, dev_partials);
	}
	check_cuda(cudaGetLastError(), "observable");
	if(c.launches) ++*c.launches;
	return blocks;
}

void launch_sum_partials(const LaunchCtx &c, const double *partials, size_t chunk_doubles, const PartialChunks &t,
                         double *out) {
	if(t.count == 0) return;
	if(t.count > kMaxPendingSums) fail(TMFQS_ERR_LOGIC, "adjoint: partial-sum table size");
	for(unsigned i = 0; i < t.count; ++i)
		if(t.stride[i] == 0 || t.stride[i] > kMaxDiagRun || (size_t)t.blocks[i] * t.stride[i] > chunk_doubles)
			fail(TMFQS_ERR_LOGIC, "adjoint: partial-sum array shape");
	k_sum_partials<<<t.count, dim3(32, kMaxDiagRun), 0, c.stream>>>(partials, chunk_doubles, t, out);
	check_cuda(cudaGetLastError(), "partial sums");
	if(c.launches) ++*c.launches;
}

unsigned launch_grad_run(const LaunchCtx &c, int prec, void *lam, void *psi, unsigned n, const DiagEntry *entries,
                         unsigned count, bool uncompute_psi, double *dev_partials) {
	if(count == 0 || count > kMaxDiagRun) fail(TMFQS_ERR_LOGIC, "adjoint: diagonal run size");
	RunParams rp{};
	for(unsigned k = 0; k < count; ++k) {
		rp.mask[k] = entries[k].mask;
		rp.cr[k] = entries[k].cr;
		rp.ci[k] = entries[k].ci;
		rp.kind[k] = entries[k].kind;
	}
	rp.count = count;
	// The caller orders the entries that depend on bits 0-2 first; count them.
	rp.nvary = 0;
	while(rp.nvary < count && (entries[rp.nvary].kind == kDiagFlip || (entries[rp.nvary].mask & 7u))) ++rp.nvary;
	for(unsigned k = rp.nvary; k < count; ++k)
		if(entries[k].kind == kDiagFlip || (entries[k].mask & 7u)) rp.nvary = count;  // not ordered: no split
	const uint64_t N = 1ull << n;
	const unsigned blocks = adj_blocks(c, N);
	const int up = uncompute_psi ? 1 : 0;
	const unsigned nbytes = (n + 7) / 8;
	if(prec == TMFQS_FP64) {
		const size_t smem = grad_smem(sizeof(double), sizeof(double2), nbytes);
		check_cuda(cudaFuncSetAttribute(k_grad_run<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "gradient smem");
		k_grad_run<double, double><<<blocks, kAdjThreads, smem, c.stream>>>(static_cast<double2 *>(lam), static_cast<double2 *>(psi), N, rp,
		                                                                    nbytes, up, dev_partials);
	} else {
		const size_t smem = grad_smem(sizeof(float), sizeof(float2), nbytes);
		check_cuda(cudaFuncSetAttribute(k_grad_run<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "gradient smem");
		k_grad_run<float, float><<<blocks, kAdjThreads, smem, c.stream>>>(static_cast<float2 *>(lam), static_cast<float2 *>(psi), N, rp,
		                                                                  nbytes, up, dev_partials);
	}
	check_cuda(cudaGetLastError(), "gradient run");
	if(c.launches) ++*c.launches;
	return blocks;
}

}  // namespace tqb
