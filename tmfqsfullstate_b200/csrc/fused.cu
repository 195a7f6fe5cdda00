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
#include <functional>
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
	unsigned sw;               // shared-memory swizzle: slot of local index j is j ^ ((j >> sw) & 7)
	uint64_t o_begin;          // the launch runs tiles [o_begin, ntiles)
	double inv;                // 1.0 / std::sqrt(2.0), formed on the host (dense_state_backend.cpp:258)
};

// Thread layout of one H-chain op of a pass with K >= 7 local bits, built on
// the host (build_chain_map).  The op's 2^(K-1) butterflies are numbered by a
// pair index p = lane + 32 q; p's bits map to the local bits other than the
// Hadamard's in an order chosen so that a warp's lanes differ, where possible,
// only in bits that are no control of the chain.  A controlled phase whose
// control is not a lane bit is then applied by all lanes of a warp or by
// none: the per-amplitude loop over the set controls does not diverge, and
// skipped phases cost no issue slots.  Entry e of the chain is bit 63 - e of
// a mask.  The three lowest lane bits are, for each i < 3, local bit i or
// local bit K-3+i: with the swizzle j ^ ((j >> (K-3)) & 7) the 16-byte shared
// accesses of each quarter-warp then hit distinct banks.
struct ChainMap {
	uint64_t ml[32];   // per lane: the chain entries whose control is set in its offset
	uint64_t mr[128];  // per warp-iteration q: the same for its offset
	uint16_t jl[32];   // per lane: local index offset
	uint16_t jr[128];  // per q: local index offset
	uint64_t mall;     // the union of ml over the lanes
	uint32_t nq;       // number of q values, 2^(K-6); a thread takes kChainPairs consecutive q together
	uint32_t ilp;      // the low bits of q that are no control (their pairs share a mask): 0, 1 or 2
	uint32_t narrow;   // the chain has at most 32 entries: masks live in their high word
	uint32_t pad;
};
constexpr uint64_t kNoChainMap = ~0ull;

// Butterflies per thread in a mapped H-chain op: independent chains of
// dependent products that hide each other's latency.
constexpr unsigned kChainPairs = 4;

// Chain products over one 32-entry word of a warp-uniform mask `mw` (the
// union of the masks of all lanes and pairs; entry e = bit 31 - e of the
// word, ascending e = circuit order): every lane walks the same entries, reads
// each phase once (a shared-memory broadcast), and applies it to each of its
// amplitudes whose own mask has it -- a separately rounded complex product
// (dense_state_backend.cpp:300-301), exactly as the per-gate path.
template <typename R, unsigned NP>
__device__ __forceinline__ void chain_word(uint32_t mw, const uint32_t (&mk)[NP], const double2 *cph, R (&r)[NP],
                                           R (&i)[NP]) {
	while(mw) {
		const unsigned e = __clz(mw);
		const uint32_t bit = 0x80000000u >> e;
		mw ^= bit;
		const double2 ph = cph[e];
		const R pr = (R)ph.x, pi = (R)ph.y;
#pragma unroll
		for(unsigned k = 0; k < NP; ++k)
			if(mk[k] & bit) cmul_ref(pr, pi, r[k], i[k]);
	}
}

__device__ __forceinline__ uint64_t expand_outer(uint64_t o, const FusedGeom &g) {
	for(unsigned i = 0; i < g.K; ++i) o = insert0(o, g.lpos[i]);
	return o;
}

template <typename R>
__device__ __forceinline__ bool is_zero(typename Vec2<R>::type v) {
	return v.x == R(0) && v.y == R(0);
}

// Hadamard butterfly of dense_state_backend.cpp:265-271 (skips all-zero pairs).
template <typename R>
__device__ __forceinline__ bool butterfly(typename Vec2<R>::type &x, typename Vec2<R>::type &y, R inv) {
	if(is_zero<R>(x) && is_zero<R>(y)) return false;
	typename Vec2<R>::type o0, o1;
	o0.x = rmul(radd(x.x, y.x), inv);
	o0.y = rmul(radd(x.y, y.y), inv);
	o1.x = rmul(rsub(x.x, y.x), inv);
	o1.y = rmul(rsub(x.y, y.y), inv);
	x = o0;
	y = o1;
	return true;
}

template <typename R>
__global__ void __launch_bounds__(kFusedThreads, 3) k_fused(typename Vec2<R>::type *a, FusedGeom g, const FusedOp *ops,
                                                            const ChainEntry *chain, const ChainMap *maps) {
	typedef typename Vec2<R>::type V;
	extern __shared__ unsigned char smem_raw[];
	const unsigned T = 1u << g.K;
	V *s = reinterpret_cast<V *>(smem_raw);
	uint64_t *hitab = reinterpret_cast<uint64_t *>(s + T);
	const unsigned nhi = 1u << (g.K - g.m);
	// Per-tile compacted chain of the current H-chain op: its entries whose
	// other bit is local (applied when that bit is set) or an outer bit that
	// is set in this tile (applied to every |1> output).
	__shared__ double2 cph[64];
	__shared__ int cloc[64];
	__shared__ unsigned ccount;
	__shared__ uint64_t cu;  // mapped chains: entries whose control is an outer bit set in this tile
	// The current chain op's thread layout, staged from the program (tile-independent).
	__shared__ uint64_t sml[32], smr[128];
	__shared__ uint16_t sjl[32], sjr[128];
	// Twiddle form: table A (outer phase x first 6 local controls) and table B
	// (next 5 local controls), built per tile in FP64.
	__shared__ double2 twa[64], twb[32];
	__shared__ int tla[6], tlb[5];
	__shared__ int tna, tnb;
	// A chunk of a run of diagonal ops, staged for the per-amplitude loop.
	constexpr unsigned kDiagChunk = 32;
	__shared__ uint64_t dmask[kDiagChunk];
	__shared__ double2 dph[kDiagChunk];
	__shared__ int dflip[kDiagChunk];
	for(unsigned h = threadIdx.x; h < nhi; h += blockDim.x) {
		uint64_t v = 0;
		for(unsigned i = 0; i < g.K - g.m; ++i)
			if((h >> i) & 1u) v |= 1ull << g.lpos[g.m + i];
		hitab[h] = v;
	}
	__syncthreads();
	const unsigned lane = threadIdx.x & 31u;
	const unsigned lowmask = (1u << g.m) - 1u;
	auto scatter = [&](unsigned j) -> uint64_t { return (uint64_t)(j & lowmask) | hitab[j >> g.m]; };
	// Shared slot of local index j (swizzled; the identity for small tiles).
	auto P = [&](unsigned j) -> unsigned { return j ^ ((j >> g.sw) & 7u); };
	const unsigned half = T >> 1, quarter = T >> 2;
	const R inv = (R)g.inv;
	for(uint64_t o = g.o_begin + blockIdx.x; o < g.ntiles; o += gridDim.x) {
		const uint64_t base = expand_outer(o, g);
		for(unsigned j = threadIdx.x; j < T; j += blockDim.x) s[P(j)] = a[base | scatter(j)];
		__syncthreads();
		for(unsigned k = 0; k < g.nops; ++k) {
			const FusedOp op = ops[k];
			switch(op.kind) {
				case kFH: {
					for(unsigned p = threadIdx.x; p < half; p += blockDim.x) {
						const unsigned j0 = (unsigned)insert0(p, op.lt), j1 = j0 | (1u << op.lt);
						V x = s[P(j0)], y = s[P(j1)];
						if(!butterfly<R>(x, y, inv)) continue;
						s[P(j0)] = x;
						s[P(j1)] = y;
					}
					__syncthreads();
					break;
				}
				case kFHChain: {
					if(op.state != kNoChainMap) {
						// Phases of all entries, and the outer-controlled entries that
						// apply in this tile (every |1> output gets them).
						if(threadIdx.x < 32) {
							uint64_t u = 0;
							for(unsigned e0 = 0; e0 < op.lc; e0 += 32) {
								const unsigned e = e0 + lane;
								bool on = false;
								if(e < op.lc) {
									const ChainEntry ce = chain[op.tab + e];
									cph[e] = make_double2(ce.cr, ce.ci);
									on = ce.local < 0 && ((base >> ce.bit) & 1ull);
								}
								const unsigned b = __ballot_sync(0xffffffffu, on);
								u |= (uint64_t)__brev(b) << (e0 == 0 ? 32 : 0);
							}
							if(lane == 0) cu = u;
						} else {
							// The other warps stage the op's layout in shared memory.
							const ChainMap &gm = maps[op.state];
							for(unsigned k = threadIdx.x - 32; k < gm.nq; k += blockDim.x - 32) {
								smr[k] = gm.mr[k];
								sjr[k] = gm.jr[k];
							}
							if(threadIdx.x < 64) {
								sml[threadIdx.x - 32] = gm.ml[threadIdx.x - 32];
								sjl[threadIdx.x - 32] = gm.jl[threadIdx.x - 32];
							}
						}
						__syncthreads();
						const ChainMap &cm = maps[op.state];
						const unsigned tb = 1u << op.lt, jl = sjl[lane];
						const uint64_t mlane = sml[lane] | cu;
						const unsigned warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
						// Two butterflies per thread (q and q+1): two independent chains
						// of dependent products.  Their |1> outputs share one mask when the
						// bit they differ in is no control.
						const unsigned nq = cm.nq;
						const bool narrow = cm.narrow != 0;
						const uint64_t mall = cm.mall | cu;  // the entries any lane of a warp can need
						constexpr unsigned NP = kChainPairs;
						for(unsigned q0 = NP * warp; q0 < nq; q0 += NP * nw) {
							unsigned jk[NP];
							uint64_t mk[NP];
							V x[NP], y[NP];
							bool w[NP];
							uint64_t mw = mall;
#pragma unroll
							for(unsigned k = 0; k < NP; ++k) {
								jk[k] = jl | sjr[q0 + k];
								mk[k] = mlane | smr[q0 + k];
								mw |= smr[q0 + k];
								x[k] = s[P(jk[k])];
								y[k] = s[P(jk[k] | tb)];
								w[k] = butterfly<R>(x[k], y[k], inv);
							}
							R r[NP], im[NP];
							uint32_t hi[NP], lo[NP];
#pragma unroll
							for(unsigned k = 0; k < NP; ++k) {
								// A zero |1> output is left alone by every phase (dense_state_backend.cpp:299).
								const bool c = w[k] && !is_zero<R>(y[k]);
								hi[k] = c ? (uint32_t)(mk[k] >> 32) : 0u;
								lo[k] = c ? (uint32_t)mk[k] : 0u;
								r[k] = y[k].x;
								im[k] = y[k].y;
							}
							chain_word<R, NP>((uint32_t)(mw >> 32), hi, cph, r, im);
							if(!narrow) chain_word<R, NP>((uint32_t)mw, lo, cph + 32, r, im);
#pragma unroll
							for(unsigned k = 0; k < NP; ++k) {
								if(!w[k]) continue;
								y[k].x = r[k];
								y[k].y = im[k];
								s[P(jk[k])] = x[k];
								s[P(jk[k] | tb)] = y[k];
							}
						}
						__syncthreads();
						break;
					}
					if(threadIdx.x < 32) {
						unsigned pos = 0;
						for(unsigned e0 = 0; e0 < op.lc; e0 += 32) {
							const unsigned e = e0 + lane;
							bool keep = false;
							ChainEntry ce{};
							if(e < op.lc) {
								ce = chain[op.tab + e];
								keep = ce.local >= 0 || ((base >> ce.bit) & 1ull);
							}
							const unsigned m = __ballot_sync(0xffffffffu, keep);
							const unsigned off = pos + __popc(m & ((1u << lane) - 1u));
							if(keep) {
								cph[off] = make_double2(ce.cr, ce.ci);
								cloc[off] = ce.local;
							}
							pos += __popc(m);
						}
						if(lane == 0) ccount = pos;
					}
					__syncthreads();
					const unsigned cnt = ccount;
					// Two butterflies per iteration: their chains are independent and
					// see the same tile-uniform outer phases (ILP).
					for(unsigned p0 = threadIdx.x; p0 < half; p0 += 2 * blockDim.x) {
						const unsigned p1 = p0 + blockDim.x;
						const bool has1 = p1 < half;
						const unsigned j00 = (unsigned)insert0(p0, op.lt), j01 = j00 | (1u << op.lt);
						const unsigned j10 = has1 ? (unsigned)insert0(p1, op.lt) : j00, j11 = j10 | (1u << op.lt);
						V x0 = s[P(j00)], y0 = s[P(j01)], x1 = s[P(j10)], y1 = s[P(j11)];
						const bool w0 = butterfly<R>(x0, y0, inv);
						const bool w1 = has1 && butterfly<R>(x1, y1, inv);
						// A zero |1> output is left alone by every phase of the chain
						// (dense_state_backend.cpp:299); a nonzero one stays nonzero.
						const bool c0 = w0 && !is_zero<R>(y0), c1 = w1 && !is_zero<R>(y1);
						if(c0 || c1) {
							R r0 = y0.x, i0 = y0.y, r1 = y1.x, i1 = y1.y;
							for(unsigned e = 0; e < cnt; ++e) {
								const double2 ph = cph[e];
								const int l = cloc[e];
								const R pr = (R)ph.x, pi = (R)ph.y;
								// An entry whose local bit is clear leaves the value as it is
								// (a product with (1, 0) could turn a -0 component into +0);
								// the products run under the condition, not through a select.
								const bool on0 = l < 0 || ((j01 >> l) & 1u), on1 = l < 0 || ((j11 >> l) & 1u);
								if(on0) cmul_ref(pr, pi, r0, i0);
								if(on1) cmul_ref(pr, pi, r1, i1);
							}
							if(c0) {
								y0.x = r0;
								y0.y = i0;
							}
							if(c1) {
								y1.x = r1;
								y1.y = i1;
							}
						}
						if(w0) {
							s[P(j00)] = x0;
							s[P(j01)] = y0;
						}
						if(w1) {
							s[P(j10)] = x1;
							s[P(j11)] = y1;
						}
					}
					__syncthreads();
					break;
				}
				case kFHTwiddle: {
					if(threadIdx.x < 96) {
						double outer = 0.0;
						int nl = 0;
						int lidx[11];
						double lth[11];
						for(unsigned e = 0; e < op.lc; ++e) {
							const ChainEntry ce = chain[op.tab + e];
							if(ce.local < 0) {
								if((base >> ce.bit) & 1ull) outer += ce.theta;
							} else if(nl < 11) {
								lidx[nl] = ce.local;
								lth[nl] = ce.theta;
								++nl;
							}
						}
						const int na = nl < 6 ? nl : 6, nb = nl - na;
						double ang = 0.0;
						bool active = false;
						unsigned m = 0;
						if(threadIdx.x < 64) {
							m = threadIdx.x;
							active = m < (1u << na);
							ang = outer;
							for(int i = 0; i < na; ++i)
								if((m >> i) & 1u) ang += lth[i];
						} else {
							m = threadIdx.x - 64;
							active = m < (1u << nb);
							for(int i = 0; i < nb; ++i)
								if((m >> i) & 1u) ang += lth[na + i];
						}
						if(active) {
							double sv, cv;
							sincos(ang, &sv, &cv);
							if(threadIdx.x < 64) twa[m] = make_double2(cv, sv);
							else twb[m] = make_double2(cv, sv);
						}
						if(threadIdx.x == 0) {
							for(int i = 0; i < na; ++i) tla[i] = lidx[i];
							for(int i = 0; i < nb; ++i) tlb[i] = lidx[na + i];
							tna = na;
							tnb = nb;
						}
					}
					__syncthreads();
					const int na = tna, nb = tnb;
					for(unsigned p = threadIdx.x; p < half; p += blockDim.x) {
						const unsigned j0 = (unsigned)insert0(p, op.lt), j1 = j0 | (1u << op.lt);
						V x = s[P(j0)], y = s[P(j1)];
						if(!butterfly<R>(x, y, inv)) continue;
						if(!is_zero<R>(y)) {
							unsigned ia = 0, ib = 0;
							for(int i = 0; i < na; ++i) ia |= ((j1 >> tla[i]) & 1u) << i;
							for(int i = 0; i < nb; ++i) ib |= ((j1 >> tlb[i]) & 1u) << i;
							const double2 ta = twa[ia], tb = twb[ib];
							// Twiddle formed in FP64 and rounded once to the storage type.
							const R tr = (R)fma(ta.x, tb.x, -(ta.y * tb.y));
							const R ti = (R)fma(ta.x, tb.y, ta.y * tb.x);
							const R nr = fma(tr, y.x, -(ti * y.y));
							const R ni = fma(tr, y.y, ti * y.x);
							y.x = nr;
							y.y = ni;
						}
						s[P(j0)] = x;
						s[P(j1)] = y;
					}
					__syncthreads();
					break;
				}
				case kFX:
				case kFCnot: {
					for(unsigned p = threadIdx.x; p < half; p += blockDim.x) {
						const unsigned j0 = (unsigned)insert0(p, op.lt), j1 = j0 | (1u << op.lt);
						if(op.kind == kFCnot && ((base | scatter(j0)) & op.mask) == 0) continue;
						const V x = s[P(j0)], y = s[P(j1)];
						if(x.x == y.x && x.y == y.y) continue;
						s[P(j0)] = y;
						s[P(j1)] = x;
					}
					__syncthreads();
					break;
				}
				case kFSwap: {
					const unsigned lo = op.lt < op.lc ? op.lt : op.lc, hi = op.lt < op.lc ? op.lc : op.lt;
					for(unsigned q = threadIdx.x; q < quarter; q += blockDim.x) {
						const unsigned j = (unsigned)insert00(q, lo, hi);
						const unsigned ja = j | (1u << op.lt), jb = j | (1u << op.lc);
						const V x = s[P(ja)], y = s[P(jb)];
						s[P(ja)] = y;
						s[P(jb)] = x;
					}
					__syncthreads();
					break;
				}
				case kFCP:
				case kFFlip: {
					// A run of consecutive diagonal ops in one sweep: each amplitude
					// still receives them one by one, in circuit order.
					unsigned e = k + 1;
					while(e < g.nops && e - k < kDiagChunk && (ops[e].kind == kFCP || ops[e].kind == kFFlip)) ++e;
					const unsigned cnt = e - k;
					for(unsigned q = threadIdx.x; q < cnt; q += blockDim.x) {
						const FusedOp d = ops[k + q];
						dflip[q] = d.kind == kFFlip;
						dmask[q] = d.kind == kFFlip ? d.state : d.mask;
						dph[q] = make_double2(d.cr, d.ci);
					}
					__syncthreads();
					for(unsigned j = threadIdx.x; j < T; j += blockDim.x) {
						const uint64_t x = base | scatter(j);
						V v = s[P(j)];
						bool dirty = false;
						for(unsigned q = 0; q < cnt; ++q) {
							const uint64_t m = dmask[q];
							if(!dflip[q]) {
								// Zero amplitudes are skipped (dense_state_backend.cpp:299).
								if((x & m) != m || (v.x == R(0) && v.y == R(0))) continue;
								const double2 ph = dph[q];
								cmul_ref((R)ph.x, (R)ph.y, v.x, v.y);
							} else {
								if(x != m) continue;
								v.x = -v.x;
								v.y = -v.y;
							}
							dirty = true;
						}
						if(dirty) s[P(j)] = v;
					}
					// Diagonal ops keep the thread->amplitude ownership; the barrier
					// also frees the staged chunk.
					__syncthreads();
					k = e - 1;
					break;
				}
				default:
					break;
			}
		}
		for(unsigned j = threadIdx.x; j < T; j += blockDim.x) a[base | scatter(j)] = s[P(j)];
		__syncthreads();
	}
}

// ---------------------------------------------------------------------------
// In-place bit permutation for disjoint transpositions of bit positions.
// Local set S = low bits {0..r-1} plus their images; the remaining ("outer")
// bits are permuted among themselves, so tile o maps to tile perm(o).  A CTA
// loads tile o and its partner, then writes each to the other's slot with the
// local bits permuted; tiles fixed by the permutation are permuted alone.
// Both the permutation of the local index and the shared-memory swizzle are
// bit-linear, so each is two table lookups (low and high halves of the index).
// The swizzle XORs the bits that the low bits map to into the low bits: the
// linear writes and the permuted reads then both spread over the banks.
// ---------------------------------------------------------------------------
constexpr unsigned kPermMaxLocal = 12;
constexpr unsigned kPermThreads = 256;
constexpr unsigned kPermHalf = 6;  // index bits per lookup table
constexpr unsigned kPermChunks = 4;  // 6-bit chunks of the tile index (up to 24 outer bits)
constexpr unsigned kPermGranules = 4;  // 16-byte granules per thread per tile (tiles of <= 16 KB)

// Local bits of a permutation tile: two tiles of 16 KB.
template <typename R>
constexpr unsigned perm_max_local() {
	return sizeof(R) == 8 ? 10u : 11u;
}

struct PermGeom {
	unsigned n, K, m;
	unsigned lpos[kPermMaxLocal];
	unsigned npairs;
	unsigned pa[32], pb[32];       // all transposed bit-position pairs
	uint64_t ntiles;
	uint16_t perm_lo[1 << kPermHalf], perm_hi[1 << kPermHalf];  // local index permutation
	uint16_t swz_lo[1 << kPermHalf], swz_hi[1 << kPermHalf];    // shared-memory swizzle (XOR)
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

// One 16-byte granule: two complex64 or one complex128 amplitude.
__device__ __forceinline__ void store_granule(float2 *p, const float2 (&y)[2]) {
	*reinterpret_cast<float4 *>(p) = make_float4(y[0].x, y[0].y, y[1].x, y[1].y);
}
__device__ __forceinline__ void store_granule(double2 *p, const double2 (&y)[1]) { *p = y[0]; }

template <typename R>
__global__ void __launch_bounds__(kPermThreads) k_bit_perm(typename Vec2<R>::type *a, PermGeom g) {
	typedef typename Vec2<R>::type V;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const unsigned T = 1u << g.K;
	// Two buffers, each the tile and its partner; the next pair's copies are in
	// flight while the current pair is written out.
	V *buf = reinterpret_cast<V *>(smem_raw);
	uint64_t *hitab = reinterpret_cast<uint64_t *>(buf + 4 * T);
	// Tile o -> (its base, the partner's base, the partner's tile index): all
	// three maps are bit-linear, so they are ORs of per-chunk table entries.
	uint64_t *otab = hitab + (1u << (g.K - g.m));  // [kPermChunks][64][3]
	uint16_t *tabs = reinterpret_cast<uint16_t *>(otab + kPermChunks * 64 * 3);
	const unsigned nhi = 1u << (g.K - g.m), H = 1u << kPermHalf, hm = H - 1u;
	for(unsigned e = threadIdx.x; e < kPermChunks * 64; e += blockDim.x) {
		uint64_t base = (uint64_t)(e & 63u) << (6u * (e >> 6));
		for(unsigned i = 0; i < g.K; ++i) base = insert0(base, g.lpos[i]);
		const uint64_t pbase = perm_global(base, g);
		otab[3 * e] = base;
		otab[3 * e + 1] = pbase;
		otab[3 * e + 2] = compress_outer(pbase, g);
	}
	for(unsigned h = threadIdx.x; h < nhi; h += blockDim.x) {
		uint64_t v = 0;
		for(unsigned i = 0; i < g.K - g.m; ++i)
			if((h >> i) & 1u) v |= 1ull << g.lpos[g.m + i];
		hitab[h] = v;
	}
	for(unsigned k = threadIdx.x; k < H; k += blockDim.x) {
		tabs[k] = g.perm_lo[k];
		tabs[H + k] = g.perm_hi[k];
		tabs[2 * H + k] = g.swz_lo[k];
		tabs[3 * H + k] = g.swz_hi[k];
	}
	__syncthreads();
	const unsigned lowmask = (1u << g.m) - 1u;
	auto scatter = [&](unsigned j) -> uint64_t { return (uint64_t)(j & lowmask) | hitab[j >> g.m]; };
	auto perm = [&](unsigned j) -> unsigned { return (unsigned)tabs[j & hm] | tabs[H + (j >> kPermHalf)]; };
	auto phys = [&](unsigned j) -> unsigned { return j ^ tabs[2 * H + (j & hm)] ^ tabs[3 * H + (j >> kPermHalf)]; };
	struct Work {
		uint64_t o, base, pbase, po;
	};
	auto work_at = [&](uint64_t o) -> Work {
		Work w{o, 0, 0, 0};
#pragma unroll
		for(unsigned c = 0; c < kPermChunks; ++c) {
			const uint64_t *t = otab + 3 * ((c << 6) | (unsigned)((o >> (6u * c)) & 63u));
			w.base |= t[0];
			w.pbase |= t[1];
			w.po |= t[2];
		}
		return w;
	};
	// The first tile of this CTA at or after o whose partner is not smaller
	// (a pair is handled once, by its smaller tile).
	auto next_work = [&](uint64_t o) -> Work {
		for(; o < g.ntiles; o += gridDim.x) {
			const Work w = work_at(o);
			if(w.po >= w.o) return w;
		}
		return Work{g.ntiles, 0, 0, 0};
	};
	// Global memory moves in 16-byte granules of G consecutive amplitudes
	// (local bit 0 is global bit 0).  The swizzle keeps granules whole.  A
	// thread's granules (q = tid + i * blockDim) and the shared slots its
	// outputs come from are the same for every tile: mapped once, here.
	constexpr unsigned G = 16 / sizeof(V);
	const unsigned TG = T / G;
	uint64_t goff[kPermGranules];
	unsigned pslot[kPermGranules], src[kPermGranules][G];
	bool gv[kPermGranules];
#pragma unroll
	for(unsigned i = 0; i < kPermGranules; ++i) {
		const unsigned q = threadIdx.x + i * blockDim.x;
		gv[i] = q < TG;
		const unsigned j = gv[i] ? q * G : 0u;
		goff[i] = scatter(j);
		pslot[i] = phys(j);
#pragma unroll
		for(unsigned e = 0; e < G; ++e) src[i][e] = phys(perm(j + e));  // involution: source of slot j+e
	}
	auto prefetch = [&](const Work &w, V *dst) {
		if(w.o < g.ntiles) {
			const bool pair = w.po != w.o;
#pragma unroll
			for(unsigned i = 0; i < kPermGranules; ++i)
				if(gv[i]) {
					cp_async16(dst + pslot[i], a + (w.base | goff[i]));
					if(pair) cp_async16(dst + T + pslot[i], a + (w.pbase | goff[i]));
				}
		}
		cp_async_commit();
	};
	Work cur = next_work(blockIdx.x);
	unsigned sel = 0;
	prefetch(cur, buf);
	while(cur.o < g.ntiles) {
		const Work nxt = next_work(cur.o + gridDim.x);
		prefetch(nxt, buf + 2 * T * (sel ^ 1u));
		cp_async_wait1();
		__syncthreads();
		const V *A = buf + 2 * T * sel, *B = A + T;
		const bool pair = cur.po != cur.o;
		// amplitude (base|scatter(j)) moves to (pbase|scatter(perm(j))).
#pragma unroll
		for(unsigned i = 0; i < kPermGranules; ++i) {
			if(!gv[i]) continue;
			V ya[G], yb[G];
#pragma unroll
			for(unsigned e = 0; e < G; ++e) {
				ya[e] = A[src[i][e]];
				if(pair) yb[e] = B[src[i][e]];
			}
			store_granule(a + (cur.pbase | goff[i]), ya);
			if(pair) store_granule(a + (cur.base | goff[i]), yb);
		}
		__syncthreads();  // every read of this buffer is done before it is refilled
		cur = nxt;
		sel ^= 1u;
	}
	cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// Temporal Grover pass.
// ---------------------------------------------------------------------------
// v <- t - v for one amplitude: exactly the rounded subtraction (complex64
// uses one paired instruction, fma(v, -1, t) rounds once like t - v).
__device__ __forceinline__ void grover_step(double2 &v, double2 t) {
	v.x = rsub(t.x, v.x);
	v.y = rsub(t.y, v.y);
}
__device__ __forceinline__ void grover_step(float2 &v, float2 t) { v = __ffma2_rn(v, make_float2(-1.0f, -1.0f), t); }

// tm[k] = 2 * mean of iteration k, already rounded to the storage type.
template <typename R, unsigned kPer>
__global__ void __launch_bounds__(256) k_grover_temporal(typename Vec2<R>::type *a, uint64_t N,
                                                        const typename Vec2<R>::type *tm, uint64_t iters,
                                                        uint64_t flip_from, const uint64_t *marked, unsigned nm) {
	typedef typename Vec2<R>::type V;
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
			uint64_t k = 0;
			// Four means per trip, loaded ahead of the dependent updates.
			for(; k + 4 <= iters; k += 4) {
				const V t0 = tm[k], t1 = tm[k + 1], t2 = tm[k + 2], t3 = tm[k + 3];
#pragma unroll
				for(unsigned u = 0; u < kPer; ++u) {
					grover_step(v[u], t0);
					grover_step(v[u], t1);
					grover_step(v[u], t2);
					grover_step(v[u], t3);
				}
			}
			for(; k < iters; ++k) {
				const V t = tm[k];
#pragma unroll
				for(unsigned u = 0; u < kPer; ++u) grover_step(v[u], t);
			}
		} else {
			for(uint64_t k = 0; k < iters; ++k) {
				const V t = tm[k];
#pragma unroll
				for(unsigned u = 0; u < kPer; ++u) {
					if(mk[u] && k >= flip_from) {
						v[u].x = -v[u].x;
						v[u].y = -v[u].y;
					}
					grover_step(v[u], t);
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

// Thread layout of an H-chain op (see ChainMap): the pair index's bits, in
// order, are local bits of the tile other than the Hadamard's.  Lane bits
// 0-2: local bit K-3+i when it is no control of the chain, else local bit i;
// lane bits 3-4 and the bit shared by a thread's two butterflies: bits that
// are no control first; then the rest.
ChainMap build_chain_map(const FusedPass &pass, const FusedOp &op) {
	const unsigned K = pass.K, lt = op.lt;
	uint32_t ctrl = 0;
	std::vector<std::pair<unsigned, unsigned>> loc;  // (entry, local bit) of the local controls
	for(unsigned e = 0; e < op.lc; ++e) {
		const ChainEntry &ce = pass.chain[op.tab + e];
		if(ce.local >= 0) {
			ctrl |= 1u << ce.local;
			loc.push_back({e, (unsigned)ce.local});
		}
	}
	auto is_free = [&](unsigned b) { return b != lt && !((ctrl >> b) & 1u); };
	uint32_t used = 1u << lt;
	std::vector<unsigned> order;
	auto take = [&](unsigned b) {
		order.push_back(b);
		used |= 1u << b;
	};
	for(unsigned i = 0; i < 3; ++i) {
		const unsigned hi = K - 3 + i;
		if(is_free(hi)) take(hi);
		else if(i != lt) take(i);
		else take(hi);
	}
	auto next = [&](bool want_free) -> int {
		for(unsigned b = 0; b < K; ++b)
			if(!((used >> b) & 1u) && (!want_free || is_free(b))) return (int)b;
		return -1;
	};
	for(unsigned i = 3; i < 5; ++i) {
		int b = next(true);
		if(b < 0) b = next(false);
		take((unsigned)b);
	}
	// Bits 0 and 1 of q: the bits a thread's butterflies differ in (free ones first).
	unsigned nfree = 0;
	for(unsigned i = 0; i < 2 && order.size() < K - 1; ++i) {
		int b = next(true);
		if(b >= 0 && nfree == i) ++nfree;
		if(b < 0) b = next(false);
		take((unsigned)b);
	}
	for(int b = next(false); b >= 0; b = next(false)) take((unsigned)b);
	if(order.size() != K - 1) fail(TMFQS_ERR_LOGIC, "fused pass: chain layout");
	ChainMap m{};
	m.nq = 1u << (K - 6);
	m.ilp = nfree;
	m.narrow = op.lc <= 32 ? 1u : 0u;
	auto mask_of = [&](unsigned j) {
		uint64_t r = 0;
		for(const auto &pe : loc)
			if((j >> pe.second) & 1u) r |= 1ull << (63 - pe.first);
		return r;
	};
	for(unsigned l = 0; l < 32; ++l) {
		unsigned j = 0;
		for(unsigned i = 0; i < 5; ++i)
			if((l >> i) & 1u) j |= 1u << order[i];
		m.jl[l] = (uint16_t)j;
		m.ml[l] = mask_of(j);
		m.mall |= m.ml[l];
	}
	for(unsigned q = 0; q < m.nq; ++q) {
		unsigned j = 0;
		for(unsigned i = 0; 5 + i < K - 1; ++i)
			if((q >> i) & 1u) j |= 1u << order[5 + i];
		m.jr[q] = (uint16_t)j;
		m.mr[q] = mask_of(j);
	}
	return m;
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
	g.o_begin = 0;
	if(pass.tile_end) {
		if(pass.tile_begin >= pass.tile_end || pass.tile_end > g.ntiles) fail(TMFQS_ERR_LOGIC, "fused pass: bad tile range");
		g.o_begin = pass.tile_begin;
		g.ntiles = pass.tile_end;
	}
	g.nops = (unsigned)pass.ops.size();
	g.inv = 1.0 / std::sqrt(2.0);
	// Tiles of >= 7 local bits: swizzled shared memory and per-chain thread layouts.
	const bool mapped = pass.K >= 7;
	g.sw = mapped ? pass.K - 3 : 31u;
	std::vector<FusedOp> ops(pass.ops);
	std::vector<ChainMap> maps;
	for(auto &op : ops) {
		if(op.kind != kFHChain) continue;
		if(mapped && op.lc <= 64) {
			op.state = maps.size();
			maps.push_back(build_chain_map(pass, op));
		} else {
			op.state = kNoChainMap;
		}
	}
	const size_t ops_bytes = ops.size() * sizeof(FusedOp);
	const size_t ph_off = (ops_bytes + 255) & ~size_t(255);
	const size_t ch_bytes = std::max<size_t>(32, pass.chain.size() * sizeof(ChainEntry));
	const size_t map_off = (ph_off + ch_bytes + 255) & ~size_t(255);
	const size_t need = map_off + std::max<size_t>(32, maps.size() * sizeof(ChainMap));
	if(need > dev_prog_bytes) {
		if(dev_prog) {
			check_cuda(cudaStreamSynchronize(c.stream), "fused program sync");
			cudaFree(dev_prog);
		}
		dev_prog = nullptr;
		dev_prog_bytes = 0;
		if(device_alloc(&dev_prog, need * 2) != cudaSuccess) {
			cudaGetLastError();
			fail(TMFQS_ERR_NOMEM, "fused pass program allocation failed");
		}
		dev_prog_bytes = need * 2;
	}
	// The program buffer is reused: the upload is ordered on the stream after the pass that read it last.
	std::vector<unsigned char> host(need, 0);
	std::memcpy(host.data(), ops.data(), ops_bytes);
	if(!pass.chain.empty()) std::memcpy(host.data() + ph_off, pass.chain.data(), pass.chain.size() * sizeof(ChainEntry));
	if(!maps.empty()) std::memcpy(host.data() + map_off, maps.data(), maps.size() * sizeof(ChainMap));
	upload_async(c, dev_prog, host.data(), need, "fused program upload");
	const size_t smem = (sizeof(typename Vec2<R>::type) << pass.K) + (sizeof(uint64_t) << (pass.K - g.m));
	check_cuda(cudaFuncSetAttribute(k_fused<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "fused smem");
	int per_sm = 1;
	check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<R>, kFusedThreads, smem), "fused occupancy");
	const uint64_t grid = std::min<uint64_t>(g.ntiles - g.o_begin, (uint64_t)c.num_sms * std::max(1, per_sm));
	k_fused<R><<<(unsigned)grid, kFusedThreads, smem, c.stream>>>(
		static_cast<typename Vec2<R>::type *>(a), g, static_cast<const FusedOp *>(dev_prog),
		reinterpret_cast<const ChainEntry *>(static_cast<unsigned char *>(dev_prog) + ph_off),
		reinterpret_cast<const ChainMap *>(static_cast<unsigned char *>(dev_prog) + map_off));
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
	const unsigned maxK = perm_max_local<R>();
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
	if(g.m < 1) fail(TMFQS_ERR_LOGIC, "bit permutation: bit 0 must be local");
	std::vector<unsigned> lmap(g.K);
	for(unsigned i = 0; i < g.K; ++i) {
		g.lpos[i] = best[i];
		const unsigned target = (unsigned)img[best[i]];
		lmap[i] = (unsigned)(std::find(best.begin(), best.end(), target) - best.begin());
	}
	// Swizzled bits: the 16-byte granule index within 128 bytes (bits s0 to
	// s0+2 of the local index), so copies of whole granules stay contiguous.
	const unsigned s0 = sizeof(R) == 8 ? 0u : 1u, b = std::min<unsigned>(g.K, s0 + 3u);
	auto perm_of = [&](unsigned j) {
		unsigned r = 0;
		for(unsigned i = 0; i < g.K; ++i)
			if((j >> i) & 1u) r |= 1u << lmap[i];
		return r;
	};
	// swizzle(j): for each bit s0 <= i < b whose image lmap[i] is at or above
	// b, the bit of j at lmap[i] is XORed into bit i.
	auto swz_of = [&](unsigned j) {
		unsigned x = 0;
		for(unsigned i = s0; i < b; ++i)
			if(lmap[i] >= b && ((j >> lmap[i]) & 1u)) x |= 1u << i;
		return x;
	};
	const unsigned H = 1u << kPermHalf;
	for(unsigned k = 0; k < H; ++k) {
		const unsigned lo = k < (1u << std::min(g.K, kPermHalf)) ? k : 0u;
		const unsigned hi = g.K > kPermHalf && k < (1u << (g.K - kPermHalf)) ? (k << kPermHalf) : 0u;
		g.perm_lo[k] = (uint16_t)perm_of(lo);
		g.perm_hi[k] = (uint16_t)perm_of(hi);
		g.swz_lo[k] = (uint16_t)swz_of(lo);
		g.swz_hi[k] = (uint16_t)swz_of(hi);
	}
	g.ntiles = 1ull << (n - g.K);
	if(n - g.K > 6 * kPermChunks) fail(TMFQS_ERR_INVALID_ARGUMENT, "bit permutation: state too large");
	if((sizeof(typename Vec2<R>::type) << g.K) > 16 * kPermGranules * kPermThreads)
		fail(TMFQS_ERR_LOGIC, "bit permutation: tile larger than the per-thread granule maps");
	const size_t smem = 4 * (sizeof(typename Vec2<R>::type) << g.K) + (sizeof(uint64_t) << (g.K - g.m)) +
	                    sizeof(uint64_t) * kPermChunks * 64 * 3 + 4 * H * sizeof(uint16_t);
	check_cuda(cudaFuncSetAttribute(k_bit_perm<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "perm smem");
	int per_sm = 1;
	check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bit_perm<R>, kPermThreads, smem), "perm occupancy");
	const uint64_t grid = std::min<uint64_t>(g.ntiles, (uint64_t)c.num_sms * std::max(1, per_sm));
	k_bit_perm<R><<<(unsigned)grid, kPermThreads, smem, c.stream>>>(static_cast<typename Vec2<R>::type *>(a), g);
	after_launch(c, "bit permutation");
}

// ---------------------------------------------------------------------------
// Register stages for exact passes of Hadamards and H-chains (the QFT).
//
// A pass's ops are cut into stages of up to four consecutive Hadamard
// targets.  In a stage every thread holds the 16 amplitudes of the tile that
// differ only in the stage's four register bits and applies the stage's ops
// to them in circuit order, in registers: each Hadamard as 8 butterflies, each
// of its chain's controlled phases as separately rounded complex products on
// the |1> outputs whose control bit is set -- the same IEEE operations, in the
// same order per amplitude, as the per-gate path (dense_state_backend.cpp:
// 255-304), so the result is bit-identical.  The first stage reads the tile
// from HBM, the last writes it back, the ones between pass it on through
// shared memory with one barrier each.  Each Hadamard's 8 |1> outputs are 8
// independent chains of dependent products per thread.
//
// The control of a chain entry is an outer bit (set or not for the whole
// tile), a local bit that indexes the thread (set or not per thread), or a
// register bit (set for half of a thread's outputs).  Lanes walk the entries
// of their warp's union together (one broadcast phase load per entry), so an
// entry whose control is a lane bit costs every lane its products while half
// of them need none.  The host therefore picks per stage which local bits are
// register, lane and warp bits: fillers of the register bits are the most
// frequent controls, lanes the least frequent (no control at all wherever the
// tile has such bits).  The thread masks of every op come from host tables.
// ---------------------------------------------------------------------------
constexpr unsigned kStRB = 4;                    // register bits per stage
constexpr unsigned kStK = 12;                    // local bits of a tile (complex128: 64 KiB)
constexpr unsigned kStTB = kStK - kStRB;         // thread index bits (0-4: the lane, 5-7: the warp)
constexpr unsigned kStThreads = 1u << kStTB;
constexpr unsigned kStMaxOps = 16;
constexpr unsigned kStMaxStages = 8;
constexpr unsigned kStMaxEntries = 1024;
// Per-op table of 64-bit entry masks (entry e = bit 63 - e): the entries
// controlled by the thread index's low and high nibble, the union over each
// warp's lanes, the entries controlled by each register bit, their union.
constexpr unsigned kStTabLo = 0, kStTabHi = 16, kStTabWarp = 32, kStTabReg = 40, kStTabRegAll = 44, kStTabWords = 48;
// Per-stage table of 16-bit offsets: thread nibbles -> local index (lo, hi)
// and -> shared slot (lo, hi), register bits -> shared slot.
constexpr unsigned kStGeoTlo = 0, kStGeoThi = 16, kStGeoSlo = 32, kStGeoShi = 48, kStGeoReg = 64, kStGeoWords = 68;

struct StageGeom {
	unsigned n, m;
	unsigned lpos[kStK];
	uint64_t ntiles, o_begin;
	unsigned nops, nstages, nentries, narrow;
	double inv;
	uint8_t st_first[kStMaxStages], st_count[kStMaxStages];
	uint8_t rbit[kStMaxStages][kStRB];  // local bit of register bit i
	uint8_t tbit[kStMaxStages][kStTB];  // local bit of thread index bit k
	uint16_t geo[kStMaxStages][kStGeoWords];
	uint8_t op_reg[kStMaxOps];                     // register bit of the op's Hadamard
	uint16_t op_tab[kStMaxOps], op_lc[kStMaxOps];  // its chain: entries [tab, tab + lc) of the pass
	uint8_t op_split[kStMaxOps];                   // entries from here on have no register-bit control
	uint8_t op_outer[kStMaxOps];                   // the chain has entries controlled by outer bits
	uint8_t scol[kStK];                            // shared slot of j: j ^ XOR of scol[b] over bits b >= 3 of j
};

// The |1> output p (of the 8 of a Hadamard on register bit I) is register r1(p).
template <unsigned I>
__device__ __forceinline__ constexpr unsigned st_r1(unsigned p) {
	return ((p >> I) << (I + 1)) | (p & ((1u << I) - 1u)) | (1u << I);
}

// Zero tests on the bit patterns (+0 and -0 compare equal to zero; so does
// this), on the integer units instead of the FP64 pipe.
__device__ __forceinline__ unsigned st_bits_nonsign(double2 x) {
	return ((unsigned)(__double2hiint(x.x) | __double2hiint(x.y)) << 1) | (unsigned)__double2loint(x.x) |
	       (unsigned)__double2loint(x.y);
}
__device__ __forceinline__ unsigned st_bits_nonsign(float2 x) {
	return (__float_as_uint(x.x) | __float_as_uint(x.y)) << 1;
}

// Hadamard butterfly (dense_state_backend.cpp:265-271) without the zero test.
template <typename R>
__device__ __forceinline__ void st_bfly(typename Vec2<R>::type &x, typename Vec2<R>::type &y, R inv) {
	typename Vec2<R>::type o0, o1;
	o0.x = rmul(radd(x.x, y.x), inv);
	o0.y = rmul(radd(x.y, y.y), inv);
	o1.x = rmul(rsub(x.x, y.x), inv);
	o1.y = rmul(rsub(x.y, y.y), inv);
	x = o0;
	y = o1;
}

// One rounded complex product (dense_state_backend.cpp:300-301) on output p
// when `on`: computed unconditionally and kept by a select, so that the
// products of independent outputs interleave (a skipped product leaves the
// value exactly as it was).  ALLNZ: every output of the warp is nonzero.
template <typename R, bool ALLNZ>
__device__ __forceinline__ void st_cmul(R pr, R pi, typename Vec2<R>::type &x, bool on) {
	R re = x.x, im = x.y;
	cmul_ref(pr, pi, re, im);
	if(ALLNZ) {
		x.x = re;
		x.y = im;
	} else {
		x.x = on ? re : x.x;
		x.y = on ? im : x.y;
	}
}

// Products of one entry whose control is register bit J: the 4 outputs with
// bit J set (a compile-time subset).
template <typename R, unsigned I, unsigned J, bool ALLNZ>
__device__ __forceinline__ void st_apply_reg(R pr, R pi, const bool (&nz)[8], typename Vec2<R>::type (&v)[16]) {
#pragma unroll
	for(unsigned p = 0; p < 8; ++p)
		if((st_r1<I>(p) >> J) & 1u) st_cmul<R, ALLNZ>(pr, pi, v[st_r1<I>(p)], nz[p]);
}

// Walks one 32-entry word W (0: high word of the masks) of the warp's union
// of entries in circuit order.  An entry controlled by a register bit (ra)
// goes to the outputs with that bit set; any other entry (an outer bit or a
// thread bit: the same for all of this thread's outputs) to all 8 when the
// thread's mask tw has it.  The next entry's phase is loaded while this one's
// products run.
template <typename R, unsigned I, int W, bool ALLNZ>
__device__ __forceinline__ void stage_walk(uint32_t tw, const uint64_t (&rm)[kStRB], uint64_t rall, uint32_t w,
                                           const double2 *cph, const bool (&nz)[8], typename Vec2<R>::type (&v)[16]) {
	if(!w) return;
	const uint32_t ra = W ? (uint32_t)rall : (uint32_t)(rall >> 32);
	const uint32_t r0 = W ? (uint32_t)rm[0] : (uint32_t)(rm[0] >> 32), r1 = W ? (uint32_t)rm[1] : (uint32_t)(rm[1] >> 32);
	const uint32_t r2 = W ? (uint32_t)rm[2] : (uint32_t)(rm[2] >> 32);
	unsigned e = __clz(w);
	double2 c = cph[e];
	for(;;) {
		const uint32_t bit = 0x80000000u >> e;
		w ^= bit;
		const R pr = (R)c.x, pi = (R)c.y;
		if(w) {
			e = __clz(w);
			c = cph[e];
		}
		if(ra & bit) {
			if(r0 & bit) {
				if constexpr(I != 0) st_apply_reg<R, I, 0, ALLNZ>(pr, pi, nz, v);
			} else if(r1 & bit) {
				if constexpr(I != 1) st_apply_reg<R, I, 1, ALLNZ>(pr, pi, nz, v);
			} else if(r2 & bit) {
				if constexpr(I != 2) st_apply_reg<R, I, 2, ALLNZ>(pr, pi, nz, v);
			} else {
				if constexpr(I != 3) st_apply_reg<R, I, 3, ALLNZ>(pr, pi, nz, v);
			}
		} else if(tw & bit) {
#pragma unroll
			for(unsigned p = 0; p < 8; ++p) st_cmul<R, ALLNZ>(pr, pi, v[st_r1<I>(p)], nz[p]);
		}
		if(!w) break;
	}
}

// Walks one 32-entry word of entries that no register bit controls: each
// applies to all 8 outputs of the thread or to none (tw).
template <typename R, unsigned I, bool ALLNZ>
__device__ __forceinline__ void stage_walk_uniform(uint32_t tw, uint32_t w, const double2 *cph, const bool (&nz)[8],
                                                   typename Vec2<R>::type (&v)[16]) {
	if(!w) return;
	unsigned e = __clz(w);
	double2 c = cph[e];
	for(;;) {
		const uint32_t bit = 0x80000000u >> e;
		w ^= bit;
		const R pr = (R)c.x, pi = (R)c.y;
		if(w) {
			e = __clz(w);
			c = cph[e];
		}
		if(tw & bit) {
#pragma unroll
			for(unsigned p = 0; p < 8; ++p) st_cmul<R, ALLNZ>(pr, pi, v[st_r1<I>(p)], nz[p]);
		}
		if(!w) break;
	}
}

// One op of a stage: the Hadamard on register bit I (all-zero pairs are left
// as they are), then, for an H-chain, its controlled phases.
template <typename R, unsigned I, bool NARROW>
__device__ __forceinline__ void stage_hchain(typename Vec2<R>::type (&v)[16], R inv, bool chain, unsigned k,
                                             const StageGeom &g, const uint64_t *tab, const double2 *ph,
                                             const uint8_t *ebit, uint64_t base, unsigned t) {
	unsigned pz = 0;  // some pair of this thread is all zero
#pragma unroll
	for(unsigned p = 0; p < 8; ++p) {
		const unsigned r1 = st_r1<I>(p), r0 = r1 ^ (1u << I);
		pz |= (st_bits_nonsign(v[r0]) | st_bits_nonsign(v[r1])) == 0u;
	}
	const bool zeros = __any_sync(0xffffffffu, pz);  // the warp holds a zero pair (rare but for sparse states)
	if(zeros) {
		unsigned pall = 1;
#pragma unroll
		for(unsigned p = 0; p < 8; ++p) {
			const unsigned r1 = st_r1<I>(p), r0 = r1 ^ (1u << I);
			if((st_bits_nonsign(v[r0]) | st_bits_nonsign(v[r1])) != 0u) {
				st_bfly<R>(v[r0], v[r1], inv);
				pall = 0;
			}
		}
		// A warp whose pairs are all zero has nothing more to do for this op:
		// zero pairs stay as they are and zero amplitudes take no phase.
		if(__all_sync(0xffffffffu, pall)) return;
	} else {
#pragma unroll
		for(unsigned p = 0; p < 8; ++p) {
			const unsigned r1 = st_r1<I>(p), r0 = r1 ^ (1u << I);
			st_bfly<R>(v[r0], v[r1], inv);
		}
	}
	if(!chain) return;
	bool nz[8];
	bool mine = true, some = false;
#pragma unroll
	for(unsigned p = 0; p < 8; ++p) {
		nz[p] = st_bits_nonsign(v[st_r1<I>(p)]) != 0u;
		mine = mine && nz[p];
		some = some || nz[p];
	}
	if(zeros && !__any_sync(0xffffffffu, some)) return;  // no |1> output of the warp takes a phase
	const bool all = __all_sync(0xffffffffu, mine);
	// The entries whose control is an outer bit set in this tile (one lane per
	// entry, the same in every warp).
	uint64_t cu = 0;
	if(g.op_outer[k]) {
		const unsigned lane = t & 31u, tb = g.op_tab[k], lc = g.op_lc[k];
		for(unsigned e0 = 0; e0 < lc; e0 += 32) {
			const unsigned e = e0 + lane;
			const unsigned b = e < lc ? ebit[tb + e] : 0xffu;
			const unsigned on = __ballot_sync(0xffffffffu, b != 0xffu && ((base >> b) & 1ull));
			cu |= (uint64_t)__brev(on) << (e0 == 0 ? 32 : 0);
		}
	}
	const uint64_t *T = tab + (size_t)k * kStTabWords;
	const uint64_t tm = cu | T[kStTabLo + (t & 15u)] | T[kStTabHi + (t >> 4)];  // this thread's fixed controls
	const uint64_t wu = cu | T[kStTabWarp + (t >> 5)];                          // their union over the warp
	const uint64_t rall = T[kStTabRegAll];
	uint64_t rm[kStRB];
#pragma unroll
	for(unsigned j = 0; j < kStRB; ++j) rm[j] = T[kStTabReg + j];
	const double2 *cph = ph + g.op_tab[k];
	// Entries [0, split) may have register-bit controls; the rest are uniform
	// per thread.
	const unsigned split = g.op_split[k];
	const uint64_t pre = split ? (~0ull << (64 - split)) : 0ull;
	const uint64_t upre = (wu | rall) & pre, upost = wu & ~pre;
	const uint32_t wh = (uint32_t)(upre >> 32), wl = (uint32_t)upre;
	const uint32_t uh = (uint32_t)(upost >> 32), ul = (uint32_t)upost;
	if(all) {
		stage_walk<R, I, 0, true>((uint32_t)(tm >> 32), rm, rall, wh, cph, nz, v);
		if constexpr(!NARROW) stage_walk<R, I, 1, true>((uint32_t)tm, rm, rall, wl, cph + 32, nz, v);
		stage_walk_uniform<R, I, true>((uint32_t)(tm >> 32), uh, cph, nz, v);
		if constexpr(!NARROW) stage_walk_uniform<R, I, true>((uint32_t)tm, ul, cph + 32, nz, v);
	} else {
		stage_walk<R, I, 0, false>((uint32_t)(tm >> 32), rm, rall, wh, cph, nz, v);
		if constexpr(!NARROW) stage_walk<R, I, 1, false>((uint32_t)tm, rm, rall, wl, cph + 32, nz, v);
		stage_walk_uniform<R, I, false>((uint32_t)(tm >> 32), uh, cph, nz, v);
		if constexpr(!NARROW) stage_walk_uniform<R, I, false>((uint32_t)tm, ul, cph + 32, nz, v);
	}
}

// Shared-memory regions of k_fused_stages, at 16-byte boundaries (phases are
// read as 16-byte values): tile, outer-offset table, op tables, phases, stage
// tables, outer control bits.
struct StageSmem {
	size_t hi, tab, ph, geo, eb, total;
};
__host__ __device__ inline StageSmem stage_smem_layout(size_t amp_bytes, unsigned m, unsigned nops, unsigned nentries,
                                                       unsigned nstages) {
	auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
	StageSmem l;
	l.hi = amp_bytes << kStK;
	l.tab = l.hi + a16(sizeof(uint64_t) << (kStK - m));
	l.ph = l.tab + a16(sizeof(uint64_t) * nops * kStTabWords);
	l.geo = l.ph + sizeof(double2) * nentries;
	l.eb = l.geo + a16(sizeof(uint16_t) * nstages * kStGeoWords);
	l.total = l.eb + nentries;
	return l;
}

template <typename R, bool NARROW>
__global__ void __launch_bounds__(kStThreads, 2) k_fused_stages(typename Vec2<R>::type *a, const __grid_constant__ StageGeom g,
                                                                const ChainEntry *chain, const double2 *gph,
                                                                const uint64_t *gtab) {
	typedef typename Vec2<R>::type V;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const StageSmem L = stage_smem_layout(sizeof(V), g.m, g.nops, g.nentries, g.nstages);
	const unsigned nhi = 1u << (kStK - g.m);
	V *s = reinterpret_cast<V *>(smem_raw);
	uint64_t *hitab = reinterpret_cast<uint64_t *>(smem_raw + L.hi);
	uint64_t *tab = reinterpret_cast<uint64_t *>(smem_raw + L.tab);
	double2 *ph = reinterpret_cast<double2 *>(smem_raw + L.ph);
	uint16_t *geo = reinterpret_cast<uint16_t *>(smem_raw + L.geo);
	uint8_t *ebit = smem_raw + L.eb;  // per entry: its outer control bit, or 0xff for a local control
	const unsigned t = threadIdx.x;
	for(unsigned h = t; h < nhi; h += blockDim.x) {
		uint64_t v = 0;
		for(unsigned i = 0; i < kStK - g.m; ++i)
			if((h >> i) & 1u) v |= 1ull << g.lpos[g.m + i];
		hitab[h] = v;
	}
	for(unsigned e = t; e < g.nops * kStTabWords; e += blockDim.x) tab[e] = gtab[e];
	for(unsigned e = t; e < g.nentries; e += blockDim.x) ph[e] = gph[e];
	for(unsigned e = t; e < g.nstages * kStGeoWords; e += blockDim.x) geo[e] = g.geo[e / kStGeoWords][e % kStGeoWords];
	for(unsigned k = 0; k < g.nops; ++k)
		for(unsigned e = t; e < g.op_lc[k]; e += blockDim.x) {
			const ChainEntry ce = chain[g.op_tab[k] + e];
			ebit[g.op_tab[k] + e] = ce.local < 0 ? (uint8_t)ce.bit : (uint8_t)0xff;
		}
	__syncthreads();
	const unsigned lowmask = (1u << g.m) - 1u;
	auto scatter = [&](unsigned j) -> uint64_t { return (uint64_t)(j & lowmask) | hitab[j >> g.m]; };
	const R inv = (R)g.inv;
	for(uint64_t o = g.o_begin + blockIdx.x; o < g.ntiles; o += gridDim.x) {
		uint64_t base = o;
		for(unsigned i = 0; i < kStK; ++i) base = insert0(base, g.lpos[i]);
		for(unsigned st = 0; st < g.nstages; ++st) {
			const bool first = st == 0, last = st + 1 == g.nstages;
			const uint16_t *G = geo + st * kStGeoWords;
			V v[16];
			if(first) {
				// The first stage reads its amplitudes straight from HBM: global
				// offsets are bit-linear in the local index (disjoint bits OR).
				const uint64_t gb = base | scatter((unsigned)G[kStGeoTlo + (t & 15u)] | G[kStGeoThi + (t >> 4)]);
				uint64_t go[kStRB];
#pragma unroll
				for(unsigned i = 0; i < kStRB; ++i) go[i] = scatter(1u << g.rbit[st][i]);
#pragma unroll
				for(unsigned r = 0; r < 16; ++r) {
					uint64_t x = gb;
#pragma unroll
					for(unsigned i = 0; i < kStRB; ++i)
						if((r >> i) & 1u) x |= go[i];
					v[r] = a[x];
				}
				// The CTA's next tile into L2 while this one is transformed: its
				// 512 runs of 8 contiguous amplitudes (local bits 0-2 are global
				// bits 0-2), two per thread.
				const uint64_t on = o + gridDim.x;
				if(g.m >= 3 && on < g.ntiles) {
					uint64_t nb = on;
					for(unsigned i = 0; i < kStK; ++i) nb = insert0(nb, g.lpos[i]);
#pragma unroll
					for(unsigned h = 0; h < 2; ++h)
						asm volatile("prefetch.global.L2 [%0];" ::"l"(a + (nb | scatter((t + h * kStThreads) << 3))));
				}
			} else {
				const unsigned jb = (unsigned)G[kStGeoSlo + (t & 15u)] ^ G[kStGeoShi + (t >> 4)];
				unsigned ro[kStRB];
#pragma unroll
				for(unsigned i = 0; i < kStRB; ++i) ro[i] = G[kStGeoReg + i];
#pragma unroll
				for(unsigned r = 0; r < 16; ++r) {
					unsigned x = jb;
#pragma unroll
					for(unsigned i = 0; i < kStRB; ++i)
						if((r >> i) & 1u) x ^= ro[i];
					v[r] = s[x];
				}
			}
			const unsigned k1 = g.st_first[st] + g.st_count[st];
			for(unsigned k = g.st_first[st]; k < k1; ++k) {
				const bool chain_op = g.op_lc[k] != 0;
				switch(g.op_reg[k]) {
					case 0: stage_hchain<R, 0, NARROW>(v, inv, chain_op, k, g, tab, ph, ebit, base, t); break;
					case 1: stage_hchain<R, 1, NARROW>(v, inv, chain_op, k, g, tab, ph, ebit, base, t); break;
					case 2: stage_hchain<R, 2, NARROW>(v, inv, chain_op, k, g, tab, ph, ebit, base, t); break;
					default: stage_hchain<R, 3, NARROW>(v, inv, chain_op, k, g, tab, ph, ebit, base, t); break;
				}
			}
			if(last) {
				// The last stage stores straight to HBM.
				const uint64_t gb = base | scatter((unsigned)G[kStGeoTlo + (t & 15u)] | G[kStGeoThi + (t >> 4)]);
				uint64_t go[kStRB];
#pragma unroll
				for(unsigned i = 0; i < kStRB; ++i) go[i] = scatter(1u << g.rbit[st][i]);
#pragma unroll
				for(unsigned r = 0; r < 16; ++r) {
					uint64_t x = gb;
#pragma unroll
					for(unsigned i = 0; i < kStRB; ++i)
						if((r >> i) & 1u) x |= go[i];
					a[x] = v[r];
				}
			} else {
				const unsigned jb = (unsigned)G[kStGeoSlo + (t & 15u)] ^ G[kStGeoShi + (t >> 4)];
				unsigned ro[kStRB];
#pragma unroll
				for(unsigned i = 0; i < kStRB; ++i) ro[i] = G[kStGeoReg + i];
#pragma unroll
				for(unsigned r = 0; r < 16; ++r) {
					unsigned x = jb;
#pragma unroll
					for(unsigned i = 0; i < kStRB; ++i)
						if((r >> i) & 1u) x ^= ro[i];
					s[x] = v[r];
				}
			}
			// Between stages, and before the next tile's first stage writes the
			// buffer the last one read.
			if(!last || g.nstages > 1) __syncthreads();
		}
	}
}

// Shared slot of local index j under the swizzle scol (XOR-linear).
unsigned stage_slot(unsigned j, const uint8_t (&scol)[kStK]) {
	unsigned x = j;
	for(unsigned b = 3; b < kStK; ++b)
		if((j >> b) & 1u) x ^= scol[b];
	return x;
}

// A swizzle under which every stage's quarter-warp lanes (thread index bits
// 0-2) move 8 distinct 16-byte bank groups: over GF(2), the slot bits 0-2
// that those three local bits flip must be independent.  Each local bit
// b >= 3 flips slot bits scol[b]; searched depth-first.  None found: no
// swizzle (correct, with some conflicts).
void stage_swizzle(StageGeom &g) {
	uint8_t col[kStK] = {};
	unsigned assigned = 0x7u;  // bits 0-2 flip themselves
	auto vec = [&](unsigned b) { return b < 3 ? (1u << b) : (unsigned)col[b]; };
	auto stages_ok = [&]() {
		for(unsigned st = 0; st < g.nstages; ++st) {
			const unsigned b0 = g.tbit[st][0], b1 = g.tbit[st][1], b2 = g.tbit[st][2];
			if(!((assigned >> b0) & (assigned >> b1) & (assigned >> b2) & 1u)) continue;
			const unsigned v0 = vec(b0), v1 = vec(b1), v2 = vec(b2);
			if(!v0 || !v1 || !v2 || v0 == v1 || v0 == v2 || v1 == v2 || (v0 ^ v1) == v2) return false;
		}
		return true;
	};
	static const uint8_t order[8] = {0, 1, 2, 4, 3, 5, 6, 7};
	unsigned nodes = 0;
	std::function<bool(unsigned)> dfs = [&](unsigned b) -> bool {
		if(b == kStK) return true;
		for(unsigned i = 0; i < 8; ++i) {
			if(++nodes > 200000) return false;
			col[b] = order[i];
			assigned |= 1u << b;
			if(stages_ok() && dfs(b + 1)) return true;
			assigned &= ~(1u << b);
		}
		col[b] = 0;
		return false;
	};
	if(!dfs(3)) std::memset(col, 0, sizeof(col));
	std::memcpy(g.scol, col, sizeof(col));
}

// Local offset flipped by each thread index bit of stage st: the lane bits
// and warp bits 0-1 (which pick the SM sub-partition) flip one local bit
// each, warp bit 2 flips all three warp-bit locals.  Warps w and w + 4 then
// share a sub-partition with complementary warp-bit controls, so that every
// sub-partition gets the same products whichever of those bits control
// chain entries.
void stage_thread_columns(const StageGeom &g, unsigned st, unsigned (&col)[kStTB]) {
	for(unsigned i = 0; i < kStTB; ++i) col[i] = 1u << g.tbit[st][i];
	col[7] = (1u << g.tbit[st][5]) | (1u << g.tbit[st][6]) | (1u << g.tbit[st][7]);
}

// The stage plan of an exact pass, when its program is Hadamards and H-chains
// on distinct local bits of a 12-bit tile; false otherwise (k_fused runs it).
// Fills the per-op thread-mask tables (kStTabWords words per op).
bool plan_stages(const FusedPass &pass, StageGeom &g, std::vector<double2> &phases, std::vector<uint64_t> &tab) {
	if(pass.K != kStK || pass.ops.empty() || pass.ops.size() > kStMaxOps) return false;
	g = StageGeom{};
	g.n = pass.n;
	g.m = 0;
	while(g.m < pass.K && pass.lpos[g.m] == g.m) ++g.m;
	if(g.m == 0) return false;
	for(unsigned i = 0; i < kStK; ++i) g.lpos[i] = pass.lpos[i];
	uint32_t seen = 0;
	unsigned maxlc = 0, nent = 0;
	for(const FusedOp &op : pass.ops) {
		if(op.kind != kFH && op.kind != kFHChain) return false;
		if(op.lt >= kStK || ((seen >> op.lt) & 1u)) return false;
		seen |= 1u << op.lt;
		const unsigned lc = op.kind == kFHChain ? op.lc : 0u;
		if(lc > 64) return false;
		for(unsigned e = 0; e < lc; ++e) {
			const int l = pass.chain[op.tab + e].local;
			if(l >= (int)kStK || l == (int)op.lt) return false;
		}
		maxlc = std::max(maxlc, lc);
		nent += lc;
	}
	if(nent > kStMaxEntries) return false;
	g.nops = (unsigned)pass.ops.size();
	g.narrow = maxlc <= 32;
	g.inv = 1.0 / std::sqrt(2.0);
	// Stages: consecutive ops while their targets fit in four register bits.
	std::vector<std::vector<unsigned>> regs;
	for(unsigned k = 0; k < g.nops; ++k) {
		const unsigned lt = pass.ops[k].lt;
		if(regs.empty() || regs.back().size() == kStRB) {
			if(g.nstages == kStMaxStages) return false;
			regs.push_back({});
			g.st_first[g.nstages] = (uint8_t)k;
			++g.nstages;
		}
		regs.back().push_back(lt);
		g.op_reg[k] = (uint8_t)(regs.back().size() - 1);
		++g.st_count[g.nstages - 1];
	}
	for(unsigned st = 0; st < g.nstages; ++st) {
		const bool edge = st == 0 || st + 1 == g.nstages;  // reads or writes HBM
		// How many of the stage's chain entries each local bit controls.
		unsigned cost[kStK] = {};
		for(unsigned k = g.st_first[st]; k < g.st_first[st] + g.st_count[st]; ++k) {
			const FusedOp &op = pass.ops[k];
			const unsigned lc = op.kind == kFHChain ? op.lc : 0u;
			for(unsigned e = 0; e < lc; ++e)
				if(pass.chain[op.tab + e].local >= 0) ++cost[pass.chain[op.tab + e].local];
		}
		std::vector<unsigned> &R = regs[st];
		auto in = [](const std::vector<unsigned> &v, unsigned b) { return std::find(v.begin(), v.end(), b) != v.end(); };
		// In a stage that reads or writes HBM, the lowest local bits (global
		// bits 0-2) stay quarter-warp lanes: each warp access then covers whole
		// 128-byte lines.
		const unsigned low = edge ? std::min(g.m, 3u) : 0u;
		// Filler register bits: the most frequent controls; on a tie, the high
		// local bits.
		while(R.size() < kStRB) {
			int best = -1;
			for(int b = (int)kStK - 1; b >= 0; --b) {
				if(in(R, (unsigned)b) || (unsigned)b < low) continue;
				if(best < 0 || cost[b] > cost[best]) best = b;
			}
			R.push_back((unsigned)best);
		}
		uint32_t rset = 0;
		for(unsigned i = 0; i < kStRB; ++i) {
			g.rbit[st][i] = (uint8_t)R[i];
			rset |= 1u << R[i];
		}
		// Lanes: those low bits first (ascending), then the least frequent
		// controls (ascending on a tie); the warp bits take the rest.
		std::vector<unsigned> rest;
		for(unsigned b = 0; b < kStK; ++b)
			if(!((rset >> b) & 1u)) rest.push_back(b);
		std::stable_sort(rest.begin(), rest.end(), [&](unsigned x, unsigned y) {
			if((x < low) != (y < low)) return x < low;
			if(cost[x] != cost[y]) return cost[x] < cost[y];
			return x < y;
		});
		std::vector<unsigned> lanes(rest.begin(), rest.begin() + 5), warps(rest.begin() + 5, rest.end());
		for(unsigned i = 0; i < 5; ++i) g.tbit[st][i] = (uint8_t)lanes[i];
		for(unsigned i = 0; i < 3; ++i) g.tbit[st][5 + i] = (uint8_t)warps[i];
	}
	stage_swizzle(g);
	for(unsigned st = 0; st < g.nstages; ++st) {
		unsigned col[kStTB];
		stage_thread_columns(g, st, col);
		for(unsigned x = 0; x < 16; ++x) {
			unsigned lo = 0, hi = 0;
			for(unsigned i = 0; i < 4; ++i) {
				if((x >> i) & 1u) lo ^= col[i];
				if((x >> i) & 1u) hi ^= col[4 + i];
			}
			g.geo[st][kStGeoTlo + x] = (uint16_t)lo;
			g.geo[st][kStGeoThi + x] = (uint16_t)hi;
			g.geo[st][kStGeoSlo + x] = (uint16_t)stage_slot(lo, g.scol);
			g.geo[st][kStGeoShi + x] = (uint16_t)stage_slot(hi, g.scol);
		}
		for(unsigned i = 0; i < kStRB; ++i) g.geo[st][kStGeoReg + i] = (uint16_t)stage_slot(1u << g.rbit[st][i], g.scol);
	}
	phases.clear();
	tab.assign((size_t)g.nops * kStTabWords, 0ull);
	for(unsigned k = 0; k < g.nops; ++k) {
		const FusedOp &op = pass.ops[k];
		const unsigned lc = op.kind == kFHChain ? op.lc : 0u;
		g.op_tab[k] = (uint16_t)phases.size();
		g.op_lc[k] = (uint16_t)lc;
		unsigned st = 0;
		while(st + 1 < g.nstages && g.st_first[st + 1] <= k) ++st;
		uint64_t *T = tab.data() + (size_t)k * kStTabWords;
		uint64_t rm[kStRB] = {};
		unsigned split = 0;
		for(unsigned e = 0; e < lc; ++e) {
			const ChainEntry &ce = pass.chain[op.tab + e];
			phases.push_back(double2{ce.cr, ce.ci});
			if(ce.local < 0) {
				g.op_outer[k] = 1;
				continue;
			}
			const uint64_t bit = 1ull << (63 - e);
			bool reg = false;
			for(unsigned i = 0; i < kStRB; ++i)
				if(g.rbit[st][i] == (unsigned)ce.local) {
					rm[i] |= bit;
					reg = true;
					split = e + 1;
				}
			if(reg) continue;
			// A thread control: set for the nibbles whose local offset has it.
			for(unsigned x = 0; x < 16; ++x) {
				if((g.geo[st][kStGeoTlo + x] >> ce.local) & 1u) T[kStTabLo + x] |= bit;
				if((g.geo[st][kStGeoThi + x] >> ce.local) & 1u) T[kStTabHi + x] |= bit;
			}
		}
		g.op_split[k] = (uint8_t)split;
		uint64_t lo_all = 0;
		for(unsigned x = 0; x < 16; ++x) lo_all |= T[kStTabLo + x];
		for(unsigned w = 0; w < kStThreads / 32; ++w) T[kStTabWarp + w] = lo_all | T[kStTabHi + 2 * w] | T[kStTabHi + 2 * w + 1];
		for(unsigned i = 0; i < kStRB; ++i) {
			T[kStTabReg + i] = rm[i];
			T[kStTabRegAll] |= rm[i];
		}
	}
	g.nentries = (unsigned)phases.size();
	return true;
}

template <typename R>
bool run_fused_stages(const LaunchCtx &c, void *a, const FusedPass &pass, void *&dev_prog, size_t &dev_prog_bytes,
                      bool upload_only = false) {
	StageGeom g;
	std::vector<double2> phases;
	std::vector<uint64_t> tab;
	if(!plan_stages(pass, g, phases, tab)) return false;
	g.ntiles = 1ull << (pass.n - kStK);
	g.o_begin = 0;
	if(pass.tile_end) {
		if(pass.tile_begin >= pass.tile_end || pass.tile_end > g.ntiles) fail(TMFQS_ERR_LOGIC, "fused pass: bad tile range");
		g.o_begin = pass.tile_begin;
		g.ntiles = pass.tile_end;
	}
	const size_t ch_bytes = std::max<size_t>(32, pass.chain.size() * sizeof(ChainEntry));
	const size_t ph_off = (ch_bytes + 255) & ~size_t(255);
	const size_t tab_off = (ph_off + std::max<size_t>(16, phases.size() * sizeof(double2)) + 255) & ~size_t(255);
	const size_t need = tab_off + tab.size() * sizeof(uint64_t);
	if(pass.program_ready) {
		if(need > dev_prog_bytes) fail(TMFQS_ERR_LOGIC, "fused pass: prepared program missing");
	} else {
		if(need > dev_prog_bytes) {
			if(dev_prog) {
				check_cuda(cudaStreamSynchronize(c.stream), "fused program sync");
				cudaFree(dev_prog);
			}
			dev_prog = nullptr;
			dev_prog_bytes = 0;
			if(device_alloc(&dev_prog, need * 2) != cudaSuccess) {
				cudaGetLastError();
				fail(TMFQS_ERR_NOMEM, "fused pass program allocation failed");
			}
			dev_prog_bytes = need * 2;
		}
		std::vector<unsigned char> host(need, 0);
		if(!pass.chain.empty()) std::memcpy(host.data(), pass.chain.data(), pass.chain.size() * sizeof(ChainEntry));
		if(!phases.empty()) std::memcpy(host.data() + ph_off, phases.data(), phases.size() * sizeof(double2));
		std::memcpy(host.data() + tab_off, tab.data(), tab.size() * sizeof(uint64_t));
		upload_async(c, dev_prog, host.data(), need, "fused program upload");
	}
	if(upload_only) return true;
	unsigned char *dp = static_cast<unsigned char *>(dev_prog);
	const size_t smem = stage_smem_layout(sizeof(typename Vec2<R>::type), g.m, g.nops, g.nentries, g.nstages).total;
	auto kern = g.narrow ? k_fused_stages<R, true> : k_fused_stages<R, false>;
	check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "stage smem");
	int per_sm = 1;
	check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStThreads, smem), "stage occupancy");
	const uint64_t grid = std::min<uint64_t>(g.ntiles - g.o_begin, (uint64_t)c.num_sms * std::max(1, per_sm));
	kern<<<(unsigned)grid, kStThreads, smem, c.stream>>>(
		static_cast<typename Vec2<R>::type *>(a), g, reinterpret_cast<const ChainEntry *>(dp),
		reinterpret_cast<const double2 *>(dp + ph_off), reinterpret_cast<const uint64_t *>(dp + tab_off));
	after_launch(c, "fused stage pass");
	return true;
}

}  // namespace

bool prepare_fused_pass(const LaunchCtx &c, int prec, const FusedPass &pass, void *&dev_prog, size_t &dev_prog_bytes) {
	if(prec != TMFQS_FP64 || pass.program_ready) return false;
	return run_fused_stages<double>(c, nullptr, pass, dev_prog, dev_prog_bytes, true);
}

void launch_fused_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, void *&dev_prog,
                       size_t &dev_prog_bytes) {
	if(prec == TMFQS_FP64) {
		if(!run_fused_stages<double>(c, a, pass, dev_prog, dev_prog_bytes)) run_fused<double>(c, a, pass, dev_prog, dev_prog_bytes);
	} else {
		run_fused<float>(c, a, pass, dev_prog, dev_prog_bytes);
	}
}

void launch_bit_permutation(const LaunchCtx &c, int prec, void *a, unsigned n,
                            const std::vector<std::pair<unsigned, unsigned>> &pairs) {
	if(prec == TMFQS_FP64) run_perm<double>(c, a, n, pairs);
	else run_perm<float>(c, a, n, pairs);
}

void launch_grover_temporal(const LaunchCtx &c, int prec, void *a, unsigned n, const void *dev_two_means,
                            uint64_t iterations, const uint64_t *dev_marked, unsigned marked_count,
                            uint64_t flip_from) {
	const uint64_t N = 1ull << n;
	const unsigned per = prec == TMFQS_FP64 ? 4u : 8u;
	const uint64_t threads = (N + per - 1) / per;
	const uint64_t blocks = std::max<uint64_t>(1, std::min<uint64_t>((threads + 255) / 256, (uint64_t)c.num_sms * 8));
	if(prec == TMFQS_FP64)
		k_grover_temporal<double, 4><<<(unsigned)blocks, 256, 0, c.stream>>>(
			static_cast<double2 *>(a), N, static_cast<const double2 *>(dev_two_means), iterations, flip_from, dev_marked,
			marked_count);
	else
		k_grover_temporal<float, 8><<<(unsigned)blocks, 256, 0, c.stream>>>(
			static_cast<float2 *>(a), N, static_cast<const float2 *>(dev_two_means), iterations, flip_from, dev_marked,
			marked_count);
	after_launch(c, "grover temporal");
}

}  // namespace tqb
