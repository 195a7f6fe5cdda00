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
	uint32_t nq;       // number of q values, 2^(K-6)
	uint32_t ilp;      // 1: bit 0 of q is no control, so q and q+1 share their mask
	uint32_t pad[2];
};
constexpr uint64_t kNoChainMap = ~0ull;

// Applies the chain entries of mask m (entry e = bit 63-e, ascending e =
// circuit order) to one amplitude: each a separately rounded complex product
// (dense_state_backend.cpp:300-301), exactly as the per-gate path.
template <typename R>
__device__ __forceinline__ void chain_apply(uint64_t m, const double2 *cph, R &r, R &i) {
	for(uint32_t hi = (uint32_t)(m >> 32); hi;) {
		const unsigned e = __clz(hi);
		hi ^= 0x80000000u >> e;
		const double2 ph = cph[e];
		cmul_ref((R)ph.x, (R)ph.y, r, i);
	}
	for(uint32_t lo = (uint32_t)m; lo;) {
		const unsigned e = __clz(lo);
		lo ^= 0x80000000u >> e;
		const double2 ph = cph[32 + e];
		cmul_ref((R)ph.x, (R)ph.y, r, i);
	}
}

// The same for two amplitudes with the same mask.
template <typename R>
__device__ __forceinline__ void chain_apply2(uint64_t m, const double2 *cph, R &ra, R &ia, R &rb, R &ib) {
	for(uint32_t hi = (uint32_t)(m >> 32); hi;) {
		const unsigned e = __clz(hi);
		hi ^= 0x80000000u >> e;
		const double2 ph = cph[e];
		cmul_ref((R)ph.x, (R)ph.y, ra, ia);
		cmul_ref((R)ph.x, (R)ph.y, rb, ib);
	}
	for(uint32_t lo = (uint32_t)m; lo;) {
		const unsigned e = __clz(lo);
		lo ^= 0x80000000u >> e;
		const double2 ph = cph[32 + e];
		cmul_ref((R)ph.x, (R)ph.y, ra, ia);
		cmul_ref((R)ph.x, (R)ph.y, rb, ib);
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
						}
						__syncthreads();
						const ChainMap &cm = maps[op.state];
						const unsigned tb = 1u << op.lt, jl = cm.jl[lane];
						const uint64_t mlane = cm.ml[lane] | cu;
						const unsigned warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
						if(cm.ilp) {
							// Two butterflies per thread whose |1> outputs take the same
							// phases (they differ in a bit that is no control).
							for(unsigned q = 2 * warp; q < cm.nq; q += 2 * nw) {
								const unsigned ja = jl | cm.jr[q], jb = jl | cm.jr[q + 1];
								const uint64_t m = mlane | cm.mr[q];
								V xa = s[P(ja)], ya = s[P(ja | tb)], xb = s[P(jb)], yb = s[P(jb | tb)];
								const bool wa = butterfly<R>(xa, ya, inv), wb = butterfly<R>(xb, yb, inv);
								// A zero |1> output is left alone by every phase (dense_state_backend.cpp:299).
								const bool ca = wa && !is_zero<R>(ya), cb = wb && !is_zero<R>(yb);
								if(ca || cb) {
									R ra = ya.x, ia = ya.y, rb = yb.x, ib = yb.y;
									chain_apply2<R>(m, cph, ra, ia, rb, ib);
									if(ca) {
										ya.x = ra;
										ya.y = ia;
									}
									if(cb) {
										yb.x = rb;
										yb.y = ib;
									}
								}
								if(wa) {
									s[P(ja)] = xa;
									s[P(ja | tb)] = ya;
								}
								if(wb) {
									s[P(jb)] = xb;
									s[P(jb | tb)] = yb;
								}
							}
						} else {
							for(unsigned q = warp; q < cm.nq; q += nw) {
								const unsigned ja = jl | cm.jr[q];
								V x = s[P(ja)], y = s[P(ja | tb)];
								if(!butterfly<R>(x, y, inv)) continue;
								if(!is_zero<R>(y)) {
									R r = y.x, i = y.y;
									chain_apply<R>(mlane | cm.mr[q], cph, r, i);
									y.x = r;
									y.y = i;
								}
								s[P(ja)] = x;
								s[P(ja | tb)] = y;
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
			float4 wa, wb;
			V *ya = reinterpret_cast<V *>(&wa), *yb = reinterpret_cast<V *>(&wb);
#pragma unroll
			for(unsigned e = 0; e < G; ++e) {
				ya[e] = A[src[i][e]];
				if(pair) yb[e] = B[src[i][e]];
			}
			*reinterpret_cast<float4 *>(a + (cur.pbase | goff[i])) = wa;
			if(pair) *reinterpret_cast<float4 *>(a + (cur.base | goff[i])) = wb;
		}
		__syncthreads();
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
	const int ilp = next(true);
	if(ilp >= 0) take((unsigned)ilp);
	for(int b = next(false); b >= 0; b = next(false)) take((unsigned)b);
	if(order.size() != K - 1) fail(TMFQS_ERR_LOGIC, "fused pass: chain layout");
	ChainMap m{};
	m.nq = 1u << (K - 6);
	m.ilp = ilp >= 0 ? 1u : 0u;
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
