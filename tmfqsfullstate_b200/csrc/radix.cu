// Radix-2^RB fused pass for the fast forms (complex64 states, and complex128
// with TMFQS_OPT_EXACT off) of Hadamard / controlled-phase programs: the QFT
// ladder and anything else built from H and controlled phases.
//
// A pass covers tiles of 2^K amplitudes (the K local bit positions).  Tiles
// stream through two shared-memory buffers: the next tile's cp.async copy is
// in flight while the current one is transformed, so HBM traffic overlaps the
// arithmetic.  The pass's circuit is split on the host into stages of RB
// register bits.  In a stage each thread holds the 2^RB amplitudes that differ
// only in those bits and applies, in registers:
//   - unscaled butterflies (a0 + a1, a0 - a1) for the Hadamards of the stage;
//     the product of all 1/sqrt(2) factors of the pass is applied once, with
//     the last stage's phase;
//   - "in-stage" phases (both qubits of the controlled phase are register
//     bits of the stage) at their place in the circuit, as one precomputed
//     2^RB-entry phase table per run of such phases;
//   - "cross-stage" phases (at most one qubit is a register bit): they commute
//     with every Hadamard of the stage that they can be moved past, so they are
//     gathered into one factor per amplitude, applied before or after the
//     stage's butterflies.  The factor for register bits r is the product of
//     per-bit factors f_i, f_i = A_i[low local bits] * B_i[high local bits] *
//     O_i(tile), where the tables hold the phases of the local control bits
//     (computed once in FP64 with sincos and rounded once to the storage type)
//     and O_i those of the tile's outer bits.
// Stages hand the tile over through the (XOR-swizzled) shared buffer.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"
#include "radix_common.cuh"

namespace tqb {

namespace {

constexpr unsigned kRadixThreads = 512;
constexpr unsigned kRadixMaxStages = 8;
constexpr unsigned kRadixMaxItems = 128;
constexpr unsigned kRadixMaxTab = 2048;
constexpr unsigned kRadixMaxSlots = 48;

// Stage program entry: kind in bits 0-7, register bit in bits 8-15, first
// table entry in bits 16-31.
//   kRIButterfly    butterflies on the register bit
//   kRIButterflyTw  butterflies, then the |1> outputs times a 2^(RB-1)-entry
//                   table (the in-stage phases that follow a Hadamard)
//   kRIDiag         every register times a 2^RB-entry table
//   kRIQft          the QFT ladder on register bits 0..d-1 (d in bits 8-15):
//                   Hadamards in bit order, and after the one on bit i the
//                   controlled phases pi/2^(j-i) with every later bit j, as a
//                   compiled butterfly network with the roots of unity below
//   kRIWalsh        butterflies on register bits 0..d-1 (d in bits 8-15), no
//                   phases between them: one compiled network
enum RadixItemKind : uint32_t { kRIButterfly = 0, kRIButterflyTw = 1, kRIDiag = 2, kRIQft = 3, kRIWalsh = 4 };

struct RadixStage {
	uint32_t first, count;    // items of the stage
	uint32_t rbit[5];         // register bit i -> local bit
	uint32_t rsorted[5];      // the register local bits, ascending
	uint32_t imask[5];        // (1 << rsorted[i]) - 1: the thread index gets a zero bit inserted above it
	uint32_t roff[5];         // swizzled shared-memory offset of register bit i
	uint64_t gbit[5];         // global index bit of register bit i (direct stores)
	uint32_t pre_slot, pre_mask;    // first factor slot; bit 0 constant factor, bit i+1 register bit i
	uint32_t post_slot, post_mask;
	uint32_t direct;                // last stage: store to HBM from registers
	uint32_t post_xfirst, post_xcount;  // per-thread terms of the post constant factor
};

// One phase term of a factor slot: theta when all its bits are set.  bit1 is
// kNoBit for single-bit terms.  Local bits are local indices (A range below
// `lo`, B range from `lo`), outer bits are global positions.
constexpr uint32_t kNoBit = 0xffffffffu;
struct RadixTerm {
	uint32_t bit0, bit1;
	double theta;
	uint32_t outer;  // thread terms: bit 0 / bit 1 set when bit0 / bit1 is an outer (global) bit
	uint32_t pad;
	double c, s;     // thread terms: cos(theta), sin(theta)
};

struct RadixSlot {
	uint32_t a_first, a_count;  // terms on A-range local bits
	uint32_t b_first, b_count;  // terms on B-range local bits
	uint32_t o_first, o_count;  // terms on outer bits
	uint32_t x_first, x_count;  // constant slot: two-bit terms the tables cannot hold (a local bit with an
	                            // outer bit, or local bits of both tables), evaluated per thread
	double scale;               // real factor folded into the slot (1, or the pass's Hadamard scale)
};

struct RadixGeom {
	unsigned K, m, lo;          // local bits, contiguous low local bits, A-range bits
	unsigned lpos[14];          // ascending local bit positions
	uint64_t ntiles;
	unsigned nstages, nitems, ntab, nslots, nterms;
	unsigned outer_free;        // no slot has outer terms: every tile's outer row is the slot scales
	RootTable roots;            // twiddles of the compiled QFT stages
};

template <typename V>
struct RadixSmem {
	V *buf[2];
	uint64_t *hitab;
	RadixStage *stages;
	uint32_t *items;
	V *tabs;          // in-stage phase tables
	V *A;             // [nslots][2^lo]
	V *B;             // [nslots][2^(K-lo)]
	V *Ot[2];         // [nslots] outer phase x scale of the current / next tile
};

template <typename V>
__device__ __forceinline__ unsigned rswz(unsigned j);
template <>
__device__ __forceinline__ unsigned rswz<double2>(unsigned j) {
	return j ^ ((j >> 3) & 7u);
}
template <>
__device__ __forceinline__ unsigned rswz<float2>(unsigned j) {
	// Keeps element pairs (16-byte copy granules) together.
	return j ^ (((j >> 4) & 7u) << 1);
}

// Angle of a slot's outer terms for the tile with base index `base`.
__device__ __forceinline__ double slot_outer_angle(const RadixSlot &s, const RadixTerm *terms, uint64_t base) {
	double ang = 0.0;
	for(unsigned t = 0; t < s.o_count; ++t) {
		const RadixTerm tm = terms[s.o_first + t];
		const bool on = ((base >> tm.bit0) & 1ull) && (tm.bit1 == kNoBit || ((base >> tm.bit1) & 1ull));
		if(on) ang += tm.theta;
	}
	return ang;
}

template <typename V>
__device__ __forceinline__ V to_v(double2 d);
template <>
__device__ __forceinline__ double2 to_v<double2>(double2 d) {
	return d;
}
template <>
__device__ __forceinline__ float2 to_v<float2>(double2 d) {
	return make_float2((float)d.x, (float)d.y);
}

// Butterflies on register bit TB (unscaled); with `tw`, the |1> output of
// pair q is then multiplied by tw[q].
template <typename V, int RB, int TB>
__device__ __forceinline__ void rbfly(V (&v)[1 << RB], const V *tw) {
	constexpr int lo = (1 << TB) - 1;
#pragma unroll
	for(int q = 0; q < (1 << (RB - 1)); ++q) {
		const int r0 = ((q & ~lo) << 1) | (q & lo), r1 = r0 | (1 << TB);
		bfly2(v[r0], v[r1]);
	}
	if(tw) {
#pragma unroll
		for(int q = 0; q < (1 << (RB - 1)); ++q) {
			const int r1 = ((q & ~lo) << 1) | (q & lo) | (1 << TB);
			v[r1] = vmul(v[r1], tw[q]);
		}
	}
}

template <typename V, int RB>
__device__ __forceinline__ void rbfly_dispatch(V (&v)[1 << RB], unsigned b, const V *tw) {
	switch(b) {
		case 0: rbfly<V, RB, 0>(v, tw); break;
		case 1: if constexpr(RB > 1) rbfly<V, RB, 1>(v, tw); break;
		case 2: if constexpr(RB > 2) rbfly<V, RB, 2>(v, tw); break;
		case 3: if constexpr(RB > 3) rbfly<V, RB, 3>(v, tw); break;
		case 4: if constexpr(RB > 4) rbfly<V, RB, 4>(v, tw); break;
		default: break;
	}
}

template <typename V, int RB, int D>
__device__ __forceinline__ void walsh_stage(V (&v)[1 << RB]) {
	if constexpr(D > 0) rbfly<V, RB, 0>(v, nullptr);
	if constexpr(D > 1) rbfly<V, RB, 1>(v, nullptr);
	if constexpr(D > 2) rbfly<V, RB, 2>(v, nullptr);
	if constexpr(D > 3) rbfly<V, RB, 3>(v, nullptr);
	if constexpr(D > 4) rbfly<V, RB, 4>(v, nullptr);
}

template <typename V, int RB>
__device__ __forceinline__ void walsh_dispatch(V (&v)[1 << RB], unsigned d) {
	switch(d) {
		case 1: walsh_stage<V, RB, 1>(v); break;
		case 2: if constexpr(RB >= 2) walsh_stage<V, RB, 2>(v); break;
		case 3: if constexpr(RB >= 3) walsh_stage<V, RB, 3>(v); break;
		case 4: if constexpr(RB >= 4) walsh_stage<V, RB, 4>(v); break;
		case 5: if constexpr(RB >= 5) walsh_stage<V, RB, 5>(v); break;
		default: break;
	}
}

template <typename V, int RB>
__device__ __forceinline__ void qft_dispatch(V (&v)[1 << RB], unsigned d, const RadixGeom &g) {
	switch(d) {
		case 1: qft_stage<V, RB, 1>(v, g.roots); break;
		case 2: if constexpr(RB >= 2) qft_stage<V, RB, 2>(v, g.roots); break;
		case 3: if constexpr(RB >= 3) qft_stage<V, RB, 3>(v, g.roots); break;
		case 4: if constexpr(RB >= 4) qft_stage<V, RB, 4>(v, g.roots); break;
		case 5: if constexpr(RB >= 5) qft_stage<V, RB, 5>(v, g.roots); break;
		default: break;
	}
}

// The constant factor times its per-thread terms (two-bit phases the tables
// cannot hold); kept out of line, off the common path.
template <typename V>
__device__ __noinline__ V thread_terms(V f, const RadixTerm *terms, unsigned first, unsigned count, unsigned jt,
                                       uint64_t base) {
	for(unsigned t = 0; t < count; ++t) {
		const RadixTerm tm = terms[first + t];
		const bool on0 = (tm.outer & 1u) ? ((base >> tm.bit0) & 1ull) : ((jt >> tm.bit0) & 1u);
		const bool on1 = (tm.outer & 2u) ? ((base >> tm.bit1) & 1ull) : ((jt >> tm.bit1) & 1u);
		if(on0 && on1) {
			V w;
			w.x = (decltype(w.x))tm.c;
			w.y = (decltype(w.y))tm.s;
			f = vmul(f, w);
		}
	}
	return f;
}

// Multiplies v[r] by the product of the active factors of a slot group:
// factor 0 for every r (if bit 0 of mask), factor i+1 for r with bit i.
template <typename V, int RB>
__device__ __forceinline__ void apply_factors(V (&v)[1 << RB], const RadixSmem<V> &sh, const V *ot, unsigned slot0,
                                              unsigned mask, unsigned ia, unsigned ib, unsigned lo, unsigned nb, const RadixTerm *terms,
                                              unsigned xfirst, unsigned xcount, unsigned jt, uint64_t base) {
	V f[RB + 1];
	unsigned s = slot0;
#pragma unroll
	for(int i = 0; i <= RB; ++i) {
		if((mask >> i) & 1u) {
			f[i] = vmul(vmul(sh.A[(s << lo) + ia], sh.B[s * nb + ib]), ot[s]);
			if(i == 0 && xcount) f[0] = thread_terms(f[0], terms, xfirst, xcount, jt, base);
			++s;
		} else {
			f[i].x = 1;
			f[i].y = 0;
		}
	}
	// F(r) = f0 * prod_{i in r} f_{i+1}, built from the lower subsets.
	V F[1 << RB];
	if(mask & 1u) {
		F[0] = f[0];
#pragma unroll
		for(int r = 1; r < (1 << RB); ++r) {
			const int hb = 31 - __clz(r);
			F[r] = vmul(F[r ^ (1 << hb)], f[hb + 1]);
		}
		v[0] = vmul(v[0], F[0]);
	} else {
#pragma unroll
		for(int r = 1; r < (1 << RB); ++r) {
			const int hb = 31 - __clz(r);
			F[r] = (r == (1 << hb)) ? f[hb + 1] : vmul(F[r ^ (1 << hb)], f[hb + 1]);
		}
	}
#pragma unroll
	for(int r = 1; r < (1 << RB); ++r) v[r] = vmul(v[r], F[r]);
}

// The constant factor alone (mask 1, no per-thread terms): one value for every
// register, and a real product when it has no imaginary part (the scale of a
// pass without phases on its non-register bits).
template <typename V, int RB>
__device__ __forceinline__ void apply_constant(V (&v)[1 << RB], const RadixSmem<V> &sh, const V *ot, unsigned s,
                                               unsigned ia, unsigned ib, unsigned lo, unsigned nb) {
	const V f = vmul(vmul(sh.A[(s << lo) + ia], sh.B[s * nb + ib]), ot[s]);
	if(f.y == 0) {
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) {
			v[r].x *= f.x;
			v[r].y *= f.x;
		}
	} else {
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) v[r] = vmul(v[r], f);
	}
}

}  // namespace

namespace {

template <typename R, int RB>
__global__ void __launch_bounds__(kRadixThreads, 1)
	k_radix(typename Vec2<R>::type *a, RadixGeom g, const unsigned char *prog, size_t off_stages, size_t off_items,
	        size_t off_tabs, size_t off_slots, size_t off_terms, const typename Vec2<R>::type *otab, unsigned ot_stride,
	        typename Vec2<R>::type *mirror) {
	typedef typename Vec2<R>::type V;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const unsigned T = 1u << g.K;
	const unsigned nhi = 1u << (g.K - g.m);
	const unsigned nb = 1u << (g.K - g.lo);
	const RadixStage *gstages = reinterpret_cast<const RadixStage *>(prog + off_stages);
	const uint32_t *gitems = reinterpret_cast<const uint32_t *>(prog + off_items);
	const double2 *gtabs = reinterpret_cast<const double2 *>(prog + off_tabs);
	const RadixSlot *gslots = reinterpret_cast<const RadixSlot *>(prog + off_slots);
	const RadixTerm *gterms = reinterpret_cast<const RadixTerm *>(prog + off_terms);

	RadixSmem<V> sh;
	size_t off = 0;
	auto take = [&](size_t bytes) -> unsigned char * {
		unsigned char *q = smem_raw + off;
		off += (bytes + 15) & ~size_t(15);
		return q;
	};
	sh.buf[0] = reinterpret_cast<V *>(take(sizeof(V) * T));
	sh.buf[1] = reinterpret_cast<V *>(take(sizeof(V) * T));
	sh.hitab = reinterpret_cast<uint64_t *>(take(sizeof(uint64_t) * nhi));
	sh.stages = reinterpret_cast<RadixStage *>(take(sizeof(RadixStage) * g.nstages));
	sh.items = reinterpret_cast<uint32_t *>(take(sizeof(uint32_t) * g.nitems));
	sh.tabs = reinterpret_cast<V *>(take(sizeof(V) * g.ntab));
	sh.A = reinterpret_cast<V *>(take(sizeof(V) * ((size_t)g.nslots << g.lo)));
	sh.B = reinterpret_cast<V *>(take(sizeof(V) * g.nslots * nb));
	sh.Ot[0] = reinterpret_cast<V *>(take(sizeof(V) * ot_stride));
	sh.Ot[1] = reinterpret_cast<V *>(take(sizeof(V) * ot_stride));

	const unsigned tid = threadIdx.x, nthr = blockDim.x;
	const unsigned lowmask = (1u << g.m) - 1u;
	for(unsigned h = tid; h < nhi; h += nthr) {
		uint64_t v = 0;
		for(unsigned i = 0; i < g.K - g.m; ++i)
			if((h >> i) & 1u) v |= 1ull << g.lpos[g.m + i];
		sh.hitab[h] = v;
	}
	__syncthreads();
	auto scatter = [&](unsigned j) -> uint64_t { return (uint64_t)(j & lowmask) | sh.hitab[j >> g.m]; };
	auto tile_base = [&](uint64_t o) -> uint64_t {
		for(unsigned i = 0; i < g.K; ++i) o = insert0(o, g.lpos[i]);
		return o;
	};
	// Granules of 16 bytes: one complex128 or two complex64 amplitudes.
	constexpr unsigned per16 = 16 / sizeof(V);
	// A tile's amplitudes and its row of outer phases (ot_stride values, a
	// multiple of 16 bytes) arrive in one copy group.
	auto prefetch = [&](uint64_t o, uint64_t base, V *dst, V *odst) {
		if(o < g.ntiles) {
			for(unsigned q = tid; q < T / per16; q += nthr) {
				const unsigned j = q * per16;
				cp_async16(dst + rswz<V>(j), a + (base | scatter(j)));
			}
			if(!g.outer_free)
				for(unsigned q = tid; q < ot_stride / per16; q += nthr)
					cp_async16(odst + q * per16, otab + o * ot_stride + q * per16);
		}
		cp_async_commit();
	};
	// The first tile's copy starts before the tables are built.
	uint64_t cbase = tile_base(blockIdx.x);
	// Thread 0 computes the base of the tile after next one iteration ahead
	// and hands it over through shared memory (the tile loop's barriers order
	// the write before the reads).
	__shared__ uint64_t nb_slot[2];
	if(tid == 0 && blockIdx.x + gridDim.x < g.ntiles) nb_slot[0] = tile_base(blockIdx.x + gridDim.x);
	prefetch(blockIdx.x, cbase, sh.buf[0], sh.Ot[0]);

	for(unsigned k = tid; k < g.nstages; k += nthr) sh.stages[k] = gstages[k];
	for(unsigned k = tid; k < g.nitems; k += nthr) sh.items[k] = gitems[k];
	for(unsigned k = tid; k < g.ntab; k += nthr) sh.tabs[k] = to_v<V>(gtabs[k]);
	// Without outer terms the outer rows of both buffers hold the slot scales
	// for every tile (cos 0 and sin 0 times the scale, as the table would).
	if(g.outer_free)
		for(unsigned s = tid; s < g.nslots; s += nthr) {
			const V w = to_v<V>(make_double2(gslots[s].scale, 0.0));
			sh.Ot[0][s] = w;
			sh.Ot[1][s] = w;
		}
	// Tile-independent phase tables of the local control bits, in FP64.
	const unsigned na = 1u << g.lo;
	for(unsigned t = tid; t < g.nslots * (na + nb); t += nthr) {
		const bool is_a = t < g.nslots * na;
		const unsigned s = is_a ? t / na : (t - g.nslots * na) / nb;
		const unsigned x = is_a ? t % na : (t - g.nslots * na) % nb;
		const RadixSlot sl = gslots[s];
		const unsigned first = is_a ? sl.a_first : sl.b_first, cnt = is_a ? sl.a_count : sl.b_count;
		const unsigned shift = is_a ? 0u : g.lo;
		double ang = 0.0;
		for(unsigned e = 0; e < cnt; ++e) {
			const RadixTerm tm = gterms[first + e];
			const bool on = ((x >> (tm.bit0 - shift)) & 1u) && (tm.bit1 == kNoBit || ((x >> (tm.bit1 - shift)) & 1u));
			if(on) ang += tm.theta;
		}
		double sv, cv;
		sincos(ang, &sv, &cv);
		if(is_a) sh.A[(s << g.lo) + x] = to_v<V>(make_double2(cv, sv));
		else sh.B[s * nb + x] = to_v<V>(make_double2(cv, sv));
	}
	__syncthreads();

	unsigned cur = 0;
	for(uint64_t o = blockIdx.x; o < g.ntiles; o += gridDim.x, cur ^= 1u) {
		const uint64_t next = o + gridDim.x;
		const uint64_t nbase = next < g.ntiles ? nb_slot[cur] : cbase;
		if(tid == 0 && next + gridDim.x < g.ntiles) nb_slot[cur ^ 1u] = tile_base(next + gridDim.x);
		prefetch(next, nbase, sh.buf[cur ^ 1u], sh.Ot[cur ^ 1u]);
		const V *ot = sh.Ot[cur];
		cp_async_wait1();
		__syncthreads();
		V *tile = sh.buf[cur];
		V v[1 << RB];
		for(unsigned st = 0; st < g.nstages; ++st) {
			const RadixStage &S = sh.stages[st];
			unsigned jt = tid;
#pragma unroll
			for(int i = 0; i < RB; ++i) jt = ((jt & ~S.imask[i]) << 1) | (jt & S.imask[i]);
			unsigned roff[RB];
#pragma unroll
			for(int i = 0; i < RB; ++i) roff[i] = S.roff[i];
			const unsigned sj = rswz<V>(jt);
			auto addr = [&](int r) -> unsigned {
				unsigned x = sj;
#pragma unroll
				for(int i = 0; i < RB; ++i)
					if((r >> i) & 1) x ^= roff[i];
				return x;
			};
#pragma unroll
			for(int r = 0; r < (1 << RB); ++r) v[r] = tile[addr(r)];
			const unsigned ia = jt & ((1u << g.lo) - 1u), ib = jt >> g.lo;
			if(S.pre_mask) apply_factors<V, RB>(v, sh, ot, S.pre_slot, S.pre_mask, ia, ib, g.lo, nb, gterms, 0, 0, jt, cbase);
			for(unsigned k = S.first; k < S.first + S.count; ++k) {
				const uint32_t it = sh.items[k];
				const unsigned kind = it & 0xffu, b = (it >> 8) & 0xffu;
				const V *tb = sh.tabs + (it >> 16);
				if(kind == kRIWalsh) {
					walsh_dispatch<V, RB>(v, b);
				} else if(kind == kRIQft) {
					qft_dispatch<V, RB>(v, b, g);
				} else if(kind == kRIDiag) {
#pragma unroll
					for(int r = 0; r < (1 << RB); ++r) v[r] = vmul(v[r], tb[r]);
				} else {
					rbfly_dispatch<V, RB>(v, b, kind == kRIButterflyTw ? tb : nullptr);
				}
			}
			if(S.post_mask == 1u && !S.post_xcount)
				apply_constant<V, RB>(v, sh, ot, S.post_slot, ia, ib, g.lo, nb);
			else if(S.post_mask)
				apply_factors<V, RB>(v, sh, ot, S.post_slot, S.post_mask, ia, ib, g.lo, nb, gterms, S.post_xfirst, S.post_xcount, jt,
				                     cbase);
			const bool last = st + 1 == g.nstages;
			if(last && S.direct) {
				// Lanes run along the low address bits: coalesced stores.
				const uint64_t gt = cbase | scatter(jt);
				uint64_t gbit[RB];
#pragma unroll
				for(int i = 0; i < RB; ++i) gbit[i] = S.gbit[i];
				auto store = [&](V *dst) {
#pragma unroll
					for(int r = 0; r < (1 << RB); ++r) {
						uint64_t x = gt;
#pragma unroll
						for(int i = 0; i < RB; ++i)
							if((r >> i) & 1) x |= gbit[i];
						dst[x] = v[r];
					}
				};
				store(a);
				if(mirror) store(mirror);
			} else {
				// Each thread rewrites only the slots it read in this stage.
#pragma unroll
				for(int r = 0; r < (1 << RB); ++r) tile[addr(r)] = v[r];
				__syncthreads();
				if(last)
					for(unsigned q = tid; q < T / per16; q += nthr) {
						const unsigned j = q * per16;
						const uint64_t x = cbase | scatter(j);
						const float4 w = *reinterpret_cast<const float4 *>(tile + rswz<V>(j));
						*reinterpret_cast<float4 *>(a + x) = w;
						if(mirror) *reinterpret_cast<float4 *>(mirror + x) = w;
					}
			}
		}
		cbase = nbase;
		__syncthreads();
	}
	// Drain the (empty) groups committed past the last tile.
	cp_async_wait_all();
}

}  // namespace

namespace {

// The outer-bit phase of every slot for every tile (times the slot's scale),
// rounded once to the storage type: otab[o * stride + s].
template <typename R>
__global__ void __launch_bounds__(256) k_outer_table(typename Vec2<R>::type *otab, unsigned stride, RadixGeom g,
                                                    const RadixSlot *slots, const RadixTerm *terms) {
	typedef typename Vec2<R>::type V;
	for(uint64_t e = gtid(); e < g.ntiles * g.nslots; e += gstride()) {
		const uint64_t o = e / g.nslots;
		const unsigned s = (unsigned)(e - o * g.nslots);
		uint64_t base = o;
		for(unsigned i = 0; i < g.K; ++i) base = insert0(base, g.lpos[i]);
		const RadixSlot sl = slots[s];
		double sv, cv;
		sincos(slot_outer_angle(sl, terms, base), &sv, &cv);
		otab[o * stride + s] = to_v<V>(make_double2(cv * sl.scale, sv * sl.scale));
	}
}

struct BitRef {
	bool local;
	unsigned idx;  // local index, or global bit position for an outer bit
};

// The pass as a flat circuit: Hadamards and two-qubit phase terms.
struct PItem {
	bool is_h;
	unsigned l;       // Hadamard: local bit
	BitRef b0, b1;    // phase term bits
	double theta;
};

// A phase term of a factor slot: one bit (register slots) or two bits (the
// constant slot), none of them a register bit of the stage.
struct STerm {
	BitRef x, y;
	bool two;
	double theta;
};

struct RadixProgram {
	RadixGeom g{};
	std::vector<RadixStage> stages;
	std::vector<uint32_t> items;
	std::vector<double2> tabs;
	std::vector<RadixSlot> slots;
	std::vector<RadixTerm> terms;
};

// Builds the staged program of a pass; false if the pass does not qualify.
template <int RB>
bool build_radix_program(const FusedPass &pass, unsigned K, size_t vbytes, RadixProgram &P) {
	RadixGeom &g = P.g;
	g.K = K;
	for(unsigned i = 0; i < K; ++i) g.lpos[i] = pass.lpos[i];
	g.m = 0;
	while(g.m < K && pass.lpos[g.m] == g.m) ++g.m;
	g.ntiles = 1ull << (pass.n - K);
	g.lo = (K + 1) / 2;
	fill_roots(g.roots);
	auto ref_of = [&](unsigned bit) -> BitRef {
		for(unsigned i = 0; i < K; ++i)
			if(pass.lpos[i] == bit) return BitRef{true, i};
		return BitRef{false, bit};
	};

	std::vector<PItem> items;
	unsigned hcount = 0;
	for(const FusedOp &f : pass.ops) {
		switch(f.kind) {
			case kFH:
			case kFHChain:
			case kFHTwiddle:
				items.push_back(PItem{true, f.lt, {}, {}, 0.0});
				++hcount;
				if(f.kind != kFH)
					for(unsigned e = 0; e < f.lc; ++e) {
						const ChainEntry &ce = pass.chain[f.tab + e];
						const BitRef other = ce.local >= 0 ? BitRef{true, (unsigned)ce.local} : BitRef{false, ce.bit};
						items.push_back(PItem{false, 0, BitRef{true, f.lt}, other, ce.theta});
					}
				break;
			case kFCP: {
				const unsigned b0 = (unsigned)__builtin_ctzll(f.mask), b1 = 63u - (unsigned)__builtin_clzll(f.mask);
				items.push_back(PItem{false, 0, ref_of(b0), ref_of(b1), f.theta});
				break;
			}
			default: return false;
		}
	}
	if(hcount == 0) return false;

	// Stages: at most RB distinct Hadamard bits, each at most once.
	struct Stage {
		std::vector<unsigned> hbits;
		std::vector<size_t> items;
	};
	std::vector<Stage> st(1);
	for(size_t k = 0; k < items.size(); ++k) {
		if(items[k].is_h) {
			Stage &s = st.back();
			const bool dup = std::find(s.hbits.begin(), s.hbits.end(), items[k].l) != s.hbits.end();
			if(dup || s.hbits.size() == (size_t)RB) st.push_back(Stage{});
			st.back().hbits.push_back(items[k].l);
		}
		st.back().items.push_back(k);
	}
	if(st.size() > kRadixMaxStages) return false;

	const double scale = std::ldexp((hcount & 1u) ? 1.0 / std::sqrt(2.0) : 1.0, -(int)(hcount / 2));
	for(size_t si = 0; si < st.size(); ++si) {
		Stage &s = st[si];
		// Register bits: the stage's Hadamard bits, then the highest local bits
		// that no phase of the stage touches (their phases stay cross-stage).
		std::vector<unsigned> rb = s.hbits;
		uint32_t touched = 0;
		for(size_t k : s.items)
			if(!items[k].is_h) {
				if(items[k].b0.local) touched |= 1u << items[k].b0.idx;
				if(items[k].b1.local) touched |= 1u << items[k].b1.idx;
			}
		for(int pass2 = 0; pass2 < 2; ++pass2)
			for(int b = (int)K - 1; b >= 0 && rb.size() < (size_t)RB; --b) {
				const bool in = std::find(rb.begin(), rb.end(), (unsigned)b) != rb.end();
				if(!in && (pass2 == 1 || !((touched >> b) & 1u))) rb.push_back((unsigned)b);
			}
		RadixStage S{};
		S.first = (uint32_t)P.items.size();
		for(int i = 0; i < RB; ++i) S.rbit[i] = rb[i];
		std::vector<unsigned> sorted(rb.begin(), rb.end());
		std::sort(sorted.begin(), sorted.end());
		for(int i = 0; i < RB; ++i) S.rsorted[i] = sorted[i];
		for(int i = 0; i < RB; ++i) {
			S.imask[i] = (1u << sorted[i]) - 1u;
			const unsigned j = 1u << rb[i];
			// rswz of the kernel: 16-byte values j ^ ((j >> 3) & 7), 8-byte values
			// j ^ (((j >> 4) & 7) << 1).
			S.roff[i] = vbytes == 16 ? (j ^ ((j >> 3) & 7u)) : (j ^ (((j >> 4) & 7u) << 1));
			S.gbit[i] = 1ull << pass.lpos[rb[i]];
		}
		auto regidx = [&](const BitRef &r) -> int {
			if(!r.local) return -1;
			for(int i = 0; i < RB; ++i)
				if(rb[i] == r.idx) return i;
			return -1;
		};
		std::vector<std::vector<STerm>> pre(RB + 1), post(RB + 1);
		std::vector<const PItem *> run;
		int last_bfly = -1;  // register bit of the item just emitted, if a plain butterfly
		auto phase_of = [&](int r) {
			double ang = 0.0;
			for(const PItem *t : run) {
				const int ra = regidx(t->b0), rc = regidx(t->b1);
				if(((r >> ra) & 1) && ((r >> rc) & 1)) ang += t->theta;
			}
			return make_double2(std::cos(ang), std::sin(ang));
		};
		auto flush_run = [&]() {
			if(run.empty()) return;
			bool on_half = last_bfly >= 0;
			for(const PItem *t : run)
				if(regidx(t->b0) != last_bfly && regidx(t->b1) != last_bfly) on_half = false;
			const uint32_t first = (uint32_t)P.tabs.size();
			if(on_half) {
				// Every phase involves the bit just transformed: they act on its
				// |1> outputs only, as a table over the other register bits.
				const int tb = last_bfly, lo = (1 << tb) - 1;
				for(int q = 0; q < (1 << (RB - 1)); ++q) P.tabs.push_back(phase_of(((q & ~lo) << 1) | (q & lo) | (1 << tb)));
				P.items.back() = kRIButterflyTw | ((uint32_t)tb << 8) | (first << 16);
			} else {
				for(int r = 0; r < (1 << RB); ++r) P.tabs.push_back(phase_of(r));
				P.items.push_back(kRIDiag | (first << 16));
			}
			last_bfly = -1;
			run.clear();
		};
		// The stage as (Hadamard register bit, in-stage phases that follow it);
		// phases before the first Hadamard have register bit -1.
		std::vector<std::pair<int, std::vector<const PItem *>>> seq;
		std::vector<unsigned> hseen;
		for(size_t k : s.items) {
			const PItem &it = items[k];
			if(it.is_h) {
				seq.push_back({regidx(BitRef{true, it.l}), {}});
				hseen.push_back(it.l);
				continue;
			}
			const int ra = regidx(it.b0), rc = regidx(it.b1);
			if(ra >= 0 && rc >= 0) {
				if(seq.empty()) seq.push_back({-1, {}});
				seq.back().second.push_back(&it);
				continue;
			}
			if(ra < 0 && rc < 0) {
				post[0].push_back(STerm{it.b0, it.b1, true, it.theta});
				continue;
			}
			const int reg = ra >= 0 ? ra : rc;
			const BitRef other = ra >= 0 ? it.b1 : it.b0;
			const unsigned lbit = rb[reg];
			const bool h_before = std::find(hseen.begin(), hseen.end(), lbit) != hseen.end();
			const bool has_h = std::find(s.hbits.begin(), s.hbits.end(), lbit) != s.hbits.end();
			// Before the stage's Hadamard on its register bit: moved to the
			// stage start; after it (or with none): moved to the stage end.
			(h_before || !has_h ? post : pre)[reg + 1].push_back(STerm{other, {}, false, it.theta});
		}
		// The QFT ladder: Hadamard i (register bit i, in order) followed by the
		// controlled phases pi/2^(j-i) with every later Hadamard bit j.
		const int d = (int)s.hbits.size();
		bool qft = (int)seq.size() == d;
		for(int i = 0; qft && i < d; ++i) {
			const auto &T = seq[i].second;
			if(seq[i].first != i || (int)T.size() != d - 1 - i) {
				qft = false;
				break;
			}
			uint32_t seen = 0;
			for(const PItem *t : T) {
				const int a = regidx(t->b0), c = regidx(t->b1);
				const int other = a == i ? c : (c == i ? a : -1);
				const double want = std::ldexp(std::acos(-1.0), -(other - i));
				if(other <= i || other >= d || ((seen >> other) & 1u) || std::fabs(t->theta - want) > 1e-12 * want) {
					qft = false;
					break;
				}
				seen |= 1u << other;
			}
		}
		// Hadamards on register bits 0..d-1 with no phase between them (they
		// commute): one compiled network, then the in-stage phases that follow
		// the last of them.  When that one is on bit d-1 and has phases, it
		// stays a butterfly item of its own (its phases then ride on its |1>
		// outputs).
		bool walsh = d > 1 && !qft && (int)seq.size() == d;
		uint32_t wseen = 0;
		for(int i = 0; walsh && i < d; ++i) {
			const int r = seq[i].first;
			if(r < 0 || r >= d || ((wseen >> r) & 1u) || (i + 1 < d && !seq[i].second.empty())) walsh = false;
			else wseen |= 1u << r;
		}
		const bool tail_own = walsh && !seq.back().second.empty() && seq.back().first == d - 1;
		if(walsh && (!tail_own || d >= 3)) {
			P.items.push_back(kRIWalsh | ((uint32_t)(tail_own ? d - 1 : d) << 8));
			if(tail_own) {
				P.items.push_back(kRIButterfly | ((uint32_t)(d - 1) << 8));
				last_bfly = d - 1;
			}
			run = seq.back().second;
			flush_run();
		} else if(qft) {
			P.items.push_back(kRIQft | ((uint32_t)d << 8));
		} else {
			for(auto &e : seq) {
				if(e.first >= 0) {
					P.items.push_back(kRIButterfly | ((uint32_t)e.first << 8));
					last_bfly = e.first;
				}
				run = e.second;
				flush_run();
			}
		}
		S.count = (uint32_t)P.items.size() - S.first;

		const bool last = si + 1 == st.size();
		auto emit = [&](std::vector<std::vector<STerm>> &grp, bool with_scale, uint32_t &slot0, uint32_t &mask) -> bool {
			slot0 = (uint32_t)P.slots.size();
			mask = 0;
			for(int i = 0; i <= RB; ++i) {
				const bool sc = i == 0 && with_scale;
				if(grp[i].empty() && !sc) continue;
				mask |= 1u << i;
				std::vector<RadixTerm> A, B, O, X;
				for(const STerm &t : grp[i]) {
					const uint32_t y = t.two ? t.y.idx : kNoBit;
					const bool cross = t.two && (t.x.local != t.y.local || (t.x.local && (t.x.idx < g.lo) != (t.y.idx < g.lo)));
					if(cross) {
						// Only the constant slot holds two-bit terms.
						X.push_back(RadixTerm{t.x.idx, t.y.idx, t.theta, (t.x.local ? 0u : 1u) | (t.y.local ? 0u : 2u), 0,
						                      std::cos(t.theta), std::sin(t.theta)});
					} else if(!t.x.local) {
						O.push_back(RadixTerm{t.x.idx, y, t.theta, 0, 0, 0.0, 0.0});
					} else {
						(t.x.idx < g.lo ? A : B).push_back(RadixTerm{t.x.idx, y, t.theta, 0, 0, 0.0, 0.0});
					}
				}
				RadixSlot sl{};
				sl.scale = sc ? scale : 1.0;
				sl.a_first = (uint32_t)P.terms.size();
				sl.a_count = (uint32_t)A.size();
				P.terms.insert(P.terms.end(), A.begin(), A.end());
				sl.b_first = (uint32_t)P.terms.size();
				sl.b_count = (uint32_t)B.size();
				P.terms.insert(P.terms.end(), B.begin(), B.end());
				sl.o_first = (uint32_t)P.terms.size();
				sl.o_count = (uint32_t)O.size();
				P.terms.insert(P.terms.end(), O.begin(), O.end());
				sl.x_first = (uint32_t)P.terms.size();
				sl.x_count = (uint32_t)X.size();
				P.terms.insert(P.terms.end(), X.begin(), X.end());
				P.slots.push_back(sl);
			}
			return true;
		};
		if(!emit(pre, false, S.pre_slot, S.pre_mask) || !emit(post, last, S.post_slot, S.post_mask)) return false;
		if(S.post_mask & 1u) {
			S.post_xfirst = P.slots[S.post_slot].x_first;
			S.post_xcount = P.slots[S.post_slot].x_count;
		}
		// Direct stores from the last stage when the lowest non-register local
		// bits (the lanes) cover 32 contiguous bytes of the state.
		if(last) {
			const unsigned need = vbytes == 8 ? 2u : 1u;
			bool ok = g.m >= need;
			for(int i = 0; i < RB; ++i)
				if(rb[i] < need) ok = false;
			S.direct = ok ? 1u : 0u;
		}
		P.stages.push_back(S);
	}
	g.nstages = (unsigned)P.stages.size();
	g.nitems = (unsigned)P.items.size();
	g.ntab = (unsigned)P.tabs.size();
	g.nslots = (unsigned)P.slots.size();
	g.nterms = (unsigned)P.terms.size();
	g.outer_free = 1;
	for(const RadixSlot &sl : P.slots)
		if(sl.o_count) g.outer_free = 0;
	return g.nitems <= kRadixMaxItems && g.ntab <= kRadixMaxTab && g.nslots <= kRadixMaxSlots;
}

size_t radix_smem_bytes(size_t vbytes, const RadixGeom &g) {
	auto a16 = [](size_t b) { return (b + 15) & ~size_t(15); };
	const size_t nb = size_t(1) << (g.K - g.lo);
	const size_t stride = (g.nslots * vbytes + 15) / 16 * 16;
	return 2 * a16(vbytes << g.K) + a16(sizeof(uint64_t) << (g.K - g.m)) + a16(sizeof(RadixStage) * g.nstages) +
	       a16(sizeof(uint32_t) * g.nitems) + a16(vbytes * g.ntab) + a16(vbytes * ((size_t)g.nslots << g.lo)) +
	       a16(vbytes * g.nslots * nb) + 2 * a16(stride);
}

template <typename R, int RB>
bool run_radix(const LaunchCtx &c, void *a, const FusedPass &pass, void *&dev_prog, size_t &dev_prog_bytes, void *mirror) {
	typedef typename Vec2<R>::type V;
	const unsigned K = pass.K;
	if(K < (unsigned)RB + 5 || K > 13 || (1u << (K - RB)) > kRadixThreads) return false;
	RadixProgram P;
	if(!build_radix_program<RB>(pass, K, sizeof(V), P)) return false;
	// 16-byte copy granules: two complex64 amplitudes must be adjacent.
	if(sizeof(V) == 8 && P.g.m < 1) return false;
	const size_t smem = radix_smem_bytes(sizeof(V), P.g);
	int dev = 0, max_optin = 0;
	check_cuda(cudaGetDevice(&dev), "radix device");
	check_cuda(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "radix smem limit");
	if(smem > (size_t)max_optin) return false;

	// Program upload: stages | items | tables | slots | terms.
	auto a256 = [](size_t b) { return (b + 255) & ~size_t(255); };
	const size_t o_st = 0, o_it = o_st + a256(P.stages.size() * sizeof(RadixStage)),
	             o_tb = o_it + a256(P.items.size() * sizeof(uint32_t)), o_sl = o_tb + a256(P.tabs.size() * sizeof(double2)),
	             o_tm = o_sl + a256(P.slots.size() * sizeof(RadixSlot)),
	             o_ot = o_tm + a256(P.terms.size() * sizeof(RadixTerm));
	// Per-tile outer phases: ot_stride storage values per tile (16-byte rows).
	const unsigned ot_stride = (unsigned)((P.g.nslots * sizeof(V) + 15) / 16 * 16 / sizeof(V));
	const size_t upload = std::max<size_t>(256, o_ot), need = o_ot + a256(P.g.ntiles * ot_stride * sizeof(V));
	if(need > dev_prog_bytes) {
		if(dev_prog) {
			check_cuda(cudaStreamSynchronize(c.stream), "radix program sync");
			cudaFree(dev_prog);
		}
		dev_prog = nullptr;
		dev_prog_bytes = 0;
		const size_t want = need + need / 8;
		if(device_alloc((void **)&dev_prog, want) != cudaSuccess) {
			cudaGetLastError();
			fail(TMFQS_ERR_NOMEM, "radix pass program allocation failed");
		}
		dev_prog_bytes = want;
	}
	std::vector<unsigned char> host(upload, 0);
	std::memcpy(host.data() + o_st, P.stages.data(), P.stages.size() * sizeof(RadixStage));
	std::memcpy(host.data() + o_it, P.items.data(), P.items.size() * sizeof(uint32_t));
	std::memcpy(host.data() + o_tb, P.tabs.data(), P.tabs.size() * sizeof(double2));
	std::memcpy(host.data() + o_sl, P.slots.data(), P.slots.size() * sizeof(RadixSlot));
	std::memcpy(host.data() + o_tm, P.terms.data(), P.terms.size() * sizeof(RadixTerm));
	upload_async(c, dev_prog, host.data(), upload, "radix program upload");
	unsigned char *pbase = static_cast<unsigned char *>(dev_prog);
	V *otab = reinterpret_cast<V *>(pbase + o_ot);
	if(P.g.nslots && !P.g.outer_free) {
		const uint64_t work = P.g.ntiles * P.g.nslots;
		const unsigned blocks = (unsigned)std::min<uint64_t>((work + 255) / 256, (uint64_t)c.num_sms * 8);
		k_outer_table<R><<<blocks, 256, 0, c.stream>>>(otab, ot_stride, P.g, reinterpret_cast<const RadixSlot *>(pbase + o_sl),
		                                               reinterpret_cast<const RadixTerm *>(pbase + o_tm));
		check_cuda(cudaGetLastError(), "radix outer phases");
		if(c.launches) ++*c.launches;
	}

	const unsigned threads = 1u << (K - RB);
	check_cuda(cudaFuncSetAttribute(k_radix<R, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "radix smem");
	const uint64_t grid = std::min<uint64_t>(P.g.ntiles, (uint64_t)c.num_sms);
	k_radix<R, RB><<<(unsigned)grid, threads, smem, c.stream>>>(static_cast<V *>(a), P.g,
	                                                           static_cast<const unsigned char *>(dev_prog), o_st, o_it,
	                                                           o_tb, o_sl, o_tm, otab, ot_stride, static_cast<V *>(mirror));
	check_cuda(cudaGetLastError(), "radix pass");
	if(c.launches) ++*c.launches;
	return true;
}

}  // namespace

bool launch_radix_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, void *&dev_prog,
                       size_t &dev_prog_bytes, void *mirror) {
	if(prec == TMFQS_FP64) return run_radix<double, 3>(c, a, pass, dev_prog, dev_prog_bytes, mirror);
	return run_radix<float, 4>(c, a, pass, dev_prog, dev_prog_bytes, mirror);
}

}  // namespace tqb
