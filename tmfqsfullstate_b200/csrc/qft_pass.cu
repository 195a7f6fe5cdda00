// QFT segment passes for the fast forms (complex64 states, and complex128 with
// TMFQS_OPT_EXACT off).
//
// A pass of the QFT ladder (circuit::appendQft, circuit.cpp:87-100) covers a
// run of qubits whose index bits b are consecutive and descending: H on b,
// then the controlled phases pi/2^(b-c) with every lower bit c of the
// register (c >= r0).  In the pass:
//   - the Hadamards and the phases between the run's own bits form a small
//     QFT on those bits, done in registers as compiled ladders of up to RB bits
//     (one "stage" each: the 2^RB amplitudes of a thread differ in the stage's
//     bits);
//   - the phases between a stage's bits and every lower bit c (later stages,
//     the low local bits, outer bits) commute with the rest of the stage, so
//     they are applied after it as one twiddle per amplitude:
//         exp(2*pi*i * W / 2^(b+1)) for each stage bit b in state |1>,
//     W = the value of the bits in [r0, lowest bit of the stage).
//     The factor of bit b splits into a per-thread part (the local bits of W:
//     the same for every tile, tabulated per thread at the start of the
//     launch) and a per-tile part (the outer bits of W, computed by one thread
//     per stage while the tile's copies are in flight).  Both come from
//     sincospi in FP64 and FP64 squarings, each rounded once.
// Tiles of 2^K amplitudes stream through a ring of shared-memory buffers with
// 16-byte cp.async copies (two tiles in flight behind the one being
// transformed); a thread's copies sit at fixed offsets from the tile base.  Stage accesses use an XOR swizzle chosen per pass on the
// host so that the lanes of each half-warp (quarter-warp for complex128) hit
// distinct banks wherever the pass's bit layout allows it.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"
#include "radix_common.cuh"

namespace tqb {

namespace {

constexpr unsigned kQftMaxStages = 4;
constexpr unsigned kQftMaxRuns = 8;

// Threads per CTA: 2^(K - RB) for tiles of 2^K amplitudes, at most 512 (a
// complex64 kernel with 4 register bits), else 256.
constexpr unsigned qft_max_threads(size_t vbytes, int RB) { return vbytes == 8 && RB == 4 ? 512u : 256u; }

// Local bits of a full-size tile (64 KiB): 13 complex64, 12 complex128.
constexpr int qft_tile_bits(size_t vbytes) { return vbytes == 8 ? 13 : 12; }
constexpr uint32_t kQftNone = 0xffffffffu;

struct QftStage {
	uint32_t d;           // Hadamards of the stage: register bits 0..d-1, in circuit order
	uint32_t bhi;         // global bit of register bit 0 (register bit i < d is bit bhi - i)
	uint32_t rsorted[5];  // the register local bits, ascending
	uint32_t roff[5];     // swizzled shared-memory offset (elements) of register bit i
	uint32_t fl;          // first per-thread factor row, kQftNone: no twiddle
	uint32_t ot;          // first per-tile factor in a factor row, kQftNone: none
	uint32_t scaled;      // the pass's real scale (1/sqrt(2))^P is applied here (the last stage)
	uint32_t direct;      // last stage: results go straight to HBM (lanes run along >= 64-byte rows)
	uint32_t top;         // register bit i is local bit kTop - 1 - i (the tile's top bits), unswizzled
	uint32_t tail;        // last stage on the tile's lowest bits, fused into the copy-out (qft_tail)
	uint32_t walsh;       // Hadamards only (a Walsh segment): butterflies, no phases
	uint32_t pad_;
	uint64_t wmask;       // the bits of W: [r0, lowest Hadamard bit of the stage)
	uint64_t gstride[5];  // global element offset of register bit i
};

struct QftGeom {
	uint32_t K;        // local bits: tiles of 2^K amplitudes
	uint32_t nstages;
	uint32_t slots;    // tile buffers in the ring (2 or 3)
	uint32_t nruns;    // runs of outer bits, ascending: tile index bits in order
	uint32_t run_pos[kQftMaxRuns], run_len[kQftMaxRuns];
	uint32_t lpos[16];               // local bit -> global bit
	uint32_t sw_src[3], sw_dst[3];   // swizzle: shared index bit sw_dst[k] ^= index bit sw_src[k] (src 0: none)
	uint32_t ot_stride;  // storage values per per-tile factor row (16-byte rows), 0: none
	uint32_t nfrows;     // per-thread factor rows
	uint64_t localmask;
	uint64_t ntiles;
	uint64_t istride;    // global element step between a thread's granules
	double scale;
	// Tiles by one tensor-map copy (complex64): the state as a tensor whose
	// dimensions are runs of index bits, ascending -- local runs (split so
	// that the innermost is 16 amplitudes = one 128-byte swizzle row and the
	// others hold at most 256) are the box, outer runs are box-1 dimensions
	// whose coordinates are the tile index bits of that run.
	uint32_t tma, tma_dims;
	uint32_t tma_outer[5], tma_shift[5], tma_len[5];
	uint64_t tma_size[5], tma_stride[5];  // elements; bytes (dimension 0: the element)
	uint32_t tma_box[5];
	QftStage st[kQftMaxStages];
	RootTable roots;
};

template <typename V>
struct Scalar;
template <>
struct Scalar<float2> {
	typedef float type;
};
template <>
struct Scalar<double2> {
	typedef double type;
};

template <typename V>
__device__ __forceinline__ V vscale(V v, typename Scalar<V>::type s) {
	v.x *= s;
	v.y *= s;
	return v;
}

template <typename V>
__device__ __forceinline__ V to_storage(double x, double y) {
	V z;
	z.x = (typename Scalar<V>::type)x;
	z.y = (typename Scalar<V>::type)y;
	return z;
}

// dst[i * stride] = exp(2*pi*i * w / 2^(bhi+1-i)), i < d: the twiddles of
// the stage bits bhi, bhi-1, ... for W = w.  The first from sincospi in FP64
// (w < 2^bhi, so the argument is exact), the rest by squaring in FP64; each
// rounded once to the storage type.
template <typename V>
__device__ __forceinline__ void stage_factors(uint64_t w, unsigned bhi, unsigned d, V *dst, unsigned stride) {
	double s, c;
	sincospi(ldexp((double)w, -(int)bhi), &s, &c);
	for(unsigned i = 0; i < d; ++i) {
		dst[i * stride] = to_storage<V>(c, s);
		const double c2 = c * c - s * s, s2 = 2.0 * c * s;
		c = c2;
		s = s2;
	}
}

__host__ __device__ __forceinline__ unsigned qft_phys(const QftGeom &g, unsigned j) {
	unsigned x = j;
#pragma unroll
	for(int k = 0; k < 3; ++k)
		if(g.sw_src[k]) x ^= ((j >> g.sw_src[k]) & 1u) << g.sw_dst[k];
	return x;
}

__device__ __forceinline__ uint64_t qft_scatter(const QftGeom &g, unsigned j) {
	uint64_t x = 0;
	for(unsigned l = 0; l < g.K; ++l)
		if((j >> l) & 1u) x |= 1ull << g.lpos[l];
	return x;
}

// Global element offset of the first amplitude of tile o: the bits of o
// deposited into the runs of outer bits.
__device__ __forceinline__ uint64_t qft_tile_base(const QftGeom &g, uint64_t o) {
	uint64_t base = 0;
	for(unsigned k = 0; k < g.nruns; ++k) {
		const unsigned len = g.run_len[k];
		base |= (o & ((1ull << len) - 1ull)) << g.run_pos[k];
		o >>= len;
	}
	return base;
}

// v[r] times prod_{i < D, r_i = 1} f[i] (the filler bits D.. carry no factor),
// and the real scale s on every value when SC.  The products come from two
// small tables over bits 0..2 and 3..D-1, applied one after the other (at most
// two complex products per amplitude; only one table is live at a time).
template <typename V, int RB, int D, bool SC>
__device__ __forceinline__ void apply_twiddle(V (&v)[1 << RB], const V (&f)[D], typename Scalar<V>::type s) {
	constexpr int LO = D < 3 ? D : 3, HI = D - LO;
	{
		V FL[1 << LO];
#pragma unroll
		for(int k = 1; k < (1 << LO); ++k) {
			const int hb = 31 - __clz(k);
			FL[k] = (k == (1 << hb)) ? f[hb] : vmul(FL[k ^ (1 << hb)], f[hb]);
			if constexpr(SC) {
				if(k == (1 << hb)) FL[k] = vscale(FL[k], s);
			}
		}
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) {
			const int lo = r & ((1 << LO) - 1);
			if(lo) v[r] = vmul(v[r], FL[lo]);
			else if(SC) v[r] = vscale(v[r], s);
		}
	}
	if constexpr(HI > 0) {
		V FH[1 << HI];
#pragma unroll
		for(int k = 1; k < (1 << HI); ++k) {
			const int hb = 31 - __clz(k);
			FH[k] = (k == (1 << hb)) ? f[LO + hb] : vmul(FH[k ^ (1 << hb)], f[LO + hb]);
		}
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) {
			const int hi = (r & ((1 << D) - 1)) >> LO;
			if(hi) v[r] = vmul(v[r], FH[hi]);
		}
	}
}

// One stage on the tile in shared memory: the thread's 2^RB amplitudes are
// read, transformed (ladder, twiddle, scale) and written back in place.
// Butterflies on register bits 0..D-1 (a Walsh-Hadamard stage), unscaled.
template <typename V, int RB, int D>
__device__ __forceinline__ void walsh_ladder(V (&v)[1 << RB]) {
#pragma unroll
	for(int i = 0; i < D; ++i) {
#pragma unroll
		for(int q = 0; q < (1 << (RB - 1)); ++q) {
			const int lo = (1 << i) - 1;
			const int r0 = ((q & ~lo) << 1) | (q & lo), r1 = r0 | (1 << i);
			bfly2(v[r0], v[r1]);
		}
	}
}

template <typename V, int RB, int D, bool TW, bool SC, bool TOP, bool W = false>
__device__ __forceinline__ void qft_stage_run(V *tile, const QftStage &S, unsigned pbase, const V *frow, unsigned nthr,
                                              const V *ot, typename Scalar<V>::type s, const RootTable &roots, V *gdst) {
	// TOP: the register bits are the tile's top local bits in order, so the
	// offsets are compile-time constants added to the thread's base.
	constexpr int kTop = qft_tile_bits(sizeof(V));
	unsigned roff[RB];
#pragma unroll
	for(int i = 0; i < RB; ++i) roff[i] = TOP ? (1u << (kTop - 1 - i)) : S.roff[i];
	V v[1 << RB];
#pragma unroll
	for(int r = 0; r < (1 << RB); ++r) {
		unsigned x = TOP ? 0u : pbase;
#pragma unroll
		for(int i = 0; i < RB; ++i)
			if((r >> i) & 1) x ^= roff[i];
		v[r] = TOP ? tile[pbase + x] : tile[x];
	}
	if constexpr(W) walsh_ladder<V, RB, D>(v);
	else qft_stage<V, RB, D>(v, roots);
	if constexpr(TW) {
		V f[D];
#pragma unroll
		for(int i = 0; i < D; ++i) f[i] = frow[i * nthr];
		const unsigned oc = S.ot;
		if(oc != kQftNone) {
#pragma unroll
			for(int i = 0; i < D; ++i) f[i] = vmul(f[i], ot[oc + i]);
		}
		apply_twiddle<V, RB, D, SC>(v, f, s);
	} else if constexpr(SC) {
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) v[r] = vscale(v[r], s);
	}
	if(SC && gdst) {
		// The last stage's lanes run along the low index bits: coalesced rows.
		uint64_t gs[RB];
#pragma unroll
		for(int i = 0; i < RB; ++i) gs[i] = S.gstride[i];
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) {
			uint64_t x = 0;
#pragma unroll
			for(int i = 0; i < RB; ++i)
				if((r >> i) & 1) x += gs[i];
			gdst[x] = v[r];
		}
		return;
	}
#pragma unroll
	for(int r = 0; r < (1 << RB); ++r) {
		unsigned x = TOP ? 0u : pbase;
#pragma unroll
		for(int i = 0; i < RB; ++i)
			if((r >> i) & 1) x ^= roff[i];
		if(TOP) tile[pbase + x] = v[r];
		else tile[x] = v[r];
	}
}

template <typename V, int RB, int D>
__device__ __forceinline__ void qft_stage_flags(V *tile, const QftStage &S, unsigned pbase, const V *frow, unsigned nthr,
                                                const V *ot, typename Scalar<V>::type s, const RootTable &roots, V *gdst) {
	const bool tw = S.fl != kQftNone;
	if(S.walsh) {
		if(S.scaled) qft_stage_run<V, RB, D, false, true, false, true>(tile, S, pbase, frow, nthr, ot, s, roots, gdst);
		else qft_stage_run<V, RB, D, false, false, false, true>(tile, S, pbase, frow, nthr, ot, s, roots, nullptr);
	} else if(tw) {
		if(S.scaled) qft_stage_run<V, RB, D, true, true, false>(tile, S, pbase, frow, nthr, ot, s, roots, gdst);
		else if(S.top) qft_stage_run<V, RB, D, true, false, true>(tile, S, pbase, frow, nthr, ot, s, roots, nullptr);
		else qft_stage_run<V, RB, D, true, false, false>(tile, S, pbase, frow, nthr, ot, s, roots, nullptr);
	} else {
		if(S.scaled) qft_stage_run<V, RB, D, false, true, false>(tile, S, pbase, frow, nthr, ot, s, roots, gdst);
		else qft_stage_run<V, RB, D, false, false, false>(tile, S, pbase, frow, nthr, ot, s, roots, nullptr);
	}
}

template <typename V, int RB>
__device__ __forceinline__ void qft_stage_dispatch(V *tile, const QftStage &S, unsigned pbase, const V *frow, unsigned nthr,
                                                   const V *ot, typename Scalar<V>::type s, const RootTable &roots,
                                                   V *gdst) {
	switch(S.d) {
		case 1: qft_stage_flags<V, RB, 1>(tile, S, pbase, frow, nthr, ot, s, roots, gdst); break;
		case 2: qft_stage_flags<V, RB, 2>(tile, S, pbase, frow, nthr, ot, s, roots, gdst); break;
		case 3: qft_stage_flags<V, RB, 3>(tile, S, pbase, frow, nthr, ot, s, roots, gdst); break;
		case 4: qft_stage_flags<V, RB, 4>(tile, S, pbase, frow, nthr, ot, s, roots, gdst); break;
		case 5: if constexpr(RB >= 5) qft_stage_flags<V, RB, 5>(tile, S, pbase, frow, nthr, ot, s, roots, gdst); break;
		default: break;
	}
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

// Arrives on the barrier once this thread's earlier cp.async copies are done
// (the barrier's count includes this arrival: .noinc).
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t *b) {
	asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, unsigned parity) {
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(smem_u32(b)), "r"(parity)
		: "memory");
	return ok != 0;
}

// Expect `bytes` of asynchronous copies on the barrier and arrive (the
// barrier's count is 1 for tensor-map tiles: the issuing thread).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *b, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

// Tile o by one tensor-map copy: coordinates 0 on the box dimensions, the
// tile index bits of each outer run on the others; completion on `bar`.
__device__ __forceinline__ void tma_tile(void *dst, const CUtensorMap *tm, const QftGeom &g, uint64_t o, uint64_t *bar) {
	int c[5] = {0, 0, 0, 0, 0};
#pragma unroll
	for(unsigned i = 0; i < 5; ++i)
		if(i < g.tma_dims && g.tma_outer[i]) c[i] = (int)((o >> g.tma_shift[i]) & ((1ull << g.tma_len[i]) - 1ull));
	const uint32_t d = smem_u32(dst), m = smem_u32(bar);
	const uint64_t t = reinterpret_cast<uint64_t>(tm);
	switch(g.tma_dims) {
		case 2:
			asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
			             ::"r"(d), "l"(t), "r"(c[0]), "r"(c[1]), "r"(m) : "memory");
			break;
		case 3:
			asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
			             ::"r"(d), "l"(t), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(m) : "memory");
			break;
		case 4:
			asm volatile(
				"cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
				::"r"(d), "l"(t), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(m) : "memory");
			break;
		default:
			asm volatile(
				"cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
				"[%7];" ::"r"(d), "l"(t), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(m) : "memory");
			break;
	}
}

// Upper bound on the polls of a tile's arrival (each poll may suspend the
// thread for a while).  Past it the thread records the failure in the
// handle's error word and goes on (every thread keeps the same barrier
// sequence; the host reports the error after the pass).
constexpr int kQftWaitPolls = 1 << 22;

// r with its low d bits reversed (a loop, not recursion, so that it folds once
// the callers' loops are unrolled).
__host__ __device__ constexpr int brev_bits(int r, int d) {
	int x = 0;
	for(int i = 0; i < d; ++i) x |= ((r >> i) & 1) << (d - 1 - i);
	return x;
}

// The pass's last D Hadamards when they sit on the tile's lowest bits (local
// bits D-1..0 = global bits D-1..0, no twiddle after them), fused into the
// copy-out: each thread takes 2^D consecutive amplitudes from shared memory,
// applies their ladder and the pass's scale, and stores them contiguously
// (consecutive threads take consecutive groups).  Register bit i is local bit
// D-1-i, so register r holds element brev(r).
template <typename V, int D, bool W>
__device__ __forceinline__ void qft_tail(const V *tile, V *dst, unsigned T, unsigned tid, unsigned nthr, const QftGeom &g,
                                         typename Scalar<V>::type s) {
	constexpr unsigned E = 1u << D;
	unsigned pe[E];
#pragma unroll
	for(unsigned e = 0; e < E; ++e) pe[e] = qft_phys(g, e);
	for(unsigned q = tid; q < T / E; q += nthr) {
		const unsigned j = q * E, pj = qft_phys(g, j);
		V in[E];
		if constexpr(sizeof(V) == 8) {
			// 16-byte reads: elements e and e + 1 stay adjacent under the swizzle.
#pragma unroll
			for(unsigned e = 0; e < E; e += 2) {
				const float4 t = *reinterpret_cast<const float4 *>(tile + (pj ^ pe[e]));
				in[e] = make_float2(t.x, t.y);
				in[e + 1] = make_float2(t.z, t.w);
			}
		} else {
#pragma unroll
			for(unsigned e = 0; e < E; ++e) in[e] = tile[pj ^ pe[e]];
		}
		V v[E];
#pragma unroll
		for(int r = 0; r < (int)E; ++r) v[r] = in[brev_bits(r, D)];
		if constexpr(W) walsh_ladder<V, D, D>(v);
		else qft_stage<V, D, D>(v, g.roots);
		V out[E];
#pragma unroll
		for(int r = 0; r < (int)E; ++r) out[brev_bits(r, D)] = vscale(v[r], s);
		// 32-byte stores where a group spans whole sectors (sm_100 vector
		// width): a lane then writes full sectors, not halves.
		auto store = [&](V *d) {
			if constexpr(sizeof(V) == 8 && E >= 4) {
#pragma unroll
				for(unsigned e = 0; e < E; e += 4)
					asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(d + j + e), "f"(out[e].x),
					             "f"(out[e].y), "f"(out[e + 1].x), "f"(out[e + 1].y), "f"(out[e + 2].x), "f"(out[e + 2].y),
					             "f"(out[e + 3].x), "f"(out[e + 3].y)
					             : "memory");
			} else if constexpr(sizeof(V) == 8) {
#pragma unroll
				for(unsigned e = 0; e < E; e += 2)
					*reinterpret_cast<float4 *>(d + j + e) = make_float4(out[e].x, out[e].y, out[e + 1].x, out[e + 1].y);
			} else if constexpr(E >= 2) {
#pragma unroll
				for(unsigned e = 0; e < E; e += 2)
					asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(d + j + e), "d"((double)out[e].x),
					             "d"((double)out[e].y), "d"((double)out[e + 1].x), "d"((double)out[e + 1].y)
					             : "memory");
			} else {
#pragma unroll
				for(unsigned e = 0; e < E; ++e) d[j + e] = out[e];
			}
		};
		store(dst);
	}
}

// The pass.  Shared memory: the ring of tile buffers, the stage descriptors,
// the per-thread twiddle factors [nfrows][nthr], the swizzled index of each
// thread's first amplitude per stage [nstages][nthr], and one row of per-tile
// factors per ring slot.  Everything is derived here from the geometry: the
// launch needs no device program.
template <typename R, int RB, bool TM>
__global__ void __launch_bounds__(qft_max_threads(sizeof(typename Vec2<R>::type), RB), 1)
	k_qft_pass(typename Vec2<R>::type *a, const __grid_constant__ QftGeom g, const __grid_constant__ CUtensorMap tmap,
	           int *err) {
	typedef typename Vec2<R>::type V;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	constexpr unsigned per16 = 16 / sizeof(V);
	constexpr unsigned kGranules = (1u << RB) / per16;  // 16-byte granules per thread per tile
	const unsigned T = 1u << g.K, tid = threadIdx.x, nthr = blockDim.x;
	// TM (tiles by tensor-map copies): the ring starts on a 1024-byte
	// boundary (the copy's 128-byte swizzle repeats every 1024 bytes of
	// shared address).
	V *ring = reinterpret_cast<V *>(TM ? smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u) : smem_raw);
	V *ftab = ring + (size_t)g.slots * T;
	V *orow = ftab + (size_t)g.nfrows * nthr;
	QftStage *sst = reinterpret_cast<QftStage *>(orow + (size_t)g.slots * g.ot_stride);
	uint64_t *mbar = reinterpret_cast<uint64_t *>(sst + kQftMaxStages);  // [slots]: arrival of each slot's tile
	uint16_t *spst = reinterpret_cast<uint16_t *>(mbar + g.slots);

	if(tid < g.nstages) sst[tid] = g.st[tid];
	if(tid == 0)
		for(unsigned k = 0; k < g.slots; ++k) mbar_init(&mbar[k], TM ? 1u : nthr);
	const uint64_t goff = qft_scatter(g, tid * per16);
	const unsigned psm = qft_phys(g, tid * per16);
	const unsigned gstep = nthr * per16;  // shared index step between a thread's granules
	__syncthreads();

	// Tile o's amplitudes (16-byte granules at fixed per-thread offsets) and,
	// from one thread per stage, its row of per-tile factors (the outer bits
	// of W), computed while the copies are in flight.
	auto prefetch = [&](uint64_t o, unsigned slot) {
		if(o < g.ntiles) {
			const uint64_t base = qft_tile_base(g, o);
			if constexpr(TM) {
				// One thread: the slot's earlier generic reads and writes are
				// ordered before the copy by the barrier that precedes this call
				// and the proxy fence.
				if(tid == 0) {
					asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
					mbar_arrive_expect_tx(&mbar[slot], (uint32_t)(T * sizeof(V)));
					tma_tile(ring + (size_t)slot * T, &tmap, g, o, &mbar[slot]);
				}
			} else {
				const V *src = a + base + goff;
				V *dst = ring + (size_t)slot * T + psm;
#pragma unroll
				for(unsigned i = 0; i < kGranules; ++i) cp_async16(dst + i * gstep, src + i * g.istride);
				cp_async_mbar_arrive(&mbar[slot]);
			}
			const unsigned st = tid >> 5;
			if((tid & 31u) == 0 && st < g.nstages && sst[st].ot != kQftNone)
				stage_factors<V>(base & sst[st].wmask & ~g.localmask, sst[st].bhi, sst[st].d,
				                 orow + slot * g.ot_stride + sst[st].ot, 1);
		}
	};
	uint64_t o = blockIdx.x;
	for(unsigned k = 0; k + 1 < g.slots; ++k) prefetch(o + (uint64_t)k * gridDim.x, k);

	// Per-thread tables (once per launch), and the global offset of the
	// thread's first amplitude in the last stage (direct stores).
	uint64_t slast = 0;
	for(unsigned st = 0; st < g.nstages; ++st) {
		const QftStage &S = sst[st];
		unsigned jt = tid;
		for(unsigned i = 0; i < RB; ++i) {
			const unsigned b = S.rsorted[i], lo = jt & ((1u << b) - 1u);
			jt = ((jt ^ lo) << 1) | lo;
		}
		spst[st * nthr + tid] = (uint16_t)qft_phys(g, jt);
		if(S.fl != kQftNone) stage_factors<V>(qft_scatter(g, jt) & S.wmask, S.bhi, S.d, ftab + (size_t)S.fl * nthr + tid, nthr);
		if(st + 1 == g.nstages) slast = qft_scatter(g, jt);
	}
	const bool direct = sst[g.nstages - 1].direct != 0;
	const bool tail = sst[g.nstages - 1].tail != 0, wtail = sst[g.nstages - 1].walsh != 0;
	const unsigned nrun = tail ? g.nstages - 1 : g.nstages;  // stages run through shared memory

	const typename Scalar<V>::type s = (typename Scalar<V>::type)g.scale;
	__syncthreads();  // tables and barrier initialisation visible
	unsigned slot = 0, phase = 0, stuck_phase = 0;
	int stuck = -1;  // a slot whose tile did not arrive in time (its copy may still land)
	for(; o < g.ntiles; o += gridDim.x) {
		// The tile's copies (every thread's) are done once the slot's barrier
		// completes this phase.
		bool ready = false;
		for(int it = 0; it < kQftWaitPolls && !ready; ++it) ready = mbar_try_wait(&mbar[slot], phase);
		if(!ready) {
			atomicExch(err, 1);
			if constexpr(TM) {
				stuck = (int)slot;
				stuck_phase = phase;
			}
		}
		V *tile = ring + (size_t)slot * T;
		const V *ot = orow + slot * g.ot_stride;
		const uint64_t tbase = qft_tile_base(g, o);
		for(unsigned st = 0; st < nrun; ++st) {
			const QftStage &S = sst[st];
			const V *frow = ftab + (size_t)(S.fl == kQftNone ? 0u : S.fl) * nthr + tid;
			const bool last = st + 1 == g.nstages;
			qft_stage_dispatch<V, RB>(tile, S, spst[st * nthr + tid], frow, nthr, ot, s, g.roots,
			                          last && direct ? a + tbase + slast : nullptr);
			if(!(last && direct)) __syncthreads();
			// Past the first stage's barrier every thread is done with the
			// previous tile's buffer: the next copies go there.  (A pass of one
			// direct stage has no barrier of its own: take one.)
			if(st == 0) {
				if(last && direct) __syncthreads();
				prefetch(o + (uint64_t)(g.slots - 1) * gridDim.x, slot == 0 ? g.slots - 1 : slot - 1);
			}
		}
		if(tail) {
			switch(sst[g.nstages - 1].d) {
				case 1: wtail ? qft_tail<V, 1, true>(tile, a + tbase, T, tid, nthr, g, s)
				              : qft_tail<V, 1, false>(tile, a + tbase, T, tid, nthr, g, s); break;
				case 2: wtail ? qft_tail<V, 2, true>(tile, a + tbase, T, tid, nthr, g, s)
				              : qft_tail<V, 2, false>(tile, a + tbase, T, tid, nthr, g, s); break;
				case 3: wtail ? qft_tail<V, 3, true>(tile, a + tbase, T, tid, nthr, g, s)
				              : qft_tail<V, 3, false>(tile, a + tbase, T, tid, nthr, g, s); break;
				default: break;
			}
		} else if(!direct) {
			V *dst = a + tbase + goff;
			const V *src = tile + psm;
#pragma unroll
			for(unsigned i = 0; i < kGranules; ++i)
				*reinterpret_cast<float4 *>(dst + i * g.istride) = *reinterpret_cast<const float4 *>(src + i * gstep);
		}
		if(++slot == g.slots) {
			slot = 0;
			phase ^= 1u;
		}
	}
	cp_async_wait_all();
	// After a timeout, wait (bounded again) for the late copy before the
	// shared memory is released.
	if constexpr(TM) {
		if(stuck >= 0)
			for(int it = 0; it < kQftWaitPolls && !mbar_try_wait(&mbar[stuck], stuck_phase); ++it) {
			}
	}
}

// ---------------------------------------------------------------------------
// Host side: recognising a QFT segment and planning its pass.

// Hadamards on consecutive descending bits hb[0] > hb[1] > ..., each followed
// by the controlled phases pi/2^(b-c) with every bit c in [r0, b) (in any
// order), and nothing else.  The compiled ladders apply the phases between the
// segment's own bits, so every Hadamard above the lowest must carry its chain
// and the lowest Hadamard bit is r0 or above (its own chain may be empty only
// when it sits at r0).  A lone Hadamard (no phases at all) is a segment too.
bool qft_segment(const FusedPass &pass, std::vector<unsigned> &hb, unsigned &r0) {
	hb.clear();
	r0 = pass.n;
	bool have_r0 = false, bare = false;
	const double pi = std::acos(-1.0);
	for(const FusedOp &f : pass.ops) {
		if(f.kind != kFH && f.kind != kFHChain && f.kind != kFHTwiddle) return false;
		if(f.lt >= pass.K) return false;
		if(bare) return false;  // only the lowest Hadamard may lack phases
		const unsigned b = pass.lpos[f.lt];
		if(!hb.empty() && b + 1 != hb.back()) return false;
		const unsigned cnt = f.kind == kFH ? 0u : f.lc;
		uint64_t seen = 0;
		unsigned lo = b;
		for(unsigned e = 0; e < cnt; ++e) {
			const ChainEntry &ce = pass.chain[f.tab + e];
			const unsigned c = ce.bit;
			if(c >= b || ((seen >> c) & 1ull)) return false;
			seen |= 1ull << c;
			lo = std::min(lo, c);
			const double want = std::ldexp(pi, -(int)(b - c));
			if(!(std::fabs(ce.theta - want) <= 1e-12 * want)) return false;
		}
		if(cnt != b - lo) return false;  // the phases cover [lo, b) exactly
		if(cnt) {
			if(!have_r0) {
				r0 = lo;
				have_r0 = true;
			} else if(lo != r0) {
				return false;
			}
		} else {
			bare = true;
		}
		hb.push_back(b);
	}
	if(hb.empty()) return false;
	if(!have_r0) return hb.size() == 1;  // Hadamards without phases: only a lone one
	if(bare && hb.back() != r0) return false;
	return hb.back() >= r0;
}

// Hadamards only, on two or more distinct local bits (a Walsh-Hadamard
// segment: the Hadamards commute, so hb is any order of their bits; here
// descending, as in a QFT segment).
// Hadamards only, on two or more distinct local bits (a Walsh-Hadamard
// segment: the Hadamards commute, so hb is any order of their bits; here
// descending, as in a QFT segment).
bool walsh_segment(const FusedPass &pass, std::vector<unsigned> &hb) {
	hb.clear();
	uint64_t seen = 0;
	for(const FusedOp &f : pass.ops) {
		if(f.kind != kFH || f.lt >= pass.K) return false;
		const unsigned b = pass.lpos[f.lt];
		if((seen >> b) & 1ull) return false;
		seen |= 1ull << b;
		hb.push_back(b);
	}
	std::sort(hb.begin(), hb.end(), [](unsigned x, unsigned y) { return x > y; });
	return hb.size() >= 2;
}

inline unsigned insert_zeros(unsigned t, const uint32_t *sorted, int count) {
	for(int i = 0; i < count; ++i) {
		const unsigned b = sorted[i], lo = t & ((1u << b) - 1u);
		t = ((t ^ lo) << 1) | lo;
	}
	return t;
}

struct Swizzle {
	unsigned src[3] = {0, 0, 0}, dst[3] = {0, 0, 0};
	unsigned operator()(unsigned j) const {
		unsigned x = j;
		for(int k = 0; k < 3; ++k)
			if(src[k]) x ^= ((j >> src[k]) & 1u) << dst[k];
		return x;
	}
};

// Plans the pass for storage values of vbytes bytes and RB register bits.
bool plan_qft(const FusedPass &pass, const std::vector<unsigned> &hb, unsigned r0, unsigned vbytes, unsigned RB,
              QftGeom &g, bool walsh, bool allow_tma = false) {
	const unsigned K = pass.K, n = pass.n, per16 = 16 / vbytes;
	const unsigned lgran = RB - (per16 == 2 ? 1u : 0u);  // log2 of the granules per thread
	if(K > 14 || K < RB + 5 || (1u << (K - RB)) > qft_max_threads(vbytes, (int)RB)) return false;
	// The granule index bits (the top lgran local bits) are contiguous.
	if(pass.lpos[K - 1] - pass.lpos[K - lgran] != lgran - 1) return false;
	if(per16 == 2 && pass.lpos[0] != 0) return false;  // two adjacent amplitudes per granule
	auto li = [&](unsigned bit) -> int {
		for(unsigned i = 0; i < K; ++i)
			if(pass.lpos[i] == bit) return (int)i;
		return -1;
	};
	const unsigned np = (unsigned)hb.size(), nst = (np + RB - 1) / RB;
	if(nst > kQftMaxStages) return false;
	g = QftGeom{};
	g.K = K;
	g.nstages = nst;
	g.ntiles = 1ull << (n - K);
	g.istride = 1ull << pass.lpos[K - lgran];
	for(unsigned i = 0; i < K; ++i) {
		g.lpos[i] = pass.lpos[i];
		g.localmask |= 1ull << pass.lpos[i];
	}
	fill_roots(g.roots);
	auto range_mask = [](unsigned lo, unsigned hi) -> uint64_t {
		if(hi <= lo) return 0ull;
		const uint64_t top = hi >= 64 ? ~0ull : ((1ull << hi) - 1ull);
		return top & ~((1ull << lo) - 1ull);
	};

	// Stages: register bits 0..d-1 are the stage's Hadamard bits in circuit
	// order; the rest are filler bits outside the twiddle range (above the
	// stage, or below r0).
	uint32_t rbit[kQftMaxStages][5] = {};
	unsigned nfrows = 0, ocol = 0;
	for(unsigned s = 0; s < nst; ++s) {
		QftStage &S = g.st[s];
		const unsigned first = s * RB;
		S.d = std::min(RB, np - first);
		const unsigned hi = hb[first], lo = hb[first + S.d - 1];
		S.bhi = hi;
		S.wmask = range_mask(r0, lo);
		uint32_t used = 0;
		for(unsigned i = 0; i < S.d; ++i) {
			const int l = li(hb[first + i]);
			if(l < 0) return false;
			rbit[s][i] = (uint32_t)l;
			used |= 1u << l;
		}
		unsigned cnt = S.d;
		for(int l = (int)K - 1; l >= 0 && cnt < RB; --l)
			if(!((used >> l) & 1u) && pass.lpos[l] > hi) {
				rbit[s][cnt++] = (uint32_t)l;
				used |= 1u << l;
			}
		for(unsigned l = 0; l < K && cnt < RB; ++l)
			if(!((used >> l) & 1u) && pass.lpos[l] < r0) {
				rbit[s][cnt++] = l;
				used |= 1u << l;
			}
		if(cnt < RB) return false;
		std::vector<uint32_t> srt(rbit[s], rbit[s] + RB);
		std::sort(srt.begin(), srt.end());
		for(unsigned i = 0; i < RB; ++i) S.rsorted[i] = srt[i];
		S.fl = kQftNone;
		S.ot = kQftNone;
		if(S.wmask) {
			S.fl = nfrows;
			nfrows += S.d;
			if(S.wmask & ~g.localmask) {
				S.ot = ocol;
				ocol += S.d;
			}
		}
		S.scaled = s + 1 == nst;
		S.walsh = walsh;
		for(unsigned i = 0; i < RB; ++i) S.gstride[i] = 1ull << pass.lpos[rbit[s][i]];
		// Direct stores from the last stage when its lanes start with the lowest
		// contiguous index bits: rows of at least 64 bytes per warp store.
		if(S.scaled) {
			const unsigned need = vbytes == 8 ? 3u : 2u;
			bool ok = true;
			for(unsigned l = 0; l < need; ++l)
				if(l >= K || pass.lpos[l] != l || ((used >> l) & 1u)) ok = false;
			S.direct = ok;
		}
	}
	g.nfrows = nfrows;
	g.ot_stride = ocol;

	// The last stage goes into the copy-out when it holds at most 3 Hadamards
	// on the tile's lowest bits, the whole tile is contiguous in the state and
	// no twiddle follows it.
	{
		QftStage &L = g.st[nst - 1];
		bool contiguous = true;
		for(unsigned l = 0; l < K; ++l)
			if(pass.lpos[l] != l) contiguous = false;
		if(nst >= 2 && L.d <= 3 && L.wmask == 0 && L.bhi == L.d - 1 && contiguous) {
			L.tail = 1;
			L.direct = 0;
		}
	}

	// Swizzle: shared index bits dst ^= local bits src, the sources among the
	// thread bits of the copies (so a thread's granules stay at fixed offsets),
	// chosen so that each stage's half-warps (quarter-warps for 16-byte
	// amplitudes) hit as few banks twice as the layout allows.
	const unsigned bank_mask = per16 == 2 ? 15u : 7u, group = per16 == 2 ? 16u : 8u;
	// The copies' thread bits are shared index bits [log2(per16), log2(per16) + K - RB).
	const unsigned dst0 = per16 == 2 ? 1u : 0u, src_lo = per16 == 2 ? 4u : 3u;
	const unsigned src_hi = (per16 == 2 ? 1u : 0u) + (K - RB) - 1u;
	const bool tail = g.st[nst - 1].tail != 0;
	auto cost = [&](const Swizzle &w) {
		unsigned total = 0;
		for(unsigned s = 0; s < nst; ++s) {
			unsigned count[16] = {0}, worst = 0;
			if(tail && s + 1 == nst) {
				// The fused tail: lane q reads the 16-byte granule at q * 2^d
				// (a quarter-warp per wavefront).
				for(unsigned lane = 0; lane < 8; ++lane) {
					const unsigned b = (w(lane << g.st[s].d) >> (per16 == 2 ? 1u : 0u)) & 7u;
					worst = std::max(worst, ++count[b]);
				}
			} else {
				for(unsigned lane = 0; lane < group; ++lane) {
					const unsigned b = w(insert_zeros(lane, g.st[s].rsorted, (int)RB)) & bank_mask;
					worst = std::max(worst, ++count[b]);
				}
			}
			total += worst;
		}
		return total;
	};
	std::vector<unsigned> cand{0};
	for(unsigned b = src_lo; b <= src_hi; ++b) cand.push_back(b);
	Swizzle best;
	for(int k = 0; k < 3; ++k) best.dst[k] = dst0 + k;
	unsigned best_cost = cost(best), best_used = 0;
	// A cost of one wavefront group per stage is the floor: no search needed.
	if(best_cost > nst) {
		for(unsigned x : cand)
			for(unsigned y : cand)
				for(unsigned z : cand) {
					Swizzle w = best;
					w.src[0] = x;
					w.src[1] = y;
					w.src[2] = z;
					const unsigned used = (x != 0) + (y != 0) + (z != 0);
					const unsigned cc = cost(w);
					if(cc < best_cost || (cc == best_cost && used < best_used)) {
						best = w;
						best_cost = cc;
						best_used = used;
					}
				}
	}
	// Tensor-map tiles (complex64, when asked): the 128-byte swizzle the copy
	// applies is shared index bits 1-3 ^= bits 4-6, so it is taken when it
	// costs the stages no more bank conflicts than the searched swizzle.
	// In 8-byte tensor elements: complex64 rows are 16 amplitudes (index bits
	// 0-3, swizzle bits 1-3 ^= 4-6), complex128 rows 8 amplitudes (bits 0-2,
	// swizzle bits 0-2 ^= 3-5, each amplitude two elements).
	g.tma = 0;
	const unsigned rowbits = vbytes == 8 ? 4u : 3u, epa = vbytes / 8;
	if(allow_tma && (vbytes == 8 || vbytes == 16) && K >= rowbits && src_hi >= dst0 + 5) {
		Swizzle t;
		for(int k = 0; k < 3; ++k) {
			t.src[k] = rowbits + (unsigned)k;
			t.dst[k] = dst0 + (unsigned)k;
		}
		bool fits = cost(t) <= best_cost;
		for(unsigned l = 0; l < rowbits && fits; ++l)
			if(pass.lpos[l] != l) fits = false;  // the innermost run: one 128-byte row at least
		unsigned dims = 0, oshift = 0;
		for(unsigned b = 0; b < n && fits;) {
			const bool local = (g.localmask >> b) & 1ull;
			unsigned e = b;
			while(e < n && (((g.localmask >> e) & 1ull) != 0) == local) ++e;
			for(unsigned p0 = b; p0 < e && fits;) {
				// Local runs in pieces: the row, then up to 8 bits; an outer run whole.
				const unsigned len = !local ? e - p0 : (p0 == 0 ? rowbits : std::min(8u, e - p0));
				if(dims == 5 || len > 31 || ((1ull << p0) * vbytes) >= (1ull << 40)) {
					fits = false;
					break;
				}
				const unsigned mult = p0 == 0 ? epa : 1u;  // dimension 0 also spans an amplitude's elements
				g.tma_outer[dims] = local ? 0u : 1u;
				g.tma_shift[dims] = local ? 0u : oshift;
				g.tma_len[dims] = len;
				g.tma_size[dims] = (1ull << len) * mult;
				g.tma_stride[dims] = (1ull << p0) * vbytes;
				g.tma_box[dims] = local ? (1u << len) * mult : 1u;
				if(!local) oshift += len;
				++dims;
				p0 += len;
			}
			b = e;
		}
		if(fits) {
			g.tma = 1;
			g.tma_dims = dims;
			best = t;
		}
	}
	for(int k = 0; k < 3; ++k) {
		g.sw_src[k] = best.src[k];
		g.sw_dst[k] = best.dst[k];
	}
	for(unsigned s = 0; s < nst; ++s) {
		bool top = K == (unsigned)qft_tile_bits(vbytes);
		for(unsigned i = 0; i < RB; ++i) {
			g.st[s].roff[i] = best(1u << rbit[s][i]);
			if(rbit[s][i] != K - 1 - i || g.st[s].roff[i] != (1u << rbit[s][i])) top = false;
		}
		g.st[s].top = top;
	}

	// Runs of outer bits, ascending.
	g.nruns = 0;
	for(unsigned b = 0; b < n;) {
		if((g.localmask >> b) & 1ull) {
			++b;
			continue;
		}
		unsigned e = b;
		while(e < n && !((g.localmask >> e) & 1ull)) ++e;
		if(g.nruns == kQftMaxRuns) return false;
		g.run_pos[g.nruns] = b;
		g.run_len[g.nruns] = e - b;
		++g.nruns;
		b = e;
	}
	g.scale = std::ldexp((np & 1u) ? 1.0 / std::sqrt(2.0) : 1.0, -(int)(np / 2));
	return true;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the runtime only).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn tile_map_encoder() {
	static EncodeTiledFn fn = [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
		   q != cudaDriverEntryPointSuccess) {
			cudaGetLastError();
			return (EncodeTiledFn) nullptr;
		}
		return reinterpret_cast<EncodeTiledFn>(p);
	}();
	return fn;
}

// The state (8-byte amplitudes) as the pass's tensor, 128-byte swizzle.
bool encode_tile_map(CUtensorMap &m, void *a, const QftGeom &g) {
	const EncodeTiledFn enc = tile_map_encoder();
	if(!enc) return false;
	cuuint64_t size[5], stride[4];
	cuuint32_t box[5], estr[5];
	for(unsigned i = 0; i < g.tma_dims; ++i) {
		size[i] = g.tma_size[i];
		box[i] = g.tma_box[i];
		estr[i] = 1;
		if(i) stride[i - 1] = g.tma_stride[i];
	}
	return enc(&m, CU_TENSOR_MAP_DATA_TYPE_UINT64, g.tma_dims, a, size, stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
	           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
	       CUDA_SUCCESS;
}

#ifndef TMFQS_QFT_PLAN_ONLY  // (host checks of the planner compile without the kernels)
template <typename R, int RB>
bool run_qft(const LaunchCtx &c, void *a, const FusedPass &pass, const std::vector<unsigned> &hb, unsigned r0,
             bool walsh) {
	typedef typename Vec2<R>::type V;
	QftGeom g;
	if(!c.err || !plan_qft(pass, hb, r0, (unsigned)sizeof(V), (unsigned)RB, g, walsh, sizeof(V) == 8)) return false;
	const unsigned nthr = 1u << (g.K - RB);
	const size_t T = size_t(1) << g.K;
	auto smem_for = [&](unsigned slots) {
		return (slots * T + (size_t)g.nfrows * nthr + (size_t)slots * g.ot_stride) * sizeof(V) +
		       kQftMaxStages * sizeof(QftStage) + slots * 8 + (size_t)g.nstages * nthr * 2 + (g.tma ? 1024 : 0);
	};
	int dev = 0, max_optin = 0;
	check_cuda(cudaGetDevice(&dev), "qft device");
	check_cuda(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "qft smem limit");
	g.slots = smem_for(3) <= (size_t)max_optin ? 3u : 2u;
	const size_t smem = smem_for(g.slots);
	if(smem > (size_t)max_optin) return false;
	CUtensorMap tmap;
	std::memset(&tmap, 0, sizeof(tmap));
	if(g.tma && !encode_tile_map(tmap, a, g)) g.tma = 0;  // no encoder: per-thread copies (same swizzle)
	void (*kern)(V *, const QftGeom, const CUtensorMap, int *) = k_qft_pass<R, RB, false>;
	if constexpr(sizeof(V) == 8) {  // tensor-map tiles: complex64 only
		if(g.tma) kern = k_qft_pass<R, RB, true>;
	}
	check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "qft smem");
	const uint64_t grid = std::min<uint64_t>(g.ntiles, (uint64_t)c.num_sms);
	kern<<<(unsigned)grid, nthr, smem, c.stream>>>(static_cast<V *>(a), g, tmap, c.err);
	check_cuda(cudaGetLastError(), "qft pass");
	if(c.launches) ++*c.launches;
	return true;
}

// One precision's launcher (recognition, plan, launch).
template <typename R, int RB>
bool launch_qft_pass_for(const LaunchCtx &c, void *a, const FusedPass &pass, bool allow_walsh) {
	std::vector<unsigned> hb;
	unsigned r0 = 0;
	bool walsh = false;
	if(!qft_segment(pass, hb, r0)) {
		if(!allow_walsh || !walsh_segment(pass, hb)) return false;
		walsh = true;
		r0 = pass.n;  // no phases: no twiddle range
	}
	return run_qft<R, RB>(c, a, pass, hb, r0, walsh);
}
#endif

}  // namespace

// The kernels of each precision are compiled in their own unit
// (qft_pass_c64.cu, qft_pass_c128.cu, which include this file), so that the
// two build in parallel; this unit holds the dispatch.
#ifndef TMFQS_QFT_PLAN_ONLY
#if defined(TMFQS_QFT_UNIT_C64)
// complex64: 5-bit stages (256 threads).  4-bit stages with 512 threads
// measured the same at 28 and 30 qubits and 2% slower at 26 with one barrier
// per tile.
bool launch_qft_pass_c64(const LaunchCtx &c, void *a, const FusedPass &pass, bool allow_walsh) {
	return launch_qft_pass_for<float, 5>(c, a, pass, allow_walsh);
}
#elif defined(TMFQS_QFT_UNIT_C128)
bool launch_qft_pass_c128(const LaunchCtx &c, void *a, const FusedPass &pass, bool allow_walsh) {
	return launch_qft_pass_for<double, 4>(c, a, pass, allow_walsh);
}
#else
bool launch_qft_pass_c64(const LaunchCtx &c, void *a, const FusedPass &pass, bool allow_walsh);
bool launch_qft_pass_c128(const LaunchCtx &c, void *a, const FusedPass &pass, bool allow_walsh);
bool launch_qft_pass(const LaunchCtx &c, int prec, void *a, const FusedPass &pass, bool allow_walsh) {
	return prec == TMFQS_FP64 ? launch_qft_pass_c128(c, a, pass, allow_walsh) : launch_qft_pass_c64(c, a, pass, allow_walsh);
}
#endif
#endif

}  // namespace tqb
