// Exact replay of the reference's sequential double sums on the GPU.
//
// Reductions replaced (all left-to-right loops in the reference):
//   totalProbability      dense_state_backend.cpp:161-171  (terms |a|^2)
//   sampleMeasurement     dense_state_backend.cpp:173-188  (first s with rnd <= running sum)
//   logicalAmplitudeSum   quantum_register.cpp:176-190     (terms re, im; signed)
//   overlay branches      quantum_register.cpp:269-310     (terms of scale*a+bias)
//
// Pipeline (tile = 1024 terms, group = 32 tiles); math in seqsum_core.h:
//   A  k_seq_a       per tile: double-double sum, sum of |term|, prefix min/max
//   S1 k_seq_groups  per group: warp scan of tile sums -> in-group prefixes
//   S2 k_seq_top     one CTA: scan of group sums -> group prefixes
//   B  k_seq_b       per tile: classify (does C provably stay in one binade?)
//                    and, for clean tiles, the parity-indexed grid increment
//   G  k_seq_groupb  per group: compose clean tiles of one binade
//   W  k_seq_walk    one warp: walk groups/tiles carrying the exact running
//                    sum; replay dirty tiles 32 terms per step.
// Passes A and B each read the state once; everything else touches only the
// small per-tile tables.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "device_common.cuh"
#include "internal.h"
#include "seqsum_core.h"

namespace tqb {

namespace {

constexpr unsigned kTile = 1024;       // terms per tile (32 per lane)
constexpr unsigned kGroup = 32;        // tiles per group
constexpr unsigned kWarpsA = 4;        // warps per CTA in passes A and B
constexpr unsigned kStage = 32 * 33;   // staged terms per warp (padded rows)
constexpr unsigned FULL = 0xffffffffu;

struct TileA {
	double s_hi, s_lo, a, mn, mx;
};
struct TilePre {
	double e_hi, e_lo, a_incl;
};
struct GroupA {
	double s_hi, s_lo, a;
};
struct GroupPre {
	double e_hi, e_lo, a_excl;
};
struct TileB {
	int32_t e;
	int32_t pad;
	long long i0, i1;
};
struct WalkOut {
	unsigned long long index;
	double value;
	int32_t error;
	int32_t pad;
};

template <typename R, int KIND>
struct TermF {
	const typename Vec2<R>::type *a;
	uint64_t N;
	int ov;
	double sr, si, br, bi;
	__device__ __forceinline__ double operator()(uint64_t j) const {
		if(j >= N) return 0.0;
		const auto v = a[j];
		double re = (double)v.x, im = (double)v.y;
		if(ov) {
			// applyAffineOverlay, quantum_register.cpp:160-165.
			const double mr = rsub(rmul(sr, re), rmul(si, im));
			const double mi = radd(rmul(sr, im), rmul(si, re));
			re = radd(mr, br);
			im = radd(mi, bi);
		}
		if(KIND == kTermProb) return radd(rmul(re, re), rmul(im, im));
		return KIND == kTermReal ? re : im;
	}
};

// Squared distance of two states at j, as experiment::compareStates forms it
// (comparison.cpp:29-38): the candidate minus the reference, per component,
// in double.
template <typename RA, typename RB>
struct TermDiff {
	const typename Vec2<RA>::type *ref;
	const typename Vec2<RB>::type *got;
	uint64_t N;
	__device__ __forceinline__ double operator()(uint64_t j) const {
		if(j >= N) return 0.0;
		const auto r = ref[j];
		const auto g = got[j];
		const double dr = rsub((double)g.x, (double)r.x), di = rsub((double)g.y, (double)r.y);
		return radd(rmul(dr, dr), rmul(di, di));
	}
};

__device__ __forceinline__ tq::DD shfl_dd(tq::DD v, int src) {
	return tq::DD{__shfl_sync(FULL, v.hi, src), __shfl_sync(FULL, v.lo, src)};
}
__device__ __forceinline__ tq::DD shfl_up_dd(tq::DD v, unsigned d) {
	return tq::DD{__shfl_up_sync(FULL, v.hi, d), __shfl_up_sync(FULL, v.lo, d)};
}
__device__ __forceinline__ tq::DD shfl_down_dd(tq::DD v, unsigned d) {
	return tq::DD{__shfl_down_sync(FULL, v.hi, d), __shfl_down_sync(FULL, v.lo, d)};
}
__device__ __forceinline__ tq::Inc shfl_inc(tq::Inc v, int src) {
	return tq::Inc{__shfl_sync(FULL, v.i0, src), __shfl_sync(FULL, v.i1, src)};
}
__device__ __forceinline__ tq::Inc shfl_up_inc(tq::Inc v, unsigned d) {
	return tq::Inc{__shfl_up_sync(FULL, v.i0, d), __shfl_up_sync(FULL, v.i1, d)};
}
__device__ __forceinline__ tq::Inc shfl_down_inc(tq::Inc v, unsigned d) {
	return tq::Inc{__shfl_down_sync(FULL, v.i0, d), __shfl_down_sync(FULL, v.i1, d)};
}

// Ordered warp reduction of increments: lane 0 gets lane0 o lane1 o ... o lane31.
__device__ __forceinline__ tq::Inc warp_compose(tq::Inc v) {
	const unsigned lane = threadIdx.x & 31u;
	for(unsigned off = 1; off < 32; off <<= 1) {
		const tq::Inc o = shfl_down_inc(v, off);
		if((lane & (2 * off - 1)) == 0 && lane + off < 32) v = tq::compose(v, o);
	}
	return v;
}

// Inclusive ordered scan of increments over lanes.
__device__ __forceinline__ tq::Inc warp_scan_inc(tq::Inc v) {
	const unsigned lane = threadIdx.x & 31u;
	for(unsigned d = 1; d < 32; d <<= 1) {
		const tq::Inc o = shfl_up_inc(v, d);
		if(lane >= d) v = tq::compose(o, v);
	}
	return v;
}

// Stage one tile's terms in shared memory: term (q*32 + lane) loaded
// coalesced; lane later owns the contiguous run [lane*32, lane*32+32).
template <class F>
__device__ __forceinline__ void stage_tile(const F &term, uint64_t base, double *st) {
	const unsigned lane = threadIdx.x & 31u;
#pragma unroll 8
	for(unsigned q = 0; q < 32; ++q) st[q * 33 + lane] = term(base + q * 32 + lane);
	__syncwarp();
}

// ---- pass A ---------------------------------------------------------------
template <class F, bool SIGNED>
__global__ void __launch_bounds__(kWarpsA * 32) k_seq_a(F term, uint64_t ntiles, TileA *ta) {
	__shared__ double stage[kWarpsA][kStage];
	const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
	double *st = stage[warp];
	for(uint64_t t = (uint64_t)blockIdx.x * kWarpsA + warp; t < ntiles; t += (uint64_t)gridDim.x * kWarpsA) {
		stage_tile(term, t * kTile, st);
		tq::DD s{0.0, 0.0};
		double A = 0.0, pre = 0.0, mn = 0.0, mx = 0.0;
#pragma unroll 8
		for(unsigned q = 0; q < 32; ++q) {
			const double p = st[lane * 33 + q];
			s = tq::dd_add_d(s, p);
			if(SIGNED) {
				A += fabs(p);
				pre += p;
				mn = fmin(mn, pre);
				mx = fmax(mx, pre);
			}
		}
		__syncwarp();
		if(SIGNED) {
			// Offset each lane's local prefix extremes by the preceding lanes' sums.
			double inc = pre;
			for(unsigned d = 1; d < 32; d <<= 1) {
				const double o = __shfl_up_sync(FULL, inc, d);
				if(lane >= d) inc += o;
			}
			const double off = inc - pre;
			mn = off + mn;
			mx = off + mx;
			for(unsigned d = 16; d > 0; d >>= 1) {
				mn = fmin(mn, __shfl_down_sync(FULL, mn, d));
				mx = fmax(mx, __shfl_down_sync(FULL, mx, d));
				A += __shfl_down_sync(FULL, A, d);
			}
		}
		for(unsigned d = 16; d > 0; d >>= 1) s = tq::dd_add(s, shfl_down_dd(s, d));
		if(lane == 0) {
			const double tot = s.hi + s.lo;
			ta[t] = TileA{s.hi, s.lo, SIGNED ? A : fabs(tot), SIGNED ? fmin(mn, 0.0) : 0.0, SIGNED ? fmax(mx, 0.0) : tot};
		}
	}
}

// ---- scan 1: in-group prefixes ---------------------------------------------
__global__ void k_seq_groups(const TileA *ta, uint64_t ntiles, uint64_t ngroups, TilePre *tp, GroupA *ga) {
	const unsigned lane = threadIdx.x & 31u;
	const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
	for(uint64_t g = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < ngroups; g += warps) {
		const uint64_t t = g * kGroup + lane;
		tq::DD s{0.0, 0.0};
		double A = 0.0;
		if(t < ntiles) {
			s = tq::DD{ta[t].s_hi, ta[t].s_lo};
			A = ta[t].a;
		}
		tq::DD inc = s;
		double ainc = A;
		for(unsigned d = 1; d < 32; d <<= 1) {
			const tq::DD o = shfl_up_dd(inc, d);
			const double ao = __shfl_up_sync(FULL, ainc, d);
			if(lane >= d) {
				inc = tq::dd_add(o, inc);
				ainc += ao;
			}
		}
		tq::DD ex = shfl_up_dd(inc, 1);
		if(lane == 0) ex = tq::DD{0.0, 0.0};
		if(t < ntiles) tp[t] = TilePre{ex.hi, ex.lo, ainc};
		if(lane == 31) ga[g] = GroupA{inc.hi, inc.lo, ainc};
	}
}

// ---- scan 2: group prefixes (one CTA) ---------------------------------------
__global__ void __launch_bounds__(1024) k_seq_top(const GroupA *ga, uint64_t ngroups, GroupPre *gp) {
	__shared__ double sh_hi[1024], sh_lo[1024], sh_a[1024];
	const unsigned tid = threadIdx.x;
	const uint64_t per = (ngroups + 1023) / 1024;
	const uint64_t g0 = (uint64_t)tid * per, g1 = std::min<uint64_t>(ngroups, g0 + per);
	tq::DD s{0.0, 0.0};
	double A = 0.0;
	for(uint64_t g = g0; g < g1; ++g) {
		s = tq::dd_add(s, tq::DD{ga[g].s_hi, ga[g].s_lo});
		A += ga[g].a;
	}
	sh_hi[tid] = s.hi;
	sh_lo[tid] = s.lo;
	sh_a[tid] = A;
	__syncthreads();
	for(unsigned d = 1; d < 1024; d <<= 1) {
		tq::DD o{0.0, 0.0};
		double ao = 0.0;
		if(tid >= d) {
			o = tq::DD{sh_hi[tid - d], sh_lo[tid - d]};
			ao = sh_a[tid - d];
		}
		__syncthreads();
		if(tid >= d) {
			const tq::DD c = tq::dd_add(o, tq::DD{sh_hi[tid], sh_lo[tid]});
			sh_hi[tid] = c.hi;
			sh_lo[tid] = c.lo;
			sh_a[tid] += ao;
		}
		__syncthreads();
	}
	tq::DD run = tid ? tq::DD{sh_hi[tid - 1], sh_lo[tid - 1]} : tq::DD{0.0, 0.0};
	double arun = tid ? sh_a[tid - 1] : 0.0;
	for(uint64_t g = g0; g < g1; ++g) {
		gp[g] = GroupPre{run.hi, run.lo, arun};
		run = tq::dd_add(run, tq::DD{ga[g].s_hi, ga[g].s_lo});
		arun += ga[g].a;
	}
}

// ---- pass B ---------------------------------------------------------------
template <class F, bool SIGNED>
__global__ void __launch_bounds__(kWarpsA * 32) k_seq_b(F term, uint64_t N, uint64_t ntiles, const TileA *ta,
                                                        const TilePre *tp, const GroupPre *gp, TileB *tb) {
	__shared__ double stage[kWarpsA][kStage];
	const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
	double *st = stage[warp];
	for(uint64_t t = (uint64_t)blockIdx.x * kWarpsA + warp; t < ntiles; t += (uint64_t)gridDim.x * kWarpsA) {
		const TileA a = ta[t];
		const TilePre p = tp[t];
		const GroupPre g = gp[t / kGroup];
		int e;
		if(a.a == 0.0) {
			e = tq::kIdentity;
		} else {
			const tq::DD E = tq::dd_add(tq::DD{g.e_hi, g.e_lo}, tq::DD{p.e_hi, p.e_lo});
			const double Ed = E.hi + E.lo;
			const double Aend = g.a_excl + p.a_incl;
			const double endIdx = (double)std::min<uint64_t>(N, (t + 1) * kTile);
			const double margin = tq::gamma_bound(endIdx) * Aend * 1.0001 + tq::gamma_bound(kTile) * a.a * 2.0 +
			                      fabs(Ed) * 1e-15 + 1e-300;
			const double lo = Ed + a.mn - margin;
			const double hi = Ed + a.mx + margin;
			e = tq::common_binade(lo, hi);
		}
		if(e == tq::kDirty || e == tq::kIdentity) {
			if(lane == 0) tb[t] = TileB{e, 0, 0, 0};
			continue;
		}
		const double scale = tq::grid_scale(e);
		stage_tile(term, t * kTile, st);
		tq::Inc acc = tq::inc_identity();
#pragma unroll 8
		for(unsigned q = 0; q < 32; ++q) acc = tq::compose(acc, tq::term_inc(st[lane * 33 + q], scale));
		__syncwarp();
		acc = warp_compose(acc);
		if(lane == 0) tb[t] = TileB{e, 0, acc.i0, acc.i1};
	}
}

// ---- group composition ------------------------------------------------------
__global__ void k_seq_groupb(const TileB *tb, uint64_t ntiles, uint64_t ngroups, TileB *gb) {
	const unsigned lane = threadIdx.x & 31u;
	const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
	for(uint64_t g = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < ngroups; g += warps) {
		const uint64_t t = g * kGroup + lane;
		TileB b{tq::kIdentity, 0, 0, 0};
		if(t < ntiles) b = tb[t];
		const unsigned ni = __ballot_sync(FULL, b.e != tq::kIdentity);
		int e0 = tq::kIdentity;
		if(ni) e0 = __shfl_sync(FULL, b.e, __ffs(ni) - 1);
		const bool ok = b.e == tq::kIdentity || (b.e == e0 && e0 != tq::kDirty);
		const bool mixed = __ballot_sync(FULL, !ok) != 0;
		tq::Inc v = b.e == tq::kIdentity ? tq::inc_identity() : tq::Inc{b.i0, b.i1};
		v = warp_compose(v);
		if(lane == 0) gb[g] = mixed ? TileB{tq::kDirty, 0, 0, 0} : TileB{e0, 0, v.i0, v.i1};
	}
}

// ---- walk -------------------------------------------------------------------
struct WalkState {
	double C;
	uint64_t answer;
	bool done;
	int err;
};

// Replays terms [a, b) exactly, 32 per step (see seqsum_core.h).
template <class F, bool STOP>
__device__ void replay_range(const F &term, uint64_t a, uint64_t b, double rnd, WalkState &st, double *stage) {
	const unsigned lane = threadIdx.x & 31u;
	// Stage up to one tile of terms (the range never exceeds a tile).
	const unsigned len = (unsigned)(b - a);
	for(unsigned q = 0; q < (len + 31) / 32; ++q) {
		const unsigned i = q * 32 + lane;
		stage[i] = i < len ? term(a + i) : 0.0;
	}
	__syncwarp();
	uint64_t j = a;
	double C = st.C;
	while(j < b) {
		const unsigned cnt = (unsigned)std::min<uint64_t>(32, b - j);
		const double p = lane < cnt ? stage[(j - a) + lane] : 0.0;
		if(C == 0.0) {
			if(STOP && rnd <= 0.0) {
				st.C = radd(C, __shfl_sync(FULL, p, 0));
				st.answer = j;
				st.done = true;
				return;
			}
			const unsigned nz = __ballot_sync(FULL, lane < cnt && p != 0.0);
			if(nz == 0) {
				j += cnt;
				continue;
			}
			const unsigned f = __ffs(nz) - 1;
			C = radd(C, __shfl_sync(FULL, p, f));
			if(STOP && rnd <= C) {
				st.C = C;
				st.answer = j + f;
				st.done = true;
				return;
			}
			j += f + 1;
			continue;
		}
		const int e = tq::tq_ilogb(fabs(C));
		if(e < -1000 || e > 1000) {
			for(unsigned l = 0; l < cnt; ++l) {
				C = radd(C, __shfl_sync(FULL, p, l));
				if(STOP && rnd <= C) {
					st.C = C;
					st.answer = j + l;
					st.done = true;
					return;
				}
			}
			j += cnt;
			continue;
		}
		const double scale = tq::grid_scale(e);
		const double inv = tq::tq_ldexp(1.0, e - 52);
		const long long c0 = (long long)(C * scale);
		tq::Inc v = lane < cnt ? tq::term_inc(p, scale) : tq::inc_identity();
		v = warp_scan_inc(v);
		const long long cl = c0 + tq::apply(v, c0);
		const bool valid = lane < cnt && tq::grid_interior(cl);
		const unsigned cntmask = cnt == 32 ? FULL : ((1u << cnt) - 1u);
		const unsigned inval = ~__ballot_sync(FULL, valid) & cntmask;
		const unsigned k = inval ? (unsigned)(__ffs(inval) - 1) : cnt;
		const double Cl = (double)cl * inv;
		if(STOP) {
			const unsigned hit = __ballot_sync(FULL, lane < k && rnd <= Cl);
			if(hit) {
				const unsigned f = __ffs(hit) - 1;
				st.C = __shfl_sync(FULL, Cl, f);
				st.answer = j + f;
				st.done = true;
				return;
			}
		}
		const double Ck = __shfl_sync(FULL, Cl, k == 0 ? 0 : k - 1);
		if(k > 0) C = Ck;
		j += k;
		if(k < cnt) {
			C = radd(C, __shfl_sync(FULL, p, k));
			if(STOP && rnd <= C) {
				st.C = C;
				st.answer = j;
				st.done = true;
				return;
			}
			j += 1;
		}
	}
	st.C = C;
	__syncwarp();
}

// Walks 32 entries (tiles of a group, or groups) carrying st.C.  `dive`
// handles entry i when it is dirty or holds the stopping point.
template <bool STOP, class Dive>
__device__ void walk_entries(const TileB *entries, uint64_t first, unsigned cnt, double rnd, WalkState &st,
                             Dive dive) {
	const unsigned lane = threadIdx.x & 31u;
	TileB info{tq::kIdentity, 0, 0, 0};
	if(lane < cnt) info = entries[first + lane];
	unsigned l = 0;
	while(l < cnt && !st.done && !st.err) {
		const int el = __shfl_sync(FULL, info.e, l);
		if(el == tq::kDirty) {
			dive(first + l, st);
			++l;
			continue;
		}
		const unsigned above = l == 0 ? FULL : (FULL << l);
		const unsigned ni = __ballot_sync(FULL, lane < cnt && info.e != tq::kIdentity) & above;
		const int erun = ni ? __shfl_sync(FULL, info.e, __ffs(ni) - 1) : tq::kIdentity;
		const bool inrun = lane >= l && lane < cnt &&
		                   (info.e == tq::kIdentity || (info.e == erun && erun != tq::kDirty));
		const unsigned runmask = __ballot_sync(FULL, inrun);
		const unsigned outside = ~runmask & above;
		const unsigned rend = outside ? (unsigned)(__ffs(outside) - 1) : 32u;
		const unsigned r = rend < cnt ? rend : cnt;
		if(erun == tq::kIdentity || erun == tq::kDirty) {
			// Only all-zero entries in [l, r): the running sum does not move.
			if(STOP && rnd <= st.C) {
				dive(first + l, st);
				return;
			}
			l = r;
			continue;
		}
		const double scale = tq::grid_scale(erun);
		const double inv = tq::tq_ldexp(1.0, erun - 52);
		const double cd = st.C * scale;
		const long long c0 = (long long)cd;
		const long long lo = 1ll << 52, hi = 1ll << 53;
		if((double)c0 != cd || !((c0 >= lo && c0 < hi) || (c0 <= -lo && c0 > -hi))) {
			st.err = 1;  // the rigorous binade bound was violated: report, never guess
			return;
		}
		tq::Inc v = tq::inc_identity();
		if(lane >= l && lane < r && info.e != tq::kIdentity) v = tq::Inc{info.i0, info.i1};
		v = warp_scan_inc(v);
		const double Cl = (double)(c0 + tq::apply(v, c0)) * inv;
		if(STOP) {
			const unsigned hit = __ballot_sync(FULL, lane >= l && lane < r && rnd <= Cl);
			if(hit) {
				const unsigned f = __ffs(hit) - 1;
				const double Cprev = __shfl_sync(FULL, Cl, f == 0 ? 0 : f - 1);
				if(f > l) st.C = Cprev;
				dive(first + f, st);
				if(!st.done) st.err = 2;  // the stop must lie inside entry f
				return;
			}
		}
		st.C = __shfl_sync(FULL, Cl, r - 1);
		l = r;
	}
}

template <class F, bool STOP>
__global__ void __launch_bounds__(32) k_seq_walk(F term, uint64_t N, uint64_t ntiles, uint64_t ngroups,
                                                 const TileB *tb, const TileB *gb, double rnd, WalkOut *out) {
	__shared__ double stage[kTile];
	WalkState st{0.0, N, false, 0};
	auto dive_tile = [&](uint64_t t, WalkState &s) {
		const uint64_t a = t * kTile, b = std::min<uint64_t>(N, a + kTile);
		if(a < b) replay_range<F, STOP>(term, a, b, rnd, s, stage);
	};
	auto dive_group = [&](uint64_t g, WalkState &s) {
		const uint64_t t0 = g * kGroup;
		const unsigned cnt = (unsigned)std::min<uint64_t>(kGroup, ntiles - t0);
		walk_entries<STOP>(tb, t0, cnt, rnd, s, dive_tile);
	};
	for(uint64_t g0 = 0; g0 < ngroups && !st.done && !st.err; g0 += 32) {
		const unsigned cnt = (unsigned)std::min<uint64_t>(32, ngroups - g0);
		walk_entries<STOP>(gb, g0, cnt, rnd, st, dive_group);
	}
	if((threadIdx.x & 31u) == 0) *out = WalkOut{st.done ? st.answer : N, st.C, st.err, 0};
}

template <class Term, bool SIGNED>
SeqResult run_engine_term(const Term &term, uint64_t N, bool stop, double rnd, SeqScratch &s, cudaStream_t stream,
                          int num_sms, uint64_t *launches) {
	const uint64_t ntiles = s.tiles, ngroups = s.groups;
	auto *ta = static_cast<TileA *>(s.tile_a);
	auto *tp = static_cast<TilePre *>(s.tile_pre);
	auto *tb = static_cast<TileB *>(s.tile_b);
	auto *ga = static_cast<GroupA *>(s.group_a);
	auto *gp = static_cast<GroupPre *>(s.group_pre);
	auto *gb = static_cast<TileB *>(s.group_b);
	auto *wo = static_cast<WalkOut *>(s.walk_out);
	const unsigned gridA = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((ntiles + kWarpsA - 1) / kWarpsA, (uint64_t)num_sms * 6));
	const unsigned gridG = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((ngroups + 7) / 8, (uint64_t)num_sms * 8));
	k_seq_a<Term, SIGNED><<<gridA, kWarpsA * 32, 0, stream>>>(term, ntiles, ta);
	k_seq_groups<<<gridG, 256, 0, stream>>>(ta, ntiles, ngroups, tp, ga);
	k_seq_top<<<1, 1024, 0, stream>>>(ga, ngroups, gp);
	k_seq_b<Term, SIGNED><<<gridA, kWarpsA * 32, 0, stream>>>(term, N, ntiles, ta, tp, gp, tb);
	k_seq_groupb<<<gridG, 256, 0, stream>>>(tb, ntiles, ngroups, gb);
	if(stop) k_seq_walk<Term, true><<<1, 32, 0, stream>>>(term, N, ntiles, ngroups, tb, gb, rnd, wo);
	else k_seq_walk<Term, false><<<1, 32, 0, stream>>>(term, N, ntiles, ngroups, tb, gb, rnd, wo);
	check_cuda(cudaGetLastError(), "exact reduction");
	if(launches) *launches += 6;
	check_cuda(cudaMemcpyAsync(s.host_out, wo, sizeof(WalkOut), cudaMemcpyDeviceToHost, stream), "reduction readback");
	check_cuda(cudaStreamSynchronize(stream), "reduction sync");
	const WalkOut r = *static_cast<WalkOut *>(s.host_out);
	if(r.error) fail(TMFQS_ERR_RUNTIME, "exact reduction invariant violated (code " + std::to_string(r.error) + ")");
	return SeqResult{r.index, r.value};
}

template <typename R, int KIND>
SeqResult run_engine(const void *amps, uint64_t N, const Overlay &ov, bool stop, double rnd, SeqScratch &s,
                     cudaStream_t stream, int num_sms, uint64_t *launches) {
	TermF<R, KIND> term{static_cast<const typename Vec2<R>::type *>(amps), N, ov.active ? 1 : 0, ov.sre, ov.sim, ov.bre, ov.bim};
	return run_engine_term<TermF<R, KIND>, KIND != kTermProb>(term, N, stop, rnd, s, stream, num_sms, launches);
}

void ensure_scratch(SeqScratch &s, uint64_t N) {
	const uint64_t tiles = (N + kTile - 1) / kTile;
	const uint64_t groups = (tiles + kGroup - 1) / kGroup;
	if(s.base && s.tiles == tiles) return;
	seq_scratch_free(s);
	auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
	const size_t b_ta = align(tiles * sizeof(TileA)), b_tp = align(tiles * sizeof(TilePre)),
	             b_tb = align(tiles * sizeof(TileB)), b_ga = align(groups * sizeof(GroupA)),
	             b_gp = align(groups * sizeof(GroupPre)), b_gb = align(groups * sizeof(TileB)),
	             b_wo = align(sizeof(WalkOut));
	const size_t total = b_ta + b_tp + b_tb + b_ga + b_gp + b_gb + b_wo;
	void *base = nullptr;
	if(device_alloc(&base, total) != cudaSuccess) {
		cudaGetLastError();
		fail(TMFQS_ERR_NOMEM, "exact reduction scratch: device allocation of " + std::to_string(total) + " bytes failed");
	}
	void *host = nullptr;
	if(cudaMallocHost(&host, sizeof(WalkOut)) != cudaSuccess) {
		cudaGetLastError();
		cudaFree(base);
		fail(TMFQS_ERR_NOMEM, "exact reduction scratch: pinned allocation failed");
	}
	char *p = static_cast<char *>(base);
	s.base = base;
	s.bytes = total;
	s.tiles = tiles;
	s.groups = groups;
	s.tile_a = p;
	p += b_ta;
	s.tile_pre = p;
	p += b_tp;
	s.tile_b = p;
	p += b_tb;
	s.group_a = p;
	p += b_ga;
	s.group_pre = p;
	p += b_gp;
	s.group_b = p;
	p += b_gb;
	s.walk_out = p;
	s.host_out = host;
}

// ---------------------------------------------------------------------------
// Fixed device scratch for the allocation-free measurement entry point.
//
// Some callers cannot let this library call cudaMalloc: a host application
// whose caching allocator has already reserved nearly all device memory for
// itself (so a fresh allocation fails or fragments its pool), or a loop that
// must not pay the device-wide synchronisation cudaMalloc/cudaFree imply.
// For them tmfqs_sample_static runs the exact measurement replay with its
// per-tile tables in this fixed array, which every GPU that loads the library
// holds until the process exits.  Every region of it is fully written before
// it is read on each call, so no clearing is needed; calls that overlap on
// the GPU share the array and race.
// ---------------------------------------------------------------------------
constexpr unsigned kStaticMaxQubits = 24;
constexpr size_t kStaticScratchBytes = size_t(2) << 20;  // 2 MiB
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mutex;
void *g_static_addr[64] = {nullptr};  // device address of g_static_scratch, per device ordinal

// Host code cannot use &g_static_scratch as a device address; the runtime
// gives the real address for the current device.  It is looked up again on
// every call made outside stream capture: a context reset (cudaDeviceReset)
// reloads the module, and the array may then sit at another address.  While
// `stream` is capturing, the address of the last call outside capture on this
// device is used (no lookup, which could load the module inside a capture);
// a capturing call on a device that never had one fails.
void *static_scratch_address(cudaStream_t stream) {
	int dev = 0;
	check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
	if(dev < 0 || dev >= 64) fail(TMFQS_ERR_INVALID_ARGUMENT, "device ordinal out of range for the static scratch");
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	check_cuda(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
	std::lock_guard<std::mutex> lock(g_static_mutex);
	if(cap == cudaStreamCaptureStatusNone) {
		void *p = nullptr;
		check_cuda(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress(static scratch)");
		g_static_addr[dev] = p;
	} else if(!g_static_addr[dev]) {
		fail(TMFQS_ERR_LOGIC, "tmfqs_sample_static: the first call on a device must come before any stream capture");
	}
	return g_static_addr[dev];
}

// Carves the engine's tables out of the static array (same layout as
// ensure_scratch, without allocating).  Throws if they would not fit.
void carve_static(SeqScratch &s, uint64_t N, void *base, void *host_out) {
	const uint64_t tiles = (N + kTile - 1) / kTile;
	const uint64_t groups = (tiles + kGroup - 1) / kGroup;
	auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
	const size_t b_ta = align(tiles * sizeof(TileA)), b_tp = align(tiles * sizeof(TilePre)),
	             b_tb = align(tiles * sizeof(TileB)), b_ga = align(groups * sizeof(GroupA)),
	             b_gp = align(groups * sizeof(GroupPre)), b_gb = align(groups * sizeof(TileB)),
	             b_wo = align(sizeof(WalkOut));
	if(b_ta + b_tp + b_tb + b_ga + b_gp + b_gb + b_wo > kStaticScratchBytes)
		fail(TMFQS_ERR_INVALID_ARGUMENT, "state too large for the static scratch");
	char *p = static_cast<char *>(base);
	s.base = nullptr;  // not owned
	s.bytes = 0;
	s.tiles = tiles;
	s.groups = groups;
	s.tile_a = p;
	p += b_ta;
	s.tile_pre = p;
	p += b_tp;
	s.tile_b = p;
	p += b_tb;
	s.group_a = p;
	p += b_ga;
	s.group_pre = p;
	p += b_gp;
	s.group_b = p;
	p += b_gb;
	s.walk_out = p;
	s.host_out = host_out;
}

}  // namespace

SeqResult seq_sample_static(int precision, const void *amps, unsigned num_qubits, double rnd, cudaStream_t stream) {
	if(num_qubits > kStaticMaxQubits)
		fail(TMFQS_ERR_INVALID_ARGUMENT, "tmfqs_sample_static: at most " + std::to_string(kStaticMaxQubits) +
		                                     " qubits (its fixed " + std::to_string(kStaticScratchBytes >> 20) +
		                                     " MiB device scratch); use tmfqs_gpu_sample for larger states");
	const uint64_t N = 1ull << num_qubits;
	int dev = 0, sms = 0;
	check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
	WalkOut host{};  // pageable: the readback copy is synchronous
	SeqScratch s;
	carve_static(s, N, static_scratch_address(stream), &host);
	if(precision == TMFQS_FP64) return run_engine<double, kTermProb>(amps, N, Overlay{}, true, rnd, s, stream, sms, nullptr);
	return run_engine<float, kTermProb>(amps, N, Overlay{}, true, rnd, s, stream, sms, nullptr);
}

void seq_scratch_free(SeqScratch &s) {
	if(s.base) cudaFree(s.base);
	if(s.host_out) cudaFreeHost(s.host_out);
	s = SeqScratch{};
}

double seq_diff_norm(int prec_ref, const void *ref, int prec_got, const void *got, uint64_t N, SeqScratch &scratch,
                     cudaStream_t stream, int num_sms, uint64_t *launches) {
	ensure_scratch(scratch, N);
	auto run = [&](auto term) { return run_engine_term<decltype(term), false>(term, N, false, 0.0, scratch, stream, num_sms, launches).value; };
	if(prec_ref == TMFQS_FP64 && prec_got == TMFQS_FP64)
		return run(TermDiff<double, double>{static_cast<const double2 *>(ref), static_cast<const double2 *>(got), N});
	if(prec_ref == TMFQS_FP64)
		return run(TermDiff<double, float>{static_cast<const double2 *>(ref), static_cast<const float2 *>(got), N});
	if(prec_got == TMFQS_FP64)
		return run(TermDiff<float, double>{static_cast<const float2 *>(ref), static_cast<const double2 *>(got), N});
	return run(TermDiff<float, float>{static_cast<const float2 *>(ref), static_cast<const float2 *>(got), N});
}

SeqResult seq_replay(int precision, const void *amps, uint64_t N, TermKind kind, const Overlay &ov, bool stop,
                     double rnd, SeqScratch &scratch, cudaStream_t stream, int num_sms, uint64_t *launches) {
	ensure_scratch(scratch, N);
	if(precision == TMFQS_FP64) {
		switch(kind) {
			case kTermProb: return run_engine<double, kTermProb>(amps, N, ov, stop, rnd, scratch, stream, num_sms, launches);
			case kTermReal: return run_engine<double, kTermReal>(amps, N, ov, false, 0.0, scratch, stream, num_sms, launches);
			case kTermImag: return run_engine<double, kTermImag>(amps, N, ov, false, 0.0, scratch, stream, num_sms, launches);
		}
	} else {
		switch(kind) {
			case kTermProb: return run_engine<float, kTermProb>(amps, N, ov, stop, rnd, scratch, stream, num_sms, launches);
			case kTermReal: return run_engine<float, kTermReal>(amps, N, ov, false, 0.0, scratch, stream, num_sms, launches);
			case kTermImag: return run_engine<float, kTermImag>(amps, N, ov, false, 0.0, scratch, stream, num_sms, launches);
		}
	}
	fail(TMFQS_ERR_INVALID_ARGUMENT, "unknown reduction kind");
}

}  // namespace tqb
