// Exact replay of a left-to-right IEEE-754 double summation, in parallel.
//
// The reference computes every reduction on the dense path as a sequential
// loop `c += term(s)` (totalProbability, dense_state_backend.cpp:161-171;
// sampleMeasurement, :173-188; logicalAmplitudeSum,
// quantum_register.cpp:176-190).  A tree reduction rounds differently, so
// its total -- and the index at which a cumulative sum first reaches a
// random draw -- can differ from the reference's.  This header holds the
// math that lets a GPU reproduce the sequential rounding exactly:
//
//  * While the running sum C stays inside one binade [2^e, 2^(e+1)) (or its
//    negative mirror), every rounded add lands on the fixed grid
//    u = 2^(e-52).  So C_j = C_{j-1} + u * inc_j, where inc_j is the term
//    rounded to the grid -- exactly, except that a term lying half-way
//    between two grid points rounds to the even result, which depends on
//    the parity of C/u.
//  * Each term is therefore a function {parity -> integer increment}; such
//    functions compose associatively (tq_compose), so a tile of terms
//    reduces to one pair (inc if C/u is even, inc if odd).
//  * A rigorous bound on |C_j - exact prefix| (recursive summation error,
//    |C_j - S_j| <= gamma_j * sum|x_i|, gamma_j = j*u0/(1-j*u0)) tells which
//    tiles provably keep C inside one binade ("clean" tiles).  Everything
//    else is replayed exactly, 32 terms at a time, speculating that the
//    binade does not change and falling back to one real double add where
//    it does.
//
// The functions are host+device so that the CPU model in the tests and the
// CUDA kernels share one implementation.
#ifndef TMFQS_B200_SEQSUM_CORE_H
#define TMFQS_B200_SEQSUM_CORE_H

#include <stdint.h>

#ifdef __CUDACC__
#define TQ_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define TQ_HD inline
#endif

namespace tq {

// Integer increment (in grid units) of a run of terms, for an even (i0) and
// an odd (i1) value of C/u at the start of the run.
struct Inc {
	int64_t i0;
	int64_t i1;
};

TQ_HD Inc inc_identity() { return Inc{0, 0}; }

// Run L followed by run R.
TQ_HD Inc compose(Inc L, Inc R) {
	const int64_t par0 = L.i0 & 1;        // parity after L when starting even
	const int64_t par1 = (L.i1 + 1) & 1;  // parity after L when starting odd
	Inc o;
	o.i0 = L.i0 + (par0 ? R.i1 : R.i0);
	o.i1 = L.i1 + (par1 ? R.i1 : R.i0);
	return o;
}

TQ_HD int64_t apply(Inc g, int64_t c) { return (c & 1) ? g.i1 : g.i0; }

#ifdef __CUDACC__
TQ_HD double tq_floor(double x) { return floor(x); }
TQ_HD double tq_ldexp(double x, int e) { return ldexp(x, e); }
TQ_HD int tq_ilogb(double x) { return ilogb(x); }
#else
inline double tq_floor(double x) { return std::floor(x); }
inline double tq_ldexp(double x, int e) { return std::ldexp(x, e); }
inline int tq_ilogb(double x) { return std::ilogb(x); }
#endif

// Grid scale 2^(52-e) for binade e (C/u = C * scale is an integer).
TQ_HD double grid_scale(int e) { return tq_ldexp(1.0, 52 - e); }

// One term p on the grid of scale `scale` (power of two, exact product).
TQ_HD Inc term_inc(double p, double scale) {
	const double q = p * scale;
	const double m = tq_floor(q);
	const double f = q - m;
	const int64_t mi = (int64_t)m;
	Inc r;
	if(f < 0.5) {
		r.i0 = mi;
		r.i1 = mi;
	} else if(f > 0.5) {
		r.i0 = mi + 1;
		r.i1 = mi + 1;
	} else {
		// Tie: C/u + m + 1/2 rounds to the even neighbour.
		r.i0 = mi + (mi & 1);
		r.i1 = mi + ((mi + 1) & 1);
	}
	return r;
}

constexpr int kDirty = -100000;
constexpr int kIdentity = 100000;  // all terms zero: C unchanged, any binade

// Binade shared by every value in [lo, hi] (lo <= hi, same sign, nonzero),
// or kDirty.  Returns e with |x| in [2^e, 2^(e+1)); the sign is the caller's.
TQ_HD int common_binade(double lo, double hi) {
	if(lo > 0.0) {
		const int a = tq_ilogb(lo), b = tq_ilogb(hi);
		if(a != b || a < -1000 || a > 1000) return kDirty;
		return a;
	}
	if(hi < 0.0) {
		const int a = tq_ilogb(-hi), b = tq_ilogb(-lo);
		if(a != b || a < -1000 || a > 1000) return kDirty;
		return a;
	}
	return kDirty;
}

// Whether integer grid value c (C = c/scale) is strictly inside the binade
// interior where the grid model is exact: 2^52 < |c| < 2^53.
TQ_HD bool grid_interior(int64_t c) {
	const int64_t lo = (int64_t)1 << 52, hi = (int64_t)1 << 53;
	return (c > lo && c < hi) || (c < -lo && c > -hi);
}

// gamma_k = k*u0 / (1 - k*u0), u0 = 2^-53, with a small safety factor.
TQ_HD double gamma_bound(double k) {
	const double u0 = 1.1102230246251565e-16;
	const double ku = k * u0;
	return ku / (1.0 - ku) * 1.0000001 + 1e-30;
}

// Error-free transformation helpers (double-double accumulation).
TQ_HD void two_sum(double a, double b, double &s, double &e) {
	s = a + b;
	const double bb = s - a;
	e = (a - (s - bb)) + (b - bb);
}

struct DD {
	double hi;
	double lo;
};

TQ_HD DD dd_add(DD a, DD b) {
	double s, e;
	two_sum(a.hi, b.hi, s, e);
	e += a.lo + b.lo;
	double h, l;
	two_sum(s, e, h, l);
	return DD{h, l};
}

TQ_HD DD dd_add_d(DD a, double b) {
	double s, e;
	two_sum(a.hi, b, s, e);
	e += a.lo;
	double h, l;
	two_sum(s, e, h, l);
	return DD{h, l};
}

}  // namespace tq

#endif
