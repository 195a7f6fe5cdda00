// Register-level building blocks shared by the radix passes of the fast forms
// (complex64 states, and complex128 with TMFQS_OPT_EXACT off): unscaled
// butterflies, complex products, and the QFT ladder on the register bits of
// one thread, compiled for each ladder width.
#ifndef TMFQS_B200_RADIX_COMMON_CUH
#define TMFQS_B200_RADIX_COMMON_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace tqb {

// cos and sin of 2*pi*k/32, k < 16, from the host C library in FP64, and the
// same values rounded once to FP32: the twiddles of the compiled QFT ladders.
constexpr unsigned kRoots = 16;
struct RootTable {
	double root[kRoots][2];
	float rootf[kRoots][2];
};

// Root k as a storage-type value (kernel parameters: uniform loads).
__device__ __forceinline__ void root_of(const RootTable &t, int k, double2 &r) {
	r = make_double2(t.root[k][0], t.root[k][1]);
}
__device__ __forceinline__ void root_of(const RootTable &t, int k, float2 &r) {
	r = make_float2(t.rootf[k][0], t.rootf[k][1]);
}

template <typename V>
__device__ __forceinline__ V vmul(V a, V b) {
	V r;
	r.x = fma(a.x, b.x, -(a.y * b.y));
	r.y = fma(a.x, b.y, a.y * b.x);
	return r;
}

// One unscaled butterfly: (x, y) <- (x + y, x - y).  Complex64 values use
// the paired FP32 instructions (one instruction per complex add).
__device__ __forceinline__ void bfly2(double2 &x, double2 &y) {
	const double2 a = x, b = y;
	x = make_double2(a.x + b.x, a.y + b.y);
	y = make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ void bfly2(float2 &x, float2 &y) {
	const float2 a = x, b = y;
	x = __fadd2_rn(a, b);
	y = __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}

// v times exp(2*pi*i*k/32), k < 16 known at compile time: exact for k = 0 and
// k = 8 (the factor i), otherwise a complex product with the tabulated root.
template <int k, typename V>
__device__ __forceinline__ V mul_root(V v, const RootTable &t) {
	if constexpr(k == 0) {
		return v;
	} else if constexpr(k == 8) {
		V r;
		r.x = -v.y;
		r.y = v.x;
		return r;
	} else {
		V w;
		root_of(t, k, w);
		return vmul(v, w);
	}
}

// The QFT ladder on register bits 0..D-1 (Hadamards in bit order, and after
// the one on bit i the controlled phases pi/2^(j-i) with every later bit j).
// After the butterflies on bit i, the |1> output at register r gets
// exp(2*pi*i*K/2^(D-i)) with K = sum_{j>i} r_j 2^(D-1-j).  Unscaled: the
// 1/sqrt(2) factors are left to the caller.
template <typename V, int RB, int D>
__device__ __forceinline__ void qft_stage(V (&v)[1 << RB], const RootTable &t) {
#pragma unroll
	for(int i = 0; i < D; ++i) {
#pragma unroll
		for(int q = 0; q < (1 << (RB - 1)); ++q) {
			const int lo = (1 << i) - 1;
			const int r0 = ((q & ~lo) << 1) | (q & lo), r1 = r0 | (1 << i);
			bfly2(v[r0], v[r1]);
		}
#pragma unroll
		for(int r = 0; r < (1 << RB); ++r) {
			if(!((r >> i) & 1)) continue;
			int K = 0;
#pragma unroll
			for(int j = i + 1; j < D; ++j) K |= ((r >> j) & 1) << (D - 1 - j);
			// exp(2 pi i K / 2^(D-i)) = root[K * 32 / 2^(D-i)]
			const int idx = K << (5 - (D - i));
			switch(idx) {
				case 0: break;
				case 1: v[r] = mul_root<1>(v[r], t); break;
				case 2: v[r] = mul_root<2>(v[r], t); break;
				case 3: v[r] = mul_root<3>(v[r], t); break;
				case 4: v[r] = mul_root<4>(v[r], t); break;
				case 5: v[r] = mul_root<5>(v[r], t); break;
				case 6: v[r] = mul_root<6>(v[r], t); break;
				case 7: v[r] = mul_root<7>(v[r], t); break;
				case 8: v[r] = mul_root<8>(v[r], t); break;
				case 9: v[r] = mul_root<9>(v[r], t); break;
				case 10: v[r] = mul_root<10>(v[r], t); break;
				case 11: v[r] = mul_root<11>(v[r], t); break;
				case 12: v[r] = mul_root<12>(v[r], t); break;
				case 13: v[r] = mul_root<13>(v[r], t); break;
				case 14: v[r] = mul_root<14>(v[r], t); break;
				case 15: v[r] = mul_root<15>(v[r], t); break;
				default: break;
			}
		}
	}
}

// The roots exp(2*pi*i*k/32), k < 16, in FP64 and rounded once to FP32.
inline void fill_roots(RootTable &t) {
	const double two_pi = 2.0 * std::acos(-1.0);
	for(unsigned k = 0; k < kRoots; ++k) {
		t.root[k][0] = std::cos(two_pi * k / 32.0);
		t.root[k][1] = std::sin(two_pi * k / 32.0);
		t.rootf[k][0] = (float)t.root[k][0];
		t.rootf[k][1] = (float)t.root[k][1];
	}
}

}  // namespace tqb

#endif
