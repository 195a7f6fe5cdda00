// Device-side helpers shared by the kernels of libtmfqs_b200.
//
// Exactness: every kernel that must match the reference uses the explicit
// round-to-nearest intrinsics below (no FMA contraction; the library is also
// compiled with -fmad=false), so each complex operation is the same sequence
// of IEEE operations as the reference C++ expression it restates.
#ifndef TMFQS_B200_DEVICE_COMMON_CUH
#define TMFQS_B200_DEVICE_COMMON_CUH

#include <cuda_runtime.h>
#include <stdint.h>

namespace tqb {

template <typename R>
struct Vec2;
template <>
struct Vec2<double> {
	typedef double2 type;
};
template <>
struct Vec2<float> {
	typedef float2 type;
};

__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }

// Insert a zero bit at position b of i.
__device__ __forceinline__ uint64_t insert0(uint64_t i, unsigned b) {
	const uint64_t lo = i & ((1ull << b) - 1ull);
	return ((i ^ lo) << 1) | lo;
}

// Insert zero bits at positions lo < hi.
__device__ __forceinline__ uint64_t insert00(uint64_t i, unsigned lo, unsigned hi) {
	return insert0(insert0(i, lo), hi);
}

// Complex product (pr + i pi) * (re + i im) as written in
// dense_state_backend.cpp:300-301: re' = pr*re - pi*im; im' = pr*im + pi*re.
template <typename R>
__device__ __forceinline__ void cmul_ref(R pr, R pi, R &re, R &im) {
	const R nr = rsub(rmul(pr, re), rmul(pi, im));
	const R ni = radd(rmul(pr, im), rmul(pi, re));
	re = nr;
	im = ni;
}

// 16-byte asynchronous global -> shared copies (both addresses 16-byte
// aligned), committed and awaited in groups.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
// 32-byte global loads and stores (sm_100 vector width; 32-byte aligned).
__device__ __forceinline__ void ld_global_v8f(const float *p, float (&r)[8]) {
	asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
	             : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
	             : "l"(p));
}
__device__ __forceinline__ void st_global_v8f(float *p, const float (&r)[8]) {
	asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(r[0]), "f"(r[1]), "f"(r[2]),
	             "f"(r[3]), "f"(r[4]), "f"(r[5]), "f"(r[6]), "f"(r[7])
	             : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Grid-stride helpers.
__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

}  // namespace tqb

#endif
