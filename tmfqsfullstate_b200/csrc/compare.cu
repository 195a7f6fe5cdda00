// experiment::compareStates (reference src/tmfqs/experiment/comparison.cpp:12-62)
// on two device states.
//
// The report's maxima, the worst state and the bitwise flag do not depend on
// the order of the scan, so one parallel pass computes them exactly: each
// state's error terms are formed with the reference's operations and operand
// order in FP64, and the worst state is the first index of the largest
// amplitude error (the reference's strict `>` update).  The three sums
// (|got - ref|^2, |ref|^2, |got|^2) are the reference's left-to-right sums,
// replayed exactly by the sequential-sum engine (seqsum.cu).
#include <algorithm>
#include <cmath>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace tqb {

namespace {

constexpr unsigned kCmpThreads = 256;

struct CmpPartial {
	double max_amp;       // largest |got - ref| ...
	uint64_t worst;       // ... first reached at this index
	double max_comp;
	double max_prob;
	unsigned differs;     // some component differs (bitwise)
	unsigned pad;
};

__device__ __forceinline__ void cmp_merge(CmpPartial &a, const CmpPartial &b) {
	if(b.max_amp > a.max_amp || (b.max_amp == a.max_amp && b.worst < a.worst)) {
		a.max_amp = b.max_amp;
		a.worst = b.worst;
	}
	if(b.max_comp > a.max_comp) a.max_comp = b.max_comp;
	if(b.max_prob > a.max_prob) a.max_prob = b.max_prob;
	a.differs |= b.differs;
}

template <typename RA, typename RB>
__global__ void __launch_bounds__(kCmpThreads) k_compare(const typename Vec2<RA>::type *ref, const typename Vec2<RB>::type *got,
                                                        uint64_t N, CmpPartial *partials) {
	// Every thread scans increasing indices, so its first maximum is its
	// lowest index; merges keep the lowest index among equal maxima.
	CmpPartial p{0.0, 0, 0.0, 0.0, 0u, 0u};
	for(uint64_t s = gtid(); s < N; s += gstride()) {
		const auto r = ref[s];
		const auto g = got[s];
		const double rr = (double)r.x, ri = (double)r.y, gr = (double)g.x, gi = (double)g.y;
		if(rr != gr || ri != gi) p.differs = 1u;
		const double dr = rsub(gr, rr), di = rsub(gi, ri);
		const double err = __dsqrt_rn(radd(rmul(dr, dr), rmul(di, di)));
		if(err > p.max_amp) {
			p.max_amp = err;
			p.worst = s;
		}
		const double ar = fabs(dr), ai = fabs(di);
		const double comp = ar < ai ? ai : ar;  // std::max(|dr|, |di|)
		if(comp > p.max_comp) p.max_comp = comp;
		const double pref = radd(rmul(rr, rr), rmul(ri, ri)), pgot = radd(rmul(gr, gr), rmul(gi, gi));
		const double pe = fabs(rsub(pgot, pref));
		if(pe > p.max_prob) p.max_prob = pe;
	}
	__shared__ CmpPartial red[kCmpThreads];
	red[threadIdx.x] = p;
	__syncthreads();
	for(unsigned w = kCmpThreads / 2; w > 0; w >>= 1) {
		if(threadIdx.x < w) cmp_merge(red[threadIdx.x], red[threadIdx.x + w]);
		__syncthreads();
	}
	if(threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

}  // namespace

void launch_compare(const LaunchCtx &c, int prec_ref, const void *ref, int prec_got, const void *got, uint64_t N,
                    CompareReport &out) {
	const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((N + kCmpThreads - 1) / kCmpThreads, (uint64_t)c.num_sms * 4));
	CmpPartial *dev = nullptr;
	if(device_alloc((void **)&dev, sizeof(CmpPartial) * blocks) != cudaSuccess) {
		cudaGetLastError();
		fail(TMFQS_ERR_NOMEM, "compare: scratch allocation failed");
	}
	struct Free {
		void *p;
		~Free() { cudaFree(p); }
	} guard{dev};
	if(prec_ref == TMFQS_FP64 && prec_got == TMFQS_FP64)
		k_compare<double, double><<<blocks, kCmpThreads, 0, c.stream>>>(static_cast<const double2 *>(ref), static_cast<const double2 *>(got), N, dev);
	else if(prec_ref == TMFQS_FP64)
		k_compare<double, float><<<blocks, kCmpThreads, 0, c.stream>>>(static_cast<const double2 *>(ref), static_cast<const float2 *>(got), N, dev);
	else if(prec_got == TMFQS_FP64)
		k_compare<float, double><<<blocks, kCmpThreads, 0, c.stream>>>(static_cast<const float2 *>(ref), static_cast<const double2 *>(got), N, dev);
	else
		k_compare<float, float><<<blocks, kCmpThreads, 0, c.stream>>>(static_cast<const float2 *>(ref), static_cast<const float2 *>(got), N, dev);
	check_cuda(cudaGetLastError(), "compare");
	if(c.launches) ++*c.launches;
	std::vector<CmpPartial> host(blocks);
	check_cuda(cudaMemcpyAsync(host.data(), dev, sizeof(CmpPartial) * blocks, cudaMemcpyDeviceToHost, c.stream), "compare read");
	check_cuda(cudaStreamSynchronize(c.stream), "compare sync");
	// Blocks cover interleaved index ranges: keep the lowest index among equal maxima.
	CmpPartial all{0.0, 0, 0.0, 0.0, 0u, 0u};
	for(const CmpPartial &p : host) {
		if(p.max_amp > all.max_amp || (p.max_amp == all.max_amp && p.worst < all.worst && p.max_amp > 0.0)) {
			all.max_amp = p.max_amp;
			all.worst = p.worst;
		}
		all.max_comp = std::max(all.max_comp, p.max_comp);
		all.max_prob = std::max(all.max_prob, p.max_prob);
		all.differs |= p.differs;
	}
	out.bitwise_equal = all.differs == 0u;
	out.max_abs_amplitude_error = all.max_amp;
	out.worst_state = all.worst;
	out.max_abs_component_error = all.max_comp;
	out.max_abs_probability_error = all.max_prob;
}

}  // namespace tqb
