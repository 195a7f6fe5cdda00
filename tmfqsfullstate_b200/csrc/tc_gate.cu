// Dense k-qubit gates on complex64 states as tensor-core GEMMs (tcgen05,
// kind::tf32, 3xTF32 split precision, FP32 accumulation in TMEM).
//
// A gate U (d x d complex, d = 2^k) maps every group of d amplitudes that
// share their non-target bits: y = U x.  In real form y_r = W x_r with
// x_r = [Re x_0..Re x_{d-1}, Im x_0..Im x_{d-1}] and W = [[Re U, -Im U],
// [Im U, Re U]] (2d x 2d).  A tile of 128 groups is the GEMM
// D[128, 2d] = X[128, 2d] . W^T: X (A operand) and W (B operand) sit in shared
// memory, K-major with the 128-byte swizzle; D sits in tensor memory.  Each
// operand is split into a TF32 high part and the FP32 remainder
// (x = x_h + x_l), and D = X_h W_h + X_l W_h + X_h W_l -- the FP32-level
// product the complex64 form needs, at tensor-core rate.
//
// Thread t of the CTA owns group row t of the tile: it loads the group's d
// amplitudes (consecutive threads, consecutive groups: coalesced when the
// lowest bits are not targets), writes the split row into the A tiles, and
// after the MMAs reads its row of D back from tensor memory (warp w reads
// lanes 32w..32w+31) and stores the outputs to the same addresses.  One
// elected thread issues the MMAs; their completion arrives on an mbarrier
// whose wait is bounded: a timeout sets an error flag instead of hanging,
// stops the tile loop, and waits (bounded again) for the outstanding MMAs
// before the tensor memory is released.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace tqb {

namespace {

constexpr unsigned kTcThreads = 128;  // one group row per thread, 4 warps = the 128 TMEM lanes
constexpr unsigned kTcRows = 128;     // groups per tile (the MMA's M)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (row r, column k) of a K-major, 128-byte-swizzled
// FP32 tile with `rows` rows: atoms of 32 columns x `rows` rows, 128 B per
// row, 16-byte chunk index XOR (row mod 8).
__device__ __forceinline__ uint32_t sw128(uint32_t r, uint32_t k, uint32_t rows) {
	const uint32_t kb = k >> 5, kk = k & 31u;
	return kb * rows * 128u + r * 128u + (((kk >> 2) ^ (r & 7u)) << 4) + (kk & 3u) * 4u;
}

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B, 8-row groups 1 KB apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
	uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
	d |= (uint64_t)1u << 16;             // leading byte offset: unused for swizzled K-major
	d |= (uint64_t)(1024u >> 4) << 32;   // stride byte offset
	d |= (uint64_t)1u << 46;             // descriptor version (sm100)
	d |= (uint64_t)2u << 61;             // layout: SWIZZLE_128B
	return d;
}

__device__ __forceinline__ float tf32_hi(float x) {
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return __uint_as_float(r);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
	asm volatile(
		"{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
		::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Sixteen TMEM columns of this thread's lane, without waiting (the caller
// waits once for a batch of these with tmem_wait_ld).
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t (&r)[16]) {
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
		  "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

struct TcGateGeom {
	unsigned n, k;
	unsigned tpos_sorted[8];  // target bit positions, ascending (for the group base)
	uint64_t ntiles;
};

// D = 2^k amplitudes per group; K = N = 2D reals.
template <int D>
__global__ void __launch_bounds__(kTcThreads) k_tc_gate(float2 *a, TcGateGeom g, const float *wh, const float *wl,
                                                       const uint64_t *offs, int *err) {
	constexpr uint32_t K = 2 * D, N = 2 * D;
	constexpr uint32_t A_BYTES = kTcRows * K * 4, B_BYTES = N * K * 4;
	constexpr uint32_t TCOLS = N < 32 ? 32 : N;  // TMEM columns (power of two >= 32)
	extern __shared__ __align__(1024) unsigned char dyn[];
	unsigned char *base = dyn + ((1024u - (smem_u32(dyn) & 1023u)) & 1023u);
	unsigned char *ah = base, *al = ah + A_BYTES, *bh = al + A_BYTES, *bl = bh + B_BYTES;
	__shared__ __align__(8) uint64_t mbar;
	__shared__ uint32_t tmem_base;
	__shared__ uint64_t soff[D];
	const unsigned tid = threadIdx.x, warp = tid >> 5;

	if(warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(TCOLS));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
	}
	for(uint32_t e = tid; e < N * K; e += kTcThreads) {
		const uint32_t r = e / K, c = e % K;
		*reinterpret_cast<float *>(bh + sw128(r, c, N)) = wh[e];
		*reinterpret_cast<float *>(bl + sw128(r, c, N)) = wl[e];
	}
	for(uint32_t c = tid; c < (uint32_t)D; c += kTcThreads) soff[c] = offs[c];
	if(tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	__syncthreads();
	const uint32_t tbase = tmem_base;
	const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((N >> 3) << 17) | ((kTcRows >> 4) << 24);
	bool ok = true;
	uint32_t phase = 0, stuck_phase = 0;
	// This thread's group in a tile: its non-target bits are the index, targets zero.
	auto group_base = [&](uint64_t tile) {
		uint64_t gb = tile * kTcRows + tid;
		for(unsigned i = 0; i < g.k; ++i) gb = insert0(gb, g.tpos_sorted[i]);
		return gb;
	};
	float2 x[D], xn[D];
	uint64_t tile = blockIdx.x;
	if(tile < g.ntiles) {
		const uint64_t gb0 = group_base(tile);
#pragma unroll
		for(int c = 0; c < D; ++c) x[c] = a[gb0 + soff[c]];
	}

	for(; tile < g.ntiles && ok; tile += gridDim.x, phase ^= 1u) {
		const uint64_t gb = group_base(tile), next = tile + gridDim.x;
		// Four consecutive columns share a 16-byte chunk of the swizzled row:
		// one 16-byte store each, so 8 consecutive rows fill the 8 chunks of a
		// 128-byte line (no bank conflict).
#pragma unroll
		for(int c = 0; c < D; c += 4) {
			float hr[4], hi[4];
#pragma unroll
			for(int j = 0; j < 4; ++j) {
				hr[j] = tf32_hi(x[c + j].x);
				hi[j] = tf32_hi(x[c + j].y);
			}
			*reinterpret_cast<float4 *>(ah + sw128(tid, c, kTcRows)) = make_float4(hr[0], hr[1], hr[2], hr[3]);
			*reinterpret_cast<float4 *>(ah + sw128(tid, D + c, kTcRows)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
			*reinterpret_cast<float4 *>(al + sw128(tid, c, kTcRows)) =
				make_float4(x[c].x - hr[0], x[c + 1].x - hr[1], x[c + 2].x - hr[2], x[c + 3].x - hr[3]);
			*reinterpret_cast<float4 *>(al + sw128(tid, D + c, kTcRows)) =
				make_float4(x[c].y - hi[0], x[c + 1].y - hi[1], x[c + 2].y - hi[2], x[c + 3].y - hi[3]);
		}
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		__syncthreads();
		if(tid == 0) {
			asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
			for(uint32_t s = 0; s < K / 8; ++s) {
				const uint32_t kb = s >> 2, kk = (s & 3u) * 32u;
				const uint64_t dah = smem_desc(smem_u32(ah) + kb * kTcRows * 128u + kk);
				const uint64_t dal = smem_desc(smem_u32(al) + kb * kTcRows * 128u + kk);
				const uint64_t dbh = smem_desc(smem_u32(bh) + kb * N * 128u + kk);
				const uint64_t dbl = smem_desc(smem_u32(bl) + kb * N * 128u + kk);
				mma_tf32(tbase, dah, dbh, idesc, s ? 1u : 0u);
				mma_tf32(tbase, dal, dbh, idesc, 1u);
				mma_tf32(tbase, dah, dbl, idesc, 1u);
			}
			asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mbar)));
		}
		// The next tile's amplitudes are in flight while this tile's MMAs run and
		// its outputs are stored (tiles are disjoint).
		if(next < g.ntiles) {
			const uint64_t gbn = group_base(next);
#pragma unroll
			for(int c = 0; c < D; ++c) xn[c] = a[gbn + soff[c]];
		}
		uint32_t done = 0;
		for(int it = 0; it < (1 << 20) && !done; ++it)
			asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
			             : "=r"(done) : "r"(smem_u32(&mbar)), "r"(phase) : "memory");
		// One decision for the whole CTA, so every thread takes the same path
		// through the barriers below.
		if(__syncthreads_or(!done)) {
			if(tid == 0) atomicExch(err, 1);
			ok = false;
			stuck_phase = phase;
		}
		asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
		if(ok) {
			// Row tid of D: columns c (real part) and D + c (imaginary part).
			// All 2D columns in flight together, one wait.
			const uint32_t lane_addr = tbase + ((32u * warp) << 16);
			uint32_t re[D / 16][16], im[D / 16][16];
#pragma unroll
			for(int q = 0; q < D / 16; ++q) {
				tmem_ld16_nowait(lane_addr + 16 * q, re[q]);
				tmem_ld16_nowait(lane_addr + D + 16 * q, im[q]);
			}
			tmem_wait_ld();
#pragma unroll
			for(int c = 0; c < D; ++c)
				a[gb + soff[c]] = make_float2(__uint_as_float(re[c / 16][c % 16]), __uint_as_float(im[c / 16][c % 16]));
		}
		asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
		__syncthreads();
#pragma unroll
		for(int c = 0; c < D; ++c) x[c] = xn[c];
	}
	if(!ok) {
		// The MMAs of the tile that timed out may still be running: wait for
		// their completion once more (bounded too) before the accumulator's
		// tensor memory is released, so no MMA writes a freed allocation.
		uint32_t done = 0;
		for(int it = 0; it < (1 << 22) && !done; ++it)
			asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
			             : "=r"(done) : "r"(smem_u32(&mbar)), "r"(stuck_phase) : "memory");
		if(tid == 0 && !done) atomicExch(err, 2);
		asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	}
	__syncthreads();
	if(warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCOLS));
}

template <int D>
size_t tc_smem() {
	return 2 * (size_t)kTcRows * 2 * D * 4 + 2 * (size_t)(2 * D) * (2 * D) * 4 + 1024;
}

}  // namespace

bool tc_gate_supported(int prec, unsigned n, unsigned k) { return prec == TMFQS_FP32 && (k == 4 || k == 5) && n >= k + 7; }

void launch_tc_gate(const LaunchCtx &c, void *a, unsigned n, unsigned k, const double *matrix_host, const unsigned *tpos,
                    void *&dev_buf, size_t &dev_buf_bytes) {
	if(!tc_gate_supported(TMFQS_FP32, n, k)) fail(TMFQS_ERR_LOGIC, "tensor-core gate: unsupported shape");
	const unsigned d = 1u << k, K = 2 * d;
	// W = [[Re U, -Im U], [Im U, Re U]] split into TF32 high parts and FP32 remainders.
	std::vector<float> wh(K * K), wl(K * K);
	auto tf32_round = [](double x) {
		float f = (float)x;
		uint32_t u;
		std::memcpy(&u, &f, 4);
		// Round to nearest (ties away) at 10 mantissa bits, as cvt.rna.tf32.f32 does.
		u = (u + 0x1000u) & 0xFFFFE000u;
		std::memcpy(&f, &u, 4);
		return f;
	};
	for(unsigned r = 0; r < d; ++r)
		for(unsigned col = 0; col < d; ++col) {
			const double ur = matrix_host[2 * (r * d + col)], ui = matrix_host[2 * (r * d + col) + 1];
			const double w[4] = {ur, -ui, ui, ur};  // blocks (0,0) (0,1) (1,0) (1,1)
			const unsigned rows[4] = {r, r, d + r, d + r}, cols[4] = {col, d + col, col, d + col};
			for(int b = 0; b < 4; ++b) {
				const float h = tf32_round(w[b]);
				wh[rows[b] * K + cols[b]] = h;
				wl[rows[b] * K + cols[b]] = (float)(w[b] - (double)h);
			}
		}
	// Block index c: target i is bit k-1-i of c (the reference's MSB-first order).
	std::vector<uint64_t> offs(d);
	for(unsigned cidx = 0; cidx < d; ++cidx) {
		uint64_t o = 0;
		for(unsigned i = 0; i < k; ++i)
			if((cidx >> (k - 1 - i)) & 1u) o |= 1ull << tpos[i];
		offs[cidx] = o;
	}
	TcGateGeom g{};
	g.n = n;
	g.k = k;
	std::vector<unsigned> sorted(tpos, tpos + k);
	std::sort(sorted.begin(), sorted.end());
	for(unsigned i = 0; i < k; ++i) g.tpos_sorted[i] = sorted[i];
	g.ntiles = (1ull << (n - k)) / kTcRows;
	const size_t b_w = (size_t)K * K * 4, b_off = d * 8, need = 2 * b_w + b_off + 256;
	if(need > dev_buf_bytes) {
		if(dev_buf) {
			check_cuda(cudaStreamSynchronize(c.stream), "tensor gate sync");
			cudaFree(dev_buf);
		}
		dev_buf = nullptr;
		dev_buf_bytes = 0;
		if(device_alloc((void **)&dev_buf, need) != cudaSuccess) {
			cudaGetLastError();
			fail(TMFQS_ERR_NOMEM, "tensor-core gate: allocation failed");
		}
		dev_buf_bytes = need;
	}
	unsigned char *p = static_cast<unsigned char *>(dev_buf);
	float *dwh = reinterpret_cast<float *>(p), *dwl = reinterpret_cast<float *>(p + b_w);
	uint64_t *doff = reinterpret_cast<uint64_t *>(p + 2 * b_w);
	int *derr = reinterpret_cast<int *>(p + 2 * b_w + b_off);
	check_cuda(cudaMemcpyAsync(dwh, wh.data(), b_w, cudaMemcpyHostToDevice, c.stream), "tensor gate upload");
	check_cuda(cudaMemcpyAsync(dwl, wl.data(), b_w, cudaMemcpyHostToDevice, c.stream), "tensor gate upload");
	check_cuda(cudaMemcpyAsync(doff, offs.data(), b_off, cudaMemcpyHostToDevice, c.stream), "tensor gate upload");
	check_cuda(cudaMemsetAsync(derr, 0, sizeof(int), c.stream), "tensor gate flag");
	int dev = 0, per_sm = 1;
	check_cuda(cudaGetDevice(&dev), "device");
	float2 *st = static_cast<float2 *>(a);
	if(k == 4) {
		const size_t smem = tc_smem<16>();
		check_cuda(cudaFuncSetAttribute(k_tc_gate<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "tensor gate smem");
		check_cuda(cudaFuncSetAttribute(k_tc_gate<16>, cudaFuncAttributePreferredSharedMemoryCarveout, 100), "tensor gate carveout");
		check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_gate<16>, kTcThreads, smem), "occupancy");
		// CTAs are independent (persistent loop over tiles): size the grid for
		// what fits in an SM's 228 KB of shared memory as well.
		per_sm = std::max<int>(per_sm, std::min<int>(4, (int)((228u << 10) / (smem + (2u << 10)))));
		const uint64_t grid = std::min<uint64_t>(g.ntiles, (uint64_t)c.num_sms * std::max(1, per_sm));
		k_tc_gate<16><<<(unsigned)grid, kTcThreads, smem, c.stream>>>(st, g, dwh, dwl, doff, derr);
	} else {
		const size_t smem = tc_smem<32>();
		check_cuda(cudaFuncSetAttribute(k_tc_gate<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "tensor gate smem");
		check_cuda(cudaFuncSetAttribute(k_tc_gate<32>, cudaFuncAttributePreferredSharedMemoryCarveout, 100), "tensor gate carveout");
		check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_gate<32>, kTcThreads, smem), "occupancy");
		// CTAs are independent (persistent loop over tiles): size the grid for
		// what fits in an SM's 228 KB of shared memory as well.
		per_sm = std::max<int>(per_sm, std::min<int>(4, (int)((228u << 10) / (smem + (2u << 10)))));
		const uint64_t grid = std::min<uint64_t>(g.ntiles, (uint64_t)c.num_sms * std::max(1, per_sm));
		k_tc_gate<32><<<(unsigned)grid, kTcThreads, smem, c.stream>>>(st, g, dwh, dwl, doff, derr);
	}
	check_cuda(cudaGetLastError(), "tensor gate");
	if(c.launches) ++*c.launches;
	int herr = 0;
	check_cuda(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, c.stream), "tensor gate flag read");
	check_cuda(cudaStreamSynchronize(c.stream), "tensor gate sync");
	if(herr == 1) fail(TMFQS_ERR_RUNTIME, "tensor-core gate: MMA completion wait timed out (drained before release)");
	if(herr) fail(TMFQS_ERR_RUNTIME, "tensor-core gate: MMA completion wait timed out, and so did the drain");
}

}  // namespace tqb
