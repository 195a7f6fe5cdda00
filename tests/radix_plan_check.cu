// Host-side check of the radix pass planner (build_radix_program in
// tmfqsfullstate_b200/csrc/radix.cu): builds the stage programs of a few
// passes of the 24-qubit layered circuit and prints their structure, one
// line per stage, for tests/test_radix_plan.py.  No GPU is touched.
#include "../tmfqsfullstate_b200/csrc/radix.cu"

#include <cstdio>
#include <cstdlib>

namespace tqb {
[[noreturn]] void fail(int, const std::string &m) {
	std::fprintf(stderr, "%s\n", m.c_str());
	std::exit(2);
}
void check_cuda(cudaError_t, const char *) {}
cudaError_t device_alloc(void **, size_t) { return cudaErrorMemoryAllocation; }
void upload_async(const LaunchCtx &, void *, const void *, size_t, const char *) {}
}  // namespace tqb

using namespace tqb;

static void dump(const char *name, const FusedPass &p) {
	RadixProgram P;
	const bool ok = build_radix_program<4>(p, p.K, 8, P);
	std::printf("pass %s ok %d nstages %u nslots %u outer_free %u\n", name, (int)ok, P.g.nstages, P.g.nslots, P.g.outer_free);
	for(size_t s = 0; s < P.stages.size(); ++s) {
		const RadixStage &S = P.stages[s];
		std::printf("stage %zu items", s);
		for(unsigned k = S.first; k < S.first + S.count; ++k) std::printf(" %u:%u", P.items[k] & 255u, (P.items[k] >> 8) & 255u);
		std::printf(" direct %u post %u rbit", S.direct, S.post_mask);
		for(int i = 0; i < 4; ++i) std::printf(" %u", S.rbit[i]);
		std::printf(" rsorted");
		for(int i = 0; i < 4; ++i) std::printf(" %u", S.rsorted[i]);
		std::printf(" imask");
		for(int i = 0; i < 4; ++i) std::printf(" %u", S.imask[i]);
		std::printf(" roff");
		for(int i = 0; i < 4; ++i) std::printf(" %u", S.roff[i]);
		std::printf(" gbit");
		for(int i = 0; i < 4; ++i) std::printf(" %llu", (unsigned long long)S.gbit[i]);
		std::printf("\n");
	}
	for(const RadixSlot &sl : P.slots) std::printf("slot scale %.17g a %u b %u o %u x %u\n", sl.scale, sl.a_count, sl.b_count, sl.o_count, sl.x_count);
}

static FusedOp hop(unsigned local) {
	FusedOp f{};
	f.kind = kFH;
	f.lt = local;
	return f;
}

int main() {
	const unsigned n = 24;
	{  // Hadamards on bits 0..12: the backward's first pass over a layer in reverse order.
		FusedPass p;
		p.n = n;
		p.K = 13;
		for(unsigned i = 0; i < 13; ++i) p.lpos[i] = i;
		for(unsigned b = 0; b < 13; ++b) p.ops.push_back(hop(b));
		dump("h0_12", p);
	}
	{  // Hadamards on bits 23..16, local bits {0..4} and {16..23}.
		FusedPass p;
		p.n = n;
		p.K = 13;
		for(unsigned i = 0; i < 5; ++i) p.lpos[i] = i;
		for(unsigned i = 0; i < 8; ++i) p.lpos[5 + i] = 16 + i;
		for(int b = 23; b >= 16; --b) p.ops.push_back(hop(5 + (unsigned)(b - 16)));
		dump("h23_16", p);
	}
	{  // Hadamards on bits 7..0 and the ring of controlled phases (q, q+1 mod n).
		FusedPass p;
		p.n = n;
		p.K = 13;
		for(unsigned i = 0; i < 13; ++i) p.lpos[i] = i;
		for(int b = 7; b >= 0; --b) p.ops.push_back(hop((unsigned)b));
		for(unsigned q = 0; q < n; ++q) {
			const unsigned b0 = n - 1 - q, b1 = n - 1 - ((q + 1) % n);
			FusedOp f{};
			f.kind = kFCP;
			f.mask = (1ull << b0) | (1ull << b1);
			f.theta = 0.1 * (q + 1);
			f.cr = std::cos(f.theta);
			f.ci = std::sin(f.theta);
			p.ops.push_back(f);
		}
		dump("ring", p);
	}
	return 0;
}
