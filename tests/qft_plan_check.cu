// Host-side check of the QFT segment recogniser and planner (qft_segment and
// plan_qft in tmfqsfullstate_b200/csrc/qft_pass.cu): one line per constructed
// pass, for tests/test_qft_plan.py.  No GPU is touched.
#include "../tmfqsfullstate_b200/csrc/qft_pass.cu"

#include <cstdio>
#include <cstdlib>

namespace tqb {
[[noreturn]] void fail(int, const std::string &m) {
	std::fprintf(stderr, "%s\n", m.c_str());
	std::exit(2);
}
void check_cuda(cudaError_t, const char *) {}
}  // namespace tqb

using namespace tqb;

// A pass of n qubits over the given local bits: Hadamards on the bits of `hs`
// (descending), each followed by the ladder's phases pi/2^(b-c) for c in
// [r0, b).  `drop` removes the last phase of the first chain, `skew` changes
// the first chain's first angle, `bare` leaves the Hadamards without phases.
static FusedPass make(unsigned n, const std::vector<unsigned> &local, const std::vector<unsigned> &hs, unsigned r0,
                      bool drop = false, bool skew = false, bool bare = false) {
	FusedPass p;
	p.n = n;
	p.K = (unsigned)local.size();
	for(unsigned i = 0; i < p.K; ++i) p.lpos[i] = local[i];
	auto li = [&](unsigned bit) -> int {
		for(unsigned i = 0; i < p.K; ++i)
			if(p.lpos[i] == bit) return (int)i;
		return -1;
	};
	const double pi = std::acos(-1.0);
	for(size_t k = 0; k < hs.size(); ++k) {
		const unsigned b = hs[k];
		FusedOp f{};
		f.lt = (unsigned)li(b);
		if(bare) {
			f.kind = kFH;
			p.ops.push_back(f);
			continue;
		}
		f.kind = kFHChain;
		f.tab = (uint32_t)p.chain.size();
		unsigned cnt = 0;
		for(int c = (int)b - 1; c >= (int)r0; --c) {
			if(drop && k == 0 && c == (int)r0) break;
			double th = std::ldexp(pi, -(int)(b - (unsigned)c));
			if(skew && k == 0 && cnt == 0) th *= 1.001;
			p.chain.push_back(ChainEntry{std::cos(th), std::sin(th), th, li((unsigned)c), (unsigned)c});
			++cnt;
		}
		f.lc = cnt;
		if(cnt == 0) f.kind = kFH;
		p.ops.push_back(f);
	}
	return p;
}

// A QFT segment, else a Walsh segment (Hadamards only), as launch_qft_pass
// tries them; for a Walsh plan, every stage is marked and the tail (if any)
// sits on the lowest bits.
static void check(const char *name, const FusedPass &p, unsigned vb = 8) {
	std::vector<unsigned> hb;
	unsigned r0 = 0;
	const bool seg = qft_segment(p, hb, r0);
	bool walsh = false;
	if(!seg) {
		walsh = walsh_segment(p, hb);
		r0 = p.n;
	}
	int planned = -1;
	unsigned nstages = 0, marked = 0, tail = 0, tma = 0, tdims = 0, tok = 1;
	double scale = 0.0;
	if(seg || walsh) {
		QftGeom g{};
		planned = plan_qft(p, hb, r0, vb, vb == 8 ? 5 : 4, g, walsh, true) ? 1 : 0;
		nstages = g.nstages;
		scale = g.scale;
		for(unsigned s = 0; s < g.nstages; ++s) {
			marked += g.st[s].walsh ? 1u : 0u;
			if(walsh && g.st[s].wmask) planned = 0;  // a Walsh stage takes no twiddle
		}
		tail = g.nstages ? g.st[g.nstages - 1].tail : 0u;
		tma = g.tma;
		tdims = g.tma ? g.tma_dims : 0u;
		if(g.tma) {
			// The box enumerates the local index in order (ascending runs, the
			// outer runs of box 1, strides 8 << first bit), and the copy's
			// 128-byte swizzle (byte bits 4-6 ^= bits 7-9) is the pass's swizzle.
			uint64_t elems = 1;
			unsigned bit = 0, local = 0;
			for(unsigned i = 0; i < g.tma_dims; ++i) {
				if(g.tma_stride[i] != ((uint64_t)vb << bit) && i) tok = 0;
				if(!g.tma_outer[i]) {
					elems *= g.tma_box[i];
					for(unsigned b = 0; b < g.tma_len[i]; ++b)
						if(g.lpos[local++] != bit + b) tok = 0;
				} else if(g.tma_box[i] != 1) {
					tok = 0;
				}
				bit += g.tma_len[i];
			}
			if(elems != (uint64_t(vb / 8) << g.K) || bit != p.n || g.tma_box[0] * 8 != 128) tok = 0;
			for(unsigned j = 0; j < (1u << g.K); ++j) {
				const unsigned byte = j * vb, tswz = byte ^ (((byte >> 7) & 7u) << 4);
				if(tswz != qft_phys(g, j) * vb) tok = 0;
			}
		}
	}
	std::printf("case %s segment %d hb %zu r0 %u planned %d nstages %u scale %.17g walsh %d marked %u tail %u tma %u dims %u tok %u\n",
	            name, (int)seg, hb.size(), seg ? r0 : 0u, planned, nstages, scale, (int)walsh, marked, tail, tma, tdims, tok);
}

static std::vector<unsigned> range(unsigned lo, unsigned hi) {  // [lo, hi)
	std::vector<unsigned> v;
	for(unsigned b = lo; b < hi; ++b) v.push_back(b);
	return v;
}
static std::vector<unsigned> down(unsigned hi, unsigned lo) {  // hi, hi-1, ..., lo
	std::vector<unsigned> v;
	for(int b = (int)hi; b >= (int)lo; --b) v.push_back((unsigned)b);
	return v;
}

int main() {
	// 28 qubits, complex64: the planner's passes hold bits {0..4} and the
	// pass's Hadamard bits, then the last pass the 13 lowest bits.
	std::vector<unsigned> first = range(0, 5), top = range(20, 28);
	first.insert(first.end(), top.begin(), top.end());
	check("qft28_first", make(28, first, down(27, 20), 0));
	check("qft28_last", make(28, range(0, 13), down(11, 0), 0));
	check("lone_h", make(28, range(0, 13), {7}, 0, false, false, true));
	check("bare_run", make(28, range(0, 13), down(7, 4), 0, false, false, true));
	check("dropped_phase", make(28, range(0, 13), down(11, 0), 0, true));
	check("wrong_angle", make(28, range(0, 13), down(11, 0), 0, false, true));
	check("sub_register", make(20, range(0, 13), down(12, 6), 3));
	// Hadamards only: the top bits of a 24-qubit state, the 13 lowest bits
	// (last stage fused into the copy-out), and scattered bits.
	std::vector<unsigned> wl = range(0, 5), wt = range(16, 24);
	wl.insert(wl.end(), wt.begin(), wt.end());
	check("walsh_top", make(24, wl, down(23, 16), 0, false, false, true));
	check("walsh_low", make(24, range(0, 13), down(12, 0), 0, false, false, true));
	check("walsh_scattered", make(24, range(0, 13), {3, 11, 7, 9}, 0, false, false, true));
	// Hadamards on bits 7..0 with a ring of controlled phases after them (the
	// layered circuits' last pass of a layer), before them, on both sides, and
	// with a phase flip: no Walsh segment (the radix pass takes them).
	auto ring = [&](FusedPass q, bool before, bool after, bool flip) {
		std::vector<FusedOp> cps;
		for(unsigned b = 0; b < 24; ++b) {
			FusedOp f{};
			f.kind = kFCP;
			f.mask = (1ull << b) | (1ull << ((b + 1) % 24));
			f.cr = std::cos(0.1 * b);
			f.ci = std::sin(0.1 * b);
			cps.push_back(f);
		}
		if(flip) {
			FusedOp f{};
			f.kind = kFFlip;
			f.state = 12345;
			cps.push_back(f);
		}
		if(before) q.ops.insert(q.ops.begin(), cps.begin(), cps.end());
		if(after) q.ops.insert(q.ops.end(), cps.begin(), cps.end());
		return q;
	};
	check("walsh_diag_after", ring(make(24, range(0, 13), down(7, 0), 0, false, false, true), false, true, false));
	check("walsh_diag_before", ring(make(24, range(0, 13), down(7, 0), 0, false, false, true), true, false, true));
	check("walsh_diag_both", ring(make(24, range(0, 13), down(7, 0), 0, false, false, true), true, true, false));
	check("walsh_diag_after_top", ring(make(24, wl, down(23, 16), 0, false, false, true), false, true, false));
	// complex128 (12-bit tiles): bits {0..3} and the pass's 8 Hadamard bits.
	std::vector<unsigned> c128 = range(0, 4), c128t = range(20, 28);
	c128.insert(c128.end(), c128t.begin(), c128t.end());
	check("qft28_first_c128", make(28, c128, down(27, 20), 0), 16);
	check("qft28_last_c128", make(28, range(0, 12), down(11, 0), 0), 16);
	return 0;
}
