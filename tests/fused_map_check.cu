// Host-side check of the exact fused pass's per-chain thread layouts
// (build_chain_map in tmfqsfullstate_b200/csrc/fused.cu), for
// tests/test_fused_map.py.  No GPU is touched.  For the passes of QFT-n in
// the exact complex128 form (low bits 0..2 plus up to 9 Hadamard bits per
// pass), and for a pass whose chains have scattered controls, every chain op
// is checked against the kernel's indexing:
//   * the butterflies (lane, q) cover every pair of the tile exactly once;
//   * the mask ml[lane] | mr[q] holds exactly the entries whose local
//     control bit is set in the pair's |1> index;
//   * with ilp set, q and q+1 (q even) differ in one bit that is no control,
//     so they share their mask;
//   * each quarter-warp's 16-byte accesses j ^ ((j >> (K-3)) & 7) fall in 8
//     distinct 16-byte bank groups, for both butterfly halves.
// Prints one line per chain op: the phase products a warp issues (its lanes'
// largest count, times 32) next to the ones its lanes need.
#include "../tmfqsfullstate_b200/csrc/fused.cu"

#include <cstdio>
#include <cstdlib>
#include <set>

namespace tqb {
[[noreturn]] void fail(int, const std::string &m) {
	std::fprintf(stderr, "%s\n", m.c_str());
	std::exit(2);
}
void check_cuda(cudaError_t, const char *) {}
void upload_async(const LaunchCtx &, void *, const void *, size_t, const char *) {}
cudaError_t device_alloc(void **, size_t) { return cudaErrorMemoryAllocation; }
}  // namespace tqb

using namespace tqb;

static int g_bad = 0;
#define EXPECT(c, ...)                        \
	do {                                      \
		if(!(c)) {                            \
			std::printf("FAIL " __VA_ARGS__); \
			std::printf("\n");                \
			++g_bad;                          \
		}                                     \
	} while(0)

// A pass over `local` (ascending global bits) with an H-chain per bit of `hs`;
// chain of bit b: controls ctrl(b) (global bits, in circuit order).
template <typename F>
static FusedPass make(unsigned n, const std::vector<unsigned> &local, const std::vector<unsigned> &hs, F ctrl) {
	FusedPass p;
	p.n = n;
	p.K = (unsigned)local.size();
	for(unsigned i = 0; i < p.K; ++i) p.lpos[i] = local[i];
	auto li = [&](unsigned bit) -> int {
		for(unsigned i = 0; i < p.K; ++i)
			if(p.lpos[i] == bit) return (int)i;
		return -1;
	};
	for(unsigned b : hs) {
		FusedOp f{};
		f.kind = kFHChain;
		f.lt = (unsigned)li(b);
		f.tab = (uint32_t)p.chain.size();
		for(unsigned c : ctrl(b)) {
			const double th = 0.1 * (c + 1);
			p.chain.push_back(ChainEntry{std::cos(th), std::sin(th), th, li(c), c});
			++f.lc;
		}
		p.ops.push_back(f);
	}
	return p;
}

static void check_pass(const char *name, const FusedPass &p) {
	const unsigned K = p.K, T = 1u << K, sw = K - 3;
	auto P = [&](unsigned j) { return j ^ ((j >> sw) & 7u); };
	for(size_t k = 0; k < p.ops.size(); ++k) {
		const FusedOp &op = p.ops[k];
		const ChainMap m = build_chain_map(p, op);
		const unsigned tb = 1u << op.lt;
		EXPECT(m.nq == (1u << (K - 6)), "%s op %zu: nq %u", name, k, m.nq);
		std::vector<int> seen(T, 0);
		double issued = 0.0, needed = 0.0;
		for(unsigned q = 0; q < m.nq; ++q) {
			unsigned wmax = 0, wsum = 0;
			for(unsigned lane = 0; lane < 32; ++lane) {
				EXPECT((m.jl[lane] & m.jr[q]) == 0 && ((m.jl[lane] | m.jr[q]) & tb) == 0, "%s op %zu: overlap", name, k);
				const unsigned j0 = m.jl[lane] | m.jr[q], j1 = j0 | tb;
				EXPECT(j1 < T, "%s op %zu: index %u out of the tile", name, k, j1);
				if(j1 >= T) continue;
				++seen[j0];
				++seen[j1];
				uint64_t want = 0;
				for(unsigned e = 0; e < op.lc; ++e) {
					const ChainEntry &ce = p.chain[op.tab + e];
					if(ce.local >= 0 && ((j1 >> ce.local) & 1u)) want |= 1ull << (63 - e);
				}
				const uint64_t got = m.ml[lane] | m.mr[q];
				EXPECT(got == want, "%s op %zu: mask of lane %u q %u", name, k, lane, q);
				const unsigned c = (unsigned)__builtin_popcountll(got);
				wmax = std::max(wmax, c);
				wsum += c;
			}
			issued += 32.0 * wmax;
			needed += wsum;
			// Quarter-warps: distinct 16-byte bank groups (low 3 bits of the slot).
			for(unsigned qw = 0; qw < 4; ++qw)
				for(unsigned half = 0; half < 2; ++half) {
					std::set<unsigned> groups;
					for(unsigned l = 8 * qw; l < 8 * qw + 8; ++l) {
						const unsigned j = (m.jl[l] | m.jr[q]) | (half ? tb : 0u);
						groups.insert(P(j) & 7u);
					}
					EXPECT(groups.size() == 8, "%s op %zu: q %u quarter-warp %u has %zu bank groups", name, k, q, qw,
					       groups.size());
				}
		}
		for(unsigned j = 0; j < T; ++j) EXPECT(seen[j] == 1, "%s op %zu: amplitude %u covered %d times", name, k, j, seen[j]);
		// The low `ilp` bits of q are no control: their q values share the mask.
		for(unsigned q = 0; q < m.nq; ++q) {
			const unsigned q0 = q & ~((1u << m.ilp) - 1u);
			EXPECT(m.mr[q] == m.mr[q0], "%s op %zu: masks of paired butterflies differ at %u", name, k, q);
		}
		uint64_t all = 0;
		for(unsigned l = 0; l < 32; ++l) all |= m.ml[l];
		EXPECT(all == m.mall, "%s op %zu: lane union", name, k);
		std::printf("case %s op %zu lt %u ilp %u pairs %u issued %.0f needed %.0f\n", name, k, op.lt, m.ilp, T / 2, issued,
		            needed);
	}
}

// The register-stage plan of a pass (plan_stages): each stage's register and
// thread bits partition the tile, the op targets are register bits, the
// shared slots are a bijection with conflict-free quarter-warps, every
// thread's walk applies exactly the entries whose local control is set in
// each of its |1> outputs, and no register-bit control follows op_split.
// Prints per op the products its warps issue for local controls against
// those its lanes need.
static void check_stages(const char *name, const FusedPass &p) {
	StageGeom g;
	std::vector<double2> phases;
	std::vector<uint64_t> tab;
	const bool planned = plan_stages(p, g, phases, tab);
	EXPECT(planned, "%s: no stage plan", name);
	if(!planned) return;
	const unsigned T = 1u << kStK;
	std::vector<int> slot_seen(T, 0);
	for(unsigned j = 0; j < T; ++j) ++slot_seen[stage_slot(j, g.scol)];
	for(unsigned j = 0; j < T; ++j) EXPECT(slot_seen[j] == 1, "%s: slot %u used %d times", name, j, slot_seen[j]);
	for(unsigned st = 0; st < g.nstages; ++st) {
		unsigned all = 0;
		for(unsigned i = 0; i < kStRB; ++i) all |= 1u << g.rbit[st][i];
		for(unsigned i = 0; i < kStTB; ++i) all |= 1u << g.tbit[st][i];
		EXPECT(all == T - 1, "%s stage %u: bits do not partition the tile", name, st);
		std::vector<int> seen(T, 0);
		for(unsigned t = 0; t < kStThreads; ++t) {
			const unsigned jl = (unsigned)g.geo[st][kStGeoTlo + (t & 15u)] | g.geo[st][kStGeoThi + (t >> 4)];
			unsigned col[kStTB], want = 0;
			stage_thread_columns(g, st, col);
			for(unsigned i = 0; i < kStTB; ++i)
				if((t >> i) & 1u) want ^= col[i];
			EXPECT(jl == want, "%s stage %u: local base of thread %u", name, st, t);
			const unsigned jb = (unsigned)g.geo[st][kStGeoSlo + (t & 15u)] ^ g.geo[st][kStGeoShi + (t >> 4)];
			for(unsigned r = 0; r < 16; ++r) {
				unsigned j = jl, x = jb;
				for(unsigned i = 0; i < kStRB; ++i)
					if((r >> i) & 1u) {
						j |= 1u << g.rbit[st][i];
						x ^= g.geo[st][kStGeoReg + i];
					}
				++seen[j];
				EXPECT(x == stage_slot(j, g.scol), "%s stage %u: slot of thread %u register %u", name, st, t, r);
			}
		}
		for(unsigned j = 0; j < T; ++j) EXPECT(seen[j] == 1, "%s stage %u: amplitude %u covered %d times", name, st, j, seen[j]);
		for(unsigned t0 = 0; t0 < kStThreads; t0 += 8)
			for(unsigned r = 0; r < 16; ++r) {
				std::set<unsigned> groups;
				for(unsigned t = t0; t < t0 + 8; ++t) {
					unsigned x = (unsigned)g.geo[st][kStGeoSlo + (t & 15u)] ^ g.geo[st][kStGeoShi + (t >> 4)];
					for(unsigned i = 0; i < kStRB; ++i)
						if((r >> i) & 1u) x ^= g.geo[st][kStGeoReg + i];
					groups.insert(x & 7u);
				}
				EXPECT(groups.size() == 8, "%s stage %u: quarter-warp at thread %u register %u has %zu bank groups", name, st,
				       t0, r, groups.size());
			}
		for(unsigned k = g.st_first[st]; k < g.st_first[st] + g.st_count[st]; ++k) {
			const FusedOp &op = p.ops[k];
			EXPECT(g.rbit[st][g.op_reg[k]] == op.lt, "%s op %u: target is not its register bit", name, k);
			bool outer = false;
			for(unsigned e = 0; e < op.lc; ++e) outer = outer || p.chain[op.tab + e].local < 0;
			EXPECT((g.op_outer[k] != 0) == outer, "%s op %u: outer-control flag", name, k);
			const uint64_t *Tb = tab.data() + (size_t)k * kStTabWords;
			const unsigned I = g.op_reg[k];
			uint64_t rall = 0;
			for(unsigned i = 0; i < kStRB; ++i) rall |= Tb[kStTabReg + i];
			EXPECT(rall == Tb[kStTabRegAll], "%s op %u: register union", name, k);
			EXPECT(Tb[kStTabReg + I] == 0, "%s op %u: entry controlled by its own target", name, k);
			const unsigned split = g.op_split[k];
			const uint64_t post = split ? ~(~0ull << (64 - split)) : ~0ull;
			EXPECT((rall & post) == 0, "%s op %u: register control after the split", name, k);
			double issued = 0.0, needed = 0.0, sub[4] = {};
			for(unsigned w = 0; w < kStThreads / 32; ++w) {
				uint64_t wu = 0;
				for(unsigned l = 0; l < 32; ++l) {
					const unsigned t = 32 * w + l;
					const uint64_t tm = Tb[kStTabLo + (t & 15u)] | Tb[kStTabHi + (t >> 4)];
					wu |= tm;
					const unsigned jl = (unsigned)g.geo[st][kStGeoTlo + (t & 15u)] | g.geo[st][kStGeoThi + (t >> 4)];
					for(unsigned r = 0; r < 16; ++r) {
						if(!((r >> I) & 1u)) continue;  // |1> outputs only
						unsigned j1 = jl;
						uint64_t got = tm;
						for(unsigned i = 0; i < kStRB; ++i)
							if((r >> i) & 1u) {
								j1 |= 1u << g.rbit[st][i];
								got |= Tb[kStTabReg + i];
							}
						uint64_t want = 0;
						for(unsigned e = 0; e < op.lc; ++e) {
							const ChainEntry &ce = p.chain[op.tab + e];
							if(ce.local >= 0 && ((j1 >> ce.local) & 1u)) want |= 1ull << (63 - e);
						}
						EXPECT(got == want, "%s op %u: mask of thread %u register %u", name, k, t, r);
						needed += (double)__builtin_popcountll(want & ~rall);
					}
				}
				EXPECT(wu == Tb[kStTabWarp + w], "%s op %u: warp %u union", name, k, w);
				issued += 32.0 * 8.0 * (double)__builtin_popcountll(wu & ~rall);
				sub[w % 4] += (double)__builtin_popcountll(wu & ~rall);
			}
			// The four sub-partitions issue the same thread-controlled products.
			EXPECT(sub[0] == sub[1] && sub[0] == sub[2] && sub[0] == sub[3], "%s op %u: sub-partitions %.0f %.0f %.0f %.0f",
			       name, k, sub[0], sub[1], sub[2], sub[3]);
			std::printf("stage %s op %u stage %u lt %u pairs %u issued %.0f needed %.0f\n", name, k, st, op.lt, T / 2, issued,
			            needed);
		}
	}
}

int main() {
	// QFT-28 in the exact complex128 form: tiles of 12 local bits, bits 0..2
	// always local; passes of 9 Hadamard bits, then the 10 lowest.
	auto below = [](unsigned b) {
		std::vector<unsigned> c;
		for(int x = (int)b - 1; x >= 0; --x) c.push_back((unsigned)x);
		return c;
	};
	auto pass_of = [&](unsigned n, unsigned hi, unsigned lo) {
		std::vector<unsigned> local = {0, 1, 2}, hs;
		for(unsigned b = lo; b <= hi; ++b) local.push_back(b);
		for(int b = (int)hi; b >= (int)lo; --b) hs.push_back((unsigned)b);
		std::sort(local.begin(), local.end());
		local.erase(std::unique(local.begin(), local.end()), local.end());
		for(unsigned b = 3; local.size() < 12; ++b)
			if(std::find(local.begin(), local.end(), b) == local.end()) local.push_back(b);
		std::sort(local.begin(), local.end());
		return make(n, local, hs, below);
	};
	check_pass("qft28_p1", pass_of(28, 27, 19));
	check_pass("qft28_p2", pass_of(28, 18, 10));
	check_pass("qft28_p3", pass_of(28, 9, 0));
	check_pass("qft32_p1", pass_of(32, 31, 23));
	check_stages("qft28_p1", pass_of(28, 27, 19));
	check_stages("qft28_p2", pass_of(28, 18, 10));
	check_stages("qft28_p3", pass_of(28, 9, 0));
	check_stages("qft32_p1", pass_of(32, 31, 23));
	check_stages("qft32_p4", pass_of(32, 4, 0));
	// Scattered controls: every other lower bit, and a repeated control.
	check_pass("scattered", make(24, {0, 1, 2, 5, 7, 9, 11, 13, 15, 17, 19, 21}, {21, 17, 13, 9},
	                             [](unsigned b) {
		                             std::vector<unsigned> c;
		                             for(int x = (int)b - 2; x >= 0; x -= 2) c.push_back((unsigned)x);
		                             c.push_back(1);
		                             c.push_back(1);
		                             return c;
	                             }));
	check_stages("scattered", make(24, {0, 1, 2, 5, 7, 9, 11, 13, 15, 17, 19, 21}, {21, 17, 13, 9},
	                               [](unsigned b) {
		                               std::vector<unsigned> c;
		                               for(int x = (int)b - 2; x >= 0; x -= 2) c.push_back((unsigned)x);
		                               c.push_back(1);
		                               c.push_back(1);
		                               return c;
	                               }));
	// Seven local bits (the smallest mapped tile) and 13 (complex64).
	check_pass("k7", make(7, {0, 1, 2, 3, 4, 5, 6}, {6, 5, 4, 3}, below));
	check_pass("k13", make(30, {0, 1, 2, 3, 20, 21, 22, 23, 24, 25, 26, 27, 28}, {28, 27, 26, 25, 24, 23, 22, 21, 20}, below));
	std::printf("result %s\n", g_bad ? "FAIL" : "OK");
	return g_bad ? 1 : 0;
}
