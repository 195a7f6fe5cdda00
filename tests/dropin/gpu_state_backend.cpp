// IStateBackend (include/tmfqs/storage/i_state_backend.h:22-164 of the
// reference) over the C ABI of libtmfqs_b200 -- the binding a maintainer adds
// to the reference tree (src/tmfqs/storage/gpu/).  One virtual, one C-ABI
// call; C-ABI status codes map back to the reference's exception classes
// (out_of_range, invalid_argument, logic_error, runtime_error).
//
// With TMFQS_DENSE_BACKEND=gpu in the environment the patched registry builds
// this backend for Dense registers too, so that unmodified programs (the
// reference's own integration tests) run on the device; at exit it reports on
// stderr how many device backends were created.
#include "tmfqs/storage/gpu/gpu_state_backend.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "tmfqs/core/state_space.h"
#include "tmfqs_b200.h"

namespace tmfqs {
namespace {

void check(int rc) {
	if(rc == TMFQS_OK) return;
	const std::string msg = tmfqs_gpu_last_error();
	switch(rc) {
		case TMFQS_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
		case TMFQS_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
		case TMFQS_ERR_LOGIC: throw std::logic_error(msg);
		default: throw std::runtime_error(msg);  // runtime, CUDA, device out of memory
	}
}

std::atomic<unsigned long> g_created{0};

struct CreationReport {
	~CreationReport() {
		if(denseRedirectedToGpu()) std::fprintf(stderr, "[tmfqs-gpu] device backends created: %lu\n", g_created.load());
	}
} g_report;

constexpr StateIndex kChunkStates = StateIndex{1} << 22;  // 64 MiB of complex128 per visitor call

class GpuStateBackend final : public IStateBackend {
	public:
		GpuStateBackend() {
			check(tmfqs_gpu_create(TMFQS_FP64, 0, &h_));
			++g_created;
		}
		GpuStateBackend(const GpuStateBackend &) = delete;
		GpuStateBackend &operator=(const GpuStateBackend &) = delete;
		~GpuStateBackend() override { tmfqs_gpu_destroy(h_); }

		std::unique_ptr<IStateBackend> clone() const override {
			tmfqs_gpu_state *c = nullptr;
			check(tmfqs_gpu_clone(h_, &c));
			++g_created;
			return std::unique_ptr<IStateBackend>(new GpuStateBackend(c, n_));
		}
		void initZero(unsigned int n) override {
			check(tmfqs_gpu_init_zero(h_, n));
			n_ = n;
		}
		void initBasis(unsigned int n, StateIndex s, Amplitude a) override {
			check(tmfqs_gpu_init_basis(h_, n, s, a.real, a.imag));
			n_ = n;
		}
		void initUniformSuperposition(unsigned int n, const BasisStateList &states) override {
			check(tmfqs_gpu_init_uniform(h_, n, states.values().data(), states.size()));
			n_ = n;
		}
		void loadAmplitudes(unsigned int n, AmplitudesVector amps) override {
			if(amps.size() != checkedAmplitudeElementCount(n))
				throw std::invalid_argument("GpuStateBackend::loadAmplitudes size mismatch");
			check(tmfqs_gpu_load(h_, n, amps.data()));
			n_ = n;
		}
		void exportAmplitudes(AmplitudesVector &out) const override {
			out.resize(checkedAmplitudeElementCount(n_));
			check(tmfqs_gpu_export(h_, out.data()));
		}
		void forEachAmplitudeChunk(const AmplitudeChunkVisitor &visitor) const override {
			const StateIndex N = StateIndex{1} << n_;
			std::vector<double> buf(2 * std::min<StateIndex>(N, kChunkStates));
			for(StateIndex base = 0; base < N; base += kChunkStates) {
				const StateIndex cnt = std::min<StateIndex>(kChunkStates, N - base);
				check(tmfqs_gpu_export_chunk(h_, base, buf.data(), cnt));
				visitor(base, buf.data(), static_cast<size_t>(2 * cnt));
			}
		}
		Amplitude amplitude(StateIndex s) const override {
			Amplitude a{};
			check(tmfqs_gpu_get_amp(h_, s, &a.real, &a.imag));
			return a;
		}
		void setAmplitude(StateIndex s, Amplitude a) override { check(tmfqs_gpu_set_amp(h_, s, a.real, a.imag)); }
		double probability(StateIndex s) const override {
			const Amplitude a = amplitude(s);
			return a.real * a.real + a.imag * a.imag;
		}
		double totalProbability() const override {
			double p = 0.0;
			check(tmfqs_gpu_total_probability(h_, &p));
			return p;
		}
		StateIndex sampleMeasurement(double rnd) const override {
			uint64_t s = 0;
			check(tmfqs_gpu_sample(h_, rnd, &s));
			return s;
		}
		void printNonZeroStates(std::ostream &os, double eps) const override {
			forEachAmplitudeChunk([&](StateIndex base, const double *d, size_t elems) {
				for(size_t i = 0; i + 1 < elems; i += 2)
					if(std::abs(d[i]) > eps || std::abs(d[i + 1]) > eps)
						os << (base + i / 2) << ": " << d[i] << " + " << d[i + 1] << "i\n";
			});
		}
		void phaseFlipBasisState(StateIndex s) override { check(tmfqs_gpu_phase_flip(h_, s)); }
		void inversionAboutMean() override { check(tmfqs_gpu_inversion(h_)); }
		void inversionAboutMean(Amplitude m) override { check(tmfqs_gpu_inversion_mean(h_, m.real, m.imag)); }
		void applyAffineTransform(Amplitude s, Amplitude b) override {
			check(tmfqs_gpu_affine(h_, s.real, s.imag, b.real, b.imag));
		}
		void applyHadamard(QubitIndex q) override { check(tmfqs_gpu_h(h_, q)); }
		void applyPauliX(QubitIndex q) override { check(tmfqs_gpu_x(h_, q)); }
		void applyControlledPhaseShift(QubitIndex c, QubitIndex t, double th) override {
			check(tmfqs_gpu_cphase(h_, c, t, th));
		}
		void applyControlledNot(QubitIndex c, QubitIndex t) override { check(tmfqs_gpu_cnot(h_, c, t)); }
		void applyGate(const QuantumGate &g, const QubitList &q) override {
			const unsigned dim = g.dimension();
			std::vector<double> m;
			m.reserve(2 * size_t(dim) * dim);
			for(unsigned r = 0; r < dim; ++r)
				for(unsigned c = 0; c < dim; ++c) {
					m.push_back(g[r][c].real);
					m.push_back(g[r][c].imag);
				}
			check(tmfqs_gpu_gate(h_, m.data(), q.values().data(), static_cast<unsigned>(q.size())));
		}
		void endOperationBatch() override { check(tmfqs_gpu_sync(h_)); }

	private:
		GpuStateBackend(tmfqs_gpu_state *h, unsigned n) : h_(h), n_(n) {}

		tmfqs_gpu_state *h_ = nullptr;
		unsigned n_ = 0;
};

}  // namespace

std::unique_ptr<IStateBackend> createGpuStateBackend(const RegisterConfig &) {
	return std::unique_ptr<IStateBackend>(new GpuStateBackend());
}

bool isGpuStateBackendAvailable() {
	tmfqs_gpu_state *h = nullptr;
	if(tmfqs_gpu_create(TMFQS_FP64, 0, &h) != TMFQS_OK) return false;
	tmfqs_gpu_destroy(h);
	return true;
}

bool denseRedirectedToGpu() {
	const char *v = std::getenv("TMFQS_DENSE_BACKEND");
	return v && std::strcmp(v, "gpu") == 0;
}

}  // namespace tmfqs
