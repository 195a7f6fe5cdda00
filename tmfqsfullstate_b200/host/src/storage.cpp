// Strategy registry and the B200 backend (GpuStateBackend) over the C ABI.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <ostream>
#include <stdexcept>
#include <string>

#include "tmfqs/core/state_space.h"
#include "tmfqs/storage/factory/state_backend_factory.h"
#include "tmfqs/storage/factory/storage_strategy_registry.h"
#include "tmfqs/storage/gpu/gpu_state_backend.h"
#include "tmfqs_b200.h"

namespace tmfqs {
namespace {

// Maps a C-ABI status to the reference's exception classes.
void check(int rc) {
	if(rc == TMFQS_OK) return;
	const std::string msg = tmfqs_gpu_last_error();
	switch(rc) {
		case TMFQS_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
		case TMFQS_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
		case TMFQS_ERR_LOGIC: throw std::logic_error(msg);
		default: throw std::runtime_error(msg);
	}
}

constexpr uint64_t kChunkStates = uint64_t(1) << 22;  // 64 MiB of complex128 per visitor call

class GpuStateBackend final : public IStateBackend {
	public:
		explicit GpuStateBackend(const GpuConfig &cfg) : cfg_(cfg) {
			check(tmfqs_gpu_create(cfg.precision == GpuPrecision::Fp64 ? TMFQS_FP64 : TMFQS_FP32, cfg.deviceOrdinal, &h_));
			check(tmfqs_gpu_set_option(h_, TMFQS_OPT_EXACT, cfg.exact ? 1 : 0));
			check(tmfqs_gpu_set_option(h_, TMFQS_OPT_FUSION, cfg.fusion ? 1 : 0));
		}
		GpuStateBackend(const GpuStateBackend &) = delete;
		GpuStateBackend &operator=(const GpuStateBackend &) = delete;
		~GpuStateBackend() override { tmfqs_gpu_destroy(h_); }

		std::unique_ptr<IStateBackend> clone() const override {
			tmfqs_gpu_state *c = nullptr;
			check(tmfqs_gpu_clone(h_, &c));
			return std::unique_ptr<IStateBackend>(new GpuStateBackend(cfg_, c, n_));
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
			if(amps.size() != checkedAmplitudeElementCount(n)) throw std::invalid_argument("GpuStateBackend: amplitudes size mismatch");
			check(tmfqs_gpu_load(h_, n, amps.data()));
			n_ = n;
		}
		void exportAmplitudes(AmplitudesVector &out) const override {
			out.resize(checkedAmplitudeElementCount(n_));
			check(tmfqs_gpu_export(h_, out.data()));
		}
		void forEachAmplitudeChunk(const AmplitudeChunkVisitor &visitor) const override {
			const StateIndex N = StateIndex{1} << n_;
			std::vector<double> buf(2 * std::min<uint64_t>(N, kChunkStates));
			for(StateIndex base = 0; base < N; base += kChunkStates) {
				const uint64_t cnt = std::min<uint64_t>(kChunkStates, N - base);
				check(tmfqs_gpu_export_chunk(h_, base, buf.data(), cnt));
				visitor(base, buf.data(), 2 * cnt);
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
			if(eps < 0.0) throw std::invalid_argument("GpuStateBackend::printNonZeroStates epsilon must be non-negative");
			forEachAmplitudeChunk([&](StateIndex base, const double *d, size_t elems) {
				for(size_t i = 0; i + 1 < elems; i += 2)
					if(std::abs(d[i]) > eps || std::abs(d[i + 1]) > eps)
						os << (base + i / 2) << ": " << d[i] << " + " << d[i + 1] << "i\n";
			});
		}
		void phaseFlipBasisState(StateIndex s) override { check(tmfqs_gpu_phase_flip(h_, s)); }
		void inversionAboutMean() override { check(tmfqs_gpu_inversion(h_)); }
		void inversionAboutMean(Amplitude m) override { check(tmfqs_gpu_inversion_mean(h_, m.real, m.imag)); }
		void applyAffineTransform(Amplitude s, Amplitude b) override { check(tmfqs_gpu_affine(h_, s.real, s.imag, b.real, b.imag)); }
		void applyHadamard(QubitIndex q) override { check(tmfqs_gpu_h(h_, q)); }
		void applyPauliX(QubitIndex q) override { check(tmfqs_gpu_x(h_, q)); }
		void applyControlledPhaseShift(QubitIndex c, QubitIndex t, double th) override { check(tmfqs_gpu_cphase(h_, c, t, th)); }
		void applyControlledNot(QubitIndex c, QubitIndex t) override { check(tmfqs_gpu_cnot(h_, c, t)); }
		void applyGate(const QuantumGate &g, const QubitList &q) override {
			const std::vector<double> m = flatten(g);
			check(tmfqs_gpu_gate(h_, m.data(), q.values().data(), static_cast<unsigned>(q.size())));
		}
		void endOperationBatch() override { check(tmfqs_gpu_sync(h_)); }

		bool applyOperationRun(const std::vector<BackendOp> &ops) override {
			std::vector<tmfqs_op> c(ops.size());
			std::vector<std::vector<double>> mats;
			mats.reserve(ops.size());
			for(size_t i = 0; i < ops.size(); ++i) {
				const BackendOp &o = ops[i];
				tmfqs_op &d = c[i];
				std::memset(&d, 0, sizeof(d));
				d.q0 = o.q0;
				d.q1 = o.q1;
				switch(o.kind) {
					case BackendOp::Kind::Hadamard: d.kind = TMFQS_OP_H; break;
					case BackendOp::Kind::PauliX: d.kind = TMFQS_OP_X; break;
					case BackendOp::Kind::ControlledNot: d.kind = TMFQS_OP_CNOT; break;
					case BackendOp::Kind::ControlledPhaseShift: d.kind = TMFQS_OP_CPHASE; d.theta = o.theta; break;
					case BackendOp::Kind::Swap: d.kind = TMFQS_OP_SWAP; break;
					case BackendOp::Kind::PhaseFlip: d.kind = TMFQS_OP_PHASE_FLIP; d.state = o.state; break;
					case BackendOp::Kind::MatrixGate:
						d.kind = TMFQS_OP_GATE;
						mats.push_back(flatten(*o.gate));
						d.matrix = mats.back().data();
						d.qubits = o.targets->values().data();
						d.k = static_cast<unsigned>(o.targets->size());
						break;
				}
			}
			check(tmfqs_gpu_apply_ops(h_, c.data(), c.size()));
			return true;
		}
		bool logicalAmplitudeSum(const AffineOverlay *ov, Amplitude &out) const override {
			if(ov) check(tmfqs_gpu_overlay_sum(h_, ov->scale.real, ov->scale.imag, ov->bias.real, ov->bias.imag, &out.real, &out.imag));
			else check(tmfqs_gpu_amplitude_sum(h_, &out.real, &out.imag));
			return true;
		}
		bool logicalTotalProbability(const AffineOverlay *ov, double &out) const override {
			if(ov) check(tmfqs_gpu_overlay_total_probability(h_, ov->scale.real, ov->scale.imag, ov->bias.real, ov->bias.imag, &out));
			else check(tmfqs_gpu_total_probability(h_, &out));
			return true;
		}
		bool logicalSample(const AffineOverlay *ov, double rnd, StateIndex &out) const override {
			uint64_t s = 0;
			if(ov) check(tmfqs_gpu_overlay_sample(h_, ov->scale.real, ov->scale.imag, ov->bias.real, ov->bias.imag, rnd, &s));
			else check(tmfqs_gpu_sample(h_, rnd, &s));
			out = s;
			return true;
		}
		bool runGroverIterations(RegisterSideState &side, const std::vector<StateIndex> &marked, uint64_t iterations,
		                         bool materialized) override {
			tmfqs_register_view v{side.hasSum ? 1 : 0, side.sum.real, side.sum.imag, side.overlayActive ? 1 : 0,
			                      side.overlay.scale.real, side.overlay.scale.imag, side.overlay.bias.real, side.overlay.bias.imag};
			check(tmfqs_gpu_grover_run(h_, &v, marked.data(), marked.size(), iterations, materialized ? 1 : 0));
			side.hasSum = v.has_sum != 0;
			side.sum = {v.sum_re, v.sum_im};
			side.overlayActive = v.overlay != 0;
			side.overlay.scale = {v.scale_re, v.scale_im};
			side.overlay.bias = {v.bias_re, v.bias_im};
			return true;
		}

		bool beginPassTrace() override {
			check(tmfqs_gpu_sync(h_));
			check(tmfqs_gpu_reset_stats(h_));
			check(tmfqs_gpu_set_option(h_, TMFQS_OPT_KERNEL_TIMING, 1));
			return true;
		}
		uint64_t markPassSegment() override {
			uint64_t seg = 0;
			check(tmfqs_gpu_pass_mark(h_, &seg));
			return seg;
		}
		bool endPassTrace(std::vector<BackendPassTrace> &out) override {
			static const char *kKinds[] = {"fused", "permute", "gate", "reduce", "grover", "adjoint"};
			size_t n = 0;
			check(tmfqs_gpu_pass_log(h_, nullptr, 0, &n));
			std::vector<tmfqs_pass_record> recs(n);
			check(tmfqs_gpu_pass_log(h_, recs.data(), n, &n));
			check(tmfqs_gpu_set_option(h_, TMFQS_OPT_KERNEL_TIMING, 0));
			out.clear();
			for(const tmfqs_pass_record &r : recs) {
				BackendPassTrace t;
				t.kind = (r.kind >= 0 && r.kind < 6) ? kKinds[r.kind] : "pass";
				t.segment = r.segment;
				t.firstOp = r.first_op;
				t.opCount = r.op_count;
				t.seconds = r.ms * 1e-3;
				out.push_back(t);
			}
			return true;
		}
		bool compareWith(const IStateBackend &candidate, BackendComparison &out) const override {
			const auto *o = dynamic_cast<const GpuStateBackend *>(&candidate);
			if(!o) return false;
			tmfqs_state_comparison c{};
			check(tmfqs_gpu_compare(h_, o->h_, &c));
			out.bitwiseEqual = c.bitwise_equal != 0;
			out.maxAbsAmplitudeError = c.max_abs_amplitude_error;
			out.maxAbsComponentError = c.max_abs_component_error;
			out.rmseAmplitude = c.rmse_amplitude;
			out.relL2 = c.rel_l2;
			out.maxAbsProbabilityError = c.max_abs_probability_error;
			out.totalProbabilityDiff = c.total_probability_diff;
			out.worstState = c.worst_state;
			return true;
		}

	private:
		GpuStateBackend(const GpuConfig &cfg, tmfqs_gpu_state *h, unsigned n) : h_(h), n_(n), cfg_(cfg) {}

		static std::vector<double> flatten(const QuantumGate &g) {
			std::vector<double> m;
			m.reserve(2 * g.entries().size());
			for(const Amplitude &a : g.entries()) {
				m.push_back(a.real);
				m.push_back(a.imag);
			}
			return m;
		}

		tmfqs_gpu_state *h_ = nullptr;
		unsigned n_ = 0;
		GpuConfig cfg_;
};

std::unique_ptr<IStateBackend> unavailable(const char *name) {
	throw std::runtime_error(std::string(name) + " backend requested but unavailable in this build");
}

}  // namespace

std::unique_ptr<IStateBackend> createGpuStateBackend(const RegisterConfig &cfg) {
	return std::make_unique<GpuStateBackend>(cfg.gpu);
}

bool isGpuStateBackendAvailable() {
	static std::once_flag once;
	static bool available = false;
	std::call_once(once, [] {
		tmfqs_gpu_state *h = nullptr;
		available = tmfqs_gpu_create(TMFQS_FP64, 0, &h) == TMFQS_OK;
		if(h) tmfqs_gpu_destroy(h);
	});
	return available;
}

// Auto and every explicit request resolve to the device backend in this
// build; the CPU backends of the reference are not part of it.
StorageStrategyKind StorageStrategyRegistry::resolve(unsigned int numQubits, const RegisterConfig &cfg) {
	(void)checkedAmplitudeElementCount(numQubits);
	return cfg.strategy == StorageStrategyKind::Auto ? StorageStrategyKind::Gpu : cfg.strategy;
}

bool StorageStrategyRegistry::isAvailable(StorageStrategyKind kind) {
	switch(kind) {
		case StorageStrategyKind::Gpu: return isGpuStateBackendAvailable();
		case StorageStrategyKind::Auto: return isGpuStateBackendAvailable();
		default: return false;
	}
}

std::vector<std::string> StorageStrategyRegistry::listAvailable() {
	std::vector<std::string> names;
	if(isGpuStateBackendAvailable()) {
		names.push_back("gpu");
		names.push_back("auto");
	}
	return names;
}

std::string StorageStrategyRegistry::toString(StorageStrategyKind kind) {
	switch(kind) {
		case StorageStrategyKind::Dense: return "dense";
		case StorageStrategyKind::Blosc: return "blosc";
		case StorageStrategyKind::Zfp: return "zfp";
		case StorageStrategyKind::Auto: return "auto";
		case StorageStrategyKind::Gpu: return "gpu";
	}
	return "unknown";
}

RegisterConfig StorageStrategyRegistry::tuneConfig(unsigned int, const RegisterConfig &cfg, StorageStrategyKind) { return cfg; }

BackendSelection StorageStrategyRegistry::createSelection(unsigned int numQubits, const RegisterConfig &cfg) {
	BackendSelection sel;
	sel.strategy = resolve(numQubits, cfg);
	sel.config = tuneConfig(numQubits, cfg, sel.strategy);
	sel.config.strategy = sel.strategy;
	switch(sel.strategy) {
		case StorageStrategyKind::Gpu: sel.backend = createGpuStateBackend(sel.config); break;
		case StorageStrategyKind::Dense: sel.backend = unavailable("Dense"); break;
		case StorageStrategyKind::Blosc: sel.backend = unavailable("Blosc"); break;
		case StorageStrategyKind::Zfp: sel.backend = unavailable("Zfp"); break;
		case StorageStrategyKind::Auto: throw std::runtime_error("StorageStrategyRegistry internal error: unresolved auto strategy");
	}
	return sel;
}

std::unique_ptr<IStateBackend> StateBackendFactory::create(unsigned int n, const RegisterConfig &cfg) { return createSelection(n, cfg).backend; }
BackendSelection StateBackendFactory::createSelection(unsigned int n, const RegisterConfig &cfg) {
	return StorageStrategyRegistry::createSelection(n, cfg);
}

}  // namespace tmfqs
