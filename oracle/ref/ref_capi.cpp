// C wrapper over the reference TMFQS public API (test infrastructure).
//
// Compiled together with the reference's own sources by oracle/ref/Makefile
// with -Dtmfqs=tmfqs_ref, so every tmfqs:: name below resolves to the
// reference library's renamed namespace and cannot collide with this
// repository's own C++ host library.  Only the functions marked REF_API are
// exported.  Everything here calls the reference through its public API
// (QuantumRegister, circuit::Circuit, sim::Simulator, state::QuantumState,
// experiment::compareStates) with the Dense strategy -- the stock CPU path.
#include "tmfqsfs.h"

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

thread_local std::string g_error;

// Same layout as or_op in oracle/tmfqs_oracle.h.
struct RefOp {
	int kind;
	unsigned q0;
	unsigned q1;
	double theta;
	std::uint64_t state;
	int materialized;
	const double *matrix;
	const unsigned *qubits;
	unsigned k;
};

enum { kH = 0, kX = 1, kCnot = 2, kCphase = 3, kSwap = 4, kGate = 5, kFlip = 6, kInv = 7 };

template <typename F>
int guarded(F &&fn) {
	try {
		fn();
		return 0;
	} catch(const std::out_of_range &e) {
		g_error = e.what();
		return 1;
	} catch(const std::invalid_argument &e) {
		g_error = e.what();
		return 2;
	} catch(const std::logic_error &e) {
		g_error = e.what();
		return 3;
	} catch(const std::runtime_error &e) {
		g_error = e.what();
		return 4;
	} catch(const std::exception &e) {
		g_error = e.what();
		return 5;
	}
}

class FixedSource final : public tmfqs::IRandomSource {
	public:
		explicit FixedSource(double v) : v_(v) {}
		double nextUnitDouble() override { return v_; }
	private:
		double v_;
};

tmfqs::RegisterConfig denseConfig() {
	tmfqs::RegisterConfig cfg;
	cfg.strategy = tmfqs::StorageStrategyKind::Dense;
	return cfg;
}

tmfqs::QuantumGate gateFrom(const RefOp &op) {
	const unsigned dim = 1u << op.k;
	tmfqs::QuantumGate g(dim);
	for(unsigned r = 0; r < dim; ++r) {
		for(unsigned c = 0; c < dim; ++c) {
			g[r][c].real = op.matrix[2u * (r * dim + c)];
			g[r][c].imag = op.matrix[2u * (r * dim + c) + 1u];
		}
	}
	return g;
}

tmfqs::circuit::Circuit circuitFrom(unsigned n, const RefOp *ops, size_t nops) {
	tmfqs::circuit::Circuit c(n);
	for(size_t i = 0; i < nops; ++i) {
		const RefOp &op = ops[i];
		switch(op.kind) {
			case kH: c.h(op.q0); break;
			case kX: c.x(op.q0); break;
			case kCnot: c.cx(op.q0, op.q1); break;
			case kCphase: c.controlledPhase(op.q0, op.q1, op.theta); break;
			case kSwap: c.swap(op.q0, op.q1); break;
			case kGate: {
				std::vector<tmfqs::QubitIndex> q(op.qubits, op.qubits + op.k);
				c.gate(gateFrom(op), tmfqs::QubitList(std::move(q)));
				break;
			}
			case kFlip: c.phaseFlip(op.state); break;
			case kInv: c.inversionAboutMean(op.materialized != 0); break;
			default: throw std::invalid_argument("unknown op kind");
		}
	}
	return c;
}

void applyOp(tmfqs::QuantumRegister &reg, const RefOp &op) {
	switch(op.kind) {
		case kH: reg.applyHadamard(op.q0); break;
		case kX: reg.applyPauliX(op.q0); break;
		case kCnot: reg.applyControlledNot(op.q0, op.q1); break;
		case kCphase: reg.applyControlledPhaseShift(op.q0, op.q1, op.theta); break;
		case kSwap: reg.applySwap(op.q0, op.q1); break;
		case kGate: {
			std::vector<tmfqs::QubitIndex> q(op.qubits, op.qubits + op.k);
			reg.applyGate(gateFrom(op), tmfqs::QubitList(std::move(q)));
			break;
		}
		case kFlip: reg.applyPhaseFlipBasisState(op.state); break;
		case kInv:
			if(op.materialized) reg.applyInversionAboutMeanMaterialized();
			else reg.applyInversionAboutMean();
			break;
		default: throw std::invalid_argument("unknown op kind");
	}
}

void opsFrom(const tmfqs::circuit::Circuit &c, RefOp *out, size_t cap, size_t *count) {
	const auto &ops = c.operations();
	*count = ops.size();
	if(out == nullptr) return;
	if(cap < ops.size()) throw std::invalid_argument("op buffer too small");
	for(size_t i = 0; i < ops.size(); ++i) {
		RefOp r{};
		std::visit(
			[&](const auto &op) {
				using Op = std::decay_t<decltype(op)>;
				if constexpr(std::is_same<Op, tmfqs::circuit::Hadamard>::value) { r.kind = kH; r.q0 = op.target; }
				else if constexpr(std::is_same<Op, tmfqs::circuit::PauliX>::value) { r.kind = kX; r.q0 = op.target; }
				else if constexpr(std::is_same<Op, tmfqs::circuit::ControlledNot>::value) { r.kind = kCnot; r.q0 = op.control; r.q1 = op.target; }
				else if constexpr(std::is_same<Op, tmfqs::circuit::ControlledPhaseShift>::value) { r.kind = kCphase; r.q0 = op.control; r.q1 = op.target; r.theta = op.theta; }
				else if constexpr(std::is_same<Op, tmfqs::circuit::Swap>::value) { r.kind = kSwap; r.q0 = op.first; r.q1 = op.second; }
				else if constexpr(std::is_same<Op, tmfqs::circuit::MatrixGate>::value) { r.kind = kGate; r.k = static_cast<unsigned>(op.targets.size()); }
				else if constexpr(std::is_same<Op, tmfqs::circuit::PhaseFlipBasisState>::value) { r.kind = kFlip; r.state = op.state; }
				else if constexpr(std::is_same<Op, tmfqs::circuit::InversionAboutMean>::value) { r.kind = kInv; r.materialized = op.materialized ? 1 : 0; }
			},
			ops[i]);
		out[i] = r;
	}
}

} // namespace

REF_API const char *ref_last_error() { return g_error.c_str(); }

REF_API void *ref_reg_new_basis(unsigned n, std::uint64_t s) {
	tmfqs::QuantumRegister *reg = nullptr;
	if(guarded([&] { reg = new tmfqs::QuantumRegister(n, s, denseConfig()); }) != 0) return nullptr;
	return reg;
}

REF_API void *ref_reg_new_amps(unsigned n, const double *amps) {
	tmfqs::QuantumRegister *reg = nullptr;
	const size_t len = static_cast<size_t>(2) << n;
	if(guarded([&] { reg = new tmfqs::QuantumRegister(n, tmfqs::AmplitudesVector(amps, amps + len), denseConfig()); }) != 0) return nullptr;
	return reg;
}

REF_API void *ref_reg_copy(void *h) {
	tmfqs::QuantumRegister *reg = nullptr;
	if(guarded([&] { reg = new tmfqs::QuantumRegister(*static_cast<tmfqs::QuantumRegister *>(h)); }) != 0) return nullptr;
	return reg;
}

REF_API void ref_reg_free(void *h) { delete static_cast<tmfqs::QuantumRegister *>(h); }

REF_API int ref_reg_init_uniform(void *h, const std::uint64_t *states, size_t count) {
	return guarded([&] {
		std::vector<tmfqs::StateIndex> v(states, states + count);
		static_cast<tmfqs::QuantumRegister *>(h)->initUniformSuperposition(tmfqs::BasisStateList(std::move(v)));
	});
}

REF_API int ref_reg_apply(void *h, const RefOp *op) {
	return guarded([&] { applyOp(*static_cast<tmfqs::QuantumRegister *>(h), *op); });
}

REF_API int ref_reg_run(void *h, const RefOp *ops, size_t nops) {
	return guarded([&] {
		auto &reg = *static_cast<tmfqs::QuantumRegister *>(h);
		for(size_t i = 0; i < nops; ++i) applyOp(reg, ops[i]);
	});
}

REF_API int ref_reg_inversion_mean(void *h, double re, double im, int materialized) {
	return guarded([&] {
		auto &reg = *static_cast<tmfqs::QuantumRegister *>(h);
		if(materialized) reg.applyInversionAboutMeanMaterialized({re, im});
		else reg.applyInversionAboutMean({re, im});
	});
}

REF_API int ref_reg_set_amplitude(void *h, std::uint64_t s, double re, double im) {
	return guarded([&] { static_cast<tmfqs::QuantumRegister *>(h)->setAmplitude(s, {re, im}); });
}

REF_API int ref_reg_amplitude(void *h, std::uint64_t s, double *re, double *im) {
	return guarded([&] {
		const tmfqs::Amplitude a = static_cast<tmfqs::QuantumRegister *>(h)->amplitude(s);
		*re = a.real;
		*im = a.imag;
	});
}

REF_API int ref_reg_export(void *h, double *out) {
	return guarded([&] {
		const tmfqs::AmplitudesVector v = static_cast<tmfqs::QuantumRegister *>(h)->amplitudes();
		std::memcpy(out, v.data(), v.size() * sizeof(double));
	});
}

REF_API int ref_reg_total_probability(void *h, double *out) {
	return guarded([&] { *out = static_cast<tmfqs::QuantumRegister *>(h)->totalProbability(); });
}

REF_API int ref_reg_measure_fixed(void *h, double rnd, std::uint64_t *out) {
	return guarded([&] {
		FixedSource src(rnd);
		*out = static_cast<tmfqs::QuantumRegister *>(h)->measure(src);
	});
}

REF_API int ref_reg_measure_seed(void *h, std::uint32_t seed, std::uint64_t *out) {
	return guarded([&] {
		tmfqs::Mt19937RandomSource src(seed);
		*out = static_cast<tmfqs::QuantumRegister *>(h)->measure(src);
	});
}

// Input state handle: state::QuantumState built by the reference's own
// factories.  kind 0 = basis(n, basis); 1 = fromAmplitudes(n, amps);
// 2 = uniformSubset(n, states); 3 = randomPhase(n, seed).
REF_API void *ref_state_new(unsigned n, int kind, std::uint64_t basis, const double *amps,
                            const std::uint64_t *states, size_t nstates, std::uint32_t seed) {
	tmfqs::state::QuantumState *st = nullptr;
	const int rc = guarded([&] {
		switch(kind) {
			case 0: st = new tmfqs::state::QuantumState(tmfqs::state::QuantumState::basis(n, basis)); break;
			case 1: {
				const size_t len = static_cast<size_t>(2) << n;
				st = new tmfqs::state::QuantumState(
					tmfqs::state::QuantumState::fromAmplitudes(n, tmfqs::AmplitudesVector(amps, amps + len)));
				break;
			}
			case 2: {
				std::vector<tmfqs::StateIndex> v(states, states + nstates);
				st = new tmfqs::state::QuantumState(tmfqs::state::QuantumState::uniformSubset(n, tmfqs::BasisStateList(std::move(v))));
				break;
			}
			case 3: st = new tmfqs::state::QuantumState(tmfqs::state::QuantumState::randomPhase(n, seed)); break;
			default: throw std::invalid_argument("unknown state kind");
		}
	});
	return rc == 0 ? st : nullptr;
}

REF_API void ref_state_free(void *h) { delete static_cast<tmfqs::state::QuantumState *>(h); }

REF_API int ref_state_export(void *h, double *out) {
	return guarded([&] {
		const tmfqs::AmplitudesVector v = static_cast<tmfqs::state::QuantumState *>(h)->amplitudes();
		std::memcpy(out, v.data(), v.size() * sizeof(double));
	});
}

// sim::Simulator(Dense).run(circuit(ops), *state).  Optional outputs: the
// final amplitudes, total probability, measure() with Mt19937RandomSource(seed)
// and the reference's own executionSeconds.
REF_API int ref_sim_run(void *state, const RefOp *ops, size_t nops, double *out_amps, double *total_prob,
                        int do_measure, std::uint32_t seed, std::uint64_t *measured, double *exec_seconds) {
	return guarded([&] {
		auto &st = *static_cast<tmfqs::state::QuantumState *>(state);
		const tmfqs::circuit::Circuit circuit = circuitFrom(st.qubitCount(), ops, nops);
		tmfqs::sim::ExecutionConfig exec;
		exec.backend = denseConfig();
		const tmfqs::sim::RunResult run = tmfqs::sim::Simulator(exec).run(circuit, st);
		if(exec_seconds) *exec_seconds = run.report.executionSeconds;
		if(out_amps) {
			const tmfqs::AmplitudesVector v = run.state.amplitudes();
			std::memcpy(out_amps, v.data(), v.size() * sizeof(double));
		}
		if(total_prob) *total_prob = run.state.totalProbability();
		if(do_measure) {
			tmfqs::Mt19937RandomSource src(seed);
			*measured = run.state.measure(src);
		}
	});
}

REF_API int ref_build_qft(unsigned n, RefOp *ops, size_t cap, size_t *count) {
	return guarded([&] { opsFrom(tmfqs::circuit::makeQft(n), ops, cap, count); });
}

REF_API int ref_build_grover(unsigned n, const std::uint64_t *marked, size_t k, int materialized, RefOp *ops,
                             size_t cap, size_t *count) {
	return guarded([&] {
		tmfqs::circuit::GroverCircuitOptions o;
		o.markedStates = tmfqs::BasisStateList(std::vector<tmfqs::StateIndex>(marked, marked + k));
		o.materializedDiffusion = materialized != 0;
		opsFrom(tmfqs::circuit::makeGrover(n, std::move(o)), ops, cap, count);
	});
}

REF_API unsigned ref_grover_iterations(std::uint64_t states, size_t marked) {
	unsigned it = 0;
	(void)guarded([&] { it = tmfqs::circuit::groverIterationCount(states, marked); });
	return it;
}

REF_API int ref_mt_unit(std::uint32_t seed, size_t k, double *out) {
	return guarded([&] {
		tmfqs::Mt19937RandomSource src(seed);
		for(size_t i = 0; i < k; ++i) out[i] = src.nextUnitDouble();
	});
}

// experiment::compareStates between two interleaved amplitude vectors.
// All of experiment::compareStates: out = {maxAbsAmplitudeError,
// maxAbsComponentError, rmseAmplitude, relL2, maxAbsProbabilityError,
// totalProbabilityDiff}.
REF_API int ref_compare_full(unsigned n, const double *ref_amps, const double *got_amps, double *out,
                             std::uint64_t *worst, int *bitwise) {
	return guarded([&] {
		const size_t len = static_cast<size_t>(2) << n;
		tmfqs::state::StateValidation v;
		v.normalization = tmfqs::state::NormalizationPolicy::AllowUnnormalized;
		const auto a = tmfqs::state::QuantumState::fromAmplitudes(n, tmfqs::AmplitudesVector(ref_amps, ref_amps + len), v);
		const auto b = tmfqs::state::QuantumState::fromAmplitudes(n, tmfqs::AmplitudesVector(got_amps, got_amps + len), v);
		const tmfqs::experiment::StateComparison c = tmfqs::experiment::compareStates(a, b);
		out[0] = c.maxAbsAmplitudeError;
		out[1] = c.maxAbsComponentError;
		out[2] = c.rmseAmplitude;
		out[3] = c.relL2;
		out[4] = c.maxAbsProbabilityError;
		out[5] = c.totalProbabilityDiff;
		*worst = c.worstState;
		*bitwise = c.bitwiseEqual ? 1 : 0;
	});
}

REF_API int ref_compare(unsigned n, const double *ref_amps, const double *got_amps, double *rel_l2,
                        double *max_abs, std::uint64_t *worst, int *bitwise) {
	return guarded([&] {
		const size_t len = static_cast<size_t>(2) << n;
		tmfqs::state::StateValidation v;
		v.normalization = tmfqs::state::NormalizationPolicy::AllowUnnormalized;
		const auto a = tmfqs::state::QuantumState::fromAmplitudes(n, tmfqs::AmplitudesVector(ref_amps, ref_amps + len), v);
		const auto b = tmfqs::state::QuantumState::fromAmplitudes(n, tmfqs::AmplitudesVector(got_amps, got_amps + len), v);
		const tmfqs::experiment::StateComparison c = tmfqs::experiment::compareStates(a, b);
		*rel_l2 = c.relL2;
		*max_abs = c.maxAbsAmplitudeError;
		*worst = c.worstState;
		*bitwise = c.bitwiseEqual ? 1 : 0;
	});
}
