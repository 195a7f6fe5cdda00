// C++ checks of the host API with the gpu strategy: the cases of the
// reference's integration tests (tests/integration/circuit/test_circuit.cpp,
// register/test_register_validation.cpp, storage/test_storage_parity.cpp)
// restated for this build, plus batched-versus-per-operation equivalence.
// Run by tests/test_gpu_host.py; prints one line per check and exits non-zero
// on the first failure.
#include <cmath>
#include <cstring>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <vector>
#include <string>
#include <variant>
#include <type_traits>

#include "tmfqsfs.h"
#include "tmfqs_b200.h"

using namespace tmfqs;

namespace {

int g_checks = 0;

void require(bool ok, const char *what, int line) {
	++g_checks;
	if(!ok) {
		std::ostringstream m;
		m << "line " << line << ": " << what;
		throw std::runtime_error(m.str());
	}
}
#define REQUIRE(x) require((x), #x, __LINE__)

template <typename E, typename F>
bool throwsAs(F &&f) {
	try {
		f();
	} catch(const E &) {
		return true;
	} catch(...) {
		return false;
	}
	return false;
}

bool close(double a, double b, double tol = 1e-10) { return std::fabs(a - b) < tol; }

class FixedSource final : public IRandomSource {
	public:
		explicit FixedSource(double v) : v_(v) {}
		double nextUnitDouble() override { return v_; }
	private:
		double v_;
};

StateIndex runGrover(unsigned n, BasisStateList marked, IRandomSource &rng, bool materialized = false) {
	circuit::GroverCircuitOptions o;
	o.markedStates = std::move(marked);
	o.materializedDiffusion = materialized;
	const sim::RunResult r = sim::Simulator().run(circuit::makeGrover(n, std::move(o)), state::QuantumState::basis(n));
	return r.state.measure(rng);
}

const std::vector<double> kFixture = {0.20, 0.10, -0.15, 0.05, 0.30, -0.20, 0.00, 0.10, -0.25, -0.15, 0.18, 0.12, -0.08, 0.04, 0.22, -0.06};

void qftKnownAnswers() {
	for(StateIndex src : {StateIndex(0), StateIndex(5)}) {
		const sim::RunResult r = sim::Simulator().run(circuit::makeQft(3), state::QuantumState::basis(3, src));
		for(StateIndex y = 0; y < 8; ++y) {
			const double ang = 2.0 * kPi * static_cast<double>(src) * static_cast<double>(y) / 8.0;
			const Amplitude a = r.state.amplitude(y);
			REQUIRE(close(a.real, std::cos(ang) / std::sqrt(8.0), 1e-6));
			REQUIRE(close(a.imag, std::sin(ang) / std::sqrt(8.0), 1e-6));
		}
		REQUIRE(close(r.state.totalProbability(), 1.0, 1e-6));
	}
}

void groverSeeds() {
	int ok = 0;
	for(int t = 0; t < 20; ++t) {
		Mt19937RandomSource rng(100u + t);
		ok += runGrover(5, {3}, rng) == 3u;
	}
	REQUIRE(ok > 0);
	for(int t = 0; t < 32; ++t) {
		Mt19937RandomSource rng(200u + t);
		REQUIRE(runGrover(2, {2}, rng) == 2u);
	}
	for(int t = 0; t < 32; ++t) {
		Mt19937RandomSource rng(300u + t);
		const StateIndex s = runGrover(3, {1, 6}, rng);
		REQUIRE(s == 1u || s == 6u);
	}
	for(int t = 0; t < 16; ++t) {
		Mt19937RandomSource rng(400u + t);
		const StateIndex s = runGrover(3, {2, 5, 2}, rng);
		REQUIRE(s == 2u || s == 5u);
	}
	Mt19937RandomSource r500(500u);
	REQUIRE(runGrover(2, {0, 1, 2, 3}, r500) < 4u);
	for(bool mat : {false, true}) {
		Mt19937RandomSource r(mat ? 610u : 600u);
		const StateIndex s = runGrover(3, {1, 6}, r, mat);
		REQUIRE(s == 1u || s == 6u);
	}
	Mt19937RandomSource a(12345u), b(12345u);
	REQUIRE(runGrover(5, {3}, a) == runGrover(5, {3}, b));
	Mt19937RandomSource e(42u);
	REQUIRE(throwsAs<std::invalid_argument>([&] { runGrover(3, {8}, e); }));
	REQUIRE(throwsAs<std::invalid_argument>([&] { runGrover(3, {1, 8}, e); }));
}

void registerPrimitivesAndInversion() {
	QuantumRegister q(2, 0);
	q.applyHadamard(0);
	q.applyHadamard(1);
	const Amplitude before = q.amplitude(3);
	q.applyPhaseFlipBasisState(3);
	const Amplitude after = q.amplitude(3);
	REQUIRE(close(after.real, -before.real, 1e-9) && close(after.imag, -before.imag, 1e-9));
	q.applyInversionAboutMean();
	REQUIRE(close(q.totalProbability(), 1.0, 1e-6));

	QuantumRegister base(3, kFixture), opt(3, kFixture);
	Amplitude mean{0.0, 0.0};
	for(StateIndex s = 0; s < 8; ++s) {
		mean.real += opt.amplitude(s).real;
		mean.imag += opt.amplitude(s).imag;
	}
	mean.real /= 8.0;
	mean.imag /= 8.0;
	base.applyInversionAboutMean();
	opt.applyInversionAboutMean(mean);
	for(StateIndex s = 0; s < 8; ++s) {
		REQUIRE(close(base.amplitude(s).real, opt.amplitude(s).real, 1e-12));
		REQUIRE(close(base.amplitude(s).imag, opt.amplitude(s).imag, 1e-12));
	}
	REQUIRE(close(base.totalProbability(), opt.totalProbability(), 1e-12));

	// Overlay measurement (test_storage_parity.cpp:151-214): the lazy overlay
	// measures the same index as the materialised state.
	QuantumRegister lazy(3, kFixture), mat(3, kFixture);
	lazy.applyInversionAboutMean(mean);
	mat.applyInversionAboutMeanMaterialized(mean);
	const double tp = lazy.totalProbability();
	FixedSource f1(tp * 0.5), f2(tp * 0.5);
	REQUIRE(lazy.measure(f1) == mat.measure(f2));
	REQUIRE(close(mat.totalProbability(), tp, 1e-12));
}

void validation() {
	QuantumRegister q;
	REQUIRE(q.qubitCount() == 0u && q.stateCount() == 1u && q.amplitudeElementCount() == 2u);
	REQUIRE(close(q.amplitude(0).real, 1.0, 1e-12) && close(q.totalProbability(), 1.0, 1e-12));
	Mt19937RandomSource r1(1u);
	REQUIRE(q.measure(r1) == 0u);
	REQUIRE(throwsAs<std::out_of_range>([&] { q.applyHadamard(0); }));

	QuantumRegister q2(2, 0);
	REQUIRE(throwsAs<std::out_of_range>([&] { (void)q2.amplitude(4); }));
	REQUIRE(throwsAs<std::out_of_range>([&] { (void)q2.probability(4); }));
	REQUIRE(throwsAs<std::out_of_range>([&] { q2.applyHadamard(2); }));
	REQUIRE(throwsAs<std::out_of_range>([&] { q2.applyPauliX(2); }));
	REQUIRE(throwsAs<std::out_of_range>([&] { q2.applyControlledNot(0, 2); }));
	REQUIRE(throwsAs<std::invalid_argument>([&] { q2.applyControlledNot(1, 1); }));
	REQUIRE(throwsAs<std::invalid_argument>([&] { q2.applySwap(0, 0); }));
	REQUIRE(throwsAs<std::invalid_argument>([&] { q2.applyGate(QuantumGate::ControlledNot(), QubitList{1, 1}); }));
	REQUIRE(throwsAs<std::out_of_range>([&] { q2.applyGate(QuantumGate::Hadamard(), QubitList{2}); }));
	QuantumRegister q3(3, 0);
	REQUIRE(throwsAs<std::invalid_argument>([&] { q3.initUniformSuperposition(BasisStateList{}); }));
	REQUIRE(throwsAs<std::out_of_range>([&] { q3.initUniformSuperposition(BasisStateList{0, 8}); }));
}

void registryAndCopies() {
	REQUIRE(StorageStrategyRegistry::toString(StorageStrategyKind::Gpu) == "gpu");
	REQUIRE(StorageStrategyRegistry::toString(StorageStrategyKind::Dense) == "dense");
	REQUIRE(StorageStrategyRegistry::isAvailable(StorageStrategyKind::Gpu));
	REQUIRE(!StorageStrategyRegistry::isAvailable(StorageStrategyKind::Dense));
	RegisterConfig cfg;
	cfg.strategy = StorageStrategyKind::Auto;
	QuantumRegister a(3, cfg);
	REQUIRE(a.storageStrategy() == StorageStrategyKind::Gpu);
	for(StorageStrategyKind k : {StorageStrategyKind::Dense, StorageStrategyKind::Blosc, StorageStrategyKind::Zfp}) {
		cfg.strategy = k;
		REQUIRE(throwsAs<std::runtime_error>([&] { (void)StateBackendFactory::create(4, cfg); }));
	}
	QuantumRegister r(5, 0);
	r.applyHadamard(0);
	r.applyHadamard(1);
	r.applyControlledNot(0, 2);
	r.applyControlledPhaseShift(1, 4, kPi / 9.0);
	r.applyPhaseFlipBasisState(9);
	r.applyInversionAboutMean();
	QuantumRegister copy(r);
	QuantumRegister assigned(5, 0);
	assigned = r;
	const Amplitude before = copy.amplitude(9);
	r.applyPhaseFlipBasisState(9);
	REQUIRE(copy.amplitude(9).real == before.real && assigned.amplitude(9).real == before.real);
	REQUIRE(r.amplitude(9).real == -before.real);
}

// The batched Simulator path and the per-operation path give bit-identical
// amplitudes, totals and measurements (gate runs, swaps, matrix gates,
// flips, both diffusion forms).
// The circuit one operation at a time through QuantumRegister's public API
// (no batching hooks): the per-operation path the batched one must equal.
QuantumRegister runPerOperation(const circuit::Circuit &c, const state::QuantumState &in) {
	QuantumRegister reg(in.qubitCount(), in.amplitudes());
	for(const circuit::Operation &operation : c.operations())
		std::visit(
			[&](const auto &op) {
				using Op = std::decay_t<decltype(op)>;
				if constexpr(std::is_same<Op, circuit::Hadamard>::value) reg.applyHadamard(op.target);
				else if constexpr(std::is_same<Op, circuit::PauliX>::value) reg.applyPauliX(op.target);
				else if constexpr(std::is_same<Op, circuit::ControlledNot>::value) reg.applyControlledNot(op.control, op.target);
				else if constexpr(std::is_same<Op, circuit::ControlledPhaseShift>::value)
					reg.applyControlledPhaseShift(op.control, op.target, op.theta);
				else if constexpr(std::is_same<Op, circuit::Swap>::value) reg.applySwap(op.first, op.second);
				else if constexpr(std::is_same<Op, circuit::MatrixGate>::value) reg.applyGate(op.gate, op.targets);
				else if constexpr(std::is_same<Op, circuit::PhaseFlipBasisState>::value) reg.applyPhaseFlipBasisState(op.state);
				else if constexpr(std::is_same<Op, circuit::InversionAboutMean>::value) {
					if(op.materialized) reg.applyInversionAboutMeanMaterialized();
					else reg.applyInversionAboutMean();
				}
			},
			operation);
	return reg;
}

// A traced run keeps the fused passes: one trace per device pass, at its first
// circuit operation, in circuit order, with a positive device time.
void checkPassTraces(const experiment::RunReport &rep, size_t ops) {
	REQUIRE(!rep.operations.empty() && rep.operations.size() <= ops);
	REQUIRE(rep.operations.front().index == 0);
	for(size_t k = 0; k < rep.operations.size(); ++k) {
		const experiment::OperationTrace &t = rep.operations[k];
		REQUIRE(t.index < ops && t.seconds > 0.0 && t.name.find(':') != std::string::npos);
		if(k) REQUIRE(t.index >= rep.operations[k - 1].index);
	}
}

void batchedEqualsPerOperation() {
	for(unsigned n : {3u, 6u, 11u, 14u}) {
		circuit::Circuit c(n);
		c.h(0).h(n - 1).cx(0, n - 1).controlledPhase(n - 1, 0, 0.37).swap(0, n / 2).x(1);
		c.gate(QuantumGate::Ising(0.8), QubitList{1, n - 1});
		c.gate(QuantumGate::Toffoli(), QubitList{n - 1, 0, 1});
		c.phaseFlip(3).inversionAboutMean(true).phaseFlip(1).phaseFlip(5).inversionAboutMean(false);
		c.phaseFlip(1).phaseFlip(5).inversionAboutMean(false).h(2).phaseFlip(2).inversionAboutMean(true);
		circuit::appendQft(c);
		sim::ExecutionConfig traced;
		traced.observability.traceOperations = true;
		const state::QuantumState in = state::QuantumState::randomPhase(n, 7u + n);
		const sim::RunResult a = sim::Simulator().run(c, in);
		const sim::RunResult b = sim::Simulator(traced).run(c, in);
		const QuantumRegister per = runPerOperation(c, in);
		const AmplitudesVector va = a.state.amplitudes(), vb = b.state.amplitudes(), vp = per.amplitudes();
		REQUIRE(va.size() == vb.size() && va.size() == vp.size());
		REQUIRE(std::memcmp(va.data(), vb.data(), va.size() * sizeof(double)) == 0 || va == vb);
		REQUIRE(std::memcmp(va.data(), vp.data(), va.size() * sizeof(double)) == 0 || va == vp);
		REQUIRE(a.state.totalProbability() == b.state.totalProbability());
		REQUIRE(a.state.totalProbability() == per.totalProbability());
		Mt19937RandomSource r1(99u), r2(99u), r3(99u);
		const StateIndex m1 = a.state.measure(r1);
		REQUIRE(m1 == b.state.measure(r2) && m1 == per.measure(r3));
		checkPassTraces(b.report, c.operationCount());
	}
	for(bool mat : {true, false}) {
		circuit::GroverCircuitOptions o;
		o.markedStates = {77, 5, 3000};
		o.materializedDiffusion = mat;
		const circuit::Circuit c = circuit::makeGrover(12, o);
		sim::ExecutionConfig traced;
		traced.observability.traceOperations = true;
		const sim::RunResult a = sim::Simulator().run(c, state::QuantumState::basis(12));
		const sim::RunResult b = sim::Simulator(traced).run(c, state::QuantumState::basis(12));
		const QuantumRegister per = runPerOperation(c, state::QuantumState::basis(12));
		REQUIRE(a.state.amplitudes() == b.state.amplitudes());
		REQUIRE(a.state.amplitudes() == per.amplitudes());
		REQUIRE(a.state.totalProbability() == b.state.totalProbability());
		checkPassTraces(b.report, c.operationCount());
	}
	// QFT-16: the passes of the fused plan (three fused passes and the bit
	// reversal), their names covering the circuit's operations.
	circuit::Circuit q(16);
	circuit::appendQft(q);
	sim::ExecutionConfig traced;
	traced.observability.traceOperations = true;
	const sim::RunResult t = sim::Simulator(traced).run(q, state::QuantumState::randomPhase(16, 5u));
	checkPassTraces(t.report, q.operationCount());
	REQUIRE(t.report.operations.size() <= 8);
	REQUIRE(t.report.operations.back().name == "permute: swap x8");
}

// experiment::compareStates of two device results runs on the device and
// equals the host loop field for field; with a lazy overlay active it falls
// back to the host.
void deviceCompareStates() {
	circuit::Circuit c(14);
	circuit::appendQft(c);
	const state::QuantumState in = state::QuantumState::randomPhase(14, 3u);
	const sim::RunResult a = sim::Simulator().run(c, in);
	sim::ExecutionConfig fast;
	fast.backend.gpu.exact = false;
	const sim::RunResult b = sim::Simulator(fast).run(c, in);
	const experiment::StateComparison dev = experiment::compareStates(a.state, b.state);
	const experiment::StateComparison host = experiment::compareStatesOnHost(a.state, b.state);
	REQUIRE(dev.bitwiseEqual == host.bitwiseEqual && dev.worstState == host.worstState);
	REQUIRE(dev.maxAbsAmplitudeError == host.maxAbsAmplitudeError && dev.maxAbsComponentError == host.maxAbsComponentError);
	REQUIRE(dev.maxAbsProbabilityError == host.maxAbsProbabilityError);
	REQUIRE(dev.relL2 == host.relL2 && dev.rmseAmplitude == host.rmseAmplitude);
	REQUIRE(dev.totalProbabilityDiff == host.totalProbabilityDiff);
	REQUIRE(!dev.bitwiseEqual && dev.relL2 > 0.0 && dev.relL2 < 1e-12);
	const experiment::StateComparison same = experiment::compareStates(a.state, a.state);
	REQUIRE(same.bitwiseEqual && same.relL2 == 0.0);
	circuit::GroverCircuitOptions o;
	o.markedStates = {77};
	const circuit::Circuit g = circuit::makeGrover(10, o);  // lazy diffusion: overlay active at the end
	const sim::RunResult ga = sim::Simulator().run(g, state::QuantumState::basis(10));
	const experiment::StateComparison gd = experiment::compareStates(ga.state, ga.state);
	REQUIRE(gd.bitwiseEqual && gd.relL2 == 0.0);
}

void operationsAndSwaps() {
	circuit::Circuit c(2);
	c.h(0).swap(0, 1).swap(0, 1);
	const sim::RunResult r = sim::Simulator().run(c, state::QuantumState::basis(2));
	REQUIRE(close(r.state.amplitude(0).real, 1.0 / std::sqrt(2.0), 1e-6));
	REQUIRE(close(r.state.amplitude(2).real, 1.0 / std::sqrt(2.0), 1e-6));
	const QuantumGate scaled = QuantumGate::Hadamard() * Amplitude{2.0, 0.0};
	REQUIRE(close(scaled[0][0].real, 2.0 / std::sqrt(2.0)) && close(scaled[1][1].real, -2.0 / std::sqrt(2.0)));
	REQUIRE(close(complexExp({0.0, kPi}).real, -1.0));
	REQUIRE(circuit::groverIterationCount(StateIndex(1) << 20, 1) == 804u);
	REQUIRE(circuit::groverIterationCount(StateIndex(1) << 30, 4) == 12867u);
	const experiment::StateComparison cmp = experiment::compareStates(r.state, r.state);
	REQUIRE(cmp.bitwiseEqual && cmp.relL2 == 0.0);
	REQUIRE(experiment::toJson(r.report).find("\"strategy\": \"gpu\"") != std::string::npos);
}

}  // namespace

// The C-ABI status classes through GpuStateBackend's exception mapping:
// out_of_range, invalid_argument, logic_error (an uninitialised backend) and
// runtime_error for device out-of-memory, injected on the host with
// tmfqs_debug_fail_allocations (no device memory is exhausted).
void failureMapping() {
	RegisterConfig cfg;
	cfg.strategy = StorageStrategyKind::Gpu;
	std::unique_ptr<IStateBackend> raw = StateBackendFactory::create(4, cfg);
	REQUIRE(throwsAs<std::logic_error>([&] { raw->applyHadamard(0); }));
	REQUIRE(throwsAs<std::logic_error>([&] { (void)raw->totalProbability(); }));
	raw->initZero(4);
	REQUIRE(throwsAs<std::out_of_range>([&] { raw->applyHadamard(4); }));
	REQUIRE(throwsAs<std::invalid_argument>([&] { raw->applyControlledNot(1, 1); }));
	REQUIRE(throwsAs<std::invalid_argument>([&] { (void)raw->sampleMeasurement(1.0); }));

	tmfqs_debug_fail_allocations(0, 1);
	REQUIRE(throwsAs<std::runtime_error>([&] { QuantumRegister q(20, 0); }));
	QuantumRegister ok(20, 0);  // the knob fired once; allocation works again
	ok.applyHadamard(3);
	tmfqs_debug_fail_allocations(0, 1);
	REQUIRE(throwsAs<std::runtime_error>([&] { QuantumRegister copy(ok); }));
	tmfqs_debug_fail_allocations(0, 0);
	QuantumRegister copy(ok);
	REQUIRE(copy.amplitude(0).real == ok.amplitude(0).real);
	REQUIRE(std::fabs(copy.totalProbability() - 1.0) < 1e-12);
}

int main() {
	try {
		qftKnownAnswers();
		groverSeeds();
		registerPrimitivesAndInversion();
		validation();
		registryAndCopies();
		batchedEqualsPerOperation();
		operationsAndSwaps();
		failureMapping();
		deviceCompareStates();
	} catch(const std::exception &e) {
		std::cout << "FAILED after " << g_checks << " checks: " << e.what() << "\n";
		return 1;
	}
	std::cout << "host API checks passed: " << g_checks << "\n";
	return 0;
}
