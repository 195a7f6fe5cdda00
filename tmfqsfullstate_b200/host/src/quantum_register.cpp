// QuantumRegister: the reference's register semantics
// (src/tmfqs/register/quantum_register.cpp) -- lazy affine overlay, cached
// logical amplitude sum, swaps as three CNOTs -- over any IStateBackend.
// When the backend offers the device hooks, reductions over logical
// amplitudes and whole gate / Grover runs execute on the device with the
// same results as the per-operation host code.
#include "tmfqs/register/quantum_register.h"

#include <cmath>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tmfqs/core/random.h"
#include "tmfqs/core/state_space.h"
#include "tmfqs/core/validation.h"
#include "tmfqs/storage/factory/state_backend_factory.h"

namespace tmfqs {
namespace {

constexpr double kPrintEpsilon = 1e-12;

Amplitude cxAdd(Amplitude a, Amplitude b) { return {a.real + b.real, a.imag + b.imag}; }
Amplitude cxSub(Amplitude a, Amplitude b) { return {a.real - b.real, a.imag - b.imag}; }
Amplitude cxNeg(Amplitude a) { return {-a.real, -a.imag}; }
Amplitude cxScale(Amplitude a, double s) { return {a.real * s, a.imag * s}; }
Amplitude cxMul(Amplitude l, Amplitude r) { return {l.real * r.real - l.imag * r.imag, l.real * r.imag + l.imag * r.real}; }
Amplitude cxDiv(Amplitude n, Amplitude d) {
	const double q = d.real * d.real + d.imag * d.imag;
	if(q == 0.0) throw std::logic_error("QuantumRegister affine overlay scale is zero");
	return {(n.real * d.real + n.imag * d.imag) / q, (n.imag * d.real - n.real * d.imag) / q};
}
double probOf(Amplitude a) { return a.real * a.real + a.imag * a.imag; }

}  // namespace

QuantumRegister::QuantumRegister() {
	initializeBackend(0);
	backend_->initBasis(numQubits_, 0, {1.0, 0.0});
}

void QuantumRegister::initializeBackend(unsigned int qubits) {
	numQubits_ = qubits;
	numStates_ = checkedStateCount(qubits);
	BackendSelection sel = StateBackendFactory::createSelection(qubits, config_);
	config_ = sel.config;
	resolvedStrategy_ = sel.strategy;
	backend_ = std::move(sel.backend);
}

QuantumRegister::QuantumRegister(unsigned int qubits, const RegisterConfig &cfg) : config_(cfg) {
	initializeBackend(qubits);
	backend_->initBasis(numQubits_, 0, {1.0, 0.0});
}

QuantumRegister::QuantumRegister(unsigned int qubits, StateIndex initState, const RegisterConfig &cfg) : config_(cfg) {
	initializeBackend(qubits);
	backend_->initBasis(numQubits_, initState, {1.0, 0.0});
}

QuantumRegister::QuantumRegister(unsigned int qubits, StateIndex initState, Amplitude amp, const RegisterConfig &cfg) : config_(cfg) {
	initializeBackend(qubits);
	backend_->initBasis(numQubits_, initState, amp);
}

QuantumRegister::QuantumRegister(unsigned int qubits, AmplitudesVector amplitudes, const RegisterConfig &cfg) : config_(cfg) {
	initializeBackend(qubits);
	backend_->loadAmplitudes(numQubits_, std::move(amplitudes));
}

QuantumRegister::QuantumRegister(const QuantumRegister &o)
	: numQubits_(o.numQubits_), numStates_(o.numStates_), config_(o.config_), resolvedStrategy_(o.resolvedStrategy_),
	  backend_(o.backend_ ? o.backend_->clone() : nullptr), cachedLogicalAmplitudeSum_(o.cachedLogicalAmplitudeSum_),
	  affineScale_(o.affineScale_), affineBias_(o.affineBias_), affineOverlayActive_(o.affineOverlayActive_) {}

QuantumRegister &QuantumRegister::operator=(const QuantumRegister &o) {
	if(this == &o) return *this;
	numQubits_ = o.numQubits_;
	numStates_ = o.numStates_;
	config_ = o.config_;
	resolvedStrategy_ = o.resolvedStrategy_;
	if(!o.backend_) {
		backend_.reset();
		resetAffineOverlay();
		return *this;
	}
	backend_ = o.backend_->clone();
	affineScale_ = o.affineScale_;
	affineBias_ = o.affineBias_;
	affineOverlayActive_ = o.affineOverlayActive_;
	cachedLogicalAmplitudeSum_ = o.cachedLogicalAmplitudeSum_;
	return *this;
}

QuantumRegister::~QuantumRegister() = default;

void QuantumRegister::requireInitialized(const char *operation) const {
	if(!backend_) throw std::logic_error(std::string("QuantumRegister is not initialized for ") + operation);
}

void QuantumRegister::resetAffineOverlay() {
	affineScale_ = {1.0, 0.0};
	affineBias_ = {0.0, 0.0};
	affineOverlayActive_ = false;
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

Amplitude QuantumRegister::applyAffineOverlay(Amplitude a) const {
	return affineOverlayActive_ ? cxAdd(cxMul(affineScale_, a), affineBias_) : a;
}

Amplitude QuantumRegister::removeAffineOverlay(Amplitude l) const {
	return affineOverlayActive_ ? cxDiv(cxSub(l, affineBias_), affineScale_) : l;
}

const AffineOverlay *QuantumRegister::overlayOrNull(AffineOverlay &storage) const {
	if(!affineOverlayActive_) return nullptr;
	storage.scale = affineScale_;
	storage.bias = affineBias_;
	return &storage;
}

Amplitude QuantumRegister::logicalAmplitudeSum() const {
	if(cachedLogicalAmplitudeSum_) return *cachedLogicalAmplitudeSum_;
	AffineOverlay ov;
	Amplitude sum{0.0, 0.0};
	if(!backend_->logicalAmplitudeSum(overlayOrNull(ov), sum)) {
		visitLogicalAmplitudeChunks([&](StateIndex, const double *d, size_t elems) {
			for(size_t e = 0; e + 1u < elems; e += 2u) {
				sum.real += d[e];
				sum.imag += d[e + 1u];
			}
		});
	}
	cachedLogicalAmplitudeSum_ = sum;
	return sum;
}

void QuantumRegister::visitLogicalAmplitudeChunks(const std::function<void(StateIndex, const double *, size_t)> &visitor) const {
	requireInitialized("amplitude chunk iteration");
	if(!affineOverlayActive_) {
		backend_->forEachAmplitudeChunk(visitor);
		return;
	}
	std::vector<double> logical;
	backend_->forEachAmplitudeChunk([&](StateIndex base, const double *d, size_t elems) {
		logical.resize(elems);
		for(size_t e = 0; e + 1u < elems; e += 2u) {
			const Amplitude l = applyAffineOverlay({d[e], d[e + 1u]});
			logical[e] = l.real;
			logical[e + 1u] = l.imag;
		}
		visitor(base, logical.data(), elems);
	});
}

AmplitudesVector QuantumRegister::snapshotLogicalAmplitudes() const {
	AmplitudesVector out;
	backend_->exportAmplitudes(out);
	if(affineOverlayActive_) {
		for(size_t e = 0; e + 1u < out.size(); e += 2u) {
			const Amplitude l = applyAffineOverlay({out[e], out[e + 1u]});
			out[e] = l.real;
			out[e + 1u] = l.imag;
		}
	}
	return out;
}

void QuantumRegister::flushAffineOverlay() {
	if(!affineOverlayActive_) return;
	const std::optional<Amplitude> saved = cachedLogicalAmplitudeSum_;
	backend_->applyAffineTransform(affineScale_, affineBias_);
	resetAffineOverlay();
	cachedLogicalAmplitudeSum_ = saved;
}

unsigned int QuantumRegister::qubitCount() const { return numQubits_; }
StateIndex QuantumRegister::stateCount() const { return numStates_; }
size_t QuantumRegister::amplitudeElementCount() const { return static_cast<size_t>(numStates_) * 2u; }
StorageStrategyKind QuantumRegister::storageStrategy() const { return resolvedStrategy_; }

Amplitude QuantumRegister::amplitude(StateIndex state) const {
	requireInitialized("amplitude query");
	validateStateIndex("QuantumRegister::amplitude", state, numStates_);
	return applyAffineOverlay(backend_->amplitude(state));
}

AmplitudesVector QuantumRegister::amplitudes() const {
	requireInitialized("amplitude export");
	return snapshotLogicalAmplitudes();
}

double QuantumRegister::probability(StateIndex state) const {
	requireInitialized("probability query");
	validateStateIndex("QuantumRegister::probability", state, numStates_);
	return probOf(amplitude(state));
}

double QuantumRegister::totalProbability() const {
	requireInitialized("probability summation");
	if(!affineOverlayActive_) return backend_->totalProbability();
	AffineOverlay ov;
	double total = 0.0;
	if(backend_->logicalTotalProbability(overlayOrNull(ov), total)) return total;
	visitLogicalAmplitudeChunks([&](StateIndex, const double *d, size_t elems) {
		for(size_t e = 0; e + 1u < elems; e += 2u) total += d[e] * d[e] + d[e + 1u] * d[e + 1u];
	});
	return total;
}

StateIndex QuantumRegister::measure(IRandomSource &randomSource) const {
	requireInitialized("measurement");
	if(!affineOverlayActive_) return backend_->sampleMeasurement(randomSource.nextUnitDouble());
	const double rnd = randomSource.nextUnitDouble();
	AffineOverlay ov;
	StateIndex out = numStates_;
	if(backend_->logicalSample(overlayOrNull(ov), rnd, out)) return out;
	double cumulative = 0.0;
	visitLogicalAmplitudeChunks([&](StateIndex base, const double *d, size_t elems) {
		if(out != numStates_) return;
		for(size_t i = 0; i < elems / 2u; ++i) {
			cumulative += d[2 * i] * d[2 * i] + d[2 * i + 1] * d[2 * i + 1];
			if(rnd <= cumulative) {
				out = base + i;
				return;
			}
		}
	});
	if(out != numStates_) return out;
	throw std::runtime_error("QuantumRegister::measure cumulative probability did not reach sample");
}

void QuantumRegister::setAmplitude(StateIndex state, Amplitude amp) {
	requireInitialized("state update");
	validateStateIndex("QuantumRegister::setAmplitude", state, numStates_);
	backend_->setAmplitude(state, removeAffineOverlay(amp));
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

void QuantumRegister::loadAmplitudes(AmplitudesVector amplitudes) {
	requireInitialized("amplitude loading");
	if(amplitudes.size() != amplitudeElementCount())
		throw std::invalid_argument("QuantumRegister::loadAmplitudes amplitudes size mismatch");
	resetAffineOverlay();
	backend_->loadAmplitudes(numQubits_, std::move(amplitudes));
}

void QuantumRegister::initUniformSuperposition(const BasisStateList &states) {
	requireInitialized("uniform superposition initialization");
	if(states.empty()) throw std::invalid_argument("QuantumRegister::initUniformSuperposition requires at least one basis state");
	for(StateIndex s : states) validateStateIndex("QuantumRegister::initUniformSuperposition", s, numStates_);
	resetAffineOverlay();
	backend_->initUniformSuperposition(numQubits_, states);
}

void QuantumRegister::printStatesVector(double epsilon) const {
	requireInitialized("state printing");
	if(epsilon < 0.0) throw std::invalid_argument("QuantumRegister::printStatesVector epsilon must be non-negative");
	if(!affineOverlayActive_) {
		backend_->printNonZeroStates(std::cout, epsilon);
		return;
	}
	visitLogicalAmplitudeChunks([&](StateIndex base, const double *d, size_t elems) {
		for(size_t i = 0; i < elems / 2u; ++i)
			if(std::abs(d[2 * i]) > epsilon || std::abs(d[2 * i + 1]) > epsilon)
				std::cout << (base + i) << ": " << d[2 * i] << " + " << d[2 * i + 1] << "i\n";
	});
}

std::ostream &operator<<(std::ostream &os, const QuantumRegister &reg) {
	reg.requireInitialized("state printing");
	if(!reg.affineOverlayActive_) {
		reg.backend_->printNonZeroStates(os, kPrintEpsilon);
		return os;
	}
	reg.visitLogicalAmplitudeChunks([&](StateIndex base, const double *d, size_t elems) {
		for(size_t i = 0; i < elems / 2u; ++i)
			if(std::abs(d[2 * i]) > kPrintEpsilon || std::abs(d[2 * i + 1]) > kPrintEpsilon)
				os << (base + i) << ": " << d[2 * i] << " + " << d[2 * i + 1] << "i\n";
	});
	return os;
}

void QuantumRegister::applyGate(const QuantumGate &gate, const QubitList &qubits) {
	requireInitialized("gate application");
	validateGateTargets("QuantumRegister::applyGate", qubits, numQubits_, gate.dimension());
	flushAffineOverlay();
	backend_->applyGate(gate, qubits);
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

// quantum_register.cpp:405-420: with a cached sum or an overlay the flip
// goes through the logical amplitude; otherwise straight to the backend.
void QuantumRegister::applyPhaseFlipBasisState(StateIndex state) {
	requireInitialized("basis-state phase flip");
	validateStateIndex("QuantumRegister::applyPhaseFlipBasisState", state, numStates_);
	if(cachedLogicalAmplitudeSum_ || affineOverlayActive_) {
		const Amplitude logical = amplitude(state);
		if(cachedLogicalAmplitudeSum_) {
			cachedLogicalAmplitudeSum_->real -= 2.0 * logical.real;
			cachedLogicalAmplitudeSum_->imag -= 2.0 * logical.imag;
		}
		if(affineOverlayActive_) {
			backend_->setAmplitude(state, removeAffineOverlay(cxNeg(logical)));
			return;
		}
	}
	backend_->phaseFlipBasisState(state);
}

void QuantumRegister::applyInversionAboutMean() {
	requireInitialized("inversion about mean");
	const Amplitude s = logicalAmplitudeSum();
	applyInversionAboutMean({s.real / static_cast<double>(numStates_), s.imag / static_cast<double>(numStates_)});
}

// Lazy form (quantum_register.cpp:433-444): scale <- -scale, bias <- 2*mean - bias.
void QuantumRegister::applyInversionAboutMean(Amplitude mean) {
	requireInitialized("inversion about mean");
	const double N = static_cast<double>(numStates_);
	if(cachedLogicalAmplitudeSum_) {
		cachedLogicalAmplitudeSum_->real = 2.0 * mean.real * N - cachedLogicalAmplitudeSum_->real;
		cachedLogicalAmplitudeSum_->imag = 2.0 * mean.imag * N - cachedLogicalAmplitudeSum_->imag;
	}
	const Amplitude scale = affineOverlayActive_ ? affineScale_ : Amplitude{1.0, 0.0};
	const Amplitude bias = affineOverlayActive_ ? affineBias_ : Amplitude{0.0, 0.0};
	affineScale_ = cxNeg(scale);
	affineBias_ = cxSub(cxScale(mean, 2.0), bias);
	affineOverlayActive_ = true;
}

void QuantumRegister::applyInversionAboutMeanMaterialized() {
	requireInitialized("inversion about mean");
	const Amplitude s = logicalAmplitudeSum();
	applyInversionAboutMeanMaterialized({s.real / static_cast<double>(numStates_), s.imag / static_cast<double>(numStates_)});
}

void QuantumRegister::applyInversionAboutMeanMaterialized(Amplitude mean) {
	requireInitialized("inversion about mean");
	const double N = static_cast<double>(numStates_);
	if(cachedLogicalAmplitudeSum_) {
		cachedLogicalAmplitudeSum_->real = 2.0 * mean.real * N - cachedLogicalAmplitudeSum_->real;
		cachedLogicalAmplitudeSum_->imag = 2.0 * mean.imag * N - cachedLogicalAmplitudeSum_->imag;
	}
	flushAffineOverlay();
	backend_->inversionAboutMean(mean);
}

void QuantumRegister::applyHadamard(QubitIndex q) {
	requireInitialized("Hadamard");
	validateQubitIndex("QuantumRegister::applyHadamard", q, numQubits_);
	flushAffineOverlay();
	backend_->applyHadamard(q);
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

void QuantumRegister::applyPauliX(QubitIndex q) {
	requireInitialized("PauliX");
	validateQubitIndex("QuantumRegister::applyPauliX", q, numQubits_);
	flushAffineOverlay();
	backend_->applyPauliX(q);
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

void QuantumRegister::applyControlledPhaseShift(QubitIndex c, QubitIndex t, double theta) {
	requireInitialized("controlled phase shift");
	validateQubitIndex("QuantumRegister::applyControlledPhaseShift", c, numQubits_);
	validateQubitIndex("QuantumRegister::applyControlledPhaseShift", t, numQubits_);
	validateDistinctQubits("QuantumRegister::applyControlledPhaseShift", c, t);
	flushAffineOverlay();
	backend_->applyControlledPhaseShift(c, t, theta);
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

void QuantumRegister::applyControlledNot(QubitIndex c, QubitIndex t) {
	requireInitialized("controlled not");
	validateQubitIndex("QuantumRegister::applyControlledNot", c, numQubits_);
	validateQubitIndex("QuantumRegister::applyControlledNot", t, numQubits_);
	validateDistinctQubits("QuantumRegister::applyControlledNot", c, t);
	flushAffineOverlay();
	backend_->applyControlledNot(c, t);
	cachedLogicalAmplitudeSum_ = std::nullopt;
}

// Three CNOTs (quantum_register.cpp:518-527).
void QuantumRegister::applySwap(QubitIndex a, QubitIndex b) {
	requireInitialized("swap");
	validateQubitIndex("QuantumRegister::applySwap", a, numQubits_);
	validateQubitIndex("QuantumRegister::applySwap", b, numQubits_);
	validateDistinctQubits("QuantumRegister::applySwap", a, b);
	applyControlledNot(a, b);
	applyControlledNot(b, a);
	applyControlledNot(a, b);
}

void QuantumRegister::beginOperationBatch() {
	requireInitialized("operation batch begin");
	backend_->beginOperationBatch();
}

void QuantumRegister::endOperationBatch() {
	requireInitialized("operation batch end");
	backend_->endOperationBatch();
}

namespace {

// The checks each single-operation method performs, in the same order.
void validateBackendOp(const BackendOp &op, unsigned int n, StateIndex N) {
	switch(op.kind) {
		case BackendOp::Kind::Hadamard: validateQubitIndex("QuantumRegister::applyHadamard", op.q0, n); break;
		case BackendOp::Kind::PauliX: validateQubitIndex("QuantumRegister::applyPauliX", op.q0, n); break;
		case BackendOp::Kind::ControlledNot:
			validateQubitIndex("QuantumRegister::applyControlledNot", op.q0, n);
			validateQubitIndex("QuantumRegister::applyControlledNot", op.q1, n);
			validateDistinctQubits("QuantumRegister::applyControlledNot", op.q0, op.q1);
			break;
		case BackendOp::Kind::ControlledPhaseShift:
			validateQubitIndex("QuantumRegister::applyControlledPhaseShift", op.q0, n);
			validateQubitIndex("QuantumRegister::applyControlledPhaseShift", op.q1, n);
			validateDistinctQubits("QuantumRegister::applyControlledPhaseShift", op.q0, op.q1);
			break;
		case BackendOp::Kind::Swap:
			validateQubitIndex("QuantumRegister::applySwap", op.q0, n);
			validateQubitIndex("QuantumRegister::applySwap", op.q1, n);
			validateDistinctQubits("QuantumRegister::applySwap", op.q0, op.q1);
			break;
		case BackendOp::Kind::MatrixGate:
			validateGateTargets("QuantumRegister::applyGate", *op.targets, n, op.gate->dimension());
			break;
		case BackendOp::Kind::PhaseFlip: validateStateIndex("QuantumRegister::applyPhaseFlipBasisState", op.state, N); break;
	}
}

void applyOnBackend(IStateBackend &b, const BackendOp &op) {
	switch(op.kind) {
		case BackendOp::Kind::Hadamard: b.applyHadamard(op.q0); break;
		case BackendOp::Kind::PauliX: b.applyPauliX(op.q0); break;
		case BackendOp::Kind::ControlledNot: b.applyControlledNot(op.q0, op.q1); break;
		case BackendOp::Kind::ControlledPhaseShift: b.applyControlledPhaseShift(op.q0, op.q1, op.theta); break;
		case BackendOp::Kind::Swap:
			b.applyControlledNot(op.q0, op.q1);
			b.applyControlledNot(op.q1, op.q0);
			b.applyControlledNot(op.q0, op.q1);
			break;
		case BackendOp::Kind::MatrixGate: b.applyGate(*op.gate, *op.targets); break;
		case BackendOp::Kind::PhaseFlip: b.phaseFlipBasisState(op.state); break;
	}
}

}  // namespace

void QuantumRegister::applyOperationRun(const std::vector<BackendOp> &ops) {
	requireInitialized("operation batch");
	size_t i = 0;
	// Leading flips under a cached sum or an overlay keep their logical semantics.
	while(i < ops.size() && ops[i].kind == BackendOp::Kind::PhaseFlip && (cachedLogicalAmplitudeSum_ || affineOverlayActive_)) {
		applyPhaseFlipBasisState(ops[i].state);
		++i;
	}
	if(i == ops.size()) return;
	// The reference applies operations one by one and throws at the first
	// invalid one: apply the valid prefix, then rethrow.
	std::exception_ptr error;
	size_t end = ops.size();
	for(size_t j = i; j < ops.size(); ++j) {
		try {
			validateBackendOp(ops[j], numQubits_, numStates_);
		} catch(...) {
			error = std::current_exception();
			end = j;
			break;
		}
	}
	if(end > i) {
		flushAffineOverlay();
		bool gate = false;
		for(size_t j = i; j < end; ++j) gate = gate || ops[j].kind != BackendOp::Kind::PhaseFlip;
		const std::vector<BackendOp> run(ops.begin() + static_cast<std::ptrdiff_t>(i), ops.begin() + static_cast<std::ptrdiff_t>(end));
		if(!backend_->applyOperationRun(run))
			for(const BackendOp &op : run) applyOnBackend(*backend_, op);
		if(gate) cachedLogicalAmplitudeSum_ = std::nullopt;
	}
	if(error) std::rethrow_exception(error);
}

void QuantumRegister::applyGroverIterations(const std::vector<StateIndex> &marked, uint64_t iterations, bool materialized) {
	requireInitialized("grover iterations");
	if(iterations == 0) return;
	bool valid = true;
	for(size_t k = 0; k < marked.size(); ++k)
		valid = valid && marked[k] < numStates_ && (k == 0 || marked[k - 1] < marked[k]);
	if(valid) {
		RegisterSideState side;
		side.hasSum = cachedLogicalAmplitudeSum_.has_value();
		if(side.hasSum) side.sum = *cachedLogicalAmplitudeSum_;
		side.overlayActive = affineOverlayActive_;
		side.overlay.scale = affineScale_;
		side.overlay.bias = affineBias_;
		if(backend_->runGroverIterations(side, marked, iterations, materialized)) {
			cachedLogicalAmplitudeSum_ = side.hasSum ? std::optional<Amplitude>(side.sum) : std::nullopt;
			affineOverlayActive_ = side.overlayActive;
			affineScale_ = side.overlay.scale;
			affineBias_ = side.overlay.bias;
			return;
		}
	}
	for(uint64_t it = 0; it < iterations; ++it) {
		for(StateIndex s : marked) applyPhaseFlipBasisState(s);
		if(materialized) applyInversionAboutMeanMaterialized();
		else applyInversionAboutMean();
	}
}

}  // namespace tmfqs
