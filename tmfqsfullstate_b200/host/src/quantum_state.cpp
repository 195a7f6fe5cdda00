// Circuit input / result value type (src/tmfqs/state/quantum_state.cpp).
// Lazy kinds (basis, uniform subset) are answered on the host from their
// definition; results stay in the device register that produced them.
#include "tmfqs/state/quantum_state.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <stdexcept>

#include "tmfqs/config/register_config.h"
#include "tmfqs/core/state_space.h"
#include "tmfqs/register/quantum_register.h"
#include "tmfqs_b200.h"

namespace tmfqs {
namespace state {
namespace {

enum class Kind { Basis, BasisAmplitude, UniformSubset, Amplitudes, Register };

double mass(const AmplitudesVector &a) {
	double t = 0.0;
	for(size_t e = 0; e + 1u < a.size(); e += 2u) t += a[e] * a[e] + a[e + 1u] * a[e + 1u];
	return t;
}

void validateOrNormalize(AmplitudesVector &a, const StateValidation &v) {
	if(a.size() % 2u != 0u) throw std::invalid_argument("Amplitude vector length must be even");
	if(v.normalization == NormalizationPolicy::AllowUnnormalized) return;
	const double t = mass(a);
	if(v.normalization == NormalizationPolicy::Normalize) {
		if(t <= 0.0) throw std::invalid_argument("Cannot normalize an all-zero amplitude vector");
		const double s = 1.0 / std::sqrt(t);
		for(double &x : a) x *= s;
		return;
	}
	if(std::abs(t - 1.0) > v.probabilityTolerance) throw std::invalid_argument("Amplitude vector is not normalized");
}

// Sorted unique members of a uniform subset and their amplitude 1/sqrt(k)
// (dense_state_backend.cpp:92-115).
std::vector<StateIndex> uniqueSorted(const BasisStateList &l) {
	std::vector<StateIndex> v = l.values();
	std::sort(v.begin(), v.end());
	v.erase(std::unique(v.begin(), v.end()), v.end());
	return v;
}

}  // namespace

struct QuantumState::Impl {
	unsigned int qubits = 0;
	Kind kind = Kind::Basis;
	StateIndex basisState = 0u;
	Amplitude basisAmplitude{1.0, 0.0};
	BasisStateList basisStates;
	AmplitudesVector amplitudes;
	std::unique_ptr<QuantumRegister> reg;

	Impl() = default;
	Impl(const Impl &o)
		: qubits(o.qubits), kind(o.kind), basisState(o.basisState), basisAmplitude(o.basisAmplitude),
		  basisStates(o.basisStates), amplitudes(o.amplitudes), reg(o.reg ? std::make_unique<QuantumRegister>(*o.reg) : nullptr) {}
};

QuantumState::QuantumState() : impl_(std::make_unique<Impl>()) {}
QuantumState::QuantumState(std::unique_ptr<Impl> impl) : impl_(std::move(impl)) {}
QuantumState::QuantumState(const QuantumState &o) : impl_(std::make_unique<Impl>(*o.impl_)) {}
QuantumState &QuantumState::operator=(const QuantumState &o) {
	if(this != &o) impl_ = std::make_unique<Impl>(*o.impl_);
	return *this;
}
QuantumState::QuantumState(QuantumState &&) noexcept = default;
QuantumState &QuantumState::operator=(QuantumState &&) noexcept = default;
QuantumState::~QuantumState() = default;

unsigned int QuantumState::qubitCount() const { return impl_->qubits; }
StateIndex QuantumState::stateCount() const { return checkedStateCount(impl_->qubits); }

Amplitude QuantumState::amplitude(StateIndex s) const {
	if(s >= stateCount()) throw std::invalid_argument("Amplitude state index is out of range");
	switch(impl_->kind) {
		case Kind::Amplitudes: return {impl_->amplitudes[2 * s], impl_->amplitudes[2 * s + 1]};
		case Kind::Basis:
		case Kind::BasisAmplitude: return s == impl_->basisState ? impl_->basisAmplitude : Amplitude{0.0, 0.0};
		case Kind::Register: return impl_->reg->amplitude(s);
		case Kind::UniformSubset: {
			const std::vector<StateIndex> u = uniqueSorted(impl_->basisStates);
			if(u.empty()) throw std::invalid_argument("QuantumRegister::initUniformSuperposition requires at least one basis state");
			return std::binary_search(u.begin(), u.end(), s) ? Amplitude{1.0 / std::sqrt(static_cast<double>(u.size())), 0.0}
			                                                : Amplitude{0.0, 0.0};
		}
	}
	return {0.0, 0.0};
}

double QuantumState::totalProbability() const {
	switch(impl_->kind) {
		case Kind::Amplitudes: return mass(impl_->amplitudes);
		case Kind::Basis:
		case Kind::BasisAmplitude:
			return impl_->basisAmplitude.real * impl_->basisAmplitude.real + impl_->basisAmplitude.imag * impl_->basisAmplitude.imag;
		case Kind::Register: return impl_->reg->totalProbability();
		case Kind::UniformSubset: {
			const std::vector<StateIndex> u = uniqueSorted(impl_->basisStates);
			const double a = 1.0 / std::sqrt(static_cast<double>(u.size()));
			double t = 0.0;
			for(size_t i = 0; i < u.size(); ++i) t += a * a;  // zeros in between add exactly 0
			return t;
		}
	}
	return 0.0;
}

AmplitudesVector QuantumState::amplitudes() const {
	switch(impl_->kind) {
		case Kind::Amplitudes: return impl_->amplitudes;
		case Kind::Register: return impl_->reg->amplitudes();
		default: {
			AmplitudesVector out(checkedAmplitudeElementCount(impl_->qubits), 0.0);
			if(impl_->kind == Kind::UniformSubset) {
				const std::vector<StateIndex> u = uniqueSorted(impl_->basisStates);
				const double a = 1.0 / std::sqrt(static_cast<double>(u.size()));
				for(StateIndex s : u) out[2 * s] = a;
			} else {
				out[2 * impl_->basisState] = impl_->basisAmplitude.real;
				out[2 * impl_->basisState + 1] = impl_->basisAmplitude.imag;
			}
			return out;
		}
	}
}

// quantum_state.cpp:176-199: first index whose running probability reaches
// the draw, summed left to right.
StateIndex QuantumState::measure(IRandomSource &rng) const {
	switch(impl_->kind) {
		case Kind::Basis:
		case Kind::BasisAmplitude: return impl_->basisState;
		case Kind::Register: return impl_->reg->measure(rng);
		case Kind::Amplitudes: {
			const double rnd = rng.nextUnitDouble();
			double c = 0.0;
			for(StateIndex s = 0; s < stateCount(); ++s) {
				c += impl_->amplitudes[2 * s] * impl_->amplitudes[2 * s] + impl_->amplitudes[2 * s + 1] * impl_->amplitudes[2 * s + 1];
				if(rnd <= c) return s;
			}
			throw std::runtime_error("QuantumState::measure cumulative probability did not reach sample");
		}
		case Kind::UniformSubset: {
			// A materialised register's CDF; the zero amplitudes between members add exactly 0.
			const double rnd = rng.nextUnitDouble();
			const std::vector<StateIndex> u = uniqueSorted(impl_->basisStates);
			const double a = 1.0 / std::sqrt(static_cast<double>(u.size()));
			double c = 0.0;
			if(rnd <= 0.0) return 0;
			for(StateIndex s : u) {
				c += a * a;
				if(rnd <= c) return s;
			}
			throw std::runtime_error("DenseStateBackend::sampleMeasurement cumulative probability did not reach sample");
		}
	}
	return 0;
}

void QuantumState::setAmplitude(StateIndex s, Amplitude a, const StateValidation &v) {
	AmplitudesVector values = amplitudes();
	if(s >= stateCount()) throw std::invalid_argument("Amplitude state index is out of range");
	values[2 * s] = a.real;
	values[2 * s + 1] = a.imag;
	loadAmplitudes(std::move(values), v);
}

void QuantumState::loadAmplitudes(AmplitudesVector a, const StateValidation &v) {
	if(a.size() != checkedAmplitudeElementCount(impl_->qubits)) throw std::invalid_argument("Amplitude vector size does not match state qubit count");
	validateOrNormalize(a, v);
	impl_->kind = Kind::Amplitudes;
	impl_->amplitudes = std::move(a);
	impl_->reg.reset();
}

QuantumState QuantumState::basis(unsigned int q, StateIndex s) {
	if(s >= checkedStateCount(q)) throw std::invalid_argument("Basis state is out of range");
	auto impl = std::make_unique<Impl>();
	impl->qubits = q;
	impl->kind = Kind::Basis;
	impl->basisState = s;
	return QuantumState(std::move(impl));
}

QuantumState QuantumState::basisAmplitude(unsigned int q, StateIndex s, Amplitude a) {
	if(s >= checkedStateCount(q)) throw std::invalid_argument("Basis state is out of range");
	auto impl = std::make_unique<Impl>();
	impl->qubits = q;
	impl->kind = Kind::BasisAmplitude;
	impl->basisState = s;
	impl->basisAmplitude = a;
	return QuantumState(std::move(impl));
}

QuantumState QuantumState::uniformSubset(unsigned int q, BasisStateList states) {
	auto impl = std::make_unique<Impl>();
	impl->qubits = q;
	impl->kind = Kind::UniformSubset;
	impl->basisStates = std::move(states);
	return QuantumState(std::move(impl));
}

QuantumState QuantumState::fromAmplitudes(unsigned int q, AmplitudesVector a, const StateValidation &v) {
	if(a.size() != checkedAmplitudeElementCount(q)) throw std::invalid_argument("Amplitude vector size does not match qubit count");
	validateOrNormalize(a, v);
	auto impl = std::make_unique<Impl>();
	impl->qubits = q;
	impl->kind = Kind::Amplitudes;
	impl->amplitudes = std::move(a);
	return QuantumState(std::move(impl));
}

// quantum_state.cpp:264-277 (std::mt19937 + uniform_real_distribution, same stream).
QuantumState QuantumState::randomPhase(unsigned int q, unsigned int seed) {
	AmplitudesVector a(checkedAmplitudeElementCount(q));
	if(tmfqs_random_phase(q, seed, a.data()) != TMFQS_OK) throw std::invalid_argument("randomPhase: unsupported size");
	return fromAmplitudes(q, std::move(a));
}

QuantumState QuantumState::sparsePattern(unsigned int q) {
	const StateIndex N = checkedStateCount(q);
	std::vector<StateIndex> sel;
	for(StateIndex x = 0;; ++x) {
		const StateIndex s = 8u * x + (x % 2u);
		if(s >= N) break;
		sel.push_back(s);
	}
	return uniformSubset(q, BasisStateList(std::move(sel)));
}

QuantumRegister QuantumState::materialize(const RegisterConfig &cfg) const {
	switch(impl_->kind) {
		case Kind::Basis: return QuantumRegister(impl_->qubits, impl_->basisState, cfg);
		case Kind::BasisAmplitude: return QuantumRegister(impl_->qubits, impl_->basisState, impl_->basisAmplitude, cfg);
		case Kind::UniformSubset: {
			QuantumRegister r(impl_->qubits, cfg);
			r.initUniformSuperposition(impl_->basisStates);
			return r;
		}
		case Kind::Amplitudes: return QuantumRegister(impl_->qubits, impl_->amplitudes, cfg);
		case Kind::Register: return *impl_->reg;
	}
	return QuantumRegister(impl_->qubits, cfg);
}

const QuantumRegister *QuantumState::registerOrNull() const {
	return impl_->kind == Kind::Register ? impl_->reg.get() : nullptr;
}

QuantumState QuantumState::fromRegister(QuantumRegister reg) {
	auto impl = std::make_unique<Impl>();
	impl->qubits = reg.qubitCount();
	impl->kind = Kind::Register;
	impl->reg = std::make_unique<QuantumRegister>(std::move(reg));
	return QuantumState(std::move(impl));
}

}  // namespace state
}  // namespace tmfqs
