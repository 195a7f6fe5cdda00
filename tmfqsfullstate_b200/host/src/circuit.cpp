// Circuit IR and the QFT / Grover builders (src/tmfqs/circuit/circuit.cpp).
#include "tmfqs/circuit/circuit.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <type_traits>

#include "tmfqs/core/constants.h"
#include "tmfqs/core/state_space.h"

namespace tmfqs {
namespace circuit {

Circuit::Circuit(unsigned int qubits) : qubits_(qubits) {}
unsigned int Circuit::qubitCount() const noexcept { return qubits_; }
const std::vector<Operation> &Circuit::operations() const noexcept { return operations_; }
size_t Circuit::operationCount() const noexcept { return operations_.size(); }
Circuit &Circuit::h(QubitIndex t) { return append(Hadamard{t}); }
Circuit &Circuit::x(QubitIndex t) { return append(PauliX{t}); }
Circuit &Circuit::cx(QubitIndex c, QubitIndex t) { return append(ControlledNot{c, t}); }
Circuit &Circuit::controlledPhase(QubitIndex c, QubitIndex t, double th) { return append(ControlledPhaseShift{c, t, th}); }
Circuit &Circuit::swap(QubitIndex a, QubitIndex b) { return append(Swap{a, b}); }
Circuit &Circuit::gate(QuantumGate g, QubitList targets) { return append(MatrixGate{std::move(g), std::move(targets)}); }
Circuit &Circuit::phaseFlip(StateIndex s) { return append(PhaseFlipBasisState{s}); }
Circuit &Circuit::inversionAboutMean(bool materialized) { return append(InversionAboutMean{materialized}); }

Circuit &Circuit::append(const Operation &op) {
	operations_.push_back(op);
	return *this;
}

Circuit &Circuit::append(Operation &&op) {
	operations_.push_back(std::move(op));
	return *this;
}

std::string operationName(const Operation &operation) {
	static const char *const names[] = {"h", "x", "cx", "controlled_phase", "swap", "gate", "phase_flip_basis_state",
	                                    "inversion_about_mean"};
	return names[operation.index()];
}

// For each target t: H(t), then controlledPhase(c, t, pi / 2^(c-t)) for
// c = t+1..n-1; then swap(l, n-1-l) for l < n/2 (circuit.cpp:87-100).
void appendQft(Circuit &circuit) {
	const unsigned int n = circuit.qubitCount();
	for(unsigned int t = 0; t < n; ++t) {
		circuit.h(t);
		for(unsigned int c = t + 1u; c < n; ++c)
			circuit.controlledPhase(c, t, kPi / static_cast<double>(StateIndex{1} << (c - t)));
	}
	for(unsigned int l = 0; l < n / 2u; ++l) circuit.swap(l, n - l - 1u);
}

Circuit makeQft(unsigned int qubits) {
	Circuit c(qubits);
	appendQft(c);
	return c;
}

// floor(pi/4 * sqrt(N/M)) (circuit.cpp:108-116).
unsigned int groverIterationCount(StateIndex stateCount, size_t markedCount) {
	if(markedCount == 0u) throw std::invalid_argument("Grover circuit requires at least one marked state");
	const double ideal = (kPi / 4.0) * std::sqrt(static_cast<double>(stateCount) / static_cast<double>(markedCount));
	return static_cast<unsigned int>(std::floor(ideal));
}

// H on every qubit, then per iteration one phase flip per sorted unique marked
// state and an inversion about the mean (circuit.cpp:118-141).
void appendGrover(Circuit &circuit, const GroverCircuitOptions &options) {
	std::vector<StateIndex> marked = options.markedStates.values();
	if(marked.empty()) throw std::invalid_argument("Grover circuit requires at least one marked state");
	std::sort(marked.begin(), marked.end());
	marked.erase(std::unique(marked.begin(), marked.end()), marked.end());
	for(unsigned int q = 0; q < circuit.qubitCount(); ++q) circuit.h(q);
	const StateIndex N = checkedStateCount(circuit.qubitCount());
	const unsigned int iterations = groverIterationCount(N, marked.size());
	for(unsigned int it = 0; it < iterations; ++it) {
		for(StateIndex s : marked) {
			if(s >= N) throw std::invalid_argument("Grover marked state is out of range");
			circuit.phaseFlip(s);
		}
		circuit.inversionAboutMean(options.materializedDiffusion);
	}
}

Circuit makeGrover(unsigned int qubits, GroverCircuitOptions options) {
	Circuit c(qubits);
	appendGrover(c, options);
	return c;
}

}  // namespace circuit
}  // namespace tmfqs
