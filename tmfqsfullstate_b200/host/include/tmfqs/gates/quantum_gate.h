// Dense gate matrices (include/tmfqs/gates/quantum_gate.h:17-137).
#ifndef TMFQS_HOST_GATES_QUANTUM_GATE_H
#define TMFQS_HOST_GATES_QUANTUM_GATE_H

#include <iosfwd>
#include <vector>

#include "tmfqs/core/types.h"

namespace tmfqs {

// Row-major dimension x dimension complex matrix.
class QuantumGate {
	public:
		QuantumGate() = default;
		explicit QuantumGate(unsigned int dimension);

		Amplitude *operator[](unsigned int row);
		const Amplitude *operator[](unsigned int row) const;
		unsigned int dimension() const noexcept { return dimension_; }
		const std::vector<Amplitude> &entries() const noexcept { return matrix_; }

		QuantumGate operator*(Amplitude x) const;
		QuantumGate operator*(const QuantumGate &other) const;
		void printQuantumGate() const;
		friend std::ostream &operator<<(std::ostream &os, const QuantumGate &g);

		static QuantumGate Identity(unsigned int dimension);
		static QuantumGate Hadamard();
		static QuantumGate PauliX();
		static QuantumGate PauliY();
		static QuantumGate PauliZ();
		static QuantumGate PhaseShift(double theta);
		static QuantumGate PiOverEight();
		static QuantumGate ControlledNot();
		static QuantumGate Toffoli();
		static QuantumGate ControlledPhaseShift(double theta);
		static QuantumGate Swap();
		static QuantumGate Ising(double theta);

	private:
		std::vector<Amplitude> matrix_;
		unsigned int dimension_ = 0;
};

QuantumGate operator*(Amplitude x, const QuantumGate &g);

}  // namespace tmfqs

#endif
