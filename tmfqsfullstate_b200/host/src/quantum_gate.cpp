// Gate matrices (src/tmfqs/gates/quantum_gate.cpp:96-210): same entries,
// computed with the same expressions, so MatrixGate results match the
// reference bit for bit.
#include "tmfqs/gates/quantum_gate.h"

#include <cmath>
#include <iostream>
#include <stdexcept>

#include "tmfqs/core/constants.h"
#include "tmfqs/core/math.h"

namespace tmfqs {

QuantumGate::QuantumGate(unsigned int dimension)
	: matrix_(static_cast<size_t>(dimension) * dimension, Amplitude{0.0, 0.0}), dimension_(dimension) {}

Amplitude *QuantumGate::operator[](unsigned int row) {
	if(row >= dimension_) throw std::out_of_range("QuantumGate row index out of range");
	return matrix_.data() + static_cast<size_t>(row) * dimension_;
}

const Amplitude *QuantumGate::operator[](unsigned int row) const {
	if(row >= dimension_) throw std::out_of_range("QuantumGate row index out of range");
	return matrix_.data() + static_cast<size_t>(row) * dimension_;
}

QuantumGate QuantumGate::operator*(Amplitude x) const {
	QuantumGate out(dimension_);
	for(size_t i = 0; i < matrix_.size(); ++i) out.matrix_[i] = amplitudeMultiply(matrix_[i], x);
	return out;
}

QuantumGate operator*(Amplitude x, const QuantumGate &g) { return g * x; }

QuantumGate QuantumGate::operator*(const QuantumGate &other) const {
	if(other.dimension_ != dimension_) throw std::invalid_argument("QuantumGate dimensions differ in multiplication");
	QuantumGate out(dimension_);
	// Accumulation order i, k, j as in quantum_gate.cpp:107-120.
	for(unsigned int i = 0; i < dimension_; ++i)
		for(unsigned int k = 0; k < dimension_; ++k) {
			const Amplitude l = (*this)[i][k];
			for(unsigned int j = 0; j < dimension_; ++j) out[i][j] = amplitudeAdd(out[i][j], amplitudeMultiply(l, other[k][j]));
		}
	return out;
}

std::ostream &operator<<(std::ostream &os, const QuantumGate &g) {
	for(unsigned int i = 0; i < g.dimension(); ++i) {
		for(unsigned int j = 0; j < g.dimension(); ++j) os << g[i][j].real << " " << g[i][j].imag << "\t";
		os << "\n";
	}
	return os;
}

void QuantumGate::printQuantumGate() const { std::cout << *this; }

QuantumGate QuantumGate::Identity(unsigned int d) {
	QuantumGate g(d);
	for(unsigned int i = 0; i < d; ++i) g[i][i].real = 1.0;
	return g;
}

QuantumGate QuantumGate::Hadamard() {
	QuantumGate g(2);
	const double s = 1.0 / std::sqrt(2.0);
	g[0][0].real = s;
	g[0][1].real = s;
	g[1][0].real = s;
	g[1][1].real = -s;
	return g;
}

QuantumGate QuantumGate::PauliX() {
	QuantumGate g(2);
	g[0][1].real = 1.0;
	g[1][0].real = 1.0;
	return g;
}

QuantumGate QuantumGate::PauliY() {
	QuantumGate g(2);
	g[0][1].imag = -1.0;
	g[1][0].imag = 1.0;
	return g;
}

QuantumGate QuantumGate::PauliZ() {
	QuantumGate g(2);
	g[0][0].real = 1.0;
	g[1][1].real = -1.0;
	return g;
}

QuantumGate QuantumGate::PhaseShift(double theta) {
	QuantumGate g(2);
	const Amplitude p = complexExp({0.0, theta});
	g[0][0].real = 1.0;
	g[1][1] = p;
	return g;
}

QuantumGate QuantumGate::PiOverEight() { return PhaseShift(kPi / 4.0); }

QuantumGate QuantumGate::ControlledNot() {
	QuantumGate g(4);
	g[0][0].real = 1.0;
	g[1][1].real = 1.0;
	g[2][3].real = 1.0;
	g[3][2].real = 1.0;
	return g;
}

QuantumGate QuantumGate::Toffoli() {
	QuantumGate g = Identity(8);
	g[6][6].real = 0.0;
	g[7][7].real = 0.0;
	g[6][7].real = 1.0;
	g[7][6].real = 1.0;
	return g;
}

QuantumGate QuantumGate::ControlledPhaseShift(double theta) {
	QuantumGate g(4);
	g[0][0].real = 1.0;
	g[1][1].real = 1.0;
	g[2][2].real = 1.0;
	g[3][3] = complexExp({0.0, theta});
	return g;
}

QuantumGate QuantumGate::Swap() {
	QuantumGate g(4);
	g[0][0].real = 1.0;
	g[1][2].real = 1.0;
	g[2][1].real = 1.0;
	g[3][3].real = 1.0;
	return g;
}

QuantumGate QuantumGate::Ising(double theta) {
	QuantumGate g(4);
	const double c = std::cos(theta / 2.0), s = std::sin(theta / 2.0);
	for(unsigned int i = 0; i < 4; ++i) g[i][i].real = c;
	g[0][3].imag = -s;
	g[1][2].imag = -s;
	g[2][1].imag = -s;
	g[3][0].imag = -s;
	return g;
}

}  // namespace tmfqs
