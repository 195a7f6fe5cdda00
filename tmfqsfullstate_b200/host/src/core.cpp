// Complex helpers and the measurement random source.
#include <cmath>

#include "tmfqs/core/math.h"
#include "tmfqs/core/random.h"

namespace tmfqs {

// (ar + i ai)(br + i bi), operand order of src/tmfqs/core/math.cpp:8-13.
Amplitude amplitudeMultiply(Amplitude a, Amplitude b) {
	return {a.real * b.real - a.imag * b.imag, a.real * b.imag + a.imag * b.real};
}

Amplitude amplitudeAdd(Amplitude a, Amplitude b) { return {a.real + b.real, a.imag + b.imag}; }

// e^(x + iy) = e^x (cos y + i sin y) (math.cpp:22-29).
Amplitude complexExp(Amplitude e) {
	const double r = std::exp(e.real);
	return {r * std::cos(e.imag), r * std::sin(e.imag)};
}

Mt19937RandomSource::Mt19937RandomSource() : engine_(std::random_device{}()) {}
Mt19937RandomSource::Mt19937RandomSource(uint32_t seed) : engine_(seed) {}
double Mt19937RandomSource::nextUnitDouble() { return distribution_(engine_); }
void Mt19937RandomSource::reseed(uint32_t seed) { engine_.seed(seed); }

}  // namespace tmfqs
