// Host-side input families and random draws of the dense path.
//
// These use the C++ standard library's std::mt19937 and
// std::uniform_real_distribution<double> and the C library's cos/sin -- the
// same facilities the reference uses -- so inputs and measurement draws are
// bit-identical to the reference's on the same toolchain:
//   QuantumState::randomPhase   src/tmfqs/state/quantum_state.cpp:264-277
//   buildRandomPhaseInput       examples/qftG.cpp:70-81 (same stream)
//   Mt19937RandomSource         include/tmfqs/core/random.h:32-58
#include <cmath>
#include <cstdint>
#include <random>
#include <string>
#include <unordered_set>

#include "../../include/tmfqs_b200.h"

extern "C" {

TMFQS_API int tmfqs_random_phase(unsigned num_qubits, uint32_t seed, double *host_out) {
	if(!host_out || num_qubits > 40) return TMFQS_ERR_INVALID_ARGUMENT;
	const uint64_t states = 1ull << num_qubits;
	std::mt19937 gen(seed);
	std::uniform_real_distribution<double> phase(0.0, 2.0 * std::acos(-1.0));
	const double norm = 1.0 / std::sqrt(static_cast<double>(states));
	for(uint64_t s = 0; s < states; ++s) {
		const double p = phase(gen);
		host_out[2 * s] = norm * std::cos(p);
		host_out[2 * s + 1] = norm * std::sin(p);
	}
	return TMFQS_OK;
}

TMFQS_API int tmfqs_mt19937_unit(uint32_t seed, uint64_t count, double *host_out) {
	if(!host_out && count) return TMFQS_ERR_INVALID_ARGUMENT;
	std::mt19937 gen(seed);
	std::uniform_real_distribution<double> unit(0.0, 1.0);
	for(uint64_t i = 0; i < count; ++i) host_out[i] = unit(gen);
	return TMFQS_OK;
}

TMFQS_API int tmfqs_uniform_states(uint64_t seed, uint64_t count, uint64_t lo, uint64_t hi, uint64_t *host_out) {
	if((!host_out && count) || lo > hi || (hi - lo < UINT64_MAX && count > hi - lo + 1)) return TMFQS_ERR_INVALID_ARGUMENT;
	std::mt19937_64 gen(seed);
	std::uniform_int_distribution<uint64_t> dist(lo, hi);
	std::unordered_set<uint64_t> seen;
	for(uint64_t i = 0; i < count;) {
		const uint64_t v = dist(gen);
		if(seen.insert(v).second) host_out[i++] = v;
	}
	return TMFQS_OK;
}

}  // extern "C"
