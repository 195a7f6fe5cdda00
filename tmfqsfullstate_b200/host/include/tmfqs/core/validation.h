// Argument checks with the reference's exception classes
// (include/tmfqs/core/validation.h:19-80); state counts are 64-bit here.
#ifndef TMFQS_HOST_CORE_VALIDATION_H
#define TMFQS_HOST_CORE_VALIDATION_H

#include <stdexcept>
#include <string>
#include <vector>

#include "tmfqs/core/state_space.h"
#include "tmfqs/core/types.h"

namespace tmfqs {

inline void validateStateIndex(const char *scope, StateIndex state, StateIndex stateCount) {
	if(state >= stateCount) throw std::out_of_range(std::string(scope) + " state index out of range");
}

inline void validateQubitIndex(const char *scope, QubitIndex qubit, unsigned int numQubits) {
	if(qubit >= numQubits) throw std::out_of_range(std::string(scope) + " qubit index out of range");
}

inline void validateDistinctQubits(const char *scope, QubitIndex a, QubitIndex b) {
	if(a == b) throw std::invalid_argument(std::string(scope) + " requires distinct qubits");
}

inline void validateGateTargets(const char *scope, const QubitList &qubits, unsigned int numQubits, unsigned int gateDimension) {
	if(qubits.size() > maxSupportedQubitsForU32States())
		throw std::invalid_argument(std::string(scope) + " qubit list exceeds supported index width");
	if(qubits.size() > numQubits) throw std::invalid_argument(std::string(scope) + " gate acts on more qubits than available");
	if(gateDimension != checkedStateCount(static_cast<unsigned int>(qubits.size())))
		throw std::invalid_argument(std::string(scope) + " gate dimension does not match qubit list");
	std::vector<bool> seen(numQubits, false);
	for(QubitIndex q : qubits) {
		validateQubitIndex(scope, q, numQubits);
		if(seen[q]) throw std::invalid_argument(std::string(scope) + " duplicate qubit index");
		seen[q] = true;
	}
}

}  // namespace tmfqs

#endif
