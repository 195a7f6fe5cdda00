// State-space sizes with 64-bit indices (include/tmfqs/core/state_space.h:16-46).
#ifndef TMFQS_HOST_CORE_STATE_SPACE_H
#define TMFQS_HOST_CORE_STATE_SPACE_H

#include <cstddef>
#include <limits>
#include <stdexcept>

#include "tmfqs/core/types.h"

namespace tmfqs {

inline constexpr unsigned int maxSupportedQubitsForStateIndex() { return std::numeric_limits<StateIndex>::digits - 1u; }
inline constexpr unsigned int maxSupportedQubitsForU32States() { return maxSupportedQubitsForStateIndex(); }

inline StateIndex checkedStateCount(unsigned int numQubits) {
	if(numQubits > maxSupportedQubitsForStateIndex())
		throw std::invalid_argument("Number of qubits exceeds supported range for state indexing");
	return StateIndex{1} << numQubits;
}

inline size_t checkedAmplitudeElementCount(unsigned int numQubits) {
	return static_cast<size_t>(checkedStateCount(numQubits)) * 2u;
}

}  // namespace tmfqs

#endif
