// Umbrella header of the TMFQS API (include/tmfqsfs.h of the reference).
#ifndef TMFQSFS_INCLUDE
#define TMFQSFS_INCLUDE

#include "tmfqs/circuit/circuit.h"
#include "tmfqs/config/register_config.h"
#include "tmfqs/core/constants.h"
#include "tmfqs/core/math.h"
#include "tmfqs/core/random.h"
#include "tmfqs/core/state_space.h"
#include "tmfqs/core/types.h"
#include "tmfqs/core/validation.h"
#include "tmfqs/experiment/comparison.h"
#include "tmfqs/experiment/report.h"
#include "tmfqs/gates/quantum_gate.h"
#include "tmfqs/register/quantum_register.h"
#include "tmfqs/sim/simulator.h"
#include "tmfqs/state/quantum_state.h"
#include "tmfqs/storage/factory/state_backend_factory.h"
#include "tmfqs/storage/factory/storage_strategy_registry.h"
#include "tmfqs/storage/gpu/gpu_state_backend.h"

#endif
