// Register and storage configuration (include/tmfqs/config/register_config.h:9-109)
// with the device strategy.  In this build the only backend is the B200 one:
// `Gpu` is the default strategy, `Auto` resolves to it, and Dense/Blosc/Zfp
// report themselves unavailable, as the reference does for backends it was
// built without (storage_strategy_registry.cpp:99-108).
#ifndef TMFQS_HOST_CONFIG_REGISTER_CONFIG_H
#define TMFQS_HOST_CONFIG_REGISTER_CONFIG_H

#include <cstddef>

namespace tmfqs {

enum class StorageStrategyKind { Dense, Blosc, Zfp, Auto, Gpu };

enum class StorageWorkloadHint { Generic, Grover, Qft };

enum class ZfpCompressionMode { FixedRate, FixedPrecision, FixedAccuracy };

struct BloscConfig {
	size_t chunkStates = 32768;
	int clevel = 1;
	int nthreads = 4;
	int compcode = 1;
	bool useShuffle = true;
	size_t gateCacheSlots = 8;
};

struct BloscTuningOverrides {
	bool chunkStates = false;
	bool clevel = false;
	bool nthreads = false;
	bool gateCacheSlots = false;
};

struct ZfpConfig {
	ZfpCompressionMode mode = ZfpCompressionMode::FixedPrecision;
	double rate = 32.0;
	unsigned int precision = 40;
	double accuracy = 1e-8;
	size_t chunkStates = 32768;
	int nthreads = 4;
	size_t gateCacheSlots = 8;
};

struct ZfpTuningOverrides {
	bool mode = false;
	bool rate = false;
	bool precision = false;
	bool accuracy = false;
	bool chunkStates = false;
	bool nthreads = false;
	bool gateCacheSlots = false;
};

// Device storage settings.
enum class GpuPrecision {
	Fp64,  // complex128, bit-identical to the reference's Dense backend
	Fp32   // complex64 amplitudes, FP64 twiddles and reductions
};

struct GpuConfig {
	GpuPrecision precision = GpuPrecision::Fp64;
	int deviceOrdinal = 0;
	// FP64 only: false applies each controlled-phase chain as one FP64 twiddle
	// (about 1e-15 relative error per pass) instead of gate by gate.
	bool exact = true;
	// Fuse consecutive gates into multi-gate passes (results are unchanged).
	bool fusion = true;
};

struct RegisterConfig {
	StorageStrategyKind strategy = StorageStrategyKind::Gpu;
	size_t autoThresholdBytes = 8u * 1024u * 1024u;
	StorageWorkloadHint workloadHint = StorageWorkloadHint::Generic;
	BloscConfig blosc;
	BloscTuningOverrides bloscOverrides;
	ZfpConfig zfp;
	ZfpTuningOverrides zfpOverrides;
	GpuConfig gpu;
};

}  // namespace tmfqs

#endif
