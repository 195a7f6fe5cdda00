// Shared argument parsing of the grover / groverLazy / qftG command lines
// (the flags of examples/grover_cli.h:102-214 and examples/qftG.cpp:114-222,
// plus the device options of this build).
#ifndef TMFQS_HOST_CLI_COMMON_H
#define TMFQS_HOST_CLI_COMMON_H

#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>

#include "tmfqsfs.h"

namespace tmfqs_cli {

inline bool parseUnsigned(const char *t, unsigned int &out) {
	char *end = nullptr;
	const unsigned long v = std::strtoul(t, &end, 10);
	if(t == end || *end != '\0') return false;
	out = static_cast<unsigned int>(v);
	return true;
}

inline bool parseStateIndex(const char *t, tmfqs::StateIndex &out) {
	char *end = nullptr;
	const unsigned long long v = std::strtoull(t, &end, 10);
	if(t == end || *end != '\0') return false;
	out = static_cast<tmfqs::StateIndex>(v);
	return true;
}

inline bool parseDouble(const char *t, double &out) {
	char *end = nullptr;
	const double v = std::strtod(t, &end);
	if(t == end || *end != '\0') return false;
	out = v;
	return true;
}

inline tmfqs::StorageStrategyKind parseStrategy(const std::string &v) {
	if(v == "dense") return tmfqs::StorageStrategyKind::Dense;
	if(v == "blosc") return tmfqs::StorageStrategyKind::Blosc;
	if(v == "zfp") return tmfqs::StorageStrategyKind::Zfp;
	if(v == "auto") return tmfqs::StorageStrategyKind::Auto;
	if(v == "gpu") return tmfqs::StorageStrategyKind::Gpu;
	throw std::invalid_argument("Unknown strategy: " + v);
}

inline tmfqs::ZfpCompressionMode parseZfpMode(const std::string &v) {
	if(v == "rate") return tmfqs::ZfpCompressionMode::FixedRate;
	if(v == "precision") return tmfqs::ZfpCompressionMode::FixedPrecision;
	if(v == "accuracy") return tmfqs::ZfpCompressionMode::FixedAccuracy;
	throw std::invalid_argument("Unknown zfp mode: " + v);
}

// Options every CLI accepts.  Returns 1 if argv[i] was consumed (i advanced
// past its value), 0 if unknown, -1 on a malformed value.
struct CommonOptions {
	tmfqs::RegisterConfig cfg;
	bool hasSeed = false;
	uint32_t seed = 0;
};

inline int parseCommon(int argc, char *argv[], int &i, CommonOptions &o) {
	const std::string a = argv[i];
	auto next = [&]() -> const char * { return i + 1 < argc ? argv[++i] : nullptr; };
	unsigned int u = 0;
	double d = 0.0;
	const char *v = nullptr;
	if(a == "--strategy") {
		if(!(v = next())) return -1;
		o.cfg.strategy = parseStrategy(v);
	} else if(a == "--seed") {
		if(!(v = next()) || !parseUnsigned(v, u)) return -1;
		o.hasSeed = true;
		o.seed = u;
	} else if(a == "--precision") {
		if(!(v = next())) return -1;
		const std::string p = v;
		if(p == "fp64") o.cfg.gpu.precision = tmfqs::GpuPrecision::Fp64;
		else if(p == "fp32") o.cfg.gpu.precision = tmfqs::GpuPrecision::Fp32;
		else throw std::invalid_argument("Unknown precision: " + p);
	} else if(a == "--fast") {
		o.cfg.gpu.exact = false;
	} else if(a == "--no-fusion") {
		o.cfg.gpu.fusion = false;
	} else if(a == "--device") {
		if(!(v = next()) || !parseUnsigned(v, u)) return -1;
		o.cfg.gpu.deviceOrdinal = static_cast<int>(u);
	} else if(a == "--chunk-states") {
		if(!(v = next()) || !parseUnsigned(v, u) || u == 0) return -1;
		o.cfg.blosc.chunkStates = u;
		o.cfg.bloscOverrides.chunkStates = true;
	} else if(a == "--cache-slots") {
		if(!(v = next()) || !parseUnsigned(v, u) || u == 0) return -1;
		o.cfg.blosc.gateCacheSlots = u;
		o.cfg.bloscOverrides.gateCacheSlots = true;
	} else if(a == "--clevel") {
		if(!(v = next()) || !parseUnsigned(v, u)) return -1;
		o.cfg.blosc.clevel = static_cast<int>(u);
		o.cfg.bloscOverrides.clevel = true;
	} else if(a == "--nthreads") {
		if(!(v = next()) || !parseUnsigned(v, u) || u == 0) return -1;
		o.cfg.blosc.nthreads = o.cfg.zfp.nthreads = static_cast<int>(u);
		o.cfg.bloscOverrides.nthreads = o.cfg.zfpOverrides.nthreads = true;
	} else if(a == "--threshold-mb") {
		if(!(v = next()) || !parseUnsigned(v, u)) return -1;
		o.cfg.autoThresholdBytes = static_cast<size_t>(u) * 1024u * 1024u;
	} else if(a == "--zfp-mode") {
		if(!(v = next())) return -1;
		o.cfg.zfp.mode = parseZfpMode(v);
		o.cfg.zfpOverrides.mode = true;
	} else if(a == "--zfp-rate") {
		if(!(v = next()) || !parseDouble(v, d) || d <= 0.0) return -1;
		o.cfg.zfp.rate = d;
		o.cfg.zfpOverrides.rate = true;
	} else if(a == "--zfp-precision") {
		if(!(v = next()) || !parseUnsigned(v, u) || u == 0) return -1;
		o.cfg.zfp.precision = u;
		o.cfg.zfpOverrides.precision = true;
	} else if(a == "--zfp-accuracy") {
		if(!(v = next()) || !parseDouble(v, d) || d <= 0.0) return -1;
		o.cfg.zfp.accuracy = d;
		o.cfg.zfpOverrides.accuracy = true;
	} else if(a == "--zfp-chunk-states") {
		if(!(v = next()) || !parseUnsigned(v, u) || u == 0) return -1;
		o.cfg.zfp.chunkStates = u;
		o.cfg.zfpOverrides.chunkStates = true;
	} else if(a == "--zfp-cache-slots") {
		if(!(v = next()) || !parseUnsigned(v, u) || u == 0) return -1;
		o.cfg.zfp.gateCacheSlots = u;
		o.cfg.zfpOverrides.gateCacheSlots = true;
	} else {
		return 0;
	}
	return 1;
}

inline const char *commonUsage() {
	return "[--strategy gpu|auto|dense|blosc|zfp] [--seed N] [--precision fp64|fp32] [--fast] [--no-fusion] "
	       "[--device N] [--chunk-states N] [--cache-slots N] [--clevel N] [--nthreads N] [--threshold-mb N] "
	       "[--zfp-mode rate|precision|accuracy] [--zfp-rate R] [--zfp-precision B] [--zfp-accuracy A] "
	       "[--zfp-chunk-states N] [--zfp-cache-slots N]";
}

inline void printAvailable() {
	std::cout << "Available strategies: ";
	const auto names = tmfqs::StorageStrategyRegistry::listAvailable();
	for(size_t i = 0; i < names.size(); ++i) std::cout << names[i] << (i + 1 < names.size() ? ", " : "");
	std::cout << "\n";
}

}  // namespace tmfqs_cli

#endif
