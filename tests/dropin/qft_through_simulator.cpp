// QFT of QuantumState::randomPhase(n, seed) through the reference's own,
// unmodified sim::Simulator and QuantumRegister (one backend call per
// circuit operation), on the strategy named on the command line, with the
// integration patch applied (tests/dropin/apply_gpu_strategy.py).  Prints
// one JSON line: the Simulator's executionSeconds, the wall time of run()
// (input load + circuit + export of the result into a QuantumState), the
// result's totalProbability and measure(Mt19937RandomSource(seed)).
//
//   qft_through_simulator <num_qubits> <dense|gpu> [seed]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "tmfqsfs.h"

int main(int argc, char **argv) {
	if(argc < 3) {
		std::fprintf(stderr, "usage: %s <num_qubits> <dense|gpu> [seed]\n", argv[0]);
		return 1;
	}
	const unsigned n = static_cast<unsigned>(std::atoi(argv[1]));
	const std::string strategy = argv[2];
	const unsigned seed = argc > 3 ? static_cast<unsigned>(std::atoi(argv[3])) : 123456u;
	try {
		const tmfqs::state::QuantumState input = tmfqs::state::QuantumState::randomPhase(n, seed);
		tmfqs::sim::ExecutionConfig ex;
		ex.backend.strategy = strategy == "gpu" ? tmfqs::StorageStrategyKind::Gpu : tmfqs::StorageStrategyKind::Dense;
		const auto t0 = std::chrono::steady_clock::now();
		const tmfqs::sim::RunResult r = tmfqs::sim::Simulator(ex).run(tmfqs::circuit::makeQft(n), input);
		const auto t1 = std::chrono::steady_clock::now();
		tmfqs::Mt19937RandomSource rs(seed);
		const tmfqs::StateIndex measured = r.state.measure(rs);
		const double total = r.state.totalProbability();
		const auto t2 = std::chrono::steady_clock::now();
		std::printf("{\"n_qubits\": %u, \"strategy\": \"%s\", \"operations\": %zu, \"execution_seconds\": %.6f, "
		            "\"run_wall_seconds\": %.6f, \"measure_and_total_seconds\": %.6f, \"total_probability\": %.17g, "
		            "\"measured\": %llu}\n",
		            n, strategy.c_str(), r.report.operationCount, r.report.executionSeconds,
		            std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count(), total,
		            static_cast<unsigned long long>(measured));
	} catch(const std::exception &e) {
		std::fprintf(stderr, "qft_through_simulator: %s\n", e.what());
		return 2;
	}
	return 0;
}
