// A circuit through the reference's own, unmodified sim::Simulator and
// QuantumRegister (one backend call per circuit operation), on the strategy
// named on the command line, with the integration patch applied
// (tests/dropin/apply_gpu_strategy.py).  Prints one JSON line: the
// Simulator's executionSeconds, the wall time of run() (input load + circuit +
// export of the result into a QuantumState), the result's totalProbability
// and measure(Mt19937RandomSource(seed)).
//
//   qft_through_simulator <num_qubits> <dense|gpu> [seed]
//       QFT of QuantumState::randomPhase(n, seed) (the qftG input)
//   qft_through_simulator grover <num_qubits> <dense|gpu> <marked> <materialized 0|1> [seed]
//       Grover search from |0...0> (circuit::makeGrover)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "tmfqsfs.h"

namespace {

tmfqs::StorageStrategyKind strategyOf(const std::string &s) {
	return s == "gpu" ? tmfqs::StorageStrategyKind::Gpu : tmfqs::StorageStrategyKind::Dense;
}

}  // namespace

int main(int argc, char **argv) {
	const bool grover = argc > 1 && std::strcmp(argv[1], "grover") == 0;
	const int a0 = grover ? 2 : 1;
	if(argc < a0 + 2 || (grover && argc < a0 + 4)) {
		std::fprintf(stderr, "usage: %s [grover] <num_qubits> <dense|gpu> [marked materialized] [seed]\n", argv[0]);
		return 1;
	}
	const unsigned n = static_cast<unsigned>(std::atoi(argv[a0]));
	const std::string strategy = argv[a0 + 1];
	const int sarg = grover ? a0 + 4 : a0 + 2;
	const unsigned seed = argc > sarg ? static_cast<unsigned>(std::atoi(argv[sarg])) : 123456u;
	try {
		tmfqs::circuit::Circuit circuit(n);
		tmfqs::state::QuantumState input;
		if(grover) {
			tmfqs::circuit::GroverCircuitOptions o;
			o.markedStates = tmfqs::BasisStateList{static_cast<tmfqs::StateIndex>(std::strtoull(argv[a0 + 2], nullptr, 10))};
			o.materializedDiffusion = std::atoi(argv[a0 + 3]) != 0;
			circuit = tmfqs::circuit::makeGrover(n, std::move(o));
			input = tmfqs::state::QuantumState::basis(n);
		} else {
			circuit = tmfqs::circuit::makeQft(n);
			input = tmfqs::state::QuantumState::randomPhase(n, seed);
		}
		tmfqs::sim::ExecutionConfig ex;
		ex.backend.strategy = strategyOf(strategy);
		const auto t0 = std::chrono::steady_clock::now();
		const tmfqs::sim::RunResult r = tmfqs::sim::Simulator(ex).run(circuit, input);
		const auto t1 = std::chrono::steady_clock::now();
		tmfqs::Mt19937RandomSource rs(seed);
		const tmfqs::StateIndex measured = r.state.measure(rs);
		const double total = r.state.totalProbability();
		const auto t2 = std::chrono::steady_clock::now();
		std::printf("{\"circuit\": \"%s\", \"n_qubits\": %u, \"strategy\": \"%s\", \"operations\": %zu, "
		            "\"execution_seconds\": %.6f, \"run_wall_seconds\": %.6f, \"measure_and_total_seconds\": %.6f, "
		            "\"total_probability\": %.17g, \"measured\": %llu}\n",
		            grover ? "grover" : "qft", n, strategy.c_str(), r.report.operationCount, r.report.executionSeconds,
		            std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count(), total,
		            static_cast<unsigned long long>(measured));
	} catch(const std::exception &e) {
		std::fprintf(stderr, "qft_through_simulator: %s\n", e.what());
		return 2;
	}
	return 0;
}
