// grover / groverLazy command line (examples/grover_cli.h:216-260 of the
// reference): builds makeGrover(n, marked), runs it through the Simulator and
// measures once.  Output lines match the reference's; --seed makes the
// measurement reproducible (without it the draw is seeded from
// std::random_device, as in the reference).
#ifndef TMFQS_HOST_CLI_GROVER_CLI_H
#define TMFQS_HOST_CLI_GROVER_CLI_H

#include <iostream>
#include <string>
#include <vector>

#include "cli_common.h"

namespace tmfqs_cli {

inline bool parseMarkedCsv(const char *text, std::vector<tmfqs::StateIndex> &out) {
	std::string token;
	const std::string s(text);
	for(size_t i = 0; i <= s.size(); ++i) {
		if(i == s.size() || s[i] == ',') {
			tmfqs::StateIndex v = 0;
			if(token.empty() || !parseStateIndex(token.c_str(), v)) return false;
			out.push_back(v);
			token.clear();
		} else {
			token.push_back(s[i]);
		}
	}
	return !out.empty();
}

inline int runGroverCli(int argc, char *argv[], const char *binary, const char *mode, bool materialized) {
	using namespace tmfqs;
	try {
		auto usage = [&] {
			std::cout << "Usage: ./" << binary << " <num_qubits> <marked_state[,marked_state...]> [--verbose] " << commonUsage() << "\n";
		};
		if(argc < 3) {
			usage();
			return 1;
		}
		unsigned int n = 0;
		if(!parseUnsigned(argv[1], n) || n == 0) {
			std::cout << "Number of qubits must be an integer >= 1\n";
			return 1;
		}
		if(n > maxSupportedQubitsForU32States()) {
			std::cout << "Number of qubits is too large for this example.\n";
			return 1;
		}
		std::vector<StateIndex> marked;
		if(!parseMarkedCsv(argv[2], marked)) {
			std::cout << "Marked states must be a comma-separated list of integers.\n";
			return 1;
		}
		CommonOptions o;
		bool verbose = false;
		for(int i = 3; i < argc; ++i) {
			if(std::string(argv[i]) == "--verbose") {
				verbose = true;
				continue;
			}
			const int r = parseCommon(argc, argv, i, o);
			if(r < 0) return 1;
			if(r == 0) {
				std::cout << "Unknown option: " << argv[i] << "\n";
				usage();
				return 1;
			}
		}
		Mt19937RandomSource rng;
		if(o.hasSeed) rng.reseed(o.seed);
		circuit::GroverCircuitOptions copts;
		copts.markedStates = BasisStateList(std::move(marked));
		copts.materializedDiffusion = materialized;
		const circuit::Circuit c = circuit::makeGrover(n, std::move(copts));
		if(o.cfg.workloadHint == StorageWorkloadHint::Generic) o.cfg.workloadHint = StorageWorkloadHint::Grover;
		sim::ExecutionConfig exec;
		exec.backend = o.cfg;
		exec.observability.traceOperations = false;
		const sim::RunResult run = sim::Simulator(exec).run(c, state::QuantumState::basis(n));
		const StateIndex result = run.state.measure(rng);
		std::cout << "Grover mode: " << mode << "\n";
		std::cout << "Resolved strategy: " << StorageStrategyRegistry::toString(StorageStrategyRegistry::resolve(n, o.cfg)) << "\n";
		std::cout << "Grover search result: " << result << "\n";
		if(verbose) {
			std::cout << "Circuit operations: " << run.report.operationCount << "\n";
			std::cout << "Execution seconds: " << run.report.executionSeconds << "\n";
		}
		return 0;
	} catch(const std::exception &ex) {
		std::cout << binary << " error: " << ex.what() << "\n";
		printAvailable();
		return 2;
	}
}

}  // namespace tmfqs_cli

#endif
