// qftG command line (examples/qftG.cpp:234-291 of the reference): QFT of the
// pattern input (states 8x + x mod 2, uniform) or the random-phase input
// (seed 123456), then one measurement.  Output lines match the reference's;
// --seed seeds the measurement, --verbose adds the execution time.
#include <algorithm>
#include <iostream>
#include <string>
#include <vector>

#include "cli_common.h"

using namespace tmfqs;
using namespace tmfqs_cli;

namespace {

constexpr unsigned int kRandomPhaseSeed = 123456u;

// chooseInputStates + sanitizeStates (qftG.cpp:48-68).
std::vector<StateIndex> patternStates(StateIndex total) {
	std::vector<StateIndex> s;
	for(StateIndex x = 0;; ++x) {
		const StateIndex y = 8u * x + (x % 2u);
		if(y >= total) break;
		s.push_back(y);
	}
	std::sort(s.begin(), s.end());
	s.erase(std::unique(s.begin(), s.end()), s.end());
	return s;
}

}  // namespace

int main(int argc, char *argv[]) {
	try {
		auto usage = [] { std::cout << "Usage: ./qftG <num_qubits> [--input-family pattern|random-phase] [--verbose] " << commonUsage() << "\n"; };
		if(argc < 2) {
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
		bool randomPhase = false, verbose = false;
		CommonOptions o;
		for(int i = 2; i < argc; ++i) {
			const std::string a = argv[i];
			if(a == "--input-family") {
				if(i + 1 >= argc) return 1;
				const std::string f = argv[++i];
				if(f == "pattern") randomPhase = false;
				else if(f == "random-phase") randomPhase = true;
				else throw std::invalid_argument("Unknown input family: " + f);
				continue;
			}
			if(a == "--verbose") {
				verbose = true;
				continue;
			}
			const int r = parseCommon(argc, argv, i, o);
			if(r < 0) return 1;
			if(r == 0) {
				std::cout << "Unknown option: " << a << "\n";
				usage();
				return 1;
			}
		}
		const StateIndex total = checkedStateCount(n);
		if(o.cfg.workloadHint == StorageWorkloadHint::Generic) o.cfg.workloadHint = StorageWorkloadHint::Qft;
		state::QuantumState input;
		if(randomPhase) {
			input = state::QuantumState::randomPhase(n, kRandomPhaseSeed);
		} else {
			std::vector<StateIndex> sel = patternStates(total);
			if(sel.empty()) {
				std::cout << "No valid selected states were generated.\n";
				return 1;
			}
			input = state::QuantumState::uniformSubset(n, BasisStateList(std::move(sel)));
		}
		sim::ExecutionConfig exec;
		exec.backend = o.cfg;
		const sim::RunResult run = sim::Simulator(exec).run(circuit::makeQft(n), input);
		Mt19937RandomSource rng;
		if(o.hasSeed) rng.reseed(o.seed);
		const StateIndex k = run.state.measure(rng);
		std::cout << "Input family: " << (randomPhase ? "random-phase" : "pattern") << "\n";
		if(randomPhase) std::cout << "Random seed: " << kRandomPhaseSeed << "\n";
		std::cout << "Measured state (k): " << k << "\n";
		std::cout << "Calculated r (N/k): ";
		if(k == 0) std::cout << "undefined (division by zero)\n";
		else std::cout << (static_cast<double>(total) / static_cast<double>(k)) << "\n";
		if(verbose) std::cout << "Execution seconds: " << run.report.executionSeconds << "\n";
		return 0;
	} catch(const std::exception &ex) {
		std::cout << "qftG error: " << ex.what() << "\n";
		printAvailable();
		return 2;
	}
}
