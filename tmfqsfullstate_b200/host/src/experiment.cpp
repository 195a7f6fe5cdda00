// Run-report serialisation and state comparison (src/tmfqs/experiment/).
#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

#include "tmfqs/experiment/comparison.h"
#include "tmfqs/experiment/report.h"
#include "tmfqs/register/quantum_register.h"
#include "tmfqs/storage/factory/storage_strategy_registry.h"

namespace tmfqs {
namespace experiment {
namespace {

std::string escapeJson(const std::string &v) {
	std::string o;
	for(char ch : v) {
		switch(ch) {
			case '\\': o += "\\\\"; break;
			case '"': o += "\\\""; break;
			case '\n': o += "\\n"; break;
			case '\r': o += "\\r"; break;
			case '\t': o += "\\t"; break;
			default: o += ch;
		}
	}
	return o;
}

void writeFile(const std::string &path, const std::string &text) {
	std::ofstream out(path);
	if(!out) throw std::runtime_error("Failed to open report output: " + path);
	out << text;
}

}  // namespace

// Same JSON layout as report.cpp:39-64.
std::string toJson(const RunReport &r) {
	std::ostringstream o;
	o << std::setprecision(17) << "{\n";
	o << "  \"qubits\": " << r.qubits << ",\n";
	o << "  \"operation_count\": " << r.operationCount << ",\n";
	o << "  \"strategy\": \"" << StorageStrategyRegistry::toString(r.strategy) << "\",\n";
	o << "  \"execution_seconds\": " << r.executionSeconds << ",\n";
	o << "  \"operations\": [";
	for(size_t i = 0; i < r.operations.size(); ++i) {
		const OperationTrace &t = r.operations[i];
		o << (i ? ",\n" : "\n") << "    {\"index\": " << t.index << ", \"name\": \"" << escapeJson(t.name)
		  << "\", \"seconds\": " << t.seconds << "}";
	}
	if(!r.operations.empty()) o << "\n  ";
	o << "]\n}\n";
	return o.str();
}

// Same CSV layout as report.cpp:66-87.
std::string toCsv(const RunReport &r) {
	std::ostringstream o;
	o << std::setprecision(17) << "qubits,strategy,total_operations,total_seconds,operation_index,operation_name,operation_seconds\n";
	const std::string strat = StorageStrategyRegistry::toString(r.strategy);
	if(r.operations.empty()) {
		o << r.qubits << ',' << strat << ',' << r.operationCount << ',' << r.executionSeconds << ",,,\n";
		return o.str();
	}
	for(const OperationTrace &t : r.operations)
		o << r.qubits << ',' << strat << ',' << r.operationCount << ',' << r.executionSeconds << ',' << t.index << ','
		  << t.name << ',' << t.seconds << '\n';
	return o.str();
}

void writeJsonReport(const RunReport &r, const std::string &path) { writeFile(path, toJson(r)); }
void writeCsvReport(const RunReport &r, const std::string &path) { writeFile(path, toCsv(r)); }

// Metrics of comparison.cpp:12-62.  When both states are device registers
// (simulation results without a lazy overlay), the comparison runs on the
// device (tmfqs_gpu_compare: every field equal to the host loop's, the sums
// replayed in the reference's order); otherwise both states are read once in
// bulk (the reference reads them one amplitude at a time).
StateComparison compareStates(const state::QuantumState &reference, const state::QuantumState &candidate) {
	if(reference.stateCount() != candidate.stateCount()) throw std::invalid_argument("Compared states must have the same state count");
	const QuantumRegister *rr = reference.registerOrNull(), *cr = candidate.registerOrNull();
	BackendComparison dev;
	if(rr && cr && rr->compareOnDevice(*cr, dev)) {
		StateComparison m;
		m.bitwiseEqual = dev.bitwiseEqual;
		m.maxAbsAmplitudeError = dev.maxAbsAmplitudeError;
		m.maxAbsComponentError = dev.maxAbsComponentError;
		m.rmseAmplitude = dev.rmseAmplitude;
		m.relL2 = dev.relL2;
		m.maxAbsProbabilityError = dev.maxAbsProbabilityError;
		m.totalProbabilityDiff = dev.totalProbabilityDiff;
		m.worstState = dev.worstState;
		return m;
	}
	return compareStatesOnHost(reference, candidate);
}

StateComparison compareStatesOnHost(const state::QuantumState &reference, const state::QuantumState &candidate) {
	if(reference.stateCount() != candidate.stateCount()) throw std::invalid_argument("Compared states must have the same state count");
	const AmplitudesVector ref = reference.amplitudes();
	const AmplitudesVector got = candidate.amplitudes();
	StateComparison m;
	m.bitwiseEqual = true;
	double diffSq = 0.0, refSq = 0.0, refTotal = 0.0, gotTotal = 0.0;
	const StateIndex N = reference.stateCount();
	for(StateIndex s = 0; s < N; ++s) {
		const double rr = ref[2 * s], ri = ref[2 * s + 1], gr = got[2 * s], gi = got[2 * s + 1];
		if(rr != gr || ri != gi) m.bitwiseEqual = false;
		const double dr = gr - rr, di = gi - ri;
		const double d2 = dr * dr + di * di;
		const double ae = std::sqrt(d2);
		if(ae > m.maxAbsAmplitudeError) {
			m.maxAbsAmplitudeError = ae;
			m.worstState = s;
		}
		m.maxAbsComponentError = std::max(m.maxAbsComponentError, std::max(std::abs(dr), std::abs(di)));
		diffSq += d2;
		refSq += rr * rr + ri * ri;
		const double rp = rr * rr + ri * ri, gp = gr * gr + gi * gi;
		refTotal += rp;
		gotTotal += gp;
		m.maxAbsProbabilityError = std::max(m.maxAbsProbabilityError, std::abs(gp - rp));
	}
	m.rmseAmplitude = std::sqrt(diffSq / static_cast<double>(N));
	m.relL2 = refSq == 0.0 ? 0.0 : std::sqrt(diffSq / refSq);
	m.totalProbabilityDiff = std::abs(gotTotal - refTotal);
	return m;
}

std::string toCsvRow(const std::string &circuit, const std::string &scenario, unsigned int qubits, const StateComparison &c) {
	std::ostringstream o;
	o << std::setprecision(17) << circuit << ',' << scenario << ',' << qubits << ',' << (c.bitwiseEqual ? "true" : "false")
	  << ',' << c.maxAbsAmplitudeError << ',' << c.maxAbsComponentError << ',' << c.relL2 << ',' << c.rmseAmplitude << ','
	  << c.maxAbsProbabilityError << ',' << c.totalProbabilityDiff << ',' << c.worstState;
	return o.str();
}

std::string toJson(const StateComparison &c) {
	std::ostringstream o;
	o << std::setprecision(17) << "{\"bitwiseEqual\":" << (c.bitwiseEqual ? "true" : "false")
	  << ",\"maxAbsAmplitudeError\":" << c.maxAbsAmplitudeError << ",\"maxAbsComponentError\":" << c.maxAbsComponentError
	  << ",\"relL2\":" << c.relL2 << ",\"rmseAmplitude\":" << c.rmseAmplitude
	  << ",\"maxAbsProbabilityError\":" << c.maxAbsProbabilityError << ",\"totalProbabilityDiff\":" << c.totalProbabilityDiff
	  << ",\"worstState\":" << c.worstState << "}";
	return o.str();
}

}  // namespace experiment
}  // namespace tmfqs
