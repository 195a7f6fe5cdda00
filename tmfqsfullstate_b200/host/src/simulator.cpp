// sim::Simulator (src/tmfqs/sim/simulator.cpp:17-96), with a batching pass:
// maximal runs of gate operations go to QuantumRegister::applyOperationRun
// (fused multi-gate passes on the device) and repeated Grover iterations --
// sorted unique phase flips followed by an inversion about the mean -- go to
// QuantumRegister::applyGroverIterations.  Both have exactly the results of
// executing the operations one by one.  With traceOperations on, a backend
// that times its device passes (CUDA events) keeps the batching, and the
// report holds one trace per device pass: its first circuit operation, the
// operations it applied, and its device time.  Other backends run the
// operations one at a time, each synchronised, so per-operation times measure
// device work rather than enqueue time.
#include "tmfqs/sim/simulator.h"

#include <algorithm>
#include <chrono>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "tmfqs/register/quantum_register.h"
#include "tmfqs/storage/factory/storage_strategy_registry.h"

namespace tmfqs {
namespace sim {
namespace {

using Clock = std::chrono::steady_clock;

void executeOperation(QuantumRegister &reg, const circuit::Operation &operation) {
	std::visit(
		[&](const auto &op) {
			using Op = std::decay_t<decltype(op)>;
			if constexpr(std::is_same<Op, circuit::Hadamard>::value) reg.applyHadamard(op.target);
			else if constexpr(std::is_same<Op, circuit::PauliX>::value) reg.applyPauliX(op.target);
			else if constexpr(std::is_same<Op, circuit::ControlledNot>::value) reg.applyControlledNot(op.control, op.target);
			else if constexpr(std::is_same<Op, circuit::ControlledPhaseShift>::value)
				reg.applyControlledPhaseShift(op.control, op.target, op.theta);
			else if constexpr(std::is_same<Op, circuit::Swap>::value) reg.applySwap(op.first, op.second);
			else if constexpr(std::is_same<Op, circuit::MatrixGate>::value) reg.applyGate(op.gate, op.targets);
			else if constexpr(std::is_same<Op, circuit::PhaseFlipBasisState>::value) reg.applyPhaseFlipBasisState(op.state);
			else if constexpr(std::is_same<Op, circuit::InversionAboutMean>::value) {
				if(op.materialized) reg.applyInversionAboutMeanMaterialized();
				else reg.applyInversionAboutMean();
			}
		},
		operation);
}

bool isFlip(const circuit::Operation &op) { return std::holds_alternative<circuit::PhaseFlipBasisState>(op); }
bool isInversion(const circuit::Operation &op) { return std::holds_alternative<circuit::InversionAboutMean>(op); }

// A Grover iteration starting at i: one or more flips on strictly increasing
// states, then an inversion.  Returns its length (0 if none).
size_t groverPattern(const std::vector<circuit::Operation> &ops, size_t i, std::vector<StateIndex> &marked, bool &materialized) {
	marked.clear();
	size_t j = i;
	while(j < ops.size() && isFlip(ops[j])) {
		const StateIndex s = std::get<circuit::PhaseFlipBasisState>(ops[j]).state;
		if(!marked.empty() && s <= marked.back()) return 0;
		marked.push_back(s);
		++j;
	}
	if(marked.empty() || j >= ops.size() || !isInversion(ops[j])) return 0;
	materialized = std::get<circuit::InversionAboutMean>(ops[j]).materialized;
	return j - i + 1;
}

bool samePattern(const std::vector<circuit::Operation> &ops, size_t i, size_t len, const std::vector<StateIndex> &marked, bool materialized) {
	if(i + len > ops.size()) return false;
	for(size_t k = 0; k < marked.size(); ++k) {
		if(!isFlip(ops[i + k]) || std::get<circuit::PhaseFlipBasisState>(ops[i + k]).state != marked[k]) return false;
	}
	const auto &last = ops[i + marked.size()];
	return isInversion(last) && std::get<circuit::InversionAboutMean>(last).materialized == materialized;
}

// Converts a gate-like operation; false for inversions.
bool toBackendOp(const circuit::Operation &operation, BackendOp &out) {
	bool ok = true;
	std::visit(
		[&](const auto &op) {
			using Op = std::decay_t<decltype(op)>;
			using K = BackendOp::Kind;
			if constexpr(std::is_same<Op, circuit::Hadamard>::value) out = BackendOp{K::Hadamard, op.target};
			else if constexpr(std::is_same<Op, circuit::PauliX>::value) out = BackendOp{K::PauliX, op.target};
			else if constexpr(std::is_same<Op, circuit::ControlledNot>::value) out = BackendOp{K::ControlledNot, op.control, op.target};
			else if constexpr(std::is_same<Op, circuit::ControlledPhaseShift>::value)
				out = BackendOp{K::ControlledPhaseShift, op.control, op.target, op.theta};
			else if constexpr(std::is_same<Op, circuit::Swap>::value) out = BackendOp{K::Swap, op.first, op.second};
			else if constexpr(std::is_same<Op, circuit::MatrixGate>::value) {
				out = BackendOp{K::MatrixGate};
				out.gate = &op.gate;
				out.targets = &op.targets;
			} else if constexpr(std::is_same<Op, circuit::PhaseFlipBasisState>::value) {
				out = BackendOp{K::PhaseFlip};
				out.state = op.state;
			} else ok = false;
		},
		operation);
	return ok;
}

// A backend call of a traced run: the circuit operations [first, first + count).
struct Segment {
	size_t first, count;
};

// `mark` (traced runs) is called before each backend call with its operation range.
template <typename Mark>
void executeBatched(QuantumRegister &reg, const std::vector<circuit::Operation> &ops, Mark &&mark) {
	std::vector<StateIndex> marked;
	bool materialized = false;
	size_t i = 0;
	while(i < ops.size()) {
		const size_t len = groverPattern(ops, i, marked, materialized);
		if(len) {
			uint64_t reps = 1;
			while(samePattern(ops, i + reps * len, len, marked, materialized)) ++reps;
			mark(i, reps * len);
			reg.applyGroverIterations(marked, reps, materialized);
			i += reps * len;
			continue;
		}
		std::vector<BackendOp> run;
		BackendOp b;
		const size_t first = i;
		while(i < ops.size() && toBackendOp(ops[i], b)) {
			std::vector<StateIndex> probe;
			bool m = false;
			if(isFlip(ops[i]) && groverPattern(ops, i, probe, m)) break;
			run.push_back(b);
			++i;
		}
		if(!run.empty()) {
			mark(first, run.size());
			reg.applyOperationRun(run);
			continue;
		}
		mark(i, 1);
		executeOperation(reg, ops[i]);
		++i;
	}
}

// "fused: h, controlled_phase x15, h" -- the operation names of [first, first + count), repeats folded.
std::string passName(const std::string &kind, const std::vector<circuit::Operation> &ops, size_t first, size_t count) {
	std::string out = kind + ":";
	size_t k = first;
	const size_t end = std::min(ops.size(), first + count);
	bool firstName = true;
	while(k < end) {
		const std::string name = circuit::operationName(ops[k]);
		size_t r = 1;
		while(k + r < end && circuit::operationName(ops[k + r]) == name) ++r;
		out += (firstName ? " " : ", ") + name + (r > 1 ? " x" + std::to_string(r) : "");
		firstName = false;
		k += r;
	}
	return out;
}

}  // namespace

Simulator::Simulator(ExecutionConfig config) : config_(std::move(config)) {}

const ExecutionConfig &Simulator::config() const noexcept { return config_; }

RunResult Simulator::run(const circuit::Circuit &circuit, const state::QuantumState &initialState) const {
	if(circuit.qubitCount() != initialState.qubitCount()) throw std::invalid_argument("Circuit and initial state qubit counts differ");
	RegisterConfig cfg = config_.backend;
	QuantumRegister reg = initialState.materialize(cfg);

	experiment::RunReport report;
	report.qubits = circuit.qubitCount();
	report.operationCount = circuit.operationCount();
	report.strategy = StorageStrategyRegistry::resolve(circuit.qubitCount(), cfg);

	const auto start = Clock::now();
	reg.beginOperationBatch();
	bool open = true;
	try {
		const std::vector<circuit::Operation> &ops = circuit.operations();
		if(config_.observability.traceOperations && reg.beginPassTrace()) {
			std::vector<Segment> segments;  // segment s (numbered from 1) = segments[s - 1]
			executeBatched(reg, ops, [&](size_t first, size_t count) {
				reg.markPassSegment();
				segments.push_back({first, count});
			});
			reg.endOperationBatch();
			std::vector<BackendPassTrace> passes;
			reg.endPassTrace(passes);
			for(const BackendPassTrace &p : passes) {
				if(p.segment == 0 || p.segment > segments.size()) continue;
				const Segment &sg = segments[p.segment - 1];
				const size_t first = p.opCount ? sg.first + p.firstOp : sg.first;
				const size_t count = p.opCount ? p.opCount : sg.count;
				report.operations.push_back({first, passName(p.kind, ops, first, count), p.seconds});
			}
		} else if(config_.observability.traceOperations) {
			for(size_t i = 0; i < ops.size(); ++i) {
				const auto t0 = Clock::now();
				executeOperation(reg, ops[i]);
				reg.endOperationBatch();
				report.operations.push_back({i, circuit::operationName(ops[i]), std::chrono::duration<double>(Clock::now() - t0).count()});
			}
		} else {
			executeBatched(reg, ops, [](size_t, size_t) {});
		}
		reg.endOperationBatch();
		open = false;
	} catch(...) {
		if(open) {
			try {
				reg.endOperationBatch();
			} catch(...) {
			}
		}
		throw;
	}
	report.executionSeconds = std::chrono::duration<double>(Clock::now() - start).count();
	return {state::QuantumState::fromRegister(std::move(reg)), std::move(report)};
}

}  // namespace sim
}  // namespace tmfqs
