// Storage backend interface (include/tmfqs/storage/i_state_backend.h:22-164),
// plus optional batched hooks a device backend implements so that
// QuantumRegister and Simulator can keep whole circuits and reductions on the
// device.  Every hook has a default that reports "not supported"; callers
// then fall back to the reference's per-operation behaviour.
#ifndef TMFQS_HOST_STORAGE_I_STATE_BACKEND_H
#define TMFQS_HOST_STORAGE_I_STATE_BACKEND_H

#include <functional>
#include <iosfwd>
#include <memory>
#include <string>
#include <vector>

#include "tmfqs/core/types.h"
#include "tmfqs/gates/quantum_gate.h"

namespace tmfqs {

using AmplitudeChunkVisitor = std::function<void(StateIndex baseState, const double *data, size_t elemCount)>;

// One operation of a batched gate run (the gate-like alternatives of
// circuit::Operation).
struct BackendOp {
	enum class Kind { Hadamard, PauliX, ControlledNot, ControlledPhaseShift, Swap, MatrixGate, PhaseFlip };
	Kind kind = Kind::Hadamard;
	QubitIndex q0 = 0;  // target / control / first
	QubitIndex q1 = 0;  // target / second
	double theta = 0.0;
	StateIndex state = 0;
	const QuantumGate *gate = nullptr;
	const QubitList *targets = nullptr;
};

// QuantumRegister's lazy affine overlay (quantum_register.h:218-224).
struct AffineOverlay {
	Amplitude scale{1.0, 0.0};
	Amplitude bias{0.0, 0.0};
};

// The register-side state a Grover run updates.
struct RegisterSideState {
	bool hasSum = false;
	Amplitude sum{0.0, 0.0};
	bool overlayActive = false;
	AffineOverlay overlay;
};

// One timed device pass of a traced run (see IStateBackend::endPassTrace).
struct BackendPassTrace {
	std::string kind;       // "fused", "permute", "gate", "reduce", "grover"
	uint64_t segment = 0;   // the markPassSegment() number it ran under
	uint64_t firstOp = 0;   // first operation within its applyOperationRun call
	unsigned opCount = 0;   // operations it applied (0: not an operation run)
	double seconds = 0.0;   // device time (CUDA events)
};

// experiment::StateComparison's fields, filled by a backend that compares two
// of its states in place.
struct BackendComparison {
	bool bitwiseEqual = false;
	double maxAbsAmplitudeError = 0.0, maxAbsComponentError = 0.0, rmseAmplitude = 0.0, relL2 = 0.0,
	       maxAbsProbabilityError = 0.0, totalProbabilityDiff = 0.0;
	StateIndex worstState = 0u;
};

class IStateBackend {
	public:
		virtual ~IStateBackend() = default;
		virtual std::unique_ptr<IStateBackend> clone() const = 0;

		virtual void initZero(unsigned int numQubits) = 0;
		virtual void initBasis(unsigned int numQubits, StateIndex initState, Amplitude amp) = 0;
		virtual void initUniformSuperposition(unsigned int numQubits, const BasisStateList &basisStates) = 0;
		virtual void loadAmplitudes(unsigned int numQubits, AmplitudesVector amplitudes) = 0;
		virtual void exportAmplitudes(AmplitudesVector &out) const = 0;
		virtual void forEachAmplitudeChunk(const AmplitudeChunkVisitor &visitor) const = 0;

		virtual Amplitude amplitude(StateIndex state) const = 0;
		virtual void setAmplitude(StateIndex state, Amplitude amp) = 0;
		virtual double probability(StateIndex state) const = 0;
		virtual double totalProbability() const = 0;
		virtual StateIndex sampleMeasurement(double rnd) const = 0;
		virtual void printNonZeroStates(std::ostream &os, double epsilon) const = 0;

		virtual void phaseFlipBasisState(StateIndex state) = 0;
		virtual void inversionAboutMean() = 0;
		virtual void inversionAboutMean(Amplitude mean) = 0;
		virtual void applyAffineTransform(Amplitude scale, Amplitude bias) = 0;
		virtual void applyHadamard(QubitIndex qubit) = 0;
		virtual void applyPauliX(QubitIndex qubit) = 0;
		virtual void applyControlledPhaseShift(QubitIndex controlQubit, QubitIndex targetQubit, double theta) = 0;
		virtual void applyControlledNot(QubitIndex controlQubit, QubitIndex targetQubit) = 0;
		virtual void applyGate(const QuantumGate &gate, const QubitList &qubits) = 0;

		virtual void beginOperationBatch() {}
		virtual void endOperationBatch() {}

		// ---- optional device hooks (defaults: unsupported) ----
		// Applies a validated run of gate operations; swaps act as one
		// permutation (same result as QuantumRegister's three CNOTs).
		virtual bool applyOperationRun(const std::vector<BackendOp> &) { return false; }
		// The reference's sequential sums over logical amplitudes
		// (scale*a+bias when `overlay` is non-null), bit for bit.
		virtual bool logicalAmplitudeSum(const AffineOverlay *, Amplitude &) const { return false; }
		virtual bool logicalTotalProbability(const AffineOverlay *, double &) const { return false; }
		virtual bool logicalSample(const AffineOverlay *, double, StateIndex &) const { return false; }
		// `iterations` Grover iterations over sorted unique marked states with
		// QuantumRegister's exact semantics, updating `side`.
		virtual bool runGroverIterations(RegisterSideState &, const std::vector<StateIndex> &, uint64_t, bool) { return false; }
		// Per-pass device timing for traced runs: begin, mark each backend call
		// (segment), then collect the passes; the batching hooks stay in use.
		virtual bool beginPassTrace() { return false; }
		virtual uint64_t markPassSegment() { return 0; }
		virtual bool endPassTrace(std::vector<BackendPassTrace> &) { return false; }
		// experiment::compareStates on two states of this backend, in place.
		virtual bool compareWith(const IStateBackend &, BackendComparison &) const { return false; }
};

}  // namespace tmfqs

#endif
