// Quantum register (include/tmfqs/register/quantum_register.h:24-251): owns a
// storage backend and the lazy affine overlay / cached logical amplitude sum
// that sit above it.
#ifndef TMFQS_HOST_REGISTER_QUANTUM_REGISTER_H
#define TMFQS_HOST_REGISTER_QUANTUM_REGISTER_H

#include <cstddef>
#include <functional>
#include <iosfwd>
#include <memory>
#include <optional>
#include <vector>

#include "tmfqs/config/register_config.h"
#include "tmfqs/core/types.h"
#include "tmfqs/gates/quantum_gate.h"
#include "tmfqs/storage/i_state_backend.h"

namespace tmfqs {

class IRandomSource;
class QuantumRegister;
namespace sim {
class Simulator;
}
namespace state {
class QuantumState;
}
namespace experiment {
struct StateComparison;
StateComparison compareStates(const state::QuantumState &reference, const state::QuantumState &candidate);
}

class QuantumRegister {
	public:
		QuantumRegister();
		explicit QuantumRegister(unsigned int numQubits, const RegisterConfig &cfg = {});
		QuantumRegister(unsigned int numQubits, StateIndex initState, const RegisterConfig &cfg = {});
		QuantumRegister(unsigned int numQubits, StateIndex initState, Amplitude amp, const RegisterConfig &cfg = {});
		QuantumRegister(unsigned int numQubits, AmplitudesVector amplitudes, const RegisterConfig &cfg = {});
		QuantumRegister(const QuantumRegister &);
		QuantumRegister(QuantumRegister &&) noexcept = default;
		QuantumRegister &operator=(const QuantumRegister &);
		QuantumRegister &operator=(QuantumRegister &&) noexcept = default;
		~QuantumRegister();

		unsigned int qubitCount() const;
		StateIndex stateCount() const;
		size_t amplitudeElementCount() const;

		double probability(StateIndex state) const;
		double totalProbability() const;
		Amplitude amplitude(StateIndex state) const;
		AmplitudesVector amplitudes() const;
		StateIndex measure(IRandomSource &randomSource) const;

		void setAmplitude(StateIndex state, Amplitude amp);
		void loadAmplitudes(AmplitudesVector amplitudes);
		void initUniformSuperposition(const BasisStateList &basisStates);
		StorageStrategyKind storageStrategy() const;

		void printStatesVector(double epsilon = 1e-12) const;
		friend std::ostream &operator<<(std::ostream &os, const QuantumRegister &reg);

		void applyGate(const QuantumGate &gate, const QubitList &qubits);
		void applyPhaseFlipBasisState(StateIndex state);
		void applyInversionAboutMean();
		void applyInversionAboutMean(Amplitude mean);
		void applyInversionAboutMeanMaterialized();
		void applyInversionAboutMeanMaterialized(Amplitude mean);
		void applyHadamard(QubitIndex qubit);
		void applyPauliX(QubitIndex qubit);
		void applyControlledPhaseShift(QubitIndex controlQubit, QubitIndex targetQubit, double theta);
		void applyControlledNot(QubitIndex controlQubit, QubitIndex targetQubit);
		void applySwap(QubitIndex qubit1, QubitIndex qubit2);
		void beginOperationBatch();
		void endOperationBatch();

		// Batched forms used by sim::Simulator.  Each has exactly the effect of
		// the corresponding sequence of single calls above (validation order and
		// partial application on error included); a backend that supports them
		// runs the whole batch on the device.
		void applyOperationRun(const std::vector<BackendOp> &ops);
		void applyGroverIterations(const std::vector<StateIndex> &sortedMarked, uint64_t iterations, bool materialized);

	private:
		friend class sim::Simulator;
		friend experiment::StateComparison experiment::compareStates(const state::QuantumState &, const state::QuantumState &);
		// Device pass traces (Simulator with traceOperations) and in-place
		// comparison of two device states without a lazy overlay.
		bool beginPassTrace() { return backend_ && backend_->beginPassTrace(); }
		uint64_t markPassSegment() { return backend_->markPassSegment(); }
		bool endPassTrace(std::vector<BackendPassTrace> &out) { return backend_->endPassTrace(out); }
		bool compareOnDevice(const QuantumRegister &candidate, BackendComparison &out) const {
			if(!backend_ || !candidate.backend_ || affineOverlayActive_ || candidate.affineOverlayActive_) return false;
			if(numQubits_ != candidate.numQubits_) return false;
			return backend_->compareWith(*candidate.backend_, out);
		}

		unsigned int numQubits_ = 0;
		StateIndex numStates_ = 0;
		RegisterConfig config_{};
		StorageStrategyKind resolvedStrategy_ = StorageStrategyKind::Gpu;
		std::unique_ptr<IStateBackend> backend_;
		mutable std::optional<Amplitude> cachedLogicalAmplitudeSum_;
		Amplitude affineScale_{1.0, 0.0};
		Amplitude affineBias_{0.0, 0.0};
		bool affineOverlayActive_ = false;

		void initializeBackend(unsigned int qubits);
		void requireInitialized(const char *operation) const;
		void resetAffineOverlay();
		void flushAffineOverlay();
		Amplitude applyAffineOverlay(Amplitude backendAmplitude) const;
		Amplitude removeAffineOverlay(Amplitude logicalAmplitude) const;
		Amplitude logicalAmplitudeSum() const;
		void visitLogicalAmplitudeChunks(const std::function<void(StateIndex, const double *, size_t)> &visitor) const;
		AmplitudesVector snapshotLogicalAmplitudes() const;
		const AffineOverlay *overlayOrNull(AffineOverlay &storage) const;
};

}  // namespace tmfqs

#endif
