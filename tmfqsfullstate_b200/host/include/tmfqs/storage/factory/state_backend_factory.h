#ifndef TMFQS_HOST_STORAGE_FACTORY_STATE_BACKEND_FACTORY_H
#define TMFQS_HOST_STORAGE_FACTORY_STATE_BACKEND_FACTORY_H

#include <memory>

#include "tmfqs/config/register_config.h"
#include "tmfqs/storage/factory/storage_strategy_registry.h"

namespace tmfqs {

// include/tmfqs/storage/factory/state_backend_factory.h:14-31.
class StateBackendFactory {
	public:
		static std::unique_ptr<IStateBackend> create(unsigned int numQubits, const RegisterConfig &cfg);
		static BackendSelection createSelection(unsigned int numQubits, const RegisterConfig &cfg);
};

inline StorageStrategyKind resolveStorageStrategy(unsigned int n, const RegisterConfig &cfg) { return StorageStrategyRegistry::resolve(n, cfg); }
inline BackendSelection createBackendSelection(unsigned int n, const RegisterConfig &cfg) { return StateBackendFactory::createSelection(n, cfg); }
inline std::unique_ptr<IStateBackend> createBackend(unsigned int n, const RegisterConfig &cfg) { return StateBackendFactory::create(n, cfg); }
inline bool isStrategyAvailable(StorageStrategyKind kind) { return StorageStrategyRegistry::isAvailable(kind); }
inline std::vector<std::string> listAvailableStrategies() { return StorageStrategyRegistry::listAvailable(); }
inline std::string storageStrategyToString(StorageStrategyKind kind) { return StorageStrategyRegistry::toString(kind); }

}  // namespace tmfqs

#endif
