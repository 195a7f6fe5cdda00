// The B200 storage backend: an IStateBackend over the C ABI of
// libtmfqs_b200 (include/tmfqs_b200.h).
#ifndef TMFQS_HOST_STORAGE_GPU_GPU_STATE_BACKEND_H
#define TMFQS_HOST_STORAGE_GPU_GPU_STATE_BACKEND_H

#include <memory>

#include "tmfqs/config/register_config.h"
#include "tmfqs/storage/i_state_backend.h"

namespace tmfqs {

std::unique_ptr<IStateBackend> createGpuStateBackend(const RegisterConfig &cfg);
// Whether a CUDA device can host a state (probes the driver once).
bool isGpuStateBackendAvailable();

}  // namespace tmfqs

#endif
