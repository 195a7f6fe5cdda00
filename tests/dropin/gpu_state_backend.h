// The B200 device backend for an unmodified TMFQS source tree
// (StorageStrategyKind::Gpu).  Installed into a copy of the reference tree as
// include/tmfqs/storage/gpu/gpu_state_backend.h by apply_gpu_strategy.py; it
// mirrors the factory functions of the reference's other backends
// (include/tmfqs/storage/dense/dense_state_backend.h:16).
#ifndef TMFQS_STORAGE_GPU_GPU_STATE_BACKEND_H
#define TMFQS_STORAGE_GPU_GPU_STATE_BACKEND_H

#include <memory>

#include "tmfqs/config/register_config.h"
#include "tmfqs/storage/i_state_backend.h"

namespace tmfqs {

/** @brief Creates the device backend (complex128, exact form, device 0). */
std::unique_ptr<IStateBackend> createGpuStateBackend(const RegisterConfig &cfg);
/** @brief Whether a CUDA device can hold a state (a handle can be created). */
bool isGpuStateBackendAvailable();
/** @brief Whether Dense registers are redirected to the device backend
 * (environment TMFQS_DENSE_BACKEND=gpu; a test-harness switch). */
bool denseRedirectedToGpu();

}  // namespace tmfqs

#endif
