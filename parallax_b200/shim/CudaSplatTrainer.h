// CudaSplatTrainer.h -- the reference engine's splat-training entry points,
// implemented on the B200 core (libpxs.so, include/pxs.h).
//
// Compiled into the engine in place of its Vulkan trainer: this header adds
// only the CUDA backend factory; trainSplatsOnGpu and splatGpuAvailability
// keep the declarations of parallax/splat/VulkanSplatTrainer.h
// (engine/native/cpp/include/parallax/splat/VulkanSplatTrainer.h:15-37), so
// callers such as Pipeline::Impl::runSplatTraining are unchanged.
#pragma once

#include <memory>

#include "parallax/splat/SplatTrainer.h"
#include "parallax/splat/VulkanSplatTrainer.h"

namespace parallax {

/// A SplatBackend (SplatTrainer.h:114-127) whose renderAndAccumulate and
/// render run on the GPU. Each call converts the cloud to the core's
/// component-major layout, runs on a context owned by the backend, and adds
/// the gradients into `gradients` (resized first when its size does not match
/// the cloud, as rasterizeSplatsBackward does). Throws std::runtime_error when
/// the device fails, since the interface has no error channel. Returns null
/// when no usable device is present.
std::unique_ptr<SplatBackend> makeCudaSplatBackend(int device = 0);

}  // namespace parallax
