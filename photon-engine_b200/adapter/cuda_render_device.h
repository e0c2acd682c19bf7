// cuda_render_device.h — the photon engine's RenderDevice over the B200 C ABI (photon_cuda.h).
//
// This is the drop-in: a maintainer adds cuda_render_device.{h,cpp} to the reference engine's
// tree (next to src/engine/render_device.cpp) and links libphoton_cuda.so; createDevice("cuda:N")
// then returns this device (render_device.cpp:110-157), and RenderSession, the CLI and the app
// drive it through the RenderDevice interface (src/engine/render_device.h:65-86) unchanged.
#pragma once

#include "engine/render_device.h"

#include <memory>
#include <string>

namespace photon {

/// The B200 device of CUDA ordinal @p ordinal, or nullptr with @p error filled (no device, no
/// driver, library missing), as createDevice reports unusable ids.
std::unique_ptr<RenderDevice> createCudaRenderDevice(int ordinal, std::string* error = nullptr);

} // namespace photon
