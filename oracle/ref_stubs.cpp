// ref_stubs.cpp — TEST INFRASTRUCTURE (oracle).  Link stubs for the seven reference symbols
// whose implementations cannot be built here: the image loaders need the un-vendored
// stb/tinyexr (src/core/image/image_io.h:58-93) and the Vulkan factory lives in a translation
// unit that embeds compiled SPIR-V (src/engine/vulkan_device.h:27-34), which this build does
// not touch.  None of them is on the path-tracing hot path.
#include "core/image/image_io.h"
#include "engine/vulkan_device.h"

namespace photon {

std::optional<Image> loadImageLDR(const std::string&, TextureEncoding) { return std::nullopt; }
std::optional<Image> loadImageHDR(const std::string&) { return std::nullopt; }
std::optional<Image> loadImageEXR(const std::string&) { return std::nullopt; }
std::optional<Image> loadOpacityImage(const std::string&) { return std::nullopt; }
std::optional<Image> loadImageLDRMemory(const unsigned char*, int, TextureEncoding) { return std::nullopt; }

std::vector<DeviceInfo> probeVulkanDevices() { return {}; }
bool isVulkanHardwareGpu(const std::string&) { return false; }
std::unique_ptr<RenderDevice> createVulkanDevice(int, const DeviceInfo&, std::string* error) {
    if (error) *error = "Vulkan backend not built in the oracle";
    return nullptr;
}

} // namespace photon
