// ref_stubs.cpp — TEST INFRASTRUCTURE (oracle).  Link stubs for the reference symbols whose
// implementations cannot be built here: the image loaders need the un-vendored stb/tinyexr
// (src/core/image/image_io.h:58-93) — the Radiance .hdr reader is restated below from stb's
// published format so project environments load — the model importer needs un-vendored
// OBJ/glTF/FBX/USD/Alembic readers (src/scene/model_import.h:61), and the Vulkan factory lives
// in a translation unit that embeds compiled SPIR-V (src/engine/vulkan_device.h:27-34), which
// this build does not touch.  None of them is on the path-tracing hot path.
#include "core/image/image_io.h"
#include "engine/vulkan_device.h"
#include "scene/model_import.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

namespace photon {

std::optional<Image> loadImageLDR(const std::string&, TextureEncoding) { return std::nullopt; }
// Radiance RGBE (.hdr) as the un-vendored stb_image reads it (its published algorithm): a "#?"
// header up to a blank line, a "-Y h +X w" size line, then flat or new-style run-length encoded
// scanlines; each texel is mantissa · 2^(exponent − 136), 0 for a zero exponent, top row first.
std::optional<Image> loadImageHDR(const std::string& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return std::nullopt;
    std::vector<unsigned char> d;
    unsigned char buf[65536];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) d.insert(d.end(), buf, buf + got);
    std::fclose(f);
    const std::string head(d.begin(), d.begin() + std::min<size_t>(d.size(), 4096));
    const size_t blank = head.find("\n\n");
    if (head.rfind("#?", 0) != 0 || blank == std::string::npos) return std::nullopt;
    size_t pos = blank + 2;
    const size_t eol = head.find('\n', pos);
    int w = 0, h = 0;
    if (eol == std::string::npos || std::sscanf(head.c_str() + pos, "-Y %d +X %d", &h, &w) != 2 || w <= 0 || h <= 0)
        return std::nullopt;
    pos = eol + 1;
    Image img(w, h);
    std::vector<unsigned char> line(static_cast<size_t>(w) * 4);
    for (int y = 0; y < h; ++y) {
        if (pos + 4 > d.size()) return std::nullopt;
        if (w >= 8 && w < 32768 && d[pos] == 2 && d[pos + 1] == 2 && !(d[pos + 2] & 0x80)) {
            if (((d[pos + 2] << 8) | d[pos + 3]) != w) return std::nullopt;
            pos += 4;
            for (int c = 0; c < 4; ++c)
                for (int x = 0; x < w;) {
                    if (pos >= d.size()) return std::nullopt;
                    int n = d[pos++];
                    if (n > 128) {
                        n -= 128;
                        if (pos >= d.size() || x + n > w) return std::nullopt;
                        for (int k = 0; k < n; ++k) line[static_cast<size_t>(x + k) * 4 + c] = d[pos];
                        ++pos;
                    } else {
                        if (n == 0 || pos + n > d.size() || x + n > w) return std::nullopt;
                        for (int k = 0; k < n; ++k) line[static_cast<size_t>(x + k) * 4 + c] = d[pos++];
                    }
                    x += n;
                }
        } else {
            if (pos + line.size() > d.size()) return std::nullopt;
            std::copy(d.begin() + static_cast<long>(pos), d.begin() + static_cast<long>(pos + line.size()), line.begin());
            pos += line.size();
        }
        for (int x = 0; x < w; ++x) {
            const unsigned char* t = &line[static_cast<size_t>(x) * 4];
            const float s = t[3] ? std::ldexp(1.0f, static_cast<int>(t[3]) - 136) : 0.0f;
            img.setPixel(x, y, Color3f(t[0] * s, t[1] * s, t[2] * s));
        }
    }
    return img;
}
std::optional<Image> loadImageEXR(const std::string&) { return std::nullopt; }
std::optional<Image> loadOpacityImage(const std::string&) { return std::nullopt; }
std::optional<Image> loadImageLDRMemory(const unsigned char*, int, TextureEncoding) { return std::nullopt; }

// Imported model files (OBJ / glTF / FBX / USD / Alembic) need un-vendored third-party readers.
std::unique_ptr<SceneNode> importModelFile(const std::string&, std::string* error, const ModelImportOptions&,
                                           std::vector<std::string>*, ImportExtras*) {
    if (error) *error = "model import is not built in the oracle";
    return nullptr;
}

std::vector<DeviceInfo> probeVulkanDevices() { return {}; }
bool isVulkanHardwareGpu(const std::string&) { return false; }
std::unique_ptr<RenderDevice> createVulkanDevice(int, const DeviceInfo&, std::string* error) {
    if (error) *error = "Vulkan backend not built in the oracle";
    return nullptr;
}

} // namespace photon
