// Image output for the RGBW accumulation buffers (host code, no GPU).
//
// Replaces FileImagePlane::Finalize (imageplane/fileimageplane.cpp:13-27) and
// the OpenImageIO writer it calls (imageio/oiioimageio.cpp:40-56) for
// headless use: the buffer holds per pixel (sum r, sum g, sum b, samples) with
// the image rows stored bottom-up (WriteSample's row flip), and Finalize turns
// it into (c / w)^(1 / 2.2) per channel.
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/banshee_gpu.h"

namespace bg {
int set_error(int code, const char* fmt, ...);   // api.cu
}

namespace {

bool ends_with(const std::string& s, const char* suf) {
    const size_t n = std::strlen(suf);
    if (s.size() < n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower(static_cast<unsigned char>(s[s.size() - n + i])) != suf[i]) return false;
    return true;
}

}  // namespace

extern "C" {

int bg_image_finalize(const float* rgbw, int32_t width, int32_t height, float* rgb) {
    if (!rgbw || !rgb) return bg::set_error(BG_ERR_INVALID_ARG, "NULL buffer");
    if (width <= 0 || height <= 0) return bg::set_error(BG_ERR_INVALID_ARG, "bad resolution");
    const int64_t n = int64_t(width) * height;
    for (int64_t i = 0; i < n; ++i) {
        const float w = rgbw[4 * i + 3];
        rgb[3 * i] = powf(rgbw[4 * i] / w, 1.f / 2.2f);
        rgb[3 * i + 1] = powf(rgbw[4 * i + 1] / w, 1.f / 2.2f);
        rgb[3 * i + 2] = powf(rgbw[4 * i + 2] / w, 1.f / 2.2f);
    }
    return BG_OK;
}

int bg_image_write(const char* path, const float* rgbw, int32_t width, int32_t height) {
    if (!path) return bg::set_error(BG_ERR_INVALID_ARG, "NULL path");
    std::vector<float> rgb(size_t(width > 0 ? width : 0) * size_t(height > 0 ? height : 0) * 3);
    int rc = bg_image_finalize(rgbw, width, height, rgb.data());
    if (rc) return rc;
    const std::string p(path);
    const bool pfm = ends_with(p, ".pfm");
    if (!pfm && !ends_with(p, ".ppm"))
        return bg::set_error(BG_ERR_UNSUPPORTED, "%s: write .ppm (8-bit) or .pfm (float)", path);
    FILE* f = std::fopen(path, "wb");
    if (!f) return bg::set_error(BG_ERR_INVALID_ARG, "cannot open %s for writing", path);
    bool ok = true;
    if (pfm) {
        // PFM: little-endian floats, scanlines bottom to top, which is the buffer's order
        ok = std::fprintf(f, "PF\n%d %d\n-1.0\n", width, height) > 0;
        ok = ok && std::fwrite(rgb.data(), sizeof(float), rgb.size(), f) == rgb.size();
    } else {
        // PPM: 8-bit, scanlines top to bottom; values clamped to [0, 1] and rounded
        ok = std::fprintf(f, "P6\n%d %d\n255\n", width, height) > 0;
        std::vector<unsigned char> row(size_t(width) * 3);
        for (int y = 0; ok && y < height; ++y) {
            const float* src = rgb.data() + size_t(height - 1 - y) * size_t(width) * 3;
            for (size_t k = 0; k < row.size(); ++k) {
                float v = src[k];
                v = v != v ? 0.f : (v < 0.f ? 0.f : (v > 1.f ? 1.f : v));
                row[k] = static_cast<unsigned char>(v * 255.f + 0.5f);
            }
            ok = std::fwrite(row.data(), 1, row.size(), f) == row.size();
        }
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) return bg::set_error(BG_ERR_INVALID_ARG, "write to %s failed", path);
    return BG_OK;
}

}  // extern "C"
