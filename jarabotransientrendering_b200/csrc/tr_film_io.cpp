// tr_film_io.cpp - reference-compatible streak/steady .hdr output.
#include "tr_film_io.h"

#include <cmath>
#include <cstdio>
#include <vector>

namespace trio {

void rgbe_encode(float r, float g, float b, unsigned char out[4]) {
    float v = r > g ? r : g;
    v = v > b ? v : b;
    if (!(v >= 1e-32f)) { out[0] = out[1] = out[2] = out[3] = 0; return; }
    int e = 0;
    float m = std::frexp(v, &e);                  // v = m * 2^e, m in [0.5, 1)
    float scale = m * 256.0f / v;
    auto q = [&](float c) { float s = c * scale; return (unsigned char)(s > 0.f ? (s < 255.f ? s : 255.f) : 0.f); };
    out[0] = q(r); out[1] = q(g); out[2] = q(b);
    out[3] = (unsigned char)(e + 128);
}

bool write_hdr(const std::string& path, uint32_t width, uint32_t height, const float* rgb, std::string* err) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { if (err) *err = "cannot open " + path; return false; }
    std::fprintf(f, "#?RADIANCE\n# b200 transient film\nFORMAT=32-bit_rle_rgbe\n\n-Y %u +X %u\n", height, width);
    std::vector<unsigned char> row((size_t)width * 4);
    for (uint32_t y = 0; y < height; ++y) {
        for (uint32_t x = 0; x < width; ++x) {
            const float* p = rgb + ((size_t)y * width + x) * 3;
            rgbe_encode(p[0], p[1], p[2], &row[(size_t)x * 4]);
        }
        if (std::fwrite(row.data(), 1, row.size(), f) != row.size()) {
            std::fclose(f);
            if (err) *err = "short write to " + path;
            return false;
        }
    }
    std::fclose(f);
    return true;
}

static inline float avg_nan0(double v, double w) {
    double t = v / w;
    return std::isnan(t) ? 0.0f : (float)t;
}

bool write_streak_film(const char* name, uint32_t W, uint32_t H, uint32_t T, const double* streak,
                       const double* steady, const double* weight, std::string* err) {
    std::vector<float> img((size_t)W * T * 3);
    std::vector<float> tr;
    char buf[4096];
    for (uint32_t y = 0; streak && y < H; ++y) {
        for (uint32_t x = 0; x < W; ++x) {
            const double w = weight[(size_t)y * W + x];
            const double* src = streak + (((size_t)y * W + x) * T) * 3;
            for (uint32_t t = 0; t < T; ++t)
                for (int c = 0; c < 3; ++c) img[((size_t)x * T + t) * 3 + c] = avg_nan0(src[(size_t)t * 3 + c], w);
        }
        std::snprintf(buf, sizeof(buf), "%s_%04u.hdr", name, y);
        bool ok;
        if (T < 8) {
            tr.resize(img.size());
            for (uint32_t x = 0; x < W; ++x)
                for (uint32_t t = 0; t < T; ++t)
                    for (int c = 0; c < 3; ++c) tr[((size_t)t * W + x) * 3 + c] = img[((size_t)x * T + t) * 3 + c];
            ok = write_hdr(buf, W, T, tr.data(), err);
        } else {
            ok = write_hdr(buf, T, W, img.data(), err);
        }
        if (!ok) return false;
    }
    if (!steady) return true;
    std::vector<float> st((size_t)W * H * 3);
    for (size_t i = 0; i < (size_t)W * H; ++i)
        for (int c = 0; c < 3; ++c) st[i * 3 + c] = avg_nan0(steady[i * 3 + c], weight[i]);
    std::snprintf(buf, sizeof(buf), "%s.hdr", name);
    return write_hdr(buf, W, H, st.data(), err);
}

bool write_component(const std::string& path, uint32_t W, uint32_t H, uint32_t channels, const double* sums,
                     const double* weight, std::string* err) {
    const size_t npix = (size_t)W * H;
    std::vector<float> avg(npix * channels);
    for (size_t i = 0; i < npix; ++i)
        for (uint32_t c = 0; c < channels; ++c) avg[i * channels + c] = avg_nan0(sums[i * channels + c], weight[i]);
    if (path.size() >= 4 && path.compare(path.size() - 4, 4, ".raw") == 0) {
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) { if (err) *err = "cannot open " + path; return false; }
        const bool ok = std::fwrite(avg.data(), sizeof(float), avg.size(), f) == avg.size();
        std::fclose(f);
        if (!ok && err) *err = "short write to " + path;
        return ok;
    }
    std::vector<float> rgb(npix * 3);
    for (size_t i = 0; i < npix; ++i)
        for (int c = 0; c < 3; ++c) rgb[i * 3 + c] = avg[i * channels + (channels == 1 ? 0 : c)];
    return write_hdr(path, W, H, rgb.data(), err);
}

}  // namespace trio
