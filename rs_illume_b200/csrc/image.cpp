// Film output and film filters on the host: the PFM writer of
// core/imageio.rs:264-310 (and a reader for round trips), the five filters of
// filters/*.rs and the film's 16 x 16 weight table (core/film.rs:70-82).
// All arithmetic is single precision in the reference's operation order
// (built with -ffp-contract=off), so the table matches the Rust code's.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "illume_gpu.h"

namespace {

constexpr float kPi = 3.14159265358979323846f;
constexpr int kTableWidth = ILM_FILTER_TABLE_WIDTH;

// filters/gaussian.rs:27-29
float gaussian1d(float d, float alpha, float expv) {
    float v = std::exp(-alpha * d * d) - expv;
    return v > 0.0f ? v : 0.0f;
}

// filters/mitchell.rs:25-36
float mitchell1d(float x, float b, float c) {
    x = std::fabs(2.0f * x);
    if (x > 1.0f)
        return ((-b - 6.0f * c) * x * x * x + (6.0f * b + 30.0f * c) * x * x + (-12.0f * b - 48.0f * c) * x +
                (8.0f * b + 24.0f * c)) *
               (1.0f / 6.0f);
    return ((12.0f - 9.0f * b - 6.0f * c) * x * x * x + (-18.0f + 12.0f * b + 6.0f * c) * x * x + (6.0f - 2.0f * b)) *
           (1.0f / 6.0f);
}

// filters/sinc.rs:23-39
float sinc(float x) {
    x = std::fabs(x);
    if (x < 1e-5f) return 1.0f;
    return std::sin(kPi * x) / (kPi * x);
}
float windowed_sinc(float x, float radius, float tau) {
    x = std::fabs(x);
    if (x > radius) return 0.0f;
    float lanczos = sinc(x / tau);
    return sinc(x) * lanczos;
}

bool valid(const ilm_filter_desc* f) {
    if (!f || !(f->radius[0] > 0.0f) || !(f->radius[1] > 0.0f)) return false;
    if (f->kind < ILM_FILTER_BOX || f->kind > ILM_FILTER_LANCZOS) return false;
    if (f->kind == ILM_FILTER_LANCZOS && !(f->a > 0.0f)) return false;
    return std::isfinite(f->radius[0]) && std::isfinite(f->radius[1]);
}

float evaluate(const ilm_filter_desc& f, float x, float y) {
    switch (f.kind) {
        case ILM_FILTER_BOX:   // box_filter.rs:30-32
            return 1.0f;
        case ILM_FILTER_TRIANGLE: {   // triangle.rs:30-32
            float wx = f.radius[0] - std::fabs(x), wy = f.radius[1] - std::fabs(y);
            return (wx > 0.0f ? wx : 0.0f) * (wy > 0.0f ? wy : 0.0f);
        }
        case ILM_FILTER_GAUSSIAN: {   // gaussian.rs:17-43
            float ex = std::exp(-f.a * f.radius[0] * f.radius[0]);
            float ey = std::exp(-f.a * f.radius[1] * f.radius[1]);
            return gaussian1d(x, f.a, ex) * gaussian1d(y, f.a, ey);
        }
        case ILM_FILTER_MITCHELL:   // mitchell.rs:48-50 (inv_radius = 1 / radius)
            return mitchell1d(x * (1.0f / f.radius[0]), f.a, f.b) * mitchell1d(y * (1.0f / f.radius[1]), f.a, f.b);
        default:   // sinc.rs:51-53
            return windowed_sinc(x, f.radius[0], f.a) * windowed_sinc(y, f.radius[1], f.a);
    }
}

bool is_space(int c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

// Reads one whitespace-delimited header token; false at end of file.
bool token(FILE* fp, char* buf, size_t cap) {
    int c;
    do { c = std::fgetc(fp); } while (c != EOF && is_space(c));
    if (c == EOF) return false;
    size_t n = 0;
    while (c != EOF && !is_space(c)) {
        if (n + 1 >= cap) return false;
        buf[n++] = (char)c;
        c = std::fgetc(fp);
    }
    buf[n] = '\0';
    return true;   // the single whitespace after the last header token is consumed here
}

bool little_endian_host() {
    uint32_t one = 1;
    unsigned char b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}

}  // namespace

extern "C" {

int32_t ilm_write_pfm(const char* path, const float* rgb, uint32_t width, uint32_t height) {
    if (!path || !rgb || width == 0 || height == 0) return ILM_ERR_INVALID_ARGUMENT;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return ILM_ERR_INVALID_ARGUMENT;
    // header: the scale's sign encodes the byte order (negative = little-endian)
    bool ok = std::fprintf(fp, "PF\n%u %u\n%s\n", width, height, little_endian_host() ? "-1" : "1") > 0;
    const size_t row = (size_t)width * 3;
    for (uint32_t k = 0; ok && k < height; ++k) {
        const float* src = rgb + (size_t)(height - 1 - k) * row;   // bottom row first
        ok = std::fwrite(src, sizeof(float), row, fp) == row;
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? ILM_OK : ILM_ERR_INVALID_ARGUMENT;
}

int32_t ilm_read_pfm(const char* path, float* rgb, uint32_t* width, uint32_t* height) {
    if (!path || !width || !height) return ILM_ERR_INVALID_ARGUMENT;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return ILM_ERR_NOT_FOUND;
    char t[64], w[64], h[64], sc[64];
    bool ok = token(fp, t, sizeof t) && std::strcmp(t, "PF") == 0 && token(fp, w, sizeof w) &&
              token(fp, h, sizeof h) && token(fp, sc, sizeof sc);
    char* end = nullptr;
    long wv = ok ? std::strtol(w, &end, 10) : 0;
    ok = ok && end && *end == '\0' && wv > 0;
    long hv = ok ? std::strtol(h, &end, 10) : 0;
    ok = ok && end && *end == '\0' && hv > 0 && wv < (1L << 20) && hv < (1L << 20);
    double scale = ok ? std::strtod(sc, &end) : 0.0;
    ok = ok && end && *end == '\0' && scale != 0.0;
    if (!ok) {
        std::fclose(fp);
        return ILM_ERR_INVALID_ARGUMENT;
    }
    if (!rgb) {
        *width = (uint32_t)wv;
        *height = (uint32_t)hv;
        std::fclose(fp);
        return ILM_OK;
    }
    if (*width != (uint32_t)wv || *height != (uint32_t)hv) {
        std::fclose(fp);
        return ILM_ERR_INVALID_ARGUMENT;
    }
    const size_t row = (size_t)wv * 3;
    std::vector<float> buf(row);
    const bool swap = (scale < 0.0) != little_endian_host();
    for (long k = 0; ok && k < hv; ++k) {
        ok = std::fread(buf.data(), sizeof(float), row, fp) == row;
        if (!ok) break;
        if (swap)
            for (float& v : buf) {
                uint32_t u;
                std::memcpy(&u, &v, 4);
                u = (u >> 24) | ((u >> 8) & 0xFF00u) | ((u << 8) & 0xFF0000u) | (u << 24);
                std::memcpy(&v, &u, 4);
            }
        std::memcpy(rgb + (size_t)(hv - 1 - k) * row, buf.data(), row * sizeof(float));
    }
    std::fclose(fp);
    return ok ? ILM_OK : ILM_ERR_INVALID_ARGUMENT;
}

int32_t ilm_filter_evaluate(const ilm_filter_desc* filter, float x, float y, float* out) {
    if (!valid(filter) || !out) return ILM_ERR_INVALID_ARGUMENT;
    *out = evaluate(*filter, x, y);
    return ILM_OK;
}

int32_t ilm_filter_table(const ilm_filter_desc* filter, float* table) {
    if (!valid(filter) || !table) return ILM_ERR_INVALID_ARGUMENT;
    int offset = 0;
    for (int y = 0; y < kTableWidth; ++y)
        for (int x = 0; x < kTableWidth; ++x) {
            // film.rs:75-78: ((x + 0.5) * radius) / 16, in f32
            float px = ((float)x + 0.5f) * filter->radius[0] / (float)kTableWidth;
            float py = ((float)y + 0.5f) * filter->radius[1] / (float)kTableWidth;
            table[offset++] = evaluate(*filter, px, py);
        }
    return ILM_OK;
}

}  // extern "C"
