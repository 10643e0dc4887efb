// Frame files of the demo driver: Particle_data%04d.bin, raw float4 records
// with w forced to 1 (hybridFastSummation/newTest.cpp:23-36); the particle
// renderer reads x, y, z and w as a density (Particle_renderer/.../
// read_particles.cpp:56-69).
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pppm.h"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

extern "C" pppm_status pppm_frame_path(const char *dir, int frame, char *out, size_t cap) {
    if (!out || cap == 0 || frame < 0) return PPPM_ERR_INVALID;
    int w = (dir && dir[0]) ? std::snprintf(out, cap, "%s/Particle_data%04d.bin", dir, frame)
                            : std::snprintf(out, cap, "Particle_data%04d.bin", frame);
    if (w < 0 || (size_t)w >= cap) {
        pppm_set_error("pppm_frame_path: buffer too small");
        return PPPM_ERR_INVALID;
    }
    return PPPM_OK;
}

extern "C" pppm_status pppm_write_frame(const char *dir, int frame, uint32_t N, const float *pos4, int on_device) {
    if (!pos4 || frame < 0) {
        pppm_set_error("pppm_write_frame: invalid argument");
        return PPPM_ERR_INVALID;
    }
    std::vector<float> buf(4 * (size_t)N);
    if (N) {
        if (on_device) {
            cudaError_t e = cudaMemcpy(buf.data(), pos4, sizeof(float) * 4 * (size_t)N, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                pppm_set_error("pppm_write_frame: %s", cudaGetErrorString(e));
                return PPPM_ERR_CUDA;
            }
        } else {
            std::memcpy(buf.data(), pos4, sizeof(float) * 4 * (size_t)N);
        }
    }
    for (uint32_t i = 0; i < N; i++) buf[4 * (size_t)i + 3] = 1.0f;
    char path[4096];
    if (pppm_frame_path(dir, frame, path, sizeof(path)) != PPPM_OK) return PPPM_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        pppm_set_error("pppm_write_frame: cannot open %s", path);
        return PPPM_ERR_INVALID;
    }
    const size_t wrote = N ? std::fwrite(buf.data(), sizeof(float) * 4, N, f) : 0;
    std::fclose(f);
    if (wrote != N) {
        pppm_set_error("pppm_write_frame: short write to %s", path);
        return PPPM_ERR_INVALID;
    }
    return PPPM_OK;
}

extern "C" pppm_status pppm_read_frame(const char *path, float *pos4_host, uint32_t cap, uint32_t *N) {
    if (!path || !N) return PPPM_ERR_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        pppm_set_error("pppm_read_frame: cannot open %s", path);
        return PPPM_ERR_INVALID;
    }
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0 || size % 16 != 0) {
        std::fclose(f);
        pppm_set_error("pppm_read_frame: %s is not a whole number of float4 records", path);
        return PPPM_ERR_INVALID;
    }
    const uint32_t n = (uint32_t)(size / 16);
    *N = n;
    if (!pos4_host) {  // size query
        std::fclose(f);
        return PPPM_OK;
    }
    if (n > cap) {
        std::fclose(f);
        pppm_set_error("pppm_read_frame: %u records, capacity %u", n, cap);
        return PPPM_ERR_INVALID;
    }
    const size_t got = n ? std::fread(pos4_host, 16, n, f) : 0;
    std::fclose(f);
    return got == n ? PPPM_OK : PPPM_ERR_INVALID;
}

// SGI image files, as Particle_renderer/.../write_sgi.cpp writes them: a
// 512-byte big-endian header (magic 474, verbatim storage, 1 or 2 bytes per
// channel, dimension 2 or 3, width, height, channels, pixmin 0, pixmax 255 or
// 65535, zero padding), then each channel as rows bottom-up, value =
// trunc(clamp(pixel * 256 (or 65536), 0, 255 (or 65535))).
extern "C" pppm_status pppm_write_sgi(const char *path, uint32_t ni, uint32_t nj, int channels, const float *pix,
                                      int high_precision) {
    if (!path || !pix || (channels != 1 && channels != 3) || ni == 0 || nj == 0 || ni > 65535 || nj > 65535) {
        pppm_set_error("pppm_write_sgi: invalid argument");
        return PPPM_ERR_INVALID;
    }
    const bool hp = high_precision != 0;
    std::vector<unsigned char> out;
    out.reserve(512 + (size_t)ni * nj * channels * (hp ? 2 : 1));
    auto u16 = [&](unsigned v) { out.push_back((unsigned char)(v >> 8)); out.push_back((unsigned char)v); };
    auto u32 = [&](unsigned v) { u16(v >> 16); u16(v & 0xFFFFu); };
    u16(474);
    out.push_back(0);
    out.push_back(hp ? 2 : 1);
    u16(channels == 1 ? 2 : 3);
    u16(ni);
    u16(nj);
    u16((unsigned)channels);
    u32(0);
    u32(hp ? 65535u : 255u);
    out.insert(out.end(), 492, 0);
    const float scale = hp ? 65536.0f : 256.0f;
    for (int c = 0; c < channels; c++)
        for (uint32_t j = 0; j < nj; j++)
            for (uint32_t i = 0; i < ni; i++) {
                float v = pix[(size_t)channels * (i + (size_t)ni * j) + c] * scale;
                if (!(v >= 0.0f)) v = 0.0f;  // negative (or NaN) -> 0
                else if (!hp && v > 255.0f) v = 255.0f;
                else if (hp && v > 65535.0f) v = 65535.0f;
                if (hp) u16((unsigned short)v);
                else out.push_back((unsigned char)v);
            }
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        pppm_set_error("pppm_write_sgi: cannot open %s", path);
        return PPPM_ERR_INVALID;
    }
    const size_t wrote = std::fwrite(out.data(), 1, out.size(), f);
    std::fclose(f);
    if (wrote != out.size()) {
        pppm_set_error("pppm_write_sgi: short write to %s", path);
        return PPPM_ERR_INVALID;
    }
    return PPPM_OK;
}
