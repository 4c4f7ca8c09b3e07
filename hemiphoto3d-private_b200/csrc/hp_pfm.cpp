// Portable FloatMap I/O (saveDepthMapPFM / loadDepthMapPFM,
// src/dense_recon/patchmatch_mvs.cu:990-1022): "Pf" grayscale or "PF" RGB
// header, width and height, scale -1.0 (little-endian), rows bottom-to-top.
// The reference writes depth only; the 3-channel form carries normals so a
// solve's full state can be checkpointed.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hp_internal.h"

extern "C" {

hp_status hp_pfm_write(const char* path, const float* data, int width, int height, int channels) {
    if (!path || !data || width < 1 || height < 1 || (channels != 1 && channels != 3)) return HP_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "wb");
    if (!f) return HP_ERR_IO;
    bool ok = std::fprintf(f, "%s\n%d %d\n-1.0\n", channels == 1 ? "Pf" : "PF", width, height) > 0;
    const size_t row = static_cast<size_t>(width) * channels;
    for (int y = height - 1; ok && y >= 0; --y)
        ok = std::fwrite(data + static_cast<size_t>(y) * row, sizeof(float), row, f) == row;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? HP_OK : HP_ERR_IO;
}

hp_status hp_pfm_read(const char* path, float* data, size_t capacity, int* width, int* height, int* channels) {
    if (!path || !width || !height || !channels) return HP_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return HP_ERR_IO;
    char magic[3] = {0, 0, 0};
    int w = 0, h = 0;
    double scale = 0;
    bool ok = std::fscanf(f, "%2s %d %d %lf", magic, &w, &h, &scale) == 4;
    int ch = 0;
    if (ok && std::strcmp(magic, "Pf") == 0) ch = 1;
    if (ok && std::strcmp(magic, "PF") == 0) ch = 3;
    if (!ok || ch == 0 || w < 1 || h < 1 || scale >= 0) {  // big-endian (scale > 0) is not produced here
        std::fclose(f);
        return HP_ERR_IO;
    }
    std::fgetc(f);  // the single whitespace byte after the scale
    *width = w;
    *height = h;
    *channels = ch;
    const size_t row = static_cast<size_t>(w) * ch;
    if (!data) {  // header query
        std::fclose(f);
        return HP_OK;
    }
    if (capacity < row * h) {
        std::fclose(f);
        return HP_ERR_INVALID_ARG;
    }
    for (int y = h - 1; ok && y >= 0; --y) ok = std::fread(data + static_cast<size_t>(y) * row, sizeof(float), row, f) == row;
    std::fclose(f);
    return ok ? HP_OK : HP_ERR_IO;
}

}  // extern "C"
