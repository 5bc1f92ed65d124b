// Frame files of the reference (host C++): the binary resume format, the text
// position dump and the resume search (src/main.cpp:283-291, 730-759, 790-811),
// plus a PPM writer for rendered images (the reference writes PNG through
// FreeImage, which this library does not depend on).
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/nbody_b200.h"

namespace {

bool exists(const char *p) {
    FILE *f = std::fopen(p, "rb");
    if (!f) return false;
    std::fclose(f);
    return true;
}

}  // namespace

extern "C" int nbody_frame_path(const char *dir, uint32_t frame, int binary, char *buf, size_t buflen) {
    if (!buf || buflen == 0) return NBODY_ERR_INVALID;
    const int k = std::snprintf(buf, buflen, "%s/%04u.%s", dir ? dir : "./data", frame, binary ? "dat" : "txt");
    return (k < 0 || (size_t)k >= buflen) ? NBODY_ERR_INVALID : NBODY_OK;
}

// One record per particle: position, velocity, acceleration (3 each), mass,
// in the reference's `datatype` (8: DOUBLE build, 4: FLOAT build), the raw
// layout of its `particle` class (src/particle.h:17-38).
extern "C" int nbody_write_dat(const char *path, uint32_t n, const double *pos, const double *vel, const double *acc,
                               const double *mass, int datatype_bytes) {
    if (!path || (datatype_bytes != 8 && datatype_bytes != 4) || (n && (!pos || !vel || !mass))) return NBODY_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) return NBODY_ERR_INVALID;
    std::vector<unsigned char> rec(10 * (size_t)datatype_bytes);
    bool ok = true;
    for (uint32_t i = 0; i < n && ok; i++) {
        double v[10];
        for (int k = 0; k < 3; k++) {
            v[k] = pos[3 * (size_t)i + k];
            v[3 + k] = vel[3 * (size_t)i + k];
            v[6 + k] = acc ? acc[3 * (size_t)i + k] : 0.0;
        }
        v[9] = mass[i];
        if (datatype_bytes == 8) {
            std::memcpy(rec.data(), v, 80);
        } else {
            float fv[10];
            for (int k = 0; k < 10; k++) fv[k] = (float)v[k];
            std::memcpy(rec.data(), fv, 40);
        }
        ok = std::fwrite(rec.data(), rec.size(), 1, f) == 1;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? NBODY_OK : NBODY_ERR_INVALID;
}

// Reads a binary frame. With null arrays only *n is set (the record count).
extern "C" int nbody_read_dat(const char *path, int datatype_bytes, uint32_t *n, double *pos, double *vel,
                              double *acc, double *mass) {
    if (!path || !n || (datatype_bytes != 8 && datatype_bytes != 4)) return NBODY_ERR_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) return NBODY_ERR_INVALID;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    const size_t rs = 10 * (size_t)datatype_bytes;
    const uint32_t count = (uint32_t)(bytes / (long)rs);
    if (!pos) {
        *n = count;
        std::fclose(f);
        return NBODY_OK;
    }
    if (*n < count || !vel || !mass) {
        std::fclose(f);
        return NBODY_ERR_INVALID;
    }
    std::vector<unsigned char> rec(rs);
    for (uint32_t i = 0; i < count; i++) {
        if (std::fread(rec.data(), rs, 1, f) != 1) {
            std::fclose(f);
            return NBODY_ERR_INVALID;
        }
        double v[10];
        if (datatype_bytes == 8) {
            std::memcpy(v, rec.data(), 80);
        } else {
            float fv[10];
            std::memcpy(fv, rec.data(), 40);
            for (int k = 0; k < 10; k++) v[k] = fv[k];
        }
        for (int k = 0; k < 3; k++) {
            pos[3 * (size_t)i + k] = v[k];
            vel[3 * (size_t)i + k] = v[3 + k];
            if (acc) acc[3 * (size_t)i + k] = v[6 + k];
        }
        mass[i] = v[9];
    }
    std::fclose(f);
    *n = count;
    return NBODY_OK;
}

// "x, y, z" per line with the stream's default formatting (6 significant
// digits, the same as %g), in the reference's datatype.
extern "C" int nbody_write_txt(const char *path, uint32_t n, const double *pos, int datatype_bytes) {
    if (!path || (datatype_bytes != 8 && datatype_bytes != 4) || (n && !pos)) return NBODY_ERR_INVALID;
    FILE *f = std::fopen(path, "w");
    if (!f) return NBODY_ERR_INVALID;
    for (uint32_t i = 0; i < n; i++) {
        double x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
        if (datatype_bytes == 4) { x = (float)x; y = (float)y; z = (float)z; }
        std::fprintf(f, "%g, %g, %g\n", x, y, z);
    }
    return std::fclose(f) == 0 ? NBODY_OK : NBODY_ERR_INVALID;
}

// The newest binary frame at or below num_frames (read_data's search); -1 when none.
extern "C" int nbody_find_resume_frame(const char *dir, uint32_t num_frames, int32_t *frame_out) {
    if (!frame_out) return NBODY_ERR_INVALID;
    char buf[4096];
    for (int64_t f = num_frames; f >= 0; f--) {
        if (nbody_frame_path(dir, (uint32_t)f, 1, buf, sizeof buf) != NBODY_OK) return NBODY_ERR_INVALID;
        if (exists(buf)) {
            *frame_out = (int32_t)f;
            return NBODY_OK;
        }
    }
    *frame_out = -1;
    return NBODY_OK;
}

extern "C" int nbody_write_ppm(const char *path, uint32_t w, uint32_t h, const uint8_t *rgb) {
    if (!path || !rgb || !w || !h) return NBODY_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) return NBODY_ERR_INVALID;
    std::fprintf(f, "P6\n%u %u\n255\n", w, h);
    bool ok = true;
    for (int64_t y = (int64_t)h - 1; y >= 0 && ok; y--)  // FreeImage row 0 is the bottom row
        ok = std::fwrite(rgb + (size_t)y * w * 3, (size_t)w * 3, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? NBODY_OK : NBODY_ERR_INVALID;
}
