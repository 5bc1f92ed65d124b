/*
 * Test infrastructure only (oracle build). A minimal stand-in for the
 * FreeImage header so that the reference's src/main.cpp compiles as a library
 * in a container without FreeImage. It keeps a 24-bit bitmap in memory:
 * FreeImage_SetPixelColor stores pixels and FreeImage_Save copies the bitmap
 * to `g_stub_last_image` (no file is written), so tests can read what the
 * reference's write_image (src/main.cpp:556-678) rendered.
 */
#ifndef NBODY_ORACLE_FREEIMAGE_STUB_H
#define NBODY_ORACLE_FREEIMAGE_STUB_H

#include <cstring>
#include <vector>

typedef unsigned char BYTE;
typedef struct RGBQUAD_STUB {
    BYTE rgbBlue;
    BYTE rgbGreen;
    BYTE rgbRed;
    BYTE rgbReserved;
} RGBQUAD;
struct FIBITMAP {
    int w, h;
    std::vector<unsigned char> rgb;  // (y * w + x) * 3 + {0: R, 1: G, 2: B}, y as FreeImage counts it
};
enum { FIF_PNG = 13 };

static FIBITMAP g_stub_last_image = {0, 0, std::vector<unsigned char>()};

static inline FIBITMAP *FreeImage_Allocate(int w, int h, int) {
    FIBITMAP *b = new FIBITMAP;
    b->w = w;
    b->h = h;
    b->rgb.assign((size_t)w * h * 3, 0);
    return b;
}
static inline bool FreeImage_SetPixelColor(FIBITMAP *b, unsigned x, unsigned y, RGBQUAD *p) {
    if (!b || x >= (unsigned)b->w || y >= (unsigned)b->h) return false;
    unsigned char *q = &b->rgb[((size_t)y * b->w + x) * 3];
    q[0] = p->rgbRed;
    q[1] = p->rgbGreen;
    q[2] = p->rgbBlue;
    return true;
}
static inline bool FreeImage_Save(int, FIBITMAP *b, const char *, int) {
    if (!b) return false;
    g_stub_last_image = *b;
    return true;
}
static inline void FreeImage_Unload(FIBITMAP *b) { delete b; }
static inline void FreeImage_Initialise(bool = false) {}
static inline void FreeImage_DeInitialise() {}

#endif
