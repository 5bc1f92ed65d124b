/*
 * Test infrastructure only (oracle build). A minimal stand-in for the
 * FreeImage header so that the reference's src/main.cpp compiles as a library
 * in a container without FreeImage. The reference only renders images when
 * `dump_image` is true (src/main.cpp:556-678); the oracle harness never sets
 * it, so none of these functions is ever called. Each returns failure.
 */
#ifndef NBODY_ORACLE_FREEIMAGE_STUB_H
#define NBODY_ORACLE_FREEIMAGE_STUB_H

typedef unsigned char BYTE;
typedef struct FIBITMAP_STUB { int unused; } FIBITMAP;
typedef struct RGBQUAD_STUB {
    BYTE rgbBlue;
    BYTE rgbGreen;
    BYTE rgbRed;
    BYTE rgbReserved;
} RGBQUAD;
enum { FIF_PNG = 13 };

static inline FIBITMAP *FreeImage_Allocate(int, int, int) { return 0; }
static inline bool FreeImage_SetPixelColor(FIBITMAP *, unsigned, unsigned, RGBQUAD *) { return false; }
static inline bool FreeImage_Save(int, FIBITMAP *, const char *, int) { return false; }
static inline void FreeImage_Unload(FIBITMAP *) {}
static inline void FreeImage_Initialise(bool = false) {}
static inline void FreeImage_DeInitialise() {}

#endif
