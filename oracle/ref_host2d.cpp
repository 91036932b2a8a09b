// ref_host2d.cpp -- TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libref2d.so).
//
// Wraps the reference's own 2D code so the oracle restatement can be checked
// against it: the rule functions of 2D/CUDA_SubiterationKernels2D.cuh are
// compiled for the host through small shims, and a host Thinning2D<T> runs
// them globally and synchronously (zero outside the image, N,S,E,W, stop
// after an iteration without deletions) in place of the CUDA tiling of
// 2D/LibThinning2D.cu:39-130.  The reference's ExtractSegments.cpp and
// CenterlineExtraction.cpp are compiled unchanged from the reference tree
// and linked beside this file (oracle/Makefile).
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#define __device__
#define __inline__ inline
// A 32-bit word holds pixels x0-1 .. x0+30; plain shifts give exact
// neighbours for bits 1..30, which are the only bits used.
static inline unsigned int ShiftLeft(unsigned int v) { return v << 1; }
static inline unsigned int ShiftRight(unsigned int v) { return v >> 1; }
static inline int min(int a, unsigned int b) { return (unsigned int)a < b ? a : (int)b; }
#include "CUDA_SubiterationKernels2D.cuh"
#include "LibThinning2D.h"
#include "ExtractSegments.h"
#include "CenterlineExtraction.h"
#include "oracle.h"

namespace {
inline unsigned int word_at(const std::vector<uint8_t> &img, int w, int h, int y, int xs)
{
    unsigned int v = 0;
    if (y < 0 || y >= h) return 0;
    for (int b = 0; b < 32; b++) {
        int x = xs + b;
        if (x >= 0 && x < w && img[(size_t)y * w + x]) v |= 1u << b;
    }
    return v;
}
}  // namespace

template <typename PixelType>
void Thinning2D(int width, int height, PixelType *data, PixelType *out)
{
    std::vector<uint8_t> cur((size_t)width * height), nxt;
    for (size_t i = 0; i < cur.size(); i++) cur[i] = (unsigned int)data[i] > 0;
    typedef int (*rule_t)(unsigned int, unsigned int, unsigned int &);
    rule_t rules[4] = {North, South, East, West};
    for (;;) {
        int changed = 0;
        for (int s = 0; s < 4; s++) {
            nxt = cur;
            for (int y = 0; y < height; y++)
                for (int x0 = 0; x0 < width; x0 += 30) {
                    unsigned int up = word_at(cur, width, height, y - 1, x0 - 1);
                    unsigned int cp = word_at(cur, width, height, y, x0 - 1);
                    unsigned int dn = word_at(cur, width, height, y + 1, x0 - 1);
                    rules[s](up, dn, cp);
                    for (int b = 1; b <= 30 && x0 + b - 1 < width; b++) {
                        uint8_t nv = (cp >> b) & 1;
                        size_t i = (size_t)y * width + x0 + b - 1;
                        if (nv != cur[i]) changed = 1;
                        nxt[i] = nv;
                    }
                }
            cur.swap(nxt);
        }
        if (!changed) break;
    }
    for (size_t i = 0; i < cur.size(); i++) out[i] = (PixelType)cur[i];
}

template void Thinning2D<unsigned char>(int, int, unsigned char *, unsigned char *);
template void Thinning2D<unsigned short>(int, int, unsigned short *, unsigned short *);
template void Thinning2D<unsigned int>(int, int, unsigned int *, unsigned int *);
template void Thinning2D<char>(int, int, char *, char *);
template void Thinning2D<signed char>(int, int, signed char *, signed char *);
template void Thinning2D<short>(int, int, short *, short *);
template void Thinning2D<int>(int, int, int *, int *);
template void Thinning2D<float>(int, int, float *, float *);
template void Thinning2D<double>(int, int, double *, double *);
template void Thinning2D<bool>(int, int, bool *, bool *);

extern "C" {

// dir 0..3 = North, South, East, West; returns the updated centre word.
unsigned int ref2d_rule(int dir, unsigned int up, unsigned int down, unsigned int cp)
{
    typedef int (*rule_t)(unsigned int, unsigned int, unsigned int &);
    rule_t rules[4] = {North, South, East, West};
    rules[dir & 3](up, down, cp);
    return cp;
}

void ref2d_thin_u8(int w, int h, uint8_t *in, uint8_t *out) { Thinning2D<unsigned char>(w, h, in, out); }

int ref2d_segments_u8(uint8_t *img, int w, int h, oracle_segs *out)
{
    std::vector<SSegment *> segs = ExtractSegmentsV<unsigned char>(img, w, h);
    int npts = 0;
    for (auto *s : segs) npts += (int)s->points.size();
    out->nseg = (int)segs.size();
    out->npts = npts;
    out->start = (int32_t *)malloc(sizeof(int32_t) * (segs.size() + 1));
    out->is_end = (uint8_t *)malloc(segs.size() + 1);
    out->x = (int16_t *)malloc(sizeof(int16_t) * (npts + 1));
    out->y = (int16_t *)malloc(sizeof(int16_t) * (npts + 1));
    out->z = nullptr;
    int p = 0;
    for (size_t k = 0; k < segs.size(); k++) {
        out->start[k] = p;
        out->is_end[k] = segs[k]->is_end_segment;
        for (auto &q : segs[k]->points) { out->x[p] = q.x; out->y[p] = q.y; p++; }
        delete segs[k];
    }
    out->start[segs.size()] = p;
    return 0;
}

void ref_segs_free(oracle_segs *s)
{
    free(s->start); free(s->is_end); free(s->x); free(s->y); free(s->z);
    memset(s, 0, sizeof(*s));
}

// dtype codes as in bgt_capi.h; outputs are new[]'ed by the reference.
unsigned int ref2d_centerline(int dtype, void *data, int w, int h, int maxlen, int span,
                              float **ox, float **oy, unsigned int **oi)
{
    switch (dtype) {
    case 0: return CenterlineExtraction<unsigned char>((unsigned char *)data, w, h, maxlen, span, ox, oy, oi);
    case 1: return CenterlineExtraction<signed char>((signed char *)data, w, h, maxlen, span, ox, oy, oi);
    case 2: return CenterlineExtraction<char>((char *)data, w, h, maxlen, span, ox, oy, oi);
    case 3: return CenterlineExtraction<unsigned short>((unsigned short *)data, w, h, maxlen, span, ox, oy, oi);
    case 4: return CenterlineExtraction<short>((short *)data, w, h, maxlen, span, ox, oy, oi);
    case 5: return CenterlineExtraction<unsigned int>((unsigned int *)data, w, h, maxlen, span, ox, oy, oi);
    case 6: return CenterlineExtraction<int>((int *)data, w, h, maxlen, span, ox, oy, oi);
    case 7: return CenterlineExtraction<float>((float *)data, w, h, maxlen, span, ox, oy, oi);
    case 8: return CenterlineExtraction<double>((double *)data, w, h, maxlen, span, ox, oy, oi);
    case 9: return CenterlineExtraction<bool>((bool *)data, w, h, maxlen, span, ox, oy, oi);
    }
    return 0;
}

void ref_free_f32(float *p) { delete[] p; }
void ref_free_u32(unsigned int *p) { delete[] p; }

}  // extern "C"
