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
#include <algorithm>
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
// Rows packed 64 pixels per word with one zero guard word on each side and
// one zero guard row above and below; window(row, xs) = the 32 pixels
// xs .. xs+31 as a rule-function word.
struct Packed {
    int w, h, nw;
    std::vector<uint64_t> v;
    Packed(int w_, int h_) : w(w_), h(h_), nw((w_ + 63) / 64), v((size_t)((w_ + 63) / 64 + 2) * (h_ + 2), 0) {}
    uint64_t *row(int y) { return v.data() + (size_t)(y + 1) * (nw + 2); }
    const uint64_t *row(int y) const { return v.data() + (size_t)(y + 1) * (nw + 2); }
    static unsigned int window(const uint64_t *r, int xs)
    {
        const int b = xs + 64, k = b >> 6, s = b & 63;
        uint64_t lo = r[k] >> s;
        if (s) lo |= r[k + 1] << (64 - s);
        return (unsigned int)lo;
    }
    static void put30(uint64_t *r, int x0, uint64_t bits)  // 30 bits at pixel x0
    {
        const int b = x0 + 64, k = b >> 6, s = b & 63;
        r[k] |= bits << s;
        if (s > 34) r[k + 1] |= bits >> (64 - s);
    }
};
}  // namespace

// Global, synchronous host execution of the reference's rule functions; each
// rule call evaluates a 32-pixel window and keeps its 30 inner pixels.
template <typename PixelType>
void Thinning2D(int width, int height, PixelType *data, PixelType *out)
{
    Packed cur(width, height), nxt(width, height);
    for (int y = 0; y < height; y++)
        for (int x = 0; x < width; x++)
            if ((unsigned int)data[(size_t)y * width + x] > 0) cur.row(y)[1 + x / 64] |= 1ull << (x % 64);
    typedef int (*rule_t)(unsigned int, unsigned int, unsigned int &);
    rule_t rules[4] = {North, South, East, West};
    const uint64_t m30 = (1ull << 30) - 1;
    for (;;) {
        long long changed = 0;
        for (int s = 0; s < 4; s++) {
            std::fill(nxt.v.begin(), nxt.v.end(), 0);
#pragma omp parallel for reduction(+ : changed) schedule(static)
            for (int y = 0; y < height; y++) {
                const uint64_t *ru = cur.row(y - 1), *rc = cur.row(y), *rd = cur.row(y + 1);
                uint64_t *ro = nxt.row(y);
                for (int x0 = 0; x0 < width; x0 += 30) {
                    unsigned int up = Packed::window(ru, x0 - 1), cp = Packed::window(rc, x0 - 1);
                    const unsigned int dn = Packed::window(rd, x0 - 1), before = cp;
                    rules[s](up, dn, cp);
                    uint64_t keep = (uint64_t)(cp >> 1) & m30;
                    const int valid = width - x0 < 30 ? width - x0 : 30;
                    keep &= (valid == 30) ? m30 : ((1ull << valid) - 1);
                    changed += __builtin_popcountll(((uint64_t)(before >> 1) & m30 & ~keep) &
                                                    ((valid == 30) ? m30 : ((1ull << valid) - 1)));
                    Packed::put30(ro, x0, keep);
                }
            }
            std::swap(cur.v, nxt.v);
        }
        if (!changed) break;
    }
    for (int y = 0; y < height; y++)
        for (int x = 0; x < width; x++)
            out[(size_t)y * width + x] = (PixelType)((cur.row(y)[1 + x / 64] >> (x % 64)) & 1);
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
