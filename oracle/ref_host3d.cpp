// ref_host3d.cpp -- TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libref3d.so).
//
// Wraps the reference's own 3D code: the rule functions of
// 3D/CUDA_SubiterationKernels3D.cuh compiled for the host, run globally and
// synchronously by a host Thinning3D<T> (per iteration: pre-test on the
// iteration-start state, then U,N,E,D,S,W with the pre-test mask as `prev`,
// as 3D/CUDA_ThinningKernel3D_Linear.cuh:746-782 does per tile; stop after an
// iteration without deletions, 3D/LibThinning3D.cu:64-74), in place of the
// CUDA tiling.  The reference's ExtractSegments.cpp and CenterlineExtraction.cpp
// are compiled unchanged from the reference tree and linked beside this file.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#define __device__
#define __inline__ inline
#include "CUDA_SubiterationKernels3D.cuh"
#include "LibThinning3D.h"
#include "ExtractSegments.h"
#include "CenterlineExctraction.h"
#include "oracle.h"

namespace {
typedef unsigned int (*rule_t)(unsigned int, unsigned int *, unsigned int);
const rule_t kOrder[6] = {Up3D, North3D, East3D, Down3D, South3D, West3D};

// Volume packed 64 voxels per word along x, with zero guard words/rows/planes.
struct Packed3 {
    int w, h, d, nw;
    std::vector<uint64_t> v;
    Packed3(int w_, int h_, int d_)
        : w(w_), h(h_), d(d_), nw((w_ + 63) / 64), v((size_t)((w_ + 63) / 64 + 2) * (h_ + 2) * (d_ + 2), 0)
    {
    }
    uint64_t *row(int z, int y) { return v.data() + ((size_t)(z + 1) * (h + 2) + (y + 1)) * (nw + 2); }
    const uint64_t *row(int z, int y) const
    {
        return v.data() + ((size_t)(z + 1) * (h + 2) + (y + 1)) * (nw + 2);
    }
    static unsigned int window(const uint64_t *r, int xs)
    {
        const int b = xs + 64, k = b >> 6, s = b & 63;
        uint64_t lo = r[k] >> s;
        if (s) lo |= r[k + 1] << (64 - s);
        return (unsigned int)lo;
    }
    static void put30(uint64_t *r, int x0, uint64_t bits)
    {
        const int b = x0 + 64, k = b >> 6, s = b & 63;
        r[k] |= bits << s;
        if (s > 34) r[k + 1] |= bits >> (64 - s);
    }
};

// n[] in the reference's neighbour order for the window starting at xs
inline void gather(const Packed3 &V, int z, int y, int xs, unsigned int n[26], unsigned int &val)
{
    int i = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++) {
            const uint64_t *r = V.row(z + dz, y + dy);
            for (int dx = -1; dx <= 1; dx++) {
                const unsigned int wv = Packed3::window(r, xs + dx);
                if (dz == 0 && dy == 0 && dx == 0) { val = wv; continue; }
                n[i++] = wv;
            }
        }
}
}  // namespace

// Global, synchronous host execution of the reference's rule functions
// (pre-test union on the iteration-start state, then U,N,E,D,S,W with that
// mask as `prev`); each rule call keeps the 30 inner voxels of its window.
template <typename PixelType>
void Thinning3D(int width, int height, int depth, PixelType *data, PixelType *out)
{
    Packed3 cur(width, height, depth), nxt(width, height, depth);
    for (int z = 0; z < depth; z++)
        for (int y = 0; y < height; y++)
            for (int x = 0; x < width; x++)
                if (data[((size_t)z * height + y) * width + x] > 0) cur.row(z, y)[1 + x / 64] |= 1ull << (x % 64);
    const int nx = (width + 29) / 30;
    std::vector<unsigned int> pv((size_t)nx * height * depth);
    const uint64_t m30 = (1ull << 30) - 1;
    const long long rows = (long long)depth * height;
    for (;;) {
        long long changed = 0;
#pragma omp parallel for schedule(static)
        for (long long zy = 0; zy < rows; zy++) {
            const int z = (int)(zy / height), y = (int)(zy % height);
            for (int c = 0; c < nx; c++) {
                unsigned int n[26], val;
                gather(cur, z, y, c * 30 - 1, n, val);
                unsigned int p = Up3D(val, n);
                p &= North3D(val, n);
                p &= East3D(val, n);
                p &= Down3D(val, n);
                p &= South3D(val, n);
                p &= West3D(val, n);
                pv[(size_t)zy * nx + c] = p;
            }
        }
        for (int s = 0; s < 6; s++) {
            std::fill(nxt.v.begin(), nxt.v.end(), 0);
#pragma omp parallel for reduction(+ : changed) schedule(static)
            for (long long zy = 0; zy < rows; zy++) {
                const int z = (int)(zy / height), y = (int)(zy % height);
                uint64_t *ro = nxt.row(z, y);
                for (int c = 0; c < nx; c++) {
                    unsigned int n[26], val;
                    gather(cur, z, y, c * 30 - 1, n, val);
                    const unsigned int r = kOrder[s](val, n, pv[(size_t)zy * nx + c]);
                    const int valid = width - c * 30 < 30 ? width - c * 30 : 30;
                    const uint64_t vm = valid == 30 ? m30 : ((1ull << valid) - 1);
                    const uint64_t keep = (uint64_t)(r >> 1) & vm;
                    changed += __builtin_popcountll((uint64_t)(val >> 1) & vm & ~keep);
                    Packed3::put30(ro, c * 30, keep);
                }
            }
            std::swap(cur.v, nxt.v);
        }
        if (!changed) break;
    }
    for (int z = 0; z < depth; z++)
        for (int y = 0; y < height; y++)
            for (int x = 0; x < width; x++)
                out[((size_t)z * height + y) * width + x] = (PixelType)((cur.row(z, y)[1 + x / 64] >> (x % 64)) & 1);
}

template void Thinning3D<unsigned char>(int, int, int, unsigned char *, unsigned char *);
template void Thinning3D<unsigned short>(int, int, int, unsigned short *, unsigned short *);
template void Thinning3D<unsigned int>(int, int, int, unsigned int *, unsigned int *);
template void Thinning3D<char>(int, int, int, char *, char *);
template void Thinning3D<short>(int, int, int, short *, short *);
template void Thinning3D<int>(int, int, int, int *, int *);
template void Thinning3D<float>(int, int, int, float *, float *);
template void Thinning3D<bool>(int, int, int, bool *, bool *);

extern "C" {

// dir 0..5 = U,N,E,D,S,W (the kernel's application order).
unsigned int ref3d_rule(int dir, unsigned int val, unsigned int *n26, unsigned int prev)
{
    return kOrder[dir % 6](val, n26, prev);
}

void ref3d_thin_u8(int w, int h, int d, uint8_t *in, uint8_t *out) { Thinning3D<unsigned char>(w, h, d, in, out); }

int ref3d_segments_u8(uint8_t *vol, int w, int h, int d, oracle_segs *out)
{
    std::vector<SSegment *> segs = ExtractSegmentsV<unsigned char>(vol, w, h, d);
    int npts = 0;
    for (auto *s : segs) npts += (int)s->points.size();
    out->nseg = (int)segs.size();
    out->npts = npts;
    out->start = (int32_t *)malloc(sizeof(int32_t) * (segs.size() + 1));
    out->is_end = (uint8_t *)malloc(segs.size() + 1);
    out->x = (int16_t *)malloc(sizeof(int16_t) * (npts + 1));
    out->y = (int16_t *)malloc(sizeof(int16_t) * (npts + 1));
    out->z = (int16_t *)malloc(sizeof(int16_t) * (npts + 1));
    int p = 0;
    for (size_t k = 0; k < segs.size(); k++) {
        out->start[k] = p;
        out->is_end[k] = segs[k]->is_end_segment;
        for (auto &q : segs[k]->points) { out->x[p] = q.x; out->y[p] = q.y; out->z[p] = q.z; p++; }
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

unsigned int ref3d_centerline(int dtype, void *data, int w, int h, int d, int maxlen, int span,
                              float **ox, float **oy, float **oz, unsigned int **oi)
{
    switch (dtype) {
    case 0: return CenterlineExtraction<unsigned char>((unsigned char *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 1: return CenterlineExtraction<signed char>((signed char *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 2: return CenterlineExtraction<char>((char *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 3: return CenterlineExtraction<unsigned short>((unsigned short *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 4: return CenterlineExtraction<short>((short *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 5: return CenterlineExtraction<unsigned int>((unsigned int *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 6: return CenterlineExtraction<int>((int *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 7: return CenterlineExtraction<float>((float *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 8: return CenterlineExtraction<double>((double *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    case 9: return CenterlineExtraction<bool>((bool *)data, w, h, d, maxlen, span, ox, oy, oz, oi);
    }
    return 0;
}

void ref_free_f32(float *p) { delete[] p; }
void ref_free_u32(unsigned int *p) { delete[] p; }

}  // extern "C"
