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
#include <vector>

#define __device__
#define __inline__ inline
#include "CUDA_SubiterationKernels3D.cuh"
#include "LibThinning3D.h"
#include "ExtractSegments.h"
#include "CenterlineExctraction.h"
#include "oracle.h"

namespace {
struct Vol {
    int w, h, d;
    std::vector<uint8_t> v;
    unsigned int word(int z, int y, int xs) const
    {
        if (z < 0 || z >= d || y < 0 || y >= h) return 0;
        unsigned int r = 0;
        for (int b = 0; b < 32; b++) {
            int x = xs + b;
            if (x >= 0 && x < w && v[((size_t)z * h + y) * w + x]) r |= 1u << b;
        }
        return r;
    }
};
typedef unsigned int (*rule_t)(unsigned int, unsigned int *, unsigned int);
const rule_t kOrder[6] = {Up3D, North3D, East3D, Down3D, South3D, West3D};

// n[] for the word whose bit b is voxel x0-1+b (valid for bits 1..30)
void gather(const Vol &V, int z, int y, int x0, unsigned int n[26], unsigned int &val)
{
    int i = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                unsigned int wv = V.word(z + dz, y + dy, x0 - 1 + dx);
                if (dz == 0 && dy == 0 && dx == 0) { val = wv; continue; }
                n[i++] = wv;
            }
}
}  // namespace

template <typename PixelType>
void Thinning3D(int width, int height, int depth, PixelType *data, PixelType *out)
{
    Vol cur{width, height, depth, std::vector<uint8_t>((size_t)width * height * depth)};
    for (size_t i = 0; i < cur.v.size(); i++) cur.v[i] = data[i] > 0;
    std::vector<unsigned int> pv;
    for (;;) {
        int changed = 0;
        // pre-test on the iteration-start state; one mask word per 30 voxels
        const int nx = (width + 29) / 30;
        pv.assign((size_t)nx * height * depth, 0);
        for (int z = 0; z < depth; z++)
            for (int y = 0; y < height; y++)
                for (int c = 0; c < nx; c++) {
                    unsigned int n[26], val;
                    gather(cur, z, y, c * 30, n, val);
                    unsigned int p = Up3D(val, n);
                    p &= North3D(val, n);
                    p &= East3D(val, n);
                    p &= Down3D(val, n);
                    p &= South3D(val, n);
                    p &= West3D(val, n);
                    pv[((size_t)z * height + y) * nx + c] = p;
                }
        for (int s = 0; s < 6; s++) {
            Vol nxt = cur;
            for (int z = 0; z < depth; z++)
                for (int y = 0; y < height; y++)
                    for (int c = 0; c < nx; c++) {
                        unsigned int n[26], val;
                        gather(cur, z, y, c * 30, n, val);
                        unsigned int r = kOrder[s](val, n, pv[((size_t)z * height + y) * nx + c]);
                        for (int b = 1; b <= 30 && c * 30 + b - 1 < width; b++) {
                            uint8_t nvb = (r >> b) & 1;
                            size_t i = ((size_t)z * height + y) * width + c * 30 + b - 1;
                            if (nvb != cur.v[i]) changed = 1;
                            nxt.v[i] = nvb;
                        }
                    }
            cur.v.swap(nxt.v);
        }
        if (!changed) break;
    }
    for (size_t i = 0; i < cur.v.size(); i++) out[i] = (PixelType)cur.v[i];
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
