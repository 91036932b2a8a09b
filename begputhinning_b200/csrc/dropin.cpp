// dropin.cpp -- the reference's C++ entry points (Thinning2D<T>,
// Thinning3D<T>, CenterlineExtraction<T> 2D and 3D) implemented over the C
// ABI, with the reference's explicit instantiations, so C++ callers link
// against libbgt.so unchanged.  Each host thread lazily gets its own context
// on the current CUDA device.
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>

#include "CenterlineExctraction.h"
#include "CenterlineExtraction.h"
#include "LibThinning2D.h"
#include "LibThinning3D.h"
#include "bgt_capi.h"

namespace {

struct ThreadCtx {
    bgt_ctx *ctx = nullptr;
    int device = -1;
    ~ThreadCtx()
    {
        if (ctx) bgt_ctx_destroy(ctx);
    }
};

bgt_ctx *thread_ctx()
{
    static thread_local ThreadCtx t;
    int dev = 0;
    cudaGetDevice(&dev);
    if (t.ctx && t.device != dev) {
        bgt_ctx_destroy(t.ctx);
        t.ctx = nullptr;
    }
    if (!t.ctx && bgt_ctx_create(dev, &t.ctx) == BGT_OK) t.device = dev;
    return t.ctx;
}

template <typename T> constexpr int dtype_of();
template <> constexpr int dtype_of<unsigned char>() { return BGT_U8; }
template <> constexpr int dtype_of<signed char>() { return BGT_I8; }
template <> constexpr int dtype_of<char>() { return BGT_CHAR; }
template <> constexpr int dtype_of<unsigned short>() { return BGT_U16; }
template <> constexpr int dtype_of<short>() { return BGT_I16; }
template <> constexpr int dtype_of<unsigned int>() { return BGT_U32; }
template <> constexpr int dtype_of<int>() { return BGT_I32; }
template <> constexpr int dtype_of<float>() { return BGT_F32; }
template <> constexpr int dtype_of<double>() { return BGT_F64; }
template <> constexpr int dtype_of<bool>() { return BGT_BOOL; }

// malloc'ed C-ABI arrays -> new[] arrays the caller delete[]s
template <typename U>
U *to_new(U *src, size_t n)
{
    U *d = new U[n ? n : 1];
    if (src && n) memcpy(d, src, n * sizeof(U));
    bgt_free(src);
    return d;
}

}  // namespace

template <typename PixelType>
void Thinning2D(int width, int height, PixelType *data, PixelType *out)
{
    bgt_ctx *c = thread_ctx();
    if (!c || bgt_thin2d(c, dtype_of<PixelType>(), data, width, height, out) != BGT_OK)
        if (out && width > 0 && height > 0) memset((void *)out, 0, sizeof(PixelType) * (size_t)width * height);
}

template <typename PixelType>
void Thinning3D(int width, int height, int depth, PixelType *data, PixelType *out)
{
    bgt_ctx *c = thread_ctx();
    if (!c || bgt_thin3d(c, dtype_of<PixelType>(), data, width, height, depth, out) != BGT_OK)
        if (out && width > 0 && height > 0 && depth > 0)
            memset((void *)out, 0, sizeof(PixelType) * (size_t)width * height * depth);
}

template <typename PixelType>
unsigned int CenterlineExtraction(PixelType *data, int width, int height, int max_segment_length, int smoothing_span,
                                  float **out_x, float **out_y, unsigned int **out_idx)
{
    float *x = nullptr, *y = nullptr;
    unsigned int *idx = nullptr, n = 0;
    bgt_ctx *c = thread_ctx();
    if (!c || bgt_centerline2d(c, dtype_of<PixelType>(), data, width, height, max_segment_length, smoothing_span, &x,
                               &y, &idx, &n) != BGT_OK) {
        *out_x = new float[1];
        *out_y = new float[1];
        *out_idx = new unsigned int[1]{0};
        return 0;
    }
    const size_t npts = idx[n];
    *out_x = to_new(x, npts);
    *out_y = to_new(y, npts);
    *out_idx = to_new(idx, (size_t)n + 1);
    return n;
}

template <typename PixelType>
unsigned int CenterlineExtraction(PixelType *data, int width, int height, int depth, int max_segment_length,
                                  int smoothing_span, float **out_x, float **out_y, float **out_z,
                                  unsigned int **out_idx)
{
    float *x = nullptr, *y = nullptr, *z = nullptr;
    unsigned int *idx = nullptr, n = 0;
    bgt_ctx *c = thread_ctx();
    if (!c || bgt_centerline3d(c, dtype_of<PixelType>(), data, width, height, depth, max_segment_length,
                               smoothing_span, &x, &y, &z, &idx, &n) != BGT_OK) {
        *out_x = new float[1];
        *out_y = new float[1];
        *out_z = new float[1];
        *out_idx = new unsigned int[1]{0};
        return 0;
    }
    const size_t npts = idx[n];
    *out_x = to_new(x, npts);
    *out_y = to_new(y, npts);
    *out_z = to_new(z, npts);
    *out_idx = to_new(idx, (size_t)n + 1);
    return n;
}

#define BGT_INST2(T)                                                                                           \
    template void Thinning2D<T>(int, int, T *, T *);                                                           \
    template unsigned int CenterlineExtraction<T>(T *, int, int, int, int, float **, float **, unsigned int **); \
    template unsigned int CenterlineExtraction<T>(T *, int, int, int, int, int, float **, float **, float **,   \
                                                  unsigned int **);
BGT_INST2(unsigned char)
BGT_INST2(unsigned short)
BGT_INST2(unsigned int)
BGT_INST2(char)
BGT_INST2(signed char)
BGT_INST2(short)
BGT_INST2(int)
BGT_INST2(float)
BGT_INST2(double)
BGT_INST2(bool)
#undef BGT_INST2

// Thinning3D: the reference's eight instantiations (3D/LibThinning3D.cu:92-99)
template void Thinning3D<unsigned char>(int, int, int, unsigned char *, unsigned char *);
template void Thinning3D<unsigned short>(int, int, int, unsigned short *, unsigned short *);
template void Thinning3D<unsigned int>(int, int, int, unsigned int *, unsigned int *);
template void Thinning3D<char>(int, int, int, char *, char *);
template void Thinning3D<short>(int, int, int, short *, short *);
template void Thinning3D<int>(int, int, int, int *, int *);
template void Thinning3D<float>(int, int, int, float *, float *);
template void Thinning3D<bool>(int, int, int, bool *, bool *);
