// centerline.cu -- C ABI for device segment extraction and for the whole
// CenterlineExtraction path (pad, thin, extract segments, prune, smooth,
// flatten), plus the tile-configuration table the autotuner fills.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host.h"
#include "kernels.cuh"

namespace bgt {

// ------------------------------------------------------------ tuning ------
// Size classes: 2D by width (<=128, <=256, <=512, <=1024, <=2048, larger);
// 3D by the largest side (<=96, <=160, <=256, larger).
static int g_tuned[2][8] = {{-1, -1, -1, -1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1, -1, -1, -1}};

static int size_class(int dims, int W, int H, int D)
{
    if (dims == 2) {
        (void)H;
        return W <= 128 ? 0 : W <= 256 ? 1 : W <= 512 ? 2 : W <= 1024 ? 3 : W <= 2048 ? 4 : 5;
    }
    const int m = std::max(W, std::max(H, D));
    return m <= 96 ? 0 : m <= 160 ? 1 : m <= 256 ? 2 : 3;
}

int tuned_cfg(int dims, int W, int H, int D)
{
    const int t = g_tuned[dims == 3][size_class(dims, W, H, D)];
    return t >= 0 ? t : default_cfg(dims, W, H, D);
}
}  // namespace bgt

using namespace bgt;

extern "C" int bgt_tune_class(int dims, int w, int h, int d) { return size_class(dims, w, h, d); }

extern "C" int bgt_tune_set(int dims, int cls, int cfg)
{
    if ((dims != 2 && dims != 3) || cls < 0 || cls >= 8) return fail(BGT_ERR_ARG, "bad tuning class");
    if (cfg >= 0) {
        const CfgInfo *c = cfg_info(cfg);
        if (!c || c->dims != dims) return fail(BGT_ERR_ARG, "configuration %d is not %dD", cfg, dims);
    }
    g_tuned[dims == 3][cls] = cfg;
    return BGT_OK;
}

extern "C" int bgt_tune_get(int dims, int cls, int *cfg)
{
    if ((dims != 2 && dims != 3) || cls < 0 || cls >= 8 || !cfg) return fail(BGT_ERR_ARG, "bad tuning class");
    *cfg = g_tuned[dims == 3][cls];
    return BGT_OK;
}

// ------------------------------------------------------------ segments ----
static int segments_device(bgt_ctx *c, int dims, int dtype, const void *d_img, int W, int H, int D, HostSegs *hs)
{
    if (!c || !d_img) return fail(BGT_ERR_ARG, "null argument");
    if (dtype_size(dtype) == 0) return fail(BGT_ERR_ARG, "bad dtype %d", dtype);
    if (W < 1 || H < 1 || D < 1) return fail(BGT_ERR_ARG, "bad size");
    cudaSetDevice(c->device);
    const int P = ((W + 31) / 32 + 3) / 4 * 4;
    void *buf = nullptr;
    int rc = ctx_scratch(c, 20, (size_t)P * H * D * 4, &buf);
    if (rc != BGT_OK) return rc;
    // ExtractSegmentsV tests pdata != 0 (2D/ExtractSegments.cpp:36, 3D/ExtractSegments.cpp:158)
    cudaError_t e = launch_pack(dtype, 2, d_img, W, H, D, W, H, D, P, (uint32_t *)buf, nullptr, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pack");
    return segments_packed(c, dims, (const uint32_t *)buf, W, H, D, P, hs);
}

extern "C" int bgt_segments2d_device(bgt_ctx *c, int dtype, const void *d_img, int w, int h, int32_t **start,
                                     uint8_t **is_end, int16_t **px, int16_t **py, int *nseg, int *npts)
{
    if (!start || !is_end || !px || !py || !nseg || !npts) return fail(BGT_ERR_ARG, "null output");
    HostSegs hs;
    int rc = segments_device(c, 2, dtype, d_img, w, h, 1, &hs);
    if (rc != BGT_OK) return rc;
    *start = hs.start;
    *is_end = hs.is_end;
    *px = hs.px;
    *py = hs.py;
    *nseg = hs.nseg;
    *npts = hs.npts;
    return BGT_OK;
}

extern "C" int bgt_segments3d_device(bgt_ctx *c, int dtype, const void *d_vol, int w, int h, int d,
                                     int32_t **start, uint8_t **is_end, int16_t **px, int16_t **py, int16_t **pz,
                                     int *nseg, int *npts)
{
    if (!start || !is_end || !px || !py || !pz || !nseg || !npts) return fail(BGT_ERR_ARG, "null output");
    HostSegs hs;
    int rc = segments_device(c, 3, dtype, d_vol, w, h, d, &hs);
    if (rc != BGT_OK) return rc;
    *start = hs.start;
    *is_end = hs.is_end;
    *px = hs.px;
    *py = hs.py;
    *pz = hs.pz;
    *nseg = hs.nseg;
    *npts = hs.npts;
    return BGT_OK;
}

// ------------------------------------------------------------ centerline --
// Pruning, smoothing and CSR flattening on the device, operation for
// operation as 2D/CenterlineExtraction.cpp:51-131 and
// 3D/CenterlineExtraction.cpp:56-144:
//  * a segment is kept when (size_t)n > (size_t)max_segment_length or it is
//    not an end segment;
//  * kept segments are renumbered in order (prefix sums of the keep flags
//    and of the kept point counts give each one its CSR slot);
//  * each kept segment is smoothed by one thread with the reference's float
//    running sum (integer coordinates added to and subtracted from it one at
//    a time, IEEE round-to-nearest adds and divide by float(count)), so the
//    float outputs are bit-identical.  A negative smoothing_span is treated
//    as 0 (the reference indexes out of bounds there).
__global__ void prune_flags_kernel(const int32_t *__restrict__ start, const uint8_t *__restrict__ is_end, int S,
                                   unsigned long long maxlen, int *keep, int *kpts)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
        const long long n = (long long)start[k + 1] - start[k];
        const bool kp = (unsigned long long)n > maxlen || !is_end[k];
        keep[k] = kp ? 1 : 0;
        kpts[k] = kp ? (int)n : 0;
    }
}

template <bool Z3>
__global__ void smooth_kernel(const int32_t *__restrict__ start, const int16_t *__restrict__ px,
                              const int16_t *__restrict__ py, const int16_t *__restrict__ pz,
                              const int *__restrict__ keep, const int *__restrict__ seg_new,
                              const int *__restrict__ pt_new, int S, int span_req, float *X, float *Y, float *Zo,
                              unsigned *I)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
        if (!keep[k]) continue;
        const int b = start[k], n = start[k + 1] - b;
        int pi = pt_new[k];
        I[seg_new[k]] = (unsigned)pi;
        const int16_t *sx = px + b, *sy = py + b, *sz = Z3 ? pz + b : nullptr;
        const int span = min(span_req, (n - 1) / 2);
        float x = sx[0], y = sy[0], z = Z3 ? (float)sz[0] : 0.f;
        int cnt = 1;
        X[pi] = (float)sx[0];
        Y[pi] = (float)sy[0];
        if (Z3) Zo[pi] = (float)sz[0];
        pi++;
        auto add = [&](int q) {
            x = __fadd_rn(x, (float)sx[q]);
            y = __fadd_rn(y, (float)sy[q]);
            if (Z3) z = __fadd_rn(z, (float)sz[q]);
        };
        auto sub = [&](int q) {
            x = __fsub_rn(x, (float)sx[q]);
            y = __fsub_rn(y, (float)sy[q]);
            if (Z3) z = __fsub_rn(z, (float)sz[q]);
        };
        auto emit = [&]() {
            const float fc = (float)cnt;
            X[pi] = __fdiv_rn(x, fc);
            Y[pi] = __fdiv_rn(y, fc);
            if (Z3) Zo[pi] = __fdiv_rn(z, fc);
            pi++;
        };
        for (int q = 1; q <= span; q++) {
            add(2 * q - 1);
            add(2 * q);
            cnt += 2;
            emit();
        }
        for (int q = span + 1; q < n - span; q++) {
            add(q + span);
            sub(q - span - 1);
            emit();
        }
        for (int q = n - span, d = span; q < n; q++, d--) {
            sub(q - d - 1);
            sub(q - d);
            cnt -= 2;
            emit();
        }
    }
}

static int prune_smooth_device(bgt_ctx *c, const DevSegs &s, int dims, int max_segment_length, int smoothing_span,
                               float **ox, float **oy, float **oz, unsigned int **oidx, unsigned int *nsegs_out)
{
    cudaStream_t st = c->stream;
    const int S = s.nseg;
    unsigned nsegs = 0, npts = 0;
    int *keep = nullptr, *kpts = nullptr, *seg_new = nullptr, *pt_new = nullptr;
    cudaError_t e;
    if (S > 0) {
        void *p;
        int rc = ctx_scratch(c, 21, (size_t)(S + 1) * 16, &p);
        if (rc != BGT_OK) return rc;
        keep = (int *)p;
        kpts = keep + (S + 1);
        seg_new = kpts + (S + 1);
        pt_new = seg_new + (S + 1);
        const int grid = std::min((S + 255) / 256, 148 * 8);
        const unsigned long long maxlen = (unsigned long long)(long long)max_segment_length;
        prune_flags_kernel<<<grid, 256, 0, st>>>(s.start, s.is_end, S, maxlen, keep, kpts);
        cudaMemsetAsync(keep + S, 0, 4, st);
        cudaMemsetAsync(kpts + S, 0, 4, st);
        if ((e = exscan(c, 14, keep, seg_new, S + 1, st)) != cudaSuccess ||
            (e = exscan(c, 14, kpts, pt_new, S + 1, st)) != cudaSuccess)
            return cuda_fail(e, "prune scan");
        int tot[2] = {0, 0};
        if ((e = cudaMemcpyAsync(&tot[0], seg_new + S, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&tot[1], pt_new + S, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(e, "prune totals");
        nsegs = (unsigned)tot[0];
        npts = (unsigned)tot[1];
    }
    float *X = (float *)malloc(sizeof(float) * std::max(1u, npts));
    float *Y = (float *)malloc(sizeof(float) * std::max(1u, npts));
    float *Z = dims == 3 ? (float *)malloc(sizeof(float) * std::max(1u, npts)) : nullptr;
    unsigned *I = (unsigned *)malloc(sizeof(unsigned) * (nsegs + 1));
    auto release = [&]() {
        free(X);
        free(Y);
        free(Z);
        free(I);
    };
    if (!X || !Y || !I || (dims == 3 && !Z)) {
        release();
        return fail(BGT_ERR_NOMEM, "host allocation of centreline arrays");
    }
    if (nsegs > 0) {
        const size_t fb = ((size_t)npts * 4 + 255) / 256 * 256;
        void *p;
        int rc = ctx_scratch(c, 22, 3 * fb + (size_t)(nsegs + 1) * 4, &p);
        if (rc != BGT_OK) {
            release();
            return rc;
        }
        float *dX = (float *)p, *dY = (float *)((char *)p + fb), *dZ = (float *)((char *)p + 2 * fb);
        unsigned *dI = (unsigned *)((char *)p + 3 * fb);
        const int grid = std::min((S + 127) / 128, 148 * 8);
        const int span = std::max(0, smoothing_span);
        if (dims == 3)
            smooth_kernel<true><<<grid, 128, 0, st>>>(s.start, s.px, s.py, s.pz, keep, seg_new, pt_new, S, span, dX,
                                                       dY, dZ, dI);
        else
            smooth_kernel<false><<<grid, 128, 0, st>>>(s.start, s.px, s.py, nullptr, keep, seg_new, pt_new, S, span,
                                                        dX, dY, nullptr, dI);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(X, dX, (size_t)npts * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(Y, dY, (size_t)npts * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && dims == 3) e = cudaMemcpyAsync(Z, dZ, (size_t)npts * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(I, dI, (size_t)nsegs * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            release();
            return cuda_fail(e, "centreline readback");
        }
    }
    I[nsegs] = npts;
    *ox = X;
    *oy = Y;
    if (oz) *oz = Z;
    *oidx = I;
    *nsegs_out = nsegs;
    return BGT_OK;
}

// Thin the padded image with the engine and extract segments on the device.
static int centerline_segments(bgt_ctx *c, int dims, int dtype, const void *in, int w, int h, int d, DevSegs *ds)
{
    if (!c || !in) return fail(BGT_ERR_ARG, "null argument");
    const size_t es = dtype_size(dtype);
    if (es == 0) return fail(BGT_ERR_ARG, "bad dtype %d", dtype);
    if (w < 1 || h < 1 || d < 1) return fail(BGT_ERR_ARG, "bad size");
    cudaSetDevice(c->device);
    // the reference's padding (2D/CenterlineExtraction.cpp:27-38, 3D/CenterlineExtraction.cpp:27-29)
    int pw, ph, pd;
    if (dims == 2) {
        pw = (w + 31) / 32 * 32;
        ph = std::max(1, (h + 63) / 128) * 128 + 64;
        pd = 1;
    } else {
        pw = (w + 31) / 32 * 32;
        ph = (h + 31) / 32 * 32;
        pd = (d + 31) / 32 * 32;
    }
    const size_t bytes = es * (size_t)w * h * d;
    void *d_in = nullptr;
    int rc = ctx_scratch(c, 0, bytes, &d_in);
    if (rc != BGT_OK) return rc;
    cudaError_t e = cudaMemcpyAsync(d_in, in, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "H2D");
    bgt_batch *b = nullptr;
    rc = single_batch(c, dims, pw, ph, pd, &b);
    if (rc == BGT_OK) rc = bgt_batch_set_io(b, 0, dtype, d_in, nullptr);
    if (rc == BGT_OK) rc = batch_set_input_extent(b, 0, w, h, d);
    if (rc == BGT_OK) rc = bgt_batch_run(b, 0, 0);
    if (rc == BGT_OK) rc = batch_check(b);
    if (rc != BGT_OK) return rc;
    const Inst &inst = b->h[0];
    return segments_device_arrays(c, dims, inst.buf[0], pw, ph, pd, inst.P, ds);
}

extern "C" int bgt_centerline2d(bgt_ctx *c, int dtype, const void *in, int w, int h, int max_segment_length,
                                int smoothing_span, float **out_x, float **out_y, unsigned int **out_idx,
                                unsigned int *nsegs)
{
    if (!out_x || !out_y || !out_idx || !nsegs) return fail(BGT_ERR_ARG, "null output");
    DevSegs ds;
    int rc = centerline_segments(c, 2, dtype, in, w, h, 1, &ds);
    if (rc == BGT_OK)
        rc = prune_smooth_device(c, ds, 2, max_segment_length, smoothing_span, out_x, out_y, nullptr, out_idx, nsegs);
    return rc;
}

extern "C" int bgt_centerline3d(bgt_ctx *c, int dtype, const void *in, int w, int h, int d, int max_segment_length,
                                int smoothing_span, float **out_x, float **out_y, float **out_z,
                                unsigned int **out_idx, unsigned int *nsegs)
{
    if (!out_x || !out_y || !out_z || !out_idx || !nsegs) return fail(BGT_ERR_ARG, "null output");
    DevSegs ds;
    int rc = centerline_segments(c, 3, dtype, in, w, h, d, &ds);
    if (rc == BGT_OK)
        rc = prune_smooth_device(c, ds, 3, max_segment_length, smoothing_span, out_x, out_y, out_z, out_idx, nsegs);
    return rc;
}
