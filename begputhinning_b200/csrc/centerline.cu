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
// Pruning, smoothing and CSR flattening, operation for operation as
// 2D/CenterlineExtraction.cpp:51-131 and 3D/CenterlineExtraction.cpp:56-144
// (a float running sum to which the integer coordinates are added and from
// which they are subtracted one at a time, divided by float(n)), so the float
// outputs are bit-identical.  A negative smoothing_span is treated as 0 (the
// reference indexes out of bounds there).
static int prune_smooth(const HostSegs &s, int dims, int max_segment_length, int smoothing_span, float **ox,
                        float **oy, float **oz, unsigned int **oidx, unsigned int *nsegs_out)
{
    const size_t maxlen = (size_t)(long long)max_segment_length;  // size_t comparison as in the reference
    unsigned nsegs = 0, npts = 0;
    for (int k = 0; k < s.nseg; k++) {
        const size_t n = (size_t)(s.start[k + 1] - s.start[k]);
        if ((n > maxlen) || !s.is_end[k]) {
            nsegs++;
            npts += (unsigned)n;
        }
    }
    float *X = (float *)malloc(sizeof(float) * std::max(1u, npts));
    float *Y = (float *)malloc(sizeof(float) * std::max(1u, npts));
    float *Z = dims == 3 ? (float *)malloc(sizeof(float) * std::max(1u, npts)) : nullptr;
    unsigned *I = (unsigned *)malloc(sizeof(unsigned) * (nsegs + 1));
    if (!X || !Y || !I || (dims == 3 && !Z)) {
        free(X); free(Y); free(Z); free(I);
        return fail(BGT_ERR_NOMEM, "host allocation of centreline arrays");
    }
    const int span_req = std::max(0, smoothing_span);
    unsigned si = 0, pi = 0;
    for (int k = 0; k < s.nseg; k++) {
        const int b = s.start[k], n = s.start[k + 1] - s.start[k];
        if (!((size_t)n > maxlen) && s.is_end[k]) continue;
        I[si++] = pi;
        const int16_t *px = s.px + b, *py = s.py + b, *pz = dims == 3 ? s.pz + b : nullptr;
        const int span = std::min(span_req, (n - 1) / 2);
        float x = px[0], y = py[0], z = pz ? pz[0] : 0.f;
        int cnt = 1;
        X[pi] = (float)px[0];
        Y[pi] = (float)py[0];
        if (Z) Z[pi] = (float)pz[0];
        pi++;
        auto emit = [&]() {
            X[pi] = x / (float)cnt;
            Y[pi] = y / (float)cnt;
            if (Z) Z[pi] = z / (float)cnt;
            pi++;
        };
        for (int q = 1; q <= span; q++) {
            x += px[2 * q - 1]; y += py[2 * q - 1]; if (pz) z += pz[2 * q - 1];
            x += px[2 * q];     y += py[2 * q];     if (pz) z += pz[2 * q];
            cnt += 2;
            emit();
        }
        for (int q = span + 1; q < n - span; q++) {
            x += px[q + span]; y += py[q + span]; if (pz) z += pz[q + span];
            x -= px[q - span - 1]; y -= py[q - span - 1]; if (pz) z -= pz[q - span - 1];
            emit();
        }
        for (int q = n - span, d = span; q < n; q++, d--) {
            x -= px[q - d - 1]; y -= py[q - d - 1]; if (pz) z -= pz[q - d - 1];
            x -= px[q - d];     y -= py[q - d];     if (pz) z -= pz[q - d];
            cnt -= 2;
            emit();
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
static int centerline_segments(bgt_ctx *c, int dims, int dtype, const void *in, int w, int h, int d, HostSegs *hs)
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
    return segments_packed(c, dims, inst.buf[0], pw, ph, pd, inst.P, hs);
}

extern "C" int bgt_centerline2d(bgt_ctx *c, int dtype, const void *in, int w, int h, int max_segment_length,
                                int smoothing_span, float **out_x, float **out_y, unsigned int **out_idx,
                                unsigned int *nsegs)
{
    if (!out_x || !out_y || !out_idx || !nsegs) return fail(BGT_ERR_ARG, "null output");
    HostSegs hs;
    int rc = centerline_segments(c, 2, dtype, in, w, h, 1, &hs);
    if (rc == BGT_OK)
        rc = prune_smooth(hs, 2, max_segment_length, smoothing_span, out_x, out_y, nullptr, out_idx, nsegs);
    free_host_segs(&hs);
    return rc;
}

extern "C" int bgt_centerline3d(bgt_ctx *c, int dtype, const void *in, int w, int h, int d, int max_segment_length,
                                int smoothing_span, float **out_x, float **out_y, float **out_z,
                                unsigned int **out_idx, unsigned int *nsegs)
{
    if (!out_x || !out_y || !out_z || !out_idx || !nsegs) return fail(BGT_ERR_ARG, "null output");
    HostSegs hs;
    int rc = centerline_segments(c, 3, dtype, in, w, h, d, &hs);
    if (rc == BGT_OK)
        rc = prune_smooth(hs, 3, max_segment_length, smoothing_span, out_x, out_y, out_z, out_idx, nsegs);
    free_host_segs(&hs);
    return rc;
}
