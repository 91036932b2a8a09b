/*
 * segments.c -- CPU restatement of the reference's segment extraction
 * (ExtractSegmentsV) and of the host tail of CenterlineExtraction
 * (pruning, moving-average smoothing, CSR flattening).
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): see oracle.h for who may use it.
 *
 * The walk is the reference's sequential raster-order greedy trace, step for
 * step, including its quirks (single-point segments, a duplicated last point
 * when a walk stalls, pure cycles emitting nothing, the +1 on the end marker):
 *   2D/ExtractSegments.cpp:16-127, 3D/ExtractSegments.cpp:135-251.
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef struct {
    int32_t *start; uint8_t *is_end; int16_t *x, *y, *z;
    int32_t nseg, npts, cap_seg, cap_pts;
    int dims;
} segbuf;

static void sb_init(segbuf *b, int dims)
{
    memset(b, 0, sizeof(*b));
    b->dims = dims;
    b->cap_seg = 1024;
    b->cap_pts = 4096;
    b->start = (int32_t *)malloc(sizeof(int32_t) * (b->cap_seg + 1));
    b->is_end = (uint8_t *)malloc(b->cap_seg);
    b->x = (int16_t *)malloc(sizeof(int16_t) * b->cap_pts);
    b->y = (int16_t *)malloc(sizeof(int16_t) * b->cap_pts);
    b->z = dims == 3 ? (int16_t *)malloc(sizeof(int16_t) * b->cap_pts) : NULL;
    b->start[0] = 0;
}

static void sb_point(segbuf *b, int x, int y, int z)
{
    if (b->npts == b->cap_pts) {
        b->cap_pts *= 2;
        b->x = (int16_t *)realloc(b->x, sizeof(int16_t) * b->cap_pts);
        b->y = (int16_t *)realloc(b->y, sizeof(int16_t) * b->cap_pts);
        if (b->z) b->z = (int16_t *)realloc(b->z, sizeof(int16_t) * b->cap_pts);
    }
    b->x[b->npts] = (int16_t)x;
    b->y[b->npts] = (int16_t)y;
    if (b->z) b->z[b->npts] = (int16_t)z;
    b->npts++;
}

static void sb_close(segbuf *b, int is_end)
{
    if (b->nseg == b->cap_seg) {
        b->cap_seg *= 2;
        b->start = (int32_t *)realloc(b->start, sizeof(int32_t) * (b->cap_seg + 1));
        b->is_end = (uint8_t *)realloc(b->is_end, b->cap_seg);
    }
    b->is_end[b->nseg] = (uint8_t)(is_end != 0);
    b->nseg++;
    b->start[b->nseg] = b->npts;
}

static void sb_export(segbuf *b, oracle_segs *out)
{
    out->nseg = b->nseg;
    out->npts = b->npts;
    out->start = b->start;
    out->is_end = b->is_end;
    out->x = b->x;
    out->y = b->y;
    out->z = b->z;
}

void oracle_segs_free(oracle_segs *s)
{
    if (!s) return;
    free(s->start); free(s->is_end); free(s->x); free(s->y); free(s->z);
    memset(s, 0, sizeof(*s));
}

/*
 * Generic walk over a linearised grid.  fg: foreground flags, nelem elements;
 * interior(i) decided by the caller through the points list; delta[]: the
 * neighbour offsets in the reference's scan order.
 */
static void trace(const uint8_t *fg, size_t nelem, const int64_t *pts, int64_t npoints,
                  const int64_t *delta, int ndelta, int w, int h, int dims, segbuf *out)
{
    signed char *v = (signed char *)calloc(nelem, 1);   /* "neighbors" */
    signed char *v0;                                   /* "onn" */
    for (int64_t k = 0; k < npoints; k++) {
        const int64_t i = pts[k];
        int nn = 0;
        for (int q = 0; q < ndelta; q++) nn += fg[i + delta[q]] != 0;
        if (nn == 0) nn = 1;
        v[i] = (signed char)(nn == 2 ? 2 : -nn);
    }
    v0 = (signed char *)malloc(nelem);
    memcpy(v0, v, nelem);

    const int64_t slice = (int64_t)w * h;
    for (int64_t k = 0; k < npoints; k++) {
        const int64_t p = pts[k];
        const signed char vp = v[p];
        if (vp >= 0) continue;
        v[p] = 0;
        int ni = -1;
        for (int branch = 0; branch < -vp; branch++) {
            int is_end = abs(v0[p]) < 2;
            const int px = (int)(p % w), py = (int)((p / w) % h), pz = (int)(p / slice);
            const int point_mark = out->npts;
            (void)point_mark;
            sb_point(out, px, py, pz);
            for (ni++; ni < ndelta; ni++)
                if (v[p + delta[ni]] != 0) break;
            if (ni >= ndelta) { sb_close(out, is_end); continue; }
            int64_t t = p + delta[ni];
            while (v[t] == 2) {
                v[t] = 0;
                sb_point(out, (int)(t % w), (int)((t / w) % h), (int)(t / slice));
                for (int q = 0; q < ndelta; q++)
                    if (v[t + delta[q]] != 0) { t += delta[q]; break; }
            }
            sb_point(out, (int)(t % w), (int)((t / w) % h), (int)(t / slice));
            if (abs(v0[t]) < 2) is_end = 1;
            v[t] = (signed char)(v[t] + 1);
            sb_close(out, is_end);
        }
    }
    (void)dims;
    free(v);
    free(v0);
}

int oracle_segments2d(const uint8_t *img, int w, int h, oracle_segs *out)
{
    segbuf b;
    sb_init(&b, 2);
    if (w >= 3 && h >= 3) {
        const size_t nelem = (size_t)w * h;
        int64_t *pts = (int64_t *)malloc(sizeof(int64_t) * (nelem ? nelem : 1));
        int64_t np = 0;
        for (int y = 1; y < h - 1; y++)
            for (int x = 1; x < w - 1; x++)
                if (img[(size_t)y * w + x]) pts[np++] = (int64_t)y * w + x;
        /* NW, N, NE, W, E, SW, S, SE (2D/ExtractSegments.cpp:29) */
        const int64_t delta[8] = {-w - 1, -w, -w + 1, -1, 1, w - 1, w, w + 1};
        trace(img, nelem, pts, np, delta, 8, w, h, 2, &b);
        free(pts);
    }
    sb_export(&b, out);
    return 0;
}

int oracle_segments3d(const uint8_t *vol, int w, int h, int d, oracle_segs *out)
{
    segbuf b;
    sb_init(&b, 3);
    if (w >= 3 && h >= 3 && d >= 3) {
        const size_t nelem = (size_t)w * h * d;
        const int64_t s = (int64_t)w * h;
        int64_t *pts = (int64_t *)malloc(sizeof(int64_t) * nelem);
        int64_t np = 0;
        for (int z = 1; z < d - 1; z++)
            for (int y = 1; y < h - 1; y++)
                for (int x = 1; x < w - 1; x++) {
                    const int64_t i = (int64_t)z * s + (int64_t)y * w + x;
                    if (vol[i]) pts[np++] = i;
                }
        /* z-major, then y, then x, centre skipped (3D/ExtractSegments.cpp:149-151) */
        int64_t delta[26];
        int q = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++)
                    if (dz || dy || dx) delta[q++] = dz * s + (int64_t)dy * w + dx;
        trace(vol, nelem, pts, np, delta, 26, w, h, 3, &b);
        free(pts);
    }
    sb_export(&b, out);
    return 0;
}

/*
 * Prune, smooth and flatten (2D/CenterlineExtraction.cpp:51-131,
 * 3D/CenterlineExtraction.cpp:56-144).  The float arithmetic follows the
 * reference operation by operation so the outputs are bit-identical: a float
 * running sum to which integer coordinates are added and subtracted one at a
 * time, divided by float(n).
 */
int oracle_prune_smooth(const oracle_segs *s, int dims, int max_segment_length,
                        int smoothing_span, oracle_cl *out)
{
    memset(out, 0, sizeof(*out));
    /* size_t comparison, as the reference compares points.size() to an int */
    const size_t maxlen = (size_t)(long long)max_segment_length;
    uint32_t nsegs = 0, npts = 0;
    for (int k = 0; k < s->nseg; k++) {
        const size_t n = (size_t)(s->start[k + 1] - s->start[k]);
        const int pruned = !(n > maxlen) && s->is_end[k];
        if (!pruned) { nsegs++; npts += (uint32_t)n; }
    }
    out->nsegs = nsegs;
    out->npts = npts;
    out->x = (float *)malloc(sizeof(float) * (npts ? npts : 1));
    out->y = (float *)malloc(sizeof(float) * (npts ? npts : 1));
    out->z = dims == 3 ? (float *)malloc(sizeof(float) * (npts ? npts : 1)) : NULL;
    out->idx = (uint32_t *)malloc(sizeof(uint32_t) * (nsegs + 1));
    const int span_req = smoothing_span < 0 ? 0 : smoothing_span;
    uint32_t si = 0, pi = 0;
    for (int k = 0; k < s->nseg; k++) {
        const int b = s->start[k];
        const int n = s->start[k + 1] - b;
        const int pruned = !((size_t)n > maxlen) && s->is_end[k];
        if (pruned) continue;
        out->idx[si++] = pi;
        const int16_t *X = s->x + b, *Y = s->y + b, *Z = dims == 3 ? s->z + b : NULL;
        int span = (n - 1) / 2;
        if (span_req < span) span = span_req;
        float x = X[0], y = Y[0], z = Z ? Z[0] : 0.f;
        int cnt = 1;
#define EMIT()                                                  \
    do {                                                        \
        out->x[pi] = x / (float)cnt;                            \
        out->y[pi] = y / (float)cnt;                            \
        if (Z) out->z[pi] = z / (float)cnt;                     \
        pi++;                                                   \
    } while (0)
        out->x[pi] = (float)X[0];
        out->y[pi] = (float)Y[0];
        if (Z) out->z[pi] = (float)Z[0];
        pi++;
        for (int q = 1; q <= span; q++) {
            x += X[2 * q - 1]; y += Y[2 * q - 1]; if (Z) z += Z[2 * q - 1];
            x += X[2 * q];     y += Y[2 * q];     if (Z) z += Z[2 * q];
            cnt += 2;
            EMIT();
        }
        for (int q = span + 1; q < n - span; q++) {
            x += X[q + span]; y += Y[q + span]; if (Z) z += Z[q + span];
            x -= X[q - span - 1]; y -= Y[q - span - 1]; if (Z) z -= Z[q - span - 1];
            EMIT();
        }
        for (int q = n - span, dd = span; q < n; q++, dd--) {
            x -= X[q - dd - 1]; y -= Y[q - dd - 1]; if (Z) z -= Z[q - dd - 1];
            x -= X[q - dd];     y -= Y[q - dd];     if (Z) z -= Z[q - dd];
            cnt -= 2;
            EMIT();
        }
#undef EMIT
    }
    out->idx[nsegs] = npts;
    return 0;
}

void oracle_cl_free(oracle_cl *c)
{
    if (!c) return;
    free(c->x); free(c->y); free(c->z); free(c->idx);
    memset(c, 0, sizeof(*c));
}

/* Reference padding (2D/CenterlineExtraction.cpp:27-38): width to a multiple
 * of 32, height to max(1,(h+63)/128)*128 + 64, zero fill, right/bottom only. */
int oracle_centerline2d(const uint8_t *img, int w, int h, int max_segment_length,
                        int smoothing_span, int nthreads, oracle_cl *out)
{
    const int pw = ((w + 31) / 32) * 32;
    int blocks = (h + 63) / 128;
    if (blocks < 1) blocks = 1;
    const int ph = blocks * 128 + 64;
    uint8_t *pad = (uint8_t *)calloc((size_t)pw * ph, 1);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) pad[(size_t)y * pw + x] = img[(size_t)y * w + x] != 0;
    oracle_thin2d(pad, pw, ph, nthreads);
    oracle_segs s;
    oracle_segments2d(pad, pw, ph, &s);
    oracle_prune_smooth(&s, 2, max_segment_length, smoothing_span, out);
    oracle_segs_free(&s);
    free(pad);
    return 0;
}

/* 3D padding: every dimension to a multiple of 32 (3D/CenterlineExtraction.cpp:27-47). */
int oracle_centerline3d(const uint8_t *vol, int w, int h, int d, int max_segment_length,
                        int smoothing_span, int nthreads, oracle_cl *out)
{
    const int pw = ((w + 31) / 32) * 32, ph = ((h + 31) / 32) * 32, pd = ((d + 31) / 32) * 32;
    uint8_t *pad = (uint8_t *)calloc((size_t)pw * ph * pd, 1);
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
                pad[((size_t)z * ph + y) * pw + x] = vol[((size_t)z * h + y) * w + x] != 0;
    oracle_thin3d(pad, pw, ph, pd, nthreads);
    oracle_segs s;
    oracle_segments3d(pad, pw, ph, pd, &s);
    oracle_prune_smooth(&s, 3, max_segment_length, smoothing_span, out);
    oracle_segs_free(&s);
    free(pad);
    return 0;
}

/* ------------------------------------------------------------------------
 * Binarisation rules per pixel type (codes of bgt_dtype in bgt_capi.h):
 * 0 u8, 1 i8 (signed char), 2 char, 3 u16, 4 i16, 5 u32, 6 i32, 7 f32,
 * 8 f64, 9 bool.
 * ---------------------------------------------------------------------- */
static int fg2d_f64(double v) { return v >= 1.0; } /* saturating truncation to u32 is nonzero */
static int fg3d_f64(double v) { return v >= 1.0 && v < 2147483648.0; } /* x86 cvtt: out of range -> INT_MIN */

int oracle_binarise(int dtype, const void *src, int64_t n, int dims, uint8_t *dst)
{
    for (int64_t i = 0; i < n; i++) {
        int f = 0;
        switch (dtype) {
        case 0: f = ((const uint8_t *)src)[i] != 0; break;
        case 1: { int v = ((const signed char *)src)[i]; f = dims == 2 ? v != 0 : v > 0; } break;
        case 2: { int v = ((const char *)src)[i]; f = dims == 2 ? v != 0 : v > 0; } break;
        case 3: f = ((const uint16_t *)src)[i] != 0; break;
        case 4: { int v = ((const int16_t *)src)[i]; f = dims == 2 ? v != 0 : v > 0; } break;
        case 5: { uint32_t v = ((const uint32_t *)src)[i]; f = dims == 2 ? v != 0 : (int32_t)v > 0; } break;
        case 6: { int32_t v = ((const int32_t *)src)[i]; f = dims == 2 ? v != 0 : v > 0; } break;
        case 7: { double v = ((const float *)src)[i]; f = dims == 2 ? fg2d_f64(v) : fg3d_f64(v); } break;
        case 8: { double v = ((const double *)src)[i]; f = dims == 2 ? fg2d_f64(v) : fg3d_f64(v); } break;
        case 9: f = ((const uint8_t *)src)[i] != 0; break;
        default: return -1;
        }
        dst[i] = (uint8_t)f;
    }
    return 0;
}
