/*
 * oracle.h -- CPU restatement of BEGPUThinning's hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load
 * it.  The product (begputhinning_b200) never links or calls it, and has no
 * CPU fallback.
 *
 * What it restates (reference file:line):
 *   - 2D directional subiteration thinning, N,S,E,W per iteration, each
 *     subiteration synchronous over the whole image, zero outside the image,
 *     stop after the first whole iteration without deletions
 *     (2D/LibThinning2D.cu:102-112, 2D/CUDA_ThinningKernelMultiBlock2D.cuh:99-135,
 *      rules 2D/CUDA_SubiterationKernels2D.cuh:15-119).
 *   - 3D thinning: per iteration a pre-test (union of the six directional
 *     deletable sets on the iteration-start state), then U,N,E,D,S,W, each
 *     synchronous; a voxel is deleted in direction d iff it is d-deletable on
 *     the current state and was in the pre-test union
 *     (3D/CUDA_ThinningKernel3D_Linear.cuh:690-782, rules
 *      3D/CUDA_SubiterationKernels3D.cuh:14-234, host loop 3D/LibThinning3D.cu:64-74).
 *   - ExtractSegmentsV 2D/3D (2D/ExtractSegments.cpp:16-127,
 *     3D/ExtractSegments.cpp:135-251).
 *   - CenterlineExtraction pruning, smoothing and CSR flattening
 *     (2D/CenterlineExtraction.cpp:22-142, 3D/CenterlineExtraction.cpp:23-155).
 *
 * Images are uint8 {0,1} (any nonzero = foreground), row-major, x fastest:
 * 2D data[y*w + x], 3D data[(z*h + y)*w + x].
 */
#ifndef BGT_ORACLE_H
#define BGT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Thinning, in place on a uint8 image. Returns the number of iterations run
 * (the last one deletes nothing).  nthreads <= 0 uses the OpenMP default. */
int oracle_thin2d(uint8_t *img, int w, int h, int nthreads);
int oracle_thin3d(uint8_t *vol, int w, int h, int d, int nthreads);

/* Segment list as ExtractSegmentsV emits it, in emission order. */
typedef struct {
    int32_t nseg;
    int32_t npts;
    int32_t *start;   /* nseg + 1 offsets into the point arrays */
    uint8_t *is_end;  /* is_end_segment flag per segment */
    int16_t *x, *y, *z; /* points; z is NULL for 2D */
} oracle_segs;

int oracle_segments2d(const uint8_t *img, int w, int h, oracle_segs *out);
int oracle_segments3d(const uint8_t *vol, int w, int h, int d, oracle_segs *out);
void oracle_segs_free(oracle_segs *s);

/* CenterlineExtraction: pad like the reference, thin, extract, prune, smooth,
 * flatten.  Outputs are malloc'ed (free with oracle_cl_free). */
typedef struct {
    uint32_t nsegs;
    uint32_t npts;
    float *x, *y, *z;   /* z NULL for 2D */
    uint32_t *idx;      /* nsegs + 1 */
} oracle_cl;

int oracle_centerline2d(const uint8_t *img, int w, int h, int max_segment_length,
                        int smoothing_span, int nthreads, oracle_cl *out);
int oracle_centerline3d(const uint8_t *vol, int w, int h, int d, int max_segment_length,
                        int smoothing_span, int nthreads, oracle_cl *out);
/* Prune + smooth + flatten an existing segment list (the host tail of
 * CenterlineExtraction). dims = 2 or 3. */
int oracle_prune_smooth(const oracle_segs *s, int dims, int max_segment_length,
                        int smoothing_span, oracle_cl *out);
void oracle_cl_free(oracle_cl *c);

/* Foreground test of the reference's binarisation for each pixel type.
 * dtype codes follow bgt_capi.h's bgt_dtype. dims 2: (unsigned)v > 0 as the
 * device conversion does it (2D/CUDA_DeviceHelperFunctions.cuh:101); dims 3:
 * int(v) > 0 on an x86-64 host (3D/CenterlineExtraction.cpp:44). */
int oracle_binarise(int dtype, const void *src, int64_t n, int dims, uint8_t *dst);

/* Single-word rule evaluation, for exhaustive rule tests:
 * 2D: x[8] = N,NE,E,SE,S,SW,W,NW words, dir 0..3 = N,S,E,W; returns deletable mask.
 * 3D: nb[27] indexed 9*(dz+1)+3*(dy+1)+(dx+1); dir 0..5 = U,N,E,D,S,W. */
uint64_t oracle_rule2d(int dir, const uint64_t *x);
uint64_t oracle_rule3d(int dir, const uint64_t *nb);

/* Exhaustive comparison of the 3D rule of direction dir (0..5 = U,N,E,D,S,W)
 * with a rule function of the reference's signature
 * (val, n[26] in the reference's neighbour order, prev) over all 2^26
 * neighbourhoods of a foreground centre.  Returns the number of
 * neighbourhoods on which the deletable sets differ. */
typedef unsigned int (*ref_rule3d_fn)(int dir, unsigned int val, unsigned int *n26, unsigned int prev);
long long oracle_rule3d_exhaustive(int dir, ref_rule3d_fn ref);

/* Deletable-set table of a direction over every neighbourhood of a
 * foreground centre: neighbour i (2D: N,NE,E,SE,S,SW,W,NW; 3D: the 26
 * neighbours in (dz,dy,dx) order, centre skipped) is bit i of the
 * neighbourhood number n, n in bit n%32 of word n/32.  2D: 8 words, 3D:
 * 2^21 words. */
void oracle_rule_table(int dims, int dir, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
