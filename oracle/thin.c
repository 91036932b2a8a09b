/*
 * thin.c -- CPU restatement of the reference's 2D and 3D directional
 * subiteration thinning (global, synchronous semantics).
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): see oracle.h for who may use it.
 *
 * Bits are packed 64 per word along x (bit b of word j = pixel 64*j + b).
 * Every subiteration reads the state from before that subiteration
 * everywhere (a second buffer), which is what the reference's per-tile
 * shared-memory write-back between subiterations implements
 * (2D/CUDA_ThinningKernelMultiBlock2D.cuh:34-44,104-135;
 *  3D/CUDA_ThinningKernel3D_Linear.cuh:755-782).
 */
#include "oracle.h"
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t w64;

/* value of the x-1 neighbour for every bit of c, l = word to the left */
static inline w64 at_xm1(w64 c, w64 l) { return (c << 1) | (l >> 63); }
/* value of the x+1 neighbour, r = word to the right */
static inline w64 at_xp1(w64 c, w64 r) { return (c >> 1) | (r << 63); }

/* ---------------------------------------------------------------------------
 * 2D rule.  One template for "north" boundary points
 * (2D/CUDA_SubiterationKernels2D.cuh:15-40); S, E and W are the same template
 * on the neighbourhood rotated by 180, 90 and 270 degrees (checked
 * exhaustively against the reference functions in tests/test_oracle.py).
 * x0..x7 = the 8 neighbours clockwise, N, NE, E, SE, S, SW, W, NW, after
 * rotation; x0 is the side that must be background for the centre to be a
 * boundary point of that direction.
 * ------------------------------------------------------------------------- */
static inline w64 north_template(w64 x0, w64 x1, w64 x2, w64 x3,
                                 w64 x4, w64 x5, w64 x6, w64 x7)
{
    w64 a = ~x1 & ~x7 & (x2 ^ x3 ^ ~x4) & (x3 ^ x5) & (x3 ^ x6);
    w64 b = x2 & x4 & (x6 | ~x7);
    w64 c = ~x1 & x4 & x6;
    w64 d = ~x6 & ~x7 & (x1 ^ x5) & (x2 ^ x5) & (x4 ^ ~x5);
    w64 e = ~x1 & ~x2 & ~x3 & x6 & x7;
    return ~x0 & (a | b | c | d | e);
}

/* rotation of the N,NE,...,NW ring for N,S,E,W (order of application) */
static const int rot2d[4] = {0, 4, 2, 6};

uint64_t oracle_rule2d(int dir, const uint64_t *X)
{
    int r = rot2d[dir & 3];
    return north_template(X[(0 + r) & 7], X[(1 + r) & 7], X[(2 + r) & 7], X[(3 + r) & 7],
                          X[(4 + r) & 7], X[(5 + r) & 7], X[(6 + r) & 7], X[(7 + r) & 7]);
}

int oracle_thin2d(uint8_t *img, int w, int h, int nthreads)
{
    if (w <= 0 || h <= 0) return 0;
    const int nw = (w + 63) / 64;
    const int stride = nw + 2;              /* one zero guard word each side */
    const size_t nwords = (size_t)stride * (size_t)(h + 2); /* guard rows */
    w64 *cur = (w64 *)calloc(nwords, sizeof(w64));
    w64 *nxt = (w64 *)calloc(nwords, sizeof(w64));
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            if (img[(size_t)y * w + x])
                cur[(size_t)(y + 1) * stride + 1 + x / 64] |= (w64)1 << (x % 64);

    int iters = 0;
    for (;;) {
        long long deleted_iter = 0;
        iters++;
        for (int s = 0; s < 4; s++) {
            const int r = rot2d[s];
            long long deleted = 0;
#pragma omp parallel for reduction(+ : deleted) schedule(static)
            for (int y = 0; y < h; y++) {
                const w64 *up = cur + (size_t)y * stride;
                const w64 *cp = up + stride;
                const w64 *dn = cp + stride;
                w64 *out = nxt + (size_t)(y + 1) * stride;
                for (int j = 1; j <= nw; j++) {
                    w64 X[8];
                    X[0] = up[j];
                    X[1] = at_xp1(up[j], up[j + 1]);
                    X[2] = at_xp1(cp[j], cp[j + 1]);
                    X[3] = at_xp1(dn[j], dn[j + 1]);
                    X[4] = dn[j];
                    X[5] = at_xm1(dn[j], dn[j - 1]);
                    X[6] = at_xm1(cp[j], cp[j - 1]);
                    X[7] = at_xm1(up[j], up[j - 1]);
                    w64 del = cp[j] & north_template(X[(0 + r) & 7], X[(1 + r) & 7], X[(2 + r) & 7],
                                                     X[(3 + r) & 7], X[(4 + r) & 7], X[(5 + r) & 7],
                                                     X[(6 + r) & 7], X[(7 + r) & 7]);
                    out[j] = cp[j] & ~del;
                    deleted += __builtin_popcountll(del);
                }
            }
            w64 *t = cur; cur = nxt; nxt = t;
            deleted_iter += deleted;
        }
        if (deleted_iter == 0) break;
    }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            img[(size_t)y * w + x] =
                (uint8_t)((cur[(size_t)(y + 1) * stride + 1 + x / 64] >> (x % 64)) & 1);
    free(cur);
    free(nxt);
    return iters;
}

/* ---------------------------------------------------------------------------
 * 3D rule.  One template, the "up" boundary rule
 * (3D/CUDA_SubiterationKernels3D.cuh:14-49); the other five directions are
 * its images under cube symmetries (found and checked exhaustively over all
 * 2^26 neighbourhoods against the reference functions).  In the template's
 * own frame, layer a = -1 is the side that must be background (T), a = +1 the
 * opposite layer (B); b = -1/+1 are its "n"/"s" rows, c = -1/+1 its "w"/"e"
 * columns.
 *
 * Direction frames: local axis k (a, b, c) maps to global axis perm[k]
 * (0 = z, 1 = y, 2 = x) with sign.  Application order per iteration is
 * U, N, E, D, S, W (3D/CUDA_ThinningKernel3D_Linear.cuh:755-782).  Note the
 * reference's 3D "East" removes points whose x-1 neighbour is background.
 * ------------------------------------------------------------------------- */
static const int frame_perm[6][3] = {
    {0, 1, 2}, /* U: T at z-1 */
    {1, 0, 2}, /* N: T at y-1 */
    {2, 0, 1}, /* E: T at x-1 */
    {0, 1, 2}, /* D: T at z+1 */
    {1, 0, 2}, /* S: T at y+1 */
    {2, 0, 1}, /* W: T at x+1 */
};
static const int frame_flip[6] = {0, 0, 0, 1, 1, 1}; /* negate local axis a */

/* local index -> global index (both 9*(.+1)+3*(.+1)+(.+1)) per direction */
static int frame_map[6][27];
static int frame_map_ready = 0;

static void build_frames(void)
{
    if (frame_map_ready) return;
    for (int d = 0; d < 6; d++)
        for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++)
                for (int c = -1; c <= 1; c++) {
                    int loc[3] = {frame_flip[d] ? -a : a, b, c};
                    int g[3];
                    for (int k = 0; k < 3; k++) g[frame_perm[d][k]] = loc[k];
                    frame_map[d][9 * (a + 1) + 3 * (b + 1) + (c + 1)] =
                        9 * (g[0] + 1) + 3 * (g[1] + 1) + (g[2] + 1);
                }
    frame_map_ready = 1;
}

#define L(a, b, c) n[9 * ((a) + 1) + 3 * ((b) + 1) + ((c) + 1)]

/* deletable mask of the up template; n[] is in the template's own frame */
static inline w64 up_template(const w64 *n)
{
    const w64 T = L(-1, 0, 0), B = L(1, 0, 0);
    const w64 Tn = L(-1, -1, 0), Ts = L(-1, 1, 0), Tw = L(-1, 0, -1), Te = L(-1, 0, 1);
    const w64 Tnw = L(-1, -1, -1), Tne = L(-1, -1, 1), Tsw = L(-1, 1, -1), Tse = L(-1, 1, 1);
    const w64 Mn = L(0, -1, 0), Ms = L(0, 1, 0), Mw = L(0, 0, -1), Me = L(0, 0, 1);
    const w64 Mnw = L(0, -1, -1), Mne = L(0, -1, 1), Msw = L(0, 1, -1), Mse = L(0, 1, 1);
    const w64 Bn = L(1, -1, 0), Bs = L(1, 1, 0), Bw = L(1, 0, -1), Be = L(1, 0, 1);
    const w64 Bnw = L(1, -1, -1), Bne = L(1, -1, 1), Bsw = L(1, 1, -1), Bse = L(1, 1, 1);

    /* anything in the middle ring or the bottom corners */
    const w64 mid = Mnw | Mn | Mne | Mw | Me | Msw | Ms | Mse | Bnw | Bne | Bsw | Bse;
    const w64 bot_we = Bw | Be, bot_ns = Bn | Bs;
    /* single bottom edge-centre "arms" with their flanks clear */
    const w64 arm_n = Bn & ~Bs & ~Ms & ~Mse & ~Bse;
    const w64 arm_s = Bs & ~Bn & ~Mn & ~Mne & ~Bne;
    const w64 arm_w = Bw & ~Be & ~Me;
    const w64 arm_e = Be & ~Bw & ~Mw;
    const w64 arm_e_s = arm_e & ~Msw & ~Bsw;
    const w64 arm_e_n = arm_e & ~Mnw & ~Bnw;

    const w64 m1 = mid | bot_we | bot_ns;
    const w64 m5 = ((mid | bot_we) & ((arm_n & ~Msw & ~Bsw) | (arm_s & ~Mnw & ~Bnw))) |
                   ((mid | bot_ns) & ((arm_e_n & ~Msw & ~Bsw) | (arm_w & ~Mne & ~Mse & ~Bne & ~Bse)));
    const w64 m6 = (arm_e_s & Bn & ~Bs & ~Ms) | (arm_e_n & Bs & ~Bn & ~Mn) | (arm_w & (arm_n | arm_s));
    const w64 m4 = (~Tnw & ~Tsw & ((Tne & Mne & ~Tse) | (Tse & Mse & ~Tne))) |
                   (~Tne & ~Tse & ((Tnw & Mnw & ~Tsw) | (Tsw & Msw & ~Tnw)));
    const w64 m2 = (~Tn & ~Tne & ~Te & ((~Tnw & ~Tw & Ms) | (~Ts & ~Tse & Mw))) |
                   (~Ts & ~Tsw & ~Tw & ((~Te & ~Tse & Mn) | (~Tnw & ~Tn & Me)));
    const w64 m3 = (~Tw & Me & ((~Ts & ~Tsw & Mn) | (~Tnw & ~Tn & Ms))) |
                   (~Te & Mw & ((~Tn & ~Tne & Ms) | (~Ts & ~Tse & Mn)));
    const w64 cross_clear = ~(Tn | Tw | Te | Ts);
    const w64 corner_clear = ~(Tnw | Tne | Tsw | Tse);
    return ~T & ((cross_clear & ((B & m4) | (corner_clear & ((B & m1) | (~B & (m5 | m6)))))) |
                 (B & (m2 | m3)));
}
#undef L

uint64_t oracle_rule3d(int dir, const uint64_t *nb)
{
    build_frames();
    w64 loc[27];
    for (int i = 0; i < 27; i++) loc[i] = nb[frame_map[dir][i]];
    return up_template(loc);
}

/* 32 neighbourhoods per call: neighbour i < 5 varies across the 32 bit
 * lanes, neighbours 5..25 (reference order, centre skipped) follow the bits
 * of `hi`. */
long long oracle_rule3d_exhaustive(int dir, ref_rule3d_fn ref)
{
    build_frames();
    long long bad = 0;
    unsigned int lane_pat[5];
    for (int i = 0; i < 5; i++) {
        unsigned int w = 0;
        for (int l = 0; l < 32; l++)
            if ((l >> i) & 1) w |= 1u << l;
        lane_pat[i] = w;
    }
    for (uint32_t hi = 0; hi < (1u << 21); hi++) {
        unsigned int n[26];
        w64 g[27], loc[27];
        for (int i = 0; i < 26; i++)
            n[i] = i < 5 ? lane_pat[i] : (((hi >> (i - 5)) & 1) ? 0xffffffffu : 0u);
        for (int p = 0, i = 0; p < 27; p++) g[p] = p == 13 ? 0xffffffffu : (w64)n[i++];
        for (int i = 0; i < 27; i++) loc[i] = g[frame_map[dir][i]];
        const unsigned int mine = (unsigned int)up_template(loc);
        /* reference returns val with the deletable bits cleared (prev = 0) */
        const unsigned int theirs = ~ref(dir, 0xffffffffu, n, 0u);
        bad += __builtin_popcount(mine ^ theirs);
    }
    return bad;
}

/* Deletable-set table of direction dir over every neighbourhood of a
 * foreground centre, in the layout of the device self-test (bgt_rule_table):
 * neighbour i is bit i of the neighbourhood number n, n in bit n%32 of word
 * n/32.  2D: 8 words, 3D: 2^21 words. */
void oracle_rule_table(int dims, int dir, uint32_t *out)
{
    unsigned int lane_pat[5];
    for (int i = 0; i < 5; i++) {
        unsigned int w = 0;
        for (int l = 0; l < 32; l++)
            if ((l >> i) & 1) w |= 1u << l;
        lane_pat[i] = w;
    }
    if (dims == 2) {
        for (uint32_t hi = 0; hi < 8; hi++) {
            uint64_t X[8];
            for (int i = 0; i < 8; i++) X[i] = i < 5 ? lane_pat[i] : (((hi >> (i - 5)) & 1) ? 0xffffffffu : 0u);
            out[hi] = (uint32_t)oracle_rule2d(dir, X);
        }
        return;
    }
    build_frames();
    for (uint32_t hi = 0; hi < (1u << 21); hi++) {
        w64 g[27], loc[27];
        for (int p = 0, i = 0; p < 27; p++) {
            if (p == 13) {
                g[p] = 0xffffffffu;
                continue;
            }
            g[p] = i < 5 ? lane_pat[i] : (((hi >> (i - 5)) & 1) ? 0xffffffffu : 0u);
            i++;
        }
        for (int i = 0; i < 27; i++) loc[i] = g[frame_map[dir][i]];
        out[hi] = (uint32_t)up_template(loc);
    }
}

int oracle_thin3d(uint8_t *vol, int w, int h, int d, int nthreads)
{
    if (w <= 0 || h <= 0 || d <= 0) return 0;
    build_frames();
    const int nw = (w + 63) / 64;
    const size_t rs = (size_t)nw + 2;          /* row stride with guard words */
    const size_t ps = rs * (size_t)(h + 2);     /* plane stride with guard rows */
    const size_t nwords = ps * (size_t)(d + 2); /* guard planes */
    w64 *cur = (w64 *)calloc(nwords, sizeof(w64));
    w64 *nxt = (w64 *)calloc(nwords, sizeof(w64));
    w64 *uni = (w64 *)calloc(nwords, sizeof(w64)); /* pre-test union */
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
                if (vol[((size_t)z * h + y) * w + x])
                    cur[(size_t)(z + 1) * ps + (size_t)(y + 1) * rs + 1 + x / 64] |= (w64)1 << (x % 64);

    int iters = 0;
    const long long nrows = (long long)d * h;
    for (;;) {
        iters++;
        long long deleted_iter = 0;
        /* step -1 = pre-test, steps 0..5 = U,N,E,D,S,W */
        for (int step = -1; step < 6; step++) {
            long long deleted = 0;
#pragma omp parallel for reduction(+ : deleted) schedule(static)
            for (long long zy = 0; zy < nrows; zy++) {
                const int z = (int)(zy / h), y = (int)(zy % h);
                const size_t base = (size_t)(z + 1) * ps + (size_t)(y + 1) * rs;
                for (int j = 1; j <= nw; j++) {
                    w64 g[27];
                    for (int dz = -1; dz <= 1; dz++)
                        for (int dy = -1; dy <= 1; dy++) {
                            const w64 *row = cur + base + (ptrdiff_t)dz * (ptrdiff_t)ps +
                                             (ptrdiff_t)dy * (ptrdiff_t)rs;
                            const int k = 9 * (dz + 1) + 3 * (dy + 1);
                            g[k + 0] = at_xm1(row[j], row[j - 1]);
                            g[k + 1] = row[j];
                            g[k + 2] = at_xp1(row[j], row[j + 1]);
                        }
                    const w64 val = g[13];
                    if (step < 0) {
                        w64 u = 0;
                        for (int dir = 0; dir < 6; dir++) {
                            w64 loc[27];
                            for (int i = 0; i < 27; i++) loc[i] = g[frame_map[dir][i]];
                            u |= up_template(loc);
                        }
                        uni[base + j] = u & val;
                    } else {
                        w64 loc[27];
                        for (int i = 0; i < 27; i++) loc[i] = g[frame_map[step][i]];
                        const w64 del = val & up_template(loc) & uni[base + j];
                        nxt[base + j] = val & ~del;
                        deleted += __builtin_popcountll(del);
                    }
                }
            }
            if (step >= 0) {
                w64 *t = cur; cur = nxt; nxt = t;
                deleted_iter += deleted;
            }
        }
        if (deleted_iter == 0) break;
    }
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
                vol[((size_t)z * h + y) * w + x] = (uint8_t)(
                    (cur[(size_t)(z + 1) * ps + (size_t)(y + 1) * rs + 1 + x / 64] >> (x % 64)) & 1);
    free(cur);
    free(nxt);
    free(uni);
    return iters;
}
