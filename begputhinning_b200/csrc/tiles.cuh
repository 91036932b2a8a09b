// tiles.cuh -- the per-tile pass bodies shared by the plain (one launch per
// pass) driver and the persistent batched engine.
//
// 2D tile, configuration (K, S, NW): a CTA of NW warps.  Warp w owns 32
// consecutive rows, one row per lane; the lane holds S+2 words of its row in
// registers (S core words plus one halo word each side).  K subiterations run
// on those registers: a lane forms the x-neighbours of its own row by funnel
// shifts of adjacent registers (two per word) and receives the three words
// of the row above and of the row below (centre, x+1, x-1) by warp shuffles,
// which keeps the integer pipe for the rule itself.  Lanes 0..K-1 and
// 32-K..31 are halo rows (their state is only valid for the lanes inside
// them), so a warp keeps 32-2K core rows and consecutive warps overlap by 2K
// rows.  The tile (core plus halo) is staged into shared memory by one TMA
// load; out-of-image parts read as zero.
//
// 3D tile, configuration (NWX, TZ): one subiteration per pass.  Warp w owns
// word column x0+w; its lanes are 32 consecutive rows (30 core rows and one
// halo row each side).  The warp marches through TZ+2 planes keeping a
// 3-plane window of 3x3 (row, word) neighbourhoods in registers: three
// shared-memory loads per plane, y-neighbours by shuffles, x-neighbours by
// funnel shifts.  Mode 0 evaluates all six directional rules (the pre-test
// union of the iteration, stored per word) and applies U; modes 1..5 apply
// N, E, D, S, W masked by the stored union.
#pragma once
#include "common.cuh"
#include "rules.cuh"

namespace bgt {

// ------------------------------------------------------------ changes -----
// A tile reports its change as a mask: kTileChanged when any core pixel was
// deleted, plus one bit per neighbour tile whose K-pixel ring reaches a
// deleted pixel (bit band_bit(dy, dx) for the neighbour at offset (dy, dx)).
// Tiles that do not work out the bands report all of them.
constexpr uint32_t kTileChanged = 0x100u;
constexpr uint32_t kAllBands = 0xFFu;
__host__ __device__ constexpr int band_bit(int dy, int dx)
{
    return (dy + 1) * 3 + (dx + 1) - ((dy + 1) * 3 + (dx + 1) > 4 ? 1 : 0);
}

// ---------------------------------------------------------------- 2D ------
// The rule on one word of the lane's row: `o` the word, `n`/`p` the words
// after/before it (pass-start values).  Returns the word after deletion.
template <int DIR>
__device__ __forceinline__ uint32_t word2d(uint32_t o, uint32_t n, uint32_t p)
{
    const uint32_t xp = at_xp1(o, n), xm = at_xm1(o, p);
    uint32_t X[8];
    X[0] = __shfl_up_sync(kFull, o, 1);
    X[1] = __shfl_up_sync(kFull, xp, 1);
    X[7] = __shfl_up_sync(kFull, xm, 1);
    X[4] = __shfl_down_sync(kFull, o, 1);
    X[3] = __shfl_down_sync(kFull, xp, 1);
    X[5] = __shfl_down_sync(kFull, xm, 1);
    X[2] = xp;
    X[6] = xm;
    return keep2d<DIR>(o, X);
}

// One subiteration on the lane's S+2 words, two words per step so that the
// shuffles and rules of both overlap.  Steps whose two centre words are empty
// in every lane of the warp are skipped (nothing to delete there).
template <int S, int DIR>
__device__ __forceinline__ void subit2d(uint32_t (&v)[S + 2])
{
    static_assert(S % 2 == 0, "pairs of words");
    uint32_t prev_old = 0;
#pragma unroll
    for (int j = 0; j < S + 2; j += 2) {
        const uint32_t o0 = v[j], o1 = v[j + 1];
        const uint32_t on = j + 2 < S + 2 ? v[j + 2] : 0u;
        if (__any_sync(kFull, (o0 | o1) != 0u)) {
            v[j] = word2d<DIR>(o0, o1, prev_old);
            v[j + 1] = word2d<DIR>(o1, on, o0);
        }
        prev_old = o1;
    }
}

// The pass's last subiteration: only the S core words are kept afterwards,
// so they are processed as the pairs (1,2) .. (S-1,S) and the two halo
// words are left as they are.
template <int S, int DIR>
__device__ __forceinline__ void subit2d_core(uint32_t (&v)[S + 2])
{
    uint32_t prev_old = v[0];
#pragma unroll
    for (int j = 1; j <= S; j += 2) {
        const uint32_t o0 = v[j], o1 = v[j + 1], on = v[j + 2];
        if (__any_sync(kFull, (o0 | o1) != 0u)) {
            v[j] = word2d<DIR>(o0, o1, prev_old);
            v[j + 1] = word2d<DIR>(o1, on, o0);
        }
        prev_old = o1;
    }
}

template <int K, int S, int PH, int I = 0>
__device__ __forceinline__ void run_subits2d(uint32_t (&v)[S + 2])
{
    if constexpr (I + 1 < K) {
        subit2d<S, (PH + I) & 3>(v);
        run_subits2d<K, S, PH, I + 1>(v);
    } else if constexpr (I + 1 == K) {
        subit2d_core<S, (PH + I) & 3>(v);
    }
}

template <int K, int S, int NW>
struct Cfg2D {
    static constexpr int kK = K, kS = S, kNW = NW;
    static constexpr int CORE = 32 - 2 * K;   // core rows per warp
    static constexpr int TH = NW * CORE;      // core rows per tile
    static constexpr int BW = S + 8;          // box width in words (x0-4 .. x0+S+4)
    static constexpr int BH = TH + 2 * K;     // box height in rows
    static constexpr int SMEM = BW * BH * 4;  // bytes
    static constexpr int THREADS = NW * 32;
    static_assert(S % 4 == 0, "S must be a multiple of 4 (TMA x alignment, 128-bit stores)");
    static_assert(BW <= 256 && BH <= 256, "TMA box too large");
};

// Issue the TMA load of the box of a 2D tile (core plus halo) for pass q
// into smem; completes on bar.  One thread calls it.  Serves Cfg2D and Cfg2DX.
template <class C>
__device__ __forceinline__ void tile2d_issue(const Inst &in, int q, int tile, uint32_t *smem, uint64_t *bar)
{
    const int tx = tile % in.tiles_x, ty = tile / in.tiles_x;
    const CUtensorMap *tm = in.tmap + (q & 1);
    tmap_acquire(tm);
    mbar_arrive_expect_tx(bar, (uint32_t)(C::BW * C::BH * 4));
    tma_load_2d(smem, tm, tx * C::kS - 4, ty * C::TH - C::kK, bar);
}

// Process one 2D tile for pass q (phase PH = first direction of the pass)
// from its box in smem.  Returns the change mask: to thread 0 with the
// border bands (accumulated in *band, which it resets), to the other tile
// threads kTileChanged or 0.
template <class C, int PH>
__device__ uint32_t tile2d(const Inst &in, int q, int tile, const uint32_t *smem, uint32_t *band)
{
    constexpr int K = C::kK, S = C::kS, CORE = C::CORE, BW = C::BW;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = tile % in.tiles_x, ty = tile / in.tiles_x;
    const int x0 = tx * S, y0 = ty * C::TH;
    uint32_t *dst = in.buf[(q + 1) & 1];

    const int r = warp * CORE + lane;  // box row of this lane
    const uint32_t *row = smem + r * BW;
    uint32_t v[S + 2];
    v[0] = row[3];
#pragma unroll
    for (int c = 0; c < S / 4; c++) {
        const uint4 t = *reinterpret_cast<const uint4 *>(row + 4 + 4 * c);
        v[1 + 4 * c] = t.x;
        v[2 + 4 * c] = t.y;
        v[3 + 4 * c] = t.z;
        v[4 + 4 * c] = t.w;
    }
    v[S + 1] = row[S + 4];

    run_subits2d<K, S, PH>(v);

    // change of the core words over the pass: the box in smem still holds
    // the pass's input
    uint32_t chg = 0;
#pragma unroll
    for (int c = 0; c < S; c++) chg |= v[1 + c] ^ row[4 + c];
    const int y = y0 + r - K;  // image row of this lane
    const bool core = lane >= K && lane < 32 - K && y < in.H;
    uint32_t bm = 0;
    if (core) {
        uint32_t *drow = dst + (size_t)y * in.P + x0;
#pragma unroll
        for (int c = 0; c < S / 4; c++)
            if (x0 + 4 * c < in.P)
                *reinterpret_cast<uint4 *>(drow + 4 * c) =
                    make_uint4(v[1 + 4 * c], v[2 + 4 * c], v[3 + 4 * c], v[4 + 4 * c]);
        // border bands: the first/last K core rows and the K pixels at each
        // x edge reach into the ring of the neighbour on that side
        const int cr = r - K;  // core row within the tile
        const bool top = cr < K, bot = cr >= C::TH - K;
        const bool lft = ((v[1] ^ row[4]) & ((1u << K) - 1u)) != 0;
        const bool rgt = ((v[S] ^ row[S + 3]) & ~(0xFFFFFFFFu >> K)) != 0;
        const bool any = chg != 0;
        bm = (top && any ? 1u << band_bit(-1, 0) : 0u) | (bot && any ? 1u << band_bit(1, 0) : 0u) |
             (lft ? 1u << band_bit(0, -1) : 0u) | (rgt ? 1u << band_bit(0, 1) : 0u) |
             (top && lft ? 1u << band_bit(-1, -1) : 0u) | (top && rgt ? 1u << band_bit(-1, 1) : 0u) |
             (bot && lft ? 1u << band_bit(1, -1) : 0u) | (bot && rgt ? 1u << band_bit(1, 1) : 0u);
    }
    bm = __reduce_or_sync(kFull, bm);
    if (lane == 0 && bm) atomicOr(band, bm);
    uint32_t m = tile_sync_or(core && chg != 0) ? kTileChanged : 0u;
    if (threadIdx.x == 0) {
        m |= *band;
        *band = 0;
    }
    return m;
}

// ------------------------------------------- 2D, shared warp edges -------
// Variant: the NW warps of a tile form one band of 32*NW rows.  After every
// subiteration each warp publishes its first and last row (lanes 0 and 31)
// in shared memory; the warp below/above reads them in place of the shuffle
// that would otherwise wrap inside the warp.  Only the band's outer K rows
// are halo: 32*NW - 2K core rows instead of NW*(32 - 2K).
template <int K, int S, int NW>
struct Cfg2DX {
    static constexpr int kK = K, kS = S, kNW = NW;
    static constexpr int TH = 32 * NW - 2 * K;  // core rows per tile
    static constexpr int BW = S + 8;            // box width in words
    static constexpr int BH = 32 * NW;          // box rows
    static constexpr int EX = S + 2;            // words of an exchanged row
    static constexpr int SMEM = BW * BH * 4 + 2 * 2 * NW * EX * 4;
    static constexpr int THREADS = NW * 32;
    static_assert(S % 4 == 0, "S must be a multiple of 4");
    static_assert(BW <= 256 && BH <= 256, "TMA box too large");
};

// One subiteration with edge rows from shared memory: ex_up is the row above
// lane 0 (warps > 0), ex_dn the row below lane 31 (warps < NW-1).
template <int S, int DIR>
__device__ __forceinline__ void subit2d_x(uint32_t (&v)[S + 2], uint32_t &chg, const uint32_t *ex_up,
                                          const uint32_t *ex_dn, bool use_up, bool use_dn)
{
    uint32_t prev_old = 0, up_prev = 0, dn_prev = 0;
    uint32_t old_j = v[0];
    uint32_t up_j = __shfl_up_sync(kFull, old_j, 1);
    uint32_t dn_j = __shfl_down_sync(kFull, old_j, 1);
    if (use_up) up_j = ex_up[0];
    if (use_dn) dn_j = ex_dn[0];
#pragma unroll
    for (int j = 0; j < S + 2; j++) {
        uint32_t old_n = 0, up_n = 0, dn_n = 0;
        if (j + 1 < S + 2) {
            old_n = v[j + 1];
            up_n = __shfl_up_sync(kFull, old_n, 1);
            dn_n = __shfl_down_sync(kFull, old_n, 1);
            if (use_up) up_n = ex_up[j + 1];
            if (use_dn) dn_n = ex_dn[j + 1];
        }
        uint32_t X[8];
        X[0] = up_j;
        X[1] = at_xp1(up_j, up_n);
        X[2] = at_xp1(old_j, old_n);
        X[3] = at_xp1(dn_j, dn_n);
        X[4] = dn_j;
        X[5] = at_xm1(dn_j, dn_prev);
        X[6] = at_xm1(old_j, prev_old);
        X[7] = at_xm1(up_j, up_prev);
        const uint32_t del = old_j & rule2d<DIR>(X);
        v[j] = old_j ^ del;
        if (j >= 1 && j <= S) chg |= del;
        prev_old = old_j;
        up_prev = up_j;
        dn_prev = dn_j;
        old_j = old_n;
        up_j = up_n;
        dn_j = dn_n;
    }
}

template <class C, int PH, int I = 0>
__device__ __forceinline__ void run_subits2d_x(uint32_t (&v)[C::kS + 2], uint32_t &chg, uint32_t *ex, int warp,
                                               int lane)
{
    if constexpr (I < C::kK) {
        constexpr int S = C::kS, NW = C::kNW, EX = C::EX;
        // publish this warp's edge rows of the current state (buffer I & 1)
        uint32_t *buf = ex + (I & 1) * 2 * NW * EX;  // [top rows of NW warps | bottom rows of NW warps]
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < S + 2; j++) buf[warp * EX + j] = v[j];
        }
        if (lane == 31) {
#pragma unroll
            for (int j = 0; j < S + 2; j++) buf[(NW + warp) * EX + j] = v[j];
        }
        tile_sync();
        const bool use_up = lane == 0 && warp > 0, use_dn = lane == 31 && warp < NW - 1;
        const uint32_t *ex_up = buf + (NW + max(warp - 1, 0)) * EX;  // bottom row of the warp above
        const uint32_t *ex_dn = buf + min(warp + 1, NW - 1) * EX;    // top row of the warp below
        subit2d_x<S, (PH + I) & 3>(v, chg, ex_up, ex_dn, use_up, use_dn);
        run_subits2d_x<C, PH, I + 1>(v, chg, ex, warp, lane);
    }
}

template <class C, int PH>
__device__ uint32_t tile2dx(const Inst &in, int q, int tile, uint32_t *smem)
{
    constexpr int K = C::kK, S = C::kS, BW = C::BW, BH = C::BH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = tile % in.tiles_x, ty = tile / in.tiles_x;
    const int x0 = tx * S, y0 = ty * C::TH;
    uint32_t *dst = in.buf[(q + 1) & 1];
    uint32_t *ex = smem + BW * BH;

    const int r = warp * 32 + lane;  // box row of this lane
    const uint32_t *row = smem + r * BW;
    uint32_t v[S + 2];
    v[0] = row[3];
#pragma unroll
    for (int c = 0; c < S / 4; c++) {
        const uint4 t = *reinterpret_cast<const uint4 *>(row + 4 + 4 * c);
        v[1 + 4 * c] = t.x;
        v[2 + 4 * c] = t.y;
        v[3 + 4 * c] = t.z;
        v[4 + 4 * c] = t.w;
    }
    v[S + 1] = row[S + 4];

    uint32_t chg = 0;
    run_subits2d_x<C, PH>(v, chg, ex, warp, lane);

    const int y = y0 + r - K;  // image row of this lane
    const bool core = r >= K && r < BH - K && y < in.H;
    if (core) {
        uint32_t *drow = dst + (size_t)y * in.P + x0;
#pragma unroll
        for (int c = 0; c < S / 4; c++)
            if (x0 + 4 * c < in.P)
                *reinterpret_cast<uint4 *>(drow + 4 * c) =
                    make_uint4(v[1 + 4 * c], v[2 + 4 * c], v[3 + 4 * c], v[4 + 4 * c]);
    }
    return tile_sync_or(core && chg != 0) ? kTileChanged | kAllBands : 0u;
}

// ---------------------------------------------------------------- 3D ------
template <int NWX, int TZ>
struct Cfg3D {
    static constexpr int kNWX = NWX, kTZ = TZ;
    static constexpr int TY = 30;             // core rows per tile (lanes 1..30)
    static constexpr int BW = NWX + 8;        // box width in words
    static constexpr int BH = 32;             // box rows
    static constexpr int BD = TZ + 2;         // box planes
    static constexpr int IMG = BW * BH * BD * 4;  // bytes of the image box
    static constexpr int UNI = NWX * BH * TZ * 4; // bytes of the union box (core words and planes)
    static constexpr int SMEM = IMG + UNI;
    static constexpr int THREADS = NWX * 32;
    static_assert(NWX % 4 == 0, "NWX must be a multiple of 4 (TMA x alignment)");
    static_assert(BD <= 256, "TMA box too large");
};

__device__ __forceinline__ void plane3x3(const uint32_t *p, int col, uint32_t (&o)[9])
{
    const uint32_t l = p[col - 1], c = p[col], r = p[col + 1];
    const uint32_t lu = __shfl_up_sync(kFull, l, 1), cu = __shfl_up_sync(kFull, c, 1),
                   ru = __shfl_up_sync(kFull, r, 1);
    const uint32_t ld = __shfl_down_sync(kFull, l, 1), cd = __shfl_down_sync(kFull, c, 1),
                   rd = __shfl_down_sync(kFull, r, 1);
    o[0] = at_xm1(cu, lu); o[1] = cu; o[2] = at_xp1(cu, ru);
    o[3] = at_xm1(c, l);   o[4] = c;  o[5] = at_xp1(c, r);
    o[6] = at_xm1(cd, ld); o[7] = cd; o[8] = at_xp1(cd, rd);
}

// Issue the TMA loads of a 3D tile for pass q: the image box (core plus
// one halo word/row/plane) and, in passes 1..5 of an iteration, the union
// box behind it.  One thread calls it.
template <class C>
__device__ __forceinline__ void tile3d_issue(const Inst &in, int q, int tile, uint32_t *smem, uint64_t *bar)
{
    const int tx = tile % in.tiles_x;
    const int ty = (tile / in.tiles_x) % in.tiles_y;
    const int tz = tile / (in.tiles_x * in.tiles_y);
    const int x0 = tx * C::kNWX, y0 = ty * C::TY, z0 = tz * C::kTZ;
    const CUtensorMap *tm = in.tmap + (q & 1);
    tmap_acquire(tm);
    if (q % 6 == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)C::IMG);
    } else {
        tmap_acquire(in.tmap + 2);
        mbar_arrive_expect_tx(bar, (uint32_t)(C::IMG + C::UNI));
        tma_load_3d(smem + C::IMG / 4, in.tmap + 2, x0, y0 - 1, z0, bar);
    }
    tma_load_3d(smem, tm, x0 - 4, y0 - 1, z0 - 1, bar);
}

// MODE 0: pre-test union (stored) + U.  MODE 1..5: N, E, D, S, W.
template <class C, int MODE>
__device__ uint32_t tile3d(const Inst &in, int q, int tile, const uint32_t *smem)
{
    constexpr int NWX = C::kNWX, TZ = C::kTZ, BW = C::BW, BH = C::BH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = tile % in.tiles_x;
    const int ty = (tile / in.tiles_x) % in.tiles_y;
    const int tz = tile / (in.tiles_x * in.tiles_y);
    const int x0 = tx * NWX, y0 = ty * C::TY, z0 = tz * TZ;
    uint32_t *dst = in.buf[(q + 1) & 1];
    const uint32_t *usm = smem + C::IMG / 4;  // union box: [plane][row][word]

    const int col = 4 + warp;
    const int x = x0 + warp, y = y0 + lane - 1;
    const int wwords = (in.W + 31) >> 5;
    const bool lane_live = lane >= 1 && lane <= 30 && y < in.H && x < wwords;
    const size_t plane_words = (size_t)in.P * in.H;
    const size_t base = (size_t)y * in.P + x;

    uint32_t A[9], B[9], Cn[9];
    plane3x3(smem + (0 * BH + lane) * BW, col, A);
    plane3x3(smem + (1 * BH + lane) * BW, col, B);
    uint32_t chg = 0;
#pragma unroll 1
    for (int zz = 0; zz < TZ; zz++) {
        plane3x3(smem + ((zz + 2) * BH + lane) * BW, col, Cn);
        const int z = z0 + zz;
        const bool live = lane_live && z < in.D;
        const uint32_t val = B[4];
        uint32_t nv = val;
        // passes 1..5 delete only voxels of the iteration's union: words whose
        // union is empty in every lane skip the rule
        const uint32_t cand = MODE == 0 ? val : val & usm[(zz * BH + lane) * NWX + warp];
        if (__any_sync(kFull, live && cand != 0u)) {
            uint32_t g[27];
#pragma unroll
            for (int i = 0; i < 9; i++) {
                g[i] = A[i];
                g[9 + i] = B[i];
                g[18 + i] = Cn[i];
            }
            const size_t idx = (size_t)z * plane_words + base;
            uint32_t del;
            if constexpr (MODE == 0) {
                const uint32_t du = rule3d<0>(g);
                const uint32_t un = du | rule3d<1>(g) | rule3d<2>(g) | rule3d<3>(g) | rule3d<4>(g) | rule3d<5>(g);
                if (live) in.uni[idx] = un & val;
                del = val & du;
            } else {
                del = cand & rule3d<MODE>(g);
            }
            nv = val & ~del;
            if (live) chg |= del;
        }
        if (live) dst[(size_t)z * plane_words + base] = nv;
#pragma unroll
        for (int i = 0; i < 9; i++) {
            A[i] = B[i];
            B[i] = Cn[i];
        }
    }
    // the barrier orders every thread's stores before thread 0's fence and
    // release (engine) or the end of the launch (plain path)
    return tile_sync_or(chg != 0u) ? kTileChanged | kAllBands : 0u;
}

// ------------------------------------------------------------ activity ----
// A tile may skip pass q when no tile of its 3x3(x3) neighbourhood changed
// during the last `window` passes: its neighbourhood has then been constant
// long enough to be a local fixed point for every direction.  Empty tiles
// (lc == kNever) never change.
__device__ __forceinline__ int nbr_last_change(const Inst &in, int tile)
{
    const int tx = tile % in.tiles_x;
    const int ty = (tile / in.tiles_x) % in.tiles_y;
    const int tz = tile / (in.tiles_x * in.tiles_y);
    int m = kNever;
    for (int dz = -1; dz <= 1; dz++) {
        const int z = tz + dz;
        if (z < 0 || z >= in.tiles_z) continue;
        for (int dy = -1; dy <= 1; dy++) {
            const int yy = ty + dy;
            if (yy < 0 || yy >= in.tiles_y) continue;
            for (int dx = -1; dx <= 1; dx++) {
                const int xx = tx + dx;
                if (xx < 0 || xx >= in.tiles_x) continue;
                m = max(m, ld_cg_int(in.lc + (z * in.tiles_y + yy) * in.tiles_x + xx));
            }
        }
    }
    return m;
}

__device__ __forceinline__ bool tile_active(const Inst &in, int tile, int q)
{
    if (ld_cg_int(in.lc + tile) == kNever) return false;
    if (in.dims == 2) return nbr_last_change(in, tile) >= q - in.window;
    // 3D: decided at the first pass of an iteration (the union pass) for the
    // whole iteration; a tile inactive there has an empty union and cannot
    // change until the next iteration.
    return nbr_last_change(in, tile) >= q - 6;
}

}  // namespace bgt
