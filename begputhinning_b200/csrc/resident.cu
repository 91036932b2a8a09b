// resident.cu -- the resident engine: every work item (an instance, or one
// band of rows of a 2D image too large for one CTA) is loaded once into one
// CTA's shared memory and thinned there from its first subiteration to its
// fixed point; only the bands of a large image (every fourth iteration) and
// the slabs of a large volume (every iteration) meet to trade boundary rows
// through global memory.
// One CTA of 768 threads per SM holds up to 225 KB (measured against two
// CTAs of 384 threads with 111 KB each: larger bands and slabs won).
//
// 2D band (dense).  Rows of the band (core plus `halo` rows on each side,
// clamped to the image) lie twice in shared memory (subiteration t reads one
// copy and writes the other) with an odd pitch of 2*ceil(wl/2)+3 words
// (wl = ceil(W/32); a zero word left of every row and zero words right of
// it).  A subiteration hands units (a strip of 32 rows x a chunk of words,
// chunks sized so that there are about two units per warp) to warps
// dynamically; lane = row, walking the chunk in pairs of words: each lane
// loads its own row and the rows above and below straight from shared
// memory and forms the x-neighbours by funnel shifts.  A unit whose 3x3
// neighbourhood of units did not change during the last four subiterations
// -- one of each direction -- is a fixed point for the next one and is
// skipped (a unit processed without a change wrote identical data to both
// copies, so a skipped unit is current in both).  A
// single band stops after four consecutive subiterations without a deletion
// (a fixed point of N, S, E and W: the reference's result, whatever the
// alignment).  Bands of one image run their iterations (N, S, E, W) in
// lockstep, meeting after every kResPassesPerExchange-th one: then a band
// writes its first and last `halo` core rows to global memory, meets the
// other bands at a per-image counter, stops if no band's core changed in
// that iteration, and otherwise reads its halo rows from its neighbours.
// With halo = 4 rows per iteration of the period, wrong values entering at a
// band's outer edge between two meetings (4 rows per iteration at most)
// reach at most its halo rows; if an iteration before the meeting was
// already a fixed point, the one at the meeting is too.
//
// 3D volume (sparse bricks, one CTA).  Deletion never adds foreground, so
// bricks of 32 voxels (one word) x 32 rows x 4 planes that are empty at the
// start stay empty.  Only the non-empty ones are stored: a brick table maps
// each brick to a slot (0: the all-zero brick), and three slot buffers hold
// the state (ping-pong) and the iteration's pre-test union.  A warp
// processes a brick, lane = row, marching through its four planes with a
// three-plane window of 3x3 (row, word) neighbourhoods loaded from the
// neighbouring bricks' slots.  Brick activity follows the iteration: a brick
// whose 3x3x3 brick neighbourhood did not change during the previous
// iteration has an empty union and cannot change (the argument of the tile
// engine), so only active bricks are processed.  A volume whose non-empty
// bricks do not fit is flagged `spill` and left to the tile engine.
//
// Rules, order of directions and termination are those of the tile engine
// (2D/CUDA_ThinningKernelMultiBlock2D.cuh:104-135,
// 3D/CUDA_ThinningKernel3D_Linear.cuh:746-782); every wait is bounded.
#include <algorithm>

#include "kernels.cuh"
#include "rules.cuh"
#include "tiles.cuh"

namespace bgt {

namespace {
constexpr int kWarps = kResThreads / 32;
constexpr int kSmemBytes = kResSmemBytes;  // dynamic shared memory per CTA
constexpr int kSlotWords = 129;      // 4 planes x 32 rows, plus one word so slots fall on different banks
constexpr int kMaxBricks = 16384;    // brick table entries of a resident volume
constexpr int kBZ = 4;               // planes per brick

__host__ __device__ inline size_t up16(size_t v) { return (v + 15) & ~size_t(15); }
}  // namespace

// ------------------------------------------------------------ geometry ----
#ifndef BGT_RES_LANE_ROWS
#define BGT_RES_LANE_ROWS 1
#endif
constexpr int kLaneRows = BGT_RES_LANE_ROWS;  // rows of a 2D unit per lane (1 or 2)
constexpr int kUnitRowsH = 32 * kLaneRows - 8, kUnitWordsH = 8;  // 2D unit (see the 2D section)

// words of shared memory a 2D band of nrows rows needs: zero row, two row
// copies and the activity record of its units
__host__ __device__ inline size_t res_words2d(int W, int nrows)
{
    const int wl = (W + 31) >> 5;
    const int nch = (wl + kUnitWordsH - 1) / kUnitWordsH;
    const int pp = (nch * kUnitWordsH + 2) | 1;
    const int ns = (nrows + kUnitRowsH - 1) / kUnitRowsH;
    return (size_t)pp * (1 + 2 * (size_t)nrows) + (size_t)ns * nch;
}

// bytes of shared memory a volume with nb bricks of which ns are non-empty needs
__host__ __device__ inline size_t res_bytes3d(int nb, int ns)
{
    return up16((size_t)nb * 2) + up16((size_t)(ns + 1) * 4) + up16((size_t)(ns + 1) * 4) +
           up16((size_t)(ns + 1) * 2) + (size_t)3 * (ns + 1) * kSlotWords * 4;
}

int res_smem_bytes() { return kSmemBytes; }

int res_rows_fit2d(int W)
{
    int lo = 0, hi = 32767;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (res_words2d(W, mid) * 4 <= (size_t)kSmemBytes) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

int res_slots_fit3d(int W, int H, int D)
{
    const long long nb = (long long)((W + 31) / 32) * ((H + 31) / 32) * ((D + kBZ - 1) / kBZ);
    if (nb > kMaxBricks) return 0;
    int ns = 0;
    while (res_bytes3d((int)nb, ns + 1) <= (size_t)kSmemBytes) ns++;
    return ns;
}

bool res_fits3d(int W, int H, int D)
{
    const long long nb = (long long)((W + 31) / 32) * ((H + 31) / 32) * ((D + kBZ - 1) / kBZ);
    return nb <= kMaxBricks && res_bytes3d((int)nb, 1) <= (size_t)kSmemBytes;
}

// ------------------------------------------------------------ helpers -----
__device__ __forceinline__ bool res_wait_at_least(const int *p, int target, long long timeout_ns)
{
    const unsigned long long t_end = globaltimer() + (unsigned long long)timeout_ns;
    for (int spin = 0;; spin++) {
        if (ld_acquire(p) >= target) return true;
        if ((spin & 63) == 63 && globaltimer() > t_end) return false;
        __nanosleep(spin < 16 ? 32 : 128);
    }
}

// Next work unit of a subiteration for this warp (dynamic distribution over
// the CTA's warps): lane 0 takes a ticket of counter `c`.
__device__ __forceinline__ int res_take(int *c)
{
    int k = 0;
    if ((threadIdx.x & 31) == 0) k = atomicAdd(c, 1);
    return __shfl_sync(kFull, k, 0);
}

// Exclusive prefix sum over the CTA of one int per thread; *total gets the sum.
__device__ int res_block_exscan(int v, int *total)
{
    __shared__ int warp_sum[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    int before = 0, all = 0;
    for (int w = 0; w < kWarps; w++) {
        const int s = warp_sum[w];
        if (w < warp) before += s;
        all += s;
    }
    __syncthreads();
    *total = all;
    return before + x - v;
}

// ------------------------------------------------------------ 2D ----------
// A pass is one iteration (N, S, E, W) run on register tiles: a warp loads a
// unit -- 24 core rows plus 4 halo rows above and below (lane = row) by 8
// core words plus one halo word on either side -- from the pass-start copy,
// runs the four subiterations in registers (rows above and below by
// shuffles, x-neighbours by funnel shifts) and writes its core to the other
// copy.  Wrong values entering at a unit's edge move one row (or bit) per
// subiteration, so after four they reach only its halo.
// BGT_RES_LANE_ROWS=2 builds units of 56 core rows, two adjacent rows per
// lane (each other's vertical neighbours, half the shuffles per row, less
// halo): measured slower on stroke images (1.13 against 1.06 ms for 512
// images), as the larger units stay active for longer.
constexpr int kUnitRows = 32 * kLaneRows - 2 * 4;  // core rows of a unit (K = 4)
constexpr int kUnitWords = 8;                      // core words of a unit
constexpr int kHaloLanes = 4 / kLaneRows;          // lanes holding the top (or bottom) halo rows

// The rule on word j of a lane's two rows a (upper) and b (lower): o the
// words, n/p the words after/before them (pass-start values).
template <int DIR>
__device__ __forceinline__ void word2d_pair(uint32_t oa, uint32_t na, uint32_t pa, uint32_t ob, uint32_t nb,
                                            uint32_t pb, uint32_t &ra, uint32_t &rb)
{
    const uint32_t xpa = at_xp1(oa, na), xma = at_xm1(oa, pa);
    const uint32_t xpb = at_xp1(ob, nb), xmb = at_xm1(ob, pb);
    uint32_t A[8], B[8];
    A[0] = __shfl_up_sync(kFull, ob, 1);   // row above a: the lower row of the lane above
    A[1] = __shfl_up_sync(kFull, xpb, 1);
    A[7] = __shfl_up_sync(kFull, xmb, 1);
    A[2] = xpa;
    A[6] = xma;
    A[4] = ob;
    A[3] = xpb;
    A[5] = xmb;
    B[4] = __shfl_down_sync(kFull, oa, 1);  // row below b: the upper row of the lane below
    B[3] = __shfl_down_sync(kFull, xpa, 1);
    B[5] = __shfl_down_sync(kFull, xma, 1);
    B[2] = xpb;
    B[6] = xmb;
    B[0] = oa;
    B[1] = xpa;
    B[7] = xma;
    ra = keep2d<DIR>(oa, A);
    rb = keep2d<DIR>(ob, B);
}

// One subiteration on the lane's two rows of S+2 words (words j0..j1-1 are
// processed; the rest keep their values).  Words that are empty in both
// rows of every lane are skipped.
template <int S, int DIR, int J0, int J1>
__device__ __forceinline__ void subit2d_pair(uint32_t (&a)[S + 2], uint32_t (&b)[S + 2])
{
    uint32_t pa = J0 > 0 ? a[J0 - 1] : 0u, pb = J0 > 0 ? b[J0 - 1] : 0u;
#pragma unroll
    for (int j = J0; j < J1; j++) {
        const uint32_t oa = a[j], ob = b[j];
        const uint32_t na = j + 1 < S + 2 ? a[j + 1] : 0u, nb = j + 1 < S + 2 ? b[j + 1] : 0u;
        if (__any_sync(kFull, (oa | ob) != 0u)) word2d_pair<DIR>(oa, na, pa, ob, nb, pb, a[j], b[j]);
        pa = oa;
        pb = ob;
    }
}

// K subiterations from phase PH; the last one only on the core words.
template <int K, int S, int PH, int I = 0>
__device__ __forceinline__ void run_subits2d_pair(uint32_t (&a)[S + 2], uint32_t (&b)[S + 2])
{
    if constexpr (I + 1 < K) {
        subit2d_pair<S, (PH + I) & 3, 0, S + 2>(a, b);
        run_subits2d_pair<K, S, PH, I + 1>(a, b);
    } else if constexpr (I + 1 == K) {
        subit2d_pair<S, (PH + I) & 3, 1, S + 1>(a, b);
    }
}

__host__ __device__ inline int res_pitch2d_tiles(int W)
{
    const int wl = (W + 31) >> 5;
    const int nch = (wl + kUnitWords - 1) / kUnitWords;
    return (nch * kUnitWords + 2) | 1;  // zero word left, zero words right, odd
}

struct Band2D {
    uint32_t *zero;     // pp zero words
    uint32_t *buf0, *buf1;  // nrows x pp each: pass q reads buf[q & 1], writes buf[(q + 1) & 1]
    int *until;         // [nstrips][nchunks]: the unit is processed while q <= until (a unit in
                        // its 3x3 neighbourhood deleted something in the previous pass)
    int pp, wl, nrows, nstrips, nchunks;
    int a;              // image row of the band's first row in shared memory
    int r0, r1;         // core rows (image coordinates)
};

// One pass q over the band's units.  A unit none of whose inputs for the
// pass -- its core and the 4-pixel border bands of its 3x3 neighbours -- had
// a deletion in the previous pass (one subiteration of every direction) is
// skipped: that region is a fixed point, and a unit processed without a
// change wrote identical data to both copies.  A unit that deletes something
// extends `until` to q + 1 for itself and for each neighbour whose border
// band the deletions reach (a reader in the same pass may see the new value:
// it then processes a unit it could have skipped).
// Returns this thread's deleted core bits (band core rows only).
__device__ uint32_t res_pass2d(const Band2D &b, int q, int *take, unsigned long long *words)
{
    const int lane = threadIdx.x & 31;
    const uint32_t *IN = (q & 1) ? b.buf1 : b.buf0;
    uint32_t *OUT = (q & 1) ? b.buf0 : b.buf1;
    const int nunits = b.nstrips * b.nchunks;
    uint32_t core = 0;
    for (;;) {
        const int u = res_take(take);
        if (u >= nunits) break;
        if (b.until[u] < q) continue;
        const int s = u / b.nchunks, c = u - s * b.nchunks;
        const int x0 = 1 + kUnitWords * c;
        const int rbase = kUnitRows * s - 4 + kLaneRows * lane;  // band row of the lane's first row
        uint32_t v[kLaneRows][kUnitWords + 2];
        const uint32_t *in[kLaneRows];
        bool valid[kLaneRows];
#pragma unroll
        for (int i = 0; i < kLaneRows; i++) {
            const int r = rbase + i;
            valid[i] = r >= 0 && r < b.nrows;
            in[i] = valid[i] ? IN + (size_t)r * b.pp : b.zero;
#pragma unroll
            for (int k = 0; k < kUnitWords + 2; k++) v[i][k] = in[i][x0 - 1 + k];
        }
        if constexpr (kLaneRows == 2) run_subits2d_pair<4, kUnitWords, 0>(v[0], v[1]);
        else run_subits2d<4, kUnitWords, 0>(v[0]);
        const bool core_lane = lane >= kHaloLanes && lane < 32 - kHaloLanes;
        uint32_t chg = 0, lft = 0, rgt = 0;
#pragma unroll
        for (int i = 0; i < kLaneRows; i++) {
            if (!(valid[i] && core_lane)) continue;
            uint32_t *out = OUT + (size_t)(rbase + i) * b.pp;
            uint32_t ci = 0;
#pragma unroll
            for (int k = 0; k < kUnitWords; k++) {
                const uint32_t d = v[i][1 + k] ^ in[i][x0 + k];
                ci |= d;
                if (k == 0) lft |= d & 0xFu;                     // within 4 pixels of the left edge
                if (k == kUnitWords - 1) rgt |= d & 0xF0000000u;  // ... of the right edge
                out[x0 + k] = v[i][1 + k];
            }
            chg |= ci;
            const int gy = b.a + rbase + i;
            if (gy >= b.r0 && gy < b.r1) core |= ci;
        }
        // The next pass of a neighbour depends on this unit only through the
        // 4 pixels next to their common border (four subiterations reach 4
        // pixels): activate the neighbours whose border band changed
        // (border bands, as the tile engine does).
        const unsigned m_any = __ballot_sync(kFull, chg != 0u);
        if (m_any) {
            const unsigned m_l = __ballot_sync(kFull, lft != 0u), m_r = __ballot_sync(kFull, rgt != 0u);
            // lanes holding the first and last 4 core rows
            constexpr unsigned band_top = ((1u << kHaloLanes) - 1u) << kHaloLanes;
            constexpr unsigned band_bot = ((1u << kHaloLanes) - 1u) << (32 - 2 * kHaloLanes);
            if (lane < 9) {
                const int dy = lane / 3 - 1, dx = lane % 3 - 1;
                const unsigned rows = dy < 0 ? band_top : dy > 0 ? band_bot : ~0u;
                const unsigned cols = dx < 0 ? m_l : dx > 0 ? m_r : m_any;
                const int ns = s + dy, nc = c + dx;
                if ((rows & cols & m_any) && ns >= 0 && ns < b.nstrips && nc >= 0 && nc < b.nchunks)
                    b.until[ns * b.nchunks + nc] = q + 1;
            }
        }
        if (lane == 0)
            *words += (unsigned long long)min(kUnitRows, b.nrows - kUnitRows * s) *
                      min(kUnitWords, b.wl - kUnitWords * c);
    }
    return core;
}

__device__ void res_run2d(Inst &in, const ResItem &it, uint32_t *sm, ResSched *S, int *take)
{
    __shared__ int s_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Band2D b;
    b.wl = (in.W + 31) >> 5;
    b.pp = res_pitch2d_tiles(in.W);
    b.nchunks = (b.wl + kUnitWords - 1) / kUnitWords;
    b.r0 = it.r0;
    b.r1 = it.r1;
    b.a = max(0, it.r0 - it.halo);
    const int bend = min(in.H, it.r1 + it.halo);
    b.nrows = bend - b.a;
    b.nstrips = (b.nrows + kUnitRows - 1) / kUnitRows;
    b.zero = sm;
    b.buf0 = sm + b.pp;
    b.buf1 = b.buf0 + (size_t)b.nrows * b.pp;
    b.until = reinterpret_cast<int *>(b.buf1 + (size_t)b.nrows * b.pp);
    const int pp = b.pp;
    const int nunits = b.nstrips * b.nchunks;

    for (int i = threadIdx.x; i < pp; i += kResThreads) b.zero[i] = 0u;
    for (int i = threadIdx.x; i < nunits; i += kResThreads) b.until[i] = -1;
    if (threadIdx.x < 2) take[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t *g0 = in.buf[0];
    for (int r = warp; r < b.nrows; r += kWarps) {
        const uint32_t *grow = g0 + (size_t)(b.a + r) * in.P;
        uint32_t *r0p = b.buf0 + (size_t)r * pp, *r1p = b.buf1 + (size_t)r * pp;
        for (int w = lane; w < pp; w += 32) {
            const uint32_t v = (w >= 1 && w <= b.wl) ? __ldcg(grow + (w - 1)) : 0u;
            r0p[w] = v;
            r1p[w] = v;
            // units holding foreground start active
            if (v) b.until[(r / kUnitRows) * b.nchunks + (w - 1) / kUnitWords] = 0;
        }
    }
    __syncthreads();

    int result = 0;  // 1 converged, -1 pass cap or failed wait
    unsigned long long words = 0;
    int q = 0;
    for (;; q++) {
        // the counter of this pass was cleared during the previous one;
        // clear the next one's (nobody uses it before the barrier below)
        if (threadIdx.x == 0) take[(q + 1) & 1] = 0;
        const uint32_t core = res_pass2d(b, q, take + (q & 1), &words);
        const bool any = __syncthreads_or(core != 0u);
        if (it.bands == 1) {
            if (!any) {
                result = 1;
                break;
            }
        } else if (q % kResPassesPerExchange == kResPassesPerExchange - 1) {
            // end of pass q (state in buf[(q+1)&1]), the last of an exchange
            // period: trade boundary rows with the neighbouring bands
            const int h = it.halo;
            const int e = q / kResPassesPerExchange;  // exchange index
            uint32_t *cur = (q & 1) ? b.buf0 : b.buf1;
            uint32_t *gx = in.buf[(e + 1) & 1];  // buf[0] holds the start state other bands may still load
            for (int k = warp; k < 2 * h; k += kWarps) {
                const bool top = k < h;
                if (top ? it.band == 0 : it.band + 1 == it.bands) continue;
                const int gy = top ? b.r0 + k : b.r1 - 2 * h + k;
                const uint32_t *srow = cur + (size_t)(gy - b.a) * pp;
                uint32_t *grow = gx + (size_t)gy * in.P;
                for (int w = lane; w < b.wl; w += 32) grow[w] = srow[w + 1];
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                if (any) atomicMax(&in.res_last, q);
                atomicAdd(&in.res_arrive, 1);
                int f;
                if (!res_wait_at_least(&in.res_arrive, it.bands * (e + 1), S->timeout_ns)) {
                    atomicOr(&S->status, kErrQueueTimeout);
                    f = 2;
                } else {
                    f = ld_acquire(&in.res_last) < q ? 1 : 0;
                }
                s_flag = f;
            }
            __syncthreads();
            const int f = s_flag;
            if (f == 1) {
                result = 1;
                break;
            }
            if (f == 2) {
                result = -1;
                break;
            }
            // halo rows: the neighbours' boundary core rows after pass q
            const int ntop = b.r0 - b.a, nh = ntop + (bend - b.r1);
            uint32_t hc = 0;
            for (int k = warp; k < nh; k += kWarps) {
                const int r = k < ntop ? k : (b.r1 - b.a) + (k - ntop);
                const uint32_t *grow = gx + (size_t)(b.a + r) * in.P;
                uint32_t *srow = cur + (size_t)r * pp;
                for (int w = lane; w < b.wl; w += 32) {
                    const uint32_t v = __ldcg(grow + w);
                    hc |= v ^ srow[w + 1];
                    srow[w + 1] = v;
                }
            }
            if (__syncthreads_or(hc != 0u)) {
                // units within reach of the halo rows go on next pass
                for (int u = threadIdx.x; u < nunits; u += kResThreads) {
                    const int st = u / b.nchunks;
                    const int ga = b.a + kUnitRows * st - kUnitRows, gb = b.a + kUnitRows * st + 2 * kUnitRows;
                    if (ga < b.r0 || gb > b.r1) b.until[u] = q + 1;
                }
                __syncthreads();
            }
        }
        if (q >= in.pass_cap) {
            if (threadIdx.x == 0) atomicOr(&S->status, kErrPassLimit);
            result = -1;
            break;
        }
    }
    // the converged core rows (in buf[(q+1)&1]) -> buf[0]
    __syncthreads();
    const uint32_t *fin = (q & 1) ? b.buf0 : b.buf1;
    uint32_t *g0w = in.buf[0];
    for (int r = b.r0 - b.a + warp; r < b.r1 - b.a; r += kWarps) {
        const uint32_t *srow = fin + (size_t)r * pp;
        uint32_t *grow = g0w + (size_t)(b.a + r) * in.P;
        for (int w = lane; w < b.wl; w += 32) grow[w] = srow[w + 1];
    }
    if (lane == 0 && words) atomicAdd(&in.work_words, words);  // core words per pass (one iteration)
    if (threadIdx.x == 0) {
        if (it.band == 0) in.passes_run = q + 1;
        if (result < 0) atomicMin(&in.converged, -1);
        atomicAdd(&in.tiles_run, 1ull);
    }
    __syncthreads();
}

// ------------------------------------------------------------ 3D ----------
struct Vol3D {
    uint16_t *tab;     // [nbz][nby][nbx] -> slot (0: empty)
    int *coord;        // slot -> linear brick index
    uint8_t *act;      // slot: active in this iteration
    uint8_t *chg;      // slot: changed in this iteration
    uint8_t *nxt;      // slot: active in the next iteration
    uint8_t *ufl;      // slot: its pre-test union of this iteration is not empty
    uint16_t *list;    // active slots of this iteration
    uint32_t *X, *Y, *U;  // slot buffers (slot 0 = the zero brick)
    int nbx, nby, nbz, nslots;
};

// The nine row/word neighbourhood words of one plane (offset `off` within
// the slots) from the slot bases of the rows above (u), this row (o) and
// below (d), each for the words x-1, x, x+1.
__device__ __forceinline__ void res_plane9(const uint32_t *__restrict__ IN, const int (&u)[3], const int (&o)[3],
                                           const int (&d)[3], int off, uint32_t (&P)[9])
{
    const uint32_t ul = IN[u[0] + off], uc = IN[u[1] + off], ur = IN[u[2] + off];
    const uint32_t ol = IN[o[0] + off], oc = IN[o[1] + off], orr = IN[o[2] + off];
    const uint32_t dl = IN[d[0] + off], dc = IN[d[1] + off], dr = IN[d[2] + off];
    P[0] = at_xm1(uc, ul); P[1] = uc; P[2] = at_xp1(uc, ur);
    P[3] = at_xm1(oc, ol); P[4] = oc; P[5] = at_xp1(oc, orr);
    P[6] = at_xm1(dc, dl); P[7] = dc; P[8] = at_xp1(dc, dr);
}

// Slot bases (word index of this lane's row) of the three x-neighbour bricks
// in the z-layer dzb (-1, 0, +1) for the rows above, at and below this lane's
// row; nb27 holds, in lane k < 27, the slot of brick offset
// (k/9 - 1, (k/3)%3 - 1, k%3 - 1) in (z, y, x).
__device__ __forceinline__ void res_bases3d(int nb27, int dzb, int (&u)[3], int (&o)[3], int (&d)[3])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const int so = __shfl_sync(kFull, nb27, 9 * (dzb + 1) + 3 + c);
        const int su = __shfl_sync(kFull, nb27, 9 * (dzb + 1) + c);
        const int sd = __shfl_sync(kFull, nb27, 9 * (dzb + 1) + 6 + c);
        o[c] = so * kSlotWords + lane;
        u[c] = lane == 0 ? su * kSlotWords + 31 : so * kSlotWords + lane - 1;
        d[c] = lane == 31 ? sd * kSlotWords : so * kSlotWords + lane + 1;
    }
}

// Subiteration J (0: pre-test union + U; 1..5: N, E, D, S, W) on brick slot s.
// J = 0 also ORs the brick's union bits into *uany.
template <int J>
__device__ uint32_t res_brick3d(const Vol3D &v, int s, const uint32_t *__restrict__ IN, uint32_t *__restrict__ OUT,
                                uint32_t *__restrict__ U, uint32_t *uany)
{
    const int lane = threadIdx.x & 31;
    const int li = v.coord[s];
    const int bx = li % v.nbx, by = (li / v.nbx) % v.nby, bz = li / (v.nbx * v.nby);
    int nb27 = 0;
    if (lane < 27) {
        const int zz = bz + lane / 9 - 1, yy = by + (lane / 3) % 3 - 1, xx = bx + lane % 3 - 1;
        if (zz >= 0 && zz < v.nbz && yy >= 0 && yy < v.nby && xx >= 0 && xx < v.nbx)
            nb27 = v.tab[(zz * v.nby + yy) * v.nbx + xx];
    }
    int u[3], o[3], d[3];
    uint32_t A[9], B[9], Cn[9];
    res_bases3d(nb27, -1, u, o, d);
    res_plane9(IN, u, o, d, 3 * 32, A);  // plane 4bz - 1: last plane of the brick below
    res_bases3d(nb27, 0, u, o, d);
    res_plane9(IN, u, o, d, 0, B);
    const int self = s * kSlotWords + lane;
    uint32_t chg = 0;
#pragma unroll 1
    for (int q = 0; q < kBZ; q++) {
        if (q == kBZ - 1) res_bases3d(nb27, 1, u, o, d);
        res_plane9(IN, u, o, d, ((q + 1) & 3) * 32, Cn);
        const uint32_t val = B[4];
        uint32_t nv = val;
        const int widx = self + q * 32;
        if constexpr (J == 0) {
            uint32_t un = 0;
            if (__any_sync(kFull, val != 0u)) {
                uint32_t g[27];
#pragma unroll
                for (int i = 0; i < 9; i++) {
                    g[i] = A[i];
                    g[9 + i] = B[i];
                    g[18 + i] = Cn[i];
                }
                const uint32_t du = rule3d<0>(g);
                un = (du | rule3d<1>(g) | rule3d<2>(g) | rule3d<3>(g) | rule3d<4>(g) | rule3d<5>(g)) & val;
                nv = val & ~du;
            }
            U[widx] = un;
            *uany |= un;
        } else {
            const uint32_t cand = val & U[widx];
            if (__any_sync(kFull, cand != 0u)) {
                uint32_t g[27];
#pragma unroll
                for (int i = 0; i < 9; i++) {
                    g[i] = A[i];
                    g[9 + i] = B[i];
                    g[18 + i] = Cn[i];
                }
                nv = val & ~(cand & rule3d<J>(g));
            }
        }
        OUT[widx] = nv;
        chg |= val ^ nv;
#pragma unroll
        for (int i = 0; i < 9; i++) {
            A[i] = B[i];
            B[i] = Cn[i];
        }
    }
    return chg;
}

// One volume, or one z-slab of a large volume: brick layers [r0, r1) are
// the slab's core, `halo` layers on each side (clamped to the volume) are
// held too and recomputed.  Slabs run whole iterations (pre-test, U, N, E, D,
// S, W) in lockstep and trade their boundary layers through global memory
// after each: errors entering at a slab's outer edge move one plane per
// subiteration (the pre-test's union reads one plane further, inside the
// same bound), six planes in an iteration, so a halo of two layers (eight
// planes) keeps the core exact.  Halo bricks and the core bricks next to
// them are processed in every iteration.
__device__ void res_run3d(Inst &in, const ResItem &it, uint8_t *smb, ResSched *S, int *take)
{
    __shared__ int s_cnt, s_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Vol3D v;
    const int wl = (in.W + 31) >> 5;
    const int nbz_all = (in.D + kBZ - 1) / kBZ;
    const bool banded = it.bands > 1;
    const int c_lo = banded ? it.r0 : 0, c_hi = banded ? it.r1 : nbz_all;
    const int e_lo = max(0, c_lo - it.halo), e_hi = min(nbz_all, c_hi + it.halo);
    v.nbx = wl;
    v.nby = (in.H + 31) >> 5;
    v.nbz = e_hi - e_lo;
    const int bz0 = e_lo;
    const int nb = v.nbx * v.nby * v.nbz;
    v.tab = reinterpret_cast<uint16_t *>(smb);
    for (int i = threadIdx.x; i < nb; i += kResThreads) v.tab[i] = 0;
    __syncthreads();
    // mark the non-empty bricks: one coalesced pass over the used words of
    // the held planes (word i of the pass = word i % wl of row i / wl)
    const uint32_t *g0 = in.buf[0];
    const int z_first = kBZ * e_lo, z_end = min(in.D, kBZ * e_hi);
    {
        const int nw = (z_end - z_first) * in.H * wl;
        const size_t base = (size_t)z_first * in.H;
        for (int i = threadIdx.x; i < nw; i += kResThreads) {
            const int r = i / wl, x = i - r * wl;
            if (__ldcg(g0 + (base + r) * in.P + x) != 0u) {
                const int zl = r / in.H, y = r - zl * in.H;
                v.tab[((zl / kBZ) * v.nby + (y >> 5)) * v.nbx + x] = 1;
            }
        }
    }
    __syncthreads();
    // slots in raster order of the bricks
    const int per = (nb + kResThreads - 1) / kResThreads;
    const int i0 = min(nb, threadIdx.x * per), i1 = min(nb, i0 + per);
    int cnt = 0;
    for (int i = i0; i < i1; i++) cnt += v.tab[i] != 0;
    int total = 0;
    const int first = res_block_exscan(cnt, &total);
    v.nslots = total;
    const bool fits = res_bytes3d(nb, total) <= (size_t)kSmemBytes;
    if (banded) {
        // every slab must fit, or the tile engine takes the whole volume:
        // the slabs agree before any of them writes anything
        if (threadIdx.x == 0) {
            if (!fits) atomicExch(&in.spill, 1);
            __threadfence();
            atomicAdd(&in.res_arrive, 1);
            int f;
            if (!res_wait_at_least(&in.res_arrive, it.bands, S->timeout_ns)) {
                atomicOr(&S->status, kErrQueueTimeout);
                f = 2;
            } else {
                f = ld_acquire(&in.spill) ? 1 : 0;
            }
            s_flag = f;
        }
        __syncthreads();
        if (s_flag) {
            if (s_flag == 2 && threadIdx.x == 0) atomicMin(&in.converged, -1);
            __syncthreads();
            return;
        }
    } else if (!fits) {
        // does not fit: the tile engine thins this volume (nothing here was written to it)
        if (threadIdx.x == 0) in.spill = 1;
        __syncthreads();
        return;
    }
    size_t off = up16((size_t)nb * 2);
    v.coord = reinterpret_cast<int *>(smb + off);
    off += up16((size_t)(total + 1) * 4);
    v.act = smb + off;
    v.chg = v.act + (total + 1);
    v.nxt = v.chg + (total + 1);
    v.ufl = v.nxt + (total + 1);
    off += up16((size_t)(total + 1) * 4);
    v.list = reinterpret_cast<uint16_t *>(smb + off);
    off += up16((size_t)(total + 1) * 2);
    v.X = reinterpret_cast<uint32_t *>(smb + off);
    v.Y = v.X + (size_t)(total + 1) * kSlotWords;
    v.U = v.Y + (size_t)(total + 1) * kSlotWords;
    {
        int sl = first + 1;
        for (int i = i0; i < i1; i++)
            if (v.tab[i]) {
                v.tab[i] = (uint16_t)sl;
                v.coord[sl] = i;
                sl++;
            }
    }
    for (int i = threadIdx.x; i < kSlotWords; i += kResThreads) {
        v.X[i] = 0u;
        v.Y[i] = 0u;
        v.U[i] = 0u;
    }
    for (int i = threadIdx.x; i <= total; i += kResThreads) {
        v.act[i] = i > 0;
        v.chg[i] = 0;
        v.nxt[i] = 0;
        v.ufl[i] = 0;
    }
    if (threadIdx.x < 2) take[threadIdx.x] = 0;
    __syncthreads();
    // brick layer (global) of a slot
    auto layer_of = [&](int s) { return bz0 + v.coord[s] / (v.nbx * v.nby); };
    // copy the slot's words from / to packed volume g (rows inside the volume only)
    auto gather = [&](const uint32_t *g, int s, bool both) {
        const int li = v.coord[s];
        const int bx = li % v.nbx, by = (li / v.nbx) % v.nby, bz = bz0 + li / (v.nbx * v.nby);
        const int y = 32 * by + lane;
#pragma unroll
        for (int q = 0; q < kBZ; q++) {
            const int z = kBZ * bz + q;
            const uint32_t w = (y < in.H && z < in.D) ? __ldcg(g + ((size_t)z * in.H + y) * in.P + bx) : 0u;
            v.X[s * kSlotWords + q * 32 + lane] = w;
            if (both) v.Y[s * kSlotWords + q * 32 + lane] = w;
        }
    };
    auto scatter = [&](uint32_t *g, int s) {
        const int li = v.coord[s];
        const int bx = li % v.nbx, by = (li / v.nbx) % v.nby, bz = bz0 + li / (v.nbx * v.nby);
        const int y = 32 * by + lane;
        if (y >= in.H) return;
#pragma unroll
        for (int q = 0; q < kBZ; q++) {
            const int z = kBZ * bz + q;
            if (z < in.D) g[((size_t)z * in.H + y) * in.P + bx] = v.X[s * kSlotWords + q * 32 + lane];
        }
    };
    // gather the non-empty bricks (both state buffers)
    for (int s = warp + 1; s <= total; s += kWarps) gather(g0, s, true);
    __syncthreads();
    // layers processed in every iteration of a slab: its halo and the core layers next to it
    const int keep_lo = it.band > 0 ? c_lo + it.halo : 0;
    const int keep_hi = it.band + 1 < it.bands ? c_hi - it.halo : nbz_all;

    int iter = 0, result = 0;
    unsigned long long words = 0, bricks = 0;
    const int cap_it = in.pass_cap / 6 + 1;
    for (;; iter++) {
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        for (int s = threadIdx.x + 1; s <= total; s += kResThreads)
            if (v.act[s]) v.list[atomicAdd(&s_cnt, 1)] = (uint16_t)s;
        __syncthreads();
        int nact = s_cnt;
        for (int j = 0; j < 6; j++) {
            if (j == 1) {
                // a brick whose union is empty cannot change in the rest of
                // the iteration (every deletion is of a union voxel), and both
                // of its buffers already hold its state: only the others go on
                if (threadIdx.x == 0) s_cnt = 0;
                __syncthreads();
                for (int s = threadIdx.x + 1; s <= total; s += kResThreads)
                    if (v.act[s] && v.ufl[s]) v.list[atomicAdd(&s_cnt, 1)] = (uint16_t)s;
                __syncthreads();
                nact = s_cnt;
            }
            if (threadIdx.x == 0) take[(j + 1) & 1] = 0;
            const uint32_t *IN = (j & 1) ? v.Y : v.X;
            uint32_t *OUT = (j & 1) ? v.X : v.Y;
            for (;;) {
                const int k = res_take(take + (j & 1));
                if (k >= nact) break;
                const int s = v.list[k];
                uint32_t c, uany = 0;
                switch (j) {
                case 0: c = res_brick3d<0>(v, s, IN, OUT, v.U, &uany); break;
                case 1: c = res_brick3d<1>(v, s, IN, OUT, v.U, &uany); break;
                case 2: c = res_brick3d<2>(v, s, IN, OUT, v.U, &uany); break;
                case 3: c = res_brick3d<3>(v, s, IN, OUT, v.U, &uany); break;
                case 4: c = res_brick3d<4>(v, s, IN, OUT, v.U, &uany); break;
                default: c = res_brick3d<5>(v, s, IN, OUT, v.U, &uany); break;
                }
                if (j == 0) {
                    const bool u = __any_sync(kFull, uany != 0u);
                    if (lane == 0) v.ufl[s] = u;
                }
                if (lane == 0) {
                    const int li = v.coord[s];
                    const int by = (li / v.nbx) % v.nby, bz = bz0 + li / (v.nbx * v.nby);
                    if (bz >= c_lo && bz < c_hi) {
                        words += (unsigned long long)min(32, in.H - 32 * by) * min(kBZ, in.D - kBZ * bz);
                        bricks++;
                    }
                }
                if (__any_sync(kFull, c != 0u) && lane == 0) v.chg[s] = 1;
            }
            __syncthreads();
        }
        // next iteration's bricks: the 3x3x3 brick neighbourhoods of the
        // changed ones; `core` = a core brick changed
        int core = 0;
        for (int s = threadIdx.x + 1; s <= total; s += kResThreads) {
            const int bzs = layer_of(s);
            if (banded && (bzs < keep_lo || bzs >= keep_hi)) v.nxt[s] = 1;
            if (!v.chg[s]) continue;
            if (bzs >= c_lo && bzs < c_hi) core = 1;
            const int li = v.coord[s];
            const int bx = li % v.nbx, by = (li / v.nbx) % v.nby, bz = li / (v.nbx * v.nby);
            for (int dz = -1; dz <= 1; dz++) {
                const int zz = bz + dz;
                if (zz < 0 || zz >= v.nbz) continue;
                for (int dy = -1; dy <= 1; dy++) {
                    const int yy = by + dy;
                    if (yy < 0 || yy >= v.nby) continue;
                    for (int dx = -1; dx <= 1; dx++) {
                        const int xx = bx + dx;
                        if (xx < 0 || xx >= v.nbx) continue;
                        const int n = v.tab[(zz * v.nby + yy) * v.nbx + xx];
                        if (n) v.nxt[n] = 1;
                    }
                }
            }
        }
        const bool any_core = __syncthreads_or(core);
        if (!banded) {
            if (!any_core) {
                result = 1;
                break;
            }
        } else {
            // trade boundary layers with the neighbouring slabs (state in X)
            uint32_t *gx = in.buf[(iter + 1) & 1];  // buf[0] holds the start state other slabs may still load
            for (int s = warp + 1; s <= total; s += kWarps) {
                const int bzs = layer_of(s);
                const bool out_lo = it.band > 0 && bzs >= c_lo && bzs < c_lo + it.halo;
                const bool out_hi = it.band + 1 < it.bands && bzs >= c_hi - it.halo && bzs < c_hi;
                if (out_lo || out_hi) scatter(gx, s);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                if (any_core) atomicMax(&in.res_last, iter);
                atomicAdd(&in.res_arrive, 1);
                int f;
                if (!res_wait_at_least(&in.res_arrive, it.bands * (iter + 2), S->timeout_ns)) {
                    atomicOr(&S->status, kErrQueueTimeout);
                    f = 2;
                } else {
                    f = ld_acquire(&in.res_last) < iter ? 1 : 0;
                }
                s_flag = f;
            }
            __syncthreads();
            const int f = s_flag;
            if (f == 1) {
                result = 1;
                break;
            }
            if (f == 2) {
                result = -1;
                break;
            }
            for (int s = warp + 1; s <= total; s += kWarps) {
                const int bzs = layer_of(s);
                if (bzs < c_lo || bzs >= c_hi) gather(gx, s, true);
            }
        }
        for (int s = threadIdx.x + 1; s <= total; s += kResThreads) {
            v.act[s] = v.nxt[s];
            v.nxt[s] = 0;
            v.chg[s] = 0;
        }
        if (iter + 1 >= cap_it) {
            if (threadIdx.x == 0) atomicOr(&S->status, kErrPassLimit);
            result = -1;
            break;
        }
    }
    __syncthreads();
    // the converged core (in X after the sixth subiteration) -> buf[0]
    uint32_t *g0w = in.buf[0];
    for (int s = warp + 1; s <= total; s += kWarps) {
        const int bzs = layer_of(s);
        if (bzs >= c_lo && bzs < c_hi) scatter(g0w, s);
    }
    if (lane == 0 && words) {
        atomicAdd(&in.work_words, words);
        atomicAdd(&in.tiles_run, bricks);
    }
    if (threadIdx.x == 0) {
        if (it.band == 0) in.passes_run = 6 * (iter + 1);
        if (result < 0) atomicMin(&in.converged, -1);
    }
    __syncthreads();
}

// ------------------------------------------------------------ kernels -----
__global__ void resident_reset_kernel(Inst *insts, int n, ResSched *S, int nitems, long long timeout_ns)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Inst &in = insts[i];
        in.res_arrive = 0;
        in.res_last = -1;
        in.spill = 0;
        if (in.res) {
            in.converged = 1;  // lowered to -1 by a band that fails
            in.passes_run = 0;
            in.tiles_run = 0;
            in.work_words = 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->head = 0;
        S->nitems = nitems;
        S->status = 0;
        S->timeout_ns = timeout_ns;
    }
}

__device__ __forceinline__ int res_smid()
{
    int v;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(v));
    return v;
}

__global__ void __launch_bounds__(kResThreads, kResCtasPerSm)
    resident_kernel(Inst *insts, const ResItem *items, ResSched *S, ResTrace *trace)
{
    extern __shared__ __align__(16) uint8_t res_smem[];
    __shared__ int s_item;
    __shared__ int s_take[2];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(&S->head, 1);
        __syncthreads();
        const int k = s_item;
        __syncthreads();
        if (k >= S->nitems) break;
        const ResItem it = items[k];
        Inst &in = insts[it.inst];
        const long long t0 = (long long)globaltimer();
        if (in.dims == 2)
            res_run2d(in, it, reinterpret_cast<uint32_t *>(res_smem), S, s_take);
        else
            res_run3d(in, it, res_smem, S, s_take);
        if (threadIdx.x == 0) trace[k] = ResTrace{t0, (long long)globaltimer(), res_smid(), 0};
    }
}

cudaError_t res_occupancy(int *per_sm)
{
    cudaError_t e = cudaFuncSetAttribute(resident_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(resident_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, resident_kernel, kResThreads, kSmemBytes);
}

cudaError_t launch_resident(int grid, Inst *d_insts, int ninst, const ResItem *d_items, int nitems,
                            ResSched *d_rs, ResTrace *d_trace, long long timeout_ns, cudaStream_t st)
{
    static bool attr_done = false;
    if (!attr_done) {
        cudaError_t e = cudaFuncSetAttribute(resident_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(resident_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    resident_reset_kernel<<<std::max(1, std::min(64, (ninst + 255) / 256)), 256, 0, st>>>(d_insts, ninst, d_rs, nitems,
                                                                                       timeout_ns);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || nitems == 0) return e;
    // cooperative: all CTAs are resident at once, which the bands of an image
    // (waiting for one another) rely on
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kResThreads);
    cfg.dynamicSmemBytes = kSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, resident_kernel, d_insts, d_items, d_rs, d_trace);
}

}  // namespace bgt
