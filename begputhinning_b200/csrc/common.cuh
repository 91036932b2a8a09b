// common.cuh -- shared device helpers for the sm_100a thinning kernels:
// bit-word neighbour shifts, TMA tile loads with mbarrier completion, bounded
// waits that report a status instead of hanging, and the instance descriptor
// every kernel reads.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "bgt_capi.h"

namespace bgt {

// ---------------------------------------------------------------------------
// Packed layout.  Foreground is packed 32 pixels/voxels per uint32 along x:
// bit b of word j of a row = pixel x = 32*j + b.  A row has P words (P a
// multiple of 4 so rows start on 16-byte boundaries); rows of a plane are
// consecutive, planes are consecutive.  Words past ceil(W/32) are zero and
// stay zero (deletion only clears bits).
// ---------------------------------------------------------------------------

// value of the x-1 neighbour for every bit of c (l = word to the left)
__device__ __forceinline__ uint32_t at_xm1(uint32_t c, uint32_t l) { return __funnelshift_l(l, c, 1); }
// value of the x+1 neighbour for every bit of c (r = word to the right)
__device__ __forceinline__ uint32_t at_xp1(uint32_t c, uint32_t r) { return __funnelshift_r(c, r, 1); }

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNever = (int)0x80808080;  // "last change" of an empty tile (byte-fillable by memset 0x80)

// Error bits written to the context's status word by kernels (never trap).
enum : int {
    kErrTmaTimeout = 1,    // an mbarrier wait for a TMA tile gave up
    kErrQueueTimeout = 2,  // a work-queue wait gave up
    kErrQueueFull = 4,     // a producer could not get a queue slot
    kErrSegOverflow = 8,   // segment output larger than its reserved region
    kErrPassLimit = 16,    // an instance hit the pass cap without converging
};

// Instance descriptor (device copy).  One per image / volume.
struct alignas(16) Inst {
    int dims;                 // 2 or 3
    int W, H, D;              // pixels / rows / planes (D = 1 in 2D)
    int P;                    // words per row
    int cfg;                  // tile configuration id
    int tiles_x, tiles_y, tiles_z, ntiles;
    int TW, TH, TZ;           // core tile extent in words / rows / planes
    int k;                    // subiterations per pass (2D); 1 in 3D
    int window;               // passes of constancy that prove a tile fixed (2D)
    uint32_t *buf[2];         // packed ping-pong buffers
    uint32_t *uni;            // 3D pre-test union (per word), null in 2D
    const CUtensorMap *tmap;  // [3] tensor maps over buf[0], buf[1], uni (3D)
    int *lc;                  // per-tile pass of the last change (kNever: empty tile)
    uint8_t *act;             // 3D: activity of the current iteration; 2D: border bands of the last change
    int *list;                // active tile ids of the wave in flight
    // engine state (device-side scheduler)
    int pass;                 // pass of the wave in flight
    int nlist;                // tiles in that wave
    int done;                 // tiles of the wave finished
    int any_change;           // any tile changed in the wave in flight
    int converged;            // 1 when the instance reached its fixed point
    int passes_run;           // passes executed
    int pass_cap;             // safety cap on passes
    int prio;                 // work ring: 0 = critical path (served first), 1 = the rest
    int gang;                 // 3D: gang arrivals so far (barrier between the gang's passes)
    unsigned long long tiles_run;   // tiles processed (skipped tiles excluded)
    unsigned long long work_words;  // packed core words processed (sum over passes and tiles)
    // resident engine (resident.cu)
    int res;                  // 1: thinned by the resident engine, 0: by the tile rings
    int spill;                // set by the resident engine when a volume's bricks do not fit: the rings take it
    int res_arrive;           // arrivals at the band barrier of a multi-CTA image (all bands, all passes)
    int res_last;             // last pass in which some band's core changed (-1: none yet)
};

// Core words of a tile (clamped to the image): the algorithmic unit of a pass.
__device__ __forceinline__ unsigned tile_core_words(const Inst &in, int tile)
{
    const int wwords = (in.W + 31) >> 5;
    const int tx = tile % in.tiles_x;
    const int ty = (tile / in.tiles_x) % in.tiles_y;
    const int tz = tile / (in.tiles_x * in.tiles_y);
    const int cw = min(in.TW, wwords - tx * in.TW);
    const int ch = min(in.TH, in.H - ty * in.TH);
    const int cz = min(in.TZ, in.D - tz * in.TZ);
    return (unsigned)(cw * ch * cz);
}

// ---------------------------------------------------------------------------
// PTX wrappers: mbarrier + TMA (no cluster multicast anywhere in this code).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after ~2^22 polls (each try_wait already suspends
// for a while) and returns false; the caller records kErrTmaTimeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 22); i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Non-blocking probe of phase completion.
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Barrier of the 128 threads (warps 0..3) that run tiles (named barrier 1,
// so a CTA may add warps of other roles that never take part); in 128-thread
// kernels it is the whole CTA.
constexpr int kTileThreads = 128;
__device__ __forceinline__ void tile_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
__device__ __forceinline__ bool tile_sync_or(bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred a, b;\n\t"
        "setp.ne.u32 a, %1, 0;\n\t"
        "bar.red.or.pred b, 1, 128, a;\n\t"
        "selp.u32 %0, 1, 0, b;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void tmap_acquire(const CUtensorMap *m)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

// Generic-proxy writes by other CTAs (published through an acquire) become
// visible to this CTA's async-proxy (TMA) reads after this fence.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// 2D tiled TMA load; x must be a multiple of 4 words (16 bytes).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *m, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(m), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 3D tiled TMA load; x must be a multiple of 4 words (16 bytes).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *m, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(m), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint32_t ld_cg(const uint32_t *p) { return __ldcg(p); }
__device__ __forceinline__ int ld_cg_int(const int *p) { return __ldcg(p); }

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// mbarrier wait bounded by the global timer: false once t_end (ns) passed.
__device__ __forceinline__ bool mbar_wait_until(uint64_t *bar, uint32_t parity, unsigned long long t_end)
{
    for (int i = 0;; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 15) == 15 && globaltimer() > t_end) return false;
    }
}

}  // namespace bgt
