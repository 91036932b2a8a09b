// kernels.cuh -- declarations shared by the kernel translation unit and the
// host-side batch/engine code.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace bgt {

// Tile configurations.  2D ids 0..7: (K, S) with NW = 4 warps, ids 8..12 the
// same with shared warp edges; 3D ids 16, 17, 19: (NWX = 4, TZ = 8, 16, 4).
// All use 128 threads so the persistent engine can run any mix of them in
// one launch.
struct CfgInfo {
    int id, dims, k, S, NW, NWX, TZ;
    int TW, TH, TZc;  // core tile extent (words, rows, planes)
    int smem;         // dynamic shared memory bytes
    int box[3];       // TMA box (words, rows, planes)
    int ubox[3];      // TMA box of the 3D union (core words, rows, core planes)
};
// Tensor maps per instance: buf[0], buf[1] and (3D) the union.
constexpr int kMapsPerInst = 3;
const CfgInfo *cfg_info(int id);  // nullptr if unknown
int max_cfg_smem();               // largest dynamic shared memory of any configuration
const int *cfg_ids_2d(int *n);
const int *cfg_ids_3d(int *n);

// Scheduler state of the persistent engine (device memory).
struct alignas(128) Ring {
    unsigned head;      // next ticket to claim
    unsigned pad0[31];  // head and tail on separate 128-byte lines
    unsigned tail;      // next ticket to reserve
    unsigned cap;       // slots
    unsigned *seq;      // [cap] slot sequence numbers
    int4 *item;         // [cap] (instance, tile, pass, tiles in the wave)
};

struct Sched {
    Ring ring[2];       // 0: critical-path instances, 1: the rest
    int live;           // instances not yet converged
    int live_prio[2];   // ... per ring (a ring with no live instance gets no more items)
    int gang_budget;    // CTAs that may still join gangs (the rest keep claiming)
    int status;         // error bits
    long long timeout_ns;
};

// Resident engine (resident.cu).  A work item is one instance, or one band
// of rows of a 2D image too large for one CTA (the bands of an image run
// together and trade `halo` boundary rows through global memory after every
// iteration).  Items are taken in order by one fetch-and-add.
struct ResItem {
    int inst;        // instance index
    int band, bands; // band index and number of bands (1: the whole instance)
    int r0, r1;      // 2D: core rows [r0, r1) of the band
    int halo;        // 2D: halo rows kept on each side of the core (0 for a single band)
};
struct ResSched {
    int head;        // next item
    int nitems;
    int status;      // error bits
    int pad;
    long long timeout_ns;
};
// Timeline of one work item of the last run (global timer, ns; SM id).
struct ResTrace {
    long long t0, t1;
    int sm, pad;
};
// 2D bands of one image meet every kResPassesPerExchange passes; wrong
// values entering at a band's edge move at most 4 rows per pass, so the
// bands keep 4 halo rows per pass of the period
#ifndef BGT_RES_PASSES_PER_EXCHANGE
#define BGT_RES_PASSES_PER_EXCHANGE 4  // measured: 1, 2, 3, 4 -> mixed batch 1.20, 1.11, 1.10, 1.09 ms
#endif
constexpr int kResPassesPerExchange = BGT_RES_PASSES_PER_EXCHANGE;
constexpr int kResHalo2D = 4 * kResPassesPerExchange;
constexpr int kResThreads = 768;
constexpr int kResCtasPerSm = 1;
constexpr int kResSmemBytes = 230400;  // dynamic shared memory of one CTA (one per SM)
// Dynamic shared memory of the resident kernel (one CTA per SM).
int res_smem_bytes();
// Rows of a W-wide 2D band (core plus halo) that one CTA holds.
int res_rows_fit2d(int W);
// Non-empty bricks a D x H x W volume (or slab) may have to fit one CTA (0: its table does not fit).
int res_slots_fit3d(int W, int H, int D);
// Whether a D x H x W volume's brick table fits (its bricks are counted on the device).
bool res_fits3d(int W, int H, int D);
cudaError_t res_occupancy(int *per_sm);  // resident CTAs per SM
cudaError_t launch_resident(int grid, Inst *d_insts, int ninst, const ResItem *d_items, int nitems,
                            ResSched *d_rs, ResTrace *d_trace, long long timeout_ns, cudaStream_t st);

// Per-instance input/output of a batch-wide pack/unpack launch.
// Unsigned 32-bit division by a divisor fixed per instance, as a multiply
// and shifts (Granlund and Montgomery, "Division by invariant integers using
// multiplication", 1994, section 4): with l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1, t = mulhi(m, n):
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), exact for every
// 32-bit n.
struct FastDiv {
    uint32_t m = 1, s1 = 0, s2 = 0, d = 1;
};
inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while (l < 32 && (1ull << l) < d) l++;
    f.m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
    f.s1 = l < 1 ? l : 1;
    f.s2 = l > 1 ? l - 1 : 0;
    return f;
}
__device__ __forceinline__ uint32_t fdiv(const FastDiv &f, uint32_t n)
{
    const uint32_t t = __umulhi(f.m, n);
    return (t + ((n - t) >> f.s1)) >> f.s2;
}

struct alignas(16) IODesc {
    const void *in;
    void *out;
    int dtype, mode;         // pixel type; binarisation 0 = 2D rule, 1 = 3D rule, 2 = nonzero
    int inW, inH, inD;       // input extents inside the instance
    int inst;                // instance index
    long long wbegin;        // first global packed-word index of the instance (pack)
    long long gbegin;        // first global unpack-word index (rows x ceil(W/32))
    // dividers of the instance: words per row P, rows H, pixels per row W,
    // used words per row ceil(W/32), and the core tile extents TW, TH, TZ
    FastDiv dP, dH, dW, dWW, dTW, dTH, dTZ;
};

// Launchers (stream-ordered, no host synchronisation).
// bytes: every input is one byte wide and tested "byte != 0" (see pack_all_kernel)
cudaError_t launch_pack_all(const Inst *d_insts, const IODesc *d_io, int n, long long total_words, bool bytes,
                            cudaStream_t st);
cudaError_t launch_unpack_all(const Inst *d_insts, const IODesc *d_io, int n, long long total_words,
                              cudaStream_t st);
// mode 0: 2D binarisation, 1: 3D binarisation, 2: nonzero.  Input extents
// inW x inH x inD (row stride inW) inside the packed W x H x D.
cudaError_t launch_pack(int dtype, int mode, const void *in, int inW, int inH, int inD, int W, int H, int D, int P,
                        uint32_t *buf0, uint32_t *buf1, cudaStream_t st);
cudaError_t launch_unpack(int dtype, const uint32_t *buf, int W, int H, int D, int P, void *out,
                          cudaStream_t st);
// per-tile nonempty marks -> lc (-1 nonempty, kNever empty); counts nonempty tiles into *count
cudaError_t launch_tile_init(const Inst *d_inst, const Inst &h_inst, int *d_count, cudaStream_t st);
cudaError_t launch_plain_pass(int cfg, Inst *d_inst, int ntiles, int q, int *d_flag, int *d_err,
                              cudaStream_t st);
// Device-side pass loop of the plain path (one per instance).
struct PlainLoop {
    int q;            // pass to run next
    int last_change;  // last pass with a change
    int flag;         // set by the pass when a tile changed
    int converged;    // 1 converged, -1 pass cap, 0 running
};
cudaError_t launch_plain_dev_pass(int cfg, Inst *d_inst, int ntiles, PlainLoop *d_loop, int *d_err, cudaStream_t st);
cudaError_t launch_plain_loop_init(PlainLoop *d_loop, cudaStream_t st);
// Records the pass in the loop state and in the instance (passes_run,
// converged; kErrPassLimit in *d_err at the cap) and sets the graph's
// conditional to 1 while another pass is needed.
cudaError_t launch_plain_loop_step(PlainLoop *d_loop, Inst *d_inst, int *d_err, cudaGraphConditionalHandle h,
                                   cudaStream_t st);
cudaError_t launch_engine(int grid, int smem, Inst *d_insts, int ninst, Sched *d_sched, cudaStream_t st);
cudaError_t launch_rule_table(int dims, int dir, uint32_t *d_out, cudaStream_t st);
int engine_max_blocks_per_sm(int smem);
cudaError_t engine_set_smem(int smem);

}  // namespace bgt
