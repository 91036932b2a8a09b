// host.h -- host-side structures behind the C ABI handles.
#pragma once
#include <cstddef>
#include <map>
#include <tuple>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "bgt_capi.h"
#include "common.cuh"
#include "kernels.cuh"

struct bgt_batch;

namespace bgt {
struct Sched;
struct IODesc;

struct Scratch {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct BatchItem {
    int dims = 2, W = 0, H = 0, D = 1, cfg = -1;
    bool auto_cfg = true;  // added with cfg < 0 (the resident engine may take it)
};

struct IO {
    int dtype = 0;
    const void *in = nullptr;
    void *out = nullptr;
    int inW = 0, inH = 0, inD = 0;  // input extents (0: the instance's own)
};

struct Stat {
    int passes = 0, converged = 0;
};

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
size_t dtype_size(int dtype);
int default_cfg(int dims, int W, int H, int D);
int tuned_cfg(int dims, int W, int H, int D);
int ctx_scratch(bgt_ctx *c, int slot, size_t bytes, void **out);
int single_batch(bgt_ctx *c, int dims, int W, int H, int D, bgt_batch **out);
int batch_check(bgt_batch *b);
int batch_set_input_extent(bgt_batch *b, int id, int inW, int inH, int inD);
size_t batch_pool_bytes(const std::vector<BatchItem> &items);
// Lay a batch out in caller-provided device memory (the serving runtime's
// arena) from the next finalize on; the memory is not freed by the batch.
int batch_use_pool(bgt_batch *b, void *pool, size_t bytes);

// Segment list on the host (malloc'ed arrays), in the reference's emission order.
struct HostSegs {
    int nseg = 0, npts = 0;
    int32_t *start = nullptr;
    uint8_t *is_end = nullptr;
    int16_t *px = nullptr, *py = nullptr, *pz = nullptr;
};
// Segment arrays in device memory (same layout as HostSegs; null when empty).
struct DevSegs {
    int nseg = 0, npts = 0;
    int32_t *start = nullptr;
    uint8_t *is_end = nullptr;
    int16_t *px = nullptr, *py = nullptr, *pz = nullptr;
};
// Device ExtractSegmentsV on a packed image (P words per row): arrays left in
// the context's scratch, or copied to host memory.
int segments_device_arrays(bgt_ctx *c, int dims, const uint32_t *d_buf, int W, int H, int D, int P, DevSegs *out);
int segments_packed(bgt_ctx *c, int dims, const uint32_t *d_buf, int W, int H, int D, int P, HostSegs *out);
// Exclusive prefix sum of n ints on the context's stream (CUB temporary
// storage in scratch slot `slot`).
cudaError_t exscan(bgt_ctx *c, int slot, const int *in, int *out, long long n, cudaStream_t st);
void free_host_segs(HostSegs *s);
}  // namespace bgt

struct bgt_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<bgt::Scratch> scratch;
    std::map<std::tuple<int, int, int, int>, bgt_batch *> cache;
};

struct bgt_batch {
    bgt_ctx *ctx = nullptr;
    std::vector<bgt::BatchItem> items;
    std::vector<bgt::Inst> h;
    std::vector<bgt::IO> io;
    std::vector<bgt::Stat> stats;
    bool finalized = false;
    bool stats_valid = false;
    int last_mode = 0;
    void *pool = nullptr;
    size_t pool_bytes = 0;
    size_t used_bytes = 0;
    bool reserved = false;              // pool pre-allocated by bgt_batch_reserve (or external)
    bool external = false;              // pool owned by the caller (batch_use_pool), never freed here
    int grid_cap = 0;                   // engine CTA cap (0: full device)
    std::vector<CUtensorMap> maps;      // host copies of uploaded tables (kept
    std::vector<bgt::IODesc> io_host;   // alive for stream-ordered uploads)
    bgt::Sched *d_sched = nullptr;
    unsigned *d_seq = nullptr;
    int4 *d_item = nullptr;
    bgt::Inst *d_insts = nullptr;
    CUtensorMap *d_tmaps = nullptr;
    int *d_flag = nullptr;
    void *d_lc = nullptr;         // contiguous per-tile "last change" arrays
    size_t lc_bytes = 0;
    bgt::IODesc *d_io = nullptr;  // per-instance I/O table of the batch-wide pack/unpack
    bool io_dirty = true;
    bool any_out = false;
    bool bytes_only = false;  // every input one byte wide, tested "byte != 0"
    long long pack_words = 0, unpack_words = 0;
    unsigned cap = 0;
    int smem = 0;
    int grid = 0;
    // stage boundaries of an engine run: pack, resident engine, tile engine, unpack
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // resident engine plan (resident.cu): items in the order they are taken
    int engine_mode = 0;              // 0: resident engine where it fits, tile rings for the rest; 1: rings only
    std::vector<bgt::ResItem> res_items;
    bgt::ResItem *d_res_items = nullptr;
    bgt::ResSched *d_rs = nullptr;
    bgt::ResTrace *d_rtrace = nullptr;  // per-item timeline of the last resident run
    int res_grid = 0;
    bool any_ring = false;            // some instance is planned for the tile rings
    bool any_res3d = false;           // some volume may spill from the resident engine to the rings
    cudaGraphExec_t gexec = nullptr;
    bool graph_valid = false;
    // plain path with the pass loop on the device (bgt_batch_run mode 2)
    cudaGraphExec_t pexec = nullptr;
    bool pgraph_valid = false;
    bgt::PlainLoop *d_ploop = nullptr;  // one loop state per instance
};
