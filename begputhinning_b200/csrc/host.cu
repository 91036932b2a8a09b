// host.cu -- host side of the C ABI: contexts, batches (device pool layout,
// TMA tensor maps, the persistent engine and the plain per-pass path, CUDA
// graph replay) and the drop-in thinning entry points.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include <cudaTypedefs.h>

#include "host.h"
#include "kernels.cuh"

using namespace bgt;

// ------------------------------------------------------------ errors -------
static thread_local std::string g_err;

int bgt::fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int bgt::cuda_fail(cudaError_t e, const char *what)
{
    return fail(e == cudaErrorMemoryAllocation ? BGT_ERR_NOMEM : BGT_ERR_CUDA, "%s: %s (%d)", what,
                cudaGetErrorString(e), (int)e);
}

extern "C" const char *bgt_last_error(void) { return g_err.c_str(); }
extern "C" int bgt_version(void) { return 100; }

size_t bgt::dtype_size(int dtype)
{
    switch (dtype) {
    case BGT_U8: case BGT_I8: case BGT_CHAR: case BGT_BOOL: return 1;
    case BGT_U16: case BGT_I16: return 2;
    case BGT_U32: case BGT_I32: case BGT_F32: return 4;
    case BGT_F64: return 8;
    default: return 0;
    }
}

// ------------------------------------------------------------ context ------
extern "C" int bgt_ctx_create(int device, bgt_ctx **out)
{
    if (!out) return fail(BGT_ERR_ARG, "bgt_ctx_create: out is null");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    bgt_ctx *c = new bgt_ctx();
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreate");
    }
    c->stream = c->own;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return BGT_OK;
}

extern "C" int bgt_ctx_destroy(bgt_ctx *c)
{
    if (!c) return BGT_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto &kv : c->cache) bgt_batch_destroy(kv.second);
    c->cache.clear();
    for (auto &p : c->scratch) cudaFree(p.ptr);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return BGT_OK;
}

extern "C" int bgt_ctx_set_stream(bgt_ctx *c, void *stream)
{
    if (!c) return fail(BGT_ERR_ARG, "null context");
    c->stream = stream ? (cudaStream_t)stream : c->own;
    for (auto &kv : c->cache) kv.second->graph_valid = kv.second->pgraph_valid = false;
    return BGT_OK;
}

// Named resident scratch buffer of at least `bytes` (grown, never shrunk).
int bgt::ctx_scratch(bgt_ctx *c, int slot, size_t bytes, void **out)
{
    if ((int)c->scratch.size() <= slot) c->scratch.resize(slot + 1);
    Scratch &s = c->scratch[slot];
    if (s.bytes < bytes) {
        if (s.ptr) {
            cudaStreamSynchronize(c->stream);
            cudaFree(s.ptr);
            s.ptr = nullptr;
            s.bytes = 0;
        }
        size_t nb = std::max(bytes, (size_t)4096);
        cudaError_t e = cudaMalloc(&s.ptr, nb);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(scratch)");
        s.bytes = nb;
    }
    *out = s.ptr;
    return BGT_OK;
}

// ------------------------------------------------------------ tensor maps --
static PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// Map over one packed buffer of the instance (`base`: buf[0], buf[1] or the
// 3D union) with the given box (words, rows, planes).
static int encode_map(CUtensorMap *m, const Inst &in, const int (&bx)[3], uint32_t *base)
{
    auto enc = get_encode();
    if (!enc) return fail(BGT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)in.P, (cuuint64_t)in.H, (cuuint64_t)in.D};
    cuuint64_t strides[2] = {(cuuint64_t)in.P * 4, (cuuint64_t)in.P * in.H * 4};
    cuuint32_t box[3] = {(cuuint32_t)bx[0], (cuuint32_t)bx[1], (cuuint32_t)bx[2]};
    cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t rank = in.dims == 2 ? 2 : 3;
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, rank, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(BGT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) P=%d H=%d D=%d box=%u,%u,%u", (int)r, in.P,
                    in.H, in.D, box[0], box[1], box[2]);
    return BGT_OK;
}

// ------------------------------------------------------------ autotune ----
// Default tile configuration by shape; the autotuner (begputhinning_b200/tune.py) may override
// through bgt::tuned_cfg.
int bgt::default_cfg(int dims, int W, int H, int D)
{
    (void)H;
    (void)D;
    (void)W;
    // measured on the mixed batch: K=4, 12-word tiles for every 2D width;
    // 4-plane tiles for volumes (shortest chain of dependent passes)
    return dims == 3 ? 19 : 2;
}

// ------------------------------------------------------------ batch -------
extern "C" int bgt_batch_create(bgt_ctx *ctx, bgt_batch **out)
{
    if (!ctx || !out) return fail(BGT_ERR_ARG, "bgt_batch_create: null argument");
    bgt_batch *b = new bgt_batch();
    b->ctx = ctx;
    *out = b;
    return BGT_OK;
}

static void batch_free_device(bgt_batch *b)
{
    for (auto &ev : b->ev)
        if (ev) {
            cudaEventDestroy(ev);
            ev = nullptr;
        }
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
    if (b->pexec) cudaGraphExecDestroy(b->pexec);
    b->pexec = nullptr;
    b->graph_valid = b->pgraph_valid = false;
    if (b->pool && !b->external) cudaFree(b->pool);
    b->pool = nullptr;
    if (b->d_ploop) cudaFree(b->d_ploop);
    b->d_ploop = nullptr;
}

int bgt::batch_use_pool(bgt_batch *b, void *pool, size_t bytes)
{
    if (!b || !pool) return fail(BGT_ERR_ARG, "null argument");
    if (b->finalized) return fail(BGT_ERR_STATE, "set the pool before finalize");
    if (b->pool && !b->external) return fail(BGT_ERR_STATE, "the batch already owns a pool");
    b->pool = pool;
    b->pool_bytes = bytes;
    b->reserved = true;
    b->external = true;
    return BGT_OK;
}

extern "C" int bgt_batch_destroy(bgt_batch *b)
{
    if (!b) return BGT_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    batch_free_device(b);
    delete b;
    return BGT_OK;
}

static int batch_add(bgt_batch *b, int dims, int W, int H, int D, int cfg, int *id)
{
    if (!b) return fail(BGT_ERR_ARG, "null batch");
    if (b->finalized) return fail(BGT_ERR_STATE, "batch already finalized");
    if (W < 1 || H < 1 || D < 1 || W > 32767 || H > 32767 || D > 32767)
        return fail(BGT_ERR_ARG, "size %dx%dx%d out of range (1..32767 per axis)", W, H, D);
    if ((long long)W * H * D >= (1LL << 31))
        return fail(BGT_ERR_LIMIT, "instance of %lld pixels: the limit is 2^31 - 1", (long long)W * H * D);
    if (cfg >= 0) {
        const CfgInfo *c = cfg_info(cfg);
        if (!c || c->dims != dims) return fail(BGT_ERR_ARG, "configuration %d is not a %dD configuration", cfg, dims);
    }
    BatchItem it;
    it.dims = dims;
    it.W = W;
    it.H = H;
    it.D = D;
    it.cfg = cfg;
    it.auto_cfg = cfg < 0;
    b->items.push_back(it);
    if (id) *id = (int)b->items.size() - 1;
    return BGT_OK;
}

extern "C" int bgt_batch_add2d(bgt_batch *b, int w, int h, int cfg, int *id) { return batch_add(b, 2, w, h, 1, cfg, id); }
extern "C" int bgt_batch_add3d(bgt_batch *b, int w, int h, int d, int cfg, int *id)
{
    return batch_add(b, 3, w, h, d, cfg, id);
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Which instances the resident engine takes and how large 2D images are cut
// into bands: a band holds at most what one CTA's shared memory does, and an
// image is cut further while it is a large share of the batch's work (so a
// batch of few large images still spreads over the SMs), keeping at least 32
// core rows per band.  Items are ordered volumes first (largest first: their
// chains of iterations are the longest), then images largest first, the bands
// of one image consecutive.
static void plan_resident(bgt_batch *b)
{
    constexpr int kHalo = kResHalo2D, kMinCore = 32;  // 2D band halo
    b->res_items.clear();
    b->any_ring = false;
    b->any_res3d = false;
    const int N = (int)b->items.size();
    const bool rings_only = b->engine_mode == 1 || (getenv("BGT_ENGINE") && !strcmp(getenv("BGT_ENGINE"), "rings"));
    double total = 0;
    for (const BatchItem &it : b->items) total += (double)((it.W + 31) / 32) * it.H * it.D;
    const double target = std::max(total / std::max(1, b->res_grid), 4096.0);
    std::vector<std::pair<double, int>> vols, imgs;
    for (int i = 0; i < N; i++) {
        const BatchItem &it = b->items[i];
        Inst &in = b->h[i];
        in.res = 0;
        if (rings_only || !it.auto_cfg || b->res_grid < 1) continue;
        if (it.dims == 3) {
            if (!res_fits3d(it.W, it.H, it.D)) continue;
            in.res = 1;
            vols.push_back({(double)it.W * it.H * it.D, i});
        } else {
            in.res = 1;
            imgs.push_back({(double)((it.W + 31) / 32) * it.H, i});
        }
    }
    std::stable_sort(vols.begin(), vols.end(), [](auto &x, auto &y) { return x.first > y.first; });
    std::stable_sort(imgs.begin(), imgs.end(), [](auto &x, auto &y) { return x.first > y.first; });
    // a large volume is cut into z-slabs of whole brick layers (4 planes),
    // each with two halo layers on either side, so its iterations spread
    // over several SMs, and so that a slab's non-empty bricks fit one CTA
    // (counted on the device: a volume is planned for a quarter of its
    // slab's bricks being non-empty; one that exceeds it goes to the tile
    // rings); at least 4 core layers per slab
    constexpr int kHalo3 = 2, kMinLayers = 4;
    double vox_per_slab = 1.0e6;
    if (const char *e = getenv("BGT_RES3D_SLAB_VOXELS")) vox_per_slab = std::max(1.0e4, atof(e));
    for (auto &v : vols) {
        const BatchItem &it = b->items[v.second];
        const int layers = (it.D + 3) / 4;
        const int gmax = std::max(1, std::min(layers / kMinLayers, b->res_grid));
        int G = std::max(1, std::min((int)std::ceil(v.first / vox_per_slab), gmax));
        auto slab_ok = [&](int g) {
            const int sl = g == 1 ? layers : (layers + g - 1) / g + 2 * kHalo3;
            const int cap = res_slots_fit3d(it.W, it.H, 4 * sl);
            const double bricks = (double)((it.W + 31) / 32) * ((it.H + 31) / 32) * sl;
            return cap > 0 && 0.25 * bricks <= cap;
        };
        while (G < gmax && !slab_ok(G)) G++;
        while (G > 1 && res_slots_fit3d(it.W, it.H, 4 * ((layers + G - 1) / G + 2 * kHalo3)) == 0) G--;
        for (int k = 0; k < G; k++) {
            const int r0 = (int)((long long)k * layers / G), r1 = (int)((long long)(k + 1) * layers / G);
            b->res_items.push_back(ResItem{v.second, k, G, r0, r1, G > 1 ? kHalo3 : 0});
        }
        b->any_res3d = true;
    }
    for (auto &m : imgs) {
        const int i = m.second;
        const BatchItem &it = b->items[i];
        const int fit = res_rows_fit2d(it.W);
        int G = 1;
        if (it.H > fit) {
            G = (it.H + (fit - 2 * kHalo) - 1) / std::max(1, fit - 2 * kHalo);
            while ((it.H + G - 1) / G + 2 * kHalo > fit) G++;
        }
        const int G_work = (int)std::ceil(m.first / target);
        const int G_rows = std::max(1, it.H / kMinCore);
        G = std::max(G, std::min(G_work, G_rows));
        G = std::min(G, b->res_grid);
        const bool fits = G == 1 ? it.H <= fit : (it.H + G - 1) / G + 2 * kHalo <= fit && it.H / G >= kHalo;
        if (!fits) {
            b->h[i].res = 0;  // cannot be cut into bands that fit: the rings take it
            continue;
        }
        for (int k = 0; k < G; k++) {
            const int r0 = (int)((long long)k * it.H / G), r1 = (int)((long long)(k + 1) * it.H / G);
            b->res_items.push_back(ResItem{i, k, G, r0, r1, G > 1 ? kHalo : 0});
        }
    }
    for (int i = 0; i < N; i++)
        if (!b->h[i].res) b->any_ring = true;
}

// Tile geometry and limits of one instance (no device memory yet).
static void init_inst(BatchItem &it, Inst &in)
{
    if (it.cfg < 0) it.cfg = tuned_cfg(it.dims, it.W, it.H, it.D);
    const CfgInfo &c = *cfg_info(it.cfg);
    memset(&in, 0, sizeof(in));
    in.dims = it.dims;
    in.W = it.W;
    in.H = it.H;
    in.D = it.D;
    in.P = (int)align_up((size_t)(it.W + 31) / 32, 4);
    in.cfg = it.cfg;
    in.TW = c.TW;
    in.TH = c.TH;
    in.TZ = c.TZc;
    in.k = c.k;
    in.window = std::max(1, (4 + c.k - 1) / c.k);
    const int wwords = (it.W + 31) / 32;
    in.tiles_x = (wwords + c.TW - 1) / c.TW;
    in.tiles_y = (it.H + c.TH - 1) / c.TH;
    in.tiles_z = (it.D + c.TZc - 1) / c.TZc;
    in.ntiles = in.tiles_x * in.tiles_y * in.tiles_z;
    const int maxdim = std::max(it.W, std::max(it.H, it.D));
    const int passes_per_iter = it.dims == 3 ? 6 : std::max(1, 4 / c.k);
    in.pass_cap = (maxdim + 16) * passes_per_iter + 64;
    // 3D instances carry the longest chains of dependent passes (six
    // passes per iteration): their waves go to the ring served first
    in.prio = it.dims == 3 ? 0 : 1;
}

// Offsets of everything a batch keeps in its device pool.
struct InstOffs {
    size_t b0, b1, uni, lc, act, list;
};
struct PoolLayout {
    std::vector<InstOffs> offs;
    size_t off_lc = 0, lc_bytes = 0, off_io = 0, off_sched = 0, off_seq = 0, off_item = 0, off_inst = 0,
           off_tmap = 0, off_flag = 0, off_res = 0, off_rs = 0, off_rt = 0, total = 0;
    unsigned cap = 0;
};

static PoolLayout layout_pool(const std::vector<Inst> &h, size_t n_res_items)
{
    PoolLayout L;
    const int N = (int)h.size();
    L.offs.resize(N);
    size_t off = 0, total_tiles = 0;
    for (int i = 0; i < N; i++) {
        const Inst &in = h[i];
        const size_t words = (size_t)in.P * in.H * in.D;
        InstOffs &o = L.offs[i];
        o.b0 = off; off = align_up(off + words * 4, 256);
        o.b1 = off; off = align_up(off + words * 4, 256);
        o.uni = 0;
        if (in.dims == 3) { o.uni = off; off = align_up(off + words * 4, 256); }
        o.act = off; off = align_up(off + (size_t)in.ntiles, 256);
        o.list = off; off = align_up(off + (size_t)in.ntiles * 4, 256);
        total_tiles += in.ntiles;
    }
    // all per-tile "last change" arrays in one block (one memset per run)
    L.off_lc = off;
    for (int i = 0; i < N; i++) {
        L.offs[i].lc = off;
        off += (size_t)h[i].ntiles * 4;
    }
    L.lc_bytes = off - L.off_lc;
    off = align_up(off, 256);
    L.off_io = off; off = align_up(off + (size_t)N * sizeof(IODesc), 256);
    // scheduler + ring + instance table + tensor maps + flags
    L.cap = (unsigned)(total_tiles + 1024);
    L.off_sched = off; off = align_up(off + sizeof(Sched), 256);
    L.off_seq = off; off = align_up(off + (size_t)L.cap * 4 * 2, 256);
    L.off_item = off; off = align_up(off + (size_t)L.cap * sizeof(int4) * 2, 256);
    L.off_inst = off; off = align_up(off + (size_t)N * sizeof(Inst), 256);
    L.off_tmap = off; off = align_up(off + (size_t)N * kMapsPerInst * sizeof(CUtensorMap), 256);
    L.off_flag = off; off = align_up(off + 64, 256);
    // resident engine: item list + its scheduler
    L.off_res = off; off = align_up(off + std::max<size_t>(1, n_res_items) * sizeof(ResItem), 256);
    L.off_rs = off; off = align_up(off + sizeof(ResSched), 256);
    L.off_rt = off; off = align_up(off + std::max<size_t>(1, n_res_items) * sizeof(ResTrace), 256);
    L.total = off;
    return L;
}

// Device pool bytes a tile-ring batch of these shapes needs (the serving
// runtime sizes its admissions with it).
size_t bgt::batch_pool_bytes(const std::vector<BatchItem> &items)
{
    std::vector<BatchItem> its = items;
    std::vector<Inst> h(its.size());
    for (size_t i = 0; i < its.size(); i++) init_inst(its[i], h[i]);
    return layout_pool(h, 0).total;
}

extern "C" int bgt_batch_finalize(bgt_batch *b)
{
    if (!b) return fail(BGT_ERR_ARG, "null batch");
    if (b->finalized) return BGT_OK;
    if (b->items.empty()) return fail(BGT_ERR_STATE, "empty batch");
    cudaSetDevice(b->ctx->device);
    const int N = (int)b->items.size();
    b->h.assign(N, Inst());
    int max_smem = 0;
    for (int i = 0; i < N; i++) {
        init_inst(b->items[i], b->h[i]);
        max_smem = std::max(max_smem, cfg_info(b->items[i].cfg)->smem);
    }
    {
        int per_sm = 0;
        if (res_occupancy(&per_sm) == cudaSuccess && per_sm > 0) b->res_grid = b->ctx->sms * per_sm;
        else b->res_grid = 0;
        if (b->grid_cap > 0) b->res_grid = std::min(b->res_grid, b->grid_cap);
    }
    plan_resident(b);
    const PoolLayout L = layout_pool(b->h, b->res_items.size());
    const std::vector<InstOffs> &offs = L.offs;
    const size_t off = L.total, off_lc = L.off_lc, off_io = L.off_io, off_sched = L.off_sched,
                 off_seq = L.off_seq, off_item = L.off_item, off_inst = L.off_inst, off_tmap = L.off_tmap,
                 off_flag = L.off_flag, off_res = L.off_res, off_rs = L.off_rs;
    const unsigned cap = L.cap;
    b->lc_bytes = L.lc_bytes;
    cudaError_t e;
    if (b->reserved) {
        // a reserved pool is re-laid-out for every set of instances, never reallocated
        if (off > b->pool_bytes)
            return fail(BGT_ERR_LIMIT, "batch needs %zu bytes, the reserved pool holds %zu", off, b->pool_bytes);
    } else {
        e = cudaMalloc(&b->pool, off);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch pool)");
        b->pool_bytes = off;
    }
    b->used_bytes = off;
    char *P = (char *)b->pool;
    b->d_sched = (Sched *)(P + off_sched);
    b->d_seq = (unsigned *)(P + off_seq);
    b->d_item = (int4 *)(P + off_item);
    b->d_insts = (Inst *)(P + off_inst);
    b->d_tmaps = (CUtensorMap *)(P + off_tmap);
    b->d_flag = (int *)(P + off_flag);
    b->d_lc = P + off_lc;
    b->d_io = (IODesc *)(P + off_io);
    b->d_res_items = (ResItem *)(P + off_res);
    b->d_rs = (ResSched *)(P + off_rs);
    b->d_rtrace = (ResTrace *)(P + L.off_rt);
    b->cap = cap;
    std::vector<CUtensorMap> &maps = b->maps;
    maps.assign((size_t)N * kMapsPerInst, CUtensorMap());
    for (int i = 0; i < N; i++) {
        Inst &in = b->h[i];
        const InstOffs &o = offs[i];
        in.buf[0] = (uint32_t *)(P + o.b0);
        in.buf[1] = (uint32_t *)(P + o.b1);
        in.uni = in.dims == 3 ? (uint32_t *)(P + o.uni) : nullptr;
        in.lc = (int *)(P + o.lc);
        in.act = (uint8_t *)(P + o.act);
        in.list = (int *)(P + o.list);
        in.tmap = b->d_tmaps + kMapsPerInst * i;
        const CfgInfo &c = *cfg_info(in.cfg);
        CUtensorMap *m = &maps[(size_t)kMapsPerInst * i];
        int rc = encode_map(&m[0], in, c.box, in.buf[0]);
        if (rc == BGT_OK) rc = encode_map(&m[1], in, c.box, in.buf[1]);
        if (rc == BGT_OK && in.dims == 3) rc = encode_map(&m[2], in, c.ubox, in.uni);
        if (rc != BGT_OK) {
            if (!b->reserved) batch_free_device(b);
            return rc;
        }
    }
    // tables are uploaded in stream order from host copies the batch keeps
    cudaStream_t st = b->ctx->stream;
    e = cudaMemcpyAsync(b->d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_insts, b->h.data(), (size_t)N * sizeof(Inst), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !b->res_items.empty())
        e = cudaMemcpyAsync(b->d_res_items, b->res_items.data(), b->res_items.size() * sizeof(ResItem),
                            cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        if (!b->reserved) batch_free_device(b);
        return cuda_fail(e, "batch table upload");
    }
    b->smem = max_smem;
    // one value for every batch (the largest configuration), so concurrent
    // batches never race on the kernel attribute
    e = engine_set_smem(max_cfg_smem());
    if (e != cudaSuccess) {
        if (!b->reserved) batch_free_device(b);
        return cuda_fail(e, "cudaFuncSetAttribute");
    }
    const int per_sm = std::max(1, engine_max_blocks_per_sm(max_smem));
    b->grid = b->ctx->sms * per_sm;
    if (b->grid_cap > 0) b->grid = std::min(b->grid, b->grid_cap);
    for (auto &ev : b->ev) {
        if (ev) continue;
        e = cudaEventCreate(&ev);
        if (e != cudaSuccess) {
            if (!b->reserved) batch_free_device(b);
            return cuda_fail(e, "cudaEventCreate");
        }
    }
    b->io.assign(N, IO());
    b->stats.assign(N, Stat());
    b->finalized = true;
    return BGT_OK;
}

// Pre-allocate `bytes` of device pool: later finalize calls lay the batch out
// in it (reset + add + finalize reuses it without any allocation) and fail
// with BGT_ERR_LIMIT when a set of instances does not fit.
extern "C" int bgt_batch_reserve(bgt_batch *b, size_t bytes)
{
    if (!b) return fail(BGT_ERR_ARG, "null batch");
    if (b->finalized || b->pool) return fail(BGT_ERR_STATE, "reserve before the first finalize");
    cudaSetDevice(b->ctx->device);
    cudaError_t e = cudaMalloc(&b->pool, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(reserved batch pool)");
    b->pool_bytes = bytes;
    b->reserved = true;
    return BGT_OK;
}

// Drop the instances (after the last run finished on the batch's stream);
// a reserved pool and the events are kept.
extern "C" int bgt_batch_reset(bgt_batch *b)
{
    if (!b) return fail(BGT_ERR_ARG, "null batch");
    if (!b->reserved && b->pool) {
        cudaStreamSynchronize(b->ctx->stream);
        cudaFree(b->pool);
        b->pool = nullptr;
        b->pool_bytes = 0;
    }
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
    if (b->pexec) cudaGraphExecDestroy(b->pexec);
    b->pexec = nullptr;
    if (b->d_ploop) cudaFree(b->d_ploop);  // sized for the old instance count
    b->d_ploop = nullptr;
    b->graph_valid = b->pgraph_valid = false;
    b->items.clear();
    b->h.clear();
    b->io.clear();
    b->stats.clear();
    b->io_dirty = true;
    b->finalized = false;
    b->stats_valid = false;
    return BGT_OK;
}

// Upper bound on the engine's CTAs (0: one full wave of the device), so that
// batches on several streams share the SMs.  Applies from the next finalize.
extern "C" int bgt_batch_set_grid(bgt_batch *b, int ctas)
{
    if (!b || ctas < 0) return fail(BGT_ERR_ARG, "bad argument");
    b->grid_cap = ctas;
    return BGT_OK;
}

// Device time of the stages of the last engine run: pack (with the mark
// reset and scheduler reset), engine (seed + persistent kernel), unpack.
extern "C" int bgt_batch_stage_ms(bgt_batch *b, float *pack_ms, float *engine_ms, float *unpack_ms)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    if (b->last_mode != 0) return fail(BGT_ERR_STATE, "stage times exist only for engine runs");
    cudaError_t e = cudaEventSynchronize(b->ev[4]);
    if (e != cudaSuccess) return cuda_fail(e, "event sync");
    float t[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; k++) {
        e = cudaEventElapsedTime(&t[k], b->ev[k], b->ev[k + 1]);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
    }
    if (pack_ms) *pack_ms = t[0];
    if (engine_ms) *engine_ms = t[1] + t[2];
    if (unpack_ms) *unpack_ms = t[3];
    return BGT_OK;
}

// The engine stage of the last run split into the resident kernel and the
// tile-ring engine that follows it (volumes that spilled, instances the
// resident engine does not take).
extern "C" int bgt_batch_engine_ms(bgt_batch *b, float *resident_ms, float *rings_ms)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    if (b->last_mode != 0) return fail(BGT_ERR_STATE, "stage times exist only for engine runs");
    cudaError_t e = cudaEventSynchronize(b->ev[4]);
    if (e != cudaSuccess) return cuda_fail(e, "event sync");
    float r = 0, g = 0;
    e = cudaEventElapsedTime(&r, b->ev[1], b->ev[2]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&g, b->ev[2], b->ev[3]);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
    if (resident_ms) *resident_ms = r;
    if (rings_ms) *rings_ms = g;
    return BGT_OK;
}

// Timeline of the resident kernel's work items in the last run, in the
// order they were taken: instance, band, start and end (global timer, ns,
// relative to the earliest start) and SM.  *n = the number of items.
extern "C" int bgt_batch_res_trace(bgt_batch *b, int *n, int *inst, int *band, long long *t0_ns, long long *t1_ns,
                                   int *sm, int cap)
{
    if (!b || !b->finalized || !n) return fail(BGT_ERR_STATE, "batch not finalized");
    const int m = (int)b->res_items.size();
    *n = m;
    if (m == 0 || cap <= 0) return BGT_OK;
    int rc = batch_check(b);
    if (rc != BGT_OK) return rc;
    std::vector<ResTrace> tr(m);
    cudaError_t e = cudaMemcpy(tr.data(), b->d_rtrace, m * sizeof(ResTrace), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "trace readback");
    long long base = tr[0].t0;
    for (const ResTrace &t : tr) base = std::min(base, t.t0);
    for (int k = 0; k < m && k < cap; k++) {
        if (inst) inst[k] = b->res_items[k].inst;
        if (band) band[k] = b->res_items[k].band;
        if (t0_ns) t0_ns[k] = tr[k].t0 - base;
        if (t1_ns) t1_ns[k] = tr[k].t1 - base;
        if (sm) sm[k] = tr[k].sm;
    }
    return BGT_OK;
}

// Engine choice for the next finalize: 0 = resident engine where an instance
// fits (the default), 1 = tile rings only.
extern "C" int bgt_batch_set_engine(bgt_batch *b, int mode)
{
    if (!b || mode < 0 || mode > 1) return fail(BGT_ERR_ARG, "bad argument");
    b->engine_mode = mode;
    return BGT_OK;
}

// How the last finalize planned instance `id`: *resident = 1 when the
// resident engine takes it, *bands = the number of bands of a 2D image.
extern "C" int bgt_batch_plan(bgt_batch *b, int id, int *resident, int *bands)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    if (id < 0 || id >= (int)b->items.size()) return fail(BGT_ERR_ARG, "bad instance id");
    int n = 0;
    for (const ResItem &r : b->res_items)
        if (r.inst == id) n++;
    if (resident) *resident = b->h[id].res;
    if (bands) *bands = n;
    return BGT_OK;
}

extern "C" int bgt_batch_set_io(bgt_batch *b, int id, int dtype, const void *d_in, void *d_out)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    if (id < 0 || id >= (int)b->items.size()) return fail(BGT_ERR_ARG, "bad instance id %d", id);
    if (dtype_size(dtype) == 0) return fail(BGT_ERR_ARG, "bad dtype %d", dtype);
    IO &io = b->io[id];
    if (io.in != d_in || io.out != d_out || io.dtype != dtype) {
        b->graph_valid = b->pgraph_valid = false;
        b->io_dirty = true;
    }
    io.dtype = dtype;
    io.in = d_in;
    io.out = d_out;
    return BGT_OK;
}

int bgt::batch_set_input_extent(bgt_batch *b, int id, int inW, int inH, int inD)
{
    if (!b || !b->finalized || id < 0 || id >= (int)b->items.size()) return fail(BGT_ERR_ARG, "bad batch/id");
    const Inst &in = b->h[id];
    if (inW > in.W || inH > in.H || inD > in.D) return fail(BGT_ERR_ARG, "input extent larger than the instance");
    IO &io = b->io[id];
    if (io.inW != inW || io.inH != inH || io.inD != inD) {
        b->graph_valid = b->pgraph_valid = false;
        b->io_dirty = true;
    }
    io.inW = inW;
    io.inH = inH;
    io.inD = inD;
    return BGT_OK;
}

// Both rings use `cap` slots; ring r's arrays are seq + r*cap, item + r*cap.
__global__ void sched_reset_kernel(Sched *S, unsigned *seq, int4 *item, unsigned cap, long long timeout_ns,
                                   int gang_budget)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        for (int r = 0; r < 2; r++) {
            S->ring[r].head = 0;
            S->ring[r].tail = 0;
            S->ring[r].cap = cap;
            S->ring[r].seq = seq + (size_t)r * cap;
            S->ring[r].item = item + (size_t)r * cap;
        }
        S->live = 0;
        S->live_prio[0] = 0;
        S->live_prio[1] = 0;
        S->status = 0;
        S->timeout_ns = timeout_ns;
        S->gang_budget = gang_budget;
    }
    for (unsigned s = i; s < cap; s += gridDim.x * blockDim.x) {
        seq[s] = s;
        seq[cap + s] = s;
    }
}

// Upload the per-instance I/O table used by the batch-wide pack/unpack, in
// stream order from a host copy the batch keeps (done before any capture).
static int upload_io(bgt_batch *b)
{
    if (!b->io_dirty) return BGT_OK;
    const int N = (int)b->items.size();
    std::vector<IODesc> &io = b->io_host;
    io.assign(N, IODesc());
    long long w = 0, g = 0;
    for (int i = 0; i < N; i++) {
        const Inst &in = b->h[i];
        const IO &s = b->io[i];
        if (!s.in) return fail(BGT_ERR_STATE, "instance %d has no input", i);
        io[i].in = s.in;
        io[i].out = s.out;
        io[i].dtype = s.dtype;
        io[i].mode = in.dims == 2 ? 0 : 1;
        io[i].inW = s.inW ? s.inW : in.W;
        io[i].inH = s.inH ? s.inH : in.H;
        io[i].inD = s.inD ? s.inD : in.D;
        io[i].inst = i;
        io[i].wbegin = w;
        io[i].gbegin = g;
        io[i].dP = make_fastdiv((uint32_t)in.P);
        io[i].dH = make_fastdiv((uint32_t)in.H);
        io[i].dW = make_fastdiv((uint32_t)in.W);
        io[i].dWW = make_fastdiv((uint32_t)((in.W + 31) / 32));
        io[i].dTW = make_fastdiv((uint32_t)in.TW);
        io[i].dTH = make_fastdiv((uint32_t)in.TH);
        io[i].dTZ = make_fastdiv((uint32_t)std::max(1, in.TZ));
        w += (long long)in.P * in.H * in.D;
        if (dtype_size(s.dtype) == 1 && s.out) {
            // unpack unit: 32-byte-aligned chunk of the output
            const uintptr_t o = reinterpret_cast<uintptr_t>(s.out);
            const uintptr_t end = o + (uintptr_t)in.W * in.H * in.D;
            g += (long long)((end - (o & ~uintptr_t(31)) + 31) / 32);
        } else {
            // unpack unit: packed word (rows x ceil(W/32))
            g += (long long)((in.W + 31) / 32) * in.H * in.D;
        }
    }
    b->pack_words = w;
    b->unpack_words = g;
    b->any_out = false;
    b->bytes_only = true;
    for (int i = 0; i < N; i++) {
        b->any_out |= b->io[i].out != nullptr;
        const int dt = io[i].dtype;
        b->bytes_only &= dtype_size(dt) == 1 && (io[i].mode == 0 || dt == BGT_U8 || dt == BGT_BOOL);
    }
    cudaError_t e = cudaMemcpyAsync(b->d_io, io.data(), (size_t)N * sizeof(IODesc), cudaMemcpyHostToDevice,
                                    b->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "I/O table upload");
    b->io_dirty = false;
    return BGT_OK;
}

// Stream-ordered sequence of the engine run (capturable): mark reset, one
// batch-wide pack (which also marks non-empty tiles), scheduler reset, seed
// + persistent engine, one batch-wide unpack.
// Stage boundary event: inside a capture it must become an event-record node
// (cudaEventRecordExternal); outside a capture it is a plain record.
static void stage_event(cudaEvent_t ev, cudaStream_t st, bool capturing)
{
    if (capturing)
        cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal);
    else
        cudaEventRecord(ev, st);
}

static int enqueue_engine(bgt_batch *b, cudaStream_t st, bool capturing)
{
    const int N = (int)b->items.size();
    stage_event(b->ev[0], st, capturing);
    cudaError_t e = cudaMemsetAsync(b->d_lc, 0x80, b->lc_bytes, st);
    if (e == cudaSuccess) e = launch_pack_all(b->d_insts, b->d_io, N, b->pack_words, b->bytes_only, st);
    if (e != cudaSuccess) return cuda_fail(e, "pack");
    sched_reset_kernel<<<std::min<unsigned>(1024, (b->cap + 255) / 256), 256, 0, st>>>(
        b->d_sched, b->d_seq, b->d_item, b->cap, 20000000000LL, b->grid);
    stage_event(b->ev[1], st, capturing);
    // bands of an image wait for one another only for the length of one
    // iteration of the slowest band: 4 s is far beyond any legitimate wait
    e = launch_resident(b->res_grid, b->d_insts, N, b->d_res_items, (int)b->res_items.size(), b->d_rs,
                        b->d_rtrace, 4000000000LL, st);
    if (e != cudaSuccess) return cuda_fail(e, "resident engine launch");
    stage_event(b->ev[2], st, capturing);
    if (b->any_ring || b->any_res3d) {
        e = launch_engine(b->grid, b->smem, b->d_insts, N, b->d_sched, st);
        if (e != cudaSuccess) return cuda_fail(e, "engine launch");
    }
    stage_event(b->ev[3], st, capturing);
    if (b->any_out) {
        e = launch_unpack_all(b->d_insts, b->d_io, N, b->unpack_words, st);
        if (e != cudaSuccess) return cuda_fail(e, "unpack");
    }
    stage_event(b->ev[4], st, capturing);
    return BGT_OK;
}

static int run_engine(bgt_batch *b, int use_graph)
{
    cudaStream_t st = b->ctx->stream;
    int rc = upload_io(b);
    if (rc != BGT_OK) return rc;
    if (use_graph) {
        if (!b->graph_valid) {
            if (b->gexec) cudaGraphExecDestroy(b->gexec);
            b->gexec = nullptr;
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
            rc = enqueue_engine(b, st, true);
            e = cudaStreamEndCapture(st, &g);
            if (rc != BGT_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&b->gexec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
            b->graph_valid = true;
        }
        cudaError_t e = cudaGraphLaunch(b->gexec, st);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    } else {
        rc = enqueue_engine(b, st, false);
        if (rc != BGT_OK) return rc;
    }
    b->stats_valid = false;
    b->last_mode = 0;
    return BGT_OK;
}

static int run_plain(bgt_batch *b)
{
    cudaStream_t st = b->ctx->stream;
    const int N = (int)b->items.size();
    cudaError_t e;
    int *h_flag = nullptr;
    e = cudaMallocHost(&h_flag, 64);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    int rc = BGT_OK;
    // per-launch status word lives in the scheduler block
    int *d_err = &b->d_sched->status;
    cudaMemsetAsync(d_err, 0, sizeof(int), st);
    for (int i = 0; i < N && rc == BGT_OK; i++) {
        const Inst &in = b->h[i];
        const IO &io = b->io[i];
        if (!io.in) { rc = fail(BGT_ERR_STATE, "instance %d has no input", i); break; }
        e = launch_pack(io.dtype, in.dims == 2 ? 0 : 1, io.in, io.inW ? io.inW : in.W, io.inH ? io.inH : in.H,
                        io.inD ? io.inD : in.D, in.W, in.H, in.D, in.P, in.buf[0], in.buf[1], st);
        if (e == cudaSuccess) e = launch_tile_init(b->d_insts + i, in, nullptr, st);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(&b->d_insts[i].tiles_run, 0, 2 * sizeof(unsigned long long), st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "pack"); break; }
        int last_change = -1;  // tiles start "changed just before pass 0"
        int q = 0;
        int converged = 0;
        for (; q < in.pass_cap; q++) {
            cudaMemsetAsync(b->d_flag, 0, sizeof(int), st);
            e = launch_plain_pass(in.cfg, b->d_insts + i, in.ntiles, q, b->d_flag, d_err, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h_flag, b->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) { rc = cuda_fail(e, "plain pass"); break; }
            if (h_flag[0]) last_change = q;
            if (in.dims == 2) {
                if (q - last_change >= in.window) { converged = 1; q++; break; }
            } else if (q % 6 == 5 && last_change < q - 5) {
                converged = 1;
                q++;
                break;
            }
        }
        b->stats[i].passes = q;
        b->stats[i].converged = converged ? 1 : -1;
        if (rc == BGT_OK && !converged) rc = fail(BGT_ERR_LIMIT, "instance %d hit the pass cap", i);
        if (rc == BGT_OK && io.out) {
            e = launch_unpack(io.dtype, in.buf[0], in.W, in.H, in.D, in.P, io.out, st);
            if (e != cudaSuccess) rc = cuda_fail(e, "unpack");
        }
    }
    cudaFreeHost(h_flag);
    b->stats_valid = true;
    b->last_mode = 1;
    return rc;
}

// The plain path with its pass loop on the device: one CUDA graph for the
// batch in which every instance is packed, thinned by a conditional WHILE
// node (body: one pass over all its tiles, then plain_loop_step_kernel, which
// applies run_plain's convergence rule and sets the condition), and
// unpacked, one instance after another.  No pass waits for the host.
static int capture_into(cudaGraph_t g, cudaStream_t st, const cudaGraphNode_t *deps, size_t ndeps)
{
    cudaError_t e = cudaStreamBeginCaptureToGraph(st, g, deps, nullptr, ndeps, cudaStreamCaptureModeThreadLocal);
    return e == cudaSuccess ? BGT_OK : cuda_fail(e, "cudaStreamBeginCaptureToGraph");
}

static int capture_tail(cudaStream_t st, std::vector<cudaGraphNode_t> &tail)
{
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *d = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &d, &nd);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamGetCaptureInfo");
    tail.assign(d, d + nd);
    return BGT_OK;
}

static int build_plain_graph(bgt_batch *b, cudaGraph_t g)
{
    cudaStream_t st = b->ctx->stream;
    const int N = (int)b->items.size();
    int *d_err = &b->d_sched->status;
    std::vector<cudaGraphNode_t> tail;
    cudaGraph_t dummy = nullptr;
    int rc = capture_into(g, st, nullptr, 0);
    if (rc != BGT_OK) return rc;
    cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
    for (int i = 0; i < N && e == cudaSuccess; i++) {
        const Inst &in = b->h[i];
        const IO &io = b->io[i];
        if (!io.in) {
            cudaStreamEndCapture(st, &dummy);
            return fail(BGT_ERR_STATE, "instance %d has no input", i);
        }
        e = launch_pack(io.dtype, in.dims == 2 ? 0 : 1, io.in, io.inW ? io.inW : in.W, io.inH ? io.inH : in.H,
                        io.inD ? io.inD : in.D, in.W, in.H, in.D, in.P, in.buf[0], in.buf[1], st);
        if (e == cudaSuccess) e = launch_tile_init(b->d_insts + i, in, nullptr, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(&b->d_insts[i].tiles_run, 0, 2 * sizeof(unsigned long long), st);
        if (e == cudaSuccess) e = launch_plain_loop_init(b->d_ploop + i, st);
        if (e != cudaSuccess) break;
        rc = capture_tail(st, tail);
        cudaStreamEndCapture(st, &dummy);
        if (rc != BGT_OK) return rc;
        cudaGraphConditionalHandle h;
        e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphConditionalHandleCreate");
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        e = cudaGraphAddNode(&cn, g, tail.data(), tail.size(), &cp);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphAddNode (while)");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        rc = capture_into(body, st, nullptr, 0);
        if (rc != BGT_OK) return rc;
        e = launch_plain_dev_pass(in.cfg, b->d_insts + i, in.ntiles, b->d_ploop + i, d_err, st);
        if (e == cudaSuccess) e = launch_plain_loop_step(b->d_ploop + i, b->d_insts + i, d_err, h, st);
        cudaStreamEndCapture(st, &dummy);
        if (e != cudaSuccess) return cuda_fail(e, "plain pass (capture)");
        rc = capture_into(g, st, &cn, 1);
        if (rc != BGT_OK) return rc;
        if (io.out) e = launch_unpack(io.dtype, in.buf[0], in.W, in.H, in.D, in.P, io.out, st);
    }
    cudaError_t e2 = cudaStreamEndCapture(st, &dummy);
    if (e != cudaSuccess) return cuda_fail(e, "plain graph");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
    return BGT_OK;
}

static int run_plain_device(bgt_batch *b)
{
    cudaStream_t st = b->ctx->stream;
    const int N = (int)b->items.size();
    if (N == 0) return BGT_OK;
    if (!b->d_ploop) {
        cudaError_t e = cudaMalloc(&b->d_ploop, sizeof(PlainLoop) * (size_t)N);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (plain loop state)");
    }
    if (!b->pgraph_valid) {
        if (b->pexec) cudaGraphExecDestroy(b->pexec);
        b->pexec = nullptr;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaGraphCreate(&g, 0);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphCreate");
        int rc = build_plain_graph(b, g);
        if (rc == BGT_OK) {
            e = cudaGraphInstantiate(&b->pexec, g, 0);
            if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate (plain)");
        }
        cudaGraphDestroy(g);
        if (rc != BGT_OK) return rc;
        b->pgraph_valid = true;
    }
    cudaError_t e = cudaGraphLaunch(b->pexec, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch (plain)");
    b->stats_valid = false;
    b->last_mode = 2;
    return BGT_OK;
}

extern "C" int bgt_batch_run(bgt_batch *b, int mode, int use_graph)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    if (mode < 0 || mode > 2) return fail(BGT_ERR_ARG, "mode must be 0 (engine), 1 (plain) or 2 (plain, device loop)");
    cudaSetDevice(b->ctx->device);
    int rc = mode == 1 ? run_plain(b) : mode == 2 ? run_plain_device(b) : run_engine(b, use_graph);
    if (rc != BGT_OK) return rc;
    return BGT_OK;
}

// Synchronise and turn the kernels' status word into an error code.
int bgt::batch_check(bgt_batch *b)
{
    cudaError_t e = cudaStreamSynchronize(b->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch run");
    int status = 0, rstatus = 0;
    e = cudaMemcpy(&status, &b->d_sched->status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && b->last_mode == 0 && !b->res_items.empty())
        e = cudaMemcpy(&rstatus, &b->d_rs->status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "status readback");
    status |= rstatus;
    if (status & (kErrTmaTimeout | kErrQueueTimeout | kErrQueueFull))
        return fail(BGT_ERR_TIMEOUT, "device wait gave up (status bits 0x%x)", status);
    if (status & kErrPassLimit) return fail(BGT_ERR_LIMIT, "an instance hit the pass cap");
    return BGT_OK;
}

extern "C" int bgt_batch_instance_stats(bgt_batch *b, int id, int *passes, int *converged, int *cfg)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    if (id < 0 || id >= (int)b->items.size()) return fail(BGT_ERR_ARG, "bad instance id");
    if (!b->stats_valid) {
        int rc = batch_check(b);
        if (rc != BGT_OK) return rc;
        std::vector<Inst> tmp(b->items.size());
        cudaError_t e = cudaMemcpy(tmp.data(), b->d_insts, tmp.size() * sizeof(Inst), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "stats readback");
        for (size_t i = 0; i < tmp.size(); i++) {
            b->stats[i].passes = tmp[i].passes_run;
            b->stats[i].converged = tmp[i].converged;
        }
        b->stats_valid = true;
    }
    if (passes) *passes = b->stats[id].passes;
    if (converged) *converged = b->stats[id].converged;
    if (cfg) *cfg = b->items[id].cfg;
    return BGT_OK;
}

extern "C" int bgt_batch_work(bgt_batch *b, unsigned long long *tiles, unsigned long long *words)
{
    if (!b || !b->finalized) return fail(BGT_ERR_STATE, "batch not finalized");
    int rc = batch_check(b);
    if (rc != BGT_OK) return rc;
    std::vector<Inst> tmp(b->items.size());
    cudaError_t e = cudaMemcpy(tmp.data(), b->d_insts, tmp.size() * sizeof(Inst), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "work readback");
    unsigned long long t = 0, w = 0;
    for (const Inst &in : tmp) {
        t += in.tiles_run;
        w += in.work_words;
    }
    if (tiles) *tiles = t;
    if (words) *words = w;
    return BGT_OK;
}

extern "C" int bgt_batch_device_bytes(bgt_batch *b, size_t *bytes)
{
    if (!b || !bytes) return fail(BGT_ERR_ARG, "null argument");
    *bytes = b->pool_bytes;
    return BGT_OK;
}

extern "C" int bgt_cfg_list(int dims, int *ids, int cap, int *n)
{
    int m = 0;
    const int *l = dims == 3 ? cfg_ids_3d(&m) : cfg_ids_2d(&m);
    if (n) *n = m;
    for (int i = 0; i < m && i < cap && ids; i++) ids[i] = l[i];
    return BGT_OK;
}

extern "C" int bgt_cfg_describe(int id, int *dims, int *k, int *tw, int *th, int *tz, int *smem_bytes)
{
    const CfgInfo *c = cfg_info(id);
    if (!c) return fail(BGT_ERR_ARG, "unknown configuration %d", id);
    if (dims) *dims = c->dims;
    if (k) *k = c->k;
    if (tw) *tw = c->TW;
    if (th) *th = c->TH;
    if (tz) *tz = c->TZc;
    if (smem_bytes) *smem_bytes = c->smem;
    return BGT_OK;
}

// Deletable-set table of the device rule of one direction over every
// neighbourhood (layout in kernels.cu, launch_rule_table): a self-test of the
// rules against any restatement of the reference's.
extern "C" int bgt_rule_table(int dims, int dir, uint32_t *d_out, void *stream)
{
    if (dims != 2 && dims != 3) return fail(BGT_ERR_ARG, "dims must be 2 or 3");
    if (dir < 0 || dir >= (dims == 2 ? 4 : 6)) return fail(BGT_ERR_ARG, "direction %d out of range", dir);
    if (!d_out) return fail(BGT_ERR_ARG, "null output");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = launch_rule_table(dims, dir, d_out, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "rule table");
    return BGT_OK;
}

// ------------------------------------------------------------ drop-in -----
// One cached single-instance batch per (dims, shape).
int bgt::single_batch(bgt_ctx *c, int dims, int W, int H, int D, bgt_batch **out)
{
    auto key = std::make_tuple(dims, W, H, D);
    auto it = c->cache.find(key);
    if (it != c->cache.end()) {
        *out = it->second;
        return BGT_OK;
    }
    if (c->cache.size() >= 16) {  // bound resident memory: drop the oldest shapes
        cudaStreamSynchronize(c->stream);
        for (auto &kv : c->cache) bgt_batch_destroy(kv.second);
        c->cache.clear();
    }
    bgt_batch *b = nullptr;
    int rc = bgt_batch_create(c, &b);
    if (rc == BGT_OK) rc = dims == 2 ? bgt_batch_add2d(b, W, H, -1, nullptr) : bgt_batch_add3d(b, W, H, D, -1, nullptr);
    if (rc == BGT_OK) rc = bgt_batch_finalize(b);
    if (rc != BGT_OK) {
        bgt_batch_destroy(b);
        return rc;
    }
    c->cache[key] = b;
    *out = b;
    return BGT_OK;
}

static int thin_device(bgt_ctx *c, int dims, int dtype, const void *d_in, int W, int H, int D, void *d_out)
{
    if (!c) return fail(BGT_ERR_ARG, "null context");
    if (!d_in || !d_out) return fail(BGT_ERR_ARG, "null buffer");
    if (dtype_size(dtype) == 0) return fail(BGT_ERR_ARG, "bad dtype %d", dtype);
    cudaSetDevice(c->device);
    bgt_batch *b = nullptr;
    int rc = single_batch(c, dims, W, H, D, &b);
    if (rc != BGT_OK) return rc;
    rc = bgt_batch_set_io(b, 0, dtype, d_in, d_out);
    if (rc == BGT_OK) rc = bgt_batch_run(b, 0, 0);
    return rc;
}

extern "C" int bgt_thin2d_device(bgt_ctx *c, int dtype, const void *d_in, int w, int h, void *d_out)
{
    return thin_device(c, 2, dtype, d_in, w, h, 1, d_out);
}

extern "C" int bgt_thin3d_device(bgt_ctx *c, int dtype, const void *d_in, int w, int h, int d, void *d_out)
{
    return thin_device(c, 3, dtype, d_in, w, h, d, d_out);
}

static int thin_host(bgt_ctx *c, int dims, int dtype, const void *in, int W, int H, int D, void *out)
{
    if (!c) return fail(BGT_ERR_ARG, "null context");
    if (!in || !out) return fail(BGT_ERR_ARG, "null buffer");
    const size_t es = dtype_size(dtype);
    if (es == 0) return fail(BGT_ERR_ARG, "bad dtype %d", dtype);
    if (W < 1 || H < 1 || D < 1) return fail(BGT_ERR_ARG, "bad size %dx%dx%d", W, H, D);
    cudaSetDevice(c->device);
    const size_t bytes = es * (size_t)W * H * D;
    void *d_io = nullptr;
    int rc = ctx_scratch(c, 0, bytes, &d_io);
    if (rc != BGT_OK) return rc;
    cudaError_t e = cudaMemcpyAsync(d_io, in, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "H2D");
    bgt_batch *b = nullptr;
    rc = single_batch(c, dims, W, H, D, &b);
    if (rc != BGT_OK) return rc;
    rc = bgt_batch_set_io(b, 0, dtype, d_io, d_io);  // unpack after the engine: in place is safe
    if (rc == BGT_OK) rc = bgt_batch_run(b, 0, 0);
    if (rc != BGT_OK) return rc;
    e = cudaMemcpyAsync(out, d_io, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "D2H");
    return batch_check(b);
}

extern "C" int bgt_thin2d(bgt_ctx *c, int dtype, const void *in, int w, int h, void *out)
{
    return thin_host(c, 2, dtype, in, w, h, 1, out);
}

extern "C" int bgt_thin3d(bgt_ctx *c, int dtype, const void *in, int w, int h, int d, void *out)
{
    return thin_host(c, 3, dtype, in, w, h, d, out);
}

extern "C" void bgt_free(void *p) { free(p); }

extern "C" int bgt_matlab_segments(int dims, unsigned int nsegs, const float *x, const float *y, const float *z,
                                   const unsigned int *idx, double *out)
{
    if (dims != 2 && dims != 3) return fail(BGT_ERR_ARG, "dims must be 2 or 3");
    if (!idx || (nsegs > 0 && (!x || !y || !out || (dims == 3 && !z)))) return fail(BGT_ERR_ARG, "null argument");
    for (unsigned i = 0; i < nsegs; i++) {
        if (idx[i + 1] < idx[i]) return fail(BGT_ERR_ARG, "idx is not ascending at segment %u", i);
        const size_t n = idx[i + 1] - idx[i];
        double *m = out + (size_t)dims * idx[i];
        for (size_t t = 0; t < n; t++) {
            const size_t p = idx[i] + t;
            m[t] = (double)y[p];
            m[n + t] = (double)x[p];
            if (dims == 3) m[2 * n + t] = (double)z[p];
        }
    }
    return BGT_OK;
}
