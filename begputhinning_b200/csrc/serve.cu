// serve.cu -- a serving runtime over the batch engine: requests (2D frames,
// 3D volumes) arrive at any time from host threads; a dispatcher thread
// admits waiting requests into free device slots of their lane and launches
// them while earlier launches are still running, so work that arrives during
// a launch overlaps with it on the device (continuous batching at launch
// granularity); a completion thread stamps each request's latency when its
// output is back in host memory.
//
// Lanes: 0 = 2D frames on high-priority streams, 1 = 3D volumes on
// low-priority streams.  Each lane has a few slots (a stream, a context and
// a batch: launches of different slots overlap on the device).  Device
// memory is one arena of the HBM budget, allocated at creation and resident:
// every launch takes one block of it (staging for its requests' inputs and
// outputs plus its batch's pool, sized from the requests' shapes) and
// returns it when its outputs are back in host memory.  A request is
// admitted when a slot of its lane is free and the arena has room for the
// launch grown by it; until then it waits.  The lanes share the arena and
// borrow each other's idle memory, except that volumes leave a guard large
// enough for one launch of frames.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "host.h"

using namespace bgt;

namespace {

double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Req {
    unsigned long long ticket = 0;
    int dtype = 0, dims = 2, w = 0, h = 0, d = 1;
    const void *host_in = nullptr;
    void *host_out = nullptr;
    size_t bytes = 0;
    double t_submit = 0, t_done = 0;
    int status = 0;
};

// One slot = one stream (of the lane's priority), a context bound to it and
// a batch laid out in the launch's arena block: slots overlap on the device.
struct Slot {
    bgt_ctx *ctx = nullptr;
    cudaStream_t stream = nullptr;
    bgt_batch *b = nullptr;
    size_t blk_off = 0, blk_len = 0;  // arena block of the launch in flight (staging, then pool)
    cudaEvent_t done = nullptr;
    bool busy = false;      // holds admitted requests
    bool launched = false;  // its work (ending with `done`) is enqueued
    int cfg = -1;           // tile configuration of the lane (-1: tuned / default)
    std::vector<Req *> reqs;
};

struct Lane {
    int dims = 2;
    std::vector<Slot> slots;
    std::deque<Req *> pending;
    int max_batch = 16;
    size_t cap = 0;   // arena bytes the lane may hold at once
    size_t used = 0;  // arena bytes its launches hold now
    std::vector<double> lat_ms;
    unsigned long long done = 0;
    double voxels = 0;
    double t_first = 0, t_last = 0;
};

// First-fit allocator over the arena, coalescing on release.
struct Arena {
    char *base = nullptr;
    size_t size = 0, used = 0;
    std::map<size_t, size_t> free;  // offset -> length
    size_t largest() const
    {
        size_t m = 0;
        for (auto &kv : free) m = std::max(m, kv.second);
        return m;
    }
    bool alloc(size_t n, size_t *off)
    {
        for (auto it = free.begin(); it != free.end(); ++it) {
            if (it->second < n) continue;
            *off = it->first;
            const size_t rest = it->second - n, at = it->first + n;
            free.erase(it);
            if (rest) free[at] = rest;
            used += n;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t n)
    {
        used -= n;
        auto it = free.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free.erase(nx);
        }
        if (it != free.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free.erase(it);
            }
        }
    }
};

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

// Host<->device copy in pieces of at most 4 MB, so that the copies of other
// slots (frames on high-priority streams) interleave with a large volume's
// instead of queueing behind all of it.
cudaError_t copy_pieces(void *dst, const void *src, size_t n, cudaMemcpyKind kind, cudaStream_t st)
{
    constexpr size_t kPiece = size_t(4) << 20;
    cudaError_t e = cudaSuccess;
    for (size_t o = 0; o < n && e == cudaSuccess; o += kPiece)
        e = cudaMemcpyAsync(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, std::min(kPiece, n - o),
                            kind, st);
    return e;
}

// Arena bytes of one launch of these requests: staging (inputs and
// outputs) plus the batch pool their shapes need.
size_t launch_bytes(const std::vector<Req *> &reqs, int cfg)
{
    size_t staging = 0;
    std::vector<BatchItem> items;
    for (const Req *r : reqs) {
        staging += 2 * up256(r->bytes);
        BatchItem it;
        it.dims = r->dims;
        it.W = r->w;
        it.H = r->h;
        it.D = r->d;
        it.cfg = cfg;
        it.auto_cfg = cfg < 0;
        items.push_back(it);
    }
    return staging + up256(batch_pool_bytes(items)) + 256;
}

}  // namespace

struct bgt_server {
    int device = 0;
    size_t budget = 0;
    Arena arena;
    std::mutex mu;
    std::condition_variable cv;
    Lane lane[2];
    std::thread dispatcher, completer;
    bool stop = false;
    unsigned long long next_ticket = 1;
    std::unordered_map<unsigned long long, Req *> live;
    std::vector<Req *> completed;  // not yet polled
    unsigned long long in_flight = 0;
    int fatal = 0;
};

namespace {

// Launch the requests now held by `s` in its arena block (called without
// the server lock).
int launch_slot(bgt_server *S, Slot &s)
{
    bgt_batch *b = s.b;
    int rc = bgt_batch_reset(b);
    char *blk = S->arena.base + s.blk_off;
    size_t off = 0;
    std::vector<size_t> in_off(s.reqs.size()), out_off(s.reqs.size());
    for (size_t i = 0; i < s.reqs.size(); i++) {
        in_off[i] = off;
        off += up256(s.reqs[i]->bytes);
    }
    for (size_t i = 0; i < s.reqs.size(); i++) {
        out_off[i] = off;
        off += up256(s.reqs[i]->bytes);
    }
    if (rc == BGT_OK) rc = batch_use_pool(b, blk + off, s.blk_len - off);
    if (rc != BGT_OK) return rc;
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < s.reqs.size() && e == cudaSuccess; i++)
        e = copy_pieces(blk + in_off[i], s.reqs[i]->host_in, s.reqs[i]->bytes, cudaMemcpyHostToDevice, s.stream);
    if (e != cudaSuccess) return cuda_fail(e, "serve H2D");
    for (size_t i = 0; i < s.reqs.size() && rc == BGT_OK; i++) {
        const Req *r = s.reqs[i];
        rc = r->dims == 2 ? bgt_batch_add2d(b, r->w, r->h, s.cfg, nullptr)
                          : bgt_batch_add3d(b, r->w, r->h, r->d, s.cfg, nullptr);
    }
    if (rc == BGT_OK) rc = bgt_batch_finalize(b);
    for (size_t i = 0; i < s.reqs.size() && rc == BGT_OK; i++)
        rc = bgt_batch_set_io(b, (int)i, s.reqs[i]->dtype, blk + in_off[i], blk + out_off[i]);
    if (rc == BGT_OK) rc = bgt_batch_run(b, 0, 0);
    if (rc != BGT_OK) return rc;
    for (size_t i = 0; i < s.reqs.size() && e == cudaSuccess; i++)
        e = copy_pieces(s.reqs[i]->host_out, blk + out_off[i], s.reqs[i]->bytes, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(s.done, s.stream);
    if (e != cudaSuccess) return cuda_fail(e, "serve D2H");
    (void)S;
    return BGT_OK;
}

void dispatcher_loop(bgt_server *S)
{
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop) {
        bool launched = false;
        for (int li = 0; li < 2; li++) {
            Lane &L = S->lane[li];
            // frames first: no volume is admitted while a frame waits
            if (li == 1 && !S->lane[0].pending.empty()) continue;
            for (Slot &s : L.slots) {
                if (s.busy || L.pending.empty()) continue;
                // admit from the front while the lane's share and the arena
                // have room for the launch grown by the next request
                size_t need = 0;
                const size_t room = std::min(L.cap - std::min(L.cap, L.used), S->arena.largest());
                while (!L.pending.empty() && (int)s.reqs.size() < L.max_batch) {
                    s.reqs.push_back(L.pending.front());
                    const size_t n = launch_bytes(s.reqs, s.cfg);
                    if (n > room) {
                        s.reqs.pop_back();
                        break;
                    }
                    need = n;
                    L.pending.pop_front();
                }
                if (s.reqs.empty()) continue;
                if (!S->arena.alloc(need, &s.blk_off)) {  // not reached: need <= the largest free block
                    for (auto it = s.reqs.rbegin(); it != s.reqs.rend(); ++it) L.pending.push_front(*it);
                    s.reqs.clear();
                    continue;
                }
                s.blk_len = need;
                L.used += need;
                s.busy = true;
                S->in_flight += s.reqs.size();
                lk.unlock();
                int rc = launch_slot(S, s);
                lk.lock();
                if (rc == BGT_OK) s.launched = true;
                if (rc != BGT_OK) {
                    // the slot's requests fail; the slot and its block are free again
                    cudaStreamSynchronize(s.stream);
                    S->arena.release(s.blk_off, s.blk_len);
                    L.used -= s.blk_len;
                    const double t = now_ms();
                    for (Req *r : s.reqs) {
                        r->status = rc;
                        r->t_done = t;
                        S->completed.push_back(r);
                    }
                    S->in_flight -= s.reqs.size();
                    s.reqs.clear();
                    s.busy = false;
                    S->cv.notify_all();
                }
                launched = true;
            }
        }
        if (!launched) S->cv.wait_for(lk, std::chrono::microseconds(200));
    }
}

void completer_loop(bgt_server *S)
{
    cudaSetDevice(S->device);
    for (;;) {
        bool any = false;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->stop) return;
        }
        for (int li = 0; li < 2; li++) {
            Lane &L = S->lane[li];
            for (Slot &s : L.slots) {
                bool busy;
                {
                    std::lock_guard<std::mutex> lk(S->mu);
                    busy = s.busy && s.launched;
                }
                if (!busy) continue;
                const cudaError_t q = cudaEventQuery(s.done);
                if (q == cudaErrorNotReady) continue;
                const double t = now_ms();
                std::lock_guard<std::mutex> lk(S->mu);
                if (!s.busy) continue;
                for (Req *r : s.reqs) {
                    r->t_done = t;
                    r->status = q == cudaSuccess ? BGT_OK : BGT_ERR_CUDA;
                    if (q == cudaSuccess) {
                        L.lat_ms.push_back(t - r->t_submit);
                        L.voxels += (double)r->w * r->h * r->d;
                        L.done++;
                        if (L.t_first == 0) L.t_first = r->t_submit;
                        L.t_last = t;
                    }
                    S->completed.push_back(r);
                }
                S->in_flight -= s.reqs.size();
                s.reqs.clear();
                S->arena.release(s.blk_off, s.blk_len);
                L.used -= s.blk_len;
                s.busy = false;
                s.launched = false;
                any = true;
                S->cv.notify_all();
            }
        }
        if (!any) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

int setup_lane(bgt_server *S, int li, int dims, int priority, int nslots, int max_batch, size_t cap, int grid_cap,
               int cfg)
{
    Lane &L = S->lane[li];
    L.dims = dims;
    L.max_batch = max_batch;
    L.cap = cap;
    L.slots.resize(nslots);
    for (Slot &s : L.slots) {
        s.cfg = cfg;
        int rc = bgt_ctx_create(S->device, &s.ctx);
        if (rc != BGT_OK) return rc;
        cudaError_t e = cudaStreamCreateWithPriority(&s.stream, cudaStreamNonBlocking, priority);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreateWithPriority");
        bgt_ctx_set_stream(s.ctx, s.stream);
        if ((rc = bgt_batch_create(s.ctx, &s.b)) != BGT_OK) return rc;
        bgt_batch_set_grid(s.b, grid_cap);
        // tile rings: the lanes share the SMs with one another, which the
        // resident kernel (one 225 KB CTA on every SM at once) cannot
        bgt_batch_set_engine(s.b, 1);
        e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
    }
    return BGT_OK;
}

void teardown(bgt_server *S)
{
    for (Lane &L : S->lane) {
        for (Slot &s : L.slots) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            if (s.b) bgt_batch_destroy(s.b);
            if (s.done) cudaEventDestroy(s.done);
            if (s.ctx) bgt_ctx_destroy(s.ctx);
            if (s.stream) cudaStreamDestroy(s.stream);
        }
        L.slots.clear();
    }
    if (S->arena.base) cudaFree(S->arena.base);
    S->arena = Arena();
    // every request not yet returned by a poll is still in `live`
    for (auto &kv : S->live) delete kv.second;
    S->live.clear();
    S->completed.clear();
}

}  // namespace

// Lane 0 serves 2D requests, up to 16 per launch; lane 1 serves 3D requests,
// up to 2 per launch.  The arena (hbm_budget_bytes) is allocated here.
extern "C" int bgt_server_create(int device, size_t hbm_budget_bytes, bgt_server **out)
{
    if (!out) return fail(BGT_ERR_ARG, "null out");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    bgt_server *S = new bgt_server();
    S->device = device;
    S->budget = hbm_budget_bytes;
    const size_t MiB = size_t(1) << 20;
    e = cudaMalloc(&S->arena.base, hbm_budget_bytes);
    if (e != cudaSuccess) {
        delete S;
        return cuda_fail(e, "cudaMalloc(serving arena)");
    }
    S->arena.size = hbm_budget_bytes;
    S->arena.free[0] = hbm_budget_bytes;
    // volumes leave room for one launch of 16 megapixel frames
    const size_t guard = std::min(hbm_budget_bytes / 4, size_t(64) * MiB);
    // frames: two slots with one CTA per SM each
    int rc = setup_lane(S, 0, 2, hi, 2, 16, hbm_budget_bytes, sms, -1);
    // volumes: two slots of at most two volumes each, with one CTA per SM,
    // so frames always find room on every SM and volume launches stay short
    // (measured at 70 % volume requests: frame p99 3.9 ms with three slots of
    // four, 1.8 ms with two of two).  Volumes use 16-plane tiles: the least
    // total work per pass (fewest halo planes), which is what a throughput
    // lane sharing the GPU with latency-bound frames wants
    if (rc == BGT_OK) rc = setup_lane(S, 1, 3, lo, 2, 2, hbm_budget_bytes - guard, sms, 17);
    if (rc != BGT_OK) {
        teardown(S);
        delete S;
        return rc;
    }
    S->dispatcher = std::thread(dispatcher_loop, S);
    S->completer = std::thread(completer_loop, S);
    *out = S;
    return BGT_OK;
}

// Submit one request (host buffers; pinned host memory keeps the copies
// asynchronous).  The buffers must stay valid until the request completes.
extern "C" int bgt_server_submit(bgt_server *S, int dtype, const void *host_in, int w, int h, int d, void *host_out,
                                 unsigned long long *ticket)
{
    if (!S || !host_in || !host_out || !ticket) return fail(BGT_ERR_ARG, "null argument");
    const size_t es = dtype_size(dtype);
    if (!es || w < 1 || h < 1 || d < 1) return fail(BGT_ERR_ARG, "bad dtype or size");
    Req *r = new Req();
    r->dtype = dtype;
    r->dims = d > 1 ? 3 : 2;
    r->w = w;
    r->h = h;
    r->d = d;
    r->host_in = host_in;
    r->host_out = host_out;
    r->bytes = es * (size_t)w * h * d;
    r->t_submit = now_ms();
    Lane &L = S->lane[r->dims == 2 ? 0 : 1];
    const size_t need = launch_bytes(std::vector<Req *>{r}, L.slots[0].cfg);
    if (need > L.cap) {
        delete r;
        return fail(BGT_ERR_LIMIT, "request needs %zu bytes of device memory; its lane may hold %zu", need, L.cap);
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        r->ticket = S->next_ticket++;
        S->live[r->ticket] = r;
        L.pending.push_back(r);
        *ticket = r->ticket;
    }
    S->cv.notify_all();
    return BGT_OK;
}

// Completed requests since the last poll: ticket, latency (submit to output
// in host memory, ms) and status.
extern "C" int bgt_server_poll(bgt_server *S, unsigned long long *tickets, double *latency_ms, int *status, int cap,
                               int *n)
{
    if (!S || !n) return fail(BGT_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    int k = 0;
    while (k < cap && !S->completed.empty()) {
        Req *r = S->completed.back();
        S->completed.pop_back();
        if (tickets) tickets[k] = r->ticket;
        if (latency_ms) latency_ms[k] = r->t_done - r->t_submit;
        if (status) status[k] = r->status;
        S->live.erase(r->ticket);
        delete r;
        k++;
    }
    *n = k;
    return BGT_OK;
}

// Wait until every submitted request has completed (or timeout_s passed).
extern "C" int bgt_server_drain(bgt_server *S, double timeout_s)
{
    if (!S) return fail(BGT_ERR_ARG, "null server");
    const double t_end = now_ms() + timeout_s * 1e3;
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            bool idle = S->in_flight == 0 && S->lane[0].pending.empty() && S->lane[1].pending.empty();
            if (idle) return BGT_OK;
        }
        if (now_ms() > t_end) return fail(BGT_ERR_TIMEOUT, "server drain timed out");
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

// Latency percentiles of completed requests of a lane (0 frames, 1 volumes)
// and its throughput in Mvoxel/s (first submit to last completion).
extern "C" int bgt_server_stats(bgt_server *S, int lane, double *p50_ms, double *p99_ms, double *mvox_per_s,
                                unsigned long long *completed)
{
    if (!S || lane < 0 || lane > 1) return fail(BGT_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> lk(S->mu);
    Lane &L = S->lane[lane];
    std::vector<double> v = L.lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
        if (v.empty()) return 0.0;
        size_t i = (size_t)std::min<double>(v.size() - 1, std::ceil(p * v.size()) - 1);
        return v[i];
    };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (mvox_per_s) *mvox_per_s = L.t_last > L.t_first ? L.voxels / ((L.t_last - L.t_first) * 1e-3) / 1e6 : 0.0;
    if (completed) *completed = L.done;
    return BGT_OK;
}

// Device memory of the server: arena bytes held by launches in flight, the
// arena's size, and requests waiting for admission (both lanes).
extern "C" int bgt_server_memory(bgt_server *S, size_t *used, size_t *budget, unsigned long long *waiting)
{
    if (!S) return fail(BGT_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    if (used) *used = S->arena.used;
    if (budget) *budget = S->arena.size;
    if (waiting) *waiting = S->lane[0].pending.size() + S->lane[1].pending.size();
    return BGT_OK;
}

extern "C" int bgt_server_reset_stats(bgt_server *S)
{
    if (!S) return fail(BGT_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    for (Lane &L : S->lane) {
        L.lat_ms.clear();
        L.done = 0;
        L.voxels = 0;
        L.t_first = L.t_last = 0;
    }
    return BGT_OK;
}

extern "C" int bgt_server_destroy(bgt_server *S)
{
    if (!S) return BGT_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv.notify_all();
    if (S->dispatcher.joinable()) S->dispatcher.join();
    if (S->completer.joinable()) S->completer.join();
    cudaSetDevice(S->device);
    teardown(S);
    delete S;
    return BGT_OK;
}
