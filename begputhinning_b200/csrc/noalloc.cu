// noalloc.cu -- 2D thinning for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: plugins that run
// inside a host application which owns all device memory through its own
// pool (an allocation behind the pool's back can fail or fragment it), and
// real-time loops where an allocation's implicit device synchronisation
// would stall the frame.  For them,
// bgt_thin2d_device_noalloc thins one 2D image using only a fixed scratch
// array compiled into the library: a file-scope __device__ array of
// kNoAllocScratchBytes that every GPU which loads the library keeps until the
// process exits.  It allocates nothing (no cudaMalloc, no cudaFree, no
// allocating library call); the caller passes the device input and output.
//
// The work is the plain path: pack, then one launch per pass with a readback
// of the change flag after each pass (the call synchronises the stream once
// per pass), then unpack, all on the caller's stream.
#include <algorithm>
#include <cstring>
#include <mutex>

#include <cudaTypedefs.h>

#include "host.h"
#include "kernels.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr int kMaxDevices = 64;

// The scratch array.  Host code must not use this name as a device address:
// on the host it is only a stand-in; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_lock;
void *g_noalloc_ptr[kMaxDevices] = {};

size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Keeps the calling thread's current device across the call: callers without
// a context of their own rely on it staying where they put it.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { cudaGetDevice(&prev); }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

using namespace bgt;

// Thin a 2D image in device memory without allocating any device memory.
// dtype, d_in and d_out as for bgt_thin2d_device; stream is a cudaStream_t
// (NULL: the legacy default stream) of `device`, which is made current for
// the call; the caller's current device is restored on return.
//
// Limits and sharing: the packed image (two copies, 2*ceil(width/32 rounded
// up to 4)*height*4 bytes) plus small tables must fit in the 8 MiB array,
// e.g. any image up to 4096 x 4096; larger images are rejected with
// BGT_ERR_LIMIT before any device work.  All calls share the one array, which
// keeps the last call's contents; everything that must start cleared is
// cleared by the call itself.  The function holds a process-wide lock and
// returns only when its work on `stream` has finished, so calls from several
// host threads are serialised; work arranged so that two calls would overlap
// on the GPU would race on the shared array.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current.  Make that first call
// before starting any stream capture.
extern "C" int bgt_thin2d_device_noalloc(int device, int dtype, const void *d_in, int width, int height,
                                         void *d_out, void *stream)
{
    if (!d_in || !d_out) return fail(BGT_ERR_ARG, "null buffer");
    if (dtype_size(dtype) == 0) return fail(BGT_ERR_ARG, "bad dtype %d", dtype);
    if (width < 1 || height < 1 || width > 32767 || height > 32767)
        return fail(BGT_ERR_ARG, "size %dx%d out of range", width, height);
    if (device < 0 || device >= kMaxDevices) return fail(BGT_ERR_ARG, "bad device %d", device);

    // tile geometry as the batch uses it
    const int cfg = tuned_cfg(2, width, height, 1);
    const CfgInfo &c = *cfg_info(cfg);
    Inst in;
    memset(&in, 0, sizeof(in));
    in.dims = 2;
    in.W = width;
    in.H = height;
    in.D = 1;
    in.P = (int)up((size_t)(width + 31) / 32, 4);
    in.cfg = cfg;
    in.TW = c.TW;
    in.TH = c.TH;
    in.TZ = 1;
    in.k = c.k;
    in.window = (4 + c.k - 1) / c.k;
    in.tiles_x = ((width + 31) / 32 + c.TW - 1) / c.TW;
    in.tiles_y = (height + c.TH - 1) / c.TH;
    in.tiles_z = 1;
    in.ntiles = in.tiles_x * in.tiles_y;
    in.pass_cap = (std::max(width, height) + 16) * std::max(1, 4 / c.k) + 64;
    in.prio = 1;

    // scratch layout: Inst | 2 tensor maps | change flag, status word | lc | buf0 | buf1
    const size_t words = (size_t)in.P * height;
    const size_t o_inst = 0;
    const size_t o_tmap = up(o_inst + sizeof(Inst), 128);
    const size_t o_flag = up(o_tmap + 2 * sizeof(CUtensorMap), 256);
    const size_t o_lc = up(o_flag + 2 * sizeof(int), 256);
    const size_t o_b0 = up(o_lc + (size_t)in.ntiles * sizeof(int), 256);
    const size_t o_b1 = up(o_b0 + words * 4, 256);
    const size_t need = up(o_b1 + words * 4, 256);
    if (need > kNoAllocScratchBytes)
        return fail(BGT_ERR_LIMIT,
                    "image %dx%d needs %zu bytes of scratch; the no-allocation entry point has %zu bytes "
                    "(use bgt_thin2d_device for larger images)",
                    width, height, need, kNoAllocScratchBytes);

    std::lock_guard<std::mutex> lock(g_noalloc_lock);
    DeviceGuard keep_device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_noalloc_ptr[device] = p;
    }
    char *base = static_cast<char *>(g_noalloc_ptr[device]);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    Inst *d_inst = reinterpret_cast<Inst *>(base + o_inst);
    int *d_flag = reinterpret_cast<int *>(base + o_flag);
    int *d_status = d_flag + 1;
    in.lc = reinterpret_cast<int *>(base + o_lc);
    in.buf[0] = reinterpret_cast<uint32_t *>(base + o_b0);
    in.buf[1] = reinterpret_cast<uint32_t *>(base + o_b1);
    in.tmap = reinterpret_cast<const CUtensorMap *>(base + o_tmap);

    // tensor maps over the two packed buffers (host-side encoding, no allocation)
    void *enc_fn = nullptr;
    cudaDriverEntryPointQueryResult qres;
    e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &enc_fn, cudaEnableDefault, &qres);
    if (e != cudaSuccess || qres != cudaDriverEntryPointSuccess || !enc_fn)
        return fail(BGT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(enc_fn);
    CUtensorMap maps[2];
    for (int k = 0; k < 2; k++) {
        cuuint64_t dims[2] = {(cuuint64_t)in.P, (cuuint64_t)height};
        cuuint64_t strides[1] = {(cuuint64_t)in.P * 4};
        cuuint32_t box[2] = {(cuuint32_t)c.box[0], (cuuint32_t)c.box[1]};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = enc(&maps[k], CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, in.buf[k], dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(BGT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    }
    e = cudaMemcpyAsync(base + o_tmap, maps, sizeof(maps), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_inst, &in, sizeof(in), cudaMemcpyHostToDevice, st);
    // pack into both buffers; lc <- kNever then -1 on tiles holding foreground
    if (e == cudaSuccess)
        e = launch_pack(dtype, 0, d_in, width, height, 1, width, height, 1, in.P, in.buf[0], in.buf[1], st);
    if (e == cudaSuccess) e = launch_tile_init(d_inst, in, nullptr, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_status, 0, sizeof(int), st);
    // Once work is queued, every return waits for it first (still holding
    // the lock), so no kernel of this call can touch the shared array after
    // the next caller has taken it.
    auto fail_after_queue = [&](int rc) {
        cudaStreamSynchronize(st);
        return rc;
    };
    if (e != cudaSuccess) return fail_after_queue(cuda_fail(e, "no-allocation set-up"));

    int last_change = -1, converged = 0;
    for (int q = 0; q < in.pass_cap; q++) {
        int h_flag = 0;
        e = cudaMemsetAsync(d_flag, 0, sizeof(int), st);
        if (e == cudaSuccess) e = launch_plain_pass(cfg, d_inst, in.ntiles, q, d_flag, d_status, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail_after_queue(cuda_fail(e, "no-allocation pass"));
        if (h_flag) last_change = q;
        if (q - last_change >= in.window) {
            converged = 1;
            break;
        }
    }
    if (!converged) return fail_after_queue(fail(BGT_ERR_LIMIT, "hit the pass cap"));
    e = launch_unpack(dtype, in.buf[0], width, height, 1, in.P, d_out, st);
    int h_status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_after_queue(cuda_fail(e, "no-allocation unpack"));
    if (h_status) return fail(BGT_ERR_TIMEOUT, "a device wait gave up (status bits 0x%x)", h_status);
    return BGT_OK;
}
