// kernels.cu -- pack/unpack, the plain one-launch-per-pass thinning kernels
// and the persistent batched engine (device work ring of (instance, tile,
// pass) items with per-instance convergence).
#include <algorithm>
#include <cstdio>

#include "kernels.cuh"
#include "tiles.cuh"

namespace bgt {

// ------------------------------------------------------------ configs -----
using C2_1_12 = Cfg2D<1, 12, 4>;
using C2_2_12 = Cfg2D<2, 12, 4>;
using C2_4_12 = Cfg2D<4, 12, 4>;
using C2_8_12 = Cfg2D<8, 12, 4>;
using C2_1_28 = Cfg2D<1, 28, 4>;
using C2_2_28 = Cfg2D<2, 28, 4>;
using C2_4_28 = Cfg2D<4, 28, 4>;
using C2_8_28 = Cfg2D<8, 28, 4>;
using C3_8 = Cfg3D<4, 8>;
using C3_16 = Cfg3D<4, 16>;
using C3_32 = Cfg3D<4, 32>;

template <class C>
constexpr CfgInfo info2d(int id)
{
    return CfgInfo{id, 2, C::kK, C::kS, C::kNW, 0, 1, C::kS, C::TH, 1, C::SMEM, {C::BW, C::BH, 1}};
}
template <class C>
constexpr CfgInfo info3d(int id)
{
    return CfgInfo{id, 3, 1, 0, 0, C::kNWX, C::kTZ, C::kNWX, C::TY, C::kTZ, C::SMEM, {C::BW, C::BH, C::BD}};
}

static const CfgInfo kCfgs[] = {
    info2d<C2_1_12>(0), info2d<C2_2_12>(1), info2d<C2_4_12>(2), info2d<C2_8_12>(3),
    info2d<C2_1_28>(4), info2d<C2_2_28>(5), info2d<C2_4_28>(6), info2d<C2_8_28>(7),
    info3d<C3_8>(16),   info3d<C3_16>(17),  info3d<C3_32>(18),
};
static const int kIds2d[] = {0, 1, 2, 3, 4, 5, 6, 7};
static const int kIds3d[] = {16, 17, 18};

const CfgInfo *cfg_info(int id)
{
    for (const auto &c : kCfgs)
        if (c.id == id) return &c;
    return nullptr;
}
const int *cfg_ids_2d(int *n) { *n = 8; return kIds2d; }
const int *cfg_ids_3d(int *n) { *n = 3; return kIds3d; }

constexpr int kThreads = 128;

// Run one tile of instance `in` at pass q with the instance's configuration.
__device__ bool run_tile(const Inst &in, int q, int tile, uint32_t *smem, uint64_t *bar, uint32_t &parity,
                         int *err)
{
    switch (in.cfg) {
#define CASE2_K1(ID, C)                                                          \
    case ID:                                                                     \
        switch (q & 3) {                                                         \
        case 0: return tile2d<C, 0>(in, q, tile, smem, bar, parity, err);       \
        case 1: return tile2d<C, 1>(in, q, tile, smem, bar, parity, err);       \
        case 2: return tile2d<C, 2>(in, q, tile, smem, bar, parity, err);       \
        default: return tile2d<C, 3>(in, q, tile, smem, bar, parity, err);      \
        }
#define CASE2_K2(ID, C)                                                          \
    case ID:                                                                     \
        if (q & 1) return tile2d<C, 2>(in, q, tile, smem, bar, parity, err);    \
        return tile2d<C, 0>(in, q, tile, smem, bar, parity, err);
#define CASE2_K4(ID, C) \
    case ID: return tile2d<C, 0>(in, q, tile, smem, bar, parity, err);
#define CASE3(ID, C)                                                             \
    case ID:                                                                     \
        switch (q % 6) {                                                         \
        case 0: return tile3d<C, 0>(in, q, tile, smem, bar, parity, err);       \
        case 1: return tile3d<C, 1>(in, q, tile, smem, bar, parity, err);       \
        case 2: return tile3d<C, 2>(in, q, tile, smem, bar, parity, err);       \
        case 3: return tile3d<C, 3>(in, q, tile, smem, bar, parity, err);       \
        case 4: return tile3d<C, 4>(in, q, tile, smem, bar, parity, err);       \
        default: return tile3d<C, 5>(in, q, tile, smem, bar, parity, err);      \
        }
        CASE2_K1(0, C2_1_12)
        CASE2_K2(1, C2_2_12)
        CASE2_K4(2, C2_4_12)
        CASE2_K4(3, C2_8_12)
        CASE2_K1(4, C2_1_28)
        CASE2_K2(5, C2_2_28)
        CASE2_K4(6, C2_4_28)
        CASE2_K4(7, C2_8_28)
        CASE3(16, C3_8)
        CASE3(17, C3_16)
        CASE3(18, C3_32)
#undef CASE2_K1
#undef CASE2_K2
#undef CASE2_K4
#undef CASE3
    default:
        return false;
    }
}

// ------------------------------------------------------------ pack --------
// Foreground tests of the reference's binarisation.  2D: (unsigned int)v > 0
// evaluated on the device (2D/CUDA_DeviceHelperFunctions.cuh:101), i.e. a
// saturating conversion for floating types.  3D: int(v) > 0 as the host
// evaluates it (3D/CenterlineExtraction.cpp:44; x86-64 conversion of
// out-of-range floats gives INT_MIN).
template <typename T>
__device__ __forceinline__ bool fg2(T v) { return (unsigned int)v > 0u; }
template <>
__device__ __forceinline__ bool fg2<bool>(bool v) { return v; }

template <typename T>
__device__ __forceinline__ bool fg3(T v) { return (int)v > 0; }
template <>
__device__ __forceinline__ bool fg3<float>(float v) { return v >= 1.0f && v < 2147483648.0f; }
template <>
__device__ __forceinline__ bool fg3<double>(double v) { return v >= 1.0 && v < 2147483648.0; }
template <>
__device__ __forceinline__ bool fg3<bool>(bool v) { return v; }

// One thread per packed word; writes both ping-pong buffers (so tiles that
// never change hold identical data in both).  The input may be smaller than
// the instance (inW x inH x inD inside W x H x D, row stride inW); the rest
// packs as background.  MODE 0: 2D thinning rule, 1: 3D rule, 2: nonzero.
template <typename T, int MODE>
__global__ void pack_kernel(const T *__restrict__ in, int inW, int inH, int inD, int W, int H, int D, int P,
                            uint32_t *buf0, uint32_t *buf1)
{
    const long long rows = (long long)H * D;
    const long long nw = rows * P;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / P;
        const int j = (int)(i - row * P);
        const int y = (int)(row % H), z = (int)(row / H);
        const int x0 = j * 32;
        uint32_t w = 0;
        if (x0 < inW && y < inH && z < inD) {
            const T *p = in + ((long long)z * inH + y) * (long long)inW + x0;
            const int n = min(32, inW - x0);
            for (int b = 0; b < n; b++) {
                const T v = p[b];
                const bool f = MODE == 0 ? fg2<T>(v) : MODE == 1 ? fg3<T>(v) : (v != (T)0);
                w |= (uint32_t)f << b;
            }
        }
        buf0[i] = w;
        if (buf1) buf1[i] = w;
    }
}

template <typename T>
__global__ void unpack_kernel(const uint32_t *__restrict__ buf, int W, int H, int D, int P, T *out)
{
    const long long rows = (long long)H * D;
    const int groups = (W + 3) / 4;  // 4 pixels per thread
    const long long n = rows * groups;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / groups;
        const int x = (int)(i - row * groups) * 4;
        const uint32_t w = __ldg(buf + row * P + (x >> 5));
        T *o = out + row * (long long)W + x;
        const int m = min(4, W - x);
        for (int b = 0; b < m; b++) o[b] = (T)((w >> ((x + b) & 31)) & 1u);
    }
}

static int grid_for(long long n, int block)
{
    long long g = (n + block - 1) / block;
    return (int)std::max(1LL, std::min(g, 148LL * 32));
}

template <typename T>
static cudaError_t pack_t(int mode, const void *in, int inW, int inH, int inD, int W, int H, int D, int P,
                          uint32_t *b0, uint32_t *b1, cudaStream_t st)
{
    const long long nw = (long long)H * D * P;
    const int g = grid_for(nw, 256);
    if (mode == 0)
        pack_kernel<T, 0><<<g, 256, 0, st>>>((const T *)in, inW, inH, inD, W, H, D, P, b0, b1);
    else if (mode == 1)
        pack_kernel<T, 1><<<g, 256, 0, st>>>((const T *)in, inW, inH, inD, W, H, D, P, b0, b1);
    else
        pack_kernel<T, 2><<<g, 256, 0, st>>>((const T *)in, inW, inH, inD, W, H, D, P, b0, b1);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t unpack_t(const uint32_t *buf, int W, int H, int D, int P, void *out, cudaStream_t st)
{
    const long long n = (long long)H * D * ((W + 3) / 4);
    unpack_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(buf, W, H, D, P, (T *)out);
    return cudaGetLastError();
}

#define BGT_DISPATCH_DTYPE(dtype, FN, ...)                         \
    switch (dtype) {                                               \
    case BGT_U8: return FN<uint8_t>(__VA_ARGS__);                  \
    case BGT_I8: return FN<int8_t>(__VA_ARGS__);                   \
    case BGT_CHAR: return FN<char>(__VA_ARGS__);                   \
    case BGT_U16: return FN<uint16_t>(__VA_ARGS__);                \
    case BGT_I16: return FN<int16_t>(__VA_ARGS__);                 \
    case BGT_U32: return FN<uint32_t>(__VA_ARGS__);                \
    case BGT_I32: return FN<int32_t>(__VA_ARGS__);                 \
    case BGT_F32: return FN<float>(__VA_ARGS__);                   \
    case BGT_F64: return FN<double>(__VA_ARGS__);                  \
    case BGT_BOOL: return FN<bool>(__VA_ARGS__);                   \
    default: return cudaErrorInvalidValue;                         \
    }

cudaError_t launch_pack(int dtype, int mode, const void *in, int inW, int inH, int inD, int W, int H, int D, int P,
                        uint32_t *buf0, uint32_t *buf1, cudaStream_t st)
{
    BGT_DISPATCH_DTYPE(dtype, pack_t, mode, in, inW, inH, inD, W, H, D, P, buf0, buf1, st)
}

cudaError_t launch_unpack(int dtype, const uint32_t *buf, int W, int H, int D, int P, void *out,
                          cudaStream_t st)
{
    BGT_DISPATCH_DTYPE(dtype, unpack_t, buf, W, H, D, P, out, st)
}

// --------------------------------------------------------- tile marks -----
// lc[t] = -1 for tiles whose core holds foreground (lc pre-filled with kNever).
__global__ void tile_mark_kernel(const Inst *__restrict__ pin)
{
    const Inst &in = *pin;
    const long long rows = (long long)in.H * in.D;
    const int wwords = (in.W + 31) >> 5;
    const long long nw = rows * wwords;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / wwords;
        const int j = (int)(i - row * wwords);
        if (in.buf[0][row * in.P + j] == 0u) continue;
        const int y = (int)(row % in.H), z = (int)(row / in.H);
        const int t = ((z / in.TZ) * in.tiles_y + y / in.TH) * in.tiles_x + j / in.TW;
        in.lc[t] = -1;
    }
}

cudaError_t launch_tile_init(const Inst *d_inst, const Inst &h, int *d_count, cudaStream_t st)
{
    (void)d_count;
    cudaError_t e = cudaMemsetAsync(h.lc, 0x80, sizeof(int) * (size_t)h.ntiles, st);
    if (e != cudaSuccess) return e;
    const long long nw = (long long)h.H * h.D * ((h.W + 31) / 32);
    tile_mark_kernel<<<grid_for(nw, 256), 256, 0, st>>>(d_inst);
    return cudaGetLastError();
}

// ---------------------------------------------------------- plain pass ----
// One launch per pass over every tile of one instance; each CTA decides its
// own activity.  *flag is set when any tile changed.
// TMA destinations are aligned to 128 bytes inside the dynamic allocation
// (which is requested 128 bytes larger than the tile box).
__device__ __forceinline__ uint32_t *align128(uint32_t *p)
{
    return reinterpret_cast<uint32_t *>((reinterpret_cast<uintptr_t>(p) + 127) & ~uintptr_t(127));
}

__global__ void __launch_bounds__(kThreads) plain_pass_kernel(Inst *pin, int q, int *flag, int *err)
{
    extern __shared__ __align__(128) uint32_t smem_raw[];
    uint32_t *smem = align128(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    __shared__ int active;
    const Inst &in = *pin;
    const int tile = blockIdx.x;
    if (threadIdx.x == 0) {
        bool a;
        if (in.dims == 3 && q % 6 != 0) {
            a = in.act[tile] != 0;
        } else {
            a = tile_active(in, tile, q);
            if (in.dims == 3) in.act[tile] = a ? 1 : 0;
        }
        active = a;
        if (a) {
            mbar_init(&bar, 1);
            fence_mbar_init();
        }
    }
    __syncthreads();
    if (!active) return;
    uint32_t parity = 0;
    const bool ch = run_tile(in, q, tile, smem, &bar, parity, err);
    if (threadIdx.x == 0 && ch) {
        in.lc[tile] = q;
        atomicExch(flag, 1);
    }
}

cudaError_t launch_plain_pass(int cfg, Inst *d_inst, int ntiles, int q, int *d_flag, int *d_err,
                              cudaStream_t st)
{
    const CfgInfo *c = cfg_info(cfg);
    if (!c) return cudaErrorInvalidValue;
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(plain_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_done = true;
    }
    plain_pass_kernel<<<ntiles, kThreads, c->smem + 128, st>>>(d_inst, q, d_flag, d_err);
    return cudaGetLastError();
}

// ------------------------------------------------------------- engine -----
// Work ring: Vyukov-style bounded MPMC queue.  seq[s] == t   : slot free for
// ticket t (producer may write); seq[s] == t+1 : item of ticket t ready;
// the consumer of ticket t then sets seq[s] = t + cap.

__device__ __forceinline__ unsigned ld_acq_u(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_rel_u(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Publish n items (instance ii, tiles list[0..n), pass q); whole CTA calls.
__device__ void produce(Sched *S, int ii, const int *list, int n, int q)
{
    __shared__ unsigned t0;
    if (threadIdx.x == 0) t0 = atomicAdd(&S->tail, (unsigned)n);
    __syncthreads();
    const unsigned cap = S->cap;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned t = t0 + (unsigned)i;
        const unsigned s = t % cap;
        const unsigned long long t_end = globaltimer() + (unsigned long long)S->timeout_ns;
        bool ok = false;
        for (int spin = 0;; spin++) {
            if (ld_acq_u(S->seq + s) == t) { ok = true; break; }
            if ((spin & 255) == 255 && globaltimer() > t_end) break;
            __nanosleep(64);
        }
        if (!ok) {
            atomicOr(&S->status, kErrQueueFull);
            continue;
        }
        S->item[s] = make_int4(ii, __ldcg(list + i), q, 0);
        st_rel_u(S->seq + s, t + 1);
    }
    __syncthreads();
}

// Build the active list for pass q1 of instance ii and publish it (or retire
// the instance).  Whole CTA calls.  Returns nothing; updates S->live.
__device__ void next_wave(Sched *S, Inst *insts, int ii, int q1)
{
    Inst &in = insts[ii];
    __shared__ int cnt;
    const bool recompute = in.dims == 2 || q1 % 6 == 0;
    if (threadIdx.x == 0) cnt = recompute ? 0 : __ldcg(&in.nlist);
    __syncthreads();
    if (recompute) {
        for (int t = threadIdx.x; t < in.ntiles; t += blockDim.x) {
            if (tile_active(in, t, q1)) {
                const int p = atomicAdd(&cnt, 1);
                in.list[p] = t;
            }
        }
    }
    __syncthreads();
    const int n = cnt;
    if (threadIdx.x == 0) {
        in.passes_run = q1;
        bool retire = n == 0;
        if (!retire && q1 >= in.pass_cap) {
            atomicOr(&S->status, kErrPassLimit);
            retire = true;
        }
        if (retire) {
            in.converged = n == 0 ? 1 : -1;
            in.nlist = 0;
        } else {
            in.pass = q1;
            in.nlist = n;
            in.done = 0;
        }
        __threadfence();
        if (retire) atomicSub(&S->live, 1);
        cnt = retire ? 0 : n;
    }
    __syncthreads();
    if (cnt > 0) {
        __threadfence();
        produce(S, ii, in.list, cnt, q1);
    }
}

// One CTA per instance: first wave (pass 0) after the tile marks.
__global__ void __launch_bounds__(kThreads) engine_seed_kernel(Inst *insts, int ninst, Sched *S)
{
    for (int ii = blockIdx.x; ii < ninst; ii += gridDim.x) {
        if (threadIdx.x == 0) {
            insts[ii].converged = 0;
            insts[ii].passes_run = 0;
            atomicAdd(&S->live, 1);
        }
        __syncthreads();
        next_wave(S, insts, ii, 0);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) engine_kernel(Inst *insts, Sched *S)
{
    extern __shared__ __align__(128) uint32_t smem_raw[];
    uint32_t *smem = align128(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    __shared__ int4 item;
    __shared__ int got, last;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t parity = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(&S->head, 1u);
            const unsigned s = t % S->cap;
            const unsigned long long t_end = globaltimer() + (unsigned long long)S->timeout_ns;
            int g = 0;
            for (int spin = 0;; spin++) {
                if (ld_acq_u(S->seq + s) == t + 1) {
                    item = __ldcg(S->item + s);
                    st_rel_u(S->seq + s, t + S->cap);
                    g = 1;
                    break;
                }
                if (ld_acquire(&S->live) == 0) break;
                if ((spin & 255) == 255 && globaltimer() > t_end) {
                    atomicOr(&S->status, kErrQueueTimeout);
                    break;
                }
                __nanosleep(spin < 64 ? 32 : 256);
            }
            got = g;
        }
        __syncthreads();
        if (!got) break;
        const int ii = item.x, tile = item.y, q = item.z;
        Inst &in = insts[ii];
        fence_proxy_async_global();
        const bool ch = run_tile(in, q, tile, smem, &bar, parity, &S->status);
        if (threadIdx.x == 0) {
            if (ch) in.lc[tile] = q;
            __threadfence();
            const int d = atomicAdd(&in.done, 1);
            last = d == __ldcg(&in.nlist) - 1;
        }
        __syncthreads();
        if (last) {
            __threadfence();
            next_wave(S, insts, ii, q + 1);
        }
        __syncthreads();
    }
}

int engine_max_blocks_per_sm(int smem)
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel, kThreads, smem + 128);
    return n;
}

cudaError_t engine_set_smem(int smem)
{
    cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem + 128);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(plain_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem + 128);
}

cudaError_t launch_engine(int grid, int smem, Inst *d_insts, int ninst, Sched *d_sched, cudaStream_t st)
{
    engine_seed_kernel<<<std::min(ninst, 148 * 8), kThreads, 0, st>>>(d_insts, ninst, d_sched);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    engine_kernel<<<grid, kThreads, smem + 128, st>>>(d_insts, d_sched);
    return cudaGetLastError();
}

}  // namespace bgt
