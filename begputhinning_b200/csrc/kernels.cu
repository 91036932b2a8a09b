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
using X2_4_12 = Cfg2DX<4, 12, 4>;
using X2_8_12 = Cfg2DX<8, 12, 4>;
using X2_16_12 = Cfg2DX<16, 12, 4>;
using X2_4_28 = Cfg2DX<4, 28, 4>;
using X2_8_28 = Cfg2DX<8, 28, 4>;
using C3_8 = Cfg3D<4, 8>;
using C3_16 = Cfg3D<4, 16>;
using C3_4 = Cfg3D<4, 4>;

template <class C>
constexpr CfgInfo info2d(int id)
{
    return CfgInfo{id, 2, C::kK, C::kS, C::kNW, 0, 1, C::kS, C::TH, 1, C::SMEM, {C::BW, C::BH, 1}, {0, 0, 0}};
}
template <class C>
constexpr CfgInfo info3d(int id)
{
    return CfgInfo{id, 3, 1, 0, 0, C::kNWX, C::kTZ, C::kNWX, C::TY, C::kTZ, C::SMEM, {C::BW, C::BH, C::BD},
                   {C::kNWX, C::BH, C::kTZ}};
}

static const CfgInfo kCfgs[] = {
    info2d<C2_1_12>(0), info2d<C2_2_12>(1), info2d<C2_4_12>(2), info2d<C2_8_12>(3),
    info2d<C2_1_28>(4), info2d<C2_2_28>(5), info2d<C2_4_28>(6), info2d<C2_8_28>(7),
    info2d<X2_4_12>(8), info2d<X2_8_12>(9), info2d<X2_16_12>(10), info2d<X2_4_28>(11), info2d<X2_8_28>(12),
    info3d<C3_8>(16),   info3d<C3_16>(17),  info3d<C3_4>(19),
};
static const int kIds2d[] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12};
static const int kIds3d[] = {19, 16, 17};

const CfgInfo *cfg_info(int id)
{
    for (const auto &c : kCfgs)
        if (c.id == id) return &c;
    return nullptr;
}
int max_cfg_smem()
{
    int m = 0;
    for (const auto &c : kCfgs) m = std::max(m, c.smem);
    return m;
}

const int *cfg_ids_2d(int *n) { *n = (int)(sizeof(kIds2d) / sizeof(kIds2d[0])); return kIds2d; }
const int *cfg_ids_3d(int *n) { *n = (int)(sizeof(kIds3d) / sizeof(kIds3d[0])); return kIds3d; }

constexpr int kThreads = 128;

// Issue the TMA load(s) of one tile of instance `in` for pass q into smem,
// completing on bar.  One thread calls it, after it has acquired the work
// item; the proxy fence orders the generic-proxy writes of earlier passes
// (made visible by that acquire) before the async-proxy reads.
__device__ void issue_tile(const Inst &in, int q, int tile, uint32_t *smem, uint64_t *bar)
{
    fence_proxy_async_global();
    switch (in.cfg) {
#define ISSUE2(ID, C) \
    case ID: tile2d_issue<C>(in, q, tile, smem, bar); break;
#define ISSUE3(ID, C) \
    case ID: tile3d_issue<C>(in, q, tile, smem, bar); break;
        ISSUE2(0, C2_1_12)
        ISSUE2(1, C2_2_12)
        ISSUE2(2, C2_4_12)
        ISSUE2(3, C2_8_12)
        ISSUE2(4, C2_1_28)
        ISSUE2(5, C2_2_28)
        ISSUE2(6, C2_4_28)
        ISSUE2(7, C2_8_28)
        ISSUE2(8, X2_4_12)
        ISSUE2(9, X2_8_12)
        ISSUE2(10, X2_16_12)
        ISSUE2(11, X2_4_28)
        ISSUE2(12, X2_8_28)
        ISSUE3(16, C3_8)
        ISSUE3(17, C3_16)
        ISSUE3(19, C3_4)
#undef ISSUE2
#undef ISSUE3
    default:
        break;
    }
}

// Run one tile of instance `in` at pass q with the instance's configuration
// on its box, already in smem.  All tile threads call it; returns the change
// mask (complete in thread 0; `band` is a zeroed shared word it may use).
__device__ uint32_t run_tile(const Inst &in, int q, int tile, uint32_t *smem, uint32_t *band)
{
    switch (in.cfg) {
#define CASE2_K1(ID, C)                                    \
    case ID:                                               \
        switch (q & 3) {                                   \
        case 0: return tile2d<C, 0>(in, q, tile, smem, band);   \
        case 1: return tile2d<C, 1>(in, q, tile, smem, band);   \
        case 2: return tile2d<C, 2>(in, q, tile, smem, band);   \
        default: return tile2d<C, 3>(in, q, tile, smem, band);  \
        }
#define CASE2_K2(ID, C)                                         \
    case ID:                                                    \
        if (q & 1) return tile2d<C, 2>(in, q, tile, smem, band);     \
        return tile2d<C, 0>(in, q, tile, smem, band);
#define CASE2_K4(ID, C) \
    case ID: return tile2d<C, 0>(in, q, tile, smem, band);
#define CASE2X(ID, C) \
    case ID: return tile2dx<C, 0>(in, q, tile, smem);
#define CASE3(ID, C)                                       \
    case ID:                                               \
        switch (q % 6) {                                   \
        case 0: return tile3d<C, 0>(in, q, tile, smem);   \
        case 1: return tile3d<C, 1>(in, q, tile, smem);   \
        case 2: return tile3d<C, 2>(in, q, tile, smem);   \
        case 3: return tile3d<C, 3>(in, q, tile, smem);   \
        case 4: return tile3d<C, 4>(in, q, tile, smem);   \
        default: return tile3d<C, 5>(in, q, tile, smem);  \
        }
        CASE2_K1(0, C2_1_12)
        CASE2_K2(1, C2_2_12)
        CASE2_K4(2, C2_4_12)
        CASE2_K4(3, C2_8_12)
        CASE2_K1(4, C2_1_28)
        CASE2_K2(5, C2_2_28)
        CASE2_K4(6, C2_4_28)
        CASE2_K4(7, C2_8_28)
        CASE2X(8, X2_4_12)
        CASE2X(9, X2_8_12)
        CASE2X(10, X2_16_12)
        CASE2X(11, X2_4_28)
        CASE2X(12, X2_8_28)
        CASE3(16, C3_8)
        CASE3(17, C3_16)
        CASE3(19, C3_4)
#undef CASE2_K1
#undef CASE2_K2
#undef CASE2_K4
#undef CASE2X
#undef CASE3
    default:
        return 0u;
    }
}

// --------------------------------------------------------- rule table -----
// Deletable sets of the device rules over every neighbourhood, 32 per word:
// neighbour i (2D: N, NE, E, SE, S, SW, W, NW; 3D: the 26 neighbours in
// (dz, dy, dx) order, centre skipped) is bit i of the neighbourhood number,
// whose low 5 bits select the bit of the word.  2D: 8 words per direction,
// 3D: 2^21 words per direction (centre foreground).
__device__ __forceinline__ uint32_t lane_pattern(int i)
{
    return i == 0 ? 0xAAAAAAAAu : i == 1 ? 0xCCCCCCCCu : i == 2 ? 0xF0F0F0F0u : i == 3 ? 0xFF00FF00u : 0xFFFF0000u;
}

template <int DIR>
__global__ void rule2d_table_kernel(uint32_t *out)
{
    const int w = threadIdx.x;
    if (w >= 8) return;
    uint32_t X[8];
    for (int i = 0; i < 8; i++) X[i] = i < 5 ? lane_pattern(i) : (((w >> (i - 5)) & 1) ? kFull : 0u);
    out[w] = rule2d<DIR>(X);
}

template <int DIR>
__global__ void rule3d_table_kernel(uint32_t *out)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= (1 << 21)) return;
    uint32_t g[27];
    for (int p = 0, i = 0; p < 27; p++) {
        if (p == 13) {
            g[p] = kFull;
            continue;
        }
        g[p] = i < 5 ? lane_pattern(i) : (((w >> (i - 5)) & 1) ? kFull : 0u);
        i++;
    }
    out[w] = rule3d<DIR>(g);
}

cudaError_t launch_rule_table(int dims, int dir, uint32_t *d_out, cudaStream_t st)
{
    if (dims == 2) {
        switch (dir) {
        case 0: rule2d_table_kernel<0><<<1, 32, 0, st>>>(d_out); break;
        case 1: rule2d_table_kernel<1><<<1, 32, 0, st>>>(d_out); break;
        case 2: rule2d_table_kernel<2><<<1, 32, 0, st>>>(d_out); break;
        case 3: rule2d_table_kernel<3><<<1, 32, 0, st>>>(d_out); break;
        default: return cudaErrorInvalidValue;
        }
    } else {
        const int grid = (1 << 21) / 256;
        switch (dir) {
        case 0: rule3d_table_kernel<0><<<grid, 256, 0, st>>>(d_out); break;
        case 1: rule3d_table_kernel<1><<<grid, 256, 0, st>>>(d_out); break;
        case 2: rule3d_table_kernel<2><<<grid, 256, 0, st>>>(d_out); break;
        case 3: rule3d_table_kernel<3><<<grid, 256, 0, st>>>(d_out); break;
        case 4: rule3d_table_kernel<4><<<grid, 256, 0, st>>>(d_out); break;
        case 5: rule3d_table_kernel<5><<<grid, 256, 0, st>>>(d_out); break;
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
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

// ------------------------------------------------------- batch-wide -------
// One launch packs (or unpacks) every instance of a batch: the global word
// index is mapped to its instance by a binary search over io[].wbegin.

// 32 one-byte pixels starting at p -> bit word.  MSB-of-byte gather:
// multiplying the MSB mask by 0x00204081 moves bits 7, 15, 23, 31 to 28..31
// without carries.
__device__ __forceinline__ uint32_t bytes4_to_bits(uint32_t cmp)
{
    return ((cmp & 0x80808080u) * 0x00204081u) >> 28;
}

// 4 bytes -> 4 bits "byte != 0" (bit k for byte k) with integer ALU ops only:
// the low seven bits of each byte plus 0x7F carry into the byte's MSB
// exactly when they are nonzero (no carry leaves the byte), and OR-ing the
// byte back in covers the MSB itself.
__device__ __forceinline__ uint32_t nz4_to_bits(uint32_t c)
{
    return bytes4_to_bits(((c & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | c);
}

// 32 bytes at word offset Q (0..3) and byte shift sh of 12 loaded words ->
// 32 "nonzero" bits
template <int Q>
__device__ __forceinline__ uint32_t pack_from12(const uint32_t (&u)[12], unsigned sh)
{
    uint32_t w = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) w |= nz4_to_bits(__funnelshift_r(u[Q + k], u[Q + k + 1], sh)) << (4 * k);
    return w;
}

// `room` = bytes readable from p onward (>= 36 allows the aligned 4-byte
// loads that cover p .. p+31 whatever p's alignment); `lead` = bytes readable
// before p (>= 15 and room >= 33 allow three 16-byte loads from the 16-byte
// boundary at or below p).
template <typename T, int MODE>
__device__ __forceinline__ uint32_t pack_word(const T *p, int n, long long room = 0, long long lead = 0)
{
    if constexpr (sizeof(T) == 1 && (MODE != 1 || std::is_unsigned<T>::value || std::is_same<T, bool>::value)) {
        // one-byte types whose test is "nonzero" (2D rule and unsigned/bool 3D rule)
        const uintptr_t pa = reinterpret_cast<uintptr_t>(p);
        if (n == 32 && (long long)(pa & 15u) <= lead && (long long)(48 - (pa & 15u)) <= room) {
            // three aligned 16-byte loads cover p .. p+31; realign by words and bytes
            const uint4 *a16 = reinterpret_cast<const uint4 *>(pa & ~uintptr_t(15));
            const uint4 A = __ldg(a16), B = __ldg(a16 + 1), C = __ldg(a16 + 2);
            const uint32_t u[12] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w, C.x, C.y, C.z, C.w};
            const unsigned sh = (unsigned)(pa & 3u) * 8u;
            switch ((pa >> 2) & 3u) {
            case 0: return pack_from12<0>(u, sh);
            case 1: return pack_from12<1>(u, sh);
            case 2: return pack_from12<2>(u, sh);
            default: return pack_from12<3>(u, sh);
            }
        }
        if (n == 32 && (reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
            const uint4 a = *reinterpret_cast<const uint4 *>(p);
            const uint4 b = *reinterpret_cast<const uint4 *>(p + 16);
            const uint32_t c[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) w |= nz4_to_bits(c[k]) << (4 * k);
            return w;
        }
        // misaligned row: nine aligned words (p-3 .. p+35 at most, all inside
        // the input: room counts bytes from p to the end, a negative room
        // marks a word within 3 bytes of the input start), realigned with
        // funnel shifts
        if (n == 32 && room >= 36) {
            const uintptr_t pa = reinterpret_cast<uintptr_t>(p);
            const uint32_t *a = reinterpret_cast<const uint32_t *>(pa & ~uintptr_t(3));
            const unsigned s = (unsigned)(pa & 3u) * 8u;
            uint32_t prev = __ldg(a);
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t next = __ldg(a + k + 1);
                const uint32_t c = __funnelshift_r(prev, next, s);
                w |= nz4_to_bits(c) << (4 * k);
                prev = next;
            }
            return w;
        }
    }
    uint32_t w = 0;
    for (int b = 0; b < n; b++) {
        const T v = p[b];
        const bool f = MODE == 0 ? fg2<T>(v) : MODE == 1 ? fg3<T>(v) : (v != (T)0);
        w |= (uint32_t)f << b;
    }
    return w;
}

// 32 one-byte pixels from p (n < 32 at a row's ragged end) -> "byte != 0"
// bits, without branches that depend on p's alignment: three aligned 16-byte
// loads cover p .. p+31 (they may run past the row into the next one, never
// past the input: `room` and `lead` as in pack_word), the 12 loaded words are
// shifted by p's word offset in two conditional-select stages and by its byte
// offset with funnel shifts, and bits at and past n are cleared.  Words too
// close to either end of the input take the byte loop.
__device__ __forceinline__ uint32_t pack_bytes32(const uint8_t *p, int n, long long room, long long lead)
{
    const uintptr_t pa = reinterpret_cast<uintptr_t>(p);
    const unsigned o = (unsigned)(pa & 15u);
    if ((long long)o <= lead && (long long)(48u - o) <= room) {
        const uint4 *a16 = reinterpret_cast<const uint4 *>(pa & ~uintptr_t(15));
        const uint4 A = __ldg(a16), B = __ldg(a16 + 1), C = __ldg(a16 + 2);
        const uint32_t u[12] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w, C.x, C.y, C.z, C.w};
        const bool s2 = (o & 8u) != 0, s1 = (o & 4u) != 0;
        uint32_t t[10], v[9];
#pragma unroll
        for (int i = 0; i < 10; i++) t[i] = s2 ? u[i + 2] : u[i];
#pragma unroll
        for (int i = 0; i < 9; i++) v[i] = s1 ? t[i + 1] : t[i];
        const unsigned sh = (o & 3u) * 8u;
        uint32_t w = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) w |= nz4_to_bits(__funnelshift_r(v[k], v[k + 1], sh)) << (4 * k);
        return n >= 32 ? w : w & ((1u << n) - 1u);
    }
    uint32_t w = 0;
    for (int b = 0; b < n; b++) w |= (uint32_t)(p[b] != 0) << b;
    return w;
}

template <typename T>
__device__ __forceinline__ uint32_t pack_word_mode(const T *p, int n, int mode, long long room, long long lead = 0)
{
    return mode == 0 ? pack_word<T, 0>(p, n, room, lead) : mode == 1 ? pack_word<T, 1>(p, n, room, lead)
                                                                     : pack_word<T, 2>(p, n, room, lead);
}

__device__ __forceinline__ int dtype_bytes(int dtype)
{
    return dtype == BGT_F64 ? 8 : (dtype == BGT_U32 || dtype == BGT_I32 || dtype == BGT_F32) ? 4
                                  : (dtype == BGT_U16 || dtype == BGT_I16) ? 2 : 1;
}

__device__ __forceinline__ int find_io(const IODesc *io, int n, long long g, bool unpack)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((unpack ? io[mid].gbegin : io[mid].wbegin) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// BYTES: every instance of the batch has a one-byte input whose test is
// "byte != 0" (uint8/bool, and int8/char under the 2D rule), so one path
// serves all and the per-word type dispatch goes away.
template <bool BYTES>
__global__ void pack_all_kernel(const Inst *__restrict__ insts, const IODesc *__restrict__ io, int n,
                                long long total)
{
    // the instance's descriptor, cached while consecutive units stay in it
    int k = -1;
    long long kb = 0, ke = 0;
    IODesc d{};
    uint32_t *buf0 = nullptr, *buf1 = nullptr;
    int *lc = nullptr;
    int P = 0, H = 0, tiles_x = 0, tiles_y = 0;
    // each block takes one contiguous range, so consecutive units of a thread
    // stay in the same instance and the instance lookup is rarely repeated
    const long long per = (total + gridDim.x - 1) / gridDim.x;
    const long long g_end = min(total, per * (blockIdx.x + 1));
    for (long long g = per * blockIdx.x + threadIdx.x; g < g_end; g += blockDim.x) {
        if (g < kb || g >= ke) {  // instance lookup only when leaving the cached range
            k = find_io(io, n, g, false);
            d = io[k];
            kb = d.wbegin;
            ke = k + 1 < n ? io[k + 1].wbegin : total;
            const Inst &in = insts[d.inst];
            buf0 = in.buf[0];
            // an image thinned by the resident kernel reads only buf[0] and
            // no tile marks (its bands write buf[1] before reading it); the
            // tile engine and volumes, which may spill to it, need both
            const bool res2d = in.res && in.dims == 2;
            buf1 = res2d ? nullptr : in.buf[1];
            lc = res2d ? nullptr : in.lc;
            P = in.P;
            H = in.H;
            tiles_x = in.tiles_x;
            tiles_y = in.tiles_y;
        }
        // 32-bit index math: an instance has fewer than 2^31 packed words
        const uint32_t i = (uint32_t)(g - kb);
        const uint32_t row = fdiv(d.dP, i);
        const int j = (int)(i - row * (uint32_t)P);
        const uint32_t z = fdiv(d.dH, row);
        const int y = (int)(row - z * (uint32_t)H);
        const int x0 = j * 32;
        uint32_t w = 0;
        if (x0 < d.inW && y < d.inH && (int)z < d.inD) {
            const long long off = ((long long)z * d.inH + y) * (long long)d.inW + x0;
            const int cnt = min(32, d.inW - x0);
            // elements from off to the end of the input; words that start in the
            // first 3 bytes of an unaligned input are kept on the scalar path
            const bool head_ok = off >= 4 || (reinterpret_cast<uintptr_t>(d.in) & 3u) == 0;
            const long long room = head_ok ? (long long)d.inW * d.inH * d.inD - off : 0;
            const long long lead = off;  // one-byte inputs: bytes before this word's first pixel
            if constexpr (BYTES) {
                w = pack_bytes32((const uint8_t *)d.in + off, cnt, room, lead);
            } else switch (d.dtype) {
            case BGT_U8: w = pack_word_mode((const uint8_t *)d.in + off, cnt, d.mode, room, lead); break;
            case BGT_I8: w = pack_word_mode((const int8_t *)d.in + off, cnt, d.mode, room, lead); break;
            case BGT_CHAR: w = pack_word_mode((const char *)d.in + off, cnt, d.mode, room, lead); break;
            case BGT_U16: w = pack_word_mode((const uint16_t *)d.in + off, cnt, d.mode, room); break;
            case BGT_I16: w = pack_word_mode((const int16_t *)d.in + off, cnt, d.mode, room); break;
            case BGT_U32: w = pack_word_mode((const uint32_t *)d.in + off, cnt, d.mode, room); break;
            case BGT_I32: w = pack_word_mode((const int32_t *)d.in + off, cnt, d.mode, room); break;
            case BGT_F32: w = pack_word_mode((const float *)d.in + off, cnt, d.mode, room); break;
            case BGT_F64: w = pack_word_mode((const double *)d.in + off, cnt, d.mode, room); break;
            default: w = pack_word_mode((const bool *)d.in + off, cnt, d.mode, room, lead); break;
            }
        }
        buf0[i] = w;
        if (!buf1) continue;
        buf1[i] = w;
        if (w) {  // tile holds foreground: lc = -1 (pre-filled with kNever)
            const int t = ((int)fdiv(d.dTZ, z) * tiles_y + (int)fdiv(d.dTH, (uint32_t)y)) * tiles_x +
                          (int)fdiv(d.dTW, (uint32_t)j);
            lc[t] = -1;
        }
    }
}

// 4 bits -> 4 bytes of value 0/1 (bit k to byte k): the multiplier places bit
// k at 8k and the mask drops the other partial products (all at distinct bits).
__device__ __forceinline__ uint32_t bits4_to_bytes(uint32_t nib) { return (nib * 0x00204081u) & 0x01010101u; }

template <typename T>
__device__ __forceinline__ void unpack_word(uint32_t w, T *o, int n)
{
    if constexpr (sizeof(T) == 1) {
        if (n == 32 && (reinterpret_cast<uintptr_t>(o) & 15u) == 0) {
            uint32_t c[8];
#pragma unroll
            for (int k = 0; k < 8; k++) c[k] = bits4_to_bytes((w >> (4 * k)) & 15u);
            *reinterpret_cast<uint4 *>(o) = make_uint4(c[0], c[1], c[2], c[3]);
            *reinterpret_cast<uint4 *>(o + 16) = make_uint4(c[4], c[5], c[6], c[7]);
            return;
        }
        if (n == 32) {
            // misaligned: head bytes up to a 4-byte boundary, seven aligned
            // words, tail bytes; exactly the 32 bytes of this word are written
            const unsigned h = (unsigned)((4u - (reinterpret_cast<uintptr_t>(o) & 3u)) & 3u);
            uint8_t *ob = reinterpret_cast<uint8_t *>(o);
            for (unsigned b = 0; b < h; b++) ob[b] = (uint8_t)((w >> b) & 1u);
            uint32_t *oa = reinterpret_cast<uint32_t *>(ob + h);
            const uint64_t ww = (uint64_t)w >> h;
#pragma unroll
            for (int k = 0; k < 7; k++) oa[k] = bits4_to_bytes((uint32_t)(ww >> (4 * k)) & 15u);
            const unsigned done = h + 28;
            for (unsigned b = done; b < 32; b++) ob[b] = (uint8_t)((w >> b) & 1u);
            return;
        }
    }
    for (int b = 0; b < n; b++) o[b] = (T)((w >> b) & 1u);
}

// 16 consecutive bits of a packed row starting at pixel x (x + 16 <= the
// row's words * 32), as the low half of a word.
__device__ __forceinline__ uint32_t row_bits16(const uint32_t *r, int x)
{
    const uint32_t w0 = __ldg(r + (x >> 5));
    const uint32_t w1 = (x & 31) > 16 ? __ldg(r + (x >> 5) + 1) : 0u;
    return __funnelshift_r(w0, w1, x & 31) & 0xffffu;
}

// One-byte outputs: unit = one 16-byte-aligned chunk of the output (absolute
// address), written with one 128-bit store when the chunk lies inside the
// instance's output, bytewise at its two ends.  Each byte is pixel
// (row, x) of the flat index; a chunk spans at most two rows when W >= 16.
__device__ __forceinline__ void unpack_chunk16(const uint32_t *buf, int W, int P, long long n, const IODesc &d,
                                               long long c)
{
    const uintptr_t out = reinterpret_cast<uintptr_t>(d.out);
    const uintptr_t a = (out & ~uintptr_t(15)) + (uintptr_t)c * 16u;
    const long long lo = (long long)(a > out ? a - out : 0);  // first flat index in the chunk
    const long long hi = min((long long)(a + 16 - out), n);   // one past the last
    // flat indices of one instance stay below 2^31 (sizes are capped at 32767
    // per axis and the batch limits an instance to < 2^31 pixels)
    uint32_t row = fdiv(d.dW, (uint32_t)lo);
    int x = (int)((uint32_t)lo - row * (uint32_t)W);
    if (hi - lo == 16 && a >= out && W >= 16) {
        uint32_t bits;
        if (x + 16 <= W) {
            bits = row_bits16(buf + (size_t)row * P, x);
        } else {  // the chunk runs into the next row
            const int n0 = W - x;
            bits = (row_bits16(buf + (size_t)row * P, x) & ((1u << n0) - 1u)) |
                   (row_bits16(buf + (size_t)(row + 1) * P, 0) << n0);
        }
        *reinterpret_cast<uint4 *>(a) = make_uint4(bits4_to_bytes(bits & 15u), bits4_to_bytes((bits >> 4) & 15u),
                                                   bits4_to_bytes((bits >> 8) & 15u),
                                                   bits4_to_bytes((bits >> 12) & 15u));
        return;
    }
    uint32_t word = __ldg(buf + (size_t)row * P + (x >> 5));
    uint32_t bytes[4] = {0u, 0u, 0u, 0u};
    const int first = (int)((out + lo) - a);  // byte position of flat index lo in the chunk
    for (long long f = lo; f < hi; f++) {
        const int pos = first + (int)(f - lo);
        bytes[pos >> 2] |= ((word >> (x & 31)) & 1u) << (8 * (pos & 3));
        if (++x == W) {
            x = 0;
            row++;
            if (f + 1 < hi) word = __ldg(buf + (size_t)row * P);
        } else if ((x & 31) == 0 && f + 1 < hi) {
            word = __ldg(buf + (size_t)row * P + (x >> 5));
        }
    }
    if (first == 0 && hi - lo == 16) {
        *reinterpret_cast<uint4 *>(a) = make_uint4(bytes[0], bytes[1], bytes[2], bytes[3]);
    } else {
        uint8_t *ob = reinterpret_cast<uint8_t *>(a);
        for (int pos = first; pos < first + (int)(hi - lo); pos++) ob[pos] = (uint8_t)(bytes[pos >> 2] >> (8 * (pos & 3)));
    }
}

// 32 consecutive bits of a packed row starting at pixel x; the word after
// x's word is read only when x is not word-aligned, and the caller
// guarantees it lies inside the packed buffer.
__device__ __forceinline__ uint32_t row_bits32(const uint32_t *r, int x)
{
    const uint32_t w0 = __ldg(r + (x >> 5));
    const uint32_t w1 = (x & 31) ? __ldg(r + (x >> 5) + 1) : 0u;
    return __funnelshift_r(w0, w1, x & 31);
}

// One-byte outputs, unit = one 32-byte-aligned chunk of the output: two
// 128-bit stores when the chunk lies inside the output and the image is at
// least 32 pixels wide (the chunk then spans at most two rows); otherwise
// its two 16-byte halves go through unpack_chunk16.
__device__ __forceinline__ void unpack_chunk32(const uint32_t *buf, int W, int P, long long n, const IODesc &d,
                                               long long c)
{
    const uintptr_t out = reinterpret_cast<uintptr_t>(d.out);
    const uintptr_t a = (out & ~uintptr_t(31)) + (uintptr_t)c * 32u;
    if (a >= out && (long long)(a + 32 - out) <= n && W >= 32) {
        const uint32_t lo = (uint32_t)(a - out);
        const uint32_t row = fdiv(d.dW, lo);
        const int x = (int)(lo - row * (uint32_t)W);
        const uint32_t *r = buf + (size_t)row * P;
        uint32_t bits;
        if (x + 32 <= W) {
            bits = row_bits32(r, x);
        } else {  // the chunk runs into the next row
            const int n0 = W - x;
            bits = (row_bits32(r, x) & ((1u << n0) - 1u)) | (__ldg(r + P) << n0);
        }
        uint4 *o = reinterpret_cast<uint4 *>(a);
        o[0] = make_uint4(bits4_to_bytes(bits & 15u), bits4_to_bytes((bits >> 4) & 15u),
                          bits4_to_bytes((bits >> 8) & 15u), bits4_to_bytes((bits >> 12) & 15u));
        o[1] = make_uint4(bits4_to_bytes((bits >> 16) & 15u), bits4_to_bytes((bits >> 20) & 15u),
                          bits4_to_bytes((bits >> 24) & 15u), bits4_to_bytes(bits >> 28));
        return;
    }
    const uintptr_t base16 = out & ~uintptr_t(15);
    for (int h = 0; h < 2; h++) {
        const uintptr_t ah = a + 16u * (uintptr_t)h;
        if (ah + 16 <= out || (ah >= out && (long long)(ah - out) >= n)) continue;  // outside the output
        unpack_chunk16(buf, W, P, n, d, (long long)((ah - base16) / 16u));
    }
}

__global__ void unpack_all_kernel(const Inst *__restrict__ insts, const IODesc *__restrict__ io, int n,
                                  long long total)
{
    int k = -1;
    long long kb = 0, ke = 0;
    IODesc d{};
    const uint32_t *buf = nullptr;
    int W = 0, P = 0, wwords = 0;
    long long npx = 0;
    bool bytes1 = false;
    // each block takes one contiguous range, so consecutive units of a thread
    // stay in the same instance and the instance lookup is rarely repeated
    const long long per = (total + gridDim.x - 1) / gridDim.x;
    const long long g_end = min(total, per * (blockIdx.x + 1));
    for (long long g = per * blockIdx.x + threadIdx.x; g < g_end; g += blockDim.x) {
        if (g < kb || g >= ke) {  // instance lookup only when leaving the cached range
            k = find_io(io, n, g, true);
            d = io[k];
            kb = d.gbegin;
            ke = k + 1 < n ? io[k + 1].gbegin : total;
            const Inst &in = insts[d.inst];
            buf = in.buf[0];
            W = in.W;
            P = in.P;
            wwords = (in.W + 31) >> 5;
            npx = (long long)in.W * in.H * in.D;
            bytes1 = dtype_bytes(d.dtype) == 1;
        }
        if (!d.out) continue;
        if (bytes1) {
            unpack_chunk32(buf, W, P, npx, d, g - kb);
            continue;
        }
        const uint32_t i = (uint32_t)(g - kb);
        const uint32_t row = fdiv(d.dWW, i);
        const int j = (int)(i - row * (uint32_t)wwords);
        const uint32_t w = __ldg(buf + (size_t)row * P + j);
        const long long off = (long long)row * W + (long long)j * 32;
        const int cnt = min(32, W - j * 32);
        switch (d.dtype) {
        case BGT_U16: unpack_word(w, (uint16_t *)d.out + off, cnt); break;
        case BGT_I16: unpack_word(w, (int16_t *)d.out + off, cnt); break;
        case BGT_U32: unpack_word(w, (uint32_t *)d.out + off, cnt); break;
        case BGT_I32: unpack_word(w, (int32_t *)d.out + off, cnt); break;
        case BGT_F32: unpack_word(w, (float *)d.out + off, cnt); break;
        case BGT_F64: unpack_word(w, (double *)d.out + off, cnt); break;
        default: break;  // one-byte types take the chunk path above
        }
    }
}

cudaError_t launch_pack_all(const Inst *d_insts, const IODesc *d_io, int n, long long total_words, bool bytes,
                            cudaStream_t st)
{
    if (bytes)
        pack_all_kernel<true><<<grid_for(total_words, 256), 256, 0, st>>>(d_insts, d_io, n, total_words);
    else
        pack_all_kernel<false><<<grid_for(total_words, 256), 256, 0, st>>>(d_insts, d_io, n, total_words);
    return cudaGetLastError();
}

cudaError_t launch_unpack_all(const Inst *d_insts, const IODesc *d_io, int n, long long total_words,
                              cudaStream_t st)
{
    unpack_all_kernel<<<grid_for(total_words, 256), 256, 0, st>>>(d_insts, d_io, n, total_words);
    return cudaGetLastError();
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

__device__ __forceinline__ void plain_pass_body(Inst *pin, int q, int *flag, int *err);

__global__ void __launch_bounds__(kThreads) plain_pass_kernel(Inst *pin, int q, int *flag, int *err)
{
    plain_pass_body(pin, q, flag, err);
}

// The plain path's pass loop kept on the device: pass q and the change flag
// live in device memory, and plain_loop_step_kernel decides whether another
// pass follows (the conditional node of a CUDA graph repeats the pass while
// it says so), with the same rule as the host loop of run_plain.
__global__ void __launch_bounds__(kThreads) plain_pass_dev_kernel(Inst *pin, PlainLoop *L, int *err)
{
    plain_pass_body(pin, L->q, &L->flag, err);
}

__global__ void plain_loop_init_kernel(PlainLoop *L)
{
    L->q = 0;
    L->last_change = -1;
    L->flag = 0;
    L->converged = 0;
}

__global__ void plain_loop_step_kernel(PlainLoop *L, Inst *pin, int *err, cudaGraphConditionalHandle h)
{
    Inst &in = *pin;
    const int q = L->q;
    if (L->flag) L->last_change = q;
    L->flag = 0;
    bool done;
    if (in.dims == 2) done = q - L->last_change >= in.window;
    else done = q % 6 == 5 && L->last_change < q - 5;
    L->q = q + 1;
    if (done) L->converged = 1;
    else if (q + 1 >= in.pass_cap) {
        L->converged = -1;
        atomicOr(err, kErrPassLimit);
    }
    in.passes_run = q + 1;
    in.converged = L->converged;
    cudaGraphSetConditional(h, L->converged == 0 ? 1u : 0u);
}

__device__ __forceinline__ void plain_pass_body(Inst *pin, int q, int *flag, int *err)
{
    extern __shared__ __align__(128) uint32_t smem_raw[];
    uint32_t *smem = align128(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    __shared__ int active;
    __shared__ uint32_t band;
    const Inst &in = *pin;
    const int tile = blockIdx.x;
    if (threadIdx.x == 0) {
        band = 0;
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
    if (threadIdx.x == 0) issue_tile(in, q, tile, smem, &bar);
    if (!mbar_wait_bounded(&bar, 0)) {
        if (threadIdx.x == 0) atomicOr(err, kErrTmaTimeout);
    }
    const bool ch = (run_tile(in, q, tile, smem, &band) & kTileChanged) != 0;
    if (threadIdx.x == 0) {
        atomicAdd(&pin->tiles_run, 1ull);
        atomicAdd(&pin->work_words, (unsigned long long)tile_core_words(in, tile));
        if (ch) {
            in.lc[tile] = q;
            atomicExch(flag, 1);
        }
    }
}

cudaError_t launch_plain_dev_pass(int cfg, Inst *d_inst, int ntiles, PlainLoop *d_loop, int *d_err, cudaStream_t st)
{
    const CfgInfo *c = cfg_info(cfg);
    if (!c) return cudaErrorInvalidValue;
    plain_pass_dev_kernel<<<ntiles, kThreads, c->smem + 128, st>>>(d_inst, d_loop, d_err);
    return cudaGetLastError();
}

cudaError_t launch_plain_loop_init(PlainLoop *d_loop, cudaStream_t st)
{
    plain_loop_init_kernel<<<1, 1, 0, st>>>(d_loop);
    return cudaGetLastError();
}

cudaError_t launch_plain_loop_step(PlainLoop *d_loop, Inst *d_inst, int *d_err, cudaGraphConditionalHandle h,
                                   cudaStream_t st)
{
    plain_loop_step_kernel<<<1, 1, 0, st>>>(d_loop, d_inst, d_err, h);
    return cudaGetLastError();
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
// Two work rings (0: critical-path instances, served first; 1: the rest),
// each a bounded MPMC queue with per-slot sequence numbers:
//   seq[s] == t    slot free for ticket t (the producer may write it)
//   seq[s] == t+1  item of ticket t ready
//   the consumer of ticket t then sets seq[s] = t + cap.
// Producers reserve tickets with an atomic on `tail`; a consumer takes a
// ticket with one fetch-and-add on `head` when the ring looks non-empty.

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
__device__ __forceinline__ unsigned ld_volatile_u(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Publish n items (instance ii, tiles list[0..n), pass q) on the instance's
// ring; item.w carries n (plus kItemGang for a gang wave) so a consumer
// knows the wave size.  The tile threads call it.
constexpr int kItemGang = 1 << 30;
__device__ void produce(Sched *S, int ii, int prio, const int *list, int n, int q, int gang)
{
    __shared__ unsigned t0;
    Ring &R = S->ring[prio];
    if (threadIdx.x == 0) t0 = atomicAdd(&R.tail, (unsigned)n);
    tile_sync();
    const unsigned cap = R.cap;
    for (int i = threadIdx.x; i < n; i += kTileThreads) {
        const unsigned t = t0 + (unsigned)i;
        const unsigned s = t % cap;
        bool ok = ld_acq_u(R.seq + s) == t;
        if (!ok) {
            const unsigned long long t_end = globaltimer() + (unsigned long long)S->timeout_ns;
            for (int spin = 0;; spin++) {
                __nanosleep(64);
                if (ld_acq_u(R.seq + s) == t) { ok = true; break; }
                if ((spin & 255) == 255 && globaltimer() > t_end) break;
            }
        }
        if (!ok) {
            atomicOr(&S->status, kErrQueueFull);
            continue;
        }
        R.item[s] = make_int4(ii, __ldcg(list + i), q, n | gang);
        st_rel_u(R.seq + s, t + 1);
    }
    tile_sync();
}

// Active tiles of pass q1 (tiles whose 3x3(x3) neighbourhood changed within
// the window), marked by scattering from the changed tiles into a bitmap in
// shared memory; falls back to gathering per tile when the instance has more
// tiles than the bitmap holds.  The tile threads call it; returns the count.
__device__ int build_list(Inst &in, int q1, int window, uint32_t *scratch, int scratch_words)
{
    __shared__ int cnt;
    const int nt = in.ntiles;
    const int nwords = (nt + 31) >> 5;
    if (threadIdx.x == 0) cnt = 0;
    const int thr = q1 - window;
    if (2 * nwords <= scratch_words) {
        uint32_t *act = scratch, *ne = scratch + nwords;
        for (int i = threadIdx.x; i < 2 * nwords; i += kTileThreads) scratch[i] = 0;
        tile_sync();
        const int tx = in.tiles_x, ty = in.tiles_y, tz = in.tiles_z;
        // 2D tiles fused over a whole iteration (window 1) recorded which
        // neighbours their change reaches (border bands); others reach all
        const bool bands = in.dims == 2 && window == 1;
        for (int t = threadIdx.x; t < nt; t += kTileThreads) {
            const int v = ld_cg_int(in.lc + t);
            if (v == kNever) continue;
            atomicOr(ne + (t >> 5), 1u << (t & 31));
            if (v < thr) continue;
            const uint32_t reach = (bands && v >= 0) ? (uint32_t)__ldcg(in.act + t) : kAllBands;
            const int x = t % tx, y = (t / tx) % ty, z = t / (tx * ty);
            for (int dz = -1; dz <= 1; dz++) {
                const int zz = z + dz;
                if (zz < 0 || zz >= tz) continue;
                for (int dy = -1; dy <= 1; dy++) {
                    const int yy = y + dy;
                    if (yy < 0 || yy >= ty) continue;
                    for (int dx = -1; dx <= 1; dx++) {
                        const int xx = x + dx;
                        if (xx < 0 || xx >= tx) continue;
                        if ((dy | dx) != 0 && dz == 0 && !((reach >> band_bit(dy, dx)) & 1u)) continue;
                        const int u = (zz * ty + yy) * tx + xx;
                        atomicOr(act + (u >> 5), 1u << (u & 31));
                    }
                }
            }
        }
        tile_sync();
        for (int w = threadIdx.x; w < nwords; w += kTileThreads) {
            uint32_t m = act[w] & ne[w];
            while (m) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                in.list[atomicAdd(&cnt, 1)] = (w << 5) + b;
            }
        }
    } else {
        tile_sync();
        for (int t = threadIdx.x; t < nt; t += kTileThreads)
            if (ld_cg_int(in.lc + t) != kNever && nbr_last_change(in, t) >= thr) in.list[atomicAdd(&cnt, 1)] = t;
    }
    tile_sync();
    return cnt;
}

// Largest 3D wave that may form a gang.
constexpr int kGangMaxTiles = 256;

// Build the active list for pass q1 of instance ii and publish it, or retire
// the instance.  The tile threads call it.  3D instances rebuild the list only at
// iteration starts (the union pass decides activity for the iteration).
__device__ void next_wave(Sched *S, Inst *insts, int ii, int q1, int nprev, uint32_t *scratch, int scratch_words)
{
    Inst &in = insts[ii];
    __shared__ int cnt, gang;
    int n;
    if (in.dims == 2) n = build_list(in, q1, in.window, scratch, scratch_words);
    else if (q1 % 6 == 0) n = build_list(in, q1, 6, scratch, scratch_words);
    else n = nprev;
    if (threadIdx.x == 0) {
        in.passes_run = q1;
        bool retire = n == 0;
        if (!retire && q1 >= in.pass_cap) {
            atomicOr(&S->status, kErrPassLimit);
            retire = true;
        }
        gang = 0;
        if (retire) {
            in.converged = n == 0 ? 1 : -1;
        } else {
            in.pass = q1;
            in.done = 0;
            // a small 3D wave whose list holds for the rest of the iteration
            // becomes a gang when the budget allows: the CTAs that take its
            // tiles keep them through the iteration's remaining passes
            if (in.dims == 3 && q1 % 6 != 5 && n <= kGangMaxTiles) {
                if (atomicSub(&S->gang_budget, n) >= n) {
                    in.gang = 0;
                    gang = kItemGang;
                } else {
                    atomicAdd(&S->gang_budget, n);
                }
            }
        }
        __threadfence();
        if (retire) {
            atomicSub(&S->live_prio[in.prio], 1);
            atomicSub(&S->live, 1);
        }
        cnt = retire ? 0 : n;
    }
    tile_sync();
    const int m = cnt;
    if (m > 0) produce(S, ii, in.prio, in.list, m, q1, gang);
}

// One CTA per instance: marks reset done by the pack; first wave (pass 0).
__global__ void __launch_bounds__(kThreads) engine_seed_kernel(Inst *insts, int ninst, Sched *S)
{
    __shared__ uint32_t scratch[2048];
    for (int ii = blockIdx.x; ii < ninst; ii += gridDim.x) {
        // instances of the resident engine are done unless they spilled
        if (insts[ii].res && !insts[ii].spill) continue;
        if (threadIdx.x == 0) {
            insts[ii].converged = 0;
            insts[ii].passes_run = 0;
            insts[ii].tiles_run = 0;
            insts[ii].work_words = 0;
            atomicAdd(&S->live_prio[insts[ii].prio], 1);
            atomicAdd(&S->live, 1);
        }
        __syncthreads();
        next_wave(S, insts, ii, 0, 0, scratch, 2048);
        __syncthreads();
    }
}

// A consumer takes a ticket of a ring (one fetch-and-add, no retry loop)
// when the ring looks non-empty.  Several CTAs may see the same last item, so
// a ticket can run past the items produced so far; its holder then waits for
// the ring's next item (see wait_ticket).
// Wait for the item of ticket t of ring r.  Returns 1 with the item, 0 when
// the ticket can never be filled (every instance of that ring retired and t
// is past the final tail: the ticket is abandoned), -1 on timeout.
__device__ __forceinline__ int wait_ticket(Sched *S, int r, unsigned t, int4 &out, unsigned long long t_end)
{
    Ring &R = S->ring[r];
    const unsigned s = t % R.cap;
    for (int w = 0;; w++) {
        if (ld_acq_u(R.seq + s) == t + 1) {
            out = __ldcg(R.item + s);
            st_rel_u(R.seq + s, t + R.cap);
            return 1;
        }
        if ((w & 15) == 15) {
            if (ld_acquire(&S->live_prio[r]) == 0 && (int)(t - ld_volatile_u(&R.tail)) >= 0) return 0;
            if (globaltimer() > t_end) return -1;
        }
        if (w > 8) __nanosleep(w < 64 ? 32 : 256);
    }
}

// Wait (bounded by the scheduler's timeout) until *p >= target; acquire.
__device__ __noinline__ bool wait_at_least(const int *p, int target, const Sched *S)
{
    const unsigned long long t_end = globaltimer() + (unsigned long long)S->timeout_ns;
    for (int spin = 0;; spin++) {
        if (ld_acquire(p) >= target) return true;
        if ((spin & 63) == 63 && globaltimer() > t_end) return false;
        __nanosleep(spin < 16 ? 20 : 100);
    }
}

// One look at ticket t of ring r (no waiting): 1 with the item (the slot is
// released as by wait_ticket), 0 when it is not filled yet.
__device__ __forceinline__ int poll_ticket(Sched *S, int r, unsigned t, int4 &out)
{
    Ring &R = S->ring[r];
    const unsigned s = t % R.cap;
    if (ld_acq_u(R.seq + s) != t + 1) return 0;
    out = __ldcg(R.item + s);
    st_rel_u(R.seq + s, t + R.cap);
    return 1;
}

// Shared-memory scratch of the engine's next-wave builder, behind the tile
// box: the next tile's box may be in flight while a wave is built.
constexpr int kEngineScratchWords = 1024;
static int engine_smem_bytes(int box_bytes)
{
    return 128 + (box_bytes + 127) / 128 * 128 + kEngineScratchWords * 4;
}

// Most bulk-ring tickets one CTA takes with one fetch-and-add.
constexpr int kMaxClaim = 4;

// Persistent engine: thread 0 of each CTA claims a work item (ring 0 first),
// stages the tile by TMA; the CTA computes it, records its change, counts it
// against its wave and, for the wave's last tile, builds and publishes the
// instance's next wave.  The CTAs holding the tiles of a gang wave (a small
// 3D wave whose tile list stays the same until the iteration ends) instead
// meet at a per-instance barrier after each pass and go on with the same
// tile.  A budget caps the tiles of all live gangs together at the number of
// CTAs, so all gangs can be staffed at once; the CTAs outside gangs finish
// their tiles and claim in ticket order, so no gang waits on a tile nobody
// can take.  Every wait is bounded and reports a status bit.
__global__ void __launch_bounds__(kThreads, 8) engine_kernel(Inst *insts, Sched *S, int box_words)
{
    extern __shared__ __align__(128) uint32_t smem_raw[];
    uint32_t *smem = align128(smem_raw);
    uint32_t *scratch = smem + (box_words + 31) / 32 * 32;
    __shared__ __align__(8) uint64_t bar;
    __shared__ int4 item, nitem;
    __shared__ int got, last, ngot;
    __shared__ uint32_t band;
    if (threadIdx.x == 0) {
        band = 0;
        ngot = 0;
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t parity = 0;
    __shared__ int cont;   // thread 0: the next tile is already staged (gang continuation)
    __shared__ int gpass;  // thread 0: passes the CTA has run with its gang tile
    // Bulk-ring tickets still held (pend_t, pend_t + 1, ...).  Thread 0 owns
    // them, except between run_tile and the next barrier, when thread 32 may
    // take the first one (and stage its tile, setting ngot/nitem) while
    // thread 0, busy recording the tile, does not touch them.
    __shared__ int pend;
    __shared__ unsigned pend_t;
    if (threadIdx.x == 0) {
        cont = 0;
        gpass = 0;
        pend = 0;
        pend_t = 0;
    }
    for (;;) {
        if (threadIdx.x == 0) {
            int g = cont;
            bool staged = false;
            if (!cont && ngot) {  // a held ticket's tile, staged by thread 32 during the bookkeeping
                item = nitem;
                ngot = 0;
                g = 1;
                gpass = 0;
                staged = true;
            } else if (!cont) {
                const unsigned long long t_end = globaltimer() + (unsigned long long)S->timeout_ns;
                for (int spin = 0;; spin++) {
                    unsigned t = 0;
                    int r = -1;
                    // held bulk tickets are consumed before anything else: a
                    // CTA that took a ring-0 (gang) ticket while holding bulk
                    // tickets could keep a 2D wave from finishing while its
                    // gang waits for members the wave's waiters would supply
                    if (pend) {  // next held ticket of the last multiple claim
                        r = 1;
                        t = pend_t;
                        pend -= 1;
                        pend_t = t + 1;
                    } else {
                        // both rings' counters in one round trip; ring 0 first
                        const unsigned h0 = ld_volatile_u(&S->ring[0].head), t0 = ld_volatile_u(&S->ring[0].tail);
                        const unsigned h1 = ld_volatile_u(&S->ring[1].head), t1 = ld_volatile_u(&S->ring[1].tail);
                        if ((int)(t0 - h0) > 0) {
                            t = atomicAdd(&S->ring[0].head, 1u);
                            r = 0;
                        } else if ((int)(t1 - h1) >= 2 * (int)gridDim.x) {
                            // deep bulk ring: k consecutive tickets for one
                            // fetch-and-add (k = items per CTA in the ring, at most
                            // kMaxClaim); each held ticket is waited for only after
                            // the tile before it is done
                            const int k = min(kMaxClaim, (int)(t1 - h1) / (int)gridDim.x);
                            t = atomicAdd(&S->ring[1].head, (unsigned)k);
                            r = 1;
                            pend = k - 1;
                            pend_t = t + 1;
                        } else if ((int)(t1 - h1) > 0) {
                            t = atomicAdd(&S->ring[1].head, 1u);
                            r = 1;
                        }
                    }
                    if (r >= 0) {
                        int4 it;
                        const int w = wait_ticket(S, r, t, it, t_end);
                        if (w < 0) {
                            atomicOr(&S->status, kErrQueueTimeout);
                            break;
                        }
                        if (w == 0) continue;  // abandoned: that ring is finished
                        item = it;
                        g = 1;
                        gpass = 0;
                        break;
                    }
                    if (ld_acquire(&S->live) == 0) break;
                    if ((spin & 63) == 63 && globaltimer() > t_end) {
                        atomicOr(&S->status, kErrQueueTimeout);
                        break;
                    }
                    __nanosleep(spin < 32 ? 20 : 200);
                }
            }
            if (g && !staged) issue_tile(insts[item.x], item.z, item.y, smem, &bar);
            got = g;
        }
        __syncthreads();
        if (!got) break;
        const int ii = item.x, tile = item.y, q = item.z, nwave = item.w & ~kItemGang;
        const bool gang_tile = (item.w & kItemGang) != 0;
        Inst &in = insts[ii];
        if (!mbar_wait_bounded(&bar, parity)) {
            if (threadIdx.x == 0) atomicOr(&S->status, kErrTmaTimeout);
        }
        parity ^= 1u;
        const uint32_t m = run_tile(in, q, tile, smem, &band);  // ends with a barrier: smem is free again
        if (threadIdx.x == 32 && pend > 0 && !(gang_tile && q % 6 != 5)) {
            // while thread 0 records this tile, stage the next held ticket's
            // tile if its item is already there (one look, no waiting)
            int4 it;
            if (poll_ticket(S, 1, pend_t, it)) {
                pend -= 1;
                pend_t += 1;
                nitem = it;
                ngot = 1;
                issue_tile(insts[it.x], it.z, it.y, smem, &bar);
            }
        }
        if (threadIdx.x == 0) {
            if (m & kTileChanged) {
                in.lc[tile] = q;
                if (in.dims == 2) in.act[tile] = (uint8_t)(m & kAllBands);  // bands the next wave reads
            }
            __threadfence();
            cont = 0;
            last = 0;
            if (gang_tile && q % 6 != 5) {
                // gang: once every member has finished pass q, take the same
                // tile in pass q + 1 without going through the ring
                atomicAdd(&in.gang, 1);
                atomicAdd(&in.tiles_run, 1ull);
                atomicAdd(&in.work_words, (unsigned long long)tile_core_words(in, tile));
                gpass += 1;
                if (wait_at_least(&in.gang, nwave * gpass, S)) {
                    item.z = q + 1;  // staged at the top of the loop
                    cont = 1;
                } else {
                    atomicOr(&S->status, kErrQueueTimeout);
                }
            } else {
                const int d = atomicAdd(&in.done, 1);
                last = d == nwave - 1;
                if (last && gang_tile) atomicAdd(&S->gang_budget, nwave);  // the gang dissolves
                atomicAdd(&in.tiles_run, 1ull);
                atomicAdd(&in.work_words, (unsigned long long)tile_core_words(in, tile));
            }
        }
        __syncthreads();
        if (last) {
            __threadfence();
            next_wave(S, insts, ii, q + 1, nwave, scratch, kEngineScratchWords);
        }
        __syncthreads();
    }
}

int engine_max_blocks_per_sm(int smem)
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel, kThreads, engine_smem_bytes(smem));
    return n;
}

cudaError_t engine_set_smem(int smem)
{
    cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         engine_smem_bytes(smem));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(plain_pass_dev_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem + 128);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(plain_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem + 128);
}

cudaError_t launch_engine(int grid, int smem, Inst *d_insts, int ninst, Sched *d_sched, cudaStream_t st)
{
    engine_seed_kernel<<<std::min(ninst, 148 * 8), kThreads, 0, st>>>(d_insts, ninst, d_sched);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    engine_kernel<<<grid, kThreads, engine_smem_bytes(smem), st>>>(d_insts, d_sched, smem / 4);
    return cudaGetLastError();
}

}  // namespace bgt
