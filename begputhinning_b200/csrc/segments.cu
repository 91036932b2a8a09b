// segments.cu -- ExtractSegmentsV on the device (2D/ExtractSegments.cpp:16-127,
// 3D/ExtractSegments.cpp:135-251), bit-exact in content and order.
//
// The reference walk is sequential in raster order, but a walk only reads and
// writes the neighbour values of points of its own 8-/26-connected component
// (it moves to neighbours whose value is nonzero, and only points carry
// nonzero values), and raster order restricted to a component is preserved.
// So components are traced independently, one warp each:
//   1. classify (one thread per packed word, bit-sliced neighbour counts):
//      value map V = 2 for points with exactly two foreground neighbours,
//      -max(n,1) otherwise, 0 for background and frame pixels; count nodes
//      (V < 0) per word;
//   2. node list in raster order (prefix sum over the per-word counts);
//   3. connected components of the points (union-find with atomics);
//   4. nodes grouped by component, raster order kept (stable radix sort);
//   5. a warp per component replays the reference walk; the lanes read the
//      8/26 neighbour values in parallel and a ballot picks the first nonzero
//      one in the reference's scan order.  The walk runs twice: once counting
//      segments and points per start node, then (after a prefix sum over the
//      nodes in raster order, which is the reference's emission order)
//      writing every segment straight to its final position.
#include <cub/cub.cuh>

#include <cstdio>
#include <vector>

#include "host.h"
#include "kernels.cuh"

namespace bgt {

// --------------------------------------------------------- classify -------
// bit-sliced counter: add one bit-word x to the counter c[0..NB)
template <int NB>
__device__ __forceinline__ void csa_add(uint32_t (&c)[NB], uint32_t x)
{
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const uint32_t t = c[i] & x;
        c[i] ^= x;
        x = t;
    }
}

__device__ __forceinline__ uint32_t word_at(const uint32_t *buf, int P, int H, int D, int z, int y, int j)
{
    if (z < 0 || z >= D || y < 0 || y >= H || j < 0 || j >= P) return 0u;
    return __ldg(buf + ((size_t)z * H + y) * P + j);
}

// interior mask of word j of a row: bits with 1 <= x <= W-2
__device__ __forceinline__ uint32_t interior_bits(int W, int j)
{
    const int x0 = j * 32;
    uint32_t m = 0xffffffffu;
    if (x0 == 0) m &= ~1u;
    const int last = W - 2 - x0;  // highest allowed bit
    if (last < 0) return 0u;
    if (last < 31) m &= (2u << last) - 1u;
    return m;
}

template <int DIMS>
__global__ void classify_kernel(const uint32_t *__restrict__ buf, int W, int H, int D, int P,
                                int8_t *__restrict__ V, int *__restrict__ node_count)
{
    const int wwords = (W + 31) >> 5;
    const long long nw = (long long)H * D * wwords;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / wwords;
        const int j = (int)(i - row * wwords);
        const int y = (int)(row % H), z = (int)(row / H);
        const uint32_t c = word_at(buf, P, H, D, z, y, j);
        uint32_t pts = c & interior_bits(W, j);
        if (y == 0 || y == H - 1) pts = 0;
        if (DIMS == 3 && (z == 0 || z == D - 1)) pts = 0;
        constexpr int NB = DIMS == 2 ? 4 : 5;
        uint32_t cnt[NB] = {};
        const int zlo = DIMS == 3 ? -1 : 0, zhi = DIMS == 3 ? 1 : 0;
        if (pts) {
            for (int dz = zlo; dz <= zhi; dz++)
                for (int dy = -1; dy <= 1; dy++) {
                    const uint32_t l = word_at(buf, P, H, D, z + dz, y + dy, j - 1);
                    const uint32_t m = word_at(buf, P, H, D, z + dz, y + dy, j);
                    const uint32_t r = word_at(buf, P, H, D, z + dz, y + dy, j + 1);
                    csa_add<NB>(cnt, at_xm1(m, l));
                    if (dz != 0 || dy != 0) csa_add<NB>(cnt, m);
                    csa_add<NB>(cnt, at_xp1(m, r));
                }
        }
        // exactly two neighbours
        uint32_t eq2 = ~cnt[0] & cnt[1] & ~cnt[2] & ~cnt[3];
        if (NB == 5) eq2 &= ~cnt[NB - 1];
        const uint32_t nodes = pts & ~eq2;
        node_count[i] = __popc(nodes);
        int8_t *vrow = V + ((size_t)z * H + y) * W + (size_t)j * 32;
        const int nb = min(32, W - j * 32);
        for (int b = 0; b < nb; b++) {
            int8_t v = 0;
            if ((pts >> b) & 1u) {
                int n = 0;
#pragma unroll
                for (int k = 0; k < NB; k++) n |= (int)((cnt[k] >> b) & 1u) << k;
                v = (int8_t)(n == 2 ? 2 : -(n == 0 ? 1 : n));
            }
            vrow[b] = v;
        }
    }
}

// node raster indices in raster order; offs = exclusive scan of node_count
template <int DIMS>
__global__ void emit_nodes_kernel(const uint32_t *__restrict__ buf, int W, int H, int D, int P,
                                  const int8_t *__restrict__ V, const int *__restrict__ offs,
                                  uint32_t *__restrict__ nodes)
{
    const int wwords = (W + 31) >> 5;
    const long long nw = (long long)H * D * wwords;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / wwords;
        const int j = (int)(i - row * wwords);
        const size_t base = (size_t)row * W + (size_t)j * 32;
        const int nb = min(32, W - j * 32);
        int o = offs[i];
        for (int b = 0; b < nb; b++)
            if (V[base + b] < 0) nodes[o++] = (uint32_t)(base + b);
    }
}

// ------------------------------------------------------------- CCL --------
__device__ __forceinline__ uint32_t uf_find(uint32_t *par, uint32_t x)
{
    for (;;) {
        const uint32_t p = __ldcg(par + x);
        if (p == x) return x;
        const uint32_t g = __ldcg(par + p);
        if (g != p) atomicCAS(par + x, p, g);  // path halving
        x = p;
    }
}

__device__ __forceinline__ void uf_union(uint32_t *par, uint32_t a, uint32_t b)
{
    for (int guard = 0; guard < 1 << 20; guard++) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (a < b) { const uint32_t t = a; a = b; b = t; }  // hook the larger root under the smaller
        const uint32_t old = atomicCAS(par + a, a, b);
        if (old == a) return;
        a = old;
    }
}

__global__ void uf_init_kernel(const int8_t *__restrict__ V, uint32_t *par, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        par[i] = V[i] != 0 ? (uint32_t)i : 0xffffffffu;
}

// union every point with its point neighbours that precede it in raster order
template <int DIMS>
__global__ void uf_hook_kernel(const int8_t *__restrict__ V, int W, int H, int D, uint32_t *par)
{
    const long long n = (long long)W * H * D;
    const long long slice = (long long)W * H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (V[i] == 0) continue;
        // points are interior, so every neighbour index is in range
        const int zlo = DIMS == 3 ? -1 : 0;
        for (int dz = zlo; dz <= 0; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const long long off = dz * slice + (long long)dy * W + dx;
                    if (off >= 0) continue;  // only predecessors
                    if (V[i + off] != 0) uf_union(par, (uint32_t)i, (uint32_t)(i + off));
                }
    }
}

__global__ void node_keys_kernel(uint32_t *par, const uint32_t *__restrict__ nodes, int nn,
                                 uint32_t *__restrict__ keys)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        keys[i] = uf_find(par, nodes[i]);
}

// component starts in the sorted node list: flags[i] = key changes at i
__global__ void comp_flags_kernel(const uint32_t *__restrict__ keys, int nn, int *__restrict__ flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void comp_starts_kernel(const int *__restrict__ flag, const int *__restrict__ pos, int nn,
                                   int *__restrict__ starts)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        if (flag[i]) starts[pos[i]] = i;
}

// ------------------------------------------------------------- walk -------
struct WalkOut {
    // count pass
    int *nseg;   // [nn] per node (indexed by position in the raster-ordered list)
    int *npts;   // [nn]
    // emit pass
    const int *seg_off;  // [nn] exclusive scan of nseg
    const int *pt_off;   // [nn] exclusive scan of npts
    int32_t *start;      // [nseg_total + 1]
    uint8_t *is_end;     // [nseg_total]
    int16_t *px, *py, *pz;
};

template <int DIMS, bool EMIT>
__global__ void walk_kernel(int8_t *V, const int8_t *__restrict__ V0, int W, int H,
                            const uint32_t *__restrict__ sorted_nodes, const uint32_t *__restrict__ sorted_rank,
                            const int *__restrict__ comp_start, int ncomp, int nn, WalkOut out)
{
    constexpr int ND = DIMS == 2 ? 8 : 26;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const long long slice = (long long)W * H;
    // this lane's neighbour offset in the reference's scan order
    long long my_off = 0;
    {
        int q = 0;
        const int zlo = DIMS == 3 ? -1 : 0, zhi = DIMS == 3 ? 1 : 0;
        for (int dz = zlo; dz <= zhi; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (!dz && !dy && !dx) continue;
                    if (q == lane) my_off = dz * slice + (long long)dy * W + dx;
                    q++;
                }
    }
    const unsigned lane_ok = lane < ND ? 1u : 0u;
    for (int comp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; comp < ncomp; comp += warps) {
        const int a = comp_start[comp];
        const int b = comp + 1 < ncomp ? comp_start[comp + 1] : nn;
        for (int k = a; k < b; k++) {
            const long long p = sorted_nodes[k];
            const int rank = (int)sorted_rank[k];  // position in raster-ordered node list
            const int vp = V[p];
            __syncwarp();
            if (vp >= 0) {
                if (!EMIT && lane == 0) {
                    out.nseg[rank] = 0;
                    out.npts[rank] = 0;
                }
                continue;
            }
            if (lane == 0) V[p] = 0;
            __syncwarp();
            int ni = -1;
            int segs = 0, pts = 0;
            int so = EMIT ? out.seg_off[rank] : 0, po = EMIT ? out.pt_off[rank] : 0;
            auto put = [&](long long t) {
                if (EMIT && lane == 0) {
                    out.px[po] = (int16_t)(t % W);
                    out.py[po] = (int16_t)((t / W) % H);
                    if (DIMS == 3) out.pz[po] = (int16_t)(t / slice);
                }
                po++;
                pts++;
            };
            for (int br = 0; br < -vp; br++) {
                int is_end = V0[p] > -2 && V0[p] < 2;
                if (EMIT && lane == 0) out.start[so] = po;
                put(p);
                // first neighbour after ni in scan order with a nonzero value
                const unsigned m = __ballot_sync(kFull, lane_ok && lane > ni && V[p + my_off] != 0);
                ni = m ? __ffs(m) - 1 : ND;
                if (ni < ND) {
                    long long t = p + __shfl_sync(kFull, my_off, ni);
                    for (int guard = 0; guard < (1 << 30); guard++) {
                        if (V[t] != 2) break;
                        __syncwarp();
                        if (lane == 0) V[t] = 0;
                        __syncwarp();
                        put(t);
                        const unsigned m2 = __ballot_sync(kFull, lane_ok && V[t + my_off] != 0);
                        if (m2) t += __shfl_sync(kFull, my_off, __ffs(m2) - 1);
                    }
                    put(t);
                    if (V0[t] > -2 && V0[t] < 2) is_end = 1;
                    __syncwarp();
                    if (lane == 0) V[t] = (int8_t)(V[t] + 1);
                    __syncwarp();
                }
                if (EMIT && lane == 0) out.is_end[so] = (uint8_t)is_end;
                so++;
                segs++;
            }
            if (!EMIT && lane == 0) {
                out.nseg[rank] = segs;
                out.npts[rank] = pts;
            }
        }
    }
}

__global__ void iota_kernel(uint32_t *a, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = (uint32_t)i;
}

__global__ void gather_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx,
                              uint32_t *__restrict__ dst, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

static size_t align16(size_t v) { return (v + 15) / 16 * 16; }

static int grid_of(long long n, int block = 256)
{
    long long g = (n + block - 1) / block;
    return (int)std::max(1LL, std::min(g, 148LL * 16));
}

// Exclusive sum via CUB; temp storage from scratch slot `slot`.
cudaError_t exscan(bgt_ctx *c, int slot, const int *in, int *out, long long n, cudaStream_t st)
{
    size_t tb = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, st);
    if (e != cudaSuccess) return e;
    void *tmp = nullptr;
    if (ctx_scratch(c, slot, tb, &tmp) != BGT_OK) return cudaErrorMemoryAllocation;
    return cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int)n, st);
}

// Device segment extraction on a packed image (P words per row, H rows, D
// planes; W x H x D pixels).  The segment arrays stay in the context's
// scratch (slot 19) until the next extraction on the context.
int segments_device_arrays(bgt_ctx *c, int dims, const uint32_t *d_buf, int W, int H, int D, int P, DevSegs *out)
{
    cudaStream_t st = c->stream;
    const long long npx = (long long)W * H * D;
    if (npx >= (1LL << 32) - 1) return fail(BGT_ERR_LIMIT, "segment extraction limited to < 2^32 pixels");
    const long long nw = (long long)H * D * ((W + 31) / 32);
    // scratch slots: 1 V, 2 V0, 3 node_count, 4 node offs, 5 nodes, 6 par, 7 keys, 8 keys_sorted,
    // 9 vals(rank), 10 vals_sorted, 11 flags, 12 flag pos, 13 comp starts, 14 cub temp,
    // 15 nseg, 16 npts, 17 seg_off, 18 pt_off, 19 out arrays
    void *p1, *p2, *p3, *p4, *p6;
    int rc;
    if ((rc = ctx_scratch(c, 1, npx, &p1)) || (rc = ctx_scratch(c, 2, npx, &p2)) ||
        (rc = ctx_scratch(c, 3, (nw + 1) * 4, &p3)) || (rc = ctx_scratch(c, 4, (nw + 1) * 4, &p4)) ||
        (rc = ctx_scratch(c, 6, npx * 4, &p6)))
        return rc;
    int8_t *V = (int8_t *)p1, *V0 = (int8_t *)p2;
    int *cnt = (int *)p3, *offs = (int *)p4;
    uint32_t *par = (uint32_t *)p6;
    cudaError_t e;
    if (dims == 2)
        classify_kernel<2><<<grid_of(nw), 256, 0, st>>>(d_buf, W, H, D, P, V, cnt);
    else
        classify_kernel<3><<<grid_of(nw), 256, 0, st>>>(d_buf, W, H, D, P, V, cnt);
    cudaMemcpyAsync(V0, V, npx, cudaMemcpyDeviceToDevice, st);  // the reference's "onn"
    cudaMemsetAsync(cnt + nw, 0, 4, st);
    if ((e = exscan(c, 14, cnt, offs, nw + 1, st)) != cudaSuccess) return cuda_fail(e, "node scan");
    int nn = 0;
    if ((e = cudaMemcpyAsync(&nn, offs + nw, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "node count");
    *out = DevSegs();
    if (nn == 0) return BGT_OK;
    void *p5, *p7, *p8, *p9, *p10, *p11, *p12, *p13, *p15, *p16, *p17, *p18;
    if ((rc = ctx_scratch(c, 5, (size_t)nn * 4, &p5)) || (rc = ctx_scratch(c, 7, (size_t)nn * 4, &p7)) ||
        (rc = ctx_scratch(c, 8, (size_t)nn * 4, &p8)) || (rc = ctx_scratch(c, 9, (size_t)nn * 4, &p9)) ||
        (rc = ctx_scratch(c, 10, (size_t)nn * 4, &p10)) || (rc = ctx_scratch(c, 11, (size_t)(nn + 1) * 4, &p11)) ||
        (rc = ctx_scratch(c, 12, (size_t)(nn + 1) * 4, &p12)) || (rc = ctx_scratch(c, 13, (size_t)nn * 4, &p13)) ||
        (rc = ctx_scratch(c, 15, (size_t)(nn + 1) * 4, &p15)) || (rc = ctx_scratch(c, 16, (size_t)(nn + 1) * 4, &p16)) ||
        (rc = ctx_scratch(c, 17, (size_t)(nn + 1) * 4, &p17)) || (rc = ctx_scratch(c, 18, (size_t)(nn + 1) * 4, &p18)))
        return rc;
    uint32_t *nodes = (uint32_t *)p5, *keys = (uint32_t *)p7, *keys_s = (uint32_t *)p8;
    uint32_t *rank = (uint32_t *)p9, *rank_s = (uint32_t *)p10;
    int *flag = (int *)p11, *fpos = (int *)p12, *cstart = (int *)p13;
    int *nseg = (int *)p15, *npts = (int *)p16, *seg_off = (int *)p17, *pt_off = (int *)p18;
    if (dims == 2)
        emit_nodes_kernel<2><<<grid_of(nw), 256, 0, st>>>(d_buf, W, H, D, P, V, offs, nodes);
    else
        emit_nodes_kernel<3><<<grid_of(nw), 256, 0, st>>>(d_buf, W, H, D, P, V, offs, nodes);
    // components
    uf_init_kernel<<<grid_of(npx), 256, 0, st>>>(V, par, npx);
    if (dims == 2)
        uf_hook_kernel<2><<<grid_of(npx), 256, 0, st>>>(V, W, H, D, par);
    else
        uf_hook_kernel<3><<<grid_of(npx), 256, 0, st>>>(V, W, H, D, par);
    node_keys_kernel<<<grid_of(nn), 256, 0, st>>>(par, nodes, nn, keys);
    iota_kernel<<<grid_of(nn), 256, 0, st>>>(rank, nn);
    // stable sort of (component, rank): keeps raster order inside a component
    {
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys_s, rank, rank_s, nn, 0, 32, st);
        void *tmp;
        if ((rc = ctx_scratch(c, 14, tb, &tmp))) return rc;
        if ((e = cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys_s, rank, rank_s, nn, 0, 32, st)) != cudaSuccess)
            return cuda_fail(e, "component sort");
    }
    comp_flags_kernel<<<grid_of(nn), 256, 0, st>>>(keys_s, nn, flag);
    cudaMemsetAsync(flag + nn, 0, 4, st);
    if ((e = exscan(c, 14, flag, fpos, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "component scan");
    comp_starts_kernel<<<grid_of(nn), 256, 0, st>>>(flag, fpos, nn, cstart);
    int ncomp = 0;
    if ((e = cudaMemcpyAsync(&ncomp, fpos + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "component count");
    // sorted node raster indices nodes[rank_s[k]] (keys are no longer needed)
    uint32_t *snodes = keys;
    gather_kernel<<<grid_of(nn), 256, 0, st>>>(nodes, rank_s, snodes, nn);
    // walk 1: count segments and points per start node
    WalkOut wo{};
    wo.nseg = nseg;
    wo.npts = npts;
    const int wgrid = (int)std::min<long long>(((long long)ncomp * 32 + 255) / 256, 148LL * 16);
    if (dims == 2)
        walk_kernel<2, false><<<wgrid, 256, 0, st>>>(V, V0, W, H, snodes, rank_s, cstart, ncomp, nn, wo);
    else
        walk_kernel<3, false><<<wgrid, 256, 0, st>>>(V, V0, W, H, snodes, rank_s, cstart, ncomp, nn, wo);
    cudaMemsetAsync(nseg + nn, 0, 4, st);
    cudaMemsetAsync(npts + nn, 0, 4, st);
    if ((e = exscan(c, 14, nseg, seg_off, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "segment scan");
    if ((e = exscan(c, 14, npts, pt_off, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "point scan");
    int tot[2] = {0, 0};
    if ((e = cudaMemcpyAsync(&tot[0], seg_off + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[1], pt_off + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "segment totals");
    const int S = tot[0], Np = tot[1];
    // output block: start[S+1] int32, is_end[S] u8, px, py (pz) int16[Np]
    const size_t o_start = 0, o_end = align16((size_t)(S + 1) * 4), o_px = o_end + align16((size_t)S + 1),
                 o_py = o_px + align16((size_t)Np * 2 + 2), o_pz = o_py + align16((size_t)Np * 2 + 2),
                 o_tot = o_pz + align16((size_t)Np * 2 + 2);
    void *p19;
    if ((rc = ctx_scratch(c, 19, o_tot, &p19))) return rc;
    char *ob = (char *)p19;
    wo.seg_off = seg_off;
    wo.pt_off = pt_off;
    wo.start = (int32_t *)(ob + o_start);
    wo.is_end = (uint8_t *)(ob + o_end);
    wo.px = (int16_t *)(ob + o_px);
    wo.py = (int16_t *)(ob + o_py);
    wo.pz = (int16_t *)(ob + o_pz);
    // walk 2 from the original values: write every segment at its final place
    cudaMemcpyAsync(V, V0, npx, cudaMemcpyDeviceToDevice, st);
    if (dims == 2)
        walk_kernel<2, true><<<wgrid, 256, 0, st>>>(V, V0, W, H, snodes, rank_s, cstart, ncomp, nn, wo);
    else
        walk_kernel<3, true><<<wgrid, 256, 0, st>>>(V, V0, W, H, snodes, rank_s, cstart, ncomp, nn, wo);
    cudaMemcpyAsync(wo.start + S, pt_off + nn, 4, cudaMemcpyDeviceToDevice, st);
    out->nseg = S;
    out->npts = Np;
    out->start = wo.start;
    out->is_end = wo.is_end;
    out->px = wo.px;
    out->py = wo.py;
    out->pz = dims == 3 ? wo.pz : nullptr;
    return BGT_OK;
}

// The same, with the segment arrays copied to host memory (malloc).
int segments_packed(bgt_ctx *c, int dims, const uint32_t *d_buf, int W, int H, int D, int P, HostSegs *out)
{
    DevSegs ds;
    int rc = segments_device_arrays(c, dims, d_buf, W, H, D, P, &ds);
    if (rc != BGT_OK) return rc;
    cudaStream_t st = c->stream;
    const int S = ds.nseg, Np = ds.npts;
    *out = HostSegs();
    out->nseg = S;
    out->npts = Np;
    out->start = (int32_t *)malloc((size_t)(S + 1) * 4);
    out->is_end = (uint8_t *)malloc((size_t)S + 1);
    out->px = (int16_t *)malloc((size_t)Np * 2 + 2);
    out->py = (int16_t *)malloc((size_t)Np * 2 + 2);
    out->pz = dims == 3 ? (int16_t *)malloc((size_t)Np * 2 + 2) : nullptr;
    if (!out->start || !out->is_end || !out->px || !out->py || (dims == 3 && !out->pz))
        return fail(BGT_ERR_NOMEM, "host allocation of segment arrays");
    if (S == 0) {
        out->start[0] = 0;
        return BGT_OK;
    }
    cudaError_t e = cudaMemcpyAsync(out->start, ds.start, (size_t)(S + 1) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out->is_end, ds.is_end, (size_t)S, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out->px, ds.px, (size_t)Np * 2, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out->py, ds.py, (size_t)Np * 2, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && dims == 3)
        e = cudaMemcpyAsync(out->pz, ds.pz, (size_t)Np * 2, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "segment readback");
    return BGT_OK;
}

void free_host_segs(HostSegs *s)
{
    free(s->start);
    free(s->is_end);
    free(s->px);
    free(s->py);
    free(s->pz);
    *s = HostSegs();
}

}  // namespace bgt
