// segments.cu -- ExtractSegmentsV on the device (2D/ExtractSegments.cpp:16-127,
// 3D/ExtractSegments.cpp:135-251), bit-exact in content and order.
//
//   1. classify (one thread per packed word, bit-sliced neighbour counts):
//      value map V = 2 for points with exactly two foreground neighbours,
//      -max(n,1) otherwise (nodes), 0 for background and frame pixels;
//   2. node list in raster order (prefix sum over per-word node counts);
//   3. node-parallel walk (node_walk_kernel): chains of two-neighbour points
//      are followed once, in parallel, into per-end pixel lists; each node
//      replays the reference's visit (budget, scan order, chain walks, +1 on
//      the node a walk ends at) as soon as the nodes it reaches through one
//      chain or one step and that precede it in raster order have run;
//      outputs go to per-node ranges and are placed in raster order of their
//      nodes, the reference's emission order;
//   4. if anything falls outside the rules that step 3 relies on, the image
//      is redone by the per-component pixel walk: components (union-find with
//      atomics), nodes grouped by component in raster order (stable radix
//      sort), and a warp per component replaying the reference walk pixel by
//      pixel (the lanes read the 8/26 neighbour values, a ballot picks the
//      first nonzero one in the reference's scan order).
#include <cub/cub.cuh>

#include <cstdio>
#include <cstdlib>
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
    int *nseg;   // [nn] per node (indexed by position in the raster-ordered list)
    int *npts;   // [nn]
    int *tpo;    // [nn] the node's first point in the temporary arrays
    int *tso;    // [nn] the node's first segment in the temporary arrays
    const int *cpb;  // [ncomp+1] each component's first point in the temporary arrays
    const int *csb;  // [ncomp+1] each component's first segment
    int16_t *tx, *ty, *tz;  // temporary points in emission order, per component
    int32_t *trel;          // temporary segment starts (point index within the node's output)
    uint8_t *tend;          // temporary is_end flags
    int *err;               // kErrSegOverflow when a component outgrows its bound
};

// One warp per component replays the reference's walk over the component's
// nodes in raster order (lanes read the 8/26 neighbours, a ballot picks the
// first nonzero one in the reference's scan order).  Writes to the value map
// are kept to the pixels that anything can look at again: a walk along a
// chain zeroes its first and last chain pixels and every original node it
// passes; the chain pixels in between (nn == 2, both neighbours on the same
// walk) are skipped, because only a walk standing next to them could read
// them and the chain is never entered again (its ends are zero).  The walk
// excludes the pixel it came from, which the reference has zeroed.  A stall
// (no nonzero neighbour) zeroes the pixel before it, so that the stalled
// pixel's later walks see it as the reference does.  Coordinates follow the
// steps instead of being divided out of the raster index.
template <int DIMS>
__global__ void walk_kernel(int8_t *V, const int8_t *__restrict__ V0, int W, int H,
                            const uint32_t *__restrict__ sorted_nodes, const uint32_t *__restrict__ sorted_rank,
                            const int *__restrict__ comp_start, int ncomp, int nn, WalkOut out)
{
    constexpr int ND = DIMS == 2 ? 8 : 26;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const long long slice = (long long)W * H;
    // this lane's neighbour offset in the reference's scan order, and its
    // (dx, dy, dz) packed as (dz+1)*9 + (dy+1)*3 + (dx+1)
    long long my_off = 0;
    int my_d = 13;
    {
        int q = 0;
        const int zlo = DIMS == 3 ? -1 : 0, zhi = DIMS == 3 ? 1 : 0;
        for (int dz = zlo; dz <= zhi; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (!dz && !dy && !dx) continue;
                    if (q == lane) {
                        my_off = dz * slice + (long long)dy * W + dx;
                        my_d = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                    }
                    q++;
                }
    }
    const unsigned lane_ok = lane < ND ? 1u : 0u;
    for (int comp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; comp < ncomp; comp += warps) {
        const int a = comp_start[comp];
        const int b = comp + 1 < ncomp ? comp_start[comp + 1] : nn;
        // the component's outputs go to its own temporary range, in emission order
        int po = out.cpb[comp], so = out.csb[comp];
        const int po_end = out.cpb[comp + 1], so_end = out.csb[comp + 1];
        for (int k = a; k < b; k++) {
            const long long p = sorted_nodes[k];
            const int rank = (int)sorted_rank[k];  // position in raster-ordered node list
            const int vp = V[p];
            __syncwarp();
            if (lane == 0) {
                out.tpo[rank] = po;
                out.tso[rank] = so;
            }
            if (vp >= 0) {
                if (lane == 0) {
                    out.nseg[rank] = 0;
                    out.npts[rank] = 0;
                }
                continue;
            }
            if (lane == 0) V[p] = 0;
            __syncwarp();
            const int p_x = (int)(p % W), p_y = (int)((p / W) % H), p_z = DIMS == 3 ? (int)(p / slice) : 0;
            int ni = -1;
            int segs = 0, pts = 0;
            int cx = p_x, cy = p_y, cz = p_z;
            auto put = [&]() {
                if (lane == 0) {
                    if (po < po_end) {
                        out.tx[po] = (int16_t)cx;
                        out.ty[po] = (int16_t)cy;
                        if (DIMS == 3) out.tz[po] = (int16_t)cz;
                    } else {
                        atomicOr(out.err, kErrSegOverflow);
                    }
                }
                po++;
                pts++;
            };
            auto step = [&](int s) {  // move the coordinates by the delta of scan index s
                const int d = __shfl_sync(kFull, my_d, s);
                cx += d % 3 - 1;
                cy += (d / 3) % 3 - 1;
                cz += d / 9 - 1;
                return __shfl_sync(kFull, my_off, s);
            };
            const int v0p = V0[p];
            for (int br = 0; br < -vp; br++) {
                int is_end = v0p > -2 && v0p < 2;
                const int seg_rel = pts;
                cx = p_x;
                cy = p_y;
                cz = p_z;
                put();
                // first neighbour after ni in scan order with a nonzero value;
                // every lane loads its neighbour's current and original value
                // at once, and the chosen one's reach the warp by shuffles
                int vn = lane_ok ? V[p + my_off] : 0, v0n = lane_ok ? V0[p + my_off] : 0;
                const unsigned m = __ballot_sync(kFull, lane_ok && lane > ni && vn != 0);
                ni = m ? __ffs(m) - 1 : ND;
                if (ni < ND) {
                    long long prev = p;
                    int back = ND - 1 - ni;  // scan index of the step back to prev
                    int vt = __shfl_sync(kFull, vn, ni), v0t = __shfl_sync(kFull, v0n, ni);
                    long long t = p + step(ni);
                    bool first = true, stall = false;
                    for (int guard = 0; guard < (1 << 30); guard++) {
                        if (vt != 2) break;
                        put();
                        vn = lane_ok ? V[t + my_off] : 0;
                        v0n = lane_ok ? V0[t + my_off] : 0;
                        const unsigned m2 = __ballot_sync(kFull, lane_ok && lane != back && vn != 0);
                        if (!m2) {
                            stall = true;
                            break;
                        }
                        if (lane == 0 && (first || v0t != 2)) V[t] = 0;
                        const int s2 = __ffs(m2) - 1;
                        prev = t;
                        back = ND - 1 - s2;
                        vt = __shfl_sync(kFull, vn, s2);
                        v0t = __shfl_sync(kFull, v0n, s2);
                        t += step(s2);
                        first = false;
                        __syncwarp();
                    }
                    __syncwarp();
                    // the last chain pixel (prev, unless the walk never left p) becomes zero in memory too
                    if (lane == 0 && prev != p) V[prev] = 0;
                    __syncwarp();
                    put();
                    if (v0t > -2 && v0t < 2) is_end = 1;
                    // a stalled walk stays on t, which the reference zeroed: it becomes 1
                    if (lane == 0) V[t] = stall ? (int8_t)1 : (int8_t)(vt + 1);
                    __syncwarp();
                }
                if (lane == 0) {
                    if (so < so_end) {
                        out.trel[so] = seg_rel;
                        out.tend[so] = (uint8_t)is_end;
                    } else {
                        atomicOr(out.err, kErrSegOverflow);
                    }
                }
                so++;
                segs++;
            }
            if (lane == 0) {
                out.nseg[rank] = segs;
                out.npts[rank] = pts;
            }
        }
    }
}

// fg pixels per union-find root (the component's pixel count)
__global__ void comp_px_kernel(const int8_t *__restrict__ V, uint32_t *par, long long n, uint32_t *cnt)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (V[i] != 0) atomicAdd(cnt + uf_find(par, (uint32_t)i), 1u);
}

// per component: branches = sum of |v| over its nodes (a bound on its
// segments), pixels from its root
__global__ void comp_sums_kernel(const int8_t *__restrict__ V0, const uint32_t *__restrict__ snodes,
                                 const uint32_t *__restrict__ keys_s, const int *__restrict__ flag,
                                 const int *__restrict__ fpos, const uint32_t *__restrict__ cnt, int nn,
                                 int *branches, int *px)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const int c = fpos[i] + flag[i] - 1;
        atomicAdd(branches + c, -(int)V0[snodes[i]]);
        if (flag[i]) px[c] = (int)cnt[keys_s[i]];
    }
}

// bounds of a component's output: segments <= branches; points <= pixels +
// 3 * branches (each branch adds its start and end point, and a pixel is
// walked through again only after two walks ended on it)
__global__ void comp_bounds_kernel(const int *__restrict__ branches, const int *__restrict__ px, int ncomp,
                                   int *bpts, int *bsegs)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncomp; c += gridDim.x * blockDim.x) {
        bpts[c] = c < ncomp ? px[c] + 3 * branches[c] : 0;
        bsegs[c] = c < ncomp ? branches[c] : 0;
    }
}

// Move each node's output from its component's temporary range to its place
// in the reference's emission order (one warp per node).
template <int DIMS>
__global__ void place_kernel(const WalkOut w, const int *__restrict__ seg_off, const int *__restrict__ pt_off,
                             int nn, int32_t *start, uint8_t *is_end, int16_t *px, int16_t *py, int16_t *pz,
                             bool ranged)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nn; r += warps) {
        int np = w.npts[r], ns = w.nseg[r];
        if (ranged) {  // node-parallel walk: node r owns [tpo[r], tpo[r+1]) and [tso[r], tso[r+1])
            np = min(np, w.tpo[r + 1] - w.tpo[r]);
            ns = min(ns, w.tso[r + 1] - w.tso[r]);
        }
        const int ti = w.tpo[r], to = pt_off[r], si = w.tso[r], so = seg_off[r];
        for (int j = lane; j < np; j += 32) {
            px[to + j] = w.tx[ti + j];
            py[to + j] = w.ty[ti + j];
            if (DIMS == 3) pz[to + j] = w.tz[ti + j];
        }
        for (int j = lane; j < ns; j += 32) {
            start[so + j] = to + w.trel[si + j];
            is_end[so + j] = w.tend[si + j];
        }
    }
}

// ---------------------------------------------------- node-parallel walk --
// The reference's walk, restated at node level.  Foreground pixels are nodes
// (v < 0: not exactly two neighbours) and chain pixels (v == 2).  Maximal
// runs of chain pixels between nodes are chains; a walk that enters a chain
// end from its node follows the whole chain (every interior pixel has
// exactly two neighbours and is reachable only through the chain), so a
// chain is one step: its pixel list, far end and exit node are worked out
// once, in parallel.  What a node does when the reference visits it depends
// only on the nodes it reaches through one chain or one step (its graph
// neighbours) that come earlier in raster order: they end walks on it, use
// up chains next to it, and are zero when it scans.  So a node runs as soon
// as those have run, and unrelated nodes run at the same time.  The only
// effect that crosses between nodes running together is +1 on a later
// node's value, which commutes (and a later node's value cannot reach zero
// while a walk can still arrive at it).  Anything outside these rules (a
// chain pixel without two neighbours, a used chain entered again, a full
// output range, a wait that runs out) sets a flag, and the caller redoes
// the image with the per-component pixel walk.
template <int DIMS>
__device__ __forceinline__ int nbr_code(int d)  // scan index -> (dz+1)*9 + (dy+1)*3 + (dx+1)
{
    const int centre = DIMS == 2 ? 4 : 13;
    const int q = d < centre ? d : d + 1;
    return DIMS == 2 ? 9 + q : q;
}
template <int DIMS>
__device__ __forceinline__ long long nbr_off(int d, int W, long long slice)
{
    const int c = nbr_code<DIMS>(d);
    return (long long)(c / 9 - 1) * slice + (long long)((c / 3) % 3 - 1) * W + (c % 3 - 1);
}

struct ChainTabs {
    const int8_t *V0;
    int *Vw;             // current values (int32 per pixel; nodes and chain pixels)
    int *idmap;          // node pixel -> raster rank, chain-end pixel -> end id
    uint16_t *nb;        // chain pixel -> its two neighbour scan indices (a | b << 5)
    uint32_t *endpix;    // end id -> pixel
    int *L;              // end id -> chain pixels from this end to the far end
    uint32_t *far;       // end id -> the far end pixel
    uint8_t *exitd;      // end id -> scan index from the far end to its node (L >= 2)
    int *listoff;        // end id -> first coordinate in the chain lists
    uint8_t *used;       // end id -> chain already walked
    int16_t *lx, *ly, *lz;  // chain lists (per end, from the end to the far end)
    int *nend;           // number of ends
    int max_ends;        // capacity of the end arrays
    int *err;
    int W, H;
    long long slice;
};

// chain pixels: their two neighbours; ends (next to a node) get an id
template <int DIMS>
__global__ void chain_nb_kernel(ChainTabs T, long long n, int max_ends)
{
    constexpr int ND = DIMS == 2 ? 8 : 26;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        T.Vw[i] = T.V0[i];
        if (T.V0[i] != 2) continue;
        int a = -1, b = -1;
        bool end = false;
        for (int d = 0; d < ND; d++) {
            const int v = T.V0[i + nbr_off<DIMS>(d, T.W, T.slice)];
            if (v == 0) continue;
            if (a < 0) a = d;
            else b = d;
            if (v < 0) end = true;
        }
        if (b < 0) {
            atomicOr(T.err, 1);  // fewer than two point neighbours: not the plain case
            continue;
        }
        T.nb[i] = (uint16_t)(a | (b << 5));
        if (end) {
            const int id = atomicAdd(T.nend, 1);
            if (id < max_ends) {
                T.endpix[id] = (uint32_t)i;
                T.idmap[i] = id;
            } else {
                atomicOr(T.err, 1);
            }
        }
    }
}

__global__ void node_ids_kernel(const uint32_t *__restrict__ nodes, int nn, int *idmap)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nn; r += gridDim.x * blockDim.x) idmap[nodes[r]] = r;
}

// One thread per chain end: follow the chain to its far end (and, in the
// second pass, write the coordinates on the way).
template <int DIMS, bool WRITE>
__global__ void chain_walk_kernel(ChainTabs T, int nend, long long n)
{
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < nend; id += gridDim.x * blockDim.x) {
        constexpr int ND = DIMS == 2 ? 8 : 26;
        const long long q = T.endpix[id];
        const int a = T.nb[q] & 31, b = T.nb[q] >> 5;
        if (a >= ND || b >= ND) {
            atomicOr(T.err, 1);
            if (!WRITE) T.L[id] = 0;
            continue;
        }
        const long long qa = q + nbr_off<DIMS>(a, T.W, T.slice), qb = q + nbr_off<DIMS>(b, T.W, T.slice);
        int x = 0, y = 0, z = 0, o = 0;
        if (WRITE) {
            x = (int)(q % T.W);
            y = (int)((q / T.W) % T.H);
            z = DIMS == 3 ? (int)(q / T.slice) : 0;
            o = T.listoff[id];
            T.lx[o] = (int16_t)x;
            T.ly[o] = (int16_t)y;
            if (DIMS == 3) T.lz[o] = (int16_t)z;
        }
        if (T.V0[qa] < 0 && T.V0[qb] < 0) {  // a one-pixel chain between two nodes
            if (!WRITE) {
                T.L[id] = 1;
                T.far[id] = (uint32_t)q;
                T.exitd[id] = 0xff;
            }
            continue;
        }
        int dstep = T.V0[qa] == 2 ? a : b;  // into the chain
        long long prev = q, cur = q + nbr_off<DIMS>(dstep, T.W, T.slice);
        int len = 2;
        bool found = false;
        if (!WRITE) T.L[id] = 0;
        for (long long guard = 0; guard < n; guard++) {
            if (WRITE) {
                const int cc = nbr_code<DIMS>(dstep);
                x += cc % 3 - 1;
                y += (cc / 3) % 3 - 1;
                z += cc / 9 - 1;
                ++o;
                T.lx[o] = (int16_t)x;
                T.ly[o] = (int16_t)y;
                if (DIMS == 3) T.lz[o] = (int16_t)z;
            }
            const int ca = T.nb[cur] & 31, cb = T.nb[cur] >> 5;
            if (ca >= ND || cb >= ND) {
                atomicOr(T.err, 1);
                break;
            }
            const int dn = (cur + nbr_off<DIMS>(ca, T.W, T.slice) == prev) ? cb : ca;
            const long long nx = cur + nbr_off<DIMS>(dn, T.W, T.slice);
            const int vnx = T.V0[nx];
            if (vnx < 0) {
                if (!WRITE) {
                    T.L[id] = len;
                    T.far[id] = (uint32_t)cur;
                    T.exitd[id] = (uint8_t)dn;
                }
                found = true;
                break;
            }
            if (vnx != 2) {
                atomicOr(T.err, 1);
                break;
            }
            prev = cur;
            cur = nx;
            dstep = dn;
            len++;
        }
        if (!found) atomicOr(T.err, 1);
    }
}

// The graph neighbour of node p through its neighbour n (scan index d): n
// itself when n is a node, else the node at the far side of n's chain.
template <int DIMS>
__device__ __forceinline__ long long graph_nbr(const ChainTabs &T, long long p, int d, int &len)
{
    const long long nbp = p + nbr_off<DIMS>(d, T.W, T.slice);
    const int v0 = T.V0[nbp];
    len = 0;
    if (v0 < 0) return nbp;
    if (v0 != 2) return -1;
    constexpr int ND = DIMS == 2 ? 8 : 26;
    const int id = T.idmap[nbp];
    if (id < 0 || id >= T.max_ends) return -1;  // not an end: the caller's flag decides
    len = T.L[id];
    long long m;
    if (len == 1) {
        const int a = T.nb[nbp] & 31, b = T.nb[nbp] >> 5, back = ND - 1 - d;
        const int ex = a == back ? b : a;
        if (a >= ND || b >= ND) return -1;
        m = nbp + nbr_off<DIMS>(ex, T.W, T.slice);
    } else {
        if (len < 1 || T.exitd[id] >= ND) return -1;
        m = (long long)T.far[id] + nbr_off<DIMS>(T.exitd[id], T.W, T.slice);
    }
    return T.V0[m] < 0 ? m : -1;
}

// per node: earlier graph neighbours (in-degree) and output bounds
template <int DIMS>
__global__ void node_graph_kernel(ChainTabs T, const uint32_t *__restrict__ nodes, int nn, int *indeg, int *pbound,
                                  int *sbound)
{
    constexpr int ND = DIMS == 2 ? 8 : 26;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nn; r += warps) {
        const long long p = nodes[r];
        int dep = 0, pb = 0;
        if (lane < ND) {
            int len;
            const long long m = graph_nbr<DIMS>(T, p, lane, len);
            if (m >= 0) {
                pb = len > 0 ? len + 1 : 1;
                dep = (m < p) ? 1 : 0;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            dep += __shfl_down_sync(kFull, dep, o);
            pb += __shfl_down_sync(kFull, pb, o);
        }
        if (lane == 0) {
            const int budget = -(int)T.V0[p];
            indeg[r] = dep;
            pbound[r] = pb + budget;
            sbound[r] = budget;
        }
    }
}

__global__ void seed_ready_kernel(const int *__restrict__ indeg, int nn, int *queue, int *qtail)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nn; r += gridDim.x * blockDim.x)
        if (indeg[r] == 0) queue[atomicAdd(qtail, 1)] = r + 1;
}

// Warps take ready nodes from the queue in order of readiness and replay the
// reference's visit of each (budget, scan order, chain walks, +1 on the node
// a walk ends at), writing the node's output to its own range.
template <int DIMS>
__global__ void node_walk_kernel(ChainTabs T, const uint32_t *__restrict__ nodes, int nn, int *indeg,
                                 int *queue, int *qhead, int *qtail, WalkOut out, long long timeout_ns)
{
    constexpr int ND = DIMS == 2 ? 8 : 26;
    const int lane = threadIdx.x & 31;
    const long long my_off = lane < ND ? nbr_off<DIMS>(lane, T.W, T.slice) : 0;
    const int my_code = lane < ND ? nbr_code<DIMS>(lane) : 13;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(qhead, 1);
        t = __shfl_sync(kFull, t, 0);
        if (t >= nn) break;
        int r = 0;
        if (lane == 0) {
            const unsigned long long t_end = globaltimer() + (unsigned long long)timeout_ns;
            for (int w = 0;; w++) {
                r = ld_acquire(queue + t);
                if (r) break;
                if ((w & 63) == 63 && globaltimer() > t_end) {
                    atomicOr(T.err, 2);
                    break;
                }
                __nanosleep(w < 32 ? 32 : 256);
            }
        }
        r = __shfl_sync(kFull, r, 0) - 1;
        if (r < 0) break;  // timed out
        const long long p = nodes[r];
        // values that lane 0 writes are read by lane 0 and broadcast, so every
        // lane takes the same branches (the loops below hold warp-wide votes)
        int vp = 0;
        if (lane == 0) vp = T.Vw[p];
        vp = __shfl_sync(kFull, vp, 0);
        int po = out.tpo[r], so = out.tso[r];
        const int po_end = out.tpo[r + 1], so_end = out.tso[r + 1];
        int segs = 0, pts = 0;
        if (vp < 0) {
            if (lane == 0) T.Vw[p] = 0;
            const int px_ = (int)(p % T.W), py_ = (int)((p / T.W) % T.H), pz_ = DIMS == 3 ? (int)(p / T.slice) : 0;
            auto put = [&](int x, int y, int z) {
                if (lane == 0) {
                    if (po < po_end) {
                        out.tx[po] = (int16_t)x;
                        out.ty[po] = (int16_t)y;
                        if (DIMS == 3) out.tz[po] = (int16_t)z;
                    } else {
                        atomicOr(T.err, 4);
                    }
                }
                po++;
                pts++;
            };
            const int v0p = T.V0[p];
            int ni = -1;
            for (int br = 0; br < -vp; br++) {
                int is_end = v0p > -2 && v0p < 2;
                const int rel = pts;
                put(px_, py_, pz_);
                const int vn = lane < ND ? T.Vw[p + my_off] : 0;
                const unsigned m = __ballot_sync(kFull, lane < ND && lane > ni && vn != 0);
                ni = m ? __ffs(m) - 1 : ND;
                if (ni < ND) {
                    const long long q = p + __shfl_sync(kFull, my_off, ni);
                    const int vq = __shfl_sync(kFull, vn, ni);
                    const int cq = __shfl_sync(kFull, my_code, ni);
                    const int qx = px_ + cq % 3 - 1, qy = py_ + (cq / 3) % 3 - 1, qz = pz_ + cq / 9 - 1;
                    const int v0q = T.V0[q];
                    const int qid = v0q == 2 ? T.idmap[q] : -1;
                    const bool chain_ok = v0q == 2 && vq == 2 && qid >= 0 && qid < T.max_ends && T.L[qid] >= 1;
                    if (vq == 2 && !chain_ok) atomicOr(T.err, 16);  // a value-2 pixel that is not a chain end
                    if (chain_ok) {
                        // a chain end entered from p: the whole chain, then its exit node
                        const int id = qid;
                        int len = T.L[id];
                        if (len > po_end - po) {  // cannot fit: the tables are inconsistent
                            atomicOr(T.err, 4);
                            len = max(0, po_end - po);
                        }
                        const long long fq = T.far[id];
                        if (lane == 0 && T.used[id]) atomicOr(T.err, 8);
                        const int lo = T.listoff[id];
                        for (int j = lane; j < len; j += 32) {
                            if (po + j < po_end) {
                                out.tx[po + j] = T.lx[lo + j];
                                out.ty[po + j] = T.ly[lo + j];
                                if (DIMS == 3) out.tz[po + j] = T.lz[lo + j];
                            } else {
                                atomicOr(T.err, 4);
                            }
                        }
                        po += len;
                        pts += len;
                        const int li = lo + max(len, 1) - 1;
                        const int16_t fx = T.lx[li], fy = T.ly[li];
                        const int16_t fz = DIMS == 3 ? T.lz[li] : (int16_t)0;
                        int ex;
                        if (len == 1) {
                            const int a = T.nb[q] & 31, b = T.nb[q] >> 5, back = ND - 1 - ni;
                            ex = a == back ? b : a;
                        } else {
                            ex = T.exitd[id];
                        }
                        if (ex >= ND) {  // tables inconsistent (flagged already); keep every access in range
                            atomicOr(T.err, 1);
                            ex = ni;
                        }
                        const long long e = fq + nbr_off<DIMS>(ex, T.W, T.slice);
                        int ve = 0;
                        if (lane == 0) ve = T.Vw[e];
                        ve = __shfl_sync(kFull, ve, 0);
                        if (lane == 0) {
                            T.used[id] = 1;
                            const int fid = T.idmap[fq];
                            if (fid >= 0 && fid < T.max_ends) T.used[fid] = 1;
                            T.Vw[q] = 0;
                            T.Vw[fq] = ve == 0 ? 1 : 0;  // a walk that stalls on the far end leaves it at 1
                        }
                        if (ve == 0) {
                            put(fx, fy, fz);  // stalled: the far end again
                            const int v0f = T.V0[fq];
                            if (v0f > -2 && v0f < 2) is_end = 1;
                        } else {
                            const int ce = nbr_code<DIMS>(ex);
                            put(fx + ce % 3 - 1, fy + (ce / 3) % 3 - 1, fz + ce / 9 - 1);
                            if (lane == 0) atomicAdd(T.Vw + e, 1);
                            const int v0e = T.V0[e];
                            if (v0e > -2 && v0e < 2) is_end = 1;
                        }
                    } else {
                        // a step onto a node (or anything else nonzero): two-point segment
                        put(qx, qy, qz);
                        if (lane == 0) atomicAdd(T.Vw + q, 1);
                        if (v0q > -2 && v0q < 2) is_end = 1;
                    }
                }
                if (lane == 0) {
                    if (so < so_end) {
                        out.trel[so] = rel;
                        out.tend[so] = (uint8_t)is_end;
                    } else {
                        atomicOr(T.err, 4);
                    }
                }
                so++;
                segs++;
                __syncwarp();
            }
        }
        if (lane == 0) {
            out.nseg[r] = segs;
            out.npts[r] = pts;
        }
        // release the later graph neighbours whose last earlier neighbour this was
        long long m = -1;
        if (lane < ND) {
            int len;
            m = graph_nbr<DIMS>(T, p, lane, len);
        }
        __threadfence();
        __syncwarp();
        if (m > p) {
            const int rm = T.idmap[m];
            if (rm >= 0 && rm < nn && atomicSub(indeg + rm, 1) == 1) {
                const int slot = atomicAdd(qtail, 1);
                if (slot < nn) st_release(queue + slot, rm + 1);
                else atomicOr(T.err, 32);
            }
        }
        __syncwarp();
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

// The node-parallel walk (see node_walk_kernel).  Returns BGT_OK with *out
// filled, 1 when the image needs the per-component pixel walk instead, or
// an error.  V0 holds the classified values, nodes the node pixels in raster
// order; nseg/npts/seg_off/pt_off are (nn + 1)-entry scratch arrays.
static int segments_parallel(bgt_ctx *c, int dims, const int8_t *V0, int W, int H, int D, const uint32_t *nodes,
                             int nn, int *nseg, int *npts, int *seg_off, int *pt_off, DevSegs *out)
{
    cudaStream_t st = c->stream;
    const long long npx = (long long)W * H * D;
    const int ND = dims == 2 ? 8 : 26;
    const long long max_ends_ll = std::min<long long>((long long)ND * nn, npx);
    if (max_ends_ll >= (1LL << 31)) return 1;
    const int max_ends = (int)max_ends_ll;
    int rc;
    void *p30, *p31, *p32, *p33, *p34;
    if ((rc = ctx_scratch(c, 30, (size_t)npx * 4, &p30)) || (rc = ctx_scratch(c, 31, (size_t)npx * 4, &p31)) ||
        (rc = ctx_scratch(c, 32, (size_t)npx * 2, &p32)) ||
        (rc = ctx_scratch(c, 33, (size_t)max_ends * 24 + 256, &p33)) ||
        (rc = ctx_scratch(c, 34, (size_t)(nn + 1) * 7 * 4 + 256, &p34)))
        return rc;
    ChainTabs T{};
    T.V0 = V0;
    T.Vw = (int *)p30;
    T.idmap = (int *)p31;
    T.nb = (uint16_t *)p32;
    char *eb = (char *)p33;
    T.endpix = (uint32_t *)eb;
    T.L = (int *)(eb + (size_t)max_ends * 4);
    T.far = (uint32_t *)(eb + (size_t)max_ends * 8);
    T.listoff = (int *)(eb + (size_t)max_ends * 12);
    T.exitd = (uint8_t *)(eb + (size_t)max_ends * 16);
    T.used = (uint8_t *)(eb + (size_t)max_ends * 17);
    int *small = (int *)(eb + (size_t)max_ends * 24);  // nend, err, qhead, qtail
    T.nend = small;
    T.err = small + 1;
    T.max_ends = max_ends;
    T.W = W;
    T.H = H;
    T.slice = (long long)W * H;
    int *indeg = (int *)p34, *pbound = indeg + (nn + 1), *sbound = pbound + (nn + 1), *tpo = sbound + (nn + 1),
        *tso = tpo + (nn + 1), *queue = tso + (nn + 1);
    int *qhead = small + 2, *qtail = small + 3;
    cudaError_t e;
    cudaMemsetAsync(T.idmap, 0xff, (size_t)npx * 4, st);
    cudaMemsetAsync(T.nb, 0xff, (size_t)npx * 2, st);
    cudaMemsetAsync(small, 0, 16, st);
    cudaMemsetAsync(T.used, 0, (size_t)max_ends, st);
    cudaMemsetAsync(queue, 0, (size_t)(nn + 1) * 4, st);
    if (dims == 2) chain_nb_kernel<2><<<grid_of(npx), 256, 0, st>>>(T, npx, max_ends);
    else chain_nb_kernel<3><<<grid_of(npx), 256, 0, st>>>(T, npx, max_ends);
    node_ids_kernel<<<grid_of(nn), 256, 0, st>>>(nodes, nn, T.idmap);
    int hv[2] = {0, 0};
    if ((e = cudaMemcpyAsync(hv, small, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "chain ends");
    if (hv[1] || hv[0] > max_ends) return 1;
    const int nend = hv[0];
    if (nend > 0) {
        if (dims == 2) chain_walk_kernel<2, false><<<grid_of(nend), 128, 0, st>>>(T, nend, npx);
        else chain_walk_kernel<3, false><<<grid_of(nend), 128, 0, st>>>(T, nend, npx);
    }
    // chain lists: one per end, L coordinates each
    void *p35;
    if ((rc = ctx_scratch(c, 35, (size_t)(nend + 1) * 4, &p35))) return rc;
    int *lsrc = (int *)p35;
    if (nend > 0) cudaMemcpyAsync(lsrc, T.L, (size_t)nend * 4, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(lsrc + nend, 0, 4, st);
    void *p36;
    if ((rc = ctx_scratch(c, 36, (size_t)(nend + 1) * 4, &p36))) return rc;
    int *loff = (int *)p36;
    if ((e = exscan(c, 14, lsrc, loff, nend + 1, st)) != cudaSuccess) return cuda_fail(e, "chain list scan");
    if (nend > 0) cudaMemcpyAsync(T.listoff, loff, (size_t)nend * 4, cudaMemcpyDeviceToDevice, st);
    // node graph and output bounds
    if (dims == 2) node_graph_kernel<2><<<grid_of((long long)nn * 32), 256, 0, st>>>(T, nodes, nn, indeg, pbound, sbound);
    else node_graph_kernel<3><<<grid_of((long long)nn * 32), 256, 0, st>>>(T, nodes, nn, indeg, pbound, sbound);
    cudaMemsetAsync(pbound + nn, 0, 4, st);
    cudaMemsetAsync(sbound + nn, 0, 4, st);
    if ((e = exscan(c, 14, pbound, tpo, nn + 1, st)) != cudaSuccess ||
        (e = exscan(c, 14, sbound, tso, nn + 1, st)) != cudaSuccess)
        return cuda_fail(e, "node bounds scan");
    int tot3[4] = {0, 0, 0, 0};
    if ((e = cudaMemcpyAsync(&tot3[0], loff + nend, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot3[1], tpo + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot3[2], tso + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot3[3], T.err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "node bounds");
    if (tot3[3] || tot3[0] < 0 || tot3[1] < 0 || tot3[2] < 0) return 1;
    const size_t NL = (size_t)tot3[0], Tp = (size_t)tot3[1], Ts = (size_t)tot3[2];
    void *p37, *p25;
    if ((rc = ctx_scratch(c, 37, 3 * (NL * 2 + 16), &p37))) return rc;
    T.lx = (int16_t *)p37;
    T.ly = T.lx + NL + 8;
    T.lz = T.ly + NL + 8;
    if (nend > 0) {
        if (dims == 2) chain_walk_kernel<2, true><<<grid_of(nend), 128, 0, st>>>(T, nend, npx);
        else chain_walk_kernel<3, true><<<grid_of(nend), 128, 0, st>>>(T, nend, npx);
    }
    const size_t t_y = align16(Tp * 2 + 2), t_z = t_y + align16(Tp * 2 + 2), t_rel = t_z + align16(Tp * 2 + 2),
                 t_end = t_rel + align16(Ts * 4 + 4), t_tot = t_end + align16(Ts + 1);
    if ((rc = ctx_scratch(c, 25, t_tot, &p25))) return rc;
    char *tbuf = (char *)p25;
    WalkOut wo{};
    wo.nseg = nseg;
    wo.npts = npts;
    wo.tpo = tpo;
    wo.tso = tso;
    wo.tx = (int16_t *)tbuf;
    wo.ty = (int16_t *)(tbuf + t_y);
    wo.tz = (int16_t *)(tbuf + t_z);
    wo.trel = (int32_t *)(tbuf + t_rel);
    wo.tend = (uint8_t *)(tbuf + t_end);
    wo.err = T.err;
    seed_ready_kernel<<<grid_of(nn), 256, 0, st>>>(indeg, nn, queue, qtail);
    const long long timeout_ns = 2000000000LL;  // 2 s: ample for any image this path accepts
    const int wgrid = (int)std::min<long long>(((long long)nn * 32 + 255) / 256, (long long)c->sms * 8);
    if (dims == 2)
        node_walk_kernel<2><<<wgrid, 256, 0, st>>>(T, nodes, nn, indeg, queue, qhead, qtail, wo, timeout_ns);
    else
        node_walk_kernel<3><<<wgrid, 256, 0, st>>>(T, nodes, nn, indeg, queue, qhead, qtail, wo, timeout_ns);
    cudaMemsetAsync(nseg + nn, 0, 4, st);
    cudaMemsetAsync(npts + nn, 0, 4, st);
    if ((e = exscan(c, 14, nseg, seg_off, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "segment scan");
    if ((e = exscan(c, 14, npts, pt_off, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "point scan");
    int tot[3] = {0, 0, 0};
    if ((e = cudaMemcpyAsync(&tot[0], seg_off + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[1], pt_off + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[2], T.err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "segment totals");
    if (tot[2]) return 1;
    const int S = tot[0], Np = tot[1];
    const size_t o_start = 0, o_end = align16((size_t)(S + 1) * 4), o_px = o_end + align16((size_t)S + 1),
                 o_py = o_px + align16((size_t)Np * 2 + 2), o_pz = o_py + align16((size_t)Np * 2 + 2),
                 o_tot = o_pz + align16((size_t)Np * 2 + 2);
    void *p19;
    if ((rc = ctx_scratch(c, 19, o_tot, &p19))) return rc;
    char *ob = (char *)p19;
    int32_t *o_st = (int32_t *)(ob + o_start);
    uint8_t *o_ie = (uint8_t *)(ob + o_end);
    int16_t *o_x = (int16_t *)(ob + o_px), *o_y = (int16_t *)(ob + o_py), *o_z = (int16_t *)(ob + o_pz);
    const int pgrid = (int)std::min<long long>(((long long)nn * 32 + 255) / 256, 148LL * 16);
    if (dims == 2) place_kernel<2><<<pgrid, 256, 0, st>>>(wo, seg_off, pt_off, nn, o_st, o_ie, o_x, o_y, o_z, true);
    else place_kernel<3><<<pgrid, 256, 0, st>>>(wo, seg_off, pt_off, nn, o_st, o_ie, o_x, o_y, o_z, true);
    cudaMemcpyAsync(o_st + S, pt_off + nn, 4, cudaMemcpyDeviceToDevice, st);
    out->nseg = S;
    out->npts = Np;
    out->start = o_st;
    out->is_end = o_ie;
    out->px = o_x;
    out->py = o_y;
    out->pz = dims == 3 ? o_z : nullptr;
    return BGT_OK;
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
    // BGT_SEGMENTS_PIXEL_WALK=1 selects the per-component pixel walk (tests compare both)
    if (!getenv("BGT_SEGMENTS_PIXEL_WALK")) {
        int *nseg_ = (int *)p15, *npts_ = (int *)p16, *seg_off_ = (int *)p17, *pt_off_ = (int *)p18;
        const int prc = segments_parallel(c, dims, V0, W, H, D, nodes, nn, nseg_, npts_, seg_off_, pt_off_, out);
        if (prc != 1) return prc;  // done, or an error
        *out = DevSegs();          // the per-component pixel walk below reproduces every case
    }
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
    // bounds of every component's output, and its temporary ranges
    void *p23, *p24, *p26;
    if ((rc = ctx_scratch(c, 23, (size_t)npx * 4, &p23)) ||
        (rc = ctx_scratch(c, 24, (size_t)(ncomp + 1) * 6 * 4, &p24)) ||
        (rc = ctx_scratch(c, 26, (size_t)(nn + 1) * 2 * 4, &p26)))
        return rc;
    uint32_t *pxcnt = (uint32_t *)p23;
    int *branches = (int *)p24, *cpx = branches + (ncomp + 1), *bpts = cpx + (ncomp + 1),
        *bsegs = bpts + (ncomp + 1), *cpb = bsegs + (ncomp + 1), *csb = cpb + (ncomp + 1);
    cudaMemsetAsync(pxcnt, 0, (size_t)npx * 4, st);
    cudaMemsetAsync(branches, 0, (size_t)(ncomp + 1) * 4, st);
    comp_px_kernel<<<grid_of(npx), 256, 0, st>>>(V, par, npx, pxcnt);
    comp_sums_kernel<<<grid_of(nn), 256, 0, st>>>(V0, snodes, keys_s, flag, fpos, pxcnt, nn, branches, cpx);
    comp_bounds_kernel<<<grid_of(ncomp + 1), 256, 0, st>>>(branches, cpx, ncomp, bpts, bsegs);
    if ((e = exscan(c, 14, bpts, cpb, ncomp + 1, st)) != cudaSuccess ||
        (e = exscan(c, 14, bsegs, csb, ncomp + 1, st)) != cudaSuccess)
        return cuda_fail(e, "component bounds scan");
    int tb[2] = {0, 0};
    if ((e = cudaMemcpyAsync(&tb[0], cpb + ncomp, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tb[1], csb + ncomp, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "component bounds");
    if (tb[0] < 0 || tb[1] < 0) return fail(BGT_ERR_LIMIT, "segment output bound exceeds 2^31 entries");
    const size_t Tp = (size_t)tb[0], Ts = (size_t)tb[1];
    const size_t t_x = 0, t_y = align16(Tp * 2 + 2), t_z = t_y + align16(Tp * 2 + 2), t_rel = t_z + align16(Tp * 2 + 2),
                 t_end = t_rel + align16(Ts * 4 + 4), t_err = t_end + align16(Ts + 1), t_tot = t_err + 16;
    void *p25;
    if ((rc = ctx_scratch(c, 25, t_tot, &p25))) return rc;
    char *tbuf = (char *)p25;
    WalkOut wo{};
    wo.nseg = nseg;
    wo.npts = npts;
    wo.tpo = (int *)p26;
    wo.tso = wo.tpo + (nn + 1);
    wo.cpb = cpb;
    wo.csb = csb;
    wo.tx = (int16_t *)(tbuf + t_x);
    wo.ty = (int16_t *)(tbuf + t_y);
    wo.tz = (int16_t *)(tbuf + t_z);
    wo.trel = (int32_t *)(tbuf + t_rel);
    wo.tend = (uint8_t *)(tbuf + t_end);
    wo.err = (int *)(tbuf + t_err);
    cudaMemsetAsync(wo.err, 0, 4, st);
    // one walk over every component (a warp each), outputs in emission order per component
    const int wgrid = (int)std::min<long long>(((long long)ncomp * 32 + 255) / 256, 148LL * 16);
    if (dims == 2)
        walk_kernel<2><<<wgrid, 256, 0, st>>>(V, V0, W, H, snodes, rank_s, cstart, ncomp, nn, wo);
    else
        walk_kernel<3><<<wgrid, 256, 0, st>>>(V, V0, W, H, snodes, rank_s, cstart, ncomp, nn, wo);
    cudaMemsetAsync(nseg + nn, 0, 4, st);
    cudaMemsetAsync(npts + nn, 0, 4, st);
    if ((e = exscan(c, 14, nseg, seg_off, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "segment scan");
    if ((e = exscan(c, 14, npts, pt_off, nn + 1, st)) != cudaSuccess) return cuda_fail(e, "point scan");
    int tot[3] = {0, 0, 0};
    if ((e = cudaMemcpyAsync(&tot[0], seg_off + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[1], pt_off + nn, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[2], wo.err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "segment totals");
    if (tot[2]) return fail(BGT_ERR_LIMIT, "segment output outgrew its bound");
    const int S = tot[0], Np = tot[1];
    // output block: start[S+1] int32, is_end[S] u8, px, py (pz) int16[Np]
    const size_t o_start = 0, o_end = align16((size_t)(S + 1) * 4), o_px = o_end + align16((size_t)S + 1),
                 o_py = o_px + align16((size_t)Np * 2 + 2), o_pz = o_py + align16((size_t)Np * 2 + 2),
                 o_tot = o_pz + align16((size_t)Np * 2 + 2);
    void *p19;
    if ((rc = ctx_scratch(c, 19, o_tot, &p19))) return rc;
    char *ob = (char *)p19;
    int32_t *o_st = (int32_t *)(ob + o_start);
    uint8_t *o_ie = (uint8_t *)(ob + o_end);
    int16_t *o_x = (int16_t *)(ob + o_px), *o_y = (int16_t *)(ob + o_py), *o_z = (int16_t *)(ob + o_pz);
    const int pgrid = (int)std::min<long long>(((long long)nn * 32 + 255) / 256, 148LL * 16);
    if (dims == 2)
        place_kernel<2><<<pgrid, 256, 0, st>>>(wo, seg_off, pt_off, nn, o_st, o_ie, o_x, o_y, o_z, false);
    else
        place_kernel<3><<<pgrid, 256, 0, st>>>(wo, seg_off, pt_off, nn, o_st, o_ie, o_x, o_y, o_z, false);
    cudaMemcpyAsync(o_st + S, pt_off + nn, 4, cudaMemcpyDeviceToDevice, st);
    out->nseg = S;
    out->npts = Np;
    out->start = o_st;
    out->is_end = o_ie;
    out->px = o_x;
    out->py = o_y;
    out->pz = dims == 3 ? o_z : nullptr;
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
