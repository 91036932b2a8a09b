// rules.cuh -- the directional deletion rules as bit-parallel boolean algebra
// over 32-pixel words (ptxas fuses the expressions into LOP3 instructions).
//
// 2D: one template for "north" boundary pixels; S, E, W are the same template
// on the neighbour ring rotated by 180, 90, 270 degrees.  The boolean function
// is the one of 2D/CUDA_SubiterationKernels2D.cuh:15-119 (North..West), which
// is exactly rotation-symmetric; order of application N, S, E, W
// (2D/CUDA_ThinningKernelMultiBlock2D.cuh:104-135).
//
// 3D: one template for "up" boundary voxels (3D/CUDA_SubiterationKernels3D.cuh:14-49);
// the other five directions are its images under cube symmetries (each of
// the reference's six functions equals the template composed with one of
// these symmetries on all 2^26 neighbourhoods).  Order U, N, E, D, S, W
// (3D/CUDA_ThinningKernel3D_Linear.cuh:755-782).
#pragma once
#include <cstdint>

namespace bgt {

// ---------------------------------------------------------------- 2D ------
// x0..x7 = neighbours clockwise N, NE, E, SE, S, SW, W, NW after rotation;
// returns the mask of centre bits that are deletable (before & centre).
//
// The reference writes the rule as a sum of five products
//   a = ~x1 ~x7 (x2^x3^~x4)(x3^x5)(x3^x6),  b = x2 x4 (x6|~x7),  c = ~x1 x4 x6,
//   d = ~x6 ~x7 (x1^x5)(x2^x5)(x4^~x5),     e = ~x1 ~x2 ~x3 x6 x7.
// Here it is factored by the context (x5, x6, x7) into fewer three-input
// operations; the two forms agree on all 256 neighbourhoods:
//   x6 | x5 ~x7          ->  H  = x4 (x2 | ~x1)
//   x6 (x5 | x7)         ->  also Z = no foreground among x1..x4
//   ~x5 ~x6 ~x7          ->  G0 = x2 (x1|x3|x4) | ~x1 ~x2 x3 x4
__device__ __forceinline__ uint32_t north_template(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3,
                                                   uint32_t x4, uint32_t x5, uint32_t x6, uint32_t x7)
{
    const uint32_t h = x4 & (x2 | ~x1);
    const uint32_t c1 = x6 | (x5 & ~x7);
    const uint32_t z = x6 & (x5 | x7) & ~(x1 | x2 | x3 | x4);
    const uint32_t g0 = (x2 & (x1 | x3 | x4)) | (~x1 & ~x2 & x3 & x4);
    const uint32_t c3 = ~(x5 | x6 | x7);
    return ~x0 & ((c1 & h) | z | (c3 & g0));
}

// Direction s in application order 0..3 = N, S, E, W -> ring rotation.
__host__ __device__ constexpr int rot2d(int s) { return s == 0 ? 0 : s == 1 ? 4 : s == 2 ? 2 : 6; }

// X[8] = N, NE, E, SE, S, SW, W, NW of the centre word.
template <int S>
__device__ __forceinline__ uint32_t rule2d(const uint32_t (&X)[8])
{
    constexpr int r = rot2d(S);
    return north_template(X[(0 + r) & 7], X[(1 + r) & 7], X[(2 + r) & 7], X[(3 + r) & 7], X[(4 + r) & 7],
                          X[(5 + r) & 7], X[(6 + r) & 7], X[(7 + r) & 7]);
}

// d = f(a, b, c) for the three-input function with truth table IMM
// (bit 4a + 2b + c of IMM), one LOP3 instruction.
template <unsigned IMM>
__device__ __forceinline__ uint32_t lop3(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(IMM));
    return d;
}

// The centre word o after one subiteration of direction S: o & ~rule2d<S>.
// Written as eleven three-input operations (the factored template above,
// with the select on x2 for G0 and the final keep folded in); the two forms
// agree on all 512 (centre, ring) combinations.
#ifndef BGT_RULE2D_LOP3
#define BGT_RULE2D_LOP3 1
#endif
template <int S>
__device__ __forceinline__ uint32_t keep2d(uint32_t o, const uint32_t (&X)[8])
{
#if BGT_RULE2D_LOP3
    constexpr int r = rot2d(S);
    const uint32_t x0 = X[(0 + r) & 7], x1 = X[(1 + r) & 7], x2 = X[(2 + r) & 7], x3 = X[(3 + r) & 7];
    const uint32_t x4 = X[(4 + r) & 7], x5 = X[(5 + r) & 7], x6 = X[(6 + r) & 7], x7 = X[(7 + r) & 7];
    const uint32_t h = lop3<0xD0>(x4, x2, x1);   // x4 & (x2 | ~x1)
    const uint32_t t = lop3<0xFE>(x1, x3, x4);   // x1 | x3 | x4
    const uint32_t q = lop3<0x08>(x1, x3, x4);   // ~x1 & x3 & x4
    const uint32_t a = lop3<0xF4>(x6, x5, x7);   // x6 | (x5 & ~x7)
    const uint32_t b = lop3<0xE0>(x6, x5, x7);   // x6 & (x5 | x7)
    const uint32_t c = lop3<0x01>(x5, x6, x7);   // ~(x5 | x6 | x7)
    const uint32_t bz = lop3<0x10>(b, t, x2);    // b & ~t & ~x2        (b & Z)
    const uint32_t g0 = lop3<0xCA>(x2, t, q);    // x2 ? t : q          (G0)
    const uint32_t ah = lop3<0xEA>(a, h, bz);    // (a & h) | bz
    const uint32_t tt = lop3<0xF8>(ah, c, g0);   // ah | (c & g0)
    return lop3<0xD0>(o, x0, tt);                // o & (x0 | ~tt)
#else
    return o & ~rule2d<S>(X);
#endif
}

// ---------------------------------------------------------------- 3D ------
// Neighbourhood words g[9*(dz+1) + 3*(dy+1) + (dx+1)] (g[13] = centre).
// Direction d in application order 0..5 = U, N, E, D, S, W.  In the
// template's frame, layer a = -1 must be background; local axis k maps to
// global axis perm(d, k) (0 = z, 1 = y, 2 = x), with axis a negated for D, S, W.
__host__ __device__ constexpr int perm3(int d, int k)
{
    return (d % 3 == 0) ? k : (d % 3 == 1) ? (k == 0 ? 1 : k == 1 ? 0 : 2) : (k == 0 ? 2 : k == 1 ? 0 : 1);
}

__host__ __device__ constexpr int gidx3(int d, int a, int b, int c)
{
    // local (a, b, c) -> global (dz, dy, dx)
    return 9 * (((perm3(d, 0) == 0) ? (d >= 3 ? -a : a) : (perm3(d, 1) == 0) ? b : c) + 1) +
           3 * (((perm3(d, 0) == 1) ? (d >= 3 ? -a : a) : (perm3(d, 1) == 1) ? b : c) + 1) +
           (((perm3(d, 0) == 2) ? (d >= 3 ? -a : a) : (perm3(d, 1) == 2) ? b : c) + 1);
}

template <int D>
__device__ __forceinline__ uint32_t rule3d(const uint32_t (&g)[27])
{
#define L(a, b, c) g[gidx3(D, a, b, c)]
    const uint32_t T = L(-1, 0, 0), B = L(1, 0, 0);
    const uint32_t Tn = L(-1, -1, 0), Ts = L(-1, 1, 0), Tw = L(-1, 0, -1), Te = L(-1, 0, 1);
    const uint32_t Tnw = L(-1, -1, -1), Tne = L(-1, -1, 1), Tsw = L(-1, 1, -1), Tse = L(-1, 1, 1);
    const uint32_t Mn = L(0, -1, 0), Ms = L(0, 1, 0), Mw = L(0, 0, -1), Me = L(0, 0, 1);
    const uint32_t Mnw = L(0, -1, -1), Mne = L(0, -1, 1), Msw = L(0, 1, -1), Mse = L(0, 1, 1);
    const uint32_t Bn = L(1, -1, 0), Bs = L(1, 1, 0), Bw = L(1, 0, -1), Be = L(1, 0, 1);
    const uint32_t Bnw = L(1, -1, -1), Bne = L(1, -1, 1), Bsw = L(1, 1, -1), Bse = L(1, 1, 1);
#undef L
    const uint32_t mid = Mnw | Mn | Mne | Mw | Me | Msw | Ms | Mse | Bnw | Bne | Bsw | Bse;
    const uint32_t bot_we = Bw | Be, bot_ns = Bn | Bs;
    const uint32_t arm_n = Bn & ~Bs & ~Ms & ~Mse & ~Bse;
    const uint32_t arm_s = Bs & ~Bn & ~Mn & ~Mne & ~Bne;
    const uint32_t arm_w = Bw & ~Be & ~Me;
    const uint32_t arm_e = Be & ~Bw & ~Mw;
    const uint32_t arm_e_s = arm_e & ~Msw & ~Bsw;
    const uint32_t arm_e_n = arm_e & ~Mnw & ~Bnw;
    const uint32_t m1 = mid | bot_we | bot_ns;
    const uint32_t m5 = ((mid | bot_we) & ((arm_n & ~Msw & ~Bsw) | (arm_s & ~Mnw & ~Bnw))) |
                        ((mid | bot_ns) & ((arm_e_n & ~Msw & ~Bsw) | (arm_w & ~Mne & ~Mse & ~Bne & ~Bse)));
    const uint32_t m6 = (arm_e_s & Bn & ~Bs & ~Ms) | (arm_e_n & Bs & ~Bn & ~Mn) | (arm_w & (arm_n | arm_s));
    const uint32_t m4 = (~Tnw & ~Tsw & ((Tne & Mne & ~Tse) | (Tse & Mse & ~Tne))) |
                        (~Tne & ~Tse & ((Tnw & Mnw & ~Tsw) | (Tsw & Msw & ~Tnw)));
    const uint32_t m2 = (~Tn & ~Tne & ~Te & ((~Tnw & ~Tw & Ms) | (~Ts & ~Tse & Mw))) |
                        (~Ts & ~Tsw & ~Tw & ((~Te & ~Tse & Mn) | (~Tnw & ~Tn & Me)));
    const uint32_t m3 = (~Tw & Me & ((~Ts & ~Tsw & Mn) | (~Tnw & ~Tn & Ms))) |
                        (~Te & Mw & ((~Tn & ~Tne & Ms) | (~Ts & ~Tse & Mn)));
    const uint32_t cross_clear = ~(Tn | Tw | Te | Ts);
    const uint32_t corner_clear = ~(Tnw | Tne | Tsw | Tse);
    return ~T & ((cross_clear & ((B & m4) | (corner_clear & ((B & m1) | (~B & (m5 | m6)))))) | (B & (m2 | m3)));
}

}  // namespace bgt
