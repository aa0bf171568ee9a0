// Finite-difference stencils that reproduce the reference CPU arithmetic bit
// for bit: each product and sum is an explicitly rounded operation, issued in
// the left-to-right order of BSSN_GR/src/derivs.cpp, so the compiler cannot
// contract them into multiply-adds.  This matters: on fields that are O(1)
// plus a small perturbation (the conformal metric is the identity plus
// noise), the 7-point sums cancel to 1e-8 of their terms, and any other
// rounding order moves the result by ~1e-8 relative -- far above the 1e-12
// agreement the right-hand side must keep with the reference.
//
// p0 addresses the value at along-axis padded coordinate 0 (value at
// coordinate m is p0[m*st]); a is the coordinate of the output point, s the
// padded side, lo/hi whether the block's lower/upper face on this axis is a
// physical boundary (one-sided closures within three points of it).
#pragma once
#include "bssn_common.cuh"

namespace bssn {
namespace ex {

template <int N>
__device__ __forceinline__ double fold(const double (&c)[N], const double* p0,
                                       const int (&pos)[N], int st) {
    double t = __dmul_rn(c[0], p0[pos[0] * st]);
#pragma unroll
    for (int q = 1; q < N; q++) t = __dadd_rn(t, __dmul_rn(c[q], p0[pos[q] * st]));
    return t;
}

// deriv644_{x,y,z}: derivs.cpp:2645-2700 (interior, closures at 3,4,5 and
// ie-3..ie-1, ie = s-3)
__device__ __forceinline__ double d1(const double* p0, int st, int a, int s,
                                     bool lo, bool hi, const AxisCoef& cf) {
    const int ie = s - 3;
    if (lo && a <= 5) {
        if (a == 3) { const double c[5] = {-25.0, 48.0, -36.0, 16.0, -3.0}; const int p[5] = {3, 4, 5, 6, 7}; return __dmul_rn(fold(c, p0, p, st), cf.ih12); }
        if (a == 4) { const double c[5] = {-3.0, -10.0, 18.0, -6.0, 1.0}; const int p[5] = {3, 4, 5, 6, 7}; return __dmul_rn(fold(c, p0, p, st), cf.ih12); }
        const double c[4] = {1.0, -8.0, 8.0, -1.0}; const int p[4] = {3, 4, 6, 7}; return __dmul_rn(fold(c, p0, p, st), cf.ih12);
    }
    if (hi && a >= ie - 3) {
        if (a == ie - 3) { const double c[4] = {1.0, -8.0, 8.0, -1.0}; const int p[4] = {ie - 5, ie - 4, ie - 2, ie - 1}; return __dmul_rn(fold(c, p0, p, st), cf.ih12); }
        if (a == ie - 2) { const double c[5] = {-1.0, 6.0, -18.0, 10.0, 3.0}; const int p[5] = {ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(fold(c, p0, p, st), cf.ih12); }
        const double c[5] = {3.0, -16.0, 36.0, -48.0, 25.0}; const int p[5] = {ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(fold(c, p0, p, st), cf.ih12);
    }
    const double c[6] = {-1.0, 9.0, -45.0, 45.0, -9.0, 1.0};
    const int p[6] = {a - 3, a - 2, a - 1, a + 1, a + 2, a + 3};
    return __dmul_rn(fold(c, p0, p, st), cf.ih60);
}

// deriv644_{xx,yy,zz}: derivs.cpp:2974-3046
__device__ __forceinline__ double d2(const double* p0, int st, int a, int s,
                                     bool lo, bool hi, const AxisCoef& cf) {
    const int ie = s - 3;
    if (lo && a <= 5) {
        if (a == 3) { const double c[6] = {45.0, -154.0, 214.0, -156.0, 61.0, -10.0}; const int p[6] = {3, 4, 5, 6, 7, 8}; return __dmul_rn(fold(c, p0, p, st), cf.ih2_12); }
        if (a == 4) { const double c[6] = {10.0, -15.0, -4.0, 14.0, -6.0, 1.0}; const int p[6] = {3, 4, 5, 6, 7, 8}; return __dmul_rn(fold(c, p0, p, st), cf.ih2_12); }
        const double c[5] = {-1.0, 16.0, -30.0, 16.0, -1.0}; const int p[5] = {3, 4, 5, 6, 7}; return __dmul_rn(fold(c, p0, p, st), cf.ih2_12);
    }
    if (hi && a >= ie - 3) {
        if (a == ie - 3) { const double c[5] = {-1.0, 16.0, -30.0, 16.0, -1.0}; const int p[5] = {ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(fold(c, p0, p, st), cf.ih2_12); }
        if (a == ie - 2) { const double c[6] = {1.0, -6.0, 14.0, -4.0, -15.0, 10.0}; const int p[6] = {ie - 6, ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(fold(c, p0, p, st), cf.ih2_12); }
        const double c[6] = {-10.0, 61.0, -156.0, 214.0, -154.0, 45.0}; const int p[6] = {ie - 6, ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(fold(c, p0, p, st), cf.ih2_12);
    }
    const double c[7] = {2.0, -27.0, 270.0, -490.0, 270.0, -27.0, 2.0};
    const int p[7] = {a - 3, a - 2, a - 1, a, a + 1, a + 2, a + 3};
    return __dmul_rn(fold(c, p0, p, st), cf.ih2_180);
}

// ko_deriv42_{x,y,z}: derivs.cpp:988-1055
__device__ __forceinline__ double ko(const double* p0, int st, int a, int s,
                                     bool lo, bool hi, const AxisCoef& cf) {
    const int ie = s - 3;
    if (lo && a <= 5) {
        if (a == 3) { const double c[4] = {1.0, -3.0, 3.0, -1.0}; const int p[4] = {6, 5, 4, 3}; return __ddiv_rn(fold(c, p0, p, st), cf.smr3); }
        if (a == 4) { const double c[5] = {1.0, -6.0, 12.0, -10.0, 3.0}; const int p[5] = {7, 6, 5, 4, 3}; return __ddiv_rn(fold(c, p0, p, st), cf.smr2); }
        const double c[6] = {1.0, -6.0, 15.0, -19.0, 12.0, -3.0}; const int p[6] = {8, 7, 6, 5, 4, 3}; return __ddiv_rn(fold(c, p0, p, st), cf.smr1);
    }
    if (hi && a >= ie - 3) {
        if (a == ie - 3) { const double c[6] = {1.0, -6.0, 15.0, -19.0, 12.0, -3.0}; const int p[6] = {ie - 6, ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __ddiv_rn(fold(c, p0, p, st), cf.smr1); }
        if (a == ie - 2) { const double c[5] = {1.0, -6.0, 12.0, -10.0, 3.0}; const int p[5] = {ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __ddiv_rn(fold(c, p0, p, st), cf.smr2); }
        const double c[4] = {1.0, -3.0, 3.0, -1.0}; const int p[4] = {ie - 4, ie - 3, ie - 2, ie - 1}; return __ddiv_rn(fold(c, p0, p, st), cf.smr3);
    }
    const double c[7] = {-1.0, 6.0, -15.0, 20.0, -15.0, 6.0, -1.0};
    const int p[7] = {a - 3, a - 2, a - 1, a, a + 1, a + 2, a + 3};
    return __dmul_rn(cf.ko_pre, fold(c, p0, p, st));
}

}  // namespace ex
}  // namespace bssn
