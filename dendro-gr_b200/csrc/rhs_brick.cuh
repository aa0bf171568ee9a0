// Shared pieces of the brick kernels (fused right-hand side, split
// derivative pass): bit-exact stencils on a shared-memory tile, the one-sided
// closures at physical faces, the brick geometry, the staging of one
// variable's tile with cp.async and the cooperative mixed-derivative pass.
//
// A "brick" is at most BX*BY*BZ interior zones of one padded block, one
// thread per zone; its tile is the brick plus the 3-point halo.  Mixed second
// derivatives are formed as in the reference, by applying the first-
// derivative stencil to first derivatives (BSSN_GR/scripts/bssnrhs_derivs.h):
// the mixed pass writes d/dx and d/dy on the halo rows to shared memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bssn_common.cuh"
#include "rhs_fused.cuh"
#include "stencil_exact.cuh"

namespace bssn {

namespace {

constexpr int PW = 3;

// Balanced split of n interior points into ceil(n/bmax) bricks.
__host__ __device__ inline void split1(int n, int bmax, int q, int& o, int& e) {
    const int nb = (n + bmax - 1) / bmax;
    const int base = n / nb, rem = n % nb;
    e = base + (q < rem ? 1 : 0);
    o = q * base + (q < rem ? q : rem);
}

// ---------------------------------------------------------------------------
// Stencils on shared memory.  `t` points at the zone's value, `st` is the
// stride along the direction, `a` the zone's padded coordinate along it, `s`
// the padded block side.  Stencils applied to the evolved variables are the
// bit-exact ones of stencil_exact.cuh; only the outer stage of the mixed
// second derivatives (a first derivative of first derivatives, which carry
// no O(1) offset) uses multiply-adds.
// ---------------------------------------------------------------------------
struct Dir3 {
    double d1, d2, ko;
};

// Interior (centred) stencils, bit-exact: the reference's left-to-right
// order, every product and sum rounded.
__device__ __forceinline__ double d1_in(const double* t, int st, const AxisCoef& c) {
    double r = -t[-3 * st];
    r = __dadd_rn(r, __dmul_rn(9.0, t[-2 * st]));
    r = __dadd_rn(r, __dmul_rn(-45.0, t[-st]));
    r = __dadd_rn(r, __dmul_rn(45.0, t[st]));
    r = __dadd_rn(r, __dmul_rn(-9.0, t[2 * st]));
    r = __dadd_rn(r, t[3 * st]);
    return __dmul_rn(r, c.ih60);
}
__device__ __forceinline__ double d2_in(const double* t, int st, const AxisCoef& c) {
    double r = __dmul_rn(2.0, t[-3 * st]);
    r = __dadd_rn(r, __dmul_rn(-27.0, t[-2 * st]));
    r = __dadd_rn(r, __dmul_rn(270.0, t[-st]));
    r = __dadd_rn(r, __dmul_rn(-490.0, t[0]));
    r = __dadd_rn(r, __dmul_rn(270.0, t[st]));
    r = __dadd_rn(r, __dmul_rn(-27.0, t[2 * st]));
    r = __dadd_rn(r, __dmul_rn(2.0, t[3 * st]));
    return __dmul_rn(r, c.ih2_180);
}
__device__ __forceinline__ double ko_in(const double* t, int st, const AxisCoef& c) {
    double r = -t[-3 * st];
    r = __dadd_rn(r, __dmul_rn(6.0, t[-2 * st]));
    r = __dadd_rn(r, __dmul_rn(-15.0, t[-st]));
    r = __dadd_rn(r, __dmul_rn(20.0, t[0]));
    r = __dadd_rn(r, __dmul_rn(-15.0, t[st]));
    r = __dadd_rn(r, __dmul_rn(6.0, t[2 * st]));
    r = __dadd_rn(r, -t[3 * st]);
    return __dmul_rn(c.ko_pre, r);
}

// One-sided closures near a physical face (derivs.cpp), table driven: case
// 0..2 = a = 3,4,5 at a lower face, 3..5 = a = ie-3, ie-2, ie-1 at an upper
// face (ie = s-3); terms listed in the reference's left-to-right order as
// (coefficient, offset from a).  A short loop over the table keeps the code
// small: the closures run only in boundary blocks, and unrolling every case
// for every variable and axis overflowed the instruction cache.
__constant__ int kCloN[3][6] = {{5, 5, 4, 4, 5, 5}, {6, 6, 5, 5, 6, 6}, {4, 5, 6, 6, 5, 4}};
__constant__ double kCloC[3][6][6] = {
    {{-25, 48, -36, 16, -3}, {-3, -10, 18, -6, 1}, {1, -8, 8, -1},
     {1, -8, 8, -1}, {-1, 6, -18, 10, 3}, {3, -16, 36, -48, 25}},
    {{45, -154, 214, -156, 61, -10}, {10, -15, -4, 14, -6, 1}, {-1, 16, -30, 16, -1},
     {-1, 16, -30, 16, -1}, {1, -6, 14, -4, -15, 10}, {-10, 61, -156, 214, -154, 45}},
    {{1, -3, 3, -1}, {1, -6, 12, -10, 3}, {1, -6, 15, -19, 12, -3},
     {1, -6, 15, -19, 12, -3}, {1, -6, 12, -10, 3}, {1, -3, 3, -1}}};
__constant__ int kCloO[3][6][6] = {
    {{0, 1, 2, 3, 4}, {-1, 0, 1, 2, 3}, {-2, -1, 1, 2},
     {-2, -1, 1, 2}, {-3, -2, -1, 0, 1}, {-4, -3, -2, -1, 0}},
    {{0, 1, 2, 3, 4, 5}, {-1, 0, 1, 2, 3, 4}, {-2, -1, 0, 1, 2},
     {-2, -1, 0, 1, 2}, {-4, -3, -2, -1, 0, 1}, {-5, -4, -3, -2, -1, 0}},
    {{3, 2, 1, 0}, {3, 2, 1, 0, -1}, {3, 2, 1, 0, -1, -2},
     {-3, -2, -1, 0, 1, 2}, {-3, -2, -1, 0, 1}, {-3, -2, -1, 0}}};

__device__ __forceinline__ double closure_fold(const double* t, int st, int kind, int c) {
    const int n = kCloN[kind][c];
    double r = __dmul_rn(kCloC[kind][c][0], t[kCloO[kind][c][0] * st]);
#pragma unroll 1
    for (int q = 1; q < n; q++) r = __dadd_rn(r, __dmul_rn(kCloC[kind][c][q], t[kCloO[kind][c][q] * st]));
    return r;
}

// Closure case of padded coordinate a (callers guarantee near_face).  Chosen
// by explicit comparisons: the arithmetic form a - (s - 6) + 3 (clamped)
// produced the wrong case at a = s - 5 in some inlined copies of this kernel
// built by nvcc 12.9 for sm_100a (reproducible; the compiled code was not
// inspected), while this form is bit-exact against the oracle.
__device__ __forceinline__ int closure_case(int a, int s, bool blo) {
    return (blo && a == 3) ? 0 : (blo && a == 4) ? 1 : (blo && a == 5) ? 2
         : (a == s - 6) ? 3 : (a == s - 5) ? 4 : 5;
}

__device__ __forceinline__ Dir3 closure3(const double* t, int st, int a, int s, bool blo,
                                         const AxisCoef& cf, bool second) {
    const int c = closure_case(a, s, blo);
    Dir3 r;
    r.d1 = __dmul_rn(closure_fold(t, st, 0, c), cf.ih12);
    r.d2 = second ? __dmul_rn(closure_fold(t, st, 1, c), cf.ih2_12) : 0.0;
    const double smr = (c == 0 || c == 5) ? cf.smr3 : ((c == 1 || c == 4) ? cf.smr2 : cf.smr1);
    r.ko = __ddiv_rn(closure_fold(t, st, 2, c), smr);
    return r;
}

__device__ __forceinline__ double closure_d1(const double* t, int st, int a, int s, bool blo,
                                             const AxisCoef& cf) {
    const int c = closure_case(a, s, blo);
    return __dmul_rn(closure_fold(t, st, 0, c), cf.ih12);
}

__device__ __forceinline__ bool near_face(int a, int s, bool blo, bool bhi) {
    return (blo && a <= 5) || (bhi && a >= s - 6);
}

// exact first derivative (mixed pass on the evolved variable)
__device__ __forceinline__ double d1_exact(const double* t, int st, int a, int s,
                                           bool blo, bool bhi, const AxisCoef& c) {
    if (near_face(a, s, blo, bhi)) return closure_d1(t, st, a, s, blo, c);
    return d1_in(t, st, c);
}

// outer stage of a mixed derivative
__device__ __forceinline__ double d1_fast(const double* t, int st, int a, int s,
                                          bool blo, bool bhi, const AxisCoef& c) {
    if (near_face(a, s, blo, bhi)) return closure_d1(t, st, a, s, blo, c);
    const double D1 = t[st] - t[-st], D2 = t[2 * st] - t[-2 * st],
                 D3 = t[3 * st] - t[-3 * st];
    return fma(45.0, D1, fma(-9.0, D2, D3)) * c.ih60;
}

// d1, d2 (optional) and KO along one direction, bit-exact.
template <bool SECOND>
__device__ __forceinline__ Dir3 dir_all(const double* t, int st, int a, int s,
                                        bool blo, bool bhi, const AxisCoef& c) {
    if (near_face(a, s, blo, bhi)) return closure3(t, st, a, s, blo, c, SECOND);
    Dir3 r;
    r.d1 = d1_in(t, st, c);
    r.d2 = SECOND ? d2_in(t, st, c) : 0.0;
    r.ko = ko_in(t, st, c);
    return r;
}

struct ZoneCtx {
    int a[3];        // padded block coordinates of the zone
    int s;           // padded side
    unsigned bflag;
    // per-axis stencil factors: the same for every zone of a block, so they
    // live in shared memory (three AxisCoef in registers would take 48)
    const AxisCoef* cf;
    int tc;          // tile index of the zone
    int st[3];       // tile strides
};

// Derivatives of the staged variable at the zone: grad (3), second (6, sym
// order xx,xy,xz,yy,yz,zz; mixed from the shared halo passes) and KO sum.
template <bool SECOND>
__device__ __forceinline__ void zone_derivs(const ZoneCtx& z, const double* tile,
                                            const double* mxj, const double* mxk,
                                            const double* myk, int mj, int mk,
                                            double d1[3], double d2[6],
                                            double& ko) {
    const double* t = tile + z.tc;
    Dir3 rx = dir_all<SECOND>(t, z.st[0], z.a[0], z.s, z.bflag & 1u, z.bflag & 2u, z.cf[0]);
    Dir3 ry = dir_all<SECOND>(t, z.st[1], z.a[1], z.s, z.bflag & 4u, z.bflag & 8u, z.cf[1]);
    Dir3 rz = dir_all<SECOND>(t, z.st[2], z.a[2], z.s, z.bflag & 16u, z.bflag & 32u, z.cf[2]);
    d1[0] = rx.d1; d1[1] = ry.d1; d1[2] = rz.d1;
    ko = rx.ko + ry.ko + rz.ko;
    if (SECOND) {
        d2[0] = rx.d2; d2[3] = ry.d2; d2[5] = rz.d2;
        // d/dy (d/dx u), d/dz (d/dx u), d/dz (d/dy u)
        d2[1] = d1_fast(mxj, mj, z.a[1], z.s, z.bflag & 4u, z.bflag & 8u, z.cf[1]);
        d2[2] = d1_fast(mxk, mk, z.a[2], z.s, z.bflag & 16u, z.bflag & 32u, z.cf[2]);
        d2[4] = d1_fast(myk, mk, z.a[2], z.s, z.bflag & 16u, z.bflag & 32u, z.cf[2]);
    }
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(src));
}
// 16-byte copy, both addresses 16-byte aligned; bypasses L1 (streamed data)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

}  // namespace

// ---------------------------------------------------------------------------
// Brick geometry and shared-memory layout: two tiles (double buffer), then
// the mixed scratch.
// ---------------------------------------------------------------------------
template <int BX_, int BY_, int BZ_>
struct Brick {
    static constexpr int BX = BX_, BY = BY_, BZ = BZ_;
    static constexpr int TX = BX + 2 * PW, TY = BY + 2 * PW, TZ = BZ + 2 * PW;
    static constexpr int TILE = TX * TY * TZ;
    static constexpr int NZ = BX * BY * BZ;
    static constexpr int THREADS = (NZ + 31) / 32 * 32;
    // mixed scratch: dx on (x brick, y all, z brick), dx on (x brick, y brick,
    // z all), dy on (x brick, y brick, z all)
    static constexpr int MXJ = BX * TY * BZ;
    static constexpr int MXK = BX * BY * TZ;
    static constexpr int SMEM_DOUBLES = 2 * TILE + MXJ + 2 * MXK;
    static constexpr size_t SMEM_BYTES = SMEM_DOUBLES * sizeof(double);
};

// Order in which the brick kernels visit the evolved variables:
//   beta0..2, gt0..5, Gt0..2, chi, alpha, At0..5, K, B0..2
// and whether a variable needs second derivatives (beta, gt, chi, alpha).
__host__ __device__ constexpr int stage_order(int step) {
    return step < 3 ? U_BETA0 + step
         : step < 9 ? U_SYMGT0 + (step - 3)
         : step < 12 ? U_GT0 + (step - 9)
         : step == 12 ? U_CHI
         : step == 13 ? U_ALPHA
         : step < 20 ? U_SYMAT0 + (step - 14)
         : step == 20 ? U_K
         : U_B0 + (step - 21);
}
__host__ __device__ constexpr bool stage_second(int step) {
    return step < 9 || step == 12 || step == 13;
}
template <bool B>
struct BoolTag {
    static constexpr bool value = B;
};

namespace {

// Copy the staged region [o, o+e+6)^3 of one variable of a padded block
// (`src` = the block's first point) into a tile, 8-byte cp.async per point,
// as one commit group.
template <class Bk>
__device__ __forceinline__ void stage_var(const double* src, double* dst, const int o[3],
                                          const int e[3], int s, int tid) {
    const int sx = e[0] + 2 * PW, sy = e[1] + 2 * PW, sz = e[2] + 2 * PW;
    const int nstage = sx * sy * sz;
    for (int idx = tid; idx < nstage; idx += Bk::THREADS) {
        const int ti = idx % sx, r = idx / sx, tj = r % sy, tk = r / sy;
        const int64_t g = (int64_t)(o[0] + ti) + (int64_t)s * ((o[1] + tj) + (int64_t)s * (o[2] + tk));
        cp_async8(dst + ti + Bk::TX * (tj + Bk::TY * tk), src + g);
    }
    cp_async_commit();
}

// Cooperative pass: exact first derivatives on the halo rows needed by the
// mixed second derivatives of the tile's variable: d/dx on (x brick, y all,
// z brick) -> mxj [BZ][TY][BX]; d/dx and d/dy on (x brick, y brick, z all)
// -> mxk, myk [TZ][BY][BX].
template <class Bk>
__device__ __forceinline__ void mixed_pass(const double* tile, double* mxj, double* mxk,
                                           double* myk, const int o[3], const int e[3], int s,
                                           unsigned bflag, const AxisCoef cf[3], int tid) {
    constexpr int BX = Bk::BX, BY = Bk::BY, TX = Bk::TX, TY = Bk::TY;
    const int nj = e[0] * (e[1] + 2 * PW) * e[2];
    const int nk = e[0] * e[1] * (e[2] + 2 * PW);
    for (int idx = tid; idx < nj + 2 * nk; idx += Bk::THREADS) {
        int q = idx;
        if (q < nj) {
            const int i = q % e[0], r = q / e[0], j = r % (e[1] + 2 * PW), k = r / (e[1] + 2 * PW);
            const double* t = tile + (i + PW) + TX * (j + TY * (k + PW));
            mxj[i + BX * (j + TY * k)] = d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, cf[0]);
            continue;
        }
        q -= nj;
        const bool ydir = q >= nk;
        if (ydir) q -= nk;
        const int i = q % e[0], r = q / e[0], j = r % e[1], k = r / e[1];
        const double* t = tile + (i + PW) + TX * ((j + PW) + TY * k);
        if (!ydir)
            mxk[i + BX * (j + BY * k)] = d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, cf[0]);
        else
            myk[i + BX * (j + BY * k)] = d1_exact(t, TX, o[1] + PW + j, s, bflag & 4u, bflag & 8u, cf[1]);
    }
}

// Staging with the index arithmetic done once per brick: a thread copies the
// tile points idx = tid + k*THREADS (k < ITER) of every variable, so it keeps
// their offsets from the block's first point (-1: outside the staged region
// [o, o+e+6)^3 of a ragged brick) in registers.
//
// Source of the tile: the padded block (offsets from its first point), or,
// for blocks of a single-level mesh, the zipped node grid directly (gx > 0:
// offsets are node indices, points outside the grid are zero -- exactly the
// values the ghost fill writes there -- marked -2).
struct ZipGrid {
    int gx, gy, gz;  // gx == 0: padded input
};

template <class Bk, bool ZIP>
struct StagePlan {
    static constexpr int ITER = (Bk::TILE + Bk::THREADS - 1) / Bk::THREADS;
    int goff[ITER];
    __device__ __forceinline__ StagePlan(const int o[3], const int e[3], int s, int tid,
                                         const ZipGrid& g, const int32_t g0[3]) {
#pragma unroll
        for (int k = 0; k < ITER; k++) {
            const int idx = tid + k * Bk::THREADS;
            const int ti = idx % Bk::TX, r = idx / Bk::TX, tj = r % Bk::TY, tk = r / Bk::TY;
            const bool in = idx < Bk::TILE && ti < e[0] + 2 * PW && tj < e[1] + 2 * PW &&
                            tk < e[2] + 2 * PW;
            if (!ZIP) {
                goff[k] = in ? (o[0] + ti) + s * ((o[1] + tj) + s * (o[2] + tk)) : -1;
            } else {
                // padded coordinate o + t is node g0 + o + t - 3
                const int x = g0[0] + o[0] + ti - PW, y = g0[1] + o[1] + tj - PW,
                          z = g0[2] + o[2] + tk - PW;
                const bool grid = x >= 0 && y >= 0 && z >= 0 && x < g.gx && y < g.gy && z < g.gz;
                goff[k] = !in ? -1 : (grid ? x + g.gx * (y + g.gy * z) : -2);
            }
        }
    }
    __device__ __forceinline__ void stage(const double* src, double* dst, int tid) const {
#pragma unroll
        for (int k = 0; k < ITER; k++) {
            if (goff[k] >= 0)
                cp_async8(dst + tid + k * Bk::THREADS, src + goff[k]);
            else if (ZIP && goff[k] == -2)
                dst[tid + k * Bk::THREADS] = 0.0;
        }
        cp_async_commit();
    }
};

// The mixed pass over the compile-time extents of the mixed scratch (items
// outside a ragged brick's region are skipped); output index = item index.
template <class Bk>
__device__ __forceinline__ void mixed_pass_fixed(const double* tile, double* mx, const int o[3],
                                                 const int e[3], int s, unsigned bflag,
                                                 const AxisCoef cf[3], int tid) {
    constexpr int BX = Bk::BX, BY = Bk::BY, TX = Bk::TX, TY = Bk::TY;
    constexpr int MXJ = Bk::MXJ, MXK = Bk::MXK;
    for (int idx = tid; idx < MXJ + 2 * MXK; idx += Bk::THREADS) {
        if (idx < MXJ) {  // d/dx on (x brick, y all, z brick)
            const int i = idx % BX, r = idx / BX, j = r % TY, k = r / TY;
            if (i < e[0] && j < e[1] + 2 * PW && k < e[2]) {
                const double* t = tile + (i + PW) + TX * (j + TY * (k + PW));
                mx[idx] = d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, cf[0]);
            }
            continue;
        }
        const bool ydir = idx >= MXJ + MXK;
        const int q = idx - (ydir ? MXJ + MXK : MXJ);
        const int i = q % BX, r = q / BX, j = r % BY, k = r / BY;
        if (i < e[0] && j < e[1] && k < e[2] + 2 * PW) {
            const double* t = tile + (i + PW) + TX * ((j + PW) + TY * k);
            mx[idx] = ydir ? d1_exact(t, TX, o[1] + PW + j, s, bflag & 4u, bflag & 8u, cf[1])
                           : d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, cf[0]);
        }
    }
}

// Interior stencils of one direction, computed for every zone whatever its
// position (the taps of a zone of the brick always lie in the staged tile);
// zones near a physical face then take the closure instead.  Doing the three
// directions without branches lets their nine FP64 chains interleave.
template <bool SECOND>
__device__ __forceinline__ Dir3 dir_in(const double* t, int st, const AxisCoef& c) {
    Dir3 r;
    r.d1 = d1_in(t, st, c);
    r.d2 = SECOND ? d2_in(t, st, c) : 0.0;
    r.ko = ko_in(t, st, c);
    return r;
}
__device__ __forceinline__ double d1_fast_in(const double* t, int st, const AxisCoef& c) {
    const double D1 = t[st] - t[-st], D2 = t[2 * st] - t[-2 * st], D3 = t[3 * st] - t[-3 * st];
    return fma(45.0, D1, fma(-9.0, D2, D3)) * c.ih60;
}

// Gradient, pure second derivatives and summed KO of the tile's variable at
// the zone (interior stencils, closures as an override in boundary blocks).
template <bool SECOND, class Bk>
__device__ __forceinline__ void zone_dirs(const ZoneCtx& z, const double* tile, Dir3 r[3]) {
    const double* t = tile + z.tc;
    // compile-time strides: every tap is an immediate offset
    r[0] = dir_in<SECOND>(t, 1, z.cf[0]);
    r[1] = dir_in<SECOND>(t, Bk::TX, z.cf[1]);
    r[2] = dir_in<SECOND>(t, Bk::TX * Bk::TY, z.cf[2]);
    if (z.bflag) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const bool lo = z.bflag & (1u << (2 * d)), hi = z.bflag & (2u << (2 * d));
            if (near_face(z.a[d], z.s, lo, hi)) r[d] = closure3(t, z.st[d], z.a[d], z.s, lo, z.cf[d], SECOND);
        }
    }
}

// The interior stencils of zone_dirs (d1_in / d2_in / ko_in along x, y, z)
// advanced one tap at a time across all nine chains: every chain keeps the
// reference's left-to-right order of rounded products and sums, but the
// chains' operations alternate, so each tap step offers nine independent
// FP64 chains to hide latency with few warps per SM.  Closures as in
// zone_dirs.
template <bool SECOND, class Bk>
__device__ __forceinline__ void zone_dirs_il(const ZoneCtx& z, const double* tile, Dir3 r[3]) {
    const double* t = tile + z.tc;
    constexpr int ST[3] = {1, Bk::TX, Bk::TX * Bk::TY};
    double a1[3], a2[3], ak[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {  // tap -3
        const double v = t[-3 * ST[d]];
        a1[d] = -v;
        a2[d] = SECOND ? __dmul_rn(2.0, v) : 0.0;
        ak[d] = -v;
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {  // tap -2
        const double v = t[-2 * ST[d]];
        a1[d] = __dadd_rn(a1[d], __dmul_rn(9.0, v));
        if (SECOND) a2[d] = __dadd_rn(a2[d], __dmul_rn(-27.0, v));
        ak[d] = __dadd_rn(ak[d], __dmul_rn(6.0, v));
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {  // tap -1
        const double v = t[-ST[d]];
        a1[d] = __dadd_rn(a1[d], __dmul_rn(-45.0, v));
        if (SECOND) a2[d] = __dadd_rn(a2[d], __dmul_rn(270.0, v));
        ak[d] = __dadd_rn(ak[d], __dmul_rn(-15.0, v));
    }
    {  // tap 0 (not in the first derivative)
        const double v = t[0];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (SECOND) a2[d] = __dadd_rn(a2[d], __dmul_rn(-490.0, v));
            ak[d] = __dadd_rn(ak[d], __dmul_rn(20.0, v));
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {  // tap 1
        const double v = t[ST[d]];
        a1[d] = __dadd_rn(a1[d], __dmul_rn(45.0, v));
        if (SECOND) a2[d] = __dadd_rn(a2[d], __dmul_rn(270.0, v));
        ak[d] = __dadd_rn(ak[d], __dmul_rn(-15.0, v));
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {  // tap 2
        const double v = t[2 * ST[d]];
        a1[d] = __dadd_rn(a1[d], __dmul_rn(-9.0, v));
        if (SECOND) a2[d] = __dadd_rn(a2[d], __dmul_rn(-27.0, v));
        ak[d] = __dadd_rn(ak[d], __dmul_rn(6.0, v));
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {  // tap 3
        const double v = t[3 * ST[d]];
        a1[d] = __dadd_rn(a1[d], v);
        if (SECOND) a2[d] = __dadd_rn(a2[d], __dmul_rn(2.0, v));
        ak[d] = __dadd_rn(ak[d], -v);
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        r[d].d1 = __dmul_rn(a1[d], z.cf[d].ih60);
        r[d].d2 = SECOND ? __dmul_rn(a2[d], z.cf[d].ih2_180) : 0.0;
        r[d].ko = __dmul_rn(z.cf[d].ko_pre, ak[d]);
    }
    if (z.bflag) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const bool lo = z.bflag & (1u << (2 * d)), hi = z.bflag & (2u << (2 * d));
            if (near_face(z.a[d], z.s, lo, hi)) r[d] = closure3(t, z.st[d], z.a[d], z.s, lo, z.cf[d], SECOND);
        }
    }
}

// The halo part of the mixed scratch: d/dx on the 6 halo rows in y (mxj) and
// d/dx, d/dy on the 6 halo planes in z (mxk, myk); the brick part is written
// by the zones themselves from their own gradient.  Halo row / plane h in
// 0..5 sits at h (below the brick) or e + h (above it).
template <class Bk>
__device__ __forceinline__ void mixed_halo_pass(const double* tile, double* mx, const int o[3],
                                                const int e[3], int s, unsigned bflag,
                                                const AxisCoef cf[3], int tid) {
    constexpr int BX = Bk::BX, BY = Bk::BY, BZ = Bk::BZ, TX = Bk::TX, TY = Bk::TY;
    constexpr int HJ = BX * 2 * PW * BZ, HK = BX * BY * 2 * PW;
    for (int idx = tid; idx < HJ + 2 * HK; idx += Bk::THREADS) {
        if (idx < HJ) {
            const int i = idx % BX, r = idx / BX, h = r % (2 * PW), k = r / (2 * PW);
            const int j = h < PW ? h : e[1] + h;
            if (i < e[0] && k < e[2]) {
                const double* t = tile + (i + PW) + TX * (j + TY * (k + PW));
                mx[i + BX * (j + TY * k)] = d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, cf[0]);
            }
            continue;
        }
        const bool ydir = idx >= HJ + HK;
        const int q = idx - (ydir ? HJ + HK : HJ);
        const int i = q % BX, r = q / BX, j = r % BY, h = r / BY;
        const int k = h < PW ? h : e[2] + h;
        if (i < e[0] && j < e[1]) {
            const double* t = tile + (i + PW) + TX * ((j + PW) + TY * k);
            const int w = i + BX * (j + BY * k);
            if (ydir)
                mx[Bk::MXJ + Bk::MXK + w] = d1_exact(t, TX, o[1] + PW + j, s, bflag & 4u, bflag & 8u, cf[1]);
            else
                mx[Bk::MXJ + w] = d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, cf[0]);
        }
    }
    (void)BZ;
}

// The zone a thread works on.  Threads without a zone (past the brick's zone
// count, or outside a ragged brick's extent) compute on the nearest zone of
// the brick, so every coordinate they use lies in the block interior [3, s-3)
// and every shared-memory read stays inside the staged tile; they store
// nothing.
template <class Bk>
struct BrickThread {
    bool active;
    int t[3];  // zone within the brick (clamped for threads without a zone)
    __device__ __forceinline__ BrickThread(int tid, const int e[3]) {
        const bool in_brick = tid < Bk::NZ;
        const int r0 = in_brick ? tid % Bk::BX : 0;
        const int r1 = in_brick ? (tid / Bk::BX) % Bk::BY : 0;
        const int r2 = in_brick ? tid / (Bk::BX * Bk::BY) : 0;
        active = in_brick && r0 < e[0] && r1 < e[1] && r2 < e[2];
        t[0] = r0 < e[0] ? r0 : e[0] - 1;
        t[1] = r1 < e[1] ? r1 : e[1] - 1;
        t[2] = r2 < e[2] ? r2 : e[2] - 1;
    }
};

// The block's per-axis stencil factors, written by threads 0..2 into shared
// memory (visible after the caller's next barrier).
// (Selects, not blk.ptmax[tid]: a run-time index into the descriptor would
// put the whole descriptor in local memory for the rest of the kernel.)
__device__ __forceinline__ void fill_axis_coefs(AxisCoef* cf, const BssnBlockDesc& blk, int tid) {
    if (tid < 3) {
        const double lo = tid == 0 ? blk.ptmin[0] : (tid == 1 ? blk.ptmin[1] : blk.ptmin[2]);
        const double hi = tid == 0 ? blk.ptmax[0] : (tid == 1 ? blk.ptmax[1] : blk.ptmax[2]);
        cf[tid] = axis_coef((hi - lo) / (blk.sz - 1));
    }
}

// Stencil context of a thread's zone in a brick (tile strides, padded
// coordinates, per-axis coefficients) and its positions in the mixed scratch.
template <class Bk>
struct BrickZone {
    ZoneCtx zc;
    int mj, mk;
    int mxj_off, mxk_off;  // offsets of the zone in mxj and in mxk / myk
    // cf: the block's three AxisCoef in shared memory (fill_axis_coefs)
    __device__ __forceinline__ BrickZone(const BssnBlockDesc& blk, const int o[3],
                                         const BrickThread<Bk>& th, const AxisCoef* cf) {
        const int s = blk.sz;
        zc.s = s;
        zc.bflag = blk.bflag;
        zc.cf = cf;
#pragma unroll
        for (int d = 0; d < 3; d++) zc.a[d] = o[d] + PW + th.t[d];
        zc.st[0] = 1;
        zc.st[1] = Bk::TX;
        zc.st[2] = Bk::TX * Bk::TY;
        zc.tc = (th.t[0] + PW) + Bk::TX * ((th.t[1] + PW) + Bk::TY * (th.t[2] + PW));
        mj = Bk::BX;
        mk = Bk::BX * Bk::BY;
        mxj_off = th.t[0] + Bk::BX * ((th.t[1] + PW) + Bk::TY * th.t[2]);
        mxk_off = th.t[0] + Bk::BX * (th.t[1] + Bk::BY * (th.t[2] + PW));
    }
};

}  // namespace

}  // namespace bssn
