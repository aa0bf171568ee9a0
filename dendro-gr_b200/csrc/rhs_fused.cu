// Fused BSSN right-hand side on padded octree blocks (sm_100a, FP64).
//
// One CTA owns a "brick" of at most BX*BY*BZ interior zones of one block
// (one thread per zone).  The 24 evolved variables stream through a
// double-buffered shared-memory tile (brick + 3-point halo) filled with
// cp.async; every derivative a zone needs is formed from that tile in
// registers and folded into the equations at once, in an order chosen to
// keep the live set small:
//   beta -> gt -> Christoffels/Ricci core -> Gt -> chi -> alpha -> At -> K -> B
// so the 138 derivatives and 72 dissipation terms never reach HBM.  Mixed
// second derivatives are formed as in the reference, by applying the first-
// derivative stencil to first derivatives (BSSN_GR/scripts/bssnrhs_derivs.h):
// a cooperative pass writes d/dx and d/dy on the halo rows to shared memory.
//
// Semantics follow BSSN_GR/src/rhs.cpp:80-504 (derivatives -> equations ->
// Sommerfeld BC on boundary faces -> + sigma * KO) with the equations of
// CodeGen/bssn.py:70-230 (standard gauge, constant eta): out = (on a physical
// boundary face ? BC : equations) + sigma * (KO_x + KO_y + KO_z).
#include <cuda_runtime.h>

#include <cstdio>

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
    AxisCoef cf[3];
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
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

}  // namespace

// ---------------------------------------------------------------------------
// The brick kernel body.
// ---------------------------------------------------------------------------
template <int BX, int BY, int BZ>
struct Brick {
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

template <int BX, int BY, int BZ>
__device__ __forceinline__ void rhs_brick(const RhsArgs& A, const BssnBlockDesc& blk,
                                          const int o[3], const int e[3],
                                          double* smem) {
    using Bk = Brick<BX, BY, BZ>;
    constexpr int TX = Bk::TX, TY = Bk::TY;
    double* tiles[2] = {smem, smem + Bk::TILE};
    double* mxj = smem + 2 * Bk::TILE;   // [BZ][TY][BX]
    double* mxk = mxj + Bk::MXJ;         // [TZ][BY][BX]
    double* myk = mxk + Bk::MXK;         // [TZ][BY][BX]

    const int tid = threadIdx.x;
    const int s = blk.sz;
    const int64_t off = blk.offset;
    const unsigned bflag = blk.bflag;
    // staged region of the padded block: [o, o+e+6) per axis
    const int sx = e[0] + 2 * PW, sy = e[1] + 2 * PW, sz = e[2] + 2 * PW;
    const int nstage = sx * sy * sz;

    auto stage = [&](int v, double* dst) {
        const double* src = A.u.p[v] + off;
        for (int idx = tid; idx < nstage; idx += Bk::THREADS) {
            const int ti = idx % sx, r = idx / sx, tj = r % sy, tk = r / sy;
            const int64_t g = (int64_t)(o[0] + ti) + (int64_t)s * ((o[1] + tj) + (int64_t)s * (o[2] + tk));
            cp_async8(dst + ti + TX * (tj + TY * tk), src + g);
        }
        cp_async_commit();
    };
    // cooperative pass: first derivatives on the halo rows needed by the
    // mixed second derivatives of the staged variable
    auto mixed_pass = [&](const double* tile, const ZoneCtx& zc) {
        const int nj = e[0] * (e[1] + 2 * PW) * e[2];
        const int nk = e[0] * e[1] * (e[2] + 2 * PW);
        for (int idx = tid; idx < nj + 2 * nk; idx += Bk::THREADS) {
            int q = idx;
            if (q < nj) {
                const int i = q % e[0], r = q / e[0], j = r % (e[1] + 2 * PW), k = r / (e[1] + 2 * PW);
                const double* t = tile + (i + PW) + TX * (j + TY * (k + PW));
                mxj[i + BX * (j + TY * k)] =
                    d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, zc.cf[0]);
                continue;
            }
            q -= nj;
            const bool ydir = q >= nk;
            if (ydir) q -= nk;
            const int i = q % e[0], r = q / e[0], j = r % e[1], k = r / e[1];
            const double* t = tile + (i + PW) + TX * ((j + PW) + TY * k);
            if (!ydir)
                mxk[i + BX * (j + BY * k)] =
                    d1_exact(t, 1, o[0] + PW + i, s, bflag & 1u, bflag & 2u, zc.cf[0]);
            else
                myk[i + BX * (j + BY * k)] =
                    d1_exact(t, TX, o[1] + PW + j, s, bflag & 4u, bflag & 8u, zc.cf[1]);
        }
    };

    // zone of this thread
    // Threads without a zone (past the brick's zone count, or outside a
    // ragged brick's extent) compute on the nearest zone of the brick, so
    // every coordinate they use lies in the block interior [3, s-3) and every
    // shared-memory read stays inside the staged tile; they store nothing.
    const bool in_brick = tid < Bk::NZ;
    const int rx = in_brick ? tid % BX : 0;
    const int ry = in_brick ? (tid / BX) % BY : 0;
    const int rz = in_brick ? tid / (BX * BY) : 0;
    const bool active = in_brick && rx < e[0] && ry < e[1] && rz < e[2];
    const int tx = rx < e[0] ? rx : e[0] - 1;
    const int ty = ry < e[1] ? ry : e[1] - 1;
    const int tz = rz < e[2] ? rz : e[2] - 1;
    ZoneCtx zc;
    zc.s = s;
    zc.bflag = bflag;
    double hh[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        hh[d] = (blk.ptmax[d] - blk.ptmin[d]) / (s - 1);
        zc.cf[d] = axis_coef(hh[d]);
    }
    zc.a[0] = o[0] + PW + tx;
    zc.a[1] = o[1] + PW + ty;
    zc.a[2] = o[2] + PW + tz;
    zc.st[0] = 1;
    zc.st[1] = TX;
    zc.st[2] = TX * TY;
    zc.tc = (tx + PW) + TX * ((ty + PW) + TY * (tz + PW));
    const int mj = BX;            // stride of mxj along y
    const int mk = BX * BY;       // stride of mxk/myk along z
    const double* mxj_z = mxj + tx + BX * ((ty + PW) + TY * tz);
    const double* mxk_z = mxk + tx + BX * (ty + BY * (tz + PW));
    const double* myk_z = myk + tx + BX * (ty + BY * (tz + PW));

    const int za0 = zc.a[0], za1 = zc.a[1], za2 = zc.a[2];
    const int64_t pidx = off + za0 + (int64_t)s * (za1 + (int64_t)s * za2);
    auto pv = [&](int v) { return __ldg(A.u.p[v] + pidx); };
    auto store = [&](int v, double val) {
        if (active) A.rhs.p[v][pidx] = val;
    };

    // coordinates and radius rounded exactly as the reference computes them
    // (pmin + i*h, no contraction), so a face point at the origin gives the
    // reference's infinite 1/r
    const double x = __dadd_rn(blk.ptmin[0], __dmul_rn((double)za0, hh[0]));
    const double y = __dadd_rn(blk.ptmin[1], __dmul_rn((double)za1, hh[1]));
    const double z = __dadd_rn(blk.ptmin[2], __dmul_rn((double)za2, hh[2]));
    const double r_coord =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    const double eta = [&] {
        const double w = r_coord / A.prm.eta_width;
        const double arg = -w * w * w * w;
        return (A.prm.eta_central - A.prm.eta_outer) * exp(arg) + A.prm.eta_outer;
    }();
    const bool onface = ((bflag & 1u) && za0 == PW) || ((bflag & 2u) && za0 == s - PW - 1) ||
                        ((bflag & 4u) && za1 == PW) || ((bflag & 8u) && za1 == s - PW - 1) ||
                        ((bflag & 16u) && za2 == PW) || ((bflag & 32u) && za2 == s - PW - 1);
    const double inv_r = onface ? 1.0 / r_coord : 0.0;

    const double alpha = pv(U_ALPHA), chi = pv(U_CHI), K = pv(U_K);
    double beta[3];
#pragma unroll
    for (int i = 0; i < 3; i++) beta[i] = pv(U_BETA0 + i);
    const double sig_c = A.prm.cako_enabled ? sqrt(chi) : 0.0;
    auto sigma = [&](int v) {
        return A.prm.cako_enabled
                   ? sig_c * (gauge_var(v) ? A.prm.eps_cako_gauge : A.prm.eps_cako_other)
                   : A.prm.ko_sigma;
    };
    // final value of variable v: (boundary face ? Sommerfeld : equations) + sigma KO
    auto finish = [&](int v, double eq, const double d1[3], double f, double ko) {
        double val = eq;
        if (onface) {
            // -inv_r (x dxf + y dyf + z dzf + falloff (f - f_inf)), rhs.cpp:542-547
            double t = __dadd_rn(__dadd_rn(__dmul_rn(x, d1[0]), __dmul_rn(y, d1[1])), __dmul_rn(z, d1[2]));
            t = __dadd_rn(t, __dmul_rn(falloff(v), __dsub_rn(f, asymptotic(v))));
            val = __dmul_rn(-inv_r, t);
        }
        return val + sigma(v) * ko;
    };
    const double l1 = A.prm.lambda[0], l2 = A.prm.lambda[1], l3 = A.prm.lambda[2],
                 l4 = A.prm.lambda[3];

    // conformal metric and its inverse (adjugate / determinant)
    double g[6];
#pragma unroll
    for (int c = 0; c < 6; c++) g[c] = pv(U_SYMGT0 + c);
    double ig[6];
    {
        const double c00 = g[3] * g[5] - g[4] * g[4];
        const double c01 = g[2] * g[4] - g[1] * g[5];
        const double c02 = g[1] * g[4] - g[2] * g[3];
        const double det = g[0] * c00 + g[1] * c01 + g[2] * c02;
        const double idet = 1.0 / det;
        ig[0] = c00 * idet;
        ig[1] = c01 * idet;
        ig[2] = c02 * idet;
        ig[3] = (g[0] * g[5] - g[2] * g[2]) * idet;
        ig[4] = (g[2] * g[1] - g[0] * g[4]) * idet;
        ig[5] = (g[0] * g[3] - g[1] * g[1]) * idet;
    }
    auto G = [&](int i, int j) { return g[sym(i, j)]; };
    auto IG = [&](int i, int j) { return ig[sym(i, j)]; };

    // staging order: beta0..2, gt0..5, Gt0..2, chi, alpha, At0..5, K, B0..2
    constexpr int order[NVARS] = {U_BETA0, U_BETA1, U_BETA2, U_SYMGT0, U_SYMGT1,
                                  U_SYMGT2, U_SYMGT3, U_SYMGT4, U_SYMGT5, U_GT0,
                                  U_GT1, U_GT2, U_CHI, U_ALPHA, U_SYMAT0, U_SYMAT1,
                                  U_SYMAT2, U_SYMAT3, U_SYMAT4, U_SYMAT5, U_K,
                                  U_B0, U_B1, U_B2};
    int step = 0;
    stage(order[0], tiles[0]);
    // Wait for the tile of order[step], start the next load, and (for
    // variables with second derivatives) run the mixed pass.
    auto next_tile = [&](bool second) -> const double* {
        cp_async_wait_all();
        __syncthreads();
        const double* cur = tiles[step & 1];
        if (step + 1 < NVARS) stage(order[step + 1], tiles[(step + 1) & 1]);
        if (second) {
            mixed_pass(cur, zc);
            __syncthreads();
        }
        step++;
        return cur;
    };

    double d1[3], d2[6], ko;

    // ---- beta: b_rhs, grad beta, and the second-derivative part of Gt_rhs
    double db[3][3];  // db[i][j] = d_j beta^i
    double GtA[3];    // accumulates the beta / CalGt / At parts of Gt_rhs
    double Gdiv[3] = {0.0, 0.0, 0.0};
    const double bfac = 0.75 * (A.prm.lambda_f[0] + A.prm.lambda_f[1] * alpha);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double* t = next_tile(true);
        zone_derivs<true>(zc, t, mxj_z, mxk_z, myk_z, mj, mk, d1, d2, ko);
#pragma unroll
        for (int j = 0; j < 3; j++) db[i][j] = d1[j];
        GtA[i] = ig[0] * d2[0] + ig[3] * d2[3] + ig[5] * d2[5] +
                 2.0 * (ig[1] * d2[1] + ig[2] * d2[2] + ig[4] * d2[4]);
#pragma unroll
        for (int j = 0; j < 3; j++) Gdiv[j] += d2[sym(j, i)];
        const double eq = bfac * pv(U_B0 + i) + l2 * (beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2]);
        store(U_BETA0 + i, finish(U_BETA0 + i, eq, d1, beta[i], ko));
    }
    const double divb = db[0][0] + db[1][1] + db[2][2];
#pragma unroll
    for (int i = 0; i < 3; i++)
        GtA[i] += (IG(i, 0) * Gdiv[0] + IG(i, 1) * Gdiv[1] + IG(i, 2) * Gdiv[2]) / 3.0;

    // ---- gt: gt_rhs, grad gt, ig^lm d_l d_m gt_ij
    double dg[6][3];
    double Lg[6];
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const int a = sym_a(c), b = sym_b(c);
        const double* t = next_tile(true);
        zone_derivs<true>(zc, t, mxj_z, mxk_z, myk_z, mj, mk, d1, d2, ko);
#pragma unroll
        for (int k = 0; k < 3; k++) dg[c][k] = d1[k];
        Lg[c] = ig[0] * d2[0] + ig[3] * d2[3] + ig[5] * d2[5] +
                2.0 * (ig[1] * d2[1] + ig[2] * d2[2] + ig[4] * d2[4]);
        double eq = beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2];
#pragma unroll
        for (int k = 0; k < 3; k++) eq += G(a, k) * db[k][b] + G(k, b) * db[k][a];
        eq += -2.0 / 3.0 * g[c] * divb - 2.0 * alpha * pv(U_SYMAT0 + c);
        store(U_SYMGT0 + c, finish(U_SYMGT0 + c, eq, d1, g[c], ko));
    }

    // ---- Christoffel symbols and the Christoffel part of the Ricci tensor
    // C1[k][i][j] = 1/2 (d_j g_ki + d_i g_kj - d_k g_ij), stored [k][sym(i,j)]
    double C1[3][6];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const int i = sym_a(c), j = sym_b(c);
            C1[k][c] = 0.5 * (dg[sym(k, i)][j] + dg[sym(k, j)][i] - dg[c][k]);
        }
    double C2[3][6];  // C2[i][sym(j,k)] = ig^im C1[m][jk]
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int c = 0; c < 6; c++)
            C2[i][c] = IG(i, 0) * C1[0][c] + IG(i, 1) * C1[1][c] + IG(i, 2) * C1[2][c];
    double CalGt[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        CalGt[i] = ig[0] * C2[i][0] + ig[3] * C2[i][3] + ig[5] * C2[i][5] +
                   2.0 * (ig[1] * C2[i][1] + ig[2] * C2[i][2] + ig[4] * C2[i][4]);
    double R[6];
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const int i = sym_a(c), j = sym_b(c);
        double rt = -0.5 * Lg[c];
#pragma unroll
        for (int k = 0; k < 3; k++) rt += 0.5 * CalGt[k] * (C1[i][sym(j, k)] + C1[j][sym(i, k)]);
        R[c] = rt;
    }
    // sum_k sum_lm ig^lm (C2[k][l][i] C1[j][k][m] + C2[k][l][j] C1[i][k][m]
    //                     + C2[k][i][m] C1[k][l][j])
    // with U[j][k][l] = ig^lm C1[j][k][m] (last index raised):
    //   = sum_kl C2[k][li] U[j][k][l] + C2[k][lj] U[i][k][l]
    //     + sum_km C2[k][im] U[k][j][m]
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double Uk[3][3];  // Uk[j][l] = U[j][k][l]
        double Uj[3][3];  // Uj[j][m] = U[k][j][m]
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int l = 0; l < 3; l++) {
                Uk[j][l] = IG(l, 0) * C1[j][sym(k, 0)] + IG(l, 1) * C1[j][sym(k, 1)] +
                           IG(l, 2) * C1[j][sym(k, 2)];
                Uj[j][l] = IG(l, 0) * C1[k][sym(j, 0)] + IG(l, 1) * C1[k][sym(j, 1)] +
                           IG(l, 2) * C1[k][sym(j, 2)];
            }
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const int i = sym_a(c), j = sym_b(c);
            double acc = 0.0;
#pragma unroll
            for (int l = 0; l < 3; l++)
                acc += C2[k][sym(l, i)] * Uk[j][l] + C2[k][sym(l, j)] * Uk[i][l] +
                       C2[k][sym(i, l)] * Uj[j][l];
            R[c] += acc;
        }
    }
    // beta / CalGt part of Gt_rhs
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double s2 = 2.0 / 3.0 * CalGt[i] * divb;
#pragma unroll
        for (int j = 0; j < 3; j++) s2 -= CalGt[j] * db[i][j];
        GtA[i] += s2;
    }

    // ---- Gt: 1/2 (g_ki d_j Gt^k + g_kj d_i Gt^k) into R; advection
    double advGt[3], koGt[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double* t = next_tile(false);
        zone_derivs<false>(zc, t, nullptr, nullptr, nullptr, 0, 0, d1, d2, ko);
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const int i = sym_a(c), j = sym_b(c);
            R[c] += 0.5 * (G(k, i) * d1[j] + G(k, j) * d1[i]);
        }
        advGt[k] = beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2];
        const double f = pv(U_GT0 + k);
        if (onface) store(U_GT0 + k, finish(U_GT0 + k, 0.0, d1, f, ko));
        koGt[k] = sigma(U_GT0 + k) * ko;
    }

    // ---- chi: Rphi into R, chi_rhs
    double dchi[3];
    {
        const double* t = next_tile(true);
        zone_derivs<true>(zc, t, mxj_z, mxk_z, myk_z, mj, mk, d1, d2, ko);
#pragma unroll
        for (int k = 0; k < 3; k++) dchi[k] = d1[k];
        const double ichi = 1.0 / chi;
        double T = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int l = 0; l < 3; l++)
                T += IG(k, l) * (d2[sym(k, l)] - 3.0 / (2.0 * chi) * dchi[k] * dchi[l]);
#pragma unroll
        for (int m = 0; m < 3; m++) T -= CalGt[m] * dchi[m];
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const int i = sym_a(c), j = sym_b(c);
            double sk = d2[c];
#pragma unroll
            for (int k = 0; k < 3; k++) sk -= C2[k][c] * dchi[k];
            R[c] += 0.5 * ichi * sk - 0.25 * ichi * ichi * dchi[i] * dchi[j] +
                    0.5 * ichi * g[c] * T;
        }
        const double eq = beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2] -
                          2.0 / 3.0 * chi * divb + 2.0 / 3.0 * chi * alpha * K;
        store(U_CHI, finish(U_CHI, eq, d1, chi, ko));
    }

    // ---- alpha: D_i D_j alpha, laplacian, a_rhs; X = alpha R - DDa
    double dal[3];
    double X[6];
    double lap;
    {
        const double* t = next_tile(true);
        zone_derivs<true>(zc, t, mxj_z, mxk_z, myk_z, mj, mk, d1, d2, ko);
#pragma unroll
        for (int k = 0; k < 3; k++) dal[k] = d1[k];
        const double ichi = 1.0 / chi;
        double igdchi_da = 0.0;  // ig^lm d_m chi d_l alpha
#pragma unroll
        for (int l = 0; l < 3; l++)
            igdchi_da += dal[l] * (IG(l, 0) * dchi[0] + IG(l, 1) * dchi[1] + IG(l, 2) * dchi[2]);
        lap = 0.0;
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const int i = sym_a(c), j = sym_b(c);
            double c3 = C2[0][c] * dal[0] + C2[1][c] * dal[1] + C2[2][c] * dal[2];
            c3 -= 0.5 * ichi * (dal[i] * dchi[j] + dal[j] * dchi[i] - g[c] * igdchi_da);
            const double dda = d2[c] - c3;
            lap += (i == j ? 1.0 : 2.0) * ig[c] * dda;
            X[c] = alpha * R[c] - dda;
        }
        lap *= chi;
        const double eq = l1 * (beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2]) - 2.0 * alpha * K;
        store(U_ALPHA, finish(U_ALPHA, eq, d1, alpha, ko));
    }

    // ---- At: A^ij, A_ij A^ij, Gt_rhs At-terms, At_rhs
    double At[6];
#pragma unroll
    for (int c = 0; c < 6; c++) At[c] = pv(U_SYMAT0 + c);
    auto AT = [&](int i, int j) { return At[sym(i, j)]; };
    double AUU[6];
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const int i = sym_a(c), j = sym_b(c);
        double sacc = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int l = 0; l < 3; l++) sacc += IG(i, k) * IG(j, l) * AT(k, l);
        AUU[c] = sacc;
    }
    const double sqrA = At[0] * AUU[0] + At[3] * AUU[3] + At[5] * AUU[5] +
                        2.0 * (At[1] * AUU[1] + At[2] * AUU[2] + At[4] * AUU[4]);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double sacc = 0.0;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            sacc -= 2.0 * AUU[sym(i, j)] * dal[j];
            sacc -= alpha * 3.0 / chi * AUU[sym(i, j)] * dchi[j];
        }
        double cc = 0.0;
#pragma unroll
        for (int c = 0; c < 6; c++) cc += (sym_a(c) == sym_b(c) ? 1.0 : 2.0) * C2[i][c] * AUU[c];
        GtA[i] += sacc + 2.0 * alpha * cc;
    }
    {
        double trX = 0.0;
#pragma unroll
        for (int c = 0; c < 6; c++) trX += (sym_a(c) == sym_b(c) ? 1.0 : 2.0) * ig[c] * X[c];
#pragma unroll
        for (int c = 0; c < 6; c++) X[c] = chi * (X[c] - g[c] * trX / 3.0);
    }
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const int a = sym_a(c), b = sym_b(c);
        const double* t = next_tile(false);
        zone_derivs<false>(zc, t, nullptr, nullptr, nullptr, 0, 0, d1, d2, ko);
        double eq = beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2];
#pragma unroll
        for (int k = 0; k < 3; k++) eq += AT(a, k) * db[k][b] + AT(k, b) * db[k][a];
        eq += -2.0 / 3.0 * At[c] * divb + X[c];
        double aa = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int l = 0; l < 3; l++) aa += AT(a, k) * IG(k, l) * AT(l, b);
        eq += alpha * (K * At[c] - 2.0 * aa);
        store(U_SYMAT0 + c, finish(U_SYMAT0 + c, eq, d1, At[c], ko));
    }

    // ---- K: K_rhs and the grad K part of Gt_rhs; final Gt_rhs
    double Gt_rhs[3];
    {
        const double* t = next_tile(false);
        zone_derivs<false>(zc, t, nullptr, nullptr, nullptr, 0, 0, d1, d2, ko);
        const double eq = beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2] - lap +
                          alpha * (K * K / 3.0 + sqrA);
        store(U_K, finish(U_K, eq, d1, K, ko));
#pragma unroll
        for (int i = 0; i < 3; i++) {
            Gt_rhs[i] = advGt[i] + GtA[i] -
                        alpha * 4.0 / 3.0 * (IG(i, 0) * d1[0] + IG(i, 1) * d1[1] + IG(i, 2) * d1[2]);
            if (!onface) store(U_GT0 + i, Gt_rhs[i] + koGt[i]);
        }
    }

    // ---- B: B_rhs
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double* t = next_tile(false);
        zone_derivs<false>(zc, t, nullptr, nullptr, nullptr, 0, 0, d1, d2, ko);
        const double Bi = pv(U_B0 + i);
        const double eq = Gt_rhs[i] - eta * Bi + l3 * (beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2]) -
                          l4 * advGt[i];
        store(U_B0 + i, finish(U_B0 + i, eq, d1, Bi, ko));
    }
}

// One brick per CTA: from the task list, or (tasks == nullptr) from
// blockIdx.x over the bricks of the single block passed by value.
template <int BX, int BY, int BZ, int MINB>
__global__ void __launch_bounds__(Brick<BX, BY, BZ>::THREADS, MINB)
rhs_kernel(RhsArgs A, const BssnBlockDesc* __restrict__ blocks,
           const BrickTask* __restrict__ tasks, BssnBlockDesc single) {
    extern __shared__ __align__(16) double smem[];
    int o[3], e[3];
    if (tasks != nullptr) {
        const BrickTask tk = tasks[blockIdx.x];
        const BssnBlockDesc blk = blocks[tk.blk];
        o[0] = tk.o[0]; o[1] = tk.o[1]; o[2] = tk.o[2];
        e[0] = tk.e[0]; e[1] = tk.e[1]; e[2] = tk.e[2];
        rhs_brick<BX, BY, BZ>(A, blk, o, e, smem);
    } else {
        const int n = single.sz - 2 * PW;
        const int nbx = (n + BX - 1) / BX, nby = (n + BY - 1) / BY;
        const int q = blockIdx.x;
        const int qx = q % nbx, qy = (q / nbx) % nby, qz = q / (nbx * nby);
        split1(n, BX, qx, o[0], e[0]);
        split1(n, BY, qy, o[1], e[1]);
        split1(n, BZ, qz, o[2], e[2]);
        rhs_brick<BX, BY, BZ>(A, single, o, e, smem);
    }
}

// ---------------------------------------------------------------------------
// Tile table and launchers.
// ---------------------------------------------------------------------------
namespace {
struct TileEntry {
    int bx, by, bz, threads;
    size_t smem;
    void (*kern)(RhsArgs, const BssnBlockDesc*, const BrickTask*, BssnBlockDesc);
};

// MINB: resident CTAs per SM the register allocation must allow
// (1 lets a thread use 255 registers; more CTAs cap registers and trade
// spills for latency hiding -- the autotuner measures which wins).
template <int BX, int BY, int BZ, int MINB = 1>
TileEntry make_entry() {
    using Bk = Brick<BX, BY, BZ>;
    return TileEntry{BX, BY, BZ, Bk::THREADS, Bk::SMEM_BYTES, rhs_kernel<BX, BY, BZ, MINB>};
}

const TileEntry* tile_table(int* count) {
    static const TileEntry table[] = {
        make_entry<8, 8, 4>(),
        make_entry<7, 7, 4>(),
        make_entry<8, 4, 4>(),
    };
    *count = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

int prepare(const TileEntry& t) {
    static bool done[16] = {false};
    int count;
    const TileEntry* base = tile_table(&count);
    const int id = (int)(&t - base);
    if (!done[id]) {
        cudaError_t e1 = cudaFuncSetAttribute(t.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
        if (e1 != cudaSuccess) return cuda_status(e1);
        done[id] = true;
    }
    return 0;
}
}  // namespace

int prepare_all_tiles() {
    int c;
    const TileEntry* tab = tile_table(&c);
    for (int t = 0; t < c; t++) {
        int st = prepare(tab[t]);
        if (st) return st;
    }
    return 0;
}

// Host replay of the brick kernel's shared-memory indexing: for a tile
// shape, every brick extent the splitter can produce (3..B per axis), every
// block-face combination and every thread, check that each tile and mixed-
// scratch element a thread reads lies inside its array.  Returns the number
// of out-of-range reads (0 = the kernel's smem accesses are all in bounds).
namespace {
// positions along one axis read by the d1/d2/KO stencils at coordinate a
void read_span(int a, int s, bool lo, bool hi, int& pmin, int& pmax) {
    const int ie = s - 3;
    if (lo && a <= 5) {
        pmin = 3;
        pmax = 8;
        return;
    }
    if (hi && a >= ie - 3) {
        pmin = ie - 6;
        pmax = ie - 1;
        return;
    }
    pmin = a - 3;
    pmax = a + 3;
}

template <int BX, int BY, int BZ>
long check_tile_shape() {
    using Bk = Brick<BX, BY, BZ>;
    const int B[3] = {BX, BY, BZ};
    const int T[3] = {Bk::TX, Bk::TY, Bk::TZ};
    long bad = 0;
    for (int e0 = 3; e0 <= BX; e0++)
        for (int e1 = 3; e1 <= BY; e1++)
            for (int e2 = 3; e2 <= BZ; e2++)
                for (int face = 0; face < 4; face++) {
                    // brick at the lower faces (o = 0) or upper faces of a 55 block
                    const int s = 55;
                    const int e[3] = {e0, e1, e2};
                    int o[3];
                    for (int d = 0; d < 3; d++) o[d] = (face & 1) ? (s - 6 - e[d]) : 0;
                    const bool blo = (face & 2) != 0, bhi = (face & 2) != 0;
                    for (int tid = 0; tid < Bk::THREADS; tid++) {
                        const bool in_brick = tid < Bk::NZ;
                        const int r3[3] = {in_brick ? tid % BX : 0,
                                           in_brick ? (tid / BX) % BY : 0,
                                           in_brick ? tid / (BX * BY) : 0};
                        const bool active = in_brick && r3[0] < e[0] && r3[1] < e[1] && r3[2] < e[2];
                        int t3[3];
                        for (int d = 0; d < 3; d++) t3[d] = r3[d] < e[d] ? r3[d] : e[d] - 1;
                        for (int d = 0; d < 3; d++) {
                            const int a = o[d] + PW + t3[d];
                            int pmin, pmax;
                            read_span(a, s, blo, bhi, pmin, pmax);
                            // tile coordinate = position - o: inside the array
                            // for every thread (tile and mixed scratch share the
                            // extent T along the axis), inside the staged region
                            // [0, e+6) for threads that own a zone
                            if (pmin - o[d] < 0 || pmax - o[d] >= T[d]) bad++;
                            if (active && pmax - o[d] >= e[d] + 2 * PW) bad++;
                            if (t3[d] >= B[d]) bad++;
                            // the closure tables cover a in [3, s-3) only
                            if (a < 3 || a > s - 4) bad++;
                        }
                    }
                }
    return bad;
}
}  // namespace

long tile_selfcheck(int tile) {
    switch (tile) {
        case 0: return check_tile_shape<8, 8, 4>();
        case 1: return check_tile_shape<7, 7, 4>();
        case 2: return check_tile_shape<8, 4, 4>();
        default: return -1;
    }
}

int tile_count() {
    int c;
    tile_table(&c);
    return c;
}

int tile_info(int tile, int info[4]) {
    int c;
    const TileEntry* t = tile_table(&c);
    if (tile < 0 || tile >= c) return BSSN_EINVAL;
    info[0] = t[tile].bx;
    info[1] = t[tile].by;
    info[2] = t[tile].bz;
    info[3] = t[tile].threads;
    return 0;
}

void build_tasks(const BssnBlockDesc* blocks, int nblocks, int tile,
                 std::vector<BrickTask>& out) {
    int c;
    const TileEntry& t = tile_table(&c)[tile];
    for (int b = 0; b < nblocks; b++) {
        const int n = blocks[b].sz - 2 * PW;
        const int nbx = (n + t.bx - 1) / t.bx, nby = (n + t.by - 1) / t.by,
                  nbz = (n + t.bz - 1) / t.bz;
        for (int qz = 0; qz < nbz; qz++)
            for (int qy = 0; qy < nby; qy++)
                for (int qx = 0; qx < nbx; qx++) {
                    BrickTask k;
                    int o, e;
                    k.blk = b;
                    split1(n, t.bx, qx, o, e); k.o[0] = (int16_t)o; k.e[0] = (int16_t)e;
                    split1(n, t.by, qy, o, e); k.o[1] = (int16_t)o; k.e[1] = (int16_t)e;
                    split1(n, t.bz, qz, o, e); k.o[2] = (int16_t)o; k.e[2] = (int16_t)e;
                    out.push_back(k);
                }
    }
}

int launch_rhs_tasks(int tile, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, cudaStream_t s) {
    int c;
    const TileEntry* tab = tile_table(&c);
    if (tile < 0 || tile >= c) return BSSN_EINVAL;
    if (ntasks <= 0) return 0;
    const TileEntry& t = tab[tile];
    int st = prepare(t);
    if (st) return st;
    t.kern<<<ntasks, t.threads, t.smem, s>>>(A, blocks_dev, tasks_dev, BssnBlockDesc{});
    return cuda_status(cudaGetLastError());
}

int launch_rhs_single(int tile, const RhsArgs& A, const BssnBlockDesc& blk,
                      cudaStream_t s) {
    int c;
    const TileEntry* tab = tile_table(&c);
    if (tile < 0 || tile >= c) return BSSN_EINVAL;
    const TileEntry& t = tab[tile];
    int st = prepare(t);
    if (st) return st;
    const int n = blk.sz - 2 * PW;
    const int nb = ((n + t.bx - 1) / t.bx) * ((n + t.by - 1) / t.by) * ((n + t.bz - 1) / t.bz);
    t.kern<<<nb, t.threads, t.smem, s>>>(A, nullptr, nullptr, blk);
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
