// The BSSN equations at one zone, generic over where the zone's derivatives
// come from (the fused kernel forms them from its shared-memory tile; the
// split path loads them from the derivative scratch).
//
// Semantics follow BSSN_GR/src/rhs.cpp:80-504 (derivatives -> equations ->
// Sommerfeld BC on boundary faces -> + sigma * KO) with the equations of
// CodeGen/bssn.py:70-230 (standard gauge, constant eta): out = (on a physical
// boundary face ? BC : equations) + sigma * (KO_x + KO_y + KO_z).  The
// derivatives are consumed in stage_order(), folded into the equations at
// once so the live set stays small:
//   beta -> gt -> Christoffels/Ricci core -> Gt -> chi -> alpha -> At -> K -> B
#pragma once
#include "rhs_brick.cuh"

namespace bssn {
namespace {

// get(BoolTag<SECOND>{}, d1, d2, ko) must deliver, on its n-th call, the
// derivatives of variable stage_order(n): gradient d1[3], (if SECOND) the
// second derivatives d2[6] (xx,xy,xz,yy,yz,zz) and the summed KO term;
// pv(v) the zone's value of variable v; store(v, r) receives the zone's
// right-hand side of variable v (each v once).  za are the zone's padded
// block coordinates.
template <class Get, class PV, class Store>
__device__ __forceinline__ void zone_equations(const RhsArgs& A, const BssnBlockDesc& blk,
                                               int za0, int za1, int za2, Get&& get, PV&& pv,
                                               Store&& store) {
    const int s = blk.sz;
    const unsigned bflag = blk.bflag;
    double hh[3];
#pragma unroll
    for (int d = 0; d < 3; d++) hh[d] = (blk.ptmax[d] - blk.ptmin[d]) / (s - 1);

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

    double d1[3], d2[6], ko;

    // ---- beta: b_rhs, grad beta, and the second-derivative part of Gt_rhs
    double db[3][3];  // db[i][j] = d_j beta^i
    double GtA[3];    // accumulates the beta / CalGt / At parts of Gt_rhs
    double Gdiv[3] = {0.0, 0.0, 0.0};
    const double bfac = 0.75 * (A.prm.lambda_f[0] + A.prm.lambda_f[1] * alpha);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        get(BoolTag<true>{}, d1, d2, ko);
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
        get(BoolTag<true>{}, d1, d2, ko);
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
        get(BoolTag<false>{}, d1, d2, ko);
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
        get(BoolTag<true>{}, d1, d2, ko);
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
        get(BoolTag<true>{}, d1, d2, ko);
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
        get(BoolTag<false>{}, d1, d2, ko);
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
        get(BoolTag<false>{}, d1, d2, ko);
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
        get(BoolTag<false>{}, d1, d2, ko);
        const double Bi = pv(U_B0 + i);
        const double eq = Gt_rhs[i] - eta * Bi + l3 * (beta[0] * d1[0] + beta[1] * d1[1] + beta[2] * d1[2]) -
                          l4 * advGt[i];
        store(U_B0 + i, finish(U_B0 + i, eq, d1, Bi, ko));
    }

}

}  // namespace
}  // namespace bssn
