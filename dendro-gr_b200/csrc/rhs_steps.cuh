// The BSSN equations at one zone, cut into one step per evolved variable so
// that a kernel can run them from a runtime loop over the variables: after
// the derivatives of variable stage_order(K) are formed, step<K>() folds them
// into the zone's equation state and stores the right-hand sides that become
// final.  The arithmetic is that of rhs_equations.cuh (same expressions, same
// order): BSSN_GR/src/rhs.cpp:80-504 semantics with the equations of
// CodeGen/bssn.py:70-230 (standard gauge), Sommerfeld BC on physical faces
// (rhs.cpp:511-631) and + sigma * KO (rhs.cpp:338-492).
//
// Every array member is indexed with compile-time constants inside each step,
// so the state stays in registers across the loop.  T[] is reused: steps 0-2
// keep the beta divergence sums in T[18..20], steps 3-8 the metric gradients
// dg[6][3] = T[0..17] and ig^lm d_l d_m gt_ij = T[18..23]; from step 8 on it
// holds advGt T[0..2], KO of Gt T[3..5], d chi T[6..8], d alpha T[9..11],
// X T[12..17], the conformal laplacian of alpha T[18], A_ij A^ij T[19] and
// Gt_rhs T[20..22].
#pragma once
#include "rhs_brick.cuh"

namespace bssn {
namespace {

struct EqSteps {
    // zone constants
    double x, y, z, inv_r, eta;
    bool onface;
    double ig[6];
    // state carried between variables
    double db[3][3];  // db[i][j] = d_j beta^i
    double GtA[3];    // beta / CalGt / At parts of Gt_rhs
    double divb;
    double T[24];
    double C2[3][6];  // C2[i][sym(j,k)] = ig^im C1[m][jk]
    double CalGt[3];
    double R[6];

    // pv(v): the zone's value of variable v
    template <class PV>
    __device__ __forceinline__ void begin(const RhsArgs& A, const BssnBlockDesc& blk, int za0,
                                          int za1, int za2, PV&& pv) {
        const int s = blk.sz;
        const unsigned bflag = blk.bflag;
        double hh[3];
#pragma unroll
        for (int d = 0; d < 3; d++) hh[d] = (blk.ptmax[d] - blk.ptmin[d]) / (s - 1);
        // coordinates and radius rounded exactly as the reference computes
        // them (pmin + i*h, no contraction)
        x = __dadd_rn(blk.ptmin[0], __dmul_rn((double)za0, hh[0]));
        y = __dadd_rn(blk.ptmin[1], __dmul_rn((double)za1, hh[1]));
        z = __dadd_rn(blk.ptmin[2], __dmul_rn((double)za2, hh[2]));
        const double r_coord =
            __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
        {
            const double w = r_coord / A.prm.eta_width;
            const double arg = -w * w * w * w;
            eta = (A.prm.eta_central - A.prm.eta_outer) * exp(arg) + A.prm.eta_outer;
        }
        onface = ((bflag & 1u) && za0 == PW) || ((bflag & 2u) && za0 == s - PW - 1) ||
                 ((bflag & 4u) && za1 == PW) || ((bflag & 8u) && za1 == s - PW - 1) ||
                 ((bflag & 16u) && za2 == PW) || ((bflag & 32u) && za2 == s - PW - 1);
        inv_r = onface ? 1.0 / r_coord : 0.0;
        double g[6];
#pragma unroll
        for (int c = 0; c < 6; c++) g[c] = pv(U_SYMGT0 + c);
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
        T[18] = T[19] = T[20] = 0.0;
    }

    __device__ __forceinline__ double IG(int i, int j) const { return ig[sym(i, j)]; }

    template <class PV>
    __device__ __forceinline__ double sigma(const RhsArgs& A, int v, PV&& pv) const {
        return A.prm.cako_enabled
                   ? sqrt(pv(U_CHI)) * (gauge_var(v) ? A.prm.eps_cako_gauge : A.prm.eps_cako_other)
                   : A.prm.ko_sigma;
    }

    // (boundary face ? Sommerfeld : equations) + sigma KO
    template <class PV>
    __device__ __forceinline__ double finish(const RhsArgs& A, int v, double eq, const double d1[3],
                                             double f, double ko, PV&& pv) const {
        double val = eq;
        if (onface) {
            double t = __dadd_rn(__dadd_rn(__dmul_rn(x, d1[0]), __dmul_rn(y, d1[1])), __dmul_rn(z, d1[2]));
            t = __dadd_rn(t, __dmul_rn(falloff(v), __dsub_rn(f, asymptotic(v))));
            val = __dmul_rn(-inv_r, t);
        }
        return val + sigma(A, v, pv) * ko;
    }

    template <class PV>
    __device__ __forceinline__ double adv(const double d1[3], PV&& pv) const {
        return pv(U_BETA0) * d1[0] + pv(U_BETA1) * d1[1] + pv(U_BETA2) * d1[2];
    }

    // One variable's step.  K = position in stage_order().
    template <int K, class PV, class Store>
    __device__ __forceinline__ void step(const RhsArgs& A, const double d1[3], const double d2[6],
                                         double ko, PV&& pv, Store&& store) {
        if constexpr (K < 3) {
            // ---- beta^i: b_rhs, grad beta, second-derivative part of Gt_rhs
            constexpr int i = K;
            const double alpha = pv(U_ALPHA);
            const double bfac = 0.75 * (A.prm.lambda_f[0] + A.prm.lambda_f[1] * alpha);
#pragma unroll
            for (int j = 0; j < 3; j++) db[i][j] = d1[j];
            GtA[i] = ig[0] * d2[0] + ig[3] * d2[3] + ig[5] * d2[5] +
                     2.0 * (ig[1] * d2[1] + ig[2] * d2[2] + ig[4] * d2[4]);
#pragma unroll
            for (int j = 0; j < 3; j++) T[18 + j] += d2[sym(j, i)];
            const double eq = bfac * pv(U_B0 + i) + A.prm.lambda[1] * adv(d1, pv);
            store(U_BETA0 + i, finish(A, U_BETA0 + i, eq, d1, pv(U_BETA0 + i), ko, pv));
            if constexpr (i == 2) {
                divb = db[0][0] + db[1][1] + db[2][2];
#pragma unroll
                for (int m = 0; m < 3; m++)
                    GtA[m] += (IG(m, 0) * T[18] + IG(m, 1) * T[19] + IG(m, 2) * T[20]) / 3.0;
            }
        } else if constexpr (K < 9) {
            // ---- gt_c: gt_rhs, grad gt, ig^lm d_l d_m gt_c
            constexpr int c = K - 3;
            constexpr int a = sym_a(c), b = sym_b(c);
#pragma unroll
            for (int k = 0; k < 3; k++) T[3 * c + k] = d1[k];
            T[18 + c] = ig[0] * d2[0] + ig[3] * d2[3] + ig[5] * d2[5] +
                        2.0 * (ig[1] * d2[1] + ig[2] * d2[2] + ig[4] * d2[4]);
            auto G = [&](int p, int q) { return pv(U_SYMGT0 + sym(p, q)); };
            double eq = adv(d1, pv);
#pragma unroll
            for (int k = 0; k < 3; k++) eq += G(a, k) * db[k][b] + G(k, b) * db[k][a];
            eq += -2.0 / 3.0 * pv(U_SYMGT0 + c) * divb - 2.0 * pv(U_ALPHA) * pv(U_SYMAT0 + c);
            store(U_SYMGT0 + c, finish(A, U_SYMGT0 + c, eq, d1, pv(U_SYMGT0 + c), ko, pv));
            if constexpr (c == 5) christoffel(pv);
        } else if constexpr (K < 12) {
            // ---- Gt^k: 1/2 (g_ki d_j Gt^k + g_kj d_i Gt^k) into R, advection
            constexpr int k = K - 9;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int i = sym_a(c), j = sym_b(c);
                R[c] += 0.5 * (pv(U_SYMGT0 + sym(k, i)) * d1[j] + pv(U_SYMGT0 + sym(k, j)) * d1[i]);
            }
            T[k] = adv(d1, pv);
            const double f = pv(U_GT0 + k);
            if (onface) store(U_GT0 + k, finish(A, U_GT0 + k, 0.0, d1, f, ko, pv));
            T[3 + k] = sigma(A, U_GT0 + k, pv) * ko;
        } else if constexpr (K == 12) {
            // ---- chi: Rphi into R, chi_rhs
            const double chi = pv(U_CHI);
#pragma unroll
            for (int k = 0; k < 3; k++) T[6 + k] = d1[k];
            const double ichi = 1.0 / chi;
            double Tr = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int l = 0; l < 3; l++)
                    Tr += IG(k, l) * (d2[sym(k, l)] - 3.0 / (2.0 * chi) * T[6 + k] * T[6 + l]);
#pragma unroll
            for (int m = 0; m < 3; m++) Tr -= CalGt[m] * T[6 + m];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int i = sym_a(c), j = sym_b(c);
                double sk = d2[c];
#pragma unroll
                for (int k = 0; k < 3; k++) sk -= C2[k][c] * T[6 + k];
                R[c] += 0.5 * ichi * sk - 0.25 * ichi * ichi * T[6 + i] * T[6 + j] +
                        0.5 * ichi * pv(U_SYMGT0 + c) * Tr;
            }
            const double eq = adv(d1, pv) - 2.0 / 3.0 * chi * divb + 2.0 / 3.0 * chi * pv(U_ALPHA) * pv(U_K);
            store(U_CHI, finish(A, U_CHI, eq, d1, chi, ko, pv));
        } else if constexpr (K == 13) {
            // ---- alpha: D_i D_j alpha, laplacian, a_rhs; X = alpha R - DDa;
            // then the At-only parts: A^ij A_ij, Gt_rhs At-terms, X trace-free
            const double chi = pv(U_CHI), alpha = pv(U_ALPHA);
#pragma unroll
            for (int k = 0; k < 3; k++) T[9 + k] = d1[k];
            const double ichi = 1.0 / chi;
            double igdchi_da = 0.0;  // ig^lm d_m chi d_l alpha
#pragma unroll
            for (int l = 0; l < 3; l++)
                igdchi_da += T[9 + l] * (IG(l, 0) * T[6] + IG(l, 1) * T[7] + IG(l, 2) * T[8]);
            double lap = 0.0;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int i = sym_a(c), j = sym_b(c);
                double c3 = C2[0][c] * T[9] + C2[1][c] * T[10] + C2[2][c] * T[11];
                c3 -= 0.5 * ichi * (T[9 + i] * T[6 + j] + T[9 + j] * T[6 + i] - pv(U_SYMGT0 + c) * igdchi_da);
                const double dda = d2[c] - c3;
                lap += (i == j ? 1.0 : 2.0) * ig[c] * dda;
                T[12 + c] = alpha * R[c] - dda;
            }
            T[18] = lap * chi;
            const double eq = A.prm.lambda[0] * adv(d1, pv) - 2.0 * alpha * pv(U_K);
            store(U_ALPHA, finish(A, U_ALPHA, eq, d1, alpha, ko, pv));

            auto AT = [&](int p, int q) { return pv(U_SYMAT0 + sym(p, q)); };
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
            T[19] = AT(0, 0) * AUU[0] + AT(1, 1) * AUU[3] + AT(2, 2) * AUU[5] +
                    2.0 * (AT(0, 1) * AUU[1] + AT(0, 2) * AUU[2] + AT(1, 2) * AUU[4]);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                double sacc = 0.0;
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    sacc -= 2.0 * AUU[sym(i, j)] * T[9 + j];
                    sacc -= alpha * 3.0 / chi * AUU[sym(i, j)] * T[6 + j];
                }
                double cc = 0.0;
#pragma unroll
                for (int c = 0; c < 6; c++) cc += (sym_a(c) == sym_b(c) ? 1.0 : 2.0) * C2[i][c] * AUU[c];
                GtA[i] += sacc + 2.0 * alpha * cc;
            }
            double trX = 0.0;
#pragma unroll
            for (int c = 0; c < 6; c++) trX += (sym_a(c) == sym_b(c) ? 1.0 : 2.0) * ig[c] * T[12 + c];
#pragma unroll
            for (int c = 0; c < 6; c++) T[12 + c] = chi * (T[12 + c] - pv(U_SYMGT0 + c) * trX / 3.0);
        } else if constexpr (K < 20) {
            // ---- At_c: At_rhs
            constexpr int c = K - 14;
            constexpr int a = sym_a(c), b = sym_b(c);
            auto AT = [&](int p, int q) { return pv(U_SYMAT0 + sym(p, q)); };
            const double Atc = pv(U_SYMAT0 + c), alpha = pv(U_ALPHA);
            double eq = adv(d1, pv);
#pragma unroll
            for (int k = 0; k < 3; k++) eq += AT(a, k) * db[k][b] + AT(k, b) * db[k][a];
            eq += -2.0 / 3.0 * Atc * divb + T[12 + c];
            double aa = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int l = 0; l < 3; l++) aa += AT(a, k) * IG(k, l) * AT(l, b);
            eq += alpha * (pv(U_K) * Atc - 2.0 * aa);
            store(U_SYMAT0 + c, finish(A, U_SYMAT0 + c, eq, d1, Atc, ko, pv));
        } else if constexpr (K == 20) {
            // ---- K: K_rhs, the grad K part of Gt_rhs, final Gt_rhs
            const double alpha = pv(U_ALPHA), Kv = pv(U_K);
            const double eq = adv(d1, pv) - T[18] + alpha * (Kv * Kv / 3.0 + T[19]);
            store(U_K, finish(A, U_K, eq, d1, Kv, ko, pv));
#pragma unroll
            for (int i = 0; i < 3; i++) {
                T[20 + i] = T[i] + GtA[i] -
                            alpha * 4.0 / 3.0 * (IG(i, 0) * d1[0] + IG(i, 1) * d1[1] + IG(i, 2) * d1[2]);
                if (!onface) store(U_GT0 + i, T[20 + i] + T[3 + i]);
            }
        } else {
            // ---- B^i: B_rhs
            constexpr int i = K - 21;
            const double Bi = pv(U_B0 + i);
            const double eq = T[20 + i] - eta * Bi + A.prm.lambda[2] * adv(d1, pv) - A.prm.lambda[3] * T[i];
            store(U_B0 + i, finish(A, U_B0 + i, eq, d1, Bi, ko, pv));
        }
    }

    // Christoffel symbols and the Christoffel part of the Ricci tensor, from
    // the metric gradients dg = T[0..17] and T[18..23] = ig^lm d_l d_m gt.
    template <class PV>
    __device__ __forceinline__ void christoffel(PV&& pv) {
        auto DG = [&](int c, int k) { return T[3 * c + k]; };
        double C1[3][6];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int i = sym_a(c), j = sym_b(c);
                C1[k][c] = 0.5 * (DG(sym(k, i), j) + DG(sym(k, j), i) - DG(c, k));
            }
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int c = 0; c < 6; c++)
                C2[i][c] = IG(i, 0) * C1[0][c] + IG(i, 1) * C1[1][c] + IG(i, 2) * C1[2][c];
#pragma unroll
        for (int i = 0; i < 3; i++)
            CalGt[i] = ig[0] * C2[i][0] + ig[3] * C2[i][3] + ig[5] * C2[i][5] +
                       2.0 * (ig[1] * C2[i][1] + ig[2] * C2[i][2] + ig[4] * C2[i][4]);
#pragma unroll
        for (int c = 0; c < 6; c++) {
            const int i = sym_a(c), j = sym_b(c);
            double rt = -0.5 * T[18 + c];
#pragma unroll
            for (int k = 0; k < 3; k++) rt += 0.5 * CalGt[k] * (C1[i][sym(j, k)] + C1[j][sym(i, k)]);
            R[c] = rt;
        }
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double Uk[3][3];  // Uk[j][l] = ig^lm C1[j][k][m]
            double Uj[3][3];  // Uj[j][m] = ig^ml C1[k][j][l]
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
        (void)pv;
    }
};

}  // namespace
}  // namespace bssn
