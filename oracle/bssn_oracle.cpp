// Test infrastructure only: the CPU oracle (see bssn_oracle.h).  Loaded by
// tests/, the smoke check and bench.py's CPU-baseline leg, never by the
// product library.  Build: make -C oracle (g++ -O2 -ffp-contract=off).
//
// The stencils keep the reference's expression order so that, compiled
// without floating-point contraction, they are bit-identical to
// BSSN_GR/src/derivs.cpp.  The pointwise BSSN equations are written from the
// symbolic definitions in CodeGen/bssn.py and CodeGen/dendro.py as plain
// tensor loops (not from the generated C), so they agree with the reference
// to rounding only.
#include "bssn_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

enum {
    U_ALPHA = 0, U_CHI, U_K, U_GT0, U_GT1, U_GT2, U_BETA0, U_BETA1, U_BETA2,
    U_B0, U_B1, U_B2, U_SYMGT0, U_SYMGT1, U_SYMGT2, U_SYMGT3, U_SYMGT4,
    U_SYMGT5, U_SYMAT0, U_SYMAT1, U_SYMAT2, U_SYMAT3, U_SYMAT4, U_SYMAT5,
    NVARS
};

inline int sym(int i, int j) {
    static const int m[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    return m[i][j];
}

// ---------------------------------------------------------------------------
// Stencils: BSSN_GR/src/derivs.cpp:2619-3312 (deriv644_*), :964-1305
// (ko_deriv42_*).  dir = 0,1,2 for x,y,z.
// ---------------------------------------------------------------------------

// Loop ranges of the first-derivative stencils: x over all j,k
// (derivs.cpp:2627-2633), y over all k (:2728-2734), z interior only.
void first_range(int dir, const unsigned* sz, int lo[3], int hi[3]) {
    for (int d = 0; d < 3; d++) {
        lo[d] = 3;
        hi[d] = (int)sz[d] - 3;
    }
    if (dir == 0) { lo[1] = 0; hi[1] = sz[1]; lo[2] = 0; hi[2] = sz[2]; }
    if (dir == 1) { lo[2] = 0; hi[2] = sz[2]; }
}

void deriv644(double* D, const double* u, double dx, const unsigned* sz,
              unsigned bflag, int dir) {
    const double idx = 1.0 / dx;
    const double idx_by_12 = idx / 12.0;
    const double idx_by_60 = idx / 60.0;
    const int nx = sz[0], ny = sz[1];
    const int n = dir == 0 ? 1 : (dir == 1 ? nx : nx * ny);
    int lo[3], hi[3];
    first_range(dir, sz, lo, hi);
    const int N = sz[dir];
    const int ie = N - 3;
    for (int k = lo[2]; k < hi[2]; k++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int i = lo[0]; i < hi[0]; i++) {
                const int pp = i + nx * (j + ny * k);
                D[pp] = (-u[pp - 3 * n] + 9.0 * u[pp - 2 * n] -
                         45.0 * u[pp - n] + 45.0 * u[pp + n] -
                         9.0 * u[pp + 2 * n] + u[pp + 3 * n]) *
                        idx_by_60;
            }
    const bool lo_face = bflag & (1u << (2 * dir));
    const bool hi_face = bflag & (1u << (2 * dir + 1));
    if (!lo_face && !hi_face) return;
    for (int k = lo[2]; k < hi[2]; k++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int i = lo[0]; i < hi[0]; i++) {
                const int c[3] = {i, j, k};
                const int a = c[dir];
                // base = index of the point with along-coordinate 0
                const int base = i + nx * (j + ny * k) - a * n;
                auto U = [&](int m) { return u[base + m * n]; };
                double* out = &D[base + a * n];
                if (lo_face) {
                    if (a == 3)
                        *out = (-25.0 * U(3) + 48.0 * U(4) - 36.0 * U(5) +
                                16.0 * U(6) - 3.0 * U(7)) * idx_by_12;
                    else if (a == 4)
                        *out = (-3.0 * U(3) - 10.0 * U(4) + 18.0 * U(5) -
                                6.0 * U(6) + U(7)) * idx_by_12;
                    else if (a == 5)
                        *out = (+U(3) - 8.0 * U(4) + 8.0 * U(6) - U(7)) *
                               idx_by_12;
                }
                if (hi_face) {
                    if (a == ie - 3)
                        *out = (+U(ie - 5) - 8.0 * U(ie - 4) + 8.0 * U(ie - 2) -
                                U(ie - 1)) * idx_by_12;
                    else if (a == ie - 2)
                        *out = (-U(ie - 5) + 6.0 * U(ie - 4) - 18.0 * U(ie - 3) +
                                10.0 * U(ie - 2) + 3.0 * U(ie - 1)) * idx_by_12;
                    else if (a == ie - 1)
                        *out = (3.0 * U(ie - 5) - 16.0 * U(ie - 4) +
                                36.0 * U(ie - 3) - 48.0 * U(ie - 2) +
                                25.0 * U(ie - 1)) * idx_by_12;
                }
            }
}

void deriv644_2(double* D, const double* u, double dx, const unsigned* sz,
                unsigned bflag, int dir) {
    const double idx_sqrd = 1.0 / (dx * dx);
    const double idx_sqrd_by_180 = idx_sqrd / 180.0;
    const double idx_sqrd_by_12 = idx_sqrd / 12.0;
    const int nx = sz[0], ny = sz[1], nz = sz[2];
    const int n = dir == 0 ? 1 : (dir == 1 ? nx : nx * ny);
    const int ie = sz[dir] - 3;
    const bool lo_face = bflag & (1u << (2 * dir));
    const bool hi_face = bflag & (1u << (2 * dir + 1));
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const int pp = i + nx * (j + ny * k);
                D[pp] = (2.0 * u[pp - 3 * n] - 27.0 * u[pp - 2 * n] +
                         270.0 * u[pp - n] - 490.0 * u[pp] + 270.0 * u[pp + n] -
                         27.0 * u[pp + 2 * n] + 2.0 * u[pp + 3 * n]) *
                        idx_sqrd_by_180;
            }
    if (!lo_face && !hi_face) return;
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const int c[3] = {i, j, k};
                const int a = c[dir];
                const int base = i + nx * (j + ny * k) - a * n;
                auto U = [&](int m) { return u[base + m * n]; };
                double* out = &D[base + a * n];
                if (lo_face) {
                    if (a == 3)
                        *out = (45.0 * U(3) - 154.0 * U(4) + 214.0 * U(5) -
                                156.0 * U(6) + 61.0 * U(7) - 10.0 * U(8)) *
                               idx_sqrd_by_12;
                    else if (a == 4)
                        *out = (10.0 * U(3) - 15.0 * U(4) - 4.0 * U(5) +
                                14.0 * U(6) - 6.0 * U(7) + U(8)) * idx_sqrd_by_12;
                    else if (a == 5)
                        *out = (-U(3) + 16.0 * U(4) - 30.0 * U(5) + 16.0 * U(6) -
                                U(7)) * idx_sqrd_by_12;
                }
                if (hi_face) {
                    if (a == ie - 3)
                        *out = (-U(ie - 5) + 16.0 * U(ie - 4) - 30.0 * U(ie - 3) +
                                16.0 * U(ie - 2) - U(ie - 1)) * idx_sqrd_by_12;
                    else if (a == ie - 2)
                        *out = (U(ie - 6) - 6.0 * U(ie - 5) + 14.0 * U(ie - 4) -
                                4.0 * U(ie - 3) - 15.0 * U(ie - 2) +
                                10.0 * U(ie - 1)) * idx_sqrd_by_12;
                    else if (a == ie - 1)
                        *out = (-10.0 * U(ie - 6) + 61.0 * U(ie - 5) -
                                156.0 * U(ie - 4) + 214.0 * U(ie - 3) -
                                154.0 * U(ie - 2) + 45.0 * U(ie - 1)) *
                               idx_sqrd_by_12;
                }
            }
}

void ko_deriv42(double* D, const double* u, double dx, const unsigned* sz,
                unsigned bflag, int dir) {
    const double pre_factor_6_dx = -1.0 / 64.0 / dx;
    const double smr3 = 59.0 / 48.0 * 64 * dx;
    const double smr2 = 43.0 / 48.0 * 64 * dx;
    const double smr1 = 49.0 / 48.0 * 64 * dx;
    const double spr3 = smr3, spr2 = smr2, spr1 = smr1;
    const int nx = sz[0], ny = sz[1], nz = sz[2];
    const int n = dir == 0 ? 1 : (dir == 1 ? nx : nx * ny);
    const int ie = sz[dir] - 3;
    const bool lo_face = bflag & (1u << (2 * dir));
    const bool hi_face = bflag & (1u << (2 * dir + 1));
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const int pp = i + nx * (j + ny * k);
                D[pp] = pre_factor_6_dx *
                        (-u[pp - 3 * n] + 6.0 * u[pp - 2 * n] -
                         15.0 * u[pp - n] + 20.0 * u[pp] - 15.0 * u[pp + n] +
                         6.0 * u[pp + 2 * n] - u[pp + 3 * n]);
            }
    if (!lo_face && !hi_face) return;
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const int c[3] = {i, j, k};
                const int a = c[dir];
                const int base = i + nx * (j + ny * k) - a * n;
                auto U = [&](int m) { return u[base + m * n]; };
                double* out = &D[base + a * n];
                if (lo_face) {
                    if (a == 3)
                        *out = (U(6) - 3.0 * U(5) + 3.0 * U(4) - U(3)) / smr3;
                    else if (a == 4)
                        *out = (U(7) - 6.0 * U(6) + 12.0 * U(5) - 10.0 * U(4) +
                                3.0 * U(3)) / smr2;
                    else if (a == 5)
                        *out = (U(8) - 6.0 * U(7) + 15.0 * U(6) - 19.0 * U(5) +
                                12.0 * U(4) - 3.0 * U(3)) / smr1;
                }
                if (hi_face) {
                    if (a == ie - 3)
                        *out = (U(ie - 6) - 6.0 * U(ie - 5) + 15.0 * U(ie - 4) -
                                19.0 * U(ie - 3) + 12.0 * U(ie - 2) -
                                3.0 * U(ie - 1)) / spr1;
                    else if (a == ie - 2)
                        *out = (U(ie - 5) - 6.0 * U(ie - 4) + 12.0 * U(ie - 3) -
                                10.0 * U(ie - 2) + 3.0 * U(ie - 1)) / spr2;
                    else if (a == ie - 1)
                        *out = (U(ie - 4) - 3.0 * U(ie - 3) + 3.0 * U(ie - 2) -
                                U(ie - 1)) / spr3;
                }
            }
}

// ---------------------------------------------------------------------------
// Pointwise BSSN equations, standard puncture gauge with constant eta:
// CodeGen/bssn.py:70-230 (bssn_puncture_gauge, unstaged) using the tensor
// helpers of CodeGen/dendro.py (lie :222, DiDj :173, laplacian :266,
// sqr :309, trace_free :323, Christoffels :395-483, compute_ricci :485-550).
// ---------------------------------------------------------------------------

// Vars whose second derivatives enter the equations (bssnrhs_derivs.h).
const bool kNeedsD2[NVARS] = {
    true,  true,  false, false, false, false, true,  true,  true,  false,
    false, false, true,  true,  true,  true,  true,  true,  false, false,
    false, false, false, false};

struct Pt {
    double u[NVARS];
    double d1[NVARS][3];
    double d2[NVARS][6];
};

void conformal_geometry(const Pt& P, double g[3][3], double ig[3][3],
                        double C1[3][3][3], double C2[3][3][3],
                        double CalGt[3]) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) g[i][j] = P.u[U_SYMGT0 + sym(i, j)];
    // inverse metric through the adjugate (dendro.py:375-392, 'ADJ')
    const double det = g[0][0] * (g[1][1] * g[2][2] - g[1][2] * g[2][1]) -
                       g[0][1] * (g[1][0] * g[2][2] - g[1][2] * g[2][0]) +
                       g[0][2] * (g[1][0] * g[2][1] - g[1][1] * g[2][0]);
    ig[0][0] = (g[1][1] * g[2][2] - g[1][2] * g[2][1]) / det;
    ig[0][1] = (g[0][2] * g[2][1] - g[0][1] * g[2][2]) / det;
    ig[0][2] = (g[0][1] * g[1][2] - g[0][2] * g[1][1]) / det;
    ig[1][1] = (g[0][0] * g[2][2] - g[0][2] * g[2][0]) / det;
    ig[1][2] = (g[0][2] * g[1][0] - g[0][0] * g[1][2]) / det;
    ig[2][2] = (g[0][0] * g[1][1] - g[0][1] * g[1][0]) / det;
    ig[1][0] = ig[0][1];
    ig[2][0] = ig[0][2];
    ig[2][1] = ig[1][2];
    // dg[i][j][k] = d_k g_ij
    double dg[3][3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) dg[i][j][k] = P.d1[U_SYMGT0 + sym(i, j)][k];
    // C1[k][i][j] = 1/2 (d_j g_ki + d_i g_kj - d_k g_ij)   (dendro.py:413-417)
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                C1[k][i][j] = 0.5 * (dg[k][i][j] + dg[k][j][i] - dg[i][j][k]);
    // C2[i][j][k] = ig[i][m] C1[m][j][k]                   (dendro.py:446-447)
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) {
                double s = 0.0;
                for (int m = 0; m < 3; m++) s += ig[i][m] * C1[m][j][k];
                C2[i][j][k] = s;
            }
    // CalGt[i] = ig[k][l] C2[i][k][l]                      (dendro.py:516)
    for (int i = 0; i < 3; i++) {
        double s = 0.0;
        for (int k = 0; k < 3; k++)
            for (int l = 0; l < 3; l++) s += ig[k][l] * C2[i][k][l];
        CalGt[i] = s;
    }
}

// Conformal Ricci tensor R = Rt + Rphi (dendro.py:485-550).
void ricci(const Pt& P, const double g[3][3], const double ig[3][3],
           const double C1[3][3][3], const double C2[3][3][3],
           const double CalGt[3], double R[3][3]) {
    const double chi = P.u[U_CHI];
    const double* dchi = P.d1[U_CHI];
    double ddchi[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) ddchi[i][j] = P.d2[U_CHI][sym(i, j)];
    // dGt[k][j] = d_j Gt^k
    double dGt[3][3];
    for (int k = 0; k < 3; k++)
        for (int j = 0; j < 3; j++) dGt[k][j] = P.d1[U_GT0 + k][j];
    // sum_{kl} ig^{kl}(d_k d_l chi - 3/(2 chi) d_k chi d_l chi) - CalGt^m d_m chi
    double trace_term = 0.0;
    for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++)
            trace_term += ig[k][l] * (ddchi[k][l] -
                                      3.0 / (2.0 * chi) * dchi[k] * dchi[l]);
    for (int m = 0; m < 3; m++) trace_term -= CalGt[m] * dchi[m];

    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double rt = 0.0;
            for (int l = 0; l < 3; l++)
                for (int m = 0; m < 3; m++)
                    rt += -0.5 * ig[l][m] * P.d2[U_SYMGT0 + sym(i, j)][sym(l, m)];
            for (int k = 0; k < 3; k++)
                rt += 0.5 * (g[k][i] * dGt[k][j] + g[k][j] * dGt[k][i]);
            for (int k = 0; k < 3; k++)
                rt += 0.5 * CalGt[k] * (C1[i][j][k] + C1[j][i][k]);
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++)
                    for (int m = 0; m < 3; m++)
                        rt += ig[l][m] * (C2[k][l][i] * C1[j][k][m] +
                                          C2[k][l][j] * C1[i][k][m] +
                                          C2[k][i][m] * C1[k][l][j]);
            double s = ddchi[i][j];
            for (int k = 0; k < 3; k++) s -= C2[k][j][i] * dchi[k];
            double rphi = 1.0 / (2.0 * chi) * s -
                          1.0 / (4.0 * chi * chi) * dchi[i] * dchi[j] +
                          1.0 / (2.0 * chi) * g[i][j] * trace_term;
            R[i][j] = rt + rphi;
        }
}

void rhs_point(const Pt& P, const OrcParams* prm, double eta,
               double out[NVARS]) {
    const double alpha = P.u[U_ALPHA], chi = P.u[U_CHI], K = P.u[U_K];
    const double l1 = prm->lambda[0], l2 = prm->lambda[1], l3 = prm->lambda[2],
                 l4 = prm->lambda[3];
    const double lf0 = prm->lambda_f[0], lf1 = prm->lambda_f[1];
    double beta[3], B[3], A[3][3];
    for (int i = 0; i < 3; i++) {
        beta[i] = P.u[U_BETA0 + i];
        B[i] = P.u[U_B0 + i];
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = P.u[U_SYMAT0 + sym(i, j)];
    double g[3][3], ig[3][3], C1[3][3][3], C2[3][3][3], CalGt[3];
    conformal_geometry(P, g, ig, C1, C2, CalGt);
    double R[3][3];
    ricci(P, g, ig, C1, C2, CalGt, R);

    const double* dalpha = P.d1[U_ALPHA];
    const double* dchi = P.d1[U_CHI];
    const double* dK = P.d1[U_K];
    double dbeta[3][3];  // dbeta[i][j] = d_j beta^i
    double divb = 0.0;
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) dbeta[i][j] = P.d1[U_BETA0 + i][j];
        divb += dbeta[i][i];
    }
    auto adv = [&](int v) {
        return beta[0] * P.d1[v][0] + beta[1] * P.d1[v][1] + beta[2] * P.d1[v][2];
    };

    // C3 = C2 - 1/(2chi)(delta_ij d_k chi + delta_ik d_j chi - g_jk ig^im d_m chi)
    // (dendro.py:452-483)
    double igdchi[3];
    for (int i = 0; i < 3; i++)
        igdchi[i] = ig[i][0] * dchi[0] + ig[i][1] * dchi[1] + ig[i][2] * dchi[2];
    double C3[3][3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++)
                C3[i][j][k] = C2[i][j][k] -
                              0.5 / chi * ((i == j ? dchi[k] : 0.0) +
                                           (i == k ? dchi[j] : 0.0) -
                                           g[j][k] * igdchi[i]);
    // DiDj alpha (dendro.py:173-184)
    double DDa[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = P.d2[U_ALPHA][sym(i, j)];
            for (int l = 0; l < 3; l++) s -= C3[l][i][j] * dalpha[l];
            DDa[i][j] = s;
        }
    // A^{ij} (dendro.py:202-209) and A_ik ig^kl A_lj
    double AUU[3][3], AikAkj[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0.0, t = 0.0;
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) {
                    s += ig[i][k] * ig[j][l] * A[k][l];
                    t += A[i][k] * ig[k][l] * A[l][j];
                }
            AUU[i][j] = s;
            AikAkj[i][j] = t;
        }
    double sqrA = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) sqrA += A[i][j] * AUU[i][j];

    // a_rhs = l1 L_beta alpha - 2 alpha K                  (bssn.py:99)
    out[U_ALPHA] = l1 * adv(U_ALPHA) - 2.0 * alpha * K;
    // b_rhs = 3/4 (lf0 + lf1 alpha) B + l2 beta.grad beta   (bssn.py:101-104)
    for (int i = 0; i < 3; i++)
        out[U_BETA0 + i] = 0.75 * (lf0 + lf1 * alpha) * B[i] + l2 * adv(U_BETA0 + i);
    // gt_rhs = L_beta gt (weight -2/3) - 2 alpha At           (bssn.py:106)
    for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++) {
            double s = 0.0;
            for (int k = 0; k < 3; k++)
                s += beta[k] * P.d1[U_SYMGT0 + sym(i, j)][k] + g[i][k] * dbeta[k][j] +
                     g[k][j] * dbeta[k][i] - 2.0 / 3.0 * g[i][j] * dbeta[k][k];
            out[U_SYMGT0 + sym(i, j)] = s - 2.0 * alpha * A[i][j];
        }
    // chi_rhs = L_beta chi (weight -2/3) + 2/3 chi alpha K    (bssn.py:108)
    out[U_CHI] = adv(U_CHI) - 2.0 / 3.0 * chi * divb + 2.0 / 3.0 * chi * alpha * K;
    // At_rhs = L_beta At + chi TF(alpha R - DiDj alpha) + alpha(K At - 2 A.A)
    // (bssn.py:129-133)
    double X[3][3], trX = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) X[i][j] = alpha * R[i][j] - DDa[i][j];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) trX += ig[i][j] * X[i][j];
    for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++) {
            double s = 0.0;
            for (int k = 0; k < 3; k++)
                s += beta[k] * P.d1[U_SYMAT0 + sym(i, j)][k] + A[i][k] * dbeta[k][j] +
                     A[k][j] * dbeta[k][i] - 2.0 / 3.0 * A[i][j] * dbeta[k][k];
            out[U_SYMAT0 + sym(i, j)] = s + chi * (X[i][j] - g[i][j] * trX / 3.0) +
                                        alpha * (K * A[i][j] - 2.0 * AikAkj[i][j]);
        }
    // K_rhs = L_beta K - laplacian(alpha) + alpha (K^2/3 + A_ij A^ij)
    // (bssn.py:135-139); the full inverse metric is chi * ig.
    double lap = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) lap += chi * ig[i][j] * DDa[i][j];
    out[U_K] = adv(U_K) - lap + alpha * (K * K / 3.0 + sqrA);
    // Gt_rhs (bssn.py:143-205)
    double Gt_rhs[3];
    for (int i = 0; i < 3; i++) {
        double s = adv(U_GT0 + i);
        for (int j = 0; j < 3; j++) s -= CalGt[j] * dbeta[i][j];
        s += 2.0 / 3.0 * CalGt[i] * divb;
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++)
                s += ig[j][k] * P.d2[U_BETA0 + i][sym(j, k)] +
                     ig[i][j] * P.d2[U_BETA0 + k][sym(j, k)] / 3.0;
        for (int j = 0; j < 3; j++) s -= 2.0 * AUU[i][j] * dalpha[j];
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) s += 2.0 * alpha * C2[i][j][k] * AUU[j][k];
        for (int j = 0; j < 3; j++)
            s -= alpha * (3.0 / chi * AUU[i][j] * dchi[j] +
                          4.0 / 3.0 * ig[i][j] * dK[j]);
        Gt_rhs[i] = s;
        out[U_GT0 + i] = s;
    }
    // B_rhs = Gt_rhs - eta B + l3 beta.grad B - l4 beta.grad Gt (bssn.py:209-217)
    for (int i = 0; i < 3; i++)
        out[U_B0 + i] = Gt_rhs[i] - eta * B[i] + l3 * adv(U_B0 + i) -
                        l4 * adv(U_GT0 + i);
}

// Sommerfeld falloff and asymptotic value per variable (rhs.cpp:275-327).
const double kFalloff[NVARS] = {1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2};
const double kAsymp[NVARS] = {1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                              1, 0, 0, 1, 0, 1, 0, 0, 0, 0, 0, 0};
// CAKO gauge split (rhs.cpp:356-433): alpha, beta and B.
const bool kGaugeVar[NVARS] = {true,  false, false, false, false, false,
                               true,  true,  true,  true,  true,  true,
                               false, false, false, false, false, false,
                               false, false, false, false, false, false};

constexpr int WS_D1 = 0;                 // 24*3 slabs
constexpr int WS_D2 = NVARS * 3;         // 24*6 slabs (only 11 vars used)
constexpr int WS_KO = NVARS * 3 + NVARS * 6;  // 24*3 slabs
constexpr int WS_SLABS = WS_KO + NVARS * 3;

// All derivatives of one variable in the reference's order: x, xx, y, yy,
// z, zz, then the mixed ones y(x), z(x), z(y) (bssnrhs_derivs.h).
void var_derivs(double* ws, int v, const double* u, const double h[3],
                const unsigned* sz, unsigned bflag, bool second) {
    const size_t n = (size_t)sz[0] * sz[1] * sz[2];
    double* d1 = ws + (size_t)(WS_D1 + 3 * v) * n;
    double* d2 = ws + (size_t)(WS_D2 + 6 * v) * n;
    deriv644(d1 + 0 * n, u, h[0], sz, bflag, 0);
    if (second) deriv644_2(d2 + 0 * n, u, h[0], sz, bflag, 0);
    deriv644(d1 + 1 * n, u, h[1], sz, bflag, 1);
    if (second) deriv644_2(d2 + 3 * n, u, h[1], sz, bflag, 1);
    deriv644(d1 + 2 * n, u, h[2], sz, bflag, 2);
    if (second) deriv644_2(d2 + 5 * n, u, h[2], sz, bflag, 2);
    if (second) {
        deriv644(d2 + 1 * n, d1 + 0 * n, h[1], sz, bflag, 1);  // xy
        deriv644(d2 + 2 * n, d1 + 0 * n, h[2], sz, bflag, 2);  // xz
        deriv644(d2 + 4 * n, d1 + 1 * n, h[2], sz, bflag, 2);  // yz
    }
}

void gather_point(Pt& P, const double** u, unsigned offset, const double* ws,
                  size_t n, size_t pp) {
    for (int v = 0; v < NVARS; v++) {
        P.u[v] = u[v][offset + pp];
        for (int d = 0; d < 3; d++) P.d1[v][d] = ws[(WS_D1 + 3 * v + d) * n + pp];
        if (kNeedsD2[v])
            for (int d = 0; d < 6; d++) P.d2[v][d] = ws[(WS_D2 + 6 * v + d) * n + pp];
        else
            for (int d = 0; d < 6; d++) P.d2[v][d] = 0.0;
    }
}

void bssnrhs_ws(double** rhs, const double** u, unsigned offset,
                const double* pmin, const double* pmax, const unsigned* sz,
                unsigned bflag, const OrcParams* prm, double* ws) {
    const int nx = sz[0], ny = sz[1], nz = sz[2];
    const size_t n = (size_t)nx * ny * nz;
    const double h[3] = {(pmax[0] - pmin[0]) / (nx - 1),
                         (pmax[1] - pmin[1]) / (ny - 1),
                         (pmax[2] - pmin[2]) / (nz - 1)};
    for (int v = 0; v < NVARS; v++)
        var_derivs(ws, v, u[v] + offset, h, sz, bflag, kNeedsD2[v]);
    Pt P;
    double out[NVARS];
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const size_t pp = i + nx * (j + ny * (size_t)k);
                const double x = pmin[0] + i * h[0];
                const double y = pmin[1] + j * h[1];
                const double z = pmin[2] + k * h[2];
                const double r_coord = sqrt(x * x + y * y + z * z);
                const double w = r_coord / prm->eta_width;
                const double arg = -w * w * w * w;
                const double eta =
                    (prm->eta_central - prm->eta_outer) * exp(arg) + prm->eta_outer;
                gather_point(P, u, offset, ws, n, pp);
                rhs_point(P, prm, eta, out);
                for (int v = 0; v < NVARS; v++) rhs[v][offset + pp] = out[v];
            }
    // Sommerfeld BC on boundary faces (rhs.cpp:272-330, 511-631): the value on
    // a face point does not depend on which face is processed last.
    if (bflag) {
        for (int k = 3; k < nz - 3; k++)
            for (int j = 3; j < ny - 3; j++)
                for (int i = 3; i < nx - 3; i++) {
                    const bool on_face =
                        ((bflag & 1u) && i == 3) || ((bflag & 2u) && i == nx - 4) ||
                        ((bflag & 4u) && j == 3) || ((bflag & 8u) && j == ny - 4) ||
                        ((bflag & 16u) && k == 3) || ((bflag & 32u) && k == nz - 4);
                    if (!on_face) continue;
                    const size_t pp = i + nx * (j + ny * (size_t)k);
                    const double x = pmin[0] + i * h[0];
                    const double y = pmin[1] + j * h[1];
                    const double z = pmin[2] + k * h[2];
                    const double inv_r = 1.0 / sqrt(x * x + y * y + z * z);
                    for (int v = 0; v < NVARS; v++) {
                        const double* d1 = ws + (size_t)(WS_D1 + 3 * v) * n;
                        rhs[v][offset + pp] =
                            -inv_r * (x * d1[pp] + y * d1[n + pp] + z * d1[2 * n + pp] +
                                      kFalloff[v] * (u[v][offset + pp] - kAsymp[v]));
                    }
                }
    }
    // KO dissipation (bssnrhs_ko_derivs.h, rhs.cpp:338-492)
    for (int v = 0; v < NVARS; v++) {
        double* ko = ws + (size_t)(WS_KO + 3 * v) * n;
        for (int d = 0; d < 3; d++) ko_deriv42(ko + d * n, u[v] + offset, h[d], sz, bflag, d);
    }
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const size_t pp = i + nx * (j + ny * (size_t)k);
                for (int v = 0; v < NVARS; v++) {
                    const double* ko = ws + (size_t)(WS_KO + 3 * v) * n;
                    double s = prm->ko_sigma;
                    if (prm->cako_enabled) {
                        const double sc = sqrt(u[U_CHI][offset + pp]);
                        s = kGaugeVar[v] ? sc * prm->eps_cako_gauge
                                         : sc * prm->eps_cako_other;
                    }
                    rhs[v][offset + pp] += s * (ko[pp] + ko[n + pp] + ko[2 * n + pp]);
                }
            }
}

// Constraint enforcement on one node, restated from
// BSSN_GR/include/bssn_constraints.h:15-172 with the same arithmetic order;
// returns 1 if the node violated a check (the reference exits there).
int enforce_node(double** u, int64_t node, double chi_floor) {
    const double one_third = 1.0 / 3.0;
    double gtd[3][3], Atd[3][3];
    int bad = 0;
    gtd[0][0] = u[U_SYMGT0][node]; gtd[0][1] = u[U_SYMGT1][node];
    gtd[0][2] = u[U_SYMGT2][node]; gtd[1][1] = u[U_SYMGT3][node];
    gtd[1][2] = u[U_SYMGT4][node]; gtd[2][2] = u[U_SYMGT5][node];
    gtd[1][0] = gtd[0][1]; gtd[2][0] = gtd[0][2]; gtd[2][1] = gtd[1][2];
    Atd[0][0] = u[U_SYMAT0][node]; Atd[0][1] = u[U_SYMAT1][node];
    Atd[0][2] = u[U_SYMAT2][node]; Atd[1][1] = u[U_SYMAT3][node];
    Atd[1][2] = u[U_SYMAT4][node]; Atd[2][2] = u[U_SYMAT5][node];
    Atd[1][0] = Atd[0][1]; Atd[2][0] = Atd[0][2]; Atd[2][1] = Atd[1][2];
    double det_gtd = gtd[0][0] * (gtd[1][1] * gtd[2][2] - gtd[1][2] * gtd[1][2]) -
                     gtd[0][1] * gtd[0][1] * gtd[2][2] +
                     2.0 * gtd[0][1] * gtd[0][2] * gtd[1][2] -
                     gtd[0][2] * gtd[0][2] * gtd[1][1];
    if (det_gtd < 0.0) {
        bad = 1;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) gtd[a][b] = a == b ? 1.0 : 0.0;
        det_gtd = 1.0;
    }
    const double det_gtd_to_neg_third = 1.0 / pow(det_gtd, one_third);
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) gtd[i][j] *= det_gtd_to_neg_third;
    det_gtd = gtd[0][0] * (gtd[1][1] * gtd[2][2] - gtd[1][2] * gtd[1][2]) -
              gtd[0][1] * gtd[0][1] * gtd[2][2] +
              2.0 * gtd[0][1] * gtd[0][2] * gtd[1][2] -
              gtd[0][2] * gtd[0][2] * gtd[1][1];
    if (fabs(det_gtd - 1.0) > 1.0e-6) bad = 1;
    double gtu[3][3];
    const double idet_gtd = 1.0 / det_gtd;
    gtu[0][0] = idet_gtd * (gtd[1][1] * gtd[2][2] - gtd[1][2] * gtd[1][2]);
    gtu[0][1] = idet_gtd * (-gtd[0][1] * gtd[2][2] + gtd[0][2] * gtd[1][2]);
    gtu[0][2] = idet_gtd * (gtd[0][1] * gtd[1][2] - gtd[0][2] * gtd[1][1]);
    gtu[1][1] = idet_gtd * (gtd[0][0] * gtd[2][2] - gtd[0][2] * gtd[0][2]);
    gtu[1][2] = idet_gtd * (-gtd[0][0] * gtd[1][2] + gtd[0][1] * gtd[0][2]);
    gtu[2][2] = idet_gtd * (gtd[0][0] * gtd[1][1] - gtd[0][1] * gtd[0][1]);
    const double one_third_trace_Atd =
        one_third *
        (Atd[0][0] * gtu[0][0] + Atd[1][1] * gtu[1][1] + Atd[2][2] * gtu[2][2] +
         2.0 * (Atd[0][1] * gtu[0][1] + Atd[0][2] * gtu[0][2] + Atd[1][2] * gtu[1][2]));
    Atd[0][0] -= one_third_trace_Atd * gtd[0][0];
    Atd[0][1] -= one_third_trace_Atd * gtd[0][1];
    Atd[0][2] -= one_third_trace_Atd * gtd[0][2];
    Atd[1][1] -= one_third_trace_Atd * gtd[1][1];
    Atd[1][2] -= one_third_trace_Atd * gtd[1][2];
    Atd[2][2] -= one_third_trace_Atd * gtd[2][2];
    const double tr_A =
        Atd[0][0] * gtu[0][0] + Atd[1][1] * gtu[1][1] + Atd[2][2] * gtu[2][2] +
        2.0 * (Atd[0][1] * gtu[0][1] + Atd[0][2] * gtu[0][2] + Atd[1][2] * gtu[1][2]);
    if (fabs(tr_A) > 1.0e-6) bad = 1;
    u[U_SYMAT0][node] = Atd[0][0]; u[U_SYMAT1][node] = Atd[0][1];
    u[U_SYMAT2][node] = Atd[0][2]; u[U_SYMAT3][node] = Atd[1][1];
    u[U_SYMAT4][node] = Atd[1][2]; u[U_SYMAT5][node] = Atd[2][2];
    u[U_SYMGT0][node] = gtd[0][0]; u[U_SYMGT1][node] = gtd[0][1];
    u[U_SYMGT2][node] = gtd[0][2]; u[U_SYMGT3][node] = gtd[1][1];
    u[U_SYMGT4][node] = gtd[1][2]; u[U_SYMGT5][node] = gtd[2][2];
    if (u[U_CHI][node] < chi_floor) u[U_CHI][node] = chi_floor;
    u[U_ALPHA][node] = std::max(u[U_ALPHA][node], chi_floor);
    return bad;
}

uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

void orc_deriv644_x(double* D, const double* u, double h, const unsigned* sz, unsigned b) { deriv644(D, u, h, sz, b, 0); }
void orc_deriv644_y(double* D, const double* u, double h, const unsigned* sz, unsigned b) { deriv644(D, u, h, sz, b, 1); }
void orc_deriv644_z(double* D, const double* u, double h, const unsigned* sz, unsigned b) { deriv644(D, u, h, sz, b, 2); }
void orc_deriv644_xx(double* D, const double* u, double h, const unsigned* sz, unsigned b) { deriv644_2(D, u, h, sz, b, 0); }
void orc_deriv644_yy(double* D, const double* u, double h, const unsigned* sz, unsigned b) { deriv644_2(D, u, h, sz, b, 1); }
void orc_deriv644_zz(double* D, const double* u, double h, const unsigned* sz, unsigned b) { deriv644_2(D, u, h, sz, b, 2); }
void orc_ko_deriv42_x(double* D, const double* u, double h, const unsigned* sz, unsigned b) { ko_deriv42(D, u, h, sz, b, 0); }
void orc_ko_deriv42_y(double* D, const double* u, double h, const unsigned* sz, unsigned b) { ko_deriv42(D, u, h, sz, b, 1); }
void orc_ko_deriv42_z(double* D, const double* u, double h, const unsigned* sz, unsigned b) { ko_deriv42(D, u, h, sz, b, 2); }

void orc_bssnrhs(double** rhs, const double** u, unsigned offset,
                 const double* pmin, const double* pmax, const unsigned* sz,
                 unsigned bflag, const OrcParams* prm, double* ws) {
    std::vector<double> own;
    if (!ws) {
        own.resize((size_t)WS_SLABS * sz[0] * sz[1] * sz[2]);
        ws = own.data();
    }
    bssnrhs_ws(rhs, u, offset, pmin, pmax, sz, bflag, prm, ws);
}

void orc_bssnRHS(double** rhs, const double** u, const OrcBlock* blks,
                 int nblk, const OrcParams* prm, int nthreads) {
    int maxs = 0;
    for (int b = 0; b < nblk; b++) maxs = std::max(maxs, (int)blks[b].sz);
    const size_t wsz = (size_t)WS_SLABS * maxs * maxs * maxs;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> ws(wsz);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nblk; b++) {
            const unsigned sz[3] = {(unsigned)blks[b].sz, (unsigned)blks[b].sz,
                                    (unsigned)blks[b].sz};
            bssnrhs_ws(rhs, u, (unsigned)blks[b].offset, blks[b].ptmin,
                       blks[b].ptmax, sz, blks[b].bflag, prm, ws.data());
        }
    }
}

int64_t orc_enforce(double** u, int64_t n, double chi_floor) {
    int64_t bad = 0;
#pragma omp parallel for reduction(+ : bad)
    for (int64_t node = 0; node < n; node++) bad += enforce_node(u, node, chi_floor);
    return bad;
}

void orc_initial_data(double** u, const int32_t* G, const double* xmin,
                      double h, const double* bh, double m1, double m2,
                      double chi_floor, double eps, uint64_t seed) {
    const int64_t N = (int64_t)G[0] * G[1] * G[2];
#pragma omp parallel for
    for (int64_t node = 0; node < N; node++) {
        const int64_t gx = node % G[0];
        const int64_t gy = (node / G[0]) % G[1];
        const int64_t gz = node / ((int64_t)G[0] * G[1]);
        const double x = xmin[0] + gx * h, y = xmin[1] + gy * h, z = xmin[2] + gz * h;
        // Brill-Lindquist conformal factor (grUtils.cpp:1033-1035,1082-1100)
        const double x1 = x - bh[0], y1 = y - bh[1], z1 = z - bh[2];
        const double x2 = x - bh[3], y2 = y - bh[4], z2 = z - bh[5];
        const double rv1 = sqrt(x1 * x1 + y1 * y1 + z1 * z1);
        const double rv2 = sqrt(x2 * x2 + y2 * y2 + z2 * z2);
        double psi = 1.0 + m1 / (2.0 * rv1);
        psi = psi + m2 / (2.0 * rv2);
        double v[NVARS] = {0};
        v[U_ALPHA] = std::max(1.0 / (psi * psi), chi_floor);
        v[U_CHI] = 1.0 / pow(psi, 4);
        if (v[U_CHI] < chi_floor) v[U_CHI] = chi_floor;
        v[U_SYMGT0] = v[U_SYMGT3] = v[U_SYMGT5] = 1.0;
        for (int k = 0; k < NVARS; k++) {
            const uint64_t r = mix64(seed + 0x9E3779B97F4A7C15ULL *
                                                (uint64_t)(k * N + node + 1));
            const double unit = (double)(r >> 11) * (1.0 / 9007199254740992.0);
            u[k][node] = v[k] + eps * (2.0 * unit - 1.0);
        }
    }
    orc_enforce(u, N, chi_floor);
}

static inline bool in_grid(const int64_t g[3], const int32_t* G) {
    return g[0] >= 0 && g[1] >= 0 && g[2] >= 0 && g[0] < G[0] && g[1] < G[1] &&
           g[2] < G[2];
}

void orc_unzip_map(int64_t* map, const OrcBlock* blks, int nblk,
                   const int32_t* G) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblk; b++) {
        const int s = blks[b].sz;
        for (int k = 0; k < s; k++)
            for (int j = 0; j < s; j++)
                for (int i = 0; i < s; i++) {
                    const int64_t g[3] = {blks[b].g0[0] + i - 3, blks[b].g0[1] + j - 3,
                                          blks[b].g0[2] + k - 3};
                    const int64_t p = blks[b].offset + i + (int64_t)s * (j + (int64_t)s * k);
                    map[p] = in_grid(g, G) ? g[0] + (int64_t)G[0] * (g[1] + (int64_t)G[1] * g[2]) : -1;
                }
    }
}

void orc_unzip(double** unzip, const double** zip, const OrcBlock* blks,
               int nblk, const int32_t* G, int nvars) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblk; b++) {
        const int s = blks[b].sz;
        for (int k = 0; k < s; k++)
            for (int j = 0; j < s; j++)
                for (int i = 0; i < s; i++) {
                    const int64_t g[3] = {blks[b].g0[0] + i - 3, blks[b].g0[1] + j - 3,
                                          blks[b].g0[2] + k - 3};
                    const int64_t p = blks[b].offset + i + (int64_t)s * (j + (int64_t)s * k);
                    const bool in = in_grid(g, G);
                    const int64_t node = in ? g[0] + (int64_t)G[0] * (g[1] + (int64_t)G[1] * g[2]) : 0;
                    for (int v = 0; v < nvars; v++) unzip[v][p] = in ? zip[v][node] : 0.0;
                }
    }
}

void orc_zip(double** zip, const double** unzip, const OrcBlock* blks,
             int nblk, const int32_t* G, int nvars) {
    const int M[3] = {(G[0] - 1) / 6, (G[1] - 1) / 6, (G[2] - 1) / 6};
    std::vector<int> owner((size_t)M[0] * M[1] * M[2], -1);
    for (int b = 0; b < nblk; b++) {
        const int w = (blks[b].sz - 7) / 6;  // octants per side
        const int o0[3] = {blks[b].g0[0] / 6, blks[b].g0[1] / 6, blks[b].g0[2] / 6};
        for (int c = 0; c < w; c++)
            for (int bb = 0; bb < w; bb++)
                for (int a = 0; a < w; a++)
                    owner[(o0[0] + a) + (size_t)M[0] * ((o0[1] + bb) + (size_t)M[1] * (o0[2] + c))] = b;
    }
    const int64_t N = (int64_t)G[0] * G[1] * G[2];
#pragma omp parallel for
    for (int64_t node = 0; node < N; node++) {
        const int64_t g[3] = {node % G[0], (node / G[0]) % G[1], node / ((int64_t)G[0] * G[1])};
        int64_t o[3];
        for (int d = 0; d < 3; d++) o[d] = std::min<int64_t>(g[d] / 6, M[d] - 1);
        const int b = owner[o[0] + (size_t)M[0] * (o[1] + (size_t)M[1] * o[2])];
        if (b < 0) continue;  // octant without a block (the box of one rank of a partition)
        const int s = blks[b].sz;
        const int64_t i = g[0] - blks[b].g0[0] + 3, j = g[1] - blks[b].g0[1] + 3,
                      k = g[2] - blks[b].g0[2] + 3;
        const int64_t p = blks[b].offset + i + s * (j + s * k);
        for (int v = 0; v < nvars; v++) zip[v][node] = unzip[v][p];
    }
}

int64_t orc_rk4_step_ws(double** u, const OrcBlock* blks, int nblk, const int32_t* G,
                        int64_t n_unzip, double dt, const OrcParams* prm, double chi_floor,
                        int enforce_stages, int nthreads, orc_rhs_fn rhs, double* ws) {
    static const double RK4_C[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    static const double RK4_U[4] = {0.0, 1.0 / 2.0, 1.0 / 2.0, 1.0};
    const int64_t N = (int64_t)G[0] * G[1] * G[2];
    if (!rhs) rhs = orc_bssnRHS;
    double* prev = ws;
    double* im = prev + NVARS * N;
    double* kst = im + NVARS * N;
    double* uz = kst + 4 * NVARS * N;
    double* rz = uz + NVARS * n_unzip;
    double *pu[NVARS], *pim[NVARS], *puz[NVARS], *prz[NVARS];
#pragma omp parallel for
    for (int v = 0; v < NVARS; v++) std::memcpy(&prev[v * N], u[v], N * sizeof(double));
    for (int v = 0; v < NVARS; v++) {
        pu[v] = u[v];
        pim[v] = &im[v * N];
        puz[v] = &uz[v * n_unzip];
        prz[v] = &rz[v * n_unzip];
    }
    int64_t bad = 0;
    for (int stage = 0; stage < 4; stage++) {
        double** cur = stage == 0 ? pu : pim;
        orc_unzip(puz, (const double**)cur, blks, nblk, G, NVARS);
        rhs(prz, (const double**)puz, blks, nblk, prm, nthreads);
        double* ks[NVARS];
        for (int v = 0; v < NVARS; v++) ks[v] = &kst[(stage * NVARS + v) * N];
        orc_zip(ks, (const double**)prz, blks, nblk, G, NVARS);
        if (stage < 3) {
#pragma omp parallel for reduction(+ : bad)
            for (int64_t node = 0; node < N; node++) {
                for (int v = 0; v < NVARS; v++) {
                    pim[v][node] = prev[v * N + node];
                    pim[v][node] += (RK4_U[stage + 1] * dt * ks[v][node]);
                }
                if (enforce_stages) bad += enforce_node(pim, node, chi_floor);
            }
        }
    }
#pragma omp parallel for reduction(+ : bad)
    for (int64_t node = 0; node < N; node++) {
        for (int v = 0; v < NVARS; v++) {
            pu[v][node] = prev[v * N + node];
            for (int s = 0; s < 4; s++)
                pu[v][node] += (RK4_C[s] * dt * kst[(s * NVARS + v) * N + node]);
        }
        bad += enforce_node(pu, node, chi_floor);
    }
    return bad;
}

int64_t orc_rk4_ws_doubles(const int32_t* G, int64_t n_unzip) {
    const int64_t N = (int64_t)G[0] * G[1] * G[2];
    return NVARS * (6 * N + 2 * n_unzip);
}

int64_t orc_rk4_step(double** u, const OrcBlock* blks, int nblk,
                     const int32_t* G, int64_t n_unzip, double dt,
                     const OrcParams* prm, double chi_floor,
                     int enforce_stages, int nthreads) {
    std::vector<double> ws((size_t)orc_rk4_ws_doubles(G, n_unzip), 0.0);
    return orc_rk4_step_ws(u, blks, nblk, G, n_unzip, dt, prm, chi_floor, enforce_stages,
                           nthreads, orc_bssnRHS, ws.data());
}

// The same RK4 step in about a third of the memory: the ghost fill and the
// right-hand side run block by block in per-thread buffers (the padded block
// is filled from the stage state exactly as orc_unzip fills it, the
// right-hand side of the one block runs through `rhs` with a one-block list
// at offset 0, and each node the block owns by orc_zip's rule takes its
// value), so no unzipped arrays exist.  Caller arrays: acc, k, im (24 x N
// each).  The arithmetic is orc_rk4_step's, in the same order: the final
// state prev + C0 dt k0 + C1 dt k1 + ... is accumulated stage by stage into
// acc, and each stage state is prev + U dt k; u holds prev until the end.
int64_t orc_rk4_step_lowmem(double** u, const OrcBlock* blks, int nblk, const int32_t* G,
                            double dt, const OrcParams* prm, double chi_floor, int enforce_stages,
                            int nthreads, orc_rhs_fn rhs, double** acc, double** kbuf, double** im) {
    static const double RK4_C[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    static const double RK4_U[4] = {0.0, 1.0 / 2.0, 1.0 / 2.0, 1.0};
    if (!rhs) rhs = orc_bssnRHS;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const int64_t N = (int64_t)G[0] * G[1] * G[2];
    const int M[3] = {(G[0] - 1) / 6, (G[1] - 1) / 6, (G[2] - 1) / 6};
    std::vector<int> owner((size_t)M[0] * M[1] * M[2], -1);
    int smax = 0;
    for (int b = 0; b < nblk; b++) {
        smax = std::max(smax, (int)blks[b].sz);
        const int w = (blks[b].sz - 7) / 6;
        const int o0[3] = {blks[b].g0[0] / 6, blks[b].g0[1] / 6, blks[b].g0[2] / 6};
        for (int c = 0; c < w; c++)
            for (int bb = 0; bb < w; bb++)
                for (int a = 0; a < w; a++)
                    owner[(o0[0] + a) + (size_t)M[0] * ((o0[1] + bb) + (size_t)M[1] * (o0[2] + c))] = b;
    }
#pragma omp parallel for num_threads(nthreads)
    for (int64_t node = 0; node < N; node++)
        for (int v = 0; v < NVARS; v++) acc[v][node] = u[v][node];
    int64_t bad = 0;
    const size_t cap = (size_t)smax * smax * smax;
    for (int stage = 0; stage < 4; stage++) {
        double** cur = stage == 0 ? u : im;
#pragma omp parallel num_threads(nthreads)
        {
            std::vector<double> P(NVARS * cap), R(NVARS * cap, 0.0);
            double *pp[NVARS], *rr[NVARS];
            for (int v = 0; v < NVARS; v++) {
                pp[v] = &P[v * cap];
                rr[v] = &R[v * cap];
            }
#pragma omp for schedule(dynamic, 1)
            for (int b = 0; b < nblk; b++) {
                OrcBlock one = blks[b];
                one.offset = 0;
                orc_unzip(pp, (const double**)cur, &one, 1, G, NVARS);
                rhs(rr, (const double**)pp, &one, 1, prm, 1);
                const int s = one.sz, n = s - 6;
                for (int k = 0; k < n; k++)
                    for (int j = 0; j < n; j++)
                        for (int i = 0; i < n; i++) {
                            const int64_t g[3] = {one.g0[0] + i, one.g0[1] + j, one.g0[2] + k};
                            int64_t o[3];
                            for (int d = 0; d < 3; d++) o[d] = std::min<int64_t>(g[d] / 6, M[d] - 1);
                            if (owner[o[0] + (size_t)M[0] * (o[1] + (size_t)M[1] * o[2])] != b) continue;
                            const int64_t node = g[0] + (int64_t)G[0] * (g[1] + (int64_t)G[1] * g[2]);
                            const int64_t p = (i + 3) + (int64_t)s * ((j + 3) + (int64_t)s * (k + 3));
                            for (int v = 0; v < NVARS; v++) kbuf[v][node] = rr[v][p];
                        }
            }
        }
#pragma omp parallel for num_threads(nthreads) reduction(+ : bad)
        for (int64_t node = 0; node < N; node++) {
            for (int v = 0; v < NVARS; v++) acc[v][node] += (RK4_C[stage] * dt * kbuf[v][node]);
            if (stage < 3) {
                for (int v = 0; v < NVARS; v++) {
                    im[v][node] = u[v][node];
                    im[v][node] += (RK4_U[stage + 1] * dt * kbuf[v][node]);
                }
                if (enforce_stages) bad += enforce_node(im, node, chi_floor);
            }
        }
    }
#pragma omp parallel for num_threads(nthreads) reduction(+ : bad)
    for (int64_t node = 0; node < N; node++) {
        for (int v = 0; v < NVARS; v++) u[v][node] = acc[v][node];
        bad += enforce_node(u, node, chi_floor);
    }
    return bad;
}

// Sums of squares of ham, mom0..2 and the node count over the nodes outside
// both radii (grUtils.tcc:36-134's L2 norm before the square root), block by
// block without unzipped arrays: each block is ghost-filled into a
// per-thread buffer, its constraints computed (orc_physical_constraints) and
// the nodes it owns by orc_zip's rule accumulated.  sums[0..3], sums[4] =
// count; norm_c = sqrt(sums[c] / sums[4]).  Node coordinates xmin[d] + g h.
void orc_constraint_sums_lowmem(const double** u, const OrcBlock* blks, int nblk, const int32_t* G,
                                const double* xmin, double h, const double* bh,
                                const double* radii, double* sums, int nthreads) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const int M[3] = {(G[0] - 1) / 6, (G[1] - 1) / 6, (G[2] - 1) / 6};
    std::vector<int> owner((size_t)M[0] * M[1] * M[2], -1);
    int smax = 0;
    for (int b = 0; b < nblk; b++) {
        smax = std::max(smax, (int)blks[b].sz);
        const int w = (blks[b].sz - 7) / 6;
        const int o0[3] = {blks[b].g0[0] / 6, blks[b].g0[1] / 6, blks[b].g0[2] / 6};
        for (int c = 0; c < w; c++)
            for (int bb = 0; bb < w; bb++)
                for (int a = 0; a < w; a++)
                    owner[(o0[0] + a) + (size_t)M[0] * ((o0[1] + bb) + (size_t)M[1] * (o0[2] + c))] = b;
    }
    const size_t cap = (size_t)smax * smax * smax;
    std::vector<double> part((size_t)nblk * 5, 0.0);
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> P(NVARS * cap), Cn(4 * cap, 0.0), ws((size_t)WS_SLABS * cap);
        double *pp[NVARS], *cc[NVARS];
        for (int v = 0; v < NVARS; v++) pp[v] = &P[v * cap];
        for (int c = 0; c < NVARS; c++) cc[c] = c < 4 ? &Cn[c * cap] : nullptr;
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nblk; b++) {
            OrcBlock one = blks[b];
            one.offset = 0;
            orc_unzip(pp, u, &one, 1, G, NVARS);
            const unsigned sz[3] = {(unsigned)one.sz, (unsigned)one.sz, (unsigned)one.sz};
            orc_physical_constraints(cc, (const double**)pp, 0, one.ptmin, one.ptmax, sz, one.bflag, ws.data());
            const int s = one.sz, n = s - 6;
            double acc[5] = {0, 0, 0, 0, 0};
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n; i++) {
                        const int64_t g[3] = {one.g0[0] + i, one.g0[1] + j, one.g0[2] + k};
                        int64_t o[3];
                        for (int d = 0; d < 3; d++) o[d] = std::min<int64_t>(g[d] / 6, M[d] - 1);
                        if (owner[o[0] + (size_t)M[0] * (o[1] + (size_t)M[1] * o[2])] != b) continue;
                        const double x = xmin[0] + g[0] * h, y = xmin[1] + g[1] * h, z = xmin[2] + g[2] * h;
                        const double d1 = std::sqrt((x - bh[0]) * (x - bh[0]) + (y - bh[1]) * (y - bh[1]) +
                                                    (z - bh[2]) * (z - bh[2]));
                        const double d2 = std::sqrt((x - bh[3]) * (x - bh[3]) + (y - bh[4]) * (y - bh[4]) +
                                                    (z - bh[5]) * (z - bh[5]));
                        if (d1 < radii[0] || d2 < radii[1]) continue;
                        const int64_t p = (i + 3) + (int64_t)s * ((j + 3) + (int64_t)s * (k + 3));
                        for (int c = 0; c < 4; c++) acc[c] += Cn[c * cap + p] * Cn[c * cap + p];
                        acc[4] += 1.0;
                    }
            for (int c = 0; c < 5; c++) part[(size_t)b * 5 + c] = acc[c];
        }
    }
    for (int c = 0; c < 5; c++) sums[c] = 0.0;
    for (int b = 0; b < nblk; b++)
        for (int c = 0; c < 5; c++) sums[c] += part[(size_t)b * 5 + c];
}

// ---------------------------------------------------------------------------
// Synthetic single-level octree meshes (the workloads' block lists), restated
// from the definition the product library's generator documents: mode 0 = a
// uniform dims[0]^3 grid of single-octant blocks (13^3); mode 1 = dims
// super-cells of 8^3 octants, visited in a seeded order, each split top-down
// (children in Morton order) where a uniform draw is not below the
// probability of staying whole, which follows from the target block-count
// fractions p = {p13, p19, p31, p55}.  Block b of w octants per side has
// padded side 6w + 7, its first interior node at 6 * octant origin, and its
// padded array at the running offset, each array rounded up to an even
// number of doubles.
// ---------------------------------------------------------------------------
namespace {
struct MeshRng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);  // splitmix64
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};
struct Oct {
    int o[3];
    int w;
};
void split_oct(const Oct& c, const double stay[4], MeshRng& r, std::vector<Oct>& out) {
    const int lvl = c.w == 8 ? 3 : (c.w == 4 ? 2 : (c.w == 2 ? 1 : 0));
    if (c.w == 1 || r.uniform() < stay[lvl]) {
        out.push_back(c);
        return;
    }
    const int h = c.w / 2;
    for (int m = 0; m < 8; m++)
        split_oct(Oct{{c.o[0] + (m & 1) * h, c.o[1] + ((m >> 1) & 1) * h, c.o[2] + ((m >> 2) & 1) * h}, h},
                  stay, r, out);
}
}  // namespace

int orc_mesh_generate(int mode, const int32_t* dims, const double* p, uint64_t seed, double xmin,
                      double L, OrcBlock* blks, int* nblk, int32_t* G, double* h_out) {
    std::vector<Oct> cubes;
    int M[3];
    if (mode == 0) {
        const int n = dims[0];
        if (n < 1) return 1;
        M[0] = M[1] = M[2] = n;
        for (int z = 0; z < n; z++)
            for (int y = 0; y < n; y++)
                for (int x = 0; x < n; x++) cubes.push_back(Oct{{x, y, z}, 1});
    } else if (mode == 1) {
        for (int d = 0; d < 3; d++) {
            if (dims[d] < 1) return 1;
            M[d] = 8 * dims[d];
        }
        if (p[0] <= 0 || p[1] <= 0 || p[2] <= 0 || p[3] <= 0) return 1;
        // expected blocks per super-cell: a, 8(1-a)b, 64(1-a)(1-b)c,
        // 512(1-a)(1-b)(1-c) for sides 55, 31, 19, 13 (a, b, c = probability
        // of staying whole at widths 8, 4, 2), solved for the fractions p
        const double c = 8.0 / (8.0 + p[0] / p[1]);
        const double b = 8.0 * c / (8.0 * c + p[1] / p[2]);
        const double a = 8.0 * b / (8.0 * b + p[2] / p[3]);
        const double stay[4] = {1.0, c, b, a};
        MeshRng r{seed};
        const int ns = dims[0] * dims[1] * dims[2];
        std::vector<int> order(ns);
        for (int i = 0; i < ns; i++) order[i] = i;
        for (int i = ns - 1; i > 0; i--) std::swap(order[i], order[(int)(r.next() % (uint64_t)(i + 1))]);
        for (int t = 0; t < ns; t++) {
            const int id = order[t];
            const int sx = id % dims[0], sy = (id / dims[0]) % dims[1], sz = id / (dims[0] * dims[1]);
            split_oct(Oct{{8 * sx, 8 * sy, 8 * sz}, 8}, stay, r, cubes);
        }
    } else {
        return 1;
    }
    for (int d = 0; d < 3; d++) G[d] = 6 * M[d] + 1;
    const int Mmax = std::max(M[0], std::max(M[1], M[2]));
    const double h = L / Mmax / 6.0;
    *h_out = h;
    *nblk = (int)cubes.size();
    if (!blks) return 0;
    int64_t off = 0;
    for (size_t b = 0; b < cubes.size(); b++) {
        const Oct& c = cubes[b];
        OrcBlock d;
        std::memset(&d, 0, sizeof(d));
        const int s = 6 * c.w + 7;
        d.offset = off;
        d.sz = s;
        for (int k = 0; k < 3; k++) {
            d.g0[k] = 6 * c.o[k];
            if (c.o[k] == 0) d.bflag |= 1u << (2 * k);
            if (c.o[k] + c.w == M[k]) d.bflag |= 1u << (2 * k + 1);
            d.ptmin[k] = xmin + (double)(d.g0[k] - 3) * h;
            d.ptmax[k] = xmin + (double)(d.g0[k] - 3 + s - 1) * h;
        }
        d.level = c.w == 1 ? 3 : (c.w == 2 ? 2 : (c.w == 4 ? 1 : 0));
        blks[b] = d;
        const int64_t npts = (int64_t)s * s * s;
        off += (npts + 1) / 2 * 2;
    }
    return 0;
}

// Hamiltonian and momentum constraints (CodeGen/constraints.py:250-283):
//   ham   = chi ig^jk R_jk - A_ij A^ij + 2/3 K^2
//   mom_i = ig^jk (d_k A_ij - C2^m_ki A_jm) - Gt^j A_ij
//           - 3/2 ig^jk A_ki d_j chi / chi - 2/3 d_i K
void orc_physical_constraints(double** cons, const double** u, unsigned offset,
                              const double* pmin, const double* pmax,
                              const unsigned* sz, unsigned bflag, double* ws) {
    std::vector<double> own;
    const int nx = sz[0], ny = sz[1], nz = sz[2];
    const size_t n = (size_t)nx * ny * nz;
    if (!ws) {
        own.resize((size_t)WS_SLABS * n);
        ws = own.data();
    }
    const double h[3] = {(pmax[0] - pmin[0]) / (nx - 1),
                         (pmax[1] - pmin[1]) / (ny - 1),
                         (pmax[2] - pmin[2]) / (nz - 1)};
    for (int v = 0; v < NVARS; v++)
        var_derivs(ws, v, u[v] + offset, h, sz, bflag, kNeedsD2[v]);
    Pt P;
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const size_t pp = i + nx * (j + ny * (size_t)k);
                gather_point(P, u, offset, ws, n, pp);
                double g[3][3], ig[3][3], C1[3][3][3], C2[3][3][3], CalGt[3], R[3][3];
                conformal_geometry(P, g, ig, C1, C2, CalGt);
                ricci(P, g, ig, C1, C2, CalGt, R);
                const double chi = P.u[U_CHI], K = P.u[U_K];
                double A[3][3];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) A[a][b] = P.u[U_SYMAT0 + sym(a, b)];
                double ham = 0.0, sqrA = 0.0;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        ham += chi * ig[a][b] * R[a][b];
                        double s = 0.0;
                        for (int c = 0; c < 3; c++)
                            for (int d = 0; d < 3; d++) s += ig[a][c] * ig[b][d] * A[c][d];
                        sqrA += A[a][b] * s;
                    }
                cons[0][offset + pp] = ham - sqrA + 2.0 / 3.0 * K * K;
                for (int a = 0; a < 3; a++) {
                    double m = 0.0;
                    for (int b = 0; b < 3; b++)
                        for (int c = 0; c < 3; c++) {
                            double t = P.d1[U_SYMAT0 + sym(a, b)][c];
                            for (int q = 0; q < 3; q++) t -= C2[q][c][a] * A[b][q];
                            m += ig[b][c] * t;
                        }
                    for (int b = 0; b < 3; b++) m -= P.u[U_GT0 + b] * A[a][b];
                    for (int b = 0; b < 3; b++)
                        for (int c = 0; c < 3; c++)
                            m -= 1.5 * ig[b][c] * A[c][a] * P.d1[U_CHI][b] / chi;
                    m -= 2.0 / 3.0 * P.d1[U_K][a];
                    cons[1 + a][offset + pp] = m;
                }
            }
}

// The Weyl scalar psi4 (CodeGen/constraints.py:45-244; per point as
// BSSN_GR/src/physcon.cpp:72-85, zero on the z axis): the tetrad r, theta,
// phi made orthonormal by Gram-Schmidt in the physical metric gt / chi at
// the point's coordinates x = pmin + i h, then
//   psi4 = -(P1 + P2 - P3 - P4) (real part), P1 + P2 - P3 - P4 (imaginary)
// with P1 = R_ij M^ij, P2 = A_temp At_ij M^ij, P3 = (MR Uu - NR Vv) / chi,
// P4 the (At r) and d chi products (M, N, MR, NR, Uu, Vv as defined there).
void orc_psi4(double* re, double* im, const double** u, unsigned offset, const double* pmin,
              const double* pmax, const unsigned* sz, unsigned bflag, double* ws) {
    std::vector<double> own;
    const int nx = sz[0], ny = sz[1], nz = sz[2];
    const size_t n = (size_t)nx * ny * nz;
    if (!ws) {
        own.resize((size_t)WS_SLABS * n);
        ws = own.data();
    }
    const double h[3] = {(pmax[0] - pmin[0]) / (nx - 1),
                         (pmax[1] - pmin[1]) / (ny - 1),
                         (pmax[2] - pmin[2]) / (nz - 1)};
    for (int v = 0; v < NVARS; v++)
        var_derivs(ws, v, u[v] + offset, h, sz, bflag, kNeedsD2[v]);
    Pt P;
    for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++)
            for (int i = 3; i < nx - 3; i++) {
                const size_t pp = i + nx * (j + ny * (size_t)k);
                const double x = pmin[0] + i * h[0], y = pmin[1] + j * h[1], z = pmin[2] + k * h[2];
                if (std::fabs(x) <= 1e-7 && std::fabs(y) <= 1e-7) {
                    re[offset + pp] = 0.0;
                    im[offset + pp] = 0.0;
                    continue;
                }
                gather_point(P, u, offset, ws, n, pp);
                double g[3][3], ig[3][3], C1[3][3][3], C2[3][3][3], CalGt[3], R[3][3];
                conformal_geometry(P, g, ig, C1, C2, CalGt);
                ricci(P, g, ig, C1, C2, CalGt, R);
                const double chi = P.u[U_CHI], K = P.u[U_K], ichi = 1.0 / chi;
                double gd[3][3], A[3][3];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        gd[a][b] = g[a][b] * ichi;
                        A[a][b] = P.u[U_SYMAT0 + sym(a, b)];
                    }
                auto dot = [&](const double* p, const double* q) {
                    double t = 0.0;
                    for (int b = 0; b < 3; b++)
                        for (int a = 0; a < 3; a++) t += gd[a][b] * p[a] * q[b];
                    return t;
                };
                double rv[3] = {x, y, z}, th[3] = {x * z, y * z, -(x * x + y * y)}, ph[3] = {-y, x, 0.0};
                const double nr = std::sqrt(dot(rv, rv));
                for (int a = 0; a < 3; a++) rv[a] /= nr;
                {
                    const double p1 = dot(th, th), p2 = dot(rv, th);
                    for (int a = 0; a < 3; a++) th[a] -= p2 * rv[a];
                    const double nt = std::sqrt(p1 - p2 * p2);
                    for (int a = 0; a < 3; a++) th[a] /= nt;
                }
                {
                    const double p1 = dot(ph, ph), p2 = dot(rv, ph), p3 = dot(th, ph);
                    for (int a = 0; a < 3; a++) ph[a] -= p2 * rv[a] + p3 * th[a];
                    const double np = std::sqrt(p1 - p2 * p2 - p3 * p3);
                    for (int a = 0; a < 3; a++) ph[a] /= np;
                }
                const double s2 = 1.0 / std::sqrt(2.0);
                double mr[3], mi[3];
                for (int a = 0; a < 3; a++) {
                    mr[a] = th[a] * s2;
                    mi[a] = ph[a] * s2;
                }
                double MM[3][3], NN[3][3], MR[3][3], NR[3][3], Uu[3][3], Vv[3][3];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        MM[a][b] = mr[a] * mr[b] - mi[a] * mi[b];
                        NN[a][b] = mr[a] * mi[b] + mr[b] * mi[a];
                        MR[a][b] = mr[a] * rv[b] - mr[b] * rv[a];
                        NR[a][b] = mi[a] * rv[b] - mi[b] * rv[a];
                        double uu = 0.0, vv = 0.0;
                        for (int c = 0; c < 3; c++) {
                            double t = P.d1[U_SYMAT0 + sym(c, a)][b];
                            for (int m = 0; m < 3; m++) t += C2[m][c][a] * A[m][b];
                            uu += mr[c] * t;
                            vv += mi[c] * t;
                        }
                        Uu[a][b] = uu;
                        Vv[a][b] = vv;
                    }
                double Av[3];
                for (int a = 0; a < 3; a++) Av[a] = A[a][0] * rv[0] + A[a][1] * rv[1] + A[a][2] * rv[2];
                double rdc = 0.0, mrdc = 0.0, midc = 0.0, rA = 0.0, mrA = 0.0, miA = 0.0;
                for (int a = 0; a < 3; a++) {
                    rdc += rv[a] * P.d1[U_CHI][a];
                    mrdc += mr[a] * P.d1[U_CHI][a];
                    midc += mi[a] * P.d1[U_CHI][a];
                    rA += Av[a] * rv[a];
                    mrA += mr[a] * Av[a];
                    miA += mi[a] * Av[a];
                }
                const double Atmp = ichi * ichi * (rA + K * chi / 3.0 + 0.5 * rdc);
                // symmetric contractions: diagonal + 2 x upper triangle
                auto sym_dot = [](const double S[3][3], const double T[3][3]) {
                    double d = S[0][0] * T[0][0] + S[1][1] * T[1][1] + S[2][2] * T[2][2];
                    return d + 2.0 * (S[0][1] * T[0][1] + S[0][2] * T[0][2] + S[1][2] * T[1][2]);
                };
                const double p1r = sym_dot(R, MM), p1i = sym_dot(R, NN);
                const double p2r = Atmp * sym_dot(A, MM), p2i = Atmp * sym_dot(A, NN);
                double s3r = 0.0, s3i = 0.0;
                for (int b = 0; b < 3; b++)
                    for (int a = 0; a < 3; a++) {
                        s3r += MR[a][b] * Uu[a][b] - NR[a][b] * Vv[a][b];
                        s3i += NR[a][b] * Uu[a][b] + MR[a][b] * Vv[a][b];
                    }
                const double p3r = ichi * s3r, p3i = ichi * s3i;
                const double p4r = ichi * ichi * (mrA * (mrA + 0.5 * mrdc) - miA * (miA + 0.5 * midc));
                const double p4i = ichi * ichi * (mrA * (miA + 0.5 * midc) + miA * (mrA + 0.5 * mrdc));
                re[offset + pp] = -(p1r + p2r - p3r - p4r);
                im[offset + pp] = p1i + p2i - p3i - p4i;
            }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Remesh: wavelet refinement scores and block features (see the header).
// ---------------------------------------------------------------------------
namespace {
// degree-5 Lagrange weights at fine patch positions 4, 6, 8 from coarse
// positions 1, 3, 5, 7, 9, 11 (exact dyadic rationals)
const double kWfine[3][6] = {
    {-7.0 / 256, 105.0 / 256, 105.0 / 128, -35.0 / 128, 21.0 / 256, -3.0 / 256},
    {3.0 / 256, -25.0 / 256, 75.0 / 128, 75.0 / 128, -25.0 / 256, 3.0 / 256},
    {-3.0 / 256, 21.0 / 256, -35.0 / 128, 105.0 / 128, 105.0 / 256, -7.0 / 256}};

// interpolation of the patch at local node (a,b,c) in [0,6]^3; p = patch
// origin (value at patch (0,0,0)), strides 1, s, s*s
double wavelet_interp(const double* p, int s, int a, int b, int c) {
    int n[3], pos[3][6];
    double w[3][6];
    const int loc[3] = {a, b, c};
    for (int d = 0; d < 3; d++) {
        if (loc[d] & 1) {
            n[d] = 6;
            for (int t = 0; t < 6; t++) {
                pos[d][t] = 1 + 2 * t;
                w[d][t] = kWfine[(loc[d] - 1) / 2][t];
            }
        } else {
            n[d] = 1;
            pos[d][0] = loc[d] + 3;
            w[d][0] = 1.0;
        }
    }
    double az = 0.0;
    for (int k = 0; k < n[2]; k++) {
        double ay = 0.0;
        for (int j = 0; j < n[1]; j++) {
            double ax = 0.0;
            for (int i = 0; i < n[0]; i++)
                ax += w[0][i] * p[pos[0][i] + (int64_t)s * (pos[1][j] + (int64_t)s * pos[2][k])];
            ay += w[1][j] * ax;
        }
        az += w[2][k] * ay;
    }
    return az;
}
}  // namespace

extern "C" void orc_wavelet_scores(const double** unzip, const OrcBlock* blks, int nblk,
                                   int nvars, double* scores) {
    std::vector<int64_t> first(nblk + 1, 0);
    for (int b = 0; b < nblk; b++) {
        const int w = (blks[b].sz - 7) / 6;
        first[b + 1] = first[b] + (int64_t)w * w * w;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblk; b++) {
        const int s = blks[b].sz, w = (s - 7) / 6;
        for (int e = 0; e < w * w * w; e++) {
            const int ox = e % w, oy = (e / w) % w, oz = e / (w * w);
            for (int v = 0; v < nvars; v++) {
                const double* p = unzip[v] + blks[b].offset + 6 * ox +
                                  (int64_t)s * (6 * oy + (int64_t)s * 6 * oz);
                double part[32] = {0};
                int q = 0;
                for (int c = 0; c < 7; c++)
                    for (int bb = 0; bb < 7; bb++)
                        for (int a = 0; a < 7; a++) {
                            if (!((a | bb | c) & 1)) continue;
                            const double u = p[(a + 3) + (int64_t)s * ((bb + 3) + (int64_t)s * (c + 3))];
                            const double wv = u - wavelet_interp(p, s, a, bb, c);
                            part[q & 31] += wv * wv;
                            q++;
                        }
                double tot = 0.0;
                for (int l = 0; l < 32; l++) tot += part[l];
                scores[(first[b] + e) * nvars + v] = sqrt(tot / 279.0);
            }
        }
    }
}

// Per-element features: the block features' definitions over each element's
// even local nodes (4 x 4 x 4 points), elements block by block, octant x
// fastest (the library's element order).
extern "C" void orc_element_features(const double** unzip, const OrcBlock* blks, int nblk,
                                     float* feats) {
    int64_t e0 = 0;
    for (int b = 0; b < nblk; b++) {
        const int s = blks[b].sz, w = (s - 7) / 6;
        const int64_t st[3] = {2, 2 * s, 2 * (int64_t)s * s};
        const double* chi = unzip[U_CHI];
        const double* al = unzip[U_ALPHA];
        const double h = (blks[b].ptmax[0] - blks[b].ptmin[0]) / (s - 1);
        for (int oz = 0; oz < w; oz++)
            for (int oy = 0; oy < w; oy++)
                for (int ox = 0; ox < w; ox++, e0++) {
                    double mx[16];
                    for (int f = 0; f < 16; f++) mx[f] = 0.0;
                    double chimin = 1e300;
                    for (int mz = 0; mz < 4; mz++)
                        for (int my = 0; my < 4; my++)
                            for (int mxi = 0; mxi < 4; mxi++) {
                                const int i = 3 + 6 * ox + 2 * mxi, j = 3 + 6 * oy + 2 * my, k = 3 + 6 * oz + 2 * mz;
                                const int64_t p = blks[b].offset + i + s * (j + (int64_t)s * k);
                                const double c0 = chi[p], a0 = al[p];
                                for (int d = 0; d < 3; d++) {
                                    const double cp = chi[p + st[d]], cm = chi[p - st[d]];
                                    const double ap = al[p + st[d]], am = al[p - st[d]];
                                    mx[d] = std::max(mx[d], fabs((cp - cm) * 0.25));
                                    mx[3 + d] = std::max(mx[3 + d], fabs((ap - am) * 0.25));
                                    mx[7 + d] = std::max(mx[7 + d], fabs(unzip[U_GT0 + d][p]));
                                    mx[13] = std::max(mx[13], fabs((cp - c0) - (c0 - cm)));
                                    mx[14] = std::max(mx[14], fabs((ap - a0) - (a0 - am)));
                                }
                                mx[6] = std::max(mx[6], fabs(unzip[U_K][p]));
                                chimin = std::min(chimin, c0);
                            }
                    float* f = feats + e0 * 16;
                    for (int q = 0; q < 10; q++) f[q] = (float)log10(mx[q] + 1e-30);
                    f[10] = (float)blks[b].level;
                    f[11] = (float)(s / 55.0);
                    f[12] = (float)log10(chimin);
                    f[13] = (float)log10(mx[13] + 1e-30);
                    f[14] = (float)log10(mx[14] + 1e-30);
                    f[15] = (float)log10(h);
                }
    }
}

extern "C" void orc_block_features(const double** unzip, const OrcBlock* blks, int nblk,
                                   float* feats) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblk; b++) {
        // even sublattice of the interior, differences over two points
        const int s = blks[b].sz;
        const int64_t st[3] = {2, 2 * s, 2 * (int64_t)s * s};
        const double* chi = unzip[U_CHI];
        const double* al = unzip[U_ALPHA];
        double mx[16];
        for (int f = 0; f < 16; f++) mx[f] = 0.0;
        double chimin = 1e300;
        for (int k = 3; k < s - 3; k += 2)
            for (int j = 3; j < s - 3; j += 2)
                for (int i = 3; i < s - 3; i += 2) {
                    const int64_t p = blks[b].offset + i + s * (j + (int64_t)s * k);
                    const double c0 = chi[p], a0 = al[p];
                    for (int d = 0; d < 3; d++) {
                        const double cp = chi[p + st[d]], cm = chi[p - st[d]];
                        const double ap = al[p + st[d]], am = al[p - st[d]];
                        mx[d] = std::max(mx[d], fabs((cp - cm) * 0.25));
                        mx[3 + d] = std::max(mx[3 + d], fabs((ap - am) * 0.25));
                        mx[7 + d] = std::max(mx[7 + d], fabs(unzip[U_GT0 + d][p]));
                        mx[13] = std::max(mx[13], fabs((cp - c0) - (c0 - cm)));
                        mx[14] = std::max(mx[14], fabs((ap - a0) - (a0 - am)));
                    }
                    mx[6] = std::max(mx[6], fabs(unzip[U_K][p]));
                    chimin = std::min(chimin, c0);
                }
        const double h = (blks[b].ptmax[0] - blks[b].ptmin[0]) / (s - 1);
        float* f = feats + (int64_t)b * 16;
        for (int q = 0; q < 10; q++) f[q] = (float)log10(mx[q] + 1e-30);
        f[10] = (float)blks[b].level;
        f[11] = (float)(s / 55.0);
        f[12] = (float)log10(chimin);
        f[13] = (float)log10(mx[13] + 1e-30);
        f[14] = (float)log10(mx[14] + 1e-30);
        f[15] = (float)log10(h);
    }
}
