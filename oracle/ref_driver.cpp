// Test infrastructure only: never linked into the product library.
//
// Driver for the reference's OWN CPU arithmetic of the BSSN right-hand side.
// The stencils (BSSN_GR/src/derivs.cpp), the derivative call lists
// (BSSN_GR/scripts/bssnrhs_{evar_derivs,derivs,ko_derivs}.h,
// constraint_derivs.h) and the generated pointwise equations
// (BSSN_GR/src/bssneqs_eta_const_standard_gauge.cpp, physconeqs.cpp) are
// compiled from where they lie in the reference tree by oracle/Makefile into
// oracle/_ref/libbssn_ref.so.  Nothing from the reference is copied here: this
// file only supplies the surrounding control flow that lives in files which
// cannot be compiled without dendrolib (rhs.cpp, physcon.cpp), restated:
//
//   ref_bssnrhs             follows BSSN_GR/src/rhs.cpp:80-504
//                           (derivatives -> equations -> Sommerfeld BC ->
//                            KO derivatives -> KO add)
//   bcs (static)            follows BSSN_GR/src/rhs.cpp:511-631
//   ref_physical_constraints follows BSSN_GR/src/physcon.cpp:12-89
//
// Parameters that the reference reads from `bssn::` globals are passed in
// RefParams.  Build flags: -DBSSN_USE_6TH_ORDER_DERIVS -O2 -ffp-contract=off.
#include <cmath>
#include <cstdint>
#include <omp.h>
#include <vector>

#include "derivs.h"

namespace {

enum {
    U_ALPHA = 0, U_CHI, U_K, U_GT0, U_GT1, U_GT2, U_BETA0, U_BETA1, U_BETA2,
    U_B0, U_B1, U_B2, U_SYMGT0, U_SYMGT1, U_SYMGT2, U_SYMGT3, U_SYMGT4,
    U_SYMGT5, U_SYMAT0, U_SYMAT1, U_SYMAT2, U_SYMAT3, U_SYMAT4, U_SYMAT5
};

// Sommerfeld outgoing-radiation condition on the boundary faces of a block,
// restated from BSSN_GR/src/rhs.cpp:511-631 (same face order, same formula).
void bcs(double* f_rhs, const double* f, const double* dxf, const double* dyf,
         const double* dzf, const double* pmin, const double* pmax,
         double f_falloff, double f_asymptotic, const unsigned* sz,
         unsigned bflag) {
    const unsigned nx = sz[0], ny = sz[1], nz = sz[2];
    const double hx = (pmax[0] - pmin[0]) / (nx - 1);
    const double hy = (pmax[1] - pmin[1]) / (ny - 1);
    const double hz = (pmax[2] - pmin[2]) / (nz - 1);
    const unsigned PW = 3;
    const unsigned ib = PW, jb = PW, kb = PW;
    const unsigned ie = nx - PW, je = ny - PW, ke = nz - PW;
    auto apply = [&](unsigned i, unsigned j, unsigned k, double x, double y,
                     double z) {
        const unsigned pp = IDX(i, j, k);
        const double inv_r = 1.0 / sqrt(x * x + y * y + z * z);
        f_rhs[pp] = -inv_r * (x * dxf[pp] + y * dyf[pp] + z * dzf[pp] +
                              f_falloff * (f[pp] - f_asymptotic));
    };
    if (bflag & (1u << OCT_DIR_LEFT)) {
        const double x = pmin[0] + ib * hx;
        for (unsigned k = kb; k < ke; k++)
            for (unsigned j = jb; j < je; j++)
                apply(ib, j, k, x, pmin[1] + j * hy, pmin[2] + k * hz);
    }
    if (bflag & (1u << OCT_DIR_RIGHT)) {
        const double x = pmin[0] + (ie - 1) * hx;
        for (unsigned k = kb; k < ke; k++)
            for (unsigned j = jb; j < je; j++)
                apply(ie - 1, j, k, x, pmin[1] + j * hy, pmin[2] + k * hz);
    }
    if (bflag & (1u << OCT_DIR_DOWN)) {
        const double y = pmin[1] + jb * hy;
        for (unsigned k = kb; k < ke; k++)
            for (unsigned i = ib; i < ie; i++)
                apply(i, jb, k, pmin[0] + i * hx, y, pmin[2] + k * hz);
    }
    if (bflag & (1u << OCT_DIR_UP)) {
        const double y = pmin[1] + (je - 1) * hy;
        for (unsigned k = kb; k < ke; k++)
            for (unsigned i = ib; i < ie; i++)
                apply(i, je - 1, k, pmin[0] + i * hx, y, pmin[2] + k * hz);
    }
    if (bflag & (1u << OCT_DIR_BACK)) {
        const double z = pmin[2] + kb * hz;
        for (unsigned j = jb; j < je; j++)
            for (unsigned i = ib; i < ie; i++)
                apply(i, j, kb, pmin[0] + i * hx, pmin[1] + j * hy, z);
    }
    if (bflag & (1u << OCT_DIR_FRONT)) {
        const double z = pmin[2] + (ke - 1) * hz;
        for (unsigned j = jb; j < je; j++)
            for (unsigned i = ib; i < ie; i++)
                apply(i, j, ke - 1, pmin[0] + i * hx, pmin[1] + j * hy, z);
    }
}

}  // namespace

extern "C" {

// Hot-path parameters the reference reads from bssn:: globals
// (BSSN_GR/src/parameters.cpp:14-16,40-43,123-136).
struct RefParams {
    double ko_sigma;        // KO_DISS_SIGMA
    unsigned lambda[4];     // BSSN_LAMBDA
    double lambda_f[2];     // BSSN_LAMBDA_F
    double eta_central;     // RIT_ETA_CENTRAL
    double eta_outer;       // RIT_ETA_OUTER
    double eta_width;       // RIT_ETA_WIDTH
    int cako_enabled;       // BSSN_CAKO_ENABLED
    double eps_cako_gauge;  // BSSN_EPSILON_CAKO_GAUGE
    double eps_cako_other;  // BSSN_EPSILON_CAKO_OTHER
};

// 138 * n doubles of derivative workspace, n = sz[0]*sz[1]*sz[2].
void ref_bssnrhs(double** unzipVarsRHS, const double** uZipVars,
                 unsigned offset, const double* pmin, const double* pmax,
                 const unsigned* sz, unsigned bflag, const RefParams* prm,
                 double* deriv_base) {
    const double* const alpha = &uZipVars[U_ALPHA][offset];
    const double* const chi = &uZipVars[U_CHI][offset];
    const double* const K = &uZipVars[U_K][offset];
    const double* const gt0 = &uZipVars[U_SYMGT0][offset];
    const double* const gt1 = &uZipVars[U_SYMGT1][offset];
    const double* const gt2 = &uZipVars[U_SYMGT2][offset];
    const double* const gt3 = &uZipVars[U_SYMGT3][offset];
    const double* const gt4 = &uZipVars[U_SYMGT4][offset];
    const double* const gt5 = &uZipVars[U_SYMGT5][offset];
    const double* const beta0 = &uZipVars[U_BETA0][offset];
    const double* const beta1 = &uZipVars[U_BETA1][offset];
    const double* const beta2 = &uZipVars[U_BETA2][offset];
    const double* const At0 = &uZipVars[U_SYMAT0][offset];
    const double* const At1 = &uZipVars[U_SYMAT1][offset];
    const double* const At2 = &uZipVars[U_SYMAT2][offset];
    const double* const At3 = &uZipVars[U_SYMAT3][offset];
    const double* const At4 = &uZipVars[U_SYMAT4][offset];
    const double* const At5 = &uZipVars[U_SYMAT5][offset];
    const double* const Gt0 = &uZipVars[U_GT0][offset];
    const double* const Gt1 = &uZipVars[U_GT1][offset];
    const double* const Gt2 = &uZipVars[U_GT2][offset];
    const double* const B0 = &uZipVars[U_B0][offset];
    const double* const B1 = &uZipVars[U_B1][offset];
    const double* const B2 = &uZipVars[U_B2][offset];

    double* const a_rhs = &unzipVarsRHS[U_ALPHA][offset];
    double* const chi_rhs = &unzipVarsRHS[U_CHI][offset];
    double* const K_rhs = &unzipVarsRHS[U_K][offset];
    double* const gt_rhs00 = &unzipVarsRHS[U_SYMGT0][offset];
    double* const gt_rhs01 = &unzipVarsRHS[U_SYMGT1][offset];
    double* const gt_rhs02 = &unzipVarsRHS[U_SYMGT2][offset];
    double* const gt_rhs11 = &unzipVarsRHS[U_SYMGT3][offset];
    double* const gt_rhs12 = &unzipVarsRHS[U_SYMGT4][offset];
    double* const gt_rhs22 = &unzipVarsRHS[U_SYMGT5][offset];
    double* const b_rhs0 = &unzipVarsRHS[U_BETA0][offset];
    double* const b_rhs1 = &unzipVarsRHS[U_BETA1][offset];
    double* const b_rhs2 = &unzipVarsRHS[U_BETA2][offset];
    double* const At_rhs00 = &unzipVarsRHS[U_SYMAT0][offset];
    double* const At_rhs01 = &unzipVarsRHS[U_SYMAT1][offset];
    double* const At_rhs02 = &unzipVarsRHS[U_SYMAT2][offset];
    double* const At_rhs11 = &unzipVarsRHS[U_SYMAT3][offset];
    double* const At_rhs12 = &unzipVarsRHS[U_SYMAT4][offset];
    double* const At_rhs22 = &unzipVarsRHS[U_SYMAT5][offset];
    double* const Gt_rhs0 = &unzipVarsRHS[U_GT0][offset];
    double* const Gt_rhs1 = &unzipVarsRHS[U_GT1][offset];
    double* const Gt_rhs2 = &unzipVarsRHS[U_GT2][offset];
    double* const B_rhs0 = &unzipVarsRHS[U_B0][offset];
    double* const B_rhs1 = &unzipVarsRHS[U_B1][offset];
    double* const B_rhs2 = &unzipVarsRHS[U_B2][offset];

    const unsigned nx = sz[0], ny = sz[1], nz = sz[2];
    const double hx = (pmax[0] - pmin[0]) / (nx - 1);
    const double hy = (pmax[1] - pmin[1]) / (ny - 1);
    const double hz = (pmax[2] - pmin[2]) / (nz - 1);
    const unsigned lambda[4] = {prm->lambda[0], prm->lambda[1], prm->lambda[2],
                                prm->lambda[3]};
    const double lambda_f[2] = {prm->lambda_f[0], prm->lambda_f[1]};
    const unsigned PW = 3;
    const unsigned n = nx * ny * nz;
    const unsigned BLK_SZ = n;

    // clang-format off
    #include "bssnrhs_evar_derivs.h"
    #include "bssnrhs_derivs.h"
    // clang-format on

    for (unsigned k = PW; k < nz - PW; k++) {
        for (unsigned j = PW; j < ny - PW; j++) {
            for (unsigned i = PW; i < nx - PW; i++) {
                const double x = pmin[0] + i * hx;
                const double y = pmin[1] + j * hy;
                const double z = pmin[2] + k * hz;
                const unsigned pp = i + nx * (j + ny * k);
                const double r_coord = sqrt(x * x + y * y + z * z);
                const double w = r_coord / prm->eta_width;
                const double arg = -w * w * w * w;
                const double eta =
                    (prm->eta_central - prm->eta_outer) * exp(arg) +
                    prm->eta_outer;
                // clang-format off
                #include "bssneqs_eta_const_standard_gauge.cpp"
                // clang-format on
            }
        }
    }

    if (bflag != 0) {
        bcs(a_rhs, alpha, grad_0_alpha, grad_1_alpha, grad_2_alpha, pmin, pmax, 1.0, 1.0, sz, bflag);
        bcs(chi_rhs, chi, grad_0_chi, grad_1_chi, grad_2_chi, pmin, pmax, 1.0, 1.0, sz, bflag);
        bcs(K_rhs, K, grad_0_K, grad_1_K, grad_2_K, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(b_rhs0, beta0, grad_0_beta0, grad_1_beta0, grad_2_beta0, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(b_rhs1, beta1, grad_0_beta1, grad_1_beta1, grad_2_beta1, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(b_rhs2, beta2, grad_0_beta2, grad_1_beta2, grad_2_beta2, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(Gt_rhs0, Gt0, grad_0_Gt0, grad_1_Gt0, grad_2_Gt0, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(Gt_rhs1, Gt1, grad_0_Gt1, grad_1_Gt1, grad_2_Gt1, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(Gt_rhs2, Gt2, grad_0_Gt2, grad_1_Gt2, grad_2_Gt2, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(B_rhs0, B0, grad_0_B0, grad_1_B0, grad_2_B0, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(B_rhs1, B1, grad_0_B1, grad_1_B1, grad_2_B1, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(B_rhs2, B2, grad_0_B2, grad_1_B2, grad_2_B2, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(At_rhs00, At0, grad_0_At0, grad_1_At0, grad_2_At0, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(At_rhs01, At1, grad_0_At1, grad_1_At1, grad_2_At1, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(At_rhs02, At2, grad_0_At2, grad_1_At2, grad_2_At2, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(At_rhs11, At3, grad_0_At3, grad_1_At3, grad_2_At3, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(At_rhs12, At4, grad_0_At4, grad_1_At4, grad_2_At4, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(At_rhs22, At5, grad_0_At5, grad_1_At5, grad_2_At5, pmin, pmax, 2.0, 0.0, sz, bflag);
        bcs(gt_rhs00, gt0, grad_0_gt0, grad_1_gt0, grad_2_gt0, pmin, pmax, 1.0, 1.0, sz, bflag);
        bcs(gt_rhs01, gt1, grad_0_gt1, grad_1_gt1, grad_2_gt1, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(gt_rhs02, gt2, grad_0_gt2, grad_1_gt2, grad_2_gt2, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(gt_rhs11, gt3, grad_0_gt3, grad_1_gt3, grad_2_gt3, pmin, pmax, 1.0, 1.0, sz, bflag);
        bcs(gt_rhs12, gt4, grad_0_gt4, grad_1_gt4, grad_2_gt4, pmin, pmax, 1.0, 0.0, sz, bflag);
        bcs(gt_rhs22, gt5, grad_0_gt5, grad_1_gt5, grad_2_gt5, pmin, pmax, 1.0, 1.0, sz, bflag);
    }

    // clang-format off
    #include "bssnrhs_ko_derivs.h"
    // clang-format on

    double* const outs[24] = {a_rhs, b_rhs0, b_rhs1, b_rhs2, gt_rhs00, gt_rhs01,
                              gt_rhs02, gt_rhs11, gt_rhs12, gt_rhs22, chi_rhs,
                              At_rhs00, At_rhs01, At_rhs02, At_rhs11, At_rhs12,
                              At_rhs22, K_rhs, Gt_rhs0, Gt_rhs1, Gt_rhs2,
                              B_rhs0, B_rhs1, B_rhs2};
    const double* const kox[24] = {grad_0_alpha, grad_0_beta0, grad_0_beta1, grad_0_beta2, grad_0_gt0, grad_0_gt1, grad_0_gt2, grad_0_gt3, grad_0_gt4, grad_0_gt5, grad_0_chi, grad_0_At0, grad_0_At1, grad_0_At2, grad_0_At3, grad_0_At4, grad_0_At5, grad_0_K, grad_0_Gt0, grad_0_Gt1, grad_0_Gt2, grad_0_B0, grad_0_B1, grad_0_B2};
    const double* const koy[24] = {grad_1_alpha, grad_1_beta0, grad_1_beta1, grad_1_beta2, grad_1_gt0, grad_1_gt1, grad_1_gt2, grad_1_gt3, grad_1_gt4, grad_1_gt5, grad_1_chi, grad_1_At0, grad_1_At1, grad_1_At2, grad_1_At3, grad_1_At4, grad_1_At5, grad_1_K, grad_1_Gt0, grad_1_Gt1, grad_1_Gt2, grad_1_B0, grad_1_B1, grad_1_B2};
    const double* const koz[24] = {grad_2_alpha, grad_2_beta0, grad_2_beta1, grad_2_beta2, grad_2_gt0, grad_2_gt1, grad_2_gt2, grad_2_gt3, grad_2_gt4, grad_2_gt5, grad_2_chi, grad_2_At0, grad_2_At1, grad_2_At2, grad_2_At3, grad_2_At4, grad_2_At5, grad_2_K, grad_2_Gt0, grad_2_Gt1, grad_2_Gt2, grad_2_B0, grad_2_B1, grad_2_B2};
    // CAKO split (rhs.cpp:356-433): alpha, beta and B use the gauge factor.
    const bool gauge_var[24] = {true, true, true, true, false, false, false,
                                false, false, false, false, false, false, false,
                                false, false, false, false, false, false, false,
                                true, true, true};

    for (unsigned k = PW; k < nz - PW; k++) {
        for (unsigned j = PW; j < ny - PW; j++) {
            for (unsigned i = PW; i < nx - PW; i++) {
                const unsigned pp = i + nx * (j + ny * k);
                for (int v = 0; v < 24; v++) {
                    double s = prm->ko_sigma;
                    if (prm->cako_enabled) {
                        const double sc = sqrt(chi[pp]);
                        s = gauge_var[v] ? sc * prm->eps_cako_gauge
                                         : sc * prm->eps_cako_other;
                    }
                    outs[v][pp] += s * (kox[v][pp] + koy[v][pp] + koz[v][pp]);
                }
            }
        }
    }
}


// One block of a mesh (same memory layout as BssnBlockDesc / OrcBlock).
struct RefBlock {
    int64_t offset;
    int32_t sz;
    uint32_t bflag;
    int32_t g0[3];
    int32_t level;
    double ptmin[3];
    double ptmax[3];
};

// The reference's block loop (rhs.cpp:10-73) over the reference bssnrhs, as
// an OpenMP loop with one derivative workspace per thread -- the pattern of
// the reference's own GPU test bed (BSSN_GR/cuda/include/test_utils.h:52-180).
void ref_bssnRHS_blocks(double** rhs, const double** u, const RefBlock* blks,
                        int nblk, const RefParams* prm, int nthreads) {
    int maxs = 0;
    for (int b = 0; b < nblk; b++) maxs = blks[b].sz > maxs ? blks[b].sz : maxs;
    const size_t wsz = (size_t)138 * maxs * maxs * maxs;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> ws(wsz);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nblk; b++) {
            const unsigned sz[3] = {(unsigned)blks[b].sz, (unsigned)blks[b].sz,
                                    (unsigned)blks[b].sz};
            ref_bssnrhs(rhs, u, (unsigned)blks[b].offset, blks[b].ptmin,
                        blks[b].ptmax, sz, blks[b].bflag, prm, ws.data());
        }
    }
}

// Hamiltonian / momentum / psi4 constraint fields on one block, following
// BSSN_GR/src/physcon.cpp:12-89.  cons[0..5] = ham, mom0..2, psi4 re, im.
void ref_physical_constraints(double** cons, const double** uZipVars,
                              unsigned offset, const double* pmin,
                              const double* pmax, const unsigned* sz,
                              unsigned bflag, double* deriv_base) {
    const unsigned nx = sz[0], ny = sz[1], nz = sz[2];
    const unsigned n = nx * ny * nz;
    const double hx = (pmax[0] - pmin[0]) / (nx - 1);
    const double hy = (pmax[1] - pmin[1]) / (ny - 1);
    const double hz = (pmax[2] - pmin[2]) / (nz - 1);
    double* const ham = &cons[0][offset];
    double* const mom0 = &cons[1][offset];
    double* const mom1 = &cons[2][offset];
    double* const mom2 = &cons[3][offset];
    double* const psi4_real = &cons[4][offset];
    double* const psi4_img = &cons[5][offset];
    const double* const alpha = &uZipVars[U_ALPHA][offset];
    const double* const chi = &uZipVars[U_CHI][offset];
    const double* const K = &uZipVars[U_K][offset];
    const double* const gt0 = &uZipVars[U_SYMGT0][offset];
    const double* const gt1 = &uZipVars[U_SYMGT1][offset];
    const double* const gt2 = &uZipVars[U_SYMGT2][offset];
    const double* const gt3 = &uZipVars[U_SYMGT3][offset];
    const double* const gt4 = &uZipVars[U_SYMGT4][offset];
    const double* const gt5 = &uZipVars[U_SYMGT5][offset];
    const double* const beta0 = &uZipVars[U_BETA0][offset];
    const double* const beta1 = &uZipVars[U_BETA1][offset];
    const double* const beta2 = &uZipVars[U_BETA2][offset];
    const double* const At0 = &uZipVars[U_SYMAT0][offset];
    const double* const At1 = &uZipVars[U_SYMAT1][offset];
    const double* const At2 = &uZipVars[U_SYMAT2][offset];
    const double* const At3 = &uZipVars[U_SYMAT3][offset];
    const double* const At4 = &uZipVars[U_SYMAT4][offset];
    const double* const At5 = &uZipVars[U_SYMAT5][offset];
    const double* const Gt0 = &uZipVars[U_GT0][offset];
    const double* const Gt1 = &uZipVars[U_GT1][offset];
    const double* const Gt2 = &uZipVars[U_GT2][offset];
    const double* const B0 = &uZipVars[U_B0][offset];
    const double* const B1 = &uZipVars[U_B1][offset];
    const double* const B2 = &uZipVars[U_B2][offset];
    (void)beta0; (void)beta1; (void)beta2; (void)B0; (void)B1; (void)B2;
    const unsigned PW = 3;
    const unsigned BLK_SZ = n;
    // clang-format off
    #include "bssnrhs_evar_derivs.h"
    #include "constraint_derivs.h"
    // clang-format on
    for (unsigned k = PW; k < nz - PW; k++) {
        for (unsigned j = PW; j < ny - PW; j++) {
            for (unsigned i = PW; i < nx - PW; i++) {
                const double x = pmin[0] + i * hx;
                const double y = pmin[1] + j * hy;
                const double z = pmin[2] + k * hz;
                const unsigned pp = i + nx * (j + ny * k);
                // clang-format off
                #include "physconeqs.cpp"
                // clang-format on
                if (fabs(x) <= 1e-7 && fabs(y) <= 1e-7) {
                    psi4_real[pp] = 0.0;
                    psi4_img[pp] = 0.0;
                }
            }
        }
    }
}

// The reference's stand-alone stencils, exported with C linkage for tests.
void ref_deriv644_x(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { deriv644_x(D, u, h, sz, bflag); }
void ref_deriv644_y(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { deriv644_y(D, u, h, sz, bflag); }
void ref_deriv644_z(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { deriv644_z(D, u, h, sz, bflag); }
void ref_deriv644_xx(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { deriv644_xx(D, u, h, sz, bflag); }
void ref_deriv644_yy(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { deriv644_yy(D, u, h, sz, bflag); }
void ref_deriv644_zz(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { deriv644_zz(D, u, h, sz, bflag); }
void ref_ko_deriv42_x(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { ko_deriv42_x(D, u, h, sz, bflag); }
void ref_ko_deriv42_y(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { ko_deriv42_y(D, u, h, sz, bflag); }
void ref_ko_deriv42_z(double* D, const double* u, double h, const unsigned* sz, unsigned bflag) { ko_deriv42_z(D, u, h, sz, bflag); }
void ref_deriv644adv_x(double* D, const double* u, double h, const unsigned* sz, const double* beta, unsigned bflag) { deriv644adv_x(D, u, h, sz, beta, bflag); }
void ref_deriv644adv_y(double* D, const double* u, double h, const unsigned* sz, const double* beta, unsigned bflag) { deriv644adv_y(D, u, h, sz, beta, bflag); }
void ref_deriv644adv_z(double* D, const double* u, double h, const unsigned* sz, const double* beta, unsigned bflag) { deriv644adv_z(D, u, h, sz, beta, bflag); }

}  // extern "C"
