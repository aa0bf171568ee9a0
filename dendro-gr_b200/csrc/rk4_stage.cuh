// RK4 stage algebra and constraint enforcement on one node held in registers,
// shared by the stage kernels (rk4.cu) and the equation pass that applies
// the stage itself (rhs_split.cu).  Every product and sum is explicitly
// rounded in the reference's order, so the stage algebra is bit-identical to
// the CPU restatement (BSSN_GR/src/rkBSSN.cpp:764-860).
#pragma once
#include <cuda_runtime.h>

#include "bssn_common.cuh"

namespace bssn {
namespace {

__constant__ double kRK4_C[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
__constant__ double kRK4_U[4] = {0.0, 1.0 / 2.0, 1.0 / 2.0, 1.0};

#define M_(a, b) __dmul_rn(a, b)
#define A_(a, b) __dadd_rn(a, b)
#define S_(a, b) __dsub_rn(a, b)

// enforce_bssn_constraints on one node held in registers
// (BSSN_GR/include/bssn_constraints.h:15-172).  Returns 1 on a violation;
// the reference exits there, this code counts it and continues with the
// reference's fallback (flat metric when det < 0).
__device__ __forceinline__ int enforce_regs(double v[NVARS], double chi_floor) {
    const double one_third = 1.0 / 3.0;
    int bad = 0;
    double g00 = v[U_SYMGT0], g01 = v[U_SYMGT1], g02 = v[U_SYMGT2],
           g11 = v[U_SYMGT3], g12 = v[U_SYMGT4], g22 = v[U_SYMGT5];
    double a00 = v[U_SYMAT0], a01 = v[U_SYMAT1], a02 = v[U_SYMAT2],
           a11 = v[U_SYMAT3], a12 = v[U_SYMAT4], a22 = v[U_SYMAT5];
    auto det3 = [&]() {
        // g00*(g11*g22 - g12*g12) - g01*g01*g22 + 2.0*g01*g02*g12 - g02*g02*g11
        double t = M_(g00, S_(M_(g11, g22), M_(g12, g12)));
        t = S_(t, M_(M_(g01, g01), g22));
        t = A_(t, M_(M_(M_(2.0, g01), g02), g12));
        t = S_(t, M_(M_(g02, g02), g11));
        return t;
    };
    double det = det3();
    if (det < 0.0) {
        bad = 1;
        g00 = g11 = g22 = 1.0;
        g01 = g02 = g12 = 0.0;
        det = 1.0;
    }
    const double f = __ddiv_rn(1.0, pow(det, one_third));
    g00 = M_(g00, f); g01 = M_(g01, f); g02 = M_(g02, f);
    g11 = M_(g11, f); g12 = M_(g12, f); g22 = M_(g22, f);
    det = det3();
    if (fabs(S_(det, 1.0)) > 1.0e-6) bad = 1;
    const double idet = __ddiv_rn(1.0, det);
    const double u00 = M_(idet, S_(M_(g11, g22), M_(g12, g12)));
    const double u01 = M_(idet, A_(M_(-g01, g22), M_(g02, g12)));
    const double u02 = M_(idet, S_(M_(g01, g12), M_(g02, g11)));
    const double u11 = M_(idet, S_(M_(g00, g22), M_(g02, g02)));
    const double u12 = M_(idet, A_(M_(-g00, g12), M_(g01, g02)));
    const double u22 = M_(idet, S_(M_(g00, g11), M_(g01, g01)));
    auto trace = [&]() {
        double t = A_(A_(M_(a00, u00), M_(a11, u11)), M_(a22, u22));
        const double o = A_(A_(M_(a01, u01), M_(a02, u02)), M_(a12, u12));
        return A_(t, M_(2.0, o));
    };
    const double tt = M_(one_third, trace());
    a00 = S_(a00, M_(tt, g00)); a01 = S_(a01, M_(tt, g01));
    a02 = S_(a02, M_(tt, g02)); a11 = S_(a11, M_(tt, g11));
    a12 = S_(a12, M_(tt, g12)); a22 = S_(a22, M_(tt, g22));
    if (fabs(trace()) > 1.0e-6) bad = 1;
    v[U_SYMAT0] = a00; v[U_SYMAT1] = a01; v[U_SYMAT2] = a02;
    v[U_SYMAT3] = a11; v[U_SYMAT4] = a12; v[U_SYMAT5] = a22;
    v[U_SYMGT0] = g00; v[U_SYMGT1] = g01; v[U_SYMGT2] = g02;
    v[U_SYMGT3] = g11; v[U_SYMGT4] = g12; v[U_SYMGT5] = g22;
    if (v[U_CHI] < chi_floor) v[U_CHI] = chi_floor;
    v[U_ALPHA] = fmax(v[U_ALPHA], chi_floor);
    return bad;
}

// One RK4 stage at one node (rkBSSN.cpp:851-858 term by term): k = the
// node's right-hand side, v = its state in u on entry.
//   stage s < 3: acc = (s == 0 ? u : acc) + RK4_C[s]*dt*k  -> returned in a
//                v   = u + RK4_U[s+1]*dt*k                  (then enforce if asked)
//   stage 3:     v   = acc + RK4_C[3]*dt*k                  (then enforce)
// Returns the enforcement violation count (0 or 1).
__device__ __forceinline__ int stage_node(int stage, double dt, const double k[NVARS],
                                          double v[NVARS], double a[NVARS], int enforce,
                                          double chi_floor) {
    if (stage < 3) {
        const double cu = M_(kRK4_U[stage + 1], dt);
        const double cc = M_(kRK4_C[stage], dt);
#pragma unroll
        for (int q = 0; q < NVARS; q++) {
            const double a0 = stage == 0 ? v[q] : a[q];
            a[q] = A_(a0, M_(cc, k[q]));
            v[q] = A_(v[q], M_(cu, k[q]));
        }
        return enforce ? enforce_regs(v, chi_floor) : 0;
    }
    const double cc = M_(kRK4_C[3], dt);
#pragma unroll
    for (int q = 0; q < NVARS; q++) v[q] = A_(a[q], M_(cc, k[q]));
    return enforce_regs(v, chi_floor);
}

}  // namespace
}  // namespace bssn
