// Shared definitions of the device code: variable order, kernel argument
// packs, stencil coefficients and the status word.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bssn_b200.h"

namespace bssn {

// Variable order of the reference (BSSN_GR/include/grDef.h:35-60).
enum Var : int {
    U_ALPHA = 0, U_CHI, U_K, U_GT0, U_GT1, U_GT2, U_BETA0, U_BETA1, U_BETA2,
    U_B0, U_B1, U_B2, U_SYMGT0, U_SYMGT1, U_SYMGT2, U_SYMGT3, U_SYMGT4,
    U_SYMGT5, U_SYMAT0, U_SYMAT1, U_SYMAT2, U_SYMAT3, U_SYMAT4, U_SYMAT5,
    NVARS
};

// 24 per-variable base pointers, passed by value in kernel parameters.
struct ConstVars { const double* p[NVARS]; };
struct MutVars { double* p[NVARS]; };

// Symmetric 3x3 component index: (0,0)(0,1)(0,2)(1,1)(1,2)(2,2) -> 0..5.
__host__ __device__ constexpr int sym(int i, int j) {
    return i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5))
                  : (j == 0 ? i : (j == 1 ? 2 + i : 5));
}
__host__ __device__ constexpr int sym_a(int c) { return c < 3 ? 0 : (c < 5 ? 1 : 2); }
__host__ __device__ constexpr int sym_b(int c) { return c < 3 ? c : (c < 5 ? c - 2 : 2); }

// Sommerfeld falloff / asymptotic value per variable (rhs.cpp:275-327).
__host__ __device__ constexpr double falloff(int v) {
    return (v >= U_GT0 && v <= U_GT2) || (v >= U_SYMAT0) ? 2.0 : 1.0;
}
__host__ __device__ constexpr double asymptotic(int v) {
    return (v == U_ALPHA || v == U_CHI || v == U_SYMGT0 || v == U_SYMGT3 ||
            v == U_SYMGT5) ? 1.0 : 0.0;
}
// CAKO gauge split (rhs.cpp:356-433): alpha, beta and B.
__host__ __device__ constexpr bool gauge_var(int v) {
    return v == U_ALPHA || (v >= U_BETA0 && v <= U_B2);
}

// Per-axis stencil factors, computed exactly as derivs.cpp computes them.
struct AxisCoef {
    double ih60;     // (1/h)/60
    double ih12;     // (1/h)/12
    double ih2_180;  // (1/(h*h))/180
    double ih2_12;   // (1/(h*h))/12
    double ko_pre;   // -1/64/h
    double smr1, smr2, smr3;  // 49/48*64*h, 43/48*64*h, 59/48*64*h
};

__host__ __device__ inline AxisCoef axis_coef(double h) {
    AxisCoef c;
    const double ih = 1.0 / h;
    c.ih60 = ih / 60.0;
    c.ih12 = ih / 12.0;
    const double ih2 = 1.0 / (h * h);
    c.ih2_180 = ih2 / 180.0;
    c.ih2_12 = ih2 / 12.0;
    c.ko_pre = -1.0 / 64.0 / h;
    c.smr3 = 59.0 / 48.0 * 64 * h;
    c.smr2 = 43.0 / 48.0 * 64 * h;
    c.smr1 = 49.0 / 48.0 * 64 * h;
    return c;
}

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? 0 : -(int)e; }

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current
// device, once per (kernel, device) pair.  The attribute belongs to the
// device, so a process that launches on several devices needs it set on each
// of them; calls from several host threads are serialised.
int set_smem_limit(const void* kernel, int bytes);

}  // namespace bssn
