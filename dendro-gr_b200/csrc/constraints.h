// Launchers of the constraint diagnostics.
#pragma once
#include <cuda_runtime.h>

namespace bssn {
struct MeshState;
// CTAs of the norm reduction; each leaves 5 partial sums.
constexpr int kNormPartials = 592;
// out[0..3] = ham, mom0..2; with psi4, out[4], out[5] = psi4 real, imaginary.
int launch_constraints(const MeshState* m, const double* const* P, double* const* out,
                       cudaStream_t s, bool psi4 = false);
int launch_l2_norms(const MeshState* m, const double* const* C, int nc, const double xmin[3],
                    double h, const double bh[6], const double radii[2], double* partial,
                    int npartial, double* norms, cudaStream_t s,
                    const uint8_t* mask = nullptr, bool sums = false);
}  // namespace bssn
