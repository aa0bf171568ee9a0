// Gravitational-wave extraction: psi4 on extraction spheres decomposed into
// spin-weight -2 spherical-harmonic modes, the computation of the
// reference's extractFarFieldPsi4 (BSSN_GR/include/gwExtract.h:48-190).
//
//   coeff[r][(l,m)] = 4 pi sum_p w_p psi4(p) conj(Y^{-2}_{lm}(p))
//   l2[r]           = (sum_p Re psi4(p)^2, sum_p Im psi4(p)^2)
//
// The reference interpolates psi4 to the sphere points with dendrolib's
// interpolateToCoords (absent from the reference tree) and integrates with a
// Lebedev rule from generated tables.  Here: the degree-6 Lagrange
// interpolation over the 7^3 nodes of the octant that holds the point (the
// element interpolation of an order-6 octree), and a product rule of
// n_theta Gauss-Legendre nodes in cos(theta) times 2 n_theta equally spaced
// phi (exact for the products of modes up to l + l' < 2 n_theta).  The
// harmonics follow Goldberg et al. (J. Math. Phys. 8, 2155 (1967)),
// -2Y_22 = (1/8) sqrt(5/pi) (1 + cos theta)^2 e^{2 i phi}.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "bssn_b200.h"
#include "bssn_common.cuh"

namespace bssn {
namespace {

// Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_n from the
// Chebyshev guesses; three-term recurrence).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; i++) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            const double pn = n == 1 ? z : p1, pm = n == 1 ? 1.0 : p0;
            dp = n * (z * pn - pm) / (z * z - 1.0);
            const double dz = pn / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

double fact(int n) {
    double f = 1.0;
    for (int k = 2; k <= n; k++) f *= k;
    return f;
}
double binom(int n, int k) { return (k < 0 || k > n) ? 0.0 : fact(n) / (fact(k) * fact(n - k)); }

// spin-weighted spherical harmonic sY_lm at (theta, phi): re, im
void swsh(int s, int l, int m, double th, double ph, double* re, double* im) {
    const double pre = ((m & 1) ? -1.0 : 1.0) *
                       std::sqrt(fact(l + m) * fact(l - m) * (2 * l + 1) / (4.0 * M_PI * fact(l + s) * fact(l - s)));
    const double sh = std::sin(0.5 * th), ch = std::cos(0.5 * th);
    double sum = 0.0;
    for (int r = 0; r <= l - s; r++) {
        const double c = binom(l - s, r) * binom(l + s, r + s - m);
        if (c == 0.0) continue;
        // sin^{2l}(th/2) cot^{2r+s-m}(th/2) = sin^{2l-2r-s+m} cos^{2r+s-m}
        const int pc = 2 * r + s - m, ps = 2 * l - pc;
        sum += (((l - r - s) & 1) ? -1.0 : 1.0) * c * std::pow(sh, ps) * std::pow(ch, pc);
    }
    *re = pre * sum * std::cos(m * ph);
    *im = pre * sum * std::sin(m * ph);
}

struct Sphere {
    std::vector<double> theta, phi, w;   // per point
    std::vector<double> yre, yim;        // [mode][point]
    int npts = 0, nmodes = 0;
};

void build_sphere(int lmax, int ntheta, Sphere* S) {
    std::vector<double> x, w;
    gauss_legendre(ntheta, x, w);
    const int nphi = 2 * ntheta;
    for (int i = 0; i < ntheta; i++)
        for (int j = 0; j < nphi; j++) {
            S->theta.push_back(std::acos(x[i]));
            S->phi.push_back(2.0 * M_PI * j / nphi);
            S->w.push_back(w[i] * 2.0 * M_PI / nphi);
        }
    S->npts = ntheta * nphi;
    S->nmodes = 0;
    for (int l = 2; l <= lmax; l++)
        for (int m = -l; m <= l; m++) {
            for (int p = 0; p < S->npts; p++) {
                double re, im;
                swsh(-2, l, m, S->theta[p], S->phi[p], &re, &im);
                S->yre.push_back(re);
                S->yim.push_back(im);
            }
            S->nmodes++;
        }
}

// degree-6 Lagrange basis on nodes 0..6 at t
__device__ __forceinline__ void lagrange7(double t, double w[7]) {
    for (int m = 0; m < 7; m++) {
        double v = 1.0;
        for (int k = 0; k < 7; k++)
            if (k != m) v *= (t - k) / (double)(m - k);
        w[m] = v;
    }
}

// psi4 at the sphere points (x, y, z given): the enclosing octant's 7^3
// nodes; points outside the node grid get weight 0 (valid[p] = 0).
__global__ void gw_interp_kernel(const double* __restrict__ re, const double* __restrict__ im,
                                 const double* __restrict__ pts, int n, int gx, int gy, int gz,
                                 double x0, double y0, double z0, double h, double* __restrict__ out,
                                 int* __restrict__ valid) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double g[3] = {(pts[3 * p] - x0) / h, (pts[3 * p + 1] - y0) / h, (pts[3 * p + 2] - z0) / h};
    const int G[3] = {gx, gy, gz};
    int t[3];
    double w[3][7];
    bool ok = true;
    for (int d = 0; d < 3; d++) {
        ok = ok && g[d] >= 0.0 && g[d] <= G[d] - 1;
        const int M = (G[d] - 1) / 6;
        int o = (int)floor(g[d] / 6.0);
        o = o < 0 ? 0 : (o > M - 1 ? M - 1 : o);
        t[d] = 6 * o;
        lagrange7(g[d] - t[d], w[d]);
    }
    valid[p] = ok;
    double sr = 0.0, si = 0.0;
    if (ok)
        for (int c = 0; c < 7; c++)
            for (int b = 0; b < 7; b++) {
                double rr = 0.0, ii = 0.0;
                const int64_t row = t[0] + (int64_t)gx * ((t[1] + b) + (int64_t)gy * (t[2] + c));
                for (int a = 0; a < 7; a++) {
                    rr += w[0][a] * re[row + a];
                    ii += w[0][a] * im[row + a];
                }
                sr += w[1][b] * w[2][c] * rr;
                si += w[1][b] * w[2][c] * ii;
            }
    out[2 * p] = sr;
    out[2 * p + 1] = si;
}

// One CTA per (radius, mode) -- mode index nmodes is the L2 sums -- with a
// fixed-order tree reduction, so the result is deterministic.
__global__ void __launch_bounds__(256) gw_modes_kernel(const double* __restrict__ val,
                                                       const int* __restrict__ valid,
                                                       const double* __restrict__ w,
                                                       const double* __restrict__ yre,
                                                       const double* __restrict__ yim, int npts,
                                                       int nmodes, double* __restrict__ coeff,
                                                       double* __restrict__ l2) {
    const int r = blockIdx.x / (nmodes + 1), k = blockIdx.x % (nmodes + 1);
    __shared__ double red[2][256];
    double a = 0.0, b = 0.0;
    for (int p = threadIdx.x; p < npts; p += blockDim.x) {
        const int q = r * npts + p;
        if (!valid[q]) continue;
        const double pr = val[2 * q], pi = val[2 * q + 1];
        if (k == nmodes) {
            a += pr * pr;
            b += pi * pi;
        } else {
            // psi4 * conj(Y) * w
            const double cr = yre[(int64_t)k * npts + p], ci = -yim[(int64_t)k * npts + p];
            a += w[p] * (pr * cr - pi * ci);
            b += w[p] * (pr * ci + pi * cr);
        }
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            red[0][threadIdx.x] += red[0][threadIdx.x + st];
            red[1][threadIdx.x] += red[1][threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (k == nmodes) {
            l2[2 * r] = red[0][0];
            l2[2 * r + 1] = red[1][0];
        } else {
            coeff[2 * ((int64_t)r * nmodes + k)] = 4.0 * M_PI * red[0][0];
            coeff[2 * ((int64_t)r * nmodes + k) + 1] = 4.0 * M_PI * red[1][0];
        }
    }
}

template <class T>
int dev_copy(const std::vector<T>& v, T** d) {
    if (cudaMalloc((void**)d, sizeof(T) * (v.empty() ? 1 : v.size())) != cudaSuccess) {
        cudaGetLastError();
        *d = nullptr;
        return BSSN_ENOMEM;
    }
    return v.empty() ? 0 : cuda_status(cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
}

}  // namespace
}  // namespace bssn

extern "C" {

int bssn_gw_modes_count(int lmax) { return lmax < 2 ? 0 : (lmax + 1) * (lmax + 1) - 4; }

int bssn_gw_sphere_tables(int lmax, int ntheta, double* theta, double* phi, double* w, double* y) {
    if (lmax < 2 || lmax > 16 || ntheta < 2 || ntheta > 512) return BSSN_EINVAL;
    bssn::Sphere S;
    bssn::build_sphere(lmax, ntheta, &S);
    if (theta) std::memcpy(theta, S.theta.data(), sizeof(double) * S.npts);
    if (phi) std::memcpy(phi, S.phi.data(), sizeof(double) * S.npts);
    if (w) std::memcpy(w, S.w.data(), sizeof(double) * S.npts);
    if (y)
        for (size_t i = 0; i < S.yre.size(); i++) {
            y[2 * i] = S.yre[i];
            y[2 * i + 1] = S.yim[i];
        }
    return 0;
}

int bssn_gw_extract_f64(const double* psi4_re_dev, const double* psi4_im_dev, const int32_t G[3],
                        const double xmin[3], double h, int nradii, const double* radii, int lmax,
                        int ntheta, double* coeff_dev, double* l2_dev, bssn_stream_t stream) {
    if (!psi4_re_dev || !psi4_im_dev || !G || !xmin || !radii || !coeff_dev || !l2_dev || !(h > 0.0) ||
        nradii < 1 || nradii > 64 || lmax < 2 || lmax > 16 || ntheta < 2 || ntheta > 512)
        return BSSN_EINVAL;
    for (int d = 0; d < 3; d++)
        if (G[d] < 7 || (G[d] - 1) % 6) return BSSN_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    bssn::Sphere S;
    bssn::build_sphere(lmax, ntheta, &S);
    std::vector<double> pts;
    pts.reserve((size_t)3 * nradii * S.npts);
    for (int r = 0; r < nradii; r++)
        for (int p = 0; p < S.npts; p++) {
            pts.push_back(radii[r] * std::sin(S.theta[p]) * std::cos(S.phi[p]));
            pts.push_back(radii[r] * std::sin(S.theta[p]) * std::sin(S.phi[p]));
            pts.push_back(radii[r] * std::cos(S.theta[p]));
        }
    const int n = nradii * S.npts;
    double *dpts = nullptr, *dval = nullptr, *dw = nullptr, *dyr = nullptr, *dyi = nullptr;
    int* dvalid = nullptr;
    int st = bssn::dev_copy(pts, &dpts);
    if (!st) st = bssn::dev_copy(S.w, &dw);
    if (!st) st = bssn::dev_copy(S.yre, &dyr);
    if (!st) st = bssn::dev_copy(S.yim, &dyi);
    if (!st) st = bssn::dev_copy(std::vector<double>((size_t)2 * n), &dval);
    if (!st) st = bssn::dev_copy(std::vector<int>((size_t)n), &dvalid);
    if (!st) {
        bssn::gw_interp_kernel<<<(n + 127) / 128, 128, 0, s>>>(psi4_re_dev, psi4_im_dev, dpts, n, G[0], G[1], G[2],
                                                                xmin[0], xmin[1], xmin[2], h, dval, dvalid);
        st = bssn::cuda_status(cudaGetLastError());
    }
    if (!st) {
        bssn::gw_modes_kernel<<<nradii * (S.nmodes + 1), 256, 0, s>>>(dval, dvalid, dw, dyr, dyi, S.npts, S.nmodes,
                                                                       coeff_dev, l2_dev);
        st = bssn::cuda_status(cudaGetLastError());
    }
    if (!st) st = bssn::cuda_status(cudaStreamSynchronize(s));
    cudaFree(dpts);
    cudaFree(dval);
    cudaFree(dw);
    cudaFree(dyr);
    cudaFree(dyi);
    cudaFree(dvalid);
    return st;
}

}  // extern "C"
