// Hamiltonian and momentum constraints and their masked L2 norms.
//
//   ham   = chi ig^jk R_jk - A_ij A^ij + 2/3 K^2
//   mom_i = ig^jk (d_k A_ij - C2^m_ki A_jm) - Gt^j A_ij
//           - 3/2 ig^jk A_ki d_j chi / chi - 2/3 d_i K
// (CodeGen/constraints.py:250-283; per block as BSSN_GR/src/physcon.cpp:12-89)
// and the norm sqrt(sum c^2 / N) over the zipped nodes outside the puncture
// radii (BSSN_GR/include/grUtils.tcc:36-134).
//
// A diagnostic, run every few steps, so it favours simplicity: one thread per
// owned interior node, derivatives read straight from the padded block in
// global memory (cached), with the bit-exact stencils of stencil_exact.cuh;
// mixed derivatives are first derivatives of on-the-fly first derivatives,
// in the reference's order (d/dy(d/dx), d/dz(d/dx), d/dz(d/dy)).
#include <cuda_runtime.h>

#include <algorithm>

#include "bssn_common.cuh"
#include "constraints.h"
#include "kernels.cuh"
#include "mesh.h"
#include "stencil_exact.cuh"

namespace bssn {
namespace {

// The bit-exact first-derivative stencil (derivs.cpp:2645-2700) on values
// produced by a functor val(m) = value at along-axis coordinate m.
template <int N, class F>
__device__ __forceinline__ double foldf(const double (&c)[N], F val, const int (&pos)[N]) {
    double t = __dmul_rn(c[0], val(pos[0]));
#pragma unroll
    for (int q = 1; q < N; q++) t = __dadd_rn(t, __dmul_rn(c[q], val(pos[q])));
    return t;
}

template <class F>
__device__ __forceinline__ double d1f(F val, int a, int s, bool lo, bool hi, const AxisCoef& cf) {
    const int ie = s - 3;
    if (lo && a <= 5) {
        if (a == 3) { const double c[5] = {-25.0, 48.0, -36.0, 16.0, -3.0}; const int p[5] = {3, 4, 5, 6, 7}; return __dmul_rn(foldf(c, val, p), cf.ih12); }
        if (a == 4) { const double c[5] = {-3.0, -10.0, 18.0, -6.0, 1.0}; const int p[5] = {3, 4, 5, 6, 7}; return __dmul_rn(foldf(c, val, p), cf.ih12); }
        const double c[4] = {1.0, -8.0, 8.0, -1.0}; const int p[4] = {3, 4, 6, 7}; return __dmul_rn(foldf(c, val, p), cf.ih12);
    }
    if (hi && a >= ie - 3) {
        if (a == ie - 3) { const double c[4] = {1.0, -8.0, 8.0, -1.0}; const int p[4] = {ie - 5, ie - 4, ie - 2, ie - 1}; return __dmul_rn(foldf(c, val, p), cf.ih12); }
        if (a == ie - 2) { const double c[5] = {-1.0, 6.0, -18.0, 10.0, 3.0}; const int p[5] = {ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(foldf(c, val, p), cf.ih12); }
        const double c[5] = {3.0, -16.0, 36.0, -48.0, 25.0}; const int p[5] = {ie - 5, ie - 4, ie - 3, ie - 2, ie - 1}; return __dmul_rn(foldf(c, val, p), cf.ih12);
    }
    const double c[6] = {-1.0, 9.0, -45.0, 45.0, -9.0, 1.0};
    const int p[6] = {a - 3, a - 2, a - 1, a + 1, a + 2, a + 3};
    return __dmul_rn(foldf(c, val, p), cf.ih60);
}

struct Blk {
    int s;
    int a[3];
    unsigned bflag;
    AxisCoef cf[3];
};

__device__ __forceinline__ int64_t stride(const Blk& b, int d) {
    return d == 0 ? 1 : (d == 1 ? b.s : (int64_t)b.s * b.s);
}

__device__ __forceinline__ const double* origin(const Blk& b, const double* u, int d) {
    const int64_t here = b.a[0] + (int64_t)b.s * (b.a[1] + (int64_t)b.s * b.a[2]);
    return u + here - b.a[d] * stride(b, d);
}

// first derivative of variable array u (padded block origin) along d
__device__ __forceinline__ double D1(const Blk& b, const double* u, int d) {
    return ex::d1(origin(b, u, d), (int)stride(b, d), b.a[d], b.s, b.bflag & (1u << 2 * d),
                  b.bflag & (1u << (2 * d + 1)), b.cf[d]);
}

__device__ __forceinline__ double D2(const Blk& b, const double* u, int d) {
    return ex::d2(origin(b, u, d), (int)stride(b, d), b.a[d], b.s, b.bflag & (1u << 2 * d),
                  b.bflag & (1u << (2 * d + 1)), b.cf[d]);
}

// d/d_outer (d/d_inner u) at the node
__device__ __forceinline__ double Dmix(const Blk& b, const double* u, int inner, int outer) {
    auto val = [&](int m) {
        Blk c = b;
        c.a[outer] = m;
        return D1(c, u, inner);
    };
    return d1f(val, b.a[outer], b.s, b.bflag & (1u << 2 * outer),
               b.bflag & (1u << (2 * outer + 1)), b.cf[outer]);
}

// PSI4: also the Weyl scalar psi4 into out.p[4] (real) and out.p[5]
// (imaginary) -- CodeGen/constraints.py:45-244, per point as
// BSSN_GR/src/physcon.cpp:72-85 (coordinates ptmin + a h of the padded
// index a, zero on the z axis): the tetrad r = (x, y, z), theta =
// (xz, yz, -(x^2 + y^2)), phi = (-y, x, 0) made orthonormal by Gram-Schmidt
// in the physical metric gt / chi, m = (theta + i phi) / sqrt 2, and
// psi4 = -(P1 + P2 - P3 - P4) real, P1 + P2 - P3 - P4 imaginary, with
// P1 = R_ij M^ij, P2 = A_temp At_ij M^ij, P3 = (MR_ij Uu_ij - NR_ij Vv_ij)/chi
// and P4 the (At r) and d chi products of the definition.
template <bool PSI4>
__device__ void constraints_node(const ConstVars& P, const MutVars& out, const BssnBlockDesc& bd,
                                 int64_t q, int gx, int gy, int gz, int64_t node_at = -1) {
    const int s = bd.sz, N = s - 6;
    const int i = (int)(q % N), j = (int)((q / N) % N), k = (int)(q / ((int64_t)N * N));
    const int64_t x = bd.g0[0] + i, y = bd.g0[1] + j, z = bd.g0[2] + k;
    const bool own = (i < N - 1 || x == gx - 1) && (j < N - 1 || y == gy - 1) &&
                     (k < N - 1 || z == gz - 1);
    if (node_at < 0 && !own) return;
    Blk b;
    b.s = s;
    b.a[0] = i + 3;
    b.a[1] = j + 3;
    b.a[2] = k + 3;
    b.bflag = bd.bflag;
    for (int d = 0; d < 3; d++) b.cf[d] = axis_coef((bd.ptmax[d] - bd.ptmin[d]) / (s - 1));
    const int64_t pidx = bd.offset + b.a[0] + (int64_t)s * (b.a[1] + (int64_t)s * b.a[2]);
    auto V = [&](int v) { return P.p[v] + bd.offset; };
    auto pv = [&](int v) { return P.p[v][pidx]; };

    double g[6], ig[6];
    for (int c = 0; c < 6; c++) g[c] = pv(U_SYMGT0 + c);
    {
        const double c00 = g[3] * g[5] - g[4] * g[4];
        const double c01 = g[2] * g[4] - g[1] * g[5];
        const double c02 = g[1] * g[4] - g[2] * g[3];
        const double idet = 1.0 / (g[0] * c00 + g[1] * c01 + g[2] * c02);
        ig[0] = c00 * idet;
        ig[1] = c01 * idet;
        ig[2] = c02 * idet;
        ig[3] = (g[0] * g[5] - g[2] * g[2]) * idet;
        ig[4] = (g[2] * g[1] - g[0] * g[4]) * idet;
        ig[5] = (g[0] * g[3] - g[1] * g[1]) * idet;
    }
    auto IG = [&](int a, int c) { return ig[sym(a, c)]; };
    auto Gm = [&](int a, int c) { return g[sym(a, c)]; };
    // metric derivatives and ig^lm d_l d_m g_ij
    double dg[6][3], Lg[6];
    for (int c = 0; c < 6; c++) {
        const double* u = V(U_SYMGT0 + c);
        double d2[6];
        for (int d = 0; d < 3; d++) dg[c][d] = D1(b, u, d);
        d2[0] = D2(b, u, 0);
        d2[3] = D2(b, u, 1);
        d2[5] = D2(b, u, 2);
        d2[1] = Dmix(b, u, 0, 1);
        d2[2] = Dmix(b, u, 0, 2);
        d2[4] = Dmix(b, u, 1, 2);
        Lg[c] = ig[0] * d2[0] + ig[3] * d2[3] + ig[5] * d2[5] +
                2.0 * (ig[1] * d2[1] + ig[2] * d2[2] + ig[4] * d2[4]);
    }
    double C1[3][6], C2[3][6], CalGt[3];
    for (int kk = 0; kk < 3; kk++)
        for (int c = 0; c < 6; c++) {
            const int a = sym_a(c), bb = sym_b(c);
            C1[kk][c] = 0.5 * (dg[sym(kk, a)][bb] + dg[sym(kk, bb)][a] - dg[c][kk]);
        }
    for (int a = 0; a < 3; a++)
        for (int c = 0; c < 6; c++)
            C2[a][c] = IG(a, 0) * C1[0][c] + IG(a, 1) * C1[1][c] + IG(a, 2) * C1[2][c];
    for (int a = 0; a < 3; a++)
        CalGt[a] = ig[0] * C2[a][0] + ig[3] * C2[a][3] + ig[5] * C2[a][5] +
                   2.0 * (ig[1] * C2[a][1] + ig[2] * C2[a][2] + ig[4] * C2[a][4]);
    // conformal Ricci tensor (CodeGen/dendro.py:485-550)
    double R[6];
    for (int c = 0; c < 6; c++) {
        const int a = sym_a(c), bb = sym_b(c);
        double rt = -0.5 * Lg[c];
        for (int kk = 0; kk < 3; kk++) rt += 0.5 * CalGt[kk] * (C1[a][sym(bb, kk)] + C1[bb][sym(a, kk)]);
        for (int kk = 0; kk < 3; kk++)
            for (int l = 0; l < 3; l++)
                for (int m = 0; m < 3; m++)
                    rt += IG(l, m) * (C2[kk][sym(l, a)] * C1[bb][sym(kk, m)] +
                                      C2[kk][sym(l, bb)] * C1[a][sym(kk, m)] +
                                      C2[kk][sym(a, m)] * C1[kk][sym(l, bb)]);
        R[c] = rt;
    }
    for (int kk = 0; kk < 3; kk++) {
        const double* u = V(U_GT0 + kk);
        double dG[3];
        for (int d = 0; d < 3; d++) dG[d] = D1(b, u, d);
        for (int c = 0; c < 6; c++) {
            const int a = sym_a(c), bb = sym_b(c);
            R[c] += 0.5 * (Gm(kk, a) * dG[bb] + Gm(kk, bb) * dG[a]);
        }
    }
    const double chi = pv(U_CHI), K = pv(U_K);
    double dchi[3], ddchi[6];
    {
        const double* u = V(U_CHI);
        for (int d = 0; d < 3; d++) dchi[d] = D1(b, u, d);
        ddchi[0] = D2(b, u, 0);
        ddchi[3] = D2(b, u, 1);
        ddchi[5] = D2(b, u, 2);
        ddchi[1] = Dmix(b, u, 0, 1);
        ddchi[2] = Dmix(b, u, 0, 2);
        ddchi[4] = Dmix(b, u, 1, 2);
    }
    {
        const double ichi = 1.0 / chi;
        double T = 0.0;
        for (int a = 0; a < 3; a++)
            for (int c = 0; c < 3; c++)
                T += IG(a, c) * (ddchi[sym(a, c)] - 3.0 / (2.0 * chi) * dchi[a] * dchi[c]);
        for (int m = 0; m < 3; m++) T -= CalGt[m] * dchi[m];
        for (int c = 0; c < 6; c++) {
            const int a = sym_a(c), bb = sym_b(c);
            double sk = ddchi[c];
            for (int kk = 0; kk < 3; kk++) sk -= C2[kk][c] * dchi[kk];
            R[c] += 0.5 * ichi * sk - 0.25 * ichi * ichi * dchi[a] * dchi[bb] + 0.5 * ichi * g[c] * T;
        }
    }
    double A[6], AUU[6];
    for (int c = 0; c < 6; c++) A[c] = pv(U_SYMAT0 + c);
    auto AM = [&](int a, int c) { return A[sym(a, c)]; };
    for (int c = 0; c < 6; c++) {
        const int a = sym_a(c), bb = sym_b(c);
        double sacc = 0.0;
        for (int kk = 0; kk < 3; kk++)
            for (int l = 0; l < 3; l++) sacc += IG(a, kk) * IG(bb, l) * AM(kk, l);
        AUU[c] = sacc;
    }
    double ham = 0.0, sqrA = 0.0;
    for (int c = 0; c < 6; c++) {
        const double w = sym_a(c) == sym_b(c) ? 1.0 : 2.0;
        ham += w * chi * ig[c] * R[c];
        sqrA += w * A[c] * AUU[c];
    }
    const int64_t node = node_at >= 0 ? node_at : x + (int64_t)gx * (y + (int64_t)gy * z);
    out.p[0][node] = ham - sqrA + 2.0 / 3.0 * K * K;
    double dK[3];
    for (int d = 0; d < 3; d++) dK[d] = D1(b, V(U_K), d);
    double dA[6][3];
    for (int c = 0; c < 6; c++)
        for (int d = 0; d < 3; d++) dA[c][d] = D1(b, V(U_SYMAT0 + c), d);
    for (int a = 0; a < 3; a++) {
        double m = 0.0;
        for (int bb = 0; bb < 3; bb++)
            for (int c = 0; c < 3; c++) {
                double t = dA[sym(a, bb)][c];
                for (int qq = 0; qq < 3; qq++) t -= C2[qq][sym(c, a)] * AM(bb, qq);
                m += IG(bb, c) * t;
            }
        for (int bb = 0; bb < 3; bb++) m -= pv(U_GT0 + bb) * AM(a, bb);
        for (int bb = 0; bb < 3; bb++)
            for (int c = 0; c < 3; c++) m -= 1.5 * IG(bb, c) * AM(c, a) * dchi[bb] / chi;
        m -= 2.0 / 3.0 * dK[a];
        out.p[1 + a][node] = m;
    }
    if constexpr (PSI4) {
        double crd[3];
        for (int d = 0; d < 3; d++) {
            const double h = (bd.ptmax[d] - bd.ptmin[d]) / (s - 1);
            crd[d] = __dadd_rn(bd.ptmin[d], __dmul_rn((double)b.a[d], h));
        }
        if (fabs(crd[0]) <= 1e-7 && fabs(crd[1]) <= 1e-7) {
            out.p[4][node] = 0.0;
            out.p[5][node] = 0.0;
            return;
        }
        const double ichi = 1.0 / chi;
        auto dot = [&](const double* p, const double* r) {  // in the physical metric
            double t = 0.0;
            for (int bb = 0; bb < 3; bb++)
                for (int a = 0; a < 3; a++) t += Gm(a, bb) * ichi * p[a] * r[bb];
            return t;
        };
        const double cx = crd[0], cy = crd[1], cz = crd[2];
        double rv[3] = {cx, cy, cz}, th[3] = {cx * cz, cy * cz, -(cx * cx + cy * cy)}, ph[3] = {-cy, cx, 0.0};
        {
            const double nr = sqrt(dot(rv, rv));
            for (int a = 0; a < 3; a++) rv[a] /= nr;
            const double p1 = dot(th, th), p2 = dot(rv, th);
            for (int a = 0; a < 3; a++) th[a] -= p2 * rv[a];
            const double nt = sqrt(p1 - p2 * p2);
            for (int a = 0; a < 3; a++) th[a] /= nt;
            const double f1 = dot(ph, ph), f2 = dot(rv, ph), f3 = dot(th, ph);
            for (int a = 0; a < 3; a++) ph[a] -= f2 * rv[a] + f3 * th[a];
            const double np = sqrt(f1 - f2 * f2 - f3 * f3);
            for (int a = 0; a < 3; a++) ph[a] /= np;
        }
        const double s2 = 1.0 / sqrt(2.0);
        double mr[3], mi[3];
        for (int a = 0; a < 3; a++) {
            mr[a] = th[a] * s2;
            mi[a] = ph[a] * s2;
        }
        double Av[3];
        for (int a = 0; a < 3; a++) Av[a] = AM(a, 0) * rv[0] + AM(a, 1) * rv[1] + AM(a, 2) * rv[2];
        double rdc = 0.0, mrdc = 0.0, midc = 0.0, rA = 0.0, mrA = 0.0, miA = 0.0;
        for (int a = 0; a < 3; a++) {
            rdc += rv[a] * dchi[a];
            mrdc += mr[a] * dchi[a];
            midc += mi[a] * dchi[a];
            rA += Av[a] * rv[a];
            mrA += mr[a] * Av[a];
            miA += mi[a] * Av[a];
        }
        const double Atmp = ichi * ichi * (rA + K * chi / 3.0 + 0.5 * rdc);
        double p1r = 0.0, p1i = 0.0, q2r = 0.0, q2i = 0.0, s3r = 0.0, s3i = 0.0;
        for (int a = 0; a < 3; a++)
            for (int bb = 0; bb < 3; bb++) {
                const double MMab = mr[a] * mr[bb] - mi[a] * mi[bb];
                const double NNab = mr[a] * mi[bb] + mr[bb] * mi[a];
                p1r += R[sym(a, bb)] * MMab;
                p1i += R[sym(a, bb)] * NNab;
                q2r += AM(a, bb) * MMab;
                q2i += AM(a, bb) * NNab;
                const double MRab = mr[a] * rv[bb] - mr[bb] * rv[a];
                const double NRab = mi[a] * rv[bb] - mi[bb] * rv[a];
                double uu = 0.0, vv = 0.0;
                for (int c = 0; c < 3; c++) {
                    double t = dA[sym(c, a)][bb];
                    for (int mm = 0; mm < 3; mm++) t += C2[mm][sym(c, a)] * AM(mm, bb);
                    uu += mr[c] * t;
                    vv += mi[c] * t;
                }
                s3r += MRab * uu - NRab * vv;
                s3i += NRab * uu + MRab * vv;
            }
        const double p4r = ichi * ichi * (mrA * (mrA + 0.5 * mrdc) - miA * (miA + 0.5 * midc));
        const double p4i = ichi * ichi * (mrA * (miA + 0.5 * midc) + miA * (mrA + 0.5 * mrdc));
        out.p[4][node] = -(p1r + Atmp * q2r - ichi * s3r - p4r);
        out.p[5][node] = p1i + Atmp * q2i - ichi * s3i - p4i;
    }
}

// One CTA per chunk of up to 1024 interior points of a block, 256 threads
// striding over it (the node function needs up to 255 registers).
template <bool PSI4>
__global__ void __launch_bounds__(256) constraints_kernel(ConstVars P, MutVars out,
                                                          const BssnBlockDesc* __restrict__ blocks,
                                                          const Chunk* __restrict__ chunks, int gx,
                                                          int gy, int gz) {
    const Chunk ck = chunks[blockIdx.x];
    const BssnBlockDesc bd = blocks[ck.blk];
    for (int r = threadIdx.x; r < ck.count; r += blockDim.x)
        constraints_node<PSI4>(P, out, bd, ck.start + r, gx, gy, gz);
}

// Multi-level meshes: node n of the zipped state (the level grids back to
// back) takes the constraints at the zone that owns it, zip_src[n] (a padded
// index); nodes filled from another level (zip_src -1: patch-boundary nodes
// and coarse nodes under a finer patch) get 0.  The owning block is the last
// one whose offset is <= the padded index (offsets ascend).
template <bool PSI4>
__global__ void __launch_bounds__(256) constraints_levels_kernel(ConstVars P, MutVars out,
                                                                 const BssnBlockDesc* __restrict__ blocks,
                                                                 int nblocks,
                                                                 const int64_t* __restrict__ zip_src,
                                                                 int64_t n_nodes) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_nodes;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = zip_src[n];
        int lo = 0, hi = nblocks - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (blocks[mid].offset <= p) lo = mid;
            else hi = mid - 1;
        }
        const BssnBlockDesc bd = blocks[lo];
        const int s = bd.sz;
        const int64_t a = p - bd.offset;
        const int ax = (int)(a % s), ay = (int)((a / s) % s), az = (int)(a / ((int64_t)s * s));
        const bool ok = p >= 0 && a >= 0 && a < (int64_t)s * s * s && ax >= 3 && ax < s - 3 && ay >= 3 &&
                        ay < s - 3 && az >= 3 && az < s - 3;
        if (!ok) {
            for (int c = 0; c < (PSI4 ? 6 : 4); c++) out.p[c][n] = 0.0;
            continue;
        }
        const int N = s - 6;
        const int64_t q = (ax - 3) + (int64_t)N * ((ay - 3) + (int64_t)N * (az - 3));
        constraints_node<PSI4>(P, out, bd, q, 0, 0, 0, n);
    }
}

}  // namespace

// Per-CTA partial sums of c^2 and node counts over nodes outside both
// puncture radii, then one thread sums the partials in CTA order: a fixed
// grid and a fixed order, so the result is deterministic.
// mask (optional): only nodes with mask[node] != 0 count (the nodes one rank
// of a partition owns).
__global__ void __launch_bounds__(256) l2_partial_kernel(ConstVars C, int nc, int64_t n, int gx, int gy, double x0,
                                  double y0, double z0, double h, double b0, double b1, double b2,
                                  double b3, double b4, double b5, double r1, double r2,
                                  const uint8_t* __restrict__ mask, double* partial) {
    __shared__ double red[256][5];
    double acc[4] = {0, 0, 0, 0};
    double cnt = 0;
    for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n;
         node += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ix = node % gx, iy = (node / gx) % gy, iz = node / ((int64_t)gx * gy);
        // coordinates and distances rounded step by step (no contraction), so
        // a node at exactly the excision radius is classified as on the CPU
        const double x = __dadd_rn(x0, __dmul_rn((double)ix, h));
        const double y = __dadd_rn(y0, __dmul_rn((double)iy, h));
        const double z = __dadd_rn(z0, __dmul_rn((double)iz, h));
        auto dist = [](double ax, double ay, double az) {
            return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)), __dmul_rn(az, az)));
        };
        const double d1 = dist(__dsub_rn(x, b0), __dsub_rn(y, b1), __dsub_rn(z, b2));
        const double d2 = dist(__dsub_rn(x, b3), __dsub_rn(y, b4), __dsub_rn(z, b5));
        if (d1 < r1 || d2 < r2) continue;
        if (mask && !mask[node]) continue;
        for (int c = 0; c < nc; c++) {
            const double v = C.p[c][node];
            acc[c] += v * v;
        }
        cnt += 1.0;
    }
    for (int c = 0; c < 4; c++) red[threadIdx.x][c] = acc[c];
    red[threadIdx.x][4] = cnt;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 5; c++) red[threadIdx.x][c] += red[threadIdx.x + w][c];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 5; c++) partial[blockIdx.x * 5 + c] = red[0][c];
}

// sums: write the raw sums of squares (out[0..nc-1]) and the node count
// (out[4]) for a reduction over ranks instead of the norms
__global__ void l2_final_kernel(const double* partial, int nblocks, int nc, double* norms, bool sums) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < nblocks; b++)
        for (int c = 0; c < 5; c++) s[c] += partial[b * 5 + c];
    if (sums) {
        for (int c = 0; c < nc; c++) norms[c] = s[c];
        norms[4] = s[4];
        return;
    }
    for (int c = 0; c < nc; c++) norms[c] = s[4] > 0 ? sqrt(s[c] / s[4]) : 0.0;
}

int launch_constraints(const MeshState* m, const double* const* P, double* const* out,
                       cudaStream_t s, bool psi4) {
    ConstVars p;
    MutVars o = {};
    for (int v = 0; v < NVARS; v++) p.p[v] = P[v];
    for (int c = 0; c < (psi4 ? 6 : 4); c++) o.p[c] = out[c];
    if (m->lv) {
        const int nb = (int)m->blocks.size();
        const int64_t nn = m->lv->n_nodes;
        if (nb == 0 || nn == 0) return 0;
        const int grid = (int)std::min<int64_t>((nn + 255) / 256, 148 * 16);
        if (psi4)
            constraints_levels_kernel<true><<<grid, 256, 0, s>>>(p, o, m->d_blocks, nb, m->lv->zip_src, nn);
        else
            constraints_levels_kernel<false><<<grid, 256, 0, s>>>(p, o, m->d_blocks, nb, m->lv->zip_src, nn);
        return cuda_status(cudaGetLastError());
    }
    if (m->n_int_chunks == 0) return 0;
    if (psi4)
        constraints_kernel<true><<<m->n_int_chunks, 256, 0, s>>>(p, o, m->d_blocks, m->d_int_chunks,
                                                                  m->G[0], m->G[1], m->G[2]);
    else
        constraints_kernel<false><<<m->n_int_chunks, 256, 0, s>>>(p, o, m->d_blocks, m->d_int_chunks,
                                                                   m->G[0], m->G[1], m->G[2]);
    return cuda_status(cudaGetLastError());
}

int launch_l2_norms(const MeshState* m, const double* const* C, int nc, const double xmin[3],
                    double h, const double bh[6], const double radii[2], double* partial,
                    int npartial, double* norms, cudaStream_t s, const uint8_t* mask, bool sums) {
    if (nc < 1 || nc > 4 || npartial < 1) return BSSN_EINVAL;
    ConstVars c = {};
    for (int q = 0; q < nc; q++) c.p[q] = C[q];
    const int64_t n = (int64_t)m->G[0] * m->G[1] * m->G[2];
    l2_partial_kernel<<<npartial, 256, 0, s>>>(c, nc, n, m->G[0], m->G[1], xmin[0], xmin[1],
                                               xmin[2], h, bh[0], bh[1], bh[2], bh[3], bh[4],
                                               bh[5], radii[0], radii[1], mask, partial);
    l2_final_kernel<<<1, 32, 0, s>>>(partial, npartial, nc, norms, sums);
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
