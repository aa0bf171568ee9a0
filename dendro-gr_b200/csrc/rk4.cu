// RK4 stage updates, constraint enforcement and puncture initial data on
// zipped node vectors.  Memory-bound elementwise kernels; every product and
// sum is explicitly rounded in the reference's order so the stage algebra is
// bit-identical to the CPU restatement (BSSN_GR/src/rkBSSN.cpp:764-860).
#include <cuda_runtime.h>

#include "bssn_common.cuh"
#include "kernels.cuh"
#include "rk4_stage.cuh"
#include "mesh.h"

namespace bssn {
namespace {

struct KPtrs { const double* p[4 * NVARS]; };

__global__ void __launch_bounds__(256) rk4_stage_kernel(int stage, MutVars out, ConstVars prev, KPtrs k,
                                 int64_t n, double dt, int enforce,
                                 double chi_floor, int* status) {
    int bad = 0;
    for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n;
         node += (int64_t)gridDim.x * blockDim.x) {
        double v[NVARS];
        if (stage < 3) {
            const double c = M_(kRK4_U[stage + 1], dt);
#pragma unroll
            for (int q = 0; q < NVARS; q++) v[q] = A_(prev.p[q][node], M_(c, k.p[q][node]));
        } else {
#pragma unroll
            for (int q = 0; q < NVARS; q++) {
                double t = prev.p[q][node];
#pragma unroll
                for (int s = 0; s < 4; s++) t = A_(t, M_(M_(kRK4_C[s], dt), k.p[s * NVARS + q][node]));
                v[q] = t;
            }
        }
        if (enforce) bad += enforce_regs(v, chi_floor);
#pragma unroll
        for (int q = 0; q < NVARS; q++) out.p[q][node] = v[q];
    }
    if (status && bad) atomicAdd(status, bad);
}

__global__ void __launch_bounds__(256) enforce_kernel(MutVars u, int64_t n, double chi_floor, int* status) {
    int bad = 0;
    for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n;
         node += (int64_t)gridDim.x * blockDim.x) {
        double v[NVARS];
#pragma unroll
        for (int q = 0; q < NVARS; q++) v[q] = u.p[q][node];
        bad += enforce_regs(v, chi_floor);
#pragma unroll
        for (int q = 0; q < NVARS; q++) u.p[q][node] = v[q];
    }
    if (status && bad) atomicAdd(status, bad);
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Brill-Lindquist data with zero momenta and spins
// (BSSN_GR/src/grUtils.cpp:1033-1035, 1082-1100), then a seeded uniform
// perturbation and enforcement.
__global__ void __launch_bounds__(256) initial_data_kernel(MutVars u, int gx, int gy, int gz, double x0,
                                    double y0, double z0, double h, double b0,
                                    double b1, double b2, double b3, double b4,
                                    double b5, double m1, double m2,
                                    double chi_floor, double eps, uint64_t seed) {
    const int64_t N = (int64_t)gx * gy * gz;
    for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < N;
         node += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ix = node % gx, iy = (node / gx) % gy, iz = node / ((int64_t)gx * gy);
        const double x = A_(x0, M_((double)ix, h)), y = A_(y0, M_((double)iy, h)),
                     z = A_(z0, M_((double)iz, h));
        const double x1 = S_(x, b0), y1 = S_(y, b1), z1 = S_(z, b2);
        const double x2 = S_(x, b3), y2 = S_(y, b4), z2 = S_(z, b5);
        const double rv1 = __dsqrt_rn(A_(A_(M_(x1, x1), M_(y1, y1)), M_(z1, z1)));
        const double rv2 = __dsqrt_rn(A_(A_(M_(x2, x2), M_(y2, y2)), M_(z2, z2)));
        double psi = A_(1.0, __ddiv_rn(m1, M_(2.0, rv1)));
        psi = A_(psi, __ddiv_rn(m2, M_(2.0, rv2)));
        double v[NVARS];
#pragma unroll
        for (int q = 0; q < NVARS; q++) v[q] = 0.0;
        v[U_ALPHA] = fmax(__ddiv_rn(1.0, M_(psi, psi)), chi_floor);
        v[U_CHI] = __ddiv_rn(1.0, pow(psi, 4.0));
        if (v[U_CHI] < chi_floor) v[U_CHI] = chi_floor;
        v[U_SYMGT0] = v[U_SYMGT3] = v[U_SYMGT5] = 1.0;
#pragma unroll
        for (int q = 0; q < NVARS; q++) {
            const uint64_t r = mix64(seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(q * N + node + 1));
            const double unit = M_((double)(r >> 11), 1.0 / 9007199254740992.0);
            v[q] = A_(v[q], M_(eps, S_(M_(2.0, unit), 1.0)));
        }
        enforce_regs(v, chi_floor);
#pragma unroll
        for (int q = 0; q < NVARS; q++) u.p[q][node] = v[q];
    }
}

// Zip fused with the RK4 stage algebra: every node owned by a block takes
// its right-hand side k from the block's padded output R and updates the
// stage state (stage 0..2) or the final state (stage 3):
//   stage s < 3:  im  = u + RK4_U[s+1]*dt*k   (then enforce, optional)
//                 acc = (s == 0 ? u : acc) + RK4_C[s]*dt*k
//   stage 3:      u   = acc + RK4_C[3]*dt*k   (then enforce)
// The accumulation order equals rkBSSN.cpp:851-858 term by term.
__global__ void __launch_bounds__(256) zip_stage_kernel(int stage, MutVars im, MutVars acc, MutVars u,
                                 ConstVars R, const BssnBlockDesc* __restrict__ blocks,
                                 const Chunk* __restrict__ chunks, int gx, int gy, int gz,
                                 double dt, int enforce, double chi_floor, int* status) {
    const Chunk c = chunks[blockIdx.x];
    const BssnBlockDesc b = blocks[c.blk];
    const int s = b.sz, N = s - 6;
    int bad = 0;
    for (int r = threadIdx.x; r < c.count; r += blockDim.x) {
        const int q = (int)c.start + r;  // < N^3, fits 32 bits
        const int i = q % N, j = (q / N) % N, k = q / (N * N);
        const int64_t x = b.g0[0] + i, y = b.g0[1] + j, z = b.g0[2] + k;
        const bool own = (i < N - 1 || x == gx - 1) && (j < N - 1 || y == gy - 1) &&
                         (k < N - 1 || z == gz - 1);
        if (own) {
            const int64_t node = x + (int64_t)gx * (y + (int64_t)gy * z);
            const int64_t p = b.offset + (i + 3) + (int64_t)s * ((j + 3) + (int64_t)s * (k + 3));
            double v[NVARS];
            if (stage < 3) {
                const double cu = M_(kRK4_U[stage + 1], dt);
                const double cc = M_(kRK4_C[stage], dt);
                // all loads before the first store (the pointer arrays may alias)
                double kk[NVARS], a0[NVARS];
#pragma unroll
                for (int q2 = 0; q2 < NVARS; q2++) {
                    kk[q2] = __ldg(R.p[q2] + p);
                    v[q2] = u.p[q2][node];
                    a0[q2] = stage == 0 ? v[q2] : acc.p[q2][node];
                }
#pragma unroll
                for (int q2 = 0; q2 < NVARS; q2++) {
                    acc.p[q2][node] = A_(a0[q2], M_(cc, kk[q2]));
                    v[q2] = A_(v[q2], M_(cu, kk[q2]));
                }
                if (enforce) bad += enforce_regs(v, chi_floor);
#pragma unroll
                for (int q2 = 0; q2 < NVARS; q2++) im.p[q2][node] = v[q2];
            } else {
                const double cc = M_(kRK4_C[3], dt);
#pragma unroll
                for (int q2 = 0; q2 < NVARS; q2++)
                    v[q2] = A_(acc.p[q2][node], M_(cc, __ldg(R.p[q2] + p)));
                bad += enforce_regs(v, chi_floor);
#pragma unroll
                for (int q2 = 0; q2 < NVARS; q2++) u.p[q2][node] = v[q2];
            }
        }
    }
    if (status && bad) atomicAdd(status, bad);
}

// The same stage algebra on the zipped node grid, with the right-hand side
// already zipped (written once per node by the block owning it): one thread
// per node, every access coalesced.
__global__ void __launch_bounds__(256) node_stage_kernel(int stage, MutVars im, MutVars acc, MutVars u,
                                  ConstVars R, int64_t n, double dt, int enforce,
                                  double chi_floor, int* status) {
    int bad = 0;
    for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n;
         node += (int64_t)gridDim.x * blockDim.x) {
        double k[NVARS], v[NVARS], a[NVARS];
#pragma unroll
        for (int q = 0; q < NVARS; q++) {  // every load before the first store
            k[q] = __ldg(R.p[q] + node);
            v[q] = stage < 3 ? u.p[q][node] : 0.0;
            a[q] = stage > 0 ? acc.p[q][node] : 0.0;
        }
        bad += stage_node(stage, dt, k, v, a, enforce, chi_floor);
#pragma unroll
        for (int q = 0; q < NVARS; q++) {
            if (stage < 3) {
                acc.p[q][node] = a[q];
                im.p[q][node] = v[q];
            } else {
                u.p[q][node] = v[q];
            }
        }
    }
    if (status && bad) atomicAdd(status, bad);
}

int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 64) b = 148 * 64;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

int launch_rk4_stage(int stage, double* const* out, const double* const* prev,
                     const double* const* k, int64_t n, double dt, int enforce,
                     double chi_floor, int* status, cudaStream_t s) {
    MutVars o;
    ConstVars p;
    KPtrs kk = {};
    for (int q = 0; q < NVARS; q++) {
        o.p[q] = out[q];
        p.p[q] = prev[q];
    }
    const int nk = stage < 3 ? NVARS : 4 * NVARS;
    for (int q = 0; q < nk; q++) kk.p[q] = k[q];
    rk4_stage_kernel<<<grid_for(n, 256), 256, 0, s>>>(stage, o, p, kk, n, dt, enforce, chi_floor, status);
    return cuda_status(cudaGetLastError());
}

int launch_enforce(double* const* u, int64_t n, double chi_floor, int* status,
                   cudaStream_t s) {
    MutVars o;
    for (int q = 0; q < NVARS; q++) o.p[q] = u[q];
    enforce_kernel<<<grid_for(n, 256), 256, 0, s>>>(o, n, chi_floor, status);
    return cuda_status(cudaGetLastError());
}

int launch_initial_data(double* const* u, const int32_t G[3], const double xmin[3],
                        double h, const double bh[6], double m1, double m2,
                        double chi_floor, double eps, uint64_t seed, cudaStream_t s) {
    MutVars o;
    for (int q = 0; q < NVARS; q++) o.p[q] = u[q];
    const int64_t n = (int64_t)G[0] * G[1] * G[2];
    initial_data_kernel<<<grid_for(n, 256), 256, 0, s>>>(
        o, G[0], G[1], G[2], xmin[0], xmin[1], xmin[2], h, bh[0], bh[1], bh[2],
        bh[3], bh[4], bh[5], m1, m2, chi_floor, eps, seed);
    return cuda_status(cudaGetLastError());
}

int launch_zip_stage(const MeshState* m, int stage, double* const* im, double* const* acc,
                     double* const* u, const double* const* R, double dt, int enforce,
                     double chi_floor, int* status, cudaStream_t s) {
    MutVars I, Ac, U;
    ConstVars Rr;
    for (int q = 0; q < NVARS; q++) {
        I.p[q] = im[q];
        Ac.p[q] = acc[q];
        U.p[q] = u[q];
        Rr.p[q] = R[q];
    }
    if (m->n_int_chunks == 0) return 0;
    zip_stage_kernel<<<m->n_int_chunks, 256, 0, s>>>(stage, I, Ac, U, Rr, m->d_blocks,
                                                      m->d_int_chunks, m->G[0], m->G[1],
                                                      m->G[2], dt, enforce, chi_floor, status);
    return cuda_status(cudaGetLastError());
}

int launch_node_stage(int stage, double* const* im, double* const* acc, double* const* u,
                      const double* const* R, int64_t n, double dt, int enforce,
                      double chi_floor, int* status, cudaStream_t s) {
    MutVars I, Ac, U;
    ConstVars Rr;
    for (int q = 0; q < NVARS; q++) {
        I.p[q] = im[q];
        Ac.p[q] = acc[q];
        U.p[q] = u[q];
        Rr.p[q] = R[q];
    }
    if (n <= 0) return 0;
    node_stage_kernel<<<grid_for(n, 256), 256, 0, s>>>(stage, I, Ac, U, Rr, n, dt, enforce,
                                                       chi_floor, status);
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
