// Stand-alone finite-difference stencils on one padded block, bit-identical
// to the reference CPU functions: every product and sum is issued as an
// explicitly rounded operation in the reference's left-to-right order, so no
// multiply-add contraction can change a bit.
//
//   deriv644_{x,y,z}   BSSN_GR/src/derivs.cpp:2619-2947
//   deriv644_{xx,yy,zz}                    :2948-3312
//   ko_deriv42_{x,y,z}                     :964-1305
//
// Loop ranges are the reference's: d/dx over all j,k, d/dy over all k, every
// other stencil over the interior only.
#include <cuda_runtime.h>

#include "bssn_common.cuh"
#include "kernels.cuh"
#include "stencil_exact.cuh"

namespace bssn {
namespace {

__global__ void __launch_bounds__(256) stencil_kernel(int kind, double* __restrict__ D,
                               const double* __restrict__ u, AxisCoef cf,
                               int nx, int ny, int nz, unsigned bflag) {
    const int dir = kind % 3;
    const int fam = kind / 3;  // 0 first, 1 second, 2 KO
    int lo[3] = {3, 3, 3}, hi[3] = {nx - 3, ny - 3, nz - 3};
    if (fam == 0 && dir == 0) { lo[1] = 0; hi[1] = ny; lo[2] = 0; hi[2] = nz; }
    if (fam == 0 && dir == 1) { lo[2] = 0; hi[2] = nz; }
    const int rx = hi[0] - lo[0], ry = hi[1] - lo[1], rz = hi[2] - lo[2];
    const int64_t total = (int64_t)rx * ry * rz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int i = lo[0] + (int)(q % rx);
        const int j = lo[1] + (int)((q / rx) % ry);
        const int k = lo[2] + (int)(q / ((int64_t)rx * ry));
        const int c3[3] = {i, j, k};
        const int a = c3[dir];
        const int st = dir == 0 ? 1 : (dir == 1 ? nx : nx * ny);
        const int pp = i + nx * (j + ny * k);
        const int base = pp - a * st;
        const int N = dir == 0 ? nx : (dir == 1 ? ny : nz);
        const bool blo = bflag & (1u << (2 * dir)), bhi = bflag & (1u << (2 * dir + 1));
        const double* p0 = u + base;
        double r;
        if (fam == 0) r = ex::d1(p0, st, a, N, blo, bhi, cf);
        else if (fam == 1) r = ex::d2(p0, st, a, N, blo, bhi, cf);
        else r = ex::ko(p0, st, a, N, blo, bhi, cf);
        D[pp] = r;
    }
}

}  // namespace

int launch_stencil(int kind, double* D, const double* u, double h,
                   const unsigned sz[3], unsigned bflag, cudaStream_t s) {
    const int nx = sz[0], ny = sz[1], nz = sz[2];
    const int64_t n = (int64_t)nx * ny * nz;
    const int threads = 256;
    const int blocks = (int)((n + threads - 1) / threads);
    stencil_kernel<<<blocks < 1 ? 1 : blocks, threads, 0, s>>>(kind, D, u, axis_coef(h), nx, ny, nz, bflag);
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
