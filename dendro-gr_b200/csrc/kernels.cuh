// Launchers of the elementwise, stencil and mesh kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bssn {

struct MeshState;

int launch_stencil(int kind, double* D, const double* u, double h,
                   const unsigned sz[3], unsigned bflag, cudaStream_t s);
int launch_rk4_stage(int stage, double* const* out, const double* const* prev,
                     const double* const* k, int64_t n, double dt, int enforce,
                     double chi_floor, int* status, cudaStream_t s);
int launch_enforce(double* const* u, int64_t n, double chi_floor, int* status,
                   cudaStream_t s);
int launch_initial_data(double* const* u, const int32_t G[3], const double xmin[3],
                        double h, const double bh[6], double m1, double m2,
                        double chi_floor, double eps, uint64_t seed, cudaStream_t s);
// small_only: the blocks smaller than kDirectMinSide only
int launch_unzip(const MeshState* m, double* const* unz, const double* const* zip,
                 int nvars, cudaStream_t s, bool small_only = false);
int launch_zip(const MeshState* m, double* const* zip, const double* const* unz,
               int nvars, cudaStream_t s);
// halo exchange buffers: buf[v*n + i] = u[v][idx[i]] and back
int launch_halo_pack(double* buf, const double* const* u, const int64_t* idx, int64_t n,
                     cudaStream_t s);
int launch_halo_unpack(double* const* u, const double* buf, const int64_t* idx, int64_t n,
                       cudaStream_t s);
int launch_zip_stage(const MeshState* m, int stage, double* const* im, double* const* acc,
                     double* const* u, const double* const* R, double dt, int enforce,
                     double chi_floor, int* status, cudaStream_t s);
// the zip-stage algebra with R already on the zipped grid (n nodes)
int launch_node_stage(int stage, double* const* im, double* const* acc, double* const* u,
                      const double* const* R, int64_t n, double dt, int enforce,
                      double chi_floor, int* status, cudaStream_t s);

}  // namespace bssn
