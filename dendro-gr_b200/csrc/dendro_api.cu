// Host-array drop-ins for the reference's C++ call surface
// (include/bssn_b200_dendro.hpp).  Each call stages the caller's host arrays
// through per-thread device buffers, runs the C ABI kernels and copies the
// written points back, synchronously on a per-thread stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "bssn_b200.h"
#include "bssn_b200_dendro.hpp"
#include "bssn_common.cuh"

namespace dendro_b200 {
namespace {

struct Staging {
    double* buf = nullptr;
    size_t cap = 0;  // doubles
    cudaStream_t stream = nullptr;
    ~Staging() {
        if (buf) cudaFree(buf);
        if (stream) cudaStreamDestroy(stream);
    }
    int reserve(size_t n) {
        if (!stream && cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
            return BSSN_ENOMEM;
        if (n <= cap) return 0;
        if (buf) cudaFree(buf);
        buf = nullptr;
        cap = 0;
        if (cudaMalloc((void**)&buf, n * sizeof(double)) != cudaSuccess) return BSSN_ENOMEM;
        cap = n;
        return 0;
    }
};

thread_local Staging tls;

int st(cudaError_t e) { return bssn::cuda_status(e); }

int stencil_host(int kind, double* D, const double* u, double h, const unsigned* sz,
                 unsigned bflag) {
    if (!D || !u || !sz) return BSSN_EINVAL;
    const size_t n = (size_t)sz[0] * sz[1] * sz[2];
    int r = tls.reserve(2 * n);
    if (r) return r;
    double* du = tls.buf;
    double* dD = tls.buf + n;
    cudaStream_t s = tls.stream;
    // D is copied in too, so points the stencil does not write keep their values
    if ((r = st(cudaMemcpyAsync(du, u, n * 8, cudaMemcpyHostToDevice, s)))) return r;
    if ((r = st(cudaMemcpyAsync(dD, D, n * 8, cudaMemcpyHostToDevice, s)))) return r;
    if ((r = bssn_deriv644_f64(kind, dD, du, h, sz, bflag, (bssn_stream_t)s))) return r;
    if ((r = st(cudaMemcpyAsync(D, dD, n * 8, cudaMemcpyDeviceToHost, s)))) return r;
    return st(cudaStreamSynchronize(s));
}

}  // namespace

int deriv644_x(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(0, D, u, h, sz, b); }
int deriv644_y(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(1, D, u, h, sz, b); }
int deriv644_z(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(2, D, u, h, sz, b); }
int deriv644_xx(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(3, D, u, h, sz, b); }
int deriv644_yy(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(4, D, u, h, sz, b); }
int deriv644_zz(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(5, D, u, h, sz, b); }
int ko_deriv42_x(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(6, D, u, h, sz, b); }
int ko_deriv42_y(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(7, D, u, h, sz, b); }
int ko_deriv42_z(double* D, const double* u, double h, const unsigned* sz, unsigned b) { return stencil_host(8, D, u, h, sz, b); }
int deriv644adv_x(double* D, const double* u, double h, const unsigned* sz, const double*, unsigned b) { return stencil_host(0, D, u, h, sz, b); }
int deriv644adv_y(double* D, const double* u, double h, const unsigned* sz, const double*, unsigned b) { return stencil_host(1, D, u, h, sz, b); }
int deriv644adv_z(double* D, const double* u, double h, const unsigned* sz, const double*, unsigned b) { return stencil_host(2, D, u, h, sz, b); }

int bssnrhs(double** rhs, const double** u, const unsigned& offset, const double* pmin,
            const double* pmax, const unsigned* sz, const unsigned& bflag,
            const BssnParams& params, double, const double**) {
    if (!rhs || !u || !sz) return BSSN_EINVAL;
    const size_t n = (size_t)sz[0] * sz[1] * sz[2];
    int r = tls.reserve(2 * bssn::NVARS * n);
    if (r) return r;
    cudaStream_t s = tls.stream;
    double* du[bssn::NVARS];
    double* dr[bssn::NVARS];
    for (int v = 0; v < bssn::NVARS; v++) {
        du[v] = tls.buf + v * n;
        dr[v] = tls.buf + (bssn::NVARS + v) * n;
        if ((r = st(cudaMemcpyAsync(du[v], u[v] + offset, n * 8, cudaMemcpyHostToDevice, s)))) return r;
        if ((r = st(cudaMemcpyAsync(dr[v], rhs[v] + offset, n * 8, cudaMemcpyHostToDevice, s)))) return r;
    }
    if ((r = bssn_bssnrhs_f64(dr, du, 0, pmin, pmax, sz, bflag, &params, (bssn_stream_t)s))) return r;
    for (int v = 0; v < bssn::NVARS; v++)
        if ((r = st(cudaMemcpyAsync(rhs[v] + offset, dr[v], n * 8, cudaMemcpyDeviceToHost, s)))) return r;
    return st(cudaStreamSynchronize(s));
}

int bssnRHS(double** rhs, const double** u, const Block* blk, unsigned nblk,
            const BssnParams& params, double, const double**) {
    if (!rhs || !u || !blk || nblk == 0) return BSSN_EINVAL;
    std::vector<BssnBlockDesc> d(nblk);
    size_t n = 0;
    for (unsigned b = 0; b < nblk; b++) {
        if (blk[b].sz[0] != blk[b].sz[1] || blk[b].sz[1] != blk[b].sz[2]) return BSSN_EBLOCKSIZE;
        std::memset(&d[b], 0, sizeof(BssnBlockDesc));
        d[b].offset = blk[b].offset;
        d[b].sz = (int32_t)blk[b].sz[0];
        d[b].bflag = blk[b].bflag;
        for (int k = 0; k < 3; k++) {
            d[b].ptmin[k] = blk[b].ptmin[k];
            d[b].ptmax[k] = blk[b].ptmax[k];
        }
        n = std::max(n, (size_t)blk[b].offset + (size_t)blk[b].sz[0] * blk[b].sz[1] * blk[b].sz[2]);
    }
    const int32_t G[3] = {1, 1, 1};
    bssn_mesh mesh = nullptr;
    int r = bssn_mesh_create(d.data(), (int)nblk, G, &mesh);
    if (r) return r;
    r = tls.reserve(2 * bssn::NVARS * n);
    cudaStream_t s = tls.stream;
    double* du[bssn::NVARS];
    double* dr[bssn::NVARS];
    for (int v = 0; v < bssn::NVARS && !r; v++) {
        du[v] = tls.buf + v * n;
        dr[v] = tls.buf + (bssn::NVARS + v) * n;
        r = st(cudaMemcpyAsync(du[v], u[v], n * 8, cudaMemcpyHostToDevice, s));
        if (!r) r = st(cudaMemcpyAsync(dr[v], rhs[v], n * 8, cudaMemcpyHostToDevice, s));
    }
    if (!r) r = bssn_rhs_blocks_f64(mesh, dr, du, &params, -1, (bssn_stream_t)s);
    for (int v = 0; v < bssn::NVARS && !r; v++)
        r = st(cudaMemcpyAsync(rhs[v], dr[v], n * 8, cudaMemcpyDeviceToHost, s));
    if (!r) r = st(cudaStreamSynchronize(s));
    bssn_mesh_destroy(mesh);
    return r;
}

int enforce_bssn_constraints(double** u, unsigned begin, unsigned end, double chi_floor) {
    if (!u || end < begin) return BSSN_EINVAL;
    const size_t n = end - begin;
    if (n == 0) return 0;
    int r = tls.reserve(bssn::NVARS * n + 1);
    if (r) return r;
    cudaStream_t s = tls.stream;
    double* du[bssn::NVARS];
    int* status = reinterpret_cast<int*>(tls.buf + bssn::NVARS * n);
    if ((r = st(cudaMemsetAsync(status, 0, sizeof(int), s)))) return r;
    for (int v = 0; v < bssn::NVARS; v++) {
        du[v] = tls.buf + v * n;
        if ((r = st(cudaMemcpyAsync(du[v], u[v] + begin, n * 8, cudaMemcpyHostToDevice, s)))) return r;
    }
    if ((r = bssn_enforce_f64(du, (int64_t)n, chi_floor, status, (bssn_stream_t)s))) return r;
    for (int v = 0; v < bssn::NVARS; v++)
        if ((r = st(cudaMemcpyAsync(u[v] + begin, du[v], n * 8, cudaMemcpyDeviceToHost, s)))) return r;
    int bad = 0;
    if ((r = st(cudaMemcpyAsync(&bad, status, sizeof(int), cudaMemcpyDeviceToHost, s)))) return r;
    if ((r = st(cudaStreamSynchronize(s)))) return r;
    return -bad;
}

// ---- reference-signature forms ---------------------------------------------
namespace {
std::mutex g_cfg_mu;
BssnParams g_params = {0.4, {1, 1, 1, 1}, {1.0, 0.0}, 2.0, 2.0, 40.0, 0, 0.99, 0.3, 1e-4};
Domain g_domain = {{-1.0, -1.0, -1.0}, {1.0, 1.0, 1.0}, {0u, 0u, 0u}, {1u, 1u, 1u}};
thread_local int t_last_status = 0;
}  // namespace

void set_params(const BssnParams& p) {
    std::lock_guard<std::mutex> lock(g_cfg_mu);
    g_params = p;
}
BssnParams get_params() {
    std::lock_guard<std::mutex> lock(g_cfg_mu);
    return g_params;
}
void set_domain(const Domain& d) {
    std::lock_guard<std::mutex> lock(g_cfg_mu);
    g_domain = d;
}
Domain get_domain() {
    std::lock_guard<std::mutex> lock(g_cfg_mu);
    return g_domain;
}
int last_status() { return t_last_status; }
void set_last_status(int status) { t_last_status = status; }

void bssnrhs(double** rhs, const double** u, const unsigned int& offset, const double* ptmin,
             const double* ptmax, const unsigned int* sz, const unsigned int& bflag, const double t,
             const double** cons) {
    t_last_status = bssnrhs(rhs, u, offset, ptmin, ptmax, sz, bflag, get_params(), t, cons);
}

void enforce_bssn_constraints(double** u, unsigned int node) {
    t_last_status = enforce_bssn_constraints(u, node, node + 1, get_params().chi_floor);
}

}  // namespace dendro_b200
