// Single-level octree meshes of padded blocks: the device block table, the
// ghost-fill (unzip) and gather-back (zip) kernels, and the synthetic mesh
// generator.  These replace the parts of dendrolib's ot::Mesh that the BSSN
// evolution step calls (unzip/zip, call sites BSSN_GR/src/rkBSSN.cpp:611-650,
// bssnCtx.cpp:73,103); dendrolib itself is absent from the reference tree.
//
// Node grid: every block is an aligned cube of octants at one level; octant
// o covers nodes [6o, 6o+6] per axis, so the zipped vector of a variable is
// the G[0] x G[1] x G[2] node grid (G = 6*M + 1) and a padded point (i,j,k)
// of a block reads node g0 + (i,j,k) - 3.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bssn_common.cuh"
#include "kernels.cuh"
#include "mesh.h"

namespace bssn {
namespace {

constexpr int CHUNK = 1024;

// Ghost fill.  One CTA per chunk of consecutive padded points of one block:
// consecutive threads read consecutive nodes of a grid row and write
// consecutive padded points.
__global__ void __launch_bounds__(CHUNK) unzip_kernel(MutVars unz, ConstVars zip, int nvars,
                             const BssnBlockDesc* __restrict__ blocks,
                             const Chunk* __restrict__ chunks, int gx, int gy,
                             int gz) {
    const Chunk c = chunks[blockIdx.x];
    const BssnBlockDesc b = blocks[c.blk];
    const int s = b.sz;
    if (threadIdx.x >= c.count) return;
    const int p = (int)c.start + (int)threadIdx.x;  // < s^3, fits 32 bits
    const int i = p % s, j = (p / s) % s, k = p / (s * s);
    const int64_t x = b.g0[0] + i - 3, y = b.g0[1] + j - 3, z = b.g0[2] + k - 3;
    const bool in = x >= 0 && y >= 0 && z >= 0 && x < gx && y < gy && z < gz;
    const int64_t node = in ? x + (int64_t)gx * (y + (int64_t)gy * z) : 0;
    double* const* out = unz.p;
    if (nvars == NVARS) {  // every load in flight before the first store
        double v[NVARS];
#pragma unroll
        for (int q = 0; q < NVARS; q++) v[q] = in ? __ldg(zip.p[q] + node) : 0.0;
#pragma unroll
        for (int q = 0; q < NVARS; q++) out[q][b.offset + p] = v[q];
        return;
    }
    for (int v = 0; v < nvars; v++) out[v][b.offset + p] = in ? __ldg(zip.p[v] + node) : 0.0;
}

// Gather back.  Each interior node of a block is written only if the block
// owns it: a node on the block's upper face belongs to the next block unless
// the face lies on the grid's upper boundary.
__global__ void __launch_bounds__(CHUNK) zip_kernel(MutVars zip, ConstVars unz, int nvars,
                           const BssnBlockDesc* __restrict__ blocks,
                           const Chunk* __restrict__ chunks, int gx, int gy,
                           int gz) {
    const Chunk c = chunks[blockIdx.x];
    const BssnBlockDesc b = blocks[c.blk];
    const int s = b.sz, N = s - 6;
    if (threadIdx.x >= c.count) return;
    const int q = (int)c.start + (int)threadIdx.x;  // < N^3
    const int i = q % N, j = (q / N) % N, k = q / (N * N);
    const int64_t x = b.g0[0] + i, y = b.g0[1] + j, z = b.g0[2] + k;
    const bool own = (i < N - 1 || x == gx - 1) && (j < N - 1 || y == gy - 1) &&
                     (k < N - 1 || z == gz - 1);
    if (!own) return;
    const int64_t node = x + (int64_t)gx * (y + (int64_t)gy * z);
    const int64_t p = b.offset + (i + 3) + (int64_t)s * ((j + 3) + (int64_t)s * (k + 3));
    if (nvars == NVARS) {
        double v[NVARS];
#pragma unroll
        for (int w = 0; w < NVARS; w++) v[w] = __ldg(unz.p[w] + p);
#pragma unroll
        for (int w = 0; w < NVARS; w++) zip.p[w][node] = v[w];
        return;
    }
    for (int v = 0; v < nvars; v++) zip.p[v][node] = __ldg(unz.p[v] + p);
}

void make_chunks(const std::vector<BssnBlockDesc>& blocks, bool interior,
                 std::vector<Chunk>& out, int max_side = 1 << 30) {
    out.clear();
    for (size_t b = 0; b < blocks.size(); b++) {
        if (blocks[b].sz > max_side) continue;
        const int64_t s = interior ? blocks[b].sz - 6 : blocks[b].sz;
        const int64_t n = s * s * s;
        for (int64_t st = 0; st < n; st += CHUNK) {
            Chunk c;
            c.blk = (int32_t)b;
            c.count = (int32_t)std::min<int64_t>(CHUNK, n - st);
            c.start = st;
            out.push_back(c);
        }
    }
}

template <class T>
int upload(const std::vector<T>& h, T** d) {
    *d = nullptr;
    if (h.empty()) return 0;
    cudaError_t e = cudaMalloc((void**)d, h.size() * sizeof(T));
    if (e != cudaSuccess) return BSSN_ENOMEM;
    e = cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return cuda_status(e);
}

}  // namespace

int mesh_create(const BssnBlockDesc* blocks, int nblocks, const int32_t G[3],
                MeshState** out) {
    MeshState* m = new MeshState();
    m->blocks.assign(blocks, blocks + nblocks);
    for (int d = 0; d < 3; d++) m->G[d] = G[d];
    m->unzip_size = 0;
    for (int b = 0; b < nblocks; b++) {
        const int64_t s = blocks[b].sz;
        m->unzip_size = std::max<int64_t>(m->unzip_size, blocks[b].offset + s * s * s);
    }
    std::vector<Chunk> pad, inner, small;
    make_chunks(m->blocks, false, pad);
    make_chunks(m->blocks, true, inner);
    make_chunks(m->blocks, false, small, kDirectMinSide - 1);
    m->n_pad_chunks = (int)pad.size();
    m->n_int_chunks = (int)inner.size();
    m->n_pad_chunks_small = (int)small.size();
    int st = upload(m->blocks, &m->d_blocks);
    if (!st) st = upload(pad, &m->d_pad_chunks);
    if (!st) st = upload(inner, &m->d_int_chunks);
    if (!st) st = upload(small, &m->d_pad_chunks_small);
    if (st) {
        mesh_destroy(m);
        return st;
    }
    *out = m;
    return 0;
}

void mesh_destroy(MeshState* m) {
    if (!m) return;
    cudaFree(m->d_blocks);
    cudaFree(m->d_pad_chunks);
    cudaFree(m->d_pad_chunks_small);
    cudaFree(m->d_int_chunks);
    cudaFree(m->d_partial);
    cudaFree(m->d_elems);
    cudaFree(m->d_elem_first);
    cudaFree(m->d_fchunks);
    cudaFree(m->d_need_off);
    cudaFree(m->d_need_list);
    cudaFree(m->d_fchunk_first);
    cudaFree(m->d_fpart);
    for (auto& t : m->tasks) cudaFree(t.second.first);
    cudaFree(m->d_scratch);
    if (m->lv) {
        levels_free(m->lv);
        delete m->lv;
    }
    delete m;
}

int mesh_scratch(MeshState* m, int64_t zones) {
    if (zones > kSplitScratchZonesMax) zones = kSplitScratchZonesMax;
    if (zones <= m->scratch_zones) return 0;
    cudaFree(m->d_scratch);
    m->d_scratch = nullptr;
    m->scratch_zones = 0;
    if (cudaMalloc((void**)&m->d_scratch, sizeof(double) * kSplitSlots * zones) != cudaSuccess) {
        cudaGetLastError();
        return BSSN_ENOMEM;
    }
    m->scratch_zones = zones;
    return 0;
}

int64_t split_need(MeshState* m, int tile, int side) {
    if (tile_mode(tile) != 1) return 0;
    const BrickTask* tk;
    int nt = 0;
    if (mesh_tasks_side(m, tile, side, &tk, &nt)) return 0;
    const int64_t need = (int64_t)nt * tile_zones(tile);
    return need < kSplitScratchZonesMax ? need : kSplitScratchZonesMax;
}

namespace {
// Z-order (Morton) key of a block's first interior node in octant units
// (6 nodes per octant), 21 bits per axis: for the leaves of an octree this is
// the space-filling-curve order, so consecutive blocks are neighbours.
uint64_t morton_key(const BssnBlockDesc& b) {
    uint64_t k = 0;
    const uint64_t c[3] = {(uint64_t)(b.g0[0] / 6), (uint64_t)(b.g0[1] / 6), (uint64_t)(b.g0[2] / 6)};
    for (int bit = 20; bit >= 0; bit--)
        for (int d = 2; d >= 0; d--) k = (k << 1) | ((c[d] >> bit) & 1u);
    return k;
}
}  // namespace

int mesh_tasks_side(MeshState* m, int tile, int side, const BrickTask** tasks, int* ntasks) {
    const auto key = std::make_pair(tile, side);
    auto it = m->tasks.find(key);
    if (it == m->tasks.end()) {
        std::vector<BrickTask> all, h;
        build_tasks(m->blocks.data(), (int)m->blocks.size(), tile, all);
        for (auto& t : all)
            if (side <= 0 || m->blocks[t.blk].sz == side) h.push_back(t);
        if (side < 0) {  // all blocks, Z-order of their origins (bricks of a block stay together)
            std::stable_sort(h.begin(), h.end(), [&](const BrickTask& a, const BrickTask& b) {
                return morton_key(m->blocks[a.blk]) < morton_key(m->blocks[b.blk]);
            });
        }
        BrickTask* d = nullptr;
        int st = upload(h, &d);
        if (st) return st;
        it = m->tasks.emplace(key, std::make_pair(d, (int)h.size())).first;
    }
    *tasks = it->second.first;
    *ntasks = it->second.second;
    return 0;
}

// Split the blocks into nparts ranges of their Z-order (the order of their
// origins' Morton keys) holding about equal numbers of interior zones, as the
// reference partitions its octree along a space-filling curve.
int mesh_partition(const BssnBlockDesc* blocks, int nblocks, int nparts, int32_t* part) {
    if (!blocks || nblocks <= 0 || nparts <= 0 || !part) return BSSN_EINVAL;
    std::vector<int> order(nblocks);
    for (int b = 0; b < nblocks; b++) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return morton_key(blocks[a]) < morton_key(blocks[b]);
    });
    double total = 0;
    for (int b = 0; b < nblocks; b++) total += std::pow((double)(blocks[b].sz - 6), 3);
    double acc = 0;
    for (int i = 0; i < nblocks; i++) {
        const int b = order[i];
        const double z = std::pow((double)(blocks[b].sz - 6), 3);
        // the part holding this block's zone midpoint
        int r = (int)((acc + 0.5 * z) / total * nparts);
        part[b] = r < nparts ? r : nparts - 1;
        acc += z;
    }
    return 0;
}

int mesh_tasks(MeshState* m, int tile, const BrickTask** tasks, int* ntasks) {
    return mesh_tasks_side(m, tile, 0, tasks, ntasks);
}

int launch_unzip(const MeshState* m, double* const* unz, const double* const* zip,
                 int nvars, cudaStream_t s, bool small_only) {
    MutVars u = {};
    ConstVars z = {};
    for (int v = 0; v < nvars; v++) {
        u.p[v] = unz[v];
        z.p[v] = zip[v];
    }
    const int n = small_only ? m->n_pad_chunks_small : m->n_pad_chunks;
    if (n == 0) return 0;
    unzip_kernel<<<n, CHUNK, 0, s>>>(u, z, nvars, m->d_blocks,
                                     small_only ? m->d_pad_chunks_small : m->d_pad_chunks,
                                     m->G[0], m->G[1], m->G[2]);
    return cuda_status(cudaGetLastError());
}

namespace {
__global__ void __launch_bounds__(256) halo_pack_kernel(double* __restrict__ buf, ConstVars u,
                                                        const int64_t* __restrict__ idx, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t node = idx[i];
#pragma unroll
        for (int v = 0; v < NVARS; v++) buf[v * n + i] = __ldg(u.p[v] + node);
    }
}
__global__ void __launch_bounds__(256) halo_unpack_kernel(MutVars u, const double* __restrict__ buf,
                                                          const int64_t* __restrict__ idx, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t node = idx[i];
        double v[NVARS];
#pragma unroll
        for (int q = 0; q < NVARS; q++) v[q] = __ldg(buf + q * n + i);
#pragma unroll
        for (int q = 0; q < NVARS; q++) u.p[q][node] = v[q];
    }
}
int halo_grid(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}
}  // namespace

int launch_halo_pack(double* buf, const double* const* u, const int64_t* idx, int64_t n,
                     cudaStream_t s) {
    if (n <= 0) return 0;
    ConstVars cu;
    for (int v = 0; v < NVARS; v++) cu.p[v] = u[v];
    halo_pack_kernel<<<halo_grid(n), 256, 0, s>>>(buf, cu, idx, n);
    return cuda_status(cudaGetLastError());
}

int launch_halo_unpack(double* const* u, const double* buf, const int64_t* idx, int64_t n,
                       cudaStream_t s) {
    if (n <= 0) return 0;
    MutVars mu;
    for (int v = 0; v < NVARS; v++) mu.p[v] = u[v];
    halo_unpack_kernel<<<halo_grid(n), 256, 0, s>>>(mu, buf, idx, n);
    return cuda_status(cudaGetLastError());
}

int launch_zip(const MeshState* m, double* const* zip, const double* const* unz,
               int nvars, cudaStream_t s) {
    MutVars z = {};
    ConstVars u = {};
    for (int v = 0; v < nvars; v++) {
        z.p[v] = zip[v];
        u.p[v] = unz[v];
    }
    if (m->n_int_chunks == 0) return 0;
    zip_kernel<<<m->n_int_chunks, CHUNK, 0, s>>>(z, u, nvars, m->d_blocks, m->d_int_chunks,
                                                 m->G[0], m->G[1], m->G[2]);
    return cuda_status(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Synthetic mesh generator (host).
// ---------------------------------------------------------------------------
namespace {

struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Cube {
    int o[3];  // octant origin
    int w;     // octants per side (1, 2, 4, 8)
};

// Split a super-cell top-down.  q[w] = probability that a cell of width w
// stays one block.
void split_cell(const Cube& c, const double q[4], Rng& r, std::vector<Cube>& out) {
    const int lvl = c.w == 8 ? 3 : (c.w == 4 ? 2 : (c.w == 2 ? 1 : 0));
    if (c.w == 1 || r.uniform() < q[lvl]) {
        out.push_back(c);
        return;
    }
    const int h = c.w / 2;
    // Morton order of the children
    for (int m = 0; m < 8; m++) {
        Cube k{{c.o[0] + (m & 1) * h, c.o[1] + ((m >> 1) & 1) * h, c.o[2] + ((m >> 2) & 1) * h}, h};
        split_cell(k, q, r, out);
    }
}

}  // namespace

int mesh_generate(int mode, const int32_t dims[3], const double p[4], uint64_t seed,
                  double xmin, double L, BssnBlockDesc* blocks, int* nblocks,
                  int32_t G[3], double* h_out) {
    std::vector<Cube> cubes;
    int M[3];
    if (mode == 0) {
        const int n = dims[0];
        if (n < 1) return BSSN_EINVAL;
        M[0] = M[1] = M[2] = n;
        for (int z = 0; z < n; z++)
            for (int y = 0; y < n; y++)
                for (int x = 0; x < n; x++) cubes.push_back(Cube{{x, y, z}, 1});
    } else if (mode == 1) {
        for (int d = 0; d < 3; d++) {
            if (dims[d] < 1) return BSSN_EINVAL;
            M[d] = 8 * dims[d];
        }
        // Conditional "stay whole" probabilities from the target block-count
        // fractions p = {p13, p19, p31, p55}: with a = P(55 whole), b = P(31
        // whole | split), c = P(19 whole | split) the expected counts per
        // super-cell are a, 8(1-a)b, 64(1-a)(1-b)c, 512(1-a)(1-b)(1-c), so
        //   p31/p55 = 8b(1-a)/a, p19/p31 = 8c(1-b)/b, p13/p19 = 8(1-c)/c.
        if (p[0] <= 0 || p[1] <= 0 || p[2] <= 0 || p[3] <= 0) return BSSN_EINVAL;
        const double c = 8.0 / (8.0 + p[0] / p[1]);
        const double b = 8.0 * c / (8.0 * c + p[1] / p[2]);
        const double a = 8.0 * b / (8.0 * b + p[2] / p[3]);
        const double q[4] = {1.0, c, b, a};
        Rng r{seed};
        // super-cells in a seeded order over the box
        const int ns = dims[0] * dims[1] * dims[2];
        std::vector<int> perm(ns);
        for (int i = 0; i < ns; i++) perm[i] = i;
        for (int i = ns - 1; i > 0; i--) std::swap(perm[i], perm[(int)(r.next() % (uint64_t)(i + 1))]);
        for (int t = 0; t < ns; t++) {
            const int id = perm[t];
            const int sx = id % dims[0], sy = (id / dims[0]) % dims[1], sz = id / (dims[0] * dims[1]);
            split_cell(Cube{{8 * sx, 8 * sy, 8 * sz}, 8}, q, r, cubes);
        }
    } else {
        return BSSN_EINVAL;
    }
    const int n = (int)cubes.size();
    for (int d = 0; d < 3; d++) G[d] = 6 * M[d] + 1;
    const int Mmax = std::max(M[0], std::max(M[1], M[2]));
    const double octw = L / Mmax;
    const double h = octw / 6.0;
    *h_out = h;
    *nblocks = n;
    if (!blocks) return 0;
    int64_t off = 0;
    for (int b = 0; b < n; b++) {
        const Cube& c = cubes[b];
        BssnBlockDesc d;
        std::memset(&d, 0, sizeof(d));
        const int s = 6 * c.w + 7;
        d.offset = off;
        d.sz = s;
        d.bflag = 0;
        for (int k = 0; k < 3; k++) {
            d.g0[k] = 6 * c.o[k];
            if (c.o[k] == 0) d.bflag |= 1u << (2 * k);
            if (c.o[k] + c.w == M[k]) d.bflag |= 1u << (2 * k + 1);
            d.ptmin[k] = xmin + (double)(d.g0[k] - 3) * h;
            d.ptmax[k] = xmin + (double)(d.g0[k] - 3 + s - 1) * h;
        }
        d.level = c.w == 1 ? 3 : (c.w == 2 ? 2 : (c.w == 4 ? 1 : 0));
        blocks[b] = d;
        const int64_t npts = (int64_t)s * s * s;
        off += (npts + 1) / 2 * 2;
    }
    return 0;
}

}  // namespace bssn
