// Fused BSSN right-hand side on padded octree blocks (sm_100a, FP64).
//
// One CTA owns a brick of at most BX*BY*BZ interior zones of one block (one
// thread per zone).  The 24 evolved variables stream through a double-
// buffered shared-memory tile (brick + 3-point halo) filled with cp.async;
// every derivative a zone needs is formed from that tile in registers and
// folded into the equations at once (rhs_equations.cuh), so the 138
// derivatives and 72 dissipation terms never reach HBM.
//
// This file also holds the tile table shared with the split path
// (rhs_split.cu), the launchers and the host replay of the shared-memory
// indexing.
#include <cuda_runtime.h>

#include <cstdio>

#include "bssn_common.cuh"
#include "rhs_brick.cuh"
#include "rhs_equations.cuh"
#include "rhs_fused.cuh"

namespace bssn {

namespace {

template <int BX, int BY, int BZ>
__device__ __forceinline__ void rhs_brick(const RhsArgs& A, const BssnBlockDesc& blk,
                                          const int o[3], const int e[3],
                                          double* smem) {
    using Bk = Brick<BX, BY, BZ>;
    double* tiles[2] = {smem, smem + Bk::TILE};
    double* mxj = smem + 2 * Bk::TILE;   // [BZ][TY][BX]
    double* mxk = mxj + Bk::MXJ;         // [TZ][BY][BX]
    double* myk = mxk + Bk::MXK;         // [TZ][BY][BX]
    const int tid = threadIdx.x;
    const int s = blk.sz;
    const int64_t off = blk.offset;
    __shared__ AxisCoef cfs[3];
    fill_axis_coefs(cfs, blk, tid);  // visible after the first get()'s barrier
    const BrickThread<Bk> th(tid, e);
    const BrickZone<Bk> bz(blk, o, th, cfs);

    int step = 0;
    stage_var<Bk>(A.u.p[stage_order(0)] + off, tiles[0], o, e, s, tid);
    // n-th call: wait for the tile of stage_order(n), start the next load,
    // run the mixed pass for variables with second derivatives, then form
    // the zone's derivatives from the tile
    auto get = [&](auto tag, double* d1, double* d2, double& ko) {
        constexpr bool SECOND = decltype(tag)::value;
        cp_async_wait_all();
        __syncthreads();
        const double* cur = tiles[step & 1];
        if (step + 1 < NVARS)
            stage_var<Bk>(A.u.p[stage_order(step + 1)] + off, tiles[(step + 1) & 1], o, e, s, tid);
        if (SECOND) {
            mixed_pass<Bk>(cur, mxj, mxk, myk, o, e, s, blk.bflag, bz.zc.cf, tid);
            __syncthreads();
        }
        step++;
        zone_derivs<SECOND>(bz.zc, cur, mxj + bz.mxj_off, mxk + bz.mxk_off, myk + bz.mxk_off,
                            bz.mj, bz.mk, d1, d2, ko);
    };
    const int64_t pidx = off + bz.zc.a[0] + (int64_t)s * (bz.zc.a[1] + (int64_t)s * bz.zc.a[2]);
    auto pv = [&](int v) { return __ldg(A.u.p[v] + pidx); };
    const bool active = th.active;
    auto store = [&](int v, double r) {
        if (active) A.rhs.p[v][pidx] = r;
    };
    zone_equations(A, blk, bz.zc.a[0], bz.zc.a[1], bz.zc.a[2], get, pv, store);
}

}  // namespace

// One brick per CTA: from the task list, or (tasks == nullptr) from
// blockIdx.x over the bricks of the single block passed by value.
template <int BX, int BY, int BZ, int MINB>
__global__ void __launch_bounds__(Brick<BX, BY, BZ>::THREADS, MINB)
rhs_kernel(RhsArgs A, const BssnBlockDesc* __restrict__ blocks,
           const BrickTask* __restrict__ tasks, BssnBlockDesc single) {
    extern __shared__ __align__(16) double smem[];
    int o[3], e[3];
    if (tasks != nullptr) {
        const BrickTask tk = tasks[blockIdx.x];
        const BssnBlockDesc blk = blocks[tk.blk];
        o[0] = tk.o[0]; o[1] = tk.o[1]; o[2] = tk.o[2];
        e[0] = tk.e[0]; e[1] = tk.e[1]; e[2] = tk.e[2];
        rhs_brick<BX, BY, BZ>(A, blk, o, e, smem);
    } else {
        const int n = single.sz - 2 * PW;
        const int nbx = (n + BX - 1) / BX, nby = (n + BY - 1) / BY;
        const int q = blockIdx.x;
        const int qx = q % nbx, qy = (q / nbx) % nby, qz = q / (nbx * nby);
        split1(n, BX, qx, o[0], e[0]);
        split1(n, BY, qy, o[1], e[1]);
        split1(n, BZ, qz, o[2], e[2]);
        rhs_brick<BX, BY, BZ>(A, single, o, e, smem);
    }
}

// ---------------------------------------------------------------------------
// Tile table and launchers.
// ---------------------------------------------------------------------------
namespace {
struct TileEntry {
    int bx, by, bz, threads;
    size_t smem;
    void (*kern)(RhsArgs, const BssnBlockDesc*, const BrickTask*, BssnBlockDesc);
    int mode;   // 0 fused, 1 split
    int shape;  // index among the split shapes (split tiles)
    int fused;  // tile id of the same shape run fused
};

template <int BX, int BY, int BZ>
TileEntry make_fused(int id) {
    using Bk = Brick<BX, BY, BZ>;
    return TileEntry{BX, BY, BZ, Bk::THREADS, Bk::SMEM_BYTES, rhs_kernel<BX, BY, BZ, 1>, 0, -1, id};
}
template <int BX, int BY, int BZ>
TileEntry make_split_tile(int shape, int fused) {
    using Bk = Brick<BX, BY, BZ>;
    return TileEntry{BX, BY, BZ, Bk::THREADS, Bk::SMEM_BYTES, nullptr, 1, shape, fused};
}
template <int BX, int BY, int BZ>
TileEntry make_onchip_tile(int shape) {
    using Bk = Brick<BX, BY, BZ>;
    return TileEntry{BX, BY, BZ, Bk::THREADS, 0, nullptr, 2, shape, -1};
}

// tiles 0..2: fused; 3..5: the same shapes split; 6..9: split-only shapes
// (13x5x5 and 9x9x5 fit the 25-zone interiors of 31^3 blocks with few idle
// threads); 10..13: on chip (128-zone bricks, every extent >= 3 for every
// block side, as the one-sided closures need; 10, 11 at two CTAs per SM,
// 12, 13 the same shapes at three)
// (rhs_split.cu's shape order).  `fused` is the tile a single-block launch
// of the shape runs (the nearest fused shape for split-only ones).
const TileEntry* tile_table(int* count) {
    static const TileEntry table[] = {
        make_fused<8, 8, 4>(0),
        make_fused<7, 7, 4>(1),
        make_fused<8, 4, 4>(2),
        make_split_tile<8, 8, 4>(0, 0),
        make_split_tile<7, 7, 4>(1, 1),
        make_split_tile<8, 4, 4>(2, 2),
        make_split_tile<7, 7, 7>(3, 1),
        make_split_tile<8, 8, 8>(4, 0),
        make_split_tile<13, 5, 5>(5, 1),
        make_split_tile<9, 9, 5>(6, 1),
        make_onchip_tile<5, 5, 5>(0),
        make_onchip_tile<7, 4, 4>(1),
        make_onchip_tile<5, 5, 5>(2),
        make_onchip_tile<7, 4, 4>(3),
    };
    *count = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

int prepare(const TileEntry& t) {
    if (t.mode == 1) return prepare_split(t.shape);
    if (t.mode == 2) return prepare_onchip(t.shape);
    return set_smem_limit((const void*)t.kern, (int)t.smem);
}
}  // namespace

int prepare_all_tiles() {
    int c;
    const TileEntry* tab = tile_table(&c);
    for (int t = 0; t < c; t++) {
        int st = prepare(tab[t]);
        if (st) return st;
    }
    return 0;
}

int tile_mode(int tile) {
    int c;
    const TileEntry* tab = tile_table(&c);
    return (tile < 0 || tile >= c) ? -1 : tab[tile].mode;
}

int default_split_tile() {
    int c;
    const TileEntry* tab = tile_table(&c);
    int first = -1;
    for (int t = 0; t < c; t++) {
        if (tab[t].mode != 1) continue;
        if (first < 0) first = t;
        if (tab[t].bx == 7 && tab[t].by == 7 && tab[t].bz == 7) return t;
    }
    return first;
}

int tile_zones(int tile) {
    int c;
    const TileEntry* tab = tile_table(&c);
    return (tile < 0 || tile >= c) ? 0 : tab[tile].bx * tab[tile].by * tab[tile].bz;
}

// Host replay of the brick kernel's shared-memory indexing: for a tile
// shape, every brick extent the splitter can produce (3..B per axis), every
// block-face combination and every thread, check that each tile and mixed-
// scratch element a thread reads lies inside its array.  Returns the number
// of out-of-range reads (0 = the kernel's smem accesses are all in bounds).
namespace {
// positions along one axis read by the d1/d2/KO stencils at coordinate a
void read_span(int a, int s, bool lo, bool hi, int& pmin, int& pmax) {
    const int ie = s - 3;
    if (lo && a <= 5) {
        pmin = 3;
        pmax = 8;
        return;
    }
    if (hi && a >= ie - 3) {
        pmin = ie - 6;
        pmax = ie - 1;
        return;
    }
    pmin = a - 3;
    pmax = a + 3;
}

template <int BX, int BY, int BZ>
long check_tile_shape() {
    using Bk = Brick<BX, BY, BZ>;
    const int B[3] = {BX, BY, BZ};
    const int T[3] = {Bk::TX, Bk::TY, Bk::TZ};
    long bad = 0;
    // the splitter's brick extents for every block side: at least 3 (a
    // one-sided closure at a physical face reads up to 5 points inward, which
    // a thinner brick's tile of brick + 3 halo points does not hold) and at
    // most the shape
    for (int side : {13, 19, 31, 55})
        for (int d = 0; d < 3; d++) {
            const int n = side - 2 * PW, nb = (n + B[d] - 1) / B[d];
            for (int q = 0; q < nb; q++) {
                int o, e;
                split1(n, B[d], q, o, e);
                if (e < 3 || e > B[d]) bad++;
            }
        }
    for (int e0 = 3; e0 <= BX; e0++)
        for (int e1 = 3; e1 <= BY; e1++)
            for (int e2 = 3; e2 <= BZ; e2++)
                for (int face = 0; face < 4; face++) {
                    // brick at the lower faces (o = 0) or upper faces of a 55 block
                    const int s = 55;
                    const int e[3] = {e0, e1, e2};
                    int o[3];
                    for (int d = 0; d < 3; d++) o[d] = (face & 1) ? (s - 6 - e[d]) : 0;
                    const bool blo = (face & 2) != 0, bhi = (face & 2) != 0;
                    for (int tid = 0; tid < Bk::THREADS; tid++) {
                        const bool in_brick = tid < Bk::NZ;
                        const int r3[3] = {in_brick ? tid % BX : 0,
                                           in_brick ? (tid / BX) % BY : 0,
                                           in_brick ? tid / (BX * BY) : 0};
                        const bool active = in_brick && r3[0] < e[0] && r3[1] < e[1] && r3[2] < e[2];
                        int t3[3];
                        for (int d = 0; d < 3; d++) t3[d] = r3[d] < e[d] ? r3[d] : e[d] - 1;
                        for (int d = 0; d < 3; d++) {
                            const int a = o[d] + PW + t3[d];
                            int pmin, pmax;
                            read_span(a, s, blo, bhi, pmin, pmax);
                            // tile coordinate = position - o: inside the array
                            // for every thread (tile and mixed scratch share the
                            // extent T along the axis), inside the staged region
                            // [0, e+6) for threads that own a zone
                            if (pmin - o[d] < 0 || pmax - o[d] >= T[d]) bad++;
                            if (active && pmax - o[d] >= e[d] + 2 * PW) bad++;
                            if (t3[d] >= B[d]) bad++;
                            // the closure tables cover a in [3, s-3) only
                            if (a < 3 || a > s - 4) bad++;
                        }
                    }
                }
    return bad;
}
}  // namespace

long tile_selfcheck(int tile) {
    int c;
    const TileEntry* tab = tile_table(&c);
    if (tile < 0 || tile >= c) return -1;
    // split tiles stage and read their tiles as fused tiles of the shape do
    const int b[3] = {tab[tile].bx, tab[tile].by, tab[tile].bz};
    auto is = [&](int x, int y, int z) { return b[0] == x && b[1] == y && b[2] == z; };
    if (is(8, 8, 4)) return check_tile_shape<8, 8, 4>();
    if (is(5, 5, 5)) return check_tile_shape<5, 5, 5>();
    if (is(7, 4, 4)) return check_tile_shape<7, 4, 4>();
    if (is(7, 7, 4)) return check_tile_shape<7, 7, 4>();
    if (is(8, 4, 4)) return check_tile_shape<8, 4, 4>();
    if (is(7, 7, 7)) return check_tile_shape<7, 7, 7>();
    if (is(8, 8, 8)) return check_tile_shape<8, 8, 8>();
    if (is(13, 5, 5)) return check_tile_shape<13, 5, 5>();
    if (is(9, 9, 5)) return check_tile_shape<9, 9, 5>();
    return -1;
}

int tile_count() {
    int c;
    tile_table(&c);
    return c;
}

int tile_info(int tile, int info[4]) {
    int c;
    const TileEntry* t = tile_table(&c);
    if (tile < 0 || tile >= c) return BSSN_EINVAL;
    info[0] = t[tile].bx;
    info[1] = t[tile].by;
    info[2] = t[tile].bz;
    info[3] = t[tile].threads;
    return 0;
}

void build_tasks(const BssnBlockDesc* blocks, int nblocks, int tile,
                 std::vector<BrickTask>& out) {
    int c;
    const TileEntry& t = tile_table(&c)[tile];
    for (int b = 0; b < nblocks; b++) {
        const int n = blocks[b].sz - 2 * PW;
        const int nbx = (n + t.bx - 1) / t.bx, nby = (n + t.by - 1) / t.by,
                  nbz = (n + t.bz - 1) / t.bz;
        for (int qz = 0; qz < nbz; qz++)
            for (int qy = 0; qy < nby; qy++)
                for (int qx = 0; qx < nbx; qx++) {
                    BrickTask k;
                    int o, e;
                    k.blk = b;
                    split1(n, t.bx, qx, o, e); k.o[0] = (int16_t)o; k.e[0] = (int16_t)e;
                    split1(n, t.by, qy, o, e); k.o[1] = (int16_t)o; k.e[1] = (int16_t)e;
                    split1(n, t.bz, qz, o, e); k.o[2] = (int16_t)o; k.e[2] = (int16_t)e;
                    out.push_back(k);
                }
    }
}

int launch_rhs_tasks(int tile, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, cudaStream_t s,
                     double* scratch, int64_t scratch_zones, KernelTimer* tm,
                     const int32_t* zip_grid, bool zip_in) {
    int c;
    const TileEntry* tab = tile_table(&c);
    if (tile < 0 || tile >= c) return BSSN_EINVAL;
    if (ntasks <= 0) return 0;
    const TileEntry& t = tab[tile];
    if (t.mode == 1)
        return launch_rhs_split(t.shape, A, blocks_dev, tasks_dev, ntasks, scratch, scratch_zones,
                                s, tm, zip_grid, zip_in);
    if (t.mode == 2)
        return launch_rhs_onchip(t.shape, A, blocks_dev, tasks_dev, ntasks, s, tm, zip_grid, zip_in);
    if (zip_grid) return BSSN_EINVAL;  // the fused kernel writes padded right-hand sides only
    int st = prepare(t);
    if (!st && tm) st = tm->start(KernelTimer::FUSED, s);
    if (st) return st;
    t.kern<<<ntasks, t.threads, t.smem, s>>>(A, blocks_dev, tasks_dev, BssnBlockDesc{});
    st = cuda_status(cudaGetLastError());
    if (!st && tm) st = tm->stop(s);
    return st;
}

int bricks_per_block(int tile, int side) {
    int c;
    const TileEntry* tab = tile_table(&c);
    if (tile < 0 || tile >= c) return 0;
    const TileEntry& t = tab[tile];
    const int n = side - 2 * PW;
    return ((n + t.bx - 1) / t.bx) * ((n + t.by - 1) / t.by) * ((n + t.bz - 1) / t.bz);
}

int rhs_launch_count(int tile, int ntasks, int64_t scratch_zones) {
    if (ntasks <= 0) return 0;
    if (tile_mode(tile) != 1) return 1;
    const int64_t chunk = scratch_zones / tile_zones(tile);
    return chunk > 0 ? (int)(2 * ((ntasks + chunk - 1) / chunk)) : 0;
}

int launch_rhs_single(int tile, const RhsArgs& A, const BssnBlockDesc& blk,
                      cudaStream_t s) {
    int c;
    const TileEntry* tab = tile_table(&c);
    if (tile < 0 || tile >= c) return BSSN_EINVAL;
    if (tab[tile].mode == 2) return launch_rhs_onchip_single(tab[tile].shape, A, blk, s);
    const TileEntry& t = tab[tab[tile].fused];
    int st = prepare(t);
    if (st) return st;
    const int n = blk.sz - 2 * PW;
    const int nb = ((n + t.bx - 1) / t.bx) * ((n + t.by - 1) / t.by) * ((n + t.bz - 1) / t.bz);
    t.kern<<<nb, t.threads, t.smem, s>>>(A, nullptr, nullptr, blk);
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
