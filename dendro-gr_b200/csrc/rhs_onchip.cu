// On-chip BSSN right-hand side: derivatives never leave the SM.
//
// One CTA of 128 threads owns a brick of at most 128 interior zones of one
// block, one thread per zone, two CTAs per SM (up to 255 registers each
// thread).  A runtime loop over the 24 evolved variables (stage_order())
// stages each variable's tile (brick + 3-point halo) into shared memory with
// cp.async, one variable ahead; forms the zone's gradient, second
// derivatives (mixed ones through the cooperative halo pass) and summed KO
// term with the bit-exact stencils of rhs_brick.cuh, in registers; and hands
// them to that variable's step of the equations (rhs_steps.cuh), chosen by a
// switch.  The derivative code thus exists once (the split path's
// derivative pass, without its 162-slot scratch round trip through HBM) and
// the equation code once (the fused rhs_kernel inlines the derivative code
// for every variable: ~1 MB of machine code).
//
// HBM traffic per brick: the 24 tiles (first touch; neighbouring bricks'
// halos mostly hit L2), the zone's 24 values, and the 24 right-hand sides of
// the zones written.  Output either padded (at the zone's padded index) or,
// given the node grid, zipped: each node written once by the zone owning it
// (the zip's owner rule); ZIP staging reads the tiles straight from the
// zipped node grid (points outside it zero, as the ghost fill writes them).
#include <cuda_runtime.h>

#include "bssn_common.cuh"
#include "rhs_brick.cuh"
#include "rhs_fused.cuh"
#include "rhs_steps.cuh"

namespace bssn {

namespace {

constexpr int kOcThreads = 128;
constexpr int kOcBuffers = 3;  // tile buffers: two variables staged ahead

template <class Bk>
constexpr size_t onchip_smem_bytes() {
    return sizeof(double) * (kOcBuffers * Bk::TILE + Bk::MXJ + 2 * Bk::MXK + NVARS * kOcThreads);
}

template <int N>
__device__ __forceinline__ void oc_wait_pending() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ bool oc_owns_node(const BssnBlockDesc& blk, const int o[3], const int t[3],
                                             const ZipGrid& g) {
    const int n = blk.sz - 2 * PW;
    const int gd[3] = {g.gx, g.gy, g.gz};
    bool own = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int i = o[d] + t[d];
        own = own && (i < n - 1 || blk.g0[d] + i == gd[d] - 1);
    }
    return own;
}

// g.gx == 0: padded input and output at the zone's padded index.  g.gx > 0:
// zipped output at the node index, written by owning zones only; ZIP: the
// tiles and the zone's values come from the zipped node grid.  MINB: CTAs
// per SM the register allocation must allow (2: up to 255 registers; 3: up
// to 168, the colder equation state spilling to local memory).
template <int BX, int BY, int BZ, bool ZIP, int MINB>
__global__ void __launch_bounds__(kOcThreads, MINB)
onchip_kernel(RhsArgs A, const BssnBlockDesc* __restrict__ blocks,
              const BrickTask* __restrict__ tasks, ZipGrid g, BssnBlockDesc single) {
    using Bk = Brick<BX, BY, BZ>;
    static_assert(Bk::THREADS == kOcThreads, "one CTA of kOcThreads threads per brick");
    extern __shared__ __align__(16) double smem[];
    __shared__ const double* src[NVARS];
    __shared__ AxisCoef cfs[3];
    double* tiles = smem;
    double* mx = smem + kOcBuffers * Bk::TILE;
    double* vals = mx + Bk::MXJ + 2 * Bk::MXK;  // [NVARS][kOcThreads]: the zone's values
    int o[3], e[3];
    BssnBlockDesc blk;
    if (tasks != nullptr) {
        const BrickTask tk = tasks[blockIdx.x];
        blk = blocks[tk.blk];
        for (int d = 0; d < 3; d++) {
            o[d] = tk.o[d];
            e[d] = tk.e[d];
        }
    } else {  // the bricks of the one block passed by value, by CTA index
        blk = single;
        const int n = single.sz - 2 * PW;
        const int nbx = (n + BX - 1) / BX, nby = (n + BY - 1) / BY;
        const int q = blockIdx.x;
        split1(n, BX, q % nbx, o[0], e[0]);
        split1(n, BY, (q / nbx) % nby, o[1], e[1]);
        split1(n, BZ, q / (nbx * nby), o[2], e[2]);
    }
    const int tid = threadIdx.x;
    const int s = blk.sz;
    if (tid < NVARS) src[tid] = A.u.p[stage_order(tid)] + (ZIP ? 0 : blk.offset);
    fill_axis_coefs(cfs, blk, tid);
    // threads past the brick's zones compute on the nearest zone (every
    // index stays in the tile) and store nothing
    const BrickThread<Bk> th(tid, e);
    const BrickZone<Bk> bz(blk, o, th, cfs);
    const StagePlan<Bk, ZIP> sp(o, e, s, tid, g, blk.g0);
    const bool zipped = g.gx > 0;
    const bool keep = th.active && (!zipped || oc_owns_node(blk, o, th.t, g));
    const int za0 = bz.zc.a[0], za1 = bz.zc.a[1], za2 = bz.zc.a[2];
    const int64_t pidx = blk.offset + za0 + (int64_t)s * (za1 + (int64_t)s * za2);
    int64_t node = pidx;
    if (zipped)
        node = (blk.g0[0] + za0 - PW) +
               (int64_t)g.gx * ((blk.g0[1] + za1 - PW) + (int64_t)g.gy * (blk.g0[2] + za2 - PW));
    const int64_t in_idx = ZIP ? node : pidx;
    // the zone's 24 values, first commit group
#pragma unroll
    for (int v = 0; v < NVARS; v++) cp_async8(vals + v * kOcThreads + tid, A.u.p[v] + in_idx);
    cp_async_commit();
    __syncthreads();  // src, cfs
#pragma unroll
    for (int k = 0; k < kOcBuffers - 1; k++) sp.stage(src[k], tiles + k * Bk::TILE, tid);

    auto pv = [&](int v) { return vals[v * kOcThreads + tid]; };
    auto store = [&](int v, double r) {
        if (keep) A.rhs.p[v][node] = r;
    };
    EqSteps eq;
    oc_wait_pending<kOcBuffers - 1>();  // this thread's values (tiles may still be in flight)
    eq.begin(A, blk, za0, za1, za2, pv);
    // one commit group per variable (empty past the last), so the tile of
    // `step` is complete once at most kOcBuffers - 2 groups are pending
#pragma unroll 1
    for (int step = 0; step < NVARS; step++) {
        oc_wait_pending<kOcBuffers - 2>();
        __syncthreads();  // tile of `step` complete; the buffer staged next was read at step - 1
        const double* cur = tiles + (step % kOcBuffers) * Bk::TILE;
        const int nxt = step + kOcBuffers - 1;
        if (nxt < NVARS)
            sp.stage(src[nxt], tiles + (nxt % kOcBuffers) * Bk::TILE, tid);
        else
            cp_async_commit();
        double d1[3], d2[6], ko;
        if (stage_second(step)) {
            Dir3 r[3];
            zone_dirs_il<true, Bk>(bz.zc, cur, r);
            if (th.active) {
                mx[bz.mxj_off] = r[0].d1;
                mx[Bk::MXJ + bz.mxk_off] = r[0].d1;
                mx[Bk::MXJ + Bk::MXK + bz.mxk_off] = r[1].d1;
            }
            mixed_halo_pass<Bk>(cur, mx, o, e, s, blk.bflag, bz.zc.cf, tid);
            __syncthreads();
            const double* mxj = mx + bz.mxj_off;
            const double* mxk = mx + Bk::MXJ + bz.mxk_off;
            const double* myk = mx + Bk::MXJ + Bk::MXK + bz.mxk_off;
            const ZoneCtx& zc = bz.zc;
            double xy = d1_fast_in(mxj, Bk::BX, zc.cf[1]);
            double xz = d1_fast_in(mxk, Bk::BX * Bk::BY, zc.cf[2]);
            double yz = d1_fast_in(myk, Bk::BX * Bk::BY, zc.cf[2]);
            if (zc.bflag) {
                if (near_face(zc.a[1], s, zc.bflag & 4u, zc.bflag & 8u))
                    xy = closure_d1(mxj, bz.mj, zc.a[1], s, zc.bflag & 4u, zc.cf[1]);
                if (near_face(zc.a[2], s, zc.bflag & 16u, zc.bflag & 32u)) {
                    xz = closure_d1(mxk, bz.mk, zc.a[2], s, zc.bflag & 16u, zc.cf[2]);
                    yz = closure_d1(myk, bz.mk, zc.a[2], s, zc.bflag & 16u, zc.cf[2]);
                }
            }
            d1[0] = r[0].d1; d1[1] = r[1].d1; d1[2] = r[2].d1;
            d2[0] = r[0].d2; d2[1] = xy; d2[2] = xz; d2[3] = r[1].d2; d2[4] = yz; d2[5] = r[2].d2;
            ko = r[0].ko + r[1].ko + r[2].ko;
        } else {
            Dir3 r[3];
            zone_dirs_il<false, Bk>(bz.zc, cur, r);
            d1[0] = r[0].d1; d1[1] = r[1].d1; d1[2] = r[2].d1;
#pragma unroll
            for (int q = 0; q < 6; q++) d2[q] = 0.0;
            ko = r[0].ko + r[1].ko + r[2].ko;
        }
        switch (step) {
#define BSSN_OC_STEP(K) \
    case K: eq.step<K>(A, d1, d2, ko, pv, store); break;
            BSSN_OC_STEP(0) BSSN_OC_STEP(1) BSSN_OC_STEP(2) BSSN_OC_STEP(3) BSSN_OC_STEP(4)
            BSSN_OC_STEP(5) BSSN_OC_STEP(6) BSSN_OC_STEP(7) BSSN_OC_STEP(8) BSSN_OC_STEP(9)
            BSSN_OC_STEP(10) BSSN_OC_STEP(11) BSSN_OC_STEP(12) BSSN_OC_STEP(13) BSSN_OC_STEP(14)
            BSSN_OC_STEP(15) BSSN_OC_STEP(16) BSSN_OC_STEP(17) BSSN_OC_STEP(18) BSSN_OC_STEP(19)
            BSSN_OC_STEP(20) BSSN_OC_STEP(21) BSSN_OC_STEP(22) BSSN_OC_STEP(23)
#undef BSSN_OC_STEP
            default: break;
        }
    }
}

struct OnchipEntry {
    int bx, by, bz, minb;
    size_t smem;
    void (*kern)(RhsArgs, const BssnBlockDesc*, const BrickTask*, ZipGrid, BssnBlockDesc);
    void (*kern_zip)(RhsArgs, const BssnBlockDesc*, const BrickTask*, ZipGrid, BssnBlockDesc);
};

template <int BX, int BY, int BZ, int MINB>
OnchipEntry make_onchip() {
    using Bk = Brick<BX, BY, BZ>;
    return OnchipEntry{BX, BY, BZ, MINB, onchip_smem_bytes<Bk>(), onchip_kernel<BX, BY, BZ, false, MINB>,
                       onchip_kernel<BX, BY, BZ, true, MINB>};
}

const OnchipEntry* onchip_table(int* count) {
    static const OnchipEntry table[] = {
        make_onchip<5, 5, 5, 2>(),
        make_onchip<7, 4, 4, 2>(),
        make_onchip<5, 5, 5, 3>(),
        make_onchip<7, 4, 4, 3>(),
    };
    *count = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

}  // namespace

int onchip_shape_count() {
    int c;
    onchip_table(&c);
    return c;
}

int onchip_shape(int shape, int b[3]) {
    int c;
    const OnchipEntry* t = onchip_table(&c);
    if (shape < 0 || shape >= c) return BSSN_EINVAL;
    b[0] = t[shape].bx;
    b[1] = t[shape].by;
    b[2] = t[shape].bz;
    return 0;
}

int prepare_onchip(int shape) {
    int c;
    const OnchipEntry* t = onchip_table(&c);
    if (shape < 0 || shape >= c) return BSSN_EINVAL;
    int st = set_smem_limit((const void*)t[shape].kern, (int)t[shape].smem);
    if (!st) st = set_smem_limit((const void*)t[shape].kern_zip, (int)t[shape].smem);
    return st;
}

int launch_rhs_onchip(int shape, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                      const BrickTask* tasks_dev, int ntasks, cudaStream_t s, KernelTimer* tm,
                      const int32_t* zip_grid, bool zip_in) {
    int c;
    const OnchipEntry* tab = onchip_table(&c);
    if (shape < 0 || shape >= c) return BSSN_EINVAL;
    if (ntasks <= 0) return 0;
    const OnchipEntry& t = tab[shape];
    int st = prepare_onchip(shape);
    if (st) return st;
    const ZipGrid g = zip_grid ? ZipGrid{zip_grid[0], zip_grid[1], zip_grid[2]} : ZipGrid{0, 0, 0};
    zip_in = zip_in && zip_grid;
    if (tm && (st = tm->start(KernelTimer::FUSED, s))) return st;
    (zip_in ? t.kern_zip : t.kern)<<<ntasks, kOcThreads, t.smem, s>>>(A, blocks_dev, tasks_dev, g,
                                                                      BssnBlockDesc{});
    st = cuda_status(cudaGetLastError());
    if (!st && tm) st = tm->stop(s);
    return st;
}

int launch_rhs_onchip_single(int shape, const RhsArgs& A, const BssnBlockDesc& blk, cudaStream_t s) {
    int c;
    const OnchipEntry* tab = onchip_table(&c);
    if (shape < 0 || shape >= c) return BSSN_EINVAL;
    const OnchipEntry& t = tab[shape];
    int st = prepare_onchip(shape);
    if (st) return st;
    const int n = blk.sz - 2 * PW;
    const int nb = ((n + t.bx - 1) / t.bx) * ((n + t.by - 1) / t.by) * ((n + t.bz - 1) / t.bz);
    t.kern<<<nb, kOcThreads, t.smem, s>>>(A, nullptr, nullptr, ZipGrid{0, 0, 0}, blk);
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
