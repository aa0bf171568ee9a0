// Split BSSN right-hand side: a derivative pass, then a pointwise equation
// pass, over the same brick task lists as the fused kernel.
//
// The fused kernel keeps every derivative of a zone in registers; its code is
// one straight run of all 24 variables (about 1 MB of instructions) at 255
// registers and one CTA per SM, so it stalls on instruction fetch and on
// FP64 latency.  Here:
//   * deriv_kernel loops over the 24 variables at run time (one copy of the
//     staging, mixed-pass and stencil code), at a few dozen registers and
//     several CTAs per SM, and writes each zone's gradient, second
//     derivatives and summed KO term to a scratch array;
//   * eq_kernel evaluates the equations per zone (rhs_equations.cuh, the same
//     code as the fused kernel) reading those derivatives back.
// The scratch holds slot pairs, [slot / 2][task * NZ + thread][slot % 2]
// (every variable has an even number of slots), so both passes move 16-byte
// pairs in whole rows of consecutive zones.  A task list longer than the scratch is
// processed in chunks, each a derivative launch followed by an equation
// launch on the same stream.
//
// Derivatives are bit-identical to the fused kernel's (same stencils, same
// tiles); the equations are the same code, so both paths give the same RHS.
#include <cuda_runtime.h>

#include "bssn_common.cuh"
#include "rhs_brick.cuh"
#include "rhs_equations.cuh"
#include "rhs_fused.cuh"

namespace bssn {

namespace {

// Scratch slots per zone: gradient (3) + second derivatives (6) + KO for the
// 11 variables with second derivatives, gradient + KO for the other 13.
constexpr int kSlotsSecond = 10;
constexpr int kSlotsFirst = 4;
__host__ __device__ constexpr int slot_len(int step) {
    return stage_second(step) ? kSlotsSecond : kSlotsFirst;
}
__host__ __device__ constexpr int slot_base(int step) {
    int b = 0;
    for (int k = 0; k < step; k++) b += slot_len(k);
    return b;
}
static_assert(slot_base(NVARS) == kSplitSlots, "scratch slot count");

// resident derivative CTAs per SM the register allocation must allow: 3 for
// up to 384 threads (56 registers at 352), 2 for up to 512, else 1
__host__ __device__ constexpr int deriv_min_ctas(int threads) {
    return threads <= 384 ? 3 : threads <= 512 ? 2 : 1;
}
// equation pass: variables whose derivatives are in flight ahead of use, and
// the per-thread ring of scratch slots (shared memory) they land in; one
// variable more than the prefetch distance, so a copy never targets a row
// read by the variable just consumed
constexpr int kPrefetchSteps = 6;
constexpr int kRingSlots = (kPrefetchSteps + 1) * kSlotsSecond;
constexpr int kRingPairs = kRingSlots / 2;
constexpr int kEqThreads = 128;
// derivative pass: shared-memory tiles (variables staged kDerivBuffers - 1 ahead)
constexpr int kDerivBuffers = 2;
template <class Bk>
constexpr size_t deriv_smem_bytes() {
    return sizeof(double) * (kDerivBuffers * Bk::TILE + Bk::MXJ + 2 * Bk::MXK);
}

template <int N>
__device__ __forceinline__ void cp_async_wait_pending() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Whether the zone at brick position t owns its node of the zipped grid: a
// node on a block's upper face belongs to the next block unless the face
// lies on the grid's upper boundary (the zip's owner rule).
__device__ __forceinline__ bool owns_node(const BssnBlockDesc& blk, const int o[3], const int t[3],
                                          const ZipGrid& g) {
    const int n = blk.sz - 2 * PW;
    const int gd[3] = {g.gx, g.gy, g.gz};
    bool own = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int i = o[d] + t[d];  // interior index
        own = own && (i < n - 1 || blk.g0[d] + i == gd[d] - 1);
    }
    return own;
}

// ZIP: stage from the zipped node grid (g) instead of the padded blocks.
template <int BX, int BY, int BZ, bool ZIP>
__global__ void __launch_bounds__(Brick<BX, BY, BZ>::THREADS,
                                   deriv_min_ctas(Brick<BX, BY, BZ>::THREADS))
deriv_kernel(ConstVars u, const BssnBlockDesc* __restrict__ blocks,
             const BrickTask* __restrict__ tasks, double* __restrict__ S, int64_t zs,
             ZipGrid g) {
    using Bk = Brick<BX, BY, BZ>;
    extern __shared__ __align__(16) double smem[];
    __shared__ const double* src[NVARS];
    __shared__ AxisCoef cfs[3];
    double* tiles = smem;                         // kDerivBuffers tiles
    double* mx = smem + kDerivBuffers * Bk::TILE;  // mxj | mxk | myk
    const BrickTask tk = tasks[blockIdx.x];
    const BssnBlockDesc blk = blocks[tk.blk];
    const int o[3] = {tk.o[0], tk.o[1], tk.o[2]};
    const int e[3] = {tk.e[0], tk.e[1], tk.e[2]};
    const int tid = threadIdx.x;
    const int s = blk.sz;
    if (tid < NVARS) src[tid] = u.p[stage_order(tid)] + (ZIP ? 0 : blk.offset);
    fill_axis_coefs(cfs, blk, tid);
    const BrickThread<Bk> th(tid, e);
    const BrickZone<Bk> bz(blk, o, th, cfs);
    const StagePlan<Bk, ZIP> sp(o, e, s, tid, g, blk.g0);
    // zones whose derivatives the equation pass reads: every zone of the
    // brick, or (node grid given: direct form or stage mode) only the zones
    // that own their node
    const bool keep = th.active && (g.gx == 0 || owns_node(blk, o, th.t, g));
    // next scratch slot pair of this zone (kept zones only advance it)
    double2* w = reinterpret_cast<double2*>(S) + (int64_t)blockIdx.x * Bk::NZ + tid;
    __syncthreads();

    // variables in flight kDerivBuffers - 1 ahead; one commit group per
    // variable (empty past the last one, so the pending count stays fixed)
#pragma unroll
    for (int k = 0; k < kDerivBuffers - 1; k++) sp.stage(src[k], tiles + k * Bk::TILE, tid);
#pragma unroll 1
    for (int step = 0; step < NVARS; step++) {
        cp_async_wait_pending<kDerivBuffers - 2>();
        __syncthreads();  // the tile of `step` is complete; the buffer below was last read at step - 1
        const double* cur = tiles + (step % kDerivBuffers) * Bk::TILE;
        const int nxt = step + kDerivBuffers - 1;
        if (nxt < NVARS)
            sp.stage(src[nxt], tiles + (nxt % kDerivBuffers) * Bk::TILE, tid);
        else
            cp_async_commit();
        if (stage_second(step)) {
            Dir3 r[3];
            zone_dirs<true, Bk>(bz.zc, cur, r);
            // the brick part of the mixed scratch from the zones' own gradient
            if (th.active) {
                mx[bz.mxj_off] = r[0].d1;  // the offsets include the halo
                mx[Bk::MXJ + bz.mxk_off] = r[0].d1;
                mx[Bk::MXJ + Bk::MXK + bz.mxk_off] = r[1].d1;
            }
            mixed_halo_pass<Bk>(cur, mx, o, e, s, blk.bflag, bz.zc.cf, tid);
            __syncthreads();
            const double* mxj = mx + bz.mxj_off;
            const double* mxk = mx + Bk::MXJ + bz.mxk_off;
            const double* myk = mx + Bk::MXJ + Bk::MXK + bz.mxk_off;
            const ZoneCtx& z = bz.zc;
            double xy = d1_fast_in(mxj, Bk::BX, z.cf[1]);
            double xz = d1_fast_in(mxk, Bk::BX * Bk::BY, z.cf[2]);
            double yz = d1_fast_in(myk, Bk::BX * Bk::BY, z.cf[2]);
            if (z.bflag) {
                if (near_face(z.a[1], s, z.bflag & 4u, z.bflag & 8u))
                    xy = closure_d1(mxj, bz.mj, z.a[1], s, z.bflag & 4u, z.cf[1]);
                if (near_face(z.a[2], s, z.bflag & 16u, z.bflag & 32u)) {
                    xz = closure_d1(mxk, bz.mk, z.a[2], s, z.bflag & 16u, z.cf[2]);
                    yz = closure_d1(myk, bz.mk, z.a[2], s, z.bflag & 16u, z.cf[2]);
                }
            }
            if (keep) {
                const double v[kSlotsSecond] = {r[0].d1, r[1].d1, r[2].d1, r[0].d2, xy, xz,
                                                r[1].d2, yz, r[2].d2, r[0].ko + r[1].ko + r[2].ko};
#pragma unroll
                for (int q = 0; q < kSlotsSecond; q += 2, w += zs) *w = make_double2(v[q], v[q + 1]);
            }
        } else {
            Dir3 r[3];
            zone_dirs<false, Bk>(bz.zc, cur, r);
            if (keep) {
                const double v[kSlotsFirst] = {r[0].d1, r[1].d1, r[2].d1,
                                               r[0].ko + r[1].ko + r[2].ko};
#pragma unroll
                for (int q = 0; q < kSlotsFirst; q += 2, w += zs) *w = make_double2(v[q], v[q + 1]);
            }
        }
    }
}

// One thread per zone, kEqThreads zones of a brick per CTA (a brick of NZ
// zones takes ceil(NZ / kEqThreads) CTAs), so two CTAs share an SM at 254
// registers.  Each thread streams its own zone's 24 variables and scratch
// slots into its own columns of shared memory with cp.async, the slots
// kPrefetchSteps variables ahead of the equations that consume them (one
// commit group per variable; a thread only reads what it copied itself, so
// no barrier).
// g.gx == 0: variables and right-hand sides at the zone's padded index.
// g.gx > 0: only zones owning their node run and write the right-hand side
// at the node index of the zipped grid; the variables are read there too
// (zip_in, direct form) or at the padded index.
template <int BX, int BY, int BZ>
__global__ void __launch_bounds__(kEqThreads, 2)
eq_kernel(RhsArgs A, const BssnBlockDesc* __restrict__ blocks,
          const BrickTask* __restrict__ tasks, const double* __restrict__ S, int64_t zs,
          ZipGrid g, int zip_in) {
    using Bk = Brick<BX, BY, BZ>;
    constexpr int PARTS = (Bk::NZ + kEqThreads - 1) / kEqThreads;
    extern __shared__ __align__(16) double ring[];  // [kRingPairs][T][2] | vals [NVARS][T]
    const int tid = threadIdx.x;
    const int task = blockIdx.x / PARTS;
    const BrickTask tk = tasks[task];
    const BssnBlockDesc blk = blocks[tk.blk];
    const int o[3] = {tk.o[0], tk.o[1], tk.o[2]};
    // the zones that run: the brick's extent, or on the zipped grid only the
    // zones owning their node (a brick on a block's upper face loses its last
    // layer there unless the face lies on the grid's upper boundary); the
    // threads are packed onto them, so no lane idles on a skipped zone
    int ex[3] = {tk.e[0], tk.e[1], tk.e[2]};
    if (g.gx) {
        const int n = blk.sz - 2 * PW;
        const int gd[3] = {g.gx, g.gy, g.gz};
#pragma unroll
        for (int d = 0; d < 3; d++)
            if (o[d] + ex[d] == n && blk.g0[d] + n - 1 != gd[d] - 1) ex[d]--;
    }
    const int j = (blockIdx.x % PARTS) * kEqThreads + tid;  // the thread's zone among them
    if (j >= ex[0] * ex[1] * ex[2]) return;
    const int r0 = j % ex[0], r1 = (j / ex[0]) % ex[1], r2 = j / (ex[0] * ex[1]);
    const int l = r0 + BX * (r1 + BY * r2);  // zone index in the brick (scratch position)
    const int za0 = o[0] + PW + r0, za1 = o[1] + PW + r1, za2 = o[2] + PW + r2;
    const int64_t pidx = blk.offset + za0 + (int64_t)blk.sz * (za1 + (int64_t)blk.sz * za2);
    int64_t node = pidx;
    if (g.gx)
        node = (blk.g0[0] + za0 - PW) +
               (int64_t)g.gx * ((blk.g0[1] + za1 - PW) + (int64_t)g.gy * (blk.g0[2] + za2 - PW));
    const int64_t in_idx = zip_in ? node : pidx;
    const double2* in = reinterpret_cast<const double2*>(S) + (int64_t)task * Bk::NZ + l;
    double2* col = reinterpret_cast<double2*>(ring) + tid;   // this thread's ring column
    double* vals = ring + kRingSlots * kEqThreads + tid;  // [NVARS][kEqThreads]
    // the zone's 24 variables first, as their own commit group
#pragma unroll
    for (int v = 0; v < NVARS; v++) cp_async8(vals + v * kEqThreads, A.u.p[v] + in_idx);
    cp_async_commit();
    // slot pair P of the zone lives in ring row P % kRingPairs (slot bases
    // and counts are even, so a variable's slots are whole pairs)
    auto issue = [&](int step) {
        if (step < NVARS) {
            const int b = slot_base(step) / 2, n = slot_len(step) / 2;
#pragma unroll
            for (int q = 0; q < kSlotsSecond / 2; q++)
                if (q < n) cp_async16(col + ((b + q) % kRingPairs) * kEqThreads, in + (int64_t)(b + q) * zs);
        }
        cp_async_commit();  // empty groups past the last variable keep the count fixed
    };
#pragma unroll
    for (int k = 0; k < kPrefetchSteps; k++) issue(k);
    cp_async_wait_pending<kPrefetchSteps>();  // the variables' group
    auto pv = [&](int v) { return vals[v * kEqThreads]; };
    int step = 0;
    auto get = [&](auto tag, double* d1, double* d2, double& ko) {
        constexpr bool SECOND = decltype(tag)::value;
        cp_async_wait_pending<kPrefetchSteps - 1>();
        const int b = slot_base(step);
        auto rd = [&](int q) {
            const double2 p = col[(((b + q) / 2) % kRingPairs) * kEqThreads];
            return ((b + q) & 1) ? p.y : p.x;
        };
#pragma unroll
        for (int q = 0; q < 3; q++) d1[q] = rd(q);
        if (SECOND) {
#pragma unroll
            for (int q = 0; q < 6; q++) d2[q] = rd(3 + q);
            ko = rd(9);
        } else {
            ko = rd(3);
        }
        issue(step + kPrefetchSteps);  // rows of variables consumed before this one
        step++;
    };
    auto store = [&](int v, double r) { A.rhs.p[v][node] = r; };
    zone_equations(A, blk, za0, za1, za2, get, pv, store);
}

constexpr size_t eq_smem_bytes() { return sizeof(double) * kEqThreads * (kRingSlots + NVARS); }

struct SplitEntry {
    int nz, threads;
    size_t smem;
    void (*deriv)(ConstVars, const BssnBlockDesc*, const BrickTask*, double*, int64_t, ZipGrid);
    void (*deriv_zip)(ConstVars, const BssnBlockDesc*, const BrickTask*, double*, int64_t, ZipGrid);
    void (*eq)(RhsArgs, const BssnBlockDesc*, const BrickTask*, const double*, int64_t, ZipGrid, int);
};

template <int BX, int BY, int BZ>
SplitEntry make_split() {
    using Bk = Brick<BX, BY, BZ>;
    return SplitEntry{Bk::NZ, Bk::THREADS, deriv_smem_bytes<Bk>(),
                      deriv_kernel<BX, BY, BZ, false>, deriv_kernel<BX, BY, BZ, true>,
                      eq_kernel<BX, BY, BZ>};
}

// the fused tiles' shapes in their order, then split-only shapes (bricks too
// large for the fused kernel's 255 registers per zone)
const SplitEntry* split_table(int* count) {
    static const SplitEntry table[] = {
        make_split<8, 8, 4>(),
        make_split<7, 7, 4>(),
        make_split<8, 4, 4>(),
        make_split<7, 7, 7>(),
        make_split<8, 8, 8>(),
        make_split<13, 5, 5>(),
        make_split<9, 9, 5>(),
    };
    *count = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

}  // namespace

int split_shape_count() {
    int c;
    split_table(&c);
    return c;
}

int split_zone_count(int shape) {
    int c;
    const SplitEntry* t = split_table(&c);
    return (shape < 0 || shape >= c) ? 0 : t[shape].nz;
}

int prepare_split(int shape) {
    int c;
    const SplitEntry* t = split_table(&c);
    if (shape < 0 || shape >= c) return BSSN_EINVAL;
    int st = set_smem_limit((const void*)t[shape].deriv, (int)t[shape].smem);
    if (!st) st = set_smem_limit((const void*)t[shape].deriv_zip, (int)t[shape].smem);
    if (!st) st = set_smem_limit((const void*)t[shape].eq, (int)eq_smem_bytes());
    return st;
}

int launch_rhs_split(int shape, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, double* scratch,
                     int64_t scratch_zones, cudaStream_t s, KernelTimer* tm,
                     const int32_t* zip_grid, bool zip_in) {
    int c;
    const SplitEntry* tab = split_table(&c);
    if (shape < 0 || shape >= c) return BSSN_EINVAL;
    if (ntasks <= 0) return 0;
    const SplitEntry& t = tab[shape];
    const int64_t chunk = scratch ? scratch_zones / t.nz : 0;
    if (chunk <= 0) return BSSN_EINVAL;
    int st = prepare_split(shape);
    if (st) return st;
    const ZipGrid g = zip_grid ? ZipGrid{zip_grid[0], zip_grid[1], zip_grid[2]} : ZipGrid{0, 0, 0};
    zip_in = zip_in && zip_grid;
    const int64_t zs = chunk * t.nz;  // slot stride
    for (int64_t c0 = 0; c0 < ntasks; c0 += chunk) {
        const int n = (int)(ntasks - c0 < chunk ? ntasks - c0 : chunk);
        if (tm && (st = tm->start(KernelTimer::DERIV, s))) return st;
        (zip_in ? t.deriv_zip : t.deriv)<<<n, t.threads, t.smem, s>>>(A.u, blocks_dev, tasks_dev + c0,
                                                                      scratch, zs, g);
        st = cuda_status(cudaGetLastError());
        if (!st && tm) st = tm->stop(s);
        if (st) return st;
        if (tm && (st = tm->start(KernelTimer::EQ, s))) return st;
        const int parts = (t.nz + kEqThreads - 1) / kEqThreads;
        t.eq<<<n * parts, kEqThreads, eq_smem_bytes(), s>>>(A, blocks_dev, tasks_dev + c0, scratch,
                                                             zs, g, zip_in ? 1 : 0);
        st = cuda_status(cudaGetLastError());
        if (!st && tm) st = tm->stop(s);
        if (st) return st;
    }
    return 0;
}

}  // namespace bssn
