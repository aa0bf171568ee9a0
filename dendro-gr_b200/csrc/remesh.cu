// Remesh decision: the exact wavelet refinement test, cheap per-block
// features, and a small BF16 MLP (16 -> 64 -> 64 -> 1, GELU, FP32
// accumulation) that predicts the test, with hand-written forward, backward
// and Adam kernels.
//
// Wavelet test: the reference scores every element with the interpolating
// wavelet transform of dendrolib (isReMeshWAMR, BSSN_GR/src/dataUtils.cpp:
// 511-624; the transform itself is absent from the reference tree).  This
// file's definition: for every node of an element (octant, 7^3 nodes) with
// an odd local index along some axis, w = u - (degree-5 Lagrange
// interpolation from the coarse nodes at patch positions 1,3,5,7,9,11 of the
// element's 13^3 patch along each odd axis); score = sqrt(sum w^2 / 279);
// the element asks for refinement when the score of any variable exceeds
// the tolerance.  Products and sums are explicitly rounded in a fixed order
// (inner x, then y, then z; squares summed into 32 partials by node index mod
// 32, partials added in order), identical to the CPU restatement.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "bssn_common.cuh"
#include "mesh.h"
#include "remesh.h"
#include "bssn_b200.h"

namespace bssn {
namespace {

__constant__ double kWfine[3][6] = {
    {-7.0 / 256, 105.0 / 256, 105.0 / 128, -35.0 / 128, 21.0 / 256, -3.0 / 256},
    {3.0 / 256, -25.0 / 256, 75.0 / 128, 75.0 / 128, -25.0 / 256, 3.0 / 256},
    {-3.0 / 256, 21.0 / 256, -35.0 / 128, 105.0 / 128, 105.0 / 256, -7.0 / 256}};

// Separable form of the test, one warp per (element, variable).  The
// interpolation at a node is a tensor product, evaluated inner x, then y,
// then z; every partial sum of that product is shared by the nodes with the
// same remaining coordinates, so the warp forms each once:
//   X[k][j][a] = x-interpolation on coarse row (j, k) at element x-index a,
//   Y[k][b][a] = y-interpolation of X over the coarse rows j,
//   Z[c][b][a] = z-interpolation of Y over the coarse planes k,
// where the coarse points are the patch positions 1,3,...,11 along each
// axis (an even element index a sits on coarse point a/2 + 1 and is taken
// with weight 1).  Each sum starts from 0 and adds the explicitly rounded
// products in index order, so every value equals the per-node evaluation
// bit for bit.  Squares of the residuals w = u - Z land in shared memory at
// their node index q (z,y,x order over the 279 nodes with an odd
// coordinate); lane l sums q = l, l+32, ... in order and lane 0 adds the 32
// partials in lane order.
constexpr int kWavWarps = 4;
constexpr int kWavC = 216, kWavX = 252, kWavY = 294;  // 6^3, 36 x 7, 6 x 49

__device__ __forceinline__ double rn_one(double v) { return __dadd_rn(0.0, __dmul_rn(1.0, v)); }

// Lane roles: a lane l < 30 always evaluates with the weight row l % 3 (its
// six weights stay in registers for the whole kernel) on the items
// g = l / 3, g + 10, ...; every lane shares the trivial copies (even index).
// The mapping only moves work between lanes: each value is still formed by
// the same rounded products and sums in the same order.
struct WavLane {
    double w[6];
    int rho, g;
    bool interp;
};

// node index q of (a, b, c) among the 279 nodes with an odd coordinate (z,y,x
// order): t = a + 7b + 49c minus the all-even nodes before it
__device__ __forceinline__ int wav_q(int a, int b, int c) {
    const int t = a + 7 * b + 49 * c;
    return t - (((c + 1) >> 1) * 16 + ((c & 1) ? 0 : ((b + 1) >> 1) * 4 + ((b & 1) ? 0 : (a + 1) >> 1)));
}

// One (element, variable) item for the calling warp: p points at patch
// position (0,0,0) of the element, s is the block side, buf the warp's
// kWavC + kWavX + kWavY doubles of shared memory, pairs the 33 (b, a) pairs
// with an odd coordinate (b * 7 + a, b-major).  Returns the sum of the
// squared residuals (the same value in every lane).
__device__ __forceinline__ double wavelet_item(const double* __restrict__ p, int64_t s, const WavLane& L,
                                               const uint8_t* __restrict__ pairs, double* buf, int lane) {
    const int64_t s2 = s * s;
    double* C = buf;
    double* X = C + kWavC;
    double* Y = X + kWavX;
    double* SQ = C;  // reused once C and X are consumed
    // the element's own nodes this lane needs in the last stage, fetched now
    // so their latency hides behind the interpolation: odd c (its role's
    // c = 2 rho + 1, pairs g + 10 j) and even c (nodes lane + 32 r)
    double uo[5], ue[5];
#pragma unroll
    for (int j = 0; j < 5; j++) {
        const int pr = L.g + 10 * j;
        uo[j] = (L.interp && pr < 49)
                    ? __ldg(p + (pr % 7 + 3) + s * (pr / 7 + 3) + s2 * (2 * L.rho + 4)) : 0.0;
    }
#pragma unroll
    for (int r = 0; r < 5; r++) {
        const int t = lane + 32 * r;
        if (t < 132) {
            const int ba = pairs[t % 33], ce = t / 33;
            ue[r] = __ldg(p + (ba % 7 + 3) + s * (ba / 7 + 3) + s2 * (2 * ce + 3));
        } else {
            ue[r] = 0.0;
        }
    }
    for (int t = lane; t < kWavC; t += 32) {
        const int i = t % 6, j = (t / 6) % 6, k = t / 36;
        C[t] = __ldg(p + (2 * i + 1) + s * (2 * j + 1) + s2 * (2 * k + 1));
    }
    __syncwarp();
    // x: 36 coarse rows x 3 odd a (interpolated), x 4 even a (taken)
    if (L.interp) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int m = L.g + 10 * k;
            if (m < 36) {
                const double* c = C + m * 6;
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < 6; i++) acc = __dadd_rn(acc, __dmul_rn(L.w[i], c[i]));
                X[m * 7 + 2 * L.rho + 1] = acc;
            }
        }
    }
    for (int t = lane; t < 144; t += 32) X[(t >> 2) * 7 + 2 * (t & 3)] = rn_one(C[(t >> 2) * 6 + (t & 3) + 1]);
    __syncwarp();
    // y: 6 coarse planes x 3 odd b x 7 a, and x 4 even b x 7 a
    if (L.interp) {
#pragma unroll
        for (int j = 0; j < 5; j++) {
            const int pr = L.g + 10 * j;
            if (pr < 42) {
                const int k = pr / 7, a = pr % 7;
                double acc = 0.0;
#pragma unroll
                for (int jj = 0; jj < 6; jj++) acc = __dadd_rn(acc, __dmul_rn(L.w[jj], X[(k * 6 + jj) * 7 + a]));
                Y[(k * 7 + 2 * L.rho + 1) * 7 + a] = acc;
            }
        }
    }
    for (int t = lane; t < 168; t += 32) {
        const int a = t % 7, be = (t / 7) % 4, k = t / 28;
        Y[(k * 7 + 2 * be) * 7 + a] = rn_one(X[(k * 6 + be + 1) * 7 + a]);
    }
    __syncwarp();
    // z and the residuals: odd c by role, then even c with an odd a or b
    if (L.interp) {
        const int c = 2 * L.rho + 1;
#pragma unroll
        for (int j = 0; j < 5; j++) {
            const int pr = L.g + 10 * j;
            if (pr < 49) {
                const int bb = pr / 7, a = pr % 7;
                double z = 0.0;
#pragma unroll
                for (int k = 0; k < 6; k++) z = __dadd_rn(z, __dmul_rn(L.w[k], Y[(k * 7 + bb) * 7 + a]));
                const double wv = __dsub_rn(uo[j], z);
                SQ[wav_q(a, bb, c)] = __dmul_rn(wv, wv);
            }
        }
    }
#pragma unroll
    for (int r = 0; r < 5; r++) {
        const int t = lane + 32 * r;
        if (t < 132) {
            const int ba = pairs[t % 33], ce = t / 33;
            const int bb = ba / 7, a = ba % 7;
            const double wv = __dsub_rn(ue[r], rn_one(Y[((ce + 1) * 7 + bb) * 7 + a]));
            SQ[wav_q(a, bb, 2 * ce)] = __dmul_rn(wv, wv);
        }
    }
    __syncwarp();
    double part = 0.0;
    for (int q = lane; q < 279; q += 32) part = __dadd_rn(part, SQ[q]);
    double tot = 0.0;
    for (int l = 0; l < 32; l++) tot = __dadd_rn(tot, __shfl_sync(0xffffffffu, part, l));
    return tot;
}

// Work items are (element, variable) pairs, variable fastest: every element
// of the mesh (list == nullptr), or the elements listed in list[0, *count)
// (the blocks a decision sends to the exact test).  Warps stride over the
// items, so a list launch runs on a grid sized for the GPU.
__global__ void __launch_bounds__(32 * kWavWarps) wavelet_kernel(ConstVars U, int nvars,
                                                                 const BssnBlockDesc* __restrict__ blocks,
                                                                 const ElemRef* __restrict__ elems,
                                                                 int64_t nelem, const int32_t* __restrict__ list,
                                                                 const int64_t* __restrict__ count,
                                                                 double* __restrict__ scores) {
    __shared__ double sbuf[kWavWarps][kWavC + kWavX + kWavY];
    __shared__ uint8_t spairs[33];
    if (threadIdx.x < 49) {
        // b-major list of the (b, a) pairs with an odd coordinate
        const int b = threadIdx.x / 7, a = threadIdx.x % 7;
        if ((a | b) & 1) {
            int k = 0;
            for (int x = 0; x < (int)threadIdx.x; x++) k += ((x % 7) | (x / 7)) & 1;
            spairs[k] = (uint8_t)threadIdx.x;
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WavLane L;
    L.interp = lane < 30;
    L.rho = lane % 3;
    L.g = lane / 3;
#pragma unroll
    for (int i = 0; i < 6; i++) L.w[i] = kWfine[L.rho][i];
    const int64_t items = (list ? *count : nelem) * nvars;
    for (int64_t wid = (int64_t)blockIdx.x * kWavWarps + warp; wid < items;
         wid += (int64_t)gridDim.x * kWavWarps) {
        const int64_t e = list ? (int64_t)list[wid / nvars] : wid / nvars;
        const int v = (int)(wid % nvars);
        const ElemRef er = elems[e];
        const BssnBlockDesc b = blocks[er.blk];
        const int64_t s = b.sz;
        const double* p = U.p[v] + b.offset + 6 * er.o[0] + s * (6 * er.o[1]) + s * s * (6 * er.o[2]);
        const double tot = wavelet_item(p, s, L, spairs, sbuf[warp], lane);
        if (lane == 0) scores[e * nvars + v] = __dsqrt_rn(__ddiv_rn(tot, 279.0));
        __syncwarp();  // the next item overwrites this warp's buffers
    }
}

// Element list of the blocks with need[b] set: one CTA scans the per-block
// element counts into offsets (off[b]) and the total (*count) ...  With
// first == nullptr every entry counts one (need[] is per element, and the
// list is of the entries themselves).
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) need_scan_kernel(const uint8_t* __restrict__ need,
                                                                 const int64_t* __restrict__ first, int nblk,
                                                                 int64_t* __restrict__ off,
                                                                 int64_t* __restrict__ count) {
    __shared__ int64_t wsum[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int per = (nblk + kScanThreads - 1) / kScanThreads;
    const int b0 = min(nblk, t * per), b1 = min(nblk, b0 + per);
    int64_t mine = 0;
    for (int b = b0; b < b1; b++) mine += need[b] ? (first ? first[b + 1] - first[b] : 1) : 0;
    int64_t x = mine;  // inclusive scan over the warp
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t z = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        wsum[lane] = z;
    }
    __syncthreads();
    int64_t run = x - mine + (w > 0 ? wsum[w - 1] : 0);
    for (int b = b0; b < b1; b++) {
        off[b] = run;
        run += need[b] ? (first ? first[b + 1] - first[b] : 1) : 0;
    }
    if (t == kScanThreads - 1) *count = run;
}

// ... and one warp per listed block writes its element numbers there.
__global__ void __launch_bounds__(256) need_list_kernel(const uint8_t* __restrict__ need,
                                                        const int64_t* __restrict__ first, int nblk,
                                                        const int64_t* __restrict__ off,
                                                        int32_t* __restrict__ list) {
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nblk || !need[b]) return;
    if (!first) {
        if (lane == 0) list[off[b]] = b;
        return;
    }
    const int64_t n = first[b + 1] - first[b];
    for (int64_t i = lane; i < n; i += 32) list[off[b] + i] = (int32_t)(first[b] + i);
}

// Per block: the largest score over its elements and variables divided by
// the tolerance, and the refine flag (ratio > 1).  One warp per block; the
// maximum does not depend on the order its lanes take.
__global__ void __launch_bounds__(256) block_flags_kernel(const double* __restrict__ scores, int nvars,
                                                          const int64_t* __restrict__ first,
                                                          int nblk, double tol, double* ratio,
                                                          uint8_t* flags, const uint8_t* need) {
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nblk || (need && !need[b])) return;  // whole warp
    double m = 0.0;
    const int64_t lo = first[b] * nvars, hi = first[b + 1] * nvars;
    for (int64_t q = lo + lane; q < hi; q += 32) m = fmax(m, scores[q]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) {
        const double r = m / tol;
        if (ratio) ratio[b] = r;
        if (flags) flags[b] = r > 1.0 ? 1 : 0;
    }
}

// Block features (16 floats) from chi, alpha, K and Gt^i on the even
// sublattice of each block's interior (every second point along each axis),
// with differences over two points: max |d chi| and |d alpha| per axis, max
// |K|, max |Gt^i|, the largest second differences of chi and alpha, the
// smallest chi; plus level, block side and spacing.  The sublattice touches
// a quarter of the rows of six of the 24 variables, a small fraction of what
// the exact test reads.  The maxima and the minimum are taken over runs of
// kFeatChunk sublattice points, one warp per run (a 13^3 block is one run of
// 64, a 55^3 block 62 runs), then per block over its runs; neither depends
// on the order.
constexpr int kFeatChunk = 256;

__host__ __device__ inline int64_t feature_points(int sz) {
    const int64_t n = (sz - 6 + 1) / 2;
    return n * n * n;
}

__global__ void __launch_bounds__(256) features_partial_kernel(ConstVars U,
                                                               const BssnBlockDesc* __restrict__ blocks,
                                                               const Chunk* __restrict__ chunks, int nchunks,
                                                               double* __restrict__ part) {
    const int ci = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (ci >= nchunks) return;  // whole warp
    const Chunk ch = chunks[ci];
    const BssnBlockDesc b = blocks[ch.blk];
    const int s = b.sz, n = (s - 6 + 1) / 2;
    const int64_t st[3] = {2, 2 * s, 2 * (int64_t)s * s};
    const double* chi = U.p[U_CHI];
    const double* al = U.p[U_ALPHA];
    double mx[15];
    for (int f = 0; f < 15; f++) mx[f] = 0.0;
    double chimin = 1e300;
    for (int64_t q = ch.start + lane; q < ch.start + ch.count; q += 32) {
        const int i = 3 + 2 * (int)(q % n), j = 3 + 2 * (int)((q / n) % n), k = 3 + 2 * (int)(q / ((int64_t)n * n));
        const int64_t p = b.offset + i + s * (j + (int64_t)s * k);
        const double c0 = chi[p], a0 = al[p];
        for (int d = 0; d < 3; d++) {
            const double cp = chi[p + st[d]], cm = chi[p - st[d]];
            const double ap = al[p + st[d]], am = al[p - st[d]];
            mx[d] = fmax(mx[d], fabs(__dmul_rn(__dsub_rn(cp, cm), 0.25)));
            mx[3 + d] = fmax(mx[3 + d], fabs(__dmul_rn(__dsub_rn(ap, am), 0.25)));
            mx[7 + d] = fmax(mx[7 + d], fabs(U.p[U_GT0 + d][p]));
            mx[13] = fmax(mx[13], fabs(__dsub_rn(__dsub_rn(cp, c0), __dsub_rn(c0, cm))));
            mx[14] = fmax(mx[14], fabs(__dsub_rn(__dsub_rn(ap, a0), __dsub_rn(a0, am))));
        }
        mx[6] = fmax(mx[6], fabs(U.p[U_K][p]));
        chimin = fmin(chimin, c0);
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int f = 0; f < 15; f++) mx[f] = fmax(mx[f], __shfl_xor_sync(0xffffffffu, mx[f], o));
        chimin = fmin(chimin, __shfl_xor_sync(0xffffffffu, chimin, o));
    }
    // lane f < 15 writes maximum f, lane 15 the minimum (static indices only)
    double mine = chimin;
#pragma unroll
    for (int f = 0; f < 15; f++)
        if (lane == f) mine = mx[f];
    if (lane < 16) part[(int64_t)ci * 16 + lane] = mine;
}

// One warp per block: reduce the block's runs, then the 16 features.
__global__ void __launch_bounds__(256) features_final_kernel(const BssnBlockDesc* __restrict__ blocks,
                                                             const double* __restrict__ part,
                                                             const int64_t* __restrict__ first, int nblk,
                                                             float* __restrict__ feats) {
    const int bi = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (bi >= nblk) return;
    double r[16];
    for (int f = 0; f < 15; f++) r[f] = 0.0;
    r[15] = 1e300;
    for (int64_t c = first[bi] + lane; c < first[bi + 1]; c += 32) {
        for (int f = 0; f < 15; f++) r[f] = fmax(r[f], part[c * 16 + f]);
        r[15] = fmin(r[15], part[c * 16 + 15]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int f = 0; f < 15; f++) r[f] = fmax(r[f], __shfl_xor_sync(0xffffffffu, r[f], o));
        r[15] = fmin(r[15], __shfl_xor_sync(0xffffffffu, r[15], o));
    }
    if (lane == 0) {
        const BssnBlockDesc b = blocks[bi];
        const int s = b.sz;
        float* f = feats + (int64_t)bi * 16;
        for (int q = 0; q < 10; q++) f[q] = (float)log10(r[q] + 1e-30);
        const double h = (b.ptmax[0] - b.ptmin[0]) / (s - 1);
        f[10] = (float)b.level;
        f[11] = (float)(s / 55.0);
        f[12] = (float)log10(r[15]);
        f[13] = (float)log10(r[13] + 1e-30);
        f[14] = (float)log10(r[14] + 1e-30);
        f[15] = (float)log10(h);
    }
}

// Element features (16 floats per element): the block features' definitions
// taken over one element's own sublattice, the nodes with even local index
// (0, 2, 4, 6 along each axis: 64 points, padded coordinates 3 + 6 o + 2 m);
// level, side and spacing are its block's.  One warp per element.
__global__ void __launch_bounds__(256) element_features_kernel(ConstVars U,
                                                               const BssnBlockDesc* __restrict__ blocks,
                                                               const ElemRef* __restrict__ elems, int64_t nelem,
                                                               float* __restrict__ feats) {
    const int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= nelem) return;  // whole warp
    const ElemRef er = elems[e];
    const BssnBlockDesc b = blocks[er.blk];
    const int s = b.sz;
    const int64_t st[3] = {2, 2 * s, 2 * (int64_t)s * s};
    const double* chi = U.p[U_CHI];
    const double* al = U.p[U_ALPHA];
    double mx[15];
    for (int f = 0; f < 15; f++) mx[f] = 0.0;
    double chimin = 1e300;
    for (int q = lane; q < 64; q += 32) {
        const int i = 3 + 6 * er.o[0] + 2 * (q & 3), j = 3 + 6 * er.o[1] + 2 * ((q >> 2) & 3),
                  k = 3 + 6 * er.o[2] + 2 * (q >> 4);
        const int64_t p = b.offset + i + s * (j + (int64_t)s * k);
        const double c0 = chi[p], a0 = al[p];
        for (int d = 0; d < 3; d++) {
            const double cp = chi[p + st[d]], cm = chi[p - st[d]];
            const double ap = al[p + st[d]], am = al[p - st[d]];
            mx[d] = fmax(mx[d], fabs(__dmul_rn(__dsub_rn(cp, cm), 0.25)));
            mx[3 + d] = fmax(mx[3 + d], fabs(__dmul_rn(__dsub_rn(ap, am), 0.25)));
            mx[7 + d] = fmax(mx[7 + d], fabs(U.p[U_GT0 + d][p]));
            mx[13] = fmax(mx[13], fabs(__dsub_rn(__dsub_rn(cp, c0), __dsub_rn(c0, cm))));
            mx[14] = fmax(mx[14], fabs(__dsub_rn(__dsub_rn(ap, a0), __dsub_rn(a0, am))));
        }
        mx[6] = fmax(mx[6], fabs(U.p[U_K][p]));
        chimin = fmin(chimin, c0);
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int f = 0; f < 15; f++) mx[f] = fmax(mx[f], __shfl_xor_sync(0xffffffffu, mx[f], o));
        chimin = fmin(chimin, __shfl_xor_sync(0xffffffffu, chimin, o));
    }
    if (lane == 0) {
        float* f = feats + e * 16;
        for (int q = 0; q < 10; q++) f[q] = (float)log10(mx[q] + 1e-30);
        const double h = (b.ptmax[0] - b.ptmin[0]) / (s - 1);
        f[10] = (float)b.level;
        f[11] = (float)(s / 55.0);
        f[12] = (float)log10(chimin);
        f[13] = (float)log10(mx[13] + 1e-30);
        f[14] = (float)log10(mx[14] + 1e-30);
        f[15] = (float)log10(h);
    }
}

// Block flags from element decisions, one warp per block: an element the
// exact test ran on (need) takes its flags from its largest score over the
// variables (ratio = max / tol: refine above 1, keep above keep_fac), the
// others the networks' decisions; a block refines (keeps) when any of its
// elements does.  stats as remesh_merge2_kernel's, counted per element.
__global__ void __launch_bounds__(256) remesh_merge_elem_kernel(int nblk, const int64_t* __restrict__ first,
                                                                const uint8_t* __restrict__ need,
                                                                const uint8_t* __restrict__ decided,
                                                                const double* __restrict__ scores, int nvars,
                                                                double tol, double keep_fac,
                                                                const float* __restrict__ lr,
                                                                const float* __restrict__ lk, float lo_r,
                                                                float lo_k, int* stats, uint8_t* flags_r,
                                                                uint8_t* flags_k) {
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nblk) return;  // whole warp
    unsigned fr = 0, fk = 0;
    for (int64_t e = first[b] + lane; e < first[b + 1]; e += 32) {
        if (need[e]) {
            double m = 0.0;
            for (int v = 0; v < nvars; v++) m = fmax(m, scores[e * nvars + v]);
            const double r = m / tol;
            const unsigned er = r > 1.0 ? 1u : 0u, ek = r > keep_fac ? 1u : 0u;
            fr |= er;
            fk |= ek;
            const float pr = 1.0f / (1.0f + expf(-lr[e])), pk = 1.0f / (1.0f + expf(-lk[e]));
            if (pr <= lo_r && er) atomicAdd(&stats[3], 1);
            if (er) atomicAdd(&stats[4], 1);
            if (pk <= lo_k && ek) atomicAdd(&stats[5], 1);
            if (ek) atomicAdd(&stats[6], 1);
        } else {
            fr |= decided[e] & 1u;
            fk |= (decided[e] >> 1) & 1u;
        }
    }
    fr = __any_sync(0xffffffffu, fr) ? 1u : 0u;
    fk = __any_sync(0xffffffffu, fk) ? 1u : 0u;
    if (lane == 0) {
        flags_r[b] = (uint8_t)fr;
        flags_k[b] = (uint8_t)fk;
    }
}

// ---------------------------------------------------------------------------
// MLP 16 -> 64 -> 64 -> 1.  Parameter layout (MLP_NPARAM values):
//   W1[64][16], b1[64], W2[64][64], b2[64], W3[64], b3
// Compute copies are BF16; all arithmetic accumulates in FP32.
// ---------------------------------------------------------------------------
constexpr int IN = 16, HID = 64;
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID,
              OW3 = OB2 + HID, OB3 = OW3 + HID;

__device__ __forceinline__ float gelu(float a) { return 0.5f * a * (1.0f + erff(a * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float a) {
    const float cdf = 0.5f * (1.0f + erff(a * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * a * a);
    return cdf + a * pdf;
}

constexpr int MLP_THREADS = 128;

// Forward for one sample per thread; parameters staged into shared memory
// as FP32 (converted from BF16 once per CTA).
__global__ void __launch_bounds__(MLP_THREADS) mlp_fwd_kernel(const __nv_bfloat16* __restrict__ wq,
                                                              const float* __restrict__ norm,
                                                              const float* __restrict__ X, int n,
                                                              float* __restrict__ logits) {
    __shared__ float w[MLP_NPARAM];
    for (int q = threadIdx.x; q < MLP_NPARAM; q += blockDim.x) w[q] = __bfloat162float(wq[q]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[IN], h1[HID];
    for (int k = 0; k < IN; k++) {
        const float xv = X[(int64_t)i * IN + k];
        x[k] = norm ? (xv - norm[k]) * norm[IN + k] : xv;
    }
    for (int o = 0; o < HID; o++) {
        float a = w[OB1 + o];
        for (int k = 0; k < IN; k++) a = fmaf(w[OW1 + o * IN + k], x[k], a);
        h1[o] = gelu(a);
    }
    float out = w[OB3];
    for (int o = 0; o < HID; o++) {
        float a = w[OB2 + o];
        for (int k = 0; k < HID; k++) a = fmaf(w[OW2 + o * HID + k], h1[k], a);
        out = fmaf(w[OW3 + o], gelu(a), out);
    }
    logits[i] = out;
}

// Forward on the tensor cores: mma.sync m16n8k16 with BF16 operands and FP32
// accumulation.  A warp evaluates 32 samples (two 16-row tiles): layer 1
// (16 -> 64) is one k-step of 8 n-tiles, its accumulators go through bias +
// GELU and, converted to BF16, are directly the A operands of layer 2
// (64 -> 64; the m16n8 accumulator layout of two adjacent n-tiles is the
// m16k16 A layout of one k-step), and the output layer (64 -> 1) is a dot
// product summed over the four threads that share a row.  The inputs and
// the hidden activations are rounded to BF16 as the operands require; every
// sum accumulates in FP32.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(MLP_THREADS) mlp_fwd_mma_kernel(const __nv_bfloat16* __restrict__ wq,
                                                                  const float* __restrict__ norm,
                                                                  const float* __restrict__ X, int n,
                                                                  float* __restrict__ logits) {
    // BF16 weights as loaded (W1 [64][16], W2 [64][64] row-major by output),
    // FP32 biases and output weights
    __shared__ __align__(16) __nv_bfloat16 w1[HID * IN], w2[HID * HID];
    __shared__ float b1[HID], b2[HID], w3[HID], b3;
    __shared__ float nm[2 * IN];
    for (int q = threadIdx.x; q < HID * IN; q += blockDim.x) w1[q] = wq[OW1 + q];
    for (int q = threadIdx.x; q < HID * HID; q += blockDim.x) w2[q] = wq[OW2 + q];
    for (int q = threadIdx.x; q < HID; q += blockDim.x) {
        b1[q] = __bfloat162float(wq[OB1 + q]);
        b2[q] = __bfloat162float(wq[OB2 + q]);
        w3[q] = __bfloat162float(wq[OW3 + q]);
    }
    if (threadIdx.x == 0) b3 = __bfloat162float(wq[OB3]);
    if (threadIdx.x < 2 * IN) nm[threadIdx.x] = norm ? norm[threadIdx.x] : (threadIdx.x < IN ? 0.0f : 1.0f);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int base = (blockIdx.x * blockDim.x + (threadIdx.x & ~31));  // first sample of the warp
    auto xin = [&](int row, int k) {
        const int i = base + row;
        return i < n ? (X[(int64_t)i * IN + k] - nm[k]) * nm[IN + k] : 0.0f;
    };
    auto wpair = [&](const __nv_bfloat16* w, int ld, int row, int col) {
        return *reinterpret_cast<const uint32_t*>(w + row * ld + col);
    };
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        // layer 1: A = normalised inputs (rows r0, r1; features 2t.., 2t+8..)
        const uint32_t a1[4] = {pack_bf16(xin(r0, 2 * t), xin(r0, 2 * t + 1)),
                                pack_bf16(xin(r1, 2 * t), xin(r1, 2 * t + 1)),
                                pack_bf16(xin(r0, 2 * t + 8), xin(r0, 2 * t + 9)),
                                pack_bf16(xin(r1, 2 * t + 8), xin(r1, 2 * t + 9))};
        float h[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            h[nt][0] = h[nt][1] = h[nt][2] = h[nt][3] = 0.0f;
            mma_bf16_16816(h[nt], a1, wpair(w1, IN, nt * 8 + g, 2 * t), wpair(w1, IN, nt * 8 + g, 2 * t + 8));
            const int c = nt * 8 + 2 * t;
            h[nt][0] = gelu(h[nt][0] + b1[c]);
            h[nt][1] = gelu(h[nt][1] + b1[c + 1]);
            h[nt][2] = gelu(h[nt][2] + b1[c]);
            h[nt][3] = gelu(h[nt][3] + b1[c + 1]);
        }
        // layer 2: A k-step kt = the activations of layer-1 n-tiles 2kt, 2kt+1
        float o0 = 0.0f, o1 = 0.0f;  // output-layer partial sums of rows r0, r1
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int kt = 0; kt < 4; kt++) {
                const uint32_t a2[4] = {pack_bf16(h[2 * kt][0], h[2 * kt][1]), pack_bf16(h[2 * kt][2], h[2 * kt][3]),
                                        pack_bf16(h[2 * kt + 1][0], h[2 * kt + 1][1]),
                                        pack_bf16(h[2 * kt + 1][2], h[2 * kt + 1][3])};
                mma_bf16_16816(d, a2, wpair(w2, HID, nt * 8 + g, kt * 16 + 2 * t),
                               wpair(w2, HID, nt * 8 + g, kt * 16 + 2 * t + 8));
            }
            const int c = nt * 8 + 2 * t;
            o0 = fmaf(w3[c], gelu(d[0] + b2[c]), o0);
            o0 = fmaf(w3[c + 1], gelu(d[1] + b2[c + 1]), o0);
            o1 = fmaf(w3[c], gelu(d[2] + b2[c]), o1);
            o1 = fmaf(w3[c + 1], gelu(d[3] + b2[c + 1]), o1);
        }
        o0 += __shfl_xor_sync(0xffffffffu, o0, 1);
        o0 += __shfl_xor_sync(0xffffffffu, o0, 2);
        o1 += __shfl_xor_sync(0xffffffffu, o1, 1);
        o1 += __shfl_xor_sync(0xffffffffu, o1, 2);
        if (t == 0) {
            if (base + r0 < n) logits[base + r0] = o0 + b3;
            if (base + r1 < n) logits[base + r1] = o1 + b3;
        }
    }
}

// Forward + backward of the weighted binary cross-entropy
//   L = sum_i c_i * BCE(sigmoid(z_i), y_i) / n
// for MLP_THREADS samples per CTA (one per thread).  Each CTA writes its
// gradient partial (MLP_NPARAM floats, summed over its samples in sample
// order) and its loss partial; mlp_reduce_kernel adds the partials in CTA
// order, so a training run is deterministic.
__global__ void __launch_bounds__(MLP_THREADS) mlp_grad_kernel(const __nv_bfloat16* __restrict__ wq,
                                                               const float* __restrict__ norm,
                                                               const float* __restrict__ X,
                                                               const float* __restrict__ Y,
                                                               const float* __restrict__ C, int n,
                                                               float* __restrict__ gpart,
                                                               float* __restrict__ lpart) {
    extern __shared__ float sm[];
    float* w = sm;                          // MLP_NPARAM
    float* XS = w + MLP_NPARAM;             // [T][IN]   inputs
    float* H1 = XS + MLP_THREADS * IN;      // [T][HID]  gelu(a1)
    float* D1 = H1 + MLP_THREADS * HID;     // [T][HID]  dL/da1
    float* D2 = D1 + MLP_THREADS * HID;     // [T][HID]  a2, then dL/da2
    float* H2 = D2 + MLP_THREADS * HID;     // [T][HID]  gelu(a2), then dz*gelu(a2)
    float* DZ = H2 + MLP_THREADS * HID;     // [T]       dL/dz
    float* LS = DZ + MLP_THREADS;           // [T]       loss terms
    const int t = threadIdx.x;
    for (int q = t; q < MLP_NPARAM; q += blockDim.x) w[q] = __bfloat162float(wq[q]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + t;
    const bool valid = i < n;
    float* xs = XS + t * IN;
    float* h1 = H1 + t * HID;
    float* d1 = D1 + t * HID;
    float* d2 = D2 + t * HID;
    float* h2 = H2 + t * HID;
    for (int k = 0; k < IN; k++) {
        const float xv = valid ? X[(int64_t)i * IN + k] : 0.0f;
        xs[k] = norm ? (xv - norm[k]) * norm[IN + k] : xv;
    }
    for (int o = 0; o < HID; o++) {
        float a = w[OB1 + o];
        for (int k = 0; k < IN; k++) a = fmaf(w[OW1 + o * IN + k], xs[k], a);
        d1[o] = a;  // a1 for now
        h1[o] = gelu(a);
    }
    float z = w[OB3];
    for (int o = 0; o < HID; o++) {
        float a = w[OB2 + o];
        for (int k = 0; k < HID; k++) a = fmaf(w[OW2 + o * HID + k], h1[k], a);
        d2[o] = a;
        h2[o] = gelu(a);
        z = fmaf(w[OW3 + o], h2[o], z);
    }
    float dz = 0.0f, loss = 0.0f;
    if (valid) {
        const float y = Y[i], c = C ? C[i] : 1.0f;
        // numerically stable BCE with logits
        loss = c * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)))) / n;
        dz = c * (1.0f / (1.0f + expf(-z)) - y) / n;
    }
    DZ[t] = dz;
    LS[t] = loss;
    for (int o = 0; o < HID; o++) {
        d2[o] = dz * w[OW3 + o] * gelu_grad(d2[o]);  // dL/da2
        h2[o] *= dz;                                 // dL/dW3[o] contribution
    }
    for (int k = 0; k < HID; k++) {
        float g = 0.0f;
        for (int o = 0; o < HID; o++) g = fmaf(w[OW2 + o * HID + k], d2[o], g);
        d1[k] = g * gelu_grad(d1[k]);  // dL/da1
    }
    __syncthreads();
    // thread t owns parameters t, t+T, ...: sums over the CTA's samples
    float* gp = gpart + (int64_t)blockIdx.x * MLP_NPARAM;
    for (int q = t; q < MLP_NPARAM; q += blockDim.x) {
        float g = 0.0f;
        if (q < OB1) {
            const int o = q / IN, k = q % IN;
            for (int r = 0; r < MLP_THREADS; r++) g = fmaf(D1[r * HID + o], XS[r * IN + k], g);
        } else if (q < OW2) {
            const int o = q - OB1;
            for (int r = 0; r < MLP_THREADS; r++) g += D1[r * HID + o];
        } else if (q < OB2) {
            const int o = (q - OW2) / HID, k = (q - OW2) % HID;
            for (int r = 0; r < MLP_THREADS; r++) g = fmaf(D2[r * HID + o], H1[r * HID + k], g);
        } else if (q < OW3) {
            const int o = q - OB2;
            for (int r = 0; r < MLP_THREADS; r++) g += D2[r * HID + o];
        } else if (q < OB3) {
            const int o = q - OW3;
            for (int r = 0; r < MLP_THREADS; r++) g += H2[r * HID + o];
        } else {
            for (int r = 0; r < MLP_THREADS; r++) g += DZ[r];
        }
        gp[q] = g;
    }
    if (t == 0) {
        float l = 0.0f;
        for (int r = 0; r < MLP_THREADS; r++) l += LS[r];
        lpart[blockIdx.x] = l;
    }
}

__global__ void __launch_bounds__(MLP_THREADS) mlp_reduce_kernel(const float* __restrict__ gpart, int nparts,
                                                                  float* __restrict__ grad) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= MLP_NPARAM) return;
    float g = 0.0f;
    for (int p = 0; p < nparts; p++) g += gpart[(int64_t)p * MLP_NPARAM + q];
    grad[q] = g;
}

__global__ void mlp_loss_reduce_kernel(const float* lpart, int nparts, float* loss) {
    if (threadIdx.x || blockIdx.x) return;
    float l = 0.0f;
    for (int p = 0; p < nparts; p++) l += lpart[p];
    *loss = l;
}

__global__ void __launch_bounds__(256) adam_kernel(float* __restrict__ master, __nv_bfloat16* __restrict__ wq,
                                                   const float* __restrict__ grad, float* __restrict__ m,
                                                   float* __restrict__ v, float lr, float b1, float b2,
                                                   float eps, float bc1, float bc2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= MLP_NPARAM) return;
    const float g = grad[q];
    const float mq = b1 * m[q] + (1.0f - b1) * g;
    const float vq = b2 * v[q] + (1.0f - b2) * g * g;
    m[q] = mq;
    v[q] = vq;
    const float p = master[q] - lr * (mq / bc1) / (sqrtf(vq / bc2) + eps);
    master[q] = p;
    wq[q] = __float2bfloat16_rn(p);
}


__device__ __forceinline__ uint64_t hmix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Decide from the network where it is confident; mark for the exact test
// the uncertain blocks (lo < p < hi) and a seeded audit sample.
// stats[0] += uncertain, stats[1] += audited.
__global__ void __launch_bounds__(256) remesh_select_kernel(const float* __restrict__ logits, int nblk,
                                                            float lo, float hi, double audit_frac,
                                                            uint64_t seed, uint8_t* need,
                                                            uint8_t* decided, int* stats) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    const float p = 1.0f / (1.0f + expf(-logits[b]));
    const bool unsure = p > lo && p < hi;
    const double u = (double)(hmix(seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(b + 1)) >> 11) *
                     (1.0 / 9007199254740992.0);
    const bool audit = u < audit_frac;
    need[b] = (unsure || audit) ? 1 : 0;
    decided[b] = p >= hi ? 1 : 0;
    if (unsure) atomicAdd(&stats[0], 1);
    if (audit && !unsure) atomicAdd(&stats[1], 1);
}

// Final flags: the exact result where the exact test ran, the network's
// decision elsewhere.  stats[2] += audited blocks the network alone would
// have missed (p <= lo but the exact test refines), stats[3] += audited
// blocks the exact test refines.
__global__ void __launch_bounds__(256) remesh_merge_kernel(int nblk, const uint8_t* need,
                                                           const uint8_t* decided,
                                                           const uint8_t* exact,
                                                           const float* logits, float lo,
                                                           int* stats, uint8_t* flags) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    if (need[b]) {
        flags[b] = exact[b];
        const float p = 1.0f / (1.0f + expf(-logits[b]));
        if (p <= lo && exact[b]) atomicAdd(&stats[2], 1);
        if (exact[b]) atomicAdd(&stats[3], 1);
    } else {
        flags[b] = decided[b];
    }
}

// Two-flag decision (refine at tol, keep at keep_fac * tol) in one pass:
// the exact test runs once on the union of both networks' uncertain blocks
// and one seeded audit sample.  stats (8 ints): uncertain for refine,
// uncertain for keep, extra audited blocks, audited refine misses, audited
// exact refines, audited keep misses, audited exact keeps, 0.
__global__ void __launch_bounds__(256) remesh_select2_kernel(const float* __restrict__ lr,
                                                             const float* __restrict__ lk, int nblk,
                                                             float lo_r, float hi_r, float lo_k,
                                                             float hi_k, double audit_frac,
                                                             uint64_t seed, uint8_t* need,
                                                             uint8_t* decided, int* stats) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    const float pr = 1.0f / (1.0f + expf(-lr[b])), pk = 1.0f / (1.0f + expf(-lk[b]));
    // refine implies keep (score > tol > keep_fac tol): a confident refine
    // settles keep, a confident "no keep" settles refine
    const bool refine_sure = pr >= hi_r, nokeep_sure = pk <= lo_k;
    const bool ur = pr > lo_r && pr < hi_r && !nokeep_sure;
    const bool uk = pk > lo_k && pk < hi_k && !refine_sure;
    const double u = (double)(hmix(seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(b + 1)) >> 11) *
                     (1.0 / 9007199254740992.0);
    const bool audit = u < audit_frac;
    need[b] = (ur || uk || audit) ? 1 : 0;
    decided[b] = (refine_sure && !nokeep_sure ? 1 : 0) | (pk >= hi_k || refine_sure ? 2 : 0);
    if (ur) atomicAdd(&stats[0], 1);
    if (uk) atomicAdd(&stats[1], 1);
    if (audit && !ur && !uk) atomicAdd(&stats[2], 1);
}

// Per element, as remesh_select2_kernel, but keeping the reasons apart for
// remesh_settle_elem_kernel: need bit 0 = unsure for refine, bit 1 = unsure
// for keep, bit 2 = audited.
__global__ void __launch_bounds__(256) remesh_select_elem_kernel(const float* __restrict__ lr,
                                                                 const float* __restrict__ lk, int n,
                                                                 float lo_r, float hi_r, float lo_k,
                                                                 float hi_k, double audit_frac,
                                                                 uint64_t seed, uint8_t* need,
                                                                 uint8_t* decided) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float pr = 1.0f / (1.0f + expf(-lr[e])), pk = 1.0f / (1.0f + expf(-lk[e]));
    const bool refine_sure = pr >= hi_r, nokeep_sure = pk <= lo_k;
    const bool ur = pr > lo_r && pr < hi_r && !nokeep_sure;
    const bool uk = pk > lo_k && pk < hi_k && !refine_sure;
    const double u = (double)(hmix(seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(e + 1)) >> 11) *
                     (1.0 / 9007199254740992.0);
    need[e] = (ur ? 1 : 0) | (uk ? 2 : 0) | (u < audit_frac ? 4 : 0);
    decided[e] = (refine_sure && !nokeep_sure ? 1 : 0) | (pk >= hi_k || refine_sure ? 2 : 0);
}

// One warp per block.  A block takes a flag when any of its elements does, so
// once the networks refine (keep) one of its elements, its other elements
// are tested only for a flag still open: need becomes 1 for an element unsure
// of an open flag or audited, else 0.  stats[0..2] += elements sent for
// refine, for keep, audited only.
__global__ void __launch_bounds__(256) remesh_settle_elem_kernel(int nblk, const int64_t* __restrict__ first,
                                                                 uint8_t* need,
                                                                 const uint8_t* __restrict__ decided,
                                                                 int* stats) {
    const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nblk) return;  // whole warp
    unsigned any = 0;
    for (int64_t e = first[b] + lane; e < first[b + 1]; e += 32) any |= decided[e] & 3u;
    for (int o = 16; o > 0; o >>= 1) any |= __shfl_xor_sync(0xffffffffu, any, o);
    const bool rs = any & 1u, ks = any & 2u;
    int cr = 0, ck = 0, ca = 0;
    for (int64_t e0 = first[b]; e0 < first[b + 1]; e0 += 32) {
        const int64_t e = e0 + lane;
        const bool in = e < first[b + 1];
        const unsigned nb = in ? need[e] : 0u;
        const bool ur = (nb & 1u) && !rs, uk = (nb & 2u) && !rs && !ks, au = nb & 4u;
        if (in) need[e] = (ur || uk || au) ? 1 : 0;
        cr += __popc(__ballot_sync(0xffffffffu, ur));
        ck += __popc(__ballot_sync(0xffffffffu, uk));
        ca += __popc(__ballot_sync(0xffffffffu, au && !ur && !uk));
    }
    if (lane == 0) {
        if (cr) atomicAdd(&stats[0], cr);
        if (ck) atomicAdd(&stats[1], ck);
        if (ca) atomicAdd(&stats[2], ca);
    }
}

// Final flags: from the exact ratio (block max score / tol) where the exact
// test ran, the networks' decisions elsewhere.
__global__ void __launch_bounds__(256) remesh_merge2_kernel(int nblk, const uint8_t* need,
                                                            const uint8_t* decided,
                                                            const double* ratio, double keep_fac,
                                                            const float* lr, const float* lk,
                                                            float lo_r, float lo_k, int* stats,
                                                            uint8_t* flags_r, uint8_t* flags_k) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    if (need[b]) {
        const uint8_t er = ratio[b] > 1.0 ? 1 : 0, ek = ratio[b] > keep_fac ? 1 : 0;
        flags_r[b] = er;
        flags_k[b] = ek;
        const float pr = 1.0f / (1.0f + expf(-lr[b])), pk = 1.0f / (1.0f + expf(-lk[b]));
        if (pr <= lo_r && er) atomicAdd(&stats[3], 1);
        if (er) atomicAdd(&stats[4], 1);
        if (pk <= lo_k && ek) atomicAdd(&stats[5], 1);
        if (ek) atomicAdd(&stats[6], 1);
    } else {
        flags_r[b] = decided[b] & 1;
        flags_k[b] = (decided[b] >> 1) & 1;
    }
}

}  // namespace

int launch_remesh_select2(const float* lr, const float* lk, int nblk, float lo_r, float hi_r,
                          float lo_k, float hi_k, double audit_frac, uint64_t seed, uint8_t* need,
                          uint8_t* decided, int* stats, cudaStream_t s) {
    remesh_select2_kernel<<<(nblk + 255) / 256, 256, 0, s>>>(lr, lk, nblk, lo_r, hi_r, lo_k, hi_k,
                                                             audit_frac, seed, need, decided, stats);
    return cuda_status(cudaGetLastError());
}

int launch_remesh_select_elem(MeshState* m, const float* lr, const float* lk, float lo_r, float hi_r,
                              float lo_k, float hi_k, double audit_frac, uint64_t seed, uint8_t* need_e,
                              uint8_t* decided_e, int* stats, cudaStream_t s) {
    int st = remesh_elements(m);
    if (st) return st;
    const int64_t ne = m->n_elems;
    const int nb = (int)m->blocks.size();
    if (ne == 0) return 0;
    remesh_select_elem_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(lr, lk, (int)ne, lo_r, hi_r, lo_k, hi_k,
                                                                           audit_frac, seed, need_e, decided_e);
    remesh_settle_elem_kernel<<<(unsigned)(((int64_t)nb * 32 + 255) / 256), 256, 0, s>>>(nb, m->d_elem_first,
                                                                                       need_e, decided_e, stats);
    return cuda_status(cudaGetLastError());
}

int launch_remesh_merge2(int nblk, const uint8_t* need, const uint8_t* decided, const double* ratio,
                         double keep_fac, const float* lr, const float* lk, float lo_r, float lo_k,
                         int* stats, uint8_t* flags_r, uint8_t* flags_k, cudaStream_t s) {
    remesh_merge2_kernel<<<(nblk + 255) / 256, 256, 0, s>>>(nblk, need, decided, ratio, keep_fac, lr,
                                                            lk, lo_r, lo_k, stats, flags_r, flags_k);
    return cuda_status(cudaGetLastError());
}

int remesh_elements(MeshState* m) {
    if (m->d_elems) return 0;
    std::vector<ElemRef> e;
    std::vector<int64_t> first(m->blocks.size() + 1, 0);
    for (size_t b = 0; b < m->blocks.size(); b++) {
        const int w = (m->blocks[b].sz - 7) / 6;
        for (int oz = 0; oz < w; oz++)
            for (int oy = 0; oy < w; oy++)
                for (int ox = 0; ox < w; ox++)
                    e.push_back(ElemRef{(int32_t)b, {(int16_t)ox, (int16_t)oy, (int16_t)oz}, 0});
        first[b + 1] = (int64_t)e.size();
    }
    if (cudaMalloc((void**)&m->d_elems, e.size() * sizeof(ElemRef)) != cudaSuccess) return BSSN_ENOMEM;
    if (cudaMalloc((void**)&m->d_elem_first, first.size() * sizeof(int64_t)) != cudaSuccess) return BSSN_ENOMEM;
    if (cudaMalloc((void**)&m->d_need_off, (first.size() + 1) * sizeof(int64_t)) != cudaSuccess) return BSSN_ENOMEM;
    if (cudaMalloc((void**)&m->d_need_list, std::max<size_t>(e.size(), 1) * sizeof(int32_t)) != cudaSuccess)
        return BSSN_ENOMEM;
    m->d_need_count = m->d_need_off + first.size();
    cudaMemcpy(m->d_elems, e.data(), e.size() * sizeof(ElemRef), cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_elem_first, first.data(), first.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
    m->n_elems = (int64_t)e.size();
    return cuda_status(cudaGetLastError());
}

int launch_wavelet_scores(MeshState* m, const double* const* U, int nvars, double* scores,
                          const uint8_t* need, cudaStream_t s) {
    int st = remesh_elements(m);
    if (st) return st;
    ConstVars u = {};
    for (int v = 0; v < nvars; v++) u.p[v] = U[v];
    const int64_t warps = m->n_elems * nvars;
    const int nb = (int)m->blocks.size();
    if (warps == 0) return 0;
    int64_t blocks = (warps + kWavWarps - 1) / kWavWarps;
    if (!need) {
        wavelet_kernel<<<(unsigned)blocks, 32 * kWavWarps, 0, s>>>(u, nvars, m->d_blocks, m->d_elems, m->n_elems,
                                                                  nullptr, nullptr, scores);
        return cuda_status(cudaGetLastError());
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    blocks = std::min<int64_t>(blocks, (int64_t)nsm * 8);
    need_scan_kernel<<<1, kScanThreads, 0, s>>>(need, m->d_elem_first, nb, m->d_need_off, m->d_need_count);
    need_list_kernel<<<(unsigned)(((int64_t)nb * 32 + 255) / 256), 256, 0, s>>>(need, m->d_elem_first, nb,
                                                                              m->d_need_off, m->d_need_list);
    wavelet_kernel<<<(unsigned)blocks, 32 * kWavWarps, 0, s>>>(u, nvars, m->d_blocks, m->d_elems, m->n_elems,
                                                              m->d_need_list, m->d_need_count, scores);
    return cuda_status(cudaGetLastError());
}

int launch_block_flags(MeshState* m, const double* scores, int nvars, double tol, double* ratio,
                       uint8_t* flags, const uint8_t* need, cudaStream_t s) {
    int st = remesh_elements(m);
    if (st) return st;
    const int nb = (int)m->blocks.size();
    block_flags_kernel<<<(unsigned)(((int64_t)nb * 32 + 255) / 256), 256, 0, s>>>(scores, nvars, m->d_elem_first, nb, tol,
                                                                          ratio, flags, need);
    return cuda_status(cudaGetLastError());
}

int launch_element_features(MeshState* m, const double* const* U, float* feats, cudaStream_t s) {
    int st = remesh_elements(m);
    if (st) return st;
    if (m->n_elems == 0) return 0;
    ConstVars u = {};
    for (int v = 0; v < NVARS; v++) u.p[v] = U[v];
    element_features_kernel<<<(unsigned)((m->n_elems * 32 + 255) / 256), 256, 0, s>>>(u, m->d_blocks, m->d_elems,
                                                                                   m->n_elems, feats);
    return cuda_status(cudaGetLastError());
}

int launch_wavelet_elements(MeshState* m, const double* const* U, int nvars, double* scores,
                            const uint8_t* need_e, int64_t* off, int64_t* count, int32_t* list,
                            cudaStream_t s) {
    int st = remesh_elements(m);
    if (st) return st;
    const int64_t ne = m->n_elems;
    if (ne == 0) return 0;
    ConstVars u = {};
    for (int v = 0; v < nvars; v++) u.p[v] = U[v];
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = std::min<int64_t>((ne * nvars + kWavWarps - 1) / kWavWarps, (int64_t)nsm * 8);
    need_scan_kernel<<<1, kScanThreads, 0, s>>>(need_e, nullptr, (int)ne, off, count);
    need_list_kernel<<<(unsigned)((ne * 32 + 255) / 256), 256, 0, s>>>(need_e, nullptr, (int)ne, off, list);
    wavelet_kernel<<<(unsigned)blocks, 32 * kWavWarps, 0, s>>>(u, nvars, m->d_blocks, m->d_elems, ne, list, count,
                                                              scores);
    return cuda_status(cudaGetLastError());
}

int launch_remesh_merge_elem(MeshState* m, const uint8_t* need_e, const uint8_t* decided_e,
                             const double* scores, int nvars, double tol, double keep_fac, const float* lr,
                             const float* lk, float lo_r, float lo_k, int* stats, uint8_t* flags_r,
                             uint8_t* flags_k, cudaStream_t s) {
    int st = remesh_elements(m);
    if (st) return st;
    const int nb = (int)m->blocks.size();
    remesh_merge_elem_kernel<<<(unsigned)(((int64_t)nb * 32 + 255) / 256), 256, 0, s>>>(
        nb, m->d_elem_first, need_e, decided_e, scores, nvars, tol, keep_fac, lr, lk, lo_r, lo_k, stats, flags_r,
        flags_k);
    return cuda_status(cudaGetLastError());
}

int feature_chunks(MeshState* m) {
    if (m->d_fchunks) return 0;
    std::vector<Chunk> c;
    std::vector<int64_t> first(m->blocks.size() + 1, 0);
    for (size_t b = 0; b < m->blocks.size(); b++) {
        const int64_t n = feature_points(m->blocks[b].sz);
        for (int64_t q = 0; q < n; q += kFeatChunk)
            c.push_back(Chunk{(int32_t)b, (int32_t)std::min<int64_t>(kFeatChunk, n - q), q});
        first[b + 1] = (int64_t)c.size();
    }
    if (cudaMalloc((void**)&m->d_fchunks, c.size() * sizeof(Chunk)) != cudaSuccess) return BSSN_ENOMEM;
    if (cudaMalloc((void**)&m->d_fchunk_first, first.size() * sizeof(int64_t)) != cudaSuccess)
        return BSSN_ENOMEM;
    if (cudaMalloc((void**)&m->d_fpart, c.size() * 16 * sizeof(double)) != cudaSuccess) return BSSN_ENOMEM;
    cudaMemcpy(m->d_fchunks, c.data(), c.size() * sizeof(Chunk), cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_fchunk_first, first.data(), first.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
    m->n_fchunks = (int)c.size();
    return cuda_status(cudaGetLastError());
}

int launch_features(MeshState* m, const double* const* U, float* feats, cudaStream_t s) {
    const int nb = (int)m->blocks.size();
    if (nb == 0) return 0;
    int st = feature_chunks(m);
    if (st) return st;
    ConstVars u = {};
    for (int v = 0; v < NVARS; v++) u.p[v] = U[v];
    features_partial_kernel<<<(unsigned)(((int64_t)m->n_fchunks * 32 + 255) / 256), 256, 0, s>>>(
        u, m->d_blocks, m->d_fchunks, m->n_fchunks, m->d_fpart);
    features_final_kernel<<<(unsigned)(((int64_t)nb * 32 + 255) / 256), 256, 0, s>>>(
        m->d_blocks, m->d_fpart, m->d_fchunk_first, nb, feats);
    return cuda_status(cudaGetLastError());
}

int launch_mlp_fwd(const void* wq, const float* norm, const float* X, int n, float* logits,
                   cudaStream_t s) {
    if (n <= 0) return 0;
    mlp_fwd_mma_kernel<<<(n + MLP_THREADS - 1) / MLP_THREADS, MLP_THREADS, 0, s>>>(
        (const __nv_bfloat16*)wq, norm, X, n, logits);
    return cuda_status(cudaGetLastError());
}

int launch_mlp_fwd_fp32(const void* wq, const float* norm, const float* X, int n, float* logits,
                        cudaStream_t s) {
    if (n <= 0) return 0;
    mlp_fwd_kernel<<<(n + MLP_THREADS - 1) / MLP_THREADS, MLP_THREADS, 0, s>>>(
        (const __nv_bfloat16*)wq, norm, X, n, logits);
    return cuda_status(cudaGetLastError());
}

size_t mlp_grad_scratch_floats(int n) {
    const int parts = (n + MLP_THREADS - 1) / MLP_THREADS;
    return (size_t)parts * (MLP_NPARAM + 1);
}

int launch_mlp_grad(const void* wq, const float* norm, const float* X, const float* Y,
                    const float* C, int n, float* grad, float* loss, float* scratch,
                    cudaStream_t s) {
    if (n <= 0) return BSSN_EINVAL;
    const int parts = (n + MLP_THREADS - 1) / MLP_THREADS;
    float* gpart = scratch;
    float* lpart = gpart + (size_t)parts * MLP_NPARAM;
    const size_t smem = sizeof(float) * (MLP_NPARAM + MLP_THREADS * (IN + 4 * HID + 2));
    const int st = set_smem_limit((const void*)mlp_grad_kernel, (int)smem);
    if (st) return st;
    mlp_grad_kernel<<<parts, MLP_THREADS, smem, s>>>((const __nv_bfloat16*)wq, norm, X, Y, C, n, gpart, lpart);
    mlp_reduce_kernel<<<(MLP_NPARAM + MLP_THREADS - 1) / MLP_THREADS, MLP_THREADS, 0, s>>>(gpart, parts, grad);
    if (loss) mlp_loss_reduce_kernel<<<1, 32, 0, s>>>(lpart, parts, loss);
    return cuda_status(cudaGetLastError());
}

int launch_adam(float* master, void* wq, const float* grad, float* m, float* v, float lr, float b1,
                float b2, float eps, int t, cudaStream_t s) {
    const float bc1 = 1.0f - powf(b1, (float)t), bc2 = 1.0f - powf(b2, (float)t);
    adam_kernel<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(master, (__nv_bfloat16*)wq, grad, m, v, lr, b1,
                                                         b2, eps, bc1, bc2);
    return cuda_status(cudaGetLastError());
}

int launch_remesh_select(const float* logits, int nblk, float lo, float hi, double audit_frac,
                         uint64_t seed, uint8_t* need, uint8_t* decided, int* stats,
                         cudaStream_t s) {
    remesh_select_kernel<<<(nblk + 255) / 256, 256, 0, s>>>(logits, nblk, lo, hi, audit_frac, seed,
                                                            need, decided, stats);
    return cuda_status(cudaGetLastError());
}

int launch_remesh_merge(int nblk, const uint8_t* need, const uint8_t* decided,
                        const uint8_t* exact, const float* logits, float lo, int* stats,
                        uint8_t* flags, cudaStream_t s) {
    remesh_merge_kernel<<<(nblk + 255) / 256, 256, 0, s>>>(nblk, need, decided, exact, logits, lo,
                                                           stats, flags);
    return cuda_status(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Gradient without allocation.  Some callers may not allocate device memory
// at the moment they need a gradient: an application that owns every byte of
// device memory through its own pool under a fixed budget and forbids
// libraries to allocate behind its back, or a time-stepping loop that must
// not pay the implicit synchronisation and latency of cudaMalloc / cudaFree,
// nor risk their failure, in the middle of a run.  For them the per-CTA partial sums that
// bssn_remesh_mlp_bwd_bf16 keeps in caller-provided scratch live here, in a
// fixed array in device memory that exists for as long as the library is
// loaded (on every GPU that loads it).
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocMaxSamples = 16384;
constexpr int kNoAllocParts = kNoAllocMaxSamples / MLP_THREADS;  // 128 CTAs
// kNoAllocParts x (MLP_NPARAM + 1) floats = 2.72 MB
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocParts * (MLP_NPARAM + 1)];

// device address of g_noalloc_scratch per device ordinal, found once per
// device with that device current (the array's host-side name is not a
// device address)
constexpr int kMaxDevices = 64;
float* g_noalloc_ptr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;
}  // namespace

}  // namespace bssn

extern "C" int bssn_remesh_mlp_bwd_noalloc_bf16(const void* wq_dev, const float* norm_dev,
                                                const float* x_dev, const float* y_dev,
                                                const float* c_dev, int n, float* grad_dev,
                                                float* loss_dev, bssn_stream_t stream) {
    using namespace bssn;
    if (!wq_dev || !x_dev || !y_dev || !grad_dev || n < 1) return BSSN_EINVAL;
    if (n > kNoAllocMaxSamples) return BSSN_ELIMIT;
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev < 0 || dev >= kMaxDevices) return BSSN_ELIMIT;
    float* scratch;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_status(e);
            g_noalloc_ptr[dev] = static_cast<float*>(p);
        }
        scratch = g_noalloc_ptr[dev];
    }
    // every CTA overwrites its whole partial slot before the reduction reads
    // it, so nothing in the array has to start at zero
    const int parts = (n + MLP_THREADS - 1) / MLP_THREADS;
    float* gpart = scratch;
    float* lpart = gpart + (size_t)kNoAllocParts * MLP_NPARAM;
    const size_t smem = sizeof(float) * (MLP_NPARAM + MLP_THREADS * (IN + 4 * HID + 2));
    e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    mlp_grad_kernel<<<parts, MLP_THREADS, smem, s>>>((const __nv_bfloat16*)wq_dev, norm_dev, x_dev, y_dev,
                                                     c_dev, n, gpart, lpart);
    mlp_reduce_kernel<<<(MLP_NPARAM + MLP_THREADS - 1) / MLP_THREADS, MLP_THREADS, 0, s>>>(gpart, parts,
                                                                                         grad_dev);
    if (loss_dev) mlp_loss_reduce_kernel<<<1, 32, 0, s>>>(lpart, parts, loss_dev);
    return cuda_status(cudaGetLastError());
}
