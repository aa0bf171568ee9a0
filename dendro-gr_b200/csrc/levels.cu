// Multi-level meshes: generator, host-side maps and their kernels (see
// levels.h and the BssnLevelBox notes in include/bssn_b200.h).
//
// The reference gets its level transitions from dendrolib's ot::Mesh (block
// construction and unzip with parent-to-child interpolation; absent from the
// reference tree, called at BSSN_GR/src/rkBSSN.cpp:611-650).  This file is
// this library's definition of them: dendrolib interpolates a child from its
// parent element's nodal values with the element's Lagrange polynomials of
// the element order (6, seven nodes per edge), which is the interpolation
// used here, applied axis by axis.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <utility>
#include <vector>

#include "bssn_common.cuh"
#include "levels.h"
#include "rk4_stage.cuh"

namespace bssn {

namespace {

constexpr int OCT = 6;  // node intervals per octant edge

// Degree-6 Lagrange weights on nodes 0..6 at x = j + 1/2, j = 0..5:
// w_m = prod_{k != m} (2j + 1 - 2k) / (2 (m - k)), formed as an exact
// integer ratio and rounded once.
void lagrange_half(double w[6][7]) {
    for (int j = 0; j < 6; j++)
        for (int m = 0; m < 7; m++) {
            long long num = 1, den = 1;
            for (int k = 0; k < 7; k++) {
                if (k == m) continue;
                num *= (2 * j + 1 - 2 * k);
                den *= 2 * (m - k);
            }
            w[j][m] = (double)num / (double)den;
        }
}

struct Box {
    int32_t lo[3], n[3];
    bool contains_cell(const int32_t o[3], int w) const {  // cell [o, o+w) inside
        for (int d = 0; d < 3; d++)
            if (o[d] < lo[d] || o[d] + w > lo[d] + n[d]) return false;
        return true;
    }
    bool disjoint_cell(const int32_t o[3], int w) const {
        for (int d = 0; d < 3; d++)
            if (o[d] >= lo[d] + n[d] || o[d] + w <= lo[d]) return true;
        return false;
    }
};

int check_patches(const std::vector<PatchDef>& P, const int32_t M0[3]) {
    const int np = (int)P.size();
    if (np < 1 || np > 64 || !M0) return BSSN_EINVAL;
    if (P[0].level != 0 || P[0].parent != -1) return BSSN_EINVAL;
    for (int d = 0; d < 3; d++)
        if (M0[d] < 1 || P[0].lo[d] != 0 || P[0].n[d] != M0[d]) return BSSN_EINVAL;
    for (int p = 1; p < np; p++) {
        const PatchDef& c = P[p];
        if (c.parent < 0 || c.parent >= p || c.level < 1 || c.level > 15 || P[c.parent].level != c.level - 1)
            return BSSN_EINVAL;
        const PatchDef& q = P[c.parent];
        for (int d = 0; d < 3; d++) {
            const int lo = c.lo[d], n = c.n[d];
            if (n < 2 || (lo & 1) || (n & 1)) return BSSN_EINVAL;
            // inside the parent with one parent octant of margin
            if (lo / 2 < q.lo[d] + 1 || lo / 2 + n / 2 > q.lo[d] + q.n[d] - 1) return BSSN_EINVAL;
        }
        // patches of one level at least one parent octant apart, so no
        // block's padding reaches another patch of its level
        for (int r = 1; r < p; r++) {
            if (P[r].level != c.level) continue;
            bool apart = false;
            for (int d = 0; d < 3; d++)
                apart = apart || c.lo[d] + c.n[d] + 2 <= P[r].lo[d] || P[r].lo[d] + P[r].n[d] + 2 <= c.lo[d];
            if (!apart) return BSSN_EINVAL;
        }
    }
    return 0;
}

// The boxes of patch p's children in p's level octants.
std::vector<Box> children_of(const std::vector<PatchDef>& P, int p) {
    std::vector<Box> out;
    for (size_t c = 0; c < P.size(); c++)
        if (P[c].parent == p) {
            Box b;
            for (int d = 0; d < 3; d++) {
                b.lo[d] = P[c].lo[d] / 2;
                b.n[d] = P[c].n[d] / 2;
            }
            out.push_back(b);
        }
    return out;
}

struct Tiler {
    Box box;
    std::vector<Box> kids;
    std::vector<std::pair<std::array<int32_t, 3>, int>> cells;  // (origin, width)
    void tile(const int32_t o[3], int w) {
        if (box.disjoint_cell(o, w)) return;
        bool apart = true;
        for (const Box& k : kids) {
            if (k.contains_cell(o, w)) return;
            apart = apart && k.disjoint_cell(o, w);
        }
        if (box.contains_cell(o, w) && apart) {
            cells.push_back({{o[0], o[1], o[2]}, w});
            return;
        }
        const int h = w / 2;  // w > 1 here: unit cells are resolved above
        for (int c = 0; c < 8; c++) {
            const int32_t oc[3] = {o[0] + (c & 1) * h, o[1] + ((c >> 1) & 1) * h, o[2] + ((c >> 2) & 1) * h};
            tile(oc, h);
        }
    }
};

}  // namespace

std::vector<PatchDef> chain_patches(int nlevels, const BssnLevelBox* boxes) {
    std::vector<PatchDef> P;
    if (nlevels < 1 || nlevels > 16 || !boxes) return P;
    for (int l = 0; l < nlevels; l++) {
        PatchDef q;
        q.level = l;
        q.parent = l - 1;
        for (int d = 0; d < 3; d++) {
            q.lo[d] = boxes[l].lo[d];
            q.n[d] = boxes[l].n[d];
        }
        P.push_back(q);
    }
    return P;
}

std::vector<PatchDef> patches_from(int npatches, const BssnPatch* patches) {
    std::vector<PatchDef> P;
    if (npatches < 1 || npatches > 64 || !patches) return P;
    for (int p = 0; p < npatches; p++) {
        PatchDef q;
        q.level = patches[p].level;
        q.parent = patches[p].parent;
        for (int d = 0; d < 3; d++) {
            q.lo[d] = patches[p].lo[d];
            q.n[d] = patches[p].n[d];
        }
        P.push_back(q);
    }
    return P;
}

int levels_generate(const std::vector<PatchDef>& P, const int32_t M0[3], double xmin, double h0,
                    BssnBlockDesc* blocks, int* nblocks, int64_t* n_nodes, int max_w) {
    if (!nblocks || !n_nodes || !(h0 > 0.0)) return BSSN_EINVAL;
    if (max_w != 1 && max_w != 2 && max_w != 4 && max_w != 8) return BSSN_EINVAL;
    int st = check_patches(P, M0);
    if (st) return st;
    int64_t nodes = 0;
    for (const PatchDef& q : P)
        nodes += int64_t(OCT * q.n[0] + 1) * (OCT * q.n[1] + 1) * (OCT * q.n[2] + 1);
    if (nodes >= (int64_t(1) << 31)) return BSSN_ELIMIT;
    int count = 0;
    int64_t offset = 0;
    for (int p = 0; p < (int)P.size(); p++) {
        const int l = P[p].level;
        Tiler t;
        for (int d = 0; d < 3; d++) {
            t.box.lo[d] = P[p].lo[d];
            t.box.n[d] = P[p].n[d];
        }
        t.kids = children_of(P, p);
        // cells of max_w octants per axis (blocks of side 6 max_w + 7), split
        // where a box or a child box cuts them
        for (int32_t z = t.box.lo[2]; z < t.box.lo[2] + t.box.n[2]; z += max_w)
            for (int32_t y = t.box.lo[1]; y < t.box.lo[1] + t.box.n[1]; y += max_w)
                for (int32_t x = t.box.lo[0]; x < t.box.lo[0] + t.box.n[0]; x += max_w) {
                    const int32_t o[3] = {x, y, z};
                    t.tile(o, max_w);
                }
        const double h = std::ldexp(h0, -l);
        for (auto& c : t.cells) {
            if (blocks) {
                BssnBlockDesc& b = blocks[count];
                std::memset(&b, 0, sizeof b);
                const int w = c.second;
                b.sz = OCT * w + 7;
                b.level = l;
                b.offset = offset;
                b.bflag = 0;
                for (int d = 0; d < 3; d++) {
                    b.g0[d] = OCT * c.first[d];
                    b.ptmin[d] = xmin + (double)(b.g0[d] - 3) * h;
                    b.ptmax[d] = b.ptmin[d] + (double)(b.sz - 1) * h;
                    if (l == 0 && c.first[d] == 0) b.bflag |= 1u << (2 * d);
                    if (l == 0 && c.first[d] + w == M0[d]) b.bflag |= 2u << (2 * d);
                }
            }
            const int64_t s = OCT * c.second + 7;
            offset += (s * s * s + 1) / 2 * 2;
            count++;
        }
    }
    *nblocks = count;
    *n_nodes = nodes;
    return 0;
}

namespace {

// Index arguments named l below are patch indices (one patch per level for
// meshes described by a box per level).
struct Builder {
    LevelMaps* out;
    std::vector<std::vector<int32_t>> owner;  // per patch: block of each octant of its box, -1 none

    const LevelGrid& grid(int l) const { return out->grids[l]; }
    bool in_grid(int l, const int64_t q[3]) const {
        const LevelGrid& g = grid(l);
        for (int d = 0; d < 3; d++)
            if (q[d] < int64_t(OCT) * g.lo[d] || q[d] > int64_t(OCT) * (g.lo[d] + g.n[d])) return false;
        return true;
    }
    int64_t node(int l, const int64_t q[3]) const {
        const LevelGrid& g = grid(l);
        const int64_t x = q[0] - int64_t(OCT) * g.lo[0], y = q[1] - int64_t(OCT) * g.lo[1],
                      z = q[2] - int64_t(OCT) * g.lo[2];
        return g.offset + x + int64_t(g.dims[0]) * (y + int64_t(g.dims[1]) * z);
    }
    int32_t owner_of(int l, const int64_t t[3]) const {
        const LevelGrid& g = grid(l);
        for (int d = 0; d < 3; d++)
            if (t[d] < g.lo[d] || t[d] >= g.lo[d] + g.n[d]) return -1;
        const int64_t i = (t[0] - g.lo[0]) + int64_t(g.n[0]) * ((t[1] - g.lo[1]) + int64_t(g.n[1]) * (t[2] - g.lo[2]));
        return owner[l][i];
    }
    // Source of patch l's level index q outside its box (level >= 1): the
    // parent's coincident node or an interpolation entry.  kBad when the
    // coarse stencil would leave the parent's grid (cannot happen for valid
    // patches).
    static constexpr int64_t kBad = std::numeric_limits<int64_t>::min();
    int64_t coarse_source(int l, const int64_t q[3]) {
        int64_t c[3];
        int8_t j[3];
        bool odd = false;
        for (int d = 0; d < 3; d++) {
            if ((q[d] & 1) == 0) {
                c[d] = q[d] / 2;
                j[d] = -1;
            } else {
                const int64_t clo = (q[d] - 1) / 2;  // q >= 1 here
                const int64_t t = clo / OCT;
                c[d] = OCT * t;
                j[d] = (int8_t)(clo - OCT * t);
                odd = true;
            }
        }
        int64_t hi[3];
        for (int d = 0; d < 3; d++) hi[d] = c[d] + (j[d] >= 0 ? OCT : 0);
        const int pa = grid(l).parent;
        if (pa < 0 || !in_grid(pa, c) || !in_grid(pa, hi)) return kBad;
        if (!odd) return node(pa, c);
        InterpEntry e;
        std::memset(&e, 0, sizeof e);
        e.base = node(pa, c);
        const LevelGrid& g = grid(pa);
        e.stride[0] = 1;
        e.stride[1] = g.dims[0];
        e.stride[2] = g.dims[0] * g.dims[1];
        for (int d = 0; d < 3; d++) e.j[d] = j[d];
        out->interp.push_back(e);
        return -2 - (int64_t)(out->interp.size() - 1);
    }
    int64_t padded_source(int l, const int64_t q[3]) {
        if (in_grid(l, q)) return node(l, q);
        if (grid(l).level == 0) return -1;  // outside the domain
        return coarse_source(l, q);
    }
};

}  // namespace

int levels_build(const BssnBlockDesc* blocks, int nblocks, const std::vector<PatchDef>& P,
                 const int32_t M0[3], LevelMaps* out) {
    if (!blocks || nblocks <= 0 || !out) return BSSN_EINVAL;
    int st = check_patches(P, M0);
    if (st) return st;
    *out = LevelMaps();
    const int np = (int)P.size();
    int maxlev = 0;
    int64_t off = 0;
    for (int p = 0; p < np; p++) {
        LevelGrid g;
        for (int d = 0; d < 3; d++) {
            g.lo[d] = P[p].lo[d];
            g.n[d] = P[p].n[d];
            g.dims[d] = OCT * g.n[d] + 1;
        }
        g.level = P[p].level;
        g.parent = P[p].parent;
        g.offset = off;
        off += int64_t(g.dims[0]) * g.dims[1] * g.dims[2];
        out->grids.push_back(g);
        maxlev = std::max(maxlev, g.level);
    }
    if (off >= (int64_t(1) << 31)) return BSSN_ELIMIT;
    out->n_nodes = off;
    Builder B{out, {}};
    B.owner.resize(np);
    std::vector<std::vector<Box>> kids(np);
    for (int p = 0; p < np; p++) {
        B.owner[p].assign(size_t(P[p].n[0]) * P[p].n[1] * P[p].n[2], -1);
        kids[p] = children_of(P, p);
    }
    auto box_of = [&](int p) {
        Box b;
        for (int d = 0; d < 3; d++) {
            b.lo[d] = P[p].lo[d];
            b.n[d] = P[p].n[d];
        }
        return b;
    };
    // each block belongs to the patch of its level that holds its octants
    std::vector<int> patch_of(nblocks, -1);
    int64_t npad = 0;
    for (int b = 0; b < nblocks; b++) {
        const BssnBlockDesc& k = blocks[b];
        const int w = (k.sz - 7) / OCT;
        if (k.level < 0 || k.level > maxlev || k.sz != OCT * w + 7 || (w != 1 && w != 2 && w != 4 && w != 8) ||
            k.offset < 0)
            return BSSN_EINVAL;
        int32_t o[3];
        for (int d = 0; d < 3; d++) {
            if (k.g0[d] % OCT) return BSSN_EINVAL;
            o[d] = k.g0[d] / OCT;
        }
        int p = -1;
        for (int q = 0; q < np && p < 0; q++)
            if (P[q].level == k.level && box_of(q).contains_cell(o, w)) p = q;
        if (p < 0) return BSSN_EINVAL;
        for (const Box& c : kids[p])
            if (!c.disjoint_cell(o, w)) return BSSN_EINVAL;
        patch_of[b] = p;
        const Box box = box_of(p);
        for (int z = 0; z < w; z++)
            for (int y = 0; y < w; y++)
                for (int x = 0; x < w; x++) {
                    const int64_t i = (o[0] + x - box.lo[0]) +
                                      int64_t(box.n[0]) * ((o[1] + y - box.lo[1]) + int64_t(box.n[1]) * (o[2] + z - box.lo[2]));
                    if (B.owner[p][i] >= 0) return BSSN_EINVAL;  // overlapping blocks
                    B.owner[p][i] = b;
                }
        npad = std::max<int64_t>(npad, k.offset + int64_t(k.sz) * k.sz * k.sz);
    }
    // every octant of every patch's region has a block
    for (int p = 0; p < np; p++) {
        for (int64_t i = 0; i < (int64_t)B.owner[p].size(); i++) {
            const int32_t t[3] = {int32_t(P[p].lo[0] + i % P[p].n[0]),
                                  int32_t(P[p].lo[1] + (i / P[p].n[0]) % P[p].n[1]),
                                  int32_t(P[p].lo[2] + i / (int64_t(P[p].n[0]) * P[p].n[1]))};
            bool under = false;
            for (const Box& c : kids[p]) under = under || c.contains_cell(t, 1);
            if (under != (B.owner[p][i] < 0)) return BSSN_EINVAL;
        }
    }
    out->n_padded = npad;
    // ghost fill sources
    out->unzip_src.assign(size_t(npad), -1);
    for (int b = 0; b < nblocks; b++) {
        const BssnBlockDesc& k = blocks[b];
        const int s = k.sz;
        for (int c = 0; c < s; c++)
            for (int r = 0; r < s; r++)
                for (int a = 0; a < s; a++) {
                    const int64_t q[3] = {int64_t(k.g0[0]) + a - 3, int64_t(k.g0[1]) + r - 3, int64_t(k.g0[2]) + c - 3};
                    const int64_t src = B.padded_source(patch_of[b], q);
                    if (src == Builder::kBad) return BSSN_EINVAL;
                    out->unzip_src[size_t(k.offset + a + int64_t(s) * (r + int64_t(s) * c))] = src;
                }
    }
    // owners
    out->zip_src.assign(size_t(out->n_nodes), -1);
    for (int p = 0; p < np; p++) {
        const LevelGrid& g = out->grids[p];
        for (int64_t z = 0; z < g.dims[2]; z++)
            for (int64_t y = 0; y < g.dims[1]; y++)
                for (int64_t x = 0; x < g.dims[0]; x++) {
                    const int64_t q[3] = {OCT * int64_t(g.lo[0]) + x, OCT * int64_t(g.lo[1]) + y,
                                          OCT * int64_t(g.lo[2]) + z};
                    const int64_t e[3] = {x, y, z};
                    bool boundary = false;
                    for (int d = 0; d < 3; d++)
                        if (g.level > 0 && (e[d] == 0 || e[d] == g.dims[d] - 1)) boundary = true;
                    bool inside_child = false;
                    for (const Box& c : kids[p]) {
                        bool in = true;
                        for (int d = 0; d < 3; d++)
                            in = in && q[d] > OCT * int64_t(c.lo[d]) && q[d] < OCT * int64_t(c.lo[d] + c.n[d]);
                        inside_child = inside_child || in;
                    }
                    if (boundary || inside_child) continue;
                    int64_t t[3];
                    for (int d = 0; d < 3; d++) t[d] = std::min<int64_t>(q[d] / OCT, g.lo[d] + g.n[d] - 1);
                    int32_t b = B.owner_of(p, t);
                    if (b < 0) {  // on a finer patch's boundary: the octant below
                        for (const Box& c : kids[p]) {
                            const int32_t ti[3] = {int32_t(t[0]), int32_t(t[1]), int32_t(t[2])};
                            if (!c.contains_cell(ti, 1)) continue;
                            for (int d = 0; d < 3; d++)
                                if (q[d] == OCT * int64_t(c.lo[d])) t[d] -= 1;
                            break;
                        }
                        b = B.owner_of(p, t);
                    }
                    if (b < 0) return BSSN_EINVAL;
                    const BssnBlockDesc& k = blocks[b];
                    int64_t loc[3];
                    for (int d = 0; d < 3; d++) {
                        loc[d] = q[d] - k.g0[d] + 3;
                        if (loc[d] < 3 || loc[d] > k.sz - 4) return BSSN_EINVAL;
                    }
                    out->zip_src[size_t(B.node(p, q))] =
                        k.offset + loc[0] + int64_t(k.sz) * (loc[1] + int64_t(k.sz) * loc[2]);
                }
    }
    // restriction, finest level first (one segment per level)
    out->inject_first.push_back(0);
    for (int lev = maxlev; lev >= 1; lev--) {
        for (int p = 0; p < np; p++) {
            if (P[p].level != lev) continue;
            const LevelGrid& g = out->grids[p];
            // the patch's box in its parent's node index: [3 lo, 3 (lo + n)]
            for (int64_t z = 3 * int64_t(g.lo[2]) + 1; z < 3 * int64_t(g.lo[2] + g.n[2]); z++)
                for (int64_t y = 3 * int64_t(g.lo[1]) + 1; y < 3 * int64_t(g.lo[1] + g.n[1]); y++)
                    for (int64_t x = 3 * int64_t(g.lo[0]) + 1; x < 3 * int64_t(g.lo[0] + g.n[0]); x++) {
                        const int64_t c[3] = {x, y, z}, f[3] = {2 * x, 2 * y, 2 * z};
                        out->inject_dst.push_back(B.node(g.parent, c));
                        out->inject_src.push_back(B.node(p, f));
                    }
        }
        out->inject_first.push_back((int)out->inject_dst.size());
    }
    // prolongation of patch boundaries, coarsest level first
    out->prolong_first.push_back(0);
    for (int lev = 1; lev <= maxlev; lev++) {
        for (int p = 0; p < np; p++) {
            if (P[p].level != lev) continue;
            const LevelGrid& g = out->grids[p];
            for (int64_t z = 0; z < g.dims[2]; z++)
                for (int64_t y = 0; y < g.dims[1]; y++)
                    for (int64_t x = 0; x < g.dims[0]; x++) {
                        const bool bd = x == 0 || y == 0 || z == 0 || x == g.dims[0] - 1 || y == g.dims[1] - 1 ||
                                        z == g.dims[2] - 1;
                        if (!bd) continue;
                        const int64_t q[3] = {OCT * int64_t(g.lo[0]) + x, OCT * int64_t(g.lo[1]) + y,
                                              OCT * int64_t(g.lo[2]) + z};
                        const int64_t src = B.coarse_source(p, q);
                        if (src == Builder::kBad) return BSSN_EINVAL;
                        out->prolong_dst.push_back(B.node(p, q));
                        out->prolong_src.push_back(src);
                    }
        }
        out->prolong_first.push_back((int)out->prolong_dst.size());
    }
    return 0;
}

namespace {

__constant__ double kLagHalf[6][7];

// grid-stride launches: at most 64 CTAs of 256 threads per SM
int grid_for(int64_t n, int threads) {
    const int64_t b = std::min<int64_t>((n + threads - 1) / threads, 148 * 64);
    return (int)std::max<int64_t>(b, 1);
}

template <class T>
int upload_vec(const std::vector<T>& v, T** d) {
    *d = nullptr;
    if (v.empty()) return 0;
    if (cudaMalloc((void**)d, sizeof(T) * v.size()) != cudaSuccess) {
        cudaGetLastError();
        return BSSN_ENOMEM;
    }
    return cuda_status(cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
}

// The interpolated value of one entry (x first, then y, then z; every
// product and sum rounded in that order, as the oracle does).
__device__ __forceinline__ double interp_value(const double* __restrict__ u, const InterpEntry& e) {
    const int nx = e.j[0] >= 0 ? 7 : 1, ny = e.j[1] >= 0 ? 7 : 1, nz = e.j[2] >= 0 ? 7 : 1;
    double tz = 0.0;
    for (int c = 0; c < nz; c++) {
        double ty = 0.0;
        for (int b = 0; b < ny; b++) {
            const double* row = u + e.base + (int64_t)b * e.stride[1] + (int64_t)c * e.stride[2];
            double tx = 0.0;
            for (int a = 0; a < nx; a++) {
                const double w = e.j[0] >= 0 ? kLagHalf[e.j[0]][a] : 1.0;
                const double p = __dmul_rn(w, __ldg(row + (int64_t)a * e.stride[0]));
                tx = a == 0 ? p : __dadd_rn(tx, p);
            }
            const double w = e.j[1] >= 0 ? kLagHalf[e.j[1]][b] : 1.0;
            const double p = __dmul_rn(w, tx);
            ty = b == 0 ? p : __dadd_rn(ty, p);
        }
        const double w = e.j[2] >= 0 ? kLagHalf[e.j[2]][c] : 1.0;
        const double p = __dmul_rn(w, ty);
        tz = c == 0 ? p : __dadd_rn(tz, p);
    }
    return tz;
}

// One pass of the separable ghost fill (PassTask): inputs from the zipped
// state (first pass) or from the previous pass's results.
__global__ void __launch_bounds__(256) levels_pass_kernel(ConstVars U, double* __restrict__ it, int64_t n_it,
                                                          int nvars, const PassTask* __restrict__ tasks,
                                                          int64_t n, int from_u) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const PassTask t = tasks[i];
        for (int v = 0; v < nvars; v++) {
            const double* in = from_u ? U.p[v] : it + (int64_t)v * n_it;
            double acc = 0.0;
            for (int k = 0; k < t.n; k++) {
                const double w = t.n == 7 ? kLagHalf[t.j][k] : 1.0;
                const double p = __dmul_rn(w, in[t.in[k]]);
                acc = k == 0 ? p : __dadd_rn(acc, p);
            }
            it[(int64_t)v * n_it + t.out] = acc;
        }
    }
}

// Ghost fill: zipped node, zero, or a third-pass result (interpolated point).
__global__ void __launch_bounds__(256) levels_unzip_kernel(MutVars P, ConstVars U, int nvars,
                                                           const int64_t* __restrict__ src,
                                                           const double* __restrict__ it, int64_t n_it,
                                                           int64_t zbase, int64_t n) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = src[p];
        for (int v = 0; v < nvars; v++)
            P.p[v][p] = s >= 0 ? __ldg(U.p[v] + s)
                               : (s == -1 ? 0.0 : it[(int64_t)v * n_it + zbase + (-2 - s)]);
    }
}

__global__ void __launch_bounds__(256) levels_zip_kernel(MutVars Rz, ConstVars R, int nvars,
                                                         const int64_t* __restrict__ src, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = src[i];
        for (int v = 0; v < nvars; v++) Rz.p[v][i] = s >= 0 ? __ldg(R.p[v] + s) : 0.0;
    }
}

// One RK4 stage at every node (the node-wise stage kernel's algebra) with
// the node's right-hand side read from the padded array at its owning zone
// (0 for nodes no block owns; the level sync sets those).
__global__ void __launch_bounds__(256) levels_stage_kernel(int stage, MutVars im, MutVars acc, MutVars u,
                                                           ConstVars R, const int64_t* __restrict__ src,
                                                           int64_t n, double dt, int enforce,
                                                           double chi_floor, int* status) {
    int bad = 0;
    for (int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; node < n;
         node += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sp = src[node];
        double k[NVARS], v[NVARS], a[NVARS];
#pragma unroll
        for (int q = 0; q < NVARS; q++) {
            k[q] = sp >= 0 ? __ldg(R.p[q] + sp) : 0.0;
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

// dst[i] <- source value of src[i]; the sources never overlap the
// destinations of the same launch.
__global__ void __launch_bounds__(256) levels_copy_kernel(MutVars U, int nvars,
                                                          const int64_t* __restrict__ dst,
                                                          const int64_t* __restrict__ src,
                                                          const InterpEntry* __restrict__ interp,
                                                          int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = src[i], d = dst[i];
        for (int v = 0; v < nvars; v++) {
            const double* u = U.p[v];
            U.p[v][d] = s >= 0 ? u[s] : (s == -1 ? 0.0 : interp_value(u, interp[-2 - s]));
        }
    }
}

}  // namespace

namespace {

// The three passes of the separable ghost fill for the interpolated padded
// points of m, deduplicated (a row or point needed by several padded
// points is computed once), and the ghost-fill sources with interpolation
// entries replaced by third-pass results.  Slots: first pass [0, n0),
// second [n0, n0 + n1), third after.
void build_passes(const LevelMaps& m, std::vector<PassTask>& tasks, int64_t n_task[3],
                  std::vector<int64_t>& unzip_code) {
    std::vector<PassTask> pass[3];
    std::unordered_map<int64_t, int32_t> key[3];
    auto task = [&](int stage, int64_t k, auto make) -> int32_t {
        auto it = key[stage].find(k);
        if (it != key[stage].end()) return it->second;
        PassTask t = make();
        t.out = (int32_t)pass[stage].size();
        pass[stage].push_back(t);
        key[stage].emplace(k, t.out);
        return t.out;
    };
    auto blank = []() {
        PassTask t;
        std::memset(&t, 0, sizeof t);
        return t;
    };
    std::vector<int32_t> zslot(m.interp.size(), -1);
    unzip_code = m.unzip_src;
    for (auto& src : unzip_code) {
        if (src > -2) continue;
        const int64_t ie = -2 - src;
        if (zslot[ie] < 0) {
            const InterpEntry& e = m.interp[ie];
            const int nn[3] = {e.j[0] >= 0 ? 7 : 1, e.j[1] >= 0 ? 7 : 1, e.j[2] >= 0 ? 7 : 1};
            const int64_t zk = e.base * 512 + (e.j[0] + 1) * 64 + (e.j[1] + 1) * 8 + (e.j[2] + 1);
            zslot[ie] = task(2, zk, [&]() {
                PassTask z = blank();
                z.n = (int8_t)nn[2];
                z.j = e.j[2] >= 0 ? e.j[2] : 0;
                for (int c = 0; c < nn[2]; c++) {
                    const int64_t plane = e.base + (int64_t)c * e.stride[2];
                    z.in[c] = task(1, plane * 64 + (e.j[0] + 1) * 8 + (e.j[1] + 1), [&]() {
                        PassTask y = blank();
                        y.n = (int8_t)nn[1];
                        y.j = e.j[1] >= 0 ? e.j[1] : 0;
                        for (int b = 0; b < nn[1]; b++) {
                            const int64_t row = plane + (int64_t)b * e.stride[1];
                            y.in[b] = task(0, row * 8 + (e.j[0] + 1), [&]() {
                                PassTask x = blank();
                                x.n = (int8_t)nn[0];
                                x.j = e.j[0] >= 0 ? e.j[0] : 0;
                                for (int a = 0; a < nn[0]; a++) x.in[a] = (int32_t)(row + (int64_t)a * e.stride[0]);
                                return x;
                            });
                        }
                        return y;
                    });
                }
                return z;
            });
        }
        src = -2 - (int64_t)zslot[ie];
    }
    // second-pass inputs and outputs after the first pass, third after both
    const int32_t n0 = (int32_t)pass[0].size(), n1 = (int32_t)pass[1].size();
    for (auto& t : pass[1]) t.out += n0;
    for (auto& t : pass[2]) {
        t.out += n0 + n1;
        for (int k = 0; k < t.n; k++) t.in[k] += n0;
    }
    tasks.clear();
    for (int k = 0; k < 3; k++) {
        n_task[k] = (int64_t)pass[k].size();
        tasks.insert(tasks.end(), pass[k].begin(), pass[k].end());
    }
}

}  // namespace

int levels_upload(const LevelMaps& m, LevelsDev* d) {
    *d = LevelsDev();
    double w[6][7];
    lagrange_half(w);
    std::vector<PassTask> tasks;
    std::vector<int64_t> code;
    build_passes(m, tasks, d->n_task, code);
    d->n_it = d->n_task[0] + d->n_task[1] + d->n_task[2];
    int st = cuda_status(cudaMemcpyToSymbol(kLagHalf, w, sizeof w));
    if (!st) st = upload_vec(code, &d->unzip_src);
    if (!st) st = upload_vec(tasks, &d->tasks);
    if (!st && d->n_it > 0 &&
        cudaMalloc((void**)&d->it, sizeof(double) * NVARS * d->n_it) != cudaSuccess) {
        cudaGetLastError();
        st = BSSN_ENOMEM;
    }
    if (!st) st = upload_vec(m.zip_src, &d->zip_src);
    if (!st) st = upload_vec(m.inject_dst, &d->inject_dst);
    if (!st) st = upload_vec(m.inject_src, &d->inject_src);
    if (!st) st = upload_vec(m.prolong_dst, &d->prolong_dst);
    if (!st) st = upload_vec(m.prolong_src, &d->prolong_src);
    if (!st) st = upload_vec(m.interp, &d->interp);
    d->n_nodes = m.n_nodes;
    d->n_padded = m.n_padded;
    d->inject_first = m.inject_first;
    d->prolong_first = m.prolong_first;
    d->grids = m.grids;
    if (st) levels_free(d);
    return st;
}

void levels_free(LevelsDev* d) {
    cudaFree(d->unzip_src);
    cudaFree(d->tasks);
    cudaFree(d->it);
    cudaFree(d->zip_src);
    cudaFree(d->inject_dst);
    cudaFree(d->inject_src);
    cudaFree(d->prolong_dst);
    cudaFree(d->prolong_src);
    cudaFree(d->interp);
    *d = LevelsDev();
}

namespace {
int vars_in(const double* const* a, int nvars, ConstVars* c) {
    if (nvars < 1 || nvars > NVARS) return BSSN_EINVAL;
    for (int v = 0; v < nvars; v++) c->p[v] = a[v];
    return 0;
}
int vars_out(double* const* a, int nvars, MutVars* c) {
    if (nvars < 1 || nvars > NVARS) return BSSN_EINVAL;
    for (int v = 0; v < nvars; v++) c->p[v] = a[v];
    return 0;
}
}  // namespace

int launch_levels_unzip(const LevelsDev& d, double* const* P, const double* const* U, int nvars,
                        cudaStream_t s) {
    MutVars p;
    ConstVars u;
    int st = vars_out(P, nvars, &p);
    if (!st) st = vars_in(U, nvars, &u);
    if (st || d.n_padded == 0) return st;
    int64_t first = 0;
    for (int k = 0; k < 3; k++) {  // rows in x, rows in y, points
        if (d.n_task[k] > 0) {
            levels_pass_kernel<<<grid_for(d.n_task[k], 256), 256, 0, s>>>(u, d.it, d.n_it, nvars, d.tasks + first,
                                                                          d.n_task[k], k == 0);
            st = cuda_status(cudaGetLastError());
            if (st) return st;
        }
        first += d.n_task[k];
    }
    levels_unzip_kernel<<<grid_for(d.n_padded, 256), 256, 0, s>>>(p, u, nvars, d.unzip_src, d.it, d.n_it,
                                                                  d.n_task[0] + d.n_task[1], d.n_padded);
    return cuda_status(cudaGetLastError());
}

int launch_levels_zip(const LevelsDev& d, double* const* Rz, const double* const* R, int nvars,
                      cudaStream_t s) {
    MutVars z;
    ConstVars r;
    int st = vars_out(Rz, nvars, &z);
    if (!st) st = vars_in(R, nvars, &r);
    if (st || d.n_nodes == 0) return st;
    levels_zip_kernel<<<grid_for(d.n_nodes, 256), 256, 0, s>>>(z, r, nvars, d.zip_src, d.n_nodes);
    return cuda_status(cudaGetLastError());
}

int launch_levels_stage(const LevelsDev& d, int stage, double* const* im, double* const* acc,
                        double* const* u, const double* const* R, double dt, int enforce, double chi_floor,
                        int* status, cudaStream_t s) {
    MutVars I, A, U;
    ConstVars Rr;
    for (int q = 0; q < NVARS; q++) {
        I.p[q] = im[q];
        A.p[q] = acc[q];
        U.p[q] = u[q];
        Rr.p[q] = R[q];
    }
    if (d.n_nodes == 0) return 0;
    levels_stage_kernel<<<grid_for(d.n_nodes, 256), 256, 0, s>>>(stage, I, A, U, Rr, d.zip_src, d.n_nodes, dt,
                                                                  enforce, chi_floor, status);
    return cuda_status(cudaGetLastError());
}

int launch_levels_sync(const LevelsDev& d, double* const* U, int nvars, cudaStream_t s) {
    MutVars u;
    int st = vars_out(U, nvars, &u);
    if (st) return st;
    auto run = [&](const std::vector<int>& first, const int64_t* dst, const int64_t* src) {
        for (size_t k = 0; k + 1 < first.size(); k++) {
            const int64_t n = first[k + 1] - first[k];
            if (n <= 0) continue;
            levels_copy_kernel<<<grid_for(n, 256), 256, 0, s>>>(u, nvars, dst + first[k], src + first[k],
                                                                d.interp, n);
            const int e = cuda_status(cudaGetLastError());
            if (e) return e;
        }
        return 0;
    };
    st = run(d.inject_first, d.inject_dst, d.inject_src);
    return st ? st : run(d.prolong_first, d.prolong_dst, d.prolong_src);
}

namespace {

__global__ void __launch_bounds__(256) levels_move_kernel(MutVars Un, ConstVars Uo, int nvars,
                                                          const int64_t* __restrict__ dst,
                                                          const int64_t* __restrict__ src, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = dst[i], s = src[i];
        for (int v = 0; v < nvars; v++) Un.p[v][d] = __ldg(Uo.p[v] + s);
    }
}

bool same_box(const LevelGrid& a, const LevelGrid& b) {
    for (int d = 0; d < 3; d++)
        if (a.lo[d] != b.lo[d] || a.n[d] != b.n[d]) return false;
    return true;
}

}  // namespace

int levels_transfer(const LevelsDev& from, const double* const* U_old, const LevelsDev& to,
                    double* const* U_new, int nvars, cudaStream_t s) {
    if (from.grids.empty() || to.grids.empty() || !same_box(from.grids[0], to.grids[0])) return BSSN_EINVAL;
    MutVars un;
    ConstVars uo;
    int st = vars_out(U_new, nvars, &un);
    if (!st) st = vars_in(U_old, nvars, &uo);
    if (st) return st;
    // the new hierarchy's grids, for its coarse sources
    LevelMaps nm;
    nm.grids = to.grids;
    Builder B{&nm, {}};
    std::vector<int64_t> cdst, csrc, fdst, fsrc;
    std::vector<int> cfirst{0}, ffirst{0};
    for (int l = 0; l < (int)to.grids.size(); l++) {
        const LevelGrid& g = to.grids[l];
        for (int64_t z = 0; z < g.dims[2]; z++)
            for (int64_t y = 0; y < g.dims[1]; y++)
                for (int64_t x = 0; x < g.dims[0]; x++) {
                    const int64_t q[3] = {OCT * int64_t(g.lo[0]) + x, OCT * int64_t(g.lo[1]) + y,
                                          OCT * int64_t(g.lo[2]) + z};
                    // an old patch of the same level holding the node (patches
                    // of one level are apart, so at most one does)
                    int op = -1;
                    for (int r = 0; r < (int)from.grids.size() && op < 0; r++) {
                        const LevelGrid& o = from.grids[r];
                        if (o.level != g.level) continue;
                        bool in = true;
                        for (int d = 0; d < 3; d++)
                            in = in && q[d] >= OCT * int64_t(o.lo[d]) && q[d] <= OCT * int64_t(o.lo[d] + o.n[d]);
                        if (in) op = r;
                    }
                    const int64_t dst = B.node(l, q);
                    if (op >= 0) {
                        const LevelGrid& o = from.grids[op];
                        cdst.push_back(dst);
                        csrc.push_back(o.offset + (q[0] - OCT * int64_t(o.lo[0])) +
                                       int64_t(o.dims[0]) * ((q[1] - OCT * int64_t(o.lo[1])) +
                                                             int64_t(o.dims[1]) * (q[2] - OCT * int64_t(o.lo[2]))));
                    } else {
                        if (g.level == 0) return BSSN_EINVAL;  // level 0 is the same grid
                        const int64_t src = B.coarse_source(l, q);
                        if (src == Builder::kBad) return BSSN_EINVAL;
                        fdst.push_back(dst);
                        fsrc.push_back(src);
                    }
                }
        cfirst.push_back((int)cdst.size());
        ffirst.push_back((int)fdst.size());
    }
    int64_t *dcd = nullptr, *dcs = nullptr, *dfd = nullptr, *dfs = nullptr;
    InterpEntry* dit = nullptr;
    st = upload_vec(cdst, &dcd);
    if (!st) st = upload_vec(csrc, &dcs);
    if (!st) st = upload_vec(fdst, &dfd);
    if (!st) st = upload_vec(fsrc, &dfs);
    if (!st) st = upload_vec(nm.interp, &dit);
    // level by level: copies from the old state, then the nodes filled from
    // the new level below (complete by then)
    for (size_t l = 0; l + 1 < cfirst.size() && !st; l++) {
        const int64_t nc = cfirst[l + 1] - cfirst[l], nf = ffirst[l + 1] - ffirst[l];
        if (nc > 0) {
            levels_move_kernel<<<grid_for(nc, 256), 256, 0, s>>>(un, uo, nvars, dcd + cfirst[l], dcs + cfirst[l], nc);
            st = cuda_status(cudaGetLastError());
        }
        if (!st && nf > 0) {
            levels_copy_kernel<<<grid_for(nf, 256), 256, 0, s>>>(un, nvars, dfd + ffirst[l], dfs + ffirst[l], dit, nf);
            st = cuda_status(cudaGetLastError());
        }
    }
    if (!st) st = launch_levels_sync(to, U_new, nvars, s);
    if (!st) st = cuda_status(cudaStreamSynchronize(s));
    cudaFree(dcd);
    cudaFree(dcs);
    cudaFree(dfd);
    cudaFree(dfs);
    cudaFree(dit);
    return st;
}

}  // namespace bssn

// Host copies of the maps for the C ABI (bssn_levels_maps, bssn_patches_maps).
static int export_maps(const bssn::LevelMaps& m, int64_t sizes[5], int64_t* unzip_src, int64_t* zip_src,
                int64_t* inject, int64_t* prolong, int64_t* interp) {
    sizes[0] = m.n_padded;
    sizes[1] = m.n_nodes;
    sizes[2] = (int64_t)m.inject_dst.size();
    sizes[3] = (int64_t)m.prolong_dst.size();
    sizes[4] = (int64_t)m.interp.size();
    if (unzip_src) std::copy(m.unzip_src.begin(), m.unzip_src.end(), unzip_src);
    if (zip_src) std::copy(m.zip_src.begin(), m.zip_src.end(), zip_src);
    if (inject)
        for (size_t i = 0; i < m.inject_dst.size(); i++) {
            inject[2 * i] = m.inject_dst[i];
            inject[2 * i + 1] = m.inject_src[i];
        }
    if (prolong)
        for (size_t i = 0; i < m.prolong_dst.size(); i++) {
            prolong[2 * i] = m.prolong_dst[i];
            prolong[2 * i + 1] = m.prolong_src[i];
        }
    if (interp)
        for (size_t i = 0; i < m.interp.size(); i++) {
            const bssn::InterpEntry& e = m.interp[i];
            int64_t* o = interp + 7 * i;
            o[0] = e.base;
            for (int d = 0; d < 3; d++) {
                o[1 + d] = e.stride[d];
                o[4 + d] = e.j[d];
            }
        }
    return 0;
}

extern "C" {

int bssn_mesh_generate_levels(int nlevels, const int32_t M0[3], const BssnLevelBox* boxes, double xmin,
                              double h0, BssnBlockDesc* blocks, int* nblocks, int64_t* n_nodes) {
    return bssn::levels_generate(bssn::chain_patches(nlevels, boxes), M0, xmin, h0, blocks, nblocks, n_nodes,
                                 8);
}

int bssn_mesh_generate_patches(int npatches, const int32_t M0[3], const BssnPatch* patches, double xmin,
                               double h0, BssnBlockDesc* blocks, int* nblocks, int64_t* n_nodes) {
    return bssn::levels_generate(bssn::patches_from(npatches, patches), M0, xmin, h0, blocks, nblocks, n_nodes,
                                 8);
}

int bssn_mesh_generate_patches_w(int npatches, const int32_t M0[3], const BssnPatch* patches, double xmin,
                                 double h0, int max_w, BssnBlockDesc* blocks, int* nblocks,
                                 int64_t* n_nodes) {
    return bssn::levels_generate(bssn::patches_from(npatches, patches), M0, xmin, h0, blocks, nblocks, n_nodes,
                                 max_w);
}

int bssn_levels_maps(const BssnBlockDesc* blocks, int nblocks, int nlevels, const int32_t M0[3],
                     const BssnLevelBox* boxes, int64_t sizes[5], int64_t* unzip_src, int64_t* zip_src,
                     int64_t* inject, int64_t* prolong, int64_t* interp) {
    if (!sizes) return BSSN_EINVAL;
    bssn::LevelMaps m;
    const int st = bssn::levels_build(blocks, nblocks, bssn::chain_patches(nlevels, boxes), M0, &m);
    return st ? st : export_maps(m, sizes, unzip_src, zip_src, inject, prolong, interp);
}

int bssn_patches_maps(const BssnBlockDesc* blocks, int nblocks, int npatches, const int32_t M0[3],
                      const BssnPatch* patches, int64_t sizes[5], int64_t* unzip_src, int64_t* zip_src,
                      int64_t* inject, int64_t* prolong, int64_t* interp) {
    if (!sizes) return BSSN_EINVAL;
    bssn::LevelMaps m;
    const int st = bssn::levels_build(blocks, nblocks, bssn::patches_from(npatches, patches), M0, &m);
    return st ? st : export_maps(m, sizes, unzip_src, zip_src, inject, prolong, interp);
}

}  // extern "C"
