// Multi-level meshes: nested level boxes with 2:1 refinement, each level's
// region tiled with blocks, the zipped state the concatenation of one dense
// node grid per level.  Host-side maps (built once per mesh) and the kernels
// that use them: the ghost fill with coarse-to-fine interpolation, the owner
// gather of the right-hand side, and the level sync (restriction by
// injection, prolongation of fine box boundaries).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "bssn_b200.h"

namespace bssn {

// One level's node grid: its box in level octants, its first node in the
// concatenated zipped arrays, and its node counts per axis (6 n + 1).
struct LevelGrid {
    int32_t lo[3], n[3];
    int64_t offset;
    int32_t dims[3];
    int32_t level = 0, parent = -1;  // the patch's level and parent patch
};

// One patch of the hierarchy (the public BssnPatch): a box of octants of
// its level inside its parent patch.
struct PatchDef {
    int32_t level, parent;
    int32_t lo[3], n[3];
};

// A point interpolated from the next coarser level: along every axis with
// j[d] >= 0 a degree-6 Lagrange interpolation over the 7 nodes of a coarse
// octant (base + m * stride[d], m = 0..6) at m = j[d] + 1/2; along the
// others the single node at base.  Axes are interpolated x first, then y,
// then z.
struct InterpEntry {
    int64_t base;
    int32_t stride[3];
    int8_t j[3];
    int8_t pad[5];
};
static_assert(sizeof(InterpEntry) == 32, "device layout");

// Source of a value: >= 0 a node of the zipped arrays, -1 zero (outside the
// domain), <= -2 interpolation entry -2 - src.
struct LevelMaps {
    std::vector<LevelGrid> grids;
    int64_t n_nodes = 0;
    int64_t n_padded = 0;
    std::vector<int64_t> unzip_src;              // per padded point
    std::vector<int64_t> zip_src;                // per node: owning zone's padded index or -1
    std::vector<int64_t> inject_dst, inject_src; // coarse node under a finer box <- fine node
    std::vector<int> inject_first;               // per level l >= 1: first entry (size L + 1)
    std::vector<int64_t> prolong_dst, prolong_src; // fine box-boundary node <- coarse source
    std::vector<int> prolong_first;
    std::vector<InterpEntry> interp;
};

// One 1-D interpolation of the separable ghost fill: out = sum over k < n
// of W[j][k] * in[k], in k order (n = 7; n = 1 is a copy with weight 1).
// The first pass reads zipped nodes and writes x-interpolated rows, the
// second reads those and writes y-interpolated rows, the third the points;
// the values are bit-identical to the per-point interpolation (same
// products, same order of sums), each computed once however many padded
// points share it.
struct PassTask {
    int32_t out;
    int32_t in[7];
    int8_t j, n;
    int16_t pad;
};
static_assert(sizeof(PassTask) == 36, "device layout");

struct LevelsDev {
    // per padded point: >= 0 node, -1 zero, <= -2 third-pass result -2 - src
    int64_t* unzip_src = nullptr;
    PassTask* tasks = nullptr;  // the three passes back to back
    int64_t n_task[3] = {0, 0, 0};
    double* it = nullptr;       // pass results, [var][n_it]
    int64_t n_it = 0;
    int64_t* zip_src = nullptr;
    int64_t* inject_dst = nullptr;
    int64_t* inject_src = nullptr;
    int64_t* prolong_dst = nullptr;
    int64_t* prolong_src = nullptr;
    InterpEntry* interp = nullptr;
    int64_t n_nodes = 0, n_padded = 0;
    std::vector<int> inject_first, prolong_first;  // host copies of the level ranges
    std::vector<LevelGrid> grids;                  // host copy of the level grids
};

// Validates the patches, tiles every patch's region (its box minus its
// children's boxes) with blocks of 1, 2, 4 or 8 octants per axis, and lays them out
// (offsets, sides 13/19/31/55, level, origin g0 in the level's node index,
// ptmin / ptmax, physical-boundary flags on level 0).  blocks == NULL: count
// only.  n_nodes: total zipped nodes over all levels.
int levels_generate(const std::vector<PatchDef>& P, const int32_t M0[3], double xmin, double h0,
                    BssnBlockDesc* blocks, int* nblocks, int64_t* n_nodes,
                    int max_w = 8);
// The maps of a generated mesh (host only).
int levels_build(const BssnBlockDesc* blocks, int nblocks, const std::vector<PatchDef>& P,
                 const int32_t M0[3], LevelMaps* out);
// One patch per level from a box per level (patch l's parent is l - 1).
std::vector<PatchDef> chain_patches(int nlevels, const BssnLevelBox* boxes);
std::vector<PatchDef> patches_from(int npatches, const BssnPatch* patches);
int levels_upload(const LevelMaps& m, LevelsDev* d);
void levels_free(LevelsDev* d);

// P <- ghost fill of the zipped state U (every padded point of every block).
int launch_levels_unzip(const LevelsDev& d, double* const* P, const double* const* U, int nvars,
                        cudaStream_t s);
// Rz[node] <- R[owner zone of node], 0 for nodes no block owns.
int launch_levels_zip(const LevelsDev& d, double* const* Rz, const double* const* R, int nvars,
                      cudaStream_t s);
// One RK4 stage at every node (as launch_node_stage) with the right-hand
// side gathered from the padded array R at each node's owning zone.
int launch_levels_stage(const LevelsDev& d, int stage, double* const* im, double* const* acc,
                        double* const* u, const double* const* R, double dt, int enforce, double chi_floor,
                        int* status, cudaStream_t s);
// Restriction (finest level first) then prolongation (coarsest first) on U.
int launch_levels_sync(const LevelsDev& d, double* const* U, int nvars, cudaStream_t s);
// Transfer of a state between two hierarchies on the same domain (after a
// remesh): every node of level l of the new hierarchy takes the old level-l
// node where the old level l has it, else the coincident node or the
// interpolation from the new level l-1 (levels in increasing order); then
// the new hierarchy's sync.  Builds its maps on the host and allocates
// device memory for them; blocking.
int levels_transfer(const LevelsDev& from, const double* const* U_old, const LevelsDev& to,
                    double* const* U_new, int nvars, cudaStream_t s);

}  // namespace bssn
