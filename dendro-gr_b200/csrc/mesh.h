// Host-side mesh state behind the bssn_mesh handle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <utility>
#include <vector>

#include "bssn_b200.h"
#include "levels.h"
#include "remesh.h"
#include "rhs_fused.cuh"

namespace bssn {

// Blocks at least this large stage the split derivative pass straight from
// the zipped stage state in the plan's zipped-right-hand-side form: a brick's
// tile is a stack of short rows in a padded block of that size anyway, so
// reading the node grid costs no more and their ghost fill is skipped.
constexpr int kDirectMinSide = 55;

// A run of consecutive points of one block handled by one CTA.
struct Chunk {
    int32_t blk;
    int32_t count;
    int64_t start;
};

struct MeshState {
    std::vector<BssnBlockDesc> blocks;
    int32_t G[3];
    int64_t unzip_size;
    BssnBlockDesc* d_blocks = nullptr;
    Chunk* d_pad_chunks = nullptr;
    Chunk* d_int_chunks = nullptr;
    int n_pad_chunks = 0;
    int n_int_chunks = 0;
    // ghost-fill chunks of the blocks smaller than kDirectMinSide only
    Chunk* d_pad_chunks_small = nullptr;
    int n_pad_chunks_small = 0;
    // brick task lists per (tile shape, block side; side 0 = all blocks):
    // (device pointer, count)
    std::map<std::pair<int, int>, std::pair<BrickTask*, int>> tasks;
    // partial sums of the constraint-norm reduction (allocated on first use)
    double* d_partial = nullptr;
    // elements (octants) of all blocks and the first element of each block
    // (remesh test; built on first use)
    ElemRef* d_elems = nullptr;
    int64_t* d_elem_first = nullptr;
    int64_t n_elems = 0;
    // element list of the blocks a decision sends to the exact test: offsets
    // per block, the count (stored after the offsets) and the list
    int64_t* d_need_off = nullptr;
    int64_t* d_need_count = nullptr;
    int32_t* d_need_list = nullptr;
    // runs of sublattice points for the block features, the first run of each
    // block and the runs' partial maxima (built on first use)
    Chunk* d_fchunks = nullptr;
    int64_t* d_fchunk_first = nullptr;
    double* d_fpart = nullptr;
    int n_fchunks = 0;
    // autotuned tile per padded side (0 = not tuned)
    std::map<int, int> tuned;
    // scratch of the split right-hand side (kSplitSlots doubles per zone)
    double* d_scratch = nullptr;
    int64_t scratch_zones = 0;
    // multi-level meshes: the level maps (nullptr for single-level meshes,
    // whose zipped state is one node grid of dims G)
    LevelsDev* lv = nullptr;
};

int mesh_create(const BssnBlockDesc* blocks, int nblocks, const int32_t G[3],
                MeshState** out);
void mesh_destroy(MeshState* m);
int mesh_tasks(MeshState* m, int tile, const BrickTask** tasks, int* ntasks);
// Brick tasks of one tile for the blocks of padded side `side` (in block
// order), for all blocks (side 0, block order) or for all blocks in the
// Z-order of their origins (side kAllZOrder).
constexpr int kAllZOrder = -1;
int mesh_tasks_side(MeshState* m, int tile, int side, const BrickTask** tasks, int* ntasks);
// Make the split-path scratch hold at least min(zones, kSplitScratchZonesMax)
// zones (allocates; call outside stream capture).
int mesh_scratch(MeshState* m, int64_t zones);
// Scratch zones a split tile needs for the task list (tile, side), capped.
int64_t split_need(MeshState* m, int tile, int side);
int mesh_partition(const BssnBlockDesc* blocks, int nblocks, int nparts, int32_t* part);
int mesh_generate(int mode, const int32_t dims[3], const double p[4], uint64_t seed,
                  double xmin, double L, BssnBlockDesc* blocks, int* nblocks,
                  int32_t G[3], double* h);

}  // namespace bssn
