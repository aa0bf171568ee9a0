// Launch interface of the fused right-hand-side kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "bssn_common.cuh"

namespace bssn {

struct RhsArgs {
    ConstVars u;
    MutVars rhs;
    BssnParams prm;
};

// One brick: block index, interior origin and extent per axis.
struct BrickTask {
    int32_t blk;
    int16_t o[3];
    int16_t e[3];
};

// Tiles: a brick shape run either fused (one kernel) or split (derivative
// pass + equation pass through a scratch of kSplitSlots doubles per zone).
constexpr int kSplitSlots = 11 * 10 + 13 * 4;
// Largest scratch the mesh allocates for the split path (zones); longer task
// lists are processed in chunks.
constexpr int64_t kSplitScratchZonesMax = int64_t(6) << 20;

int tile_count();
int tile_mode(int tile);   // 0 fused, 1 split, -1 unknown
int tile_zones(int tile);  // zones per brick (BX*BY*BZ)
long tile_selfcheck(int tile);
int prepare_all_tiles();
int tile_info(int tile, int info[4]);
void build_tasks(const BssnBlockDesc* blocks, int nblocks, int tile,
                 std::vector<BrickTask>& out);
// scratch / scratch_zones: the split path's scratch (kSplitSlots * zones
// doubles); ignored by fused tiles.
int launch_rhs_tasks(int tile, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, cudaStream_t s,
                     double* scratch, int64_t scratch_zones);
// one block; a split tile runs its shape fused
int launch_rhs_single(int tile, const RhsArgs& A, const BssnBlockDesc& blk,
                      cudaStream_t s);

// split path (rhs_split.cu); shape = index among the split shapes
int split_shape_count();
int split_zone_count(int shape);
int prepare_split(int shape);
int launch_rhs_split(int shape, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, double* scratch,
                     int64_t scratch_zones, cudaStream_t s);

}  // namespace bssn
