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

int tile_count();
long tile_selfcheck(int tile);
int prepare_all_tiles();
int tile_info(int tile, int info[4]);
void build_tasks(const BssnBlockDesc* blocks, int nblocks, int tile,
                 std::vector<BrickTask>& out);
int launch_rhs_tasks(int tile, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, cudaStream_t s);
int launch_rhs_single(int tile, const RhsArgs& A, const BssnBlockDesc& blk,
                      cudaStream_t s);

}  // namespace bssn
