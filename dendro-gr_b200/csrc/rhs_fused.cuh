// Launch interface of the fused right-hand-side kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "bssn_b200.h"
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

// Tiles: a brick shape run fused (one kernel, rhs_kernel), split (derivative
// pass + equation pass through a scratch of kSplitSlots doubles per zone) or
// on chip (one kernel, derivatives handed to the equations in registers,
// rhs_onchip.cu).
constexpr int kSplitSlots = 11 * 10 + 13 * 4;
// Largest scratch the mesh allocates for the split path (zones); longer task
// lists are processed in chunks.
constexpr int64_t kSplitScratchZonesMax = int64_t(6) << 20;

int tile_count();
int tile_mode(int tile);   // 0 fused, 1 split, 2 on chip, -1 unknown
// whether a tile's kernels can write zipped right-hand sides (split, on chip)
inline bool tile_zipped(int mode) { return mode == 1 || mode == 2; }
int default_split_tile();  // the split tile used before autotuning
int tile_zones(int tile);  // zones per brick (BX*BY*BZ)
long tile_selfcheck(int tile);
int prepare_all_tiles();
int tile_info(int tile, int info[4]);
void build_tasks(const BssnBlockDesc* blocks, int nblocks, int tile,
                 std::vector<BrickTask>& out);
// Optional timing of every right-hand-side launch: CUDA events recorded on
// the launch stream around each kernel, summed per kernel kind by collect()
// (blocking).
struct KernelTimer {
    enum Kind { FUSED = 0, DERIV = 1, EQ = 2, NKIND = 3 };
    std::vector<int> kind;
    std::vector<cudaEvent_t> ev;  // start, stop per launch
    int start(int k, cudaStream_t s) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return BSSN_ENOMEM;
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            return BSSN_ENOMEM;
        }
        kind.push_back(k);
        ev.push_back(a);
        ev.push_back(b);
        return cuda_status(cudaEventRecord(a, s));
    }
    int stop(cudaStream_t s) { return cuda_status(cudaEventRecord(ev.back(), s)); }
    // adds each kind's summed milliseconds to ms[NKIND] and its launch count
    // to n[NKIND]; releases the events
    int collect(double ms[NKIND], int n[NKIND]) {
        int st = 0;
        for (size_t i = 0; i < kind.size(); i++) {
            float t = 0;
            cudaError_t e = cudaEventSynchronize(ev[2 * i + 1]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
            if (e != cudaSuccess && !st) st = cuda_status(e);
            ms[kind[i]] += t;
            n[kind[i]] += 1;
        }
        for (auto e : ev) cudaEventDestroy(e);
        kind.clear();
        ev.clear();
        return st;
    }
};

// scratch / scratch_zones: the split path's scratch (kSplitSlots * zones
// doubles); ignored by fused tiles.  tm (optional): time each launch.
// zip_grid (optional, split tiles only): the node-grid dimensions of a
// single-level mesh; A.rhs then holds zipped right-hand sides, written once
// per node by the block owning it (zones that do not own their node are
// skipped), and A.u the zipped stage state (zip_in, direct form) or the
// padded one.
int launch_rhs_tasks(int tile, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, cudaStream_t s,
                     double* scratch, int64_t scratch_zones, KernelTimer* tm = nullptr,
                     const int32_t* zip_grid = nullptr, bool zip_in = true);
// bricks of one block of padded side `side` under a tile (build_tasks keeps
// a block's bricks together, blocks in mesh order)
int bricks_per_block(int tile, int side);
// kernel launches launch_rhs_tasks makes for a task list of ntasks bricks
int rhs_launch_count(int tile, int ntasks, int64_t scratch_zones);
// one block; a split tile runs its shape fused
int launch_rhs_single(int tile, const RhsArgs& A, const BssnBlockDesc& blk,
                      cudaStream_t s);

// on-chip path (rhs_onchip.cu); shape = index among the on-chip shapes
int onchip_shape_count();
int onchip_shape(int shape, int b[3]);
int prepare_onchip(int shape);
int launch_rhs_onchip(int shape, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                      const BrickTask* tasks_dev, int ntasks, cudaStream_t s, KernelTimer* tm,
                      const int32_t* zip_grid, bool zip_in);
int launch_rhs_onchip_single(int shape, const RhsArgs& A, const BssnBlockDesc& blk, cudaStream_t s);

// split path (rhs_split.cu); shape = index among the split shapes
int split_shape_count();
int split_zone_count(int shape);
int prepare_split(int shape);
int launch_rhs_split(int shape, const RhsArgs& A, const BssnBlockDesc* blocks_dev,
                     const BrickTask* tasks_dev, int ntasks, double* scratch,
                     int64_t scratch_zones, cudaStream_t s, KernelTimer* tm = nullptr,
                     const int32_t* zip_grid = nullptr, bool zip_in = true);

}  // namespace bssn
