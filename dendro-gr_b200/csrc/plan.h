// RK4 plan state behind the bssn_rk4_plan handle.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "bssn_b200.h"
#include "bssn_common.cuh"
#include "mesh.h"

namespace bssn {

struct Plan {
    MeshState* mesh = nullptr;
    BssnParams prm;
    int flags = 0;
    int64_t n_nodes = 0;
    // direct: the right-hand side reads the zipped stage state and writes a
    // zipped right-hand side (no ghost fill, no padded arrays); otherwise the
    // ghost fill -> padded right-hand side -> zip-stage sequence
    bool direct = false;
    double* Rz = nullptr;   // zipped right-hand side (direct form, or split buckets)
    double* P = nullptr;    // padded stage state (24 x unzip size)
    double* R = nullptr;    // padded right-hand side
    double* im = nullptr;   // zipped intermediate stage state
    double* acc = nullptr;  // zipped RK4 accumulator
    int* status = nullptr;  // enforcement violations (device)
    std::vector<int> sides; // block-size buckets present
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap_stream = nullptr;  // capture stream of the graph
    double* graph_u[NVARS] = {nullptr};
    double graph_dt = 0.0;
    // constraint diagnostics: zipped ham, mom0..2 (allocated on first use)
    // and the graph of one step followed by the diagnostics
    double* cons = nullptr;
    cudaGraph_t graph_diag = nullptr;
    cudaGraphExec_t exec_diag = nullptr;
    double* diag_u[NVARS] = {nullptr};
    double diag_key[14] = {0};  // dt, xmin[3], h, bh[6], radii[2], norms pointer
};

// Where the diagnostics go: masked L2 norms of ham, mom0..2 over the nodes
// farther than radii from the punctures bh (node coordinates xmin + g*h),
// written to norms (4 doubles, device).
struct DiagArgs {
    double xmin[3];
    double h;
    double bh[6];
    double radii[2];
    double* norms;
};

int plan_create(MeshState* m, const BssnParams& prm, int flags, Plan** out);
void plan_destroy(Plan* p);
int plan_step(Plan* p, double* const* u, double dt, cudaStream_t s);
int plan_enqueue_stage(Plan* p, double* const* u, double dt, int stage, cudaStream_t s);
int plan_autotune(Plan* p, double* const* u, int reps, cudaStream_t s, float* times_out);
int plan_tile(const Plan* p, int side);
int plan_set_tile(Plan* p, int side, int tile);
int plan_time_rhs(Plan* p, int reps, cudaStream_t s, float* ms);
int plan_time_kernels(Plan* p, int reps, cudaStream_t s, double out[6]);
int plan_launches_per_step(Plan* p);
int plan_diag(Plan* p, double* const* u, const DiagArgs& d, cudaStream_t s);
int plan_step_diag(Plan* p, double* const* u, double dt, const DiagArgs& d, cudaStream_t s);
int fp64_probe(double* scratch, int iters, cudaStream_t s, double* tflops);

}  // namespace bssn
