// The extern "C" entry points of include/bssn_b200.h: argument checks and
// kernel launches.  No entry point allocates device memory except the mesh
// handle's creation and its first use of a tile shape (task list upload),
// plan creation, and the first diagnostics call of a plan.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

#include "bssn_b200.h"
#include "bssn_common.cuh"
#include "kernels.cuh"
#include "mesh.h"
#include "plan.h"
#include "constraints.h"
#include "remesh.h"
#include "rhs_fused.cuh"

struct bssn_mesh_s {
    bssn::MeshState* st;
};

struct bssn_rk4_plan_s {
    bssn::Plan* p;
};

namespace {

bool valid_side(int s) { return s == 13 || s == 19 || s == 31 || s == 55; }

cudaStream_t S(bssn_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// the tile used before tuning: the split 7x7x7 brick (fastest on every
// block size measured on B200)
int default_tile() { return bssn::default_split_tile(); }

int tile_for_side(const bssn::MeshState* m, int side) {
    auto it = m->tuned.find(side);
    return it == m->tuned.end() ? default_tile() : it->second;
}

}  // namespace

extern "C" {

const char* bssn_version(void) { return "bssn-b200 0.1 (sm_100a, FP64)"; }

int bssn_deriv644_f64(int kind, double* D_dev, const double* u_dev, double h,
                      const unsigned sz[3], unsigned bflag, bssn_stream_t stream) {
    if (!D_dev || !u_dev || !sz) return BSSN_EINVAL;
    if (kind < 0 || kind > 8) return BSSN_EKIND;
    for (int d = 0; d < 3; d++)
        if (sz[d] < 12) return BSSN_EBLOCKSIZE;
    return bssn::launch_stencil(kind, D_dev, u_dev, h, sz, bflag, S(stream));
}

int bssn_deriv644adv_f64(int dir, double* D_dev, const double* u_dev, double h,
                         const unsigned sz[3], const double* beta_dev, unsigned bflag,
                         bssn_stream_t stream) {
    (void)beta_dev;
    if (dir < 0 || dir > 2) return BSSN_EKIND;
    return bssn_deriv644_f64(dir, D_dev, u_dev, h, sz, bflag, stream);
}

int bssn_bssnrhs_f64(double* const* rhs_dev, const double* const* u_dev, int64_t offset,
                     const double pmin[3], const double pmax[3], const unsigned sz[3],
                     unsigned bflag, const BssnParams* params, bssn_stream_t stream) {
    if (!rhs_dev || !u_dev || !pmin || !pmax || !sz || !params) return BSSN_EINVAL;
    if (sz[0] != sz[1] || sz[1] != sz[2] || !valid_side((int)sz[0])) return BSSN_EBLOCKSIZE;
    bssn::RhsArgs A;
    for (int v = 0; v < bssn::NVARS; v++) {
        if (!u_dev[v] || !rhs_dev[v]) return BSSN_EINVAL;
        A.u.p[v] = u_dev[v];
        A.rhs.p[v] = rhs_dev[v];
    }
    A.prm = *params;
    BssnBlockDesc b;
    std::memset(&b, 0, sizeof(b));
    b.offset = offset;
    b.sz = (int32_t)sz[0];
    b.bflag = bflag;
    for (int d = 0; d < 3; d++) {
        b.ptmin[d] = pmin[d];
        b.ptmax[d] = pmax[d];
    }
    return bssn::launch_rhs_single(default_tile(), A, b, S(stream));
}

int bssn_mesh_create(const BssnBlockDesc* blocks, int nblocks, const int32_t G[3],
                     bssn_mesh* out) {
    if (!blocks || nblocks <= 0 || !G || !out) return BSSN_EINVAL;
    for (int b = 0; b < nblocks; b++)
        if (!valid_side(blocks[b].sz) || blocks[b].offset < 0) return BSSN_EBLOCKSIZE;
    bssn::MeshState* st = nullptr;
    int r = bssn::mesh_create(blocks, nblocks, G, &st);
    if (r) return r;
    *out = new bssn_mesh_s{st};
    return 0;
}

int bssn_mesh_destroy(bssn_mesh mesh) {
    if (!mesh) return BSSN_EINVAL;
    bssn::mesh_destroy(mesh->st);
    delete mesh;
    return 0;
}

int64_t bssn_mesh_unzip_size(bssn_mesh mesh) { return mesh ? mesh->st->unzip_size : -1; }

int bssn_rhs_blocks_f64(bssn_mesh mesh, double* const* rhs_dev, const double* const* u_dev,
                        const BssnParams* params, int tile, bssn_stream_t stream) {
    if (!mesh || !rhs_dev || !u_dev || !params) return BSSN_EINVAL;
    if (tile < -1 || tile >= bssn::tile_count()) return BSSN_EINVAL;
    bssn::RhsArgs A;
    for (int v = 0; v < bssn::NVARS; v++) {
        if (!u_dev[v] || !rhs_dev[v]) return BSSN_EINVAL;
        A.u.p[v] = u_dev[v];
        A.rhs.p[v] = rhs_dev[v];
    }
    A.prm = *params;
    const int t = tile >= 0 ? tile : tile_for_side(mesh->st, 0);
    const bssn::BrickTask* tasks;
    int ntasks;
    int r = bssn::mesh_tasks(mesh->st, t, &tasks, &ntasks);
    if (!r) r = bssn::mesh_scratch(mesh->st, bssn::split_need(mesh->st, t, 0));
    if (r) return r;
    return bssn::launch_rhs_tasks(t, A, mesh->st->d_blocks, tasks, ntasks, S(stream),
                                  mesh->st->d_scratch, mesh->st->scratch_zones);
}

int bssn_unzip_f64(bssn_mesh mesh, double* const* unzip_dev, const double* const* zip_dev,
                   int nvars, bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !zip_dev || nvars < 1 || nvars > bssn::NVARS) return BSSN_EINVAL;
    if (mesh->st->lv) return bssn::launch_levels_unzip(*mesh->st->lv, unzip_dev, zip_dev, nvars, S(stream));
    return bssn::launch_unzip(mesh->st, unzip_dev, zip_dev, nvars, S(stream));
}

int bssn_zip_f64(bssn_mesh mesh, double* const* zip_dev, const double* const* unzip_dev,
                 int nvars, bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !zip_dev || nvars < 1 || nvars > bssn::NVARS) return BSSN_EINVAL;
    if (mesh->st->lv) return bssn::launch_levels_zip(*mesh->st->lv, zip_dev, unzip_dev, nvars, S(stream));
    return bssn::launch_zip(mesh->st, zip_dev, unzip_dev, nvars, S(stream));
}

namespace {
int create_patch_mesh(const BssnBlockDesc* blocks, int nblocks, const std::vector<bssn::PatchDef>& P,
                      const int32_t M0[3], bssn_mesh* out);
}

int bssn_mesh_create_levels(const BssnBlockDesc* blocks, int nblocks, int nlevels, const int32_t M0[3],
                            const BssnLevelBox* boxes, bssn_mesh* out) {
    return create_patch_mesh(blocks, nblocks, bssn::chain_patches(nlevels, boxes), M0, out);
}

int bssn_mesh_create_patches(const BssnBlockDesc* blocks, int nblocks, int npatches, const int32_t M0[3],
                             const BssnPatch* patches, bssn_mesh* out) {
    return create_patch_mesh(blocks, nblocks, bssn::patches_from(npatches, patches), M0, out);
}

}  // extern "C"

namespace {
int create_patch_mesh(const BssnBlockDesc* blocks, int nblocks, const std::vector<bssn::PatchDef>& P,
                      const int32_t M0[3], bssn_mesh* out) {
    if (!blocks || nblocks <= 0 || !out) return BSSN_EINVAL;
    for (int b = 0; b < nblocks; b++)
        if (!valid_side(blocks[b].sz) || blocks[b].offset < 0) return BSSN_EBLOCKSIZE;
    bssn::LevelMaps maps;
    int r = bssn::levels_build(blocks, nblocks, P, M0, &maps);
    if (r) return r;
    // the node "grid" of a multi-level mesh is its concatenated level grids
    const int32_t G[3] = {(int32_t)maps.n_nodes, 1, 1};
    bssn::MeshState* st = nullptr;
    r = bssn::mesh_create(blocks, nblocks, G, &st);
    if (r) return r;
    st->lv = new bssn::LevelsDev();
    r = bssn::levels_upload(maps, st->lv);
    if (r) {
        bssn::mesh_destroy(st);
        return r;
    }
    *out = new bssn_mesh_s{st};
    return 0;
}
}  // namespace

extern "C" {

int bssn_levels_transfer(bssn_mesh from, const double* const* u_old_dev, bssn_mesh to,
                         double* const* u_new_dev, int nvars, bssn_stream_t stream) {
    if (!from || !to || !u_old_dev || !u_new_dev || nvars < 1 || nvars > bssn::NVARS) return BSSN_EINVAL;
    if (!from->st->lv || !to->st->lv) return BSSN_ESTATE;  // level meshes only
    for (int v = 0; v < nvars; v++)
        if (!u_old_dev[v] || !u_new_dev[v]) return BSSN_EINVAL;
    return bssn::levels_transfer(*from->st->lv, u_old_dev, *to->st->lv, u_new_dev, nvars, S(stream));
}

int bssn_mesh_levels_sync(bssn_mesh mesh, double* const* u_dev, int nvars, bssn_stream_t stream) {
    if (!mesh || !u_dev || nvars < 1 || nvars > bssn::NVARS) return BSSN_EINVAL;
    for (int v = 0; v < nvars; v++)
        if (!u_dev[v]) return BSSN_EINVAL;
    if (!mesh->st->lv) return 0;  // single-level meshes have nothing to sync
    return bssn::launch_levels_sync(*mesh->st->lv, u_dev, nvars, S(stream));
}

int bssn_rk4_stage_f64(int stage, double* const* out_dev, const double* const* u_prev_dev,
                       const double* const* k_dev, int64_t n, double dt, int enforce,
                       double chi_floor, int* status_dev, bssn_stream_t stream) {
    if (stage < 0 || stage > 3 || !out_dev || !u_prev_dev || !k_dev || n < 0) return BSSN_EINVAL;
    if (n == 0) return 0;
    return bssn::launch_rk4_stage(stage, out_dev, u_prev_dev, k_dev, n, dt, enforce,
                                  chi_floor, status_dev, S(stream));
}

int bssn_enforce_f64(double* const* u_dev, int64_t n, double chi_floor, int* status_dev,
                     bssn_stream_t stream) {
    if (!u_dev || n < 0) return BSSN_EINVAL;
    if (n == 0) return 0;
    return bssn::launch_enforce(u_dev, n, chi_floor, status_dev, S(stream));
}

int bssn_initial_data_f64(double* const* u_dev, const int32_t G[3], const double xmin[3],
                          double h, const double bh[6], double m1, double m2,
                          double chi_floor, double eps, uint64_t seed, bssn_stream_t stream) {
    if (!u_dev || !G || !xmin || !bh) return BSSN_EINVAL;
    return bssn::launch_initial_data(u_dev, G, xmin, h, bh, m1, m2, chi_floor, eps, seed,
                                     S(stream));
}

int bssn_mesh_generate(int mode, const int32_t dims[3], const double p[4], uint64_t seed,
                       double xmin, double L, BssnBlockDesc* blocks, int* nblocks,
                       int32_t G[3], double* h) {
    if (!dims || !nblocks || !G || !h || (mode == 1 && !p)) return BSSN_EINVAL;
    return bssn::mesh_generate(mode, dims, p, seed, xmin, L, blocks, nblocks, G, h);
}

int bssn_rk4_plan_create(bssn_mesh mesh, const BssnParams* params, int flags,
                         bssn_rk4_plan* out) {
    if (!mesh || !params || !out) return BSSN_EINVAL;
    bssn::Plan* p = nullptr;
    int st = bssn::plan_create(mesh->st, *params, flags, &p);
    if (st) return st;
    *out = new bssn_rk4_plan_s{p};
    return 0;
}

int bssn_rk4_plan_step(bssn_rk4_plan plan, double* const* u_dev, double dt,
                       bssn_stream_t stream) {
    if (!plan || !u_dev) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++)
        if (!u_dev[v]) return BSSN_EINVAL;
    return bssn::plan_step(plan->p, u_dev, dt, S(stream));
}

namespace {
int diag_args(const double xmin[3], double h, const double bh[6], const double radii[2],
              double* norms_dev, bssn::DiagArgs* d) {
    if (!xmin || !bh || !radii || !norms_dev || !(h > 0.0)) return BSSN_EINVAL;
    for (int i = 0; i < 3; i++) d->xmin[i] = xmin[i];
    for (int i = 0; i < 6; i++) d->bh[i] = bh[i];
    d->radii[0] = radii[0];
    d->radii[1] = radii[1];
    d->h = h;
    d->norms = norms_dev;
    return BSSN_OK;
}
}  // namespace

int bssn_rk4_plan_diagnostics(bssn_rk4_plan plan, double* const* u_dev, const double xmin[3],
                              double h, const double bh[6], const double radii[2],
                              double* norms_dev, bssn_stream_t stream) {
    if (!plan || !u_dev) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++)
        if (!u_dev[v]) return BSSN_EINVAL;
    bssn::DiagArgs d;
    const int st = diag_args(xmin, h, bh, radii, norms_dev, &d);
    return st ? st : bssn::plan_diag(plan->p, u_dev, d, S(stream));
}

int bssn_rk4_plan_diag_fields(bssn_rk4_plan plan, double** fields_dev) {
    if (!plan || !fields_dev) return BSSN_EINVAL;
    bssn::Plan* p = plan->p;
    if (!p->cons) return BSSN_ESTATE;
    const int nf = (p->flags & BSSN_PLAN_DIAG_PSI4) ? 6 : 4;
    for (int c = 0; c < 6; c++) fields_dev[c] = c < nf ? p->cons + (size_t)c * p->n_nodes : nullptr;
    return 0;
}

int bssn_rk4_plan_copy_diag_fields(bssn_rk4_plan plan, double* const* dst_dev, int nfields,
                                   bssn_stream_t stream) {
    double* f[6];
    int st = bssn_rk4_plan_diag_fields(plan, f);
    if (st) return st;
    if (!dst_dev || nfields < 1 || nfields > 6 || !f[nfields - 1]) return BSSN_EINVAL;
    for (int c = 0; c < nfields; c++) {
        if (!dst_dev[c]) return BSSN_EINVAL;
        st = bssn::cuda_status(cudaMemcpyAsync(dst_dev[c], f[c], sizeof(double) * plan->p->n_nodes,
                                               cudaMemcpyDeviceToDevice, S(stream)));
        if (st) return st;
    }
    return 0;
}

int bssn_rk4_plan_step_diag(bssn_rk4_plan plan, double* const* u_dev, double dt,
                            const double xmin[3], double h, const double bh[6],
                            const double radii[2], double* norms_dev, bssn_stream_t stream) {
    if (!plan || !u_dev) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++)
        if (!u_dev[v]) return BSSN_EINVAL;
    bssn::DiagArgs d;
    const int st = diag_args(xmin, h, bh, radii, norms_dev, &d);
    return st ? st : bssn::plan_step_diag(plan->p, u_dev, dt, d, S(stream));
}

int bssn_rk4_plan_autotune(bssn_rk4_plan plan, double* const* u_dev, int reps,
                           bssn_stream_t stream, float* times) {
    if (!plan || !u_dev || reps < 1) return BSSN_EINVAL;
    return bssn::plan_autotune(plan->p, u_dev, reps, S(stream), times);
}

int bssn_rk4_plan_set_tile(bssn_rk4_plan plan, int side, int tile) {
    if (!plan) return BSSN_EINVAL;
    return bssn::plan_set_tile(plan->p, side, tile);
}

int bssn_rk4_plan_tile(bssn_rk4_plan plan, int side) {
    if (!plan) return -BSSN_EINVAL;
    return bssn::plan_tile(plan->p, side);
}

int bssn_rk4_plan_violations(bssn_rk4_plan plan, int* count) {
    if (!plan || !count) return BSSN_EINVAL;
    return bssn::cuda_status(cudaMemcpy(count, plan->p->status, sizeof(int), cudaMemcpyDeviceToHost));
}

int bssn_rk4_plan_time_rhs(bssn_rk4_plan plan, int reps, bssn_stream_t stream, float* ms) {
    if (!plan || reps < 1 || !ms) return BSSN_EINVAL;
    return bssn::plan_time_rhs(plan->p, reps, S(stream), ms);
}

int bssn_rk4_plan_time_kernels(bssn_rk4_plan plan, int reps, bssn_stream_t stream, double out[6]) {
    if (!plan || reps < 1 || !out) return BSSN_EINVAL;
    return bssn::plan_time_kernels(plan->p, reps, S(stream), out);
}

int bssn_rk4_plan_launches_per_step(bssn_rk4_plan plan) {
    if (!plan) return BSSN_EINVAL;
    return bssn::plan_launches_per_step(plan->p);
}

int bssn_fp64_probe(double* scratch_dev, int iters, bssn_stream_t stream, double* tflops) {
    if (!scratch_dev || iters < 1 || !tflops) return BSSN_EINVAL;
    return bssn::fp64_probe(scratch_dev, iters, S(stream), tflops);
}

int bssn_rk4_plan_destroy(bssn_rk4_plan plan) {
    if (!plan) return BSSN_EINVAL;
    bssn::plan_destroy(plan->p);
    delete plan;
    return 0;
}

int bssn_constraints_f64(bssn_mesh mesh, const double* const* unzip_dev, double* const* cons_dev,
                         bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !cons_dev) return BSSN_EINVAL;
    for (int c = 0; c < 4; c++)
        if (!cons_dev[c]) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++)
        if (!unzip_dev[v]) return BSSN_EINVAL;
    return bssn::launch_constraints(mesh->st, unzip_dev, cons_dev, S(stream));
}

int bssn_constraints_psi4_f64(bssn_mesh mesh, const double* const* unzip_dev, double* const* cons_dev,
                              bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !cons_dev) return BSSN_EINVAL;
    for (int c = 0; c < 6; c++)
        if (!cons_dev[c]) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++)
        if (!unzip_dev[v]) return BSSN_EINVAL;
    return bssn::launch_constraints(mesh->st, unzip_dev, cons_dev, S(stream), true);
}

int bssn_constraint_norms_f64(bssn_mesh mesh, const double* const* cons_dev, int ncons,
                              const double xmin[3], double h, const double bh[6],
                              const double radii[2], double* norms_dev, bssn_stream_t stream) {
    if (!mesh || !cons_dev || ncons < 1 || ncons > 4 || !xmin || !bh || !radii || !norms_dev)
        return BSSN_EINVAL;
    if (mesh->st->lv) return BSSN_ESTATE;
    for (int c = 0; c < ncons; c++)
        if (!cons_dev[c]) return BSSN_EINVAL;
    // the reduction's partial sums live in a device buffer owned by the mesh
    // handle, allocated on the first call (5 doubles per reduction CTA)
    bssn::MeshState* m = mesh->st;
    const int npartial = bssn::kNormPartials;
    if (!m->d_partial) {
        if (cudaMalloc((void**)&m->d_partial, sizeof(double) * 5 * npartial) != cudaSuccess)
            return BSSN_ENOMEM;
    }
    return bssn::launch_l2_norms(m, cons_dev, ncons, xmin, h, bh, radii, m->d_partial, npartial,
                                 norms_dev, S(stream));
}

int bssn_constraint_sums_f64(bssn_mesh mesh, const double* const* cons_dev, int ncons,
                             const double xmin[3], double h, const double bh[6],
                             const double radii[2], const uint8_t* mask_dev, double* sums_dev,
                             bssn_stream_t stream) {
    if (!mesh || !cons_dev || ncons < 1 || ncons > 4 || !xmin || !bh || !radii || !sums_dev)
        return BSSN_EINVAL;
    if (mesh->st->lv) return BSSN_ESTATE;
    for (int c = 0; c < ncons; c++)
        if (!cons_dev[c]) return BSSN_EINVAL;
    bssn::MeshState* m = mesh->st;
    const int npartial = bssn::kNormPartials;
    if (!m->d_partial) {
        if (cudaMalloc((void**)&m->d_partial, sizeof(double) * 5 * npartial) != cudaSuccess)
            return BSSN_ENOMEM;
    }
    return bssn::launch_l2_norms(m, cons_dev, ncons, xmin, h, bh, radii, m->d_partial, npartial,
                                 sums_dev, S(stream), mask_dev, true);
}

int64_t bssn_mesh_num_elements(bssn_mesh mesh) {
    if (!mesh) return -1;
    int64_t n = 0;
    for (auto& b : mesh->st->blocks) {
        const int64_t w = (b.sz - 7) / 6;
        n += w * w * w;
    }
    return n;
}

int bssn_remesh_wavelet_f64(bssn_mesh mesh, const double* const* unzip_dev, int nvars, double tol,
                            double* scores_dev, double* ratio_dev, uint8_t* flags_dev,
                            bssn_stream_t stream) {
    if (!mesh || !unzip_dev || nvars < 1 || nvars > bssn::NVARS || !(tol > 0) || !scores_dev)
        return BSSN_EINVAL;
    int st = bssn::launch_wavelet_scores(mesh->st, unzip_dev, nvars, scores_dev, nullptr, S(stream));
    if (!st && (ratio_dev || flags_dev))
        st = bssn::launch_block_flags(mesh->st, scores_dev, nvars, tol, ratio_dev, flags_dev, nullptr,
                                      S(stream));
    return st;
}

int bssn_remesh_features_f64(bssn_mesh mesh, const double* const* unzip_dev, float* feats_dev,
                             bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !feats_dev) return BSSN_EINVAL;
    return bssn::launch_features(mesh->st, unzip_dev, feats_dev, S(stream));
}

int bssn_remesh_mlp_fwd_bf16(const void* wq_dev, const float* norm_dev, const float* x_dev, int n,
                             float* logits_dev, bssn_stream_t stream) {
    if (!wq_dev || !x_dev || !logits_dev || n < 0) return BSSN_EINVAL;
    return bssn::launch_mlp_fwd(wq_dev, norm_dev, x_dev, n, logits_dev, S(stream));
}

int bssn_remesh_mlp_fwd_fp32_bf16(const void* wq_dev, const float* norm_dev, const float* x_dev, int n,
                                  float* logits_dev, bssn_stream_t stream) {
    if (!wq_dev || !x_dev || !logits_dev || n < 0) return BSSN_EINVAL;
    return bssn::launch_mlp_fwd_fp32(wq_dev, norm_dev, x_dev, n, logits_dev, S(stream));
}

size_t bssn_remesh_mlp_grad_scratch(int n) { return n > 0 ? bssn::mlp_grad_scratch_floats(n) : 0; }

int bssn_remesh_mlp_bwd_bf16(const void* wq_dev, const float* norm_dev, const float* x_dev,
                             const float* y_dev, const float* c_dev, int n, float* grad_dev,
                             float* loss_dev, float* scratch_dev, bssn_stream_t stream) {
    if (!wq_dev || !x_dev || !y_dev || !grad_dev || !scratch_dev || n < 1) return BSSN_EINVAL;
    return bssn::launch_mlp_grad(wq_dev, norm_dev, x_dev, y_dev, c_dev, n, grad_dev, loss_dev,
                                 scratch_dev, S(stream));
}

int bssn_remesh_mlp_step_bf16(float* master_dev, void* wq_dev, const float* grad_dev, float* m_dev,
                              float* v_dev, float lr, float beta1, float beta2, float eps, int t,
                              bssn_stream_t stream) {
    if (!master_dev || !wq_dev || !grad_dev || !m_dev || !v_dev || t < 1) return BSSN_EINVAL;
    return bssn::launch_adam(master_dev, wq_dev, grad_dev, m_dev, v_dev, lr, beta1, beta2, eps, t,
                             S(stream));
}

size_t bssn_remesh_decide_work_bytes(bssn_mesh mesh) {
    if (!mesh) return 0;
    const size_t nb = mesh->st->blocks.size();
    const size_t ne = (size_t)bssn_mesh_num_elements(mesh);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    return al(nb * 16 * sizeof(float)) + al(nb * sizeof(float)) + 3 * al(nb) +
           al(ne * bssn::NVARS * sizeof(double));
}

int bssn_remesh_decide_f64(bssn_mesh mesh, const double* const* unzip_dev, const void* wq_dev,
                           const float* norm_dev, float lo, float hi, double audit_frac,
                           uint64_t seed, double tol, uint8_t* flags_dev, int* stats_dev,
                           void* work_dev, size_t work_bytes, bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !wq_dev || !flags_dev || !stats_dev || !work_dev) return BSSN_EINVAL;
    if (!(lo <= hi) || audit_frac < 0 || audit_frac > 1 || !(tol > 0)) return BSSN_EINVAL;
    if (work_bytes < bssn_remesh_decide_work_bytes(mesh)) return BSSN_EINVAL;
    bssn::MeshState* m = mesh->st;
    const int nb = (int)m->blocks.size();
    const int64_t ne = bssn_mesh_num_elements(mesh);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    char* w = (char*)work_dev;
    float* feats = (float*)w;
    w += al((size_t)nb * 16 * sizeof(float));
    float* logits = (float*)w;
    w += al((size_t)nb * sizeof(float));
    uint8_t* need = (uint8_t*)w;
    w += al(nb);
    uint8_t* decided = (uint8_t*)w;
    w += al(nb);
    uint8_t* exact = (uint8_t*)w;
    w += al(nb);
    double* scores = (double*)w;
    (void)ne;
    cudaStream_t s = S(stream);
    int st = cudaMemsetAsync(stats_dev, 0, 4 * sizeof(int), s) == cudaSuccess ? 0 : BSSN_EINVAL;
    if (!st) st = bssn::launch_features(m, unzip_dev, feats, s);
    if (!st) st = bssn::launch_mlp_fwd(wq_dev, norm_dev, feats, nb, logits, s);
    if (!st) st = bssn::launch_remesh_select(logits, nb, lo, hi, audit_frac, seed, need, decided, stats_dev, s);
    if (!st) st = bssn::launch_wavelet_scores(m, unzip_dev, bssn::NVARS, scores, need, s);
    if (!st) st = bssn::launch_block_flags(m, scores, bssn::NVARS, tol, nullptr, exact, need, s);
    if (!st) st = bssn::launch_remesh_merge(nb, need, decided, exact, logits, lo, stats_dev, flags_dev, s);
    return st;
}

size_t bssn_remesh_decide2_work_bytes(bssn_mesh mesh) {
    if (!mesh) return 0;
    const size_t nb = mesh->st->blocks.size();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    return bssn_remesh_decide_work_bytes(mesh) + al(nb * sizeof(float)) + al(nb * sizeof(double));
}

int bssn_remesh_decide2_f64(bssn_mesh mesh, const double* const* unzip_dev, const void* wq_refine,
                            const float* norm_refine, float lo_r, float hi_r, const void* wq_keep,
                            const float* norm_keep, float lo_k, float hi_k, double audit_frac,
                            uint64_t seed, double tol, double keep_fac, uint8_t* refine_dev,
                            uint8_t* keep_dev, int* stats_dev, void* work_dev, size_t work_bytes,
                            bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !wq_refine || !wq_keep || !refine_dev || !keep_dev || !stats_dev ||
        !work_dev)
        return BSSN_EINVAL;
    if (!(lo_r <= hi_r) || !(lo_k <= hi_k) || audit_frac < 0 || audit_frac > 1 || !(tol > 0) ||
        !(keep_fac > 0) || keep_fac > 1)
        return BSSN_EINVAL;
    if (work_bytes < bssn_remesh_decide2_work_bytes(mesh)) return BSSN_EINVAL;
    bssn::MeshState* m = mesh->st;
    const int nb = (int)m->blocks.size();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    char* w = (char*)work_dev;
    float* feats = (float*)w;
    w += al((size_t)nb * 16 * sizeof(float));
    float* lr = (float*)w;
    w += al((size_t)nb * sizeof(float));
    float* lk = (float*)w;
    w += al((size_t)nb * sizeof(float));
    uint8_t* need = (uint8_t*)w;
    w += al(nb);
    uint8_t* decided = (uint8_t*)w;
    w += al(nb);
    w += al(nb);  // (the one-flag decision's exact flags)
    double* ratio = (double*)w;
    w += al((size_t)nb * sizeof(double));
    double* scores = (double*)w;
    cudaStream_t s = S(stream);
    int st = cudaMemsetAsync(stats_dev, 0, 8 * sizeof(int), s) == cudaSuccess ? 0 : BSSN_EINVAL;
    if (!st) st = bssn::launch_features(m, unzip_dev, feats, s);
    if (!st) st = bssn::launch_mlp_fwd(wq_refine, norm_refine, feats, nb, lr, s);
    if (!st) st = bssn::launch_mlp_fwd(wq_keep, norm_keep, feats, nb, lk, s);
    if (!st)
        st = bssn::launch_remesh_select2(lr, lk, nb, lo_r, hi_r, lo_k, hi_k, audit_frac, seed, need,
                                         decided, stats_dev, s);
    if (!st) st = bssn::launch_wavelet_scores(m, unzip_dev, bssn::NVARS, scores, need, s);
    if (!st) st = bssn::launch_block_flags(m, scores, bssn::NVARS, tol, ratio, nullptr, need, s);
    if (!st)
        st = bssn::launch_remesh_merge2(nb, need, decided, ratio, keep_fac, lr, lk, lo_r, lo_k,
                                        stats_dev, refine_dev, keep_dev, s);
    return st;
}

int bssn_remesh_element_features_f64(bssn_mesh mesh, const double* const* unzip_dev, float* feats_dev,
                                     bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !feats_dev) return BSSN_EINVAL;
    return bssn::launch_element_features(mesh->st, unzip_dev, feats_dev, S(stream));
}

size_t bssn_remesh_decide2_elem_work_bytes(bssn_mesh mesh) {
    if (!mesh) return 0;
    const size_t ne = (size_t)bssn_mesh_num_elements(mesh);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    return al(ne * 16 * sizeof(float)) + 2 * al(ne * sizeof(float)) + 2 * al(ne) +
           al((ne + 2) * sizeof(int64_t)) + al(ne * sizeof(int32_t)) + al(ne * bssn::NVARS * sizeof(double));
}

int bssn_remesh_decide2_elem_f64(bssn_mesh mesh, const double* const* unzip_dev, const void* wq_refine,
                                 const float* norm_refine, float lo_r, float hi_r, const void* wq_keep,
                                 const float* norm_keep, float lo_k, float hi_k, double audit_frac,
                                 uint64_t seed, double tol, double keep_fac, uint8_t* refine_dev,
                                 uint8_t* keep_dev, int* stats_dev, void* work_dev, size_t work_bytes,
                                 bssn_stream_t stream) {
    if (!mesh || !unzip_dev || !wq_refine || !wq_keep || !refine_dev || !keep_dev || !stats_dev ||
        !work_dev)
        return BSSN_EINVAL;
    if (!(lo_r <= hi_r) || !(lo_k <= hi_k) || audit_frac < 0 || audit_frac > 1 || !(tol > 0) ||
        !(keep_fac > 0) || keep_fac > 1)
        return BSSN_EINVAL;
    if (work_bytes < bssn_remesh_decide2_elem_work_bytes(mesh)) return BSSN_EINVAL;
    bssn::MeshState* m = mesh->st;
    int st = bssn::remesh_elements(m);
    if (st) return st;
    const int64_t ne = m->n_elems;
    if (ne > 0x7fffffff) return BSSN_ELIMIT;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    char* w = (char*)work_dev;
    float* feats = (float*)w;
    w += al((size_t)ne * 16 * sizeof(float));
    float* lr = (float*)w;
    w += al((size_t)ne * sizeof(float));
    float* lk = (float*)w;
    w += al((size_t)ne * sizeof(float));
    uint8_t* need = (uint8_t*)w;
    w += al(ne);
    uint8_t* decided = (uint8_t*)w;
    w += al(ne);
    int64_t* off = (int64_t*)w;  // ne offsets, then the count
    w += al((size_t)(ne + 2) * sizeof(int64_t));
    int32_t* list = (int32_t*)w;
    w += al((size_t)ne * sizeof(int32_t));
    double* scores = (double*)w;
    cudaStream_t s = S(stream);
    st = cudaMemsetAsync(stats_dev, 0, 8 * sizeof(int), s) == cudaSuccess ? 0 : BSSN_EINVAL;
    if (!st) st = bssn::launch_element_features(m, unzip_dev, feats, s);
    if (!st) st = bssn::launch_mlp_fwd(wq_refine, norm_refine, feats, (int)ne, lr, s);
    if (!st) st = bssn::launch_mlp_fwd(wq_keep, norm_keep, feats, (int)ne, lk, s);
    if (!st)
        st = bssn::launch_remesh_select_elem(m, lr, lk, lo_r, hi_r, lo_k, hi_k, audit_frac, seed, need, decided,
                                             stats_dev, s);
    if (!st)
        st = bssn::launch_wavelet_elements(m, unzip_dev, bssn::NVARS, scores, need, off, off + ne + 1, list, s);
    if (!st)
        st = bssn::launch_remesh_merge_elem(m, need, decided, scores, bssn::NVARS, tol, keep_fac, lr, lk, lo_r,
                                            lo_k, stats_dev, refine_dev, keep_dev, s);
    return st;
}

int bssn_mesh_partition(const BssnBlockDesc* blocks, int nblocks, int nparts, int32_t* part) {
    return bssn::mesh_partition(blocks, nblocks, nparts, part);
}

int bssn_rk4_plan_stage(bssn_rk4_plan plan, double* const* u_dev, double dt, int stage,
                        bssn_stream_t stream) {
    if (!plan || !u_dev || stage < 0 || stage > 3) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++)
        if (!u_dev[v]) return BSSN_EINVAL;
    return bssn::plan_enqueue_stage(plan->p, u_dev, dt, stage, S(stream));
}

int bssn_rk4_plan_stage_state(bssn_rk4_plan plan, double** im_dev) {
    if (!plan || !im_dev) return BSSN_EINVAL;
    for (int v = 0; v < bssn::NVARS; v++) im_dev[v] = plan->p->im + (int64_t)v * plan->p->n_nodes;
    return 0;
}

int bssn_halo_pack_f64(double* buf_dev, const double* const* u_dev, const int64_t* idx_dev,
                       int64_t n, bssn_stream_t stream) {
    if (n < 0 || (n > 0 && (!buf_dev || !u_dev || !idx_dev))) return BSSN_EINVAL;
    return bssn::launch_halo_pack(buf_dev, u_dev, idx_dev, n, S(stream));
}

int bssn_halo_unpack_f64(double* const* u_dev, const double* buf_dev, const int64_t* idx_dev,
                         int64_t n, bssn_stream_t stream) {
    if (n < 0 || (n > 0 && (!buf_dev || !u_dev || !idx_dev))) return BSSN_EINVAL;
    return bssn::launch_halo_unpack(u_dev, buf_dev, idx_dev, n, S(stream));
}

int bssn_tile_count(void) { return bssn::tile_count(); }

long bssn_tile_selfcheck(int tile) { return bssn::tile_selfcheck(tile); }

int bssn_tile_mode(int tile) { return bssn::tile_mode(tile); }

int bssn_tile_info(int tile, int info[4]) {
    if (!info) return BSSN_EINVAL;
    return bssn::tile_info(tile, info);
}

}  // extern "C"

namespace bssn {

int set_smem_limit(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;  // (kernel, device)
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    std::lock_guard<std::mutex> lock(mu);
    if (done.count({kernel, dev})) return 0;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_status(e);
    done.insert({kernel, dev});
    return 0;
}

}  // namespace bssn
