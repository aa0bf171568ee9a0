// The whole RK4 step as one plan: per stage a ghost fill (unzip), the fused
// right-hand side over every brick of every block (one launch per block-size
// bucket with that bucket's autotuned tile), and the zip fused with the stage
// algebra.  Optionally captured once as a CUDA graph and replayed, or run as
// the plain path with one right-hand-side launch per block (the structure of
// the reference's bssnRHS block loop, rhs.cpp:10-73) for comparison.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <vector>

#include "bssn_b200.h"
#include "bssn_common.cuh"
#include "constraints.h"
#include "kernels.cuh"
#include "mesh.h"
#include "plan.h"
#include "rhs_fused.cuh"

namespace bssn {

namespace {

int alloc(double** p, size_t n) {
    *p = nullptr;
    if (n == 0) return 0;
    return cudaMalloc((void**)p, n * sizeof(double)) == cudaSuccess ? 0 : BSSN_ENOMEM;
}

void set_ptrs(double* base, int64_t n, double* out[NVARS]) {
    for (int v = 0; v < NVARS; v++) out[v] = base + v * n;
}

}  // namespace

int plan_create(MeshState* m, const BssnParams& prm, int flags, Plan** out) {
    Plan* p = new Plan();
    p->mesh = m;
    p->prm = prm;
    p->flags = flags;
    const int64_t nu = m->unzip_size;
    const int64_t nn = (int64_t)m->G[0] * m->G[1] * m->G[2];
    p->n_nodes = nn;
    // node indices of the direct path are 32-bit
    p->direct = (flags & BSSN_PLAN_DIRECT) && !(flags & BSSN_PLAN_PER_BLOCK) && !m->lv &&
                nn < (int64_t(1) << 31);
    int st = 0;
    if (p->direct) {
        st = alloc(&p->Rz, (size_t)NVARS * nn);
        if (!st) st = cuda_status(cudaMemset(p->Rz, 0, sizeof(double) * NVARS * nn));
    } else {
        st = alloc(&p->P, (size_t)NVARS * nu);
        if (!st) st = alloc(&p->R, (size_t)NVARS * nu);
        // zipped right-hand side of the split passes (32-bit node indices)
        if (!st && nn < (int64_t(1) << 31)) st = alloc(&p->Rz, (size_t)NVARS * nn);
        // padded buffers start at zero so never-written points stay finite
        if (!st) st = cuda_status(cudaMemset(p->P, 0, sizeof(double) * NVARS * nu));
        if (!st) st = cuda_status(cudaMemset(p->R, 0, sizeof(double) * NVARS * nu));
    }
    if (!st) st = alloc(&p->im, (size_t)NVARS * nn);
    if (!st) st = alloc(&p->acc, (size_t)NVARS * nn);
    if (!st) st = cuda_status(cudaMemset(p->im, 0, sizeof(double) * NVARS * nn));
    if (!st) st = cuda_status(cudaMemset(p->acc, 0, sizeof(double) * NVARS * nn));
    if (!st && cudaMalloc((void**)&p->status, sizeof(int)) != cudaSuccess) st = BSSN_ENOMEM;
    if (!st) st = cuda_status(cudaMemset(p->status, 0, sizeof(int)));
    if (st) {
        plan_destroy(p);
        return st;
    }
    std::set<int> sides;
    for (auto& b : m->blocks) sides.insert(b.sz);
    p->sides.assign(sides.begin(), sides.end());
    // task lists, the split-path scratch and kernel attributes must exist
    // before any graph capture
    int64_t need = 0;
    // direct plans: one Z-ordered list over all blocks per split tile;
    // padded plans: one list per block-size bucket and tile
    std::vector<int> keys = p->direct ? std::vector<int>{kAllZOrder} : p->sides;
    for (int key : keys) {
        for (int t = 0; t < tile_count(); t++) {
            if (p->direct && !tile_zipped(tile_mode(t))) continue;
            const BrickTask* tk;
            int nt;
            st = mesh_tasks_side(m, t, key, &tk, &nt);
            if (st) {
                plan_destroy(p);
                return st;
            }
            need = std::max(need, split_need(m, t, key));
        }
    }
    st = mesh_scratch(m, need);
    if (st) {
        plan_destroy(p);
        return st;
    }
    st = prepare_all_tiles();
    if (st) {
        plan_destroy(p);
        return st;
    }
    *out = p;
    return 0;
}

// Ghost fill of every block of the mesh (through the level maps on a
// multi-level mesh).
static int unzip_all(MeshState* m, double* const* P, const double* const* U, cudaStream_t s) {
    return m->lv ? launch_levels_unzip(*m->lv, P, U, NVARS, s) : launch_unzip(m, P, U, NVARS, s);
}

// Releases the captured graphs (the next step captures them again).
static void drop_graphs(Plan* p) {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->exec_diag) cudaGraphExecDestroy(p->exec_diag);
    if (p->graph_diag) cudaGraphDestroy(p->graph_diag);
    p->exec = p->exec_diag = nullptr;
    p->graph = p->graph_diag = nullptr;
}

void plan_destroy(Plan* p) {
    if (!p) return;
    drop_graphs(p);
    if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
    cudaFree(p->cons);
    cudaFree(p->Rz);
    cudaFree(p->P);
    cudaFree(p->R);
    cudaFree(p->im);
    cudaFree(p->acc);
    cudaFree(p->status);
    delete p;
}

// The tile a plan runs for blocks of side `side`: direct plans run one split
// tile over all blocks (tuned under the key kAllZOrder), padded plans the
// tile tuned for the side.
int plan_tile(const Plan* p, int side) {
    auto it = p->mesh->tuned.find(p->direct ? kAllZOrder : side);
    const int t = it == p->mesh->tuned.end() ? -1 : it->second;
    if (p->direct) return (t >= 0 && tile_zipped(tile_mode(t))) ? t : default_split_tile();
    return t >= 0 ? t : default_split_tile();
}

int plan_set_tile(Plan* p, int side, int tile) {
    if (tile < 0 || tile >= tile_count()) return BSSN_EINVAL;
    if (p->direct) {
        if (!tile_zipped(tile_mode(tile))) return BSSN_EINVAL;
        p->mesh->tuned[kAllZOrder] = tile;
    } else if (side == 0) {
        for (int sd : p->sides) p->mesh->tuned[sd] = tile;
    } else {
        p->mesh->tuned[side] = tile;
    }
    drop_graphs(p);  // recapture with the new tile on the next step
    return 0;
}

// Whether a padded plan writes its right-hand side zipped (every bucket on a
// split tile): the split passes then write each node once, from the block
// owning it, and a node-wise kernel applies the stage (no zip gather).
bool plan_zipped_rhs(const Plan* p) {
    if (p->direct || !p->Rz || (p->flags & BSSN_PLAN_PER_BLOCK) || p->mesh->lv) return false;
    for (int side : p->sides)
        if (!tile_zipped(tile_mode(plan_tile(p, side)))) return false;
    return true;
}

// One right-hand-side pass over every bucket.  Direct plans read the zipped
// stage state `src` and write Rz; the others read the padded P (filled by
// the ghost fill) and write R, or Rz when plan_zipped_rhs.
int plan_rhs(Plan* p, cudaStream_t s, KernelTimer* tm, const double* const* src) {
    MeshState* m = p->mesh;
    RhsArgs A;
    A.prm = p->prm;
    if (p->direct) {
        double* Rz[NVARS];
        set_ptrs(p->Rz, p->n_nodes, Rz);
        for (int v = 0; v < NVARS; v++) {
            A.u.p[v] = src[v];
            A.rhs.p[v] = Rz[v];
        }
        const int t = plan_tile(p, kAllZOrder);
        const BrickTask* tk;
        int nt;
        int st = mesh_tasks_side(m, t, kAllZOrder, &tk, &nt);
        if (!st)
            st = launch_rhs_tasks(t, A, m->d_blocks, tk, nt, s, m->d_scratch, m->scratch_zones, tm,
                                  m->G);
        return st;
    }
    double* Pp[NVARS];
    double* Rp[NVARS];
    const bool zrhs = plan_zipped_rhs(p);
    set_ptrs(p->P, m->unzip_size, Pp);
    if (zrhs)
        set_ptrs(p->Rz, p->n_nodes, Rp);
    else
        set_ptrs(p->R, m->unzip_size, Rp);
    for (int v = 0; v < NVARS; v++) {
        A.u.p[v] = Pp[v];
        A.rhs.p[v] = Rp[v];
    }
    if (p->flags & BSSN_PLAN_PER_BLOCK) {
        // the reference's block loop (rhs.cpp:10-73): blocks in mesh order,
        // each with its own launch(es) of the kernel the batched plan runs
        // for its side (split tiles: the block's bricks of the bucket's task
        // list, derivative + equation launch; the others: one launch)
        std::map<int, int> seen;  // blocks of each side visited so far
        for (auto& b : m->blocks) {
            const int t = plan_tile(p, b.sz);
            const int j = seen[b.sz]++;
            int st;
            if (tile_mode(t) == 1) {
                const BrickTask* tk;
                int nt;
                st = mesh_tasks_side(m, t, b.sz, &tk, &nt);
                const int per = bricks_per_block(t, b.sz);
                if (!st && (j + 1) * per > nt) st = BSSN_ESTATE;
                if (!st)
                    st = launch_rhs_tasks(t, A, m->d_blocks, tk + (size_t)j * per, per, s, m->d_scratch,
                                          m->scratch_zones, tm);
            } else {
                st = launch_rhs_single(t, A, b, s);
            }
            if (st) return st;
        }
        return 0;
    }
    // zipped right-hand side: blocks of kDirectMinSide and more stage from
    // the zipped stage state `src` (no ghost fill for them)
    RhsArgs Ad = A;
    if (zrhs && src)
        for (int v = 0; v < NVARS; v++) Ad.u.p[v] = src[v];
    for (int side : p->sides) {
        const int t = plan_tile(p, side);
        const BrickTask* tk;
        int nt;
        int st = mesh_tasks_side(m, t, side, &tk, &nt);
        const bool direct = zrhs && src && side >= kDirectMinSide;
        if (!st)
            st = launch_rhs_tasks(t, direct ? Ad : A, m->d_blocks, tk, nt, s, m->d_scratch,
                                  m->scratch_zones, tm, zrhs ? m->G : nullptr, direct);
        if (st) return st;
    }
    return 0;
}

// One RK4 stage (0..3) of the step from state u: stage 0 reads u, the others
// the plan's intermediate stage state; stages 0..2 write that state and the
// accumulator, stage 3 writes u.  Each form's own sequence (see the header).
int plan_enqueue_stage(Plan* p, double* const* u, double dt, int stage, cudaStream_t s) {
    MeshState* m = p->mesh;
    double* Pp[NVARS];
    double* Rp[NVARS];
    double* Ip[NVARS];
    double* Ap[NVARS];
    set_ptrs(p->P, m->unzip_size, Pp);
    set_ptrs(p->R, m->unzip_size, Rp);
    set_ptrs(p->im, p->n_nodes, Ip);
    set_ptrs(p->acc, p->n_nodes, Ap);
    const int enf = (p->flags & BSSN_PLAN_ENFORCE_STAGES) ? 1 : 0;
    const double* const* src = stage == 0 ? (const double* const*)u : (const double* const*)Ip;
    if (m->lv) {
        // multi-level mesh: ghost fill through the level maps, right-hand
        // side per block (each with its level's spacing), node-wise stage
        // reading each node's right-hand side at its owning zone, level sync
        // of the state just written
        int st = launch_levels_unzip(*m->lv, Pp, src, NVARS, s);
        if (!st) st = plan_rhs(p, s, nullptr, nullptr);
        if (!st)
            st = launch_levels_stage(*m->lv, stage, Ip, Ap, u, (const double* const*)Rp, dt, enf, p->prm.chi_floor,
                                     p->status, s);
        if (!st) st = launch_levels_sync(*m->lv, stage < 3 ? Ip : u, NVARS, s);
        return st;
    }
    if (p->direct || plan_zipped_rhs(p)) {
        double* Rz[NVARS];
        set_ptrs(p->Rz, p->n_nodes, Rz);
        // ghost fill of the blocks staged from padded blocks only
        int st = p->direct ? 0 : launch_unzip(m, Pp, src, NVARS, s, true);
        if (!st) st = plan_rhs(p, s, nullptr, src);
        if (!st) st = launch_node_stage(stage, Ip, Ap, u, Rz, p->n_nodes, dt, enf, p->prm.chi_floor,
                                        p->status, s);
        return st;
    }
    int st = launch_unzip(m, Pp, src, NVARS, s);
    if (!st) st = plan_rhs(p, s, nullptr, nullptr);
    if (!st) st = launch_zip_stage(m, stage, Ip, Ap, u, Rp, dt, enf, p->prm.chi_floor, p->status, s);
    return st;
}

int plan_enqueue(Plan* p, double* const* u, double dt, cudaStream_t s) {
    for (int stage = 0; stage < 4; stage++) {
        const int st = plan_enqueue_stage(p, u, dt, stage, s);
        if (st) return st;
    }
    return 0;
}

// Captures body(stream) into *graph / *exec on the plan's own capture
// stream (the caller's stream may be the legacy default stream, which cannot
// be captured; the graph is then launched onto the caller's stream, which
// orders it after prior work).
template <class F>
static int capture(Plan* p, cudaGraph_t* graph, cudaGraphExec_t* exec, F body) {
    if (*exec) cudaGraphExecDestroy(*exec);
    if (*graph) cudaGraphDestroy(*graph);
    *exec = nullptr;
    *graph = nullptr;
    if (!p->cap_stream && cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return BSSN_ENOMEM;
    }
    cudaError_t e = cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGetLastError();  // do not leave the failure for a later launch check
        return cuda_status(e);
    }
    int st = body(p->cap_stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(p->cap_stream, &g);
    if (st || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return st ? st : cuda_status(e);
    }
    *graph = g;
    e = cudaGraphInstantiate(exec, g, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_status(e);
    }
    return 0;
}

int plan_step(Plan* p, double* const* u, double dt, cudaStream_t s) {
    if (!(p->flags & BSSN_PLAN_GRAPH)) return plan_enqueue(p, u, dt, s);
    bool same = p->exec && p->graph_dt == dt;
    for (int v = 0; v < NVARS && same; v++) same = p->graph_u[v] == u[v];
    if (!same) {
        int st = capture(p, &p->graph, &p->exec, [&](cudaStream_t cs) { return plan_enqueue(p, u, dt, cs); });
        if (st) return st;
        for (int v = 0; v < NVARS; v++) p->graph_u[v] = u[v];
        p->graph_dt = dt;
    }
    return cuda_status(cudaGraphLaunch(p->exec, s));
}

// Constraint diagnostics of the zipped state u: ghost fill of every block
// into the padded stage array, Hamiltonian and momentum constraints into the
// plan's zipped constraint arrays, their masked L2 norms into d.norms.  The
// reference's time loop computes the same norms every BSSN_IO_OUTPUT_FREQ
// steps (BSSN_GR/src/bssnCtx.cpp:597-685, computeConstraintL2Norm).
static int diag_prepare(Plan* p) {
    // needs the padded stage array and a single-level node grid
    if (p->direct || !p->P || p->mesh->lv) return BSSN_ESTATE;
    MeshState* m = p->mesh;
    const size_t nf = (p->flags & BSSN_PLAN_DIAG_PSI4) ? 6 : 4;  // ham, mom0..2 (, psi4 re, im)
    if (!p->cons && alloc(&p->cons, nf * p->n_nodes)) return BSSN_ENOMEM;
    if (!m->d_partial &&
        cudaMalloc((void**)&m->d_partial, sizeof(double) * 5 * kNormPartials) != cudaSuccess) {
        cudaGetLastError();
        return BSSN_ENOMEM;
    }
    return 0;
}

static int enqueue_diag(Plan* p, double* const* u, const DiagArgs& d, cudaStream_t s) {
    MeshState* m = p->mesh;
    double* Pp[NVARS];
    set_ptrs(p->P, m->unzip_size, Pp);
    int st = unzip_all(m, Pp, (const double* const*)u, s);
    if (st) return st;
    const bool psi4 = (p->flags & BSSN_PLAN_DIAG_PSI4) != 0;
    double* cons[6];
    for (int c = 0; c < (psi4 ? 6 : 4); c++) cons[c] = p->cons + (size_t)c * p->n_nodes;
    st = launch_constraints(m, (const double* const*)Pp, cons, s, psi4);
    if (st) return st;
    return launch_l2_norms(m, (const double* const*)cons, 4, d.xmin, d.h, d.bh, d.radii, m->d_partial,
                           kNormPartials, d.norms, s);
}

int plan_diag(Plan* p, double* const* u, const DiagArgs& d, cudaStream_t s) {
    const int st = diag_prepare(p);
    return st ? st : enqueue_diag(p, u, d, s);
}

// One RK4 step followed by the diagnostics of the new state, captured as one
// graph (a second one beside the plain step's) when the plan has
// BSSN_PLAN_GRAPH, so a time loop that reports the norms every k steps
// replays graphs only and never synchronises with the host.
int plan_step_diag(Plan* p, double* const* u, double dt, const DiagArgs& d, cudaStream_t s) {
    int st = diag_prepare(p);
    if (st) return st;
    auto body = [&](cudaStream_t cs) {
        int r = plan_enqueue(p, u, dt, cs);
        return r ? r : enqueue_diag(p, u, d, cs);
    };
    if (!(p->flags & BSSN_PLAN_GRAPH)) return body(s);
    double key[14] = {dt, d.xmin[0], d.xmin[1], d.xmin[2], d.h, d.bh[0], d.bh[1], d.bh[2],
                      d.bh[3], d.bh[4], d.bh[5], d.radii[0], d.radii[1], 0.0};
    std::memcpy(&key[13], &d.norms, sizeof(double*));
    bool same = p->exec_diag && std::memcmp(key, p->diag_key, sizeof key) == 0;
    for (int v = 0; v < NVARS && same; v++) same = p->diag_u[v] == u[v];
    if (!same) {
        st = capture(p, &p->graph_diag, &p->exec_diag, body);
        if (st) return st;
        for (int v = 0; v < NVARS; v++) p->diag_u[v] = u[v];
        std::memcpy(p->diag_key, key, sizeof key);
    }
    return cuda_status(cudaGraphLaunch(p->exec_diag, s));
}

// Project-written autotuner: for every block-size bucket of the mesh, time
// the fused right-hand side of that bucket with every compiled tile shape on
// the current padded state (CUDA events, best of `reps` after one warm-up)
// and keep the fastest.  Blocking.
int plan_autotune(Plan* p, double* const* u, int reps, cudaStream_t s, float* times_out) {
    MeshState* m = p->mesh;
    RhsArgs A;
    A.prm = p->prm;
    int st = 0;
    if (p->direct) {  // split tiles on the zipped state u
        double* Rz[NVARS];
        set_ptrs(p->Rz, p->n_nodes, Rz);
        for (int v = 0; v < NVARS; v++) {
            A.u.p[v] = u[v];
            A.rhs.p[v] = Rz[v];
        }
    } else {
        double* Pp[NVARS];
        set_ptrs(p->P, m->unzip_size, Pp);
        st = unzip_all(m, Pp, (const double* const*)u, s);
        if (st) return st;
        double* Rp[NVARS];
        set_ptrs(p->R, m->unzip_size, Rp);
        for (int v = 0; v < NVARS; v++) {
            A.u.p[v] = Pp[v];
            A.rhs.p[v] = Rp[v];
        }
    }
    const int32_t* zg = p->direct ? m->G : nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int nt = tile_count();
    if (p->direct) {
        // every split tile over the whole Z-ordered list; each bucket row of
        // `times` gets the same figures
        float best = 1e30f;
        int best_t = default_split_tile();
        std::vector<float> tt(nt, 1e30f);
        for (int t = 0; t < nt && !st; t++) {
            if (!tile_zipped(tile_mode(t))) continue;
            const BrickTask* tk;
            int ntask;
            st = mesh_tasks_side(m, t, kAllZOrder, &tk, &ntask);
            for (int r = 0; r <= reps && !st; r++) {
                cudaEventRecord(e0, s);
                st = launch_rhs_tasks(t, A, m->d_blocks, tk, ntask, s, m->d_scratch,
                                      m->scratch_zones, nullptr, zg);
                cudaEventRecord(e1, s);
                if (st) break;
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (r > 0) tt[t] = std::min(tt[t], ms);
            }
            if (!st && tt[t] < best) {
                best = tt[t];
                best_t = t;
            }
        }
        if (!st) m->tuned[kAllZOrder] = best_t;
        if (times_out)
            for (size_t i = 0; i < p->sides.size(); i++)
                for (int t = 0; t < nt; t++) times_out[i * nt + t] = tt[t];
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        drop_graphs(p);  // tile choice changed: recapture on the next step
        return st;
    }
    int idx = 0;
    for (int side : p->sides) {
        float best = 1e30f;
        int best_t = 0;
        for (int t = 0; t < nt; t++) {
            float tbest = 1e30f;
            const BrickTask* tk;
            int ntask;
            st = mesh_tasks_side(m, t, side, &tk, &ntask);
            if (st) break;
            for (int r = 0; r <= reps; r++) {
                cudaEventRecord(e0, s);
                st = launch_rhs_tasks(t, A, m->d_blocks, tk, ntask, s, m->d_scratch, m->scratch_zones);
                cudaEventRecord(e1, s);
                if (st) break;
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (r > 0) tbest = std::min(tbest, ms);
            }
            if (st) break;
            if (times_out) times_out[idx * nt + t] = tbest;
            if (tbest < best) {
                best = tbest;
                best_t = t;
            }
        }
        if (st) break;
        m->tuned[side] = best_t;
        idx++;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs(p);  // tile choice changed: recapture on the next step
    return st;
}

// Average duration of one full fused-RHS pass (all buckets) on the plan's
// current padded state, CUDA events on `s` around `reps` back-to-back passes
// after one warm-up pass.  Blocking.
// The stage state the timing functions run the right-hand side on: the
// padded P of the last ghost fill, or (direct) the zipped intermediate state.
const double* const* timing_src(Plan* p, double* buf[NVARS]) {
    if (!p->direct && !plan_zipped_rhs(p)) return nullptr;
    set_ptrs(p->im, p->n_nodes, buf);
    return (const double* const*)buf;
}

int plan_time_rhs(Plan* p, int reps, cudaStream_t s, float* ms) {
    double* buf[NVARS];
    const double* const* src = timing_src(p, buf);
    int st = plan_rhs(p, s, nullptr, src);
    if (st) return st;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && !st; r++) st = plan_rhs(p, s, nullptr, src);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st ? st : cuda_status(cudaGetLastError());
}

// Per-kernel timing of the right-hand-side pass: `reps` passes after one
// warm-up, CUDA events around every launch; out[k] = milliseconds per pass
// spent in kernels of kind k (fused, derivative, equation), out[3 + k] =
// launches of kind k per pass.  Blocking.
int plan_time_kernels(Plan* p, int reps, cudaStream_t s, double out[6]) {
    double* buf[NVARS];
    const double* const* src = timing_src(p, buf);
    int st = plan_rhs(p, s, nullptr, src);
    if (st) return st;
    double ms[KernelTimer::NKIND] = {0, 0, 0};
    int n[KernelTimer::NKIND] = {0, 0, 0};
    for (int r = 0; r < reps && !st; r++) {
        KernelTimer tm;
        st = plan_rhs(p, s, &tm, src);
        const int st2 = tm.collect(ms, n);
        if (!st) st = st2;
    }
    for (int k = 0; k < KernelTimer::NKIND; k++) {
        out[k] = reps > 0 ? ms[k] / reps : 0.0;
        out[3 + k] = reps > 0 ? (double)n[k] / reps : 0.0;
    }
    return st ? st : cuda_status(cudaGetLastError());
}

// Kernel launches of one RK4 step: per stage the ghost fill, the
// right-hand-side launches of every bucket, and the zip-stage kernel.
int plan_launches_per_step(Plan* p) {
    MeshState* m = p->mesh;
    int rhs = 0;
    if (p->flags & BSSN_PLAN_PER_BLOCK) {
        for (auto& b : m->blocks) rhs += tile_mode(plan_tile(p, b.sz)) == 1 ? 2 : 1;
    } else if (p->direct) {
        const int t = plan_tile(p, kAllZOrder);
        const BrickTask* tk;
        int nt = 0;
        if (mesh_tasks_side(m, t, kAllZOrder, &tk, &nt)) return -1;
        rhs = rhs_launch_count(t, nt, m->scratch_zones);
    } else {
        for (int side : p->sides) {
            const int t = plan_tile(p, side);
            const BrickTask* tk;
            int nt = 0;
            if (mesh_tasks_side(m, t, side, &tk, &nt)) return -1;
            rhs += rhs_launch_count(t, nt, m->scratch_zones);
        }
    }
    if (m->lv) {  // interpolation passes, ghost fill, stage, one launch per non-empty sync segment
        int extra = 2;
        for (int k = 0; k < 3; k++) extra += m->lv->n_task[k] > 0 ? 1 : 0;
        for (const auto* f : {&m->lv->inject_first, &m->lv->prolong_first})
            for (size_t k = 0; k + 1 < f->size(); k++) extra += (*f)[k + 1] > (*f)[k] ? 1 : 0;
        return 4 * (rhs + extra);
    }
    return 4 * (rhs + (p->direct ? 1 : 2));
}

namespace {
// FP64 multiply-add throughput probe: 8 independent chains per thread.
__global__ void __launch_bounds__(256) fp64_probe_kernel(double* out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = threadIdx.x * 1e-3 + q;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int q = 0; q < 8; q++) x[q] = fma(x[q], a, b);
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) s += x[q];
    if (s == 12345.678) out[0] = s;  // keeps the chains alive
}
}  // namespace

int fp64_probe(double* scratch, int iters, cudaStream_t s, double* tflops) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256;
    fp64_probe_kernel<<<blocks, threads, 0, s>>>(scratch, 16, 0.999999, 1e-7);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    fp64_probe_kernel<<<blocks, threads, 0, s>>>(scratch, iters, 0.999999, 1e-7);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return cuda_status(cudaGetLastError());
}

}  // namespace bssn
