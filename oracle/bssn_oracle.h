/* Test infrastructure only: the CPU oracle.  Nothing in the product library
 * links, includes or calls this code; only tests/, the smoke check in
 * __graft_entry__.py and bench.py's CPU-baseline leg load liboracle.so, and
 * only as the checker.
 *
 * A plain CPU restatement of the reference's BSSN evolution hot path.  Each
 * function cites the reference file:line it follows.  It is pinned against
 * the reference's own compiled arithmetic (oracle/_ref/libbssn_ref.so, built
 * from the reference sources in place) by tests/test_oracle_pin.py and by the
 * committed fixtures under tests/golden/.
 *
 * Layout conventions (same as the reference):
 *   variable order   alpha, chi, K, Gt0..2, beta0..2, B0..2, gt0..5, At0..5
 *                    (BSSN_GR/include/grDef.h:35-60)
 *   block arrays     u[v][offset + i + nx*(j + ny*k)], padding width 3
 *   bflag bits       x-min, x-max, y-min, y-max, z-min, z-max = bits 0..5
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcParams {
    double ko_sigma;        /* KO_DISS_SIGMA */
    unsigned lambda[4];     /* BSSN_LAMBDA */
    double lambda_f[2];     /* BSSN_LAMBDA_F */
    double eta_central;     /* RIT_ETA_CENTRAL */
    double eta_outer;       /* RIT_ETA_OUTER */
    double eta_width;       /* RIT_ETA_WIDTH */
    int cako_enabled;       /* BSSN_CAKO_ENABLED */
    double eps_cako_gauge;  /* BSSN_EPSILON_CAKO_GAUGE */
    double eps_cako_other;  /* BSSN_EPSILON_CAKO_OTHER */
} OrcParams;

/* One block of a single-level octree mesh: an aligned cube of octants whose
 * interior holds s-6 = 6*2^k+1 nodes per side. */
typedef struct OrcBlock {
    int64_t offset;   /* start of the padded s^3 array in the unzipped vector */
    int32_t sz;       /* padded side s */
    uint32_t bflag;   /* physical-boundary faces */
    int32_t g0[3];    /* global node index of the first interior node */
    int32_t level;
    double ptmin[3];  /* coordinate of padded point (0,0,0) */
    double ptmax[3];  /* coordinate of padded point (s-1,s-1,s-1) */
} OrcBlock;

/* --- stencils (BSSN_GR/src/derivs.cpp) -------------------------------- */
void orc_deriv644_x(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_deriv644_y(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_deriv644_z(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_deriv644_xx(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_deriv644_yy(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_deriv644_zz(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_ko_deriv42_x(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_ko_deriv42_y(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);
void orc_ko_deriv42_z(double* D, const double* u, double h, const unsigned* sz, unsigned bflag);

/* --- per-block RHS (BSSN_GR/src/rhs.cpp:80-504) ------------------------ */
/* ws: NULL (allocated internally) or 288*n doubles, n = sz[0]*sz[1]*sz[2]. */
void orc_bssnrhs(double** rhs, const double** u, unsigned offset,
                 const double* pmin, const double* pmax, const unsigned* sz,
                 unsigned bflag, const OrcParams* prm, double* ws);
/* Block loop (BSSN_GR/src/rhs.cpp:10-73) with an OpenMP loop over blocks and
 * one workspace per thread (BSSN_GR/cuda/include/test_utils.h:52-180). */
void orc_bssnRHS(double** rhs, const double** u, const OrcBlock* blks,
                 int nblk, const OrcParams* prm, int nthreads);

/* --- constraint enforcement (BSSN_GR/include/bssn_constraints.h:15-172)
 * Returns the number of nodes that violated det(gt)>0, |det-1|<=1e-6 or
 * |tr A|<=1e-6 (the reference exits on the first one). */
int64_t orc_enforce(double** u, int64_t n, double chi_floor);

/* --- Brill-Lindquist puncture data (BSSN_GR/src/grUtils.cpp:864-1178 with
 * zero momenta and spins), plus a seeded uniform perturbation of amplitude
 * eps on every variable, followed by enforcement.  Fills zipped nodes of a
 * G[0] x G[1] x G[2] node grid with coordinates xmin + g*h. */
void orc_initial_data(double** u, const int32_t* G, const double* xmin,
                      double h, const double* bh, double m1, double m2,
                      double chi_floor, double eps, uint64_t seed);

/* --- ghost fill (absent dendrolib ot::Mesh::unzip / zip; parity with Dendro
 * itself unpinned).  Zipped vector = every node of the G[0]xG[1]xG[2] grid.
 * unzip: every padded point whose node lies inside the grid gets that node's
 * value; points outside the grid get 0.  zip: each node takes its value from
 * the block containing octant floor(g/6) (clamped), found by searching the
 * block list. */
void orc_unzip(double** unzip, const double** zip, const OrcBlock* blks,
               int nblk, const int32_t* G, int nvars);
void orc_zip(double** zip, const double** unzip, const OrcBlock* blks,
             int nblk, const int32_t* G, int nvars);
/* The source node index of every padded point (or -1), per block, as a flat
 * int64 array in unzipped order: the ghost-fill index map. */
void orc_unzip_map(int64_t* map, const OrcBlock* blks, int nblk,
                   const int32_t* G);

/* --- one classical RK4 step on the zipped state (BSSN_GR/src/rkBSSN.cpp:
 * 764-860, coefficients BSSN_GR/include/rkBSSN.h:50-53).  enforce_stages
 * enforces constraints on every intermediate stage state as rkBSSN does;
 * the final state is always enforced.  Returns total enforcement
 * violations. */
int64_t orc_rk4_step(double** u, const OrcBlock* blks, int nblk,
                     const int32_t* G, int64_t n_unzip, double dt,
                     const OrcParams* prm, double chi_floor,
                     int enforce_stages, int nthreads);
/* The same step with a caller-provided workspace of orc_rk4_ws_doubles()
 * doubles and the block-loop right-hand side as a parameter: orc_bssnRHS
 * (NULL) or any function of the same form -- the reference's own compiled
 * block loop (ref_bssnRHS_blocks in oracle/_ref, same block and parameter
 * layouts) turns this into the reference CPU RK4 step. */
typedef void (*orc_rhs_fn)(double** rhs, const double** u, const OrcBlock* blks, int nblk,
                           const OrcParams* prm, int nthreads);
int64_t orc_rk4_ws_doubles(const int32_t* G, int64_t n_unzip);
int64_t orc_rk4_step_ws(double** u, const OrcBlock* blks, int nblk, const int32_t* G,
                        int64_t n_unzip, double dt, const OrcParams* prm, double chi_floor,
                        int enforce_stages, int nthreads, orc_rhs_fn rhs, double* ws);

/* The same step without unzipped arrays (ghost fill and right-hand side per
 * block in per-thread buffers; acc, kbuf, im: caller arrays of N per
 * variable): identical arithmetic, for meshes whose unzipped copies do not
 * fit in host memory. */
int64_t orc_rk4_step_lowmem(double** u, const OrcBlock* blks, int nblk, const int32_t* G,
                            double dt, const OrcParams* prm, double chi_floor, int enforce_stages,
                            int nthreads, orc_rhs_fn rhs, double** acc, double** kbuf, double** im);

/* Constraint L2 sums (ham, mom0..2, count) over nodes outside both radii,
 * block by block without unzipped arrays; norm = sqrt(sums[c] / sums[4]). */
void orc_constraint_sums_lowmem(const double** u, const OrcBlock* blks, int nblk, const int32_t* G,
                                const double* xmin, double h, const double* bh,
                                const double* radii, double* sums, int nthreads);

/* --- the workloads' synthetic single-level octree meshes (block lists; see
 * bssn_oracle.cpp).  blks NULL: only *nblk, G and *h are set.  0 = ok. */
int orc_mesh_generate(int mode, const int32_t* dims, const double* p, uint64_t seed,
                      double xmin, double L, OrcBlock* blks, int* nblk, int32_t* G,
                      double* h);

/* --- Hamiltonian and momentum constraints (BSSN_GR/src/physcon.cpp:12-89,
 * equations from CodeGen/constraints.py) on a block's interior, and the
 * masked L2 norm of a zipped field (BSSN_GR/include/grUtils.tcc:36-134). */
void orc_physical_constraints(double** cons, const double** u, unsigned offset,
                              const double* pmin, const double* pmax,
                              const unsigned* sz, unsigned bflag, double* ws);
/* --- The Weyl scalar psi4 (CodeGen/constraints.py:45-244) on a block's
 * interior: re / im arrays indexed like u (offset + point). */
void orc_psi4(double* re, double* im, const double** u, unsigned offset, const double* pmin,
              const double* pmax, const unsigned* sz, unsigned bflag, double* ws);


/* --- remesh (the absent dendrolib wavelet transform behind isReMeshWAMR,
 * BSSN_GR/src/dataUtils.cpp:511-624; parity with Dendro unpinned).
 * Element = one octant of a block (7^3 nodes), its 13^3 patch = the element
 * plus 3 halo nodes.  Interpolating-wavelet coefficient at every element
 * node with an odd local index along some axis: the value minus its
 * degree-5 Lagrange interpolation from the coarse (even local index) nodes
 * at patch positions {1,3,5,7,9,11} along each odd axis.  Score of an
 * (element, variable) = sqrt(sum w^2 / 279), summed in the canonical order:
 * node q (z, y, x ascending over the 279 wavelet nodes) goes to partial
 * q mod 32, partials added in ascending order.  scores: one per element per
 * variable, elements numbered block by block, octant x fastest. */
void orc_wavelet_scores(const double** unzip, const OrcBlock* blks, int nblk,
                        int nvars, double* scores);
/* Per-element remesh features (16 floats per element, see bssn_b200.h). */
void orc_element_features(const double** unzip, const OrcBlock* blks, int nblk, float* feats);
/* Per-block remesh features (16 floats per block, see bssn_b200.h). */
void orc_block_features(const double** unzip, const OrcBlock* blks, int nblk,
                        float* feats);

#ifdef __cplusplus
}
#endif
