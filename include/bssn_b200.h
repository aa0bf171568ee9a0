/* bssn_b200.h -- C ABI of the B200-native BSSN evolution hot path.
 *
 * Plain pointers and sizes only.  Every array argument named *_dev is device
 * memory; the caller owns all of it.  Variable arrays follow the reference's
 * structure-of-arrays layout: an array of 24 per-variable base pointers
 * indexed u[v][offset + i + nx*(j + ny*k)], variable order
 *   alpha, chi, K, Gt0..2, beta0..2, B0..2, gt0..5, At0..5
 * (BSSN_GR/include/grDef.h:35-60).  Blocks are padded cubes of side
 * s in {13, 19, 31, 55} with a 3-point halo; only interior points
 * [3, s-3)^3 of a right-hand side are written.
 *
 * Boundary flag bits: x-min, x-max, y-min, y-max, z-min, z-max = bits 0..5
 * (the reference's 1u << OCT_DIR_{LEFT,RIGHT,DOWN,UP,BACK,FRONT}).
 *
 * Return codes: 0 success; > 0 invalid argument (BSSN_E*); < 0 a CUDA error
 * (the negated cudaError_t).  No entry point traps, asserts or exits.  All
 * calls are asynchronous on the given stream unless stated otherwise, and a
 * handle may be used from one stream at a time.
 */
#ifndef BSSN_B200_H
#define BSSN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* bssn_stream_t; /* == cudaStream_t */

#define BSSN_OK 0
#define BSSN_EINVAL 1       /* null pointer or bad size */
#define BSSN_EBLOCKSIZE 2   /* block side not in {13,19,31,55} or not cubic */
#define BSSN_EKIND 3        /* unknown stencil kind */
#define BSSN_ENOMEM 4       /* device allocation failed */
#define BSSN_ESTATE 5       /* handle used out of order */
#define BSSN_ELIMIT 6       /* size exceeds a documented fixed maximum */

#define BSSN_NUM_VARS 24

/* Hot-path parameters the reference reads from bssn:: globals
 * (BSSN_GR/src/parameters.cpp:14-16,40-43,123-136). */
typedef struct BssnParams {
    double ko_sigma;        /* KO_DISS_SIGMA */
    unsigned lambda[4];     /* BSSN_LAMBDA */
    double lambda_f[2];     /* BSSN_LAMBDA_F */
    double eta_central;     /* RIT_ETA_CENTRAL */
    double eta_outer;       /* RIT_ETA_OUTER */
    double eta_width;       /* RIT_ETA_WIDTH */
    int cako_enabled;       /* BSSN_CAKO_ENABLED */
    double eps_cako_gauge;  /* BSSN_EPSILON_CAKO_GAUGE */
    double eps_cako_other;  /* BSSN_EPSILON_CAKO_OTHER */
    double chi_floor;       /* CHI_FLOOR */
} BssnParams;

/* One block (the reference's ot::Block as read by bssnRHS, rhs.cpp:50-67 and
 * BlockGPU3D, bssn_kernels.cuh:1352-1357).  ptmin/ptmax are the coordinates
 * of padded points (0,0,0) and (s-1,s-1,s-1); the grid spacing is
 * (ptmax-ptmin)/(s-1) per axis exactly as the reference computes it.
 * g0 is the global node index of the block's first interior node in the
 * zipped node grid (used by unzip/zip only). */
typedef struct BssnBlockDesc {
    int64_t offset;
    int32_t sz;
    uint32_t bflag;
    int32_t g0[3];
    int32_t level;
    double ptmin[3];
    double ptmax[3];
} BssnBlockDesc;

/* ---------------------------------------------------------------------- */
/* Stand-alone stencils on one padded block, bit-identical to the reference
 * (same expression order, no contraction).
 * kind: 0 deriv644_x, 1 _y, 2 _z, 3 _xx, 4 _yy, 5 _zz,
 *       6 ko_deriv42_x, 7 _y, 8 _z.
 * Replaces deriv644_{x,y,z,xx,yy,zz} (BSSN_GR/src/derivs.cpp:2619-3312,
 * include/derivs.h:76-130) and ko_deriv42_{x,y,z} (derivs.cpp:964-1305).
 * Writes exactly the points the reference writes. */
int bssn_deriv644_f64(int kind, double* D_dev, const double* u_dev, double h,
                      const unsigned sz[3], unsigned bflag,
                      bssn_stream_t stream);
/* deriv644adv_{x,y,z}(..., beta, ...) (derivs.cpp:3313-3347): the reference
 * hard-wires them to the centred stencil; beta_dev is accepted and unused. */
int bssn_deriv644adv_f64(int dir, double* D_dev, const double* u_dev, double h,
                         const unsigned sz[3], const double* beta_dev,
                         unsigned bflag, bssn_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Fused right-hand side of one block: derivatives, pointwise BSSN
 * equations, Sommerfeld boundary conditions and Kreiss-Oliger dissipation in
 * one kernel; derivatives never leave the chip.
 * Replaces bssnrhs(unzipVarsRHS, uZipVars, offset, pmin, pmax, sz, bflag,
 * t, uZipConstVars) (BSSN_GR/src/rhs.cpp:80-504, include/rhs.h:32-36); t and
 * the constraint arrays are unused by the standard-gauge equations. */
int bssn_bssnrhs_f64(double* const* rhs_dev, const double* const* u_dev,
                     int64_t offset, const double pmin[3],
                     const double pmax[3], const unsigned sz[3],
                     unsigned bflag, const BssnParams* params,
                     bssn_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Mesh handle: a device copy of a block list plus the zipped node grid
 * dims G (the zipped vector of each variable holds G[0]*G[1]*G[2] nodes,
 * node index gx + G[0]*(gy + G[1]*gz)).  Created once per mesh; blocking. */
typedef struct bssn_mesh_s* bssn_mesh;
int bssn_mesh_create(const BssnBlockDesc* blocks, int nblocks,
                     const int32_t G[3], bssn_mesh* out);
int bssn_mesh_destroy(bssn_mesh mesh);
/* total padded points (sum of s^3 rounded per block to the layout's
 * offsets) = one past the largest offset + s^3 */
int64_t bssn_mesh_unzip_size(bssn_mesh mesh);

/* All blocks of a mesh in one launch.  Replaces bssnRHS(unzipVarsRHS,
 * uZipVars, blkList, numBlocks, t, uZipConstVars) (rhs.cpp:10-73) and the
 * GPU comparator device::bssnrhs3 (cuda/include/bssn_kernels.cuh:1526-1538).
 * tile: -1 = the split 7x7x7 tile; otherwise a tile id in
 * [0, bssn_tile_count()). */
int bssn_rhs_blocks_f64(bssn_mesh mesh, double* const* rhs_dev,
                        const double* const* u_dev, const BssnParams* params,
                        int tile, bssn_stream_t stream);

/* Ghost fill: zipped node vectors -> padded block arrays (interior and
 * halo).  Padded points whose node lies outside the node grid get 0.
 * Replaces ot::Mesh::unzip (dendrolib, absent; call sites
 * BSSN_GR/src/rkBSSN.cpp:611-650, bssnCtx.cpp:73). */
int bssn_unzip_f64(bssn_mesh mesh, double* const* unzip_dev,
                   const double* const* zip_dev, int nvars,
                   bssn_stream_t stream);
/* Padded block interiors -> zipped nodes; each node is written by exactly
 * one block (the one containing octant floor(g/6), clamped to the grid).
 * Replaces ot::Mesh::zip (dendrolib; rkBSSN.cpp:633,647, bssnCtx.cpp:103). */
int bssn_zip_f64(bssn_mesh mesh, double* const* zip_dev,
                 const double* const* unzip_dev, int nvars,
                 bssn_stream_t stream);

/* ---------------------------------------------------------------------- */
/* RK4 stage updates on zipped vectors of n nodes (rkBSSN.cpp:764-860,
 * coefficients rkBSSN.h:50-53).
 *   stage in 0..2:  u_im = u_prev + RK4_U[stage+1]*dt*k   (then optionally
 *                   enforce constraints on u_im)
 *   stage 3:        u = u_prev + sum_s RK4_C[s]*dt*k_s, k_s given as 4
 *                   arrays of 24 pointers (k_dev[s*24 + v]); then enforce.
 * enforce: 1 = apply enforce_bssn_constraints to every written node.
 * status_dev (optional, may be NULL): an int the kernel atomically adds the
 * number of nodes that violated det(gt)>0 / |det-1|<=1e-6 / |trA|<=1e-6
 * (the reference exits at the first one; this library counts and goes on). */
int bssn_rk4_stage_f64(int stage, double* const* out_dev,
                       const double* const* u_prev_dev,
                       const double* const* k_dev, int64_t n, double dt,
                       int enforce, double chi_floor, int* status_dev,
                       bssn_stream_t stream);

/* enforce_bssn_constraints on n zipped nodes in place
 * (BSSN_GR/include/bssn_constraints.h:15-172); violations counted as above. */
int bssn_enforce_f64(double* const* u_dev, int64_t n, double chi_floor,
                     int* status_dev, bssn_stream_t stream);

/* Brill-Lindquist puncture data (BSSN_GR/src/grUtils.cpp:864-1178 with zero
 * momenta and spins) on the G[0]xG[1]xG[2] node grid with coordinates
 * xmin + g*h, plus a seeded uniform perturbation of amplitude eps on every
 * variable (counter-based: node and variable index hashed with the seed),
 * then enforcement.  bh = {x1,y1,z1,x2,y2,z2}. */
int bssn_initial_data_f64(double* const* u_dev, const int32_t G[3],
                          const double xmin[3], double h, const double bh[6],
                          double m1, double m2, double chi_floor, double eps,
                          uint64_t seed, bssn_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Hamiltonian and momentum constraints (CodeGen/constraints.py:250-283,
 * per block as physical_constraints, BSSN_GR/src/physcon.cpp:12-89) from
 * the padded stage state of every block, written to the zipped node arrays
 * cons_dev[0..3] = ham, mom0, mom1, mom2 (owned nodes only).  On a
 * multi-level mesh every zipped node (the level grids back to back) takes
 * the value at the zone that owns it; nodes filled from another level
 * (patch-boundary nodes, coarse nodes under a finer patch) are set to 0, so
 * each physical point carries its value once. */
int bssn_constraints_f64(bssn_mesh mesh, const double* const* unzip_dev,
                         double* const* cons_dev, bssn_stream_t stream);
/* The same constraints plus the Weyl scalar psi4 for gravitational-wave
 * extraction (the psi4_real / psi4_img outputs of physical_constraints,
 * BSSN_GR/src/physcon.cpp:12-89; definition CodeGen/constraints.py:45-244):
 * cons_dev[0..5] = ham, mom0, mom1, mom2, psi4 real, psi4 imaginary (owned
 * nodes; psi4 = 0 on the z axis, |x|, |y| <= 1e-7, as the reference sets
 * it). */
int bssn_constraints_psi4_f64(bssn_mesh mesh, const double* const* unzip_dev,
                              double* const* cons_dev, bssn_stream_t stream);
/* Gravitational-wave extraction from psi4 (extractFarFieldPsi4,
 * BSSN_GR/include/gwExtract.h:48-190): psi4 on spheres of the given radii
 * about the origin, interpolated from a single-level node grid (G nodes per
 * axis, node (i,j,k) at xmin + (i,j,k) h) with the degree-6 Lagrange
 * polynomial over the 7^3 nodes of the enclosing octant, and decomposed
 * into the spin-weight -2 harmonics of every (l, m), l = 2..lmax, m = -l..l
 * (Goldberg et al. 1967 convention: -2Y_22 = sqrt(5/pi)/8 (1+cos th)^2
 * e^{2i ph}):
 *   coeff_dev[(r * nmodes + k) * 2 + {0,1}] = 4 pi sum_p w_p psi4(p)
 *                                             conj(-2Y_lm(p)),  k in (l, m) order
 *   l2_dev[r * 2 + {0,1}] = sum_p (Re psi4)^2, sum_p (Im psi4)^2
 * over n_theta Gauss-Legendre nodes in cos(theta) x 2 n_theta uniform phi
 * (weights sum to 4 pi; the reference integrates with a Lebedev rule).
 * Points outside the grid are skipped, as the reference skips points
 * outside its mesh.  nmodes = bssn_gw_modes_count(lmax).  Allocates and
 * frees device memory for its tables; blocking. */
int bssn_gw_modes_count(int lmax);
int bssn_gw_extract_f64(const double* psi4_re_dev, const double* psi4_im_dev, const int32_t G[3],
                        const double xmin[3], double h, int nradii, const double* radii, int lmax,
                        int ntheta, double* coeff_dev, double* l2_dev, bssn_stream_t stream);
/* The quadrature and harmonics the extraction uses (host only, for tests):
 * per point theta, phi, weight; y = -2Y_lm per mode and point as (re, im)
 * pairs, mode-major.  Any output may be NULL. */
int bssn_gw_sphere_tables(int lmax, int ntheta, double* theta, double* phi, double* w, double* y);
/* Masked L2 norms sqrt(sum c^2 / N) over the zipped nodes farther than
 * radii[0] / radii[1] from the punctures bh = {x1,y1,z1,x2,y2,z2}
 * (computeConstraintL2Norm, BSSN_GR/include/grUtils.tcc:36-134); node
 * coordinates xmin + g*h.  Writes ncons (<= 4) doubles to norms_dev.  The
 * reduction's partial sums live in a buffer the mesh handle allocates on
 * the first call. */
int bssn_constraint_norms_f64(bssn_mesh mesh, const double* const* cons_dev,
                              int ncons, const double xmin[3], double h,
                              const double bh[6], const double radii[2],
                              double* norms_dev, bssn_stream_t stream);
/* The pieces of those norms for a reduction over the ranks of a partition
 * (the reference's par::Mpi_Reduce of the local sums,
 * BSSN_GR/include/grUtils.tcc:31): sums_dev[c] = sum of cons_c^2 over the
 * counted nodes (c < ncons), sums_dev[4] = their number; counted are the
 * nodes outside both radii with mask_dev[node] != 0 (mask_dev NULL: every
 * node).  Same fixed reduction order as bssn_constraint_norms_f64.  After
 * summing sums_dev over the ranks, norm_c = sqrt(sum_c / count). */
int bssn_constraint_sums_f64(bssn_mesh mesh, const double* const* cons_dev,
                             int ncons, const double xmin[3], double h,
                             const double bh[6], const double radii[2],
                             const uint8_t* mask_dev, double* sums_dev,
                             bssn_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Remesh decision.  The reference scores each element with dendrolib's
 * wavelet transform inside isReMeshWAMR (BSSN_GR/src/dataUtils.cpp:511-624;
 * the transform is absent from the reference tree, so this library defines
 * it: for every node of an element (octant, 7^3 nodes) with an odd local
 * index on some axis, w = u - degree-5 Lagrange interpolation from the
 * element patch's coarse nodes at positions 1,3,5,7,9,11 along each odd
 * axis; score = sqrt(sum w^2 / 279); an element asks for refinement when
 * the score of any variable exceeds tol).  Elements are numbered block by
 * block, octant x fastest. */
int64_t bssn_mesh_num_elements(bssn_mesh mesh);
/* Exact test: scores_dev (num_elements x nvars doubles) always; optionally
 * per-block max score / tol (ratio_dev) and refine flags (flags_dev). */
int bssn_remesh_wavelet_f64(bssn_mesh mesh, const double* const* unzip_dev,
                            int nvars, double tol, double* scores_dev,
                            double* ratio_dev, uint8_t* flags_dev,
                            bssn_stream_t stream);
/* 16 cheap features per block (floats), taken on the even sublattice of the
 * interior (every second point per axis, differences over two points, so
 * a quarter of the rows of chi, alpha, K and Gt^i are read): log10 of max
 * |centred difference| of chi (x,y,z), of alpha (x,y,z), max |K|, max |Gt^i|
 * (3), level, side/55, log10 min chi, log10 max |second difference| of chi
 * and of alpha, log10 h. */
int bssn_remesh_features_f64(bssn_mesh mesh, const double* const* unzip_dev,
                             float* feats_dev, bssn_stream_t stream);
/* The indicator network: 16 -> 64 -> 64 -> 1 with GELU, parameters
 * W1[64][16], b1[64], W2[64][64], b2[64], W3[64], b3 (BSSN_MLP_NPARAM
 * values) held in BF16 for compute, all accumulation in FP32.  norm_dev
 * (optional): 16 means then 16 inverse standard deviations applied to the
 * inputs. */
#define BSSN_MLP_NPARAM 5313
/* Logits on the tensor cores (mma.sync, BF16 operands: the normalised
 * inputs and hidden activations are rounded to BF16; FP32 accumulation).
 * The learned decisions use this forward. */
int bssn_remesh_mlp_fwd_bf16(const void* wq_dev, const float* norm_dev,
                             const float* x_dev, int n, float* logits_dev,
                             bssn_stream_t stream);
/* The same network with FP32 activations (the forward of the training
 * gradient, bssn_remesh_mlp_bwd_bf16). */
int bssn_remesh_mlp_fwd_fp32_bf16(const void* wq_dev, const float* norm_dev,
                                  const float* x_dev, int n, float* logits_dev,
                                  bssn_stream_t stream);
/* floats of scratch bssn_remesh_mlp_bwd_bf16 needs for n samples */
size_t bssn_remesh_mlp_grad_scratch(int n);
/* Gradient of L = sum_i c_i BCE(sigmoid(z_i), y_i) / n with respect to the
 * parameters (FP32, deterministic order); c_dev optional (1); loss_dev
 * optional. */
int bssn_remesh_mlp_bwd_bf16(const void* wq_dev, const float* norm_dev,
                             const float* x_dev, const float* y_dev,
                             const float* c_dev, int n, float* grad_dev,
                             float* loss_dev, float* scratch_dev,
                             bssn_stream_t stream);
/* The same gradient without any device allocation, for callers that cannot
 * allocate when they need it: an application that owns all device memory
 * through its own pool under a fixed budget and forbids libraries to
 * allocate behind its back, or a time-stepping loop that must not pay the
 * implicit synchronisation and latency of cudaMalloc / cudaFree, nor risk
 * their failure, in the middle of a run.  No
 * counterpart in the reference.  The per-CTA partial sums live in one fixed
 * array in device memory (2.72 MB, held on every GPU that loads the library
 * until the process exits), so n is limited to 16384 samples: larger n
 * returns BSSN_ELIMIT before any launch.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  All calls on a
 * device share the array, so calls whose kernels overlap on the GPU (for
 * example issued on two streams) race on it; serialise them.  The address is
 * kept for the life of the process: a device reset (cudaDeviceReset) is not
 * supported between calls. */
int bssn_remesh_mlp_bwd_noalloc_bf16(const void* wq_dev, const float* norm_dev,
                                     const float* x_dev, const float* y_dev,
                                     const float* c_dev, int n, float* grad_dev,
                                     float* loss_dev, bssn_stream_t stream);
/* Adam step on FP32 master parameters, refreshing the BF16 copy (step t>=1). */
int bssn_remesh_mlp_step_bf16(float* master_dev, void* wq_dev,
                              const float* grad_dev, float* m_dev, float* v_dev,
                              float lr, float beta1, float beta2, float eps,
                              int t, bssn_stream_t stream);
/* The learned decision: features -> network -> refine where p >= hi, keep
 * where p <= lo, run the exact test on the uncertain blocks and on a seeded
 * audit sample (fraction audit_frac); flags_dev gets one byte per block.
 * stats_dev (4 ints): uncertain blocks, extra audited blocks, audited
 * blocks the network alone would have missed, audited blocks the exact test
 * refines.  work_dev: bssn_remesh_decide_work_bytes(mesh) bytes. */
size_t bssn_remesh_decide_work_bytes(bssn_mesh mesh);
int bssn_remesh_decide_f64(bssn_mesh mesh, const double* const* unzip_dev,
                           const void* wq_dev, const float* norm_dev, float lo,
                           float hi, double audit_frac, uint64_t seed,
                           double tol, uint8_t* flags_dev, int* stats_dev,
                           void* work_dev, size_t work_bytes,
                           bssn_stream_t stream);

/* Both flags of isReMeshWAMR (BSSN_GR/src/dataUtils.cpp:413-480) learned in
 * one pass: refine (exact: block score > tol) from the network wq_refine
 * with thresholds lo_r / hi_r, keep (exact: score > keep_fac * tol,
 * BSSN_DENDRO_AMR_FAC) from wq_keep with lo_k / hi_k.  The features are
 * computed once; the exact wavelet test runs once, on the blocks either
 * network is unsure of plus one seeded audit sample (fraction audit_frac),
 * and gives both flags there.  Refine implies keep: a block the refine
 * network is sure to refine (p_r >= hi_r) keeps its level without asking
 * the keep network, and a block the keep network is sure to release
 * (p_k <= lo_k) is not refined.  stats_dev (8 ints): blocks uncertain for
 * refine, uncertain for keep, extra audited blocks, audited refine misses of
 * the network (p_r <= lo_r, exact refines), audited exact refines, audited
 * keep misses, audited exact keeps, 0.  work_dev:
 * bssn_remesh_decide2_work_bytes(mesh) bytes. */
size_t bssn_remesh_decide2_work_bytes(bssn_mesh mesh);
int bssn_remesh_decide2_f64(bssn_mesh mesh, const double* const* unzip_dev,
                            const void* wq_refine, const float* norm_refine,
                            float lo_r, float hi_r, const void* wq_keep,
                            const float* norm_keep, float lo_k, float hi_k,
                            double audit_frac, uint64_t seed, double tol,
                            double keep_fac, uint8_t* refine_dev,
                            uint8_t* keep_dev, int* stats_dev, void* work_dev,
                            size_t work_bytes, bssn_stream_t stream);

/* The two-flag decision per element instead of per block (the learned
 * decision has no counterpart in the reference; the exact test it stands in
 * for, isReMeshWAMR, BSSN_GR/src/dataUtils.cpp:511-624, also scores each
 * element): 16 features per element
 * (bssn_remesh_element_features_f64), both networks per element, the exact
 * test only on the elements either network is unsure of plus the seeded audit
 * sample (a fraction of the elements); a block refines (keeps its level)
 * when any of its elements does, so once the networks refine (keep) one
 * element of a block, its other elements go to the exact test only for a
 * flag still open.  Same parameters and stats as
 * bssn_remesh_decide2_f64, with every count per element; work_dev:
 * bssn_remesh_decide2_elem_work_bytes(mesh) bytes; BSSN_ELIMIT for meshes of
 * 2^31 elements or more.  A deferred large block no longer sends all of its
 * elements to the exact test. */
size_t bssn_remesh_decide2_elem_work_bytes(bssn_mesh mesh);
int bssn_remesh_decide2_elem_f64(bssn_mesh mesh, const double* const* unzip_dev,
                                 const void* wq_refine, const float* norm_refine, float lo_r,
                                 float hi_r, const void* wq_keep, const float* norm_keep,
                                 float lo_k, float hi_k, double audit_frac, uint64_t seed,
                                 double tol, double keep_fac, uint8_t* refine_dev,
                                 uint8_t* keep_dev, int* stats_dev, void* work_dev,
                                 size_t work_bytes, bssn_stream_t stream);
/* 16 features per element (num_elements x 16 floats): the block features'
 * definitions over the element's own sublattice (local node indices 0, 2,
 * 4, 6 along each axis: 64 points); level, side and spacing are the
 * block's. */
int bssn_remesh_element_features_f64(bssn_mesh mesh, const double* const* unzip_dev,
                                     float* feats_dev, bssn_stream_t stream);

/* ---------------------------------------------------------------------- */
/* One whole RK4 step as a plan over a mesh (the reference's per-step
 * sequence rkBSSN.cpp:764-860: per stage unzip -> bssnRHS -> zip -> stage
 * update), same result.  The plan owns its scratch buffers, allocated at
 * creation.  Default form: per stage the ghost fill into padded blocks, the
 * right-hand side on them (one launch sequence per block-size bucket with
 * that bucket's tile, or one launch per block with BSSN_PLAN_PER_BLOCK) and
 * the zip fused with the stage algebra; scratch: two padded 24-variable
 * arrays of bssn_mesh_unzip_size doubles and two zipped ones.
 * BSSN_PLAN_DIRECT (split tiles; meshes of fewer than 2^31 nodes): every
 * block of the single-level mesh is a box of the node grid, so the right-hand
 * side reads the zipped stage state directly (points outside the grid read
 * as zero, as the ghost fill writes them), writes each node's right-hand
 * side once from the block owning it (the zip's owner rule), and a node-wise
 * kernel applies the stage algebra; scratch: three zipped 24-variable arrays
 * (no padded ones).  Same result; on B200 the padded form is faster (the
 * derivative pass stages contiguous padded rows), the direct form needs far
 * less memory.  With BSSN_PLAN_GRAPH the 4-stage sequence is captured once as
 * a CUDA graph and replayed (recaptured when u_dev or dt change).  u_dev (24
 * zipped arrays of G[0]*G[1]*G[2] doubles) is advanced in place. */
#define BSSN_PLAN_ENFORCE_STAGES 1 /* enforce constraints on stage states */
#define BSSN_PLAN_GRAPH 2          /* capture / replay as a CUDA graph */
#define BSSN_PLAN_PER_BLOCK 4      /* one RHS launch per block (plain path) */
#define BSSN_PLAN_DIRECT 8         /* right-hand side on the zipped grid */
#define BSSN_PLAN_DIAG_PSI4 16     /* diagnostics also compute psi4 */
typedef struct bssn_rk4_plan_s* bssn_rk4_plan;
int bssn_rk4_plan_create(bssn_mesh mesh, const BssnParams* params, int flags,
                         bssn_rk4_plan* out);
int bssn_rk4_plan_step(bssn_rk4_plan plan, double* const* u_dev, double dt,
                       bssn_stream_t stream);
/* Constraint diagnostics of the zipped state u_dev: ghost fill of every
 * block, Hamiltonian and momentum constraints (as bssn_constraints_f64) into
 * plan-owned zipped arrays (4 x nodes, allocated on the first call), and
 * their masked L2 norms (as bssn_constraint_norms_f64) into norms_dev[0..3]
 * on the device -- the norms the reference's time loop computes every
 * BSSN_IO_OUTPUT_FREQ steps (BSSN_GR/src/bssnCtx.cpp:597-685).  Uses the
 * plan's padded stage array: BSSN_ESTATE for direct plans. */
int bssn_rk4_plan_diagnostics(bssn_rk4_plan plan, double* const* u_dev,
                              const double xmin[3], double h, const double bh[6],
                              const double radii[2], double* norms_dev,
                              bssn_stream_t stream);
/* One bssn_rk4_plan_step followed by bssn_rk4_plan_diagnostics of the new
 * state; with BSSN_PLAN_GRAPH both are captured as one graph (kept beside
 * the plain step's graph and replayed while u_dev, dt and the diagnostic
 * arguments are unchanged), so a loop that reports the norms every k steps
 * never synchronises with the host. */
int bssn_rk4_plan_step_diag(bssn_rk4_plan plan, double* const* u_dev, double dt,
                            const double xmin[3], double h, const double bh[6],
                            const double radii[2], double* norms_dev,
                            bssn_stream_t stream);
/* The plan's diagnostic fields (zipped, n_nodes doubles each) as written by
 * its last diagnostics call: fields_dev[0..3] = ham, mom0..2 and, with
 * BSSN_PLAN_DIAG_PSI4, fields_dev[4..5] = psi4 real, imaginary (ready for
 * bssn_gw_extract_f64); BSSN_ESTATE before the first diagnostics call. */
int bssn_rk4_plan_diag_fields(bssn_rk4_plan plan, double** fields_dev);
/* Copies the first nfields of those fields into caller arrays (device to
 * device, on `stream`). */
int bssn_rk4_plan_copy_diag_fields(bssn_rk4_plan plan, double* const* dst_dev, int nfields,
                                   bssn_stream_t stream);
/* Autotuner: times every tile the plan can run (direct plans: split tiles
 * only) on every block-size bucket of the mesh with the state u_dev (best of
 * reps) and keeps the fastest per bucket in the mesh handle.  Blocking.
 * times (optional): nbuckets x bssn_tile_count() milliseconds, buckets in
 * increasing side order, 1e30 for tiles not timed. */
int bssn_rk4_plan_autotune(bssn_rk4_plan plan, double* const* u_dev, int reps,
                           bssn_stream_t stream, float* times);
/* The tile the plan runs for block side `side` (the autotuned or pinned
 * one; before either, the split 7x7x7 tile). */
int bssn_rk4_plan_tile(bssn_rk4_plan plan, int side);
/* Pin the tile for block side `side` (0: every side; direct plans take one
 * split tile for all sides), as the autotuner would; the next step
 * recaptures its graph.  BSSN_EINVAL for a tile the plan cannot run. */
int bssn_rk4_plan_set_tile(bssn_rk4_plan plan, int side, int tile);
/* Enforcement violations accumulated since creation (blocking read). */
int bssn_rk4_plan_violations(bssn_rk4_plan plan, int* count);
int bssn_rk4_plan_destroy(bssn_rk4_plan plan);
/* Average milliseconds of one right-hand-side pass over all blocks (every
 * bucket with its tile) on the plan's current stage state (CUDA events,
 * after one warm-up).  Blocking. */
int bssn_rk4_plan_time_rhs(bssn_rk4_plan plan, int reps, bssn_stream_t stream,
                           float* ms);
/* Per-kernel timing of the right-hand-side pass (CUDA events around every
 * launch, `reps` passes after one warm-up): out[0..2] = milliseconds per pass
 * in fused, derivative and equation kernels; out[3..5] = their launches per
 * pass.  Blocking.  Used for the kernels' rooflines. */
int bssn_rk4_plan_time_kernels(bssn_rk4_plan plan, int reps, bssn_stream_t stream,
                               double out[6]);
/* Kernel launches one bssn_rk4_plan_step makes with the current tiles. */
int bssn_rk4_plan_launches_per_step(bssn_rk4_plan plan);
/* Measured FP64 fused-multiply-add throughput of this device in TFLOP/s
 * (2 flops per FMA, all SMs, independent chains); scratch_dev: 1 double. */
int bssn_fp64_probe(double* scratch_dev, int iters, bssn_stream_t stream,
                    double* tflops);

/* ---------------------------------------------------------------------- */
/* Synthetic single-level octree meshes (host only, no device work).
 * The domain is a box of super-cells of 8^3 octants; each super-cell is
 * split top-down with seeded choices into blocks of 1, 2, 4 or 8 octants
 * per side (padded sides 13, 19, 31, 55) so that the expected block-count
 * fractions are p[0..3].  mode 0: uniform 13^3 blocks on an M^3 octant box
 * (M = dims[0]); mode 1: seeded mix on a dims[0]xdims[1]xdims[2] super-cell
 * box.  Coordinates: the box spans [xmin, xmin + L] along its longest axis,
 * octant width L / octants, h = octant width / 6.  Block offsets are packed
 * in block order, each rounded up to an even number of doubles.
 * Call once with blocks == NULL to get the count in *nblocks. */
int bssn_mesh_generate(int mode, const int32_t dims[3], const double p[4],
                       uint64_t seed, double xmin, double L,
                       BssnBlockDesc* blocks, int* nblocks, int32_t G[3],
                       double* h);

/* ---------------------------------------------------------------------- */
/* Multi-GPU form: the blocks are split along their Z-order and each rank
 * evolves its own blocks on the bounding box of their padded regions in the
 * node grid; before each stage the halo nodes its blocks read but other
 * ranks own are exchanged (the reference's ghostExchangeStart / RecvSync
 * around its unzip, rkBSSN.cpp:620-641, over MPI; here any point-to-point
 * transport, e.g. NCCL send/recv, with these pack / unpack kernels). */

/* part[b] = the rank of block b: nparts Z-order ranges (Morton keys of the
 * blocks' origins) with about equal interior-zone counts; the reference
 * partitions its octree along a space-filling curve (CMakeLists.txt:51).
 * Host only. */
int bssn_mesh_partition(const BssnBlockDesc* blocks, int nblocks, int nparts,
                        int32_t* part);
/* One RK4 stage (0..3) of a plan's step (the per-stage body of
 * rkBSSN.cpp:764-860): stage 0 reads u_dev, stages 1..3 the plan's stage
 * state; stages 0..2 write the stage state and the accumulator, stage 3
 * writes u_dev.  Four calls with the same u_dev and dt make one step of
 * bssn_rk4_plan_step (eagerly, no graph), with room for a halo exchange
 * before each. */
int bssn_rk4_plan_stage(bssn_rk4_plan plan, double* const* u_dev, double dt,
                        int stage, bssn_stream_t stream);
/* The 24 device arrays of the plan's intermediate stage state (G[0]*G[1]*G[2]
 * doubles each; stages 1..3 read it). */
int bssn_rk4_plan_stage_state(bssn_rk4_plan plan, double** im_dev);
/* buf_dev[v*n + i] = u_dev[v][idx_dev[i]] for the 24 variables, and back. */
int bssn_halo_pack_f64(double* buf_dev, const double* const* u_dev,
                       const int64_t* idx_dev, int64_t n, bssn_stream_t stream);
int bssn_halo_unpack_f64(double* const* u_dev, const double* buf_dev,
                         const int64_t* idx_dev, int64_t n, bssn_stream_t stream);

/* Number of compiled tiles and their brick shape (bx, by, bz, threads).
 * A tile runs its brick shape either fused (one kernel forms the derivatives
 * in registers and evaluates the equations) or split (a derivative pass
 * writes every zone's derivatives to a mesh-owned scratch of 162 doubles per
 * zone, at most 6 Mi zones, allocated by bssn_rk4_plan_create or by the
 * first bssn_rhs_blocks_f64 call with that tile; an equation pass reads them
 * back).  Both give the same result. */
int bssn_tile_count(void);
int bssn_tile_info(int tile, int info[4]);
/* 0 fused, 1 split, -1 unknown tile. */
int bssn_tile_mode(int tile);
/* Host-only replay of a tile's shared-memory indexing over every brick
 * extent, face case and thread: the number of out-of-range reads (0 when
 * every access is in bounds), or -1 for an unknown tile. */
long bssn_tile_selfcheck(int tile);

/* ---------------------------------------------------------------------- */
/* Multi-level meshes (the level-transition ghost fill of dendrolib's
 * ot::Mesh, absent from the reference tree; call sites
 * BSSN_GR/src/rkBSSN.cpp:611-650).  Level l has node spacing h0 / 2^l and
 * a box of level-l octants (6 node intervals each); level 0's box is the
 * whole domain (M0 octants per axis); the box of level l >= 1 lies inside
 * level l-1's box with at least one level-(l-1) octant of margin and starts
 * and ends on level-(l-1) octant corners (even lo and n).  Level l's blocks
 * tile its box minus level l+1's box.  The zipped state of every variable is
 * the concatenation of one dense node grid per level, (6 n + 1) nodes per
 * axis, node (x, y, z) of level l at offset_l + x + dx (y + dy z) with
 * coordinates relative to the box corner.  Ghost fill of a level-l block:
 * level-l nodes where its padded points lie in level l's box, otherwise the
 * level-(l-1) node (even fine index on every axis) or a degree-6 Lagrange
 * interpolation over the 7 nodes of the enclosing level-(l-1) octant along
 * every odd axis (x, then y, then z).  Level sync after every stage: level-
 * (l-1) nodes strictly inside level l's box take the coincident level-l
 * value (finest level first); level-l nodes on its box boundary take the
 * level-(l-1) value or interpolation (coarsest first).  A node no block owns
 * (under a finer box, on a fine box boundary) gets its value only from the
 * sync. */
typedef struct BssnLevelBox {
    int32_t lo[3];          /* first octant, in level-l octants */
    int32_t n[3];           /* octants per axis */
} BssnLevelBox;
/* Several refined regions per level (octree-like refinement around
 * separate sources, e.g. each puncture): a patch hierarchy.  Patch 0 is
 * level 0 (the domain, parent -1); every other patch has a level >= 1, a
 * parent patch of the level below listed before it, and a box of its own
 * level's octants inside the parent's box with one parent octant of margin
 * (even lo and n); patches of one level lie at least one parent octant apart.
 * A patch's region is its box minus its children's boxes.  Every level rule
 * above holds per patch (its own node grid; ghost fill from the patch or
 * its parent; restriction into the parent; prolongation of its boundary
 * from the parent).  A box per level is the chain of patches l, parent l-1. */
typedef struct BssnPatch {
    int32_t level;
    int32_t parent;         /* patch index, -1 for patch 0 */
    int32_t lo[3];
    int32_t n[3];
} BssnPatch;
int bssn_mesh_generate_patches(int npatches, const int32_t M0[3], const BssnPatch* patches,
                               double xmin, double h0, BssnBlockDesc* blocks, int* nblocks,
                               int64_t* n_nodes);
int bssn_mesh_create_patches(const BssnBlockDesc* blocks, int nblocks, int npatches,
                             const int32_t M0[3], const BssnPatch* patches, bssn_mesh* out);
int bssn_patches_maps(const BssnBlockDesc* blocks, int nblocks, int npatches, const int32_t M0[3],
                      const BssnPatch* patches, int64_t sizes[5], int64_t* unzip_src,
                      int64_t* zip_src, int64_t* inject, int64_t* prolong, int64_t* interp);
/* Tiles the levels with blocks (sides 13/19/31/55, level, g0 = first
 * interior node in the level's global node index, ptmin/ptmax from
 * xmin + (g0 - 3) h_l, physical-boundary flags on level 0).  blocks == NULL
 * returns the count only.  *n_nodes: zipped nodes of all levels (< 2^31).
 * Host only. */
int bssn_mesh_generate_levels(int nlevels, const int32_t M0[3], const BssnLevelBox* boxes,
                              double xmin, double h0, BssnBlockDesc* blocks, int* nblocks,
                              int64_t* n_nodes);
/* The same tiling with blocks of at most max_w octants per axis (1, 2, 4 or
 * 8: padded sides up to 13, 19, 31 or 55), the patches given as in
 * bssn_mesh_generate_patches (a chain of one box per level is the patch list
 * level l, parent l - 1). */
int bssn_mesh_generate_patches_w(int npatches, const int32_t M0[3], const BssnPatch* patches,
                                 double xmin, double h0, int max_w, BssnBlockDesc* blocks,
                                 int* nblocks, int64_t* n_nodes);
/* Mesh handle of a generated multi-level mesh.  bssn_unzip_f64 and
 * bssn_zip_f64 on it use the level maps; RK4 plans on it run the padded form
 * (ghost fill, right-hand side per block with its own spacing, owner gather,
 * node-wise stage, level sync). */
int bssn_mesh_create_levels(const BssnBlockDesc* blocks, int nblocks, int nlevels,
                            const int32_t M0[3], const BssnLevelBox* boxes, bssn_mesh* out);
/* State transfer after a remesh (BSSNCtx::grid_transfer,
 * BSSN_GR/src/bssnCtx.cpp:1319-1340, which calls dendrolib's
 * DVec::grid_transfer; the remesh loop is bssnCtx.cpp:393-445): u_new on
 * the hierarchy `to` from u_old on `from` (same level-0 domain).  Every node
 * of level l of `to` takes the node of level l of `from` where that grid has
 * it, otherwise the coincident level-(l-1) node or the ghost-fill
 * interpolation from `to`'s level l-1 (levels in increasing order); then
 * the level sync of `to`.  Builds its maps on the host and allocates (and
 * frees) device memory for them; blocking. */
int bssn_levels_transfer(bssn_mesh from, const double* const* u_old_dev, bssn_mesh to,
                         double* const* u_new_dev, int nvars, bssn_stream_t stream);
/* Level sync of a zipped state (after initial data or any outside update). */
int bssn_mesh_levels_sync(bssn_mesh mesh, double* const* u_dev, int nvars,
                          bssn_stream_t stream);
/* Host-only copies of the level maps, for tests: per padded point the
 * ghost-fill source (>= 0 node, -1 zero, <= -2 interpolation entry
 * -2 - src), per node the owning zone's padded index (-1: none), and the
 * injection / prolongation pairs (dst node, src as above).  Call with NULL
 * arrays to get the sizes (sizes[0..4] = padded points, nodes, injections,
 * prolongations, interpolation entries); interp receives per entry
 * {base, stride x, stride y, stride z, jx, jy, jz} as int64. */
int bssn_levels_maps(const BssnBlockDesc* blocks, int nblocks, int nlevels, const int32_t M0[3],
                     const BssnLevelBox* boxes, int64_t sizes[5], int64_t* unzip_src,
                     int64_t* zip_src, int64_t* inject, int64_t* prolong, int64_t* interp);

/* ---------------------------------------------------------------------- */
/* Checkpoint and restart: BSSNCtx::write_checkpt / restore_checkpt
 * (BSSN_GR/src/bssnCtx.cpp:783-862, 864-1170).  Files, as the reference
 * names them:
 *   <prefix>_step_<i>.cp          JSON header, the reference's keys (rank 0)
 *   <prefix>_octree_<i>_<r>.oct   rank r's mesh: grid dims, spacing, origin
 *                                 and block list (this library's own binary
 *                                 layout; the reference stores dendrolib
 *                                 octants)
 *   <prefix>_<i>_<r>.var          rank r's 24 zipped variables (binary)
 * Binary files carry a magic word and a checksum; a file that fails either
 * reads as BSSN_EIO.  Slot i alternates as the reference's does (see
 * bssn_checkpoint_index); restart takes the slot of 0 and 1 with the larger
 * step. */
#define BSSN_EIO 7          /* checkpoint file unreadable or corrupted */
#define BSSN_ENOENT 8       /* no checkpoint file found */

typedef struct BssnCheckpointInfo {
    double time_begin;      /* DENDRO_TS_TIME_BEGIN */
    double time_end;        /* DENDRO_TS_TIME_END */
    double time_current;    /* DENDRO_TS_TIME_CURRENT (and _LAST_IO_TIME) */
    double time_step;       /* DENDRO_TS_TIME_STEP_SIZE */
    int64_t step;           /* DENDRO_TS_STEP_CURRENT */
    int32_t element_order;  /* DENDRO_TS_ELEMENT_ORDER (6) */
    int32_t num_vars;       /* DENDRO_TS_NUM_VARS (24) */
    int32_t active_comm_size; /* DENDRO_TS_ACTIVE_COMM_SZ */
    int32_t reserved;
    double wavelet_tol;     /* DENDRO_TS_WAVELET_TOLERANCE */
    double load_imb_tol;    /* DENDRO_TS_LOAD_IMB_TOLERANCE */
    double bh[2][3];        /* DENDRO_BH1_X .. DENDRO_BH2_Z */
} BssnCheckpointInfo;

/* The slot a checkpoint at `step` goes to: 0 when step % (2*freq) == 0,
 * else 1; 3 for the first checkpoint after the punctures merged (merged
 * nonzero and *merged_written zero; sets *merged_written).  bssnCtx.cpp:786-796. */
int bssn_checkpoint_index(int64_t step, int freq, int merged, int* merged_written);
/* Writes rank `rank`'s .oct and .var files of slot `index` (the 24 arrays of
 * n_nodes doubles at u_dev, device or host memory, copied through a pinned
 * buffer on `stream`), and the .cp header when write_header is nonzero. */
int bssn_checkpoint_write(const char* prefix, int index, int rank, int write_header,
                          const BssnCheckpointInfo* info, const BssnBlockDesc* blocks,
                          int nblocks, const int32_t G[3], double h, const double origin[3],
                          const double* const* u_dev, int64_t n_nodes,
                          bssn_stream_t stream);
/* Reads the .cp headers of slots 0 and 1 and returns the one with the larger
 * step (slot 0 on a tie) in *index and *info.  BSSN_ENOENT when neither
 * exists, BSSN_EIO when the chosen one does not parse. */
int bssn_checkpoint_latest(const char* prefix, int* index, BssnCheckpointInfo* info);
/* Rank r's mesh of slot `index`.  Call with blocks == NULL to get *nblocks;
 * then with room for *nblocks descriptors. */
int bssn_checkpoint_read_mesh(const char* prefix, int index, int rank,
                              BssnBlockDesc* blocks, int* nblocks, int32_t G[3],
                              double* h, double origin[3]);
/* Rank r's 24 zipped variables of slot `index` into u_dev (device or host
 * memory, n_nodes doubles each; n_nodes must match the file). */
int bssn_checkpoint_read_vars(const char* prefix, int index, int rank,
                              double* const* u_dev, int64_t n_nodes,
                              bssn_stream_t stream);

const char* bssn_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BSSN_B200_H */
