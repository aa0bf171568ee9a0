// bssn_b200_dendro.hpp -- the reference's C++ call surface, drop-in.
//
// Same names, argument meaning and array layout as Dendro-GR's CPU functions,
// taking HOST arrays; each call stages the data to the GPU, runs the sm_100a
// kernels of libbssn_b200.so and copies the results back.  Declared in
// namespace dendro_b200 so they can be linked beside the reference; a caller
// switches with `using dendro_b200::bssnrhs;` etc.  Callers that keep their
// state on the device should use the C ABI in bssn_b200.h directly.
//
// Differences from the reference, by design:
//   * functions return int status codes (0 ok) instead of void / exit(0);
//   * parameters are passed explicitly (BssnParams) instead of bssn:: globals;
//   * calls are reentrant per thread (each thread owns its device staging
//     buffers) -- the reference's bssnrhs shares one global workspace.
#ifndef BSSN_B200_DENDRO_HPP
#define BSSN_B200_DENDRO_HPP

#include <vector>

#include "bssn_b200.h"

namespace dendro_b200 {

// The fields of ot::Block that bssnRHS reads (BSSN_GR/src/rhs.cpp:50-67):
// offset, allocation size, boundary flag and the padded-block corner
// coordinates ptmin = block min - PW*dx, ptmax = block max + PW*dx.
struct Block {
    unsigned offset;
    unsigned sz[3];
    unsigned bflag;
    double ptmin[3];
    double ptmax[3];
};

// deriv644_{x,y,z}, deriv644_{xx,yy,zz}, ko_deriv42_{x,y,z}
// (BSSN_GR/include/derivs.h:42-130, src/derivs.cpp): one padded block of
// sz[0]*sz[1]*sz[2] host doubles; writes exactly the points the reference
// writes, bit-identical values.
int deriv644_x(double* Dxu, const double* u, double dx, const unsigned* sz, unsigned bflag);
int deriv644_y(double* Dyu, const double* u, double dy, const unsigned* sz, unsigned bflag);
int deriv644_z(double* Dzu, const double* u, double dz, const unsigned* sz, unsigned bflag);
int deriv644_xx(double* Du, const double* u, double dx, const unsigned* sz, unsigned bflag);
int deriv644_yy(double* Du, const double* u, double dy, const unsigned* sz, unsigned bflag);
int deriv644_zz(double* Du, const double* u, double dz, const unsigned* sz, unsigned bflag);
int ko_deriv42_x(double* Du, const double* u, double dx, const unsigned* sz, unsigned bflag);
int ko_deriv42_y(double* Du, const double* u, double dy, const unsigned* sz, unsigned bflag);
int ko_deriv42_z(double* Du, const double* u, double dz, const unsigned* sz, unsigned bflag);
// deriv644adv_{x,y,z}: the reference hard-wires them to the centred stencil.
int deriv644adv_x(double* Dxu, const double* u, double dx, const unsigned* sz, const double* betax, unsigned bflag);
int deriv644adv_y(double* Dyu, const double* u, double dy, const unsigned* sz, const double* betay, unsigned bflag);
int deriv644adv_z(double* Dzu, const double* u, double dz, const unsigned* sz, const double* betaz, unsigned bflag);

// bssnrhs (BSSN_GR/src/rhs.cpp:80-504, include/rhs.h:32-36): the RHS of one
// padded block at `offset` in each of the 24 host arrays; interior points of
// unzipVarsRHS are written, its halo is left as it was.  t and uZipConstVars
// are accepted and unused, as in the standard-gauge equations.
int bssnrhs(double** unzipVarsRHS, const double** uZipVars, const unsigned& offset,
            const double* pmin, const double* pmax, const unsigned* sz,
            const unsigned& bflag, const BssnParams& params, double t = 0.0,
            const double** uZipConstVars = nullptr);

// bssnRHS (BSSN_GR/src/rhs.cpp:10-73): all blocks of a block list in one
// batched launch.  Arrays hold n_unzip doubles per variable.
int bssnRHS(double** uzipVarsRHS, const double** uZipVars, const Block* blkList,
            unsigned numBlocks, const BssnParams& params, double curr_time = 0.0,
            const double** uZipConstVars = nullptr);

// enforce_bssn_constraints (BSSN_GR/include/bssn_constraints.h:15-172) on
// zipped nodes [begin, end) of 24 host arrays; returns 0, or the number of
// nodes that violated det(gt) > 0 / |det - 1| <= 1e-6 / |tr A| <= 1e-6 (the
// reference exits there) as a negative count.
int enforce_bssn_constraints(double** uiVar, unsigned begin, unsigned end, double chi_floor);
inline int enforce_bssn_constraints(double** uiVar, unsigned node, double chi_floor) {
    return enforce_bssn_constraints(uiVar, node, node + 1, chi_floor);
}

// ---------------------------------------------------------------------------
// Reference-signature forms.  These take exactly the reference's parameter
// lists (BSSN_GR/include/rhs.h:28-36, BSSN_GR/include/bssn_constraints.h:15),
// so a reference call site compiles unchanged after
//     using dendro_b200::bssnrhs; using dendro_b200::bssnRHS;
//     using dendro_b200::enforce_bssn_constraints;
// and one dendro_b200::set_params(...) (plus set_domain(...) for bssnRHS) at
// start-up, in place of the bssn:: globals the reference reads.  They return
// void like the reference; the status of the calling thread's last call is
// last_status() (0 ok, BSSN_E* otherwise) -- no exit(), no trap.
// ---------------------------------------------------------------------------

// Parameters of the reference-signature forms (thread safe; default: KO sigma
// 0.4, lambda {1,1,1,1}, lambda_f {1,0}, eta 2 everywhere, no CAKO, chi floor
// 1e-4).
void set_params(const BssnParams& params);
BssnParams get_params();

// The coordinate map of BSSN_GR/include/grDef.h:16-21 (GRIDX_TO_X ...):
// x = (compd_max - compd_min) / (octree_max - octree_min) * (xg - octree_min)
//     + compd_min, per axis; octree bounds in octree integer units as
// bssn::BSSN_OCTREE_MIN / MAX, domain bounds as bssn::BSSN_COMPD_MIN / MAX.
struct Domain {
    double compd_min[3];
    double compd_max[3];
    unsigned octree_min[3];
    unsigned octree_max[3];
};
void set_domain(const Domain& d);
Domain get_domain();

int last_status();
void set_last_status(int status);

// bssnrhs, BSSN_GR/include/rhs.h:32-36 (t and uZipConstVars are unused by the
// standard-gauge equations, as in the reference).
void bssnrhs(double** uzipVarsRHS, const double** uZipVars, const unsigned int& offset,
             const double* ptmin, const double* ptmax, const unsigned int* sz,
             const unsigned int& bflag, const double t, const double** uZipConstVars);

namespace detail {
// the Point type a block's computeDx takes (dendrolib's Point)
template <class B, class P>
P point_of(double (B::*)(const P&, const P&) const);
template <class B, class P>
P point_of(double (B::*)(const P&, const P&));
}  // namespace detail

// bssnRHS, BSSN_GR/include/rhs.h:28-30, for the caller's own block type
// (dendrolib's ot::Block): per block the offset, allocation sizes, face flag,
// spacings and padded-block corners are taken exactly as
// BSSN_GR/src/rhs.cpp:50-67 takes them, then every block runs in one batched
// launch.
template <class BlockT>
void bssnRHS(double** uzipVarsRHS, const double** uZipVars, const BlockT* blkList,
             unsigned int numBlocks, const double curr_time, const double** uZipConstVars) {
    using PointT = decltype(detail::point_of(&BlockT::computeDx));
    const Domain d = get_domain();
    const PointT pt_min(d.compd_min[0], d.compd_min[1], d.compd_min[2]);
    const PointT pt_max(d.compd_max[0], d.compd_max[1], d.compd_max[2]);
    const unsigned int PW = 3;
    auto grid_to = [&d](int a, unsigned int xg) {
        return (((d.compd_max[a] - d.compd_min[a]) / (d.octree_max[a] - d.octree_min[a])) *
                (xg - d.octree_min[a])) + d.compd_min[a];
    };
    std::vector<Block> list(numBlocks);
    for (unsigned int b = 0; b < numBlocks; b++) {
        const BlockT& blk = blkList[b];
        Block& o = list[b];
        o.offset = blk.getOffset();
        o.sz[0] = blk.getAllocationSzX();
        o.sz[1] = blk.getAllocationSzY();
        o.sz[2] = blk.getAllocationSzZ();
        o.bflag = blk.getBlkNodeFlag();
        const double dx = blk.computeDx(pt_min, pt_max);
        const double dy = blk.computeDy(pt_min, pt_max);
        const double dz = blk.computeDz(pt_min, pt_max);
        o.ptmin[0] = grid_to(0, blk.getBlockNode().minX()) - PW * dx;
        o.ptmin[1] = grid_to(1, blk.getBlockNode().minY()) - PW * dy;
        o.ptmin[2] = grid_to(2, blk.getBlockNode().minZ()) - PW * dz;
        o.ptmax[0] = grid_to(0, blk.getBlockNode().maxX()) + PW * dx;
        o.ptmax[1] = grid_to(1, blk.getBlockNode().maxY()) + PW * dy;
        o.ptmax[2] = grid_to(2, blk.getBlockNode().maxZ()) + PW * dz;
    }
    set_last_status(numBlocks == 0 ? 0
                                   : bssnRHS(uzipVarsRHS, uZipVars, list.data(), numBlocks,
                                             get_params(), curr_time, uZipConstVars));
}

// enforce_bssn_constraints, BSSN_GR/include/bssn_constraints.h:15: one zipped
// node, chi / alpha floor from set_params().  A node that violates det(gt) > 0,
// |det - 1| <= 1e-6 or |tr A| <= 1e-6 sets last_status() to -1 where the
// reference exits (a device error sets it to the negated CUDA error).  (Each call is one device round trip: callers enforcing
// many nodes should use the range form above.)
void enforce_bssn_constraints(double** uiVar, unsigned int node);

}  // namespace dendro_b200

#endif  // BSSN_B200_DENDRO_HPP
