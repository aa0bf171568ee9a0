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

}  // namespace dendro_b200

#endif  // BSSN_B200_DENDRO_HPP
