// Test helper: exercises the host-array drop-in surface
// (include/bssn_b200_dendro.hpp) the way a reference caller would, reading
// inputs from and writing outputs to raw float64 files.
//   dropin_main rhs   <side> <bflag> <pmin x y z> <pmax x y z> <in.bin> <out.bin>
//   dropin_main deriv <kind> <side> <bflag> <h> <in.bin> <out.bin>
//   dropin_main refsig <side> <bflag> <in.bin> <rhs.bin> <enforced.bin>
// refsig calls the reference-signature forms with the reference's own
// argument lists (rhs.h:28-36, bssn_constraints.h:15) through stand-ins for
// dendrolib's ot::Block, TreeNode and Point, and writes the right-hand side
// followed by the block's ptmin / ptmax (6 doubles), then the state after
// enforce_bssn_constraints(u, node) on every node.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bssn_b200_dendro.hpp"

// Stand-ins for the dendrolib types bssnRHS reads (accessor names of
// BSSN_GR/src/rhs.cpp:50-67).
struct Point {
    double v[3];
    Point(double x, double y, double z) : v{x, y, z} {}
    double x() const { return v[0]; }
    double y() const { return v[1]; }
    double z() const { return v[2]; }
};
struct TreeNode {
    unsigned lo[3], hi[3];
    unsigned minX() const { return lo[0]; }
    unsigned minY() const { return lo[1]; }
    unsigned minZ() const { return lo[2]; }
    unsigned maxX() const { return hi[0]; }
    unsigned maxY() const { return hi[1]; }
    unsigned maxZ() const { return hi[2]; }
};
namespace ot {
class Block {
   public:
    Block(unsigned off, unsigned s, unsigned flag, TreeNode n, unsigned span)
        : off_(off), s_(s), flag_(flag), node_(n), span_(span) {}
    unsigned getOffset() const { return off_; }
    unsigned getAllocationSzX() const { return s_; }
    unsigned getAllocationSzY() const { return s_; }
    unsigned getAllocationSzZ() const { return s_; }
    unsigned getBlkNodeFlag() const { return flag_; }
    const TreeNode& getBlockNode() const { return node_; }
    // grid spacing: the node's physical width over its s - 7 intervals
    double computeDx(const Point& a, const Point& b) const { return w(b.x() - a.x(), 0); }
    double computeDy(const Point& a, const Point& b) const { return w(b.y() - a.y(), 1); }
    double computeDz(const Point& a, const Point& b) const { return w(b.z() - a.z(), 2); }

   private:
    double w(double L, int d) const { return L * (node_.hi[d] - node_.lo[d]) / ((double)span_ * (s_ - 7)); }
    unsigned off_, s_, flag_;
    TreeNode node_;
    unsigned span_;
};
}  // namespace ot

static std::vector<double> readf(const char* p, size_t n) {
    std::vector<double> v(n);
    FILE* f = std::fopen(p, "rb");
    if (!f || std::fread(v.data(), 8, n, f) != n) std::exit(3);
    std::fclose(f);
    return v;
}
static void writef(const char* p, const std::vector<double>& v) {
    FILE* f = std::fopen(p, "wb");
    std::fwrite(v.data(), 8, v.size(), f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    if (!std::strcmp(argv[1], "rhs")) {
        const unsigned s = std::atoi(argv[2]), bflag = std::atoi(argv[3]);
        const double pmin[3] = {atof(argv[4]), atof(argv[5]), atof(argv[6])};
        const double pmax[3] = {atof(argv[7]), atof(argv[8]), atof(argv[9])};
        const size_t n = (size_t)s * s * s;
        std::vector<double> U = readf(argv[10], 24 * n), R(24 * n, -7.0);
        const double* up[24];
        double* rp[24];
        for (int v = 0; v < 24; v++) {
            up[v] = &U[v * n];
            rp[v] = &R[v * n];
        }
        BssnParams p = {0.4, {1, 1, 1, 1}, {1.0, 0.0}, 2.0, 2.0, 40.0, 0, 0.99, 0.3, 1e-4};
        const unsigned sz[3] = {s, s, s};
        const unsigned off = 0;
        int rc = dendro_b200::bssnrhs(rp, up, off, pmin, pmax, sz, bflag, p);
        if (rc) return 10 + rc;
        // also the batched block-list form on the same block
        std::vector<double> R2(24 * n, -7.0);
        double* rp2[24];
        for (int v = 0; v < 24; v++) rp2[v] = &R2[v * n];
        dendro_b200::Block b = {0, {s, s, s}, bflag, {pmin[0], pmin[1], pmin[2]}, {pmax[0], pmax[1], pmax[2]}};
        rc = dendro_b200::bssnRHS(rp2, up, &b, 1, p);
        if (rc) return 20 + rc;
        if (std::memcmp(R.data(), R2.data(), R.size() * 8)) return 30;
        writef(argv[11], R);
        return 0;
    }
    if (!std::strcmp(argv[1], "refsig")) {
        using dendro_b200::bssnrhs;
        using dendro_b200::bssnRHS;
        using dendro_b200::enforce_bssn_constraints;
        const unsigned s = std::atoi(argv[2]), bflag = std::atoi(argv[3]);
        const size_t n = (size_t)s * s * s;
        std::vector<double> U = readf(argv[4], 24 * n), R(24 * n, -7.0), R2(24 * n, -7.0);
        BssnParams p = {0.4, {1, 1, 1, 1}, {1.0, 0.0}, 2.0, 2.0, 40.0, 0, 0.99, 0.3, 1e-4};
        dendro_b200::set_params(p);
        // domain [-8, 8]^3 on an octree of 2^6 units per axis; the block's
        // node spans (s - 7) / 6 octants of 2 units
        const unsigned span = 64, w = 2 * (s - 7) / 6;
        dendro_b200::set_domain({{-8.0, -8.0, -8.0}, {8.0, 8.0, 8.0}, {0, 0, 0}, {span, span, span}});
        const TreeNode node = {{10, 20, 30}, {10 + w, 20 + w, 30 + w}};
        const ot::Block blk(0, s, bflag, node, span);
        // ptmin / ptmax exactly as BSSN_GR/src/rhs.cpp:50-67 forms them
        const Point pt_min(-8.0, -8.0, -8.0), pt_max(8.0, 8.0, 8.0);
        const unsigned PW = 3;
        auto gx = [&](unsigned g) { return ((16.0 / span) * (g - 0u)) + -8.0; };
        const double dx = blk.computeDx(pt_min, pt_max), dy = blk.computeDy(pt_min, pt_max),
                     dz = blk.computeDz(pt_min, pt_max);
        const double ptmin[3] = {gx(node.minX()) - PW * dx, gx(node.minY()) - PW * dy, gx(node.minZ()) - PW * dz};
        const double ptmax[3] = {gx(node.maxX()) + PW * dx, gx(node.maxY()) + PW * dy, gx(node.maxZ()) + PW * dz};
        const double* up[24];
        double *rp[24], *rp2[24];
        for (int v = 0; v < 24; v++) {
            up[v] = &U[v * n];
            rp[v] = &R[v * n];
            rp2[v] = &R2[v * n];
        }
        const unsigned sz[3] = {s, s, s};
        const unsigned offset = blk.getOffset();
        const double t = 0.0;
        const double** cons = nullptr;
        bssnrhs(rp, up, offset, ptmin, ptmax, sz, bflag, t, cons);
        if (dendro_b200::last_status()) return 40;
        bssnRHS(rp2, up, &blk, 1u, t, cons);
        if (dendro_b200::last_status()) return 41;
        if (std::memcmp(R.data(), R2.data(), R.size() * 8)) return 42;
        for (int d = 0; d < 3; d++) R.push_back(ptmin[d]);
        for (int d = 0; d < 3; d++) R.push_back(ptmax[d]);
        writef(argv[5], R);
        double* uu[24];
        for (int v = 0; v < 24; v++) uu[v] = &U[v * n];
        for (unsigned node_i = 0; node_i < n; node_i++) {
            enforce_bssn_constraints(uu, node_i);
            if (dendro_b200::last_status() > 0) return 43;
        }
        writef(argv[6], U);
        return 0;
    }
    if (!std::strcmp(argv[1], "deriv")) {
        const int kind = std::atoi(argv[2]);
        const unsigned s = std::atoi(argv[3]), bflag = std::atoi(argv[4]);
        const double h = std::atof(argv[5]);
        const size_t n = (size_t)s * s * s;
        std::vector<double> u = readf(argv[6], n), D(n, 0.0);
        const unsigned sz[3] = {s, s, s};
        int (*fn[9])(double*, const double*, double, const unsigned*, unsigned) = {
            dendro_b200::deriv644_x, dendro_b200::deriv644_y, dendro_b200::deriv644_z,
            dendro_b200::deriv644_xx, dendro_b200::deriv644_yy, dendro_b200::deriv644_zz,
            dendro_b200::ko_deriv42_x, dendro_b200::ko_deriv42_y, dendro_b200::ko_deriv42_z};
        int rc = fn[kind](D.data(), u.data(), h, sz, bflag);
        if (rc) return 10 + rc;
        writef(argv[7], D);
        return 0;
    }
    return 2;
}
