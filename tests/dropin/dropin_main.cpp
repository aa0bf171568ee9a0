// Test helper: exercises the host-array drop-in surface
// (include/bssn_b200_dendro.hpp) the way a reference caller would, reading
// inputs from and writing outputs to raw float64 files.
//   dropin_main rhs   <side> <bflag> <pmin x y z> <pmax x y z> <in.bin> <out.bin>
//   dropin_main deriv <kind> <side> <bflag> <h> <in.bin> <out.bin>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bssn_b200_dendro.hpp"

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
