// geometry.h -- curved-wall geometry of one case (the product's restatement of get_coord,
// 2d_mrlbm.f90:931-1156, and finding_incoming_outgoing_pops, 2d_mrlbm.f90:2005-2057).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/mrlbm.h"
#include "lattice.h"

namespace mrlbm {

struct Lattice64 {
    double w[Q];          // single-precision literals widened (2d_mrlbm.f90:129)
    double hxx[Q], hyy[Q], hxy[Q];
    double cs2, hm, hp;   // hm = 0 - cs2, hp = 1 - cs2
};
Lattice64 make_lattice();

// Is/Os rows (bit k = population k) for quadrant label 0..15.
void link_tables(int label15_rule, int incs[16], int outs[16]);

struct Geometry {
    int nx = 0, ny = 0;
    double x_c = 0, y_c = 0, r_c = 0, r_cyl = 0;
    bool cylinder = false;
    std::vector<int8_t> cls;              // per node (Fortran order): 0 fluid, 1 solid, 2 boundary
    int nb = 0;                           // nbct
    std::vector<int> bi, bj, label;       // boundary nodes in reference order
    std::vector<double> delta;            // delta_uk
    std::vector<double> ref;              // [8*nb]: x_ref1..4, y_ref1..4 (point-major per node)
    std::vector<int> sten;                // [24*nb]: i_p2(1..4), j_p2, i_p3, j_p3, i_p4, j_p4
    std::vector<double> theta;            // theta_c (2d_mrlbm.f90:1132-1133)
    int n_label15 = 0;
    // device tables (field-major), FP64 values computed exactly as the reference
    std::vector<int> tint;                // I_NFIELDS * nb
    std::vector<double> tgeo;             // G_NFIELDS * nb
    int box_x0 = 1, box_y0 = 1, box_w = 0, box_h = 0;
    std::vector<int> boxmap;
};

// Build and validate.  Returns MRLBM_OK or an error code with `err` set.
int build_geometry(const mrlbm_config& cfg, int nx, int ny, double x_c, double y_c, double r_c,
                   Geometry& g, std::string& err);

// nx, ny, centre and radius the config selects (2d_mrlbm.f90:86-92, 946-948 or explicit).
void resolve_domain(const mrlbm_config& cfg, int& nx, int& ny, double& x_c, double& y_c, double& r_c);

// Namelist reader for input.dat (the six groups of 2d_mrlbm.f90:2227-2233).
int read_namelist_file(const char* path, mrlbm_config& cfg, std::string& err);
void config_defaults(mrlbm_config& cfg);

// Seeded-noise initial state (extension INIT_NOISE) and the reference rest state:
// f(nx,ny,0:8) in Fortran order.
void initial_state(const mrlbm_config& cfg, const Lattice64& lat, int nx, int ny, std::vector<double>& f);

}  // namespace mrlbm
