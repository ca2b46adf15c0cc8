// mrlbm_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference program 2d_mrlbm.f90 (sakthi-lbm/mrlbm_2d), used as the
// checker for the CUDA step and as the timed CPU baseline ("port").  Nothing in the product
// links or calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU arm do.
//
// Fidelity rules (the reference's own arithmetic, restated):
//   * FP64 everywhere; the lattice weights are single-precision literals (2d_mrlbm.f90:129),
//     so w(k) = (double)(float)(16/36) etc. and sum(w) = 1 + 7.45e-9.
//   * Hermite tables are e*e - cs2 with cs2 = 1.0d0/3.0d0 (2d_mrlbm.f90:153,171-178).
//   * Sums run k = 0..8 in order from 0 (gfortran's sum intrinsic), products left to right,
//     division only where the Fortran divides.  Compile with -ffp-contract=off (the
//     reference's x86-64 gfortran -O3 build emits no FMA).
//   * Loop structure kept: OpenMP only where the reference has `!$omp parallel do`, serial
//     streaming and serial boundary loops elsewhere.
//
// Parity of this restatement against the reference: the reference has no tests, golden
// vectors or fixtures, and no Fortran compiler exists in this image.  The restatement is
// pinned against outputs of the reference's own source executed by the Fortran-subset
// interpreter in tests/golden/ (fixtures committed there); cases the reference cannot
// express (the extensions below) are unpinned by the reference.
//
// Extensions (mrlbm_config fields, all 0 = reference behaviour):
//   geometry_mode  EXPLICIT: real-valued centre and radius instead of 2d_mrlbm.f90:946-948
//   wall_mode      FREESLIP: halfway specular reflection of the populations leaving through
//                  rows 1 / ny (no closure and no Dirichlet velocity on those rows)
//   label15_rule   ALLNINE: Incs_b(15,:) = Outs_b(15,:) = 1 (the reference leaves row 15 zero)
//   nu_length      DIAMETER: nu = U*(2 r_c)/Re instead of U*(2 r_cyl)/Re (2d_mrlbm.f90:134)
//   init_mode      NOISE: rho = 1, u = (U,0) + seeded Gaussian noise, regularized equilibrium
//   inlet profile  per-row u_in(j) instead of uinlet at 2d_mrlbm.f90:258

#include "../include/mrlbm.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int Q = 9;

// SplitMix64 (Steele, Lea, Flood 2014) keyed by (seed, counter); shared definition of the
// seeded-noise initial state (extension INIT_NOISE).
inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
inline double uniform01(uint64_t seed, uint64_t counter) {
    uint64_t r = splitmix64(seed ^ splitmix64(counter));
    return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
// Box-Muller normal for node n (0-based Fortran linear index) and component c (0 = x, 1 = y).
inline double normal_noise(uint64_t seed, uint64_t n, int c) {
    const double two_pi = 6.283185307179586;
    double u1 = uniform01(seed, 4 * n + 2 * (uint64_t)c);
    double u2 = uniform01(seed, 4 * n + 2 * (uint64_t)c + 1);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2);
}

struct Oracle {
    mrlbm_config cfg;
    int nx = 0, ny = 0;
    // lattice (2d_mrlbm.f90:129-131, 153, 171-178)
    double w[Q], Hxx[Q], Hyy[Q], Hxy[Q];
    int e[Q][2];
    double cs2, nu, omega, uinlet, vinlet, dx = 1.0, dy = 1.0, delx = 0.0, PI;
    double x_c = 0, y_c = 0, r_c = 0, r_cyl = 0;
    bool cyl = false;
    // fields
    std::vector<double> f, f_tmp, fout, rho, p, ux, uy, mxx, myy, mxy, mxxp, myyp;
    std::vector<double> mxx_s, myy_s, mxy_s;
    std::vector<int> isfluid, issolid, isbound;
    std::vector<double> cth_glb, sth_glb, s2th_glb, c2th_glb;
    std::vector<double> cx_p, cy_p, Hxx_p, Hyy_p, Hxy_p;
    // cylinder (2d_mrlbm.f90:2304-2332)
    int nbct = 0;
    std::vector<int> bou_i, bou_j, label_bc, idx;
    std::vector<double> radii, xb, yb, delta_uk, theta_c, thetas_cy, cth_cyl, sth_cyl;
    std::vector<double> x_ref[5], y_ref[5];            // index 1..4 used
    std::vector<int> i_p[5], j_p[5];                   // index 2..4 used, [m + 4*(k-1)], m = 0..3
    std::vector<double> uxp_b, uyp_b, F_drag, F_lift;
    int Incs_b[16][Q], Outs_b[16][Q];
    // run state
    int iter = 0;
    std::vector<double> u_in;                         // extension: per-row inlet velocity
    double rho_inf_mean = 0.0, rho_infty = 1.0;
    std::vector<int> h_iter;
    std::vector<double> h_fd, h_fl, h_rhoin;
    std::vector<double> h_psurf, h_psmooth, h_probe;   // per stats step: nbct, nbct, 12 values
    int i_probe[4] = {0, 0, 0, 0}, j_probe[4] = {0, 0, 0, 0};
    void write_statistics_out();                       // 2d_mrlbm.f90:593-616 (records, no files)
    std::string err;

    inline size_t I(int i, int j) const { return (size_t)(i - 1) + (size_t)nx * (size_t)(j - 1); }
    inline size_t F(int i, int j, int k) const { return I(i, j) + (size_t)nx * (size_t)ny * (size_t)k; }
    inline double X(int i) const { return (double)i; }    // x(i,:) = real(i)  (2d_mrlbm.f90:950-952)
    inline double Y(int j) const { return (double)j; }    // y(:,j) = real(j)  (2d_mrlbm.f90:954-956)
    inline int& IP(int r, int m, int k) { return i_p[r][(size_t)m + 4 * (size_t)(k - 1)]; }
    inline int& JP(int r, int m, int k) { return j_p[r][(size_t)m + 4 * (size_t)(k - 1)]; }

    bool setup(const mrlbm_config& c);
    void get_coord();
    void finding_incoming_outgoing_pops();
    void initialize();
    void step();
    void velocity_interpolation_boundary_nodes();
    void moments_interpolation_boundary_nodes();
    void numerical_boundary_cases(int xi, int yj, int label, double uxp, double uyp);
    void numerical_boundary_cases_rotation(int xi, int yj, int label, double uxp, double uyp);
    void numerical_boundary_cases_rotation_weak(int xi, int yj, int label, double uxp, double uyp);
    void numerical_boundary_cases_rotation_rhoeq(int xi, int yj, int label, double uxp, double uyp);
    void apply_bc(int xi, int yj, int bc);
    void apply_bc_incomp(int xi, int yj, int bc);
    void evaluate_forces(int xi, int yj, int label, double& Fx, double& Fy);
};

enum { OUTLET = 0, INLET = 1, TOPWALL = 2, BOTTOMWALL = 3 };

// ---------------------------------------------------------------------------------------
// Setup: 2d_mrlbm.f90:83-214
bool Oracle::setup(const mrlbm_config& c) {
    cfg = c;
    PI = 4.0 * std::atan(1.0);                                      // 2d_mrlbm.f90:4
    cyl = c.channel_with_cylinder != 0;
    if (c.geometry_mode == MRLBM_GEOM_REFERENCE && cyl) {           // 2d_mrlbm.f90:86-92
        int nfront = c.L_front * c.ncy, nback = c.L_back * c.ncy;
        int ntop = c.L_top * c.ncy, nbot = c.L_bot * c.ncy;
        nx = nfront + c.ncy + nback;
        ny = ntop + c.ncy + nbot;
        x_c = (double)(float)(nfront + (c.ncy / 2) + 1);            // 2d_mrlbm.f90:946-948
        y_c = (double)(float)(nbot + c.ncy / 2);
        r_c = (double)(float)(c.ncy / 2);
        const int base = nfront + c.ncy + 1;                        // probes, 2d_mrlbm.f90:102-109
        i_probe[0] = base + (c.ncy / 2); i_probe[1] = base + c.ncy;
        i_probe[2] = base + (3 * c.ncy / 2); i_probe[3] = base + (2 * c.ncy);
        for (int q = 0; q < 4; ++q) j_probe[q] = nbot + (c.ncy / 2) + 1;
    } else {
        nx = c.nx;
        ny = c.ny;
        x_c = c.x_c;
        y_c = c.y_c;
        r_c = c.r_c;
        // extension: probes 1, 1.5, 2 and 2.5 diameters behind the centre, one row above it
        for (int q = 0; q < 4; ++q) {
            i_probe[q] = (int)std::floor(x_c + (1.0 + 0.5 * q) * 2.0 * r_c + 0.5);
            j_probe[q] = (int)std::floor(y_c) + 1;
        }
    }
    for (int q = 0; q < 4; ++q) {                                   // keep probe reads in range
        i_probe[q] = std::min(std::max(i_probe[q], 1), nx);
        j_probe[q] = std::min(std::max(j_probe[q], 1), ny);
    }
    if (nx < 4 || ny < 4) { err = "nx and ny must be >= 4"; return false; }
    const size_t N = (size_t)nx * ny;
    f.assign(N * Q, 0.0); f_tmp.assign(N * Q, 0.0); fout.assign(N * Q, 0.0);
    for (auto* v : {&rho, &p, &ux, &uy, &mxx, &myy, &mxy, &mxxp, &myyp, &mxx_s, &myy_s, &mxy_s,
                    &cth_glb, &sth_glb, &s2th_glb, &c2th_glb})
        v->assign(N, 0.0);
    isfluid.assign(N, 0); issolid.assign(N, 0); isbound.assign(N, 0);
    cx_p.assign(N * Q, 0.0); cy_p.assign(N * Q, 0.0);
    Hxx_p.assign(N * Q, 0.0); Hyy_p.assign(N * Q, 0.0); Hxy_p.assign(N * Q, 0.0);

    if (cyl) get_coord();
    if (!err.empty()) return false;

    // weights and lattice velocities (2d_mrlbm.f90:129-131): single-precision literals
    const float w0 = 16.0f / 36.0f, w1 = 4.0f / 36.0f, w5 = 1.0f / 36.0f;
    const double wl[Q] = {w0, w1, w1, w1, w1, w5, w5, w5, w5};
    const int ex[Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    const int ey[Q] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    for (int k = 0; k < Q; ++k) { w[k] = wl[k]; e[k][0] = ex[k]; e[k][1] = ey[k]; }
    uinlet = c.uo;                                                  // 2d_mrlbm.f90:125-126
    vinlet = 0.0;
    nu = uinlet * (double)(ny - 1) / c.Re;                          // 2d_mrlbm.f90:133
    if (cyl) {
        double L = (c.nu_length == MRLBM_NU_DIAMETER) ? r_c : r_cyl;
        nu = uinlet * (2.0 * L) / c.Re;                             // 2d_mrlbm.f90:134
    }
    omega = 1.0 / ((3.0 * nu) + (1.0 / 2.0));                       // 2d_mrlbm.f90:135
    cs2 = 1.0 / 3.0;                                                // 2d_mrlbm.f90:153
    rho_infty = c.rho_infty;
    for (int k = 0; k < Q; ++k) {                                   // 2d_mrlbm.f90:171-178
        Hxx[k] = (double)(e[k][0] * e[k][0]) - cs2;
        Hyy[k] = (double)(e[k][1] * e[k][1]) - cs2;
        Hxy[k] = (double)(e[k][0] * e[k][1]);
    }
    if (cyl) {                                                      // 2d_mrlbm.f90:183-197
#pragma omp parallel for collapse(2)
        for (int i = 1; i <= nx; ++i)
            for (int j = 1; j <= ny; ++j) {
                const double ct = cth_glb[I(i, j)], st = sth_glb[I(i, j)];
                const double s2 = s2th_glb[I(i, j)], c2 = c2th_glb[I(i, j)];
                for (int k = 0; k < Q; ++k) {
                    const size_t o = F(i, j, k);
                    cx_p[o] = (double)e[k][0] * ct + (double)e[k][1] * st;
                    cy_p[o] = -((double)e[k][0] * st) + (double)e[k][1] * ct;
                    Hxx_p[o] = Hxx[k] * (ct * ct) + Hyy[k] * (st * st) + Hxy[k] * s2;
                    Hyy_p[o] = Hxx[k] * (st * st) + Hyy[k] * (ct * ct) - Hxy[k] * s2;
                    Hxy_p[o] = (Hyy[k] - Hxx[k]) * 0.50 * s2 + Hxy[k] * c2;
                }
            }
    }
    initialize();                                                   // 2d_mrlbm.f90:199-204
    finding_incoming_outgoing_pops();                               // 2d_mrlbm.f90:214
    if (cyl) {
        for (int l = 1; l <= nbct; ++l) {
            int lab = label_bc[l - 1];
            bool any = false;
            for (int k = 0; k < Q; ++k) any = any || Incs_b[lab][k] || Outs_b[lab][k];
            if (!any) {
                char b[160];
                std::snprintf(b, sizeof b, "boundary node %d at (%d,%d) has label %d with empty link rows",
                              l, bou_i[l - 1], bou_j[l - 1], lab);
                err = b;
                return false;
            }
        }
    }
    // restart_step is initialised to 1 (2d_mrlbm.f90:7): a fresh run's first step is iter 2
    iter = 1;
    return true;
}

// get_coord: 2d_mrlbm.f90:931-1156 (the data_geo/theta.dat dumps are not restated)
void Oracle::get_coord() {
    const double epsilon = (double)0.5f;                            // real, parameter (2d_mrlbm.f90:935)
    for (int i = 1; i <= nx; ++i)                                   // 2d_mrlbm.f90:958-966
        for (int j = 1; j <= ny; ++j) {
            double radi = std::sqrt(((X(i) - x_c) * (X(i) - x_c)) + ((Y(j) - y_c) * (Y(j) - y_c)));
            cth_glb[I(i, j)] = (X(i) - x_c) / radi;
            sth_glb[I(i, j)] = (Y(j) - y_c) / radi;
            s2th_glb[I(i, j)] = 2.0 * sth_glb[I(i, j)] * cth_glb[I(i, j)];
            c2th_glb[I(i, j)] = (cth_glb[I(i, j)] * cth_glb[I(i, j)]) - (sth_glb[I(i, j)] * sth_glb[I(i, j)]);
        }
    for (int i = 1; i <= nx; ++i)                                   // 2d_mrlbm.f90:969-980
        for (int j = 1; j <= ny; ++j) {
            double distance = std::sqrt((X(i) - x_c) * (X(i) - x_c) + (Y(j) - y_c) * (Y(j) - y_c));
            if (std::fabs(distance - r_c) <= epsilon) isbound[I(i, j)] = 1;
            else if (std::fabs(distance) <= r_c) issolid[I(i, j)] = 1;
            else isfluid[I(i, j)] = 1;
        }
    for (int i = 2; i <= nx - 1; ++i)                               // 2d_mrlbm.f90:982-1002
        for (int j = 2; j <= ny - 1; ++j) {
            if (isfluid[I(i, j)] == 1) {
                const int ni[9] = {i, i - 1, i, i + 1, i, i - 1, i + 1, i + 1, i - 1};
                const int nj[9] = {j, j, j - 1, j, j + 1, j - 1, j - 1, j + 1, j + 1};
                for (int l = 0; l < Q; ++l) {
                    size_t o = I(ni[l], nj[l]);
                    if (isfluid[o] == 0 && isbound[o] == 0) { isbound[o] = 1; issolid[o] = 0; }
                }
            }
        }
    nbct = 0;                                                       // 2d_mrlbm.f90:1004
    for (size_t o = 0; o < (size_t)nx * ny; ++o) nbct += isbound[o];
    bou_i.assign(nbct, 0); bou_j.assign(nbct, 0); label_bc.assign(nbct, 0);
    radii.assign(nbct, 0); xb.assign(nbct, 0); yb.assign(nbct, 0); delta_uk.assign(nbct, 0);
    theta_c.assign(nbct, 0); thetas_cy.assign(nbct, 0); idx.assign(nbct, 0);
    cth_cyl.assign(nbct, 0); sth_cyl.assign(nbct, 0);
    uxp_b.assign(nbct, 0); uyp_b.assign(nbct, 0); F_drag.assign(nbct, 0); F_lift.assign(nbct, 0);
    for (int r = 1; r <= 4; ++r) { x_ref[r].assign(nbct, 0); y_ref[r].assign(nbct, 0); }
    for (int r = 2; r <= 4; ++r) { i_p[r].assign(4 * (size_t)nbct, 0); j_p[r].assign(4 * (size_t)nbct, 0); }

    int cnt = 1;                                                    // 2d_mrlbm.f90:1007-1036
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            if (isbound[I(i, j)] == 1) {
                if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) {
                    err = "a boundary node lies on the domain edge (label needs all 8 neighbours)";
                    return;
                }
                bou_i[cnt - 1] = i;
                bou_j[cnt - 1] = j;
                int flag0 = 1, flag1 = 1, flag2 = 1, flag3 = 1;
                if (isfluid[I(i - 1, j)] == 0 && isfluid[I(i - 1, j + 1)] == 0 && isfluid[I(i, j + 1)] == 0) flag0 = 0;
                if (isfluid[I(i + 1, j)] == 0 && isfluid[I(i + 1, j + 1)] == 0 && isfluid[I(i, j + 1)] == 0) flag1 = 0;
                if (isfluid[I(i - 1, j)] == 0 && isfluid[I(i - 1, j - 1)] == 0 && isfluid[I(i, j - 1)] == 0) flag2 = 0;
                if (isfluid[I(i + 1, j)] == 0 && isfluid[I(i + 1, j - 1)] == 0 && isfluid[I(i, j - 1)] == 0) flag3 = 0;
                label_bc[cnt - 1] = flag0 * 1 + flag1 * 2 + flag2 * 4 + flag3 * 8;
                ++cnt;
            }
        }
    for (int k = 1; k <= nbct; ++k) {                               // 2d_mrlbm.f90:1038-1050
        int i = bou_i[k - 1], j = bou_j[k - 1];
        radii[k - 1] = std::sqrt(((X(i) - x_c) * (X(i) - x_c)) + ((Y(j) - y_c) * (Y(j) - y_c)));
    }
    double max_radii = nbct > 0 ? radii[0] : 0.0;
    for (int k = 2; k <= nbct; ++k)
        if (radii[k - 1] > max_radii) max_radii = radii[k - 1];
    r_cyl = max_radii;

    delx = std::sqrt(2.0);                                          // 2d_mrlbm.f90:1055
    for (int k = 1; k <= nbct; ++k) {                               // 2d_mrlbm.f90:1056-1135
        const int bi = bou_i[k - 1], bj = bou_j[k - 1];
        double rr = std::sqrt((X(bi) - x_c) * (X(bi) - x_c) + (Y(bj) - y_c) * (Y(bj) - y_c));
        double unit_nx, unit_ny;
        if (rr > 1.0e-12) {
            unit_nx = (X(bi) - x_c) / rr;
            unit_ny = (Y(bj) - y_c) / rr;
            xb[k - 1] = x_c + (r_cyl * unit_nx);
            yb[k - 1] = y_c + (r_cyl * unit_ny);
        } else {
            unit_nx = 0.0;
            unit_ny = 0.0;
            xb[k - 1] = x_c;
            yb[k - 1] = y_c;
        }
        cth_cyl[k - 1] = unit_nx;
        sth_cyl[k - 1] = unit_ny;
        x_ref[1][k - 1] = xb[k - 1];
        y_ref[1][k - 1] = yb[k - 1];
        x_ref[2][k - 1] = xb[k - 1] + (delx * unit_nx);
        y_ref[2][k - 1] = yb[k - 1] + (delx * unit_ny);
        x_ref[3][k - 1] = xb[k - 1] + (2.0 * delx * unit_nx);
        y_ref[3][k - 1] = yb[k - 1] + (2.0 * delx * unit_ny);
        x_ref[4][k - 1] = xb[k - 1] + (3.0 * delx * unit_nx);
        y_ref[4][k - 1] = yb[k - 1] + (3.0 * delx * unit_ny);
        double delta_x = X(bi) - xb[k - 1];
        double delta_y = Y(bj) - yb[k - 1];
        delta_uk[k - 1] = std::sqrt(delta_x * delta_x + delta_y * delta_y);
        for (int r = 2; r <= 4; ++r) {                              // 2d_mrlbm.f90:1099-1129
            int fx = (int)std::floor(x_ref[r][k - 1]);
            int fy = (int)std::floor(y_ref[r][k - 1]);
            IP(r, 0, k) = fx;     JP(r, 0, k) = fy;
            IP(r, 1, k) = fx + 1; JP(r, 1, k) = fy;
            IP(r, 2, k) = fx;     JP(r, 2, k) = fy + 1;
            IP(r, 3, k) = fx + 1; JP(r, 3, k) = fy + 1;
        }
        theta_c[k - 1] = std::atan2(yb[k - 1] - y_c, xb[k - 1] - x_c);   // 2d_mrlbm.f90:1132-1133
        if (theta_c[k - 1] < 0) theta_c[k - 1] = theta_c[k - 1] + 2.0 * PI;
    }
    for (int i = 1; i <= nbct; ++i) idx[i - 1] = i;                // 2d_mrlbm.f90:1139-1156
    for (int i = 1; i <= nbct - 1; ++i)
        for (int j = i + 1; j <= nbct; ++j)
            if (theta_c[idx[i - 1] - 1] > theta_c[idx[j - 1] - 1]) {
                int temp = idx[i - 1]; idx[i - 1] = idx[j - 1]; idx[j - 1] = temp;
            }
    for (int i = 1; i <= nbct; ++i) thetas_cy[i - 1] = theta_c[idx[i - 1] - 1];

    // The parallel boundary kernels rely on these two properties of the geometry, which
    // the serial reference loop does not need: every bilinear stencil node is an interior
    // fluid node.  Checked here so a violating case fails in the oracle too.
    for (int k = 1; k <= nbct; ++k)
        for (int r = 2; r <= 4; ++r)
            for (int m = 0; m < 4; ++m) {
                int si = IP(r, m, k), sj = JP(r, m, k);
                if (si < 2 || si > nx - 1 || sj < 2 || sj > ny - 1 || isfluid[I(si, sj)] != 1) {
                    char b[200];
                    std::snprintf(b, sizeof b, "stencil node (%d,%d) of boundary node %d is not an interior fluid node",
                                  si, sj, k);
                    err = b;
                    return;
                }
            }
}

// finding_incoming_outgoing_pops: 2d_mrlbm.f90:2005-2057 (Incs_f/Outs_f are unused there)
void Oracle::finding_incoming_outgoing_pops() {
    std::memset(Incs_b, 0, sizeof Incs_b);
    std::memset(Outs_b, 0, sizeof Outs_b);
    static const int tab[][2][Q] = {
        {{1, 1, 0, 0, 1, 0, 0, 0, 1}, {1, 0, 1, 1, 0, 0, 1, 0, 0}},   // 1
        {{1, 0, 0, 1, 1, 0, 0, 1, 0}, {1, 1, 1, 0, 0, 1, 0, 0, 0}},   // 2
        {{1, 1, 0, 1, 1, 0, 0, 1, 1}, {1, 1, 1, 1, 0, 1, 1, 0, 0}},   // 3
        {{1, 1, 1, 0, 0, 1, 0, 0, 0}, {1, 0, 0, 1, 1, 0, 0, 1, 0}},   // 4
        {{1, 1, 1, 0, 1, 1, 0, 0, 1}, {1, 0, 1, 1, 1, 0, 1, 1, 0}},   // 5
        {{1, 1, 1, 1, 1, 1, 0, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1, 0}},   // 7
        {{1, 0, 1, 1, 0, 0, 1, 0, 0}, {1, 1, 0, 0, 1, 0, 0, 0, 1}},   // 8
        {{1, 0, 1, 1, 1, 0, 1, 1, 0}, {1, 1, 1, 0, 1, 1, 0, 0, 1}},   // 10
        {{1, 1, 1, 1, 1, 0, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 0, 1}},   // 11
        {{1, 1, 1, 1, 0, 1, 1, 0, 0}, {1, 1, 0, 1, 1, 0, 0, 1, 1}},   // 12
        {{1, 1, 1, 1, 1, 1, 1, 0, 1}, {1, 1, 1, 1, 1, 0, 1, 1, 1}},   // 13
        {{1, 1, 1, 1, 1, 1, 1, 1, 0}, {1, 1, 1, 1, 1, 1, 0, 1, 1}},   // 14
    };
    static const int labels[] = {1, 2, 3, 4, 5, 7, 8, 10, 11, 12, 13, 14};
    for (int r = 0; r < 12; ++r)
        for (int k = 0; k < Q; ++k) {
            Incs_b[labels[r]][k] = tab[r][0][k];
            Outs_b[labels[r]][k] = tab[r][1][k];
        }
    if (cfg.label15_rule == MRLBM_LABEL15_ALLNINE)
        for (int k = 0; k < Q; ++k) { Incs_b[15][k] = 1; Outs_b[15][k] = 1; }
}

// initialize: 2d_mrlbm.f90:199-204, 1220-1235; INIT_NOISE extension
void Oracle::initialize() {
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            if (cfg.init_mode == MRLBM_INIT_NOISE) {
                const uint64_t n = (uint64_t)I(i, j);
                double r = 1.0;
                double u = uinlet + cfg.noise_amp * uinlet * normal_noise(cfg.seed, n, 0);
                double v = cfg.noise_amp * uinlet * normal_noise(cfg.seed, n, 1);
                double m_xx = u * u, m_yy = v * v, m_xy = u * v;
                rho[I(i, j)] = r; ux[I(i, j)] = u; uy[I(i, j)] = v;
                for (int k = 0; k < Q; ++k) {
                    double cu = (double)e[k][0] * u + (double)e[k][1] * v;
                    f[F(i, j, k)] = w[k] * r * (1.0 + (3.0 * cu) + 4.50 * m_xx * Hxx[k] +
                                                4.50 * m_yy * Hyy[k] + 9.00 * m_xy * Hxy[k]);
                }
            } else {
                rho[I(i, j)] = 1.0;
                ux[I(i, j)] = 0.0;
                uy[I(i, j)] = 0.0;
                for (int k = 0; k < Q; ++k) f[F(i, j, k)] = w[k] * rho[I(i, j)];
            }
        }
}

// velocity_interpolation_boundary_nodes: 2d_mrlbm.f90:768-819
void Oracle::velocity_interpolation_boundary_nodes() {
    for (int k = 1; k <= nbct; ++k) {
        const int i = bou_i[k - 1], j = bou_j[k - 1];
        const double ux_ref1 = 0.0, uy_ref1 = 0.0;
        double ref_ux[4], ref_uy[4];
        for (int r = 2; r <= 3; ++r) {
            double xd = (x_ref[r][k - 1] - X(IP(r, 0, k))) / dx;
            double yd = (y_ref[r][k - 1] - Y(JP(r, 0, k))) / dy;
            size_t p1 = I(IP(r, 0, k), JP(r, 0, k)), p2 = I(IP(r, 1, k), JP(r, 1, k));
            size_t p3 = I(IP(r, 2, k), JP(r, 2, k)), p4 = I(IP(r, 3, k), JP(r, 3, k));
            double ux_0 = (1.0 - xd) * ux[p1] + xd * ux[p2];
            double uy_0 = (1.0 - xd) * uy[p1] + xd * uy[p2];
            double ux_1 = (1.0 - xd) * ux[p3] + xd * ux[p4];
            double uy_1 = (1.0 - xd) * uy[p3] + xd * uy[p4];
            ref_ux[r] = (1.0 - yd) * ux_0 + yd * ux_1;
            ref_uy[r] = (1.0 - yd) * uy_0 + yd * uy_1;
        }
        const double d = delta_uk[k - 1];
        double term1 = (2.0 * delx * delx - (d * d) + 3.0 * d * delx) / (2.0 * (delx * delx));
        double term2 = d * (d - 2.0 * delx) / (delx * delx);
        double term3 = d * (d - delx) / (2.0 * (delx * delx));
        ux[I(i, j)] = term1 * ux_ref1 + term2 * ref_ux[2] - term3 * ref_ux[3];
        uy[I(i, j)] = term1 * uy_ref1 + term2 * ref_uy[2] - term3 * ref_uy[3];
    }
}

// moments_interpolation_boundary_nodes: 2d_mrlbm.f90:821-928
void Oracle::moments_interpolation_boundary_nodes() {
    for (int k = 1; k <= nbct; ++k) {
        const int i = bou_i[k - 1], j = bou_j[k - 1];
        const double mxxp_ref1 = 0.0, myyp_ref1 = 0.0;
        double ref_mxx[4], ref_myy[4];
        for (int r = 2; r <= 3; ++r) {
            double xd = (x_ref[r][k - 1] - X(IP(r, 0, k))) / dx;
            double yd = (y_ref[r][k - 1] - Y(JP(r, 0, k))) / dy;
            double mxxpv[4], myypv[4];
            for (int m = 0; m < 4; ++m) {
                size_t o = I(IP(r, m, k), JP(r, m, k));
                const double c = cth_glb[o], s = sth_glb[o], s2 = s2th_glb[o];
                mxxpv[m] = mxx[o] * (c * c) + myy[o] * (s * s) + mxy[o] * s2;
                myypv[m] = mxx[o] * (s * s) + myy[o] * (c * c) - mxy[o] * s2;
            }
            double mxx_0 = (1.0 - xd) * mxxpv[0] + xd * mxxpv[1];
            double myy_0 = (1.0 - xd) * myypv[0] + xd * myypv[1];
            double mxx_1 = (1.0 - xd) * mxxpv[2] + xd * mxxpv[3];
            double myy_1 = (1.0 - xd) * myypv[2] + xd * myypv[3];
            ref_mxx[r] = (1.0 - yd) * mxx_0 + yd * mxx_1;
            ref_myy[r] = (1.0 - yd) * myy_0 + yd * myy_1;
        }
        const double d = delta_uk[k - 1];
        double term1 = (2.0 * delx * delx - (d * d) + 3.0 * d * delx) / (2.0 * (delx * delx));
        double term2 = d * (d - 2.0 * delx) / (delx * delx);
        double term3 = d * (d - delx) / (2.0 * (delx * delx));
        mxxp[I(i, j)] = term1 * mxxp_ref1 + term2 * ref_mxx[2] - term3 * ref_mxx[3];
        myyp[I(i, j)] = term1 * myyp_ref1 + term2 * ref_myy[2] - term3 * ref_myy[3];
    }
}

// solve_system: 2d_mrlbm.f90:1974-2003 (Cramer's rule on the 3x3 system)
static void solve_system(const double A[3][3], const double b[3], double& x_11, double& x_22, double& x_12) {
    double a1 = A[0][0], b1 = A[0][1], c1 = A[0][2], d1 = b[0];
    double a2 = A[1][0], b2 = A[1][1], c2 = A[1][2], d2 = b[1];
    double a3 = A[2][0], b3 = A[2][1], c3 = A[2][2], d3 = b[2];
    double denom = a3 * b2 * c1 - a2 * b3 * c1 - a3 * b1 * c2 + a1 * b3 * c2 + a2 * b1 * c3 - a1 * b2 * c3;
    x_11 = -((-b3 * c2 * d1 + b2 * c3 * d1 + b3 * c1 * d2 - b1 * c3 * d2 - b2 * c1 * d3 + b1 * c2 * d3) / denom);
    x_22 = -((a3 * c2 * d1 - a2 * c3 * d1 - a3 * c1 * d2 + a1 * c3 * d2 + a2 * c1 * d3 - a1 * c2 * d3) / denom);
    x_12 = -((-a3 * b2 * d1 + a2 * b3 * d1 + a3 * b1 * d2 - a1 * b3 * d2 - a2 * b1 * d3 + a1 * b2 * d3) / denom);
}

// numerical_boundary_cases (unrotated): 2d_mrlbm.f90:1496-1633
void Oracle::numerical_boundary_cases(int xi, int yj, int label, double uxp, double uyp) {
    const int* Is = Incs_b[label];
    const int* Os = Outs_b[label];
    double A_i[Q], E_i[Q], B11_i[Q], B22_i[Q], B12_i[Q];
    for (int k = 0; k < Q; ++k) {
        A_i[k] = w[k] * (1.0 + 3.0 * uxp * e[k][0] + 3.0 * uyp * e[k][1]);
        E_i[k] = w[k] * (1.0 + 3.0 * uxp * e[k][0] + 3.0 * uyp * e[k][1] + 4.50 * (uxp * uxp) * Hxx[k] +
                         4.50 * (uyp * uyp) * Hyy[k] + 9.0 * (uxp * uyp) * Hxy[k]);
        B11_i[k] = 4.50 * w[k] * Hxx[k];
        B22_i[k] = 4.50 * w[k] * Hyy[k];
        B12_i[k] = 4.50 * w[k] * Hxy[k];
    }
    double rhoI_b = 0, mxxI_b = 0, myyI_b = 0, mxyI_b = 0, A_prime = 0, E_prime = 0;
    double B11_prime = 0, B22_prime = 0, B12_prime = 0, D_xx = 0, D_yy = 0, D_xy = 0;
    double F11_xx = 0, F12_xx = 0, F22_xx = 0, F11_yy = 0, F12_yy = 0, F22_yy = 0;
    double F11_xy = 0, F12_xy = 0, F22_xy = 0;
    for (int k = 0; k < Q; ++k) {
        if (Os[k] == 1) {
            A_prime = A_prime + A_i[k];
            E_prime = E_prime + E_i[k];
            B11_prime = B11_prime + B11_i[k];
            B22_prime = B22_prime + B22_i[k];
            B12_prime = B12_prime + B12_i[k];
        }
        if (Is[k] == 1) {
            const double fk = f[F(xi, yj, k)];
            rhoI_b = rhoI_b + fk;
            mxxI_b = mxxI_b + fk * Hxx[k];
            myyI_b = myyI_b + fk * Hyy[k];
            mxyI_b = mxyI_b + fk * Hxy[k];
            D_xx = D_xx + A_i[k] * Hxx[k];
            D_yy = D_yy + A_i[k] * Hyy[k];
            D_xy = D_xy + A_i[k] * Hxy[k];
            F11_xx = F11_xx + B11_i[k] * Hxx[k];
            F22_xx = F22_xx + B22_i[k] * Hxx[k];
            F12_xx = F12_xx + B12_i[k] * Hxx[k];
            F11_yy = F11_yy + B11_i[k] * Hyy[k];
            F22_yy = F22_yy + B22_i[k] * Hyy[k];
            F12_yy = F12_yy + B12_i[k] * Hyy[k];
            F11_xy = F11_xy + B11_i[k] * Hxy[k];
            F22_xy = F22_xy + B22_i[k] * Hxy[k];
            F12_xy = F12_xy + B12_i[k] * Hxy[k];
        }
    }
    double inv_rhoIb = 1.0 / rhoI_b;
    mxxI_b = mxxI_b * inv_rhoIb;
    myyI_b = myyI_b * inv_rhoIb;
    mxyI_b = mxyI_b * inv_rhoIb;
    double G_prime = (1.0 - omega) * A_prime + omega * E_prime;
    double J11 = (1.0 - omega) * B11_prime, J22 = (1.0 - omega) * B22_prime, J12 = (1.0 - omega) * B12_prime;
    double J11_xx = J11 * mxxI_b, J22_xx = J22 * mxxI_b, J12_xx = J12 * mxxI_b;
    double J11_yy = J11 * myyI_b, J22_yy = J22 * myyI_b, J12_yy = J12 * myyI_b;
    double J11_xy = J11 * mxyI_b, J22_xy = J22 * mxyI_b, J12_xy = J12 * mxyI_b;
    double L_11_xx = J11_xx - F11_xx, L_11_yy = J11_yy - F11_yy, L_11_xy = J11_xy - F11_xy;
    double L_22_xx = J22_xx - F22_xx, L_22_yy = J22_yy - F22_yy, L_22_xy = J22_xy - F22_xy;
    double L_12_xx = 2.0 * (J12_xx - F12_xx), L_12_yy = 2.0 * (J12_yy - F12_yy), L_12_xy = 2.0 * (J12_xy - F12_xy);
    double R_xx = D_xx - G_prime * mxxI_b, R_yy = D_yy - G_prime * myyI_b, R_xy = D_xy - G_prime * mxyI_b;
    const double A[3][3] = {{L_11_xx, L_22_xx, L_12_xx}, {L_11_yy, L_22_yy, L_12_yy}, {L_11_xy, L_22_xy, L_12_xy}};
    const double b[3] = {R_xx, R_yy, R_xy};
    double Mxx, Myy, Mxy;
    solve_system(A, b, Mxx, Myy, Mxy);
    double denominator = (1.0 - omega) * A_prime +
                         (1.0 - omega) * (Mxx * B11_prime + Myy * B22_prime + 2.0 * Mxy * B12_prime) + omega * E_prime;
    double rho_prime_b = rhoI_b / denominator;
    rho[I(xi, yj)] = rho_prime_b;
    mxx[I(xi, yj)] = Mxx;
    myy[I(xi, yj)] = Myy;
    mxy[I(xi, yj)] = Mxy;
}

// numerical_boundary_cases_rotation: 2d_mrlbm.f90:1635-1765 (the default closure)
void Oracle::numerical_boundary_cases_rotation(int xi, int yj, int label, double uxp, double uyp) {
    const int* Is = Incs_b[label];
    const int* Os = Outs_b[label];
    double A_i[Q], E_i[Q], B11_i[Q], B22_i[Q], B12_i[Q];
    for (int k = 0; k < Q; ++k) {
        const size_t o = F(xi, yj, k);
        A_i[k] = w[k] * (1.0 + 3.0 * uxp * cx_p[o] + 3.0 * uyp * cy_p[o]);
        E_i[k] = w[k] * (1.0 + 3.0 * uxp * cx_p[o] + 3.0 * uyp * cy_p[o] + 4.50 * (uxp * uxp) * Hxx_p[o] +
                         4.50 * (uyp * uyp) * Hyy_p[o] + 9.0 * (uxp * uyp) * Hxy_p[o]);
        B11_i[k] = 4.50 * w[k] * Hxx_p[o];
        B22_i[k] = 4.50 * w[k] * Hyy_p[o];
        B12_i[k] = 4.50 * w[k] * Hxy_p[o];
    }
    double rhoI_b = 0, mxxI_b = 0, myyI_b = 0, mxyI_b = 0, A_prime = 0, E_prime = 0;
    double B11_prime = 0, B22_prime = 0, B12_prime = 0, D_xx = 0, D_yy = 0, D_xy = 0;
    double F11_xx = 0, F12_xx = 0, F22_xx = 0, F11_yy = 0, F12_yy = 0, F22_yy = 0;
    double F11_xy = 0, F12_xy = 0, F22_xy = 0;
    for (int k = 0; k < Q; ++k) {
        const size_t o = F(xi, yj, k);
        if (Os[k] == 1) {
            A_prime = A_prime + A_i[k];
            E_prime = E_prime + E_i[k];
            B11_prime = B11_prime + B11_i[k];
            B22_prime = B22_prime + B22_i[k];
            B12_prime = B12_prime + B12_i[k];
        }
        if (Is[k] == 1) {
            const double fk = f[o];
            rhoI_b = rhoI_b + fk;
            mxxI_b = mxxI_b + fk * Hxx_p[o];
            myyI_b = myyI_b + fk * Hyy_p[o];
            mxyI_b = mxyI_b + fk * Hxy_p[o];
            D_xx = D_xx + A_i[k] * Hxx_p[o];
            D_yy = D_yy + A_i[k] * Hyy_p[o];
            D_xy = D_xy + A_i[k] * Hxy_p[o];
            F11_xx = F11_xx + B11_i[k] * Hxx_p[o];
            F22_xx = F22_xx + B22_i[k] * Hxx_p[o];
            F12_xx = F12_xx + B12_i[k] * Hxx_p[o];
            F11_yy = F11_yy + B11_i[k] * Hyy_p[o];
            F22_yy = F22_yy + B22_i[k] * Hyy_p[o];
            F12_yy = F12_yy + B12_i[k] * Hyy_p[o];
            F11_xy = F11_xy + B11_i[k] * Hxy_p[o];
            F22_xy = F22_xy + B22_i[k] * Hxy_p[o];
            F12_xy = F12_xy + B12_i[k] * Hxy_p[o];
        }
    }
    double inv_rhoIb = 1.0 / rhoI_b;
    mxxI_b = mxxI_b * inv_rhoIb;
    myyI_b = myyI_b * inv_rhoIb;
    mxyI_b = mxyI_b * inv_rhoIb;
    double G_prime = (1.0 - omega) * A_prime + omega * E_prime;
    double J11 = (1.0 - omega) * B11_prime, J22 = (1.0 - omega) * B22_prime, J12 = (1.0 - omega) * B12_prime;
    double J11_xy = J11 * mxyI_b, J22_xy = J22 * mxyI_b, J12_xy = J12 * mxyI_b;
    double L_11_xy = J11_xy - F11_xy;
    double L_22_xy = J22_xy - F22_xy;
    double L_12_xy = 2.0 * (J12_xy - F12_xy);
    double R_xy = D_xy - G_prime * mxyI_b;
    (void)F11_xx; (void)F12_xx; (void)F22_xx; (void)F11_yy; (void)F12_yy; (void)F22_yy; (void)D_xx; (void)D_yy;
    double Mxx = mxxp[I(xi, yj)];
    double Myy = myyp[I(xi, yj)];
    double Mxy = (R_xy - Mxx * L_11_xy - Myy * L_22_xy) / L_12_xy;
    double denominator = (1.0 - omega) * A_prime +
                         (1.0 - omega) * (Mxx * B11_prime + Myy * B22_prime + 2.0 * Mxy * B12_prime) + omega * E_prime;
    double rho_prime_b = rhoI_b / denominator;
    const size_t n = I(xi, yj);
    const double c = cth_glb[n], s = sth_glb[n], s2 = s2th_glb[n], c2 = c2th_glb[n];
    rho[n] = rho_prime_b;
    mxx[n] = Mxx * (c * c) + Myy * (s * s) - Mxy * s2;
    myy[n] = Mxx * (s * s) + Myy * (c * c) + Mxy * s2;
    mxy[n] = (Mxx - Myy) * 0.50 * s2 + Mxy * c2;
}

// numerical_boundary_cases_rotation_weak: 2d_mrlbm.f90:1767-1871
void Oracle::numerical_boundary_cases_rotation_weak(int xi, int yj, int label, double uxp, double uyp) {
    const int* Is = Incs_b[label];
    double A_i[Q], B11_i[Q], B22_i[Q], B12_i[Q];
    for (int k = 0; k < Q; ++k) {
        const size_t o = F(xi, yj, k);
        A_i[k] = w[k] * (1.0 + 3.0 * uxp * cx_p[o] + 3.0 * uyp * cy_p[o]);
        B11_i[k] = 4.50 * w[k] * Hxx_p[o];
        B22_i[k] = 4.50 * w[k] * Hyy_p[o];
        B12_i[k] = 4.50 * w[k] * Hxy_p[o];
    }
    double rhoI_b = 0, mxxI_b = 0, myyI_b = 0, mxyI_b = 0, A_prime = 0;
    double B11_prime = 0, B22_prime = 0, B12_prime = 0, D_xy = 0;
    double F11_xy = 0, F12_xy = 0, F22_xy = 0;
    for (int k = 0; k < Q; ++k) {
        const size_t o = F(xi, yj, k);
        if (Is[k] == 1) {
            const double fk = f[o];
            rhoI_b = rhoI_b + fk;
            mxxI_b = mxxI_b + fk * Hxx_p[o];
            myyI_b = myyI_b + fk * Hyy_p[o];
            mxyI_b = mxyI_b + fk * Hxy_p[o];
            A_prime = A_prime + A_i[k];
            B11_prime = B11_prime + B11_i[k];
            B22_prime = B22_prime + B22_i[k];
            B12_prime = B12_prime + B12_i[k];
            D_xy = D_xy + A_i[k] * Hxy_p[o];
            F11_xy = F11_xy + B11_i[k] * Hxy_p[o];
            F22_xy = F22_xy + B22_i[k] * Hxy_p[o];
            F12_xy = F12_xy + B12_i[k] * Hxy_p[o];
        }
    }
    double inv_rhoIb = 1.0 / rhoI_b;
    mxxI_b = mxxI_b * inv_rhoIb;
    myyI_b = myyI_b * inv_rhoIb;
    mxyI_b = mxyI_b * inv_rhoIb;
    double L_11_xy = B11_prime * mxyI_b - F11_xy;
    double L_22_xy = B22_prime * mxyI_b - F22_xy;
    double L_12_xy = 2.0 * (B12_prime * mxyI_b - F12_xy);
    double R_xy = D_xy - A_prime * mxyI_b;
    double Mxx = mxxp[I(xi, yj)];
    double Myy = myyp[I(xi, yj)];
    double Mxy = (R_xy - Mxx * L_11_xy - Myy * L_22_xy) / L_12_xy;
    double denominator = A_prime + (Mxx * B11_prime + Myy * B22_prime + 2.0 * Mxy * B12_prime);
    double rho_prime_b = rhoI_b / denominator;
    const size_t n = I(xi, yj);
    const double c = cth_glb[n], s = sth_glb[n], s2 = s2th_glb[n], c2 = c2th_glb[n];
    rho[n] = rho_prime_b;
    mxx[n] = Mxx * (c * c) + Myy * (s * s) - Mxy * s2;
    myy[n] = Mxx * (s * s) + Myy * (c * c) + Mxy * s2;
    mxy[n] = (Mxx - Myy) * 0.50 * s2 + Mxy * c2;
}

// numerical_boundary_cases_rotation_rhoeq: 2d_mrlbm.f90:1873-1972
void Oracle::numerical_boundary_cases_rotation_rhoeq(int xi, int yj, int label, double uxp, double uyp) {
    const int* Is = Incs_b[label];
    double A_i[Q], E_i[Q], B11_i[Q], B22_i[Q], B12_i[Q];
    for (int k = 0; k < Q; ++k) {
        const size_t o = F(xi, yj, k);
        A_i[k] = w[k] * (1.0 + 3.0 * uxp * cx_p[o] + 3.0 * uyp * cy_p[o]);
        E_i[k] = w[k] * (1.0 + 3.0 * uxp * cx_p[o] + 3.0 * uyp * cy_p[o] + 4.50 * (uxp * uxp) * Hxx_p[o] +
                         4.50 * (uyp * uyp) * Hyy_p[o] + 9.0 * (uxp * uyp) * Hxy_p[o]);
        B11_i[k] = 4.50 * w[k] * Hxx_p[o];
        B22_i[k] = 4.50 * w[k] * Hyy_p[o];
        B12_i[k] = 4.50 * w[k] * Hxy_p[o];
    }
    double rhoI_b = 0, mxxI_b = 0, myyI_b = 0, mxyI_b = 0, E_prime = 0, D_xy = 0;
    double F11_xy = 0, F12_xy = 0, F22_xy = 0;
    for (int k = 0; k < Q; ++k) {
        const size_t o = F(xi, yj, k);
        if (Is[k] == 1) {
            const double fk = f[o];
            rhoI_b = rhoI_b + fk;
            mxxI_b = mxxI_b + fk * Hxx_p[o];
            myyI_b = myyI_b + fk * Hyy_p[o];
            mxyI_b = mxyI_b + fk * Hxy_p[o];
            E_prime = E_prime + E_i[k];
            D_xy = D_xy + A_i[k] * Hxy_p[o];
            F11_xy = F11_xy + B11_i[k] * Hxy_p[o];
            F22_xy = F22_xy + B22_i[k] * Hxy_p[o];
            F12_xy = F12_xy + B12_i[k] * Hxy_p[o];
        }
    }
    double inv_rhoIb = 1.0 / rhoI_b;
    mxxI_b = mxxI_b * inv_rhoIb;
    myyI_b = myyI_b * inv_rhoIb;
    mxyI_b = mxyI_b * inv_rhoIb;
    double L_11_xy = F11_xy, L_22_xy = F22_xy, L_12_xy = 2.0 * F12_xy;
    double R_xy = E_prime * mxyI_b - D_xy;
    double Mxx = mxxp[I(xi, yj)];
    double Myy = myyp[I(xi, yj)];
    double Mxy = (R_xy - Mxx * L_11_xy - Myy * L_22_xy) / L_12_xy;
    double rho_prime_b = rhoI_b / E_prime;
    const size_t n = I(xi, yj);
    const double c = cth_glb[n], s = sth_glb[n], s2 = s2th_glb[n], c2 = c2th_glb[n];
    rho[n] = rho_prime_b;
    mxx[n] = Mxx * (c * c) + Myy * (s * s) - Mxy * s2;
    myy[n] = Mxx * (s * s) + Myy * (c * c) + Mxy * s2;
    mxy[n] = (Mxx - Myy) * 0.50 * s2 + Mxy * c2;
}

// incoming sums over a fixed mask (shared prologue of apply_bc / apply_bc_incomp)
static inline void incoming_moments(const double* fk, const int* Is, const double* Hxx, const double* Hyy,
                                    const double* Hxy, double& rhoI, double& mxxI, double& myyI, double& mxyI) {
    rhoI = 0.0; mxxI = 0.0; myyI = 0.0; mxyI = 0.0;
    for (int k = 0; k < Q; ++k)
        if (Is[k] == 1) {
            rhoI = rhoI + fk[k];
            mxxI = mxxI + fk[k] * Hxx[k];
            myyI = myyI + fk[k] * Hyy[k];
            mxyI = mxyI + fk[k] * Hxy[k];
        }
    double inv = 1.0 / rhoI;
    mxxI = mxxI * inv;
    myyI = myyI * inv;
    mxyI = mxyI * inv;
}

static const int IS_OUTLET[Q] = {1, 1, 1, 0, 1, 1, 0, 0, 1};
static const int IS_INLET[Q] = {1, 0, 1, 1, 1, 0, 1, 1, 0};
static const int IS_TOP[Q] = {1, 1, 1, 1, 0, 1, 1, 0, 0};
static const int IS_BOTTOM[Q] = {1, 1, 0, 1, 1, 0, 0, 1, 1};

// apply_bc: 2d_mrlbm.f90:1237-1366
void Oracle::apply_bc(int xi, int yj, int bc) {
    double fk[Q];
    for (int k = 0; k < Q; ++k) fk[k] = f[F(xi, yj, k)];
    const size_t n = I(xi, yj);
    double rhoI_b, mxxI_b, myyI_b, mxyI_b, rho_prime_b;
    switch (bc) {
    case OUTLET:
        incoming_moments(fk, IS_OUTLET, Hxx, Hyy, Hxy, rhoI_b, mxxI_b, myyI_b, mxyI_b);
        rho_prime_b = rho[n];
        mxx[n] = (rho_prime_b + 9.0 * rhoI_b * mxxI_b - 3.0 * rho_prime_b * ux[n]) / (6.0 * rho_prime_b);
        myy[n] = 6.0 * rhoI_b * myyI_b / (5.0 * rho_prime_b);
        mxy[n] = (6.0 * rhoI_b * mxyI_b - rho_prime_b * uy[n]) / (3.0 * rho_prime_b);
        break;
    case INLET:
        incoming_moments(fk, IS_INLET, Hxx, Hyy, Hxy, rhoI_b, mxxI_b, myyI_b, mxyI_b);
        rho[n] = (4.0 * rhoI_b + 3.0 * rhoI_b * mxxI_b) / (3.0 - 3.0 * ux[n]);
        rho_prime_b = rho[n];
        mxx[n] = (rho_prime_b + 9.0 * rhoI_b * mxxI_b + 3.0 * rho_prime_b * ux[n]) / (6.0 * rho_prime_b);
        myy[n] = 6.0 * rhoI_b * myyI_b / (5.0 * rho_prime_b);
        mxy[n] = 2.0 * rhoI_b * mxyI_b / rho_prime_b;
        break;
    case TOPWALL:
    case BOTTOMWALL:
        incoming_moments(fk, bc == TOPWALL ? IS_TOP : IS_BOTTOM, Hxx, Hyy, Hxy, rhoI_b, mxxI_b, myyI_b, mxyI_b);
        rho[n] = 3.0 * rhoI_b * (4.0 + 3.0 * (1.0 - omega) * myyI_b) / (9.0 + omega);
        rho_prime_b = rho[n];
        mxx[n] = 6.0 * rhoI_b * mxxI_b / (5.0 * rho_prime_b);
        myy[n] = (rho_prime_b + 9.0 * rhoI_b * myyI_b) / (6.0 * rho_prime_b);
        mxy[n] = 2.0 * rhoI_b * mxyI_b / rho_prime_b;
        break;
    }
}

// apply_bc_incomp: 2d_mrlbm.f90:1368-1494
void Oracle::apply_bc_incomp(int xi, int yj, int bc) {
    double fk[Q];
    for (int k = 0; k < Q; ++k) fk[k] = f[F(xi, yj, k)];
    const size_t n = I(xi, yj);
    double rhoI_b, mxxI_b, myyI_b, mxyI_b, rho_prime_b;
    switch (bc) {
    case OUTLET:
        incoming_moments(fk, IS_OUTLET, Hxx, Hyy, Hxy, rhoI_b, mxxI_b, myyI_b, mxyI_b);
        rho_prime_b = rho[n];
        mxx[n] = ux[n] * ux[n];
        myy[n] = uy[n] * uy[n];
        mxy[n] = (6.0 * rhoI_b * mxyI_b - rho_prime_b * uy[n]) / (3.0 * rho_prime_b);
        break;
    case INLET:
        incoming_moments(fk, IS_INLET, Hxx, Hyy, Hxy, rhoI_b, mxxI_b, myyI_b, mxyI_b);
        rho[n] = 6.0 * rhoI_b / (5.0 - 3.0 * ux[n] - 3.0 * (ux[n] * ux[n]));
        rho_prime_b = rho[n];
        mxx[n] = ux[n] * ux[n];
        myy[n] = 0.0;
        mxy[n] = 2.0 * rhoI_b * mxyI_b / rho_prime_b;
        break;
    case TOPWALL:
    case BOTTOMWALL:
        incoming_moments(fk, bc == TOPWALL ? IS_TOP : IS_BOTTOM, Hxx, Hyy, Hxy, rhoI_b, mxxI_b, myyI_b, mxyI_b);
        rho[n] = 6.0 * rhoI_b / 5.0;
        mxx[n] = 0.0;
        myy[n] = 0.0;
        mxy[n] = 5.0 * mxyI_b / 3.0;
        break;
    }
}

// evaluate_forces: 2d_mrlbm.f90:558-591
void Oracle::evaluate_forces(int xi, int yj, int label, double& Fx, double& Fy) {
    const int* Is = Incs_b[label];
    const int* Os = Outs_b[label];
    double Fx_inc = 0.0, Fy_inc = 0.0, Fx_out = 0.0, Fy_out = 0.0;
    for (int k = 0; k < Q; ++k) {
        if (Os[k] == 1) {
            Fx_out = Fx_out + fout[F(xi, yj, k)] * e[k][0];
            Fy_out = Fy_out + fout[F(xi, yj, k)] * e[k][1];
        }
        if (Is[k] == 1) {
            Fx_inc = Fx_inc + f[F(xi, yj, k)] * e[k][0];
            Fy_inc = Fy_inc + f[F(xi, yj, k)] * e[k][1];
        }
    }
    Fx = Fx_inc - Fx_out;
    Fy = Fy_inc - Fy_out;
}

// One iteration of the main loop: 2d_mrlbm.f90:229-535
void Oracle::step() {
    iter += 1;
    const bool xper = cfg.x_periodic != 0, yper = cfg.y_periodic != 0;
    const bool walls_ref = !yper && cfg.wall_mode == MRLBM_WALL_REFERENCE;
    const bool walls_free = !yper && cfg.wall_mode == MRLBM_WALL_FREESLIP;

    // Macroscopic variables (2d_mrlbm.f90:232-245)
#pragma omp parallel for
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            const size_t n = I(i, j);
            double s = 0.0, sx = 0.0, sy = 0.0, sxx = 0.0, syy = 0.0, sxy = 0.0;
            for (int k = 0; k < Q; ++k) s = s + f[F(i, j, k)];
            rho[n] = s;
            double inv_rho = 1.0 / rho[n];
            p[n] = rho[n] * cs2;
            for (int k = 0; k < Q; ++k) sx = sx + f[F(i, j, k)] * (double)e[k][0];
            for (int k = 0; k < Q; ++k) sy = sy + f[F(i, j, k)] * (double)e[k][1];
            for (int k = 0; k < Q; ++k) sxx = sxx + f[F(i, j, k)] * Hxx[k];
            for (int k = 0; k < Q; ++k) syy = syy + f[F(i, j, k)] * Hyy[k];
            for (int k = 0; k < Q; ++k) sxy = sxy + f[F(i, j, k)] * Hxy[k];
            ux[n] = sx * inv_rho;
            uy[n] = sy * inv_rho;
            mxx[n] = sxx * inv_rho;
            myy[n] = syy * inv_rho;
            mxy[n] = sxy * inv_rho;
        }

    // Dirichlet (2d_mrlbm.f90:249-272)
    if (!xper)
        for (int j = 1; j <= ny; ++j) {
            rho[I(nx, j)] = rho[I(nx - 1, j)];
            ux[I(nx, j)] = ux[I(nx - 1, j)];
            uy[I(nx, j)] = uy[I(nx - 1, j)];
        }
    if (!xper)
        for (int j = 1; j <= ny; ++j) {
            ux[I(1, j)] = u_in.empty() ? uinlet : u_in[j - 1];
            uy[I(1, j)] = vinlet;
        }
    if (walls_ref) {
        for (int i = 1; i <= nx; ++i) { ux[I(i, ny)] = 0.0; uy[I(i, ny)] = 0.0; }
        for (int i = 1; i <= nx; ++i) { ux[I(i, 1)] = 0.0; uy[I(i, 1)] = 0.0; }
    }

    // Cylinder (2d_mrlbm.f90:280-311)
    if (cyl && !cfg.rotated_coordinate) {
        velocity_interpolation_boundary_nodes();
        for (int l = 1; l <= nbct; ++l) {
            int i = bou_i[l - 1], j = bou_j[l - 1];
            numerical_boundary_cases(i, j, label_bc[l - 1], ux[I(i, j)], uy[I(i, j)]);
        }
    }
    if (cyl && cfg.rotated_coordinate) {
        if (cfg.vel_interp) velocity_interpolation_boundary_nodes();
        if (cfg.mom_interp) moments_interpolation_boundary_nodes();
        for (int l = 1; l <= nbct; ++l) {
            int i = bou_i[l - 1], j = bou_j[l - 1];
            const size_t n = I(i, j);
            uxp_b[l - 1] = ux[n] * cth_glb[n] + uy[n] * sth_glb[n];
            uyp_b[l - 1] = uy[n] * cth_glb[n] - ux[n] * sth_glb[n];
            if (cfg.strong_mass_bc) numerical_boundary_cases_rotation(i, j, label_bc[l - 1], uxp_b[l - 1], uyp_b[l - 1]);
            if (cfg.eq_mass_bc) numerical_boundary_cases_rotation_rhoeq(i, j, label_bc[l - 1], uxp_b[l - 1], uyp_b[l - 1]);
            if (cfg.weak_mass_bc) numerical_boundary_cases_rotation_weak(i, j, label_bc[l - 1], uxp_b[l - 1], uyp_b[l - 1]);
        }
    }

    // Edge boundaries (2d_mrlbm.f90:313-351)
    if (!xper)
        for (int j = 1; j <= ny; ++j) cfg.incomp_bc ? apply_bc_incomp(nx, j, OUTLET) : apply_bc(nx, j, OUTLET);
    if (!xper)
        for (int j = 1; j <= ny; ++j) cfg.incomp_bc ? apply_bc_incomp(1, j, INLET) : apply_bc(1, j, INLET);
    if (walls_ref)
        for (int i = 1; i <= nx; ++i) cfg.incomp_bc ? apply_bc_incomp(i, ny, TOPWALL) : apply_bc(i, ny, TOPWALL);
    if (walls_ref)
        for (int i = 1; i <= nx; ++i) cfg.incomp_bc ? apply_bc_incomp(i, 1, BOTTOMWALL) : apply_bc(i, 1, BOTTOMWALL);

    const bool in_stats = cfg.post_process && iter >= cfg.statsbegin && iter <= cfg.statsend;
    double rho_in_sum = 0.0;
    if (cfg.post_process) {                                         // 2d_mrlbm.f90:355-387
        if (in_stats) {
            double rho_mean_counter = (double)(float)(iter - cfg.statsbegin);
            for (int j = 1; j <= ny; ++j) rho_in_sum = rho_in_sum + rho[I(1, j)];
            rho_infty = rho_in_sum / (double)ny;
            rho_inf_mean = ((rho_mean_counter * rho_inf_mean) + rho_infty) / (rho_mean_counter + 1.0);
        }
        if (cfg.iplot > 0 && iter % cfg.iplot == 0 && (cyl || cfg.channel_with_square))
            for (int i = 1; i <= nx; ++i)
                for (int j = 1; j <= ny; ++j)
                    if (issolid[I(i, j)] == 1) { ux[I(i, j)] = 0.0; uy[I(i, j)] = 0.0; }
    }

    // Collision in moment space (2d_mrlbm.f90:407-415)
#pragma omp parallel for collapse(2)
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            const size_t n = I(i, j);
            mxx[n] = (1.0 - omega) * mxx[n] + omega * ux[n] * ux[n];
            myy[n] = (1.0 - omega) * myy[n] + omega * uy[n] * uy[n];
            mxy[n] = (1.0 - omega) * mxy[n] + omega * ux[n] * uy[n];
        }
    if (cfg.incomp_bulk) {                                          // 2d_mrlbm.f90:419-442
#pragma omp parallel for collapse(2)
        for (int i = 1; i <= nx; ++i)
            for (int j = 1; j <= ny; ++j) {
                const size_t n = I(i, j);
                mxx_s[n] = mxx[n] - (0.50 * (mxx[n] + myy[n] - ux[n] * ux[n] - uy[n] * uy[n]));
                myy_s[n] = myy[n] - (0.50 * (mxx[n] + myy[n] - ux[n] * ux[n] - uy[n] * uy[n]));
                mxy_s[n] = mxy[n];
            }
    }
    const std::vector<double>& Mxx = cfg.incomp_bulk ? mxx_s : mxx;
    const std::vector<double>& Myy = cfg.incomp_bulk ? myy_s : myy;
    const std::vector<double>& Mxy = cfg.incomp_bulk ? mxy_s : mxy;
    // Regularization / reconstruction (2d_mrlbm.f90:445-457)
#pragma omp parallel for collapse(2)
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            const size_t n = I(i, j);
            for (int k = 0; k < Q; ++k) {
                double cu = (double)e[k][0] * ux[n] + (double)e[k][1] * uy[n];
                fout[F(i, j, k)] = w[k] * rho[n] * (1.0 + (3.0 * cu) + 4.50 * Mxx[n] * Hxx[k] +
                                                   4.50 * Myy[n] * Hyy[k] + 9.00 * Mxy[n] * Hxy[k]);
            }
        }

    // Forces (2d_mrlbm.f90:469-496)
    if (in_stats && cyl) {
        for (int l = 1; l <= nbct; ++l)
            evaluate_forces(bou_i[l - 1], bou_j[l - 1], label_bc[l - 1], F_drag[l - 1], F_lift[l - 1]);
        double fd = 0.0, fl = 0.0;
        for (int l = 1; l <= nbct; ++l) fd = fd + F_drag[l - 1];
        for (int l = 1; l <= nbct; ++l) fl = fl + F_lift[l - 1];
        h_iter.push_back(iter);
        h_fd.push_back(fd);
        h_fl.push_back(fl);
        h_rhoin.push_back(rho_in_sum);
        // probe records (2d_mrlbm.f90:470-475) and the surface pressure (2d_mrlbm.f90:478)
        for (int q = 0; q < 4; ++q) h_probe.push_back(rho[I(i_probe[q], j_probe[q])] / 3.0);
        for (int q = 0; q < 4; ++q) h_probe.push_back(ux[I(i_probe[q], j_probe[q])] / 3.0);
        for (int q = 0; q < 4; ++q) h_probe.push_back(uy[I(i_probe[q], j_probe[q])] / 3.0);
        write_statistics_out();
    } else if (in_stats) {
        h_iter.push_back(iter);
        h_fd.push_back(0.0);
        h_fl.push_back(0.0);
        h_rhoin.push_back(rho_in_sum);
    }

    // Streaming (2d_mrlbm.f90:508-535), serial as in the reference
    f_tmp = fout;
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j)
            for (int k = 0; k < Q; ++k) {
                int ti = i + e[k][0], tj = j + e[k][1];
                if (ti > 0 && ti <= nx && tj > 0 && tj <= ny) f[F(ti, tj, k)] = f_tmp[F(i, j, k)];
            }
    if (xper)
        for (int j = 1; j <= ny; ++j)
            for (int k = 0; k < Q; ++k) {
                if (1 - e[k][0] < 1) f[F(1, j, k)] = f_tmp[F(nx, j, k)];
                if (nx - e[k][0] > nx) f[F(nx, j, k)] = f_tmp[F(1, j, k)];
            }
    if (yper)
        for (int i = 1; i <= nx; ++i)
            for (int k = 0; k < Q; ++k) {
                if (1 - e[k][1] < 1) f[F(i, 1, k)] = f_tmp[F(i, ny, k)];
                if (ny - e[k][1] > ny) f[F(i, ny, k)] = f_tmp[F(i, 1, k)];
            }
    if (walls_free) {
        // Extension: halfway specular reflection.  A population leaving row ny upwards
        // returns to the same row with its y-velocity reversed after one step; rows 1
        // likewise.  The source column wraps when x is periodic, else nothing arrives.
        static const int mirror[Q] = {0, 1, 4, 3, 2, 8, 7, 6, 5};
        for (int i = 1; i <= nx; ++i)
            for (int k = 0; k < Q; ++k) {
                for (int side = 0; side < 2; ++side) {
                    const int j = side == 0 ? ny : 1;
                    if ((side == 0 && e[k][1] != -1) || (side == 1 && e[k][1] != 1)) continue;
                    int si = i - e[k][0];
                    if (si < 1 || si > nx) {
                        if (!xper) continue;
                        si = si < 1 ? nx : 1;
                    }
                    f[F(i, j, k)] = f_tmp[F(si, j, mirror[k])];
                }
            }
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// ctypes surface (test infrastructure)
// write_statistics_out (2d_mrlbm.f90:593-616): extrapolate_var_on_cylinder on p
// (2d_mrlbm.f90:619-672), quadratic_interpolation (2d_mrlbm.f90:742-766), reorder by theta,
// gaussian_smoothing (2d_mrlbm.f90:718-740); the two unformatted records become history rows.
void Oracle::write_statistics_out() {
    std::vector<double> p_cy(nbct), ps(nbct), fit(nbct);
    for (int k = 1; k <= nbct; ++k) {
        double var[5];
        for (int r = 2; r <= 4; ++r) {
            const double xd = (x_ref[r][k - 1] - X(IP(r, 0, k))) / dx;
            const double yd = (y_ref[r][k - 1] - Y(JP(r, 0, k))) / dy;
            const double v0 = (1.0 - xd) * p[I(IP(r, 0, k), JP(r, 0, k))] + xd * p[I(IP(r, 1, k), JP(r, 1, k))];
            const double v1 = (1.0 - xd) * p[I(IP(r, 2, k), JP(r, 2, k))] + xd * p[I(IP(r, 3, k), JP(r, 3, k))];
            var[r] = (1.0 - yd) * v0 + yd * v1;
        }
        const double xs = x_ref[1][k - 1] - x_c, ys = y_ref[1][k - 1] - y_c;
        const double x1 = x_ref[2][k - 1] - x_c, y1 = y_ref[2][k - 1] - y_c;
        const double x2 = x_ref[3][k - 1] - x_c, y2 = y_ref[3][k - 1] - y_c;
        const double x3 = x_ref[4][k - 1] - x_c, y3 = y_ref[4][k - 1] - y_c;
        const double p1 = var[2], p2 = var[3], p3 = var[4];
        const double r1 = std::sqrt((x1 * x1) + (y1 * y1)), r2 = std::sqrt((x2 * x2) + (y2 * y2));
        const double r3 = std::sqrt((x3 * x3) + (y3 * y3)), rs = std::sqrt((xs * xs) + (ys * ys));
        const double denom = (r1 - r2) * (r1 - r3) * (r2 - r3);
        const double a0 = (r1 * r3 * p2 * (r3 - r1) + (r2 * r2) * (r3 * p1 - r1 * p3) + r2 * ((r1 * r1) * p3 - (r3 * r3) * p1)) / denom;
        const double a1 = ((r3 * r3) * (p1 - p2) + (r1 * r1) * (p2 - p3) + (r2 * r2) * (p3 - p1)) / denom;
        const double a2 = (r3 * (p2 - p1) + r2 * (p1 - p3) + r1 * (p3 - p2)) / denom;
        p_cy[k - 1] = a0 + a1 * rs + a2 * (rs * rs);
    }
    for (int k = 1; k <= nbct; ++k) ps[k - 1] = p_cy[idx[k - 1] - 1];
    const double sigma = 0.1;
    for (int i = 1; i <= nbct; ++i) {
        double sw = 0.0, sv = 0.0;
        for (int j = 1; j <= nbct; ++j) {
            const double d = thetas_cy[i - 1] - thetas_cy[j - 1];
            const double wgt = std::exp(-(d * d) / (2.0 * (sigma * sigma)));
            sw = sw + wgt;
            sv = sv + wgt * ps[j - 1];
        }
        fit[i - 1] = sv / sw;
    }
    h_psurf.insert(h_psurf.end(), ps.begin(), ps.end());
    h_psmooth.insert(h_psmooth.end(), fit.begin(), fit.end());
}

extern "C" {

void* orc_create(const mrlbm_config* cfg, char* errbuf, int errlen) {
    Oracle* o = new Oracle();
    if (cfg->num_threads > 0) {
#ifdef _OPENMP
        omp_set_num_threads(cfg->num_threads);
#endif
    }
    if (!o->setup(*cfg)) {
        if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", o->err.c_str());
        delete o;
        return nullptr;
    }
    return o;
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

int orc_step(void* h, int n) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int s = 0; s < n; ++s) o->step();
    return 0;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

static const std::vector<double>* dvec(Oracle* o, const char* name) {
    struct { const char* n; std::vector<double>* v; } t[] = {
        {"f", &o->f}, {"fout", &o->fout}, {"rho", &o->rho}, {"p", &o->p}, {"ux", &o->ux}, {"uy", &o->uy},
        {"mxx", &o->mxx}, {"myy", &o->myy}, {"mxy", &o->mxy}, {"mxxp", &o->mxxp}, {"myyp", &o->myyp},
        {"cth_glb", &o->cth_glb}, {"sth_glb", &o->sth_glb}, {"s2th_glb", &o->s2th_glb}, {"c2th_glb", &o->c2th_glb},
        {"cx_p", &o->cx_p}, {"cy_p", &o->cy_p}, {"Hxx_p", &o->Hxx_p}, {"Hyy_p", &o->Hyy_p}, {"Hxy_p", &o->Hxy_p},
        {"radii", &o->radii}, {"xb", &o->xb}, {"yb", &o->yb}, {"delta_uk", &o->delta_uk},
        {"theta_c", &o->theta_c}, {"thetas_cy", &o->thetas_cy}, {"x_ref1", &o->x_ref[1]}, {"y_ref1", &o->y_ref[1]},
        {"x_ref2", &o->x_ref[2]}, {"y_ref2", &o->y_ref[2]}, {"x_ref3", &o->x_ref[3]}, {"y_ref3", &o->y_ref[3]},
        {"x_ref4", &o->x_ref[4]}, {"y_ref4", &o->y_ref[4]}, {"F_drag", &o->F_drag}, {"F_lift", &o->F_lift},
        {"uxp_b", &o->uxp_b}, {"uyp_b", &o->uyp_b}, {"p_surface", &o->h_psurf}, {"p_surface_smooth", &o->h_psmooth},
        {"probes", &o->h_probe},
    };
    for (auto& e : t)
        if (std::strcmp(e.n, name) == 0) return e.v;
    return nullptr;
}
static const std::vector<int>* ivec(Oracle* o, const char* name) {
    struct { const char* n; std::vector<int>* v; } t[] = {
        {"isfluid", &o->isfluid}, {"issolid", &o->issolid}, {"isbound", &o->isbound}, {"bou_i", &o->bou_i},
        {"bou_j", &o->bou_j}, {"label_bc", &o->label_bc}, {"idx", &o->idx}, {"i_p2", &o->i_p[2]},
        {"j_p2", &o->j_p[2]}, {"i_p3", &o->i_p[3]}, {"j_p3", &o->j_p[3]}, {"i_p4", &o->i_p[4]}, {"j_p4", &o->j_p[4]},
    };
    for (auto& e : t)
        if (std::strcmp(e.n, name) == 0) return e.v;
    return nullptr;
}

// Element count of a named array (-1 if unknown); kind: 0 double, 1 int32.
long long orc_size(void* h, const char* name, int* kind) {
    Oracle* o = static_cast<Oracle*>(h);
    if (auto* v = dvec(o, name)) { *kind = 0; return (long long)v->size(); }
    if (auto* v = ivec(o, name)) { *kind = 1; return (long long)v->size(); }
    return -1;
}

int orc_get(void* h, const char* name, void* out, long long n) {
    Oracle* o = static_cast<Oracle*>(h);
    if (auto* v = dvec(o, name)) {
        if ((long long)v->size() != n) return 1;
        std::memcpy(out, v->data(), (size_t)n * sizeof(double));
        return 0;
    }
    if (auto* v = ivec(o, name)) {
        if ((long long)v->size() != n) return 1;
        std::memcpy(out, v->data(), (size_t)n * sizeof(int));
        return 0;
    }
    return 2;
}

int orc_set(void* h, const char* name, const void* in, long long n) {
    Oracle* o = static_cast<Oracle*>(h);
    if (std::strcmp(name, "u_in") == 0) {
        if (in == nullptr) { o->u_in.clear(); return 0; }
        if (n != o->ny) return 1;
        o->u_in.assign((const double*)in, (const double*)in + n);
        return 0;
    }
    if (std::strcmp(name, "f") == 0) {
        if ((long long)o->f.size() != n) return 1;
        std::memcpy(o->f.data(), in, (size_t)n * sizeof(double));
        return 0;
    }
    return 2;
}

// scalars: nx, ny, nbct, iter, r_cyl, nu, omega, x_c, y_c, r_c, rho_inf_mean
int orc_scalars(void* h, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    out[0] = o->nx; out[1] = o->ny; out[2] = o->nbct; out[3] = o->iter; out[4] = o->r_cyl;
    out[5] = o->nu; out[6] = o->omega; out[7] = o->x_c; out[8] = o->y_c; out[9] = o->r_c;
    out[10] = o->rho_inf_mean;
    return 0;
}

int orc_set_iter(void* h, int it) { static_cast<Oracle*>(h)->iter = it; return 0; }

// Force history (one record per stats step); copies up to cap, returns the total count.
int orc_forces(void* h, int* iters, double* fd, double* fl, double* rhoin, int cap) {
    Oracle* o = static_cast<Oracle*>(h);
    int n = (int)o->h_iter.size();
    for (int t = 0; t < n && t < cap; ++t) {
        iters[t] = o->h_iter[t]; fd[t] = o->h_fd[t]; fl[t] = o->h_fl[t]; rhoin[t] = o->h_rhoin[t];
    }
    return n;
}

}  // extern "C"
