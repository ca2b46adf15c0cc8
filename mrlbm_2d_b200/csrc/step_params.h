// step_params.h -- parameter block of one fused time-step launch (host <-> device contract).
#pragma once
#include <cstdint>
#include "lattice.h"

namespace mrlbm {

// Per-stats-step record written to the device ring: iter, F_drag_net, F_lift_net,
// sum(rho(1,:)) -- the values of 2d_mrlbm.f90:359 and 488-494.
constexpr int REC_WORDS = 4;

// Constants of the deviation (FP32) form, precomputed in FP64 on the host from the
// reference's single-rounded weights so the FP32 kernel works only with small quantities.
struct DevConsts {
    float eps_mass;        // sum(w) - 1   (the reference's weights sum to 1 + 7.45e-9)
    float cxx, cyy;        // sum_k w_k Hxx_k, sum_k w_k Hyy_k
    // edge closures, per edge e in {outlet, inlet, top, bottom}:
    float wI[4];           // sum_{Is} w
    float swxx[4], swyy[4], swxy[4];   // sum_{Is} w H
    // cylinder closure, per label (0..15):
    float lab_wI[16];      // sum_{Is} w  ( == sum_{Os} w for every handled label)
};

template <class T>
struct StepParams {
    const T* __restrict__ src;    // fout of the previous step (+ ghost ring)
    T* __restrict__ dst;          // fout of this step
    Layout L;
    // lattice constants, computed on the host exactly as 2d_mrlbm.f90:129-178
    T w[Q];
    T hm, hp;                     // Hxx/Hyy values: 0 - cs2 and 1 - cs2
    T omega, omega1;              // omega and (1 - omega)
    T uinlet, vinlet;
    const T* u_in;                // optional per-row inlet velocity (ny entries) or null
    int xper, yper, freeslip, walls_ref, incomp_bc, incomp_bulk;
    int zero_solid_u;             // plot step: u = 0 at solid nodes (2d_mrlbm.f90:375-384)
    int do_stats;                 // stats step: forces + inlet density sum
    // curved wall
    int nb, nbblk;                // boundary nodes, boundary blocks at the start of the grid
    const int* __restrict__ bint; // IntField table [I_NFIELDS * nb]
    const T* __restrict__ bgeo;   // GeoField table [G_NFIELDS * nb]
    int closure, vel_interp, mom_interp;
    int box_x0, box_y0, box_w, box_h;
    const int* __restrict__ boxmap;
    int label15_allnine;
    // reduction scratch and output
    double* partials;             // [nbblk * 3]
    unsigned* counter;            // arrival counter of boundary blocks (reset by the last)
    double* rec;                  // REC_WORDS doubles for this step, or null
    double* node_force;           // optional per-boundary-node (Fx, Fy) [2 * nb], or null
    int iter;
    int* errflag;
    // optional macroscopic output (Fortran order nx*ny): rho, ux, uy, mxx, myy, mxy
    double* macro;                // [6 * nx * ny] or null
    int tiles_x;                  // bulk tiles along x
    DevConsts dc;                 // deviation-form constants (FP32 only)
};

// Host-side launch entry points (defined in step_f64.cu / step_f32.cu).
int launch_step_f64(const StepParams<double>& p, int tile_cfg, void* stream);
int launch_step_f32(const StepParams<float>& p, int tile_cfg, void* stream);

// Tile configurations (bulk threads: 32 x BY, each thread NJ nodes along y).
struct TileCfg { int bx, by, nj; };
constexpr int N_TILE_CFGS = 4;
constexpr TileCfg TILE_CFGS[N_TILE_CFGS] = {{32, 8, 1}, {32, 8, 2}, {32, 4, 4}, {64, 4, 2}};

}  // namespace mrlbm
