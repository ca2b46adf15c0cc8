// step_params.h -- parameter block of one fused time-step launch (host <-> device contract).
#pragma once
#include <cstdint>
#include "lattice.h"

namespace mrlbm {

// Per-stats-step record written to the device ring: iter, F_drag_net, F_lift_net,
// sum(rho(1,:)) -- the values of 2d_mrlbm.f90:359 and 488-494.
constexpr int REC_WORDS = 4;

// Constants of the deviation (FP32) form, computed once in FP64 on the host from the
// reference's single-rounded weights w_k and FP64 Hermite tables H_k.  Each is the rest-state
// part of a closure that cancels in exact arithmetic; with single-rounded weights it is
// O(1e-9) and is added back so the FP32 step keeps the FP64 step's arithmetic content.
// SW_ab(e) = sum over edge e's incoming set of w_k H_ab,k; W(e) = sum of w_k over it.
struct DevConsts {
    float eps_mass;          // sum_k w_k - 1
    float cxx, cyy;          // sum_k w_k H_xx,k, sum_k w_k H_yy,k
    float k_out_mxx;         // outlet: 1 + 9 SW_xx
    float sw_out_yy;         //         SW_yy
    float k_in_rho;          // inlet:  4 W + 3 SW_xx - 3
    float k_in_mxx;          //         1 + 9 SW_xx
    float sw_in_yy;          //         SW_yy
    float k_in_rho_inc;      //         6 W - 5                       (apply_bc_incomp)
    float k_w_rho[2];        // walls (top, bottom): 12 W - 9 - omega + 9 (1 - omega) SW_yy
    float sw_w_xx[2];        //         SW_xx
    float k_w_myy[2];        //         1 + 9 SW_yy
    float k_w_rho_inc[2];    //         6 W - 5                       (apply_bc_incomp)
    float w_wall[2];         //         W
    float lab_w[16];         // curved wall: sum of w_k over the label's Is (== over its Os)
};

// A population of the loaded state that the buffer cannot hold: with periodic wraps
// (and free-slip with x-periodic) the reference copies one corner population to two
// destinations (2d_mrlbm.f90:519-535), so after any step those two agree; a loaded state
// may not.  Such destinations are served from this list on the first step after a load.
struct OvrEntry { int i, j, k, pad; double v; };

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
    const OvrEntry* ovr;          // loaded-state overrides for this step, or null
    int n_ovr;
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
