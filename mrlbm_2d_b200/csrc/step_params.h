// step_params.h -- parameter block of one fused time-step launch (host <-> device contract).
#pragma once
#include <cuda.h>
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
struct alignas(64) StepParams {
    CUtensorMap tmap;             // 2-D map of src (rows = 9 planes x (ny+2)), TMA shapes only
    CUtensorMap tmap_st;          // 2-D map of dst with the store box (BX x BY), TMA-store shapes only
    unsigned long long* tile_ctr; // tile claim counter of the TMA shapes
    unsigned long long tile_base; // counter value at the start of this step
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
    int neblk;                    // edge blocks (one thread per domain-edge node) after them
    int halo_l, halo_r;           // x-slab of a larger domain: column 0 / nx+1 hold the neighbour's populations
    const int* __restrict__ bint; // IntField table [I_NFIELDS * nb]
    const T* __restrict__ bgeo;   // GeoField table [G_NFIELDS * nb]
    int closure, vel_interp, mom_interp;
    int box_x0, box_y0, box_w, box_h;
    const int* __restrict__ boxmap;
    int label15_allnine;
    // reduction scratch and output
    double* partials;             // per-step scratch: Fx[nb], Fy[nb], rho(1,j)[ny]
    unsigned* counter;            // [0] arrivals of boundary blocks, [1] of inlet edge blocks (reset by the last)
    double* rec;                  // REC_WORDS doubles for this step, or null
    // Deferred record sums (single-case steps): with defer set, a stats step leaves its terms in
    // `partials` and no block of it waits for the others to sum them; the next launch's first
    // edge block (or the finishing kernel, launch_finish_record) sums them in index order into
    // prev_rec, taking the in-order sums off the step's critical path.
    int defer;
    const double* prev_partials;  // terms of the last stats step still to be summed, or null
    double* prev_rec;             // its record
    int prev_iter;
    double* node_force;           // optional per-boundary-node (Fx, Fy) [2 * nb], or null
    int iter;
    // A launch captured once into a replayed graph (a batch's per-case streams schedule): `call`
    // points at the state {iter0, ring_n0} uploaded before each replay, and the record fields
    // (iter, do_stats, rec) come from it instead (step_rec): iteration iter0 + bstep + 1, a
    // record when it lies in [stats_lo, stats_hi], in `ring` after the call's earlier records.
    const int* call;
    int bstep, stats_lo, stats_hi;
    double* ring;
    int plot_every;               // replayed launches: solid velocities zeroed when iter % plot_every == 0 (0: never)
    int* errflag;
    // optional macroscopic output (Fortran order nx*ny): rho, ux, uy, mxx, myy, mxy
    double* macro;                // [6 * nx * ny] or null
    double* fstat;                // [6 * nx * ny] running sums of u, v, p, u^2, v^2, p^2, or null
    const T* body;                // [2 * nx * ny] body force (x then y), node order, or null
    int tiles_x;                  // bulk tiles along x
    unsigned long long tx_magic;  // tile_div_magic(tiles_x, tiles), or 0: t / tiles_x by division
    DevConsts dc;                 // deviation-form constants (FP32 only)
};

// ceil(2^32 / d), so that t / d == (t * m) >> 32 for every t with t * d < 2^32 (writing
// m d = 2^32 + e, 0 <= e < d, the quotient's error term t e / (d 2^32) stays below 1/d); 0 when
// the tiles of a launch reach that bound.
inline unsigned long long tile_div_magic(int d, long long tiles) {
    return (unsigned long long)tiles * (unsigned long long)d < (1ull << 32) ? ((1ull << 32) + (unsigned)d - 1) / (unsigned)d : 0ull;
}

// Bulk tile shapes of step_kernel (threads BX x BY, NJ rows per thread, MINB resident blocks
// per SM, which sets the register budget 65536 / (BX*BY*MINB)); MINB is given per precision
// (FP64, FP32): the FP32 node path needs fewer registers, so more of its blocks can be
// resident.  The autotuner picks one.
struct TileCfg { int bx, by, nj, minb64, minb32; };
#define MRLBM_TILE_LIST(X) \
    X(0, 32, 8, 1, 4, 4)   \
    X(1, 32, 8, 2, 4, 4)   \
    X(2, 32, 8, 2, 3, 5)   \
    X(3, 32, 4, 4, 4, 4)   \
    X(4, 32, 4, 4, 6, 6)   \
    X(5, 32, 8, 4, 3, 3)   \
    X(6, 64, 4, 2, 4, 4)   \
    X(7, 32, 4, 2, 6, 10)  \
    X(8, 32, 8, 4, 2, 2)   \
    X(9, 32, 4, 2, 8, 8)
constexpr int N_TILE_CFGS = 10;
#define MRLBM_TILE_ENTRY(id, bx, by, nj, mb64, mb32) {bx, by, nj, mb64, mb32},
constexpr TileCfg TILE_CFGS[N_TILE_CFGS] = {MRLBM_TILE_LIST(MRLBM_TILE_ENTRY)};
#undef MRLBM_TILE_ENTRY

// TMA-fed persistent shapes of step_kernel_tma (BX threads = columns per tile, BY rows per
// tile, STAGES tiles in flight per CTA).  Shape ids continue after the step_kernel ones.
// The copy box is BX + 32 bytes wide, which must stay within the 256-element box limit.
struct TmaCfg { int bx, by, stages; };
#define MRLBM_TMA_LIST(X) \
    X(10, 128, 4, 4)      \
    X(11, 128, 2, 6)      \
    X(12, 224, 2, 4)      \
    X(13, 128, 8, 3)      \
    X(14, 64, 4, 6)       \
    X(15, 224, 4, 3)
constexpr int N_TMA_CFGS = 6;
constexpr int TMA_CFG0 = N_TILE_CFGS;
#define MRLBM_TMA_ENTRY(id, bx, by, st) {bx, by, st},
constexpr TmaCfg TMA_CFGS[N_TMA_CFGS] = {MRLBM_TMA_LIST(MRLBM_TMA_ENTRY)};
#undef MRLBM_TMA_ENTRY

// TMA shapes whose fully interior tiles are also written back by tensor stores from a
// shared-memory output tile (ids after the pipelined shapes).
#define MRLBM_TMAS_LIST(X) \
    X(27, 224, 4, 2)       \
    X(28, 128, 4, 3)       \
    X(29, 224, 2, 3)       \
    X(30, 128, 8, 2)
constexpr int N_TMAS_CFGS = 4;
#define MRLBM_TMA_ENTRY(id, bx, by, st) {bx, by, st},
constexpr TmaCfg TMAS_CFGS[N_TMAS_CFGS] = {MRLBM_TMAS_LIST(MRLBM_TMA_ENTRY)};
#undef MRLBM_TMA_ENTRY

// 128-bit vector shapes of step_kernel_vec (WARPS warps per block, each lane 16 bytes of a
// row; NJ rows per warp; MINB resident blocks per SM).
#define MRLBM_VEC_LIST(X) \
    X(16, 8, 1, 2)        \
    X(17, 8, 2, 2)        \
    X(18, 4, 2, 4)        \
    X(19, 8, 1, 1)        \
    X(20, 4, 1, 4)        \
    X(21, 2, 4, 8)
constexpr int N_VEC_CFGS = 6;
struct VecCfg { int warps, nj, minb; };
#define MRLBM_VEC_ENTRY(id, w, nj, mb) {w, nj, mb},
constexpr VecCfg VEC_CFGS[N_VEC_CFGS] = {MRLBM_VEC_LIST(MRLBM_VEC_ENTRY)};
#undef MRLBM_VEC_ENTRY
constexpr int VEC_CFG0 = TMA_CFG0 + N_TMA_CFGS;

// Resident blocks per SM of the batched bulk kernels, per tile shape (ids 0..9) and vector
// shape (ids VEC_CFG0..): a batched block reads its case's parameters from shared memory into
// registers, where a single case reads them from the constant bank, so a batched shape needs
// more registers than the same single-case shape.  These are the largest counts at which the
// lean FP32 / FP64 batched instantiations keep every value in registers.
constexpr int BATCH_MINB32[N_TILE_CFGS] = {4, 3, 2, 4, 3, 2, 3, 7, 1, 6};
constexpr int BATCH_MINB64[N_TILE_CFGS] = {3, 2, 1, 2, 1, 1, 2, 4, 1, 3};
constexpr int BATCH_VEC_MINB32[N_VEC_CFGS] = {2, 2, 3, 2, 3, 6};
constexpr int BATCH_VEC_MINB64[N_VEC_CFGS] = {1, 1, 3, 2, 3, 6};

// Persistent software-pipelined shapes of step_kernel_pipe (B threads per block, MINB
// resident blocks per SM; the grid is the resident set).
#define MRLBM_PIPE_LIST(X) \
    X(22, 128, 8)          \
    X(23, 256, 4)          \
    X(24, 128, 6)          \
    X(25, 256, 3)          \
    X(26, 128, 4)
constexpr int N_PIPE_CFGS = 5;
constexpr int PIPE_CFG0 = VEC_CFG0 + N_VEC_CFGS;
constexpr int TMAS_CFG0 = PIPE_CFG0 + N_PIPE_CFGS;
constexpr int N_ALL_CFGS = TMAS_CFG0 + N_TMAS_CFGS;
inline bool is_tma_store_cfg(int c) { return c >= TMAS_CFG0 && c < N_ALL_CFGS; }
inline bool is_tma_cfg(int c) { return (c >= TMA_CFG0 && c < VEC_CFG0) || is_tma_store_cfg(c); }
inline TmaCfg tma_cfg(int c) { return is_tma_store_cfg(c) ? TMAS_CFGS[c - TMAS_CFG0] : TMA_CFGS[c - TMA_CFG0]; }
inline bool is_vec_cfg(int c) { return c >= VEC_CFG0 && c < PIPE_CFG0; }
// Kernel launches of one time step: FP32 tile shapes run the step as one launch (the wall and
// edge blocks first in the grid), every other shape as an auxiliary launch and a bulk launch.
inline int step_launches(bool fp32, int c) { return fp32 && c >= 0 && c < N_TILE_CFGS ? 1 : 2; }

// Host-side launch entry points (step_f64.cu / step_f32.cu).  `workers` is the persistent
// CTA count for TMA shapes (ignored otherwise).  Return 0, -1 on a launch error, -2 when the
// shape does not fit this precision.
int launch_step_f64(const StepParams<double>& p, int tile_cfg, void* stream, int workers);
int launch_step_f32(const StepParams<float>& p, int tile_cfg, void* stream, int workers);
// Record (iter, sum Fx, sum Fy, sum rho(1,:)) of a stats step run with deferred sums, from its
// terms (Fx[nb], Fy[nb], rho(1,j)[ny]), summed in index order by one small launch.
int launch_finish_record(const double* partials, int nb, int ny, int halo_l, double* rec, int iter, void* stream);
// Halo-face columns of an x-slab ahead of its step (face_kernel, step_common.cuh).
int launch_face_f64(const StepParams<double>& p, bool full, void* stream);
int launch_face_f32(const StepParams<float>& p, bool full, void* stream);
// Persistent CTAs one SM holds for a TMA shape (0 when the shape does not fit).
int tma_ctas_per_sm(int precision, int tile_cfg);
// Bytes of one tensor-map box row and rows per box for a TMA shape.
void tma_box(int precision, int tile_cfg, int* box_w, int* box_h, int* stages);

}  // namespace mrlbm
