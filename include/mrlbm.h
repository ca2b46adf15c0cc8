/*
 * mrlbm.h -- C ABI of the B200-native moment-regularized D2Q9 cylinder-flow step.
 *
 * The reference (sakthi-lbm/mrlbm_2d) is one Fortran program whose time-loop body
 * (2d_mrlbm.f90:231-535) is the hot path.  It has no library interface: all state is
 * program-scope globals (2d_mrlbm.f90:1-73) and every routine is an internal subroutine
 * (2d_mrlbm.f90:557).  This header is the seam a Fortran host (ISO_C_BINDING), a C/C++
 * driver or Python ctypes binds to; each entry point names the reference code it replaces.
 *
 * Conventions
 *   - Every function returns int: 0 = OK, >0 = configuration / geometry error,
 *     <0 = CUDA error or a device-side error flag (NaN / non-positive density).
 *   - Arrays are contiguous, Fortran order: a field v(nx,ny) has v(i,j) at (i-1)+nx*(j-1);
 *     populations f(nx,ny,0:8) have f(i,j,k) at (i-1)+nx*(j-1)+nx*ny*k, exactly the
 *     reference's f(1:nx,1:ny,0:q-1) (2d_mrlbm.f90:2285).
 *   - The handle owns all device memory.  Host arrays passed in are borrowed for the
 *     duration of the call only.  One host thread per handle; calls are ordered on the
 *     handle's stream; every call that returns host data synchronises that stream.
 *   - D2Q9 order k = 0 rest, 1 +x, 2 +y, 3 -x, 4 -y, 5 (+,+), 6 (-,+), 7 (-,-), 8 (+,-)
 *     (2d_mrlbm.f90:129-131).
 */
#ifndef MRLBM_H
#define MRLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------- */
#define MRLBM_OK              0
#define MRLBM_EINVAL          1   /* bad argument or configuration value              */
#define MRLBM_ENAMELIST       2   /* input.dat could not be read (2d_mrlbm.f90:2235-2238) */
#define MRLBM_EGEOMETRY       3   /* unhandled boundary label / stencil on a non-fluid node */
#define MRLBM_EUNSUPPORTED    4   /* flag combination the reference leaves undefined   */
#define MRLBM_ESTATE          5   /* call out of order (e.g. step before init)          */
#define MRLBM_ECUDA          -1   /* CUDA runtime error                                  */
#define MRLBM_EDEVICE_NAN    -2   /* device flag: NaN or non-positive density           */
#define MRLBM_ENODEVICE      -3   /* no CUDA device / kernels not loadable              */
#define MRLBM_EDEVICE_TIMEOUT -4  /* device flag: a bounded wait in a kernel gave up      */

/* ---- precision of a handle ----------------------------------------------------- */
#define MRLBM_FP64  64            /* populations and arithmetic in FP64 (reference form) */
#define MRLBM_FP32  32            /* populations stored as FP32 deviations from w_k      */

/* ---- extension switches (0 is always the reference behaviour) -------------------- */
#define MRLBM_GEOM_REFERENCE   0  /* nx,ny,centre,radius from ncy and L_* (2d_mrlbm.f90:86-92, 946-948) */
#define MRLBM_GEOM_EXPLICIT    1  /* nx,ny,x_c,y_c,r_c taken as given (real-valued centre)      */
#define MRLBM_WALL_REFERENCE   0  /* no-slip regularized walls when !y_periodic (2d_mrlbm.f90:263-272, 1305-1359) */
#define MRLBM_WALL_FREESLIP    1  /* free-slip: halfway specular reflection in streaming        */
#define MRLBM_LABEL15_REJECT   0  /* label 15 has empty link rows in the reference (2d_mrlbm.f90:2008) */
#define MRLBM_LABEL15_ALLNINE  1  /* label 15 closes over all nine links                        */
#define MRLBM_NU_REFERENCE     0  /* nu = U * 2 r_cyl / Re, r_cyl = max boundary radius (2d_mrlbm.f90:134) */
#define MRLBM_NU_DIAMETER      1  /* nu = U * 2 r_c / Re (nominal diameter)                     */
#define MRLBM_INIT_REFERENCE   0  /* rho = 1, u = 0, f = w (2d_mrlbm.f90:1220-1235)             */
#define MRLBM_INIT_NOISE       1  /* rho = 1, u = (U,0) + seeded Gaussian noise, regularized equilibrium */

/*
 * Run configuration.  The first block mirrors the reference namelists
 * DomainSize, Cylinder, Numbers, Parallel, Controls and LogicalControls
 * (2d_mrlbm.f90:2227-2233, input.dat:1-45); the last block holds the extensions
 * the benchmark-suite cylinder cases need (explicit centre, free-slip walls, seeded noise
 * start).  Field order is part of the ABI.
 */
typedef struct mrlbm_config {
    double   x_c, y_c, r_c;          /* cylinder centre / classification radius (lattice units, node (i,j) sits at (i,j)) */
    double   Re, uo, rho_infty;      /* &Numbers Re; &Controls uo, rho_infty */
    double   noise_amp;              /* INIT_NOISE: noise standard deviation as a fraction of uo */
    uint64_t seed;                   /* INIT_NOISE: counter-based RNG key */
    int32_t  nx, ny;                 /* &DomainSize (overwritten from ncy/L_* in GEOM_REFERENCE) */
    int32_t  channel_with_cylinder;
    int32_t  ncy, L_front, L_back, L_top, L_bot;                     /* &Cylinder */
    int32_t  iplot, max_iter, isave, irestart, statsbegin, statsend, iplotstats; /* &Controls */
    int32_t  num_threads, lattice_type;                              /* &Parallel, &DomainSize */
    int32_t  post_process, x_periodic, y_periodic, channel_with_square;
    int32_t  incomp_bc, incomp_bulk, vel_interp, mom_interp, rotated_coordinate;
    int32_t  strong_mass_bc, eq_mass_bc, weak_mass_bc;               /* &LogicalControls */
    int32_t  geometry_mode, wall_mode, label15_rule, nu_length, init_mode;
    int32_t  reserved;
} mrlbm_config;

/* Boundary-node geometry as the reference builds it in get_coord (2d_mrlbm.f90:931-1156). */
typedef struct mrlbm_geometry_info {
    int32_t nx, ny, nbct;            /* nbct = number of curved-wall boundary nodes (2d_mrlbm.f90:1004) */
    int32_t n_label15;               /* boundary nodes whose quadrant label is 15 */
    double  x_c, y_c, r_c, r_cyl;    /* r_cyl = max boundary-node radius (2d_mrlbm.f90:1038-1050) */
    double  nu, omega;               /* 2d_mrlbm.f90:133-135 */
    /* padded population layout of one time level: population k of node (i,j), with i in
     * 0..nx+1 and j in 0..ny+1 (ghost ring included), is element k*plane + j*pitch + i + off */
    int32_t pitch, off;
    int64_t plane;
    int64_t state_bytes;             /* bytes of the two time levels mrlbm_step_noalloc needs */
} mrlbm_geometry_info;

typedef struct mrlbm_handle mrlbm_handle;

/* sizeof(mrlbm_config), for bindings that mirror the struct (ctypes, ISO_C_BINDING). */
size_t mrlbm_config_sizeof(void);

/* Reference defaults: the values of the shipped input.dat (input.dat:1-45). */
int mrlbm_config_defaults(mrlbm_config* cfg);

/* Read the six namelist groups of an input.dat file into cfg, in the order the reference
 * reads them; replaces read_input_file (2d_mrlbm.f90:2222-2275).  Returns MRLBM_ENAMELIST
 * where the reference prints "Error while reading input.dat file..." and stops. */
int mrlbm_config_from_namelist(const char* path, mrlbm_config* cfg);

/* Fill nx, ny, x_c, y_c, r_c from ncy and L_* as the reference does
 * (2d_mrlbm.f90:86-92 and 946-948).  No-op unless geometry_mode == GEOM_REFERENCE. */
int mrlbm_config_resolve_geometry(mrlbm_config* cfg);

/* Build geometry and device state for one case; replaces the setup part of the main
 * program (2d_mrlbm.f90:83-214: allocate_memory, get_coord, weights, nu/omega, Hermite
 * and rotated tables, finding_incoming_outgoing_pops).  precision = MRLBM_FP64 or
 * MRLBM_FP32.  The initial state follows cfg->init_mode (initialize, 2d_mrlbm.f90:1220).
 * device = -1 creates a host-only handle (configuration and geometry queries only; the
 * stepping and state calls then return MRLBM_ENODEVICE). */
int mrlbm_create(const mrlbm_config* cfg, int precision, int device, mrlbm_handle** out);
int mrlbm_destroy(mrlbm_handle* h);

/* Last error text of a handle (or of the last failed mrlbm_create when h == NULL). */
int mrlbm_last_error(const mrlbm_handle* h, char* buf, size_t len);

/* Sticky device status: MRLBM_OK, MRLBM_EDEVICE_NAN or MRLBM_EDEVICE_TIMEOUT.  Synchronises. */
int mrlbm_status(mrlbm_handle* h);

/* Run subsequent work on a caller-owned cudaStream_t (NULL = the legacy default stream).
 * A new handle works on a private non-blocking stream until this is called. */
int mrlbm_set_stream(mrlbm_handle* h, void* cuda_stream);

int mrlbm_get_geometry_info(const mrlbm_handle* h, mrlbm_geometry_info* info);

/* Per boundary node l = 1..nbct, in the reference's order (i-major, j-minor,
 * 2d_mrlbm.f90:1007-1036): bou_i, bou_j, label_bc (int32[nbct]); delta_uk (double[nbct],
 * 2d_mrlbm.f90:1089-1091); ref_xy = x_ref1..4,y_ref1..4 (double[8*nbct], point-major);
 * stencil = i_p2,j_p2,i_p3,j_p3,i_p4,j_p4 (int32[24*nbct], 2d_mrlbm.f90:1099-1129).
 * Any pointer may be NULL. */
int mrlbm_get_boundary_nodes(const mrlbm_handle* h, int32_t* bou_i, int32_t* bou_j,
                             int32_t* label_bc, double* delta_uk, double* ref_xy,
                             int32_t* stencil);

/* Node classes isfluid/issolid/isbound (int32[nx*ny] each, 2d_mrlbm.f90:968-1002). */
int mrlbm_get_node_classes(const mrlbm_handle* h, int32_t* isfluid, int32_t* issolid,
                           int32_t* isbound);

/* Replace the state by post-streaming populations f(nx,ny,0:8) (what read_restart_file
 * loads, 2d_mrlbm.f90:2204-2220) and set the iteration counter. */
int mrlbm_load_state(mrlbm_handle* h, const double* f, int32_t iter);

/* Post-streaming populations after the last step (the f of write_restart_file,
 * 2d_mrlbm.f90:2186-2202).  On a host-only handle: the configured initial populations. */
int mrlbm_get_state(mrlbm_handle* h, double* f);

/* Per-row inlet velocity u_in(1..ny) replacing the uniform uinlet of 2d_mrlbm.f90:258
 * (extension; NULL restores the uniform inlet). */
int mrlbm_set_inlet_profile(mrlbm_handle* h, const double* u_in);

/* Advance nsteps time steps (2d_mrlbm.f90:229-535 per step).  Forces are reduced on
 * the steps post_process and statsbegin <= iter <= statsend select (2d_mrlbm.f90:461-502).
 * With flags & MRLBM_STEP_MACRO the last step also stores its post-boundary-condition
 * macroscopic fields for mrlbm_get_macro. */
#define MRLBM_STEP_MACRO   1
int mrlbm_step(mrlbm_handle* h, int32_t nsteps, int32_t flags);

/* Current iteration number (the reference's iter after the last step).  A new handle is at
 * iteration 1: the reference's restart_step starts at 1 (2d_mrlbm.f90:7), so its first step
 * is iter 2 (2d_mrlbm.f90:229). */
int mrlbm_get_iter(const mrlbm_handle* h, int32_t* iter);

/* Macroscopic fields of the last step run with MRLBM_STEP_MACRO, after the Dirichlet and
 * regularized boundary conditions and before collision (the values write_function_plot3d
 * writes, 2d_mrlbm.f90:371-386).  Any pointer may be NULL; mxx/myy/mxy are the Hermite
 * second moments the collision starts from. */
int mrlbm_get_macro(mrlbm_handle* h, double* rho, double* ux, double* uy,
                    double* mxx, double* myy, double* mxy);

/* Drain the force history: one record per stats step (the lines of forces_time.dat,
 * 2d_mrlbm.f90:492-494) plus the inlet-column density sum sum(rho(1,:))
 * (2d_mrlbm.f90:359).  Copies up to cap records, returns the count in *n and removes them. */
int mrlbm_get_forces(mrlbm_handle* h, int32_t* iter, double* f_drag, double* f_lift,
                     double* rho_inlet_sum, int32_t cap, int32_t* n);

/* Strouhal number, mean drag coefficient and rms lift coefficient of a force history, as
 * 2d_statistics.f90 computes them: period = distance of the first two strict local maxima of
 * the lift (find_peaks, 2d_statistics.f90:183-214), averages over the n_cycle whole cycles
 * after the first peak (2d_statistics.f90:90-131), forces normalised by
 * 0.5 rho_infty uo^2 (2 r_cy) (2d_statistics.f90:28-32).  Host-only; returns MRLBM_ESTATE
 * where the reference stops with "Could not detect two peaks". */
int mrlbm_force_statistics(const double* f_drag, const double* f_lift, int32_t nstep,
                           double r_cy, double uo, double rho_infty,
                           double* St, double* Cd_mean, double* Cl_rms,
                           int32_t* cycle_start, int32_t* period, int32_t* n_cycle);

/* Cycle-averaged surface pressure coefficient Cp(k), k = 1..nbct (2d_statistics.f90:114-122);
 * p_surface is the step-major history (nstep x nbct) of the surface pressure records
 * (data_mean/p_surface_time.dat, 2d_mrlbm.f90:609-612). Host-only. */
int mrlbm_cp_statistics(const double* p_surface, int32_t nstep, int32_t nbct,
                        int32_t cycle_start, int32_t period, int32_t n_cycle,
                        double rho_infty, double uo, double* cp);

/* Step without any device allocation by this library (no counterpart in the reference).
 *
 * For hosts that own all device memory themselves and cannot let a library call cudaMalloc:
 * a Fortran host whose device arrays come from its CUDA Fortran or OpenACC runtime, a
 * framework whose caching allocator or arena holds the GPU, a service that freezes
 * allocation after start-up.  `h` is a host-only handle (mrlbm_create with device -1, which
 * allocates no device memory); the caller passes
 *   d_state  device buffer of info.state_bytes bytes (both time levels, the padded layout of
 *            mrlbm_geometry_info; FP64 values, or FP32 deviations f_k - w_k),
 *   d_f0     device array f(nx,ny,0:8) (Fortran order, FP64) to start from, or NULL to
 *            continue from the state left in d_state by the previous call,
 *   records  host array of nsteps * 4 doubles receiving (iter, F_drag_net, F_lift_net,
 *            sum(rho(1,:))) for each stats step; *n_records receives the count.
 * The handle's mrlbm_get_state returns the configured initial populations to seed d_f0.
 * Everything else the step kernel uses (its force-reduction partials and arrival counter,
 * the per-step records, the curved-wall tables) lives in fixed-size file-scope device arrays
 * of about 2 MB that every GPU loading this library holds until the process exits.  Limits:
 * at most 1024 curved-wall nodes, 8192 rows and a cylinder bounding box of at most 512 x 512
 * cells; larger cases are rejected with MRLBM_EINVAL.  d_state must be 16-byte aligned (the
 * vector tile shapes access it 16 bytes at a time) and d_f0 8-byte aligned; a misaligned
 * pointer (a sub-allocation or a view at an odd offset) is rejected with MRLBM_EINVAL.  The
 * first call on a device looks up the arrays' device addresses (cudaGetSymbolAddress) with
 * that device current and caches them for the life of the process (they assume the device's
 * primary context is not reset meanwhile); make that first call before any stream capture.
 * Every call uploads the case tables from host memory and synchronises cuda_stream at its end,
 * to read the device error flag and the step records.  All calls share the arrays and
 * re-upload the case tables and clear the counters each time, so calls that overlap on the
 * GPU (other streams or other host threads using the same device) race; serialise them.
 * Allocates nothing: no cudaMalloc, cudaFree or allocating library routine on any path. */
int mrlbm_step_noalloc(mrlbm_handle* h, void* d_state, const double* d_f0, int32_t nsteps,
                       double* records, int32_t* n_records, void* cuda_stream);

/* Bulk tile shape of the step kernel.  Shapes 0..9 are one-tile-per-block grids (threads per
 * block, rows per thread, register budget; TILE_CFGS in mrlbm_2d_b200/csrc/step_params.h);
 * shapes 10..15 are persistent blocks fed by tensor copies (TMA) with several tiles in flight
 * (TMA_CFGS there); shapes 16..21 read and write 16 bytes per lane and plane, with the
 * neighbouring columns exchanged by warp shuffles (MRLBM_VEC_LIST there); shapes 22..26 are
 * resident grids that walk the rows with the next node's loads issued before the current
 * node's arithmetic (MRLBM_PIPE_LIST there); shapes 27..30 are TMA shapes whose fully interior
 * tiles are written back by tensor stores from a shared-memory output tile (MRLBM_TMAS_LIST).
 * Every shape computes the same bits.  The default is 1; MRLBM_TILE_CFG in
 * the environment overrides it at creation.  A shape that does not fit the handle's precision
 * makes the next mrlbm_step return MRLBM_EUNSUPPORTED.  mrlbm_step_noalloc runs shape 1 when a
 * TMA shape is selected (its counters live in the handle). */
#define MRLBM_N_TILE_CONFIGS 31
int mrlbm_set_tile_config(mrlbm_handle* h, int32_t cfg);
int mrlbm_get_tile_config(const mrlbm_handle* h, int32_t* cfg);

/* Autotuner: time every tile shape for trial_steps steps on this handle's own case (after one
 * warm-up step each), keep the fastest, and restore the populations, the iteration counter
 * and the force history, so a simulation is unaffected.  Trial steps record no surface
 * pressure; with a field-statistics window they accumulate like the run will (so the choice
 * fits it) into sums that are saved beforehand and put back.  Returns the chosen shape and its
 * time per step in milliseconds. */
int mrlbm_autotune(mrlbm_handle* h, int32_t trial_steps, int32_t* best_cfg, double* best_ms);

/* Field statistics (no counterpart in the reference, whose 2d_statistics post-processes
 * forces only): every step whose iteration lies in [begin_iter, end_iter] adds the
 * post-closure u, v and p = rho cs2 (cs2 = 1/3, 2d_mrlbm.f90:153, 237) of every node to FP64
 * running sums of x and x^2, fused into the step kernel (+96 bytes per node and step).  A call
 * clears the sums and sets the window; iterations are those of mrlbm_get_iter. */
int mrlbm_field_stats_window(mrlbm_handle* h, int32_t begin_iter, int32_t end_iter);

/* Time-mean and fluctuation rms, sqrt(max(<x^2> - <x>^2, 0)), of u, v and p over the steps
 * accumulated so far, each nx*ny in Fortran order; any pointer may be NULL.  n_samples
 * receives the number of steps.  MRLBM_ESTATE before the first step in the window. */
int mrlbm_field_stats_get(mrlbm_handle* h, double* mean_u, double* mean_v, double* mean_p, double* rms_u,
                          double* rms_v, double* rms_p, int64_t* n_samples);

/* ---- surface pressure and probes (write_statistics_out and the probe files) -------------
 * When enabled, every statistics step (post_process, statsbegin <= iter <= statsend) also
 * records, from the populations that step gathers: the wall pressure p = rho cs2 extrapolated
 * quadratically in r from reference points 2, 3 and 4 (extrapolate_var_on_cylinder,
 * 2d_mrlbm.f90:619-672), ordered by theta (the rows of data_mean/p_surface_time.dat,
 * 2d_mrlbm.f90:602-612); its Gaussian smoothing over theta, sigma = 0.1 (gaussian_smoothing,
 * 2d_mrlbm.f90:718-740, p_surface_smooth_time.dat); and the four probes' rho/3, ux/3, uy/3
 * (the data_probe files, 2d_mrlbm.f90:468-476; probe nodes 2d_mrlbm.f90:102-109, or 1, 1.5, 2 and
 * 2.5 diameters behind the centre, one row above it, for explicit geometry). */
int mrlbm_surface_enable(mrlbm_handle* h, int32_t enable);
int mrlbm_get_probe_nodes(const mrlbm_handle* h, int32_t* pi, int32_t* pj);
/* Drain up to cap records: iter[r], p_surface[r*nbct + k], p_smooth[r*nbct + k] (k in theta
 * order) and probes[r*12 + q] = (p1..p4, ux1..ux4, uy1..uy4); any array may be NULL. */
int mrlbm_get_surface(mrlbm_handle* h, int32_t* iter, double* p_surface, double* p_smooth, double* probes,
                      int32_t cap, int32_t* n);

/* ---- body force and the adjoint of mean drag (no counterpart in the reference) ----------
 * Body force: g (2 x nx*ny, x components then y, Fortran node order) adds the momentum
 * source fout_k += 3 w_k (c_k . g) after collision at every bulk and edge node (not at
 * curved-wall nodes); NULL removes it.  An extension: the reference has no forcing term. */
int mrlbm_set_body_force(mrlbm_handle* h, const double* g);

/* Gradient of J = mean net drag over the last `window` of the next `nsteps` steps, from the
 * handle's current state (the handle is not advanced), with respect to the body force (grad_body,
 * 2 x nx*ny) and the inlet profile u_in(j) (grad_uin, ny; the uniform inlet value when no
 * profile is set).  Discrete adjoint of the FP64 step: a forward pass keeps a checkpoint every
 * checkpoint_every steps; the backward pass recomputes each segment from its checkpoint and runs
 * the adjoint kernels step by step.  Either gradient pointer may be NULL; both NULL computes J
 * only.  Every wall, edge-closure, collision and curved-wall closure option of the step is
 * differentiated; x-periodic lattices (no inlet or outlet) and x-slab handles return
 * MRLBM_EUNSUPPORTED.  On an FP32 handle the trajectory is the
 * FP32 step's (checkpoints in FP32) and the adjoint arithmetic is FP64.  The device workspace
 * (nsteps / checkpoint_every + 2 x checkpoint_every population levels, two FP64 adjoint levels)
 * is allocated by the first call, grown when a later call needs more, and kept until
 * mrlbm_destroy; the backward pass recomputes the next segment on a second stream while the
 * adjoint kernels sweep the current one. */
int mrlbm_adjoint_drag(mrlbm_handle* h, int32_t nsteps, int32_t window, int32_t checkpoint_every, double* J,
                       double* grad_body, double* grad_uin);

/* ---- x-slabs of one domain (no counterpart in the reference, which runs on one node) ----
 * mrlbm_create_slab builds the handle of global columns gx0..gx1 (1-based, at least 4) of the
 * domain cfg describes; its lattice is that slab, with column 0 / nx+1 holding the incoming
 * populations of the left / right neighbour when gx0 > 1 / gx1 < global nx.  Geometry and
 * initial state are the domain's, sliced; the cylinder and its bilinear stencils must lie
 * strictly inside one slab.  After every step the neighbours exchange one halo column per face
 * (3 x ny values: the populations crossing the face), either through mrlbm_slabs_step
 * (slabs of one process, on one or several devices) or through mrlbm_halo_pack /
 * mrlbm_halo_unpack around the caller's own transport (e.g. NCCL send/recv between ranks).
 * Force records: the slab holding the cylinder has the drag and lift, the slab holding column
 * 1 the inlet density; the others record zeros.  Every slab's populations equal the
 * corresponding columns of the single-domain run bit for bit. */
int mrlbm_create_slab(const mrlbm_config* cfg, int precision, int device, int32_t gx0, int32_t gx1,
                      mrlbm_handle** out);
/* Values per halo face (3 x ny) and the bytes per value (the handle's storage type). */
int mrlbm_halo_size(const mrlbm_handle* h, int64_t* n_values, int32_t* elem_bytes);
/* side 0 = left face, 1 = right face.  pack copies the outgoing populations of the current
 * state into device buffer dst; unpack copies a neighbour's packed face into the ghost column
 * (both ordered on the handle's stream). */
int mrlbm_halo_pack(mrlbm_handle* h, int32_t side, void* dst);
int mrlbm_halo_unpack(mrlbm_handle* h, int32_t side, const void* src);
/* Exchange overlapped with the step.  mrlbm_step_faces computes the halo-face columns (1 on a
 * left halo face, nx on a right one) of the next step into the next time level, on the
 * handle's stream; mrlbm_step then computes the whole slab and writes the same bits again.
 * Between the two, mrlbm_halo_pack_next / mrlbm_halo_unpack_next (same layout as pack /
 * unpack, on the handle's stream) can move the faces of that next level while the step runs
 * elsewhere: per step, step_faces; on a second stream ordered after it, pack_next, the
 * transport and the neighbour's unpack_next into its next level; mrlbm_step; the next
 * step_faces waits for the second stream. */
int mrlbm_step_faces(mrlbm_handle* h);
int mrlbm_halo_pack_next(mrlbm_handle* h, int32_t side, void* dst);
int mrlbm_halo_unpack_next(mrlbm_handle* h, int32_t side, const void* src);
/* Advance adjacent slabs (given left to right) nsteps steps with the halo exchange between
 * them (device-to-device copies; peer copies across devices), each slab's faces computed
 * first and copied on a second stream while its step kernel runs.  Synchronises at the end. */
int mrlbm_slabs_step(mrlbm_handle** hs, int32_t n, int32_t nsteps);

/* ---- batched cases (no counterpart in the reference, which runs one case per process) ----
 * Many independent cases of one precision on one device advance together: one kernel covers
 * the work of every case, either as a persistent cooperative launch that loops over steps
 * with a grid barrier (MRLBM_BATCH_PERSISTENT, steps_per_launch steps per launch) or as one
 * launch per step captured once into a CUDA graph of steps_per_launch launches and replayed
 * (MRLBM_BATCH_GRAPH); or each case's own single-case step launches run on a stream of the
 * case's own, steps_per_launch steps per case captured into one graph and replayed with the
 * per-call iteration and record slots uploaded before each replay (MRLBM_BATCH_STREAMS; a call
 * with macroscopic output, field statistics or a loaded state's first step runs as
 * MRLBM_BATCH_GRAPH instead).  Each case's results are bit-identical to stepping it alone.  The
 * cases are ordinary handles owned by the batch (mrlbm_batch_case): read their forces,
 * fields and state, load states, set inlet profiles and field-statistics windows with the
 * single-case calls, but step them only through mrlbm_batch_step and do not destroy them.
 * Surface-pressure records (mrlbm_surface_enable) are taken by single-case steps only: a
 * batch step with such a case returns MRLBM_EUNSUPPORTED. */
typedef struct mrlbm_batch mrlbm_batch;
#define MRLBM_BATCH_PERSISTENT 0
#define MRLBM_BATCH_GRAPH      1
#define MRLBM_BATCH_STREAMS    2

int mrlbm_batch_create(const mrlbm_config* cfgs, int32_t ncases, int precision, int device, mrlbm_batch** out);
int mrlbm_batch_destroy(mrlbm_batch* b);
int mrlbm_batch_case(mrlbm_batch* b, int32_t c, mrlbm_handle** h);
/* Advance every case by nsteps (flags: MRLBM_STEP_MACRO stores each case's fields on the last). */
int mrlbm_batch_step(mrlbm_batch* b, int32_t nsteps, int32_t flags);
/* tile_cfg: a 128-bit vector shape (16..21) for MRLBM_BATCH_PERSISTENT; a vector or a
 * one-tile-per-block shape (0..9) for MRLBM_BATCH_GRAPH; a one-tile-per-block shape for
 * MRLBM_BATCH_STREAMS.  steps_per_launch: 1..8192 (1..1024 for MRLBM_BATCH_STREAMS, whose graph
 * holds a launch per case and step). */
int mrlbm_batch_set_schedule(mrlbm_batch* b, int32_t tile_cfg, int32_t schedule, int32_t steps_per_launch);
int mrlbm_batch_get_schedule(const mrlbm_batch* b, int32_t* tile_cfg, int32_t* schedule, int32_t* steps_per_launch);
/* Time every shape under every schedule that takes it for trial_steps steps (rounded up to
 * even; states, counters and histories restored afterwards) and keep the fastest; returns its
 * time per batch step. */
int mrlbm_batch_autotune(mrlbm_batch* b, int32_t trial_steps, double* best_ms_per_step);
/* Watchdog of the persistent schedule: how many times a block polls the grid barrier between
 * two steps before it decides the launch has lost a block, raises MRLBM_EDEVICE_TIMEOUT and
 * ends the launch (every other waiting block follows).  Each poll sleeps about 0.1 us; the
 * default (polls = 0) is 2^24 polls, a few seconds.  A tiny limit makes a healthy launch give up
 * (the timeout path is testable that way); the cases' states are then undefined. */
int mrlbm_batch_set_wait_limit(mrlbm_batch* b, int64_t polls);
/* Sticky status: a grid-barrier timeout (MRLBM_EDEVICE_TIMEOUT) or the first case's error. */
int mrlbm_batch_status(mrlbm_batch* b);
int mrlbm_batch_last_error(const mrlbm_batch* b, char* buf, size_t len);
int mrlbm_batch_launch_count(const mrlbm_batch* b, int64_t* n);
/* The batch's own CUDA stream (all its cases' work is ordered on it), e.g. to time it with events. */
int mrlbm_batch_get_stream(const mrlbm_batch* b, void** stream);

/* Number of kernel launches issued by this handle so far (all kinds). */
int mrlbm_get_launch_count(const mrlbm_handle* h, int64_t* n);

#ifdef __cplusplus
}
#endif
#endif /* MRLBM_H */
