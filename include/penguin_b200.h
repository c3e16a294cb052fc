/*
 * penguin_b200 -- B200-native (sm_100a) Godunov timestep of the PEnGUIn
 * protoplanetary-disk code, behind a C ABI.
 *
 * Two ways in:
 *
 *  1. The drop-in "grid" entry points replace the reference's host functions
 *     that main.cu's step loop calls, on the caller's own device buffers
 *     (a struct laid out exactly like the reference's Grid, include/structs.h:122-392):
 *        pg_grid_global_dt  <- double global_dt(Grid* hst, Grid* dev, double dt)   include/timestep.h:4
 *        pg_grid_solve      <- void solve(Grid* dev, double time, double dt)        include/solver.h:4
 *        pg_grid_init_orbadv<- void init_OrbAdv(Grid* dev)                          include/orbit.h:4
 *     A C++ shim (penguin_b200/shim/penguin_shim.cu) keeps those original
 *     names so that main.cu relinks unchanged.  The reference fixes its
 *     parameters at compile time in include/parameters.h; here they are
 *     passed once through pg_configure().
 *
 *  2. The handle API (pg_disk_*) owns its buffers: used by the Python binding,
 *     the benchmark and the multi-step device-resident loop (CUDA graph).
 *
 * Every function returns a pg_status; nothing aborts the process.
 */
#ifndef PENGUIN_B200_H
#define PENGUIN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PG_OK = 0,
    PG_ERR_CONFIG = 1,   /* unsupported or inconsistent parameters / sizes */
    PG_ERR_CUDA = 2,     /* a CUDA runtime call failed (pg_last_error() has the text) */
    PG_ERR_NAN = 3,      /* the device error word saw a NaN or non-positive density */
    PG_ERR_TIMEOUT = 4,  /* a bounded device wait gave up */
    PG_ERR_ARG = 5       /* null pointer / bad argument */
} pg_status;

/* One cell, AoS, 5 x FP64 (include/structs.h:48-103). */
typedef struct { double r, p, u, v, w; } pg_cell;
/* Dust cell (include/structs.h:19-46). */
typedef struct { double r, u, v, w; } pg_dust;
/* Planet (include/structs.h:105-120). */
typedef struct { double m, a, e, x, y, z, vx, vy, vz, rs; } pg_body;

/*
 * Runtime copy of include/parameters.h (names kept; see penguin_b200/params.py).
 * kill_width_out is an addition: the reference uses kill_width for both
 * damping zones.
 */
typedef struct {
    int ndim, xres, yres;
    int geomx, geomy, gridx, gridy;
    double xmin, xmax, ymin, ymax;
    int eos_flag, internal_e_flag;
    double gam, cfl;
    int bound_lft, bound_rgh, init_flag;
    double frame_omega;
    double p_alpha, p_beta, ss_alpha, sc_h, planet_radius;
    int visc_flag, orbadv_flag, kill_flag;
    double kill_width, kill_width_out;
    int n_planet;
    double planet_mass, planet_ecc, rs_fac, ramp_time;
    double zmin, zmax;
    int dust_flag;
    double stokes, d_g_ratio;
    /* Newtonian cooling of p/r towards cs^2 (src/solver/cool/cool.cu): cool_flag 0
       off, 1 t_c = beta_cool r^1.5, 2 t_c = beta_cool / Sigma sqrt(p/Sigma) / h */
    int cool_flag;
    double beta_cool;
    /* twobd_flag 1: the star and the planet orbit their barycentre
       (src/planet/planet.cu:135-175) and pull as inertial point masses; with
       n_planet 1 (the planet).  Through pg_grid_* the caller's planets array
       holds the star (planets[0]) and the planet (planets[1]). */
    int twobd_flag;
    /* ndim 3 (spherical r, phi, theta or cartesian x, y, z): polar cells, the
       polar geometry (0 cartesian, 5 polar angle) and grid (0 linear, 1 log,
       2/3/4 the reference's non-uniform spacings, src/geom/geom.cu:35-89), and
       the polar boundaries (bound_bom at zmin, bound_top at zmax: 0 analytic
       state, 1 zero gradient, 2 reflecting, 3 periodic;
       src/boundary/boundary.cu:270-320).  Ignored when ndim < 3. */
    int zres, geomz, gridz;
    int bound_bom, bound_top;
} pg_params;

/*
 * Layout twin of the reference's Grid (include/structs.h:122-183).  Only the
 * members the timestep touches are read: stream, x/y sizes, xa/xv/ya/yv,
 * orb_rot/orb_res/orb_shf/orb_inc, C, T, vis_tensor, planets.  C and T may be
 * swapped by pg_grid_solve exactly as the reference swaps them
 * (src/solver/sweeps.cu:353-355): afterwards C holds the newest state.
 * In 1D and 2D the cells' z-velocity w must be 0, as the reference's own 1D/2D
 * states always hold it (init_C writes 0 and no 1D/2D force changes it): the
 * passes skip its reconstruction and flux there.
 */
typedef struct {
    void* stream; /* cudaStream_t */
    int xbgn, xres, xarr;
    int ybgn, yres, yarr;
    int zbgn, zres, zarr;
    double *xa, *xv, *ya, *yv, *za, *zv;
    double *dt, *sum, *Buff;
    double *orb_rot, *orb_res;
    int *orb_shf, *orb_inc, *shfL, *shfR;
    pg_cell *C, *T, *A;
    pg_dust *CD, *TD;
    pg_cell *BuffL, *BuffR;
    pg_dust *BuffLD, *BuffRD;
    double *vis_tensor, *fx, *fy, *fz, *fx_d, *fy_d, *fz_d, *ext;
    pg_body* planets;
} pg_grid;

/* ------------------------------------------------------------ common */
const char* pg_version(void);
const char* pg_last_error(void);
/* Validate a parameter set without touching the GPU. */
pg_status pg_check_params(const pg_params* P);
/* Host copy of the grid the library builds (src/init/init.cu:472-500):
   xa[xres+7], xv[xres+6], ya[yarr+1], yv[yarr]. */
pg_status pg_make_grid(const pg_params* P, double* xa, double* xv, double* ya, double* yv);

/* ------------------------------------------- drop-in (reference Grid) */
/* Parameters for the pg_grid_* calls (replaces the compile-time parameters.h). */
pg_status pg_configure(const pg_params* P);
/* init_OrbAdv (src/orbit/orbit.cu:51-72,111-120): orb_rot = v_init(r) - r*frame_omega, orb_shf = 0. */
pg_status pg_grid_init_orbadv(pg_grid* dev);
/* global_dt (src/timestep/timestep.cu:113-140): blocking; min(CFL dt, 1.1*dt_prev). */
pg_status pg_grid_global_dt(pg_grid* hst, pg_grid* dev, double dt_prev, double* dt_out);
/* solve (src/solver/solve.cu:279-292): one Godunov step on dev->C, stream-ordered on dev->stream. */
pg_status pg_grid_solve(pg_grid* dev, double time, double dt);
/* Releases the private tables cached for the caller's grids. */
pg_status pg_grid_release(void);

/*
 * No counterpart in the reference.  The CFL step size of global_dt for callers
 * that cannot allocate device memory (their own pool or fixed budget owns the
 * GPU): it reads the caller's state C (xarr*yarr cells), the dust state CD
 * (same layout; required when P->dust_flag is set, ignored otherwise: the dust
 * speeds bound dt as in timestep.cu:64-75), faces xa and ya (ya unused and may
 * be NULL when ndim == 1) and orb_rot (NULL = no orbital advection), and keeps
 * its scratch in a fixed 64 KiB file-scope device array instead of
 * cudaMalloc'd memory.  Grids above 8192*4096 interior cells are rejected
 * (PG_ERR_CONFIG), as is a 1D grid with yres != 1.  The first call on a device
 * resolves the array's device address once, with that device current; a
 * process that resets that device must not call it there again.  Calls that
 * overlap on the GPU share the array and race.
 * Blocking; dt = min(CFL dt, 1.1*dt_prev) like pg_grid_global_dt.
 */
pg_status pg_global_dt_noalloc(const pg_params* P, const pg_cell* C, const pg_dust* CD, const double* xa,
                               const double* ya, const double* orb_rot, double dt_prev, double* dt_out, void* stream);

/* ------------------------------------------------------- handle API */
typedef struct pg_disk pg_disk;

/* Allocates the state (two AoS buffers), scratch and tables on `device`.
   stream may be NULL (the library creates one). */
pg_status pg_disk_create(const pg_params* P, int device, void* stream, pg_disk** out);
pg_status pg_disk_destroy(pg_disk* d);
/* Sizes: interior cells and padded array dims. */
pg_status pg_disk_dims(const pg_disk* d, int* xarr, int* yarr, int* npad);
/* Restart injection from host arrays (yres x xres, x fastest), like load_grid
   (src/output/output.cu:182-248): ghosts take init_C, time is set to t.  v may
   be NULL when ndim == 1.  Also initialises the planet at t (planet.cu:319). */
pg_status pg_disk_set_state(pg_disk* d, double t, const double* r, const double* p, const double* u,
                            const double* v);
/* The newest state back to host arrays; t_out may be NULL. */
pg_status pg_disk_get_state(pg_disk* d, double* r, double* p, double* u, double* v, double* t_out);
/* Autotuner: times every launch configuration of each pass of the step on the
   disk's current state over `reps` launches and keeps the fastest; the state is
   unchanged and results stay bit for bit the same.  The sweeps and the
   residual advection choose a tile variant (pg_sweep_variant: pencils per
   tile, outputs per pencil, cells per thread, TMA stages in flight), every pass
   its CTAs per SM.  It replaces the reference's fixed tiling
   (include/parameters.h:81-97, x_xdiv / x_ydiv / y_xdiv / y_ydiv).  choice (may
   be NULL, 8 ints): the variants of sweep_x, sweep_y, advect, then the CTAs per
   SM of kick1, sweep_x, sweep_y, advect, kick2 (0: all that fit).
   pg_disk_set_tuning applies a choice found earlier. */
pg_status pg_disk_autotune(pg_disk* d, int reps, int* choice);
pg_status pg_disk_set_tuning(pg_disk* d, const int* choice);
/* Tile variant v of the FP64 sweeps and advection (0 .. 9), 6 ints: pencils
   per tile, outputs per pencil, cells per thread, TMA stages, threads per CTA,
   CTAs per SM its registers are compiled for.  PG_ERR_ARG past the last. */
pg_status pg_sweep_variant(int v, int* out6);
/* test support: the per-index 4th-order slope weights the kernels apply in
   direction dir (0 radial, 1 azimuthal) of the grid P builds, 6 per index
   (sL on the three differences left of the cell, then sR), host array of
   6 * (xres + 6) or 6 * (yres + 6) doubles.  The reference evaluates the same
   slopes per call (src/solver/recon/recon.cu:216-378).  Uses the GPU. */
pg_status pg_recon_weights(const pg_params* P, int dir, double* w);
/* Snapshots in the reference's checkpoint format (write_check_point /
   load_grid, src/output/output.cu:125-248; file names binary_<label>_<frame>,
   main.cu:403): t, interior faces, r, p, u, v (2D), then the dust fields.
   average = 1 writes the time average (ave_flag).  Reading restarts the disk
   from t and the gas fields. */
pg_status pg_disk_write_snapshot(pg_disk* d, const char* path, int average);
pg_status pg_disk_read_snapshot(pg_disk* d, const char* path, double* t_out);
/* ave_flag: the gas state averaged over a save interval by the trapezoid rule
   of main.cu:343-351, accumulated inside the step; interval <= 0: off.
   reset = init_average after a save. */
pg_status pg_disk_set_average(pg_disk* d, double interval);
pg_status pg_disk_reset_average(pg_disk* d);
pg_status pg_disk_get_average(pg_disk* d, double* r, double* p, double* u, double* v);
/* dust_flag: the interior dust (density, radial and azimuthal velocity, host
   arrays of xres*yres) of the newest state.  pg_disk_set_state resets the dust
   to init_CD, as the reference's restart does (load_grid reads the gas only,
   src/output/output.cu:182-248); pg_disk_set_dust then overwrites it. */
pg_status pg_disk_set_dust(pg_disk* d, const double* r, const double* u, const double* v);
pg_status pg_disk_get_dust(pg_disk* d, double* r, double* u, double* v);
/* Device pointer of the newest AoS state (xarr*yarr pg_cell) and of the scratch. */
pg_status pg_disk_state_ptr(pg_disk* d, pg_cell** cells);
/* global_dt (blocking) and one step with host-supplied t, dt, as in main.cu.
   pg_disk_solve launches the step as one kernel taking t and dt and one CUDA
   graph of the rest, captured on the disk's stream at the first call from
   each of the two state buffers: call it outside a stream capture. */
pg_status pg_disk_global_dt(pg_disk* d, double dt_prev, double* dt_out);
pg_status pg_disk_solve(pg_disk* d, double t, double dt);
/* main.cu's loop (main.cu:320-360) driven from the host, as pg_disk_global_dt and
   pg_disk_solve called once per step: dt read back every step and clipped at
   end_time, at most max_step steps.  *t, *dt: the time and the previous step on
   entry (*dt 0: the first step is capped by end_time - t), the new ones on
   return; *n: the steps taken. */
pg_status pg_disk_step_host(pg_disk* d, int max_step, double end_time, double* t, double* dt, int* n);
/* main.cu's loop on the device: nsteps of (dt = min(CFL dt, 1.1 dt_prev), clipped
   at end_time; solve; t += dt) with dt and t resident in device memory and the
   step captured in a CUDA graph.  Stream-ordered; pg_disk_sync waits.  A run
   continuing one that stopped on a clip at its end_time caps its first dt by
   the step the clip replaced, as main.cu does after a dump (main.cu:333-338). */
pg_status pg_disk_run(pg_disk* d, int nsteps, double end_time);
pg_status pg_disk_sync(pg_disk* d);
/* Time, last dt and step count of the device-resident loop (syncs). */
pg_status pg_disk_clock(pg_disk* d, double* t, double* dt, long long* steps);
/* Planet state (syncs). */
pg_status pg_disk_planet(pg_disk* d, pg_body* out);
/* Device error word: 0 or a pg_status; cleared by the call (syncs). */
pg_status pg_disk_check(pg_disk* d);
/* Torque of the planet on the disk, sum of r g_phi Sigma dV over the interior
   with the current planet (src/output/output.cu:336-412, global_sum; main.cu
   prints it divided by q^2/h^2).  2D polar disks with a planet; FP64 with
   compensated per-thread sums; syncs. */
pg_status pg_disk_torque(pg_disk* d, double* torque);
/* Launch count of the library's own kernels per step (for reporting). */
int pg_kernels_per_step(const pg_disk* d);
/* Runs nsteps of the device-resident loop launching the kernels one by one with
   CUDA events between them on the disk's stream; ms[k] receives the average
   milliseconds per step of stage k (0 time, 1 kick1, 2 sweep_x, 3 sweep_y,
   4 advect, 5 kick2; absent stages get 0).  nslot >= 6.  Blocking. */
pg_status pg_disk_profile(pg_disk* d, int nsteps, double end_time, float* ms, int nslot);

/* ------------------------------------------- FP32-mixed ensembles of disks
 * No counterpart in the reference, which runs one compile-time configured disk
 * per process.  n planet-disks (each its own pg_params: size, q, alpha, h/r ...)
 * advanced together by the FP32-mixed step: FP32 residual state against the
 * FP64 initial disk, FP32 reconstruction and HLLC in deviation form, FP64
 * orbital shift, dt and totals.  One persistent launch per pass for all disks;
 * the step is a CUDA graph.  Each disk keeps its own clock and CFL dt.  Only
 * polar, isothermal disks with analytic radial boundaries and orbital advection
 * (the planet-disk family) are accepted: PG_ERR_CONFIG otherwise. */
typedef struct pg_ens pg_ens;

/* Validates n parameter sets for the FP32 form (no GPU needed). */
pg_status pg_ens_check_params(const pg_params* P, int n);
pg_status pg_ens_create(const pg_params* P, int n, int device, void* stream, pg_ens** out);
pg_status pg_ens_destroy(pg_ens* e);
int pg_ens_size(const pg_ens* e);
pg_status pg_ens_dims(const pg_ens* e, int k, int* xres, int* yres);
/* Disk k's state from host arrays of xres*yres interior cells (density,
   radial and azimuthal velocity; the pressure is cs^2 Sigma); v may be NULL
   (the initial disk's v).  Blocking. */
pg_status pg_ens_set_state(pg_ens* e, int k, double t, const double* r, const double* u, const double* v);
pg_status pg_ens_get_state(pg_ens* e, int k, double* r, double* p, double* u, double* v, double* t_out);
/* nsteps steps of every disk (each with its own dt, clipped at end_time; a disk
   that reached end_time stays unchanged).  Stream-ordered; pg_ens_sync waits. */
pg_status pg_ens_run(pg_ens* e, int nsteps, double end_time);
pg_status pg_ens_sync(pg_ens* e);
pg_status pg_ens_clock(pg_ens* e, int k, double* t, double* dt, long long* steps);
pg_status pg_ens_planet(pg_ens* e, int k, pg_body* out);
/* Device error words of all disks, cleared by the call (syncs). */
pg_status pg_ens_check(pg_ens* e);
/* Disk k's mass sum(Sigma dV) and angular momentum sum(Sigma r v dV), FP64
   with compensated summation (syncs). */
pg_status pg_ens_totals(pg_ens* e, int k, double* mass, double* angmom);
/* Disk k's torque of the planet on the disk, as pg_disk_torque (syncs). */
/* dust_flag members (one pressureless dust fluid, FP32-mixed like the gas):
   the interior dust r, v_r, v_phi of the newest state; set_state resets it to
   init_CD. */
pg_status pg_ens_set_dust(pg_ens* e, int k, const double* r, const double* u, const double* v);
pg_status pg_ens_get_dust(pg_ens* e, int k, double* r, double* u, double* v);
pg_status pg_ens_torque(pg_ens* e, int k, double* torque);
int pg_ens_kernels_per_step(const pg_ens* e);
/* As pg_disk_profile, for the whole ensemble (slots 0 clocks + planet tables,
   1 kick1, 2 sweep_x, 3 sweep_y, 4 advect, 5 kick2). */
pg_status pg_ens_profile(pg_ens* e, int nsteps, double end_time, float* ms, int nslot);
/* Launch-configuration autotuner of the five FP32 passes: for each pass the
   compiled occupancy variant (0/1) and CTAs-per-SM cap (0 = none) with the
   shortest time on the current state, `reps` launches per candidate.  The
   state is not changed and results are bit for bit the same under any choice.
   out10 (optional): variants of kick1, sweep x, sweep y, advect, kick2, then
   their caps. */
pg_status pg_ens_autotune(pg_ens* e, int reps, int* out10);
pg_status pg_ens_set_tuning(pg_ens* e, const int* in10);

/* ---------------------------------------------------------------- adjoint
 * Gradient of a loss on the surface density after N steps of the FP64 step
 * with respect to the initial surface density field and (q, alpha, h/r).  No
 * reference counterpart: the reference has no derivative code.  Covers 2D
 * polar isothermal disks with analytic radial boundaries, no wave damping and
 * at most one planet on a circular orbit (pg_adj_check_params).  The run
 * starts from Sigma0 with v_r = 0 and v_phi = the disk's init_C; dt is the
 * CFL schedule of the recorded forward run (frozen for differentiation).
 * Device arrays are interior fields of xres*yres doubles, index i + xres*j. */
typedef struct pg_adj pg_adj;
pg_status pg_adj_check_params(const pg_params* P);
pg_status pg_adj_create(const pg_params* P, int device, void* stream, int checkpoint_every, pg_adj** out);
pg_status pg_adj_destroy(pg_adj* a);
/* new (q, alpha, h/r): the disk's tables and their derivatives are rebuilt; a
   recorded schedule stays valid for replay */
pg_status pg_adj_set_params(pg_adj* a, double q, double alpha, double h);
/* nsteps of main.cu's loop from Sigma0 at t0; replay = 0 records the CFL dt
   schedule, 1 reuses it (finite-difference checks); Sigma after the run into
   sigma_out (device, may be NULL) */
pg_status pg_adj_forward(pg_adj* a, const double* sigma0, double t0, int nsteps, int replay, double* sigma_out);
/* dL/dSigma (device) -> dL/dSigma0 (device, may be NULL), dL/d(q, alpha, h)
   (host double[3], may be NULL) for the last forward run */
pg_status pg_adj_backward(pg_adj* a, const double* grad_out, double* grad_sigma0, double* grad_theta);
/* test support: one step with dt from the newest state; the adjoint's
   restatement of each pass against the production kernels (max relative
   difference per pass: kick1, sweep_x, sweep_y, advect, kick2) */
pg_status pg_adj_model_error(pg_adj* a, double dt, double* err5);
/* test support: adjoint dot-product test of every pass over one step with dt
   from the newest state.  dir, lam: device, 5 interior planes (Sigma, v_r,
   v_phi, kick1's force x, y).  out10[2p] = <lam, J_p dir> (forward mode),
   out10[2p+1] = <J_p^T lam, dir> (the adjoint), p = kick1, sweep_x, sweep_y,
   advect, kick2 */
pg_status pg_adj_dot_test(pg_adj* a, double dt, const double* dir, const double* lam, double* out10);
/* test support: the tangent of every pass (forward mode on the restated pass)
   against central differences of the production kernel itself over one step
   with dt from the newest state; err30[3p + f] = |fd - tangent|_2 / |tangent|_2
   for f = Sigma, v_r, v_phi; err30[15 + 3p + f] the same with central
   differences of the restated pass.  Overwrites the disk's state. */
pg_status pg_adj_pass_check(pg_adj* a, double dt, double eps, const double* dir, double* err30);
/* test support: each production pass re-run on its recorded input against its
   recorded output over one step with dt (max relative difference per pass) */
pg_status pg_adj_replay_diff(pg_adj* a, double dt, double* diff5);
/* test support: one pass over one step with dt from the newest state; the
   production outputs for the inputs +- eps dir (fd: 6 interior planes, plus
   then minus) and the tangent along dir (tlm5: 5 planes).  Overwrites the
   disk's state. */
pg_status pg_adj_pass_fields(pg_adj* a, int pass, double dt, double eps, const double* dir, double* fd, double* tlm5);
pg_status pg_adj_schedule(const pg_adj* a, double* dts, int n);
int pg_adj_steps(const pg_adj* a);
long long pg_adj_device_bytes(const pg_adj* a);
/* The face fluxes of the sweeps are transposed by hand-written reverse-mode
   kernels (hand = 1, the default) or by the dual-number kernels (hand = 0,
   kept as their check).  Both give the same gradient to rounding. */
pg_status pg_adj_set_sweep_reverse(pg_adj* a, int hand);

/* ------------------------------------------------------ 3D (ndim 3) */
/*
 * One 3D grid on one B200: the reference's DS() with the polar sweep
 * (src/solver/solve.cu:212-292 with ndim 3; sweepz_inplace, src/solver/sweeps.cu:
 * 458-554) on the spherical (r, phi, theta) grid of its 3D preset
 * (include/para_files/Adiabatic_CPD.h: geomx 2, geomy 4, geomz 5) or on a
 * cartesian box (0, 0, 0); ideal or isothermal gas, a periodic azimuth, radial
 * boundaries 0-2 and polar boundaries 0-3 (bound_bom, bound_top), optional
 * planet and wave damping; no viscosity, orbital advection, dust, cooling or
 * two-body frame (PG_ERR_CONFIG).  Fields are interior arrays of
 * xres*yres*zres values, x fastest, then y, then z (the checkpoint order of
 * src/output/output.cu:95-123).
 */
typedef struct pg_disk3 pg_disk3;
pg_status pg_disk3_create(const pg_params* P, int device, void* stream, pg_disk3** out);
pg_status pg_disk3_destroy(pg_disk3* d);
/* Restart injection (load_grid, src/output/output.cu:182-248): ghosts take
   init_C, time is set to t, the planet is initialised at t. */
pg_status pg_disk3_set_state(pg_disk3* d, double t, const double* r, const double* p, const double* u,
                             const double* v, const double* w);
pg_status pg_disk3_get_state(pg_disk3* d, double* r, double* p, double* u, double* v, double* w, double* t_out);
/* global_dt (src/timestep/timestep.cu:113-140, ndim 3): min(CFL dt, 1.1 dt_prev); blocking. */
pg_status pg_disk3_global_dt(pg_disk3* d, double dt_prev, double* dt_out);
/* solve (src/solver/solve.cu:279-292) with host t and dt; stream-ordered. */
pg_status pg_disk3_solve(pg_disk3* d, double t, double dt);
/* nsteps of main.cu's loop (main.cu:320-360) with t, dt and the planet on the
   device, each step replayed as a CUDA graph; stream-ordered. */
pg_status pg_disk3_run(pg_disk3* d, int nsteps, double end_time);
pg_status pg_disk3_clock(pg_disk3* d, double* t, double* dt, long long* steps);
/* Synchronises and reports (then clears) the device error word. */
pg_status pg_disk3_check(pg_disk3* d);
/* nsteps device-clocked steps with CUDA events between the passes: average ms
   of the clock, kick1, sweep_x, sweep_y, sweep_z and kick2 (ms6). */
pg_status pg_disk3_pass_times(pg_disk3* d, int nsteps, double* ms6);
/* Checkpoint files in the reference's format (write_check_point / load_grid,
   src/output/output.cu:125-248, ndim 3): t, the x, y, z faces, then the r, p,
   u, v, w planes.  read_snapshot restarts from the file at its t. */
pg_status pg_disk3_write_snapshot(pg_disk3* d, const char* path);
pg_status pg_disk3_read_snapshot(pg_disk3* d, const char* path, double* t_out);
/* test support: the passes' bounded wait on a tile copy that is never issued
   (one CTA).  err_bits: the device error word afterwards (PG_ERR_TIMEOUT's bit
   set when the wait gave up); left: 1 when the CTA left through the timed-out
   path; ms: the kernel's duration (the wait's limit is 50 ms, then up to 50 ms
   more for copies in flight). */
pg_status pg_test_bounded_wait(int* err_bits, int* left, float* ms);
/* test support: out2[2k] = the kernels' division-free x[k] / 1.5, out2[2k+1] =
   the IEEE quotient, for n host values.  Uses the GPU. */
pg_status pg_test_div_1p5(const double* x, long long n, double* out2);
/* test support: one step with host t and dt, the whole cell array (ghosts
   included) after each pass into out[5][zarr][yarr][xarr]: kick1, sweep_x,
   sweep_y, sweep_z, kick2 with the damping.  Blocking. */
pg_status pg_disk3_stages(pg_disk3* d, double t, double dt, pg_cell* out);
/* Host copy of one axis of the grid the library builds (src/init/init.cu:472-500
   with src/geom/geom.cu): axis 0 x, 1 y, 2 z; faces a[arr+1], volumes v[arr]. */
pg_status pg_make_axis(const pg_params* P, int axis, double* a, double* v);

#ifdef __cplusplus
}
#endif
#endif
