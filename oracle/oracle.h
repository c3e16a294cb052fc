/*
 * CPU oracle for the PEnGUIn Godunov timestep -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64 restatement of the reference's step loop (main.cu:320-360),
 * its Godunov step DS()/solve() (src/solver/solve.cu:212-292) and its CFL
 * reduction global_dt() (src/timestep/timestep.cu:113-140).  It is the checker
 * for the CUDA product path: only tests, the smoke check and the CPU-baseline
 * leg of bench.py may load it.  Nothing in the product calls it.
 *
 * Parity pinning: the oracle is validated against outputs of the reference
 * itself (its own CUDA build, compiled for sm_100a from the unmodified sources
 * and run on a B200 from restart-injected initial states); the fixtures and the
 * script that generated them live under tests/golden/.
 *
 * Known, documented deviations from the GPU reference (all below 1e-12
 * relative in the fixtures):
 *   - killwave's ramp uses the FP32 intrinsic __sinf (src/killwave/killwave.cu:11);
 *     the oracle evaluates sinf() of the same float argument instead;
 *   - nvcc contracts a*b+c into FMA; the oracle is compiled without contraction;
 *   - pow/sin/sincos/atan come from glibc rather than CUDA's libdevice.
 *
 * The parameters are runtime values with the names of include/parameters.h
 * (the reference fixes them at compile time).
 */
#ifndef PENGUIN_ORACLE_H
#define PENGUIN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double r, p, u, v, w; } orc_cell;          /* include/structs.h:48 */
typedef struct { double m, a, e, x, y, z, vx, vy, vz, rs; } orc_body;
typedef struct { double r, u, v, w; } orc_dust;                /* include/structs.h:19 */  /* include/structs.h:105 */

typedef struct {
    int ndim;                 /* 1, 2 or 3 (3: oracle3d.c) */
    int xres, yres;           /* interior cells */
    int geomx, geomy;         /* x: 0 cartesian, 1 cylindrical radius; y: 0 cartesian, 3 azimuth */
    int gridx, gridy;         /* 0 linear, 1 logarithmic */
    double xmin, xmax, ymin, ymax;
    int eos_flag;             /* 0 locally isothermal, 2 adiabatic */
    int internal_e_flag;      /* 0 total energy, 1 internal energy (EOS_flag 2 only) */
    double gam;
    double cfl;
    int bound_lft, bound_rgh; /* 0 analytic init_C, 1 zero gradient, 2 reflecting; y is periodic */
    int init_flag;            /* 2: 2D polar disk (the only analytic state used for ghosts / damping) */
    double frame_omega;
    double p_alpha, p_beta, ss_alpha, sc_h, planet_radius;
    int visc_flag, orbadv_flag, kill_flag;
    double kill_width;        /* inner damping width in units of H(xmin) */
    double kill_width_out;    /* outer damping width in units of H(xmax) (the reference uses kill_width for both) */
    int n_planet;             /* 0 or 1 */
    double planet_mass, planet_ecc, rs_fac, ramp_time;
    double zmin, zmax;        /* only enter through the z grid (2D: unused by the physics) */
    int dust_flag;            /* 1: one pressureless dust fluid (src/solver/dust/dust.cu) */
    double stokes, d_g_ratio; /* Stokes and D_G_ratio of include/parameters.h */
    int cool_flag;            /* 0 off, 1 t_c = beta r^1.5, 2 t_c = beta / r sqrt(p/r) / h (src/solver/cool/cool.cu) */
    double beta_cool;
    int twobd_flag;           /* 1: star and planet orbit their barycentre (src/planet/planet.cu:135-175) */
    int zres, geomz, gridz;   /* ndim 3: polar cells, geometry (0 cartesian, 5 polar angle), grid (0-4) */
    int bound_bom, bound_top; /* ndim 3: polar boundaries at zmin / zmax (0 analytic, 1 zero gradient, 2 reflecting, 3 periodic) */
} orc_params;

typedef struct orc_state orc_state;

orc_state* orc_create(const orc_params* P);
void orc_destroy(orc_state* S);

/* geometry (with ghosts): xa[xarr+1], xv[xarr], ya[yarr+1], yv[yarr] */
int orc_dims(const orc_state* S, int* xarr, int* yarr);
void orc_get_grid(const orc_state* S, double* xa, double* xv, double* ya, double* yv);

/* fill every cell (ghosts included) with init_C (src/init/init.cu:502-519) */
void orc_fill_init(orc_state* S);
/* restart injection: interior fields, x fastest (src/output/output.cu:182-248) */
void orc_set_interior(orc_state* S, const double* r, const double* p, const double* u, const double* v);
void orc_get_interior(const orc_state* S, double* r, double* p, double* u, double* v);
/* the whole AoS array incl. ghosts, xarr*yarr cells */
void orc_get_cells(const orc_state* S, orc_cell* out);
/* dust interior (dust_flag); the dust starts from init_CD (src/init/init.cu:351-454):
   the reference's restart path does not load dust (src/output/output.cu:182-248) */
void orc_set_dust(orc_state* S, const double* r, const double* u, const double* v);
void orc_get_dust(const orc_state* S, double* r, double* u, double* v);

void orc_init_planet(orc_state* S, double t);   /* src/planet/planet.cu:319 */
void orc_init_orbadv(orc_state* S);             /* src/orbit/orbit.cu:51,111 */
void orc_get_planet(const orc_state* S, orc_body* out);

double orc_global_dt(orc_state* S, double dt_prev);  /* src/timestep/timestep.cu:113 */
double orc_torque(const orc_state* S);                /* src/output/output.cu:336-412 */
void orc_solve(orc_state* S, double t, double dt);   /* src/solver/solve.cu:279 */

/* main.cu:320-360 with max_step and end_time: returns steps taken, writes final time and last dt */
int orc_run(orc_state* S, double t0, double dt_prev, int max_step, double end_time, double* t_out, double* dt_out);

/* stages exposed for component parity tests (each acts on the current state like the reference) */
void orc_boundx(orc_state* S, int which);      /* which: 0 = C, 1 = T */
void orc_boundy(orc_state* S, int which);
void orc_viscous_forces(orc_state* S, int which, double* vis_out /* 2*xarr*yarr or NULL */);
void orc_sweepx(orc_state* S, double dt);
void orc_sweepy(orc_state* S, double dt);
int orc_solve_stages(orc_state* S, double t, double dt, orc_cell* out, orc_dust* dout /* or NULL */);

/* ---- ndim 3 (oracle3d.c): the reference's step with the polar sweep ---- */
typedef struct orc3_state orc3_state;
orc3_state* orc3_create(const orc_params* P);
void orc3_destroy(orc3_state* S);
int orc3_dims(const orc3_state* S, int* xarr, int* yarr, int* zarr);  /* returns the ghost width */
void orc3_get_axis(const orc3_state* S, int axis, double* a, double* v);  /* faces arr+1, volumes arr */
void orc3_fill_init(orc3_state* S);
/* interior fields, x fastest, then y, then z (src/output/output.cu:182-248) */
void orc3_set_interior(orc3_state* S, const double* r, const double* p, const double* u, const double* v,
                       const double* w);
void orc3_get_interior(const orc3_state* S, double* r, double* p, double* u, double* v, double* w);
void orc3_init_planet(orc3_state* S, double t);
void orc3_get_planet(const orc3_state* S, orc_body* out);
void orc3_boundx(orc3_state* S);
void orc3_boundy(orc3_state* S);
void orc3_boundz(orc3_state* S);
void orc3_sweepx(orc3_state* S, double dt);
void orc3_sweepy(orc3_state* S, double dt);
void orc3_sweepz(orc3_state* S, double dt);
double orc3_global_dt(orc3_state* S, double dt_prev);
void orc3_solve(orc3_state* S, double t, double dt);
int orc3_run(orc3_state* S, double t0, double dt_prev, int max_step, double end_time, double* t_out, double* dt_out);
/* one step, the cell array after each stage (see oracle3d.c); returns the stage count */
int orc3_solve_stages(orc3_state* S, double t, double dt, orc_cell* out);

#ifdef __cplusplus
}
#endif
#endif
