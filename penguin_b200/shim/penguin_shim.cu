// Drop-in shim: keeps the host entry points that PEnGUIn's main.cu calls and
// forwards them to libpenguin_b200's C ABI.  Compile it in the PEnGUIn tree
// (it includes that tree's parameters.h and structs.h) and link main.o, the
// I/O and initialisation objects and libpenguin_b200.so instead of solver.o,
// timestep.o and orbit.o:
//
//   global_dt   (include/timestep.h:4)  -> pg_grid_global_dt
//   solve       (include/solver.h:4)    -> pg_grid_solve
//   init_OrbAdv (include/orbit.h:4)     -> pg_grid_init_orbadv
//
// The compile-time configuration of parameters.h becomes the runtime pg_params
// handed to pg_configure() on first use.
#include <cstdio>
#include <cstdlib>

#include "parameters.h"
#include "structs.h"

// parameters.h configures with macros some of which share names with pg_params
// fields: capture their values, then retire the macros before the C ABI header.
static const int pgs_ndim = ndim;
static const int pgs_geomx = geomx;
static const int pgs_geomy = geomy;
static const int pgs_geomz = geomz;
static const int pgs_eos = EOS_flag;
static const int pgs_ie = internal_e_flag;
static const int pgs_init = init_flag;
#ifdef visc_flag
static const int pgs_visc = 1;
#else
static const int pgs_visc = 0;
#endif
#ifdef OrbAdv_flag
static const int pgs_orbadv = 1;
#else
static const int pgs_orbadv = 0;
#endif
#ifdef kill_flag
static const int pgs_kill = 1;
#else
static const int pgs_kill = 0;
#endif
#ifdef dust_flag
static const int pgs_dust = 1;
#else
static const int pgs_dust = 0;
#endif
#if defined(cool_flag) && cool_flag > 0
static const int pgs_cool = cool_flag;
#else
static const int pgs_cool = 0;
#endif
#if defined(twobd_flag) && twobd_flag == 1
static const int pgs_twobd = 1;
#else
static const int pgs_twobd = 0;
#endif
#undef ndim
#undef geomx
#undef geomy
#undef geomz
#undef EOS_flag
#undef internal_e_flag
#undef init_flag
#undef visc_flag
#undef kill_flag
#undef dust_flag
#undef cool_flag
#undef twobd_flag

#include "penguin_b200.h"

static_assert(sizeof(Grid) == sizeof(pg_grid), "Grid and pg_grid must have the same layout");
static_assert(sizeof(Cell) == sizeof(pg_cell), "Cell and pg_cell must have the same layout");
static_assert(sizeof(body) == sizeof(pg_body), "body and pg_body must have the same layout");

static void pg_shim_configure() {
    static bool done = false;
    if (done) return;
    pg_params P{};
    P.ndim = pgs_ndim;
    P.xres = xres;
    P.yres = yres;
    P.geomx = pgs_geomx;
    P.geomy = pgs_geomy;
    P.gridx = gridx;
    P.gridy = gridy;
    P.xmin = xmin;
    P.xmax = xmax;
    P.ymin = ymin;
    P.ymax = ymax;
    P.eos_flag = pgs_eos;
    P.internal_e_flag = pgs_ie;
    P.gam = gam;
    P.cfl = CFL;
    P.bound_lft = bound_lft;
    P.bound_rgh = bound_rgh;
    P.init_flag = pgs_init;
    P.frame_omega = frame_omega;
    P.p_alpha = p_alpha;
    P.p_beta = p_beta;
    P.ss_alpha = ss_alpha;
    P.sc_h = sc_h;
    P.planet_radius = planet_radius;
    P.visc_flag = pgs_visc;
    P.orbadv_flag = pgs_orbadv;
    P.kill_flag = pgs_kill;
    P.kill_width = kill_width;
    P.kill_width_out = kill_width;
    P.n_planet = pgs_twobd ? 1 : n_planet;  // the two-body frame's n_planet 2 counts the star
    P.planet_mass = planet_mass;
    P.planet_ecc = planet_ecc;
    P.rs_fac = rs_fac;
    P.ramp_time = ramp_time;
    P.zmin = zmin;
    P.zmax = zmax;
    P.dust_flag = pgs_dust;
    P.stokes = Stokes;
    P.d_g_ratio = D_G_ratio;
    P.cool_flag = pgs_cool;
    P.beta_cool = beta_cool;
    P.twobd_flag = pgs_twobd;
    P.zres = zres;
    P.geomz = pgs_geomz;
    P.gridz = gridz;
    P.bound_bom = bound_bom;
    P.bound_top = bound_top;
    if (pg_configure(&P) != PG_OK) {
        fprintf(stderr, "penguin_b200: %s\n", pg_last_error());
        exit(1);
    }
    done = true;
}

static void pg_shim_check(pg_status s) {
    if (s != PG_OK) {
        fprintf(stderr, "penguin_b200: %s\n", pg_last_error());
        exit(1);
    }
}

double global_dt(Grid* hst, Grid* dev, double dt) {
    pg_shim_configure();
    double out = 0.0;
    pg_shim_check(pg_grid_global_dt(reinterpret_cast<pg_grid*>(hst), reinterpret_cast<pg_grid*>(dev), dt, &out));
    return out;
}

void solve(Grid* dev, double time, double dt) {
    pg_shim_configure();
    pg_shim_check(pg_grid_solve(reinterpret_cast<pg_grid*>(dev), time, dt));
}

void init_OrbAdv(Grid* dev) {
    pg_shim_configure();
    pg_shim_check(pg_grid_init_orbadv(reinterpret_cast<pg_grid*>(dev)));
}
