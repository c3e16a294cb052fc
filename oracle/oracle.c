/*
 * CPU oracle for the PEnGUIn Godunov timestep -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for scope and the list of known deviations from the GPU
 * reference.  Every function cites the reference file:line it restates; the
 * floating-point expressions keep the reference's operation order so that
 * differences stay at the rounding level.  Compile without FMA contraction.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NPAD 3  /* recon_flag 6 -> npad 3 (include/parameters.h:49-53) */

static const double PI = 3.1415926535897932384626434;
#define HPI (0.5 * PI)
#define TWOPI (2.0 * PI)
static const double SMALLP = 1.0e-10, SMALLR = 1.0e-10;

struct orc_state {
    orc_params P;
    int xarr, yarr, ypad;
    double *xa, *xv, *ya, *yv, *za, *zv;
    orc_cell *C, *T;
    orc_dust *CD, *TD;   /* dust_flag only */
    double *vis;
    double *orb_rot, *orb_res;
    int *orb_inc;
    orc_body planet;
    orc_body star;       /* twobd_flag: planets[0] of the reference (planet = planets[1]) */
};

#define IND(S, i, j) ((i) + (S)->xarr * (j))

/* ------------------------------------------------------------------ grid */
/* src/geom/geom.cu:3-33 */
static double get_dv_dr(int geom, double ra, double dr)
{
    if (geom == 2) return ra * ra + ra * dr + dr * dr / 3.0;
    else if (geom == 1) return ra + dr / 2.0;
    return 1.0;
}
static double get_volume(int geom, double ra, double dr) { return dr * get_dv_dr(geom, ra, dr); }

/* src/init/init.cu:472-500 (linspace/logspace from src/geom/geom.cu:22-33) */
static void make_grid(double* a, double* v, double amin, double amax, int res, int pad, int geom, int grid)
{
    int len = res + 1;
    if (grid == 1) {
        double tmp = log(amax / amin);
        for (int i = 0; i < len; i++) a[pad + i] = amin * exp(tmp * (double)i / (double)(len - 1));
    } else {
        for (int i = 0; i < len; i++) a[pad + i] = amin + (amax - amin) * (double)i / (double)(len - 1);
    }
    for (int i = 0; i < pad; i++) {
        if (grid == 1) {
            a[i] = amin * exp(log(amax / amin) * (double)(i - pad) / (double)(res));
            a[res + pad + 1 + i] = amin * exp(log(amax / amin) * (double)(res + 1 + i) / (double)(res));
        } else {
            a[i] = a[pad] - (a[2 * pad - i] - a[pad]);
            a[res + pad + 1 + i] = a[res + pad] + (a[res + pad] - a[res + pad - 1 - i]);
        }
    }
    for (int i = 0; i < res + 2 * pad; i++) v[i] = get_volume(geom, a[i], a[i + 1] - a[i]);
}

static double xc(const orc_state* S, int i) { return 0.5 * (S->xa[i + 1] + S->xa[i]); }
static double yc(const orc_state* S, int j) { return 0.5 * (S->ya[j + 1] + S->ya[j]); }

/* ------------------------------------------------------- analytic state */
/* src/init/init.cu:7-17 */
static double get_cs2(const orc_params* P, double x)
{
    double coeff = P->sc_h * P->sc_h * (1.0 / P->planet_radius);
    if (P->geomx == 0) return coeff;
    return coeff * pow(x / P->planet_radius, -P->p_beta);
}
/* src/init/init.cu:20-29 */
static double get_h(const orc_params* P, double x)
{
    if (P->geomx == 0) return P->sc_h;
    return sqrt(get_cs2(P, x) * pow(x, 3));
}
/* src/init/init.cu:31-50 */
static double get_nu(const orc_params* P, double x)
{
    if (!P->visc_flag) return 0.0;
    double coeff = P->ss_alpha * sqrt(get_cs2(P, P->planet_radius)) * get_h(P, P->planet_radius);
    if (P->geomx == 0) return coeff;
    return coeff * pow(x / P->planet_radius, P->p_alpha);
}
/* init_flag 2 branches of src/init/init.cu:72-349 */
static double init_r(const orc_params* P, double x) { return pow(x / P->planet_radius, -P->p_alpha) * 1.0; }
static double init_p(const orc_params* P, double x) { return get_cs2(P, x) * init_r(P, x); }
static orc_cell init_C(const orc_params* P, double x, double y, double z)
{
    orc_cell Q;
    (void)y; (void)z;
    if (P->init_flag == 2) {
        double rho, dr, dP_dr;
        Q.r = init_r(P, x);
        Q.p = init_p(P, x);
        Q.u = -1.5 * get_nu(P, x) / x;
        rho = init_r(P, x);
        dr = 1.1514178e-7;
        dP_dr = (init_p(P, x + dr) - init_p(P, x - dr)) / (2.0 * dr);
        Q.v = sqrt(1.0 / x + (x / rho) * dP_dr);
        Q.w = 0.0;
    } else {
        /* other init_flags only seed a state; the configs that use them never read init_C */
        Q.r = 1.0; Q.p = 1.0; Q.u = 0.0; Q.v = 0.0; Q.w = 0.0;
    }
    return Q;
}
static double init_v(const orc_params* P, double x) { return init_C(P, x, 0.0, 0.0).v; }

/* init_CD (src/init/init.cu:351-454, init_flag 2, 2D: get_vertical = 1): dust density
   D_G_ratio Sigma_0, Keplerian azimuthal velocity and the radial drift solution */
static orc_dust init_CD(const orc_params* P, double x)
{
    orc_dust Q;
    Q.r = P->d_g_ratio * pow(x / P->planet_radius, -P->p_alpha);
    double f_gas = init_v(P, x) / sqrt(1.0 / x);
    double tmp = P->stokes * P->stokes * f_gas;
    double L = ((1.0 + tmp) / tmp) * (1.0 - sqrt(1.0 - 2.0 * tmp * (1.0 - f_gas) / (1.0 + tmp) / (1.0 + tmp)));
    double u0 = P->stokes * (L * L - 2.0 * L);
    double u = (1.0 - sqrt(1.0 - 2.0 * P->stokes * u0)) / P->stokes;
    L = (1.0 - f_gas + P->stokes * u / 2.0) / (1.0 + P->stokes * u / 2.0);
    u0 = P->stokes * (L * L - 2.0 * L);
    u = (1.0 - sqrt(1.0 - 2.0 * P->stokes * u0)) / P->stokes;
    Q.u = u * sqrt(1.0 / x);
    Q.v = sqrt(1.0 / x);
    Q.w = 0.0;
    return Q;
}

/* src/EOS/EOS.cu:4-18 */
static double get_energy(const orc_params* P, double r, double p, double u, double v, double w)
{
    double e;
    if (P->eos_flag == 2) {
        e = p / ((P->gam - 1.0) * r);
        if (P->internal_e_flag == 0) e += u * u / 2.0 + v * v / 2.0 + w * w / 2.0;
    } else if (P->eos_flag == 1) {
        e = p / pow(r, P->gam);
    } else {
        e = p / r;
    }
    return e;
}

/* ------------------------------------------------------------ lifecycle */
orc_state* orc_create(const orc_params* P)
{
    orc_state* S = (orc_state*)calloc(1, sizeof(orc_state));
    S->P = *P;
    if (S->P.kill_width_out <= 0.0) S->P.kill_width_out = S->P.kill_width;
    S->ypad = (P->ndim > 1) ? NPAD : 0;
    S->xarr = P->xres + 2 * NPAD;
    S->yarr = P->yres + 2 * S->ypad;
    S->xa = (double*)calloc(S->xarr + 1, sizeof(double));
    S->xv = (double*)calloc(S->xarr, sizeof(double));
    S->ya = (double*)calloc(S->yarr + 1, sizeof(double));
    S->yv = (double*)calloc(S->yarr, sizeof(double));
    S->za = (double*)calloc(2, sizeof(double));
    S->zv = (double*)calloc(1, sizeof(double));
    make_grid(S->xa, S->xv, P->xmin, P->xmax, P->xres, NPAD, P->geomx, P->gridx);
    make_grid(S->ya, S->yv, P->ymin, P->ymax, P->yres, S->ypad, P->geomy, P->gridy);
    make_grid(S->za, S->zv, P->zmin, P->zmax, 1, 0, 0, 0);
    size_t n = (size_t)S->xarr * S->yarr;
    S->C = (orc_cell*)calloc(n, sizeof(orc_cell));
    S->T = (orc_cell*)calloc(n, sizeof(orc_cell));
    S->vis = (double*)calloc(2 * n, sizeof(double));
    if (P->dust_flag) {
        S->CD = (orc_dust*)calloc(n, sizeof(orc_dust));
        S->TD = (orc_dust*)calloc(n, sizeof(orc_dust));
    }
    S->orb_rot = (double*)calloc(S->xarr, sizeof(double));
    S->orb_res = (double*)calloc(S->xarr, sizeof(double));
    S->orb_inc = (int*)calloc(S->xarr, sizeof(int));
    return S;
}

void orc_destroy(orc_state* S)
{
    if (!S) return;
    free(S->xa); free(S->xv); free(S->ya); free(S->yv); free(S->za); free(S->zv);
    free(S->C); free(S->T); free(S->vis); free(S->CD); free(S->TD);
    free(S->orb_rot); free(S->orb_res); free(S->orb_inc);
    free(S);
}

int orc_dims(const orc_state* S, int* xarr, int* yarr)
{
    *xarr = S->xarr;
    *yarr = S->yarr;
    return NPAD;
}

void orc_get_grid(const orc_state* S, double* xa, double* xv, double* ya, double* yv)
{
    memcpy(xa, S->xa, (S->xarr + 1) * sizeof(double));
    memcpy(xv, S->xv, S->xarr * sizeof(double));
    memcpy(ya, S->ya, (S->yarr + 1) * sizeof(double));
    memcpy(yv, S->yv, S->yarr * sizeof(double));
}

/* src/init/init.cu:502-519 */
void orc_fill_init(orc_state* S)
{
    double zc = 0.5 * (S->za[1] + S->za[0]);
    for (int j = 0; j < S->yarr; j++)
        for (int i = 0; i < S->xarr; i++) S->C[IND(S, i, j)] = init_C(&S->P, xc(S, i), yc(S, j), zc);
    if (S->P.dust_flag)
        for (int j = 0; j < S->yarr; j++)
            for (int i = 0; i < S->xarr; i++) S->CD[IND(S, i, j)] = init_CD(&S->P, xc(S, i));
}

void orc_set_dust(orc_state* S, const double* r, const double* u, const double* v)
{
    if (!S->CD) return;
    int nx = S->P.xres, ny = S->P.yres;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            orc_dust* d = &S->CD[IND(S, i + NPAD, j + S->ypad)];
            size_t k = (size_t)i + (size_t)nx * j;
            d->r = r[k];
            d->u = u[k];
            d->v = v[k];
        }
}

void orc_get_dust(const orc_state* S, double* r, double* u, double* v)
{
    if (!S->CD) return;
    int nx = S->P.xres, ny = S->P.yres;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const orc_dust* d = &S->CD[IND(S, i + NPAD, j + S->ypad)];
            size_t k = (size_t)i + (size_t)nx * j;
            r[k] = d->r;
            u[k] = d->u;
            v[k] = d->v;
        }
}

/* src/output/output.cu:182-248 (only the interior is loaded) */
void orc_set_interior(orc_state* S, const double* r, const double* p, const double* u, const double* v)
{
    int nx = S->P.xres, ny = S->P.yres;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            orc_cell* c = &S->C[IND(S, i + NPAD, j + S->ypad)];
            size_t k = (size_t)i + (size_t)nx * j;
            c->r = r[k];
            c->p = p[k];
            c->u = u[k];
            if (S->P.ndim > 1 && v) c->v = v[k];
        }
}

void orc_get_interior(const orc_state* S, double* r, double* p, double* u, double* v)
{
    int nx = S->P.xres, ny = S->P.yres;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const orc_cell* c = &S->C[IND(S, i + NPAD, j + S->ypad)];
            size_t k = (size_t)i + (size_t)nx * j;
            if (r) r[k] = c->r;
            if (p) p[k] = c->p;
            if (u) u[k] = c->u;
            if (v) v[k] = c->v;
        }
}

void orc_get_cells(const orc_state* S, orc_cell* out)
{
    memcpy(out, S->C, (size_t)S->xarr * S->yarr * sizeof(orc_cell));
}

/* ---------------------------------------------------------------- planet */
/* src/planet/planet.cu:7-17 */
static double ramp_function(double t, double tau, double val)
{
    if (t < tau) return val * sin(HPI * t / tau);
    return val;
}
/* src/planet/planet.cu:60-103 */
static double ecc_anomaly(double n, double e, double t)
{
    double l = fmod(n * t, TWOPI);
    double D = -e * sin(l);
    if (e == 0.0) return l;
    else if (l == 0.0) return l;
    else if (l == PI) return l;
    else if (l == TWOPI) return l;
    double tor = 1.0e-12, x, dx, d2x, eps, step, esinu, ecosu;
    int count = 0;
    do {
        esinu = sin(l - D) * e;
        ecosu = cos(l - D) * e;
        x = D + esinu;
        dx = 1.0 - ecosu;
        d2x = -esinu;
        eps = 2.0 * x * d2x / dx / dx;
        if (fabs(eps) < 1.0) step = -(x / dx) * (1.0 + eps / 4.0 + eps * eps / 8.0 + 5.0 * eps * eps * eps / 64.0);
        else step = copysign(fmin(fabs(x / dx), HPI / 2.0), -x);
        D += step;
        count++;
    } while (fabs(step) > tor || count < 10);
    return l - D;
}
/* src/planet/planet.cu:105-133 */
static void orbit_solution(const orc_params* P, orc_body* b, double t)
{
    double a = b->a, e = b->e;
    double n = sqrt(1.0 / a / a / a);
    double efac = sqrt(1.0 - e * e);
    double B = e / (1.0 + efac);
    double u = ecc_anomaly(n, e, t);
    double sinu = sin(u), cosu = cos(u);
    double f = u + 2.0 * atan(B * sinu / (1.0 - B * cosu));
    double esinf = sin(f) * e, ecosf = cos(f) * e;
    b->m = ramp_function(t, P->ramp_time, P->planet_mass);
    b->x = a * efac * efac / (1.0 + ecosf);
    b->y = f - fmod(P->frame_omega * t, TWOPI) + PI;
    b->z = HPI;
    b->vx = n * a * esinf / efac;
    b->vy = n * (1.0 + ecosf) * (1.0 + ecosf) / efac / efac / efac;
    b->vz = 0.0;
}
/* src/planet/planet.cu:135-175: star and planet on the reduced orbit about their
   barycentre, in the frame rotating at frame_omega */
static void two_body_solution(const orc_params* P, orc_body* star, orc_body* planet, double t)
{
    double a = star->a, e = star->e;
    double n = sqrt(1.0 / a / a / a);
    double efac = sqrt(1.0 - e * e);
    double B = e / (1.0 + efac);
    double u = ecc_anomaly(n, e, t);
    double sinu = sin(u), cosu = cos(u);
    double f = u + 2.0 * atan(B * sinu / (1.0 - B * cosu));
    double esinf = sin(f) * e, ecosf = cos(f) * e;
    double reduced_r = a * efac * efac / (1.0 + ecosf);
    double reduced_p = f - fmod(P->frame_omega * t, TWOPI) + PI;
    double mp = ramp_function(t, P->ramp_time, P->planet_mass);
    star->m = 1.0 / (1.0 + mp);
    star->x = reduced_r * mp / (1.0 + mp);
    star->y = fmod(reduced_p + PI, TWOPI);
    star->z = HPI;
    star->vx = n * a * esinf / efac * mp / (1.0 + mp);
    star->vy = n * (1.0 + ecosf) * (1.0 + ecosf) / efac / efac / efac;
    star->vz = 0.0;
    planet->m = mp / (1.0 + mp);
    planet->x = reduced_r * 1.0 / (1.0 + mp);
    planet->y = reduced_p;
    planet->z = HPI;
    planet->vx = n * a * esinf / efac * 1.0 / (1.0 + mp);
    planet->vy = n * (1.0 + ecosf) * (1.0 + ecosf) / efac / efac / efac;
    planet->vz = 0.0;
}

/* evolve_planet (src/planet/planet.cu:291-304) */
static void evolve_bodies(orc_state* S, double t)
{
    if (S->P.n_planet <= 0) return;
    if (S->P.twobd_flag) two_body_solution(&S->P, &S->star, &S->planet, t);
    else orbit_solution(&S->P, &S->planet, t);
}

/* src/planet/planet.cu:308-317, 319-402: one planet, or the star-planet pair of
   the two-body frame (the star unsmoothed) */
void orc_init_planet(orc_state* S, double t)
{
    const orc_params* P = &S->P;
    S->planet.a = S->star.a = P->planet_radius;
    S->planet.e = S->star.e = P->planet_ecc;
    if (P->twobd_flag) two_body_solution(P, &S->star, &S->planet, t);
    else orbit_solution(P, &S->planet, t);
    S->star.rs = 0.0;
    if (P->ndim == 2) S->planet.rs = P->rs_fac * P->sc_h * P->planet_radius;
    else S->planet.rs = P->rs_fac * pow(P->planet_mass / 3.0, 1.0 / 3.0) * P->planet_radius;
}

void orc_get_planet(const orc_state* S, orc_body* out) { *out = S->planet; }

/* ---------------------------------------------------- orbital advection */
/* src/orbit/orbit.cu:51-72 */
void orc_init_orbadv(orc_state* S)
{
    for (int i = 0; i < S->xarr; i++) {
        double rad = xc(S, i);
        S->orb_rot[i] = S->P.orbadv_flag ? init_v(&S->P, rad) - rad * S->P.frame_omega : 0.0;
    }
}

/* -------------------------------------------------------------- boundary */
/* src/boundary/boundary.cu:13-62 (ghost columns for every row) */
void orc_boundx(orc_state* S, int which)
{
    orc_cell* X = which ? S->T : S->C;
    const orc_params* P = &S->P;
    int nx = P->xres + NPAD;
    double zc = 0.5 * (S->za[1] + S->za[0]);
    for (int j = 0; j < S->yarr; j++) {
        orc_cell* C = &X[S->xarr * j];
        for (int n = 0; n < NPAD; n++) {
            if (P->bound_lft == 2) { C[n] = C[2 * NPAD - 1 - n]; C[n].u *= -1.0; }
            else if (P->bound_lft == 1) C[n] = C[NPAD];
            else C[n] = init_C(P, xc(S, n), yc(S, j), zc);
        }
        for (int n = 0; n < NPAD; n++) {
            if (P->bound_rgh == 2) { C[nx + n] = C[nx - 1 - n]; C[nx + n].u *= -1.0; }
            else if (P->bound_rgh == 1) C[nx + n] = C[nx - 1];
            else C[nx + n] = init_C(P, xc(S, nx + n), yc(S, j), zc);
        }
    }
}

/* src/boundary/boundary.cu:141-209 with bound_bak = bound_frn = 3 (periodic) */
void orc_boundy(orc_state* S, int which)
{
    if (S->P.ndim < 2) return;
    orc_cell* C = which ? S->T : S->C;
    int yres = S->P.yres, yp = S->ypad;
    for (int i = 0; i < S->xarr; i++)
        for (int n = 0; n < yp; n++) {
            C[IND(S, i, n)] = C[IND(S, i, yres + n)];
            C[IND(S, i, yres + yp + n)] = C[IND(S, i, yp + n)];
        }
}

/* boundx_dust (src/boundary/boundary.cu:64-113, 592-704 with one device) */
static void boundx_dust(orc_state* S)
{
    const orc_params* P = &S->P;
    int nx = P->xres + NPAD;
    for (int j = 0; j < S->yarr; j++) {
        orc_dust* D = &S->CD[S->xarr * j];
        for (int n = 0; n < NPAD; n++) {
            if (P->bound_lft == 2) { D[n] = D[2 * NPAD - 1 - n]; D[n].u *= -1.0; }
            else if (P->bound_lft == 1) D[n] = D[NPAD];
            else D[n] = init_CD(P, xc(S, n));
        }
        for (int n = 0; n < NPAD; n++) {
            if (P->bound_rgh == 2) { D[nx + n] = D[nx - 1 - n]; D[nx + n].u *= -1.0; }
            else if (P->bound_rgh == 1) D[nx + n] = D[nx - 1];
            else D[nx + n] = init_CD(P, xc(S, nx + n));
        }
    }
}

/* boundy_dust (src/boundary/boundary.cu:211-268, periodic) */
static void boundy_dust(orc_state* S)
{
    if (S->P.ndim < 2) return;
    int yres = S->P.yres, yp = S->ypad;
    for (int i = 0; i < S->xarr; i++)
        for (int n = 0; n < yp; n++) {
            S->CD[IND(S, i, n)] = S->CD[IND(S, i, yres + n)];
            S->CD[IND(S, i, yres + yp + n)] = S->CD[IND(S, i, yp + n)];
        }
}

/* ------------------------------------------------------ reconstruction */
static double lim01(double a) { return fmin(fmax(a, 0.0), 1.0); }   /* src/solver/solve.cu:14 */
/* src/solver/solve.cu:19-27 */
static double dimensionless_x(double rL, double r0, double rR) { return lim01((r0 - rL) / (rR - rL)); }
static double exp_lim(double x) { return fmax(1.0 + x, 1.0e-6); }  /* src/solver/solve.cu:29 */

/* src/solver/recon/recon.cu:216-378 (4th-order slopes on a non-uniform grid) */
static void get_4th_parameters(int i, int geom, const double* x, const double* a, double* par)
{
    double a0 = a[i - 2], a1 = a[i - 1], a2 = a[i], a3 = a[i + 1], a4 = a[i + 2];
    double x0 = x[i - 2], x1 = x[i - 1], x2 = x[i], x3 = x[i + 1], x4 = x[i + 2], x5 = x[i + 3];
    double B02, B12, B22, B32, B42, B03, B13, B23, B33, B43, B04, B14, B24, B34, B44;
    double D02, D12, D22, D03, D13, D23, D04, D14, D24;
    double c1, c2, c3, sL, sR, tmp;

    if (geom == 2) {
        B02 = (x1*x1*x1*x1-x0*x0*x0*x0)/(x1*x1*x1-x0*x0*x0)/(4.0/3.0);
        B12 = (x2*x2*x2*x2-x1*x1*x1*x1)/(x2*x2*x2-x1*x1*x1)/(4.0/3.0);
        B22 = (x3*x3*x3*x3-x2*x2*x2*x2)/(x3*x3*x3-x2*x2*x2)/(4.0/3.0);
        B32 = (x4*x4*x4*x4-x3*x3*x3*x3)/(x4*x4*x4-x3*x3*x3)/(4.0/3.0);
        B42 = (x5*x5*x5*x5-x4*x4*x4*x4)/(x5*x5*x5-x4*x4*x4)/(4.0/3.0);
        B03 = (x1*x1*x1*x1*x1-x0*x0*x0*x0*x0)/(x1*x1*x1-x0*x0*x0)/(5.0/3.0);
        B13 = (x2*x2*x2*x2*x2-x1*x1*x1*x1*x1)/(x2*x2*x2-x1*x1*x1)/(5.0/3.0);
        B23 = (x3*x3*x3*x3*x3-x2*x2*x2*x2*x2)/(x3*x3*x3-x2*x2*x2)/(5.0/3.0);
        B33 = (x4*x4*x4*x4*x4-x3*x3*x3*x3*x3)/(x4*x4*x4-x3*x3*x3)/(5.0/3.0);
        B43 = (x5*x5*x5*x5*x5-x4*x4*x4*x4*x4)/(x5*x5*x5-x4*x4*x4)/(5.0/3.0);
        B04 = (x1*x1*x1*x1*x1*x1-x0*x0*x0*x0*x0*x0)/(x1*x1*x1-x0*x0*x0)/2.0;
        B14 = (x2*x2*x2*x2*x2*x2-x1*x1*x1*x1*x1*x1)/(x2*x2*x2-x1*x1*x1)/2.0;
        B24 = (x3*x3*x3*x3*x3*x3-x2*x2*x2*x2*x2*x2)/(x3*x3*x3-x2*x2*x2)/2.0;
        B34 = (x4*x4*x4*x4*x4*x4-x3*x3*x3*x3*x3*x3)/(x4*x4*x4-x3*x3*x3)/2.0;
        B44 = (x5*x5*x5*x5*x5*x5-x4*x4*x4*x4*x4*x4)/(x5*x5*x5-x4*x4*x4)/2.0;
    } else if (geom == 1) {
        B02 = (x1*x1*x1-x0*x0*x0)/(x1*x1-x0*x0)/1.5;
        B12 = (x2*x2*x2-x1*x1*x1)/(x2*x2-x1*x1)/1.5;
        B22 = (x3*x3*x3-x2*x2*x2)/(x3*x3-x2*x2)/1.5;
        B32 = (x4*x4*x4-x3*x3*x3)/(x4*x4-x3*x3)/1.5;
        B42 = (x5*x5*x5-x4*x4*x4)/(x5*x5-x4*x4)/1.5;
        B03 = (x1*x1*x1*x1-x0*x0*x0*x0)/(x1*x1-x0*x0)/2.0;
        B13 = (x2*x2*x2*x2-x1*x1*x1*x1)/(x2*x2-x1*x1)/2.0;
        B23 = (x3*x3*x3*x3-x2*x2*x2*x2)/(x3*x3-x2*x2)/2.0;
        B33 = (x4*x4*x4*x4-x3*x3*x3*x3)/(x4*x4-x3*x3)/2.0;
        B43 = (x5*x5*x5*x5-x4*x4*x4*x4)/(x5*x5-x4*x4)/2.0;
        B04 = (x1*x1*x1*x1*x1-x0*x0*x0*x0*x0)/(x1*x1-x0*x0)/2.5;
        B14 = (x2*x2*x2*x2*x2-x1*x1*x1*x1*x1)/(x2*x2-x1*x1)/2.5;
        B24 = (x3*x3*x3*x3*x3-x2*x2*x2*x2*x2)/(x3*x3-x2*x2)/2.5;
        B34 = (x4*x4*x4*x4*x4-x3*x3*x3*x3*x3)/(x4*x4-x3*x3)/2.5;
        B44 = (x5*x5*x5*x5*x5-x4*x4*x4*x4*x4)/(x5*x5-x4*x4)/2.5;
    } else {
        B02 = (x1*x1-x0*x0)/(x1-x0)/2.0;
        B12 = (x2*x2-x1*x1)/(x2-x1)/2.0;
        B22 = (x3*x3-x2*x2)/(x3-x2)/2.0;
        B32 = (x4*x4-x3*x3)/(x4-x3)/2.0;
        B42 = (x5*x5-x4*x4)/(x5-x4)/2.0;
        B03 = (x1*x1*x1-x0*x0*x0)/(x1-x0)/3.0;
        B13 = (x2*x2*x2-x1*x1*x1)/(x2-x1)/3.0;
        B23 = (x3*x3*x3-x2*x2*x2)/(x3-x2)/3.0;
        B33 = (x4*x4*x4-x3*x3*x3)/(x4-x3)/3.0;
        B43 = (x5*x5*x5-x4*x4*x4)/(x5-x4)/3.0;
        B04 = (x1*x1*x1*x1-x0*x0*x0*x0)/(x1-x0)/4.0;
        B14 = (x2*x2*x2*x2-x1*x1*x1*x1)/(x2-x1)/4.0;
        B24 = (x3*x3*x3*x3-x2*x2*x2*x2)/(x3-x2)/4.0;
        B34 = (x4*x4*x4*x4-x3*x3*x3*x3)/(x4-x3)/4.0;
        B44 = (x5*x5*x5*x5-x4*x4*x4*x4)/(x5-x4)/4.0;
    }

    D02 = B12 - B02; D12 = B22 - B12; D22 = B32 - B22;
    D03 = B13 - B03; D13 = B23 - B13; D23 = B33 - B23;
    D04 = B14 - B04; D14 = B24 - B14; D24 = B34 - B24;

    c3 = (D02*(a3-a2) - D22*(a1-a0))/(D23*D02-D03*D22) - ((a2-a1)*D02 - (a1-a0)*D12)/(D13*D02 - D03*D12);
    tmp = (D02*D24 - D22*D04)/(D23*D02-D03*D22) - (D14*D02 - D04*D12)/(D13*D02 - D03*D12);
    c3 /= tmp;
    tmp = ((a2-a1)*D02 - (a1-a0)*D12)/(D13*D02 - D03*D12);
    c2 = tmp - c3*(D14*D02 - D04*D12)/(D13*D02 - D03*D12);
    tmp = (a1-a0)/D02;
    c1 = tmp - c2*D03/D02 - c3*D04/D02;
    sL = c1*(B22-x2) + c2*(B23-x2*x2) + c3*(B24-x2*x2*x2);

    D02 = B22 - B12; D12 = B32 - B22; D22 = B42 - B32;
    D03 = B23 - B13; D13 = B33 - B23; D23 = B43 - B33;
    D04 = B24 - B14; D14 = B34 - B24; D24 = B44 - B34;

    c3 = (D02*(a4-a3) - D22*(a2-a1))/(D23*D02-D03*D22) - ((a3-a2)*D02 - (a2-a1)*D12)/(D13*D02 - D03*D12);
    tmp = (D02*D24 - D22*D04)/(D23*D02-D03*D22) - (D14*D02 - D04*D12)/(D13*D02 - D03*D12);
    c3 /= tmp;
    tmp = ((a3-a2)*D02 - (a2-a1)*D12)/(D13*D02 - D03*D12);
    c2 = tmp - c3*(D14*D02 - D04*D12)/(D13*D02 - D03*D12);
    tmp = (a2-a1)/D02;
    c1 = tmp - c2*D03/D02 - c3*D04/D02;
    sR = c1*(x3-B22) + c2*(x3*x3-B23) + c3*(x3*x3*x3-B24);

    sL = copysign(fmin(fabs(sL), fabs(a2 - a1)), a2 - a1);
    sR = copysign(fmin(fabs(sR), fabs(a3 - a2)), a3 - a2);

    if (sR * sL <= 0.0) { par[0] = 0.0; par[1] = a2; par[2] = 0.0; }
    else { par[0] = sL; par[1] = a2; par[2] = sR; }
}

/* src/solver/recon/PPM.cu:64-91 (recon_flag 6) */
static void adjust_PPM_parameters(double flat, double* par)
{
    double sL = par[0], sR = par[2];
    sR *= (1.0 - flat);
    sL *= (1.0 - flat);
    double t3 = sR + sL;
    double t2 = t3 * t3;
    double t1 = t3 * 3.0 * (sL - sR);
    if (t2 < t1) sL = 2.0 * sR;
    else if (t2 < -t1) sR = 2.0 * sL;
    par[0] = sL;
    par[2] = sR;
}

/* recon_flag 6: get_CON_parameters / get_PRM_parameters (src/solver/recon/recon.cu:383-463) */
static void get_params(int i, int geom, const double* x, const double* a, const double* flat, double* par)
{
    get_4th_parameters(i, geom, x, a, par);
    adjust_PPM_parameters(flat[i], par);
}

/* src/solver/recon/PPM.cu:95-113 */
static double ppm_aveR(double x, const double* par)
{
    double a6 = 3.0 * (par[0] - par[2]);
    double aR = par[1] + par[2];
    double S = par[2] + par[0];
    x = 1.0 - x;
    return aR - (x / 2.0) * (S - (1.0 - x / 1.5) * a6);
}
static double ppm_aveL(double x, const double* par)
{
    double a6 = 3.0 * (par[0] - par[2]);
    double aL = par[1] - par[0];
    double S = par[2] + par[0];
    return aL + (x / 2.0) * (S + (1.0 - x / 1.5) * a6);
}

/* src/solver/recon/PPM.cu:7-62 : shock flattening coefficient of every cell of a pencil */
static void flatten(int n, double gam, const double* r, const double* p, const double* u, double* flat)
{
    for (int i = 0; i < n; i++) {
        double f = 0.0;
        if (i >= 2 && i < n - 2) {
            double pb = p[i - 1], p0 = p[i], pf = p[i + 1];
            double cs = sqrt(gam * p0 / r[i]);
            double dp1f = pf - p0, dp2f = p[i + 2] - pb;
            double dp1b = p0 - pb, dp2b = pf - p[i - 2];
            double Mf = (u[i] - u[i + 1]) / cs;
            double Mb = (u[i - 1] - u[i]) / cs;
            if (Mf > 0.0 || Mb > 0.0) {
                if (dp2f != 0.0 && dp2b != 0.0) {
                    double ddp;
                    ddp = 10.0 * fmax(0.0, fabs(dp1f / dp2f - 0.5) - 0.25);
                    f = ddp;
                    ddp = 10.0 * fmax(0.0, fabs(dp1b / dp2b - 0.5) - 0.25);
                    f = fmax(f, ddp);
                    f = fmin(0.5, f * fmax(fabs(dp1f), fabs(dp1b)) / p0);
                }
            }
        }
        flat[i] = f;
    }
}

/* ------------------------------------------------------- Riemann solver */
typedef struct { double rl, pl, ul, vl, wl, rr, pr, ur, vr, wr; } rstate;

/* src/solver/riemann/states.cu:1-135 : states at face i (between cells i-1 and i) */
static void set_state(int i, int geom, double gam, const double* xa, const double* flat,
                      const double* r, const double* p, const double* u, const double* v, const double* w,
                      double dt, double us, rstate* S)
{
    double r_par[3], p_par[3], u_par[3];
    double ul, ur, xl, xr, tmp, dis, q, r0, p0, u0, p_, u_, cs, rmin, pmin;
    double hdt = 0.5 * dt;

    get_params(i, geom, xa, r, flat, r_par);
    get_params(i, geom, xa, p, flat, p_par);
    get_params(i, geom, xa, u, flat, u_par);
    xl = xa[i];
    xr = xa[i + 1];
    cs = sqrt(gam * p[i] / r[i]);
    tmp = fmin(u[i], 0.0);
    tmp = xl - tmp * dt + cs * dt;
    q = dimensionless_x(xl, tmp, xr);
    rmin = r[i] * 1.0e-10;
    pmin = p[i] * 1.0e-10;
    ur = ppm_aveL(q, u_par);
    dis = fmin(ur, 0.0) * dt;
    tmp = xl - dis;
    q = dimensionless_x(xl, tmp, xr);
    r0 = ppm_aveL(q, r_par);
    p0 = ppm_aveL(q, p_par);
    u0 = ppm_aveL(q, u_par);
    r0 = fmax(r0, rmin);
    p0 = fmax(p0, pmin);
    cs = sqrt(gam * p0 / r0);
    tmp = xl - dis + cs * dt;
    q = dimensionless_x(xl, tmp, xr);
    u_ = ppm_aveL(q, u_par);
    p_ = ppm_aveL(q, p_par);
    u_ = 2.0 * (u_ - u0) / (cs * dt);
    p_ = 2.0 * (p_ - p0) / (cs * dt);
    u_ *= -hdt;
    p_ *= -hdt;
    S->rr = r0 * exp_lim(u_);
    S->pr = p0 * exp_lim(gam * u_);
    S->ur = u0 + p_ / r0 + us;
    get_params(i, geom, xa, v, flat, r_par);
    get_params(i, geom, xa, w, flat, p_par);
    S->vr = ppm_aveL(q, r_par);
    S->wr = ppm_aveL(q, p_par);

    get_params(i - 1, geom, xa, r, flat, r_par);
    get_params(i - 1, geom, xa, p, flat, p_par);
    get_params(i - 1, geom, xa, u, flat, u_par);
    xl = xa[i - 1];
    xr = xa[i];
    cs = sqrt(gam * p[i - 1] / r[i - 1]);
    tmp = fmax(u[i - 1], 0.0);
    tmp = xr - tmp * dt - cs * dt;
    q = dimensionless_x(xl, tmp, xr);
    rmin = r[i - 1] * 1.0e-10;
    pmin = p[i - 1] * 1.0e-10;
    ul = ppm_aveR(q, u_par);
    dis = fmax(ul, 0.0) * dt;
    tmp = xr - dis;
    q = dimensionless_x(xl, tmp, xr);
    r0 = ppm_aveR(q, r_par);
    p0 = ppm_aveR(q, p_par);
    u0 = ppm_aveR(q, u_par);
    r0 = fmax(r0, rmin);
    p0 = fmax(p0, pmin);
    cs = sqrt(gam * p0 / r0);
    tmp = xr - dis - cs * dt;
    q = dimensionless_x(xl, tmp, xr);
    u_ = ppm_aveR(q, u_par);
    p_ = ppm_aveR(q, p_par);
    u_ = 2.0 * (u0 - u_) / (cs * dt);
    p_ = 2.0 * (p0 - p_) / (cs * dt);
    u_ *= -hdt;
    p_ *= -hdt;
    S->rl = r0 * exp_lim(u_);
    S->pl = p0 * exp_lim(gam * u_);
    S->ul = u0 + p_ / r0 + us;
    get_params(i - 1, geom, xa, v, flat, r_par);
    get_params(i - 1, geom, xa, w, flat, p_par);
    S->vl = ppm_aveR(q, r_par);
    S->wl = ppm_aveR(q, p_par);
}

/* src/solver/riemann/wave_speeds.cu:24-35,288-333 */
static void wave_speeds(const rstate* S, double gam, double us, double* pm, double* sl, double* sm, double* sr)
{
    double cl = sqrt(gam * S->pl / S->rl);
    double cr = sqrt(gam * S->pr / S->rr);
    double c_ = 0.5 * (cr + cl);
    double p_ = 0.5 * (S->pr + S->pl);
    *pm = p_ * exp_lim(0.5 * gam * (S->ul - S->ur) / c_);

    cl = sqrt(gam * S->pl / S->rl);
    cr = sqrt(gam * S->pr / S->rr);
    double srl = sqrt(S->rl), srr = sqrt(S->rr);
    double u_ = (srl * S->ul + srr * S->ur) / (srl + srr);
    double n2 = 0.5 * srl * srr / ((srl + srr) * (srl + srr));
    double cc = sqrt((cl * cl * srl + cr * cr * srr) / (srl + srr) + n2 * (S->ur - S->ul) * (S->ur - S->ul));
    *sl = u_ - cc;
    *sr = u_ + cc;

    double s;
    s = (S->rl * S->ul * cl + S->rr * S->ur * cr) / (S->rl * cl + S->rr * cr);
    s += (S->pl - S->pr) / (S->rl + S->rr) / (0.5 * (cl + cr));
    s += us * (fmax(S->ul, 0.0) + fmax(-S->ur, 0.0)) / (cl + cr);
    *sm = s;
}

/* src/solver/riemann/HLLC.cu:2-8 */
static double get_flux(double FL, double F_L, double F_R, double FR, double sl, double sm, double sr)
{
    if (signbit(sl) == 0) return FL;
    else if (signbit(sr) != 0) return FR;
    else if (signbit(sm) == 0) return F_L;
    return F_R;
}

/* src/solver/riemann/HLLC.cu:10-77 */
static void hllc_fluxes(const orc_params* P, const rstate* S, double pm, double sl, double sm, double sr,
                        orc_cell* F, double* pres, double* uprs)
{
    double fl, f_l, f_r, fr;
    fl = S->ul * S->rl;
    f_l = sm * S->rl * (sl - S->ul) / (sl - sm);
    f_r = sm * S->rr * (sr - S->ur) / (sr - sm);
    fr = S->ur * S->rr;
    F->r = get_flux(fl, f_l, f_r, fr, sl, sm, sr);
    F->u = get_flux(S->ul, S->ul, S->ur, S->ur, sl, sm, sr) * F->r;
    F->v = get_flux(S->vl, S->vl, S->vr, S->vr, sl, sm, sr) * F->r;
    F->w = get_flux(S->wl, S->wl, S->wr, S->wr, sl, sm, sr) * F->r;
    if (P->eos_flag > 0) {
        fl = get_energy(P, S->rl, S->pl, S->ul, 0.0, 0.0);
        fr = get_energy(P, S->rr, S->pr, S->ur, 0.0, 0.0);
        F->p = get_flux(fl, fl, fr, fr, sl, sm, sr) * F->r;
    } else {
        F->p = 0.0;
    }
    fl = S->pl;
    f_l = (sl * pm - sm * S->pl) / (sl - sm);
    f_r = (sr * pm - sm * S->pr) / (sr - sm);
    fr = S->pr;
    *pres = get_flux(fl, f_l, f_r, fr, sl, sm, sr);
    if (P->eos_flag == 2) {
        if (P->internal_e_flag == 0) {
            fl = S->ul * S->pl;
            f_l = sm * (sl * pm - S->ul * S->pl) / (sl - sm);
            f_r = sm * (sr * pm - S->ur * S->pr) / (sr - sm);
            fr = S->ur * S->pr;
        } else {
            fl = S->ul;
            f_l = sm * (sl * pm - S->ul * S->pl) / (sl * pm - sm * S->pl);
            f_r = sm * (sr * pm - S->ur * S->pr) / (sr * pm - sm * S->pr);
            fr = S->ur;
        }
        *uprs = get_flux(fl, f_l, f_r, fr, sl, sm, sr);
    } else {
        *uprs = 0.0;
    }
}

/* src/solver/riemann/riemann.cu:5-11 */
static double eval_gfac(int geom, double x)
{
    if (geom == 1) return x;
    else if (geom == 2) return x * x;
    else if (geom == 5) return sin(x);
    return 1.0;
}

/*
 * One pencil of n cells (3 ghost cells each side): riemann() + net_source()
 * (src/solver/riemann/riemann.cu:40-131).  Faces f in [3, n-3] get fluxes; cell
 * c in [3, n-4] gets del[c] = flux differences with geometric factors and the
 * pressure / pdV source terms.
 */
static void pencil_update_fluxes(const orc_params* P, int n, int geom, const double* xa, double rad,
                                 const double* r, const double* p, const double* u, const double* v, const double* w,
                                 double dt, orc_cell* del, double* flat, orc_cell* F, double* pres, double* uprs)
{
    double gam = P->gam;
    double sdt = dt / rad;   /* set_state receives dt/rad (riemann.cu:111) */
    double us = 0.5 * dt * 0.0;
    flatten(n, gam, r, p, u, flat);
    for (int f = NPAD; f <= n - NPAD; f++) {
        rstate S;
        double pm, sl, sm, sr;
        set_state(f, geom, gam, xa, flat, r, p, u, v, w, sdt, us, &S);
        wave_speeds(&S, gam, us, &pm, &sl, &sm, &sr);
        hllc_fluxes(P, &S, pm, sl, sm, sr, &F[f], &pres[f], &uprs[f]);
    }
    for (int c = NPAD; c < n - NPAD; c++) {
        double g0 = eval_gfac(geom, xa[c]), g1 = eval_gfac(geom, xa[c + 1]);
        double du = 0.5 * (g0 + g1) * (pres[c] - pres[c + 1]);
        double de = 0.0;
        if (P->eos_flag == 2) {
            double t0 = uprs[c] * g0, t1 = uprs[c + 1] * g1;
            if (P->internal_e_flag == 0) de = t0 - t1;
            else de = 0.5 * (pres[c] + pres[c + 1]) * (t0 - t1);
        }
        del[c].r = F[c].r * g0 - F[c + 1].r * g1;
        del[c].p = (F[c].p * g0 - F[c + 1].p * g1) + de;
        del[c].u = (F[c].u * g0 - F[c + 1].u * g1) + du;
        del[c].v = F[c].v * g0 - F[c + 1].v * g1;
        del[c].w = F[c].w * g0 - F[c + 1].w * g1;
    }
}

/* src/solver/sweeps.cu:218-261 */
static orc_cell update_Cell(const orc_params* P, double x, orc_cell Q, orc_cell D)
{
    double r_min = fmax(Q.r * 1.0e-10, SMALLR);
    double p_min = fmax(Q.p * 1.0e-10, SMALLP);
    double u_old = Q.u, v_old = Q.v, w_old = Q.w;
    Q.p = get_energy(P, Q.r, Q.p, Q.u, Q.v, Q.w);
    Q.p *= Q.r;
    Q.u *= Q.r;
    Q.v *= Q.r;
    Q.w *= Q.r;
    Q.r += D.r; Q.p += D.p; Q.u += D.u; Q.v += D.v; Q.w += D.w;
    Q.u /= Q.r;
    Q.v /= Q.r;
    Q.w /= Q.r;
    if (Q.r < r_min) {
        Q.r = r_min; Q.p = p_min; Q.u = u_old; Q.v = v_old; Q.w = w_old;
    } else if (P->eos_flag == 2) {
        double gamm = P->gam - 1.0;
        if (P->internal_e_flag == 0) Q.p = fmax(Q.p * gamm - gamm * Q.r * (Q.u * Q.u + Q.v * Q.v + Q.w * Q.w) / 2.0, p_min);
        else Q.p = fmax(Q.p * gamm, p_min);
    } else if (P->eos_flag == 0) {
        Q.p = get_cs2(P, x) * Q.r;
    }
    return Q;
}

typedef struct {
    double *r, *p, *u, *v, *w, *flat, *pres, *uprs;
    orc_cell *F, *del;
} pencil_buf;

static void pb_alloc(pencil_buf* b, int n)
{
    b->r = (double*)malloc(8 * (size_t)(n + 1) * sizeof(double));
    b->p = b->r + (n + 1); b->u = b->p + (n + 1); b->v = b->u + (n + 1); b->w = b->v + (n + 1);
    b->flat = b->w + (n + 1); b->pres = b->flat + (n + 1); b->uprs = b->pres + (n + 1);
    b->F = (orc_cell*)malloc(2 * (size_t)(n + 1) * sizeof(orc_cell));
    b->del = b->F + (n + 1);
}
static void pb_free(pencil_buf* b) { free(b->r); free(b->F); }

/* src/solver/sweeps.cu:263-335 : radial sweep C -> T over the interior rows */
void orc_sweepx(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->xarr;
    #pragma omp parallel
    {
        pencil_buf b;
        pb_alloc(&b, n);
        #pragma omp for schedule(static)
        for (int j = S->ypad; j < S->ypad + P->yres; j++) {
            for (int i = 0; i < n; i++) {
                const orc_cell* c = &S->C[IND(S, i, j)];
                double rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
                b.r[i] = c->r; b.p[i] = c->p; b.u[i] = c->u; b.v[i] = c->v; b.w[i] = c->w;
                if (P->geomx == 1) b.v[i] *= rad;
            }
            pencil_update_fluxes(P, n, P->geomx, S->xa, 1.0, b.r, b.p, b.u, b.v, b.w, dt, b.del, b.flat, b.F, b.pres, b.uprs);
            for (int i = NPAD; i < n - NPAD; i++) {
                orc_cell D = b.del[i];
                double f = dt / S->xv[i];
                double rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (P->geomx == 1) D.v /= rad;
                S->T[IND(S, i, j)] = update_Cell(P, xc(S, i), S->C[IND(S, i, j)], D);
            }
        }
        pb_free(&b);
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
}

/* src/solver/sweeps.cu:361-433 : azimuthal sweep C -> T on the velocity residual */
void orc_sweepy(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->yarr;
    #pragma omp parallel
    {
        pencil_buf b;
        pb_alloc(&b, n);
        #pragma omp for schedule(static)
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            double rad_cyl = (P->geomy == 3) ? xc(S, i) : 1.0;
            double rot = S->orb_rot[i];
            for (int j = 0; j < n; j++) {
                const orc_cell* c = &S->C[IND(S, i, j)];
                b.r[j] = c->r; b.p[j] = c->p;
                b.u[j] = c->v - rot;
                b.v[j] = c->w; b.w[j] = c->u;
                if (P->geomy == 3) b.u[j] -= rad_cyl * P->frame_omega;
            }
            pencil_update_fluxes(P, n, P->geomy, S->ya, rad_cyl, b.r, b.p, b.u, b.v, b.w, dt, b.del, b.flat, b.F, b.pres, b.uprs);
            for (int j = NPAD; j < n - NPAD; j++) {
                orc_cell D = b.del[j], E;
                double f = dt / S->yv[j] / rad_cyl;
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (P->geomy == 3) D.u += (rot + rad_cyl * P->frame_omega) * D.r;
                else D.u += rot * D.r;
                E.r = D.r; E.p = D.p; E.v = D.u; E.u = D.w; E.w = D.v;
                S->T[IND(S, i, j)] = update_Cell(P, xc(S, i), S->C[IND(S, i, j)], E);
            }
        }
        pb_free(&b);
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
}

/* ----------------------------------------------------------------- dust */
/* dust_flux (src/solver/dust/dust.cu:6-103): upwind PPM fluxes at the left face of
   cell i.  The reference reads the flattening coefficient of recon_flag 6 from
   shared memory that dust_flow never writes (src/solver/recon/PPM.cu:68-77 vs
   dust.cu:110-117); here it is 0, the value zero-initialised memory gives. */
static void dust_flux(int i, int geom, const double* xa, const double* r, const double* u, const double* v,
                      const double* w, const double* flat, double dt, double us, orc_dust* F)
{
    double r_par[3], u_par[3];
    double xl = xa[i], xr = xa[i + 1], tmp, q, ur, ul, u_, r0, u0;
    double Srr, Sur, Svr, Swr, Srl, Sul, Svl, Swl;
    get_params(i, geom, xa, u, flat, u_par);
    tmp = xl - fmin(u_par[1] - u_par[0], 0.0) * dt;
    q = dimensionless_x(xl, tmp, xr);
    ur = ppm_aveL(q, u_par);
    u_ = 0.5 * dt * (ur - u[i]) / (0.5 * (xr - tmp));
    tmp = xl - fmin(ur, 0.0) * dt;
    q = dimensionless_x(xl, tmp, xr);
    get_params(i, geom, xa, r, flat, r_par);
    r0 = ppm_aveL(q, r_par);
    u0 = ppm_aveL(q, u_par);
    Srr = r0 * exp_lim(u_);
    Sur = u0 + us;
    get_params(i, geom, xa, v, flat, r_par);
    get_params(i, geom, xa, w, flat, u_par);
    Svr = ppm_aveL(q, r_par);
    Swr = ppm_aveL(q, u_par);

    xl = xa[i - 1];
    xr = xa[i];
    get_params(i - 1, geom, xa, u, flat, u_par);
    tmp = xr - fmax(u_par[1] + u_par[2], 0.0) * dt;
    q = dimensionless_x(xl, tmp, xr);
    ul = ppm_aveR(q, u_par);
    u_ = 0.5 * dt * (u[i - 1] - ul) / (0.5 * (tmp - xl));
    tmp = xr - fmax(ul, 0.0) * dt;
    q = dimensionless_x(xl, tmp, xr);
    get_params(i - 1, geom, xa, r, flat, r_par);
    r0 = ppm_aveR(q, r_par);
    u0 = ppm_aveR(q, u_par);
    Srl = r0 * exp_lim(u_);
    Sul = u0 + us;
    get_params(i - 1, geom, xa, v, flat, r_par);
    get_params(i - 1, geom, xa, w, flat, u_par);
    Svl = ppm_aveR(q, r_par);
    Swl = ppm_aveR(q, u_par);

    Srl = fmin(r[i - 1] * dt / (xa[i] - xa[i - 1]), fmax(Sul * Srl, 0.0));
    Srr = fmax(r[i] * dt / (xa[i] - xa[i + 1]), fmin(Sur * Srr, 0.0));
    F->r = Srl + Srr;
    F->u = Srl * Sul + Srr * Sur;
    F->v = Srl * Svl + Srr * Svr;
    F->w = Srl * Swl + Srr * Swr;
}

/* update_Dust (src/solver/dust/dust.cu:149-176) */
static orc_dust update_dust(const orc_params* P, orc_dust Q, orc_dust D)
{
    double r_min = fmax(Q.r * 1.0e-10, P->d_g_ratio * SMALLR);
    double u_old = Q.u, v_old = Q.v, w_old = Q.w;
    Q.u *= Q.r; Q.v *= Q.r; Q.w *= Q.r;
    Q.r += D.r; Q.u += D.u; Q.v += D.v; Q.w += D.w;
    Q.u /= Q.r; Q.v /= Q.r; Q.w /= Q.r;
    if (Q.r < r_min) {
        Q.r = r_min; Q.u = u_old; Q.v = v_old; Q.w = w_old;
    }
    return Q;
}

/* dust_flow (src/solver/dust/dust.cu:105-147) over one pencil: del[c] for c in [3, n-4] */
static void dust_pencil(int n, int geom, const double* xa, double rad, const double* r, const double* u,
                        const double* v, const double* w, double dt, double* flat, orc_dust* F, orc_dust* del)
{
    double us = 0.5 * dt * 0.0;
    if (geom > 2) dt /= rad;
    for (int k = 0; k < n; k++) flat[k] = 0.0;
    for (int f = NPAD; f <= n - NPAD; f++) dust_flux(f, geom, xa, r, u, v, w, flat, dt, us, &F[f]);
    for (int c = NPAD; c < n - NPAD; c++) {
        double g0 = eval_gfac(geom, xa[c]), g1 = eval_gfac(geom, xa[c + 1]);
        del[c].r = F[c].r * g0 - F[c + 1].r * g1;
        del[c].u = F[c].u * g0 - F[c + 1].u * g1;
        del[c].v = F[c].v * g0 - F[c + 1].v * g1;
        del[c].w = F[c].w * g0 - F[c + 1].w * g1;
    }
}

/* sweepx_dust_inplace (src/solver/dust/dust.cu:178-235): CD -> TD, then swap */
static void sweepx_dust(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->xarr;
    #pragma omp parallel
    {
        double* b = (double*)malloc(5 * (size_t)(n + 1) * sizeof(double));
        orc_dust* F = (orc_dust*)malloc(2 * (size_t)(n + 1) * sizeof(orc_dust));
        double *r = b, *u = b + (n + 1), *v = b + 2 * (n + 1), *w = b + 3 * (n + 1), *flat = b + 4 * (n + 1);
        orc_dust* del = F + (n + 1);
        #pragma omp for schedule(static)
        for (int j = S->ypad; j < S->ypad + P->yres; j++) {
            for (int i = 0; i < n; i++) {
                const orc_dust* d = &S->CD[IND(S, i, j)];
                r[i] = d->r; u[i] = d->u; v[i] = d->v; w[i] = d->w;
                if (P->geomx == 1) v[i] *= xc(S, i);
            }
            dust_pencil(n, P->geomx, S->xa, 1.0, r, u, v, w, dt, flat, F, del);
            for (int i = NPAD; i < n - NPAD; i++) {
                orc_dust D = del[i];
                double f = dt / S->xv[i];
                D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                if (P->geomx == 1) D.v /= xc(S, i);
                S->TD[IND(S, i, j)] = update_dust(P, S->CD[IND(S, i, j)], D);
            }
        }
        free(b);
        free(F);
    }
    orc_dust* t = S->CD; S->CD = S->TD; S->TD = t;
}

/* sweepy_dust_inplace (src/solver/dust/dust.cu:256-326) */
static void sweepy_dust(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->yarr;
    #pragma omp parallel
    {
        double* b = (double*)malloc(5 * (size_t)(n + 1) * sizeof(double));
        orc_dust* F = (orc_dust*)malloc(2 * (size_t)(n + 1) * sizeof(orc_dust));
        double *r = b, *u = b + (n + 1), *v = b + 2 * (n + 1), *w = b + 3 * (n + 1), *flat = b + 4 * (n + 1);
        orc_dust* del = F + (n + 1);
        #pragma omp for schedule(static)
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            double rad_cyl = (P->geomy == 3) ? xc(S, i) : 1.0;
            double rot = S->orb_rot[i];
            for (int j = 0; j < n; j++) {
                const orc_dust* d = &S->CD[IND(S, i, j)];
                r[j] = d->r;
                u[j] = d->v - rot;
                v[j] = d->w;
                w[j] = d->u;
                if (P->geomy == 3) u[j] -= rad_cyl * P->frame_omega;
            }
            dust_pencil(n, P->geomy, S->ya, rad_cyl, r, u, v, w, dt, flat, F, del);
            for (int j = NPAD; j < n - NPAD; j++) {
                orc_dust D = del[j], E;
                double f = dt / S->yv[j];
                D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                if (P->geomy > 2) {
                    f = 1.0 / rad_cyl;
                    D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                }
                if (P->geomy == 3) D.u += (rot + rad_cyl * P->frame_omega) * D.r;
                else D.u += rot * D.r;
                E.r = D.r; E.v = D.u; E.u = D.w; E.w = D.v;
                S->TD[IND(S, i, j)] = update_dust(P, S->CD[IND(S, i, j)], E);
            }
        }
        free(b);
        free(F);
    }
    orc_dust* t = S->CD; S->CD = S->TD; S->TD = t;
}

/* advecty (Dust) + advecty_dust (src/solver/advection/advection.cu:175-357) */
static void advecty_dust(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->yarr;
    boundy_dust(S);
    #pragma omp parallel
    {
        double* b = (double*)malloc(5 * (size_t)(n + 1) * sizeof(double));
        orc_dust* F = (orc_dust*)malloc((size_t)(n + 1) * sizeof(orc_dust));
        double *r = b, *u = b + (n + 1), *v = b + 2 * (n + 1), *w = b + 3 * (n + 1), *flat = b + 4 * (n + 1);
        double par[3];
        #pragma omp for schedule(static)
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            double rad = (P->geomy == 3) ? xc(S, i) : 1.0;
            double speed = S->orb_res[i];
            double sdt = dt / rad;
            const double* xa = S->ya;
            for (int j = 0; j < n; j++) {
                const orc_dust* d = &S->CD[IND(S, i, j)];
                r[j] = d->r; u[j] = d->v; v[j] = d->w; w[j] = d->u;
                flat[j] = 0.0;
            }
            for (int f = NPAD; f <= n - NPAD; f++) {
                orc_dust* D = &F[f];
                double xl, xr, x0, q;
                if (speed > 0.0) {
                    xl = xa[f - 1]; xr = xa[f];
                    x0 = xr - speed * sdt;
                    q = dimensionless_x(xl, x0, xr);
                    get_params(f - 1, P->geomy, xa, r, flat, par); D->r = ppm_aveR(q, par);
                    get_params(f - 1, P->geomy, xa, u, flat, par); D->u = ppm_aveR(q, par) * D->r;
                    get_params(f - 1, P->geomy, xa, v, flat, par); D->v = ppm_aveR(q, par) * D->r;
                    get_params(f - 1, P->geomy, xa, w, flat, par); D->w = ppm_aveR(q, par) * D->r;
                } else {
                    xl = xa[f]; xr = xa[f + 1];
                    x0 = xl - speed * sdt;
                    q = dimensionless_x(xl, x0, xr);
                    get_params(f, P->geomy, xa, r, flat, par); D->r = ppm_aveL(q, par);
                    get_params(f, P->geomy, xa, u, flat, par); D->u = ppm_aveL(q, par) * D->r;
                    get_params(f, P->geomy, xa, v, flat, par); D->v = ppm_aveL(q, par) * D->r;
                    get_params(f, P->geomy, xa, w, flat, par); D->w = ppm_aveL(q, par) * D->r;
                }
                D->r *= speed; D->u *= speed; D->v *= speed; D->w *= speed;
            }
            for (int j = NPAD; j < n - NPAD; j++) {
                double g0 = eval_gfac(P->geomy, xa[j]), g1 = eval_gfac(P->geomy, xa[j + 1]);
                orc_dust D, E;
                double f;
                D.r = F[j].r * g0 - F[j + 1].r * g1;
                D.u = F[j].u * g0 - F[j + 1].u * g1;
                D.v = F[j].v * g0 - F[j + 1].v * g1;
                D.w = F[j].w * g0 - F[j + 1].w * g1;
                f = dt / S->yv[j];
                D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                if (P->geomy > 2) {
                    f = 1.0 / rad;
                    D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                }
                E.r = D.r; E.v = D.u; E.u = D.w; E.w = D.v;
                S->TD[IND(S, i, j)] = update_dust(P, S->CD[IND(S, i, j)], E);
            }
        }
        free(b);
        free(F);
    }
    orc_dust* t = S->CD; S->CD = S->TD; S->TD = t;
}

/* src/orbit/orbit.cu:74-99 */
static void set_orbadv(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    double dy0 = (P->ymax - P->ymin) / (double)P->yres;
    for (int i = NPAD; i < NPAD + P->xres; i++) {
        double rad_cyl = xc(S, i);
        double dy = dy0 * rad_cyl;
        double rot = S->orb_rot[i];
        int shift = (int)floor(rot * dt / dy + 0.5);
        double speed = shift * dy / dt;
        S->orb_res[i] = rot - speed;
        S->orb_inc[i] = shift;
    }
}

/* src/orbit/orbit.cu:17-49 (+ CT_change at :150) */
static void shift_orbadv(orc_state* S)
{
    const orc_params* P = &S->P;
    int jmax = P->yres;
    for (int i = NPAD; i < NPAD + P->xres; i++) {
        int inc = S->orb_inc[i];
        for (int j = 0; j < jmax; j++) {
            int js = (j + inc) % jmax;
            if (js < 0) js += jmax;
            S->T[IND(S, i, js + S->ypad)] = S->C[IND(S, i, j + S->ypad)];
            if (S->CD) S->TD[IND(S, i, js + S->ypad)] = S->CD[IND(S, i, j + S->ypad)];
        }
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
    if (S->CD) {
        orc_dust* td = S->CD; S->CD = S->TD; S->TD = td;
    }
}

/* src/solver/advection/advection.cu:1-173 : residual orbital advection C -> T */
static void advecty(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->yarr;
    orc_boundy(S, 0);
    #pragma omp parallel
    {
        pencil_buf b;
        pb_alloc(&b, n);
        double* par = (double*)malloc(3 * sizeof(double));
        #pragma omp for schedule(static)
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            double rad = (P->geomy == 3) ? xc(S, i) : 1.0;
            double speed = S->orb_res[i];
            double sdt = dt / rad;
            const double* xa = S->ya;
            for (int j = 0; j < n; j++) {
                const orc_cell* c = &S->C[IND(S, i, j)];
                b.r[j] = c->r; b.p[j] = c->p; b.u[j] = c->v; b.v[j] = c->w; b.w[j] = c->u;
                b.flat[j] = 0.0;
            }
            for (int f = NPAD; f <= n - NPAD; f++) {
                orc_cell* D = &b.F[f];
                double xl, xr, x0, q;
                if (speed > 0.0) {
                    xl = xa[f - 1]; xr = xa[f];
                    x0 = xr - speed * sdt;
                    q = dimensionless_x(xl, x0, xr);
                    get_params(f - 1, P->geomy, xa, b.r, b.flat, par); D->r = ppm_aveR(q, par);
                    get_params(f - 1, P->geomy, xa, b.p, b.flat, par); D->p = ppm_aveR(q, par);
                    get_params(f - 1, P->geomy, xa, b.u, b.flat, par); D->u = ppm_aveR(q, par) * D->r;
                    get_params(f - 1, P->geomy, xa, b.v, b.flat, par); D->v = ppm_aveR(q, par) * D->r;
                    get_params(f - 1, P->geomy, xa, b.w, b.flat, par); D->w = ppm_aveR(q, par) * D->r;
                } else {
                    xl = xa[f]; xr = xa[f + 1];
                    x0 = xl - speed * sdt;
                    q = dimensionless_x(xl, x0, xr);
                    get_params(f, P->geomy, xa, b.r, b.flat, par); D->r = ppm_aveL(q, par);
                    get_params(f, P->geomy, xa, b.p, b.flat, par); D->p = ppm_aveL(q, par);
                    get_params(f, P->geomy, xa, b.u, b.flat, par); D->u = ppm_aveL(q, par) * D->r;
                    get_params(f, P->geomy, xa, b.v, b.flat, par); D->v = ppm_aveL(q, par) * D->r;
                    get_params(f, P->geomy, xa, b.w, b.flat, par); D->w = ppm_aveL(q, par) * D->r;
                }
                D->r *= speed; D->p *= speed; D->u *= speed; D->v *= speed; D->w *= speed;
            }
            for (int j = NPAD; j < n - NPAD; j++) {
                double g0 = eval_gfac(P->geomy, xa[j]), g1 = eval_gfac(P->geomy, xa[j + 1]);
                orc_cell D, Q;
                double f;
                D.r = b.F[j].r * g0 - b.F[j + 1].r * g1;
                D.p = b.F[j].p * g0 - b.F[j + 1].p * g1;
                D.u = b.F[j].u * g0 - b.F[j + 1].u * g1;
                D.v = b.F[j].v * g0 - b.F[j + 1].v * g1;
                D.w = b.F[j].w * g0 - b.F[j + 1].w * g1;
                f = dt / S->yv[j];
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (P->geomy > 2) {
                    f = 1.0 / rad;
                    D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                }
                /* field swap (advection.cu:164-167) then update_Cell_advect (:88-105) */
                Q = S->C[IND(S, i, j)];
                Q.u *= Q.r; Q.v *= Q.r; Q.w *= Q.r;
                Q.r += D.r; Q.p += D.p; Q.u += D.w; Q.v += D.u; Q.w += D.v;
                Q.u /= Q.r; Q.v /= Q.r; Q.w /= Q.r;
                if (P->eos_flag == 0) Q.p = get_cs2(P, xc(S, i)) * Q.r;
                S->T[IND(S, i, j)] = Q;
            }
        }
        free(par);
        pb_free(&b);
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
}

/* ------------------------------------------------------------- viscosity */
/* src/viscosity/viscosity.cu:9-22 */
static void deri_1D(const double* u, const double* r, double* dudx, double* d2udx2)
{
    *dudx = (u[2] - u[0]) / (r[2] - r[0]);
    *d2udx2 = ((u[2] - u[1]) / (r[2] - r[1]) - (u[1] - u[0]) / (r[1] - r[0])) / (0.5 * (r[2] - r[0]));
}
static void deri_2D(const double* u, const double* r, const double* t, double* dudy, double* d2udy2, double* d2udxy)
{
    *dudy = (u[7] - u[4]) / (t[2] - t[0]) / r[1];
    *d2udy2 = ((u[7] - u[1]) / (t[2] - t[1]) - (u[1] - u[4]) / (t[1] - t[0])) / (0.5 * (t[2] - t[0])) / r[1] / r[1];
    *d2udxy = (u[8] - u[6] - u[5] + u[3]) / (r[2] - r[0]) / (t[2] - t[0]) / r[1];
}

/* src/viscosity/viscosity.cu:34-197 (ndim 2) */
void orc_viscous_forces(orc_state* S, int which, double* vis_out)
{
    const orc_params* P = &S->P;
    const orc_cell* C = which ? S->T : S->C;
    if (P->ndim != 2) return;
    #pragma omp parallel for schedule(static)
    for (int j = 1; j < S->yarr - 1; j++) {
        for (int i = 1; i < S->xarr - 1; i++) {
            double u[9], v[9], nr[9], r[3], t[3];
            double dudx, d2udx2, dudy, d2udy2, d2udxy, dvdx, d2vdx2, dvdy, d2vdy2, d2vdxy, dndx, dndy;
            double nu0, nu1, nu2;
            for (int n = 0; n < 3; n++) { r[n] = xc(S, i + n - 1); t[n] = yc(S, j + n - 1); }
            nu0 = get_nu(P, r[0]); nu1 = get_nu(P, r[1]); nu2 = get_nu(P, r[2]);
            for (int n = 0; n < 9; n++) {
                int ind;
                if (n < 3) ind = IND(S, i + n - 1, j);
                else if (n < 6) ind = IND(S, i + n - 4, j - 1);
                else ind = IND(S, i + n - 7, j + 1);
                nr[n] = C[ind].r;
                u[n] = C[ind].u;
                v[n] = C[ind].v;
                if (n == 0 || n == 3 || n == 6) nr[n] *= nu0;
                else if (n == 2 || n == 5 || n == 8) nr[n] *= nu2;
                else nr[n] *= nu1;
            }
            deri_1D(u, r, &dudx, &d2udx2);
            dndx = (nr[2] - nr[0]) / (r[2] - r[0]);
            deri_1D(v, r, &dvdx, &d2vdx2);
            deri_2D(v, r, t, &dvdy, &d2vdy2, &d2vdxy);
            deri_2D(u, r, t, &dudy, &d2udy2, &d2udxy);
            dndy = (nr[7] - nr[4]) / (t[2] - t[0]) / r[1];

            double sxx = 2.0 * nr[1] * dudx;
            double fx = 2.0 * dndx * dudx + 2.0 * nr[1] * d2udx2 + sxx / r[1];
            double syy = 2.0 * nr[1] * (dvdy + u[1] / r[1]);
            double sxy = nr[1] * (dudy + dvdx - v[1] / r[1]);
            double fy = 2.0 * dndy * dvdy + 2.0 * nr[1] * d2vdy2 + 2.0 * nr[1] * dudy / r[1] + 2.0 * dndy * u[1] / r[1];
            fx += dndy * (dudy + dvdx) + nr[1] * (d2udy2 + d2vdxy) - dndy * v[1] / r[1] - nr[1] * dvdy / r[1] - syy / r[1];
            fy += dndx * (dudy + dvdx) + nr[1] * (d2udxy + d2vdx2) - dndx * v[1] / r[1] - nr[1] * dvdx / r[1] + nr[1] * v[1] / r[1] / r[1] + 2.0 * sxy / r[1];
            S->vis[2 * IND(S, i, j) + 0] = fx;
            S->vis[2 * IND(S, i, j) + 1] = fy;
        }
    }
    if (vis_out) memcpy(vis_out, S->vis, 2 * (size_t)S->xarr * S->yarr * sizeof(double));
}

/* ---------------------------------------------------------- source terms */
/* src/solver/force/forces.cu:89-106 (two-body frame, z = 0): a body pulling as
   an inertial point mass, no indirect term */
static void star_planet_grav_cyl_inertial(double rad, double azi, double z, const orc_body* p, double* fx,
                                          double* fy, double* fz)
{
    double sinfac = sin(azi - (p->y + 0.0 * p->vy));
    double cosfac = cos(azi - (p->y + 0.0 * p->vy));
    double plm = p->m, plx = p->x;
    double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p->rs * p->rs);
    double rs_fac = 1.0 / Rp / Rp / Rp;
    *fx = -plm * (rad - plx * cosfac) * rs_fac;
    *fy = -plm * plx * sinfac * rs_fac;
    *fz = -plm * z * rs_fac;
}
/* src/solver/force/forces.cu:41-58 (2D: z = 0) */
static void star_planet_grav_cyl(double rad, double azi, double z, const orc_body* p, double* fx, double* fy, double* fz)
{
    double sinfac = sin(azi - (p->y + 0.0 * p->vy));
    double cosfac = cos(azi - (p->y + 0.0 * p->vy));
    double plm = p->m, plx = p->x;
    double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + z * z + p->rs * p->rs);
    double rs_fac = 1.0 / Rp / Rp / Rp;
    *fx = -plm * (rad - plx * cosfac) * rs_fac - plm * cosfac / plx / plx;
    *fy = -plm * plx * sinfac * rs_fac + plm * sinfac / plx / plx;
    *fz = -plm * z * rs_fac;
}

/*
 * src/solver/sweeps.cu:555-711 with geomx 0/1, ndim <= 2: half-kick of the velocities by curvature, star+planet gravity and
 * the viscous force density; when mdt != 0 the forces are re-evaluated at the
 * mdt-predicted velocities.  With dust (in_d != NULL) the dust velocities relax
 * towards the gas ones over the stopping time t_s = Stokes h / (c_s Sigma)
 * (dust.cu:1-4) with the exponential integrator of sweeps.cu:655-707.  out may
 * equal in, out_d may equal in_d.
 */
/* ------------------------------------------------------------- cooling */
/* Relaxation of the specific energy p/r towards cs^2(x) over dt
   (src/solver/cool/cool.cu:1-33): t_c = beta r_cyl^1.5 (cool_flag 1) or
   beta / r sqrt(p/r) / h (cool_flag 2, r the density). */
static double p_cool(const orc_params* P, double x, double p, double r, double dt)
{
    double rad_cyl = (P->geomx == 1) ? x : 1.0;
    double tc = (P->cool_flag == 1) ? pow(rad_cyl, 1.5) * P->beta_cool
                                    : P->beta_cool * (1.0 / r) * (sqrt(p / r) / P->sc_h);
    double e = p / r;
    double e0 = get_cs2(P, x);
    return r * (e0 + (e - e0) * exp(-dt / tc));
}

static void apply_source_terms(orc_state* S, const orc_cell* in, orc_cell* out, const orc_dust* in_d,
                               orc_dust* out_d, double mdt, double dt)
{
    const orc_params* P = &S->P;
    int i0 = NPAD - 1, i1 = S->xarr - NPAD + 1;
    int j0 = (S->ypad > 0) ? S->ypad - 1 : 0, j1 = (S->ypad > 0) ? S->yarr - S->ypad + 1 : S->yarr;
    #pragma omp parallel for schedule(static)
    for (int j = j0; j < j1; j++) {
        for (int i = i0; i < i1; i++) {
            int ind = IND(S, i, j);
            orc_cell C = in[ind], T = C;
            orc_dust Q = {0.0, 0.0, 0.0, 0.0}, D = Q;
            double ts = 0.0, fxd = 0.0, fyd = 0.0, dtau;
            if (in_d) {
                Q = in_d[ind];
                D = Q;
            }
            double x = xc(S, i);
            double y = (P->ndim > 1) ? yc(S, j) + S->orb_rot[i] * 0.0 : 0.0;
            double z = 0.0;
            double gx = 0.0, gy = 0.0, gz = 0.0, fx, fy = 0.0, fz = 0.0;
            if (P->geomx == 1 && P->twobd_flag) {
                /* get_gx/get_gy/get_gz with twobd_flag 1 (forces.cu:194-201, 243-270, 285-292) */
                const orc_body* B[2] = {&S->star, &S->planet};
                for (int m = 0; m < 2; m++) {
                    double tx, ty, tz;
                    star_planet_grav_cyl_inertial(x, y, z, B[m], &tx, &ty, &tz);
                    gx += tx;
                    gy += ty;
                    gz += tz;
                }
            } else if (P->geomx == 1) {
                double dis = sqrt(x * x + z * z);
                double tx, ty, tz;
                gx = -x / dis / dis / dis;
                gz = -z / dis / dis / dis;
                if (P->n_planet > 0) {
                    star_planet_grav_cyl(x, y, z, &S->planet, &tx, &ty, &tz);
                    gx += tx;
                    gy += ty;
                    gz += tz;
                }
            }
            if (in_d) {
                /* get_t_stop (dust.cu:1-4) and get_d_forces (sweeps.cu:578-595) */
                ts = P->stokes / (sqrt(P->gam * T.p / T.r) / P->sc_h) / T.r;
                fxd = (P->geomx == 1) ? D.v * D.v / x : 0.0;
                fxd = fxd * ts + T.u - Q.u;
                fyd = 0.0 * ts + T.v - Q.v;
            }
            /* get_g_forces (sweeps.cu:555-576) */
            fx = (P->geomx == 1) ? T.v * T.v / x : 0.0;
            if (P->visc_flag) fx += S->vis[2 * ind + 0] / T.r;
            if (P->ndim > 1) {
                fy = 0.0;
                if (P->visc_flag) fy += S->vis[2 * ind + 1] / T.r;
            }
            if (mdt != 0.0) {
                T.u = C.u + fx * mdt + gx * mdt;
                T.v = C.v + fy * mdt + gy * mdt;
                T.w = C.w + fz * mdt + gz * mdt;
                if (P->cool_flag > 0) T.p = p_cool(P, x, T.p, T.r, mdt);  /* sweeps.cu:668-670 */
                if (in_d) {
                    dtau = 1.0 - exp(-mdt / ts);
                    D.u = Q.u + fxd * dtau + gx * ts * dtau;
                    D.v = Q.v + fyd * dtau + gy * ts * dtau;
                    D.w = Q.w + 0.0 * dtau + gz * ts * dtau;
                    ts = P->stokes / (sqrt(P->gam * T.p / T.r) / P->sc_h) / T.r;
                    fxd = (P->geomx == 1) ? D.v * D.v / x : 0.0;
                    fxd = fxd * ts + T.u - Q.u;
                    fyd = 0.0 * ts + T.v - Q.v;
                }
                fx = (P->geomx == 1) ? T.v * T.v / x : 0.0;
                if (P->visc_flag) fx += S->vis[2 * ind + 0] / T.r;
                if (P->ndim > 1) {
                    fy = 0.0;
                    if (P->visc_flag) fy += S->vis[2 * ind + 1] / T.r;
                }
            }
            orc_cell o;
            o.u = C.u + fx * dt + gx * dt;
            o.v = C.v + fy * dt + gy * dt;
            o.w = C.w + fz * dt + gz * dt;
            o.r = in[ind].r;
            o.p = (P->cool_flag > 0) ? p_cool(P, x, in[ind].p, in[ind].r, dt) : in[ind].p;  /* sweeps.cu:695-699 */
            out[ind] = o;
            if (in_d) {
                orc_dust od;
                dtau = 1.0 - exp(-dt / ts);
                od.u = Q.u + fxd * dtau + gx * ts * dtau;
                od.v = Q.v + fyd * dtau + gy * ts * dtau;
                od.w = Q.w + 0.0 * dtau + gz * ts * dtau;
                od.r = in_d[ind].r;
                out_d[ind] = od;
            }
        }
    }
}

/* ------------------------------------------------------------- killwave */
/* src/killwave/killwave.cu:8-14 ; the reference's __sinf is evaluated as sinf of the same float */
static double get_ramping_fac(double x)
{
    double f = (double)sinf((float)(HPI * x));
    f *= f;
    return f;
}

/* src/killwave/killwave.cu:17-103 */
static void killwave(orc_state* S, double dt)
{
    const orc_params* P = &S->P;
    double d_in = get_h(P, P->xmin) * P->kill_width;
    double d_out = get_h(P, P->xmax) * P->kill_width_out;
    double inner = P->xmin + d_in;
    double outer = P->xmax - d_out;
    double zc = 0.5 * (S->za[1] + S->za[0]);
    #pragma omp parallel for schedule(static)
    for (int j = S->ypad; j < S->ypad + P->yres; j++) {
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            double rad = xc(S, i), f, tau;
            orc_cell* C = &S->C[IND(S, i, j)];
            for (int side = 0; side < 2; side++) {
                if (side == 0 && !(rad < inner)) continue;
                if (side == 1 && !(rad > outer)) continue;
                f = side == 0 ? (inner - rad) / d_in : (rad - outer) / d_out;
                tau = (P->geomx == 0) ? 1.0 : pow(rad, 1.5);
                f = get_ramping_fac(f);
                f *= dt / tau;
                orc_cell I = init_C(P, rad, yc(S, j), zc);
                C->r += f * (I.r - C->r);
                C->p += f * (I.p - C->p);
                C->u += f * (I.u - C->u);
                C->v += f * (I.v - C->v);
                C->w += f * (I.w - C->w);
            }
        }
    }
}

/* ------------------------------------------------------------------- dt */
/* src/timestep/timestep.cu:18-140 */
double orc_global_dt(orc_state* S, double dt_prev)
{
    const orc_params* P = &S->P;
    double mx = 0.0;
    #pragma omp parallel for reduction(max : mx) schedule(static)
    for (int j = S->ypad; j < S->ypad + P->yres; j++) {
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            const orc_cell* c = &S->C[IND(S, i, j)];
            double rad_cyl = (P->geomy == 3) ? 0.5 * (S->xa[i + 1] + S->xa[i]) : 1.0;
            double cs = sqrt(P->gam * c->p / c->r);
            double spd = fabs(c->u) + cs;
            if (S->CD) spd = fmax(fabs(S->CD[IND(S, i, j)].u), spd);
            double wid = fabs(S->xa[i + 1] - S->xa[i]);
            double tmp = fmax(spd / wid, 0.0);
            if (P->ndim > 1) {
                spd = fabs(c->v - rad_cyl * P->frame_omega - S->orb_rot[i]) + cs;
                if (S->CD) spd = fmax(fabs(S->CD[IND(S, i, j)].v - rad_cyl * P->frame_omega - S->orb_rot[i]), spd);
                wid = fabs(S->ya[j + 1] - S->ya[j]) * rad_cyl;
                tmp = fmax(spd / wid, tmp);
            }
            mx = fmax(mx, tmp);
        }
    }
    double dt = P->cfl / mx;
    double lim = dt_prev * 1.1;
    return (dt < lim) ? dt : lim;
}

/* ---------------------------------------------------------------- torque */
/* Torque of the planet on the disk, sum over cells of r g_phi Sigma dV (2D polar
 * disk): cal_torque + get_sum_lv1 (src/output/output.cu:336-412) with g_phi of
 * o_star_planet_grav_cyl at z = 0 (src/output/forces.cu:39-57) for the current
 * planet; dV = (xa[i+1]^2 - xa[i]^2)/2 (ya[j+1] - ya[j]).  Summed in a fixed
 * order with compensation (the reference sums in its block order). */
double orc_torque(const orc_state* S)
{
    const orc_params* P = &S->P;
    if (P->ndim != 2 || P->geomy != 3 || P->n_planet < 1) return 0.0;
    const orc_body* p = &S->planet;
    double sum = 0.0, comp = 0.0;
    for (int j = S->ypad; j < S->ypad + P->yres; j++) {
        const double azi = 0.5 * (S->ya[j + 1] + S->ya[j]);
        const double sinfac = sin(azi - p->y), cosfac = cos(azi - p->y);
        for (int i = NPAD; i < NPAD + P->xres; i++) {
            const double rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
            const double Rp = sqrt(rad * rad + p->x * p->x - 2.0 * p->x * rad * cosfac + p->rs * p->rs);
            const double rs_fac = 1.0 / Rp / Rp / Rp;
            /* output_gy (src/output/forces.cu:103-127): inertial in the two-body frame */
            const double gy = P->twobd_flag ? -p->m * p->x * sinfac * rs_fac
                                            : -p->m * p->x * sinfac * rs_fac + p->m * sinfac / p->x / p->x;
            const double dv = 0.5 * (S->xa[i + 1] * S->xa[i + 1] - S->xa[i] * S->xa[i]) * (S->ya[j + 1] - S->ya[j]);
            const double y = rad * gy * (S->C[IND(S, i, j)].r * dv) - comp;
            const double t = sum + y;
            comp = (t - sum) - y;
            sum = t;
        }
    }
    return sum;
}

/* ------------------------------------------------------------- the step */
/* src/solver/solve.cu:212-292 */
void orc_solve(orc_state* S, double t, double dt)
{
    const orc_params* P = &S->P;
    double hdt = 0.5 * dt;
    if (P->visc_flag && P->ndim == 2) {
        orc_boundy(S, 0);
        orc_boundx(S, 0);
        orc_viscous_forces(S, 0, NULL);
    }
    orc_boundx(S, 0);
    if (S->CD) boundx_dust(S);
    apply_source_terms(S, S->C, S->C, S->CD, S->CD, 0.0, hdt);
    orc_boundx(S, 0);
    orc_sweepx(S, dt);
    if (P->ndim > 1) {
        orc_boundy(S, 0);
        orc_sweepy(S, dt);
    }
    if (S->CD) {  /* DS(), src/solver/solve.cu:240-247 */
        boundx_dust(S);
        sweepx_dust(S, dt);
        if (P->ndim > 1) {
            boundy_dust(S);
            sweepy_dust(S, dt);
        }
    }
    if (P->orbadv_flag && P->ndim > 1) {
        set_orbadv(S, dt);
        shift_orbadv(S);
        advecty(S, dt);
        if (S->CD) advecty_dust(S, dt);
    }
    evolve_bodies(S, t + dt);
    if (P->visc_flag && P->ndim == 2) {
        apply_source_terms(S, S->C, S->T, S->CD, S->TD, hdt, hdt);
        orc_boundy(S, 1);
        orc_boundx(S, 1);
        orc_viscous_forces(S, 1, NULL);
        apply_source_terms(S, S->C, S->C, S->CD, S->CD, hdt, hdt);
    } else {
        apply_source_terms(S, S->C, S->C, S->CD, S->CD, hdt, hdt);
    }
    if (P->kill_flag) killwave(S, dt);
}

/* The same step, stage by stage, copying the cell array after every stage the
   stage driver oracle/ref_stages.cu dumps (visc1 if viscous, kick1, sweepx,
   sweepy, with dust dsweepx and dsweepy, shift and advect with orbital
   advection (+ dadvect with dust), kick2, kill if damping), and with dust the
   dust array into dout after the same stages.  Returns the number of stages
   written (each xarr*yarr cells). */
int orc_solve_stages(orc_state* S, double t, double dt, orc_cell* out, orc_dust* dout)
{
    const orc_params* P = &S->P;
    double hdt = 0.5 * dt;
    size_t n = (size_t)S->xarr * S->yarr;
    int k = 0;
#define DUMP()                                                                   \
    do {                                                                         \
        memcpy(out + (size_t)k * n, S->C, n * sizeof(orc_cell));                 \
        if (dout && S->CD) memcpy(dout + (size_t)k * n, S->CD, n * sizeof(orc_dust)); \
        k++;                                                                     \
    } while (0)
    if (P->visc_flag && P->ndim == 2) {
        orc_boundy(S, 0);
        orc_boundx(S, 0);
        orc_viscous_forces(S, 0, NULL);
        DUMP();
    }
    orc_boundx(S, 0);
    if (S->CD) boundx_dust(S);
    apply_source_terms(S, S->C, S->C, S->CD, S->CD, 0.0, hdt);
    DUMP();
    orc_boundx(S, 0);
    orc_sweepx(S, dt);
    DUMP();
    if (P->ndim > 1) {
        orc_boundy(S, 0);
        orc_sweepy(S, dt);
        DUMP();
    }
    if (S->CD) {
        boundx_dust(S);
        sweepx_dust(S, dt);
        DUMP();
        if (P->ndim > 1) {
            boundy_dust(S);
            sweepy_dust(S, dt);
            DUMP();
        }
    }
    if (P->orbadv_flag && P->ndim > 1) {
        set_orbadv(S, dt);
        shift_orbadv(S);
        DUMP();
        advecty(S, dt);
        DUMP();
        if (S->CD) {
            advecty_dust(S, dt);
            DUMP();
        }
    }
    evolve_bodies(S, t + dt);
    if (P->visc_flag && P->ndim == 2) {
        apply_source_terms(S, S->C, S->T, S->CD, S->TD, hdt, hdt);
        orc_boundy(S, 1);
        orc_boundx(S, 1);
        orc_viscous_forces(S, 1, NULL);
        apply_source_terms(S, S->C, S->C, S->CD, S->CD, hdt, hdt);
    } else {
        apply_source_terms(S, S->C, S->C, S->CD, S->CD, hdt, hdt);
    }
    DUMP();
    if (P->kill_flag) {
        killwave(S, dt);
        DUMP();
    }
#undef DUMP
    return k;
}

/* main.cu:320-360 without I/O: dt from global_dt, clipped at end_time.  dt_prev <= 0
   starts like a fresh (re)start, where the first cap is end_time - t0. */
int orc_run(orc_state* S, double t0, double dt_prev, int max_step, double end_time, double* t_out, double* dt_out)
{
    double cur = t0, dt = (dt_prev > 0.0) ? dt_prev : end_time - cur;
    int nstep = 0, contu = 1;
    while (contu && nstep < max_step) {
        dt = orc_global_dt(S, dt);
        if (cur + dt > end_time) {
            dt = end_time - cur;
            contu = 0;
        }
        orc_solve(S, cur, dt);
        cur += dt;
        nstep++;
    }
    if (t_out) *t_out = cur;
    if (dt_out) *dt_out = dt;
    return nstep;
}

/* the 3D part shares this file's pencil routines */
#include "oracle3d.c"
