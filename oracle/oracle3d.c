/*
 * CPU oracle, 3D part (ndim 3) -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference's step loop and DS()/solve() with the polar (z) direction
 * (src/solver/solve.cu:212-292 with ndim 3): half-kick, radial, azimuthal and
 * polar sweeps (src/solver/sweeps.cu:263-554), corrector kick, wave damping and
 * the CFL reduction (src/timestep/timestep.cu:18-140), on the spherical (r, phi,
 * theta) grid of include/para_files/Adiabatic_CPD.h or on a cartesian box.
 * This file is compiled as part of oracle.c (it is included at its end) and
 * uses that file's pencil routines (PPM reconstruction, characteristic states,
 * HLLC, net_source) unchanged: the 3D reference calls the same riemann() for
 * every direction, with the direction's geometry.
 *
 * Scope: no viscosity, orbital advection, dust, cooling or two-body frame (the
 * reference's 3D preset runs none of them); azimuthal boundaries periodic.
 */

struct orc3_state {
    orc_params P;
    int xarr, yarr, zarr;
    double *xa, *xv, *ya, *yv, *za, *zv;
    orc_cell *C, *T;
    orc_body planet;
};

#define IND3(S, i, j, k) ((size_t)(i) + (size_t)(S)->xarr * ((size_t)(j) + (size_t)(S)->yarr * (size_t)(k)))

/* ------------------------------------------------------------------ grid */
/* src/geom/geom.cu:3-20 (geom 5: polar angle; 4 and 3 take the default 1) */
static double get_dv_dr3(int geom, double ra, double dr)
{
    if (geom == 5) {
        if (dr < 1.0e-4) return sin(ra + 0.5 * dr);
        return (cos(ra) - cos(ra + dr)) / dr;
    } else if (geom == 2) return ra * ra + ra * dr + dr * dr / 3.0;
    else if (geom == 1) return ra + dr / 2.0;
    return 1.0;
}

/* src/geom/geom.cu:35-54 : fine spacing at the middle of the range */
static void nonuspace(const orc_params* P, double* a, double start, double end, int len)
{
    (void)P;
    int N = (len - 1) / 2;
    double L = (end - start) / 2.0;
    double dx_min = (L / (double)N) / 32.0;
    double dx_max = (PI - L) / N;
    double k = log(1.0 - (dx_max - dx_min) / (L - (double)N * dx_min)) / log(1.0 - 1.0 / (double)N);
    for (int i = 0; i < N; i++) a[i] = (end + start) / 2.0 - (N - i) * dx_min - (L - N * dx_min) * pow((double)(N - i) / (double)N, k);
    for (int i = 0; i < N + 1; i++) a[N + i] = (end + start) / 2.0 + i * dx_min + (L - N * dx_min) * pow((double)i / (double)N, k);
}

/* src/geom/geom.cu:56-75 : uniform outer parts, fine spacing over the radial
   extent around the middle (sized from the radial grid's xres, xmin, xmax) */
static void nonuspace_mix(const orc_params* P, double* a, double start, double end, int len)
{
    int N = P->xres / 2;
    int N2 = (len - 1 - 2 * N) / 2;
    double L = (P->xmax - P->xmin) / 2.0;
    double L2 = (end - start - 2.0 * L) / 2.0;
    double dx_min = (L / (double)N) / 32.0;
    double dx_max = L2 / (double)N2;
    double k = log(1.0 - (dx_max - dx_min) / (L - (double)N * dx_min)) / log(1.0 - 1.0 / (double)N);
    for (int i = 0; i < N2; i++) a[i] = start + (double)i * dx_max;
    for (int i = 0; i < N; i++) a[i + N2] = (end + start) / 2.0 - (N - i) * dx_min - (L - N * dx_min) * pow((double)(N - i) / (double)N, k);
    for (int i = 0; i < N; i++) a[i + N2 + N] = (end + start) / 2.0 + i * dx_min + (L - N * dx_min) * pow((double)i / (double)N, k);
    for (int i = 0; i < N2 + 1; i++) a[i + N2 + 2 * N] = start + 2.0 * L + L2 + (double)i * dx_max;
}

/* src/geom/geom.cu:77-89 : fine spacing towards the end of the range (the midplane) */
static void nonuspace_half(const orc_params* P, double* a, double start, double end, int len)
{
    int N = len - 1;
    double L = end - start;
    double dx_min = ((P->xmax - P->xmin) / (double)P->xres) / 32.0;
    double dx_max = P->sc_h / 16.0;
    double k = log(1.0 - (dx_max - dx_min) / (L - (double)N * dx_min)) / log(1.0 - 1.0 / (double)N);
    for (int i = 0; i < N + 1; i++) a[i] = end - (N - i) * dx_min - (L - N * dx_min) * pow((double)(N - i) / (double)N, k);
}

/* src/init/init.cu:472-500 with every spacing of src/geom/geom.cu */
static void make_grid3(const orc_params* P, double* a, double* v, double amin, double amax, int res, int pad, int geom,
                       int grid)
{
    int len = res + 1;
    if (grid == 0) {
        for (int i = 0; i < len; i++) a[pad + i] = amin + (amax - amin) * (double)i / (double)(len - 1);
    } else if (grid == 1) {
        double tmp = log(amax / amin);
        for (int i = 0; i < len; i++) a[pad + i] = amin * exp(tmp * (double)i / (double)(len - 1));
    } else if (grid == 2) {
        nonuspace(P, &a[pad], amin, amax, len);
    } else if (grid == 3) {
        nonuspace_half(P, &a[pad], amin, amax, len);
    } else {
        nonuspace_mix(P, &a[pad], amin, amax, len);
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
    for (int i = 0; i < res + 2 * pad; i++) v[i] = (a[i + 1] - a[i]) * get_dv_dr3(geom, a[i], a[i + 1] - a[i]);
}

static double xc3(const orc3_state* S, int i) { return 0.5 * (S->xa[i + 1] + S->xa[i]); }
static double yc3(const orc3_state* S, int j) { return 0.5 * (S->ya[j + 1] + S->ya[j]); }
static double zc3(const orc3_state* S, int k) { return 0.5 * (S->za[k + 1] + S->za[k]); }

/* ------------------------------------------------------- analytic state */
/* src/init/init.cu:7-17 */
static double get_cs2_3(const orc_params* P, double x, double z)
{
    double coeff = P->sc_h * P->sc_h * (1.0 / P->planet_radius);
    if (P->geomx == 0) return coeff;
    if (P->geomx == 1) return coeff * pow(x / P->planet_radius, -P->p_beta);
    return coeff * pow(x * sin(z) / P->planet_radius, -P->p_beta);
}
/* src/init/init.cu:20-29 */
static double get_h3(const orc_params* P, double x, double z)
{
    if (P->geomx == 0) return P->sc_h;
    if (P->geomx == 1) return sqrt(get_cs2_3(P, x, z) * pow(x, 3));
    return sqrt(get_cs2_3(P, x, z) * pow(x * sin(z), 3));
}
/* src/init/init.cu:53-71 (ndim 3) */
static double get_vertical3(const orc_params* P, double x, double z)
{
    if (P->geomx == 0) return exp(-z * z / (2.0 * P->sc_h * P->sc_h));
    double cs2 = get_cs2_3(P, x, z);
    if (P->geomx == 1) {
        double s = sqrt(x * x + z * z);
        return exp((1.0 / s - 1.0 / x) / cs2);
    }
    double r = x * sin(z);
    return exp((1.0 / x - 1.0 / r) / cs2);
}
/* init_flag 3 (src/init/init.cu:90-91, 157-158, 196-198, 269-274, 322-323): the
   spherical disk in vertical hydrostatic balance; get_nu is 0 without viscosity */
static double init_r3(const orc_params* P, double x, double z)
{
    return pow(x * sin(z) / P->planet_radius, -P->p_alpha) * get_vertical3(P, x, z);
}
static double init_p3(const orc_params* P, double x, double z) { return get_cs2_3(P, x, z) * init_r3(P, x, z); }
static orc_cell init_C3(const orc_params* P, double x, double y, double z)
{
    orc_cell Q;
    (void)y;
    if (P->init_flag == 3) {
        double rho, dr, dP_dr, r = x * sin(z);
        Q.r = init_r3(P, x, z);
        Q.p = init_p3(P, x, z);
        Q.u = -1.5 * 0.0 / r;
        rho = init_r3(P, x, z);
        dr = 1.1514178e-7;
        dP_dr = (init_p3(P, x + dr, z) - init_p3(P, x - dr, z)) / (2.0 * dr);
        Q.v = sqrt(1.0 / x + (x / rho) * dP_dr);
        Q.w = 0.0;
    } else {
        /* configurations without analytic ghosts or damping never read it */
        Q.r = 1.0; Q.p = 1.0; Q.u = 0.0; Q.v = 0.0; Q.w = 0.0;
    }
    return Q;
}

/* ------------------------------------------------------------ lifecycle */
orc3_state* orc3_create(const orc_params* P)
{
    orc3_state* S = (orc3_state*)calloc(1, sizeof(orc3_state));
    S->P = *P;
    if (S->P.kill_width_out <= 0.0) S->P.kill_width_out = S->P.kill_width;
    S->xarr = P->xres + 2 * NPAD;
    S->yarr = P->yres + 2 * NPAD;
    S->zarr = P->zres + 2 * NPAD;
    S->xa = (double*)calloc(S->xarr + 1, sizeof(double));
    S->xv = (double*)calloc(S->xarr, sizeof(double));
    S->ya = (double*)calloc(S->yarr + 1, sizeof(double));
    S->yv = (double*)calloc(S->yarr, sizeof(double));
    S->za = (double*)calloc(S->zarr + 1, sizeof(double));
    S->zv = (double*)calloc(S->zarr, sizeof(double));
    make_grid3(P, S->xa, S->xv, P->xmin, P->xmax, P->xres, NPAD, P->geomx, P->gridx);
    make_grid3(P, S->ya, S->yv, P->ymin, P->ymax, P->yres, NPAD, P->geomy, P->gridy);
    make_grid3(P, S->za, S->zv, P->zmin, P->zmax, P->zres, NPAD, P->geomz, P->gridz);
    size_t n = (size_t)S->xarr * S->yarr * S->zarr;
    S->C = (orc_cell*)calloc(n, sizeof(orc_cell));
    S->T = (orc_cell*)calloc(n, sizeof(orc_cell));
    return S;
}

void orc3_destroy(orc3_state* S)
{
    if (!S) return;
    free(S->xa); free(S->xv); free(S->ya); free(S->yv); free(S->za); free(S->zv);
    free(S->C); free(S->T);
    free(S);
}

int orc3_dims(const orc3_state* S, int* xarr, int* yarr, int* zarr)
{
    *xarr = S->xarr;
    *yarr = S->yarr;
    *zarr = S->zarr;
    return NPAD;
}

/* faces (arr + 1) and volumes (arr) of axis 0 (x), 1 (y) or 2 (z) */
void orc3_get_axis(const orc3_state* S, int axis, double* a, double* v)
{
    int n = axis == 0 ? S->xarr : (axis == 1 ? S->yarr : S->zarr);
    const double* fa = axis == 0 ? S->xa : (axis == 1 ? S->ya : S->za);
    const double* fv = axis == 0 ? S->xv : (axis == 1 ? S->yv : S->zv);
    memcpy(a, fa, (n + 1) * sizeof(double));
    memcpy(v, fv, n * sizeof(double));
}

/* fill_grid (src/init/init.cu:502-519): every cell, ghosts included */
void orc3_fill_init(orc3_state* S)
{
    for (int k = 0; k < S->zarr; k++)
        for (int j = 0; j < S->yarr; j++)
            for (int i = 0; i < S->xarr; i++) S->C[IND3(S, i, j, k)] = init_C3(&S->P, xc3(S, i), yc3(S, j), zc3(S, k));
}

/* load_grid (src/output/output.cu:182-248): interior fields, x fastest, then y, then z */
void orc3_set_interior(orc3_state* S, const double* r, const double* p, const double* u, const double* v,
                       const double* w)
{
    const orc_params* P = &S->P;
    size_t m = 0;
    for (int k = NPAD; k < NPAD + P->zres; k++)
        for (int j = NPAD; j < NPAD + P->yres; j++)
            for (int i = NPAD; i < NPAD + P->xres; i++, m++) {
                orc_cell* c = &S->C[IND3(S, i, j, k)];
                c->r = r[m]; c->p = p[m]; c->u = u[m]; c->v = v[m]; c->w = w[m];
            }
}

void orc3_get_interior(const orc3_state* S, double* r, double* p, double* u, double* v, double* w)
{
    const orc_params* P = &S->P;
    size_t m = 0;
    for (int k = NPAD; k < NPAD + P->zres; k++)
        for (int j = NPAD; j < NPAD + P->yres; j++)
            for (int i = NPAD; i < NPAD + P->xres; i++, m++) {
                const orc_cell* c = &S->C[IND3(S, i, j, k)];
                r[m] = c->r; p[m] = c->p; u[m] = c->u; v[m] = c->v; w[m] = c->w;
            }
}

/* src/planet/planet.cu:308-317, 319-402 (ndim 3 smoothing length) */
void orc3_init_planet(orc3_state* S, double t)
{
    const orc_params* P = &S->P;
    S->planet.a = P->planet_radius;
    S->planet.e = P->planet_ecc;
    orbit_solution(P, &S->planet, t);
    S->planet.rs = P->rs_fac * pow(P->planet_mass / 3.0, 1.0 / 3.0) * P->planet_radius;
}

void orc3_get_planet(const orc3_state* S, orc_body* out) { *out = S->planet; }

/* -------------------------------------------------------------- boundary */
/* src/boundary/boundary.cu:13-62 (every row and plane) */
void orc3_boundx(orc3_state* S)
{
    const orc_params* P = &S->P;
    int nx = P->xres + NPAD;
    for (int k = 0; k < S->zarr; k++)
        for (int j = 0; j < S->yarr; j++) {
            orc_cell* C = &S->C[IND3(S, 0, j, k)];
            for (int n = 0; n < NPAD; n++) {
                if (P->bound_lft == 2) {
                    C[n] = C[2 * NPAD - 1 - n];
                    C[n].u *= -1.0;
                } else if (P->bound_lft == 1) {
                    C[n] = C[NPAD];
                } else if (P->bound_lft == 0) {
                    C[n] = init_C3(P, xc3(S, n), yc3(S, j), zc3(S, k));
                }
                if (P->bound_rgh == 2) {
                    C[nx + n] = C[nx - 1 - n];
                    C[nx + n].u *= -1.0;
                } else if (P->bound_rgh == 1) {
                    C[nx + n] = C[nx - 1];
                } else if (P->bound_rgh == 0) {
                    C[nx + n] = init_C3(P, xc3(S, nx + n), yc3(S, j), zc3(S, k));
                }
            }
        }
}

/* src/boundary/boundary.cu:140-209, periodic (bound_bak / bound_frn 3), interior planes */
void orc3_boundy(orc3_state* S)
{
    const orc_params* P = &S->P;
    for (int k = NPAD; k < NPAD + P->zres; k++)
        for (int i = 0; i < S->xarr; i++)
            for (int n = 0; n < NPAD; n++) {
                S->C[IND3(S, i, n, k)] = S->C[IND3(S, i, P->yres + n, k)];
                S->C[IND3(S, i, P->yres + NPAD + n, k)] = S->C[IND3(S, i, NPAD + n, k)];
            }
}

/* src/boundary/boundary.cu:270-320 (every column and row) */
void orc3_boundz(orc3_state* S)
{
    const orc_params* P = &S->P;
    int nz = P->zres;
    for (int j = 0; j < S->yarr; j++)
        for (int i = 0; i < S->xarr; i++)
            for (int n = 0; n < NPAD; n++) {
                orc_cell T;
                if (P->bound_bom == 3) {
                    T = S->C[IND3(S, i, j, nz + n)];
                } else if (P->bound_bom == 2) {
                    T = S->C[IND3(S, i, j, 2 * NPAD - 1 - n)];
                    T.w *= -1.0;
                } else if (P->bound_bom == 1) {
                    T = S->C[IND3(S, i, j, NPAD)];
                } else {
                    T = init_C3(P, xc3(S, i), yc3(S, j), zc3(S, n));
                }
                S->C[IND3(S, i, j, n)] = T;
                if (P->bound_top == 3) {
                    T = S->C[IND3(S, i, j, NPAD + n)];
                } else if (P->bound_top == 2) {
                    T = S->C[IND3(S, i, j, nz + NPAD - 1 - n)];
                    T.w *= -1.0;
                } else if (P->bound_top == 1) {
                    T = S->C[IND3(S, i, j, nz + NPAD - 1)];
                } else {
                    T = init_C3(P, xc3(S, i), yc3(S, j), zc3(S, nz + NPAD + n));
                }
                S->C[IND3(S, i, j, nz + NPAD + n)] = T;
            }
}

/* --------------------------------------------------------------- sweeps */
/* src/solver/sweeps.cu:218-261 with get_cs2 at the cell */
static orc_cell update_cell3(const orc_params* P, double cs2, orc_cell Q, orc_cell D)
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
        Q.p = cs2 * Q.r;
    }
    return Q;
}

static double cs2_at(const orc3_state* S, int i, int k) { return get_cs2_3(&S->P, xc3(S, i), zc3(S, k)); }

/* src/solver/sweeps.cu:263-335 : radial pencils of every interior (j, k) */
void orc3_sweepx(orc3_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->xarr;
    #pragma omp parallel
    {
        pencil_buf b;
        pb_alloc(&b, n);
        #pragma omp for collapse(2) schedule(static)
        for (int k = NPAD; k < NPAD + P->zres; k++)
            for (int j = NPAD; j < NPAD + P->yres; j++) {
                double sinz = sin(zc3(S, k));
                for (int i = 0; i < n; i++) {
                    const orc_cell* c = &S->C[IND3(S, i, j, k)];
                    double rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
                    b.r[i] = c->r; b.p[i] = c->p; b.u[i] = c->u; b.v[i] = c->v; b.w[i] = c->w;
                    if (P->geomx == 1) b.v[i] *= rad;
                    else if (P->geomx == 2) {
                        b.v[i] *= rad * sinz;
                        b.w[i] *= rad;
                    }
                }
                pencil_update_fluxes(P, n, P->geomx, S->xa, 1.0, b.r, b.p, b.u, b.v, b.w, dt, b.del, b.flat, b.F,
                                     b.pres, b.uprs);
                for (int i = NPAD; i < n - NPAD; i++) {
                    orc_cell D = b.del[i];
                    double f = dt / S->xv[i];
                    double rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
                    D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                    if (P->geomx == 1) D.v /= rad;
                    else if (P->geomx == 2) {
                        D.v /= rad * sinz;
                        D.w /= rad;
                    }
                    S->T[IND3(S, i, j, k)] = update_cell3(P, cs2_at(S, i, k), S->C[IND3(S, i, j, k)], D);
                }
            }
        pb_free(&b);
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
}

/* src/solver/sweeps.cu:361-433 : azimuthal pencils of every interior (i, k) (orb_rot 0) */
void orc3_sweepy(orc3_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->yarr;
    #pragma omp parallel
    {
        pencil_buf b;
        pb_alloc(&b, n);
        #pragma omp for collapse(2) schedule(static)
        for (int k = NPAD; k < NPAD + P->zres; k++)
            for (int i = NPAD; i < NPAD + P->xres; i++) {
                double rad_cyl = 1.0, rot = 0.0;
                if (P->geomy == 3) rad_cyl = xc3(S, i);
                else if (P->geomy == 4) rad_cyl = xc3(S, i) * sin(zc3(S, k));
                for (int j = 0; j < n; j++) {
                    const orc_cell* c = &S->C[IND3(S, i, j, k)];
                    b.r[j] = c->r; b.p[j] = c->p;
                    b.u[j] = c->v - rot;
                    b.v[j] = c->w; b.w[j] = c->u;
                    if (P->geomy == 3 || P->geomy == 4) b.u[j] -= rad_cyl * P->frame_omega;
                }
                pencil_update_fluxes(P, n, P->geomy, S->ya, rad_cyl, b.r, b.p, b.u, b.v, b.w, dt, b.del, b.flat,
                                     b.F, b.pres, b.uprs);
                for (int j = NPAD; j < n - NPAD; j++) {
                    orc_cell D = b.del[j], E;
                    double f = dt / S->yv[j] / rad_cyl;
                    D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                    if (P->geomy == 3 || P->geomy == 4) D.u += (rot + rad_cyl * P->frame_omega) * D.r;
                    else D.u += rot * D.r;
                    E.r = D.r; E.p = D.p; E.v = D.u; E.u = D.w; E.w = D.v;
                    S->T[IND3(S, i, j, k)] = update_cell3(P, cs2_at(S, i, k), S->C[IND3(S, i, j, k)], E);
                }
            }
        pb_free(&b);
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
}

/* src/solver/sweeps.cu:458-554 : polar pencils of every interior (i, j) */
void orc3_sweepz(orc3_state* S, double dt)
{
    const orc_params* P = &S->P;
    int n = S->zarr;
    #pragma omp parallel
    {
        pencil_buf b;
        pb_alloc(&b, n);
        #pragma omp for collapse(2) schedule(static)
        for (int j = NPAD; j < NPAD + P->yres; j++)
            for (int i = NPAD; i < NPAD + P->xres; i++) {
                double rad = (P->geomz == 5) ? xc3(S, i) : 1.0;
                for (int k = 0; k < n; k++) {
                    const orc_cell* c = &S->C[IND3(S, i, j, k)];
                    b.r[k] = c->r; b.p[k] = c->p;
                    b.u[k] = c->w; b.v[k] = c->u; b.w[k] = c->v;
                    if (P->geomz == 5) b.w[k] *= rad * sin(0.5 * (S->za[k + 1] + S->za[k]));
                }
                pencil_update_fluxes(P, n, P->geomz, S->za, rad, b.r, b.p, b.u, b.v, b.w, dt, b.del, b.flat, b.F,
                                     b.pres, b.uprs);
                for (int k = NPAD; k < n - NPAD; k++) {
                    orc_cell D = b.del[k], E;
                    double f = dt / S->zv[k];
                    D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                    if (P->geomz == 5) {
                        double g = 1.0 / rad;
                        D.r *= g; D.p *= g; D.u *= g; D.v *= g; D.w *= g;
                        D.w /= rad * sin(0.5 * (S->za[k + 1] + S->za[k]));
                    }
                    E.r = D.r; E.p = D.p; E.u = D.v; E.v = D.w; E.w = D.u;
                    S->T[IND3(S, i, j, k)] = update_cell3(P, cs2_at(S, i, k), S->C[IND3(S, i, j, k)], E);
                }
            }
        pb_free(&b);
    }
    orc_cell* t = S->C; S->C = S->T; S->T = t;
}

/* ---------------------------------------------------------- source terms */
/* star_planet_grav (src/solver/force/forces.cu:14-39), dt = 0 */
static void star_planet_grav3(double rad, double azi, double pol, const orc_body* p, double* fx, double* fy,
                              double* fz)
{
    double sinfac = sin(azi - (p->y + 0.0 * p->vy)), cosfac = cos(azi - (p->y + 0.0 * p->vy));
    double sinpol = sin(pol), cospol = cos(pol);
    double plm = p->m, plx = p->x;
    double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol);
    double rs_fac = fmax(4.0 - 3.0 * Rp / p->rs, 1.0) / fmax(p->rs * p->rs * p->rs, Rp * Rp * Rp);
    *fx = -plm * (rad - plx * cosfac * sinpol) * rs_fac - plm * sinpol * cosfac / plx / plx;
    *fy = -plm * plx * sinfac * rs_fac + plm * sinpol * sinfac / plx / plx;
    *fz = plm * plx * cosfac * cospol * rs_fac - plm * cospol * cosfac / (sinpol * plx * plx);
}

/* get_gx / get_gy / get_gz (src/solver/force/forces.cu:182-327, twobd_flag 0) */
static void gravity3(const orc3_state* S, double rad, double azi, double pol, double* gx, double* gy, double* gz)
{
    const orc_params* P = &S->P;
    *gx = 0.0; *gy = 0.0; *gz = 0.0;
    if (P->geomx != 2) return;
    *gx = -1.0 / rad / rad;
    for (int m = 0; m < P->n_planet; m++) {
        double fx, fy, fz;
        star_planet_grav3(rad, azi, pol, &S->planet, &fx, &fy, &fz);
        *gx += fx;
        *gy += fy;
        *gz += fz;
    }
    if (pol < P->zmin) *gz *= -1.0;
}

/* get_fx / get_fy / get_fz (src/solver/force/forces.cu:110-177) */
static void fict3(const orc_params* P, double rad, double pol, const orc_cell* T, double* fx, double* fy, double* fz)
{
    *fx = 0.0; *fy = 0.0; *fz = 0.0;
    if (P->geomx == 2) {
        *fx = T->v * T->v / rad + T->w * T->w / rad;
        *fz = T->v * T->v / rad / tan(pol);
        if (pol < P->zmin) *fz *= -1.0;
    }
}

/* apply_source_terms (src/solver/sweeps.cu:597-711) in place, x_dt = 0, without
   viscosity, dust or cooling: interior plus one ghost layer in every direction */
static void apply_source_terms3(orc3_state* S, double mdt, double dt)
{
    const orc_params* P = &S->P;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = NPAD - 1; k < S->zarr - NPAD + 1; k++)
        for (int j = NPAD - 1; j < S->yarr - NPAD + 1; j++)
            for (int i = NPAD - 1; i < S->xarr - NPAD + 1; i++) {
                orc_cell* out = &S->C[IND3(S, i, j, k)];
                orc_cell C = *out, T = C;
                double xc = xc3(S, i), yc = yc3(S, j), zc = zc3(S, k);
                double gx, gy, gz, fx, fy, fz;
                gravity3(S, xc, yc, zc, &gx, &gy, &gz);
                fict3(P, xc, zc, &T, &fx, &fy, &fz);
                if (mdt != 0.0) {
                    T.u = C.u + fx * mdt + gx * mdt;
                    T.v = C.v + fy * mdt + gy * mdt;
                    T.w = C.w + fz * mdt + gz * mdt;
                    fict3(P, xc, zc, &T, &fx, &fy, &fz);
                }
                out->u = C.u + fx * dt + gx * dt;
                out->v = C.v + fy * dt + gy * dt;
                out->w = C.w + fz * dt + gz * dt;
            }
}

/* src/killwave/killwave.cu:17-103 (the same ramp as the 2D oracle) */
static void killwave3(orc3_state* S, double dt)
{
    const orc_params* P = &S->P;
    double d_in = get_h3(P, P->xmin, HPI) * P->kill_width;
    double d_out = get_h3(P, P->xmax, HPI) * P->kill_width_out;
    double inner = P->xmin + d_in;
    double outer = P->xmax - d_out;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int k = NPAD; k < NPAD + P->zres; k++)
        for (int j = NPAD; j < NPAD + P->yres; j++)
            for (int i = NPAD; i < NPAD + P->xres; i++) {
                double rad = xc3(S, i), f, tau;
                orc_cell* C = &S->C[IND3(S, i, j, k)];
                for (int side = 0; side < 2; side++) {
                    if (side == 0 && !(rad < inner)) continue;
                    if (side == 1 && !(rad > outer)) continue;
                    f = side == 0 ? (inner - rad) / d_in : (rad - outer) / d_out;
                    tau = (P->geomx == 0) ? 1.0 : pow(rad, 1.5);
                    f = get_ramping_fac(f);
                    f *= dt / tau;
                    orc_cell I = init_C3(P, rad, yc3(S, j), zc3(S, k));
                    C->r += f * (I.r - C->r);
                    C->p += f * (I.p - C->p);
                    C->u += f * (I.u - C->u);
                    C->v += f * (I.v - C->v);
                    C->w += f * (I.w - C->w);
                }
            }
}

/* src/timestep/timestep.cu:18-140 (ndim 3, orb_rot 0) */
double orc3_global_dt(orc3_state* S, double dt_prev)
{
    const orc_params* P = &S->P;
    double mx = 0.0;
    #pragma omp parallel for collapse(2) reduction(max : mx) schedule(static)
    for (int k = NPAD; k < NPAD + P->zres; k++)
        for (int j = NPAD; j < NPAD + P->yres; j++)
            for (int i = NPAD; i < NPAD + P->xres; i++) {
                const orc_cell* c = &S->C[IND3(S, i, j, k)];
                double rad = 1.0, rad_cyl = 1.0;
                if (P->geomy == 3) {
                    rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
                    rad_cyl = rad;
                } else if (P->geomy == 4) {
                    rad = 0.5 * (S->xa[i + 1] + S->xa[i]);
                    rad_cyl = rad * sin(0.5 * (S->za[k + 1] + S->za[k]));
                }
                double cs = sqrt(P->gam * c->p / c->r);
                double spd = fabs(c->u) + cs;
                double wid = fabs(S->xa[i + 1] - S->xa[i]);
                double tmp = fmax(spd / wid, 0.0);
                spd = fabs(c->v - rad_cyl * P->frame_omega - 0.0) + cs;
                wid = fabs(S->ya[j + 1] - S->ya[j]) * rad_cyl;
                tmp = fmax(spd / wid, tmp);
                spd = fabs(c->w) + cs;
                wid = fabs(S->za[k + 1] - S->za[k]) * rad;
                tmp = fmax(spd / wid, tmp);
                mx = fmax(mx, tmp);
            }
    double dt = P->cfl / mx;
    double lim = dt_prev * 1.1;
    return (dt < lim) ? dt : lim;
}

/* ------------------------------------------------------------- the step */
/* DS() + killwave (src/solver/solve.cu:212-292) with ndim 3 */
void orc3_solve(orc3_state* S, double t, double dt)
{
    const orc_params* P = &S->P;
    double hdt = 0.5 * dt;
    orc3_boundx(S);
    apply_source_terms3(S, 0.0, hdt);
    orc3_boundx(S);
    orc3_sweepx(S, dt);
    orc3_boundy(S);
    orc3_sweepy(S, dt);
    orc3_boundz(S);
    orc3_sweepz(S, dt);
    if (P->n_planet > 0) orbit_solution(P, &S->planet, t + dt);  /* evolve_planet (planet.cu:291-304) */
    apply_source_terms3(S, hdt, hdt);
    if (P->kill_flag) killwave3(S, dt);
}

/* The same step, copying the cell array (xarr*yarr*zarr cells) into out after
   every stage the stage driver oracle/ref_stages.cu dumps: kick1, sweepx,
   sweepy, sweepz, kick2 and, with damping, kill.  Returns the stages written. */
int orc3_solve_stages(orc3_state* S, double t, double dt, orc_cell* out)
{
    const orc_params* P = &S->P;
    double hdt = 0.5 * dt;
    size_t n = (size_t)S->xarr * S->yarr * S->zarr;
    int k = 0;
#define DUMP3() do { memcpy(out + (size_t)k * n, S->C, n * sizeof(orc_cell)); k++; } while (0)
    orc3_boundx(S);
    apply_source_terms3(S, 0.0, hdt);
    DUMP3();
    orc3_boundx(S);
    orc3_sweepx(S, dt);
    DUMP3();
    orc3_boundy(S);
    orc3_sweepy(S, dt);
    DUMP3();
    orc3_boundz(S);
    orc3_sweepz(S, dt);
    DUMP3();
    if (P->n_planet > 0) orbit_solution(P, &S->planet, t + dt);
    apply_source_terms3(S, hdt, hdt);
    DUMP3();
    if (P->kill_flag) {
        killwave3(S, dt);
        DUMP3();
    }
#undef DUMP3
    return k;
}

/* main.cu:320-360 without I/O (see orc_run) */
int orc3_run(orc3_state* S, double t0, double dt_prev, int max_step, double end_time, double* t_out, double* dt_out)
{
    double cur = t0, dt = (dt_prev > 0.0) ? dt_prev : end_time - cur;
    int nstep = 0, contu = 1;
    while (contu && nstep < max_step) {
        dt = orc3_global_dt(S, dt);
        if (cur + dt > end_time) {
            dt = end_time - cur;
            contu = 0;
        }
        orc3_solve(S, cur, dt);
        cur += dt;
        nstep++;
    }
    if (t_out) *t_out = cur;
    if (dt_out) *dt_out = dt;
    return nstep;
}
