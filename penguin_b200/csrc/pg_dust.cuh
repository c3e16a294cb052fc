// One pressureless dust fluid next to the gas (dust_flag): AoS {r, u, v, w}
// FP64 (include/structs.h:19-46), transported by upwind PPM fluxes without a
// Riemann solver (src/solver/dust/dust.cu) and relaxed towards the gas velocity
// by an exponential drag integrator in both half-kicks (src/solver/sweeps.cu:
// 578-707).  No back-reaction on the gas.
#pragma once

#include "pg_common.cuh"

namespace pg {

struct DCell {
    double r, u, v, w;
};

__device__ __forceinline__ DCell load_dust(const pg_dust* buf, int xarr, int i, int j) {
    const double* q = reinterpret_cast<const double*>(buf + (size_t)i + (size_t)xarr * j);
    return DCell{q[0], q[1], q[2], q[3]};
}
__device__ __forceinline__ void store_dust(pg_dust* buf, int xarr, int i, int j, const DCell& c) {
    double* q = reinterpret_cast<double*>(buf + (size_t)i + (size_t)xarr * j);
    q[0] = c.r;
    q[1] = c.u;
    q[2] = c.v;
    q[3] = c.w;
}
__device__ __forceinline__ void store_dust_row_images(const DiskView& d, pg_dust* out, int i, int j, const DCell& c) {
    store_dust(out, d.xarr, i, j, c);
    if (d.ndim > 1) {
        if (j < 2 * NPAD) store_dust(out, d.xarr, i, j + d.yres, c);
        else if (j >= d.yres) store_dust(out, d.xarr, i, j - d.yres, c);
    }
}
// Interior dust cell and its ghost images (boundy_dust periodic, boundx_dust
// zero-gradient / reflecting: src/boundary/boundary.cu:64-113, 211-268); bound-0
// radial ghosts hold init_CD for good.
__device__ __forceinline__ void emit_dust(const DiskView& d, pg_dust* out, int i, int j, DCell c) {
    store_dust_row_images(d, out, i, j, c);
    const int nx = d.xres + NPAD;
    if (d.bound_lft == 1 && i == NPAD) {
        for (int n = 0; n < NPAD; ++n) store_dust_row_images(d, out, n, j, c);
    } else if (d.bound_lft == 2 && i < 2 * NPAD) {
        DCell m = c;
        m.u = -m.u;
        store_dust_row_images(d, out, 2 * NPAD - 1 - i, j, m);
    }
    if (d.bound_rgh == 1 && i == nx - 1) {
        for (int n = 0; n < NPAD; ++n) store_dust_row_images(d, out, nx + n, j, c);
    } else if (d.bound_rgh == 2 && i >= nx - NPAD) {
        DCell m = c;
        m.u = -m.u;
        store_dust_row_images(d, out, 2 * nx - 1 - i, j, m);
    }
}

// update_Dust (dust.cu:149-176)
__device__ __forceinline__ DCell update_dust(const DiskView& d, DCell Q, const DCell& D) {
    const double r_min = fmax(Q.r * 1.0e-10, d.dust_rmin);
    const double u_old = Q.u, v_old = Q.v, w_old = Q.w;
    Q.u *= Q.r;
    Q.v *= Q.r;
    Q.w *= Q.r;
    Q.r += D.r;
    Q.u += D.u;
    Q.v += D.v;
    Q.w += D.w;
    const double ir = 1.0 / Q.r;
    Q.u *= ir;
    Q.v *= ir;
    Q.w *= ir;
    if (Q.r < r_min) {
        Q.r = r_min;
        Q.u = u_old;
        Q.v = v_old;
        Q.w = w_old;
    }
    return Q;
}

// Dust part of apply_source_terms (sweeps.cu:578-595, 626-707, geomx 1 or 0,
// 2D): t_s from the gas cell C (T.r = C.r, T.p = C.p); the forces towards the gas
// velocity T (C itself when mdt = 0, else the gas velocity the kick predicted
// over mdt: Tu, Tv), re-evaluated at the dust velocity predicted over mdt with
// t_s at the predicted pressure Tp (C.p unless cooling changed it).
__device__ __forceinline__ DCell dust_kick(const DiskView& d, const Cell& C, double Tu, double Tv, double Tp,
                                           const DCell& Q, double gx, double gy, double gz, double ix, double mdt,
                                           double dt) {
    double ts = d.stokes / (sqrt(d.gam * C.p / C.r) / d.sc_h) / C.r;
    double fxd = (d.geomx == 1) ? Q.v * Q.v * ix : 0.0;
    fxd = fxd * ts + C.u - Q.u;
    double fyd = 0.0 * ts + C.v - Q.v;
    if (mdt != 0.0) {
        const double dtau = 1.0 - exp(-mdt / ts);
        DCell D;
        D.u = Q.u + fxd * dtau + gx * ts * dtau;
        D.v = Q.v + fyd * dtau + gy * ts * dtau;
        ts = d.stokes / (sqrt(d.gam * Tp / C.r) / d.sc_h) / C.r;  // at the predicted (cooled) pressure
        fxd = (d.geomx == 1) ? D.v * D.v * ix : 0.0;
        fxd = fxd * ts + Tu - Q.u;
        fyd = 0.0 * ts + Tv - Q.v;
    }
    const double dtau = 1.0 - exp(-dt / ts);
    DCell o;
    o.u = Q.u + fxd * dtau + gx * ts * dtau;
    o.v = Q.v + fyd * dtau + gy * ts * dtau;
    o.w = Q.w + 0.0 * dtau + gz * ts * dtau;
    o.r = Q.r;
    return o;
}

}  // namespace pg
