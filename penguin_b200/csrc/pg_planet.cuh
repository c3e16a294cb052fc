// Analytic planet orbit (src/planet/planet.cu) and the device-resident clock,
// shared by the FP64 and FP32 kernels.  orbit_solution reads d.ramp_time,
// d.planet_mass and d.frame_omega of the disk.
#pragma once

#include "pg_common.cuh"

namespace pg {

__host__ __device__ inline double ramp_function(double t, double tau, double val) {  // planet.cu:7-17
    if (t < tau) return val * sin(HPI * t / tau);
    return val;
}
__device__ inline double ecc_anomaly(double n, double e, double t) {  // planet.cu:60-103
    double l = fmod(n * t, TWOPI);
    double D = -e * sin(l);
    if (e == 0.0) return l;
    else if (l == 0.0) return l;
    else if (l == PI) return l;
    else if (l == TWOPI) return l;
    double x, dx, d2x, eps, step, esinu, ecosu;
    int count = 0;
    do {
        sincos(l - D, &esinu, &ecosu);
        esinu *= e;
        ecosu *= e;
        x = D + esinu;
        dx = 1.0 - ecosu;
        d2x = -esinu;
        eps = 2.0 * x * d2x / dx / dx;
        if (fabs(eps) < 1.0) step = -(x / dx) * (1.0 + eps / 4.0 + eps * eps / 8.0 + 5.0 * eps * eps * eps / 64.0);
        else step = copysign(fmin(fabs(x / dx), HPI / 2.0), -x);
        D += step;
        count++;
    } while ((fabs(step) > 1.0e-12 || count < 10) && count < 200);
    return l - D;
}
template <class D>
__device__ inline void orbit_solution(const D& d, pg_body& b, double t) {  // planet.cu:105-133
    const double a = b.a, e = b.e;
    const double n = sqrt(1.0 / a / a / a);
    const double efac = sqrt(1.0 - e * e);
    const double B = e / (1.0 + efac);
    double u, cosu, sinu;
    u = ecc_anomaly(n, e, t);
    sincos(u, &sinu, &cosu);
    double f, ecosf, esinf;
    f = u + 2.0 * atan(B * sinu / (1.0 - B * cosu));
    sincos(f, &esinf, &ecosf);
    esinf *= e;
    ecosf *= e;
    b.m = ramp_function(t, d.ramp_time, d.planet_mass);
    b.x = a * efac * efac / (1.0 + ecosf);
    b.y = f - fmod(d.frame_omega * t, TWOPI) + PI;
    b.z = HPI;
    b.vx = n * a * esinf / efac;
    b.vy = n * (1.0 + ecosf) * (1.0 + ecosf) / efac / efac / efac;
    b.vz = 0.0;
}

// The star-planet pair on the reduced orbit (src/planet/planet.cu:135-175),
// both in the frame rotating at frame_omega: star = planets[0] (mass 1/(1+mp)),
// planet = planets[1] (mass mp/(1+mp)), mp ramped like a single planet's mass.
// The a, e and rs members of both bodies are kept.
template <class D>
__device__ inline void two_body_solution(const D& d, pg_body& star, pg_body& planet, double t) {
    const double a = star.a, e = star.e;
    const double n = sqrt(1.0 / a / a / a);
    const double efac = sqrt(1.0 - e * e);
    const double B = e / (1.0 + efac);
    double u, cosu, sinu;
    u = ecc_anomaly(n, e, t);
    sincos(u, &sinu, &cosu);
    double f, ecosf, esinf;
    f = u + 2.0 * atan(B * sinu / (1.0 - B * cosu));
    sincos(f, &esinf, &ecosf);
    esinf *= e;
    ecosf *= e;
    const double reduced_r = a * efac * efac / (1.0 + ecosf);
    const double reduced_p = f - fmod(d.frame_omega * t, TWOPI) + PI;
    const double mp = ramp_function(t, d.ramp_time, d.planet_mass);
    star.m = 1.0 / (1.0 + mp);
    star.x = reduced_r * mp / (1.0 + mp);
    star.y = fmod(reduced_p + PI, TWOPI);
    star.z = HPI;
    star.vx = n * a * esinf / efac * mp / (1.0 + mp);
    star.vy = n * (1.0 + ecosf) * (1.0 + ecosf) / efac / efac / efac;
    star.vz = 0.0;
    planet.m = mp / (1.0 + mp);
    planet.x = reduced_r * 1.0 / (1.0 + mp);
    planet.y = reduced_p;
    planet.z = HPI;
    planet.vx = n * a * esinf / efac * 1.0 / (1.0 + mp);
    planet.vy = n * (1.0 + ecosf) * (1.0 + ecosf) / efac / efac / efac;
    planet.vz = 0.0;
}

// evolve_planet (src/planet/planet.cu:291-304): the bodies at time t
__device__ inline void evolve_bodies(const DiskView& d, Scalars* sc, double t) {
    if (d.nplanet <= 0) return;
    if (d.twobd) two_body_solution(d, sc->star_next, sc->planet_next, t);
    else orbit_solution(d, sc->planet_next, t);
}

// Device-resident loop step (main.cu:322-339): dt = min(CFL/vmax, 1.1 dt_prev),
// clipped at end_time; then the planet at t + dt.  A step after the one that
// reached end_time only sets the done flag.
__device__ inline void advance_clock(const DiskView& d) {
    Scalars* sc = d.sc;
    if (sc->done) return;
    if (sc->pad_ || sc->t >= sc->end_time) {  // the previous step reached end_time
        sc->done = 1;
        return;
    }
    const double vmax = __longlong_as_double((long long)sc->vmax_bits);
    const double dtc = d.cfl / vmax;
    const double lim = sc->dt_prev * 1.1;
    double dt = (dtc < lim) ? dtc : lim;
    const double t = sc->t;
    if (t + dt > sc->end_time) {
        sc->dt_hold = dt;
        dt = sc->end_time - t;
        sc->pad_ = 1;
    }
    sc->dt = dt;
    sc->planet_cur = sc->planet_next;
    sc->star_cur = sc->star_next;
    evolve_bodies(d, sc, t + dt);
    sc->t = t + dt;
    sc->dt_prev = dt;
    sc->vmax_bits = 0ull;
    sc->steps += 1;
}

}  // namespace pg
