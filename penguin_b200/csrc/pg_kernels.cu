// penguin_b200 kernels for sm_100a: one Godunov timestep of PEnGUIn
// (src/solver/solve.cu:212-292) as five fused passes over the AoS state:
//
//   kick1   C -> T : viscous stress (src/viscosity/viscosity.cu:34-197) + first half-kick
//                    (src/solver/sweeps.cu:597-711, mdt = 0); stores the stress for kick2
//   sweep_x T -> C : radial Godunov sweep (src/solver/sweeps.cu:263-335)
//   sweep_y C -> T : azimuthal sweep (sweeps.cu:361-433) writing each cell at its
//                    orbital-advection shifted row (src/orbit/orbit.cu:17-99)
//   advect  T -> C : residual orbital advection (src/solver/advection/advection.cu:1-173)
//   kick2   C -> T : predictor kick, viscous stress of the predicted state and
//                    corrector kick (solve.cu:266-269), wave damping
//                    (src/killwave/killwave.cu:17-103) and the CFL signal speed
//                    for the next step (src/timestep/timestep.cu:18-97)
//
// plus a one-thread time kernel (dt, planet).  Every pass reads its tile with a
// TMA bulk tensor copy into shared memory and writes each cell together with its
// ghost images, so no separate boundary pass is needed between stages.
#include <cstdio>

#include "pg_common.cuh"
#include "pg_hydro.cuh"
#include "pg_internal.h"
#include "pg_planet.cuh"
#include "pg_dust.cuh"

namespace pg {

// ---------------------------------------------------------------- tiles
// Sweep and advection tiles: L outputs along the sweep times W pencils per CTA,
// each thread taking CPT cells (or faces, or outputs) of a phase, with NS TMA
// stages in flight (SwCfg).  The autotuner (pg_disk_autotune) picks one of the
// variants listed in SWEEP_VARIANTS per pass; the per-cell arithmetic does not
// depend on the choice.
template <int W_, int L_, int CPT_, int NS_, int MINB_ = 0>
struct SwCfg {
    static constexpr int W = W_, L = L_, CPT = CPT_, NS = NS_;
    static constexpr int TL = L + 2 * NPAD;                       // tile cells along the sweep
    static constexpr int P1 = L + 2;                               // cells reconstructed per pencil
    static constexpr int P2 = L + 1;                               // faces per pencil
    static constexpr int NST = P1 * W;                             // reconstructed cells
    static constexpr int NFX = P2 * W;                             // faces
    static constexpr int NOUT = L * W;                             // outputs
    static constexpr int THREADS = ((NST + CPT - 1) / CPT + 31) / 32 * 32;
    // CTAs per SM the registers allow at ~96 registers a thread, unless given
    static constexpr int MINB = MINB_ > 0 ? MINB_ : (65536 / (THREADS * 96) > 0 ? 65536 / (THREADS * 96) : 1);
    static constexpr int YCOLS = W + 2;                            // y tiles start one column early (16-B TMA x)
    static constexpr int XTILE = W * TL * 5;                       // doubles
    static constexpr int YTILE = TL * YCOLS * 5;
    static constexpr int TILE_MAX = ((XTILE > YTILE ? XTILE : YTILE) + 15) / 16 * 16;
    static constexpr bool X_OK = 5 * TL <= 256;                    // a TMA box is at most 256 elements wide
    static constexpr size_t SMEM = (size_t)(NS * TILE_MAX + 10 * NST + 7 * NFX) * 8 + 8 * NS + 128;
    static constexpr size_t AD_SMEM = (size_t)(NS * TILE_MAX + 5 * TL * W) * 8 + 8 * NS + 128;
};
// The variants, in the order of SweepVariant ids (pg_internal.h SWEEP_VARIANTS).
template <int V> struct SV;
template <> struct SV<0> { using G = SwCfg<8, 32, 1, 2>; };   // default
template <> struct SV<1> { using G = SwCfg<4, 32, 1, 2>; };
template <> struct SV<2> { using G = SwCfg<16, 16, 1, 2>; };
template <> struct SV<3> { using G = SwCfg<8, 16, 1, 2>; };
template <> struct SV<4> { using G = SwCfg<8, 32, 2, 2>; };
template <> struct SV<5> { using G = SwCfg<8, 32, 1, 3>; };
template <> struct SV<6> { using G = SwCfg<4, 32, 1, 3>; };
template <> struct SV<7> { using G = SwCfg<4, 64, 1, 2>; };   // azimuthal passes only (x box too wide)
template <> struct SV<8> { using G = SwCfg<4, 32, 1, 2, 5>; };  // registers capped for 5 CTAs per SM
template <> struct SV<9> { using G = SwCfg<8, 32, 1, 2, 3>; };  // registers capped for 3 CTAs per SM
static_assert(NSWEEP_VARIANTS == 10, "SV<> and SWEEP_VARIANTS list the same variants");

constexpr int ST_TX = 32, ST_TY = 8;        // stencil kernels: 32 x 8 outputs
constexpr int ST_HX = ST_TX + 2, ST_HY = ST_TY + 2;
constexpr int ST_THREADS = ST_TX * ST_TY;
constexpr int ST_TILE_N = ST_HX * ST_HY * 5;          // doubles in one cell tile
constexpr int ST_TILE = (ST_TILE_N + 15) / 16 * 16;     // rounded so every TMA target is 128-B aligned
constexpr int ST_VIS_N = ST_HX * ST_HY * 2;
constexpr int ST_VIS = (ST_VIS_N + 15) / 16 * 16;
constexpr size_t K1_SMEM = (size_t)2 * ST_TILE * 8 + 16 + 128;
constexpr int ST_GRAV = (ST_HX * ST_HY * 3 + 15) / 16 * 16;  // kick2: gravity of the predictor, per tile cell
// kick2: the tile's per-radius (34) and per-row (10) tables, staged once per tile
enum KRad { KR_RAD, KR_IRAD, KR_GSTAR, KR_NU, KR_IDX, KR_ROT, KR_VX, KR_KILL = KR_VX + 5, KR_N = KR_KILL + 4 };
enum KRow { KY_SIN, KY_COS, KY_IDY, KY_VY, KY_N = KY_VY + 4 };
constexpr int ST_TAB = (KR_N * ST_HX + KY_N * ST_HY + 15) / 16 * 16;
constexpr size_t K5_SMEM = (size_t)(3 * ST_TILE + 2 * ST_VIS + ST_GRAV + ST_TAB) * 8 + 16 + 128;

// --------------------------------------------------------- source terms
struct Grav {
    double gx, gy, gz;
};
// Star + planet gravity in the 2D cylindrical frame (src/solver/force/forces.cu:41-58,
// 182-327 with twobd_flag 0, pol = 0).  The star term is a per-radius table; the
// planet's angle enters through the per-row sin/cos table of this step
// (k_planet_trig) and 1/x_p^2 through the table's tail.
__device__ __forceinline__ Grav gravity_at(const DiskView& d, double gstar, double rad, double sinfac,
                                           double cosfac, double iplx2, const pg_body& p) {
    Grav g{0.0, 0.0, 0.0};
    if (d.geomx == 1) {
        g.gx = gstar;
        g.gz = -0.0;
        if (d.nplanet > 0) {
            const double plm = p.m, plx = p.x;
            const double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + p.rs * p.rs);
            const double ir = 1.0 / Rp;
            const double rs_fac = ir * ir * ir;
            g.gx += -plm * (rad - plx * cosfac) * rs_fac - plm * cosfac * iplx2;
            g.gy += -plm * plx * sinfac * rs_fac + plm * sinfac * iplx2;
        }
    }
    return g;
}
__device__ __forceinline__ Grav gravity(const DiskView& d, int i, double rad, double sinfac, double cosfac,
                                        double iplx2, const pg_body& p) {
    return gravity_at(d, d.geomx == 1 ? d.gstar[i] : 0.0, rad, sinfac, cosfac, iplx2, p);
}

// One body of the two-body frame as an inertial point mass
// (star_planet_grav_cyl_inertial, src/solver/force/forces.cu:89-106, z = 0).
__device__ __forceinline__ void inertial_pull(double rad, double sinfac, double cosfac, const pg_body& p, Grav& g) {
    const double plm = p.m, plx = p.x;
    const double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac + 0.0 * 0.0 + p.rs * p.rs);
    const double rs_fac = 1.0 / Rp / Rp / Rp;
    g.gx += -plm * (rad - plx * cosfac) * rs_fac;
    g.gy += -plm * plx * sinfac * rs_fac;
    g.gz += -plm * 0.0 * rs_fac;
}

// Gravity at cell (i, j) with the bodies of the first half-kick (which 0) or at
// t + dt (which 1).  In the two-body frame (twobd_flag 1, forces.cu:182-327)
// the star (planets[0]) and the planet (planets[1]) pull as inertial point
// masses and the fixed-star term and the indirect term drop out.
__device__ __forceinline__ Grav body_gravity(const DiskView& d, int i, int j, int which, const pg_body& pl,
                                             const pg_body& st) {
    const double* tr = d.trig + 4 * j + 2 * which;
    if (!d.twobd) return gravity(d, i, d.radx[i], tr[0], tr[1], d.trig[4 * d.yarr + which], pl);
    Grav g{0.0, 0.0, 0.0};
    if (d.geomx == 1) {
        const double* ts = d.strig + 4 * j + 2 * which;
        inertial_pull(d.radx[i], ts[0], ts[1], st, g);
        inertial_pull(d.radx[i], tr[0], tr[1], pl, g);
    }
    return g;
}

// One cell of apply_source_terms (src/solver/sweeps.cu:597-711): curvature,
// gravity and viscous acceleration; with mdt != 0 the forces are re-evaluated
// at the mdt-predicted velocities (sweeps.cu:663-687).

// Newtonian cooling of the pressure over dt (src/solver/cool/cool.cu:1-33): the
// specific energy p/r relaxes towards cs^2(xc) with t_c = beta r_cyl^1.5
// (cool 1, tabulated) or beta / r sqrt(p/r) / h (cool 2, r the density).
__device__ __forceinline__ double p_cool(const DiskView& d, int i, double p, double r, double dt) {
    const double tc = (d.cool == 1) ? d.coolx[i] : d.beta_cool * (1.0 / r) * (sqrt(p / r) / d.sc_h);
    const double e = p / r;
    const double e0 = d.cs2x[i];
    return r * (e0 + (e - e0) * exp(-dt / tc));
}

template <bool VISC>
__device__ __forceinline__ Cell kick(const DiskView& d, const Cell& C, double ix, const Grav& g, double vx,
                                     double vy, double mdt, double dt, double* Tu = nullptr, double* Tv = nullptr) {
    Cell T = C;
    const double ir = VISC ? 1.0 / C.r : 0.0;  // T.r == C.r throughout
    double fx = (d.geomx == 1) ? T.v * T.v * ix : 0.0;
    double fy = 0.0;
    const double fz = 0.0;
    if (VISC) {
        fx += vx * ir;
        if (d.ndim > 1) fy += vy * ir;
    }
    if (mdt != 0.0) {
        T.u = C.u + fx * mdt + g.gx * mdt;
        T.v = C.v + fy * mdt + g.gy * mdt;
        T.w = C.w + fz * mdt + g.gz * mdt;
        if (Tu) *Tu = T.u;  // the gas velocity the dust drag relaxes towards (sweeps.cu:679-687)
        if (Tv) *Tv = T.v;
        fx = (d.geomx == 1) ? T.v * T.v * ix : 0.0;
        fy = 0.0;
        if (VISC) {
            fx += vx * ir;
            if (d.ndim > 1) fy += vy * ir;
        }
    }
    Cell o;
    o.u = C.u + fx * dt + g.gx * dt;
    o.v = C.v + fy * dt + g.gy * dt;
    o.w = C.w + fz * dt + g.gz * dt;
    o.r = C.r;
    o.p = C.p;
    return o;
}

// Gathers the 3x3 stencil around tile cell (hx, hy) of a [ST_HY][ST_HX][5] tile.
__device__ __forceinline__ void gather9(const double* tile, int hx, int hy, const double nu[3], double* u,
                                        double* v, double* nr) {
#pragma unroll
    for (int n = 0; n < 9; ++n) {
        const int dx = (n % 3) - 1;
        const int dy = (n < 3) ? 0 : (n < 6 ? -1 : 1);
        const double* c = tile + ((hy + dy) * ST_HX + (hx + dx)) * 5;
        nr[n] = c[0] * nu[n % 3];
        u[n] = c[2];
        v[n] = c[3];
    }
}

// add_grid (src/output/output.cu:250-275): A += C (0.5 dt) / T on the interior
__device__ __forceinline__ void accumulate_average(const DiskView& d, int i, int j, const Cell& C, double hdt) {
    const double fac = hdt / d.ave_T;
    Cell* a = d.ave + (size_t)i + (size_t)d.xarr * j;
    a->r += C.r * fac;
    a->p += C.p * fac;
    a->u += C.u * fac;
    a->v += C.v * fac;
    a->w += C.w * fac;
}

__device__ __forceinline__ double signal_rate(const DiskView& d, const Cell& c, int i, int j,
                                              const DCell* dc = nullptr) {
    // src/timestep/timestep.cu:46-77 (cell widths as reciprocals); with dust the
    // dust speeds also bound dt (:64-74)
    const double rad_cyl = (d.geomy == 3) ? d.radx[i] : 1.0;
    const double cs = sqrt(d.gam * c.p / c.r);
    double spd = fabs(c.u) + cs;
    if (dc) spd = fmax(fabs(dc->u), spd);
    double tmp = fmax(spd * d.idx_x[i], 0.0);
    if (d.ndim > 1) {
        spd = fabs(c.v - rad_cyl * d.frame_omega - d.rot[i]) + cs;
        if (dc) spd = fmax(fabs(dc->v - rad_cyl * d.frame_omega - d.rot[i]), spd);
        tmp = fmax(spd * (d.idx_y[j] * ((d.geomy == 3) ? d.irad[i] : 1.0)), tmp);
    }
    return tmp;
}

// signal_rate with the cell's table entries passed in (kick2's staged tables):
// the same expressions
__device__ __forceinline__ double signal_rate_at(const DiskView& d, const Cell& c, double radx, double idxx,
                                                 double rot, double idyj, double irad, const DCell* dc = nullptr) {
    const double rad_cyl = (d.geomy == 3) ? radx : 1.0;
    const double cs = sqrt(d.gam * c.p / c.r);
    double spd = fabs(c.u) + cs;
    if (dc) spd = fmax(fabs(dc->u), spd);
    double tmp = fmax(spd * idxx, 0.0);
    if (d.ndim > 1) {
        spd = fabs(c.v - rad_cyl * d.frame_omega - rot) + cs;
        if (dc) spd = fmax(fabs(dc->v - rad_cyl * d.frame_omega - rot), spd);
        tmp = fmax(spd * (idyj * ((d.geomy == 3) ? irad : 1.0)), tmp);
    }
    return tmp;
}

// ================================================================ sweeps
// DIR 0: radial pencils (rows of the array), DIR 1: azimuthal pencils (columns).
// G: the tile configuration (SwCfg).
template <int DIR, class G>
__global__ void __launch_bounds__(G::THREADS, G::MINB)
    k_sweep(const __grid_constant__ CUtensorMap tm, const DiskView d, Cell* __restrict__ out, int ntx, int ntiles) {
    constexpr int SW_W = G::W, SW_LEN = G::L, SW_TL = G::TL, SW_P1 = G::P1, SW_P2 = G::P2;
    constexpr int SW_TILE_MAX = G::TILE_MAX, SW_NST = G::NST, SW_NFX = G::NFX, SWY_COLS = G::YCOLS;
    constexpr int SWX_TILE = G::XTILE, SWY_TILE = G::YTILE, NS = G::NS, NT = G::THREADS;
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    auto stage = [&](int n) { return smem + (n % NS) * SW_TILE_MAX; };
    double* st = smem + NS * SW_TILE_MAX;  // [10][SW_NST] interface states
    double* fl = st + 10 * SW_NST;         // [7][SW_NFX] fluxes
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 7 * SW_NFX);
    __shared__ int s_inc[SW_W];
    Scalars* sc = d.sc;
    if (sc->done) return;

    const int tid = threadIdx.x;
    const double dt = sc->dt;
    const double gam = d.gam;
    const uint32_t bytes = (DIR == 0 ? SWX_TILE : SWY_TILE) * 8;
    auto origin = [&](int tile, int& s0, int& q0) {
        const int bx = tile % ntx, by = tile / ntx;
        s0 = NPAD + SW_LEN * bx;                     // first output along the sweep
        q0 = (DIR == 0 ? d.ypad : NPAD) + SW_W * by;  // first pencil
    };
    auto issue = [&](int tile, int k) {
        int s0, q0;
        origin(tile, s0, q0);
        issue_begin(&bar[k % NS], bytes);
        if (DIR == 0) issue_box(stage(k), &tm, 5 * (s0 - NPAD), q0, &bar[k % NS]);
        else issue_box(stage(k), &tm, 5 * (q0 - 1), s0 - NPAD, &bar[k % NS]);
    };
    pipe_init<NS>(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0)
        for (int m = 0; m < NS - 1; ++m)
            if ((int)blockIdx.x + m * (int)gridDim.x < ntiles) issue(blockIdx.x + m * gridDim.x, m);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
    // tiles issued beyond this one (the one NS - 1 ahead is issued now)
    int ahead = 0;
    while (ahead < NS - 1 && tile_id + (ahead + 1) * (int)gridDim.x < ntiles) ++ahead;
    if (tid == 0 && ahead == NS - 1) issue(tile_id + (NS - 1) * gridDim.x, kt + NS - 1);
    int s0, q0;
    origin(tile_id, s0, q0);
    double* tile = stage(kt);

    if (DIR == 1 && tid < SW_W) {
        // set_orbital_advection (src/orbit/orbit.cu:74-99) for this column
        const int i = q0 + tid;
        int shift = 0;
        if (d.orbadv && i < NPAD + d.xres) {
            const double rad = d.radx[i];
            const double dy = d.dy0 * rad;
            const double rot = d.rot[i];
            shift = __double2int_rd(rot * dt / dy + 0.5);
            double speed = shift * dy / dt;
            speed = rot - speed;
            if (s0 == NPAD) {
                d.res[i] = speed;
                d.inc[i] = shift;
            }
        }
        s_inc[tid] = shift;
    }
    if (!pipe_wait<NS>(bar, kt, sc)) {
        pipe_drain<NS>(bar, kt, ahead, sc);
        return;
    }

    // ---- P1: reconstruction + both edge states of every cell
    for (int it = tid; it < SW_NST; it += NT) {
        const int q = (DIR == 0) ? it / SW_P1 : it % SW_W;
        const int t = 2 + ((DIR == 0) ? it % SW_P1 : it / SW_W);
        const int s = s0 - NPAD + t;
        const int qq = q0 + q;
        double r[5], p[5], u[5], v[5], w[5];
        double rad = 1.0, rot = 0.0, irad_q = 1.0;
        if (DIR == 1) {
            const int i = min(qq, d.xarr - 1);
            rad = (d.geomy == 3) ? d.radx[i] : 1.0;
            irad_q = (d.geomy == 3) ? d.irad[i] : 1.0;
            rot = d.rot[i];
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double* c = (DIR == 0) ? tile + (q * SW_TL + (t - 2 + k)) * 5
                                         : tile + ((t - 2 + k) * SWY_COLS + (q + 1)) * 5;
            r[k] = c[0];
            p[k] = c[1];
            if (DIR == 0) {
                u[k] = c[2];
                v[k] = c[3];
                if (d.geomx == 1) v[k] *= d.radx[min(max(s - 2 + k, 0), d.xarr - 1)];
                w[k] = c[4];
            } else {
                u[k] = c[3] - rot;
                if (d.geomy == 3) u[k] -= rad * d.frame_omega;
                v[k] = c[4];
                w[k] = c[2];
            }
        }
        const double cs0 = sqrt(gam * p[2] / r[2]);
        const double flat = flatten(1.0 / cs0, p[2], p[0], p[1], p[3], p[4], u[1], u[2], u[3]);
        const int sc_ = (DIR == 0) ? min(s, d.xarr - 1) : min(s, d.yarr - 1);
        const double* wt = ((DIR == 0) ? d.wx : d.wy) + 6 * sc_;
        const double* fa = (DIR == 0) ? d.xa : d.ya;
        const double idx = ((DIR == 0) ? d.idx_x : d.idx_y)[sc_];
        const Par R = recon(wt, r[0], r[1], r[2], r[3], r[4], flat);
        const Par P = recon(wt, p[0], p[1], p[2], p[3], p[4], flat);
        const Par U = recon(wt, u[0], u[1], u[2], u[3], u[4], flat);
        // in 2D the z-velocity (v here for DIR 1, w for DIR 0) is identically zero, and the
        // reconstruction of a zero stencil is exactly {+0, a0, +0}: skip it (CTA-uniform)
        const bool flat2d = d.ndim == 2;
        const Par V = (DIR == 1 && flat2d) ? Par{0.0, v[2], 0.0} : recon(wt, v[0], v[1], v[2], v[3], v[4], flat);
        const Par W = (DIR == 0 && flat2d) ? Par{0.0, w[2], 0.0} : recon(wt, w[0], w[1], w[2], w[3], w[4], flat);
        const double xl = fa[sc_], xr = fa[sc_ + 1];
        const double sdt = (DIR == 0) ? dt : dt * irad_q;
        const Half a = state_at_left_edge(gam, xl, idx, sdt, cs0, r[2], p[2], u[2], R, P, U, V, W);
        const Half b = state_at_right_edge(gam, xl, xr, idx, sdt, cs0, r[2], p[2], u[2], R, P, U, V, W);
        st[0 * SW_NST + it] = a.r;
        st[1 * SW_NST + it] = a.p;
        st[2 * SW_NST + it] = a.u;
        st[3 * SW_NST + it] = a.v;
        st[4 * SW_NST + it] = a.w;
        st[5 * SW_NST + it] = b.r;
        st[6 * SW_NST + it] = b.p;
        st[7 * SW_NST + it] = b.u;
        st[8 * SW_NST + it] = b.v;
        st[9 * SW_NST + it] = b.w;
    }
    __syncthreads();

    // ---- P2: HLLC flux at every face (left state from cell t-1, right from cell t)
    for (int it = tid; it < SW_NFX; it += NT) {
        const int q = (DIR == 0) ? it / SW_P2 : it % SW_W;
        const int t = 3 + ((DIR == 0) ? it % SW_P2 : it / SW_W);
        const int iL = (DIR == 0) ? q * SW_P1 + (t - 3) : (t - 3) * SW_W + q;
        const int iR = (DIR == 0) ? q * SW_P1 + (t - 2) : (t - 2) * SW_W + q;
        Half L, R;
        L.r = st[5 * SW_NST + iL];
        L.p = st[6 * SW_NST + iL];
        L.u = st[7 * SW_NST + iL];
        L.v = st[8 * SW_NST + iL];
        L.w = st[9 * SW_NST + iL];
        R.r = st[0 * SW_NST + iR];
        R.p = st[1 * SW_NST + iR];
        R.u = st[2 * SW_NST + iR];
        R.v = st[3 * SW_NST + iR];
        R.w = st[4 * SW_NST + iR];
        const Flux F = hllc(d.eos, d.ie, gam, L, R);
        fl[0 * SW_NFX + it] = F.r;
        fl[1 * SW_NFX + it] = F.p;
        fl[2 * SW_NFX + it] = F.u;
        fl[3 * SW_NFX + it] = F.v;
        fl[4 * SW_NFX + it] = F.w;
        fl[5 * SW_NFX + it] = F.pres;
        fl[6 * SW_NFX + it] = F.uprs;
    }
    __syncthreads();

    // ---- P3: flux differences, geometric sources, conservative update
    for (int it = tid; it < SW_LEN * SW_W; it += NT) {
        const int q = (DIR == 0) ? it / SW_LEN : it % SW_W;
        const int t = 3 + ((DIR == 0) ? it % SW_LEN : it / SW_W);
        const int s = s0 - NPAD + t;
        const int qq = q0 + q;
        const bool valid = (DIR == 0) ? (s < NPAD + d.xres && qq < d.ypad + d.yres)
                                      : (s < NPAD + d.yres && qq < NPAD + d.xres);
        if (valid) {
            const int f0 = (DIR == 0) ? q * SW_P2 + (t - 3) : (t - 3) * SW_W + q;
            const int f1 = (DIR == 0) ? f0 + 1 : f0 + SW_W;
            const double g0 = (DIR == 0 && d.geomx == 1) ? d.xa[s] : 1.0;  // eval_gfac (riemann.cu:5-11)
            const double g1 = (DIR == 0 && d.geomx == 1) ? d.xa[s + 1] : 1.0;
            const double pres0 = fl[5 * SW_NFX + f0], pres1 = fl[5 * SW_NFX + f1];
            // net_source (src/solver/riemann/riemann.cu:40-87)
            const double du = 0.5 * (g0 + g1) * (pres0 - pres1);
            double de = 0.0;
            if (d.eos == 2) {
                const double t0 = fl[6 * SW_NFX + f0] * g0, t1 = fl[6 * SW_NFX + f1] * g1;
                de = (d.ie == 0) ? t0 - t1 : 0.5 * (pres0 + pres1) * (t0 - t1);
            }
            Cell D;
            D.r = fl[0 * SW_NFX + f0] * g0 - fl[0 * SW_NFX + f1] * g1;
            D.p = (fl[1 * SW_NFX + f0] * g0 - fl[1 * SW_NFX + f1] * g1) + de;
            D.u = (fl[2 * SW_NFX + f0] * g0 - fl[2 * SW_NFX + f1] * g1) + du;
            D.v = fl[3 * SW_NFX + f0] * g0 - fl[3 * SW_NFX + f1] * g1;
            D.w = fl[4 * SW_NFX + f0] * g0 - fl[4 * SW_NFX + f1] * g1;
            const double* c = (DIR == 0) ? tile + (q * SW_TL + t) * 5 : tile + (t * SWY_COLS + (q + 1)) * 5;
            const Cell C0{c[0], c[1], c[2], c[3], c[4]};
            if (DIR == 0) {
                const double f = dt * d.ixv[s];
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (d.geomx == 1) D.v *= d.irad[s];
                const Cell Q = update_cell(d.eos, d.ie, gam, d.cs2x[s], C0, D, &sc->floor_hits);
                if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                emit(d, out, s, qq, Q);
            } else {
                const double rad = (d.geomy == 3) ? d.radx[qq] : 1.0;
                const double rot = d.rot[qq];
                const double f = dt * d.iyv[s] * ((d.geomy == 3) ? d.irad[qq] : 1.0);
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (d.geomy == 3) D.u += (rot + rad * d.frame_omega) * D.r;
                else D.u += rot * D.r;
                const Cell E{D.r, D.p, D.w, D.u, D.v};
                const Cell Q = update_cell(d.eos, d.ie, gam, d.cs2x[qq], C0, E, &sc->floor_hits);
                if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                int j = s;
                if (d.orbadv) {  // orbital shift T[(j+inc) mod N] = C[j] (orbit.cu:30-46)
                    int js = (s - d.ypad + s_inc[q]) % d.yres;
                    if (js < 0) js += d.yres;
                    j = js + d.ypad;
                }
                emit(d, out, qq, j, Q);
            }
        }
    }
    __syncthreads();  // stage k % NS, the state / flux arrays and s_inc are free again
    }
}

// ===================================================== residual advection
template <class G>
__global__ void __launch_bounds__(G::THREADS, G::MINB)
    k_advect(const __grid_constant__ CUtensorMap tm, const DiskView d, Cell* __restrict__ out, int ntx, int ntiles) {
    constexpr int SW_W = G::W, SW_LEN = G::L, SW_TL = G::TL, SW_TILE_MAX = G::TILE_MAX, SW_NST = G::NST;
    constexpr int SWY_COLS = G::YCOLS, SWY_TILE = G::YTILE, NS = G::NS, NT = G::THREADS;
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    auto stage = [&](int n) { return smem + (n % NS) * SW_TILE_MAX; };
    double* fl = smem + NS * SW_TILE_MAX;  // [5][SW_TL * SW_W] face fluxes, indexed by face t
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 5 * SW_TL * SW_W);
    Scalars* sc = d.sc;
    if (sc->done) return;
    const int tid = threadIdx.x;
    const double dt = sc->dt;
    constexpr int NFL = SW_TL * SW_W;
    auto origin = [&](int tile, int& s0, int& q0) {
        s0 = NPAD + SW_LEN * (tile % ntx);
        q0 = NPAD + SW_W * (tile / ntx);
    };
    auto issue = [&](int tile, int k) {
        int s0, q0;
        origin(tile, s0, q0);
        issue_begin(&bar[k % NS], SWY_TILE * 8);
        issue_box(stage(k), &tm, 5 * (q0 - 1), s0 - NPAD, &bar[k % NS]);
    };
    pipe_init<NS>(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0)
        for (int m = 0; m < NS - 1; ++m)
            if ((int)blockIdx.x + m * (int)gridDim.x < ntiles) issue(blockIdx.x + m * gridDim.x, m);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
    int ahead = 0;
    while (ahead < NS - 1 && tile_id + (ahead + 1) * (int)gridDim.x < ntiles) ++ahead;
    if (tid == 0 && ahead == NS - 1) issue(tile_id + (NS - 1) * gridDim.x, kt + NS - 1);
    int s0, q0;
    origin(tile_id, s0, q0);
    double* tile = stage(kt);
    if (!pipe_wait<NS>(bar, kt, sc)) {
        pipe_drain<NS>(bar, kt, ahead, sc);
        return;
    }

    // ---- P1: upwind PPM average over the swept fraction (advection.cu:20-67)
    for (int it = tid; it < SW_NST; it += NT) {
        const int q = it % SW_W;
        const int t = 2 + it / SW_W;
        const int s = min(s0 - NPAD + t, d.yarr - 1);
        const int i = min(q0 + q, d.xarr - 1);
        const double speed = d.res[i];
        const double sdt = dt * ((d.geomy == 3) ? d.irad[i] : 1.0);
        const double idx = d.idx_y[s];
        double r[5], p[5], u[5], v[5], w[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double* c = tile + ((t - 2 + k) * SWY_COLS + (q + 1)) * 5;
            r[k] = c[0]; p[k] = c[1]; u[k] = c[3]; v[k] = c[4]; w[k] = c[2];
        }
        const double* wt = d.wy + 6 * s;
        // CTA-uniform: with the isothermal EOS the pressure is reset from the density
        // after the update, so its flux is never used; in 2D the z-velocity is
        // identically zero, so its flux is zero
        const bool need_p = d.eos != 0, need_w = d.ndim != 2;
        const Par R = recon(wt, r[0], r[1], r[2], r[3], r[4], 0.0);
        const Par U = recon(wt, u[0], u[1], u[2], u[3], u[4], 0.0);
        const Par W = recon(wt, w[0], w[1], w[2], w[3], w[4], 0.0);
        Par P = R, V = R;
        if (need_p) P = recon(wt, p[0], p[1], p[2], p[3], p[4], 0.0);
        if (need_w) V = recon(wt, v[0], v[1], v[2], v[3], v[4], 0.0);
        const double xl = d.ya[s], xr = d.ya[s + 1];
        double fr, fp = 0.0, fu, fv = 0.0, fw;
        int face;
        if (speed > 0.0) {  // this cell is upwind of its upper face
            const double x0 = xr - speed * sdt;
            const Frac q_ = frac_right(lim01((x0 - xl) * idx));
            fr = aveR(q_, R);
            if (need_p) fp = aveR(q_, P);
            fu = aveR(q_, U) * fr;
            if (need_w) fv = aveR(q_, V) * fr;
            fw = aveR(q_, W) * fr;
            face = t + 1;
        } else {  // ... of its lower face
            const double x0 = xl - speed * sdt;
            const Frac q_ = frac_left(lim01((x0 - xl) * idx));
            fr = aveL(q_, R);
            if (need_p) fp = aveL(q_, P);
            fu = aveL(q_, U) * fr;
            if (need_w) fv = aveL(q_, V) * fr;
            fw = aveL(q_, W) * fr;
            face = t;
        }
        const int k = face * SW_W + q;
        fl[0 * NFL + k] = fr * speed;
        fl[1 * NFL + k] = fp * speed;
        fl[2 * NFL + k] = fu * speed;
        fl[3 * NFL + k] = fv * speed;
        fl[4 * NFL + k] = fw * speed;
    }
    __syncthreads();

    // ---- P2: flux difference and update_Cell_advect (advection.cu:88-105, 153-170)
    for (int it = tid; it < SW_LEN * SW_W; it += NT) {
        const int q = it % SW_W;
        const int t = 3 + it / SW_W;
        const int s = s0 - NPAD + t;
        const int i = q0 + q;
        if (s < NPAD + d.yres && i < NPAD + d.xres) {
            const int k0 = t * SW_W + q, k1 = (t + 1) * SW_W + q;
            Cell D;
            D.r = fl[0 * NFL + k0] * 1.0 - fl[0 * NFL + k1] * 1.0;
            D.p = fl[1 * NFL + k0] * 1.0 - fl[1 * NFL + k1] * 1.0;
            D.u = fl[2 * NFL + k0] * 1.0 - fl[2 * NFL + k1] * 1.0;
            D.v = fl[3 * NFL + k0] * 1.0 - fl[3 * NFL + k1] * 1.0;
            D.w = fl[4 * NFL + k0] * 1.0 - fl[4 * NFL + k1] * 1.0;
            double f = dt * d.iyv[s];
            D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
            if (d.geomy > 2) {
                f = d.irad[i];
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
            }
            const double* c = tile + (t * SWY_COLS + (q + 1)) * 5;
            Cell Q{c[0], c[1], c[2], c[3], c[4]};
            Q.u *= Q.r;
            Q.v *= Q.r;
            Q.w *= Q.r;
            Q.r += D.r;
            Q.p += D.p;
            Q.u += D.w;
            Q.v += D.u;
            Q.w += D.v;
            const double ir = 1.0 / Q.r;
            Q.u *= ir;
            Q.v *= ir;
            Q.w *= ir;
            if (d.eos == 0) Q.p = d.cs2x[i] * Q.r;
            if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
            emit(d, out, i, s, Q);
        }
    }
    __syncthreads();
    }
}

// ====================================================== kick 1 (+ stress)
// 4 CTAs per SM (64 registers, a few bytes of spills with the stress): 32 warps
// hide the table and tile loads better than 24 (0.120 -> 0.106 ms)
template <bool VISC>
__global__ void __launch_bounds__(ST_THREADS, 4)
    k_kick1(const __grid_constant__ CUtensorMap tm, const DiskView d, Cell* __restrict__ out,
            double* __restrict__ vis, int ntx, int ntiles, const pg_dust* __restrict__ din,
            pg_dust* __restrict__ dout) {
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    auto stage = [&](int n) { return smem + (n & 1) * ST_TILE; };
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * ST_TILE);
    Scalars* sc = d.sc;
    if (sc->done) return;
    const int tid = threadIdx.x;
    const double hdt = 0.5 * sc->dt;
    auto origin = [&](int tile, int& i0, int& j0) {
        i0 = NPAD + ST_TX * (tile % ntx);
        j0 = d.ypad + ST_TY * (tile / ntx);
    };
    auto issue = [&](int tile, int k) {
        int i0, j0;
        origin(tile, i0, j0);
        issue_begin(&bar[k & 1], ST_TILE_N * 8);
        issue_box(stage(k), &tm, 5 * (i0 - 1), j0 - 1, &bar[k & 1]);
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int i0, j0;
        origin(tile_id, i0, j0);
        const double* tile = stage(kt);
        if (!pipe_wait(bar, kt, sc)) {
        pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
        return;
    }
        const int hx = 1 + tid % ST_TX, hy = 1 + tid / ST_TX;
        const int i = i0 + hx - 1, j = j0 + hy - 1;
        if (i < NPAD + d.xres && j < d.ypad + d.yres) {
            const double* c = tile + (hy * ST_HX + hx) * 5;
            const Cell C{c[0], c[1], c[2], c[3], c[4]};
            double vx = 0.0, vy = 0.0;
            if (VISC) {
                double nu[3], u[9], v[9], nr[9];
#pragma unroll
                for (int n = 0; n < 3; ++n) nu[n] = d.nux[i + n - 1];
                gather9(tile, hx, hy, nu, u, v, nr);
                viscous(d.visx + 5 * i, d.visy + 4 * j, u, v, nr, vx, vy);
                // the stress is kept for the predictor of kick2, with its periodic images
                const size_t m0 = (size_t)i + (size_t)d.xarr * j;
                vis[2 * m0] = vx;
                vis[2 * m0 + 1] = vy;
                int jimg = -1;
                if (j < 2 * NPAD) jimg = j + d.yres;
                else if (j >= d.yres) jimg = j - d.yres;
                if (jimg >= 0) {
                    const size_t m = (size_t)i + (size_t)d.xarr * jimg;
                    vis[2 * m] = vx;
                    vis[2 * m + 1] = vy;
                }
            }
            const Grav g = body_gravity(d, i, j, 0, sc->planet_cur, sc->star_cur);
            Cell Q = kick<VISC>(d, C, d.irad[i], g, vx, vy, 0.0, hdt);
            if (d.cool) Q.p = p_cool(d, i, C.p, C.r, hdt);  // sweeps.cu:695-699
            emit(d, out, i, j, Q);
            if (d.ave) accumulate_average(d, i, j, C, hdt);  // averaging(dev, 0.5 dt, T) before solve
            if (din) {  // dust half-kick: drag towards the gas cell C (sweeps.cu:626-707, mdt = 0)
                const DCell D = dust_kick(d, C, C.u, C.v, C.p, load_dust(din, d.xarr, i, j), g.gx, g.gy, g.gz,
                                          d.irad[i], 0.0, hdt);
                emit_dust(d, dout, i, j, D);
            }
        }
        __syncthreads();
    }
}

// ============================================ kick 2 + damping + CFL speed
// 3 CTAs per SM (80 registers, no spills; 65 KB of shared memory each): the
// pass waits on table and tile loads, and 24 warps per SM hide them better than
// the 16 its natural 102 registers allow (0.222 -> 0.181 ms on the 1024x3072 disk)
template <bool VISC>
__global__ void __launch_bounds__(ST_THREADS, 3)
    k_kick2(const __grid_constant__ CUtensorMap tm, const __grid_constant__ CUtensorMap tv, const DiskView d,
            Cell* __restrict__ out, int ntx, int ntiles, const pg_dust* __restrict__ din,
            pg_dust* __restrict__ dout) {
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    auto stage = [&](int n) { return smem + (n & 1) * ST_TILE; };                   // C with 1 halo
    auto vstage = [&](int n) { return smem + 2 * ST_TILE + (n & 1) * ST_VIS; };  // stress of the first evaluation
    double* tp = smem + 2 * ST_TILE + 2 * ST_VIS;                      // predicted state with 1 halo
    double* gc = tp + ST_TILE;  // gravity at the predictor's cells: the corrector's is the same (time `next`)
    double* tb = gc + ST_GRAV;  // the tile's tables: [KR_N][ST_HX] per radius, then [KY_N][ST_HY] per row
    double* ty = tb + KR_N * ST_HX;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tb + ST_TAB);
    Scalars* sc = d.sc;
    if (sc->done) return;
    const int tid = threadIdx.x;
    const double dt = sc->dt, hdt = 0.5 * dt;
    const pg_body pl = sc->planet_next;
    const pg_body st = sc->star_next;
    // the disk's gravity comes from the staged tables; the two-body frame reads its own
    const bool disk_grav = !d.twobd;
    const double iplx2 = disk_grav ? d.trig[4 * d.yarr + 1] : 0.0;
    auto origin = [&](int tile, int& i0, int& j0) {
        i0 = NPAD + ST_TX * (tile % ntx);
        j0 = d.ypad + ST_TY * (tile / ntx);
    };
    // Per-radius and per-row table entries of the tile and its halo, read once per
    // tile (coalesced) instead of once per cell: the pass is bound by the latency of
    // those loads.  Indices past the grid are clamped; those cells are not used.
    auto stage_tables = [&](int i0, int j0) {
        for (int it = tid; it < KR_N * ST_HX; it += ST_THREADS) {
            const int f = it / ST_HX, hx = it % ST_HX;
            const int i = min(max(i0 - 1 + hx, 0), d.xarr - 1);
            double v = 0.0;
            if (f == KR_RAD) v = d.radx[i];
            else if (f == KR_IRAD) v = d.irad[i];
            else if (f == KR_GSTAR) v = d.geomx == 1 ? d.gstar[i] : 0.0;
            else if (f == KR_NU) v = VISC ? d.nux[i] : 0.0;
            else if (f == KR_IDX) v = d.idx_x[i];
            else if (f == KR_ROT) v = d.ndim > 1 ? d.rot[i] : 0.0;
            else if (f < KR_KILL) v = VISC ? d.visx[5 * i + (f - KR_VX)] : 0.0;
            else v = d.kill ? d.killx[4 * i + (f - KR_KILL)] : 0.0;
            tb[it] = v;
        }
        for (int it = tid; it < KY_N * ST_HY; it += ST_THREADS) {
            const int f = it / ST_HY, hy = it % ST_HY;
            const int j = min(max(j0 - 1 + hy, 0), d.yarr - 1);  // 1D: one row, no ghost rows
            double v = 0.0;
            if (f == KY_SIN) v = disk_grav ? d.trig[4 * j + 2] : 0.0;
            else if (f == KY_COS) v = disk_grav ? d.trig[4 * j + 3] : 0.0;
            else if (f == KY_IDY) v = d.ndim > 1 ? d.idx_y[j] : 0.0;
            else v = VISC ? d.visy[4 * j + (f - KY_VY)] : 0.0;
            ty[it] = v;
        }
    };
    // gravity at tile cell (hx, hy), bodies at t + dt
    auto grav = [&](int hx, int hy, int i, int j) {
        if (disk_grav)
            return gravity_at(d, tb[KR_GSTAR * ST_HX + hx], tb[KR_RAD * ST_HX + hx], ty[KY_SIN * ST_HY + hy],
                              ty[KY_COS * ST_HY + hy], iplx2, pl);
        return body_gravity(d, i, j, 1, pl, st);
    };
    auto issue = [&](int tile, int k) {
        int i0, j0;
        origin(tile, i0, j0);
        issue_begin(&bar[k & 1], (ST_TILE_N + (VISC ? ST_VIS_N : 0)) * 8);
        issue_box(stage(k), &tm, 5 * (i0 - 1), j0 - 1, &bar[k & 1]);
        if (VISC) issue_box(vstage(k), &tv, 2 * (i0 - 1), j0 - 1, &bar[k & 1]);
    };
    pipe_init(bar);
    double vmax = 0.0;
    if ((int)blockIdx.x < ntiles) {
        if (tid == 0) issue(blockIdx.x, 0);
        int kt = 0;
        for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
            if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
            int i0, j0;
            origin(tile_id, i0, j0);
            const double* tile = stage(kt);
            const double* tvis = vstage(kt);
            stage_tables(i0, j0);  // while the tile's copy is in flight
            __syncthreads();
            if (!pipe_wait(bar, kt, sc)) {
        pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
        return;
    }

            if (VISC) {
                // predictor (sweeps.cu:713-729 with mdt = dt = dt/2) on the tile and its halo
                for (int it = tid; it < ST_HX * ST_HY; it += ST_THREADS) {
                    const int hx = it % ST_HX, hy = it / ST_HX;
                    const int i = i0 - 1 + hx, j = j0 - 1 + hy;
                    if (i < NPAD || i >= NPAD + d.xres || j < 0 || j >= d.yarr) continue;
                    const double* c = tile + it * 5;
                    const Cell C{c[0], c[1], c[2], c[3], c[4]};
                    const Grav g = grav(hx, hy, i, j);
                    gc[3 * it] = g.gx;
                    gc[3 * it + 1] = g.gy;
                    gc[3 * it + 2] = g.gz;
                    const Cell Q = kick<true>(d, C, tb[KR_IRAD * ST_HX + hx], g, tvis[2 * it], tvis[2 * it + 1], hdt,
                                              hdt);
                    double* o = tp + it * 5;
                    o[0] = Q.r; o[1] = Q.p; o[2] = Q.u; o[3] = Q.v; o[4] = Q.w;
                }
                __syncthreads();
                // radial ghosts of the predicted state (boundx2, src/boundary/boundary.cu:722-820):
                // the stencil only reaches the innermost ghost column on either side, which
                // only tiles at the radial edges hold (a CTA-uniform test, so the barrier
                // below is skipped by all threads or none)
                const bool redge = i0 - 1 <= NPAD - 1 || i0 - 2 + ST_HX >= NPAD + d.xres;
                if (redge) {
                for (int it = tid; it < ST_HX * ST_HY; it += ST_THREADS) {
                    const int hx = it % ST_HX, hy = it / ST_HX;
                    const int i = i0 - 1 + hx;
                    const int side = (i == NPAD - 1) ? 0 : ((i == NPAD + d.xres) ? 1 : -1);
                    if (side < 0) continue;
                    const int bnd = side == 0 ? d.bound_lft : d.bound_rgh;
                    double* o = tp + (hy * ST_HX + hx) * 5;
                    const double* src;
                    if (bnd == 0) src = tile + (hy * ST_HX + hx) * 5;  // constant analytic state
                    else {
                        // the adjacent interior cell is both the copy and the reflection source
                        const int hs = side == 0 ? hx + 1 : hx - 1;
                        src = tp + (hy * ST_HX + hs) * 5;
                    }
                    o[0] = src[0]; o[1] = src[1]; o[2] = src[2]; o[3] = src[3]; o[4] = src[4];
                    if (bnd == 2) o[2] = -o[2];
                }
                __syncthreads();
                }
            }

            const int hx = 1 + tid % ST_TX, hy = 1 + tid / ST_TX;
            const int i = i0 + hx - 1, j = j0 + hy - 1;
            if (i < NPAD + d.xres && j < d.ypad + d.yres) {
                const double* c = tile + (hy * ST_HX + hx) * 5;
                const Cell C{c[0], c[1], c[2], c[3], c[4]};
                double vx = 0.0, vy = 0.0;
                const double irad = tb[KR_IRAD * ST_HX + hx];
                if (VISC) {
                    double nu[3], u[9], v[9], nr[9], X[5], Y[4];
#pragma unroll
                    for (int n = 0; n < 3; ++n) nu[n] = tb[KR_NU * ST_HX + hx + n - 1];
#pragma unroll
                    for (int n = 0; n < 5; ++n) X[n] = tb[(KR_VX + n) * ST_HX + hx];
#pragma unroll
                    for (int n = 0; n < 4; ++n) Y[n] = ty[(KY_VY + n) * ST_HY + hy];
                    gather9(tp, hx, hy, nu, u, v, nr);
                    viscous(X, Y, u, v, nr, vx, vy);
                }
                const int ic = 3 * (hy * ST_HX + hx);
                const Grav g = VISC ? Grav{gc[ic], gc[ic + 1], gc[ic + 2]} : grav(hx, hy, i, j);
                double Tu = C.u, Tv = C.v;
                Cell Q = kick<VISC>(d, C, irad, g, vx, vy, hdt, hdt, &Tu, &Tv);
                // cooling over dt/2; the predictor cools over mdt = dt/2 as well, so Q.p is also
                // the predicted pressure the dust's second stopping time reads (sweeps.cu:668-699)
                if (d.cool) Q.p = p_cool(d, i, C.p, C.r, hdt);
                const double Tp = Q.p;
                if (d.kill) {
                    // killwave (src/killwave/killwave.cu:48-100): relax towards init_C
                    const double* I = d.initx + 5 * i;
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        const double tau = tb[(KR_KILL + 2 * side + 1) * ST_HX + hx];
                        if (tau > 0.0) {
                            double f = tb[(KR_KILL + 2 * side) * ST_HX + hx];
                            f *= dt / tau;
                            Q.r += f * (I[0] - Q.r);
                            Q.p += f * (I[1] - Q.p);
                            Q.u += f * (I[2] - Q.u);
                            Q.v += f * (I[3] - Q.v);
                            Q.w += f * (I[4] - Q.w);
                        }
                    }
                }
                if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                if (din) {  // dust corrector half-kick towards the predicted gas velocity (sweeps.cu:663-707)
                    const DCell D = dust_kick(d, C, Tu, Tv, Tp, load_dust(din, d.xarr, i, j), g.gx, g.gy, g.gz,
                                              irad, hdt, hdt);
                    emit_dust(d, dout, i, j, D);
                    vmax = fmax(vmax, signal_rate_at(d, Q, tb[KR_RAD * ST_HX + hx], tb[KR_IDX * ST_HX + hx],
                                                     tb[KR_ROT * ST_HX + hx], ty[KY_IDY * ST_HY + hy], irad, &D));
                } else {
                    vmax = fmax(vmax, signal_rate_at(d, Q, tb[KR_RAD * ST_HX + hx], tb[KR_IDX * ST_HX + hx],
                                                     tb[KR_ROT * ST_HX + hx], ty[KY_IDY * ST_HY + hy], irad));
                }
                emit(d, out, i, j, Q);
                if (d.ave) accumulate_average(d, i, j, Q, hdt);  // ... and after it
            }
            __syncthreads();
        }
    }
    block_max_to<ST_THREADS>(&sc->vmax_bits, vmax);
}

// ================================================================ misc
__global__ void k_cfl(const DiskView d, const Cell* __restrict__ in, const pg_dust* __restrict__ din) {
    const long long n = (long long)d.xres * d.yres;
    double vmax = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(k % d.xres);
        const int j = d.ypad + (int)(k / d.xres);
        if (din) {
            const DCell D = load_dust(din, d.xarr, i, j);
            vmax = fmax(vmax, signal_rate(d, load_cell(in, d.xarr, i, j), i, j, &D));
        } else {
            vmax = fmax(vmax, signal_rate(d, load_cell(in, d.xarr, i, j), i, j));
        }
    }
    block_max_to<256>(&d.sc->vmax_bits, vmax);
}

__global__ void k_reset_vmax(Scalars* sc) { sc->vmax_bits = 0ull; }

// Opens a device-resident run without a host round trip.  main.cu:144 + 322:
// the first step after a (re)start is capped by end_time - t; after a clip at
// end_time the step the clip replaced caps the next one (main.cu:333-338, 425).
__global__ void k_run_begin(Scalars* sc, double end_time, int fresh) {
    if (fresh) sc->dt_prev = end_time - sc->t;
    else if (sc->dt_hold > 0.0) sc->dt_prev = sc->dt_hold;
    sc->dt_hold = 0.0;
    sc->end_time = end_time;
    sc->done = 0;
    sc->pad_ = 0;
}

// Host-supplied t, dt (pg_*_solve): planet for this step, reset of the signal-speed max.
__global__ void k_set_time(const DiskView d, double t, double dt) {
    Scalars* sc = d.sc;
    sc->done = 0;
    sc->dt = dt;
    sc->planet_cur = sc->planet_next;
    sc->star_cur = sc->star_next;
    evolve_bodies(d, sc, t + dt);  // evolve_planet (solve.cu:264)
    sc->t = t + dt;
    sc->dt_prev = dt;
    sc->vmax_bits = 0ull;
    sc->steps += 1;
}

// Device-resident loop step of one disk (advance_clock).
__global__ void k_time_step(const DiskView d) { advance_clock(d); }

__global__ void k_init_planet(const DiskView d, double a, double e, double rs, double t) {
    // init_planet (src/planet/planet.cu:319-402): one planet, or the star-planet
    // pair of the two-body frame (the star unsmoothed)
    pg_body b{}, s{};
    b.a = s.a = a;
    b.e = s.e = e;
    b.rs = 0.0;
    if (d.twobd) two_body_solution(d, s, b, t);
    else orbit_solution(d, b, t);
    b.rs = rs;
    d.sc->planet_next = b;
    d.sc->planet_cur = b;
    d.sc->star_next = s;
    d.sc->star_cur = s;
}

// Per-index tables evaluated with the device's own pow/sqrt/__sinf so they carry
// the same bits as the reference's device-side evaluations.
struct TabArgs {
    double sc_h, planet_radius, p_alpha, p_beta, ss_alpha, frame_omega;
    double xmin, xmax, kill_width, kill_width_out;
    int visc, orbadv, kill, init_flag, geomx;
};
__device__ inline double d_cs2(const TabArgs& a, double x) {  // init.cu:7-17
    double coeff = a.sc_h * a.sc_h * (1.0 / a.planet_radius);
    if (a.geomx == 0) return coeff;
    return coeff * pow(x / a.planet_radius, -a.p_beta);
}
__device__ inline double d_h(const TabArgs& a, double x) {  // init.cu:20-29
    if (a.geomx == 0) return a.sc_h;
    return sqrt(d_cs2(a, x) * pow(x, 3));
}
__device__ inline double d_nu(const TabArgs& a, double x) {  // init.cu:31-50
    if (!a.visc) return 0.0;
    double coeff = a.ss_alpha * sqrt(d_cs2(a, a.planet_radius)) * d_h(a, a.planet_radius);
    if (a.geomx == 0) return coeff;
    return coeff * pow(x / a.planet_radius, a.p_alpha);
}
__device__ inline double d_r(const TabArgs& a, double x) { return pow(x / a.planet_radius, -a.p_alpha) * 1.0; }
__device__ inline double d_p(const TabArgs& a, double x) { return d_cs2(a, x) * d_r(a, x); }
__device__ inline void d_initC(const TabArgs& a, double x, double* q) {  // init.cu:431-442 (init_flag 2)
    if (a.init_flag == 2) {
        q[0] = d_r(a, x);
        q[1] = d_p(a, x);
        q[2] = -1.5 * d_nu(a, x) / x;
        const double rho = d_r(a, x);
        const double dr = 1.1514178e-7;
        const double dP_dr = (d_p(a, x + dr) - d_p(a, x - dr)) / (2.0 * dr);
        q[3] = sqrt(1.0 / x + (x / rho) * dP_dr);
        q[4] = 0.0;
    } else {
        q[0] = 1.0; q[1] = 1.0; q[2] = 0.0; q[3] = 0.0; q[4] = 0.0;
    }
}
__device__ inline double ramping_fac(double x) {  // killwave.cu:8-14
    double f = __sinf(HPI * x);
    f *= f;
    return f;
}

__global__ void k_init_tables(const DiskView d, TabArgs a, double* radx, double* cs2x, double* nux, double* initx,
                              double* killx, double* rot, double* ycraw, double* ycj, double* xrec, double* yrec) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < d.xarr) {
        const double x = 0.5 * (d.xa[k + 1] + d.xa[k]);
        radx[k] = x;
        cs2x[k] = d_cs2(a, x);
        nux[k] = d_nu(a, x);
        d_initC(a, x, initx + 5 * k);
        // orb_rot (src/orbit/orbit.cu:57-69)
        if (rot) rot[k] = a.orbadv ? initx[5 * k + 3] - x * a.frame_omega : 0.0;
        // cooling time of cool_flag 1 (src/solver/cool/cool.cu:1-12, 15-27)
        if (d.coolx) const_cast<double*>(d.coolx)[k] = pow((a.geomx == 1) ? x : 1.0, 1.5) * d.beta_cool;
        const double d_in = d_h(a, a.xmin) * a.kill_width;
        const double d_out = d_h(a, a.xmax) * a.kill_width_out;
        const double inner = a.xmin + d_in;
        const double outer = a.xmax - d_out;
        double* kt = killx + 4 * k;
        kt[0] = kt[1] = kt[2] = kt[3] = 0.0;
        if (a.kill && k >= NPAD && k < NPAD + d.xres) {
            if (x < inner) {
                double f = (inner - x) / d_in;
                kt[1] = (a.geomx == 0) ? 1.0 : pow(x, 1.5);
                kt[0] = ramping_fac(f);
            }
            if (x > outer) {
                double f = (x - outer) / d_out;
                kt[3] = (a.geomx == 0) ? 1.0 : pow(x, 1.5);
                kt[2] = ramping_fac(f);
            }
        }
        // reciprocals and star gravity; xrec layout: idx_x, ixv, irad, gstar [xarr each], visx [5 xarr]
        xrec[k] = 1.0 / (d.xa[k + 1] - d.xa[k]);
        xrec[d.xarr + k] = 1.0 / d.xv[k];
        xrec[2 * d.xarr + k] = 1.0 / x;
        if (a.geomx == 1) {
            const double dis = sqrt(x * x + 0.0 * 0.0);
            xrec[3 * d.xarr + k] = -x / dis / dis / dis;  // forces.cu:203-204
        } else {
            xrec[3 * d.xarr + k] = 0.0;
        }
        double* vx = xrec + 4 * d.xarr + 5 * k;
        vx[0] = vx[1] = vx[2] = vx[3] = vx[4] = 0.0;
        if (k >= 1 && k + 1 < d.xarr) {
            const double r0 = 0.5 * (d.xa[k] + d.xa[k - 1]), r2 = 0.5 * (d.xa[k + 2] + d.xa[k + 1]);
            vx[0] = 1.0 / (r2 - r0);
            vx[1] = 1.0 / (r2 - x);
            vx[2] = 1.0 / (x - r0);
            vx[3] = 1.0 / (0.5 * (r2 - r0));
            vx[4] = 1.0 / x;
        }
    }
    if (k < d.yarr) {
        ycraw[k] = 0.5 * (d.ya[k + 1] + d.ya[k]);
        int jm = k;
        if (d.ndim > 1) {
            if (k < d.ypad) jm = k + d.yres;
            else if (k >= d.ypad + d.yres) jm = k - d.yres;
        }
        ycj[k] = 0.5 * (d.ya[jm + 1] + d.ya[jm]);
        // yrec layout: idx_y, iyv [yarr each], visy [4 yarr]
        yrec[k] = 1.0 / (d.ya[k + 1] - d.ya[k]);
        yrec[d.yarr + k] = 1.0 / d.yv[k];
        double* vy = yrec + 2 * d.yarr + 4 * k;
        vy[0] = vy[1] = vy[2] = vy[3] = 0.0;
        if (k >= 1 && k + 1 < d.yarr) {
            const double t0 = 0.5 * (d.ya[k] + d.ya[k - 1]), t1 = 0.5 * (d.ya[k + 1] + d.ya[k]);
            const double t2 = 0.5 * (d.ya[k + 2] + d.ya[k + 1]);
            vy[0] = 1.0 / (t2 - t0);
            vy[1] = 1.0 / (t2 - t1);
            vy[2] = 1.0 / (t1 - t0);
            vy[3] = 1.0 / (0.5 * (t2 - t0));
        }
    }
}

// Per row, sin and cos of (azimuth - planet angle) for the planet of the first
// half-kick and for the planet at t+dt, and 1/x_p^2 of both (forces.cu:41-58).
__global__ void k_planet_trig(const DiskView d) {
    const Scalars* sc = d.sc;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const pg_body& a = sc->planet_cur;
    const pg_body& b = sc->planet_next;
    if (j < d.yarr) {
        double* t = d.trig + 4 * j;
        sincos(d.ycj[j] - (a.y + 0.0 * a.vy), &t[0], &t[1]);
        sincos(d.ycj[j] - (b.y + 0.0 * b.vy), &t[2], &t[3]);
        if (d.twobd) {
            double* u = d.strig + 4 * j;
            sincos(d.ycj[j] - (sc->star_cur.y + 0.0 * sc->star_cur.vy), &u[0], &u[1]);
            sincos(d.ycj[j] - (sc->star_next.y + 0.0 * sc->star_next.vy), &u[2], &u[3]);
        }
    }
    if (j == 0) {
        d.trig[4 * d.yarr] = 1.0 / a.x / a.x;
        d.trig[4 * d.yarr + 1] = 1.0 / b.x / b.x;
    }
}

// Bound-0 radial ghosts hold init_C (src/boundary/boundary.cu:30-33, 56-59) in every row.
__global__ void k_init_xghosts(const DiskView d, Cell* buf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 2 * NPAD * d.yarr) return;
    const int j = k / (2 * NPAD);
    const int n = k % (2 * NPAD);
    const int i = n < NPAD ? n : d.xres + n;
    const int bnd = n < NPAD ? d.bound_lft : d.bound_rgh;
    if (bnd != 0) return;
    const double* I = d.initx + 5 * i;
    store_cell(buf, d.xarr, i, j, Cell{I[0], I[1], I[2], I[3], I[4]});
}

// boundy then boundx (src/boundary/boundary.cu:141-209, 13-62) on one buffer.
__global__ void k_bound_y(const DiskView d, Cell* buf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (d.ndim < 2 || k >= d.xarr * NPAD) return;
    const int i = k % d.xarr, n = k / d.xarr;
    store_cell(buf, d.xarr, i, n, load_cell(buf, d.xarr, i, d.yres + n));
    store_cell(buf, d.xarr, i, d.yres + NPAD + n, load_cell(buf, d.xarr, i, NPAD + n));
}
__global__ void k_bound_x(const DiskView d, Cell* buf) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.yarr) return;
    const int nx = d.xres + NPAD;
    for (int n = 0; n < NPAD; ++n) {
        if (d.bound_lft == 2) {
            Cell c = load_cell(buf, d.xarr, 2 * NPAD - 1 - n, j);
            c.u *= -1.0;
            store_cell(buf, d.xarr, n, j, c);
        } else if (d.bound_lft == 1) {
            store_cell(buf, d.xarr, n, j, load_cell(buf, d.xarr, NPAD, j));
        }
        if (d.bound_rgh == 2) {
            Cell c = load_cell(buf, d.xarr, nx - 1 - n, j);
            c.u *= -1.0;
            store_cell(buf, d.xarr, nx + n, j, c);
        } else if (d.bound_rgh == 1) {
            store_cell(buf, d.xarr, nx + n, j, load_cell(buf, d.xarr, nx - 1, j));
        }
    }
}

// Torque of the planet on the disk (src/output/output.cu:336-412 with g_phi of
// src/output/forces.cu:39-57 at z = 0, 2D polar): one compensated partial sum of
// r g_phi Sigma dV per thread, summed per block, dV = (xa[i+1]^2 - xa[i]^2)/2 (ya[j+1] - ya[j]).
__global__ void k_torque(const DiskView d, const Cell* __restrict__ buf, double* part) {
    const pg_body p = d.sc->planet_next;
    const long long n = (long long)d.xres * d.yres;
    double sum = 0.0, comp = 0.0;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres), j = d.ypad + (int)(m / d.xres);
        const double rad = d.radx[i];
        double sinfac, cosfac;
        sincos(d.ycraw[j] - p.y, &sinfac, &cosfac);
        const double Rp = sqrt(rad * rad + p.x * p.x - 2.0 * p.x * rad * cosfac + p.rs * p.rs);
        const double rs_fac = 1.0 / Rp / Rp / Rp;
        // the planet's pull (output_gy, src/output/forces.cu:103-127): with the indirect
        // term, or as an inertial point mass in the two-body frame (global_sum(.., 1))
        const double gy = d.twobd ? -p.m * p.x * sinfac * rs_fac
                                  : -p.m * p.x * sinfac * rs_fac + p.m * sinfac / p.x / p.x;
        const double dv = 0.5 * (d.xa[i + 1] * d.xa[i + 1] - d.xa[i] * d.xa[i]) * (d.ya[j + 1] - d.ya[j]);
        const double y = rad * gy * (load_cell(buf, d.xarr, i, j).r * dv) - comp;
        const double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    __shared__ double red[256];
    red[threadIdx.x] = sum;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ============================================================== launchers
static inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

cudaError_t set_kernel_attributes() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f, size_t bytes) {
        cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (r != cudaSuccess) e = r;
        r = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (r != cudaSuccess) e = r;
    };
    auto set_v = [&](auto tag) {
        using G = typename decltype(tag)::G;
        if constexpr (G::X_OK) set((const void*)k_sweep<0, G>, G::SMEM);
        set((const void*)k_sweep<1, G>, G::SMEM);
        set((const void*)k_advect<G>, G::AD_SMEM);
    };
    set_v(SV<0>{});
    set_v(SV<1>{});
    set_v(SV<2>{});
    set_v(SV<3>{});
    set_v(SV<4>{});
    set_v(SV<5>{});
    set_v(SV<6>{});
    set_v(SV<7>{});
    set_v(SV<8>{});
    set_v(SV<9>{});
    set((const void*)k_kick1<true>, K1_SMEM);
    set((const void*)k_kick1<false>, K1_SMEM);
    set((const void*)k_kick2<true>, K5_SMEM);
    set((const void*)k_kick2<false>, K5_SMEM);
    return e;
}

void launch_init_tables(const DiskView& d, const pg_params& P, double* tab, cudaStream_t s) {
    TabArgs a{P.sc_h, P.planet_radius, P.p_alpha, P.p_beta, P.ss_alpha, P.frame_omega, P.xmin, P.xmax,
              P.kill_width, P.kill_width_out > 0.0 ? P.kill_width_out : P.kill_width,
              P.visc_flag, P.orbadv_flag, P.kill_flag, P.init_flag, P.geomx};
    // tab layout (doubles), see table_layout() in pg_engine.cu
    double* radx = tab;
    double* cs2x = radx + d.xarr;
    double* nux = cs2x + d.xarr;
    double* initx = nux + d.xarr;
    double* killx = initx + 5 * d.xarr;
    double* xrec = killx + 4 * d.xarr;    // 9 xarr
    double* ycraw = xrec + 9 * d.xarr;
    double* ycj = ycraw + d.yarr;
    double* yrec = ycj + d.yarr;          // 6 yarr
    const int n = d.xarr > d.yarr ? d.xarr : d.yarr;
    k_init_tables<<<cdiv(n, 128), 128, 0, s>>>(d, a, radx, cs2x, nux, initx, killx, const_cast<double*>(d.rot),
                                                ycraw, ycj, xrec, yrec);
}

void launch_torque(const DiskView& d, const Cell* buf, double* part, int nblocks, cudaStream_t s) {
    k_torque<<<nblocks, 256, 0, s>>>(d, buf, part);
}

void launch_init_xghosts(const DiskView& d, Cell* buf, cudaStream_t s) {
    k_init_xghosts<<<cdiv(2 * NPAD * d.yarr, 256), 256, 0, s>>>(d, buf);
}

void launch_bound(const DiskView& d, Cell* buf, cudaStream_t s) {
    if (d.ndim > 1) k_bound_y<<<cdiv(d.xarr * NPAD, 256), 256, 0, s>>>(d, buf);
    if (d.bound_lft != 0 || d.bound_rgh != 0) k_bound_x<<<cdiv(d.yarr, 256), 256, 0, s>>>(d, buf);
}

void launch_cfl(const DiskView& d, const Cell* buf, cudaStream_t s, const pg_dust* dbuf) {
    k_reset_vmax<<<1, 1, 0, s>>>(d.sc);
    const long long n = (long long)d.xres * d.yres;
    unsigned blocks = cdiv(n, 256);
    if (blocks > 148u * 8u) blocks = 148u * 8u;
    k_cfl<<<blocks, 256, 0, s>>>(d, buf, dbuf);
}

void launch_set_time(const DiskView& d, double t, double dt, cudaStream_t s) {
    launch_set_time_only(d, t, dt, s);
    launch_planet_trig(d, s);
}
void launch_set_time_only(const DiskView& d, double t, double dt, cudaStream_t s) {
    k_set_time<<<1, 1, 0, s>>>(d, t, dt);
}
void launch_planet_trig(const DiskView& d, cudaStream_t s) {
    k_planet_trig<<<cdiv(d.yarr, 256), 256, 0, s>>>(d);
}
void launch_run_begin(Scalars* sc, double end_time, bool fresh, cudaStream_t s) {
    k_run_begin<<<1, 1, 0, s>>>(sc, end_time, fresh ? 1 : 0);
}

void launch_time_step(const DiskView& d, cudaStream_t s) {
    k_time_step<<<1, 1, 0, s>>>(d);
    k_planet_trig<<<cdiv(d.yarr, 256), 256, 0, s>>>(d);
}

void launch_init_planet(const DiskView& d, const pg_params& P, double t, cudaStream_t s) {
    const double a = P.planet_radius;
    const double rs = (P.ndim == 2) ? P.rs_fac * P.sc_h * a : P.rs_fac * pow(P.planet_mass / 3.0, 1.0 / 3.0) * a;
    k_init_planet<<<1, 1, 0, s>>>(d, a, P.planet_ecc, rs, t);
}

// Persistent grid: as many CTAs as fit on the GPU at once, each looping over tiles.
static int kernel_occupancy(const void* kernel, int threads, size_t smem);

// Persistent grid: as many CTAs as fit on the GPU at once (at most cps per SM
// when cps > 0), each looping over tiles.
static unsigned persistent_grid(const void* kernel, int threads, size_t smem, long long ntiles, int cps = 0) {
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm <= 0) nsm = 148;
    }
    int per_sm = kernel_occupancy(kernel, threads, smem);
    if (cps > 0 && cps < per_sm) per_sm = cps;
    long long g = (long long)per_sm * nsm;
    if (g > ntiles) g = ntiles;
    return (unsigned)(g < 1 ? 1 : g);
}

static int kernel_occupancy(const void* kernel, int threads, size_t smem) {
    // occupancy of each kernel, queried once (launches repeat every step)
    static const void* keys[64] = {nullptr};
    static int vals[64] = {0};
    int per_sm = 0;
    for (int n = 0; n < 64 && keys[n]; ++n)
        if (keys[n] == kernel) per_sm = vals[n];
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        for (int n = 0; n < 64; ++n)
            if (!keys[n]) {
                keys[n] = kernel;
                vals[n] = per_sm;
                break;
            }
    }
    return per_sm;
}

void launch_kick1(const DiskView& d, const CellMaps& in, Cell* out, double* vis, cudaStream_t s, const pg_dust* din,
                  pg_dust* dout, const Tune* t) {
    const int ntx = (int)cdiv(d.xres, ST_TX), nt = ntx * (int)cdiv(d.yres, ST_TY);
    const int cps = t ? t->cps[0] : 0;
    if (d.visc && d.ndim == 2) {
        const unsigned g = persistent_grid((const void*)k_kick1<true>, ST_THREADS, K1_SMEM, nt, cps);
        k_kick1<true><<<g, ST_THREADS, K1_SMEM, s>>>(in.stencil, d, out, vis, ntx, nt, din, dout);
    } else {
        const unsigned g = persistent_grid((const void*)k_kick1<false>, ST_THREADS, K1_SMEM, nt, cps);
        k_kick1<false><<<g, ST_THREADS, K1_SMEM, s>>>(in.stencil, d, out, vis, ntx, nt, din, dout);
    }
}

template <int DIR, class G>
static void sweep_g(const DiskView& d, const CUtensorMap& m, Cell* out, cudaStream_t s, int cps) {
    if constexpr (DIR == 0 && !G::X_OK) {
        return;  // never chosen: the autotuner skips radial variants whose box does not fit
    } else {
        const int ntx = (int)cdiv(DIR == 0 ? d.xres : d.yres, G::L);
        const int nt = ntx * (int)cdiv(DIR == 0 ? d.yres : d.xres, G::W);
        const unsigned g = persistent_grid((const void*)k_sweep<DIR, G>, G::THREADS, G::SMEM, nt, cps);
        k_sweep<DIR, G><<<g, G::THREADS, G::SMEM, s>>>(m, d, out, ntx, nt);
    }
}

template <class G>
static void advect_g(const DiskView& d, const CUtensorMap& m, Cell* out, cudaStream_t s, int cps) {
    const int ntx = (int)cdiv(d.yres, G::L), nt = ntx * (int)cdiv(d.xres, G::W);
    const unsigned g = persistent_grid((const void*)k_advect<G>, G::THREADS, G::AD_SMEM, nt, cps);
    k_advect<G><<<g, G::THREADS, G::AD_SMEM, s>>>(m, d, out, ntx, nt);
}

// calls f(SV<v>{}) for the variant id v
template <class F>
static void with_variant(int v, F&& f) {
    switch (v) {
        case 1: f(SV<1>{}); break;
        case 2: f(SV<2>{}); break;
        case 3: f(SV<3>{}); break;
        case 4: f(SV<4>{}); break;
        case 5: f(SV<5>{}); break;
        case 6: f(SV<6>{}); break;
        case 7: f(SV<7>{}); break;
        case 8: f(SV<8>{}); break;
        case 9: f(SV<9>{}); break;
        default: f(SV<0>{}); break;
    }
}

static int variant_of(const Tune* t, int k, int dir) {
    const int v = t ? t->v[k] : 0;
    if (v < 0 || v >= NSWEEP_VARIANTS || (dir == 0 && !sweep_variant_x_ok(v))) return 0;
    return v;
}

void launch_sweep_x(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s, const Tune* t) {
    const int v = variant_of(t, 0, 0);
    with_variant(v, [&](auto tag) { sweep_g<0, typename decltype(tag)::G>(d, in.sx[v], out, s, t ? t->cps[1] : 0); });
}

void launch_sweep_y(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s, const Tune* t) {
    const int v = variant_of(t, 1, 1);
    with_variant(v, [&](auto tag) { sweep_g<1, typename decltype(tag)::G>(d, in.sy[v], out, s, t ? t->cps[2] : 0); });
}

void launch_advect(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s, const Tune* t) {
    const int v = variant_of(t, 2, 1);
    with_variant(v, [&](auto tag) { advect_g<typename decltype(tag)::G>(d, in.sy[v], out, s, t ? t->cps[3] : 0); });
}

void launch_kick2(const DiskView& d, const CellMaps& in, const VisMaps& vis, Cell* out, cudaStream_t s,
                  const pg_dust* din, pg_dust* dout, const Tune* t) {
    const int ntx = (int)cdiv(d.xres, ST_TX), nt = ntx * (int)cdiv(d.yres, ST_TY);
    const int cps = t ? t->cps[4] : 0;
    if (d.visc && d.ndim == 2) {
        const unsigned g = persistent_grid((const void*)k_kick2<true>, ST_THREADS, K5_SMEM, nt, cps);
        k_kick2<true><<<g, ST_THREADS, K5_SMEM, s>>>(in.stencil, vis.stencil, d, out, ntx, nt, din, dout);
    } else {
        const unsigned g = persistent_grid((const void*)k_kick2<false>, ST_THREADS, K5_SMEM, nt, cps);
        k_kick2<false><<<g, ST_THREADS, K5_SMEM, s>>>(in.stencil, vis.stencil, d, out, ntx, nt, din, dout);
    }
}

// CTAs per SM that fit for a pass (0 kick1, 1 sweep_x, 2 sweep_y, 3 advect, 4 kick2) with tile variant v
int pass_occupancy(const DiskView& d, int pass, int v) {
    const bool vis = d.visc && d.ndim == 2;
    int occ = 1;
    switch (pass) {
        case 0: return kernel_occupancy(vis ? (const void*)k_kick1<true> : (const void*)k_kick1<false>, ST_THREADS, K1_SMEM);
        case 4: return kernel_occupancy(vis ? (const void*)k_kick2<true> : (const void*)k_kick2<false>, ST_THREADS, K5_SMEM);
        case 1:
            with_variant(v, [&](auto tag) {
                using G = typename decltype(tag)::G;
                if constexpr (G::X_OK) occ = kernel_occupancy((const void*)k_sweep<0, G>, G::THREADS, G::SMEM);
            });
            return occ;
        case 2:
            with_variant(v, [&](auto tag) {
                using G = typename decltype(tag)::G;
                occ = kernel_occupancy((const void*)k_sweep<1, G>, G::THREADS, G::SMEM);
            });
            return occ;
        default:
            with_variant(v, [&](auto tag) {
                using G = typename decltype(tag)::G;
                occ = kernel_occupancy((const void*)k_advect<G>, G::THREADS, G::AD_SMEM);
            });
            return occ;
    }
}

// threads per CTA and the CTAs per SM its registers were compiled for, of a tile variant
void sweep_variant_launch(int v, int* threads, int* minb) {
    with_variant(v, [&](auto tag) {
        using G = typename decltype(tag)::G;
        *threads = G::THREADS;
        *minb = G::MINB;
    });
}

int kernels_per_step(const DiskView& d) {
    int n = 2 /*time, planet trig*/ + 1 /*kick1*/ + 1 /*sweep x*/ + 1 /*kick2*/;
    if (d.ndim > 1) n += 1;
    if (d.ndim > 1 && d.orbadv) n += 1;
    if (d.dust) n += 1 + (d.ndim > 1 ? 1 : 0) + (d.ndim > 1 && d.orbadv ? 1 : 0);  // dust sweeps, advection
    return n;
}

}  // namespace pg

namespace pg {
// test support: the passes' bounded wait (pipe_wait) on a tile whose copy is
// never issued: the stage's barrier expects `bytes` that nothing delivers, so
// every thread gives up after the wait's limit, PG_ERR_TIMEOUT is recorded and
// the CTA leaves together; nothing is in flight when it does.
__global__ void k_test_bounded_wait(Scalars* sc, uint32_t bytes, int* left) {
    __shared__ __align__(8) uint64_t bar[2];
    pipe_init<2>(bar);
    if (threadIdx.x == 0) issue_begin(&bar[0], bytes);
    __syncthreads();
    if (!pipe_wait<2>(bar, 0, sc)) {
        pipe_drain<2>(bar, 0, 0, sc);
        if (threadIdx.x == 0) *left = 1;
        return;
    }
    if (threadIdx.x == 0) *left = 2;  // the copy "landed": not expected
}

// test support: div_1p5 (pg_hydro.cuh) against the IEEE quotient x / 1.5
__global__ void k_test_div_1p5(const double* x, long long n, double* out) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const double a = x[k];
        out[2 * k] = div_1p5(a);
        out[2 * k + 1] = __ddiv_rn(a, 1.5);
    }
}
}  // namespace pg

extern "C" pg_status pg_test_bounded_wait(int* err_bits, int* left, float* ms) {
    if (!err_bits || !left || !ms) return PG_ERR_ARG;
    pg::Scalars* sc = nullptr;
    int* dleft = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&sc, sizeof(pg::Scalars));
    if (e == cudaSuccess) e = cudaMalloc(&dleft, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(sc, 0, sizeof(pg::Scalars));
    if (e == cudaSuccess) e = cudaMemset(dleft, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        cudaEventRecord(e0);
        pg::k_test_bounded_wait<<<1, 64>>>(sc, 4096, dleft);
        e = cudaGetLastError();
        cudaEventRecord(e1);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    pg::Scalars h{};
    if (e == cudaSuccess) e = cudaMemcpy(&h, sc, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(left, dleft, sizeof(int), cudaMemcpyDeviceToHost);
    *err_bits = h.err;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sc);
    cudaFree(dleft);
    return e == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

extern "C" pg_status pg_test_div_1p5(const double* x, long long n, double* out2) {
    if (!x || !out2 || n <= 0) return PG_ERR_ARG;
    double *dx = nullptr, *dout = nullptr;
    if (cudaMalloc(&dx, n * sizeof(double)) != cudaSuccess) return PG_ERR_CUDA;
    if (cudaMalloc(&dout, 2 * n * sizeof(double)) != cudaSuccess) {
        cudaFree(dx);
        return PG_ERR_CUDA;
    }
    cudaError_t e = cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        pg::k_test_div_1p5<<<592, 256>>>(dx, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out2, dout, 2 * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    return e == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}
