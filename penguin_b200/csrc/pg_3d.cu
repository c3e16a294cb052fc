// penguin_b200 3D form (ndim 3) for sm_100a: the reference's DS() with the
// polar sweep (src/solver/solve.cu:212-292 with ndim 3) as five passes over the
// AoS state, on the spherical (r, phi, theta) grid of the reference's 3D preset
// (include/para_files/Adiabatic_CPD.h: geometries 2/4/5) or on a cartesian box:
//
//   kick1   C -> T : first half-kick (src/solver/sweeps.cu:597-711, mdt = 0) with
//                    the spherical gravity and fictitious forces
//                    (src/solver/force/forces.cu:14-39, 110-327); radial ghost images
//   sweep_x T -> C : radial sweep (sweeps.cu:263-335); azimuthal ghost images
//   sweep_y C -> T : azimuthal sweep (sweeps.cu:361-433); polar ghost images
//   sweep_z T -> C : polar sweep (sweeps.cu:458-554)
//   kick2   C -> T : predictor + corrector half-kick, wave damping
//                    (src/killwave/killwave.cu:17-103) and the CFL signal rate
//                    (src/timestep/timestep.cu:18-97, ndim 3)
//
// plus the one-thread clock kernel and the per-row planet angle table of the 2D
// form.  The sweeps are persistent CTAs that stage each tile (32 outputs along
// the sweep plus 3 ghosts a side, 4 pencils) with one 3D TMA box copy, two
// stages in flight, and compute it in three phases (reconstruction and both
// edge states per cell, HLLC per face, update per cell) with the 2D form's
// building blocks (pg_hydro.cuh).  Each pass writes the ghost cells the next
// pass reads (the images the reference's boundx/boundy/boundz copy in place),
// so no boundary pass runs between stages.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "pg_common.cuh"
#include "pg_hydro.cuh"
#include "pg_internal.h"
#include "pg_planet.cuh"

namespace pg {

// ------------------------------------------------------------ tile shape
constexpr int S3_W = 4;                       // pencils per tile
constexpr int S3_L = 32;                      // outputs per pencil
constexpr int S3_TL = S3_L + 2 * NPAD;        // tile cells along the sweep
constexpr int S3_P1 = S3_L + 2;               // cells reconstructed per pencil
constexpr int S3_P2 = S3_L + 1;               // faces per pencil
constexpr int S3_NST = S3_P1 * S3_W;
constexpr int S3_NFX = S3_P2 * S3_W;
constexpr int S3_THREADS = (S3_NST + 31) / 32 * 32;
constexpr int S3_COLS = S3_W + 2;             // y/z tiles start one column early (16-byte TMA x)
constexpr int S3_TILE = (S3_TL * S3_COLS * 5 + 15) / 16 * 16;  // doubles, covers the x tile too
constexpr int S3_NS = 2;
constexpr size_t S3_SMEM = (size_t)(S3_NS * S3_TILE + 10 * S3_NST + 7 * S3_NFX) * 8 + 8 * S3_NS + 128;
constexpr int K3_THREADS = 256;
static_assert(S3_W * S3_TL * 5 <= S3_TILE, "the radial tile fits a stage");
static_assert(5 * S3_TL <= 256 && 5 * S3_COLS <= 256 && S3_TL <= 256, "TMA boxes are at most 256 wide");

// Everything a 3D kernel reads: the 2D view's scalars, grid and tables for x
// and y (and the clock), plus the polar grid and the (x, z) tables.
struct View3 {
    DiskView d;
    int zres, zarr, geomz, bound_bom, bound_top, init3;
    double zmin;
    const double* za;
    const double* zv;
    const double* wz;      // 6 slope weights per polar index
    const double* idx_z;   // 1 / (za[k+1] - za[k])
    const double* zc;      // 0.5 (za[k+1] + za[k])
    const double* sinz;    // sin(zc) (the sweeps' and the CFL's rad_cyl)
    const double* sinpol;  // sincos(zc) (the planet's pull, forces.cu:18-21)
    const double* cospol;
    const double* tanz;    // tan(zc) (get_fz)
    const double* gfx;     // eval_gfac(geomx, xa[i]) (riemann.cu:5-11)
    const double* gfz;     // eval_gfac(geomz, za[k])
    const double* cs2;     // get_cs2(xc(i), zc(k)), xarr * zarr
    const double* initc;   // init_C(xc(i), zc(k)), 5 per (i, k)
};

__device__ __forceinline__ size_t at3(const View3& v, int i, int j, int k) {
    return (size_t)i + (size_t)v.d.xarr * ((size_t)j + (size_t)v.d.yarr * (size_t)k);
}
__device__ __forceinline__ void put3(Cell* out, const View3& v, int i, int j, int k, const Cell& c) {
    double* q = reinterpret_cast<double*>(out + at3(v, i, j, k));
    q[0] = c.r;
    q[1] = c.p;
    q[2] = c.u;
    q[3] = c.v;
    q[4] = c.w;
}
__device__ __forceinline__ Cell get3(const Cell* in, const View3& v, int i, int j, int k) {
    const double* q = reinterpret_cast<const double*>(in + at3(v, i, j, k));
    return Cell{q[0], q[1], q[2], q[3], q[4]};
}

// Ghost images.  Radial (kick1 output, read by the radial sweep; boundary.cu:13-62):
// bound 1 copies the edge cell, 2 mirrors it with u negated; bound-0 ghosts hold
// init_C and are never rewritten.
__device__ __forceinline__ void emit_x(const View3& v, Cell* out, int i, int j, int k, const Cell& c) {
    const DiskView& d = v.d;
    put3(out, v, i, j, k, c);
    const int nx = d.xres + NPAD;
    if (d.bound_lft == 1 && i == NPAD) {
        for (int n = 0; n < NPAD; ++n) put3(out, v, n, j, k, c);
    } else if (d.bound_lft == 2 && i < 2 * NPAD) {
        Cell m = c;
        m.u = -m.u;
        put3(out, v, 2 * NPAD - 1 - i, j, k, m);
    }
    if (d.bound_rgh == 1 && i == nx - 1) {
        for (int n = 0; n < NPAD; ++n) put3(out, v, nx + n, j, k, c);
    } else if (d.bound_rgh == 2 && i >= nx - NPAD) {
        Cell m = c;
        m.u = -m.u;
        put3(out, v, 2 * nx - 1 - i, j, k, m);
    }
}
// Azimuthal (radial sweep output, read by the azimuthal sweep): periodic
// (boundary.cu:140-209 with bound_bak / bound_frn 3).
__device__ __forceinline__ void emit_y(const View3& v, Cell* out, int i, int j, int k, const Cell& c) {
    put3(out, v, i, j, k, c);
    if (j < 2 * NPAD) put3(out, v, i, j + v.d.yres, k, c);
    else if (j >= v.d.yres) put3(out, v, i, j - v.d.yres, k, c);
}
// Polar (azimuthal sweep output, read by the polar sweep; boundary.cu:270-320):
// 1 zero gradient, 2 reflecting (w negated), 3 periodic; 0 holds init_C.
__device__ __forceinline__ void emit_z(const View3& v, Cell* out, int i, int j, int k, const Cell& c) {
    put3(out, v, i, j, k, c);
    const int nz = v.zres + NPAD;
    if (v.bound_bom == 2 && k < 2 * NPAD) {
        Cell m = c;
        m.w = -m.w;
        put3(out, v, i, j, 2 * NPAD - 1 - k, m);
    } else if (v.bound_bom == 1 && k == NPAD) {
        for (int n = 0; n < NPAD; ++n) put3(out, v, i, j, n, c);
    } else if (v.bound_bom == 3 && k >= v.zres) {
        put3(out, v, i, j, k - v.zres, c);
    }
    if (v.bound_top == 2 && k >= nz - NPAD) {
        Cell m = c;
        m.w = -m.w;
        put3(out, v, i, j, 2 * nz - 1 - k, m);
    } else if (v.bound_top == 1 && k == nz - 1) {
        for (int n = 0; n < NPAD; ++n) put3(out, v, i, j, nz + n, c);
    } else if (v.bound_top == 3 && k < 2 * NPAD) {
        put3(out, v, i, j, k + v.zres, c);
    }
}

// ================================================================ sweeps
// DIR 0 radial pencils (tile rows j, one plane k), DIR 1 azimuthal pencils
// (columns i, one plane k), DIR 2 polar pencils (columns i, one row j).
// Tile t: a = t % nta along the sweep, b = (t / nta) % ntb across the pencils,
// c = t / (nta ntb) the plane (DIR 0, 1) or row (DIR 2).
// 4 CTAs per SM (96 registers; the radial instance spills 12 bytes): 20 warps
// instead of the 15 its natural 106-110 registers allow, 8-11 % faster
template <int DIR>
__global__ void __launch_bounds__(S3_THREADS, 4)
    k3_sweep(const __grid_constant__ CUtensorMap tm, const View3 v, Cell* __restrict__ out, int nta, int ntb,
             int ntiles) {
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    double* st = smem + S3_NS * S3_TILE;  // [10][S3_NST] edge states
    double* fl = st + 10 * S3_NST;        // [7][S3_NFX] fluxes
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 7 * S3_NFX);
    const DiskView& d = v.d;
    Scalars* sc = d.sc;
    if (sc->done) return;

    const int tid = threadIdx.x;
    const double dt = sc->dt;
    const double gam = d.gam;
    const int res = DIR == 0 ? d.xres : (DIR == 1 ? d.yres : v.zres);  // cells along the sweep
    const int qres = DIR == 0 ? d.yres : d.xres;                         // pencils
    const int arr = DIR == 0 ? d.xarr : (DIR == 1 ? d.yarr : v.zarr);
    constexpr uint32_t BYTES = (DIR == 0 ? S3_W * S3_TL * 5 : S3_COLS * S3_TL * 5) * 8;
    auto origin = [&](int tile, int& s0, int& q0, int& c) {
        const int r = tile / nta;
        s0 = NPAD + S3_L * (tile % nta);  // first output along the sweep
        q0 = NPAD + S3_W * (r % ntb);     // first pencil
        c = NPAD + r / ntb;               // plane k (DIR 0, 1) or row j (DIR 2)
    };
    auto issue = [&](int tile, int k) {
        int s0, q0, c;
        origin(tile, s0, q0, c);
        double* dst = smem + (k % S3_NS) * S3_TILE;
        issue_begin(&bar[k % S3_NS], BYTES);
        if (DIR == 0) tma_load_3d(dst, &tm, 5 * (s0 - NPAD), q0, c, &bar[k % S3_NS]);
        else if (DIR == 1) tma_load_3d(dst, &tm, 5 * (q0 - 1), s0 - NPAD, c, &bar[k % S3_NS]);
        else tma_load_3d(dst, &tm, 5 * (q0 - 1), c, s0 - NPAD, &bar[k % S3_NS]);
    };
    pipe_init<S3_NS>(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++kt) {
        const int ahead = (tile + (int)gridDim.x < ntiles) ? 1 : 0;
        if (tid == 0 && ahead) issue(tile + gridDim.x, kt + 1);
        int s0, q0, c;
        origin(tile, s0, q0, c);
        const double* tl = smem + (kt % S3_NS) * S3_TILE;
        if (!pipe_wait<S3_NS>(bar, kt, sc)) {
            pipe_drain<S3_NS>(bar, kt, ahead, sc);
            return;
        }

        // ---- P1: reconstruction and both edge states of every cell
        for (int it = tid; it < S3_NST; it += S3_THREADS) {
            const int q = DIR == 0 ? it / S3_P1 : it % S3_W;
            const int t = 2 + (DIR == 0 ? it % S3_P1 : it / S3_W);
            const int s = s0 - NPAD + t;
            const int qq = min(q0 + q, d.xarr - 1);
            // geometry of the pencil: DIR 1 rad_cyl (sweeps.cu:380-386), DIR 2 rad (:486-489)
            double radp = 1.0;
            if (DIR == 1 && d.geomy == 4) radp = d.radx[qq] * v.sinz[c];
            if (DIR == 2 && v.geomz == 5) radp = d.radx[qq];
            double r[5], p[5], u[5], vv[5], w[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const double* cp = DIR == 0 ? tl + (q * S3_TL + (t - 2 + m)) * 5 : tl + ((t - 2 + m) * S3_COLS + q + 1) * 5;
                const int sm = min(max(s - 2 + m, 0), arr - 1);
                r[m] = cp[0];
                p[m] = cp[1];
                if (DIR == 0) {  // angular momenta r sin(theta) v_phi and r v_theta (sweeps.cu:283-300)
                    u[m] = cp[2];
                    vv[m] = cp[3];
                    w[m] = cp[4];
                    if (d.geomx == 2) {
                        const double rad = d.radx[sm];
                        vv[m] *= rad * v.sinz[c];
                        w[m] *= rad;
                    } else if (d.geomx == 1) {
                        vv[m] *= d.radx[sm];
                    }
                } else if (DIR == 1) {  // residual of the frame rotation (sweeps.cu:388-396)
                    u[m] = cp[3];
                    if (d.geomy == 4) u[m] -= radp * d.frame_omega;
                    vv[m] = cp[4];
                    w[m] = cp[2];
                } else {  // r sin(theta) v_phi of each cell of the pencil (sweeps.cu:491-500)
                    u[m] = cp[4];
                    vv[m] = cp[2];
                    w[m] = cp[3];
                    if (v.geomz == 5) w[m] *= radp * v.sinz[sm];
                }
            }
            const double cs0 = sqrt(gam * p[2] / r[2]);
            const double flat = flatten(1.0 / cs0, p[2], p[0], p[1], p[3], p[4], u[1], u[2], u[3]);
            const int sc_ = min(s, arr - 1);
            const double* wt = (DIR == 0 ? d.wx : (DIR == 1 ? d.wy : v.wz)) + 6 * sc_;
            const double idx = (DIR == 0 ? d.idx_x : (DIR == 1 ? d.idx_y : v.idx_z))[sc_];
            const double* fa = DIR == 0 ? d.xa : (DIR == 1 ? d.ya : v.za);
            const Par R = recon(wt, r[0], r[1], r[2], r[3], r[4], flat);
            const Par P = recon(wt, p[0], p[1], p[2], p[3], p[4], flat);
            const Par U = recon(wt, u[0], u[1], u[2], u[3], u[4], flat);
            const Par V = recon(wt, vv[0], vv[1], vv[2], vv[3], vv[4], flat);
            const Par W = recon(wt, w[0], w[1], w[2], w[3], w[4], flat);
            const double xl = fa[sc_], xr = fa[sc_ + 1];
            const double sdt = DIR == 0 ? dt : dt / radp;  // set_state receives dt/rad (riemann.cu:111)
            const Half a = state_at_left_edge(gam, xl, idx, sdt, cs0, r[2], p[2], u[2], R, P, U, V, W);
            const Half b = state_at_right_edge(gam, xl, xr, idx, sdt, cs0, r[2], p[2], u[2], R, P, U, V, W);
            st[0 * S3_NST + it] = a.r;
            st[1 * S3_NST + it] = a.p;
            st[2 * S3_NST + it] = a.u;
            st[3 * S3_NST + it] = a.v;
            st[4 * S3_NST + it] = a.w;
            st[5 * S3_NST + it] = b.r;
            st[6 * S3_NST + it] = b.p;
            st[7 * S3_NST + it] = b.u;
            st[8 * S3_NST + it] = b.v;
            st[9 * S3_NST + it] = b.w;
        }
        __syncthreads();

        // ---- P2: HLLC flux at every face (left state from cell t-1, right from cell t)
        for (int it = tid; it < S3_NFX; it += S3_THREADS) {
            const int q = DIR == 0 ? it / S3_P2 : it % S3_W;
            const int t = 3 + (DIR == 0 ? it % S3_P2 : it / S3_W);
            const int iL = DIR == 0 ? q * S3_P1 + (t - 3) : (t - 3) * S3_W + q;
            const int iR = DIR == 0 ? q * S3_P1 + (t - 2) : (t - 2) * S3_W + q;
            Half L, R;
            L.r = st[5 * S3_NST + iL];
            L.p = st[6 * S3_NST + iL];
            L.u = st[7 * S3_NST + iL];
            L.v = st[8 * S3_NST + iL];
            L.w = st[9 * S3_NST + iL];
            R.r = st[0 * S3_NST + iR];
            R.p = st[1 * S3_NST + iR];
            R.u = st[2 * S3_NST + iR];
            R.v = st[3 * S3_NST + iR];
            R.w = st[4 * S3_NST + iR];
            const Flux F = hllc(d.eos, d.ie, gam, L, R);
            fl[0 * S3_NFX + it] = F.r;
            fl[1 * S3_NFX + it] = F.p;
            fl[2 * S3_NFX + it] = F.u;
            fl[3 * S3_NFX + it] = F.v;
            fl[4 * S3_NFX + it] = F.w;
            fl[5 * S3_NFX + it] = F.pres;
            fl[6 * S3_NFX + it] = F.uprs;
        }
        __syncthreads();

        // ---- P3: flux differences, pressure sources, geometry, conservative update
        for (int it = tid; it < S3_L * S3_W; it += S3_THREADS) {
            const int q = DIR == 0 ? it / S3_L : it % S3_W;
            const int t = 3 + (DIR == 0 ? it % S3_L : it / S3_W);
            const int s = s0 - NPAD + t;
            const int qq = q0 + q;
            if (s >= NPAD + res || qq >= NPAD + qres) continue;
            const int f0 = DIR == 0 ? q * S3_P2 + (t - 3) : (t - 3) * S3_W + q;
            const int f1 = DIR == 0 ? f0 + 1 : f0 + S3_W;
            // net_source (src/solver/riemann/riemann.cu:40-87) with the face areas; the
            // reference stores each flux times its area in shared memory before
            // differencing, so the products are rounded on their own (__dmul_rn: no FMA)
            const double g0 = DIR == 0 ? v.gfx[s] : (DIR == 1 ? 1.0 : v.gfz[s]);
            const double g1 = DIR == 0 ? v.gfx[s + 1] : (DIR == 1 ? 1.0 : v.gfz[s + 1]);
            const double pres0 = fl[5 * S3_NFX + f0], pres1 = fl[5 * S3_NFX + f1];
            const double du = 0.5 * (g0 + g1) * (pres0 - pres1);
            auto net = [&](int k) { return __dmul_rn(fl[k * S3_NFX + f0], g0) - __dmul_rn(fl[k * S3_NFX + f1], g1); };
            double de = 0.0;
            if (d.eos == 2) de = (d.ie == 0) ? net(6) : 0.5 * (pres0 + pres1) * net(6);
            Cell D;
            D.r = net(0);
            D.p = net(1) + de;
            D.u = net(2) + du;
            D.v = net(3);
            D.w = net(4);
            const double* cp = DIR == 0 ? tl + (q * S3_TL + t) * 5 : tl + (t * S3_COLS + q + 1) * 5;
            const Cell C0{cp[0], cp[1], cp[2], cp[3], cp[4]};
            if (DIR == 0) {  // sweeps.cu:306-332
                const double f = dt / d.xv[s];
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (d.geomx == 2) {
                    const double rad = d.radx[s];
                    D.v /= rad * v.sinz[c];
                    D.w /= rad;
                } else if (d.geomx == 1) {
                    D.v /= d.radx[s];
                }
                const Cell Q = update_cell(d.eos, d.ie, gam, v.cs2[s + d.xarr * c], C0, D, &sc->floor_hits);
                if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                emit_y(v, out, s, qq, c, Q);
            } else if (DIR == 1) {  // sweeps.cu:403-425 (orb_rot 0)
                const double radp = d.geomy == 4 ? d.radx[qq] * v.sinz[c] : 1.0;
                const double f = dt / d.yv[s] / radp;
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (d.geomy == 4) D.u += (0.0 + radp * d.frame_omega) * D.r;
                else D.u += 0.0 * D.r;
                const Cell E{D.r, D.p, D.w, D.u, D.v};
                const Cell Q = update_cell(d.eos, d.ie, gam, v.cs2[qq + d.xarr * c], C0, E, &sc->floor_hits);
                if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                emit_z(v, out, qq, s, c, Q);
            } else {  // sweeps.cu:507-532
                const double f = dt / v.zv[s];
                D.r *= f; D.p *= f; D.u *= f; D.v *= f; D.w *= f;
                if (v.geomz == 5) {
                    const double rad = d.radx[qq];
                    const double g = 1.0 / rad;
                    D.r *= g; D.p *= g; D.u *= g; D.v *= g; D.w *= g;
                    D.w /= rad * v.sinz[s];
                }
                const Cell E{D.r, D.p, D.v, D.w, D.u};
                const Cell Q = update_cell(d.eos, d.ie, gam, v.cs2[qq + d.xarr * s], C0, E, &sc->floor_hits);
                if (!(Q.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                put3(out, v, qq, c, s, Q);
            }
        }
        __syncthreads();  // the stage and the state / flux arrays are free again
    }
}

// ================================================================= kicks
// Gravity of the star and the planet and the fictitious forces in spherical
// coordinates (get_gx/gy/gz, star_planet_grav and get_fx/fy/fz of
// src/solver/force/forces.cu:14-39, 110-327, twobd_flag 0; cartesian: none).
struct Grav3 {
    double gx, gy, gz;
};
__device__ __forceinline__ Grav3 gravity3(const View3& v, int j, int k, double rad, double pol, const pg_body& pl,
                                          int which) {
    const DiskView& d = v.d;
    Grav3 g{0.0, 0.0, 0.0};
    if (d.geomx != 2) return g;
    g.gx = -1.0 / rad / rad;
    if (d.nplanet > 0) {
        const double sinfac = d.trig[4 * j + 2 * which], cosfac = d.trig[4 * j + 2 * which + 1];
        const double sinpol = v.sinpol[k], cospol = v.cospol[k];
        const double plm = pl.m, plx = pl.x;
        const double Rp = sqrt(rad * rad + plx * plx - 2.0 * plx * rad * cosfac * sinpol);
        const double rs_fac = fmax(4.0 - 3.0 * Rp / pl.rs, 1.0) / fmax(pl.rs * pl.rs * pl.rs, Rp * Rp * Rp);
        const double fx = -plm * (rad - plx * cosfac * sinpol) * rs_fac - plm * sinpol * cosfac / plx / plx;
        const double fy = -plm * plx * sinfac * rs_fac + plm * sinpol * sinfac / plx / plx;
        const double fz = plm * plx * cosfac * cospol * rs_fac - plm * cospol * cosfac / (sinpol * plx * plx);
        g.gx += fx;
        g.gy += fy;
        g.gz += fz;
    }
    if (pol < v.zmin) g.gz *= -1.0;
    return g;
}
__device__ __forceinline__ void fict3(const View3& v, int k, double rad, double pol, const Cell& T, double& fx,
                                      double& fy, double& fz) {
    fx = 0.0;
    fy = 0.0;
    fz = 0.0;
    if (v.d.geomx == 2) {
        fx = T.v * T.v / rad + T.w * T.w / rad;
        fz = T.v * T.v / rad / v.tanz[k];
        if (pol < v.zmin) fz *= -1.0;
    }
}

// CFL signal rate of one cell (src/timestep/timestep.cu:46-88, ndim 3, orb_rot 0).
__device__ __forceinline__ double rate3(const View3& v, const Cell& c, int i, int j, int k) {
    const DiskView& d = v.d;
    double rad = 1.0, rad_cyl = 1.0;
    if (d.geomy == 4) {
        rad = d.radx[i];
        rad_cyl = rad * v.sinz[k];
    }
    const double cs = sqrt(d.gam * c.p / c.r);
    double spd = fabs(c.u) + cs;
    double tmp = fmax(spd / fabs(d.xa[i + 1] - d.xa[i]), 0.0);
    spd = fabs(c.v - rad_cyl * d.frame_omega - 0.0) + cs;
    tmp = fmax(spd / (fabs(d.ya[j + 1] - d.ya[j]) * rad_cyl), tmp);
    spd = fabs(c.w) + cs;
    tmp = fmax(spd / (fabs(v.za[k + 1] - v.za[k]) * rad), tmp);
    return tmp;
}

// PASS 1: first half-kick with the bodies of the previous step; PASS 2: the
// predictor / corrector half-kick with the bodies at t + dt, then wave damping
// and the signal rate of the result.  One thread per interior cell.
// 4 CTAs of 256 threads per SM (64 registers; kick2 spills ~40 bytes): the
// passes wait on loads, and 32 warps hide them better than 16-24 (20-23 % faster)
template <int PASS>
__global__ void __launch_bounds__(K3_THREADS, 4) k3_kick(const View3 v, const Cell* __restrict__ in, Cell* __restrict__ out) {
    const DiskView& d = v.d;
    Scalars* sc = d.sc;
    if (sc->done) return;
    const double dt = sc->dt, hdt = 0.5 * dt;
    const pg_body pl = PASS == 1 ? sc->planet_cur : sc->planet_next;
    const long long n = (long long)d.xres * d.yres * v.zres;
    double vmax = 0.0;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres);
        const long long rest = m / d.xres;
        const int j = NPAD + (int)(rest % d.yres);
        const int k = NPAD + (int)(rest / d.yres);
        const Cell C = get3(in, v, i, j, k);
        const double rad = d.radx[i], pol = v.zc[k];
        const Grav3 g = gravity3(v, j, k, rad, pol, pl, PASS - 1);
        double fx, fy, fz;
        fict3(v, k, rad, pol, C, fx, fy, fz);
        if (PASS == 2) {  // the predictor over mdt = dt/2 (sweeps.cu:658-675)
            Cell T = C;
            T.u = C.u + fx * hdt + g.gx * hdt;
            T.v = C.v + fy * hdt + g.gy * hdt;
            T.w = C.w + fz * hdt + g.gz * hdt;
            fict3(v, k, rad, pol, T, fx, fy, fz);
        }
        Cell Q;
        Q.u = C.u + fx * hdt + g.gx * hdt;
        Q.v = C.v + fy * hdt + g.gy * hdt;
        Q.w = C.w + fz * hdt + g.gz * hdt;
        Q.r = C.r;
        Q.p = C.p;
        if (PASS == 1) {
            emit_x(v, out, i, j, k, Q);
            continue;
        }
        if (d.kill) {  // relax towards init_C (killwave.cu:48-100)
            const double* kt = d.killx + 4 * i;
            const double* I = v.initc + 5 * ((size_t)i + (size_t)d.xarr * k);
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const double tau = kt[2 * side + 1];
                if (tau > 0.0) {
                    double f = kt[2 * side];
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
        put3(out, v, i, j, k, Q);
        vmax = fmax(vmax, rate3(v, Q, i, j, k));
    }
    if (PASS == 2) block_max_to<K3_THREADS>(&sc->vmax_bits, vmax);
}

__global__ void __launch_bounds__(K3_THREADS) k3_cfl(const View3 v, const Cell* __restrict__ in) {
    const DiskView& d = v.d;
    const long long n = (long long)d.xres * d.yres * v.zres;
    double vmax = 0.0;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres);
        const long long rest = m / d.xres;
        const int j = NPAD + (int)(rest % d.yres);
        const int k = NPAD + (int)(rest / d.yres);
        vmax = fmax(vmax, rate3(v, get3(in, v, i, j, k), i, j, k));
    }
    block_max_to<K3_THREADS>(&d.sc->vmax_bits, vmax);
}

// ======================================================== state transfer
// Both buffers: interior from the planes (x fastest, then y, then z), every
// ghost cell init_C (fill_grid, src/init/init.cu:502-519, as the device
// evaluates it for the bound-0 ghosts of boundary.cu:30-33, 276-318).
__global__ void k3_fill(const View3 v, Cell* a, Cell* b, const double* r, const double* p, const double* u,
                        const double* vv, const double* w) {
    const DiskView& d = v.d;
    const long long n = (long long)d.xarr * d.yarr * v.zarr;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(m % d.xarr);
        const long long rest = m / d.xarr;
        const int j = (int)(rest % d.yarr);
        const int k = (int)(rest / d.yarr);
        Cell c;
        if (i >= NPAD && i < NPAD + d.xres && j >= NPAD && j < NPAD + d.yres && k >= NPAD && k < NPAD + v.zres) {
            const size_t q = (size_t)(i - NPAD) + (size_t)d.xres * ((size_t)(j - NPAD) + (size_t)d.yres * (k - NPAD));
            c = Cell{r[q], p[q], u[q], vv[q], w[q]};
        } else {
            const double* I = v.initc + 5 * ((size_t)i + (size_t)d.xarr * k);
            c = Cell{I[0], I[1], I[2], I[3], I[4]};
        }
        put3(a, v, i, j, k, c);
        put3(b, v, i, j, k, c);
    }
}

__global__ void k3_extract(const View3 v, const Cell* in, double* r, double* p, double* u, double* vv, double* w) {
    const DiskView& d = v.d;
    const long long n = (long long)d.xres * d.yres * v.zres;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres);
        const long long rest = m / d.xres;
        const int j = NPAD + (int)(rest % d.yres);
        const int k = NPAD + (int)(rest / d.yres);
        const Cell c = get3(in, v, i, j, k);
        r[m] = c.r;
        p[m] = c.p;
        u[m] = c.u;
        vv[m] = c.v;
        w[m] = c.w;
    }
}

// The bound-0 radial and polar ghosts of a caller's buffer: init_C as the device
// evaluates it (boundary.cu:30-33, 56-59, 293-294, 315-316); never rewritten.
__global__ void k3_analytic_ghosts(const View3 v, Cell* buf) {
    const DiskView& d = v.d;
    const long long n = (long long)d.xarr * d.yarr * v.zarr;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(m % d.xarr);
        const long long rest = m / d.xarr;
        const int j = (int)(rest % d.yarr);
        const int k = (int)(rest / d.yarr);
        const bool gx = (i < NPAD && d.bound_lft == 0) || (i >= NPAD + d.xres && d.bound_rgh == 0);
        const bool gz = (k < NPAD && v.bound_bom == 0) || (k >= NPAD + v.zres && v.bound_top == 0);
        if (!gx && !gz) continue;
        const double* I = v.initc + 5 * ((size_t)i + (size_t)d.xarr * k);
        put3(buf, v, i, j, k, Cell{I[0], I[1], I[2], I[3], I[4]});
    }
}

// ================================================================ tables
// Evaluated on the device with its own sin / cos / tan / pow / exp / sqrt, as
// the reference evaluates them in its kernels.
struct Tab3Args {
    double sc_h, planet_radius, p_alpha, p_beta, xmin, xmax, kill_width, kill_width_out;
    int geomx, init_flag, kill;
};
__device__ inline double t3_cs2(const Tab3Args& a, double x, double z) {  // init.cu:7-17
    const double coeff = a.sc_h * a.sc_h * (1.0 / a.planet_radius);
    if (a.geomx == 0) return coeff;
    return coeff * pow(x * sin(z) / a.planet_radius, -a.p_beta);
}
__device__ inline double t3_h(const Tab3Args& a, double x, double z) {  // init.cu:20-29
    if (a.geomx == 0) return a.sc_h;
    return sqrt(t3_cs2(a, x, z) * pow(x * sin(z), 3));
}
__device__ inline double t3_rho(const Tab3Args& a, double x, double z) {  // init.cu:53-71, 90-91 (init_flag 3)
    const double cs2 = t3_cs2(a, x, z);
    const double r = x * sin(z);
    return pow(x * sin(z) / a.planet_radius, -a.p_alpha) * exp((1.0 / x - 1.0 / r) / cs2);
}
__device__ inline double t3_p(const Tab3Args& a, double x, double z) { return t3_cs2(a, x, z) * t3_rho(a, x, z); }

__global__ void k3_tables(const View3 v, Tab3Args a, double* zc, double* sinz, double* sinpol, double* cospol,
                          double* tanz, double* idx_z, double* gfx, double* gfz, double* radx, double* idx_x,
                          double* killx, double* ycj, double* idx_y, double* cs2, double* initc) {
    const DiskView& d = v.d;
    const long long nxz = (long long)d.xarr * v.zarr;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid <= v.zarr) gfz[tid] = (v.geomz == 5) ? sin(v.za[tid]) : 1.0;
    if (tid <= d.xarr) {
        const double x = d.xa[tid];
        gfx[tid] = (d.geomx == 2) ? x * x : (d.geomx == 1 ? x : 1.0);
    }
    if (tid < v.zarr) {
        const int k = (int)tid;
        const double z = 0.5 * (v.za[k + 1] + v.za[k]);
        zc[k] = z;
        sinz[k] = sin(z);
        sincos(z, &sinpol[k], &cospol[k]);
        tanz[k] = tan(z);
        idx_z[k] = 1.0 / (v.za[k + 1] - v.za[k]);
    }
    if (tid < d.yarr) {
        const int j = (int)tid;
        ycj[j] = 0.5 * (d.ya[j + 1] + d.ya[j]);
        idx_y[j] = 1.0 / (d.ya[j + 1] - d.ya[j]);
    }
    if (tid < d.xarr) {
        const int i = (int)tid;
        const double x = 0.5 * (d.xa[i + 1] + d.xa[i]);
        radx[i] = x;
        idx_x[i] = 1.0 / (d.xa[i + 1] - d.xa[i]);
        // killwave.cu:24-34 with the ndim-3 scale height at the midplane
        const double d_in = t3_h(a, a.xmin, HPI) * a.kill_width;
        const double d_out = t3_h(a, a.xmax, HPI) * a.kill_width_out;
        const double inner = a.xmin + d_in, outer = a.xmax - d_out;
        double* kt = killx + 4 * i;
        kt[0] = kt[1] = kt[2] = kt[3] = 0.0;
        if (a.kill && i >= NPAD && i < NPAD + d.xres) {
            if (x < inner) {
                kt[1] = (a.geomx == 0) ? 1.0 : pow(x, 1.5);
                double f = __sinf(HPI * ((inner - x) / d_in));  // get_ramping_fac (killwave.cu:8-14)
                kt[0] = f * f;
            }
            if (x > outer) {
                kt[3] = (a.geomx == 0) ? 1.0 : pow(x, 1.5);
                double f = __sinf(HPI * ((x - outer) / d_out));
                kt[2] = f * f;
            }
        }
    }
    if (tid < nxz) {
        const int i = (int)(tid % d.xarr), k = (int)(tid / d.xarr);
        const double x = 0.5 * (d.xa[i + 1] + d.xa[i]);
        const double z = 0.5 * (v.za[k + 1] + v.za[k]);
        cs2[tid] = t3_cs2(a, x, z);
        double* q = initc + 5 * tid;
        if (a.init_flag == 3) {  // init_C of init_flag 3 (init.cu:90-91, 157-158, 196-198, 269-274, 322-323)
            const double r = x * sin(z);
            q[0] = t3_rho(a, x, z);
            q[1] = t3_p(a, x, z);
            q[2] = -1.5 * 0.0 / r;
            const double rho = t3_rho(a, x, z);
            const double dr = 1.1514178e-7;
            const double dP_dr = (t3_p(a, x + dr, z) - t3_p(a, x - dr, z)) / (2.0 * dr);
            q[3] = sqrt(1.0 / x + (x / rho) * dP_dr);
            q[4] = 0.0;
        } else {
            q[0] = 1.0;
            q[1] = 1.0;
            q[2] = q[3] = q[4] = 0.0;
        }
    }
}

// ================================================================ engine
struct Engine3 {
    pg_params P{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    View3 v{};
    Cell* buf[2] = {nullptr, nullptr};
    bool own_buffers = true;  // false: the caller's Grid buffers (pg_grid_*)
    CUtensorMap maps[2][3];  // per buffer: radial, azimuthal, polar boxes
    const void* map_base[2] = {nullptr, nullptr};
    std::vector<const void*> ghosted;  // caller buffers whose bound-0 ghosts hold the device init_C
    std::vector<double> hxa, hya, hza; // host faces of each axis (ghosts included), for snapshots
    double* tables = nullptr;
    double* stage = nullptr;
    size_t stage_n = 0;
    Scalars* sc = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int cur = 0;
    int cur_base = 0;
    long long steps_base = 0;
    bool pending = false;
    bool fresh = true;
    unsigned grid_sweep[3] = {0, 0, 0};
    unsigned grid_kick = 0;
    int nta[3], ntb[3], ntiles[3];
};

static pg_status fail3(pg_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return s;
}

#define PG3_CUDA(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return fail3(PG_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)

static pg_status check3(const pg_params* P) {
    if (!P) return fail3(PG_ERR_ARG, "null params");
    if (P->ndim != 3) return fail3(PG_ERR_CONFIG, "the 3D form needs ndim 3");
    const bool sph = P->geomx == 2 && P->geomy == 4 && P->geomz == 5;
    const bool cart = P->geomx == 0 && P->geomy == 0 && P->geomz == 0;
    if (!sph && !cart) return fail3(PG_ERR_CONFIG, "3D geometries: spherical (2, 4, 5) or cartesian (0, 0, 0)");
    if (P->xres < 2 * NPAD || P->yres < 2 * NPAD || P->zres < 2 * NPAD || P->xres % 2)
        return fail3(PG_ERR_CONFIG, "3D resolutions: at least 6 cells per axis, even xres");
    if (P->gridx < 0 || P->gridx > 4 || P->gridy < 0 || P->gridy > 4 || P->gridz < 0 || P->gridz > 4)
        return fail3(PG_ERR_CONFIG, "grids must be 0 to 4");
    if (P->eos_flag != 0 && P->eos_flag != 2) return fail3(PG_ERR_CONFIG, "EOS_flag must be 0 or 2");
    if (P->bound_lft < 0 || P->bound_lft > 2 || P->bound_rgh < 0 || P->bound_rgh > 2)
        return fail3(PG_ERR_CONFIG, "radial boundaries must be 0, 1 or 2");
    if (P->bound_bom < 0 || P->bound_bom > 3 || P->bound_top < 0 || P->bound_top > 3)
        return fail3(PG_ERR_CONFIG, "polar boundaries must be 0 to 3");
    if (P->visc_flag || P->orbadv_flag || P->dust_flag || P->cool_flag || P->twobd_flag)
        return fail3(PG_ERR_CONFIG, "3D runs without viscosity, orbital advection, dust, cooling and two-body frame");
    if (P->n_planet < 0 || P->n_planet > 1) return fail3(PG_ERR_CONFIG, "n_planet must be 0 or 1");
    const bool analytic = P->kill_flag || P->bound_lft == 0 || P->bound_rgh == 0 || P->bound_bom == 0 ||
                          P->bound_top == 0;
    if (analytic && (!sph || P->init_flag != 3))
        return fail3(PG_ERR_CONFIG, "analytic ghosts or wave damping need the spherical disk (init_flag 3)");
    return PG_OK;
}

static unsigned occupancy_grid(const void* kernel, int threads, size_t smem, long long work) {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
    long long g = (long long)nsm * (per > 0 ? per : 1);
    if (g > work) g = work;
    return (unsigned)(g > 0 ? g : 1);
}

static pg_status make_maps(Engine3& E, int b) {
    const DiskView& d = E.v.d;
    const uint64_t d0 = 5ull * d.xarr, d1 = d.yarr, d2 = E.v.zarr;
    pg_status s;
    if ((s = make_map3_f64(&E.maps[b][0], E.buf[b], d0, d1, d2, 5 * S3_TL, S3_W, 1)) != PG_OK) return s;
    if ((s = make_map3_f64(&E.maps[b][1], E.buf[b], d0, d1, d2, 5 * S3_COLS, S3_TL, 1)) != PG_OK) return s;
    if ((s = make_map3_f64(&E.maps[b][2], E.buf[b], d0, d1, d2, 5 * S3_COLS, 1, S3_TL)) != PG_OK) return s;
    E.map_base[b] = E.buf[b];
    return PG_OK;
}

// the five passes of one step from buffer c (newest state ends in 1 - c)
static void enqueue_passes(Engine3& E, int c) {
    const View3& v = E.v;
    cudaStream_t s = E.stream;
    Cell* A = E.buf[c];
    Cell* B = E.buf[1 - c];
    k3_kick<1><<<E.grid_kick, K3_THREADS, 0, s>>>(v, A, B);
    k3_sweep<0><<<E.grid_sweep[0], S3_THREADS, S3_SMEM, s>>>(E.maps[1 - c][0], v, A, E.nta[0], E.ntb[0], E.ntiles[0]);
    k3_sweep<1><<<E.grid_sweep[1], S3_THREADS, S3_SMEM, s>>>(E.maps[c][1], v, B, E.nta[1], E.ntb[1], E.ntiles[1]);
    k3_sweep<2><<<E.grid_sweep[2], S3_THREADS, S3_SMEM, s>>>(E.maps[1 - c][2], v, A, E.nta[2], E.ntb[2], E.ntiles[2]);
    k3_kick<2><<<E.grid_kick, K3_THREADS, 0, s>>>(v, A, B);
}

static pg_status resolve3(Engine3& E) {
    if (!E.pending) return PG_OK;
    long long steps = 0;
    PG3_CUDA(cudaMemcpyAsync(&steps, &E.sc->steps, sizeof(steps), cudaMemcpyDeviceToHost, E.stream));
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    E.cur = (int)((E.cur_base + (steps - E.steps_base)) & 1);
    E.pending = false;
    return PG_OK;
}

static pg_status stage_buffer(Engine3& E, size_t n, double** out) {
    if (E.stage_n < n) {
        if (E.stage) cudaFree(E.stage);
        E.stage = nullptr;
        E.stage_n = 0;
        PG3_CUDA(cudaMalloc(&E.stage, n * sizeof(double)));
        E.stage_n = n;
    }
    *out = E.stage;
    return PG_OK;
}

static void release3(Engine3* E) {
    if (!E) return;
    for (int b = 0; b < 2; ++b) {
        if (E->graph[b]) cudaGraphExecDestroy(E->graph[b]);
        if (E->buf[b] && E->own_buffers) cudaFree(E->buf[b]);
    }
    if (E->tables) cudaFree(E->tables);
    if (E->stage) cudaFree(E->stage);
    if (E->sc) cudaFree(E->sc);
    if (E->own_stream && E->stream) cudaStreamDestroy(E->stream);
    delete E;
}

static pg_status create3(const pg_params* P, int device, cudaStream_t stream, Engine3** out, bool own = true) {
    pg_status s = check3(P);
    if (s != PG_OK) return s;
    PG3_CUDA(cudaSetDevice(device));
    Engine3* E = new Engine3();
    E->P = *P;
    if (E->P.kill_width_out <= 0.0) E->P.kill_width_out = E->P.kill_width;
    E->device = device;
    auto bad = [&](pg_status st) {
        release3(E);
        return st;
    };
    if (stream) {
        E->stream = stream;
    } else {
        if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bad(fail3(PG_ERR_CUDA, "stream creation failed"));
        E->own_stream = true;
    }
    const pg_params& Q = E->P;
    const int xarr = Q.xres + 2 * NPAD, yarr = Q.yres + 2 * NPAD, zarr = Q.zres + 2 * NPAD;
    std::vector<double> xa(xarr + 1), xv(xarr), ya(yarr + 1), yv(yarr), za(zarr + 1), zv(zarr);
    make_grid(xa.data(), xv.data(), Q.xmin, Q.xmax, Q.xres, NPAD, Q.geomx, Q.gridx, &Q);
    make_grid(ya.data(), yv.data(), Q.ymin, Q.ymax, Q.yres, NPAD, Q.geomy, Q.gridy, &Q);
    make_grid(za.data(), zv.data(), Q.zmin, Q.zmax, Q.zres, NPAD, Q.geomz, Q.gridz, &Q);
    for (double a : xa) if (!std::isfinite(a)) return bad(fail3(PG_ERR_CONFIG, "the radial spacing needs more cells"));
    for (double a : ya) if (!std::isfinite(a)) return bad(fail3(PG_ERR_CONFIG, "the azimuthal spacing needs more cells"));
    for (double a : za) if (!std::isfinite(a)) return bad(fail3(PG_ERR_CONFIG, "the polar spacing needs more cells"));
    E->hxa = xa;
    E->hya = ya;
    E->hza = za;
    // table block: faces and volumes, weights, per-index and (x, z) tables, trig
    const size_t nxz = (size_t)xarr * zarr;
    const size_t ntab = (xarr + 1) + xarr + (yarr + 1) + yarr + (zarr + 1) + zarr   // grid
                        + 6 * (size_t)(xarr + yarr + zarr)                             // slope weights
                        + 6 * (size_t)zarr + (zarr + 1) + (xarr + 1)                   // zc sinz sinpol cospol tanz idx_z gfz gfx
                        + 2 * (size_t)xarr + 4 * (size_t)xarr                          // radx idx_x killx
                        + 2 * (size_t)yarr                                             // ycj idx_y
                        + nxz + 5 * nxz                                                // cs2 initc
                        + 4 * (size_t)yarr + 2;                                        // trig
    if (cudaMalloc(&E->tables, ntab * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&E->sc, sizeof(Scalars)) != cudaSuccess)
        return bad(fail3(PG_ERR_CUDA, "table allocation failed"));
    const size_t ncell = (size_t)xarr * yarr * zarr;
    E->own_buffers = own;
    for (int b = 0; own && b < 2; ++b)
        if (cudaMalloc(&E->buf[b], ncell * sizeof(Cell)) != cudaSuccess)
            return bad(fail3(PG_ERR_CUDA, "state allocation failed (%zu cells)", ncell));
    cudaMemsetAsync(E->sc, 0, sizeof(Scalars), E->stream);
    double* t = E->tables;
    auto take = [&](size_t n) {
        double* p = t;
        t += n;
        return p;
    };
    double* dxa = take(xarr + 1);
    double* dxv = take(xarr);
    double* dya = take(yarr + 1);
    double* dyv = take(yarr);
    double* dza = take(zarr + 1);
    double* dzv = take(zarr);
    double* wx = take(6 * (size_t)xarr);
    double* wy = take(6 * (size_t)yarr);
    double* wz = take(6 * (size_t)zarr);
    double* zc = take(zarr);
    double* sinz = take(zarr);
    double* sinpol = take(zarr);
    double* cospol = take(zarr);
    double* tanz = take(zarr);
    double* idx_z = take(zarr);
    double* gfz = take(zarr + 1);
    double* gfx = take(xarr + 1);
    double* radx = take(xarr);
    double* idx_x = take(xarr);
    double* killx = take(4 * (size_t)xarr);
    double* ycj = take(yarr);
    double* idx_y = take(yarr);
    double* cs2 = take(nxz);
    double* initc = take(5 * nxz);
    double* trig = take(4 * (size_t)yarr + 2);
    cudaMemcpyAsync(dxa, xa.data(), xa.size() * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(dxv, xv.data(), xv.size() * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(dya, ya.data(), ya.size() * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(dyv, yv.data(), yv.size() * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(dza, za.data(), za.size() * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(dzv, zv.data(), zv.size() * 8, cudaMemcpyHostToDevice, E->stream);
    // 4th-order slope weights of each direction from the reference's own rounded
    // grid moments (evaluated on the device with its expressions)
    std::vector<double> w(6 * (size_t)std::max(xarr, std::max(yarr, zarr)));
    const int geoms[3] = {Q.geomx, Q.geomy, Q.geomz};
    const int ns[3] = {xarr, yarr, zarr};
    const double* faces[3] = {dxa, dya, dza};
    double* wdst[3] = {wx, wy, wz};
    for (int a = 0; a < 3; ++a) {
        s = recon_weights(geoms[a], faces[a], ns[a], w.data(), E->stream);
        if (s != PG_OK) return bad(s);
        cudaMemcpyAsync(wdst[a], w.data(), 6 * (size_t)ns[a] * 8, cudaMemcpyHostToDevice, E->stream);
        if (cudaStreamSynchronize(E->stream) != cudaSuccess) return bad(fail3(PG_ERR_CUDA, "weight upload failed"));
    }
    DiskView& d = E->v.d;
    d.xres = Q.xres;
    d.yres = Q.yres;
    d.xarr = xarr;
    d.yarr = yarr;
    d.ypad = NPAD;
    d.ndim = 3;
    d.geomx = Q.geomx;
    d.geomy = Q.geomy;
    d.eos = Q.eos_flag;
    d.ie = Q.internal_e_flag;
    d.bound_lft = Q.bound_lft;
    d.bound_rgh = Q.bound_rgh;
    d.kill = Q.kill_flag;
    d.nplanet = Q.n_planet;
    d.gam = Q.gam;
    d.cfl = Q.cfl;
    d.frame_omega = Q.frame_omega;
    d.planet_mass = Q.planet_mass;
    d.ramp_time = Q.ramp_time;
    d.xa = dxa;
    d.xv = dxv;
    d.wx = wx;
    d.wy = wy;
    d.ya = dya;
    d.yv = dyv;
    d.radx = radx;
    d.ycj = ycj;
    d.ycraw = ycj;
    d.killx = killx;
    d.idx_x = idx_x;
    d.idx_y = idx_y;
    d.trig = trig;
    d.sc = E->sc;
    View3& v = E->v;
    v.zres = Q.zres;
    v.zarr = zarr;
    v.geomz = Q.geomz;
    v.bound_bom = Q.bound_bom;
    v.bound_top = Q.bound_top;
    v.init3 = Q.init_flag == 3;
    v.zmin = Q.zmin;
    v.za = dza;
    v.zv = dzv;
    v.wz = wz;
    v.idx_z = idx_z;
    v.zc = zc;
    v.sinz = sinz;
    v.sinpol = sinpol;
    v.cospol = cospol;
    v.tanz = tanz;
    v.gfx = gfx;
    v.gfz = gfz;
    v.cs2 = cs2;
    v.initc = initc;
    Tab3Args ta{Q.sc_h, Q.planet_radius, Q.p_alpha, Q.p_beta, Q.xmin, Q.xmax, Q.kill_width, E->P.kill_width_out,
                Q.geomx, Q.init_flag, Q.kill_flag};
    const long long nt = std::max((long long)nxz, (long long)std::max(xarr, std::max(yarr, zarr)) + 1);
    k3_tables<<<(unsigned)((nt + 127) / 128), 128, 0, E->stream>>>(v, ta, zc, sinz, sinpol, cospol, tanz, idx_z, gfx,
                                                                      gfz, radx, idx_x, killx, ycj, idx_y, cs2, initc);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(E->stream) != cudaSuccess)
        return bad(fail3(PG_ERR_CUDA, "table kernel failed"));
    for (int b = 0; own && b < 2; ++b)
        if ((s = make_maps(*E, b)) != PG_OK) return bad(s);
    cudaFuncSetAttribute(k3_sweep<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S3_SMEM);
    cudaFuncSetAttribute(k3_sweep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S3_SMEM);
    cudaFuncSetAttribute(k3_sweep<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S3_SMEM);
    const int res[3] = {Q.xres, Q.yres, Q.zres};
    for (int a = 0; a < 3; ++a) {
        E->nta[a] = (res[a] + S3_L - 1) / S3_L;
        E->ntb[a] = ((a == 0 ? Q.yres : Q.xres) + S3_W - 1) / S3_W;
        E->ntiles[a] = E->nta[a] * E->ntb[a] * (a == 2 ? Q.yres : Q.zres);
    }
    E->grid_sweep[0] = occupancy_grid((const void*)k3_sweep<0>, S3_THREADS, S3_SMEM, E->ntiles[0]);
    E->grid_sweep[1] = occupancy_grid((const void*)k3_sweep<1>, S3_THREADS, S3_SMEM, E->ntiles[1]);
    E->grid_sweep[2] = occupancy_grid((const void*)k3_sweep<2>, S3_THREADS, S3_SMEM, E->ntiles[2]);
    const long long ncin = (long long)Q.xres * Q.yres * Q.zres;
    E->grid_kick = occupancy_grid((const void*)k3_kick<2>, K3_THREADS, 0, (ncin + K3_THREADS - 1) / K3_THREADS);
    *out = E;
    return PG_OK;
}

// ------------------------------------------------------- drop-in (Grid)
// pg_grid_* with ndim 3: the engine's tables for the caller's grid, keyed by
// its device xa; the state lives in the caller's C and T.
static std::map<const double*, Engine3*> g_grids3;

pg_status check_params3(const pg_params* P) { return check3(P); }

static pg_status grid3_engine(const pg_params& P, pg_grid* dev, Engine3** out) {
    if (!dev) return fail3(PG_ERR_ARG, "null grid");
    if (dev->xres != P.xres || dev->yres != P.yres || dev->zres != P.zres)
        return fail3(PG_ERR_CONFIG, "grid dimensions differ from the configured parameters");
    if (dev->xbgn != 0) return fail3(PG_ERR_CONFIG, "radial domain decomposition is not supported");
    auto it = g_grids3.find(dev->xa);
    if (it != g_grids3.end()) {
        *out = it->second;
        return PG_OK;
    }
    int device = 0;
    PG3_CUDA(cudaGetDevice(&device));
    Engine3* E = nullptr;
    pg_status s = create3(&P, device, (cudaStream_t)dev->stream, &E, false);
    if (s != PG_OK) return s;
    g_grids3[dev->xa] = E;
    *out = E;
    return PG_OK;
}

pg_status grid3_init_orbadv(const pg_params& P, pg_grid* dev) {
    Engine3* E = nullptr;
    pg_status s = grid3_engine(P, dev, &E);
    if (s != PG_OK) return s;
    // init_OrbAdv (src/orbit/orbit.cu:51-72) without OrbAdv_flag: orb_rot 0, orb_shf 0
    const size_t nxz = (size_t)dev->xarr * dev->zarr;
    if (dev->orb_rot) PG3_CUDA(cudaMemsetAsync(dev->orb_rot, 0, sizeof(double) * nxz, E->stream));
    if (dev->orb_shf) PG3_CUDA(cudaMemsetAsync(dev->orb_shf, 0, sizeof(int) * nxz, E->stream));
    PG3_CUDA(cudaStreamSynchronize(E->stream));
    return PG_OK;
}

pg_status grid3_global_dt(const pg_params& P, pg_grid* dev, double dt_prev, double* dt_out) {
    Engine3* E = nullptr;
    pg_status s = grid3_engine(P, dev, &E);
    if (s != PG_OK) return s;
    PG3_CUDA(cudaMemsetAsync(&E->sc->vmax_bits, 0, sizeof(unsigned long long), E->stream));
    k3_cfl<<<E->grid_kick, K3_THREADS, 0, E->stream>>>(E->v, reinterpret_cast<const Cell*>(dev->C));
    PG3_CUDA(cudaGetLastError());
    unsigned long long bits = 0;
    PG3_CUDA(cudaMemcpyAsync(&bits, &E->sc->vmax_bits, sizeof(bits), cudaMemcpyDeviceToHost, E->stream));
    PG3_CUDA(cudaStreamSynchronize(E->stream));
    double vmax;
    std::memcpy(&vmax, &bits, sizeof vmax);
    const double dt = E->P.cfl / vmax;  // get_dt_lv2 (timestep.cu:108)
    double tmp = dt_prev * 1.1;         // timestep.cu:133-139
    if (dt < tmp) tmp = dt;
    *dt_out = tmp;
    return PG_OK;
}

pg_status grid3_solve(const pg_params& P, pg_grid* dev, double time, double dt) {
    Engine3* E = nullptr;
    pg_status s = grid3_engine(P, dev, &E);
    if (s != PG_OK) return s;
    E->buf[0] = reinterpret_cast<Cell*>(dev->C);
    E->buf[1] = reinterpret_cast<Cell*>(dev->T);
    for (int b = 0; b < 2; ++b) {
        if (E->map_base[b] != E->buf[b] && (s = make_maps(*E, b)) != PG_OK) return s;
        if (std::find(E->ghosted.begin(), E->ghosted.end(), E->buf[b]) == E->ghosted.end()) {
            k3_analytic_ghosts<<<1184, 256, 0, E->stream>>>(E->v, E->buf[b]);
            E->ghosted.push_back(E->buf[b]);
        }
    }
    if (E->v.d.nplanet > 0 && dev->planets) k_grid_planet_in<<<1, 1, 0, E->stream>>>(E->sc, dev->planets, 0);
    launch_set_time(E->v.d, time, dt, E->stream);
    enqueue_passes(*E, 0);
    if (E->v.d.nplanet > 0 && dev->planets) k_grid_planet_out<<<1, 1, 0, E->stream>>>(E->sc, dev->planets, 0);
    PG3_CUDA(cudaGetLastError());
    // the newest state is in T: swap like the reference (src/solver/sweeps.cu:353-355, 550-552)
    pg_cell* t = dev->C;
    dev->C = dev->T;
    dev->T = t;
    return PG_OK;
}

void grid3_release() {
    for (auto& kv : g_grids3) release3(kv.second);
    g_grids3.clear();
}

// Device-clocked steps from here on run towards end_time (main.cu:322-339).
static pg_status begin_run(Engine3& E, double end_time) {
    PG3_CUDA(cudaSetDevice(E.device));
    pg_status s = resolve3(E);
    if (s != PG_OK) return s;
    Scalars h{};
    PG3_CUDA(cudaMemcpyAsync(&h, E.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, E.stream));
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    // main.cu:144 + 322: the first cap on dt is end_time - t after a (re)start;
    // a run that stopped on a clip at its end_time continues like main.cu after a
    // dump (main.cu:333-338, 425)
    if (E.fresh) h.dt_prev = end_time - h.t;
    else if (h.dt_hold > 0.0) h.dt_prev = h.dt_hold;
    h.dt_hold = 0.0;
    h.end_time = end_time;
    h.done = 0;
    h.pad_ = 0;
    PG3_CUDA(cudaMemcpyAsync(E.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, E.stream));
    E.fresh = false;
    E.cur_base = E.cur;
    E.steps_base = h.steps;
    E.pending = true;
    return PG_OK;
}

}  // namespace pg

using namespace pg;

struct pg_disk3 {
    Engine3* E;
};

extern "C" {

pg_status pg_make_axis(const pg_params* P, int axis, double* a, double* v) {
    if (!P || !a || !v || axis < 0 || axis > 2) return fail3(PG_ERR_ARG, "bad argument");
    const int pad = (axis == 0 || (axis == 1 && P->ndim > 1) || (axis == 2 && P->ndim > 2)) ? NPAD : 0;
    if (axis == 0) make_grid(a, v, P->xmin, P->xmax, P->xres, pad, P->geomx, P->gridx, P);
    else if (axis == 1) make_grid(a, v, P->ymin, P->ymax, P->yres, pad, P->geomy, P->gridy, P);
    else make_grid(a, v, P->zmin, P->zmax, P->zres, pad, P->geomz, P->gridz, P);
    return PG_OK;
}

pg_status pg_disk3_create(const pg_params* P, int device, void* stream, pg_disk3** out) {
    if (!out) return fail3(PG_ERR_ARG, "null argument");
    Engine3* E = nullptr;
    pg_status s = create3(P, device, (cudaStream_t)stream, &E);
    if (s != PG_OK) return s;
    *out = new pg_disk3{E};
    return PG_OK;
}

pg_status pg_disk3_destroy(pg_disk3* dk) {
    if (!dk) return PG_OK;
    cudaSetDevice(dk->E->device);
    cudaStreamSynchronize(dk->E->stream);
    release3(dk->E);
    delete dk;
    return PG_OK;
}

pg_status pg_disk3_set_state(pg_disk3* dk, double t, const double* r, const double* p, const double* u,
                             const double* v, const double* w) {
    if (!dk || !r || !p || !u || !v || !w) return fail3(PG_ERR_ARG, "null argument");
    Engine3& E = *dk->E;
    PG3_CUDA(cudaSetDevice(E.device));
    const size_t n = (size_t)E.P.xres * E.P.yres * E.P.zres;
    double* st = nullptr;
    pg_status s = stage_buffer(E, 5 * n, &st);
    if (s != PG_OK) return s;
    const double* src[5] = {r, p, u, v, w};
    for (int f = 0; f < 5; ++f)
        PG3_CUDA(cudaMemcpyAsync(st + f * n, src[f], n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    k3_fill<<<1184, 256, 0, E.stream>>>(E.v, E.buf[0], E.buf[1], st, st + n, st + 2 * n, st + 3 * n, st + 4 * n);
    PG3_CUDA(cudaGetLastError());
    E.cur = 0;
    E.pending = false;
    E.fresh = true;
    launch_init_planet(E.v.d, E.P, t, E.stream);
    Scalars h{};
    PG3_CUDA(cudaMemcpyAsync(&h, E.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, E.stream));
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    h.t = t;
    h.dt = 0.0;
    h.dt_prev = 0.0;
    h.end_time = 1.0e30;
    h.vmax_bits = 0ull;
    h.steps = 0;
    h.done = 0;
    h.pad_ = 0;
    h.err = 0;
    h.floor_hits = 0;
    h.dt_hold = 0.0;
    PG3_CUDA(cudaMemcpyAsync(E.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, E.stream));
    k3_cfl<<<E.grid_kick, K3_THREADS, 0, E.stream>>>(E.v, E.buf[0]);
    PG3_CUDA(cudaGetLastError());
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

pg_status pg_disk3_get_state(pg_disk3* dk, double* r, double* p, double* u, double* v, double* w, double* t_out) {
    if (!dk || !r || !p || !u || !v || !w) return fail3(PG_ERR_ARG, "null argument");
    Engine3& E = *dk->E;
    PG3_CUDA(cudaSetDevice(E.device));
    pg_status s = resolve3(E);
    if (s != PG_OK) return s;
    const size_t n = (size_t)E.P.xres * E.P.yres * E.P.zres;
    double* st = nullptr;
    if ((s = stage_buffer(E, 5 * n, &st)) != PG_OK) return s;
    k3_extract<<<1184, 256, 0, E.stream>>>(E.v, E.buf[E.cur], st, st + n, st + 2 * n, st + 3 * n, st + 4 * n);
    PG3_CUDA(cudaGetLastError());
    double* dst[5] = {r, p, u, v, w};
    for (int f = 0; f < 5; ++f)
        PG3_CUDA(cudaMemcpyAsync(dst[f], st + f * n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    if (t_out) PG3_CUDA(cudaMemcpyAsync(t_out, &E.sc->t, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

pg_status pg_disk3_global_dt(pg_disk3* dk, double dt_prev, double* dt_out) {
    if (!dk || !dt_out) return fail3(PG_ERR_ARG, "null argument");
    Engine3& E = *dk->E;
    PG3_CUDA(cudaSetDevice(E.device));
    unsigned long long bits = 0;
    PG3_CUDA(cudaMemcpyAsync(&bits, &E.sc->vmax_bits, sizeof(bits), cudaMemcpyDeviceToHost, E.stream));
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    double vmax;
    std::memcpy(&vmax, &bits, sizeof vmax);
    const double dt = E.P.cfl / vmax;  // get_dt_lv2 (timestep.cu:108)
    double tmp = dt_prev * 1.1;        // timestep.cu:133-139
    if (dt < tmp) tmp = dt;
    *dt_out = tmp;
    return PG_OK;
}

pg_status pg_disk3_solve(pg_disk3* dk, double t, double dt) {
    if (!dk) return fail3(PG_ERR_ARG, "null disk");
    Engine3& E = *dk->E;
    PG3_CUDA(cudaSetDevice(E.device));
    pg_status s = resolve3(E);
    if (s != PG_OK) return s;
    launch_set_time(E.v.d, t, dt, E.stream);
    enqueue_passes(E, E.cur);
    PG3_CUDA(cudaGetLastError());
    E.cur = 1 - E.cur;
    E.fresh = false;
    return PG_OK;
}

pg_status pg_disk3_run(pg_disk3* dk, int nsteps, double end_time) {
    if (!dk) return fail3(PG_ERR_ARG, "null disk");
    if (nsteps <= 0) return PG_OK;
    Engine3& E = *dk->E;
    pg_status s = begin_run(E, end_time);
    if (s != PG_OK) return s;
    const bool may_finish = end_time < 1.0e29;
    for (int step = 0; step < nsteps; ++step) {
        if (may_finish && step > 0 && step % 256 == 0) {
            int done = 0;
            PG3_CUDA(cudaMemcpyAsync(&done, &E.sc->done, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
            PG3_CUDA(cudaStreamSynchronize(E.stream));
            if (done) break;
        }
        const int c0 = E.cur;
        if (!E.graph[c0]) {  // one step (clock + five passes) from buffer c0, captured once
            cudaGraph_t g;
            PG3_CUDA(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
            launch_time_step(E.v.d, E.stream);
            enqueue_passes(E, c0);
            cudaError_t ce = cudaStreamEndCapture(E.stream, &g);
            PG3_CUDA(ce);
            PG3_CUDA(cudaGraphInstantiate(&E.graph[c0], g, 0));
            cudaGraphDestroy(g);
        }
        PG3_CUDA(cudaGraphLaunch(E.graph[c0], E.stream));
        E.cur = 1 - c0;
    }
    if (!may_finish) E.pending = false;
    else E.cur = E.cur_base;  // resolved from the device step count on next use
    return PG_OK;
}

pg_status pg_disk3_clock(pg_disk3* dk, double* t, double* dt, long long* steps) {
    if (!dk) return fail3(PG_ERR_ARG, "null disk");
    Scalars h{};
    PG3_CUDA(cudaMemcpyAsync(&h, dk->E->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, dk->E->stream));
    PG3_CUDA(cudaStreamSynchronize(dk->E->stream));
    if (t) *t = h.t;
    if (dt) *dt = h.dt;
    if (steps) *steps = h.steps;
    return PG_OK;
}

pg_status pg_disk3_check(pg_disk3* dk) {
    if (!dk) return fail3(PG_ERR_ARG, "null disk");
    Engine3& E = *dk->E;
    int err = 0;
    PG3_CUDA(cudaMemcpyAsync(&err, &E.sc->err, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    const int zero = 0;
    PG3_CUDA(cudaMemcpy(&E.sc->err, &zero, sizeof(int), cudaMemcpyHostToDevice));
    if (err & (1 << PG_ERR_TIMEOUT)) return fail3(PG_ERR_TIMEOUT, "a device wait timed out");
    if (err & (1 << PG_ERR_NAN)) return fail3(PG_ERR_NAN, "non-positive or NaN density produced");
    return PG_OK;
}

// Average device time of each pass over nsteps device-clocked steps (CUDA
// events on the disk's stream): clock, kick1, sweep_x, sweep_y, sweep_z, kick2.
pg_status pg_disk3_pass_times(pg_disk3* dk, int nsteps, double* ms6) {
    if (!dk || !ms6 || nsteps <= 0) return fail3(PG_ERR_ARG, "bad argument");
    Engine3& E = *dk->E;
    pg_status s = begin_run(E, 1.0e30);
    if (s != PG_OK) return s;
    E.pending = false;  // no end_time: every step runs
    cudaEvent_t ev[7];
    for (auto& e : ev) PG3_CUDA(cudaEventCreate(&e));
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const View3& v = E.v;
    for (int step = 0; step < nsteps; ++step) {
        const int c = E.cur;
        Cell* A = E.buf[c];
        Cell* B = E.buf[1 - c];
        cudaEventRecord(ev[0], E.stream);
        launch_time_step(v.d, E.stream);
        cudaEventRecord(ev[1], E.stream);
        k3_kick<1><<<E.grid_kick, K3_THREADS, 0, E.stream>>>(v, A, B);
        cudaEventRecord(ev[2], E.stream);
        k3_sweep<0><<<E.grid_sweep[0], S3_THREADS, S3_SMEM, E.stream>>>(E.maps[1 - c][0], v, A, E.nta[0], E.ntb[0],
                                                                          E.ntiles[0]);
        cudaEventRecord(ev[3], E.stream);
        k3_sweep<1><<<E.grid_sweep[1], S3_THREADS, S3_SMEM, E.stream>>>(E.maps[c][1], v, B, E.nta[1], E.ntb[1],
                                                                          E.ntiles[1]);
        cudaEventRecord(ev[4], E.stream);
        k3_sweep<2><<<E.grid_sweep[2], S3_THREADS, S3_SMEM, E.stream>>>(E.maps[1 - c][2], v, A, E.nta[2], E.ntb[2],
                                                                          E.ntiles[2]);
        cudaEventRecord(ev[5], E.stream);
        k3_kick<2><<<E.grid_kick, K3_THREADS, 0, E.stream>>>(v, A, B);
        cudaEventRecord(ev[6], E.stream);
        PG3_CUDA(cudaGetLastError());
        PG3_CUDA(cudaEventSynchronize(ev[6]));
        for (int k = 0; k < 6; ++k) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            acc[k] += ms;
        }
        E.cur = 1 - c;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 6; ++k) ms6[k] = acc[k] / nsteps;
    return PG_OK;
}

// write_check_point (src/output/output.cu:125-180, ndim 3): t, the interior
// faces of x, y and z, then the r, p, u, v, w planes (x fastest, then y, then z)
pg_status pg_disk3_write_snapshot(pg_disk3* dk, const char* path) {
    if (!dk || !path) return fail3(PG_ERR_ARG, "null argument");
    Engine3& E = *dk->E;
    const size_t n = (size_t)E.P.xres * E.P.yres * E.P.zres;
    std::vector<double> h(5 * n);
    double t = 0.0;
    pg_status s = pg_disk3_get_state(dk, h.data(), h.data() + n, h.data() + 2 * n, h.data() + 3 * n, h.data() + 4 * n, &t);
    if (s != PG_OK) return s;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail3(PG_ERR_ARG, "cannot open %s", path);
    bool ok = std::fwrite(&t, sizeof(double), 1, f) == 1;
    ok = ok && std::fwrite(&E.hxa[NPAD], sizeof(double), E.P.xres + 1, f) == (size_t)E.P.xres + 1;
    ok = ok && std::fwrite(&E.hya[NPAD], sizeof(double), E.P.yres + 1, f) == (size_t)E.P.yres + 1;
    ok = ok && std::fwrite(&E.hza[NPAD], sizeof(double), E.P.zres + 1, f) == (size_t)E.P.zres + 1;
    ok = ok && std::fwrite(h.data(), sizeof(double), 5 * n, f) == 5 * n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PG_OK : fail3(PG_ERR_ARG, "short write to %s", path);
}

// load_grid (src/output/output.cu:182-248, ndim 3): t and the five planes of a
// checkpoint file (the faces are skipped), then a restart at t like set_state
pg_status pg_disk3_read_snapshot(pg_disk3* dk, const char* path, double* t_out) {
    if (!dk || !path) return fail3(PG_ERR_ARG, "null argument");
    Engine3& E = *dk->E;
    const size_t n = (size_t)E.P.xres * E.P.yres * E.P.zres;
    std::vector<double> h(5 * n);
    double t = 0.0;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail3(PG_ERR_ARG, "cannot open %s", path);
    bool ok = std::fread(&t, sizeof(double), 1, f) == 1;
    ok = ok && std::fseek(f, (long)sizeof(double) * (1 + E.P.xres + 1 + E.P.yres + 1 + E.P.zres + 1), SEEK_SET) == 0;
    ok = ok && std::fread(h.data(), sizeof(double), 5 * n, f) == 5 * n;
    std::fclose(f);
    if (!ok) return fail3(PG_ERR_ARG, "%s is not a checkpoint of this grid", path);
    if (t_out) *t_out = t;
    return pg_disk3_set_state(dk, t, h.data(), h.data() + n, h.data() + 2 * n, h.data() + 3 * n, h.data() + 4 * n);
}

// test support: one step with host t and dt (as pg_disk3_solve), copying the
// whole buffer (ghosts included, xarr*yarr*zarr cells) after each of the five
// passes into out (5 x that many cells): kick1, sweep_x, sweep_y, sweep_z,
// kick2 (with the damping).  Blocking.
pg_status pg_disk3_stages(pg_disk3* dk, double t, double dt, pg_cell* out) {
    if (!dk || !out) return fail3(PG_ERR_ARG, "null argument");
    Engine3& E = *dk->E;
    PG3_CUDA(cudaSetDevice(E.device));
    pg_status s = resolve3(E);
    if (s != PG_OK) return s;
    const View3& v = E.v;
    const size_t n = (size_t)v.d.xarr * v.d.yarr * v.zarr;
    const int c = E.cur;
    Cell* A = E.buf[c];
    Cell* B = E.buf[1 - c];
    launch_set_time(v.d, t, dt, E.stream);
    auto grab = [&](const Cell* src, int k) {
        return cudaMemcpyAsync(out + k * n, src, n * sizeof(Cell), cudaMemcpyDeviceToHost, E.stream);
    };
    k3_kick<1><<<E.grid_kick, K3_THREADS, 0, E.stream>>>(v, A, B);
    PG3_CUDA(grab(B, 0));
    k3_sweep<0><<<E.grid_sweep[0], S3_THREADS, S3_SMEM, E.stream>>>(E.maps[1 - c][0], v, A, E.nta[0], E.ntb[0],
                                                                      E.ntiles[0]);
    PG3_CUDA(grab(A, 1));
    k3_sweep<1><<<E.grid_sweep[1], S3_THREADS, S3_SMEM, E.stream>>>(E.maps[c][1], v, B, E.nta[1], E.ntb[1],
                                                                      E.ntiles[1]);
    PG3_CUDA(grab(B, 2));
    k3_sweep<2><<<E.grid_sweep[2], S3_THREADS, S3_SMEM, E.stream>>>(E.maps[1 - c][2], v, A, E.nta[2], E.ntb[2],
                                                                      E.ntiles[2]);
    PG3_CUDA(grab(A, 3));
    k3_kick<2><<<E.grid_kick, K3_THREADS, 0, E.stream>>>(v, A, B);
    PG3_CUDA(grab(B, 4));
    PG3_CUDA(cudaGetLastError());
    PG3_CUDA(cudaStreamSynchronize(E.stream));
    E.cur = 1 - c;
    E.fresh = false;
    return PG_OK;
}

}  // extern "C"
