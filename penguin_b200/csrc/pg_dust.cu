// Dust passes of the FP64 step (dust_flag): the radial and azimuthal dust
// sweeps (src/solver/dust/dust.cu:6-326; the azimuthal one writes each cell at
// its orbital-advection shifted row like the gas, src/orbit/orbit.cu:17-49) and
// the dust residual advection (src/solver/advection/advection.cu:175-357).
// The dust half-kicks are fused into the gas kick passes (pg_kernels.cu).
//
// The reference's dust reconstruction reads the recon_flag 6 flattening
// coefficient from shared memory that dust_flow / advection never write
// (src/solver/recon/PPM.cu:68-77); it is 0 here, which is what the reference
// computes when that memory holds zeros.
#include "pg_common.cuh"
#include "pg_dust.cuh"
#include "pg_hydro.cuh"
#include "pg_internal.h"

namespace pg {

constexpr int DS_LEN = 32, DS_W = 8;
constexpr int DS_TL = DS_LEN + 2 * NPAD;               // 38
constexpr int DS_P1 = DS_LEN + 2, DS_P2 = DS_LEN + 1;  // cells with edge states, faces per pencil
constexpr int DS_THREADS = 288;
constexpr int DS_NST = DS_P1 * DS_W, DS_NFX = DS_P2 * DS_W;
constexpr int DSY_COLS = DS_W + 2;                     // y tiles start one column early (16-B TMA x)
constexpr int DSX_TILE = 4 * DS_TL * DS_W;             // 1216 doubles
constexpr int DSY_TILE = 4 * DS_TL * DSY_COLS;         // 1520 doubles
constexpr int DS_STAGE = (DSY_TILE + 15) / 16 * 16;    // 128-B aligned stages
constexpr size_t DS_SMEM = (size_t)(2 * DS_STAGE + 8 * DS_NST + 4 * DS_NFX) * 8 + 16 + 128;
constexpr int DA_NF = DS_TL * DS_W;                    // advection faces per tile
constexpr size_t DA_SMEM = (size_t)(2 * DS_STAGE + 4 * DA_NF) * 8 + 16 + 128;

// src/solver/riemann/riemann.cu:5-11
__device__ __forceinline__ double gfac(int geom, double x) {
    if (geom == 1) return x;
    if (geom == 2) return x * x;
    return 1.0;
}

// ============================================================ dust sweeps
// DIR 0: radial pencils of rows (fields r, u, r v, w); DIR 1: azimuthal pencils of
// columns (r, v - orb_rot - r Omega, w, u).
template <int DIR>
__global__ void __launch_bounds__(DS_THREADS) k_dsweep(const __grid_constant__ CUtensorMap tm, const DiskView d,
                                                      pg_dust* __restrict__ out, int ntx, int ntiles) {
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    auto stage = [&](int n) { return smem + (n & 1) * DS_STAGE; };
    double* st = smem + 2 * DS_STAGE;  // [8][DS_NST]: right state of the left face, left state of the right face
    double* fl = st + 8 * DS_NST;      // [4][DS_NFX]
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 4 * DS_NFX);
    __shared__ int s_inc[DS_W];
    Scalars* sc = d.sc;
    if (sc->done) return;
    const int tid = threadIdx.x;
    const double dt = sc->dt;
    const double* fa = (DIR == 0) ? d.xa : d.ya;
    const int geom = (DIR == 0) ? d.geomx : d.geomy;
    auto origin = [&](int tile, int& s0, int& q0) {
        s0 = NPAD + DS_LEN * (tile % ntx);
        q0 = (DIR == 0 ? d.ypad : NPAD) + DS_W * (tile / ntx);
    };
    auto issue = [&](int tile, int k) {
        int s0, q0;
        origin(tile, s0, q0);
        issue_begin(&bar[k & 1], (DIR == 0 ? DSX_TILE : DSY_TILE) * 8);
        if (DIR == 0) tma_load_2d(stage(k), &tm, 4 * (s0 - NPAD), q0, &bar[k & 1]);
        else tma_load_2d(stage(k), &tm, 4 * (q0 - 1), s0 - NPAD, &bar[k & 1]);
    };
    // tile cell (position along the pencil t, pencil q) -> its 4 doubles
    auto cellp = [&](const double* T, int t, int q) {
        return (DIR == 0) ? T + (q * DS_TL + t) * 4 : T + (t * DSY_COLS + (q + 1)) * 4;
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int s0, q0;
        origin(tile_id, s0, q0);
        const double* T = stage(kt);
        if (DIR == 1 && tid < DS_W) {
            // the gas's set_orbital_advection (orbit.cu:74-99): the same shift for the dust
            const int i = q0 + tid;
            int shift = 0;
            if (d.orbadv && i < NPAD + d.xres) {
                const double dy = d.dy0 * d.radx[i];
                shift = __double2int_rd(d.rot[i] * dt / dy + 0.5);
            }
            s_inc[tid] = shift;
        }
        if (!pipe_wait(bar, kt, sc)) {
            pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
            return;
        }

        // ---- P1: per cell, the state at its left face (seen from the right) and at
        // its right face (seen from the left), dust_flux (dust.cu:6-103)
        if (tid < DS_NST) {
            const int q = (DIR == 0) ? tid / DS_P1 : tid % DS_W;
            const int t = 2 + ((DIR == 0) ? tid % DS_P1 : tid / DS_W);
            const int s = s0 - NPAD + t;
            const int sc_ = (DIR == 0) ? min(s, d.xarr - 1) : min(s, d.yarr - 1);
            const int i = (DIR == 0) ? 0 : min(q0 + q, d.xarr - 1);
            double rad = 1.0, rot = 0.0;
            if (DIR == 1) {
                rad = (d.geomy == 3) ? d.radx[i] : 1.0;
                rot = d.rot[i];
            }
            double r[5], u[5], v[5], w[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const double* c = cellp(T, t - 2 + m, q);
                r[m] = c[0];
                if (DIR == 0) {
                    u[m] = c[1];
                    v[m] = c[2];
                    if (d.geomx == 1) v[m] *= d.radx[min(max(s - 2 + m, 0), d.xarr - 1)];
                    w[m] = c[3];
                } else {
                    u[m] = c[2] - rot;
                    if (d.geomy == 3) u[m] -= rad * d.frame_omega;
                    v[m] = c[3];
                    w[m] = c[1];
                }
            }
            const double* wt = ((DIR == 0) ? d.wx : d.wy) + 6 * sc_;
            const Par R = recon(wt, r[0], r[1], r[2], r[3], r[4], 0.0);
            const Par U = recon(wt, u[0], u[1], u[2], u[3], u[4], 0.0);
            const Par V = recon(wt, v[0], v[1], v[2], v[3], v[4], 0.0);
            const Par W = recon(wt, w[0], w[1], w[2], w[3], w[4], 0.0);
            const double sdt = (DIR == 0 || geom <= 2) ? dt : dt / rad;  // dust_flow (dust.cu:120-121)
            const double xl = fa[sc_], xr = fa[sc_ + 1];
            // left face, from this cell
            double tmp = xl - fmin(U.a - U.sL, 0.0) * sdt;
            Frac fq = frac_left(lim01((tmp - xl) / (xr - xl)));
            const double ur = aveL(fq, U);
            double u_ = 0.5 * sdt * (ur - u[2]) / (0.5 * (xr - tmp));
            tmp = xl - fmin(ur, 0.0) * sdt;
            fq = frac_left(lim01((tmp - xl) / (xr - xl)));
            const double Srr = aveL(fq, R) * exp_lim(u_);
            const double Sur = aveL(fq, U) + 0.0;
            const double Svr = aveL(fq, V), Swr = aveL(fq, W);
            // right face, from this cell
            tmp = xr - fmax(U.a + U.sR, 0.0) * sdt;
            fq = frac_right(lim01((tmp - xl) / (xr - xl)));
            const double ul = aveR(fq, U);
            u_ = 0.5 * sdt * (u[2] - ul) / (0.5 * (tmp - xl));
            tmp = xr - fmax(ul, 0.0) * sdt;
            fq = frac_right(lim01((tmp - xl) / (xr - xl)));
            const double Srl = aveR(fq, R) * exp_lim(u_);
            const double Sul = aveR(fq, U) + 0.0;
            const double Svl = aveR(fq, V), Swl = aveR(fq, W);
            double* o = st + tid;
            o[0] = Srr;
            o[DS_NST] = Sur;
            o[2 * DS_NST] = Svr;
            o[3 * DS_NST] = Swr;
            o[4 * DS_NST] = Srl;
            o[5 * DS_NST] = Sul;
            o[6 * DS_NST] = Svl;
            o[7 * DS_NST] = Swl;
        }
        __syncthreads();

        // ---- P2: limited mass flux and the upwind transport at every face
        if (tid < DS_NFX) {
            const int q = (DIR == 0) ? tid / DS_P2 : tid % DS_W;
            const int f = (DIR == 0) ? tid % DS_P2 : tid / DS_W;  // between tile cells 2+f and 3+f
            const int iL = (DIR == 0) ? q * DS_P1 + f : f * DS_W + q;
            const int iR = (DIR == 0) ? iL + 1 : iL + DS_W;
            const int sf = s0 + f;  // face index = index of the right cell
            const int sfc = (DIR == 0) ? min(sf, d.xarr - 1) : min(sf, d.yarr - 1);
            double rad = 1.0;
            if (DIR == 1) rad = (d.geomy == 3) ? d.radx[min(q0 + q, d.xarr - 1)] : 1.0;
            const double sdt = (DIR == 0 || geom <= 2) ? dt : dt / rad;
            const double rL = cellp(T, 2 + f, q)[0], rR = cellp(T, 3 + f, q)[0];
            const double Srl = fmin(rL * sdt / (fa[sfc] - fa[sfc - 1]), fmax(st[5 * DS_NST + iL] * st[4 * DS_NST + iL], 0.0));
            const double Srr = fmax(rR * sdt / (fa[sfc] - fa[sfc + 1]), fmin(st[DS_NST + iR] * st[iR], 0.0));
            fl[tid] = Srl + Srr;
            fl[DS_NFX + tid] = Srl * st[5 * DS_NST + iL] + Srr * st[DS_NST + iR];
            fl[2 * DS_NFX + tid] = Srl * st[6 * DS_NST + iL] + Srr * st[2 * DS_NST + iR];
            fl[3 * DS_NFX + tid] = Srl * st[7 * DS_NST + iL] + Srr * st[3 * DS_NST + iR];
        }
        __syncthreads();

        // ---- P3: flux differences and update_Dust (dust.cu:149-235, 256-326)
        if (tid < DS_LEN * DS_W) {
            const int q = (DIR == 0) ? tid / DS_LEN : tid % DS_W;
            const int o = (DIR == 0) ? tid % DS_LEN : tid / DS_W;
            const int s = s0 + o, qq = q0 + q;
            const bool valid = (DIR == 0) ? (s < NPAD + d.xres && qq < d.ypad + d.yres)
                                          : (s < NPAD + d.yres && qq < NPAD + d.xres);
            if (valid) {
                const int f0 = (DIR == 0) ? q * DS_P2 + o : o * DS_W + q;
                const int f1 = (DIR == 0) ? f0 + 1 : f0 + DS_W;
                const double g0 = gfac(geom, fa[s]), g1 = gfac(geom, fa[s + 1]);
                DCell D;
                D.r = fl[f0] * g0 - fl[f1] * g1;
                D.u = fl[DS_NFX + f0] * g0 - fl[DS_NFX + f1] * g1;
                D.v = fl[2 * DS_NFX + f0] * g0 - fl[2 * DS_NFX + f1] * g1;
                D.w = fl[3 * DS_NFX + f0] * g0 - fl[3 * DS_NFX + f1] * g1;
                const double* c = cellp(T, NPAD + o, q);
                const DCell Q{c[0], c[1], c[2], c[3]};
                if (DIR == 0) {
                    const double f = dt / d.xv[s];
                    D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                    if (d.geomx == 1) D.v /= d.radx[s];
                    const DCell N = update_dust(d, Q, D);
                    if (!(N.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                    emit_dust(d, out, s, qq, N);
                } else {
                    const double rad = (d.geomy == 3) ? d.radx[qq] : 1.0;
                    double f = dt / d.yv[s];
                    D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                    if (d.geomy > 2) {
                        f = 1.0 / rad;
                        D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                    }
                    if (d.geomy == 3) D.u += (d.rot[qq] + rad * d.frame_omega) * D.r;
                    else D.u += d.rot[qq] * D.r;
                    const DCell E{D.r, D.w, D.u, D.v};
                    const DCell N = update_dust(d, Q, E);
                    if (!(N.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                    int j = s;
                    if (d.orbadv) {  // TD[(j+inc) mod N] = CD[j] (orbit.cu:30-46)
                        int js = (s - d.ypad + s_inc[q]) % d.yres;
                        if (js < 0) js += d.yres;
                        j = js + d.ypad;
                    }
                    emit_dust(d, out, qq, j, N);
                }
            }
        }
        __syncthreads();
    }
}

// ===================================================== dust residual advection
// advection() on Dust (advection.cu:175-233) + advecty (:235-290): the gas's
// residual speed orb_res, fields (r, v, w, u), update_Dust.
__global__ void __launch_bounds__(DS_THREADS) k_dadvect(const __grid_constant__ CUtensorMap tm, const DiskView d,
                                                       pg_dust* __restrict__ out, int ntx, int ntiles) {
    extern __shared__ __align__(128) double smem_raw[];
    double* smem = smem_base128(smem_raw);
    auto stage = [&](int n) { return smem + (n & 1) * DS_STAGE; };
    double* fl = smem + 2 * DS_STAGE;  // [4][DA_NF] upwind fluxes, indexed by face t
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 4 * DA_NF);
    Scalars* sc = d.sc;
    if (sc->done) return;
    const int tid = threadIdx.x;
    const double dt = sc->dt;
    auto origin = [&](int tile, int& s0, int& q0) {
        s0 = NPAD + DS_LEN * (tile % ntx);
        q0 = NPAD + DS_W * (tile / ntx);
    };
    auto issue = [&](int tile, int k) {
        int s0, q0;
        origin(tile, s0, q0);
        issue_begin(&bar[k & 1], DSY_TILE * 8);
        tma_load_2d(stage(k), &tm, 4 * (q0 - 1), s0 - NPAD, &bar[k & 1]);
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int s0, q0;
        origin(tile_id, s0, q0);
        const double* T = stage(kt);
        if (!pipe_wait(bar, kt, sc)) {
            pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
            return;
        }
        if (tid < DS_NST) {
            const int q = tid % DS_W, t = 2 + tid / DS_W;
            const int s = min(s0 - NPAD + t, d.yarr - 1);
            const int i = min(q0 + q, d.xarr - 1);
            const double speed = d.res[i];
            const double rad = (d.geomy == 3) ? d.radx[i] : 1.0;
            const double sdt = dt / rad;
            double r[5], u[5], v[5], w[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const double* c = T + ((t - 2 + m) * DSY_COLS + (q + 1)) * 4;
                r[m] = c[0];
                u[m] = c[2];
                v[m] = c[3];
                w[m] = c[1];
            }
            const double* wt = d.wy + 6 * s;
            const Par R = recon(wt, r[0], r[1], r[2], r[3], r[4], 0.0);
            const Par U = recon(wt, u[0], u[1], u[2], u[3], u[4], 0.0);
            const Par V = recon(wt, v[0], v[1], v[2], v[3], v[4], 0.0);
            const Par W = recon(wt, w[0], w[1], w[2], w[3], w[4], 0.0);
            const double xl = d.ya[s], xr = d.ya[s + 1];
            double fr, fu, fv, fw;
            int face;
            if (speed > 0.0) {
                const double x0 = xr - speed * sdt;
                const Frac fq = frac_right(lim01((x0 - xl) / (xr - xl)));
                fr = aveR(fq, R);
                fu = aveR(fq, U) * fr;
                fv = aveR(fq, V) * fr;
                fw = aveR(fq, W) * fr;
                face = t + 1;
            } else {
                const double x0 = xl - speed * sdt;
                const Frac fq = frac_left(lim01((x0 - xl) / (xr - xl)));
                fr = aveL(fq, R);
                fu = aveL(fq, U) * fr;
                fv = aveL(fq, V) * fr;
                fw = aveL(fq, W) * fr;
                face = t;
            }
            const int k = face * DS_W + q;
            fl[k] = fr * speed;
            fl[DA_NF + k] = fu * speed;
            fl[2 * DA_NF + k] = fv * speed;
            fl[3 * DA_NF + k] = fw * speed;
        }
        __syncthreads();
        if (tid < DS_LEN * DS_W) {
            const int q = tid % DS_W, o = tid / DS_W;
            const int s = s0 + o, i = q0 + q;
            if (s < NPAD + d.yres && i < NPAD + d.xres) {
                const int t = NPAD + o;
                const int k0 = t * DS_W + q, k1 = (t + 1) * DS_W + q;
                DCell D;
                D.r = fl[k0] * 1.0 - fl[k1] * 1.0;
                D.u = fl[DA_NF + k0] * 1.0 - fl[DA_NF + k1] * 1.0;
                D.v = fl[2 * DA_NF + k0] * 1.0 - fl[2 * DA_NF + k1] * 1.0;
                D.w = fl[3 * DA_NF + k0] * 1.0 - fl[3 * DA_NF + k1] * 1.0;
                double f = dt / d.yv[s];
                D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                if (d.geomy > 2) {
                    f = 1.0 / ((d.geomy == 3) ? d.radx[i] : 1.0);
                    D.r *= f; D.u *= f; D.v *= f; D.w *= f;
                }
                const double* c = T + (t * DSY_COLS + (q + 1)) * 4;
                const DCell Q{c[0], c[1], c[2], c[3]};
                const DCell N = update_dust(d, Q, DCell{D.r, D.w, D.u, D.v});
                if (!(N.r > 0.0)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                emit_dust(d, out, i, s, N);
            }
        }
        __syncthreads();
    }
}

// ================================================================ misc
// init_CD everywhere (fill_grid, src/init/init.cu:502-519): the dust of a restart
// (the reference's load_grid reads the gas only, src/output/output.cu:182-248).
__global__ void k_dust_init(const DiskView d, pg_dust* buf) {
    const long long n = (long long)d.xarr * d.yarr;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % d.xarr), j = (int)(k / d.xarr);
        const double* I = d.initd + 4 * i;
        store_dust(buf, d.xarr, i, j, DCell{I[0], I[1], I[2], I[3]});
    }
}

// Bound-0 radial ghosts of a dust buffer: init_CD (boundx_dust,
// src/boundary/boundary.cu:64-113), every row.
__global__ void k_dust_xghosts(const DiskView d, pg_dust* buf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 2 * NPAD * d.yarr) return;
    const int j = k / (2 * NPAD), n = k % (2 * NPAD);
    const int i = n < NPAD ? n : d.xres + n;  // 0..NPAD-1 and NPAD+xres..xarr-1
    const bool bound0 = (n < NPAD) ? d.bound_lft == 0 : d.bound_rgh == 0;
    if (!bound0) return;
    const double* I = d.initd + 4 * i;
    store_dust(buf, d.xarr, i, j, DCell{I[0], I[1], I[2], I[3]});
}

// The ghost images of every interior dust cell (boundy_dust and the bound 1/2
// radial ghosts), for a dust state written by the caller.
__global__ void k_dust_images(const DiskView d, pg_dust* buf) {
    const long long n = (long long)d.xres * d.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres), j = d.ypad + (int)(m / d.xres);
        emit_dust(d, buf, i, j, load_dust(buf, d.xarr, i, j));
    }
}

// Interior dust from host arrays (r, u, v) with its ghost images.
__global__ void k_dust_fill(const DiskView d, pg_dust* buf, const double* r, const double* u, const double* v) {
    const long long n = (long long)d.xres * d.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres), j = d.ypad + (int)(m / d.xres);
        emit_dust(d, buf, i, j, DCell{r[m], u[m], v[m], 0.0});
    }
}

__global__ void k_dust_extract(const DiskView d, const pg_dust* buf, double* r, double* u, double* v) {
    const long long n = (long long)d.xres * d.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres), j = d.ypad + (int)(m / d.xres);
        const DCell c = load_dust(buf, d.xarr, i, j);
        r[m] = c.r;
        u[m] = c.u;
        v[m] = c.v;
    }
}

// ============================================================== launchers
static inline unsigned dcdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

static unsigned dust_grid(const void* kernel, size_t smem, long long ntiles) {
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm <= 0) nsm = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, DS_THREADS, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    long long g = (long long)per_sm * nsm;
    if (g > ntiles) g = ntiles;
    return (unsigned)(g < 1 ? 1 : g);
}

cudaError_t set_dust_attributes() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f, size_t bytes) {
        cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (r != cudaSuccess) e = r;
    };
    set((const void*)k_dsweep<0>, DS_SMEM);
    set((const void*)k_dsweep<1>, DS_SMEM);
    set((const void*)k_dadvect, DA_SMEM);
    return e;
}

void launch_dsweep_x(const DiskView& d, const DustMaps& in, pg_dust* out, cudaStream_t s) {
    const int ntx = (int)dcdiv(d.xres, DS_LEN), nt = ntx * (int)dcdiv(d.yres, DS_W);
    k_dsweep<0><<<dust_grid((const void*)k_dsweep<0>, DS_SMEM, nt), DS_THREADS, DS_SMEM, s>>>(in.sweep_x, d, out, ntx, nt);
}
void launch_dsweep_y(const DiskView& d, const DustMaps& in, pg_dust* out, cudaStream_t s) {
    const int ntx = (int)dcdiv(d.yres, DS_LEN), nt = ntx * (int)dcdiv(d.xres, DS_W);
    k_dsweep<1><<<dust_grid((const void*)k_dsweep<1>, DS_SMEM, nt), DS_THREADS, DS_SMEM, s>>>(in.sweep_y, d, out, ntx, nt);
}
void launch_dadvect(const DiskView& d, const DustMaps& in, pg_dust* out, cudaStream_t s) {
    const int ntx = (int)dcdiv(d.yres, DS_LEN), nt = ntx * (int)dcdiv(d.xres, DS_W);
    k_dadvect<<<dust_grid((const void*)k_dadvect, DA_SMEM, nt), DS_THREADS, DA_SMEM, s>>>(in.sweep_y, d, out, ntx, nt);
}
void launch_dust_init(const DiskView& d, pg_dust* buf, cudaStream_t s) { k_dust_init<<<592, 256, 0, s>>>(d, buf); }
void launch_dust_xghosts(const DiskView& d, pg_dust* buf, cudaStream_t s) {
    k_dust_xghosts<<<(2 * NPAD * d.yarr + 255) / 256, 256, 0, s>>>(d, buf);
}
void launch_dust_images(const DiskView& d, pg_dust* buf, cudaStream_t s) { k_dust_images<<<592, 256, 0, s>>>(d, buf); }
void launch_dust_fill(const DiskView& d, pg_dust* buf, const double* r, const double* u, const double* v,
                      cudaStream_t s) {
    k_dust_fill<<<592, 256, 0, s>>>(d, buf, r, u, v);
}
void launch_dust_extract(const DiskView& d, const pg_dust* buf, double* r, double* u, double* v, cudaStream_t s) {
    k_dust_extract<<<592, 256, 0, s>>>(d, buf, r, u, v);
}

}  // namespace pg
