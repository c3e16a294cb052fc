// FP32-mixed Godunov step for ensembles of 2D polar planet-disks (sm_100a).
//
// The same five fused passes as the FP64 kernels (kick1 C->T, radial sweep T->C,
// azimuthal sweep + orbital shift C->T, residual advection T->C, kick2 +
// damping + CFL rate C->T), on FP32 residual planes.  Every pass is ONE
// persistent launch over the concatenated tile lists of all disks in the
// ensemble: a CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... and finds
// each tile's disk by binary search over per-disk tile offsets, so disks of
// uneven size share the GPU without one launch per disk.  Tiles arrive through
// 3D TMA copies (x, y, plane) whose tensor maps live in device memory, one set
// per disk, double-buffered as in the FP64 kernels.
//
// A disk whose clock reached end_time has its tiles copied through unchanged, so
// the two state buffers of all disks stay in step.
#include <cstdio>

#include "pg_common.cuh"
#include "pg_f32.cuh"
#include "pg_internal.h"
#include "pg_planet.cuh"

namespace pg {
namespace f32 {

constexpr int T_LEN = 32, T_W = 8;           // outputs along / across the sweep per tile
constexpr int P1N = (T_LEN + 2) * T_W;       // 272 reconstructed cells
constexpr int P2N = (T_LEN + 1) * T_W;       // 264 faces
constexpr int SWT = 288;                     // sweep threads
constexpr int XB_W = 40, XB_H = 8, XPL = XB_W * XB_H, XS = XPL * NPL;                  // radial tile: 960 floats
constexpr int YB_W = 12, YB_H = 38, YPL = YB_W * YB_H, YS = (YPL * NPL + 31) / 32 * 32;  // azimuthal: 1376
constexpr int SB_W = 36, SB_H = 10, SPL = SB_W * SB_H, SS = (SPL * NPL + 31) / 32 * 32;  // stencil: 1088
constexpr int VS = (SPL * 2 + 31) / 32 * 32;                                            // stress: 736
constexpr int STT = 256;                     // stencil threads (32 x 8 cells)
constexpr int NSX = 13, NSY = 8;             // floats kept per reconstructed cell
constexpr int NFA = (T_LEN + 6) * T_W;       // advection faces per tile
constexpr size_t SX_SMEM = (size_t)(2 * XS + NSX * P1N + 4 * P2N) * 4 + 16 + 128;
constexpr size_t SY_SMEM = (size_t)(2 * YS + NSY * P1N + 4 * P2N) * 4 + 16 + 128;
constexpr size_t AD_SMEM = (size_t)(2 * YS + 3 * NFA) * 4 + 16 + 128;
constexpr size_t K1_SMEM = (size_t)(2 * SS) * 4 + 16 + 128;
constexpr size_t K2_SMEM = (size_t)(3 * SS + 2 * VS) * 4 + 16 + 128;
static_assert(XS % 32 == 0 && YS % 32 == 0 && SS % 32 == 0 && VS % 32 == 0, "128-B aligned TMA stages");
static_assert((2 * XS + NSX * P1N + 4 * P2N) % 2 == 0 && (2 * YS + NSY * P1N + 4 * P2N) % 2 == 0 &&
                  (2 * YS + 3 * NFA) % 2 == 0 && (3 * SS + 2 * VS) % 2 == 0,
              "8-B aligned barriers");

__device__ __forceinline__ float* smem_base128f(float* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    return reinterpret_cast<float*>((a + 127) & ~uintptr_t(127));
}

// disk owning global tile `tile`: the largest k with first[k] <= tile
__device__ __forceinline__ int find_disk(const int* __restrict__ first, int nd, int tile) {
    int lo = 0, hi = nd - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Planar multi-value tables: value m of slot group `slot` at index i.
template <int N>
__device__ __forceinline__ void xload(const View32& w, int slot, int i, float* out) {
#pragma unroll
    for (int m = 0; m < N; ++m) out[m] = w.tx[(size_t)(slot + m) * w.xn + i];
}
template <int N>
__device__ __forceinline__ void yload(const View32& w, int slot, int j, float* out) {
#pragma unroll
    for (int m = 0; m < N; ++m) out[m] = w.ty[(size_t)(slot + m) * w.yn + j];
}

// Interior cell (i, j) and its periodic azimuthal image (boundary.cu:141-209).
__device__ __forceinline__ void emit32(const View32& w, float* out, int i, int j, float a, float b, float c) {
    const size_t pl = w.plane();
    size_t m = (size_t)j * w.pitch + i;
    out[m] = a;
    out[pl + m] = b;
    out[2 * pl + m] = c;
    int jimg = -1;
    if (j < 2 * NPAD) jimg = j + w.yres;
    else if (j >= w.yres) jimg = j - w.yres;
    if (jimg >= 0) {
        m = (size_t)jimg * w.pitch + i;
        out[m] = a;
        out[pl + m] = b;
        out[2 * pl + m] = c;
    }
}

// Star + planet gravity (forces.cu:182-327) without the star term, which is in
// X_ABG.  |r - r_p|^2 = (r - x_p)^2 + 2 r x_p (1 - cos) + rs^2 has no cancellation.
// which: 0 = planet of the first half-kick, 1 = planet at t + dt.
__device__ __forceinline__ void gravity32(const View32& w, int i, int j, int which, float& gx, float& gy) {
    gx = 0.0f;
    gy = 0.0f;
    if (w.nplanet == 0) return;
    const float* tr = w.trow(j) + 3 * which;
    const float* s = w.tscal() + 4 * which;
    const float m = s[0], xp = s[1], rs2 = s[2], ip2 = s[3];
    const float dr = w.tcol()[2 * i + which];
    const float rad = w.x(X_RAD)[i];
    const float R2 = dr * dr + 2.0f * rad * xp * tr[2] + rs2;
    const float ir = rsqrtf(R2);
    const float rf = ir * ir * ir;
    gx = -m * (dr + xp * tr[2]) * rf - m * tr[1] * ip2;
    gy = -m * xp * tr[0] * rf + m * tr[0] * ip2;
}

// Half-kick of the residual velocities (sweeps.cu:597-711 with geomx 1):
// v^2/r - 1/r^2 = X_ABG + (2 v0/r + dv/r) dv.  mdt != 0 re-evaluates the
// curvature term at the mdt-predicted velocity (sweeps.cu:663-687).
__device__ __forceinline__ void kick32(const View32& w, int i, float dS, float& du, float& dv, float vx, float vy,
                                       float gx, float gy, float mdt, float dt, bool visc) {
    const float iS = visc ? 1.0f / (w.x(X_SBG)[i] + dS) : 0.0f;
    const float abg = w.x(X_ABG)[i], v2r = w.x(X_V2R)[i], ir = w.x(X_IRAD)[i];
    float fx = abg + (v2r + dv * ir) * dv + vx * iS;
    const float fy = vy * iS;
    if (mdt != 0.0f) {
        const float dvT = dv + fy * mdt + gy * mdt;
        fx = abg + (v2r + dvT * ir) * dvT + vx * iS;
    }
    du = du + fx * dt + gx * dt;
    dv = dv + fy * dt + gy * dt;
}

// Viscous force density at stencil-tile cell (x, y) of planes {dS, du, dv} with
// row length SB_W: residual part plus background part (viscosity.cu:84-194).
__device__ __forceinline__ void stress32(const View32& w, const float* tile, int x, int y, int i, int j, float& vx,
                                         float& vy) {
    const float* nu = w.x(X_NU);
    float vb[7], X[5], Y[4];
    xload<7>(w, X_VBG, i, vb);
    xload<5>(w, X_VISX, i, X);
    yload<4>(w, Y_VISY, j, Y);
    const float* S = tile;
    const float* U = tile + SPL;
    const float* V = tile + 2 * SPL;
    const int c = y * SB_W + x;
    const float n1 = nu[i];
    const float nr1 = (w.x(X_SBG)[i] + S[c]) * n1;
    const float dndx = (vb[6] + S[c + 1] * nu[i + 1] - S[c - 1] * nu[i - 1]) * X[0];
    const float dndy = (S[c + SB_W] - S[c - SB_W]) * n1 * Y[0] * X[4];
    float u[9], v[9];
#pragma unroll
    for (int n = 0; n < 9; ++n) {
        const int dx = (n % 3) - 1;
        const int dy = (n < 3) ? 0 : (n < 6 ? -1 : 1);
        u[n] = U[c + dy * SB_W + dx];
        v[n] = V[c + dy * SB_W + dx];
    }
    float fx, fy;
    viscous32(X, Y, u, v, nr1, dndx, dndy, fx, fy);
    vx = fx + vb[0] * nr1 + vb[1] * dndx + vb[2] * dndy;
    vy = fy + vb[3] * nr1 + vb[4] * dndx + vb[5] * dndy;
}

// CFL signal rate (timestep.cu:46-77) in FP64 from the residuals.
__device__ __forceinline__ double rate64(const View32& w, int i, int j, float du, float dv) {
    const DiskView& d = w.d64;
    const double cs = w.cs64[i];
    const double u = d.initx[5 * i + 2] + (double)du;
    const double vn = (d.initx[5 * i + 3] - d.radx[i] * d.frame_omega - d.rot[i]) + (double)dv;
    const double a = (fabs(u) + cs) * d.idx_x[i];
    const double b = (fabs(vn) + cs) * (d.idx_y[j] * d.irad[i]);
    return fmax(a, b);
}

// the dust's CFL rate (timestep.cu:64-74): its speeds without a sound speed
__device__ __forceinline__ double drate64(const View32& w, int i, int j, float du, float dv) {
    const DiskView& d = w.d64;
    const double u = d.initd[4 * i + 1] + (double)du;
    const double vn = (d.initd[4 * i + 2] - d.radx[i] * d.frame_omega - d.rot[i]) + (double)dv;
    return fmax(fabs(u) * d.idx_x[i], fabs(vn) * (d.idx_y[j] * d.irad[i]));
}

// ================================================================ dust
// One pressureless dust fluid (dust_flag) in the FP32-mixed form: residual
// planes {dSigma_d, dv_r,d, dv_phi,d} against init_CD, transported by the
// reference's upwind PPM fluxes with the compression factor and the flux
// limiter (src/solver/dust/dust.cu:6-147) and updated by update_Dust
// (dust.cu:149-176) in residual form, e.g. v_new - v = (D(Sigma v) - v D Sigma) /
// Sigma_new with the transported field taken relative to a neighbouring cell.
// Each sweep is two launches over all dust disks: one thread per face (the two
// edge states it needs and the limited fluxes into a scratch array), then one
// thread per cell.  The dust planes carry no ghost images: rows wrap, and the
// radial ghosts of boundary 0 hold init_CD, i.e. zero residuals.
struct DR {
    float S, u, v;  // residuals
};
__device__ __forceinline__ int wrap32(const View32& w, int j) {
    if (j < NPAD) return j + w.yres;
    if (j >= NPAD + w.yres) return j - w.yres;
    return j;
}
__device__ __forceinline__ DR dload(const View32& w, const float* b, int i, int j) {
    if (i < NPAD || i >= NPAD + w.xres) return {0.0f, 0.0f, 0.0f};
    const size_t pl = w.plane(), m = (size_t)wrap32(w, j) * w.pitch + i;
    return {b[m], b[pl + m], b[2 * pl + m]};
}
__device__ __forceinline__ void dstore(const View32& w, float* b, int i, int j, const DR& c) {
    const size_t pl = w.plane(), m = (size_t)j * w.pitch + i;
    b[m] = c.S;
    b[pl + m] = c.u;
    b[2 * pl + m] = c.v;
}
__device__ __forceinline__ float exp_limf(float x) { return fmaxf(1.0f + x, 1.0e-6f); }

struct DEdge {
    float S, u, t;  // density and normal velocity (absolute), transported field relative to the cell
};

// Both edge states of dust cell c of a pencil (dust.cu:6-103): DIR 0 radial
// (row q; normal v_r, transported r v_phi), DIR 1 azimuthal (column q; normal
// v_phi - orb_rot - r Omega, transported v_r).  Also the cell's averages.
template <int DIR>
__device__ __forceinline__ void dust_edges(const View32& w, const float* b, int c, int q, float dtf, DEdge& L,
                                           DEdge& R, float& Sc, float& tc) {
    float aS[5], aU[5], aT[5];
    const DR C = (DIR == 0) ? dload(w, b, c, q) : dload(w, b, q, c);
    float idx, sdt, uc;
    const float* wt;
    float wts[6];
    if (DIR == 0) {
        float db[12];
        xload<12>(w, X_DDBG, c, db);
        const float* rad = w.x(X_RAD);
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            if (m == 2) {
                aS[m] = aU[m] = aT[m] = 0.0f;
                continue;
            }
            const int kk = m < 2 ? m : m - 1;
            const DR N = dload(w, b, c - 2 + m, q);
            aS[m] = db[kk] + (N.S - C.S);
            aU[m] = db[4 + kk] + (N.u - C.u);
            aT[m] = db[8 + kk] + (rad[c - 2 + m] * N.v - rad[c] * C.v);
        }
        xload<6>(w, X_WX, c, wts);
        wt = wts;
        idx = w.x(X_IDX)[c];
        sdt = dtf;
        Sc = w.x(X_DSBG)[c] + C.S;
        uc = w.x(X_DUBG)[c] + C.u;
        tc = C.v;  // only differences of r v_phi are used
    } else {
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            if (m == 2) {
                aS[m] = aU[m] = aT[m] = 0.0f;
                continue;
            }
            const DR N = dload(w, b, q, c - 2 + m);
            aS[m] = N.S - C.S;
            aU[m] = N.v - C.v;
            aT[m] = N.u - C.u;
        }
        const int cw = wrap32(w, c);
        yload<6>(w, Y_WY, cw, wts);
        wt = wts;
        idx = w.y(Y_IDY)[cw];
        sdt = dtf * w.x(X_IRAD)[q];
        Sc = w.x(X_DSBG)[q] + C.S;
        uc = w.x(X_DEPS)[q] + C.v;
        tc = C.u;
    }
    const Par32 Rp = recon32(wt, aS[0], aS[1], aS[3], aS[4], 0.0f);
    const Par32 Up = recon32(wt, aU[0], aU[1], aU[3], aU[4], 0.0f);
    const Par32 Tp = recon32(wt, aT[0], aT[1], aT[3], aT[4], 0.0f);
    const float dx = 1.0f / idx;
    {  // left edge: the right state of the face below
        const float ue = uc - Up.sL;
        const Frac32 q1 = frac32(lim01f(-fminf(ue, 0.0f) * sdt * idx));
        const float urd = aveL32(q1, Up);
        const float u_ = sdt * urd / (dx + fminf(ue, 0.0f) * sdt);
        const float ur = uc + urd;
        const Frac32 q2 = frac32(lim01f(-fminf(ur, 0.0f) * sdt * idx));
        L.S = (Sc + aveL32(q2, Rp)) * exp_limf(u_);
        L.u = uc + aveL32(q2, Up);
        L.t = aveL32(q2, Tp);
    }
    {  // right edge: the left state of the face above
        const float ue = uc + Up.sR;
        const Frac32 q1 = frac32(lim01f(fmaxf(ue, 0.0f) * sdt * idx));
        const float uld = aveR32(q1, Up);
        const float u_ = -sdt * uld / (dx - fmaxf(ue, 0.0f) * sdt);
        const float ul = uc + uld;
        const Frac32 q2 = frac32(lim01f(fmaxf(ul, 0.0f) * sdt * idx));
        R.S = (Sc + aveR32(q2, Rp)) * exp_limf(u_);
        R.u = uc + aveR32(q2, Up);
        R.t = aveR32(q2, Tp);
    }
}

// dust offsets: [3][nd + 1] running counts of radial faces, azimuthal faces, cells
__device__ __forceinline__ bool dust_unit(const int* doff, int nd, int row, long long g, int& k, int& loc) {
    const int* o = doff + row * (nd + 1);
    if (g >= o[nd]) return false;
    k = find_disk(o, nd, (int)g);
    loc = (int)(g - o[k]);
    return true;
}

// face fluxes of the dust sweeps: DIR 0 radial, DIR 1 azimuthal
template <int DIR>
__global__ void __launch_bounds__(256) k32d_faces(const View32* __restrict__ V, const int* __restrict__ doff, int nd,
                                                 int in) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int k, loc;
    if (!dust_unit(doff, nd, DIR, g, k, loc)) return;
    const View32& w = V[k];
    if (w.d64.sc->done) return;
    const float dtf = (float)w.d64.sc->dt;
    const float* b = w.dbuf[in];
    int f, q;
    if (DIR == 0) {
        f = NPAD + loc % (w.xres + 1);
        q = NPAD + loc / (w.xres + 1);
    } else {
        q = NPAD + loc % w.xres;
        f = NPAD + loc / w.xres;
    }
    DEdge La, Ra, Lb, Rb;
    float Sa, ta, Sb, tb;
    dust_edges<DIR>(w, b, f - 1, q, dtf, La, Ra, Sa, ta);
    dust_edges<DIR>(w, b, f, q, dtf, Lb, Rb, Sb, tb);
    float ia, ib, sdt;
    if (DIR == 0) {
        ia = w.x(X_IDX)[f - 1];
        ib = w.x(X_IDX)[f];
        sdt = dtf;
    } else {
        ia = w.y(Y_IDY)[wrap32(w, f - 1)];
        ib = w.y(Y_IDY)[wrap32(w, f)];
        sdt = dtf * w.x(X_IRAD)[q];
    }
    // dust_flow's limiter (dust.cu:120-147)
    const float Fl = fminf(Sa * sdt * ia, fmaxf(Ra.u * Ra.S, 0.0f));
    const float Fr = fmaxf(-Sb * sdt * ib, fminf(Lb.u * Lb.S, 0.0f));
    // the jump of the transported field from cell a to cell b
    float jab;
    if (DIR == 0) jab = w.x(X_DDBG + 10)[f - 1] + (w.x(X_RAD)[f] * tb - w.x(X_RAD)[f - 1] * ta);
    else jab = tb - ta;
    const size_t fp = (size_t)(w.xres + 1) * (w.yres + 1);
    const size_t m = (DIR == 0) ? (size_t)(q - NPAD) * (w.xres + 1) + (f - NPAD)
                                : (size_t)(f - NPAD) * (w.xres + 1) + (q - NPAD);
    w.dflux[m] = Fl + Fr;
    w.dflux[fp + m] = Fl * Ra.u + Fr * Lb.u;
    w.dflux[2 * fp + m] = Fl * Ra.t + Fr * (jab + Lb.t);  // relative to cell a
}

// update_Dust of one cell from its two faces; DIR 1 writes at the orbital-shifted row
template <int DIR>
__global__ void __launch_bounds__(256) k32d_update(const View32* __restrict__ V, const int* __restrict__ doff, int nd,
                                                  int in) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int k, loc;
    if (!dust_unit(doff, nd, 2, g, k, loc)) return;
    const View32& w = V[k];
    Scalars* sc = w.d64.sc;
    const int i = NPAD + loc % w.xres, j = NPAD + loc / w.xres;
    const float* b = w.dbuf[in];
    DR Q = dload(w, b, i, j);
    int jo = j;
    if (!sc->done) {
        const float dtf = (float)sc->dt;
        const size_t fp = (size_t)(w.xres + 1) * (w.yres + 1);
        size_t m0, m1;
        float f, g0 = 1.0f, g1 = 1.0f;
        if (DIR == 0) {
            m0 = (size_t)(j - NPAD) * (w.xres + 1) + (i - NPAD);
            m1 = m0 + 1;
            g0 = w.x(X_XA)[i];
            g1 = w.x(X_XA)[i + 1];
            f = dtf * w.x(X_IXV)[i];
        } else {
            m0 = (size_t)(j - NPAD) * (w.xres + 1) + (i - NPAD);
            m1 = m0 + (w.xres + 1);
            f = dtf * w.y(Y_IYV)[j] * w.x(X_IRAD)[i];
        }
        const float F0 = w.dflux[m0], F1 = w.dflux[m1];
        const float U0 = w.dflux[fp + m0], U1 = w.dflux[fp + m1];
        const float T0 = w.dflux[2 * fp + m0], T1 = w.dflux[2 * fp + m1];
        float un, jm;  // normal velocity of the cell; jump of the transported field from the cell below
        if (DIR == 0) {
            un = w.x(X_DUBG)[i] + Q.u;
            const DR P = dload(w, b, i - 1, j);
            jm = -(w.x(X_DDBG + 9)[i] + (w.x(X_RAD)[i - 1] * P.v - w.x(X_RAD)[i] * Q.v));
        } else {
            un = w.x(X_DEPS)[i] + Q.v;
            const DR P = dload(w, b, i, j - 1);
            jm = Q.u - P.u;
        }
        const float DS = (F0 * g0 - F1 * g1) * f;
        const float Dn = (g0 * (U0 - F0 * un) - g1 * (U1 - F1 * un)) * f;  // D(Sigma u_n) - u_n D Sigma
        const float Dt = (g0 * (T0 - F0 * jm) - g1 * T1) * f;              // D(Sigma t) - t D Sigma
        const float Sc = w.x(X_DSBG)[i] + Q.S;
        const float Sn = Sc + DS;
        const float rmin = fmaxf(Sc * 1.0e-10f, w.dust_rmin);
        if (Sn < rmin) {
            Q.S = rmin - w.x(X_DSBG)[i];
        } else {
            const float iS = 1.0f / Sn;
            Q.S += DS;
            if (DIR == 0) {
                Q.u += Dn * iS;
                Q.v += Dt * w.x(X_IRAD)[i] * iS;
            } else {
                Q.v += Dn * iS;
                Q.u += Dt * iS;
            }
        }
        if (!(Sn > 0.0f)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
        if (DIR == 1 && w.orbadv) {  // the gas's shift of this radius (orbit.cu:30-46)
            int js = (j - NPAD + w.d64.inc[i]) % w.yres;
            if (js < 0) js += w.yres;
            jo = js + NPAD;
        }
    }
    dstore(w, w.dbuf[in ^ 1], i, jo, Q);
}

// residual advection of the dust by orb_res (advection.cu:175-357): the face
// flux from the upwind cell
__global__ void __launch_bounds__(256) k32d_adv_faces(const View32* __restrict__ V, const int* __restrict__ doff,
                                                     int nd, int in) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int k, loc;
    if (!dust_unit(doff, nd, 1, g, k, loc)) return;
    const View32& w = V[k];
    if (w.d64.sc->done) return;
    const float dtf = (float)w.d64.sc->dt;
    const float* b = w.dbuf[in];
    const int q = NPAD + loc % w.xres, f = NPAD + loc / w.xres;
    const float speed = (float)w.d64.res[q];
    const int c = speed > 0.0f ? f - 1 : f;  // the upwind cell
    float aS[5], aV[5], aU[5];
    const DR C = dload(w, b, q, c);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const DR N = dload(w, b, q, c - 2 + m);
        aS[m] = N.S - C.S;
        aV[m] = N.v - C.v;
        aU[m] = N.u - C.u;
    }
    const int cw = wrap32(w, c);
    float wt[6];
    yload<6>(w, Y_WY, cw, wt);
    const Par32 Rp = recon32(wt, aS[0], aS[1], aS[3], aS[4], 0.0f);
    const Par32 Vp = recon32(wt, aV[0], aV[1], aV[3], aV[4], 0.0f);
    const Par32 Up = recon32(wt, aU[0], aU[1], aU[3], aU[4], 0.0f);
    const float sdt = dtf * w.x(X_IRAD)[q], idx = w.y(Y_IDY)[cw];
    const float Sc = w.x(X_DSBG)[q] + C.S;
    float fr, fv, fu;
    if (speed > 0.0f) {
        const Frac32 fq = frac32(lim01f(speed * sdt * idx));
        fr = Sc + aveR32(fq, Rp);
        fv = aveR32(fq, Vp);
        fu = aveR32(fq, Up);
    } else {
        const Frac32 fq = frac32(lim01f(-speed * sdt * idx));
        fr = Sc + aveL32(fq, Rp);
        fv = aveL32(fq, Vp);
        fu = aveL32(fq, Up);
    }
    if (c == f) {  // relative to the face's lower cell f - 1
        const DR P = dload(w, b, q, f - 1);
        fv += C.v - P.v;
        fu += C.u - P.u;
    }
    const float F = fr * speed;
    const size_t fp = (size_t)(w.xres + 1) * (w.yres + 1);
    const size_t m = (size_t)(f - NPAD) * (w.xres + 1) + (q - NPAD);
    w.dflux[m] = F;
    w.dflux[fp + m] = F * fv;
    w.dflux[2 * fp + m] = F * fu;
}

__global__ void __launch_bounds__(256) k32d_adv_update(const View32* __restrict__ V, const int* __restrict__ doff,
                                                      int nd, int in) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int k, loc;
    if (!dust_unit(doff, nd, 2, g, k, loc)) return;
    const View32& w = V[k];
    Scalars* sc = w.d64.sc;
    const int i = NPAD + loc % w.xres, j = NPAD + loc / w.xres;
    const float* b = w.dbuf[in];
    DR Q = dload(w, b, i, j);
    if (!sc->done) {
        const float dtf = (float)sc->dt;
        const size_t fp = (size_t)(w.xres + 1) * (w.yres + 1);
        const size_t m0 = (size_t)(j - NPAD) * (w.xres + 1) + (i - NPAD), m1 = m0 + (w.xres + 1);
        const float f = dtf * w.y(Y_IYV)[j] * w.x(X_IRAD)[i];
        const DR P = dload(w, b, i, j - 1);
        const float F0 = w.dflux[m0], F1 = w.dflux[m1];
        const float DS = (F0 - F1) * f;
        const float Dv = ((w.dflux[fp + m0] - F0 * (Q.v - P.v)) - w.dflux[fp + m1]) * f;
        const float Du = ((w.dflux[2 * fp + m0] - F0 * (Q.u - P.u)) - w.dflux[2 * fp + m1]) * f;
        const float Sc = w.x(X_DSBG)[i] + Q.S;
        const float Sn = Sc + DS;
        const float rmin = fmaxf(Sc * 1.0e-10f, w.dust_rmin);
        if (Sn < rmin) {
            Q.S = rmin - w.x(X_DSBG)[i];
        } else {
            const float iS = 1.0f / Sn;
            Q.S += DS;
            Q.v += Dv * iS;
            Q.u += Du * iS;
        }
        if (!(Sn > 0.0f)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
    }
    dstore(w, w.dbuf[in ^ 1], i, j, Q);
}

// Drag of the dust towards the gas in a half-kick (sweeps.cu:626-707, the
// exponential integrator with t_s = St h / (c_s Sigma), dust.cu:1-4) in
// residual form.  gu, gv: the gas residuals the drag relaxes to at the start;
// with mdt != 0 the forces are re-evaluated at the mdt-predicted dust velocity
// and towards the mdt-predicted gas velocity (tu, tv).  gx, gy: planet gravity.
__device__ __forceinline__ void dust_drag32(const View32& w, int i, float Sg, float gu, float gv, float tu, float tv,
                                            float gx, float gy, float mdt, float dt, DR& D) {
    const float ts = w.st_h / (w.x(X_CS0)[i] * Sg);
    const float ir = w.x(X_IRAD)[i], dabg = w.x(X_DABG)[i], dv2r = w.x(X_DV2R)[i];
    const float dgu = w.x(X_DGU)[i], dgv = w.x(X_DGV)[i];
    float vd = D.v;  // dust v_phi residual entering the curvature term
    float ru = gu, rv = gv;
    if (mdt != 0.0f) {
        const float dtm = -expm1f(-mdt / ts);
        vd = D.v + dtm * ((dgv + gv - D.v) + ts * gy);
        ru = tu;
        rv = tv;
    }
    const float dtau = -expm1f(-dt / ts);
    const float fx = (dgu + ru - D.u) + ts * (dabg + (dv2r + vd * ir) * vd + gx);
    const float fy = (dgv + rv - D.v) + ts * gy;
    D.u += dtau * fx;
    D.v += dtau * fy;
}

// ============================================================ radial sweep
// Each pass is compiled for two occupancies (MB: the CTAs per SM its register
// budget must allow); the ensemble's autotuner picks one per pass.
template <int MB>
__global__ void __launch_bounds__(SWT, MB) k32_sweep_x(const View32* __restrict__ V, const int4* __restrict__ tiles,
                                                   int nd, int ntiles, int in) {
    extern __shared__ __align__(128) float fsm_raw[];
    float* sm = smem_base128f(fsm_raw);
    auto stage = [&](int n) { return sm + (n & 1) * XS; };
    float* st = sm + 2 * XS;      // [NSX][P1N]
    float* fl = st + NSX * P1N;   // [4][P2N]
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 4 * P2N);
    const int tid = threadIdx.x;
    auto locate = [&](int tile, int& k, int& s0, int& q0) {  // the tile's disk and origin (pg_ens tile table)
        const int4 t = tiles[tile];
        k = t.x;
        s0 = t.y;
        q0 = t.z;
    };
    auto issue = [&](int tile, int kt) {
        int k, s0, q0;
        locate(tile, k, s0, q0);
        issue_begin(&bar[kt & 1], XS * 4);
        tma_load_3d(stage(kt), V[k].maps + 3 * in + 0, s0 - NPAD, q0, 0, &bar[kt & 1]);
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int k, s0, q0;
        locate(tile_id, k, s0, q0);
        const View32& w = V[k];
        Scalars* sc = w.d64.sc;
        const float* T = stage(kt);
        if (!pipe_wait(bar, kt, sc)) {
            pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
            return;
        }
        const bool done = sc->done != 0;
        const float dtf = (float)sc->dt;
        const float gam = w.gam;
        if (!done) {
            // ---- P1: deviations, reconstruction, both edge states of every cell
            if (tid < P1N) {
                const int q = tid / (T_LEN + 2), t = 2 + tid % (T_LEN + 2);
                const int s = s0 - NPAD + t;
                const int sc_ = min(s, w.xarr - 1);
                const float* r0 = T + q * XB_W + (t - 2);
                float dS[5], du[5], dv[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    dS[m] = r0[m];
                    du[m] = r0[XPL + m];
                    dv[m] = r0[2 * XPL + m];
                }
                float db[16];
                xload<16>(w, X_DBG, sc_, db);
                const float* cs2t = w.x(X_CS2);
                const float* radt = w.x(X_RAD);
                const float cs2c = cs2t[sc_], radc = radt[sc_];
                float aS[5], aP[5], aU[5], aL[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    if (m == 2) {
                        aS[m] = aP[m] = aU[m] = aL[m] = 0.0f;
                        continue;
                    }
                    const int kk = m < 2 ? m : m - 1;
                    const int sk = min(max(s - 2 + m, 0), w.xarr - 1);
                    aS[m] = (dS[m] - dS[2]) + db[kk];
                    aP[m] = (cs2t[sk] * dS[m] - cs2c * dS[2]) + db[4 + kk];
                    aU[m] = (du[m] - du[2]) + db[8 + kk];
                    aL[m] = (radt[sk] * dv[m] - radc * dv[2]) + db[12 + kk];
                }
                const float Sc = w.x(X_SBG)[sc_] + dS[2];
                const float pc = w.x(X_PBG)[sc_] + cs2c * dS[2];
                const float uc = w.x(X_UBG)[sc_] + du[2];
                const float cs0 = sqrtf(gam * pc / Sc);
                const float flat = flatten32(1.0f / cs0, pc, aP[0], aP[1], aP[3], aP[4], aU[1], aU[3]);
                float wt[6];
                xload<6>(w, X_WX, sc_, wt);
                const Par32 R = recon32(wt, aS[0], aS[1], aS[3], aS[4], flat);
                const Par32 P = recon32(wt, aP[0], aP[1], aP[3], aP[4], flat);
                const Par32 U = recon32(wt, aU[0], aU[1], aU[3], aU[4], flat);
                const Par32 L = recon32(wt, aL[0], aL[1], aL[3], aL[4], flat);
                const float idx = w.x(X_IDX)[sc_];
                const HS a = left_edge32(gam, idx, dtf, cs0, Sc, pc, uc, R, P, U, L);
                const HS b = right_edge32(gam, idx, dtf, cs0, Sc, pc, uc, R, P, U, L);
                float* o = st + tid;
                o[0] = a.rd;
                o[P1N] = a.pd;
                o[2 * P1N] = a.u;
                o[3 * P1N] = a.v;
                o[4 * P1N] = b.rd;
                o[5 * P1N] = b.pd;
                o[6 * P1N] = b.u;
                o[7 * P1N] = b.v;
                o[8 * P1N] = aS[3];  // jumps to the right neighbour
                o[9 * P1N] = aP[3];
                o[10 * P1N] = aL[3];
                o[11 * P1N] = Sc;
                o[12 * P1N] = pc;
            }
            __syncthreads();
            // ---- P2: HLLC at every face, referenced to the face's left cell
            if (tid < P2N) {
                const int q = tid / (T_LEN + 1), f = tid % (T_LEN + 1);
                const int iL = q * (T_LEN + 2) + f, iR = iL + 1;
                HS L, R;
                L.rd = st[4 * P1N + iL];
                L.pd = st[5 * P1N + iL];
                L.u = st[6 * P1N + iL];
                L.v = st[7 * P1N + iL];
                R.rd = st[iR] + st[8 * P1N + iL];
                R.pd = st[P1N + iR] + st[9 * P1N + iL];
                R.u = st[2 * P1N + iR];
                R.v = st[3 * P1N + iR] + st[10 * P1N + iL];
                const FX F = hllc32(gam, st[11 * P1N + iL], st[12 * P1N + iL], L, R);
                fl[tid] = F.r;
                fl[P2N + tid] = F.u;
                fl[2 * P2N + tid] = F.v;
                fl[3 * P2N + tid] = F.pd;
            }
            __syncthreads();
        }
        // ---- P3: residual update (sweeps.cu:218-261, 300-335)
        if (tid < T_LEN * T_W) {
            const int q = tid / T_LEN, o = tid % T_LEN;
            const int s = s0 + o, j = q0 + q;
            if (s < NPAD + w.xres && j < NPAD + w.yres) {
                const float* c = T + q * XB_W + NPAD + o;
                const float dS0 = c[0], du0 = c[XPL], dv0 = c[2 * XPL];
                float dSn = dS0, dun = du0, dvn = dv0;
                if (!done) {
                    const int iC = q * (T_LEN + 2) + 1 + o;
                    const int f0 = q * (T_LEN + 1) + o, f1 = f0 + 1;
                    const float g0 = w.x(X_XA)[s], g1 = w.x(X_XA)[s + 1];
                    const float f = dtf * w.x(X_IXV)[s];
                    const float Fr0 = fl[f0], Fr1 = fl[f1];
                    const float Dr = (Fr0 * g0 - Fr1 * g1) * f;
                    // pres0 - pres1 = (p[s-1] - p[s]) + (pd0 - pd1)
                    const float dpres = (fl[3 * P2N + f0] - fl[3 * P2N + f1]) - st[9 * P1N + iC - 1];
                    const float Du = ((fl[P2N + f0] * g0 - fl[P2N + f1] * g1) + 0.5f * (g0 + g1) * dpres) * f;
                    // D(Sigma v) - v D(Sigma) with l = r v: faces referenced to cells s-1 and s
                    const float Dv = (g0 * Fr0 * (fl[2 * P2N + f0] - st[10 * P1N + iC - 1]) - g1 * Fr1 * fl[2 * P2N + f1]) *
                                     f * w.x(X_IRAD)[s];
                    const float Sc = st[11 * P1N + iC];
                    const float uc = w.x(X_UBG)[s] + du0;
                    const float Sn = Sc + Dr;
                    const float rmin = fmaxf(Sc * 1.0e-10f, 1.0e-10f);
                    if (Sn < rmin) {
                        dSn = rmin - w.x(X_SBG)[s];
                        atomicAdd(&sc->floor_hits, 1);
                    } else {
                        const float iS = 1.0f / Sn;
                        dSn = dS0 + Dr;
                        dun = du0 + (Du - uc * Dr) * iS;
                        dvn = dv0 + Dv * iS;
                    }
                    if (!(Sn > 0.0f)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                }
                emit32(w, w.buf[in ^ 1], s, j, dSn, dun, dvn);
            }
        }
        __syncthreads();
    }
}

// ========================================= azimuthal sweep + orbital shift
template <int MB>
__global__ void __launch_bounds__(SWT, MB) k32_sweep_y(const View32* __restrict__ V, const int4* __restrict__ tiles,
                                                   int nd, int ntiles, int in) {
    extern __shared__ __align__(128) float fsm_raw[];
    float* sm = smem_base128f(fsm_raw);
    auto stage = [&](int n) { return sm + (n & 1) * YS; };
    float* st = sm + 2 * YS;      // [NSY][P1N]
    float* fl = st + NSY * P1N;   // [4][P2N]
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 4 * P2N);
    __shared__ int s_inc[T_W];
    const int tid = threadIdx.x;
    auto locate = [&](int tile, int& k, int& s0, int& q0) {  // the tile's disk and origin (pg_ens tile table)
        const int4 t = tiles[tile];
        k = t.x;
        s0 = t.y;
        q0 = t.z;
    };
    auto issue = [&](int tile, int kt) {
        int k, s0, q0;
        locate(tile, k, s0, q0);
        issue_begin(&bar[kt & 1], YPL * NPL * 4);
        tma_load_3d(stage(kt), V[k].maps + 3 * in + 1, q0 - NPAD, s0 - NPAD, 0, &bar[kt & 1]);
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int k, s0, q0;
        locate(tile_id, k, s0, q0);
        const View32& w = V[k];
        Scalars* sc = w.d64.sc;
        const float* T = stage(kt);
        const bool done = sc->done != 0;
        const double dt = sc->dt;
        const float dtf = (float)dt;
        const float gam = w.gam;
        if (tid < T_W) {
            // set_orbital_advection (src/orbit/orbit.cu:74-99) in FP64 for this column
            const int i = q0 + tid;
            int shift = 0;
            if (!done && w.orbadv && i < NPAD + w.xres) {
                const DiskView& d = w.d64;
                const double dy = d.dy0 * d.radx[i];
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
        if (!pipe_wait(bar, kt, sc)) {
            pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
            return;
        }
        if (!done) {
            // ---- P1: background-relative deviations along the column
            if (tid < P1N) {
                const int q = tid % T_W, t = 2 + tid / T_W;
                const int i = min(q0 + q, w.xarr - 1);
                const int jc = min(s0 - NPAD + t, w.yarr - 1);
                const float* col = T + (q + NPAD) + (t - 2) * YB_W;
                float dS[5], du[5], dv[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    dS[m] = col[m * YB_W];
                    du[m] = col[YPL + m * YB_W];
                    dv[m] = col[2 * YPL + m * YB_W];
                }
                float aS[5], aN[5], aT[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    aS[m] = dS[m] - dS[2];
                    aN[m] = dv[m] - dv[2];
                    aT[m] = du[m] - du[2];
                }
                const float cs2 = w.x(X_CS2)[i];
                const float Sc = w.x(X_SBG)[i] + dS[2];
                const float pc = cs2 * Sc;
                const float cs0 = w.x(X_CS0)[i];
                const float un = dv[2] + w.x(X_EPS)[i];
                // p = cs2 Sigma along the column: pressure ratios are density ratios
                const float flat = flatten32(1.0f / cs0, Sc, aS[0], aS[1], aS[3], aS[4], aN[1], aN[3]);
                float wt[6];
                yload<6>(w, Y_WY, jc, wt);
                const Par32 R = recon32(wt, aS[0], aS[1], aS[3], aS[4], flat);
                const Par32 N = recon32(wt, aN[0], aN[1], aN[3], aN[4], flat);
                const Par32 Tt = recon32(wt, aT[0], aT[1], aT[3], aT[4], flat);
                const Par32 P{cs2 * R.sL, cs2 * R.sR};
                const float sdt = dtf * w.x(X_IRAD)[i];
                const float idy = w.y(Y_IDY)[jc];
                HS a = left_edge32(gam, idy, sdt, cs0, Sc, pc, un, R, P, N, Tt);
                HS b = right_edge32(gam, idy, sdt, cs0, Sc, pc, un, R, P, N, Tt);
                a.rd += dS[2];
                a.pd += cs2 * dS[2];
                a.v += du[2];
                b.rd += dS[2];
                b.pd += cs2 * dS[2];
                b.v += du[2];
                float* o = st + tid;
                o[0] = a.rd;
                o[P1N] = a.pd;
                o[2 * P1N] = a.u;
                o[3 * P1N] = a.v;
                o[4 * P1N] = b.rd;
                o[5 * P1N] = b.pd;
                o[6 * P1N] = b.u;
                o[7 * P1N] = b.v;
            }
            __syncthreads();
            // ---- P2: HLLC referenced to the background (constant along the column)
            if (tid < P2N) {
                const int q = tid % T_W, f = tid / T_W;
                const int i = min(q0 + q, w.xarr - 1);
                const int iL = f * T_W + q, iR = iL + T_W;
                HS L, R;
                L.rd = st[4 * P1N + iL];
                L.pd = st[5 * P1N + iL];
                L.u = st[6 * P1N + iL];
                L.v = st[7 * P1N + iL];
                R.rd = st[iR];
                R.pd = st[P1N + iR];
                R.u = st[2 * P1N + iR];
                R.v = st[3 * P1N + iR];
                const FX F = hllc32(gam, w.x(X_SBG)[i], w.x(X_PBG)[i], L, R);
                fl[tid] = F.r;
                fl[P2N + tid] = F.u;
                fl[2 * P2N + tid] = F.v;
                fl[3 * P2N + tid] = F.pd;
            }
            __syncthreads();
        }
        // ---- P3: residual update (sweeps.cu:361-433) and the orbital shift (orbit.cu:30-46)
        if (tid < T_LEN * T_W) {
            const int q = tid % T_W, o = tid / T_W;
            const int j = s0 + o, i = q0 + q;
            if (j < NPAD + w.yres && i < NPAD + w.xres) {
                const float* c = T + (NPAD + o) * YB_W + NPAD + q;
                const float dS0 = c[0], du0 = c[YPL], dv0 = c[2 * YPL];
                float dSn = dS0, dun = du0, dvn = dv0;
                int jo = j;
                if (!done) {
                    const int f0 = o * T_W + q, f1 = f0 + T_W;
                    const float f = dtf * w.y(Y_IYV)[j] * w.x(X_IRAD)[i];
                    const float Fr0 = fl[f0], Fr1 = fl[f1];
                    const float Dr = (Fr0 - Fr1) * f;
                    const float Dn = ((fl[P2N + f0] - fl[P2N + f1]) + (fl[3 * P2N + f0] - fl[3 * P2N + f1])) * f;
                    const float Dt = (Fr0 * (fl[2 * P2N + f0] - du0) - Fr1 * (fl[2 * P2N + f1] - du0)) * f;
                    const float Sc = w.x(X_SBG)[i] + dS0;
                    const float Sn = Sc + Dr;
                    const float un = dv0 + w.x(X_EPS)[i];
                    const float rmin = fmaxf(Sc * 1.0e-10f, 1.0e-10f);
                    if (Sn < rmin) {
                        dSn = rmin - w.x(X_SBG)[i];
                        atomicAdd(&sc->floor_hits, 1);
                    } else {
                        const float iS = 1.0f / Sn;
                        dSn = dS0 + Dr;
                        dvn = dv0 + (Dn - un * Dr) * iS;
                        dun = du0 + Dt * iS;
                    }
                    if (!(Sn > 0.0f)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                    if (w.orbadv) {
                        int js = (j - NPAD + s_inc[q]) % w.yres;
                        if (js < 0) js += w.yres;
                        jo = js + NPAD;
                    }
                }
                emit32(w, w.buf[in ^ 1], i, jo, dSn, dun, dvn);
            }
        }
        __syncthreads();
    }
}

// ===================================================== residual advection
template <int MB>
__global__ void __launch_bounds__(SWT, MB) k32_advect(const View32* __restrict__ V, const int4* __restrict__ tiles,
                                                  int nd, int ntiles, int in) {
    extern __shared__ __align__(128) float fsm_raw[];
    float* sm = smem_base128f(fsm_raw);
    auto stage = [&](int n) { return sm + (n & 1) * YS; };
    float* fl = sm + 2 * YS;  // [3][NFA]: mass flux, then the upwind carriers of v and u
    uint64_t* bar = reinterpret_cast<uint64_t*>(fl + 3 * NFA);
    const int tid = threadIdx.x;
    auto locate = [&](int tile, int& k, int& s0, int& q0) {  // the tile's disk and origin (pg_ens tile table)
        const int4 t = tiles[tile];
        k = t.x;
        s0 = t.y;
        q0 = t.z;
    };
    auto issue = [&](int tile, int kt) {
        int k, s0, q0;
        locate(tile, k, s0, q0);
        issue_begin(&bar[kt & 1], YPL * NPL * 4);
        tma_load_3d(stage(kt), V[k].maps + 3 * in + 1, q0 - NPAD, s0 - NPAD, 0, &bar[kt & 1]);
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int k, s0, q0;
        locate(tile_id, k, s0, q0);
        const View32& w = V[k];
        Scalars* sc = w.d64.sc;
        const float* T = stage(kt);
        if (!pipe_wait(bar, kt, sc)) {
            pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
            return;
        }
        const bool done = sc->done != 0;
        const double dt = sc->dt;
        const float dtf = (float)dt;
        if (!done) {
            // ---- P1: upwind PPM average over the swept fraction (advection.cu:20-67)
            if (tid < P1N) {
                const int q = tid % T_W, t = 2 + tid / T_W;
                const int i = min(q0 + q, w.xarr - 1);
                const int jc = min(s0 - NPAD + t, w.yarr - 1);
                const DiskView& d = w.d64;
                const double speed = d.res[i];
                // the swept fraction in FP64: |res| dt / (r dphi)
                const float yf = (float)fmin(fmax(fabs(speed) * (dt * d.irad[i]) * d.idx_y[jc], 0.0), 1.0);
                const float* col = T + (q + NPAD) + (t - 2) * YB_W;
                float dS[5], du[5], dv[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    dS[m] = col[m * YB_W];
                    du[m] = col[YPL + m * YB_W];
                    dv[m] = col[2 * YPL + m * YB_W];
                }
                float wt[6];
                yload<6>(w, Y_WY, jc, wt);
                const Par32 R = recon32(wt, dS[0] - dS[2], dS[1] - dS[2], dS[3] - dS[2], dS[4] - dS[2], 0.0f);
                const Par32 N = recon32(wt, dv[0] - dv[2], dv[1] - dv[2], dv[3] - dv[2], dv[4] - dv[2], 0.0f);
                const Par32 Tt = recon32(wt, du[0] - du[2], du[1] - du[2], du[3] - du[2], du[4] - du[2], 0.0f);
                const Frac32 qf = frac32(yf);
                float fr, fn, ft;
                int face;
                if (speed > 0.0) {
                    fr = aveR32(qf, R);
                    fn = aveR32(qf, N);
                    ft = aveR32(qf, Tt);
                    face = t + 1;
                } else {
                    fr = aveL32(qf, R);
                    fn = aveL32(qf, N);
                    ft = aveL32(qf, Tt);
                    face = t;
                }
                const float Sc = w.x(X_SBG)[i] + dS[2];
                const int m = face * T_W + q;
                fl[m] = (Sc + fr) * (float)speed;
                fl[NFA + m] = dv[2] + fn;
                fl[2 * NFA + m] = du[2] + ft;
            }
            __syncthreads();
        }
        // ---- P2: flux difference and update_Cell_advect (advection.cu:88-105, 153-170)
        if (tid < T_LEN * T_W) {
            const int q = tid % T_W, o = tid / T_W;
            const int s = s0 + o, i = q0 + q;
            if (s < NPAD + w.yres && i < NPAD + w.xres) {
                const float* c = T + (NPAD + o) * YB_W + NPAD + q;
                const float dS0 = c[0], du0 = c[YPL], dv0 = c[2 * YPL];
                float dSn = dS0, dun = du0, dvn = dv0;
                if (!done) {
                    const int k0 = (NPAD + o) * T_W + q, k1 = k0 + T_W;
                    const float f = dtf * w.y(Y_IYV)[s] * w.x(X_IRAD)[i];
                    const float F0 = fl[k0], F1 = fl[k1];
                    const float Dr = (F0 - F1) * f;
                    const float Sn = (w.x(X_SBG)[i] + dS0) + Dr;
                    const float iS = 1.0f / Sn;
                    dSn = dS0 + Dr;
                    dvn = dv0 + (F0 * (fl[NFA + k0] - dv0) - F1 * (fl[NFA + k1] - dv0)) * f * iS;
                    dun = du0 + (F0 * (fl[2 * NFA + k0] - du0) - F1 * (fl[2 * NFA + k1] - du0)) * f * iS;
                    if (!(Sn > 0.0f)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                }
                emit32(w, w.buf[in ^ 1], i, s, dSn, dun, dvn);
            }
        }
        __syncthreads();
    }
}

// ====================================================== kick 1 (+ stress)
template <int MB>
__global__ void __launch_bounds__(STT, MB) k32_kick1(const View32* __restrict__ V, const int4* __restrict__ tiles, int nd,
                                                 int ntiles, int in) {
    extern __shared__ __align__(128) float fsm_raw[];
    float* sm = smem_base128f(fsm_raw);
    auto stage = [&](int n) { return sm + (n & 1) * SS; };
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * SS);
    const int tid = threadIdx.x;
    auto locate = [&](int tile, int& k, int& i0, int& j0) {  // the tile's disk and origin (pg_ens tile table)
        const int4 t = tiles[tile];
        k = t.x;
        i0 = t.y;
        j0 = t.z;
    };
    auto issue = [&](int tile, int kt) {
        int k, i0, j0;
        locate(tile, k, i0, j0);
        issue_begin(&bar[kt & 1], SPL * NPL * 4);
        tma_load_3d(stage(kt), V[k].maps + 3 * in + 2, i0 - NPAD, j0 - 1, 0, &bar[kt & 1]);
    };
    pipe_init(bar);
    if ((int)blockIdx.x >= ntiles) return;
    if (tid == 0) issue(blockIdx.x, 0);
    int kt = 0;
    for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
        if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
        int k, i0, j0;
        locate(tile_id, k, i0, j0);
        const View32& w = V[k];
        Scalars* sc = w.d64.sc;
        const float* T = stage(kt);
        if (!pipe_wait(bar, kt, sc)) {
            pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
            return;
        }
        const bool done = sc->done != 0;
        const float hdt = (float)(0.5 * sc->dt);
        const int hx = tid % T_LEN, hy = tid / T_LEN;
        const int i = i0 + hx, j = j0 + hy;
        if (i < NPAD + w.xres && j < NPAD + w.yres) {
            const int x = hx + NPAD, y = hy + 1;
            const int c = y * SB_W + x;
            const float dS0 = T[c];
            float du = T[SPL + c], dv = T[2 * SPL + c];
            const float gu = du, gv = dv;  // the gas cell the dust drag relaxes to
            DR D{0.0f, 0.0f, 0.0f};
            if (w.dust) D = dload(w, w.dbuf[in], i, j);
            if (!done) {
                float vx = 0.0f, vy = 0.0f;
                if (w.visc) {
                    stress32(w, T, x, y, i, j, vx, vy);
                    // kept for the predictor of kick2, with the periodic image
                    const size_t pl = w.plane();
                    size_t m = (size_t)j * w.pitch + i;
                    w.vis[m] = vx;
                    w.vis[pl + m] = vy;
                    int jimg = -1;
                    if (j < 2 * NPAD) jimg = j + w.yres;
                    else if (j >= w.yres) jimg = j - w.yres;
                    if (jimg >= 0) {
                        m = (size_t)jimg * w.pitch + i;
                        w.vis[m] = vx;
                        w.vis[pl + m] = vy;
                    }
                }
                float gx, gy;
                gravity32(w, i, j, 0, gx, gy);
                kick32(w, i, dS0, du, dv, vx, vy, gx, gy, 0.0f, hdt, w.visc != 0);
                if (w.dust) dust_drag32(w, i, w.x(X_SBG)[i] + dS0, gu, gv, 0.0f, 0.0f, gx, gy, 0.0f, hdt, D);
            }
            emit32(w, w.buf[in ^ 1], i, j, dS0, du, dv);
            if (w.dust) dstore(w, w.dbuf[in ^ 1], i, j, D);
        }
        __syncthreads();
    }
}

// ============================================ kick 2 + damping + CFL speed
template <int MB>
__global__ void __launch_bounds__(STT, MB) k32_kick2(const View32* __restrict__ V, const int4* __restrict__ tiles, int nd,
                                                 int ntiles, int in) {
    extern __shared__ __align__(128) float fsm_raw[];
    float* sm = smem_base128f(fsm_raw);
    auto stage = [&](int n) { return sm + (n & 1) * SS; };
    auto vstage = [&](int n) { return sm + 2 * SS + (n & 1) * VS; };
    float* tp = sm + 2 * SS + 2 * VS;  // predicted state with 1 halo, same layout as a stage
    uint64_t* bar = reinterpret_cast<uint64_t*>(tp + SS);
    const int tid = threadIdx.x;
    auto locate = [&](int tile, int& k, int& i0, int& j0) {  // the tile's disk and origin (pg_ens tile table)
        const int4 t = tiles[tile];
        k = t.x;
        i0 = t.y;
        j0 = t.z;
    };
    auto issue = [&](int tile, int kt) {
        int k, i0, j0;
        locate(tile, k, i0, j0);
        const View32& w = V[k];
        issue_begin(&bar[kt & 1], (SPL * NPL + (w.visc ? SPL * 2 : 0)) * 4);
        tma_load_3d(stage(kt), w.maps + 3 * in + 2, i0 - NPAD, j0 - 1, 0, &bar[kt & 1]);
        if (w.visc) tma_load_3d(vstage(kt), w.maps + 6, i0 - NPAD, j0 - 1, 0, &bar[kt & 1]);
    };
    pipe_init(bar);
    double vmax = 0.0;
    int vk = -1;  // disk whose signal rate vmax holds
    if ((int)blockIdx.x < ntiles) {
        if (tid == 0) issue(blockIdx.x, 0);
        int kt = 0;
        for (int tile_id = blockIdx.x; tile_id < ntiles; tile_id += gridDim.x, ++kt) {
            if (tid == 0 && tile_id + (int)gridDim.x < ntiles) issue(tile_id + gridDim.x, kt + 1);
            int k, i0, j0;
            locate(tile_id, k, i0, j0);
            const View32& w = V[k];
            Scalars* sc = w.d64.sc;
            if (k != vk) {  // uniform over the CTA: flush the previous disk's maximum
                if (vk >= 0) block_max_to<STT>(&V[vk].d64.sc->vmax_bits, vmax);
                vmax = 0.0;
                vk = k;
            }
            const float* T = stage(kt);
            const float* TV = vstage(kt);
            if (!pipe_wait(bar, kt, sc)) {
                pipe_drain(bar, kt, tile_id + (int)gridDim.x < ntiles, sc);
                return;
            }
            const bool done = sc->done != 0;
            const double dt = sc->dt;
            const float dtf = (float)dt, hdt = (float)(0.5 * dt);
            const bool visc = w.visc != 0;
            if (!done && visc) {
                // predictor (sweeps.cu:713-729, mdt = dt = dt/2) with the stress of kick1, on
                // the tile and its halo; outside the radial range the ghosts keep init_C (zero
                // residuals) as boundx2 does for boundary 0 (boundary.cu:722-820)
                for (int it = tid; it < (T_LEN + 2) * SB_H; it += STT) {
                    const int hx = it % (T_LEN + 2), hy = it / (T_LEN + 2);
                    const int x = hx + NPAD - 1, y = hy;
                    const int i = i0 - 1 + hx, j = j0 - 1 + hy;
                    const int c = y * SB_W + x;
                    float dS = T[c], du = T[SPL + c], dv = T[2 * SPL + c];
                    if (i >= NPAD && i < NPAD + w.xres && j < w.yarr) {
                        float gx, gy;
                        gravity32(w, i, j, 1, gx, gy);
                        kick32(w, i, dS, du, dv, TV[c], TV[SPL + c], gx, gy, hdt, hdt, true);
                    }
                    tp[c] = dS;
                    tp[SPL + c] = du;
                    tp[2 * SPL + c] = dv;
                }
                __syncthreads();
            }
            const int hx = tid % T_LEN, hy = tid / T_LEN;
            const int i = i0 + hx, j = j0 + hy;
            if (i < NPAD + w.xres && j < NPAD + w.yres) {
                const int x = hx + NPAD, y = hy + 1;
                const int c = y * SB_W + x;
                float dS = T[c], du = T[SPL + c], dv = T[2 * SPL + c];
                DR D{0.0f, 0.0f, 0.0f};
                if (w.dust) D = dload(w, w.dbuf[in], i, j);
                if (!done) {
                    float vx = 0.0f, vy = 0.0f;
                    if (visc) stress32(w, tp, x, y, i, j, vx, vy);
                    float gx, gy;
                    gravity32(w, i, j, 1, gx, gy);
                    if (w.dust) {
                        // the gas velocity predicted over mdt (sweeps.cu:679-687), towards which
                        // the dust's corrector relaxes
                        const float iS = visc ? 1.0f / (w.x(X_SBG)[i] + dS) : 0.0f;
                        const float ir = w.x(X_IRAD)[i];
                        const float fx0 = w.x(X_ABG)[i] + (w.x(X_V2R)[i] + dv * ir) * dv + vx * iS;
                        const float tu = du + fx0 * hdt + gx * hdt, tv = dv + vy * iS * hdt + gy * hdt;
                        dust_drag32(w, i, w.x(X_SBG)[i] + dS, du, dv, tu, tv, gx, gy, hdt, hdt, D);
                        vmax = fmax(vmax, drate64(w, i, j, D.u, D.v));
                    }
                    kick32(w, i, dS, du, dv, vx, vy, gx, gy, hdt, hdt, visc);
                    if (w.kill) {
                        // killwave (killwave.cu:48-100): relax towards init_C, i.e. residuals towards 0
                        float kw[4];
                        xload<4>(w, X_KILL, i, kw);
#pragma unroll
                        for (int side = 0; side < 2; ++side) {
                            const float itau = kw[2 * side + 1];
                            if (itau > 0.0f) {
                                const float f = kw[2 * side] * (dtf * itau);
                                dS -= f * dS;
                                du -= f * du;
                                dv -= f * dv;
                            }
                        }
                    }
                    if (!(w.x(X_SBG)[i] + dS > 0.0f)) atomicOr(&sc->err, 1 << PG_ERR_NAN);
                    vmax = fmax(vmax, rate64(w, i, j, du, dv));
                }
                emit32(w, w.buf[in ^ 1], i, j, dS, du, dv);
                if (w.dust) dstore(w, w.dbuf[in ^ 1], i, j, D);
            }
            __syncthreads();
        }
    }
    if (vk >= 0) block_max_to<STT>(&V[vk].d64.sc->vmax_bits, vmax);
}

// ================================================================ misc
// One thread per disk: dt, clock and planet of the step.
__global__ void k32_time(const View32* __restrict__ V, int nd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nd) advance_clock(V[k].d64);
}

// Per disk (blockIdx.y): the step's planet table (see TRIG_ROW).
__global__ void k32_trig(const View32* __restrict__ V) {
    const View32& w = V[blockIdx.y];
    const Scalars* sc = w.d64.sc;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const pg_body& a = sc->planet_cur;
    const pg_body& b = sc->planet_next;
    if (k < w.yarr) {
        float* t = w.trig + (size_t)TRIG_ROW * k;
#pragma unroll
        for (int which = 0; which < 2; ++which) {
            const pg_body& p = which ? b : a;
            double s, c;
            sincos(0.5 * (w.d64.ycj[k] - (p.y + 0.0 * p.vy)), &s, &c);
            t[3 * which] = (float)(2.0 * s * c);
            t[3 * which + 1] = (float)(1.0 - 2.0 * s * s);
            t[3 * which + 2] = (float)(2.0 * s * s);
        }
    }
    if (k < w.xarr) {
        float* c = w.trig + (size_t)TRIG_ROW * w.yn + 2 * k;
        c[0] = (float)(w.d64.radx[k] - a.x);
        c[1] = (float)(w.d64.radx[k] - b.x);
    }
    if (k == 0) {
        float* s = w.trig + (size_t)TRIG_ROW * w.yn + 2 * (size_t)w.xn;
        s[0] = (float)a.m;
        s[1] = (float)a.x;
        s[2] = (float)(a.rs * a.rs);
        s[3] = (float)(1.0 / a.x / a.x);
        s[4] = (float)b.m;
        s[5] = (float)b.x;
        s[6] = (float)(b.rs * b.rs);
        s[7] = (float)(1.0 / b.x / b.x);
    }
}

// Signal rate of a state just written by set_state (one disk).
__global__ void k32_cfl(const View32* __restrict__ V, int b) {
    const View32& w = *V;
    const float* buf = w.buf[b];
    const size_t pl = w.plane();
    const long long n = (long long)w.xres * w.yres;
    double vmax = 0.0;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const size_t c = (size_t)j * w.pitch + i;
        vmax = fmax(vmax, rate64(w, i, j, buf[pl + c], buf[2 * pl + c]));
        if (w.dust) vmax = fmax(vmax, drate64(w, i, j, w.dbuf[b][pl + c], w.dbuf[b][2 * pl + c]));
    }
    block_max_to<256>(&w.d64.sc->vmax_bits, vmax);
}

// dust (absolute FP64 interior arrays) <-> residual planes against init_CD
__global__ void k32_dfill(const View32* __restrict__ V, int b, const double* r, const double* u, const double* v) {
    const View32& w = *V;
    const long long n = (long long)w.xres * w.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const double* I = w.d64.initd + 4 * i;
        dstore(w, w.dbuf[b], i, j, DR{(float)(r[m] - I[0]), (float)(u[m] - I[1]), (float)(v[m] - I[2])});
    }
}
__global__ void k32_dextract(const View32* __restrict__ V, int b, double* r, double* u, double* v) {
    const View32& w = *V;
    const long long n = (long long)w.xres * w.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const double* I = w.d64.initd + 4 * i;
        const DR c = dload(w, w.dbuf[b], i, j);
        r[m] = I[0] + (double)c.S;
        u[m] = I[1] + (double)c.u;
        v[m] = I[2] + (double)c.v;
    }
}

// Host state (FP64 interior arrays) -> residual planes with their azimuthal images.
__global__ void k32_fill(const View32* __restrict__ V, int b, const double* r, const double* u, const double* v) {
    const View32& w = *V;
    const long long n = (long long)w.xres * w.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const double* I = w.d64.initx + 5 * i;
        emit32(w, w.buf[b], i, j, (float)(r[m] - I[0]), (float)(u[m] - I[2]), v ? (float)(v[m] - I[3]) : 0.0f);
    }
}

__global__ void k32_extract(const View32* __restrict__ V, int b, double* r, double* p, double* u, double* v) {
    const View32& w = *V;
    const float* buf = w.buf[b];
    const size_t pl = w.plane();
    const long long n = (long long)w.xres * w.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const size_t c = (size_t)j * w.pitch + i;
        const double* I = w.d64.initx + 5 * i;
        const double rr = I[0] + (double)buf[c];
        r[m] = rr;
        p[m] = w.d64.cs2x[i] * rr;
        u[m] = I[2] + (double)buf[pl + c];
        v[m] = I[3] + (double)buf[2 * pl + c];
    }
}

// Mass and angular momentum, sum Sigma dV and sum Sigma r v dV with dV = xv yv,
// in FP64 with compensated (Kahan) accumulation per thread, then one partial
// pair per block, summed on the host in block order (deterministic).
__global__ void k32_totals(const View32* __restrict__ V, int b, double* part) {
    const View32& w = *V;
    const DiskView& d = w.d64;
    const float* buf = w.buf[b];
    const size_t pl = w.plane();
    const long long n = (long long)w.xres * w.yres;
    double sm = 0.0, cm = 0.0, sl = 0.0, cl = 0.0;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const size_t c = (size_t)j * w.pitch + i;
        const double dV = d.xv[i] * d.yv[j];
        const double S = d.initx[5 * i] + (double)buf[c];
        const double vv = d.initx[5 * i + 3] + (double)buf[2 * pl + c];
        double y = S * dV - cm;
        double t = sm + y;
        cm = (t - sm) - y;
        sm = t;
        y = S * d.radx[i] * vv * dV - cl;
        t = sl + y;
        cl = (t - sl) - y;
        sl = t;
    }
    __shared__ double rm[256], rl[256];
    rm[threadIdx.x] = sm;
    rl[threadIdx.x] = sl;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            rm[threadIdx.x] += rm[threadIdx.x + h];
            rl[threadIdx.x] += rl[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rm[0];
        part[2 * blockIdx.x + 1] = rl[0];
    }
}

// Torque of the planet on the disk, as k_torque of the FP64 kernels
// (src/output/output.cu:336-412), in FP64 from the residual state.
__global__ void k32_torque(const View32* __restrict__ V, int b, double* part) {
    const View32& w = *V;
    const DiskView& d = w.d64;
    const pg_body p = d.sc->planet_next;
    const float* buf = w.buf[b];
    const long long n = (long long)w.xres * w.yres;
    double sum = 0.0, comp = 0.0;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % w.xres), j = NPAD + (int)(m / w.xres);
        const double rad = d.radx[i];
        double sinfac, cosfac;
        sincos(d.ycraw[j] - p.y, &sinfac, &cosfac);
        const double Rp = sqrt(rad * rad + p.x * p.x - 2.0 * p.x * rad * cosfac + p.rs * p.rs);
        const double rs_fac = 1.0 / Rp / Rp / Rp;
        const double gy = -p.m * p.x * sinfac * rs_fac + p.m * sinfac / p.x / p.x;
        const double dv = 0.5 * (d.xa[i + 1] * d.xa[i + 1] - d.xa[i] * d.xa[i]) * (d.ya[j + 1] - d.ya[j]);
        const double S = d.initx[5 * i] + (double)buf[(size_t)j * w.pitch + i];
        const double y = rad * gy * (S * dv) - comp;
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

// FP32 tables of one disk from its FP64 tables (slots in pg_f32.cuh).
__global__ void k32_init_tables(const View32 w, float* tx, float* ty, double* cs64) {
    const DiskView& d = w.d64;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    auto X = [&](int slot) { return tx + (size_t)slot * w.xn; };
    auto Y = [&](int slot) { return ty + (size_t)slot * w.yn; };
    if (k < w.xarr) {
        const int i = k;
        const double* I = d.initx + 5 * i;
        X(X_SBG)[i] = (float)I[0];
        X(X_PBG)[i] = (float)I[1];
        X(X_UBG)[i] = (float)I[2];
        X(X_CS2)[i] = (float)d.cs2x[i];
        X(X_RAD)[i] = (float)d.radx[i];
        X(X_IRAD)[i] = (float)d.irad[i];
        X(X_IDX)[i] = (float)d.idx_x[i];
        X(X_IXV)[i] = (float)d.ixv[i];
        X(X_XA)[i] = (float)d.xa[i];
        if (i == w.xarr - 1) X(X_XA)[i + 1] = (float)d.xa[i + 1];
        X(X_NU)[i] = (float)d.nux[i];
        X(X_ABG)[i] = (float)(I[3] * I[3] * d.irad[i] + d.gstar[i]);
        X(X_V2R)[i] = (float)(2.0 * I[3] * d.irad[i]);
        X(X_EPS)[i] = (float)(I[3] - d.radx[i] * d.frame_omega - d.rot[i]);
        const double cs = sqrt(d.gam * d.cs2x[i]);
        X(X_CS0)[i] = (float)cs;
        cs64[i] = cs;

        const int offs[4] = {-2, -1, 1, 2};
        for (int kk = 0; kk < 4; ++kk) {
            const int ik = min(max(i + offs[kk], 0), w.xarr - 1);
            const double* J = d.initx + 5 * ik;
            X(X_DBG + kk)[i] = (float)(J[0] - I[0]);
            X(X_DBG + 4 + kk)[i] = (float)(J[1] - I[1]);
            X(X_DBG + 8 + kk)[i] = (float)(J[2] - I[2]);
            X(X_DBG + 12 + kk)[i] = (float)(d.radx[ik] * J[3] - d.radx[i] * I[3]);
        }
        for (int m = 0; m < 6; ++m) X(X_WX + m)[i] = (float)d.wx[6 * i + m];
        for (int m = 0; m < 5; ++m) X(X_VISX + m)[i] = (float)d.visx[5 * i + m];
        float vb[7] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (i >= 1 && i + 1 < w.xarr) {
            // the background's viscous force density, linear in (nr1, dndx, dndy): the
            // reference's stencil with v_r0, v_phi0 axisymmetric (all d/dphi terms vanish)
            const double* Xr = d.visx + 5 * i;
            const double i_r20 = Xr[0], i_r21 = Xr[1], i_r10 = Xr[2], i_hr20 = Xr[3], i_r1 = Xr[4];
            const double u0 = d.initx[5 * (i - 1) + 2], u1 = I[2], u2 = d.initx[5 * (i + 1) + 2];
            const double v0 = d.initx[5 * (i - 1) + 3], v1 = I[3], v2 = d.initx[5 * (i + 1) + 3];
            const double dudx = (u2 - u0) * i_r20;
            const double d2udx2 = ((u2 - u1) * i_r21 - (u1 - u0) * i_r10) * i_hr20;
            const double dvdx = (v2 - v0) * i_r20;
            const double d2vdx2 = ((v2 - v1) * i_r21 - (v1 - v0) * i_r10) * i_hr20;
            vb[0] = (float)(2.0 * d2udx2 + 2.0 * dudx * i_r1 - 2.0 * u1 * i_r1 * i_r1);
            vb[1] = (float)(2.0 * dudx);
            vb[2] = (float)(dvdx - v1 * i_r1);
            vb[3] = (float)(d2vdx2 - dvdx * i_r1 + v1 * i_r1 * i_r1 + 2.0 * (dvdx - v1 * i_r1) * i_r1);
            vb[4] = (float)(dvdx - v1 * i_r1);
            vb[5] = (float)(2.0 * u1 * i_r1);
            vb[6] = (float)(d.initx[5 * (i + 1)] * d.nux[i + 1] - d.initx[5 * (i - 1)] * d.nux[i - 1]);
        }
        for (int m = 0; m < 7; ++m) X(X_VBG + m)[i] = vb[m];
        if (d.initd) {
            const double* D = d.initd + 4 * i;
            X(X_DSBG)[i] = (float)D[0];
            X(X_DUBG)[i] = (float)D[1];
            X(X_DVBG)[i] = (float)D[2];
            X(X_DEPS)[i] = (float)(D[2] - d.radx[i] * d.frame_omega - d.rot[i]);
            X(X_DABG)[i] = (float)(D[2] * D[2] * d.irad[i] + d.gstar[i]);
            X(X_DV2R)[i] = (float)(2.0 * D[2] * d.irad[i]);
            X(X_DGU)[i] = (float)(I[2] - D[1]);
            X(X_DGV)[i] = (float)(I[3] - D[2]);
            for (int kk = 0; kk < 4; ++kk) {
                const int ik = min(max(i + offs[kk], 0), w.xarr - 1);
                const double* E = d.initd + 4 * ik;
                X(X_DDBG + kk)[i] = (float)(E[0] - D[0]);
                X(X_DDBG + 4 + kk)[i] = (float)(E[1] - D[1]);
                X(X_DDBG + 8 + kk)[i] = (float)(d.radx[ik] * E[2] - d.radx[i] * D[2]);
            }
        }
        const double* kt = d.killx + 4 * i;
        X(X_KILL + 0)[i] = (float)kt[0];
        X(X_KILL + 1)[i] = kt[1] > 0.0 ? (float)(1.0 / kt[1]) : 0.0f;
        X(X_KILL + 2)[i] = (float)kt[2];
        X(X_KILL + 3)[i] = kt[3] > 0.0 ? (float)(1.0 / kt[3]) : 0.0f;
    }
    if (k < w.yarr) {
        Y(Y_IDY)[k] = (float)d.idx_y[k];
        Y(Y_IYV)[k] = (float)d.iyv[k];
        for (int m = 0; m < 6; ++m) Y(Y_WY + m)[k] = (float)d.wy[6 * k + m];
        for (int m = 0; m < 4; ++m) Y(Y_VISY + m)[k] = (float)d.visy[4 * k + m];
    }
}

// ============================================================== launchers
static inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

static unsigned persistent_grid(const void* kernel, int threads, size_t smem, long long ntiles, int cap = 0) {
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm <= 0) nsm = 148;
    }
    static const void* keys[16] = {nullptr};
    static int vals[16] = {0};
    int per_sm = 0;
    for (int n = 0; n < 16 && keys[n]; ++n)
        if (keys[n] == kernel) per_sm = vals[n];
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        for (int n = 0; n < 16; ++n)
            if (!keys[n]) {
                keys[n] = kernel;
                vals[n] = per_sm;
                break;
            }
    }
    if (cap > 0 && cap < per_sm) per_sm = cap;
    long long g = (long long)per_sm * nsm;
    if (g > ntiles) g = ntiles;
    return (unsigned)(g < 1 ? 1 : g);
}

// The two compiled occupancies of each pass (kick1, sweep x, sweep y, advect,
// kick2): variant 0 is the one the register count allows by itself, variant 1
// one CTA per SM more (fewer registers, possibly spills).
constexpr int MB32[5][2] = {{4, 5}, {3, 4}, {4, 5}, {5, 6}, {4, 5}};

template <int P, int V>
static const void* pass_kernel() {
    constexpr int MB = MB32[P][V];
    if constexpr (P == 0) return (const void*)k32_kick1<MB>;
    else if constexpr (P == 1) return (const void*)k32_sweep_x<MB>;
    else if constexpr (P == 2) return (const void*)k32_sweep_y<MB>;
    else if constexpr (P == 3) return (const void*)k32_advect<MB>;
    else return (const void*)k32_kick2<MB>;
}
static const void* pass_kernel(int pass, int v) {
    static const void* const k[5][2] = {{pass_kernel<0, 0>(), pass_kernel<0, 1>()},
                                        {pass_kernel<1, 0>(), pass_kernel<1, 1>()},
                                        {pass_kernel<2, 0>(), pass_kernel<2, 1>()},
                                        {pass_kernel<3, 0>(), pass_kernel<3, 1>()},
                                        {pass_kernel<4, 0>(), pass_kernel<4, 1>()}};
    return k[pass][v ? 1 : 0];
}
static const int PASS_THREADS[5] = {STT, SWT, SWT, SWT, STT};
static const size_t PASS_SMEM[5] = {K1_SMEM, SX_SMEM, SY_SMEM, AD_SMEM, K2_SMEM};

int pass_occupancy32(int pass, int variant) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass_kernel(pass, variant), PASS_THREADS[pass],
                                                      PASS_SMEM[pass]) != cudaSuccess)
        return 1;
    return per_sm < 1 ? 1 : per_sm;
}

cudaError_t set_attributes32() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f, size_t bytes) {
        cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (r != cudaSuccess) e = r;
        r = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (r != cudaSuccess) e = r;
    };
    for (int p = 0; p < 5; ++p)
        for (int v = 0; v < 2; ++v) set(pass_kernel(p, v), PASS_SMEM[p]);
    return e;
}

void launch_time32(const View32* V, int nd, cudaStream_t s) { k32_time<<<cdiv(nd, 64), 64, 0, s>>>(V, nd); }
void launch_trig32(const View32* V, int nd, int maxn, cudaStream_t s) {
    k32_trig<<<dim3(cdiv(maxn, 128), nd), 128, 0, s>>>(V);
}
template <int P, int V>
static void launch_variant(const View32* V_, const int4* first, int nd, int nt, int in, int cap, cudaStream_t s) {
    constexpr int MB = MB32[P][V];
    const unsigned g = persistent_grid(pass_kernel<P, V>(), PASS_THREADS[P], PASS_SMEM[P], nt, cap);
    if constexpr (P == 0) k32_kick1<MB><<<g, STT, K1_SMEM, s>>>(V_, first, nd, nt, in);
    else if constexpr (P == 1) k32_sweep_x<MB><<<g, SWT, SX_SMEM, s>>>(V_, first, nd, nt, in);
    else if constexpr (P == 2) k32_sweep_y<MB><<<g, SWT, SY_SMEM, s>>>(V_, first, nd, nt, in);
    else if constexpr (P == 3) k32_advect<MB><<<g, SWT, AD_SMEM, s>>>(V_, first, nd, nt, in);
    else k32_kick2<MB><<<g, STT, K2_SMEM, s>>>(V_, first, nd, nt, in);
}
template <int P>
static void launch_p(const View32* V, const int4* first, int nd, int nt, int in, const Tune32* t, cudaStream_t s) {
    const int v = t ? t->v[P] : DEFAULT_TUNE32.v[P];
    const int cap = t ? t->cps[P] : 0;
    if (v) launch_variant<P, 1>(V, first, nd, nt, in, cap, s);
    else launch_variant<P, 0>(V, first, nd, nt, in, cap, s);
}
// tiles: the ensemble's tile table, radial-sweep tiles, then azimuthal, then stencil
void launch_pass32(int pass, const View32* V, const int4* tiles, int nd, const int* ntiles, int in, cudaStream_t s,
                   const Tune32* t) {
    const int4* tx = tiles;
    const int4* ty = tiles + ntiles[0];
    const int4* ts = tiles + ntiles[0] + ntiles[1];
    switch (pass) {
        case 0: launch_p<0>(V, ts, nd, ntiles[2], in, t, s); break;
        case 1: launch_p<1>(V, tx, nd, ntiles[0], in, t, s); break;
        case 2: launch_p<2>(V, ty, nd, ntiles[1], in, t, s); break;
        case 3: launch_p<3>(V, ty, nd, ntiles[1], in, t, s); break;
        default: launch_p<4>(V, ts, nd, ntiles[2], in, t, s); break;
    }
}
void launch_cfl32(const View32* Vk, int b, cudaStream_t s) { k32_cfl<<<592, 256, 0, s>>>(Vk, b); }
// the dust part of pass 1 (radial sweep), 2 (azimuthal sweep), 3 (advection);
// counts: radial faces, azimuthal faces, cells of all dust disks
void launch_dust_pass32(int pass, const View32* V, const int* doff, int nd, const long long* counts, int in,
                        cudaStream_t s) {
    auto grid = [](long long n) { return (unsigned)((n + 255) / 256); };
    if (counts[2] == 0) return;
    if (pass == 1) {
        k32d_faces<0><<<grid(counts[0]), 256, 0, s>>>(V, doff, nd, in);
        k32d_update<0><<<grid(counts[2]), 256, 0, s>>>(V, doff, nd, in);
    } else if (pass == 2) {
        k32d_faces<1><<<grid(counts[1]), 256, 0, s>>>(V, doff, nd, in);
        k32d_update<1><<<grid(counts[2]), 256, 0, s>>>(V, doff, nd, in);
    } else if (pass == 3) {
        k32d_adv_faces<<<grid(counts[1]), 256, 0, s>>>(V, doff, nd, in);
        k32d_adv_update<<<grid(counts[2]), 256, 0, s>>>(V, doff, nd, in);
    }
}
void launch_dfill32(const View32* Vk, int b, const double* r, const double* u, const double* v, cudaStream_t s) {
    k32_dfill<<<592, 256, 0, s>>>(Vk, b, r, u, v);
}
void launch_dextract32(const View32* Vk, int b, double* r, double* u, double* v, cudaStream_t s) {
    k32_dextract<<<592, 256, 0, s>>>(Vk, b, r, u, v);
}
void launch_fill32(const View32* Vk, int b, const double* r, const double* u, const double* v, cudaStream_t s) {
    k32_fill<<<1184, 256, 0, s>>>(Vk, b, r, u, v);
}
void launch_extract32(const View32* Vk, int b, double* r, double* p, double* u, double* v, cudaStream_t s) {
    k32_extract<<<1184, 256, 0, s>>>(Vk, b, r, p, u, v);
}
void launch_totals32(const View32* Vk, int b, double* part, int nblocks, cudaStream_t s) {
    k32_totals<<<nblocks, 256, 0, s>>>(Vk, b, part);
}
void launch_torque32(const View32* Vk, int b, double* part, int nblocks, cudaStream_t s) {
    k32_torque<<<nblocks, 256, 0, s>>>(Vk, b, part);
}
void launch_init_tables32(const View32& w, float* tx, float* ty, double* cs64, cudaStream_t s) {
    const int n = w.xarr > w.yarr ? w.xarr : w.yarr;
    k32_init_tables<<<cdiv(n, 128), 128, 0, s>>>(w, tx, ty, cs64);
}

}  // namespace f32
}  // namespace pg
