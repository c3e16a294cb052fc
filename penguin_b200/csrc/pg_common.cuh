// Shared device-side types and helpers of the penguin_b200 kernels (sm_100a).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "penguin_b200.h"

namespace pg {

constexpr int NPAD = 3;  // ghost cells per side (recon_flag 6, include/parameters.h:49-53)
constexpr double PI = 3.1415926535897932384626434;
constexpr double HPI = 0.5 * PI;
constexpr double TWOPI = 2.0 * PI;
constexpr double SMALLR = 1.0e-10;  // include/parameters.h:36-37
constexpr double SMALLP = 1.0e-10;

struct Cell {
    double r, p, u, v, w;
};

// Device scalars of one disk: time, step size, planet and the error word.
struct Scalars {
    double t;          // time at the end of the step being taken (advanced by the step's time kernel)
    double dt;         // current step size
    double dt_prev;    // previous (possibly clipped) step size: the 1.1x growth cap
    double end_time;
    unsigned long long vmax_bits;  // max signal rate of the current state (positive double as ordered bits)
    long long steps;
    int done;          // end_time reached: later steps are no-ops
    int err;           // pg_status bits set by kernels
    int floor_hits;
    int pad_;
    pg_body planet_cur;   // planet used by the first half-kick (from the previous step)
    pg_body planet_next;  // planet at t+dt (src/solver/solve.cu:264)
    double dt_hold;       // the CFL step a clip at end_time replaced (main.cu:333-338 old_dt)
    pg_body star_cur;     // two-body frame (twobd_flag): the star of the first half-kick
    pg_body star_next;    // ... and at t+dt (planets[0] of the reference; the planet is planets[1])
};

// Everything a kernel needs to know about one disk (passed by value).
struct DiskView {
    int xres, yres, xarr, yarr, ypad, ndim;
    int geomx, geomy, eos, ie, bound_lft, bound_rgh;
    int visc, orbadv, kill, nplanet;
    double gam, cfl, frame_omega, dy0;  // dy0 = (ymax-ymin)/yres (src/orbit/orbit.cu:127)
    double planet_mass, ramp_time;      // planet mass ramp (src/planet/planet.cu:7-17)
    // grid (with ghosts)
    const double* xa;
    const double* xv;
    const double* ya;
    const double* yv;
    // per-index tables
    const double* wx;     // 6 reconstruction weights per x index
    const double* wy;     // 6 per y index
    const double* radx;   // xc(i) = 0.5 (xa[i+1] + xa[i])
    const double* ycj;    // yc(j); for ghost rows: yc of the periodic image row
    const double* ycraw;  // yc(j) exactly as the reference computes it for row j
    const double* cs2x;   // get_cs2(xc(i))
    const double* nux;    // get_nu(xc(i))
    const double* initx;  // init_C(xc(i)) (5 per i; the disk's analytic state is axisymmetric)
    const double* killx;  // per i: {ramp_in, tau_in, ramp_out, tau_out} (0 ramp = no damping)
    const double* idx_x;  // 1 / (xa[i+1] - xa[i])
    const double* ixv;    // 1 / xv[i]
    const double* irad;   // 1 / xc(i)
    const double* gstar;  // star gravity -r/|r|^3 at xc(i) (z = 0)
    const double* visx;   // per i: 1/(r[i+1]-r[i-1]), 1/(r[i+1]-r[i]), 1/(r[i]-r[i-1]), 1/(0.5 (r[i+1]-r[i-1])), 1/r[i]
    const double* idx_y;  // 1 / (ya[j+1] - ya[j])
    const double* iyv;    // 1 / yv[j]
    const double* visy;   // per j: 1/(t[j+1]-t[j-1]), 1/(t[j+1]-t[j]), 1/(t[j]-t[j-1]), 1/(0.5 (t[j+1]-t[j-1]))
    double* trig;         // per step, per row: sin, cos of (azimuth - planet y) for planet_cur, then planet_next
    const double* rot;    // orb_rot
    double* res;          // orb_res
    int* inc;             // orb_inc
    Scalars* sc;
    // one pressureless dust fluid (dust_flag, src/solver/dust/dust.cu)
    int dust;
    double stokes, sc_h;  // Stokes number; h/r (stopping time t_s = Stokes h / (c_s Sigma), dust.cu:1-4)
    double dust_rmin;     // D_G_ratio * smallr: the dust density floor of update_Dust (dust.cu:149-176)
    const double* initd;  // init_CD(xc(i)) (4 per i: r, u, v, w; src/init/init.cu:351-454)
    // Newtonian cooling (cool_flag, src/solver/cool/cool.cu)
    int cool;
    double beta_cool;
    const double* coolx;  // cool 1: t_c(xc(i)) = beta_cool r_cyl^1.5
    // two-body frame (twobd_flag, src/planet/planet.cu:135-175): star and planet
    // orbit their barycentre; gravity of both as point masses, no indirect term
    int twobd;
    double* strig;        // per row: sin, cos of (azimuth - star y) for star_cur, then star_next
    // time average of the gas state over a save interval (ave_flag, src/output/output.cu:250-330)
    Cell* ave;            // null: off
    double ave_T;         // the save interval
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------------ TMA
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait on a TMA completion: a tile lands in microseconds, so after 50 ms
// the wait records PG_ERR_TIMEOUT, waits up to another 50 ms for the copy that
// may still be in flight (the CTA must not leave with it pending) and returns
// false so the caller can exit.  A count of polls bounds both loops as well,
// should the timer not advance.
constexpr uint32_t MBAR_MAX_POLLS = 1u << 24;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, Scalars* sc) {
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = globaltimer_ns();
    uint32_t polls = 0;
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > 50000000ull || ++polls > MBAR_MAX_POLLS) {
            atomicOr(&sc->err, 1 << PG_ERR_TIMEOUT);
            t0 = globaltimer_ns();
            polls = 0;
            while (!mbar_try_wait(bar, parity))
                if (globaltimer_ns() - t0 > 50000000ull || ++polls > MBAR_MAX_POLLS) break;
            return false;
        }
    return true;
}
// Dynamic shared memory rounded up to 128 B (TMA destinations); kernels request 128 B extra.
__device__ __forceinline__ double* smem_base128(double* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    return reinterpret_cast<double*>((a + 127) & ~uintptr_t(127));
}
// 2D tiled bulk tensor load global -> shared, completion on an mbarrier.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 3D tiled bulk tensor load global -> shared, completion on an mbarrier.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// --------------------------------------------------------- state writes
__device__ __forceinline__ void store_cell(Cell* out, int xarr, int i, int j, const Cell& c) {
    double* q = reinterpret_cast<double*>(out + (size_t)i + (size_t)xarr * j);
    q[0] = c.r;
    q[1] = c.p;
    q[2] = c.u;
    q[3] = c.v;
    q[4] = c.w;
}

__device__ __forceinline__ void store_row_images(const DiskView& d, Cell* out, int i, int j, const Cell& c) {
    store_cell(out, d.xarr, i, j, c);
    if (d.ndim > 1) {
        // periodic azimuthal ghosts (src/boundary/boundary.cu:141-209, bound_bak/frn 3)
        if (j < 2 * NPAD) store_cell(out, d.xarr, i, j + d.yres, c);
        else if (j >= d.yres) store_cell(out, d.xarr, i, j - d.yres, c);
    }
}

// Writes interior cell (i, j) and every ghost cell that is an image of it, so
// that the ghost zones always hold what the reference's boundx/boundy would put
// there (src/boundary/boundary.cu:13-62 for bound 1/2; bound 0 ghosts hold the
// constant analytic state and are never rewritten).
__device__ __forceinline__ void emit(const DiskView& d, Cell* out, int i, int j, Cell c) {
    store_row_images(d, out, i, j, c);
    const int nx = d.xres + NPAD;
    if (d.bound_lft == 1 && i == NPAD) {
        for (int n = 0; n < NPAD; ++n) store_row_images(d, out, n, j, c);
    } else if (d.bound_lft == 2 && i < 2 * NPAD) {
        Cell m = c;
        m.u = -m.u;
        store_row_images(d, out, 2 * NPAD - 1 - i, j, m);
    }
    if (d.bound_rgh == 1 && i == nx - 1) {
        for (int n = 0; n < NPAD; ++n) store_row_images(d, out, nx + n, j, c);
    } else if (d.bound_rgh == 2 && i >= nx - NPAD) {
        Cell m = c;
        m.u = -m.u;
        store_row_images(d, out, 2 * nx - 1 - i, j, m);
    }
}

__device__ __forceinline__ Cell load_cell(const Cell* in, int xarr, int i, int j) {
    const double* q = reinterpret_cast<const double*>(in + (size_t)i + (size_t)xarr * j);
    Cell c;
    c.r = q[0];
    c.p = q[1];
    c.u = q[2];
    c.v = q[3];
    c.w = q[4];
    return c;
}

// max of positive doubles through their ordered bit patterns
__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
    if (!(v > 0.0)) return;
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

template <int NT>
__device__ __forceinline__ void block_max_to(unsigned long long* dst, double v) {
    __shared__ double red[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = (threadIdx.x < NT / 32) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) atomic_max_pos(dst, v);
    }
}

// TMA pipeline of a persistent CTA with NS stages (NS - 1 tiles in flight while
// one is computed): tile k computes from stage k % NS, barrier k % NS completes
// phase (k / NS) & 1 when tile k has landed.
template <int NS = 2>
__device__ __forceinline__ void pipe_init(uint64_t* bar) {
    if (threadIdx.x == 0) {
        for (int n = 0; n < NS; ++n) mbar_init(&bar[n], 1);
        fence_barrier_init();
    }
    __syncthreads();
}
// thread 0: one box into a stage (the stage's previous generic reads are ordered
// before the async-proxy write by the fence)
__device__ __forceinline__ void issue_box(double* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    tma_load_2d(dst, map, x, y, bar);
}
__device__ __forceinline__ void issue_begin(uint64_t* bar, uint32_t bytes) {
    fence_proxy_async();
    mbar_arrive_expect_tx(bar, bytes);
}
// every thread of the CTA gets the same answer, so a timed-out wait makes the
// whole CTA leave together
template <int NS = 2>
__device__ __forceinline__ bool pipe_wait(uint64_t* bar, int k, Scalars* sc) {
    const bool ok = mbar_wait(&bar[k % NS], (uint32_t)((k / NS) & 1), sc);
    return __syncthreads_and(ok ? 1 : 0) != 0;
}
// after a timed-out wait: before the CTA leaves, wait (again bounded) for the
// copies of tiles k+1 .. k+NS-1 that were issued (issued_ahead of them), so no
// copy lands in released shared memory
template <int NS = 2>
__device__ __forceinline__ void pipe_drain(uint64_t* bar, int k, int issued_ahead, Scalars* sc) {
    if (threadIdx.x == 0)
        for (int m = 1; m <= issued_ahead && m < NS; ++m)
            mbar_wait(&bar[(k + m) % NS], (uint32_t)(((k + m) / NS) & 1), sc);
}

}  // namespace pg
