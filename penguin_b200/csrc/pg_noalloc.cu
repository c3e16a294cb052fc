// pg_global_dt_noalloc: the CFL time step (src/timestep/timestep.cu:18-140)
// for callers that cannot allocate device memory.
//
// Who needs it: code that owns all of a GPU's memory through its own pool or
// arena (a host application or framework that forbids stray cudaMalloc calls,
// or that runs with a fixed, pre-reserved device budget), and code that must not
// trigger an allocation mid-run at all.  pg_grid_global_dt needs per-grid private
// scratch (an accumulator, reciprocal tables) that it cudaMallocs on first use;
// this entry point instead reads the state (and the dust state, when the
// parameters carry dust_flag), the faces and orb_rot the caller already owns and
// keeps its scratch in the file-scope device array below.
//
// The scratch array is PG_NOALLOC_MAX_PARTIALS + 1 doubles (64 KiB + 8 B) per
// GPU; every GPU that loads the library holds it until the process exits.  Each
// call writes one partial maximum per 4096 interior cells and the final step
// size, so it needs no clearing beforehand; grids above
// PG_NOALLOC_MAX_PARTIALS * 4096 cells are rejected.  All calls share the array:
// calls whose kernels overlap on the GPU (different streams, or several host
// threads) race on it.  The array's device address is looked up once per device
// (first call with that device current) and kept; a cudaDeviceReset of that
// device unloads the module, so a process that resets a device must not call
// this entry point on it again.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "pg_common.cuh"
#include "pg_internal.h"

#define PG_NOALLOC_MAX_PARTIALS 8192
#define PG_NOALLOC_CELLS_PER_BLOCK 4096
#define PG_NOALLOC_THREADS 256

static __device__ __align__(256) double pg_noalloc_scratch[PG_NOALLOC_MAX_PARTIALS + 1];

namespace {

std::mutex g_mu;
void* g_scratch[64] = {nullptr};  // device address of pg_noalloc_scratch per device

// one partial per block: max over its cells of the signal rate (timestep.cu:46-77),
// evaluated from the faces the caller owns; with dust the dust speeds bound it
// too (timestep.cu:64-66, 73-75)
__global__ void k_cfl_partial(pg_params P, const pg_cell* __restrict__ C, const pg_dust* __restrict__ CD,
                              const double* __restrict__ xa, const double* __restrict__ ya,
                              const double* __restrict__ rot, double* scratch) {
    const int xarr = P.xres + 2 * pg::NPAD;
    const int ypad = P.ndim > 1 ? pg::NPAD : 0;
    const long long n = (long long)P.xres * P.yres;
    const long long base = (long long)blockIdx.x * PG_NOALLOC_CELLS_PER_BLOCK;
    double tmp = 0.0;
    for (int k = threadIdx.x; k < PG_NOALLOC_CELLS_PER_BLOCK; k += blockDim.x) {
        const long long m = base + k;
        if (m >= n) break;
        const int i = pg::NPAD + (int)(m % P.xres);
        const int j = ypad + (int)(m / P.xres);
        const size_t ind = (size_t)i + (size_t)xarr * j;
        const pg_cell c = C[ind];
        const double rad_cyl = (P.geomy == 3) ? 0.5 * (xa[i + 1] + xa[i]) : 1.0;
        const double cs = sqrt(P.gam * c.p / c.r);
        double spd = fabs(c.u) + cs;
        if (CD) spd = fmax(fabs(CD[ind].u), spd);
        double wid = fabs(xa[i + 1] - xa[i]);
        tmp = fmax(spd / wid, tmp);
        if (P.ndim > 1) {
            const double rot_i = rot ? rot[i] : 0.0;
            spd = fabs(c.v - rad_cyl * P.frame_omega - rot_i) + cs;
            if (CD) spd = fmax(fabs(CD[ind].v - rad_cyl * P.frame_omega - rot_i), spd);
            wid = fabs(ya[j + 1] - ya[j]) * rad_cyl;
            tmp = fmax(spd / wid, tmp);
        }
    }
    __shared__ double red[PG_NOALLOC_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) tmp = fmax(tmp, __shfl_xor_sync(0xffffffffu, tmp, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tmp;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < PG_NOALLOC_THREADS / 32; ++w) m = fmax(m, red[w]);
        scratch[blockIdx.x] = m;
    }
}

// max of the partials, then CFL / max (timestep.cu:99-111) into the last slot
__global__ void k_cfl_final(double cfl, int nparts, double* scratch) {
    double tmp = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) tmp = fmax(tmp, scratch[k]);
    __shared__ double red[PG_NOALLOC_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) tmp = fmax(tmp, __shfl_xor_sync(0xffffffffu, tmp, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tmp;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < PG_NOALLOC_THREADS / 32; ++w) m = fmax(m, red[w]);
        scratch[PG_NOALLOC_MAX_PARTIALS] = cfl / m;
    }
}

pg_status fail(pg_status s, const char* msg) {
    pg::set_last_error(msg);  // readable through pg_last_error()
    return s;
}

}  // namespace

extern "C" pg_status pg_global_dt_noalloc(const pg_params* P, const pg_cell* C, const pg_dust* CD, const double* xa,
                                          const double* ya, const double* orb_rot, double dt_prev, double* dt_out,
                                          void* stream) {
    if (!P || !C || !xa || !dt_out) return fail(PG_ERR_ARG, "pg_global_dt_noalloc: null argument");
    if (P->ndim != 1 && P->ndim != 2) return fail(PG_ERR_CONFIG, "pg_global_dt_noalloc: ndim must be 1 or 2");
    if (P->ndim == 1 && P->yres != 1)
        return fail(PG_ERR_CONFIG, "pg_global_dt_noalloc: a 1D grid has yres 1");
    if (P->ndim == 2 && !ya) return fail(PG_ERR_ARG, "pg_global_dt_noalloc: a 2D grid needs its faces ya");
    if (P->dust_flag && !CD) return fail(PG_ERR_ARG, "pg_global_dt_noalloc: dust_flag needs the dust state CD");
    if (!P->dust_flag) CD = nullptr;
    const long long n = (long long)P->xres * P->yres;
    const long long nparts = (n + PG_NOALLOC_CELLS_PER_BLOCK - 1) / PG_NOALLOC_CELLS_PER_BLOCK;
    if (n <= 0) return fail(PG_ERR_CONFIG, "pg_global_dt_noalloc: empty grid");
    if (nparts > PG_NOALLOC_MAX_PARTIALS) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "pg_global_dt_noalloc: %lld interior cells exceed the fixed scratch limit of %d cells",
                 n, PG_NOALLOC_MAX_PARTIALS * PG_NOALLOC_CELLS_PER_BLOCK);
        return fail(PG_ERR_CONFIG, buf);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return fail(PG_ERR_CUDA, "pg_global_dt_noalloc: no current device");
    void* scratch = nullptr;
    {
        // set-up, once per device, with that device current: the address of the
        // file-scope array (the array's name is only a host-side stand-in)
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, pg_noalloc_scratch);
            if (e != cudaSuccess) {
                std::string m = std::string("pg_global_dt_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return fail(PG_ERR_CUDA, m.c_str());
            }
            g_scratch[dev] = p;
        }
        scratch = g_scratch[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    k_cfl_partial<<<(unsigned)nparts, PG_NOALLOC_THREADS, 0, s>>>(*P, C, CD, xa, ya, orb_rot,
                                                                   static_cast<double*>(scratch));
    k_cfl_final<<<1, PG_NOALLOC_THREADS, 0, s>>>(P->cfl, (int)nparts, static_cast<double*>(scratch));
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
        std::string m = std::string("pg_global_dt_noalloc: launch: ") + cudaGetErrorString(le);
        return fail(PG_ERR_CUDA, m.c_str());
    }
    double dt = 0.0;
    cudaError_t e = cudaMemcpyAsync(&dt, static_cast<double*>(scratch) + PG_NOALLOC_MAX_PARTIALS, sizeof(double),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        std::string m = std::string("pg_global_dt_noalloc: ") + cudaGetErrorString(e);
        return fail(PG_ERR_CUDA, m.c_str());
    }
    double tmp = dt_prev * 1.1;  // timestep.cu:133-139
    if (dt < tmp) tmp = dt;
    *dt_out = tmp;
    return PG_OK;
}
