// Host-side declarations shared by the engine and the kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "pg_common.cuh"

namespace pg {

// Tile variants of the FP64 sweeps and residual advection, the autotuner's knobs
// (pg_disk_autotune): pencils per tile W, outputs per pencil L, cells per thread
// in each phase, TMA stages in flight, and CTAs per SM the registers are
// compiled for (0: as many as ~96 registers a thread allow; more caps the
// registers and may spill).  pg_kernels.cu instantiates each (SV<v>).
struct SweepVariant {
    int w, len, cpt, stages, minb;
};
constexpr int NSWEEP_VARIANTS = 10;
constexpr SweepVariant SWEEP_VARIANTS[NSWEEP_VARIANTS] = {
    {8, 32, 1, 2, 0}, {4, 32, 1, 2, 0}, {16, 16, 1, 2, 0}, {8, 16, 1, 2, 0}, {8, 32, 2, 2, 0},
    {8, 32, 1, 3, 0}, {4, 32, 1, 3, 0}, {4, 64, 1, 2, 0}, {4, 32, 1, 2, 5}, {8, 32, 1, 2, 3}};
// the radial box holds 5 (L + 6) doubles in one row, at most 256 TMA elements
inline bool sweep_variant_x_ok(int v) { return 5 * (SWEEP_VARIANTS[v].len + 2 * NPAD) <= 256; }

// Tensor maps of one AoS cell buffer, one per tile shape.
struct CellMaps {
    const void* base = nullptr;
    CUtensorMap stencil;                   // box {5*34, 10}: 32x8 cells + 1 halo
    CUtensorMap sx[NSWEEP_VARIANTS];       // box {5*(L+6), W}: x-pencils (variants whose box fits)
    CUtensorMap sy[NSWEEP_VARIANTS];       // box {5*(W+2), L+6}: y-pencils, one extra column each side
};
// Launch configuration of the FP64 passes (pg_disk_autotune).
struct Tune {
    int v[3] = {0, 0, 0};          // tile variant of sweep_x, sweep_y, advect (SWEEP_VARIANTS)
    int cps[5] = {0, 0, 0, 0, 0};  // CTAs per SM: kick1, sweep_x, sweep_y, advect, kick2 (0: all that fit)
};
struct VisMaps {
    const void* base = nullptr;
    CUtensorMap stencil;   // box {2*34, 10}
};
// Tensor maps of one AoS dust buffer (4 doubles per cell).
struct DustMaps {
    const void* base = nullptr;
    CUtensorMap sweep_x;   // box {4*38, 8}
    CUtensorMap sweep_y;   // box {4*10, 38}
};

// Pass inputs of one FP64 step, saved for its adjoint (pg_adjoint.cu).
struct StepRecord {
    Cell* stage[5];     // inputs of kick1, sweep_x, sweep_y, advect, kick2 (xarr*yarr AoS each)
    double* vis;        // kick1's viscous force density (2 per cell, xarr*yarr)
    pg_body* planets;   // planet of the first half-kick, planet at t + dt
    double* res;        // orbital-advection residual speed per radius (xarr)
    int* inc;           // orbital-advection shift per radius (xarr)
};

// grid, slope weights and tensor maps (pg_engine.cu)
void make_grid(double* a, double* v, double amin, double amax, int res, int pad, int geom, int grid,
               const pg_params* P);
pg_status recon_weights(int geom, const double* dev_x, int ncell, double* w, cudaStream_t s);
pg_status make_map3_f64(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0,
                        uint32_t b1, uint32_t b2);

// the caller's planets array in and out of the device scalars (pg_engine.cu)
__global__ void k_grid_planet_in(Scalars* sc, const pg_body* planets, int twobd);
__global__ void k_grid_planet_out(const Scalars* sc, pg_body* planets, int twobd);
// the drop-in entry points with ndim 3 (pg_3d.cu)
pg_status check_params3(const pg_params* P);
pg_status grid3_init_orbadv(const pg_params& P, pg_grid* dev);
pg_status grid3_global_dt(const pg_params& P, pg_grid* dev, double dt_prev, double* dt_out);
pg_status grid3_solve(const pg_params& P, pg_grid* dev, double time, double dt);
void grid3_release();

// launch helpers (pg_kernels.cu)
void launch_init_tables(const DiskView& d, const pg_params& P, double* tab_base, cudaStream_t s);
void launch_init_xghosts(const DiskView& d, Cell* buf, cudaStream_t s);
void launch_bound(const DiskView& d, Cell* buf, cudaStream_t s);
void launch_cfl(const DiskView& d, const Cell* buf, cudaStream_t s, const pg_dust* dbuf = nullptr);
void launch_set_time(const DiskView& d, double t, double dt, cudaStream_t s);  // the two below
void launch_set_time_only(const DiskView& d, double t, double dt, cudaStream_t s);
void launch_planet_trig(const DiskView& d, cudaStream_t s);
void launch_time_step(const DiskView& d, cudaStream_t s);
void launch_run_begin(Scalars* sc, double end_time, bool fresh, cudaStream_t s);
void launch_kick1(const DiskView& d, const CellMaps& in, Cell* out, double* vis, cudaStream_t s,
                  const pg_dust* din = nullptr, pg_dust* dout = nullptr, const Tune* t = nullptr);
void launch_sweep_x(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s, const Tune* t = nullptr);
void launch_sweep_y(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s, const Tune* t = nullptr);
void launch_advect(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s, const Tune* t = nullptr);
void launch_kick2(const DiskView& d, const CellMaps& in, const VisMaps& vis, Cell* out, cudaStream_t s,
                  const pg_dust* din = nullptr, pg_dust* dout = nullptr, const Tune* t = nullptr);
int pass_occupancy(const DiskView& d, int pass, int v);
void sweep_variant_launch(int v, int* threads, int* minb);
// the ghost rows of the periodic azimuth take the weights of the rows they image
void periodic_seam_weights(double* wy, int ypad, int yres);
void launch_init_planet(const DiskView& d, const pg_params& P, double t, cudaStream_t s);
void launch_torque(const DiskView& d, const Cell* buf, double* part, int nblocks, cudaStream_t s);
// compensated sum of n doubles in index order
double compensated_sum(const double* a, int n);
int kernels_per_step(const DiskView& d);
void set_last_error(const char* msg);

// tables-only disks and FP32 tensor maps for the FP32 form (pg_engine.cu)
struct Engine;
// FP64 disks driven by the adjoint (pg_engine.cu)
Engine* disk_engine(pg_disk* d);
pg_status engine_set_state_device(Engine* E, double t, const double* r, const double* p, const double* u,
                                  const double* v);
pg_status engine_step(Engine* E, double t, double dt, const StepRecord* rec);
pg_status engine_save(Engine* E, Cell* cells, Scalars* sc);
pg_status engine_restore(Engine* E, const Cell* cells, const Scalars* sc);
// the stream the engine launches on; returns the previous one
cudaStream_t engine_set_stream(Engine* E, cudaStream_t s);
pg_status engine_extract_device(Engine* E, double* r, double* p, double* u, double* v);
pg_status engine_run_pass(Engine* E, int pass, const Cell* in, Cell* out, const double* vis_in, double* vis_out);
pg_status table_engine_create(const pg_params* P, int device, cudaStream_t s, Engine** out);
void engine_destroy(Engine* E);
const DiskView& engine_view(const Engine* E);
void engine_init_planet(Engine* E, double t);
pg_status make_map3_f32(CUtensorMap* m, const float* base, uint64_t pitch, uint64_t rows, uint64_t planes,
                        uint32_t bx, uint32_t by, uint32_t bz);
cudaError_t set_kernel_attributes();

// dust passes (pg_dust.cu)
cudaError_t set_dust_attributes();
void launch_dsweep_x(const DiskView& d, const DustMaps& in, pg_dust* out, cudaStream_t s);
void launch_dsweep_y(const DiskView& d, const DustMaps& in, pg_dust* out, cudaStream_t s);
void launch_dadvect(const DiskView& d, const DustMaps& in, pg_dust* out, cudaStream_t s);
void launch_dust_init(const DiskView& d, pg_dust* buf, cudaStream_t s);
void launch_dust_xghosts(const DiskView& d, pg_dust* buf, cudaStream_t s);
void launch_dust_images(const DiskView& d, pg_dust* buf, cudaStream_t s);
void launch_dust_fill(const DiskView& d, pg_dust* buf, const double* r, const double* u, const double* v,
                      cudaStream_t s);
void launch_dust_extract(const DiskView& d, const pg_dust* buf, double* r, double* u, double* v, cudaStream_t s);


namespace f32 {
struct View32;
// FP32-form launchers (pg_f32.cu); pass 0 kick1, 1 radial sweep, 2 azimuthal sweep,
// 3 advection, 4 kick2, reading buffer `in` and writing the other one
cudaError_t set_attributes32();
void launch_time32(const View32* V, int nd, cudaStream_t s);
void launch_trig32(const View32* V, int nd, int maxn, cudaStream_t s);
// Launch configuration of the five FP32 passes (kick1, sweep x, sweep y, advect,
// kick2): the compiled occupancy variant (0 or 1) and a CTAs-per-SM cap (0 = none).
struct Tune32 {
    int v[5];
    int cps[5];
};
constexpr Tune32 DEFAULT_TUNE32{{0, 1, 0, 0, 1}, {0, 0, 0, 0, 0}};
void launch_pass32(int pass, const View32* V, const int4* tiles, int nd, const int* ntiles, int in, cudaStream_t s,
                   const Tune32* t = nullptr);
int pass_occupancy32(int pass, int variant);
void launch_cfl32(const View32* Vk, int b, cudaStream_t s);
void launch_dust_pass32(int pass, const View32* V, const int* doff, int nd, const long long* counts, int in,
                        cudaStream_t s);
void launch_dfill32(const View32* Vk, int b, const double* r, const double* u, const double* v, cudaStream_t s);
void launch_dextract32(const View32* Vk, int b, double* r, double* u, double* v, cudaStream_t s);
void launch_fill32(const View32* Vk, int b, const double* r, const double* u, const double* v, cudaStream_t s);
void launch_extract32(const View32* Vk, int b, double* r, double* p, double* u, double* v, cudaStream_t s);
void launch_totals32(const View32* Vk, int b, double* part, int nblocks, cudaStream_t s);
void launch_torque32(const View32* Vk, int b, double* part, int nblocks, cudaStream_t s);
void launch_init_tables32(const View32& w, float* tx, float* ty, double* cs64, cudaStream_t s);
}  // namespace f32

}  // namespace pg
