// Host-side declarations shared by the engine and the kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "pg_common.cuh"

namespace pg {

// Tensor maps of one AoS cell buffer, one per tile shape.
struct CellMaps {
    const void* base = nullptr;
    CUtensorMap sweep_x;   // box {5*38, 8}: x-pencils
    CUtensorMap sweep_y;   // box {5*10, 38}: y-pencils (one extra column each side for 16-B alignment)
    CUtensorMap stencil;   // box {5*34, 10}: 32x8 cells + 1 halo
};
struct VisMaps {
    const void* base = nullptr;
    CUtensorMap stencil;   // box {2*34, 10}
};

// launch helpers (pg_kernels.cu)
void launch_init_tables(const DiskView& d, const pg_params& P, double* tab_base, cudaStream_t s);
void launch_init_xghosts(const DiskView& d, Cell* buf, cudaStream_t s);
void launch_bound(const DiskView& d, Cell* buf, cudaStream_t s);
void launch_cfl(const DiskView& d, const Cell* buf, cudaStream_t s);
void launch_set_time(const DiskView& d, double t, double dt, cudaStream_t s);
void launch_time_step(const DiskView& d, cudaStream_t s);
void launch_kick1(const DiskView& d, const CellMaps& in, Cell* out, double* vis, cudaStream_t s);
void launch_sweep_x(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s);
void launch_sweep_y(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s);
void launch_advect(const DiskView& d, const CellMaps& in, Cell* out, cudaStream_t s);
void launch_kick2(const DiskView& d, const CellMaps& in, const VisMaps& vis, Cell* out, cudaStream_t s);
void launch_init_planet(const DiskView& d, const pg_params& P, double t, cudaStream_t s);
int kernels_per_step(const DiskView& d);
void set_last_error(const char* msg);
cudaError_t set_kernel_attributes();

}  // namespace pg
