// Stage-by-stage driver of the reference's own timestep -- TEST INFRASTRUCTURE.
//
// Linked against the reference's unmodified object files (everything but
// main.o, built by oracle/ref_build.py) and compiled with the same generated
// parameters.h, this program repeats main.cu's set-up (main.cu:154-305,
// restart path) and then runs DS() (src/solver/solve.cu:212-277) and killwave
// one stage at a time, checking for CUDA errors and dumping the whole cell
// array (ghosts included) after every stage, followed by the dust array in
// dust_flag builds (main.cu's dust allocations are repeated).  Used to pin the
// oracle stage by stage and to locate discrepancies.
//
//   stages <restart file> <steps> <dump file> [scrub] [last]
//
// With "last", only the final stage of the last step is written (the state a
// run of that many steps ends with), for grids whose every stage is too large.
//
// With "scrub", a kernel of this driver writes zeros over the dynamic shared
// memory of every SM right before each dust stage: the reference's dust
// reconstruction reads a flattening coefficient from shared memory that it never
// writes under recon_flag 6 (src/solver/recon/PPM.cu:68-77 reached from
// src/solver/dust/dust.cu:105-147 and src/solver/advection/advection.cu:175-233),
// so this shows what it computes when that memory holds zeros.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "structs.h"

double load_grid(Grid*, std::string);
void init(Grid*);
void init_planet(Grid*, double);
void init_OrbAdv(Grid*);
double global_dt(Grid*, Grid*, double);
void boundx(Grid*);
void boundy(Grid*, double);
void apply_source_terms(Grid*, double, double, double);
void apply_source_terms_inplace(Grid*, double, double, double);
void sweepx_inplace(Grid*, double);
void sweepy_inplace(Grid*, double);
#if ndim > 2
void boundz(Grid*);
void sweepz_inplace(Grid*, double);
#endif
void set_OrbAdv(Grid*, double);
void shift_OrbAdv(Grid*);
void advecty(Grid*, double);
void evolve_planet(Grid*, double, double);
void viscosity_tensor_evaluation1(Grid*);
void viscosity_tensor_evaluation2(Grid*);
void killwave(Grid*, double);
#ifdef dust_flag
void boundx_dust(Grid*);
void boundy_dust(Grid*, double);
void sweepx_dust_inplace(Grid*, double);
void sweepy_dust_inplace(Grid*, double);
void advecty_dust(Grid*, double);
static Dust* g_dhost = nullptr;
#endif

static FILE* g_dump = nullptr;
static bool g_scrub = false;
static bool g_last_only = false;  // write only the final stage of the last step
static bool g_final_step = false;

// Zeros the dynamic shared memory of many blocks per SM (diagnostic only).
__global__ void scrub_smem(int nd) {
    extern __shared__ double smem[];
    for (int k = threadIdx.x; k < nd; k += blockDim.x) smem[k] = 0.0;
}
static Cell* g_host = nullptr;
static int g_stage = 0;

static void check(const char* what) {
    cudaError_t e = cudaDeviceSynchronize();
    cudaError_t l = cudaGetLastError();
    if (e != cudaSuccess || l != cudaSuccess) {
        printf("CUDA error after %s: %s / %s\n", what, cudaGetErrorString(e), cudaGetErrorString(l));
        fflush(stdout);
    }
}

static void scrub() {
    if (!g_scrub) return;
    const int bytes = 227 * 1024;  // one block per SM covering (nearly) all of its shared memory
    cudaFuncSetAttribute(scrub_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(scrub_smem, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    scrub_smem<<<148 * 4, 1024, bytes>>>(bytes / 8);
    check("scrub");
}

static void dump(Grid* dev, const char* name, double t, double dt) {
    check(name);
#ifdef kill_flag
    const bool final_stage = std::string(name) == "kill";
#else
    const bool final_stage = std::string(name) == "kick2";
#endif
    if (g_last_only && !(g_final_step && final_stage)) {
        printf("stage %2d %-10s t=%.12f dt=%.6e (not written)\n", g_stage++, name, t, dt);
        return;
    }
    size_t n = (size_t)dev[0].xarr * dev[0].yarr * dev[0].zarr;
    cudaMemcpy(g_host, dev[0].C, n * sizeof(Cell), cudaMemcpyDeviceToHost);
    char tag[32] = {0};
    snprintf(tag, sizeof tag, "%s", name);
    fwrite(tag, 1, 32, g_dump);
    double td[2] = {t, dt};
    fwrite(td, sizeof(double), 2, g_dump);
    fwrite(g_host, sizeof(Cell), n, g_dump);
#ifdef dust_flag
    cudaMemcpy(g_dhost, dev[0].CD, n * sizeof(Dust), cudaMemcpyDeviceToHost);
    fwrite(g_dhost, sizeof(Dust), n, g_dump);
#endif
    int bad = 0;
    for (size_t k = 0; k < n; ++k)
        if (g_host[k].r != g_host[k].r) ++bad;
    printf("stage %2d %-10s t=%.12f dt=%.6e nan_cells=%d\n", g_stage++, name, t, dt, bad);
}

int main(int argc, char** argv) {
    if (argc < 4) {
        printf("usage: %s <restart> <steps> <dump> [scrub] [last]\n", argv[0]);
        return 2;
    }
    int steps = atoi(argv[2]);
    for (int a = 4; a < argc; ++a) {
        if (std::string(argv[a]) == "scrub") g_scrub = true;
        if (std::string(argv[a]) == "last") g_last_only = true;
    }
    g_dump = fopen(argv[3], "wb");
    Grid* hst;
    Grid* dev;
    cudaMallocHost((void**)&hst, sizeof(Grid));
    cudaMallocHost((void**)&dev, sizeof(Grid));
    for (Grid* G : {hst, dev}) {
        G->xres = xres; G->xarr = xres + 2 * xpad; G->xbgn = 0;
        G->yres = yres; G->yarr = yres + 2 * ypad; G->ybgn = 0;
        G->zres = zres; G->zarr = zres + 2 * zpad; G->zbgn = 0;
    }
    size_t n = (size_t)xarr * yarr * zarr;
    cudaMallocHost((void**)&hst->xa, (xarr + 1) * sizeof(double));
    cudaMallocHost((void**)&hst->xv, xarr * sizeof(double));
    cudaMallocHost((void**)&hst->ya, (yarr + 1) * sizeof(double));
    cudaMallocHost((void**)&hst->yv, yarr * sizeof(double));
    cudaMallocHost((void**)&hst->za, (zarr + 1) * sizeof(double));
    cudaMallocHost((void**)&hst->zv, zarr * sizeof(double));
    cudaMallocHost((void**)&hst->C, n * sizeof(Cell));
    cudaMallocHost((void**)&hst->orb_shf, xarr * zarr * sizeof(int));
    cudaMallocHost((void**)&hst->planets, n_planet * sizeof(body));
    cudaMallocHost((void**)&hst->dt, sizeof(double));
    cudaMallocHost((void**)&hst->sum, sizeof(double));
    cudaMallocHost((void**)&g_host, n * sizeof(Cell));
    cudaStreamCreate(&dev->stream);
    cudaMalloc((void**)&dev->xa, (xarr + 1) * sizeof(double));
    cudaMalloc((void**)&dev->xv, xarr * sizeof(double));
    cudaMalloc((void**)&dev->ya, (yarr + 1) * sizeof(double));
    cudaMalloc((void**)&dev->yv, yarr * sizeof(double));
    cudaMalloc((void**)&dev->za, (zarr + 1) * sizeof(double));
    cudaMalloc((void**)&dev->zv, zarr * sizeof(double));
    cudaMalloc((void**)&dev->dt, sizeof(double));
    cudaMalloc((void**)&dev->sum, sizeof(double));
    cudaMalloc((void**)&dev->Buff, n * sizeof(double));
    cudaMalloc((void**)&dev->C, n * sizeof(Cell));
    cudaMalloc((void**)&dev->T, n * sizeof(Cell));
    cudaMalloc((void**)&dev->fx, n * sizeof(double));
    cudaMalloc((void**)&dev->fy, n * sizeof(double));
    cudaMalloc((void**)&dev->fz, n * sizeof(double));
    cudaMalloc((void**)&dev->vis_tensor, ndim * n * sizeof(double));
    cudaMalloc((void**)&dev->BuffL, xpad * yarr * zarr * sizeof(Cell));
    cudaMalloc((void**)&dev->BuffR, xpad * yarr * zarr * sizeof(Cell));
    cudaMalloc((void**)&dev->orb_rot, xarr * zarr * sizeof(double));
    cudaMalloc((void**)&dev->orb_res, xarr * zarr * sizeof(double));
    cudaMalloc((void**)&dev->orb_shf, xarr * zarr * sizeof(int));
    cudaMalloc((void**)&dev->orb_inc, xarr * zarr * sizeof(int));
    cudaMalloc((void**)&dev->shfL, xpad * zres * sizeof(int));
    cudaMalloc((void**)&dev->shfR, xpad * zres * sizeof(int));
    cudaMalloc((void**)&dev->planets, n_planet * sizeof(body));
    cudaMemset(dev->T, 0, n * sizeof(Cell));
#ifdef dust_flag
    cudaMallocHost((void**)&hst->CD, n * sizeof(Dust));
    cudaMallocHost((void**)&g_dhost, n * sizeof(Dust));
    cudaMalloc((void**)&dev->CD, n * sizeof(Dust));
    cudaMalloc((void**)&dev->TD, n * sizeof(Dust));
    cudaMalloc((void**)&dev->BuffLD, xpad * yarr * zarr * sizeof(Dust));
    cudaMalloc((void**)&dev->BuffRD, xpad * yarr * zarr * sizeof(Dust));
    cudaMemset(dev->TD, 0, n * sizeof(Dust));
#endif

    init(hst);
    double t = load_grid(hst, argv[1]);
    init_planet(hst, t);
    cudaMemcpy(dev->xa, hst->xa, (xarr + 1) * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dev->xv, hst->xv, xarr * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dev->ya, hst->ya, (yarr + 1) * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dev->yv, hst->yv, yarr * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dev->za, hst->za, (zarr + 1) * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dev->zv, hst->zv, zarr * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dev->C, hst->C, n * sizeof(Cell), cudaMemcpyHostToDevice);
#ifdef dust_flag
    cudaMemcpy(dev->CD, hst->CD, n * sizeof(Dust), cudaMemcpyHostToDevice);
#endif
    cudaMemcpy(dev->planets, hst->planets, n_planet * sizeof(body), cudaMemcpyHostToDevice);
    init_OrbAdv(dev);
    dump(dev, "start", t, 0.0);

    double dt = end_time - t;
    for (int s = 0; s < steps; ++s) {
        g_final_step = (s == steps - 1);
        dt = global_dt(hst, dev, dt);
        double hdt = 0.5 * dt;
#ifdef visc_flag
        viscosity_tensor_evaluation1(dev);
        dump(dev, "visc1", t, dt);
#endif
        boundx(dev);
#ifdef dust_flag
        boundx_dust(dev);
#endif
        apply_source_terms_inplace(dev, 0.0, 0.0, hdt);
        dump(dev, "kick1", t, dt);
        boundx(dev);
        sweepx_inplace(dev, dt);
        dump(dev, "sweepx", t, dt);
#if ndim > 1
        boundy(dev, t + dt);
        sweepy_inplace(dev, dt);
        dump(dev, "sweepy", t, dt);
#endif
#if ndim > 2
        boundz(dev);
        sweepz_inplace(dev, dt);
        dump(dev, "sweepz", t, dt);
#endif
#ifdef dust_flag
        boundx_dust(dev);
        scrub();
        sweepx_dust_inplace(dev, dt);
        dump(dev, "dsweepx", t, dt);
#if ndim > 1
        boundy_dust(dev, t + dt);
        scrub();
        sweepy_dust_inplace(dev, dt);
        dump(dev, "dsweepy", t, dt);
#endif
#endif
#ifdef OrbAdv_flag
        set_OrbAdv(dev, dt);
        shift_OrbAdv(dev);
        dump(dev, "shift", t, dt);
        advecty(dev, dt);
        dump(dev, "advect", t, dt);
#ifdef dust_flag
        scrub();
        advecty_dust(dev, dt);
        dump(dev, "dadvect", t, dt);
#endif
#endif
        evolve_planet(dev, t + dt, dt);
#ifdef visc_flag
        apply_source_terms(dev, 0.0, hdt, hdt);
        viscosity_tensor_evaluation2(dev);
        apply_source_terms_inplace(dev, 0.0, hdt, hdt);
#else
        apply_source_terms_inplace(dev, 0.0, hdt, hdt);
#endif
        dump(dev, "kick2", t, dt);
#ifdef kill_flag
        killwave(dev, dt);
        dump(dev, "kill", t, dt);
#endif
        t += dt;
    }
    fclose(g_dump);
    return 0;
}
