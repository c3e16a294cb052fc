// pg_ens_*: ensembles of 2D planet-disks advanced by the FP32-mixed step, one
// persistent launch per pass for all disks, the whole step captured in a CUDA
// graph.  Each disk keeps its own clock, dt (CFL of its own state), planet and
// error word in its FP64 device scalars; a single disk is an ensemble of one.
//
// The reference runs one compile-time configured disk per process
// (include/parameters.h); an ensemble has no counterpart there.  Per disk the
// step is main.cu:322-347 (global_dt, solve) with the FP32-mixed arithmetic of
// pg_f32.cuh.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pg_common.cuh"
#include "pg_f32.cuh"
#include "pg_internal.h"

using namespace pg;
using namespace pg::f32;

namespace {

pg_status ens_fail(pg_status s, const std::string& m) {
    set_last_error(m.c_str());
    return s;
}

#define ENS_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return ens_fail(PG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline int cdivi(int a, int b) { return (a + b - 1) / b; }

constexpr int kPasses = 5;       // kick1, radial sweep, azimuthal sweep, advection, kick2
constexpr int kTotalsBlocks = 296;

// The FP32 form covers the planet-disk family: polar, isothermal, analytic radial
// boundaries, orbital advection.  Everything else stays on the FP64 path.
pg_status check32(const pg_params* P, int k) {
    pg_status s = pg_check_params(P);
    if (s != PG_OK) return s;
    const std::string pre = "disk " + std::to_string(k) + ": the FP32 form needs ";
    if (P->ndim != 2) return ens_fail(PG_ERR_CONFIG, pre + "ndim 2");
    if (P->geomx != 1 || P->geomy != 3) return ens_fail(PG_ERR_CONFIG, pre + "a polar grid (geomx 1, geomy 3)");
    if (P->eos_flag != 0) return ens_fail(PG_ERR_CONFIG, pre + "the isothermal EOS (EOS_flag 0)");
    if (P->cool_flag != 0) return ens_fail(PG_ERR_CONFIG, pre + "no cooling (cool_flag 0)");
    if (P->twobd_flag != 0) return ens_fail(PG_ERR_CONFIG, pre + "a fixed star (twobd_flag 0)");
    if (P->bound_lft != 0 || P->bound_rgh != 0)
        return ens_fail(PG_ERR_CONFIG, pre + "analytic radial boundaries (bound 0)");
    if (!P->orbadv_flag) return ens_fail(PG_ERR_CONFIG, pre + "orbital advection (OrbAdv_flag 1)");
    if (P->init_flag != 2) return ens_fail(PG_ERR_CONFIG, pre + "the disk initial state (init_flag 2)");
    if (P->xres < 64 || P->yres < 64) return ens_fail(PG_ERR_CONFIG, pre + "xres and yres of at least 64");
    return PG_OK;
}

struct EDisk {
    Engine* E = nullptr;
    float* buf = nullptr;  // two buffers of NPL planes
    float* vis = nullptr;
    float* tab = nullptr;
    float* trig = nullptr;
    double* cs64 = nullptr;
    float* dbuf = nullptr;   // dust_flag: two buffers of NPL residual planes
    float* dflux = nullptr;  // dust face fluxes
    bool fresh = true;
    View32 v{};
};

}  // namespace

struct pg_ens {
    int n = 0, device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<EDisk> disks;
    View32* dV = nullptr;
    int* dFirst = nullptr;
    int4* dTiles = nullptr;             // per tile of each kind: {disk, origin along the fast index, along the slow}
    CUtensorMap* dMaps = nullptr;
    double* dPart = nullptr;
    int ntiles[3] = {0, 0, 0};
    int* dDoff = nullptr;               // [3][n + 1] running counts of dust faces and cells
    long long dcount[3] = {0, 0, 0};    // radial faces, azimuthal faces, cells of all dust disks
    int maxn = 0;
    int cur = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    Tune32 tune = DEFAULT_TUNE32;  // launch configuration of the passes (pg_ens_autotune)
    double* xfer = nullptr;        // device staging of host exchanges, kept between calls
    size_t xfer_n = 0;

    ~pg_ens() {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& D : disks) {
            cudaFree(D.buf);
            cudaFree(D.vis);
            cudaFree(D.tab);
            cudaFree(D.trig);
            cudaFree(D.cs64);
            cudaFree(D.dbuf);
            cudaFree(D.dflux);
            if (D.E) engine_destroy(D.E);
        }
        cudaFree(dV);
        cudaFree(dFirst);
        cudaFree(dTiles);
        cudaFree(dMaps);
        cudaFree(dPart);
        cudaFree(dDoff);
        cudaFree(xfer);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Device staging for a member's state or dust on its way to or from the host
// (up to 4 interior planes of the largest member), allocated on first use and
// kept: exchanges allocate nothing.  All users run on e->stream; a larger
// request waits for the stream before replacing the buffer.
pg_status xfer_buffer(pg_ens* e, size_t count, double** out);

// Kernels of one step reading buffer `in`: clocks, planet tables, five passes.
pg_status enqueue_step(pg_ens* e, int in) {
    launch_time32(e->dV, e->n, e->stream);
    launch_trig32(e->dV, e->n, e->maxn, e->stream);
    for (int p = 0; p < kPasses; ++p) {
        launch_pass32(p, e->dV, e->dTiles, e->n, e->ntiles, in ^ (p & 1), e->stream, &e->tune);
        launch_dust_pass32(p, e->dV, e->dDoff, e->n, e->dcount, in ^ (p & 1), e->stream);
    }
    ENS_CUDA(cudaGetLastError());
    return PG_OK;
}

pg_status read_scalars(pg_ens* e, int k, Scalars* h) {
    ENS_CUDA(cudaMemcpyAsync(h, e->disks[k].v.d64.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    return PG_OK;
}

// main.cu:144 + 322: after a (re)start the first dt cap is end_time - t.
pg_status arm_clocks(pg_ens* e, double end_time) {
    for (int k = 0; k < e->n; ++k) {
        EDisk& D = e->disks[k];
        Scalars h{};
        pg_status s = read_scalars(e, k, &h);
        if (s != PG_OK) return s;
        if (D.fresh) h.dt_prev = end_time - h.t;
        h.end_time = end_time;
        h.done = 0;
        h.pad_ = 0;
        ENS_CUDA(cudaMemcpyAsync(D.v.d64.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, e->stream));
        ENS_CUDA(cudaStreamSynchronize(e->stream));
        D.fresh = false;
    }
    return PG_OK;
}

pg_status check_index(const pg_ens* e, int k) {
    if (!e) return ens_fail(PG_ERR_ARG, "null ensemble");
    if (k < 0 || k >= e->n) return ens_fail(PG_ERR_ARG, "disk index out of range");
    return PG_OK;
}

pg_status xfer_buffer(pg_ens* e, size_t count, double** out) {
    if (e->xfer_n < count) {
        ENS_CUDA(cudaStreamSynchronize(e->stream));
        cudaFree(e->xfer);
        e->xfer = nullptr;
        e->xfer_n = 0;
        ENS_CUDA(cudaMalloc(&e->xfer, count * sizeof(double)));
        e->xfer_n = count;
    }
    *out = e->xfer;
    return PG_OK;
}

}  // namespace

extern "C" {

pg_status pg_ens_check_params(const pg_params* P, int n) {
    if (!P || n <= 0) return ens_fail(PG_ERR_ARG, "pg_ens_check_params: need n >= 1 parameter sets");
    for (int k = 0; k < n; ++k) {
        pg_status s = check32(&P[k], k);
        if (s != PG_OK) return s;
    }
    return PG_OK;
}

pg_status pg_ens_create(const pg_params* P, int n, int device, void* stream, pg_ens** out) {
    if (!out) return ens_fail(PG_ERR_ARG, "null out");
    *out = nullptr;
    pg_status s = pg_ens_check_params(P, n);
    if (s != PG_OK) return s;
    ENS_CUDA(cudaSetDevice(device));
    static std::once_flag attrs;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attrs, [] { attr_err = set_attributes32(); });
    ENS_CUDA(attr_err);
    pg_ens* e = new pg_ens();
    auto bail = [&](pg_status st) {
        delete e;
        return st;
    };
    e->n = n;
    e->device = device;
    if (stream) e->stream = (cudaStream_t)stream;
    else {
        cudaError_t ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) return bail(ens_fail(PG_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(ce)));
        e->own_stream = true;
    }
    e->disks.resize(n);
    std::vector<int> first(3 * (n + 1), 0);
    cudaError_t ce;
    if ((ce = cudaMalloc(&e->dMaps, sizeof(CUtensorMap) * 7 * (size_t)n)) != cudaSuccess ||
        (ce = cudaMalloc(&e->dV, sizeof(View32) * (size_t)n)) != cudaSuccess ||
        (ce = cudaMalloc(&e->dFirst, sizeof(int) * first.size())) != cudaSuccess ||
        (ce = cudaMalloc(&e->dPart, sizeof(double) * 2 * kTotalsBlocks)) != cudaSuccess)
        return bail(ens_fail(PG_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(ce)));
    std::vector<CUtensorMap> maps(7 * (size_t)n);
    std::vector<View32> hv(n);
    std::vector<int> doff(3 * (n + 1), 0);
    for (int k = 0; k < n; ++k) {
        EDisk& D = e->disks[k];
        if ((s = table_engine_create(&P[k], device, e->stream, &D.E)) != PG_OK) return bail(s);
        const DiskView& d = engine_view(D.E);
        View32& v = D.v;
        v.xres = d.xres;
        v.yres = d.yres;
        v.xarr = d.xarr;
        v.yarr = d.yarr;
        v.pitch = (d.xarr + 3) / 4 * 4;
        v.xn = d.xarr + 1;
        v.yn = d.yarr + 1;
        v.visc = d.visc;
        v.orbadv = d.orbadv;
        v.kill = d.kill;
        v.nplanet = d.nplanet;
        v.ntx[0] = cdivi(d.xres, 32);
        v.ntx[1] = cdivi(d.yres, 32);
        v.ntx[2] = cdivi(d.xres, 32);
        v.gam = (float)d.gam;
        const size_t plane = (size_t)v.pitch * v.yarr;
        const size_t ntab = (size_t)X_NSLOT * v.xn + (size_t)Y_NSLOT * v.yn;
        if ((ce = cudaMalloc(&D.buf, sizeof(float) * 2 * NPL * plane)) != cudaSuccess ||
            (ce = cudaMalloc(&D.vis, sizeof(float) * 2 * plane)) != cudaSuccess ||
            (ce = cudaMalloc(&D.tab, sizeof(float) * ntab)) != cudaSuccess ||
            (ce = cudaMalloc(&D.trig, sizeof(float) * trig_floats(v.xn, v.yn))) != cudaSuccess ||
            (ce = cudaMalloc(&D.cs64, sizeof(double) * v.xarr)) != cudaSuccess)
            return bail(ens_fail(PG_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(ce)));
        // zero residuals everywhere: the radial ghosts of boundary 0 keep init_C for good
        cudaMemsetAsync(D.buf, 0, sizeof(float) * 2 * NPL * plane, e->stream);
        cudaMemsetAsync(D.vis, 0, sizeof(float) * 2 * plane, e->stream);
        cudaMemsetAsync(D.trig, 0, sizeof(float) * trig_floats(v.xn, v.yn), e->stream);
        v.buf[0] = D.buf;
        v.buf[1] = D.buf + NPL * plane;
        v.vis = D.vis;
        v.tx = D.tab;
        v.ty = D.tab + (size_t)X_NSLOT * v.xn;
        v.trig = D.trig;
        v.cs64 = D.cs64;
        v.d64 = d;
        v.maps = e->dMaps + 7 * (size_t)k;
        CUtensorMap* m = &maps[7 * (size_t)k];
        for (int b = 0; b < 2; ++b) {
            if ((s = make_map3_f32(&m[3 * b + 0], v.buf[b], v.pitch, v.yarr, NPL, 40, 8, NPL)) != PG_OK ||
                (s = make_map3_f32(&m[3 * b + 1], v.buf[b], v.pitch, v.yarr, NPL, 12, 38, NPL)) != PG_OK ||
                (s = make_map3_f32(&m[3 * b + 2], v.buf[b], v.pitch, v.yarr, NPL, 36, 10, NPL)) != PG_OK)
                return bail(s);
        }
        if ((s = make_map3_f32(&m[6], v.vis, v.pitch, v.yarr, 2, 36, 10, 2)) != PG_OK) return bail(s);
        long long nd3[3] = {0, 0, 0};
        if (P[k].dust_flag) {
            // init_CD everywhere: zero residuals
            const size_t nf = (size_t)(v.xres + 1) * (v.yres + 1);
            if ((ce = cudaMalloc(&D.dbuf, sizeof(float) * 2 * NPL * plane)) != cudaSuccess ||
                (ce = cudaMalloc(&D.dflux, sizeof(float) * 3 * nf)) != cudaSuccess)
                return bail(ens_fail(PG_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(ce)));
            cudaMemsetAsync(D.dbuf, 0, sizeof(float) * 2 * NPL * plane, e->stream);
            cudaMemsetAsync(D.dflux, 0, sizeof(float) * 3 * nf, e->stream);
            v.dbuf[0] = D.dbuf;
            v.dbuf[1] = D.dbuf + NPL * plane;
            v.dflux = D.dflux;
            v.dust = 1;
            v.st_h = (float)(P[k].stokes * P[k].sc_h);
            v.dust_rmin = (float)(P[k].d_g_ratio * SMALLR);
            nd3[0] = (long long)(v.xres + 1) * v.yres;
            nd3[1] = (long long)v.xres * (v.yres + 1);
            nd3[2] = (long long)v.xres * v.yres;
        }
        for (int r = 0; r < 3; ++r) {
            doff[r * (n + 1) + k + 1] = doff[r * (n + 1) + k] + (int)nd3[r];
            e->dcount[r] += nd3[r];
        }
        launch_init_tables32(v, D.tab, D.tab + (size_t)X_NSLOT * v.xn, D.cs64, e->stream);
        first[0 * (n + 1) + k + 1] = first[0 * (n + 1) + k] + v.ntx[0] * cdivi(d.yres, 8);
        first[1 * (n + 1) + k + 1] = first[1 * (n + 1) + k] + v.ntx[1] * cdivi(d.xres, 8);
        first[2 * (n + 1) + k + 1] = first[2 * (n + 1) + k] + v.ntx[2] * cdivi(d.yres, 8);
        e->maxn = std::max(e->maxn, std::max(v.xn, v.yn));
        hv[k] = v;
    }
    for (int p = 0; p < 3; ++p) e->ntiles[p] = first[p * (n + 1) + n];
    // tile table: a tile's disk and origin (32 cells along the fast index x 8
    // along the slow), so the passes need no search over the disks' offsets
    std::vector<int4> tiles;
    tiles.reserve((size_t)e->ntiles[0] + e->ntiles[1] + e->ntiles[2]);
    for (int p = 0; p < 3; ++p)
        for (int k = 0; k < n; ++k) {
            const int ntx = hv[k].ntx[p];
            for (int loc = 0; loc < first[p * (n + 1) + k + 1] - first[p * (n + 1) + k]; ++loc)
                tiles.push_back(make_int4(k, NPAD + 32 * (loc % ntx), NPAD + 8 * (loc / ntx), 0));
        }
    if ((ce = cudaMalloc(&e->dTiles, sizeof(int4) * tiles.size())) != cudaSuccess ||
        (ce = cudaMemcpyAsync(e->dTiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice,
                              e->stream)) != cudaSuccess ||
        (ce = cudaMalloc(&e->dDoff, sizeof(int) * doff.size())) != cudaSuccess ||
        (ce = cudaMemcpyAsync(e->dDoff, doff.data(), sizeof(int) * doff.size(), cudaMemcpyHostToDevice, e->stream)) !=
            cudaSuccess ||
        (ce = cudaMemcpyAsync(e->dMaps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice,
                              e->stream)) != cudaSuccess ||
        (ce = cudaMemcpyAsync(e->dV, hv.data(), sizeof(View32) * hv.size(), cudaMemcpyHostToDevice, e->stream)) !=
            cudaSuccess ||
        (ce = cudaMemcpyAsync(e->dFirst, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice,
                              e->stream)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(e->stream)) != cudaSuccess || (ce = cudaGetLastError()) != cudaSuccess)
        return bail(ens_fail(PG_ERR_CUDA, std::string("ensemble set-up: ") + cudaGetErrorString(ce)));
    *out = e;
    return PG_OK;
}

pg_status pg_ens_destroy(pg_ens* e) {
    if (!e) return PG_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    delete e;
    return PG_OK;
}

int pg_ens_size(const pg_ens* e) { return e ? e->n : 0; }

pg_status pg_ens_dims(const pg_ens* e, int k, int* xres, int* yres) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (xres) *xres = e->disks[k].v.xres;
    if (yres) *yres = e->disks[k].v.yres;
    return PG_OK;
}

pg_status pg_ens_set_state(pg_ens* e, int k, double t, const double* r, const double* u, const double* v) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (!r || !u) return ens_fail(PG_ERR_ARG, "null state array");
    ENS_CUDA(cudaSetDevice(e->device));
    EDisk& D = e->disks[k];
    const size_t n = (size_t)D.v.xres * D.v.yres;
    double* st = nullptr;
    {
        const pg_status sx = xfer_buffer(e, 3 * n, &st);
        if (sx != PG_OK) return sx;
    }
    ENS_CUDA(cudaMemcpyAsync(st, r, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    ENS_CUDA(cudaMemcpyAsync(st + n, u, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    if (v) ENS_CUDA(cudaMemcpyAsync(st + 2 * n, v, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    launch_fill32(e->dV + k, e->cur, st, st + n, v ? st + 2 * n : nullptr, e->stream);
    ENS_CUDA(cudaGetLastError());
    if (D.v.dust)  // a restart's dust is init_CD (the reference's load_grid reads the gas only)
        ENS_CUDA(cudaMemsetAsync(D.v.dbuf[e->cur], 0, sizeof(float) * NPL * (size_t)D.v.pitch * D.v.yarr,
                                 e->stream));
    engine_init_planet(D.E, t);
    ENS_CUDA(cudaMemsetAsync(&D.v.d64.sc->vmax_bits, 0, sizeof(unsigned long long), e->stream));
    launch_cfl32(e->dV + k, e->cur, e->stream);
    ENS_CUDA(cudaGetLastError());
    Scalars h{};
    if ((s = read_scalars(e, k, &h)) != PG_OK) return s;
    h.t = t;
    h.dt = 0.0;
    h.dt_prev = 0.0;
    h.steps = 0;
    h.done = 0;
    h.pad_ = 0;
    h.err = 0;
    h.floor_hits = 0;
    ENS_CUDA(cudaMemcpyAsync(D.v.d64.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    D.fresh = true;
    return PG_OK;
}

pg_status pg_ens_get_state(pg_ens* e, int k, double* r, double* p, double* u, double* v, double* t_out) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (!r || !p || !u || !v) return ens_fail(PG_ERR_ARG, "null state array");
    ENS_CUDA(cudaSetDevice(e->device));
    EDisk& D = e->disks[k];
    const size_t n = (size_t)D.v.xres * D.v.yres;
    double* st = nullptr;
    {
        const pg_status sx = xfer_buffer(e, 4 * n, &st);
        if (sx != PG_OK) return sx;
    }
    launch_extract32(e->dV + k, e->cur, st, st + n, st + 2 * n, st + 3 * n, e->stream);
    ENS_CUDA(cudaGetLastError());
    ENS_CUDA(cudaMemcpyAsync(r, st, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaMemcpyAsync(p, st + n, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaMemcpyAsync(u, st + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaMemcpyAsync(v, st + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    if (t_out) ENS_CUDA(cudaMemcpyAsync(t_out, &D.v.d64.sc->t, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    return PG_OK;
}

pg_status pg_ens_run(pg_ens* e, int nsteps, double end_time) {
    if (!e) return ens_fail(PG_ERR_ARG, "null ensemble");
    if (nsteps <= 0) return PG_OK;
    ENS_CUDA(cudaSetDevice(e->device));
    pg_status s = arm_clocks(e, end_time);
    if (s != PG_OK) return s;
    // with a finite end_time every disk may finish early: poll the done flags
    // every 256 launched steps (finished disks are copied through meanwhile)
    const bool may_finish = end_time < 1.0e29;
    std::vector<int> done(e->n, 0);
    for (int step = 0; step < nsteps; ++step) {
        if (may_finish && step > 0 && step % 256 == 0) {
            for (int k = 0; k < e->n; ++k)
                ENS_CUDA(cudaMemcpyAsync(&done[k], &e->disks[k].v.d64.sc->done, sizeof(int), cudaMemcpyDeviceToHost,
                                         e->stream));
            ENS_CUDA(cudaStreamSynchronize(e->stream));
            bool all = true;
            for (int k = 0; k < e->n; ++k) all = all && done[k];
            if (all) break;
        }
        const int c0 = e->cur;
        if (!e->graph[c0]) {
            cudaGraph_t g;
            ENS_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            pg_status st = enqueue_step(e, c0);
            cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
            if (st != PG_OK) return st;
            ENS_CUDA(ce);
            ENS_CUDA(cudaGraphInstantiate(&e->graph[c0], g, 0));
            cudaGraphDestroy(g);
        }
        ENS_CUDA(cudaGraphLaunch(e->graph[c0], e->stream));
        e->cur = c0 ^ 1;  // five passes: the newest state alternates every step
    }
    return PG_OK;
}

pg_status pg_ens_sync(pg_ens* e) {
    if (!e) return ens_fail(PG_ERR_ARG, "null ensemble");
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    return PG_OK;
}

pg_status pg_ens_clock(pg_ens* e, int k, double* t, double* dt, long long* steps) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    Scalars h{};
    if ((s = read_scalars(e, k, &h)) != PG_OK) return s;
    if (t) *t = h.t;
    if (dt) *dt = h.dt;
    if (steps) *steps = h.steps;
    return PG_OK;
}

pg_status pg_ens_planet(pg_ens* e, int k, pg_body* out) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (!out) return ens_fail(PG_ERR_ARG, "null out");
    Scalars h{};
    if ((s = read_scalars(e, k, &h)) != PG_OK) return s;
    *out = h.planet_next;
    return PG_OK;
}

pg_status pg_ens_check(pg_ens* e) {
    if (!e) return ens_fail(PG_ERR_ARG, "null ensemble");
    int any = 0, bad = -1;
    for (int k = 0; k < e->n; ++k) {
        int err = 0;
        ENS_CUDA(cudaMemcpyAsync(&err, &e->disks[k].v.d64.sc->err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
        ENS_CUDA(cudaStreamSynchronize(e->stream));
        if (err) {
            if (bad < 0) bad = k;
            any |= err;
            ENS_CUDA(cudaMemsetAsync(&e->disks[k].v.d64.sc->err, 0, sizeof(int), e->stream));
        }
    }
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    if (any & (1 << PG_ERR_TIMEOUT))
        return ens_fail(PG_ERR_TIMEOUT, "disk " + std::to_string(bad) + ": a device wait timed out");
    if (any & (1 << PG_ERR_NAN))
        return ens_fail(PG_ERR_NAN, "disk " + std::to_string(bad) + ": non-positive or NaN density produced");
    return PG_OK;
}

pg_status pg_ens_totals(pg_ens* e, int k, double* mass, double* angmom) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    ENS_CUDA(cudaSetDevice(e->device));
    launch_totals32(e->dV + k, e->cur, e->dPart, kTotalsBlocks, e->stream);
    ENS_CUDA(cudaGetLastError());
    std::vector<double> part(2 * kTotalsBlocks);
    ENS_CUDA(cudaMemcpyAsync(part.data(), e->dPart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    double m = 0.0, cm = 0.0, l = 0.0, cl = 0.0;
    for (int b = 0; b < kTotalsBlocks; ++b) {  // compensated, in block order
        double y = part[2 * b] - cm, t = m + y;
        cm = (t - m) - y;
        m = t;
        y = part[2 * b + 1] - cl;
        t = l + y;
        cl = (t - l) - y;
        l = t;
    }
    if (mass) *mass = m;
    if (angmom) *angmom = l;
    return PG_OK;
}

pg_status pg_ens_torque(pg_ens* e, int k, double* torque) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (!torque) return ens_fail(PG_ERR_ARG, "null out");
    ENS_CUDA(cudaSetDevice(e->device));
    launch_torque32(e->dV + k, e->cur, e->dPart, kTotalsBlocks, e->stream);
    ENS_CUDA(cudaGetLastError());
    std::vector<double> part(kTotalsBlocks);
    ENS_CUDA(cudaMemcpyAsync(part.data(), e->dPart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    *torque = compensated_sum(part.data(), kTotalsBlocks);
    return PG_OK;
}

int pg_ens_kernels_per_step(const pg_ens* e) { return e ? 2 + kPasses + (e->dcount[2] > 0 ? 6 : 0) : 0; }

// dust_flag members: the interior dust (absolute r, v_r, v_phi) of the newest state
pg_status pg_ens_set_dust(pg_ens* e, int k, const double* r, const double* u, const double* v) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (!r || !u || !v) return ens_fail(PG_ERR_ARG, "null dust array");
    EDisk& D = e->disks[k];
    if (!D.v.dust) return ens_fail(PG_ERR_CONFIG, "the disk has no dust (dust_flag 0)");
    ENS_CUDA(cudaSetDevice(e->device));
    const size_t n = (size_t)D.v.xres * D.v.yres;
    double* st = nullptr;
    {
        const pg_status sx = xfer_buffer(e, 3 * n, &st);
        if (sx != PG_OK) return sx;
    }
    ENS_CUDA(cudaMemcpyAsync(st, r, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    ENS_CUDA(cudaMemcpyAsync(st + n, u, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    ENS_CUDA(cudaMemcpyAsync(st + 2 * n, v, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    launch_dfill32(e->dV + k, e->cur, st, st + n, st + 2 * n, e->stream);
    ENS_CUDA(cudaMemsetAsync(&D.v.d64.sc->vmax_bits, 0, sizeof(unsigned long long), e->stream));
    launch_cfl32(e->dV + k, e->cur, e->stream);
    ENS_CUDA(cudaGetLastError());
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    return PG_OK;
}

pg_status pg_ens_get_dust(pg_ens* e, int k, double* r, double* u, double* v) {
    pg_status s = check_index(e, k);
    if (s != PG_OK) return s;
    if (!r || !u || !v) return ens_fail(PG_ERR_ARG, "null dust array");
    EDisk& D = e->disks[k];
    if (!D.v.dust) return ens_fail(PG_ERR_CONFIG, "the disk has no dust (dust_flag 0)");
    ENS_CUDA(cudaSetDevice(e->device));
    const size_t n = (size_t)D.v.xres * D.v.yres;
    double* st = nullptr;
    {
        const pg_status sx = xfer_buffer(e, 3 * n, &st);
        if (sx != PG_OK) return sx;
    }
    launch_dextract32(e->dV + k, e->cur, st, st + n, st + 2 * n, e->stream);
    ENS_CUDA(cudaGetLastError());
    ENS_CUDA(cudaMemcpyAsync(r, st, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaMemcpyAsync(u, st + n, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaMemcpyAsync(v, st + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    return PG_OK;
}

pg_status pg_ens_profile(pg_ens* e, int nsteps, double end_time, float* ms, int nslot) {
    if (!e || !ms || nslot < 6) return ens_fail(PG_ERR_ARG, "bad argument");
    ENS_CUDA(cudaSetDevice(e->device));
    for (int k = 0; k < nslot; ++k) ms[k] = 0.0f;
    pg_status s = arm_clocks(e, end_time);
    if (s != PG_OK) return s;
    cudaEvent_t ev[7];
    for (auto& x : ev) ENS_CUDA(cudaEventCreate(&x));
    for (int step = 0; step < nsteps; ++step) {
        const int c0 = e->cur;
        ENS_CUDA(cudaEventRecord(ev[0], e->stream));
        launch_time32(e->dV, e->n, e->stream);
        launch_trig32(e->dV, e->n, e->maxn, e->stream);
        for (int p = 0; p < kPasses; ++p) {
            ENS_CUDA(cudaEventRecord(ev[1 + p], e->stream));
            launch_pass32(p, e->dV, e->dTiles, e->n, e->ntiles, c0 ^ (p & 1), e->stream, &e->tune);
            launch_dust_pass32(p, e->dV, e->dDoff, e->n, e->dcount, c0 ^ (p & 1), e->stream);
        }
        ENS_CUDA(cudaEventRecord(ev[6], e->stream));
        ENS_CUDA(cudaGetLastError());
        e->cur = c0 ^ 1;
        ENS_CUDA(cudaEventSynchronize(ev[6]));
        for (int k = 0; k < 6; ++k) {
            float t = 0.0f;
            ENS_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
            ms[k] += t / (float)nsteps;
        }
    }
    for (auto& x : ev) cudaEventDestroy(x);
    return PG_OK;
}

// For each pass and each compiled occupancy variant, every CTAs-per-SM cap up to
// what the variant allows: the mean time of `reps` launches on the current
// state (read from the current buffer, written to the other, which the next
// step overwrites), and the fastest is kept.  The disks' device scalars (the
// signal-rate maximum the timed kick2 launches raise, floor counters) are saved
// before and restored after.  Results do not depend on the choice: tiles are
// independent and the CFL rate is a maximum.
pg_status pg_ens_autotune(pg_ens* e, int reps, int* out10) {
    if (!e || reps < 1) return ens_fail(PG_ERR_ARG, "bad argument");
    ENS_CUDA(cudaSetDevice(e->device));
    Scalars* saved = nullptr;
    ENS_CUDA(cudaMalloc(&saved, sizeof(Scalars) * (size_t)e->n));
    for (int k = 0; k < e->n; ++k)
        ENS_CUDA(cudaMemcpyAsync(saved + k, e->disks[k].v.d64.sc, sizeof(Scalars), cudaMemcpyDeviceToDevice,
                                 e->stream));
    cudaEvent_t a, b;
    ENS_CUDA(cudaEventCreate(&a));
    ENS_CUDA(cudaEventCreate(&b));
    for (int p = 0; p < kPasses; ++p) {
        float best = -1.0f;
        int bv = e->tune.v[p], bc = e->tune.cps[p];
        for (int v = 0; v < 2; ++v) {
            const int occ = pass_occupancy32(p, v);
            for (int cap = 1; cap <= occ; ++cap) {
                Tune32 t = e->tune;
                t.v[p] = v;
                t.cps[p] = (cap == occ) ? 0 : cap;
                launch_pass32(p, e->dV, e->dTiles, e->n, e->ntiles, e->cur, e->stream, &t);  // warm-up
                ENS_CUDA(cudaEventRecord(a, e->stream));
                for (int r = 0; r < reps; ++r)
                    launch_pass32(p, e->dV, e->dTiles, e->n, e->ntiles, e->cur, e->stream, &t);
                ENS_CUDA(cudaEventRecord(b, e->stream));
                ENS_CUDA(cudaEventSynchronize(b));
                ENS_CUDA(cudaGetLastError());
                float ms = 0.0f;
                ENS_CUDA(cudaEventElapsedTime(&ms, a, b));
                if (best < 0.0f || ms < best) {
                    best = ms;
                    bv = v;
                    bc = t.cps[p];
                }
            }
        }
        e->tune.v[p] = bv;
        e->tune.cps[p] = bc;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (int k = 0; k < e->n; ++k)
        ENS_CUDA(cudaMemcpyAsync(e->disks[k].v.d64.sc, saved + k, sizeof(Scalars), cudaMemcpyDeviceToDevice,
                                 e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    cudaFree(saved);
    for (auto& g : e->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    if (out10)
        for (int p = 0; p < kPasses; ++p) {
            out10[p] = e->tune.v[p];
            out10[5 + p] = e->tune.cps[p];
        }
    return PG_OK;
}

pg_status pg_ens_set_tuning(pg_ens* e, const int* in10) {
    if (!e || !in10) return ens_fail(PG_ERR_ARG, "bad argument");
    for (int p = 0; p < kPasses; ++p) {
        if (in10[p] != 0 && in10[p] != 1) return ens_fail(PG_ERR_ARG, "variant must be 0 or 1");
        if (in10[5 + p] < 0) return ens_fail(PG_ERR_ARG, "CTA cap must be >= 0");
        e->tune.v[p] = in10[p];
        e->tune.cps[p] = in10[5 + p];
    }
    for (auto& g : e->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    return PG_OK;
}

}  // extern "C"
