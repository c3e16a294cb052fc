// Host side of penguin_b200: grid and table construction, tensor maps, step
// orchestration, the CUDA-graph device loop and the C ABI of include/penguin_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pg_common.cuh"
#include "pg_internal.h"

namespace pg {

static thread_local std::string g_err;

static pg_status fail(pg_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

void set_last_error(const char* msg) { g_err = msg; }

double compensated_sum(const double* a, int n) {
    double sum = 0.0, comp = 0.0;
    for (int k = 0; k < n; ++k) {
        const double y = a[k] - comp;
        const double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    return sum;
}

#define PG_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(PG_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ grid
// Power-law stretch of the non-uniform spacings (src/geom/geom.cu:43,65,84).
static double stretch(double dx_max, double dx_min, double L, int N) {
    return std::log(1.0 - (dx_max - dx_min) / (L - (double)N * dx_min)) / std::log(1.0 - 1.0 / (double)N);
}

// Faces a[pad .. pad+res] of one axis (src/geom/geom.cu:22-89): 0 linear,
// 1 logarithmic, 2 fine in the middle, 3 fine towards amax (the midplane),
// 4 fine over the radial extent around the middle.  2-4 read the radial grid's
// xres / xmin / xmax and sc_h of P, as the reference reads its constants.
static void spacing(double* a, double start, double end, int len, int grid, const pg_params* P) {
    if (grid == 1) {
        const double tmp = std::log(end / start);
        for (int i = 0; i < len; i++) a[i] = start * std::exp(tmp * (double)i / (double)(len - 1));
    } else if (grid == 2) {
        const int N = (len - 1) / 2;
        const double L = (end - start) / 2.0;
        const double dx_min = (L / (double)N) / 32.0;
        const double dx_max = (PI - L) / N;
        const double k = stretch(dx_max, dx_min, L, N);
        for (int i = 0; i < N; i++)
            a[i] = (end + start) / 2.0 - (N - i) * dx_min - (L - N * dx_min) * std::pow((double)(N - i) / (double)N, k);
        for (int i = 0; i < N + 1; i++)
            a[N + i] = (end + start) / 2.0 + i * dx_min + (L - N * dx_min) * std::pow((double)i / (double)N, k);
    } else if (grid == 3) {
        const int N = len - 1;
        const double L = end - start;
        const double dx_min = ((P->xmax - P->xmin) / (double)P->xres) / 32.0;
        const double dx_max = P->sc_h / 16.0;
        const double k = stretch(dx_max, dx_min, L, N);
        for (int i = 0; i < N + 1; i++)
            a[i] = end - (N - i) * dx_min - (L - N * dx_min) * std::pow((double)(N - i) / (double)N, k);
    } else if (grid == 4) {
        const int N = P->xres / 2;
        const int N2 = (len - 1 - 2 * N) / 2;
        const double L = (P->xmax - P->xmin) / 2.0;
        const double L2 = (end - start - 2.0 * L) / 2.0;
        const double dx_min = (L / (double)N) / 32.0;
        const double dx_max = L2 / (double)N2;
        const double k = stretch(dx_max, dx_min, L, N);
        for (int i = 0; i < N2; i++) a[i] = start + (double)i * dx_max;
        for (int i = 0; i < N; i++)
            a[i + N2] = (end + start) / 2.0 - (N - i) * dx_min - (L - N * dx_min) * std::pow((double)(N - i) / (double)N, k);
        for (int i = 0; i < N; i++)
            a[i + N2 + N] = (end + start) / 2.0 + i * dx_min + (L - N * dx_min) * std::pow((double)i / (double)N, k);
        for (int i = 0; i < N2 + 1; i++) a[i + N2 + 2 * N] = start + 2.0 * L + L2 + (double)i * dx_max;
    } else {
        for (int i = 0; i < len; i++) a[i] = start + (end - start) * (double)i / (double)(len - 1);
    }
}

// make_grid of src/init/init.cu:472-500: faces with ghosts and cell volumes
// dr * get_dv_dr (src/geom/geom.cu:3-20; geom 5 the polar angle)
void make_grid(double* a, double* v, double amin, double amax, int res, int pad, int geom, int grid,
               const pg_params* P) {
    spacing(&a[pad], amin, amax, res + 1, grid, P);
    for (int i = 0; i < pad; i++) {
        if (grid == 1) {
            a[i] = amin * std::exp(std::log(amax / amin) * (double)(i - pad) / (double)(res));
            a[res + pad + 1 + i] = amin * std::exp(std::log(amax / amin) * (double)(res + 1 + i) / (double)(res));
        } else {
            a[i] = a[pad] - (a[2 * pad - i] - a[pad]);
            a[res + pad + 1 + i] = a[res + pad] + (a[res + pad] - a[res + pad - 1 - i]);
        }
    }
    for (int i = 0; i < res + 2 * pad; i++) {
        const double ra = a[i], dr = a[i + 1] - a[i];
        double dvdr = 1.0;
        if (geom == 5) dvdr = (dr < 1.0e-4) ? std::sin(ra + 0.5 * dr) : (std::cos(ra) - std::cos(ra + dr)) / dr;
        else if (geom == 2) dvdr = ra * ra + ra * dr + dr * dr / 3.0;
        else if (geom == 1) dvdr = ra + dr / 2.0;
        v[i] = dr * dvdr;
    }
}

// ------------------------------------------------- reconstruction weights
// The reference fits, for every cell, the cubic whose (r-weighted for geom 1)
// averages over 4 consecutive cells match the data, and takes the jump between
// the cell average and the cubic at the cell's left / right face as the PPM
// slopes sL / sR (src/solver/recon/recon.cu:216-378, cells i-2..i+1 for sL and
// i-1..i+2 for sR).  Those slopes are linear in the data with coefficients that
// depend only on the grid, so the kernels apply them as 3 weights per slope on
// the differences of neighbouring averages.
//
// The reference evaluates the fit per call from grid moments (B, D below) whose
// differences cancel: on the 1024-cell unit interval a third difference loses
// ~11 of 53 bits, on the azimuthal grid ~20.  The rounded moments are the same
// on every call, so they are a fixed, per-index deviation of the reference's
// effective weights from the exact fit.  k_recon_terms evaluates exactly those
// rounded moments with the reference's expressions (on the device, where the
// compiler contracts them into FMAs as it does the reference's); the host then
// expands the fit's algebra on them in extended precision.  The weights thus
// carry the reference's fixed deviation; what remains is the rounding of its
// per-call arithmetic on the data, which no weight can reproduce.
typedef long double ld;

// grid-only terms of one side of one cell: D02 D12 D22 D03 D04 E1 E2 T N g1 g2 g3
constexpr int kReconTerms = 12;

__global__ void k_recon_terms(const double* __restrict__ x, int ncell, int geom, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 2 || i + 3 > ncell) return;
    // recon.cu:222-301
    const double x0 = x[i - 2], x1 = x[i - 1], x2 = x[i], x3 = x[i + 1], x4 = x[i + 2], x5 = x[i + 3];
    double B02, B12, B22, B32, B42;
    double B03, B13, B23, B33, B43;
    double B04, B14, B24, B34, B44;
    if (geom == 2) {
        B02 = (x1*x1*x1*x1-x0*x0*x0*x0)/(x1*x1*x1-x0*x0*x0)/(4.0/3.0);
        B12 = (x2*x2*x2*x2-x1*x1*x1*x1)/(x2*x2*x2-x1*x1*x1)/(4.0/3.0);
        B22 = (x3*x3*x3*x3-x2*x2*x2*x2)/(x3*x3*x3-x2*x2*x2)/(4.0/3.0);
        B32 = (x4*x4*x4*x4-x3*x3*x3*x3)/(x4*x4*x4-x3*x3*x3)/(4.0/3.0);
        B42 = (x5*x5*x5*x5-x4*x4*x4*x4)/(x5*x5*x5-x4*x4*x4)/(4.0/3.0);
        B03 = (x1*x1*x1*x1*x1-x0*x0*x0*x0*x0)/(x1*x1*x1-x0*x0*x0)/(5.0/3.0);
        B13 = (x2*x2*x2*x2*x2-x1*x1*x1*x1*x1)/(x2*x2*x2-x1*x1*x1)/(5.0/3.0);
        B23 = (x3*x3*x3*x3*x3-x2*x2*x2*x2*x2)/(x3*x3*x3-x2*x2*x2)/(5.0/3.0);
        B33 = (x4*x4*x4*x4*x4-x3*x3*x3*x3*x3)/(x4*x4*x4-x3*x3*x3)/(5.0/3.0);
        B43 = (x5*x5*x5*x5*x5-x4*x4*x4*x4*x4)/(x5*x5*x5-x4*x4*x4)/(5.0/3.0);
        B04 = (x1*x1*x1*x1*x1*x1-x0*x0*x0*x0*x0*x0)/(x1*x1*x1-x0*x0*x0)/2.0;
        B14 = (x2*x2*x2*x2*x2*x2-x1*x1*x1*x1*x1*x1)/(x2*x2*x2-x1*x1*x1)/2.0;
        B24 = (x3*x3*x3*x3*x3*x3-x2*x2*x2*x2*x2*x2)/(x3*x3*x3-x2*x2*x2)/2.0;
        B34 = (x4*x4*x4*x4*x4*x4-x3*x3*x3*x3*x3*x3)/(x4*x4*x4-x3*x3*x3)/2.0;
        B44 = (x5*x5*x5*x5*x5*x5-x4*x4*x4*x4*x4*x4)/(x5*x5*x5-x4*x4*x4)/2.0;
    } else if (geom == 1) {
        B02 = (x1*x1*x1-x0*x0*x0)/(x1*x1-x0*x0)/1.5;
        B12 = (x2*x2*x2-x1*x1*x1)/(x2*x2-x1*x1)/1.5;
        B22 = (x3*x3*x3-x2*x2*x2)/(x3*x3-x2*x2)/1.5;
        B32 = (x4*x4*x4-x3*x3*x3)/(x4*x4-x3*x3)/1.5;
        B42 = (x5*x5*x5-x4*x4*x4)/(x5*x5-x4*x4)/1.5;
        B03 = (x1*x1*x1*x1-x0*x0*x0*x0)/(x1*x1-x0*x0)/2.0;
        B13 = (x2*x2*x2*x2-x1*x1*x1*x1)/(x2*x2-x1*x1)/2.0;
        B23 = (x3*x3*x3*x3-x2*x2*x2*x2)/(x3*x3-x2*x2)/2.0;
        B33 = (x4*x4*x4*x4-x3*x3*x3*x3)/(x4*x4-x3*x3)/2.0;
        B43 = (x5*x5*x5*x5-x4*x4*x4*x4)/(x5*x5-x4*x4)/2.0;
        B04 = (x1*x1*x1*x1*x1-x0*x0*x0*x0*x0)/(x1*x1-x0*x0)/2.5;
        B14 = (x2*x2*x2*x2*x2-x1*x1*x1*x1*x1)/(x2*x2-x1*x1)/2.5;
        B24 = (x3*x3*x3*x3*x3-x2*x2*x2*x2*x2)/(x3*x3-x2*x2)/2.5;
        B34 = (x4*x4*x4*x4*x4-x3*x3*x3*x3*x3)/(x4*x4-x3*x3)/2.5;
        B44 = (x5*x5*x5*x5*x5-x4*x4*x4*x4*x4)/(x5*x5-x4*x4)/2.5;
    } else {
        B02 = (x1*x1-x0*x0)/(x1-x0)/2.0;
        B12 = (x2*x2-x1*x1)/(x2-x1)/2.0;
        B22 = (x3*x3-x2*x2)/(x3-x2)/2.0;
        B32 = (x4*x4-x3*x3)/(x4-x3)/2.0;
        B42 = (x5*x5-x4*x4)/(x5-x4)/2.0;
        B03 = (x1*x1*x1-x0*x0*x0)/(x1-x0)/3.0;
        B13 = (x2*x2*x2-x1*x1*x1)/(x2-x1)/3.0;
        B23 = (x3*x3*x3-x2*x2*x2)/(x3-x2)/3.0;
        B33 = (x4*x4*x4-x3*x3*x3)/(x4-x3)/3.0;
        B43 = (x5*x5*x5-x4*x4*x4)/(x5-x4)/3.0;
        B04 = (x1*x1*x1*x1-x0*x0*x0*x0)/(x1-x0)/4.0;
        B14 = (x2*x2*x2*x2-x1*x1*x1*x1)/(x2-x1)/4.0;
        B24 = (x3*x3*x3*x3-x2*x2*x2*x2)/(x3-x2)/4.0;
        B34 = (x4*x4*x4*x4-x3*x3*x3*x3)/(x4-x3)/4.0;
        B44 = (x5*x5*x5*x5-x4*x4*x4*x4)/(x5-x4)/4.0;
    }
    double* o = out + 2 * kReconTerms * (size_t)i;
    // left face (recon.cu:315-337): moments of cells i-2..i+1
    {
        const double D02 = B12-B02, D12 = B22-B12, D22 = B32-B22;
        const double D03 = B13-B03, D13 = B23-B13, D23 = B33-B23;
        const double D04 = B14-B04, D14 = B24-B14, D24 = B34-B24;
        o[0] = D02; o[1] = D12; o[2] = D22; o[3] = D03; o[4] = D04;
        o[5] = (D23*D02-D03*D22);
        o[6] = (D13*D02 - D03*D12);
        o[7] = (D02*D24 - D22*D04)/(D23*D02-D03*D22) - (D14*D02 - D04*D12)/(D13*D02 - D03*D12);
        o[8] = (D14*D02 - D04*D12);
        o[9] = (B22-x2); o[10] = (B23-x2*x2); o[11] = (B24-x2*x2*x2);
    }
    // right face (recon.cu:341-359): moments of cells i-1..i+2
    {
        const double D02 = B22-B12, D12 = B32-B22, D22 = B42-B32;
        const double D03 = B23-B13, D13 = B33-B23, D23 = B43-B33;
        const double D04 = B24-B14, D14 = B34-B24, D24 = B44-B34;
        o += kReconTerms;
        o[0] = D02; o[1] = D12; o[2] = D22; o[3] = D03; o[4] = D04;
        o[5] = (D23*D02-D03*D22);
        o[6] = (D13*D02 - D03*D12);
        o[7] = (D02*D24 - D22*D04)/(D23*D02-D03*D22) - (D14*D02 - D04*D12)/(D13*D02 - D03*D12);
        o[8] = (D14*D02 - D04*D12);
        o[9] = (x3-B22); o[10] = (x3*x3-B23); o[11] = (x3*x3*x3-B24);
    }
}

// The slope of one side as the reference forms it from the differences
// (d10, d21, d32) of its 4 cells (recon.cu:315-337 / 341-359):
//   c3 = ((D02 d32 - D22 d10)/E1 - (D02 d21 - D12 d10)/E2) / T
//   c2 = (D02 d21 - D12 d10)/E2 - c3 N/E2
//   c1 = d10/D02 - c2 D03/D02 - c3 D04/D02
//   s  = c1 g1 + c2 g2 + c3 g3
// expanded into weights on (d10, d21, d32), in extended precision.
static void side_weights(const double* q, double* w3) {
    const ld D02 = q[0], D12 = q[1], D22 = q[2], D03 = q[3], D04 = q[4];
    const ld E1 = q[5], E2 = q[6], T = q[7], N = q[8], g1 = q[9], g2 = q[10], g3 = q[11];
    for (int k = 0; k < 3; ++k) {
        const ld d10 = (k == 0), d21 = (k == 1), d32 = (k == 2);
        const ld n2 = D02 * d21 - D12 * d10;
        const ld c3 = ((D02 * d32 - D22 * d10) / E1 - n2 / E2) / T;
        const ld c2 = n2 / E2 - c3 * N / E2;
        const ld c1 = d10 / D02 - c2 * D03 / D02 - c3 * D04 / D02;
        w3[k] = (double)(c1 * g1 + c2 * g2 + c3 * g3);
    }
}

// the ghost rows of the periodic azimuth take the weights of the rows they image
// (the adjoint's transposition of the sweep treats the seam as one face)
void periodic_seam_weights(double* wy, int ypad, int yres) {
    for (int k = 1; k <= ypad; ++k)
        for (int m = 0; m < 6; ++m) {
            wy[6 * (ypad - k) + m] = wy[6 * (ypad + yres - k) + m];
            wy[6 * (ypad + yres - 1 + k) + m] = wy[6 * (ypad - 1 + k) + m];
        }
}

// weights of every index of one direction from the device faces x[ncell+1]
pg_status recon_weights(int geom, const double* dev_x, int ncell, double* w, cudaStream_t s) {
    for (int k = 0; k < 6 * ncell; ++k) w[k] = 0.0;
    if (ncell < 6) return PG_OK;  // no cell has the 6 faces of a 4-cell fit (1D tube: y)
    double* terms = nullptr;
    const size_t n = 2 * kReconTerms * (size_t)ncell;
    PG_CUDA(cudaMalloc(&terms, sizeof(double) * n));
    k_recon_terms<<<(ncell + 127) / 128, 128, 0, s>>>(dev_x, ncell, geom, terms);
    cudaError_t e = cudaGetLastError();
    std::vector<double> q(n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.data(), terms, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(terms);
    PG_CUDA(e);
    for (int i = 2; i + 3 <= ncell; ++i) {
        side_weights(&q[2 * kReconTerms * (size_t)i], w + 6 * i);
        side_weights(&q[2 * kReconTerms * (size_t)i + kReconTerms], w + 6 * i + 3);
    }
    return PG_OK;
}

// ------------------------------------------------------------- init_CD
// The dust's initial and bound-0 ghost state, evaluated on the host like the
// reference's fill_grid (src/init/init.cu:502-519) so it carries the same bits:
// init_CD (init.cu:351-454, init_flag 2, 2D) is D_G_ratio Sigma_0, the
// Keplerian azimuthal speed and the radial drift of the steady drag solution,
// refined once from its first-order estimate.  Its drift term takes the
// difference of nearly equal square roots and the gas v_phi a centred
// difference of P over 2.3e-7, so one ulp of pow moves it by ~1e-9.
static void init_cd_table(const pg_params& P, const double* xa, int xarr, double* q) {
    auto cs2 = [&](double x) {
        const double coeff = P.sc_h * P.sc_h * (1.0 / P.planet_radius);
        return P.geomx == 0 ? coeff : coeff * std::pow(x / P.planet_radius, -P.p_beta);
    };
    auto rho = [&](double x) { return std::pow(x / P.planet_radius, -P.p_alpha) * 1.0; };
    auto prs = [&](double x) { return cs2(x) * rho(x); };
    for (int i = 0; i < xarr; ++i) {
        const double x = 0.5 * (xa[i + 1] + xa[i]);
        const double dr = 1.1514178e-7;
        const double dP_dr = (prs(x + dr) - prs(x - dr)) / (2.0 * dr);
        const double v_gas = std::sqrt(1.0 / x + (x / rho(x)) * dP_dr);
        const double st = P.stokes;
        const double f_gas = v_gas / std::sqrt(1.0 / x);
        const double tmp = st * st * f_gas;
        double L = ((1.0 + tmp) / tmp) * (1.0 - std::sqrt(1.0 - 2.0 * tmp * (1.0 - f_gas) / (1.0 + tmp) / (1.0 + tmp)));
        double u0 = st * (L * L - 2.0 * L);
        double u = (1.0 - std::sqrt(1.0 - 2.0 * st * u0)) / st;
        L = (1.0 - f_gas + st * u / 2.0) / (1.0 + st * u / 2.0);
        u0 = st * (L * L - 2.0 * L);
        u = (1.0 - std::sqrt(1.0 - 2.0 * st * u0)) / st;
        q[4 * i + 0] = P.d_g_ratio * std::pow(x / P.planet_radius, -P.p_alpha);
        q[4 * i + 1] = u * std::sqrt(1.0 / x);
        q[4 * i + 2] = std::sqrt(1.0 / x);
        q[4 * i + 3] = 0.0;
    }
}

// ----------------------------------------------------------- tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

static pg_status make_map(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint32_t box_inner,
                          uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return fail(PG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (reinterpret_cast<uintptr_t>(base) % 16 != 0 || (inner * 8) % 16 != 0)
        return fail(PG_ERR_CONFIG, "state rows must be 16-byte aligned (even xres)");
    cuuint64_t dims[2] = {inner, rows};
    cuuint64_t strides[1] = {inner * 8};
    cuuint32_t box[2] = {box_inner, box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PG_OK;
}

// A 3D FP64 tensor map: dims {d0, d1, d2} elements (d0 innermost, contiguous),
// box {b0, b1, b2}.
pg_status make_map3_f64(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0,
                        uint32_t b1, uint32_t b2) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return fail(PG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (reinterpret_cast<uintptr_t>(base) % 16 != 0 || (d0 * 8) % 16 != 0)
        return fail(PG_ERR_CONFIG, "state rows must be 16-byte aligned (even xres)");
    cuuint64_t dims[3] = {d0, d1, d2};
    cuuint64_t strides[2] = {d0 * 8, d0 * d1 * 8};
    cuuint32_t box[3] = {b0, b1, b2};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PG_OK;
}

static pg_status make_cell_maps(CellMaps& M, const Cell* buf, int xarr, int yarr) {
    if (M.base == buf) return PG_OK;
    pg_status s;
    if ((s = make_map(&M.stencil, buf, 5ull * xarr, yarr, 5 * 34, 10)) != PG_OK) return s;
    for (int v = 0; v < NSWEEP_VARIANTS; ++v) {
        const SweepVariant& g = SWEEP_VARIANTS[v];
        const uint32_t tl = (uint32_t)(g.len + 2 * NPAD);
        if (sweep_variant_x_ok(v)) {
            if ((s = make_map(&M.sx[v], buf, 5ull * xarr, yarr, 5 * tl, (uint32_t)g.w)) != PG_OK) return s;
        } else {
            memset(&M.sx[v], 0, sizeof(CUtensorMap));
        }
        if ((s = make_map(&M.sy[v], buf, 5ull * xarr, yarr, 5 * (uint32_t)(g.w + 2), tl)) != PG_OK) return s;
    }
    M.base = buf;
    return PG_OK;
}

static pg_status make_dust_maps(DustMaps& M, const pg_dust* buf, int xarr, int yarr) {
    if (M.base == buf) return PG_OK;
    pg_status s;
    if ((s = make_map(&M.sweep_x, buf, 4ull * xarr, yarr, 4 * 38, 8)) != PG_OK) return s;
    if ((s = make_map(&M.sweep_y, buf, 4ull * xarr, yarr, 4 * 10, 38)) != PG_OK) return s;
    M.base = buf;
    return PG_OK;
}

static pg_status make_vis_maps(VisMaps& M, const double* vis, int xarr, int yarr) {
    if (M.base == vis) return PG_OK;
    pg_status s;
    if ((s = make_map(&M.stencil, vis, 2ull * xarr, yarr, 2 * 34, 10)) != PG_OK) return s;
    M.base = vis;
    return PG_OK;
}

// ---------------------------------------------------------------- engine
static pg_status check_params(const pg_params* P) {
    if (!P) return fail(PG_ERR_ARG, "null params");
    if (P->ndim != 1 && P->ndim != 2) return fail(PG_ERR_CONFIG, "ndim must be 1 or 2");
    if (P->ndim == 1 && P->yres != 1) return fail(PG_ERR_CONFIG, "ndim 1 needs yres 1");
    if (P->xres < 2 * NPAD || (P->ndim == 2 && P->yres < 2 * NPAD))
        return fail(PG_ERR_CONFIG, "resolution below the stencil width");
    if (P->xres % 2) return fail(PG_ERR_CONFIG, "xres must be even (16-byte aligned rows)");
    if (P->eos_flag != 0 && P->eos_flag != 2) return fail(PG_ERR_CONFIG, "EOS_flag must be 0 or 2");
    if ((P->geomx != 0 && P->geomx != 1) || (P->geomy != 0 && P->geomy != 3))
        return fail(PG_ERR_CONFIG, "supported geometries: geomx 0/1, geomy 0/3");
    if (P->bound_lft < 0 || P->bound_lft > 2 || P->bound_rgh < 0 || P->bound_rgh > 2)
        return fail(PG_ERR_CONFIG, "radial boundaries must be 0, 1 or 2");
    if (P->n_planet != 0 && P->n_planet != 1) return fail(PG_ERR_CONFIG, "n_planet must be 0 or 1");
    if (P->dust_flag) {
        if (P->ndim != 2) return fail(PG_ERR_CONFIG, "dust needs ndim 2");
        if (P->init_flag != 2) return fail(PG_ERR_CONFIG, "dust needs init_flag 2 (init_CD)");
        if (!(P->stokes > 0.0)) return fail(PG_ERR_CONFIG, "dust needs Stokes > 0");
    }
    if (P->cool_flag < 0 || P->cool_flag > 2) return fail(PG_ERR_CONFIG, "cool_flag must be 0, 1 or 2");
    if (P->twobd_flag != 0 && P->twobd_flag != 1) return fail(PG_ERR_CONFIG, "twobd_flag must be 0 or 1");
    if (P->twobd_flag && (P->ndim != 2 || P->geomx != 1 || P->n_planet != 1))
        return fail(PG_ERR_CONFIG, "the two-body frame needs a 2D polar disk with n_planet 1 (the planet; the star is the second body)");
    if (P->cool_flag && !(P->beta_cool > 0.0)) return fail(PG_ERR_CONFIG, "cooling needs beta_cool > 0");
    if (P->gridx < 0 || P->gridx > 1 || P->gridy != 0) return fail(PG_ERR_CONFIG, "grids: x linear/log, y linear");
    if (P->gridx == 1 && !(P->xmin > 0.0)) return fail(PG_ERR_CONFIG, "log grid needs xmin > 0");
    return PG_OK;
}

struct Engine {
    pg_params P{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DiskView view{};
    Scalars* sc = nullptr;
    Cell* buf[2] = {nullptr, nullptr};
    bool own_buffers = false;
    double* vis = nullptr;
    bool own_vis = false;
    double* rot = nullptr;
    double* res = nullptr;
    int* inc = nullptr;
    bool own_orb = false;
    double* grid = nullptr;  // xa | xv | ya | yv (owned mode)
    double* tab = nullptr;   // weights and per-index tables
    CellMaps maps[2];
    VisMaps vmap;
    int cur = 0;
    bool fresh = true;       // no step taken since the state was set
    // device-loop bookkeeping: steps past end_time are no-ops on the device, so the
    // buffer holding the newest state follows the device's executed-step count
    bool pending = false;
    int cur_base = 0;
    long long steps_base = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // pg_disk_run: one step from buffer k
    cudaGraphExec_t sgraph[2] = {nullptr, nullptr};  // pg_disk_solve: the step after k_set_time, from buffer k
    std::vector<const void*> ghosted;  // buffers whose constant radial ghosts are initialised
    std::vector<const void*> dghosted; // dust buffers likewise (drop-in mode)
    pg_body* grid_planet = nullptr;    // drop-in mode: the caller's planets array
    double* part = nullptr;            // per-block partial sums of diagnostics
    pg_dust* dbuf[2] = {nullptr, nullptr};  // dust_flag: the dust of buf[k] is dbuf[k]
    DustMaps dmaps[2];
    Tune tune;                               // launch configuration (pg_disk_autotune)
    Cell* ave = nullptr;                     // time average (pg_disk_set_average)
    double* snap = nullptr;                  // pinned staging of snapshots
    size_t snap_n = 0;
    double* xfer = nullptr;                  // device staging of host exchanges (xfer_buffer)
    size_t xfer_n = 0;
    unsigned long long* hbits = nullptr;     // pinned read-back of the signal-rate maximum (global_dt)

    ~Engine() {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& g : sgraph)
            if (g) cudaGraphExecDestroy(g);
        if (own_buffers) {
            cudaFree(buf[0]);
            cudaFree(buf[1]);
        }
        if (own_vis) cudaFree(vis);
        if (own_orb) {
            cudaFree(rot);
            cudaFree(res);
            cudaFree(inc);
        }
        cudaFree(dbuf[0]);
        cudaFree(dbuf[1]);
        cudaFree(ave);
        if (snap) cudaFreeHost(snap);
        if (hbits) cudaFreeHost(hbits);
        cudaFree(xfer);
        cudaFree(grid);
        cudaFree(tab);
        cudaFree(part);
        cudaFree(sc);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

// Device staging for the host <-> device exchanges of the state, the dust and
// the time average (interior planes, up to 4 x xres*yres doubles).  Allocated on
// first use and kept, so an exchange neither allocates nor frees device memory
// (a per-call stream-ordered allocation goes back to the driver at every
// synchronisation under the default pool threshold and is mapped again at the
// next call).  Every user runs on E.stream; a larger request waits for the
// stream before replacing the buffer.
static pg_status xfer_buffer(Engine& E, size_t count, double** out) {
    if (E.xfer_n < count) {
        PG_CUDA(cudaStreamSynchronize(E.stream));
        cudaFree(E.xfer);
        E.xfer = nullptr;
        E.xfer_n = 0;
        PG_CUDA(cudaMalloc(&E.xfer, count * sizeof(double)));
        E.xfer_n = count;
    }
    *out = E.xfer;
    return PG_OK;
}

// Builds the grid (owned mode) or adopts the caller's device grid, then all tables.
static pg_status engine_setup(Engine& E, const double* dev_xa, const double* dev_xv, const double* dev_ya,
                              const double* dev_yv) {
    const pg_params& P = E.P;
    const int xarr = P.xres + 2 * NPAD;
    const int ypad = P.ndim > 1 ? NPAD : 0;
    const int yarr = P.yres + 2 * ypad;
    std::vector<double> xa(xarr + 1), xv(xarr), ya(yarr + 1), yv(yarr);
    make_grid(xa.data(), xv.data(), P.xmin, P.xmax, P.xres, NPAD, P.geomx, P.gridx, &P);
    make_grid(ya.data(), yv.data(), P.ymin, P.ymax, P.yres, ypad, P.geomy, P.gridy, &P);
    if (!dev_xa) {
        PG_CUDA(cudaMalloc(&E.grid, sizeof(double) * (2 * xarr + 2 * yarr + 2)));
        double* g = E.grid;
        PG_CUDA(cudaMemcpyAsync(g, xa.data(), sizeof(double) * (xarr + 1), cudaMemcpyHostToDevice, E.stream));
        PG_CUDA(cudaMemcpyAsync(g + xarr + 1, xv.data(), sizeof(double) * xarr, cudaMemcpyHostToDevice, E.stream));
        PG_CUDA(cudaMemcpyAsync(g + 2 * xarr + 1, ya.data(), sizeof(double) * (yarr + 1), cudaMemcpyHostToDevice, E.stream));
        PG_CUDA(cudaMemcpyAsync(g + 2 * xarr + yarr + 2, yv.data(), sizeof(double) * yarr, cudaMemcpyHostToDevice, E.stream));
        dev_xa = g;
        dev_xv = g + xarr + 1;
        dev_ya = g + 2 * xarr + 1;
        dev_yv = g + 2 * xarr + yarr + 2;
    } else {
        // the caller built its grid with the same routine on its host; read it back so
        // the weights are computed from exactly those faces
        PG_CUDA(cudaMemcpyAsync(xa.data(), dev_xa, sizeof(double) * (xarr + 1), cudaMemcpyDeviceToHost, E.stream));
        PG_CUDA(cudaMemcpyAsync(ya.data(), dev_ya, sizeof(double) * (yarr + 1), cudaMemcpyDeviceToHost, E.stream));
        PG_CUDA(cudaStreamSynchronize(E.stream));
    }
    // tables: wx[6 xarr] wy[6 yarr] | radx cs2x nux initx(5) killx(4) idx_x ixv irad gstar visx(5) [xarr each]
    //         | ycraw ycj idx_y iyv visy(4) [yarr each] | trig [4 yarr + 2]
    //         | initd(4) [xarr] with dust | coolx [xarr] with cool_flag 1 | strig [4 yarr] with twobd_flag
    const size_t ntab = 6 * (size_t)xarr + 6 * (size_t)yarr + 21 * (size_t)xarr + 8 * (size_t)yarr + 4 * (size_t)yarr + 2 +
                        (P.dust_flag ? 4 * (size_t)xarr : 0) + (P.cool_flag == 1 ? (size_t)xarr : 0) +
                        (P.twobd_flag ? 4 * (size_t)yarr : 0);
    PG_CUDA(cudaMalloc(&E.tab, sizeof(double) * ntab));
    std::vector<double> wx(6 * xarr), wy(6 * yarr);
    {
        pg_status ws = recon_weights(P.geomx, dev_xa, xarr, wx.data(), E.stream);
        if (ws == PG_OK) ws = recon_weights(P.geomy, dev_ya, yarr, wy.data(), E.stream);
        if (ws != PG_OK) return ws;
        // The ghost rows of the periodic azimuth keep the weights of their own
        // coordinates, as the reference evaluates them: their rounding differs
        // from the rows they image (on a 3072-cell azimuth by ~1e-9 of a slope),
        // so the seam has two slightly different faces, in the reference as here.
    }
    PG_CUDA(cudaMemcpyAsync(E.tab, wx.data(), sizeof(double) * wx.size(), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(E.tab + 6 * xarr, wy.data(), sizeof(double) * wy.size(), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));  // host vectors go out of scope

    if (!E.sc) PG_CUDA(cudaMalloc(&E.sc, sizeof(Scalars)));
    PG_CUDA(cudaMemsetAsync(E.sc, 0, sizeof(Scalars), E.stream));

    DiskView& d = E.view;
    d.xres = P.xres;
    d.yres = P.yres;
    d.xarr = xarr;
    d.yarr = yarr;
    d.ypad = ypad;
    d.ndim = P.ndim;
    d.geomx = P.geomx;
    d.geomy = P.geomy;
    d.eos = P.eos_flag;
    d.ie = P.internal_e_flag;
    d.bound_lft = P.bound_lft;
    d.bound_rgh = P.bound_rgh;
    d.visc = P.visc_flag && P.ndim == 2;
    d.orbadv = P.orbadv_flag && P.ndim == 2;
    d.kill = P.kill_flag;
    d.nplanet = P.n_planet;
    d.gam = P.gam;
    d.cfl = P.cfl;
    d.frame_omega = P.frame_omega;
    d.dy0 = (P.ymax - P.ymin) / (double)P.yres;
    d.planet_mass = P.planet_mass;
    d.ramp_time = P.ramp_time;
    d.xa = dev_xa;
    d.xv = dev_xv;
    d.ya = dev_ya;
    d.yv = dev_yv;
    d.wx = E.tab;
    d.wy = E.tab + 6 * xarr;
    double* t = E.tab + 6 * xarr + 6 * yarr;
    d.radx = t;
    d.cs2x = t + xarr;
    d.nux = t + 2 * xarr;
    d.initx = t + 3 * xarr;
    d.killx = t + 8 * xarr;
    d.idx_x = t + 12 * xarr;
    d.ixv = t + 13 * xarr;
    d.irad = t + 14 * xarr;
    d.gstar = t + 15 * xarr;
    d.visx = t + 16 * xarr;
    d.ycraw = t + 21 * xarr;
    d.ycj = t + 21 * xarr + yarr;
    d.idx_y = t + 21 * xarr + 2 * yarr;
    d.iyv = t + 21 * xarr + 3 * yarr;
    d.visy = t + 21 * xarr + 4 * yarr;
    d.trig = t + 21 * xarr + 8 * yarr;
    PG_CUDA(cudaMemsetAsync(d.trig, 0, sizeof(double) * (4 * (size_t)yarr + 2), E.stream));
    d.dust = P.dust_flag ? 1 : 0;
    d.stokes = P.stokes;
    d.sc_h = P.sc_h;
    d.dust_rmin = P.d_g_ratio * SMALLR;
    d.initd = P.dust_flag ? d.trig + 4 * (size_t)yarr + 2 : nullptr;
    if (P.dust_flag) {
        std::vector<double> cd(4 * (size_t)xarr);
        init_cd_table(P, xa.data(), xarr, cd.data());
        PG_CUDA(cudaMemcpyAsync(const_cast<double*>(d.initd), cd.data(), sizeof(double) * cd.size(),
                                cudaMemcpyHostToDevice, E.stream));
        PG_CUDA(cudaStreamSynchronize(E.stream));
    }
    d.cool = P.cool_flag;
    d.beta_cool = P.beta_cool;
    d.coolx = (P.cool_flag == 1) ? d.trig + 4 * (size_t)yarr + 2 + (P.dust_flag ? 4 * (size_t)xarr : 0) : nullptr;
    d.twobd = P.twobd_flag;
    d.strig = P.twobd_flag ? d.trig + 4 * (size_t)yarr + 2 + (P.dust_flag ? 4 * (size_t)xarr : 0) +
                                 (P.cool_flag == 1 ? (size_t)xarr : 0)
                           : nullptr;
    if (d.strig) PG_CUDA(cudaMemsetAsync(d.strig, 0, sizeof(double) * 4 * (size_t)yarr, E.stream));
    d.rot = E.rot;
    d.res = E.res;
    d.inc = E.inc;
    d.sc = E.sc;
    launch_init_tables(d, P, t, E.stream);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

static pg_status ensure_ghosts(Engine& E, Cell* b) {
    for (const void* p : E.ghosted)
        if (p == b) return PG_OK;
    launch_init_xghosts(E.view, b, E.stream);
    PG_CUDA(cudaGetLastError());
    E.ghosted.push_back(b);
    return PG_OK;
}

static int passes_per_step(const DiskView& d) {
    return 3 + (d.ndim > 1 ? 1 : 0) + (d.ndim > 1 && d.orbadv ? 1 : 0);
}

// Resolves which buffer holds the newest state after device-loop launches.
static pg_status resolve_cur(Engine& E) {
    if (!E.pending) return PG_OK;
    long long steps = 0;
    PG_CUDA(cudaMemcpyAsync(&steps, &E.sc->steps, sizeof(steps), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    const long long flips = (passes_per_step(E.view) % 2) ? (steps - E.steps_base) : 0;
    E.cur = (int)((E.cur_base + flips) & 1);
    E.pending = false;
    return PG_OK;
}

// Kernels of one step after the time kernel; in = E.cur.  With rec, the input
// of every pass, kick1's stress and the orbital-advection arrays are copied
// out for the adjoint.
// the captured steps hold the view, the tensor maps and the launch configuration
static void drop_graphs(Engine& E) {
    for (auto* gs : {E.graph, E.sgraph})
        for (int k = 0; k < 2; ++k)
            if (gs[k]) {
                cudaGraphExecDestroy(gs[k]);
                gs[k] = nullptr;
            }
}

static pg_status enqueue_stages(Engine& E, const StepRecord* rec = nullptr) {
    const DiskView& d = E.view;
    pg_status s;
    int c = E.cur;
    const size_t ncell = (size_t)d.xarr * d.yarr;
    auto save = [&](int k) {
        if (rec) cudaMemcpyAsync(rec->stage[k], E.buf[c], ncell * sizeof(Cell), cudaMemcpyDeviceToDevice, E.stream);
    };
    auto maps = [&](int k) -> const CellMaps& { return E.maps[k]; };
    for (int k = 0; k < 2; ++k)
        if ((s = make_cell_maps(E.maps[k], E.buf[k], d.xarr, d.yarr)) != PG_OK) return s;
    if (d.visc && (s = make_vis_maps(E.vmap, E.vis, d.xarr, d.yarr)) != PG_OK) return s;
    // dust (dust_flag) takes as many passes as the gas, so dbuf[k] pairs with buf[k]
    pg_dust* const* D = E.dbuf;
    const bool dust = d.dust != 0;
    if (dust)
        for (int k = 0; k < 2; ++k)
            if ((s = make_dust_maps(E.dmaps[k], E.dbuf[k], d.xarr, d.yarr)) != PG_OK) return s;
    save(0);
    launch_kick1(d, maps(c), E.buf[1 - c], E.vis, E.stream, dust ? D[c] : nullptr, dust ? D[1 - c] : nullptr,
                 &E.tune);
    if (rec && d.visc)
        cudaMemcpyAsync(rec->vis, E.vis, 2 * ncell * sizeof(double), cudaMemcpyDeviceToDevice, E.stream);
    c = 1 - c;
    save(1);
    launch_sweep_x(d, maps(c), E.buf[1 - c], E.stream, &E.tune);
    if (dust) launch_dsweep_x(d, E.dmaps[c], D[1 - c], E.stream);
    c = 1 - c;
    if (d.ndim > 1) {
        save(2);
        launch_sweep_y(d, maps(c), E.buf[1 - c], E.stream, &E.tune);
        if (dust) launch_dsweep_y(d, E.dmaps[c], D[1 - c], E.stream);
        if (rec) {
            cudaMemcpyAsync(rec->res, E.res, d.xarr * sizeof(double), cudaMemcpyDeviceToDevice, E.stream);
            cudaMemcpyAsync(rec->inc, E.inc, d.xarr * sizeof(int), cudaMemcpyDeviceToDevice, E.stream);
        }
        c = 1 - c;
    }
    if (d.ndim > 1 && d.orbadv) {
        save(3);
        launch_advect(d, maps(c), E.buf[1 - c], E.stream, &E.tune);
        if (dust) launch_dadvect(d, E.dmaps[c], D[1 - c], E.stream);
        c = 1 - c;
    }
    save(4);
    launch_kick2(d, maps(c), E.vmap, E.buf[1 - c], E.stream, dust ? D[c] : nullptr, dust ? D[1 - c] : nullptr,
                 &E.tune);
    c = 1 - c;
    E.cur = c;
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

static pg_status engine_create(const pg_params* P, int device, void* stream, Engine** out) {
    pg_status s = check_params(P);
    if (s != PG_OK) return s;
    PG_CUDA(cudaSetDevice(device));
    static bool attrs = false;
    if (!attrs) {
        PG_CUDA(set_kernel_attributes());
        PG_CUDA(set_dust_attributes());
        attrs = true;
    }
    Engine* E = new Engine();
    E->P = *P;
    if (E->P.kill_width_out <= 0.0) E->P.kill_width_out = E->P.kill_width;
    E->device = device;
    if (stream) E->stream = (cudaStream_t)stream;
    else {
        cudaError_t e = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete E;
            return fail(PG_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        }
        E->own_stream = true;
    }
    *out = E;
    return PG_OK;
}

// Tables-only disk for the FP32 form: grid, FP64 tables, orbital-advection
// arrays and device scalars of one disk on stream s, without state buffers.
pg_status table_engine_create(const pg_params* P, int device, cudaStream_t s, Engine** out) {
    *out = nullptr;
    Engine* E = nullptr;
    pg_status st = engine_create(P, device, s, &E);
    if (st != PG_OK) return st;
    const int xarr = E->P.xres + 2 * NPAD;
    cudaError_t e;
    if ((e = cudaMalloc(&E->rot, xarr * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&E->res, xarr * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&E->inc, xarr * sizeof(int))) != cudaSuccess) {
        delete E;
        return fail(PG_ERR_CUDA, "cudaMalloc: %s", cudaGetErrorString(e));
    }
    E->own_orb = true;
    cudaMemsetAsync(E->res, 0, xarr * sizeof(double), E->stream);
    cudaMemsetAsync(E->inc, 0, xarr * sizeof(int), E->stream);
    if ((st = engine_setup(*E, nullptr, nullptr, nullptr, nullptr)) != PG_OK) {
        delete E;
        return st;
    }
    *out = E;
    return PG_OK;
}
void engine_destroy(Engine* E) { delete E; }
const DiskView& engine_view(const Engine* E) { return E->view; }
void engine_init_planet(Engine* E, double t) { launch_init_planet(E->view, E->P, t, E->stream); }

// 3D FP32 tensor map over `planes` planes of rows x pitch floats.
pg_status make_map3_f32(CUtensorMap* m, const float* base, uint64_t pitch, uint64_t rows, uint64_t planes,
                        uint32_t bx, uint32_t by, uint32_t bz) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return fail(PG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (reinterpret_cast<uintptr_t>(base) % 16 != 0 || (pitch * 4) % 16 != 0)
        return fail(PG_ERR_CONFIG, "FP32 planes must have 16-byte aligned rows");
    cuuint64_t dims[3] = {pitch, rows, planes};
    cuuint64_t strides[2] = {pitch * 4, pitch * rows * 4};
    cuuint32_t box[3] = {bx, by, bz};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PG_ERR_CUDA, "cuTensorMapEncodeTiled (3D FP32) failed (%d)", (int)r);
    return PG_OK;
}

__global__ void k_fill(const DiskView d, Cell* buf, const double* r, const double* p, const double* u,
                       const double* v) {
    // fill_grid (src/init/init.cu:502-519) then load_grid's interior fields (src/output/output.cu:197-243)
    const long long n = (long long)d.xarr * d.yarr;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % d.xarr), j = (int)(k / d.xarr);
        const double* I = d.initx + 5 * i;
        Cell c{I[0], I[1], I[2], I[3], I[4]};
        if (i >= NPAD && i < NPAD + d.xres && j >= d.ypad && j < d.ypad + d.yres) {
            const size_t m = (size_t)(i - NPAD) + (size_t)d.xres * (j - d.ypad);
            c.r = r[m];
            c.p = p[m];
            c.u = u[m];
            if (v) c.v = v[m];
        }
        store_cell(buf, d.xarr, i, j, c);
    }
}

__global__ void k_extract(const DiskView d, const Cell* buf, double* r, double* p, double* u, double* v) {
    const long long n = (long long)d.xres * d.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres), j = d.ypad + (int)(m / d.xres);
        const Cell c = load_cell(buf, d.xarr, i, j);
        r[m] = c.r;
        p[m] = c.p;
        u[m] = c.u;
        v[m] = c.v;
    }
}

// the caller's planets array: the planet, or the star (planets[0]) and the planet
// (planets[1]) of the two-body frame
__global__ void k_grid_planet_in(Scalars* sc, const pg_body* planets, int twobd) {
    if (twobd) {
        sc->star_next = planets[0];
        sc->planet_next = planets[1];
    } else {
        sc->planet_next = planets[0];
    }
}

// write_check_point's fields (src/output/output.cu:125-180): interior r, p, u,
// v (2D) of the gas source, then with dust r, u, v (2D), w (2D); x fastest
__global__ void k_snapshot_planes(const DiskView d, const Cell* gas, const pg_dust* dust, double* out) {
    const long long n = (long long)d.xres * d.yres;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int i = NPAD + (int)(m % d.xres), j = d.ypad + (int)(m / d.xres);
        const size_t k = (size_t)i + (size_t)d.xarr * j;
        const Cell c = gas[k];
        double* o = out + m;
        o[0] = c.r;
        o[n] = c.p;
        o[2 * n] = c.u;
        int f = 3;
        if (d.ndim > 1) o[(f++) * n] = c.v;
        if (dust) {
            const pg_dust q = dust[k];
            o[(f++) * n] = q.r;
            o[(f++) * n] = q.u;
            if (d.ndim > 1) {
                o[(f++) * n] = q.v;
                o[(f++) * n] = q.w;
            }
        }
    }
}
__global__ void k_grid_planet_out(const Scalars* sc, pg_body* planets, int twobd) {
    if (twobd) {
        planets[0] = sc->star_next;
        planets[1] = sc->planet_next;
    } else {
        planets[0] = sc->planet_next;
    }
}

}  // namespace pg

// ======================================================================
//                                C ABI
// ======================================================================
using namespace pg;

struct pg_disk {
    Engine* E;
};

static pg_status set_state_device(Engine& E, double t, const double* r, const double* p, const double* u,
                                  const double* v);

extern "C" {

const char* pg_version(void) { return "penguin_b200 0.1 (sm_100a, FP64 Godunov step)"; }
const char* pg_last_error(void) { return g_err.c_str(); }

pg_status pg_check_params(const pg_params* P) {
    if (P && P->ndim == 3) return check_params3(P);
    return check_params(P);
}

pg_status pg_make_grid(const pg_params* P, double* xa, double* xv, double* ya, double* yv) {
    pg_status s = check_params(P);
    if (s != PG_OK) return s;
    if (!xa || !xv || !ya || !yv) return fail(PG_ERR_ARG, "null output");
    const int ypad = P->ndim > 1 ? NPAD : 0;
    make_grid(xa, xv, P->xmin, P->xmax, P->xres, NPAD, P->geomx, P->gridx, P);
    make_grid(ya, yv, P->ymin, P->ymax, P->yres, ypad, P->geomy, P->gridy, P);
    return PG_OK;
}

// ---------------------------------------------------------- handle API
pg_status pg_disk_create(const pg_params* P, int device, void* stream, pg_disk** out) {
    if (!out) return fail(PG_ERR_ARG, "null out");
    *out = nullptr;
    Engine* E = nullptr;
    pg_status s = engine_create(P, device, stream, &E);
    if (s != PG_OK) return s;
    const int xarr = E->P.xres + 2 * NPAD;
    const int yarr = E->P.yres + 2 * (E->P.ndim > 1 ? NPAD : 0);
    const size_t n = (size_t)xarr * yarr;
    auto bail = [&](pg_status st) {
        delete E;
        return st;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&E->buf[0], n * sizeof(Cell))) != cudaSuccess ||
        (e = cudaMalloc(&E->buf[1], n * sizeof(Cell))) != cudaSuccess ||
        (e = cudaMalloc(&E->vis, 2 * n * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&E->rot, xarr * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&E->res, xarr * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&E->inc, xarr * sizeof(int))) != cudaSuccess)
        return bail(fail(PG_ERR_CUDA, "cudaMalloc: %s", cudaGetErrorString(e)));
    E->own_buffers = E->own_vis = E->own_orb = true;
    cudaMemsetAsync(E->buf[0], 0, n * sizeof(Cell), E->stream);
    cudaMemsetAsync(E->buf[1], 0, n * sizeof(Cell), E->stream);
    cudaMemsetAsync(E->vis, 0, 2 * n * sizeof(double), E->stream);
    cudaMemsetAsync(E->res, 0, xarr * sizeof(double), E->stream);
    cudaMemsetAsync(E->inc, 0, xarr * sizeof(int), E->stream);
    if ((s = engine_setup(*E, nullptr, nullptr, nullptr, nullptr)) != PG_OK) return bail(s);
    if ((s = ensure_ghosts(*E, E->buf[0])) != PG_OK) return bail(s);
    if ((s = ensure_ghosts(*E, E->buf[1])) != PG_OK) return bail(s);
    if (E->P.dust_flag) {
        // both dust buffers hold init_CD everywhere: the bound-0 radial ghosts keep it
        if ((e = cudaMalloc(&E->dbuf[0], n * sizeof(pg_dust))) != cudaSuccess ||
            (e = cudaMalloc(&E->dbuf[1], n * sizeof(pg_dust))) != cudaSuccess)
            return bail(fail(PG_ERR_CUDA, "cudaMalloc: %s", cudaGetErrorString(e)));
        launch_dust_init(E->view, E->dbuf[0], E->stream);
        launch_dust_init(E->view, E->dbuf[1], E->stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return bail(fail(PG_ERR_CUDA, "%s", cudaGetErrorString(e)));
    }
    pg_disk* d = new pg_disk{E};
    *out = d;
    return PG_OK;
}

pg_status pg_disk_destroy(pg_disk* d) {
    if (!d) return PG_OK;
    cudaSetDevice(d->E->device);
    cudaStreamSynchronize(d->E->stream);
    delete d->E;
    delete d;
    return PG_OK;
}

pg_status pg_disk_dims(const pg_disk* d, int* xarr, int* yarr, int* npad) {
    if (!d) return fail(PG_ERR_ARG, "null disk");
    if (xarr) *xarr = d->E->view.xarr;
    if (yarr) *yarr = d->E->view.yarr;
    if (npad) *npad = NPAD;
    return PG_OK;
}

pg_status pg_disk_set_state(pg_disk* dk, double t, const double* r, const double* p, const double* u,
                            const double* v) {
    if (!dk || !r || !p || !u) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    PG_CUDA(cudaSetDevice(E.device));
    const size_t n = (size_t)d.xres * d.yres;
    double* stage = nullptr;
    {
        const pg_status sx = xfer_buffer(E, 4 * n, &stage);
        if (sx != PG_OK) return sx;
    }
    PG_CUDA(cudaMemcpyAsync(stage, r, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(stage + n, p, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(stage + 2 * n, u, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    if (v) PG_CUDA(cudaMemcpyAsync(stage + 3 * n, v, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    const pg_status s = set_state_device(E, t, stage, stage + n, stage + 2 * n, v ? stage + 3 * n : nullptr);
    return s;
}

}  // extern "C"

// The state of a disk from interior device arrays (xres*yres each; v may be null).
static pg_status set_state_device(Engine& E, double t, const double* r, const double* p, const double* u,
                                  const double* v) {
    const DiskView& d = E.view;
    E.cur = 0;
    E.pending = false;
    k_fill<<<1184, 256, 0, E.stream>>>(d, E.buf[0], r, p, u, v);
    PG_CUDA(cudaGetLastError());
    launch_bound(d, E.buf[0], E.stream);
    if (d.dust) launch_dust_init(d, E.dbuf[0], E.stream);  // a restart's dust is init_CD (the gas file only)
    launch_init_planet(d, E.P, t, E.stream);
    launch_cfl(d, E.buf[0], E.stream, d.dust ? E.dbuf[0] : nullptr);
    PG_CUDA(cudaGetLastError());
    Scalars h{};
    PG_CUDA(cudaMemcpyAsync(&h, E.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    h.t = t;
    h.dt = 0.0;
    h.dt_prev = 0.0;
    h.steps = 0;
    h.done = 0;
    h.pad_ = 0;
    h.err = 0;
    h.floor_hits = 0;
    h.dt_hold = 0.0;
    PG_CUDA(cudaMemcpyAsync(E.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    E.fresh = true;
    return PG_OK;
}

namespace pg {

Engine* disk_engine(pg_disk* d) { return d ? d->E : nullptr; }

pg_status engine_set_state_device(Engine* E, double t, const double* r, const double* p, const double* u,
                                  const double* v) {
    PG_CUDA(cudaSetDevice(E->device));
    return set_state_device(*E, t, r, p, u, v);
}

// One step of main.cu's loop with a given dt (pg_disk_solve), optionally recording.
pg_status engine_step(Engine* E, double t, double dt, const StepRecord* rec) {
    pg_status s0 = resolve_cur(*E);
    if (s0 != PG_OK) return s0;
    launch_set_time(E->view, t, dt, E->stream);
    if (rec) PG_CUDA(cudaMemcpyAsync(rec->planets, &E->sc->planet_cur, 2 * sizeof(pg_body), cudaMemcpyDeviceToDevice,
                                     E->stream));
    E->fresh = false;
    return enqueue_stages(*E, rec);
}

// The newest state (all cells, ghosts included) and the device scalars (clock, planets).
pg_status engine_save(Engine* E, Cell* cells, Scalars* sc) {
    pg_status s0 = resolve_cur(*E);
    if (s0 != PG_OK) return s0;
    const size_t n = (size_t)E->view.xarr * E->view.yarr;
    PG_CUDA(cudaMemcpyAsync(cells, E->buf[E->cur], n * sizeof(Cell), cudaMemcpyDeviceToDevice, E->stream));
    PG_CUDA(cudaMemcpyAsync(sc, E->sc, sizeof(Scalars), cudaMemcpyDeviceToDevice, E->stream));
    return PG_OK;
}

cudaStream_t engine_set_stream(Engine* E, cudaStream_t s) {
    cudaStream_t old = E->stream;
    E->stream = s;
    return old;
}

pg_status engine_restore(Engine* E, const Cell* cells, const Scalars* sc) {
    const size_t n = (size_t)E->view.xarr * E->view.yarr;
    E->cur = 0;
    E->pending = false;
    PG_CUDA(cudaMemcpyAsync(E->buf[0], cells, n * sizeof(Cell), cudaMemcpyDeviceToDevice, E->stream));
    PG_CUDA(cudaMemcpyAsync(E->sc, sc, sizeof(Scalars), cudaMemcpyDeviceToDevice, E->stream));
    E->fresh = false;
    return PG_OK;
}

// One production pass on a given input (test support for the adjoint): in ->
// out (all cells), kick2 reading vis_in as kick1's force, kick1 leaving its
// force in vis_out.  The planet and dt are those of the last step taken; the
// disk's own state is overwritten.
pg_status engine_run_pass(Engine* E, int pass, const Cell* in, Cell* out, const double* vis_in, double* vis_out) {
    const DiskView& d = E->view;
    const size_t n = (size_t)d.xarr * d.yarr;
    pg_status s;
    PG_CUDA(cudaMemcpyAsync(E->buf[0], in, n * sizeof(Cell), cudaMemcpyDeviceToDevice, E->stream));
    for (int k = 0; k < 2; ++k)
        if ((s = make_cell_maps(E->maps[k], E->buf[k], d.xarr, d.yarr)) != PG_OK) return s;
    if (d.visc && (s = make_vis_maps(E->vmap, E->vis, d.xarr, d.yarr)) != PG_OK) return s;
    if (pass == 4 && d.visc && vis_in)
        PG_CUDA(cudaMemcpyAsync(E->vis, vis_in, 2 * n * sizeof(double), cudaMemcpyDeviceToDevice, E->stream));
    switch (pass) {
        case 0: launch_kick1(d, E->maps[0], E->buf[1], E->vis, E->stream, nullptr, nullptr, &E->tune); break;
        case 1: launch_sweep_x(d, E->maps[0], E->buf[1], E->stream, &E->tune); break;
        case 2: launch_sweep_y(d, E->maps[0], E->buf[1], E->stream, &E->tune); break;
        case 3: launch_advect(d, E->maps[0], E->buf[1], E->stream, &E->tune); break;
        default: launch_kick2(d, E->maps[0], E->vmap, E->buf[1], E->stream, nullptr, nullptr, &E->tune); break;
    }
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemcpyAsync(out, E->buf[1], n * sizeof(Cell), cudaMemcpyDeviceToDevice, E->stream));
    if (pass == 0 && d.visc && vis_out)
        PG_CUDA(cudaMemcpyAsync(vis_out, E->vis, 2 * n * sizeof(double), cudaMemcpyDeviceToDevice, E->stream));
    E->cur = 1;
    E->pending = false;
    return PG_OK;
}

// Interior fields of the newest state into device arrays (xres*yres each).
pg_status engine_extract_device(Engine* E, double* r, double* p, double* u, double* v) {
    pg_status s0 = resolve_cur(*E);
    if (s0 != PG_OK) return s0;
    k_extract<<<1184, 256, 0, E->stream>>>(E->view, E->buf[E->cur], r, p, u, v);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

}  // namespace pg

extern "C" {

pg_status pg_disk_get_state(pg_disk* dk, double* r, double* p, double* u, double* v, double* t_out) {
    if (!dk || !r || !p || !u) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    PG_CUDA(cudaSetDevice(E.device));
    const size_t n = (size_t)d.xres * d.yres;
    double* stage = nullptr;
    {
        const pg_status sx = xfer_buffer(E, 4 * n, &stage);
        if (sx != PG_OK) return sx;
    }
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    k_extract<<<1184, 256, 0, E.stream>>>(d, E.buf[E.cur], stage, stage + n, stage + 2 * n, stage + 3 * n);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemcpyAsync(r, stage, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(p, stage + n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(u, stage + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    if (v) PG_CUDA(cudaMemcpyAsync(v, stage + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    if (t_out) PG_CUDA(cudaMemcpyAsync(t_out, &E.sc->t, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

pg_status pg_disk_set_dust(pg_disk* dk, const double* r, const double* u, const double* v) {
    if (!dk || !r || !u || !v) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    if (!d.dust) return fail(PG_ERR_CONFIG, "the disk has no dust (dust_flag 0)");
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    const size_t n = (size_t)d.xres * d.yres;
    double* stage = nullptr;
    {
        const pg_status sx = xfer_buffer(E, 3 * n, &stage);
        if (sx != PG_OK) return sx;
    }
    PG_CUDA(cudaMemcpyAsync(stage, r, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(stage + n, u, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(stage + 2 * n, v, n * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    launch_dust_fill(d, E.dbuf[E.cur], stage, stage + n, stage + 2 * n, E.stream);
    PG_CUDA(cudaGetLastError());
    // the CFL rate of the first step includes the dust speeds
    launch_cfl(d, E.buf[E.cur], E.stream, E.dbuf[E.cur]);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

pg_status pg_disk_get_dust(pg_disk* dk, double* r, double* u, double* v) {
    if (!dk || !r || !u || !v) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    if (!d.dust) return fail(PG_ERR_CONFIG, "the disk has no dust (dust_flag 0)");
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    const size_t n = (size_t)d.xres * d.yres;
    double* stage = nullptr;
    {
        const pg_status sx = xfer_buffer(E, 3 * n, &stage);
        if (sx != PG_OK) return sx;
    }
    launch_dust_extract(d, E.dbuf[E.cur], stage, stage + n, stage + 2 * n, E.stream);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemcpyAsync(r, stage, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(u, stage + n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(v, stage + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

pg_status pg_disk_state_ptr(pg_disk* dk, pg_cell** cells) {
    if (!dk || !cells) return fail(PG_ERR_ARG, "null argument");
    pg_status s0 = resolve_cur(*dk->E);
    if (s0 != PG_OK) return s0;
    *cells = reinterpret_cast<pg_cell*>(dk->E->buf[dk->E->cur]);
    return PG_OK;
}

pg_status pg_disk_global_dt(pg_disk* dk, double dt_prev, double* dt_out) {
    if (!dk || !dt_out) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    // into pinned memory: a pageable destination would add a staged copy to every step
    if (!E.hbits) PG_CUDA(cudaMallocHost(&E.hbits, sizeof(unsigned long long)));
    PG_CUDA(cudaMemcpyAsync(E.hbits, &E.sc->vmax_bits, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    const unsigned long long bits = *E.hbits;
    double vmax;
    std::memcpy(&vmax, &bits, sizeof vmax);
    const double dt = E.P.cfl / vmax;  // get_dt_lv2 (timestep.cu:108)
    double tmp = dt_prev * 1.1;        // timestep.cu:133-139
    if (dt < tmp) tmp = dt;
    *dt_out = tmp;
    return PG_OK;
}

pg_status pg_disk_solve(pg_disk* dk, double t, double dt) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    Engine& E = *dk->E;
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    // this step's t and dt go in as launch arguments of k_set_time; the rest of the
    // step (planet angles, five passes) is one captured graph per starting buffer,
    // one launch instead of six behind the host's dt read-back
    launch_set_time_only(E.view, t, dt, E.stream);
    PG_CUDA(cudaGetLastError());
    const int c0 = E.cur;
    if (!E.sgraph[c0]) {
        cudaGraph_t g;
        PG_CUDA(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
        launch_planet_trig(E.view, E.stream);
        pg_status s = enqueue_stages(E);
        cudaError_t ce = cudaStreamEndCapture(E.stream, &g);
        E.cur = c0;
        if (s != PG_OK) {
            if (ce == cudaSuccess) cudaGraphDestroy(g);
            return s;
        }
        PG_CUDA(ce);
        cudaError_t ie = cudaGraphInstantiate(&E.sgraph[c0], g, 0);
        cudaGraphDestroy(g);
        PG_CUDA(ie);
    }
    PG_CUDA(cudaGraphLaunch(E.sgraph[c0], E.stream));
    E.cur = (passes_per_step(E.view) % 2) ? 1 - c0 : c0;
    E.fresh = false;
    return PG_OK;
}

pg_status pg_disk_step_host(pg_disk* dk, int max_step, double end_time, double* t, double* dt, int* n) {
    if (!dk || !t || !dt || !n) return fail(PG_ERR_ARG, "null argument");
    // main.cu:320-360: dt from global_dt (read back every step), clipped at end_time,
    // then solve and t += dt; a first call without a previous step caps dt by end_time - t
    double tt = *t, step = (*dt != 0.0) ? *dt : end_time - *t;
    int k = 0;
    pg_status s = PG_OK;
    while (k < max_step) {
        if ((s = pg_disk_global_dt(dk, step, &step)) != PG_OK) break;
        bool last = false;
        if (tt + step > end_time) {
            step = end_time - tt;
            last = true;
        }
        if ((s = pg_disk_solve(dk, tt, step)) != PG_OK) break;
        tt += step;
        ++k;
        if (last) break;
    }
    *t = tt;
    *dt = step;
    *n = k;
    return s;
}

pg_status pg_disk_run(pg_disk* dk, int nsteps, double end_time) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    if (nsteps <= 0) return PG_OK;
    Engine& E = *dk->E;
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    // with a finite end_time the device may finish early: check its done flag
    // every 256 launched steps so the host does not keep launching no-op steps
    const bool may_finish = end_time < 1.0e29;
    if (may_finish) {
        // main.cu:144 + 322: the first cap on dt is end_time - t after a (re)start
        Scalars h{};
        PG_CUDA(cudaMemcpyAsync(&h, E.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, E.stream));
        PG_CUDA(cudaStreamSynchronize(E.stream));
        if (E.fresh) h.dt_prev = end_time - h.t;
        // a run that stopped on a clip at its end_time continues like main.cu after
        // a dump (main.cu:333-338, 425): the step before the clip caps the next one
        else if (h.dt_hold > 0.0) h.dt_prev = h.dt_hold;
        h.dt_hold = 0.0;
        h.end_time = end_time;
        h.done = 0;
        h.pad_ = 0;
        PG_CUDA(cudaMemcpyAsync(E.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, E.stream));
        E.steps_base = h.steps;  // the step count the device reached decides the newest buffer
        E.pending = true;
    } else {
        // every launched step runs, so the newest buffer is known on the host: the
        // same opening of the run as above, on the device, with no host round trip
        launch_run_begin(E.sc, end_time, E.fresh, E.stream);
        PG_CUDA(cudaGetLastError());
        E.pending = false;
    }
    E.fresh = false;
    E.cur_base = E.cur;
    for (int k = 0; k < 2; ++k) {
        pg_status s = make_cell_maps(E.maps[k], E.buf[k], E.view.xarr, E.view.yarr);
        if (s != PG_OK) return s;
    }
    for (int step = 0; step < nsteps; ++step) {
        if (may_finish && step > 0 && step % 256 == 0) {
            int done = 0;
            PG_CUDA(cudaMemcpyAsync(&done, &E.sc->done, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
            PG_CUDA(cudaStreamSynchronize(E.stream));
            if (done) break;
        }
        const int c0 = E.cur;
        if (!E.graph[c0]) {
            // capture one step (time kernel + stages) starting from buffer c0
            cudaGraph_t g;
            PG_CUDA(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
            launch_time_step(E.view, E.stream);
            pg_status s = enqueue_stages(E);
            cudaError_t ce = cudaStreamEndCapture(E.stream, &g);
            if (s != PG_OK) return s;
            PG_CUDA(ce);
            PG_CUDA(cudaGraphInstantiate(&E.graph[c0], g, 0));
            cudaGraphDestroy(g);
            E.cur = c0;
        }
        PG_CUDA(cudaGraphLaunch(E.graph[c0], E.stream));
        // the captured step leaves the newest state in the other buffer iff it has an
        // odd number of passes (if the device actually ran it: see resolve_cur)
        E.cur = (passes_per_step(E.view) % 2) ? 1 - c0 : c0;
    }
    if (!may_finish) {  // every launched step ran: the index above is exact
        E.pending = false;
    } else {
        E.cur = E.cur_base;  // resolved from the device step count on next use
    }
    return PG_OK;
}

pg_status pg_disk_sync(pg_disk* dk) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    PG_CUDA(cudaStreamSynchronize(dk->E->stream));
    return PG_OK;
}

pg_status pg_disk_clock(pg_disk* dk, double* t, double* dt, long long* steps) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    Scalars h{};
    PG_CUDA(cudaMemcpyAsync(&h, dk->E->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, dk->E->stream));
    PG_CUDA(cudaStreamSynchronize(dk->E->stream));
    if (t) *t = h.t;
    if (dt) *dt = h.dt;
    if (steps) *steps = h.steps;
    return PG_OK;
}

pg_status pg_disk_planet(pg_disk* dk, pg_body* out) {
    if (!dk || !out) return fail(PG_ERR_ARG, "null argument");
    Scalars h{};
    PG_CUDA(cudaMemcpyAsync(&h, dk->E->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, dk->E->stream));
    PG_CUDA(cudaStreamSynchronize(dk->E->stream));
    *out = h.planet_next;
    return PG_OK;
}

pg_status pg_disk_check(pg_disk* dk) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    int err = 0;
    PG_CUDA(cudaMemcpyAsync(&err, &dk->E->sc->err, sizeof(int), cudaMemcpyDeviceToHost, dk->E->stream));
    PG_CUDA(cudaStreamSynchronize(dk->E->stream));
    const int zero = 0;
    PG_CUDA(cudaMemcpy(&dk->E->sc->err, &zero, sizeof(int), cudaMemcpyHostToDevice));
    if (err & (1 << PG_ERR_TIMEOUT)) return fail(PG_ERR_TIMEOUT, "a device wait timed out");
    if (err & (1 << PG_ERR_NAN)) return fail(PG_ERR_NAN, "non-positive or NaN density produced");
    return PG_OK;
}

pg_status pg_disk_torque(pg_disk* dk, double* torque) {
    if (!dk || !torque) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    if (d.ndim != 2 || d.geomy != 3 || d.nplanet < 1)
        return fail(PG_ERR_CONFIG, "pg_disk_torque: needs a 2D polar disk with a planet");
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    constexpr int nb = 296;
    if (!E.part) PG_CUDA(cudaMalloc(&E.part, nb * sizeof(double)));
    launch_torque(d, E.buf[E.cur], E.part, nb, E.stream);
    PG_CUDA(cudaGetLastError());
    double h[nb];
    PG_CUDA(cudaMemcpyAsync(h, E.part, sizeof h, cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    *torque = compensated_sum(h, nb);
    return PG_OK;
}

int pg_kernels_per_step(const pg_disk* dk) { return dk ? kernels_per_step(dk->E->view) : 0; }

// Autotuner: for every pass, times each launch configuration (for the sweeps
// and the advection each tile variant of SWEEP_VARIANTS: pencils per tile,
// outputs per pencil, cells per thread, TMA stages; for every pass the CTAs per
// SM from 1 to what fits) on the disk's current state with CUDA events over
// `reps` launches and keeps the fastest.  The state, clock and planet are
// restored afterwards; the per-cell arithmetic does not depend on the
// configuration, so results stay bit for bit the same.  choice (may be NULL):
// the variants of sweep_x, sweep_y, advect, then the CTA caps of the 5 passes.
pg_status pg_disk_autotune(pg_disk* dk, int reps, int* choice) {
    if (!dk || reps < 1) return fail(PG_ERR_ARG, "bad argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s = resolve_cur(E);
    if (s != PG_OK) return s;
    const size_t n = (size_t)d.xarr * d.yarr;
    Cell* saved = nullptr;
    Scalars* ssc = nullptr;
    PG_CUDA(cudaMallocAsync(&saved, n * sizeof(Cell), E.stream));
    PG_CUDA(cudaMallocAsync(&ssc, sizeof(Scalars), E.stream));
    const int c = E.cur;
    PG_CUDA(cudaMemcpyAsync(saved, E.buf[c], n * sizeof(Cell), cudaMemcpyDeviceToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(ssc, E.sc, sizeof(Scalars), cudaMemcpyDeviceToDevice, E.stream));
    double dt = 0.0;
    if ((s = pg_disk_global_dt(dk, 1.0e30, &dt)) != PG_OK) return s;
    Scalars h{};
    PG_CUDA(cudaMemcpyAsync(&h, E.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    launch_set_time(d, h.t, dt, E.stream);
    for (int k = 0; k < 2; ++k)
        if ((s = make_cell_maps(E.maps[k], E.buf[k], d.xarr, d.yarr)) != PG_OK) return s;
    if (d.visc && (s = make_vis_maps(E.vmap, E.vis, d.xarr, d.yarr)) != PG_OK) return s;
    cudaEvent_t e0, e1;
    PG_CUDA(cudaEventCreate(&e0));
    PG_CUDA(cudaEventCreate(&e1));
    auto launch = [&](int p, const Tune& t) {
        switch (p) {
            case 0: launch_kick1(d, E.maps[c], E.buf[1 - c], E.vis, E.stream, nullptr, nullptr, &t); break;
            case 1: launch_sweep_x(d, E.maps[c], E.buf[1 - c], E.stream, &t); break;
            case 2: launch_sweep_y(d, E.maps[c], E.buf[1 - c], E.stream, &t); break;
            case 3: launch_advect(d, E.maps[c], E.buf[1 - c], E.stream, &t); break;
            default: launch_kick2(d, E.maps[c], E.vmap, E.buf[1 - c], E.stream, nullptr, nullptr, &t); break;
        }
    };
    Tune best = E.tune;
    for (int p = 0; p < 5; ++p) {
        if ((p == 2 && d.ndim < 2) || (p == 3 && !(d.ndim > 1 && d.orbadv))) continue;
        float best_ms = 1.0e30f;
        const int nv = (p >= 1 && p <= 3) ? NSWEEP_VARIANTS : 1;
        for (int v = 0; v < nv; ++v) {
            if (p == 1 && !sweep_variant_x_ok(v)) continue;
            const int occ = pass_occupancy(d, p, v);
            for (int cps = 1; cps <= occ; ++cps) {
                Tune t = best;
                if (p >= 1 && p <= 3) t.v[p - 1] = v;
                t.cps[p] = cps;
                launch(p, t);  // warm-up
                PG_CUDA(cudaEventRecord(e0, E.stream));
                for (int r = 0; r < reps; ++r) launch(p, t);
                PG_CUDA(cudaEventRecord(e1, E.stream));
                PG_CUDA(cudaEventSynchronize(e1));
                PG_CUDA(cudaGetLastError());
                float ms = 0.0f;
                PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best_ms) {
                    best_ms = ms;
                    if (p >= 1 && p <= 3) best.v[p - 1] = v;
                    best.cps[p] = cps;
                }
            }
        }
        if (p == 0) launch(0, best);  // kick2 reads the force kick1 leaves
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    E.tune = best;
    drop_graphs(E);
    PG_CUDA(cudaMemcpyAsync(E.buf[c], saved, n * sizeof(Cell), cudaMemcpyDeviceToDevice, E.stream));
    PG_CUDA(cudaMemcpyAsync(E.sc, ssc, sizeof(Scalars), cudaMemcpyDeviceToDevice, E.stream));
    PG_CUDA(cudaFreeAsync(saved, E.stream));
    PG_CUDA(cudaFreeAsync(ssc, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    if (choice) {
        for (int k = 0; k < 3; ++k) choice[k] = best.v[k];
        for (int k = 0; k < 5; ++k) choice[3 + k] = best.cps[k];
    }
    return PG_OK;
}

static int snapshot_fields(const DiskView& d) {
    return (d.ndim > 1 ? 4 : 3) + (d.dust ? (d.ndim > 1 ? 4 : 2) : 0);
}


// ave_flag: the gas state averaged over a save interval T by the trapezoid rule
// of main.cu:343-351 (A += C (dt/2)/T before and after each step), accumulated
// in the first and last pass of the step.  interval <= 0 switches it off.
pg_status pg_disk_set_average(pg_disk* dk, double interval) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    Engine& E = *dk->E;
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    const size_t n = (size_t)E.view.xarr * E.view.yarr;
    if (interval > 0.0) {
        if (!E.ave) PG_CUDA(cudaMalloc(&E.ave, n * sizeof(Cell)));
        PG_CUDA(cudaMemsetAsync(E.ave, 0, n * sizeof(Cell), E.stream));
        E.view.ave = E.ave;
        E.view.ave_T = interval;
    } else {
        E.view.ave = nullptr;
        E.view.ave_T = 0.0;
    }
    drop_graphs(E);
    PG_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

// init_average (src/output/output.cu:315-330)
pg_status pg_disk_reset_average(pg_disk* dk) {
    if (!dk) return fail(PG_ERR_ARG, "null disk");
    Engine& E = *dk->E;
    if (!E.view.ave) return fail(PG_ERR_CONFIG, "no time average (pg_disk_set_average)");
    PG_CUDA(cudaMemsetAsync(E.ave, 0, (size_t)E.view.xarr * E.view.yarr * sizeof(Cell), E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

pg_status pg_disk_get_average(pg_disk* dk, double* r, double* p, double* u, double* v) {
    if (!dk || !r || !p || !u) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    if (!d.ave) return fail(PG_ERR_CONFIG, "no time average (pg_disk_set_average)");
    PG_CUDA(cudaSetDevice(E.device));
    const size_t n = (size_t)d.xres * d.yres;
    double* stage = nullptr;
    {
        const pg_status sx = xfer_buffer(E, 4 * n, &stage);
        if (sx != PG_OK) return sx;
    }
    k_extract<<<1184, 256, 0, E.stream>>>(d, E.ave, stage, stage + n, stage + 2 * n, stage + 3 * n);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemcpyAsync(r, stage, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(p, stage + n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(u, stage + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    if (v) PG_CUDA(cudaMemcpyAsync(v, stage + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    return PG_OK;
}

// A snapshot in the reference's checkpoint format (write_check_point,
// src/output/output.cu:125-180): t, the interior faces xa (and ya in 2D), then
// the fields.  average = 1 writes the time average of the gas (with the
// current dust, like main.cu:411-419).  The fields are gathered into planes on
// the device and written with one host write.
pg_status pg_disk_write_snapshot(pg_disk* dk, const char* path, int average) {
    if (!dk || !path) return fail(PG_ERR_ARG, "null argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    if (average && !d.ave) return fail(PG_ERR_CONFIG, "no time average (pg_disk_set_average)");
    PG_CUDA(cudaSetDevice(E.device));
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    const size_t n = (size_t)d.xres * d.yres, nf = (size_t)snapshot_fields(d);
    const size_t head = 1 + (size_t)d.xres + 1 + (d.ndim > 1 ? (size_t)d.yres + 1 : 0);
    const size_t total = head + nf * n;
    if (E.snap_n < total) {
        if (E.snap) cudaFreeHost(E.snap);
        E.snap = nullptr;
        PG_CUDA(cudaMallocHost(&E.snap, total * sizeof(double)));
        E.snap_n = total;
    }
    double* h = E.snap;
    double* planes = nullptr;
    PG_CUDA(cudaMallocAsync(&planes, nf * n * sizeof(double), E.stream));
    k_snapshot_planes<<<1184, 256, 0, E.stream>>>(d, average ? E.ave : E.buf[E.cur], d.dust ? E.dbuf[E.cur] : nullptr,
                                                  planes);
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaMemcpyAsync(h, &E.sc->t, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaMemcpyAsync(h + 1, d.xa + NPAD, (d.xres + 1) * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    if (d.ndim > 1)
        PG_CUDA(cudaMemcpyAsync(h + 2 + d.xres, d.ya + d.ypad, (d.yres + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                                E.stream));
    PG_CUDA(cudaMemcpyAsync(h + head, planes, nf * n * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaFreeAsync(planes, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(PG_ERR_ARG, "cannot open %s for writing", path);
    const size_t w = std::fwrite(h, sizeof(double), total, f);
    const int c = std::fclose(f);
    if (w != total || c != 0) return fail(PG_ERR_ARG, "short write to %s", path);
    return PG_OK;
}

// Restart from a snapshot (load_grid, src/output/output.cu:182-248): t and the
// gas fields; the faces are skipped and any dust fields ignored (the dust
// restarts from init_CD, as in the reference).
pg_status pg_disk_read_snapshot(pg_disk* dk, const char* path, double* t_out) {
    if (!dk || !path) return fail(PG_ERR_ARG, "null argument");
    const DiskView& d = dk->E->view;
    const size_t n = (size_t)d.xres * d.yres, ng = d.ndim > 1 ? 4 : 3;
    const size_t head = 1 + (size_t)d.xres + 1 + (d.ndim > 1 ? (size_t)d.yres + 1 : 0);
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(PG_ERR_ARG, "cannot open %s", path);
    std::vector<double> buf(head + ng * n);
    const size_t r = std::fread(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    if (r != buf.size()) return fail(PG_ERR_ARG, "%s: %zu values, expected at least %zu", path, r, buf.size());
    const double* F = buf.data() + head;
    pg_status s = pg_disk_set_state(dk, buf[0], F, F + n, F + 2 * n, d.ndim > 1 ? F + 3 * n : nullptr);
    if (s == PG_OK && t_out) *t_out = buf[0];
    return s;
}

pg_status pg_recon_weights(const pg_params* P, int dir, double* w) {
    if (!P || !w || (dir != 0 && dir != 1)) return fail(PG_ERR_ARG, "bad argument");
    pg_status s = pg_check_params(P);
    if (s != PG_OK) return s;
    const int ypad = P->ndim > 1 ? NPAD : 0;
    const int n = dir == 0 ? P->xres + 2 * NPAD : P->yres + 2 * ypad;
    std::vector<double> a(n + 1), v(n);
    if (dir == 0) make_grid(a.data(), v.data(), P->xmin, P->xmax, P->xres, NPAD, P->geomx, P->gridx, P);
    else make_grid(a.data(), v.data(), P->ymin, P->ymax, P->yres, ypad, P->geomy, P->gridy, P);
    double* dev = nullptr;
    PG_CUDA(cudaMalloc(&dev, sizeof(double) * (n + 1)));
    cudaError_t e = cudaMemcpy(dev, a.data(), sizeof(double) * (n + 1), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(dev);
        PG_CUDA(e);
    }
    s = recon_weights(dir == 0 ? P->geomx : P->geomy, dev, n, w, 0);
    cudaFree(dev);
    return s;
}

pg_status pg_sweep_variant(int v, int* out6) {
    if (v < 0 || v >= NSWEEP_VARIANTS || !out6) return fail(PG_ERR_ARG, "no such tile variant");
    const SweepVariant& g = SWEEP_VARIANTS[v];
    out6[0] = g.w;
    out6[1] = g.len;
    out6[2] = g.cpt;
    out6[3] = g.stages;
    sweep_variant_launch(v, &out6[4], &out6[5]);
    return PG_OK;
}

pg_status pg_disk_set_tuning(pg_disk* dk, const int* choice) {
    if (!dk || !choice) return fail(PG_ERR_ARG, "bad argument");
    Tune t;
    for (int k = 0; k < 3; ++k) {
        if (choice[k] < 0 || choice[k] >= NSWEEP_VARIANTS || (k == 0 && !sweep_variant_x_ok(choice[k])))
            return fail(PG_ERR_ARG, "no such tile variant for this pass");
        t.v[k] = choice[k];
    }
    for (int k = 0; k < 5; ++k) {
        if (choice[3 + k] < 0) return fail(PG_ERR_ARG, "CTAs per SM must be >= 0");
        t.cps[k] = choice[3 + k];
    }
    Engine& E = *dk->E;
    E.tune = t;
    drop_graphs(E);
    return PG_OK;
}

pg_status pg_disk_profile(pg_disk* dk, int nsteps, double end_time, float* ms, int nslot) {
    if (!dk || !ms || nslot < 6) return fail(PG_ERR_ARG, "bad argument");
    Engine& E = *dk->E;
    const DiskView& d = E.view;
    PG_CUDA(cudaSetDevice(E.device));
    for (int k = 0; k < nslot; ++k) ms[k] = 0.0f;
    pg_status s0 = resolve_cur(E);
    if (s0 != PG_OK) return s0;
    Scalars h{};
    PG_CUDA(cudaMemcpyAsync(&h, E.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, E.stream));
    PG_CUDA(cudaStreamSynchronize(E.stream));
    if (E.fresh) h.dt_prev = end_time - h.t;
    h.end_time = end_time;
    h.done = 0;
    h.pad_ = 0;
    PG_CUDA(cudaMemcpyAsync(E.sc, &h, sizeof(Scalars), cudaMemcpyHostToDevice, E.stream));
    E.fresh = false;
    pg_status s;
    for (int k = 0; k < 2; ++k)
        if ((s = make_cell_maps(E.maps[k], E.buf[k], d.xarr, d.yarr)) != PG_OK) return s;
    if (d.visc && (s = make_vis_maps(E.vmap, E.vis, d.xarr, d.yarr)) != PG_OK) return s;
    pg_dust* const* D = E.dbuf;
    const bool dust = d.dust != 0;
    if (dust)
        for (int k = 0; k < 2; ++k)
            if ((s = make_dust_maps(E.dmaps[k], E.dbuf[k], d.xarr, d.yarr)) != PG_OK) return s;
    cudaEvent_t ev[7];
    for (auto& x : ev) PG_CUDA(cudaEventCreate(&x));
    for (int step = 0; step < nsteps; ++step) {
        int c = E.cur;
        PG_CUDA(cudaEventRecord(ev[0], E.stream));
        launch_time_step(d, E.stream);
        PG_CUDA(cudaEventRecord(ev[1], E.stream));
        launch_kick1(d, E.maps[c], E.buf[1 - c], E.vis, E.stream, dust ? D[c] : nullptr, dust ? D[1 - c] : nullptr,
                     &E.tune);
        c = 1 - c;
        PG_CUDA(cudaEventRecord(ev[2], E.stream));
        launch_sweep_x(d, E.maps[c], E.buf[1 - c], E.stream, &E.tune);
        if (dust) launch_dsweep_x(d, E.dmaps[c], D[1 - c], E.stream);
        c = 1 - c;
        PG_CUDA(cudaEventRecord(ev[3], E.stream));
        if (d.ndim > 1) {
            launch_sweep_y(d, E.maps[c], E.buf[1 - c], E.stream, &E.tune);
            if (dust) launch_dsweep_y(d, E.dmaps[c], D[1 - c], E.stream);
            c = 1 - c;
        }
        PG_CUDA(cudaEventRecord(ev[4], E.stream));
        if (d.ndim > 1 && d.orbadv) {
            launch_advect(d, E.maps[c], E.buf[1 - c], E.stream, &E.tune);
            if (dust) launch_dadvect(d, E.dmaps[c], D[1 - c], E.stream);
            c = 1 - c;
        }
        PG_CUDA(cudaEventRecord(ev[5], E.stream));
        launch_kick2(d, E.maps[c], E.vmap, E.buf[1 - c], E.stream, dust ? D[c] : nullptr, dust ? D[1 - c] : nullptr,
                     &E.tune);
        c = 1 - c;
        PG_CUDA(cudaEventRecord(ev[6], E.stream));
        PG_CUDA(cudaGetLastError());
        E.cur = c;
        PG_CUDA(cudaEventSynchronize(ev[6]));
        for (int k = 0; k < 6; ++k) {
            float t = 0.0f;
            PG_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
            ms[k] += t / (float)nsteps;
        }
    }
    for (auto& x : ev) cudaEventDestroy(x);
    return PG_OK;
}

// ------------------------------------------------------ drop-in (Grid)
static std::mutex g_mu;
static pg_params g_params;
static bool g_configured = false;
static std::map<const double*, Engine*> g_grids;  // keyed by the caller's device xa

pg_status pg_configure(const pg_params* P) {
    pg_status s = (P && P->ndim == 3) ? check_params3(P) : check_params(P);
    if (s != PG_OK) return s;
    std::lock_guard<std::mutex> lk(g_mu);
    g_params = *P;
    g_configured = true;
    return PG_OK;
}

static pg_status grid_engine(pg_grid* dev, Engine** out) {
    if (!dev) return fail(PG_ERR_ARG, "null grid");
    if (!g_configured) return fail(PG_ERR_CONFIG, "pg_configure was not called");
    if (dev->xres != g_params.xres || dev->yres != g_params.yres)
        return fail(PG_ERR_CONFIG, "grid dimensions differ from the configured parameters");
    if (dev->xbgn != 0) return fail(PG_ERR_CONFIG, "radial domain decomposition is not supported");
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_grids.find(dev->xa);
    if (it != g_grids.end()) {
        *out = it->second;
        return PG_OK;
    }
    int device = 0;
    PG_CUDA(cudaGetDevice(&device));
    Engine* E = nullptr;
    pg_status s = engine_create(&g_params, device, dev->stream, &E);
    if (s != PG_OK) return s;
    E->rot = dev->orb_rot;
    E->res = dev->orb_res;
    E->inc = dev->orb_inc;
    E->vis = dev->vis_tensor;
    if ((s = engine_setup(*E, dev->xa, dev->xv, dev->ya, dev->yv)) != PG_OK) {
        delete E;
        return s;
    }
    g_grids[dev->xa] = E;
    *out = E;
    return PG_OK;
}

pg_status pg_grid_init_orbadv(pg_grid* dev) {
    if (g_configured && g_params.ndim == 3) {
        std::lock_guard<std::mutex> lk(g_mu);
        return grid3_init_orbadv(g_params, dev);
    }
    Engine* E = nullptr;
    pg_status s = grid_engine(dev, &E);
    if (s != PG_OK) return s;
    // orb_rot was written by the table kernel of engine_setup; orb_shf starts at 0
    if (dev->orb_shf) PG_CUDA(cudaMemsetAsync(dev->orb_shf, 0, sizeof(int) * dev->xarr * dev->zarr, E->stream));
    PG_CUDA(cudaStreamSynchronize(E->stream));
    return PG_OK;
}

pg_status pg_grid_global_dt(pg_grid* hst, pg_grid* dev, double dt_prev, double* dt_out) {
    (void)hst;
    if (!dt_out) return fail(PG_ERR_ARG, "null dt_out");
    if (g_configured && g_params.ndim == 3) {
        std::lock_guard<std::mutex> lk(g_mu);
        return grid3_global_dt(g_params, dev, dt_prev, dt_out);
    }
    Engine* E = nullptr;
    pg_status s = grid_engine(dev, &E);
    if (s != PG_OK) return s;
    launch_cfl(E->view, reinterpret_cast<Cell*>(dev->C), E->stream, E->view.dust ? dev->CD : nullptr);
    PG_CUDA(cudaGetLastError());
    pg_disk tmp{E};
    return pg_disk_global_dt(&tmp, dt_prev, dt_out);
}

pg_status pg_grid_solve(pg_grid* dev, double time, double dt) {
    if (g_configured && g_params.ndim == 3) {
        std::lock_guard<std::mutex> lk(g_mu);
        return grid3_solve(g_params, dev, time, dt);
    }
    Engine* E = nullptr;
    pg_status s = grid_engine(dev, &E);
    if (s != PG_OK) return s;
    E->buf[0] = reinterpret_cast<Cell*>(dev->C);
    E->buf[1] = reinterpret_cast<Cell*>(dev->T);
    E->cur = 0;
    if ((s = ensure_ghosts(*E, E->buf[1])) != PG_OK) return s;
    // the caller may have written the state: refresh the ghost images first
    launch_bound(E->view, E->buf[0], E->stream);
    if (E->view.dust) {
        if (!dev->CD || !dev->TD) return fail(PG_ERR_ARG, "dust_flag needs the grid's CD and TD");
        E->dbuf[0] = dev->CD;
        E->dbuf[1] = dev->TD;
        for (pg_dust* b : {dev->CD, dev->TD}) {
            bool seen = false;
            for (const void* p : E->dghosted) seen = seen || p == b;
            if (!seen) {
                launch_dust_xghosts(E->view, b, E->stream);
                E->dghosted.push_back(b);
            }
        }
        launch_dust_images(E->view, dev->CD, E->stream);
    }
    if (E->view.nplanet > 0 && dev->planets)
        k_grid_planet_in<<<1, 1, 0, E->stream>>>(E->sc, dev->planets, E->view.twobd);
    launch_set_time(E->view, time, dt, E->stream);
    if ((s = enqueue_stages(*E)) != PG_OK) return s;
    if (E->view.nplanet > 0 && dev->planets)
        k_grid_planet_out<<<1, 1, 0, E->stream>>>(E->sc, dev->planets, E->view.twobd);
    PG_CUDA(cudaGetLastError());
    if (E->cur == 1) {  // newest state in T: swap like the reference (src/solver/sweeps.cu:353-355)
        pg_cell* t = dev->C;
        dev->C = dev->T;
        dev->T = t;
        if (E->view.dust) {  // the dust pairs with the gas (src/solver/dust/dust.cu:230-233)
            pg_dust* td = dev->CD;
            dev->CD = dev->TD;
            dev->TD = td;
        }
    }
    return PG_OK;
}

pg_status pg_grid_release(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& kv : g_grids) delete kv.second;
    g_grids.clear();
    grid3_release();
    return PG_OK;
}

}  // extern "C"
