// The reference's own 4th-order PPM slopes on given data -- TEST INFRASTRUCTURE.
//
// Linked against the reference's unmodified object files (built by
// oracle/ref_build.py; the solver object holds get_4th_parameters,
// src/solver/recon/recon.cu:216-378, compiled for sm_100a with relocatable
// device code), this program evaluates that function for every index of a
// pencil of face coordinates and cell averages read from a file, and writes
// the three parameters (sL, a, sR) per index.  Used to compare the library's
// per-index slope weights with what the reference computes on the same grid.
//
//   slopes <in file> <out file>
//   in:  int32 n, int32 geom, double x[n + 1], int32 m, double a[m][n]  (m data rows)
//   out: double par[m][n][3] (zero where the 6 faces of the fit are not all there)
#include <cstdio>
#include <cstdlib>
#include <vector>

__device__ void get_4th_parameters(int i, int geom, double* x, double* dx, double* dv, double* a, double* par);

__global__ void k_slopes(const double* x, const double* a, int n, int m, int geom, double* out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * m) return;
    const int row = (int)(t / n), i = (int)(t % n);
    double* o = out + 3 * t;
    o[0] = o[1] = o[2] = 0.0;
    if (i < 2 || i + 3 > n) return;
    double par[3];
    get_4th_parameters(i, geom, const_cast<double*>(x), nullptr, nullptr, const_cast<double*>(a) + (size_t)row * n, par);
    o[0] = par[0];
    o[1] = par[1];
    o[2] = par[2];
}

static void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error in %s: %s\n", what, cudaGetErrorString(e));
        std::exit(2);
    }
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: slopes <in> <out>\n");
        return 1;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int n = 0, geom = 0, m = 0;
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&geom, 4, 1, f) != 1 || n < 1 || n > (1 << 24)) return 1;
    std::vector<double> x(n + 1);
    if (std::fread(x.data(), 8, n + 1, f) != (size_t)(n + 1) || std::fread(&m, 4, 1, f) != 1 || m < 1 || m > 64)
        return 1;
    std::vector<double> a((size_t)m * n);
    if (std::fread(a.data(), 8, a.size(), f) != a.size()) return 1;
    std::fclose(f);
    double *dx, *da, *dout;
    check(cudaMalloc(&dx, 8 * x.size()), "malloc");
    check(cudaMalloc(&da, 8 * a.size()), "malloc");
    check(cudaMalloc(&dout, 8 * 3 * a.size()), "malloc");
    check(cudaMemcpy(dx, x.data(), 8 * x.size(), cudaMemcpyHostToDevice), "copy");
    check(cudaMemcpy(da, a.data(), 8 * a.size(), cudaMemcpyHostToDevice), "copy");
    const long long total = (long long)n * m;
    k_slopes<<<(unsigned)((total + 127) / 128), 128>>>(dx, da, n, m, geom, dout);
    check(cudaGetLastError(), "launch");
    check(cudaDeviceSynchronize(), "kernel");
    std::vector<double> out(3 * a.size());
    check(cudaMemcpy(out.data(), dout, 8 * out.size(), cudaMemcpyDeviceToHost), "copy back");
    FILE* g = std::fopen(argv[2], "wb");
    if (!g) return 1;
    std::fwrite(out.data(), 8, out.size(), g);
    std::fclose(g);
    cudaFree(dx);
    cudaFree(da);
    cudaFree(dout);
    return 0;
}
