// Harmonic band powers on the GPU: the windowed current is assembled from the
// solve's per-step sums in place, then a direct DFT is taken at exactly the
// frequency bins the harmonic bands cover (a few hundred of the Nt bins), one
// CTA per bin with a fixed-order reduction; the band sums are formed on the
// host from those bins with the bin frequencies computed as numpy.fft.fftfreq
// computes them.  FP64 throughout; twiddles from exact integer phase
// reduction (j n mod Nt).
#include "sbe_spectrum.h"

#include <algorithm>
#include <cmath>
#include <string>

#include "sbe_engine.h"

namespace sbe {

namespace {

__global__ void assemble_window(HarmonicsInput in, double *x)
{
    __shared__ double cst[2];
    if (threadIdx.x < 2) {
        double c = 0.0;
        if (in.cp)
            for (int t = 0; t < in.ntiles; ++t) c += in.cp[(size_t)t * in.cp_stride + in.cp_slot + threadIdx.x];
        cst[threadIdx.x] = c;
    }
    __syncthreads();
    const int N = in.nt;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        // numpy.blackman(N): 0.42 - 0.5 cos(2 pi n/(N-1)) + 0.08 cos(4 pi n/(N-1))
        double w = 1.0;
        if (N > 1) {
            const double r = double(n) / double(N - 1);
            w = 0.42 - 0.5 * cospi(2.0 * r) + 0.08 * cospi(4.0 * r);
        }
        for (int a = 0; a < 2; ++a) {
            const double *row = in.jout + (size_t)n * in.stride;
            double J = row[in.s_inter + a] + row[in.s_intra + a] + cst[a];
            if (in.A) J += in.nvw * in.A[2 * (size_t)n + a];
            x[2 * (size_t)n + a] = w * (J * in.dV);
        }
    }
}

// one CTA per bin j0 + blockIdx.x: X_a = sum_n x_a[n] e^{-2 pi i j n / N}
__global__ void __launch_bounds__(256) dft_bins(const double *x, int N, int j0, double *re_im)
{
    __shared__ double red[4][256];
    const long long j = j0 + blockIdx.x;
    double r0 = 0, i0 = 0, r1 = 0, i1 = 0;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const long long m = (j * n) % N;
        double s, c;
        sincospi(2.0 * double(m) / double(N), &s, &c);
        const double x0 = x[2 * (size_t)n], x1 = x[2 * (size_t)n + 1];
        r0 = fma(x0, c, r0);
        i0 = fma(-x0, s, i0);
        r1 = fma(x1, c, r1);
        i1 = fma(-x1, s, i1);
    }
    red[0][threadIdx.x] = r0;
    red[1][threadIdx.x] = i0;
    red[2][threadIdx.x] = r1;
    red[3][threadIdx.x] = i1;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 4) re_im[4 * (size_t)blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

void harmonics_on_device(const HarmonicsInput &in, double w0, int hmax, double *band_power, cudaStream_t st)
{
    const int N = in.nt;
    if (N < 2 || hmax < 1 || !(w0 > 0.0)) throw CfgError("harmonics: need Nt >= 2, hmax >= 1, w0 > 0");
    // bins of the positive half of numpy.fft.fftfreq(N, dt): f_j = j * (1 / (N dt)),
    // j = 0 .. (N - 1) / 2; the bands need h - 1/2 <= 2 pi f_j / w0 < hmax + 1/2
    const double val = 1.0 / (N * in.dt), two_pi = 2 * 3.141592653589793;
    const int jmax = (N - 1) / 2;
    int j0 = jmax + 1, j1 = -1;
    for (int j = 0; j <= jmax; ++j) {
        const double order = two_pi * (j * val) / w0;
        if (order >= 0.5 && order < hmax + 0.5) {
            j0 = std::min(j0, j);
            j1 = j;
        }
    }
    for (int h = 0; h < hmax; ++h) band_power[h] = 0.0;
    if (j1 < j0) return;
    const int nb = j1 - j0 + 1;
    double *x = nullptr, *ri = nullptr;
    check(cudaMallocAsync(&x, sizeof(double) * 2 * (size_t)N, st), "harmonics: alloc");
    check(cudaMallocAsync(&ri, sizeof(double) * 4 * (size_t)nb, st), "harmonics: alloc");
    assemble_window<<<(N + 255) / 256, 256, 0, st>>>(in, x);
    check(cudaGetLastError(), "harmonics: assemble");
    dft_bins<<<nb, 256, 0, st>>>(x, N, j0, ri);
    check(cudaGetLastError(), "harmonics: dft");
    std::vector<double> h_ri(4 * (size_t)nb);
    check(cudaMemcpyAsync(h_ri.data(), ri, h_ri.size() * 8, cudaMemcpyDeviceToHost, st), "harmonics: copy");
    cudaFreeAsync(x, st);
    cudaFreeAsync(ri, st);
    check(cudaStreamSynchronize(st), "harmonics: sync");
    for (int b = 0; b < nb; ++b) {
        const int j = j0 + b;
        const double omega = two_pi * (j * val), order = omega / w0;
        const int h = (int)std::floor(order + 0.5);
        if (h < 1 || h > hmax || order < h - 0.5 || order >= h + 0.5) continue;
        // |-i w F|^2 with F = X dt, summed over x and y
        const double *v = &h_ri[4 * (size_t)b];
        const double f = omega * in.dt;
        band_power[h - 1] += f * f * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
    }
}

}  // namespace sbe
