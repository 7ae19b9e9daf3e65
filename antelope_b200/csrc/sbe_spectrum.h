// Harmonic band powers of a solve's total current, computed on the GPU from
// the device-resident per-step sums (the analysis convention of the
// reference's AlsisPythonShort/AnalysisReader_PyDir.py:252-354 and
// IntegrateSpectrumOrder.py:57-70).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace sbe {

// Where the per-step sums live and how they assemble into J_a(t_n), a = x, y:
//   J_a(t_n) = (jout[n*stride + s_inter + a] + jout[n*stride + s_intra + a]
//               + sum_t cp[t*cp_stride + cp_slot + a] + nvw * A[n][a]) * dV
struct HarmonicsInput {
    const double *jout = nullptr;
    int stride = 0, s_inter = 0, s_intra = 2;
    const double *cp = nullptr;  // per-tile constant parts (device) or null
    int ntiles = 0, cp_stride = 0, cp_slot = 2;
    const double *A = nullptr;   // [nt][2] vector potential at t_n (device) or null
    double nvw = 0.0, dV = 1.0;
    int nt = 0;
    double dt = 0.1;
};

// Band powers P_h, h = 1..hmax: S(w) = sum_{x,y} |-i w FFT(blackman * J) dt|^2
// summed over the bins with h - 1/2 <= w / w0 < h + 1/2.  Synchronises `st`.
void harmonics_on_device(const HarmonicsInput &in, double w0, int hmax, double *band_power, cudaStream_t st);

}  // namespace sbe
