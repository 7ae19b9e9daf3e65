// One N-band Wannier solve (length gauge) on the GPU; see sbe_wannier.cu.
#pragma once

#include <cuda_runtime.h>

#include "sbe_engine.h"
#include "sbe_wannier.h"

namespace sbe {

class WannierSolve {
public:
    WannierSolve(const Problem &p, int precision, int device, cudaStream_t st);
    ~WannierSolve();
    WannierSolve(const WannierSolve &) = delete;
    WannierSolve &operator=(const WannierSolve &) = delete;
    // Run every attempted step on `st` (returns when the solve is done).
    void run(cudaStream_t st);
    SolveOutputs outputs();
    // harmonic band powers h = 1..hmax from the device-resident sums
    void harmonics(double w0, int hmax, double *band_power);
    int launches() const { return launches_; }
    const WanCtl &control() const { return *h_ctl_; }

private:
    Problem prob_;
    int precision_, device_;
    cudaStream_t stream_;
    WanDev w_{};
    WanDev *d_w_ = nullptr;
    WanCtl *h_ctl_ = nullptr;
    int launches_ = 0;
};

}  // namespace sbe
