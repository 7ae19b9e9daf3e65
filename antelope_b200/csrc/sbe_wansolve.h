// One N-band Wannier solve (length gauge) on the GPU; see sbe_wannier.cu.
#pragma once

#include <cuda_runtime.h>

#include "sbe_engine.h"
#include "sbe_wannier.h"

namespace sbe {

class WannierSolve {
public:
    // k_begin/k_end: a k-slice [k_begin, k_end) of the grid (0, 0: all of it)
    WannierSolve(const Problem &p, int precision, int device, cudaStream_t st, int k_begin = 0, int k_end = 0);
    ~WannierSolve();
    WannierSolve(const WannierSolve &) = delete;
    WannierSolve &operator=(const WannierSolve &) = delete;
    // Run every attempted step on `st` (returns when the solve is done).
    void run(cudaStream_t st);
    SolveOutputs outputs();
    // per-step sums [Nt][WAN_NSLOT] of this solve's k-points (host copy)
    std::vector<double> sums();
    // harmonic band powers h = 1..hmax from the device-resident sums
    void harmonics(double w0, int hmax, double *band_power);
    // density snapshots (as Engine::snapshots); returns their number
    int snapshots(double *occ1d, double *nc, double *pi);
    int launches() const { return launches_; }
    const WanCtl &control() const { return *h_ctl_; }

private:
    Problem prob_;
    int precision_, device_, nshots_ = 0;
    cudaStream_t stream_;
    WanDev w_{};
    WanDev *d_w_ = nullptr;
    WanCtl *h_ctl_ = nullptr;
    int launches_ = 0;
};

// The reference's output arrays of a table model from its per-step sums
// [Nt][WAN_NSLOT] (possibly summed over k-slices; antelope.cpp:514-548).
void assemble_table_outputs(const Problem &p, const std::vector<double> &sums, SolveOutputs &o);

}  // namespace sbe
