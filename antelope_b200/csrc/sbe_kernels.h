// Launch interface between the host engine (sbe_engine.cpp) and the kernels.
#pragma once

#include <cuda_runtime.h>

#include "sbe_dev.h"

namespace sbe {

struct LaunchArgs {
    const TileDev *tiles;    // device array of the tiles to advance
    const SolveDev *solves;  // device array of solve descriptors
    int ntiles;              // grid size (one CTA per tile)
    int threads;             // CTA size: tile_k / kpt, multiple of 32, <= 256
    int tick, S;             // launch index and steps per launch
    int variant, precision, rk, kpt;
    bool has_g1;             // T1 dephasing active
    cudaStream_t stream;
};

struct InitArgs {
    int nk, nk_pad, tile_k, variant, nval, use_fermi;
    int k_offset;  // flat grid index of local k-point 0 (a k-slice of the grid)
    int N[3];
    double axes[9], origin[3];
    double t1, t2, M0, phi0, va[3][2], vb[3][2];
    double Ef, dt;
};

// largest CTA (threads) the propagate kernel of a class of solves accepts
int propagate_max_threads(int variant, int precision, int rk, int kpt);
cudaError_t launch_propagate(const LaunchArgs &la);
cudaError_t launch_reduce(const SolveDev *solves, const int *solve_ids, int nsolves, int tick, int S,
                          cudaStream_t stream);
cudaError_t launch_init_haldane(const InitArgs &ia, int precision, void *kc, void *st, double *constpart,
                                cudaStream_t stream);
// occ1d[nshots][N0] from the per-k snapshot values nc[nshots][nk] of a solve
// whose k-points are the flat grid indices [k_offset, k_offset + nk)
cudaError_t launch_snapshot_bins(const double *nc, int nk, int k_offset, const int N[3], int nshots, double *occ1d,
                                 cudaStream_t stream);
cudaError_t launch_fma_peak(int which, int blocks, int iters, void *out, cudaStream_t stream);

}  // namespace sbe
