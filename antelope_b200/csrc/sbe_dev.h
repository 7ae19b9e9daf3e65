// Device-side data layout shared by the host engine and the kernels.
//
// A *solve* is one propagation of one problem (one inputParam.cfg).  Its
// k-points are cut into *tiles* of at most `tile_k` consecutive flat k
// indices; one CTA owns one tile for a launch.  A launch ("tick") advances
// every listed tile by up to S time steps, so single solves, batched scans and
// the continuous-batching server all run the same kernels.
//
// Per-step outputs: every tile writes NSLOT doubles per step into the solve's
// partial buffer [S][ntiles][NSLOT]; a second kernel sums the tiles in tile
// order into jout[Nt][NSLOT].  No floating-point atomics are used, so a
// solve's result depends only on its own tiling, never on co-resident solves.
#pragma once

#include <stdint.h>

namespace sbe {

enum Variant : int {
    VAR_HALDANE_VG = 0,  // 2 bands, velocity gauge, rho stored as deviation from rho0 (band basis)
    VAR_HALDANE_LW = 1,  // 2 bands, length gauge, rho as Bloch vector (Wannier basis)
    VAR_WANNIER_LW = 2,  // N <= 8 bands, length gauge, N x N rho per k
};

enum Precision : int { PREC_FP64 = 0, PREC_MIXED = 1 };

constexpr int NSLOT = 8;   // reduced values per step (see slot map below)
constexpr int SUB = 16;    // steps staged in shared memory between tile reductions

// Slot map of jout / partial for the 2-band variants:
//   0,1: inter x,y   2,3: intra x,y   4,5: sum w rho_00, sum w rho_11
//   6,7: sum w Re rho_01, sum w Im rho_01
// (VG: the time-independent parts -- w rho0 P and w rho0 -- are kept
//  separately per solve and added on the host; VG's N_val*A term too.)

// Per-k constant arrays (structure of arrays, stride nk_pad), velocity gauge.
// All dynamical constants are pre-multiplied by the solve's dt so that the
// RK stage slopes come out as dt*f directly.
enum VgConst : int {
    VG_DE = 0,     // dt*(eps0 - eps1)
    VG_DPX, VG_DPY,  // dt*(P00 - P11) for x, y
    VG_PXR, VG_PXI, VG_PYR, VG_PYI,  // dt*P01 for x, y (re, im)
    VG_C0,         // rho0_11 - rho0_00
    VG_WPX0, VG_WPX1, VG_WPY0, VG_WPY1,  // w*P00, w*P11 for x, y
    VG_WQXR, VG_WQXI, VG_WQYR, VG_WQYI,  // 2*w*P01 for x, y (re, im)
    VG_W,          // w (trapezoid weight)
    VG_NCONST      // constants the propagate kernels hold in registers
};
// One more per-k value stored after those (not loaded by the propagate
// kernels): rho0_11, read only when a density snapshot is taken.
constexpr int VG_R11 = VG_NCONST, VG_NCONST_ALL = VG_NCONST + 1;
enum VgState : int { VG_DA = 0, VG_DB, VG_ZR, VG_ZI, VG_NSTATE };
// Three more FP64 rows after those: the packed mixed kernel's FP32 sum of the
// increments not yet folded into the state (folds happen at absolute step
// multiples of 8, so a run split into launches anywhere gives the same bits).
constexpr int VG_ACC = VG_NSTATE, VG_NSTATE_ALL = VG_NSTATE + 3;

// Length gauge, Haldane: per-k cos/sin of k.a_i and k.b_i, and the weight.
enum LwConst : int {
    LW_CA0 = 0, LW_CA1, LW_CA2, LW_SA0, LW_SA1, LW_SA2,
    LW_CB0, LW_CB1, LW_CB2, LW_SB0, LW_SB1, LW_SB2,
    LW_W, LW_NCONST
};
enum LwState : int { LW_AL = 0, LW_SX, LW_SY, LW_SZ, LW_NSTATE };
// the packed mixed kernel's unfolded FP32 increments of the four components
// (see propagate_lw_x2), kept after the state so that a launch split changes no bit
constexpr int LW_ACC = LW_NSTATE, LW_NSTATE_ALL = LW_NSTATE + 4;
// Phase table per stage time: cos(A.a_i) x3, sin(A.a_i) x3, cos(A.b_i) x3, sin(A.b_i) x3
constexpr int LW_NPHASE = 12;

struct SolveDev {
    int nk, ntiles, Nt, admit_tick;
    int nk_pad, nts, variant, precision;
    const void *kc;    // per-k constants [NC][nk_pad] (double for FP64, float for mixed)
    void *st;          // per-k state [NS][nk_pad] (same type)
    const void *tab;   // VG: A table [Nt][nts] of (x,y); LW: phase table [Nt][nts][12]
    double *partial;   // [S][ntiles][NSLOT]
    double *jout;      // [Nt][NSLOT]
    double g1, g2;     // dt/T1, dt/T2 (0 when disabled)
    // Haldane length gauge: dt-scaled field terms and the unscaled ones for J
    double t1dt, t2sdt, Mdt;      // dt*t1, dt*2*t2*sin(phi0), dt*M0
    double t1, t2c, t2s;          // t1, 2*t2*cos(phi0), 2*t2*sin(phi0)
    double va[3][2], vb[3][2];    // NN and NNN vectors (bohr)
    int *status;                  // device status word (0 = ok)
    // density snapshots (antelope.cpp:340-422): after every step s with
    // s % shot_every == 0 the kernels store, per k, the conduction occupation
    // snap_nc[s / shot_every][k] and the coherence snap_pi[..][k] (re, im) of
    // rho in the band basis (VG) or in the eigenbasis of H0(k + A(t_s)) (LW);
    // shot_every = 0: none
    int shot_every;
    double *snap_nc;   // [nshots][nk]
    double *snap_pi;   // [nshots][nk][2]
};

struct TileDev {
    int solve;   // index into the SolveDev array
    int k0;      // first flat k index of the tile
    int kcount;  // number of k-points in the tile
    int tile;    // tile index within its solve (partial-buffer row)
};

}  // namespace sbe
