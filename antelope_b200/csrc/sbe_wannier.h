// Device structures of the N-band (N <= 8) Wannier tight-binding solves,
// length gauge (SBEs.h:762-872 with a Wannier model, Materials/Wannier90.h:
// 297-387 model form).  One warp advances one k-point; a launch performs one
// attempted step of every k-point of the solve; a one-block controller kernel
// accepts or rejects it (Cash-Karp, one step size per solve) or always
// accepts (fixed-step RK4 / Fehlberg-5) and prepares the next attempt's stage
// fields.
#pragma once

#include <cuda_runtime.h>

namespace sbe {

constexpr int WAN_MAXN = 8;
constexpr int WAN_MAXR = 64;       // lattice vectors
constexpr int WAN_NSLOT = 16;      // inter x,y; intra x,y; occupations (N); coherence re, im; ...
constexpr int WAN_SLOT_INTER_Z = 14, WAN_SLOT_INTRA_Z = 15;   // ... z currents (N <= 8: past the others)
constexpr int WAN_WARPS = 4;       // warps (k-points) per CTA

struct PulseDev {
    double E0x, E0y, A0x, A0y, w0, cep, t0, twidth, twidth_clipped, envfactor;
    double xdir[3], ydir[3];
    int env;
};

constexpr int MAX_PULSES = 16;   // laser pulses a problem may have (device layout)

struct LaserDev {
    int npulses;
    PulseDev p[MAX_PULSES];
    double init_A[3], init_E[3];
};

struct WanCtl {
    double tc;          // time of the committed state
    double h;           // proposed step size
    double hs;          // step size of the next attempt
    double emax;        // error of the last attempt
    int n;              // output interval: the committed state is at t_n <= tc < t_{n+1}
    int buf;            // committed state buffer (0/1)
    int last;           // the next attempt ends the interval
    int need_current;   // the next attempt records the currents at tc = t_n first
    int done;
    int error;          // 1: step-size underflow / too many rejections
    int shot;           // output step whose density snapshot is due (the interval just completed), or -1
    long long steps, attempts, rejects;
};

struct WanDev {
    int N, nval, nR, nk, Nt, ntiles, rk, inter_intra, use_fermi, has_dip, has_jtab;
    int vg;                 // 1: velocity gauge (band basis), 0: length gauge (Wannier basis)
    // 1: the continuum MultiWSM model (Materials/MultiWSM.h): H and the
    // current operator from formulas at k + A instead of Fourier tables (nR = 0),
    // a z current; its parameters n, v, alphan
    int cont;
    double mw_n, mw_v, mw_alphan;
    int k_offset;           // flat grid index of local k-point 0 (a k-slice of the grid)
    double Ef, dt, atmin, tol, g1, g2;  // g1 = 1/T1, g2 = 1/T2 (0 when disabled)
    int Ngrid[3];
    double axes[9], origin[3];
    LaserDev laser;
    const double *V;        // [nR][2] hopping vectors, Cartesian (bohr)
    const void *h;          // [nR][N*N] complex, FP32 for the mixed method, FP64 otherwise
    const void *d;          // [nR][2][N*N] complex, same precision (or null)
    const void *jt;         // [nR][2][N*N] current-operator tables, same precision (or null:
                            // J_a = -dH/dk_a + i[D_a, H])
    // h and d re-laid for the grouped attempt kernel by lattice-vector pairs
    // (R, -R): [npair][NO][3][2][8] complex (NO = ceil(N(N+1)/2 / 8)), the pair
    // sum h_R + h_-R and i (h_R - h_-R) of quantity q (h, d_x, d_y) of upper
    // element l + 8 j; same precision; null: not used
    const void *gtab;
    const int *gpair;       // [npair] index of each pair's vector R (the other is -R)
    int npair;
    // with dipoles, per stage of the next attempt the pair table of
    // E_x(t_s) d_x + E_y(t_s) d_y ([6][npair][NO][2][8] complex, Fourier
    // precision), whose sum is E.D in one sum; written by the controller
    void *stage_gt;
    double2 *rho[2];        // [nk][N*N] committed / trial state (Wannier basis, full matrix), FP64
    double2 *U[2];          // [nk][N*N] tracked eigenbasis of H0(k+A), FP64
    double *weight;         // [nk]
    double *tile_err;       // [ntiles]
    double *cur_part;       // [ntiles][WAN_NSLOT]
    double *jout;           // [Nt][WAN_NSLOT]
    WanCtl *ctl;
    double *vg_eps;         // velocity gauge: [nk][N] band energies (ascending)
    double *vg_f;           // velocity gauge: [nk][N] initial occupations
    double2 *vg_P;          // velocity gauge: [nk][2 or 3 (cont)][N*N] P_a = U^dag J_a U
    double *stage_AE;       // [6][6] A and E at the stage times of the next attempt
    void *stage_cA;         // [6][nR] e^{i A(t_s) R} of the next attempt (Fourier precision)
    // density snapshots (antelope.cpp:340-422): every shot_every output steps
    // (0: none), per k the conduction occupation and coherence of rho after
    // the step, in the band basis (velocity gauge) or in the eigenbasis of
    // H0(k + A(t_n)) (length gauge); [nshots][nk] and [nshots][nk][2]
    int shot_every;
    double *snap_nc;
    double *snap_pi;
};

// A tile of a batched launch: tile `tile` (WAN_WARPS k-points) of solve
// `solve` of the launch's descriptor array.  Batches of N-band solves advance
// every solve of a launch class (same N, gauge and precision) with one
// attempt launch over all their tiles and one control launch with one block
// per solve, each solve keeping its own step-size controller.
struct WanTileRef {
    int solve, tile;
};

struct Laser;
// The laser of a problem in the device layout (throws CfgError beyond 8 pulses).
LaserDev laser_dev(const Laser &L);

// Field tables of the two-band kernels, computed on the device with the same
// laser evaluation as the N-band path: at t = (atmin + dt n) + c_j dt for the
// nts stage-time fractions c (c_0 = 0), either A_x, A_y ([Nt][nts][2], VG) or
// cos / sin of A.a_i and A.b_i ([Nt][nts][12], Haldane length gauge; a, b:
// the [3][2] vectors).  out: doubles (f32 = 0) or floats (f32 = 1).
cudaError_t launch_field_table(const LaserDev &L, double atmin, double dt, int Nt, int nts, const double *c,
                               bool vg, const double (*va)[2], const double (*vb)[2], void *out, bool f32,
                               cudaStream_t st);

size_t wan_smem_bytes(int N, int nR, int precision);
// The grouped attempt kernel (eight lanes per k-point) runs the length-gauge
// attempts of explicit tables with the -dH/dk + i[D, H] current operator at
// N = 4 and 6: wan_grouped_applies says whether a solve qualifies (before its
// re-laid tables exist), wan_grouped whether it runs on it; its blocks cover
// WAN_GROUP_TILES tiles, so batched tile lists of such a class are in blocks.
constexpr int WAN_GROUP_TILES = 4;
bool wan_grouped_applies(const WanDev &w);
bool wan_grouped(const WanDev &w);
// entries of the re-laid table per lattice-vector pair (complex numbers)
int wan_gtab_row(int N);
// lattice-vector pairs (R, -R) a grouped solve may have (its vectors pair up
// but for R = 0)
int wan_npair_cap(int nR);
cudaError_t launch_wan_init(const WanDev &w, int precision, cudaStream_t st);
cudaError_t launch_wan_prepare(const WanDev *dw, int precision, cudaStream_t st);
cudaError_t launch_wan_attempt(const WanDev &w, const WanDev *dw, int precision, cudaStream_t st);
cudaError_t launch_wan_control(const WanDev *dw, int precision, cudaStream_t st);
// the snapshot of the interval the last control step completed, if one is due
cudaError_t launch_wan_snapshot(const WanDev &w, const WanDev *dw, int precision, cudaStream_t st);
// Batched forms: `descs` [nsolves] device pointers to the solves' descriptors,
// `tiles` [ntiles] the tiles of all of them (device memory); N, nR_max and
// the gauge (vg) of the launch class size the shared memory and pick the
// instance.  Control: one block per solve.
// grouped_rk != 0: the class runs on the grouped kernel with that RK order
// (`tiles` then lists blocks of WAN_GROUP_TILES tiles: tile = the first one)
cudaError_t launch_wan_attempt_batch(int N, int nR_max, bool vg, const WanDev *const *descs, const WanTileRef *tiles,
                                     int ntiles, int precision, cudaStream_t st, int grouped_rk = 0);
cudaError_t launch_wan_control_batch(const WanDev *const *descs, int nsolves, int precision, cudaStream_t st);
cudaError_t launch_wan_snapshot_batch(int N, int nR_max, const WanDev *const *descs, const WanTileRef *tiles,
                                      int ntiles, int precision, cudaStream_t st);

}  // namespace sbe
