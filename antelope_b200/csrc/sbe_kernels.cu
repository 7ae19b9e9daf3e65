// sm_100a kernels of the SBE propagator.
//
//   init_haldane      per-k set-up: k-grid point and trapezoid weight
//                     (momaxis.h:147-186, 349-383), H0(k) and J(k)
//                     (Haldane.h:86-127), closed-form 2x2 eigensystem standing
//                     in for zheevr, rho0 (SBEs.h:319-356) and P = U^dag J U
//                     (SBEs.h:366-372).
//   propagate_vg      velocity gauge, 2 bands: one thread per k-point (or
//                     KPT of them), rho in registers for every step of the
//                     launch, RK4 or fixed-step Fehlberg-5 (SBEs.h:395-416,
//                     596-624) of dRho/dt = -i[H,rho] - G o (rho - rho0)
//                     (SBEs.h:787-805, 862-871), fused with the per-step
//                     weighted k-sum of the currents and occupations
//                     (SBEs.h:694-760, antelope.cpp:302-334).
//   propagate_lw      length gauge, 2 bands (Haldane): H0(k+A) in place,
//                     dephasing in the instantaneous eigenbasis (SBEs.h:762-
//                     786, 831-861), written for the Bloch vector of rho.
//   reduce_tiles      deterministic second pass: tile partials -> per-step sums.
//
// Precision: every kernel is a template on Real.  Real = double is the plain
// FP64 method.  Real = float is the mixed method: the RK stages and the step
// increment in FP32, the per-k state kept in FP64 (the increment is added in
// FP64 once per step -- rounding the state itself to FP32 every step is what
// limits an all-FP32 propagation), the A(t) table computed in FP64 on the
// host and rounded per stage, and the k-sum of the currents accumulated in
// FP64 from the warp level up.  In the velocity gauge the state is the
// deviation rho - rho0, and the time-independent rho0 parts of the currents
// are summed once, in FP64.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <type_traits>

#include "sbe_dev.h"
#include "sbe_kernels.h"

namespace sbe {

// ------------------------------------------------------------ RK tableaux
// Butcher tableaux of SBEs.h:395-416.  The stage slopes carry the factor dt
// (all per-k constants are dt-scaled), so only the pure coefficients appear.
// ti(i): the field-table column of stage i; END: the column at t + dt, whose
// field terms are the next step's terms at its own start.
template <int RK> struct Tableau;
template <> struct Tableau<4> {
    static constexpr int S = 4, NT = 3, END = 2;
    __device__ static constexpr double a(int i, int j)
    {
        return (i == 1 && j == 0) ? 0.5 : (i == 2 && j == 1) ? 0.5 : (i == 3 && j == 2) ? 1.0 : 0.0;
    }
    __device__ static constexpr double b(int i)
    {
        return (i == 0 || i == 3) ? 1.0 / 6.0 : 2.0 / 6.0;
    }
    __device__ static constexpr int ti(int i) { return i == 0 ? 0 : (i == 3 ? 2 : 1); }
};
template <> struct Tableau<5> {  // Fehlberg tableau with its 5th-order weights
    static constexpr int S = 6, NT = 6, END = 4;
    __device__ static constexpr double a(int i, int j)
    {
        return i == 1 ? (j == 0 ? 1.0 / 4.0 : 0.0)
             : i == 2 ? (j == 0 ? 3. / 32. : j == 1 ? 9. / 32. : 0.0)
             : i == 3 ? (j == 0 ? 1932. / 2197. : j == 1 ? -7200. / 2197. : j == 2 ? 7296. / 2197. : 0.0)
             : i == 4 ? (j == 0 ? 439. / 216. : j == 1 ? -8. : j == 2 ? 3680. / 513. : j == 3 ? -845. / 4104. : 0.0)
             : i == 5 ? (j == 0 ? -8. / 27. : j == 1 ? 2. : j == 2 ? -3544. / 2565 : j == 3 ? 1859. / 4104
                        : j == 4 ? -11. / 40. : 0.0)
             : 0.0;
    }
    __device__ static constexpr double b(int i)
    {
        return i == 0 ? 16. / 135. : i == 1 ? 0.0 : i == 2 ? 6656. / 12825. : i == 3 ? 28561. / 56430.
             : i == 4 ? -9. / 50. : 2. / 55.;
    }
    __device__ static constexpr int ti(int i) { return i; }
};

// ------------------------------------------------------ density snapshots
// Snapshots follow the steps s = 0, F, 2F, ... (antelope.cpp:340-342); the
// first one at or after a launch's first step s0.
__device__ __forceinline__ int first_shot(int s0, int F)
{
    return F > 0 ? ((s0 + F - 1) / F) * F : 0x7fffffff;
}

// Velocity gauge: rho_11 = rho0_11 + db = rho0_11 - da and rho_10 = conj(z)
// in the band basis, the elements the reference reads at index Nval*N + Nval
// and Nval*N + Nval - 1 (antelope.cpp:391-398).
__device__ __forceinline__ void vg_snapshot(const SolveDev &sd, int s, int k, double r11, double da, double zr,
                                            double zi)
{
    const size_t i = (size_t)(s / sd.shot_every) * sd.nk + k;
    sd.snap_nc[i] = r11 - da;
    sd.snap_pi[2 * i] = zr;
    sd.snap_pi[2 * i + 1] = -zi;
}

// ---------------------------------------------- packed FP32 (f32x2) math
// Two k-points per thread share every instruction: .x belongs to the first,
// .y to the second (PTX f32x2 arithmetic, sm_100+).
__device__ __forceinline__ unsigned long long pk(float2 a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r)
{
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
    return upk(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
}
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }

template <class Real> struct V2;
template <> struct V2<double> { using T = double2; };
template <> struct V2<float> { using T = float2; };

// ---------------------------------------------------- warp reduce-scatter
// Sums 8 doubles over the 32 lanes of a warp.  Three halving exchanges leave
// each lane with one partially summed value (index lane>>2 for lanes that are
// multiples of 4), two more exchanges finish it: 9 shuffles instead of 40.
// The pattern is fixed, so the result is deterministic.
template <class T>
__device__ __forceinline__ T warp_sum8(const T (&v)[8], int lane)
{
    const bool h4 = lane & 16, h2 = lane & 8, h1 = lane & 4;
    T u[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        T send = h4 ? v[i] : v[i + 4];
        T keep = h4 ? v[i + 4] : v[i];
        u[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    T x[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        T send = h2 ? u[i] : u[i + 2];
        T keep = h2 ? u[i + 2] : u[i];
        x[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    T send = h1 ? x[0] : x[1];
    T y = (h1 ? x[1] : x[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
    y += __shfl_xor_sync(0xffffffffu, y, 2);
    y += __shfl_xor_sync(0xffffffffu, y, 1);
    return y;  // lanes 4*i hold the sum of v[i]
}

constexpr int MAX_WARPS = 8;

// Per-step tile reduction staged through shared memory: each warp deposits
// its 8 sums per step; every SUB steps (and at the end of the launch) the
// block sums over warps and writes one row of the partial buffer per step.
// The staging area has two halves used in turn, so one barrier per flush
// suffices: a warp writes a half again only after the next flush's barrier,
// which every thread reaches after finishing its reads of that half.  A
// kernel sizes the area by its own warp count in dynamic shared memory
// (red_stage_bytes), so that small tiles leave the SM's L1 to the table
// reads, or declares the fixed 8-warp RedStage.
using RedStage = double[2][SUB][MAX_WARPS][NSLOT];

constexpr int red_stage_bytes(int threads) { return 2 * SUB * (threads / 32) * NSLOT * (int)sizeof(double); }

struct TileReducer {
    double *red;
    int nw, half;   // warp stride of the area, half in use
    __device__ __forceinline__ explicit TileReducer(RedStage &s) : red(&s[0][0][0][0]), nw(MAX_WARPS), half(0) {}
    __device__ __forceinline__ TileReducer(double *s, int nwarps) : red(s), nw(nwarps), half(0) {}
    __device__ __forceinline__ double &at(int h, int r, int w, int slot)
    {
        return red[((h * SUB + r) * nw + w) * NSLOT + slot];
    }
    __device__ __forceinline__ void put(double y, int r)
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if ((lane & 3) == 0) at(half, r, warp, lane >> 2) = y;
    }
    __device__ __forceinline__ void push(const double (&v)[8], int r)
    {
        put(warp_sum8<double>(v, threadIdx.x & 31), r);
    }
    __device__ __forceinline__ void flush(int nrows, int row0, int ntiles, int tile, double *partial)
    {
        __syncthreads();
        const int nwarp = blockDim.x >> 5;
        for (int idx = threadIdx.x; idx < nrows * NSLOT; idx += blockDim.x) {
            const int row = idx / NSLOT, slot = idx % NSLOT;
            double acc = 0.0;
            for (int w = 0; w < nwarp; ++w) acc += at(half, row, w, slot);
            partial[((size_t)(row0 + row) * ntiles + tile) * NSLOT + slot] = acc;
        }
        half ^= 1;
    }
};

// ------------------------------------------------------ velocity gauge
// The state is rho - rho0 in the band basis: (da, db, z) = (drho_00,
// drho_11, rho_01).  Starting from rho = rho0, d(db)/dt = -d(da)/dt term by
// term (SBEs.h:787-805 with Hermitian rho), and every floating-point
// operation on db is the sign-mirrored operation on da; round-to-nearest is
// symmetric under negation, so db == -da holds bit for bit at every stage.
// The kernels therefore carry three components (da, Re z, Im z) and use -da
// wherever the reference's arithmetic reads db.
enum VgDof : int { D_DA = 0, D_ZR, D_ZI, D_N };

// Field terms of the velocity-gauge Hamiltonian at one stage time:
// dt (h0 - h1) and dt w = dt A.P01 (SBEs.h:787-805 with H = diag eps + A.P).
// They depend on the stage time only through A, so a step evaluates them once
// per distinct stage time (RK4: t, t + dt/2, t + dt), and the terms at t + dt
// serve again as the next step's terms at its start.
template <class Real> struct VgField { Real d, wr, wi; };

// Table entry of the field at the start of step s0: step 0 starts at t_min;
// every later step s starts with the field of step s-1 at t_{s-1} + dt, which
// the host evaluated at that sum (SBEs.h:612) -- the reference's own start
// time t_s = t_min + s dt (antelope.cpp:299) differs from it by at most an
// ulp of t.  Loading that same entry when a launch begins at s0 makes the
// result independent of where launches split the time loop.
template <class TB>
__device__ __forceinline__ size_t vg_start_row(int s0)
{
    return s0 == 0 ? 0 : (size_t)(s0 - 1) * TB::NT + TB::END;
}

template <class Real>
__device__ __forceinline__ VgField<Real> vg_field(const Real (&c)[VG_NCONST], typename V2<Real>::T A)
{
    return {fma(A.y, c[VG_DPY], fma(A.x, c[VG_DPX], c[VG_DE])), fma(A.y, c[VG_PYR], A.x * c[VG_PXR]),
            fma(A.y, c[VG_PYI], A.x * c[VG_PXI])};
}

// The factor 2 of 2 Im(w z*) and of (rho_11 - rho_00) w is folded into the
// constants: the kernel doubles the P01 coefficients (so h.wr, h.wi hold
// 2 dt w) and halves c0.  Scaling by 2 is exact and commutes with rounding,
// so every result is bit for bit that of the unscaled arithmetic, one
// multiplication per right-hand side cheaper.
template <class Real, bool G1>
__device__ __forceinline__ void vg_rhs(const VgField<Real> &h, Real hc0, const Real (&y)[D_N], Real g1, Real g2,
                                       Real (&k)[D_N])
{
    const Real im2 = fma(h.wi, y[D_ZR], -(h.wr * y[D_ZI]));   // 2 Im(w z*)
    k[D_DA] = G1 ? fma(-g1, y[D_DA], im2) : im2;
    const Real hbma = hc0 - y[D_DA];                         // (rho_11 - rho_00) / 2 = (c0 + db - da) / 2
    const Real xr = fma(hbma, h.wr, h.d * y[D_ZR]);
    const Real xi = fma(hbma, h.wi, h.d * y[D_ZI]);
    k[D_ZR] = fma(-g2, y[D_ZR], xi);                           // -i X - g2 z
    k[D_ZI] = fma(-g2, y[D_ZI], -xr);
}

// RK4 fits in 128 registers without spilling (4 CTAs of 128 threads per SM
// instead of 3 at the compiler's unbounded choice); Fehlberg-5 would spill.
// RK4 CTAs may have up to 512 threads at the same 128 registers, so that the
// autotuner can choose a tile count that fills the last wave of CTAs.
template <class Real, int RK, int KPT, bool G1>
__global__ void __launch_bounds__(RK == 4 ? 512 : 256, 1) propagate_vg(const TileDev *__restrict__ tiles,
                                                    const SolveDev *__restrict__ solves, int tick, int S)
{
    using T2 = typename V2<Real>::T;
    using TB = Tableau<RK>;
    constexpr bool F64 = std::is_same<Real, double>::value;
    extern __shared__ double red_dyn[];   // red_stage_bytes(blockDim.x)
    const TileDev tl = tiles[blockIdx.x];
    const SolveDev &sd = solves[tl.solve];
    const int s0 = (tick - sd.admit_tick) * S;
    const int Nt = sd.Nt;
    if (s0 < 0 || s0 >= Nt) return;
    const int s1 = min(s0 + S, Nt);
    const int nkp = sd.nk_pad, ntiles = sd.ntiles;
    const Real *__restrict__ kc = static_cast<const Real *>(sd.kc);
    double *__restrict__ st = static_cast<double *>(sd.st);
    const T2 *__restrict__ tab = static_cast<const T2 *>(sd.tab);
    const Real g1 = Real(sd.g1), g2 = Real(sd.g2);
    double *partial = sd.partial;

    // the state (rho - rho0) is kept in FP64 in both methods; the mixed
    // method rounds it to FP32 once per step for the stage arithmetic and
    // adds the FP32 step increment back in FP64
    constexpr int slot[D_N] = {VG_DA, VG_ZR, VG_ZI};
    Real c[KPT][VG_NCONST];
    double y64[KPT][D_N];
    int kidx[KPT];
    bool ok[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        const int local = threadIdx.x + j * blockDim.x;
        ok[j] = local < tl.kcount;
        kidx[j] = tl.k0 + local;
#pragma unroll
        for (int q = 0; q < VG_NCONST; ++q) c[j][q] = ok[j] ? kc[(size_t)q * nkp + kidx[j]] : Real(0);
#pragma unroll
        for (int q = VG_PXR; q <= VG_PYI; ++q) c[j][q] = c[j][q] + c[j][q];   // see vg_rhs
        c[j][VG_C0] = c[j][VG_C0] * Real(0.5);
#pragma unroll
        for (int q = 0; q < D_N; ++q) y64[j][q] = ok[j] ? st[(size_t)slot[q] * nkp + kidx[j]] : 0.0;
    }
    TileReducer red(red_dyn, blockDim.x >> 5);
    // field terms at the start of the launch's first step (see vg_start_row)
    VgField<Real> hstart[KPT];
    {
        const T2 A0 = __ldg(tab + vg_start_row<TB>(s0));
#pragma unroll
        for (int j = 0; j < KPT; ++j) hstart[j] = vg_field<Real>(c[j], A0);
    }
    int next_shot = first_shot(s0, sd.shot_every);

    for (int s = s0; s < s1; ++s) {
        Real y0[KPT][D_N];
#pragma unroll
        for (int j = 0; j < KPT; ++j)
#pragma unroll
            for (int q = 0; q < D_N; ++q) y0[j][q] = Real(y64[j][q]);
        // currents and occupations at t_s, before rho advances (antelope.cpp:309-334)
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = 0.0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const Real *cc = c[j];
            const Real *yy = y0[j];
            const Real db = -yy[D_DA];
            v[0] += double(fma(yy[D_ZR], cc[VG_WQXR], yy[D_ZI] * cc[VG_WQXI]));
            v[1] += double(fma(yy[D_ZR], cc[VG_WQYR], yy[D_ZI] * cc[VG_WQYI]));
            v[2] += double(fma(yy[D_DA], cc[VG_WPX0], db * cc[VG_WPX1]));
            v[3] += double(fma(yy[D_DA], cc[VG_WPY0], db * cc[VG_WPY1]));
            v[4] += double(cc[VG_W] * yy[D_DA]);
            v[6] += double(cc[VG_W] * yy[D_ZR]);
            v[7] += double(cc[VG_W] * yy[D_ZI]);
        }
        v[5] = -v[4];
        const int r = (s - s0) % SUB;
        red.push(v, r);

        // one RK step of the thread's k-points, stage by stage so that their
        // independent dependency chains interleave
        T2 A[TB::NT];
#pragma unroll
        for (int i = 1; i < TB::NT; ++i) A[i] = __ldg(tab + (size_t)s * TB::NT + i);
        VgField<Real> h[KPT][TB::NT];
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            h[j][0] = hstart[j];
#pragma unroll
            for (int i = 1; i < TB::NT; ++i) h[j][i] = vg_field<Real>(c[j], A[i]);
            hstart[j] = h[j][TB::END];
        }
        // FP64: acc = rho + sum_i dt b_i k_i in the reference's order
        // (SBEs.h:614-623); mixed: the sum is formed in FP32 first
        Real kk[KPT][TB::S][D_N], acc[KPT][D_N];
#pragma unroll
        for (int j = 0; j < KPT; ++j)
#pragma unroll
            for (int q = 0; q < D_N; ++q) acc[j][q] = F64 ? y0[j][q] : Real(0);
#pragma unroll
        for (int i = 0; i < TB::S; ++i) {
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                Real y[D_N];
#pragma unroll
                for (int q = 0; q < D_N; ++q) {
                    Real t = y0[j][q];
#pragma unroll
                    for (int m = 0; m < i; ++m)
                        if (TB::a(i, m) != 0.0) t = fma(Real(TB::a(i, m)), kk[j][m][q], t);
                    y[q] = t;
                }
                vg_rhs<Real, G1>(h[j][TB::ti(i)], c[j][VG_C0], y, g1, g2, kk[j][i]);
                if (TB::b(i) != 0.0) {
#pragma unroll
                    for (int q = 0; q < D_N; ++q) acc[j][q] = fma(Real(TB::b(i)), kk[j][i][q], acc[j][q]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j)
#pragma unroll
            for (int q = 0; q < D_N; ++q) y64[j][q] = F64 ? double(acc[j][q]) : y64[j][q] + double(acc[j][q]);
        if (s == next_shot) {   // density snapshot of the state after step s
#pragma unroll
            for (int j = 0; j < KPT; ++j)
                if (ok[j])
                    vg_snapshot(sd, s, kidx[j], double(kc[(size_t)VG_R11 * nkp + kidx[j]]), y64[j][D_DA],
                                y64[j][D_ZR], y64[j][D_ZI]);
            next_shot += sd.shot_every;
        }
        // the staged sums reach the partial buffer after the step's arithmetic,
        // so the warp reduction above can overlap it
        if (r == SUB - 1 || s == s1 - 1) red.flush(r + 1, s - r - s0, ntiles, tl.tile, partial);
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j)
        if (ok[j]) {
#pragma unroll
            for (int q = 0; q < D_N; ++q) st[(size_t)slot[q] * nkp + kidx[j]] = y64[j][q];
            st[(size_t)VG_DB * nkp + kidx[j]] = -y64[j][D_DA];
        }
}

// Mixed method, velocity gauge, two k-points per thread packed into f32x2
// registers: every RK instruction advances both.  The state stays FP64.
//
// The per-step current sums are reduced over the warp through shared memory
// instead of a shuffle butterfly: each lane writes its 7 pair-summed values
// (FP32) for the step into the warp's stage, and every XSTEP steps the warp
// sums the staged rows -- lane l owns row (l & 15) >> 1, slot group l & 1,
// and half l >> 4 of the source lanes, adds its 16 sources in FP32 (stage
// rows are 33 float4s long, so the 8 lanes of each 16-byte load phase read 8
// different bank groups), one shuffle adds the halves (64 k-points per FP32 sum, as a
// warp butterfly would), and the FP64 value goes to the block stage that is
// summed over warps every SUB steps.  Per step that costs two 16-byte stores
// instead of 9 shuffles, 9 adds and 14 selects.
constexpr int XSTEP = 8;                                // steps per warp-stage flush
constexpr int XROW = 33;                                // float4s per stage row (32 lanes + 1 pad)
constexpr int XSTAGE_F4 = XSTEP * 2 * XROW;             // float4s per warp stage
constexpr int xstage_bytes(int threads) { return (threads / 32) * XSTAGE_F4 * 16; }

// Packed field terms and right-hand side on (da, Re z, Im z) of two
// k-points.  The factor 2 of 2 Im(w z*) and of (rho_11 - rho_00) w is folded
// into w (cw = 2 w, hc0 = c0 / 2: exact power-of-two scalings), and the Im z
// slope is produced with the opposite sign (nzi = -dt dIm z/dt) so that no
// operand needs negating; the stage and step combinations apply that sign
// through their coefficients.
struct VgField2 { float2 d, cwr, cwi; };   // dt (h0 - h1), 2 dt Re w, 2 dt Im w

__device__ __forceinline__ VgField2 vg_field2(const float2 (&c)[VG_NCONST], float2 A)
{
    const float2 ax = bc2(A.x), ay = bc2(A.y);
    return {fma2(ay, c[VG_DPY], fma2(ax, c[VG_DPX], c[VG_DE])), fma2(ay, c[VG_PYR], mul2(ax, c[VG_PXR])),
            fma2(ay, c[VG_PYI], mul2(ax, c[VG_PXI]))};
}

template <bool G1>
__device__ __forceinline__ void vg_rhs2(const VgField2 &h, float2 hc0, const float2 (&y)[D_N], float2 ng1,
                                        float2 ng2, float2 g2, float2 (&k)[D_N])
{
    const float2 im2 = sub2(mul2(h.cwi, y[D_ZR]), mul2(h.cwr, y[D_ZI]));  // 2 Im(w z*)
    k[D_DA] = G1 ? fma2(ng1, y[D_DA], im2) : im2;
    const float2 hbma = sub2(hc0, y[D_DA]);                               // (rho_11 - rho_00) / 2
    k[D_ZR] = fma2(hbma, h.cwi, fma2(h.d, y[D_ZI], mul2(ng2, y[D_ZR])));
    k[D_ZI] = fma2(hbma, h.cwr, fma2(h.d, y[D_ZR], mul2(g2, y[D_ZI])));  // negated slope
}

template <int RK, bool G1>
__global__ void __launch_bounds__(256) propagate_vg_x2(const TileDev *__restrict__ tiles,
                                                       const SolveDev *__restrict__ solves, int tick, int S)
{
    using TB = Tableau<RK>;
    __shared__ RedStage red_s;
    extern __shared__ float4 xstage_all[];
    const TileDev tl = tiles[blockIdx.x];
    const SolveDev &sd = solves[tl.solve];
    const int s0 = (tick - sd.admit_tick) * S;
    const int Nt = sd.Nt;
    if (s0 < 0 || s0 >= Nt) return;
    const int s1 = min(s0 + S, Nt);
    const int nkp = sd.nk_pad, ntiles = sd.ntiles;
    const float *__restrict__ kc = static_cast<const float *>(sd.kc);
    double *__restrict__ st = static_cast<double *>(sd.st);
    const float2 *__restrict__ tab = static_cast<const float2 *>(sd.tab);
    const float2 ng1 = bc2(-float(sd.g1)), ng2 = bc2(-float(sd.g2)), g2 = bc2(float(sd.g2));
    double *partial = sd.partial;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float4 *const xst = xstage_all + warp * XSTAGE_F4;   // this warp's stage [XSTEP][2][32]
    constexpr int slot[D_N] = {VG_DA, VG_ZR, VG_ZI};
    // sign of each component's slope as produced by vg_rhs2
    constexpr float sg[D_N] = {1.f, 1.f, -1.f};

    const int l0 = threadIdx.x, l1 = threadIdx.x + blockDim.x;
    const bool ok0 = l0 < tl.kcount, ok1 = l1 < tl.kcount;
    const int k0 = tl.k0 + l0, k1 = tl.k0 + l1;
    float2 c[VG_NCONST];
    double y64[2][D_N];
#pragma unroll
    for (int q = 0; q < VG_NCONST; ++q)
        c[q] = make_float2(ok0 ? kc[(size_t)q * nkp + k0] : 0.f, ok1 ? kc[(size_t)q * nkp + k1] : 0.f);
    // derived constants: 2 w's coefficients, c0 / 2, and the intra-current
    // weights of da alone (w P00 - w P11, since db = -da)
#pragma unroll
    for (int q = VG_PXR; q <= VG_PYI; ++q) c[q] = add2(c[q], c[q]);
    c[VG_C0] = mul2(c[VG_C0], bc2(0.5f));
    c[VG_WPX0] = sub2(c[VG_WPX0], c[VG_WPX1]);
    c[VG_WPY0] = sub2(c[VG_WPY0], c[VG_WPY1]);
#pragma unroll
    for (int q = 0; q < D_N; ++q) {
        y64[0][q] = ok0 ? st[(size_t)slot[q] * nkp + k0] : 0.0;
        y64[1][q] = ok1 ? st[(size_t)slot[q] * nkp + k1] : 0.0;
    }
    // field terms at the start of the first step (see vg_start_row);
    // afterwards the terms at t_s + dt of step s serve as step s+1's
    VgField2 hstart = vg_field2(c, __ldg(tab + vg_start_row<TB>(s0)));
    const float2 *arow = tab + (size_t)s0 * TB::NT;   // field-table row of the current step
    float2 An[TB::NT];
#pragma unroll
    for (int i = 1; i < TB::NT; ++i) An[i] = __ldg(arow + i);
    // The FP64 state is y64 = (rounded to FP32: yhi) and the FP32 sum `acc` of
    // the increments since the last fold (each step's b_i k_i are added onto
    // it directly); after every step s with (s + 1) % XSTEP == 0 acc is added
    // to y64 in FP64.  An unfolded acc is kept in the state rows VG_ACC.. at
    // the end of a launch, so splitting the time loop changes no bit.  The stage input yhi + acc is rounded once, as float(y64)
    // would be, and acc holds only a few increments, so the state keeps its
    // FP64 accumulation while the f64<->f32 conversions drop XSTEP-fold.
    float2 yhi[D_N], acc[D_N];
#pragma unroll
    for (int q = 0; q < D_N; ++q) {
        yhi[q] = make_float2(float(y64[0][q]), float(y64[1][q]));
        acc[q] = make_float2(ok0 ? float(st[(size_t)(VG_ACC + q) * nkp + k0]) : 0.f,
                             ok1 ? float(st[(size_t)(VG_ACC + q) * nkp + k1]) : 0.f);
    }
    TileReducer red(red_s);
    // warp-stage reduction role of this lane (see above)
    const int xrow = (lane & 15) >> 1, xgrp = lane & 1;
    const float4 *const xsrc = xst + (lane & 15) * XROW + (lane >> 4) * 16;

    int next_shot = first_shot(s0, sd.shot_every);

    // one time step s, staged in row j of the warp stage
    auto step = [&](int j, int s) {
        VgField2 h[TB::NT];
        h[0] = hstart;
#pragma unroll
        for (int i = 1; i < TB::NT; ++i) h[i] = vg_field2(c, An[i]);
        hstart = h[TB::END];
        arow += TB::NT;
        if (s + 1 < s1) {
#pragma unroll
            for (int i = 1; i < TB::NT; ++i) An[i] = __ldg(arow + i);
        }
        float2 y0[D_N];
#pragma unroll
        for (int q = 0; q < D_N; ++q) y0[q] = add2(yhi[q], acc[q]);
        // currents and occupations at t_s (antelope.cpp:309-334), summed
        // over the pair and staged for the warp reduction
        {
            const float2 t0 = fma2(y0[D_ZR], c[VG_WQXR], mul2(y0[D_ZI], c[VG_WQXI]));
            const float2 t1 = fma2(y0[D_ZR], c[VG_WQYR], mul2(y0[D_ZI], c[VG_WQYI]));
            const float2 t2 = mul2(y0[D_DA], c[VG_WPX0]);
            const float2 t3 = mul2(y0[D_DA], c[VG_WPY0]);
            const float2 t4 = mul2(c[VG_W], y0[D_DA]);
            const float2 t5 = mul2(c[VG_W], y0[D_ZR]);
            const float2 t6 = mul2(c[VG_W], y0[D_ZI]);
            xst[(j * 2 + 0) * XROW + lane] = make_float4(t0.x + t0.y, t1.x + t1.y, t2.x + t2.y, t3.x + t3.y);
            xst[(j * 2 + 1) * XROW + lane] = make_float4(t4.x + t4.y, t5.x + t5.y, t6.x + t6.y, 0.f);
        }
        // one RK step of both k-points
        float2 kk[TB::S][D_N], yy[D_N];
#pragma unroll
        for (int i = 0; i < TB::S; ++i) {
#pragma unroll
            for (int q = 0; q < D_N; ++q) {
                float2 t = y0[q];
#pragma unroll
                for (int m = 0; m < i; ++m)
                    if (TB::a(i, m) != 0.0) t = fma2(bc2(sg[q] * float(TB::a(i, m))), kk[m][q], t);
                yy[q] = t;
            }
            vg_rhs2<G1>(h[TB::ti(i)], c[VG_C0], yy, ng1, ng2, g2, kk[i]);
            // the step increment sum_i b_i k_i goes straight onto acc
#pragma unroll
            for (int q = 0; q < D_N; ++q)
                if (TB::b(i) != 0.0) acc[q] = fma2(bc2(sg[q] * float(TB::b(i))), kk[i][q], acc[q]);
        }
        if (s == next_shot) {   // density snapshot: the FP64 state after step s
            // is y64 plus the increments not yet folded into it
            if (ok0)
                vg_snapshot(sd, s, k0, double(kc[(size_t)VG_R11 * nkp + k0]), y64[0][D_DA] + double(acc[D_DA].x),
                            y64[0][D_ZR] + double(acc[D_ZR].x), y64[0][D_ZI] + double(acc[D_ZI].x));
            if (ok1)
                vg_snapshot(sd, s, k1, double(kc[(size_t)VG_R11 * nkp + k1]), y64[1][D_DA] + double(acc[D_DA].y),
                            y64[1][D_ZR] + double(acc[D_ZR].y), y64[1][D_ZI] + double(acc[D_ZI].y));
            next_shot += sd.shot_every;
        }
    };

    // blocks of SUB steps (block stage) and XSTEP steps (warp stage, fold),
    // both aligned to absolute step multiples
    for (int b0 = s0; b0 < s1;) {
        const int b1 = min(s1, (b0 / SUB + 1) * SUB);
        for (int e0 = b0; e0 < b1;) {
            const int e1 = min(b1, (e0 / XSTEP + 1) * XSTEP), m = e1 - e0;
            if (m == XSTEP) {
#pragma unroll
                for (int j = 0; j < XSTEP; ++j) step(j, e0 + j);
            } else {
#pragma unroll 1
                for (int j = 0; j < m; ++j) step(j, e0 + j);
            }
            if (e1 % XSTEP == 0) {
                // fold the FP32 increments into the FP64 state
#pragma unroll
                for (int q = 0; q < D_N; ++q) {
                    y64[0][q] += double(acc[q].x);
                    y64[1][q] += double(acc[q].y);
                    yhi[q] = make_float2(float(y64[0][q]), float(y64[1][q]));
                    acc[q] = make_float2(0.f, 0.f);
                }
            }
            // warp sums of the m staged rows
            __syncwarp();
            float2 alo = make_float2(0.f, 0.f), ahi = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float4 b = xsrc[i];
                alo = add2(alo, make_float2(b.x, b.y));
                ahi = add2(ahi, make_float2(b.z, b.w));
            }
            float4 a = make_float4(alo.x, alo.y, ahi.x, ahi.y);
            a.x += __shfl_xor_sync(0xffffffffu, a.x, 16);
            a.y += __shfl_xor_sync(0xffffffffu, a.y, 16);
            a.z += __shfl_xor_sync(0xffffffffu, a.z, 16);
            a.w += __shfl_xor_sync(0xffffffffu, a.w, 16);
            __syncwarp();
            if (lane < 16 && xrow < m) {
                double *dst = &red.at(red.half, (e0 - b0) + xrow, warp, 0);
                if (xgrp == 0) {
                    dst[0] = double(a.x); dst[1] = double(a.y); dst[2] = double(a.z); dst[3] = double(a.w);
                } else {
                    dst[4] = double(a.x); dst[5] = -double(a.x);   // sum w db = -sum w da
                    dst[6] = double(a.y); dst[7] = double(a.z);
                }
            }
            e0 = e1;
        }
        red.flush(b1 - b0, b0 - s0, ntiles, tl.tile, partial);
        b0 = b1;
    }
#pragma unroll
    for (int q = 0; q < D_N; ++q) {
        if (ok0) {
            st[(size_t)slot[q] * nkp + k0] = y64[0][q];
            st[(size_t)(VG_ACC + q) * nkp + k0] = double(acc[q].x);
        }
        if (ok1) {
            st[(size_t)slot[q] * nkp + k1] = y64[1][q];
            st[(size_t)(VG_ACC + q) * nkp + k1] = double(acc[q].y);
        }
    }
    if (ok0) st[(size_t)VG_DB * nkp + k0] = -y64[0][D_DA];
    if (ok1) st[(size_t)VG_DB * nkp + k1] = -y64[1][D_DA];
}

// Closed-form eigenvectors of n.sigma for unit n: |+> (eigenvalue +1) and
// |-> (eigenvalue -1), choosing the chart that avoids 1 +/- nz -> 0.
__device__ __forceinline__ void spinors(double nx, double ny, double nz, double2 (&up)[2], double2 (&dn)[2])
{
    if (nz >= 0.0) {
        const double r = 1.0 / sqrt(2.0 * (1.0 + nz));
        up[0] = make_double2((1.0 + nz) * r, 0.0);
        up[1] = make_double2(nx * r, ny * r);
        dn[0] = make_double2(-nx * r, ny * r);
        dn[1] = make_double2((1.0 + nz) * r, 0.0);
    } else {
        const double r = 1.0 / sqrt(2.0 * (1.0 - nz));
        up[0] = make_double2(nx * r, -ny * r);
        up[1] = make_double2((1.0 - nz) * r, 0.0);
        dn[0] = make_double2((1.0 - nz) * r, 0.0);
        dn[1] = make_double2(-nx * r, -ny * r);
    }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconjmul(double2 a, double2 b)  // conj(a) * b
{
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// -------------------------------------------------------- length gauge
// rho = al*I + s.sigma, H0(k+A) = B0*I + B.sigma.  -i[H, rho] = 2 (B x s).sigma
// and the eigenbasis dephasing U[G o (U^dag rho U)]U^dag of SBEs.h:831-861 is
// g1*al*I + g1*(s.n)n.sigma + g2*(s - (s.n)n).sigma with n = B/|B|.
template <class Real>
__device__ __forceinline__ void lw_field(const Real (&c)[LW_NCONST], const Real *ph, Real (&ca)[3], Real (&sa)[3],
                                         Real (&cb)[3], Real (&sb)[3])
{
    // one table entry, 48 or 96 bytes at a 16-byte boundary, in 16-byte loads
    Real p[LW_NPHASE];
    constexpr int PER = 16 / sizeof(Real);
#pragma unroll
    for (int i = 0; i < LW_NPHASE / PER; ++i) {
        if constexpr (sizeof(Real) == 4) {
            const float4 u = __ldg(reinterpret_cast<const float4 *>(ph) + i);
            p[4 * i] = u.x; p[4 * i + 1] = u.y; p[4 * i + 2] = u.z; p[4 * i + 3] = u.w;
        } else {
            const double2 u = __ldg(reinterpret_cast<const double2 *>(ph) + i);
            p[2 * i] = u.x; p[2 * i + 1] = u.y;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        // cos/sin(k.v + A.v) from the per-k and per-stage-time factors
        ca[i] = fma(c[LW_CA0 + i], p[i], -(c[LW_SA0 + i] * p[3 + i]));
        sa[i] = fma(c[LW_SA0 + i], p[i], c[LW_CA0 + i] * p[3 + i]);
        cb[i] = fma(c[LW_CB0 + i], p[6 + i], -(c[LW_SB0 + i] * p[9 + i]));
        sb[i] = fma(c[LW_SB0 + i], p[6 + i], c[LW_CB0 + i] * p[9 + i]);
    }
}

// cos / sin of k.v + A(t).v for the three a and three b vectors at one
// stage time.
template <class Real> struct LwTrig {
    Real ca[3], sa[3], cb[3], sb[3];
};

// Field terms of H0(k + A) at one stage time: B = (B1, B2, B3) (dt-scaled),
// ib = 1 / |B|^2 and q = (g2 - g1) ib, the dephasing's weight of (s.B) B, so
// that neither the right-hand side nor the currents divide.
template <class Real> struct LwField {
    Real B1, B2, B3, q, ib;
};

template <class Real> __device__ __forceinline__ Real lw_recip(Real x);
template <> __device__ __forceinline__ double lw_recip<double>(double x) { return 1.0 / x; }
// the FP32 stages of the mixed method take the fast reciprocal (2 ulp)
template <> __device__ __forceinline__ float lw_recip<float>(float x) { return __fdividef(1.0f, x); }

template <class Real>
__device__ __forceinline__ LwField<Real> lw_field_terms(const LwTrig<Real> &T, Real t1dt, Real t2sdt, Real Mdt,
                                                        Real gd)
{
    LwField<Real> F;
    F.B1 = t1dt * (T.ca[0] + T.ca[1] + T.ca[2]);
    F.B2 = t1dt * (T.sa[0] + T.sa[1] + T.sa[2]);
    F.B3 = fma(-t2sdt, T.sb[0] + T.sb[1] + T.sb[2], Mdt);
    const Real bb = fma(F.B1, F.B1, fma(F.B2, F.B2, F.B3 * F.B3));
    F.ib = bb > Real(0) ? lw_recip<Real>(bb) : Real(0);
    F.q = gd * F.ib;
    return F;
}

template <class Real>
__device__ __forceinline__ LwField<Real> lw_field_terms(const Real (&c)[LW_NCONST], const Real *ph, Real t1dt,
                                                        Real t2sdt, Real Mdt, Real gd)
{
    LwTrig<Real> T;
    lw_field<Real>(c, ph, T.ca, T.sa, T.cb, T.sb);
    return lw_field_terms<Real>(T, t1dt, t2sdt, Mdt, gd);
}

template <class Real, bool G1>
__device__ __forceinline__ void lw_rhs(const LwField<Real> &F, const Real (&y)[4], Real g1, Real g2, Real (&k)[4])
{
    const Real sx = y[LW_SX], sy = y[LW_SY], sz = y[LW_SZ];
    const Real sB = fma(sx, F.B1, fma(sy, F.B2, sz * F.B3));
    const Real f = sB * F.q;  // (g2-g1) (s.n)/|B|
    k[LW_AL] = G1 ? -g1 * y[LW_AL] : Real(0);
    k[LW_SX] = fma(Real(2), fma(F.B2, sz, -(F.B3 * sy)), fma(f, F.B1, -g2 * sx));
    k[LW_SY] = fma(Real(2), fma(F.B3, sx, -(F.B1 * sz)), fma(f, F.B2, -g2 * sy));
    k[LW_SZ] = fma(Real(2), fma(F.B1, sy, -(F.B2 * sx)), fma(f, F.B3, -g2 * sz));
}

template <class Real> struct LwCurrentConsts {
    Real t1, t2c, t2s;
    Real va[3][2], vb[3][2];
};

// Currents and density-matrix sums at k + A(t) (SBEs.h:694-760) from that
// time's trig factors T and field terms F and the state y at t, in the stage
// arithmetic (the per-k terms of the mixed method in FP32, like the velocity
// gauge's), summed over the warp: lanes 4i return slot i.  The tile and
// k-sums above the warp are FP64 in both methods.
template <class Real>
__device__ __forceinline__ double lw_current_sum(const LwCurrentConsts<Real> &K, const LwTrig<Real> &T,
                                                 const LwField<Real> &F, const Real (&y)[4], Real w)
{
    Real j0[2], j1[2], j2[2], j3[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        j0[a] = K.t2c * fma(K.vb[0][a], T.sb[0], fma(K.vb[1][a], T.sb[1], K.vb[2][a] * T.sb[2]));
        j1[a] = K.t1 * fma(K.va[0][a], T.sa[0], fma(K.va[1][a], T.sa[1], K.va[2][a] * T.sa[2]));
        j2[a] = -K.t1 * fma(K.va[0][a], T.ca[0], fma(K.va[1][a], T.ca[1], K.va[2][a] * T.ca[2]));
        j3[a] = K.t2s * fma(K.vb[0][a], T.cb[0], fma(K.vb[1][a], T.cb[1], K.vb[2][a] * T.cb[2]));
    }
    const Real al = y[LW_AL], sx = y[LW_SX], sy = y[LW_SY], sz = y[LW_SZ];
    const Real sBi = fma(sx, F.B1, fma(sy, F.B2, sz * F.B3)) * F.ib;   // (s.B) / |B|^2
    const Real w2 = w + w;
    Real v[8];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const Real sj = fma(sx, j1[a], fma(sy, j2[a], sz * j3[a]));
        const Real par = sBi * fma(j1[a], F.B1, fma(j2[a], F.B2, j3[a] * F.B3));
        v[a] = w2 * (sj - par);                // interband
        v[2 + a] = w2 * fma(al, j0[a], par);   // intraband
    }
    v[4] = w * (al + sz);
    v[5] = w * (al - sz);
    v[6] = w * sx;
    v[7] = -w * sy;
    return double(warp_sum8<Real>(v, threadIdx.x & 31));
}

// B of H0(k + A(t)) in FP64 from the field-table entry ph of time t (the
// eigenbasis of a density snapshot).
template <class Real>
__device__ __forceinline__ void lw_B64(const Real (&c)[LW_NCONST], const Real *ph, double t1dt, double t2sdt,
                                       double Mdt, double (&Bt)[3])
{
    Real ca[3], sa[3], cb[3], sb[3];
    lw_field<Real>(c, ph, ca, sa, cb, sb);
    Bt[0] = t1dt * (double(ca[0]) + double(ca[1]) + double(ca[2]));
    Bt[1] = t1dt * (double(sa[0]) + double(sa[1]) + double(sa[2]));
    Bt[2] = Mdt - t2sdt * (double(sb[0]) + double(sb[1]) + double(sb[2]));
}

// One k-point per thread.  Field terms once per distinct stage time (RK4:
// t, t + dt/2 for stages 2 and 3, t + dt), the t + dt terms carried into the
// next step (a launch beginning at s loads the entry of step s-1 at its end,
// see vg_start_row); the currents of step s+1 are formed at the end of step s
// from that entry's trig factors and the new state.
template <class Real, int RK, bool G1>
__global__ void __launch_bounds__(256, 2) propagate_lw(const TileDev *__restrict__ tiles,
                                                    const SolveDev *__restrict__ solves, int tick, int S)
{
    using TB = Tableau<RK>;
    extern __shared__ double red_dyn[];   // red_stage_bytes(blockDim.x)
    const TileDev tl = tiles[blockIdx.x];
    const SolveDev &sd = solves[tl.solve];
    const int s0 = (tick - sd.admit_tick) * S;
    const int Nt = sd.Nt;
    if (s0 < 0 || s0 >= Nt) return;
    const int s1 = min(s0 + S, Nt);
    const int nkp = sd.nk_pad, ntiles = sd.ntiles;
    constexpr bool F64 = std::is_same<Real, double>::value;
    const Real *__restrict__ kc = static_cast<const Real *>(sd.kc);
    double *__restrict__ st = static_cast<double *>(sd.st);
    const Real *__restrict__ tab = static_cast<const Real *>(sd.tab);
    const Real g1 = Real(sd.g1), g2 = Real(sd.g2), gd = Real(sd.g2 - sd.g1);
    const Real t1dt = Real(sd.t1dt), t2sdt = Real(sd.t2sdt), Mdt = Real(sd.Mdt);
    LwCurrentConsts<Real> K;
    K.t1 = Real(sd.t1);
    K.t2c = Real(sd.t2c);
    K.t2s = Real(sd.t2s);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int a = 0; a < 2; ++a) { K.va[i][a] = Real(sd.va[i][a]); K.vb[i][a] = Real(sd.vb[i][a]); }

    const int local = threadIdx.x;
    const bool ok = local < tl.kcount;
    const int kidx = tl.k0 + local;
    Real c[LW_NCONST];
    double y64[4];
    Real yr[4];   // the state rounded to the stage arithmetic
#pragma unroll
    for (int q = 0; q < LW_NCONST; ++q) c[q] = ok ? kc[(size_t)q * nkp + kidx] : Real(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        y64[q] = ok ? st[(size_t)q * nkp + kidx] : 0.0;
        yr[q] = Real(y64[q]);
    }
    if (!ok) c[LW_CA0] = c[LW_CB0] = Real(1);  // padding lanes: a harmless k = 0 point, weight 0
    const Real w = c[LW_W];
    TileReducer red(red_dyn, blockDim.x >> 5);
    int next_shot = first_shot(s0, sd.shot_every);

    // field and currents at the launch's first step
    LwTrig<Real> Te;   // trig factors at the end of the step (t + dt)
    lw_field<Real>(c, tab + vg_start_row<TB>(s0) * LW_NPHASE, Te.ca, Te.sa, Te.cb, Te.sb);
    LwField<Real> F0 = lw_field_terms<Real>(Te, t1dt, t2sdt, Mdt, gd);
    red.put(lw_current_sum<Real>(K, Te, F0, yr, w), 0);

    for (int s = s0; s < s1; ++s) {
        const Real *row = tab + (size_t)s * TB::NT * LW_NPHASE;
        LwField<Real> Fc = F0;   // field at the current stage's time; a new time evaluates it once
        Real kk[TB::S][4], y[4], acc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = F64 ? yr[q] : Real(0);
#pragma unroll
        for (int i = 0; i < TB::S; ++i) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                Real t = yr[q];
#pragma unroll
                for (int m = 0; m < i; ++m)
                    if (TB::a(i, m) != 0.0) t = fma(Real(TB::a(i, m)), kk[m][q], t);
                y[q] = t;
            }
            if (TB::ti(i) == TB::END) {   // its trig factors also give the next step's currents
                lw_field<Real>(c, row + TB::END * LW_NPHASE, Te.ca, Te.sa, Te.cb, Te.sb);
                Fc = F0 = lw_field_terms<Real>(Te, t1dt, t2sdt, Mdt, gd);
            } else if (i > 0 && TB::ti(i) != TB::ti(i - 1)) {
                Fc = lw_field_terms<Real>(c, row + TB::ti(i) * LW_NPHASE, t1dt, t2sdt, Mdt, gd);
            }
            lw_rhs<Real, G1>(Fc, y, g1, g2, kk[i]);
            if (TB::b(i) != 0.0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = fma(Real(TB::b(i)), kk[i][q], acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            y64[q] = F64 ? double(acc[q]) : y64[q] + double(acc[q]);
            yr[q] = Real(y64[q]);
        }
        // currents of step s+1 at k + A(t_{s+1}) with the state after step s,
        // summed over the warp now and staged after this step's flush
        const double jsum = s + 1 < s1 ? lw_current_sum<Real>(K, Te, F0, yr, w) : 0.0;
        if (s == next_shot) {
            // density snapshot: rho after the step in the eigenbasis of
            // H0(k + A(t_s)) (SBEs::WannierToHamiltonian at the step's start
            // time, as antelope.cpp:358 calls it); conduction = |+>, valence = |->
            if (ok) {
                double Bt[3];
                lw_B64<Real>(c, tab + vg_start_row<TB>(s) * LW_NPHASE, sd.t1dt, sd.t2sdt, sd.Mdt, Bt);
                const double bn = sqrt(Bt[0] * Bt[0] + Bt[1] * Bt[1] + Bt[2] * Bt[2]);
                double nx = 0.0, ny = 0.0, nz = 1.0;
                if (bn > 0.0) { nx = Bt[0] / bn; ny = Bt[1] / bn; nz = Bt[2] / bn; }
                const double al = y64[LW_AL], sx = y64[LW_SX], sy = y64[LW_SY], sz = y64[LW_SZ];
                double2 up[2], dn[2];
                spinors(nx, ny, nz, up, dn);
                // rho |-> with rho = [[al + sz, sx - i sy], [sx + i sy, al - sz]]
                const double2 r0 = make_double2((al + sz) * dn[0].x + sx * dn[1].x + sy * dn[1].y,
                                                (al + sz) * dn[0].y + sx * dn[1].y - sy * dn[1].x);
                const double2 r1 = make_double2(sx * dn[0].x - sy * dn[0].y + (al - sz) * dn[1].x,
                                                sx * dn[0].y + sy * dn[0].x + (al - sz) * dn[1].y);
                const double2 q0 = cconjmul(up[0], r0), q1 = cconjmul(up[1], r1);
                const size_t i = (size_t)(s / sd.shot_every) * sd.nk + kidx;
                sd.snap_nc[i] = al + sx * nx + sy * ny + sz * nz;
                sd.snap_pi[2 * i] = q0.x + q1.x;
                sd.snap_pi[2 * i + 1] = q0.y + q1.y;
            }
            next_shot += sd.shot_every;
        }
        const int r = (s - s0) % SUB;
        if (r == SUB - 1 || s == s1 - 1) red.flush(r + 1, s - r - s0, ntiles, tl.tile, sd.partial);
        if (s + 1 < s1) red.put(jsum, (s + 1 - s0) % SUB);
    }
    if (ok)
#pragma unroll
        for (int q = 0; q < 4; ++q) st[(size_t)q * nkp + kidx] = y64[q];
}

// Mixed method, length gauge, two k-points per thread in f32x2 registers (as
// propagate_vg_x2): every field, right-hand-side and current instruction
// advances both.  The table entry of a stage time is shared by both k-points
// (its values broadcast); the per-k cos/sin factors, the state rounded to
// FP32 and the stage slopes are packed.  The field terms carry 2B and -2B
// so that each component of 2 B x s + f B - g2 s is three packed FMAs on a
// packed product; the FP64 state receives the FP32 increments every XSTEP
// steps (see the kernel).
struct LwField2 { float2 B1, B2, B3, q, ib, d1, d2, d3, n1, n2, n3; };   // d = 2B, n = -2B

__device__ __forceinline__ void lw_trig2(const float2 (&c)[LW_NCONST], const float *ph, float2 (&ca)[3],
                                         float2 (&sa)[3], float2 (&cb)[3], float2 (&sb)[3])
{
    float p[LW_NPHASE];
#pragma unroll
    for (int i = 0; i < LW_NPHASE / 4; ++i) {
        const float4 u = __ldg(reinterpret_cast<const float4 *>(ph) + i);
        p[4 * i] = u.x; p[4 * i + 1] = u.y; p[4 * i + 2] = u.z; p[4 * i + 3] = u.w;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        ca[i] = fma2(c[LW_CA0 + i], bc2(p[i]), mul2(c[LW_SA0 + i], bc2(-p[3 + i])));
        sa[i] = fma2(c[LW_SA0 + i], bc2(p[i]), mul2(c[LW_CA0 + i], bc2(p[3 + i])));
        cb[i] = fma2(c[LW_CB0 + i], bc2(p[6 + i]), mul2(c[LW_SB0 + i], bc2(-p[9 + i])));
        sb[i] = fma2(c[LW_SB0 + i], bc2(p[6 + i]), mul2(c[LW_CB0 + i], bc2(p[9 + i])));
    }
}

struct LwTrig2 { float2 ca[3], sa[3], cb[3], sb[3]; };

__device__ __forceinline__ LwField2 lw_field_terms2(const LwTrig2 &T, float2 t1dt, float2 nt2sdt, float2 Mdt, float2 gd)
{
    LwField2 F;
    F.B1 = mul2(t1dt, add2(add2(T.ca[0], T.ca[1]), T.ca[2]));
    F.B2 = mul2(t1dt, add2(add2(T.sa[0], T.sa[1]), T.sa[2]));
    F.B3 = fma2(nt2sdt, add2(add2(T.sb[0], T.sb[1]), T.sb[2]), Mdt);
    const float2 bb = fma2(F.B1, F.B1, fma2(F.B2, F.B2, mul2(F.B3, F.B3)));
    F.ib = make_float2(bb.x > 0.f ? __fdividef(1.0f, bb.x) : 0.f, bb.y > 0.f ? __fdividef(1.0f, bb.y) : 0.f);
    F.q = mul2(gd, F.ib);
    F.d1 = add2(F.B1, F.B1); F.d2 = add2(F.B2, F.B2); F.d3 = add2(F.B3, F.B3);
    F.n1 = mul2(F.B1, bc2(-2.f)); F.n2 = mul2(F.B2, bc2(-2.f)); F.n3 = mul2(F.B3, bc2(-2.f));
    return F;
}

template <bool G1>
__device__ __forceinline__ void lw_rhs2(const LwField2 &F, const float2 (&y)[4], float2 ng1, float2 ng2, float2 (&k)[4])
{
    const float2 sx = y[LW_SX], sy = y[LW_SY], sz = y[LW_SZ];
    const float2 f = mul2(fma2(sx, F.B1, fma2(sy, F.B2, mul2(sz, F.B3))), F.q);   // (g2-g1)(s.n)/|B|
    k[LW_AL] = G1 ? mul2(ng1, y[LW_AL]) : make_float2(0.f, 0.f);
    k[LW_SX] = fma2(F.d2, sz, fma2(F.n3, sy, fma2(f, F.B1, mul2(ng2, sx))));
    k[LW_SY] = fma2(F.d3, sx, fma2(F.n1, sz, fma2(f, F.B2, mul2(ng2, sy))));
    k[LW_SZ] = fma2(F.d1, sy, fma2(F.n2, sx, fma2(f, F.B3, mul2(ng2, sz))));
}

// j-vector constants of the currents, premultiplied: j0 = t2c vb.sin(kb),
// j1 = t1 va.sin(ka), j2 = -t1 va.cos(ka), j3 = t2s vb.cos(kb) per axis
struct LwCurK2 { float j0[2][3], j1[2][3], j2[2][3], j3[2][3]; };

// The currents and density sums of both k-points (as lw_current_sum), added
// over the pair in FP32 and over the warp: lanes 4i return slot i.
__device__ __forceinline__ double lw_current_sum2(const LwCurK2 &K, const LwTrig2 &T, const LwField2 &F,
                                                  const float2 (&y)[4], float2 w)
{
    float2 j0[2], j1[2], j2[2], j3[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        j0[a] = fma2(bc2(K.j0[a][0]), T.sb[0], fma2(bc2(K.j0[a][1]), T.sb[1], mul2(bc2(K.j0[a][2]), T.sb[2])));
        j1[a] = fma2(bc2(K.j1[a][0]), T.sa[0], fma2(bc2(K.j1[a][1]), T.sa[1], mul2(bc2(K.j1[a][2]), T.sa[2])));
        j2[a] = fma2(bc2(K.j2[a][0]), T.ca[0], fma2(bc2(K.j2[a][1]), T.ca[1], mul2(bc2(K.j2[a][2]), T.ca[2])));
        j3[a] = fma2(bc2(K.j3[a][0]), T.cb[0], fma2(bc2(K.j3[a][1]), T.cb[1], mul2(bc2(K.j3[a][2]), T.cb[2])));
    }
    const float2 al = y[LW_AL], sx = y[LW_SX], sy = y[LW_SY], sz = y[LW_SZ];
    const float2 sBi = mul2(fma2(sx, F.B1, fma2(sy, F.B2, mul2(sz, F.B3))), F.ib);   // (s.B) / |B|^2
    const float2 w2 = add2(w, w);
    float v[8];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const float2 sj = fma2(sx, j1[a], fma2(sy, j2[a], mul2(sz, j3[a])));
        const float2 par = mul2(sBi, fma2(j1[a], F.B1, fma2(j2[a], F.B2, mul2(j3[a], F.B3))));
        const float2 ie = mul2(w2, sub2(sj, par));       // interband
        const float2 ia = mul2(w2, fma2(al, j0[a], par)); // intraband
        v[a] = ie.x + ie.y;
        v[2 + a] = ia.x + ia.y;
    }
    const float2 o0 = mul2(w, add2(al, sz)), o1 = mul2(w, sub2(al, sz)), o2 = mul2(w, sx), o3 = mul2(w, sy);
    v[4] = o0.x + o0.y;
    v[5] = o1.x + o1.y;
    v[6] = o2.x + o2.y;
    v[7] = -(o3.x + o3.y);
    return double(warp_sum8<float>(v, threadIdx.x & 31));
}

template <int RK, bool G1>
__global__ void __launch_bounds__(256, 2) propagate_lw_x2(const TileDev *__restrict__ tiles,
                                                       const SolveDev *__restrict__ solves, int tick, int S)
{
    using TB = Tableau<RK>;
    extern __shared__ double red_dyn[];   // red_stage_bytes(blockDim.x)
    const TileDev tl = tiles[blockIdx.x];
    const SolveDev &sd = solves[tl.solve];
    const int s0 = (tick - sd.admit_tick) * S;
    const int Nt = sd.Nt;
    if (s0 < 0 || s0 >= Nt) return;
    const int s1 = min(s0 + S, Nt);
    const int nkp = sd.nk_pad, ntiles = sd.ntiles;
    const float *__restrict__ kc = static_cast<const float *>(sd.kc);
    double *__restrict__ st = static_cast<double *>(sd.st);
    const float *__restrict__ tab = static_cast<const float *>(sd.tab);
    const float2 ng1 = bc2(-float(sd.g1)), ng2 = bc2(-float(sd.g2)), gd = bc2(float(sd.g2 - sd.g1));
    const float2 t1dt = bc2(float(sd.t1dt)), nt2sdt = bc2(-float(sd.t2sdt)), Mdt = bc2(float(sd.Mdt));
    LwCurK2 K;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            K.j0[a][i] = float(sd.t2c) * float(sd.vb[i][a]);
            K.j1[a][i] = float(sd.t1) * float(sd.va[i][a]);
            K.j2[a][i] = -float(sd.t1) * float(sd.va[i][a]);
            K.j3[a][i] = float(sd.t2s) * float(sd.vb[i][a]);
        }

    const int l0 = threadIdx.x, l1 = threadIdx.x + blockDim.x;
    const bool ok0 = l0 < tl.kcount, ok1 = l1 < tl.kcount;
    const int k0 = tl.k0 + l0, k1 = tl.k0 + l1;
    float2 c[LW_NCONST];
#pragma unroll
    for (int q = 0; q < LW_NCONST; ++q)
        c[q] = make_float2(ok0 ? kc[(size_t)q * nkp + k0] : 0.f, ok1 ? kc[(size_t)q * nkp + k1] : 0.f);
    // padding lanes: a harmless k = 0 point of weight 0
    if (!ok0) c[LW_CA0].x = c[LW_CB0].x = 1.f;
    if (!ok1) c[LW_CA0].y = c[LW_CB0].y = 1.f;
    const float2 w = c[LW_W];
    // The FP64 state is y64 = (rounded to FP32: yhi) plus the FP32 sum `acc`
    // of the increments since the last fold; after every step s with
    // (s + 1) % XSTEP == 0 acc is added to y64 in FP64 (as propagate_vg_x2),
    // and an unfolded acc is kept in the state rows LW_ACC.. at a launch's
    // end, so splitting the time loop changes no bit.  The stage input
    // yhi + acc is rounded once per step, as float(y64) would be.
    double y64[2][4];
    float2 yhi[4], acc[4], yr[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        y64[0][q] = ok0 ? st[(size_t)q * nkp + k0] : 0.0;
        y64[1][q] = ok1 ? st[(size_t)q * nkp + k1] : 0.0;
        yhi[q] = make_float2(float(y64[0][q]), float(y64[1][q]));
        acc[q] = make_float2(ok0 ? float(st[(size_t)(LW_ACC + q) * nkp + k0]) : 0.f,
                             ok1 ? float(st[(size_t)(LW_ACC + q) * nkp + k1]) : 0.f);
        yr[q] = add2(yhi[q], acc[q]);
    }
    TileReducer red(red_dyn, blockDim.x >> 5);
    int next_shot = first_shot(s0, sd.shot_every);

    LwTrig2 Te;   // trig factors at the end of the step (t + dt)
    lw_trig2(c, tab + vg_start_row<TB>(s0) * LW_NPHASE, Te.ca, Te.sa, Te.cb, Te.sb);
    LwField2 F0 = lw_field_terms2(Te, t1dt, nt2sdt, Mdt, gd);
    red.put(lw_current_sum2(K, Te, F0, yr, w), 0);

    for (int s = s0; s < s1; ++s) {
        const float *row = tab + (size_t)s * TB::NT * LW_NPHASE;
        LwField2 Fc = F0;
        float2 kk[TB::S][4], y[4];
#pragma unroll
        for (int i = 0; i < TB::S; ++i) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float2 t = yr[q];
#pragma unroll
                for (int m = 0; m < i; ++m)
                    if (TB::a(i, m) != 0.0) t = fma2(bc2(float(TB::a(i, m))), kk[m][q], t);
                y[q] = t;
            }
            if (TB::ti(i) == TB::END) {
                lw_trig2(c, row + TB::END * LW_NPHASE, Te.ca, Te.sa, Te.cb, Te.sb);
                Fc = F0 = lw_field_terms2(Te, t1dt, nt2sdt, Mdt, gd);
            } else if (i > 0 && TB::ti(i) != TB::ti(i - 1)) {
                LwTrig2 Tm;
                lw_trig2(c, row + TB::ti(i) * LW_NPHASE, Tm.ca, Tm.sa, Tm.cb, Tm.sb);
                Fc = lw_field_terms2(Tm, t1dt, nt2sdt, Mdt, gd);
            }
            lw_rhs2<G1>(Fc, y, ng1, ng2, kk[i]);
            if (TB::b(i) != 0.0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = fma2(bc2(float(TB::b(i))), kk[i][q], acc[q]);
            }
        }
        if ((s + 1) % XSTEP == 0) {   // fold the FP32 increments into the FP64 state
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                y64[0][q] += double(acc[q].x);
                y64[1][q] += double(acc[q].y);
                yhi[q] = make_float2(float(y64[0][q]), float(y64[1][q]));
                acc[q] = make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) yr[q] = add2(yhi[q], acc[q]);
        const double jsum = s + 1 < s1 ? lw_current_sum2(K, Te, F0, yr, w) : 0.0;
        if (s == next_shot) {
            // density snapshot of each k-point (as propagate_lw)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const bool okh = h == 0 ? ok0 : ok1;
                if (!okh) continue;
                float cf[LW_NCONST];
#pragma unroll
                for (int q = 0; q < LW_NCONST; ++q) cf[q] = h == 0 ? c[q].x : c[q].y;
                double Bt[3];
                lw_B64<float>(cf, tab + vg_start_row<TB>(s) * LW_NPHASE, sd.t1dt, sd.t2sdt, sd.Mdt, Bt);
                const double bn = sqrt(Bt[0] * Bt[0] + Bt[1] * Bt[1] + Bt[2] * Bt[2]);
                double nx = 0.0, ny = 0.0, nz = 1.0;
                if (bn > 0.0) { nx = Bt[0] / bn; ny = Bt[1] / bn; nz = Bt[2] / bn; }
                // the FP64 state after step s: y64 plus the increments not yet folded into it
                const double al = y64[h][LW_AL] + double(h == 0 ? acc[LW_AL].x : acc[LW_AL].y);
                const double sx = y64[h][LW_SX] + double(h == 0 ? acc[LW_SX].x : acc[LW_SX].y);
                const double sy = y64[h][LW_SY] + double(h == 0 ? acc[LW_SY].x : acc[LW_SY].y);
                const double sz = y64[h][LW_SZ] + double(h == 0 ? acc[LW_SZ].x : acc[LW_SZ].y);
                double2 up[2], dn[2];
                spinors(nx, ny, nz, up, dn);
                const double2 r0 = make_double2((al + sz) * dn[0].x + sx * dn[1].x + sy * dn[1].y,
                                                (al + sz) * dn[0].y + sx * dn[1].y - sy * dn[1].x);
                const double2 r1 = make_double2(sx * dn[0].x - sy * dn[0].y + (al - sz) * dn[1].x,
                                                sx * dn[0].y + sy * dn[0].x + (al - sz) * dn[1].y);
                const double2 q0 = cconjmul(up[0], r0), q1 = cconjmul(up[1], r1);
                const size_t ix = (size_t)(s / sd.shot_every) * sd.nk + (h == 0 ? k0 : k1);
                sd.snap_nc[ix] = al + sx * nx + sy * ny + sz * nz;
                sd.snap_pi[2 * ix] = q0.x + q1.x;
                sd.snap_pi[2 * ix + 1] = q0.y + q1.y;
            }
            next_shot += sd.shot_every;
        }
        const int r = (s - s0) % SUB;
        if (r == SUB - 1 || s == s1 - 1) red.flush(r + 1, s - r - s0, ntiles, tl.tile, sd.partial);
        if (s + 1 < s1) red.put(jsum, (s + 1 - s0) % SUB);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (ok0) {
            st[(size_t)q * nkp + k0] = y64[0][q];
            st[(size_t)(LW_ACC + q) * nkp + k0] = double(acc[q].x);
        }
        if (ok1) {
            st[(size_t)q * nkp + k1] = y64[1][q];
            st[(size_t)(LW_ACC + q) * nkp + k1] = double(acc[q].y);
        }
    }
}

// ------------------------------------------------------- second pass
// One CTA per (step, solve): its 8 warps split the tile rows into 8 fixed
// contiguous ranges; within a warp, lanes 8g..8g+7 sum slots 0..7 over tiles
// g, g+4, ... of the range and two fixed shuffles combine the four groups;
// the 8 warp sums are added in warp order.  The order depends only on the
// solve's tile count, so the sums are deterministic.
__global__ void __launch_bounds__(256) reduce_tiles(const SolveDev *__restrict__ solves,
                                                    const int *__restrict__ solve_ids, int tick, int S)
{
    __shared__ double part[8][NSLOT];
    const SolveDev &sd = solves[solve_ids[blockIdx.y]];
    const int s0 = (tick - sd.admit_tick) * S;
    const int j = blockIdx.x;
    if (s0 < 0 || j >= S || s0 + j >= sd.Nt) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane & 7, g = lane >> 3, nt = sd.ntiles;
    const int chunk = (nt + 7) / 8;
    const int t0 = min(nt, warp * chunk), t1 = min(nt, t0 + chunk);
    const double *p = sd.partial + (size_t)j * nt * NSLOT;
    double acc = 0.0;
    for (int t = t0 + g; t < t1; t += 4) acc += p[(size_t)t * NSLOT + slot];
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    if (lane < 8) part[warp][lane] = acc;
    __syncthreads();
    if (threadIdx.x < NSLOT) {
        double sum = 0.0;
        for (int w = 0; w < 8; ++w) sum += part[w][threadIdx.x];
        sd.jout[(size_t)(s0 + j) * NSLOT + threadIdx.x] = sum;
    }
}

// ------------------------------------------------------------ set-up
template <class Real>
__global__ void __launch_bounds__(256) init_haldane(InitArgs ia, Real *__restrict__ kc, double *__restrict__ st,
                                                    double *__restrict__ constpart)
{
    // one block per tile; threads loop over the tile's k-points
    const int tile = blockIdx.x;
    const int k0 = tile * ia.tile_k;
    const int k1 = min(k0 + ia.tile_k, ia.nk);
    double cp[4] = {0, 0, 0, 0};  // sum w rho0 P00/P11 (x, y), sum w rho0_00, sum w rho0_11
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        // momaxis grid point and weight (of flat index k_offset + k)
        const int N0 = ia.N[0], N1 = ia.N[1], N2 = ia.N[2];
        const int kg = ia.k_offset + k;
        const int ii[3] = {kg / (N1 * N2), (kg / N2) % N1, kg % N2};
        const int NN[3] = {N0, N1, N2};
        double f[3], w = 1.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            f[d] = (NN[d] == 1) ? 0.0 : double(ii[d]) / (NN[d] - 1) - 0.5;
            if (NN[d] != 1 && (ii[d] == 0 || ii[d] == NN[d] - 1)) w /= 2;
        }
        double kv[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            kv[d] = ia.origin[d] + f[0] * ia.axes[0 * 3 + d] + f[1] * ia.axes[1 * 3 + d] + f[2] * ia.axes[2 * 3 + d];
        // Haldane B(k) and J(k) = -dH/dk
        double ca[3], sa[3], cb[3], sb[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double aa = kv[0] * ia.va[i][0] + kv[1] * ia.va[i][1];
            const double ab = kv[0] * ia.vb[i][0] + kv[1] * ia.vb[i][1];
            sincos(aa, &sa[i], &ca[i]);
            sincos(ab, &sb[i], &cb[i]);
        }
        const double t2c = 2.0 * ia.t2 * cos(ia.phi0), t2s = 2.0 * ia.t2 * sin(ia.phi0);
        const double B0 = t2c * (cb[0] + cb[1] + cb[2]);
        const double B1 = ia.t1 * (ca[0] + ca[1] + ca[2]);
        const double B2 = ia.t1 * (sa[0] + sa[1] + sa[2]);
        const double B3 = ia.M0 - t2s * (sb[0] + sb[1] + sb[2]);
        const double bn = sqrt(B1 * B1 + B2 * B2 + B3 * B3);
        double nx = 0.0, ny = 0.0, nz = 1.0;
        if (bn > 0.0) { nx = B1 / bn; ny = B2 / bn; nz = B3 / bn; }
        const double e0 = B0 - bn, e1 = B0 + bn;   // ascending, as zheevr
        double f0, f1;                             // rho0 in the band basis
        if (ia.use_fermi) {
            const double kT = 300. / 3.15775024804e5;
            const double o0 = 1.0 / (exp((e0 - ia.Ef) / kT) + 1.0), o1 = 1.0 / (exp((e1 - ia.Ef) / kT) + 1.0);
            f0 = o0 / (o0 + o1);
            f1 = o1 / (o0 + o1);
        } else {
            f0 = ia.nval >= 1 ? 1.0 : 0.0;
            f1 = ia.nval >= 2 ? 1.0 : 0.0;
        }
        const size_t P = ia.nk_pad;
        if (ia.variant == VAR_HALDANE_VG) {
            double j0[2], jv[2][3];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                j0[a] = t2c * (ia.vb[0][a] * sb[0] + ia.vb[1][a] * sb[1] + ia.vb[2][a] * sb[2]);
                jv[a][0] = ia.t1 * (ia.va[0][a] * sa[0] + ia.va[1][a] * sa[1] + ia.va[2][a] * sa[2]);
                jv[a][1] = -ia.t1 * (ia.va[0][a] * ca[0] + ia.va[1][a] * ca[1] + ia.va[2][a] * ca[2]);
                jv[a][2] = t2s * (ia.vb[0][a] * cb[0] + ia.vb[1][a] * cb[1] + ia.vb[2][a] * cb[2]);
            }
            double2 up[2], dn[2];
            spinors(nx, ny, nz, up, dn);
            double P00[2], P11[2];
            double2 P01[2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const double jn = jv[a][0] * nx + jv[a][1] * ny + jv[a][2] * nz;
                P00[a] = j0[a] - jn;
                P11[a] = j0[a] + jn;
                // <-| j.sigma |+>
                const double2 m00 = make_double2(jv[a][2], 0.0), m11 = make_double2(-jv[a][2], 0.0);
                const double2 m01 = make_double2(jv[a][0], -jv[a][1]), m10 = make_double2(jv[a][0], jv[a][1]);
                const double2 v0 = make_double2(cmul(m00, up[0]).x + cmul(m01, up[1]).x,
                                                cmul(m00, up[0]).y + cmul(m01, up[1]).y);
                const double2 v1 = make_double2(cmul(m10, up[0]).x + cmul(m11, up[1]).x,
                                                cmul(m10, up[0]).y + cmul(m11, up[1]).y);
                const double2 q0 = cconjmul(dn[0], v0), q1 = cconjmul(dn[1], v1);
                P01[a] = make_double2(q0.x + q1.x, q0.y + q1.y);
            }
            const double dt = ia.dt;
            const double cv[VG_NCONST] = {
                dt * (e0 - e1),
                dt * (P00[0] - P11[0]), dt * (P00[1] - P11[1]),
                dt * P01[0].x, dt * P01[0].y, dt * P01[1].x, dt * P01[1].y,
                f1 - f0,
                w * P00[0], w * P11[0], w * P00[1], w * P11[1],
                2.0 * w * P01[0].x, 2.0 * w * P01[0].y, 2.0 * w * P01[1].x, 2.0 * w * P01[1].y,
                w};
#pragma unroll
            for (int q = 0; q < VG_NCONST; ++q) kc[q * P + k] = Real(cv[q]);
            kc[VG_R11 * P + k] = Real(f1);
#pragma unroll
            for (int q = 0; q < VG_NSTATE; ++q) st[q * P + k] = 0.0;
            cp[0] += w * (f0 * P00[0] + f1 * P11[0]);
            cp[1] += w * (f0 * P00[1] + f1 * P11[1]);
            cp[2] += w * f0;
            cp[3] += w * f1;
        } else {
            const double cv[LW_NCONST] = {ca[0], ca[1], ca[2], sa[0], sa[1], sa[2],
                                          cb[0], cb[1], cb[2], sb[0], sb[1], sb[2], w};
#pragma unroll
            for (int q = 0; q < LW_NCONST; ++q) kc[q * P + k] = Real(cv[q]);
            // rho0 = f0 |-><-| + f1 |+><+| = (f0+f1)/2 I + (f1-f0)/2 n.sigma (SBEs.h:352-356)
            st[LW_AL * P + k] = 0.5 * (f0 + f1);
            st[LW_SX * P + k] = 0.5 * (f1 - f0) * nx;
            st[LW_SY * P + k] = 0.5 * (f1 - f0) * ny;
            st[LW_SZ * P + k] = 0.5 * (f1 - f0) * nz;
        }
    }
    // deterministic block sum of the constant parts -> constpart[tile][8]
    __shared__ double sh[256][4];
    for (int q = 0; q < 4; ++q) sh[threadIdx.x][q] = cp[q];
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off)
            for (int q = 0; q < 4; ++q) sh[threadIdx.x][q] += sh[threadIdx.x + off][q];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double *o = constpart + (size_t)tile * NSLOT;
        o[0] = 0.0; o[1] = 0.0;
        o[2] = sh[0][0]; o[3] = sh[0][1];
        o[4] = sh[0][2]; o[5] = sh[0][3];
        o[6] = 0.0; o[7] = 0.0;
    }
}

// ------------------------------------------------- FMA peak microbench
// 1-D integrated conduction occupation of the snapshots (antelope.cpp:343-
// 370): for every snapshot and first grid index m, the weighted sum of the
// per-k values over the solve's k-points with that index, divided by N1.  One
// CTA per (m, snapshot), fixed summation order.
__global__ void __launch_bounds__(256) snapshot_bins(const double *__restrict__ nc, int nk, int k_offset, int N0,
                                                     int N1, int N2, double *__restrict__ occ1d)
{
    __shared__ double red[256];
    const int m = blockIdx.x, shot = blockIdx.y, blk = N1 * N2;
    const int g0 = max(m * blk, k_offset), g1 = min((m + 1) * blk, k_offset + nk);
    const double wi = (N0 != 1 && (m == 0 || m == N0 - 1)) ? 0.5 : 1.0;
    double acc = 0.0;
    for (int g = g0 + (int)threadIdx.x; g < g1; g += blockDim.x) {
        const int j = (g / N2) % N1, l = g % N2;
        double w = wi;   // trapezoid weight (momaxis.h:147-186)
        if (N1 != 1 && (j == 0 || j == N1 - 1)) w *= 0.5;
        if (N2 != 1 && (l == 0 || l == N2 - 1)) w *= 0.5;
        acc += w * nc[(size_t)shot * nk + (g - k_offset)];
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) occ1d[(size_t)shot * N0 + m] = red[0] / (double)N1;
}

// Independent FMA chains (8 per thread) to measure the FP64 / FP32 vector
// pipe peaks that the roofline fractions are quoted against.
template <class Real>
__global__ void __launch_bounds__(256) fma_peak(Real *out, int iters, Real a, Real b)
{
    Real x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = Real(threadIdx.x + i) * Real(1e-3);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = fma(x[i], a, b);
    }
    Real s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == Real(-12345.678)) out[threadIdx.x] = s;  // keeps the chains live
}

// FFMA2 variant of the microbenchmark: 8 independent packed chains.
__global__ void __launch_bounds__(256) fma_peak_x2(float *out, int iters, float a, float b)
{
    float2 x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = make_float2(float(threadIdx.x + i) * 1e-3f, float(i) * 1e-3f);
    const float2 aa = bc2(a), bb = bc2(b);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = fma2(x[i], aa, bb);
    }
    float s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i].x + x[i].y;
    if (s == -12345.678f) out[threadIdx.x] = s;
}

// ------------------------------------------------------------- launchers
#define SBE_CHECK_LAUNCH() return cudaGetLastError()

template <class Real, int RK, int KPT>
static cudaError_t launch_vg_t(const LaunchArgs &la, bool g1)
{
    if (g1)
        propagate_vg<Real, RK, KPT, true><<<la.ntiles, la.threads, red_stage_bytes(la.threads), la.stream>>>(la.tiles, la.solves, la.tick, la.S);
    else
        propagate_vg<Real, RK, KPT, false><<<la.ntiles, la.threads, red_stage_bytes(la.threads), la.stream>>>(la.tiles, la.solves, la.tick, la.S);
    SBE_CHECK_LAUNCH();
}

// The packed kernel's warp stages live in dynamic shared memory (64 KiB at
// 256 threads, above the 48 KiB default): the limit is raised once per device
// and kernel instance.
template <int RK, bool G1>
static cudaError_t launch_vg_x2_t(const LaunchArgs &la)
{
    constexpr int kMaxDev = 64;
    static std::atomic<int> raised[kMaxDev];
    const int bytes = xstage_bytes(la.threads);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    if (raised[dev].load(std::memory_order_acquire) == 0) {
        e = cudaFuncSetAttribute(propagate_vg_x2<RK, G1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 xstage_bytes(256));
        if (e != cudaSuccess) return e;
        raised[dev].store(1, std::memory_order_release);
    }
    propagate_vg_x2<RK, G1><<<la.ntiles, la.threads, bytes, la.stream>>>(la.tiles, la.solves, la.tick, la.S);
    SBE_CHECK_LAUNCH();
}

template <int RK>
static cudaError_t launch_vg_x2(const LaunchArgs &la, bool g1)
{
    return g1 ? launch_vg_x2_t<RK, true>(la) : launch_vg_x2_t<RK, false>(la);
}

template <class Real, int RK>
static cudaError_t launch_lw_t(const LaunchArgs &la, bool g1)
{
    if (g1)
        propagate_lw<Real, RK, true><<<la.ntiles, la.threads, red_stage_bytes(la.threads), la.stream>>>(la.tiles, la.solves, la.tick, la.S);
    else
        propagate_lw<Real, RK, false><<<la.ntiles, la.threads, red_stage_bytes(la.threads), la.stream>>>(la.tiles, la.solves, la.tick, la.S);
    SBE_CHECK_LAUNCH();
}

template <int RK, bool G1>
static cudaError_t launch_lw_x2_t(const LaunchArgs &la)
{
    propagate_lw_x2<RK, G1><<<la.ntiles, la.threads, red_stage_bytes(la.threads), la.stream>>>(la.tiles, la.solves,
                                                                                              la.tick, la.S);
    SBE_CHECK_LAUNCH();
}

int propagate_max_threads(int variant, int precision, int rk, int kpt)
{
    // propagate_vg with RK4 (FP64, or one k-point per thread in FP32); the
    // packed mixed kernels and the length gauge stage 8 warps at most
    const bool vg_scalar = variant == VAR_HALDANE_VG && rk == 4 && (precision == PREC_FP64 || kpt == 1);
    return vg_scalar ? 512 : 256;
}

cudaError_t launch_propagate(const LaunchArgs &la)
{
    if (la.ntiles <= 0) return cudaSuccess;
    if (la.threads <= 0 || la.threads > propagate_max_threads(la.variant, la.precision, la.rk, la.kpt) ||
        (la.threads & 31))
        return cudaErrorInvalidValue;
    const bool g1 = la.has_g1;
    if (la.variant == VAR_HALDANE_VG) {
#define SBE_VG(R, RK)                                                       \
    switch (la.kpt) {                                                       \
        case 1: return launch_vg_t<R, RK, 1>(la, g1);                       \
        case 2: return launch_vg_t<R, RK, 2>(la, g1);                       \
        default: return cudaErrorInvalidValue;                              \
    }
        if (la.precision == PREC_FP64) {
            if (la.rk == 4) { SBE_VG(double, 4) } else if (la.rk == 5) { SBE_VG(double, 5) }
        } else if (la.kpt == 2) {
            if (la.rk == 4) return launch_vg_x2<4>(la, g1);
            if (la.rk == 5) return launch_vg_x2<5>(la, g1);
        } else {
            if (la.rk == 4) { SBE_VG(float, 4) } else if (la.rk == 5) { SBE_VG(float, 5) }
        }
#undef SBE_VG
        return cudaErrorInvalidValue;
    }
    if (la.variant == VAR_HALDANE_LW) {
        if (la.kpt == 2 && la.precision != PREC_FP64) {   // the packed mixed kernel
            if (la.rk == 4) return g1 ? launch_lw_x2_t<4, true>(la) : launch_lw_x2_t<4, false>(la);
            if (la.rk == 5) return g1 ? launch_lw_x2_t<5, true>(la) : launch_lw_x2_t<5, false>(la);
            return cudaErrorInvalidValue;
        }
        if (la.kpt != 1) return cudaErrorInvalidValue;
        if (la.precision == PREC_FP64) {
            if (la.rk == 4) return launch_lw_t<double, 4>(la, g1);
            if (la.rk == 5) return launch_lw_t<double, 5>(la, g1);
        } else {
            if (la.rk == 4) return launch_lw_t<float, 4>(la, g1);
            if (la.rk == 5) return launch_lw_t<float, 5>(la, g1);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_reduce(const SolveDev *solves, const int *solve_ids, int nsolves, int tick, int S,
                          cudaStream_t stream)
{
    if (nsolves <= 0) return cudaSuccess;
    dim3 grid(S, nsolves);
    reduce_tiles<<<grid, 256, 0, stream>>>(solves, solve_ids, tick, S);
    return cudaGetLastError();
}

cudaError_t launch_init_haldane(const InitArgs &ia, int precision, void *kc, void *st, double *constpart,
                                cudaStream_t stream)
{
    const int ntiles = (ia.nk + ia.tile_k - 1) / ia.tile_k;
    if (precision == PREC_FP64)
        init_haldane<double><<<ntiles, 256, 0, stream>>>(ia, static_cast<double *>(kc), static_cast<double *>(st),
                                                         constpart);
    else
        init_haldane<float><<<ntiles, 256, 0, stream>>>(ia, static_cast<float *>(kc), static_cast<double *>(st),
                                                        constpart);
    return cudaGetLastError();
}

cudaError_t launch_snapshot_bins(const double *nc, int nk, int k_offset, const int N[3], int nshots, double *occ1d,
                                 cudaStream_t stream)
{
    if (nshots <= 0 || nk <= 0) return cudaSuccess;
    dim3 grid(N[0], nshots);
    snapshot_bins<<<grid, 256, 0, stream>>>(nc, nk, k_offset, N[0], N[1], N[2], occ1d);
    return cudaGetLastError();
}

cudaError_t launch_fma_peak(int which, int blocks, int iters, void *out, cudaStream_t stream)
{
    if (which == 0) fma_peak<double><<<blocks, 256, 0, stream>>>(static_cast<double *>(out), iters, 0.999999, 1e-7);
    else if (which == 1) fma_peak<float><<<blocks, 256, 0, stream>>>(static_cast<float *>(out), iters, 0.999999f, 1e-7f);
    else fma_peak_x2<<<blocks, 256, 0, stream>>>(static_cast<float *>(out), iters, 0.999999f, 1e-7f);
    return cudaGetLastError();
}

}  // namespace sbe
