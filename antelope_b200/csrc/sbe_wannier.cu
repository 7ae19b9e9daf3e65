// N-band Wannier tight-binding solves, length gauge (sm_100a).
//
// Reference: SBEs::GenDifferentialDM (SBEs.h:762-872) with a Wannier model
// (model form of Materials/Wannier90.h:297-387), the currents of
// SBEs::GenInterIntraCurrent / GenCurrent (SBEs.h:626-760) and the driver's
// k-sum (antelope.cpp:302-334).  Extension: Cash-Karp 4(5) steps with one
// step size per solve chosen from the max-norm error over all k.
//
// Work decomposition: one warp per k-point, the lanes own the upper-triangle
// elements of the Hermitian N x N matrices, the full matrices of the warp live
// in shared memory.  Per RK stage the warp
//   1. forms the phases e^{i(k+A)R} (per-k e^{ikR} times per-stage e^{iAR}),
//   2. sums H0(k+A), D_x, D_y over the lattice vectors (exact Fourier sums),
//   3. tracks the eigenbasis U of H0(k+A) with Jacobi rounds started from the
//      previous stage's U (the field moves k+A a little per stage),
//   4. evaluates -i[H0 + E.D, rho] and the eigenbasis dephasing, written as
//      g2 rho + (g1 - g2) U diag(U^dag rho U) U^dag (SBEs.h:831-861).
// The state rho (Wannier basis) is FP64 in global memory between attempts.
// Precision: the plain method is FP64 throughout; the mixed method does the
// Fourier synthesis (the dominant work) in FP32 and the dynamics in FP64.
// In the length gauge rho is O(1) (the valence projector moving with k+A), so
// FP32 rounding of -i[H0, rho] or of the eigenbasis would add a field-
// independent source that accumulates over the pulse; an FP32-synthesised H0
// only perturbs the model itself, smoothly.
#include <cuda_runtime.h>

#include <type_traits>

#include "sbe_wannier.h"

namespace sbe {

namespace {

template <class Real> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };

template <class T> __device__ __forceinline__ T cx(double re, double im)
{
    T r;
    r.x = (decltype(r.x))re;
    r.y = (decltype(r.y))im;
    return r;
}
template <class T> __device__ __forceinline__ T cmul(T a, T b)
{
    T r;
    r.x = fma(a.x, b.x, -(a.y * b.y));
    r.y = fma(a.x, b.y, a.y * b.x);
    return r;
}
template <class T> __device__ __forceinline__ T cmulc(T a, T b)  // conj(a) * b
{
    T r;
    r.x = fma(a.x, b.x, a.y * b.y);
    r.y = fma(a.x, b.y, -(a.y * b.x));
    return r;
}
template <class T> __device__ __forceinline__ void cfma(T &acc, T a, T b)  // acc += a b
{
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
template <class T> __device__ __forceinline__ void cfmac(T &acc, T a, T b)  // acc += conj(a) b
{
    acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
}
template <class T> __device__ __forceinline__ T cconj(T a)
{
    a.y = -a.y;
    return a;
}

// ---- laser on the device (laser.h:150-322), FP64
__device__ double envelope(const PulseDev &q, double t, bool d)
{
    const double ef = q.envfactor;
    double to;
    switch (q.env) {
        case 2:  // cos4
            if (fabs(t) > q.twidth) return 0;
            if (d) return -4. * ef * sin(t * ef) * pow(cos(t * ef), 3.);
            return pow(cos(t * ef), 4.);
        case 4:  // sin2 (extension)
            if (fabs(t) > q.twidth) return 0;
            if (d) return -2. * ef * sin(t * ef) * cos(t * ef);
            return cos(t * ef) * cos(t * ef);
        case 3:  // cos4_clipped
            if (fabs(t) > q.twidth) return 0;
            if (t > q.twidth_clipped) to = t - q.twidth_clipped;
            else if (t > -q.twidth_clipped) return d ? 0. : 1.;
            else to = t + q.twidth_clipped;
            if (d) return -4. * ef * sin(to * ef) * pow(cos(to * ef), 3.);
            return pow(cos(to * ef), 4.);
        case 0:  // gauss
            if (d) return 2 * t * ef * exp(ef * t * t);
            return exp(ef * t * t);
        default:  // gauss_clipped
            if (t > q.twidth_clipped) to = t - q.twidth_clipped;
            else if (t > -q.twidth_clipped) return d ? 0. : 1.;
            else to = t + q.twidth_clipped;
            if (d) return 2 * to * ef * exp(ef * to * to);
            return exp(ef * to * to);
    }
}

__device__ void laser_eval(const LaserDev &L, double t, double *A, double *E)
{
    double a[3] = {0, 0, 0}, e[3] = {0, 0, 0};
    for (int i = 0; i < L.npulses; ++i) {
        const PulseDev &q = L.p[i];
        const double kt = t - q.t0;
        double s, c;
        sincos(kt * q.w0 - q.cep, &s, &c);
        const double f = envelope(q, kt, false), fp = envelope(q, kt, true);
        const double ax = -q.A0x * s * f, ay = q.A0y * c * f;
        const double ex = q.E0x * c * f - q.A0x * s * fp;
        const double ey = q.E0y * s * f + q.A0y * c * fp;
        for (int dd = 0; dd < 3; ++dd) {
            a[dd] += ax * q.xdir[dd] + ay * q.ydir[dd];
            e[dd] += ex * q.xdir[dd] + ey * q.ydir[dd];
        }
    }
    for (int dd = 0; dd < 3; ++dd) {
        A[dd] = a[dd] - L.init_A[dd];
        E[dd] = e[dd] - L.init_E[dd];
    }
}

// ---- tableaux (SBEs.h:395-416; Cash-Karp 4(5) for the adaptive steps)
struct WTab {
    int S;
    double c[6], a[6][6], b[6], e[6];  // e = b - b* (error weights)
};
__device__ void tableau(int rk, WTab &T)
{
    for (int i = 0; i < 6; ++i) {
        T.c[i] = T.b[i] = T.e[i] = 0;
        for (int j = 0; j < 6; ++j) T.a[i][j] = 0;
    }
    if (rk == 4) {
        T.S = 4;
        T.c[1] = 0.5; T.c[2] = 0.5; T.c[3] = 1.0;
        T.a[1][0] = 0.5; T.a[2][1] = 0.5; T.a[3][2] = 1.0;
        T.b[0] = 1.0 / 6.0; T.b[1] = 2.0 / 6.0; T.b[2] = 2.0 / 6.0; T.b[3] = 1.0 / 6.0;
    } else if (rk == 5) {
        T.S = 6;
        T.c[1] = 0.25; T.c[2] = 3. / 8.; T.c[3] = 12. / 13.; T.c[4] = 1.0; T.c[5] = 0.5;
        T.a[1][0] = 1.0 / 4.0;
        T.a[2][0] = 3. / 32.; T.a[2][1] = 9. / 32.;
        T.a[3][0] = 1932. / 2197.; T.a[3][1] = -7200. / 2197.; T.a[3][2] = 7296. / 2197.;
        T.a[4][0] = 439. / 216.; T.a[4][1] = -8.; T.a[4][2] = 3680. / 513.; T.a[4][3] = -845. / 4104.;
        T.a[5][0] = -8. / 27.; T.a[5][1] = 2.; T.a[5][2] = -3544. / 2565; T.a[5][3] = 1859. / 4104;
        T.a[5][4] = -11. / 40.;
        T.b[0] = 16. / 135.; T.b[2] = 6656. / 12825.; T.b[3] = 28561. / 56430.; T.b[4] = -9. / 50.;
        T.b[5] = 2. / 55.;
    } else {  // Cash-Karp (J. R. Cash, A. H. Karp, ACM TOMS 16 (1990) 201)
        T.S = 6;
        T.c[1] = 1. / 5.; T.c[2] = 3. / 10.; T.c[3] = 3. / 5.; T.c[4] = 1.; T.c[5] = 7. / 8.;
        T.a[1][0] = 1. / 5.;
        T.a[2][0] = 3. / 40.; T.a[2][1] = 9. / 40.;
        T.a[3][0] = 3. / 10.; T.a[3][1] = -9. / 10.; T.a[3][2] = 6. / 5.;
        T.a[4][0] = -11. / 54.; T.a[4][1] = 5. / 2.; T.a[4][2] = -70. / 27.; T.a[4][3] = 35. / 27.;
        T.a[5][0] = 1631. / 55296.; T.a[5][1] = 175. / 512.; T.a[5][2] = 575. / 13824.;
        T.a[5][3] = 44275. / 110592.; T.a[5][4] = 253. / 4096.;
        T.b[0] = 37. / 378.; T.b[2] = 250. / 621.; T.b[3] = 125. / 594.; T.b[5] = 512. / 1771.;
        const double bs[6] = {2825. / 27648., 0., 18575. / 48384., 13525. / 55296., 277. / 14336., 1. / 4.};
        for (int i = 0; i < 6; ++i) T.e[i] = T.b[i] - bs[i];
    }
}

// upper-triangle element u of an N x N matrix -> (m, n), m <= n
__device__ __forceinline__ void upper_mn(int u, int N, int &m, int &n)
{
    m = 0;
    int row = N;
    while (u >= row) {
        u -= row;
        ++m;
        --row;
    }
    n = m + u;
}

// Per-warp shared-memory workspace (full N x N matrices, row-major).  Real
// is the precision of the dynamics, RF the precision of the Fourier sums.
template <class Real, class RF> struct WarpMem {
    using T = typename Cx<Real>::T;
    using TF = typename Cx<RF>::T;
    T Y[64], H0[64], HT[64], U[64], B[64], Tm[64], D0[64], D1[64], S0[64], S1[64];
    TF ph[WAN_MAXR];  // e^{i(k+A)R} of the current stage
    TF pk[WAN_MAXR];  // e^{ikR}
    T dv[WAN_MAXN];   // diag(U^dag Y U)
    T rot[WAN_MAXN / 2 + 1];
    Real rc[WAN_MAXN / 2 + 1], rs[WAN_MAXN / 2 + 1];
    int mate[WAN_MAXN + 1], role[WAN_MAXN + 1], pidx[WAN_MAXN + 1];
};

// C = op(A) * B over the full matrices, lanes stride over the elements.
template <class T> __device__ void mat_mul(T *C, const T *A, const T *B, int N, bool conjA, int lane)
{
    for (int e = lane; e < N * N; e += 32) {
        const int m = e / N, n = e % N;
        T acc = cx<T>(0, 0);
        for (int l = 0; l < N; ++l) {
            if (conjA) cfmac(acc, A[l * N + m], B[l * N + n]);
            else cfma(acc, A[m * N + l], B[l * N + n]);
        }
        C[e] = acc;
    }
}

// One parallel Jacobi round on (B, U): the round-robin pairs of round r are
// disjoint, so their rotations are applied at once.  B <- J^dag B J, U <- U J.
template <class Real, class RF> __device__ void jacobi_round(WarpMem<Real, RF> &w, int N, int r, int lane)
{
    using T = typename Cx<Real>::T;
    const int P = N + (N & 1), np = P / 2;
    if (lane < np) {
        int p, q;
        if (lane == 0) { p = P - 1; q = r; }
        else { p = (r + lane) % (P - 1); q = (r - lane + (P - 1)) % (P - 1); }
        if (p > q) { const int t = p; p = q; q = t; }
        Real c = 1, s = 0;
        T e = cx<T>(1, 0);
        if (q < N) {
            const T g = w.B[p * N + q];
            const Real rr = sqrt(g.x * g.x + g.y * g.y);
            const Real app = w.B[p * N + p].x, aqq = w.B[q * N + q].x;
            if (rr > Real(0)) {
                e.x = g.x / rr;
                e.y = g.y / rr;
                const Real zeta = (aqq - app) / (Real(2) * rr);
                const Real t = (zeta >= 0 ? Real(1) : Real(-1)) / (fabs(zeta) + sqrt(zeta * zeta + Real(1)));
                c = Real(1) / sqrt(t * t + Real(1));
                s = t * c;
            }
            w.mate[p] = q; w.role[p] = 0; w.pidx[p] = lane;
            w.mate[q] = p; w.role[q] = 1; w.pidx[q] = lane;
        } else {
            if (p < N) { w.mate[p] = -1; }
        }
        w.rc[lane] = c;
        w.rs[lane] = s;
        w.rot[lane] = e;
    }
    __syncwarp();
    // column operation on B and U: tasks (row i, pair k)
    for (int task = lane; task < N * np; task += 32) {
        const int i = task / np, k = task % np;
        int p = -1, q = -1;
        for (int x = 0; x < N; ++x)
            if (w.pidx[x] == k && w.mate[x] >= 0 && w.role[x] == 0) { p = x; q = w.mate[x]; }
        if (p < 0) continue;
        const Real c = w.rc[k], s = w.rs[k];
        const T e = w.rot[k];
        // J_pp = c, J_pq = s, J_qp = -s conj(e), J_qq = c conj(e)
        const T Jqp = cx<T>(-s * e.x, s * e.y), Jqq = cx<T>(c * e.x, -c * e.y);
        T bp = w.B[i * N + p], bq = w.B[i * N + q];
        T np_ = cx<T>(c * bp.x, c * bp.y), nq = cx<T>(s * bp.x, s * bp.y);
        cfma(np_, bq, Jqp);
        cfma(nq, bq, Jqq);
        w.B[i * N + p] = np_;
        w.B[i * N + q] = nq;
        T up = w.U[i * N + p], uq = w.U[i * N + q];
        T nup = cx<T>(c * up.x, c * up.y), nuq = cx<T>(s * up.x, s * up.y);
        cfma(nup, uq, Jqp);
        cfma(nuq, uq, Jqq);
        w.U[i * N + p] = nup;
        w.U[i * N + q] = nuq;
    }
    __syncwarp();
    // row operation on B: tasks (column j, pair k)
    for (int task = lane; task < N * np; task += 32) {
        const int j = task / np, k = task % np;
        int p = -1, q = -1;
        for (int x = 0; x < N; ++x)
            if (w.pidx[x] == k && w.mate[x] >= 0 && w.role[x] == 0) { p = x; q = w.mate[x]; }
        if (p < 0) continue;
        const Real c = w.rc[k], s = w.rs[k];
        const T e = w.rot[k];
        const T Jqp = cx<T>(-s * e.x, s * e.y), Jqq = cx<T>(c * e.x, -c * e.y);
        const T bp = w.B[p * N + j], bq = w.B[q * N + j];
        // B'_pj = conj(J_pp) b_pj + conj(J_qp) b_qj ; B'_qj = conj(J_pq) b_pj + conj(J_qq) b_qj
        T np_ = cx<T>(c * bp.x, c * bp.y), nq = cx<T>(s * bp.x, s * bp.y);
        cfmac(np_, Jqp, bq);
        cfmac(nq, Jqq, bq);
        w.B[p * N + j] = np_;
        w.B[q * N + j] = nq;
    }
    __syncwarp();
    if (lane < N) { w.pidx[lane] = -1; w.mate[lane] = -1; }
    __syncwarp();
}

// Sweeps until the off-diagonal part of B is negligible against its diagonal
// (|offdiag|^2 <= tol2 |diag|^2, warp-uniform test), at most max_sweeps.
template <class Real, class RF>
__device__ void jacobi_sweeps(WarpMem<Real, RF> &w, int N, int max_sweeps, double tol2, int lane)
{
    const int P = N + (N & 1);
    for (int s = 0; s < max_sweeps; ++s) {
        double off = 0.0, dia = 0.0;
        for (int e = lane; e < N * N; e += 32) {
            const double v = double(w.B[e].x) * double(w.B[e].x) + double(w.B[e].y) * double(w.B[e].y);
            if (e / N == e % N) dia += v;
            else off += v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            dia += __shfl_xor_sync(0xffffffffu, dia, o);
        }
        if (off <= tol2 * dia) break;
        for (int r = 0; r < P - 1; ++r) jacobi_round<Real, RF>(w, N, r, lane);
    }
}

// Fourier sums at the phases w.ph: H0, D0, D1 and (optionally) S_a = sum R_a h_R e^{i(k+A)R}.
template <class Real, class RF>
__device__ void fourier(WarpMem<Real, RF> &w, const WanDev &P, bool with_S, const RF (*Rc)[2], int lane)
{
    using T = typename Cx<Real>::T;
    using TF = typename Cx<RF>::T;
    const int N = P.N, NN = N * N, NU = N * (N + 1) / 2;
    const TF *h = static_cast<const TF *>(P.h);
    const TF *d = static_cast<const TF *>(P.d);
    for (int u = lane; u < NU; u += 32) {
        int m, n;
        upper_mn(u, N, m, n);
        const int e = m * N + n;
        TF hs = cx<TF>(0, 0), d0 = cx<TF>(0, 0), d1 = cx<TF>(0, 0), s0 = cx<TF>(0, 0), s1 = cx<TF>(0, 0);
        for (int r = 0; r < P.nR; ++r) {
            const TF t = cmul(h[(size_t)r * NN + e], w.ph[r]);
            hs.x += t.x;
            hs.y += t.y;
            if (with_S) {
                s0.x = fma(Rc[r][0], t.x, s0.x);
                s0.y = fma(Rc[r][0], t.y, s0.y);
                s1.x = fma(Rc[r][1], t.x, s1.x);
                s1.y = fma(Rc[r][1], t.y, s1.y);
            }
            if (P.has_dip) {
                cfma(d0, d[((size_t)r * 2 + 0) * NN + e], w.ph[r]);
                cfma(d1, d[((size_t)r * 2 + 1) * NN + e], w.ph[r]);
            }
        }
        const T H = cx<T>(hs.x, hs.y), Dx = cx<T>(d0.x, d0.y), Dy = cx<T>(d1.x, d1.y);
        w.H0[e] = H;
        w.H0[n * N + m] = cconj(H);
        w.D0[e] = Dx;
        w.D0[n * N + m] = cconj(Dx);
        w.D1[e] = Dy;
        w.D1[n * N + m] = cconj(Dy);
        if (with_S) {
            w.S0[e] = cx<T>(s0.x, s0.y);
            w.S1[e] = cx<T>(s1.x, s1.y);
        }
    }
    if (with_S) {
        // S_a = sum R_a h_R e^{iKR} is anti-Hermitian (h_{-R} = h_R^dag), so
        // (S_a)_nm = -conj((S_a)_mn) and -i S_a = -dH/dk_a is Hermitian
        __syncwarp();
        for (int u = lane; u < NU; u += 32) {
            int m, n;
            upper_mn(u, N, m, n);
            if (m != n) {
                const T a = w.S0[m * N + n], b = w.S1[m * N + n];
                w.S0[n * N + m] = cx<T>(-a.x, a.y);
                w.S1[n * N + m] = cx<T>(-b.x, b.y);
            }
        }
    }
    __syncwarp();
}

template <class Real, class RF> struct BlockMem {
    using TF = typename Cx<RF>::T;
    TF cA[6][WAN_MAXR];         // e^{i A(t_s) R} per stage
    RF Rc[WAN_MAXR][2];         // Cartesian lattice vectors
    double AE[6][6];            // A and E at the stage times
    double part[WAN_WARPS][WAN_NSLOT];
    double errw[WAN_WARPS];
    WTab tab;
};

template <class Real, class RF> constexpr size_t wan_smem_bytes()
{
    return ((sizeof(BlockMem<Real, RF>) + 15) / 16) * 16 + sizeof(WarpMem<Real, RF>) * WAN_WARPS;
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace

// ============================================================= init
template <class Real, class RF>
__global__ void __launch_bounds__(32 * WAN_WARPS) wan_init(WanDev P)
{
    using T = typename Cx<Real>::T;
    using TF = typename Cx<RF>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BlockMem<Real, RF> &bm = *reinterpret_cast<BlockMem<Real, RF> *>(smem_raw);
    WarpMem<Real, RF> *wm =
        reinterpret_cast<WarpMem<Real, RF> *>(smem_raw + ((sizeof(BlockMem<Real, RF>) + 15) / 16) * 16);
    RF(*Rc)[2] = bm.Rc;
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    for (int r = threadIdx.x; r < P.nR; r += blockDim.x) {
        Rc[r][0] = RF(P.R[2 * r] * P.lat[0] + P.R[2 * r + 1] * P.lat[2]);
        Rc[r][1] = RF(P.R[2 * r] * P.lat[1] + P.R[2 * r + 1] * P.lat[3]);
    }
    __syncthreads();
    const int k = blockIdx.x * WAN_WARPS + wi;
    if (k >= P.nk) return;
    WarpMem<Real, RF> &w = wm[wi];
    const int N = P.N, NN = N * N;
    // k-grid point and trapezoid weight (momaxis.h:147-186, 349-383)
    const int N0 = P.Ngrid[0], N1 = P.Ngrid[1], N2 = P.Ngrid[2];
    const int ii[3] = {k / (N1 * N2), (k / N2) % N1, k % N2};
    const int NNg[3] = {N0, N1, N2};
    double f[3], wt = 1.0;
    for (int dd = 0; dd < 3; ++dd) {
        f[dd] = (NNg[dd] == 1) ? 0.0 : double(ii[dd]) / (NNg[dd] - 1) - 0.5;
        if (NNg[dd] != 1 && (ii[dd] == 0 || ii[dd] == NNg[dd] - 1)) wt /= 2;
    }
    double kv[3];
    for (int dd = 0; dd < 3; ++dd)
        kv[dd] = P.origin[dd] + f[0] * P.axes[0 * 3 + dd] + f[1] * P.axes[1 * 3 + dd] + f[2] * P.axes[2 * 3 + dd];
    if (lane == 0) P.weight[k] = wt;
    for (int r = lane; r < P.nR; r += 32) {
        const double Rx = P.R[2 * r] * P.lat[0] + P.R[2 * r + 1] * P.lat[2];
        const double Ry = P.R[2 * r] * P.lat[1] + P.R[2 * r + 1] * P.lat[3];
        double s, c;
        sincos(kv[0] * Rx + kv[1] * Ry, &s, &c);
        w.ph[r] = cx<TF>(c, s);
    }
    for (int e = lane; e < NN; e += 32) w.U[e] = cx<T>((e / N) == (e % N) ? 1 : 0, 0);
    if (lane < WAN_MAXN + 1) { w.pidx[lane] = -1; w.mate[lane] = -1; }
    __syncwarp();
    fourier<Real, RF>(w, P, false, Rc, lane);
    for (int e = lane; e < NN; e += 32) w.B[e] = w.H0[e];
    __syncwarp();
    jacobi_sweeps<Real, RF>(w, N, 16, 1e-30, lane);
    // occupations of the eigenstates: the Nval lowest filled, or Fermi-Dirac (SBEs.h:319-340)
    if (lane < N) {
        const Real ev = w.B[lane * N + lane].x;
        int rank = 0;
        for (int j = 0; j < N; ++j) {
            const Real ej = w.B[j * N + j].x;
            rank += (ej < ev) || (ej == ev && j < lane);
        }
        double occ;
        if (P.use_fermi) occ = 1.0 / (exp((double(ev) - P.Ef) / (300. / 3.15775024804e5)) + 1.0);
        else occ = rank < P.nval ? 1.0 : 0.0;
        w.dv[lane] = cx<T>(occ, 0);
    }
    __syncwarp();
    if (P.use_fermi && lane == 0) {
        double s = 0;
        for (int j = 0; j < N; ++j) s += double(w.dv[j].x);
        for (int j = 0; j < N; ++j) w.dv[j] = cx<T>(double(w.dv[j].x) / s, 0);
    }
    __syncwarp();
    // rho0 = U diag(f) U^dag (SBEs.h:352-356), FP64 state
    for (int e = lane; e < NN; e += 32) {
        const int m = e / N, n = e % N;
        double2 acc = make_double2(0, 0);
        for (int p = 0; p < N; ++p) {
            const T a = w.U[m * N + p], b = w.U[n * N + p];
            const double fp = double(w.dv[p].x);
            acc.x += fp * (double(a.x) * double(b.x) + double(a.y) * double(b.y));
            acc.y += fp * (double(a.y) * double(b.x) - double(a.x) * double(b.y));
        }
        P.rho[0][(size_t)k * NN + e] = acc;
        static_cast<T *>(P.U[0])[(size_t)k * NN + e] = w.U[e];
    }
}

// ============================================================= attempt
template <class Real, class RF>
__global__ void __launch_bounds__(32 * WAN_WARPS) wan_attempt(const WanDev *__restrict__ Pp)
{
    using T = typename Cx<Real>::T;
    using TF = typename Cx<RF>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BlockMem<Real, RF> &bm = *reinterpret_cast<BlockMem<Real, RF> *>(smem_raw);
    WarpMem<Real, RF> *wm =
        reinterpret_cast<WarpMem<Real, RF> *>(smem_raw + ((sizeof(BlockMem<Real, RF>) + 15) / 16) * 16);
    TF(*cA)[WAN_MAXR] = bm.cA;
    RF(*Rc)[2] = bm.Rc;
    double(*AE)[6] = bm.AE;
    WTab &tab = bm.tab;
    const WanDev &P = *Pp;
    const WanCtl ctl = *P.ctl;
    if (ctl.done) return;
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const int N = P.N, NN = N * N, NU = N * (N + 1) / 2;
    const double h = ctl.hs, tc = ctl.tc;
    const int buf = ctl.buf;
    const bool cur = ctl.need_current;
    if (threadIdx.x == 0) tableau(P.rk, tab);
    for (int r = threadIdx.x; r < P.nR; r += blockDim.x) {
        Rc[r][0] = RF(P.R[2 * r] * P.lat[0] + P.R[2 * r + 1] * P.lat[2]);
        Rc[r][1] = RF(P.R[2 * r] * P.lat[1] + P.R[2 * r + 1] * P.lat[3]);
    }
    __syncthreads();
    const int S = tab.S;
    if (threadIdx.x < S) {  // field at the stage times (SBEs.h:764-766)
        double A[3], E[3];
        const double ts = threadIdx.x == 0 ? tc : tc + tab.c[threadIdx.x] * h;
        laser_eval(P.laser, ts, A, E);
        for (int dd = 0; dd < 3; ++dd) { AE[threadIdx.x][dd] = A[dd]; AE[threadIdx.x][3 + dd] = E[dd]; }
    }
    __syncthreads();
    for (int task = threadIdx.x; task < S * P.nR; task += blockDim.x) {
        const int s = task / P.nR, r = task % P.nR;
        const double Rx = P.R[2 * r] * P.lat[0] + P.R[2 * r + 1] * P.lat[2];
        const double Ry = P.R[2 * r] * P.lat[1] + P.R[2 * r + 1] * P.lat[3];
        double sn, cs;
        sincos(AE[s][0] * Rx + AE[s][1] * Ry, &sn, &cs);
        cA[s][r] = cx<TF>(cs, sn);
    }
    for (int q = threadIdx.x; q < WAN_WARPS * WAN_NSLOT; q += blockDim.x) bm.part[q / WAN_NSLOT][q % WAN_NSLOT] = 0.0;
    if (threadIdx.x < WAN_WARPS) bm.errw[threadIdx.x] = 0.0;
    __syncthreads();

    const int k = blockIdx.x * WAN_WARPS + wi;
    double emax = 0.0;
    if (k < P.nk) {
        WarpMem<Real, RF> &w = wm[wi];
        if (lane < WAN_MAXN + 1) { w.pidx[lane] = -1; w.mate[lane] = -1; }
        // grid point (momaxis.h:349-383) and e^{ikR}
        const int N1 = P.Ngrid[1], N2 = P.Ngrid[2];
        const int ii[3] = {k / (N1 * N2), (k / N2) % N1, k % N2};
        const int NNg[3] = {P.Ngrid[0], N1, N2};
        double kv[3], f[3];
        for (int dd = 0; dd < 3; ++dd) f[dd] = (NNg[dd] == 1) ? 0.0 : double(ii[dd]) / (NNg[dd] - 1) - 0.5;
        for (int dd = 0; dd < 3; ++dd)
            kv[dd] = P.origin[dd] + f[0] * P.axes[dd] + f[1] * P.axes[3 + dd] + f[2] * P.axes[6 + dd];
        for (int r = lane; r < P.nR; r += 32) {
            const double Rx = P.R[2 * r] * P.lat[0] + P.R[2 * r + 1] * P.lat[2];
            const double Ry = P.R[2 * r] * P.lat[1] + P.R[2 * r + 1] * P.lat[3];
            double sn, cs;
            sincos(kv[0] * Rx + kv[1] * Ry, &sn, &cs);
            w.pk[r] = cx<TF>(cs, sn);
        }
        const double2 *rho = P.rho[buf] + (size_t)k * NN;
        const T *Ug = static_cast<const T *>(P.U[buf]) + (size_t)k * NN;
        for (int e = lane; e < NN; e += 32) w.U[e] = Ug[e];
        // owned upper elements: committed state (FP64) and the stage slopes
        constexpr int MAXO = 2;
        double2 r64[MAXO];
        T ks[6][MAXO];
        int om[MAXO], on[MAXO];
        const int no = (NU + 31 - lane) / 32;
        for (int o = 0; o < MAXO; ++o) {
            om[o] = on[o] = 0;
            r64[o] = make_double2(0, 0);
            if (o < no) {
                upper_mn(lane + 32 * o, N, om[o], on[o]);
                r64[o] = rho[om[o] * N + on[o]];
            }
        }
        const double wk = P.weight[k];
        for (int s = 0; s < S; ++s) {
            // stage input Y = rho + h sum_j a_sj k_j (owned elements, mirrored)
            for (int o = 0; o < no; ++o) {
                T y = cx<T>(r64[o].x, r64[o].y);
                for (int j = 0; j < s; ++j) {
                    const Real a = Real(h * tab.a[s][j]);
                    if (a != Real(0)) {
                        y.x = fma(a, ks[j][o].x, y.x);
                        y.y = fma(a, ks[j][o].y, y.y);
                    }
                }
                const int m = om[o], n = on[o];
                if (m == n) y.y = 0;
                w.Y[m * N + n] = y;
                w.Y[n * N + m] = cconj(y);
            }
            for (int r = lane; r < P.nR; r += 32) w.ph[r] = cmul(w.pk[r], cA[s][r]);
            __syncwarp();
            const bool with_cur = cur && s == 0;
            fourier<Real, RF>(w, P, with_cur, Rc, lane);
            // H = H0 + E.D (SBEs.h:770-783)
            const Real Ex = Real(AE[s][3]), Ey = Real(AE[s][4]);
            for (int e = lane; e < NN; e += 32) {
                T v = w.H0[e];
                if (P.has_dip) {
                    v.x = fma(Ex, w.D0[e].x, fma(Ey, w.D1[e].x, v.x));
                    v.y = fma(Ex, w.D0[e].y, fma(Ey, w.D1[e].y, v.y));
                }
                w.HT[e] = v;
            }
            // eigenbasis of H0(k+A): B = U^dag H0 U, then Jacobi rounds (warm start)
            mat_mul<T>(w.Tm, w.H0, w.U, N, false, lane);
            __syncwarp();
            mat_mul<T>(w.B, w.U, w.Tm, N, true, lane);
            __syncwarp();
            jacobi_sweeps<Real, RF>(w, N, 6, 1e-30, lane);
            // diag(U^dag Y U)
            mat_mul<T>(w.Tm, w.Y, w.U, N, false, lane);
            __syncwarp();
            if (lane < N) {
                T acc = cx<T>(0, 0);
                for (int l = 0; l < N; ++l) cfmac(acc, w.U[l * N + lane], w.Tm[l * N + lane]);
                w.dv[lane] = acc;
            }
            __syncwarp();
            if (with_cur) {
                // currents at k + A(t_n) (SBEs.h:694-760): J_a = -i S_a + i[D_a, H0]
                double val[WAN_NSLOT];
                for (int q = 0; q < WAN_NSLOT; ++q) val[q] = 0.0;
                for (int a = 0; a < 2; ++a) {
                    T *Da = a == 0 ? w.D0 : w.D1;
                    T *Sa = a == 0 ? w.S0 : w.S1;
                    // J_a into B (B is free after the rounds above), then total = Re Tr(Y J_a)
                    for (int e = lane; e < NN; e += 32) {
                        const int m = e / N, n = e % N;
                        T c = cx<T>(0, 0);
                        for (int l = 0; l < N; ++l) {
                            cfma(c, Da[m * N + l], w.H0[l * N + n]);
                            const T t2 = cmul(w.H0[m * N + l], Da[l * N + n]);
                            c.x -= t2.x;
                            c.y -= t2.y;
                        }
                        // -i S + i c = (S.y - c.y, -S.x + c.x)
                        w.B[e] = cx<T>(Sa[e].y - c.y, c.x - Sa[e].x);
                    }
                    __syncwarp();
                    double tot = 0.0;
                    for (int e = lane; e < NN; e += 32) {
                        const int m = e / N, n = e % N;
                        const T y = w.Y[e], j = w.B[n * N + m];
                        tot += double(y.x) * double(j.x) - double(y.y) * double(j.y);
                    }
                    tot = warp_sum(tot);
                    // intra = sum_n Re[(U^dag Y U)_nn (U^dag J_a U)_nn]
                    mat_mul<T>(w.Tm, w.B, w.U, N, false, lane);
                    __syncwarp();
                    double intra = 0.0;
                    if (lane < N) {
                        T p = cx<T>(0, 0);
                        for (int l = 0; l < N; ++l) cfmac(p, w.U[l * N + lane], w.Tm[l * N + lane]);
                        intra = double(w.dv[lane].x) * double(p.x) - double(w.dv[lane].y) * double(p.y);
                    }
                    intra = warp_sum(intra);
                    val[a] = wk * (tot - intra);
                    val[2 + a] = wk * intra;
                    __syncwarp();
                }
                for (int m = 0; m < N; ++m) val[4 + m] = wk * double(w.Y[m * N + m].x);
                const int ce = (P.nval * N + P.nval + 1) % NN;  // antelope.cpp:539-542
                val[4 + N] = wk * double(w.Y[ce].x);
                val[5 + N] = wk * double(w.Y[ce].y);
                if (lane == 0)
                    for (int q = 0; q < WAN_NSLOT; ++q) bm.part[wi][q] = val[q];
                __syncwarp();
            }
            // RHS for owned elements: -i[HT, Y] - (g2 Y + (g1-g2) U diag(dv) U^dag)
            const Real g1 = Real(P.g1), g2 = Real(P.g2);
            for (int o = 0; o < no; ++o) {
                const int m = om[o], n = on[o];
                T c = cx<T>(0, 0);
                for (int l = 0; l < N; ++l) {
                    cfma(c, w.HT[m * N + l], w.Y[l * N + n]);
                    const T t2 = cmul(w.Y[m * N + l], w.HT[l * N + n]);
                    c.x -= t2.x;
                    c.y -= t2.y;
                }
                T kv2 = cx<T>(c.y, -c.x);  // -i [H, Y]
                if (g1 != Real(0) || g2 != Real(0)) {
                    T pr = cx<T>(0, 0);
                    for (int p = 0; p < N; ++p) {
                        const T um = w.U[m * N + p], un = w.U[n * N + p];
                        const T t2 = cmul(um, w.dv[p]);
                        cfma(pr, t2, cconj(un));
                    }
                    const T y = w.Y[m * N + n];
                    kv2.x -= g2 * y.x + (g1 - g2) * pr.x;
                    kv2.y -= g2 * y.y + (g1 - g2) * pr.y;
                }
                ks[s][o] = kv2;
            }
            __syncwarp();
        }
        // trial state and error estimate
        double2 *rout = P.rho[1 - buf] + (size_t)k * NN;
        for (int o = 0; o < no; ++o) {
            T inc = cx<T>(0, 0), er = cx<T>(0, 0);
            for (int s = 0; s < S; ++s) {
                const Real b = Real(h * tab.b[s]);
                if (b != Real(0)) {
                    inc.x = fma(b, ks[s][o].x, inc.x);
                    inc.y = fma(b, ks[s][o].y, inc.y);
                }
                const Real eb = Real(h * tab.e[s]);
                if (eb != Real(0)) {
                    er.x = fma(eb, ks[s][o].x, er.x);
                    er.y = fma(eb, ks[s][o].y, er.y);
                }
            }
            double2 v = make_double2(r64[o].x + double(inc.x), r64[o].y + double(inc.y));
            const int m = om[o], n = on[o];
            if (m == n) v.y = 0.0;
            rout[m * N + n] = v;
            rout[n * N + m] = make_double2(v.x, -v.y);
            emax = fmax(emax, sqrt(double(er.x) * double(er.x) + double(er.y) * double(er.y)));
        }
        T *Uo = static_cast<T *>(P.U[1 - buf]) + (size_t)k * NN;
        for (int e = lane; e < NN; e += 32) Uo[e] = w.U[e];
        emax = warp_max(emax);
        if (lane == 0) bm.errw[wi] = emax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < WAN_WARPS; ++i) m = fmax(m, bm.errw[i]);
        P.tile_err[blockIdx.x] = m;
    }
    if (cur && threadIdx.x < WAN_NSLOT) {
        double s = 0.0;
        for (int i = 0; i < WAN_WARPS; ++i) s += bm.part[i][threadIdx.x];
        P.cur_part[(size_t)blockIdx.x * WAN_NSLOT + threadIdx.x] = s;
    }
}

// ============================================================= control
// One block: reduce the attempt's tile results (fixed order), record the
// currents, accept or reject, and prepare the next attempt.  The step-size
// rule is the oracle's (oracle/sbe_oracle.c, run_adaptive).
__global__ void __launch_bounds__(1024) wan_control(const WanDev *__restrict__ Pp)
{
    __shared__ double red[1024];
    __shared__ double cs[WAN_NSLOT][64];
    const WanDev &P = *Pp;
    WanCtl *ctl = P.ctl;
    if (ctl->done) return;
    const int t = threadIdx.x, nt = P.ntiles;
    double m = 0.0;
    for (int i = t; i < nt; i += blockDim.x) m = fmax(m, P.tile_err[i]);
    red[t] = m;
    if (ctl->need_current) {
        // 16 slots x 64 groups; group g sums tiles g, g+64, ...
        const int slot = t % WAN_NSLOT, g = t / WAN_NSLOT;
        double s = 0.0;
        for (int i = g; i < nt; i += 64) s += P.cur_part[(size_t)i * WAN_NSLOT + slot];
        cs[slot][g] = s;
    }
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (t < o) red[t] = fmax(red[t], red[t + o]);
        __syncthreads();
    }
    if (ctl->need_current && t < WAN_NSLOT) {
        double s = 0.0;
        for (int g = 0; g < 64; ++g) s += cs[t][g];
        P.jout[(size_t)ctl->n * WAN_NSLOT + t] = s;
    }
    __syncthreads();
    if (t != 0) return;
    const double emax = red[0];
    ctl->attempts++;
    ctl->need_current = 0;
    ctl->emax = emax;
    const double dt = P.dt, tend = P.atmin + dt * (ctl->n + 1);
    bool accept = true;
    if (P.rk == 45) {
        if (emax <= P.tol) {
            double fac = emax > 0 ? 0.9 * pow(P.tol / emax, 0.2) : 5.0;
            if (fac > 5.0) fac = 5.0;
            if (!ctl->last || fac < 1.0) ctl->h = ctl->hs * (fac < 0.2 ? 0.2 : fac);
            if (ctl->h > dt) ctl->h = dt;
        } else {
            accept = false;
            double fac = 0.9 * pow(P.tol / emax, 0.25);
            ctl->h = ctl->hs * (fac < 0.1 ? 0.1 : fac);
            ctl->rejects++;
            if (!(ctl->h > 1e-12 * dt)) { ctl->error = 1; ctl->done = 1; return; }
        }
    }
    if (accept) {
        ctl->buf ^= 1;
        ctl->steps++;
        if (ctl->last) {
            ctl->tc = tend;
            ctl->n++;
            if (ctl->n >= P.Nt) { ctl->done = 1; return; }
            ctl->need_current = 1;
        } else {
            ctl->tc = ctl->tc + ctl->hs;
        }
    }
    // next attempt
    const double tend2 = P.atmin + dt * (ctl->n + 1);
    ctl->hs = ctl->h;
    ctl->last = 0;
    if (ctl->tc + ctl->hs >= tend2 - 1e-12 * dt) {
        ctl->hs = tend2 - ctl->tc;
        ctl->last = 1;
    }
}

// ============================================================= launchers
template <class RF> static cudaError_t allow_smem()
{
    static bool done = false;  // per process; the attribute applies to every device
    if (done) return cudaSuccess;
    const int bytes = (int)wan_smem_bytes<double, RF>();
    cudaError_t e = cudaFuncSetAttribute(wan_init<double, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(wan_attempt<double, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    done = e == cudaSuccess;
    return e;
}

cudaError_t launch_wan_init(const WanDev &w, int precision, cudaStream_t st)
{
    const int grid = (w.nk + WAN_WARPS - 1) / WAN_WARPS;
    cudaError_t e = precision == 0 ? allow_smem<double>() : allow_smem<float>();
    if (e != cudaSuccess) return e;
    if (precision == 0) wan_init<double, double><<<grid, 32 * WAN_WARPS, wan_smem_bytes<double, double>(), st>>>(w);
    else wan_init<double, float><<<grid, 32 * WAN_WARPS, wan_smem_bytes<double, float>(), st>>>(w);
    return cudaGetLastError();
}

cudaError_t launch_wan_attempt(const WanDev &w, const WanDev *dw, int precision, cudaStream_t st)
{
    const int grid = (w.nk + WAN_WARPS - 1) / WAN_WARPS;
    cudaError_t e = precision == 0 ? allow_smem<double>() : allow_smem<float>();
    if (e != cudaSuccess) return e;
    if (precision == 0)
        wan_attempt<double, double><<<grid, 32 * WAN_WARPS, wan_smem_bytes<double, double>(), st>>>(dw);
    else
        wan_attempt<double, float><<<grid, 32 * WAN_WARPS, wan_smem_bytes<double, float>(), st>>>(dw);
    return cudaGetLastError();
}

cudaError_t launch_wan_control(const WanDev *dw, cudaStream_t st)
{
    wan_control<<<1, 1024, 0, st>>>(dw);
    return cudaGetLastError();
}

}  // namespace sbe
