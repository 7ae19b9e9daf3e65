// Grouped attempt kernel of the N-band length gauge (included by
// sbe_wannier.cu inside its anonymous namespace; uses its helpers).
//
// The same step as wan_attempt -- SBEs::GenDifferentialDM (SBEs.h:762-872)
// with the Wannier model form (Materials/Wannier90.h:297-387), the currents
// of SBEs::GenInterIntraCurrent (SBEs.h:694-760), tracking of the eigenbasis
// and the eigenbasis dephasing -- laid out for throughput:
//
//  - eight lanes per k-point, four k-points per warp (one warp is one tile of
//    WAN_WARPS k-points, so the controller's tile reduction is unchanged);
//    the four groups of a warp run in lockstep, so every Fourier-table load is
//    one 128-byte row shared by the four k-points;
//  - the tables are re-laid per lane and per lattice-vector pair (R, -R)
//    ([pair][j][q][sigma|tau][lane], built on the host, WanDev::gtab): lane l
//    of a group owns the upper elements u = l + 8j and computes H0, E.D (or
//    D_x, D_y at output steps, and S_a = sum R_a h_R e^{iKR}) for exactly
//    those, with one phase and half the multiply-adds per pair;
//  - the matrix products (B = U^dag H0 U, the tracking steps, dv, the
//    commutators, the dephasing) are formed one row per lane, the second
//    factor read by element at an address shared by the group's lanes;
//  - Hermitian matrices (Y, H0, H0 + E.D, B = U^dag H0 U) are stored as packed
//    upper triangles, the unitary U and one scratch matrix in full: ~3.6 KB
//    of shared memory per k-point, so 3 blocks fit with 60 KB of L1 left for
//    the tables;
//  - the stage slopes live in registers and the stage loop is unrolled for the
//    compile-time tableau, so only the slopes still needed are live.
//
// The intraband current uses (U^dag J_a U)_nn = (U^dag (-i S_a) U)_nn: the
// i[D_a, H0] part of the current operator has zero diagonal in the eigenbasis
// of H0 (eps_n D_nn - D_nn eps_n), which the reference evaluates to rounding.
// Used for the tables of the SyntheticWannier group (current operator
// -dH/dk + i[D, H], BaseMaterial.h:62-68) at N = 4 and 6; other models and
// band counts run on wan_attempt.

// Tuning: resident blocks per SM the registers are sized for.  (Tables
// staged in shared memory, one copy per block, measured no faster than
// reading them through L1 and leave room for fewer blocks.)
#ifndef SBE_WG_MINB
#define SBE_WG_MINB 3
#endif
// |X|^2 up to which the plain method's larger tracking steps are second
// order (then U is restored to unitary once per attempt); 0: fourth order
#ifndef SBE_WG_X2_LOW
#define SBE_WG_X2_LOW 1e-6
#endif
constexpr int WG = 8;          // lanes per k-point
constexpr int WG_WARPS = 4;    // warps per block (tiles per block)
constexpr unsigned WG_FULL = 0xffffffffu;
static_assert(32 / WG == WAN_WARPS, "a warp of the grouped kernel is one tile");
static_assert(WG_WARPS == WAN_GROUP_TILES, "a block of the grouped kernel covers WAN_GROUP_TILES tiles");
static_assert(WG_WARPS == WAN_GROUP_TILES, "a block of the grouped kernel covers WAN_GROUP_TILES tiles");

__host__ __device__ constexpr int pidx(int m, int n, int N) { return m * N - m * (m - 1) / 2 + (n - m); }

template <int N> struct GDim {
    static constexpr int NN = N * N, NU = N * (N + 1) / 2;
    static constexpr int NO = (NU + WG - 1) / WG;   // owned upper elements per lane
    static constexpr int NF = (NN + WG - 1) / WG;   // full-matrix elements per lane
    static constexpr int NJ = (NU + NN + WG - 1) / WG;   // Jacobi tasks per lane
    static constexpr int P = N + (N & 1);           // indices of the round-robin schedule
};

// Hermitian element (a, b) of a packed upper triangle
template <int N> __device__ __forceinline__ double2 herm(const double2 *Pk, int a, int b)
{
    return a <= b ? Pk[pidx(a, b, N)] : cconj(Pk[pidx(b, a, N)]);
}
// anti-Hermitian element (a, b) of a packed upper triangle
template <int N> __device__ __forceinline__ double2 aherm(const double2 *Pk, int a, int b)
{
    if (a <= b) return Pk[pidx(a, b, N)];
    const double2 v = Pk[pidx(b, a, N)];
    return make_double2(-v.x, v.y);
}

__device__ __forceinline__ double grp_sum(double v)
{
    v += __shfl_xor_sync(WG_FULL, v, 1);
    v += __shfl_xor_sync(WG_FULL, v, 2);
    v += __shfl_xor_sync(WG_FULL, v, 4);
    return v;
}
__device__ __forceinline__ double grp_max(double v)
{
    v = fmax(v, __shfl_xor_sync(WG_FULL, v, 1));
    v = fmax(v, __shfl_xor_sync(WG_FULL, v, 2));
    v = fmax(v, __shfl_xor_sync(WG_FULL, v, 4));
    return v;
}

// Shared memory: block head, stage phase factors e^{iA(t_s)R} and the
// pairs' lattice vectors, then one region per k-point.
struct GHead {
    double AE[6][6];
    double part[WG_WARPS][WAN_WARPS][WAN_NSLOT];
    double errw[WG_WARPS];
    WTab tab;
    int gp[WAN_MAXR];   // lattice-vector index of each pair (R, -R)
    unsigned char ut[WAN_MAXU_][2];
    signed char mate[WAN_MAXN - 1][WAN_MAXN];
};
struct GSmem {
    size_t cA, Rc, k0, kbytes, total;
    // offsets inside a k-point region
    size_t Y, H0, HT, B, U, Tm, pk, ph, dv;
};
// lattice-vector pairs the per-k phase arrays hold: a grouped solve's vectors
// come in pairs (R, -R) but for at most one (R = 0)
__host__ __device__ constexpr int g_npair_cap(int nR) { return nR / 2 + 1; }
__host__ __device__ inline GSmem g_smem(int N, int nR, int rf_bytes)
{
    GSmem L;
    const size_t NU = (size_t)N * (N + 1) / 2, NN = (size_t)N * N, tf = 2 * (size_t)rf_bytes;
    L.cA = al16(sizeof(GHead));
    L.Rc = L.cA + al16(6 * (size_t)nR * tf);   // R of each lattice-vector pair
    L.k0 = L.Rc + al16((size_t)nR * 2 * rf_bytes);
    size_t o = 0;
    L.Y = o;  o += al16(NU * 16);
    L.H0 = o; o += al16(NU * 16);
    L.HT = o; o += al16(NU * 16);
    L.B = o;  o += al16(NU * 16);
    L.U = o;  o += al16(NN * 16);
    L.Tm = o; o += al16(NN * 16);
    const size_t np = (size_t)g_npair_cap(nR);
    L.pk = o; o += al16(np * tf);
    // the stage phases; also S_x (packed) at current steps, the tracker's
    // full scratch matrix and the rotations of a Jacobi round (c, s, phase)
    L.ph = o; o += al16(std::max(np * tf, std::max(NN * 16, (size_t)WAN_MAXN * 32)));
    L.dv = o; o += al16((size_t)N * 16);
    // k-point regions 32 bytes past a multiple of 128: the four groups of a
    // warp reading the same element of their matrices hit distinct banks
    L.kbytes = (o + 127) / 128 * 128 + 32;
    L.total = L.k0 + (size_t)WG_WARPS * WAN_WARPS * L.kbytes;
    return L;
}

template <class RF> struct GView {
    using TF = typename Cx<RF>::T;
    double2 *Y, *H0, *HT, *B, *U, *Tm, *je, *dv;
    double *jc, *js;
    TF *pk, *ph;
    __device__ GView(unsigned char *b, const GSmem &L)
    {
        Y = reinterpret_cast<double2 *>(b + L.Y);
        H0 = reinterpret_cast<double2 *>(b + L.H0);
        HT = reinterpret_cast<double2 *>(b + L.HT);
        B = reinterpret_cast<double2 *>(b + L.B);
        U = reinterpret_cast<double2 *>(b + L.U);
        Tm = reinterpret_cast<double2 *>(b + L.Tm);
        pk = reinterpret_cast<TF *>(b + L.pk);
        ph = reinterpret_cast<TF *>(b + L.ph);
        jc = reinterpret_cast<double *>(b + L.ph);
        js = jc + WAN_MAXN;
        je = reinterpret_cast<double2 *>(js + WAN_MAXN);
        dv = reinterpret_cast<double2 *>(b + L.dv);
    }
};

// Column j of a Jacobi round's rotation: J_jj and J_{mj,j} (as jcol)
template <class RF>
__device__ __forceinline__ void g_jcol(const GView<RF> &w, const signed char *mt, int j, int N, double2 &Jjj,
                                       double2 &Jmj, int &mj)
{
    mj = mt[j];
    if (mj >= N) {
        Jjj = make_double2(1, 0);
        Jmj = make_double2(0, 0);
        mj = j;
        return;
    }
    const int p = min(j, mj);
    const double c = w.jc[p], s = w.js[p];
    const double2 e = w.je[p];
    if (j == p) {
        Jjj = make_double2(c, 0);
        Jmj = make_double2(-s * e.x, s * e.y);
    } else {
        Jjj = make_double2(c * e.x, -c * e.y);
        Jmj = make_double2(s, 0);
    }
}

// One parallel Jacobi round on (B packed, U) of the group's k-point; `act`:
// this group still rotates (group-uniform).  All lanes of the warp call it.
template <class RF, int N>
__device__ __forceinline__ void g_round(const GView<RF> &w, const GHead &gh, int r, int gl, bool act)
{
    using D = GDim<N>;
    const signed char *mt = gh.mate[r];
    if (act && gl < N) {
        const int q = mt[gl];
        if (q < N && gl < q) {
            const int p = gl;
            const double2 g = w.B[pidx(p, q, N)];
            const double r2 = g.x * g.x + g.y * g.y;
            double c = 1, s = 0;
            double2 e = make_double2(1, 0);
            if (r2 > 0.0) {
                const double d = w.B[pidx(q, q, N)].x - w.B[pidx(p, p, N)].x;
                const double ir = rsqrt(r2);
                const double hh = sqrt(fma(d, d, 4.0 * r2));
                const double t = copysign(2.0 * r2 * ir, d) / (fabs(d) + hh);
                c = rsqrt(fma(t, t, 1.0));
                s = t * c;
                e.x = g.x * ir;
                e.y = g.y * ir;
            }
            w.jc[p] = c;
            w.js[p] = s;
            w.je[p] = e;
        }
    }
    __syncwarp();
    double2 out[D::NJ];
#pragma unroll
    for (int x = 0; x < D::NJ; ++x) {
        const int t = gl + WG * x;
        out[x] = make_double2(0, 0);
        if (!act || t >= D::NU + D::NN) continue;
        int i, j;
        if (t < D::NU) {
            i = gh.ut[t][0];
            j = gh.ut[t][1];
        } else {
            i = -1 - (t - D::NU) / N;
            j = (t - D::NU) % N;
        }
        double2 Jjj, Jmj;
        int mj;
        g_jcol<RF>(w, mt, j, N, Jjj, Jmj, mj);
        if (i >= 0) {   // B'_ij = sum_ab conj(J_ai) B_ab J_bj
            double2 Jii, Jmi;
            int mi;
            g_jcol<RF>(w, mt, i, N, Jii, Jmi, mi);
            double2 t1 = cmul(herm<N>(w.B, i, j), Jjj), t2 = cmul(herm<N>(w.B, mi, j), Jjj);
            cfma(t1, herm<N>(w.B, i, mj), Jmj);
            cfma(t2, herm<N>(w.B, mi, mj), Jmj);
            double2 o = make_double2(0, 0);
            cfmac(o, Jii, t1);
            cfmac(o, Jmi, t2);
            out[x] = o;
        } else {        // U'_ij = U_ij J_jj + U_i,mj J_mj,j
            const int row = -1 - i;
            double2 o = cmul(w.U[row * N + j], Jjj);
            cfma(o, w.U[row * N + mj], Jmj);
            out[x] = o;
        }
    }
    __syncwarp();
#pragma unroll
    for (int x = 0; x < D::NJ; ++x) {
        const int t = gl + WG * x;
        if (!act || t >= D::NU + D::NN) continue;
        if (t < D::NU) {
            const int i = gh.ut[t][0], j = gh.ut[t][1];
            w.B[t] = i == j ? make_double2(out[x].x, 0.0) : out[x];
        } else {
            w.U[t - D::NU] = out[x];
        }
    }
    __syncwarp();
}

// Eigenbasis tracking of the group's k-point (as jacobi_track): sweeps until
// |offdiag|^2 <= tol2 |diag|^2; once |offdiag|^2 <= 1e-10 |diag|^2 a
// first-order step U (I + X), X_mn = B_mn / (B_nn - B_mm), finishes when
// max |X| <= xmax.  Warp-uniform loop; groups that are done idle.
template <class RF, int N>
__device__ __forceinline__ void g_track(const GView<RF> &w, const GHead &gh, int gl, int max_sweeps, double tol2,
                                        double xmax, bool live)
{
    using D = GDim<N>;
    bool need = live;
    for (int sw = 0; sw < max_sweeps; ++sw) {
        double off = 0.0, dia = 0.0;
        for (int u = gl; u < D::NU; u += WG) {
            const double2 b = w.B[u];
            const double v = b.x * b.x + b.y * b.y;
            if (gh.ut[u][0] == gh.ut[u][1]) dia += v;
            else off += 2.0 * v;
        }
        off = grp_sum(off);
        dia = grp_sum(dia);
        need = need && !(off <= tol2 * dia);
        const bool try_fo = need && off <= 1e-10 * dia;
        if (__any_sync(WG_FULL, try_fo)) {
            // X (anti-Hermitian, full) into Tm with unit diagonal; fail flag per group
            double fail = 0.0;
            if (try_fo) {
                for (int u = gl; u < D::NU; u += WG) {
                    const int m = gh.ut[u][0], n = gh.ut[u][1];
                    if (m == n) {
                        w.Tm[m * N + m] = make_double2(1.0, 0.0);
                        continue;
                    }
                    const double d = w.B[pidx(n, n, N)].x - w.B[pidx(m, m, N)].x;
                    const double2 b = w.B[u];
                    const double bb = sqrt(b.x * b.x + b.y * b.y);
                    if (bb == 0.0) {
                        w.Tm[m * N + n] = make_double2(0, 0);
                        w.Tm[n * N + m] = make_double2(0, 0);
                        continue;
                    }
                    if (!(bb <= xmax * fabs(d))) {
                        fail = 1.0;
                        continue;
                    }
                    const double2 x = make_double2(b.x / d, b.y / d);
                    w.Tm[m * N + n] = x;
                    w.Tm[n * N + m] = make_double2(-x.x, x.y);
                }
            }
            fail = grp_max(fail);
            const bool ok = try_fo && fail == 0.0;
            __syncwarp();
            double2 nu[D::NF];
#pragma unroll
            for (int x = 0; x < D::NF; ++x) {
                const int e = gl + WG * x;
                nu[x] = make_double2(0, 0);
                if (!ok || e >= D::NN) continue;
                const int m = e / N, n = e % N;
                double2 a = make_double2(0, 0);
#pragma unroll
                for (int l = 0; l < N; ++l) cfma(a, w.U[m * N + l], w.Tm[l * N + n]);
                nu[x] = a;
            }
            __syncwarp();
#pragma unroll
            for (int x = 0; x < D::NF; ++x) {
                const int e = gl + WG * x;
                if (ok && e < D::NN) w.U[e] = nu[x];
            }
            __syncwarp();
            need = need && !ok;
        }
        if (!__any_sync(WG_FULL, need)) break;
#pragma unroll 1
        for (int r = 0; r < D::P - 1; ++r) g_round<RF, N>(w, gh, r, gl, need);
    }
}

// B = U^dag H0 U (packed) for the groups with `act` (all lanes call it).
// Row m of each product is lane m's (m < N): lane m holds row m of H0 (then
// column m of U) in registers and reads the other factor's element (l, n),
// the same address for every lane of the group, so one shared-memory
// wavefront serves the group's lanes instead of one load per lane and term.
template <class RF, int N>
__device__ __forceinline__ void g_formB(const GView<RF> &w, const GHead &gh, int gl, bool act)
{
    const bool on = act && gl < N;
    if (on) {
        double2 hr[N];
#pragma unroll
        for (int l = 0; l < N; ++l) hr[l] = herm<N>(w.H0, gl, l);
        // the whole row first, then its stores: a store between the loads
        // would keep the compiler from overlapping the rows' chains
        double2 a[N];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            a[n] = make_double2(0, 0);
#pragma unroll
            for (int l = 0; l < N; ++l) cfma(a[n], hr[l], w.U[l * N + n]);
        }
#pragma unroll
        for (int n = 0; n < N; ++n) w.Tm[gl * N + n] = a[n];
    }
    __syncwarp();
    if (on) {
        double2 uc[N], a[N];
#pragma unroll
        for (int l = 0; l < N; ++l) uc[l] = w.U[l * N + gl];
        const int row = pidx(gl, gl, N) - gl;
#pragma unroll
        for (int n = 0; n < N; ++n) {
            a[n] = make_double2(0, 0);
            if (n < gl) continue;
#pragma unroll
            for (int l = 0; l < N; ++l) cfmac(a[n], uc[l], w.Tm[l * N + n]);
        }
#pragma unroll
        for (int n = 0; n < N; ++n) {
            if (n < gl) continue;
            if (n == gl) a[n].y = 0.0;
            w.B[row + n] = a[n];
        }
    }
    __syncwarp();
}

// U <- U (3I - U^dag U) / 2 (one Newton-Schulz step): with U^dag U = I + F
// the result has U^dag U = I + O(F^2), which removes the unitarity defect
// that second-order rotation steps leave (|X|^4 / 4 each).  Rows as in
// g_formB; all lanes call it.
template <class RF, int N>
__device__ __forceinline__ void g_orthonormalize(const GView<RF> &w, int gl)
{
    __syncwarp();
    if (gl < N) {
        double2 uc[N], a[N];
#pragma unroll
        for (int l = 0; l < N; ++l) uc[l] = w.U[l * N + gl];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            a[n] = make_double2(0, 0);
#pragma unroll
            for (int l = 0; l < N; ++l) cfmac(a[n], uc[l], w.U[l * N + n]);
        }
#pragma unroll
        for (int n = 0; n < N; ++n)   // (3I - U^dag U) / 2, row gl
            w.Tm[gl * N + n] = make_double2((n == gl ? 1.5 : 0.0) - 0.5 * a[n].x, -0.5 * a[n].y);
    }
    __syncwarp();
    if (gl < N) {
        double2 ur[N], a[N];
#pragma unroll
        for (int l = 0; l < N; ++l) ur[l] = w.U[gl * N + l];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            a[n] = make_double2(0, 0);
#pragma unroll
            for (int l = 0; l < N; ++l) cfma(a[n], ur[l], w.Tm[l * N + n]);
        }
#pragma unroll
        for (int n = 0; n < N; ++n) w.U[gl * N + n] = a[n];
    }
    __syncwarp();
}

// |offdiag(B)|^2 <= tol2 |diag(B)|^2 of the group's k-point (group-uniform);
// full-mask shuffles: every lane of the warp must call it
template <int N>
__device__ __forceinline__ bool g_diagonal(const double2 *B, const GHead &gh, int gl, double tol2)
{
    using D = GDim<N>;
    double off = 0.0, dia = 0.0;
    for (int u = gl; u < D::NU; u += WG) {
        const double v = B[u].x * B[u].x + B[u].y * B[u].y;
        if (gh.ut[u][0] == gh.ut[u][1]) dia += v;
        else off += 2.0 * v;
    }
    return grp_sum(off) <= tol2 * grp_sum(dia);
}

// One perturbative step of the eigenbasis for the groups with `act`: with
// X_mn = B_mn / (B_nn - B_mm) (m != n; anti-Hermitian, the first-order
// rotation that diagonalises B = U^dag H0 U) and x = max |X_mn|:
//   x <= xfin:  U <- U exp(X) to second order, which finishes the tracking
//               (an O(x^2) error, as g_track's first-order finish) -> 1;
//   x <= 1e-2:  U <- U exp(X) to second order if x^2 <= x2_low, else to
//               fourth (unitary to x^4 / 4 or O(x^6)) -> 2, and B must be
//               formed again;
//   otherwise (or a zero gap): nothing changes -> 3 (Jacobi sweeps needed).
// Lane m (m < N) forms row m of X (scratch matrix) and row m of
// U + UX + (UX)X/2 + ..., reading X by element (the same address for the
// group's lanes).  B is left stale.  Returns 0 for groups
// without `act`.  Group-uniform result; all lanes call it.
template <class RF, int N>
__device__ __forceinline__ int g_pstep(const GView<RF> &w, const GHead &gh, int gl, double xfin, double x2_low,
                                       bool act)
{
    const bool on = act && gl < N;
    double xm2 = 0.0, zero_gap = 0.0;   // max |X_mn|^2
    if (on) {
        const double dm = w.B[pidx(gl, gl, N)].x;
#pragma unroll
        for (int n = 0; n < N; ++n) {
            double2 x = make_double2(0.0, 0.0);
            if (n != gl) {
                const double2 b = herm<N>(w.B, gl, n);
                const double d = w.B[pidx(n, n, N)].x - dm;
                if (d != 0.0) {
                    const double id = 1.0 / d;
                    x = make_double2(b.x * id, b.y * id);
                    xm2 = fmax(xm2, x.x * x.x + x.y * x.y);
                } else if (b.x != 0.0 || b.y != 0.0) {
                    zero_gap = 1.0;
                }
            }
            w.Tm[gl * N + n] = x;
        }
    }
    xm2 = grp_max(xm2);
    zero_gap = grp_max(zero_gap);
    const int st = !act ? 0 : (zero_gap != 0.0 || !(xm2 <= 1e-4)) ? 3 : (xm2 <= xfin * xfin ? 1 : 2);
    const bool go = (st == 1 || st == 2) && gl < N;
    // Taylor order of this group: a finishing step 2, a larger step 2 or 4.
    // With X anti-Hermitian the truncated series E of order 2 has
    // E^dag E = I + X^4 / 4 and of order 4 I + O(X^6): U stays unitary to that,
    // a defect no later rotation removes (orders are even for that reason)
    const int nt = st == 2 && !(xm2 <= x2_low) ? 4 : 2;
    __syncwarp();
    if (go) {
        // row m of U X, then of (U X) X / 2, ...: each term's row is kept in
        // the lane's own row of the scratch matrix and added to row m of U; a
        // row is formed whole before its stores
        double2 *Pb = reinterpret_cast<double2 *>(w.ph) + gl * N;
        double2 *Um = w.U + gl * N;
#pragma unroll 1
        for (int t = 1; t <= nt; ++t) {
            const double c = t == 1 ? 1.0 : t == 2 ? 0.5 : (t == 3 ? 1.0 / 3.0 : 0.25);
            const double2 *src = t == 1 ? Um : Pb;
            double2 qr[N], a[N];
#pragma unroll
            for (int l = 0; l < N; ++l) qr[l] = src[l];
#pragma unroll
            for (int n = 0; n < N; ++n) {
                a[n] = make_double2(0, 0);
#pragma unroll
                for (int l = 0; l < N; ++l) cfma(a[n], qr[l], w.Tm[l * N + n]);
            }
#pragma unroll
            for (int n = 0; n < N; ++n) {
                const double2 q = make_double2(a[n].x * c, a[n].y * c);
                const double2 un = t == 1 ? qr[n] : Um[n];
                Pb[n] = q;
                Um[n] = make_double2(un.x + q.x, un.y + q.y);
            }
        }
    }
    __syncwarp();
    return st;
}

// Eigenbasis tracking by perturbative steps (g_pstep) while B = U^dag H0 U is
// not diagonal to tol2: a larger step forms B again and repeats, a finishing
// step ends it; groups whose rotation is not small (near-
// degenerate bands) or that are not done after three rounds fall back on
// Jacobi sweeps (g_track), which end in the same tolerances.
template <class RF, int N>
__device__ __forceinline__ void g_track_pert(const GView<RF> &w, const GHead &gh, int gl, double tol2, double xmax,
                                             bool live)
{
    bool need = live, rest = false;
#pragma unroll 1
    for (int round = 0; round < 3; ++round) {
        // every lane takes part in the group reduction (full-mask shuffles),
        // whatever its group's state
        const bool diag = g_diagonal<N>(w.B, gh, gl, tol2);
        need = need && !diag;
        if (!__any_sync(WG_FULL, need)) break;
        // second-order steps up to |X| = 1e-3 (unitary to 2.5e-13; the plain
        // method restores unitarity once per attempt) or, in the mixed
        // method, whose tolerance is looser, up to 1e-2; fourth order above
        const int st = g_pstep<RF, N>(w, gh, gl, xmax, std::is_same<RF, float>::value ? 1e-4 : SBE_WG_X2_LOW, need);
        rest = rest || st == 3;
        need = st == 2;
        if (!__any_sync(WG_FULL, need)) break;
        g_formB<RF, N>(w, gh, gl, need);
    }
    rest = rest || need;
    if (__any_sync(WG_FULL, rest)) g_track<RF, N>(w, gh, gl, 6, tol2, xmax, rest);
}

// Table loads through the read-only path with the L1 eviction priority
// evict_last: the re-laid tables (about 44 KB in FP64 at N = 6, 37 vectors)
// are read by every stage of every k-point and should stay in the L1 that
// the blocks' shared memory leaves, while the per-k state streams past it
// (loaded and stored at the L2 only).
__device__ __forceinline__ double2 g_ldtab(const double2 *p)
{
    double2 v;
    asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float2 g_ldtab(const float2 *p)
{
    float2 v;
    asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}

// Fourier sums of the lane's owned upper elements over the lattice-vector
// pairs: quantity q (h, d_x, d_y; Q of them) accumulates c sig + s tau per
// pair, e^{iKR} = c + i s; with CUR also S_a = sum R_a h_R e^{iKR}, whose pair
// term is R_a (h_R e^{iKR} - h_-R e^{-iKR}) = R_a (c (-i tau) + s (i sig)).
// All accumulator chains of a pair are independent, so the loads of one pair
// and the multiply-adds of the previous one overlap.
template <class RF, int N, int Q, bool CUR>
__device__ __forceinline__ void g_fourier(const typename Cx<RF>::T *tb, int gstride, const typename Cx<RF>::T *ph,
                                          const RF *Rp, int np, typename Cx<RF>::T (&a)[3][GDim<N>::NO],
                                          typename Cx<RF>::T (&sx)[GDim<N>::NO], typename Cx<RF>::T (&sy)[GDim<N>::NO])
{
    using TF = typename Cx<RF>::T;
    constexpr int NO = GDim<N>::NO;
#pragma unroll 1
    for (int p = 0; p < np; ++p) {
        const TF e = ph[p];
        const TF *tr = tb + (size_t)p * gstride;
        RF rx = RF(0), ry = RF(0);
        if (CUR) {
            rx = Rp[2 * p];
            ry = Rp[2 * p + 1];
        }
#pragma unroll
        for (int j = 0; j < NO; ++j) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const TF sg = g_ldtab(tr + (j * 3 + q) * 2 * WG), ta = g_ldtab(tr + ((j * 3 + q) * 2 + 1) * WG);
                a[q][j].x = fma(e.x, sg.x, fma(e.y, ta.x, a[q][j].x));
                a[q][j].y = fma(e.x, sg.y, fma(e.y, ta.y, a[q][j].y));
                if (CUR && q == 0) {
                    const RF ox = fma(e.x, ta.y, -e.y * sg.y), oy = fma(e.y, sg.x, -e.x * ta.x);
                    sx[j].x = fma(rx, ox, sx[j].x);
                    sx[j].y = fma(rx, oy, sx[j].y);
                    sy[j].x = fma(ry, ox, sy[j].x);
                    sy[j].y = fma(ry, oy, sy[j].y);
                }
            }
        }
    }
}

// The same sums for H0 and E.D at a stage without currents: the second from
// the stage's table of E_x d_x + E_y d_y (tT, [pair][j][half][lane]), so D_x
// and D_y need no sums of their own.  (A table of h + E.D would give H0 + E.D
// directly, but in the mixed method its single-precision rounding of h, not
// of E.D, would then drive the field term: 3x the spectral error.)
template <class RF, int N>
__device__ __forceinline__ void g_fourier_ht(const typename Cx<RF>::T *tb, int gstride, const typename Cx<RF>::T *tT,
                                             const typename Cx<RF>::T *ph, int np,
                                             typename Cx<RF>::T (&a)[3][GDim<N>::NO])
{
    using TF = typename Cx<RF>::T;
    constexpr int NO = GDim<N>::NO;
#pragma unroll 1
    for (int p = 0; p < np; ++p) {
        const TF e = ph[p];
        const TF *tr = tb + (size_t)p * gstride, *ts = tT + (size_t)p * NO * 2 * WG;
#pragma unroll
        for (int j = 0; j < NO; ++j) {
            const TF sg = g_ldtab(tr + j * 3 * 2 * WG), ta = g_ldtab(tr + (j * 3 * 2 + 1) * WG);
            const TF sT = g_ldtab(ts + j * 2 * WG), tT2 = g_ldtab(ts + (j * 2 + 1) * WG);
            a[0][j].x = fma(e.x, sg.x, fma(e.y, ta.x, a[0][j].x));
            a[0][j].y = fma(e.x, sg.y, fma(e.y, ta.y, a[0][j].y));
            a[1][j].x = fma(e.x, sT.x, fma(e.y, tT2.x, a[1][j].x));
            a[1][j].y = fma(e.x, sT.y, fma(e.y, tT2.y, a[1][j].y));
        }
    }
}

template <class RF, int N, int RK>
__global__ void __launch_bounds__(32 * WG_WARPS, SBE_WG_MINB)
    wan_attempt_g(const WanDev *__restrict__ Pp, const WanDev *const *__restrict__ descs,
                  const WanTileRef *__restrict__ tiles)
{
    using TF = typename Cx<RF>::T;
    using T = double2;
    using D = GDim<N>;
    constexpr bool F32 = std::is_same<RF, float>::value;
    constexpr int S = RK == 4 ? 4 : 6;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // a single solve (block b = tiles WG_WARPS b ...) or a block tile of a batch
    const int tile0 = tiles ? tiles[blockIdx.x].tile : (int)blockIdx.x * WG_WARPS;
    const WanDev &P = tiles ? *descs[tiles[blockIdx.x].solve] : *Pp;
    const WanCtl ctl = *P.ctl;
    if (ctl.done) return;
    const int nR = P.nR;
    const GSmem L = g_smem(N, nR, sizeof(RF));
    GHead &gh = *reinterpret_cast<GHead *>(smem_raw);
    TF *cA = reinterpret_cast<TF *>(smem_raw + L.cA);
    RF *Rc = reinterpret_cast<RF *>(smem_raw + L.Rc);
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, grp = lane >> 3, gl = lane & 7;
    const double h = ctl.hs;
    const int buf = ctl.buf;
    const bool cur = ctl.need_current;
    if (threadIdx.x == 0) {
        tableau(P.rk, gh.tab);
        int u = 0;
        for (int m = 0; m < N; ++m)
            for (int n = m; n < N; ++n, ++u) {
                gh.ut[u][0] = (unsigned char)m;
                gh.ut[u][1] = (unsigned char)n;
            }
        for (int r = 0; r < D::P - 1; ++r)
            for (int i = 0; i < N; ++i) gh.mate[r][i] = (signed char)rr_mate(i, r, D::P);
    }
    const int np = P.npair;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        const int r = P.gpair[i];
        gh.gp[i] = r;
        Rc[2 * i] = RF(P.V[2 * r]);
        Rc[2 * i + 1] = RF(P.V[2 * r + 1]);
    }
    const TF *cAg = static_cast<const TF *>(P.stage_cA);
    for (int i = threadIdx.x; i < S * nR; i += blockDim.x) cA[i] = cAg[i];
    for (int i = threadIdx.x; i < 36; i += blockDim.x) gh.AE[i / 6][i % 6] = P.stage_AE[i];
    for (int q = threadIdx.x; q < WG_WARPS * WAN_WARPS * WAN_NSLOT; q += blockDim.x)
        (&gh.part[0][0][0])[q] = 0.0;
    if (threadIdx.x < WG_WARPS) gh.errw[threadIdx.x] = 0.0;
    __syncthreads();

    const int tile = tile0 + wi;
    if (tile < P.ntiles) {
        const int k = tile * WAN_WARPS + grp;
        const bool live = k < P.nk;
        const int kc = live ? k : P.nk - 1;   // a group past the grid shadows the last k-point
        const GView<RF> w(smem_raw + L.k0 + (size_t)(wi * WAN_WARPS + grp) * L.kbytes, L);
        double kv[3], wk;
        kpoint(P, kc, kv, wk);
        for (int q = gl; q < np; q += WG) {
            const int r = gh.gp[q];
            double sn, cs;
            sincos(kv[0] * P.V[2 * r] + kv[1] * P.V[2 * r + 1], &sn, &cs);
            w.pk[q] = cx<TF>(cs, sn);
        }
        const T *Ug = P.U[buf] + (size_t)kc * D::NN;
        for (int e = gl; e < D::NN; e += WG) w.U[e] = __ldcg(Ug + e);
        if (!F32 && SBE_WG_X2_LOW > 0.0) g_orthonormalize<RF, N>(w, gl);
        const double2 *rho = P.rho[buf] + (size_t)kc * D::NN;
        T r64[D::NO];
        // row and column of the owned upper element j (read from the block's
        // table when needed rather than held in registers)
        auto om = [&](int j) { return (int)gh.ut[min(gl + WG * j, D::NU - 1)][0]; };
        auto on = [&](int j) { return (int)gh.ut[min(gl + WG * j, D::NU - 1)][1]; };
#pragma unroll
        for (int j = 0; j < D::NO; ++j) {
            const int u = gl + WG * j;
            r64[j] = make_double2(0, 0);
            if (u < D::NU) r64[j] = __ldcg(rho + om(j) * N + on(j));
        }
        T ks[S][D::NO];
        const TF *gt = static_cast<const TF *>(P.gtab);
        const int gstride = D::NO * 3 * 2 * WG;   // table entries per lattice-vector pair
        const bool dip = P.has_dip;
        double emax = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            // stage input Y = rho + h sum_j a_sj k_j (owned elements, packed)
#pragma unroll
            for (int j = 0; j < D::NO; ++j) {
                const int u = gl + WG * j;
                if (u >= D::NU) continue;
                T y = r64[j];
#pragma unroll
                for (int i = 0; i < s; ++i) {
                    const double a = h * gh.tab.a[s][i];
                    if (a != 0.0) {
                        y.x = fma(a, ks[i][j].x, y.x);
                        y.y = fma(a, ks[i][j].y, y.y);
                    }
                }
                if (om(j) == on(j)) y.y = 0;
                w.Y[u] = y;
            }
            for (int q = gl; q < np; q += WG) w.ph[q] = cmul(w.pk[q], cA[s * nR + gh.gp[q]]);
            __syncwarp();
            const bool with_cur = cur && s == 0;
            // Fourier sums of the owned elements: H0, D_x, D_y (and S_x, S_y)
            const double Ex = gh.AE[s][3], Ey = gh.AE[s][4];
            T d0[D::NO], d1[D::NO], s0[D::NO], s1[D::NO];
            {
                TF a[3][D::NO], sx[D::NO], sy[D::NO];
#pragma unroll
                for (int j = 0; j < D::NO; ++j) a[0][j] = a[1][j] = a[2][j] = sx[j] = sy[j] = cx<TF>(0, 0);
                const TF *tb = gt + gl;
                // E.D from the stage's combined table where the currents need
                // no D_a (dipole models)
                const bool ht = !with_cur && dip && P.stage_gt != nullptr;
                if (with_cur) g_fourier<RF, N, 3, true>(tb, gstride, w.ph, Rc, np, a, sx, sy);
                else if (ht) {
                    const TF *tT = static_cast<const TF *>(P.stage_gt) + (size_t)s * np * D::NO * 2 * WG + gl;
                    g_fourier_ht<RF, N>(tb, gstride, tT, w.ph, np, a);
                } else if (dip) g_fourier<RF, N, 3, false>(tb, gstride, w.ph, Rc, np, a, sx, sy);
                else g_fourier<RF, N, 1, false>(tb, gstride, w.ph, Rc, np, a, sx, sy);
#pragma unroll
                for (int j = 0; j < D::NO; ++j) {
                    const int u = gl + WG * j;
                    const T v0 = make_double2(a[0][j].x, a[0][j].y), v1 = make_double2(a[1][j].x, a[1][j].y),
                            v2 = make_double2(a[2][j].x, a[2][j].y);
                    d0[j] = v1;
                    d1[j] = v2;
                    s0[j] = make_double2(sx[j].x, sx[j].y);
                    s1[j] = make_double2(sy[j].x, sy[j].y);
                    if (u >= D::NU) continue;
                    w.H0[u] = v0;
                    w.HT[u] = ht ? make_double2(v0.x + v1.x, v0.y + v1.y)
                                 : make_double2(fma(Ex, v1.x, fma(Ey, v2.x, v0.x)), fma(Ex, v1.y, fma(Ey, v2.y, v0.y)));
                }
            }
            __syncwarp();
            // total current at the output step: computed before the tracking,
            // which needs no D_a, so D_a leaves the registers early
            double tot[2] = {0.0, 0.0};
            if (with_cur) {
                // total: Re Tr(Y J_a), J_a = -i S_a + i [D_a, H0], over the owned
                // upper elements: diagonal Y_mm Im(S_mm) - Im(C_mm) Re(D_mm),
                // off-diagonal -2 Im(Y_mn conj(S_mn)) - 2 Im(C_mn conj(D_mn)),
                // C = [H0, Y] = H0 Y - (H0 Y)^dag; lane m forms row m of H0 Y
                if (gl < N) {
                    T hr[N];
#pragma unroll
                    for (int l = 0; l < N; ++l) hr[l] = herm<N>(w.H0, gl, l);
                    T a[N];
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        a[n] = make_double2(0, 0);
#pragma unroll
                        for (int l = 0; l < N; ++l) cfma(a[n], hr[l], herm<N>(w.Y, l, n));
                    }
#pragma unroll
                    for (int n = 0; n < N; ++n) w.Tm[gl * N + n] = a[n];
                }
                __syncwarp();
#pragma unroll
                for (int j = 0; j < D::NO; ++j) {
                    const int u = gl + WG * j;
                    if (u >= D::NU) continue;
                    const int m = om(j), n = on(j);
                    const T c1 = w.Tm[m * N + n], c2 = w.Tm[n * N + m];
                    const T c = make_double2(c1.x - c2.x, c1.y + c2.y);
                    const T y = w.Y[u];
#pragma unroll
                    for (int a = 0; a < 2; ++a) {
                        const T sv = a == 0 ? s0[j] : s1[j];
                        const T dd = a == 0 ? d0[j] : d1[j];
                        if (m == n) {
                            tot[a] += y.x * sv.y - c.y * dd.x;
                        } else {
                            // Im(z conj(w)) = z.y w.x - z.x w.y
                            tot[a] -= 2.0 * (y.y * sv.x - y.x * sv.y) + 2.0 * (c.y * dd.x - c.x * dd.y);
                        }
                    }
                }
                __syncwarp();
            }
            // B = U^dag H0 U
            g_formB<RF, N>(w, gh, gl, true);
            // eigenbasis tracking (tolerances as wan_attempt)
            g_track_pert<RF, N>(w, gh, gl, F32 ? 1e-20 : 1e-30, F32 ? 1e-5 : 1e-7, live);
            if (gh.tab.c[s] == 1.0 && live) {
                T *Uo = P.U[1 - buf] + (size_t)kc * D::NN;
                for (int e = gl; e < D::NN; e += WG) __stcg(Uo + e, w.U[e]);
            }
            // dv = diag(U^dag Y U) and, at an output step, the intraband
            // current sum_n Re[dv_n (U^dag (-i S_a) U)_nn]: lane n holds column n
            // of U and reads Y (S_a) by element, the same address for the
            // group's lanes.  S_x goes packed into the phase buffer and S_y into
            // B, both free after the tracking.
            if (with_cur) {
#pragma unroll
                for (int j = 0; j < D::NO; ++j) {
                    const int u = gl + WG * j;
                    if (u < D::NU) {
                        reinterpret_cast<T *>(w.ph)[u] = s0[j];
                        w.B[u] = s1[j];
                    }
                }
                __syncwarp();
            }
            double intra[2] = {0.0, 0.0};
            if (gl < N) {
                T uc[N];
#pragma unroll
                for (int l = 0; l < N; ++l) uc[l] = w.U[l * N + gl];
                T dvn = make_double2(0, 0);
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    T t = make_double2(0, 0);
#pragma unroll
                    for (int p = 0; p < N; ++p) cfma(t, herm<N>(w.Y, l, p), uc[p]);
                    cfmac(dvn, uc[l], t);
                }
                w.dv[gl] = dvn;
                if (with_cur) {
#pragma unroll
                    for (int a = 0; a < 2; ++a) {
                        const T *Sa = a == 0 ? reinterpret_cast<const T *>(w.ph) : w.B;
                        T pn = make_double2(0, 0);
#pragma unroll
                        for (int l = 0; l < N; ++l) {
                            T q = make_double2(0, 0);   // (S U)_ln
#pragma unroll
                            for (int p = 0; p < N; ++p) cfma(q, aherm<N>(Sa, l, p), uc[p]);
                            cfmac(pn, uc[l], q);
                        }
                        // Re[dv_n (-i pn)]
                        intra[a] = dvn.x * pn.y + dvn.y * pn.x;
                    }
                }
            }
            __syncwarp();
            if (with_cur) {
                double *val = gh.part[wi][grp];
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const double tt = grp_sum(tot[a]), ii = grp_sum(intra[a]);
                    if (gl == 0 && live) {
                        val[a] = wk * (tt - ii);
                        val[2 + a] = wk * ii;
                    }
                }
                if (gl < N && live) val[4 + gl] = wk * w.Y[pidx(gl, gl, N)].x;
                const int ce = (P.nval * N + P.nval + 1) % D::NN;   // antelope.cpp:539-542
                if (gl == 0 && live) {
                    const T yc = herm<N>(w.Y, ce / N, ce % N);
                    val[4 + N] = wk * yc.x;
                    val[5 + N] = wk * yc.y;
                }
                __syncwarp();
            }
            // right-hand side of the owned elements: -i((HY) - (HY)^dag)
            // - (g2 Y + (g1 - g2) U diag(dv) U^dag)   (SBEs.h:808-861).  Lane m
            // forms row m of HY (scratch matrix) and of U diag(dv) U^dag (phase
            // buffer, free after the currents) with the second factor read by
            // element; then each lane combines its owned elements.
            const double g1 = P.g1, g2 = P.g2;
            const bool deph = g1 != 0.0 || g2 != 0.0;
            T *Pr = reinterpret_cast<T *>(w.ph);
            if (gl < N) {
                T hr[N];
#pragma unroll
                for (int l = 0; l < N; ++l) hr[l] = herm<N>(w.HT, gl, l);
                T a[N];
#pragma unroll
                for (int n = 0; n < N; ++n) {
                    a[n] = make_double2(0, 0);
#pragma unroll
                    for (int l = 0; l < N; ++l) cfma(a[n], hr[l], herm<N>(w.Y, l, n));
                }
#pragma unroll
                for (int n = 0; n < N; ++n) w.Tm[gl * N + n] = a[n];
                if (deph) {
#pragma unroll
                    for (int p = 0; p < N; ++p) hr[p] = cmul(w.U[gl * N + p], w.dv[p]);
#pragma unroll
                    for (int n = 0; n < N; ++n) {
                        a[n] = make_double2(0, 0);
#pragma unroll
                        for (int p = 0; p < N; ++p) cfma(a[n], hr[p], cconj(w.U[n * N + p]));
                    }
#pragma unroll
                    for (int n = 0; n < N; ++n) Pr[gl * N + n] = a[n];
                }
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < D::NO; ++j) {
                const int u = gl + WG * j;
                if (u >= D::NU) continue;
                const int m = om(j), n = on(j);
                const T c = w.Tm[m * N + n], c2 = w.Tm[n * N + m];
                T kv2 = make_double2(c.y + c2.y, -(c.x - c2.x));
                if (deph) {
                    const T pr = Pr[m * N + n], y = w.Y[u];
                    kv2.x -= g2 * y.x + (g1 - g2) * pr.x;
                    kv2.y -= g2 * y.y + (g1 - g2) * pr.y;
                }
                ks[s][j] = kv2;
            }
            __syncwarp();
        }
        // trial state and error estimate
        double2 *rout = P.rho[1 - buf] + (size_t)kc * D::NN;
#pragma unroll
        for (int j = 0; j < D::NO; ++j) {
            const int u = gl + WG * j;
            if (u >= D::NU) continue;
            T inc = make_double2(0, 0), er = make_double2(0, 0);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double b = h * gh.tab.b[s];
                if (b != 0.0) {
                    inc.x = fma(b, ks[s][j].x, inc.x);
                    inc.y = fma(b, ks[s][j].y, inc.y);
                }
                const double eb = h * gh.tab.e[s];
                if (eb != 0.0) {
                    er.x = fma(eb, ks[s][j].x, er.x);
                    er.y = fma(eb, ks[s][j].y, er.y);
                }
            }
            double2 v = make_double2(r64[j].x + inc.x, r64[j].y + inc.y);
            const int m = om(j), n = on(j);
            if (m == n) v.y = 0.0;
            if (live) {
                __stcg(rout + m * N + n, v);
                __stcg(rout + n * N + m, make_double2(v.x, -v.y));
                emax = fmax(emax, sqrt(er.x * er.x + er.y * er.y));
            }
        }
        emax = warp_max(emax);
        if (lane == 0) gh.errw[wi] = emax;
    }
    __syncthreads();
    if (threadIdx.x < WG_WARPS) {
        const int t = tile0 + threadIdx.x;
        if (t < P.ntiles) P.tile_err[t] = gh.errw[threadIdx.x];
    }
    if (cur && threadIdx.x < WG_WARPS * WAN_NSLOT) {
        const int wq = threadIdx.x / WAN_NSLOT, slot = threadIdx.x % WAN_NSLOT, t = tile0 + wq;
        if (t < P.ntiles) {
            double s = 0.0;
            for (int g = 0; g < WAN_WARPS; ++g) s += gh.part[wq][g][slot];
            P.cur_part[(size_t)t * WAN_NSLOT + slot] = s;
        }
    }
}
