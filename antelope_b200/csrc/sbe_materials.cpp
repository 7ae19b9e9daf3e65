// The reference's analytic tight-binding materials (src/GeneralModel/Materials)
// restated as Fourier tables: H(k) = sum_v h_v e^{ik.v} and the current
// operator the material's GenJMatrix returns, J_a(k) = sum_v j_{a,v} e^{ik.v},
// over a small set of Cartesian vectors v.  Every cos / sin / exp term of the
// reference's formulas becomes one or two table entries, so the tables
// reproduce its H and J -- including where its J is not -dH/dk (noted per
// material) -- and the N-band length- and velocity-gauge kernels run them
// unchanged.  Parameter keys, defaults, unit conversions, Brillouin-zone axes
// and error texts follow each material's constructor.
#include <array>
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "sbe_problem.h"

namespace sbe {

namespace {

using cplx = std::complex<double>;
const cplx I1(0.0, 1.0);

// Accumulates table entries on a set of vectors (entries on the same vector
// are merged; vectors are compared with a relative tolerance of 1e-12).
struct TBBuilder {
    int N;
    std::vector<std::array<double, 2>> v;
    std::vector<cplx> h, j;  // [nv][N*N], [nv][2][N*N]
    explicit TBBuilder(int n) : N(n) {}

    int vec(double x, double y)
    {
        for (size_t i = 0; i < v.size(); ++i) {
            const double s = 1e-12 * (1.0 + std::fabs(x) + std::fabs(y));
            if (std::fabs(v[i][0] - x) <= s && std::fabs(v[i][1] - y) <= s) return (int)i;
        }
        v.push_back({x, y});
        h.resize(v.size() * N * N);
        j.resize(v.size() * 2 * N * N);
        return (int)v.size() - 1;
    }
    // c e^{ik.v} into H(m, n), or into J_a(m, n) for a = 0, 1
    void exp_(int a, int m, int n, double vx, double vy, cplx c)
    {
        if (c == cplx(0.0)) return;
        const int r = vec(vx, vy);
        if (a < 0) h[(size_t)r * N * N + m * N + n] += c;
        else j[((size_t)r * 2 + a) * N * N + m * N + n] += c;
    }
    // c cos(k.v) and c sin(k.v) as two exponentials
    void cos_(int a, int m, int n, double vx, double vy, cplx c)
    {
        exp_(a, m, n, vx, vy, 0.5 * c);
        exp_(a, m, n, -vx, -vy, 0.5 * c);
    }
    void sin_(int a, int m, int n, double vx, double vy, cplx c)
    {
        exp_(a, m, n, vx, vy, -0.5 * I1 * c);
        exp_(a, m, n, -vx, -vy, 0.5 * I1 * c);
    }
    void const_(int a, int m, int n, cplx c) { exp_(a, m, n, 0.0, 0.0, c); }

    void to_problem(Problem &p) const
    {
        p.nband = N;
        p.w_nR = (int)v.size();
        p.w_vec.resize(2 * v.size());
        for (size_t i = 0; i < v.size(); ++i) {
            p.w_vec[2 * i] = v[i][0];
            p.w_vec[2 * i + 1] = v[i][1];
        }
        p.w_h.resize(2 * h.size());
        for (size_t i = 0; i < h.size(); ++i) {
            p.w_h[2 * i] = h[i].real();
            p.w_h[2 * i + 1] = h[i].imag();
        }
        p.w_j.resize(2 * j.size());
        for (size_t i = 0; i < j.size(); ++i) {
            p.w_j[2 * i] = j[i].real();
            p.w_j[2 * i + 1] = j[i].imag();
        }
        p.w_d.clear();
    }
};

void set_bz(Problem &p, double kxMax, double kyMax)
{
    const double axes[9] = {2 * kxMax, 0, 0, 0, 2 * kyMax, 0, 0, 0, 0};
    for (int i = 0; i < 9; ++i) p.bzaxes[i] = axes[i];
    for (int i = 0; i < 3; ++i) p.bzorigin[i] = 0.0;
}

// Honeycomb nearest- and next-nearest-neighbour vectors (SetBasis of
// Haldane.h:134-143, KaneMele.h, Haldane2L.h)
void honeycomb(double a, double va[3][2], double vb[3][2])
{
    const double r3 = std::sqrt(3.);
    const double A[3][2] = {{0., a}, {-r3 / 2 * a, -0.5 * a}, {r3 / 2 * a, -0.5 * a}};
    const double B[3][2] = {{r3 * a, 0.}, {-r3 / 2 * a, 3. / 2. * a}, {-r3 / 2 * a, -3. / 2. * a}};
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 2; ++c) {
            va[i][c] = A[i][c];
            vb[i][c] = B[i][c];
        }
}

// One Haldane block on rows/columns (o, o+1) of H:
//   B0 = 2 t2 cos(phi) sum cos(k.b), B1 = t1 sum cos(k.a), B2 = t1 sum sin(k.a),
//   B3 = M0 - f3 sum sin(k.b)  with f3 = 2 t2 sin(phi) (GenBcomp),
//   H = [[B0 + B3, B1 - s i B2], [B1 + s i B2, B0 - B3]]   (s = B2 sign).
// b3const / b3sin allow the Haldane2L bottom-layer form of B3.
void haldane_block_h(TBBuilder &tb, int o, double va[3][2], double vb[3][2], double t1, double c0, double b3const,
                     double b3sin, double s)
{
    for (int i = 0; i < 3; ++i) {
        const double *a = va[i], *b = vb[i];
        // B0 on both diagonal entries
        tb.cos_(-1, o, o, b[0], b[1], c0);
        tb.cos_(-1, o + 1, o + 1, b[0], b[1], c0);
        // +/- B3 (sin part)
        tb.sin_(-1, o, o, b[0], b[1], -b3sin);
        tb.sin_(-1, o + 1, o + 1, b[0], b[1], b3sin);
        // B1 -/+ s i B2
        tb.cos_(-1, o, o + 1, a[0], a[1], t1);
        tb.sin_(-1, o, o + 1, a[0], a[1], -s * I1 * t1);
        tb.cos_(-1, o + 1, o, a[0], a[1], t1);
        tb.sin_(-1, o + 1, o, a[0], a[1], s * I1 * t1);
    }
    tb.const_(-1, o, o, b3const);
    tb.const_(-1, o + 1, o + 1, -b3const);
}

// -d/dk of that block (GenJMatrix of Haldane.h:94-127 and the layered forms):
//   xder0 = -c0 sum b_x sin(k.b), xder1 = -t1 sum a_x sin(k.a),
//   xder2 = t1 sum a_x cos(k.a),  xder3 = -f3 sum b_x cos(k.b),
//   J = -[[x0 + x3, x1 - s i x2], [x1 + s i x2, x0 - x3]]
// (sw swaps the roles of +x3 / -x3 on the diagonal: Kane-Mele's lower block).
void haldane_block_j(TBBuilder &tb, int o, double va[3][2], double vb[3][2], double t1, double c0, double f3,
                     double s, bool sw)
{
    for (int ax = 0; ax < 2; ++ax)
        for (int i = 0; i < 3; ++i) {
            const double *a = va[i], *b = vb[i];
            // x0 = -c0 b sin(k.b): -x0 on both diagonal entries
            tb.sin_(ax, o, o, b[0], b[1], c0 * b[ax]);
            tb.sin_(ax, o + 1, o + 1, b[0], b[1], c0 * b[ax]);
            // x3 = -f3 b cos(k.b): -x3 on (o,o), +x3 on (o+1,o+1) (swapped when sw)
            const double d3 = sw ? -1.0 : 1.0;
            tb.cos_(ax, o, o, b[0], b[1], d3 * f3 * b[ax]);
            tb.cos_(ax, o + 1, o + 1, b[0], b[1], -d3 * f3 * b[ax]);
            // x1 = -t1 a sin(k.a), x2 = t1 a cos(k.a): -(x1 -/+ s i x2)
            tb.sin_(ax, o, o + 1, a[0], a[1], t1 * a[ax]);
            tb.cos_(ax, o, o + 1, a[0], a[1], s * I1 * t1 * a[ax]);
            tb.sin_(ax, o + 1, o, a[0], a[1], t1 * a[ax]);
            tb.cos_(ax, o + 1, o, a[0], a[1], -s * I1 * t1 * a[ax]);
        }
}

// ------------------------------------------------------------ WilsonMass
// WilsonMass.h: 2 bands, B1 = delta sin(a0 kx), B2 = delta sin(a1 ky),
// B3 = -2t (cos(a0 kx) + cos(a1 ky)) - mu; J = -dH/dk.  Lengths in bohr.
void wilson_mass(const CfgValue *mat, Problem &p)
{
    double t, delta, mu, a0, a1;
    if (!(mat && get_double(mat, "t", t) && get_double(mat, "delta", delta) && get_double(mat, "mu", mu) &&
          get_double(mat, "a0", a0)))
        throw CfgError("Some Haldane paramters are missing");  // the reference's text
    if (!get_double(mat, "a1", a1)) a1 = a0;
    TBBuilder tb(2);
    // H = [[B3, B1 - i B2], [B1 + i B2, -B3]]
    tb.cos_(-1, 0, 0, a0, 0, -2 * t);
    tb.cos_(-1, 0, 0, 0, a1, -2 * t);
    tb.const_(-1, 0, 0, -mu);
    tb.cos_(-1, 1, 1, a0, 0, 2 * t);
    tb.cos_(-1, 1, 1, 0, a1, 2 * t);
    tb.const_(-1, 1, 1, mu);
    tb.sin_(-1, 0, 1, a0, 0, delta);
    tb.sin_(-1, 0, 1, 0, a1, -I1 * delta);
    tb.sin_(-1, 1, 0, a0, 0, delta);
    tb.sin_(-1, 1, 0, 0, a1, I1 * delta);
    // J (WilsonMass.h GenJMatrix): x: [-2t a0 s, -a0 d c; -a0 d c, 2t a0 s] with s, c of a0 kx
    tb.sin_(0, 0, 0, a0, 0, -2 * t * a0);
    tb.sin_(0, 1, 1, a0, 0, 2 * t * a0);
    tb.cos_(0, 0, 1, a0, 0, -a0 * delta);
    tb.cos_(0, 1, 0, a0, 0, -a0 * delta);
    tb.sin_(1, 0, 0, 0, a1, -2 * t * a1);
    tb.sin_(1, 1, 1, 0, a1, 2 * t * a1);
    tb.cos_(1, 0, 1, 0, a1, I1 * a1 * delta);
    tb.cos_(1, 1, 0, 0, a1, -I1 * a1 * delta);
    tb.to_problem(p);
    p.nval = 1;
    set_bz(p, PI / a0, PI / a1);
}

// ------------------------------------------------------------ KaneMele
// KaneMele.h: two Haldane blocks with phi0 and -phi0 and a Rashba coupling
// between them.  Reference specifics kept: J's Rashba entries are +dH/dk
// (the Haldane blocks are -dH/dk), and its (3,0) entry is not multiplied by
// i tR (the scaling loop stops at index 2).
void kane_mele(const CfgValue *mat, Problem &p)
{
    double t1, t2, tR, M0, phi0, a0;
    if (!(mat && get_double(mat, "t1", t1) && get_double(mat, "t2", t2) && get_double(mat, "tR", tR) &&
          get_double(mat, "Mt2", M0) && get_double(mat, "phi0", phi0) && get_double(mat, "a0", a0)))
        throw CfgError("Some KaneMele paramters are missing");
    a0 /= AU_ANGSTROM;
    M0 *= t2;
    double va[3][2], vb[3][2];
    honeycomb(a0, va, vb);
    const double cR[3][2] = {{1., 0.}, {-0.5, std::sqrt(3.) / 2}, {-0.5, -std::sqrt(3.) / 2}};
    TBBuilder tb(4);
    // upper block: phi0; lower block: -phi0 (cos unchanged, sin flips)
    haldane_block_h(tb, 0, va, vb, t1, 2. * t2 * std::cos(phi0), M0, 2. * t2 * std::sin(phi0), 1.0);
    haldane_block_h(tb, 2, va, vb, t1, 2. * t2 * std::cos(-phi0), M0, 2. * t2 * std::sin(-phi0), 1.0);
    // the reference's lower-block J takes the upper block's derivatives with
    // x3 swapped between the diagonal entries (KaneMele.h GenJMatrix)
    haldane_block_j(tb, 0, va, vb, t1, 2. * t2 * std::cos(phi0), 2. * t2 * std::sin(phi0), 1.0, false);
    haldane_block_j(tb, 2, va, vb, t1, 2. * t2 * std::cos(phi0), 2. * t2 * std::sin(phi0), 1.0, true);
    for (int i = 0; i < 3; ++i) {
        const double *a = va[i];
        const cplx cm(cR[i][0], -cR[i][1]), cp(cR[i][0], cR[i][1]);
        // H(0,3) = i tR sum cm e^{ik.a}, H(1,2) = i tR sum cm e^{-ik.a},
        // H(2,1) = conj(H(1,2)), H(3,0) = conj(H(0,3))
        tb.exp_(-1, 0, 3, a[0], a[1], I1 * tR * cm);
        tb.exp_(-1, 1, 2, -a[0], -a[1], I1 * tR * cm);
        tb.exp_(-1, 2, 1, a[0], a[1], -I1 * tR * cp);
        tb.exp_(-1, 3, 0, -a[0], -a[1], -I1 * tR * cp);
        for (int ax = 0; ax < 2; ++ax) {
            tb.exp_(ax, 0, 3, a[0], a[1], I1 * tR * cm * (I1 * a[ax]));
            tb.exp_(ax, 1, 2, -a[0], -a[1], I1 * tR * cm * (-I1 * a[ax]));
            tb.exp_(ax, 2, 1, a[0], a[1], I1 * tR * (-cp) * (I1 * a[ax]));
            tb.exp_(ax, 3, 0, -a[0], -a[1], (-cp) * (-I1 * a[ax]));
        }
    }
    tb.to_problem(p);
    p.nval = 2;
    set_bz(p, PI / std::sqrt(3.) / a0, 2. * PI / 3. / a0);
}

// ------------------------------------------------------------ Haldane2L
// Haldane2L.h: two Haldane layers (4 bands) with a stacking-dependent
// interlayer hopping t11.  Reference specifics kept: the bottom-layer
// parameters t1_bottom / t2_bottom / phi0_bottom are read with a
// short-circuiting OR (after the first one found, the others keep the top
// values); with distinct layers, the bottom B3 is M0_b - 2 t2_b sin(phi0_b)
// times the top layer's B3 (not its own sine sum) while J uses the bottom
// layer's own derivatives.
void haldane_2l(const CfgValue *mat, Problem &p)
{
    double t1[2], t2[2], phi0[2], M0[2], a0, t11;
    std::string polytype;
    if (!(mat && get_double(mat, "t1", t1[0]) && get_double(mat, "t2", t2[0]) &&
          get_double(mat, "phi0", phi0[0]) && get_double(mat, "a0", a0) && get_double(mat, "t11", t11) &&
          get_string(mat, "polytype", polytype)))
        throw CfgError("Some Haldane2L paramters are missing");
    a0 /= AU_ANGSTROM;
    if (!get_double(mat, "M0", M0[0])) {
        if (get_double(mat, "Mt2", M0[0])) M0[0] *= t2[0];
        else throw CfgError("M0 param missing");
    }
    bool same = true;
    t1[1] = t1[0];
    t2[1] = t2[0];
    phi0[1] = phi0[0];
    M0[1] = M0[0];
    if (get_double(mat, "t1_bottom", t1[1]) || get_double(mat, "t2_bottom", t2[1]) ||
        get_double(mat, "phi0_bottom", phi0[1]))
        same = false;
    if (get_double(mat, "M0_bottom", M0[1])) {
        same = false;
    } else if (get_double(mat, "Mt2_bottom", M0[1])) {
        M0[1] *= t2[1];
        same = false;
    }
    double B2sign[2] = {1., 1.}, hi[4] = {0, 0, 0, 0};
    if (polytype == "AA") { hi[0] = t11; hi[3] = t11; }
    else if (polytype == "AB" || polytype == "AB1") { hi[1] = t11; }
    else if (polytype == "AB2" || polytype == "3R") { hi[2] = t11; }
    else if (polytype == "AA'" || polytype == "2H") { hi[1] = t11; hi[2] = t11; B2sign[1] = -1.; }
    else if (polytype == "A'B") { hi[3] = t11; B2sign[0] = -1.; }
    else if (polytype == "AB'") { hi[0] = t11; B2sign[1] = -1.; }
    else throw CfgError("Undefined polytype");
    double va[3][2], vb[3][2];
    honeycomb(a0, va, vb);
    TBBuilder tb(4);
    const double f3t = 2. * t2[0] * std::sin(phi0[0]);
    haldane_block_h(tb, 0, va, vb, t1[0], 2. * t2[0] * std::cos(phi0[0]), M0[0], f3t, B2sign[0]);
    if (same) {
        haldane_block_h(tb, 2, va, vb, t1[0], 2. * t2[0] * std::cos(phi0[0]), M0[0], f3t, B2sign[1]);
    } else {
        // B3_b = M0_b - f3b * (M0_t - f3t sum sin(k.b))
        const double f3b = 2. * t2[1] * std::sin(phi0[1]);
        haldane_block_h(tb, 2, va, vb, t1[1], 2. * t2[1] * std::cos(phi0[1]), M0[1] - f3b * M0[0], -f3b * f3t,
                        B2sign[1]);
    }
    haldane_block_j(tb, 0, va, vb, t1[0], 2. * t2[0] * std::cos(phi0[0]), f3t, B2sign[0], false);
    haldane_block_j(tb, 2, va, vb, t1[1], 2. * t2[1] * std::cos(phi0[1]), 2. * t2[1] * std::sin(phi0[1]),
                    B2sign[1], false);
    // interlayer: H(0,2) = hi0, (0,3) = hi1, (1,2) = hi2, (1,3) = hi3 and their conjugates
    const int im[4][2] = {{0, 2}, {0, 3}, {1, 2}, {1, 3}};
    for (int i = 0; i < 4; ++i) {
        tb.const_(-1, im[i][0], im[i][1], hi[i]);
        tb.const_(-1, im[i][1], im[i][0], hi[i]);
    }
    tb.to_problem(p);
    p.nval = 2;
    set_bz(p, PI / std::sqrt(3.) / a0, 2. * PI / 3. / a0);
}

// ------------------------------------------------------------ XYHlattice
// XYHlattice.h: 4 bands, phases e^{-ik.a_i} of three bond vectors,
// alpha_+- = e^{-ik.a_0} +- e^{-ik.a_1}, beta = e^{-ik.a_2}.  Reference
// specific kept: its J is +dH/dk.
void xyh_lattice(const CfgValue *mat, Problem &p)
{
    double tl, tr, lambda, a0;
    if (!(mat && get_double(mat, "tl", tl) && get_double(mat, "tr", tr) && get_double(mat, "lambda", lambda) &&
          get_double(mat, "a0", a0)))
        throw CfgError("Some XYHlattice paramters are missing");
    a0 /= AU_ANGSTROM;
    const double r3 = std::sqrt(3.);
    const double va[3][2] = {{0., a0 / r3}, {-0.5 * a0, -0.5 * a0 / r3}, {0.5 * a0, -0.5 * a0 / r3}};
    TBBuilder tb(4);
    tb.const_(-1, 0, 0, lambda);
    tb.const_(-1, 1, 1, lambda);
    tb.const_(-1, 2, 2, -lambda);
    tb.const_(-1, 3, 3, -lambda);
    // upper blocks as coefficients of e^{-ik.a_i}, i = 0, 1, 2
    const double c02[3] = {0.75 * tl + 0.25 * tr, 0.75 * tl + 0.25 * tr, tr};
    const double c03[3] = {r3 / 4 * (tl - tr), -r3 / 4 * (tl - tr), 0.};
    const double c13[3] = {0.25 * tl + 0.75 * tr, 0.25 * tl + 0.75 * tr, tl};
    const double *cs[3] = {c02, c03, c13};
    // (row, col) of the three independent entries; (1,2) equals (0,3)
    const int ent[4][3] = {{0, 2, 0}, {0, 3, 1}, {1, 2, 1}, {1, 3, 2}};
    for (int e = 0; e < 4; ++e) {
        const int m = ent[e][0], n = ent[e][1];
        const double *c = cs[ent[e][2]];
        for (int i = 0; i < 3; ++i) {
            const double *a = va[i];
            tb.exp_(-1, m, n, -a[0], -a[1], c[i]);
            tb.exp_(-1, n, m, a[0], a[1], c[i]);  // conjugate entry
            for (int ax = 0; ax < 2; ++ax) {
                tb.exp_(ax, m, n, -a[0], -a[1], c[i] * (-I1 * a[ax]));
                tb.exp_(ax, n, m, a[0], a[1], c[i] * (I1 * a[ax]));
            }
        }
    }
    tb.to_problem(p);
    p.nval = 2;
    set_bz(p, PI / a0, 2. * PI / r3 / a0);
}

// ------------------------------------------------------------ SquareSBand
// SquareSBand.h: H = [[M0, B1], [B1, -M0]], B1 = 2 t1 (cos(a kx) + cos(a ky)).
// Reference specific kept: its GenJMatrix sets only the (0,1) entries,
// J_x(0,1) = 2 t1 a sin(a kx), J_y(0,1) = 2 t1 a sin(a ky) -- a
// non-Hermitian current operator.  The kernels use full J tables and the
// reference's -i(HY - (HY)^dag) commutator, so the velocity-gauge
// H = diag(eps) + A.P it implies is propagated as the reference does.
void square_sband(const CfgValue *mat, Problem &p)
{
    double t1, M0, a0;
    if (!(mat && get_double(mat, "t1", t1) && get_double(mat, "M0", M0) && get_double(mat, "a0", a0)))
        throw CfgError("Some SquareSBand paramters are missing");
    a0 /= AU_ANGSTROM;
    TBBuilder tb(2);
    tb.const_(-1, 0, 0, M0);
    tb.const_(-1, 1, 1, -M0);
    for (int m = 0; m < 2; ++m) {
        tb.cos_(-1, m, 1 - m, a0, 0, 2 * t1);
        tb.cos_(-1, m, 1 - m, 0, a0, 2 * t1);
    }
    tb.sin_(0, 0, 1, a0, 0, 2 * t1 * a0);
    tb.sin_(1, 0, 1, 0, a0, 2 * t1 * a0);
    tb.to_problem(p);
    p.nval = 1;
    set_bz(p, PI / a0, PI / a0);
}

// ------------------------------------------------------------ Bi2Se3surf
// Bi2Se3surf.h (surface states, PRA 103, 023101): two bands, parameters
// hard-coded in the constructor (the cfg group is not read), triangular
// vectors a_i and b_i (SetBasis).  With A = sum over i of cos / sin (k.a_i),
// B likewise, and w = -2 pi / 3 (GenBcomp):
//   h0 = 2 A0 cosA + 2 B0 cosB,   h5 = 2 A1 cosA + 2 B1 cosB + m11,
//   h1 = -2 A3 sin(w) (sin a_1 - sin a_2) + 2 B3 (sin b_0 + cos(w) (sin b_1 - sin b_2)),
//   h2 = -2 B3 sin(w) (sin b_1 - sin b_2) - 2 A3 (sin a_0 + cos(w) (sin a_1 + sin a_2)),
//   h3 = 2 A2 sinA;
//   B0 = h0 + (B0/B1)(h5(Gamma) - h5), B_{1,2,3} = sqrt(1 - B0^2/B1^2) h_{1,2,3},
//   H = [[B0 + B3, B1 - i B2], [B1 + i B2, B0 - B3]].
// GenJMatrix writes J = -(dB/dk) term by term: its derivative of the B3 part
// of h1 carries (b_1 + b_2) where h1 has (b_1 - b_2) -- transcribed as
// written; B3 = 0 in the hard-coded set, so the term vanishes.
void bi2se3_surface(Problem &p)
{
    const double AU_EV = 27.211386245988;  // constant.h:35
    const double Ac[4] = {-0.0255 / AU_EV, 0.1937 / AU_EV, 0.2240 / AU_EV, 0.0551 / AU_EV};
    const double Bc[4] = {0.0164 / AU_EV, 0.1203 / AU_EV, 0.3264 / AU_EV, 0.0 / AU_EV};
    const double m11 = -1.6978 / AU_EV, a0 = 4.14 / AU_ANGSTROM, r3 = std::sqrt(3.);
    const double va[3][2] = {{a0, 0.}, {-a0 / 2, r3 / 2 * a0}, {-a0 / 2, -r3 / 2 * a0}};
    const double vb[3][2] = {{0., r3 * a0 / 3}, {-a0 / 2, -r3 / 6 * a0}, {a0 / 2, -r3 / 6 * a0}};
    const double w = -2. * PI / 3., sw = std::sin(w), cw = std::cos(w);
    const double rb = Bc[0] / Bc[1], bco = std::sqrt(1. - Bc[0] * Bc[0] / (Bc[1] * Bc[1]));
    const double h5g = 6. * Ac[1] + 6. * Bc[1] + m11;
    TBBuilder tb(2);
    // B0 on both diagonal entries; B3 = +/- on them
    auto diag = [&](int a, int sign, auto add) {
        add(a, 0, 0, 1.0);
        add(a, 1, 1, sign);
    };
    for (int i = 0; i < 3; ++i) {
        // B0 = h0 - rb h5 + rb h5(Gamma)
        diag(-1, 1, [&](int a, int m, int n, double sg) {
            tb.cos_(a, m, n, va[i][0], va[i][1], sg * (2. * Ac[0] - rb * 2. * Ac[1]));
            tb.cos_(a, m, n, vb[i][0], vb[i][1], sg * (2. * Bc[0] - rb * 2. * Bc[1]));
        });
        // B3 = bco 2 A2 sinA: +H00, -H11
        diag(-1, -1, [&](int a, int m, int n, double sg) {
            tb.sin_(a, m, n, va[i][0], va[i][1], sg * bco * 2. * Ac[2]);
        });
    }
    diag(-1, 1, [&](int a, int m, int n, double sg) { tb.const_(a, m, n, sg * rb * (h5g - m11)); });
    // B1 -/+ i B2 off the diagonal: (0,1) gets B1 - i B2, (1,0) B1 + i B2
    auto offd = [&](int a, double vx, double vy, bool is_cos, double c1, double c2) {
        // c1 f(k.v) into B1 and c2 f(k.v) into B2
        for (int m = 0; m < 2; ++m) {
            const cplx c = c1 + (m == 0 ? -1.0 : 1.0) * I1 * c2;
            if (is_cos) tb.cos_(a, m, 1 - m, vx, vy, c);
            else tb.sin_(a, m, 1 - m, vx, vy, c);
        }
    };
    // h1 = -2 A3 sw (sin a1 - sin a2) + 2 B3 (sin b0 + cw (sin b1 - sin b2))
    offd(-1, va[1][0], va[1][1], false, bco * (-2. * Ac[3] * sw), 0.);
    offd(-1, va[2][0], va[2][1], false, bco * (2. * Ac[3] * sw), 0.);
    offd(-1, vb[0][0], vb[0][1], false, bco * (2. * Bc[3]), 0.);
    offd(-1, vb[1][0], vb[1][1], false, bco * (2. * Bc[3] * cw), 0.);
    offd(-1, vb[2][0], vb[2][1], false, bco * (-2. * Bc[3] * cw), 0.);
    // h2 = -2 B3 sw (sin b1 - sin b2) - 2 A3 (sin a0 + cw (sin a1 + sin a2))
    offd(-1, vb[1][0], vb[1][1], false, 0., bco * (-2. * Bc[3] * sw));
    offd(-1, vb[2][0], vb[2][1], false, 0., bco * (2. * Bc[3] * sw));
    offd(-1, va[0][0], va[0][1], false, 0., bco * (-2. * Ac[3]));
    offd(-1, va[1][0], va[1][1], false, 0., bco * (-2. * Ac[3] * cw));
    offd(-1, va[2][0], va[2][1], false, 0., bco * (-2. * Ac[3] * cw));
    // J_a = -(dB/dk_a), GenJMatrix term by term
    for (int a = 0; a < 2; ++a) {
        for (int i = 0; i < 3; ++i) {
            // d/dk_a cos(k.v) = -v_a sin(k.v); J gets the minus sign of -(dB0 +/- dB3)
            diag(a, 1, [&](int aa, int m, int n, double sg) {
                tb.sin_(aa, m, n, va[i][0], va[i][1], -sg * -va[i][a] * (2. * Ac[0] - rb * 2. * Ac[1]));
                tb.sin_(aa, m, n, vb[i][0], vb[i][1], -sg * -vb[i][a] * (2. * Bc[0] - rb * 2. * Bc[1]));
            });
            diag(a, -1, [&](int aa, int m, int n, double sg) {
                tb.cos_(aa, m, n, va[i][0], va[i][1], -sg * va[i][a] * bco * 2. * Ac[2]);
            });
        }
        // dh1 = -2 A3 sw (a1 cos a1 - a2 cos a2) + 2 B3 (b0 cos b0 + cw (b1 cos b1 + b2 cos b2))
        offd(a, va[1][0], va[1][1], true, -bco * (-2. * Ac[3] * sw * va[1][a]), 0.);
        offd(a, va[2][0], va[2][1], true, -bco * (2. * Ac[3] * sw * va[2][a]), 0.);
        offd(a, vb[0][0], vb[0][1], true, -bco * (2. * Bc[3] * vb[0][a]), 0.);
        offd(a, vb[1][0], vb[1][1], true, -bco * (2. * Bc[3] * cw * vb[1][a]), 0.);
        offd(a, vb[2][0], vb[2][1], true, -bco * (2. * Bc[3] * cw * vb[2][a]), 0.);
        // dh2 = -2 B3 sw (b1 cos b1 - b2 cos b2) - 2 A3 (a0 cos a0 + cw (a1 cos a1 + a2 cos a2))
        offd(a, vb[1][0], vb[1][1], true, 0., -bco * (-2. * Bc[3] * sw * vb[1][a]));
        offd(a, vb[2][0], vb[2][1], true, 0., -bco * (2. * Bc[3] * sw * vb[2][a]));
        offd(a, va[0][0], va[0][1], true, 0., -bco * (-2. * Ac[3] * va[0][a]));
        offd(a, va[1][0], va[1][1], true, 0., -bco * (-2. * Ac[3] * cw * va[1][a]));
        offd(a, va[2][0], va[2][1], true, 0., -bco * (-2. * Ac[3] * cw * va[2][a]));
    }
    tb.to_problem(p);
    p.nval = 1;
    set_bz(p, PI / a0, 2. * PI / r3 / a0);
}

// ------------------------------------------------------------ TMDCs
// TMDCs.h: the three-band (d_z2, d_xy, d_x2-y2) tight-binding model of
// monolayer MX2 with up to third-neighbour hoppings (G.-B. Liu et al.,
// Phys. Rev. B 88, 085433 (2013), GGA parameters), optionally doubled with
// on-site spin-orbit coupling (6 bands).  H is a trigonometric polynomial in
// alpha = kx a/2 and beta = ky a sqrt(3)/2; its entries are expanded here on
// the vectors (p a/2, q a sqrt(3)/2).  Reference specific kept: its J is the
// written derivative +dH/dk of each entry (GenJMatrix), transcribed term by
// term.
struct FPoly {  // sum over (p, q) of c e^{i (p alpha + q beta)}
    std::vector<std::array<int, 2>> pq;
    std::vector<cplx> c;
    void add(int p, int q, cplx v)
    {
        for (size_t i = 0; i < pq.size(); ++i)
            if (pq[i][0] == p && pq[i][1] == q) {
                c[i] += v;
                return;
            }
        pq.push_back({p, q});
        c.push_back(v);
    }
};
FPoly operator+(FPoly a, const FPoly &b)
{
    for (size_t i = 0; i < b.pq.size(); ++i) a.add(b.pq[i][0], b.pq[i][1], b.c[i]);
    return a;
}
FPoly operator*(cplx s, FPoly a)
{
    for (auto &v : a.c) v *= s;
    return a;
}
FPoly operator-(const FPoly &a, const FPoly &b) { return a + cplx(-1.0) * b; }
FPoly operator*(const FPoly &a, const FPoly &b)
{
    FPoly r;
    for (size_t i = 0; i < a.pq.size(); ++i)
        for (size_t j = 0; j < b.pq.size(); ++j)
            r.add(a.pq[i][0] + b.pq[j][0], a.pq[i][1] + b.pq[j][1], a.c[i] * b.c[j]);
    return r;
}
FPoly fconst(cplx v)
{
    FPoly r;
    r.add(0, 0, v);
    return r;
}
// cos(n x), sin(n x) of x = alpha (axis 0) or beta (axis 1)
FPoly fcos(int axis, int n)
{
    FPoly r;
    r.add(axis == 0 ? n : 0, axis == 1 ? n : 0, 0.5);
    r.add(axis == 0 ? -n : 0, axis == 1 ? -n : 0, 0.5);
    return r;
}
FPoly fsin(int axis, int n)
{
    FPoly r;
    r.add(axis == 0 ? n : 0, axis == 1 ? n : 0, -0.5 * I1);
    r.add(axis == 0 ? -n : 0, axis == 1 ? -n : 0, 0.5 * I1);
    return r;
}

void tmdcs(const CfgValue *mat, Problem &p)
{
    bool soc = false;
    std::string name;
    if (mat) {
        get_bool(mat, "isSOCEnabled", soc);
        get_string(mat, "Material", name);
    }
    // GGA parameters (eV) e1 e2 t0 t1 t2 t11 t12 t22 r0 r1 r2 r11 r12 u0 u1 u2 u11 u12 u22
    // of MoS2, WS2, MoSe2, WSe2, MoTe2, WTe2 (Liu et al. 2013, Table III; TMDCs.h)
    static const double gga[6][19] = {
        {0.683, 1.707, -0.146, -0.114, 0.506, 0.085, 0.162, 0.073, 0.060, -0.236, 0.067, 0.016, 0.087, -0.038,
         0.046, 0.001, 0.266, -0.176, -0.150},
        {0.717, 1.916, -0.152, -0.097, 0.590, 0.047, 0.178, 0.016, 0.069, -0.261, 0.107, -0.003, 0.109, -0.054,
         0.045, 0.002, 0.325, -0.206, -0.163},
        {0.684, 1.546, -0.146, -0.130, 0.432, 0.144, 0.117, 0.075, 0.039, -0.209, 0.069, 0.052, 0.060, -0.042,
         0.036, 0.008, 0.272, -0.172, -0.150},
        {0.728, 1.655, -0.146, -0.124, 0.507, 0.117, 0.127, 0.015, 0.036, -0.234, 0.107, 0.044, 0.075, -0.061,
         0.032, 0.007, 0.329, -0.202, -0.164},
        {0.588, 1.303, -0.226, -0.234, 0.036, 0.400, 0.098, 0.017, 0.003, -0.025, -0.169, 0.082, 0.051, 0.057,
         0.103, 0.187, -0.045, -0.141, 0.087},
        {0.697, 1.380, -0.109, -0.164, 0.368, 0.204, 0.093, 0.038, -0.015, -0.209, 0.107, 0.115, 0.009, -0.066,
         0.011, -0.013, 0.312, -0.177, -0.132}};
    static const char *names[6] = {"MoS2", "WS2", "MoSe2", "WSe2", "MoTe2", "WTe2"};
    static const double lat[6] = {3.190, 3.191, 3.326, 3.325, 3.557, 3.560};   // Angstrom
    static const double socp[6] = {0.073, 0.211, 0.091, 0.228, 0.107, 0.237};  // eV
    int mi = -1;
    for (int i = 0; i < 6; ++i)
        if (name == names[i]) mi = i;
    if (mi < 0) throw CfgError("Unknowm material: " + name);
    const double AU_EV = 27.211386245988;  // constant.h:35
    double P[19];
    for (int i = 0; i < 19; ++i) P[i] = gga[mi][i] / AU_EV;
    const double a0 = lat[mi] / AU_ANGSTROM, sp = socp[mi] / AU_EV;
    const double e1 = P[0], e2 = P[1], t0 = P[2], t1 = P[3], t2 = P[4], t11 = P[5], t12 = P[6], t22 = P[7];
    const double r0 = P[8], r1 = P[9], r2 = P[10], r11 = P[11], r12 = P[12];
    const double u0 = P[13], u1 = P[14], u2 = P[15], u11 = P[16], u12 = P[17], u22 = P[18];
    const double r3 = std::sqrt(3.);
    auto ca = [](int i) { return fcos(0, i + 1); };
    auto sa = [](int i) { return fsin(0, i + 1); };
    auto cb = [](int i) { return fcos(1, i + 1); };
    auto sb = [](int i) { return fsin(1, i + 1); };
    auto C = [](double v) { return fconst(v); };
    const cplx i1 = I1;
    // GenHamiltonian
    const FPoly V0 = C(e1) + C(2 * t0) * (C(2) * ca(0) * cb(0) + ca(1)) + C(2 * r0) * (C(2) * ca(2) * cb(0) + cb(1)) +
                     C(2 * u0) * (C(2) * ca(1) * cb(1) + ca(3));
    const FPoly V1 = (C(-2 * r3 * t2) * sa(0) * sb(0) + C(2 * (r1 + r2)) * sa(2) * sb(0) - C(2 * r3 * u2) * sa(1) * sb(1)) +
                     i1 * (C(2 * t1) * sa(0) * (C(2) * ca(0) + cb(0)) + C(2 * (r1 - r2)) * sa(2) * cb(0) +
                           C(2 * u1) * sa(1) * (C(2) * ca(1) + cb(1)));
    const FPoly V2 = (C(2 * t2) * (ca(1) - ca(0) * cb(0)) - C(2 / r3 * (r1 + r2)) * (ca(2) * cb(0) - cb(1)) +
                      C(2 * u2) * (ca(3) - ca(1) * cb(1))) +
                     i1 * (C(2 * r3 * t1) * ca(0) * sb(0) + C(2 / r3) * sb(0) * C(r1 - r2) * (ca(2) + C(2) * cb(0)) +
                           C(2 * r3 * u1) * ca(1) * sb(1));
    const FPoly V11 = C(e2) + C(t11 + 3 * t22) * ca(0) * cb(0) + C(2 * t11) * ca(1) + C(4 * r11) * ca(2) * cb(0) +
                      C(2 * (r11 + r3 * r12)) * cb(1) + C(u11 + 3 * u22) * ca(1) * cb(1) + C(2 * u11) * ca(3);
    const FPoly V12 = (C(r3 * (t22 - t11)) * sa(0) * sb(0) + C(4 * r12) * sa(2) * sb(0) +
                       C(r3 * (u22 - u11)) * sa(1) * sb(1)) +
                      i1 * (C(4 * t12) * sa(0) * (ca(0) - cb(0)) + C(4 * u12) * sa(1) * (ca(1) - cb(1)));
    const FPoly V22 = C(e2) + C(3 * t11 + t22) * ca(0) * cb(0) + C(2 * t22) * ca(1) +
                      C(2 * r11) * (C(2) * ca(2) * cb(0) + cb(1)) + C(2 / r3 * r12) * (C(4) * ca(2) * cb(0) - cb(1)) +
                      C(3 * u11 + u22) * ca(1) * cb(1) + C(2 * u22) * ca(3);
    // GenJMatrix: d/dkx of cos/sin((i+1) alpha) and d/dky of cos/sin((i+1) beta)
    const double da = a0 / 2, db = a0 * r3 / 2;
    auto dca = [&](int i) { return C(-(i + 1) * da) * sa(i); };
    auto dsa = [&](int i) { return C((i + 1) * da) * ca(i); };
    auto dcb = [&](int i) { return C(-(i + 1) * db) * sb(i); };
    auto dsb = [&](int i) { return C((i + 1) * db) * cb(i); };
    const FPoly dxV0 = C(2 * t0) * (C(2) * dca(0) * cb(0) + dca(1)) + C(2 * r0) * (C(2) * dca(2) * cb(0)) +
                       C(2 * u0) * (C(2) * dca(1) * cb(1) + dca(3));
    const FPoly dxV1 =
        (C(-2 * r3 * t2) * dsa(0) * sb(0) + C(2 * (r1 + r2)) * dsa(2) * sb(0) - C(2 * r3 * u2) * dsa(1) * sb(1)) +
        i1 * (C(2 * t1) * dsa(0) * (C(2) * ca(0) + cb(0)) + C(2 * t1) * sa(0) * (C(2) * dca(0)) +
              C(2 * (r1 - r2)) * dsa(2) * cb(0) + C(2 * u1) * dsa(1) * (C(2) * ca(1) + cb(1)) +
              C(2 * u1) * sa(1) * (C(2) * dca(1)));
    const FPoly dxV2 = (C(2 * t2) * (dca(1) - dca(0) * cb(0)) - C(2 / r3 * (r1 + r2)) * (dca(2) * cb(0)) +
                        C(2 * u2) * (dca(3) - dca(1) * cb(1))) +
                       i1 * (C(2 * r3 * t1) * dca(0) * sb(0) + C(2 / r3) * sb(0) * C(r1 - r2) * dca(2) +
                             C(2 * r3 * u1) * dca(1) * sb(1));
    const FPoly dxV11 = C(t11 + 3 * t22) * dca(0) * cb(0) + C(2 * t11) * dca(1) + C(4 * r11) * dca(2) * cb(0) +
                        C(u11 + 3 * u22) * dca(1) * cb(1) + C(2 * u11) * dca(3);
    const FPoly dxV12 = (C(r3 * (t22 - t11)) * dsa(0) * sb(0) + C(4 * r12) * dsa(2) * sb(0) +
                         C(r3 * (u22 - u11)) * dsa(1) * sb(1)) +
                        i1 * (C(4 * t12) * dsa(0) * (ca(0) - cb(0)) + C(4 * t12) * sa(0) * dca(0) +
                              C(4 * u12) * dsa(1) * (ca(1) - cb(1)) + C(4 * u12) * sa(1) * dca(1));
    const FPoly dxV22 = C(3 * t11 + t22) * dca(0) * cb(0) + C(2 * t22) * dca(1) + C(2 * r11) * (C(2) * dca(2) * cb(0)) +
                        C(2 / r3 * r12) * (C(4) * dca(2) * cb(0)) + C(3 * u11 + u22) * dca(1) * cb(1) +
                        C(2 * u22) * dca(3);
    const FPoly dyV0 = C(2 * t0) * (C(2) * ca(0) * dcb(0)) + C(2 * r0) * (C(2) * ca(2) * dcb(0) + dcb(1)) +
                       C(2 * u0) * (C(2) * ca(1) * dcb(1));
    const FPoly dyV1 =
        (C(-2 * r3 * t2) * sa(0) * dsb(0) + C(2 * (r1 + r2)) * sa(2) * dsb(0) - C(2 * r3 * u2) * sa(1) * dsb(1)) +
        i1 * (C(2 * t1) * sa(0) * dcb(0) + C(2 * (r1 - r2)) * sa(2) * dcb(0) + C(2 * u1) * sa(1) * dcb(1));
    const FPoly dyV2 = (C(2 * t2) * (C(-1) * ca(0) * dcb(0)) - C(2 / r3 * (r1 + r2)) * (ca(2) * dcb(0) - dcb(1)) +
                        C(2 * u2) * (C(-1) * ca(1) * dcb(1))) +
                       i1 * (C(2 * r3 * t1) * ca(0) * dsb(0) + C(2 / r3) * dsb(0) * C(r1 - r2) * (ca(2) + C(2) * cb(0)) +
                             C(2 / r3) * sb(0) * C(r1 - r2) * (C(2) * dcb(0)) + C(2 * r3 * u1) * ca(1) * dsb(1));
    const FPoly dyV11 = C(t11 + 3 * t22) * ca(0) * dcb(0) + C(4 * r11) * ca(2) * dcb(0) +
                        C(2 * (r11 + r3 * r12)) * dcb(1) + C(u11 + 3 * u22) * ca(1) * dcb(1);
    const FPoly dyV12 = (C(r3 * (t22 - t11)) * sa(0) * dsb(0) + C(4 * r12) * sa(2) * dsb(0) +
                         C(r3 * (u22 - u11)) * sa(1) * dsb(1)) +
                        i1 * (C(4 * t12) * sa(0) * (C(-1) * dcb(0)) + C(4 * u12) * sa(1) * (C(-1) * dcb(1)));
    const FPoly dyV22 = C(3 * t11 + t22) * ca(0) * dcb(0) + C(2 * r11) * (C(2) * ca(2) * dcb(0) + dcb(1)) +
                        C(2 / r3 * r12) * (C(4) * ca(2) * dcb(0) - dcb(1)) + C(3 * u11 + u22) * ca(1) * dcb(1);
    auto conjp = [](FPoly a) {  // conj(sum c e^{i(p,q)}) = sum conj(c) e^{-i(p,q)}
        for (auto &x : a.pq) x = {-x[0], -x[1]};
        for (auto &v : a.c) v = std::conj(v);
        return a;
    };
    const int N = soc ? 6 : 3;
    TBBuilder tb(N);
    auto put = [&](int a, int m, int n, const FPoly &f) {
        for (size_t i = 0; i < f.pq.size(); ++i) tb.exp_(a, m, n, f.pq[i][0] * da, f.pq[i][1] * db, f.c[i]);
    };
    // one 3x3 block at offset o; s = +1 / -1: sign of the soc term on (1,2) / (2,1)
    auto block = [&](int o, double s) {
        const FPoly *H[3][3] = {{&V0, &V1, &V2}, {nullptr, &V11, &V12}, {nullptr, nullptr, &V22}};
        const FPoly *Jx[3][3] = {{&dxV0, &dxV1, &dxV2}, {nullptr, &dxV11, &dxV12}, {nullptr, nullptr, &dxV22}};
        const FPoly *Jy[3][3] = {{&dyV0, &dyV1, &dyV2}, {nullptr, &dyV11, &dyV12}, {nullptr, nullptr, &dyV22}};
        for (int m = 0; m < 3; ++m)
            for (int n = m; n < 3; ++n) {
                put(-1, o + m, o + n, *H[m][n]);
                put(0, o + m, o + n, *Jx[m][n]);
                put(1, o + m, o + n, *Jy[m][n]);
                if (n != m) {
                    put(-1, o + n, o + m, conjp(*H[m][n]));
                    put(0, o + n, o + m, conjp(*Jx[m][n]));
                    put(1, o + n, o + m, conjp(*Jy[m][n]));
                }
            }
        if (soc) {
            tb.const_(-1, o + 1, o + 2, s * sp * I1);
            tb.const_(-1, o + 2, o + 1, -s * sp * I1);
        }
    };
    block(0, 1.0);
    if (soc) block(3, -1.0);
    tb.to_problem(p);
    p.nval = soc ? 2 : 1;
    set_bz(p, PI / a0, 2. * PI / r3 / a0);
}

}  // namespace

bool build_material(const std::string &target, const CfgValue *mat, Problem &p)
{
    if (target == "WilsonMass") wilson_mass(mat, p);
    else if (target == "KaneMele") kane_mele(mat, p);
    else if (target == "Haldane2L") haldane_2l(mat, p);
    else if (target == "XYHlattice") xyh_lattice(mat, p);
    else if (target == "TMDCs") tmdcs(mat, p);
    else if (target == "SquareSBand") square_sband(mat, p);
    else if (target == "Bi2Se3surf") bi2se3_surface(p);   // SBEs.h:183-186; no parameters read
    else return false;
    p.model = MODEL_TB;
    return true;
}

}  // namespace sbe
