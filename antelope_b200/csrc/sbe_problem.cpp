// inputParam.cfg parsing, the reference's defaults and checks, and the FP64
// laser.  Diagnostics reuse the reference's own wording so that a user sees
// the same message for the same mistake.
#include "sbe_problem.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <sstream>

namespace sbe {

extern const double PI = 4.0 * std::atan(1.0);   // constant.h:19
extern const double AU_ANGSTROM = 0.529177210903;  // constant.h:32

// ================================================================= parser
const CfgValue *CfgValue::get(const std::string &key) const
{
    if (type != Group) return nullptr;
    for (const auto &it : items)
        if (it->name == key) return it.get();
    return nullptr;
}

namespace {

struct Lexer {
    const std::string &s;
    size_t i = 0;
    explicit Lexer(const std::string &text) : s(text) {}

    int line_at(size_t pos) const { return 1 + (int)std::count(s.begin(), s.begin() + std::min(pos, s.size()), '\n'); }
    [[noreturn]] void fail(const std::string &m) const
    {
        throw CfgError("line " + std::to_string(line_at(i)) + ": " + m);
    }
    void ws()
    {
        for (;;) {
            while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
            if (i >= s.size()) return;
            if (s[i] == '#' || s.compare(i, 2, "//") == 0) {
                while (i < s.size() && s[i] != '\n') ++i;
            } else if (s.compare(i, 2, "/*") == 0) {
                size_t e = s.find("*/", i + 2);
                if (e == std::string::npos) fail("unterminated comment");
                i = e + 2;
            } else if (s[i] == '@') {
                fail("@include is not supported");
            } else {
                return;
            }
        }
    }
    bool eat(char c)
    {
        ws();
        if (i < s.size() && s[i] == c) { ++i; return true; }
        return false;
    }
    char peek()
    {
        ws();
        return i < s.size() ? s[i] : '\0';
    }
};

void parse_value(Lexer &L, CfgValue &out);

void parse_group_body(Lexer &L, CfgValue &g, char close)
{
    g.type = CfgValue::Group;
    for (;;) {
        char c = L.peek();
        if (c == '\0') {
            if (close) L.fail("unexpected end of input");
            return;
        }
        if (close && c == close) { ++L.i; return; }
        size_t b = L.i;
        if (!(std::isalpha((unsigned char)c) || c == '*')) L.fail("expected a setting name");
        while (L.i < L.s.size() && (std::isalnum((unsigned char)L.s[L.i]) || L.s[L.i] == '_' ||
                                    L.s[L.i] == '-' || L.s[L.i] == '*'))
            ++L.i;
        auto item = std::make_unique<CfgValue>();
        item->name = L.s.substr(b, L.i - b);
        if (g.get(item->name)) L.fail("duplicate setting '" + item->name + "'");
        if (!L.eat('=') && !L.eat(':')) L.fail("expected '=' or ':' after '" + item->name + "'");
        parse_value(L, *item);
        g.items.push_back(std::move(item));
        if (!L.eat(';')) L.eat(',');
    }
}

void parse_scalar(Lexer &L, CfgValue &out)
{
    char c = L.peek();
    if (c == '"') {
        out.type = CfgValue::String;
        while (L.peek() == '"') {
            ++L.i;
            while (L.i < L.s.size() && L.s[L.i] != '"') {
                char d = L.s[L.i++];
                if (d == '\\' && L.i < L.s.size()) {
                    char e = L.s[L.i++];
                    d = e == 'n' ? '\n' : e == 't' ? '\t' : e == 'r' ? '\r' : e == 'f' ? '\f' : e;
                }
                out.sval.push_back(d);
            }
            if (L.i >= L.s.size()) L.fail("unterminated string");
            ++L.i;
        }
        return;
    }
    size_t b = L.i;
    while (L.i < L.s.size() && (std::isalnum((unsigned char)L.s[L.i]) || L.s[L.i] == '.' || L.s[L.i] == '+' ||
                                L.s[L.i] == '-'))
        ++L.i;
    std::string tok = L.s.substr(b, L.i - b);
    if (tok.empty()) L.fail("expected a value");
    std::string low = tok;
    for (auto &ch : low) ch = (char)std::tolower((unsigned char)ch);
    if (low == "true" || low == "false") {
        out.type = CfgValue::Bool;
        out.bval = low == "true";
        return;
    }
    const bool hex = low.find("0x") != std::string::npos;
    char *end = nullptr;
    if (!hex && (low.find('.') != std::string::npos || low.find('e') != std::string::npos)) {
        out.type = CfgValue::Float;
        out.fval = std::strtod(tok.c_str(), &end);
        if (*end) L.fail("malformed number '" + tok + "'");
        return;
    }
    std::string t = tok;
    bool i64 = false;
    while (!t.empty() && (t.back() == 'L' || t.back() == 'l')) { t.pop_back(); i64 = true; }
    out.type = i64 ? CfgValue::Int64 : CfgValue::Int;
    out.ival = std::strtoll(t.c_str(), &end, 0);
    if (t.empty() || *end) L.fail("malformed value '" + tok + "'");
}

void parse_value(Lexer &L, CfgValue &out)
{
    char c = L.peek();
    if (c == '{') {
        ++L.i;
        parse_group_body(L, out, '}');
    } else if (c == '[' || c == '(') {
        ++L.i;
        const char close = c == '[' ? ']' : ')';
        out.type = c == '[' ? CfgValue::Array : CfgValue::List;
        if (L.eat(close)) return;
        for (;;) {
            auto item = std::make_unique<CfgValue>();
            parse_value(L, *item);
            if (out.type == CfgValue::Array) {
                if (item->type == CfgValue::Group || item->type == CfgValue::Array || item->type == CfgValue::List)
                    L.fail("an array holds scalars only");
                if (!out.items.empty() && out.items[0]->type != item->type)
                    L.fail("array elements must have one type");
            }
            out.items.push_back(std::move(item));
            if (L.eat(',')) continue;
            if (L.eat(close)) return;
            L.fail(std::string("expected ',' or '") + close + "'");
        }
    } else {
        parse_scalar(L, out);
    }
}

}  // namespace

// ---- typed access with libconfig's strict rules (no auto-conversion)
bool get_double(const CfgValue *g, const char *key, double &v)
{
    const CfgValue *x = g ? g->get(key) : nullptr;
    if (!x || x->type != CfgValue::Float) return false;
    v = x->fval;
    return true;
}
bool get_int(const CfgValue *g, const char *key, int &v)
{
    const CfgValue *x = g ? g->get(key) : nullptr;
    if (!x || (x->type != CfgValue::Int && x->type != CfgValue::Int64)) return false;
    v = (int)x->ival;
    return true;
}
bool get_bool(const CfgValue *g, const char *key, bool &v)
{
    const CfgValue *x = g ? g->get(key) : nullptr;
    if (!x || x->type != CfgValue::Bool) return false;
    v = x->bval;
    return true;
}
bool get_string(const CfgValue *g, const char *key, std::string &v)
{
    const CfgValue *x = g ? g->get(key) : nullptr;
    if (!x || x->type != CfgValue::String) return false;
    v = x->sval;
    return true;
}

namespace {
// element i of an array/list setting as a float (type error otherwise)
double elem_double(const CfgValue &arr, size_t i, const char *err)
{
    if (i >= arr.items.size() || arr.items[i]->type != CfgValue::Float) throw CfgError(err);
    return arr.items[i]->fval;
}
int elem_int(const CfgValue &arr, size_t i, const char *err)
{
    if (i >= arr.items.size() || (arr.items[i]->type != CfgValue::Int && arr.items[i]->type != CfgValue::Int64))
        throw CfgError(err);
    return (int)arr.items[i]->ival;
}

}  // namespace

std::unique_ptr<CfgValue> parse_cfg(const std::string &text)
{
    Lexer L(text);
    auto root = std::make_unique<CfgValue>();
    parse_group_body(L, *root, 0);
    return root;
}

// ================================================================= laser
void Pulse::derive()
{
    period0 = 2.0 * PI / w0;                                    // laser.h:75
    twidth_clipped = 0.0;
    switch (env) {                                              // laser.h:88-113
        case ENV_GAUSS:
            twidth = 2.0 * ncycles * period0;
            envfactor = -4 * std::log(2) / (ncycles * period0 * ncycles * period0);
            break;
        case ENV_GAUSS_CLIPPED:
            twidth = 2.0 * ncycles * period0 + ncycles_clipped * period0 / 2;
            twidth_clipped = ncycles_clipped * period0 / 2;
            envfactor = -4 * std::log(2) / (ncycles * period0 * ncycles * period0);
            break;
        case ENV_COS4:
        case ENV_SIN2:
            twidth = ncycles * period0 / 2;
            envfactor = w0 / (2 * ncycles);
            break;
        default:
            twidth = (ncycles + ncycles_clipped) * period0 / 2;
            twidth_clipped = ncycles_clipped * period0 / 2;
            envfactor = w0 / (2 * ncycles);
            break;
    }
    const double factor = std::sqrt(1.0 / (1.0 + ellip * ellip));  // laser.h:116-127
    E0x = factor * E0;
    E0y = ellip * factor * E0;
    if (w0 > 1.0e-30) { A0x = E0x / w0; A0y = E0y / w0; }
    else { A0x = 0.; A0y = 0.; }
    const double tx0[3] = {std::cos(thetaz) * std::cos(phiz), std::cos(thetaz) * std::sin(phiz), -std::sin(thetaz)};
    const double ty0[3] = {-std::sin(phiz), std::cos(phiz), 0.};
    for (int i = 0; i < 3; ++i) {                                // laser.h:133-140
        xdir[i] = std::cos(phix) * tx0[i] + std::sin(phix) * ty0[i];
        ydir[i] = -std::sin(phix) * tx0[i] + std::cos(phix) * ty0[i];
    }
}

// laser.h:150-206; sin2 (extension): cos^2(t w0 / (2N)) on |t| <= N T / 2
double Pulse::envelope(double t, bool d) const
{
    const double ef = envfactor;
    double to;
    switch (env) {
        case ENV_COS4:
            if (std::fabs(t) > twidth) return 0;
            if (d) return -4. * ef * std::sin(t * ef) * std::pow(std::cos(t * ef), 3.);
            return std::pow(std::cos(t * ef), 4.);
        case ENV_SIN2:
            if (std::fabs(t) > twidth) return 0;
            if (d) return -2. * ef * std::sin(t * ef) * std::cos(t * ef);
            return std::cos(t * ef) * std::cos(t * ef);
        case ENV_COS4_CLIPPED:
            if (std::fabs(t) > twidth) return 0;
            if (t > twidth_clipped) to = t - twidth_clipped;
            else if (t > -twidth_clipped) return d ? 0. : 1.;
            else to = t + twidth_clipped;
            if (d) return -4. * ef * std::sin(to * ef) * std::pow(std::cos(to * ef), 3.);
            return std::pow(std::cos(to * ef), 4.);
        case ENV_GAUSS:
            if (d) return 2 * t * ef * std::exp(ef * t * t);
            return std::exp(ef * t * t);
        default:  // ENV_GAUSS_CLIPPED
            if (t > twidth_clipped) to = t - twidth_clipped;
            else if (t > -twidth_clipped) return d ? 0. : 1.;
            else to = t + twidth_clipped;
            if (d) return 2 * to * ef * std::exp(ef * to * to);
            return std::exp(ef * to * to);
    }
}

void Pulse::eval(double t, double *A, double *E) const  // laser.h:209-238
{
    const double kt = t - t0;
    const double s = std::sin(kt * w0 - cep), c = std::cos(kt * w0 - cep);
    const double f = envelope(kt, false), fp = envelope(kt, true);
    const double ax = -A0x * s * f, ay = A0y * c * f;
    const double ex = E0x * c * f - A0x * s * fp;
    const double ey = E0y * s * f + A0y * c * fp;
    for (int i = 0; i < 3; ++i) {
        if (A) A[i] = ax * xdir[i] + ay * ydir[i];
        if (E) E[i] = ex * xdir[i] + ey * ydir[i];
    }
}

void Laser::eval(double t, double *A, double *E) const
{
    double a[3] = {0, 0, 0}, e[3] = {0, 0, 0}, pa[3], pe[3];
    for (const auto &p : pulses) {
        p.eval(t, pa, pe);
        for (int d = 0; d < 3; ++d) { a[d] += pa[d]; e[d] += pe[d]; }
    }
    for (int d = 0; d < 3; ++d) {
        if (A) A[d] = a[d] - init_A[d];
        if (E) E[d] = e[d] - init_E[d];
    }
}

void Laser::initialize()
{
    double mn = pulses[0].t0 - pulses[0].twidth, mx = pulses[0].t0 + pulses[0].twidth;
    for (const auto &p : pulses) {
        mn = std::min(mn, p.t0 - p.twidth);
        mx = std::max(mx, p.t0 + p.twidth);
    }
    atmin = mn - offset_before;
    atmax = mx + offset_after;
    for (int d = 0; d < 3; ++d) init_A[d] = init_E[d] = 0.0;
    double A0[3], E0[3];
    eval(atmin, A0, E0);
    for (int d = 0; d < 3; ++d) { init_A[d] = A0[d]; init_E[d] = E0[d]; }
    Nt = (int)std::floor((atmax - atmin) / dt);
}

// ================================================================= problem
void Problem::derive_grid()
{
    double ax[3][3];
    int na = 0;
    for (int i = 0; i < 3; ++i)
        if (Nk[i] != 1) {
            for (int j = 0; j < 3; ++j) ax[na][j] = bzaxes[3 * i + j];
            ++na;
        }
    double c[3];
    switch (na) {  // momaxis.h:217-236
        case 1: volume = std::sqrt(ax[0][0] * ax[0][0] + ax[0][1] * ax[0][1] + ax[0][2] * ax[0][2]); break;
        case 2:
        case 3:
            c[0] = ax[0][1] * ax[1][2] - ax[0][2] * ax[1][1];
            c[1] = ax[0][2] * ax[1][0] - ax[0][0] * ax[1][2];
            c[2] = ax[0][0] * ax[1][1] - ax[1][0] * ax[0][1];
            volume = na == 2 ? std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2])
                             : std::sqrt(c[0] * ax[2][0] + c[1] * ax[2][1] + c[2] * ax[2][2]);
            break;
        default: volume = 1.0; break;
    }
    dV = std::fabs(volume) / ntotal();
    // trapezoid weights: product over axes of (1/2 at either end of an axis of N != 1)
    double tw = 1.0;
    for (int d = 0; d < 3; ++d) tw *= (Nk[d] == 1) ? 1.0 : (Nk[d] - 1.0);
    total_weight = tw;
}

// shotFrequency of antelope.cpp:274-278, from the first pulse's period
// (laser.h:75); snapshots follow the steps n = 0, F, 2F, ... < Nt
int Problem::shot_every() const
{
    if (shot_number <= 0 || laser.pulses.empty()) return 0;
    return (int)(laser.pulses[0].period0 / shot_number / laser.dt);
}

int Problem::nshots() const
{
    const int F = shot_every();
    return F > 0 ? (laser.Nt - 1) / F + 1 : 0;
}

Problem problem_from_cfg(const CfgValue &root, std::string *unsupported)
{
    Problem p;
    auto unsup = [&](const std::string &m) {
        if (unsupported && unsupported->empty()) *unsupported = m;
    };
    // gauge (antelope.cpp:111-129): unknown or absent -> LengthWannier
    std::string g;
    get_string(&root, "gauge", g);
    if (g == "Wannier" || g == "LengthWannier") p.gauge = GAUGE_LENGTH_WANNIER;
    else if (g == "Hamiltonian" || g == "LengthHamiltonian") p.gauge = GAUGE_LENGTH_HAMILTONIAN;
    else if (g == "Velocity" || g == "VelocityHamiltonian") p.gauge = GAUGE_VELOCITY;
    else { p.gauge = GAUGE_LENGTH_WANNIER; p.gauge_given = false; }

    // calc group (SBEs.h:432-509)
    const CfgValue *calc = root.get("calc");
    if (!calc || calc->type != CfgValue::Group) throw CfgError("Setting not found while search calc group ");
    const CfgValue *np = calc->get("Npoints");
    if (!np || (np->type != CfgValue::Array && np->type != CfgValue::List))
        throw CfgError("Setting not found while search calc group ");
    if (np->items.empty() || np->items.size() > 3) throw CfgError("Type exception in calc group");
    for (size_t i = 0; i < np->items.size(); ++i) p.Nk[i] = elem_int(*np, i, "Type exception in calc group");
    for (int i = 0; i < 3; ++i)
        if (p.Nk[i] <= 0) throw CfgError("Number of grid is negative or zero. check N");  // momaxis.h:133-137
    p.dt = 0.1;
    get_double(calc, "dt", p.dt);
    get_double(calc, "T1", p.T1);
    get_double(calc, "T2", p.T2);
    get_int(calc, "shotNumber", p.shot_number);
    get_int(calc, "diagnostic", p.diagnostic);
    int rko = 5;
    get_int(calc, "RKorder", rko);
    get_bool(calc, "InterIntra", p.inter_intra);
    const CfgValue *ks = calc->get("ksfactor");
    if (!ks) throw CfgError("Setting not found while search calc group ");
    if (ks->type != CfgValue::Array && ks->type != CfgValue::List) throw CfgError("Type exception in calc group");
    for (size_t i = 0; i < ks->items.size() && i < 3; ++i)
        p.ksfactor[i] = elem_double(*ks, i, "Type exception in calc group");
    if (rko != 4 && rko != 5) throw CfgError("Not-implemented RK order: " + std::to_string(rko));
    p.rk = rko;
    // extensions: precision, adaptive Cash-Karp
    std::string s;
    if (get_string(calc, "precision", s)) {
        if (s == "fp64") p.precision = 0;
        else if (s == "mixed" || s == "fp32") p.precision = 1;
        else throw CfgError("calc.precision must be \"fp64\" or \"mixed\"");
    }
    if (get_string(calc, "rk", s)) {
        if (s == "rk4") p.rk = 4;
        else if (s == "rk5" || s == "fehlberg5") p.rk = 5;
        else if (s == "cashkarp45") p.rk = 45;
        else throw CfgError("calc.rk must be \"rk4\", \"rk5\" or \"cashkarp45\"");
    }
    get_double(calc, "tol", p.rk_tol);
    if (!(p.dt > 0.0)) throw CfgError("calc.dt must be positive");

    // laser (SBEs.h:511-561)
    const CfgValue *las = root.get("laser");
    const CfgValue *pul = las ? las->get("pulses") : nullptr;
    if (!pul || (pul->type != CfgValue::List && pul->type != CfgValue::Array))
        throw CfgError("No laser, check config file ");
    if (pul->items.empty()) throw CfgError("No laser, check config file ");
    for (const auto &it : pul->items) {
        Pulse q{};
        std::string env;
        const CfgValue *g2 = it.get();
        if (!(get_double(g2, "E0", q.E0) && get_double(g2, "ellip", q.ellip) && get_double(g2, "w0", q.w0) &&
              get_double(g2, "ncycles", q.ncycles) && get_double(g2, "cep", q.cep) && get_double(g2, "t0", q.t0) &&
              get_double(g2, "phix", q.phix) && get_string(g2, "env_name", env)))
            throw CfgError("Error while initilizng laser pulses. Check config file");
        q.cep *= PI / 180.0;
        q.thetaz = q.phiz = 0.0;
        get_double(g2, "thetaz", q.thetaz);
        get_double(g2, "phiz", q.phiz);
        q.phix *= PI / 180.0;
        q.thetaz *= PI / 180.0;
        q.phiz *= PI / 180.0;
        q.ncycles_clipped = 0.0;
        get_double(g2, "ncycles_clipped", q.ncycles_clipped);
        if (env == "cos4") q.env = ENV_COS4;
        else if (env == "gauss") q.env = ENV_GAUSS;
        else if (env == "gauss_clipped") q.env = ENV_GAUSS_CLIPPED;
        else if (env == "cos4_clipped") q.env = ENV_COS4_CLIPPED;
        else if (env == "sin2") q.env = ENV_SIN2;
        else throw CfgError("invalid envelope type");
        q.derive();
        p.laser.pulses.push_back(q);
    }
    if (const CfgValue *off = las->get("offset")) {
        p.laser.offset_before = elem_double(*off, 0, "laser.offset must hold two floats");
        p.laser.offset_after = elem_double(*off, 1, "laser.offset must hold two floats");
    }
    p.laser.dt = p.dt;
    p.laser.initialize();
    if (p.laser.Nt < 1) throw CfgError("the laser time window holds no time step");

    // target and material (SBEs.h:131-241)
    if (!get_string(&root, "target", p.target)) throw CfgError("No 'target' in input file");
    const CfgValue *mat = root.get(p.target);
    bool custom = false;
    if (mat) get_bool(mat, "UsingCustomInitial", custom);
    if (mat && !custom && get_double(mat, "Ef", p.Ef)) p.use_fermi = true;
    if (p.target == "Haldane") {
        p.model = MODEL_HALDANE;
        p.nband = 2;
        p.nval = 1;
        double a0;
        if (!(mat && get_double(mat, "t1", p.hal_t1) && get_double(mat, "t2", p.hal_t2) &&
              get_double(mat, "phi0", p.hal_phi0) && get_double(mat, "a0", a0)))
            throw CfgError("Some Haldane paramters are missing");
        p.hal_a0 = a0 / AU_ANGSTROM;
        if (!get_double(mat, "M0", p.hal_M0)) {
            if (get_double(mat, "Mt2", p.hal_M0)) p.hal_M0 *= p.hal_t2;
            else throw CfgError("M0 param missing");
        }
        const double a = p.hal_a0;  // Haldane::SetBasis (Haldane.h:134-143)
        const double va[3][2] = {{0., a}, {-std::sqrt(3.) / 2 * a, -0.5 * a}, {std::sqrt(3.) / 2 * a, -0.5 * a}};
        const double vb[3][2] = {{std::sqrt(3.) * a, 0.}, {-std::sqrt(3.) / 2 * a, 3. / 2. * a},
                                 {-std::sqrt(3.) / 2 * a, -3. / 2. * a}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 2; ++j) { p.hal_va[i][j] = va[i][j]; p.hal_vb[i][j] = vb[i][j]; }
        const double kxMax = PI / std::sqrt(3.) / a, kyMax = 2. * PI / 3. / a;  // Haldane.h:77-81
        const double axes[9] = {2 * kxMax, 0, 0, 0, 2 * kyMax, 0, 0, 0, 0};
        for (int i = 0; i < 9; ++i) p.bzaxes[i] = axes[i];
        for (int i = 0; i < 3; ++i) p.bzorigin[i] = 0.0;
        if (custom)
            throw CfgError("Error: Try to using custom inital value without implementing GenInitialValue.");
    } else if (p.target == "SyntheticWannier") {
        // explicit tight-binding tables (model form of Materials/Wannier90.h:297-387)
        p.model = MODEL_SYNTHETIC_WANNIER;
        if (!mat || !get_int(mat, "Nband", p.nband) || !get_int(mat, "Nval", p.nval))
            throw CfgError("SyntheticWannier needs Nband and Nval");
        if (p.nband < 2 || p.nband > 8 || p.nval < 0 || p.nval > p.nband)
            throw CfgError("SyntheticWannier: 2 <= Nband <= 8 and 0 <= Nval <= Nband");
        const int N = p.nband;
        auto arr = [&](const char *key) -> const CfgValue & {
            const CfgValue *x = mat->get(key);
            if (!x || (x->type != CfgValue::Array && x->type != CfgValue::List))
                throw CfgError(std::string("SyntheticWannier.") + key + " missing");
            return *x;
        };
        const CfgValue &lat = arr("lattice"), &R = arr("R"), &hre = arr("h_re"), &him = arr("h_im");
        if (lat.items.size() != 4) throw CfgError("SyntheticWannier.lattice needs 4 floats");
        for (int i = 0; i < 4; ++i) p.w_lat[i] = elem_double(lat, i, "SyntheticWannier.lattice: floats");
        if (R.items.empty() || R.items.size() % 2) throw CfgError("SyntheticWannier.R needs pairs of integers");
        p.w_nR = (int)R.items.size() / 2;
        p.w_R.resize(R.items.size());
        for (size_t i = 0; i < R.items.size(); ++i) p.w_R[i] = elem_int(R, i, "SyntheticWannier.R: integers");
        const size_t nh = (size_t)p.w_nR * N * N;
        if (hre.items.size() != nh || him.items.size() != nh)
            throw CfgError("SyntheticWannier.h_re/h_im need nR*Nband*Nband floats");
        p.w_h.resize(2 * nh);
        for (size_t i = 0; i < nh; ++i) {
            p.w_h[2 * i] = elem_double(hre, i, "SyntheticWannier.h_re: floats");
            p.w_h[2 * i + 1] = elem_double(him, i, "SyntheticWannier.h_im: floats");
        }
        if (mat->get("d_re")) {
            const CfgValue &dre = arr("d_re"), &dim = arr("d_im");
            if (dre.items.size() != 2 * nh || dim.items.size() != 2 * nh)
                throw CfgError("SyntheticWannier.d_re/d_im need nR*2*Nband*Nband floats");
            p.w_d.resize(4 * nh);
            for (size_t i = 0; i < 2 * nh; ++i) {
                p.w_d[2 * i] = elem_double(dre, i, "SyntheticWannier.d_re: floats");
                p.w_d[2 * i + 1] = elem_double(dim, i, "SyntheticWannier.d_im: floats");
            }
        }
        // Hermiticity: h_{-R} = h_R^dagger (and the same for d)
        for (int r = 0; r < p.w_nR; ++r) {
            int m = -1;
            for (int q = 0; q < p.w_nR; ++q)
                if (p.w_R[2 * q] == -p.w_R[2 * r] && p.w_R[2 * q + 1] == -p.w_R[2 * r + 1]) m = q;
            if (m < 0) throw CfgError("SyntheticWannier.R must contain -R for every R");
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j) {
                    const size_t a = ((size_t)r * N + i) * N + j, b = ((size_t)m * N + j) * N + i;
                    if (std::fabs(p.w_h[2 * a] - p.w_h[2 * b]) > 1e-12 ||
                        std::fabs(p.w_h[2 * a + 1] + p.w_h[2 * b + 1]) > 1e-12)
                        throw CfgError("SyntheticWannier: h_{-R} must equal h_R^dagger");
                }
        }
        p.w_vec.resize(2 * (size_t)p.w_nR);
        for (int r = 0; r < p.w_nR; ++r) {
            p.w_vec[2 * r] = p.w_R[2 * r] * p.w_lat[0] + p.w_R[2 * r + 1] * p.w_lat[2];
            p.w_vec[2 * r + 1] = p.w_R[2 * r] * p.w_lat[1] + p.w_R[2 * r + 1] * p.w_lat[3];
        }
        // reciprocal basis b_i . a_j = 2 pi delta_ij (Wannier90.h:489-502)
        const double det = p.w_lat[0] * p.w_lat[3] - p.w_lat[1] * p.w_lat[2];
        if (det == 0.0) throw CfgError("SyntheticWannier.lattice is singular");
        const double axes[9] = {2 * PI * p.w_lat[3] / det, -2 * PI * p.w_lat[2] / det, 0,
                                -2 * PI * p.w_lat[1] / det, 2 * PI * p.w_lat[0] / det, 0, 0, 0, 0};
        for (int i = 0; i < 9; ++i) p.bzaxes[i] = axes[i];
        for (int i = 0; i < 3; ++i) p.bzorigin[i] = 0.0;
        if (custom)
            throw CfgError("Error: Try to using custom inital value without implementing GenInitialValue.");
    } else if (build_material(p.target, mat, p)) {
        if (custom)
            throw CfgError("Error: Try to using custom inital value without implementing GenInitialValue.");
    } else if (p.target == "MultiWSM") {
        // MultiWSM.h:45-70: strict double lookups (an integer value is missing
        // to libconfig's lookupValue(double&)), a0 in Angstrom, the zone the
        // cube [-pi/a0, pi/a0]^3
        p.model = MODEL_MULTIWSM;
        p.nband = 2;
        p.nval = 1;
        if (!(mat && get_double(mat, "n", p.mw_n) && get_double(mat, "v", p.mw_v) &&
              get_double(mat, "alphan", p.mw_alphan) && get_double(mat, "phi0", p.mw_phi0) &&
              get_double(mat, "a0", p.mw_a0)))
            throw CfgError("Some MultiWSM paramters are missing");
        p.mw_a0 /= AU_ANGSTROM;
        const double kmax = PI / p.mw_a0;
        const double axes[9] = {2 * kmax, 0, 0, 0, 2 * kmax, 0, 0, 0, 2 * kmax};
        for (int i = 0; i < 9; ++i) p.bzaxes[i] = axes[i];
        for (int i = 0; i < 3; ++i) p.bzorigin[i] = 0.0;
        if (custom)
            throw CfgError("Error: Try to using custom inital value without implementing GenInitialValue.");
    } else if (p.target == "WDSM_TaAs") {
        unsup("material '" + p.target + "' is not built on the GPU path");
        return p;
    } else {
        throw CfgError("Undefined Material");
    }
    // ksfactor scaling and BZ overrides (SBEs.h:221-241)
    for (int i = 0; i < 9; ++i) p.bz_model[i] = p.bzaxes[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) p.bzaxes[3 * i + j] *= p.ksfactor[i];
    if (const CfgValue *bz = calc->get("BZaxes"))
        for (size_t i = 0; i < bz->items.size() && i < 9; ++i)
            p.bzaxes[i] = elem_double(*bz, i, "Type exception in calc group");
    if (const CfgValue *bo = calc->get("BZorigin"))
        for (size_t i = 0; i < bo->items.size() && i < 3; ++i)
            p.bzorigin[i] = elem_double(*bo, i, "Type exception in calc group");
    p.derive_grid();

    if (p.laser.pulses.size() > 16) unsup("more than 16 laser pulses");
    if (p.gauge == GAUGE_LENGTH_HAMILTONIAN) unsup("gauge LengthHamiltonian is not implemented in the reference either");
    if (p.shot_number > 0 && p.shot_every() <= 0)   // the reference would take ktime % 0
        throw CfgError("calc.shotNumber gives a snapshot interval of 0 steps (period / shotNumber < dt)");
    if (p.rk == 45 && p.model == MODEL_HALDANE)
        unsup("adaptive Cash-Karp steps are built for the N-band (table) models only");
    return p;
}

// ================================================================= tables
std::vector<double> stage_fractions(int rk)
{
    if (rk == 4) return {0.0, 0.5, 1.0};                            // SBEs.h:398
    return {0.0, 0.25, 3. / 8., 12. / 13., 1.0, 0.5};               // SBEs.h:405
}

std::vector<double> a_table(const Problem &p)
{
    const auto c = stage_fractions(p.rk);
    const int nts = (int)c.size(), Nt = p.laser.Nt;
    std::vector<double> tab((size_t)Nt * nts * 2);
    double A[3];
    for (int n = 0; n < Nt; ++n) {
        const double t = p.laser.atmin + p.laser.dt * n;            // antelope.cpp:299
        for (int j = 0; j < nts; ++j) {
            p.laser.eval(j == 0 ? t : t + c[j] * p.laser.dt, A, nullptr);  // SBEs.h:612
            tab[((size_t)n * nts + j) * 2 + 0] = A[0];
            tab[((size_t)n * nts + j) * 2 + 1] = A[1];
        }
    }
    return tab;
}

std::vector<double> laser_rows(const Problem &p)
{
    const Laser &L = p.laser;
    std::vector<double> rows((size_t)L.Nt * 7);
    for (int n = 0; n < L.Nt; ++n) {
        double *r = &rows[(size_t)n * 7];
        r[0] = L.atmin + L.dt * n;  // antelope.cpp:215
        L.eval(r[0], r + 4, r + 1);
    }
    return rows;
}

std::vector<double> phase_table(const Problem &p, const std::vector<double> &atab)
{
    const size_t rows = atab.size() / 2;
    std::vector<double> ph(rows * 12);
    for (size_t r = 0; r < rows; ++r) {
        const double ax = atab[2 * r], ay = atab[2 * r + 1];
        for (int i = 0; i < 3; ++i) {
            const double aa = ax * p.hal_va[i][0] + ay * p.hal_va[i][1];
            const double ab = ax * p.hal_vb[i][0] + ay * p.hal_vb[i][1];
            ph[r * 12 + i] = std::cos(aa);
            ph[r * 12 + 3 + i] = std::sin(aa);
            ph[r * 12 + 6 + i] = std::cos(ab);
            ph[r * 12 + 9 + i] = std::sin(ab);
        }
    }
    return ph;
}

}  // namespace sbe
