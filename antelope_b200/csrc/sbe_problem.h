// Host-side problem description: the contents of an inputParam.cfg after the
// reference's defaults and checks (SBEs.h:125-241, 432-561; antelope.cpp:
// 90-152), plus the laser A(t)/E(t) evaluation of laser.h, in FP64.
#pragma once

#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace sbe {

// ---------------------------------------------------------------- config
// A parsed libconfig document.  Values keep their libconfig type so that the
// reference's strict typing (an integer is not a float) can be reproduced.
struct CfgValue {
    enum Type { None, Int, Int64, Float, String, Bool, Group, Array, List } type = None;
    std::string name;
    long long ival = 0;
    double fval = 0.0;
    bool bval = false;
    std::string sval;
    std::vector<std::unique_ptr<CfgValue>> items;

    const CfgValue *get(const std::string &key) const;  // group member or nullptr
    bool is_number() const { return type == Int || type == Int64 || type == Float; }
};

struct CfgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Parse libconfig text (groups, lists, arrays, scalars, comments).  Throws
// CfgError with "line N: message" on malformed input.
std::unique_ptr<CfgValue> parse_cfg(const std::string &text);

// ---------------------------------------------------------------- laser
enum Envelope { ENV_GAUSS = 0, ENV_GAUSS_CLIPPED = 1, ENV_COS4 = 2, ENV_COS4_CLIPPED = 3, ENV_SIN2 = 4 };

struct Pulse {
    // as given (angles converted to radians as SBEs.h:531-537)
    double E0, w0, ellip, ncycles, cep, t0, phix, ncycles_clipped, thetaz, phiz;
    int env;
    // derived (laser.h:73-140)
    double period0, E0x, E0y, A0x, A0y, twidth, twidth_clipped, envfactor;
    double xdir[3], ydir[3];
    void derive();
    double envelope(double t, bool derivative) const;
    void eval(double t, double *A, double *E) const;
};

struct Laser {
    std::vector<Pulse> pulses;
    double dt = 0.1, offset_before = 0.0, offset_after = 0.0;
    double atmin = 0.0, atmax = 0.0, init_A[3] = {0, 0, 0}, init_E[3] = {0, 0, 0};
    int Nt = 0;
    void initialize();                               // laser::Initialize (laser.h:278-298)
    void eval(double t, double *A, double *E) const;  // laser::avlaser/elaser (laser.h:301-322)
};

// ---------------------------------------------------------------- problem
enum Gauge { GAUGE_LENGTH_WANNIER = 0, GAUGE_LENGTH_HAMILTONIAN = 1, GAUGE_VELOCITY = 2 };
enum Model {
    MODEL_HALDANE = 0,
    MODEL_SYNTHETIC_WANNIER = 1,  // tight-binding tables given in the cfg
    MODEL_TB = 2,                 // an analytic material restated as tables (sbe_materials.cpp)
    MODEL_MULTIWSM = 3,           // the continuum two-band model of Materials/MultiWSM.h
};

struct Problem {
    std::string target;
    int gauge = GAUGE_LENGTH_WANNIER;
    bool gauge_given = true;
    Laser laser;
    double dt = 0.1, T1 = -1.0, T2 = -1.0;
    int rk = 5;               // 4, 5 (fixed-step Fehlberg) or 45 (adaptive Cash-Karp, extension)
    double rk_tol = 1e-8;
    bool inter_intra = false;
    int shot_number = 0, diagnostic = 0;
    int Nk[3] = {1, 1, 1};
    double ksfactor[3] = {1.0, 1.0, 1.0};
    double bzaxes[9] = {0}, bzorigin[3] = {0};
    double bz_model[9] = {0};  // the material's own axes, before ksfactor and calc.BZaxes
    int precision = 0;        // 0 = FP64 (plain), 1 = mixed FP32/FP64 (extension)
    int model = MODEL_HALDANE;
    int nband = 2, nval = 1;
    bool use_fermi = false;
    double Ef = 0.0;
    // Haldane (Materials/Haldane.h:46-84): a0 in bohr
    double hal_t1 = 0, hal_t2 = 0, hal_M0 = 0, hal_phi0 = 0, hal_a0 = 0;
    double hal_va[3][2] = {{0}}, hal_vb[3][2] = {{0}};
    // MultiWSM (Materials/MultiWSM.h:45-70): B = (alphan |k_p|^n cos(n phi),
    // alphan |k_p|^n sin(n phi), v k_z); a0 in bohr (sets the zone); phi0 is
    // read, as the reference reads it, and unused by its formulas
    double mw_n = 0, mw_v = 0, mw_alphan = 0, mw_phi0 = 0, mw_a0 = 0;
    // Synthetic Wannier model (N <= 8 bands): H(k) = sum_R h_R e^{ik.R},
    // D_a(k) = sum_R d_{a,R} e^{ik.R}, R = n1 a1 + n2 a2
    int w_nR = 0;
    double w_lat[4] = {0, 0, 0, 0};   // a1 = (w_lat[0], w_lat[1]), a2 = (w_lat[2], w_lat[3])
    std::vector<int> w_R;             // [nR][2] lattice coordinates (SyntheticWannier input)
    std::vector<double> w_vec;        // [nR][2] hopping vectors, Cartesian (bohr)
    std::vector<double> w_h;          // [nR][N][N] complex, interleaved
    std::vector<double> w_d;          // [nR][2][N][N] complex, interleaved (empty: no dipoles)
    std::vector<double> w_j;          // [nR][2][N][N] complex current-operator tables (empty:
                                      // J_a = -dH/dk_a + i[D_a, H], BaseMaterial.h:62-68)

    // density snapshots: steps between them (shotFrequency,
    // antelope.cpp:274-278) and how many the run takes; 0 when off
    int shot_every() const;
    int nshots() const;

    // derived grid quantities (momaxis.h:192-240)
    int ntotal() const { return Nk[0] * Nk[1] * Nk[2]; }
    double volume = 0.0, dV = 0.0, total_weight = 0.0;
    void derive_grid();
};

// Build a Problem from a parsed cfg.  Throws CfgError carrying the
// reference's own diagnostic for the condition (where it has one).
// `unsupported` is set instead of throwing when the input is valid for the
// reference but names something this library does not build.
// libconfig-typed lookups (no auto-conversion) and the material tables
bool get_double(const CfgValue *g, const char *key, double &v);
bool get_int(const CfgValue *g, const char *key, int &v);
bool get_bool(const CfgValue *g, const char *key, bool &v);
bool get_string(const CfgValue *g, const char *key, std::string &v);
// Fills nband, nval, the tables and the Brillouin zone for an analytic
// material of the reference; false if `target` is not one of them.
bool build_material(const std::string &target, const CfgValue *mat, Problem &p);
extern const double PI;           // constant.h:19
extern const double AU_ANGSTROM;  // constant.h:32

Problem problem_from_cfg(const CfgValue &root, std::string *unsupported);

// Stage-time tables for the kernels.
// c[]: distinct stage-time fractions of the RK tableau (0 first).
std::vector<double> stage_fractions(int rk);
// A(t) table [Nt][nts][2] (x, y) at t = (atmin + dt n) + c dt, FP64.
std::vector<double> a_table(const Problem &p);
// The columns of outlaserdata.dat, [Nt][7]: t_n, E(t_n), A(t_n)
// (antelope.cpp:208-235; laser.h:301-322).
std::vector<double> laser_rows(const Problem &p);
// Haldane length gauge: [Nt][nts][12] cos/sin of A.a_i and A.b_i.
std::vector<double> phase_table(const Problem &p, const std::vector<double> &atab);

}  // namespace sbe
