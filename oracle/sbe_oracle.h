/* CPU oracle for the SBE time propagation: a plain-C restatement of the
 * reference algorithm (ftachacon/antelope, src/GeneralModel).  TEST
 * INFRASTRUCTURE ONLY: it is the checker that the CUDA product is compared
 * against, and the timed "port" CPU baseline.  Nothing in antelope_b200/
 * links, loads or calls it.
 *
 * Parity pin: tests/test_oracle_golden.py compares this restatement with
 * outputs of the unmodified reference compiled here (oracle/_ref, see
 * oracle/Makefile) on the committed golden cases in tests/golden/.  The one
 * third-party arithmetic dependency of the reference, LAPACK zheevr
 * (SBEs.h:289, SBEs.h:877), is replaced on both sides by a Jacobi solver; its
 * eigenvector phases are not pinned, which the written outputs do not depend
 * on (see oracle/refshim/lapacke.h).
 */
#ifndef SBE_ORACLE_H
#define SBE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_ENV_GAUSS = 0, ORC_ENV_GAUSS_CLIPPED = 1, ORC_ENV_COS4 = 2, ORC_ENV_COS4_CLIPPED = 3,
       ORC_ENV_SIN2 = 4 };
enum { ORC_GAUGE_LENGTH_WANNIER = 0, ORC_GAUGE_LENGTH_HAMILTONIAN = 1, ORC_GAUGE_VELOCITY = 2 };
enum { ORC_MODEL_HALDANE = 0, ORC_MODEL_WANNIER = 1, ORC_MODEL_MULTIWSM = 2 };
enum { ORC_RK4 = 4, ORC_RK5_FEHLBERG = 5, ORC_RK45_CASHKARP = 45 };

#define ORC_MAX_PULSES 8
#define ORC_MAX_BANDS 8

/* One laser pulse as written in the config file: angles in degrees
 * (converted as SBEs.h:531-537 does). */
typedef struct {
    double E0, w0, ellip, ncycles, cep_deg, t0, phix_deg, ncycles_clipped, thetaz_deg, phiz_deg;
    int env;
} orc_pulse;

typedef struct {
    int npulses;
    orc_pulse pulses[ORC_MAX_PULSES];
    double offset_before, offset_after;
    double dt, T1, T2;
    int rk;          /* ORC_RK4, ORC_RK5_FEHLBERG or ORC_RK45_CASHKARP */
    double rk_tol;   /* Cash-Karp only: max-norm error tolerance per step */
    int inter_intra; /* calc.InterIntra */
    int gauge;
    int Nk[3];
    double ksfactor[3];
    int n_bzaxes;    /* number of calc.BZaxes entries given (0 = none) */
    double bzaxes[9];
    int n_bzorigin;
    double bzorigin[3];
    int model;
    /* Haldane (Materials/Haldane.h): a0 in Angstrom, M0 absolute */
    double hal_a0_ang, hal_t1, hal_t2, hal_M0, hal_phi0;
    /* initial state: valence bands filled (default) or Fermi-Dirac at 300 K */
    int use_fermi;
    double Ef;
    /* Wannier tight-binding model: H(k) = sum_R h_R e^{i k.R},
     * D_a(k) = sum_R d_{a,R} e^{i k.R}, R = n1 a1 + n2 a2 (2-D lattice). */
    int w_nband, w_nval, w_nR;
    const int *w_R;      /* [nR][2] lattice coordinates (n1, n2) */
    double w_lat[4];     /* a1 = (w_lat[0], w_lat[1]), a2 = (w_lat[2], w_lat[3]) in bohr */
    const double *w_h;   /* [nR][N][N] complex, interleaved re/im */
    const double *w_d;   /* [nR][2][N][N] complex, interleaved re/im, or NULL for no dipoles */
    /* Table models of analytic materials: Cartesian vectors instead of
     * R = n1 a1 + n2 a2, the material's own current operator
     * J_a(k) = sum_v j_{a,v} e^{ik.v} (its GenJMatrix) instead of
     * -dH/dk + i[D, H], and the material's Brillouin-zone axes. */
    const double *w_vec; /* [nR][2] Cartesian vectors (bohr), or NULL */
    const double *w_j;   /* [nR][2][N][N] complex, interleaved re/im, or NULL */
    double w_bz[9];      /* used when w_vec != NULL */
    int nthreads;        /* k-range split as ParaRange (utility.h:104-115); 1 = sequential */
    /* MultiWSM (Materials/MultiWSM.h): the continuum two-band model with
     * B = (alphan |k_p|^n cos(n phi_k), alphan |k_p|^n sin(n phi_k), v k_z);
     * a0 in Angstrom (sets the Brillouin zone). */
    double mw_n, mw_v, mw_alphan, mw_a0_ang;
} orc_problem;

typedef struct {
    int Nt, nband, nval, ntotal;
    double atmin, dV, total_weight;
} orc_dims;

int orc_get_dims(const orc_problem *p, orc_dims *out);

/* Runs the whole propagation.  Outputs (caller-allocated):
 *   inter[Nt*3], intra[Nt*3]: the columns of interband_dipole_full_evol.dat and
 *     intraband_current_full_evol.dat, i.e. Re(sum_k w_k J(k,t)) * dV
 *     (antelope.cpp:522-527);
 *   dmi[Nt*N*N*2]: sum_k w_k rho_k(t), complex interleaved, NOT divided by
 *     Ntotal (antelope.cpp:326-333);
 *   steps_taken (Cash-Karp only, may be NULL): accepted RK steps.
 * Returns 0 on success, nonzero on a bad problem. */
int orc_run(const orc_problem *p, double *inter, double *intra, double *dmi, long *steps_taken);

/* Density snapshots (calc.shotNumber > 0, antelope.cpp:267-422): every
 * F = int(period0 / shot_number / dt) steps (period0 of the first pulse), after
 * the step n with n % F == 0:
 *   occ1d[nshots*N0]  occupation_1d_integration.dat: Re sum_k w_k rho'_cc over the
 *                     k with first index i, divided by Nk[1];
 *   nc[nshots*Ntotal] fisrt_conduction.dat: rho'_cc per k (each k's own value);
 *   pi[nshots*Ntotal*2] fisrt_coherence.dat: rho'[Nval][Nval-1] per k, complex;
 * rho' = rho (velocity gauge, band basis) or U^dag rho U at k + A(t_n) (length
 * gauge).  nshots = (Nt - 1) / F + 1.  orc_shot_dims returns -3 when F is 0
 * (the reference then takes ktime % 0). */
int orc_shot_dims(const orc_problem *p, int shot_number, int *every, int *nshots);
int orc_run_shots(const orc_problem *p, int shot_number, double *inter, double *intra, double *dmi,
                  long *steps_taken, double *occ1d, double *nc, double *pi);

/* Building blocks exported for unit tests. */
void orc_laser_eval(const orc_problem *p, double t, double *A3, double *E3);
int orc_kgrid(const orc_problem *p, double *k3, double *w);
int orc_model_hj(const orc_problem *p, const double *k3, double *H, double *J3);
int orc_eigh(int n, const double *a, double *w, double *v);
/* The Butcher tableau the propagator uses for `rk` (ORC_RK4, ORC_RK5_FEHLBERG,
 * ORC_RK45_CASHKARP): c[7], a[7*7] (row-major), b[7] (the weights that
 * advance the state) and bstar[7] (the embedded weights; zeros when the method
 * has none).  Returns the number of stages, or -1 for an unknown rk. */
int orc_tableau(int rk, double *c, double *a, double *b, double *bstar);

#ifdef __cplusplus
}
#endif
#endif
