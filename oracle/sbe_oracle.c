/* CPU oracle for the SBE time propagation -- plain-C restatement of the
 * reference algorithm.  TEST INFRASTRUCTURE ONLY (the checker and the "port"
 * CPU baseline); the product never links or calls it.  See sbe_oracle.h.
 *
 * Every function names the reference lines it restates; paths are relative to
 * src/GeneralModel/ of ftachacon/antelope.
 */
#define _GNU_SOURCE
#include "sbe_oracle.h"

#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

static const double PI = 3.14159265358979323846;      /* constant.h:19 (4*atan(1)) */
static const double AU_ANGSTROM = 0.529177210903;     /* constant.h:32 */

/* ------------------------------------------------------------------ laser */
/* One pulse, as built by Pulse::Pulse (laser.h:68-141). */
typedef struct {
    double E0, w0, ellip, ncycles, cep, t0, phix, thetaz, phiz, ncycles_clipped;
    int env;
    double period0, E0x, E0y, A0x, A0y, twidth, twidth_clipped, envfactor;
    double xdir[3], ydir[3];
} pulse_t;

typedef struct {
    int n;
    pulse_t p[ORC_MAX_PULSES];
    double dt, atmin, atmax;
    double init_A[3], init_E[3];
    int Nt;
} laser_t;

static void pulse_build(pulse_t *q, const orc_pulse *c)
{
    /* degrees -> radians as SBEs::InitializeLaser (SBEs.h:531-537) */
    q->E0 = c->E0; q->w0 = c->w0; q->ellip = c->ellip; q->ncycles = c->ncycles;
    q->cep = c->cep_deg * PI / 180.0;
    q->t0 = c->t0;
    q->phix = c->phix_deg * PI / 180.0;
    q->thetaz = c->thetaz_deg * PI / 180.0;
    q->phiz = c->phiz_deg * PI / 180.0;
    q->ncycles_clipped = c->ncycles_clipped;
    q->env = c->env;
    q->period0 = 2.0 * PI / q->w0;                                  /* laser.h:75 */
    q->twidth_clipped = 0.0;
    switch (q->env) {                                               /* laser.h:88-113 */
    case ORC_ENV_GAUSS:
        q->twidth = 2.0 * q->ncycles * q->period0;
        q->envfactor = -4 * log(2) / (q->ncycles * q->period0 * q->ncycles * q->period0);
        break;
    case ORC_ENV_GAUSS_CLIPPED:
        q->twidth = 2.0 * q->ncycles * q->period0 + q->ncycles_clipped * q->period0 / 2;
        q->twidth_clipped = q->ncycles_clipped * q->period0 / 2;
        q->envfactor = -4 * log(2) / (q->ncycles * q->period0 * q->ncycles * q->period0);
        break;
    case ORC_ENV_COS4:
    case ORC_ENV_SIN2: /* extension: same support and argument scale as cos4 */
        q->twidth = q->ncycles * q->period0 / 2;
        q->envfactor = q->w0 / (2 * q->ncycles);
        break;
    case ORC_ENV_COS4_CLIPPED:
    default:
        q->twidth = (q->ncycles + q->ncycles_clipped) * q->period0 / 2;
        q->twidth_clipped = q->ncycles_clipped * q->period0 / 2;
        q->envfactor = q->w0 / (2 * q->ncycles);
        break;
    }
    double factor = sqrt(1.0 / (1.0 + q->ellip * q->ellip));       /* laser.h:116-127 */
    q->E0x = factor * q->E0;
    q->E0y = q->ellip * factor * q->E0;
    if (q->w0 > 1.0e-30) { q->A0x = q->E0x / q->w0; q->A0y = q->E0y / q->w0; }
    else { q->A0x = 0.; q->A0y = 0.; }
    double tx0[3] = {cos(q->thetaz) * cos(q->phiz), cos(q->thetaz) * sin(q->phiz), -sin(q->thetaz)};
    double ty0[3] = {-sin(q->phiz), cos(q->phiz), 0.};            /* laser.h:133-140 */
    for (int i = 0; i < 3; ++i) {
        q->xdir[i] = cos(q->phix) * tx0[i] + sin(q->phix) * ty0[i];
        q->ydir[i] = -sin(q->phix) * tx0[i] + cos(q->phix) * ty0[i];
    }
}

/* Pulse::f_envelope (laser.h:150-206), plus the sin2 extension
 * f = cos^2(t w0 / (2 N)) on |t| <= N T / 2. */
static double envelope(const pulse_t *q, double t, int dt_flag)
{
    double ef = q->envfactor, to;
    switch (q->env) {
    case ORC_ENV_COS4:
        if (fabs(t) > q->twidth) return 0;
        if (dt_flag) return -4. * ef * sin(t * ef) * pow(cos(t * ef), 3.);
        return pow(cos(t * ef), 4.);
    case ORC_ENV_SIN2:
        if (fabs(t) > q->twidth) return 0;
        if (dt_flag) return -2. * ef * sin(t * ef) * cos(t * ef);
        return cos(t * ef) * cos(t * ef);
    case ORC_ENV_COS4_CLIPPED:
        if (fabs(t) > q->twidth) return 0;
        if (t > q->twidth_clipped) to = t - q->twidth_clipped;
        else if (t > -q->twidth_clipped) return dt_flag ? 0. : 1.;
        else to = t + q->twidth_clipped;
        if (dt_flag) return -4. * ef * sin(to * ef) * pow(cos(to * ef), 3.);
        return pow(cos(to * ef), 4.);
    case ORC_ENV_GAUSS:
        if (dt_flag) return 2 * t * ef * exp(ef * t * t);
        return exp(ef * t * t);
    case ORC_ENV_GAUSS_CLIPPED:
    default:
        if (t > q->twidth_clipped) to = t - q->twidth_clipped;
        else if (t > -q->twidth_clipped) return dt_flag ? 0. : 1.;
        else to = t + q->twidth_clipped;
        if (dt_flag) return 2 * to * ef * exp(ef * to * to);
        return exp(ef * to * to);
    }
}

/* Pulse::avlaser / elaser (laser.h:209-238) */
static void pulse_AE(const pulse_t *q, double t, double *A, double *E)
{
    double kt = t - q->t0;
    double s = sin(kt * q->w0 - q->cep), c = cos(kt * q->w0 - q->cep);
    double f = envelope(q, kt, 0), fp = envelope(q, kt, 1);
    double ax = -q->A0x * s * f, ay = q->A0y * c * f;
    double ex = q->E0x * c * f - q->A0x * s * fp;
    double ey = q->E0y * s * f + q->A0y * c * fp;
    for (int i = 0; i < 3; ++i) {
        if (A) A[i] = ax * q->xdir[i] + ay * q->ydir[i];
        if (E) E[i] = ex * q->xdir[i] + ey * q->ydir[i];
    }
}

/* laser::avlaser / elaser (laser.h:301-322): sum of pulses minus the value at
 * atmin. */
static void laser_AE(const laser_t *L, double t, double *A, double *E)
{
    double a[3] = {0, 0, 0}, e[3] = {0, 0, 0}, pa[3], pe[3];
    for (int i = 0; i < L->n; ++i) {
        pulse_AE(&L->p[i], t, pa, pe);
        for (int d = 0; d < 3; ++d) { a[d] += pa[d]; e[d] += pe[d]; }
    }
    for (int d = 0; d < 3; ++d) {
        if (A) A[d] = a[d] - L->init_A[d];
        if (E) E[d] = e[d] - L->init_E[d];
    }
}

/* laser::Initialize (laser.h:278-298) */
static int laser_build(laser_t *L, const orc_problem *p)
{
    if (p->npulses < 1 || p->npulses > ORC_MAX_PULSES || !(p->dt > 0)) return -1;
    L->n = p->npulses;
    for (int i = 0; i < L->n; ++i) pulse_build(&L->p[i], &p->pulses[i]);
    double mn = L->p[0].t0 - L->p[0].twidth, mx = L->p[0].t0 + L->p[0].twidth;
    for (int i = 1; i < L->n; ++i) {
        if (L->p[i].t0 - L->p[i].twidth < mn) mn = L->p[i].t0 - L->p[i].twidth;
        if (L->p[i].t0 + L->p[i].twidth > mx) mx = L->p[i].t0 + L->p[i].twidth;
    }
    L->dt = p->dt;
    L->atmin = mn - p->offset_before;
    L->atmax = mx + p->offset_after;
    for (int d = 0; d < 3; ++d) { L->init_A[d] = 0; L->init_E[d] = 0; }
    double A0[3], E0[3];
    laser_AE(L, L->atmin, A0, E0);
    for (int d = 0; d < 3; ++d) { L->init_A[d] = A0[d]; L->init_E[d] = E0[d]; }
    L->Nt = (int)floor((L->atmax - L->atmin) / L->dt);
    return L->Nt > 0 ? 0 : -1;
}

/* ------------------------------------------------------------------ model */
typedef struct {
    int kind, N, nval, dipole;
    /* Haldane (Materials/Haldane.h:46-84, 134-143) */
    double t1, t2, M0, phi0, a0, va[3][2], vb[3][2];
    /* MultiWSM (Materials/MultiWSM.h:45-70) */
    double mw_n, mw_v, mw_alphan;
    /* Wannier */
    int nR;
    double (*Rc)[2];        /* Cartesian R vectors */
    const double *h, *d, *j; /* j: explicit current-operator tables or NULL */
    double bzaxes[9], bzorigin[3];
} model_t;

static int model_build(model_t *m, const orc_problem *p)
{
    memset(m, 0, sizeof(*m));
    m->kind = p->model;
    for (int i = 0; i < 9; ++i) m->bzaxes[i] = 0;
    if (p->model == ORC_MODEL_HALDANE) {
        m->N = 2; m->nval = 1; m->dipole = 0;
        m->t1 = p->hal_t1; m->t2 = p->hal_t2; m->M0 = p->hal_M0; m->phi0 = p->hal_phi0;
        m->a0 = p->hal_a0_ang / AU_ANGSTROM;
        double a0 = m->a0;
        m->va[0][0] = 0.;                 m->va[0][1] = a0;
        m->va[1][0] = -sqrt(3.) / 2 * a0; m->va[1][1] = -0.5 * a0;
        m->va[2][0] = sqrt(3.) / 2 * a0;  m->va[2][1] = -0.5 * a0;
        m->vb[0][0] = sqrt(3.) * a0;      m->vb[0][1] = 0.;
        m->vb[1][0] = -sqrt(3.) / 2 * a0; m->vb[1][1] = 3. / 2. * a0;
        m->vb[2][0] = -sqrt(3.) / 2 * a0; m->vb[2][1] = -3. / 2. * a0;
        double kxMax = PI / sqrt(3.) / a0, kyMax = 2. * PI / 3. / a0;   /* Haldane.h:77-81 */
        m->bzaxes[0] = 2 * kxMax; m->bzaxes[4] = 2 * kyMax;
        return 0;
    }
    if (p->model == ORC_MODEL_MULTIWSM) {   /* MultiWSM.h:45-70 */
        if (!(p->mw_a0_ang > 0)) return -1;
        m->N = 2; m->nval = 1; m->dipole = 0;
        m->mw_n = p->mw_n; m->mw_v = p->mw_v; m->mw_alphan = p->mw_alphan;
        m->a0 = p->mw_a0_ang / AU_ANGSTROM;
        double kmax = PI / m->a0;
        m->bzaxes[0] = 2 * kmax; m->bzaxes[4] = 2 * kmax; m->bzaxes[8] = 2 * kmax;
        return 0;
    }
    if (p->model == ORC_MODEL_WANNIER) {
        if (p->w_nband < 1 || p->w_nband > ORC_MAX_BANDS || p->w_nR < 1 || (!p->w_R && !p->w_vec) || !p->w_h)
            return -1;
        m->N = p->w_nband; m->nval = p->w_nval; m->dipole = p->w_d != NULL;
        m->nR = p->w_nR; m->h = p->w_h; m->d = p->w_d; m->j = p->w_j;
        m->Rc = malloc(sizeof(double[2]) * (size_t)m->nR);
        if (p->w_vec) {
            for (int r = 0; r < m->nR; ++r) { m->Rc[r][0] = p->w_vec[2 * r]; m->Rc[r][1] = p->w_vec[2 * r + 1]; }
            for (int i = 0; i < 9; ++i) m->bzaxes[i] = p->w_bz[i];
            return 0;
        }
        for (int r = 0; r < m->nR; ++r) {
            m->Rc[r][0] = p->w_R[2 * r] * p->w_lat[0] + p->w_R[2 * r + 1] * p->w_lat[2];
            m->Rc[r][1] = p->w_R[2 * r] * p->w_lat[1] + p->w_R[2 * r + 1] * p->w_lat[3];
        }
        /* reciprocal basis b_i . a_j = 2 pi delta_ij */
        double det = p->w_lat[0] * p->w_lat[3] - p->w_lat[1] * p->w_lat[2];
        m->bzaxes[0] = 2 * PI * p->w_lat[3] / det;  m->bzaxes[1] = -2 * PI * p->w_lat[2] / det;
        m->bzaxes[3] = -2 * PI * p->w_lat[1] / det; m->bzaxes[4] = 2 * PI * p->w_lat[0] / det;
        return 0;
    }
    return -1;
}

static void model_free(model_t *m) { free(m->Rc); }

/* Haldane::GenBcomp + GenHamiltonian (Haldane.h:86-92, 157-170) */
static void haldane_H(const model_t *m, const double *k, cplx *H)
{
    double B[4] = {0, 0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        double aa = k[0] * m->va[i][0] + k[1] * m->va[i][1];
        double ab = k[0] * m->vb[i][0] + k[1] * m->vb[i][1];
        B[0] += cos(ab); B[1] += cos(aa); B[2] += sin(aa); B[3] += sin(ab);
    }
    B[0] *= 2. * m->t2 * cos(m->phi0); B[1] *= m->t1;
    B[2] *= m->t1;                     B[3] = m->M0 - 2. * m->t2 * sin(m->phi0) * B[3];
    H[0] = B[0] + B[3]; H[1] = B[1] - I * B[2];
    H[2] = B[1] + I * B[2]; H[3] = B[0] - B[3];
}

/* Haldane::GenJMatrix (Haldane.h:94-127): J = -dH/dk, z component zero */
static void haldane_J(const model_t *m, const double *k, cplx *J /* [3][4] */)
{
    double xd[4] = {0, 0, 0, 0}, yd[4] = {0, 0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        double aa = k[0] * m->va[i][0] + k[1] * m->va[i][1];
        double ab = k[0] * m->vb[i][0] + k[1] * m->vb[i][1];
        xd[0] += m->vb[i][0] * sin(ab); yd[0] += m->vb[i][1] * sin(ab);
        xd[1] += m->va[i][0] * sin(aa); yd[1] += m->va[i][1] * sin(aa);
        xd[2] += m->va[i][0] * cos(aa); yd[2] += m->va[i][1] * cos(aa);
        xd[3] += m->vb[i][0] * cos(ab); yd[3] += m->vb[i][1] * cos(ab);
    }
    xd[0] *= -2. * m->t2 * cos(m->phi0); yd[0] *= -2. * m->t2 * cos(m->phi0);
    xd[1] *= -m->t1;                     yd[1] *= -m->t1;
    xd[2] *= m->t1;                      yd[2] *= m->t1;
    xd[3] *= -2. * m->t2 * sin(m->phi0); yd[3] *= -2. * m->t2 * sin(m->phi0);
    J[0] = -(xd[0] + xd[3]);     J[4 + 0] = -(yd[0] + yd[3]);
    J[1] = -(xd[1] - I * xd[2]); J[4 + 1] = -(yd[1] - I * yd[2]);
    J[2] = -(xd[1] + I * xd[2]); J[4 + 2] = -(yd[1] + I * yd[2]);
    J[3] = -(xd[0] - xd[3]);     J[4 + 3] = -(yd[0] - yd[3]);
    for (int i = 0; i < 4; ++i) J[8 + i] = 0;
}

/* Wannier model form (Materials/Wannier90.h:297-387, exact Fourier sums):
 * H = sum_R h_R e^{ikR}; D_a = sum_R d_aR e^{ikR};
 * J_a = -dH/dk_a + i[D_a, H] (BaseMaterial.h:62-68), or, for a material's
 * tables, J_a = sum_v j_{a,v} e^{ikv} (its GenJMatrix). */
static void wannier_HDJ(const model_t *m, const double *k, cplx *H, cplx *D, cplx *J)
{
    int N = m->N, NN = N * N;
    cplx dH[2][ORC_MAX_BANDS * ORC_MAX_BANDS];
    for (int i = 0; i < NN; ++i) {
        H[i] = 0;
        dH[0][i] = dH[1][i] = 0;
        if (D) D[i] = D[NN + i] = D[2 * NN + i] = 0;
    }
    for (int r = 0; r < m->nR; ++r) {
        double ph = k[0] * m->Rc[r][0] + k[1] * m->Rc[r][1];
        cplx e = cos(ph) + I * sin(ph);
        const double *hr = m->h + (size_t)r * NN * 2;
        for (int i = 0; i < NN; ++i) {
            cplx hv = (hr[2 * i] + I * hr[2 * i + 1]) * e;
            H[i] += hv;
            dH[0][i] += I * m->Rc[r][0] * hv;
            dH[1][i] += I * m->Rc[r][1] * hv;
        }
        if (D && m->d) {
            const double *dr = m->d + (size_t)r * 2 * NN * 2;
            for (int a = 0; a < 2; ++a)
                for (int i = 0; i < NN; ++i)
                    D[a * NN + i] += (dr[2 * (a * NN + i)] + I * dr[2 * (a * NN + i) + 1]) * e;
        }
    }
    if (J && m->j) {
        for (int i = 0; i < 3 * NN; ++i) J[i] = 0;
        for (int r = 0; r < m->nR; ++r) {
            double ph = k[0] * m->Rc[r][0] + k[1] * m->Rc[r][1];
            cplx e = cos(ph) + I * sin(ph);
            const double *jr = m->j + (size_t)r * 2 * NN * 2;
            for (int a = 0; a < 2; ++a)
                for (int i = 0; i < NN; ++i)
                    J[a * NN + i] += (jr[2 * (a * NN + i)] + I * jr[2 * (a * NN + i) + 1]) * e;
        }
    } else if (J) {
        for (int a = 0; a < 2; ++a)
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j) {
                    cplx v = -dH[a][i * N + j];
                    if (D && m->d) {
                        cplx c = 0;
                        for (int l = 0; l < N; ++l)
                            c += D[a * NN + i * N + l] * H[l * N + j] - H[i * N + l] * D[a * NN + l * N + j];
                        v += I * c;
                    }
                    J[a * NN + i * N + j] = v;
                }
        for (int i = 0; i < NN; ++i) J[2 * NN + i] = 0;
    }
}

/* MultiWSM::GenBcomp + GenHamiltonian (MultiWSM.h:76-82, 186-200) */
static void multiwsm_H(const model_t *m, const double *k, cplx *H)
{
    const double n = m->mw_n, al = m->mw_alphan;
    double B[4];
    B[0] = 0.;
    B[1] = al * pow(k[0] * k[0] + k[1] * k[1], n / 2.) * cos(n * atan2(k[1], k[0]));
    B[2] = al * pow(k[0] * k[0] + k[1] * k[1], n / 2.) * sin(n * atan2(k[1], k[0]));
    B[3] = m->mw_v * k[2];
    H[0] = B[0] + B[3]; H[1] = B[1] - I * B[2];
    H[2] = B[1] + I * B[2]; H[3] = B[0] - B[3];
}

/* MultiWSM::GenJMatrix (MultiWSM.h:84-147), the derivative of B as written
 * there (it is undefined on the k_x = k_y = 0 line) */
static void multiwsm_J(const model_t *m, const double *k, cplx *J /* [3][4] */)
{
    const double n = m->mw_n, al = m->mw_alphan;
    const double phip = atan2(k[1], k[0]);
    const double psq = k[0] * k[0] + k[1] * k[1];
    double xd[4] = {0, 0, 0, 0}, yd[4] = {0, 0, 0, 0}, zd[4] = {0, 0, 0, 0};
    xd[1] = n * al * k[0] * cos(n * phip) * pow(psq, n / 2. - 1) + n * al * sin(n * phip) * pow(psq, n / 2.) * k[1] / psq;
    yd[1] = n * al * k[1] * cos(n * phip) * pow(psq, n / 2. - 1) - n * al * sin(n * phip) * pow(psq, n / 2.) * k[0] / psq;
    xd[2] = +n * al * k[0] * sin(n * phip) * pow(psq, n / 2. - 1) - n * al * k[1] * cos(n * phip) * pow(psq, n / 2.) / psq;
    yd[2] = +n * al * k[1] * sin(n * phip) * pow(psq, n / 2. - 1) + n * al * k[0] * cos(n * phip) * pow(psq, n / 2.) / psq;
    zd[3] = m->mw_v;
    const double *d[3] = {xd, yd, zd};
    for (int a = 0; a < 3; ++a) {
        J[4 * a + 0] = -(d[a][0] + d[a][3]);
        J[4 * a + 1] = -(d[a][1] - I * d[a][2]);
        J[4 * a + 2] = -(d[a][1] + I * d[a][2]);
        J[4 * a + 3] = -(d[a][0] - d[a][3]);
    }
}

static void model_H(const model_t *m, const double *k, cplx *H)
{
    if (m->kind == ORC_MODEL_HALDANE) haldane_H(m, k, H);
    else if (m->kind == ORC_MODEL_MULTIWSM) multiwsm_H(m, k, H);
    else wannier_HDJ(m, k, H, NULL, NULL);
}
static void model_J(const model_t *m, const double *k, cplx *J)
{
    if (m->kind == ORC_MODEL_HALDANE) { haldane_J(m, k, J); return; }
    if (m->kind == ORC_MODEL_MULTIWSM) { multiwsm_J(m, k, J); return; }
    cplx H[ORC_MAX_BANDS * ORC_MAX_BANDS], D[3 * ORC_MAX_BANDS * ORC_MAX_BANDS];
    wannier_HDJ(m, k, H, D, J);
}
static void model_D(const model_t *m, const double *k, cplx *D)
{
    cplx H[ORC_MAX_BANDS * ORC_MAX_BANDS];
    wannier_HDJ(m, k, H, D, NULL);
}

/* ------------------------------------------------------- linear algebra */
/* MatrixMult (utility.h:79-98): out = A B, row-major, zero-initialised */
static void matmul(cplx *out, const cplx *A, const cplx *B, int n)
{
    for (int i = 0; i < n * n; ++i) out[i] = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int l = 0; l < n; ++l) out[i * n + j] += A[i * n + l] * B[l * n + j];
}

/* Hermitian eigen-decomposition standing in for LAPACKE_zheevr(ROW_MAJOR,
 * 'V', 'A', 'U') at SBEs.h:289 and SBEs.h:877: reads the upper triangle,
 * returns ascending eigenvalues and unit eigenvectors in columns.  Cyclic
 * complex Jacobi rotations. */
static void eigh(int n, const cplx *Ain, double *w, cplx *U)
{
    cplx A[ORC_MAX_BANDS * ORC_MAX_BANDS], V[ORC_MAX_BANDS * ORC_MAX_BANDS];
    for (int i = 0; i < n; ++i) {
        A[i * n + i] = creal(Ain[i * n + i]);
        for (int j = i + 1; j < n; ++j) { A[i * n + j] = Ain[i * n + j]; A[j * n + i] = conj(Ain[i * n + j]); }
        for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1.0 : 0.0;
    }
    double scale = 0;
    for (int i = 0; i < n * n; ++i) scale += creal(A[i] * conj(A[i]));
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += creal(A[p * n + q] * conj(A[p * n + q]));
        if (off == 0.0 || off <= 1e-34 * scale) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double r = cabs(A[p * n + q]);
                if (r == 0.0) continue;
                cplx e = A[p * n + q] / r;
                double app = creal(A[p * n + p]), aqq = creal(A[q * n + q]);
                double zeta = (aqq - app) / (2.0 * r);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(zeta * zeta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                cplx Jpp = c, Jpq = s, Jqp = -s * conj(e), Jqq = c * conj(e);
                for (int k = 0; k < n; ++k) {
                    cplx akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = akp * Jpp + akq * Jqp;
                    A[k * n + q] = akp * Jpq + akq * Jqq;
                    cplx vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = vkp * Jpp + vkq * Jqp;
                    V[k * n + q] = vkp * Jpq + vkq * Jqq;
                }
                for (int k = 0; k < n; ++k) {
                    cplx apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = conj(Jpp) * apk + conj(Jqp) * aqk;
                    A[q * n + k] = conj(Jpq) * apk + conj(Jqq) * aqk;
                }
                A[p * n + q] = 0; A[q * n + p] = 0;
                A[p * n + p] = creal(A[p * n + p]); A[q * n + q] = creal(A[q * n + q]);
            }
    }
    int order[ORC_MAX_BANDS];
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int i = 1; i < n; ++i) {
        int k = order[i], j = i - 1;
        while (j >= 0 && creal(A[order[j] * n + order[j]]) > creal(A[k * n + k])) { order[j + 1] = order[j]; --j; }
        order[j + 1] = k;
    }
    for (int j = 0; j < n; ++j) {
        w[j] = creal(A[order[j] * n + order[j]]);
        for (int i = 0; i < n; ++i) U[i * n + j] = V[i * n + order[j]];
    }
}

static void dagger(cplx *out, const cplx *U, int n)
{
    for (int m = 0; m < n; ++m)
        for (int k = 0; k < n; ++k) out[m * n + k] = conj(U[k * n + m]);
}

/* ------------------------------------------------------------------ grid */
typedef struct {
    int N[3], Ntotal;
    double axes[9], origin[3], Volume, dV;
} grid_t;

/* SBEs ctor BZ set-up (SBEs.h:219-241) + momaxis::steps_sizes
 * (momaxis.h:192-240) */
static int grid_build(grid_t *g, const orc_problem *p, const model_t *m)
{
    for (int i = 0; i < 3; ++i) g->N[i] = p->Nk[i] > 0 ? p->Nk[i] : 1;
    for (int i = 0; i < 9; ++i) g->axes[i] = m->bzaxes[i];
    for (int i = 0; i < 3; ++i) g->origin[i] = m->bzorigin[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) g->axes[3 * i + j] *= p->ksfactor[i];
    for (int i = 0; i < p->n_bzaxes && i < 9; ++i) g->axes[i] = p->bzaxes[i];
    for (int i = 0; i < p->n_bzorigin && i < 3; ++i) g->origin[i] = p->bzorigin[i];
    g->Ntotal = g->N[0] * g->N[1] * g->N[2];
    double ax[3][3];
    int na = 0;
    for (int i = 0; i < 3; ++i)
        if (g->N[i] != 1) { for (int j = 0; j < 3; ++j) ax[na][j] = g->axes[3 * i + j]; ++na; }
    double c[3];
    switch (na) {
    case 1: g->Volume = sqrt(ax[0][0] * ax[0][0] + ax[0][1] * ax[0][1] + ax[0][2] * ax[0][2]); break;
    case 2:
    case 3:
        c[0] = ax[0][1] * ax[1][2] - ax[0][2] * ax[1][1];   /* CrossProduct, utility.h:66-69 */
        c[1] = ax[0][2] * ax[1][0] - ax[0][0] * ax[1][2];
        c[2] = ax[0][0] * ax[1][1] - ax[1][0] * ax[0][1];
        if (na == 2) g->Volume = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        else g->Volume = sqrt(c[0] * ax[2][0] + c[1] * ax[2][1] + c[2] * ax[2][2]); /* momaxis.h:228 as written */
        break;
    default: g->Volume = 1.; break;
    }
    g->dV = fabs(g->Volume) / g->Ntotal;
    return 0;
}

/* momaxis::set_brillouin_zone_grid (momaxis.h:349-383) and basic_mem
 * (momaxis.h:147-186): inclusive endpoints, trapezoid weights */
static void grid_point(const grid_t *g, int idx, double *k, double *w)
{
    int i = idx / (g->N[1] * g->N[2]), j = (idx / g->N[2]) % g->N[1], l = idx % g->N[2];
    double f[3];
    int ii[3] = {i, j, l};
    double wt = 1.0;
    for (int d = 0; d < 3; ++d) {
        f[d] = (g->N[d] == 1) ? 0. : (double)ii[d] / (g->N[d] - 1) - 0.5;
        if (g->N[d] != 1 && (ii[d] == 0 || ii[d] == g->N[d] - 1)) wt /= 2;
    }
    for (int d = 0; d < 3; ++d)
        k[d] = g->origin[d] + f[0] * g->axes[0 * 3 + d] + f[1] * g->axes[1 * 3 + d] + f[2] * g->axes[2 * 3 + d];
    if (w) *w = wt;
}

/* -------------------------------------------------------------- tableaus */
typedef struct {
    int stages;
    double c[7], b[7], a[7][7], bstar[7];
    int adaptive;
} tableau_t;

/* SBEs.h:395-416 (RK4, Fehlberg-5 weights) and the published Cash-Karp
 * 4(5) pair (extension for the adaptive Wannier runs). */
static int tableau_build(tableau_t *T, int rk)
{
    memset(T, 0, sizeof(*T));
    if (rk == ORC_RK4) {
        T->stages = 4;
        T->c[1] = 0.5; T->c[2] = 0.5; T->c[3] = 1.0;
        T->b[0] = 1.0 / 6.0; T->b[1] = 2.0 / 6.0; T->b[2] = 2.0 / 6.0; T->b[3] = 1.0 / 6.0;
        T->a[1][0] = 0.5;
        T->a[2][0] = 0.0; T->a[2][1] = 0.5;
        T->a[3][0] = 0.0; T->a[3][1] = 0.0; T->a[3][2] = 1.0;
        return 0;
    }
    if (rk == ORC_RK5_FEHLBERG) {
        T->stages = 6;
        T->c[1] = 0.25; T->c[2] = 3. / 8.; T->c[3] = 12. / 13.; T->c[4] = 1.0; T->c[5] = 0.5;
        T->b[0] = 16. / 135.; T->b[1] = 0; T->b[2] = 6656. / 12825.; T->b[3] = 28561. / 56430.;
        T->b[4] = -9. / 50.; T->b[5] = 2. / 55.;
        T->a[1][0] = 1.0 / 4.0;
        T->a[2][0] = 3. / 32.; T->a[2][1] = 9. / 32.;
        T->a[3][0] = 1932. / 2197.; T->a[3][1] = -7200. / 2197.; T->a[3][2] = 7296. / 2197.;
        T->a[4][0] = 439. / 216.; T->a[4][1] = -8.; T->a[4][2] = 3680. / 513.; T->a[4][3] = -845. / 4104.;
        T->a[5][0] = -8. / 27.; T->a[5][1] = 2.; T->a[5][2] = -3544. / 2565; T->a[5][3] = 1859. / 4104;
        T->a[5][4] = -11. / 40.;
        return 0;
    }
    if (rk == ORC_RK45_CASHKARP) {
        T->stages = 6; T->adaptive = 1;
        T->c[1] = 1. / 5.; T->c[2] = 3. / 10.; T->c[3] = 3. / 5.; T->c[4] = 1.; T->c[5] = 7. / 8.;
        T->a[1][0] = 1. / 5.;
        T->a[2][0] = 3. / 40.; T->a[2][1] = 9. / 40.;
        T->a[3][0] = 3. / 10.; T->a[3][1] = -9. / 10.; T->a[3][2] = 6. / 5.;
        T->a[4][0] = -11. / 54.; T->a[4][1] = 5. / 2.; T->a[4][2] = -70. / 27.; T->a[4][3] = 35. / 27.;
        T->a[5][0] = 1631. / 55296.; T->a[5][1] = 175. / 512.; T->a[5][2] = 575. / 13824.;
        T->a[5][3] = 44275. / 110592.; T->a[5][4] = 253. / 4096.;
        T->b[0] = 37. / 378.; T->b[2] = 250. / 621.; T->b[3] = 125. / 594.; T->b[5] = 512. / 1771.;
        T->bstar[0] = 2825. / 27648.; T->bstar[2] = 18575. / 48384.; T->bstar[3] = 13525. / 55296.;
        T->bstar[4] = 277. / 14336.; T->bstar[5] = 1. / 4.;
        return 0;
    }
    return -1;
}

/* ------------------------------------------------------------ propagator */
#define MAXNN (ORC_MAX_BANDS * ORC_MAX_BANDS)

typedef struct {
    const orc_problem *p;
    const laser_t *L;
    const model_t *m;
    const grid_t *g;
    const tableau_t *T;
    double gam_inter, gam_intra;
    int N, gauge, k0, k1, Nt;
    /* per-k state owned by this worker */
    cplx *rho, *init, *P; /* [nk][NN], [nk][NN], [nk][3][NN] */
    double *eps;          /* [nk][N] */
    double *kpt, *wgt;    /* [nk][3], [nk] */
    /* outputs (partials of this worker) */
    double *inter, *intra; /* [Nt][3] */
    cplx *dmi;             /* [Nt][NN] */
    long steps;
    int err;
    /* density snapshots (antelope.cpp:340-422): every shot_every steps */
    int shot_every;
    double *occ1d;         /* this worker's partial sums [nshots][N0] */
    double *nc;            /* [nshots][Ntotal], shared, written at global k */
    double *pi;            /* [nshots][Ntotal][2], shared */
} worker_t;

/* SBEs::GenDifferentialDM (SBEs.h:762-872) */
static void rhs(const worker_t *W, int kl, double t, const cplx *in, cplx *out)
{
    int N = W->N, NN = N * N;
    double A[3], E[3];
    laser_AE(W->L, t, A, E);
    const double *k = W->kpt + 3 * kl;
    double kt[3] = {k[0] + A[0], k[1] + A[1], k[2] + A[2]};   /* GenKpulsA, SBEs.h:900-925 */
    cplx H[MAXNN], tmp1[MAXNN], tmp2[MAXNN], U[MAXNN], Uh[MAXNN];
    double ev[ORC_MAX_BANDS];
    if (W->gauge == ORC_GAUGE_LENGTH_WANNIER) {
        model_H(W->m, kt, H);
        if (W->m->dipole) {
            cplx D[3 * MAXNN];
            model_D(W->m, kt, D);
            for (int i = 0; i < NN; ++i) H[i] += (E[0] * D[i] + E[1] * D[NN + i] + E[2] * D[2 * NN + i]);
        }
        matmul(out, H, in, N);
    } else {
        const cplx *P = W->P + (size_t)kl * 3 * NN;
        for (int i = 0; i < NN; ++i) {
            tmp1[i] = 0;
            for (int a = 0; a < 3; ++a) tmp1[i] += A[a] * P[a * NN + i];
        }
        for (int i = 0; i < N; ++i) tmp1[i * N + i] += W->eps[kl * N + i];
        matmul(out, tmp1, in, N);
    }
    for (int i = 0; i < NN; ++i) H[i] = out[i];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            out[i * N + j] -= conj(H[j * N + i]);
            out[i * N + j] *= -I;
        }
    if (W->gauge == ORC_GAUGE_LENGTH_WANNIER) {
        cplx H0[MAXNN];
        model_H(W->m, kt, H0);
        eigh(N, H0, ev, U);
        dagger(Uh, U, N);
        matmul(tmp1, in, U, N);
        matmul(tmp2, Uh, tmp1, N);
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) tmp2[i * N + j] *= (i == j) ? W->gam_intra : W->gam_inter;
        matmul(tmp1, U, tmp2, N);
        matmul(tmp2, tmp1, Uh, N);
        for (int i = 0; i < NN; ++i) out[i] -= tmp2[i];
    } else {
        const cplx *init = W->init + (size_t)kl * NN;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j)
                out[i * N + j] -= (in[i * N + j] - init[i * N + j]) * ((i == j) ? W->gam_intra : W->gam_inter);
    }
}

/* SBEs::GenInterIntraCurrent (SBEs.h:694-760) and GenCurrent (626-693) */
static void current(const worker_t *W, int kl, double t, double *jinter, double *jintra)
{
    int N = W->N, NN = N * N;
    double A[3];
    laser_AE(W->L, t, A, NULL);
    const double *k = W->kpt + 3 * kl;
    double kt[3] = {k[0], k[1], k[2]};
    if (W->gauge != ORC_GAUGE_VELOCITY) { kt[0] += A[0]; kt[1] += A[1]; kt[2] += A[2]; }
    const cplx *rho = W->rho + (size_t)kl * NN;
    cplx J[3 * MAXNN], U[MAXNN], Uh[MAXNN], H0[MAXNN], tmp1[MAXNN], tmp2[MAXNN], rh[MAXNN];
    double ev[ORC_MAX_BANDS];
    for (int a = 0; a < 3; ++a) jinter[a] = jintra[a] = 0;
    if (W->gauge == ORC_GAUGE_VELOCITY) {
        /* U(k) is the init-time eigenbasis, so U^dag J U is the stored P */
        const cplx *P = W->P + (size_t)kl * 3 * NN;
        for (int a = 0; a < 3; ++a)
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j) {
                    double v = creal(rho[i * N + j] * P[a * NN + j * N + i]);
                    if (!W->p->inter_intra || i != j) jinter[a] += v;
                    else jintra[a] += v;
                }
        if (W->p->inter_intra)
            for (int a = 0; a < 3; ++a) jintra[a] += W->m->nval * A[a];
        else
            for (int a = 0; a < 3; ++a) jinter[a] += W->m->nval * A[a];
        return;
    }
    model_J(W->m, kt, J);
    if (!W->p->inter_intra) {   /* GenCurrent, LengthWannier branch (SBEs.h:644-657) */
        for (int a = 0; a < 3; ++a)
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j) jinter[a] += creal(rho[N * i + j] * J[a * NN + N * j + i]);
        return;
    }
    model_H(W->m, kt, H0);
    eigh(N, H0, ev, U);
    dagger(Uh, U, N);
    matmul(tmp1, rho, U, N);
    matmul(rh, Uh, tmp1, N);
    for (int a = 0; a < 3; ++a) {
        matmul(tmp1, J + a * NN, U, N);
        matmul(tmp2, Uh, tmp1, N);
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                double v = creal(rh[N * i + j] * tmp2[N * j + i]);
                if (i == j) jintra[a] += v;
                else jinter[a] += v;
            }
    }
}

/* SBEs ctor per-k initialisation (SBEs.h:284-373) */
static void init_k(worker_t *W, int kl)
{
    int N = W->N, NN = N * N;
    double *k = W->kpt + 3 * kl;
    cplx H[MAXNN], U[MAXNN], Uh[MAXNN], tmp[MAXNN], J[3 * MAXNN];
    double *ev = W->eps + (size_t)kl * N;
    model_H(W->m, k, H);
    eigh(N, H, ev, U);
    dagger(Uh, U, N);
    cplx *rho = W->rho + (size_t)kl * NN;
    for (int i = 0; i < NN; ++i) rho[i] = 0;
    if (W->p->use_fermi) {
        const double thermalE = 300. / 3.15775024804e5;
        double f[ORC_MAX_BANDS], s = 0;
        for (int i = 0; i < N; ++i) { f[i] = 1.0 / (exp((ev[i] - W->p->Ef) / thermalE) + 1.0); s += f[i]; }
        for (int i = 0; i < N; ++i) rho[i * N + i] = f[i] / s;
    } else {
        for (int i = 0; i < N; ++i)
            if (i < W->m->nval) rho[i * N + i] = 1.0;
    }
    if (W->gauge == ORC_GAUGE_LENGTH_WANNIER) {
        matmul(tmp, rho, Uh, N);
        matmul(rho, U, tmp, N);
    }
    for (int i = 0; i < NN; ++i) W->init[(size_t)kl * NN + i] = rho[i];
    model_J(W->m, k, J);
    for (int a = 0; a < 3; ++a) {
        matmul(tmp, J + a * NN, U, N);
        matmul(W->P + ((size_t)kl * 3 + a) * NN, Uh, tmp, N);
    }
}

/* Snapshot of step n (antelope.cpp:340-422), taken after every k of the
 * worker has advanced past t_n.  The conduction occupation rho'[Nval][Nval]
 * and the coherence rho'[Nval][Nval-1] are read from rho' = rho in the band
 * basis (velocity gauge) or rho' = U^dag rho U with U the eigenvectors of
 * H0(k + A(t_n)) (length gauge: SBEs::WannierToHamiltonian, SBEs.h:927-940,
 * evaluated at the time of the step's start, as the reference calls it).
 * The 1-D integration adds w rho'_cc into the bin of the first k index
 * (antelope.cpp:343-370).  The per-k values are stored at each k's own index:
 * the reference's own loop (antelope.cpp:384-400) indexes them with a stale
 * k index, so its binary files hold one k-point's value (velocity gauge) or
 * unset memory (length gauge) everywhere but at the last k of each rank. */
static void snapshot(worker_t *W, int n)
{
    int N = W->N, NN = N * N, nk = W->k1 - W->k0, nv = W->m->nval;
    const grid_t *g = W->g;
    int shot = n / W->shot_every;
    double t = W->L->atmin + W->L->dt * n, A[3];
    laser_AE(W->L, t, A, NULL);
    for (int kl = 0; kl < nk; ++kl) {
        const cplx *rho = W->rho + (size_t)kl * NN;
        cplx r[MAXNN];
        if (W->gauge == ORC_GAUGE_LENGTH_WANNIER) {
            const double *k = W->kpt + 3 * kl;
            double kt[3] = {k[0] + A[0], k[1] + A[1], k[2] + A[2]};
            cplx H0[MAXNN], U[MAXNN], Uh[MAXNN], tmp[MAXNN];
            double ev[ORC_MAX_BANDS];
            model_H(W->m, kt, H0);
            eigh(N, H0, ev, U);
            dagger(Uh, U, N);
            matmul(tmp, rho, U, N);
            matmul(r, Uh, tmp, N);
        } else {
            memcpy(r, rho, sizeof(cplx) * NN);
        }
        int kg = W->k0 + kl;
        double cc = creal(r[nv * N + nv]);
        cplx cv = r[nv * N + nv - 1];
        W->occ1d[(size_t)shot * g->N[0] + kg / (g->N[1] * g->N[2])] += cc * W->wgt[kl];
        W->nc[(size_t)shot * g->Ntotal + kg] = cc;
        W->pi[2 * ((size_t)shot * g->Ntotal + kg)] = creal(cv);
        W->pi[2 * ((size_t)shot * g->Ntotal + kg) + 1] = cimag(cv);
    }
}

/* SBEs::RunSBEs (SBEs.h:596-624) for one k and one step of size h */
static void rk_step(const worker_t *W, int kl, double t, double h, cplx *rho, cplx *errv)
{
    int N = W->N, NN = N * N, S = W->T->stages;
    cplx k[7][MAXNN], y[MAXNN];
    rhs(W, kl, t, rho, k[0]);
    for (int s = 1; s < S; ++s) {
        for (int i = 0; i < NN; ++i) {
            y[i] = rho[i];
            for (int j = 0; j < s; ++j) y[i] += h * W->T->a[s][j] * k[j][i];
        }
        rhs(W, kl, t + W->T->c[s] * h, y, k[s]);
    }
    if (errv)
        for (int i = 0; i < NN; ++i) {
            errv[i] = 0;
            for (int s = 0; s < S; ++s) errv[i] += h * (W->T->b[s] - W->T->bstar[s]) * k[s][i];
        }
    for (int i = 0; i < NN; ++i)
        for (int s = 0; s < S; ++s) rho[i] += h * W->T->b[s] * k[s][i];
}

/* The driver's time loop (antelope.cpp:297-338): the currents and the
 * weighted density matrix at t_n are accumulated BEFORE rho advances. */
static void *worker_run(void *arg)
{
    worker_t *W = (worker_t *)arg;
    int N = W->N, NN = N * N, nk = W->k1 - W->k0;
    for (int kl = 0; kl < nk; ++kl) {
        grid_point(W->g, W->k0 + kl, W->kpt + 3 * kl, W->wgt + kl);
        init_k(W, kl);
    }
    double ji[3], ja[3];
    for (int n = 0; n < W->Nt; ++n) {
        double t = W->L->atmin + W->L->dt * n;
        for (int kl = 0; kl < nk; ++kl) {
            double w = W->wgt[kl];
            current(W, kl, t, ji, ja);
            for (int a = 0; a < 3; ++a) {
                W->intra[n * 3 + a] += ja[a] * w;
                W->inter[n * 3 + a] += ji[a] * w;
            }
            cplx *rho = W->rho + (size_t)kl * NN;
            for (int i = 0; i < NN; ++i) W->dmi[(size_t)n * NN + i] += rho[i] * w;
            rk_step(W, kl, t, W->L->dt, rho, NULL);
        }
        if (W->shot_every > 0 && n % W->shot_every == 0) snapshot(W, n);
    }
    W->steps = W->Nt;
    return NULL;
}

/* Adaptive Cash-Karp variant (extension, no reference counterpart): one step
 * size shared by all k of the solve, chosen from the max-norm error estimate
 * reduced over k; steps never cross an output time t_n = atmin + n dt, so the
 * currents land on the same time axis as the fixed-step runs.  Sequential
 * over k only (the shared step size couples all k). */
static int run_adaptive(worker_t *W)
{
    int N = W->N, NN = N * N, nk = W->k1 - W->k0;
    for (int kl = 0; kl < nk; ++kl) {
        grid_point(W->g, W->k0 + kl, W->kpt + 3 * kl, W->wgt + kl);
        init_k(W, kl);
    }
    cplx *trial = malloc(sizeof(cplx) * (size_t)nk * NN);
    cplx err[MAXNN];
    double ji[3], ja[3], tol = W->p->rk_tol > 0 ? W->p->rk_tol : 1e-8;
    double h = W->L->dt;
    long steps = 0;
    for (int n = 0; n < W->Nt; ++n) {
        double t = W->L->atmin + W->L->dt * n;
        for (int kl = 0; kl < nk; ++kl) {
            double w = W->wgt[kl];
            current(W, kl, t, ji, ja);
            for (int a = 0; a < 3; ++a) {
                W->intra[n * 3 + a] += ja[a] * w;
                W->inter[n * 3 + a] += ji[a] * w;
            }
            for (int i = 0; i < NN; ++i) W->dmi[(size_t)n * NN + i] += W->rho[(size_t)kl * NN + i] * w;
        }
        double tend = W->L->atmin + W->L->dt * (n + 1), tc = t;
        int guard = 0;
        while (tc < tend && guard++ < 100000) {
            double hs = h;
            int last = 0;
            if (tc + hs >= tend - 1e-12 * W->L->dt) { hs = tend - tc; last = 1; }
            double emax = 0;
            for (int kl = 0; kl < nk; ++kl) {
                cplx *y = trial + (size_t)kl * NN;
                memcpy(y, W->rho + (size_t)kl * NN, sizeof(cplx) * NN);
                rk_step(W, kl, tc, hs, y, err);
                for (int i = 0; i < NN; ++i) {
                    double e = cabs(err[i]);
                    if (e > emax) emax = e;
                }
            }
            if (emax <= tol) {
                memcpy(W->rho, trial, sizeof(cplx) * (size_t)nk * NN);
                tc = last ? tend : tc + hs;
                ++steps;
                double fac = emax > 0 ? 0.9 * pow(tol / emax, 0.2) : 5.0;
                if (fac > 5.0) fac = 5.0;
                if (!last || fac < 1.0) h = hs * (fac < 0.2 ? 0.2 : fac);
                if (h > W->L->dt) h = W->L->dt;
            } else {
                double fac = 0.9 * pow(tol / emax, 0.25);
                h = hs * (fac < 0.1 ? 0.1 : fac);
            }
        }
        if (guard >= 100000) { free(trial); return -1; }
        if (W->shot_every > 0 && n % W->shot_every == 0) snapshot(W, n);
    }
    W->steps = steps;
    free(trial);
    return 0;
}

/* ------------------------------------------------------------- public API */
int orc_get_dims(const orc_problem *p, orc_dims *out)
{
    laser_t L;
    model_t m;
    grid_t g;
    if (laser_build(&L, p) || model_build(&m, p)) return -1;
    grid_build(&g, p, &m);
    out->Nt = L.Nt;
    out->atmin = L.atmin;
    out->nband = m.N;
    out->nval = m.nval;
    out->ntotal = g.Ntotal;
    out->dV = g.dV;
    double tw = 0, k[3], w;
    for (int i = 0; i < g.Ntotal; ++i) { grid_point(&g, i, k, &w); tw += w; }
    out->total_weight = tw;
    model_free(&m);
    return 0;
}

static void para_range(int total, int size, int rank, int *s, int *e)   /* utility.h:104-115 */
{
    int w1 = total / size, w2 = total % size;
    *s = w1 * rank + (w2 < rank ? w2 : rank);
    *e = *s + w1 + (w2 > rank ? 1 : 0);
}

/* shotFrequency of antelope.cpp:274-278: steps between snapshots, from the
 * first pulse's period (laser.h:75) */
static int shot_every(const laser_t *L, int shot_number)
{
    if (shot_number <= 0) return 0;
    return (int)(L->p[0].period0 / shot_number / L->dt);
}

int orc_shot_dims(const orc_problem *p, int shot_number, int *every, int *nshots)
{
    laser_t L;
    if (laser_build(&L, p)) return -1;
    int F = shot_every(&L, shot_number);
    if (shot_number > 0 && F <= 0) return -3;   /* ktime % 0 in the reference */
    if (every) *every = F;
    if (nshots) *nshots = F > 0 ? (L.Nt - 1) / F + 1 : 0;
    return 0;
}

int orc_run(const orc_problem *p, double *inter, double *intra, double *dmi, long *steps_taken)
{
    return orc_run_shots(p, 0, inter, intra, dmi, steps_taken, NULL, NULL, NULL);
}

int orc_run_shots(const orc_problem *p, int shot_number, double *inter, double *intra, double *dmi,
                  long *steps_taken, double *occ1d, double *nc, double *pi)
{
    laser_t L;
    model_t m;
    grid_t g;
    tableau_t T;
    if (laser_build(&L, p) || model_build(&m, p) || tableau_build(&T, p->rk)) return -1;
    if (p->gauge == ORC_GAUGE_LENGTH_HAMILTONIAN) { model_free(&m); return -2; } /* SBEs.h:806-810 */
    const int F = shot_every(&L, shot_number);
    if (shot_number > 0 && (F <= 0 || !occ1d || !nc || !pi)) { model_free(&m); return -3; }
    grid_build(&g, p, &m);
    int N = m.N, NN = N * N, Nt = L.Nt;
    const int nshots = F > 0 ? (Nt - 1) / F + 1 : 0;
    int nth = T.adaptive ? 1 : (p->nthreads > 0 ? p->nthreads : 1);
    if (nth > g.Ntotal) nth = g.Ntotal;
    worker_t *W = calloc((size_t)nth, sizeof(worker_t));
    pthread_t *th = calloc((size_t)nth, sizeof(pthread_t));
    int rc = 0;
    for (int r = 0; r < nth; ++r) {
        worker_t *w = &W[r];
        w->p = p; w->L = &L; w->m = &m; w->g = &g; w->T = &T;
        w->gam_inter = p->T2 <= 1.0e-16 ? 0. : 1.0 / p->T2;     /* SBEs.h:484-493 */
        w->gam_intra = p->T1 <= 1.0e-16 ? 0. : 1.0 / p->T1;
        w->N = N; w->gauge = p->gauge; w->Nt = Nt;
        para_range(g.Ntotal, nth, r, &w->k0, &w->k1);
        int nk = w->k1 - w->k0;
        w->rho = calloc((size_t)nk * NN, sizeof(cplx));
        w->init = calloc((size_t)nk * NN, sizeof(cplx));
        w->P = calloc((size_t)nk * 3 * NN, sizeof(cplx));
        w->eps = calloc((size_t)nk * N, sizeof(double));
        w->kpt = calloc((size_t)nk * 3, sizeof(double));
        w->wgt = calloc((size_t)nk, sizeof(double));
        w->inter = calloc((size_t)Nt * 3, sizeof(double));
        w->intra = calloc((size_t)Nt * 3, sizeof(double));
        w->dmi = calloc((size_t)Nt * NN, sizeof(cplx));
        w->shot_every = F;
        w->occ1d = calloc((size_t)nshots * g.N[0] + 1, sizeof(double));
        w->nc = nc;
        w->pi = pi;
    }
    if (T.adaptive) rc = run_adaptive(&W[0]);
    else {
        for (int r = 1; r < nth; ++r) pthread_create(&th[r], NULL, worker_run, &W[r]);
        worker_run(&W[0]);
        for (int r = 1; r < nth; ++r) pthread_join(th[r], NULL);
    }
    /* rank-ordered sum of the partials, then the output scaling of
     * antelope.cpp:518-527 (currents times dV) */
    for (int n = 0; n < Nt; ++n) {
        for (int a = 0; a < 3; ++a) {
            double si = 0, sa = 0;
            for (int r = 0; r < nth; ++r) { si += W[r].inter[n * 3 + a]; sa += W[r].intra[n * 3 + a]; }
            inter[n * 3 + a] = si * g.dV;
            intra[n * 3 + a] = sa * g.dV;
        }
        for (int i = 0; i < NN; ++i) {
            cplx s = 0;
            for (int r = 0; r < nth; ++r) s += W[r].dmi[(size_t)n * NN + i];
            dmi[2 * ((size_t)n * NN + i)] = creal(s);
            dmi[2 * ((size_t)n * NN + i) + 1] = cimag(s);
        }
    }
    /* 1-D integrated occupation: rank-ordered sum, real part over Nk[1]
     * (antelope.cpp:354-370) */
    for (int sh = 0; sh < nshots; ++sh)
        for (int i = 0; i < g.N[0]; ++i) {
            double s = 0;
            for (int r = 0; r < nth; ++r) s += W[r].occ1d[(size_t)sh * g.N[0] + i];
            occ1d[(size_t)sh * g.N[0] + i] = s / (double)g.N[1];
        }
    if (steps_taken) *steps_taken = W[0].steps;
    for (int r = 0; r < nth; ++r) {
        free(W[r].rho); free(W[r].init); free(W[r].P); free(W[r].eps); free(W[r].kpt);
        free(W[r].wgt); free(W[r].inter); free(W[r].intra); free(W[r].dmi); free(W[r].occ1d);
    }
    free(W);
    free(th);
    model_free(&m);
    return rc;
}

void orc_laser_eval(const orc_problem *p, double t, double *A3, double *E3)
{
    laser_t L;
    if (laser_build(&L, p)) return;
    laser_AE(&L, t, A3, E3);
}

int orc_kgrid(const orc_problem *p, double *k3, double *w)
{
    model_t m;
    grid_t g;
    if (model_build(&m, p)) return -1;
    grid_build(&g, p, &m);
    for (int i = 0; i < g.Ntotal; ++i) grid_point(&g, i, k3 + 3 * i, w + i);
    model_free(&m);
    return 0;
}

int orc_model_hj(const orc_problem *p, const double *k3, double *H, double *J3)
{
    model_t m;
    if (model_build(&m, p)) return -1;
    int NN = m.N * m.N;
    cplx h[MAXNN], j[3 * MAXNN];
    model_H(&m, k3, h);
    model_J(&m, k3, j);
    for (int i = 0; i < NN; ++i) { H[2 * i] = creal(h[i]); H[2 * i + 1] = cimag(h[i]); }
    for (int i = 0; i < 3 * NN; ++i) { J3[2 * i] = creal(j[i]); J3[2 * i + 1] = cimag(j[i]); }
    model_free(&m);
    return 0;
}

int orc_eigh(int n, const double *a, double *w, double *v)
{
    if (n < 1 || n > ORC_MAX_BANDS) return -1;
    cplx A[MAXNN], U[MAXNN];
    for (int i = 0; i < n * n; ++i) A[i] = a[2 * i] + I * a[2 * i + 1];
    eigh(n, A, w, U);
    for (int i = 0; i < n * n; ++i) { v[2 * i] = creal(U[i]); v[2 * i + 1] = cimag(U[i]); }
    return 0;
}

int orc_tableau(int rk, double *c, double *a, double *b, double *bstar)
{
    tableau_t T;
    if (tableau_build(&T, rk)) return -1;
    for (int i = 0; i < 7; ++i) {
        c[i] = T.c[i];
        b[i] = T.b[i];
        bstar[i] = T.bstar[i];
        for (int j = 0; j < 7; ++j) a[i * 7 + j] = T.a[i][j];
    }
    return T.stages;
}
