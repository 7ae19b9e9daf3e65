/* Stand-in for the one LAPACKE routine the reference calls, LAPACKE_zheevr
 * (SBEs.h:289-291 and SBEs.h:877-879, always jobz='V', range='A', uplo='U',
 * row-major), so the unmodified reference sources compile without LAPACK.
 * Test infrastructure only: on the include path of the oracle/_ref build.
 *
 * Algorithm: cyclic complex Jacobi rotations on the Hermitian matrix rebuilt
 * from its upper triangle, then eigenvalues sorted ascending with their
 * eigenvectors as unit columns -- the same output contract as zheevr.  The
 * per-column phase of an eigenvector is a free choice in zheevr and differs
 * here; every quantity the reference writes out (currents, occupations) is
 * invariant under those phases for non-degenerate spectra, because the
 * dephasing matrix acts element-wise in the eigenbasis and the currents are
 * Re Tr of products in that same basis.
 *
 * The reference defines lapack_complex_double as std::complex<double> before
 * including this header (SBEs.h:20-22) and keeps a `complex` macro around it,
 * so only lapack_complex_double is used below.
 */
#ifndef ORACLE_REFSHIM_LAPACKE_H
#define ORACLE_REFSHIM_LAPACKE_H

#include <cmath>
#include <vector>

#ifndef lapack_complex_double
#error "define lapack_complex_double before including lapacke.h"
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

static inline lapack_int LAPACKE_zheevr(int matrix_layout, char jobz, char range, char uplo,
                                        lapack_int n, lapack_complex_double *a, lapack_int lda,
                                        double vl, double vu, lapack_int il, lapack_int iu,
                                        double abstol, lapack_int *m, double *w,
                                        lapack_complex_double *z, lapack_int ldz,
                                        lapack_int *isuppz)
{
    (void)vl; (void)vu; (void)il; (void)iu; (void)abstol; (void)isuppz;
    if (matrix_layout != LAPACK_ROW_MAJOR || (jobz != 'V' && jobz != 'v') ||
        (range != 'A' && range != 'a') || (uplo != 'U' && uplo != 'u') || n < 1)
        return -1;
    typedef lapack_complex_double cplx;
    std::vector<cplx> A(static_cast<size_t>(n) * n), V(static_cast<size_t>(n) * n);
    for (int i = 0; i < n; ++i) {
        A[i * n + i] = cplx(a[i * lda + i].real(), 0.0);
        for (int j = i + 1; j < n; ++j) {
            A[i * n + j] = a[i * lda + j];
            A[j * n + i] = std::conj(a[i * lda + j]);
        }
        for (int j = 0; j < n; ++j) V[i * n + j] = cplx(i == j ? 1.0 : 0.0, 0.0);
    }
    double scale = 0.0;
    for (int i = 0; i < n * n; ++i) scale += std::norm(A[i]);
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += std::norm(A[p * n + q]);
        if (off <= 1e-34 * scale || off == 0.0) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double r = std::abs(A[p * n + q]);
                if (r == 0.0) continue;
                const cplx e = A[p * n + q] / r;
                const double app = A[p * n + p].real(), aqq = A[q * n + q].real();
                const double zeta = (aqq - app) / (2.0 * r);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(zeta * zeta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                /* J = diag(1, conj(e)) * [[c, s], [-s, c]] on the (p, q) plane */
                const cplx Jpp(c, 0.0), Jpq(s, 0.0), Jqp = -s * std::conj(e), Jqq = c * std::conj(e);
                for (int k = 0; k < n; ++k) { /* A <- A J, V <- V J */
                    cplx akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = akp * Jpp + akq * Jqp;
                    A[k * n + q] = akp * Jpq + akq * Jqq;
                    cplx vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = vkp * Jpp + vkq * Jqp;
                    V[k * n + q] = vkp * Jpq + vkq * Jqq;
                }
                for (int k = 0; k < n; ++k) { /* A <- J^H A */
                    cplx apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = std::conj(Jpp) * apk + std::conj(Jqp) * aqk;
                    A[q * n + k] = std::conj(Jpq) * apk + std::conj(Jqq) * aqk;
                }
                A[p * n + q] = cplx(0.0, 0.0);
                A[q * n + p] = cplx(0.0, 0.0);
                A[p * n + p] = cplx(A[p * n + p].real(), 0.0);
                A[q * n + q] = cplx(A[q * n + q].real(), 0.0);
            }
        }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int i = 1; i < n; ++i) { /* stable insertion sort, ascending */
        int k = order[i], j = i - 1;
        while (j >= 0 && A[order[j] * n + order[j]].real() > A[k * n + k].real()) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = k;
    }
    for (int j = 0; j < n; ++j) {
        const int src = order[j];
        w[j] = A[src * n + src].real();
        for (int i = 0; i < n; ++i) z[i * ldz + j] = V[i * n + src];
    }
    *m = n;
    return 0;
}

#endif
