/*
 * Project-written stand-ins for the four LAPACK routines the reference's
 * tri_basis/initialize.cpp calls (dgetrf_, dgetrs_, dpbtrf_, dpbtrs_),
 * written from the textbook algorithms: LU with partial pivoting and banded
 * upper Cholesky (U^T U), both on column-major storage as LAPACK defines it.
 *
 * TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libtri_basis_ref.so so
 * that the reference's basis tables can be generated here. LAPACK itself is
 * absent from this image, so tables built through this file agree with the
 * reference built against a vendor LAPACK to rounding only.
 */
#include <math.h>

#define A_(i, j) a[(i) + (long)(j) * (*lda)]

int dgetrf_(const int *m, const int *n, double *a, const int *lda, int *ipiv, int *info) {
    int mn = (*m < *n ? *m : *n);
    *info = 0;
    for (int j = 0; j < mn; ++j) {
        int p = j;
        double best = fabs(A_(j, j));
        for (int i = j + 1; i < *m; ++i) {
            if (fabs(A_(i, j)) > best) { best = fabs(A_(i, j)); p = i; }
        }
        ipiv[j] = p + 1;
        if (A_(p, j) != 0.0) {
            if (p != j) {
                for (int c = 0; c < *n; ++c) { double t = A_(j, c); A_(j, c) = A_(p, c); A_(p, c) = t; }
            }
            double r = 1.0 / A_(j, j);
            for (int i = j + 1; i < *m; ++i) A_(i, j) *= r;
        } else if (*info == 0) {
            *info = j + 1;
        }
        for (int c = j + 1; c < *n; ++c) {
            double ajc = A_(j, c);
            if (ajc != 0.0)
                for (int i = j + 1; i < *m; ++i) A_(i, c) -= A_(i, j) * ajc;
        }
    }
    return 0;
}

int dgetrs_(const char *trans, const int *n, const int *nrhs, const double *a, const int *lda,
            const int *ipiv, double *b, const int *ldb, int *info) {
    *info = 0;
    for (int r = 0; r < *nrhs; ++r) {
        double *x = b + (long)r * (*ldb);
        if (trans[0] == 'N' || trans[0] == 'n') {
            for (int i = 0; i < *n; ++i) {
                int p = ipiv[i] - 1;
                if (p != i) { double t = x[i]; x[i] = x[p]; x[p] = t; }
            }
            for (int i = 0; i < *n; ++i)
                for (int k = 0; k < i; ++k) x[i] -= A_(i, k) * x[k];
            for (int i = *n - 1; i >= 0; --i) {
                for (int k = i + 1; k < *n; ++k) x[i] -= A_(i, k) * x[k];
                x[i] /= A_(i, i);
            }
        } else {
            /* A^T x = b with A = P L U:  U^T y = b, L^T z = y, x = P z */
            for (int i = 0; i < *n; ++i) {
                for (int k = 0; k < i; ++k) x[i] -= A_(k, i) * x[k];
                x[i] /= A_(i, i);
            }
            for (int i = *n - 1; i >= 0; --i)
                for (int k = i + 1; k < *n; ++k) x[i] -= A_(k, i) * x[k];
            for (int i = *n - 1; i >= 0; --i) {
                int p = ipiv[i] - 1;
                if (p != i) { double t = x[i]; x[i] = x[p]; x[p] = t; }
            }
        }
    }
    return 0;
}

#undef A_
#define AB_(r, c) ab[(r) + (long)(c) * (*ldab)]

int dpbtrf_(const char *uplo, const int *n, const int *kd, double *ab, const int *ldab, int *info) {
    (void)uplo;
    *info = 0;
    for (int j = 0; j < *n; ++j) {
        double ajj = AB_(*kd, j);
        if (!(ajj > 0.0)) { *info = j + 1; return 0; }
        ajj = sqrt(ajj);
        AB_(*kd, j) = ajj;
        int kn = (*kd < *n - 1 - j ? *kd : *n - 1 - j);
        double r = 1.0 / ajj;
        for (int c = 1; c <= kn; ++c) AB_(*kd - c, j + c) *= r;
        for (int a = 1; a <= kn; ++a) {
            double ua = AB_(*kd - a, j + a);
            for (int b = a; b <= kn; ++b) AB_(*kd + a - b, j + b) -= ua * AB_(*kd - b, j + b);
        }
    }
    return 0;
}

int dpbtrs_(const char *uplo, const int *n, const int *kd, const int *nrhs, const double *ab,
            const int *ldab, double *b, const int *ldb, int *info) {
    (void)uplo;
    *info = 0;
    for (int r = 0; r < *nrhs; ++r) {
        double *x = b + (long)r * (*ldb);
        for (int i = 0; i < *n; ++i) {
            int k0 = (i - *kd > 0 ? i - *kd : 0);
            for (int k = k0; k < i; ++k) x[i] -= AB_(*kd + k - i, i) * x[k];
            x[i] /= AB_(*kd, i);
        }
        for (int i = *n - 1; i >= 0; --i) {
            int k1 = (i + *kd < *n - 1 ? i + *kd : *n - 1);
            for (int k = i + 1; k <= k1; ++k) x[i] -= AB_(*kd + i - k, k) * x[k];
            x[i] /= AB_(*kd, i);
        }
    }
    return 0;
}
#undef AB_
