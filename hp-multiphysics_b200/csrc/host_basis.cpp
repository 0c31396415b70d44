// Host-side construction of the modal triangle basis tables (tri_basis<p,0>).
//
// Restates tri_basis<_p,ep>::initialize_values, lumpinv and lumpinv1d
// (tri_basis/initialize.cpp:161-455, 590-1082, 1085-1232) for a runtime p,
// with project-written numerics in place of the reference's dependencies:
//  * recurrence coefficients of monic Legendre / Jacobi(al,be) polynomials in
//    closed form (the reference calls Gautschi's recur, utilities/myblas.c:257);
//  * Gauss nodes and weights as the eigen-decomposition of the Jacobi matrix
//    (Golub-Welsch), solved here by cyclic Jacobi rotations (the reference's
//    gauss, utilities/myblas.c:766, uses an implicit QL);
//  * LU with partial pivoting and banded Cholesky in place of LAPACK's
//    dgetrf/dgetrs/dpbtrf/dpbtrs.
// The sequence of linear solves in lumpinv is kept exactly as the reference
// performs it, including its persistent work matrix: for p >= 6 some of the
// interior static-inversion systems have fewer equations than unknowns and the
// reference then solves with rows left over from the previous factorisation
// (its own comment: "THIS ONLY WORKS UP TO _sm = 5"); those rows get the exact
// static inversion here (see lumpinv). For p <= 4 every system is square and the
// same buffers are reused in the same order, so the tables agree with the
// reference's to rounding.
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

#include "hp_gpu.h"

namespace {

// Monic recurrence p_{k+1} = (x - a_k) p_k - b_k p_{k-1}; b_0 = total mass.
void legendre_recur(int n, double *a, double *b) {
    for (int k = 0; k < n; ++k) a[k] = 0.0;
    b[0] = 2.0;
    for (int k = 1; k < n; ++k) {
        double fk = k;
        b[k] = 1.0 / (4.0 - 1.0 / (fk * fk));
    }
}

// Jacobi weight (1-x)^al (1+x)^be on [-1,1].
void jacobi_recur(int n, double al, double be, double *a, double *b) {
    const double s = al + be;
    a[0] = (be - al) / (s + 2.0);
    b[0] = std::exp((s + 1.0) * std::log(2.0) + std::lgamma(al + 1.0) + std::lgamma(be + 1.0) -
                    std::lgamma(s + 2.0));
    if (n == 1) return;
    a[1] = (be * be - al * al) / ((s + 2.0) * (s + 4.0));
    b[1] = 4.0 * (al + 1.0) * (be + 1.0) / ((s + 3.0) * (s + 2.0) * (s + 2.0));
    for (int k = 2; k < n; ++k) {
        double t = 2.0 * k + s;
        a[k] = (be * be - al * al) / (t * (t + 2.0));
        b[k] = 4.0 * k * (k + al) * (k + be) * (k + s) / (t * t * (t + 1.0) * (t - 1.0));
    }
}

// Gauss rule with n nodes from the first n recurrence coefficients.
// Nodes ascending; weight_k = b_0 * (first eigenvector component)^2.
void gauss_rule(int n, const double *a, const double *b, double *x, double *w) {
    std::vector<double> A(n * n, 0.0), V(n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        A[i * n + i] = a[i];
        V[i * n + i] = 1.0;
        if (i + 1 < n) A[i * n + i + 1] = A[(i + 1) * n + i] = std::sqrt(b[i + 1]);
    }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += A[p * n + q] * A[p * n + q];
        if (off < 1e-300) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                double apq = A[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p,q
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p,q
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int i, int j) { return A[i * n + i] < A[j * n + j]; });
    for (int k = 0; k < n; ++k) {
        int e = ord[k];
        x[k] = A[e * n + e];
        w[k] = b[0] * V[0 * n + e] * V[0 * n + e];
    }
}

// Solves M x = v in place (M row-major n x n inside an ld-wide buffer, overwritten
// by its LU factors exactly where a column-major LAPACK dgetrf of M^T would leave them).
int lu_solve_rows(int n, double *M, int ld, double *v) {
    // A(i,j) := M[j*ld + i]  (the transposed view LAPACK would see)
    std::vector<int> piv(n);
    int info = 0;
    for (int j = 0; j < n; ++j) {
        int p = j;
        double best = std::fabs(M[j * ld + j]);
        for (int i = j + 1; i < n; ++i)
            if (std::fabs(M[j * ld + i]) > best) { best = std::fabs(M[j * ld + i]); p = i; }
        piv[j] = p;
        if (M[j * ld + p] != 0.0) {
            if (p != j)
                for (int c = 0; c < n; ++c) std::swap(M[c * ld + j], M[c * ld + p]);
            double r = 1.0 / M[j * ld + j];
            for (int i = j + 1; i < n; ++i) M[j * ld + i] *= r;
        } else if (!info) {
            info = j + 1;
        }
        for (int c = j + 1; c < n; ++c) {
            double ajc = M[c * ld + j];
            if (ajc != 0.0)
                for (int i = j + 1; i < n; ++i) M[c * ld + i] -= M[j * ld + i] * ajc;
        }
    }
    if (info) return info;
    // A^T x = v with A = P L U: U^T y = v, L^T z = y, x = P z
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < i; ++k) v[i] -= M[i * ld + k] * v[k];
        v[i] /= M[i * ld + i];
    }
    for (int i = n - 1; i >= 0; --i)
        for (int k = i + 1; k < n; ++k) v[i] -= M[i * ld + k] * v[k];
    for (int i = n - 1; i >= 0; --i)
        if (piv[i] != i) std::swap(v[i], v[piv[i]]);
    return 0;
}

// Upper banded Cholesky, band storage ab[col][kd+1] with ab[j][kd] the diagonal
// (the reference's _idiag / _sdiag1d layout, i.e. LAPACK 'U' band, ldab = kd+1).
int band_chol(int n, int kd, double *ab) {
    const int ld = kd + 1;
    for (int j = 0; j < n; ++j) {
        double ajj = ab[j * ld + kd];
        if (!(ajj > 0.0)) return j + 1;
        ajj = std::sqrt(ajj);
        ab[j * ld + kd] = ajj;
        int kn = std::min(kd, n - 1 - j);
        double r = 1.0 / ajj;
        for (int c = 1; c <= kn; ++c) ab[(j + c) * ld + kd - c] *= r;
        for (int a = 1; a <= kn; ++a) {
            double ua = ab[(j + a) * ld + kd - a];
            for (int b = a; b <= kn; ++b) ab[(j + b) * ld + kd + a - b] -= ua * ab[(j + b) * ld + kd - b];
        }
    }
    return 0;
}

void band_solve(int n, int kd, const double *ab, double *x) {
    const int ld = kd + 1;
    for (int i = 0; i < n; ++i) {
        for (int k = std::max(0, i - kd); k < i; ++k) x[i] -= ab[i * ld + kd + k - i] * x[k];
        x[i] /= ab[i * ld + kd];
    }
    for (int i = n - 1; i >= 0; --i) {
        for (int k = i + 1; k <= std::min(n - 1, i + kd); ++k) x[i] -= ab[k * ld + kd + i - k] * x[k];
        x[i] /= ab[i * ld + kd];
    }
}

struct Builder {
    hp_basis_tables &t;
    int p, sm, im, tm, bm, nx, gpx, gpn;
    // recurrence rows: [row][k], row 0 = x-direction sides, 1 = eta sides, m>=2 interior
    std::vector<double> a0, b0;
    int rlen;

    explicit Builder(hp_basis_tables &tt, int pp) : t(tt), p(pp) {
        sm = p - 1; im = (p - 1) * (p - 2) / 2; tm = (p + 1) * (p + 2) / 2; bm = 3 * p;
        nx = p + 2; gpx = gpn = p + 1;
        rlen = gpx + 2;
        a0.assign((sm + 2) * rlen, 0.0);
        b0.assign((sm + 2) * rlen, 0.0);
        std::memset(&t, 0, sizeof(t));
        t.p = p; t.sm = sm; t.im = im; t.tm = tm; t.bm = bm; t.nmodx = nx; t.gpx = gpx; t.gpn = gpn;
        t.ibwth = 1; t.sbwth = 2;
    }
    double &A(int r, int k) { return a0[r * rlen + k]; }
    double &B(int r, int k) { return b0[r * rlen + k]; }

    // Values and derivatives of the x functions at x and the eta functions at eta
    // (tri_basis/ptvalues.cpp:82-191), with the current norm() factors.
    void ptvalues_deriv(double x, double eta, double *pgx, double *dpgx, double *pgn, double *dpgn) {
        pgx[0] = 1.0; dpgx[0] = 0.0;
        pgx[1] = 0.5 * (1 - x); dpgx[1] = -0.5;
        pgx[2] = 0.5 * (1 + x); dpgx[2] = 0.5;
        double pk = 1.0, pkm = 0.0, dpk = 0.0, dpkm = 0.0;
        for (int m = 0; m < sm; ++m) {
            pgx[m + 3] = (1. + x) * (1. - x) * .25 * pk * t.norm[m + 3];
            dpgx[m + 3] = (-x * .5 * pk + (1. + x) * (1. - x) * .25 * dpk) * t.norm[m + 3];
            double pkp = (x - A(0, m)) * pk - B(0, m) * pkm;
            double dpkp = pk + (x - A(0, m)) * dpk - B(0, m) * dpkm;
            dpkm = dpk; dpk = dpkp; pkm = pk; pk = pkp;
        }
        int ind = 0;
        pgn[ind] = (1 + eta) * .5; dpgn[ind++] = 0.5;
        pgn[ind] = (1 - eta) * .5; dpgn[ind++] = -0.5;
        pgn[ind] = (1 - eta) * .5; dpgn[ind++] = -0.5;
        for (int m = 2; m <= sm + 1; ++m) {
            pgn[ind] = std::pow(.5 * (1 - eta), (double)m);
            dpgn[ind] = -.5 * m * std::pow(.5 * (1. - eta), (double)(m - 1));
            ++ind;
        }
        for (int side = 1; side <= 2; ++side) {
            pk = 1.0; pkm = 0.0; dpk = 0.0; dpkm = 0.0;
            for (int n = 0; n < sm; ++n) {
                double sg = (side == 2 && (n % 2)) ? -1.0 : 1.0;
                pgn[ind] = sg * (1. - eta) * (1. + eta) * .25 * pk * t.norm[n + 3];
                dpgn[ind] = sg * (-.5 * eta * pk + (1. - eta) * (1. + eta) * .25 * dpk) * t.norm[n + 3];
                double pkp = (eta - A(1, n)) * pk - B(1, n) * pkm;
                double dpkp = pk + (eta - A(1, n)) * dpk - B(1, n) * dpkm;
                dpkm = dpk; dpk = dpkp; pkm = pk; pk = pkp;
                ++ind;
            }
        }
        for (int m = 2; m < sm + 1; ++m) {
            pk = 1.0; pkm = 0.0; dpk = 0.0; dpkm = 0.0;
            for (int k = 0; k < sm + 1 - m; ++k) {
                double e1 = std::pow(.5 * (1. - eta), (double)m);
                pgn[ind] = (e1 * .5 * (1. + eta) * pk) * t.norm[ind];
                dpgn[ind] = (-.25 * m * std::pow(.5 * (1. - eta), (double)(m - 1)) * (1. + eta) * pk +
                             e1 * .5 * (pk + (1. + eta) * dpk)) * t.norm[ind];
                double pkp = (eta - A(m, k)) * pk - B(m, k) * pkm;
                double dpkp = pk + (eta - A(m, k)) * dpk - B(m, k) * dpkm;
                dpkm = dpk; dpk = dpkp; pkm = pk; pk = pkp;
                ++ind;
            }
        }
    }

    void initialize_values() {
        double tmpx[HP_MXGP + 2], tmpw[HP_MXGP + 2];
        // Gauss-Legendre points (x direction)
        legendre_recur(gpx + 1, &A(0, 0), &B(0, 0));
        gauss_rule(gpx, &A(0, 0), &B(0, 0), tmpx, tmpw);
        for (int i = 0; i < gpx; ++i) { t.x0[i] = tmpx[i]; t.wtx[i] = tmpw[i]; }
        for (int i = 0; i < gpx; ++i) {
            double d = 1.0;
            for (int k = 0; k < gpx; ++k)
                if (k != i) d *= (t.x0[i] - t.x0[k]);
            t.dltx[i] = d;
        }
        for (int i = 0; i < gpx; ++i)
            for (int n = 0; n < gpx; ++n)
                if (n != i) {
                    t.dltx1[i][n] = t.dltx[i] / (t.x0[i] - t.x0[n]);
                    t.dltn1[i][n] = t.dltx[i] / (t.x0[i] - t.x0[n]) * .5 * (1 + t.x0[i]);
                }
        for (int i = 0; i < gpx; ++i) t.dltx[i] = 1.0 / t.dltx[i];

        // side polynomials: Jacobi(2,2)
        jacobi_recur(sm + 1, 2.0, 2.0, &A(0, 0), &B(0, 0));
        for (int i = 0; i < HP_MXTM; ++i) t.norm[i] = 1.0;
        double pgx[HP_MXX], dpgx[HP_MXX], pgn[HP_MXTM], dpgn[HP_MXTM];
        for (int i = 0; i < gpx; ++i) {
            double x = t.x0[i];
            t.xp[i] = x;
            t.x0[i] = 0.5 * (1 + x);
            ptvalues_deriv(x, 0.0, pgx, dpgx, pgn, dpgn);
            for (int m = 0; m < nx; ++m) { t.gx[i][m] = pgx[m]; t.dgx[i][m] = dpgx[m]; }
        }

        // Gauss-Jacobi(1,0) points (eta direction), weights halved
        jacobi_recur(gpn + 1, 1.0, 0.0, &A(1, 0), &B(1, 0));
        gauss_rule(gpn, &A(1, 0), &B(1, 0), tmpx, tmpw);
        for (int i = 0; i < gpn; ++i) { t.n0[i] = tmpx[i]; t.wtn[i] = tmpw[i] * 0.5; }
        for (int i = 0; i < gpn; ++i) {
            double d = 1.0;
            for (int k = 0; k < gpn; ++k)
                if (k != i) d *= (t.n0[i] - t.n0[k]);
            t.dltn[i] = d;
        }
        for (int j = 0; j < gpn; ++j)
            for (int n = 0; n < gpn; ++n)
                if (n != j) t.dltn2[j][n] = t.dltn[j] / (t.n0[j] - t.n0[n]);
        for (int j = 0; j < gpn; ++j) t.dltn[j] = 1.0 / t.dltn[j];

        jacobi_recur(sm + 1, 2.0, 2.0, &A(1, 0), &B(1, 0));
        for (int m = 2; m < sm + 1; ++m) jacobi_recur(sm + 2 - m, 2. * m + 1, 2.0, &A(m, 0), &B(m, 0));

        for (int j = 0; j < gpn; ++j) {
            double eta = t.n0[j];
            t.np[j] = eta;
            t.n0[j] = 2.0 / (1 - eta);
            ptvalues_deriv(0.0, eta, pgx, dpgx, pgn, dpgn);
            for (int m = 0; m < tm; ++m) { t.gn[j][m] = pgn[m]; t.dgn[j][m] = dpgn[m]; }
        }

        for (int n = 0; n < 3; ++n) t.norm[n] = 1.0;
        for (int n = 3; n < sm + 3; ++n) {
            double s = 0.0;
            for (int i = 0; i < gpx; ++i) s += t.wtx[i] * t.gx[i][n] * t.gx[i][n];
            t.norm[n] = 1. / std::sqrt(s);
            t.norm[n + sm] = t.norm[n];
            t.norm[n + 2 * sm] = t.norm[n];
        }
        for (int m = bm; m < tm; ++m) {
            double s = 0.0;
            for (int j = 0; j < gpn; ++j) s += t.wtn[j] * t.gn[j][m] * t.gn[j][m];
            t.norm[m] = 1. / std::sqrt(s);
        }
        for (int n = 3; n < nx; ++n) {
            for (int i = 0; i < gpx; ++i) { t.gx[i][n] *= t.norm[n]; t.dgx[i][n] *= t.norm[n]; }
            for (int j = 0; j < gpn; ++j) {
                t.gn[j][n + sm] *= t.norm[n]; t.dgn[j][n + sm] *= t.norm[n];
                t.gn[j][n + 2 * sm] *= t.norm[n]; t.dgn[j][n + 2 * sm] *= t.norm[n];
            }
        }
        for (int m = bm; m < tm; ++m)
            for (int j = 0; j < gpn; ++j) { t.gn[j][m] = t.gn[j][m] * t.norm[m]; t.dgn[j][m] = t.dgn[j][m] * t.norm[m]; }

        for (int m = 0; m < nx; ++m)
            for (int i = 0; i < gpx; ++i) {
                t.gxwtx[m][i] = t.gx[i][m] * t.wtx[i];
                t.dgxwtx[m][i] = t.dgx[i][m] * t.wtx[i];
            }
        for (int m = 0; m < tm; ++m)
            for (int j = 0; j < gpn; ++j) {
                t.gnwtn[m][j] = t.gn[j][m] * t.wtn[j];
                t.gnwtnn0[m][j] = t.gn[j][m] * t.wtn[j] * t.n0[j];
                t.dgnwtn[m][j] = t.dgn[j][m] * t.wtn[j];
            }
    }

    // value-only projection and test-function integration on a [gpx][gpn] grid
    // (tri_basis/proj.cpp:121-186, intgrt.cpp:22-78)
    void proj_val(const double *lin, double *f) {
        double wk0[HP_MXGP][HP_MXX];
        const int bs1 = sm + 3, bs2 = 2 * sm + 3;
        for (int j = 0; j < gpn; ++j) {
            wk0[j][0] = lin[0] * t.gn[j][0];
            double l = lin[1] * t.gn[j][1];
            for (int m = bs2; m < bm; ++m) l += lin[m] * t.gn[j][m];
            wk0[j][1] = l;
            l = lin[2] * t.gn[j][2];
            for (int m = bs1; m < bs2; ++m) l += lin[m] * t.gn[j][m];
            wk0[j][2] = l;
            int ind = bm, cnt = sm - 1;
            for (int m = 3; m < bs1; ++m) {
                l = lin[m] * t.gn[j][m];
                for (int n = 0; n < cnt; ++n) l += lin[ind + n] * t.gn[j][ind + n];
                ind += cnt--;
                wk0[j][m] = l;
            }
        }
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                double l = 0.0;
                for (int n = 0; n < nx; ++n) l += wk0[j][n] * t.gx[i][n];
                f[i * gpn + j] = l;
            }
    }
    void intgrt(double *r, const double *f) {
        double wk0[HP_MXX][HP_MXGP];
        const int bs1 = sm + 3, bs2 = 2 * sm + 3;
        for (int n = 0; n < nx; ++n)
            for (int j = 0; j < gpn; ++j) {
                double l = f[0 * gpn + j] * t.gxwtx[n][0];
                for (int i = 1; i < gpx; ++i) l += f[i * gpn + j] * t.gxwtx[n][i];
                wk0[n][j] = l;
            }
        for (int m = 0; m < bs1; ++m) {
            double l = 0.0;
            for (int j = 0; j < gpn; ++j) l += t.gnwtn[m][j] * wk0[m][j];
            r[m] = l;
        }
        for (int m = bs1; m < bs2; ++m) {
            double l = 0.0;
            for (int j = 0; j < gpn; ++j) l += t.gnwtn[m][j] * wk0[2][j];
            r[m] = l;
        }
        for (int m = bs2; m < bm; ++m) {
            double l = 0.0;
            for (int j = 0; j < gpn; ++j) l += t.gnwtn[m][j] * wk0[1][j];
            r[m] = l;
        }
        int indx = bm;
        for (int m = 3; m < sm + 2; ++m)
            for (int n = 0; n < sm + 2 - m; ++n) {
                double l = 0.0;
                for (int j = 0; j < gpn; ++j) l += t.gnwtn[indx][j] * wk0[m][j];
                r[indx++] = l;
            }
    }

    int lumpinv() {
        const int TM = tm;
        std::vector<double> mm(TM * TM), mwk(TM * TM, 0.0), u(TM), l(TM), vwk(TM, 0.0), wk1(TM * gpx);
        auto MM = [&](int i, int j) -> double & { return mm[i * TM + j]; };
        auto MW = [&](int i, int j) -> double & { return mwk[i * TM + j]; };
        for (int m = 0; m < TM; ++m) {
            for (int i = 0; i < TM; ++i) u[i] = 0.0;
            u[m] = 1.0;
            proj_val(u.data(), wk1.data());
            intgrt(l.data(), wk1.data());
            for (int i = 0; i < TM; ++i) MM(m, i) = l[i];
        }
        int err = 0;
        if (p > 1) {
            const int N = (sm + 1) * (sm + 2) / 2 - 1;
            for (int i = 0; i < 3; ++i) {
                int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
                for (int k = 0; k < 2; ++k) {
                    int ind = (i + 1 + k) % 3;
                    vwk[k] = MM(ind, i);
                    for (int j = 0; j < sm; ++j) {
                        MW(k, j) = MM(ind, 3 + j + i1 * sm);
                        MW(k, j + sm) = MM(ind, 3 + j + i2 * sm);
                    }
                    for (int j = 0; j < im; ++j) MW(k, 2 * sm + j) = MM(ind, j + bm);
                }
                for (int k = 0; k < 3; ++k)
                    for (int m = 0; m < sm - 1; ++m) {
                        int r = m + 2 + k * (sm - 1);
                        vwk[r] = MM(3 + m + k * sm, i);
                        for (int j = 0; j < sm; ++j) {
                            MW(r, j) = MM(3 + m + k * sm, 3 + j + i1 * sm);
                            MW(r, j + sm) = MM(3 + m + k * sm, 3 + j + i2 * sm);
                        }
                        for (int j = 0; j < im; ++j) MW(r, 2 * sm + j) = MM(3 + m + k * sm, j + bm);
                    }
                int ind = 3 * sm - 1, ind1 = 0;
                for (int m = 2; m < sm + 1; ++m) {
                    for (int n = 1; n < sm + 1 - m; ++n) {
                        vwk[ind] = MM(ind1 + bm, i);
                        for (int j = 0; j < sm; ++j) {
                            MW(ind, j) = MM(ind1 + bm, 3 + j + i1 * sm);
                            MW(ind, j + sm) = MM(ind1 + bm, 3 + j + i2 * sm);
                        }
                        for (int j = 0; j < im; ++j) MW(ind, 2 * sm + j) = MM(ind1 + bm, j + bm);
                        ++ind; ++ind1;
                    }
                    ++ind1;
                }
                if (lu_solve_rows(N, mwk.data(), TM, vwk.data())) err = 1;
                for (int k = 0; k < im; ++k) t.ifmb[i][k] = vwk[k + 2 * sm];
            }
            for (int k = 0; k < sm; ++k) {
                t.sfmv[0][k] = vwk[k + sm];
                t.sfmv[1][k] = vwk[k];
            }
            double vd = MM(2, 2);
            for (int k = 0; k < sm; ++k) {
                vd -= t.sfmv[0][k] * MM(2, 3 + k + 1 * sm);
                vd -= t.sfmv[1][k] * MM(2, 3 + k);
            }
            for (int k = 0; k < im; ++k) vd -= t.ifmb[2][k] * MM(2, k + bm);
            t.vdiag = vd;
        } else {
            t.vdiag = MM(0, 0) + MM(0, 1) + MM(0, 2);
        }

        if (im > 0) {
            for (int i = 0; i < 3; ++i) {
                int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
                for (int k = 0; k < sm - 1; ++k) {
                    // Equation count of the reference's system for this side mode; when it is
                    // below im (sm >= 4, i.e. p >= 5) the reference factors stale rows left
                    // from the previous solve and its result is numerically undefined (it
                    // reaches 1e13 at p = 5). There, this library uses the exact static
                    // inversion of all interior modes instead, as the reference itself does
                    // for the highest side mode.
                    const int nrows = (sm - 1 - k) + (std::min(2 * k, sm - 1) - k) + (sm - 2) * (sm - 1) / 2;
                    if (nrows < im) {
                        for (int j = 0; j < im; ++j) {
                            vwk[j] = MM(i * sm + 3 + k, j + bm);
                            for (int kk = 0; kk < im; ++kk) MW(j, kk) = MM(kk + bm, j + bm);
                        }
                        if (lu_solve_rows(im, mwk.data(), TM, vwk.data())) err = 1;
                        for (int j = 0; j < im; ++j) t.ifmb[i * sm + 3 + k][j] = vwk[j];
                        continue;
                    }
                    int ind = 0;
                    for (int j = k; j < sm - 1; ++j) {
                        vwk[ind] = MM(i * sm + 3 + k, i1 * sm + 3 + j);
                        for (int m = 0; m < im; ++m) MW(ind, m) = MM(bm + m, i1 * sm + 3 + j);
                        ++ind;
                    }
                    for (int j = k; j < std::min(2 * k, sm - 1); ++j) {
                        vwk[ind] = MM(i * sm + 3 + k, i2 * sm + 3 + j);
                        for (int m = 0; m < im; ++m) MW(ind, m) = MM(bm + m, i2 * sm + 3 + j);
                        ++ind;
                    }
                    int ind1 = 0;
                    for (int m = 2; m < sm + 1; ++m) {
                        for (int n = 1; n < sm + 1 - m; ++n) {
                            vwk[ind] = MM(i * sm + 3 + k, bm + ind1);
                            for (int j = 0; j < im; ++j) MW(ind, j) = MM(bm + j, bm + ind1);
                            ++ind; ++ind1;
                        }
                        ++ind1;
                    }
                    if (lu_solve_rows(im, mwk.data(), TM, vwk.data())) err = 1;
                    for (int j = 0; j < im; ++j) t.ifmb[i * sm + 3 + k][j] = vwk[j];
                }
                for (int j = 0; j < im; ++j) {
                    vwk[j] = MM(i * sm + sm + 2, j + bm);
                    for (int k = 0; k < im; ++k) MW(j, k) = MM(k + bm, j + bm);
                }
                if (lu_solve_rows(im, mwk.data(), TM, vwk.data())) err = 1;
                for (int j = 0; j < im; ++j) t.ifmb[i * sm + sm + 2][j] = vwk[j];
            }
        }

        for (int k = 0; k < sm; ++k) {
            for (int j = 0; j < TM; ++j) u[j] = 0.0;
            u[k + 3] = 1.0;
            for (int j = 0; j < im; ++j) u[j + bm] = -t.ifmb[k + 3][j];
            proj_val(u.data(), wk1.data());
            intgrt(l.data(), wk1.data());
            for (int j = 0; j < 3; ++j) t.vfms[j][k] = l[j];
            t.sdiag[k] = 1.0 / l[3 + k];
            for (int j = 0; j < k; ++j) {
                t.sfms[j][k][0] = l[3 + j];
                t.sfms[j][k][1] = l[3 + j + sm];
                t.sfms[j][k][2] = l[3 + j + 2 * sm];
            }
        }

        if (im > 0) {
            const int kd = 1;
            for (int j = 0; j < im; ++j)
                for (int i = std::max(0, j - kd); i <= j; ++i) t.idiag[j][i - (j - kd)] = MM(i + bm, j + bm);
            if (band_chol(im, kd, &t.idiag[0][0])) err = 1;
            for (int i = 0; i < bm; ++i) {
                double x[HP_MXIM];
                for (int j = 0; j < im; ++j) x[j] = MM(i, j + bm);
                band_solve(im, kd, &t.idiag[0][0], x);
                for (int j = 0; j < im; ++j) t.bfmi[i][j] = x[j];
            }
        }
        return err;
    }

    int lumpinv1d() {
        const int n1 = p + 1;
        std::vector<double> mm(n1 * n1);
        auto MM = [&](int i, int j) -> double & { return mm[i * n1 + j]; };
        for (int m = 1; m < p + 2; ++m)
            for (int k = 1; k < p + 2; ++k) {
                double s = 0.0;
                for (int i = 0; i < gpx; ++i) s += t.wtx[i] * t.gx[i][m] * t.gx[i][k];
                MM(m - 1, k - 1) = s;
            }
        int err = 0;
        if (p > 1) {
            const int kd = 2;
            // sdiag1d stored [sm][3]
            double ab[HP_MXSM * 3];
            std::memset(ab, 0, sizeof(ab));
            for (int j = 0; j < sm; ++j)
                for (int i = std::max(0, j - kd); i <= j; ++i) ab[j * 3 + i - (j - kd)] = MM(i + 2, j + 2);
            if (band_chol(sm, kd, ab)) err = 1;
            for (int j = 0; j < sm; ++j)
                for (int k = 0; k < 3; ++k) t.sdiag1d[j][k] = ab[j * 3 + k];
            for (int i = 0; i < 2; ++i) {
                double x[HP_MXSM];
                for (int j = 0; j < sm; ++j) x[j] = MM(i, j + 2);
                band_solve(sm, kd, ab, x);
                for (int j = 0; j < sm; ++j) t.vfms1d[i][j] = x[j];
            }
            std::vector<double> mwk(sm * sm), vwk(sm);
            for (int i = 0; i < 2; ++i) {
                vwk[0] = MM(i, (i + 1) % 2);
                for (int m = 0; m < sm; ++m) mwk[0 * sm + m] = MM((i + 1) % 2, m + 2);
                for (int m = 0; m < sm - 1; ++m) {
                    vwk[m + 1] = MM(i, m + 2);
                    for (int k = 0; k < sm; ++k) mwk[(m + 1) * sm + k] = MM(m + 2, k + 2);
                }
                if (lu_solve_rows(sm, mwk.data(), sm, vwk.data())) err = 1;
                for (int k = 0; k < sm; ++k) t.sfmv1d[i][k] = vwk[k];
            }
            double vd = MM(0, 0);
            for (int k = 0; k < sm; ++k) vd -= t.sfmv1d[0][k] * MM(0, 2 + k);
            t.vdiag1d = vd;
        } else {
            t.vdiag1d = MM(0, 0) + MM(0, 1);
        }
        return err;
    }
};

}  // namespace

extern "C" int hp_basis_build(int p, hp_basis_tables *out) {
    if (!out || p < 1 || p > HP_MAXP) return HP_EINVAL;
    Builder b(*out, p);
    b.initialize_values();
    int e = b.lumpinv();
    e += b.lumpinv1d();
    return e;
}

// ---------------------------------------------------------------------------
// Modal tetrahedral basis (tet_basis, runtime p <= 4).
//
// Restates tet_basis::initialize_values (tet_basis/initialize.cpp:73-380) and the
// 1D functions of tet_basis::ptvalues_deriv (tet_basis/ptvalues.cpp:154-330) with
// the recurrence and Gauss routines above, then forms dense per-point operators
// from the factorisation that tet_basis::proj (proj.cpp:22-265) applies: every
// mode is sgn * gx(x_i, mx) gy(y_j, my) gz(z_k, mz) in the collapsed coordinates.
// ---------------------------------------------------------------------------
#include "hp_tet.h"

namespace {

// Monic three-term recurrence value and derivative, p_0 = 1, from (a, b).
struct Rec {
    double pk = 1.0, pkm = 0.0, dpk = 0.0, dpkm = 0.0;
    void step(double x, double a, double b) {
        const double pkp = (x - a) * pk - b * pkm;
        const double dpkp = pk + (x - a) * dpk - b * dpkm;
        dpkm = dpk;
        dpk = dpkp;
        pkm = pk;
        pk = pkp;
    }
};

struct TetRecur {
    int em;
    std::vector<double> a22, b22;              // Jacobi(2,2): edges
    std::vector<std::vector<double>> af, bf;   // Jacobi(2m+3,2), m = 1..em: faces
    std::vector<std::vector<double>> ai, bi;   // Jacobi(2n+2m+4,2): interiors
    explicit TetRecur(int em_) : em(em_) {
        const int n = em + 1;
        a22.resize(n); b22.resize(n);
        jacobi_recur(n, 2.0, 2.0, a22.data(), b22.data());
        af.assign(em + 1, std::vector<double>(n)); bf = af;
        for (int m = 1; m <= em; ++m) jacobi_recur(n, 2.0 * m + 3.0, 2.0, af[m].data(), bf[m].data());
        for (int nn = 1; nn <= em - 1; ++nn)
            for (int m = 1; m <= em - nn; ++m) {
                ai.emplace_back(n); bi.emplace_back(n);
                jacobi_recur(n, 2.0 * nn + 2.0 * m + 4.0, 2.0, ai.back().data(), bi.back().data());
            }
    }
    // x direction: vertex 0,1 / edge 4; vertex 2 etc.; vertex 3 etc.; edge 1 bubbles
    void fx(double x, double *g, double *dg) const {
        int k = 0;
        g[k] = 1.0; dg[k++] = 0.0;
        g[k] = 0.5 * (1 - x); dg[k++] = -0.5;
        g[k] = 0.5 * (1 + x); dg[k++] = 0.5;
        Rec r;
        for (int m = 0; m < em; ++m) {
            g[k] = 0.25 * (1.0 + x) * (1.0 - x) * r.pk;
            dg[k++] = -x * 0.5 * r.pk + (1.0 + x) * (1.0 - x) * 0.25 * r.dpk;
            r.step(x, a22[m], b22[m]);
        }
    }
    void fy(double y, double *g, double *dg) const {
        int k = 0;
        g[k] = 1.0; dg[k++] = 0.0;
        g[k] = (1 + y) * 0.5; dg[k++] = 0.5;
        g[k] = (1 - y) * 0.5; dg[k++] = -0.5;
        for (int m = 2; m <= em + 1; ++m) {
            g[k] = std::pow(0.5 * (1 - y), m);
            dg[k++] = -0.5 * m * std::pow(0.5 * (1. - y), m - 1);
        }
        Rec r;
        for (int n = 0; n < em; ++n) {
            g[k] = (1.0 - y) * (1.0 + y) * 0.25 * r.pk;
            dg[k++] = -0.5 * y * r.pk + (1.0 - y) * (1.0 + y) * 0.25 * r.dpk;
            r.step(y, a22[n], b22[n]);
        }
        for (int m = 1; m <= em - 1; ++m) {
            Rec q;
            for (int kk = 1; kk <= em - m; ++kk) {
                g[k] = std::pow(0.5 * (1.0 - y), m + 1) * 0.5 * (1.0 + y) * q.pk;
                dg[k++] = -0.25 * (m + 1.0) * std::pow(0.5 * (1.0 - y), m) * (1.0 + y) * q.pk +
                          std::pow(0.5 * (1.0 - y), m + 1) * 0.5 * (q.pk + (1.0 + y) * q.dpk);
                q.step(y, af[m][kk - 1], bf[m][kk - 1]);
            }
        }
    }
    void fz(double z, double *g, double *dg) const {
        int k = 0;
        g[k] = (1 + z) * 0.5; dg[k++] = 0.5;
        g[k] = (1 - z) * 0.5; dg[k++] = -0.5;
        for (int m = 2; m <= em + 1; ++m) {
            g[k] = std::pow(0.5 * (1 - z), m);
            dg[k++] = -0.5 * m * std::pow(0.5 * (1. - z), m - 1);
        }
        Rec r;
        for (int n = 0; n < em; ++n) {
            g[k] = (1.0 - z) * (1.0 + z) * 0.25 * r.pk;
            dg[k++] = -0.5 * z * r.pk + (1.0 - z) * (1.0 + z) * 0.25 * r.dpk;
            r.step(z, a22[n], b22[n]);
        }
        for (int m = 1; m <= em - 1; ++m) {
            Rec q;
            for (int kk = 1; kk <= em - m; ++kk) {
                g[k] = std::pow(0.5 * (1.0 - z), m + 1) * 0.5 * (1.0 + z) * q.pk;
                dg[k++] = -0.25 * (m + 1.0) * std::pow(0.5 * (1.0 - z), m) * (1.0 + z) * q.pk +
                          std::pow(.5 * (1.0 - z), m + 1) * .5 * (q.pk + (1.0 + z) * q.dpk);
                q.step(z, af[m][kk - 1], bf[m][kk - 1]);
            }
        }
        int ind2 = 0;
        for (int n = 1; n <= em - 1; ++n)
            for (int m = 1; m <= em - n; ++m) {
                Rec q;
                for (int kk = 1; kk <= em - m - n; ++kk) {
                    g[k] = std::pow(0.5 * (1.0 - z), m + n + 1) * 0.5 * (1.0 + z) * q.pk;
                    dg[k++] = -0.25 * (m + n + 1) * std::pow(0.5 * (1.0 - z), m + n) * (1.0 + z) * q.pk +
                              std::pow(.5 * (1.0 - z), m + n + 1) * .5 * (q.pk + (1. + z) * q.dpk);
                    q.step(z, ai[ind2][kk - 1], bi[ind2][kk - 1]);
                }
                ++ind2;
            }
    }
};

// Lagrange-derivative factors of one Gauss direction (initialize.cpp:157-180):
// d(i) = 1 / prod_{k != i} (x_i - x_k); d2(i,n) = prod_{k != i}(x_i - x_k) / (x_i - x_n);
// d3 = d2 (1 + x_i) / 2 (on the raw nodes).
void lagrange_factors(int g, const double *x, double *d, double (*d2)[HP_TET_MAXG], double (*d3)[HP_TET_MAXG]) {
    for (int i = 0; i < g; ++i) {
        double pr = 1.0;
        for (int k = 0; k < g; ++k)
            if (k != i) pr *= (x[i] - x[k]);
        for (int n = 0; n < g; ++n) {
            d2[i][n] = (n == i) ? 0.0 : pr / (x[i] - x[n]);
            if (d3) d3[i][n] = (n == i) ? 0.0 : d2[i][n] * (1. + x[i]) / 2.;
        }
        d[i] = 1.0 / pr;
    }
}

// (A f)(i) = sum_n A(i,n) f(n) equal to sum_{n != i} (f_i d_i + f_n d_n) c(i,n)
// (the pairwise form of derivr / derivs / derivt, proj.cpp:781-911).
void deriv_operator(int g, const double *d, const double (*c)[HP_TET_MAXG], double (*A)[HP_TET_MAXG]) {
    for (int i = 0; i < g; ++i) {
        double diag = 0.0;
        for (int n = 0; n < g; ++n) {
            if (n == i) continue;
            diag += c[i][n];
            A[i][n] = d[n] * c[i][n];
        }
        A[i][i] = d[i] * diag;
    }
}

}  // namespace

// Gaussian elimination with partial pivoting: solves A x = b (A n x n, row-major, destroyed).
static bool dense_solve(int n, std::vector<double> &A, std::vector<double> &b) {
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
        if (A[(size_t)piv * n + c] == 0.0) return false;
        if (piv != c) {
            for (int k = 0; k < n; ++k) std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
            std::swap(b[c], b[piv]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double f = A[(size_t)r * n + c] / A[(size_t)c * n + c];
            for (int k = c; k < n; ++k) A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
            b[r] -= f * b[c];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        double acc = b[c];
        for (int k = c + 1; k < n; ++k) acc -= A[(size_t)c * n + k] * b[k];
        b[c] = acc / A[(size_t)c * n + c];
    }
    return true;
}

// The edge part of tet_basis::lumpinv at p = 3 (tet_basis/initialize.cpp:846-1040): for edge i
// and each side of it, its second mode and the adjacent face modes (dofs) combine with its
// first mode so that the mass products with the first modes of three edges of its cone
// (constraints, the reference's edgecone table, 1-based edge numbers) vanish. The face
// coefficients of edges 0..2 give ffms; the last system's edge coefficient gives sfms(0), and
// mdiag / odiag are the first-mode mass of the combination against edge modes 0 and 2.
static void tet_edge_cones(hp_tet_tables &t) {
    const int em = t.em, fm = t.fm;  // 2, 1
    static const int cone[6][3][2] = {{{2, 3}, {4, 4}, {6, 5}}, {{3, 1}, {4, 5}, {5, 6}}, {{2, 1}, {4, 5}, {6, 6}},
                                      {{1, 1}, {5, 2}, {6, 3}}, {{2, 1}, {4, 2}, {6, 3}}, {{3, 1}, {4, 2}, {5, 3}}};
    const int f0 = 4 + 6 * em;
    const int dind[6][3] = {{5, f0, f0 + fm},          {5 + em, f0, f0 + 2 * fm},     {5 + 2 * em, f0, f0 + 3 * fm},
                            {5 + 3 * em, f0 + 2 * fm, f0 + 3 * fm}, {5 + 4 * em, f0 + fm, f0 + 3 * fm},
                            {5 + 5 * em, f0 + fm, f0 + 2 * fm}};
    std::vector<double> x(3);
    for (int side = 0; side < 2; ++side)
        for (int i = 0; i < 6; ++i) {
            int lind[3];
            for (int j = 0; j < 3; ++j) lind[j] = 4 + (cone[i][j][side] - 1) * em;
            std::vector<double> A(9);
            for (int j = 0; j < 3; ++j) {
                for (int k = 0; k < 3; ++k) A[j * 3 + k] = t.mm[lind[j]][dind[i][k]];
                x[j] = -t.mm[lind[j]][4 + i * em];
            }
            if (!dense_solve(3, A, x)) return;
            if (i < 3)
                for (int k = 0; k < fm; ++k) t.ffms[i][k][side] = x[k + em - 1];
        }
    t.sfms0 = -x[0];
    const int omode = 8;
    t.mdiag = t.mm[4][4];
    t.odiag = t.mm[4][omode];
    for (int k = 1; k < em; ++k) {
        t.mdiag += t.sfms0 * t.mm[4 + k][4];
        t.odiag += t.sfms0 * t.mm[4 + k][omode];
    }
    for (int k = 0; k < fm; ++k) {
        t.mdiag += t.ffms[0][k][0] * (t.mm[4 + k + 6 * em][4] + t.mm[4 + k + 6 * em + fm][4]);
        t.odiag += t.ffms[0][k][0] * (t.mm[4 + k + 6 * em][omode] + t.mm[4 + k + 6 * em + fm][omode]);
    }
}

// The vertex part of tet_basis::lumpinv (tet_basis/initialize.cpp:642-808) for p >= 2: for
// vertex i, the combination of vertex mode i with the higher modes that touch it (dofs) whose
// mass products with every lower-order mode (constraints) vanish, except the unit coefficient
// of vertex mode i. The solution of vertex 3 gives sfmv and ffmv, vertex 0's interior part
// and sfmv give the constrained vdiag. The constraint and dof lists follow the reference's
// orderings (vertices, edges by local index, faces, interiors); with p <= 4 both have
// (em+1)(em+2)(em+3)/6 entries.
static void tet_vertex_constraints(hp_tet_tables &t) {
    const int em = t.em, fm = t.fm, im = t.im, bm = t.bm, tm = t.T;
    std::vector<int> lind;
    for (int i = 0; i < 4; ++i) lind.push_back(i);
    for (int m = 0; m < 6; ++m)
        for (int j = 4 + em * m; j < 3 + em * (m + 1); ++j) lind.push_back(j);
    for (int m = 0; m < 4; ++m) {
        int ind2 = 0;
        for (int i = 1; i <= em - 1; ++i) {
            for (int j = 1; j <= em - i - 1; ++j) lind.push_back(4 + 6 * em + fm * m + ind2++);
            ++ind2;
        }
    }
    {
        int ind2 = 0;
        for (int i = 1; i <= em - 1; ++i) {
            for (int j = 1; j <= em - i - 1; ++j) {
                for (int k = 1; k <= em - i - j - 1; ++k) lind.push_back(bm + ind2++);
                ++ind2;
            }
            ++ind2;
        }
    }
    auto range = [](std::vector<int> &v, int a, int b) { for (int i = a; i < b; ++i) v.push_back(i); };
    std::vector<int> dind[4];
    dind[0] = {0}; range(dind[0], 4 + 3 * em, 4 + 6 * em); range(dind[0], 4 + 6 * em + fm, tm);
    dind[1] = {1}; range(dind[1], 4 + em, 4 + 4 * em); range(dind[1], 4 + 6 * em, 4 + 6 * em + fm);
    range(dind[1], 4 + 6 * em + 2 * fm, tm);
    dind[2] = {2}; range(dind[2], 4, 4 + em); range(dind[2], 4 + 2 * em, 4 + 3 * em);
    range(dind[2], 4 + 4 * em, 4 + 5 * em); range(dind[2], 4 + 6 * em, 4 + 6 * em + 2 * fm);
    range(dind[2], 4 + 6 * em + 3 * fm, tm);
    dind[3] = {3}; range(dind[3], 4, 4 + 2 * em); range(dind[3], 4 + 5 * em, 4 + 6 * em);
    range(dind[3], 4 + 6 * em, 4 + 6 * em + 3 * fm); range(dind[3], bm, tm);
    const int n = (int)lind.size();
    std::vector<double> x, ifmb0(std::max(im, 1), 0.0);
    for (int i = 0; i < 4; ++i) {
        if ((int)dind[i].size() != n) return;  // not square: beyond the supported p
        std::vector<double> A((size_t)n * n), b(n, 0.0);
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) A[(size_t)j * n + k] = t.mm[lind[j]][dind[i][k]];
        for (int k = 0; k < n; ++k) A[(size_t)i * n + k] = 0.0;
        A[(size_t)i * n] = 1.0;
        b[i] = 1.0;
        if (!dense_solve(n, A, b)) return;
        if (i == 0)
            for (int k = 0; k < im; ++k) ifmb0[k] = -b[k + 3 * em + 3 * fm + 1];
        x = b;
    }
    for (int k = 0; k < em; ++k) {
        t.sfmv[1][k] = -x[k + 1];
        t.sfmv[0][k] = -x[k + 1 + em];
    }
    for (int k = 0; k < fm; ++k) {
        t.ffmv[0][k] = 0.0;
        t.ffmv[1][k] = -x[k + 3 * em + 1 + fm];
        t.ffmv[2][k] = -x[k + 3 * em + 1 + 2 * fm];
    }
    double vd = t.mm[0][0];
    for (int k = 0; k < em; ++k)
        vd -= t.sfmv[1][k] * (t.mm[4 + k + 3 * em][0] + t.mm[4 + k + 4 * em][0] + t.mm[4 + k + 5 * em][0]);
    for (int k = 0; k < fm; ++k)
        vd -= t.ffmv[0][k] * (t.mm[4 + k + 6 * em + fm][0] + t.mm[4 + k + 6 * em + 2 * fm][0] +
                              t.mm[4 + k + 6 * em + 3 * fm][0]);
    for (int k = 0; k < im; ++k) vd -= ifmb0[k] * t.mm[4 + k + 6 * em + 4 * fm][0];
    t.vdiag = 1.0 / vd;
}

extern "C" int hp_tet_basis_build(int p, hp_tet_tables *out) {
    if (!out || p < 1 || p > HP_TET_MAXP) return -1;
    hp_tet_tables &t = *out;
    std::memset(&t, 0, sizeof(t));
    const int G = p + 1, em = p - 1, fm = std::max((p - 1) * (p - 2) / 2, 0);
    const int T = (p + 1) * (p + 2) * (p + 3) / 6;
    const int im = std::max(T - 4 * fm - 6 * em - 4, 0);
    t.p = p; t.G = G; t.T = T; t.em = em; t.fm = fm; t.im = im; t.bm = 4 + 6 * em + 4 * fm;
    t.nmodx = em + 3; t.nmody = 3 + 2 * em + fm; t.nmodz = 2 + 2 * em + fm + im;
    // Gauss rules: Legendre in x, Jacobi(1,0) in y (weights / 2), Jacobi(2,0) in z (weights / 4)
    std::vector<double> a(G + 1), b(G + 1);
    legendre_recur(G + 1, a.data(), b.data());
    gauss_rule(G, a.data(), b.data(), t.xp, t.wtx);
    jacobi_recur(G + 1, 1.0, 0.0, a.data(), b.data());
    gauss_rule(G, a.data(), b.data(), t.yp, t.wty);
    jacobi_recur(G + 1, 2.0, 0.0, a.data(), b.data());
    gauss_rule(G, a.data(), b.data(), t.zp, t.wtz);
    for (int i = 0; i < G; ++i) {
        t.wty[i] *= 0.5;
        t.wtz[i] *= 0.25;
    }
    lagrange_factors(G, t.xp, t.dltx, t.dltx2, t.dltx3);
    lagrange_factors(G, t.yp, t.dlty, t.dlty2, t.dlty3);
    lagrange_factors(G, t.zp, t.dltz, t.dltz2, nullptr);
    TetRecur rc(em);
    for (int i = 0; i < G; ++i) {
        rc.fx(t.xp[i], t.gx[i], t.dgx[i]);
        rc.fy(t.yp[i], t.gy[i], t.dgy[i]);
        rc.fz(t.zp[i], t.gz[i], t.dgz[i]);
        t.x0[i] = 0.5 * (1 + t.xp[i]);
        t.y0[i] = 2.0 / (1 - t.yp[i]);
        t.y1[i] = 0.5 * (1 + t.yp[i]);
        t.z0[i] = 2.0 / (1 - t.zp[i]);
    }
    // mode -> (x, y, z function, sign), in the order of tet_basis::proj
    auto set = [&](int m, int ix, int iy, int iz, double s) {
        t.mx[m] = ix; t.my[m] = iy; t.mz[m] = iz; t.msg[m] = s;
    };
    const int be1 = 4, be2 = be1 + em, be3 = be2 + em, be4 = be3 + em, be5 = be4 + em, be6 = be5 + em;
    const int bf0 = be6 + em, bf1 = bf0 + fm, bf2 = bf1 + fm, bf3 = bf2 + fm, bi = bf3 + fm;
    set(0, 0, 0, 0, 1.0);
    set(1, 0, 1, 1, 1.0);
    set(2, 1, 2, 1, 1.0);
    set(3, 2, 2, 1, 1.0);
    for (int i = 0; i < em; ++i) {
        set(be4 + i, 0, 1, 2 + em + i, 1.0);
        set(be5 + i, 1, 2, 2 + em + i, 1.0);
        set(be6 + i, 2, 2, 2 + em + i, 1.0);
    }
    for (int i = 1; i <= em; ++i) {
        set(be1 + i - 1, i + 2, i + 2, i + 1, 1.0);
        set(be2 + i - 1, 2, 2 + em + i, i + 1, 1.0);
        set(be3 + i - 1, 1, 2 + em + i, i + 1, 1.0);
    }
    {
        int ind2 = 0;
        double s = 1.0;
        for (int i = 1; i <= em; ++i, s = -s)
            for (int j = 1; j <= em - i; ++j, ++ind2) {
                set(bf1 + ind2, i + 2, i + 2, 2 + 2 * em + ind2, s);
                set(bf2 + ind2, 2, 2 + em + i, 2 + 2 * em + ind2, s);
                set(bf3 + ind2, 1, 2 + em + i, 2 + 2 * em + ind2, 1.0);
            }
    }
    {
        int ind2 = 0, ind3 = 0;
        for (int i = 1; i <= em - 1; ++i)
            for (int j = 1; j <= em - i; ++j, ++ind2) {
                set(bf0 + ind2, i + 2, 3 + 2 * em + ind2, i + j + 1, 1.0);
                for (int k = 1; k <= em - i - j; ++k, ++ind3)
                    set(bi + ind3, i + 2, 3 + 2 * em + ind2, 2 + 2 * em + fm + ind3, 1.0);
            }
    }
    // dense operators of proj (r, s, t derivatives through the collapsed coordinates)
    for (int i = 0; i < G; ++i)
        for (int j = 0; j < G; ++j)
            for (int k = 0; k < G; ++k) {
                const int q = (i * G + j) * G + k;
                t.w[q] = t.wtx[i] * t.wty[j] * t.wtz[k];
                for (int m = 0; m < T; ++m) {
                    const double s = t.msg[m];
                    const double gx = t.gx[i][t.mx[m]], dgx = t.dgx[i][t.mx[m]];
                    const double gy = t.gy[j][t.my[m]], dgy = t.dgy[j][t.my[m]];
                    const double gz = t.gz[k][t.mz[m]], dgz = t.dgz[k][t.mz[m]];
                    const double dx = s * dgx * gy * gz * t.y0[j] * t.z0[k];
                    t.F[q][m] = s * gx * gy * gz;
                    t.DX[q][m] = dx;
                    t.DY[q][m] = s * gx * dgy * gz * t.z0[k] + t.x0[i] * dx;
                    t.DZ[q][m] = s * (gx * gy * dgz + t.y1[j] * gx * dgy * gz * t.z0[k]) + t.x0[i] * dx;
                }
            }
    // face basis (proj2d / intgrt2d): mode k = sgn gx(x_i, fx) gy(y_j, fy)
    {
        const int T2 = 3 + 3 * em + fm;
        t.T2 = T2;
        std::vector<int> fx(T2), fy(T2), dyg(T2, 1);  // dyg 0: proj2d's y derivative uses gy
        std::vector<double> fs(T2, 1.0);
        fx[0] = 0; fy[0] = 1;
        fx[1] = 1; fy[1] = 2;
        fx[2] = 2; fy[2] = 2;
        const int be2 = em + 3, be3 = 2 * em + 3, bint = 3 + 3 * em;
        for (int p2 = 3; p2 < em + 3; ++p2) { fx[p2] = p2; fy[p2] = p2; dyg[p2] = 0; }
        for (int i = 0; i < em; ++i) {
            fx[be2 + i] = 2; fy[be2 + i] = 3 + em + i;
            fx[be3 + i] = 1; fy[be3 + i] = 3 + em + i; fs[be3 + i] = (i & 1) ? -1.0 : 1.0;
        }
        int ind2 = 0;
        for (int p2 = 3; p2 < em + 3; ++p2)
            for (int i = 1; i <= em - p2 + 2; ++i, ++ind2) {
                fx[bint + ind2] = p2; fy[bint + ind2] = 3 + 2 * em + ind2; dyg[bint + ind2] = 0;
            }
        for (int i = 0; i < G; ++i)
            for (int j = 0; j < G; ++j) {
                const int q = i * G + j;
                t.W2[q] = t.wtx[i] * t.wty[j];
                for (int k = 0; k < T2; ++k) {
                    const double gx = t.gx[i][fx[k]], dgx = t.dgx[i][fx[k]];
                    const double gy = t.gy[j][fy[k]], dgy = t.dgy[j][fy[k]];
                    const double dx = fs[k] * dgx * gy * t.y0[j];
                    t.F2[q][k] = fs[k] * gx * gy;
                    t.DX2[q][k] = dx;
                    t.DY2[q][k] = fs[k] * gx * (dyg[k] ? dgy : gy) + t.x0[i] * dx;
                }
            }
    }
    // lumpinv's mass matrix and lumped vertex inverse
    const int NQ3 = G * G * G;
    for (int m = 0; m < T; ++m)
        for (int k = 0; k < T; ++k) {
            double acc = 0.0;
            for (int q = 0; q < NQ3; ++q) acc += t.w[q] * t.F[q][m] * t.F[q][k];
            t.mm[m][k] = acc;
        }
    t.vdiag = 1.0 / (t.mm[0][0] + t.mm[0][1] + t.mm[0][2] + t.mm[0][3]);
    if (p >= 2) tet_vertex_constraints(t);
    if (p == 3) tet_edge_cones(t);
    deriv_operator(G, t.dltx, t.dltx2, t.Ax);
    deriv_operator(G, t.dltx, t.dltx3, t.Bx);
    deriv_operator(G, t.dlty, t.dlty2, t.Ay);
    deriv_operator(G, t.dlty, t.dlty3, t.By);
    deriv_operator(G, t.dltz, t.dltz2, t.Az);
    return 0;
}
