/*
 * C entry points around the REFERENCE's own tet_basis class, compiled from its
 * unmodified sources (tet_basis/{initialize,proj,intgrt,proj1d,proj2d,intgrt1d,
 * intgrt2d,ptvalues}.cpp, included from where they lie in the reference tree by
 * the Makefile's -I path) against the blitz shim in ./blitz and the LAPACK
 * stand-ins in lapack_subset.c.
 *
 * TEST INFRASTRUCTURE ONLY. The resulting oracle/_ref/libtet_basis_ref.so pins
 * the project's tet basis tables and dense basis operators against the
 * reference's tables and its sum-factorised proj / intgrt / intgrtrst /
 * derivr / derivs / derivt.
 *
 * Point arrays are compact: value at Gauss point (x i, y j, z k) at
 * (i * G + j) * G + k (the reference's stridex = G*G, stridey = G).
 */
#include "tet_basis.h"
#include "initialize.cpp"
#include "proj.cpp"
#include "intgrt.cpp"
#include "proj1d.cpp"
#include "proj2d.cpp"
#include "intgrt1d.cpp"
#include "intgrt2d.cpp"
#include "ptvalues.cpp"

#include <string>

static tet_basis *g_tet[5] = {nullptr};

static tet_basis *get_tet(int p) {
    if (p < 1 || p > MAXP) return nullptr;
    if (!g_tet[p]) {
        tet_basis *b = new tet_basis;
        b->initialize(p);
        g_tet[p] = b;
    }
    return g_tet[p];
}

extern "C" {

int ref_tet_sizes(int p, int *out) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    out[0] = b->p; out[1] = b->em; out[2] = b->fm; out[3] = b->im; out[4] = b->bm; out[5] = b->tm;
    out[6] = b->nmodx; out[7] = b->nmody; out[8] = b->nmodz; out[9] = b->gpx;
    return 0;
}

/* Copies the named table into out (row-major, the reference's index order) and
 * returns its element count, -1 for an unknown name. */
int ref_tet_get(int p, const char *name, double *out) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    const int g = b->gpx;
    std::string n(name);
    int c = 0;
#define T1(N, EXPR) for (int i = 0; i < (N); ++i) out[c++] = (EXPR);
#define T2(R, C, EXPR) for (int i = 0; i < (R); ++i) for (int j = 0; j < (C); ++j) out[c++] = (EXPR);
    if (n == "gx") { T2(g, b->nmodx, b->gx(i, j)) }
    else if (n == "dgx") { T2(g, b->nmodx, b->dgx(i, j)) }
    else if (n == "gy") { T2(g, b->nmody, b->gy(i, j)) }
    else if (n == "dgy") { T2(g, b->nmody, b->dgy(i, j)) }
    else if (n == "gz") { T2(g, b->nmodz, b->gz(i, j)) }
    else if (n == "dgz") { T2(g, b->nmodz, b->dgz(i, j)) }
    else if (n == "wtx") { T1(g, b->wtx(i)) }
    else if (n == "wty") { T1(g, b->wty(i)) }
    else if (n == "wtz") { T1(g, b->wtz(i)) }
    else if (n == "xp") { T1(g, b->xp(i)) }
    else if (n == "yp") { T1(g, b->yp(i)) }
    else if (n == "zp") { T1(g, b->zp(i)) }
    else if (n == "x0") { T1(g, b->x0(i)) }
    else if (n == "y0") { T1(g, b->y0(i)) }
    else if (n == "y1") { T1(g, b->y1(i)) }
    else if (n == "z0") { T1(g, b->z0(i)) }
    else if (n == "dltx") { T1(g, b->dltx(i)) }
    else if (n == "dlty") { T1(g, b->dlty(i)) }
    else if (n == "dltz") { T1(g, b->dltz(i)) }
    else if (n == "dltx2") { T2(g, g, i == j ? 0.0 : b->dltx2(i, j)) }
    else if (n == "dltx3") { T2(g, g, i == j ? 0.0 : b->dltx3(i, j)) }
    else if (n == "dlty2") { T2(g, g, i == j ? 0.0 : b->dlty2(i, j)) }
    else if (n == "dlty3") { T2(g, g, i == j ? 0.0 : b->dlty3(i, j)) }
    else if (n == "dltz2") { T2(g, g, i == j ? 0.0 : b->dltz2(i, j)) }
    else if (n == "mm") { T2(b->tm, b->tm, b->mm(i, j)) }
    else if (n == "vdiag") { T1(1, b->vdiag) }
    else if (n == "sfmv") { T2(2, b->em, b->sfmv(i, j)) }
    else if (n == "ffmv") { T2(3, b->fm, b->ffmv(i, j)) }
    else if (n == "ffms") { for (int i = 0; i < 3; ++i) for (int k = 0; k < b->fm; ++k) for (int sd = 0; sd < 2; ++sd) out[c++] = b->ffms(i, k, sd); }
    else if (n == "sfms") { T1(1, b->sfms(0)) }
    else if (n == "mdiag") { T1(1, b->mdiag) }
    else if (n == "odiag") { T1(1, b->odiag) }
    else return -1;
#undef T1
#undef T2
    return c;
}

/* proj with r, s, t derivatives of the modal coefficients lin[tm]. */
int ref_tet_proj(int p, const double *lin, double *f, double *dx, double *dy, double *dz) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    const int g = b->gpx;
    b->proj(const_cast<double *>(lin), f, dx, dy, dz, g * g, g);
    return 0;
}

/* intgrt: rslt[tm] = integral of f against every mode (overwrites). */
int ref_tet_intgrt(int p, double *rslt, const double *f) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    const int g = b->gpx;
    b->intgrt(rslt, const_cast<double *>(f), g * g, g);
    return 0;
}

/* intgrtrst: SUBTRACTS the integrals of dx, dy, dz against the r, s, t derivatives. */
int ref_tet_intgrtrst(int p, double *rslt, const double *dx, const double *dy, const double *dz) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    const int g = b->gpx;
    b->intgrtrst(rslt, const_cast<double *>(dx), const_cast<double *>(dy), const_cast<double *>(dz), g * g, g);
    return 0;
}

/* derivr / derivs / derivt: ADD the derivative of the point values f. */
int ref_tet_deriv(int p, int dir, const double *f, double *d) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    const int g = b->gpx;
    double *ff = const_cast<double *>(f);
    if (dir == 0) b->derivr(ff, d, g * g, g);
    else if (dir == 1) b->derivs(ff, d, g * g, g);
    else if (dir == 2) b->derivt(ff, d, g * g, g);
    else return -1;
    return 0;
}

/* proj2d with derivatives of face coefficients lin[3 + 3 em + fm]; f(i, j) at i * G + j */
int ref_tet_proj2d(int p, const double *lin, double *f, double *dx, double *dy) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    b->proj2d(const_cast<double *>(lin), f, dx, dy, b->gpx);
    return 0;
}

/* intgrt2d: rslt[3 + 3 em + fm] (overwritten) */
int ref_tet_intgrt2d(int p, double *rslt, const double *f) {
    tet_basis *b = get_tet(p);
    if (!b) return -1;
    b->intgrt2d(rslt, const_cast<double *>(f), b->gpx);
    return 0;
}

}  // extern "C"
