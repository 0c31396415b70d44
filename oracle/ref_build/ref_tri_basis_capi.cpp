/*
 * C entry points around the REFERENCE's own tri_basis<p,0> class, compiled
 * from its unmodified sources (tri_basis/{initialize,proj,intgrt,proj1d,
 * intgrt1d,ptvalues,probe}.cpp, included from where they lie in the reference
 * tree by the Makefile's -I path) against the blitz shim in ./blitz and the
 * LAPACK stand-ins in lapack_subset.c.
 *
 * TEST INFRASTRUCTURE ONLY. The resulting oracle/_ref/libtri_basis_ref.so is
 * the strongest pin this project has: the reference's basis tables and basis
 * operators, evaluated by the reference's code. Tests compare the shipped
 * library's tables and the oracle's operators against it.
 *
 * Layouts written by ref_tb_get are row-major with the index order of the
 * reference accessor (e.g. "gx" is [gpx][nmodx], "gnwtn" is [tm][gpn]).
 */
#include "tri_basis.h"
#include "intgrt.cpp"
#include "initialize.cpp"
#include "probe.cpp"
#include "intgrt1d.cpp"
#include "proj.cpp"
#include "proj1d.cpp"
#include "ptvalues.cpp"

#include <cstring>
#include <string>

template class tri_basis<1, 0>;
template class tri_basis<2, 0>;
template class tri_basis<3, 0>;
template class tri_basis<4, 0>;
template class tri_basis<5, 0>;
template class tri_basis<6, 0>;
template class tri_basis<7, 0>;
template class tri_basis<8, 0>;

static tri_basis_interface *g_basis[9] = {nullptr};

static tri_basis_interface *get_basis(int p) {
    if (p < 1 || p > 8) return nullptr;
    if (!g_basis[p]) {
        tri_basis_interface *b = nullptr;
        switch (p) {
            case 1: b = new tri_basis<1, 0>; break;
            case 2: b = new tri_basis<2, 0>; break;
            case 3: b = new tri_basis<3, 0>; break;
            case 4: b = new tri_basis<4, 0>; break;
            case 5: b = new tri_basis<5, 0>; break;
            case 6: b = new tri_basis<6, 0>; break;
            case 7: b = new tri_basis<7, 0>; break;
            case 8: b = new tri_basis<8, 0>; break;
        }
        b->initialize();
        g_basis[p] = b;
    }
    return g_basis[p];
}

extern "C" {

int ref_tb_sizes(int p, int *out) {
    tri_basis_interface *b = get_basis(p);
    if (!b) return -1;
    out[0] = b->p(); out[1] = b->sm(); out[2] = b->im(); out[3] = b->tm(); out[4] = b->bm();
    out[5] = b->nmodx(); out[6] = b->gpx(); out[7] = b->gpn(); out[8] = b->ibwth(); out[9] = b->sbwth();
    return 0;
}

/* Copies the named table into out (row-major) and returns its element count. */
int ref_tb_get(int p, const char *name, double *out) {
    tri_basis_interface *b = get_basis(p);
    if (!b) return -1;
    const int gx = b->gpx(), gn = b->gpn(), nx = b->nmodx(), tm = b->tm(), sm = b->sm(), im = b->im(),
              bm = b->bm();
    std::string n(name);
    int c = 0;
#define T2(R, C, EXPR)                                         \
    for (int i = 0; i < (R); ++i)                              \
        for (int j = 0; j < (C); ++j) out[c++] = (EXPR);
    if (n == "gx") { T2(gx, nx, b->gx(i, j)) }
    else if (n == "dgx") { T2(gx, nx, b->dgx(i, j)) }
    else if (n == "wtx") { T2(1, gx, b->wtx(j)) }
    else if (n == "xp") { T2(1, gx, b->xp(j)) }
    else if (n == "x0") { T2(1, gx, b->x0(j)) }
    else if (n == "gxwtx") { T2(nx, gx, b->gxwtx(i, j)) }
    else if (n == "dgxwtx") { T2(nx, gx, b->dgxwtx(i, j)) }
    else if (n == "dltx") { T2(1, gx, b->dltx(j)) }
    else if (n == "dltx1") { T2(gx, gx, (i == j ? 0.0 : b->dltx1(i, j))) }
    else if (n == "gn") { T2(gn, tm, b->gn(i, j)) }
    else if (n == "dgn") { T2(gn, tm, b->dgn(i, j)) }
    else if (n == "wtn") { T2(1, gn, b->wtn(j)) }
    else if (n == "np") { T2(1, gn, b->np(j)) }
    else if (n == "n0") { T2(1, gn, b->n0(j)) }
    else if (n == "gnwtn") { T2(tm, gn, b->gnwtn(i, j)) }
    else if (n == "gnwtnn0") { T2(tm, gn, b->gnwtnn0(i, j)) }
    else if (n == "dgnwtn") { T2(tm, gn, b->dgnwtn(i, j)) }
    else if (n == "dltn") { T2(1, gn, b->dltn(j)) }
    else if (n == "dltn1") { T2(gx, gx, (i == j ? 0.0 : b->dltn1(i, j))) }
    else if (n == "dltn2") { T2(gn, gn, (i == j ? 0.0 : b->dltn2(i, j))) }
    else if (n == "norm") { T2(1, tm, b->norm(j)) }
    else if (n == "vdiag") { out[c++] = b->vdiag(); }
    else if (n == "vdiag1d") { out[c++] = b->vdiag1d(); }
    else if (n == "sfmv") { if (sm > 0) { T2(2, sm, b->sfmv(i, j)) } }
    else if (n == "vfms") { if (sm > 0) { T2(3, sm, b->vfms(i, j)) } }
    else if (n == "sdiag") { if (sm > 0) { T2(1, sm, b->sdiag(j)) } }
    else if (n == "sfms") {
        if (sm > 1)
            for (int ml = 0; ml < sm - 1; ++ml)
                for (int mh = 0; mh < sm; ++mh)
                    for (int sd = 0; sd < 3; ++sd) out[c++] = (ml < mh ? b->sfms(ml, mh, sd) : 0.0);
    }
    else if (n == "ifmb") { if (im > 0) { T2(bm, im, b->ifmb(i, j)) } }
    else if (n == "bfmi") { if (im > 0) { T2(bm, im, b->bfmi(i, j)) } }
    else if (n == "idiag") { if (im > 0) { T2(im, b->ibwth() + 1, b->idiag(i, j)) } }
    else if (n == "msi") { T2(bm, bm, b->msi(i, j)) }
    else if (n == "sfmv1d") { if (sm > 0) { T2(2, sm, b->sfmv1d(i, j)) } }
    else if (n == "vfms1d") { if (sm > 0) { T2(2, sm, b->vfms1d(i, j)) } }
    else if (n == "sdiag1d") { if (sm > 0) { T2(sm, b->sbwth() + 1, b->sdiag1d(i, j)) } }
    else if (n == "dgnorm") {
        for (int s = 0; s < 3; ++s) { T2(tm, gx, b->dgnorm(s, i, j)) }
    }
    else return -2;
#undef T2
    return c;
}

int ref_proj(int p, const double *lin, double *f, double *dx, double *dy, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->proj(lin, f, dx, dy, stride); return 0;
}
int ref_proj_val(int p, const double *lin, double *f, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->proj(lin, f, stride); return 0;
}
int ref_proj_lin(int p, double u1, double u2, double u3, double *f, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->proj(u1, u2, u3, f, stride); return 0;
}
int ref_proj_bdry(int p, const double *lin, double *f, double *dx, double *dy, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->proj_bdry(lin, f, dx, dy, stride); return 0;
}
int ref_derivr(int p, const double *f, double *dr, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->derivr(f, dr, stride); return 0;
}
int ref_derivs(int p, const double *f, double *ds, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->derivs(f, ds, stride); return 0;
}
int ref_intgrt(int p, double *rslt, const double *f, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->intgrt(rslt, f, stride); return 0;
}
int ref_intgrtrs(int p, double *rslt, const double *dx, const double *dy, int stride) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->intgrtrs(rslt, dx, dy, stride); return 0;
}
int ref_proj1d(int p, const double *lin, double *f, double *dx) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->proj1d(lin, f, dx); return 0;
}
int ref_intgrt1d(int p, double *rslt, const double *f) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->intgrt1d(rslt, f); return 0;
}
int ref_intgrtx1d(int p, double *rslt, const double *f) {
    tri_basis_interface *b = get_basis(p); if (!b) return -1;
    b->intgrtx1d(rslt, f); return 0;
}

}  // extern "C"
