/*
 * CPU ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * A scalar FP64 restatement of the reference's 2D element-residual and
 * multistage-smoothing path, used by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg as the checker. It is never linked into or called
 * by the shipped library. Loops follow the reference statement by statement
 * (same accumulation order within an element); only the containers differ.
 *
 * Followed files (reference paths):
 *   tri_basis/proj.cpp:22-199,339-402   proj (3 forms), derivr, derivs
 *   tri_basis/intgrt.cpp:22-158         intgrt, intgrtrs
 *   tri_basis/proj1d.cpp:19-76, intgrt1d.cpp:17-43
 *   tri_hp/gtol.cpp:14-55,156-171,364-402  ugtouht, ugtouht1d, lftog
 *   tri_hp/nstage.cpp:12-110,256-427    rsdl, update
 *   tri_hp/cd/rsdl.cpp:14-154           tri_hp_cd::element_rsdl (CONST_A, straight elements)
 *   tri_hp/ins/rsdl.cpp:17-436          tri_hp_ins::element_rsdl (CALC_TAU2, straight branch :259-433)
 *   tri_hp/hp_boundary.cpp:973-1049     hp_edge_bdry::element_rsdl / rsdl
 *   tri_hp/ins/bdry_ins.h:35-50         bdry_ins::generic::flux
 *   tri_hp/hp_boundary.cpp:680-704      vdirichlet / sdirichlet
 *   tri_hp/cd/setup_preconditioner.cpp:6-97, ins/setup_preconditioner.cpp:9-221 (REFINED_WAY)
 *   tri_hp/setup_preconditioner.cpp:9-399  setup_preconditioner (invert), minvrt, restouht_bdry
 *   utilities/myblas.c:91-120           DPBTRSNU2, restated with its indexing as written
 *   tri_hp/allocate.cpp:496-525         maxres
 *   tri_mesh/tprims.cpp:66-80,224-241   area, inscribedradius
 * Steady problems only (bd(0) = 0): mesh velocity and unsteady sources vanish.
 */
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../include/hp_gpu.h"

namespace {

const int MXGP = HP_MXGP;  // point-array stride
typedef double PtArr[HP_MXGP][HP_MXGP];

struct Basis {
    const hp_basis_tables &t;
    int p, sm, im, tm, bm, nx, gpx, gpn;
    explicit Basis(const hp_basis_tables &tt)
        : t(tt), p(tt.p), sm(tt.sm), im(tt.im), tm(tt.tm), bm(tt.bm), nx(tt.nmodx), gpx(tt.gpx), gpn(tt.gpn) {}

    // tri_basis/proj.cpp:22-119
    void proj(const double *lin, double *f, double *dx, double *dy, int st) const {
        double wk0[HP_MXGP][HP_MXX], wk1[HP_MXGP][HP_MXX], wk2[HP_MXGP][HP_MXX];
        const int bs1 = sm + 3, bs2 = 2 * sm + 3, bint = bm;
        for (int j = 0; j < gpn; ++j) {
            double oeta = t.n0[j];
            wk0[j][0] = lin[0] * t.gn[j][0];
            wk1[j][0] = lin[0] * t.dgn[j][0];
            wk2[j][0] = wk0[j][0] * oeta;
            double l0 = lin[1] * t.gn[j][1], l1 = lin[1] * t.dgn[j][1];
            for (int m = bs2; m < bint; ++m) { l0 += lin[m] * t.gn[j][m]; l1 += lin[m] * t.dgn[j][m]; }
            wk0[j][1] = l0; wk1[j][1] = l1; wk2[j][1] = l0 * oeta;
            l0 = lin[2] * t.gn[j][2]; l1 = lin[2] * t.dgn[j][2];
            for (int m = bs1; m < bs2; ++m) { l0 += lin[m] * t.gn[j][m]; l1 += lin[m] * t.dgn[j][m]; }
            wk0[j][2] = l0; wk1[j][2] = l1; wk2[j][2] = l0 * oeta;
            int ind = bint, bint1 = sm + 2 - 3;
            for (int m = 3; m < bs1; ++m) {
                l0 = lin[m] * t.gn[j][m]; l1 = lin[m] * t.dgn[j][m];
                for (int n = 0; n < bint1; ++n) { l0 += lin[ind + n] * t.gn[j][ind + n]; l1 += lin[ind + n] * t.dgn[j][ind + n]; }
                ind += bint1--;
                wk0[j][m] = l0; wk1[j][m] = l1; wk2[j][m] = l0 * oeta;
            }
        }
        for (int i = 0; i < gpx; ++i) {
            double xp1 = t.x0[i];
            for (int j = 0; j < gpn; ++j) {
                double l0 = wk0[j][0] * t.gx[i][0], l1 = wk1[j][0] * t.gx[i][0], l2 = wk2[j][0] * t.dgx[i][0];
                for (int n = 1; n < nx; ++n) {
                    l0 += wk0[j][n] * t.gx[i][n]; l1 += wk1[j][n] * t.gx[i][n]; l2 += wk2[j][n] * t.dgx[i][n];
                }
                f[i * st + j] = l0;
                dy[i * st + j] = l1 + xp1 * l2;
                dx[i * st + j] = l2;
            }
        }
    }
    // tri_basis/proj.cpp:121-186
    void proj(const double *lin, double *f, int st) const {
        double wk0[HP_MXGP][HP_MXX];
        const int bs1 = sm + 3, bs2 = 2 * sm + 3, bint = bm;
        for (int j = 0; j < gpn; ++j) {
            wk0[j][0] = lin[0] * t.gn[j][0];
            double l0 = lin[1] * t.gn[j][1];
            for (int m = bs2; m < bint; ++m) l0 += lin[m] * t.gn[j][m];
            wk0[j][1] = l0;
            l0 = lin[2] * t.gn[j][2];
            for (int m = bs1; m < bs2; ++m) l0 += lin[m] * t.gn[j][m];
            wk0[j][2] = l0;
            int ind = bint, bint1 = sm + 2 - 3;
            for (int m = 3; m < bs1; ++m) {
                l0 = lin[m] * t.gn[j][m];
                for (int n = 0; n < bint1; ++n) l0 += lin[ind + n] * t.gn[j][ind + n];
                ind += bint1--;
                wk0[j][m] = l0;
            }
        }
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                double l0 = 0.0;
                for (int n = 0; n < nx; ++n) l0 += wk0[j][n] * t.gx[i][n];
                f[i * st + j] = l0;
            }
    }
    // tri_basis/proj.cpp:188-199
    void proj(double u1, double u2, double u3, double *f, int st) const {
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j)
                f[i * st + j] = u1 * t.gx[i][0] * t.gn[j][0] + u2 * t.gx[i][1] * t.gn[j][1] + u3 * t.gx[i][2] * t.gn[j][2];
    }
    // tri_basis/proj.cpp:339-363
    void derivr(const double *f, double *dx, int st) const {
        double wk0[HP_MXGP];
        for (int j = 0; j < gpn; ++j) {
            double ln0 = t.n0[j];
            for (int i = 0; i < gpx; ++i) wk0[i] = f[i * st + j] * t.dltx[i] * ln0;
            for (int i = 0; i < gpx; ++i) {
                double l0 = dx[i * st + j];
                for (int n = 0; n < i; ++n) l0 += (wk0[i] + wk0[n]) * t.dltx1[i][n];
                for (int n = i + 1; n < gpx; ++n) l0 += (wk0[i] + wk0[n]) * t.dltx1[i][n];
                dx[i * st + j] = l0;
            }
        }
    }
    // tri_basis/proj.cpp:365-402
    void derivs(const double *f, double *dy, int st) const {
        double wk0[HP_MXGP];
        for (int j = 0; j < gpn; ++j) {
            double ln0 = t.n0[j];
            for (int i = 0; i < gpx; ++i) wk0[i] = f[i * st + j] * t.dltx[i] * ln0;
            for (int i = 0; i < gpx; ++i) {
                double l0 = dy[i * st + j];
                for (int n = 0; n < i; ++n) l0 += (wk0[i] + wk0[n]) * t.dltn1[i][n];
                for (int n = i + 1; n < gpx; ++n) l0 += (wk0[i] + wk0[n]) * t.dltn1[i][n];
                dy[i * st + j] = l0;
            }
        }
        for (int i = 0; i < gpx; ++i) {
            for (int j = 0; j < gpn; ++j) wk0[j] = f[i * st + j] * t.dltn[j];
            for (int j = 0; j < gpn; ++j) {
                double l0 = dy[i * st + j];
                for (int n = 0; n < j; ++n) l0 += (wk0[j] + wk0[n]) * t.dltn2[j][n];
                for (int n = j + 1; n < gpn; ++n) l0 += (wk0[j] + wk0[n]) * t.dltn2[j][n];
                dy[i * st + j] = l0;
            }
        }
    }
    // tri_basis/intgrt.cpp:22-78
    void intgrt(double *r, const double *f, int st) const {
        double wk0[HP_MXX][HP_MXGP];
        const int bs1 = sm + 3, bs2 = 2 * sm + 3, bint = bm, lsm2 = sm + 2;
        for (int n = 0; n < nx; ++n)
            for (int j = 0; j < gpn; ++j) {
                double l0 = f[0 * st + j] * t.gxwtx[n][0];
                for (int i = 1; i < gpx; ++i) l0 += f[i * st + j] * t.gxwtx[n][i];
                wk0[n][j] = l0;
            }
        for (int m = 0; m < bs1; ++m) {
            double l0 = 0.0;
            for (int j = 0; j < gpn; ++j) l0 += t.gnwtn[m][j] * wk0[m][j];
            r[m] = l0;
        }
        for (int m = bs1; m < bs2; ++m) {
            double l0 = 0.0;
            for (int j = 0; j < gpn; ++j) l0 += t.gnwtn[m][j] * wk0[2][j];
            r[m] = l0;
        }
        for (int m = bs2; m < bint; ++m) {
            double l0 = 0.0;
            for (int j = 0; j < gpn; ++j) l0 += t.gnwtn[m][j] * wk0[1][j];
            r[m] = l0;
        }
        int indx = bint;
        for (int m = 3; m < lsm2; ++m)
            for (int n = 0; n < lsm2 - m; ++n) {
                double l0 = 0.0;
                for (int j = 0; j < gpn; ++j) l0 += t.gnwtn[indx][j] * wk0[m][j];
                r[indx] = l0;
                ++indx;
            }
    }
    // tri_basis/intgrt.cpp:81-158 (accumulates, subtracting)
    void intgrtrs(double *r, const double *dx, const double *dy, int st) const {
        double wk0[HP_MXX][HP_MXGP], wk1[HP_MXX][HP_MXGP], wk2[HP_MXGP][HP_MXGP];
        const int bs1 = sm + 3, bs2 = 2 * sm + 3, bint = bm, lsm2 = sm + 2;
        for (int j = 0; j < gpn; ++j) {
            wk2[0][j] = dx[0 * st + j] + dy[0 * st + j] * t.x0[0];
            double l0 = wk2[0][j] * t.dgxwtx[0][0], l1 = dy[0 * st + j] * t.gxwtx[0][0];
            for (int i = 1; i < gpx; ++i) {
                wk2[i][j] = dx[i * st + j] + dy[i * st + j] * t.x0[i];
                l0 += wk2[i][j] * t.dgxwtx[0][i];
                l1 += dy[i * st + j] * t.gxwtx[0][i];
            }
            wk0[0][j] = l0; wk1[0][j] = l1;
        }
        for (int n = 1; n < nx; ++n)
            for (int j = 0; j < gpn; ++j) {
                double l0 = wk2[0][j] * t.dgxwtx[n][0], l1 = dy[0 * st + j] * t.gxwtx[n][0];
                for (int i = 1; i < gpx; ++i) { l0 += wk2[i][j] * t.dgxwtx[n][i]; l1 += dy[i * st + j] * t.gxwtx[n][i]; }
                wk0[n][j] = l0; wk1[n][j] = l1;
            }
        for (int m = 0; m < bs1; ++m) {
            double l0 = r[m];
            for (int j = 0; j < gpn; ++j) l0 -= t.gnwtnn0[m][j] * wk0[m][j] + t.dgnwtn[m][j] * wk1[m][j];
            r[m] = l0;
        }
        for (int j = 0; j < gpn; ++j) {
            double l0 = wk0[2][j], l1 = wk1[2][j];
            for (int m = bs1; m < bs2; ++m) r[m] -= t.gnwtnn0[m][j] * l0 + t.dgnwtn[m][j] * l1;
            l0 = wk0[1][j]; l1 = wk1[1][j];
            for (int m = bs2; m < bint; ++m) r[m] -= t.gnwtnn0[m][j] * l0 + t.dgnwtn[m][j] * l1;
        }
        int indx = bint;
        for (int m = 3; m < lsm2; ++m) {
            int nmax = lsm2 - m;
            for (int j = 0; j < gpn; ++j) {
                double l0 = wk0[m][j], l1 = wk1[m][j];
                for (int n = 0; n < nmax; ++n) {
                    r[indx] -= t.gnwtnn0[indx][j] * l0 + t.dgnwtn[indx][j] * l1;
                    ++indx;
                }
                indx -= nmax;
            }
            indx += nmax;
        }
    }
    // tri_basis/proj1d.cpp:19-40
    void proj1d(const double *lin, double *f, double *dx) const {
        for (int i = 0; i < gpx; ++i) {
            double l0 = lin[0] * t.gx[i][1] + lin[1] * t.gx[i][2];
            double l1 = lin[0] * t.dgx[i][1] + lin[1] * t.dgx[i][2];
            for (int n = 2; n < sm + 2; ++n) { l0 += lin[n] * t.gx[i][n + 1]; l1 += lin[n] * t.dgx[i][n + 1]; }
            f[i] = l0; dx[i] = l1;
        }
    }
    // tri_basis/intgrt1d.cpp:17-43
    void intgrt1d(double *r, const double *f) const {
        double l0 = 0.0;
        for (int i = 0; i < gpx; ++i) l0 += t.gxwtx[1][i] * f[i];
        r[0] = l0;
        l0 = 0.0;
        for (int i = 0; i < gpx; ++i) l0 += t.gxwtx[2][i] * f[i];
        r[1] = l0;
        for (int n = 3; n < nx; ++n) {
            l0 = 0.0;
            for (int i = 0; i < gpx; ++i) l0 += t.gxwtx[n][i] * f[i];
            r[n - 1] = l0;
        }
    }
};

// utilities/myblas.c:91-120, with its forward/backward index "ba + j" exactly as written
void dpbtrsnu2(const double *abd, int stride, int ordr, int ofdg, double *b, int rhs) {
    for (int i = 0; i < ordr; ++i) {
        int frst = (ofdg - i > 0 ? ofdg - i : 0);
        int ba = -frst;
        for (int j = frst; j < ofdg; ++j)
            for (int n = 0; n < rhs; ++n) b[rhs * i + n] -= abd[i * stride + j] * b[(ba + j) * rhs + n];
        for (int n = 0; n < rhs; ++n) b[i * rhs + n] /= abd[i * stride + ofdg];
    }
    for (int i = ordr - 1; i >= 0; --i) {
        for (int n = 0; n < rhs; ++n) b[i * rhs + n] /= abd[i * stride + ofdg];
        int frst = (ofdg - i > 0 ? ofdg - i : 0);
        int ba = -frst;
        for (int j = frst; j < ofdg; ++j)
            for (int n = 0; n < rhs; ++n) b[rhs * (ba + j) + n] -= abd[i * stride + j] * b[i * rhs + n];
    }
}

}  // namespace

struct or_ctx {
    hp_basis_tables tab;
    Basis *B;
    hp_phys_params ph;
    int NV, npnt, nseg, ntri, sm, im, tm, bm, gpx, gpn;
    std::vector<double> pnts;
    std::vector<int> seg_pnt, seg_tri, tri_pnt, tri_seg, tri_sgn;
    std::vector<int> bseg, bkind;
    std::vector<double> bpibc;
    std::vector<int> vess, sess;  // essential masks
    std::vector<double> bcrd;     // [nbseg][sm][2] curved side position modes (empty: straight)
    std::vector<int> seg_bdry;    // [nseg] boundary index e of a segment or -1
    std::vector<char> curved;     // [ntri] tri.info > -1
    // vsi arrays
    std::vector<double> ugv, ugs, ugi, resv, ress, resi, rrv, rrs, rri, u0v, u0s, u0i;
    std::vector<double> vprcn, sprcn, tprcn, tau;  // tau [ntri][NV] (cd uses column 0)
    // work
    double uht[3][HP_MXTM], lf[3][HP_MXTM];
    // multigrid: a coarse level (mg_kind 1: p-level of the same mesh, 2: h-level at p = 1)
    // keeps its fine level, the restricted residual res0, the FAS source dres, the
    // isfrst flag of mg_source, and for h-levels the transfer weights (ccnnct of the fine
    // vertices f2c_*, fcnnct of the coarse vertices c2f_*) and vug_frst
    or_ctx *fine = nullptr;
    int mg_kind = 0;
    double fadd = 1.0;
    bool isfrst = false;
    std::vector<double> res0v, res0s, res0i, dresv, dress, dresi, vugfrst;
    std::vector<int> f2c_tri, c2f_tri;
    std::vector<double> f2c_wt, c2f_wt;
};

static double tri_area(const or_ctx *c, int t) {  // tri_mesh/tprims.cpp:66-80 (2x area)
    int p0 = c->tri_pnt[3 * t], p1 = c->tri_pnt[3 * t + 1], p2 = c->tri_pnt[3 * t + 2];
    double dx1 = c->pnts[2 * p0] - c->pnts[2 * p2], dy1 = c->pnts[2 * p0 + 1] - c->pnts[2 * p2 + 1];
    double dx2 = c->pnts[2 * p1] - c->pnts[2 * p0], dy2 = c->pnts[2 * p1 + 1] - c->pnts[2 * p0 + 1];
    return dx1 * dy2 - dy1 * dx2;
}
static double inscribedradius(const or_ctx *c, int t) {  // tri_mesh/tprims.cpp:224-241
    int p0 = c->tri_pnt[3 * t], p1 = c->tri_pnt[3 * t + 1], p2 = c->tri_pnt[3 * t + 2];
    double dx1 = c->pnts[2 * p0] - c->pnts[2 * p2], dy1 = c->pnts[2 * p0 + 1] - c->pnts[2 * p2 + 1];
    double dx2 = c->pnts[2 * p1] - c->pnts[2 * p0], dy2 = c->pnts[2 * p1 + 1] - c->pnts[2 * p0 + 1];
    double area = dx1 * dy2 - dy1 * dx2;
    double perim = std::sqrt(dx1 * dx1 + dy1 * dy1) + std::sqrt(dx2 * dx2 + dy2 * dy2) +
                   std::sqrt((dx1 + dx2) * (dx1 + dx2) + (dy1 + dy2) * (dy1 + dy2));
    return area / perim;
}

static bool side_is_curved(const or_ctx *c, int e) {
    if (c->bcrd.empty() || e < 0) return false;
    for (int k = 0; k < 2 * c->sm; ++k)
        if (c->bcrd[(size_t)e * c->sm * 2 + k] != 0.0) return true;
    return false;
}

// tri_hp::crdtocht (gtol.cpp:204-248): vertex coordinates, then per side the boundary
// side's position modes (hp_ebdry->crds) on curved sides and 0 elsewhere; interior 0
static void crdtocht(const or_ctx *c, int tind, double (*cht)[HP_MXTM]) {
    for (int n = 0; n < 2; ++n)
        for (int m = 0; m < HP_MXTM; ++m) cht[n][m] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int n = 0; n < 2; ++n) cht[n][i] = c->pnts[2 * c->tri_pnt[3 * tind + i] + n];
    int cnt = 3;
    for (int i = 0; i < 3; ++i) {
        const int sind = c->tri_seg[3 * tind + i];
        const int e = c->seg_bdry[sind];
        const bool cv = c->seg_tri[2 * sind + 1] < 0 && side_is_curved(c, e);
        for (int m = 0; m < c->sm; ++m, ++cnt)
            for (int n = 0; n < 2; ++n) cht[n][cnt] = cv ? c->bcrd[((size_t)e * c->sm + m) * 2 + n] : 0.0;
    }
}

// Metrics at the quadrature points: curved element (tri.info > -1) from proj_bdry of
// crdtocht (metric.cpp:12-20, proj.cpp:201-281: the projection of a coefficient vector
// whose interior modes are zero), straight element the constant ldcrd.
static void element_metrics(const or_ctx *c, int tind, PtArr (*dc)[2]) {
    const Basis &B = *c->B;
    if (c->curved[tind]) {
        double cht[2][HP_MXTM];
        static PtArr crd;
        crdtocht(c, tind, cht);
        for (int n = 0; n < 2; ++n) B.proj(cht[n], &crd[0][0], &dc[n][0][0][0], &dc[n][1][0][0], MXGP);
        return;
    }
    const int v[3] = {c->tri_pnt[3 * tind], c->tri_pnt[3 * tind + 1], c->tri_pnt[3 * tind + 2]};
    for (int n = 0; n < 2; ++n) {
        const double a = 0.5 * (c->pnts[2 * v[2] + n] - c->pnts[2 * v[1] + n]);
        const double b = 0.5 * (c->pnts[2 * v[0] + n] - c->pnts[2 * v[1] + n]);
        for (int i = 0; i < c->gpx; ++i)
            for (int j = 0; j < c->gpn; ++j) { dc[n][0][i][j] = a; dc[n][1][i][j] = b; }
    }
}

// tri_hp/gtol.cpp:14-55 (fine level: sm == sm0)
static void ugtouht(or_ctx *c, int tind) {
    const int NV = c->NV, sm = c->sm;
    for (int i = 0; i < 3; ++i) {
        int indx = c->tri_pnt[3 * tind + i];
        for (int n = 0; n < NV; ++n) c->uht[n][i] = c->ugv[indx * NV + n];
    }
    int cnt = 3;
    for (int i = 0; i < 3; ++i) {
        int sind = c->tri_seg[3 * tind + i], sign = c->tri_sgn[3 * tind + i], msgn = 1;
        for (int m = 0; m < sm; ++m) {
            for (int n = 0; n < NV; ++n) c->uht[n][cnt] = msgn * c->ugs[(sind * sm + m) * NV + n];
            msgn *= sign;
            ++cnt;
        }
    }
    for (int k = 0; k < c->im; ++k)
        for (int n = 0; n < NV; ++n) c->uht[n][cnt + k] = c->ugi[(tind * c->im + k) * NV + n];
}

// tri_hp/gtol.cpp:364-402
static void lftog(or_ctx *c, int tind, double (*lfl)[HP_MXTM], double *gv, double *gs, double *gi) {
    const int NV = c->NV, sm = c->sm;
    for (int m = 0; m < 3; ++m) {
        int g = c->tri_pnt[3 * tind + m];
        for (int n = 0; n < NV; ++n) gv[g * NV + n] += lfl[n][m];
    }
    if (c->tab.p > 1) {
        int indx = 3;
        for (int i = 0; i < 3; ++i) {
            int sind = c->tri_seg[3 * tind + i], sgn = c->tri_sgn[3 * tind + i], msgn = 1;
            for (int m = 0; m < sm; ++m) {
                for (int n = 0; n < NV; ++n) gs[(sind * sm + m) * NV + n] += msgn * lfl[n][indx];
                msgn *= sgn;
                ++indx;
            }
        }
        indx = c->bm;
        for (int m = 0; m < c->im; ++m) {
            for (int n = 0; n < NV; ++n) gi[(tind * c->im + m) * NV + n] += lfl[n][indx];
            ++indx;
        }
    }
}

// tri_hp/cd/rsdl.cpp:14-154 (CONST_A, steady; curved elements with the metrics of calc_metrics)
static void element_rsdl_cd(or_ctx *c, int tind, int stage, double (*lf_re)[HP_MXTM], double (*lf_im)[HP_MXTM]) {
    const Basis &B = *c->B;
    const int gpx = c->gpx, gpn = c->gpn;
    const hp_phys_params &ph = c->ph;
    static PtArr crd[2], u, du0, du1, res, cjcb, cv00, cv01, e00, e01;
    static PtArr dc[2][2];
    int v[3] = {c->tri_pnt[3 * tind], c->tri_pnt[3 * tind + 1], c->tri_pnt[3 * tind + 2]};
    for (int n = 0; n < 2; ++n)
        B.proj(c->pnts[2 * v[0] + n], c->pnts[2 * v[1] + n], c->pnts[2 * v[2] + n], &crd[n][0][0], MXGP);
    element_metrics(c, tind, dc);
    const double mv0 = 0.0, mv1 = 0.0;  // bd(0)*(crd - dxdt) with bd(0) = 0
    B.proj(&c->uht[0][0], &u[0][0], &du0[0][0], &du1[0][0], MXGP);
    for (int i = 0; i < B.tm; ++i) { lf_re[0][i] = 0.0; lf_im[0][i] = 0.0; }
    for (int i = 0; i < gpx; ++i)
        for (int j = 0; j < gpn; ++j) {
            double fluxx = ph.rhocv * (ph.ax - mv0) * u[i][j];
            double fluxy = ph.rhocv * (ph.ay - mv1) * u[i][j];
            cv00[i][j] = +dc[1][1][i][j] * fluxx - dc[0][1][i][j] * fluxy;
            cv01[i][j] = -dc[1][0][i][j] * fluxx + dc[0][0][i][j] * fluxy;
        }
    B.intgrtrs(&lf_im[0][0], &cv00[0][0], &cv01[0][0], MXGP);
    const double beta = ph.beta[stage];
    if (beta > 0.0) {
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                cjcb[i][j] = dc[0][0][i][j] * dc[1][1][i][j] - dc[1][0][i][j] * dc[0][1][i][j];
                res[i][j] = ph.rhocv * ph.bd0 * u[i][j] * cjcb[i][j] + 0.0;
                res[i][j] -= cjcb[i][j] * ph.src;
            }
        B.intgrt(&lf_re[0][0], &res[0][0], MXGP);
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                cjcb[i][j] = ph.kcond / cjcb[i][j];
                double v0000 = -cjcb[i][j] * (dc[1][1][i][j] * dc[1][1][i][j] + dc[0][1][i][j] * dc[0][1][i][j]);
                double v0011 = -cjcb[i][j] * (dc[1][0][i][j] * dc[1][0][i][j] + dc[0][0][i][j] * dc[0][0][i][j]);
                double v0001 = cjcb[i][j] * (dc[1][1][i][j] * dc[1][0][i][j] + dc[0][1][i][j] * dc[0][0][i][j]);
                e00[i][j] = +v0000 * du0[i][j] + v0001 * du1[i][j];
                e01[i][j] = +v0001 * du0[i][j] + v0011 * du1[i][j];
                cv00[i][j] += e00[i][j];
                cv01[i][j] += e01[i][j];
            }
        B.derivr(&cv00[0][0], &res[0][0], MXGP);
        B.derivs(&cv01[0][0], &res[0][0], MXGP);
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                double tres = c->tau[tind * c->NV] * res[i][j];
                e00[i][j] -= (dc[1][1][i][j] * (ph.ax - mv0) - dc[0][1][i][j] * (ph.ay - mv1)) * tres;
                e01[i][j] -= (-dc[1][0][i][j] * (ph.ax - mv0) + dc[0][0][i][j] * (ph.ay - mv1)) * tres;
            }
        B.intgrtrs(&lf_re[0][0], &e00[0][0], &e01[0][0], MXGP);
        for (int i = 0; i < B.tm; ++i) lf_re[0][i] *= beta;
    }
}

// tri_hp/ins/rsdl.cpp:17-80 + the curved (:83-258) and straight (:259-433) branches (CALC_TAU2,
// steady); both are the same arithmetic on metrics per point, constant when straight
static void element_rsdl_ins(or_ctx *c, int tind, int stage, double (*lf_re)[HP_MXTM], double (*lf_im)[HP_MXTM]) {
    const Basis &B = *c->B;
    const int NV = 3, gpx = c->gpx, gpn = c->gpn;
    const hp_phys_params &ph = c->ph;
    static PtArr crd[2], u[3], du[3][2], res[3], cv[2][2], df[2][2], mvel[2];
    static PtArr dc[2][2];
    int v[3] = {c->tri_pnt[3 * tind], c->tri_pnt[3 * tind + 1], c->tri_pnt[3 * tind + 2]};
    const double rhobd0 = ph.rho * ph.bd0, lmu = ph.mu;
    for (int n = 0; n < 2; ++n)
        B.proj(c->pnts[2 * v[0] + n], c->pnts[2 * v[1] + n], c->pnts[2 * v[2] + n], &crd[n][0][0], MXGP);
    element_metrics(c, tind, dc);
    for (int i = 0; i < gpx; ++i)
        for (int j = 0; j < gpn; ++j) { mvel[0][i][j] = 0.0; mvel[1][i][j] = 0.0; }
    const double beta = ph.beta[stage];
    if (beta > 0.0) {
        for (int n = 0; n < NV - 1; ++n) B.proj(&c->uht[n][0], &u[n][0][0], &du[n][0][0][0], &du[n][1][0][0], MXGP);
        B.proj(&c->uht[NV - 1][0], &u[NV - 1][0][0], MXGP);
    } else {
        for (int n = 0; n < NV; ++n) B.proj(&c->uht[n][0], &u[n][0][0], MXGP);
    }
    for (int n = 0; n < NV; ++n)
        for (int i = 0; i < B.tm; ++i) { lf_re[n][i] = 0.0; lf_im[n][i] = 0.0; }

    for (int i = 0; i < gpx; ++i)
        for (int j = 0; j < gpn; ++j) {
            double fluxx = ph.rho * (u[0][i][j] - mvel[0][i][j]);
            double fluxy = ph.rho * (u[1][i][j] - mvel[1][i][j]);
            du[NV - 1][0][i][j] = +dc[1][1][i][j] * fluxx - dc[0][1][i][j] * fluxy;
            du[NV - 1][1][i][j] = -dc[1][0][i][j] * fluxx + dc[0][0][i][j] * fluxy;
            for (int n = 0; n < NV - 1; ++n) {
                cv[n][0][i][j] = u[n][i][j] * du[NV - 1][0][i][j];
                cv[n][1][i][j] = u[n][i][j] * du[NV - 1][1][i][j];
            }
            cv[0][0][i][j] += dc[1][1][i][j] * u[NV - 1][i][j];
            cv[0][1][i][j] -= dc[1][0][i][j] * u[NV - 1][i][j];
            cv[1][0][i][j] -= dc[0][1][i][j] * u[NV - 1][i][j];
            cv[1][1][i][j] += dc[0][0][i][j] * u[NV - 1][i][j];
        }
    for (int n = 0; n < NV - 1; ++n) B.intgrtrs(&lf_im[n][0], &cv[n][0][0][0], &cv[n][1][0][0], MXGP);
    B.intgrtrs(&lf_im[NV - 1][0], &du[NV - 1][0][0][0], &du[NV - 1][1][0][0], MXGP);

    if (beta > 0.0) {
        static PtArr cjcbp;
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                const double cjcb = dc[0][0][i][j] * dc[1][1][i][j] - dc[1][0][i][j] * dc[0][1][i][j];
                cjcbp[i][j] = cjcb;
                const double cjcbi = lmu / cjcb;
                double rhorbd0 = rhobd0 * cjcb;
                double visc[2][2][2][2];
                visc[0][0][0][0] = -cjcbi * (2. * dc[1][1][i][j] * dc[1][1][i][j] + dc[0][1][i][j] * dc[0][1][i][j]);
                visc[0][0][1][1] = -cjcbi * (2. * dc[1][0][i][j] * dc[1][0][i][j] + dc[0][0][i][j] * dc[0][0][i][j]);
                visc[0][0][0][1] = cjcbi * (2. * dc[1][1][i][j] * dc[1][0][i][j] + dc[0][1][i][j] * dc[0][0][i][j]);
                visc[1][1][0][0] = -cjcbi * (dc[1][1][i][j] * dc[1][1][i][j] + 2. * dc[0][1][i][j] * dc[0][1][i][j]);
                visc[1][1][1][1] = -cjcbi * (dc[1][0][i][j] * dc[1][0][i][j] + 2. * dc[0][0][i][j] * dc[0][0][i][j]);
                visc[1][1][0][1] = cjcbi * (dc[1][1][i][j] * dc[1][0][i][j] + 2. * dc[0][1][i][j] * dc[0][0][i][j]);
                visc[0][1][0][0] = cjcbi * dc[0][1][i][j] * dc[1][1][i][j];
                visc[0][1][1][1] = cjcbi * dc[0][0][i][j] * dc[1][0][i][j];
                visc[0][1][0][1] = -cjcbi * dc[0][1][i][j] * dc[1][0][i][j];
                visc[0][1][1][0] = -cjcbi * dc[0][0][i][j] * dc[1][1][i][j];
                const double v0010 = visc[0][0][0][1];  // viscI0II0II1II0I
                const double v1110 = visc[1][1][0][1];  // viscI1II1II1II0I
                const double v1000 = visc[0][1][0][0], v1011 = visc[0][1][1][1], v1001 = visc[0][1][1][0],
                             v1010 = visc[0][1][0][1];

                for (int n = 0; n < NV - 1; ++n) res[n][i][j] = rhorbd0 * u[n][i][j] + 0.0;
                res[NV - 1][i][j] = rhorbd0 + 0.0;
                df[0][0][i][j] = (+visc[0][0][0][0] * du[0][0][i][j] + visc[0][1][0][0] * du[1][0][i][j] +
                                  visc[0][0][0][1] * du[0][1][i][j] + visc[0][1][0][1] * du[1][1][i][j]);
                df[0][1][i][j] = (+v0010 * du[0][0][i][j] + visc[0][1][1][0] * du[1][0][i][j] +
                                  visc[0][0][1][1] * du[0][1][i][j] + visc[0][1][1][1] * du[1][1][i][j]);
                df[1][0][i][j] = (+v1000 * du[0][0][i][j] + visc[1][1][0][0] * du[1][0][i][j] +
                                  v1001 * du[0][1][i][j] + visc[1][1][0][1] * du[1][1][i][j]);
                df[1][1][i][j] = (+v1010 * du[0][0][i][j] + v1110 * du[1][0][i][j] + v1011 * du[0][1][i][j] +
                                  visc[1][1][1][1] * du[1][1][i][j]);
                for (int n = 0; n < NV - 1; ++n) {
                    cv[n][0][i][j] += df[n][0][i][j];
                    cv[n][1][i][j] += df[n][1][i][j];
                }
            }
        for (int n = 0; n < NV; ++n) B.intgrt(&lf_re[n][0], &res[n][0][0], MXGP);
        for (int n = 0; n < NV - 1; ++n) {
            B.derivr(&cv[n][0][0][0], &res[n][0][0], MXGP);
            B.derivs(&cv[n][1][0][0], &res[n][0][0], MXGP);
        }
        B.derivr(&du[NV - 1][0][0][0], &res[NV - 1][0][0], MXGP);
        B.derivs(&du[NV - 1][1][0][0], &res[NV - 1][0][0], MXGP);

        double h = inscribedradius(c, tind) / (0.25 * (B.p + 1) * (B.p + 1));
        for (int i = 0; i < gpx; ++i)
            for (int j = 0; j < gpn; ++j) {
                double q = std::pow(u[0][i][j] - 0.5 * mvel[0][i][j], 2.0) + std::pow(u[1][i][j] - 0.5 * mvel[1][i][j], 2.0);
                double rho = ph.rho, nu = ph.mu / rho;
                double gam = 3.0 * q + (0.5 * h * ph.bd0 + 2. * nu / h) * (0.5 * h * ph.bd0 + 2. * nu / h);
                if (ph.mu + ph.bd0 == 0.0) gam = std::max(gam, 0.1);
                double tau0 = ph.adis * h / (cjcbp[i][j] * std::sqrt(gam));
                double tau2 = std::sqrt(q) * tau0;
                c->tau[tind * 3 + 0] = tau0;
                c->tau[tind * 3 + NV - 1] = tau2;
                double tr0 = tau0 * res[0][i][j], tr1 = tau0 * res[1][i][j], tr2 = tau2 * res[NV - 1][i][j];
                df[0][0][i][j] -= (dc[1][1][i][j] * (2 * u[0][i][j] - mvel[0][i][j]) - dc[0][1][i][j] * (u[1][i][j] - mvel[1][i][j])) * tr0 -
                                  dc[0][1][i][j] * u[0][i][j] * tr1 + dc[1][1][i][j] * tr2;
                df[0][1][i][j] -= (-dc[1][0][i][j] * (2 * u[0][i][j] - mvel[0][i][j]) + dc[0][0][i][j] * (u[1][i][j] - mvel[1][i][j])) * tr0 +
                                  dc[0][0][i][j] * u[0][i][j] * tr1 - dc[1][0][i][j] * tr2;
                df[1][0][i][j] -= +dc[1][1][i][j] * u[1][i][j] * tr0 +
                                  (dc[1][1][i][j] * (u[0][i][j] - mvel[0][i][j]) - dc[0][1][i][j] * (2. * u[1][i][j] - mvel[1][i][j])) * tr1 -
                                  dc[0][1][i][j] * tr2;
                df[1][1][i][j] -= -dc[1][0][i][j] * u[1][i][j] * tr0 +
                                  (-dc[1][0][i][j] * (u[0][i][j] - mvel[0][i][j]) + dc[0][0][i][j] * (2. * u[1][i][j] - mvel[1][i][j])) * tr1 +
                                  dc[0][0][i][j] * tr2;
                du[NV - 1][0][i][j] = -(dc[1][1][i][j] * tr0 - dc[0][1][i][j] * tr1);
                du[NV - 1][1][i][j] = -(-dc[1][0][i][j] * tr0 + dc[0][0][i][j] * tr1);
            }
        for (int n = 0; n < NV - 1; ++n) B.intgrtrs(&lf_re[n][0], &df[n][0][0][0], &df[n][1][0][0], MXGP);
        B.intgrtrs(&lf_re[NV - 1][0], &du[NV - 1][0][0][0], &du[NV - 1][1][0][0], MXGP);
        for (int n = 0; n < NV; ++n)
            for (int i = 0; i < B.tm; ++i) lf_re[n][i] *= beta;
    }
}

// hp_edge_bdry::rsdl for bdry_ins::generic (hp_boundary.cpp:973-1049, ins/bdry_ins.h:35-50)
static void bdry_rsdl(or_ctx *c) {
    const Basis &B = *c->B;
    const int NV = c->NV, sm = c->sm;
    for (int e = 0; e < (int)c->bseg.size(); ++e) {
        if ((c->bkind[e] & HP_BC_FLUX_MASK) != HP_BC_FLUX_INS_GENERIC) continue;
        int sind = c->bseg[e];
        int v0 = c->seg_pnt[2 * sind], v1 = c->seg_pnt[2 * sind + 1];
        double u1d[3][HP_MXX], cht[2][HP_MXX];
        for (int n = 0; n < NV; ++n) {
            u1d[n][0] = c->ugv[v0 * NV + n];
            u1d[n][1] = c->ugv[v1 * NV + n];
            for (int m = 0; m < sm; ++m) u1d[n][m + 2] = c->ugs[(sind * sm + m) * NV + n];
        }
        const bool cv = side_is_curved(c, e);
        for (int n = 0; n < 2; ++n) {  // crdtocht1d (gtol.cpp:296-327)
            cht[n][0] = c->pnts[2 * v0 + n];
            cht[n][1] = c->pnts[2 * v1 + n];
            for (int m = 0; m < sm; ++m) cht[n][m + 2] = cv ? c->bcrd[((size_t)e * sm + m) * 2 + n] : 0.0;
        }
        double crd[2][HP_MXGP], dcrd[2][HP_MXGP], uu[3][HP_MXGP], dum[HP_MXGP], rr[3][HP_MXGP], lf1[3][HP_MXX];
        for (int n = 0; n < 2; ++n) B.proj1d(cht[n], crd[n], dcrd[n]);
        for (int n = 0; n < NV; ++n) B.proj1d(u1d[n], uu[n], dum);
        for (int k = 0; k < c->gpx; ++k) {
            double nrm0 = dcrd[1][k], nrm1 = -dcrd[0][k];
            double jcb = std::sqrt(nrm0 * nrm0 + nrm1 * nrm1);
            nrm0 /= jcb; nrm1 /= jcb;
            double mv0 = 0.0, mv1 = 0.0;
            double flx[3];
            flx[NV - 1] = c->ph.rho * ((uu[0][k] - mv0) * nrm0 + (uu[1][k] - mv1) * nrm1);
            double pb = c->bpibc[e * c->gpx + k];
            flx[0] = flx[NV - 1] * uu[0][k] + pb * nrm0;
            flx[1] = flx[NV - 1] * uu[1][k] + pb * nrm1;
            for (int n = 0; n < NV; ++n) rr[n][k] = flx[n] * jcb;
        }
        for (int n = 0; n < NV; ++n) B.intgrt1d(lf1[n], rr[n]);
        for (int n = 0; n < NV; ++n) c->resv[v0 * NV + n] += lf1[n][0];
        for (int n = 0; n < NV; ++n) c->resv[v1 * NV + n] += lf1[n][1];
        for (int k = 0; k < sm; ++k)
            for (int n = 0; n < NV; ++n) c->ress[(sind * sm + k) * NV + n] += lf1[n][k + 2];
    }
}

extern "C" {

or_ctx *or_create(const hp_mesh_desc *m, const hp_basis_tables *b, const hp_phys_params *ph) {
    or_ctx *c = new or_ctx();
    c->tab = *b;
    c->B = new Basis(c->tab);
    c->ph = *ph;
    c->NV = (ph->physics == HP_PHYS_INS ? 3 : 1);
    c->npnt = m->npnt; c->nseg = m->nseg; c->ntri = m->ntri;
    c->sm = b->sm; c->im = b->im; c->tm = b->tm; c->bm = b->bm; c->gpx = b->gpx; c->gpn = b->gpn;
    c->pnts.assign(m->pnts, m->pnts + 2 * m->npnt);
    c->seg_pnt.assign(m->seg_pnt, m->seg_pnt + 2 * m->nseg);
    c->seg_tri.assign(m->seg_tri, m->seg_tri + 2 * m->nseg);
    c->tri_pnt.assign(m->tri_pnt, m->tri_pnt + 3 * m->ntri);
    c->tri_seg.assign(m->tri_seg, m->tri_seg + 3 * m->ntri);
    c->tri_sgn.assign(m->tri_sgn, m->tri_sgn + 3 * m->ntri);
    c->bseg.assign(m->bseg, m->bseg + m->nbseg);
    c->bkind.assign(m->bseg_kind, m->bseg_kind + m->nbseg);
    if (m->bseg_pibc) c->bpibc.assign(m->bseg_pibc, m->bseg_pibc + m->nbseg * b->gpx);
    else c->bpibc.assign(m->nbseg * b->gpx, 0.0);
    c->seg_bdry.assign(m->nseg, -1);
    for (int e = 0; e < m->nbseg; ++e) c->seg_bdry[m->bseg[e]] = e;
    if (m->bseg_crd && b->sm > 0) c->bcrd.assign(m->bseg_crd, m->bseg_crd + (size_t)m->nbseg * b->sm * 2);
    // tri_hp::metric::setinfo (metric.cpp:44-70): owners of curved boundary sides, p > 1
    c->curved.assign(m->ntri, 0);
    for (int e = 0; e < m->nbseg; ++e)
        if (side_is_curved(c, e)) c->curved[m->seg_tri[2 * m->bseg[e]]] = 1;
    c->vess.assign(m->npnt, 0);
    c->sess.assign(m->nseg, 0);
    for (int e = 0; e < m->nbseg; ++e) {
        int s = m->bseg[e], mask = m->bseg_kind[e] & 0xFF;
        c->sess[s] |= mask;
        c->vess[m->seg_pnt[2 * s]] |= mask;
        c->vess[m->seg_pnt[2 * s + 1]] |= mask;
    }
    const int NV = c->NV;
    size_t nv = (size_t)c->npnt * NV, ns = (size_t)c->nseg * c->sm * NV, ni = (size_t)c->ntri * c->im * NV;
    for (auto *v : {&c->ugv, &c->resv, &c->rrv, &c->u0v}) v->assign(nv, 0.0);
    for (auto *v : {&c->ugs, &c->ress, &c->rrs, &c->u0s}) v->assign(ns, 0.0);
    for (auto *v : {&c->ugi, &c->resi, &c->rri, &c->u0i}) v->assign(ni, 0.0);
    c->vprcn.assign((size_t)c->npnt * NV, 0.0);
    c->sprcn.assign((size_t)c->nseg * NV, 0.0);
    c->tprcn.assign((size_t)c->ntri * NV, 0.0);
    c->tau.assign((size_t)c->ntri * NV, 0.0);
    return c;
}

void or_destroy(or_ctx *c) { delete c->B; delete c; }

void or_set_state(or_ctx *c, const double *v, const double *s, const double *i) {
    std::copy(v, v + c->ugv.size(), c->ugv.begin());
    if (s) std::copy(s, s + c->ugs.size(), c->ugs.begin());
    if (i) std::copy(i, i + c->ugi.size(), c->ugi.begin());
}
void or_get_state(or_ctx *c, double *v, double *s, double *i) {
    std::copy(c->ugv.begin(), c->ugv.end(), v);
    if (s) std::copy(c->ugs.begin(), c->ugs.end(), s);
    if (i) std::copy(c->ugi.begin(), c->ugi.end(), i);
}
void or_get_res(or_ctx *c, double *v, double *s, double *i) {
    std::copy(c->resv.begin(), c->resv.end(), v);
    if (s) std::copy(c->ress.begin(), c->ress.end(), s);
    if (i) std::copy(c->resi.begin(), c->resi.end(), i);
}
void or_get_prcn(or_ctx *c, double *vp, double *sp, double *tp, double *tau) {
    std::copy(c->vprcn.begin(), c->vprcn.end(), vp);
    if (sp) std::copy(c->sprcn.begin(), c->sprcn.end(), sp);
    if (tp) std::copy(c->tprcn.begin(), c->tprcn.end(), tp);
    if (tau) std::copy(c->tau.begin(), c->tau.end(), tau);
}
void or_set_prcn(or_ctx *c, const double *vp, const double *sp, const double *tp, const double *tau) {
    std::copy(vp, vp + c->vprcn.size(), c->vprcn.begin());
    std::copy(sp, sp + c->sprcn.size(), c->sprcn.begin());
    std::copy(tp, tp + c->tprcn.size(), c->tprcn.begin());
    std::copy(tau, tau + c->tau.size(), c->tau.begin());
}

// tri_hp::mg_source (nstage.cpp:113-129) on a coarse level: on the first residual after
// mg_restrict (isfrst) the driving term dres = fadd*res0 - res, then res += dres
static void mg_source(or_ctx *c) {
    if (c->isfrst) {
        for (size_t k = 0; k < c->resv.size(); ++k) c->dresv[k] = c->fadd * c->res0v[k] - c->resv[k];
        for (size_t k = 0; k < c->ress.size(); ++k) c->dress[k] = c->fadd * c->res0s[k] - c->ress[k];
        for (size_t k = 0; k < c->resi.size(); ++k) c->dresi[k] = c->fadd * c->res0i[k] - c->resi[k];
        c->isfrst = false;
    }
    for (size_t k = 0; k < c->resv.size(); ++k) c->resv[k] += c->dresv[k];
    for (size_t k = 0; k < c->ress.size(); ++k) c->ress[k] += c->dress[k];
    for (size_t k = 0; k < c->resi.size(); ++k) c->resi[k] += c->dresi[k];
}

// tri_hp::rsdl(stage) (nstage.cpp:12-110), one block; on a coarse level with mg_source
void or_rsdl(or_ctx *c, int stage) {
    const int nstage = c->ph.nstage;
    if (stage < nstage) {
        double omb = 1.0 - c->ph.beta[stage];
        std::fill(c->resv.begin(), c->resv.end(), 0.0);
        for (auto &x : c->rrv) x *= omb;
        std::fill(c->ress.begin(), c->ress.end(), 0.0);
        for (auto &x : c->rrs) x *= omb;
        std::fill(c->resi.begin(), c->resi.end(), 0.0);
        for (auto &x : c->rri) x *= omb;
    } else {
        for (auto *v : {&c->resv, &c->rrv, &c->ress, &c->rrs, &c->resi, &c->rri}) std::fill(v->begin(), v->end(), 0.0);
    }
    double lf_re[3][HP_MXTM], lf_im[3][HP_MXTM];
    for (int tind = 0; tind < c->ntri; ++tind) {
        ugtouht(c, tind);
        if (c->ph.physics == HP_PHYS_INS) element_rsdl_ins(c, tind, stage, lf_re, lf_im);
        else element_rsdl_cd(c, tind, stage, lf_re, lf_im);
        lftog(c, tind, lf_im, c->resv.data(), c->ress.data(), c->resi.data());
        lftog(c, tind, lf_re, c->rrv.data(), c->rrs.data(), c->rri.data());
    }
    for (size_t k = 0; k < c->resv.size(); ++k) c->resv[k] += c->rrv[k];
    for (size_t k = 0; k < c->ress.size(); ++k) c->ress[k] += c->rrs[k];
    for (size_t k = 0; k < c->resi.size(); ++k) c->resi[k] += c->rri[k];
    bdry_rsdl(c);
    if (c->mg_kind) mg_source(c);
}

// tri_hp_{cd,ins}::setup_preconditioner + tri_hp::setup_preconditioner (diagonal)
int or_setup_preconditioner(or_ctx *c) {
    const Basis &B = *c->B;
    const int NV = c->NV;
    const hp_phys_params &ph = c->ph;
    int err = 0;
    std::fill(c->vprcn.begin(), c->vprcn.end(), 0.0);
    std::fill(c->sprcn.begin(), c->sprcn.end(), 0.0);
    static PtArr u[2];
    for (int tind = 0; tind < c->ntri; ++tind) {
        double jcb = 0.25 * tri_area(c, tind);
        int v[3] = {c->tri_pnt[3 * tind], c->tri_pnt[3 * tind + 1], c->tri_pnt[3 * tind + 2]};
        double hmax = 0.0, h;
        for (int j = 0; j < 3; ++j) {
            h = std::pow(c->pnts[2 * v[j]] - c->pnts[2 * v[(j + 1) % 3]], 2.0) +
                std::pow(c->pnts[2 * v[j] + 1] - c->pnts[2 * v[(j + 1) % 3] + 1], 2.0);
            hmax = (h > hmax ? h : hmax);
        }
        const double p1 = 0.25 * (B.p + 1) * (B.p + 1);
        if (ph.physics == HP_PHYS_CD) {
            // cd/setup_preconditioner.cpp:25-82
            hmax = std::sqrt(hmax);
            if (!(jcb > 0.0)) { err = 1; break; }
            h = 4. * jcb / (p1 * hmax);
            double qmax = 0.0;
            for (int j = 0; j < 3; ++j) {
                double q = std::pow(ph.ax - 0.0, 2.0) + std::pow(ph.ay - 0.0, 2.0);
                qmax = std::max(qmax, q);
            }
            double q = std::sqrt(qmax);
            double alpha = ph.kcond / ph.rhocv;
            double lam1 = (q + 1.5 * alpha / h + h * ph.bd0);
            c->tau[tind * NV] = ph.adis * h / (jcb * lam1);
            jcb *= ph.rhocv * lam1 / h;
            c->tprcn[tind * NV] = jcb;
        } else {
            // ins/setup_preconditioner.cpp:33-174 (REFINED_WAY, straight element)
            ugtouht(c, tind);
            for (int n = 0; n < 2; ++n) B.proj(&c->uht[n][0], &u[n][0][0], MXGP);
            double qmax = 0.0;
            for (int i = 0; i < c->gpx; ++i)
                for (int j = 0; j < c->gpn; ++j) {
                    double q = std::pow(u[0][i][j] - 0.5 * 0.0, 2.0) + std::pow(u[1][i][j] - 0.5 * 0.0, 2.0);
                    qmax = std::max(qmax, q);
                }
            if (c->curved[tind]) {
                // curved element (ins/setup_preconditioner.cpp:45-87)
                static PtArr dc[2][2];
                element_metrics(c, tind, dc);
                double jcbmin = jcb, hm = 0.0;
                for (int i = 0; i < c->gpx; ++i)
                    for (int j = 0; j < c->gpn; ++j) {
                        jcbmin = std::min(jcbmin, dc[0][0][i][j] * dc[1][1][i][j] - dc[1][0][i][j] * dc[0][1][i][j]);
                        double hh = 0.0;
                        for (int n = 0; n < 2; ++n) hh += dc[n][0][i][j] * dc[n][0][i][j];
                        hm = std::max(hh, hm);
                        hh = 0.0;
                        for (int n = 0; n < 2; ++n) hh += dc[n][1][i][j] * dc[n][1][i][j];
                        hm = std::max(hh, hm);
                        hh = 0.0;
                        for (int n = 0; n < 2; ++n) hh += (dc[n][1][i][j] - dc[n][0][i][j]) * (dc[n][1][i][j] - dc[n][0][i][j]);
                        hm = std::max(hh, hm);
                    }
                hmax = 2. * std::sqrt(hm);
                h = 4. * jcbmin / (p1 * hmax);
                hmax = hmax / p1;
            } else {
                hmax = std::sqrt(hmax);
                h = 4. * jcb / (p1 * hmax);
                hmax = hmax / p1;
            }
            if (!(h > 0.0)) { err = 1; break; }
            if (std::isnan(qmax)) { err = 1; break; }
            double nu = ph.mu / ph.rho;
            double gam = 3.0 * qmax + (0.5 * hmax * ph.bd0 + 2. * nu / hmax) * (0.5 * hmax * ph.bd0 + 2. * nu / hmax);
            if (ph.mu + ph.bd0 == 0.0) gam = std::max(gam, 0.1);
            double q = std::sqrt(qmax);
            double lam1 = q + std::sqrt(qmax + gam);
            c->tau[tind * NV + 0] = ph.adis * h / (jcb * std::sqrt(gam));
            c->tau[tind * NV + NV - 1] = qmax * c->tau[tind * NV + 0];
            jcb *= 2. * nu * (1. / (hmax * hmax) + 1. / (h * h)) + 3 * lam1 / h;
            c->tprcn[tind * NV + 0] = ph.rho * jcb;
            c->tprcn[tind * NV + 1] = ph.rho * jcb;
            c->tprcn[tind * NV + 2] = jcb / gam;
        }
        for (int i = 0; i < 3; ++i) {
            for (int n = 0; n < NV; ++n) c->vprcn[v[i] * NV + n] += c->tprcn[tind * NV + n];
            if (c->sm > 0) {
                int side = c->tri_seg[3 * tind + i];
                for (int n = 0; n < NV; ++n) c->sprcn[side * NV + n] += c->tprcn[tind * NV + n];
            }
        }
    }
    // tri_hp::setup_preconditioner: pre-invert (setup_preconditioner.cpp:64-76)
    for (auto &x : c->vprcn) x = 1.0 / (c->tab.vdiag * x);
    if (c->tab.p > 1)
        for (auto &x : c->sprcn) x = 1.0 / x;
    return err;
}

// tri_hp::minvrt, diagonal preconditioner (setup_preconditioner.cpp:102-373)
void or_minvrt(or_ctx *c) {
    const hp_basis_tables &t = c->tab;
    const int NV = c->NV, sm = c->sm, im = c->im;
    auto RV = [&](int v, int n) -> double & { return c->resv[v * NV + n]; };
    auto RS = [&](int s, int m, int n) -> double & { return c->ress[(s * sm + m) * NV + n]; };
    auto RI = [&](int e, int k, int n) -> double & { return c->resi[(e * im + k) * NV + n]; };
    if (sm > 0) {
        for (int sind = 0; sind < c->nseg; ++sind)
            for (int k = 0; k < sm; ++k)
                for (int i = 0; i < 2; ++i) {
                    int v0 = c->seg_pnt[2 * sind + i];
                    for (int n = 0; n < NV; ++n) RV(v0, n) -= t.sfmv[i][k] * RS(sind, k, n);
                }
        if (im > 0) {
            for (int tind = 0; tind < c->ntri; ++tind) {
                int indx2 = 3;
                for (int i = 0; i < 3; ++i) {
                    int v0 = c->tri_pnt[3 * tind + i];
                    for (int k = 0; k < im; ++k)
                        for (int n = 0; n < NV; ++n) RV(v0, n) -= t.ifmb[i][k] * RI(tind, k, n);
                    int sind = c->tri_seg[3 * tind + i], sgn = c->tri_sgn[3 * tind + i], msgn = 1;
                    for (int j = 0; j < sm; ++j) {
                        for (int k = 0; k < im; ++k)
                            for (int n = 0; n < NV; ++n) RS(sind, j, n) -= msgn * t.ifmb[indx2][k] * RI(tind, k, n);
                        msgn *= sgn;
                        ++indx2;
                    }
                }
            }
        }
    }
    for (int v = 0; v < c->npnt; ++v)
        for (int n = 0; n < NV; ++n) RV(v, n) *= c->vprcn[v * NV + n];
    for (int v = 0; v < c->npnt; ++v)  // vdirichlet
        for (int n = 0; n < NV; ++n)
            if (c->vess[v] & (1 << n)) RV(v, n) = 0.0;
    if (sm == 0) return;
    double uh[3][3];
    for (int tind = 0; tind < c->ntri; ++tind) {
        for (int i = 0; i < 3; ++i) {
            int v0 = c->tri_pnt[3 * tind + i];
            for (int n = 0; n < NV; ++n) uh[n][i] = RV(v0, n) * c->tprcn[tind * NV + n];
        }
        for (int i = 0; i < 3; ++i) {
            int sind = c->tri_seg[3 * tind + i], sgn = c->tri_sgn[3 * tind + i];
            for (int j = 0; j < 3; ++j) {
                int indx1 = (i + j) % 3, msgn = 1;
                for (int k = 0; k < sm; ++k) {
                    for (int n = 0; n < NV; ++n) RS(sind, k, n) -= msgn * t.vfms[j][k] * uh[n][indx1];
                    msgn *= sgn;
                }
            }
        }
    }
    for (int mode = 0; mode < sm - 1; ++mode) {
        for (int s = 0; s < c->nseg; ++s)
            for (int n = 0; n < NV; ++n) RS(s, mode, n) *= c->sprcn[s * NV + n] * t.sdiag[mode];
        for (int s = 0; s < c->nseg; ++s)
            for (int n = 0; n < NV; ++n)
                if (c->sess[s] & (1 << n)) RS(s, mode, n) = 0.0;
        for (int tind = 0; tind < c->ntri; ++tind) {
            int side[3], sign[3];
            for (int i = 0; i < 3; ++i) {
                side[i] = c->tri_seg[3 * tind + i];
                sign[i] = c->tri_sgn[3 * tind + i];
                int sgn = (mode % 2 ? sign[i] : 1);
                for (int n = 0; n < NV; ++n) uh[n][i] = sgn * RS(side[i], mode, n) * c->tprcn[tind * NV + n];
            }
            for (int i = 0; i < 3; ++i) {
                int msgn = ((mode + 1) % 2 ? sign[i] : 1);
                for (int m = mode + 1; m < sm; ++m) {
                    for (int j = 0; j < 3; ++j) {
                        int indx = (i + j) % 3;
                        for (int n = 0; n < NV; ++n) RS(side[i], m, n) -= msgn * t.sfms[mode][m][j] * uh[n][indx];
                    }
                    msgn *= sign[i];
                }
            }
        }
    }
    int mode = sm - 1;
    for (int s = 0; s < c->nseg; ++s)
        for (int n = 0; n < NV; ++n) RS(s, mode, n) *= c->sprcn[s * NV + n] * t.sdiag[mode];
    for (int s = 0; s < c->nseg; ++s)
        for (int n = 0; n < NV; ++n)
            if (c->sess[s] & (1 << n)) RS(s, mode, n) = 0.0;
    if (im == 0) return;
    double ub[3][HP_MXBM];
    for (int tind = 0; tind < c->ntri; ++tind) {
        dpbtrsnu2(&t.idiag[0][0], t.ibwth + 1, im, t.ibwth, &RI(tind, 0, 0), NV);
        // restouht_bdry (setup_preconditioner.cpp:375-399)
        for (int i = 0; i < 3; ++i) {
            int indx = c->tri_pnt[3 * tind + i];
            for (int n = 0; n < NV; ++n) ub[n][i] = RV(indx, n);
        }
        int cnt = 3;
        for (int i = 0; i < 3; ++i) {
            int indx = c->tri_seg[3 * tind + i], sign = c->tri_sgn[3 * tind + i], msgn = 1;
            for (int m = 0; m < sm; ++m) {
                for (int n = 0; n < NV; ++n) ub[n][cnt] = msgn * RS(indx, m, n);
                msgn *= sign;
                ++cnt;
            }
        }
        for (int k = 0; k < im; ++k) {
            for (int n = 0; n < NV; ++n) RI(tind, k, n) /= c->tprcn[tind * NV + n];
            for (int i = 0; i < c->bm; ++i)
                for (int n = 0; n < NV; ++n) RI(tind, k, n) -= t.bfmi[i][k] * ub[n][i];
        }
    }
}

// tri_hp::update (nstage.cpp:256-427), fine level
void or_update(or_ctx *c) {
    c->u0v = c->ugv; c->u0s = c->ugs; c->u0i = c->ugi;
    for (int stage = 0; stage < c->ph.nstage; ++stage) {
        or_rsdl(c, stage);
        or_minvrt(c);
        double cflalpha = c->ph.alpha[stage] * c->ph.cfl;
        for (size_t k = 0; k < c->ugv.size(); ++k) c->ugv[k] = c->u0v[k] - cflalpha * c->resv[k];
        for (size_t k = 0; k < c->ugs.size(); ++k) c->ugs[k] = c->u0s[k] - cflalpha * c->ress[k];
        for (size_t k = 0; k < c->ugi.size(); ++k) c->ugi[k] = c->u0i[k] - cflalpha * c->resi[k];
    }
}

// tri_hp::maxres (allocate.cpp:496-525)
double or_maxres(or_ctx *c, double *out) {
    const int NV = c->NV;
    double mx[3] = {0, 0, 0};
    for (int i = 0; i < c->npnt; ++i)
        for (int n = 0; n < NV; ++n) mx[n] = std::max(mx[n], std::fabs(c->resv[i * NV + n]));
    double e = 0.0;
    for (int n = 0; n < NV; ++n) { if (out) out[n] = mx[n]; e = std::max(e, mx[n]); }
    return e;
}

// ---------------------------------------------------------------------------
// Multigrid: tri_hp::mg_restrict (movco.cpp:4-106), mg_prolongate (movfin.cpp:7-82) and
// block::cycle (tri_mesh/blocks.cpp:1267-1348). The reference keeps the p-levels of one
// mesh in one object whose state ug is shared, so a coarse p-level reads and updates the
// lower modes of the fine state in place (ugtouht's interior index step sm0 - sm,
// gtol.cpp:42-52; update's, nstage.cpp:395-406). Here every level is its own context:
// restriction copies the lower modes in and prolongation copies them back, which is the
// same arithmetic.
// ---------------------------------------------------------------------------
static void mg_alloc(or_ctx *c) {
    c->res0v.assign(c->ugv.size(), 0.0); c->res0s.assign(c->ugs.size(), 0.0); c->res0i.assign(c->ugi.size(), 0.0);
    c->dresv.assign(c->ugv.size(), 0.0); c->dress.assign(c->ugs.size(), 0.0); c->dresi.assign(c->ugi.size(), 0.0);
}

// lower modes of fine-level arrays (v, s [nseg][sm_f][NV], i [ntri][im_f][NV]) to or from a
// coarse p-level's arrays; interior rows m = 1 .. sm_c - 1 hold sm_c - m coarse modes, and the
// fine index skips sm_f - sm_c entries after each row (movco.cpp:22-36: the skip is the coarse
// p, which equals sm_f - sm_c when p halves)
static void plevel_copy(const or_ctx *c, const or_ctx *f, double *fv, double *fs, double *fi, double *cv,
                        double *cs, double *ci, bool to_coarse) {
    const int NV = c->NV, smc = c->sm, smf = f->sm, imc = c->im, imf = f->im;
    auto mv = [to_coarse](double &fine, double &coarse) {
        if (to_coarse) coarse = fine;
        else fine = coarse;
    };
    for (int i = 0; i < c->npnt * NV; ++i) mv(fv[i], cv[i]);
    for (int sd = 0; sd < c->nseg; ++sd)
        for (int m = 0; m < smc; ++m)
            for (int n = 0; n < NV; ++n) mv(fs[(sd * smf + m) * NV + n], cs[(sd * smc + m) * NV + n]);
    if (imc > 0)
        for (int t = 0; t < c->ntri; ++t) {
            int indx = 0, indx1 = 0;
            for (int m = 1; m < smc; ++m) {
                for (int k = 0; k < smc - m; ++k) {
                    for (int n = 0; n < NV; ++n)
                        mv(fi[((size_t)t * imf + indx1) * NV + n], ci[((size_t)t * imc + indx) * NV + n]);
                    ++indx; ++indx1;
                }
                indx1 += smf - smc;
            }
        }
}

// Needs the fine level's full residual rsdl(nstage), which block::cycle evaluates just
// before mg_restrict (blocks.cpp:1323-1325).
void or_mg_restrict(or_ctx *c) {
    or_ctx *f = c->fine;
    const int NV = c->NV;
    c->isfrst = true;
    if (c->mg_kind == 1) {
        plevel_copy(c, f, f->resv.data(), f->ress.data(), f->resi.data(), c->res0v.data(), c->res0s.data(),
                    c->res0i.data(), true);
        plevel_copy(c, f, f->ugv.data(), f->ugs.data(), f->ugi.data(), c->ugv.data(), c->ugs.data(), c->ugi.data(),
                    true);
    } else {
        std::fill(c->res0v.begin(), c->res0v.end(), 0.0);
        for (int i = 0; i < f->npnt; ++i) {  // movco.cpp:51-58
            const int tind = c->f2c_tri[i];
            for (int j = 0; j < 3; ++j) {
                const int v0 = c->tri_pnt[3 * tind + j];
                for (int n = 0; n < NV; ++n) c->res0v[v0 * NV + n] += c->f2c_wt[3 * i + j] * f->resv[i * NV + n];
            }
        }
        for (int i = 0; i < c->npnt; ++i) {  // movco.cpp:88-99
            const int tind = c->c2f_tri[i];
            for (int n = 0; n < NV; ++n) c->ugv[i * NV + n] = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int n = 0; n < NV; ++n)
                    c->ugv[i * NV + n] += c->c2f_wt[3 * i + j] * f->ugv[f->tri_pnt[3 * tind + j] * NV + n];
            for (int n = 0; n < NV; ++n) c->vugfrst[i * NV + n] = c->ugv[i * NV + n];
        }
    }
}

void or_mg_prolongate(or_ctx *c) {
    or_ctx *f = c->fine;
    const int NV = c->NV;
    if (c->mg_kind == 1) {
        plevel_copy(c, f, f->ugv.data(), f->ugs.data(), f->ugi.data(), c->ugv.data(), c->ugs.data(), c->ugi.data(),
                    false);
        return;
    }
    for (size_t k = 0; k < c->vugfrst.size(); ++k) c->vugfrst[k] -= c->ugv[k];  // movfin.cpp:24
    for (int i = 0; i < f->npnt; ++i) {                                          // movfin.cpp:33-43, 79
        const int tind = c->f2c_tri[i];
        double corr[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 3; ++j) {
            const int ind = c->tri_pnt[3 * tind + j];
            for (int n = 0; n < NV; ++n) corr[n] -= c->f2c_wt[3 * i + j] * c->vugfrst[ind * NV + n];
        }
        for (int n = 0; n < NV; ++n) f->ugv[i * NV + n] += corr[n];
    }
}

int or_mg_attach_p(or_ctx *c, or_ctx *f, double fadd) {
    if (c->npnt != f->npnt || c->ntri != f->ntri || c->NV != f->NV || c->tm >= f->tm) return -1;
    c->fine = f; c->mg_kind = 1; c->fadd = fadd;
    mg_alloc(c);
    return 0;
}

int or_mg_attach_h(or_ctx *c, or_ctx *f, const int *f2c_tri, const double *f2c_wt, const int *c2f_tri,
                   const double *c2f_wt, double fadd) {
    if (c->sm != 0 || c->NV != f->NV) return -1;
    c->fine = f; c->mg_kind = 2; c->fadd = fadd;
    c->f2c_tri.assign(f2c_tri, f2c_tri + f->npnt);
    c->f2c_wt.assign(f2c_wt, f2c_wt + 3 * f->npnt);
    c->c2f_tri.assign(c2f_tri, c2f_tri + c->npnt);
    c->c2f_wt.assign(c2f_wt, c2f_wt + 3 * c->npnt);
    c->vugfrst.assign(c->ugv.size(), 0.0);
    mg_alloc(c);
    return 0;
}

// block::cycle (blocks.cpp:1267-1348) without the error-control branch; returns the
// count of bad elements met by a preconditioner set-up (the reference throws)
static int cycle(or_ctx **lv, int n, int lvl, int vw, int itercrsn, int iterrfne, int eval) {
    or_ctx *c = lv[lvl];
    for (int vc = 0; vc < vw; ++vc) {
        if (eval) { int e = or_setup_preconditioner(c); if (e) return e; }
        for (int it = 0; it < itercrsn; ++it) or_update(c);
        if (lvl == n - 1) return 0;
        or_rsdl(c, c->ph.nstage);
        or_mg_restrict(lv[lvl + 1]);
        int e = cycle(lv, n, lvl + 1, vw, itercrsn, iterrfne, eval);
        if (e) return e;
        or_mg_prolongate(lv[lvl + 1]);
        if (eval && iterrfne) { e = or_setup_preconditioner(c); if (e) return e; }
        for (int it = 0; it < iterrfne; ++it) or_update(c);
    }
    return 0;
}

int or_cycle(or_ctx **lv, int n, int vw, int itercrsn, int iterrfne, int eval) {
    return cycle(lv, n, 0, vw, itercrsn, iterrfne, eval);
}

// ||R64(u)||_2 over every v/s/i coefficient of rsdl(nstage) with the rows of essential
// boundary values zeroed (hp_edge_bdry::vdirichlet / sdirichlet, hp_boundary.cpp:680-704)
double or_resnorm_essential(or_ctx *c) {
    or_rsdl(c, c->ph.nstage);
    const int NV = c->NV;
    double ss = 0.0;
    for (int i = 0; i < c->npnt; ++i)
        for (int n = 0; n < NV; ++n)
            if (!(c->vess[i] & (1 << n))) ss += c->resv[i * NV + n] * c->resv[i * NV + n];
    for (int sd = 0; sd < c->nseg; ++sd)
        for (int m = 0; m < c->sm; ++m)
            for (int n = 0; n < NV; ++n)
                if (!(c->sess[sd] & (1 << n))) {
                    const double r = c->ress[(sd * c->sm + m) * NV + n];
                    ss += r * r;
                }
    for (double r : c->resi) ss += r * r;
    return std::sqrt(ss);
}

// Convergence driver of the plain FP64 method (block::go's loop over block::cycle with
// the reference's preconditioner_interval): cycles until ||R64|| has dropped by `drop`
// or max_cycles ran; preconditioners on the first cycle and every prcn_every cycles.
// hist[k] = ||R64|| / ||R64(entry)|| after cycle k (hist[0] = 1). Returns the cycles run,
// or -(bad elements) when a set-up failed. nlevels = 1 runs itercrsn updates per cycle.
int or_solve_mg(or_ctx **lv, int n, double drop, int max_cycles, int vw, int itercrsn, int iterrfne,
                int prcn_every, double *hist, int hist_cap) {
    int nc = 0, nh = 0;
    int e = or_setup_preconditioner(lv[0]);
    if (e) return -e;
    const double r0 = or_resnorm_essential(lv[0]);
    if (hist && nh < hist_cap) hist[nh++] = 1.0;
    while (nc < max_cycles) {
        const int eval = (nc == 0 || (prcn_every > 0 && nc % prcn_every == 0)) ? 1 : 0;
        e = cycle(lv, n, 0, vw, itercrsn, iterrfne, eval);
        if (e) return -e;
        ++nc;
        const double d = or_resnorm_essential(lv[0]) / r0;
        if (hist && nh < hist_cap) hist[nh++] = d;
        if (!(d == d) || d <= drop) break;
    }
    return nc;
}

// Basis-operator probes for pinning against the reference's tri_basis.
// tri_hp::element_jacobian (nstage.cpp:131-165), fixed mesh: K [ntri][tm*NV][tm*NV], row
// i*NV + n, column mode*NV + var = (lf_re + lf_im - Rbar) / dw(var) at stage 0, the column's
// unknown raised by dw(var) = eps_r sum_{i<3} |uht(var)(i)| + eps_a (eps_r = eps_a = 1e-8,
// tri_hp/hp_boundary.h:22) and lowered again afterwards, as the reference does.
void or_element_jacobian(or_ctx *c, double *K) {
    const int NV = c->NV, tm = c->tm, NJ = NV * tm;
    const double eps_r = 1.0e-8, eps_a = 1.0e-8;
    double lf_re[3][HP_MXTM], lf_im[3][HP_MXTM], rbar[3][HP_MXTM];
    auto elem = [&](int tind) {
        if (c->ph.physics == HP_PHYS_INS) element_rsdl_ins(c, tind, 0, lf_re, lf_im);
        else element_rsdl_cd(c, tind, 0, lf_re, lf_im);
    };
    for (int tind = 0; tind < c->ntri; ++tind) {
        ugtouht(c, tind);
        double dw[3];
        for (int n = 0; n < NV; ++n) {
            dw[n] = 0.0;
            for (int i = 0; i < 3; ++i) dw[n] += std::fabs(c->uht[n][i]);
            dw[n] = dw[n] * eps_r + eps_a;
        }
        elem(tind);
        for (int i = 0; i < tm; ++i)
            for (int n = 0; n < NV; ++n) rbar[n][i] = lf_re[n][i] + lf_im[n][i];
        int kcol = 0;
        for (int mode = 0; mode < tm; ++mode)
            for (int var = 0; var < NV; ++var, ++kcol) {
                c->uht[var][mode] += dw[var];
                elem(tind);
                int krow = 0;
                for (int i = 0; i < tm; ++i)
                    for (int n = 0; n < NV; ++n, ++krow)
                        K[((size_t)tind * NJ + krow) * NJ + kcol] = (lf_re[n][i] + lf_im[n][i] - rbar[n][i]) / dw[var];
                c->uht[var][mode] -= dw[var];
            }
    }
}

void or_basis_proj(const hp_basis_tables *t, const double *lin, double *f, double *dx, double *dy, int st) { Basis(*t).proj(lin, f, dx, dy, st); }
void or_basis_proj_val(const hp_basis_tables *t, const double *lin, double *f, int st) { Basis(*t).proj(lin, f, st); }
void or_basis_derivr(const hp_basis_tables *t, const double *f, double *d, int st) { Basis(*t).derivr(f, d, st); }
void or_basis_derivs(const hp_basis_tables *t, const double *f, double *d, int st) { Basis(*t).derivs(f, d, st); }
void or_basis_intgrt(const hp_basis_tables *t, double *r, const double *f, int st) { Basis(*t).intgrt(r, f, st); }
void or_basis_intgrtrs(const hp_basis_tables *t, double *r, const double *dx, const double *dy, int st) { Basis(*t).intgrtrs(r, dx, dy, st); }
void or_basis_proj1d(const hp_basis_tables *t, const double *lin, double *f, double *dx) { Basis(*t).proj1d(lin, f, dx); }
void or_basis_intgrt1d(const hp_basis_tables *t, double *r, const double *f) { Basis(*t).intgrt1d(r, f); }
void or_dpbtrsnu2(const double *abd, int stride, int ordr, int ofdg, double *b, int rhs) { dpbtrsnu2(abd, stride, ordr, ofdg, b, rhs); }

}  // extern "C"
