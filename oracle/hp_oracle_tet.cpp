// CPU oracle of the 3D (tet_hp, ins) residual path. TEST INFRASTRUCTURE ONLY:
// only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it.
//
// Restates, element by element in plain loops:
//   tet_hp::rsdl                        tet_hp/update.cpp:9-118
//   tet_hp::ugtouht / lftog             tet_hp/gtol.cpp:16-82, 815-873
//   tet_hp_ins::element_rsdl (straight) tet_hp/ins/rsdl.cpp:442-781
//   tet_hp_ins::setup_preconditioner    tet_hp/ins/setup_preconditioner.cpp (diagonal: tau, iprcn)
//   bdry_ins::neumann / inflow rsdl     tet_hp/ins/bdry.cpp:16-102, bdry_ins.h:85-132
//   tet_hp::jacobian_diagonal, jacobi_relaxation   tet_hp/jacobi.cpp:14-111
//   tet_hp::minvrt (p = 1, 2 and 3)     tet_hp/setup_preconditioner.cpp:11-354
//   tet_hp::spoke (p = 3)               tet_hp/setup_preconditioner.cpp:530-583
//   tet_hp::update                      tet_hp/update.cpp:181-390
// with the basis operators of tet_basis in the dense form of hp_tet_tables
// (pinned against the reference's own proj / intgrt / intgrtrst / derivr / derivs /
// derivt / proj2d / intgrt2d and lumpinv by tests/test_tet_basis_pin.py). Parity: the
// stages of the reference's loops are kept; sums over points and modes run in the
// natural order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/hp_gpu.h"
#include "../include/hp_tet.h"

namespace {

constexpr int NV = 4;

struct OT {
    hp_tet_tables t;
    hp_phys_params ph;
    int npnt, nseg, ntri, ntet;
    std::vector<double> pnts, vol;
    std::vector<int> tp, ts, tsg, tt, trot;
    std::vector<double> ugv, uge, ugf, ugi;           // state
    std::vector<double> rv, re, rf, ri;               // res
    std::vector<double> rrv, rre, rrf, rri;           // res_r
    std::vector<double> tau;                          // [ntet][2]: tau(tind,0), tau(tind,NV-1)
    std::vector<double> iprcn;                        // [ntet][NV]
    std::vector<double> vprcn, eprcn, fprcn;          // accumulated diagonals
    std::vector<double> jv, je, jf, ji;               // jacob_diag (tet_hp/jacobi.cpp)
    std::vector<unsigned char> mv, me, mf;            // 1 where a boundary condition fixes the row
    std::vector<double> u0v, u0e, u0f, u0i;           // ug0 of the nstage update
    // boundary faces with a flux: global face, vertices, edges (opposite each vertex) and
    // signs [3], kind (0 inflow, 1 neumann), imposed pressure at the face points [G * G]
    std::vector<int> bf_tri, bf_pnt, bf_seg, bf_sgn, bf_kind;
    std::vector<double> bf_pbc;
    int smoother = 0;  // 0: JACOBI build, 1: minvrt
};

// the face vertices of local face i (tet_mesh/setup.cpp:307-310)
const int VF[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};

void gather(const OT &o, int tind, double uht[NV][HP_TET_MAXT]) {
    const hp_tet_tables &t = o.t;
    for (int i = 0; i < 4; ++i)
        for (int n = 0; n < NV; ++n) uht[n][i] = o.ugv[(size_t)o.tp[4 * tind + i] * NV + n];
    int cnt = 4;
    for (int i = 0; i < 6; ++i) {
        const int e = o.ts[6 * tind + i], sg = o.tsg[6 * tind + i];
        int msgn = 1;
        for (int m = 0; m < t.em; ++m, ++cnt) {
            for (int n = 0; n < NV; ++n) uht[n][cnt] = msgn * o.uge[((size_t)e * t.em + m) * NV + n];
            msgn *= sg;
        }
    }
    for (int i = 0; i < 4; ++i) {
        const int f = o.tt[4 * tind + i], sg = -o.trot[4 * tind + i];
        int msgn = 1, indx = 0;
        for (int m = 1; m <= t.em - 1; ++m) {
            for (int k = 1; k <= t.em - m; ++k, ++cnt, ++indx)
                for (int n = 0; n < NV; ++n) uht[n][cnt] = msgn * o.ugf[((size_t)f * t.fm + indx) * NV + n];
            msgn *= sg;
        }
    }
    for (int m = 0; m < t.im; ++m, ++cnt)
        for (int n = 0; n < NV; ++n) uht[n][cnt] = o.ugi[((size_t)tind * t.im + m) * NV + n];
}

void scatter(const OT &o, int tind, const double lf[NV][HP_TET_MAXT], double *gv, double *ge, double *gf,
             double *gi) {
    const hp_tet_tables &t = o.t;
    for (int i = 0; i < 4; ++i)
        for (int n = 0; n < NV; ++n) gv[(size_t)o.tp[4 * tind + i] * NV + n] += lf[n][i];
    int indx = 4;
    for (int i = 0; i < 6; ++i) {
        const int e = o.ts[6 * tind + i], sg = o.tsg[6 * tind + i];
        int msgn = 1;
        for (int m = 0; m < t.em; ++m, ++indx) {
            for (int n = 0; n < NV; ++n) ge[((size_t)e * t.em + m) * NV + n] += msgn * lf[n][indx];
            msgn *= sg;
        }
    }
    for (int i = 0; i < 4; ++i) {
        const int f = o.tt[4 * tind + i], sg = -o.trot[4 * tind + i];
        int msgn = 1, gindx = 0;
        for (int m = 1; m <= t.em - 1; ++m) {
            for (int j = 1; j <= t.em - m; ++j, ++gindx, ++indx)
                for (int n = 0; n < NV; ++n) gf[((size_t)f * t.fm + gindx) * NV + n] += msgn * lf[n][indx];
            msgn *= sg;
        }
    }
    for (int m = 0; m < t.im; ++m, ++indx)
        for (int n = 0; n < NV; ++n) gi[((size_t)tind * t.im + m) * NV + n] += lf[n][indx];
}

// r(m) -= sum_q w (DX fr + DY fs + DZ ft)  (tet_basis::intgrtrst)
void intgrtrst(const hp_tet_tables &t, double *r, const double *fr, const double *fs, const double *ft) {
    const int Q = t.G * t.G * t.G;
    for (int m = 0; m < t.T; ++m) {
        double s = 0.0;
        for (int q = 0; q < Q; ++q) s += t.w[q] * (t.DX[q][m] * fr[q] + t.DY[q][m] * fs[q] + t.DZ[q][m] * ft[q]);
        r[m] -= s;
    }
}

// dst += derivative `dir` (0 r, 1 s, 2 t) of point values f  (tet_basis::derivr/s/t)
void deriv(const hp_tet_tables &t, int dir, const double *f, double *dst) {
    const int G = t.G;
    for (int i = 0; i < G; ++i)
        for (int j = 0; j < G; ++j)
            for (int k = 0; k < G; ++k) {
                const int q = (i * G + j) * G + k;
                double ax = 0.0, bx = 0.0, ay = 0.0, by = 0.0, az = 0.0;
                for (int n = 0; n < G; ++n) {
                    const double fx = f[(n * G + j) * G + k], fy = f[(i * G + n) * G + k], fz = f[(i * G + j) * G + n];
                    ax += t.Ax[i][n] * fx;
                    bx += t.Bx[i][n] * fx;
                    ay += t.Ay[j][n] * fy;
                    by += t.By[j][n] * fy;
                    az += t.Az[k][n] * fz;
                }
                const double yz = t.y0[j] * t.z0[k], z = t.z0[k];
                if (dir == 0) dst[q] += yz * ax;
                else if (dir == 1) dst[q] += yz * bx + z * ay;
                else dst[q] += yz * bx + z * by + az;
            }
}

void element_rsdl_uht(const OT &o, int tind, int stage, const double uht[NV][HP_TET_MAXT],
                      double lf_re[NV][HP_TET_MAXT], double lf_im[NV][HP_TET_MAXT]) {
    const hp_tet_tables &t = o.t;
    const int Q = t.G * t.G * t.G, T = t.T;
    // straight element: ldcrd(n, 0..2) = (v3 - v2, v1 - v2, v0 - v2) / 2
    const int *v = &o.tp[4 * tind];
    double ld[3][3];
    for (int n = 0; n < 3; ++n) {
        ld[n][0] = 0.5 * (o.pnts[3 * v[3] + n] - o.pnts[3 * v[2] + n]);
        ld[n][1] = 0.5 * (o.pnts[3 * v[1] + n] - o.pnts[3 * v[2] + n]);
        ld[n][2] = 0.5 * (o.pnts[3 * v[0] + n] - o.pnts[3 * v[2] + n]);
    }
    double d[3][3];
    d[0][0] = ld[1][1] * ld[2][2] - ld[1][2] * ld[2][1];
    d[0][1] = -ld[0][1] * ld[2][2] + ld[0][2] * ld[2][1];
    d[0][2] = ld[0][1] * ld[1][2] - ld[0][2] * ld[1][1];
    d[1][0] = -ld[1][0] * ld[2][2] + ld[1][2] * ld[2][0];
    d[1][1] = ld[0][0] * ld[2][2] - ld[0][2] * ld[2][0];
    d[1][2] = -ld[0][0] * ld[1][2] + ld[0][2] * ld[1][0];
    d[2][0] = ld[1][0] * ld[2][1] - ld[1][1] * ld[2][0];
    d[2][1] = -ld[0][0] * ld[2][1] + ld[0][1] * ld[2][0];
    d[2][2] = ld[0][0] * ld[1][1] - ld[0][1] * ld[1][0];
    const double cjcb = ld[0][0] * (ld[1][1] * ld[2][2] - ld[1][2] * ld[2][1]) -
                        ld[0][1] * (ld[1][0] * ld[2][2] - ld[2][0] * ld[1][2]) +
                        ld[0][2] * (ld[1][0] * ld[2][1] - ld[2][0] * ld[1][1]);
    const double beta = o.ph.beta[stage], rho = o.ph.rho;
    // proj (with r, s, t derivatives of u, v, w when beta > 0)
    std::vector<double> u(NV * Q, 0.0), du(NV * 3 * Q, 0.0);
    auto U = [&](int n, int q) -> double & { return u[n * Q + q]; };
    auto DU = [&](int n, int c, int q) -> double & { return du[(n * 3 + c) * Q + q]; };
    for (int q = 0; q < Q; ++q)
        for (int n = 0; n < NV; ++n) {
            double f = 0, dr = 0, ds = 0, dt = 0;
            for (int m = 0; m < T; ++m) {
                f += t.F[q][m] * uht[n][m];
                dr += t.DX[q][m] * uht[n][m];
                ds += t.DY[q][m] * uht[n][m];
                dt += t.DZ[q][m] * uht[n][m];
            }
            U(n, q) = f;
            if (beta > 0.0 && n < NV - 1) { DU(n, 0, q) = dr; DU(n, 1, q) = ds; DU(n, 2, q) = dt; }
        }
    for (int n = 0; n < NV; ++n)
        for (int m = 0; m < T; ++m) lf_re[n][m] = lf_im[n][m] = 0.0;
    // convective, continuity and pressure fluxes (imaginary part)
    std::vector<double> cv(3 * 3 * Q), df(3 * 3 * Q), res(NV * Q);
    auto CV = [&](int n, int c, int q) -> double & { return cv[(n * 3 + c) * Q + q]; };
    auto DF = [&](int n, int c, int q) -> double & { return df[(n * 3 + c) * Q + q]; };
    for (int q = 0; q < Q; ++q) {
        const double fx = rho * U(0, q), fy = rho * U(1, q), fz = rho * U(2, q);
        for (int c = 0; c < 3; ++c) DU(NV - 1, c, q) = d[c][0] * fx + d[c][1] * fy + d[c][2] * fz;
        for (int n = 0; n < NV - 1; ++n)
            for (int c = 0; c < 3; ++c) CV(n, c, q) = U(n, q) * DU(NV - 1, c, q) + d[c][n] * U(NV - 1, q);
    }
    for (int n = 0; n < NV - 1; ++n) intgrtrst(t, lf_im[n], &CV(n, 0, 0), &CV(n, 1, 0), &CV(n, 2, 0));
    intgrtrst(t, lf_im[NV - 1], &DU(NV - 1, 0, 0), &DU(NV - 1, 1, 0), &DU(NV - 1, 2, 0));
    if (!(beta > 0.0)) return;
    // viscous tensor visc(a,b)(c,e) (rsdl.cpp:521-612)
    const double cjcbi = o.ph.mu / cjcb;
    double visc[3][3][3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c)
                for (int e = 0; e < 3; ++e) {
                    if (a == b) {
                        double s = d[c][a] * d[e][a];
                        for (int f = 0; f < 3; ++f) s += d[c][f] * d[e][f];
                        visc[a][b][c][e] = -cjcbi * s;
                    } else {
                        visc[a][b][c][e] = -cjcbi * d[c][b] * d[e][a];
                    }
                }
    // steady: res = rho*bd0*cjcb*u + dugdt = 0, intgrt of it into lf_re = 0
    for (int q = 0; q < Q; ++q) {
        for (int n = 0; n < NV; ++n) res[n * Q + q] = 0.0;
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
                for (int b = 0; b < 3; ++b)
                    for (int e = 0; e < 3; ++e) s += visc[a][b][c][e] * DU(b, e, q);
                DF(a, c, q) = s;
                CV(a, c, q) += s;
            }
    }
    // strong residual: derivatives of the total fluxes
    for (int n = 0; n < NV - 1; ++n)
        for (int c = 0; c < 3; ++c) deriv(t, c, &CV(n, c, 0), &res[n * Q]);
    for (int c = 0; c < 3; ++c) deriv(t, c, &DU(NV - 1, c, 0), &res[(NV - 1) * Q]);
    // SUPG (rsdl.cpp:693-766), mesh velocity zero
    const double tau0 = o.tau[2 * tind], tau3 = o.tau[2 * tind + 1];
    for (int q = 0; q < Q; ++q) {
        double tr[NV];
        for (int n = 0; n < NV - 1; ++n) tr[n] = tau0 * res[n * Q + q];
        tr[NV - 1] = tau3 * res[(NV - 1) * Q + q];
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) {
                double s = d[c][a] * (2.0 * U(a, q));
                for (int b = 0; b < 3; ++b)
                    if (b != a) s += d[c][b] * U(b, q);
                double r = s * tr[a];
                for (int b = 0; b < 3; ++b)
                    if (b != a) r += d[c][b] * U(a, q) * tr[b];
                r += d[c][a] * tr[NV - 1];
                DF(a, c, q) -= r;
            }
        for (int c = 0; c < 3; ++c) DU(NV - 1, c, q) = -d[c][0] * tr[0] - d[c][1] * tr[1] - d[c][2] * tr[2];
    }
    for (int n = 0; n < NV - 1; ++n) intgrtrst(t, lf_re[n], &DF(n, 0, 0), &DF(n, 1, 0), &DF(n, 2, 0));
    intgrtrst(t, lf_re[NV - 1], &DU(NV - 1, 0, 0), &DU(NV - 1, 1, 0), &DU(NV - 1, 2, 0));
    for (int n = 0; n < NV; ++n)
        for (int m = 0; m < T; ++m) lf_re[n][m] *= beta;
}

void element_rsdl(const OT &o, int tind, int stage, double lf_re[NV][HP_TET_MAXT], double lf_im[NV][HP_TET_MAXT]) {
    double uht[NV][HP_TET_MAXT];
    gather(o, tind, uht);
    element_rsdl_uht(o, tind, stage, uht, lf_re, lf_im);
}

// lftog without the edge / face signs (for diagonal entries: sign * sign = 1)
void scatter_unsigned(const OT &o, int tind, const double lf[NV][HP_TET_MAXT], double *gv, double *ge, double *gf,
                      double *gi) {
    const hp_tet_tables &t = o.t;
    for (int i = 0; i < 4; ++i)
        for (int n = 0; n < NV; ++n) gv[(size_t)o.tp[4 * tind + i] * NV + n] += lf[n][i];
    int indx = 4;
    for (int i = 0; i < 6; ++i)
        for (int m = 0; m < t.em; ++m, ++indx)
            for (int n = 0; n < NV; ++n) ge[((size_t)o.ts[6 * tind + i] * t.em + m) * NV + n] += lf[n][indx];
    for (int i = 0; i < 4; ++i)
        for (int m = 0; m < t.fm; ++m, ++indx)
            for (int n = 0; n < NV; ++n) gf[((size_t)o.tt[4 * tind + i] * t.fm + m) * NV + n] += lf[n][indx];
    for (int m = 0; m < t.im; ++m, ++indx)
        for (int n = 0; n < NV; ++n) gi[((size_t)tind * t.im + m) * NV + n] += lf[n][indx];
}

// hp_face_bdry::rsdl of bdry_ins::neumann / inflow (tet_hp/ins/bdry.cpp:16-102): for face b,
// ugtouht2d (tet_hp/gtol.cpp:257-299), the straight-face coordinates (crdtocht2d), proj2d of
// the coordinates and the velocity, the flux at every face point with the normal
// nrm = d(crd)/dr x d(crd)/ds (tet_hp/ins/bdry_ins.h:85-132), intgrt2d, and the sum into res.
void face_flux(OT &o, int b) {
    const hp_tet_tables &t = o.t;
    const int G2 = t.G * t.G, T2 = t.T2, em = t.em, fm = t.fm;
    const int find = o.bf_tri[b], *pv = &o.bf_pnt[3 * b], *ps = &o.bf_seg[3 * b], *sg = &o.bf_sgn[3 * b];
    double uht[3][HP_TET_MAXT];
    for (int v = 0; v < 3; ++v)
        for (int n = 0; n < 3; ++n) uht[n][v] = o.ugv[(size_t)pv[v] * NV + n];
    int cnt = 3;
    for (int i = 0; i < 3; ++i) {
        int msgn = 1;
        for (int m = 0; m < em; ++m, ++cnt) {
            for (int n = 0; n < 3; ++n) uht[n][cnt] = msgn * o.uge[((size_t)ps[i] * em + m) * NV + n];
            msgn *= sg[i];
        }
    }
    for (int k = 0; k < fm; ++k, ++cnt)
        for (int n = 0; n < 3; ++n) uht[n][cnt] = o.ugf[((size_t)find * fm + k) * NV + n];
    double lf[NV][HP_TET_MAXT];
    for (int n = 0; n < NV; ++n)
        for (int k = 0; k < T2; ++k) lf[n][k] = 0.0;
    for (int q = 0; q < G2; ++q) {
        double dr[3], ds[3], u[3];
        for (int d = 0; d < 3; ++d) {
            dr[d] = ds[d] = 0.0;
            for (int v = 0; v < 3; ++v) {
                dr[d] += t.DX2[q][v] * o.pnts[3 * (size_t)pv[v] + d];
                ds[d] += t.DY2[q][v] * o.pnts[3 * (size_t)pv[v] + d];
            }
        }
        const double nrm[3] = {dr[1] * ds[2] - dr[2] * ds[1], dr[2] * ds[0] - dr[0] * ds[2],
                               dr[0] * ds[1] - dr[1] * ds[0]};
        for (int n = 0; n < 3; ++n) {
            u[n] = 0.0;
            for (int k = 0; k < T2; ++k) u[n] += t.F2[q][k] * uht[n][k];
        }
        double flx[NV];
        flx[3] = o.ph.rho * (u[0] * nrm[0] + u[1] * nrm[1] + u[2] * nrm[2]);
        for (int n = 0; n < 3; ++n)
            flx[n] = o.bf_kind[b] ? flx[3] * u[n] + o.bf_pbc[(size_t)b * G2 + q] * nrm[n] : 0.0;
        for (int n = 0; n < NV; ++n)
            for (int k = 0; k < T2; ++k) lf[n][k] += t.W2[q] * t.F2[q][k] * flx[n];
    }
    for (int v = 0; v < 3; ++v)
        for (int n = 0; n < NV; ++n) o.rv[(size_t)pv[v] * NV + n] += lf[n][v];
    int indx = 3;
    for (int i = 0; i < 3; ++i) {
        double msgn = 1.0;
        for (int m = 0; m < em; ++m, ++indx) {
            for (int n = 0; n < NV; ++n) o.re[((size_t)ps[i] * em + m) * NV + n] += msgn * lf[n][indx];
            msgn *= sg[i];
        }
    }
    for (int k = 0; k < fm; ++k, ++indx)
        for (int n = 0; n < NV; ++n) o.rf[((size_t)find * fm + k) * NV + n] += lf[n][indx];
}

}  // namespace

extern "C" {

// boundary faces with a flux (same arguments as hp_tet_set_flux_faces)
void ot_set_flux_faces(void *h, int nface, const int *face_tri, const int *face_pnt, const int *face_seg,
                       const int *face_sgn, const int *kind, const double *pbc) {
    OT &o = *static_cast<OT *>(h);
    const size_t G2 = (size_t)o.t.G * o.t.G;
    o.bf_tri.assign(face_tri, face_tri + nface);
    o.bf_pnt.assign(face_pnt, face_pnt + 3 * (size_t)nface);
    o.bf_seg.assign(face_seg, face_seg + 3 * (size_t)nface);
    o.bf_sgn.assign(face_sgn, face_sgn + 3 * (size_t)nface);
    o.bf_kind.assign(kind, kind + nface);
    o.bf_pbc.assign(G2 * nface, 0.0);
    if (pbc) std::copy(pbc, pbc + G2 * nface, o.bf_pbc.begin());
}

void *ot_create(const hp_tet_tables *t, const hp_phys_params *ph, int npnt, int nseg, int ntri, int ntet,
                const double *pnts, const int *tet_pnt, const int *tet_seg, const int *tet_sgn, const int *tet_tri,
                const int *tet_rot, const double *vol) {
    OT *o = new OT;
    o->t = *t;
    o->ph = *ph;
    o->npnt = npnt; o->nseg = nseg; o->ntri = ntri; o->ntet = ntet;
    o->pnts.assign(pnts, pnts + 3 * (size_t)npnt);
    o->vol.assign(vol, vol + ntet);
    o->tp.assign(tet_pnt, tet_pnt + 4 * (size_t)ntet);
    o->ts.assign(tet_seg, tet_seg + 6 * (size_t)ntet);
    o->tsg.assign(tet_sgn, tet_sgn + 6 * (size_t)ntet);
    o->tt.assign(tet_tri, tet_tri + 4 * (size_t)ntet);
    o->trot.assign(tet_rot, tet_rot + 4 * (size_t)ntet);
    const size_t lv = (size_t)npnt * NV, le = (size_t)nseg * t->em * NV, lf = (size_t)ntri * t->fm * NV,
                 li = (size_t)ntet * t->im * NV;
    for (auto *a : {&o->ugv, &o->rv, &o->rrv}) a->assign(lv, 0.0);
    for (auto *a : {&o->uge, &o->re, &o->rre}) a->assign(le, 0.0);
    for (auto *a : {&o->ugf, &o->rf, &o->rrf}) a->assign(lf, 0.0);
    for (auto *a : {&o->ugi, &o->ri, &o->rri}) a->assign(li, 0.0);
    o->tau.assign(2 * (size_t)ntet, 0.0);
    o->iprcn.assign(NV * (size_t)ntet, 0.0);
    o->vprcn.assign(lv, 0.0);
    o->eprcn.assign((size_t)nseg * NV, 0.0);
    o->fprcn.assign((size_t)ntri * NV, 0.0);
    return o;
}

void ot_destroy(void *h) { delete static_cast<OT *>(h); }

void ot_set_state(void *h, const double *v, const double *e, const double *f, const double *i) {
    OT &o = *static_cast<OT *>(h);
    std::memcpy(o.ugv.data(), v, o.ugv.size() * 8);
    if (!o.uge.empty()) std::memcpy(o.uge.data(), e, o.uge.size() * 8);
    if (!o.ugf.empty()) std::memcpy(o.ugf.data(), f, o.ugf.size() * 8);
    if (!o.ugi.empty()) std::memcpy(o.ugi.data(), i, o.ugi.size() * 8);
}

// which: 0 res, 1 res_r, 2 state
void ot_get(void *h, int which, double *v, double *e, double *f, double *i) {
    OT &o = *static_cast<OT *>(h);
    const std::vector<double> *a[4];
    if (which == 0) { a[0] = &o.rv; a[1] = &o.re; a[2] = &o.rf; a[3] = &o.ri; }
    else if (which == 1) { a[0] = &o.rrv; a[1] = &o.rre; a[2] = &o.rrf; a[3] = &o.rri; }
    else { a[0] = &o.ugv; a[1] = &o.uge; a[2] = &o.ugf; a[3] = &o.ugi; }
    double *dst[4] = {v, e, f, i};
    for (int k = 0; k < 4; ++k)
        if (dst[k] && !a[k]->empty()) std::memcpy(dst[k], a[k]->data(), a[k]->size() * 8);
}

// tau [ntet][2], iprcn [ntet][4]
void ot_get_prcn(void *h, double *tau, double *iprcn) {
    OT &o = *static_cast<OT *>(h);
    std::memcpy(tau, o.tau.data(), o.tau.size() * 8);
    std::memcpy(iprcn, o.iprcn.data(), o.iprcn.size() * 8);
}

// tet_hp_ins::setup_preconditioner, diagonal branch, steady (bd0 = 0), mesh velocity 0
int ot_setup_preconditioner(void *h) {
    OT &o = *static_cast<OT *>(h);
    const double nu = o.ph.mu / o.ph.rho;
    const int p = o.t.p;
    int err = 0;
    std::fill(o.vprcn.begin(), o.vprcn.end(), 0.0);
    std::fill(o.eprcn.begin(), o.eprcn.end(), 0.0);
    std::fill(o.fprcn.begin(), o.fprcn.end(), 0.0);
    for (int tind = 0; tind < o.ntet; ++tind) {
        double jcb = 0.125 * o.vol[tind];
        const int *v = &o.tp[4 * tind];
        double amin = 1.0e99, amax = 0.0;
        for (int j = 0; j < 4; ++j) {
            const double *a = &o.pnts[3 * v[VF[j][0]]], *b = &o.pnts[3 * v[VF[j][1]]], *c = &o.pnts[3 * v[VF[j][2]]];
            const double v1[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
            const double v2[3] = {a[0] - c[0], a[1] - c[1], a[2] - c[2]};
            const double cr[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                                  v1[0] * v2[1] - v1[1] * v2[0]};
            const double ar = .5 * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            amax = ar > amax ? ar : amax;
            amin = ar < amin ? ar : amin;
        }
        const double h = 4.0 * jcb / (0.25 * (p + 1) * (p + 1) * amax);
        const double hmax = 4.0 * jcb / (0.25 * (p + 1) * (p + 1) * amin);
        double qmax = 0.0;
        for (int j = 0; j < 4; ++j) {
            const double *uu = &o.ugv[(size_t)v[j] * NV];
            const double q = uu[0] * uu[0] + uu[1] * uu[1] + uu[2] * uu[2];
            qmax = q > qmax ? q : qmax;
        }
        if (!(jcb > 0.0) || !(qmax >= 0.0)) err = 1;
        double gam = 3.0 * qmax + (0.5 * hmax * o.ph.bd0 + 2. * nu / hmax) * (0.5 * hmax * o.ph.bd0 + 2. * nu / hmax);
        if (o.ph.mu + o.ph.bd0 == 0.0) gam = gam > 0.1 ? gam : 0.1;
        const double q = std::sqrt(qmax);
        const double lam1 = q + std::sqrt(qmax + gam);
        o.tau[2 * tind] = o.ph.adis * h / (jcb * std::sqrt(gam));
        o.tau[2 * tind + 1] = qmax * o.tau[2 * tind];
        jcb *= 2. * nu * (1. / (h * h) + 1. / (h * h) + 1. / (h * h)) + 3 * lam1 / h;
        double ip[NV] = {o.ph.rho * jcb, o.ph.rho * jcb, o.ph.rho * jcb, jcb / gam};
        for (int n = 0; n < NV; ++n) o.iprcn[(size_t)tind * NV + n] = ip[n];
        for (int i = 0; i < 4; ++i)
            for (int n = 0; n < NV; ++n) o.vprcn[(size_t)v[i] * NV + n] += ip[n];
        if (o.t.em > 0)
            for (int i = 0; i < 6; ++i)
                for (int n = 0; n < NV; ++n) o.eprcn[(size_t)o.ts[6 * tind + i] * NV + n] += ip[n];
        if (o.t.fm > 0)
            for (int i = 0; i < 4; ++i)
                for (int n = 0; n < NV; ++n) o.fprcn[(size_t)o.tt[4 * tind + i] * NV + n] += ip[n];
    }
    return err;
}

// Rows fixed by essential (velocity) conditions: mask arrays over vertices [npnt][NV],
// edges [nseg][NV], faces [ntri][NV] (1 = zero this row; the boundary faces' vdirichlet /
// edirichlet / fdirichlet of bdry_ins::inflow, tet_hp/ins/bdry_ins.h:141-183).
void ot_set_dirichlet(void *h, const unsigned char *mv, const unsigned char *me, const unsigned char *mf) {
    OT &o = *static_cast<OT *>(h);
    o.mv.assign(mv, mv + (size_t)o.npnt * NV);
    o.me.assign(me, me + (size_t)o.nseg * NV);
    o.mf.assign(mf, mf + (size_t)o.ntri * NV);
}

static void all_dirichlet(OT &o) {
    if (o.mv.empty()) return;
    for (size_t k = 0; k < o.rv.size(); ++k)
        if (o.mv[k]) o.rv[k] = 0.0;
    for (int e = 0; e < o.nseg; ++e)
        for (int m = 0; m < o.t.em; ++m)
            for (int n = 0; n < NV; ++n)
                if (o.me[(size_t)e * NV + n]) o.re[((size_t)e * o.t.em + m) * NV + n] = 0.0;
    for (int f = 0; f < o.ntri; ++f)
        for (int m = 0; m < o.t.fm; ++m)
            for (int n = 0; n < NV; ++n)
                if (o.mf[(size_t)f * NV + n]) o.rf[((size_t)f * o.t.fm + m) * NV + n] = 0.0;
}

// tet_hp::jacobian_diagonal (jacobi.cpp:32-111): finite-difference diagonal of every
// element's Jacobian at stage 0, summed into the global diagonal.
void ot_jacobian_diagonal(void *h) {
    OT &o = *static_cast<OT *>(h);
    const hp_tet_tables &t = o.t;
    const int T = t.T;
    o.jv.assign(o.ugv.size(), 0.0);
    o.je.assign(o.uge.size(), 0.0);
    o.jf.assign(o.ugf.size(), 0.0);
    o.ji.assign(o.ugi.size(), 0.0);
    const double eps_r = 1.0e-6, eps_a = 1.0e-10;
    double lf_re[NV][HP_TET_MAXT], lf_im[NV][HP_TET_MAXT], rbar[NV][HP_TET_MAXT], lf[NV][HP_TET_MAXT];
    std::vector<double> kd((size_t)T * NV);
    for (int tind = 0; tind < o.ntet; ++tind) {
        double uht[NV][HP_TET_MAXT];
        gather(o, tind, uht);
        double dw = 0.0;  // the same for every variable (jacobi.cpp:63-67 adds to all entries)
        for (int i = 0; i < 4; ++i)
            for (int n = 0; n < NV; ++n) dw += std::fabs(uht[n][i]);
        dw = dw * eps_r + eps_a;
        element_rsdl_uht(o, tind, 0, uht, lf_re, lf_im);
        for (int i = 0; i < T; ++i)
            for (int n = 0; n < NV; ++n) rbar[n][i] = lf_re[n][i] + lf_im[n][i];
        int ind = 0;
        for (int i = 0; i < T; ++i)
            for (int n = 0; n < NV; ++n) {
                uht[n][i] += dw;
                element_rsdl_uht(o, tind, 0, uht, lf_re, lf_im);
                kd[ind++] = (lf_re[n][i] + lf_im[n][i] - rbar[n][i]) / dw;
                uht[n][i] -= dw;
            }
        // kd is in (mode, variable) order; add to the global diagonal (no signs: sign^2 = 1)
        for (int i = 0; i < T; ++i)
            for (int n = 0; n < NV; ++n) lf[n][i] = kd[(size_t)i * NV + n];
        scatter_unsigned(o, tind, lf, o.jv.data(), o.je.data(), o.jf.data(), o.ji.data());
    }
}

// tet_hp::jacobi_relaxation (jacobi.cpp:14-30): res = omega res / jacob_diag, then the
// essential rows are zeroed.
static void jacobi_relaxation(OT &o) {
    const double omega = 0.5;
    for (size_t k = 0; k < o.rv.size(); ++k) o.rv[k] = omega * o.rv[k] / o.jv[k];
    for (size_t k = 0; k < o.re.size(); ++k) o.re[k] = omega * o.re[k] / o.je[k];
    for (size_t k = 0; k < o.rf.size(); ++k) o.rf[k] = omega * o.rf[k] / o.jf[k];
    for (size_t k = 0; k < o.ri.size(); ++k) o.ri[k] = omega * o.ri[k] / o.ji[k];
    all_dirichlet(o);
}

// tet_hp::minvrt at p = 1 (setup_preconditioner.cpp:57-74): vprcn pre-inverted by
// tet_hp::setup_preconditioner (:451-453), res.v *= vprcn vdiag, then the vertex Dirichlet
// rows are zeroed; em = 0 ends it.
static void minvrt_p1(OT &o) {
    for (size_t k = 0; k < o.rv.size(); ++k) o.rv[k] *= (1.0 / o.vprcn[k]) * o.t.vdiag;
    all_dirichlet(o);
}

// tet_hp::minvrt at p = 2 (setup_preconditioner.cpp:16-30, 57-131, 197-221): edge modes
// removed from their end vertices with sfmv, the vertex rows scaled by vdiag / vprcn and
// fixed, the vertex values times the element diagonal removed from the edge modes with the
// mass matrix, the edge rows scaled by ediag(0) / eprcn (minvrt sets ediag(0) = 100 at p = 2)
// and fixed.
static void minvrt_p2(OT &o) {
    const hp_tet_tables &t = o.t;
    const int em = t.em;
    static const int VS[6][2] = {{2, 3}, {3, 1}, {2, 1}, {1, 0}, {2, 0}, {3, 0}};
    std::vector<int> sp(2 * (size_t)o.nseg);
    for (int tind = 0; tind < o.ntet; ++tind)
        for (int i = 0; i < 6; ++i) {
            const int s = o.ts[6 * tind + i], a = o.tp[4 * tind + VS[i][0]], b = o.tp[4 * tind + VS[i][1]];
            sp[2 * (size_t)s] = o.tsg[6 * tind + i] > 0 ? a : b;
            sp[2 * (size_t)s + 1] = o.tsg[6 * tind + i] > 0 ? b : a;
        }
    for (int s = 0; s < o.nseg; ++s)
        for (int k = 0; k < em; ++k)
            for (int i = 0; i < 2; ++i)
                for (int n = 0; n < NV; ++n)
                    o.rv[(size_t)sp[2 * s + i] * NV + n] -= t.sfmv[i][k] * o.re[((size_t)s * em + k) * NV + n];
    for (size_t k = 0; k < o.rv.size(); ++k) o.rv[k] *= (1.0 / o.vprcn[k]) * t.vdiag;
    all_dirichlet(o);
    for (int tind = 0; tind < o.ntet; ++tind) {
        double uh[4][NV];
        for (int j = 0; j < 4; ++j)
            for (int n = 0; n < NV; ++n) uh[j][n] = o.rv[(size_t)o.tp[4 * tind + j] * NV + n] * o.iprcn[(size_t)tind * NV + n];
        for (int i = 0; i < 6; ++i) {
            const int s = o.ts[6 * tind + i], sg = o.tsg[6 * tind + i];
            for (int j = 0; j < 4; ++j) {
                double msgn = 1.0;
                for (int k = 0; k < em; ++k) {
                    for (int n = 0; n < NV; ++n)
                        o.re[((size_t)s * em + k) * NV + n] -= msgn * t.mm[j][4 + k + i * em] * uh[j][n];
                    msgn *= sg;
                }
            }
        }
    }
    for (int s = 0; s < o.nseg; ++s)
        for (int n = 0; n < NV; ++n) o.re[((size_t)s * em) * NV + n] *= (1.0 / o.eprcn[(size_t)s * NV + n]) * 100.0;
    all_dirichlet(o);
}

// Edge end points in the global direction: tet_sgn = +1 where the tetrahedron's local edge i
// runs from its first to its second local vertex (VS) the way the global edge does.
static const int VS[6][2] = {{2, 3}, {3, 1}, {2, 1}, {1, 0}, {2, 0}, {3, 0}};
static std::vector<int> seg_ends(const OT &o) {
    std::vector<int> sp(2 * (size_t)o.nseg);
    for (int tind = 0; tind < o.ntet; ++tind)
        for (int i = 0; i < 6; ++i) {
            const int s = o.ts[6 * tind + i], a = o.tp[4 * tind + VS[i][0]], b = o.tp[4 * tind + VS[i][1]];
            sp[2 * (size_t)s] = o.tsg[6 * tind + i] > 0 ? a : b;
            sp[2 * (size_t)s + 1] = o.tsg[6 * tind + i] > 0 ? b : a;
        }
    return sp;
}

// Face vertices and edges. A face takes its vertices from the tetrahedron that numbered it
// (rot = +1), in that tetrahedron's order VF of the face (tet_mesh::create_tri_from_tet,
// tet_mesh/setup.cpp:301-374); face edge i is the edge opposite face vertex i. That is the
// numbering tet_basis's face basis uses (proj2d.cpp:46-91), and with it tet_hp::minvrt's
// face steps (setup_preconditioner.cpp:16-44, 142-175) name the right edge ends.
static void face_topology(const OT &o, std::vector<int> &fp, std::vector<int> &fs) {
    fp.assign(3 * (size_t)o.ntri, -1);
    fs.assign(3 * (size_t)o.ntri, -1);
    for (int tind = 0; tind < o.ntet; ++tind)
        for (int i = 0; i < 4; ++i) {
            if (o.trot[4 * tind + i] < 0) continue;
            const int f = o.tt[4 * tind + i];
            for (int j = 0; j < 3; ++j) fp[3 * (size_t)f + j] = o.tp[4 * tind + VF[i][j]];
            for (int j = 0; j < 3; ++j) {
                const int a = VF[i][(j + 1) % 3], b = VF[i][(j + 2) % 3];
                for (int e = 0; e < 6; ++e)
                    if ((VS[e][0] == a && VS[e][1] == b) || (VS[e][0] == b && VS[e][1] == a))
                        fs[3 * (size_t)f + j] = o.ts[6 * tind + e];
            }
        }
}

// LU with partial pivoting of an n x n matrix, row-major, in place (the unblocked
// algorithm of LAPACK's dgetrf); piv[k] = the row swapped with row k. Returns 0, or k + 1
// when the pivot of column k is zero.
static int lu_factor(int n, double *a, int *piv) {
    for (int k = 0; k < n; ++k) {
        int r = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)r * n + k])) r = i;
        piv[k] = r;
        if (a[(size_t)r * n + k] == 0.0) return k + 1;
        if (r != k)
            for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)r * n + j]);
        for (int i = k + 1; i < n; ++i) {
            const double l = a[(size_t)i * n + k] / a[(size_t)k * n + k];
            a[(size_t)i * n + k] = l;
            for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
        }
    }
    return 0;
}

static void lu_solve(int n, const double *a, const int *piv, double *b) {
    for (int k = 0; k < n; ++k)
        if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int i = 1; i < n; ++i)
        for (int j = 0; j < i; ++j) b[i] -= a[(size_t)i * n + j] * b[j];
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) b[i] -= a[(size_t)i * n + j] * b[j];
        b[i] /= a[(size_t)i * n + i];
    }
}

// tet_hp::spoke (setup_preconditioner.cpp:530-583), p = 3: for every vertex the matrix of its
// spokes (the edges at the vertex, numbered in the order the vertex ball first meets them:
// tetrahedra by index, then local edges 0..5), summed over the tetrahedra of the ball with
// the tetrahedron's iprcn(tind, 0): mdiag on the diagonal of each of its three edges at the
// vertex, odiag between them; factored by LU. The matrix is symmetric, so the transposed
// solve of minvrt (dgetrs "T") is the plain one.
struct Spokes {
    std::vector<int> ptr, seg, end, fptr, piv;
    std::vector<double> lu;
};
static int spoke(const OT &o, const std::vector<int> &sp, Spokes &S) {
    std::vector<std::vector<int>> ball(o.npnt);
    for (int tind = 0; tind < o.ntet; ++tind)
        for (int j = 0; j < 4; ++j) ball[o.tp[4 * tind + j]].push_back(tind);
    S.ptr.assign(o.npnt + 1, 0);
    S.fptr.assign(o.npnt + 1, 0);
    S.seg.clear(); S.end.clear(); S.lu.clear(); S.piv.clear();
    std::vector<int> local(o.nseg, -1);
    for (int v = 0; v < o.npnt; ++v) {
        const int base = (int)S.seg.size();
        std::vector<int> tri3;  // per ball tetrahedron: its three spokes
        for (int tind : ball[v])
            for (int j = 0; j < 6; ++j) {
                const int s = o.ts[6 * tind + j];
                for (int k = 0; k < 2; ++k)
                    if (sp[2 * (size_t)s + k] == v) {
                        if (local[s] < 0) {
                            local[s] = (int)S.seg.size() - base;
                            S.seg.push_back(s);
                            S.end.push_back(k);
                        }
                        tri3.push_back(local[s]);
                    }
            }
        const int n = (int)S.seg.size() - base;
        S.ptr[v + 1] = (int)S.seg.size();
        std::vector<double> a((size_t)n * n, 0.0);
        for (size_t b = 0; b < ball[v].size(); ++b) {
            const double jcb = o.iprcn[(size_t)ball[v][b] * NV];
            const int *e0 = &tri3[3 * b];
            for (int j = 0; j < 3; ++j) {
                a[(size_t)e0[j] * n + e0[j]] += jcb * o.t.mdiag;
                for (int k = 0; k < 3; ++k)
                    if (k != j) a[(size_t)e0[j] * n + e0[k]] += jcb * o.t.odiag;
            }
        }
        std::vector<int> piv(n);
        if (lu_factor(n, a.data(), piv.data())) return v + 1;
        S.lu.insert(S.lu.end(), a.begin(), a.end());
        S.piv.insert(S.piv.end(), piv.begin(), piv.end());
        S.fptr[v + 1] = (int)S.lu.size();
        for (int k = base; k < (int)S.seg.size(); ++k) local[S.seg[k]] = -1;
    }
    return 0;
}

static void edirichlet(OT &o) {
    if (o.me.empty()) return;
    for (int e = 0; e < o.nseg; ++e)
        for (int m = 0; m < o.t.em; ++m)
            for (int n = 0; n < NV; ++n)
                if (o.me[(size_t)e * NV + n]) o.re[((size_t)e * o.t.em + m) * NV + n] = 0.0;
}
static void fdirichlet(OT &o) {
    if (o.mf.empty()) return;
    for (int f = 0; f < o.ntri; ++f)
        for (int m = 0; m < o.t.fm; ++m)
            for (int n = 0; n < NV; ++n)
                if (o.mf[(size_t)f * NV + n]) o.rf[((size_t)f * o.t.fm + m) * NV + n] = 0.0;
}

// tet_hp::minvrt at p = 3 (setup_preconditioner.cpp:16-354, em = 2, fm = 1, im = 0; iprcn is
// not inverted at im = 0, tet_hp::setup_preconditioner :463-465):
//  (1) edge and face modes removed from the vertices (sfmv, ffmv), the vertex rows scaled by
//      vdiag / vprcn and fixed;
//  (2) the vertex values times iprcn removed from the edge and face modes (mass matrix);
//  (3) the edges' first modes from the vertex-ball solves: per edge end the spoke value
//      e0 +- sfms(0) e1 plus the face modes times ffms, solved per vertex with its spoke
//      factor, each edge receiving half of each end's solution; fixed edges zeroed;
//  (4) the first edge modes times iprcn removed from the second edge modes and the faces
//      (mass matrix), the second edge modes scaled by ediag(1) / eprcn, ediag(1) = 1000 as
//      minvrt sets it, and fixed;
//  (5) the second edge modes times iprcn removed from the faces (minvrt takes res.e(side,1)
//      without the tetrahedron's edge sign here, and so does this restatement), the faces
//      scaled by fdiag(0) / fprcn, fdiag(0) = 3000, and fixed.
static void minvrt_p3(OT &o, const Spokes &S, const std::vector<int> &sp, const std::vector<int> &fp,
                      const std::vector<int> &fs) {
    const hp_tet_tables &t = o.t;
    const int em = t.em, fm = t.fm;
    auto E = [&](int s, int k, int n) -> double & { return o.re[((size_t)s * em + k) * NV + n]; };
    auto F = [&](int f, int k, int n) -> double & { return o.rf[((size_t)f * fm + k) * NV + n]; };
    // (1)
    for (int s = 0; s < o.nseg; ++s)
        for (int k = 0; k < em; ++k)
            for (int i = 0; i < 2; ++i)
                for (int n = 0; n < NV; ++n) o.rv[(size_t)sp[2 * s + i] * NV + n] -= t.sfmv[i][k] * E(s, k, n);
    for (int f = 0; f < o.ntri; ++f)
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < fm; ++k)
                for (int n = 0; n < NV; ++n) o.rv[(size_t)fp[3 * f + i] * NV + n] -= t.ffmv[i][k] * F(f, k, n);
    for (size_t k = 0; k < o.rv.size(); ++k) o.rv[k] *= (1.0 / o.vprcn[k]) * t.vdiag;
    all_dirichlet(o);
    // (2)
    for (int tind = 0; tind < o.ntet; ++tind) {
        double uh[4][NV];
        for (int j = 0; j < 4; ++j)
            for (int n = 0; n < NV; ++n) uh[j][n] = o.rv[(size_t)o.tp[4 * tind + j] * NV + n] * o.iprcn[(size_t)tind * NV + n];
        for (int i = 0; i < 6; ++i) {
            const int s = o.ts[6 * tind + i], sg = o.tsg[6 * tind + i];
            for (int j = 0; j < 4; ++j) {
                double msgn = 1.0;
                for (int k = 0; k < em; ++k) {
                    for (int n = 0; n < NV; ++n) E(s, k, n) -= msgn * t.mm[j][4 + k + i * em] * uh[j][n];
                    msgn *= sg;
                }
            }
        }
        for (int i = 0; i < 4; ++i) {
            const int f = o.tt[4 * tind + i], sg = -o.trot[4 * tind + i];
            for (int j = 0; j < 4; ++j) {
                double msgn = 1.0;
                int ind = 0;
                for (int m = 1; m <= em - 1; ++m) {
                    for (int k = 1; k <= em - m; ++k, ++ind)
                        for (int n = 0; n < NV; ++n) F(f, ind, n) -= msgn * t.mm[j][4 + 6 * em + i * fm + ind] * uh[j][n];
                    msgn *= sg;
                }
            }
        }
    }
    // (3)
    std::vector<double> w((size_t)o.nseg * 2 * NV);
    for (int s = 0; s < o.nseg; ++s)
        for (int n = 0; n < NV; ++n) {
            w[((size_t)s * 2 + 0) * NV + n] = E(s, 0, n) + t.sfms0 * E(s, 1, n);
            w[((size_t)s * 2 + 1) * NV + n] = E(s, 0, n) - t.sfms0 * E(s, 1, n);
            E(s, 0, n) = 0.0;
        }
    for (int f = 0; f < o.ntri; ++f)
        for (int i = 0; i < 3; ++i) {
            const int s = fs[3 * f + i], x = fp[3 * f + (i == 0 ? 2 : 0)];
            const int c1 = sp[2 * (size_t)s] == x ? 0 : 1;  // the spoke end that takes ffms(i, k, 1)
            for (int k = 0; k < fm; ++k)
                for (int n = 0; n < NV; ++n) {
                    w[((size_t)s * 2 + c1) * NV + n] += t.ffms[i][k][1] * F(f, k, n);
                    w[((size_t)s * 2 + 1 - c1) * NV + n] += t.ffms[i][k][0] * F(f, k, n);
                }
        }
    std::vector<double> rhs;
    for (int v = 0; v < o.npnt; ++v) {
        const int b = S.ptr[v], nspk = S.ptr[v + 1] - b;
        rhs.resize(nspk);
        for (int n = 0; n < NV; ++n) {
            for (int k = 0; k < nspk; ++k) rhs[k] = w[((size_t)S.seg[b + k] * 2 + S.end[b + k]) * NV + n];
            lu_solve(nspk, &S.lu[S.fptr[v]], &S.piv[b], rhs.data());
            for (int k = 0; k < nspk; ++k) E(S.seg[b + k], 0, n) += rhs[k] / 2.0;
        }
    }
    edirichlet(o);
    // (4)
    for (int tind = 0; tind < o.ntet; ++tind) {
        double uh[6][NV];
        for (int i = 0; i < 6; ++i)
            for (int n = 0; n < NV; ++n) uh[i][n] = E(o.ts[6 * tind + i], 0, n) * o.iprcn[(size_t)tind * NV + n];
        for (int i = 0; i < 6; ++i) {
            const int s = o.ts[6 * tind + i], sg = o.tsg[6 * tind + i];
            for (int j = 0; j < 6; ++j) {
                double msgn = sg;
                for (int k = 1; k < em; ++k) {
                    for (int n = 0; n < NV; ++n) E(s, k, n) -= msgn * t.mm[k + 4 + i * em][4 + j * em] * uh[j][n];
                    msgn *= sg;
                }
            }
        }
        for (int i = 0; i < 4; ++i) {
            const int f = o.tt[4 * tind + i], sg = -o.trot[4 * tind + i];
            for (int j = 0; j < 6; ++j) {
                double msgn = 1.0;
                int ind = 0;
                for (int m = 1; m <= em - 1; ++m) {
                    for (int k = 1; k <= em - m; ++k, ++ind)
                        for (int n = 0; n < NV; ++n)
                            F(f, ind, n) -= msgn * t.mm[4 + 6 * em + i * fm + ind][4 + j * em] * uh[j][n];
                    msgn *= sg;
                }
            }
        }
    }
    for (int s = 0; s < o.nseg; ++s)
        for (int n = 0; n < NV; ++n) E(s, 1, n) *= (1.0 / o.eprcn[(size_t)s * NV + n]) * 1000.0;
    edirichlet(o);
    // (5)
    for (int tind = 0; tind < o.ntet; ++tind) {
        double uh[6][NV];
        for (int i = 0; i < 6; ++i)
            for (int n = 0; n < NV; ++n) uh[i][n] = E(o.ts[6 * tind + i], 1, n) * o.iprcn[(size_t)tind * NV + n];
        for (int i = 0; i < 4; ++i) {
            const int f = o.tt[4 * tind + i], sg = -o.trot[4 * tind + i];
            for (int j = 0; j < 6; ++j) {
                double msgn = 1.0;
                int ind = 0;
                for (int m = 1; m <= em - 1; ++m) {
                    for (int k = 1; k <= em - m; ++k, ++ind)
                        for (int n = 0; n < NV; ++n)
                            F(f, ind, n) -= msgn * t.mm[4 + 6 * em + i * fm + ind][5 + j * em] * uh[j][n];
                    msgn *= sg;
                }
            }
        }
    }
    for (int f = 0; f < o.ntri; ++f)
        for (int k = 0; k < fm; ++k)
            for (int n = 0; n < NV; ++n) F(f, k, n) *= (1.0 / o.fprcn[(size_t)f * NV + n]) * 3000.0;
    fdirichlet(o);
}

// The face vertices and edges minvrt at p = 3 uses, [ntri][3] each (face_topology).
void ot_face_topology(void *h, int *fp, int *fs) {
    const OT &o = *static_cast<const OT *>(h);
    std::vector<int> a, b;
    face_topology(o, a, b);
    std::memcpy(fp, a.data(), a.size() * 4);
    std::memcpy(fs, b.data(), b.size() * 4);
}

// 0: the JACOBI build's smoother, 1: minvrt (p = 1, 2 and 3; -1 otherwise)
int ot_set_smoother(void *h, int kind) {
    OT &o = *static_cast<OT *>(h);
    if (kind != 0 && (kind != 1 || o.t.p > 3)) return -1;
    o.smoother = kind;
    return 0;
}

void ot_rsdl(void *h, int stage);

// tet_hp::update (update.cpp:181-390): nstage stages of rsdl, boundary zeroing, the
// smoother (jacobi_relaxation in the JACOBI build, else minvrt) and
// ug = ug0 - alpha(stage) cfl res.
void ot_update(void *h) {
    OT &o = *static_cast<OT *>(h);
    o.u0v = o.ugv; o.u0e = o.uge; o.u0f = o.ugf; o.u0i = o.ugi;
    // p = 3: the spoke factors of tet_hp::setup_preconditioner, from the iprcn of the last
    // ot_setup_preconditioner (the same for every stage)
    Spokes S;
    std::vector<int> sp, fp, fs;
    if (o.smoother && o.t.p == 3) {
        sp = seg_ends(o);
        face_topology(o, fp, fs);
        spoke(o, sp, S);
    }
    for (int stage = 0; stage < o.ph.nstage; ++stage) {
        ot_rsdl(h, stage);
        all_dirichlet(o);
        if (o.smoother) {
            if (o.t.p == 1) minvrt_p1(o);
            else if (o.t.p == 2) minvrt_p2(o);
            else minvrt_p3(o, S, sp, fp, fs);
        } else {
            jacobi_relaxation(o);
        }
        const double ca = o.ph.alpha[stage] * o.ph.cfl;
        for (size_t k = 0; k < o.ugv.size(); ++k) o.ugv[k] = o.u0v[k] - ca * o.rv[k];
        for (size_t k = 0; k < o.uge.size(); ++k) o.uge[k] = o.u0e[k] - ca * o.re[k];
        for (size_t k = 0; k < o.ugf.size(); ++k) o.ugf[k] = o.u0f[k] - ca * o.rf[k];
        for (size_t k = 0; k < o.ugi.size(); ++k) o.ugi[k] = o.u0i[k] - ca * o.ri[k];
    }
}

void ot_get_jacobian_diagonal(void *h, double *v, double *e, double *f, double *i) {
    OT &o = *static_cast<OT *>(h);
    std::memcpy(v, o.jv.data(), o.jv.size() * 8);
    if (!o.je.empty()) std::memcpy(e, o.je.data(), o.je.size() * 8);
    if (!o.jf.empty()) std::memcpy(f, o.jf.data(), o.jf.size() * 8);
    if (!o.ji.empty()) std::memcpy(i, o.ji.data(), o.ji.size() * 8);
}

// tet_hp::rsdl (update.cpp:9-118): boundary-face fluxes, then the element loop; no
// coarse-level terms
void ot_rsdl(void *h, int stage) {
    OT &o = *static_cast<OT *>(h);
    const double omb = 1.0 - o.ph.beta[stage];
    for (auto *a : {&o.rv, &o.re, &o.rf, &o.ri}) std::fill(a->begin(), a->end(), 0.0);
    for (auto *a : {&o.rrv, &o.rre, &o.rrf, &o.rri})
        for (auto &x : *a) x *= omb;
    for (size_t b = 0; b < o.bf_tri.size(); ++b) face_flux(o, (int)b);
    double lf_re[NV][HP_TET_MAXT], lf_im[NV][HP_TET_MAXT];
    for (int tind = 0; tind < o.ntet; ++tind) {
        element_rsdl(o, tind, stage, lf_re, lf_im);
        scatter(o, tind, lf_im, o.rv.data(), o.re.data(), o.rf.data(), o.ri.data());
        scatter(o, tind, lf_re, o.rrv.data(), o.rre.data(), o.rrf.data(), o.rri.data());
    }
    for (size_t k = 0; k < o.rv.size(); ++k) o.rv[k] += o.rrv[k];
    for (size_t k = 0; k < o.re.size(); ++k) o.re[k] += o.rre[k];
    for (size_t k = 0; k < o.rf.size(); ++k) o.rf[k] += o.rrf[k];
    for (size_t k = 0; k < o.ri.size(); ++k) o.ri[k] += o.rri[k];
}

}  // extern "C"
