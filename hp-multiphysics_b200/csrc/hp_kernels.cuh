// Device code of the element-residual / multistage-smoothing path (sm_100a).
//
// Layout in HBM (element-major blocks, the reference's own blitz layouts):
//   ug.v/res.v/res_r.v [npnt][NV], ug.s/... [nseg][sm][NV], ug.i/... [ntri][im][NV]
//   mesh: tri_pnt/tri_seg/tri_sgn [ntri][3] int32,
//         seg_pnt/seg_tri/seg_loc [nseg][2], vertex incidence in CSR form.
// Each element is processed by one warp: the warp gathers the element's modes,
// runs the sum-factorised contractions (proj -> point fluxes -> intgrtrs,
// derivr/derivs for the strong residual) through shared memory, and scatters the
// local residual: vertex and side modes with FP64/FP32 atomics, interior modes
// with plain stores (they belong to one element).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hpb {

// Compact per-p tables on the device (copied from hp_basis_tables).
template <typename R, int P>
struct DevTables {
    static constexpr int G = P + 1, X = P + 2, T = (P + 1) * (P + 2) / 2, SM = P - 1, IM = (P - 1) * (P - 2) / 2,
                         BM = 3 * P;
    R gx[G][X], dgx[G][X], x0[G];
    R gn[G][T], dgn[G][T], n0[G];
    R gxwtx[X][G], dgxwtx[X][G];
    R gnwtn[T][G], gnwtnn0[T][G], dgnwtn[T][G];
    R dltx[G], dltx1[G][G], dltn[G], dltn1[G][G], dltn2[G][G];
    R wtx[G];
    int colstart[X + 1], colmodes[T], colof[T];
};

// minvrt tables (FP64 or FP32 copies)
template <typename R>
struct DevMinv {
    R sfmv[2][8], vfms[3][8], sdiag[8], sfms[8][8][3];
    R ifmb[24][21], bfmi[24][21], idiag[21][2];
    R vdiag;
};

struct Phys {
    int physics, NV, nstage;
    double alpha[8], beta[8];
    double cfl, bd0, adis, rho, mu, rhocv, kcond, ax, ay, src;
};

struct Mesh {
    int npnt, nseg, ntri, nbseg;
    const double *pnts;  // [npnt][2]
    const int *tri_pnt, *tri_seg;
    const int *tri_sgn;  // [ntri][3]
    const int *seg_pnt, *seg_tri, *seg_loc;  // [nseg][2]
    const int *vs_ptr, *vs_idx;  // vertex -> (seg*2+end)
    const int *vt_ptr, *vt_idx;  // vertex -> (tri*4+local)
    const int *vess, *sess;      // essential masks
    const int *bseg, *bkind;
    const double *bpibc;  // [nbseg][G]
    // curved elements (tri.info > -1): tri_cv[t] = index into crv_cht or -1;
    // crv_cht[cv][2][BM] = vertex and side position modes (crdtocht); bcrd[e][sm][2] =
    // side position modes of boundary edge e (NULL: all straight)
    const int *tri_cv;
    const double *crv_cht;
    const double *bcrd;
    int ncurved;         // number of curved elements
    const int *crv_tri;  // [ncurved] their triangle indices (crv_cht order)
    // boundary edges seen from the entities: seg_bdry[s] = boundary edge of segment s or -1;
    // vb_idx[v][2] = 2 e + end of the (at most two) boundary edges ending at vertex v, or -1
    const int *seg_bdry, *vb_idx;
    // owner order of the assembly buffers: vpos[3 t + c] = position of (t, corner c) in the
    // vertex-incidence list (vt_idx), spos[3 t + i] = 2 s + k for side i of t being
    // seg.tri(k) of segment s
    const int *vpos, *spos;
    // per-triangle constants of the straight-element branch [ntri][8]: ldcrd d00, d01, d10,
    // d11, 1 / |J|, the tau length scale h (inscribed radius / (0.25 (p+1)^2)), 1 / h, unused
    const double *tgeo;
};

// Slot of an element's vertex / side residual in the assembly buffers (State::elim,
// elre): vertex values in vertex-incidence order [3 ntri][NV], then side values in
// segment order [2 nseg][SM][NV], so that k_assemble reads each vertex's and each side's
// contributions contiguously.
__device__ __forceinline__ size_t asm_slot(const Mesh &m, int NV, int SM, int vp, int sp, int mode, int n) {
    if (mode < 3) return (size_t)vp * NV + n;
    const int kk = (mode - 3) % SM;
    return (size_t)3 * m.ntri * NV + ((size_t)sp * SM + kk) * NV + n;
}

template <typename R>
struct State {
    R *ugv, *ugs, *ugi;
    R *u0v, *u0s, *u0i;
    R *resv, *ress, *resi;
    R *rrv, *rrs, *rri;
    R *vprcn, *sprcn, *tprcn, *tau;
    // Correction (defect) form: ug holds a correction d about the base state ub and
    // the residual is R(ub + d) - R(ub) + dres (the FP64 residual of the base, as the
    // reference's mg_source adds dres on coarse levels, nstage.cpp:113-129). NULL
    // pointers = plain form.
    const R *ubv, *ubs, *ubi;
    const R *dresv, *dress, *dresi;
    // Assembly by gather (FP64): when elim != NULL, the element kernels write each
    // element's vertex and side residuals (lftog's values, side signs applied) to
    // elim / elre [ntri][BM][NV] (imaginary / beta-scaled real part) and the boundary
    // fluxes go to bres [nbseg][SM+2][NV] (end 0, end 1, side modes), without atomics;
    // k_assemble then sums them per vertex and side in a fixed order, so repeated
    // residual evaluations are bitwise identical. NULL: FP64/FP32 atomics.
    R *elim, *elre, *bres;
    // Correction form on the tensor cores: the base state's point values (u, v)
    // [ntri][2][GG] (k_base_points), fixed for a correction cycle; NULL: not computed.
    const R *bpt;
};

__device__ __forceinline__ void atomic_add(double *a, double v) { atomicAdd(a, v); }
__device__ __forceinline__ void atomic_add(float *a, float v) { atomicAdd(a, v); }

template <typename R>
__device__ __forceinline__ R rsqrt_(R x);
template <>
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_(float x) { return sqrtf(x); }

// ---------------------------------------------------------------------------
// Element residual: one warp per element.
// ---------------------------------------------------------------------------
template <typename R, int P, int PHYS>
struct ElemCfg {
    static constexpr int G = P + 1, X = P + 2, T = (P + 1) * (P + 2) / 2, SM = P - 1, IM = (P - 1) * (P - 2) / 2,
                         BM = 3 * P;
    static constexpr int NV = (PHYS == 1 ? 3 : 1);
    static constexpr int NPAIR = NV;               // flux pairs integrated by intgrtrs
    static constexpr int NQ = (PHYS == 1 ? 16 : 7);  // per-point scratch values
    static constexpr int WPC = (P <= 4 ? 8 : 4);   // warps per CTA
    static constexpr int EPW = (P == 1 ? 4 : (P <= 3 ? 2 : 1));  // elements per warp (lane groups)
    static constexpr int NB = (PHYS == 1 ? 2 : 0);  // base-state variables gathered in correction form
    // per-warp scratch (in R units)
    static constexpr int S_UHT = (NV + NB) * T;
    static constexpr int S_WK = (PHYS == 1 ? 7 : 6) * G * X;
    static constexpr int S_PT = (NQ + NV + 1) * G * G;
    static constexpr int S_WARP = S_UHT + S_WK + S_PT;
};

// Point-array slot indices (each slot is a [G][G] array)
// ins: 0..3 cvI (cv00,cv01,cv10,cv11)  4,5 mI  6..9 cvT  10..13 df  14,15 u,v  16..18 res  19 q
// cd : 0,1 cvI  2,3 cvT  4,5 e  6 u      7 res
// Correction form (diff != 0, ins): uht holds d, uht+NV*T the base velocity b; the
// fluxes are the exact differences F(b+d) - F(b) of the convective, pressure and
// viscous terms, the SUPG term A(b+d) tau(b) res(d) with tau frozen at the base.

// Element operators of the linear cd residual. For uht = e_j, aim(t, j, m) = lf_im(m)
// and are(t, j, m) = lf_re(m) at beta = 1; bre[t][m] = lf_re(m) of the source alone
// (uht = 0). Storage is in tiles of EB elements, column-major inside a tile (the EB*T
// entries of one column that a CTA reads together are contiguous), each tile padded to
// a 16-byte multiple:
//   index(t, j, m) = (t / EB) * TS + j * (EB * T) + (t % EB) * T + m,  TS >= T * EB * T.
// Finite-difference element Jacobians (tri_hp::element_jacobian, nstage.cpp:131-165, fixed
// mesh): pass 0 stores every element's stage-0 residual lf_re + lf_im in rbar [ntri][T][NV];
// pass 1 runs one item per (element, column kcol = mode * NV + var) with that unknown raised
// by dw(var) = 1e-8 sum_{i<3} |uht(var)(i)| + 1e-8 and writes
// K[tind][krow = i * NV + n][kcol] = (lf_re(n)(i) + lf_im(n)(i) - rbar) / dw(var).
template <typename R>
struct ElemJac {
    R *K, *rbar;
    int pass;
};

template <typename R>
struct ElemMat {
    R *aim, *are, *bre;
};

template <int P>
struct EmatCfg {
    static constexpr int T = (P + 1) * (P + 2) / 2;
    static constexpr int EB = (128 / T > 0 ? 128 / T : 1);            // elements per tile
    static constexpr int TS = ((T * EB * T + 3) / 4) * 4;             // tile stride (entries)
    __host__ __device__ static size_t idx(long t, int j, int m) {
        return (size_t)(t / EB) * TS + (size_t)j * (EB * T) + (size_t)(t % EB) * T + m;
    }
    static size_t len(long ntri) { return (size_t)((ntri + EB - 1) / EB) * TS; }
};

// Column of mode m in the sum factorisation (proj.cpp:46-95, intgrt.cpp:44-76): vertex
// modes 0, 1, 2 own columns 0, 1, 2; side-0 modes own columns 3 .. sm+2; side-1 modes
// join column 2, side-2 modes column 1; interior blocks of sm-1, sm-2, ... modes join
// columns 3, 4, .... A compile-time function of p, so unrolled loops index registers.
template <int P>
struct ModeCols {
    static constexpr int SM = P - 1, BM = 3 * P, BS1 = SM + 3, BS2 = 2 * SM + 3;
    __host__ __device__ static constexpr int col(int m) {
        if (m < BS1) return m;
        if (m < BS2) return 2;
        if (m < BM) return 1;
        int idx = m - BM, c = 3, cnt = SM - 1;
        while (idx >= cnt) { idx -= cnt; --cnt; ++c; }
        return c;
    }
};

// Isoparametric metrics of a curved element at quadrature point (i, j): the r and s
// derivatives of x and y from the element's vertex and side position modes (interior
// modes zero), dcrd(n,0) = d x_n / dr and dcrd(n,1) = d x_n / ds (proj_bdry with
// derivatives, tri_basis/proj.cpp:201-281, of crdtocht, tri_hp/gtol.cpp:204-248).
template <typename R, int P>
__device__ __forceinline__ void curved_metrics(const DevTables<R, P> &tb, const double *cht, int i, int j, R &d00,
                                               R &d01, R &d10, R &d11) {
    constexpr int X = P + 2, BM = 3 * P;
    R l1[2] = {(R)0, (R)0}, l2[2] = {(R)0, (R)0};
    const R oeta = tb.n0[j];
    for (int n = 0; n < X; ++n) {
        R w0[2] = {(R)0, (R)0}, w1[2] = {(R)0, (R)0};
        for (int c = tb.colstart[n]; c < tb.colstart[n + 1]; ++c) {
            const int m = tb.colmodes[c];
            if (m >= BM) continue;
            for (int k = 0; k < 2; ++k) {
                const R v = (R)cht[k * BM + m];
                w0[k] += v * tb.gn[j][m];
                w1[k] += v * tb.dgn[j][m];
            }
        }
        for (int k = 0; k < 2; ++k) {
            l1[k] += w1[k] * tb.gx[i][n];
            l2[k] += (w0[k] * oeta) * tb.dgx[i][n];
        }
    }
    d00 = l2[0];
    d01 = l1[0] + tb.x0[i] * l2[0];
    d10 = l2[1];
    d11 = l1[1] + tb.x0[i] * l2[1];
}

// CTAs per SM the straight-element kernel keeps resident (caps its registers): cd 64
// registers a thread; ins 85 (FP64, 8 warps), 128 (FP64, 4 warps), 64 (FP32).
template <typename R, int P, int PHYS, bool CURVED>
struct ElemMinBlocks {
    static constexpr int WPC = ElemCfg<R, P, PHYS>::WPC;
    static constexpr int value = CURVED ? 1
                                 : PHYS == 0 ? 256 / WPC / 8
                                 : sizeof(R) == 8 ? (WPC == 8 ? 3 : 4)
                                                  : (WPC == 8 ? 4 : 8);
};

// CURVED = false: the straight elements (curved ones are skipped); CURVED = true: the
// mesh's curved elements only (mesh.crv_tri), with metrics at every quadrature point.
template <typename R, int P, int PHYS, bool CURVED>
__global__ void __launch_bounds__(ElemCfg<R, P, PHYS>::WPC * 32, ElemMinBlocks<R, P, PHYS, CURVED>::value)
    k_rsdl_elem(const DevTables<R, P> *__restrict__ gtab, Mesh mesh, State<R> st, Phys ph, int stage, int zero_rr,
                int diff, ElemMat<R> build, ElemJac<R> jac) {
    using C = ElemCfg<R, P, PHYS>;
    constexpr int G = C::G, X = C::X, T = C::T, IM = C::IM, BM = C::BM, NV = C::NV, GG = G * G;
    constexpr int SM = (C::SM > 0 ? C::SM : 1);  // side-mode stride (unused when p = 1)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevTables<R, P> &tb = *reinterpret_cast<DevTables<R, P> *>(smem_raw);
    R *warp_base = reinterpret_cast<R *>(smem_raw + ((sizeof(DevTables<R, P>) + 15) / 16) * 16);
    {
        const int n4 = sizeof(DevTables<R, P>) / 4;
        const int *src = reinterpret_cast<const int *>(gtab);
        int *dst = reinterpret_cast<int *>(smem_raw);
        for (int k = threadIdx.x; k < n4; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // EPW elements per warp, one group of LW lanes each (all groups pass the same
    // __syncwarp sequence; a group without an element idles through it)
    constexpr int EPW = C::EPW, LW = 32 / EPW;
    const int grp = lane / LW, sl = lane - grp * LW;
    R *uht = warp_base + (warp * EPW + grp) * C::S_WARP;
    R *wk = uht + C::S_UHT;
    R *pt = wk + C::S_WK;
    auto PT = [&](int q) -> R * { return pt + q * GG; };

    const R beta = (R)ph.beta[stage];
    const R omb = zero_rr ? (R)0 : (R)1 - beta;

    // build mode (cd): one item per (element, column j) with uht = e_j, j = T: uht = 0
    const bool bmode = (PHYS == 0) && build.aim != nullptr;
    const bool jmode = jac.rbar != nullptr, jcols = jmode && jac.pass == 1;
    constexpr int NJ = NV * T;  // Jacobian columns per element
    const long nel = CURVED ? (long)mesh.ncurved : (long)mesh.ntri;
    const long nitems = bmode ? nel * (T + 1) : (jcols ? nel * NJ : nel);
    for (long wbase = ((long)blockIdx.x * C::WPC + warp) * EPW; wbase < nitems;
         wbase += (long)gridDim.x * C::WPC * EPW) {
        const long item = (wbase + grp < nitems) ? wbase + grp : wbase;
        const int eidx = bmode ? (int)(item / (T + 1)) : (jcols ? (int)(item / NJ) : (int)item);
        const int bcol = bmode ? (int)(item - (long)eidx * (T + 1)) : -1;
        const int jcol = jcols ? (int)(item - (long)eidx * NJ) : 0;
        const int tind = CURVED ? mesh.crv_tri[eidx] : eidx;
        // curved elements are done by the curved launch
        const bool act = (wbase + grp < nitems) && (CURVED || !mesh.tri_cv || mesh.tri_cv[tind] < 0);
        if (EPW == 1 && !act) continue;
        const int p0 = mesh.tri_pnt[3 * tind], p1 = mesh.tri_pnt[3 * tind + 1], p2 = mesh.tri_pnt[3 * tind + 2];
        // ---- gather (ugtouht, gtol.cpp:14-55)
        for (int w = sl; act && w < NV * T; w += LW) {
            const int n = w / T, m = w - n * T;
            R val;
            if (bmode) {
                val = (m == bcol) ? (R)1 : (R)0;
            } else if (m < 3) {
                const int v = (m == 0 ? p0 : (m == 1 ? p1 : p2));
                val = st.ugv[v * NV + n];
            } else if (m < BM) {
                const int i = (m - 3) / SM, k = (m - 3) - i * SM;
                const int sind = mesh.tri_seg[3 * tind + i], sg = mesh.tri_sgn[3 * tind + i];
                val = st.ugs[(sind * SM + k) * NV + n];
                if ((k & 1) && sg < 0) val = -val;
            } else {
                val = st.ugi[((size_t)tind * IM + (m - BM)) * NV + n];
            }
            uht[n * T + m] = val;
        }
        if (PHYS == 1 && diff) {
            for (int w = sl; act && w < 2 * T; w += LW) {
                const int n = w / T, m = w - n * T;
                R val;
                if (m < 3) {
                    const int v = (m == 0 ? p0 : (m == 1 ? p1 : p2));
                    val = st.ubv[v * NV + n];
                } else if (m < BM) {
                    const int i = (m - 3) / SM, k = (m - 3) - i * SM;
                    const int sind = mesh.tri_seg[3 * tind + i], sg = mesh.tri_sgn[3 * tind + i];
                    val = st.ubs[(sind * SM + k) * NV + n];
                    if ((k & 1) && sg < 0) val = -val;
                } else {
                    val = st.ubi[((size_t)tind * IM + (m - BM)) * NV + n];
                }
                uht[(NV + n) * T + m] = val;
            }
        }
        R jdw = (R)1;
        if (jcols) {
            __syncwarp();
            const int jm = jcol / NV, jn = jcol - jm * NV;
            jdw = (R)1e-8 * (fabs(uht[jn * T]) + fabs(uht[jn * T + 1]) + fabs(uht[jn * T + 2])) + (R)1e-8;
            __syncwarp();
            if (act && sl == 0) uht[jn * T + jm] += jdw;
        }
        // geometry (straight element): ldcrd(n,0) = (v2-v1)/2, ldcrd(n,1) = (v0-v1)/2
        const double x0d = mesh.pnts[2 * p0], y0d = mesh.pnts[2 * p0 + 1];
        const double x1d = mesh.pnts[2 * p1], y1d = mesh.pnts[2 * p1 + 1];
        const double x2d = mesh.pnts[2 * p2], y2d = mesh.pnts[2 * p2 + 1];
        const R g00 = (R)(0.5 * (x2d - x1d)), g01 = (R)(0.5 * (x0d - x1d));
        const R g10 = (R)(0.5 * (y2d - y1d)), g11 = (R)(0.5 * (y0d - y1d));
        // curved element: metrics at every point from its position modes (rsdl.cpp:83-258)
        const double *cht = CURVED ? mesh.crv_cht + (size_t)eidx * 2 * BM : nullptr;
        auto metric = [&](int i, int j, R &a, R &b, R &c, R &d) {
            if constexpr (CURVED) curved_metrics<R, P>(tb, cht, i, j, a, b, c, d);
            else { a = g00; b = g01; c = g10; d = g11; }
        };
        __syncwarp();
        // ---- proj stage I (proj.cpp:46-95): wk[q][j][n]; q = 2*var (value), 2*var+1 (d/deta)
        {
            constexpr int NDV = (PHYS == 1 ? 2 : 1);  // variables projected with derivatives
            constexpr int NQW = 2 * NDV + (NV - NDV);
            const int nqw = NQW + ((PHYS == 1 && diff) ? 2 : 0);  // + base u, v values
            // one lane per (quantity, eta point): all X column sums in registers, modes in
            // increasing order within each column (the order of the column lists)
            for (int w = sl; act && w < nqw * G; w += LW) {
                const int q = w / G, j = w - q * G;
                int var, der;
                if (q < 2 * NDV) { var = q >> 1; der = q & 1; }
                else { var = NDV + (q - 2 * NDV); der = 0; }
                const R *lin = uht + var * T;
                const R *g = der ? &tb.dgn[j][0] : &tb.gn[j][0];
                R acc[X];
#pragma unroll
                for (int n = 0; n < X; ++n) acc[n] = (R)0;
#pragma unroll
                for (int m = 0; m < T; ++m) acc[ModeCols<P>::col(m)] += lin[m] * g[m];
#pragma unroll
                for (int n = 0; n < X; ++n) wk[(q * G + j) * X + n] = acc[n];
            }
        }
        __syncwarp();
        // ---- proj stage II + pointwise fluxes
        for (int w = sl; act && w < GG; w += LW) {
            const int i = w / G, j = w - i * G;
            const R oeta = tb.n0[j], xp1 = tb.x0[i];
            R d00, d01, d10, d11;
            metric(i, j, d00, d01, d10, d11);
            if (PHYS == 1) {
                R uu[3], dr[2], ds[2];
                for (int var = 0; var < 2; ++var) {
                    const R *w0 = wk + ((2 * var) * G + j) * X, *w1 = wk + ((2 * var + 1) * G + j) * X;
                    R l0 = 0, l1 = 0, l2 = 0;
                    for (int n = 0; n < X; ++n) {
                        l0 += w0[n] * tb.gx[i][n];
                        l1 += w1[n] * tb.gx[i][n];
                        l2 += (w0[n] * oeta) * tb.dgx[i][n];
                    }
                    uu[var] = l0; ds[var] = l1 + xp1 * l2; dr[var] = l2;
                }
                {
                    const R *w0 = wk + (4 * G + j) * X;
                    R l0 = 0;
                    for (int n = 0; n < X; ++n) l0 += w0[n] * tb.gx[i][n];
                    uu[2] = l0;
                }
                const R rho = (R)ph.rho;
                const R fluxx = rho * uu[0], fluxy = rho * uu[1];
                const R m0 = +d11 * fluxx - d01 * fluxy;
                const R m1 = -d10 * fluxx + d00 * fluxy;
                R c00, c01, c10, c11, uf0 = uu[0], uf1 = uu[1], qt;
                if (diff) {
                    R ub[2];
                    for (int var = 0; var < 2; ++var) {
                        const R *w0 = wk + ((5 + var) * G + j) * X;
                        R l0 = 0;
                        for (int n = 0; n < X; ++n) l0 += w0[n] * tb.gx[i][n];
                        ub[var] = l0;
                    }
                    const R mb0 = +d11 * (rho * ub[0]) - d01 * (rho * ub[1]);
                    const R mb1 = -d10 * (rho * ub[0]) + d00 * (rho * ub[1]);
                    uf0 = ub[0] + uu[0];
                    uf1 = ub[1] + uu[1];
                    c00 = uf0 * m0 + uu[0] * mb0;
                    c01 = uf0 * m1 + uu[0] * mb1;
                    c10 = uf1 * m0 + uu[1] * mb0;
                    c11 = uf1 * m1 + uu[1] * mb1;
                    qt = ub[0] * ub[0] + ub[1] * ub[1];
                } else {
                    c00 = uu[0] * m0; c01 = uu[0] * m1; c10 = uu[1] * m0; c11 = uu[1] * m1;
                    qt = uu[0] * uu[0] + uu[1] * uu[1];
                }
                c00 += d11 * uu[2];
                c01 -= d10 * uu[2];
                c10 -= d01 * uu[2];
                c11 += d00 * uu[2];
                PT(0)[w] = c00; PT(1)[w] = c01; PT(2)[w] = c10; PT(3)[w] = c11;
                PT(4)[w] = m0; PT(5)[w] = m1;
                if (beta > (R)0) {
                    const R cjcb = d00 * d11 - d10 * d01;
                    const R cjcbi = (R)ph.mu / cjcb;
                    const R v0000 = -cjcbi * ((R)2. * d11 * d11 + d01 * d01);
                    const R v0011 = -cjcbi * ((R)2. * d10 * d10 + d00 * d00);
                    const R v0001 = cjcbi * ((R)2. * d11 * d10 + d01 * d00);
                    const R v1100 = -cjcbi * (d11 * d11 + (R)2. * d01 * d01);
                    const R v1111 = -cjcbi * (d10 * d10 + (R)2. * d00 * d00);
                    const R v1101 = cjcbi * (d11 * d10 + (R)2. * d01 * d00);
                    const R v0100 = cjcbi * d01 * d11;
                    const R v0111 = cjcbi * d00 * d10;
                    const R v0101 = -cjcbi * d01 * d10;
                    const R v0110 = -cjcbi * d00 * d11;
                    const R f00 = (v0000 * dr[0] + v0100 * dr[1] + v0001 * ds[0] + v0101 * ds[1]);
                    const R f01 = (v0001 * dr[0] + v0110 * dr[1] + v0011 * ds[0] + v0111 * ds[1]);
                    const R f10 = (v0100 * dr[0] + v1100 * dr[1] + v0110 * ds[0] + v1101 * ds[1]);
                    const R f11 = (v0101 * dr[0] + v1101 * dr[1] + v0111 * ds[0] + v1111 * ds[1]);
                    PT(6)[w] = c00 + f00; PT(7)[w] = c01 + f01; PT(8)[w] = c10 + f10; PT(9)[w] = c11 + f11;
                    PT(10)[w] = f00; PT(11)[w] = f01; PT(12)[w] = f10; PT(13)[w] = f11;
                    PT(14)[w] = uf0; PT(15)[w] = uf1;
                    PT(19)[w] = qt;
                }
            } else {
                const R *w0 = wk + (0 * G + j) * X, *w1 = wk + (1 * G + j) * X;
                R l0 = 0, l1 = 0, l2 = 0;
                for (int n = 0; n < X; ++n) {
                    l0 += w0[n] * tb.gx[i][n];
                    l1 += w1[n] * tb.gx[i][n];
                    l2 += (w0[n] * oeta) * tb.dgx[i][n];
                }
                const R u = l0, ds = l1 + xp1 * l2, dr = l2;
                const R fluxx = (R)ph.rhocv * (R)ph.ax * u, fluxy = (R)ph.rhocv * (R)ph.ay * u;
                const R c00 = +d11 * fluxx - d01 * fluxy;
                const R c01 = -d10 * fluxx + d00 * fluxy;
                PT(0)[w] = c00; PT(1)[w] = c01;
                if (beta > (R)0) {
                    const R cj = d00 * d11 - d10 * d01;
                    const R kc = (R)ph.kcond / cj;
                    const R v00 = -kc * (d11 * d11 + d01 * d01);
                    const R v11 = -kc * (d10 * d10 + d00 * d00);
                    const R v01 = kc * (d11 * d10 + d01 * d00);
                    const R e00 = v00 * dr + v01 * ds, e01 = v01 * dr + v11 * ds;
                    PT(2)[w] = c00 + e00; PT(3)[w] = c01 + e01;
                    PT(4)[w] = e00; PT(5)[w] = e01;
                    PT(6)[w] = u;
                }
            }
        }
        __syncwarp();
        // ---- intgrtrs of the imaginary fluxes (intgrt.cpp:81-158) -> res (and res.i)
        // pair k: ins (cv0x,cv0y)=slots(0,1), (cv1x,cv1y)=(2,3), (mx,my)=(4,5); cd (0,1)
        auto intgrtrs_stageI = [&](int sx0) {
            for (int w = sl; act && w < C::NPAIR * X * G; w += LW) {
                const int k = w / (X * G), r = w - k * (X * G), n = r / G, j = r - n * G;
                const R *dx = PT(sx0 + 2 * k), *dy = PT(sx0 + 2 * k + 1);
                R l0 = 0, l1 = 0;
                for (int i = 0; i < G; ++i) {
                    const R w2 = dx[i * G + j] + dy[i * G + j] * tb.x0[i];
                    l0 += w2 * tb.dgxwtx[n][i];
                    l1 += dy[i * G + j] * tb.gxwtx[n][i];
                }
                wk[((2 * k) * X + n) * G + j] = l0;
                wk[((2 * k + 1) * X + n) * G + j] = l1;
            }
        };
        auto mode_result = [&](int k, int m) -> R {
            const int col = tb.colof[m];
            const R *w0 = wk + ((2 * k) * X + col) * G, *w1 = wk + ((2 * k + 1) * X + col) * G;
            R l0 = 0;
            for (int j = 0; j < G; ++j) l0 -= tb.gnwtnn0[m][j] * w0[j] + tb.dgnwtn[m][j] * w1[j];
            return l0;
        };
        // scatter of one local coefficient of variable n, mode m (lftog, gtol.cpp:364-402)
        auto scatter = [&](R *gv, R *gs, R *el, int n, int m, R val) {
            if (el) {
                int vp = 0, sp = 0;
                if (m >= 3) {
                    const int i = (m - 3) / SM, k = (m - 3) - i * SM;
                    if ((k & 1) && mesh.tri_sgn[3 * tind + i] < 0) val = -val;
                    sp = mesh.spos[3 * tind + i];
                } else {
                    vp = mesh.vpos[3 * tind + m];
                }
                el[asm_slot(mesh, NV, SM, vp, sp, m, n)] = val;
            } else if (m < 3) {
                const int v = (m == 0 ? p0 : (m == 1 ? p1 : p2));
                atomic_add(&gv[v * NV + n], val);
            } else {
                const int i = (m - 3) / SM, k = (m - 3) - i * SM;
                const int sind = mesh.tri_seg[3 * tind + i], sg = mesh.tri_sgn[3 * tind + i];
                if ((k & 1) && sg < 0) val = -val;
                atomic_add(&gs[(sind * SM + k) * NV + n], val);
            }
        };
        intgrtrs_stageI(0);
        __syncwarp();
        // the cd source enters only the uht = 0 column of the build
        const R srcv = (bmode && bcol < T) ? (R)0 : (R)ph.src;
        for (int w = sl; act && w < NV * T; w += LW) {
            const int n = w / T, m = w - n * T;
            const R val = mode_result(n, m);
            if (bmode) {
                if (bcol < T) build.aim[EmatCfg<P>::idx(tind, bcol, m)] = val;
            } else if (jmode) {
                uht[n * T + m] = val;  // uht is dead after stage I: lf_im collects there
            } else if (m < BM) {
                scatter(st.resv, st.ress, st.elim, n, m, val);
            } else {
                const size_t gi = ((size_t)tind * IM + (m - BM)) * NV + n;
                const R src = st.dresi ? st.dresi[gi] : (R)0;
                if (beta > (R)0) st.resi[gi] = val + src;
                else st.resi[gi] = val + st.rri[gi] * omb + src;  // res_r unchanged when beta = 0
            }
        }
        if (beta > (R)0) {
            // ---- strong residual: res = source + derivr(F_r) + derivs(F_s) (proj.cpp:339-402)
            __syncwarp();
            constexpr int SRES = (PHYS == 1 ? 16 : 7);
            for (int w = sl; act && w < NV * GG; w += LW) {
                const int n = w / GG, r = w - n * GG, i = r / G, j = r - i * G;
                int sr, ss;
                if (PHYS == 1) { sr = (n < 2 ? 6 + 2 * n : 4); ss = sr + 1; }
                else { sr = 2; ss = 3; }
                const R *fr = PT(sr), *fs = PT(ss);
                R acc;
                if (PHYS == 1) acc = (R)0;  // rhorbd0*u + dugdt with bd(0) = 0
                else {
                    R d00, d01, d10, d11;
                    metric(i, j, d00, d01, d10, d11);
                    acc = -(d00 * d11 - d10 * d01) * srcv;
                    if (CURVED) PT(8)[r] = acc;  // the source field, integrated below
                }
                const R ln0 = tb.n0[j];
                {
                    const R wi = fr[i * G + j] * tb.dltx[i] * ln0;
                    for (int q = 0; q < G; ++q)
                        if (q != i) acc += (wi + fr[q * G + j] * tb.dltx[q] * ln0) * tb.dltx1[i][q];
                }
                {
                    const R wi = fs[i * G + j] * tb.dltx[i] * ln0;
                    for (int q = 0; q < G; ++q)
                        if (q != i) acc += (wi + fs[q * G + j] * tb.dltx[q] * ln0) * tb.dltn1[i][q];
                    const R wj = fs[i * G + j] * tb.dltn[j];
                    for (int q = 0; q < G; ++q)
                        if (q != j) acc += (wj + fs[i * G + q] * tb.dltn[q]) * tb.dltn2[j][q];
                }
                PT(SRES + n)[r] = acc;
            }
            __syncwarp();
            // ---- pointwise SUPG terms
            if (PHYS == 1) {
                // inscribed radius (tri_mesh/tprims.cpp:224-241)
                const double dx1 = x0d - x2d, dy1 = y0d - y2d, dx2 = x1d - x0d, dy2 = y1d - y0d;
                const double area = dx1 * dy2 - dy1 * dx2;
                const double perim = sqrt(dx1 * dx1 + dy1 * dy1) + sqrt(dx2 * dx2 + dy2 * dy2) +
                                     sqrt((dx1 + dx2) * (dx1 + dx2) + (dy1 + dy2) * (dy1 + dy2));
                const R h = (R)((area / perim) / (0.25 * (P + 1) * (P + 1)));
                const R nu = (R)(ph.mu / ph.rho);
                for (int w = sl; act && w < GG; w += LW) {
                    R d00, d01, d10, d11;
                    metric(w / G, w - (w / G) * G, d00, d01, d10, d11);
                    const R cjcb = d00 * d11 - d10 * d01;
                    const R u0 = PT(14)[w], u1 = PT(15)[w];
                    const R q = PT(19)[w];
                    const R t2 = (R)2. * nu / h;
                    R gam = (R)3.0 * q + t2 * t2;
                    if (ph.mu + ph.bd0 == 0.0) gam = (gam > (R)0.1 ? gam : (R)0.1);
                    const R tau0 = (R)ph.adis * h / (cjcb * rsqrt_<R>(gam));
                    const R tau2 = rsqrt_<R>(q) * tau0;
                    const R tr0 = tau0 * PT(16)[w], tr1 = tau0 * PT(17)[w], tr2 = tau2 * PT(18)[w];
                    PT(10)[w] -= (d11 * ((R)2 * u0) - d01 * u1) * tr0 - d01 * u0 * tr1 + d11 * tr2;
                    PT(11)[w] -= (-d10 * ((R)2 * u0) + d00 * u1) * tr0 + d00 * u0 * tr1 - d10 * tr2;
                    PT(12)[w] -= +d11 * u1 * tr0 + (d11 * u0 - d01 * ((R)2. * u1)) * tr1 - d01 * tr2;
                    PT(13)[w] -= -d10 * u1 * tr0 + (-d10 * u0 + d00 * ((R)2. * u1)) * tr1 + d00 * tr2;
                    PT(14)[w] = -(d11 * tr0 - d01 * tr1);
                    PT(15)[w] = -(-d10 * tr0 + d00 * tr1);
                }
            } else {
                const R taue = st.tau[tind];
                const R ax = (R)ph.ax, ay = (R)ph.ay;
                for (int w = sl; act && w < GG; w += LW) {
                    R d00, d01, d10, d11;
                    metric(w / G, w - (w / G) * G, d00, d01, d10, d11);
                    const R tres = taue * PT(7)[w];
                    PT(4)[w] -= (d11 * ax - d01 * ay) * tres;
                    PT(5)[w] -= (-d10 * ax + d00 * ay) * tres;
                }
            }
            __syncwarp();
            // ---- intgrtrs of the real part -> res_r; ins pairs (10,11),(12,13),(14,15); cd (4,5)
            intgrtrs_stageI(PHYS == 1 ? 10 : 4);
            // cd source term: intgrt(res0) with res0 = -cjcb*src (constant over the element)
            __syncwarp();
            for (int w = sl; act && w < NV * T; w += LW) {
                const int n = w / T, m = w - n * T;
                R val = mode_result(n, m);
                if (PHYS == 0 && srcv != (R)0) {
                    // intgrt (intgrt.cpp:22-78) of res0 = -cjcb*src: sum_j gnwtn(m,j) sum_i
                    // res0(i,j) gxwtx(col,i); constant over a straight element
                    const R cval = -(g00 * g11 - g10 * g01) * srcv;
                    const int col = tb.colof[m];
                    R l0 = 0;
                    for (int j = 0; j < G; ++j) {
                        R s = (CURVED ? PT(8)[j] : cval) * tb.gxwtx[col][0];
                        for (int i = 1; i < G; ++i) s += (CURVED ? PT(8)[i * G + j] : cval) * tb.gxwtx[col][i];
                        l0 += tb.gnwtn[m][j] * s;
                    }
                    val = l0 + val;
                }
                val *= beta;
                if (bmode) {
                    if (bcol < T) build.are[EmatCfg<P>::idx(tind, bcol, m)] = val;
                    else build.bre[(size_t)tind * T + m] = val;
                } else if (jmode) {
                    uht[n * T + m] += val;
                } else if (m < BM) {
                    scatter(st.rrv, st.rrs, st.elre, n, m, val);
                } else {
                    const size_t gi = ((size_t)tind * IM + (m - BM)) * NV + n;
                    const R rr = st.rri[gi] * omb + val;
                    st.rri[gi] = rr;
                    st.resi[gi] += rr;
                }
            }
        }
        if (jmode) {
            __syncwarp();
            for (int w = sl; act && w < NJ; w += LW) {
                const int n = w / T, m = w - n * T;
                const size_t rb = ((size_t)tind * T + m) * NV + n;
                if (!jcols) jac.rbar[rb] = uht[n * T + m];
                else jac.K[((size_t)tind * NJ + (m * NV + n)) * NJ + jcol] = (uht[n * T + m] - jac.rbar[rb]) / jdw;
            }
        }
        __syncwarp();
    }
}

// Linear cd residual from the stored element operators: lf_im = A_im uht and
// lf_re = beta (A_re uht + b_re), with the gather, scatter, res_r mixing and dres of
// k_rsdl_elem (tri_hp/cd/rsdl.cpp:14-154 through tri_hp/nstage.cpp:21-82). Persistent
// CTAs walk tiles of EB elements. Each thread owns one operator row (A_im rows, plus the
// A_re rows when beta > 0) and at most one (element, mode) slot. The work of three tiles
// is software-pipelined across one barrier per tile: in the phase of tile k a thread
// scatters its slot of tile k-1, forms its row's dot product for tile k (the operator
// entries stream from HBM, coalesced across the CTA) and gathers its slot of tile k+1,
// so the dependent index -> value gather loads and the scatter atomics overlap the
// operator stream instead of separating it. TPP tiles (consecutive, one contiguous
// operator run) go through each phase together: TPP rows and slots per thread, more
// loads in flight per barrier, at more registers per thread (a per-level tuning choice).
// Threads of one CTA: at p <= 2 FP32 threads own two adjacent operator rows (one 8-byte
// load per column, so each request moves as many bytes as an FP64 row's; 9% faster FP32
// updates at p = 2), otherwise one row (at p = 4 and 6 the paired rows measured 3% and 11%
// slower: fewer threads to hide the gather latency, and spills at p = 6); at least one
// thread per (element, mode) slot of the tile.
template <typename R, int P, bool RE>
struct EmatShape {
    static constexpr int VW = (sizeof(R) == 4 && P <= 2) ? 2 : 1;
    static constexpr int SLOTS = EmatCfg<P>::EB * EmatCfg<P>::T;
    static constexpr int ROWS = (RE ? 2 : 1) * SLOTS;
    static constexpr int RT = ROWS / VW;  // row groups
    static constexpr int THREADS = (((RT > SLOTS ? RT : SLOTS) + 31) / 32) * 32;
};

template <typename R, int P, bool RE, int TPP>
__global__ void __launch_bounds__(EmatShape<R, P, RE>::THREADS, 2048 / EmatShape<R, P, RE>::THREADS / TPP)
    k_rsdl_emat(ElemMat<R> em, Mesh mesh, State<R> st, Phys ph, int stage, int zero_rr) {
    using E = EmatCfg<P>;
    using S = EmatShape<R, P, RE>;
    constexpr int T = E::T, EB = E::EB, TS = E::TS, BM = 3 * P, IM = (P - 1) * (P - 2) / 2;
    constexpr int SM = (P > 1 ? P - 1 : 1);  // side-mode stride (unused when p = 1)
    constexpr int NH = RE ? 2 : 1;
    constexpr int ROWS = NH * EB * T, SLOTS = EB * T, VW = S::VW, RT = S::RT;
    static_assert(SLOTS % 2 == 0, "row pairs must not straddle the A_im / A_re halves");
    __shared__ R su[2][TPP * SLOTS];
    __shared__ R sr[2][TPP * ROWS];
    const R beta = (R)ph.beta[stage];
    const R omb = zero_rr ? (R)0 : (R)1 - beta;
    const bool src = RE && ph.src != 0.0;
    const long ntiles = ((long)mesh.ntri + EB - 1) / EB;
    const long step = gridDim.x;
    const int w = threadIdx.x;
    const int r0 = w * VW, hr = r0 / SLOTS, qr = r0 - hr * SLOTS, er = qr / T;  // first operator row (w < RT)
    const int es = w / T, ms = w - es * T;                       // gather / scatter slot (w < SLOTS)
    auto gather = [&](long tile) -> R {
        const long t = tile * EB + es;
        R val = (R)0;
        if (w < SLOTS && t < mesh.ntri) {
            if (ms < 3) {
                val = st.ugv[mesh.tri_pnt[3 * t + ms]];
            } else if (ms < BM) {
                const int i = (ms - 3) / SM, kk = (ms - 3) - i * SM;
                val = st.ugs[mesh.tri_seg[3 * t + i] * SM + kk];
                if ((kk & 1) && mesh.tri_sgn[3 * t + i] < 0) val = -val;
            } else {
                val = st.ugi[t * IM + (ms - BM)];
            }
        }
        return val;
    };
    auto matvec = [&](long tile, const R *u_s, R *r_s) {
        if (w >= RT || tile * EB + er >= mesh.ntri) return;
        const R *a = (hr ? em.are : em.aim) + (size_t)tile * TS + qr;
        if constexpr (VW == 1) {
            const R *u = u_s + er * T;
            R acc = (R)0;
#pragma unroll
            for (int j = 0; j < T; ++j) acc = fma(__ldg(a + (size_t)j * SLOTS), u[j], acc);
            if (hr) {
                if (src) acc += __ldg(em.bre + (size_t)tile * EB * T + qr);
                acc *= beta;
            }
            r_s[w] = acc;
        } else {
            // rows qr, qr+1 of every column: one aligned 8-byte load (tile stride and
            // column length are even); the two rows may belong to consecutive elements
            const float2 *a2 = reinterpret_cast<const float2 *>(a);
            const R *u0 = u_s + er * T, *u1 = u_s + ((qr + 1) / T) * T;
            R acc0 = (R)0, acc1 = (R)0;
#pragma unroll
            for (int j = 0; j < T; ++j) {
                const float2 x = __ldg(a2 + (size_t)j * (SLOTS / 2));
                acc0 = fmaf(x.x, u0[j], acc0);
                acc1 = fmaf(x.y, u1[j], acc1);
            }
            const bool row1 = tile * EB + (qr + 1) / T < mesh.ntri;  // b_re holds ntri * T entries
            if (hr) {
                if (src) {
                    acc0 += __ldg(em.bre + (size_t)tile * EB * T + qr);
                    if (row1) acc1 += __ldg(em.bre + (size_t)tile * EB * T + qr + 1);
                }
                acc0 *= beta;
                acc1 *= beta;
            }
            r_s[r0] = acc0;
            if (row1) r_s[r0 + 1] = acc1;
        }
    };
    auto scatter = [&](long tile, const R *r_s) {
        if (w >= SLOTS) return;
        const long t = tile * EB + es;
        if (t >= mesh.ntri) return;
        const R vim = r_s[w];
        const R vre = RE ? r_s[SLOTS + w] : (R)0;
        if (st.elim && ms < BM) {  // assembly by gather (NV = 1)
            bool flip = false;
            int vp = 0, sp = 0;
            if (ms >= 3) {
                const int i = (ms - 3) / SM, kk = (ms - 3) - i * SM;
                flip = (kk & 1) && mesh.tri_sgn[3 * t + i] < 0;
                sp = mesh.spos[3 * t + i];
            } else {
                vp = mesh.vpos[3 * t + ms];
            }
            const size_t slot = asm_slot(mesh, 1, SM, vp, sp, ms, 0);
            st.elim[slot] = flip ? -vim : vim;
            if (RE) st.elre[slot] = flip ? -vre : vre;
        } else if (ms < 3) {
            const int v = mesh.tri_pnt[3 * t + ms];
            atomic_add(&st.resv[v], vim);
            if (RE) atomic_add(&st.rrv[v], vre);
        } else if (ms < BM) {
            const int i = (ms - 3) / SM, kk = (ms - 3) - i * SM;
            const int g = mesh.tri_seg[3 * t + i] * SM + kk;
            const bool flip = (kk & 1) && mesh.tri_sgn[3 * t + i] < 0;
            atomic_add(&st.ress[g], flip ? -vim : vim);
            if (RE) atomic_add(&st.rrs[g], flip ? -vre : vre);
        } else {
            const size_t gi = (size_t)t * IM + (ms - BM);
            const R d = st.dresi ? st.dresi[gi] : (R)0;
            if (RE) {
                const R rr = st.rri[gi] * omb + vre;
                st.rri[gi] = rr;
                st.resi[gi] = vim + d + rr;
            } else {
                st.resi[gi] = vim + st.rri[gi] * omb + d;  // res_r unchanged when beta = 0
            }
        }
    };
    const long ngroups = (ntiles + TPP - 1) / TPP;
    long grp = blockIdx.x;
    if (grp >= ngroups) return;
#pragma unroll
    for (int i = 0; i < TPP; ++i)
        if (w < SLOTS) su[0][i * SLOTS + w] = gather(grp * TPP + i);
    __syncthreads();
    int k = 0;
    for (; grp < ngroups; grp += step, ++k) {
        const int b = k & 1;
        // the next group's gather loads are issued first and stored last, so their
        // index -> value latency runs under the scatter and the operator stream
        R g[TPP];
        const bool more = grp + step < ngroups;
#pragma unroll
        for (int i = 0; i < TPP; ++i) g[i] = more ? gather((grp + step) * TPP + i) : (R)0;
        if (k > 0) {
#pragma unroll
            for (int i = 0; i < TPP; ++i) scatter((grp - step) * TPP + i, sr[b ^ 1] + i * ROWS);
        }
#pragma unroll
        for (int i = 0; i < TPP; ++i) matvec(grp * TPP + i, su[b] + i * SLOTS, sr[b] + i * ROWS);
        if (w < SLOTS) {
#pragma unroll
            for (int i = 0; i < TPP; ++i) su[b ^ 1][i * SLOTS + w] = g[i];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TPP; ++i) scatter((grp - step) * TPP + i, sr[(k - 1) & 1] + i * ROWS);
}

// res.v = res.s = 0 ; res_r.{v,s} *= (1-beta) (or = 0) : nstage.cpp:21-49
template <typename R>
__global__ void k_rsdl_pre(int nv_len, int ns_len, R *resv, R *ress, R *rrv, R *rrs, R omb, int zero_rr) {
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nv_len + ns_len; k += stride) {
        if (k < nv_len) {
            resv[k] = (R)0;
            rrv[k] = zero_rr ? (R)0 : rrv[k] * omb;
        } else {
            const int q = k - nv_len;
            ress[q] = (R)0;
            rrs[q] = zero_rr ? (R)0 : rrs[q] * omb;
        }
    }
}

// Boundary-edge flux of bdry_ins::generic (hp_boundary.cpp:973-1049, ins/bdry_ins.h:35-50).
// One thread per boundary edge.
template <typename R, int P>
__global__ void k_bdry_flux_ins(const DevTables<R, P> *__restrict__ tb, Mesh mesh, State<R> st, Phys ph, int diff) {
    constexpr int G = P + 1, X = P + 2, SM = P - 1, NV = 3;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= mesh.nbseg) return;
    if ((mesh.bkind[e] & (0xF << 8)) != (1 << 8)) return;
    const int sind = mesh.bseg[e];
    const int v0 = mesh.seg_pnt[2 * sind], v1 = mesh.seg_pnt[2 * sind + 1];
    R lin[NV][SM + 2], linb[2][SM + 2];
    for (int n = 0; n < NV; ++n) {
        lin[n][0] = st.ugv[v0 * NV + n];
        lin[n][1] = st.ugv[v1 * NV + n];
        for (int m = 0; m < SM; ++m) lin[n][m + 2] = st.ugs[(sind * SM + m) * NV + n];
    }
    for (int n = 0; n < 2; ++n) {
        linb[n][0] = diff ? st.ubv[v0 * NV + n] : (R)0;
        linb[n][1] = diff ? st.ubv[v1 * NV + n] : (R)0;
        for (int m = 0; m < SM; ++m) linb[n][m + 2] = diff ? st.ubs[(sind * SM + m) * NV + n] : (R)0;
    }
    const R xa = (R)mesh.pnts[2 * v0], ya = (R)mesh.pnts[2 * v0 + 1];
    const R xb = (R)mesh.pnts[2 * v1], yb = (R)mesh.pnts[2 * v1 + 1];
    R acc[NV][X - 1];
    for (int n = 0; n < NV; ++n)
        for (int m = 0; m < X - 1; ++m) acc[n][m] = 0;
    for (int k = 0; k < G; ++k) {
        // proj1d of the side coordinates: derivative only
        R dx = xa * tb->dgx[k][1] + xb * tb->dgx[k][2];
        R dy = ya * tb->dgx[k][1] + yb * tb->dgx[k][2];
        if (mesh.bcrd) {  // curved side: its position modes (crdtocht1d)
            for (int m = 0; m < SM; ++m) {
                dx += (R)mesh.bcrd[((size_t)e * SM + m) * 2] * tb->dgx[k][m + 3];
                dy += (R)mesh.bcrd[((size_t)e * SM + m) * 2 + 1] * tb->dgx[k][m + 3];
            }
        }
        R nrm0 = dy, nrm1 = -dx;
        const R jcb = rsqrt_<R>(nrm0 * nrm0 + nrm1 * nrm1);
        nrm0 /= jcb; nrm1 /= jcb;
        R u[NV];
        for (int n = 0; n < NV; ++n) {
            R l0 = lin[n][0] * tb->gx[k][1] + lin[n][1] * tb->gx[k][2];
            for (int m = 2; m < SM + 2; ++m) l0 += lin[n][m] * tb->gx[k][m + 1];
            u[n] = l0;
        }
        R flx[NV];
        flx[2] = (R)ph.rho * (u[0] * nrm0 + u[1] * nrm1);
        if (diff) {
            // F(b+d) - F(b) = rho (d.n)(b+d) + rho (b.n) d ; the boundary pressure cancels
            R ub[2];
            for (int n = 0; n < 2; ++n) {
                R l0 = linb[n][0] * tb->gx[k][1] + linb[n][1] * tb->gx[k][2];
                for (int m = 2; m < SM + 2; ++m) l0 += linb[n][m] * tb->gx[k][m + 1];
                ub[n] = l0;
            }
            const R mb = (R)ph.rho * (ub[0] * nrm0 + ub[1] * nrm1);
            flx[0] = flx[2] * (ub[0] + u[0]) + mb * u[0];
            flx[1] = flx[2] * (ub[1] + u[1]) + mb * u[1];
        } else {
            const R pb = (R)mesh.bpibc[e * G + k];
            flx[0] = flx[2] * u[0] + pb * nrm0;
            flx[1] = flx[2] * u[1] + pb * nrm1;
        }
        for (int n = 0; n < NV; ++n) {
            const R r = flx[n] * jcb;
            acc[n][0] += tb->gxwtx[1][k] * r;
            acc[n][1] += tb->gxwtx[2][k] * r;
            for (int m = 3; m < X; ++m) acc[n][m - 1] += tb->gxwtx[m][k] * r;
        }
    }
    if (st.bres) {  // assembly by gather: k_assemble adds them
        for (int n = 0; n < NV; ++n)
            for (int m = 0; m < SM + 2; ++m) st.bres[((size_t)e * (SM + 2) + m) * NV + n] = acc[n][m];
        return;
    }
    for (int n = 0; n < NV; ++n) {
        atomic_add(&st.resv[v0 * NV + n], acc[n][0]);
        atomic_add(&st.resv[v1 * NV + n], acc[n][1]);
        for (int m = 0; m < SM; ++m) atomic_add(&st.ress[(sind * SM + m) * NV + n], acc[n][m + 2]);
    }
}

// Assembly by gather of rsdl(stage)'s vertex and side residuals (lftog, gtol.cpp:364-402,
// summed per entity instead of scattered): res = sum of the elements' imaginary parts
// (+ the boundary fluxes, hp_edge_bdry::rsdl), res_r = (1 - beta) res_r + sum of their
// real parts (nstage.cpp:21-49; zero_rr: res_r = sum). A vertex sums its triangles in
// vertex-incidence order, a side its two triangles in seg.tri order, so the result does
// not depend on the scheduling. One thread per vertex, then one per (side, mode).
template <typename R>
__global__ void k_assemble(Mesh mesh, State<R> st, int NV, int SM, R omb, int zero_rr, int with_re, int with_b) {
    const size_t soff = (size_t)3 * mesh.ntri * NV;  // side section of the buffers
    const long nitems = (long)mesh.npnt + (long)mesh.nseg * SM;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nitems; k += (long)gridDim.x * blockDim.x) {
        if (k < mesh.npnt) {
            const int v = (int)k, j0 = mesh.vt_ptr[v], j1 = mesh.vt_ptr[v + 1];
            for (int n = 0; n < NV; ++n) {
                R sim = (R)0, sre = (R)0;
                for (int j = j0; j < j1; ++j) {  // contiguous: the buffers are in incidence order
                    sim += st.elim[(size_t)j * NV + n];
                    if (with_re) sre += st.elre[(size_t)j * NV + n];
                }
                if (with_b)
                    for (int q = 0; q < 2; ++q) {
                        const int b = mesh.vb_idx[2 * v + q];
                        if (b >= 0 && (mesh.bkind[b >> 1] & (0xF << 8)) == (1 << 8))
                            sim += st.bres[((size_t)(b >> 1) * (SM + 2) + (b & 1)) * NV + n];
                    }
                st.resv[v * NV + n] = sim;
                const R r0 = zero_rr ? (R)0 : st.rrv[v * NV + n] * omb;
                st.rrv[v * NV + n] = with_re ? r0 + sre : r0;
            }
        } else {
            const long q = k - mesh.npnt;
            const int sd = (int)(q / SM), kk = (int)(q - (long)sd * SM);
            const int e = with_b ? mesh.seg_bdry[sd] : -1;
            const bool bf = e >= 0 && (mesh.bkind[e] & (0xF << 8)) == (1 << 8);
            for (int n = 0; n < NV; ++n) {
                R sim = (R)0, sre = (R)0;
                for (int side = 0; side < 2; ++side) {
                    if (mesh.seg_tri[2 * sd + side] < 0) continue;
                    const size_t idx = soff + ((size_t)(2 * sd + side) * SM + kk) * NV + n;
                    sim += st.elim[idx];
                    if (with_re) sre += st.elre[idx];
                }
                if (bf) sim += st.bres[((size_t)e * (SM + 2) + 2 + kk) * NV + n];
                const size_t g = ((size_t)sd * SM + kk) * NV + n;
                st.ress[g] = sim;
                const R r0 = zero_rr ? (R)0 : st.rrs[g] * omb;
                st.rrs[g] = with_re ? r0 + sre : r0;
            }
        }
    }
}

// Preconditioner assembly by gather with the inversion of tri_hp::setup_preconditioner
// (setup_preconditioner.cpp:68-76): vprcn = 1 / (vdiag sum of the vertex's triangles'
// tprcn), sprcn = 1 / (sum over the side's triangles), in a fixed order.
template <typename R>
__global__ void k_prcn_gather(Mesh mesh, State<R> st, int NV, int with_s, R vdiag) {
    const long nitems = (long)mesh.npnt + (with_s ? (long)mesh.nseg : 0);
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nitems; k += (long)gridDim.x * blockDim.x) {
        if (k < mesh.npnt) {
            const int v = (int)k;
            for (int n = 0; n < NV; ++n) {
                R sum = (R)0;
                for (int j = mesh.vt_ptr[v]; j < mesh.vt_ptr[v + 1]; ++j) sum += st.tprcn[(mesh.vt_idx[j] >> 2) * NV + n];
                st.vprcn[v * NV + n] = (R)1.0 / (vdiag * sum);
            }
        } else {
            const int sd = (int)(k - mesh.npnt);
            for (int n = 0; n < NV; ++n) {
                R sum = (R)0;
                for (int side = 0; side < 2; ++side) {
                    const int t = mesh.seg_tri[2 * sd + side];
                    if (t >= 0) sum += st.tprcn[t * NV + n];
                }
                st.sprcn[sd * NV + n] = (R)1.0 / sum;
            }
        }
    }
}

// Order-preserving key of a non-negative floating value (for atomicMax).
__device__ __forceinline__ unsigned long long ord_key(double v) { return (unsigned long long)__double_as_longlong(v); }
__device__ __forceinline__ unsigned long long ord_key(float v) { return (unsigned long long)__double_as_longlong((double)v); }

// ---------------------------------------------------------------------------
// minvrt (setup_preconditioner.cpp:102-373) fused with the stage update
// (nstage.cpp:387-409).
// ---------------------------------------------------------------------------
// Vertex phase: assemble res.v + res_r.v, remove side and interior parts, apply
// the vertex preconditioner and Dirichlet zeroing, update ug.v, maxres.
template <typename R, int NV>
__global__ void k_minv_vert(Mesh mesh, State<R> st, const DevMinv<R> *__restrict__ mt, int sm, int im, R cflalpha,
                            int do_update, int fold, unsigned long long *maxres_slot) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    R r[NV];
    bool active = v < mesh.npnt;
    if (active) {
        for (int n = 0; n < NV; ++n)
            r[n] = st.resv[v * NV + n] + (fold ? st.rrv[v * NV + n] : (R)0) + (st.dresv ? st.dresv[v * NV + n] : (R)0);
        for (int q = mesh.vs_ptr[v]; q < mesh.vs_ptr[v + 1]; ++q) {
            const int code = mesh.vs_idx[q], s = code >> 1, end = code & 1;
            for (int k = 0; k < sm; ++k) {
                const R f = mt->sfmv[end][k];
                for (int n = 0; n < NV; ++n) {
                    const int gi = (s * sm + k) * NV + n;
                    r[n] -= f * (st.ress[gi] + (fold ? st.rrs[gi] : (R)0) + (st.dress ? st.dress[gi] : (R)0));
                }
            }
        }
        if (im > 0)
            for (int q = mesh.vt_ptr[v]; q < mesh.vt_ptr[v + 1]; ++q) {
                const int code = mesh.vt_idx[q], t = code >> 2, i = code & 3;
                for (int k = 0; k < im; ++k) {
                    const R f = mt->ifmb[i][k];
                    for (int n = 0; n < NV; ++n) r[n] -= f * st.resi[((size_t)t * im + k) * NV + n];
                }
            }
        const int ess = mesh.vess[v];
        for (int n = 0; n < NV; ++n) {
            r[n] *= st.vprcn[v * NV + n];
            if (ess & (1 << n)) r[n] = (R)0;
            st.resv[v * NV + n] = r[n];
            if (do_update) st.ugv[v * NV + n] = st.u0v[v * NV + n] - cflalpha * r[n];
        }
    }
    if (maxres_slot) {
        for (int n = 0; n < NV; ++n) {
            R a = active ? fabs(r[n]) : (R)0;
            for (int o = 16; o > 0; o >>= 1) {
                R b = __shfl_xor_sync(0xffffffffu, a, o);
                a = a > b ? a : b;
            }
            if ((threadIdx.x & 31) == 0) atomicMax(&maxres_slot[n], ord_key(a));
        }
    }
}

// The vertex phase with LPV lanes per vertex (p >= 2): the lanes split the vertex's
// (side, mode) and (triangle, interior mode) removal terms, each reading NV consecutive
// values, and sum them by shuffles in a fixed order, so that a vertex's gather is spread over
// a lane group instead of one thread's sequential loop. Same result as k_minv_vert up to the
// order of the removal sums.
template <typename R, int NV, int SM, int IM, int LPV>
__global__ void k_minv_vert_coop(Mesh mesh, State<R> st, const DevMinv<R> *__restrict__ mt, R cflalpha, int do_update,
                                 int fold, unsigned long long *maxres_slot) {
    static_assert(32 % LPV == 0, "lane groups within a warp");
    constexpr int S1 = SM > 0 ? SM : 1, I1 = IM > 0 ? IM : 1;
    __shared__ R s_sfmv[2][S1], s_ifmb[3][I1];  // the tables, staged per block
    for (int x = threadIdx.x; x < 2 * S1; x += blockDim.x) s_sfmv[x / S1][x % S1] = SM > 0 ? mt->sfmv[x / S1][x % S1] : (R)0;
    for (int x = threadIdx.x; x < 3 * I1; x += blockDim.x) s_ifmb[x / I1][x % I1] = IM > 0 ? mt->ifmb[x / I1][x % I1] : (R)0;
    __syncthreads();
    const int sub = threadIdx.x % LPV;
    const long gv = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LPV;
    const bool active = gv < mesh.npnt;
    const int v = active ? (int)gv : 0;
    R acc[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) acc[n] = (R)0;
    if (active) {
        if constexpr (SM > 0) {
            const int q0 = mesh.vs_ptr[v], ns = (mesh.vs_ptr[v + 1] - q0) * SM;
            for (int w = sub; w < ns; w += LPV) {
                const int j = w / SM, k = w - j * SM;
                const int code = mesh.vs_idx[q0 + j], sd = code >> 1, end = code & 1;
                const R f = s_sfmv[end][k];
                const size_t gi = ((size_t)sd * SM + k) * NV;
#pragma unroll
                for (int n = 0; n < NV; ++n)
                    acc[n] += f * (st.ress[gi + n] + (fold ? st.rrs[gi + n] : (R)0) +
                                   (st.dress ? st.dress[gi + n] : (R)0));
            }
        }
        if constexpr (IM > 0) {
            const int q0 = mesh.vt_ptr[v], ni = (mesh.vt_ptr[v + 1] - q0) * IM;
            for (int w = sub; w < ni; w += LPV) {
                const int j = w / IM, k = w - j * IM;
                const int code = mesh.vt_idx[q0 + j], t = code >> 2, i = code & 3;
                const R f = s_ifmb[i][k];
                const size_t gi = ((size_t)t * IM + k) * NV;
#pragma unroll
                for (int n = 0; n < NV; ++n) acc[n] += f * st.resi[gi + n];
            }
        }
    }
#pragma unroll
    for (int o = LPV / 2; o > 0; o >>= 1)
#pragma unroll
        for (int n = 0; n < NV; ++n) acc[n] += __shfl_xor_sync(0xffffffffu, acc[n], o, LPV);
    R r[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) r[n] = (R)0;
    if (active && sub == 0) {
        const int ess = mesh.vess[v];
#pragma unroll
        for (int n = 0; n < NV; ++n) {
            R x = st.resv[v * NV + n] + (fold ? st.rrv[v * NV + n] : (R)0) + (st.dresv ? st.dresv[v * NV + n] : (R)0);
            x = (x - acc[n]) * st.vprcn[v * NV + n];
            if (ess & (1 << n)) x = (R)0;
            st.resv[v * NV + n] = x;
            if (do_update) st.ugv[v * NV + n] = st.u0v[v * NV + n] - cflalpha * x;
            r[n] = x;
        }
    }
    if (maxres_slot) {
#pragma unroll
        for (int n = 0; n < NV; ++n) {
            R a = fabs(r[n]);
            for (int o = 16; o > 0; o >>= 1) {
                R b = __shfl_xor_sync(0xffffffffu, a, o);
                a = a > b ? a : b;
            }
            if ((threadIdx.x & 31) == 0) atomicMax(&maxres_slot[n], ord_key(a));
        }
    }
}

// Side phase for mode MODE (setup_preconditioner.cpp:131-340), one thread per (side,
// variable) with its modes k >= MODE in registers. MODE 0 assembles res.s + res_r.s (+ dres)
// and removes the interior and vertex parts; MODE > 0 removes the finished mode MODE - 1 of the
// three sides of each adjacent element. Then mode MODE is finished: preconditioner, sdiag,
// Dirichlet zeroing, update of ug.s. The values a side's modes share (the triangles' interior
// modes and vertex values in mode 0, the three sides' mode MODE - 1 in the others) are read
// once per thread, and the tables come from shared memory, staged per block. Each output
// subtracts its terms in the reference's order (side by side, each side's triangles in
// seg.tri order).
template <typename R, int NV, int SM, int IM, int MODE>
__global__ void k_minv_side_vn(Mesh mesh, State<R> st, const DevMinv<R> *__restrict__ mt, R cflalpha,
                               int do_update, int fold) {
    constexpr int I1 = IM > 0 ? IM : 1, NK = SM - MODE;
    __shared__ R s_ifmb[3 * SM][I1], s_vfms[3][SM], s_sfms[SM][3], s_sdiag;
    for (int x = threadIdx.x; x < 3 * SM * I1; x += blockDim.x)
        s_ifmb[x / I1][x % I1] = IM > 0 ? mt->ifmb[3 + x / I1][x % I1] : (R)0;
    for (int x = threadIdx.x; x < 3 * SM; x += blockDim.x) {
        s_vfms[x / SM][x % SM] = mt->vfms[x / SM][x % SM];
        s_sfms[x / 3][x % 3] = MODE > 0 ? mt->sfms[MODE > 0 ? MODE - 1 : 0][x / 3][x % 3] : (R)0;
    }
    if (threadIdx.x == 0) s_sdiag = mt->sdiag[MODE];
    __syncthreads();
    const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long)mesh.nseg * NV) return;
    const int s = (int)(gid / NV), n = (int)(gid - (long)s * NV);
    const size_t g0 = (size_t)s * SM * NV + n;  // mode k at g0 + k NV
    R r[NK];
#pragma unroll
    for (int q = 0; q < NK; ++q) {
        const size_t gi = g0 + (size_t)(MODE + q) * NV;
        if constexpr (MODE == 0)
            r[q] = st.ress[gi] + (fold ? st.rrs[gi] : (R)0) + (st.dress ? st.dress[gi] : (R)0);
        else
            r[q] = st.ress[gi];
    }
    for (int side = 0; side < 2; ++side) {
        const int t = mesh.seg_tri[2 * s + side];
        if (t < 0) continue;
        const int i = mesh.seg_loc[2 * s + side];
        const bool neg = mesh.tri_sgn[3 * t + i] < 0;
        const R tp = st.tprcn[t * NV + n];
        if constexpr (MODE == 0) {
            // interior removal (setup_preconditioner.cpp:131-145)
            R ri[I1];
#pragma unroll
            for (int kk = 0; kk < IM; ++kk) ri[kk] = st.resi[((size_t)t * IM + kk) * NV + n];
            R uh[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) uh[j] = st.resv[mesh.tri_pnt[3 * t + (i + j) % 3] * NV + n] * tp;
#pragma unroll
            for (int k = 0; k < SM; ++k) {
                const R msgn = ((k & 1) && neg) ? (R)-1 : (R)1;
#pragma unroll
                for (int kk = 0; kk < IM; ++kk) {
                    const R f = msgn * s_ifmb[i * SM + k][kk];
                    r[k] -= f * ri[kk];
                }
                // vertex removal (setup_preconditioner.cpp:192-214)
#pragma unroll
                for (int j = 0; j < 3; ++j) r[k] -= msgn * s_vfms[j][k] * uh[j];
            }
        } else {
            // removal of mode-1 from higher modes (setup_preconditioner.cpp:264-284)
            constexpr int pm = MODE - 1;
            R uh[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int sidx = (i + j) % 3;
                const int sj = mesh.tri_seg[3 * t + sidx];
                const int sgj = mesh.tri_sgn[3 * t + sidx];
                const R sg = ((pm & 1) && sgj < 0) ? (R)-1 : (R)1;
                uh[j] = sg * st.ress[((size_t)sj * SM + pm) * NV + n] * tp;
            }
            R msgn = (((pm + 1) & 1) && neg) ? (R)-1 : (R)1;
#pragma unroll
            for (int q = 0; q < NK; ++q) {
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const R f = msgn * s_sfms[MODE + q][j];
                    r[q] -= f * uh[j];
                }
                if (neg) msgn = -msgn;
            }
        }
    }
    {
        R v = r[0] * (st.sprcn[s * NV + n] * s_sdiag);
        if (mesh.sess[s] & (1 << n)) v = (R)0;
        r[0] = v;
        if (do_update) st.ugs[g0 + (size_t)MODE * NV] = st.u0s[g0 + (size_t)MODE * NV] - cflalpha * v;
    }
#pragma unroll
    for (int q = 0; q < NK; ++q) st.ress[g0 + (size_t)(MODE + q) * NV] = r[q];
}

// Interior phase (setup_preconditioner.cpp:341-370, DPBTRSNU2 as written in
// utilities/myblas.c:91-120) + update of ug.i, one thread per (triangle, variable): the
// variables' banded solves and removals are independent.
template <typename R, int NV, int SM, int IM>
__global__ void k_minv_int_flat(Mesh mesh, State<R> st, const DevMinv<R> *__restrict__ mt, R cflalpha,
                                int do_update) {
    // the tables in shared memory, staged per block
    __shared__ R s_bfmi[3 + 3 * SM][IM], s_idiag[IM][2];
    for (int x = threadIdx.x; x < (3 + 3 * SM) * IM; x += blockDim.x) s_bfmi[x / IM][x % IM] = mt->bfmi[x / IM][x % IM];
    for (int x = threadIdx.x; x < 2 * IM; x += blockDim.x) s_idiag[x / 2][x % 2] = mt->idiag[x / 2][x % 2];
    __syncthreads();
    const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long)mesh.ntri * NV) return;
    const int t = (int)(gid / NV), n = (int)(gid - (long)t * NV);
    R b[IM];
#pragma unroll
    for (int k = 0; k < IM; ++k) b[k] = st.resi[((size_t)t * IM + k) * NV + n];
#pragma unroll
    for (int i = 0; i < IM; ++i) {
        if (i >= 1) b[i] -= s_idiag[i][0] * b[0];
        b[i] /= s_idiag[i][1];
    }
#pragma unroll
    for (int i = IM - 1; i >= 0; --i) {
        b[i] /= s_idiag[i][1];
        if (i >= 1) b[0] -= s_idiag[i][0] * b[i];
    }
    const R tp = st.tprcn[t * NV + n];
#pragma unroll
    for (int k = 0; k < IM; ++k) b[k] /= tp;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const R u = st.resv[mesh.tri_pnt[3 * t + i] * NV + n];
#pragma unroll
        for (int k = 0; k < IM; ++k) b[k] -= s_bfmi[i][k] * u;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int sd = mesh.tri_seg[3 * t + i], sg = mesh.tri_sgn[3 * t + i];
#pragma unroll
        for (int m = 0; m < SM; ++m) {
            const R msgn = ((m & 1) && sg < 0) ? (R)-1 : (R)1;
            const R u = msgn * st.ress[((size_t)sd * SM + m) * NV + n];
#pragma unroll
            for (int k = 0; k < IM; ++k) b[k] -= s_bfmi[3 + i * SM + m][k] * u;
        }
    }
#pragma unroll
    for (int k = 0; k < IM; ++k) {
        const size_t gi = ((size_t)t * IM + k) * NV + n;
        st.resi[gi] = b[k];
        if (do_update) st.ugi[gi] = st.u0i[gi] - cflalpha * b[k];
    }
}

// ---------------------------------------------------------------------------
// Diagonal preconditioner (ins/setup_preconditioner.cpp:9-221 REFINED_WAY,
// cd/setup_preconditioner.cpp:6-97) with tau, scatter to vprcn/sprcn.
// ---------------------------------------------------------------------------
template <typename R, int P, int PHYS>
__global__ void k_prcn_elem(const DevTables<R, P> *__restrict__ tb, Mesh mesh, State<R> st, Phys ph, int *err,
                            const float *__restrict__ lsc, int ld, float clampv) {
    constexpr int G = P + 1, X = P + 2, T = (P + 1) * (P + 2) / 2, SM = P - 1, BM = 3 * P, NV = (PHYS == 1 ? 3 : 1);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mesh.ntri) return;
    const int v[3] = {mesh.tri_pnt[3 * t], mesh.tri_pnt[3 * t + 1], mesh.tri_pnt[3 * t + 2]};
    const double px[3] = {mesh.pnts[2 * v[0]], mesh.pnts[2 * v[1]], mesh.pnts[2 * v[2]]};
    const double py[3] = {mesh.pnts[2 * v[0] + 1], mesh.pnts[2 * v[1] + 1], mesh.pnts[2 * v[2] + 1]};
    // area (tprims.cpp:66-80), 2x triangle area
    const double dx1 = px[0] - px[2], dy1 = py[0] - py[2], dx2 = px[1] - px[0], dy2 = py[1] - py[0];
    double jcb = 0.25 * (dx1 * dy2 - dy1 * dx2);
    double hmax = 0.0;
    for (int j = 0; j < 3; ++j) {
        const double ex = px[j] - px[(j + 1) % 3], ey = py[j] - py[(j + 1) % 3];
        const double h = ex * ex + ey * ey;
        hmax = (h > hmax ? h : hmax);
    }
    const double p1 = 0.25 * (P + 1) * (P + 1);
    double tp[3];
    if (PHYS == 0) {
        hmax = sqrt(hmax);
        if (!(jcb > 0.0)) { atomicAdd(err, 1); return; }
        const double h = 4. * jcb / (p1 * hmax);
        const double q = sqrt(ph.ax * ph.ax + ph.ay * ph.ay);
        const double alpha = ph.kcond / ph.rhocv;
        const double lam1 = (q + 1.5 * alpha / h + h * ph.bd0);
        st.tau[t] = (R)(ph.adis * h / (jcb * lam1));
        jcb *= ph.rhocv * lam1 / h;
        tp[0] = jcb;
    } else {
        // u, v at Gauss points (values only): proj.cpp:121-186 on the element's modes
        double lin[2][T];
        for (int n = 0; n < 2; ++n) {
            for (int i = 0; i < 3; ++i) lin[n][i] = (double)st.ugv[v[i] * NV + n];
            for (int i = 0; i < 3; ++i) {
                const int sd = mesh.tri_seg[3 * t + i], sg = mesh.tri_sgn[3 * t + i];
                for (int k = 0; k < SM; ++k) {
                    double val = (double)st.ugs[(sd * SM + k) * NV + n];
                    if ((k & 1) && sg < 0) val = -val;
                    lin[n][3 + i * SM + k] = val;
                }
            }
            for (int k = 0; k < T - BM; ++k) lin[n][BM + k] = (double)st.ugi[((size_t)t * (T - BM) + k) * NV + n];
        }
        double qmax = 0.0;
        for (int j = 0; j < G; ++j) {
            double wk[2][X];
            for (int n = 0; n < 2; ++n)
                for (int c = 0; c < X; ++c) {
                    double acc = 0.0;
                    for (int q = tb->colstart[c]; q < tb->colstart[c + 1]; ++q) {
                        const int m = tb->colmodes[q];
                        acc += lin[n][m] * (double)tb->gn[j][m];
                    }
                    wk[n][c] = acc;
                }
            for (int i = 0; i < G; ++i) {
                double u0 = 0.0, u1 = 0.0;
                for (int c = 0; c < X; ++c) {
                    u0 += wk[0][c] * (double)tb->gx[i][c];
                    u1 += wk[1][c] * (double)tb->gx[i][c];
                }
                const double q = u0 * u0 + u1 * u1;
                qmax = (q > qmax ? q : qmax);
            }
        }
        double h;
        const int cvi = mesh.tri_cv ? mesh.tri_cv[t] : -1;
        if (cvi >= 0) {
            // curved element (setup_preconditioner.cpp:45-87): smallest point Jacobian and
            // longest side tangent over the quadrature points
            const double *cht = mesh.crv_cht + (size_t)cvi * 2 * BM;
            double jcbmin = jcb, hm = 0.0;
            for (int i = 0; i < G; ++i)
                for (int j = 0; j < G; ++j) {
                    R a, b, c, d;
                    curved_metrics<R, P>(*tb, cht, i, j, a, b, c, d);
                    const double d00 = a, d01 = b, d10 = c, d11 = d;
                    jcbmin = fmin(jcbmin, d00 * d11 - d10 * d01);
                    hm = fmax(hm, d00 * d00 + d10 * d10);
                    hm = fmax(hm, d01 * d01 + d11 * d11);
                    hm = fmax(hm, (d01 - d00) * (d01 - d00) + (d11 - d10) * (d11 - d10));
                }
            hmax = 2. * sqrt(hm);
            h = 4. * jcbmin / (p1 * hmax);
            hmax = hmax / p1;
        } else {
            hmax = sqrt(hmax);
            h = 4. * jcb / (p1 * hmax);
            hmax = hmax / p1;
        }
        if (!(h > 0.0) || isnan(qmax)) { atomicAdd(err, 1); return; }
        const double nu = ph.mu / ph.rho;
        double gam = 3.0 * qmax + (0.5 * hmax * ph.bd0 + 2. * nu / hmax) * (0.5 * hmax * ph.bd0 + 2. * nu / hmax);
        if (ph.mu + ph.bd0 == 0.0) gam = (gam > 0.1 ? gam : 0.1);
        const double q = sqrt(qmax);
        const double lam1 = q + sqrt(qmax + gam);
        const double tau0 = ph.adis * h / (jcb * sqrt(gam));
        st.tau[t * NV + 0] = (R)tau0;
        st.tau[t * NV + 1] = (R)0;
        st.tau[t * NV + 2] = (R)(qmax * tau0);
        jcb *= 2. * nu * (1. / (hmax * hmax) + 1. / (h * h)) + 3 * lam1 / h;
        tp[0] = ph.rho * jcb;
        tp[1] = ph.rho * jcb;
        tp[2] = jcb / gam;
    }
    if (lsc) {  // learned per-element correction (include/hp_mlp.h)
        for (int n = 0; n < NV; ++n) {
            float sc = lsc[(size_t)t * ld + (n < ld ? n : ld - 1)];
            sc = sc > clampv ? clampv : (sc < -clampv ? -clampv : sc);
            if (!(sc == sc)) sc = 0.f;
            tp[n] *= exp((double)sc);
        }
    }
    for (int n = 0; n < NV; ++n) st.tprcn[t * NV + n] = (R)tp[n];
    if (st.elim) return;  // assembly by gather: k_prcn_gather sums tprcn per vertex and side
    for (int i = 0; i < 3; ++i) {
        for (int n = 0; n < NV; ++n) atomic_add(&st.vprcn[v[i] * NV + n], (R)tp[n]);
        if (SM > 0) {
            const int sd = mesh.tri_seg[3 * t + i];
            for (int n = 0; n < NV; ++n) atomic_add(&st.sprcn[sd * NV + n], (R)tp[n]);
        }
    }
}

// res.{v,s} += res_r.{v,s} (nstage.cpp:76-82) for callers of the stand-alone rsdl
template <typename R>
__global__ void k_rsdl_fold(int n1, int n2, R *resv, const R *rrv, R *ress, const R *rrs, const R *dv, const R *ds) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n1) resv[k] += rrv[k] + (dv ? dv[k] : (R)0);
    else if (k < n1 + n2) ress[k - n1] += rrs[k - n1] + (ds ? ds[k - n1] : (R)0);
}

// ---------------------------------------------------------------------------
// Multigrid transfers (tri_hp/movco.cpp:4-106, movfin.cpp:7-82).
// p-levels: the hierarchical basis makes the coarse modes a subset of the fine
// ones: all vertices, the first smc side modes, interior modes (m, k) with the
// fine index offset_f(m) + k. h-levels: barycentric weights of each point in a
// triangle of the other mesh (tri_mesh::mgconnect, connect.cpp:49-87).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int interior_fine_index(int kc, int smc, int smf) {
    // coarse interior index kc -> (m, k) with rows of length smc - m, m = 1..smc-1
    int m = 1, off_c = 0, off_f = 0;
    while (kc >= off_c + (smc - m)) {
        off_c += smc - m;
        off_f += smf - m;
        ++m;
    }
    return off_f + (kc - off_c);
}

// dst_c = src_f restricted to the coarse modes
template <typename R>
__global__ void k_mg_truncate(int npnt, int nseg, int ntri, int NV, int smf, int imf, int smc, int imc,
                              const R *fv, const R *fs, const R *fi, R *cv, R *cs, R *ci) {
    const long nv = (long)npnt * NV, ns = (long)nseg * smc * NV, ni = (long)ntri * imc * NV;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nv + ns + ni; k += (long)gridDim.x * blockDim.x) {
        if (k < nv) {
            cv[k] = fv[k];
        } else if (k < nv + ns) {
            const long q = k - nv;
            const long s = q / (smc * NV), r = q - s * smc * NV, m = r / NV, n = r - m * NV;
            cs[q] = fs[(s * smf + m) * NV + n];
        } else {
            const long q = k - nv - ns;
            const long t = q / (imc * NV), r = q - t * imc * NV, kc = r / NV, n = r - kc * NV;
            ci[q] = fi[(t * imf + interior_fine_index((int)kc, smc, smf)) * NV + n];
        }
    }
}

// fine low modes += (coarse state - coarse state at restriction)
template <typename R>
__global__ void k_mg_prolong_p(int npnt, int nseg, int ntri, int NV, int smf, int imf, int smc, int imc,
                               const R *cv, const R *cs, const R *ci, const R *c0v, const R *c0s, const R *c0i, R *fv,
                               R *fs, R *fi) {
    const long nv = (long)npnt * NV, ns = (long)nseg * smc * NV, ni = (long)ntri * imc * NV;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nv + ns + ni; k += (long)gridDim.x * blockDim.x) {
        if (k < nv) {
            fv[k] += cv[k] - c0v[k];
        } else if (k < nv + ns) {
            const long q = k - nv;
            const long s = q / (smc * NV), r = q - s * smc * NV, m = r / NV, n = r - m * NV;
            fs[(s * smf + m) * NV + n] += cs[q] - c0s[q];
        } else {
            const long q = k - nv - ns;
            const long t = q / (imc * NV), r = q - t * imc * NV, kc = r / NV, n = r - kc * NV;
            fi[(t * imf + interior_fine_index((int)kc, smc, smf)) * NV + n] += ci[q] - c0i[q];
        }
    }
}

// h restriction of the vertex residual: res0_c(v0) += wt * res_f(i) over fine vertices i
template <typename R>
__global__ void k_mg_restrict_hres(int nfine, int NV, const int *f2c_tri, const double *f2c_wt, const int *ctri_pnt,
                                   const R *resf, R *res0c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfine) return;
    const int t = f2c_tri[i];
    for (int j = 0; j < 3; ++j) {
        const int v0 = ctri_pnt[3 * t + j];
        const double w = f2c_wt[3 * i + j];
        for (int n = 0; n < NV; ++n) atomic_add(&res0c[v0 * NV + n], (R)(w * (double)resf[i * NV + n]));
    }
}

// h interpolation of the vertex state: u_c(i) = sum_j wt_j u_f(fine tri pnt j)
template <typename R>
__global__ void k_mg_restrict_hstate(int ncoarse, int NV, const int *c2f_tri, const double *c2f_wt,
                                     const int *ftri_pnt, const R *uf, R *uc, R *uc0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncoarse) return;
    const int t = c2f_tri[i];
    for (int n = 0; n < NV; ++n) {
        double a = 0.0;
        for (int j = 0; j < 3; ++j) a += c2f_wt[3 * i + j] * (double)uf[ftri_pnt[3 * t + j] * NV + n];
        uc[i * NV + n] = (R)a;
        if (uc0) uc0[i * NV + n] = (R)a;
    }
}

// h prolongation: u_f(i) += sum_j wt_j (u_c - u_c0)(coarse tri pnt j)
template <typename R>
__global__ void k_mg_prolong_h(int nfine, int NV, const int *f2c_tri, const double *f2c_wt, const int *ctri_pnt,
                               const R *uc, const R *uc0, R *uf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfine) return;
    const int t = f2c_tri[i];
    for (int n = 0; n < NV; ++n) {
        double a = 0.0;
        for (int j = 0; j < 3; ++j) {
            const int v0 = ctri_pnt[3 * t + j];
            a += f2c_wt[3 * i + j] * (double)(uc[v0 * NV + n] - uc0[v0 * NV + n]);
        }
        uf[i * NV + n] += (R)a;
    }
}

// FAS source (tri_hp::mg_source, nstage.cpp:113-129): dres = fadd*res0 - res(first)
template <typename R>
__global__ void k_fas_source(long n, double fadd, const R *res0, const R *res, R *dres) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        dres[k] = (R)fadd * res0[k] - res[k];
}

template <typename R>
__global__ void k_prcn_invert(int nv_len, int ns_len, R *vprcn, R *sprcn, R vdiag) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nv_len) vprcn[k] = (R)1.0 / (vdiag * vprcn[k]);
    else if (k < nv_len + ns_len) sprcn[k - nv_len] = (R)1.0 / sprcn[k - nv_len];
}

// Sum of squares and max |.| of a vector, block partials into out[2*blockIdx]
template <typename R>
__global__ void k_norm_partial(const R *a, size_t n, double *out) {
    double s = 0.0, mx = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const double v = (double)a[k];
        s += v * v;
        const double av = fabs(v);
        mx = av > mx ? av : mx;
    }
    __shared__ double ss[32], sx[32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        const double b = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = b > mx ? b : mx;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { ss[w] = s; sx[w] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a2 = 0.0, m2 = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            a2 += ss[q];
            m2 = sx[q] > m2 ? sx[q] : m2;
        }
        out[2 * blockIdx.x] = a2;
        out[2 * blockIdx.x + 1] = m2;
    }
}

// History slot bookkeeping for hp_gpu_iterate: maxres of iteration *it goes to
// hist[*it], then *it advances (all on the device, so one captured graph replays).
__global__ void k_hist_advance(unsigned long long *slot, double *hist, int *it, int NV, int cap) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double mx = 0.0;
        for (int n = 0; n < NV; ++n) {
            const double v = __longlong_as_double((long long)slot[n]);
            mx = v > mx ? v : mx;
            slot[n] = 0ull;
        }
        const int k = *it;
        if (k < cap) hist[k] = mx;
        *it = k + 1;
    }
}

// Conversions for the correction form: lo = (lo_t) hi ; hi += (hi_t) lo
template <typename A, typename B>
__global__ void k_convert(long n, const A *src, B *dst) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) dst[k] = (B)src[k];
}
template <typename A, typename B>
__global__ void k_add_into(long n, const A *src, B *dst) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) dst[k] += (B)src[k];
}

}  // namespace hpb

namespace hpb {
// Zeroes the essential (Dirichlet) components of an unpreconditioned residual,
// the rows that vdirichlet/sdirichlet replace by the boundary condition
// (hp_boundary.cpp:680-704), so that its norm measures the equations solved.
template <typename R>
__global__ void k_mask_essential(Mesh mesh, R *resv, R *ress, int NV, int sm) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < mesh.npnt) {
        const int e = mesh.vess[k];
        if (e)
            for (int n = 0; n < NV; ++n)
                if (e & (1 << n)) resv[k * NV + n] = (R)0;
    } else if (k < mesh.npnt + mesh.nseg && sm > 0) {
        const int s = k - mesh.npnt, e = mesh.sess[s];
        if (e)
            for (int m = 0; m < sm; ++m)
                for (int n = 0; n < NV; ++n)
                    if (e & (1 << n)) ress[(s * sm + m) * NV + n] = (R)0;
    }
}
// ---------------------------------------------------------------------------
// tri_hp::l2error (tri_hp/l2error.cpp:13-67) on the device: L2 and L_inf error of the
// state against an analytic field at the quadrature points, sum err^2 wtx wtn cjcb.
// Curved elements take their point coordinates from proj_bdry of crdtocht and their
// Jacobians from calc_metrics, as the reference does.
// ---------------------------------------------------------------------------
struct DevField {
    int kind;
    double prm[4];
};

// The built-in closed forms of include/hp_host.h's hp_field kinds.
__device__ inline double field_value_dev(const DevField &f, int n, double x, double y) {
    const double PI = 3.14159265358979323846;
    switch (f.kind) {
        case 1: {  // Kovasznay, prm[0] = Re
            const double re = f.prm[0], lda = .5 * re - sqrt(re * re / 4 + 4 * PI * PI);
            if (n == 0) return 1.0 - cos(2 * PI * y) * exp(lda * x);
            if (n == 1) return lda / (2 * PI) * sin(2 * PI * y) * exp(lda * x);
            return -.5 * exp(2. * lda * x);
        }
        case 2: return f.prm[0] * sin(PI * x) * sin(PI * y);
        case 3: return f.prm[0] * (x - f.prm[1]) * (x - f.prm[1]);
        case 4: return (n == 0 && y >= 1.0 - 1e-12) ? 1.0 : 0.0;
        case 5: {
            const double d = hypot(x - f.prm[0], y - f.prm[1]);
            return (n == 0 && d > f.prm[2] * (1.0 + 1e-9)) ? 1.0 : 0.0;
        }
        default: return f.prm[n < 4 ? n : 3];
    }
}

template <int P>
struct WtN {
    double w[P + 1];
};

// one thread per element; per-block partials part[block][2 NV] = (sum err^2 per variable,
// max err per variable), reduced on the host in block order
template <int P>
__global__ void __launch_bounds__(128) k_l2error(const DevTables<double, P> *__restrict__ tb, Mesh mesh,
                                                 State<double> st, int NV, DevField fld, WtN<P> wtn, double *part) {
    constexpr int G = P + 1, T = (P + 1) * (P + 2) / 2, SM = (P > 1 ? P - 1 : 1), IM = (P - 1) * (P - 2) / 2,
                  BM = 3 * P;
    double l2[3] = {0.0, 0.0, 0.0}, mx[3] = {0.0, 0.0, 0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mesh.ntri; t += gridDim.x * blockDim.x) {
        const int p0 = mesh.tri_pnt[3 * t], p1 = mesh.tri_pnt[3 * t + 1], p2 = mesh.tri_pnt[3 * t + 2];
        const int cv = mesh.tri_cv ? mesh.tri_cv[t] : -1;
        const double *cht = cv >= 0 ? mesh.crv_cht + (size_t)cv * 2 * BM : nullptr;
        const double g00 = 0.5 * (mesh.pnts[2 * p2] - mesh.pnts[2 * p1]);
        const double g01 = 0.5 * (mesh.pnts[2 * p0] - mesh.pnts[2 * p1]);
        const double g10 = 0.5 * (mesh.pnts[2 * p2 + 1] - mesh.pnts[2 * p1 + 1]);
        const double g11 = 0.5 * (mesh.pnts[2 * p0 + 1] - mesh.pnts[2 * p1 + 1]);
        for (int i = 0; i < G; ++i)
            for (int j = 0; j < G; ++j) {
                double x, y, cjcb;
                if (cht) {  // proj_bdry of the position modes (interior modes zero)
                    x = y = 0.0;
                    for (int m = 0; m < BM; ++m) {
                        const double b = tb->gn[j][m] * tb->gx[i][tb->colof[m]];
                        x += cht[m] * b;
                        y += cht[BM + m] * b;
                    }
                    double d00, d01, d10, d11;
                    curved_metrics<double, P>(*tb, cht, i, j, d00, d01, d10, d11);
                    cjcb = d00 * d11 - d10 * d01;
                } else {  // proj.cpp:188-199 of the vertex coordinates
                    const double b0 = tb->gx[i][0] * tb->gn[j][0], b1 = tb->gx[i][1] * tb->gn[j][1],
                                 b2 = tb->gx[i][2] * tb->gn[j][2];
                    x = mesh.pnts[2 * p0] * b0 + mesh.pnts[2 * p1] * b1 + mesh.pnts[2 * p2] * b2;
                    y = mesh.pnts[2 * p0 + 1] * b0 + mesh.pnts[2 * p1 + 1] * b1 + mesh.pnts[2 * p2 + 1] * b2;
                    cjcb = g00 * g11 - g10 * g01;
                }
                const double wt = tb->wtx[i] * wtn.w[j] * cjcb;
                for (int n = 0; n < NV; ++n) {
                    double u = 0.0;
                    for (int m = 0; m < T; ++m) {  // ugtouht + proj
                        double c;
                        if (m < 3) {
                            c = st.ugv[(m == 0 ? p0 : (m == 1 ? p1 : p2)) * NV + n];
                        } else if (m < BM) {
                            const int si = (m - 3) / SM, k = (m - 3) - si * SM;
                            c = st.ugs[(mesh.tri_seg[3 * t + si] * SM + k) * NV + n];
                            if ((k & 1) && mesh.tri_sgn[3 * t + si] < 0) c = -c;
                        } else {
                            c = st.ugi[((size_t)t * IM + (m - BM)) * NV + n];
                        }
                        u += c * tb->gn[j][m] * tb->gx[i][tb->colof[m]];
                    }
                    const double err = fabs(u - field_value_dev(fld, n, x, y));
                    if (err >= mx[n]) mx[n] = err;
                    l2[n] += err * err * wt;
                }
            }
    }
    __shared__ double sl[3][4], sm_[3][4];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int n = 0; n < 3; ++n) {
        double a = l2[n], b = mx[n];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            const double c = __shfl_xor_sync(0xffffffffu, b, o);
            b = c > b ? c : b;
        }
        if (l == 0) { sl[n][w] = a; sm_[n][w] = b; }
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int n = 0; n < NV; ++n) {
            double a = 0.0, b = 0.0;
            for (int q = 0; q < 4; ++q) { a += sl[n][q]; b = sm_[n][q] > b ? sm_[n][q] : b; }
            part[(size_t)blockIdx.x * 2 * NV + n] = a;
            part[(size_t)blockIdx.x * 2 * NV + NV + n] = b;
        }
}
}  // namespace hpb

namespace hpb {
// Element features of the learned preconditioner (see include/hp_mlp.h).
__global__ void k_elem_features(Mesh mesh, State<double> st, Phys ph, int NV, int sm, int im, int p, float *feat) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mesh.ntri) return;
    float *f = feat + (size_t)t * 17;
    const int v[3] = {mesh.tri_pnt[3 * t], mesh.tri_pnt[3 * t + 1], mesh.tri_pnt[3 * t + 2]};
    double vmax_q = 0.0;
    for (int n = 0; n < 3; ++n) {
        if (n >= NV) { f[4 * n] = f[4 * n + 1] = f[4 * n + 2] = f[4 * n + 3] = 0.f; continue; }
        double a = st.ugv[v[0] * NV + n], b = st.ugv[v[1] * NV + n], c = st.ugv[v[2] * NV + n];
        double mx = fmax(a, fmax(b, c)), mn = fmin(a, fmin(b, c));
        double ss = 0.0;
        for (int i = 0; i < 3; ++i) {
            const int s = mesh.tri_seg[3 * t + i];
            for (int m = 0; m < sm; ++m) { const double x = st.ugs[(s * sm + m) * NV + n]; ss += x * x; }
        }
        double si = 0.0;
        for (int k = 0; k < im; ++k) { const double x = st.ugi[((size_t)t * im + k) * NV + n]; si += x * x; }
        f[4 * n] = (float)((a + b + c) / 3.0);
        f[4 * n + 1] = (float)(mx - mn);
        f[4 * n + 2] = (float)(sm > 0 ? sqrt(ss / (3.0 * sm)) : 0.0);
        f[4 * n + 3] = (float)(im > 0 ? sqrt(si / im) : 0.0);
    }
    if (ph.physics == 1) {
        for (int i = 0; i < 3; ++i) {
            const double u = st.ugv[v[i] * NV], w = st.ugv[v[i] * NV + 1];
            vmax_q = fmax(vmax_q, sqrt(u * u + w * w));
        }
    } else {
        vmax_q = sqrt(ph.ax * ph.ax + ph.ay * ph.ay);
    }
    const double px[3] = {mesh.pnts[2 * v[0]], mesh.pnts[2 * v[1]], mesh.pnts[2 * v[2]]};
    const double py[3] = {mesh.pnts[2 * v[0] + 1], mesh.pnts[2 * v[1] + 1], mesh.pnts[2 * v[2] + 1]};
    const double area2 = (px[0] - px[2]) * (py[1] - py[0]) - (py[0] - py[2]) * (px[1] - px[0]);
    double h2 = 0.0;
    for (int j = 0; j < 3; ++j) {
        const double ex = px[j] - px[(j + 1) % 3], ey = py[j] - py[(j + 1) % 3];
        h2 = fmax(h2, ex * ex + ey * ey);
    }
    const double nu = ph.physics == 1 ? ph.mu / ph.rho : ph.kcond / ph.rhocv;
    f[12] = (float)log(0.25 * fabs(area2) + 1e-300);
    f[13] = (float)(0.5 * log(h2 + 1e-300));
    f[14] = (float)(h2 / (fabs(area2) + 1e-300));
    f[15] = (float)log1p(vmax_q * sqrt(h2) / (nu > 0 ? nu : 1e-300));
    f[16] = (float)p / 8.0f;
}

// Sum of squares of an element's own residual coefficients (vertex, side, interior).
__global__ void k_elem_resnorm(Mesh mesh, State<double> st, int NV, int sm, int im, double *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mesh.ntri) return;
    double s2 = 0.0;
    for (int i = 0; i < 3; ++i) {
        const int v = mesh.tri_pnt[3 * t + i], s = mesh.tri_seg[3 * t + i];
        for (int n = 0; n < NV; ++n) { const double x = st.resv[v * NV + n]; s2 += x * x; }
        for (int m = 0; m < sm; ++m)
            for (int n = 0; n < NV; ++n) { const double x = st.ress[(s * sm + m) * NV + n]; s2 += x * x; }
    }
    for (int k = 0; k < im * NV; ++k) { const double x = st.resi[(size_t)t * im * NV + k]; s2 += x * x; }
    out[t] = s2;
}
}  // namespace hpb
