// 3D (tet_hp) ins residual path on the GPU: context, preconditioner set-up (tau and
// the diagonal element terms) and tet_hp::rsdl with tet_hp_ins::element_rsdl for
// straight tetrahedra.
//
// Reference path (tet_hp/update.cpp:9-118, tet_hp/ins/rsdl.cpp:442-781, tet_hp/ins/bdry.cpp:16-102,
// tet_hp/ins/setup_preconditioner.cpp, tet_hp/gtol.cpp:16-82 and 815-873). The
// basis operators are the dense per-point forms of tet_basis::proj / intgrtrst and
// the 1D operators of derivr / derivs / derivt (include/hp_tet.h), pinned against
// the reference's own tet_basis.
//
// Layout in HBM: one buffer per field (state, res, res_r) holding the vertex, edge,
// face and interior sections back to back, each [entity][mode][4 variables]; the
// dense operators (G^3 x T each) are stored in DMMA fragment order, read through the
// read-only path and stay in L1 / L2. One warp per pair of tetrahedra: the
// projections and integrations run on the FP64 tensor cores, lanes own (tetrahedron,
// point) pairs for the pointwise fluxes, and the per-point arrays live in the warp's
// shared-memory slice. Boundary faces with a flux take one warp each.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hp_gpu.h"
#include "hp_tet.h"
#include "hp_mlp.h"

namespace {

thread_local std::string g_err;
void set_err(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

#define TCK(call)                                                                                    \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);     \
            return HP_ECUDA;                                                                         \
        }                                                                                            \
    } while (0)

constexpr int NV = 4;

template <int P>
struct TetCfg {
    static constexpr int G = P + 1, Q = G * G * G, T = (P + 1) * (P + 2) * (P + 3) / 6;
    static constexpr int EM = P - 1, FM = (P - 1) * (P - 2) / 2, IM = T - 4 - 6 * EM - 4 * FM;
    static constexpr int BM = 4 + 6 * EM + 4 * FM;
};

template <typename R, int P>
struct TetSmall {  // by-value kernel parameter: the 1D derivative operators and factors
    R Ax[P + 1][P + 1], Bx[P + 1][P + 1], Ay[P + 1][P + 1], By[P + 1][P + 1], Az[P + 1][P + 1];
    R y0[P + 1], z0[P + 1];
};

struct TetMeshD {
    int npnt, nseg, ntri, ntet;
    const double *pnts, *vol;
    const int *tp, *ts, *tsg, *tt, *trot;
};

template <typename R>
struct TetFields {
    R *v, *e, *f, *i;
};

// The global location and sign of local mode m of tetrahedron tind (ugtouht / lftog).
template <typename R, int P>
__device__ __forceinline__ R *mode_slot(const TetMeshD &m, const TetFields<R> &g, int tind, int mode, int n,
                                        R &sgn) {
    using C = TetCfg<P>;
    constexpr int EM = C::EM > 0 ? C::EM : 1, FM = C::FM > 0 ? C::FM : 1, IM = C::IM > 0 ? C::IM : 1;
    sgn = (R)1;
    if (mode < 4) return g.v + (size_t)m.tp[4 * tind + mode] * NV + n;
    if (mode < 4 + 6 * C::EM) {
        const int i = (mode - 4) / EM, k = (mode - 4) - i * EM;
        if ((k & 1) && m.tsg[6 * tind + i] < 0) sgn = (R)-1;
        return g.e + ((size_t)m.ts[6 * tind + i] * EM + k) * NV + n;
    }
    if (mode < C::BM) {
        const int r = mode - 4 - 6 * C::EM, i = r / FM, idx = r - i * FM;
        // row of face mode idx: rows 1 .. EM-1 hold EM-1, EM-2, ... modes
        int row = 1, left = idx;
        while (left >= C::EM - row) {
            left -= C::EM - row;
            ++row;
        }
        if (((row - 1) & 1) && m.trot[4 * tind + i] > 0) sgn = (R)-1;  // (-rot)^(row-1)
        return g.f + ((size_t)m.tt[4 * tind + i] * FM + idx) * NV + n;
    }
    return g.i + ((size_t)tind * IM + (mode - C::BM)) * NV + n;
}


// Row (1-based) of face mode idx in the face's triangle of modes: rows 1 .. EM-1 hold EM-1,
// EM-2, ... modes (the sign of a face mode is (-rot)^(row-1)).
template <int EM>
__device__ __forceinline__ int face_mode_row(int idx) {
    int row = 1, left = idx;
    while (left >= EM - row) {
        left -= EM - row;
        ++row;
    }
    return row;
}

// ugtouht (tet_hp/gtol.cpp:16-82) of NE tetrahedra into dst(e)[n T + m], one mode kind per
// loop so that the lanes of an iteration take the same branch and read consecutive values:
// the vertex values, the edge modes (EM NV per edge), the face modes (FM NV per face), the
// interior modes (IM NV per tetrahedron). te(e) is tetrahedron e, act(e) whether it is
// gathered (zeros otherwise). The same values and signs as mode_slot.
template <typename R, int P, int NE, typename TEF, typename ACTF, typename DSTF>
__device__ __forceinline__ void tet_gather_kinds(const TetMeshD &mesh, const TetFields<R> &ug, int lane, TEF te,
                                                 ACTF act, DSTF dst) {
    using C = TetCfg<P>;
    constexpr int T = C::T, EM = C::EM, FM = C::FM, IM = C::IM;
    constexpr int EMD = EM > 0 ? EM : 1, FMD = FM > 0 ? FM : 1, IMD = IM > 0 ? IM : 1;
    constexpr int NVX = NE * 4 * NV, NED = NE * 6 * EM * NV, NFC = NE * 4 * FM * NV, NIN = NE * IM * NV;
#pragma unroll
    for (int it = 0; it < (NVX + 31) / 32; ++it) {
        const int w = lane + 32 * it;
        if (w >= NVX) continue;
        const int e = w / (4 * NV), r = w - e * (4 * NV), m = r / NV, n = r - m * NV;
        dst(e)[n * T + m] = act(e) ? ug.v[(size_t)mesh.tp[4 * te(e) + m] * NV + n] : (R)0;
    }
#pragma unroll
    for (int it = 0; it < (NED + 31) / 32; ++it) {
        const int w = lane + 32 * it;
        if (w >= NED) continue;
        const int b = w / (EMD * NV), r = w - b * (EMD * NV), e = b / 6, i = b - e * 6, k = r / NV, n = r - k * NV;
        R v = (R)0;
        if (act(e)) {
            const int t = te(e);
            v = ug.e[(size_t)mesh.ts[6 * t + i] * (EMD * NV) + r];
            if ((k & 1) && mesh.tsg[6 * t + i] < 0) v = -v;
        }
        dst(e)[n * T + 4 + i * EMD + k] = v;
    }
#pragma unroll
    for (int it = 0; it < (NFC + 31) / 32; ++it) {
        const int w = lane + 32 * it;
        if (w >= NFC) continue;
        const int b = w / (FMD * NV), r = w - b * (FMD * NV), e = b / 4, i = b - e * 4, idx = r / NV,
                  n = r - idx * NV;
        R v = (R)0;
        if (act(e)) {
            const int t = te(e);
            v = ug.f[(size_t)mesh.tt[4 * t + i] * (FMD * NV) + r];
            if (((face_mode_row<EM>(idx) - 1) & 1) && mesh.trot[4 * t + i] > 0) v = -v;
        }
        dst(e)[n * T + 4 + 6 * EM + i * FMD + idx] = v;
    }
#pragma unroll
    for (int it = 0; it < (NIN + 31) / 32; ++it) {
        const int w = lane + 32 * it;
        if (w >= NIN) continue;
        const int e = w / (IMD * NV), r = w - e * (IMD * NV), k = r / NV, n = r - k * NV;
        dst(e)[n * T + C::BM + k] = act(e) ? ug.i[(size_t)te(e) * (IMD * NV) + r] : (R)0;
    }
}

// tet_hp::rsdl element loop (res: imaginary terms, res_r: beta-scaled real terms) on the
// FP64 tensor cores (DMMA, mma.m8n8k4.f64): one warp takes two tetrahedra, so the 8 rows of an A fragment are (tetrahedron, variable) pairs.
//   projection:  C[8 x Q] = U[8 x T] * Op^T[T x Q]   for Op = F, DX, DY, DZ
//   intgrtrst:   C[8 x T] = Flux[8 x 3Q] * WD[3Q x T] (WD = w * (DX; DY; DZ))
// The B operands are constant: the host stores them in fragment order (one 8-byte
// coalesced load per lane per MMA). The pointwise fluxes, the strong residual and
// the SUPG terms stay scalar, lanes owning (tetrahedron, point) pairs.
template <int P>
struct TetMma {
    using C = TetCfg<P>;
    static constexpr int KS = (C::T + 3) / 4;        // projection k-steps
    static constexpr int NT = (C::Q + 7) / 8;        // projection n-tiles
    static constexpr int KS2 = (3 * C::Q + 3) / 4;   // intgrtrst k-steps
    static constexpr int NT2 = (C::T + 7) / 8;       // intgrtrst n-tiles
    static constexpr int WPC = 2;
    // strides padded to 4 (mod 16) doubles: the 4 rows (variables) a half-warp reads
    // in one fragment load fall on distinct shared-memory banks
    static constexpr int pad4(int x) { return x + ((4 - x % 16) + 16) % 16; }
    static constexpr int QP = pad4(C::Q);       // u [NV][QP]
    static constexpr int VS = pad4(3 * C::Q);   // fim / fre [NV][VS], component c at c * Q
    // per tetrahedron: uht [NV][T], u [NV][QP], fim [NV][VS], fre [NV][VS]
    // per tetrahedron: u [3][QP] (u, v, w), fim [NV][VS], fre [NV][VS]; the gathered modes
    // uht [NV][T] and then the pressure at the points share fre's variable-3 slot, which
    // holds nothing else until the SUPG phase (uht is read into registers before the
    // projection stores anything; the pressure values are last read by the pointwise phase)
    static constexpr int S_EL = 3 * QP + 2 * NV * VS;
    static_assert(NV * C::T <= VS && C::Q <= VS, "uht / pressure must fit fre's variable-3 slot");
    static constexpr int NG = NT < 8 ? NT : 8;  // projection n-tiles accumulated together
    static constexpr int S_WARP = 2 * S_EL;
    static constexpr size_t PROJ_LEN = (size_t)4 * NT * KS * 32, INT_LEN = (size_t)NT2 * KS2 * 32;
    static constexpr size_t SMEM = (size_t)S_WARP * WPC * sizeof(double);
};

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// MODE 0: tet_hp::rsdl element loop (res, res_r). MODE 1: the stage-0 element residual
// lf_re + lf_im of every tetrahedron into rbar [ntet][T][NV]. MODE 2: tet_hp::
// jacobian_diagonal (tet_hp/jacobi.cpp:32-111): one item per (tetrahedron, mode m,
// variable n) with uht(n)(m) raised by dw; (lf(n)(m) - rbar) / dw is added, without the
// edge / face sign (its square is 1), to the global diagonal jd.
template <int P, int MODE>
__global__ void __launch_bounds__(TetMma<P>::WPC * 32)
    k_tet_rsdl_mma(const double *__restrict__ projB, const double *__restrict__ intB, TetSmall<double, P> sm,
                   TetMeshD mesh, TetFields<double> ug, TetFields<double> res, TetFields<double> rr,
                   const double *__restrict__ tau, double rho, double mu, double beta, double *rbar,
                   TetFields<double> jd, const float *__restrict__ lsc, float clampv) {
    using C = TetCfg<P>;
    using M = TetMma<P>;
    constexpr int G = C::G, Q = C::Q, T = C::T;
    constexpr int NJ = NV * T;  // items per tetrahedron in MODE 2
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grow = lane >> 2, gcol = lane & 3;  // fragment row / column group
    double *base = reinterpret_cast<double *>(smem_raw) + warp * M::S_WARP;
    constexpr int QP = M::QP, VS = M::VS;
    auto UQ = [&](int e) { return base + e * M::S_EL; };
    auto FIM = [&](int e) { return base + e * M::S_EL + 3 * QP; };
    auto FRE = [&](int e) { return base + e * M::S_EL + 3 * QP + NV * VS; };
    auto UHT = [&](int e) { return FRE(e) + 3 * VS; };
    auto PV = [&](int e) { return FRE(e) + 3 * VS; };
    const long nitems = MODE == 2 ? (long)mesh.ntet * NJ : (long)mesh.ntet;
    const long npair = (nitems + 1) / 2;
    for (long pr = (long)blockIdx.x * M::WPC + warp; pr < npair; pr += (long)gridDim.x * M::WPC) {
        const long it0 = 2 * pr;
        const bool has1 = it0 + 1 < nitems;
        // tetrahedron of item e (a missing second item repeats the first)
        int te[2];
        for (int e = 0; e < 2; ++e) {
            const long it = (e == 1 && has1) ? it0 + 1 : it0;
            te[e] = MODE == 2 ? (int)(it / NJ) : (int)it;
        }
        // ---- gather both tetrahedra (a missing second one gets zeros)
        tet_gather_kinds<double, P, 2>(
            mesh, ug, lane, [&](int e) { return e ? te[1] : te[0]; }, [&](int e) { return e == 0 || has1; },
            [&](int e) { return UHT(e); });
        double dw[2] = {0.0, 0.0};
        int jm[2] = {0, 0}, jn[2] = {0, 0};
        if constexpr (MODE == 2) {
            __syncwarp();
            // dw = 1e-6 sum over the 4 vertex modes of all variables + 1e-10, the same for
            // every variable (jacobi.cpp:63-67)
            for (int e = 0; e < 2; ++e) {
                double sdw = 0.0;
                for (int n = 0; n < NV; ++n)
                    for (int i = 0; i < 4; ++i) sdw += fabs(UHT(e)[n * T + i]);
                dw[e] = sdw * 1.0e-6 + 1.0e-10;
                const long it = (e == 1 && has1) ? it0 + 1 : it0;
                const int j = (int)(it - (long)te[e] * NJ);
                jm[e] = j / NV;
                jn[e] = j - jm[e] * NV;
            }
            __syncwarp();
            if (lane < 2 && (lane == 0 || has1)) UHT(lane)[jn[lane] * T + jm[lane]] += dw[lane];
        }
        // geometry of both (the missing one repeats the first)
        double d[2][3][3], cj[2];
        for (int e = 0; e < 2; ++e) {
            const int t = te[e];
            const int v0 = mesh.tp[4 * t], v1 = mesh.tp[4 * t + 1], v2 = mesh.tp[4 * t + 2], v3 = mesh.tp[4 * t + 3];
            double ld[3][3];
            for (int n = 0; n < 3; ++n) {
                const double c2 = mesh.pnts[3 * v2 + n];
                ld[n][0] = 0.5 * (mesh.pnts[3 * v3 + n] - c2);
                ld[n][1] = 0.5 * (mesh.pnts[3 * v1 + n] - c2);
                ld[n][2] = 0.5 * (mesh.pnts[3 * v0 + n] - c2);
            }
            d[e][0][0] = ld[1][1] * ld[2][2] - ld[1][2] * ld[2][1];
            d[e][0][1] = -ld[0][1] * ld[2][2] + ld[0][2] * ld[2][1];
            d[e][0][2] = ld[0][1] * ld[1][2] - ld[0][2] * ld[1][1];
            d[e][1][0] = -ld[1][0] * ld[2][2] + ld[1][2] * ld[2][0];
            d[e][1][1] = ld[0][0] * ld[2][2] - ld[0][2] * ld[2][0];
            d[e][1][2] = -ld[0][0] * ld[1][2] + ld[0][2] * ld[1][0];
            d[e][2][0] = ld[1][0] * ld[2][1] - ld[1][1] * ld[2][0];
            d[e][2][1] = -ld[0][0] * ld[2][1] + ld[0][1] * ld[2][0];
            d[e][2][2] = ld[0][0] * ld[1][1] - ld[0][1] * ld[1][0];
            cj[e] = ld[0][0] * (ld[1][1] * ld[2][2] - ld[1][2] * ld[2][1]) -
                    ld[0][1] * (ld[1][0] * ld[2][2] - ld[2][0] * ld[1][2]) +
                    ld[0][2] * (ld[1][0] * ld[2][1] - ld[2][0] * ld[1][1]);
        }
        __syncwarp();
        // ---- projection on the tensor cores: row (e, n) = (grow >> 2, grow & 3)
        {
            const int e = grow >> 2, n = grow & 3;
            double a[M::KS];
#pragma unroll
            for (int ks = 0; ks < M::KS; ++ks) {
                const int m = ks * 4 + gcol;
                a[ks] = m < T ? UHT(e)[n * T + m] : 0.0;
            }
            __syncwarp();  // uht is dead from here: its slot takes the pressure values
            const bool needd = beta > 0.0;
            for (int op = 0; op < (needd ? 4 : 1); ++op) {
                double *dst = op == 0 ? (n < 3 ? UQ(e) + n * QP : PV(e))
                                      : (n < 3 ? FRE(e) + n * VS + (op - 1) * Q : nullptr);
                for (int nt0 = 0; nt0 < M::NT; nt0 += M::NG) {
                    // NG independent accumulator chains
                    double c[M::NG][2];
#pragma unroll
                    for (int g = 0; g < M::NG; ++g) c[g][0] = c[g][1] = 0.0;
                    const double *b = projB + ((size_t)(op * M::NT + nt0) * M::KS) * 32 + lane;
#pragma unroll
                    for (int ks = 0; ks < M::KS; ++ks)
#pragma unroll
                        for (int g = 0; g < M::NG; ++g)
                            if (nt0 + g < M::NT) dmma(c[g][0], c[g][1], a[ks], __ldg(b + ((size_t)g * M::KS + ks) * 32));
                    if (dst) {
#pragma unroll
                        for (int g = 0; g < M::NG; ++g) {
                            const int q = (nt0 + g) * 8 + gcol * 2;
                            if (q < Q) dst[q] = c[g][0];
                            if (q + 1 < Q) dst[q + 1] = c[g][1];
                        }
                    }
                }
            }
        }
        __syncwarp();
        // ---- pointwise fluxes, lanes own (e, q): fim = convective + pressure / continuity;
        //      fre = viscous flux from the velocity derivatives stored there
        for (int w = lane; w < 2 * Q; w += 32) {
            const int e = w / Q, q = w - e * Q;
            const double *uq = UQ(e);
            double *fim = FIM(e), *fre = FRE(e);
            const double uu[4] = {uq[q], uq[QP + q], uq[2 * QP + q], PV(e)[q]};
            const double fx = rho * uu[0], fy = rho * uu[1], fz = rho * uu[2];
            double f3[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                f3[c] = d[e][c][0] * fx + d[e][c][1] * fy + d[e][c][2] * fz;
                fim[3 * VS + c * Q + q] = f3[c];
            }
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int c = 0; c < 3; ++c) fim[n * VS + c * Q + q] = uu[n] * f3[c] + d[e][c][n] * uu[3];
            if (beta > 0.0) {
                double du[3][3];
#pragma unroll
                for (int n = 0; n < 3; ++n)
#pragma unroll
                    for (int c = 0; c < 3; ++c) du[n][c] = fre[n * VS + c * Q + q];
                const double cjcbi = mu / cj[e];
                double h[3][3];
#pragma unroll
                for (int b = 0; b < 3; ++b)
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        h[b][a] = d[e][0][a] * du[b][0] + d[e][1][a] * du[b][1] + d[e][2][a] * du[b][2];
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double s = 0.0;
#pragma unroll
                        for (int ee = 0; ee < 3; ++ee) {
                            const double gce = d[e][c][0] * d[e][ee][0] + d[e][c][1] * d[e][ee][1] + d[e][c][2] * d[e][ee][2];
                            s += gce * du[a][ee];
                        }
                        s += d[e][c][0] * h[0][a] + d[e][c][1] * h[1][a] + d[e][c][2] * h[2][a];
                        fre[a * VS + c * Q + q] = -cjcbi * s;
                    }
            }
        }
        __syncwarp();
        if (beta > 0.0) {
            // ---- strong residual at the owned points
            constexpr int NW = (2 * Q + 31) / 32;
            double rsd[NW][NV];
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                const int w = lane + 32 * k;
                if (w >= 2 * Q) break;
                const int e = w / Q, q = w - e * Q;
                const int i = q / (G * G), j = (q / G) % G, kk = q % G;
                const double yz = sm.y0[j] * sm.z0[kk], zz = sm.z0[kk];
                const double *fim = FIM(e), *fre = FRE(e);
#pragma unroll
                for (int n = 0; n < NV; ++n) {
                    auto fl = [&](int c, int i2, int j2, int k2) -> double {
                        const int q2 = (i2 * G + j2) * G + k2;
                        return n < 3 ? fim[n * VS + c * Q + q2] + fre[n * VS + c * Q + q2] : fim[3 * VS + c * Q + q2];
                    };
                    double ax = 0, bxs = 0, bxt = 0, ays = 0, byt = 0, azt = 0;
#pragma unroll
                    for (int l = 0; l < G; ++l) {
                        ax += sm.Ax[i][l] * fl(0, l, j, kk);
                        bxs += sm.Bx[i][l] * fl(1, l, j, kk);
                        bxt += sm.Bx[i][l] * fl(2, l, j, kk);
                        ays += sm.Ay[j][l] * fl(1, i, l, kk);
                        byt += sm.By[j][l] * fl(2, i, l, kk);
                        azt += sm.Az[kk][l] * fl(2, i, j, l);
                    }
                    rsd[k][n] = yz * ax + (yz * bxs + zz * ays) + (yz * bxt + zz * byt + azt);
                }
            }
            __syncwarp();
            // ---- SUPG terms into fre (viscous + SUPG; variable 3: the continuity SUPG term)
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                const int w = lane + 32 * k;
                if (w >= 2 * Q) break;
                const int e = w / Q, q = w - e * Q;
                const int t = te[e];
                const double tau0 = tau[2 * t], tau3 = tau[2 * t + 1];
                double *fre = FRE(e);
                const double *uq = UQ(e);
                double tr[NV], uu[3];
#pragma unroll
                for (int n = 0; n < 3; ++n) {
                    tr[n] = tau0 * rsd[k][n];
                    uu[n] = uq[n * QP + q];
                }
                tr[3] = tau3 * rsd[k][3];
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double s2 = d[e][c][a] * (2.0 * uu[a]);
#pragma unroll
                        for (int b = 0; b < 3; ++b)
                            if (b != a) s2 += d[e][c][b] * uu[b];
                        double r = s2 * tr[a];
#pragma unroll
                        for (int b = 0; b < 3; ++b)
                            if (b != a) r += d[e][c][b] * uu[a] * tr[b];
                        r += d[e][c][a] * tr[3];
                        fre[a * VS + c * Q + q] -= r;
                    }
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    fre[3 * VS + c * Q + q] = -d[e][c][0] * tr[0] - d[e][c][1] * tr[1] - d[e][c][2] * tr[2];
            }
            __syncwarp();
        }
        // ---- intgrtrst on the tensor cores (imaginary into res, real * beta into res_r); with a
        //      real part both share each operator fragment load
        {
            const int e = grow >> 2, n = grow & 3;
            const bool two = beta > 0.0;
            double tot[M::NT2][2];
            const double *fai = FIM(e) + n * VS, *far = FRE(e) + n * VS;  // [3][Q] = k order
            double ci[M::NT2][2], cr[M::NT2][2];
#pragma unroll
            for (int nt = 0; nt < M::NT2; ++nt) ci[nt][0] = ci[nt][1] = cr[nt][0] = cr[nt][1] = 0.0;
#pragma unroll 2
            for (int ks = 0; ks < M::KS2; ++ks) {
                const int k = ks * 4 + gcol;
                const double ai = k < 3 * Q ? fai[k] : 0.0;
                const double ar = (two && k < 3 * Q) ? far[k] : 0.0;
#pragma unroll
                for (int nt = 0; nt < M::NT2; ++nt) {
                    const double bf = __ldg(intB + ((size_t)nt * M::KS2 + ks) * 32 + lane);
                    dmma(ci[nt][0], ci[nt][1], ai, bf);
                    if (two) dmma(cr[nt][0], cr[nt][1], ar, bf);
                }
            }
            const bool ok = (e == 0 || has1);
#pragma unroll
            for (int nt = 0; nt < M::NT2; ++nt)
#pragma unroll
                for (int h2 = 0; h2 < 2; ++h2) {
                    // row grow = (e, n); columns m = nt*8 + gcol*2 + {0, 1}
                    const int m = nt * 8 + gcol * 2 + h2;
                    tot[nt][h2] = 0.0;
                    if (!ok || m >= T) continue;
                    const double vi = -ci[nt][h2], vr = -cr[nt][h2];
                    if constexpr (MODE != 0) {
                        tot[nt][h2] = two ? vi + beta * vr : vi;
                    } else {
                        double sg;
                        double *dst = mode_slot<double, P>(mesh, res, te[e], m, n, sg);
                        if (m < C::BM) atomicAdd(dst, sg * vi);
                        else *dst = vi;
                        if (two) {
                            double *dr = mode_slot<double, P>(mesh, rr, te[e], m, n, sg);
                            if (m < C::BM) atomicAdd(dr, beta * sg * vr);
                            else *dr += beta * vr;
                        }
                    }
                }
            if constexpr (MODE != 0) {
                const bool ok = (e == 0 || has1);
#pragma unroll
                for (int nt = 0; nt < M::NT2; ++nt)
#pragma unroll
                    for (int h2 = 0; h2 < 2; ++h2) {
                        const int m = nt * 8 + gcol * 2 + h2;
                        if (!ok || m >= T) continue;
                        const size_t rb = ((size_t)te[e] * T + m) * NV + n;
                        if constexpr (MODE == 1) {
                            rbar[rb] = tot[nt][h2];
                        } else {
                            if (m != jm[e] || n != jn[e]) continue;
                            double sg;
                            double *dst = mode_slot<double, P>(mesh, jd, te[e], m, n, sg);
                            double sc = 1.0;  // learned per-tetrahedron scale of its contribution
                            if (lsc) {
                                float c = lsc[te[e]];
                                c = c > clampv ? clampv : (c < -clampv ? -clampv : c);
                                if (!(c == c)) c = 0.f;
                                sc = exp((double)c);
                            }
                            atomicAdd(dst, sc * (tot[nt][h2] - rbar[rb]) / dw[e]);
                        }
                    }
            }
        }
        __syncwarp();
    }
}

// res = 0; res_r *= 1 - beta  (tet_hp::rsdl prologue)
template <typename R>
__global__ void k_tet_pre(long n, R *res, R *rr, R omb) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        res[k] = (R)0;
        rr[k] *= omb;
    }
}

struct TetFacesD {  // boundary faces with a flux
    int n;
    const int *tri, *pnt, *seg, *sgn, *kind;  // [n], [n][3], [n][3], [n][3], [n]
    const double *pbc;                        // [n][G * G]
};

// hp_face_bdry::rsdl of bdry_ins::neumann / inflow (tet_hp/ins/bdry.cpp:16-102, fluxes
// tet_hp/ins/bdry_ins.h:85-132), straight faces: one warp per face. Lane k < T2 gathers face
// mode k (ugtouht2d, tet_hp/gtol.cpp:257-299); lane q < G*G evaluates u, the normal
// d(x)/dr x d(x)/ds and the flux at face point q; lane k integrates (intgrt2d) and adds into
// res. ftab = F2, DX2, DY2 [G*G][T2], W2 [G*G].
template <int P>
__global__ void __launch_bounds__(128) k_tet_face_flux(TetFacesD fc, const double *__restrict__ ftab, TetMeshD mesh,
                                                       TetFields<double> u, TetFields<double> res, double rho) {
    constexpr int G = P + 1, G2 = G * G, EM = P - 1, FM = (P - 1) * (P - 2) / 2, T2 = 3 + 3 * EM + FM;
    constexpr int EMD = EM > 0 ? EM : 1, FMD = FM > 0 ? FM : 1, WPB = 4;
    static_assert(G2 <= 32 && T2 <= 32, "one lane per face point and per face mode");
    __shared__ double sflx[WPB][NV][G2];
    const double *F2 = ftab, *DX2 = ftab + G2 * T2, *DY2 = ftab + 2 * G2 * T2, *W2 = ftab + 3 * G2 * T2;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (int b = blockIdx.x * WPB + wib; b < fc.n; b += gridDim.x * WPB) {  // warp-uniform
        const int find = fc.tri[b], kind = fc.kind[b];
        int pv[3], ps[3], sg[3];
        for (int i = 0; i < 3; ++i) {
            pv[i] = fc.pnt[3 * b + i];
            ps[i] = fc.seg[3 * b + i];
            sg[i] = fc.sgn[3 * b + i];
        }
        double lin[3] = {0.0, 0.0, 0.0};
        if (lane < 3) {
            for (int n = 0; n < 3; ++n) lin[n] = u.v[(size_t)pv[lane] * NV + n];
        } else if (lane < 3 + 3 * EM) {
            const int i = (lane - 3) / EMD, m = (lane - 3) - i * EMD;
            const double s = ((m & 1) && sg[i] < 0) ? -1.0 : 1.0;
            for (int n = 0; n < 3; ++n) lin[n] = s * u.e[((size_t)ps[i] * EMD + m) * NV + n];
        } else if (lane < T2) {
            const int k = lane - 3 - 3 * EM;
            for (int n = 0; n < 3; ++n) lin[n] = u.f[((size_t)find * FMD + k) * NV + n];
        }
        double uq[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < T2; ++k) {
            const double f = lane < G2 ? __ldg(F2 + lane * T2 + k) : 0.0;
            for (int n = 0; n < 3; ++n) uq[n] += f * __shfl_sync(0xffffffffu, lin[n], k);
        }
        if (lane < G2) {
            double dr[3] = {0.0, 0.0, 0.0}, ds[3] = {0.0, 0.0, 0.0};
            for (int v = 0; v < 3; ++v) {
                const double a = __ldg(DX2 + lane * T2 + v), c = __ldg(DY2 + lane * T2 + v);
                for (int d = 0; d < 3; ++d) {
                    const double x = mesh.pnts[3 * (size_t)pv[v] + d];
                    dr[d] += a * x;
                    ds[d] += c * x;
                }
            }
            const double nrm[3] = {dr[1] * ds[2] - dr[2] * ds[1], dr[2] * ds[0] - dr[0] * ds[2],
                                   dr[0] * ds[1] - dr[1] * ds[0]};
            const double mf = rho * (uq[0] * nrm[0] + uq[1] * nrm[1] + uq[2] * nrm[2]);
            const double pb = kind ? fc.pbc[(size_t)b * G2 + lane] : 0.0;
            for (int n = 0; n < 3; ++n) sflx[wib][n][lane] = kind ? mf * uq[n] + pb * nrm[n] : 0.0;
            sflx[wib][3][lane] = mf;
        }
        __syncwarp();
        if (lane < T2) {
            double r[NV] = {0.0, 0.0, 0.0, 0.0};
            for (int q = 0; q < G2; ++q) {
                const double wf = __ldg(W2 + q) * __ldg(F2 + q * T2 + lane);
                for (int n = 0; n < NV; ++n) r[n] += wf * sflx[wib][n][q];
            }
            const int n0 = kind ? 0 : 3;  // inflow: the momentum fluxes are zero
            if (lane < 3) {
                for (int n = n0; n < NV; ++n) atomicAdd(res.v + (size_t)pv[lane] * NV + n, r[n]);
            } else if (lane < 3 + 3 * EM) {
                const int i = (lane - 3) / EMD, m = (lane - 3) - i * EMD;
                const double s = ((m & 1) && sg[i] < 0) ? -1.0 : 1.0;
                for (int n = n0; n < NV; ++n) atomicAdd(res.e + ((size_t)ps[i] * EMD + m) * NV + n, s * r[n]);
            } else {
                const int k = lane - 3 - 3 * EM;
                for (int n = n0; n < NV; ++n) atomicAdd(res.f + ((size_t)find * FMD + k) * NV + n, r[n]);
            }
        }
        __syncwarp();
    }
}

// res += res_r
template <typename R>
__global__ void k_tet_fold(long n, R *res, const R *rr) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        res[k] += rr[k];
}

// tet_hp_ins::setup_preconditioner, diagonal branch, steady, mesh velocity zero
__global__ void k_tet_prcn(TetMeshD mesh, const double *ugv, double *tau, double *iprcn, double *vprcn,
                           double *eprcn, double *fprcn, int p, int em, int fm, double rho, double mu, double adis,
                           double bd0, int *err, const float *lsc, float clampv) {
    const int VF[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};
    const double nu = mu / rho;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mesh.ntet; t += gridDim.x * blockDim.x) {
        double jcb = 0.125 * mesh.vol[t];
        const int *v = mesh.tp + 4 * t;
        double amin = 1.0e99, amax = 0.0;
        for (int j = 0; j < 4; ++j) {
            const double *a = mesh.pnts + 3 * v[VF[j][0]], *b = mesh.pnts + 3 * v[VF[j][1]],
                         *c = mesh.pnts + 3 * v[VF[j][2]];
            const double v1[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
            const double v2[3] = {a[0] - c[0], a[1] - c[1], a[2] - c[2]};
            const double cr[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                                  v1[0] * v2[1] - v1[1] * v2[0]};
            const double ar = .5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            amax = ar > amax ? ar : amax;
            amin = ar < amin ? ar : amin;
        }
        const double h = 4.0 * jcb / (0.25 * (p + 1) * (p + 1) * amax);
        const double hmax = 4.0 * jcb / (0.25 * (p + 1) * (p + 1) * amin);
        double qmax = 0.0;
        for (int j = 0; j < 4; ++j) {
            const double *uu = ugv + (size_t)v[j] * NV;
            const double q = uu[0] * uu[0] + uu[1] * uu[1] + uu[2] * uu[2];
            qmax = q > qmax ? q : qmax;
        }
        if (!(jcb > 0.0) || !(qmax >= 0.0)) atomicAdd(err, 1);
        const double tm = 0.5 * hmax * bd0 + 2. * nu / hmax;
        double gam = 3.0 * qmax + tm * tm;
        if (mu + bd0 == 0.0) gam = gam > 0.1 ? gam : 0.1;
        const double q = sqrt(qmax);
        const double lam1 = q + sqrt(qmax + gam);
        tau[2 * t] = adis * h / (jcb * sqrt(gam));
        tau[2 * t + 1] = qmax * tau[2 * t];
        jcb *= 2. * nu * (1. / (h * h) + 1. / (h * h) + 1. / (h * h)) + 3 * lam1 / h;
        double ip[NV] = {rho * jcb, rho * jcb, rho * jcb, jcb / gam};
        if (lsc) {  // learned per-tetrahedron scale of its diagonal block (minvrt's preconditioner)
            float cs = lsc[t];
            cs = cs > clampv ? clampv : (cs < -clampv ? -clampv : cs);
            if (!(cs == cs)) cs = 0.f;
            for (int n = 0; n < NV; ++n) ip[n] *= exp((double)cs);
        }
        for (int n = 0; n < NV; ++n) iprcn[(size_t)t * NV + n] = ip[n];
        for (int i = 0; i < 4; ++i)
            for (int n = 0; n < NV; ++n) atomicAdd(vprcn + (size_t)v[i] * NV + n, ip[n]);
        if (em > 0)
            for (int i = 0; i < 6; ++i)
                for (int n = 0; n < NV; ++n) atomicAdd(eprcn + (size_t)mesh.ts[6 * t + i] * NV + n, ip[n]);
        if (fm > 0)
            for (int i = 0; i < 4; ++i)
                for (int n = 0; n < NV; ++n) atomicAdd(fprcn + (size_t)mesh.tt[4 * t + i] * NV + n, ip[n]);
    }
}

// tet_hp::update stage, JACOBI build (update.cpp:206-390, jacobi.cpp:14-30): essential rows
// zeroed, res = 0.5 res / jacob_diag, ug = ug0 - cflalpha res
// tet_hp::minvrt at p = 1 (its em = 0 branch, tet_hp/setup_preconditioner.cpp:57-74, vprcn
// pre-inverted as in tet_hp::setup_preconditioner) with the nstage update of tet_hp::update
// (tet_hp/update.cpp:181-390): res.v *= (1 / vprcn) vdiag, fixed rows zeroed, ug = ug0 - ca res.
template <typename R>
__global__ void k_tet_minvrt1(long n, R *res, const R *vprcn, R vdiag, const unsigned char *mask, R *u, const R *u0,
                              R ca) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const R r = mask[k] ? (R)0 : res[k] * (((R)1 / vprcn[k]) * vdiag);
        res[k] = r;
        u[k] = u0[k] - ca * r;
    }
}

// tet_hp::minvrt at p = 2 (tet_hp/setup_preconditioner.cpp:16-30, 57-131, 197-221), in four
// passes. (1) Edge modes removed from their end vertices: res.v -= sfmv(end, k) res.e.
// The rows fixed by essential conditions were zeroed before minvrt (mask_e: the edge section).
template <typename R>
__global__ void k_tet_minv_e2v(int nseg, int em, const int *seg_pnt, const R *sfmv, R *resv, const R *rese,
                               const unsigned char *mask_e) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
        for (int k = 0; k < em; ++k)
            for (int i = 0; i < 2; ++i) {
                const int v = seg_pnt[2 * s + i];
                for (int n = 0; n < NV; ++n) {
                    const size_t e = ((size_t)s * em + k) * NV + n;
                    if (!mask_e[e]) atomicAdd(resv + (size_t)v * NV + n, -sfmv[i * (HP_TET_MAXP - 1) + k] * rese[e]);
                }
            }
}

// (2) / (4) res *= (1 / prcn(entity, var)) diag on one section, fixed rows zeroed
template <typename R>
__global__ void k_tet_minv_scale(long n, int modes, R *res, const R *prcn, R diag, const unsigned char *mask) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const long ent = k / ((long)modes * NV), var = k % NV;
        res[k] = mask[k] ? (R)0 : res[k] * (((R)1 / prcn[ent * NV + var]) * diag);
    }
}

// (3) Vertex values (times the element diagonal iprcn) removed from the edge modes:
// res.e(edge, k) -= sgn^k mm(j, 4 + k + i em) res.v(v_j) iprcn(tet)
template <typename R>
__global__ void k_tet_minv_v2e(TetMeshD m, int em, const R *mm, const R *iprcn, const R *resv, R *rese) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m.ntet; t += gridDim.x * blockDim.x) {
        R uh[4][NV];
        for (int j = 0; j < 4; ++j)
            for (int n = 0; n < NV; ++n) uh[j][n] = resv[(size_t)m.tp[4 * t + j] * NV + n] * iprcn[(size_t)t * NV + n];
        for (int i = 0; i < 6; ++i) {
            const int sind = m.ts[6 * t + i], sg = m.tsg[6 * t + i];
            for (int j = 0; j < 4; ++j) {
                R msgn = 1;
                for (int k = 0; k < em; ++k) {
                    const R c = mm[j * HP_TET_MAXT + 4 + k + i * em];
                    for (int n = 0; n < NV; ++n) atomicAdd(rese + ((size_t)sind * em + k) * NV + n, -msgn * c * uh[j][n]);
                    msgn *= sg;
                }
            }
        }
    }
}

// ---- tet_hp::minvrt at p = 3 (tet_hp/setup_preconditioner.cpp:16-354) and its vertex-ball
// spoke factors (tet_hp::spoke, :530-583). em = 2, fm = 1, im = 0; iprcn is not inverted at
// im = 0. Faces carry their vertices in the order of the tetrahedron that numbered them and
// face edge i is the edge opposite face vertex i (tri_pnt / tri_seg below).
constexpr int SPK_MAX = 64;  // spokes (edges) per vertex the solve kernel takes

// rows fixed by essential conditions zeroed (the vdirichlet / edirichlet / fdirichlet of
// tet_hp::update before minvrt, and minvrt's own)
template <typename R>
__global__ void k_tet_zero_fixed(long n, R *res, const unsigned char *mask) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        if (mask[k]) res[k] = (R)0;
}

// face modes removed from the face's vertices: res.v(tri.pnt(i)) -= ffmv(i, k) res.f(k)
template <typename R>
__global__ void k_tet_minv_f2v(int ntri, int fm, const int *tri_pnt, const R *ffmv, R *resv, const R *resf) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < ntri; f += gridDim.x * blockDim.x)
        for (int i = 0; i < 3; ++i) {
            const int v = tri_pnt[3 * f + i];
            for (int k = 0; k < fm; ++k)
                for (int n = 0; n < NV; ++n)
                    atomicAdd(resv + (size_t)v * NV + n,
                              -ffmv[i * (HP_TET_MAXP * (HP_TET_MAXP - 1) / 2) + k] * resf[((size_t)f * fm + k) * NV + n]);
        }
}

// the face modes' share of a tetrahedron's removal: res.f(tri(i), ind) -= msgn mm(row, col(j))
// u(j) iprcn, with msgn = (-rot)^(m-1) over the face-mode pairs (m, k); col(j) = j for the
// vertex values (src = 0: u(j) = res.v of vertex j), 4 + j em (src = 1: res.e(seg(j), 0)) or
// 5 + j em (src = 2: res.e(seg(j), 1)). src = 1 also removes the first edge modes from the
// higher edge modes: res.e(seg(i), k) -= sgn^k mm(k + 4 + i em, 4 + j em) u(j).
template <typename R>
__global__ void k_tet_minv3_remove(TetMeshD m, int em, int fm, int src, const R *mm, const R *iprcn, const R *resv,
                                   R *rese, R *resf) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m.ntet; t += gridDim.x * blockDim.x) {
        const int nj = src == 0 ? 4 : 6;
        R uh[6][NV];
        for (int j = 0; j < nj; ++j)
            for (int n = 0; n < NV; ++n) {
                const R x = src == 0 ? resv[(size_t)m.tp[4 * t + j] * NV + n]
                                     : rese[((size_t)m.ts[6 * t + j] * em + (src - 1)) * NV + n];
                uh[j][n] = x * iprcn[(size_t)t * NV + n];
            }
        if (src == 0) {
            for (int i = 0; i < 6; ++i) {
                const int sind = m.ts[6 * t + i], sg = m.tsg[6 * t + i];
                for (int j = 0; j < 4; ++j) {
                    R msgn = 1;
                    for (int k = 0; k < em; ++k) {
                        const R c = mm[j * HP_TET_MAXT + 4 + k + i * em];
                        for (int n = 0; n < NV; ++n)
                            atomicAdd(rese + ((size_t)sind * em + k) * NV + n, -msgn * c * uh[j][n]);
                        msgn *= sg;
                    }
                }
            }
        } else if (src == 1) {
            for (int i = 0; i < 6; ++i) {
                const int sind = m.ts[6 * t + i], sg = m.tsg[6 * t + i];
                for (int j = 0; j < 6; ++j) {
                    R msgn = (R)sg;
                    for (int k = 1; k < em; ++k) {
                        const R c = mm[(k + 4 + i * em) * HP_TET_MAXT + 4 + j * em];
                        for (int n = 0; n < NV; ++n)
                            atomicAdd(rese + ((size_t)sind * em + k) * NV + n, -msgn * c * uh[j][n]);
                        msgn *= sg;
                    }
                }
            }
        }
        for (int i = 0; i < 4; ++i) {
            const int f = m.tt[4 * t + i], sg = -m.trot[4 * t + i];
            for (int j = 0; j < nj; ++j) {
                R msgn = 1;
                int ind = 0;
                const int col = src == 0 ? j : (src == 1 ? 4 + j * em : 5 + j * em);
                for (int mm_ = 1; mm_ <= em - 1; ++mm_) {
                    for (int k = 1; k <= em - mm_; ++k, ++ind) {
                        const R c = src == 0 ? mm[col * HP_TET_MAXT + 4 + 6 * em + i * fm + ind]
                                             : mm[(4 + 6 * em + i * fm + ind) * HP_TET_MAXT + col];
                        for (int n = 0; n < NV; ++n) atomicAdd(resf + ((size_t)f * fm + ind) * NV + n, -msgn * c * uh[j][n]);
                    }
                    msgn *= sg;
                }
            }
        }
    }
}

// the spoke values of each edge end: w(s, 0 / 1) = e0 +- sfms(0) e1, and e0 = 0
template <typename R>
__global__ void k_tet_spoke_w(int nseg, int em, R sfms0, R *rese, R *w) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
        for (int n = 0; n < NV; ++n) {
            R *e = rese + (size_t)s * em * NV + n;
            const R e0 = e[0], e1 = e[NV];
            w[((size_t)s * 2) * NV + n] = e0 + sfms0 * e1;
            w[((size_t)s * 2 + 1) * NV + n] = e0 - sfms0 * e1;
            e[0] = (R)0;
        }
}

// the face modes' share of the spoke values: edge i of face f takes ffms(i, k, 1) at the end
// that is face vertex 2 (i = 0) or 0 (i = 1, 2), ffms(i, k, 0) at the other
template <typename R>
__global__ void k_tet_spoke_faces(int ntri, int fm, const int *tri_pnt, const int *tri_seg, const int *seg_pnt,
                                  const R *ffms, const R *resf, R *w) {
    constexpr int FS = HP_TET_MAXP * (HP_TET_MAXP - 1) / 2;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < ntri; f += gridDim.x * blockDim.x)
        for (int i = 0; i < 3; ++i) {
            const int s = tri_seg[3 * f + i], x = tri_pnt[3 * f + (i == 0 ? 2 : 0)];
            const int c1 = seg_pnt[2 * s] == x ? 0 : 1;
            for (int k = 0; k < fm; ++k) {
                const R a = ffms[(i * FS + k) * 2], b = ffms[(i * FS + k) * 2 + 1];
                for (int n = 0; n < NV; ++n) {
                    const R rf = resf[((size_t)f * fm + k) * NV + n];
                    atomicAdd(w + ((size_t)s * 2 + c1) * NV + n, b * rf);
                    atomicAdd(w + ((size_t)s * 2 + 1 - c1) * NV + n, a * rf);
                }
            }
        }
}

// the vertex-ball solve, one thread per (vertex, variable): the spoke values of the vertex's
// edges, solved with its LU factor (unit lower, upper; no row exchanges: the spoke matrix is
// diagonally dominant), half of each solution added to the edge's first mode
template <typename R>
__global__ void k_tet_spoke_solve(int npnt, int em, const int *vs_ptr, const int *vs_seg, const int *vs_end,
                                  const long long *fptr, const R *fac, const R *w, R *rese) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < (long)npnt * NV; q += (long)gridDim.x * blockDim.x) {
        const int v = (int)(q / NV), n = (int)(q % NV);
        const int b = vs_ptr[v], ns = vs_ptr[v + 1] - b;
        const R *a = fac + fptr[v];
        R x[SPK_MAX];
        for (int k = 0; k < ns; ++k) x[k] = w[((size_t)vs_seg[b + k] * 2 + vs_end[b + k]) * NV + n];
        for (int i = 1; i < ns; ++i) {
            R sacc = x[i];
            for (int j = 0; j < i; ++j) sacc -= a[(size_t)i * ns + j] * x[j];
            x[i] = sacc;
        }
        for (int i = ns - 1; i >= 0; --i) {
            R sacc = x[i];
            for (int j = i + 1; j < ns; ++j) sacc -= a[(size_t)i * ns + j] * x[j];
            x[i] = sacc / a[(size_t)i * ns + i];
        }
        for (int k = 0; k < ns; ++k) atomicAdd(rese + ((size_t)vs_seg[b + k] * em) * NV + n, x[k] / (R)2);
    }
}

// the spoke matrices (tet_hp::spoke): per vertex, summed over its ball with the tetrahedron's
// iprcn(tind, 0): mdiag on the diagonal of each of its three edges at the vertex, odiag
// between them; LU-factored in place (no row exchanges), one thread per vertex. err counts
// vertices with a pivot that is not positive.
__global__ void k_tet_spoke_factor(int npnt, const int *vs_ptr, const int *vt_ptr, const int *vt_tet, const int *vt_spk,
                                   const double *iprcn, double mdiag, double odiag, const long long *fptr, double *fac,
                                   int *err) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < npnt; v += gridDim.x * blockDim.x) {
        const int ns = vs_ptr[v + 1] - vs_ptr[v];
        double *a = fac + fptr[v];
        for (int k = 0; k < ns * ns; ++k) a[k] = 0.0;
        for (int b = vt_ptr[v]; b < vt_ptr[v + 1]; ++b) {
            const double jcb = iprcn[(size_t)vt_tet[b] * NV];
            const int *e0 = vt_spk + 3 * b;
            for (int j = 0; j < 3; ++j) {
                a[e0[j] * ns + e0[j]] += jcb * mdiag;
                for (int k = 0; k < 3; ++k)
                    if (k != j) a[e0[j] * ns + e0[k]] += jcb * odiag;
            }
        }
        bool ok = true;
        for (int k = 0; k < ns; ++k) {
            const double piv = a[k * ns + k];
            ok = ok && piv > 0.0;
            for (int i = k + 1; i < ns; ++i) {
                const double l = a[i * ns + k] / piv;
                a[i * ns + k] = l;
                for (int j = k + 1; j < ns; ++j) a[i * ns + j] -= l * a[k * ns + j];
            }
        }
        if (!ok) atomicAdd(err, 1);
    }
}

// res *= (1 / prcn(entity, var)) diag on mode `mode` of a section with `modes` per entity, fixed rows zeroed
template <typename R>
__global__ void k_tet_minv_scale_mode(long nent, int modes, int mode, R *res, const R *prcn, R diag,
                                      const unsigned char *mask) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nent * NV; k += (long)gridDim.x * blockDim.x) {
        const long ent = k / NV, var = k % NV, idx = (ent * modes + mode) * NV + var;
        res[idx] = mask[idx] ? (R)0 : res[idx] * (((R)1 / prcn[ent * NV + var]) * diag);
    }
}

// ug = ug0 - ca res
template <typename R>
__global__ void k_tet_advance(long n, const R *res, R *u, const R *u0, R ca) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        u[k] = u0[k] - ca * res[k];
}

template <typename R>
__global__ void k_tet_relax(long n, R *res, const R *jd, const unsigned char *mask, R *u, const R *u0, R ca) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const R r = mask[k] ? (R)0 : (R)0.5 * res[k] / jd[k];
        res[k] = r;
        u[k] = u0[k] - ca * r;
    }
}

// per-block sums of squares of the unmasked residual entries (fixed grid: deterministic)
template <typename R>
__global__ void k_tet_sq(long n, const R *res, const unsigned char *mask, double *part) {
    __shared__ double sh[256];
    double s = 0.0;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        if (!mask[k]) s += (double)res[k] * (double)res[k];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// ---- multigrid transfers (tet_hp/mg_restrict.cpp, mg_prolongate.cpp) ----
// p-levels share the mesh: coarse entry c is fine entry map[c] (mode truncation)
template <typename R>
__global__ void k_tet_p_restrict(long n, const int *map, const R *fu, const R *fres, R *u, R *uf, R *res0) {
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const R v = fu[map[c]];
        u[c] = v;
        uf[c] = v;
        res0[c] = fres[map[c]];
    }
}
template <typename R>
__global__ void k_tet_p_prolong(long n, const int *map, const R *u, const R *uf, R *fu) {
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x)
        fu[map[c]] += u[c] - uf[c];
}
// h-levels at p = 1: vertex values, each point in a tetrahedron of the other mesh
template <typename R>
__global__ void k_tet_h_restrict_state(int ncp, const int *tet, const double *w, const int *ftp, const R *fu, R *u,
                                       R *uf) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < ncp; v += gridDim.x * blockDim.x)
        for (int n = 0; n < NV; ++n) {
            double s = 0.0;
            for (int j = 0; j < 4; ++j) s += w[4 * v + j] * (double)fu[(size_t)ftp[4 * tet[v] + j] * NV + n];
            u[(size_t)v * NV + n] = (R)s;
            uf[(size_t)v * NV + n] = (R)s;
        }
}
template <typename R>
__global__ void k_tet_h_restrict_res(int nfp, const int *tet, const double *w, const int *ctp, const R *fres,
                                     R *res0) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nfp; v += gridDim.x * blockDim.x)
        for (int j = 0; j < 4; ++j)
            for (int n = 0; n < NV; ++n)
                atomicAdd(res0 + (size_t)ctp[4 * tet[v] + j] * NV + n, (R)(w[4 * v + j] * fres[(size_t)v * NV + n]));
}
template <typename R>
__global__ void k_tet_h_prolong(int nfp, const int *tet, const double *w, const int *ctp, const R *u, const R *uf,
                                R *fu) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nfp; v += gridDim.x * blockDim.x)
        for (int n = 0; n < NV; ++n) {
            double s = 0.0;
            for (int j = 0; j < 4; ++j) {
                const size_t c = (size_t)ctp[4 * tet[v] + j] * NV + n;
                s += w[4 * v + j] * (double)(u[c] - uf[c]);
            }
            fu[(size_t)v * NV + n] += (R)s;
        }
}
// FAS driving term (tet_hp::rsdl, update.cpp:97-117): on the first residual after a
// restriction dres = fadd res0 - res; every coarse residual then adds dres
template <typename R>
__global__ void k_tet_fas(long n, R *res, const R *res0, R *dres, R fadd, int first) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        if (first) dres[k] = fadd * res0[k] - res[k];
        res[k] += dres[k];
    }
}

#include "hp_tet_mixed.cuh"

// Inputs of the learned correction per tetrahedron (17, the widths of include/hp_mlp.h):
// per variable (u, v, w, p) the mean and the range of its four vertex values and the rms
// of its edge, face and interior modes (12); log volume, log longest edge, longest edge^3
// / volume, log(1 + cell Peclet number of the vertex velocities) (4); p / 4.
__global__ void k_tet_elem_features(TetMeshD mesh, TetFields<double> u, int p, int em, int fm, int im, double nu,
                                    float *feat) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mesh.ntet) return;
    float *f = feat + (size_t)t * 17;
    const int *v = mesh.tp + 4 * t;
    double vmax = 0.0;
    for (int n = 0; n < NV; ++n) {
        double sum = 0.0, mx = -1e300, mn = 1e300;
        for (int j = 0; j < 4; ++j) {
            const double x = u.v[(size_t)v[j] * NV + n];
            sum += x;
            mx = fmax(mx, x);
            mn = fmin(mn, x);
        }
        double ss = 0.0;
        int cnt = 0;
        for (int i = 0; i < 6 && em > 0; ++i)
            for (int k = 0; k < em; ++k, ++cnt) {
                const double x = u.e[((size_t)mesh.ts[6 * t + i] * em + k) * NV + n];
                ss += x * x;
            }
        for (int i = 0; i < 4 && fm > 0; ++i)
            for (int k = 0; k < fm; ++k, ++cnt) {
                const double x = u.f[((size_t)mesh.tt[4 * t + i] * fm + k) * NV + n];
                ss += x * x;
            }
        for (int k = 0; k < im; ++k, ++cnt) {
            const double x = u.i[((size_t)t * im + k) * NV + n];
            ss += x * x;
        }
        f[3 * n] = (float)(sum / 4.0);
        f[3 * n + 1] = (float)(mx - mn);
        f[3 * n + 2] = (float)(cnt > 0 ? sqrt(ss / cnt) : 0.0);
    }
    for (int j = 0; j < 4; ++j) {
        const double *uu = u.v + (size_t)v[j] * NV;
        vmax = fmax(vmax, sqrt(uu[0] * uu[0] + uu[1] * uu[1] + uu[2] * uu[2]));
    }
    double h2 = 0.0;
    for (int a = 0; a < 4; ++a)
        for (int b = a + 1; b < 4; ++b) {
            double d2 = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double d = mesh.pnts[3 * v[a] + k] - mesh.pnts[3 * v[b] + k];
                d2 += d * d;
            }
            h2 = fmax(h2, d2);
        }
    const double vol = fabs(mesh.vol[t]) / 6.0 + 1e-300, h = sqrt(h2);
    f[12] = (float)log(vol);
    f[13] = (float)log(h + 1e-300);
    f[14] = (float)(h * h2 / vol);
    f[15] = (float)log1p(vmax * h / (nu > 0 ? nu : 1e-300));
    f[16] = (float)p / 4.0f;
}

// Sum of squares of a tetrahedron's own residual coefficients (vertex, edge, face, interior).
template <int P>
__global__ void k_tet_elem_resnorm(TetMeshD mesh, TetFields<double> res, double *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mesh.ntet) return;
    double s2 = 0.0;
    for (int m = 0; m < TetCfg<P>::T; ++m)
        for (int n = 0; n < NV; ++n) {
            double sg;
            const double x = *mode_slot<double, P>(mesh, res, t, m, n, sg);
            s2 += x * x;
        }
    out[t] = s2;
}

int nblk(long n, int b) { return (int)std::max<long>(1, (n + b - 1) / b); }

}  // namespace

struct hp_tet_ctx {
    int device = 0, nsm = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int p = 0, em = 0, fm = 0, im = 0, T = 0, Q = 0;
    hp_phys_params ph{};
    TetMeshD mesh{};
    size_t lv = 0, le = 0, lf = 0, li = 0, ltot = 0;  // section lengths (values)
    std::vector<void *> allocs;
    double *U = nullptr, *RES = nullptr, *RR = nullptr;  // [v | e | f | i]
    double *tau = nullptr, *iprcn = nullptr, *vprcn = nullptr, *eprcn = nullptr, *fprcn = nullptr;
    int *d_err = nullptr;
    double *projB = nullptr, *intB = nullptr;  // the same operators in DMMA fragment order
    double *U0 = nullptr, *JD = nullptr, *rbar = nullptr, *part = nullptr;  // update, jacob_diag
    unsigned char *mask = nullptr;  // 1: row fixed by an essential condition
    bool jd_ready = false;
    int smoother = 0;  // 0: JACOBI build (jacobi_relaxation), 1: minvrt (p <= 2)
    int *seg_pnt = nullptr;           // [nseg][2] edge end points (global direction)
    double *d_mm = nullptr, *d_sfmv = nullptr;  // lumpinv tables for minvrt
    // minvrt at p = 3: face vertices / edges [ntri][3]; per vertex its spokes (edge, end) in
    // ball order (vs_*), its ball's tetrahedra with their three spokes (vt_*), the offsets of
    // its LU factor (fptr) and the factors; the spoke values scratch [nseg][2][NV]
    int *tri_pnt = nullptr, *tri_seg = nullptr, *vs_ptr = nullptr, *vs_seg = nullptr, *vs_end = nullptr;
    int *vt_ptr = nullptr, *vt_tet = nullptr, *vt_spk = nullptr;
    long long *fptr = nullptr;
    long long nfac = 0;
    int max_spk = 0;
    double *fac = nullptr, *spk_w = nullptr, *d_ffmv = nullptr, *d_ffms = nullptr;
    bool smoother_ready() const { return smoother ? prcn_ready : jd_ready; }
    // multigrid: this level is coarser than `fine` (kind 1: p-level, 2: h-level)
    hp_tet_ctx *fine = nullptr;
    int kind = 0;
    double fadd = 1.0;
    bool fas_pending = false;
    int *pmap = nullptr;                    // p-level: fine index of every coarse entry
    int *c2f_tet = nullptr, *f2c_tet = nullptr;
    double *c2f_w = nullptr, *f2c_w = nullptr;
    double *RES0 = nullptr, *DRES = nullptr, *UF = nullptr;
    hp_tet_tables tab{};
    bool prcn_ready = false;
    double *ftab = nullptr;  // face operators F2, DX2, DY2, W2
    TetFacesD faces{};       // boundary faces with a flux (device arrays below)
    int *face_int = nullptr;
    double *face_pbc = nullptr;
    TetFields<double> fields(double *base) const {
        return TetFields<double>{base, base + lv, base + lv + le, base + lv + le + lf};
    }
    // FP32 smoother of the mixed-precision solve (hp_tet_solve_mg_mixed): the correction d
    // (U), its stage copy, residuals, the base state and its point values, the FP32 copies
    // of the preconditioner (tau, Jacobian diagonal, minvrt's), the source DRES (the FP64
    // defect on the finest level, the FAS term below), the restricted residual and the
    // entry correction of a coarse level, and the TF32 operators
    struct Mixed {
        float *U = nullptr, *U0 = nullptr, *RES = nullptr, *RR = nullptr, *UB = nullptr, *DRES = nullptr;
        float *JD = nullptr, *BPT = nullptr, *TAU = nullptr, *RES0 = nullptr, *UF = nullptr;
        float *vprcn = nullptr, *eprcn = nullptr, *iprcn = nullptr, *mm = nullptr, *sfmv = nullptr;
        float *fprcn = nullptr, *ffmv = nullptr, *ffms = nullptr, *fac = nullptr, *spk_w = nullptr;
        float2 *projB = nullptr, *intB = nullptr;
        float *F = nullptr;
        bool fas_pending = false;
    } mx;
    bool mixed_ready = false;
    // learned correction: a per-tetrahedron log-scale of its contributions to the Jacobian
    // diagonal (JACOBI smoother) and to minvrt's preconditioner, from a network or given
    const float *lsc = nullptr;
    float lsc_clamp = 0.f;
    hp_mlp *net = nullptr;
    float *d_feat = nullptr, *d_netout = nullptr;
    TetFields<float> fields32(float *base) const {
        return TetFields<float>{base, base + lv, base + lv + le, base + lv + le + lf};
    }
};

namespace {

int talloc(hp_tet_ctx *c, void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        set_err("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return HP_ECUDA;
    }
    c->allocs.push_back(*p);
    return HP_OK;
}

// DMMA B fragments (lane = 4 * group + column): projection B[k = mode][n = point]
// = Op(q, m) at [op][nt][ks][lane]; intgrtrst B[k = (c, q)][n = mode] = w(q) Dc(q, m)
// at [nt][ks][lane]; zero beyond T, Q, 3Q.
template <int P>
void tet_fragments(const hp_tet_tables &b, std::vector<double> &proj, std::vector<double> &intg) {
    using C = TetCfg<P>;
    using M = TetMma<P>;
    proj.assign(M::PROJ_LEN, 0.0);
    intg.assign(M::INT_LEN, 0.0);
    const double(*ops[4])[HP_TET_MAXT] = {b.F, b.DX, b.DY, b.DZ};
    for (int op = 0; op < 4; ++op)
        for (int nt = 0; nt < M::NT; ++nt)
            for (int ks = 0; ks < M::KS; ++ks)
                for (int lane = 0; lane < 32; ++lane) {
                    const int q = nt * 8 + (lane >> 2), m = ks * 4 + (lane & 3);
                    if (q < C::Q && m < C::T)
                        proj[(((size_t)op * M::NT + nt) * M::KS + ks) * 32 + lane] = ops[op][q][m];
                }
    for (int nt = 0; nt < M::NT2; ++nt)
        for (int ks = 0; ks < M::KS2; ++ks)
            for (int lane = 0; lane < 32; ++lane) {
                const int k = ks * 4 + (lane & 3), m = nt * 8 + (lane >> 2);
                if (k >= 3 * C::Q || m >= C::T) continue;
                const int c = k / C::Q, q = k - c * C::Q;
                intg[((size_t)nt * M::KS2 + ks) * 32 + lane] = b.w[q] * ops[1 + c][q][m];
            }
}

// dynamic shared memory above 48 KB for every instantiation, once per process
template <int P>
int ensure_attrs() {
    using M = TetMma<P>;
    static bool done = false;
    if (done) return HP_OK;
    TCK(cudaFuncSetAttribute(k_tet_rsdl_mma<P, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::SMEM));
    TCK(cudaFuncSetAttribute(k_tet_rsdl_mma<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::SMEM));
    TCK(cudaFuncSetAttribute(k_tet_rsdl_mma<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::SMEM));
    done = true;
    return HP_OK;
}

template <int P>
int launch_rsdl(hp_tet_ctx *c, int stage) {
    TetSmall<double, P> sm;
    const hp_tet_tables &t = c->tab;
    for (int i = 0; i <= P; ++i) {
        for (int j = 0; j <= P; ++j) {
            sm.Ax[i][j] = t.Ax[i][j];
            sm.Bx[i][j] = t.Bx[i][j];
            sm.Ay[i][j] = t.Ay[i][j];
            sm.By[i][j] = t.By[i][j];
            sm.Az[i][j] = t.Az[i][j];
        }
        sm.y0[i] = t.y0[i];
        sm.z0[i] = t.z0[i];
    }
    const double omb = stage >= c->ph.nstage ? 0.0 : 1.0 - c->ph.beta[stage];
    const double beta = c->ph.beta[stage];
    k_tet_pre<double><<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>((long)c->ltot, c->RES,
                                                                                           c->RR, omb);
    if (c->faces.n > 0)
        k_tet_face_flux<P><<<std::min(nblk(c->faces.n, 4), c->nsm * 16), 128, 0, c->stream>>>(
            c->faces, c->ftab, c->mesh, c->fields(c->U), c->fields(c->RES), c->ph.rho);
    using M = TetMma<P>;
    const size_t smem2 = (size_t)M::S_WARP * M::WPC * sizeof(double);
    if (int r = ensure_attrs<P>()) return r;
    const long npair = ((long)c->mesh.ntet + 1) / 2;
    int blocks = std::min(nblk(npair, M::WPC), c->nsm * 32);
    k_tet_rsdl_mma<P, 0><<<blocks, M::WPC * 32, smem2, c->stream>>>(
        c->projB, c->intB, sm, c->mesh, c->fields(c->U), c->fields(c->RES), c->fields(c->RR), c->tau, c->ph.rho,
        c->ph.mu, beta, nullptr, TetFields<double>{}, nullptr, 0.f);
    k_tet_fold<double><<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>((long)c->ltot, c->RES,
                                                                                            c->RR);
    if (c->fine) {
        k_tet_fas<<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
            (long)c->ltot, c->RES, c->RES0, c->DRES, c->fadd, c->fas_pending ? 1 : 0);
        c->fas_pending = false;
    }
    TCK(cudaGetLastError());
    return HP_OK;
}

template <int P>
int launch_jacdiag(hp_tet_ctx *c) {
    using C = TetCfg<P>;
    using M = TetMma<P>;
    int r = ensure_attrs<P>();
    if (r) return r;
    TetSmall<double, P> sm;
    const hp_tet_tables &t = c->tab;
    for (int i = 0; i <= P; ++i) {
        for (int j = 0; j <= P; ++j) {
            sm.Ax[i][j] = t.Ax[i][j];
            sm.Bx[i][j] = t.Bx[i][j];
            sm.Ay[i][j] = t.Ay[i][j];
            sm.By[i][j] = t.By[i][j];
            sm.Az[i][j] = t.Az[i][j];
        }
        sm.y0[i] = t.y0[i];
        sm.z0[i] = t.z0[i];
    }
    const double beta0 = c->ph.beta[0];
    const long n1 = ((long)c->mesh.ntet + 1) / 2, n2 = ((long)c->mesh.ntet * NV * C::T + 1) / 2;
    k_tet_rsdl_mma<P, 1><<<std::min(nblk(n1, M::WPC), c->nsm * 32), M::WPC * 32, M::SMEM, c->stream>>>(
        c->projB, c->intB, sm, c->mesh, c->fields(c->U), c->fields(c->RES), c->fields(c->RR), c->tau, c->ph.rho,
        c->ph.mu, beta0, c->rbar, c->fields(c->JD), nullptr, 0.f);
    TCK(cudaMemsetAsync(c->JD, 0, 8 * c->ltot, c->stream));
    k_tet_rsdl_mma<P, 2><<<std::min(nblk(n2, M::WPC), c->nsm * 32), M::WPC * 32, M::SMEM, c->stream>>>(
        c->projB, c->intB, sm, c->mesh, c->fields(c->U), c->fields(c->RES), c->fields(c->RR), c->tau, c->ph.rho,
        c->ph.mu, beta0, c->rbar, c->fields(c->JD), c->lsc, c->lsc_clamp);
    TCK(cudaGetLastError());
    return HP_OK;
}

}  // namespace

extern "C" const char *hp_tet_last_error(void) { return g_err.c_str(); }

// The mesh data of minvrt at p = 3. Faces: the vertices of the tetrahedron that numbered the
// face (rot = +1), in its order VF of that face (tet_mesh::create_tri_from_tet,
// tet_mesh/setup.cpp:301-374); face edge i is the edge opposite face vertex i. Vertex balls:
// the tetrahedra at a vertex by index, the vertex's edges numbered in the order the ball's
// tetrahedra (local edges 0..5) first meet them (tet_hp::spoke, setup_preconditioner.cpp:530-561).
static int spoke_topology(hp_tet_ctx *c, const hp_tet_mesh_desc *m, const std::vector<int> &sp) {
    static const int VF[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};
    static const int VS[6][2] = {{2, 3}, {3, 1}, {2, 1}, {1, 0}, {2, 0}, {3, 0}};
    const int npnt = m->npnt, ntet = m->ntet, ntri = m->ntri;
    std::vector<int> fp(3 * (size_t)ntri, -1), fs(3 * (size_t)ntri, -1);
    for (int t = 0; t < ntet; ++t)
        for (int i = 0; i < 4; ++i) {
            if (m->tet_rot[4 * t + i] < 0) continue;
            const int f = m->tet_tri[4 * t + i];
            if (f < 0 || f >= ntri) { set_err("hp_tet_create: tet_tri out of range"); return HP_EINVAL; }
            for (int j = 0; j < 3; ++j) fp[3 * (size_t)f + j] = m->tet_pnt[4 * t + VF[i][j]];
            for (int j = 0; j < 3; ++j) {
                const int a = VF[i][(j + 1) % 3], bb = VF[i][(j + 2) % 3];
                for (int e = 0; e < 6; ++e)
                    if ((VS[e][0] == a && VS[e][1] == bb) || (VS[e][0] == bb && VS[e][1] == a))
                        fs[3 * (size_t)f + j] = m->tet_seg[6 * t + e];
            }
        }
    for (size_t k = 0; k < fp.size(); ++k)
        if (fp[k] < 0 || fs[k] < 0) {
            set_err("hp_tet_create: face %zu is numbered by no tetrahedron (tet_rot +1)", k / 3);
            return HP_EINVAL;
        }
    std::vector<int> vt_ptr(npnt + 1, 0), vt_tet(4 * (size_t)ntet);
    for (int t = 0; t < ntet; ++t)
        for (int j = 0; j < 4; ++j) ++vt_ptr[m->tet_pnt[4 * t + j] + 1];
    for (int v = 0; v < npnt; ++v) vt_ptr[v + 1] += vt_ptr[v];
    {
        std::vector<int> fill(vt_ptr.begin(), vt_ptr.end() - 1);
        for (int t = 0; t < ntet; ++t)
            for (int j = 0; j < 4; ++j) vt_tet[fill[m->tet_pnt[4 * t + j]]++] = t;
    }
    std::vector<int> vs_ptr(npnt + 1, 0), vs_seg, vs_end, vt_spk(3 * (size_t)4 * ntet);
    std::vector<long long> fptr(npnt + 1, 0);
    std::vector<int> local(m->nseg, -1);
    int max_spk = 0;
    for (int v = 0; v < npnt; ++v) {
        const int base = (int)vs_seg.size();
        for (int b = vt_ptr[v]; b < vt_ptr[v + 1]; ++b) {
            const int t = vt_tet[b];
            int ind2 = 0;
            for (int j = 0; j < 6; ++j) {
                const int sidx = m->tet_seg[6 * t + j];
                for (int k = 0; k < 2; ++k)
                    if (sp[2 * (size_t)sidx + k] == v) {
                        if (local[sidx] < 0) {
                            local[sidx] = (int)vs_seg.size() - base;
                            vs_seg.push_back(sidx);
                            vs_end.push_back(k);
                        }
                        if (ind2 < 3) vt_spk[3 * (size_t)b + ind2] = local[sidx];
                        ++ind2;
                    }
            }
            if (ind2 != 3) { set_err("hp_tet_create: tetrahedron %d does not have three edges at its vertex %d", t, v); return HP_EINVAL; }
        }
        const int ns = (int)vs_seg.size() - base;
        max_spk = std::max(max_spk, ns);
        vs_ptr[v + 1] = (int)vs_seg.size();
        fptr[v + 1] = fptr[v] + (long long)ns * ns;
        for (int k = base; k < (int)vs_seg.size(); ++k) local[vs_seg[k]] = -1;
    }
    c->max_spk = max_spk;
    c->nfac = fptr[npnt];
    int r;
    auto up = [&](const void *src, size_t bytes, void **dst) -> int {
        if ((r = talloc(c, dst, bytes))) return r;
        if (bytes) TCK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        return HP_OK;
    };
    if ((r = up(fp.data(), 4 * fp.size(), (void **)&c->tri_pnt)) || (r = up(fs.data(), 4 * fs.size(), (void **)&c->tri_seg)) ||
        (r = up(vs_ptr.data(), 4 * vs_ptr.size(), (void **)&c->vs_ptr)) ||
        (r = up(vs_seg.data(), 4 * vs_seg.size(), (void **)&c->vs_seg)) ||
        (r = up(vs_end.data(), 4 * vs_end.size(), (void **)&c->vs_end)) ||
        (r = up(vt_ptr.data(), 4 * vt_ptr.size(), (void **)&c->vt_ptr)) ||
        (r = up(vt_tet.data(), 4 * vt_tet.size(), (void **)&c->vt_tet)) ||
        (r = up(vt_spk.data(), 4 * vt_spk.size(), (void **)&c->vt_spk)) ||
        (r = up(fptr.data(), 8 * fptr.size(), (void **)&c->fptr)) ||
        (r = up(&c->tab.ffmv[0][0], sizeof(c->tab.ffmv), (void **)&c->d_ffmv)) ||
        (r = up(&c->tab.ffms[0][0][0], sizeof(c->tab.ffms), (void **)&c->d_ffms)))
        return r;
    return HP_OK;
}

extern "C" int hp_tet_create(const hp_tet_mesh_desc *m, const hp_tet_tables *b, const hp_phys_params *ph, int device,
                             void *stream, hp_tet_ctx **out) {
    if (!m || !b || !ph || !out || b->p < 1 || b->p > HP_TET_MAXP || m->ntet < 1) {
        set_err("hp_tet_create: bad arguments");
        return HP_EINVAL;
    }
    if (ph->physics != HP_PHYS_INS || ph->nstage < 1 || ph->nstage > 7) {
        set_err("hp_tet_create: ins physics with 1..7 stages only");
        return HP_EINVAL;
    }
    auto *c = new hp_tet_ctx;
    if (device >= 0) TCK(cudaSetDevice(device));
    TCK(cudaGetDevice(&c->device));
    TCK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
    if (stream) c->stream = (cudaStream_t)stream;
    else {
        TCK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    c->tab = *b;
    c->p = b->p; c->em = b->em; c->fm = b->fm; c->im = b->im; c->T = b->T; c->Q = b->G * b->G * b->G;
    c->ph = *ph;
    c->lv = (size_t)m->npnt * NV; c->le = (size_t)m->nseg * c->em * NV;
    c->lf = (size_t)m->ntri * c->fm * NV; c->li = (size_t)m->ntet * c->im * NV;
    c->ltot = c->lv + c->le + c->lf + c->li;
    int r;
    void *p;
    auto up = [&](const void *src, size_t bytes, void **dst) -> int {
        if ((r = talloc(c, dst, bytes))) return r;
        if (bytes) TCK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        return HP_OK;
    };
    TetMeshD &md = c->mesh;
    md.npnt = m->npnt; md.nseg = m->nseg; md.ntri = m->ntri; md.ntet = m->ntet;
    if ((r = up(m->pnts, 24 * (size_t)m->npnt, &p))) { hp_tet_destroy(c); return r; }
    md.pnts = (const double *)p;
    if ((r = up(m->vol, 8 * (size_t)m->ntet, &p))) { hp_tet_destroy(c); return r; }
    md.vol = (const double *)p;
    if ((r = up(m->tet_pnt, 16 * (size_t)m->ntet, &p))) { hp_tet_destroy(c); return r; }
    md.tp = (const int *)p;
    if ((r = up(m->tet_seg, 24 * (size_t)m->ntet, &p))) { hp_tet_destroy(c); return r; }
    md.ts = (const int *)p;
    if ((r = up(m->tet_sgn, 24 * (size_t)m->ntet, &p))) { hp_tet_destroy(c); return r; }
    md.tsg = (const int *)p;
    if ((r = up(m->tet_tri, 16 * (size_t)m->ntet, &p))) { hp_tet_destroy(c); return r; }
    md.tt = (const int *)p;
    if ((r = up(m->tet_rot, 16 * (size_t)m->ntet, &p))) { hp_tet_destroy(c); return r; }
    md.trot = (const int *)p;
    for (double **f : {&c->U, &c->RES, &c->RR}) {
        if ((r = talloc(c, (void **)f, 8 * c->ltot))) { hp_tet_destroy(c); return r; }
        TCK(cudaMemset(*f, 0, 8 * c->ltot));
    }
    if ((r = talloc(c, (void **)&c->tau, 16 * (size_t)m->ntet)) ||
        (r = talloc(c, (void **)&c->iprcn, 32 * (size_t)m->ntet)) ||
        (r = talloc(c, (void **)&c->vprcn, 32 * (size_t)m->npnt)) ||
        (r = talloc(c, (void **)&c->eprcn, 32 * (size_t)m->nseg)) ||
        (r = talloc(c, (void **)&c->fprcn, 32 * (size_t)m->ntri)) || (r = talloc(c, (void **)&c->d_err, 16))) {
        hp_tet_destroy(c);
        return r;
    }
    TCK(cudaMemset(c->tau, 0, 16 * (size_t)m->ntet));
    {
        const int G2 = b->G * b->G, T2 = b->T2;
        std::vector<double> ft((size_t)3 * G2 * T2 + G2);
        for (int q = 0; q < G2; ++q) {
            for (int k = 0; k < T2; ++k) {
                ft[(size_t)q * T2 + k] = b->F2[q][k];
                ft[(size_t)(G2 + q) * T2 + k] = b->DX2[q][k];
                ft[(size_t)(2 * G2 + q) * T2 + k] = b->DY2[q][k];
            }
            ft[(size_t)3 * G2 * T2 + q] = b->W2[q];
        }
        if ((r = up(ft.data(), 8 * ft.size(), (void **)&c->ftab))) { hp_tet_destroy(c); return r; }
    }
    {
        std::vector<double> pb, ib;
        switch (c->p) {
            case 1: tet_fragments<1>(*b, pb, ib); break;
            case 2: tet_fragments<2>(*b, pb, ib); break;
            case 3: tet_fragments<3>(*b, pb, ib); break;
            case 4: tet_fragments<4>(*b, pb, ib); break;
        }
        if ((r = up(pb.data(), 8 * pb.size(), (void **)&c->projB)) ||
            (r = up(ib.data(), 8 * ib.size(), (void **)&c->intB))) {
            hp_tet_destroy(c);
            return r;
        }
    }
    {   // edge end points in the global direction (tet_sgn = +1 where the tetrahedron's local
        // edge runs from its first to its second local vertex the same way) and lumpinv tables
        static const int VS[6][2] = {{2, 3}, {3, 1}, {2, 1}, {1, 0}, {2, 0}, {3, 0}};
        std::vector<int> sp(2 * (size_t)m->nseg, -1);
        for (int t = 0; t < m->ntet; ++t)
            for (int i = 0; i < 6; ++i) {
                const int sidx = m->tet_seg[6 * t + i];
                if (sidx < 0 || sidx >= m->nseg) { set_err("hp_tet_create: tet_seg out of range"); hp_tet_destroy(c); return HP_EINVAL; }
                const int a = m->tet_pnt[4 * t + VS[i][0]], bb = m->tet_pnt[4 * t + VS[i][1]];
                sp[2 * (size_t)sidx] = m->tet_sgn[6 * t + i] > 0 ? a : bb;
                sp[2 * (size_t)sidx + 1] = m->tet_sgn[6 * t + i] > 0 ? bb : a;
            }
        if ((r = up(sp.data(), 4 * sp.size(), (void **)&c->seg_pnt)) ||
            (r = up(&b->mm[0][0], sizeof(b->mm), (void **)&c->d_mm)) ||
            (r = up(&b->sfmv[0][0], sizeof(b->sfmv), (void **)&c->d_sfmv))) {
            hp_tet_destroy(c);
            return r;
        }
        if (c->p == 3 && (r = spoke_topology(c, m, sp))) {
            hp_tet_destroy(c);
            return r;
        }
    }
    if ((r = talloc(c, (void **)&c->U0, 8 * c->ltot)) || (r = talloc(c, (void **)&c->JD, 8 * c->ltot)) ||
        (r = talloc(c, (void **)&c->mask, c->ltot)) || (r = talloc(c, (void **)&c->part, 8 * 1024))) {
        hp_tet_destroy(c);
        return r;
    }
    TCK(cudaMemset(c->mask, 0, c->ltot));
    *out = c;
    return HP_OK;
}

extern "C" int hp_tet_set_flux_faces(hp_tet_ctx *c, int nface, const int *face_tri, const int *face_pnt,
                                     const int *face_seg, const int *face_sgn, const int *kind, const double *pbc) {
    if (!c || nface < 0 || (nface > 0 && (!face_tri || !face_pnt || !face_seg || !face_sgn || !kind))) {
        set_err("hp_tet_set_flux_faces: bad arguments");
        return HP_EINVAL;
    }
    const TetMeshD &m = c->mesh;
    bool any_neumann = false;
    for (int b = 0; b < nface; ++b) {
        bool ok = face_tri[b] >= 0 && face_tri[b] < m.ntri && (kind[b] == 0 || kind[b] == 1);
        for (int i = 0; i < 3; ++i)
            ok = ok && face_pnt[3 * b + i] >= 0 && face_pnt[3 * b + i] < m.npnt && face_seg[3 * b + i] >= 0 &&
                 face_seg[3 * b + i] < m.nseg && (face_sgn[3 * b + i] == 1 || face_sgn[3 * b + i] == -1);
        if (!ok) {
            set_err("hp_tet_set_flux_faces: face %d has an index out of range or a bad sign / kind", b);
            return HP_EINVAL;
        }
        any_neumann = any_neumann || kind[b] == 1;
    }
    if (any_neumann && !pbc) {
        set_err("hp_tet_set_flux_faces: neumann faces need pbc");
        return HP_EINVAL;
    }
    TCK(cudaSetDevice(c->device));
    TCK(cudaStreamSynchronize(c->stream));
    if (c->face_int) cudaFree(c->face_int);
    if (c->face_pbc) cudaFree(c->face_pbc);
    c->face_int = nullptr;
    c->face_pbc = nullptr;
    c->faces = TetFacesD{};
    if (nface == 0) return HP_OK;
    const size_t G2 = (size_t)c->tab.G * c->tab.G;
    std::vector<int> h((size_t)11 * nface);
    std::copy(face_tri, face_tri + nface, h.begin());
    std::copy(face_pnt, face_pnt + 3 * (size_t)nface, h.begin() + nface);
    std::copy(face_seg, face_seg + 3 * (size_t)nface, h.begin() + 4 * (size_t)nface);
    std::copy(face_sgn, face_sgn + 3 * (size_t)nface, h.begin() + 7 * (size_t)nface);
    std::copy(kind, kind + nface, h.begin() + 10 * (size_t)nface);
    std::vector<double> hp(G2 * nface, 0.0);
    if (pbc) std::copy(pbc, pbc + G2 * nface, hp.begin());
    TCK(cudaMalloc((void **)&c->face_int, 4 * h.size()));
    TCK(cudaMalloc((void **)&c->face_pbc, 8 * hp.size()));
    TCK(cudaMemcpy(c->face_int, h.data(), 4 * h.size(), cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(c->face_pbc, hp.data(), 8 * hp.size(), cudaMemcpyHostToDevice));
    const int *d = c->face_int;
    c->faces = TetFacesD{nface, d, d + nface, d + 4 * (size_t)nface, d + 7 * (size_t)nface, d + 10 * (size_t)nface,
                         c->face_pbc};
    return HP_OK;
}

extern "C" int hp_tet_destroy(hp_tet_ctx *c) {
    if (!c) return HP_EINVAL;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->face_int) cudaFree(c->face_int);
    if (c->face_pbc) cudaFree(c->face_pbc);
    for (void *p : c->allocs) cudaFree(p);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HP_OK;
}

extern "C" int hp_tet_sync(hp_tet_ctx *c) {
    if (!c) return HP_EINVAL;
    TCK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}

static int copy_fields(hp_tet_ctx *c, double *dev, const double *v, const double *e, const double *f, const double *i,
                       double *ov, double *oe, double *of, double *oi) {
    const size_t len[4] = {c->lv, c->le, c->lf, c->li};
    size_t off = 0;
    const double *src[4] = {v, e, f, i};
    double *dst[4] = {ov, oe, of, oi};
    for (int k = 0; k < 4; ++k) {
        if (len[k]) {
            if (src[k]) TCK(cudaMemcpyAsync(dev + off, src[k], 8 * len[k], cudaMemcpyHostToDevice, c->stream));
            if (dst[k]) TCK(cudaMemcpyAsync(dst[k], dev + off, 8 * len[k], cudaMemcpyDeviceToHost, c->stream));
        }
        off += len[k];
    }
    TCK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}

extern "C" int hp_tet_upload_state(hp_tet_ctx *c, const double *v, const double *e, const double *f, const double *i) {
    if (!c || !v) return HP_EINVAL;
    return copy_fields(c, c->U, v, e, f, i, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int hp_tet_download_state(hp_tet_ctx *c, double *v, double *e, double *f, double *i) {
    if (!c) return HP_EINVAL;
    return copy_fields(c, c->U, nullptr, nullptr, nullptr, nullptr, v, e, f, i);
}

extern "C" int hp_tet_download_residual(hp_tet_ctx *c, int which, double *v, double *e, double *f, double *i) {
    if (!c || which < 0 || which > 1) return HP_EINVAL;
    return copy_fields(c, which ? c->RR : c->RES, nullptr, nullptr, nullptr, nullptr, v, e, f, i);
}

static int tet_net_scale(hp_tet_ctx *c);

extern "C" int hp_tet_setup_preconditioner(hp_tet_ctx *c) {
    if (!c) return HP_EINVAL;
    if (c->net) {
        int r0 = tet_net_scale(c);
        if (r0) return r0;
    }
    TCK(cudaMemsetAsync(c->d_err, 0, 4, c->stream));
    TCK(cudaMemsetAsync(c->vprcn, 0, 32 * (size_t)c->mesh.npnt, c->stream));
    TCK(cudaMemsetAsync(c->eprcn, 0, 32 * (size_t)c->mesh.nseg, c->stream));
    TCK(cudaMemsetAsync(c->fprcn, 0, 32 * (size_t)c->mesh.ntri, c->stream));
    k_tet_prcn<<<std::min(nblk(c->mesh.ntet, 128), c->nsm * 16), 128, 0, c->stream>>>(
        c->mesh, c->U, c->tau, c->iprcn, c->vprcn, c->eprcn, c->fprcn, c->p, c->em, c->fm, c->ph.rho, c->ph.mu,
        c->ph.adis, c->ph.bd0, c->d_err, c->lsc, c->lsc_clamp);
    // minvrt at p = 3: the vertex-ball spoke factors from this iprcn (tet_hp::spoke)
    if (c->smoother == 1 && c->p == 3)
        k_tet_spoke_factor<<<nblk(c->mesh.npnt, 128), 128, 0, c->stream>>>(
            c->mesh.npnt, c->vs_ptr, c->vt_ptr, c->vt_tet, c->vt_spk, c->iprcn, c->tab.mdiag, c->tab.odiag, c->fptr,
            c->fac, c->d_err);
    TCK(cudaGetLastError());
    int herr = 0;
    TCK(cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream));
    TCK(cudaStreamSynchronize(c->stream));
    c->prcn_ready = true;
    return herr;
}

extern "C" int hp_tet_download_prcn(hp_tet_ctx *c, double *tau, double *iprcn) {
    if (!c || !tau || !iprcn) return HP_EINVAL;
    TCK(cudaMemcpyAsync(tau, c->tau, 16 * (size_t)c->mesh.ntet, cudaMemcpyDeviceToHost, c->stream));
    TCK(cudaMemcpyAsync(iprcn, c->iprcn, 32 * (size_t)c->mesh.ntet, cudaMemcpyDeviceToHost, c->stream));
    TCK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}

extern "C" int hp_tet_enqueue_rsdl(hp_tet_ctx *c, int stage) {
    if (!c || stage < 0 || stage > c->ph.nstage) return HP_EINVAL;
    if (c->ph.beta[stage] > 0.0 && !c->prcn_ready) {
        set_err("tet rsdl with beta > 0 needs tau from hp_tet_setup_preconditioner");
        return HP_ESTATE;
    }
    switch (c->p) {
        case 1: return launch_rsdl<1>(c, stage);
        case 2: return launch_rsdl<2>(c, stage);
        case 3: return launch_rsdl<3>(c, stage);
        case 4: return launch_rsdl<4>(c, stage);
    }
    return HP_EINVAL;
}

extern "C" int hp_tet_rsdl(hp_tet_ctx *c, int stage) {
    int r = hp_tet_enqueue_rsdl(c, stage);
    if (r) return r;
    return hp_tet_sync(c);
}

namespace {
// 8 independent accumulator pairs per warp; out keeps the compiler from dropping them
__global__ void k_dmma_peak(long iters, double *out) {
    double c[8][2];
    for (int g = 0; g < 8; ++g) c[g][0] = c[g][1] = 0.0;
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
    for (long it = 0; it < iters; ++it)
#pragma unroll
        for (int g = 0; g < 8; ++g) dmma(c[g][0], c[g][1], a, b);
    double s = 0.0;
    for (int g = 0; g < 8; ++g) s += c[g][0] + c[g][1];
    if (s == -1.0) out[0] = s;  // never true; keeps the chains live
}
}  // namespace

extern "C" int hp_tet_fp64_mma_peak(int device, double ms, double *tflops) {
    if (!tflops || ms <= 0) return HP_EINVAL;
    if (device >= 0) TCK(cudaSetDevice(device));
    int dev, nsm;
    TCK(cudaGetDevice(&dev));
    TCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double *out;
    TCK(cudaMalloc(&out, 8));
    cudaEvent_t e0, e1;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    const int blocks = nsm * 4, threads = 256;
    long iters = 1000;
    float el = 0.f;
    for (int tries = 0; tries < 12; ++tries) {
        TCK(cudaEventRecord(e0));
        k_dmma_peak<<<blocks, threads>>>(iters, out);
        TCK(cudaEventRecord(e1));
        TCK(cudaEventSynchronize(e1));
        TCK(cudaEventElapsedTime(&el, e0, e1));
        if (el >= ms) break;
        iters = (long)(iters * std::min(16.0, 1.2 * ms / std::max(el, 0.01f)));
    }
    const double mmas = (double)blocks * (threads / 32) * iters * 8;
    *tflops = mmas * 8 * 8 * 4 * 2 / (el * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return HP_OK;
}

extern "C" int hp_tet_set_dirichlet(hp_tet_ctx *c, const unsigned char *mv, const unsigned char *me,
                                    const unsigned char *mf) {
    if (!c || !mv) return HP_EINVAL;
    std::vector<unsigned char> h(c->ltot, 0);
    for (size_t k = 0; k < c->lv; ++k) h[k] = mv[k] ? 1 : 0;
    if (c->em && me)
        for (int e = 0; e < c->mesh.nseg; ++e)
            for (int m = 0; m < c->em; ++m)
                for (int n = 0; n < NV; ++n) h[c->lv + ((size_t)e * c->em + m) * NV + n] = me[(size_t)e * NV + n] ? 1 : 0;
    if (c->fm && mf)
        for (int f = 0; f < c->mesh.ntri; ++f)
            for (int m = 0; m < c->fm; ++m)
                for (int n = 0; n < NV; ++n)
                    h[c->lv + c->le + ((size_t)f * c->fm + m) * NV + n] = mf[(size_t)f * NV + n] ? 1 : 0;
    TCK(cudaMemcpyAsync(c->mask, h.data(), c->ltot, cudaMemcpyHostToDevice, c->stream));
    TCK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}

extern "C" int hp_tet_jacobian_diagonal(hp_tet_ctx *c) {
    if (!c) return HP_EINVAL;
    if (c->net) {
        int r0 = tet_net_scale(c);
        if (r0) return r0;
    }
    if (!c->prcn_ready) {
        set_err("hp_tet_jacobian_diagonal needs tau from hp_tet_setup_preconditioner");
        return HP_ESTATE;
    }
    if (!c->rbar) {
        int r = talloc(c, (void **)&c->rbar, 8 * (size_t)c->mesh.ntet * c->T * NV);
        if (r) return r;
    }
    int r = HP_EINVAL;
    switch (c->p) {
        case 1: r = launch_jacdiag<1>(c); break;
        case 2: r = launch_jacdiag<2>(c); break;
        case 3: r = launch_jacdiag<3>(c); break;
        case 4: r = launch_jacdiag<4>(c); break;
    }
    if (r) return r;
    TCK(cudaStreamSynchronize(c->stream));
    c->jd_ready = true;
    return HP_OK;
}

extern "C" int hp_tet_download_jacobian_diagonal(hp_tet_ctx *c, double *v, double *e, double *f, double *i) {
    if (!c || !c->jd_ready) return HP_ESTATE;
    return copy_fields(c, c->JD, nullptr, nullptr, nullptr, nullptr, v, e, f, i);
}

extern "C" int hp_tet_set_smoother(hp_tet_ctx *c, int kind) {
    if (!c || (kind != 0 && kind != 1)) {
        set_err("hp_tet_set_smoother: kind 0 (JACOBI build) or 1 (minvrt)");
        return HP_EINVAL;
    }
    if (kind == 1 && c->p > 3) {
        set_err("hp_tet_set_smoother: tet_hp::minvrt is built for p = 1, 2 and 3 only");
        return HP_EINVAL;
    }
    if (kind == 1 && c->p == 3 && !c->fac) {
        if (c->max_spk > SPK_MAX) {
            set_err("hp_tet_set_smoother: a vertex has %d edges; the vertex-ball solve takes at most %d", c->max_spk,
                    SPK_MAX);
            return HP_ENOTSUP;
        }
        int r;
        if ((r = talloc(c, (void **)&c->fac, 8 * (size_t)std::max<long long>(c->nfac, 1))) ||
            (r = talloc(c, (void **)&c->spk_w, 8 * (size_t)c->mesh.nseg * 2 * NV)))
            return r;
        c->prcn_ready = false;  // the spoke factors come with the next preconditioner set-up
    }
    c->smoother = kind;
    return HP_OK;
}

// tet_hp::minvrt at p = 3 (tet_hp/setup_preconditioner.cpp:16-354) on res, in either precision:
//  (1) edge and face modes removed from the vertices (sfmv, ffmv), the vertex rows scaled by
//      vdiag / vprcn and fixed;
//  (2) the vertex values times iprcn removed from the edge and face modes (mass matrix);
//  (3) the edges' first modes from the vertex-ball solves: per edge end the spoke value
//      e0 +- sfms(0) e1 plus the face modes times ffms, solved per vertex with its spoke
//      factor, half of each end's solution to the edge; fixed edges zeroed;
//  (4) the first edge modes times iprcn removed from the second edge modes and the faces, the
//      second edge modes scaled by ediag(1) / eprcn (ediag(1) = 1000 as minvrt sets it at
//      p = 3) and fixed;
//  (5) the second edge modes times iprcn removed from the faces (minvrt reads res.e(side, 1)
//      without the tetrahedron's edge sign there), the faces scaled by fdiag(0) / fprcn
//      (fdiag(0) = 3000) and fixed.
// The rows fixed by essential conditions are zeroed first, as tet_hp::update does.
template <typename R>
void enqueue_minvrt3(hp_tet_ctx *c, R *res, const R *vprcn, const R *eprcn, const R *fprcn, const R *iprcn,
                     const R *mm, const R *sfmv, const R *ffmv, const R *ffms, const R *fac, R *w) {
    const int g = c->nsm * 8, em = c->em, fm = c->fm;
    const TetMeshD &m = c->mesh;
    R *rv = res, *re = res + c->lv, *rf = res + c->lv + c->le;
    const unsigned char *mv = c->mask, *me = c->mask + c->lv, *mf = c->mask + c->lv + c->le;
    cudaStream_t st = c->stream;
    k_tet_zero_fixed<R><<<std::min(nblk((long)c->ltot, 256), g), 256, 0, st>>>((long)c->ltot, res, c->mask);
    k_tet_minv_e2v<R><<<std::min(nblk(m.nseg, 256), g), 256, 0, st>>>(m.nseg, em, c->seg_pnt, sfmv, rv, re, me);
    k_tet_minv_f2v<R><<<std::min(nblk(m.ntri, 256), g), 256, 0, st>>>(m.ntri, fm, c->tri_pnt, ffmv, rv, rf);
    k_tet_minv_scale<R><<<std::min(nblk((long)c->lv, 256), g), 256, 0, st>>>((long)c->lv, 1, rv, vprcn,
                                                                           (R)c->tab.vdiag, mv);
    k_tet_minv3_remove<R><<<std::min(nblk(m.ntet, 128), g), 128, 0, st>>>(m, em, fm, 0, mm, iprcn, rv, re, rf);
    k_tet_spoke_w<R><<<std::min(nblk(m.nseg, 256), g), 256, 0, st>>>(m.nseg, em, (R)c->tab.sfms0, re, w);
    k_tet_spoke_faces<R><<<std::min(nblk(m.ntri, 256), g), 256, 0, st>>>(m.ntri, fm, c->tri_pnt, c->tri_seg,
                                                                         c->seg_pnt, ffms, rf, w);
    k_tet_spoke_solve<R><<<std::min(nblk((long)m.npnt * NV, 128), g), 128, 0, st>>>(
        m.npnt, em, c->vs_ptr, c->vs_seg, c->vs_end, c->fptr, fac, w, re);
    k_tet_zero_fixed<R><<<std::min(nblk((long)c->le, 256), g), 256, 0, st>>>((long)c->le, re, me);
    k_tet_minv3_remove<R><<<std::min(nblk(m.ntet, 128), g), 128, 0, st>>>(m, em, fm, 1, mm, iprcn, rv, re, rf);
    k_tet_minv_scale_mode<R><<<std::min(nblk((long)m.nseg * NV, 256), g), 256, 0, st>>>((long)m.nseg, em, 1, re,
                                                                                      eprcn, (R)1000, me);
    k_tet_minv3_remove<R><<<std::min(nblk(m.ntet, 128), g), 128, 0, st>>>(m, em, fm, 2, mm, iprcn, rv, re, rf);
    k_tet_minv_scale<R><<<std::min(nblk((long)c->lf, 256), g), 256, 0, st>>>((long)c->lf, fm, rf, fprcn, (R)3000,
                                                                           mf);
}

extern "C" int hp_tet_enqueue_update(hp_tet_ctx *c) {
    if (!c) return HP_EINVAL;
    if (!c->smoother_ready()) {
        set_err(c->smoother ? "hp_tet_update (minvrt) needs hp_tet_setup_preconditioner first"
                            : "hp_tet_update needs hp_tet_jacobian_diagonal first");
        return HP_ESTATE;
    }
    TCK(cudaMemcpyAsync(c->U0, c->U, 8 * c->ltot, cudaMemcpyDeviceToDevice, c->stream));
    for (int stage = 0; stage < c->ph.nstage; ++stage) {
        int r = hp_tet_enqueue_rsdl(c, stage);
        if (r) return r;
        const double ca = c->ph.alpha[stage] * c->ph.cfl;
        if (c->smoother && c->p == 1)  // the state is the vertex section alone (ltot = lv)
            k_tet_minvrt1<<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
                (long)c->ltot, c->RES, c->vprcn, c->tab.vdiag, c->mask, c->U, c->U0, ca);
        else if (c->smoother && c->p == 3) {
            enqueue_minvrt3<double>(c, c->RES, c->vprcn, c->eprcn, c->fprcn, c->iprcn, c->d_mm, c->d_sfmv, c->d_ffmv,
                                    c->d_ffms, c->fac, c->spk_w);
            k_tet_advance<<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
                (long)c->ltot, c->RES, c->U, c->U0, ca);
        } else if (c->smoother) {
            const int g = c->nsm * 8;
            double *rv = c->RES, *re = c->RES + c->lv;
            k_tet_minv_e2v<<<std::min(nblk(c->mesh.nseg, 256), g), 256, 0, c->stream>>>(
                c->mesh.nseg, c->em, c->seg_pnt, c->d_sfmv, rv, re, c->mask + c->lv);
            k_tet_minv_scale<<<std::min(nblk((long)c->lv, 256), g), 256, 0, c->stream>>>(
                (long)c->lv, 1, rv, c->vprcn, c->tab.vdiag, c->mask);
            k_tet_minv_v2e<<<std::min(nblk(c->mesh.ntet, 128), g), 128, 0, c->stream>>>(
                c->mesh, c->em, c->d_mm, c->iprcn, rv, re);
            // p = 2: tet_hp::minvrt sets ediag(0) = 100 before scaling the edge modes
            k_tet_minv_scale<<<std::min(nblk((long)c->le, 256), g), 256, 0, c->stream>>>(
                (long)c->le, c->em, re, c->eprcn, 100.0, c->mask + c->lv);
            k_tet_advance<<<std::min(nblk((long)c->ltot, 256), g), 256, 0, c->stream>>>(
                (long)c->ltot, c->RES, c->U, c->U0, ca);
        } else
            k_tet_relax<<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
                (long)c->ltot, c->RES, c->JD, c->mask, c->U, c->U0, ca);
    }
    TCK(cudaGetLastError());
    return HP_OK;
}

extern "C" int hp_tet_update(hp_tet_ctx *c) {
    int r = hp_tet_enqueue_update(c);
    if (r) return r;
    return hp_tet_sync(c);
}

extern "C" int hp_tet_resnorm(hp_tet_ctx *c, double *l2) {
    if (!c || !l2) return HP_EINVAL;
    int r = hp_tet_enqueue_rsdl(c, c->ph.nstage);
    if (r) return r;
    const int nb = 1024;
    k_tet_sq<<<nb, 256, 0, c->stream>>>((long)c->ltot, c->RES, c->mask, c->part);
    std::vector<double> h(nb);
    TCK(cudaMemcpyAsync(h.data(), c->part, 8 * nb, cudaMemcpyDeviceToHost, c->stream));
    TCK(cudaStreamSynchronize(c->stream));
    double s2 = 0.0;
    for (int k = 0; k < nb; ++k) s2 += h[k];
    *l2 = std::sqrt(s2);
    return HP_OK;
}

// Smooths until the residual norm falls by `drop` (checked every check_every updates) or
// max_updates; the preconditioner (tau and the Jacobian diagonal) is set up once.
extern "C" int hp_tet_solve(hp_tet_ctx *c, double drop, int max_updates, int check_every, double *hist, int cap,
                            int *nhist, double *seconds, int *updates) {
    if (!c || drop <= 0 || max_updates < 1 || check_every < 1 || !hist || cap < 1) return HP_EINVAL;
    cudaEvent_t e0, e1;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    TCK(cudaEventRecord(e0, c->stream));
    int r = hp_tet_setup_preconditioner(c);
    if (r) return r < 0 ? r : HP_ESTATE;
    if (!c->smoother && (r = hp_tet_jacobian_diagonal(c))) return r;
    double r0;
    if ((r = hp_tet_resnorm(c, &r0))) return r;
    int nh = 0, nu = 0;
    hist[nh++] = 1.0;
    while (nu < max_updates) {
        for (int k = 0; k < check_every && nu < max_updates; ++k, ++nu)
            if ((r = hp_tet_enqueue_update(c))) return r;
        double rn;
        if ((r = hp_tet_resnorm(c, &rn))) return r;
        const double d = r0 > 0 ? rn / r0 : 0.0;
        if (nh < cap) hist[nh++] = d;
        if (!(d == d) || d <= drop) break;
    }
    TCK(cudaEventRecord(e1, c->stream));
    TCK(cudaEventSynchronize(e1));
    float ms = 0.f;
    TCK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (nhist) *nhist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (updates) *updates = nu;
    return HP_OK;
}

namespace {
int attach_common(hp_tet_ctx *c, hp_tet_ctx *f, double fadd) {
    int r;
    c->fine = f;
    c->fadd = fadd;
    for (double **b : {&c->RES0, &c->DRES, &c->UF}) {
        if (!*b && (r = talloc(c, (void **)b, 8 * c->ltot))) return r;
        TCK(cudaMemset(*b, 0, 8 * c->ltot));
    }
    return HP_OK;
}
}  // namespace

// p-level: coarse has the fine level's mesh at a lower p (mode truncation of the
// hierarchical basis: edge mode k, face mode (row m, k), interior (m, k, j) keep their
// indices; tet_hp/mg_restrict.cpp:9-57)
extern "C" int hp_tet_mg_attach_p(hp_tet_ctx *coarse, hp_tet_ctx *fine, double fadd) {
    if (!coarse || !fine || coarse->p >= fine->p || coarse->mesh.ntet != fine->mesh.ntet) return HP_EINVAL;
    hp_tet_ctx *c = coarse, *f = fine;
    std::vector<int> map(c->ltot);
    size_t k = 0;
    for (size_t v = 0; v < c->lv; ++v) map[k++] = (int)v;
    for (int e = 0; e < c->mesh.nseg; ++e)
        for (int m = 0; m < c->em; ++m)
            for (int n = 0; n < NV; ++n) map[k++] = (int)(f->lv + ((size_t)e * f->em + m) * NV + n);
    auto face_index = [](int em, int row, int col) {  // (row m >= 1, col k >= 1) -> index
        int idx = 0;
        for (int m = 1; m < row; ++m) idx += em - m;
        return idx + col - 1;
    };
    for (int t = 0; t < c->mesh.ntri; ++t)
        for (int m = 1; m <= c->em - 1; ++m)
            for (int kk = 1; kk <= c->em - m; ++kk)
                for (int n = 0; n < NV; ++n)
                    map[k++] = (int)(f->lv + f->le + ((size_t)t * f->fm + face_index(f->em, m, kk)) * NV + n);
    auto int_index = [](int em, int a, int b, int cc) {
        int idx = 0;
        for (int m = 1; m <= em - 1; ++m)
            for (int kk = 1; kk <= em - m; ++kk)
                for (int j = 1; j <= em - m - kk; ++j) {
                    if (m == a && kk == b && j == cc) return idx;
                    ++idx;
                }
        return -1;
    };
    for (int t = 0; t < c->mesh.ntet; ++t)
        for (int m = 1; m <= c->em - 1; ++m)
            for (int kk = 1; kk <= c->em - m; ++kk)
                for (int j = 1; j <= c->em - m - kk; ++j)
                    for (int n = 0; n < NV; ++n)
                        map[k++] = (int)(f->lv + f->le + f->lf + ((size_t)t * f->im + int_index(f->em, m, kk, j)) * NV + n);
    if (k != c->ltot) {
        set_err("p-level map size mismatch");
        return HP_EINVAL;
    }
    int r;
    if (!c->pmap && (r = talloc(c, (void **)&c->pmap, 4 * c->ltot))) return r;
    TCK(cudaMemcpy(c->pmap, map.data(), 4 * c->ltot, cudaMemcpyHostToDevice));
    c->kind = 1;
    return attach_common(c, f, fadd);
}

// h-level at p = 1: f2c [fine npnt] tetrahedron of the coarse mesh holding each fine
// vertex with its 4 barycentric weights (tet_mesh ccnnct), c2f [coarse npnt] likewise in
// the fine mesh (fcnnct)
extern "C" int hp_tet_mg_attach_h(hp_tet_ctx *coarse, hp_tet_ctx *fine, const int *f2c_tet, const double *f2c_w,
                                  const int *c2f_tet, const double *c2f_w, double fadd) {
    if (!coarse || !fine || coarse->p != 1 || fine->p != 1 || !f2c_tet || !f2c_w || !c2f_tet || !c2f_w)
        return HP_EINVAL;
    hp_tet_ctx *c = coarse;
    int r;
    const size_t nf = fine->mesh.npnt, nc = c->mesh.npnt;
    if ((r = talloc(c, (void **)&c->f2c_tet, 4 * nf)) || (r = talloc(c, (void **)&c->f2c_w, 32 * nf)) ||
        (r = talloc(c, (void **)&c->c2f_tet, 4 * nc)) || (r = talloc(c, (void **)&c->c2f_w, 32 * nc)))
        return r;
    TCK(cudaMemcpy(c->f2c_tet, f2c_tet, 4 * nf, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(c->f2c_w, f2c_w, 32 * nf, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(c->c2f_tet, c2f_tet, 4 * nc, cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(c->c2f_w, c2f_w, 32 * nc, cudaMemcpyHostToDevice));
    c->kind = 2;
    return attach_common(c, fine, fadd);
}

// mg_restrict: the fine residual (rsdl(nstage) already enqueued on the fine level) and
// state onto this level; the next residual evaluation here forms the FAS term
static int tet_mg_restrict(hp_tet_ctx *c) {
    hp_tet_ctx *f = c->fine;
    if (c->kind == 1) {
        k_tet_p_restrict<<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
            (long)c->ltot, c->pmap, f->U, f->RES, c->U, c->UF, c->RES0);
    } else {
        k_tet_h_restrict_state<<<nblk(c->mesh.npnt, 128), 128, 0, c->stream>>>(c->mesh.npnt, c->c2f_tet, c->c2f_w,
                                                                             f->mesh.tp, f->U, c->U, c->UF);
        TCK(cudaMemsetAsync(c->RES0, 0, 8 * c->ltot, c->stream));
        k_tet_h_restrict_res<<<nblk(f->mesh.npnt, 128), 128, 0, c->stream>>>(f->mesh.npnt, c->f2c_tet, c->f2c_w,
                                                                          c->mesh.tp, f->RES, c->RES0);
    }
    TCK(cudaGetLastError());
    c->fas_pending = true;
    return HP_OK;
}

static int tet_mg_prolongate(hp_tet_ctx *c) {
    hp_tet_ctx *f = c->fine;
    if (c->kind == 1)
        k_tet_p_prolong<<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>((long)c->ltot, c->pmap,
                                                                                             c->U, c->UF, f->U);
    else
        k_tet_h_prolong<<<nblk(f->mesh.npnt, 128), 128, 0, c->stream>>>(f->mesh.npnt, c->f2c_tet, c->f2c_w,
                                                                     c->mesh.tp, c->U, c->UF, f->U);
    TCK(cudaGetLastError());
    return HP_OK;
}

// block::cycle (tri_mesh/blocks.cpp:1267-1348) over levels[0] (finest) .. levels[n-1];
// a level's preconditioner (tau and the Jacobian diagonal) is set up on its first visit
static int tet_cycle(hp_tet_ctx **lv, int n, int lvl, int vw, int itercrsn, int iterrfne) {
    hp_tet_ctx *c = lv[lvl];
    int r;
    for (int vc = 0; vc < vw; ++vc) {
        if (!c->smoother_ready()) {
            r = hp_tet_setup_preconditioner(c);
            if (r) return r < 0 ? r : HP_ESTATE;
            if (!c->smoother && (r = hp_tet_jacobian_diagonal(c))) return r;
        }
        for (int it = 0; it < itercrsn; ++it)
            if ((r = hp_tet_enqueue_update(c))) return r;
        if (lvl == n - 1) return HP_OK;
        if ((r = hp_tet_enqueue_rsdl(c, c->ph.nstage))) return r;
        if ((r = tet_mg_restrict(lv[lvl + 1]))) return r;
        if ((r = tet_cycle(lv, n, lvl + 1, vw, itercrsn, iterrfne))) return r;
        if ((r = tet_mg_prolongate(lv[lvl + 1]))) return r;
        for (int it = 0; it < iterrfne; ++it)
            if ((r = hp_tet_enqueue_update(c))) return r;
    }
    return HP_OK;
}

extern "C" int hp_tet_solve_mg(hp_tet_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                               int iterrfne, double *hist, int cap, int *nhist, double *seconds, int *cycles) {
    if (!levels || nlevels < 1 || drop <= 0 || max_cycles < 1 || vw < 1 || !hist || cap < 1) return HP_EINVAL;
    for (int l = 1; l < nlevels; ++l)
        if (!levels[l]->fine || levels[l]->fine != levels[l - 1] || levels[l]->stream != levels[0]->stream) {
            set_err("hp_tet_solve_mg: levels must be attached in order and share one stream");
            return HP_EINVAL;
        }
    hp_tet_ctx *f = levels[0];
    cudaEvent_t e0, e1;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    TCK(cudaEventRecord(e0, f->stream));
    int r;
    if (!f->prcn_ready) {
        r = hp_tet_setup_preconditioner(f);
        if (r) return r < 0 ? r : HP_ESTATE;
    }
    double r0;
    if ((r = hp_tet_resnorm(f, &r0))) return r;
    int nh = 0, nc = 0;
    hist[nh++] = 1.0;
    while (nc < max_cycles) {
        if ((r = tet_cycle(levels, nlevels, 0, vw, itercrsn, iterrfne))) return r;
        ++nc;
        double rn;
        if ((r = hp_tet_resnorm(f, &rn))) return r;
        const double d = r0 > 0 ? rn / r0 : 0.0;
        if (nh < cap) hist[nh++] = d;
        if (!(d == d) || d <= drop) break;
    }
    TCK(cudaEventRecord(e1, f->stream));
    TCK(cudaEventSynchronize(e1));
    float ms = 0.f;
    TCK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (nhist) *nhist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (cycles) *cycles = nc;
    return HP_OK;
}

// ---------------------------------------------------------------------------
// Multigrid inside FP64 defect correction with FP32 smoothing (the FP32 arm of the 3D
// workload). Every cycle: the FP64 residual R64(u) of the finest level; the base states
// (u and its FP64 restriction down the levels) in FP32 with their point values; one FP32
// cycle of block::cycle (tri_mesh/blocks.cpp:1267-1348) on the correction equation of
// every level (residual in correction form plus the level's source: R64 on the finest,
// the FAS term below it), smoothed as the FP64 levels are (tet_hp's JACOBI relaxation,
// or minvrt at p <= 2); then u += d in FP64. The preconditioners (tau, the Jacobian
// diagonal, minvrt's) are set up once at the initial state, as in hp_tet_solve_mg, and
// copied to FP32. Inflow flux faces only (their continuity flux is linear in the state).
// ---------------------------------------------------------------------------
namespace {

template <int P>
void tet_fragments_tf32(const hp_tet_tables &b, std::vector<float> &proj, std::vector<float> &intg,
                        std::vector<float> &F) {
    using C = TetCfg<P>;
    using M = TetTf32<P>;
    auto tf = [](double v) {
        float f = (float)v;
        uint32_t u;
        std::memcpy(&u, &f, 4);
        u = (u + 0x1000u) & 0xFFFFE000u;  // round to TF32 (nearest, ties away), as cvt.rna
        std::memcpy(&f, &u, 4);
        return f;
    };
    proj.assign(M::PROJ_LEN, 0.f);
    intg.assign(M::INT_LEN, 0.f);
    const double(*ops[4])[HP_TET_MAXT] = {b.F, b.DX, b.DY, b.DZ};
    auto op = [&](int o, int q, int m) { return (q < C::Q && m < C::T) ? ops[o][q][m] : 0.0; };
    auto wd = [&](int k, int m) {
        if (k >= 3 * C::Q || m >= C::T) return 0.0;
        const int c = k / C::Q, q = k - c * C::Q;
        return b.w[q] * ops[1 + c][q][m];
    };
    // m16n8k8 B fragments: lane l holds B[k = l & 3][n = l >> 2] and B[k + 4][n]
    for (int o = 0; o < 4; ++o)
        for (int nt = 0; nt < M::NT; ++nt)
            for (int ks = 0; ks < M::KS; ++ks)
                for (int l = 0; l < 32; ++l) {
                    const size_t at = ((((size_t)o * M::NT + nt) * M::KS + ks) * 32 + l) * 2;
                    const int q = nt * 8 + (l >> 2), m = ks * 8 + (l & 3);
                    proj[at] = tf(op(o, q, m));
                    proj[at + 1] = tf(op(o, q, m + 4));
                }
    for (int nt = 0; nt < M::NT2; ++nt)
        for (int ks = 0; ks < M::KS2; ++ks)
            for (int l = 0; l < 32; ++l) {
                const size_t at = (((size_t)nt * M::KS2 + ks) * 32 + l) * 2;
                const int k = ks * 8 + (l & 3), m = nt * 8 + (l >> 2);
                intg[at] = tf(wd(k, m));
                intg[at + 1] = tf(wd(k + 4, m));
            }
    F.assign((size_t)C::Q * C::T, 0.f);
    for (int q = 0; q < C::Q; ++q)
        for (int m = 0; m < C::T; ++m) F[(size_t)q * C::T + m] = (float)b.F[q][m];
}

template <int P>
TetSmall<float, P> small32(const hp_tet_tables &t) {
    TetSmall<float, P> sm;
    for (int i = 0; i <= P; ++i) {
        for (int j = 0; j <= P; ++j) {
            sm.Ax[i][j] = (float)t.Ax[i][j];
            sm.Bx[i][j] = (float)t.Bx[i][j];
            sm.Ay[i][j] = (float)t.Ay[i][j];
            sm.By[i][j] = (float)t.By[i][j];
            sm.Az[i][j] = (float)t.Az[i][j];
        }
        sm.y0[i] = (float)t.y0[i];
        sm.z0[i] = (float)t.z0[i];
    }
    return sm;
}

int mixed_alloc(hp_tet_ctx *c) {
    if (c->mixed_ready) return HP_OK;
    hp_tet_ctx::Mixed &x = c->mx;
    int r;
    for (float **f : {&x.U, &x.U0, &x.RES, &x.RR, &x.UB, &x.DRES, &x.JD, &x.RES0, &x.UF}) {
        if ((r = talloc(c, (void **)f, 4 * std::max<size_t>(c->ltot, 1)))) return r;
        TCK(cudaMemset(*f, 0, 4 * std::max<size_t>(c->ltot, 1)));
    }
    if ((r = talloc(c, (void **)&x.BPT, 4 * (size_t)c->mesh.ntet * 3 * c->Q)) ||
        (r = talloc(c, (void **)&x.TAU, 8 * (size_t)c->mesh.ntet)) ||
        (r = talloc(c, (void **)&x.iprcn, 16 * (size_t)c->mesh.ntet)) ||
        (r = talloc(c, (void **)&x.vprcn, 16 * (size_t)c->mesh.npnt)) ||
        (r = talloc(c, (void **)&x.eprcn, 16 * (size_t)std::max(1, c->mesh.nseg))))
        return r;
    {
        std::vector<float> mm(sizeof(c->tab.mm) / 8), sf(sizeof(c->tab.sfmv) / 8);
        const double *pm = &c->tab.mm[0][0], *ps = &c->tab.sfmv[0][0];
        for (size_t k = 0; k < mm.size(); ++k) mm[k] = (float)pm[k];
        for (size_t k = 0; k < sf.size(); ++k) sf[k] = (float)ps[k];
        if ((r = talloc(c, (void **)&x.mm, 4 * mm.size())) || (r = talloc(c, (void **)&x.sfmv, 4 * sf.size()))) return r;
        TCK(cudaMemcpy(x.mm, mm.data(), 4 * mm.size(), cudaMemcpyHostToDevice));
        TCK(cudaMemcpy(x.sfmv, sf.data(), 4 * sf.size(), cudaMemcpyHostToDevice));
    }
    std::vector<float> pb, ib, F;
    switch (c->p) {
        case 1: tet_fragments_tf32<1>(c->tab, pb, ib, F); break;
        case 2: tet_fragments_tf32<2>(c->tab, pb, ib, F); break;
        case 3: tet_fragments_tf32<3>(c->tab, pb, ib, F); break;
        case 4: tet_fragments_tf32<4>(c->tab, pb, ib, F); break;
        default: return HP_EINVAL;
    }
    if ((r = talloc(c, (void **)&x.projB, 4 * pb.size())) || (r = talloc(c, (void **)&x.intB, 4 * ib.size())) ||
        (r = talloc(c, (void **)&x.F, 4 * F.size())))
        return r;
    TCK(cudaMemcpy(x.projB, pb.data(), 4 * pb.size(), cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(x.intB, ib.data(), 4 * ib.size(), cudaMemcpyHostToDevice));
    TCK(cudaMemcpy(x.F, F.data(), 4 * F.size(), cudaMemcpyHostToDevice));
    c->mixed_ready = true;
    return HP_OK;
}

template <typename A, typename B>
void conv(hp_tet_ctx *c, long n, const A *src, B *dst) {
    if (n > 0) k_tet_convert<A, B><<<std::min(nblk(n, 256), c->nsm * 8), 256, 0, c->stream>>>(n, src, dst);
}

// FP32 copies of the preconditioner set up in FP64 at the base state (and, for minvrt at
// p = 3, of the face diagonals, the face tables and the spoke factors)
int mixed_prcn(hp_tet_ctx *c) {
    hp_tet_ctx::Mixed &x = c->mx;
    conv(c, 2L * c->mesh.ntet, c->tau, x.TAU);
    conv(c, (long)c->ltot, c->JD, x.JD);
    conv(c, (long)c->mesh.ntet * NV, c->iprcn, x.iprcn);
    conv(c, (long)c->mesh.npnt * NV, c->vprcn, x.vprcn);
    conv(c, (long)c->mesh.nseg * NV, c->eprcn, x.eprcn);
    if (c->smoother == 1 && c->p == 3 && c->fac) {
        int r;
        if (!x.fac) {
            std::vector<float> ff(sizeof(c->tab.ffmv) / 8), fs(sizeof(c->tab.ffms) / 8);
            for (size_t k = 0; k < ff.size(); ++k) ff[k] = (float)(&c->tab.ffmv[0][0])[k];
            for (size_t k = 0; k < fs.size(); ++k) fs[k] = (float)(&c->tab.ffms[0][0][0])[k];
            if ((r = talloc(c, (void **)&x.fac, 4 * (size_t)std::max<long long>(c->nfac, 1))) ||
                (r = talloc(c, (void **)&x.spk_w, 4 * (size_t)c->mesh.nseg * 2 * NV)) ||
                (r = talloc(c, (void **)&x.fprcn, 16 * (size_t)std::max(1, c->mesh.ntri))) ||
                (r = talloc(c, (void **)&x.ffmv, 4 * ff.size())) || (r = talloc(c, (void **)&x.ffms, 4 * fs.size())))
                return r;
            TCK(cudaMemcpy(x.ffmv, ff.data(), 4 * ff.size(), cudaMemcpyHostToDevice));
            TCK(cudaMemcpy(x.ffms, fs.data(), 4 * fs.size(), cudaMemcpyHostToDevice));
        }
        conv(c, (long)c->mesh.ntri * NV, c->fprcn, x.fprcn);
        conv(c, (long)c->nfac, c->fac, x.fac);
    }
    return HP_OK;
}

template <int P>
int base_points(hp_tet_ctx *c) {
    k_tet_base_points<P><<<nblk(3L * c->mesh.ntet, 128), 128, 0, c->stream>>>(c->mx.F, c->mesh, c->fields32(c->mx.UB),
                                                                            c->mx.BPT);
    TCK(cudaGetLastError());
    return HP_OK;
}

int base_points_any(hp_tet_ctx *c) {
    switch (c->p) {
        case 1: return base_points<1>(c);
        case 2: return base_points<2>(c);
        case 3: return base_points<3>(c);
        case 4: return base_points<4>(c);
    }
    return HP_EINVAL;
}

template <int P>
int launch_rsdl32(hp_tet_ctx *c, int stage) {
    using M = TetTf32<P>;
    static bool attr = false;
    if (!attr) {
        TCK(cudaFuncSetAttribute(k_tet_rsdl_tf32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::SMEM));
        attr = true;
    }
    hp_tet_ctx::Mixed &x = c->mx;
    const float omb = stage >= c->ph.nstage ? 0.f : (float)(1.0 - c->ph.beta[stage]);
    const float beta = (float)c->ph.beta[stage];
    const int g = std::min(nblk((long)c->ltot, 256), c->nsm * 8);
    k_tet_pre<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.RR, omb);
    if (c->faces.n > 0)
        k_tet_face_flux32<P><<<std::min(nblk(c->faces.n, 4), c->nsm * 16), 128, 0, c->stream>>>(
            c->faces, c->ftab, c->mesh, c->fields32(x.U), c->fields32(x.RES), (float)c->ph.rho);
    const long nquad = ((long)c->mesh.ntet + 3) / 4;
    k_tet_rsdl_tf32<P><<<std::min(nblk(nquad, M::WPC), c->nsm * 32), M::WPC * 32, M::SMEM, c->stream>>>(
        x.projB, x.intB, small32<P>(c->tab), c->mesh, c->fields32(x.U), c->fields32(x.RES), c->fields32(x.RR), x.TAU,
        x.BPT, (float)c->ph.rho, (float)c->ph.mu, beta);
    k_tet_fold<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.RR);
    // the source: the FP64 defect on the finest level; the FAS term, formed at the first
    // residual after a restriction, below it
    k_tet_fas<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.RES0, x.DRES, (float)c->fadd,
                                               (c->fine && x.fas_pending) ? 1 : 0);
    x.fas_pending = false;
    TCK(cudaGetLastError());
    return HP_OK;
}

int rsdl32(hp_tet_ctx *c, int stage) {
    switch (c->p) {
        case 1: return launch_rsdl32<1>(c, stage);
        case 2: return launch_rsdl32<2>(c, stage);
        case 3: return launch_rsdl32<3>(c, stage);
        case 4: return launch_rsdl32<4>(c, stage);
    }
    return HP_EINVAL;
}

// tet_hp::update in FP32 on the correction: the stages of hp_tet_enqueue_update
int update32(hp_tet_ctx *c) {
    hp_tet_ctx::Mixed &x = c->mx;
    TCK(cudaMemcpyAsync(x.U0, x.U, 4 * c->ltot, cudaMemcpyDeviceToDevice, c->stream));
    const int g = std::min(nblk((long)c->ltot, 256), c->nsm * 8);
    for (int stage = 0; stage < c->ph.nstage; ++stage) {
        int r = rsdl32(c, stage);
        if (r) return r;
        const float ca = (float)(c->ph.alpha[stage] * c->ph.cfl);
        if (c->smoother && c->p == 1) {
            k_tet_minvrt1<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.vprcn, (float)c->tab.vdiag, c->mask,
                                                           x.U, x.U0, ca);
        } else if (c->smoother && c->p == 3) {
            enqueue_minvrt3<float>(c, x.RES, x.vprcn, x.eprcn, x.fprcn, x.iprcn, x.mm, x.sfmv, x.ffmv, x.ffms, x.fac,
                                   x.spk_w);
            k_tet_advance<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.U, x.U0, ca);
        } else if (c->smoother) {
            float *rv = x.RES, *re = x.RES + c->lv;
            k_tet_minv_e2v<float><<<std::min(nblk(c->mesh.nseg, 256), c->nsm * 8), 256, 0, c->stream>>>(
                c->mesh.nseg, c->em, c->seg_pnt, x.sfmv, rv, re, c->mask + c->lv);
            k_tet_minv_scale<float><<<std::min(nblk((long)c->lv, 256), c->nsm * 8), 256, 0, c->stream>>>(
                (long)c->lv, 1, rv, x.vprcn, (float)c->tab.vdiag, c->mask);
            k_tet_minv_v2e<float><<<std::min(nblk(c->mesh.ntet, 128), c->nsm * 8), 128, 0, c->stream>>>(
                c->mesh, c->em, x.mm, x.iprcn, rv, re);
            k_tet_minv_scale<float><<<std::min(nblk((long)c->le, 256), c->nsm * 8), 256, 0, c->stream>>>(
                (long)c->le, c->em, re, x.eprcn, 100.f, c->mask + c->lv);
            k_tet_advance<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.U, x.U0, ca);
        } else {
            k_tet_relax<float><<<g, 256, 0, c->stream>>>((long)c->ltot, x.RES, x.JD, c->mask, x.U, x.U0, ca);
        }
    }
    TCK(cudaGetLastError());
    return HP_OK;
}

int restrict32(hp_tet_ctx *c) {
    hp_tet_ctx *f = c->fine;
    hp_tet_ctx::Mixed &x = c->mx;
    if (c->kind == 1) {
        k_tet_p_restrict<float><<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
            (long)c->ltot, c->pmap, f->mx.U, f->mx.RES, x.U, x.UF, x.RES0);
    } else {
        k_tet_h_restrict_state<float><<<nblk(c->mesh.npnt, 128), 128, 0, c->stream>>>(
            c->mesh.npnt, c->c2f_tet, c->c2f_w, f->mesh.tp, f->mx.U, x.U, x.UF);
        TCK(cudaMemsetAsync(x.RES0, 0, 4 * c->ltot, c->stream));
        k_tet_h_restrict_res<float><<<nblk(f->mesh.npnt, 128), 128, 0, c->stream>>>(
            f->mesh.npnt, c->f2c_tet, c->f2c_w, c->mesh.tp, f->mx.RES, x.RES0);
    }
    TCK(cudaGetLastError());
    x.fas_pending = true;
    return HP_OK;
}

int prolong32(hp_tet_ctx *c) {
    hp_tet_ctx *f = c->fine;
    if (c->kind == 1)
        k_tet_p_prolong<float><<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
            (long)c->ltot, c->pmap, c->mx.U, c->mx.UF, f->mx.U);
    else
        k_tet_h_prolong<float><<<nblk(f->mesh.npnt, 128), 128, 0, c->stream>>>(f->mesh.npnt, c->f2c_tet, c->f2c_w,
                                                                              c->mesh.tp, c->mx.U, c->mx.UF, f->mx.U);
    TCK(cudaGetLastError());
    return HP_OK;
}

int cycle32(hp_tet_ctx **lv, int n, int lvl, int vw, int itercrsn, int iterrfne) {
    hp_tet_ctx *c = lv[lvl];
    int r;
    for (int vc = 0; vc < vw; ++vc) {
        for (int it = 0; it < itercrsn; ++it)
            if ((r = update32(c))) return r;
        if (lvl == n - 1) return HP_OK;
        if ((r = rsdl32(c, c->ph.nstage))) return r;
        if ((r = restrict32(lv[lvl + 1]))) return r;
        if ((r = cycle32(lv, n, lvl + 1, vw, itercrsn, iterrfne))) return r;
        if ((r = prolong32(lv[lvl + 1]))) return r;
        for (int it = 0; it < iterrfne; ++it)
            if ((r = update32(c))) return r;
    }
    return HP_OK;
}

// Base states of every level for one correction cycle: the FP64 state restricted down
// the levels (FP64 transfers), in FP32 with its point values; the corrections start at 0
int mixed_bases(hp_tet_ctx **lv, int n) {
    for (int l = 1; l < n; ++l) {
        hp_tet_ctx *c = lv[l], *f = lv[l - 1];
        if (c->kind == 1)
            k_tet_p_restrict<double><<<std::min(nblk((long)c->ltot, 256), c->nsm * 8), 256, 0, c->stream>>>(
                (long)c->ltot, c->pmap, f->U, f->RES, c->U, c->UF, c->RES0);
        else
            k_tet_h_restrict_state<double><<<nblk(c->mesh.npnt, 128), 128, 0, c->stream>>>(
                c->mesh.npnt, c->c2f_tet, c->c2f_w, f->mesh.tp, f->U, c->U, c->UF);
    }
    for (int l = 0; l < n; ++l) {
        hp_tet_ctx *c = lv[l];
        conv(c, (long)c->ltot, c->U, c->mx.UB);
        int r = base_points_any(c);
        if (r) return r;
        TCK(cudaMemsetAsync(c->mx.U, 0, 4 * c->ltot, c->stream));
    }
    TCK(cudaGetLastError());
    return HP_OK;
}

}  // namespace

extern "C" int hp_tet_solve_mg_mixed(hp_tet_ctx **levels, int nlevels, double drop, int max_cycles, int vw,
                                     int itercrsn, int iterrfne, double *hist, int cap, int *nhist, double *seconds,
                                     int *cycles) {
    if (!levels || nlevels < 1 || drop <= 0 || max_cycles < 1 || vw < 1 || !hist || cap < 1) return HP_EINVAL;
    for (int l = 1; l < nlevels; ++l)
        if (!levels[l]->fine || levels[l]->fine != levels[l - 1] || levels[l]->stream != levels[0]->stream) {
            set_err("hp_tet_solve_mg_mixed: levels must be attached in order and share one stream");
            return HP_EINVAL;
        }
    int r;
    for (int l = 0; l < nlevels; ++l) {
        hp_tet_ctx *c = levels[l];
        std::vector<int> kind(c->faces.n);
        if (c->faces.n)
            TCK(cudaMemcpy(kind.data(), c->faces.kind, 4 * (size_t)c->faces.n, cudaMemcpyDeviceToHost));
        for (int k : kind)
            if (k != 0) {
                set_err("hp_tet_solve_mg_mixed: flux faces other than inflow are not built in FP32");
                return HP_ENOTSUP;
            }
        if ((r = mixed_alloc(c))) return r;
    }
    hp_tet_ctx *f = levels[0];
    cudaEvent_t e0, e1;
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    TCK(cudaEventRecord(e0, f->stream));
    // preconditioners at the initial state of every level (as hp_tet_solve_mg's first visits)
    if ((r = mixed_bases(levels, nlevels))) return r;
    for (int l = 0; l < nlevels; ++l) {
        hp_tet_ctx *c = levels[l];
        r = hp_tet_setup_preconditioner(c);
        if (r) return r < 0 ? r : HP_ESTATE;
        if (!c->smoother && (r = hp_tet_jacobian_diagonal(c))) return r;
        if ((r = mixed_prcn(c))) return r;
    }
    double r0;
    if ((r = hp_tet_resnorm(f, &r0))) return r;  // leaves R64(u) in f->RES
    int nh = 0, nc = 0;
    hist[nh++] = 1.0;
    while (nc < max_cycles) {
        if ((r = mixed_bases(levels, nlevels))) return r;
        conv(f, (long)f->ltot, f->RES, f->mx.DRES);
        if ((r = cycle32(levels, nlevels, 0, vw, itercrsn, iterrfne))) return r;
        k_tet_add_correction<<<std::min(nblk((long)f->ltot, 256), f->nsm * 8), 256, 0, f->stream>>>((long)f->ltot,
                                                                                                  f->U, f->mx.U);
        ++nc;
        double rn;
        if ((r = hp_tet_resnorm(f, &rn))) return r;
        const double d = r0 > 0 ? rn / r0 : 0.0;
        if (nh < cap) hist[nh++] = d;
        if (!(d == d) || d <= drop) break;
    }
    TCK(cudaEventRecord(e1, f->stream));
    TCK(cudaEventSynchronize(e1));
    float ms = 0.f;
    TCK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (nhist) *nhist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (cycles) *cycles = nc;
    return HP_OK;
}

// ---------------------------------------------------------------------------
// Learned correction of the tet smoother (no counterpart in the reference)
// ---------------------------------------------------------------------------
static int tet_net_scale(hp_tet_ctx *c) {
    if (!c->d_feat && talloc(c, (void **)&c->d_feat, (size_t)c->mesh.ntet * 17 * 4)) return HP_ECUDA;
    if (!c->d_netout && talloc(c, (void **)&c->d_netout, (size_t)c->mesh.ntet * 4)) return HP_ECUDA;
    int r = hp_tet_elem_features(c, c->d_feat);
    if (r) return r;
    if (hp_mlp_forward(c->net, c->d_feat, c->mesh.ntet, c->d_netout, c->stream)) {
        set_err("network forward failed: %s", hp_mlp_last_error());
        return HP_ECUDA;
    }
    c->lsc = c->d_netout;
    return HP_OK;
}

extern "C" int hp_tet_elem_features(hp_tet_ctx *c, float *d_feat) {
    if (!c || !d_feat) return HP_EINVAL;
    k_tet_elem_features<<<nblk(c->mesh.ntet, 128), 128, 0, c->stream>>>(c->mesh, c->fields(c->U), c->p, c->em, c->fm,
                                                                       c->im, c->ph.mu / c->ph.rho, d_feat);
    TCK(cudaGetLastError());
    return HP_OK;
}

extern "C" int hp_tet_elem_resnorm(hp_tet_ctx *c, double *d_out) {
    if (!c || !d_out) return HP_EINVAL;
    const int g = nblk(c->mesh.ntet, 128);
    switch (c->p) {
        case 1: k_tet_elem_resnorm<1><<<g, 128, 0, c->stream>>>(c->mesh, c->fields(c->RES), d_out); break;
        case 2: k_tet_elem_resnorm<2><<<g, 128, 0, c->stream>>>(c->mesh, c->fields(c->RES), d_out); break;
        case 3: k_tet_elem_resnorm<3><<<g, 128, 0, c->stream>>>(c->mesh, c->fields(c->RES), d_out); break;
        case 4: k_tet_elem_resnorm<4><<<g, 128, 0, c->stream>>>(c->mesh, c->fields(c->RES), d_out); break;
    }
    TCK(cudaGetLastError());
    return HP_OK;
}

extern "C" int hp_tet_set_prcn_scale(hp_tet_ctx *c, const float *d_logscale, float clampv) {
    if (!c) return HP_EINVAL;
    c->lsc = d_logscale;
    c->lsc_clamp = clampv;
    c->net = nullptr;
    return HP_OK;
}

extern "C" int hp_tet_set_prcn_net(hp_tet_ctx *c, hp_mlp *net, float clampv) {
    if (!c) return HP_EINVAL;
    if (net) {
        int nin = 0, nout = 0;
        if (hp_mlp_dims(net, &nin, &nout) || nin != 17 || nout != 1) {
            set_err("hp_tet_set_prcn_net: the network must map 17 inputs to 1 output");
            return HP_EINVAL;
        }
    }
    c->net = net;
    c->lsc = nullptr;
    c->lsc_clamp = clampv;
    return HP_OK;
}
