// FP64 ins element residual on the tensor cores (straight triangles).
//
// tri_hp::rsdl's element loop (tri_hp/nstage.cpp:52-73: ugtouht, element_rsdl, lftog)
// with tri_hp_ins::element_rsdl's straight-element branch (tri_hp/ins/rsdl.cpp:259-433)
// and the tri_basis operators it calls (proj.cpp:22-119, intgrt.cpp:81-158,
// derivr / derivs proj.cpp:339-402). One warp takes two triangles; the 8 rows of a
// DMMA fragment (mma.m8n8k4.f64) are (triangle, variable) pairs, variable slot 3
// unused:
//   projection  C[8 x GG] = U[8 x T] * Op^T[T x GG]   for Op = value, d/dr, d/ds
//   intgrtrs    C[8 x T]  = F[8 x 2GG] * W[2GG x T]   (F = [flux_r | flux_s] at the points)
// The operators are the sum-factorised proj / intgrtrs written out per point (dense),
// built on the host from the basis tables and stored in fragment order (one coalesced
// 8-byte read-only load per lane per MMA). Pointwise fluxes, the strong residual
// (derivr / derivs) and the SUPG terms stay scalar, lanes owning (triangle, point)
// pairs, on per-warp shared-memory arrays. Vertex and side residuals go to the
// assembly-by-gather buffers (State::elim / elre) or, without them, FP64 atomics;
// interior residuals are written directly.
#pragma once
#include "hp_kernels.cuh"

namespace hpb {

template <int P>
struct InsMma {
    static constexpr int G = P + 1, GG = G * G, X = P + 2, T = (P + 1) * (P + 2) / 2, SM = P - 1,
                         IM = (P - 1) * (P - 2) / 2, BM = 3 * P, NV = 3;
    static constexpr int KS = (T + 3) / 4;        // projection k-steps
    static constexpr int NT = (GG + 7) / 8;       // projection n-tiles
    static constexpr int KS2 = (2 * GG + 3) / 4;  // intgrtrs k-steps
    static constexpr int NT2 = (T + 7) / 8;       // intgrtrs n-tiles
    // flux-pair stride: [flux_r (GG) | flux_s (GG) | zeros], 4 (mod 16) doubles so that the
    // 4 variable rows a half-warp reads in one A-fragment load fall on distinct banks
    static constexpr int pad4(int x) { return x + ((4 - x % 16) + 16) % 16; }
    static constexpr int VS = pad4(KS2 * 4);
    static constexpr int QP = NT * 8 + 4;  // point-array stride
    // per triangle: PV [3][QP] u, v, p; PD [4][QP] du/dr, dv/dr, du/ds, dv/ds (the gathered
    // modes [4][T] before the projection, the strong residual [3][QP] after the fluxes);
    // FI [3][VS] imaginary flux pairs; FR [3][VS] real flux pairs
    static constexpr int S_EL = 7 * QP + 6 * VS;
    static constexpr int WPC = 4;                  // warps per CTA
    static constexpr int MINB = P <= 4 ? 4 : 3;    // CTAs per SM the register budget allows
    static constexpr int NG = NT < 8 ? NT : 8;     // projection n-tiles accumulated together
    static constexpr size_t PROJ_LEN = (size_t)3 * NT * KS * 32, INT_LEN = (size_t)NT2 * KS2 * 32;
    // strong residual (derivr + derivs) as tensor products of the 1D derivative operators:
    // A fragments of Ar | As1 ([MT][2 KR][32], rows i, k = q) and As2 ([MT][KR][32], rows j,
    // k = l); the point data are the B operands, columns (triangle, variable, point)
    static constexpr int KR = (G + 3) / 4, MT = (G + 7) / 8, NCOL = 6 * G, NTB = (NCOL + 7) / 8;
    static constexpr size_t DER_LEN = (size_t)MT * 3 * KR * 32;
    static constexpr int IDX = 16;  // staged mesh integers per triangle: pnt[3], seg[3], sgn[3], vpos[3], spos[3]
    static constexpr size_t SMEM_IDX = (size_t)WPC * 2 * IDX * sizeof(int);
    // per triangle: the metrics d00, d01, d10, d11 (ldcrd), mu / |J|, 2 nu / h, adis h / |J|, unused
    static constexpr int GEO = 8;
    static constexpr size_t SMEM_GEO = (size_t)WPC * 2 * GEO * sizeof(double);
    static_assert(4 * T <= 4 * QP, "gathered modes must fit the PD block");
};

// The 1D derivative tables of derivr / derivs and the collapsed-coordinate factors.
template <typename R, int P>
struct InsSmall {
    R dltx[P + 1], dltx1[P + 1][P + 1], dltn[P + 1], dltn1[P + 1][P + 1], dltn2[P + 1][P + 1];
    R n0[P + 1], x0[P + 1];
};
template <int P>
using InsMmaSmall = InsSmall<double, P>;
template <int P>
using InsMmaSmallF = InsSmall<float, P>;

__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// C[8 x N] += A[8 x K] * B[K x N] of one warp's fragment rows, A read from a shared-memory
// row of K (padded) entries, B in fragment order [nt][ks][lane]; the k-steps alternate
// between two accumulator sets so that consecutive DMMAs of a tile are independent.
template <int KS, int NTL>
__device__ __forceinline__ void warp_gemm(const double *__restrict__ arow, const double *__restrict__ B, int gcol,
                                          int lane, double (&c)[NTL][2]) {
    double c2[NTL][2];
#pragma unroll
    for (int nt = 0; nt < NTL; ++nt) c[nt][0] = c[nt][1] = c2[nt][0] = c2[nt][1] = 0.0;
#pragma unroll 4
    for (int ks = 0; ks < KS; ks += 2) {
        const double a0 = arow[ks * 4 + gcol];
        const double a1 = ks + 1 < KS ? arow[(ks + 1) * 4 + gcol] : 0.0;
#pragma unroll
        for (int nt = 0; nt < NTL; ++nt) {
            dmma884(c[nt][0], c[nt][1], a0, __ldg(B + ((size_t)nt * KS + ks) * 32 + lane));
            if (ks + 1 < KS) dmma884(c2[nt][0], c2[nt][1], a1, __ldg(B + ((size_t)nt * KS + ks + 1) * 32 + lane));
        }
    }
#pragma unroll
    for (int nt = 0; nt < NTL; ++nt) {
        c[nt][0] += c2[nt][0];
        c[nt][1] += c2[nt][1];
    }
}

// The imaginary and the real intgrtrs of the same rows at once: Ca = A_a B, Cb = A_b B with
// each B fragment loaded once for both (the real part's B is the imaginary part's).
template <int KS, int NTL>
__device__ __forceinline__ void warp_gemm2(const double *__restrict__ arow_a, const double *__restrict__ arow_b,
                                           const double *__restrict__ B, int gcol, int lane, double (&ca)[NTL][2],
                                           double (&cb)[NTL][2]) {
#pragma unroll
    for (int nt = 0; nt < NTL; ++nt) ca[nt][0] = ca[nt][1] = cb[nt][0] = cb[nt][1] = 0.0;
#pragma unroll 4
    for (int ks = 0; ks < KS; ++ks) {
        const double a = arow_a[ks * 4 + gcol], b = arow_b[ks * 4 + gcol];
#pragma unroll
        for (int nt = 0; nt < NTL; ++nt) {
            const double bf = __ldg(B + ((size_t)nt * KS + ks) * 32 + lane);
            dmma884(ca[nt][0], ca[nt][1], a, bf);
            dmma884(cb[nt][0], cb[nt][1], b, bf);
        }
    }
}

template <int P>
__global__ void __launch_bounds__(InsMma<P>::WPC * 32, InsMma<P>::MINB)
    k_rsdl_ins_mma(const double *__restrict__ projB, const double *__restrict__ intB,
                   const double *__restrict__ derB, InsMmaSmall<P> small, Mesh mesh, State<double> st, Phys ph,
                   int stage, int zero_rr) {
    using M = InsMma<P>;
    constexpr int G = M::G, GG = M::GG, T = M::T, BM = M::BM, IM = M::IM, NV = 3, QP = M::QP, VS = M::VS;
    constexpr int SM = (M::SM > 0 ? M::SM : 1);  // side-mode stride (unused when p = 1)
    constexpr int IMD = (IM > 0 ? IM : 1);        // interior-mode stride (unused when p < 3)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InsMmaSmall<P> &tb = *reinterpret_cast<InsMmaSmall<P> *>(smem_raw);
    {
        const int n4 = sizeof(InsMmaSmall<P>) / 4;
        const int *src = reinterpret_cast<const int *>(&small);
        int *dst = reinterpret_cast<int *>(smem_raw);
        for (int k = threadIdx.x; k < n4; k += blockDim.x) dst[k] = src[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grow = lane >> 2, gcol = lane & 3;
    const int re_ = grow >> 2, rv = grow & 3;  // fragment row -> (triangle, variable)
    double *base = reinterpret_cast<double *>(smem_raw + ((sizeof(InsMmaSmall<P>) + 15) / 16) * 16) +
                   (size_t)warp * 2 * M::S_EL;
    double *geo = reinterpret_cast<double *>(smem_raw + ((sizeof(InsMmaSmall<P>) + 15) / 16) * 16) +
                  (size_t)M::WPC * 2 * M::S_EL + warp * 2 * M::GEO;
    int *midx = reinterpret_cast<int *>(reinterpret_cast<double *>(smem_raw + ((sizeof(InsMmaSmall<P>) + 15) / 16) * 16) +
                                        (size_t)M::WPC * 2 * (M::S_EL + M::GEO)) + warp * 2 * M::IDX;
    // per triangle: PV u, v, p at the points; PD the gathered modes, then du/dr, dv/dr,
    // du/ds, dv/ds, then the strong residual; FI the imaginary flux pairs (convective +
    // pressure for u, v; the mass flux for p); FX the viscous flux pairs (zero for p), then
    // the real flux pairs (viscous - SUPG; the continuity SUPG term for p). The strong
    // residual differentiates FI + FX.
    auto PV = [&](int e) { return base + e * M::S_EL; };
    auto PD = [&](int e) { return base + e * M::S_EL + 3 * QP; };
    auto FI = [&](int e) { return base + e * M::S_EL + 7 * QP; };
    auto FX = [&](int e) { return base + e * M::S_EL + 7 * QP + 3 * VS; };
    // the K padding of the flux pairs stays zero (their B rows are zero too)
    for (int e = 0; e < 2; ++e)
        for (int k = 2 * GG + lane; k < VS; k += 32)
            for (int v = 0; v < 3; ++v) FI(e)[v * VS + k] = FX(e)[v * VS + k] = 0.0;
    __syncthreads();
    const double beta = ph.beta[stage];
    const double omb = zero_rr ? 0.0 : 1.0 - beta;
    const double rho = ph.rho, mu = ph.mu;
    const long ntri = mesh.ntri, npair = (ntri + 1) / 2;
    for (long pr = (long)blockIdx.x * M::WPC + warp; pr < npair; pr += (long)gridDim.x * M::WPC) {
        const int t0 = (int)(2 * pr);
        const bool has1 = t0 + 1 < ntri;
        // triangle e (0, 1) of the pair and whether it is done here (curved triangles are
        // done by the curved launch; a missing second triangle repeats the first, unwritten).
        // Per-triangle values are selected, not indexed, so that they stay in registers.
        const int ta = t0, tb1 = has1 ? t0 + 1 : t0;
        const bool acta = !mesh.tri_cv || mesh.tri_cv[ta] < 0;
        const bool actb = has1 && (!mesh.tri_cv || mesh.tri_cv[tb1] < 0);
        auto TE = [&](int e) { return e ? tb1 : ta; };
        auto ACT = [&](int e) { return e ? actb : acta; };
        __syncwarp();
        // the pair's connectivity, staged once: pnt[0..2], seg[3..5], sgn[6..8], and the
        // assembly slots vpos[9..11], spos[12..14]
        if (lane < 30) {
            const int e = lane / 15, k = lane - e * 15, t = TE(e), c = k % 3;
            const int *src = k < 3 ? mesh.tri_pnt : (k < 6 ? mesh.tri_seg : (k < 9 ? mesh.tri_sgn : (k < 12 ? mesh.vpos : mesh.spos)));
            midx[e * M::IDX + k] = src ? src[3 * t + c] : 0;
        }
        __syncwarp();
        // ---- gather (ugtouht, gtol.cpp:14-55) into the PD block, one mode kind per loop so that
        //      the lanes of an iteration take the same branch and read consecutive values: the
        //      vertex values, the side modes (SM NV per side), the interior modes (IM NV per
        //      triangle)
        {
            constexpr int NVX = 2 * 3 * NV, NSD = 2 * 3 * M::SM * NV, NIN = 2 * IM * NV;
#pragma unroll
            for (int it = 0; it < (NVX + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NVX) continue;
                const int e = w / (3 * NV), r = w - e * (3 * NV), m = r / NV, n = r - m * NV;
                PD(e)[n * T + m] = ACT(e) ? st.ugv[midx[e * M::IDX + m] * NV + n] : 0.0;
            }
#pragma unroll
            for (int it = 0; it < (NSD + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NSD) continue;
                const int b = w / (SM * NV), r = w - b * (SM * NV), e = b / 3, i = b - e * 3, kk = r / NV,
                          n = r - kk * NV;
                const int *ix = midx + e * M::IDX;
                double val = ACT(e) ? st.ugs[ix[3 + i] * (SM * NV) + r] : 0.0;
                if ((kk & 1) && ix[6 + i] < 0) val = -val;
                PD(e)[n * T + 3 + i * SM + kk] = val;
            }
#pragma unroll
            for (int it = 0; it < (NIN + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NIN) continue;
                const int e = w / (IMD * NV), r = w - e * (IMD * NV), k = r / NV, n = r - k * NV;
                PD(e)[n * T + BM + k] = ACT(e) ? st.ugi[(size_t)TE(e) * (IMD * NV) + r] : 0.0;
            }
        }
        // geometry of both triangles into the warp's geo block, from the per-triangle
        // constants (Mesh::tgeo: ldcrd(n,0) = (v2-v1)/2, ldcrd(n,1) = (v0-v1)/2, 1 / |J|, and
        // the inscribed-radius length scale of the SUPG tau, tri_mesh/tprims.cpp:224-241)
        if (lane < 2) {
            const double *tg = mesh.tgeo + (size_t)8 * TE(lane);
            double *gg = geo + lane * M::GEO;
            const double icj = tg[4], he = tg[5], ihe = tg[6];
            gg[0] = tg[0]; gg[1] = tg[1]; gg[2] = tg[2]; gg[3] = tg[3];
            gg[4] = mu * icj;
            gg[5] = 2. * (mu / rho) * ihe;
            gg[6] = ph.adis * he * icj;
        }
        __syncwarp();
        // ---- projection on the tensor cores (proj.cpp:22-119 as dense per-point operators)
        {
            double a[M::KS];
#pragma unroll
            for (int ks = 0; ks < M::KS; ++ks) {
                const int m = ks * 4 + gcol;
                a[ks] = (rv < 3 && m < T) ? PD(re_)[rv * T + m] : 0.0;
            }
            __syncwarp();  // the gathered modes are dead: PD takes the derivatives
            const int nop = beta > 0.0 ? 3 : 1;  // derivatives feed the viscous (real) part only
            for (int op = 0; op < nop; ++op) {
                double *dst = op == 0 ? (rv < 3 ? PV(re_) + rv * QP : nullptr)
                                      : (rv < 2 ? PD(re_) + ((op - 1) * 2 + rv) * QP : nullptr);
#pragma unroll
                for (int nt0 = 0; nt0 < M::NT; nt0 += M::NG) {
                    double c[M::NG][2];
#pragma unroll
                    for (int g = 0; g < M::NG; ++g) c[g][0] = c[g][1] = 0.0;
                    const double *b = projB + ((size_t)(op * M::NT + nt0) * M::KS) * 32 + lane;
#pragma unroll
                    for (int ks = 0; ks < M::KS; ++ks)
#pragma unroll
                        for (int g = 0; g < M::NG; ++g)
                            if (nt0 + g < M::NT) dmma884(c[g][0], c[g][1], a[ks], __ldg(b + ((size_t)g * M::KS + ks) * 32));
                    if (dst) {
#pragma unroll
                        for (int g = 0; g < M::NG; ++g)
                            if (nt0 + g < M::NT) {
                                const int q = (nt0 + g) * 8 + gcol * 2;
                                dst[q] = c[g][0];
                                dst[q + 1] = c[g][1];
                            }
                    }
                }
            }
        }
        __syncwarp();
        // ---- pointwise fluxes (ins/rsdl.cpp:259-340), lanes own (triangle, point)
#pragma unroll
        for (int it = 0; it < (2 * GG + 31) / 32; ++it) {
            const int w = lane + 32 * it;
            if (w >= 2 * GG) continue;
            const int e = w / GG, q = w - e * GG;
            const double *gg = geo + e * M::GEO;
            const double d00 = gg[0], d01 = gg[1], d10 = gg[2], d11 = gg[3];
            const double u0 = PV(e)[q], u1 = PV(e)[QP + q], pp = PV(e)[2 * QP + q];
            const double fluxx = rho * u0, fluxy = rho * u1;
            const double m0 = +d11 * fluxx - d01 * fluxy;
            const double m1 = -d10 * fluxx + d00 * fluxy;
            const double c00 = u0 * m0 + d11 * pp, c01 = u0 * m1 - d10 * pp;
            const double c10 = u1 * m0 - d01 * pp, c11 = u1 * m1 + d00 * pp;
            double *fi = FI(e);
            fi[q] = c00;
            fi[GG + q] = c01;
            fi[VS + q] = c10;
            fi[VS + GG + q] = c11;
            fi[2 * VS + q] = m0;
            fi[2 * VS + GG + q] = m1;
            if (beta > 0.0) {
                const double dr0 = PD(e)[q], dr1 = PD(e)[QP + q], ds0 = PD(e)[2 * QP + q], ds1 = PD(e)[3 * QP + q];
                const double cjcbi = gg[4];
                const double v0000 = -cjcbi * (2. * d11 * d11 + d01 * d01);
                const double v0011 = -cjcbi * (2. * d10 * d10 + d00 * d00);
                const double v0001 = cjcbi * (2. * d11 * d10 + d01 * d00);
                const double v1100 = -cjcbi * (d11 * d11 + 2. * d01 * d01);
                const double v1111 = -cjcbi * (d10 * d10 + 2. * d00 * d00);
                const double v1101 = cjcbi * (d11 * d10 + 2. * d01 * d00);
                const double v0100 = cjcbi * d01 * d11;
                const double v0111 = cjcbi * d00 * d10;
                const double v0101 = -cjcbi * d01 * d10;
                const double v0110 = -cjcbi * d00 * d11;
                double *fx = FX(e);
                fx[q] = v0000 * dr0 + v0100 * dr1 + v0001 * ds0 + v0101 * ds1;
                fx[GG + q] = v0001 * dr0 + v0110 * dr1 + v0011 * ds0 + v0111 * ds1;
                fx[VS + q] = v0100 * dr0 + v1100 * dr1 + v0110 * ds0 + v1101 * ds1;
                fx[VS + GG + q] = v0101 * dr0 + v1101 * dr1 + v0111 * ds0 + v1111 * ds1;
                fx[2 * VS + q] = 0.0;
                fx[2 * VS + GG + q] = 0.0;
            }
        }
        __syncwarp();
        // lftog of one fragment (rows (triangle, variable), 2 modes per n-tile): vertex and
        // side modes to the assembly buffers (or atomics), interiors directly
        auto scatter = [&](const double (&c)[M::NT2][2], int part) {
            if (rv >= 3 || !ACT(re_)) return;
            const int t = TE(re_);
            const int *ix = midx + re_ * M::IDX;
#pragma unroll
            for (int nt = 0; nt < M::NT2; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int m = nt * 8 + gcol * 2 + h;
                    if (m >= T) continue;
                    double val = part ? c[nt][h] * beta : c[nt][h];
                    if (m < BM) {
                        int gsi = -1;
                        if (m >= 3) {
                            const int i = (m - 3) / SM, kk = (m - 3) - i * SM;
                            if ((kk & 1) && ix[6 + i] < 0) val = -val;
                            gsi = (ix[3 + i] * SM + kk) * NV + rv;
                        }
                        double *el = part ? st.elre : st.elim;
                        if (el) el[asm_slot(mesh, NV, SM, ix[9 + (m < 3 ? m : 0)], ix[12 + (m < 3 ? 0 : (m - 3) / SM)], m, rv)] = val;
                        else if (gsi < 0) atomicAdd((part ? st.rrv : st.resv) + ix[m] * NV + rv, val);
                        else atomicAdd((part ? st.rrs : st.ress) + gsi, val);
                    } else {
                        const size_t gi = ((size_t)t * IM + (m - BM)) * NV + rv;
                        if (!part) {
                            const double src = st.dresi ? st.dresi[gi] : 0.0;
                            if (beta > 0.0) st.resi[gi] = val + src;
                            else st.resi[gi] = val + st.rri[gi] * omb + src;  // res_r unchanged when beta = 0
                        } else {
                            const double rr = st.rri[gi] * omb + val;
                            st.rri[gi] = rr;
                            st.resi[gi] += rr;
                        }
                    }
                }
        };
        // lftog of both parts of one fragment at once (beta > 0): the slot and the side sign
        // are found once for the imaginary value (-> res) and the beta-scaled real value (->
        // res_r); interiors: res = im + dres + res_r with res_r = (1 - beta) res_r + re
        auto scatter2 = [&](const double (&ci)[M::NT2][2], const double (&cr)[M::NT2][2]) {
            if (rv >= 3 || !ACT(re_)) return;
            const int t = TE(re_);
            const int *ix = midx + re_ * M::IDX;
#pragma unroll
            for (int nt = 0; nt < M::NT2; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int m = nt * 8 + gcol * 2 + h;
                    if (m >= T) continue;
                    double vi = ci[nt][h], vr = cr[nt][h] * beta;
                    if (m < BM) {
                        size_t slot;
                        int g;
                        if (m < 3) {
                            slot = (size_t)ix[9 + m] * NV + rv;
                            g = ix[m] * NV + rv;
                        } else {
                            const int i = (m - 3) / SM, kk = (m - 3) - i * SM;
                            if ((kk & 1) && ix[6 + i] < 0) {
                                vi = -vi;
                                vr = -vr;
                            }
                            slot = (size_t)3 * mesh.ntri * NV + ((size_t)ix[12 + i] * SM + kk) * NV + rv;
                            g = (ix[3 + i] * SM + kk) * NV + rv;
                        }
                        if (st.elim) {
                            st.elim[slot] = vi;
                            st.elre[slot] = vr;
                        } else if (m < 3) {
                            atomicAdd(st.resv + g, vi);
                            atomicAdd(st.rrv + g, vr);
                        } else {
                            atomicAdd(st.ress + g, vi);
                            atomicAdd(st.rrs + g, vr);
                        }
                    } else {
                        const size_t gi = ((size_t)t * IM + (m - BM)) * NV + rv;
                        const double src = st.dresi ? st.dresi[gi] : 0.0;
                        const double rr = st.rri[gi] * omb + vr;
                        st.rri[gi] = rr;
                        st.resi[gi] = (vi + src) + rr;
                    }
                }
        };
        // ---- imaginary part: intgrtrs (intgrt.cpp:81-158, weak divergence with its minus
        //      sign in the operator) on the tensor cores -> res; with a real part (beta > 0)
        //      it is done together with that one below, sharing the operator loads
        if (beta == 0.0) {
            double c[M::NT2][2];
            warp_gemm<M::KS2, M::NT2>(FI(re_) + (rv < 3 ? rv : 2) * VS, intB, gcol, lane, c);
            scatter(c, 0);
        } else {
            // ---- strong residual at the points (derivr + derivs of the full fluxes FI + FX,
            //      proj.cpp:339-402) on the tensor cores as tensor products of the 1D
            //      operators, the point data as the A operand: part 1 rows (triangle, variable,
            //      j), k = q of [fr | fs], columns i: res(i, j) = n0(j) (Ar fr + As1 fs)(i, j);
            //      part 2 rows (triangle, variable, i), k = l of fs, columns j: res(i, j) +=
            //      (As2 fs^T)(j, i); into PD. The operator fragments are B operands here:
            //      lane (g, t) holds A[8 nt + g][4 ks + t] = B[k = t][n = g] of the transpose.
            {
                const double *AR = derB, *AS = derB + M::MT * 2 * M::KR * 32;
                auto col = [&](int n, int &e, int &var, int &j) {
                    e = n / (3 * G);
                    const int rem = n - e * 3 * G;
                    var = rem / G;
                    j = rem - var * G;
                };
                double br[M::MT][2 * M::KR], bs2[M::MT][M::KR];
#pragma unroll
                for (int nt = 0; nt < M::MT; ++nt) {
#pragma unroll
                    for (int ks = 0; ks < 2 * M::KR; ++ks) br[nt][ks] = __ldg(AR + ((size_t)nt * 2 * M::KR + ks) * 32 + lane);
#pragma unroll
                    for (int ks = 0; ks < M::KR; ++ks) bs2[nt][ks] = __ldg(AS + ((size_t)nt * M::KR + ks) * 32 + lane);
                }
                constexpr int MTS = (M::NCOL + 7) / 8;
#pragma unroll
                for (int part = 0; part < 2; ++part) {
#pragma unroll
                    for (int mt = 0; mt < MTS; ++mt) {
                        const int r = mt * 8 + grow;
                        const bool ok = r < M::NCOL;
                        int e, var, x;
                        col(ok ? r : 0, e, var, x);
                        const double *fi = FI(e) + var * VS, *fx = FX(e) + var * VS;
                        double c[M::MT][2];
#pragma unroll
                        for (int nt = 0; nt < M::MT; ++nt) c[nt][0] = c[nt][1] = 0.0;
                        if (part == 0) {
#pragma unroll
                            for (int ks = 0; ks < 2 * M::KR; ++ks) {
                                const int blk = ks / M::KR, q = (ks - blk * M::KR) * 4 + gcol;
                                const int off = blk * GG + q * G + x;
                                const double av = (ok && q < G) ? fi[off] + fx[off] : 0.0;
#pragma unroll
                                for (int nt = 0; nt < M::MT; ++nt) dmma884(c[nt][0], c[nt][1], av, br[nt][ks]);
                            }
                        } else {
#pragma unroll
                            for (int ks = 0; ks < M::KR; ++ks) {
                                const int l = ks * 4 + gcol;
                                const int off = GG + x * G + l;
                                const double av = (ok && l < G) ? fi[off] + fx[off] : 0.0;
#pragma unroll
                                for (int nt = 0; nt < M::MT; ++nt) dmma884(c[nt][0], c[nt][1], av, bs2[nt][ks]);
                            }
                        }
                        if (ok) {
#pragma unroll
                            for (int nt = 0; nt < M::MT; ++nt)
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    const int n = nt * 8 + gcol * 2 + h;
                                    if (n >= G) continue;
                                    if (part == 0) PD(e)[var * QP + n * G + x] = c[nt][h] * tb.n0[x];
                                    else PD(e)[var * QP + x * G + n] += c[nt][h];
                                }
                        }
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            // ---- pointwise SUPG terms (ins/rsdl.cpp:341-431, CALC_TAU2): FX becomes the real
            //      flux pairs, viscous minus SUPG for u, v and the continuity term for p
#pragma unroll
            for (int it = 0; it < (2 * GG + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= 2 * GG) continue;
                const int e = w / GG, q = w - e * GG;
                const double *gg = geo + e * M::GEO;
                const double d00 = gg[0], d01 = gg[1], d10 = gg[2], d11 = gg[3];
                const double u0 = PV(e)[q], u1 = PV(e)[QP + q];
                const double qv = u0 * u0 + u1 * u1;
                const double t2 = gg[5];
                double gam = 3.0 * qv + t2 * t2;
                if (ph.mu + ph.bd0 == 0.0) gam = (gam > 0.1 ? gam : 0.1);
                const double tau0 = gg[6] / sqrt(gam);
                const double tau2 = sqrt(qv) * tau0;
                const double tr0 = tau0 * PD(e)[q], tr1 = tau0 * PD(e)[QP + q], tr2 = tau2 * PD(e)[2 * QP + q];
                double *fx = FX(e);
                fx[q] -= (d11 * (2. * u0) - d01 * u1) * tr0 - d01 * u0 * tr1 + d11 * tr2;
                fx[GG + q] -= (-d10 * (2. * u0) + d00 * u1) * tr0 + d00 * u0 * tr1 - d10 * tr2;
                fx[VS + q] -= +d11 * u1 * tr0 + (d11 * u0 - d01 * (2. * u1)) * tr1 - d01 * tr2;
                fx[VS + GG + q] -= -d10 * u1 * tr0 + (-d10 * u0 + d00 * (2. * u1)) * tr1 + d00 * tr2;
                fx[2 * VS + q] = -(d11 * tr0 - d01 * tr1);
                fx[2 * VS + GG + q] = -(-d10 * tr0 + d00 * tr1);
            }
            __syncwarp();
            // ---- both parts: intgrtrs of the imaginary pairs -> res, and of the viscous + SUPG
            //      pairs, x beta -> res_r
            double ci[M::NT2][2], c[M::NT2][2];
            warp_gemm2<M::KS2, M::NT2>(FI(re_) + (rv < 3 ? rv : 2) * VS, FX(re_) + (rv < 3 ? rv : 2) * VS, intB, gcol,
                                       lane, ci, c);
            scatter2(ci, c);
        }
        __syncwarp();
    }
}

}  // namespace hpb
