// FP32 ins element residual on the tensor cores (TF32 mma.m16n8k8, FP32 accumulation),
// straight triangles, plain or correction form.
//
// The FP32 smoother of the defect correction evaluates the residual in correction form
// R(b + d) - R(b) + R64(u) about the base state b = fp32(u) (tri_hp::mg_source's shape,
// tri_hp/nstage.cpp:113-129, with R64 as the source): the convective and pressure fluxes
// as exact differences F(b + d) - F(b), the viscous flux (linear) of d, the SUPG term with
// the tau of the base. Same element loop and basis operators as the FP64 tensor-core
// kernel (hp_elem_mma.cuh; tri_hp/ins/rsdl.cpp:259-433, proj.cpp:22-119,
// intgrt.cpp:81-158, proj.cpp:339-402), four triangles per warp: the 16 rows of an
// m16n8k8 fragment are (triangle, variable) pairs. The contractions round their
// operands to TF32 (10-bit mantissa) and accumulate in FP32: the smoother's residual is
// accurate to ~1e-3 relative, which the FP64 defect residual absorbs (the converged
// state is the FP64 one). The base state's point values (u, v) are fixed for a whole
// correction cycle and are read from State::bpt (k_base_points) instead of being
// gathered and projected every residual.
#pragma once
#include "hp_kernels.cuh"

namespace hpb {

template <int P>
struct InsTf32 {
    static constexpr int G = P + 1, GG = G * G, T = (P + 1) * (P + 2) / 2, SM = P - 1,
                         IM = (P - 1) * (P - 2) / 2, BM = 3 * P, NV = 3;
    static constexpr int KS = (T + 7) / 8;        // projection k-steps
    static constexpr int NT = (GG + 7) / 8;       // projection n-tiles
    static constexpr int KS2 = (2 * GG + 7) / 8;  // intgrtrs k-steps
    static constexpr int NT2 = (T + 7) / 8;       // intgrtrs n-tiles
    // flux-pair stride 8 (mod 32) floats and triangle stride 4 (mod 32): the 32 A-fragment
    // elements a warp loads at once (8 rows = 2 triangles x 4 variables, 4 columns) fall on
    // distinct banks
    static constexpr int pad_to(int x, int r) { return x + ((r - x % 32) + 32) % 32; }
    static constexpr int VS = pad_to(KS2 * 8, 8);
    static constexpr int QP = NT * 8;
    static constexpr int S_EL = pad_to(7 * QP + 6 * VS, 4);
    static constexpr int WPC = 4;
    static constexpr int MINB = P <= 4 ? 4 : 3;
    static constexpr int NG = NT < 8 ? NT : 8;
    // B fragments: two floats per lane per MMA. DER: the strong residual (derivr + derivs)
    // as tensor products of the 1D operators, transposed so that the point data are the A
    // operand: rows (triangle, variable, point of the other direction), 16 per m-tile, and
    // the operators the B operand, B fragments of [Ar | As1]^T (2 KR k-steps) and As2^T (KR
    // k-steps), NTI n-tiles of 8 operator rows each
    static constexpr size_t PROJ_LEN = (size_t)3 * NT * KS * 64, INT_LEN = (size_t)NT2 * KS2 * 64;
    static constexpr int KR = (G + 7) / 8, NTI = KR, NCOL = 12 * G, MTS = (NCOL + 15) / 16;
    static constexpr size_t DER_LEN = (size_t)3 * KR * NTI * 64;
    static constexpr int IDX = 12;  // staged mesh integers per triangle: pnt[3], seg[3], sgn[3]
    // per triangle: metrics d00, d01, d10, d11, mu / |J|, 2 nu / h, adis h / |J|, unused
    static constexpr int GEO = 8;
    static constexpr size_t SMEM_IDX = (size_t)WPC * 4 * (IDX * sizeof(int) + GEO * sizeof(float));
    static_assert(4 * T <= 4 * QP, "gathered modes must fit the PD block");
    static_assert(2 * NV * T <= 4 * QP, "the staged residual parts must fit the PD block");
};

__device__ __forceinline__ unsigned f2tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, float2 b) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                 "{%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(__float_as_uint(b.x)), "r"(__float_as_uint(b.y)));
}

// Point values (u, v) of the base state b of every triangle, bpt [ntri][2][GG]: the
// projection (proj.cpp:121-186 as dense sums) of the gathered base modes.
template <int P>
__global__ void k_base_points(const DevTables<float, P> *__restrict__ tb, Mesh mesh, const float *__restrict__ ubv,
                              const float *__restrict__ ubs, const float *__restrict__ ubi, float *bpt) {
    constexpr int G = P + 1, GG = G * G, T = (P + 1) * (P + 2) / 2, SM = (P > 1 ? P - 1 : 1),
                  IM = (P - 1) * (P - 2) / 2, BM = 3 * P, NV = 3;
    const long item = (long)blockIdx.x * blockDim.x + threadIdx.x;  // (triangle, variable)
    if (item >= 2L * mesh.ntri) return;
    const int t = (int)(item >> 1), n = (int)(item & 1);
    float lin[T];
#pragma unroll
    for (int m = 0; m < T; ++m) {
        float val;
        if (m < 3) {
            val = ubv[mesh.tri_pnt[3 * t + m] * NV + n];
        } else if (m < BM) {
            const int i = (m - 3) / SM, k = (m - 3) - i * SM;
            val = ubs[(mesh.tri_seg[3 * t + i] * SM + k) * NV + n];
            if ((k & 1) && mesh.tri_sgn[3 * t + i] < 0) val = -val;
        } else {
            val = ubi[((size_t)t * IM + (m - BM)) * NV + n];
        }
        lin[m] = val;
    }
    float *out = bpt + ((size_t)t * 2 + n) * GG;
    for (int q = 0; q < GG; ++q) {
        const int i = q / G, j = q - i * G;
        float acc = 0.f;
#pragma unroll
        for (int m = 0; m < T; ++m) acc += lin[m] * tb->gn[j][m] * tb->gx[i][ModeCols<P>::col(m)];
        out[q] = acc;
    }
}

// C[16 x 8 NTL] of one warp's fragment rows (triangles ra, ra + 2 at variable rv) from
// A rows read in shared memory (a0/a2 from ra0, a1/a3 from ra1, plus the optional second
// rows added in, K padded with zeros) and B in fragment order [nt][ks][lane].
template <int KS, int NTL>
__device__ __forceinline__ void warp_gemm_tf32(const float *ra0, const float *ra1, const float *rb0, const float *rb1,
                                               const float2 *__restrict__ B, int tig, int lane, float (&c)[NTL][4]) {
#pragma unroll
    for (int nt = 0; nt < NTL; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.f;
#pragma unroll 4
    for (int ks = 0; ks < KS; ++ks) {
        const int k = ks * 8 + tig;
        float x0 = ra0[k], x1 = ra1[k], x2 = ra0[k + 4], x3 = ra1[k + 4];
        if (rb0) {
            x0 += rb0[k]; x1 += rb1[k]; x2 += rb0[k + 4]; x3 += rb1[k + 4];
        }
        const unsigned a0 = f2tf32(x0), a1 = f2tf32(x1), a2 = f2tf32(x2), a3 = f2tf32(x3);
#pragma unroll
        for (int nt = 0; nt < NTL; ++nt) mma_tf32(c[nt], a0, a1, a2, a3, __ldg(B + ((size_t)nt * KS + ks) * 32 + lane));
    }
}

// Two products with the same B fragments: Ca from rows (ra0, ra1), Cb from rows (rb0, rb1),
// each B fragment loaded once (the imaginary and the real intgrtrs of the same triangles).
template <int KS, int NTL>
__device__ __forceinline__ void warp_gemm2_tf32(const float *ra0, const float *ra1, const float *rb0, const float *rb1,
                                                const float2 *__restrict__ B, int tig, int lane, float (&ca)[NTL][4],
                                                float (&cb)[NTL][4]) {
#pragma unroll
    for (int nt = 0; nt < NTL; ++nt)
        ca[nt][0] = ca[nt][1] = ca[nt][2] = ca[nt][3] = cb[nt][0] = cb[nt][1] = cb[nt][2] = cb[nt][3] = 0.f;
#pragma unroll 2
    for (int ks = 0; ks < KS; ++ks) {
        const int k = ks * 8 + tig;
        const unsigned a0 = f2tf32(ra0[k]), a1 = f2tf32(ra1[k]), a2 = f2tf32(ra0[k + 4]), a3 = f2tf32(ra1[k + 4]);
        const unsigned b0 = f2tf32(rb0[k]), b1 = f2tf32(rb1[k]), b2 = f2tf32(rb0[k + 4]), b3 = f2tf32(rb1[k + 4]);
#pragma unroll
        for (int nt = 0; nt < NTL; ++nt) {
            const float2 bf = __ldg(B + ((size_t)nt * KS + ks) * 32 + lane);
            mma_tf32(ca[nt], a0, a1, a2, a3, bf);
            mma_tf32(cb[nt], b0, b1, b2, b3, bf);
        }
    }
}

template <int P>
__global__ void __launch_bounds__(InsTf32<P>::WPC * 32, InsTf32<P>::MINB)
    k_rsdl_ins_tf32(const float2 *__restrict__ projB, const float2 *__restrict__ intB,
                    const float2 *__restrict__ derB, InsMmaSmallF<P> small, Mesh mesh, State<float> st, Phys ph,
                    int stage, int zero_rr, int diff) {
    using M = InsTf32<P>;
    constexpr int G = M::G, GG = M::GG, T = M::T, BM = M::BM, IM = M::IM, NV = 3, QP = M::QP, VS = M::VS;
    constexpr int SM = (M::SM > 0 ? M::SM : 1), IMD = (IM > 0 ? IM : 1);  // divisors
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InsMmaSmallF<P> &tb = *reinterpret_cast<InsMmaSmallF<P> *>(smem_raw);
    {
        const int n4 = sizeof(InsMmaSmallF<P>) / 4;
        const int *src = reinterpret_cast<const int *>(&small);
        int *dst = reinterpret_cast<int *>(smem_raw);
        for (int k = threadIdx.x; k < n4; k += blockDim.x) dst[k] = src[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 2, tig = lane & 3;
    const int ra = grp >> 2, rv = grp & 3;  // fragment row grp -> (triangle ra, variable rv); row grp + 8 -> ra + 2
    constexpr size_t SMALL = ((sizeof(InsMmaSmallF<P>) + 15) / 16) * 16;
    float *base = reinterpret_cast<float *>(smem_raw + SMALL) + (size_t)warp * 4 * M::S_EL;
    int *midx = reinterpret_cast<int *>(reinterpret_cast<float *>(smem_raw + SMALL) + (size_t)M::WPC * 4 * M::S_EL) +
                warp * 4 * M::IDX;
    float *geo = reinterpret_cast<float *>(reinterpret_cast<int *>(reinterpret_cast<float *>(smem_raw + SMALL) +
                                                                   (size_t)M::WPC * 4 * M::S_EL) +
                                           M::WPC * 4 * M::IDX) +
                 warp * 4 * M::GEO;
    // per triangle as in k_rsdl_ins_mma: PV u, v, p; PD modes / derivatives / strong
    // residual; FI imaginary flux pairs; FX viscous, then real flux pairs
    auto PV = [&](int e) { return base + e * M::S_EL; };
    auto PD = [&](int e) { return base + e * M::S_EL + 3 * QP; };
    auto FI = [&](int e) { return base + e * M::S_EL + 7 * QP; };
    auto FX = [&](int e) { return base + e * M::S_EL + 7 * QP + 3 * VS; };
    for (int e = 0; e < 4; ++e)
        for (int k = 2 * GG + lane; k < VS; k += 32)
            for (int v = 0; v < 3; ++v) FI(e)[v * VS + k] = FX(e)[v * VS + k] = 0.f;
    __syncthreads();
    const float beta = (float)ph.beta[stage];
    const float omb = zero_rr ? 0.f : 1.f - beta;
    const float rho = (float)ph.rho;
    const bool corr = diff && st.bpt;
    const long ntri = mesh.ntri, nquad = (ntri + 3) / 4;
    const int rvv = rv < 3 ? rv : 2;  // variable slot 3 repeats slot 2 (its rows are discarded)
    for (long pr = (long)blockIdx.x * M::WPC + warp; pr < nquad; pr += (long)gridDim.x * M::WPC) {
        const int t0 = (int)(4 * pr);
        // triangle e of the quad (a missing one repeats the first, unwritten); curved
        // triangles are done by the curved launch
        unsigned actm = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (t0 + e < ntri && (!mesh.tri_cv || mesh.tri_cv[t0 + e] < 0)) actm |= 1u << e;
        auto TE = [&](int e) { return t0 + e < ntri ? t0 + e : t0; };
        auto ACT = [&](int e) { return (actm >> e) & 1u; };
        __syncwarp();
        for (int w = lane; w < 36; w += 32) {  // the quad's connectivity: pnt, seg, sgn
            const int e = w / 9, k = w - e * 9, t = TE(e);
            midx[e * M::IDX + k] = k < 3 ? mesh.tri_pnt[3 * t + k]
                                         : (k < 6 ? mesh.tri_seg[3 * t + k - 3] : mesh.tri_sgn[3 * t + k - 6]);
        }
        __syncwarp();
        if (lane < 4) {  // per-triangle geometry (Mesh::tgeo): ldcrd metrics and the tau length scale
            const double *tg = mesh.tgeo + (size_t)8 * TE(lane);
            float *gg = geo + lane * M::GEO;
            gg[0] = (float)tg[0]; gg[1] = (float)tg[1]; gg[2] = (float)tg[2]; gg[3] = (float)tg[3];
            gg[4] = (float)(ph.mu * tg[4]);
            gg[5] = (float)(2. * (ph.mu / ph.rho) * tg[6]);
            gg[6] = (float)(ph.adis * tg[5] * tg[4]);
        }
        __syncwarp();
        // ---- gather the modes (ugtouht, gtol.cpp:14-55) into the PD block, one mode kind per
        //      loop so that the lanes of an iteration take the same branch: the vertex values,
        //      the side modes (SM NV consecutive values per side), the interior modes (IM NV
        //      consecutive values per triangle)
        {
            constexpr int NVX = 4 * 3 * NV, NSD = 4 * 3 * M::SM * NV, NIN = 4 * IM * NV;
#pragma unroll
            for (int it = 0; it < (NVX + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NVX) continue;
                const int e = w / (3 * NV), r = w - e * (3 * NV), m = r / NV, n = r - m * NV;
                PD(e)[n * T + m] = ACT(e) ? st.ugv[midx[e * M::IDX + m] * NV + n] : 0.f;
            }
#pragma unroll
            for (int it = 0; it < (NSD + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NSD) continue;
                const int b = w / (SM * NV), r = w - b * (SM * NV), e = b / 3, i = b - e * 3, kk = r / NV,
                          n = r - kk * NV;
                const int *ix = midx + e * M::IDX;
                float val = ACT(e) ? st.ugs[ix[3 + i] * (SM * NV) + r] : 0.f;
                if ((kk & 1) && ix[6 + i] < 0) val = -val;
                PD(e)[n * T + 3 + i * SM + kk] = val;
            }
#pragma unroll
            for (int it = 0; it < (NIN + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NIN) continue;
                const int e = w / (IMD * NV), r = w - e * (IMD * NV), k = r / NV, n = r - k * NV;
                PD(e)[n * T + BM + k] = ACT(e) ? st.ugi[(size_t)TE(e) * (IMD * NV) + r] : 0.f;
            }
        }
        __syncwarp();
        // ---- projection (TF32): A rows (triangle, variable), B = dense operators
        {
            unsigned a[M::KS][4];
#pragma unroll
            for (int ks = 0; ks < M::KS; ++ks) {
                const int m0 = ks * 8 + tig, m1 = m0 + 4;
                a[ks][0] = f2tf32((rv < 3 && m0 < T) ? PD(ra)[rv * T + m0] : 0.f);
                a[ks][1] = f2tf32((rv < 3 && m0 < T) ? PD(ra + 2)[rv * T + m0] : 0.f);
                a[ks][2] = f2tf32((rv < 3 && m1 < T) ? PD(ra)[rv * T + m1] : 0.f);
                a[ks][3] = f2tf32((rv < 3 && m1 < T) ? PD(ra + 2)[rv * T + m1] : 0.f);
            }
            __syncwarp();
            const int nop = beta > 0.f ? 3 : 1;
            for (int op = 0; op < nop; ++op) {
                float *d0, *d1;  // destination rows for triangles ra and ra + 2
                if (op == 0) {
                    d0 = rv < 3 ? PV(ra) + rv * QP : nullptr;
                    d1 = rv < 3 ? PV(ra + 2) + rv * QP : nullptr;
                } else {
                    d0 = rv < 2 ? PD(ra) + ((op - 1) * 2 + rv) * QP : nullptr;
                    d1 = rv < 2 ? PD(ra + 2) + ((op - 1) * 2 + rv) * QP : nullptr;
                }
#pragma unroll
                for (int nt0 = 0; nt0 < M::NT; nt0 += M::NG) {
                    float c[M::NG][4];
#pragma unroll
                    for (int g = 0; g < M::NG; ++g) c[g][0] = c[g][1] = c[g][2] = c[g][3] = 0.f;
                    const float2 *b = projB + ((size_t)(op * M::NT + nt0) * M::KS) * 32 + lane;
#pragma unroll
                    for (int ks = 0; ks < M::KS; ++ks)
#pragma unroll
                        for (int g = 0; g < M::NG; ++g)
                            if (nt0 + g < M::NT)
                                mma_tf32(c[g], a[ks][0], a[ks][1], a[ks][2], a[ks][3], __ldg(b + ((size_t)g * M::KS + ks) * 32));
                    if (d0) {
#pragma unroll
                        for (int g = 0; g < M::NG; ++g)
                            if (nt0 + g < M::NT) {
                                const int q = (nt0 + g) * 8 + tig * 2;
                                d0[q] = c[g][0]; d0[q + 1] = c[g][1];
                                d1[q] = c[g][2]; d1[q + 1] = c[g][3];
                            }
                    }
                }
            }
        }
        __syncwarp();
        // ---- pointwise fluxes, lanes own (triangle, point)
#pragma unroll
        for (int it = 0; it < (4 * GG + 31) / 32; ++it) {
            const int w = lane + 32 * it;
            if (w >= 4 * GG) continue;
            const int e = w / GG, q = w - e * GG;
            const int t = TE(e);
            const float *gg = geo + e * M::GEO;
            const float d00 = gg[0], d01 = gg[1], d10 = gg[2], d11 = gg[3];
            const float u0 = PV(e)[q], u1 = PV(e)[QP + q], pp = PV(e)[2 * QP + q];
            const float m0 = +d11 * (rho * u0) - d01 * (rho * u1);
            const float m1 = -d10 * (rho * u0) + d00 * (rho * u1);
            float c00, c01, c10, c11;
            if (corr) {  // F(b + d) - F(b), products expanded
                const float b0 = st.bpt[((size_t)t * 2) * GG + q], b1 = st.bpt[((size_t)t * 2 + 1) * GG + q];
                const float mb0 = +d11 * (rho * b0) - d01 * (rho * b1);
                const float mb1 = -d10 * (rho * b0) + d00 * (rho * b1);
                const float uf0 = b0 + u0, uf1 = b1 + u1;
                c00 = uf0 * m0 + u0 * mb0;
                c01 = uf0 * m1 + u0 * mb1;
                c10 = uf1 * m0 + u1 * mb0;
                c11 = uf1 * m1 + u1 * mb1;
            } else {
                c00 = u0 * m0; c01 = u0 * m1; c10 = u1 * m0; c11 = u1 * m1;
            }
            float *fi = FI(e);
            fi[q] = c00 + d11 * pp;
            fi[GG + q] = c01 - d10 * pp;
            fi[VS + q] = c10 - d01 * pp;
            fi[VS + GG + q] = c11 + d00 * pp;
            fi[2 * VS + q] = m0;
            fi[2 * VS + GG + q] = m1;
            if (beta > 0.f) {
                const float dr0 = PD(e)[q], dr1 = PD(e)[QP + q], ds0 = PD(e)[2 * QP + q], ds1 = PD(e)[3 * QP + q];
                const float cjcbi = gg[4];
                const float v0000 = -cjcbi * (2.f * d11 * d11 + d01 * d01);
                const float v0011 = -cjcbi * (2.f * d10 * d10 + d00 * d00);
                const float v0001 = cjcbi * (2.f * d11 * d10 + d01 * d00);
                const float v1100 = -cjcbi * (d11 * d11 + 2.f * d01 * d01);
                const float v1111 = -cjcbi * (d10 * d10 + 2.f * d00 * d00);
                const float v1101 = cjcbi * (d11 * d10 + 2.f * d01 * d00);
                const float v0100 = cjcbi * d01 * d11;
                const float v0111 = cjcbi * d00 * d10;
                const float v0101 = -cjcbi * d01 * d10;
                const float v0110 = -cjcbi * d00 * d11;
                float *fx = FX(e);
                fx[q] = v0000 * dr0 + v0100 * dr1 + v0001 * ds0 + v0101 * ds1;
                fx[GG + q] = v0001 * dr0 + v0110 * dr1 + v0011 * ds0 + v0111 * ds1;
                fx[VS + q] = v0100 * dr0 + v1100 * dr1 + v0110 * ds0 + v1101 * ds1;
                fx[VS + GG + q] = v0101 * dr0 + v1101 * dr1 + v0111 * ds0 + v1111 * ds1;
                fx[2 * VS + q] = 0.f;
                fx[2 * VS + GG + q] = 0.f;
            }
        }
        __syncwarp();
        // lftog (gtol.cpp:364-402) through shared memory: the lanes' fragment values are staged
        // in the PD block (free after SUPG) as [imaginary | real x beta][variable][mode] per
        // triangle, then scattered one mode kind per loop: vertex and side modes by FP32
        // atomics (imaginary -> res, real -> res_r), interiors directly (two parts: res =
        // im + dres + res_r with res_r = (1 - beta) res_r + re; imaginary only (beta = 0):
        // res = im + (1 - beta) res_r + dres)
        auto scatter = [&](const float (&ci)[M::NT2][4], const float (&cr)[M::NT2][4], bool two) {
            if (rv < 3) {
#pragma unroll
                for (int hh = 0; hh < 2; ++hh)
#pragma unroll
                    for (int nt = 0; nt < M::NT2; ++nt)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int m = nt * 8 + tig * 2 + h;
                            if (m >= T) continue;
                            float *d = PD(ra + 2 * hh) + rv * T + m;
                            d[0] = ci[nt][2 * hh + h];
                            if (two) d[NV * T] = cr[nt][2 * hh + h] * beta;
                        }
            }
            __syncwarp();
            constexpr int NVX = 4 * 3 * NV, NSD = 4 * 3 * M::SM * NV, NIN = 4 * IM * NV;
#pragma unroll
            for (int it = 0; it < (NVX + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NVX) continue;
                const int e = w / (3 * NV), r = w - e * (3 * NV), m = r / NV, n = r - m * NV;
                if (!ACT(e)) continue;
                const int g = midx[e * M::IDX + m] * NV + n;
                atomicAdd(st.resv + g, PD(e)[n * T + m]);
                if (two) atomicAdd(st.rrv + g, PD(e)[NV * T + n * T + m]);
            }
#pragma unroll
            for (int it = 0; it < (NSD + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NSD) continue;
                const int b = w / (SM * NV), r = w - b * (SM * NV), e = b / 3, i = b - e * 3, kk = r / NV,
                          n = r - kk * NV;
                if (!ACT(e)) continue;
                const int *ix = midx + e * M::IDX;
                const int m = 3 + i * SM + kk, g = ix[3 + i] * (SM * NV) + r;
                const bool flip = (kk & 1) && ix[6 + i] < 0;
                const float vi = PD(e)[n * T + m];
                atomicAdd(st.ress + g, flip ? -vi : vi);
                if (two) {
                    const float vr = PD(e)[NV * T + n * T + m];
                    atomicAdd(st.rrs + g, flip ? -vr : vr);
                }
            }
#pragma unroll
            for (int it = 0; it < (NIN + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= NIN) continue;
                const int e = w / (IMD * NV), r = w - e * (IMD * NV), k = r / NV, n = r - k * NV;
                if (!ACT(e)) continue;
                const size_t gi = (size_t)TE(e) * (IMD * NV) + r;
                const float vi = PD(e)[n * T + BM + k];
                const float src = st.dresi ? st.dresi[gi] : 0.f;
                if (two) {
                    const float rr = st.rri[gi] * omb + PD(e)[NV * T + n * T + BM + k];
                    st.rri[gi] = rr;
                    st.resi[gi] = (vi + src) + rr;
                } else {
                    st.resi[gi] = vi + st.rri[gi] * omb + src;
                }
            }
        };
        // imaginary part -> res; with a real part (beta > 0) it is done together with that one
        // below, sharing the operator loads
        if (beta == 0.f) {
            float c[M::NT2][4];
            warp_gemm_tf32<M::KS2, M::NT2>(FI(ra) + rvv * VS, FI(ra + 2) + rvv * VS, nullptr, nullptr, intB, tig,
                                            lane, c);
            scatter(c, c, false);
        } else {
            // ---- strong residual of FI + FX at the points (derivr / derivs, proj.cpp:339-402)
            //      on TF32 as tensor products of the 1D operators, the point data as the A
            //      operand: part 1 rows (triangle, variable, j), k = q of [fr | fs], columns i:
            //      res(i, j) = n0(j) (Ar fr + As1 fs)(i, j); part 2 rows (triangle, variable, i),
            //      k = l of fs, columns j: res(i, j) += (As2 fs^T)(j, i); into PD
            {
                auto col = [&](int n, int &e, int &var, int &j) {
                    e = n / (3 * G);
                    const int rem = n - e * 3 * G;
                    var = rem / G;
                    j = rem - var * G;
                };
                // the B fragments of the transposed 1D operators, the same for every m-tile
                float2 bop[3 * M::KR][M::NTI];
#pragma unroll
                for (int k = 0; k < 3 * M::KR; ++k)
#pragma unroll
                    for (int nt = 0; nt < M::NTI; ++nt) bop[k][nt] = __ldg(derB + ((size_t)k * M::NTI + nt) * 32 + lane);
#pragma unroll
                for (int part = 0; part < 2; ++part) {
                    const int nks = part ? M::KR : 2 * M::KR;
#pragma unroll
                    for (int mt = 0; mt < M::MTS; ++mt) {
                        const int r0 = mt * 16 + grp, r1 = r0 + 8;
                        const bool ok0 = r0 < M::NCOL, ok1 = r1 < M::NCOL;
                        int e0, v0, x0, e1, v1, x1;
                        col(ok0 ? r0 : 0, e0, v0, x0);
                        col(ok1 ? r1 : 0, e1, v1, x1);
                        const float *fi0 = FI(e0) + v0 * VS, *fx0 = FX(e0) + v0 * VS;
                        const float *fi1 = FI(e1) + v1 * VS, *fx1 = FX(e1) + v1 * VS;
                        float c[M::NTI][4];
#pragma unroll
                        for (int nt = 0; nt < M::NTI; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.f;
#pragma unroll
                        for (int ks = 0; ks < nks; ++ks) {
                            // the offsets of (row, k) in its flux block: k = q (part 1) of
                            // [fr | fs] at point x, or k = l (part 2) of fs at point x
                            int o00, o10, o01, o11;
                            bool k0, k1;
                            if (part == 0) {
                                const int blk = ks / M::KR, q0 = (ks - blk * M::KR) * 8 + tig, q1 = q0 + 4;
                                k0 = q0 < G;
                                k1 = q1 < G;
                                o00 = blk * GG + q0 * G + x0; o10 = blk * GG + q0 * G + x1;
                                o01 = blk * GG + q1 * G + x0; o11 = blk * GG + q1 * G + x1;
                            } else {
                                const int l0 = ks * 8 + tig, l1 = l0 + 4;
                                k0 = l0 < G;
                                k1 = l1 < G;
                                o00 = GG + x0 * G + l0; o10 = GG + x1 * G + l0;
                                o01 = GG + x0 * G + l1; o11 = GG + x1 * G + l1;
                            }
                            const unsigned a0 = f2tf32((ok0 && k0) ? fi0[o00] + fx0[o00] : 0.f);
                            const unsigned a1 = f2tf32((ok1 && k0) ? fi1[o10] + fx1[o10] : 0.f);
                            const unsigned a2 = f2tf32((ok0 && k1) ? fi0[o01] + fx0[o01] : 0.f);
                            const unsigned a3 = f2tf32((ok1 && k1) ? fi1[o11] + fx1[o11] : 0.f);
#pragma unroll
                            for (int nt = 0; nt < M::NTI; ++nt)
                                mma_tf32(c[nt], a0, a1, a2, a3, bop[(part ? 2 * M::KR : 0) + ks][nt]);
                        }
                        // c[nt][h]: row r0, operator row nt * 8 + 2 tig + h; c[nt][2 + h]: row r1
#pragma unroll
                        for (int nt = 0; nt < M::NTI; ++nt)
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                const int n = nt * 8 + 2 * tig + h;
                                if (n >= G) continue;
                                if (part == 0) {
                                    if (ok0) PD(e0)[v0 * QP + n * G + x0] = c[nt][h] * tb.n0[x0];
                                    if (ok1) PD(e1)[v1 * QP + n * G + x1] = c[nt][2 + h] * tb.n0[x1];
                                } else {
                                    if (ok0) PD(e0)[v0 * QP + x0 * G + n] += c[nt][h];
                                    if (ok1) PD(e1)[v1 * QP + x1 * G + n] += c[nt][2 + h];
                                }
                            }
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            // ---- SUPG with tau of the base state (correction form) or of the state (plain)
#pragma unroll
            for (int it = 0; it < (4 * GG + 31) / 32; ++it) {
                const int w = lane + 32 * it;
                if (w >= 4 * GG) continue;
                const int e = w / GG, q = w - e * GG;
                const int t = TE(e);
                const float *gg = geo + e * M::GEO;
                const float d00 = gg[0], d01 = gg[1], d10 = gg[2], d11 = gg[3];
                float u0 = PV(e)[q], u1 = PV(e)[QP + q], qv;
                if (corr) {
                    const float b0 = st.bpt[((size_t)t * 2) * GG + q], b1 = st.bpt[((size_t)t * 2 + 1) * GG + q];
                    qv = b0 * b0 + b1 * b1;
                    u0 += b0;
                    u1 += b1;
                } else {
                    qv = u0 * u0 + u1 * u1;
                }
                const float t2 = gg[5];
                float gam = 3.0f * qv + t2 * t2;
                if (ph.mu + ph.bd0 == 0.0) gam = (gam > 0.1f ? gam : 0.1f);
                const float tau0 = gg[6] * rsqrtf(gam);
                const float tau2 = sqrtf(qv) * tau0;
                const float tr0 = tau0 * PD(e)[q], tr1 = tau0 * PD(e)[QP + q], tr2 = tau2 * PD(e)[2 * QP + q];
                float *fr = FX(e);
                fr[q] -= (d11 * (2.f * u0) - d01 * u1) * tr0 - d01 * u0 * tr1 + d11 * tr2;
                fr[GG + q] -= (-d10 * (2.f * u0) + d00 * u1) * tr0 + d00 * u0 * tr1 - d10 * tr2;
                fr[VS + q] -= +d11 * u1 * tr0 + (d11 * u0 - d01 * (2.f * u1)) * tr1 - d01 * tr2;
                fr[VS + GG + q] -= -d10 * u1 * tr0 + (-d10 * u0 + d00 * (2.f * u1)) * tr1 + d00 * tr2;
                fr[2 * VS + q] = -(d11 * tr0 - d01 * tr1);
                fr[2 * VS + GG + q] = -(-d10 * tr0 + d00 * tr1);
            }
            __syncwarp();
            float ci[M::NT2][4], c[M::NT2][4];
            warp_gemm2_tf32<M::KS2, M::NT2>(FI(ra) + rvv * VS, FI(ra + 2) + rvv * VS, FX(ra) + rvv * VS,
                                             FX(ra + 2) + rvv * VS, intB, tig, lane, ci, c);
            scatter(ci, c, true);
        }
        __syncwarp();
    }
}

}  // namespace hpb
