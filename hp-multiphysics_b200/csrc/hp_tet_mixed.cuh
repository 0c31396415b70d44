// FP32 smoothing of the 3D (tet_hp ins) path inside FP64 defect correction.
//
// Included by hp_tet.cu after the FP64 kernels (it uses TetCfg, TetSmall, TetMeshD,
// TetFields, mode_slot and NV from there). The FP32 smoother works on a correction d about
// the base state b = fp32(u) of each level, with the residual in correction form
//   R(b + d) - R(b) + s
// (s: the FP64 residual R64(u) on the finest level, the FAS source on coarser ones; the
// shape of tet_hp::rsdl's coarse-level driving term, tet_hp/update.cpp:97-117):
//   * convective flux as the exact difference (b + d)_n f(d) + d_n f(b), f the mass flux
//     rho (u . adj J) (linear), pressure and viscous fluxes of d (linear), SUPG with the
//     base state's tau (tet_hp_ins::setup_preconditioner at the base) and velocity b + d;
//   * the inflow faces' continuity flux rho d . n (linear);
//   * tet_hp::rsdl's element loop on the tensor cores in TF32 (mma.m16n8k8, FP32
//     accumulation): four tetrahedra per warp, the 16 rows of a fragment being
//     (tetrahedron, variable) pairs; projection U[16 x T] Op^T[T x Q] for Op = F, DX, DY,
//     DZ and intgrtrst Flux[16 x 3Q] (w D)[3Q x T] as in the FP64 kernel; pointwise
//     fluxes, the strong residual (1D operators along the collapsed directions) and SUPG
//     scalar in FP32.
// The converged state is the FP64 one: convergence is judged by the FP64 residual.
#pragma once

template <int P>
struct TetTf32 {
    using C = TetCfg<P>;
    static constexpr int G = C::G, Q = C::Q, T = C::T;
    static constexpr int KS = (T + 7) / 8;        // projection k-steps
    static constexpr int NT = (Q + 7) / 8;        // projection n-tiles
    static constexpr int KS2 = (3 * Q + 7) / 8;   // intgrtrst k-steps
    static constexpr int NT2 = (T + 7) / 8;       // intgrtrst n-tiles
    static constexpr int pad_to(int x, int r) { return x + ((r - x % 32) + 32) % 32; }
    // flux stride 8 (mod 32) floats, tetrahedron stride 4 (mod 32): the A-fragment loads of
    // (2 tetrahedra x 4 variables) x 4 columns fall on distinct banks
    static constexpr int VS = pad_to(KS2 * 8, 8);
    static constexpr int QP = NT * 8;
    // per tetrahedron: u [3][QP] (u, v, w of d), fim [NV][VS], fre [NV][VS] (fre's
    // variable-3 slot holds the gathered modes, then the pressure of d at the points)
    static constexpr int S_EL = pad_to(3 * QP + 2 * NV * VS, 4);
    static constexpr int WPC = 2;
    static constexpr int GEO = 12;  // per tetrahedron: the 9 metrics d(c, k) and |J|
    static constexpr int NG = NT < 8 ? NT : 8;
    static constexpr size_t PROJ_LEN = (size_t)4 * NT * KS * 64, INT_LEN = (size_t)NT2 * KS2 * 64;
    static constexpr size_t SMEM = (size_t)WPC * (4 * S_EL + 4 * GEO) * sizeof(float);
    static_assert(NV * T <= VS && Q <= VS, "modes / pressure must fit fre's variable-3 slot");
    static_assert(2 * T <= VS, "the staged residual parts must fit the fim block");
};

__device__ __forceinline__ unsigned tet_tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void tet_mma_tf32(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                             float2 b) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                 "{%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(__float_as_uint(b.x)), "r"(__float_as_uint(b.y)));
}

// tet_hp::rsdl's element loop in correction form on TF32 (see the file comment). res and rr
// are the FP32 correction residual arrays (pre-zeroed / pre-scaled by k_tet_pre).
template <int P>
__global__ void __launch_bounds__(TetTf32<P>::WPC * 32)
    k_tet_rsdl_tf32(const float2 *__restrict__ projB, const float2 *__restrict__ intB, TetSmall<float, P> sm,
                    TetMeshD mesh, TetFields<float> ug, TetFields<float> res, TetFields<float> rr,
                    const float *__restrict__ tau, const float *__restrict__ bpt, float rho, float mu, float beta) {
    using C = TetCfg<P>;
    using M = TetTf32<P>;
    constexpr int G = C::G, Q = C::Q, T = C::T, QP = M::QP, VS = M::VS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 2, tig = lane & 3;
    const int ra = grp >> 2, rv = grp & 3;  // fragment row grp -> (tetrahedron ra, variable rv); grp + 8 -> ra + 2
    float *base = reinterpret_cast<float *>(smem_raw) + (size_t)warp * (4 * M::S_EL + 4 * M::GEO);
    float *geo = base + 4 * M::S_EL;
    auto UQ = [&](int e) { return base + e * M::S_EL; };
    auto FIM = [&](int e) { return base + e * M::S_EL + 3 * QP; };
    auto FRE = [&](int e) { return base + e * M::S_EL + 3 * QP + NV * VS; };
    auto PV = [&](int e) { return FRE(e) + 3 * VS; };  // the modes, then the pressure of d
    for (int e = 0; e < 4; ++e)
        for (int k = 3 * Q + lane; k < VS; k += 32)
            for (int n = 0; n < NV; ++n) FIM(e)[n * VS + k] = FRE(e)[n * VS + k] = 0.f;
    __syncwarp();
    const long ntet = mesh.ntet, nquad = (ntet + 3) / 4;
    for (long pr = (long)blockIdx.x * M::WPC + warp; pr < nquad; pr += (long)gridDim.x * M::WPC) {
        const int t0 = (int)(4 * pr);
        auto TE = [&](int e) { return t0 + e < ntet ? t0 + e : t0; };
        auto ACT = [&](int e) { return t0 + e < ntet; };
        __syncwarp();
        // ---- gather d (ugtouht) into the variable-3 slot of fre
        tet_gather_kinds<float, P, 4>(mesh, ug, lane, TE, ACT, PV);
        // ---- geometry of the four tetrahedra (lanes 0..3): d(c, k) = the cofactors of
        //      ldcrd, |J| (tet_hp/ins/rsdl.cpp straight branch)
        if (lane < 4) {
            const int t = TE(lane);
            const int v0 = mesh.tp[4 * t], v1 = mesh.tp[4 * t + 1], v2 = mesh.tp[4 * t + 2], v3 = mesh.tp[4 * t + 3];
            double ld[3][3];
            for (int n = 0; n < 3; ++n) {
                const double c2 = mesh.pnts[3 * v2 + n];
                ld[n][0] = 0.5 * (mesh.pnts[3 * v3 + n] - c2);
                ld[n][1] = 0.5 * (mesh.pnts[3 * v1 + n] - c2);
                ld[n][2] = 0.5 * (mesh.pnts[3 * v0 + n] - c2);
            }
            float *g = geo + lane * M::GEO;
            g[0] = (float)(ld[1][1] * ld[2][2] - ld[1][2] * ld[2][1]);
            g[1] = (float)(-ld[0][1] * ld[2][2] + ld[0][2] * ld[2][1]);
            g[2] = (float)(ld[0][1] * ld[1][2] - ld[0][2] * ld[1][1]);
            g[3] = (float)(-ld[1][0] * ld[2][2] + ld[1][2] * ld[2][0]);
            g[4] = (float)(ld[0][0] * ld[2][2] - ld[0][2] * ld[2][0]);
            g[5] = (float)(-ld[0][0] * ld[1][2] + ld[0][2] * ld[1][0]);
            g[6] = (float)(ld[1][0] * ld[2][1] - ld[1][1] * ld[2][0]);
            g[7] = (float)(-ld[0][0] * ld[2][1] + ld[0][1] * ld[2][0]);
            g[8] = (float)(ld[0][0] * ld[1][1] - ld[0][1] * ld[1][0]);
            g[9] = (float)(ld[0][0] * (ld[1][1] * ld[2][2] - ld[1][2] * ld[2][1]) -
                           ld[0][1] * (ld[1][0] * ld[2][2] - ld[2][0] * ld[1][2]) +
                           ld[0][2] * (ld[1][0] * ld[2][1] - ld[2][0] * ld[1][1]));
        }
        __syncwarp();
        // ---- projection (TF32): rows (tetrahedron, variable)
        {
            unsigned a[M::KS][4];
#pragma unroll
            for (int ks = 0; ks < M::KS; ++ks) {
                const int m0 = ks * 8 + tig, m1 = m0 + 4;
                a[ks][0] = tet_tf32(m0 < T ? PV(ra)[rv * T + m0] : 0.f);
                a[ks][1] = tet_tf32(m0 < T ? PV(ra + 2)[rv * T + m0] : 0.f);
                a[ks][2] = tet_tf32(m1 < T ? PV(ra)[rv * T + m1] : 0.f);
                a[ks][3] = tet_tf32(m1 < T ? PV(ra + 2)[rv * T + m1] : 0.f);
            }
            __syncwarp();  // the modes are dead: the slot takes the pressure values
            for (int op = 0; op < (beta > 0.f ? 4 : 1); ++op) {
                float *d0, *d1;
                if (op == 0) {
                    d0 = rv < 3 ? UQ(ra) + rv * QP : PV(ra);
                    d1 = rv < 3 ? UQ(ra + 2) + rv * QP : PV(ra + 2);
                } else {
                    d0 = rv < 3 ? FRE(ra) + rv * VS + (op - 1) * Q : nullptr;
                    d1 = rv < 3 ? FRE(ra + 2) + rv * VS + (op - 1) * Q : nullptr;
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
                                tet_mma_tf32(c[g], a[ks][0], a[ks][1], a[ks][2], a[ks][3],
                                             __ldg(b + ((size_t)g * M::KS + ks) * 32));
                    if (d0) {
#pragma unroll
                        for (int g = 0; g < M::NG; ++g) {
                            const int q = (nt0 + g) * 8 + tig * 2;
                            if (nt0 + g < M::NT && q < Q) {
                                d0[q] = c[g][0]; d1[q] = c[g][2];
                                if (q + 1 < Q) { d0[q + 1] = c[g][1]; d1[q + 1] = c[g][3]; }
                            }
                        }
                    }
                }
            }
        }
        __syncwarp();
        // ---- pointwise fluxes, lanes own (tetrahedron, point): fim = convective + pressure
        //      in correction form / continuity; fre = viscous flux of d
        for (int w = lane; w < 4 * Q; w += 32) {
            const int e = w / Q, q = w - e * Q, t = TE(e);
            const float *g = geo + e * M::GEO;
            float d[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 3; ++k) d[c][k] = g[3 * c + k];
            const float *uq = UQ(e);
            float *fim = FIM(e), *fre = FRE(e);
            const float uu[3] = {uq[q], uq[QP + q], uq[2 * QP + q]};
            const float pp = PV(e)[q];
            float ub[3];
#pragma unroll
            for (int n = 0; n < 3; ++n) ub[n] = bpt[((size_t)t * 3 + n) * Q + q];
            float f3[3], fb[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                f3[c] = d[c][0] * (rho * uu[0]) + d[c][1] * (rho * uu[1]) + d[c][2] * (rho * uu[2]);
                fb[c] = d[c][0] * (rho * ub[0]) + d[c][1] * (rho * ub[1]) + d[c][2] * (rho * ub[2]);
                fim[3 * VS + c * Q + q] = f3[c];
            }
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    fim[n * VS + c * Q + q] = (ub[n] + uu[n]) * f3[c] + uu[n] * fb[c] + d[c][n] * pp;
            if (beta > 0.f) {
                float du[3][3];
#pragma unroll
                for (int n = 0; n < 3; ++n)
#pragma unroll
                    for (int c = 0; c < 3; ++c) du[n][c] = fre[n * VS + c * Q + q];
                const float cjcbi = mu / g[9];
                float h[3][3];
#pragma unroll
                for (int b = 0; b < 3; ++b)
#pragma unroll
                    for (int a2 = 0; a2 < 3; ++a2)
                        h[b][a2] = d[0][a2] * du[b][0] + d[1][a2] * du[b][1] + d[2][a2] * du[b][2];
#pragma unroll
                for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float s = 0.f;
#pragma unroll
                        for (int ee = 0; ee < 3; ++ee) {
                            const float gce = d[c][0] * d[ee][0] + d[c][1] * d[ee][1] + d[c][2] * d[ee][2];
                            s += gce * du[a2][ee];
                        }
                        s += d[c][0] * h[0][a2] + d[c][1] * h[1][a2] + d[c][2] * h[2][a2];
                        fre[a2 * VS + c * Q + q] = -cjcbi * s;
                    }
            }
        }
        __syncwarp();
        if (beta > 0.f) {
            // ---- strong residual of the full fluxes at the owned points
            constexpr int NW = (4 * Q + 31) / 32;
            float rsd[NW][NV];
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                const int w = lane + 32 * k;
                if (w >= 4 * Q) break;
                const int e = w / Q, q = w - e * Q;
                const int i = q / (G * G), j = (q / G) % G, kk = q % G;
                const float yz = sm.y0[j] * sm.z0[kk], zz = sm.z0[kk];
                const float *fim = FIM(e), *fre = FRE(e);
#pragma unroll
                for (int n = 0; n < NV; ++n) {
                    auto fl = [&](int c, int i2, int j2, int k2) -> float {
                        const int q2 = (i2 * G + j2) * G + k2;
                        return n < 3 ? fim[n * VS + c * Q + q2] + fre[n * VS + c * Q + q2] : fim[3 * VS + c * Q + q2];
                    };
                    float ax = 0, bxs = 0, bxt = 0, ays = 0, byt = 0, azt = 0;
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
            // ---- SUPG with the base's tau and the velocity b + d
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                const int w = lane + 32 * k;
                if (w >= 4 * Q) break;
                const int e = w / Q, q = w - e * Q, t = TE(e);
                const float *g = geo + e * M::GEO;
                float d[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int kk2 = 0; kk2 < 3; ++kk2) d[c][kk2] = g[3 * c + kk2];
                const float tau0 = tau[2 * t], tau3 = tau[2 * t + 1];
                float *fre = FRE(e);
                const float *uq = UQ(e);
                float tr[NV], uu[3];
#pragma unroll
                for (int n = 0; n < 3; ++n) {
                    tr[n] = tau0 * rsd[k][n];
                    uu[n] = uq[n * QP + q] + bpt[((size_t)t * 3 + n) * Q + q];
                }
                tr[3] = tau3 * rsd[k][3];
#pragma unroll
                for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float s2 = d[c][a2] * (2.f * uu[a2]);
#pragma unroll
                        for (int b = 0; b < 3; ++b)
                            if (b != a2) s2 += d[c][b] * uu[b];
                        float r = s2 * tr[a2];
#pragma unroll
                        for (int b = 0; b < 3; ++b)
                            if (b != a2) r += d[c][b] * uu[a2] * tr[b];
                        r += d[c][a2] * tr[3];
                        fre[a2 * VS + c * Q + q] -= r;
                    }
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    fre[3 * VS + c * Q + q] = -d[c][0] * tr[0] - d[c][1] * tr[1] - d[c][2] * tr[2];
            }
            __syncwarp();
        }
        // ---- intgrtrst on TF32 (imaginary into res, real * beta into res_r); lftog
        {
            // with a real part both products share each operator fragment load
            const bool two = beta > 0.f;
            const float *i0 = FIM(ra) + rv * VS, *i1 = FIM(ra + 2) + rv * VS;
            const float *q0 = FRE(ra) + rv * VS, *q1 = FRE(ra + 2) + rv * VS;
            float ci[M::NT2][4], cr[M::NT2][4];
#pragma unroll
            for (int nt = 0; nt < M::NT2; ++nt)
                ci[nt][0] = ci[nt][1] = ci[nt][2] = ci[nt][3] = cr[nt][0] = cr[nt][1] = cr[nt][2] = cr[nt][3] = 0.f;
#pragma unroll 2
            for (int ks = 0; ks < M::KS2; ++ks) {
                const int k = ks * 8 + tig;
                const unsigned a0 = tet_tf32(i0[k]), a1 = tet_tf32(i1[k]), a2 = tet_tf32(i0[k + 4]),
                               a3 = tet_tf32(i1[k + 4]);
                unsigned b0 = 0, b1 = 0, b2 = 0, b3 = 0;
                if (two) {
                    b0 = tet_tf32(q0[k]); b1 = tet_tf32(q1[k]); b2 = tet_tf32(q0[k + 4]); b3 = tet_tf32(q1[k + 4]);
                }
#pragma unroll
                for (int nt = 0; nt < M::NT2; ++nt) {
                    const float2 bf = __ldg(intB + ((size_t)nt * M::KS2 + ks) * 32 + lane);
                    tet_mma_tf32(ci[nt], a0, a1, a2, a3, bf);
                    if (two) tet_mma_tf32(cr[nt], b0, b1, b2, b3, bf);
                }
            }
            // lftog (tet_hp/gtol.cpp) through shared memory: the lanes' values (-intgrtrst) are
            // staged in the fim block (free once every lane's products are done) as
            // [imaginary | real][variable][mode] per tetrahedron, then added one mode kind per
            // loop: vertex, edge and face modes by FP32 atomics (imaginary -> res, real x beta
            // -> res_r), interiors directly (res = im, res_r += beta re)
            __syncwarp();
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
#pragma unroll
                for (int nt = 0; nt < M::NT2; ++nt)
#pragma unroll
                    for (int h2 = 0; h2 < 2; ++h2) {
                        const int m = nt * 8 + tig * 2 + h2;
                        if (m >= T) continue;
                        float *d = FIM(ra + 2 * hh) + rv * T + m;
                        d[0] = -ci[nt][2 * hh + h2];
                        if (two) d[NV * T] = -cr[nt][2 * hh + h2];
                    }
            __syncwarp();
            {
                constexpr int EM = C::EM, FM = C::FM, IM = C::IM;
                constexpr int EMD = EM > 0 ? EM : 1, FMD = FM > 0 ? FM : 1, IMD = IM > 0 ? IM : 1;
                constexpr int NVX = 4 * 4 * NV, NED = 4 * 6 * EM * NV, NFC = 4 * 4 * FM * NV, NIN = 4 * IM * NV;
                auto VI = [&](int e, int n, int m) { return FIM(e)[n * T + m]; };
                auto VR = [&](int e, int n, int m) { return FIM(e)[NV * T + n * T + m]; };
#pragma unroll
                for (int it = 0; it < (NVX + 31) / 32; ++it) {
                    const int w = lane + 32 * it;
                    if (w >= NVX) continue;
                    const int e = w / (4 * NV), r = w - e * (4 * NV), m = r / NV, n = r - m * NV;
                    if (!ACT(e)) continue;
                    const size_t g = (size_t)mesh.tp[4 * TE(e) + m] * NV + n;
                    atomicAdd(res.v + g, VI(e, n, m));
                    if (two) atomicAdd(rr.v + g, beta * VR(e, n, m));
                }
#pragma unroll
                for (int it = 0; it < (NED + 31) / 32; ++it) {
                    const int w = lane + 32 * it;
                    if (w >= NED) continue;
                    const int b = w / (EMD * NV), r = w - b * (EMD * NV), e = b / 6, i = b - e * 6, k = r / NV,
                              n = r - k * NV;
                    if (!ACT(e)) continue;
                    const int t = TE(e), m = 4 + i * EMD + k;
                    const float sg = ((k & 1) && mesh.tsg[6 * t + i] < 0) ? -1.f : 1.f;
                    const size_t g = (size_t)mesh.ts[6 * t + i] * (EMD * NV) + r;
                    atomicAdd(res.e + g, sg * VI(e, n, m));
                    if (two) atomicAdd(rr.e + g, beta * sg * VR(e, n, m));
                }
#pragma unroll
                for (int it = 0; it < (NFC + 31) / 32; ++it) {
                    const int w = lane + 32 * it;
                    if (w >= NFC) continue;
                    const int b = w / (FMD * NV), r = w - b * (FMD * NV), e = b / 4, i = b - e * 4, idx = r / NV,
                              n = r - idx * NV;
                    if (!ACT(e)) continue;
                    const int t = TE(e), m = 4 + 6 * EM + i * FMD + idx;
                    const float sg = (((face_mode_row<EM>(idx) - 1) & 1) && mesh.trot[4 * t + i] > 0) ? -1.f : 1.f;
                    const size_t g = (size_t)mesh.tt[4 * t + i] * (FMD * NV) + r;
                    atomicAdd(res.f + g, sg * VI(e, n, m));
                    if (two) atomicAdd(rr.f + g, beta * sg * VR(e, n, m));
                }
#pragma unroll
                for (int it = 0; it < (NIN + 31) / 32; ++it) {
                    const int w = lane + 32 * it;
                    if (w >= NIN) continue;
                    const int e = w / (IMD * NV), r = w - e * (IMD * NV), k = r / NV, n = r - k * NV;
                    if (!ACT(e)) continue;
                    const size_t g = (size_t)TE(e) * (IMD * NV) + r;
                    res.i[g] = VI(e, n, C::BM + k);
                    if (two) rr.i[g] += beta * VR(e, n, C::BM + k);
                }
            }
        }
        __syncwarp();
    }
}

// Point values (u, v, w) of the base state of every tetrahedron, bpt [ntet][3][Q]:
// tet_basis::proj of the gathered base modes with the dense value operator F [Q][T].
template <int P>
__global__ void k_tet_base_points(const float *__restrict__ F, TetMeshD mesh, TetFields<float> ub, float *bpt) {
    using C = TetCfg<P>;
    constexpr int Q = C::Q, T = C::T;
    const long item = (long)blockIdx.x * blockDim.x + threadIdx.x;  // (tetrahedron, variable)
    if (item >= 3L * mesh.ntet) return;
    const int t = (int)(item / 3), n = (int)(item - 3L * (item / 3));
    float lin[T];
#pragma unroll
    for (int m = 0; m < T; ++m) {
        float s;
        const float *src = mode_slot<float, P>(mesh, ub, t, m, n, s);
        lin[m] = s * *src;
    }
    float *out = bpt + ((size_t)t * 3 + n) * Q;
    for (int q = 0; q < Q; ++q) {
        float acc = 0.f;
#pragma unroll
        for (int m = 0; m < T; ++m) acc += lin[m] * __ldg(F + q * T + m);
        out[q] = acc;
    }
}

// Continuity flux rho d . n of the inflow faces (bdry_ins::inflow, tet_hp/ins/bdry.cpp:16-102;
// linear in the state, so the correction form is the flux of d): one warp per face, FP32.
template <int P>
__global__ void __launch_bounds__(128) k_tet_face_flux32(TetFacesD fc, const double *__restrict__ ftab, TetMeshD mesh,
                                                         TetFields<float> u, TetFields<float> res, float rho) {
    constexpr int G = P + 1, G2 = G * G, EM = P - 1, FM = (P - 1) * (P - 2) / 2, T2 = 3 + 3 * EM + FM;
    constexpr int EMD = EM > 0 ? EM : 1, FMD = FM > 0 ? FM : 1, WPB = 4;
    __shared__ float sflx[WPB][G2];
    const double *F2 = ftab, *DX2 = ftab + G2 * T2, *DY2 = ftab + 2 * G2 * T2, *W2 = ftab + 3 * G2 * T2;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (int b = blockIdx.x * WPB + wib; b < fc.n; b += gridDim.x * WPB) {
        const int find = fc.tri[b];
        int pv[3], ps[3], sg[3];
        for (int i = 0; i < 3; ++i) {
            pv[i] = fc.pnt[3 * b + i];
            ps[i] = fc.seg[3 * b + i];
            sg[i] = fc.sgn[3 * b + i];
        }
        float lin[3] = {0.f, 0.f, 0.f};
        if (lane < 3) {
            for (int n = 0; n < 3; ++n) lin[n] = u.v[(size_t)pv[lane] * NV + n];
        } else if (lane < 3 + 3 * EM) {
            const int i = (lane - 3) / EMD, m = (lane - 3) - i * EMD;
            const float s = ((m & 1) && sg[i] < 0) ? -1.f : 1.f;
            for (int n = 0; n < 3; ++n) lin[n] = s * u.e[((size_t)ps[i] * EMD + m) * NV + n];
        } else if (lane < T2) {
            const int k = lane - 3 - 3 * EM;
            for (int n = 0; n < 3; ++n) lin[n] = u.f[((size_t)find * FMD + k) * NV + n];
        }
        float uq[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < T2; ++k) {
            const float f = lane < G2 ? (float)__ldg(F2 + lane * T2 + k) : 0.f;
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
            const float nrm[3] = {(float)(dr[1] * ds[2] - dr[2] * ds[1]), (float)(dr[2] * ds[0] - dr[0] * ds[2]),
                                  (float)(dr[0] * ds[1] - dr[1] * ds[0])};
            sflx[wib][lane] = rho * (uq[0] * nrm[0] + uq[1] * nrm[1] + uq[2] * nrm[2]);
        }
        __syncwarp();
        if (lane < T2) {
            float r = 0.f;
            for (int q = 0; q < G2; ++q) r += (float)(__ldg(W2 + q) * __ldg(F2 + q * T2 + lane)) * sflx[wib][q];
            if (lane < 3) {
                atomicAdd(res.v + (size_t)pv[lane] * NV + 3, r);
            } else if (lane < 3 + 3 * EM) {
                const int i = (lane - 3) / EMD, m = (lane - 3) - i * EMD;
                const float s = ((m & 1) && sg[i] < 0) ? -1.f : 1.f;
                atomicAdd(res.e + ((size_t)ps[i] * EMD + m) * NV + 3, s * r);
            } else {
                const int k = lane - 3 - 3 * EM;
                atomicAdd(res.f + ((size_t)find * FMD + k) * NV + 3, r);
            }
        }
        __syncwarp();
    }
}

// Precision conversions and the FP64 correction u += d.
template <typename A, typename B>
__global__ void k_tet_convert(long n, const A *src, B *dst) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        dst[k] = (B)src[k];
}
__global__ void k_tet_add_correction(long n, double *u, const float *d) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        u[k] += (double)d[k];
}
