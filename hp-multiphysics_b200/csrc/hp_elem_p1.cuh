// ins element residual at p = 1 with four lanes per triangle, one per Gauss point.
//
// At p = 1 an element has 3 modes (its vertices) and 2 x 2 Gauss points, too little work
// for a warp or for a tensor-core fragment. Here lane 4 e + q of a warp owns point
// q = 2 i + j of triangle e (8 triangles per warp). Each lane projects the three vertex
// values of u, v, p (and the velocity derivatives) to its point with the dense per-point
// operators, forms the fluxes there, and contributes its point's share of intgrtrs to the
// 9 (variable, mode) residual entries; the four shares are summed with two butterfly
// shuffles. The strong residual (derivr + derivs) at a point needs the fluxes at the
// points that share its i or its j, which come from lanes q ^ 2 and q ^ 1. Same physics
// and operators as the tensor-core kernels: tri_hp_ins::element_rsdl's straight branch
// (tri_hp/ins/rsdl.cpp:259-433), proj.cpp:22-119, intgrt.cpp:81-158, derivr / derivs
// proj.cpp:339-402, with tri_hp::rsdl's gather and scatter (nstage.cpp:52-73). Either
// precision; in correction form (FP32 smoother) the fluxes are the exact differences
// F(b + d) - F(b) about the base state b (State::ubv) with tau frozen at b.
#pragma once
#include "hp_kernels.cuh"

namespace hpb {

// The operators at p = 1 (G = 2, T = 3) as dense arrays, q = 2 i + j:
//   V, DR, DS [q][m]: value, d/dr, d/ds of mode m at point q (proj);
//   WR, WS [q][m]: the intgrtrs weights of flux_r, flux_s (with its minus sign);
//   AR, AS1, AS2 [2][2], N0 [2]: the 1D derivative operators of the strong residual,
//   res(i, j) = N0(j) (sum_k AR(i, k) fr(k, j) + AS1(i, k) fs(k, j)) + sum_l AS2(j, l) fs(i, l).
template <typename R>
struct InsP1Ops {
    R V[4][3], DR[4][3], DS[4][3], WR[4][3], WS[4][3];
    R AR[2][2], AS1[2][2], AS2[2][2], N0[2];
};

template <typename R>
__device__ __forceinline__ R quad_sum(R v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    return v;
}

template <typename R>
__global__ void __launch_bounds__(256, 2)
    k_rsdl_ins_p1(const InsP1Ops<R> *__restrict__ ops, Mesh mesh, State<R> st, Phys ph, int stage, int zero_rr,
                  int diff) {
    constexpr int NV = 3;
    const int lane = threadIdx.x & 31, q = lane & 3, i = q >> 1, j = q & 1;
    const R beta = (R)ph.beta[stage];
    const R rho = (R)ph.rho;
    const bool corr = diff && st.ubv;
    (void)zero_rr;  // no interior modes at p = 1: res_r is folded by the caller's pre / assembly
    // this lane's rows of the operators
    R V[3], DR[3], DS[3], WR[3], WS[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        V[m] = ops->V[q][m]; DR[m] = ops->DR[q][m]; DS[m] = ops->DS[q][m];
        WR[m] = ops->WR[q][m]; WS[m] = ops->WS[q][m];
    }
    const R ar_ii = ops->AR[i][i], ar_io = ops->AR[i][1 - i], as1_ii = ops->AS1[i][i], as1_io = ops->AS1[i][1 - i];
    const R as2_jj = ops->AS2[j][j], as2_jo = ops->AS2[j][1 - j], n0j = ops->N0[j];
    const long ntri = mesh.ntri;
    const long step = (long)gridDim.x * (blockDim.x >> 2);
    // every lane of a warp runs the same number of passes (the shuffles need all 32)
    for (long t0 = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) >> 2; t0 < ntri; t0 += step) {
        const long tl = t0 + (lane >> 2);
        const bool act = tl < ntri && (!mesh.tri_cv || mesh.tri_cv[tl] < 0);
        const int t = (int)(tl < ntri ? tl : ntri - 1);
        const int p0 = mesh.tri_pnt[3 * t], p1 = mesh.tri_pnt[3 * t + 1], p2 = mesh.tri_pnt[3 * t + 2];
        // gather (ugtouht) and geometry: ldcrd(n,0) = (v2-v1)/2, ldcrd(n,1) = (v0-v1)/2, and the
        // inscribed-radius length scale of tau (tri_mesh/tprims.cpp:224-241)
        R u[NV][3];
#pragma unroll
        for (int n = 0; n < NV; ++n) {
            u[n][0] = st.ugv[p0 * NV + n];
            u[n][1] = st.ugv[p1 * NV + n];
            u[n][2] = st.ugv[p2 * NV + n];
        }
        const double *tg = mesh.tgeo + (size_t)8 * t;  // per-triangle constants (Mesh::tgeo)
        const R d00 = (R)tg[0], d01 = (R)tg[1], d10 = (R)tg[2], d11 = (R)tg[3];
        // projection to this lane's point
        R u0 = 0, u1 = 0, pp = 0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            u0 += V[m] * u[0][m];
            u1 += V[m] * u[1][m];
            pp += V[m] * u[2][m];
        }
        R b0 = 0, b1 = 0;
        if (corr) {
            const R bv[2][3] = {{st.ubv[p0 * NV], st.ubv[p1 * NV], st.ubv[p2 * NV]},
                                {st.ubv[p0 * NV + 1], st.ubv[p1 * NV + 1], st.ubv[p2 * NV + 1]}};
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                b0 += V[m] * bv[0][m];
                b1 += V[m] * bv[1][m];
            }
        }
        // pointwise fluxes (ins/rsdl.cpp:259-340): imaginary flux pairs fr/fs of u, v, p
        const R m0 = +d11 * (rho * u0) - d01 * (rho * u1);
        const R m1 = -d10 * (rho * u0) + d00 * (rho * u1);
        R c00, c01, c10, c11;
        if (corr) {  // F(b + d) - F(b), products expanded
            const R mb0 = +d11 * (rho * b0) - d01 * (rho * b1);
            const R mb1 = -d10 * (rho * b0) + d00 * (rho * b1);
            const R uf0 = b0 + u0, uf1 = b1 + u1;
            c00 = uf0 * m0 + u0 * mb0;
            c01 = uf0 * m1 + u0 * mb1;
            c10 = uf1 * m0 + u1 * mb0;
            c11 = uf1 * m1 + u1 * mb1;
        } else {
            c00 = u0 * m0; c01 = u0 * m1; c10 = u1 * m0; c11 = u1 * m1;
        }
        R fir[NV] = {c00 + d11 * pp, c10 - d01 * pp, m0};
        R fis[NV] = {c01 - d10 * pp, c11 + d00 * pp, m1};
        // imaginary part: this point's share of intgrtrs, summed over the four points
        R lf[NV][3];
#pragma unroll
        for (int n = 0; n < NV; ++n)
#pragma unroll
            for (int m = 0; m < 3; ++m) lf[n][m] = quad_sum(WR[m] * fir[n] + WS[m] * fis[n]);
        // lftog of the 9 entries, lane q writing entries k = n * 3 + m with k % 4 == q
        auto scatter = [&](const R (&v)[NV][3], int part) {
            if (!act) return;
            const int pv[3] = {p0, p1, p2};
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                if ((k & 3) != q) continue;
                const int n = k / 3, m = k - 3 * (k / 3);
                const R val = part ? v[n][m] * beta : v[n][m];
                R *el = part ? st.elre : st.elim;
                if (el) el[asm_slot(mesh, NV, 1, mesh.vpos[3 * t + m], 0, m, n)] = val;
                else atomicAdd((part ? st.rrv : st.resv) + pv[m] * NV + n, val);
            }
        };
        scatter(lf, 0);
        if (beta > (R)0) {
            // viscous flux pairs of u, v (zero for p)
            R dr0 = 0, dr1 = 0, ds0 = 0, ds1 = 0;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                dr0 += DR[m] * u[0][m]; dr1 += DR[m] * u[1][m];
                ds0 += DS[m] * u[0][m]; ds1 += DS[m] * u[1][m];
            }
            const R cjcbi = (R)(ph.mu * tg[4]);
            const R v0000 = -cjcbi * ((R)2 * d11 * d11 + d01 * d01);
            const R v0011 = -cjcbi * ((R)2 * d10 * d10 + d00 * d00);
            const R v0001 = cjcbi * ((R)2 * d11 * d10 + d01 * d00);
            const R v1100 = -cjcbi * (d11 * d11 + (R)2 * d01 * d01);
            const R v1111 = -cjcbi * (d10 * d10 + (R)2 * d00 * d00);
            const R v1101 = cjcbi * (d11 * d10 + (R)2 * d01 * d00);
            const R v0100 = cjcbi * d01 * d11;
            const R v0111 = cjcbi * d00 * d10;
            const R v0101 = -cjcbi * d01 * d10;
            const R v0110 = -cjcbi * d00 * d11;
            R fxr[NV] = {v0000 * dr0 + v0100 * dr1 + v0001 * ds0 + v0101 * ds1,
                         v0100 * dr0 + v1100 * dr1 + v0110 * ds0 + v1101 * ds1, (R)0};
            R fxs[NV] = {v0001 * dr0 + v0110 * dr1 + v0011 * ds0 + v0111 * ds1,
                         v0101 * dr0 + v1101 * dr1 + v0111 * ds0 + v1111 * ds1, (R)0};
            // strong residual of the full fluxes at this point (derivr + derivs)
            R res[NV];
#pragma unroll
            for (int n = 0; n < NV; ++n) {
                const R fr = fir[n] + fxr[n], fs = fis[n] + fxs[n];
                const R fr_oi = __shfl_xor_sync(0xffffffffu, fr, 2), fs_oi = __shfl_xor_sync(0xffffffffu, fs, 2);
                const R fs_oj = __shfl_xor_sync(0xffffffffu, fs, 1);
                res[n] = n0j * (ar_ii * fr + ar_io * fr_oi + as1_ii * fs + as1_io * fs_oi) + (as2_jj * fs + as2_jo * fs_oj);
            }
            // SUPG (ins/rsdl.cpp:341-431, CALC_TAU2), tau of the base in correction form
            R a0 = u0, a1 = u1, qv;
            if (corr) {
                qv = b0 * b0 + b1 * b1;
                a0 += b0;
                a1 += b1;
            } else {
                qv = u0 * u0 + u1 * u1;
            }
            const R t2 = (R)(2. * (ph.mu / ph.rho) * tg[6]);
            R gam = (R)3 * qv + t2 * t2;
            if (ph.mu + ph.bd0 == 0.0) gam = (gam > (R)0.1 ? gam : (R)0.1);
            const R tau0 = (R)(ph.adis * tg[5] * tg[4]) / sqrt(gam);
            const R tau2 = sqrt(qv) * tau0;
            const R tr0 = tau0 * res[0], tr1 = tau0 * res[1], tr2 = tau2 * res[2];
            fxr[0] -= (d11 * ((R)2 * a0) - d01 * a1) * tr0 - d01 * a0 * tr1 + d11 * tr2;
            fxs[0] -= (-d10 * ((R)2 * a0) + d00 * a1) * tr0 + d00 * a0 * tr1 - d10 * tr2;
            fxr[1] -= +d11 * a1 * tr0 + (d11 * a0 - d01 * ((R)2 * a1)) * tr1 - d01 * tr2;
            fxs[1] -= -d10 * a1 * tr0 + (-d10 * a0 + d00 * ((R)2 * a1)) * tr1 + d00 * tr2;
            fxr[2] = -(d11 * tr0 - d01 * tr1);
            fxs[2] = -(-d10 * tr0 + d00 * tr1);
            // real part: intgrtrs of the viscous + SUPG pairs, x beta -> res_r
#pragma unroll
            for (int n = 0; n < NV; ++n)
#pragma unroll
                for (int m = 0; m < 3; ++m) lf[n][m] = quad_sum(WR[m] * fxr[n] + WS[m] * fxs[n]);
            scatter(lf, 1);
        }
    }
}

}  // namespace hpb
