// C-ABI of the B200 library: context set-up, per-(p, physics) dispatch,
// stream-ordered launches of the element-residual / minvrt / update kernels, and
// CUDA-graph capture of one multistage update.
#include <cuda_runtime.h>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <vector>
#include <string>
#include <algorithm>
#include <map>
#include <mutex>
#include <cstdint>

#include "hp_gpu.h"
#include "hp_host.h"
#include "hp_mlp.h"
#include "hp_kernels.cuh"
#include "hp_elem_mma.cuh"
#include "hp_elem_p1.cuh"
#include "hp_elem_tf32.cuh"

using namespace hpb;

static thread_local std::string g_err;
static void set_err(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return HP_ECUDA;                                                            \
        }                                                                               \
    } while (0)

namespace {

template <typename R, int P>
void fill_tables(const hp_basis_tables &b, DevTables<R, P> &t) {
    constexpr int G = P + 1, X = P + 2, T = (P + 1) * (P + 2) / 2, SM = P - 1, BM = 3 * P;
    std::memset(&t, 0, sizeof(t));
    for (int i = 0; i < G; ++i) {
        for (int n = 0; n < X; ++n) { t.gx[i][n] = (R)b.gx[i][n]; t.dgx[i][n] = (R)b.dgx[i][n]; }
        for (int m = 0; m < T; ++m) { t.gn[i][m] = (R)b.gn[i][m]; t.dgn[i][m] = (R)b.dgn[i][m]; }
        t.x0[i] = (R)b.x0[i]; t.n0[i] = (R)b.n0[i]; t.wtx[i] = (R)b.wtx[i];
        t.dltx[i] = (R)b.dltx[i]; t.dltn[i] = (R)b.dltn[i];
        for (int q = 0; q < G; ++q) {
            t.dltx1[i][q] = (R)b.dltx1[i][q];
            t.dltn1[i][q] = (R)b.dltn1[i][q];
            t.dltn2[i][q] = (R)b.dltn2[i][q];
        }
    }
    for (int n = 0; n < X; ++n)
        for (int i = 0; i < G; ++i) { t.gxwtx[n][i] = (R)b.gxwtx[n][i]; t.dgxwtx[n][i] = (R)b.dgxwtx[n][i]; }
    for (int m = 0; m < T; ++m)
        for (int j = 0; j < G; ++j) {
            t.gnwtn[m][j] = (R)b.gnwtn[m][j];
            t.gnwtnn0[m][j] = (R)b.gnwtnn0[m][j];
            t.dgnwtn[m][j] = (R)b.dgnwtn[m][j];
        }
    // column structure of the sum factorisation (proj.cpp:46-95, intgrt.cpp:44-76)
    const int bs1 = SM + 3, bs2 = 2 * SM + 3;
    std::vector<std::vector<int>> cols(X);
    cols[0].push_back(0);
    cols[1].push_back(1);
    for (int m = bs2; m < BM; ++m) cols[1].push_back(m);
    if (X > 2) {
        cols[2].push_back(2);
        for (int m = bs1; m < bs2; ++m) cols[2].push_back(m);
    }
    int ind = BM, cnt = SM - 1;
    for (int m = 3; m < bs1; ++m) {
        cols[m].push_back(m);
        for (int n = 0; n < cnt; ++n) cols[m].push_back(ind + n);
        ind += cnt--;
    }
    int c = 0;
    for (int n = 0; n < X; ++n) {
        t.colstart[n] = c;
        for (int m : cols[n]) { t.colmodes[c++] = m; t.colof[m] = n; }
    }
    t.colstart[X] = c;
}

// Dense per-point forms of tri_basis::proj (value, d/dr, d/ds; proj.cpp:22-119) and
// intgrtrs (intgrt.cpp:81-158) for the tensor-core ins kernel, in DMMA fragment order
// (B operand of mma.m8n8k4 .row.col: lane l holds B[k = l & 3][n = l >> 2]). Point
// q = i * G + j (i along the x-direction Gauss points, j along eta). With c = the column
// of mode m in the sum factorisation:
//   value(q, m) = gn(j, m) gx(i, c)
//   d/dr (q, m) = n0(j) gn(j, m) dgx(i, c)
//   d/ds (q, m) = dgn(j, m) gx(i, c) + x0(i) d/dr(q, m)
//   W_r(q, m)   = -dgxwtx(c, i) gnwtnn0(m, j)
//   W_s(q, m)   = -(x0(i) dgxwtx(c, i) gnwtnn0(m, j) + gxwtx(c, i) dgnwtn(m, j))
// so that lf(m) = sum_q flux_r(q) W_r(q, m) + flux_s(q) W_s(q, m) is intgrtrs' result.
// The 1D derivative operators of derivr / derivs (proj.cpp:339-402) as matrices, so that
// the strong residual at point (i, j) is
//   res(i, j) = n0(j) (sum_q Ar(i, q) flux_r(q, j) + sum_q As1(i, q) flux_s(q, j))
//             + sum_l As2(j, l) flux_s(i, l), with (which = 0: Ar, 1: As1, 2: As2)
//   Ar(i, q)  = q == i ? dltx(i) sum_{q' != i} dltx1(i, q') : dltx(q) dltx1(i, q)
//   As1(i, q) = q == i ? dltx(i) sum_{q' != i} dltn1(i, q') : dltx(q) dltn1(i, q)
//   As2(j, l) = l == j ? dltn(j) sum_{l' != j} dltn2(j, l') : dltn(l) dltn2(j, l).
inline double deriv_op(const hp_basis_tables &b, int G, int which, int r, int k) {
    if (r >= G || k >= G) return 0.0;
    auto tab = [&](int a, int c) {
        return which == 0 ? b.dltx1[a][c] : (which == 1 ? b.dltn1[a][c] : b.dltn2[a][c]);
    };
    const double *dl = which == 2 ? b.dltn : b.dltx;
    if (k != r) return dl[k] * tab(r, k);
    double sum = 0.0;
    for (int c = 0; c < G; ++c)
        if (c != r) sum += tab(r, c);
    return dl[r] * sum;
}

template <int P>
void build_ins_mma(const hp_basis_tables &b, std::vector<double> &ops, InsMmaSmall<P> &sm) {
    using M = InsMma<P>;
    constexpr int G = M::G, GG = M::GG, T = M::T;
    ops.assign(M::PROJ_LEN + M::INT_LEN + M::DER_LEN, 0.0);
    for (int op = 0; op < 3; ++op)
        for (int nt = 0; nt < M::NT; ++nt)
            for (int ks = 0; ks < M::KS; ++ks)
                for (int l = 0; l < 32; ++l) {
                    const int q = nt * 8 + (l >> 2), m = ks * 4 + (l & 3);
                    if (q >= GG || m >= T) continue;
                    const int i = q / G, j = q - i * G, c = ModeCols<P>::col(m);
                    const double dr = b.n0[j] * b.gn[j][m] * b.dgx[i][c];
                    const double v = op == 0 ? b.gn[j][m] * b.gx[i][c]
                                             : (op == 1 ? dr : b.dgn[j][m] * b.gx[i][c] + b.x0[i] * dr);
                    ops[((size_t)(op * M::NT + nt) * M::KS + ks) * 32 + l] = v;
                }
    double *ib = ops.data() + M::PROJ_LEN;
    for (int nt = 0; nt < M::NT2; ++nt)
        for (int ks = 0; ks < M::KS2; ++ks)
            for (int l = 0; l < 32; ++l) {
                const int k = ks * 4 + (l & 3), m = nt * 8 + (l >> 2);
                if (k >= 2 * GG || m >= T) continue;
                const int q = k % GG, i = q / G, j = q - i * G, c = ModeCols<P>::col(m);
                const double w = k < GG ? -b.dgxwtx[c][i] * b.gnwtnn0[m][j]
                                        : -(b.x0[i] * b.dgxwtx[c][i] * b.gnwtnn0[m][j] + b.gxwtx[c][i] * b.dgnwtn[m][j]);
                ib[((size_t)nt * M::KS2 + ks) * 32 + l] = w;
            }
    // A fragments of the 1D derivative operators (lane l holds A[row = l >> 2][k = l & 3]):
    // [Ar | As1] per m-tile over 2 KR k-steps, then As2 over KR k-steps
    double *db = ops.data() + M::PROJ_LEN + M::INT_LEN;
    for (int mt = 0; mt < M::MT; ++mt)
        for (int ks = 0; ks < 2 * M::KR; ++ks)
            for (int l = 0; l < 32; ++l) {
                const int blk = ks / M::KR, r = mt * 8 + (l >> 2), k = (ks - blk * M::KR) * 4 + (l & 3);
                db[((size_t)mt * 2 * M::KR + ks) * 32 + l] = deriv_op(b, G, blk, r, k);
            }
    double *da = db + M::MT * 2 * M::KR * 32;
    for (int mt = 0; mt < M::MT; ++mt)
        for (int ks = 0; ks < M::KR; ++ks)
            for (int l = 0; l < 32; ++l)
                da[((size_t)mt * M::KR + ks) * 32 + l] = deriv_op(b, G, 2, mt * 8 + (l >> 2), ks * 4 + (l & 3));
    for (int i = 0; i < G; ++i) {
        sm.dltx[i] = b.dltx[i]; sm.dltn[i] = b.dltn[i]; sm.n0[i] = b.n0[i]; sm.x0[i] = b.x0[i];
        for (int q = 0; q < G; ++q) {
            sm.dltx1[i][q] = b.dltx1[i][q]; sm.dltn1[i][q] = b.dltn1[i][q]; sm.dltn2[i][q] = b.dltn2[i][q];
        }
    }
}

// The dense operators of the p = 1 point kernel (k_rsdl_ins_p1), the same entries as
// build_ins_mma's at G = 2, T = 3, indexed by point q = 2 i + j.
template <typename R>
void build_ins_p1(const hp_basis_tables &b, InsP1Ops<R> &o) {
    constexpr int G = 2;
    for (int q = 0; q < 4; ++q)
        for (int m = 0; m < 3; ++m) {
            const int i = q / G, j = q - i * G, c = ModeCols<1>::col(m);
            const double dr = b.n0[j] * b.gn[j][m] * b.dgx[i][c];
            o.V[q][m] = (R)(b.gn[j][m] * b.gx[i][c]);
            o.DR[q][m] = (R)dr;
            o.DS[q][m] = (R)(b.dgn[j][m] * b.gx[i][c] + b.x0[i] * dr);
            o.WR[q][m] = (R)(-b.dgxwtx[c][i] * b.gnwtnn0[m][j]);
            o.WS[q][m] = (R)(-(b.x0[i] * b.dgxwtx[c][i] * b.gnwtnn0[m][j] + b.gxwtx[c][i] * b.dgnwtn[m][j]));
        }
    for (int r = 0; r < G; ++r) {
        for (int k = 0; k < G; ++k) {
            o.AR[r][k] = (R)deriv_op(b, G, 0, r, k);
            o.AS1[r][k] = (R)deriv_op(b, G, 1, r, k);
            o.AS2[r][k] = (R)deriv_op(b, G, 2, r, k);
        }
        o.N0[r] = (R)b.n0[r];
    }
}

// TF32 rounding of an operator entry (round to nearest, ties away from zero, as
// cvt.rna.tf32.f32 does for the A operands)
float to_tf32(double v) {
    float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = (u + 0x1000u) & 0xFFFFE000u;
    std::memcpy(&f, &u, 4);
    return f;
}

// The same dense operators as build_ins_mma for the TF32 kernel (mma.m16n8k8 .row.col:
// lane l holds B[k = l & 3][n = l >> 2] and B[k = (l & 3) + 4][n = l >> 2], stored as one
// float2 per lane per MMA), rounded to TF32.
template <int P>
void build_ins_tf32(const hp_basis_tables &b, std::vector<float> &ops, InsMmaSmallF<P> &sm) {
    using M = InsTf32<P>;
    constexpr int G = M::G, GG = M::GG, T = M::T;
    ops.assign(M::PROJ_LEN + M::INT_LEN + M::DER_LEN, 0.f);
    auto proj = [&](int op, int q, int m) -> double {
        if (q >= GG || m >= T) return 0.0;
        const int i = q / G, j = q - i * G, c = ModeCols<P>::col(m);
        const double dr = b.n0[j] * b.gn[j][m] * b.dgx[i][c];
        return op == 0 ? b.gn[j][m] * b.gx[i][c] : (op == 1 ? dr : b.dgn[j][m] * b.gx[i][c] + b.x0[i] * dr);
    };
    auto wgt = [&](int k, int m) -> double {
        if (k >= 2 * GG || m >= T) return 0.0;
        const int q = k % GG, i = q / G, j = q - i * G, c = ModeCols<P>::col(m);
        return k < GG ? -b.dgxwtx[c][i] * b.gnwtnn0[m][j]
                      : -(b.x0[i] * b.dgxwtx[c][i] * b.gnwtnn0[m][j] + b.gxwtx[c][i] * b.dgnwtn[m][j]);
    };
    for (int op = 0; op < 3; ++op)
        for (int nt = 0; nt < M::NT; ++nt)
            for (int ks = 0; ks < M::KS; ++ks)
                for (int l = 0; l < 32; ++l) {
                    const size_t at = (((size_t)(op * M::NT + nt) * M::KS + ks) * 32 + l) * 2;
                    const int q = nt * 8 + (l >> 2), m = ks * 8 + (l & 3);
                    ops[at] = to_tf32(proj(op, q, m));
                    ops[at + 1] = to_tf32(proj(op, q, m + 4));
                }
    float *ib = ops.data() + M::PROJ_LEN;
    for (int nt = 0; nt < M::NT2; ++nt)
        for (int ks = 0; ks < M::KS2; ++ks)
            for (int l = 0; l < 32; ++l) {
                const size_t at = (((size_t)nt * M::KS2 + ks) * 32 + l) * 2;
                const int k = ks * 8 + (l & 3), m = nt * 8 + (l >> 2);
                ib[at] = to_tf32(wgt(k, m));
                ib[at + 1] = to_tf32(wgt(k + 4, m));
            }
    // B fragments of the transposed 1D derivative operators (mma.m16n8k8 .col: lane l holds
    // B[k = t][n = g], B[k = t + 4][n = g] with g = l >> 2 + 8 nt, t = l & 3 + 8 kb and
    // B[k][n] = A[n][k]): [Ar | As1]^T in 2 KR k-steps, then As2^T in KR k-steps
    float *db = ops.data() + M::PROJ_LEN + M::INT_LEN;
    for (int kk = 0; kk < 3 * M::KR; ++kk)
        for (int nt = 0; nt < M::NTI; ++nt)
            for (int l = 0; l < 32; ++l) {
                const bool part2 = kk >= 2 * M::KR;
                const int ks = part2 ? kk - 2 * M::KR : kk;
                const int blk = part2 ? 2 : ks / M::KR, kb = part2 ? ks : ks - (ks / M::KR) * M::KR;
                const int n = nt * 8 + (l >> 2), k = kb * 8 + (l & 3);
                float *bb = db + (((size_t)kk * M::NTI + nt) * 32 + l) * 2;
                bb[0] = to_tf32(deriv_op(b, G, blk, n, k));
                bb[1] = to_tf32(deriv_op(b, G, blk, n, k + 4));
            }
    for (int i = 0; i < G; ++i) {
        sm.dltx[i] = (float)b.dltx[i]; sm.dltn[i] = (float)b.dltn[i];
        sm.n0[i] = (float)b.n0[i]; sm.x0[i] = (float)b.x0[i];
        for (int q = 0; q < G; ++q) {
            sm.dltx1[i][q] = (float)b.dltx1[i][q];
            sm.dltn1[i][q] = (float)b.dltn1[i][q];
            sm.dltn2[i][q] = (float)b.dltn2[i][q];
        }
    }
}

template <typename R>
void fill_minv(const hp_basis_tables &b, DevMinv<R> &m) {
    std::memset(&m, 0, sizeof(m));
    for (int i = 0; i < 2; ++i)
        for (int k = 0; k < b.sm; ++k) m.sfmv[i][k] = (R)b.sfmv[i][k];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < b.sm; ++k) m.vfms[i][k] = (R)b.vfms[i][k];
    for (int k = 0; k < b.sm; ++k) m.sdiag[k] = (R)b.sdiag[k];
    for (int a = 0; a < b.sm; ++a)
        for (int c = 0; c < b.sm; ++c)
            for (int s = 0; s < 3; ++s) m.sfms[a][c][s] = (R)b.sfms[a][c][s];
    for (int i = 0; i < b.bm; ++i)
        for (int k = 0; k < b.im; ++k) { m.ifmb[i][k] = (R)b.ifmb[i][k]; m.bfmi[i][k] = (R)b.bfmi[i][k]; }
    for (int k = 0; k < b.im; ++k) { m.idiag[k][0] = (R)b.idiag[k][0]; m.idiag[k][1] = (R)b.idiag[k][1]; }
    m.vdiag = (R)b.vdiag;
}

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// Launch shapes chosen per context (per mesh level) and precision by hp_gpu_autotune.
struct Tune {
    int elem_cap = 16;       // matrix-free element kernel: CTAs per SM at most
    int emat_tpp = 1;        // stored-operator kernel: tiles per pipeline phase (1 or 2)
    int emat_ctas = 0;       // stored-operator kernel: CTAs per SM (0 = as many as fit)
    int minv_threads = 128;  // minvrt kernels: threads per CTA
};

// Per-(precision, p, physics) launchers.
template <typename R>
struct Launchers {
    size_t tab_bytes;
    void (*fill)(const hp_basis_tables &, void *);
    void (*elem)(const void *tab, const Mesh &, const State<R> &, const Phys &, int stage, int zero_rr, int diff,
                 int nsm, const Tune &, cudaStream_t);
    void (*bflux)(const void *tab, const Mesh &, const State<R> &, const Phys &, int diff, cudaStream_t);
    void (*side)(const Mesh &, const State<R> &, const DevMinv<R> *, int im, int mode, double cfla, int upd, int fold,
                 int threads, cudaStream_t);
    void (*intr)(const Mesh &, const State<R> &, const DevMinv<R> *, double cfla, int upd, int threads, cudaStream_t);
    void (*vert)(const Mesh &, const State<R> &, const DevMinv<R> *, int sm, int im, double cfla, int upd, int fold,
                 unsigned long long *slot, int threads, cudaStream_t);
    int elem_smem;
    cudaError_t (*set_smem)();
    // cd element operators: length of one operator array, build, apply
    size_t (*emat_len)(long ntri);
    void (*emat_build)(const void *tab, const Mesh &, const State<R> &, const Phys &, ElemMat<R>, int nsm,
                       cudaStream_t);
    void (*emat_apply)(ElemMat<R>, const Mesh &, const State<R> &, const Phys &, int stage, int zero_rr, int nsm,
                       const Tune &, cudaStream_t);
    void (*elem_jac)(const void *tab, const Mesh &, const State<R> &, const Phys &, R *K, R *rbar, int nsm,
                     cudaStream_t);
    // FP64 ins only: the tensor-core element kernel (k_rsdl_ins_mma) with its operators
    // (mma_build: dense operators in fragment order + the small derivative tables) and
    // the curved elements through the scalar kernel
    // (FP64: DMMA k_rsdl_ins_mma; FP32: TF32 k_rsdl_ins_tf32, plain or correction form)
    void (*elem_mma)(const void *ops, const void *small, const void *tab, const Mesh &, const State<R> &,
                     const Phys &, int stage, int zero_rr, int diff, int nsm, const Tune &, cudaStream_t);
    void (*mma_build)(const hp_basis_tables &, std::vector<unsigned char> &ops, std::vector<unsigned char> &small);
    // FP32 ins: the base state's point values for the correction form (State::bpt)
    void (*base_pts)(const void *tab, const Mesh &, const State<R> &, R *bpt, cudaStream_t);
    int bpt_per_elem;  // 2 GG
    // ins at p = 1: the point kernel (k_rsdl_ins_p1, four lanes per triangle) with its
    // operators (point_build: InsP1Ops<R>), curved triangles through the scalar kernel
    void (*elem_point)(const void *ops, const void *tab, const Mesh &, const State<R> &, const Phys &, int stage,
                       int zero_rr, int diff, int nsm, const Tune &, cudaStream_t);
    void (*point_build)(const hp_basis_tables &, std::vector<unsigned char> &ops);
    // tri_hp::l2error on the device (FP64): per-block partials into part
    void (*l2err)(const void *tab, const double *wtn, const Mesh &, const State<R> &, int NV, const DevField &,
                  double *part, int blocks, cudaStream_t);
};

template <typename R, int P, int PHYS>
struct LaunchImpl {
    using C = ElemCfg<R, P, PHYS>;
    static constexpr int NV = C::NV, SM = P - 1, IM = (P - 1) * (P - 2) / 2;
    static int smem() {
        return (int)(((sizeof(DevTables<R, P>) + 15) / 16) * 16 + (size_t)C::WPC * C::EPW * C::S_WARP * sizeof(R));
    }
    static void fill(const hp_basis_tables &b, void *out) { fill_tables<R, P>(b, *reinterpret_cast<DevTables<R, P> *>(out)); }
    static void elem(const void *tab, const Mesh &m, const State<R> &s, const Phys &ph, int stage, int zero_rr, int diff,
                     int nsm, const Tune &tn, cudaStream_t st) {
        constexpr int EPC = C::WPC * C::EPW;  // elements per CTA and pass
        int blocks = nblk(m.ntri, EPC);
        const int cap = nsm * tn.elem_cap;
        if (blocks > cap) blocks = cap;
        const auto *t = reinterpret_cast<const DevTables<R, P> *>(tab);
        k_rsdl_elem<R, P, PHYS, false><<<blocks, C::WPC * 32, smem(), st>>>(t, m, s, ph, stage, zero_rr, diff,
                                                                           ElemMat<R>{}, ElemJac<R>{});
        if (m.ncurved > 0)
            k_rsdl_elem<R, P, PHYS, true><<<std::min(nblk(m.ncurved, EPC), cap), C::WPC * 32, smem(), st>>>(
                t, m, s, ph, stage, zero_rr, diff, ElemMat<R>{}, ElemJac<R>{});
    }
    // finite-difference element Jacobians at stage 0: pass 0 (rbar) then pass 1 (columns)
    static void elem_jac(const void *tab, const Mesh &m, const State<R> &s, const Phys &ph, R *K, R *rbar, int nsm,
                         cudaStream_t st) {
        const auto *t = reinterpret_cast<const DevTables<R, P> *>(tab);
        constexpr int EPC = C::WPC * C::EPW, NJ = NV * C::T;
        for (int pass = 0; pass < 2; ++pass)
            for (int cv = 0; cv < 2; ++cv) {
                const long nel = cv ? (long)m.ncurved : (long)m.ntri;
                if (nel == 0) continue;
                const long items = pass ? nel * NJ : nel;
                const int blocks = (int)std::min<long>((items + EPC - 1) / EPC, (long)nsm * 16);
                const ElemJac<R> jac{K, rbar, pass};
                if (cv)
                    k_rsdl_elem<R, P, PHYS, true><<<blocks, C::WPC * 32, smem(), st>>>(t, m, s, ph, 0, 1, 0,
                                                                                       ElemMat<R>{}, jac);
                else
                    k_rsdl_elem<R, P, PHYS, false><<<blocks, C::WPC * 32, smem(), st>>>(t, m, s, ph, 0, 1, 0,
                                                                                        ElemMat<R>{}, jac);
            }
    }
    static size_t emat_len(long ntri) { return EmatCfg<P>::len(ntri); }
    // one warp item per (element, column j <= T) at beta(nstage) = 1
    static void emat_build(const void *tab, const Mesh &m, const State<R> &s, const Phys &ph, ElemMat<R> em, int nsm,
                           cudaStream_t st) {
        if constexpr (PHYS == 0) {
            const auto *t = reinterpret_cast<const DevTables<R, P> *>(tab);
            for (int cv = 0; cv < 2; ++cv) {
                const long items = (cv ? (long)m.ncurved : (long)m.ntri) * (C::T + 1);
                if (items == 0) continue;
                long blocks = (items + C::WPC * C::EPW - 1) / (C::WPC * C::EPW);
                if (blocks > (long)nsm * 16) blocks = (long)nsm * 16;
                if (cv)
                    k_rsdl_elem<R, P, PHYS, true><<<(int)blocks, C::WPC * 32, smem(), st>>>(t, m, s, ph, ph.nstage, 1, 0,
                                                                                            em, ElemJac<R>{});
                else
                    k_rsdl_elem<R, P, PHYS, false><<<(int)blocks, C::WPC * 32, smem(), st>>>(t, m, s, ph, ph.nstage, 1,
                                                                                             0, em, ElemJac<R>{});
            }
        }
    }
    template <bool RE>
    static void emat_launch(ElemMat<R> em, const Mesh &m, const State<R> &s, const Phys &ph, int stage, int zero_rr,
                            int nsm, const Tune &tn, cudaStream_t st) {
        using E = EmatCfg<P>;
        constexpr int TH = EmatShape<R, P, RE>::THREADS;
        const long ntiles = ((long)m.ntri + E::EB - 1) / E::EB;
        const int tpp = tn.emat_tpp == 2 ? 2 : 1;
        const int maxc = std::max(1, 2048 / TH / tpp);
        const int cps = (tn.emat_ctas > 0 && tn.emat_ctas < maxc) ? tn.emat_ctas : maxc;
        const long groups = (ntiles + tpp - 1) / tpp;
        const int blocks = (int)std::min(groups, (long)nsm * cps);
        if (tpp == 2)
            k_rsdl_emat<R, P, RE, 2><<<blocks, TH, 0, st>>>(em, m, s, ph, stage, zero_rr);
        else
            k_rsdl_emat<R, P, RE, 1><<<blocks, TH, 0, st>>>(em, m, s, ph, stage, zero_rr);
    }
    static void emat_apply(ElemMat<R> em, const Mesh &m, const State<R> &s, const Phys &ph, int stage, int zero_rr,
                           int nsm, const Tune &tn, cudaStream_t st) {
        if constexpr (PHYS == 0) {
            if (ph.beta[stage] > 0.0)
                emat_launch<true>(em, m, s, ph, stage, zero_rr, nsm, tn, st);
            else
                emat_launch<false>(em, m, s, ph, stage, zero_rr, nsm, tn, st);
        }
    }
    static void bflux(const void *tab, const Mesh &m, const State<R> &s, const Phys &ph, int diff, cudaStream_t st) {
        if (PHYS == 1 && m.nbseg > 0)
            k_bdry_flux_ins<R, P><<<nblk(m.nbseg, 128), 128, 0, st>>>(reinterpret_cast<const DevTables<R, P> *>(tab), m,
                                                                       s, ph, diff);
    }
    template <int MODE>
    static void side_mode(const Mesh &m, const State<R> &s, const DevMinv<R> *mt, int im, int mode, double cfla,
                          int upd, int fold, int th, cudaStream_t st) {
        if constexpr (MODE < SM) {
            if (mode == MODE)
                k_minv_side_vn<R, NV, SM, IM, MODE><<<nblk((long)m.nseg * NV, th), th, 0, st>>>(m, s, mt, (R)cfla, upd,
                                                                                             fold);
            else
                side_mode<MODE + 1>(m, s, mt, im, mode, cfla, upd, fold, th, st);
        }
    }
    static void side(const Mesh &m, const State<R> &s, const DevMinv<R> *mt, int im, int mode, double cfla, int upd,
                     int fold, int th, cudaStream_t st) {
        if constexpr (SM > 0) side_mode<0>(m, s, mt, im, mode, cfla, upd, fold, th, st);
    }
    static void intr(const Mesh &m, const State<R> &s, const DevMinv<R> *mt, double cfla, int upd, int th,
                     cudaStream_t st) {
        if constexpr (IM > 0)
            k_minv_int_flat<R, NV, SM, IM><<<nblk((long)m.ntri * NV, th), th, 0, st>>>(m, s, mt, (R)cfla, upd);
    }
    static void vert(const Mesh &m, const State<R> &s, const DevMinv<R> *mt, int sm, int im, double cfla, int upd,
                     int fold, unsigned long long *slot, int th, cudaStream_t st) {
        if constexpr (SM > 0) {
            // a lane group per vertex, sized to the vertex's removal terms (about 6 sides x SM
            // and 6 triangles x IM)
            constexpr int LPV = SM + IM >= 8 ? 32 : (SM + IM >= 3 ? 8 : 4);
            k_minv_vert_coop<R, NV, SM, IM, LPV><<<nblk((long)m.npnt * LPV, th), th, 0, st>>>(m, s, mt, (R)cfla, upd,
                                                                                             fold, slot);
        } else {
            k_minv_vert<R, NV><<<nblk(m.npnt, th), th, 0, st>>>(m, s, mt, sm, im, (R)cfla, upd, fold, slot);
        }
    }
    static constexpr bool HAS_MMA = PHYS == 1;
    static constexpr bool DBL = std::is_same<R, double>::value;
    static int mma_smem() {
        if constexpr (DBL)
            return (int)(((sizeof(InsMmaSmall<P>) + 15) / 16) * 16 + (size_t)2 * InsMma<P>::S_EL * InsMma<P>::WPC * 8 +
                         InsMma<P>::SMEM_GEO + InsMma<P>::SMEM_IDX);
        else
            return (int)(((sizeof(InsMmaSmallF<P>) + 15) / 16) * 16 + (size_t)4 * InsTf32<P>::S_EL * InsTf32<P>::WPC * 4 +
                         InsTf32<P>::SMEM_IDX);
    }
    static void elem_mma(const void *ops, const void *small, const void *tab, const Mesh &m, const State<R> &s,
                         const Phys &ph, int stage, int zero_rr, int diff, int nsm, const Tune &tn, cudaStream_t st) {
        if constexpr (HAS_MMA) {
            if constexpr (DBL) {
                using MM = InsMma<P>;
                const double *o = static_cast<const double *>(ops);
                const long npair = ((long)m.ntri + 1) / 2;
                const int blocks = (int)std::min<long>((npair + MM::WPC - 1) / MM::WPC, (long)nsm * MM::MINB * 4);
                k_rsdl_ins_mma<P><<<blocks, MM::WPC * 32, mma_smem(), st>>>(
                    o, o + MM::PROJ_LEN, o + MM::PROJ_LEN + MM::INT_LEN, *static_cast<const InsMmaSmall<P> *>(small), m,
                    s, ph, stage, zero_rr);
            } else {
                using MM = InsTf32<P>;
                const float2 *o = static_cast<const float2 *>(ops);
                const long nquad = ((long)m.ntri + 3) / 4;
                const int blocks = (int)std::min<long>((nquad + MM::WPC - 1) / MM::WPC, (long)nsm * MM::MINB * 4);
                k_rsdl_ins_tf32<P><<<blocks, MM::WPC * 32, mma_smem(), st>>>(
                    o, o + MM::PROJ_LEN / 2, o + (MM::PROJ_LEN + MM::INT_LEN) / 2,
                    *static_cast<const InsMmaSmallF<P> *>(small), m, s, ph, stage, zero_rr, diff);
            }
            if (m.ncurved > 0) {
                constexpr int EPC = C::WPC * C::EPW;
                const int cap = nsm * tn.elem_cap;
                k_rsdl_elem<R, P, PHYS, true><<<std::min(nblk(m.ncurved, EPC), cap), C::WPC * 32, smem(), st>>>(
                    reinterpret_cast<const DevTables<R, P> *>(tab), m, s, ph, stage, zero_rr, diff, ElemMat<R>{},
                    ElemJac<R>{});
            }
        }
    }
    static constexpr bool HAS_POINT = PHYS == 1 && P == 1;
    static void elem_point(const void *ops, const void *tab, const Mesh &m, const State<R> &s, const Phys &ph,
                           int stage, int zero_rr, int diff, int nsm, const Tune &tn, cudaStream_t st) {
        if constexpr (HAS_POINT) {
            const long tri_per_cta = 256 / 4;
            const int blocks = (int)std::min<long>(((long)m.ntri + tri_per_cta - 1) / tri_per_cta, (long)nsm * 8);
            k_rsdl_ins_p1<R><<<blocks, 256, 0, st>>>(static_cast<const InsP1Ops<R> *>(ops), m, s, ph, stage, zero_rr,
                                                     diff);
            if (m.ncurved > 0) {
                constexpr int EPC = C::WPC * C::EPW;
                const int cap = nsm * tn.elem_cap;
                k_rsdl_elem<R, P, PHYS, true><<<std::min(nblk(m.ncurved, EPC), cap), C::WPC * 32, smem(), st>>>(
                    reinterpret_cast<const DevTables<R, P> *>(tab), m, s, ph, stage, zero_rr, diff, ElemMat<R>{},
                    ElemJac<R>{});
            }
        }
    }
    static void point_build(const hp_basis_tables &b, std::vector<unsigned char> &ops) {
        InsP1Ops<R> o;
        build_ins_p1<R>(b, o);
        ops.resize(sizeof(o));
        std::memcpy(ops.data(), &o, sizeof(o));
    }
    static void mma_build(const hp_basis_tables &b, std::vector<unsigned char> &ops, std::vector<unsigned char> &small) {
        if constexpr (DBL) {
            InsMmaSmall<P> sm;
            std::vector<double> o;
            build_ins_mma<P>(b, o, sm);
            ops.resize(o.size() * sizeof(double));
            std::memcpy(ops.data(), o.data(), ops.size());
            small.resize(sizeof(sm));
            std::memcpy(small.data(), &sm, sizeof(sm));
        } else {
            InsMmaSmallF<P> sm;
            std::vector<float> o;
            build_ins_tf32<P>(b, o, sm);
            ops.resize(o.size() * sizeof(float));
            std::memcpy(ops.data(), o.data(), ops.size());
            small.resize(sizeof(sm));
            std::memcpy(small.data(), &sm, sizeof(sm));
        }
    }
    static void base_pts(const void *tab, const Mesh &m, const State<R> &s, R *bpt, cudaStream_t st) {
        if constexpr (HAS_MMA && !DBL)
            k_base_points<P><<<nblk(2L * m.ntri, 128), 128, 0, st>>>(reinterpret_cast<const DevTables<float, P> *>(tab),
                                                                     m, s.ubv, s.ubs, s.ubi, bpt);
    }
    static cudaError_t set_smem_attr() {
        cudaError_t e = cudaFuncSetAttribute(k_rsdl_elem<R, P, PHYS, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem());
        if (e != cudaSuccess) return e;
        if constexpr (HAS_MMA) {
            if constexpr (DBL)
                e = cudaFuncSetAttribute(k_rsdl_ins_mma<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, mma_smem());
            else
                e = cudaFuncSetAttribute(k_rsdl_ins_tf32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, mma_smem());
            if (e != cudaSuccess) return e;
        }
        return cudaFuncSetAttribute(k_rsdl_elem<R, P, PHYS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem());
    }
    static void l2err(const void *tab, const double *wtn, const Mesh &m, const State<R> &s, int NV,
                      const DevField &f, double *part, int blocks, cudaStream_t st) {
        if constexpr (std::is_same<R, double>::value) {
            WtN<P> w;
            for (int j = 0; j <= P; ++j) w.w[j] = wtn[j];
            k_l2error<P><<<blocks, 128, 0, st>>>(reinterpret_cast<const DevTables<double, P> *>(tab), m, s, NV, f, w,
                                                 part);
        }
    }
    static Launchers<R> get() {
        Launchers<R> L;
        L.tab_bytes = sizeof(DevTables<R, P>);
        L.fill = &fill;
        L.elem = &elem;
        L.bflux = &bflux;
        L.side = &side;
        L.intr = &intr;
        L.vert = &vert;
        L.elem_smem = smem();
        L.set_smem = &set_smem_attr;
        L.emat_len = &emat_len;
        L.emat_build = &emat_build;
        L.emat_apply = &emat_apply;
        L.elem_jac = &elem_jac;
        L.elem_mma = HAS_MMA ? &elem_mma : nullptr;
        L.elem_point = HAS_POINT ? &elem_point : nullptr;
        L.point_build = HAS_POINT ? &point_build : nullptr;
        L.mma_build = HAS_MMA ? &mma_build : nullptr;
        L.base_pts = (HAS_MMA && !DBL) ? &base_pts : nullptr;
        L.bpt_per_elem = 2 * (P + 1) * (P + 1);
        L.l2err = std::is_same<R, double>::value ? &l2err : nullptr;
        return L;
    }
};

template <typename R, int PHYS>
static bool get_launchers_phys(int p, Launchers<R> &L) {
    switch (p) {
        case 1: L = LaunchImpl<R, 1, PHYS>::get(); return true;
        case 2: L = LaunchImpl<R, 2, PHYS>::get(); return true;
        case 3: L = LaunchImpl<R, 3, PHYS>::get(); return true;
        case 4: L = LaunchImpl<R, 4, PHYS>::get(); return true;
        case 5: L = LaunchImpl<R, 5, PHYS>::get(); return true;
        case 6: L = LaunchImpl<R, 6, PHYS>::get(); return true;
        case 7: L = LaunchImpl<R, 7, PHYS>::get(); return true;
        case 8: L = LaunchImpl<R, 8, PHYS>::get(); return true;
    }
    return false;
}

template <typename R>
static bool get_launchers(int p, int phys, Launchers<R> &L) {
    return phys ? get_launchers_phys<R, 1>(p, L) : get_launchers_phys<R, 0>(p, L);
}

// FP64 preconditioner set-up kernel launch (double only)
static void launch_prcn(int p, int phys, const void *tab, const Mesh &m, const State<double> &s, const Phys &ph,
                        int *err, const float *lsc, int ld, float clampv, cudaStream_t st) {
#define PR_CASE(PP)                                                                                           \
    case PP:                                                                                                  \
        if (phys)                                                                                             \
            k_prcn_elem<double, PP, 1><<<nblk(m.ntri, 128), 128, 0, st>>>(                                      \
                reinterpret_cast<const DevTables<double, PP> *>(tab), m, s, ph, err, lsc, ld, clampv);        \
        else                                                                                                  \
            k_prcn_elem<double, PP, 0><<<nblk(m.ntri, 128), 128, 0, st>>>(                                      \
                reinterpret_cast<const DevTables<double, PP> *>(tab), m, s, ph, err, lsc, ld, clampv);        \
        break;
    switch (p) { PR_CASE(1) PR_CASE(2) PR_CASE(3) PR_CASE(4) PR_CASE(5) PR_CASE(6) PR_CASE(7) PR_CASE(8) }
#undef PR_CASE
}

struct hp_gpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int p = 0, NV = 0, npnt = 0, nseg = 0, ntri = 0, nbseg = 0, sm = 0, im = 0, nsm = 148;
    int ncurved = 0;  // curved elements (tri.info > -1)
    Phys ph{};
    Launchers<double> L{};
    Launchers<float> L32{};
    Mesh mesh{};
    State<double> st{};
    State<float> s32{};  // correction-form FP32 smoother state (allocated on first mixed solve)
    bool mixed_ready = false;
    void *d_tab = nullptr, *d_tab32 = nullptr;
    DevMinv<double> *d_minv = nullptr;
    DevMinv<float> *d_minv32 = nullptr;
    cudaGraphExec_t g_update32 = nullptr;
    // learned preconditioner correction
    const float *lsc = nullptr;
    int lsc_ld = 1;
    float lsc_clamp = 0.f;
    hp_mlp *net = nullptr;
    float *d_feat = nullptr, *d_netout = nullptr;
    double vdiag = 0.0;
    unsigned long long *d_slot = nullptr;
    double *d_hist = nullptr;
    int hist_cap = 0;
    int *d_iter = nullptr;
    int *d_err = nullptr;
    double *d_part = nullptr;
    int npart = 0;
    std::vector<void *> allocs;
    cudaMemPool_t pool = nullptr;
    cudaGraphExec_t g_update = nullptr;  // one update() incl. maxres -> hist slot advance
    bool prcn_ready = false;
    size_t lv = 0, ls = 0, li = 0;  // element counts of v/s/i arrays
    // multigrid: this context as a coarse level of `fine` (tri_hp's coarse/fine pointers)
    hp_gpu_ctx *fine = nullptr;
    int mg_kind = 0;  // 0 none, 1 p-level on the same mesh, 2 h-level (coarser mesh, p = 1)
    double fadd = 1.0;
    bool fas_pending = false;  // restricted, driving term not formed yet (tri_hp::isfrst)
    double *res0v = nullptr, *res0s = nullptr, *res0i = nullptr;  // restricted fine residual
    double *uc0v = nullptr, *uc0s = nullptr, *uc0i = nullptr;     // state at restriction (vug_frst)
    double *fasv = nullptr, *fass = nullptr, *fasi = nullptr;     // FAS source dres
    int *f2c_tri = nullptr, *c2f_tri = nullptr;
    double *f2c_wt = nullptr, *c2f_wt = nullptr;
    Tune tune[2];  // launch shapes for FP64 [0] and FP32 [1]
    // FP64 element kernel: HP_ELEM_TENSOR (ins: k_rsdl_ins_mma) or HP_ELEM_SCALAR (k_rsdl_elem)
    int elem_kind = 0;
    void *d_mma = nullptr, *d_mma32 = nullptr;            // dense operators in fragment order (FP64, TF32)
    void *d_p1 = nullptr, *d_p1_32 = nullptr;             // operators of the p = 1 point kernel (FP64, FP32)
    std::vector<unsigned char> mma_small, mma_small32;  // derivative tables (kernel parameters)
    float *d_bpt32 = nullptr;                           // FP32 base point values (correction form)
    double wtn[HP_MXGP] = {0};                // Gauss-Jacobi weights (l2error)
    double *d_l2part = nullptr;               // l2error per-block partials
    float tune_ms[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // tuned element-part and minvrt times
    // cd element operators (FP64 built by the element kernel, FP32 converted copy)
    bool emat_on = false, emat_built = false;
    ElemMat<double> em{};
    ElemMat<float> em32{};
    // FP32 multigrid on the correction equation: restricted residual and entry state
    float *r0v32 = nullptr, *r0s32 = nullptr, *r0i32 = nullptr, *c0v32 = nullptr, *c0s32 = nullptr, *c0i32 = nullptr;
};

// Device memory comes from one library-private stream-ordered pool per device: a
// context's buffers return to the pool when it is destroyed and the next context
// reuses them without a driver allocation (creating and destroying whole solver
// hierarchies stays cheap). The pool keeps up to 16 GiB reserved between uses.
static cudaMemPool_t pool_for(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = 16ull << 30;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[device] = pool;
    return pool;
}

static int dalloc(hp_gpu_ctx *c, void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = c->pool ? cudaMallocFromPoolAsync(p, bytes, c->pool, c->stream) : cudaErrorInvalidValue;
    if (e != cudaSuccess) {
        set_err("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return HP_ENOMEM;
    }
    c->allocs.push_back(*p);
    // every buffer starts zeroed: nothing reads leftovers of an earlier allocation
    e = cudaMemsetAsync(*p, 0, bytes, c->stream);
    if (e != cudaSuccess) {
        set_err("cudaMemsetAsync(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return HP_ECUDA;
    }
    return HP_OK;
}

template <typename T>
static int upload(hp_gpu_ctx *c, T **d, const T *h, size_t n) {
    int r = dalloc(c, (void **)d, n * sizeof(T));
    if (r) return r;
    if (n && h) CK(cudaMemcpyAsync(*d, h, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return HP_OK;
}

extern "C" const char *hp_gpu_last_error(void) { return g_err.c_str(); }

extern "C" int hp_gpu_create(const hp_mesh_desc *m, const hp_basis_tables *b, const hp_phys_params *ph, int device,
                             void *stream, hp_gpu_ctx **out) {
    g_err.clear();
    if (!m || !b || !ph || !out) { set_err("null argument"); return HP_EINVAL; }
    if (b->p < 1 || b->p > HP_MAXP) { set_err("p=%d outside [1,%d]", b->p, HP_MAXP); return HP_EINVAL; }
    if (ph->physics != HP_PHYS_CD && ph->physics != HP_PHYS_INS) { set_err("unknown physics"); return HP_EINVAL; }
    if (ph->nstage < 1 || ph->nstage > 7) { set_err("nstage=%d outside [1,7]", ph->nstage); return HP_EINVAL; }
    if (ph->bd0 != 0.0) { set_err("only steady problems (bd0 = 0) are supported"); return HP_ENOTSUP; }
    if (m->npnt <= 0 || m->nseg <= 0 || m->ntri <= 0) { set_err("empty mesh"); return HP_EINVAL; }
    if (ph->physics == HP_PHYS_INS && m->nbseg > 0 && !m->bseg_pibc) {
        for (int e = 0; e < m->nbseg; ++e)
            if ((m->bseg_kind[e] & HP_BC_FLUX_MASK) == HP_BC_FLUX_INS_GENERIC) {
                set_err("ins generic boundary flux needs bseg_pibc");
                return HP_EINVAL;
            }
    }
    hp_gpu_ctx *c = new hp_gpu_ctx();
    auto fail = [&](int code) {
        hp_gpu_destroy(c);
        return code;
    };
    if (device >= 0) {
        if (cudaSetDevice(device) != cudaSuccess) { set_err("cudaSetDevice(%d) failed", device); delete c; return HP_ECUDA; }
        c->device = device;
    } else {
        cudaGetDevice(&c->device);
    }
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    c->nsm = nsm > 0 ? nsm : 148;
    if (stream) c->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_err("cudaStreamCreate failed");
            delete c;
            return HP_ECUDA;
        }
        c->own_stream = true;
    }
    c->pool = pool_for(c->device);
    if (!c->pool) { set_err("cudaMemPoolCreate failed on device %d", c->device); return fail(HP_ECUDA); }
    const int physics = ph->physics;
    c->p = b->p; c->sm = b->sm; c->im = b->im;
    c->NV = physics == HP_PHYS_INS ? 3 : 1;
    c->npnt = m->npnt; c->nseg = m->nseg; c->ntri = m->ntri; c->nbseg = m->nbseg;
    bool ok = get_launchers<double>(c->p, physics, c->L) && get_launchers<float>(c->p, physics, c->L32);
    if (!ok) { set_err("p=%d not built", c->p); return fail(HP_ENOTSUP); }
    if (c->L.set_smem() != cudaSuccess || c->L32.set_smem() != cudaSuccess) {
        set_err("smem attribute (%d bytes) rejected", c->L.elem_smem);
        return fail(HP_ECUDA);
    }
    Phys &P = c->ph;
    P.physics = physics; P.NV = c->NV; P.nstage = ph->nstage;
    for (int k = 0; k < 8; ++k) { P.alpha[k] = ph->alpha[k]; P.beta[k] = ph->beta[k]; }
    P.alpha[ph->nstage] = 1.0; P.beta[ph->nstage] = 1.0;
    P.cfl = ph->cfl; P.bd0 = ph->bd0; P.adis = ph->adis; P.rho = ph->rho; P.mu = ph->mu;
    P.rhocv = ph->rhocv; P.kcond = ph->kcond; P.ax = ph->ax; P.ay = ph->ay; P.src = ph->src;

    // host-side mesh preprocessing: seg_loc and vertex incidence
    const int np = m->npnt, ns = m->nseg, nt = m->ntri;
    std::vector<int> seg_loc(2 * ns, -1);
    for (int s = 0; s < ns; ++s)
        for (int k = 0; k < 2; ++k) {
            int t = m->seg_tri[2 * s + k];
            if (t < 0) continue;
            if (t >= nt) { set_err("seg_tri out of range"); return fail(HP_EINVAL); }
            for (int i = 0; i < 3; ++i)
                if (m->tri_seg[3 * t + i] == s) seg_loc[2 * s + k] = i;
            if (seg_loc[2 * s + k] < 0) { set_err("seg %d not a side of tri %d", s, t); return fail(HP_EINVAL); }
        }
    std::vector<int> vs_ptr(np + 1, 0), vt_ptr(np + 1, 0);
    for (int s = 0; s < ns; ++s)
        for (int k = 0; k < 2; ++k) {
            int v = m->seg_pnt[2 * s + k];
            if (v < 0 || v >= np) { set_err("seg_pnt out of range"); return fail(HP_EINVAL); }
            vs_ptr[v + 1]++;
        }
    for (int t = 0; t < nt; ++t)
        for (int i = 0; i < 3; ++i) {
            int v = m->tri_pnt[3 * t + i];
            if (v < 0 || v >= np) { set_err("tri_pnt out of range"); return fail(HP_EINVAL); }
            int s = m->tri_seg[3 * t + i];
            if (s < 0 || s >= ns) { set_err("tri_seg out of range"); return fail(HP_EINVAL); }
            vt_ptr[v + 1]++;
        }
    for (int v = 0; v < np; ++v) { vs_ptr[v + 1] += vs_ptr[v]; vt_ptr[v + 1] += vt_ptr[v]; }
    std::vector<int> vs_idx(vs_ptr[np]), vt_idx(vt_ptr[np]);
    {
        std::vector<int> a(vs_ptr.begin(), vs_ptr.end() - 1), bb(vt_ptr.begin(), vt_ptr.end() - 1);
        for (int s = 0; s < ns; ++s)
            for (int k = 0; k < 2; ++k) vs_idx[a[m->seg_pnt[2 * s + k]]++] = 2 * s + k;
        for (int t = 0; t < nt; ++t)
            for (int i = 0; i < 3; ++i) vt_idx[bb[m->tri_pnt[3 * t + i]]++] = 4 * t + i;
    }
    std::vector<int> vess(np, 0), sess(ns, 0), seg_bdry(ns, -1), vb_idx(2 * (size_t)np, -1);
    for (int e = 0; e < m->nbseg; ++e) {
        int s = m->bseg[e];
        if (s < 0 || s >= ns) { set_err("bseg out of range"); return fail(HP_EINVAL); }
        if (seg_bdry[s] >= 0) { set_err("segment %d listed twice as a boundary edge", s); return fail(HP_EINVAL); }
        seg_bdry[s] = e;
        for (int end = 0; end < 2; ++end) {
            int *slot = &vb_idx[2 * (size_t)m->seg_pnt[2 * s + end]];
            if (slot[0] < 0) slot[0] = 2 * e + end;
            else if (slot[1] < 0) slot[1] = 2 * e + end;
            else { set_err("vertex %d ends more than two boundary edges", m->seg_pnt[2 * s + end]); return fail(HP_EINVAL); }
        }
        int mask = m->bseg_kind[e] & 0xFF;
        sess[s] |= mask;
        vess[m->seg_pnt[2 * s]] |= mask;
        vess[m->seg_pnt[2 * s + 1]] |= mask;
    }
    int r = 0;
    double *d_pnts;
    int *d_tp, *d_ts, *d_tg, *d_sp, *d_st, *d_sl, *d_vsp, *d_vsi, *d_vtp, *d_vti, *d_vess, *d_sess, *d_bseg, *d_bkind;
    double *d_bpibc;
    if ((r = upload(c, &d_pnts, m->pnts, 2 * (size_t)np))) return fail(r);
    if ((r = upload(c, &d_tp, m->tri_pnt, 3 * (size_t)nt))) return fail(r);
    if ((r = upload(c, &d_ts, m->tri_seg, 3 * (size_t)nt))) return fail(r);
    if ((r = upload(c, &d_tg, m->tri_sgn, 3 * (size_t)nt))) return fail(r);
    if ((r = upload(c, &d_sp, m->seg_pnt, 2 * (size_t)ns))) return fail(r);
    if ((r = upload(c, &d_st, m->seg_tri, 2 * (size_t)ns))) return fail(r);
    if ((r = upload(c, &d_sl, seg_loc.data(), seg_loc.size()))) return fail(r);
    if ((r = upload(c, &d_vsp, vs_ptr.data(), vs_ptr.size()))) return fail(r);
    if ((r = upload(c, &d_vsi, vs_idx.data(), vs_idx.size()))) return fail(r);
    if ((r = upload(c, &d_vtp, vt_ptr.data(), vt_ptr.size()))) return fail(r);
    if ((r = upload(c, &d_vti, vt_idx.data(), vt_idx.size()))) return fail(r);
    if ((r = upload(c, &d_vess, vess.data(), vess.size()))) return fail(r);
    if ((r = upload(c, &d_sess, sess.data(), sess.size()))) return fail(r);
    if ((r = upload(c, &d_bseg, m->bseg, (size_t)m->nbseg))) return fail(r);
    if ((r = upload(c, &d_bkind, m->bseg_kind, (size_t)m->nbseg))) return fail(r);
    int *d_sbd, *d_vbi;
    if ((r = upload(c, &d_sbd, seg_bdry.data(), seg_bdry.size()))) return fail(r);
    if ((r = upload(c, &d_vbi, vb_idx.data(), vb_idx.size()))) return fail(r);
    // owner order of the assembly buffers (Mesh::vpos, spos)
    std::vector<int> vpos(3 * (size_t)nt, -1), spos(3 * (size_t)nt, -1);
    for (int j = 0; j < vt_ptr[np]; ++j) vpos[3 * (size_t)(vt_idx[j] >> 2) + (vt_idx[j] & 3)] = j;
    for (int sd = 0; sd < ns; ++sd)
        for (int k = 0; k < 2; ++k) {
            const int t = m->seg_tri[2 * sd + k];
            if (t >= 0) spos[3 * (size_t)t + seg_loc[2 * sd + k]] = 2 * sd + k;
        }
    for (size_t q = 0; q < spos.size(); ++q)
        if (spos[q] < 0 || vpos[q] < 0) {
            set_err("triangle %zu side %zu is not listed in seg.tri", q / 3, q % 3);
            return fail(HP_EINVAL);
        }
    int *d_vpos, *d_spos;
    if ((r = upload(c, &d_vpos, vpos.data(), vpos.size()))) return fail(r);
    if ((r = upload(c, &d_spos, spos.data(), spos.size()))) return fail(r);
    std::vector<double> pibc((size_t)std::max(1, m->nbseg) * b->gpx, 0.0);
    if (m->bseg_pibc) std::copy(m->bseg_pibc, m->bseg_pibc + (size_t)m->nbseg * b->gpx, pibc.begin());
    if ((r = upload(c, &d_bpibc, pibc.data(), pibc.size()))) return fail(r);
    Mesh &M = c->mesh;
    M.npnt = np; M.nseg = ns; M.ntri = nt; M.nbseg = m->nbseg;
    M.pnts = d_pnts; M.tri_pnt = d_tp; M.tri_seg = d_ts; M.tri_sgn = d_tg;
    M.seg_pnt = d_sp; M.seg_tri = d_st; M.seg_loc = d_sl;
    M.vs_ptr = d_vsp; M.vs_idx = d_vsi; M.vt_ptr = d_vtp; M.vt_idx = d_vti;
    M.vess = d_vess; M.sess = d_sess; M.bseg = d_bseg; M.bkind = d_bkind; M.bpibc = d_bpibc;
    M.tri_cv = nullptr; M.crv_cht = nullptr; M.bcrd = nullptr; M.ncurved = 0; M.crv_tri = nullptr;
    M.seg_bdry = d_sbd; M.vb_idx = d_vbi; M.vpos = d_vpos; M.spos = d_spos;
    {   // per-triangle constants of the straight branch (tri_hp_ins::element_rsdl's ldcrd and
        // the inscribed-radius length scale of tau, tri_mesh/tprims.cpp:224-241)
        std::vector<double> g((size_t)8 * nt, 0.0);
        const double pf = 0.25 * (b->p + 1) * (b->p + 1);
        for (int t = 0; t < nt; ++t) {
            const double *x0 = m->pnts + 2 * m->tri_pnt[3 * t], *x1 = m->pnts + 2 * m->tri_pnt[3 * t + 1],
                         *x2 = m->pnts + 2 * m->tri_pnt[3 * t + 2];
            double *o = &g[(size_t)8 * t];
            o[0] = 0.5 * (x2[0] - x1[0]); o[1] = 0.5 * (x0[0] - x1[0]);
            o[2] = 0.5 * (x2[1] - x1[1]); o[3] = 0.5 * (x0[1] - x1[1]);
            const double dx1 = x0[0] - x2[0], dy1 = x0[1] - x2[1], dx2 = x1[0] - x0[0], dy2 = x1[1] - x0[1];
            const double area = dx1 * dy2 - dy1 * dx2;
            const double perim = std::sqrt(dx1 * dx1 + dy1 * dy1) + std::sqrt(dx2 * dx2 + dy2 * dy2) +
                                 std::sqrt((dx1 + dx2) * (dx1 + dx2) + (dy1 + dy2) * (dy1 + dy2));
            const double he = (area / perim) / pf;
            o[4] = 1.0 / (o[0] * o[3] - o[2] * o[1]);
            o[5] = he;
            o[6] = 1.0 / he;
        }
        double *d_g;
        if ((r = upload(c, &d_g, g.data(), g.size()))) return fail(r);
        M.tgeo = d_g;
    }

    // curved elements (tri_hp::metric::setinfo, metric.cpp:44-70, for p > 1): the
    // owner triangle of every boundary side with non-zero position modes, with its
    // vertex and side position modes (crdtocht, gtol.cpp:204-248)
    if (m->bseg_crd && b->sm > 0 && m->nbseg > 0) {
        const int sm = b->sm, bmv = b->bm;
        std::vector<int> tri_cv(nt, -1);
        std::vector<const double *> side_modes((size_t)3 * nt, nullptr);
        int ncv = 0;
        for (int e = 0; e < m->nbseg; ++e) {
            const double *md = m->bseg_crd + (size_t)e * sm * 2;
            bool nz = false;
            for (int k = 0; k < 2 * sm; ++k) nz = nz || md[k] != 0.0;
            if (!nz) continue;
            const int sg = m->bseg[e], t = m->seg_tri[2 * sg], i = seg_loc[2 * sg];
            if (t < 0 || i < 0) { set_err("curved boundary side %d has no triangle", sg); return fail(HP_EINVAL); }
            side_modes[3 * (size_t)t + i] = md;
            if (tri_cv[t] < 0) tri_cv[t] = ncv++;
        }
        if (ncv > 0) {
            std::vector<double> cht((size_t)ncv * 2 * bmv, 0.0);
            std::vector<int> crv_tri(ncv);
            for (int t = 0; t < nt; ++t) {
                if (tri_cv[t] < 0) continue;
                crv_tri[tri_cv[t]] = t;
                double *cc = &cht[(size_t)tri_cv[t] * 2 * bmv];
                for (int n = 0; n < 2; ++n) {
                    for (int k = 0; k < 3; ++k) cc[n * bmv + k] = m->pnts[2 * m->tri_pnt[3 * t + k] + n];
                    for (int i = 0; i < 3; ++i) {
                        const double *md = side_modes[3 * (size_t)t + i];
                        if (!md) continue;
                        const int sgn = m->tri_sgn[3 * t + i];
                        for (int k = 0; k < sm; ++k)
                            cc[n * bmv + 3 + i * sm + k] = ((k & 1) && sgn < 0 ? -1.0 : 1.0) * md[k * 2 + n];
                    }
                }
            }
            int *d_cv, *d_ctri;
            double *d_cht, *d_bcrd;
            if ((r = upload(c, &d_cv, tri_cv.data(), tri_cv.size()))) return fail(r);
            if ((r = upload(c, &d_cht, cht.data(), cht.size()))) return fail(r);
            if ((r = upload(c, &d_bcrd, m->bseg_crd, (size_t)m->nbseg * sm * 2))) return fail(r);
            if ((r = upload(c, &d_ctri, crv_tri.data(), crv_tri.size()))) return fail(r);
            M.tri_cv = d_cv; M.crv_cht = d_cht; M.bcrd = d_bcrd; M.ncurved = ncv; M.crv_tri = d_ctri;
            c->ncurved = ncv;
        }
    }

    // tables
    std::vector<unsigned char> htab(c->L.tab_bytes);
    c->L.fill(*b, htab.data());
    if ((r = upload(c, (unsigned char **)&c->d_tab, htab.data(), htab.size()))) return fail(r);
    for (int j = 0; j < b->gpn && j < HP_MXGP; ++j) c->wtn[j] = b->wtn[j];
    if (c->L.mma_build && c->L32.mma_build) {
        std::vector<unsigned char> ops, ops32;
        c->L.mma_build(*b, ops, c->mma_small);
        c->L32.mma_build(*b, ops32, c->mma_small32);
        if ((r = upload(c, (unsigned char **)&c->d_mma, ops.data(), ops.size()))) return fail(r);
        if ((r = upload(c, (unsigned char **)&c->d_mma32, ops32.data(), ops32.size()))) return fail(r);
        // at p = 1 and 2 the scalar kernel's lane groups (4 and 2 triangles per warp) are
        // faster than two triangles per tensor-core warp (measured: 0.080 vs 0.153 ms and
        // 0.205 vs 0.205 ms for 131k triangles); at p = 1 the point kernel is faster still
        c->elem_kind = c->p >= 3 ? HP_ELEM_TENSOR : HP_ELEM_SCALAR;
    }
    if (c->L.point_build && c->L32.point_build) {
        std::vector<unsigned char> ops, ops32;
        c->L.point_build(*b, ops);
        c->L32.point_build(*b, ops32);
        if ((r = upload(c, (unsigned char **)&c->d_p1, ops.data(), ops.size()))) return fail(r);
        if ((r = upload(c, (unsigned char **)&c->d_p1_32, ops32.data(), ops32.size()))) return fail(r);
        c->elem_kind = HP_ELEM_POINT;
    }
    DevMinv<double> hm;
    fill_minv<double>(*b, hm);
    c->vdiag = b->vdiag;
    if ((r = upload(c, &c->d_minv, &hm, 1))) return fail(r);
    std::vector<unsigned char> htab32(c->L32.tab_bytes);
    c->L32.fill(*b, htab32.data());
    if ((r = upload(c, (unsigned char **)&c->d_tab32, htab32.data(), htab32.size()))) return fail(r);
    DevMinv<float> hm32;
    fill_minv<float>(*b, hm32);
    if ((r = upload(c, &c->d_minv32, &hm32, 1))) return fail(r);

    // state
    const int NV = c->NV;
    c->lv = (size_t)np * NV; c->ls = (size_t)ns * c->sm * NV; c->li = (size_t)nt * c->im * NV;
    double **vptrs[] = {&c->st.ugv, &c->st.u0v, &c->st.resv, &c->st.rrv};
    double **sptrs[] = {&c->st.ugs, &c->st.u0s, &c->st.ress, &c->st.rrs};
    double **iptrs[] = {&c->st.ugi, &c->st.u0i, &c->st.resi, &c->st.rri};
    for (auto pp : vptrs) { if ((r = dalloc(c, (void **)pp, c->lv * 8))) return fail(r); CK(cudaMemsetAsync(*pp, 0, c->lv * 8, c->stream)); }
    for (auto pp : sptrs) { if ((r = dalloc(c, (void **)pp, c->ls * 8))) return fail(r); CK(cudaMemsetAsync(*pp, 0, std::max<size_t>(c->ls, 2) * 8, c->stream)); }
    for (auto pp : iptrs) { if ((r = dalloc(c, (void **)pp, c->li * 8))) return fail(r); CK(cudaMemsetAsync(*pp, 0, std::max<size_t>(c->li, 2) * 8, c->stream)); }
    if ((r = dalloc(c, (void **)&c->st.vprcn, (size_t)np * NV * 8))) return fail(r);
    if ((r = dalloc(c, (void **)&c->st.sprcn, (size_t)ns * NV * 8))) return fail(r);
    if ((r = dalloc(c, (void **)&c->st.tprcn, (size_t)nt * NV * 8))) return fail(r);
    if ((r = dalloc(c, (void **)&c->st.tau, (size_t)nt * NV * 8))) return fail(r);
    // per-element vertex / side residuals and per-edge boundary fluxes of the FP64
    // assembly by gather (State::elim)
    const size_t nel = (size_t)3 * nt * NV + (size_t)2 * ns * std::max(1, b->sm) * NV,
                 nbr = (size_t)std::max(1, m->nbseg) * (b->sm + 2) * NV;
    if ((r = dalloc(c, (void **)&c->st.elim, nel * 8))) return fail(r);
    if ((r = dalloc(c, (void **)&c->st.elre, nel * 8))) return fail(r);
    if ((r = dalloc(c, (void **)&c->st.bres, nbr * 8))) return fail(r);
    CK(cudaMemsetAsync(c->st.elre, 0, nel * 8, c->stream));
    if ((r = dalloc(c, (void **)&c->d_slot, 4 * 8))) return fail(r);
    CK(cudaMemsetAsync(c->d_slot, 0, 32, c->stream));
    c->hist_cap = 1 << 16;
    if ((r = dalloc(c, (void **)&c->d_hist, (size_t)c->hist_cap * 8))) return fail(r);
    if ((r = dalloc(c, (void **)&c->d_iter, 16))) return fail(r);
    CK(cudaMemsetAsync(c->d_iter, 0, 16, c->stream));
    if ((r = dalloc(c, (void **)&c->d_err, 16))) return fail(r);
    c->npart = 4 * c->nsm;
    if ((r = dalloc(c, (void **)&c->d_part, (size_t)c->npart * 2 * 8))) return fail(r);
    CK(cudaStreamSynchronize(c->stream));
    *out = c;
    return HP_OK;
}

extern "C" int hp_gpu_destroy(hp_gpu_ctx *c) {
    if (!c) return HP_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->g_update) cudaGraphExecDestroy(c->g_update);
    if (c->g_update32) cudaGraphExecDestroy(c->g_update32);
    for (void *p : c->allocs) cudaFreeAsync(p, c->stream);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HP_OK;
}

extern "C" int hp_gpu_sizes(const hp_gpu_ctx *c, int *nv, int *sm, int *im) {
    if (!c) return HP_EINVAL;
    if (nv) *nv = c->NV;
    if (sm) *sm = c->sm;
    if (im) *im = c->im;
    return HP_OK;
}

extern "C" int hp_gpu_enqueue_upload_state(hp_gpu_ctx *c, const double *v, const double *s, const double *i) {
    if (!c || !v || (c->ls && !s) || (c->li && !i)) return HP_EINVAL;
    CK(cudaMemcpyAsync(c->st.ugv, v, c->lv * 8, cudaMemcpyHostToDevice, c->stream));
    if (c->ls) CK(cudaMemcpyAsync(c->st.ugs, s, c->ls * 8, cudaMemcpyHostToDevice, c->stream));
    if (c->li) CK(cudaMemcpyAsync(c->st.ugi, i, c->li * 8, cudaMemcpyHostToDevice, c->stream));
    return HP_OK;
}

extern "C" int hp_gpu_upload_state(hp_gpu_ctx *c, const double *v, const double *s, const double *i) {
    const int r = hp_gpu_enqueue_upload_state(c, v, s, i);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}

static int enqueue_download3(hp_gpu_ctx *c, const double *dv, const double *ds, const double *di, double *v,
                             double *s, double *i) {
    if (v) CK(cudaMemcpyAsync(v, dv, c->lv * 8, cudaMemcpyDeviceToHost, c->stream));
    if (s && c->ls) CK(cudaMemcpyAsync(s, ds, c->ls * 8, cudaMemcpyDeviceToHost, c->stream));
    if (i && c->li) CK(cudaMemcpyAsync(i, di, c->li * 8, cudaMemcpyDeviceToHost, c->stream));
    return HP_OK;
}

static int download3(hp_gpu_ctx *c, const double *dv, const double *ds, const double *di, double *v, double *s,
                     double *i) {
    const int r = enqueue_download3(c, dv, ds, di, v, s, i);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}

extern "C" int hp_gpu_enqueue_download_residual(hp_gpu_ctx *c, double *v, double *s, double *i) {
    if (!c) return HP_EINVAL;
    return enqueue_download3(c, c->st.resv, c->st.ress, c->st.resi, v, s, i);
}

extern "C" int hp_gpu_download_state(hp_gpu_ctx *c, double *v, double *s, double *i) {
    if (!c) return HP_EINVAL;
    return download3(c, c->st.ugv, c->st.ugs, c->st.ugi, v, s, i);
}
extern "C" int hp_gpu_download_residual(hp_gpu_ctx *c, double *v, double *s, double *i) {
    if (!c) return HP_EINVAL;
    return download3(c, c->st.resv, c->st.ress, c->st.resi, v, s, i);
}
extern "C" int hp_gpu_download_prcn(hp_gpu_ctx *c, double *vp, double *sp, double *tp, double *tau) {
    if (!c) return HP_EINVAL;
    if (vp) CK(cudaMemcpyAsync(vp, c->st.vprcn, (size_t)c->npnt * c->NV * 8, cudaMemcpyDeviceToHost, c->stream));
    if (sp) CK(cudaMemcpyAsync(sp, c->st.sprcn, (size_t)c->nseg * c->NV * 8, cudaMemcpyDeviceToHost, c->stream));
    if (tp) CK(cudaMemcpyAsync(tp, c->st.tprcn, (size_t)c->ntri * c->NV * 8, cudaMemcpyDeviceToHost, c->stream));
    if (tau) CK(cudaMemcpyAsync(tau, c->st.tau, (size_t)c->ntri * c->NV * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return HP_OK;
}
extern "C" int hp_gpu_device_ptrs(hp_gpu_ctx *c, double **ugv, double **ugs, double **ugi, double **resv,
                                  double **ress, double **resi) {
    if (!c) return HP_EINVAL;
    if (ugv) *ugv = c->st.ugv;
    if (ugs) *ugs = c->st.ugs;
    if (ugi) *ugi = c->st.ugi;
    if (resv) *resv = c->st.resv;
    if (ress) *ress = c->st.ress;
    if (resi) *resi = c->st.resi;
    return HP_OK;
}

static ElemMat<double> emat_of(hp_gpu_ctx *c, double) { return c->em; }
static ElemMat<float> emat_of(hp_gpu_ctx *c, float) { return c->em32; }
static const Tune &tune_of(hp_gpu_ctx *c, double) { return c->tune[0]; }
static const Tune &tune_of(hp_gpu_ctx *c, float) { return c->tune[1]; }

// Element part of rsdl(stage): the stored cd element operators once built, else the
// matrix-free element kernel.
template <typename R>
static void launch_elem(hp_gpu_ctx *c, const Launchers<R> &L, const void *tab, const State<R> &st, const Phys &ph,
                        int stage, int zero_rr, int diff) {
    if (c->emat_on && c->emat_built && ph.physics == HP_PHYS_CD && !diff)
        L.emat_apply(emat_of(c, R()), c->mesh, st, ph, stage, zero_rr, c->nsm, tune_of(c, R()), c->stream);
    // FP64: the DMMA kernel; FP32: the TF32 kernel in correction form only (the operand
    // rounding to TF32 is ~5e-4 of the fluxes, which a plain-form residual near convergence,
    // much smaller than its fluxes, would not resolve; the correction form has no such
    // cancellation)
    else if (c->elem_kind == HP_ELEM_TENSOR && L.elem_mma &&
             (std::is_same<R, double>::value ? !diff : (diff && st.bpt != nullptr)))
        L.elem_mma(std::is_same<R, double>::value ? c->d_mma : c->d_mma32,
                   std::is_same<R, double>::value ? c->mma_small.data() : c->mma_small32.data(), tab, c->mesh, st, ph,
                   stage, zero_rr, diff, c->nsm, tune_of(c, R()), c->stream);
    else if (c->elem_kind == HP_ELEM_POINT && L.elem_point)
        L.elem_point(std::is_same<R, double>::value ? c->d_p1 : c->d_p1_32, tab, c->mesh, st, ph, stage, zero_rr, diff,
                     c->nsm, tune_of(c, R()), c->stream);
    else
        L.elem(tab, c->mesh, st, ph, stage, zero_rr, diff, c->nsm, tune_of(c, R()), c->stream);
}

// Stream-ordered body of rsdl(stage) (no sync, capturable), either precision.
template <typename R>
static void enqueue_rsdl_t(hp_gpu_ctx *c, const Launchers<R> &L, const void *tab, const State<R> &st, const Phys &ph,
                           int stage, int diff) {
    const int nstage = ph.nstage;
    const int zero_rr = (stage >= nstage) ? 1 : 0;
    const double omb = zero_rr ? 0.0 : 1.0 - ph.beta[stage];
    if (st.elim) {
        // assembly by gather: the element and boundary kernels write per-element and
        // per-edge values, k_assemble forms res and res_r of the vertices and sides
        launch_elem<R>(c, L, tab, st, ph, stage, zero_rr, diff);
        L.bflux(tab, c->mesh, st, ph, diff, c->stream);
        const long n = (long)c->npnt + (long)c->nseg * c->sm;
        const int with_b = (ph.physics == HP_PHYS_INS && c->nbseg > 0) ? 1 : 0;
        k_assemble<R><<<std::min(nblk(n, 256), c->nsm * 16), 256, 0, c->stream>>>(
            c->mesh, st, c->NV, c->sm, (R)omb, zero_rr, ph.beta[stage] > 0.0 ? 1 : 0, with_b);
        return;
    }
    const long n = (long)(c->lv + c->ls);
    k_rsdl_pre<R><<<std::min(nblk(n, 256), c->nsm * 8), 256, 0, c->stream>>>((int)c->lv, (int)c->ls, st.resv, st.ress,
                                                                           st.rrv, st.rrs, (R)omb, zero_rr);
    launch_elem<R>(c, L, tab, st, ph, stage, zero_rr, diff);
    L.bflux(tab, c->mesh, st, ph, diff, c->stream);
}
static void enqueue_rsdl(hp_gpu_ctx *c, int stage) { enqueue_rsdl_t<double>(c, c->L, c->d_tab, c->st, c->ph, stage, 0); }

// minvrt (+ update of ug with cflalpha when upd) ; maxres into slot when slot != NULL
template <typename R>
static void enqueue_minvrt_t(hp_gpu_ctx *c, const Launchers<R> &L, const State<R> &st, const DevMinv<R> *mt,
                             double cfla, int upd, int fold, unsigned long long *slot) {
    const int th = tune_of(c, R()).minv_threads;
    L.vert(c->mesh, st, mt, c->sm, c->im, cfla, upd, fold, slot, th, c->stream);
    for (int mode = 0; mode < c->sm; ++mode) L.side(c->mesh, st, mt, c->im, mode, cfla, upd, fold, th, c->stream);
    if (c->im > 0) L.intr(c->mesh, st, mt, cfla, upd, th, c->stream);
}
static void enqueue_minvrt(hp_gpu_ctx *c, double cfla, int upd, int fold, unsigned long long *slot) {
    enqueue_minvrt_t<double>(c, c->L, c->st, c->d_minv, cfla, upd, fold, slot);
}

template <typename R>
static void enqueue_update_t(hp_gpu_ctx *c, const Launchers<R> &L, const void *tab, const State<R> &st,
                             const DevMinv<R> *mt, const Phys &ph, int diff, unsigned long long *slot) {
    cudaMemcpyAsync(st.u0v, st.ugv, c->lv * sizeof(R), cudaMemcpyDeviceToDevice, c->stream);
    if (c->ls) cudaMemcpyAsync(st.u0s, st.ugs, c->ls * sizeof(R), cudaMemcpyDeviceToDevice, c->stream);
    if (c->li) cudaMemcpyAsync(st.u0i, st.ugi, c->li * sizeof(R), cudaMemcpyDeviceToDevice, c->stream);
    for (int stage = 0; stage < ph.nstage; ++stage) {
        enqueue_rsdl_t<R>(c, L, tab, st, ph, stage, diff);
        const double cfla = ph.alpha[stage] * ph.cfl;
        enqueue_minvrt_t<R>(c, L, st, mt, cfla, 1, 1, stage == ph.nstage - 1 ? slot : nullptr);
    }
}

static void enqueue_update(hp_gpu_ctx *c) {
    enqueue_update_t<double>(c, c->L, c->d_tab, c->st, c->d_minv, c->ph, 0, c->d_slot);
    k_hist_advance<<<1, 32, 0, c->stream>>>(c->d_slot, c->d_hist, c->d_iter, c->NV, c->hist_cap);
}

template <typename A, typename B>
static void conv(hp_gpu_ctx *c, long n, const A *src, B *dst) {
    if (n > 0) k_convert<A, B><<<std::min(nblk(n, 256), c->nsm * 8), 256, 0, c->stream>>>(n, src, dst);
}

static int check_launch(hp_gpu_ctx *c) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { set_err("kernel launch failed: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    return HP_OK;
}

static int mg_source_enqueue(hp_gpu_ctx *c);

// A coarse level's first residual evaluation after mg_restrict forms its driving term.
static int fas_first(hp_gpu_ctx *c) {
    if (!c->fas_pending) return HP_OK;
    if (!c->prcn_ready) {
        set_err("coarse level: setup_preconditioner before its first residual after mg_restrict");
        return HP_ESTATE;
    }
    return mg_source_enqueue(c);
}

extern "C" int hp_gpu_enqueue_rsdl(hp_gpu_ctx *c, int stage) {
    if (!c || stage < 0 || stage > c->ph.nstage) { set_err("bad stage"); return HP_EINVAL; }
    if (c->ph.physics == HP_PHYS_CD && c->ph.beta[stage] > 0.0 && !c->prcn_ready) {
        set_err("cd rsdl needs tau from setup_preconditioner");
        return HP_ESTATE;
    }
    int r = fas_first(c);
    if (r) return r;
    enqueue_rsdl(c, stage);
    // the reference's rsdl leaves res = res + res_r (nstage.cpp:76-82); the element kernel
    // already folded the interiors, fold vertices and sides here for the caller
    const long n = (long)(c->lv + c->ls);
    k_rsdl_fold<double><<<nblk(n, 256), 256, 0, c->stream>>>((int)c->lv, (int)c->ls, c->st.resv, c->st.rrv, c->st.ress,
                                                             c->st.rrs, c->st.dresv, c->st.dress);
    return check_launch(c);
}

extern "C" int hp_gpu_enqueue_element_rsdl(hp_gpu_ctx *c, int stage) {
    if (!c || stage < 0 || stage > c->ph.nstage) { set_err("bad stage"); return HP_EINVAL; }
    if (c->ph.physics == HP_PHYS_CD && c->ph.beta[stage] > 0.0 && !c->prcn_ready) {
        set_err("cd rsdl needs tau from setup_preconditioner");
        return HP_ESTATE;
    }
    launch_elem<double>(c, c->L, c->d_tab, c->st, c->ph, stage, stage >= c->ph.nstage, 0);
    return check_launch(c);
}

static int alloc_mixed(hp_gpu_ctx *c);
static void mixed_prcn(hp_gpu_ctx *c);

extern "C" int hp_gpu_rsdl(hp_gpu_ctx *c, int stage, int precision) {
    if (!c) return HP_EINVAL;
    if (precision == HP_PREC_FP64) {
        int r = hp_gpu_enqueue_rsdl(c, stage);
        if (r) return r;
        return hp_gpu_sync(c);
    }
    if (precision != HP_PREC_FP32) { set_err("precision must be HP_PREC_FP64 or HP_PREC_FP32"); return HP_EINVAL; }
    if (stage < 0 || stage > c->ph.nstage) { set_err("bad stage"); return HP_EINVAL; }
    if (c->ph.physics == HP_PHYS_CD && c->ph.beta[stage] > 0.0 && !c->prcn_ready) {
        set_err("cd rsdl needs tau from setup_preconditioner");
        return HP_ESTATE;
    }
    int r;
    if ((r = fas_first(c))) return r;
    if ((r = alloc_mixed(c))) return r;
    // the FP32 element kernels in plain form on fp32(u), with the level's FAS source; the
    // preconditioner arrays (cd tau) are FP32 copies of the FP64 ones
    if (c->prcn_ready) mixed_prcn(c);
    State<float> f = c->s32;
    f.ubv = f.ubs = f.ubi = nullptr;
    conv(c, (long)c->lv, c->st.ugv, f.ugv);
    conv(c, (long)c->ls, c->st.ugs, f.ugs);
    conv(c, (long)c->li, c->st.ugi, f.ugi);
    if (c->mg_kind) {
        conv(c, (long)c->lv, (const double *)c->fasv, (float *)f.dresv);
        conv(c, (long)c->ls, (const double *)c->fass, (float *)f.dress);
        if (c->li) conv(c, (long)c->li, (const double *)c->fasi, (float *)f.dresi);
    } else {
        f.dresv = f.dress = f.dresi = nullptr;
    }
    enqueue_rsdl_t<float>(c, c->L32, c->d_tab32, f, c->ph, stage, 0);
    const long n = (long)(c->lv + c->ls);
    k_rsdl_fold<float><<<nblk(n, 256), 256, 0, c->stream>>>((int)c->lv, (int)c->ls, f.resv, f.rrv, f.ress, f.rrs,
                                                            f.dresv, f.dress);
    conv(c, (long)c->lv, (const float *)f.resv, c->st.resv);
    conv(c, (long)c->ls, (const float *)f.ress, c->st.ress);
    conv(c, (long)c->li, (const float *)f.resi, c->st.resi);
    if ((r = check_launch(c))) return r;
    return hp_gpu_sync(c);
}

extern "C" int hp_gpu_l2error(hp_gpu_ctx *c, const hp_field *fld, double *l2, double *linf) {
    if (!c || !fld || !l2 || !linf) return HP_EINVAL;
    if (!c->L.l2err) { set_err("l2error not built"); return HP_ENOTSUP; }
    const int blocks = std::max(1, std::min(c->nsm * 4, nblk(c->ntri, 128)));
    int r;
    if (!c->d_l2part && (r = dalloc(c, (void **)&c->d_l2part, (size_t)c->nsm * 4 * 2 * 3 * 8))) return r;
    double *part = c->d_l2part;
    DevField f;
    f.kind = fld->kind;
    for (int k = 0; k < 4; ++k) f.prm[k] = fld->prm[k];
    c->L.l2err(c->d_tab, c->wtn, c->mesh, c->st, c->NV, f, part, blocks, c->stream);
    std::vector<double> h((size_t)blocks * 2 * c->NV);
    CK(cudaMemcpyAsync(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int n = 0; n < c->NV; ++n) {
        double a = 0.0, m = 0.0;
        for (int b = 0; b < blocks; ++b) {
            a += h[(size_t)b * 2 * c->NV + n];
            m = std::max(m, h[(size_t)b * 2 * c->NV + c->NV + n]);
        }
        l2[n] = std::sqrt(a);
        linf[n] = m;
    }
    return HP_OK;
}

extern "C" int hp_gpu_set_element_kernel(hp_gpu_ctx *c, int kind) {
    if (!c || (kind != HP_ELEM_SCALAR && kind != HP_ELEM_TENSOR && kind != HP_ELEM_POINT)) return HP_EINVAL;
    if (kind == HP_ELEM_TENSOR && !c->d_mma) {
        set_err("the tensor-core element kernel is built for ins only");
        return HP_ENOTSUP;
    }
    if (kind == HP_ELEM_POINT && !c->d_p1) {
        set_err("the point element kernel is built for ins at p = 1 only");
        return HP_ENOTSUP;
    }
    if (c->elem_kind != kind) {  // captured updates hold the old kernel
        if (c->g_update) { cudaGraphExecDestroy(c->g_update); c->g_update = nullptr; }
        if (c->g_update32) { cudaGraphExecDestroy(c->g_update32); c->g_update32 = nullptr; }
    }
    c->elem_kind = kind;
    return HP_OK;
}

static void drop_update_graphs(hp_gpu_ctx *c) {
    if (c->g_update) { cudaGraphExecDestroy(c->g_update); c->g_update = nullptr; }
    if (c->g_update32) { cudaGraphExecDestroy(c->g_update32); c->g_update32 = nullptr; }
}

// The cd element operators depend on the geometry, the fixed physics parameters and
// tau; cd tau is a function of the geometry and those parameters alone (steady
// problems), so one build stays valid for every later state.
static int build_element_matrices(hp_gpu_ctx *c) {
    const size_t n = c->L.emat_len(c->ntri), nb = (size_t)c->ntri * ((c->p + 1) * (c->p + 2) / 2);
    int r;
    if (!c->em.aim) {
        if ((r = dalloc(c, (void **)&c->em.aim, n * 8))) return r;
        if ((r = dalloc(c, (void **)&c->em.are, n * 8))) return r;
        if ((r = dalloc(c, (void **)&c->em.bre, nb * 8))) return r;
        if ((r = dalloc(c, (void **)&c->em32.aim, n * 4))) return r;
        if ((r = dalloc(c, (void **)&c->em32.are, n * 4))) return r;
        if ((r = dalloc(c, (void **)&c->em32.bre, nb * 4))) return r;
    }
    // operator tiles start on 16-byte boundaries
    for (const void *q : {(const void *)c->em.aim, (const void *)c->em.are, (const void *)c->em32.aim,
                          (const void *)c->em32.are})
        if ((uintptr_t)q % 16) {
            set_err("element operator storage not 16-byte aligned");
            return HP_ECUDA;
        }
    c->L.emat_build(c->d_tab, c->mesh, c->st, c->ph, c->em, c->nsm, c->stream);
    conv(c, (long)n, c->em.aim, c->em32.aim);
    conv(c, (long)n, c->em.are, c->em32.are);
    conv(c, (long)nb, c->em.bre, c->em32.bre);
    if ((r = check_launch(c))) return r;
    CK(cudaStreamSynchronize(c->stream));
    c->emat_built = true;
    drop_update_graphs(c);
    return HP_OK;
}

extern "C" int hp_gpu_set_element_matrices(hp_gpu_ctx *c, int on) {
    if (!c) return HP_EINVAL;
    if (on && c->ph.physics != HP_PHYS_CD) {
        set_err("element operators are built for the linear cd residual only");
        return HP_ENOTSUP;
    }
    if ((bool)on == c->emat_on) return HP_OK;
    c->emat_on = on != 0;
    drop_update_graphs(c);
    if (c->emat_on && !c->emat_built) {
        if (!c->prcn_ready) {  // tau
            int r = hp_gpu_setup_preconditioner(c);
            if (r) return r < 0 ? r : HP_ESTATE;
        }
        return build_element_matrices(c);
    }
    return HP_OK;
}

// Stream-ordered body of setup_preconditioner (capturable: no host synchronisation).
// Bad elements are counted into d_err, which the caller zeroes and reads.
static int enqueue_prcn(hp_gpu_ctx *c) {
    if (!c->st.elim) {
        CK(cudaMemsetAsync(c->st.vprcn, 0, (size_t)c->npnt * c->NV * 8, c->stream));
        CK(cudaMemsetAsync(c->st.sprcn, 0, (size_t)c->nseg * c->NV * 8, c->stream));
    }
    if (c->net) {
        int r0 = hp_gpu_elem_features(c, c->d_feat);
        if (r0) return r0;
        if (hp_mlp_forward(c->net, c->d_feat, c->ntri, c->d_netout, c->stream)) {
            set_err("network forward failed: %s", hp_mlp_last_error());
            return HP_ECUDA;
        }
        c->lsc = c->d_netout;
    }
    launch_prcn(c->p, c->ph.physics, c->d_tab, c->mesh, c->st, c->ph, c->d_err, c->lsc, c->lsc_ld, c->lsc_clamp,
                c->stream);
    if (c->st.elim) {  // assembly by gather, inversion fused
        const long n = (long)c->npnt + (c->p > 1 ? (long)c->nseg : 0);
        k_prcn_gather<double><<<std::min(nblk(n, 256), c->nsm * 16), 256, 0, c->stream>>>(c->mesh, c->st, c->NV,
                                                                                        c->p > 1 ? 1 : 0, c->vdiag);
        return check_launch(c);
    }
    const int nv = c->npnt * c->NV, ns = (c->p > 1 ? c->nseg * c->NV : 0);
    k_prcn_invert<double><<<nblk(nv + ns, 256), 256, 0, c->stream>>>(nv, ns, c->st.vprcn, c->st.sprcn, c->vdiag);
    return check_launch(c);
}

extern "C" int hp_gpu_setup_preconditioner(hp_gpu_ctx *c) {
    if (!c) return HP_EINVAL;
    CK(cudaMemsetAsync(c->d_err, 0, 4, c->stream));
    int r = enqueue_prcn(c);
    if (r) return r;
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->prcn_ready = true;
    return herr;
}

extern "C" int hp_gpu_minvrt(hp_gpu_ctx *c) {
    if (!c) return HP_EINVAL;
    if (!c->prcn_ready) { set_err("minvrt before setup_preconditioner"); return HP_ESTATE; }
    enqueue_minvrt(c, 0.0, 0, 0, nullptr);
    int r = check_launch(c);
    if (r) return r;
    return hp_gpu_sync(c);
}

static int ensure_update_graph(hp_gpu_ctx *c) {
    if (c->g_update) return HP_OK;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_update(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) { set_err("graph capture failed: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    e = cudaGraphInstantiate(&c->g_update, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { set_err("graph instantiate failed: %s", cudaGetErrorString(e)); c->g_update = nullptr; return HP_ECUDA; }
    return HP_OK;
}

extern "C" int hp_gpu_enqueue_update(hp_gpu_ctx *c) {
    if (!c) return HP_EINVAL;
    if (!c->prcn_ready) { set_err("update before setup_preconditioner"); return HP_ESTATE; }
    int r = fas_first(c);
    if (r) return r;
    if ((r = ensure_update_graph(c))) return r;
    CK(cudaGraphLaunch(c->g_update, c->stream));
    return HP_OK;
}

extern "C" int hp_gpu_update(hp_gpu_ctx *c) {
    int r = hp_gpu_enqueue_update(c);
    if (r) return r;
    return hp_gpu_sync(c);
}

extern "C" int hp_gpu_iterate(hp_gpu_ctx *c, int iters, int prcn_interval, double *hist) {
    if (!c || iters < 0) return HP_EINVAL;
    if (iters > c->hist_cap) { set_err("iters > %d", c->hist_cap); return HP_EINVAL; }
    int r = ensure_update_graph(c);
    if (r) return r;
    CK(cudaMemsetAsync(c->d_iter, 0, 4, c->stream));
    for (int it = 0; it < iters; ++it) {
        if (!c->prcn_ready || (prcn_interval > 0 && it % prcn_interval == 0 && it > 0)) {
            r = hp_gpu_setup_preconditioner(c);
            if (r) return r;
            if ((r = ensure_update_graph(c))) return r;  // a first set-up may switch the element path
        }
        if ((r = fas_first(c))) return r;
        CK(cudaGraphLaunch(c->g_update, c->stream));
    }
    if (hist && iters) CK(cudaMemcpyAsync(hist, c->d_hist, (size_t)iters * 8, cudaMemcpyDeviceToHost, c->stream));
    return hp_gpu_sync(c);
}

extern "C" int hp_gpu_maxres(hp_gpu_ctx *c, double *out, double *mx) {
    if (!c) return HP_EINVAL;
    CK(cudaMemsetAsync(c->d_slot, 0, 32, c->stream));
    // per-variable max over vertices of |res.v|
    const int np = c->npnt, NV = c->NV;
    std::vector<double> hv((size_t)np * NV);
    CK(cudaMemcpyAsync(hv.data(), c->st.resv, hv.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double m[3] = {0, 0, 0}, e = 0.0;
    for (int i = 0; i < np; ++i)
        for (int n = 0; n < NV; ++n) m[n] = std::max(m[n], std::fabs(hv[(size_t)i * NV + n]));
    for (int n = 0; n < NV; ++n) { if (out) out[n] = m[n]; e = std::max(e, m[n]); }
    if (mx) *mx = e;
    return HP_OK;
}

static int device_norm(hp_gpu_ctx *c, const double *a, size_t n, double &ss, double &mx) {
    if (n == 0) return HP_OK;
    int blocks = std::min(c->npart, nblk((long)n, 256));
    k_norm_partial<double><<<blocks, 256, 0, c->stream>>>(a, n, c->d_part);
    std::vector<double> h(2 * blocks);
    CK(cudaMemcpyAsync(h.data(), c->d_part, h.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int b = 0; b < blocks; ++b) { ss += h[2 * b]; mx = std::max(mx, h[2 * b + 1]); }
    return HP_OK;
}

extern "C" int hp_gpu_resnorm(hp_gpu_ctx *c, double *l2, double *linf) {
    if (!c) return HP_EINVAL;
    int r = hp_gpu_rsdl(c, c->ph.nstage, HP_PREC_FP64);
    if (r) return r;
    double ss = 0.0, mx = 0.0;
    if ((r = device_norm(c, c->st.resv, c->lv, ss, mx))) return r;
    if ((r = device_norm(c, c->st.ress, c->ls, ss, mx))) return r;
    if ((r = device_norm(c, c->st.resi, c->li, ss, mx))) return r;
    if (l2) *l2 = std::sqrt(ss);
    if (linf) *linf = mx;
    return HP_OK;
}

extern "C" int hp_gpu_sync(hp_gpu_ctx *c) {
    if (!c) return HP_EINVAL;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { set_err("stream sync: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    e = cudaGetLastError();
    if (e != cudaSuccess) { set_err("cuda error: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    return HP_OK;
}

// ---------------------------------------------------------------------------
// Convergence drivers: plain FP64 smoothing and FP32 correction smoothing with
// FP64 defect correction.
// ---------------------------------------------------------------------------
static int alloc_mixed(hp_gpu_ctx *c) {
    if (c->mixed_ready) return HP_OK;
    State<float> &f = c->s32;
    int r;
    float **v[] = {&f.ugv, &f.u0v, &f.resv, &f.rrv};
    float **sp[] = {&f.ugs, &f.u0s, &f.ress, &f.rrs};
    float **ip[] = {&f.ugi, &f.u0i, &f.resi, &f.rri};
    for (auto q : v) if ((r = dalloc(c, (void **)q, c->lv * 4))) return r;
    for (auto q : sp) if ((r = dalloc(c, (void **)q, std::max<size_t>(c->ls, 1) * 4))) return r;
    for (auto q : ip) if ((r = dalloc(c, (void **)q, std::max<size_t>(c->li, 1) * 4))) return r;
    float *ubv, *ubs, *ubi, *dv, *ds, *di;
    if ((r = dalloc(c, (void **)&ubv, c->lv * 4))) return r;
    if ((r = dalloc(c, (void **)&ubs, std::max<size_t>(c->ls, 1) * 4))) return r;
    if ((r = dalloc(c, (void **)&ubi, std::max<size_t>(c->li, 1) * 4))) return r;
    if ((r = dalloc(c, (void **)&dv, c->lv * 4))) return r;
    if ((r = dalloc(c, (void **)&ds, std::max<size_t>(c->ls, 1) * 4))) return r;
    if ((r = dalloc(c, (void **)&di, std::max<size_t>(c->li, 1) * 4))) return r;
    f.ubv = ubv; f.ubs = ubs; f.ubi = ubi;
    f.dresv = dv; f.dress = ds; f.dresi = c->li ? di : nullptr;
    if ((r = dalloc(c, (void **)&f.vprcn, (size_t)c->npnt * c->NV * 4))) return r;
    if ((r = dalloc(c, (void **)&f.sprcn, (size_t)c->nseg * c->NV * 4))) return r;
    if ((r = dalloc(c, (void **)&f.tprcn, (size_t)c->ntri * c->NV * 4))) return r;
    if ((r = dalloc(c, (void **)&f.tau, (size_t)c->ntri * c->NV * 4))) return r;
    // the base state's point values of the TF32 correction-form kernel (refreshed with the
    // base by base_points); the pointer is fixed here so that captured updates see it
    if (c->L32.base_pts && c->d_mma32) {
        if ((r = dalloc(c, (void **)&c->d_bpt32, (size_t)c->ntri * c->L32.bpt_per_elem * 4))) return r;
        f.bpt = c->d_bpt32;
    }
    // res_r is scaled by (1 - beta) before it is first written: it must start finite
    CK(cudaMemsetAsync(f.rrv, 0, c->lv * 4, c->stream));
    if (c->ls) CK(cudaMemsetAsync(f.rrs, 0, c->ls * 4, c->stream));
    if (c->li) CK(cudaMemsetAsync(f.rri, 0, c->li * 4, c->stream));
    CK(cudaMemsetAsync(f.resv, 0, c->lv * 4, c->stream));
    if (c->ls) CK(cudaMemsetAsync(f.ress, 0, c->ls * 4, c->stream));
    if (c->li) CK(cudaMemsetAsync(f.resi, 0, c->li * 4, c->stream));
    c->mixed_ready = true;
    return HP_OK;
}

// FP32 copies of the FP64 preconditioner (computed at the base state)
static void mixed_prcn(hp_gpu_ctx *c) {
    State<float> &f = c->s32;
    conv(c, (long)c->npnt * c->NV, c->st.vprcn, f.vprcn);
    conv(c, (long)c->nseg * c->NV, c->st.sprcn, f.sprcn);
    conv(c, (long)c->ntri * c->NV, c->st.tprcn, f.tprcn);
    conv(c, (long)c->ntri * c->NV, c->st.tau, f.tau);
}

// Point values of the FP32 base state (State::bpt) after it changed.
static void base_points(hp_gpu_ctx *c) {
    if (c->s32.bpt) c->L32.base_pts(c->d_tab32, c->mesh, c->s32, c->d_bpt32, c->stream);
}

// Start of one correction cycle: base = fp32(u64), dres = fp32(R64(u64)) (the FP64
// residual left in res by rsdl(nstage)), correction d = 0, res_r = 0.
static void mixed_prepare(hp_gpu_ctx *c) {
    State<float> &f = c->s32;
    conv(c, (long)c->lv, c->st.ugv, (float *)f.ubv);
    conv(c, (long)c->ls, c->st.ugs, (float *)f.ubs);
    conv(c, (long)c->li, c->st.ugi, (float *)f.ubi);
    base_points(c);
    conv(c, (long)c->lv, c->st.resv, (float *)f.dresv);
    conv(c, (long)c->ls, c->st.ress, (float *)f.dress);
    if (c->li) conv(c, (long)c->li, c->st.resi, (float *)f.dresi);
    cudaMemsetAsync(f.ugv, 0, c->lv * 4, c->stream);
    if (c->ls) cudaMemsetAsync(f.ugs, 0, c->ls * 4, c->stream);
    if (c->li) cudaMemsetAsync(f.ugi, 0, c->li * 4, c->stream);
}

static void mixed_apply(hp_gpu_ctx *c) {
    const State<float> &f = c->s32;
    auto add = [&](long n, const float *src, double *dst) {
        if (n > 0) k_add_into<float, double><<<std::min(nblk(n, 256), c->nsm * 8), 256, 0, c->stream>>>(n, src, dst);
    };
    add((long)c->lv, f.ugv, c->st.ugv);
    add((long)c->ls, f.ugs, c->st.ugs);
    add((long)c->li, f.ugi, c->st.ugi);
}

static int ensure_update32_graph(hp_gpu_ctx *c) {
    if (c->g_update32) return HP_OK;
    Phys ph = c->ph;
    if (ph.physics == HP_PHYS_CD) ph.src = 0.0;  // the cd residual is affine: R(b+d) - R(b) = R_0(d)
    const int diff = (ph.physics == HP_PHYS_INS) ? 1 : 0;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_update_t<float>(c, c->L32, c->d_tab32, c->s32, c->d_minv32, ph, diff, nullptr);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) { set_err("graph capture failed: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    e = cudaGraphInstantiate(&c->g_update32, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { set_err("graph instantiate failed: %s", cudaGetErrorString(e)); c->g_update32 = nullptr; return HP_ECUDA; }
    return HP_OK;
}

static int fp64_norm(hp_gpu_ctx *c, double *l2) {
    int r = hp_gpu_enqueue_rsdl(c, c->ph.nstage);
    if (r) return r;
    k_mask_essential<double><<<nblk(c->npnt + c->nseg, 256), 256, 0, c->stream>>>(c->mesh, c->st.resv, c->st.ress,
                                                                                 c->NV, c->sm);
    double ss = 0.0, mx = 0.0;
    if ((r = device_norm(c, c->st.resv, c->lv, ss, mx))) return r;
    if ((r = device_norm(c, c->st.ress, c->ls, ss, mx))) return r;
    if ((r = device_norm(c, c->st.resi, c->li, ss, mx))) return r;
    *l2 = std::sqrt(ss);
    return HP_OK;
}

extern "C" int hp_gpu_solve(hp_gpu_ctx *c, int mode, double drop, int max_updates, int inner, int check_every,
                            int prcn_every, double *hist, int hist_cap, int *n_hist, double *seconds, int *updates) {
    if (!c || (mode != HP_PREC_FP64 && mode != HP_PREC_FP32) || drop <= 0.0 || max_updates < 1) {
        set_err("hp_gpu_solve: bad argument");
        return HP_EINVAL;
    }
    if (check_every < 1) check_every = 10;
    if (inner < 1) inner = 10;
    int r;
    if ((r = ensure_update_graph(c))) return r;
    if (mode == HP_PREC_FP32) {
        if ((r = alloc_mixed(c))) return r;
        if ((r = ensure_update32_graph(c))) return r;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c->stream));
    int nh = 0, nupd = 0, nchk = 0;
    double r0 = 0.0, rn = 0.0;
    r = hp_gpu_setup_preconditioner(c);
    if (r) return r < 0 ? r : HP_ESTATE;
    // the first set-up may have built element operators and dropped the update graphs
    if ((r = ensure_update_graph(c))) return r;
    if (mode == HP_PREC_FP32 && (r = ensure_update32_graph(c))) return r;
    if ((r = fp64_norm(c, &r0))) return r;
    if (hist && nh < hist_cap) hist[nh++] = 1.0;
    if (mode == HP_PREC_FP32) mixed_prcn(c);
    while (nupd < max_updates) {
        if (mode == HP_PREC_FP64) {
            for (int k = 0; k < check_every && nupd < max_updates; ++k, ++nupd) CK(cudaGraphLaunch(c->g_update, c->stream));
        } else {
            // the FP64 residual R64(u) is in res from the last norm evaluation
            mixed_prepare(c);
            for (int k = 0; k < inner && nupd < max_updates; ++k, ++nupd) CK(cudaGraphLaunch(c->g_update32, c->stream));
            mixed_apply(c);
        }
        ++nchk;
        if (prcn_every > 0 && nchk % prcn_every == 0) {
            r = hp_gpu_setup_preconditioner(c);
            if (r) return r < 0 ? r : HP_ESTATE;
            if (mode == HP_PREC_FP32) mixed_prcn(c);
        }
        if ((r = fp64_norm(c, &rn))) return r;
        const double d = rn / r0;
        if (hist && nh < hist_cap) hist[nh++] = d;
        if (!(d == d)) break;  // NaN
        if (d <= drop) break;
    }
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_hist) *n_hist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (updates) *updates = nupd;
    return hp_gpu_sync(c);
}

// Diagnostic: `n` multistage updates of the FP32 smoother in plain form (the FP32
// state is fp32(u), no source, no correction), written back to the FP64 state.
// Lets tests compare the FP32 kernels with the FP64 ones update by update.
extern "C" int hp_gpu_fp32_updates(hp_gpu_ctx *c, int n) {
    if (!c || n < 0) return HP_EINVAL;
    int r;
    if ((r = alloc_mixed(c))) return r;
    if (!c->prcn_ready) { set_err("fp32 updates before setup_preconditioner"); return HP_ESTATE; }
    mixed_prcn(c);
    State<float> f = c->s32;
    f.ubv = f.ubs = f.ubi = nullptr;
    f.dresv = f.dress = f.dresi = nullptr;
    conv(c, (long)c->lv, c->st.ugv, f.ugv);
    conv(c, (long)c->ls, c->st.ugs, f.ugs);
    conv(c, (long)c->li, c->st.ugi, f.ugi);
    for (int k = 0; k < n; ++k) enqueue_update_t<float>(c, c->L32, c->d_tab32, f, c->d_minv32, c->ph, 0, nullptr);
    conv(c, (long)c->lv, (const float *)f.ugv, c->st.ugv);
    conv(c, (long)c->ls, (const float *)f.ugs, c->st.ugs);
    conv(c, (long)c->li, (const float *)f.ugi, c->st.ugi);
    if ((r = check_launch(c))) return r;
    return hp_gpu_sync(c);
}

// ---------------------------------------------------------------------------
// Learned preconditioner hooks (include/hp_mlp.h)
// ---------------------------------------------------------------------------
extern "C" int hp_gpu_elem_features(hp_gpu_ctx *c, float *d_feat) {
    if (!c || !d_feat) return HP_EINVAL;
    k_elem_features<<<nblk(c->ntri, 128), 128, 0, c->stream>>>(c->mesh, c->st, c->ph, c->NV, c->sm, c->im, c->p, d_feat);
    return check_launch(c);
}

extern "C" int hp_gpu_elem_resnorm(hp_gpu_ctx *c, double *d_out) {
    if (!c || !d_out) return HP_EINVAL;
    k_elem_resnorm<<<nblk(c->ntri, 128), 128, 0, c->stream>>>(c->mesh, c->st, c->NV, c->sm, c->im, d_out);
    return check_launch(c);
}

extern "C" int hp_gpu_set_prcn_scale(hp_gpu_ctx *c, const float *d_logscale, int ld, float clampv) {
    if (!c || (d_logscale && ld < 1)) return HP_EINVAL;
    c->lsc = d_logscale;
    c->lsc_ld = ld < 1 ? 1 : ld;
    c->lsc_clamp = clampv;
    c->net = nullptr;
    return HP_OK;
}

extern "C" int hp_gpu_set_prcn_net(hp_gpu_ctx *c, hp_mlp *net, float clampv) {
    if (!c) return HP_EINVAL;
    if (!net) {
        c->net = nullptr;
        c->lsc = nullptr;
        return HP_OK;
    }
    int nin = 0, nout = 0;
    if (hp_mlp_dims(net, &nin, &nout) || nin != HP_NFEAT) { set_err("network must take %d inputs", HP_NFEAT); return HP_EINVAL; }
    int r;
    if (!c->d_feat && (r = dalloc(c, (void **)&c->d_feat, (size_t)c->ntri * HP_NFEAT * 4))) return r;
    if (!c->d_netout && (r = dalloc(c, (void **)&c->d_netout, (size_t)c->ntri * 64 * 4))) return r;
    c->net = net;
    c->lsc_ld = nout;
    c->lsc_clamp = clampv;
    return HP_OK;
}

// ---------------------------------------------------------------------------
// Multigrid (tri_hp::mg_restrict / mg_prolongate / mg_source and block::cycle)
// ---------------------------------------------------------------------------
static int mg_alloc(hp_gpu_ctx *c) {
    int r;
    const size_t lv = std::max<size_t>(c->lv, 1), ls = std::max<size_t>(c->ls, 1), li = std::max<size_t>(c->li, 1);
    double **v[] = {&c->res0v, &c->uc0v, &c->fasv};
    double **s[] = {&c->res0s, &c->uc0s, &c->fass};
    double **i[] = {&c->res0i, &c->uc0i, &c->fasi};
    for (auto q : v) if (!*q && (r = dalloc(c, (void **)q, lv * 8))) return r;
    for (auto q : s) if (!*q && (r = dalloc(c, (void **)q, ls * 8))) return r;
    for (auto q : i) if (!*q && (r = dalloc(c, (void **)q, li * 8))) return r;
    CK(cudaMemsetAsync(c->fasv, 0, lv * 8, c->stream));
    CK(cudaMemsetAsync(c->fass, 0, ls * 8, c->stream));
    CK(cudaMemsetAsync(c->fasi, 0, li * 8, c->stream));
    // the source enters every stage residual of this level (captured into its update graph)
    c->st.dresv = c->fasv;
    c->st.dress = c->ls ? c->fass : nullptr;
    c->st.dresi = c->li ? c->fasi : nullptr;
    if (c->g_update) {
        cudaGraphExecDestroy(c->g_update);
        c->g_update = nullptr;
    }
    return HP_OK;
}

extern "C" int hp_gpu_mg_attach_p(hp_gpu_ctx *coarse, hp_gpu_ctx *fine, double fadd) {
    if (!coarse || !fine || coarse == fine) return HP_EINVAL;
    if (coarse->npnt != fine->npnt || coarse->nseg != fine->nseg || coarse->ntri != fine->ntri ||
        coarse->NV != fine->NV || coarse->p >= fine->p) {
        set_err("p-level must share the mesh and physics of its fine level and have a lower p");
        return HP_EINVAL;
    }
    coarse->fine = fine;
    coarse->mg_kind = 1;
    coarse->fadd = fadd;
    return mg_alloc(coarse);
}

extern "C" int hp_gpu_mg_attach_h(hp_gpu_ctx *coarse, hp_gpu_ctx *fine, const int *f2c_tri, const double *f2c_wt,
                                  const int *c2f_tri, const double *c2f_wt, double fadd) {
    if (!coarse || !fine || !f2c_tri || !f2c_wt || !c2f_tri || !c2f_wt) return HP_EINVAL;
    if (coarse->p != 1 || coarse->NV != fine->NV) {
        set_err("h-level must be p = 1 with the physics of its fine level");
        return HP_EINVAL;
    }
    for (int i = 0; i < fine->npnt; ++i)
        if (f2c_tri[i] < 0 || f2c_tri[i] >= coarse->ntri) { set_err("f2c_tri out of range"); return HP_EINVAL; }
    for (int i = 0; i < coarse->npnt; ++i)
        if (c2f_tri[i] < 0 || c2f_tri[i] >= fine->ntri) { set_err("c2f_tri out of range"); return HP_EINVAL; }
    int r;
    if ((r = upload(coarse, &coarse->f2c_tri, f2c_tri, (size_t)fine->npnt))) return r;
    if ((r = upload(coarse, &coarse->f2c_wt, f2c_wt, (size_t)fine->npnt * 3))) return r;
    if ((r = upload(coarse, &coarse->c2f_tri, c2f_tri, (size_t)coarse->npnt))) return r;
    if ((r = upload(coarse, &coarse->c2f_wt, c2f_wt, (size_t)coarse->npnt * 3))) return r;
    coarse->fine = fine;
    coarse->mg_kind = 2;
    coarse->fadd = fadd;
    return mg_alloc(coarse);
}

// Transfers the fine level's current full residual (rsdl(nstage), folded) and
// state to this coarse level and sets its FAS source.
static int mg_restrict_enqueue(hp_gpu_ctx *c) {
    hp_gpu_ctx *f = c->fine;
    if (!f || !c->mg_kind) { set_err("not a coarse level"); return HP_ESTATE; }
    if (c->stream != f->stream) {  // order the coarse stream after the fine one
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, f->stream));
        CK(cudaStreamWaitEvent(c->stream, ev, 0));
        cudaEventDestroy(ev);
    }
    const int NV = c->NV;
    if (c->mg_kind == 1) {
        const long tot = (long)(c->lv + c->ls + c->li);
        const int g = std::min(nblk(tot, 256), c->nsm * 8);
        k_mg_truncate<double><<<g, 256, 0, c->stream>>>(c->npnt, c->nseg, c->ntri, NV, f->sm, f->im, c->sm, c->im, f->st.resv,
                                                f->st.ress, f->st.resi, c->res0v, c->res0s, c->res0i);
        k_mg_truncate<double><<<g, 256, 0, c->stream>>>(c->npnt, c->nseg, c->ntri, NV, f->sm, f->im, c->sm, c->im, f->st.ugv,
                                                f->st.ugs, f->st.ugi, c->st.ugv, c->st.ugs, c->st.ugi);
        CK(cudaMemcpyAsync(c->uc0v, c->st.ugv, c->lv * 8, cudaMemcpyDeviceToDevice, c->stream));
        if (c->ls) CK(cudaMemcpyAsync(c->uc0s, c->st.ugs, c->ls * 8, cudaMemcpyDeviceToDevice, c->stream));
        if (c->li) CK(cudaMemcpyAsync(c->uc0i, c->st.ugi, c->li * 8, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        CK(cudaMemsetAsync(c->res0v, 0, c->lv * 8, c->stream));
        k_mg_restrict_hres<double><<<nblk(f->npnt, 128), 128, 0, c->stream>>>(f->npnt, NV, c->f2c_tri, c->f2c_wt,
                                                                        c->mesh.tri_pnt, f->st.resv, c->res0v);
        k_mg_restrict_hstate<double><<<nblk(c->npnt, 128), 128, 0, c->stream>>>(c->npnt, NV, c->c2f_tri, c->c2f_wt,
                                                                          f->mesh.tri_pnt, f->st.ugv, c->st.ugv,
                                                                          c->uc0v);
    }
    // the driving term is formed at the coarse level's first residual evaluation (isfrst)
    c->fas_pending = true;
    return check_launch(c);
}

// tri_hp::mg_source on first entry (nstage.cpp:113-129): res(first) of the coarse level
// at the restricted state without its source, then dres = fadd*res0 - res(first). Runs
// where the reference's first coarse rsdl runs: after that level's own preconditioner
// set-up, so that res(first) uses its tau.
static int mg_source_enqueue(hp_gpu_ctx *c) {
    c->fas_pending = false;
    State<double> plain = c->st;
    plain.dresv = plain.dress = plain.dresi = nullptr;
    enqueue_rsdl_t<double>(c, c->L, c->d_tab, plain, c->ph, c->ph.nstage, 0);
    const long n2 = (long)(c->lv + c->ls);
    k_rsdl_fold<double><<<nblk(n2, 256), 256, 0, c->stream>>>((int)c->lv, (int)c->ls, c->st.resv, c->st.rrv,
                                                              c->st.ress, c->st.rrs, nullptr, nullptr);
    const int g2 = c->nsm * 8;
    k_fas_source<double><<<g2, 256, 0, c->stream>>>((long)c->lv, c->fadd, c->res0v, c->st.resv, c->fasv);
    if (c->ls) k_fas_source<double><<<g2, 256, 0, c->stream>>>((long)c->ls, c->fadd, c->res0s, c->st.ress, c->fass);
    if (c->li) k_fas_source<double><<<g2, 256, 0, c->stream>>>((long)c->li, c->fadd, c->res0i, c->st.resi, c->fasi);
    return check_launch(c);
}

static int mg_prolong_enqueue(hp_gpu_ctx *c) {
    hp_gpu_ctx *f = c->fine;
    if (!f || !c->mg_kind) { set_err("not a coarse level"); return HP_ESTATE; }
    const int NV = c->NV;
    if (c->mg_kind == 1) {
        const long tot = (long)(c->lv + c->ls + c->li);
        k_mg_prolong_p<double><<<std::min(nblk(tot, 256), c->nsm * 8), 256, 0, c->stream>>>(
            c->npnt, c->nseg, c->ntri, NV, f->sm, f->im, c->sm, c->im, c->st.ugv, c->st.ugs, c->st.ugi, c->uc0v,
            c->uc0s, c->uc0i, f->st.ugv, f->st.ugs, f->st.ugi);
    } else {
        k_mg_prolong_h<double><<<nblk(f->npnt, 128), 128, 0, c->stream>>>(f->npnt, NV, c->f2c_tri, c->f2c_wt, c->mesh.tri_pnt,
                                                                    c->st.ugv, c->uc0v, f->st.ugv);
    }
    if (c->stream != f->stream) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, c->stream));
        CK(cudaStreamWaitEvent(f->stream, ev, 0));
        cudaEventDestroy(ev);
    }
    return check_launch(c);
}

extern "C" int hp_gpu_mg_restrict(hp_gpu_ctx *coarse) {
    int r = mg_restrict_enqueue(coarse);
    if (r) return r;
    return hp_gpu_sync(coarse);
}

extern "C" int hp_gpu_mg_prolongate(hp_gpu_ctx *coarse) {
    int r = mg_prolong_enqueue(coarse);
    if (r) return r;
    return hp_gpu_sync(coarse->fine);
}

// block::cycle (tri_mesh/blocks.cpp:1267-1348) over levels[0] (finest) .. levels[n-1]
static int cycle(hp_gpu_ctx **lv, int n, int lvl, int vw, int itercrsn, int iterrfne, int eval_prcn) {
    hp_gpu_ctx *c = lv[lvl];
    int r;
    for (int vc = 0; vc < vw; ++vc) {
        if (eval_prcn) {
            r = hp_gpu_setup_preconditioner(c);
            if (r) return r < 0 ? r : HP_ESTATE;
        }
        if ((r = fas_first(c))) return r;
        if ((r = ensure_update_graph(c))) return r;
        for (int it = 0; it < itercrsn; ++it) CK(cudaGraphLaunch(c->g_update, c->stream));
        if (lvl == n - 1) return HP_OK;
        if ((r = hp_gpu_enqueue_rsdl(c, c->ph.nstage))) return r;
        if ((r = mg_restrict_enqueue(lv[lvl + 1]))) return r;
        if ((r = cycle(lv, n, lvl + 1, vw, itercrsn, iterrfne, eval_prcn))) return r;
        if ((r = mg_prolong_enqueue(lv[lvl + 1]))) return r;
        if (eval_prcn && iterrfne) {
            r = hp_gpu_setup_preconditioner(c);
            if (r) return r < 0 ? r : HP_ESTATE;
        }
        for (int it = 0; it < iterrfne; ++it) CK(cudaGraphLaunch(c->g_update, c->stream));
    }
    return HP_OK;
}

extern "C" int hp_gpu_vcycle(hp_gpu_ctx **levels, int nlevels, int vw, int itercrsn, int iterrfne, int eval_prcn) {
    if (!levels || nlevels < 1 || vw < 1 || itercrsn < 0 || iterrfne < 0) return HP_EINVAL;
    for (int l = 1; l < nlevels; ++l)
        if (!levels[l] || levels[l]->fine != levels[l - 1]) { set_err("level %d is not attached to level %d", l, l - 1); return HP_EINVAL; }
    int r = cycle(levels, nlevels, 0, vw, itercrsn, iterrfne, eval_prcn);
    if (r) return r;
    return hp_gpu_sync(levels[0]);
}

extern "C" int hp_gpu_solve_mg(hp_gpu_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                               int iterrfne, int prcn_every, double *hist, int hist_cap, int *n_hist,
                               double *seconds, int *cycles) {
    if (!levels || nlevels < 1 || drop <= 0.0 || max_cycles < 1) return HP_EINVAL;
    hp_gpu_ctx *f = levels[0];
    int nh = 0, nc = 0, r;
    for (int l = 0; l < nlevels; ++l)  // graph instantiation is set-up, outside the solve time
        if ((r = ensure_update_graph(levels[l]))) return r;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, f->stream));
    double r0 = 0.0, rn = 0.0;
    r = hp_gpu_setup_preconditioner(f);
    if (r) return r < 0 ? r : HP_ESTATE;
    if ((r = fp64_norm(f, &r0))) return r;
    if (hist && nh < hist_cap) hist[nh++] = 1.0;
    while (nc < max_cycles) {
        // every level's preconditioner is evaluated at its state on the first cycle
        // and then every prcn_every cycles (block::cycle's evaluate_preconditioner)
        const int eval = (nc == 0 || (prcn_every > 0 && nc % prcn_every == 0)) ? 1 : 0;
        if ((r = cycle(levels, nlevels, 0, vw, itercrsn, iterrfne, eval))) return r;
        ++nc;
        if ((r = fp64_norm(f, &rn))) return r;
        const double d = rn / r0;
        if (hist && nh < hist_cap) hist[nh++] = d;
        if (!(d == d) || d <= drop) break;
    }
    CK(cudaEventRecord(e1, f->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_hist) *n_hist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (cycles) *cycles = nc;
    return hp_gpu_sync(f);
}

// One V/W-cycle captured as a single CUDA graph (all levels must share one
// stream). The preconditioners are evaluated before capture and frozen inside it;
// the level updates are enqueued as plain kernels so the whole cycle is one graph.
// block::cycle as stream operations only (for capture). With eval_prcn the
// preconditioners are set up at the same points as in cycle(); bad elements then
// accumulate in each level's d_err, which the driver checks between replays.
static int cycle_enqueue(hp_gpu_ctx **lv, int n, int lvl, int vw, int itercrsn, int iterrfne, int eval_prcn) {
    hp_gpu_ctx *c = lv[lvl];
    int r;
    for (int vc = 0; vc < vw; ++vc) {
        if (eval_prcn && (r = enqueue_prcn(c))) return r;
        if (c->fas_pending && (r = mg_source_enqueue(c))) return r;
        for (int it = 0; it < itercrsn; ++it) enqueue_update(c);
        if (lvl == n - 1) return HP_OK;
        if ((r = hp_gpu_enqueue_rsdl(c, c->ph.nstage))) return r;
        if ((r = mg_restrict_enqueue(lv[lvl + 1]))) return r;
        if ((r = cycle_enqueue(lv, n, lvl + 1, vw, itercrsn, iterrfne, eval_prcn))) return r;
        if ((r = mg_prolong_enqueue(lv[lvl + 1]))) return r;
        if (eval_prcn && iterrfne && (r = enqueue_prcn(c))) return r;
        for (int it = 0; it < iterrfne; ++it) enqueue_update(c);
    }
    return HP_OK;
}

struct VGraph {
    cudaGraphExec_t exec = nullptr;
};

extern "C" int hp_gpu_capture_vcycle(hp_gpu_ctx **levels, int nlevels, int vw, int itercrsn, int iterrfne,
                                     int eval_prcn, void **graph_out) {
    if (!levels || nlevels < 1 || !graph_out) return HP_EINVAL;
    for (int l = 0; l < nlevels; ++l) {
        if (levels[l]->stream != levels[0]->stream) { set_err("all levels must share one stream"); return HP_EINVAL; }
        if (l > 0 && levels[l]->fine != levels[l - 1]) { set_err("levels not attached in order"); return HP_EINVAL; }
        if (!levels[l]->prcn_ready) { set_err("setup_preconditioner every level before capture"); return HP_ESTATE; }
    }
    cudaStream_t s = levels[0]->stream;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int r = cycle_enqueue(levels, nlevels, 0, vw, itercrsn, iterrfne, eval_prcn);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (r) return r;
    if (e != cudaSuccess) { set_err("V-cycle capture failed: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    VGraph *vg = new VGraph();
    e = cudaGraphInstantiate(&vg->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { delete vg; set_err("V-cycle instantiate failed: %s", cudaGetErrorString(e)); return HP_ECUDA; }
    *graph_out = vg;
    return HP_OK;
}

extern "C" int hp_gpu_launch_vcycle(void *graph, hp_gpu_ctx *finest, int count) {
    if (!graph || !finest || count < 0) return HP_EINVAL;
    VGraph *vg = static_cast<VGraph *>(graph);
    for (int k = 0; k < count; ++k) CK(cudaGraphLaunch(vg->exec, finest->stream));
    return HP_OK;
}

extern "C" int hp_gpu_destroy_vcycle(void *graph) {
    if (!graph) return HP_OK;
    VGraph *vg = static_cast<VGraph *>(graph);
    if (vg->exec) cudaGraphExecDestroy(vg->exec);
    delete vg;
    return HP_OK;
}

// hp_gpu_solve_mg with every cycle after the first replayed from a captured graph:
// one with the preconditioner set-ups inside (cycles where nc % prcn_every == 0) and
// one with them frozen (prcn_every = 0: every cycle).
extern "C" int hp_gpu_solve_mg_graph(hp_gpu_ctx **levels, int nlevels, double drop, int max_cycles, int vw,
                                     int itercrsn, int iterrfne, int check_every, int prcn_every, double *hist,
                                     int hist_cap, int *n_hist, double *seconds, int *cycles) {
    if (!levels || nlevels < 1 || drop <= 0.0 || max_cycles < 1) return HP_EINVAL;
    if (check_every < 1) check_every = 1;
    hp_gpu_ctx *f = levels[0];
    for (int l = 0; l < nlevels; ++l) {
        int r0_ = ensure_update_graph(levels[l]);
        if (r0_) return r0_;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, f->stream));
    int r, nh = 0, nc = 0;
    double r0 = 0.0, rn = 0.0;
    r = hp_gpu_setup_preconditioner(f);
    if (r) return r < 0 ? r : HP_ESTATE;
    if ((r = fp64_norm(f, &r0))) return r;
    if (hist && nh < hist_cap) hist[nh++] = 1.0;
    // first cycle evaluates every level's preconditioner at its own state
    if ((r = cycle(levels, nlevels, 0, vw, itercrsn, iterrfne, 1))) return r;
    ++nc;
    void *g_frozen = nullptr, *g_eval = nullptr;
    if ((r = hp_gpu_capture_vcycle(levels, nlevels, vw, itercrsn, iterrfne, 0, &g_frozen))) return r;
    if (prcn_every > 0 && (r = hp_gpu_capture_vcycle(levels, nlevels, vw, itercrsn, iterrfne, 1, &g_eval))) {
        hp_gpu_destroy_vcycle(g_frozen);
        return r;
    }
    for (int l = 0; l < nlevels; ++l) cudaMemsetAsync(levels[l]->d_err, 0, 4, f->stream);
    std::vector<int> bad(nlevels, 0);
    while (true) {
        if ((r = fp64_norm(f, &rn))) break;
        for (int l = 0; l < nlevels && g_eval; ++l)
            cudaMemcpyAsync(&bad[l], levels[l]->d_err, 4, cudaMemcpyDeviceToHost, f->stream);
        if (g_eval) cudaStreamSynchronize(f->stream);
        int nbad = 0;
        for (int l = 0; l < nlevels; ++l) nbad += bad[l];
        if (nbad) { r = nbad; set_err("%d bad elements in a preconditioner set-up", nbad); break; }
        const double d = rn / r0;
        if (hist && nh < hist_cap) hist[nh++] = d;
        if (!(d == d) || d <= drop || nc >= max_cycles) break;
        const int k = std::min(check_every, max_cycles - nc);
        for (int q = 0; q < k && !r; ++q, ++nc)
            r = hp_gpu_launch_vcycle((g_eval && nc % prcn_every == 0) ? g_eval : g_frozen, f, 1);
        if (r) break;
    }
    hp_gpu_destroy_vcycle(g_frozen);
    hp_gpu_destroy_vcycle(g_eval);
    if (r) return r;
    CK(cudaEventRecord(e1, f->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_hist) *n_hist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (cycles) *cycles = nc;
    return hp_gpu_sync(f);
}

// ---------------------------------------------------------------------------
// FP32 multigrid on the correction equation, inside FP64 defect correction.
// Every level l carries a base state b_l (fp32 of its FP64 state: the fine u,
// or u restricted down the hierarchy) and a correction d_l; its residual is the
// correction form F_l(d) = R_l(b_l + d) - R_l(b_l) + s_l with s_fine = R64(u)
// and s_coarse the FAS source fadd*restrict(F_fine) - F_coarse(d_entry).
// ---------------------------------------------------------------------------
static int alloc_mixed_mg(hp_gpu_ctx *c) {
    int r;
    if ((r = alloc_mixed(c))) return r;
    if (c->r0v32) return HP_OK;
    const size_t lv = std::max<size_t>(c->lv, 1), ls = std::max<size_t>(c->ls, 1), li = std::max<size_t>(c->li, 1);
    if ((r = dalloc(c, (void **)&c->r0v32, lv * 4)) || (r = dalloc(c, (void **)&c->r0s32, ls * 4)) ||
        (r = dalloc(c, (void **)&c->r0i32, li * 4)) || (r = dalloc(c, (void **)&c->c0v32, lv * 4)) ||
        (r = dalloc(c, (void **)&c->c0s32, ls * 4)) || (r = dalloc(c, (void **)&c->c0i32, li * 4)))
        return r;
    return HP_OK;
}

static Phys phys32(const hp_gpu_ctx *c) {
    Phys ph = c->ph;
    if (ph.physics == HP_PHYS_CD) ph.src = 0.0;
    return ph;
}

// F(d) of this level folded into s32.res (the source included when `with_src`)
static void rsdl32_folded(hp_gpu_ctx *c, bool with_src) {
    State<float> st = c->s32;
    if (!with_src) st.dresv = st.dress = st.dresi = nullptr;
    const int diff = (c->ph.physics == HP_PHYS_INS) ? 1 : 0;
    enqueue_rsdl_t<float>(c, c->L32, c->d_tab32, st, phys32(c), c->ph.nstage, diff);
    const long n = (long)(c->lv + c->ls);
    k_rsdl_fold<float><<<nblk(n, 256), 256, 0, c->stream>>>((int)c->lv, (int)c->ls, st.resv, st.rrv, st.ress, st.rrs,
                                                            st.dresv, st.dress);
}

static int mg_restrict32(hp_gpu_ctx *c) {
    hp_gpu_ctx *f = c->fine;
    const int NV = c->NV;
    State<float> &fs = f->s32, &cs = c->s32;
    rsdl32_folded(f, true);  // F_fine(d) with its source
    if (c->mg_kind == 1) {
        const long tot = (long)(c->lv + c->ls + c->li);
        const int g = std::min(nblk(tot, 256), c->nsm * 8);
        k_mg_truncate<float><<<g, 256, 0, c->stream>>>(c->npnt, c->nseg, c->ntri, NV, f->sm, f->im, c->sm, c->im,
                                                       fs.resv, fs.ress, fs.resi, c->r0v32, c->r0s32, c->r0i32);
        k_mg_truncate<float><<<g, 256, 0, c->stream>>>(c->npnt, c->nseg, c->ntri, NV, f->sm, f->im, c->sm, c->im,
                                                       fs.ugv, fs.ugs, fs.ugi, cs.ugv, cs.ugs, cs.ugi);
        CK(cudaMemcpyAsync(c->c0v32, cs.ugv, c->lv * 4, cudaMemcpyDeviceToDevice, c->stream));
        if (c->ls) CK(cudaMemcpyAsync(c->c0s32, cs.ugs, c->ls * 4, cudaMemcpyDeviceToDevice, c->stream));
        if (c->li) CK(cudaMemcpyAsync(c->c0i32, cs.ugi, c->li * 4, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        CK(cudaMemsetAsync(c->r0v32, 0, c->lv * 4, c->stream));
        k_mg_restrict_hres<float><<<nblk(f->npnt, 128), 128, 0, c->stream>>>(f->npnt, NV, c->f2c_tri, c->f2c_wt,
                                                                               c->mesh.tri_pnt, fs.resv, c->r0v32);
        k_mg_restrict_hstate<float><<<nblk(c->npnt, 128), 128, 0, c->stream>>>(c->npnt, NV, c->c2f_tri, c->c2f_wt,
                                                                                 f->mesh.tri_pnt, fs.ugv, cs.ugv,
                                                                                 c->c0v32);
    }
    rsdl32_folded(c, false);  // F_coarse(d_entry) without source
    const int g2 = c->nsm * 8;
    k_fas_source<float><<<g2, 256, 0, c->stream>>>((long)c->lv, c->fadd, c->r0v32, cs.resv, (float *)cs.dresv);
    if (c->ls) k_fas_source<float><<<g2, 256, 0, c->stream>>>((long)c->ls, c->fadd, c->r0s32, cs.ress, (float *)cs.dress);
    if (c->li) k_fas_source<float><<<g2, 256, 0, c->stream>>>((long)c->li, c->fadd, c->r0i32, cs.resi, (float *)cs.dresi);
    return check_launch(c);
}

static int mg_prolong32(hp_gpu_ctx *c) {
    hp_gpu_ctx *f = c->fine;
    const int NV = c->NV;
    State<float> &fs = f->s32, &cs = c->s32;
    if (c->mg_kind == 1) {
        const long tot = (long)(c->lv + c->ls + c->li);
        k_mg_prolong_p<float><<<std::min(nblk(tot, 256), c->nsm * 8), 256, 0, c->stream>>>(
            c->npnt, c->nseg, c->ntri, NV, f->sm, f->im, c->sm, c->im, cs.ugv, cs.ugs, cs.ugi, c->c0v32, c->c0s32,
            c->c0i32, fs.ugv, fs.ugs, fs.ugi);
    } else {
        k_mg_prolong_h<float><<<nblk(f->npnt, 128), 128, 0, c->stream>>>(f->npnt, NV, c->f2c_tri, c->f2c_wt,
                                                                           c->mesh.tri_pnt, cs.ugv, c->c0v32, fs.ugv);
    }
    return check_launch(c);
}

static int cycle32(hp_gpu_ctx **lv, int n, int lvl, int vw, int itercrsn, int iterrfne) {
    hp_gpu_ctx *c = lv[lvl];
    int r;
    if ((r = ensure_update32_graph(c))) return r;
    for (int vc = 0; vc < vw; ++vc) {
        for (int it = 0; it < itercrsn; ++it) CK(cudaGraphLaunch(c->g_update32, c->stream));
        if (lvl == n - 1) return HP_OK;
        if ((r = mg_restrict32(lv[lvl + 1]))) return r;
        if ((r = cycle32(lv, n, lvl + 1, vw, itercrsn, iterrfne))) return r;
        if ((r = mg_prolong32(lv[lvl + 1]))) return r;
        for (int it = 0; it < iterrfne; ++it) CK(cudaGraphLaunch(c->g_update32, c->stream));
    }
    return HP_OK;
}

// FP64 states of the coarse levels from the fine one (no FAS), their FP64
// preconditioners, and the FP32 copies (prcn and base states) of every level.
static int mixed_levels_setup(hp_gpu_ctx **lv, int n, bool prcn) {
    int r;
    for (int l = 1; l < n; ++l) {
        hp_gpu_ctx *c = lv[l], *f = lv[l - 1];
        if (c->mg_kind == 1) {
            const long tot = (long)(c->lv + c->ls + c->li);
            k_mg_truncate<double><<<std::min(nblk(tot, 256), c->nsm * 8), 256, 0, c->stream>>>(
                c->npnt, c->nseg, c->ntri, c->NV, f->sm, f->im, c->sm, c->im, f->st.ugv, f->st.ugs, f->st.ugi,
                c->st.ugv, c->st.ugs, c->st.ugi);
        } else {
            k_mg_restrict_hstate<double><<<nblk(c->npnt, 128), 128, 0, c->stream>>>(
                c->npnt, c->NV, c->c2f_tri, c->c2f_wt, f->mesh.tri_pnt, f->st.ugv, c->st.ugv, (double *)nullptr);
        }
    }
    for (int l = 0; l < n; ++l) {
        hp_gpu_ctx *c = lv[l];
        if (prcn || !c->prcn_ready) {
            r = hp_gpu_setup_preconditioner(c);
            if (r) return r < 0 ? r : HP_ESTATE;
            mixed_prcn(c);
        }
        State<float> &f = c->s32;
        conv(c, (long)c->lv, c->st.ugv, (float *)f.ubv);
        conv(c, (long)c->ls, c->st.ugs, (float *)f.ubs);
        conv(c, (long)c->li, c->st.ugi, (float *)f.ubi);
        base_points(c);
    }
    return check_launch(lv[0]);
}

extern "C" int hp_gpu_solve_mg_mixed(hp_gpu_ctx **levels, int nlevels, double drop, int max_cycles, int vw,
                                     int itercrsn, int iterrfne, int prcn_every, double *hist, int hist_cap,
                                     int *n_hist, double *seconds, int *cycles) {
    if (!levels || nlevels < 1 || drop <= 0.0 || max_cycles < 1) return HP_EINVAL;
    for (int l = 1; l < nlevels; ++l)
        if (!levels[l] || levels[l]->fine != levels[l - 1]) { set_err("levels not attached in order"); return HP_EINVAL; }
    hp_gpu_ctx *f = levels[0];
    int r;
    for (int l = 0; l < nlevels; ++l)
        if ((r = alloc_mixed_mg(levels[l])) || (r = ensure_update32_graph(levels[l]))) return r;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, f->stream));
    int nh = 0, nc = 0;
    double r0 = 0.0, rn = 0.0;
    r = hp_gpu_setup_preconditioner(f);
    if (r) return r < 0 ? r : HP_ESTATE;
    if ((r = fp64_norm(f, &r0))) return r;
    if (hist && nh < hist_cap) hist[nh++] = 1.0;
    while (nc < max_cycles) {
        const bool eval = (nc == 0) || (prcn_every > 0 && nc % prcn_every == 0);
        if ((r = mixed_levels_setup(levels, nlevels, eval))) return r;
        // the FP64 residual R64(u) from the last norm evaluation is the fine source
        mixed_prepare(f);
        if ((r = cycle32(levels, nlevels, 0, vw, itercrsn, iterrfne))) return r;
        mixed_apply(f);
        ++nc;
        if ((r = fp64_norm(f, &rn))) return r;
        const double d = rn / r0;
        if (hist && nh < hist_cap) hist[nh++] = d;
        if (!(d == d) || d <= drop) break;
    }
    CK(cudaEventRecord(e1, f->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_hist) *n_hist = nh;
    if (seconds) *seconds = ms * 1e-3;
    if (cycles) *cycles = nc;
    return hp_gpu_sync(f);
}

// ---------------------------------------------------------------------------
// Launch-shape autotuner. Each context is one mesh level at one p, so the best
// shapes differ between the levels of a hierarchy: the tuner times the candidate
// shapes of this context's element part (matrix-free kernel: CTAs per SM; stored
// operators: tiles per phase x CTAs per SM) and of its minvrt kernels (threads per
// CTA) on its own mesh, in FP64 and FP32, and keeps the fastest of each.
// ---------------------------------------------------------------------------
template <typename R>
static int tune_prec(hp_gpu_ctx *c, const Launchers<R> &L, const void *tab, const State<R> &st, const Phys &ph,
                     const DevMinv<R> *mt, int diff, Tune &tn, int reps, float *ms_out) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time = [&](auto &&fn) -> float {
        fn();  // warm
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < reps; ++r) fn();
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / reps;
    };
    const int ns = ph.nstage;
    auto elem = [&]() { launch_elem<R>(c, L, tab, st, ph, ns, 1, diff); };
    Tune keep = tn;
    float best = 1e30f;
    if (c->emat_on && c->emat_built && ph.physics == HP_PHYS_CD && !diff) {
        const int tpps[2] = {1, 2}, ctas[3] = {0, 4, 2};
        for (int a : tpps)
            for (int b : ctas) {
                tn.emat_tpp = a;
                tn.emat_ctas = b;
                const float t = time(elem);
                if (t < best) { best = t; keep = tn; }
            }
    } else {
        const int caps[3] = {4, 8, 16};
        for (int a : caps) {
            tn.elem_cap = a;
            const float t = time(elem);
            if (t < best) { best = t; keep = tn; }
        }
    }
    tn = keep;
    ms_out[0] = best;
    best = 1e30f;
    const int ths[3] = {64, 128, 256};
    for (int a : ths) {
        tn.minv_threads = a;
        const float t = time([&]() { enqueue_minvrt_t<R>(c, L, st, mt, 0.0, 0, 0, nullptr); });
        if (t < best) { best = t; keep = tn; }
    }
    tn = keep;
    ms_out[1] = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return check_launch(c);
}

extern "C" int hp_gpu_autotune(hp_gpu_ctx *c, int reps) {
    if (!c) return HP_EINVAL;
    if (!c->prcn_ready) { set_err("autotune before setup_preconditioner"); return HP_ESTATE; }
    if (reps < 1) reps = 5;
    int r;
    if ((r = tune_prec<double>(c, c->L, c->d_tab, c->st, c->ph, c->d_minv, 0, c->tune[0], reps, c->tune_ms[0])))
        return r;
    if ((r = alloc_mixed(c))) return r;
    mixed_prcn(c);
    const Phys p32 = phys32(c);
    if ((r = tune_prec<float>(c, c->L32, c->d_tab32, c->s32, p32, c->d_minv32, c->ph.physics == HP_PHYS_INS ? 1 : 0,
                              c->tune[1], reps, c->tune_ms[1])))
        return r;
    drop_update_graphs(c);  // captured graphs hold the old shapes
    return hp_gpu_sync(c);
}

extern "C" int hp_gpu_get_tuning(const hp_gpu_ctx *c, int *shapes, float *ms) {
    if (!c) return HP_EINVAL;
    for (int k = 0; k < 2; ++k) {
        const Tune &t = c->tune[k];
        if (shapes) {
            shapes[4 * k] = t.elem_cap;
            shapes[4 * k + 1] = t.emat_tpp;
            shapes[4 * k + 2] = t.emat_ctas;
            shapes[4 * k + 3] = t.minv_threads;
        }
        if (ms) { ms[2 * k] = c->tune_ms[k][0]; ms[2 * k + 1] = c->tune_ms[k][1]; }
    }
    return HP_OK;
}

// tri_hp::element_jacobian (nstage.cpp:131-165, fixed mesh) of every element, batched:
// one pass for the stage-0 residuals, one item per (element, column) for the columns.
extern "C" int hp_gpu_element_jacobian(hp_gpu_ctx *c, double *K) {
    if (!c || !K) return HP_EINVAL;
    if (!c->prcn_ready) {
        set_err("hp_gpu_element_jacobian needs tau from setup_preconditioner");
        return HP_ESTATE;
    }
    const size_t T = (size_t)(c->p + 1) * (c->p + 2) / 2, NJ = (size_t)c->NV * T;
    const size_t kb = (size_t)c->ntri * NJ * NJ * sizeof(double), rb = (size_t)c->ntri * NJ * sizeof(double);
    double *dK = nullptr, *dR = nullptr;
    if (!c->pool || cudaMallocFromPoolAsync((void **)&dK, kb, c->pool, c->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync((void **)&dR, rb, c->pool, c->stream) != cudaSuccess) {
        if (dK) cudaFreeAsync(dK, c->stream);
        set_err("device allocation of %zu bytes for the element Jacobians failed", kb + rb);
        return HP_ENOMEM;
    }
    c->L.elem_jac(c->d_tab, c->mesh, c->st, c->ph, dK, dR, c->nsm, c->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(K, dK, kb, cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(dK, c->stream);
    cudaFreeAsync(dR, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        set_err("element Jacobians: %s", cudaGetErrorString(e));
        return HP_ECUDA;
    }
    return HP_OK;
}
