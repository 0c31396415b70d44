// Learned correction of the Jacobi preconditioner: a small multilayer perceptron
// (no counterpart in the reference) with hand-written BF16 inference and
// training kernels, FP32 accumulation.
//
// Layout: layers l = 0..L-1 map n_l -> n_{l+1}; W_l is [n_{l+1}][n_l] row-major,
// b_l [n_{l+1}]; ReLU between layers, linear output. Inputs are standardised with
// (x - mean) / std inside the first layer. Parameters live on the device as an
// FP32 master copy (training, Adam moments beside it) and a BF16 copy used by
// the forward pass; activations are rounded to BF16 between layers, every dot
// product accumulates in FP32.
//
// Kernels: inference of the learned corrections' shape (inputs <= 32, hidden layers of
// 64, one output) on the BF16 tensor cores (k_mlp_forward_mma); other shapes and the
// training pass one thread per sample, the parameters staged in shared memory (all
// threads of a warp read the same weight: broadcast, no bank conflicts). The
// backward pass reduces each weight's per-sample gradient across the warp with
// shuffles, then across the block in shared memory, then into the global FP32
// gradient with one atomic per weight per block.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hp_gpu.h"
#include "hp_mlp.h"

namespace {

constexpr int kMaxLayers = 6;
constexpr int kMaxWidth = 64;
constexpr int kThreads = 128;

thread_local std::string g_mlp_err;

struct Dims {
    int L;                 // number of affine layers
    int n[kMaxLayers + 1];  // widths n[0] = inputs ... n[L] = outputs
    int woff[kMaxLayers], boff[kMaxLayers];
    int nparam;
};

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Forward pass of one sample; acts[l][k] = activation after layer l (BF16-rounded),
// returns outputs in y. params: [W0 b0 W1 b1 ...] (already BF16-rounded floats).
__device__ void forward_one(const Dims &d, const float *p, const float *mean, const float *istd, const float *x,
                            float acts[kMaxLayers + 1][kMaxWidth]) {
    for (int k = 0; k < d.n[0]; ++k) acts[0][k] = bf((x[k] - mean[k]) * istd[k]);
    for (int l = 0; l < d.L; ++l) {
        const float *W = p + d.woff[l], *b = p + d.boff[l];
        const int ni = d.n[l], no = d.n[l + 1];
        for (int o = 0; o < no; ++o) {
            float acc = b[o];
            for (int i = 0; i < ni; ++i) acc += W[o * ni + i] * acts[l][i];
            if (l < d.L - 1) acc = acc > 0.f ? acc : 0.f;
            acts[l + 1][o] = (l < d.L - 1) ? bf(acc) : acc;
        }
    }
}

__global__ void k_mlp_forward(Dims d, const float *__restrict__ pbf, const float *__restrict__ mean,
                              const float *__restrict__ istd, const float *__restrict__ X, int n, float *__restrict__ Y) {
    extern __shared__ float sp[];
    for (int k = threadIdx.x; k < d.nparam; k += blockDim.x) sp[k] = pbf[k];
    __shared__ float sm[kMaxWidth], ss[kMaxWidth];
    for (int k = threadIdx.x; k < d.n[0]; k += blockDim.x) { sm[k] = mean[k]; ss[k] = istd[k]; }
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float acts[kMaxLayers + 1][kMaxWidth];
    forward_one(d, sp, sm, ss, X + (size_t)s * d.n[0], acts);
    for (int o = 0; o < d.n[d.L]; ++o) Y[(size_t)s * d.n[d.L] + o] = acts[d.L][o];
}

// Gradient of 0.5/n * sum_s sum_o mask_o (y_so - t_so)^2 w.r.t. the FP32 master
// parameters (straight-through for the BF16 roundings), accumulated into grad;
// loss accumulated into *loss.
__global__ void k_mlp_backward(Dims d, const float *__restrict__ pbf, const float *__restrict__ mean,
                               const float *__restrict__ istd, const float *__restrict__ X,
                               const float *__restrict__ Tg, const float *__restrict__ mask, int n, float inv_n,
                               float *__restrict__ grad, float *__restrict__ loss) {
    extern __shared__ float sh[];
    float *sp = sh;               // parameters (BF16-rounded)
    float *sg = sh + d.nparam;    // block gradient accumulator
    for (int k = threadIdx.x; k < d.nparam; k += blockDim.x) { sp[k] = pbf[k]; sg[k] = 0.f; }
    __shared__ float sm[kMaxWidth], ss[kMaxWidth], sl;
    for (int k = threadIdx.x; k < d.n[0]; k += blockDim.x) { sm[k] = mean[k]; ss[k] = istd[k]; }
    if (threadIdx.x == 0) sl = 0.f;
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = s < n;
    const int lane = threadIdx.x & 31;
    float acts[kMaxLayers + 1][kMaxWidth];
    float delta[kMaxWidth], prev[kMaxWidth];
    if (act) forward_one(d, sp, sm, ss, X + (size_t)s * d.n[0], acts);
    const int nout = d.n[d.L];
    float l2 = 0.f;
    for (int o = 0; o < nout; ++o) {
        const float e = act ? acts[d.L][o] - Tg[(size_t)s * nout + o] : 0.f;
        l2 += mask[o] * e * e;
        delta[o] = mask[o] * e * inv_n;
    }
    for (int l = d.L - 1; l >= 0; --l) {
        const int ni = d.n[l], no = d.n[l + 1];
        const float *W = sp + d.woff[l];
        // weight and bias gradients: dW[o][i] = delta[o] * acts[l][i]
        for (int o = 0; o < no; ++o) {
            for (int i = 0; i <= ni; ++i) {
                float g = act ? delta[o] * (i < ni ? acts[l][i] : 1.f) : 0.f;
                for (int off = 16; off > 0; off >>= 1) g += __shfl_xor_sync(0xffffffffu, g, off);
                if (lane == 0) atomicAdd(&sg[i < ni ? d.woff[l] + o * ni + i : d.boff[l] + o], g);
            }
        }
        if (l > 0) {
            for (int i = 0; i < ni; ++i) {
                float acc = 0.f;
                for (int o = 0; o < no; ++o) acc += W[o * ni + i] * delta[o];
                prev[i] = acts[l][i] > 0.f ? acc : 0.f;  // ReLU' of the layer that produced acts[l]
            }
            for (int i = 0; i < ni; ++i) delta[i] = prev[i];
        }
    }
    for (int off = 16; off > 0; off >>= 1) l2 += __shfl_xor_sync(0xffffffffu, l2, off);
    if (lane == 0) atomicAdd(&sl, l2);
    __syncthreads();
    for (int k = threadIdx.x; k < d.nparam; k += blockDim.x) atomicAdd(&grad[k], sg[k]);
    if (threadIdx.x == 0) atomicAdd(loss, 0.5f * sl * inv_n);
}

// Forward pass on the BF16 tensor cores (mma.sync.m16n8k16, FP32 accumulation) for the
// shape of the learned corrections: n0 <= 32 inputs, hidden layers of 64, one output.
// A warp takes 16 samples: each layer's C fragments (+ bias, ReLU, rounded to BF16) are
// the next layer's A fragments as they sit in the registers (n-tiles 2t and 2t + 1 of the
// output are k-step t of the next product); the weights are the B operands, staged in
// shared memory as BF16 with padded rows; the 64 -> 1 output layer is a dot product per
// sample summed over the four lanes that hold a row. Same arithmetic as forward_one up to
// the order of the FP32 sums.
constexpr int kMmaW = 64, kMmaP0 = 40, kMmaPH = 72;  // hidden width; padded row lengths (BF16)

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                 "{%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(128) k_mlp_forward_mma(Dims d, const float *__restrict__ pbf,
                                                         const float *__restrict__ mean,
                                                         const float *__restrict__ istd, const float *__restrict__ X,
                                                         int n, float *__restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nh = d.L - 1;  // hidden layers (each followed by ReLU)
    __nv_bfloat16 *w0 = reinterpret_cast<__nv_bfloat16 *>(smraw);     // [64][kMmaP0]
    __nv_bfloat16 *wh = w0 + kMmaW * kMmaP0;                            // [nh-1][64][kMmaPH]
    float *bias = reinterpret_cast<float *>(wh + (size_t)(nh - 1) * kMmaW * kMmaPH);  // [nh][64]
    float *wout = bias + nh * kMmaW;                                      // [64], then bout
    float *smean = wout + kMmaW + 1, *sistd = smean + 32;
    const int n0 = d.n[0];
    for (int k = threadIdx.x; k < kMmaW * kMmaP0; k += blockDim.x) {
        const int o = k / kMmaP0, i = k - o * kMmaP0;
        w0[k] = __float2bfloat16_rn(i < n0 ? pbf[d.woff[0] + o * n0 + i] : 0.f);
    }
    for (int l = 1; l < nh; ++l)
        for (int k = threadIdx.x; k < kMmaW * kMmaPH; k += blockDim.x) {
            const int o = k / kMmaPH, i = k - o * kMmaPH;
            wh[(size_t)(l - 1) * kMmaW * kMmaPH + k] =
                __float2bfloat16_rn(i < kMmaW ? pbf[d.woff[l] + o * kMmaW + i] : 0.f);
        }
    for (int k = threadIdx.x; k < nh * kMmaW; k += blockDim.x) bias[k] = pbf[d.boff[k / kMmaW] + k % kMmaW];
    for (int k = threadIdx.x; k <= kMmaW; k += blockDim.x) wout[k] = pbf[k < kMmaW ? d.woff[nh] + k : d.boff[nh]];
    for (int k = threadIdx.x; k < 32; k += blockDim.x) {
        smean[k] = k < n0 ? mean[k] : 0.f;
        sistd[k] = k < n0 ? istd[k] : 0.f;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    const long step = (long)gridDim.x * (blockDim.x >> 5) * 16;
    for (long base = ((long)blockIdx.x * (blockDim.x >> 5) + warp) * 16; base < n; base += step) {
        const long r0 = base + g, r1 = base + g + 8;
        // layer 0 A fragments: standardised inputs, rounded to BF16, K padded to 32
        unsigned a[4][4];
        auto xin = [&](long r, int k) -> float {
            return (r < n && k < n0) ? (X[(size_t)r * n0 + k] - smean[k]) * sistd[k] : 0.f;
        };
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const int k = ks * 16 + 2 * t4;
            a[ks][0] = pack_bf16(xin(r0, k), xin(r0, k + 1));
            a[ks][1] = pack_bf16(xin(r1, k), xin(r1, k + 1));
            a[ks][2] = pack_bf16(xin(r0, k + 8), xin(r0, k + 9));
            a[ks][3] = pack_bf16(xin(r1, k + 8), xin(r1, k + 9));
        }
        float c[8][4];
        for (int l = 0; l < nh; ++l) {
            const float *bl = bias + l * kMmaW;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int col = nt * 8 + 2 * t4;
                c[nt][0] = c[nt][2] = bl[col];
                c[nt][1] = c[nt][3] = bl[col + 1];
            }
            const int nks = l == 0 ? 2 : 4, ld = l == 0 ? kMmaP0 : kMmaPH;
            const __nv_bfloat16 *W = l == 0 ? w0 : wh + (size_t)(l - 1) * kMmaW * kMmaPH;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                if (ks >= nks) break;
#pragma unroll
                for (int nt = 0; nt < 8; ++nt) {
                    const __nv_bfloat16 *wr = W + (size_t)(nt * 8 + g) * ld + ks * 16 + 2 * t4;
                    const unsigned b0 = *reinterpret_cast<const unsigned *>(wr);
                    const unsigned b1 = *reinterpret_cast<const unsigned *>(wr + 8);
                    mma_bf16(c[nt], a[ks], b0, b1);
                }
            }
            // ReLU, BF16: the next layer's A fragments
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                auto rl = [](float v) { return v > 0.f ? v : 0.f; };
                a[t][0] = pack_bf16(rl(c[2 * t][0]), rl(c[2 * t][1]));
                a[t][1] = pack_bf16(rl(c[2 * t][2]), rl(c[2 * t][3]));
                a[t][2] = pack_bf16(rl(c[2 * t + 1][0]), rl(c[2 * t + 1][1]));
                a[t][3] = pack_bf16(rl(c[2 * t + 1][2]), rl(c[2 * t + 1][3]));
            }
        }
        // output layer 64 -> 1 on the BF16 activations
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = (2 * t + h) * 8 + 2 * t4;
                const __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162 *>(&a[t][2 * h]);
                const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162 *>(&a[t][2 * h + 1]);
                y0 += wout[col] * __low2float(lo) + wout[col + 1] * __high2float(lo);
                y1 += wout[col] * __low2float(hi) + wout[col + 1] * __high2float(hi);
            }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (t4 == 0) {
            if (r0 < n) Y[r0] = wout[kMmaW] + y0;
            if (r1 < n) Y[r1] = wout[kMmaW] + y1;
        }
    }
}

static bool mma_shape(const Dims &d) {
    if (d.L < 2 || d.n[0] > 32 || d.n[d.L] != 1) return false;
    for (int l = 1; l < d.L; ++l)
        if (d.n[l] != kMmaW) return false;
    return true;
}

static size_t mma_smem(const Dims &d) {
    const int nh = d.L - 1;
    return (size_t)kMmaW * kMmaP0 * 2 + (size_t)(nh - 1) * kMmaW * kMmaPH * 2 + (size_t)nh * kMmaW * 4 +
           (kMmaW + 1) * 4 + 64 * 4;
}

__global__ void k_round_bf16(const float *w, float *wb, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) wb[k] = bf(w[k]);
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

}  // namespace

struct hp_mlp {
    Dims d;
    float *w = nullptr, *wb = nullptr, *m = nullptr, *v = nullptr, *g = nullptr, *mean = nullptr, *istd = nullptr,
          *loss = nullptr;
    int step = 0;
};

extern "C" const char *hp_mlp_last_error(void) { return g_mlp_err.c_str(); }

static int merr(int code, const char *m) {
    g_mlp_err = m;
    return code;
}

#define MCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return merr(HP_ECUDA, cudaGetErrorString(e_));              \
    } while (0)

extern "C" int hp_mlp_create(int nlayers, const int *widths, unsigned long long seed, hp_mlp **out) {
    if (!widths || !out || nlayers < 1 || nlayers > kMaxLayers) return merr(HP_EINVAL, "bad layer count");
    hp_mlp *net = new hp_mlp();
    Dims &d = net->d;
    d.L = nlayers;
    int off = 0;
    for (int l = 0; l <= nlayers; ++l) {
        if (widths[l] < 1 || widths[l] > kMaxWidth) { delete net; return merr(HP_EINVAL, "width outside [1,64]"); }
        d.n[l] = widths[l];
    }
    for (int l = 0; l < nlayers; ++l) {
        d.woff[l] = off;
        off += d.n[l] * d.n[l + 1];
        d.boff[l] = off;
        off += d.n[l + 1];
    }
    d.nparam = off;
    // He-uniform initialisation from a splitmix64 stream (deterministic)
    std::vector<float> h(off, 0.f);
    unsigned long long z = seed;
    auto next = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        unsigned long long x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < nlayers; ++l) {
        const float a = std::sqrt(6.0f / d.n[l]) * (l == nlayers - 1 ? 0.1f : 1.0f);
        for (int k = 0; k < d.n[l] * d.n[l + 1]; ++k) h[d.woff[l] + k] = (float)((2.0 * next() - 1.0) * a);
    }
    const size_t B = (size_t)off * 4;
    if (cudaMalloc(&net->w, B) || cudaMalloc(&net->wb, B) || cudaMalloc(&net->m, B) || cudaMalloc(&net->v, B) ||
        cudaMalloc(&net->g, B) || cudaMalloc(&net->mean, kMaxWidth * 4) || cudaMalloc(&net->istd, kMaxWidth * 4) ||
        cudaMalloc(&net->loss, 4)) {
        hp_mlp_destroy(net);
        return merr(HP_ENOMEM, "cudaMalloc failed");
    }
    cudaMemcpy(net->w, h.data(), B, cudaMemcpyHostToDevice);
    cudaMemset(net->m, 0, B);
    cudaMemset(net->v, 0, B);
    std::vector<float> mu(kMaxWidth, 0.f), sd(kMaxWidth, 1.f);
    cudaMemcpy(net->mean, mu.data(), kMaxWidth * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(net->istd, sd.data(), kMaxWidth * 4, cudaMemcpyHostToDevice);
    k_round_bf16<<<(off + 255) / 256, 256>>>(net->w, net->wb, off);
    MCK(cudaDeviceSynchronize());
    *out = net;
    return HP_OK;
}

extern "C" int hp_mlp_destroy(hp_mlp *net) {
    if (!net) return HP_OK;
    for (float *p : {net->w, net->wb, net->m, net->v, net->g, net->mean, net->istd, net->loss})
        if (p) cudaFree(p);
    delete net;
    return HP_OK;
}

extern "C" int hp_mlp_nparams(const hp_mlp *net) { return net ? net->d.nparam : HP_EINVAL; }

extern "C" int hp_mlp_set_norm(hp_mlp *net, const float *mean, const float *stdv) {
    if (!net || !mean || !stdv) return merr(HP_EINVAL, "null argument");
    std::vector<float> is(net->d.n[0]);
    for (int k = 0; k < net->d.n[0]; ++k) is[k] = stdv[k] > 0.f ? 1.f / stdv[k] : 1.f;
    MCK(cudaMemcpy(net->mean, mean, net->d.n[0] * 4, cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(net->istd, is.data(), net->d.n[0] * 4, cudaMemcpyHostToDevice));
    return HP_OK;
}

extern "C" int hp_mlp_get_params(const hp_mlp *net, float *host) {
    if (!net || !host) return merr(HP_EINVAL, "null argument");
    MCK(cudaMemcpy(host, net->w, (size_t)net->d.nparam * 4, cudaMemcpyDeviceToHost));
    return HP_OK;
}

extern "C" int hp_mlp_set_params(hp_mlp *net, const float *host) {
    if (!net || !host) return merr(HP_EINVAL, "null argument");
    MCK(cudaMemcpy(net->w, host, (size_t)net->d.nparam * 4, cudaMemcpyHostToDevice));
    k_round_bf16<<<(net->d.nparam + 255) / 256, 256>>>(net->w, net->wb, net->d.nparam);
    MCK(cudaDeviceSynchronize());
    return HP_OK;
}

static size_t fwd_smem(const hp_mlp *net) { return (size_t)net->d.nparam * 4; }

extern "C" int hp_mlp_forward(hp_mlp *net, const float *d_x, int n, float *d_y, void *stream) {
    if (!net || (n > 0 && (!d_x || !d_y)) || n < 0) return merr(HP_EINVAL, "bad argument");
    if (n == 0) return HP_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (mma_shape(net->d)) {  // the learned corrections' shape: BF16 tensor cores
        const size_t smm = mma_smem(net->d);
        if (smm > 48 * 1024)
            MCK(cudaFuncSetAttribute(k_mlp_forward_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smm));
        const long groups = ((long)n + 15) / 16;
        const int blocks = (int)std::min<long>((groups + 3) / 4, 148L * 16);
        k_mlp_forward_mma<<<blocks, 128, smm, st>>>(net->d, net->wb, net->mean, net->istd, d_x, n, d_y);
        MCK(cudaGetLastError());
        return HP_OK;
    }
    const size_t sm = fwd_smem(net);
    if (sm > 48 * 1024) MCK(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_mlp_forward<<<(n + kThreads - 1) / kThreads, kThreads, sm, st>>>(net->d, net->wb, net->mean, net->istd, d_x, n,
                                                                       d_y);
    MCK(cudaGetLastError());
    return HP_OK;
}

// Gradient of the masked MSE over n samples into host_grad (FP32, nparam) and the
// loss into *loss; nothing is updated.
static int grad_device(hp_mlp *net, const float *d_x, const float *d_t, const float *mask, int n, cudaStream_t st) {
    const int P = net->d.nparam;
    MCK(cudaMemsetAsync(net->g, 0, (size_t)P * 4, st));
    MCK(cudaMemsetAsync(net->loss, 0, 4, st));
    const size_t sm = (size_t)2 * P * 4;
    MCK(cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_mlp_backward<<<(n + kThreads - 1) / kThreads, kThreads, sm, st>>>(net->d, net->wb, net->mean, net->istd, d_x, d_t,
                                                                        mask, n, 1.f / (float)n, net->g, net->loss);
    MCK(cudaGetLastError());
    return HP_OK;
}

extern "C" int hp_mlp_grad(hp_mlp *net, const float *d_x, const float *d_t, const float *d_mask, int n,
                           float *host_grad, float *loss) {
    if (!net || !d_x || !d_t || !d_mask || n < 1 || !host_grad) return merr(HP_EINVAL, "bad argument");
    int r = grad_device(net, d_x, d_t, d_mask, n, 0);
    if (r) return r;
    MCK(cudaMemcpy(host_grad, net->g, (size_t)net->d.nparam * 4, cudaMemcpyDeviceToHost));
    if (loss) MCK(cudaMemcpy(loss, net->loss, 4, cudaMemcpyDeviceToHost));
    return HP_OK;
}

extern "C" int hp_mlp_train_step(hp_mlp *net, const float *d_x, const float *d_t, const float *d_mask, int n, float lr,
                                 float *loss) {
    if (!net || !d_x || !d_t || !d_mask || n < 1) return merr(HP_EINVAL, "bad argument");
    int r = grad_device(net, d_x, d_t, d_mask, n, 0);
    if (r) return r;
    net->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)net->step), c2 = 1.f - std::pow(b2, (float)net->step);
    const int P = net->d.nparam;
    k_adam<<<(P + 255) / 256, 256>>>(net->w, net->g, net->m, net->v, P, lr, b1, b2, 1e-8f, c1, c2);
    k_round_bf16<<<(P + 255) / 256, 256>>>(net->w, net->wb, P);
    MCK(cudaGetLastError());
    if (loss) MCK(cudaMemcpy(loss, net->loss, 4, cudaMemcpyDeviceToHost));
    return HP_OK;
}

extern "C" int hp_mlp_dims(const hp_mlp *net, int *nin, int *nout) {
    if (!net) return merr(HP_EINVAL, "null network");
    if (nin) *nin = net->d.n[0];
    if (nout) *nout = net->d.n[net->d.L];
    return HP_OK;
}
