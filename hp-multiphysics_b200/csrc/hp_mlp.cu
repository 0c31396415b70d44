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
// Kernels: one thread per sample, the parameters staged in shared memory (all
// threads of a warp read the same weight: broadcast, no bank conflicts). The
// backward pass reduces each weight's per-sample gradient across the warp with
// shuffles, then across the block in shared memory, then into the global FP32
// gradient with one atomic per weight per block.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
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
