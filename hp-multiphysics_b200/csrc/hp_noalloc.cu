// Residual norm over caller-owned device arrays without any device allocation.
//
// hp_gpu_resnorm reduces the residual through a partials buffer that its
// context allocated with cudaMalloc. Some callers of this library cannot
// allocate at the moment they need the norm: an application that hands all
// device memory to its own pool when it starts and forbids further
// cudaMalloc/cudaFree, or a solver embedded in a host program whose memory
// budget is fixed before the solve begins. hp_resnorm_noalloc serves them: its
// only scratch is the file-scope device array below, of fixed size, which every
// GPU that loads the library keeps until the process exits.
//
// Host code must not pass the array's name to a kernel (in host code that name
// is a host-side stand-in, not a device address): the device address is looked
// up with cudaGetSymbolAddress, with the device current, on the first call made
// in each CUDA context, and kept per context (a new context, e.g. after
// cudaDeviceReset, gets its own lookup). The call launches two kernels on
// `stream`, copies the two results to the host and synchronises `stream` before
// it returns. All calls share the one array, so calls whose work overlaps on
// the GPU (different streams, or different host threads on the same device)
// race on it and must be serialised by the caller. Every call writes each
// partial it reads before reading it, so nothing has to start at zero.
#include <cuda.h>
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include <cstdio>

#include "hp_gpu.h"

namespace {

constexpr int kThreads = 256;

// [0, 2*MAX): per-chunk (sum of squares, max |x|); [2*MAX, 2*MAX+2): final pair
static __device__ __align__(256) double g_norm_scratch[2 * HP_NOALLOC_MAX_CHUNKS + 2];

std::mutex g_mu;
// device address of g_norm_scratch, per device ordinal, valid for the context whose
// unique id (cuCtxGetId) is g_scratch_ctx[dev]
double *g_scratch_dev[64] = {nullptr};
unsigned long long g_scratch_ctx[64] = {0};
thread_local std::string g_noalloc_err;

__device__ __forceinline__ void block_reduce(double &s, double &m) {
    __shared__ double ss[kThreads / 32], sx[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        const double b = __shfl_xor_sync(0xffffffffu, m, o);
        m = b > m ? b : m;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { ss[w] = s; sx[w] = m; }
    __syncthreads();
    if (threadIdx.x == 0) {
        s = 0.0; m = 0.0;
        for (int q = 0; q < kThreads / 32; ++q) {
            s += ss[q];
            m = sx[q] > m ? sx[q] : m;
        }
    }
}

// One block per chunk of HP_NOALLOC_CHUNK elements of the concatenation (a | b | c).
__global__ void k_chunk_norm(const double *a, long long na, long long ca, const double *b, long long nb, long long cb,
                             const double *c, long long nc, double *scratch) {
    long long chunk = blockIdx.x;
    const double *x;
    long long n;
    if (chunk < ca) { x = a; n = na; }
    else if (chunk < ca + cb) { x = b; n = nb; chunk -= ca; }
    else { x = c; n = nc; chunk -= ca + cb; }
    const long long beg = chunk * HP_NOALLOC_CHUNK;
    long long end = beg + HP_NOALLOC_CHUNK;
    if (end > n) end = n;
    double s = 0.0, m = 0.0;
    for (long long k = beg + threadIdx.x; k < end; k += kThreads) {
        const double v = x[k];
        s += v * v;
        const double av = fabs(v);
        m = av > m ? av : m;
    }
    block_reduce(s, m);
    if (threadIdx.x == 0) {
        scratch[2 * blockIdx.x] = s;
        scratch[2 * blockIdx.x + 1] = m;
    }
}

__global__ void k_chunk_final(int nchunks, double *scratch) {
    double s = 0.0, m = 0.0;
    for (int k = threadIdx.x; k < nchunks; k += kThreads) {
        s += scratch[2 * k];
        const double v = scratch[2 * k + 1];
        m = v > m ? v : m;
    }
    block_reduce(s, m);
    if (threadIdx.x == 0) {
        scratch[2 * HP_NOALLOC_MAX_CHUNKS] = sqrt(s);
        scratch[2 * HP_NOALLOC_MAX_CHUNKS + 1] = m;
    }
}

int fail(int code, const char *msg) {
    g_noalloc_err = msg;
    return code;
}

int fail_cuda(const char *what, cudaError_t e) {
    g_noalloc_err = std::string("hp_resnorm_noalloc: ") + what + ": " + cudaGetErrorString(e);
    return HP_ECUDA;
}

// Unique id of the calling thread's current context, through the driver entry points
// the runtime hands out (the library does not link libcuda itself). Called with g_mu held.
bool current_context_id(unsigned long long *id) {
    using get_current_t = CUresult (*)(CUcontext *);
    using get_id_t = CUresult (*)(CUcontext, unsigned long long *);
    static get_current_t get_current = nullptr;
    static get_id_t get_id = nullptr;
    if (!get_current || !get_id) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return false;
        get_current = reinterpret_cast<get_current_t>(f0);
        get_id = reinterpret_cast<get_id_t>(f1);
    }
    CUcontext cu = nullptr;
    return get_current(&cu) == CUDA_SUCCESS && cu != nullptr && get_id(cu, id) == CUDA_SUCCESS;
}

}  // namespace

extern "C" const char *hp_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" int hp_resnorm_noalloc(const double *resv, long long nv, const double *ress, long long ns,
                                  const double *resi, long long ni, double *l2, double *linf, void *stream) {
    g_noalloc_err.clear();
    if (!l2 || !linf) return fail(HP_EINVAL, "hp_resnorm_noalloc: null output pointer");
    if (nv < 0 || ns < 0 || ni < 0) return fail(HP_EINVAL, "hp_resnorm_noalloc: negative length");
    if ((nv && !resv) || (ns && !ress) || (ni && !resi))
        return fail(HP_EINVAL, "hp_resnorm_noalloc: null input pointer with non-zero length");
    const long long ca = (nv + HP_NOALLOC_CHUNK - 1) / HP_NOALLOC_CHUNK;
    const long long cb = (ns + HP_NOALLOC_CHUNK - 1) / HP_NOALLOC_CHUNK;
    const long long cc = (ni + HP_NOALLOC_CHUNK - 1) / HP_NOALLOC_CHUNK;
    const long long nchunks = ca + cb + cc;
    if (nchunks > HP_NOALLOC_MAX_CHUNKS) {
        static char msg[160];
        snprintf(msg, sizeof(msg),
                 "hp_resnorm_noalloc: %lld values need %lld chunks of %d; the static scratch holds %d "
                 "(at most %lld values per call)",
                 nv + ns + ni, nchunks, HP_NOALLOC_CHUNK, HP_NOALLOC_MAX_CHUNKS,
                 (long long)HP_NOALLOC_MAX_CHUNKS * HP_NOALLOC_CHUNK);
        return fail(HP_EINVAL, msg);
    }
    if (nchunks == 0) {
        *l2 = 0.0;
        *linf = 0.0;
        return HP_OK;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda("no current CUDA device", e);
    if (dev < 0 || dev >= 64) return fail(HP_ECUDA, "hp_resnorm_noalloc: device ordinal beyond 63");
    // an error left by an earlier, unrelated call is reported as such, not as this call's
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail_cuda("a CUDA error was pending before this call", e);
    double *scratch;
    {
        std::lock_guard<std::mutex> lk(g_mu);  // also guards the driver entry points' lookup
        // the context's unique id keys the cache; with no context current on this thread,
        // cudaSetDevice of the current device initialises its primary context (CUDA >= 12)
        // and makes it current
        unsigned long long ctx_id = 0;
        if (!current_context_id(&ctx_id)) {
            e = cudaSetDevice(dev);
            if (e != cudaSuccess) return fail_cuda("context initialisation failed", e);
            if (!current_context_id(&ctx_id)) return fail(HP_ECUDA, "hp_resnorm_noalloc: no current CUDA context");
        }
        if (!g_scratch_dev[dev] || g_scratch_ctx[dev] != ctx_id) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_norm_scratch);
            if (e != cudaSuccess || !p) return fail_cuda("cudaGetSymbolAddress failed", e);
            g_scratch_dev[dev] = static_cast<double *>(p);
            g_scratch_ctx[dev] = ctx_id;
        }
        scratch = g_scratch_dev[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_chunk_norm<<<(unsigned)nchunks, kThreads, 0, st>>>(resv, nv, ca, ress, ns, cb, resi, ni, scratch);
    k_chunk_final<<<1, kThreads, 0, st>>>((int)nchunks, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda("kernel launch failed", e);
    double out[2];
    e = cudaMemcpyAsync(out, scratch + 2 * HP_NOALLOC_MAX_CHUNKS, sizeof(out), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return fail_cuda("result copy failed", e);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda("stream synchronisation failed", e);
    *l2 = out[0];
    *linf = out[1];
    return HP_OK;
}
