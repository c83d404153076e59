// Error statistics of a reconstruction without any allocation: the scratch lives in a
// file-scope device array, so the call needs no context and no cudaMalloc.
//
// Result: max |x - y| as a float and PSNR = 10 log10(range^2 / mse), the figures
// asz_compress_stats reports (the reference prints them after compressing,
// c_codes/asz_core/compress.tpp:307-319). The squared differences are summed in a fixed order
// (per-tile partials, then one ordered pass over the partials), so repeated calls on the same
// data return identical bits.
//
// Layout of the scratch (kScratchBytes = 1 MiB):
//   [0, 256)          control: the count of finished tiles (must start at zero) and the result
//   [256, 1 MiB)      one Partial (max, sse) per tile of kTile elements
// so n is limited to kMaxTiles * kTile = 65520 * 65536 elements (about 4.29e9 floats).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/asz_b200.h"

namespace {

constexpr size_t kScratchBytes = 1u << 20;
constexpr size_t kControlBytes = 256;
constexpr uint64_t kTile = 1u << 16;  // elements per tile (one CTA each)
constexpr int kThreads = 256;

struct Partial {
    float max;
    float pad;
    double sse;
};

struct Control {
    unsigned int done;  // tiles finished; the last one to finish reduces the partials
    unsigned int pad;
    Partial result;
};

constexpr uint64_t kMaxTiles = (kScratchBytes - kControlBytes) / sizeof(Partial);
static_assert(sizeof(Control) <= kControlBytes, "control block too large");

static __device__ __align__(256) unsigned char g_stats_scratch[kScratchBytes];

// Fixed-order block reduction of (max, sse) over kThreads threads.
__device__ Partial block_reduce(float mx, double s, Partial *sh) {
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sh[warp] = Partial{mx, 0.0f, s};
    __syncthreads();
    Partial r{0.0f, 0.0f, 0.0};
    if (threadIdx.x == 0) {
        for (int w = 0; w < kThreads / 32; w++) {
            r.max = fmaxf(r.max, sh[w].max);
            r.sse += sh[w].sse;
        }
    }
    return r;
}

__global__ void __launch_bounds__(kThreads)
    stats_noalloc_kernel(const float *__restrict__ x, const float *__restrict__ y, uint64_t n, unsigned char *scratch) {
    __shared__ Partial sh[kThreads / 32];
    __shared__ bool last;
    Control *ctl = (Control *)scratch;
    Partial *part = (Partial *)(scratch + kControlBytes);
    const uint64_t begin = (uint64_t)blockIdx.x * kTile;
    const uint64_t end = begin + kTile < n ? begin + kTile : n;
    float mx = 0.0f;
    double s = 0.0;
    for (uint64_t i = begin + threadIdx.x; i < end; i += kThreads) {
        const float a = x[i], b = y[i];
        mx = fmaxf(mx, fabsf(__fsub_rn(a, b)));
        const double d = (double)a - (double)b;
        s = __fma_rn(d, d, s);
    }
    Partial p = block_reduce(mx, s, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = p;
        __threadfence();
        last = atomicAdd(&ctl->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // The last tile to finish: ordered pass over all partials.
    __threadfence();
    mx = 0.0f;
    s = 0.0;
    for (uint64_t t = threadIdx.x; t < gridDim.x; t += kThreads) {
        // L2 loads: the partials were written by other CTAs.
        mx = fmaxf(mx, __ldcg(&part[t].max));
        s += __ldcg(&part[t].sse);
    }
    __syncthreads();
    p = block_reduce(mx, s, sh);
    if (threadIdx.x == 0) {
        ctl->result = p;
        ctl->done = 0;
    }
}

void set_err(char *err, size_t err_len, const char *msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
}

}  // namespace

extern "C" int asz_error_stats_noalloc(const float *x, const float *y, uint64_t n, double value_range, void *cuda_stream,
                                       double *max_err, double *psnr, char *err, size_t err_len) {
    if (err && err_len) err[0] = '\0';
    if (!x || !y || n == 0) {
        set_err(err, err_len, "error_stats_noalloc: null pointer or empty input");
        return ASZ_E_ARG;
    }
    const uint64_t tiles = (n + kTile - 1) / kTile;
    if (tiles > kMaxTiles) {
        char m[160];
        std::snprintf(m, sizeof(m), "error_stats_noalloc: %llu values exceed the fixed scratch limit of %llu",
                      (unsigned long long)n, (unsigned long long)(kMaxTiles * kTile));
        set_err(err, err_len, m);
        return ASZ_E_ARG;
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        set_err(err, err_len, "error_stats_noalloc: no usable current CUDA device");
        return ASZ_E_CUDA;
    }
    // The array's device address in the current device's context. Host code cannot use the
    // symbol g_stats_scratch itself (it names a host-side shadow), so the address is looked up
    // on every call: the lookup allocates nothing, a failed lookup is not remembered, and a
    // context created after a device reset gets its own address.
    void *sym = nullptr;
    const cudaError_t se = cudaGetSymbolAddress(&sym, g_stats_scratch);
    if (se != cudaSuccess || !sym) {
        char m[160];
        std::snprintf(m, sizeof(m), "error_stats_noalloc: cudaGetSymbolAddress failed for the scratch array: %s",
                      cudaGetErrorString(se));
        set_err(err, err_len, m);
        return ASZ_E_CUDA;
    }
    unsigned char *scratch = (unsigned char *)sym;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    Control h;
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(Control), st);
    if (e == cudaSuccess) {
        stats_noalloc_kernel<<<(unsigned)tiles, kThreads, 0, st>>>(x, y, n, scratch);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, scratch, sizeof(Control), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        char m[160];
        std::snprintf(m, sizeof(m), "error_stats_noalloc: %s", cudaGetErrorString(e));
        set_err(err, err_len, m);
        return ASZ_E_CUDA;
    }
    const double mse = h.result.sse / (double)n;
    if (max_err) *max_err = h.result.max;
    if (psnr) *psnr = 10.0 * std::log10(value_range * value_range / mse);
    return ASZ_OK;
}
