// Huffman stage on the GPU: symbol histograms, encoding into the reference's LSB-first bit
// layout (c_codes/asz_core/huffman.hpp:340-381, 610-632), and decoding of that layout.
//
// The reference decodes serially (huffman.hpp:383-526). Here the payload is cut into chunks
// of a fixed number of bits, and one thread decodes each chunk from a guessed codeword boundary.
// Huffman codes resynchronise after a few codewords, so a chunk decoded from the true start of
// its predecessor's last codeword ends at the same place as the guess. Passes repeat until no
// chunk start changes. A final pass writes the symbols at offsets from a scan of per-chunk counts.
// Every loop is bounded by the chunk length plus the longest code.
#include <cuda_runtime.h>

#include <algorithm>

#include <cub/device/device_scan.cuh>

#include "dev_common.cuh"
#include "launch.h"

namespace asz {

// ---------------------------------------------------------------------------------------------
// Histogram of symbols in [offset, offset+range). Counts are 64-bit.
template <class T>
__global__ void histogram_kernel(const T *__restrict__ s, uint64_t n, int64_t offset, uint64_t range,
                                 unsigned long long *__restrict__ hist) {
    extern __shared__ unsigned int sh[];
    const bool use_sh = range <= 8192;
    if (use_sh) {
        for (uint64_t i = threadIdx.x; i < range; i += blockDim.x) sh[i] = 0;
        __syncthreads();
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t v = (uint64_t)((int64_t)s[i] - offset);
        if (use_sh) atomicAdd(&sh[v], 1u);
        else atomicAdd(&hist[v], 1ull);
    }
    if (use_sh) {
        __syncthreads();
        for (uint64_t i = threadIdx.x; i < range; i += blockDim.x)
            if (sh[i]) atomicAdd(&hist[i], (unsigned long long)sh[i]);
    }
}

// Code table entries (launch.h): length in bits and the code, LSB-first (bit k = branch at depth k+1).

template <class T>
__global__ void code_len_kernel(const T *__restrict__ s, uint64_t n, int64_t offset, const CodeEntry *__restrict__ tab,
                                uint64_t *__restrict__ len) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        len[i] = tab[(uint64_t)((int64_t)s[i] - offset)].len;
}

// Writes each symbol's code at its bit offset. out is zero-initialised; codes are <= 32 bits.
template <class T>
__global__ void encode_kernel(const T *__restrict__ s, uint64_t n, int64_t offset, const CodeEntry *__restrict__ tab,
                              const uint64_t *__restrict__ bitoff, uint32_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        CodeEntry e = tab[(uint64_t)((int64_t)s[i] - offset)];
        uint64_t o = bitoff[i];
        uint64_t v = (uint64_t)e.code << (o & 31);
        uint64_t w = o >> 5;
        if ((uint32_t)v) atomicOr(&out[w], (uint32_t)v);
        if ((o & 31) + e.len > 32 && (uint32_t)(v >> 32)) atomicOr(&out[w + 1], (uint32_t)(v >> 32));
    }
}

// ---------------------------------------------------------------------------------------------
// Decoding. The host builds a lookup table of 2^lut_bits entries indexed by the next lut_bits
// payload bits (LSB-first): len>0 gives a complete code of that length and its symbol index;
// len==0 means the code is longer, and `node` is the tree node reached after lut_bits bits.
// Longer codes continue through child[2*node+bit] (a value >= 0x80000000 marks a leaf whose
// symbol index is the low bits).

__device__ __forceinline__ uint64_t peek64(const uint8_t *__restrict__ p, uint64_t bit) {
    // Little-endian 64-bit window starting at `bit`; the buffer is padded by 16 bytes.
    const uint64_t byte = bit >> 3;
    const uint32_t *w = (const uint32_t *)(p + (byte & ~3ull));
    uint64_t lo = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
    uint64_t hi = (uint64_t)w[2];
    uint32_t sh = (uint32_t)((byte & 3) * 8 + (bit & 7));
    return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
}

// Decode one codeword at `bit`; returns its symbol index and advances `bit`.
__device__ __forceinline__ uint32_t decode_one(const uint8_t *__restrict__ p, uint64_t &bit, DecodeTables dt) {
    uint64_t win = peek64(p, bit);
    LutEntry e = dt.lut[win & ((1u << dt.lut_bits) - 1)];
    if (e.len) {
        bit += e.len;
        return e.sym;
    }
    uint32_t node = e.sym;
    uint32_t used = dt.lut_bits;
    win >>= dt.lut_bits;
    // Codes are at most 32 bits, so the 64-bit window always holds the rest.
    while (true) {
        uint32_t c = dt.child[2 * node + (uint32_t)(win & 1)];
        win >>= 1;
        used++;
        if (c & 0x80000000u) {
            bit += used;
            return c & 0x7fffffffu;
        }
        node = c;
        if (used > 40) {  // impossible for a validated tree; stop instead of running on
            bit += used;
            return 0xffffffffu;
        }
    }
}

// Pass A: each chunk decodes from start[k] until it reaches the next chunk's start bit and
// records where it stopped (end[k]) and how many symbols it produced (count[k]).
// Bit positions are absolute from the 4-byte-aligned `payload` base: the stream occupies
// [bit_begin, bit_end) and chunk k covers [bit_begin + k*chunk_bits, bit_begin + (k+1)*chunk_bits).
__global__ void decode_sync_kernel(const uint8_t *__restrict__ payload, uint64_t bit_begin, uint64_t bit_end,
                                   uint64_t chunk_bits, uint64_t nchunks, DecodeTables dt, const uint64_t *__restrict__ start,
                                   uint64_t *__restrict__ end, uint64_t *__restrict__ count, uint32_t *err_word) {
    uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= nchunks) return;
    uint64_t bit = start[k];
    const uint64_t lim = min(bit_begin + (k + 1) * chunk_bits, bit_end);
    uint64_t c = 0;
    while (bit < lim) {
        uint32_t s = decode_one(payload, bit, dt);
        if (s == 0xffffffffu) {
            atomicOr(err_word, 8u);
            break;
        }
        c++;
    }
    end[k] = bit;
    count[k] = c;
}

// After a pass: the next start of chunk k+1 is end[k]. Flags whether anything moved.
__global__ void decode_restart_kernel(uint64_t nchunks, const uint64_t *__restrict__ end, uint64_t *__restrict__ start,
                                      uint32_t *changed) {
    uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k == 0 || k >= nchunks) return;
    uint64_t s = end[k - 1];
    if (s != start[k]) {
        start[k] = s;
        *changed = 1u;
    }
}

// Pass B: write symbols (value = index + offset) at out[off[k] ...].
template <class T>
__global__ void decode_write_kernel(const uint8_t *__restrict__ payload, uint64_t bit_begin, uint64_t bit_end,
                                    uint64_t chunk_bits, uint64_t nchunks, DecodeTables dt, int64_t offset,
                                    const uint64_t *__restrict__ start, const uint64_t *__restrict__ off, T *__restrict__ out,
                                    uint64_t nout, uint32_t *err_word) {
    uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= nchunks) return;
    uint64_t bit = start[k];
    const uint64_t lim = min(bit_begin + (k + 1) * chunk_bits, bit_end);
    uint64_t o = off[k];
    while (bit < lim) {
        uint32_t s = decode_one(payload, bit, dt);
        if (s == 0xffffffffu || o >= nout) {
            atomicOr(err_word, 16u);
            break;
        }
        out[o++] = (T)((int64_t)s + offset);
    }
}

template <class T>
__global__ void fill_kernel(T *__restrict__ out, uint64_t n, T v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) out[i] = v;
}

// ---------------------------------------------------------------------------------------------
// Host-callable launchers (declared in launch.h).

template <class T>
cudaError_t launch_histogram(const T *s, uint64_t n, int64_t offset, uint64_t range, unsigned long long *hist,
                             cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    size_t sh = range <= 8192 ? range * sizeof(unsigned int) : 0;
    uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 8);
    histogram_kernel<T><<<(unsigned)blocks, 256, sh, st>>>(s, n, offset, range, hist);
    count_launch();
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_encode(const T *s, uint64_t n, int64_t offset, const CodeEntry *tab, uint64_t *bitoff, void *tmp,
                          size_t &tmp_bytes, uint32_t *out, cudaStream_t st) {
    if (tmp == nullptr) return cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, bitoff, bitoff, (int64_t)n, st);
    if (n == 0) return cudaSuccess;
    uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    code_len_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(s, n, offset, tab, bitoff);
    count_launch();
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, bitoff, bitoff, (int64_t)n, st);
    if (e != cudaSuccess) return e;
    encode_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(s, n, offset, tab, bitoff, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, void *tmp, size_t &tmp_bytes, cudaStream_t st) {
    if (tmp == nullptr) return cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, (int64_t)n, st);
    return cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, (int64_t)n, st);
}

cudaError_t launch_decode_sync(const uint8_t *payload, uint64_t bit_begin, uint64_t bit_end, uint64_t chunk_bits,
                               uint64_t nchunks, DecodeTables dt, const uint64_t *start, uint64_t *end, uint64_t *count,
                               uint32_t *err, cudaStream_t st) {
    decode_sync_kernel<<<(unsigned)((nchunks + 127) / 128), 128, 0, st>>>(payload, bit_begin, bit_end, chunk_bits, nchunks,
                                                                           dt, start, end, count, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_restart(uint64_t nchunks, const uint64_t *end, uint64_t *start, uint32_t *changed,
                                  cudaStream_t st) {
    decode_restart_kernel<<<(unsigned)((nchunks + 255) / 256), 256, 0, st>>>(nchunks, end, start, changed);
    count_launch();
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_decode_write(const uint8_t *payload, uint64_t bit_begin, uint64_t bit_end, uint64_t chunk_bits,
                                uint64_t nchunks, DecodeTables dt, int64_t offset, const uint64_t *start, const uint64_t *off,
                                T *out, uint64_t nout, uint32_t *err, cudaStream_t st) {
    decode_write_kernel<T><<<(unsigned)((nchunks + 127) / 128), 128, 0, st>>>(payload, bit_begin, bit_end, chunk_bits,
                                                                               nchunks, dt, offset, start, off, out, nout, err);
    count_launch();
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_fill(T *out, uint64_t n, T v, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    fill_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(out, n, v);
    count_launch();
    return cudaGetLastError();
}

template cudaError_t launch_histogram<int32_t>(const int32_t *, uint64_t, int64_t, uint64_t, unsigned long long *, cudaStream_t);
template cudaError_t launch_histogram<int64_t>(const int64_t *, uint64_t, int64_t, uint64_t, unsigned long long *, cudaStream_t);
template cudaError_t launch_encode<int32_t>(const int32_t *, uint64_t, int64_t, const CodeEntry *, uint64_t *, void *, size_t &,
                                            uint32_t *, cudaStream_t);
template cudaError_t launch_encode<int64_t>(const int64_t *, uint64_t, int64_t, const CodeEntry *, uint64_t *, void *, size_t &,
                                            uint32_t *, cudaStream_t);
template cudaError_t launch_decode_write<int32_t>(const uint8_t *, uint64_t, uint64_t, uint64_t, uint64_t, DecodeTables,
                                                  int64_t, const uint64_t *, const uint64_t *, int32_t *, uint64_t, uint32_t *,
                                                  cudaStream_t);
template cudaError_t launch_decode_write<int64_t>(const uint8_t *, uint64_t, uint64_t, uint64_t, uint64_t, DecodeTables,
                                                  int64_t, const uint64_t *, const uint64_t *, int64_t *, uint64_t, uint32_t *,
                                                  cudaStream_t);
template cudaError_t launch_fill<int32_t>(int32_t *, uint64_t, int32_t, cudaStream_t);
template cudaError_t launch_fill<int64_t>(int64_t *, uint64_t, int64_t, cudaStream_t);

}  // namespace asz
