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
    // A thread takes runs of kHistRun consecutive symbols and adds equal neighbours together:
    // most symbols of a stream are a few values, often repeated, so this saves most atomics.
    constexpr uint32_t kHistRun = 8;
    auto add = [&](uint64_t v, uint32_t c) {
        if (use_sh) atomicAdd(&sh[v], c);
        else atomicAdd(&hist[v], (unsigned long long)c);
    };
    const uint64_t nruns = (n + kHistRun - 1) / kHistRun;
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < nruns; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = r * kHistRun, i1 = min(i0 + kHistRun, n);
        uint64_t cur = (uint64_t)((int64_t)s[i0] - offset);
        uint32_t c = 1;
        for (uint64_t i = i0 + 1; i < i1; i++) {
            const uint64_t v = (uint64_t)((int64_t)s[i] - offset);
            if (v == cur) {
                c++;
            } else {
                add(cur, c);
                cur = v;
                c = 1;
            }
        }
        add(cur, c);
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
// Tiled encoding of several streams in one launch: tiles of enc_tile<T>() symbols, a stream's
// tiles consecutive. A CTA takes tiles in order from a ticket counter and copies the next tile's
// symbols into shared memory (asynchronous copies) while it encodes the current one. Per tile it
// counts the tile's bits, publishes the count, and finds the tile's bit offset in its stream by
// looking back over the tiles before it (decoupled look-back: each tile's state word holds its
// count, then its inclusive prefix); it then builds the tile's bits in shared memory and writes
// them as whole words, with atomicOr only on its first and last word, which it may share with the
// neighbouring tiles. Tiles are handed out in order, so every tile a CTA waits for is held by a
// CTA that is running; every wait is bounded and a wait that runs out sets the error word.

__device__ __forceinline__ uint32_t stream_of(const uint64_t *toff, uint32_t ns, uint64_t t) {
    uint32_t lo = 0, hi = ns;  // toff[lo] <= t < toff[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (toff[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Tile state words: status in the top two bits, bits (count or inclusive prefix) below.
constexpr unsigned long long kTileCount = 1ull << 62, kTilePrefix = 2ull << 62, kTileValue = (1ull << 62) - 1;
constexpr uint32_t kLookbackPolls = 1u << 22;

template <class T>
__device__ __forceinline__ void cp_async_sym(T *dst, const T *src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_older() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <class T>
__global__ void __launch_bounds__(kEncThreads, 4)
    encode_tiles_kernel(const EncStream *__restrict__ S, uint32_t ns, const uint64_t *__restrict__ toff, uint64_t ntiles,
                        unsigned long long *state, unsigned long long *err) {
    constexpr uint32_t kTile = enc_tile<T>(), kPer = kTile / kEncThreads;
    // Symbol i of a tile sits at i + i / kPer: each thread reads its own kPer consecutive symbols,
    // and the one-slot gap between runs spreads a warp's reads over all banks.
    // Dynamic shared memory: two stages of symbols, then the tile's words (codes are at most 32
    // bits, plus the leading shift).
    extern __shared__ __align__(16) unsigned char enc_smem[];
    T(*sym_sh)[kTile + kEncThreads] = reinterpret_cast<T(*)[kTile + kEncThreads]>(enc_smem);
    uint32_t *buf = reinterpret_cast<uint32_t *>(enc_smem + 2 * (kTile + kEncThreads) * sizeof(T));
    __shared__ uint32_t wsum[kEncThreads / 32];
    __shared__ unsigned long long s_next, s_excl;
    unsigned long long *const ticket = state + ntiles;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    // Copies of tile t's symbols into stage b (this thread's share), committed as one group.
    auto issue = [&](uint64_t t, uint32_t b) {
        if (t < ntiles) {
            const uint32_t si = stream_of(toff, ns, t);
            const EncStream &E = S[si];
            const T *sym = reinterpret_cast<const T *>(E.s);
            const uint64_t i0 = (t - toff[si]) * kTile;
            const uint32_t cnt = (uint32_t)min((uint64_t)kTile, E.n - i0);
            for (uint32_t i = tid; i < cnt; i += kEncThreads) cp_async_sym(&sym_sh[b][i + i / kPer], sym + i0 + i);
        }
        cp_async_commit_group();
    };
    if (tid == 0) s_next = atomicAdd(ticket, 1ull);
    __syncthreads();
    uint64_t t = s_next;
    issue(t, 0);
    uint32_t b = 0;
    while (t < ntiles) {
        // Every thread has read s_next and is done with stage b ^ 1 (the tile before this one).
        __syncthreads();
        if (tid == 0) s_next = atomicAdd(ticket, 1ull);
        for (uint32_t i = tid; i < kTile + 2; i += kEncThreads) buf[i] = 0u;
        __syncthreads();
        const uint64_t tn = s_next;
        issue(tn, b ^ 1);
        cp_async_wait_older();
        __syncthreads();  // this tile's symbols, copied by every thread, are in place
        const uint32_t si = stream_of(toff, ns, t);
        const EncStream &E = S[si];
        const uint64_t t0 = toff[si];
        const uint64_t i0 = (t - t0) * kTile;
        const uint32_t cnt = (uint32_t)min((uint64_t)kTile, E.n - i0);
        // This thread's symbols: kPer consecutive ones, so its bits are one consecutive run.
        const uint32_t j0 = tid * kPer;
        uint32_t code[kPer], len[kPer];
        uint32_t mine = 0;
#pragma unroll
        for (uint32_t k = 0; k < kPer; k++) {
            CodeEntry e{0u, 0u};
            if (j0 + k < cnt) e = E.tab[(uint64_t)((int64_t)sym_sh[b][j0 + k + tid] - E.offset)];
            code[k] = e.code;
            len[k] = e.len;
            mine += e.len;
        }
        // Exclusive scan of the threads' bit counts (warp shuffles, then the warps' sums).
        uint32_t incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        if (lane == 31) wsum[tid >> 5] = incl;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < kEncThreads / 32; w++) {
            if (w < (tid >> 5)) before += wsum[w];
            total += wsum[w];
        }
        // Pack the run at bit 0 of the tile's words (the tile's offset in its stream is applied when
        // the words are written, so the packing need not wait for it): the run's first and last
        // words may be shared with the neighbouring runs and are or-ed in; the words between belong
        // to this thread alone.
        const uint32_t pos = before + incl - mine;
        if (mine) {
            uint32_t w = pos >> 5, nacc = pos & 31;
            uint64_t acc = 0;
            bool first = true;
#pragma unroll
            for (uint32_t k = 0; k < kPer; k++) {
                acc |= (uint64_t)code[k] << nacc;
                nacc += len[k];
                if (nacc >= 32) {
                    if (first) atomicOr(&buf[w], (uint32_t)acc);
                    else buf[w] = (uint32_t)acc;
                    first = false;
                    w++;
                    acc >>= 32;
                    nacc -= 32;
                }
            }
            if (nacc) atomicOr(&buf[w], (uint32_t)acc);
        }
        // The tile's bit offset in its stream: publish the count, then add up the counts back to
        // the nearest published prefix (or the stream's first tile).
        if (tid < 32) {
            unsigned long long excl = 0;
            if (t == t0) {
                if (lane == 0) atomicExch(&state[t], kTilePrefix | total);
            } else {
                if (lane == 0) atomicExch(&state[t], kTileCount | total);
                for (int64_t j = (int64_t)t - 1;; j -= 32) {
                    const int64_t pidx = j - (int64_t)lane;
                    unsigned long long v = kTilePrefix;  // before the stream's first tile: prefix 0
                    if (pidx >= (int64_t)t0) {
                        const volatile unsigned long long *w = state + pidx;
                        v = *w;
                        for (uint32_t polls = 0; !(v >> 62) && polls < kLookbackPolls; polls++) {
                            __nanosleep(64);
                            v = *w;
                        }
                        if (!(v >> 62)) {
                            atomicOr(err, 1ull);
                            v = kTilePrefix;
                        }
                    }
                    const uint32_t pref = __ballot_sync(0xffffffffu, (v >> 62) == 2);
                    const uint32_t upto = pref ? (uint32_t)(__ffs(pref) - 1) : 31u;
                    unsigned long long x = lane <= upto ? (v & kTileValue) : 0ull;
                    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                    excl += x;
                    if (pref) break;
                }
                if (lane == 0) atomicExch(&state[t], kTilePrefix | (excl + total));
            }
            if (lane == 0) s_excl = excl;
        }
        __syncthreads();
        // Words out, shifted to the tile's offset: word i takes the high bits of packed word i - 1.
        const uint64_t bit0 = s_excl;
        const uint32_t shift = (uint32_t)(bit0 & 31);
        const uint32_t nw = (shift + total + 31) >> 5;
        uint32_t *out = E.out + (bit0 >> 5);
        for (uint32_t i = tid; i < nw; i += kEncThreads) {
            const uint32_t v = shift ? (buf[i] << shift) | (i ? buf[i - 1] >> (32 - shift) : 0u) : buf[i];
            if (i == 0 || i == nw - 1) {
                if (v) atomicOr(&out[i], v);
            } else {
                out[i] = v;
            }
        }
        t = tn;
        b ^= 1;
    }
    cp_async_wait_older();  // the last committed group (past the end) holds no copies
}

// ---------------------------------------------------------------------------------------------
// Decoding. The host builds a lookup table of 2^lut_bits entries indexed by the next lut_bits
// payload bits (LSB-first): len>0 gives a complete code of that length and its symbol index;
// len==0 means the code is longer, and `node` is the tree node reached after lut_bits bits.
// Longer codes continue through child[2*node+bit] (a value >= 0x80000000 marks a leaf whose
// symbol index is the low bits).

// Bit reader with read-ahead: `buf` holds the next `nb` payload bits (LSB-first) and is topped up
// to at least 32 bits (the longest code) before each codeword from a queue of 32-bit words. The
// queue is fed by 16-byte loads issued one block ahead, so a load's latency overlaps the decoding
// of the ~128 bits before it is needed. `payload` is 16-byte aligned; reads run at most 48 bytes
// past the current position and the stream buffer is padded for that.
struct BitReader {
    const uint4 *p;
    uint64_t idx;      // next 16-byte block to request
    uint4 nxt;         // requested block
    uint64_t c0, c1;   // current block, words consumed from the low end
    uint32_t cw;       // words left in (c0, c1)
    uint64_t buf;
    uint32_t nb;

    __device__ __forceinline__ void load_cur(const uint4 &v) {
        c0 = (uint64_t)v.x | ((uint64_t)v.y << 32);
        c1 = (uint64_t)v.z | ((uint64_t)v.w << 32);
        cw = 4;
    }
    __device__ __forceinline__ uint32_t take() {
        const uint32_t w = (uint32_t)c0;
        c0 = (c0 >> 32) | (c1 << 32);
        c1 >>= 32;
        if (--cw == 0) {
            load_cur(nxt);
            nxt = __ldg(p + idx++);
        }
        return w;
    }
    __device__ __forceinline__ void init(const uint8_t *payload, uint64_t bit) {
        p = reinterpret_cast<const uint4 *>(payload);
        idx = bit >> 7;
        load_cur(__ldg(p + idx));
        nxt = __ldg(p + idx + 1);
        idx += 2;
        for (uint32_t i = (uint32_t)((bit >> 5) & 3); i; i--) take();
        const uint32_t skip = (uint32_t)(bit & 31);
        buf = (uint64_t)(take() >> skip);
        nb = 32 - skip;
        refill();
    }
    __device__ __forceinline__ void refill() {
        if (nb < 32) {
            buf |= (uint64_t)take() << nb;
            nb += 32;
        }
    }
    __device__ __forceinline__ void drop(uint32_t n) {
        buf >>= n;
        nb -= n;
    }
};

// Decode one codeword through the shared-memory table `lut`; returns the symbol index, or
// 0xffffffff for a path that leaves the tree. Advances `bit` by the code length.
__device__ __forceinline__ uint32_t decode_sym(BitReader &br, uint64_t &bit, const LutEntry *lut, uint32_t lut_bits,
                                               const uint32_t *__restrict__ child) {
    br.refill();
    const LutEntry e = lut[br.buf & ((1u << lut_bits) - 1)];
    if (e.len) {
        br.drop(e.len);
        bit += e.len;
        return e.sym;
    }
    uint32_t node = e.sym;
    uint32_t used = lut_bits;
    uint64_t b = br.buf >> lut_bits;
    // Codes are at most 32 bits and the buffer holds at least 32.
    while (true) {
        const uint32_t c = __ldg(child + 2 * node + (uint32_t)(b & 1));
        b >>= 1;
        used++;
        if (c & 0x80000000u) {
            br.drop(used);
            bit += used;
            return c & 0x7fffffffu;
        }
        node = c;
        if (used >= 32) {  // impossible for a validated tree; stop instead of running on
            br.drop(used);
            bit += used;
            return 0xffffffffu;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Batched decoding of every stream of a .asz in one launch per pass. Chunks of chunk_bits bits
// are numbered globally (stream after stream); tiles of blockDim.x chunks never cross a stream,
// so a CTA stages one stream's lookup table for a tile. Bit positions are absolute from the
// 16-byte aligned stream buffer `base`.

__device__ __forceinline__ void stage_lut(LutEntry *lut_sh, const LutEntry *__restrict__ lut, uint32_t lut_bits) {
    for (uint32_t i = threadIdx.x; i < (1u << lut_bits); i += blockDim.x) lut_sh[i] = lut[i];
}

// Pass A over all tiles: chunk k decodes from its start until it reaches the next chunk's first
// bit, recording where it stopped (end[k]) and how many values it produced (count[k]). On the
// first pass the start is the chunk's first bit; later passes start where chunk k-1 ended, and a
// chunk whose start did not move (moved[k] == 0) keeps its end and count without decoding.
__global__ void __launch_bounds__(256)
    decode_sync_kernel(const uint8_t *__restrict__ base, uint64_t chunk_bits, const DecStream *__restrict__ streams,
                       const uint32_t *__restrict__ tile_stream, uint64_t ntiles, const LutEntry *__restrict__ luts,
                       const uint32_t *__restrict__ childs, int first_pass, uint64_t *__restrict__ start,
                       uint64_t *__restrict__ end, uint64_t *__restrict__ count, const uint32_t *__restrict__ moved,
                       uint32_t *err_word) {
    extern __shared__ LutEntry lut_sh[];
    uint32_t staged = 0xffffffffu;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t si = tile_stream[tile];
        const DecStream d = streams[si];
        if (si != staged) {
            __syncthreads();
            stage_lut(lut_sh, luts + d.lut_off, d.lut_bits);
            __syncthreads();
            staged = si;
        }
        const uint64_t kl = (tile - d.tile0) * blockDim.x + threadIdx.x;
        if (kl >= d.nchunks) continue;
        const uint64_t k = d.chunk0 + kl;
        if (!first_pass && !moved[k]) continue;
        uint64_t bit = first_pass ? d.bit_begin + kl * chunk_bits : start[k];
        if (first_pass) start[k] = bit;
        const uint64_t lim = min(d.bit_begin + (kl + 1) * chunk_bits, d.bit_end);
        uint64_t c = 0;
        if (bit < lim) {
            BitReader br;
            br.init(base, bit);
            while (bit < lim) {
                const uint32_t sym = decode_sym(br, bit, lut_sh, d.lut_bits, childs + d.child_off);
                if (sym == 0xffffffffu) {
                    atomicOr(err_word, 8u);
                    break;
                }
                c++;
            }
        }
        end[k] = bit;
        count[k] = c;
    }
}

__device__ __forceinline__ uint32_t stream_of_chunk(const DecStream *__restrict__ streams, uint32_t nstreams, uint64_t k) {
    uint32_t lo = 0, hi = nstreams;  // last stream with chunk0 <= k
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (streams[mid].chunk0 <= k) lo = mid;
        else hi = mid;
    }
    return lo;
}

// After a pass: the start of chunk k (not the first of its stream) becomes end[k-1]. Marks the
// chunks whose start moved (moved[k]) and flags whether any did.
__global__ void decode_restart_kernel(const DecStream *__restrict__ streams, uint32_t nstreams, uint64_t nchunks,
                                      const uint64_t *__restrict__ end, uint64_t *__restrict__ start, uint32_t *__restrict__ moved,
                                      uint32_t *changed) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nchunks; k += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t m = 0;
        if (streams[stream_of_chunk(streams, nstreams, k)].chunk0 != k) {
            const uint64_t s = end[k - 1];
            if (s != start[k]) {
                start[k] = s;
                m = 1;
                *changed = 1u;
            }
        }
        moved[k] = m;
    }
}

// Per stream, once the starts are stable: the values decoded must equal the stream's count and
// the last chunk must end exactly at the payload's last bit. off[] is the exclusive scan of
// count[] over all chunks (nchunks + 1 entries).
__global__ void decode_check_kernel(const DecStream *__restrict__ streams, uint32_t nstreams, const uint64_t *__restrict__ off,
                                    const uint64_t *__restrict__ end, uint32_t *err_word) {
    const uint32_t si = blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= nstreams) return;
    const DecStream d = streams[si];
    const uint64_t got = off[d.chunk0 + d.nchunks] - off[d.chunk0];
    if (got < d.count) atomicOr(err_word, 32u);
    if (got > d.count) atomicOr(err_word, 64u);
    if (end[d.chunk0 + d.nchunks - 1] != d.bit_end) atomicOr(err_word, 128u);
}

// Pass B over all tiles: write the values (symbol index + offset) of chunk k at its offset in its
// stream's output (int64 for the t stream, int32 for QB streams).
__global__ void __launch_bounds__(256)
    decode_write_kernel(const uint8_t *__restrict__ base, uint64_t chunk_bits, const DecStream *__restrict__ streams,
                        const uint32_t *__restrict__ tile_stream, uint64_t ntiles, const LutEntry *__restrict__ luts,
                        const uint32_t *__restrict__ childs, const uint64_t *__restrict__ start,
                        const uint64_t *__restrict__ off, uint32_t *err_word) {
    extern __shared__ LutEntry lut_sh[];
    uint32_t staged = 0xffffffffu;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t si = tile_stream[tile];
        const DecStream d = streams[si];
        if (si != staged) {
            __syncthreads();
            stage_lut(lut_sh, luts + d.lut_off, d.lut_bits);
            __syncthreads();
            staged = si;
        }
        const uint64_t kl = (tile - d.tile0) * blockDim.x + threadIdx.x;
        if (kl >= d.nchunks) continue;
        const uint64_t k = d.chunk0 + kl;
        uint64_t bit = start[k];
        const uint64_t lim = min(d.bit_begin + (kl + 1) * chunk_bits, d.bit_end);
        if (bit >= lim) continue;
        uint64_t o = off[k] - off[d.chunk0];
        BitReader br;
        br.init(base, bit);
        if (d.wide) {
            while (bit < lim) {
                const uint32_t sym = decode_sym(br, bit, lut_sh, d.lut_bits, childs + d.child_off);
                if (sym == 0xffffffffu || o >= d.count) {
                    atomicOr(err_word, 16u);
                    break;
                }
                static_cast<int64_t *>(d.out)[o++] = (int64_t)sym + d.offset;
            }
            continue;
        }
        // int32 values go out four at a time as one 16-byte store once the position is aligned:
        // whole sectors leave the thread instead of one value per store.
        int32_t *out = static_cast<int32_t *>(d.out);
        int32_t b0 = 0, b1 = 0, b2 = 0;
        uint32_t nb = 0;  // values held, to be stored from out + o
        while (bit < lim) {
            const uint32_t sym = decode_sym(br, bit, lut_sh, d.lut_bits, childs + d.child_off);
            if (sym == 0xffffffffu || o + nb >= d.count) {
                atomicOr(err_word, 16u);
                break;
            }
            const int32_t v = (int32_t)((int64_t)sym + d.offset);
            if (nb == 0 && ((uintptr_t)(out + o) & 15u) != 0) {
                out[o++] = v;
            } else if (nb == 3) {
                *reinterpret_cast<int4 *>(out + o) = make_int4(b0, b1, b2, v);
                o += 4;
                nb = 0;
            } else {
                if (nb == 0) b0 = v;
                else if (nb == 1) b1 = v;
                else b2 = v;
                nb++;
            }
        }
        if (nb > 0) out[o] = b0;
        if (nb > 1) out[o + 1] = b1;
        if (nb > 2) out[o + 2] = b2;
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
    uint64_t blocks = std::min<uint64_t>((n + 8 * 256 - 1) / (8 * 256), 148 * 8);
    histogram_kernel<T><<<(unsigned)blocks, 256, sh, st>>>(s, n, offset, range, hist);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Exclusive prefix sums of n 64-bit values (in == out allowed): tiles of kScanTile values, a CTA
// each, scanned in registers and shared memory; the tiles' totals are scanned the same way (in
// tmp, a level per kScanTile-fold reduction), then added back to their tiles.
constexpr uint32_t kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads)
    scan_tiles_kernel(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *tile_sums) {
    __shared__ uint64_t wsum[kScanThreads / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t first = (uint64_t)blockIdx.x * kScanTile + (uint64_t)tid * kScanPer;
    uint64_t v[kScanPer], mine = 0;
#pragma unroll
    for (uint32_t k = 0; k < kScanPer; k++) {
        v[k] = first + k < n ? in[first + k] : 0;
        mine += v[k];
    }
    uint64_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint64_t w = wsum[lane];
        uint64_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (uint32_t)o) wi += t;
        }
        wsum[lane] = wi - w;
    }
    __syncthreads();
    uint64_t run = wsum[warp] + incl - mine;
#pragma unroll
    for (uint32_t k = 0; k < kScanPer; k++) {
        if (first + k < n) out[first + k] = run;
        run += v[k];
    }
    if (tile_sums && tid == kScanThreads - 1) tile_sums[blockIdx.x] = run;  // the tile's total
}

__global__ void scan_add_kernel(uint64_t *out, uint64_t n, const uint64_t *__restrict__ tile_offsets) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] += tile_offsets[i / kScanTile];
}

static uint64_t scan_tmp_words(uint64_t n) {
    uint64_t w = 0;
    while (n > kScanTile) {
        n = (n + kScanTile - 1) / kScanTile;
        w += n;
    }
    return w;
}

static cudaError_t scan_u64_levels(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *tmp, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    uint64_t *sums = tiles > 1 ? tmp : nullptr;
    scan_tiles_kernel<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, sums);
    count_launch();
    if (tiles > 1) {
        cudaError_t e = scan_u64_levels(sums, sums, tiles, tmp + tiles, st);
        if (e != cudaSuccess) return e;
        scan_add_kernel<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(out, n, sums);
        count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, void *tmp, size_t &tmp_bytes, cudaStream_t st) {
    if (tmp == nullptr) {
        tmp_bytes = std::max<size_t>(scan_tmp_words(n) * sizeof(uint64_t), 16);
        return cudaSuccess;
    }
    if (tmp_bytes < scan_tmp_words(n) * sizeof(uint64_t)) return cudaErrorInvalidValue;
    return scan_u64_levels(in, out, n, reinterpret_cast<uint64_t *>(tmp), st);
}

template <class T>
cudaError_t launch_encode(const T *s, uint64_t n, int64_t offset, const CodeEntry *tab, uint64_t *bitoff, void *tmp,
                          size_t &tmp_bytes, uint32_t *out, cudaStream_t st) {
    if (tmp == nullptr) return launch_scan_u64(bitoff, bitoff, n, nullptr, tmp_bytes, st);
    if (n == 0) return cudaSuccess;
    uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    code_len_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(s, n, offset, tab, bitoff);
    count_launch();
    cudaError_t e = launch_scan_u64(bitoff, bitoff, n, tmp, tmp_bytes, st);
    if (e != cudaSuccess) return e;
    encode_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(s, n, offset, tab, bitoff, out);
    count_launch();
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_encode_tiles(const EncStream *streams, uint32_t ns, const uint64_t *toff, uint64_t ntiles, uint64_t *tile_state,
                                uint64_t *err, void *tmp, size_t &tmp_bytes, cudaStream_t st) {
    if (tmp == nullptr) {
        tmp_bytes = 0;
        return cudaSuccess;
    }
    if (ntiles == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(tile_state, 0, (ntiles + 1) * sizeof(uint64_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(uint64_t), st);
    if (e != cudaSuccess) return e;
    constexpr uint32_t kTile = enc_tile<T>();
    const int smem = (int)(2 * (kTile + kEncThreads) * sizeof(T) + (kTile + 2) * sizeof(uint32_t));
    e = cudaFuncSetAttribute(encode_tiles_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, 148 * 4);
    encode_tiles_kernel<T><<<grid, kEncThreads, smem, st>>>(streams, ns, toff, ntiles, (unsigned long long *)tile_state,
                                                            (unsigned long long *)err);
    count_launch();
    return cudaGetLastError();
}

template cudaError_t launch_encode_tiles<int32_t>(const EncStream *, uint32_t, const uint64_t *, uint64_t, uint64_t *, uint64_t *,
                                                  void *, size_t &, cudaStream_t);
template cudaError_t launch_encode_tiles<int64_t>(const EncStream *, uint32_t, const uint64_t *, uint64_t, uint64_t *, uint64_t *,
                                                  void *, size_t &, cudaStream_t);

// Persistent decode grid: up to 6 CTAs of 256 threads per SM (a table takes up to 32 KB).
static unsigned decode_grid(uint64_t ntiles) { return (unsigned)(ntiles < 148 * 6 ? (ntiles ? ntiles : 1) : 148 * 6); }

cudaError_t launch_decode_sync(const uint8_t *base, uint64_t chunk_bits, const DecStream *streams, const uint32_t *tile_stream,
                               uint64_t ntiles, uint32_t max_lut_bits, const LutEntry *luts, const uint32_t *childs,
                               int first_pass, uint64_t *start, uint64_t *end, uint64_t *count, const uint32_t *moved,
                               uint32_t *err, cudaStream_t st) {
    const size_t sh = ((size_t)1 << max_lut_bits) * sizeof(LutEntry);
    decode_sync_kernel<<<decode_grid(ntiles), kDecodeTile, sh, st>>>(base, chunk_bits, streams, tile_stream, ntiles, luts,
                                                                      childs, first_pass, start, end, count, moved, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_restart(const DecStream *streams, uint32_t nstreams, uint64_t nchunks, const uint64_t *end,
                                  uint64_t *start, uint32_t *moved, uint32_t *changed, cudaStream_t st) {
    const uint64_t b = (nchunks + 255) / 256;
    decode_restart_kernel<<<(unsigned)(b < 148 * 8 ? (b ? b : 1) : 148 * 8), 256, 0, st>>>(streams, nstreams, nchunks, end, start,
                                                                                         moved, changed);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_check(const DecStream *streams, uint32_t nstreams, const uint64_t *off, const uint64_t *end,
                                uint32_t *err, cudaStream_t st) {
    decode_check_kernel<<<(nstreams + 63) / 64, 64, 0, st>>>(streams, nstreams, off, end, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_decode_write(const uint8_t *base, uint64_t chunk_bits, const DecStream *streams, const uint32_t *tile_stream,
                                uint64_t ntiles, uint32_t max_lut_bits, const LutEntry *luts, const uint32_t *childs,
                                const uint64_t *start, const uint64_t *off, uint32_t *err, cudaStream_t st) {
    const size_t sh = ((size_t)1 << max_lut_bits) * sizeof(LutEntry);
    decode_write_kernel<<<decode_grid(ntiles), kDecodeTile, sh, st>>>(base, chunk_bits, streams, tile_stream, ntiles, luts, childs,
                                                                       start, off, err);
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
template cudaError_t launch_fill<int32_t>(int32_t *, uint64_t, int32_t, cudaStream_t);
template cudaError_t launch_fill<int64_t>(int64_t *, uint64_t, int64_t, cudaStream_t);

}  // namespace asz
