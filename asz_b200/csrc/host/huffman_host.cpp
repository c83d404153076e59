// Host side of the Huffman stage (see huffman_host.h).
#include "huffman_host.h"

#include <algorithm>

#include <queue>
#include <utility>

namespace asz {

uint64_t HuffCode::save_size() const {
    uint64_t s = 1 + 8 + 8 + 8;
    if (n > 1) s += (n * (uint64_t)(mbft + 2) - 1 + 7) >> 3;
    return s;
}

uint64_t HuffCode::encode_size() const { return 8 + (maxval == 1 ? 0 : (bits + 7) >> 3); }

bool build_code(const std::vector<uint64_t> &hist, int64_t min_sym, int64_t max_sym, uint64_t count, bool wide,
                HuffCode &c, std::string &err) {
    c = HuffCode();
    c.count = count;
    c.offset = min_sym;
    // huffman.hpp:275-281: maxval = max-min+1 in the symbol type; the usemp flag only changes the
    // first header byte (the map and vector forms build the same tree).
    if (wide) {
        int64_t mv = (int64_t)((uint64_t)max_sym - (uint64_t)min_sym + 1);
        c.maxval = (uint64_t)mv;
        c.usemp = (mv >= (1 << 12) && count < 2ull * (uint64_t)max_sym) || mv >= (1 << 28);
    } else {
        int32_t mv = (int32_t)((uint32_t)(int32_t)max_sym - (uint32_t)(int32_t)min_sym + 1u);
        c.maxval = (uint64_t)(int64_t)mv;
        c.usemp = (mv >= (1 << 12) && count < 2ull * (uint64_t)(int64_t)(int32_t)max_sym) || mv >= (1 << 28);
    }
    std::vector<uint64_t> freq;
    for (uint64_t i = 0; i < hist.size(); i++)
        if (hist[i]) {
            c.leaf_sym.push_back(i);
            freq.push_back(hist[i]);
        }
    c.n = c.leaf_sym.size();
    if (c.n == 0) {
        err = "empty Huffman stream";
        return false;
    }
    c.table.assign(hist.size(), CodeEntry{0, 0});
    if (c.n == 1 || c.maxval == 1) {  // huffman.hpp:193-210
        c.mbft = 1;
        c.maxval = 1;
        c.offset = min_sym + (int64_t)c.leaf_sym[0];
        c.table[c.leaf_sym[0]] = CodeEntry{0, 1};
        c.max_len = 1;
        c.bits = 0;
        return true;
    }
    c.mbft = 1;
    while ((1ull << c.mbft) < c.maxval) ++c.mbft;
    const uint64_t n = c.n;
    c.left.assign(n, -1);
    c.right.assign(n, -1);
    // The reference pops a min-heap on (frequency, node index) (huffman.hpp:222-240). Merged
    // weights come out nondecreasing and internal nodes are numbered after all leaves, so the
    // leaves sorted by (frequency, index) and a FIFO of internal nodes in creation order give
    // the same pops: at each step take the smaller front, the leaf on a frequency tie.
    // Leaves in (frequency, index) order: a stable radix sort on the frequency, one byte per
    // pass over the bytes that are not zero in every frequency, from leaves in index order.
    std::vector<uint32_t> order(n), tmp(n);
    uint64_t maxf = 0;
    for (uint64_t i = 0; i < n; i++) {
        order[i] = (uint32_t)i;
        maxf = std::max(maxf, freq[i]);
    }
    for (unsigned shift = 0; shift < 64 && (maxf >> shift) != 0; shift += 8) {
        uint64_t cnt[257] = {0};
        for (uint64_t i = 0; i < n; i++) cnt[((freq[order[i]] >> shift) & 255u) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (uint64_t i = 0; i < n; i++) tmp[cnt[(freq[order[i]] >> shift) & 255u]++] = order[i];
        order.swap(tmp);
    }
    std::vector<uint64_t> ifreq;
    ifreq.reserve(n);
    uint64_t ia = 0, ib = 0;
    auto pop = [&](uint64_t &node, uint64_t &f) {
        if (ia < n && (ib == ifreq.size() || freq[order[ia]] <= ifreq[ib])) {
            node = order[ia];
            f = freq[order[ia]];
            ia++;
        } else {
            node = n + ib;
            f = ifreq[ib];
            ib++;
        }
    };
    for (uint64_t k = 0; k + 1 < n; k++) {
        uint64_t u, fu, v, fv;
        pop(u, fu);
        pop(v, fv);
        c.left.push_back((int32_t)u);
        c.right.push_back((int32_t)v);
        ifreq.push_back(fu + fv);
    }
    c.root = c.left.size() - 1;
    // dfs_vec (huffman.hpp:80-95): bit k of the code is the branch taken at depth k+1.
    struct Item {
        uint64_t node;
        uint32_t len;
        uint64_t code;
    };
    std::vector<Item> st{{c.root, 0, 0}};
    while (!st.empty()) {
        Item it = st.back();
        st.pop_back();
        if (it.node < n) {
            if (it.len > 32) {
                err = "Huffman code longer than 32 bits";
                return false;
            }
            c.table[c.leaf_sym[it.node]] = CodeEntry{(uint32_t)it.code, it.len};
            c.max_len = std::max(c.max_len, it.len);
            c.bits += freq[it.node] * it.len;
            continue;
        }
        st.push_back({(uint64_t)c.right[it.node], it.len + 1, it.code | (1ull << it.len)});
        st.push_back({(uint64_t)c.left[it.node], it.len + 1, it.code});
    }
    return true;
}

static void put_be64(uint8_t *b, uint64_t v) {
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (56 - 8 * i));
}
static uint64_t get_be64(const uint8_t *b) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | b[i];
    return v;
}

void write_tree(const HuffCode &c, uint8_t *dst) {
    uint8_t *p = dst;
    *p++ = (uint8_t)((c.usemp ? 0x80 : 0) | (c.n == 1 ? 0x40 : 0) | c.mbft);
    uint64_t ob = (uint64_t)c.offset;
    for (int i = 0; i < 8; i++) *p++ = (uint8_t)(ob >> (8 * i));
    put_be64(p, c.n);
    p += 8;
    put_be64(p, c.maxval);
    p += 8;
    if (c.n <= 1) return;
    // Preorder: internal node -> 0, leaf -> 1 followed by mbft bits of its symbol, LSB-first.
    uint64_t nbits = c.n * (uint64_t)(c.mbft + 2) - 1;
    std::fill(p, p + ((nbits + 7) >> 3), 0);
    uint64_t bit = 0;
    auto put = [&](unsigned v) {
        if (v) p[bit >> 3] |= (uint8_t)(1u << (bit & 7));
        bit++;
    };
    std::vector<uint64_t> st{c.root};
    while (!st.empty()) {
        uint64_t u = st.back();
        st.pop_back();
        if (u < c.n) {
            put(1);
            for (unsigned j = 0; j < c.mbft; j++) put((unsigned)((c.leaf_sym[u] >> j) & 1));
        } else {
            put(0);
            st.push_back((uint64_t)c.right[u]);
            st.push_back((uint64_t)c.left[u]);
        }
    }
}

void write_len_word(const HuffCode &c, uint8_t *dst) {
    put_be64(dst, (c.maxval == 1 ? c.count : c.bits) ^ 0x1234abcdull);
}

bool parse_stream(const uint8_t *buf, uint64_t len, uint64_t &pos, HuffParsed &o, std::string &err) {
    o = HuffParsed();
    if (len - pos < 25 || pos > len) {
        err = "truncated Huffman header";
        return false;
    }
    const uint8_t *b = buf + pos;
    o.mbft = b[0] & 0x3f;
    uint64_t ob = 0;
    for (int i = 0; i < 8; i++) ob |= (uint64_t)b[1 + i] << (8 * i);
    o.offset = (int64_t)ob;
    o.n = get_be64(b + 9);
    o.maxval = get_be64(b + 17);
    pos += 25;
    if (o.n == 0) {
        err = "Huffman stream with no symbols";
        return false;
    }
    if (o.n > 1) {
        if (o.mbft == 0 || o.mbft > 63 || o.n > (1ull << 31)) {
            err = "corrupt Huffman tree header";
            return false;
        }
        // Rebuild the tree from its preorder bits, starting after the root's bit.
        struct N {
            int32_t c[2] = {-1, -1};
            int64_t sym = -1;
            uint32_t depth = 0;
        };
        std::vector<N> nodes(1);
        std::vector<int32_t> st{0};
        uint64_t i = 1;
        const uint64_t avail_bits = (len - pos) * 8;
        auto rd = [&](uint64_t k, unsigned &v) {
            if (k >= avail_bits) return false;
            v = (buf[pos + (k >> 3)] >> (k & 7)) & 1;
            return true;
        };
        uint64_t leaves = 0;
        uint32_t max_len = 0;
        while (!st.empty()) {
            int32_t u = st.back();
            unsigned bit;
            if (!rd(i++, bit)) {
                err = "truncated Huffman tree";
                return false;
            }
            N nd;
            nd.depth = nodes[u].depth + 1;
            if (bit == 0) {
                nodes.push_back(nd);
                int32_t id = (int32_t)nodes.size() - 1;
                if (nodes[u].c[0] < 0) nodes[u].c[0] = id;
                else nodes[u].c[1] = id;
                st.push_back(id);
            } else {
                uint64_t s = 0;
                for (unsigned j = 0; j < o.mbft; j++) {
                    unsigned v;
                    if (!rd(i++, v)) {
                        err = "truncated Huffman tree";
                        return false;
                    }
                    s |= (uint64_t)v << j;
                }
                nd.sym = (int64_t)s;
                nodes.push_back(nd);
                int32_t id = (int32_t)nodes.size() - 1;
                if (nodes[u].c[0] < 0) nodes[u].c[0] = id;
                else nodes[u].c[1] = id;
                leaves++;
                max_len = std::max(max_len, nd.depth);
                while (!st.empty() && nodes[st.back()].c[1] >= 0) st.pop_back();
            }
            if (nodes.size() > 2 * o.n + 1 || nd.depth > 40) {
                err = "corrupt Huffman tree";
                return false;
            }
        }
        if (leaves != o.n) {
            err = "Huffman tree does not match its symbol count";
            return false;
        }
        pos += (i + 7) >> 3;
        if (max_len > 32) {
            err = "Huffman code longer than 32 bits";
            return false;
        }
        o.lut_bits = std::min<uint32_t>(max_len, 12);
        o.child.assign(2 * nodes.size(), 0);
        auto ref = [&](int32_t id) -> uint32_t {
            return nodes[id].sym >= 0 ? (0x80000000u | (uint32_t)nodes[id].sym) : (uint32_t)id;
        };
        for (size_t u = 0; u < nodes.size(); u++)
            if (nodes[u].sym < 0) {
                o.child[2 * u] = ref(nodes[u].c[0]);
                o.child[2 * u + 1] = ref(nodes[u].c[1]);
            }
        for (size_t u = 0; u < nodes.size(); u++)
            if (nodes[u].sym >= 0 && (uint64_t)nodes[u].sym >= std::max<uint64_t>(o.maxval, 1) && o.maxval < (1ull << 31)) {
                err = "Huffman symbol outside its range";
                return false;
            }
        o.lut.resize(1ull << o.lut_bits);
        for (uint64_t pre = 0; pre < o.lut.size(); pre++) {
            int32_t u = 0;
            uint32_t l = 0;
            while (l < o.lut_bits && nodes[u].sym < 0) u = nodes[u].c[(pre >> l++) & 1];
            if (nodes[u].sym >= 0) o.lut[pre] = LutEntry{(uint32_t)nodes[u].sym, l};
            else o.lut[pre] = LutEntry{(uint32_t)u, 0};
        }
    } else {
        o.single = true;
    }
    if (len - pos < 8) {
        err = "truncated Huffman payload";
        return false;
    }
    uint64_t w = get_be64(buf + pos) ^ 0x1234abcdull;
    pos += 8;
    if (o.single || o.maxval == 1) {
        o.single = true;
        o.single_count = w;
        o.payload_off = pos;
        return true;
    }
    // Compare in bits first: a corrupt length near 2^64 must not wrap when rounded up to bytes.
    if (w > (len - pos) * 8) {
        err = "truncated Huffman payload";
        return false;
    }
    o.payload_bits = w;
    o.payload_off = pos;
    uint64_t bytes = (w + 7) >> 3;
    if (bytes > len - pos) {
        err = "truncated Huffman payload";
        return false;
    }
    pos += bytes;
    return true;
}

}  // namespace asz
