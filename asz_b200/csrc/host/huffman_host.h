// Host side of the Huffman stage: the code of one stream built from its GPU histogram, its
// serialised form, and the parsing of a serialised stream for the GPU decoder.
//
// Follows huffman_encoder_class (c_codes/asz_core/huffman.hpp): leaves in ascending symbol
// order, a min-heap on (frequency, node index) whose first pop becomes the left child, codes
// LSB-first by depth, preorder serialisation, and the 0x1234abcd-masked big-endian length word.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../launch.h"

namespace asz {

struct HuffCode {
    bool usemp = false;
    int64_t offset = 0;       // smallest symbol (after the single-symbol adjustment)
    uint64_t n = 0;           // distinct symbols
    uint64_t maxval = 0;      // symbol range, 1 for a single symbol
    unsigned mbft = 0;        // bits per serialised symbol
    uint64_t count = 0;       // symbols in the stream
    uint64_t bits = 0;        // payload bits
    uint32_t max_len = 0;
    std::vector<CodeEntry> table;   // per symbol index (value - offset), dense over the range
    std::vector<int32_t> left, right;  // tree: nodes [0,n) are leaves, internal nodes follow
    std::vector<uint64_t> leaf_sym;    // symbol index of each leaf
    uint64_t root = 0;

    uint64_t save_size() const;     // header + serialised tree (huffman.hpp:322-332)
    uint64_t encode_size() const;   // length word + payload (huffman.hpp:334-338)
};

// Build the code from a dense histogram over [min_sym, max_sym]. `wide` selects int64 symbol
// semantics (the t stream) instead of int32 (QB streams) for the reference's maxval arithmetic.
bool build_code(const std::vector<uint64_t> &hist, int64_t min_sym, int64_t max_sym, uint64_t count, bool wide,
                HuffCode &out, std::string &err);

// Serialise the header and tree (saveAsDFSOrder, huffman.hpp:650-691) into dst[0, save_size).
void write_tree(const HuffCode &c, uint8_t *dst);
// Length word: total bits (or the count for a single symbol) xor 0x1234abcd, big-endian.
void write_len_word(const HuffCode &c, uint8_t *dst);

// A parsed stream for decoding (loadAsDFSOrder, huffman.hpp:693-783).
struct HuffParsed {
    int64_t offset = 0;
    uint64_t n = 0, maxval = 0;
    unsigned mbft = 0;
    bool single = false;           // one symbol (or maxval == 1): every value equals offset
    uint64_t payload_bits = 0;     // from the length word
    uint64_t single_count = 0;     // from the length word when single
    uint64_t payload_off = 0;      // byte offset of the payload in the stream buffer
    std::vector<LutEntry> lut;
    std::vector<uint32_t> child;   // 2 per internal node
    uint32_t lut_bits = 0;
};

// Parse the tree at buf[pos] and the length word that follows; advances pos past the payload.
bool parse_stream(const uint8_t *buf, uint64_t len, uint64_t &pos, HuffParsed &out, std::string &err);

}  // namespace asz
