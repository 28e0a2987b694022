// Lossless WebP (VP8L) decoder for the SOG images, written from the published
// WebP lossless bitstream format (RFC 9649): LSB-first bit reader, canonical
// prefix codes (simple and normal, code-length codes with repeats), color
// cache, LZ77 backward references with the 2-D distance map, meta prefix
// codes, and the four inverse transforms (predictor, cross-color, subtract
// green, color indexing).  Containers: RIFF/WEBP with a VP8L chunk (simple or
// behind VP8X and other chunks) and a raw VP8L bitstream.  Lossy (VP8)
// images are not decoded: SOG writes its images lossless.
//
// The SOG loader reads its images with WebPGetInfo + WebPDecodeRGBA
// (src/gaussian_loader_sog.cpp:98-124); webp_decode_rgba returns the same
// RGBA8 pixels for every lossless image those accept.
#include "gs_webp.h"

#include <algorithm>
#include <cstring>
#include <new>

namespace gs {
namespace {

uint32_t le32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

// LSB-first bit reader; reads past the end return zeros and mark the stream
// as overrun (an error once decoding ends).
struct Bits {
    const uint8_t* p;
    size_t n;
    uint64_t pos = 0;   // bits consumed
    Bits(const uint8_t* data, size_t size) : p(data), n(size) {}
    // the next `count` (<= 32) bits: one 8-byte window (zeros past the end)
    uint32_t peek(int count) const {
        const uint64_t byte = pos >> 3;
        uint64_t w = 0;
        if (byte + 8 <= n) {
            std::memcpy(&w, p + byte, 8);
        } else if (byte < n) {
            std::memcpy(&w, p + byte, (size_t)(n - byte));
        }
        w >>= (pos & 7);
        return count >= 32 ? (uint32_t)w : (uint32_t)(w & ((1ull << count) - 1));
    }
    uint32_t read(int count) {
        const uint32_t v = peek(count);
        pos += (uint64_t)count;
        return v;
    }
    bool overrun() const { return pos > (uint64_t)n * 8; }
};

constexpr int kMaxLength = 15;
constexpr int kTableBits = 8;

// Canonical prefix code over one alphabet.  A code with a single used
// symbol takes no bits.
struct Prefix {
    bool single = false;
    int single_symbol = 0;
    // first-level table on the next kTableBits stream bits: symbol << 4 | length, or 0 for longer codes
    std::vector<uint32_t> table;
    int first_code[kMaxLength + 2] = {};
    int count[kMaxLength + 1] = {};
    int offset[kMaxLength + 2] = {};
    std::vector<int> sorted;

    bool build(const std::vector<uint8_t>& lengths) {
        std::fill(count, count + kMaxLength + 1, 0);
        int used = 0, last = 0;
        for (size_t s = 0; s < lengths.size(); ++s) {
            if (lengths[s]) {
                ++count[lengths[s]];
                ++used;
                last = (int)s;
            }
        }
        if (used == 0) return false;
        if (used == 1) {
            single = true;
            single_symbol = last;
            return true;
        }
        // complete and not over-subscribed
        int left = 1;
        for (int l = 1; l <= kMaxLength; ++l) {
            left <<= 1;
            left -= count[l];
            if (left < 0) return false;
        }
        if (left != 0) return false;
        offset[1] = 0;
        for (int l = 1; l <= kMaxLength; ++l) offset[l + 1] = offset[l] + count[l];
        sorted.assign((size_t)used, 0);
        int next[kMaxLength + 2];
        std::copy(offset, offset + kMaxLength + 2, next);
        for (size_t s = 0; s < lengths.size(); ++s)
            if (lengths[s]) sorted[(size_t)next[lengths[s]]++] = (int)s;
        int code = 0;
        for (int l = 1; l <= kMaxLength; ++l) {
            first_code[l] = code;
            code = (code + count[l]) << 1;
        }
        // fast table: codes of length <= kTableBits, indexed by their bits in stream order
        table.assign((size_t)1 << kTableBits, 0u);
        for (int l = 1; l <= kTableBits; ++l) {
            for (int k = 0; k < count[l]; ++k) {
                const int c = first_code[l] + k;
                uint32_t rev = 0;
                for (int b = 0; b < l; ++b) rev |= (uint32_t)((c >> (l - 1 - b)) & 1) << b;
                const uint32_t entry = (uint32_t)sorted[(size_t)(offset[l] + k)] << 4 | (uint32_t)l;
                for (uint32_t hi = 0; hi < (1u << (kTableBits - l)); ++hi) table[rev | hi << l] = entry;
            }
        }
        return true;
    }

    int read(Bits& br) const {
        if (single) return single_symbol;
        const uint32_t e = table[br.peek(kTableBits)];
        if (e) {
            br.pos += e & 15u;
            return (int)(e >> 4);
        }
        int code = 0;
        for (int l = 1; l <= kMaxLength; ++l) {
            code = code << 1 | (int)br.read(1);
            const int k = code - first_code[l];
            if (k < count[l]) return sorted[(size_t)(offset[l] + k)];
        }
        return 0;   // unreachable for a complete code
    }
};

const int kCodeLengthOrder[19] = {17, 18, 0, 1, 2, 3, 4, 5, 16, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};

bool read_code(Bits& br, int alphabet, Prefix& out) {
    std::vector<uint8_t> lengths((size_t)alphabet, 0);
    if (br.read(1)) {   // simple code: one or two symbols, length 1
        const int symbols = (int)br.read(1) + 1;
        const int first_bits = br.read(1) ? 8 : 1;
        const int s0 = (int)br.read(first_bits);
        if (s0 < alphabet) lengths[(size_t)s0] = 1;
        if (symbols == 2) {
            const int s1 = (int)br.read(8);
            if (s1 < alphabet) lengths[(size_t)s1] = 1;
        }
    } else {
        std::vector<uint8_t> cl(19, 0);
        const int num = 4 + (int)br.read(4);
        for (int i = 0; i < num; ++i) cl[(size_t)kCodeLengthOrder[i]] = (uint8_t)br.read(3);
        Prefix lc;
        if (!lc.build(cl)) return false;
        int max_symbol = alphabet;
        if (br.read(1)) {
            const int nbits = 2 + 2 * (int)br.read(3);
            max_symbol = 2 + (int)br.read(nbits);
            if (max_symbol > alphabet) return false;
        }
        int symbol = 0, prev = 8;
        while (symbol < alphabet) {
            if (max_symbol-- == 0) break;
            const int len = lc.read(br);
            if (len < 16) {
                lengths[(size_t)symbol++] = (uint8_t)len;
                if (len) prev = len;
            } else {
                const int slot = len - 16;
                static const int extra[3] = {2, 3, 7}, base[3] = {3, 3, 11};
                const int repeat = (int)br.read(extra[slot]) + base[slot];
                if (symbol + repeat > alphabet) return false;
                const uint8_t v = (uint8_t)(len == 16 ? prev : 0);
                for (int r = 0; r < repeat; ++r) lengths[(size_t)symbol++] = v;
            }
        }
    }
    if (br.overrun()) return false;
    return out.build(lengths);
}

// LZ77 length or distance from its prefix symbol.
uint32_t copy_value(Bits& br, int symbol) {
    if (symbol < 4) return (uint32_t)symbol + 1;
    const int extra = (symbol - 2) >> 1;
    const uint32_t offset = (uint32_t)(2 + (symbol & 1)) << extra;
    return offset + br.read(extra) + 1;
}

// The 120 short 2-D distances (dx, dy) of distance codes 1..120.
const int8_t kPlane[120][2] = {
    {0, 1}, {1, 0}, {1, 1}, {-1, 1}, {0, 2}, {2, 0}, {1, 2}, {-1, 2}, {2, 1}, {-2, 1}, {2, 2}, {-2, 2},
    {0, 3}, {3, 0}, {1, 3}, {-1, 3}, {3, 1}, {-3, 1}, {2, 3}, {-2, 3}, {3, 2}, {-3, 2}, {0, 4}, {4, 0},
    {1, 4}, {-1, 4}, {4, 1}, {-4, 1}, {3, 3}, {-3, 3}, {2, 4}, {-2, 4}, {4, 2}, {-4, 2}, {0, 5}, {3, 4},
    {-3, 4}, {4, 3}, {-4, 3}, {5, 0}, {1, 5}, {-1, 5}, {5, 1}, {-5, 1}, {2, 5}, {-2, 5}, {5, 2}, {-5, 2},
    {4, 4}, {-4, 4}, {3, 5}, {-3, 5}, {5, 3}, {-5, 3}, {0, 6}, {6, 0}, {1, 6}, {-1, 6}, {6, 1}, {-6, 1},
    {2, 6}, {-2, 6}, {6, 2}, {-6, 2}, {4, 5}, {-4, 5}, {5, 4}, {-5, 4}, {3, 6}, {-3, 6}, {6, 3}, {-6, 3},
    {0, 7}, {7, 0}, {1, 7}, {-1, 7}, {5, 5}, {-5, 5}, {7, 1}, {-7, 1}, {4, 6}, {-4, 6}, {6, 4}, {-6, 4},
    {2, 7}, {-2, 7}, {7, 2}, {-7, 2}, {3, 7}, {-3, 7}, {7, 3}, {-7, 3}, {5, 6}, {-5, 6}, {6, 5}, {-6, 5},
    {8, 0}, {4, 7}, {-4, 7}, {7, 4}, {-7, 4}, {8, 1}, {8, 2}, {6, 6}, {-6, 6}, {8, 3}, {5, 7}, {-5, 7},
    {7, 5}, {-7, 5}, {8, 4}, {6, 7}, {-6, 7}, {7, 6}, {-7, 6}, {8, 5}, {7, 7}, {-7, 7}, {8, 6}, {8, 7},
};

uint32_t plane_distance(uint32_t xsize, uint32_t code) {
    if (code > 120) return code - 120;
    const int64_t d = (int64_t)kPlane[code - 1][0] + (int64_t)kPlane[code - 1][1] * (int64_t)xsize;
    return d >= 1 ? (uint32_t)d : 1u;
}

struct Group {
    Prefix green, red, blue, alpha, dist;
};

uint32_t div_round_up(uint32_t a, uint32_t bits) { return (a + (1u << bits) - 1) >> bits; }

// One entropy-coded image of xsize x ysize ARGB pixels.  `main` images may
// carry meta prefix codes.
bool read_image(Bits& br, uint32_t xsize, uint32_t ysize, bool main, std::vector<uint32_t>& out) {
    int cache_bits = 0;
    if (br.read(1)) {
        cache_bits = (int)br.read(4);
        if (cache_bits < 1 || cache_bits > 11) return false;
    }
    uint32_t prefix_bits = 0, groups_x = 0;
    std::vector<uint32_t> meta;
    int num_groups = 1;
    if (main && br.read(1)) {
        prefix_bits = br.read(3) + 2;
        groups_x = div_round_up(xsize, prefix_bits);
        std::vector<uint32_t> entropy;
        if (!read_image(br, groups_x, div_round_up(ysize, prefix_bits), false, entropy)) return false;
        meta.resize(entropy.size());
        for (size_t i = 0; i < entropy.size(); ++i) {
            meta[i] = (entropy[i] >> 8) & 0xffffu;
            num_groups = std::max(num_groups, (int)meta[i] + 1);
        }
    }
    if (br.overrun()) return false;
    const int cache_size = cache_bits ? 1 << cache_bits : 0;
    std::vector<Group> groups((size_t)num_groups);
    for (Group& g : groups) {
        if (!read_code(br, 256 + 24 + cache_size, g.green) || !read_code(br, 256, g.red) ||
            !read_code(br, 256, g.blue) || !read_code(br, 256, g.alpha) || !read_code(br, 40, g.dist))
            return false;
    }
    const uint64_t total = (uint64_t)xsize * ysize;
    // grown pixel by pixel within reserved space: a stream that ends early
    // never touches the pages of the size its header declared
    out.clear();
    out.reserve((size_t)total);
    std::vector<uint32_t> cache((size_t)cache_size, 0u);
    const int cache_shift = 32 - cache_bits;
    // every decoded pixel enters the color cache, in order
    auto emit = [&](uint32_t argb) {
        out.push_back(argb);
        if (cache_bits) cache[(0x1e35a7bdu * argb) >> cache_shift] = argb;
    };
    uint64_t pos = 0;
    uint32_t x = 0, y = 0;
    while (pos < total) {
        const Group& g = meta.empty() ? groups[0]
                                      : groups[meta[(size_t)((y >> prefix_bits) * groups_x + (x >> prefix_bits))]];
        const int code = g.green.read(br);
        uint32_t advance = 1;
        if (code < 256) {
            const uint32_t r = (uint32_t)g.red.read(br), b = (uint32_t)g.blue.read(br), a = (uint32_t)g.alpha.read(br);
            emit(a << 24 | r << 16 | (uint32_t)code << 8 | b);
        } else if (code < 256 + 24) {
            const uint32_t length = copy_value(br, code - 256);
            const int dsym = g.dist.read(br);
            const uint32_t dist = plane_distance(xsize, copy_value(br, dsym));
            if (br.overrun() || dist > pos || length > total - pos) return false;
            for (uint32_t k = 0; k < length; ++k) emit(out[(size_t)(pos + k - dist)]);
            advance = length;
        } else {
            if (!cache_bits) return false;
            emit(cache[(size_t)(code - 280)]);
        }
        pos += advance;
        x += advance;
        if (x >= xsize) {
            y += x / xsize;
            x %= xsize;
        }
        if (br.overrun()) return false;
    }
    return !br.overrun();
}

uint32_t add_pixels(uint32_t a, uint32_t b) {
    const uint32_t ag = (a & 0xff00ff00u) + (b & 0xff00ff00u);
    const uint32_t rb = (a & 0x00ff00ffu) + (b & 0x00ff00ffu);
    return (ag & 0xff00ff00u) | (rb & 0x00ff00ffu);
}
uint32_t average2(uint32_t a, uint32_t b) { return (((a ^ b) & 0xfefefefeu) >> 1) + (a & b); }
int chan(uint32_t p, int s) { return (int)((p >> s) & 0xffu); }
int clip255(int v) { return v < 0 ? 0 : v > 255 ? 255 : v; }

uint32_t select_pred(uint32_t L, uint32_t T, uint32_t TL) {
    int pl = 0, pt = 0;
    for (int s = 0; s < 32; s += 8) {
        pl += std::abs(chan(T, s) - chan(TL, s));   // |estimate - L| per channel
        pt += std::abs(chan(L, s) - chan(TL, s));   // |estimate - T| per channel
    }
    return pl < pt ? L : T;
}
uint32_t clamp_full(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r = 0;
    for (int s = 0; s < 32; s += 8) r |= (uint32_t)clip255(chan(a, s) + chan(b, s) - chan(c, s)) << s;
    return r;
}
uint32_t clamp_half(uint32_t a, uint32_t b) {
    uint32_t r = 0;
    for (int s = 0; s < 32; s += 8) r |= (uint32_t)clip255(chan(a, s) + (chan(a, s) - chan(b, s)) / 2) << s;
    return r;
}

uint32_t predict(int mode, uint32_t L, uint32_t T, uint32_t TR, uint32_t TL) {
    switch (mode) {
        case 1: return L;
        case 2: return T;
        case 3: return TR;
        case 4: return TL;
        case 5: return average2(average2(L, TR), T);
        case 6: return average2(L, TL);
        case 7: return average2(L, T);
        case 8: return average2(TL, T);
        case 9: return average2(T, TR);
        case 10: return average2(average2(L, TL), average2(T, TR));
        case 11: return select_pred(L, T, TL);
        case 12: return clamp_full(L, T, TL);
        case 13: return clamp_half(average2(L, T), TL);
        default: return 0xff000000u;   // 0, and the unused modes 14 and 15
    }
}

int8_t s8(uint32_t v) { return (int8_t)(uint8_t)v; }
int delta(int8_t t, int8_t c) { return ((int)t * (int)c) >> 5; }

struct Transform {
    int type;
    uint32_t xsize;          // image width this transform outputs
    uint32_t bits;           // block size bits (predictor, cross-color) or width bits (indexing)
    std::vector<uint32_t> data;
};

bool decode_vp8l(const uint8_t* data, size_t size, int* w, int* h, std::vector<uint8_t>* rgba) {
    if (size < 5 || data[0] != 0x2f || (data[4] >> 5) != 0) return false;
    Bits br(data, size);
    br.read(8);
    const uint32_t width = br.read(14) + 1, height = br.read(14) + 1;
    br.read(1);   // alpha hint
    br.read(3);   // version (0, checked above)
    *w = (int)width;
    *h = (int)height;
    if (!rgba) return true;
    std::vector<Transform> transforms;
    uint32_t xsize = width;
    unsigned seen = 0;
    while (br.read(1)) {
        const int type = (int)br.read(2);
        if (seen & (1u << type)) return false;
        seen |= 1u << type;
        Transform t{type, xsize, 0, {}};
        if (type == 0 || type == 1) {
            t.bits = br.read(3) + 2;
            if (!read_image(br, div_round_up(xsize, t.bits), div_round_up(height, t.bits), false, t.data)) return false;
        } else if (type == 3) {
            const uint32_t colors = br.read(8) + 1;
            t.bits = colors > 16 ? 0 : colors > 4 ? 1 : colors > 2 ? 2 : 3;
            std::vector<uint32_t> table;
            if (!read_image(br, colors, 1, false, table)) return false;
            t.data.assign(256, 0u);   // indices past the table give transparent black
            for (uint32_t i = 0; i < colors; ++i) t.data[i] = i ? add_pixels(table[i], t.data[i - 1]) : table[0];
            xsize = div_round_up(xsize, t.bits);
        }
        transforms.push_back(std::move(t));
    }
    std::vector<uint32_t> img;
    if (!read_image(br, xsize, height, true, img)) return false;
    for (size_t k = transforms.size(); k-- > 0;) {
        const Transform& t = transforms[k];
        const uint32_t W = t.xsize;
        if (t.type == 0) {
            const uint32_t bw = div_round_up(W, t.bits);
            for (uint32_t y = 0; y < height; ++y) {
                for (uint32_t x = 0; x < W; ++x) {
                    const size_t i = (size_t)y * W + x;
                    uint32_t pred;
                    if (y == 0) pred = x == 0 ? 0xff000000u : img[i - 1];
                    else if (x == 0) pred = img[i - W];
                    else {
                        const int mode = (int)((t.data[(size_t)(y >> t.bits) * bw + (x >> t.bits)] >> 8) & 15u);
                        pred = predict(mode, img[i - 1], img[i - W], img[i - W + 1], img[i - W - 1]);
                    }
                    img[i] = add_pixels(img[i], pred);
                }
            }
        } else if (t.type == 1) {
            const uint32_t bw = div_round_up(W, t.bits);
            for (uint32_t y = 0; y < height; ++y) {
                for (uint32_t x = 0; x < W; ++x) {
                    const uint32_t m = t.data[(size_t)(y >> t.bits) * bw + (x >> t.bits)];
                    const int8_t g2r = s8(m), g2b = s8(m >> 8), r2b = s8(m >> 16);
                    uint32_t& p = img[(size_t)y * W + x];
                    const int8_t g = s8(p >> 8);
                    int r = chan(p, 16) + delta(g2r, g);
                    r &= 0xff;
                    int b = chan(p, 0) + delta(g2b, g);
                    b += delta(r2b, s8((uint32_t)r));
                    b &= 0xff;
                    p = (p & 0xff00ff00u) | (uint32_t)r << 16 | (uint32_t)b;
                }
            }
        } else if (t.type == 2) {
            for (uint32_t& p : img) {
                const uint32_t g = (p >> 8) & 0xffu;
                const uint32_t rb = ((p & 0x00ff00ffu) + (g << 16 | g)) & 0x00ff00ffu;
                p = (p & 0xff00ff00u) | rb;
            }
        } else {
            const uint32_t packed_w = div_round_up(W, t.bits);
            const uint32_t bpp = 8u >> t.bits, mask = (1u << bpp) - 1u;
            std::vector<uint32_t> full((size_t)W * height);
            for (uint32_t y = 0; y < height; ++y) {
                for (uint32_t x = 0; x < W; ++x) {
                    const uint32_t packed = img[(size_t)y * packed_w + (x >> t.bits)];
                    const uint32_t index = (packed >> 8 >> ((x & ((1u << t.bits) - 1u)) * bpp)) & mask;
                    full[(size_t)y * W + x] = t.data[index];
                }
            }
            img.swap(full);
        }
    }
    rgba->resize((size_t)width * height * 4);
    for (size_t i = 0; i < img.size(); ++i) {
        const uint32_t p = img[i];
        (*rgba)[i * 4 + 0] = (uint8_t)(p >> 16);
        (*rgba)[i * 4 + 1] = (uint8_t)(p >> 8);
        (*rgba)[i * 4 + 2] = (uint8_t)p;
        (*rgba)[i * 4 + 3] = (uint8_t)(p >> 24);
    }
    return true;
}

// The VP8L bitstream inside a RIFF/WEBP container (directly, or after a VP8X
// chunk and any other chunks), or a raw VP8L bitstream.
bool find_vp8l(const uint8_t* data, size_t size, const uint8_t** bits, size_t* bits_size) {
    if (size >= 12 && !std::memcmp(data, "RIFF", 4)) {
        const uint32_t riff = le32(data + 4);
        if (std::memcmp(data + 8, "WEBP", 4) || riff < 12 || (uint64_t)riff > (uint64_t)size - 8) return false;
        size_t at = 12;
        const size_t end = (size_t)riff + 8;
        bool first = true;
        while (at + 8 <= end) {
            const uint32_t len = le32(data + at + 4);
            if ((uint64_t)at + 8 + len > end) return false;
            if (!std::memcmp(data + at, "VP8L", 4)) {
                // the bitstream may run on past its chunk into the rest of the data
                *bits = data + at + 8;
                *bits_size = size - (at + 8);
                return true;
            }
            if (!std::memcmp(data + at, "VP8 ", 4)) return false;   // lossy
            if (first && std::memcmp(data + at, "VP8X", 4)) return false;
            if (first && len != 10) return false;
            if (first && (data[at + 8] & 0x02)) return false;   // animation
            first = false;
            at += 8 + (size_t)len + (len & 1u);
        }
        return false;
    }
    *bits = data;
    *bits_size = size;
    return true;
}

}  // namespace

bool webp_decode_rgba(const uint8_t* data, size_t size, int* width, int* height, std::vector<uint8_t>* rgba) {
    *width = *height = 0;
    const uint8_t* bits;
    size_t bits_size;
    if (!data || !find_vp8l(data, size, &bits, &bits_size)) return false;
    int w = 0, h = 0;
    if (!decode_vp8l(bits, bits_size, &w, &h, rgba)) return false;
    *width = w;
    *height = h;
    return true;
}

}  // namespace gs

extern "C" int gs_webp_decode_rgba(const uint8_t* data, uint64_t size, int32_t* width, int32_t* height,
                                   uint8_t* rgba, uint64_t capacity) {
    if (!data || !width || !height) return GS_ERR_BAD_ARG;
    std::vector<uint8_t> px;
    int w = 0, h = 0;
    bool ok = false;
    try {
        ok = gs::webp_decode_rgba(data, (size_t)size, &w, &h, &px);
    } catch (const std::bad_alloc&) {
        *width = *height = 0;
        return GS_ERR_OOM;
    }
    if (!ok) {
        *width = *height = 0;
        return GS_ERR_FORMAT;
    }
    *width = w;
    *height = h;
    if (rgba && px.size() <= capacity) std::memcpy(rgba, px.data(), px.size());
    return GS_OK;
}
