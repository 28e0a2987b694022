// JSON text reading for the asset loaders (host code): a strict syntax check
// (RFC 8259 grammar, UTF-8 checked, escapes checked, nesting depth bounded)
// that keeps a tree of the text, and the typed field readers the manifests
// use.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace gs {

// Strict syntax check and tree of one JSON text.  Strings keep their raw
// bytes between the quotes (escapes undecoded), numbers their text.
struct Json {
    enum Type { kNull, kBool, kNum, kStr, kArr, kObj };
    struct Node {
        Type type;
        const char* b;
        const char* e;
        std::vector<int> kids;   // arrays: elements; objects: key, value, key, value, ...
    };
    std::vector<Node> nodes;
    const unsigned char* p = nullptr;
    const unsigned char* end = nullptr;

    void space() {
        while (p != end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
    }
    bool take(char c) {
        space();
        if (p == end || *p != (unsigned char)c) return false;
        ++p;
        return true;
    }
    int add(Type t, const unsigned char* b, const unsigned char* e) {
        nodes.push_back(Node{t, (const char*)b, (const char*)e, {}});
        return (int)nodes.size() - 1;
    }
    static bool is_hex(unsigned char c) {
        return (c >= '0' && c <= '9') || (c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F');
    }
    // A string: UTF-8 and escapes checked.
    int string() {
        if (!take('"')) return -1;
        const unsigned char* b = p;
        while (p != end) {
            unsigned c = *p++;
            if (c == '"') return add(kStr, b, p - 1);
            if (c < 32) return -1;
            if (c == '\\') {
                if (p == end) return -1;
                c = *p++;
                if (c == 'u') {
                    for (int i = 0; i < 4; ++i) {
                        if (p == end || !is_hex(*p)) return -1;
                        ++p;
                    }
                } else if (c != 0 && !std::strchr("\"\\/bfnrt", (int)c)) {
                    // (a NUL after the backslash passes the reference's
                    // strchr test, which finds the terminator)
                    return -1;
                }
            } else if (c >= 128) {
                if (c < 0xc2 || c > 0xf4) return -1;
                const unsigned count = c >= 0xf0 ? 3 : c >= 0xe0 ? 2 : 1;
                unsigned value = c & (count == 3 ? 7u : count == 2 ? 15u : 31u);
                for (unsigned i = 0; i < count; ++i) {
                    if (p == end || (*p & 0xc0) != 0x80) return -1;
                    value = (value << 6) | (*p++ & 63u);
                }
                const unsigned least = count == 3 ? 65536u : count == 2 ? 2048u : 128u;
                if (value < least || value > 0x10ffff || (value >= 0xd800 && value <= 0xdfff)) return -1;
            }
        }
        return -1;
    }
    int max_depth = 32;   // deepest value nesting accepted (the root is depth 0)

    int value(int depth = 0) {
        space();
        if (p == end || depth > max_depth) return -1;
        if (*p == '"') return string();
        if (*p == '{' || *p == '[') {
            const bool object = *p++ == '{';
            const int me = add(object ? kObj : kArr, p - 1, p);
            const char close = object ? '}' : ']';
            if (take(close)) return me;
            do {
                if (object) {
                    const int k = string();
                    if (k < 0 || !take(':')) return -1;
                    nodes[me].kids.push_back(k);
                }
                const int v = value(depth + 1);
                if (v < 0) return -1;
                nodes[me].kids.push_back(v);
                if (take(close)) return me;
            } while (take(','));
            return -1;
        }
        static const char* words[] = {"true", "false", "null"};
        for (int w = 0; w < 3; ++w) {
            const size_t n = std::strlen(words[w]);
            if ((size_t)(end - p) >= n && !std::memcmp(p, words[w], n)) {
                p += n;
                return add(w == 2 ? kNull : kBool, p - n, p);
            }
        }
        const unsigned char* b = p;
        if (*p == '-') ++p;
        if (p == end) return -1;
        if (*p == '0') {
            ++p;
        } else {
            if (*p < '1' || *p > '9') return -1;
            while (p != end && *p >= '0' && *p <= '9') ++p;
        }
        if (p != end && *p == '.') {
            ++p;
            const unsigned char* s = p;
            while (p != end && *p >= '0' && *p <= '9') ++p;
            if (p == s) return -1;
        }
        if (p != end && (*p == 'e' || *p == 'E')) {
            ++p;
            if (p != end && (*p == '-' || *p == '+')) ++p;
            const unsigned char* s = p;
            while (p != end && *p >= '0' && *p <= '9') ++p;
            if (p == s) return -1;
        }
        return add(kNum, b, p);
    }
    // The whole text must be one value (whitespace around it allowed).
    int parse(const std::vector<uint8_t>& text) {
        p = text.data();
        end = text.data() + text.size();
        const int root = value();
        if (root < 0) return -1;
        space();
        return p == end ? root : -1;
    }

    const Node& at(int i) const { return nodes[(size_t)i]; }

    // A finite number written in at most 64 characters.
    bool number(int i, double& out) const {
        const Node& v = at(i);
        if (v.type != kNum || v.e - v.b > 64) return false;
        const std::string text(v.b, v.e);
        char* stop = nullptr;
        out = std::strtod(text.c_str(), &stop);
        return stop == text.c_str() + text.size() && std::isfinite(out);
    }
    // A number in [0, max] written with digits only (an optional minus sign).
    bool integer(int i, uint32_t& out, uint32_t max) const {
        double n;
        if (!number(i, n) || n < 0 || n > max) return false;
        const Node& v = at(i);
        for (const char* q = v.b + (*v.b == '-' ? 1 : 0); q != v.e; ++q)
            if (*q < '0' || *q > '9') return false;
        out = (uint32_t)n;
        return true;
    }
    static unsigned hex4(const char* q) {
        unsigned n = 0;
        for (int k = 0; k < 4; ++k) {
            const unsigned c = (unsigned char)q[k];
            n = n * 16 + (c <= '9' ? c - '0' : (c | 32) - 'a' + 10);
        }
        return n;
    }
    // A string equal to the ASCII text `want`, \uXXXX escapes allowed (no
    // other escape).
    bool identifier(int i, const char* want) const {
        const Node& v = at(i);
        if (v.type != kStr) return false;
        for (const char* q = v.b; q != v.e; ++q) {
            unsigned c = (unsigned char)*q;
            if (c == '\\') {
                if (++q == v.e || *q != 'u' || v.e - q < 5) return false;
                c = hex4(q + 1);
                q += 4;
            }
            if (!*want || c != (unsigned char)*want++) return false;
        }
        return *want == 0;
    }
    // The decoded bytes (UTF-8) of a string; unpaired surrogates fail.
    bool decoded(int i, std::string& out) const {
        const Node& v = at(i);
        if (v.type != kStr) return false;
        for (const char* q = v.b; q != v.e;) {
            unsigned c = (unsigned char)*q++;
            if (c != '\\') {
                out += (char)c;
                continue;
            }
            c = (unsigned char)*q++;
            if (c != 'u') {
                static const char from[] = "\"\\/bfnrt";
                static const char to[] = "\"\\/\b\f\n\r\t";
                out += c == 0 ? '\0' : to[std::strchr(from, (int)c) - from];
                continue;
            }
            c = hex4(q);
            q += 4;
            if (c >= 0xd800 && c <= 0xdbff) {
                if (v.e - q < 6 || q[0] != '\\' || q[1] != 'u') return false;
                const unsigned low = hex4(q + 2);
                q += 6;
                if (low < 0xdc00 || low > 0xdfff) return false;
                c = 0x10000 + ((c - 0xd800) << 10) + (low - 0xdc00);
            } else if (c >= 0xdc00 && c <= 0xdfff) {
                return false;
            }
            if (c < 128) {
                out += (char)c;
            } else if (c < 2048) {
                out += (char)(0xc0 | (c >> 6));
                out += (char)(0x80 | (c & 63));
            } else if (c < 65536) {
                out += (char)(0xe0 | (c >> 12));
                out += (char)(0x80 | ((c >> 6) & 63));
                out += (char)(0x80 | (c & 63));
            } else {
                out += (char)(0xf0 | (c >> 18));
                out += (char)(0x80 | ((c >> 12) & 63));
                out += (char)(0x80 | ((c >> 6) & 63));
                out += (char)(0x80 | (c & 63));
            }
        }
        return true;
    }
    bool mode(int i, bool& linear) const {
        linear = identifier(i, "linear");
        return linear || identifier(i, "step");
    }
};

}  // namespace gs
