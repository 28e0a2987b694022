// SOG archives (PlayCanvas "spatially ordered Gaussians", version 2) on the
// host: gaussian_load_sog (src/gaussian_loader_sog.cpp:126-551) decoded into
// GpuGaussian rows (pack_gpu_gaussians, src/gaussian.cpp:53-73), the input
// of gs_upload_rows.
//
// An archive is a ZIP of meta.json and lossless WebP images: means (low and
// high bytes of 16-bit log-space positions), scales (codebook labels),
// quats (smallest-three quaternions), sh0 (DC colour labels + opacity) and
// optionally shN (centroid image + label image).  The meta fields are read
// with the reference's rules: numbers through strtol / strtof of their text,
// strings with the escapes \" \\ \/ \n \t \r only and cut to 127 bytes, a
// later duplicate field overriding an earlier one, unknown fields ignored.
// The meta text must be valid JSON (RFC 8259); the reference's token reader
// also accepts some malformed texts.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gs_api.h"
#include "gs_json.h"
#include "gs_webp.h"
#include "gs_zip.h"

namespace {

using gs::Json;

struct Meta {
    int version = 0;
    uint32_t count = 0;
    float means_mins[3] = {}, means_maxs[3] = {};
    std::string means_files[2];
    float scales_codebook[256] = {};
    std::string scales_file;
    std::string quats_file;
    float sh0_codebook[256] = {};
    std::string sh0_file;
    bool has_shN = false;
    int shN_count = 0, shN_bands = 0;
    float shN_codebook[256] = {};
    std::string shN_files[2];
};

// Field readers with the reference meta reader's rules.
bool key_is(const Json& j, int k, const char* name) {
    const Json::Node& v = j.at(k);
    const size_t len = (size_t)(v.e - v.b);
    return v.type == Json::kStr && std::strlen(name) == len && !std::memcmp(v.b, name, len);
}
bool token(const Json& j, int i, char (&tmp)[64]) {
    const Json::Node& v = j.at(i);
    const size_t len = (size_t)(v.e - v.b);
    if (v.type != Json::kNum || len >= sizeof(tmp)) return false;
    std::memcpy(tmp, v.b, len);
    tmp[len] = 0;
    return true;
}
bool read_int(const Json& j, int i, int& out) {
    char tmp[64];
    if (!token(j, i, tmp)) return false;
    out = (int)std::strtol(tmp, nullptr, 10);
    return true;
}
bool read_float(const Json& j, int i, float& out) {
    char tmp[64];
    if (!token(j, i, tmp)) return false;
    out = std::strtof(tmp, nullptr);
    return true;
}
bool read_string(const Json& j, int i, std::string& out) {
    const Json::Node& v = j.at(i);
    if (v.type != Json::kStr) return false;
    out.clear();
    for (const char* q = v.b; q != v.e; ++q) {
        char c = *q;
        if (c == '\\') {
            if (++q == v.e) return false;
            const char esc = *q;
            if (esc == '"' || esc == '\\' || esc == '/') c = esc;
            else if (esc == 'n') c = '\n';
            else if (esc == 't') c = '\t';
            else if (esc == 'r') c = '\r';
            else return false;
        }
        if (out.size() < 127) out += c;
    }
    return true;
}
bool read_floats(const Json& j, int i, float* out, int expected) {
    if (j.at(i).type != Json::kArr) return false;
    int count = 0;
    for (int e : j.at(i).kids) {
        if (count >= expected || !read_float(j, e, out[count])) return false;
        ++count;
    }
    return count == expected;
}
bool read_strings(const Json& j, int i, std::string* out, int expected) {
    if (j.at(i).type != Json::kArr) return false;
    int count = 0;
    for (int e : j.at(i).kids) {
        if (count >= expected || !read_string(j, e, out[count])) return false;
        ++count;
    }
    return count == expected;
}
bool codebook_file(const Json& j, int obj, float* codebook, std::string& file) {
    if (j.at(obj).type != Json::kObj) return false;
    bool has_codebook = false, has_files = false;
    const auto& kids = j.at(obj).kids;
    for (size_t m = 0; m + 1 < kids.size(); m += 2) {
        if (key_is(j, kids[m], "codebook")) {
            if (!read_floats(j, kids[m + 1], codebook, 256)) return false;
            has_codebook = true;
        } else if (key_is(j, kids[m], "files")) {
            if (!read_strings(j, kids[m + 1], &file, 1)) return false;
            has_files = true;
        }
    }
    return has_codebook && has_files;
}

bool parse_meta(const std::vector<uint8_t>& text, Meta& meta) {
    Json j;
    j.max_depth = 512;
    const int root = j.parse(text);
    if (root < 0 || j.at(root).type != Json::kObj) return false;
    bool has_version = false, has_count = false, has_means = false, has_scales = false, has_quats = false,
         has_sh0 = false;
    const auto& kids = j.at(root).kids;
    for (size_t m = 0; m + 1 < kids.size(); m += 2) {
        const int k = kids[m], v = kids[m + 1];
        if (key_is(j, k, "version")) {
            if (!read_int(j, v, meta.version)) return false;
            has_version = true;
        } else if (key_is(j, k, "count")) {
            int count = 0;
            if (!read_int(j, v, count) || count <= 0) return false;
            meta.count = (uint32_t)count;
            has_count = true;
        } else if (key_is(j, k, "antialias")) {
            if (j.at(v).type != Json::kBool) return false;
        } else if (key_is(j, k, "means")) {
            if (j.at(v).type != Json::kObj) return false;
            bool mins = false, maxs = false, files = false;
            const auto& mk = j.at(v).kids;
            for (size_t q = 0; q + 1 < mk.size(); q += 2) {
                if (key_is(j, mk[q], "mins")) {
                    if (!read_floats(j, mk[q + 1], meta.means_mins, 3)) return false;
                    mins = true;
                } else if (key_is(j, mk[q], "maxs")) {
                    if (!read_floats(j, mk[q + 1], meta.means_maxs, 3)) return false;
                    maxs = true;
                } else if (key_is(j, mk[q], "files")) {
                    if (!read_strings(j, mk[q + 1], meta.means_files, 2)) return false;
                    files = true;
                }
            }
            if (!mins || !maxs || !files) return false;
            has_means = true;
        } else if (key_is(j, k, "scales")) {
            if (!codebook_file(j, v, meta.scales_codebook, meta.scales_file)) return false;
            has_scales = true;
        } else if (key_is(j, k, "quats")) {
            if (j.at(v).type != Json::kObj) return false;
            bool files = false;
            const auto& qk = j.at(v).kids;
            for (size_t q = 0; q + 1 < qk.size(); q += 2) {
                if (key_is(j, qk[q], "files")) {
                    if (!read_strings(j, qk[q + 1], &meta.quats_file, 1)) return false;
                    files = true;
                }
            }
            if (!files) return false;
            has_quats = true;
        } else if (key_is(j, k, "sh0")) {
            if (!codebook_file(j, v, meta.sh0_codebook, meta.sh0_file)) return false;
            has_sh0 = true;
        } else if (key_is(j, k, "shN")) {
            if (j.at(v).type != Json::kObj) return false;
            bool count = false, bands = false, codebook = false, files = false;
            const auto& sk = j.at(v).kids;
            for (size_t q = 0; q + 1 < sk.size(); q += 2) {
                const int name = sk[q], val = sk[q + 1];
                if (key_is(j, name, "count")) {
                    if (!read_int(j, val, meta.shN_count)) return false;
                    count = true;
                } else if (key_is(j, name, "bands")) {
                    if (!read_int(j, val, meta.shN_bands)) return false;
                    bands = true;
                } else if (key_is(j, name, "codebook")) {
                    if (!read_floats(j, val, meta.shN_codebook, 256)) return false;
                    codebook = true;
                } else if (key_is(j, name, "files")) {
                    if (!read_strings(j, val, meta.shN_files, 2)) return false;
                    files = true;
                }
            }
            if (!count || !bands || !codebook || !files) return false;
            if (meta.shN_count <= 0 || meta.shN_count > 65536 || meta.shN_bands < 1 || meta.shN_bands > 3) return false;
            meta.has_shN = true;
        }
    }
    return has_version && has_count && has_means && has_scales && has_quats && has_sh0 && meta.version == 2;
}

struct Image {
    std::vector<uint8_t> px;
    int w = 0, h = 0;
};

struct Archive {
    std::vector<std::string> names;             // as C strings: cut at NUL and at 511 bytes
    std::vector<std::vector<uint8_t>> data;

    const std::vector<uint8_t>* find(const std::string& name) const {
        for (size_t i = 0; i < names.size(); ++i)
            if (names[i] == name) return &data[i];
        return nullptr;
    }
    bool image(const std::string& name, Image& out) const {
        const std::vector<uint8_t>* d = find(name);
        return d && gs::webp_decode_rgba(d->data(), d->size(), &out.w, &out.h, &out.px) && out.w > 0 && out.h > 0;
    }
};

int load(const char* path, std::vector<float>& rows) {
    gs::Zip zip;
    {
        FILE* f = std::fopen(path, "rb");
        if (!f) return GS_ERR_FORMAT;
        long length = -1;
        if (!std::fseek(f, 0, SEEK_END)) length = std::ftell(f);
        if (length < 0 || std::fseek(f, 0, SEEK_SET)) {
            std::fclose(f);
            return GS_ERR_FORMAT;
        }
        zip.bytes.resize((size_t)length);
        const bool ok = std::fread(zip.bytes.data(), 1, zip.bytes.size(), f) == zip.bytes.size();
        std::fclose(f);
        if (!ok || !zip.open()) return GS_ERR_FORMAT;
    }
    Archive ar;
    for (const gs::ZipEntry& z : zip.entries) {
        if (gs::Zip::is_directory(z)) continue;
        // (an entry without compressed bytes reads as empty whatever its method or flags)
        std::vector<uint8_t> payload;
        if ((z.csize && !gs::Zip::usable(z)) || !zip.extract(z, payload)) return GS_ERR_FORMAT;
        std::string name = z.name.substr(0, std::min<size_t>(z.name.size(), 511));
        name = name.substr(0, std::strlen(name.c_str()));
        ar.names.push_back(std::move(name));
        ar.data.push_back(std::move(payload));
    }
    const std::vector<uint8_t>* meta_text = ar.find("meta.json");
    Meta meta;
    if (!meta_text || !parse_meta(*meta_text, meta)) return GS_ERR_FORMAT;
    for (const std::string* f : {&meta.means_files[0], &meta.means_files[1], &meta.scales_file, &meta.quats_file,
                                 &meta.sh0_file})
        if (!ar.find(*f)) return GS_ERR_FORMAT;
    if (meta.has_shN && (!ar.find(meta.shN_files[0]) || !ar.find(meta.shN_files[1]))) return GS_ERR_FORMAT;

    // The images decode independently, each on its own thread; their
    // results are then checked in the order a serial decode would meet them,
    // so the verdict (and an allocation failure) is the serial one.
    enum { kMeansL, kMeansU, kScales, kQuats, kSh0, kCentroids, kLabels, kImages };
    const std::string* files[kImages] = {&meta.means_files[0], &meta.means_files[1], &meta.scales_file,
                                         &meta.quats_file, &meta.sh0_file, &meta.shN_files[0], &meta.shN_files[1]};
    const int count = meta.has_shN ? kImages : kCentroids;
    Image img[kImages];
    int state[kImages] = {};   // 1 decoded, 0 invalid, -1 out of memory
    auto decode = [&](int k) {
        try {
            state[k] = ar.image(*files[k], img[k]) ? 1 : 0;
        } catch (const std::bad_alloc&) {
            state[k] = -1;
        }
    };
    {
        std::vector<std::thread> pool;
        int next = 0;
        try {
            pool.reserve((size_t)count);
            for (; next < count; ++next) pool.emplace_back(decode, next);
        } catch (const std::exception&) {   // no more threads: the rest decode here
        }
        for (int k = next; k < count; ++k) decode(k);
        for (auto& t : pool) t.join();
    }
    auto usable = [&](int k) {
        if (state[k] < 0) throw std::bad_alloc();
        return state[k] == 1;
    };
    for (int k = kMeansL; k <= kSh0; ++k)
        if (!usable(k)) return GS_ERR_FORMAT;
    Image &means_l = img[kMeansL], &means_u = img[kMeansU], &scales = img[kScales], &quats = img[kQuats],
          &sh0 = img[kSh0];
    const int w = means_l.w, h = means_l.h;
    for (const Image* im : {&means_u, &scales, &quats, &sh0})
        if (im->w != w || im->h != h) return GS_ERR_FORMAT;
    const uint32_t n = meta.count;
    if ((uint64_t)n > (uint64_t)w * (uint64_t)h) return GS_ERR_FORMAT;

    rows.assign((size_t)n * 64, 0.0f);
    const float root2 = std::sqrt(2.0f);
    for (uint32_t i = 0; i < n; ++i) {
        const uint8_t* ml = &means_l.px[(size_t)i * 4];
        const uint8_t* mu = &means_u.px[(size_t)i * 4];
        const uint8_t* sc = &scales.px[(size_t)i * 4];
        const uint8_t* qt = &quats.px[(size_t)i * 4];
        const uint8_t* s0 = &sh0.px[(size_t)i * 4];
        float* d = &rows[(size_t)i * 64];
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t q = (uint32_t)mu[axis] << 8 | (uint32_t)ml[axis];
            const float t = (float)q / 65535.0f;
            const float lo = meta.means_mins[axis], hi = meta.means_maxs[axis];
            const float v = lo + (hi - lo) * t;                                   // log-space position
            d[axis] = v < 0.0f ? -(std::exp(-v) - 1.0f) : (std::exp(v) - 1.0f);   // signed exp(|v|) - 1
            d[4 + axis] = std::exp(meta.scales_codebook[sc[axis]]);
            d[12 + axis] = meta.sh0_codebook[s0[axis]];
        }
        float c3[3];
        for (int k = 0; k < 3; ++k) c3[k] = ((float)qt[k] / 255.0f - 0.5f) * 2.0f / root2;
        const int mode = (int)qt[3] - 252;
        if (mode < 0 || mode > 3) return GS_ERR_FORMAT;
        const float omitted = std::sqrt(std::fmax(0.0f, 1.0f - (c3[0] * c3[0] + c3[1] * c3[1] + c3[2] * c3[2])));
        // the omitted (largest) component goes to slot `mode`, the three stored ones fill the rest in order
        int k = 0;
        for (int slot = 0; slot < 4; ++slot) d[8 + slot] = slot == mode ? omitted : c3[k++];
        d[3] = (float)s0[3] / 255.0f;
    }
    if (meta.has_shN) {
        const int coeffs = meta.shN_bands == 1 ? 3 : meta.shN_bands == 2 ? 8 : 15;
        if (!usable(kCentroids) || !usable(kLabels)) return GS_ERR_FORMAT;
        const Image &centroids = img[kCentroids], &labels = img[kLabels];
        if ((uint64_t)n > (uint64_t)labels.w * (uint64_t)labels.h) return GS_ERR_FORMAT;
        if (centroids.w < 64 * coeffs || centroids.h < (meta.shN_count + 63) / 64) return GS_ERR_FORMAT;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t* lp = &labels.px[(size_t)i * 4];
            const uint32_t label = (uint32_t)lp[0] | (uint32_t)lp[1] << 8;
            if (label >= (uint32_t)meta.shN_count) return GS_ERR_FORMAT;
            float* d = &rows[(size_t)i * 64];
            for (int c = 0; c < coeffs; ++c) {
                const size_t u = (size_t)(label % 64) * (size_t)coeffs + (size_t)c, v = label / 64;
                const uint8_t* cp = &centroids.px[(v * (size_t)centroids.w + u) * 4];
                d[16 + c * 3 + 0] = meta.shN_codebook[cp[0]];
                d[16 + c * 3 + 1] = meta.shN_codebook[cp[1]];
                d[16 + c * 3 + 2] = meta.shN_codebook[cp[2]];
            }
        }
    }
    return GS_OK;
}

}  // namespace

extern "C" int64_t gs_load_sog(const char* path, float* rows, uint64_t capacity) {
    if (!path) return GS_ERR_BAD_ARG;
    try {
        std::vector<float> all;
        const int rc = load(path, all);
        if (rc != GS_OK) return rc;
        const uint64_t n = all.size() / 64;
        if (rows) std::memcpy(rows, all.data(), (size_t)(n < capacity ? n : capacity) * 64 * sizeof(float));
        return (int64_t)n;
    } catch (const std::bad_alloc&) {
        return GS_ERR_OOM;
    }
}
