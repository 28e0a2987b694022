// gsanim assets on the host: the archive reader, manifest validation, base
// PLY decode and playback sampling of src/gaussian_loader_gsanim.cpp
// (gaussian_load_gsanim :386-495, gsanim_sample :497-509,
// gsanim_layer_weights :511-531).  The result feeds the device path:
// gs_gsanim_rows -> gs_upload_rows, gs_gsanim_deltas -> gs_upload_anim,
// gs_gsanim_sample -> gs_set_anim_state, gs_gsanim_display_lut ->
// gs_set_display_lut.
//
// An asset is accepted exactly when the reference loader accepts it:
//   * a ZIP archive of at most 512 MiB with exactly four entries, stored or
//     deflated, unencrypted, none a directory, each name one of the six
//     payload names and none repeated, every payload's CRC-32 verified;
//   * manifest.json: at most 1 MiB of strict JSON (UTF-8 checked, escapes
//     checked, nesting depth at most 32), then the version-specific fields;
//   * base.ply: the 62-float little-endian layout, comment lines allowed
//     between header lines, every value finite, decoded scales finite with
//     finite squares, quaternion norms above 1e-8; every decoded appearance
//     state finite (0.1 / 0.2), no appearance in the base (0.3);
//   * scales.bin: 48 finite positive floats; deltas.bin: (states - 1) x N x 48
//     int8 without -128 (0.1 / 0.2); layers.bin: layers x N x 48 finite
//     halves; display_lut.bin: size^3 RGB uint16 (0.3).
// The archive reader (gs_zip.h) follows the reference archive reader's
// acceptance rules; archives with ZIP64 records are rejected (a 512 MiB
// archive of four entries never needs them).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/gs_api.h"
#include "gs_json.h"
#include "gs_parallel.h"
#include "gs_zip.h"

struct gs_gsanim {
    struct Key {
        double time_seconds = 0;
        uint32_t state = 0;
        bool linear = false;              // outgoing interval (0.2)
        bool has_interpolation = false;
    };
    struct LayerKey {
        double time_seconds = 0;
        std::array<float, 3> weight{};
        bool linear = false;
    };
    struct Layer {
        std::string name;
        std::vector<LayerKey> keys;
    };
    uint32_t version = 0;                 // 1, 2, 3 for "0.1", "0.2", "0.3"
    uint32_t gaussian_count = 0;
    uint32_t state_count = 0;
    double duration = 0;
    bool linear = false;
    std::vector<Key> keys;
    std::vector<Layer> layers;
    std::vector<uint16_t> layer_data;     // IEEE half bits, layer / row / coefficient
    std::vector<uint16_t> display_lut;    // RGB uint16 UNORM, red fastest
    uint32_t lut_size = 0;
    float log2_min = 0, log2_max = 0;
    std::vector<int8_t> deltas;           // state-major, original row order, 48 per row
    float scales[48] = {};
    std::vector<float> rows;              // GpuGaussian rows, 64 floats each
};

namespace {

using gs::Json;
using gs::Zip;
using gs::ZipEntry;

constexpr size_t kMaxText = 1024 * 1024;              // manifest, PLY header
constexpr size_t kMaxPayload = 256u * 1024 * 1024;    // deltas / layer coefficients
constexpr uint32_t kMaxGaussians = 1000000;
constexpr long kMaxArchive = 512l * 1024 * 1024;

uint16_t le16(const uint8_t* p) { return (uint16_t)(p[0] | p[1] << 8); }
uint32_t le32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
float lef32(const uint8_t* p) {
    const uint32_t b = le32(p);
    float v;
    std::memcpy(&v, &b, 4);
    return v;
}

// ---- manifest ---------------------------------------------------------------

bool parse_layers(const Json& j, int arr, gs_gsanim& a) {
    if (j.at(arr).type != Json::kArr) return false;
    for (int li : j.at(arr).kids) {
        if (j.at(li).type != Json::kObj || a.layers.size() >= 256) return false;
        gs_gsanim::Layer layer;
        unsigned fields = 0;
        const auto& lk = j.at(li).kids;
        for (size_t m = 0; m + 1 < lk.size(); m += 2) {
            const int k = lk[m], v = lk[m + 1];
            if (j.identifier(k, "name")) {
                if ((fields & 1) || !j.decoded(v, layer.name) || layer.name.empty()) return false;
                fields |= 1;
            } else if (j.identifier(k, "keys")) {
                if ((fields & 2) || j.at(v).type != Json::kArr) return false;
                fields |= 2;
                for (int ki : j.at(v).kids) {
                    if (j.at(ki).type != Json::kObj || layer.keys.size() >= 65536) return false;
                    gs_gsanim::LayerKey key;
                    unsigned seen = 0;
                    const auto& kk = j.at(ki).kids;
                    for (size_t q = 0; q + 1 < kk.size(); q += 2) {
                        const int name = kk[q], val = kk[q + 1];
                        const unsigned bit = j.identifier(name, "time_seconds") ? 1u
                                             : j.identifier(name, "weight")     ? 2u
                                             : j.identifier(name, "interpolation") ? 4u : 0u;
                        if (!bit) continue;
                        if (seen & bit) return false;
                        seen |= bit;
                        if (bit == 1 && !j.number(val, key.time_seconds)) return false;
                        if (bit == 4 && !j.mode(val, key.linear)) return false;
                        if (bit == 2) {
                            if (j.at(val).type != Json::kArr) return false;
                            unsigned c = 0;
                            for (int comp : j.at(val).kids) {
                                double n;
                                if (c == 3 || !j.number(comp, n) || n < 0 || !std::isfinite((float)n)) return false;
                                key.weight[c++] = (float)n;
                            }
                            if (c != 3) return false;
                        }
                    }
                    if (seen != 7) return false;
                    layer.keys.push_back(key);
                }
            }
        }
        if (fields != 3 || layer.keys.empty()) return false;
        for (const auto& prev : a.layers)
            if (prev.name == layer.name) return false;
        a.layers.push_back(std::move(layer));
    }
    return !a.layers.empty();
}

bool parse_display(const Json& j, int obj, gs_gsanim& a) {
    if (j.at(obj).type != Json::kObj) return false;
    static const char* names[] = {"type", "encoding", "layout", "size", "log2_min", "log2_max"};
    static const char* values[] = {"lut3d_log2", "uint16_unorm_rgb", "r_fastest"};
    unsigned seen = 0;
    const auto& kids = j.at(obj).kids;
    for (size_t m = 0; m + 1 < kids.size(); m += 2) {
        const int k = kids[m], v = kids[m + 1];
        int field = -1;
        for (int i = 0; i < 6; ++i)
            if (j.identifier(k, names[i])) field = i;
        if (field < 0) continue;
        if (seen & (1u << field)) return false;
        seen |= 1u << field;
        if (field < 3 && !j.identifier(v, values[field])) return false;
        if (field == 3 && (!j.integer(v, a.lut_size, 256) || a.lut_size < 2)) return false;
        if (field >= 4) {
            double n;
            if (!j.number(v, n) || !std::isfinite((float)n)) return false;
            (field == 4 ? a.log2_min : a.log2_max) = (float)n;
        }
    }
    return seen == 63 && a.log2_min < a.log2_max;
}

bool parse_manifest(const std::vector<uint8_t>& text, gs_gsanim& a) {
    Json j;
    const int root = j.parse(text);
    if (root < 0 || j.at(root).type != Json::kObj) return false;
    const auto& kids = j.at(root).kids;
    // the version first, wherever it stands: it decides which fields count
    bool version_seen = false;
    for (size_t m = 0; m + 1 < kids.size(); m += 2) {
        if (!j.identifier(kids[m], "version")) continue;
        if (version_seen) return false;
        version_seen = true;
        const int v = kids[m + 1];
        a.version = j.identifier(v, "0.1") ? 1 : j.identifier(v, "0.2") ? 2 : j.identifier(v, "0.3") ? 3 : 0;
    }
    if (!version_seen || !a.version) return false;
    static const char* names[] = {"format", "version", "gaussian_count", "state_count", "sh_degree",
                                  "coordinate_system", "color_encoding", "duration_seconds", "interpolation",
                                  "keys", "layers", "display_transform"};
    bool linear_color = false;
    unsigned seen = 0;
    for (size_t m = 0; m + 1 < kids.size(); m += 2) {
        const int k = kids[m], v = kids[m + 1];
        int field = -1;
        for (int i = 0; i < 12; ++i)
            if (j.identifier(k, names[i])) field = i;
        if (field < 0) continue;
        if (a.version != 3 && field >= 10) continue;
        if (a.version == 3 && (field == 3 || field == 8 || field == 9)) continue;
        if (seen & (1u << field)) return false;
        seen |= 1u << field;
        uint32_t degree;
        switch (field) {
            case 0: if (!j.identifier(v, "gsanim")) return false; break;
            case 1: break;
            case 2: if (!j.integer(v, a.gaussian_count, kMaxGaussians) || !a.gaussian_count) return false; break;
            case 3: if (!j.integer(v, a.state_count, 256) || a.state_count < 2) return false; break;
            case 4: if (!j.integer(v, degree, 3) || degree != 3) return false; break;
            case 5: if (!j.identifier(v, "blender_world_z_up_meters")) return false; break;
            case 6:
                linear_color = j.identifier(v, "scene_linear_rec709");
                if (!linear_color && !j.identifier(v, "display_referred_agx_baked")) return false;
                break;
            case 7: if (!j.number(v, a.duration) || a.duration <= 0) return false; break;
            case 8:
                if (!j.mode(v, a.linear)) return false;
                break;
            case 9: {
                if (j.at(v).type != Json::kArr) return false;
                for (int ki : j.at(v).kids) {
                    if (j.at(ki).type != Json::kObj || a.keys.size() >= 65536) return false;
                    gs_gsanim::Key key;
                    unsigned fields = 0;
                    const auto& kk = j.at(ki).kids;
                    for (size_t q = 0; q + 1 < kk.size(); q += 2) {
                        const int name = kk[q], val = kk[q + 1];
                        if (j.identifier(name, "time_seconds")) {
                            if ((fields & 1) || !j.number(val, key.time_seconds)) return false;
                            fields |= 1;
                        } else if (j.identifier(name, "state")) {
                            if ((fields & 2) || !j.integer(val, key.state, 255)) return false;
                            fields |= 2;
                        } else if (a.version == 2 && j.identifier(name, "interpolation")) {
                            if (key.has_interpolation) return false;
                            key.has_interpolation = true;
                            if (!j.mode(val, key.linear)) return false;
                        }
                    }
                    if (fields != 3) return false;
                    a.keys.push_back(key);
                }
                break;
            }
            case 10: if (!parse_layers(j, v, a)) return false; break;
            case 11: if (!parse_display(j, v, a)) return false; break;
        }
    }
    const unsigned required = a.version == 3 ? 0xcf7u : 0x3ffu;
    if ((seen & required) != required || linear_color != (a.version == 3)) return false;
    if (a.version == 3) {
        for (const auto& layer : a.layers) {
            if (layer.keys.front().time_seconds != 0) return false;
            double previous = -1;
            for (const auto& key : layer.keys) {
                if (key.time_seconds <= previous || key.time_seconds >= a.duration) return false;
                previous = key.time_seconds;
            }
        }
        return true;
    }
    if (a.keys.empty() || a.keys.front().time_seconds != 0) return false;
    double previous = -1;
    for (const auto& key : a.keys) {
        if (a.version == 2 && !key.has_interpolation) return false;
        if (key.state >= a.state_count || key.time_seconds <= previous || key.time_seconds >= a.duration) return false;
        previous = key.time_seconds;
    }
    return true;
}

// ---- base.ply -----------------------------------------------------------------

// Header check; on success `offset` is the first body byte.
bool ply_header(const std::vector<uint8_t>& bytes, uint32_t count, size_t& offset) {
    offset = 0;
    std::string text;
    auto line = [&]() {
        const size_t start = offset;
        while (offset < bytes.size() && offset < kMaxText && bytes[offset] != '\n') ++offset;
        if (offset == bytes.size() || offset == kMaxText) return false;
        text.assign((const char*)bytes.data() + start, offset - start);
        ++offset;
        return text.find('\r') == std::string::npos;
    };
    if (!line() || text != "ply" || !line() || text != "format binary_little_endian 1.0") return false;
    std::vector<std::string> expected{"element vertex " + std::to_string(count)};
    for (const char* n : {"x", "y", "z", "nx", "ny", "nz"}) expected.push_back(std::string("property float ") + n);
    for (int i = 0; i < 3; ++i) expected.push_back("property float f_dc_" + std::to_string(i));
    for (int i = 0; i < 45; ++i) expected.push_back("property float f_rest_" + std::to_string(i));
    expected.push_back("property float opacity");
    for (int i = 0; i < 3; ++i) expected.push_back("property float scale_" + std::to_string(i));
    for (int i = 0; i < 4; ++i) expected.push_back("property float rot_" + std::to_string(i));
    expected.push_back("end_header");
    for (const std::string& want : expected) {
        do {
            if (!line()) return false;
        } while (text == "comment" || text.compare(0, 8, "comment ") == 0);
        if (text != want) return false;
    }
    return bytes.size() - offset == (size_t)count * 248;
}

int load(const char* path, gs_gsanim* a) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return GS_ERR_FORMAT;
    long length = -1;
    if (!std::fseek(f, 0, SEEK_END)) length = std::ftell(f);
    if (length < 0 || length > kMaxArchive || std::fseek(f, 0, SEEK_SET)) {
        std::fclose(f);
        return GS_ERR_FORMAT;
    }
    Zip zip;
    zip.bytes.resize((size_t)length);
    const bool read_ok = std::fread(zip.bytes.data(), 1, zip.bytes.size(), f) == zip.bytes.size();
    std::fclose(f);
    if (!read_ok || !zip.open() || zip.entries.size() != 4) return GS_ERR_FORMAT;

    static const char* names[] = {"manifest.json", "base.ply", "scales.bin", "deltas.bin", "layers.bin",
                                  "display_lut.bin"};
    const ZipEntry* stats[6] = {};
    unsigned seen = 0;
    for (const ZipEntry& z : zip.entries) {
        if (Zip::is_directory(z) || !Zip::usable(z)) return GS_ERR_FORMAT;
        int which = -1;
        for (int i = 0; i < 6; ++i)
            if (z.name == names[i]) which = i;
        if (which < 0 || (seen & (1u << which))) return GS_ERR_FORMAT;
        seen |= 1u << which;
        stats[which] = &z;
    }
    if (!stats[0] || !stats[0]->usize || stats[0]->usize > kMaxText) return GS_ERR_FORMAT;
    std::vector<uint8_t> bytes;
    if (!zip.extract(*stats[0], bytes) || !parse_manifest(bytes, *a)) return GS_ERR_FORMAT;
    if (seen != (a->version == 3 ? 51u : 15u)) return GS_ERR_FORMAT;
    const uint64_t n = a->gaussian_count;
    const uint64_t body = n * 248;
    if (stats[1]->usize <= body || stats[1]->usize > body + kMaxText) return GS_ERR_FORMAT;
    if (a->version == 3) {
        const uint64_t layer_bytes = (uint64_t)a->layers.size() * n * 96;
        const uint64_t lut_bytes = (uint64_t)a->lut_size * a->lut_size * a->lut_size * 6;
        if (layer_bytes > kMaxPayload || stats[4]->usize != layer_bytes || stats[5]->usize != lut_bytes)
            return GS_ERR_FORMAT;
        for (int entry : {4, 5}) {
            if (!zip.extract(*stats[entry], bytes)) return GS_ERR_FORMAT;
            auto& out = entry == 4 ? a->layer_data : a->display_lut;
            out.resize(bytes.size() / 2);
            for (size_t i = 0; i < out.size(); ++i) {
                out[i] = le16(&bytes[i * 2]);
                if (entry == 4 && (out[i] & 0x7c00) == 0x7c00) return GS_ERR_FORMAT;   // inf / NaN half
            }
        }
    } else {
        const uint64_t delta_bytes = (uint64_t)(a->state_count - 1) * n * 48;
        if (delta_bytes > kMaxPayload || stats[3]->usize != delta_bytes || stats[2]->usize != 192)
            return GS_ERR_FORMAT;
        if (!zip.extract(*stats[2], bytes)) return GS_ERR_FORMAT;
        for (int k = 0; k < 48; ++k) {
            a->scales[k] = lef32(&bytes[k * 4]);
            if (!std::isfinite(a->scales[k]) || a->scales[k] <= 0) return GS_ERR_FORMAT;
        }
        if (!zip.extract(*stats[3], bytes)) return GS_ERR_FORMAT;
        a->deltas.assign(bytes.begin(), bytes.end());
        for (int8_t q : a->deltas)
            if (q == -128) return GS_ERR_FORMAT;
    }
    if (!zip.extract(*stats[1], bytes)) return GS_ERR_FORMAT;
    size_t offset;
    if (!ply_header(bytes, a->gaussian_count, offset)) return GS_ERR_FORMAT;
    // Decode and validate every row (the reference's Gaussian checks), then
    // pack: raw order x y z, f_dc, f_rest, opacity, scale, rot (gs_pack_raw).
    // Rows are independent: they are checked on worker threads in slices, and
    // the asset is rejected when any row fails, whichever slice finds it.
    std::vector<float> raw((size_t)n * 59);
    const gs_gsanim& asset = *a;
    const bool rows_ok = gs::parallel_ranges(n, 4096, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            float v[62];
            for (int k = 0; k < 62; ++k) {
                v[k] = lef32(&bytes[offset + (size_t)i * 248 + (size_t)k * 4]);
                if (!std::isfinite(v[k])) return false;
                if (asset.version == 3 && k >= 6 && k < 54 && v[k] != 0) return false;
            }
            for (int k = 0; k < 3; ++k) {
                const float s = std::exp(v[55 + k]);
                if (!std::isfinite(s) || s <= 0 || !std::isfinite(s * s)) return false;
            }
            const float norm = std::sqrt(v[58] * v[58] + v[59] * v[59] + v[60] * v[60] + v[61] * v[61]);
            if (!std::isfinite(norm) || norm <= 1e-8f) return false;
            // every appearance state must decode to finite coefficients
            for (uint32_t s = 1; asset.version != 3 && s < asset.state_count; ++s) {
                for (int k = 0; k < 48; ++k) {
                    const float delta =
                        (float)asset.deltas[((size_t)(s - 1) * n + i) * 48 + (size_t)k] * asset.scales[k];
                    if (!std::isfinite(delta) || !std::isfinite(v[6 + k] + delta)) return false;
                }
            }
            float* r = &raw[(size_t)i * 59];
            r[0] = v[0];
            r[1] = v[1];
            r[2] = v[2];
            std::memcpy(r + 3, v + 6, 56 * sizeof(float));   // f_dc, f_rest, opacity, scale, rot
        }
        return true;
    });
    if (!rows_ok) return GS_ERR_FORMAT;
    a->rows.resize((size_t)n * 64);
    return gs_pack_raw(raw.data(), n, a->rows.data());
}

// Playback position in [0, duration) (negative times wrap).
double wrap(double seconds, double duration) {
    double u = std::fmod(seconds, duration);
    if (u < 0) u += duration;
    if (u >= duration) u = 0;
    return u;
}

}  // namespace

extern "C" {

int gs_gsanim_load(const char* path, gs_gsanim** out) {
    if (!out) return GS_ERR_BAD_ARG;
    *out = nullptr;
    if (!path) return GS_ERR_BAD_ARG;
    try {
        gs_gsanim* a = new gs_gsanim;
        const int rc = load(path, a);
        if (rc != GS_OK) {
            delete a;
            return rc;
        }
        *out = a;
        return GS_OK;
    } catch (const std::bad_alloc&) {
        return GS_ERR_OOM;
    }
}

void gs_gsanim_free(gs_gsanim* a) { delete a; }

int gs_gsanim_get_info(const gs_gsanim* a, gs_gsanim_info* out) {
    if (!a || !out) return GS_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    out->version = a->version;
    out->gaussian_count = a->gaussian_count;
    out->state_count = a->version == 3 ? 0 : a->state_count;
    out->layer_count = (uint32_t)a->layers.size();
    out->key_count = (uint32_t)a->keys.size();
    out->lut_size = a->lut_size;
    out->linear = a->linear ? 1 : 0;
    out->log2_min = a->log2_min;
    out->log2_max = a->log2_max;
    out->duration_seconds = a->duration;
    return GS_OK;
}

int gs_gsanim_rows(const gs_gsanim* a, float* rows) {
    if (!a || !rows) return GS_ERR_BAD_ARG;
    std::memcpy(rows, a->rows.data(), a->rows.size() * sizeof(float));
    return GS_OK;
}

int gs_gsanim_deltas(const gs_gsanim* a, int8_t* deltas, float* scales) {
    if (!a) return GS_ERR_BAD_ARG;
    if (deltas && !a->deltas.empty()) std::memcpy(deltas, a->deltas.data(), a->deltas.size());
    if (scales) std::memcpy(scales, a->scales, sizeof(a->scales));
    return GS_OK;
}

int gs_gsanim_layer_data(const gs_gsanim* a, uint16_t* halves) {
    if (!a || !halves) return GS_ERR_BAD_ARG;
    if (!a->layer_data.empty()) std::memcpy(halves, a->layer_data.data(), a->layer_data.size() * 2);
    return GS_OK;
}

int gs_gsanim_display_lut(const gs_gsanim* a, uint16_t* rgb) {
    if (!a || !rgb) return GS_ERR_BAD_ARG;
    if (!a->display_lut.empty()) std::memcpy(rgb, a->display_lut.data(), a->display_lut.size() * 2);
    return GS_OK;
}

int64_t gs_gsanim_layer_name(const gs_gsanim* a, uint32_t layer, char* buf, uint64_t capacity) {
    if (!a || layer >= a->layers.size() || (!buf && capacity)) return GS_ERR_BAD_ARG;
    const std::string& n = a->layers[layer].name;
    if (capacity) std::memcpy(buf, n.data(), n.size() < capacity ? n.size() : (size_t)capacity);
    return (int64_t)n.size();
}

int gs_gsanim_sample(const gs_gsanim* a, double seconds, int32_t* state_a, int32_t* state_b, float* weight) {
    if (!a || !state_a || !state_b || !weight) return GS_ERR_BAD_ARG;
    *state_a = *state_b = 0;
    *weight = 0.0f;
    if (!std::isfinite(seconds) || !std::isfinite(a->duration) || a->duration <= 0 || a->keys.empty())
        return GS_OK;
    const double u = wrap(seconds, a->duration);
    const auto next = std::upper_bound(a->keys.begin(), a->keys.end(), u,
                                       [](double t, const gs_gsanim::Key& k) { return t < k.time_seconds; });
    const size_t i = next == a->keys.begin() ? 0 : (size_t)(next - a->keys.begin() - 1);
    const int state = (int)a->keys[i].state;
    *state_a = *state_b = state;
    if (!(a->version == 2 ? a->keys[i].linear : a->linear) || a->keys.size() == 1) return GS_OK;
    const size_t jn = (i + 1) % a->keys.size();
    const double end = jn ? a->keys[jn].time_seconds : a->duration;
    *state_b = (int)a->keys[jn].state;
    *weight = (float)((u - a->keys[i].time_seconds) / (end - a->keys[i].time_seconds));
    return GS_OK;
}

int gs_gsanim_layer_weights(const gs_gsanim* a, double seconds, float* weights) {
    if (!a || (!weights && !a->layers.empty())) return GS_ERR_BAD_ARG;
    if (a->version != 3 || !std::isfinite(seconds) || !std::isfinite(a->duration) || a->duration <= 0) return 0;
    const double u = wrap(seconds, a->duration);
    for (size_t l = 0; l < a->layers.size(); ++l) {
        const auto& keys = a->layers[l].keys;
        if (keys.empty()) return 0;
        const auto next = std::upper_bound(keys.begin(), keys.end(), u,
                                           [](double t, const gs_gsanim::LayerKey& k) { return t < k.time_seconds; });
        const size_t i = next == keys.begin() ? 0 : (size_t)(next - keys.begin() - 1);
        const size_t jn = (i + 1) % keys.size();
        const double end = jn ? keys[jn].time_seconds : a->duration;
        const double w = keys[i].linear && keys.size() > 1 ? (u - keys[i].time_seconds) / (end - keys[i].time_seconds) : 0;
        for (int c = 0; c < 3; ++c) weights[l * 3 + c] = (float)((1 - w) * keys[i].weight[c] + w * keys[jn].weight[c]);
    }
    return (int)a->layers.size();
}

}  // extern "C"
