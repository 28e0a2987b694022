// Host-side helpers of the C ABI that need no GPU: camera uniforms and PLY
// ingestion into GpuGaussian rows.  Compiled with -ffp-contract=off so the
// float results match the reference's own host code bit for bit.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <thread>

#include "gs_parallel.h"
#include <vector>

#include "../../include/gs_api.h"

namespace {

void cross3(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

void normalize3(float v[3]) {
    float len = std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    if (len <= 1e-8f) return;
    v[0] /= len;
    v[1] /= len;
    v[2] /= len;
}

// Camera forward vector: src/camera.cpp:22-33.
void forward_of(float yaw, float pitch, bool z_up, float out[3]) {
    if (z_up) {
        float cp = std::cos(pitch);
        out[0] = std::sin(yaw) * cp;
        out[1] = std::cos(yaw) * cp;
        out[2] = std::sin(pitch);
        return;
    }
    out[0] = std::cos(pitch) * std::sin(yaw);
    out[1] = std::sin(pitch);
    out[2] = std::cos(pitch) * std::cos(yaw);
}

// View matrix, column-major: src/camera.cpp:137-191.
void view_matrix(const float pos[3], float yaw, float pitch, bool z_up, float m[16]) {
    float f[3], r[3], u[3];
    forward_of(yaw, pitch, z_up, f);
    if (z_up) {
        float back[3] = {-f[0], -f[1], -f[2]};
        const float world_up[3] = {0.0f, 0.0f, 1.0f};
        cross3(f, world_up, r);
        normalize3(r);
        cross3(back, r, u);
        std::memset(m, 0, 16 * sizeof(float));
        for (int k = 0; k < 3; ++k) {
            m[k * 4] = -r[k];
            m[k * 4 + 1] = -u[k];
            m[k * 4 + 2] = back[k];
            m[12] += r[k] * pos[k];
            m[13] += u[k] * pos[k];
            m[14] -= back[k] * pos[k];
        }
        m[15] = 1.0f;
        return;
    }
    const float world_up[3] = {0.0f, 1.0f, 0.0f};
    cross3(f, world_up, r);
    normalize3(r);
    cross3(r, f, u);
    m[0] = r[0]; m[1] = u[0]; m[2] = -f[0]; m[3] = 0.0f;
    m[4] = r[1]; m[5] = u[1]; m[6] = -f[1]; m[7] = 0.0f;
    m[8] = r[2]; m[9] = u[2]; m[10] = -f[2]; m[11] = 0.0f;
    m[12] = -(r[0] * pos[0] + r[1] * pos[1] + r[2] * pos[2]);
    m[13] = -(u[0] * pos[0] + u[1] * pos[1] + u[2] * pos[2]);
    m[14] = (f[0] * pos[0] + f[1] * pos[1] + f[2] * pos[2]);
    m[15] = 1.0f;
}

// Hybrid perspective/orthographic projection: src/camera.cpp:217-245.
void proj_matrix(float fov_y, float near_plane, float far_plane, float ortho_size, float t, float aspect,
                 float m[16]) {
    const float n = near_plane, fa = far_plane;
    float persp[16] = {};
    float f = 1.0f / std::tan(fov_y * 0.5f);
    persp[0] = -f / aspect;
    persp[5] = -f;
    persp[10] = (n + fa) / (n - fa);
    persp[11] = -1.0f;
    persp[14] = (2.0f * n * fa) / (n - fa);
    float ortho[16] = {};
    float half_h = ortho_size;
    float half_w = half_h * aspect;
    ortho[0] = -1.0f / half_w;
    ortho[5] = -1.0f / half_h;
    ortho[10] = 2.0f / (n - fa);
    ortho[14] = (n + fa) / (n - fa);
    ortho[15] = 1.0f;
    for (int i = 0; i < 16; ++i) m[i] = persp[i] * (1.0f - t) + ortho[i] * t;
}

float sigmoid(float x) { return 1.0f / (1.0f + std::exp(-x)); }

// Attribute transforms of src/gaussian_loader_ply.cpp:148-203 and the row
// packing of src/gaussian.cpp:53-73.  `get(name_index)` returns a pointer to
// the attribute or nullptr when the property is absent.
enum Attr {
    A_X, A_Y, A_Z, A_S0, A_S1, A_S2, A_R0, A_R1, A_R2, A_R3, A_OP, A_DC0, A_DC1, A_DC2, A_REST0,
    A_COUNT = A_REST0 + 45
};

template <class Get>
void pack_row(Get get, float* d) {
    std::memset(d, 0, 64 * sizeof(float));
    auto val = [&](int a) {
        float v;
        std::memcpy(&v, get(a), 4);
        return v;
    };
    d[0] = val(A_X);
    d[1] = val(A_Y);
    d[2] = val(A_Z);
    if (get(A_S0)) {
        d[4] = std::exp(val(A_S0));
        d[5] = std::exp(val(A_S1));
        d[6] = std::exp(val(A_S2));
    } else {
        d[4] = d[5] = d[6] = 0.01f;
    }
    if (get(A_R0)) {
        float rw = val(A_R0), rx = val(A_R1), ry = val(A_R2), rz = val(A_R3);
        float len = std::sqrt(rw * rw + rx * rx + ry * ry + rz * rz);
        if (len > 1e-8f) {
            rw /= len;
            rx /= len;
            ry /= len;
            rz /= len;
        }
        d[8] = rw; d[9] = rx; d[10] = ry; d[11] = rz;
    } else {
        d[8] = 1.0f;
    }
    d[3] = get(A_OP) ? sigmoid(val(A_OP)) : 1.0f;
    if (get(A_DC0)) {
        d[12] = val(A_DC0);
        d[13] = val(A_DC1);
        d[14] = val(A_DC2);
    }
    for (int k = 0; k < 15; ++k) {
        d[16 + k * 3 + 0] = get(A_REST0 + k) ? val(A_REST0 + k) : 0.0f;
        d[16 + k * 3 + 1] = get(A_REST0 + 15 + k) ? val(A_REST0 + 15 + k) : 0.0f;
        d[16 + k * 3 + 2] = get(A_REST0 + 30 + k) ? val(A_REST0 + 30 + k) : 0.0f;
    }
}

std::string attr_name(int a) {
    static const char* base[] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2",
                                 "rot_3", "opacity", "f_dc_0", "f_dc_1", "f_dc_2"};
    if (a < A_REST0) return base[a];
    return "f_rest_" + std::to_string(a - A_REST0);
}

int type_size(const char* t) {
    if (!std::strcmp(t, "float") || !std::strcmp(t, "float32") || !std::strcmp(t, "int") ||
        !std::strcmp(t, "int32") || !std::strcmp(t, "uint") || !std::strcmp(t, "uint32"))
        return 4;
    if (!std::strcmp(t, "double") || !std::strcmp(t, "float64")) return 8;
    if (!std::strcmp(t, "uchar") || !std::strcmp(t, "uint8")) return 1;
    if (!std::strcmp(t, "short") || !std::strcmp(t, "int16") || !std::strcmp(t, "ushort") ||
        !std::strcmp(t, "uint16"))
        return 2;
    return 4;
}

}  // namespace

extern "C" int gs_camera_uniforms(const float position[3], float yaw, float pitch, float fov_y, float near_plane,
                                  float far_plane, int z_up, float ortho_size, float ortho_blend, int width,
                                  int height, int webgpu, gs_camera* out) {
    if (!position || !out || width <= 0 || height <= 0) return GS_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    view_matrix(position, yaw, pitch, z_up != 0, out->view);
    const float aspect = (float)width / (float)height;   // src/main.cpp:1231
    proj_matrix(fov_y, near_plane, far_plane, ortho_size, ortho_blend, aspect, out->proj);
    out->viewport[0] = (float)width;                    // src/main.cpp:1264-1281
    out->viewport[1] = (float)height;
    out->orthographic = ortho_blend;
    out->persp_focal = (1.0f / std::tan(fov_y * 0.5f)) * (float)height * 0.5f;
    out->ortho_focal = (float)height / (2.0f * ortho_size);
    out->clip_y_sign = webgpu ? -1.0f : 1.0f;
    out->clip_z_01 = webgpu ? 1.0f : 0.0f;
    return GS_OK;
}

extern "C" int gs_pack_raw(const float* raw, uint64_t count, float* rows) {
    if ((!raw || !rows) && count) return GS_ERR_BAD_ARG;
    // raw order: x y z, f_dc_0..2, f_rest_0..44, opacity, scale_0..2, rot_0..3 (59 floats)
    static int off[A_COUNT];
    static bool init = false;
    if (!init) {
        off[A_X] = 0; off[A_Y] = 1; off[A_Z] = 2;
        off[A_DC0] = 3; off[A_DC1] = 4; off[A_DC2] = 5;
        for (int k = 0; k < 45; ++k) off[A_REST0 + k] = 6 + k;
        off[A_OP] = 51;
        off[A_S0] = 52; off[A_S1] = 53; off[A_S2] = 54;
        off[A_R0] = 55; off[A_R1] = 56; off[A_R2] = 57; off[A_R3] = 58;
        init = true;
    }
    for (uint64_t i = 0; i < count; ++i) {
        const float* r = raw + i * 59;
        pack_row([&](int a) -> const void* { return r + off[a]; }, rows + i * 64);
    }
    return GS_OK;
}

namespace {
int64_t load_ply(const char* path, float* rows, uint64_t capacity) {
    if (!path) return GS_ERR_BAD_ARG;
    std::unique_ptr<FILE, int (*)(FILE*)> file(std::fopen(path, "rb"), &std::fclose);   // closed on every return
    FILE* const f = file.get();
    if (!f) return GS_ERR_BAD_ARG;
    // Header rules of src/gaussian_loader_ply.cpp:27-75: lines read 511
    // bytes at a time; any "format" line without binary_little_endian fails
    // (no format line is accepted); the vertex count is atoi's, as 32 bits;
    // every vertex property advances the stride, and the first 128 keep
    // their names for lookup.
    char line[512];
    uint32_t vertex_count = 0;
    bool in_vertex = false, header_done = false;
    int stride = 0;
    std::vector<std::pair<std::string, int>> props;  // name, byte offset
    while (std::fgets(line, sizeof(line), f)) {
        size_t len = std::strlen(line);
        while (len > 0 && (line[len - 1] == '\n' || line[len - 1] == '\r')) line[--len] = 0;
        if (!std::strcmp(line, "end_header")) { header_done = true; break; }
        if (!std::strncmp(line, "format ", 7) && !std::strstr(line, "binary_little_endian")) {
            return GS_ERR_BAD_ARG;
        }
        if (!std::strncmp(line, "element vertex ", 15)) {
            vertex_count = (uint32_t)std::atoi(line + 15);
            in_vertex = true;
            continue;
        }
        if (!std::strncmp(line, "element ", 8)) { in_vertex = false; continue; }
        if (in_vertex && !std::strncmp(line, "property ", 9)) {
            char type[32], name[64];
            if (std::sscanf(line, "property %31s %63s", type, name) == 2) {
                if (props.size() < 128) props.emplace_back(name, stride);
                stride += type_size(type);
            }
        }
    }
    if (!header_done || vertex_count == 0) {
        return GS_ERR_BAD_ARG;
    }
    int off[A_COUNT];
    for (int a = 0; a < A_COUNT; ++a) {
        off[a] = -1;
        std::string nm = attr_name(a);
        for (auto& p : props)
            if (p.first == nm) { off[a] = p.second; break; }
    }
    if (off[A_X] < 0 || off[A_Y] < 0 || off[A_Z] < 0) { return GS_ERR_BAD_ARG; }
    // scale_0, rot_0 and f_dc_0 each stand for their whole group: a file
    // that names the first without the others has no defined decode (the
    // reference reads a byte before the row for the missing ones), so it is
    // rejected.
    for (int first : {A_S0, A_R0, A_DC0}) {
        const int last = first == A_R0 ? first + 3 : first + 2;
        for (int a = first + 1; a <= last && off[first] >= 0; ++a)
            if (off[a] < 0) { return GS_ERR_BAD_ARG; }
    }
    // the body must hold every vertex (the reference's loader fails on a short read)
    const long body_at = std::ftell(f);
    long body_end = -1;
    if (body_at >= 0 && !std::fseek(f, 0, SEEK_END)) body_end = std::ftell(f);
    if (body_end < body_at || std::fseek(f, body_at, SEEK_SET) ||
        (uint64_t)(body_end - body_at) < (uint64_t)vertex_count * (uint64_t)stride) {
        return GS_ERR_BAD_ARG;
    }
    if (!rows) { return (int64_t)vertex_count; }
    const uint64_t n = vertex_count < capacity ? vertex_count : capacity;
    // Blocks of rows: while worker threads transform block b (rows are
    // independent, so the result does not depend on the split), this thread
    // reads block b + 1.  Every value is read as 4 bytes whatever its
    // declared size: the padding keeps a narrower last property of the last
    // row inside the buffer.
    const uint64_t batch = 65536;
    std::vector<unsigned char> raw[2];
    raw[0].assign((size_t)batch * stride + 4, 0);
    raw[1].assign((size_t)batch * stride + 4, 0);
    auto transform = [&](const unsigned char* buf, uint64_t first, uint64_t lo, uint64_t hi) {
        for (uint64_t k = lo; k < hi; ++k) {
            const unsigned char* v = buf + k * stride;
            pack_row([&](int a) -> const void* { return off[a] >= 0 ? v + off[a] : nullptr; },
                     rows + (first + k) * 64);
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned workers = hw > 1 ? (hw - 1 < 15 ? hw - 1 : 15) : 0;
    // one set of worker threads for the whole body (the other loaders use
    // gs::parallel_ranges; here the calling thread also reads the next block)
    gs::WorkerPool pool(n >= 2 * 2048 ? workers : 0);
    uint64_t cnt = n < batch ? n : batch;
    bool ok = std::fread(raw[0].data(), stride, cnt, f) == cnt;
    for (uint64_t i = 0, b = 0; ok && i < n; i += cnt, b ^= 1) {
        cnt = n - i < batch ? n - i : batch;
        const uint64_t next = n - (i + cnt) < batch ? n - (i + cnt) : batch;
        const unsigned char* buf = raw[b].data();
        bool next_ok = true;
        // the workers transform this block while this thread reads the next
        // one, then takes its own slice of the block
        pool.run(cnt, [&](uint64_t lo, uint64_t hi) {
            if (lo == 0 && next) next_ok = std::fread(raw[b ^ 1].data(), stride, next, f) == next;
            transform(buf, i, lo, hi);
        });
        ok = next_ok;
    }
    return ok ? (int64_t)vertex_count : GS_ERR_BAD_ARG;
}
}  // namespace

extern "C" int64_t gs_load_ply(const char* path, float* rows, uint64_t capacity) {
    try {
        return load_ply(path, rows, capacity);
    } catch (const std::bad_alloc&) {   // a header declaring more properties than memory holds
        return GS_ERR_OOM;
    }
}

namespace {
bool ends_with_ci(const char* s, const char* suffix) {
    const size_t sl = std::strlen(s), tl = std::strlen(suffix);
    if (tl > sl) return false;
    s += sl - tl;
    for (size_t i = 0; i < tl; ++i)
        if (std::tolower((unsigned char)s[i]) != std::tolower((unsigned char)suffix[i])) return false;
    return true;
}
}  // namespace

extern "C" int64_t gs_load_scene(const char* path, float* rows, uint64_t capacity) {
    if (!path) return GS_ERR_BAD_ARG;
    // load_gaussian_scene (src/gaussian.cpp:27-40): the format by the file
    // name's extension, case-insensitively
    if (ends_with_ci(path, ".gsanim")) {
        gs_gsanim* a = nullptr;
        const int rc = gs_gsanim_load(path, &a);
        if (rc != GS_OK) return rc;
        gs_gsanim_info info;
        gs_gsanim_get_info(a, &info);
        int64_t n = (int64_t)info.gaussian_count;
        if (rows) {
            if (capacity >= info.gaussian_count) {
                gs_gsanim_rows(a, rows);
            } else {
                std::vector<float> all;
                try {
                    all.resize((size_t)info.gaussian_count * 64);
                } catch (const std::bad_alloc&) {
                    gs_gsanim_free(a);
                    return GS_ERR_OOM;
                }
                gs_gsanim_rows(a, all.data());
                std::memcpy(rows, all.data(), (size_t)capacity * 64 * sizeof(float));
            }
        }
        gs_gsanim_free(a);
        return n;
    }
    if (ends_with_ci(path, ".ply")) return gs_load_ply(path, rows, capacity);
    if (ends_with_ci(path, ".sog")) return gs_load_sog(path, rows, capacity);
    return GS_ERR_FORMAT;
}
