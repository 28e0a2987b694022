// Runs the reference's own shader stages (shaders/cull.glsl, sort.glsl,
// splat.glsl, gps.glsl, accum.glsl), translated to C++ by extract.py and compiled against
// glsl.h, over whole frames on the CPU.
//
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/libglslref.so from the
// reference's shader sources; the tests compare it with the oracle
// (gs_oracle.c), and through the oracle with the CUDA path.
//
// Each entry point mirrors the oracle function of the same name (oc_cull,
// oc_sort_pairs, oc_composite_alpha, oc_stochastic_sample, oc_gps_frame,
// oc_accum, oc_taa, oc_display):
// same arguments, same output layout.  Only the fixed-function steps between
// the stages are written here, as the oracle defines them: the quad's
// rasterization (viewport transform, 1/256-pixel snap, pixel centres at
// k + 0.5, left and top edges inclusive, primitives whose constant NDC depth
// lies outside [-1, 1] clipped), the premultiplied blend
// (ONE, ONE_MINUS_SRC_ALPHA) in draw order, the D24 LESS depth test, and
// varyings that are constant over a primitive passed through unchanged.
#include "glsl.h"

#include <ucontext.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

// Workgroups of compute stages with barrier(): each of the 256 invocations
// is a fiber (ucontext) on its own stack; the scheduler resumes them in
// invocation order, each running to its next barrier() or its end, until all
// have ended.  One phase thus completes for every invocation before any
// starts the next, as barrier() requires, with no concurrency (atomics on
// shared variables are plain read-modify-writes).
namespace wg {
constexpr int kLocal = 256;
constexpr size_t kStack = 64 * 1024;
struct Fiber {
    ucontext_t ctx;
    bool done;
};
ucontext_t sched;
Fiber fibers[kLocal];
std::vector<char> stacks;
int cur = 0;
void (*entry)() = nullptr;

void trampoline() {
    entry();
    fibers[cur].done = true;   // returns to uc_link: the scheduler
}
inline void barrier() { swapcontext(&fibers[cur].ctx, &sched); }

// Runs one workgroup of main_fn; set_ids(i) sets the stage's built-in ids
// for invocation i before each resume.
template <typename SetIds> void run(void (*main_fn)(), SetIds set_ids) {
    if (stacks.empty()) stacks.resize((size_t)kLocal * kStack);
    entry = main_fn;
    for (int i = 0; i < kLocal; ++i) {
        getcontext(&fibers[i].ctx);
        fibers[i].ctx.uc_stack.ss_sp = stacks.data() + (size_t)i * kStack;
        fibers[i].ctx.uc_stack.ss_size = kStack;
        fibers[i].ctx.uc_link = &sched;
        makecontext(&fibers[i].ctx, trampoline, 0);
        fibers[i].done = false;
    }
    for (bool live = true; live;) {
        live = false;
        for (int i = 0; i < kLocal; ++i) {
            if (fibers[i].done) continue;
            cur = i;
            set_ids(i);
            swapcontext(&sched, &fibers[i].ctx);
            live = true;
        }
    }
}
}  // namespace wg

#define GLSL_WORKGROUP_BUILTINS                             \
    uvec3 gl_GlobalInvocationID, gl_LocalInvocationID, gl_WorkGroupID; \
    inline void barrier() { wg::barrier(); }                \
    inline void memoryBarrierShared() {}

namespace st_radix_hist {
using namespace glsl;
GLSL_WORKGROUP_BUILTINS
#include "radix_hist_cs.inc"
}  // namespace st_radix_hist

namespace st_radix_prefix {
using namespace glsl;
GLSL_WORKGROUP_BUILTINS
#include "radix_prefix_cs.inc"
}  // namespace st_radix_prefix

namespace st_radix_scatter {
using namespace glsl;
GLSL_WORKGROUP_BUILTINS
#include "radix_scatter_cs.inc"
}  // namespace st_radix_scatter

namespace st_cull_reset {
using namespace glsl;
uvec3 gl_GlobalInvocationID;
#include "cull_reset_cs.inc"
}  // namespace st_cull_reset

namespace st_cull {
using namespace glsl;
uvec3 gl_GlobalInvocationID;
#include "cull_cs.inc"
}  // namespace st_cull

namespace st_splat_vs {
using namespace glsl;
int gl_VertexIndex, gl_InstanceIndex;
vec4 gl_Position;
#include "splat_vs.inc"
}  // namespace st_splat_vs

namespace st_splat_fs {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
// The oracle's alpha composite takes the C library's expf (the CUDA path is
// compared with it within a tolerance); the stochastic sample below keeps
// glsl.h's oc_expf, which the CUDA path reproduces bit for bit.
inline float exp(float x) { return ::expf(x); }
#include "splat_fs.inc"
}  // namespace st_splat_fs

namespace st_splat_stoch_fs {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "splat_stochastic_fs.inc"
}  // namespace st_splat_stoch_fs

namespace st_gps_clear {
using namespace glsl;
uvec3 gl_GlobalInvocationID;
#include "gps_clear_cs.inc"
}  // namespace st_gps_clear

namespace st_gps_expand {
using namespace glsl;
uvec3 gl_GlobalInvocationID;
#include "gps_expand_cs.inc"
}  // namespace st_gps_expand

namespace st_gps_splat {
using namespace glsl;
uvec3 gl_GlobalInvocationID;
#include "gps_splat_cs.inc"
}  // namespace st_gps_splat

namespace st_gps_resolve {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "gps_resolve_fs.inc"
}  // namespace st_gps_resolve

namespace st_accum {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "accum_fs.inc"
}  // namespace st_accum

namespace st_blit {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "blit_fs.inc"
}  // namespace st_blit

namespace st_display {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "layers_display_fs.inc"
}  // namespace st_display

namespace st_taa {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "taa_accum_fs.inc"
}  // namespace st_taa

// The reference's mat4_inverse (src/renderer.cpp:86-206), cut from its
// source unchanged.
namespace ref_renderer {
#include "mat4_inverse.inc"
}  // namespace ref_renderer

namespace {

using glsl::mat4;
using glsl::vec2;
using glsl::vec4;

mat4 mat4_of(const float* m) {
    mat4 r;
    for (int c = 0; c < 4; ++c)
        for (int i = 0; i < 4; ++i) r.c[c].d[i] = m[c * 4 + i];
    return r;
}

vec4 vec4_of(const float* v) { return vec4(v[0], v[1], v[2], v[3]); }

// Pixel rectangle [i0, i1) x [j0, j1) (GL rows, bottom first) whose centres a
// quad covers, from its corners in clip space (w = 1); false when the quad
// is clipped or covers no pixel centre.
int64_t floor_div256(int64_t a) { return a >= 0 ? a / 256 : -((-a + 255) / 256); }
int64_t ceil_div256(int64_t a) { return -floor_div256(-a); }
int64_t snap256(float w) {
    float s = w * 256.0f;
    if (s > 1.0e15f) s = 1.0e15f;
    if (s < -1.0e15f) s = -1.0e15f;
    return (int64_t)std::rint(s);
}

bool quad_rect(const vec4 pos[6], int width, int height, int rect[4]) {
    const float z = pos[0].z / pos[0].w;
    if (!(z >= -1.0f && z <= 1.0f)) return false;
    const float hw = (float)width * 0.5f, hh = (float)height * 0.5f;
    int64_t X0 = INT64_MAX, X1 = INT64_MIN, Y0 = INT64_MAX, Y1 = INT64_MIN;
    for (int v = 0; v < 6; ++v) {
        const int64_t X = snap256((pos[v].x / pos[v].w) * hw + hw);
        const int64_t Y = snap256((pos[v].y / pos[v].w) * hh + hh);
        X0 = X < X0 ? X : X0;
        X1 = X > X1 ? X : X1;
        Y0 = Y < Y0 ? Y : Y0;
        Y1 = Y > Y1 ? Y : Y1;
    }
    int64_t i0 = ceil_div256(X0 - 128), i1 = ceil_div256(X1 - 128);
    int64_t j0 = floor_div256(Y0 - 128) + 1, j1 = floor_div256(Y1 - 128) + 1;
    i0 = i0 < 0 ? 0 : i0;
    j0 = j0 < 0 ? 0 : j0;
    i1 = i1 > width ? width : i1;
    j1 = j1 > height ? height : j1;
    if (i1 <= i0 || j1 <= j0) return false;
    rect[0] = (int)i0;
    rect[1] = (int)i1;
    rect[2] = (int)j0;
    rect[3] = (int)j1;
    return true;
}

// The vertex stage for instance s: its six vertices' positions; the
// varyings (equal for every vertex of the instance) are left in st_splat_vs.
void run_splat_vs(uint32_t s, vec4 pos[6]) {
    namespace V = st_splat_vs;
    for (int v = 0; v < 6; ++v) {
        V::gl_VertexIndex = v;
        V::gl_InstanceIndex = (int)s;
        V::stage_main();
        pos[v] = V::gl_Position;
    }
}

void setup_splat_vs(const uint32_t* ids, const float* projected, float vp_w, float vp_h, float clip_y_sign,
                    float jx, float jy) {
    namespace V = st_splat_vs;
    V::projected_splats = reinterpret_cast<V::ProjectedSplatData*>(const_cast<float*>(projected));
    V::splat_ids = reinterpret_cast<V::SplatIdData*>(const_cast<uint32_t*>(ids));
    V::viewport = vec2(vp_w, vp_h);
    V::jitter_px = vec2(jx, jy);
    V::clip_y_sign = clip_y_sign;
}

template <typename FS> void copy_varyings(FS& fs) {
    namespace V = st_splat_vs;
    fs.frag_color = V::frag_color;
    fs.frag_opacity = V::frag_opacity;
    fs.frag_alpha_power_cutoff = V::frag_alpha_power_cutoff;
    fs.frag_center = V::frag_center;
    fs.frag_conic = V::frag_conic;
    fs.frag_splat_id = V::frag_splat_id;
}

struct SplatFsVars {
    glsl::vec3& frag_color = st_splat_fs::frag_color;
    float& frag_opacity = st_splat_fs::frag_opacity;
    float& frag_alpha_power_cutoff = st_splat_fs::frag_alpha_power_cutoff;
    glsl::vec2& frag_center = st_splat_fs::frag_center;
    glsl::vec3& frag_conic = st_splat_fs::frag_conic;
    uint32_t& frag_splat_id = st_splat_fs::frag_splat_id;
};
struct StochFsVars {
    glsl::vec3& frag_color = st_splat_stoch_fs::frag_color;
    float& frag_opacity = st_splat_stoch_fs::frag_opacity;
    float& frag_alpha_power_cutoff = st_splat_stoch_fs::frag_alpha_power_cutoff;
    glsl::vec2& frag_center = st_splat_stoch_fs::frag_center;
    glsl::vec3& frag_conic = st_splat_stoch_fs::frag_conic;
    uint32_t& frag_splat_id = st_splat_stoch_fs::frag_splat_id;
};

// Top-first image <-> GL rows (bottom first).
void flip_rows(const float* src, float* dst, int width, int height, int ch) {
    for (int y = 0; y < height; ++y)
        std::memcpy(dst + (size_t)(height - 1 - y) * width * ch, src + (size_t)y * width * ch,
                    (size_t)width * ch * sizeof(float));
}

}  // namespace

extern "C" {

int ref_mat4_inverse(const float* m, float* out) { return ref_renderer::mat4_inverse(m, out) ? 1 : 0; }

// cull_reset_cs then cull_cs over n rows (shaders/cull.glsl:3-476).  cam is
// the 40-float CameraUniforms block (view, proj, viewport, orthographic,
// persp_focal, ortho_focal, clip_y_sign, clip_z_01, pad).  words, when not
// null, is the animation buffer: int8 deltas of anim_states states (4 per
// word) or, with layer_count > 0, half-float layers (2 per word).
void glsl_cull(const float* rows, uint32_t n, const float* cam, int sh_degree, float sh_lod_distance,
               int collect_stats, const uint32_t* words, int anim_states, int state_a, int state_b,
               float weight, const float* scales48, int layer_count, const float* layer_weights,
               uint32_t* ids, uint32_t* keys, float* projected, uint32_t* visible_count, uint32_t* diag) {
    namespace R = st_cull_reset;
    namespace C = st_cull;
    R::sort_count = (int)n;
    R::visible_count = reinterpret_cast<R::ResetUIntData*>(visible_count);
    R::output_splat_ids = reinterpret_cast<R::ResetUIntData*>(ids);
    R::output_depth_keys = reinterpret_cast<R::ResetUIntData*>(keys);
    R::splat_diagnostics = reinterpret_cast<R::ResetUIntData*>(diag);
    for (uint32_t i = 0; i < (n ? n : 1u); ++i) {
        R::gl_GlobalInvocationID = glsl::uvec3(i, 0u, 0u);
        R::stage_main();
    }

    C::view = mat4_of(cam);
    C::proj = mat4_of(cam + 16);
    C::viewport = vec2(cam[32], cam[33]);
    C::gaussian_count = (int)n;
    C::gaussian_first = 0;
    C::orthographic = cam[34];
    C::persp_focal = cam[35];
    C::ortho_focal = cam[36];
    C::clip_y_sign = cam[37];
    C::clip_z_01 = cam[38];
    C::collect_stats = collect_stats;
    C::sh_degree = sh_degree;
    C::sh_lod_distance = sh_lod_distance;
    C::effect_center_radius = vec4(0.0f);
    C::effect_params = vec4(0.0f);
    C::effect_color = vec4(0.0f);
    C::gaussian_data = reinterpret_cast<C::CullGaussianData*>(const_cast<float*>(rows));
    C::output_splat_ids = reinterpret_cast<C::UIntData*>(ids);
    C::output_depth_keys = reinterpret_cast<C::UIntData*>(keys);
    C::projected_splats = reinterpret_cast<C::CullProjectedSplatData*>(projected);
    C::visible_count = reinterpret_cast<C::UIntData*>(visible_count);
    C::splat_diagnostics = reinterpret_cast<C::UIntData*>(diag);
    C::animation_deltas = reinterpret_cast<C::UIntData*>(const_cast<uint32_t*>(words));
    C::layer_weights = reinterpret_cast<C::LayerWeight*>(const_cast<float*>(layer_weights));
    C::animation_count = words ? (int)n : 0;
    C::animation_state_a = state_a;
    C::animation_state_b = state_b;
    C::animation_weight = weight;
    for (int k = 0; k < 12; ++k) C::animation_scales[k] = scales48 ? vec4_of(scales48 + 4 * k) : vec4(0.0f);
    C::layer_count = words ? layer_count : 0;
    (void)anim_states;
    for (uint32_t i = 0; i < n; ++i) {
        C::current_layer = -1;
        C::gl_GlobalInvocationID = glsl::uvec3(i, 0u, 0u);
        C::stage_main();
    }
}

// splat_vs + splat_fs over the sorted draw order with the premultiplied
// blend, as oc_composite_alpha (FP32 blending): out is top-first RGBA.
uint64_t glsl_composite_alpha(const uint32_t* sorted_ids, uint32_t count, const float* projected, int width,
                              int height, float vp_w, float vp_h, float clip_y_sign, float bg, float jx, float jy,
                              float* out) {
    namespace F = st_splat_fs;
    const size_t npix = (size_t)width * (size_t)height;
    std::vector<float> img(npix * 4);
    for (size_t p = 0; p < npix; ++p) {
        img[p * 4 + 0] = bg;
        img[p * 4 + 1] = bg;
        img[p * 4 + 2] = bg;
        img[p * 4 + 3] = 0.0f;
    }
    setup_splat_vs(sorted_ids, projected, vp_w, vp_h, clip_y_sign, jx, jy);
    SplatFsVars fs;
    uint64_t frags = 0;
    for (uint32_t s = 0; s < count; ++s) {
        vec4 pos[6];
        run_splat_vs(s, pos);
        int rc[4];
        if (!quad_rect(pos, width, height, rc)) continue;
        copy_varyings(fs);
        for (int j = rc[2]; j < rc[3]; ++j) {
            for (int i = rc[0]; i < rc[1]; ++i) {
                F::gl_FragCoord = vec4((float)i + 0.5f, (float)j + 0.5f, pos[0].z * 0.5f + 0.5f, 1.0f);
                F::gl_discarded = false;
                F::stage_main();
                if (F::gl_discarded) continue;
                const vec4 src = F::out_color;
                float* d = &img[((size_t)j * width + i) * 4];
                const float om = 1.0f - src.w;
                for (int k = 0; k < 4; ++k) d[k] = src.d[k] + om * d[k];
                ++frags;
            }
        }
    }
    flip_rows(img.data(), out, width, height, 4);
    return frags;
}

// splat_vs + splat_stochastic_fs with a D24 LESS depth test (writes on), as
// oc_stochastic_sample: out_rgba (top-first, optionally quantised to RGBA8)
// and out_depth (the D24 value / (2^24 - 1)).
uint64_t glsl_stochastic_sample(const uint32_t* ids, uint32_t count, const float* projected, int width, int height,
                                float vp_w, float vp_h, float clip_y_sign, float bg, float jx, float jy,
                                float frame_seed, int rgba8, float* out_rgba, float* out_depth) {
    namespace F = st_splat_stoch_fs;
    const size_t npix = (size_t)width * (size_t)height;
    std::vector<uint32_t> zbuf(npix, 16777215u);
    std::vector<float> col(npix * 4);
    for (size_t p = 0; p < npix; ++p) {
        col[p * 4 + 0] = bg;
        col[p * 4 + 1] = bg;
        col[p * 4 + 2] = bg;
        col[p * 4 + 3] = 0.0f;
    }
    setup_splat_vs(ids, projected, vp_w, vp_h, clip_y_sign, jx, jy);
    F::frame_seed = frame_seed;
    StochFsVars fs;
    uint64_t kept = 0;
    for (uint32_t s = 0; s < count; ++s) {
        vec4 pos[6];
        run_splat_vs(s, pos);
        int rc[4];
        if (!quad_rect(pos, width, height, rc)) continue;
        copy_varyings(fs);
        const float zw = pos[0].z * 0.5f + 0.5f;
        const float zc = zw < 0.0f ? 0.0f : (zw > 1.0f ? 1.0f : zw);
        const uint32_t z24 = (uint32_t)std::rint(zc * 16777215.0f);
        for (int j = rc[2]; j < rc[3]; ++j) {
            for (int i = rc[0]; i < rc[1]; ++i) {
                const size_t p = (size_t)j * width + i;
                F::gl_FragCoord = vec4((float)i + 0.5f, (float)j + 0.5f, zw, 1.0f);
                F::gl_discarded = false;
                F::stage_main();
                if (F::gl_discarded || !(z24 < zbuf[p])) continue;
                zbuf[p] = z24;
                for (int k = 0; k < 4; ++k) col[p * 4 + k] = F::out_color.d[k];
                ++kept;
            }
        }
    }
    for (int j = 0; j < height; ++j) {
        for (int i = 0; i < width; ++i) {
            const size_t p = (size_t)j * width + i, o = (size_t)(height - 1 - j) * width + i;
            for (int k = 0; k < 4; ++k) {
                float v = col[p * 4 + k];
                if (rgba8) v = std::rint((v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v)) * 255.0f) / 255.0f;
                out_rgba[o * 4 + k] = v;
            }
            out_depth[o] = (float)zbuf[p] / 16777215.0f;
        }
    }
    return kept;
}

// gps_clear_cs, gps_expand_cs, gps_splat_cs and gps_resolve_fs
// (shaders/gps.glsl), as oc_gps_frame: top-first out_rgba and out_depth,
// work_stats = {requested work items, overflow flag}.
void glsl_gps_frame(const uint32_t* ids, uint32_t count, const float* projected, int width, int height,
                    int supersample, uint32_t max_work_items, float clip_z_01, int linear_color, float frame_seed,
                    float bg, float* out_rgba, float* out_depth, uint32_t* work_stats) {
    namespace GC = st_gps_clear;
    namespace GE = st_gps_expand;
    namespace GS = st_gps_splat;
    namespace GR = st_gps_resolve;
    const int ss = supersample < 1 ? 1 : (supersample > 4 ? 4 : supersample);
    const uint32_t cap = max_work_items < 1u ? 1u : max_work_items;
    const uint32_t gw = (uint32_t)width * ss, gh = (uint32_t)height * ss;
    const size_t gpix = (size_t)gw * gh;
    std::vector<uint32_t> keys(gpix), colors(gpix), wc(2, 0u), work((size_t)cap * 2);
    std::vector<float> prep((size_t)(count ? count : 1) * 12, 0.0f);

    GC::pixel_count = (int)gpix;
    GC::pixels_per_row = (int)gpix;
    GC::gps_depth_keys = reinterpret_cast<GC::GpsUIntData*>(keys.data());
    GC::gps_colors = reinterpret_cast<GC::GpsUIntData*>(colors.data());
    GC::work_count = reinterpret_cast<GC::GpsUIntData*>(wc.data());
    for (size_t p = 0; p < gpix; ++p) {
        GC::gl_GlobalInvocationID = glsl::uvec3((uint32_t)p, 0u, 0u);
        GC::stage_main();
    }

    GE::gaussian_count = (int)count;
    GE::max_work_items = (int)cap;
    GE::supersample_factor = (float)ss;
    GE::clip_z_01 = clip_z_01;
    GE::linear_color = linear_color;
    GE::projected_splats = reinterpret_cast<GE::GpsExpandProjectedSplatData*>(const_cast<float*>(projected));
    GE::work_count = reinterpret_cast<GE::GpsExpandUIntData*>(wc.data());
    GE::point_work = reinterpret_cast<GE::GpsWorkData*>(work.data());
    GE::splat_ids = reinterpret_cast<GE::GpsExpandSplatIdData*>(const_cast<uint32_t*>(ids));
    GE::prepared_splats = reinterpret_cast<GE::GpsPreparedData*>(prep.data());
    for (uint32_t i = 0; i < count; ++i) {
        GE::gl_GlobalInvocationID = glsl::uvec3(i, 0u, 0u);
        GE::stage_main();
    }

    GS::viewport = vec2((float)gw, (float)gh);
    GS::max_work_items = (int)cap;
    GS::clip_z_01 = clip_z_01;
    GS::frame_seed = frame_seed;
    GS::work_items_per_row = 1 << 30;
    GS::supersample_factor = (float)ss;
    GS::prepared_splats = reinterpret_cast<GS::GpsPreparedSplatData*>(prep.data());
    GS::gps_depth_keys = reinterpret_cast<GS::GpsSplatUIntData*>(keys.data());
    GS::gps_colors = reinterpret_cast<GS::GpsSplatUIntData*>(colors.data());
    GS::point_work = reinterpret_cast<GS::GpsSplatWorkData*>(work.data());
    GS::work_count = reinterpret_cast<GS::GpsSplatUIntData*>(wc.data());
    const uint32_t actual = wc[0] < cap ? wc[0] : cap;
    for (uint32_t w = 0; w < actual; ++w) {
        GS::gl_GlobalInvocationID = glsl::uvec3(w, 0u, 0u);
        GS::stage_main();
    }

    GR::viewport = vec2((float)width, (float)height);
    GR::gps_viewport = vec2((float)gw, (float)gh);
    GR::supersample_factor = ss;
    GR::background = bg;
    GR::linear_color = linear_color;
    GR::gps_depth_keys = reinterpret_cast<GR::GpsResolveUIntData*>(keys.data());
    GR::gps_colors = reinterpret_cast<GR::GpsResolveUIntData*>(colors.data());
    GR::projected_splats = reinterpret_cast<GR::GpsResolveProjectedData*>(const_cast<float*>(projected));
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            GR::gl_FragCoord = vec4((float)x + 0.5f, (float)y + 0.5f, 0.0f, 1.0f);
            GR::gl_discarded = false;
            GR::stage_main();
            const size_t o = (size_t)(height - 1 - y) * width + x;
            for (int k = 0; k < 4; ++k) out_rgba[o * 4 + k] = GR::out_color.d[k];
            out_depth[o] = GR::out_depth.x;
        }
    }
    work_stats[0] = wc[0];
    work_stats[1] = wc[1];
}

// accum_fs (shaders/accum.glsl:19-45) over a width x height frame (any row
// order: the pass is per pixel), as oc_accum.
void glsl_accum(const float* sample, const float* history, float sample_count, int width, int height, float* out) {
    namespace A = st_accum;
    glsl::texture2D ts, th;
    ts.data = sample;
    th.data = history;
    ts.width = th.width = width;
    ts.height = th.height = height;
    A::sample_tex = ts;
    A::history_tex = th;
    A::sample_count = sample_count;
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            A::uv = vec2(((float)x + 0.5f) / (float)width, ((float)y + 0.5f) / (float)height);
            A::gl_FragCoord = vec4((float)x + 0.5f, (float)y + 0.5f, 0.0f, 1.0f);
            A::gl_discarded = false;
            A::stage_main();
            for (int k = 0; k < 4; ++k) out[((size_t)y * width + x) * 4 + k] = A::out_color.d[k];
        }
    }
}

// taa_accum_fs (shaders/accum.glsl:47-179), as oc_taa: top-first inputs and
// outputs; vo, fc, pfc and proj_z are the four vec4 uniforms.
void glsl_taa(const float* cur_color, const float* cur_depth, const float* hist_color, const float* hist_xyz,
              int width, int height, const float* inv_view, const float* prev_view, const float* vo, const float* fc,
              const float* pfc, const float* proj_z, float history_valid, float view_changed, float* out_color,
              float* out_xyz) {
    namespace T = st_taa;
    const size_t npix = (size_t)width * (size_t)height;
    std::vector<float> cc(npix * 4), cd(npix), hc(npix * 4), hx(npix * 4), oc(npix * 4), ox(npix * 4);
    flip_rows(cur_color, cc.data(), width, height, 4);
    flip_rows(cur_depth, cd.data(), width, height, 1);
    flip_rows(hist_color, hc.data(), width, height, 4);
    flip_rows(hist_xyz, hx.data(), width, height, 4);
    glsl::texture2D t_cc, t_cd, t_hc, t_hx;
    t_cc.data = cc.data();
    t_cd.data = cd.data();
    t_cd.channels = 1;
    t_hc.data = hc.data();
    t_hx.data = hx.data();
    for (glsl::texture2D* t : {&t_cc, &t_cd, &t_hc, &t_hx}) {
        t->width = width;
        t->height = height;
    }
    T::current_color_tex = t_cc;
    T::current_depth_tex = t_cd;
    T::history_color_tex = t_hc;
    T::history_xyz_tex = t_hx;
    T::inv_view = mat4_of(inv_view);
    T::prev_view = mat4_of(prev_view);
    T::viewport_orthographic = vec4_of(vo);
    T::focal_clip = vec4_of(fc);
    T::prev_focal_clip = vec4_of(pfc);
    T::proj_z = vec4_of(proj_z);
    T::history_valid = history_valid;
    T::view_changed = view_changed;
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            T::uv = vec2(((float)x + 0.5f) / (float)width, ((float)y + 0.5f) / (float)height);
            T::gl_FragCoord = vec4((float)x + 0.5f, (float)y + 0.5f, 0.0f, 1.0f);
            T::gl_discarded = false;
            T::out_color = vec4(0.0f);
            T::out_xyz = vec4(0.0f);
            T::stage_main();
            const size_t p = (size_t)y * width + x;
            for (int k = 0; k < 4; ++k) {
                oc[p * 4 + k] = T::out_color.d[k];
                ox[p * 4 + k] = T::out_xyz.d[k];
            }
        }
    }
    flip_rows(oc.data(), out_color, width, height, 4);
    flip_rows(ox.data(), out_xyz, width, height, 4);
}

// blit_fs, or with a LUT layers_display_fs (shaders/accum.glsl:181-240),
// over an RGBA16F frame, as oc_display: lut is n x n x n x 3 uint16 (z, y, x,
// rgb), null for the blit; out is RGBA32F in the input's row order.
void glsl_display(const uint16_t* in_half, int width, int height, const uint16_t* lut, int lut_size, float log2_min,
                  float log2_max, float exposure_ev, float* out) {
    const size_t npix = (size_t)width * (size_t)height;
    std::vector<float> tex(npix * 4);
    for (size_t i = 0; i < npix * 4; ++i) tex[i] = oc_half_to_float(in_half[i]);
    glsl::texture2D t;
    t.data = tex.data();
    t.width = width;
    t.height = height;
    std::vector<uint32_t> words;
    if (lut) {
        const size_t entries = (size_t)lut_size * lut_size * lut_size * 3;
        words.assign((entries + 1) / 2, 0u);
        for (size_t i = 0; i < entries; ++i) words[i / 2] |= (uint32_t)lut[i] << ((i % 2) * 16);
        st_display::linear_tex = t;
        st_display::display_lut = reinterpret_cast<st_display::LutWord*>(words.data());
        st_display::lut_size = lut_size;
        st_display::log2_min = log2_min;
        st_display::log2_max = log2_max;
        st_display::exposure_ev = exposure_ev;
    } else {
        st_blit::display_tex = t;
    }
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            const vec2 uv(((float)x + 0.5f) / (float)width, ((float)y + 0.5f) / (float)height);
            const vec4 frag((float)x + 0.5f, (float)y + 0.5f, 0.0f, 1.0f);
            vec4 c;
            if (lut) {
                st_display::uv = uv;
                st_display::gl_FragCoord = frag;
                st_display::stage_main();
                c = st_display::out_color;
            } else {
                st_blit::uv = uv;
                st_blit::gl_FragCoord = frag;
                st_blit::stage_main();
                c = st_blit::out_color;
            }
            for (int k = 0; k < 4; ++k) out[((size_t)y * width + x) * 4 + k] = c.d[k];
        }
    }
}

// radix_hist_cs, radix_prefix_cs and radix_scatter_cs for the four 8-bit
// passes of the reference's sort driver (src/renderer.cpp:1873-1962): every
// pass over all n entries, ceil(n / 256) workgroups, ping-pong buffers.
void glsl_sort_pairs(const uint32_t* keys_in, const uint32_t* ids_in, uint32_t n, uint32_t* keys_out,
                     uint32_t* ids_out) {
    namespace RH = st_radix_hist;
    namespace RP = st_radix_prefix;
    namespace RS = st_radix_scatter;
    std::vector<uint32_t> keys[2] = {std::vector<uint32_t>(keys_in, keys_in + n), std::vector<uint32_t>(n)};
    std::vector<uint32_t> ids[2] = {std::vector<uint32_t>(ids_in, ids_in + n), std::vector<uint32_t>(n)};
    if (n > 1) {   // renderer_sort_gaussians_gpu returns for a capacity of 0 or 1
        const uint32_t groups = (n + 255u) / 256u;
        std::vector<uint32_t> hist((size_t)groups * 256u);
        for (uint32_t pass = 0; pass < 4u; ++pass) {
            const int shift = (int)(pass * 8u);
            const uint32_t src = pass & 1u, dst = src ^ 1u;
            RH::sort_count = (int)n;
            RH::shift = shift;
            RH::hist_keys = reinterpret_cast<RH::RadixUIntData*>(keys[src].data());
            RH::histograms = reinterpret_cast<RH::RadixUIntData*>(hist.data());
            for (uint32_t g = 0; g < groups; ++g)
                wg::run(RH::stage_main, [&](int i) {
                    RH::gl_LocalInvocationID = glsl::uvec3((uint32_t)i, 0u, 0u);
                    RH::gl_GlobalInvocationID = glsl::uvec3(g * 256u + (uint32_t)i, 0u, 0u);
                    RH::gl_WorkGroupID = glsl::uvec3(g, 0u, 0u);
                });
            RP::group_count = (int)groups;
            RP::histograms = reinterpret_cast<RP::RadixPrefixUIntData*>(hist.data());
            wg::run(RP::stage_main, [&](int i) {
                RP::gl_LocalInvocationID = glsl::uvec3((uint32_t)i, 0u, 0u);
                RP::gl_GlobalInvocationID = glsl::uvec3((uint32_t)i, 0u, 0u);
                RP::gl_WorkGroupID = glsl::uvec3(0u, 0u, 0u);
            });
            RS::sort_count = (int)n;
            RS::shift = shift;
            RS::keys_in = reinterpret_cast<RS::RadixScatterUIntData*>(keys[src].data());
            RS::keys_out = reinterpret_cast<RS::RadixScatterUIntData*>(keys[dst].data());
            RS::ids_in = reinterpret_cast<RS::RadixScatterUIntData*>(ids[src].data());
            RS::ids_out = reinterpret_cast<RS::RadixScatterUIntData*>(ids[dst].data());
            RS::histograms = reinterpret_cast<RS::RadixScatterUIntData*>(hist.data());
            for (uint32_t g = 0; g < groups; ++g)
                wg::run(RS::stage_main, [&](int i) {
                    RS::gl_LocalInvocationID = glsl::uvec3((uint32_t)i, 0u, 0u);
                    RS::gl_GlobalInvocationID = glsl::uvec3(g * 256u + (uint32_t)i, 0u, 0u);
                    RS::gl_WorkGroupID = glsl::uvec3(g, 0u, 0u);
                });
        }
    }
    std::memcpy(keys_out, keys[0].data(), (size_t)n * 4);
    std::memcpy(ids_out, ids[0].data(), (size_t)n * 4);
}

}  // extern "C"
