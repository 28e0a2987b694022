// Test-infrastructure glue around the reference's own CPU code (compiled from
// the reference sources in place by oracle/Makefile into oracle/_ref/).
// Exposes extern "C" entry points for ctypes so tests can pin the oracle
// against the reference:
//   - gaussian_load_ply + pack_gpu_gaussians   (src/gaussian_loader_ply.cpp:14-228,
//                                                src/gaussian.cpp:53-73)
//   - cull_gaussians + sort_gaussians           (src/gaussian.cpp:77-181)
//   - camera_get_view_matrix / camera_get_proj_matrix (src/camera.cpp:137-245),
//     and the CameraUniforms setup around them (src/main.cpp:1264-1281)
//   - gaussian_load_gsanim, gsanim_sample, gsanim_layer_weights
//                                               (src/gaussian_loader_gsanim.cpp:386-531)
//   - gaussian_load_sog + pack_gpu_gaussians    (src/gaussian_loader_sog.cpp:126-551)
//   - WebPGetInfo + WebPDecodeRGBA (the vendored libwebp decoder the SOG loader calls)
// Never linked into the product.
#include <SDL3/SDL.h>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <ctime>
#define SJ_IMPL
#include "sj.h"
#include "gaussian.h"
#include "gsanim.h"
#include "camera.h"

#include "gaussian_loader.h"
#include "webp/decode.h"

extern "C" {

// Load a 3DGS binary PLY with the reference loader; returns the count (0 on failure).
// If rows != NULL it must hold count*64 floats and receives pack_gpu_gaussians output.
uint32_t ref_load_ply_rows(const char* path, float* rows, uint32_t capacity) {
    GaussianScene scene;
    memset(&scene, 0, sizeof(scene));
    if (!load_gaussian_scene(path, &scene)) return 0;
    uint32_t n = scene.gaussian_count;
    if (rows && n <= capacity) pack_gpu_gaussians(&scene, 0, n, (GpuGaussian*)rows);
    free_scene(&scene);
    return n;
}

// Reference CPU cull then sort of a PLY scene. visible/depths/sorted hold >= n entries.
// Returns visible count.
uint32_t ref_cull_sort_ply(const char* path, const float* view, const float* proj, float ortho_blend,
                           uint32_t* visible, float* depths, uint32_t* sorted) {
    GaussianScene scene;
    memset(&scene, 0, sizeof(scene));
    if (!load_gaussian_scene(path, &scene)) return 0;
    cull_gaussians(&scene, view, proj, ortho_blend);
    uint32_t vc = scene.visible_count;
    memcpy(visible, scene.visible_indices, vc * sizeof(uint32_t));
    memcpy(depths, scene.visible_depths, vc * sizeof(float));
    SortContext ctx;
    ctx.depths = scene.visible_depths;
    ctx.input_indices = scene.visible_indices;
    ctx.count = vc;
    ctx.sorted_indices = scene.sorted_indices;
    ctx.scratch_indices = scene.scratch_indices;
    ctx.scratch_keys = scene.scratch_keys;
    ctx.scratch_keys2 = scene.scratch_keys2;
    sort_gaussians(&ctx);
    memcpy(sorted, scene.sorted_indices, vc * sizeof(uint32_t));
    free_scene(&scene);
    return vc;
}

}  // extern "C"

// A reference scene holding GpuGaussian rows, unpacked field by field into
// its Gaussian structs (the inverse of pack_gpu_gaussians).
static void scene_from_rows(GaussianScene& scene, const float* rows, uint32_t n) {
    memset(&scene, 0, sizeof(scene));
    scene.gaussian_count = n;
    scene.gaussians = (Gaussian*)calloc(n, sizeof(Gaussian));
    scene.visible_indices = (uint32_t*)malloc((size_t)n * 4);
    scene.visible_depths = (float*)malloc((size_t)n * 4);
    scene.sorted_indices = (uint32_t*)malloc((size_t)n * 4);
    scene.scratch_indices = (uint32_t*)malloc((size_t)n * 4);
    scene.scratch_keys = (uint32_t*)malloc((size_t)n * 4);
    scene.scratch_keys2 = (uint32_t*)malloc((size_t)n * 4);
    for (uint32_t i = 0; i < n; ++i) {
        const float* d = rows + (size_t)i * 64;
        Gaussian& g = scene.gaussians[i];
        memcpy(g.position, d, 12);
        g.opacity = d[3];
        memcpy(g.scale, d + 4, 12);
        memcpy(g.rotation, d + 8, 16);
        memcpy(g.color, d + 12, 12);
        memcpy(g.sh_rest, d + 16, 45 * 4);
    }
}

extern "C" {

// The reference's CPU cull_gaussians (src/gaussian.cpp:77-102) on GpuGaussian
// rows: visible indices and their positive view depths; returns the count.
uint32_t ref_cull_rows(const float* rows, uint32_t n, const float* view, const float* proj, float ortho_blend,
                       uint32_t* visible, float* depths) {
    GaussianScene scene;
    scene_from_rows(scene, rows, n);
    cull_gaussians(&scene, view, proj, ortho_blend);
    const uint32_t vc = scene.visible_count;
    memcpy(visible, scene.visible_indices, (size_t)vc * 4);
    memcpy(depths, scene.visible_depths, (size_t)vc * 4);
    free_scene(&scene);
    return vc;
}

// The reference's CPU cull_gaussians + sort_gaussians (src/gaussian.cpp:77-181)
// on GpuGaussian rows: its back-to-front order of the visible indices;
// returns the visible count.
uint32_t ref_cull_sort_rows(const float* rows, uint32_t n, const float* view, const float* proj, float ortho_blend,
                            uint32_t* sorted) {
    GaussianScene scene;
    scene_from_rows(scene, rows, n);
    cull_gaussians(&scene, view, proj, ortho_blend);
    SortContext ctx;
    ctx.depths = scene.visible_depths;
    ctx.input_indices = scene.visible_indices;
    ctx.count = scene.visible_count;
    ctx.sorted_indices = scene.sorted_indices;
    ctx.scratch_indices = scene.scratch_indices;
    ctx.scratch_keys = scene.scratch_keys;
    ctx.scratch_keys2 = scene.scratch_keys2;
    sort_gaussians(&ctx);
    const uint32_t vc = scene.visible_count;
    memcpy(sorted, scene.sorted_indices, (size_t)vc * 4);
    free_scene(&scene);
    return vc;
}

// Seconds of the reference's single-threaded CPU cull_gaussians +
// sort_gaussians (src/gaussian.cpp:77-181) on a scene given as GpuGaussian
// rows (unpacked into the reference's Gaussian structs first, outside the
// timed region); the visible count in *visible.
double ref_time_cull_sort_rows(const float* rows, uint32_t n, const float* view, const float* proj,
                               float ortho_blend, uint32_t* visible) {
    GaussianScene scene;
    scene_from_rows(scene, rows, n);
    timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    cull_gaussians(&scene, view, proj, ortho_blend);
    SortContext ctx;
    ctx.depths = scene.visible_depths;
    ctx.input_indices = scene.visible_indices;
    ctx.count = scene.visible_count;
    ctx.sorted_indices = scene.sorted_indices;
    ctx.scratch_indices = scene.scratch_indices;
    ctx.scratch_keys = scene.scratch_keys;
    ctx.scratch_keys2 = scene.scratch_keys2;
    sort_gaussians(&ctx);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    *visible = scene.visible_count;
    free_scene(&scene);
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

void ref_camera_matrices(const float pos[3], float yaw, float pitch, float fov_y, float near_plane,
                         float far_plane, int z_up, float ortho_size, float ortho_blend, float aspect,
                         float* view16, float* proj16) {
    Camera cam;
    camera_init(&cam);
    cam.position[0] = pos[0]; cam.position[1] = pos[1]; cam.position[2] = pos[2];
    cam.yaw = yaw; cam.pitch = pitch; cam.fov_y = fov_y;
    cam.near_plane = near_plane; cam.far_plane = far_plane;
    cam.z_up = z_up != 0; cam.ortho_size = ortho_size; cam.ortho_blend = ortho_blend;
    camera_get_view_matrix(&cam, view16);
    camera_get_proj_matrix(&cam, aspect, proj16);
}

// A whole CameraUniforms block (src/camera.h:23-38, 40 floats) of the
// reference fly camera for a width x height GL target: view and projection
// from camera_get_view_matrix / camera_get_proj_matrix, the rest as the
// reference's frame setup fills it (src/main.cpp:1231, 1264-1281, GL branch).
void ref_camera_uniforms(const float pos[3], float yaw, float pitch, float fov_y, float near_plane,
                         float far_plane, int width, int height, float* out40) {
    memset(out40, 0, 40 * sizeof(float));
    const float aspect = (float)width / (float)height;
    ref_camera_matrices(pos, yaw, pitch, fov_y, near_plane, far_plane, 0, 1.0f, 0.0f, aspect, out40, out40 + 16);
    out40[32] = (float)width;
    out40[33] = (float)height;
    out40[34] = 0.0f;                                                  // orthographic blend
    out40[35] = (1.0f / tanf(fov_y * 0.5f)) * (float)height * 0.5f;   // persp_focal
    out40[36] = (float)height / (2.0f * 1.0f);                         // ortho_focal, ortho_size 1
    out40[37] = 1.0f;                                                  // clip_y_sign (GL)
    out40[38] = 0.0f;                                                  // clip_z_01 (GL)
}

// ---- gsanim archives --------------------------------------------------------
// A loaded scene behind an opaque handle (NULL when the reference loader
// rejects the file).
void* ref_gsanim_open(const char* path) {
    GaussianScene* scene = new GaussianScene;
    memset(scene, 0, sizeof(*scene));
    if (!gaussian_load_gsanim(path, scene)) {
        delete scene;
        return nullptr;
    }
    return scene;
}

void ref_gsanim_close(void* h) {
    GaussianScene* scene = (GaussianScene*)h;
    if (!scene) return;
    free_scene(scene);
    delete scene;
}

// ints: version, gaussian_count, state_count, layer_count, key_count, lut_size, linear
// floats: log2_min, log2_max; duration: seconds
void ref_gsanim_info(void* h, uint32_t* ints, float* floats, double* duration) {
    const GSAnim& a = *((GaussianScene*)h)->animation;
    ints[0] = (uint32_t)a.version;
    ints[1] = a.gaussian_count;
    ints[2] = a.state_count;
    ints[3] = (uint32_t)a.layers.size();
    ints[4] = (uint32_t)a.keys.size();
    ints[5] = a.lut_size;
    ints[6] = a.linear ? 1u : 0u;
    floats[0] = a.log2_min;
    floats[1] = a.log2_max;
    *duration = a.duration;
}

void ref_gsanim_rows(void* h, float* rows) {
    const GaussianScene* scene = (const GaussianScene*)h;
    pack_gpu_gaussians(scene, 0, scene->gaussian_count, (GpuGaussian*)rows);
}

void ref_gsanim_deltas(void* h, int8_t* deltas, float* scales) {
    const GSAnim& a = *((GaussianScene*)h)->animation;
    if (!a.deltas.empty()) memcpy(deltas, a.deltas.data(), a.deltas.size());
    memcpy(scales, a.scales, sizeof(a.scales));
}

void ref_gsanim_layer_data(void* h, uint16_t* out) {
    const GSAnim& a = *((GaussianScene*)h)->animation;
    if (!a.layer_data.empty()) memcpy(out, a.layer_data.data(), a.layer_data.size() * 2);
}

void ref_gsanim_display_lut(void* h, uint16_t* out) {
    const GSAnim& a = *((GaussianScene*)h)->animation;
    if (!a.display_lut.empty()) memcpy(out, a.display_lut.data(), a.display_lut.size() * 2);
}

// Byte length of layer i's name; copies min(length, cap) bytes.
uint32_t ref_gsanim_layer_name(void* h, uint32_t i, char* buf, uint32_t cap) {
    const GSAnim& a = *((GaussianScene*)h)->animation;
    const std::string& n = a.layers[i].name;
    memcpy(buf, n.data(), n.size() < cap ? n.size() : cap);
    return (uint32_t)n.size();
}

void ref_gsanim_sample(void* h, double seconds, int32_t* state_a, int32_t* state_b, float* weight) {
    const GSAnimSample s = gsanim_sample(*((GaussianScene*)h)->animation, seconds);
    *state_a = s.state_a;
    *state_b = s.state_b;
    *weight = s.weight;
}

// Number of layers weighted (0 = the reference's empty result).
uint32_t ref_gsanim_layer_weights(void* h, double seconds, float* out) {
    const auto w = gsanim_layer_weights(*((GaussianScene*)h)->animation, seconds);
    for (size_t i = 0; i < w.size(); ++i) memcpy(out + 3 * i, w[i].data(), 12);
    return (uint32_t)w.size();
}

// ---- SOG archives and their WebP images ----------------------------------------
// Gaussian count of a .sog archive (0 when the reference loader rejects it);
// with rows != NULL and count <= capacity, also its pack_gpu_gaussians rows.
uint32_t ref_sog_rows(const char* path, float* rows, uint32_t capacity) {
    GaussianScene scene;
    memset(&scene, 0, sizeof(scene));
    if (!gaussian_load_sog(path, &scene)) return 0;
    const uint32_t n = scene.gaussian_count;
    if (rows && n <= capacity) pack_gpu_gaussians(&scene, 0, n, (GpuGaussian*)rows);
    free_scene(&scene);
    return n;
}

// The SOG loader's image decode (load_sog_image, src/gaussian_loader_sog.cpp:98-124):
// 1 and the image size when WebPGetInfo and WebPDecodeRGBA both succeed; the
// RGBA8 pixels go to rgba when it holds w * h * 4 bytes (capacity).
int ref_webp_decode(const uint8_t* data, size_t size, int* w, int* h, uint8_t* rgba, size_t capacity) {
    *w = *h = 0;
    int iw = 0, ih = 0;
    if (!WebPGetInfo(data, size, &iw, &ih) || iw <= 0 || ih <= 0) return 0;
    uint8_t* px = WebPDecodeRGBA(data, size, &iw, &ih);
    if (!px) return 0;
    *w = iw;
    *h = ih;
    if (rgba && (size_t)iw * (size_t)ih * 4 <= capacity) memcpy(rgba, px, (size_t)iw * (size_t)ih * 4);
    WebPFree(px);
    return 1;
}

}  // extern "C"
