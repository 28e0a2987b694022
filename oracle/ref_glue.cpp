// Test-infrastructure glue around the reference's own CPU code (compiled from
// the reference sources in place by oracle/Makefile into oracle/_ref/).
// Exposes extern "C" entry points for ctypes so tests can pin the oracle
// against the reference:
//   - gaussian_load_ply + pack_gpu_gaussians   (src/gaussian_loader_ply.cpp:14-228,
//                                                src/gaussian.cpp:53-73)
//   - cull_gaussians + sort_gaussians           (src/gaussian.cpp:77-181)
//   - camera_get_view_matrix / camera_get_proj_matrix (src/camera.cpp:137-245)
// Never linked into the product.
#include <SDL3/SDL.h>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include "gaussian.h"
#include "camera.h"

// The reference's load_gaussian_scene dispatches to loaders we do not build.
bool gaussian_load_sog(const char*, GaussianScene*) { return false; }
bool gaussian_load_gsanim(const char*, GaussianScene*) { return false; }
struct GSAnim;

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

}  // extern "C"
