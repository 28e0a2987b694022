/* CPU oracle for the gamesplat per-frame splatting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * GLSL compute/fragment programs and of the GL fixed-function raster and blend
 * state they rely on.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it, and only as the checker.  The product library
 * (gamesplat_b200/libgs_cuda.so) never links or calls it.
 *
 * Every float operation is written in the operand order of the GLSL source it
 * restates; the file is compiled with -ffp-contract=off so that no FMA is
 * formed, which makes the results reproducible bit-for-bit by a CUDA kernel
 * that uses the same order with __fmul_rn/__fadd_rn.
 *
 * Parity status: cull visibility and depth keys are pinned against the
 * reference's own CPU cull_gaussians / sort_gaussians (src/gaussian.cpp:77-181)
 * compiled from the reference sources into oracle/_ref; the camera builder
 * against src/camera.cpp:137-245; GpuGaussian rows against the reference PLY
 * loader.  The composited image itself is "parity unpinned": the reference
 * produces it with a GL driver's rasterizer and blender, which is not part of
 * the reference sources and cannot run on these machines.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Byte-for-byte CameraUniforms (src/camera.h:23-38), 40 floats = 160 B. */
typedef struct oc_camera {
    float view[16];
    float proj[16];
    float viewport[2];
    float orthographic;
    float persp_focal;
    float ortho_focal;
    float clip_y_sign;
    float clip_z_01;
    float pad[1];
} oc_camera;

#define OC_SENTINEL 0xFFFFFFFFu

/* Deterministic transcendental functions built only from IEEE +,-,*,/ (see
 * gs_oracle.c for the methods).  The CUDA path implements the same methods. */
float oc_logf(float x);
float oc_expf(float x);
void  oc_sincosf(float x, float* s, float* c);
float oc_dilog(float x);      /* shaders/cull.glsl:116-123 */
float oc_inv_dilog(float x);  /* shaders/gps.glsl:225-230 */

/* shaders/cull.glsl:166-424 + cull_reset (:456-473) over all n rows.
 * rows: n * 64 floats (GpuGaussian, src/gaussian.h:63-73).
 * ids/keys: n entries, reset to 0xFFFFFFFF then written for visible rows.
 * projected: n * 16 floats (CullProjectedSplatData, shaders/cull.glsl:12-17).
 * diag: 8 counters (shaders/cull.glsl:296-318), filled if collect_stats. */
void oc_cull(const float* rows, uint32_t n, const oc_camera* cam, int sh_degree,
             float sh_lod_distance, int collect_stats, uint32_t* ids, uint32_t* keys,
             float* projected, uint32_t* visible_count, uint32_t* diag);

/* oc_cull with gsanim int8 appearance deltas applied to the DC and SH
 * coefficients (shaders/cull.glsl:125-164): deltas[((s-1)*n + row)*48 + j],
 * scales[48], states a/b and blend weight as in the renderer's
 * animation_state_a/b and animation_weight. */
void oc_cull_anim(const float* rows, uint32_t n, const oc_camera* cam, int sh_degree,
                  float sh_lod_distance, int collect_stats, const int8_t* deltas, const float* scales,
                  int state_a, int state_b, float weight, uint32_t* ids, uint32_t* keys,
                  float* projected, uint32_t* visible_count, uint32_t* diag);

/* oc_cull with gsanim 0.3 appearance layers (shaders/cull.glsl:141-148,
 * 354-416): halves[(l*n + row)*48 + j] replace the DC and SH coefficients of
 * layer l; the colour is the sum over layers of max(SH colour, 0) * weights[l*3 + c]
 * (no +0.5 bias).  layer_count 0 is oc_cull. */
void oc_cull_layers(const float* rows, uint32_t n, const oc_camera* cam, int sh_degree,
                    float sh_lod_distance, int collect_stats, const uint16_t* halves, int layer_count,
                    const float* weights, uint32_t* ids, uint32_t* keys, float* projected,
                    uint32_t* visible_count, uint32_t* diag);

/* Stable ascending LSD radix sort (8-bit digits, 4 passes) of (key, id) pairs,
 * the order shaders/sort.glsl:26-163 produces. */
void oc_sort_pairs(const uint32_t* keys_in, const uint32_t* ids_in, uint32_t n,
                   uint32_t* keys_out, uint32_t* ids_out);

/* Covered pixel rectangle [rect[0],rect[1]) x [rect[2],rect[3]) in GL window
 * coordinates (row 0 = bottom) of one splat quad (shaders/splat.glsl:39-75),
 * after the NDC round trip, 8-bit sub-pixel snapping and a top-left fill rule
 * (top = larger window y).  Returns 0 when the quad is clipped in z. */
int oc_quad_rect(const float* projected16, float jitter_x, float jitter_y, float vp_w, float vp_h,
                 float clip_y_sign, int width, int height, int32_t rect[4]);

/* Sorted back-to-front premultiplied alpha compositing of `count` instances
 * (shaders/splat.glsl:39-104, blend ONE / ONE_MINUS_SRC_ALPHA,
 * src/renderer.cpp:276-299) into a (bg,bg,bg,0)-cleared target.
 * fp16_per_blend = 0: FP32 blending (round to fp16 once, by the caller);
 * fp16_per_blend = 1: every blend result rounded to fp16 (RGBA16F blender).
 * out_rgba: width*height*4 floats, top row first.  Returns shaded fragments. */
uint64_t oc_composite_alpha(const uint32_t* sorted_ids, uint32_t count, const float* projected,
                            int width, int height, float vp_w, float vp_h, float clip_y_sign,
                            float bg, float jitter_x, float jitter_y, int fp16_per_blend,
                            float* out_rgba);

/* One stochastic sample (shaders/splat.glsl:121-145 with depth LESS + write,
 * src/renderer.cpp:302-320): instances in id-buffer order.  out_rgba top-first,
 * out_depth = window depth of the kept fragment (1.0 where none), top-first.
 * rgba8 != 0 quantises the stored colour like an RGBA8 UNORM target. */
uint64_t oc_stochastic_sample(const uint32_t* ids, uint32_t count, const float* projected,
                              int width, int height, float vp_w, float vp_h, float clip_y_sign,
                              float bg, float jitter_x, float jitter_y, float frame_seed, int rgba8,
                              float* out_rgba, float* out_depth);

/* Gaussian Point Splatting frame: clear/expand/splat/resolve
 * (shaders/gps.glsl:32-385).  Depth/colour is resolved with a 64-bit
 * (depth << 32 | colour) minimum.  out_rgba (RGBA32F) and out_depth are
 * width*height, top row first.  work_stats[0] = requested work items,
 * work_stats[1] = overflow flag. */
void oc_gps_frame(const uint32_t* ids, uint32_t count, const float* projected, int width,
                  int height, int supersample, uint32_t max_work_items, float clip_z_01,
                  int linear_color, float frame_seed, float bg, float* out_rgba, float* out_depth,
                  uint32_t* work_stats);

/* Running mean h + (s - h) / max(n, 1) (shaders/accum.glsl:39-44). */
void oc_accum(const float* sample, const float* history, float sample_count, uint64_t count4,
              float* out);

/* Reprojection TAA (shaders/accum.glsl:148-178).  All images top row first,
 * depth = window depth.  params: see gs_oracle.c. */
void oc_taa(const float* cur_color, const float* cur_depth, const float* hist_color,
            const float* hist_xyz, int width, int height, const float* inv_view,
            const float* prev_view, const float* viewport_ortho, const float* focal_clip,
            const float* prev_focal_clip, const float* proj_z, float history_valid,
            float view_changed, float* out_color, float* out_xyz);

/* Display transform of a linear RGBA16F frame (shaders/accum.glsl:201-240,
 * src/renderer.cpp:2120-2137): in_half = width*height*4 IEEE half bit
 * patterns, lut = lut_size^3 x RGB uint16 (x fastest), or NULL for the plain
 * blit (shaders/accum.glsl:181-192).  out_rgba: width*height*4 floats.
 * exp2/log2 are oc_expf/oc_logf scaled by ln 2. */
void oc_display(const uint16_t* in_half, int width, int height, const uint16_t* lut, int lut_size,
                float log2_min, float log2_max, float exposure_ev, float* out_rgba);

/* IEEE half bit pattern -> float (exact). */
float oc_half_to_float(uint16_t h);

/* Halton radical inverse (src/renderer.cpp:246-255). */
int oc_mat4_inverse(const float* m, float* out);  /* src/renderer.cpp:86-206 */
float oc_halton(uint32_t index, uint32_t base);

#ifdef __cplusplus
}
#endif
