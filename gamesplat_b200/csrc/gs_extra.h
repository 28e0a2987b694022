// Internal interfaces of the stochastic-accumulation, TAA and Gaussian Point
// Splatting stages (gs_accum.cu, gs_gps.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "gs_internal.h"

namespace gs {

// Stochastic / GPS image targets (src/renderer.h:215-229): sample colour
// (RGBA, as floats), sample window depth, accumulation ping-pong (RGBA32F),
// TAA world-position history, frame-average ping-pong.  Top row first.
struct StochasticTargets {
    int width = 0, height = 0;
    float4* sample = nullptr;
    float* depth = nullptr;
    float4* accum[2] = {nullptr, nullptr};
    float4* xyz[2] = {nullptr, nullptr};
    float4* frame_avg[2] = {nullptr, nullptr};
    const float4* display = nullptr;  // what the last frame displayed
};

int ensure_stochastic_targets(StochasticTargets& t, int width, int height, cudaStream_t s);
void release_stochastic_targets(StochasticTargets& t);

// TaaAccumUBO (shaders/accum.glsl:65-76).
struct TaaUniforms {
    float inv_view[16];
    float prev_view[16];
    float viewport_orthographic[4];
    float focal_clip[4];
    float prev_focal_clip[4];
    float proj_z[4];
    float history_valid;
    float view_changed;
};

int launch_accum(const float4* sample, const float4* history, float sample_count, float4* out, size_t npix,
                 cudaStream_t s);
// features (optional, 16 bf16 per pixel, top row first): the denoiser's input,
// (current RGBA, depth, the new history RGB, 8 zeros), written beside the history
int launch_taa(const float4* cur_color, const float* cur_depth, const float4* hist_color, const float4* hist_xyz,
               int width, int height, const TaaUniforms& u, float4* out_color, float4* out_xyz, cudaStream_t s,
               void* features = nullptr);
int launch_to_half(const float4* src, uint16_t* dst, size_t npix, cudaStream_t s);

bool mat4_inverse(const float m[16], float out[16]);

// Gaussian Point Splatting buffers (src/renderer.h:85-112): the packed
// (depth << 32 | colour) sub-pixel buffer, prepared records and work items.
struct GpsTargets {
    int width = 0, height = 0;
    uint32_t ss = 0;
    unsigned long long* packed = nullptr;
    float4* prepared = nullptr;   // 3 float4 per visible Gaussian
    uint32_t prepared_cap = 0;
    uint2* work = nullptr;
    uint32_t work_cap = 0;
};

struct GpsParams {
    const float4* projected;
    const uint32_t* vis_ids;      // compacted visible ids (index order)
    FrameCounters* fc;
    int width, height;
    uint32_t supersample;
    uint32_t max_work_items;
    float clip_z_01;
    int linear_color;
    float frame_seed;
    float bg;
    float4* out_color;            // resolved RGBA (top row first)
    float* out_depth;             // resolved depth (top row first)
};

int ensure_gps_targets(GpsTargets& g, int width, int height, uint32_t ss, uint32_t n, uint32_t max_work_items,
                       cudaStream_t s);
int resize_gps_work(GpsTargets& g, uint32_t max_work_items, cudaStream_t s);
void release_gps_targets(GpsTargets& g);
void release_gps_scene(GpsTargets& g);
int launch_gps(GpsTargets& g, const GpsParams& p, uint32_t n_cap, uint32_t num_sms, cudaStream_t s);

}  // namespace gs
