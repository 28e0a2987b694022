// Internal interface of the denoiser object (gs_denoiser.cpp) for the
// renderer's denoised mode (gs_host.cpp).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/gs_api.h"

namespace gs {
namespace dn {

constexpr int kLayers = 5;
constexpr float kTrainSsimWeight = 0.2f;   // L = L1 + 0.2 (1 - SSIM) + 0.01 error-head term
constexpr float kTrainErrWeight = 0.01f;

uint64_t parameter_count();
// Forward pass of the last-layer output (16 channels, f32) into the
// denoiser's own buffer, returned by output(), issued on stream s (the
// renderer's, whose kernels produced x).
int forward(gs_denoiser* d, const __nv_bfloat16* x, int n, int h, int w, cudaStream_t s);
const float* output(const gs_denoiser* d);

// The denoised mode's frame: the forward pass of one h x w frame whose last
// layer writes the RGBA16F image out16 (the input's history RGB and alpha plus
// the network's correction) and, per 16x16 tile (tiles_x across, GL rows from
// the bottom), tile_err = the estimated mean squared error; tiles at or above
// err_budget are appended to fallback_tiles (count in *fallback_count).  The
// last layer's 16 output channels are not stored.
int forward_frame(gs_denoiser* d, const __nv_bfloat16* x, int h, int w, uint16_t* out16, int tiles_x,
                  float err_budget, uint32_t* fallback_count, uint32_t* fallback_tiles, float* tile_err,
                  cudaStream_t s);

}  // namespace dn
}  // namespace gs
