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

}  // namespace dn
}  // namespace gs
