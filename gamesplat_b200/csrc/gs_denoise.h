// Denoiser kernels other than the convolutions (gs_denoise.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace gs {
namespace dn {

constexpr int kInC = 16;    // input features (8 used)
constexpr int kHidC = 32;   // hidden channels
constexpr int kOutC = 16;   // output channels (5 used)

void set_gauss_window(cudaStream_t s);
int launch_upsample_grad(const __nv_bfloat16* du, const __nv_bfloat16* e3, int n, int h, int w, __nv_bfloat16* dz3,
                         cudaStream_t s);
int launch_skip_pool_grad(const __nv_bfloat16* du, const __nv_bfloat16* dp1, const __nv_bfloat16* e1, int n, int h,
                          int w, __nv_bfloat16* dz1, cudaStream_t s);
int launch_head_moments(const float* o, const __nv_bfloat16* x, const float4* target, int npix, float4* pred,
                        float* mom, cudaStream_t s);
int launch_blur(const float* in, int n, int h, int w, int nmaps, int dir, float* out, cudaStream_t s);
int launch_ssim_partials(const float* bm, int n, int h, int w, float* part, float* acc, cudaStream_t s);
int launch_loss_grad(const float* o, const float4* pred, const float4* target, const float* bp, int npix,
                     float inv_l1, float ssim_scale, float err_scale, __nv_bfloat16* dout, float* acc,
                     cudaStream_t s);
int launch_adam(float* w, const float* g, float* m, float* v, int count, float lr, float b1, float b2, float eps,
                float bc1, float bc2, cudaStream_t s);

}  // namespace dn
}  // namespace gs
