// Elementwise and reduction kernels of the stochastic-splat denoiser: the
// backward passes of pooling and upsampling (the input features are written by
// the TAA pass, the 2x average pooling by conv1's epilogue), the output head
// of training, the L1 + SSIM training loss with
// its gradient and Adam.  The convolutions are in gs_conv.cu; in the denoised
// render mode the last convolution's epilogue writes the frame and the
// per-tile error estimate that picks the tiles the sorted-alpha rasterizer
// renders again (conv::ConvArgs::head_x).
//
// Network (NHWC bf16 activations, FP32 accumulation):
//   x   16 ch  = noisy RGB, alpha, expected depth, reprojected history RGB, 8 zero channels
//   e1  = relu(conv1(x))            32 ch, full resolution
//   p1  = avgpool2(e1)              32 ch, half
//   e2  = relu(conv2(p1))           32 ch, half
//   e3  = relu(conv3(e2))           32 ch, half
//   d4  = relu(conv4(up2(e3) + e1)) 32 ch, full (U-Net skip)
//   o   = conv5(d4)                 16 ch (f32): 0..3 RGBA residual, 4 error estimate
//   RGBA = (history RGB, alpha) + o[0..3];  error = o[4] (1000 x squared error)
#include <cuda_bf16.h>

#include "gs_denoise.h"

namespace gs {
namespace dn {

__device__ __forceinline__ float bf(const __nv_bfloat16& v) { return __bfloat162float(v); }

// Backward of the decoder input u = up2(e3) + e1 for its e3 term, with the
// ReLU of e3: dz3[q] = (e3[q] > 0) * sum of du over the 2x2 block of q.
__global__ void upsample_grad_kernel(const __nv_bfloat16* __restrict__ du, const __nv_bfloat16* __restrict__ e3,
                                     int n, int h, int w, __nv_bfloat16* __restrict__ dz3) {
    const int hh = h / 2, hw = w / 2;
    const size_t total = (size_t)n * hh * hw * kHidC;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % kHidC);
        const size_t op = i / kHidC;
        const int ox = (int)(op % hw), oy = (int)((op / hw) % hh), b = (int)(op / ((size_t)hw * hh));
        float s = 0.0f;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx)
                s += bf(du[(((size_t)b * h + 2 * oy + dy) * w + 2 * ox + dx) * kHidC + c]);
        dz3[i] = __float2bfloat16_rn(bf(e3[i]) > 0.0f ? s : 0.0f);
    }
}

// Gradient of e1 (skip term du plus the pooling term dp1 / 4) through the
// ReLU of e1: dz1 = (e1 > 0) * (du + dp1[p / 2] / 4).
__global__ void skip_pool_grad_kernel(const __nv_bfloat16* __restrict__ du, const __nv_bfloat16* __restrict__ dp1,
                                      const __nv_bfloat16* __restrict__ e1, int n, int h, int w,
                                      __nv_bfloat16* __restrict__ dz1) {
    const int hh = h / 2, hw = w / 2;
    const size_t total = (size_t)n * h * w * kHidC;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % kHidC);
        const size_t p = i / kHidC;
        const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((size_t)w * h));
        const float g = bf(du[i]) + 0.25f * bf(dp1[(((size_t)b * hh + y / 2) * hw + x / 2) * kHidC + c]);
        dz1[i] = __float2bfloat16_rn(bf(e1[i]) > 0.0f ? g : 0.0f);
    }
}

// ---------------------------------------------------------------------------
// Output head and the training loss.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 head_rgba(const float* o, const __nv_bfloat16* x) {
    return make_float4(bf(x[5]) + o[0], bf(x[6]) + o[1], bf(x[7]) + o[2], bf(x[3]) + o[3]);
}

// pred = head(o, x) (RGBA, f32); moments of (pred, target) per RGB channel
// for SSIM: x, y, x^2, y^2, xy (15 maps, f32, channel-major per pixel).
__global__ void head_moments_kernel(const float* __restrict__ o, const __nv_bfloat16* __restrict__ x,
                                    const float4* __restrict__ target, int npix, float4* __restrict__ pred,
                                    float* __restrict__ mom) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const float4 p = head_rgba(o + (size_t)i * kOutC, x + (size_t)i * kInC);
        pred[i] = p;
        if (!mom) continue;
        const float4 t = target[i];
        const float pc[3] = {p.x, p.y, p.z}, tc[3] = {t.x, t.y, t.z};
        float* m = mom + (size_t)i * 15;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            m[c * 5 + 0] = pc[c];
            m[c * 5 + 1] = tc[c];
            m[c * 5 + 2] = pc[c] * pc[c];
            m[c * 5 + 3] = tc[c] * tc[c];
            m[c * 5 + 4] = pc[c] * tc[c];
        }
    }
}

// Separable Gaussian blur (11 taps, sigma 1.5, zero outside the image) of
// `nmaps` interleaved f32 maps along x (dir 0) or y (dir 1).
__constant__ float c_gauss[11];

__global__ void blur_kernel(const float* __restrict__ in, int n, int h, int w, int nmaps, int dir,
                            float* __restrict__ out) {
    const size_t total = (size_t)n * h * w * nmaps;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(i % nmaps);
        const size_t p = i / nmaps;
        const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((size_t)w * h));
        float s = 0.0f;
#pragma unroll
        for (int k = -5; k <= 5; ++k) {
            const int xx = dir == 0 ? x + k : x, yy = dir == 0 ? y : y + k;
            if (xx < 0 || xx >= w || yy < 0 || yy >= h) continue;
            s += c_gauss[k + 5] * in[(((size_t)b * h + yy) * w + xx) * nmaps + m];
        }
        out[i] = s;
    }
}

constexpr float kC1 = 0.0001f, kC2 = 0.0009f;   // (0.01)^2, (0.03)^2 for a data range of 1

// From the blurred moments: SSIM per interior pixel and channel (pixels
// closer than 5 to the border are left out) and its partial derivatives
// with respect to mu_x, E[x^2] and E[xy] (9 maps); the SSIM sum and count
// go to acc[0], acc[1].
__global__ void ssim_partials_kernel(const float* __restrict__ bm, int n, int h, int w, float* __restrict__ part,
                                     float* __restrict__ acc) {
    const size_t total = (size_t)n * h * w;
    float local = 0.0f, cnt = 0.0f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % w), y = (int)((p / w) % h);
        const bool inside = x >= 5 && x < w - 5 && y >= 5 && y < h - 5;
        float* q = part + p * 9;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float* m = bm + p * 15 + c * 5;
            const float mx = m[0], my = m[1];
            const float sxx = m[2] - mx * mx, syy = m[3] - my * my, sxy = m[4] - mx * my;
            const float A1 = 2.0f * mx * my + kC1, A2 = 2.0f * sxy + kC2;
            const float B1 = mx * mx + my * my + kC1, B2 = sxx + syy + kC2;
            const float S = (A1 * A2) / (B1 * B2);
            float dmx = 0.0f, dxx = 0.0f, dxy = 0.0f;
            if (inside) {
                local += S;
                cnt += 1.0f;
                const float dS_dA1 = A2 / (B1 * B2), dS_dA2 = A1 / (B1 * B2);
                const float dS_dB1 = -S / B1, dS_dB2 = -S / B2;
                // A1(mx), A2(sxy(mx)), B1(mx), B2(sxx(mx)); sxx = E[x^2] - mx^2, sxy = E[xy] - mx my
                dxx = dS_dB2;                                   // dB2 / dE[x^2] = 1
                dxy = 2.0f * dS_dA2;                            // dA2 / dE[xy] = 2
                dmx = dS_dA1 * 2.0f * my + dS_dA2 * (-2.0f * my) + dS_dB1 * 2.0f * mx + dS_dB2 * (-2.0f * mx);
            }
            q[c * 3 + 0] = dmx;
            q[c * 3 + 1] = dxx;
            q[c * 3 + 2] = dxy;
        }
    }
    for (int off = 16; off; off >>= 1) {
        local += __shfl_xor_sync(0xffffffffu, local, off);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc + 0, local);
        atomicAdd(acc + 1, cnt);
    }
}

// Gradient of the loss
//   L = mean |pred - t| (RGBA) + ssim_w (1 - mean SSIM) + err_w mean (o4 - 1000 e)^2,
//   e = mean over RGBA of (pred - t)^2 (not differentiated),
// with respect to o (16 channels, bf16 for the backward convolutions); the
// blurred SSIM partials `bp` give dSSIM/dpred = B_mu + 2 pred B_xx + t B_xy.
// acc[2] += sum |pred - t|, acc[3] += sum (o4 - 1000 e)^2.  The SSIM count
// acc[1] is the one of ssim_partials_kernel (read by the host as ssim_count).
__global__ void loss_grad_kernel(const float* __restrict__ o, const float4* __restrict__ pred,
                                 const float4* __restrict__ target, const float* __restrict__ bp, int npix,
                                 float inv_l1, float ssim_scale, float err_scale, __nv_bfloat16* __restrict__ dout,
                                 float* __restrict__ acc) {
    float l1 = 0.0f, le = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const float4 p = pred[i], t = target[i];
        const float pv[4] = {p.x, p.y, p.z, p.w}, tv[4] = {t.x, t.y, t.z, t.w};
        float g[kOutC];
#pragma unroll
        for (int c = 0; c < kOutC; ++c) g[c] = 0.0f;
        float e = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float d = pv[c] - tv[c];
            l1 += fabsf(d);
            e += d * d;
            g[c] = inv_l1 * (d > 0.0f ? 1.0f : d < 0.0f ? -1.0f : 0.0f);
        }
        e *= 0.25f;
        if (bp) {
            const float* b = bp + (size_t)i * 9;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                g[c] += -ssim_scale * (b[c * 3 + 0] + 2.0f * pv[c] * b[c * 3 + 1] + tv[c] * b[c * 3 + 2]);
        }
        const float r = o[(size_t)i * kOutC + 4] - 1000.0f * e;
        le += r * r;
        g[4] = err_scale * 2.0f * r;
        uint4* op = reinterpret_cast<uint4*>(dout + (size_t)i * kOutC);
#pragma unroll
        for (int q = 0; q < kOutC / 8; ++q) {
            uint4 pk;
            __nv_bfloat162* pb = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
            for (int k = 0; k < 4; ++k) pb[k] = __floats2bfloat162_rn(g[q * 8 + 2 * k], g[q * 8 + 2 * k + 1]);
            op[q] = pk;
        }
    }
    for (int off = 16; off; off >>= 1) {
        l1 += __shfl_xor_sync(0xffffffffu, l1, off);
        le += __shfl_xor_sync(0xffffffffu, le, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc + 2, l1);
        atomicAdd(acc + 3, le);
    }
}

// Adam (Kingma & Ba, bias-corrected), FP32 masters.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int count, float lr, float b1, float b2, float eps, float bc1,
                            float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / bc1, vh = vi / bc2;
        w[i] -= lr * mh / (sqrtf(vh) + eps);
    }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
static int grid_for(size_t n, int threads = 256) {
    size_t b = (n + threads - 1) / threads;
    return (int)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

void set_gauss_window(cudaStream_t s) {
    float g[11], sum = 0.0f;
    for (int k = -5; k <= 5; ++k) {
        g[k + 5] = expf(-(float)(k * k) / (2.0f * 1.5f * 1.5f));
        sum += g[k + 5];
    }
    for (float& v : g) v /= sum;
    cudaMemcpyToSymbolAsync(c_gauss, g, sizeof(g), 0, cudaMemcpyHostToDevice, s);
}

int launch_upsample_grad(const __nv_bfloat16* du, const __nv_bfloat16* e3, int n, int h, int w, __nv_bfloat16* dz3,
                         cudaStream_t s) {
    upsample_grad_kernel<<<grid_for((size_t)n * (h / 2) * (w / 2) * kHidC), 256, 0, s>>>(du, e3, n, h, w, dz3);
    return 1;
}
int launch_skip_pool_grad(const __nv_bfloat16* du, const __nv_bfloat16* dp1, const __nv_bfloat16* e1, int n, int h,
                          int w, __nv_bfloat16* dz1, cudaStream_t s) {
    skip_pool_grad_kernel<<<grid_for((size_t)n * h * w * kHidC), 256, 0, s>>>(du, dp1, e1, n, h, w, dz1);
    return 1;
}
int launch_head_moments(const float* o, const __nv_bfloat16* x, const float4* target, int npix, float4* pred,
                        float* mom, cudaStream_t s) {
    head_moments_kernel<<<grid_for(npix), 256, 0, s>>>(o, x, target, npix, pred, mom);
    return 1;
}
int launch_blur(const float* in, int n, int h, int w, int nmaps, int dir, float* out, cudaStream_t s) {
    blur_kernel<<<grid_for((size_t)n * h * w * nmaps), 256, 0, s>>>(in, n, h, w, nmaps, dir, out);
    return 1;
}
int launch_ssim_partials(const float* bm, int n, int h, int w, float* part, float* acc, cudaStream_t s) {
    ssim_partials_kernel<<<grid_for((size_t)n * h * w), 256, 0, s>>>(bm, n, h, w, part, acc);
    return 1;
}
int launch_loss_grad(const float* o, const float4* pred, const float4* target, const float* bp, int npix,
                     float inv_l1, float ssim_scale, float err_scale, __nv_bfloat16* dout, float* acc, cudaStream_t s) {
    loss_grad_kernel<<<grid_for(npix), 256, 0, s>>>(o, pred, target, bp, npix, inv_l1, ssim_scale, err_scale, dout,
                                                    acc);
    return 1;
}
int launch_adam(float* w, const float* g, float* m, float* v, int count, float lr, float b1, float b2, float eps,
                float bc1, float bc2, cudaStream_t s) {
    adam_kernel<<<grid_for(count), 256, 0, s>>>(w, g, m, v, count, lr, b1, b2, eps, bc1, bc2);
    return 1;
}
}  // namespace dn
}  // namespace gs
