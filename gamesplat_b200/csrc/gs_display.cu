// Display transform of the linear RGBA16F frame: the gsanim 0.3 "layers"
// display pass (renderer_display_appearance, src/renderer.cpp:2120-2137;
// shaders/accum.glsl:201-240) or, without a LUT, the plain blit
// (shaders/accum.glsl:181-192).  One thread per pixel; the sampler is
// non-filtering at the frame's own resolution, so every output pixel reads
// its own input pixel.
//
// Per pixel: radiance = rgb * exp2(exposure_ev);
//   s = clamp((log2(max(radiance, exp2(log2_min))) - log2_min) / (log2_max - log2_min), 0, 1);
//   p = s * (lut_size - 1); trilinear lookup of the uint16 RGB lattice
//   (entry / 65535) between floor(p) and min(floor(p) + 1, lut_size - 1)
//   with weights fract(p), mixed x, then y, then z; alpha = 1.
// exp2 and log2 are the deterministic exp / log of gs_common.cuh scaled by
// ln 2 (the CPU oracle uses the same operations), so results are bit-exact
// against it.
#include <cuda_fp16.h>

#include "gs_common.cuh"
#include "gs_display.h"

namespace gs {

__device__ __forceinline__ float det_exp2f(float x) { return det_expf(mul(x, kLn2f)); }
__device__ __forceinline__ float det_log2f(float x) { return mul(det_logf(x), kInvLn2); }

__device__ __forceinline__ float lut_entry(const uint16_t* __restrict__ lut, int n, int x, int y, int z, int c) {
    const int i = ((z * n + y) * n + x) * 3 + c;
    return dv((float)__ldg(lut + i), 65535.0f);
}

__global__ void display_lut_kernel(DisplayParams p) {
    const size_t npix = (size_t)p.width * p.height;
    const float gain = det_exp2f(p.exposure_ev);
    const float lo_clamp = det_exp2f(p.log2_min);
    const float range = sub(p.log2_max, p.log2_min);
    const float top = (float)(p.lut_size - 1);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
        const uint2 h = reinterpret_cast<const uint2*>(p.in_rgba16f)[i];
        const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&h.x));
        const float2 ba = __half22float2(*reinterpret_cast<const __half2*>(&h.y));
        if (!p.lut) {
            p.out_rgba32f[i] = make_float4(rg.x, rg.y, ba.x, ba.y);
            continue;
        }
        const float rad[3] = {mul(rg.x, gain), mul(rg.y, gain), mul(ba.x, gain)};
        int lo[3], hi[3];
        float f[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float s = g_clamp(dv(sub(det_log2f(g_max(rad[c], lo_clamp)), p.log2_min), range), 0.0f, 1.0f);
            if (s != s) s = 0.0f;   // NaN input: first lattice entry (as the oracle)
            const float pc = mul(s, top);
            const float fl = floorf(pc);
            lo[c] = (int)fl;
            hi[c] = min(lo[c] + 1, p.lut_size - 1);
            f[c] = sub(pc, fl);
        }
        float o[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int n = p.lut_size;
            const float a = g_mix(g_mix(lut_entry(p.lut, n, lo[0], lo[1], lo[2], c), lut_entry(p.lut, n, hi[0], lo[1], lo[2], c), f[0]),
                                  g_mix(lut_entry(p.lut, n, lo[0], hi[1], lo[2], c), lut_entry(p.lut, n, hi[0], hi[1], lo[2], c), f[0]),
                                  f[1]);
            const float b = g_mix(g_mix(lut_entry(p.lut, n, lo[0], lo[1], hi[2], c), lut_entry(p.lut, n, hi[0], lo[1], hi[2], c), f[0]),
                                  g_mix(lut_entry(p.lut, n, lo[0], hi[1], hi[2], c), lut_entry(p.lut, n, hi[0], hi[1], hi[2], c), f[0]),
                                  f[1]);
            o[c] = g_mix(a, b, f[2]);
        }
        p.out_rgba32f[i] = make_float4(o[0], o[1], o[2], 1.0f);
    }
}

int launch_display(const DisplayParams& p, uint32_t num_sms, cudaStream_t s) {
    const size_t npix = (size_t)p.width * p.height;
    if (npix == 0) return 0;
    size_t grid = (npix + 255) / 256;
    if (grid > (size_t)num_sms * 16) grid = (size_t)num_sms * 16;
    display_lut_kernel<<<(unsigned)grid, 256, 0, s>>>(p);
    return 1;
}

}  // namespace gs
