// Accumulation, reprojection TAA and output conversion for the stochastic and
// GPS modes: shaders/accum.glsl:39-178 as per-pixel CUDA kernels (the
// reference runs them as fullscreen-triangle fragment passes).  Images are
// stored top row first; the kernels address texel (x, y) in GL orientation
// at buffer row height-1-y.  Arithmetic uses unfused intrinsics in GLSL
// operand order to match the CPU oracle bit for bit.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>

#include "gs_common.cuh"
#include "gs_extra.h"

namespace gs {

__global__ void accum_kernel(const float4* __restrict__ sample, const float4* __restrict__ history, float n,
                             float4* __restrict__ out, size_t npix) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    const float nn = g_max(n, 1.0f);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
        float4 s = sample[i], h = history[i];
        float4 o;
        o.x = add(h.x, dv(sub(s.x, h.x), nn));
        o.y = add(h.y, dv(sub(s.y, h.y), nn));
        o.z = add(h.z, dv(sub(s.z, h.z), nn));
        o.w = add(h.w, dv(sub(s.w, h.w), nn));
        out[i] = o;
    }
}

__global__ void to_half_kernel(const float4* __restrict__ src, uint2* __restrict__ dst, size_t npix) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
        float4 c = src[i];
        __half2 a = __floats2half2_rn(c.x, c.y), b = __floats2half2_rn(c.z, c.w);
        uint2 v;
        v.x = *reinterpret_cast<uint32_t*>(&a);
        v.y = *reinterpret_cast<uint32_t*>(&b);
        dst[i] = v;
    }
}

__device__ __forceinline__ float4 texel4(const float4* img, int w, int h, int x, int y) {
    return img[(size_t)(h - 1 - y) * w + x];
}

__device__ __forceinline__ float4 mix4(float4 a, float4 b, float t) {
    return make_float4(g_mix(a.x, b.x, t), g_mix(a.y, b.y, t), g_mix(a.z, b.z, t), g_mix(a.w, b.w, t));
}

// sample_history_*_bilinear (shaders/accum.glsl:116-146)
__device__ float4 bilinear(const float4* img, int w, int h, float u, float v) {
    float px = sub(mul(u, (float)w), 0.5f), py = sub(mul(v, (float)h), 0.5f);
    int x0 = (int)floorf(px), y0 = (int)floorf(py);
    int x1 = x0 + 1, y1 = y0 + 1;
    float fx = g_fract(px), fy = g_fract(py);
    int cx0 = min(max(x0, 0), w - 1), cx1 = min(max(x1, 0), w - 1);
    int cy0 = min(max(y0, 0), h - 1), cy1 = min(max(y1, 0), h - 1);
    float4 c00 = texel4(img, w, h, cx0, cy0), c10 = texel4(img, w, h, cx1, cy0);
    float4 c01 = texel4(img, w, h, cx0, cy1), c11 = texel4(img, w, h, cx1, cy1);
    return mix4(mix4(c00, c10, fx), mix4(c01, c11, fx), fy);
}

__global__ void taa_kernel(const float4* __restrict__ cur_color, const float* __restrict__ cur_depth,
                           const float4* __restrict__ hist_color, const float4* __restrict__ hist_xyz, int w, int h,
                           TaaUniforms U, float4* __restrict__ out_color, float4* __restrict__ out_xyz,
                           __nv_bfloat16* __restrict__ features) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float* vo = U.viewport_orthographic;
    const float* fc = U.focal_clip;
    const float* pfc = U.prev_focal_clip;
    const float u = dv(add((float)x, 0.5f), (float)w), v = dv(add((float)y, 0.5f), (float)h);
    const float4 cc = texel4(cur_color, w, h, x, y);
    const float depth = cur_depth[(size_t)(h - 1 - y) * w + x];
    // reconstruct_view_pos (:82-94)
    float z_ndc = sub(mul(depth, 2.0f), 1.0f);
    float view_z = dv(-U.proj_z[1], add(z_ndc, U.proj_z[0]));
    float pxx = mul(u, vo[0]), pxy = mul(v, vo[1]);
    float unflip = mul(sub(1.0f, fc[2]), 0.5f);
    pxy = g_mix(pxy, sub(vo[1], pxy), unflip);
    float cex = sub(pxx, mul(vo[0], 0.5f)), cey = sub(pxy, mul(vo[1], 0.5f));
    float denom = g_mix(dv(fc[0], view_z), -fc[1], vo[2]);
    float vp3[3] = {dv(cex, denom), dv(cey, denom), view_z};
    float world[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        world[r] = add(add(add(mul(U.inv_view[r], vp3[0]), mul(U.inv_view[4 + r], vp3[1])), mul(U.inv_view[8 + r], vp3[2])),
                       U.inv_view[12 + r]);
    // project_prev_uv (:96-114)
    float pv[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        pv[r] = add(add(add(mul(U.prev_view[r], world[0]), mul(U.prev_view[4 + r], world[1])),
                        mul(U.prev_view[8 + r], world[2])),
                    U.prev_view[12 + r]);
    float puv_x = -1.0f, puv_y = -1.0f;
    if (!(pv[2] >= -0.001f)) {
        float t = vo[3];
        float ppx = add(dv(mul(pfc[0], pv[0]), pv[2]), mul(vo[0], 0.5f));
        float ppy = add(mul(vo[1], 0.5f), dv(mul(pfc[0], pv[1]), pv[2]));
        float opx = add(mul(-pfc[1], pv[0]), mul(vo[0], 0.5f));
        float opy = sub(mul(vo[1], 0.5f), mul(pfc[1], pv[1]));
        float qx = g_mix(ppx, opx, t), qy = g_mix(ppy, opy, t);
        float y_flip = mul(sub(1.0f, pfc[2]), 0.5f);
        qy = g_mix(qy, sub(vo[1], qy), y_flip);
        puv_x = dv(qx, vo[0]);
        puv_y = dv(qy, vo[1]);
    }
    bool valid = U.history_valid != 0.0f && puv_x >= 0.0f && puv_x <= 1.0f && puv_y >= 0.0f && puv_y <= 1.0f;
    float4 hc = make_float4(0.f, 0.f, 0.f, 0.f), hx = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
        hc = bilinear(hist_color, w, h, puv_x, puv_y);
        hx = bilinear(hist_xyz, w, h, puv_x, puv_y);
        float ddx = sub(world[0], hx.x), ddy = sub(world[1], hx.y), ddz = sub(world[2], hx.z);
        float len = __fsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
        valid = hc.w > 0.0f && (U.view_changed == 0.0f || len < 100.0f);
    }
    const size_t o = (size_t)(h - 1 - y) * w + x;
    float4 oc;
    if (valid) {
        float n = g_min(hc.w, 128.0f);
        float n1 = add(n, 1.0f);
        oc = make_float4(dv(add(mul(hc.x, n), cc.x), n1), dv(add(mul(hc.y, n), cc.y), n1),
                         dv(add(mul(hc.z, n), cc.z), n1), g_min(n1, 128.0f));
        out_xyz[o] = make_float4(dv(add(mul(hx.x, n), world[0]), n1), dv(add(mul(hx.y, n), world[1]), n1),
                                 dv(add(mul(hx.z, n), world[2]), n1), 1.0f);
    } else {
        oc = make_float4(cc.x, cc.y, cc.z, 1.0f);
        out_xyz[o] = make_float4(world[0], world[1], world[2], 1.0f);
    }
    out_color[o] = oc;
    if (features) {
        // the denoiser's input: current RGBA, depth, the new history RGB (bf16 pairs), 8 zero channels
        uint4 lo, hi = make_uint4(0u, 0u, 0u, 0u);
        __nv_bfloat162* pp = reinterpret_cast<__nv_bfloat162*>(&lo);
        pp[0] = __floats2bfloat162_rn(cc.x, cc.y);
        pp[1] = __floats2bfloat162_rn(cc.z, cc.w);
        pp[2] = __floats2bfloat162_rn(depth, oc.x);
        pp[3] = __floats2bfloat162_rn(oc.y, oc.z);
        uint4* fo = reinterpret_cast<uint4*>(features + o * 16);
        fo[0] = lo;
        fo[1] = hi;
    }
}

static unsigned grid_for(size_t n, unsigned cap = 148 * 16) {
    size_t g = (n + 255) / 256;
    if (g > cap) g = cap;
    return g ? (unsigned)g : 1u;
}

int launch_accum(const float4* sample, const float4* history, float n, float4* out, size_t npix, cudaStream_t s) {
    launch_pdl(accum_kernel, dim3(grid_for(npix)), dim3(256), 0, s, sample, history, n, out, npix);
    return 1;
}

int launch_to_half(const float4* src, uint16_t* dst, size_t npix, cudaStream_t s) {
    launch_pdl(to_half_kernel, dim3(grid_for(npix)), dim3(256), 0, s, src, reinterpret_cast<uint2*>(dst), npix);
    return 1;
}

int launch_taa(const float4* cur_color, const float* cur_depth, const float4* hist_color, const float4* hist_xyz,
               int w, int h, const TaaUniforms& u, float4* out_color, float4* out_xyz, cudaStream_t s,
               void* features) {
    dim3 block(16, 16), grid((w + 15) / 16, (h + 15) / 16);
    launch_pdl(taa_kernel, grid, block, 0, s, cur_color, cur_depth, hist_color, hist_xyz, w, h, u, out_color, out_xyz,
               static_cast<__nv_bfloat16*>(features));
    return 1;
}

int ensure_stochastic_targets(StochasticTargets& t, int w, int h, cudaStream_t s) {
    if (t.width == w && t.height == h && t.sample) return 0;
    release_stochastic_targets(t);
    const size_t npix = (size_t)w * h;
    if (gs::device_malloc(reinterpret_cast<void**>(&t.sample), npix * 16) != cudaSuccess) return GS_ERR_OOM;
    if (gs::device_malloc(reinterpret_cast<void**>(&t.depth), npix * 4) != cudaSuccess) return GS_ERR_OOM;
    for (int k = 0; k < 2; ++k) {
        if (gs::device_malloc(reinterpret_cast<void**>(&t.accum[k]), npix * 16) != cudaSuccess) return GS_ERR_OOM;
        if (gs::device_malloc(reinterpret_cast<void**>(&t.xyz[k]), npix * 16) != cudaSuccess) return GS_ERR_OOM;
        if (gs::device_malloc(reinterpret_cast<void**>(&t.frame_avg[k]), npix * 16) != cudaSuccess) return GS_ERR_OOM;
        cudaMemsetAsync(t.accum[k], 0, npix * 16, s);
        cudaMemsetAsync(t.xyz[k], 0, npix * 16, s);
        cudaMemsetAsync(t.frame_avg[k], 0, npix * 16, s);
    }
    cudaMemsetAsync(t.sample, 0, npix * 16, s);
    cudaMemsetAsync(t.depth, 0, npix * 4, s);
    t.width = w;
    t.height = h;
    return 0;
}

void release_stochastic_targets(StochasticTargets& t) {
    cudaFree(t.sample);
    cudaFree(t.depth);
    for (int k = 0; k < 2; ++k) {
        cudaFree(t.accum[k]);
        cudaFree(t.xyz[k]);
        cudaFree(t.frame_avg[k]);
    }
    t = StochasticTargets{};
}

bool mat4_inverse(const float m[16], float out[16]) {
    // The reference's inverse (src/renderer.cpp:86-206, used for the TAA's
    // inv_view at :2324): the adjugate by cofactor expansion, with the same
    // products in the same order so the uniforms match bit for bit.  Entry
    // k = 4c + r (m is column-major, m[4 * col + row]) is (-1)^(c+r) times the
    // 3x3 determinant over rows R != c and columns Q != r, summed as six
    // triple products m[a][R0] * m[b][Rx] * m[d][Ry] left to right: a runs
    // over Q in order (signs +, -, + per a), b < d are the other two columns,
    // (Rx, Ry) = (R1, R2) then (R2, R1) with the opposite sign.
    float inv[16];
    for (int k = 0; k < 16; ++k) {
        const int c = k >> 2, r = k & 3;
        int R[3], Q[3];
        for (int i = 0, n = 0; i < 4; ++i)
            if (i != c) R[n++] = i;
        for (int i = 0, n = 0; i < 4; ++i)
            if (i != r) Q[n++] = i;
        const bool flip = ((c + r) & 1) != 0;
        float acc = 0.0f;
        for (int t = 0; t < 6; ++t) {
            const int ai = t >> 1, sw = t & 1;
            const int a = Q[ai], b = Q[ai == 0 ? 1 : 0], d = Q[ai == 2 ? 1 : 2];
            const float p = (m[a * 4 + R[0]] * m[b * 4 + (sw ? R[2] : R[1])]) * m[d * 4 + (sw ? R[1] : R[2])];
            const bool minus = ((ai == 1) != (sw == 1)) != flip;
            acc = t == 0 ? (minus ? -p : p) : (minus ? acc - p : acc + p);
        }
        inv[k] = acc;
    }
    float det = ((m[0] * inv[0] + m[1] * inv[4]) + m[2] * inv[8]) + m[3] * inv[12];
    if (std::fabs(det) <= 1.0e-8f) return false;
    det = 1.0f / det;
    for (int i = 0; i < 16; ++i) out[i] = inv[i] * det;
    return true;
}

}  // namespace gs
