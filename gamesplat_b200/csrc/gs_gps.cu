// Gaussian Point Splatting (shaders/gps.glsl, driven by
// src/renderer.cpp:1964-2118) for the B200.
//
//   clear    packed[] = (0xFFFFFFFF << 32) | 0           (gps.glsl:32-41)
//   expand   per visible Gaussian: expected point count ss^2 2pi sqrt(det)
//            Li2(alpha) with stochastic rounding, atomic reservation of work
//            items bounded by the budget (overflow flag), prepared record,
//            work list                                       (gps.glsl:120-174)
//   splat    one thread per work item, ss^2 points each by inverse-dilog
//            radial sampling; depth and colour are resolved with ONE 64-bit
//            atomicMin on (depth_key << 32 | colour), the race-free form the
//            reference names as its final design (gps.glsl:1-4) -- its
//            prototype's separate atomicMin + colour store (gps.glsl:277-283)
//            can keep a farther splat's colour.  A plain load skips the atomic
//            when the stored value is already smaller.   (gps.glsl:232-285)
//   resolve  ss x ss box average to RGBA + depth             (gps.glsl:344-385)
// The packed buffer (8 B per sub-pixel, 66 MB at 1080p ss=2) stays in L2.
// Transcendentals use the deterministic device functions, so every point
// lands on the same sub-pixel as in the CPU oracle.
#include <algorithm>

#include "gs_common.cuh"
#include "gs_extra.h"

namespace gs {

__device__ __forceinline__ float hash01(uint32_t x) {
    x ^= x >> 16u;
    x *= 0x7feb352du;
    x ^= x >> 15u;
    x *= 0x846ca68bu;
    x ^= x >> 16u;
    return mul(__uint2float_rn(x), 1.0f / 4294967296.0f);
}

__global__ void gps_clear_kernel(unsigned long long* packed, size_t count) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        packed[i] = 0xFFFFFFFF00000000ull;
}

__global__ void gps_expand_kernel(GpsParams p, float4* __restrict__ prepared, uint2* __restrict__ work) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    const uint32_t n_vis = p.fc->visible_count;
    const float ss = (float)p.supersample;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n_vis; v += gridDim.x * blockDim.x) {
        const uint32_t splat_id = p.vis_ids[v];
        const float4* P = p.projected + (size_t)splat_id * 4;
        const float4 co = P[0], cr = P[1], cd = P[2], cv = P[3];
        const float ssf = g_max(ss, 1.0f);
        const float cov_a = add(cv.x, 0.3f), cov_b = cv.y, cov_c = add(cv.z, 0.3f);
        const float det = sub(mul(cov_a, cov_c), mul(cov_b, cov_b));
        const float expected = mul(mul(mul(mul(ssf, ssf), 6.28318530718f), __fsqrt_rn(g_max(det, 0.0f))),
                                   det_dilog(g_clamp(co.w, 0.0f, 1.0f)));
        const float ppw = g_max(mul(ssf, ssf), 1.0f);
        const float scaled = g_max(dv(expected, ppw), 0.0f);
        uint32_t wic = g_f2u_sat(g_clamp(floorf(scaled), 0.0f, 4294967295.0f));
        if (hash01(splat_id + 0x9e3779b9u) < g_fract(scaled) && wic < 0xFFFFFFFFu) wic += 1u;
        if (wic == 0u) continue;
        const uint32_t base = atomicAdd(&p.fc->gps_work[0], wic);
        const uint32_t cap = p.max_work_items;
        if (base >= cap || wic > cap - base) atomicOr(&p.fc->gps_work[1], 1u);
        if (base >= cap) continue;
        const uint32_t write_count = min(wic, cap - base);
        const float l00 = __fsqrt_rn(g_max(cov_a, 1.0e-5f));
        const float l10 = dv(cov_b, l00);
        const float l11 = __fsqrt_rn(g_max(sub(cov_c, mul(l10, l10)), 1.0e-5f));
        const float alpha = g_clamp(co.w, 1.0e-6f, 1.0f);
        const float dilog_alpha = det_dilog(alpha);
        const float ndc = cd.w;
        const float z = g_mix(add(mul(ndc, 0.5f), 0.5f), ndc, p.clip_z_01);
        const uint32_t depth_key = g_f2u_sat(mul(g_clamp(z, 0.0f, 1.0f), 4294967294.0f));
        uint32_t color;
        if (p.linear_color) {
            color = splat_id;
        } else {
            uint32_t r = __float2uint_rn(mul(g_clamp(co.x, 0.0f, 1.0f), 255.0f));
            uint32_t g = __float2uint_rn(mul(g_clamp(co.y, 0.0f, 1.0f), 255.0f));
            uint32_t b = __float2uint_rn(mul(g_clamp(co.z, 0.0f, 1.0f), 255.0f));
            color = r | (g << 8u) | (b << 16u) | 0xFF000000u;
        }
        float4* pr = prepared + (size_t)v * 3;
        pr[0] = make_float4(cr.x, cr.y, l00, l10);
        pr[1] = make_float4(l11, alpha, dilog_alpha, 0.0f);
        pr[2] = make_float4(__uint_as_float(depth_key), __uint_as_float(color), __uint_as_float(splat_id), 0.0f);
        for (uint32_t i = 0; i < write_count; ++i) work[base + i] = make_uint2(v, i);
    }
}

__global__ void gps_splat_kernel(GpsParams p, const float4* __restrict__ prepared, const uint2* __restrict__ work,
                                 unsigned long long* __restrict__ packed) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    const uint32_t total = min(p.fc->gps_work[0], p.max_work_items);
    const int gw = p.width * (int)p.supersample, gh = p.height * (int)p.supersample;
    const float ss = (float)p.supersample;
    const int ppw = max((int)rintf(mul(ss, ss)), 1);
    const uint32_t fseed = g_f2u_sat(p.frame_seed);
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < total; w += gridDim.x * blockDim.x) {
        const uint2 wk = work[w];
        const float4* pr = prepared + (size_t)wk.x * 3;
        const float4 mb = pr[0], sm = pr[1], pk = pr[2];
        const uint32_t depth_key = __float_as_uint(pk.x), color = __float_as_uint(pk.y);
        const uint32_t splat_id = __float_as_uint(pk.z);
        const unsigned long long val = ((unsigned long long)depth_key << 32) | color;
        const uint32_t seed_x = splat_id * 747796405u + fseed * 2891336453u;
        const uint32_t seed_y = splat_id * 277803737u + 0x9E3779B9u;
        for (int pt = 0; pt < ppw; ++pt) {
            uint32_t sx = seed_x + (wk.y * (uint32_t)ppw + (uint32_t)pt) * 374761393u, sy = seed_y;
            sx = 1664525u * sx + 1013904223u;
            sy = 1664525u * sy + 1013904223u;
            sx += 1664525u * sy;
            sy += 1664525u * sx;
            sx ^= sx >> 16u;
            sy ^= sy >> 16u;
            sx += 1664525u * sy;
            sy += 1664525u * sx;
            sx ^= sx >> 16u;
            sy ^= sy >> 16u;
            const float r0 = mul(__uint2float_rn(sx), 2.32830643654e-10f);
            const float r1 = mul(__uint2float_rn(sy), 2.32830643654e-10f);
            float arg = dv(det_inv_dilog(mul(sub(1.0f, r0), sm.z)), sm.y);
            arg = g_clamp(arg, 1.0e-7f, 1.0f);
            const float radius = __fsqrt_rn(mul(-2.0f, det_logf(arg)));
            const float az = mul(6.28318530718f, r1);
            float sn, cs;
            det_sincosf(az, &sn, &cs);
            const float lx = mul(cs, radius), ly = mul(sn, radius);
            const float ptx = mul(add(mb.x, mul(mb.z, lx)), g_max(ss, 1.0f));
            const float pty = mul(add(mb.y, add(mul(mb.w, lx), mul(sm.x, ly))), g_max(ss, 1.0f));
            const float fx = floorf(add(ptx, 0.5f)), fy = floorf(add(pty, 0.5f));
            if (fx >= 0.0f && fy >= 0.0f && fx < (float)gw && fy < (float)gh) {
                unsigned long long* dst = packed + (size_t)fy * gw + (size_t)fx;
                if (val < *reinterpret_cast<volatile unsigned long long*>(dst)) atomicMin(dst, val);
            }
        }
    }
}

__global__ void gps_resolve_kernel(GpsParams p, const unsigned long long* __restrict__ packed) {
    pdl_wait();   // launched as a programmatic dependent of the frame's previous kernel
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.width || y >= p.height) return;
    const int ss = (int)p.supersample;
    const int gw = p.width * ss, gh = p.height * ss;
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, cov = 0.0f;
    uint32_t min_key = 0xFFFFFFFFu;
    for (int yy = 0; yy < ss; ++yy) {
        for (int xx = 0; xx < ss; ++xx) {
            const int sxp = x * ss + xx, syp = y * ss + yy;
            if (sxp >= gw || syp >= gh) continue;
            const unsigned long long v = packed[(size_t)syp * gw + sxp];
            const uint32_t key = (uint32_t)(v >> 32), payload = (uint32_t)v;
            if (key != 0xFFFFFFFFu) {
                if (p.linear_color) {
                    const float4 q = p.projected[(size_t)payload * 4];
                    s0 = add(s0, q.x);
                    s1 = add(s1, q.y);
                    s2 = add(s2, q.z);
                } else {
                    s0 = add(s0, dv((float)(payload & 255u), 255.0f));
                    s1 = add(s1, dv((float)((payload >> 8u) & 255u), 255.0f));
                    s2 = add(s2, dv((float)((payload >> 16u) & 255u), 255.0f));
                }
                cov = add(cov, 1.0f);
                min_key = min(min_key, key);
            }
        }
    }
    const size_t o = (size_t)(p.height - 1 - y) * p.width + x;
    if (cov <= 0.0f) {
        p.out_color[o] = make_float4(p.bg, p.bg, p.bg, 0.0f);
        p.out_depth[o] = 1.0f;
    } else {
        const float spc = (float)(ss * ss);
        p.out_color[o] = make_float4(dv(s0, spc), dv(s1, spc), dv(s2, spc), dv(cov, spc));
        p.out_depth[o] = dv(__uint2float_rn(min_key), 4294967294.0f);
    }
}

int ensure_gps_targets(GpsTargets& g, int width, int height, uint32_t ss, uint32_t n, uint32_t max_work_items,
                       cudaStream_t s) {
    (void)s;
    if (g.width != width || g.height != height || g.ss != ss || !g.packed) {
        cudaFree(g.packed);
        g.packed = nullptr;
        g.width = g.height = 0;
        g.ss = 0;
        size_t count = (size_t)width * ss * height * ss;
        if (gs::device_malloc(reinterpret_cast<void**>(&g.packed), count * 8) != cudaSuccess) return GS_ERR_OOM;
        g.width = width;
        g.height = height;
        g.ss = ss;
    }
    if (g.prepared_cap < n || !g.prepared) {
        cudaFree(g.prepared);
        g.prepared = nullptr;
        g.prepared_cap = 0;
        if (gs::device_malloc(reinterpret_cast<void**>(&g.prepared), (size_t)(n ? n : 1) * 48) != cudaSuccess) return GS_ERR_OOM;
        g.prepared_cap = n;
    }
    if (!g.work || g.work_cap != max_work_items) {
        int rc = resize_gps_work(g, max_work_items, s);
        if (rc) return rc;
    }
    return 0;
}

// src/renderer.cpp:1076-1123: allocate the replacement first, keep the old
// buffer when that fails.
int resize_gps_work(GpsTargets& g, uint32_t max_work_items, cudaStream_t s) {
    (void)s;
    if (max_work_items == 0) return GS_ERR_BAD_ARG;
    if (g.work && g.work_cap == max_work_items) return 0;
    uint2* nw = nullptr;
    if (gs::device_malloc(reinterpret_cast<void**>(&nw), (size_t)max_work_items * sizeof(uint2)) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_OOM;
    }
    cudaFree(g.work);
    g.work = nw;
    g.work_cap = max_work_items;
    return 0;
}

void release_gps_targets(GpsTargets& g) {
    cudaFree(g.packed);
    g.packed = nullptr;
    g.width = g.height = 0;
    g.ss = 0;
}

void release_gps_scene(GpsTargets& g) {
    cudaFree(g.prepared);
    g.prepared = nullptr;
    g.prepared_cap = 0;
    cudaFree(g.work);
    g.work = nullptr;
    g.work_cap = 0;
}

int launch_gps(GpsTargets& g, const GpsParams& p, uint32_t n_cap, uint32_t num_sms, cudaStream_t s) {
    const size_t count = (size_t)g.width * g.ss * g.height * g.ss;
    unsigned cg = (unsigned)std::min<size_t>((count + 255) / 256, (size_t)num_sms * 16);
    launch_pdl(gps_clear_kernel, dim3(cg ? cg : 1), dim3(256), 0, s, g.packed, count);
    unsigned eg = (unsigned)std::min<size_t>((n_cap + 255) / 256, (size_t)num_sms * 8);
    launch_pdl(gps_expand_kernel, dim3(eg ? eg : 1), dim3(256), 0, s, p, g.prepared, g.work);
    unsigned sg = (unsigned)std::min<size_t>(((size_t)g.work_cap + 255) / 256, (size_t)num_sms * 16);
    launch_pdl(gps_splat_kernel, dim3(sg ? sg : 1), dim3(256), 0, s, p, g.prepared, g.work, g.packed);
    dim3 block(16, 16), grid((p.width + 15) / 16, (p.height + 15) / 16);
    launch_pdl(gps_resolve_kernel, grid, block, 0, s, p, g.packed);
    return 4;
}

}  // namespace gs
