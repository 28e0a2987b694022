// Tile rasterizer: replaces the reference's GL instanced-quad draw, fragment
// shader and fixed-function blender (shaders/splat.glsl:39-145,
// src/renderer.cpp:266-320, 1687-1720).
//
// One CTA per 16x16 pixel tile, two pixels per thread, each warp an 8x8 pixel
// block (GL window coordinates, row 0 at the bottom; the image is written
// top row first).  Control flow is warp-uniform: lanes never diverge around
// the per-splat loop (per-pixel work is predicated), a warp skips splats whose
// rectangle misses its block and leaves the loop when all its pixels are done.  The tile's
// depth-ordered splat list is walked front to back (reverse of the
// reference's back-to-front draw order, so equal depth keys are visited in
// descending splat index, which reproduces "later instance on top").
// Batches of 128 64-byte RasterRecords are staged into shared memory by TMA
// 1-D bulk copies (cp.async.bulk, completion on an mbarrier), double
// buffered so the next batch lands while the current one is composited.
//
// Alpha mode: premultiplied "over" in FP32, front to back:
//   C += T * alpha * rgb,  T *= 1 - alpha,  output (C + T*bg, 1 - T),
// which equals the reference's back-to-front ONE / ONE_MINUS_SRC_ALPHA
// blend into a (bg,bg,bg,0) target up to FP32 rounding.  A pixel stops once
// T < 2^-13: the skipped remainder is below T * max(rgb, bg).  Coverage
// (quad rectangle) and the two discards (power > 0, power < cutoff) are
// evaluated bit-exactly like the CPU oracle; alpha uses the hardware exp.
//
// Stochastic mode: a fragment is kept iff hash13(fragcoord, id + seed) <
// alpha; the depth test (LESS, writes on) keeps the kept fragment with the
// smallest (D24 depth, instance index).  Walking front to back, a pixel stops
// once a splat's D24 exceeds the kept one's by more than 8 (the float
// depth-to-D24 mapping is monotone to within 5 units).  Deterministic exp and
// hash, so the kept set matches the oracle bit for bit.
#include <cuda_fp16.h>

#include "gs_common.cuh"
#include "gs_internal.h"
#include "gs_tma.cuh"

namespace gs {

constexpr int kRasterThreads = kTileW * kTileH / 2;   // two pixels per thread
constexpr int kBatch = 128;
constexpr float kTransmittanceMin = 1.0f / 8192.0f;
constexpr uint32_t kDepthMargin = 8;

__device__ __forceinline__ float hash13(float p0, float p1, float p2) {
    p0 = g_fract(mul(p0, 0.1031f));
    p1 = g_fract(mul(p1, 0.1031f));
    p2 = g_fract(mul(p2, 0.1031f));
    float d = add(add(mul(p0, add(p1, 33.33f)), mul(p1, add(p2, 33.33f))), mul(p2, add(p0, 33.33f)));
    p0 = add(p0, d);
    p1 = add(p1, d);
    p2 = add(p2, d);
    return g_fract(mul(add(p0, p1), p2));
}

struct AlphaState {
    float T, c0, c1, c2;
};

struct StochState {
    uint32_t best_d24, best_id;
    float r, g, b;
};

// Per-pixel compositing state and the per-pixel step of each mode.
__device__ __forceinline__ void alpha_step(AlphaState& A, bool& done, float power, float opacity, float r, float g,
                                           float b) {
    const float alpha = fminf(opacity * __expf(power), 0.99f);
    const float w = alpha * A.T;
    A.c0 = fmaf(w, r, A.c0);
    A.c1 = fmaf(w, g, A.c1);
    A.c2 = fmaf(w, b, A.c2);
    A.T = A.T * (1.0f - alpha);
    done = A.T < kTransmittanceMin;
}

__device__ __forceinline__ void stoch_step(StochState& S, float power, float opacity, float fcx, float fcy,
                                           float hz, uint32_t z24, uint32_t id, float r, float g, float b) {
    const float alpha = g_min(mul(opacity, det_expf(power)), 0.99f);
    const float rnd = hash13(fcx, fcy, hz);
    if (rnd < alpha) {
        S.best_d24 = z24;
        S.best_id = id;
        S.r = r;
        S.g = g;
        S.b = b;
    }
}

__device__ __forceinline__ void write_pixel_alpha(const RasterParams& p, int px, int py, const AlphaState& A) {
    const size_t o = (size_t)(p.height - 1 - py) * p.width + px;
    const float r = fmaf(A.T, p.bg, A.c0), g = fmaf(A.T, p.bg, A.c1), b = fmaf(A.T, p.bg, A.c2);
    const float a = 1.0f - A.T;
    __half2 h01 = __floats2half2_rn(r, g), h23 = __floats2half2_rn(b, a);
    uint2 packed;
    packed.x = *reinterpret_cast<uint32_t*>(&h01);
    packed.y = *reinterpret_cast<uint32_t*>(&h23);
    reinterpret_cast<uint2*>(p.out_rgba16f)[o] = packed;
}

__device__ __forceinline__ void write_pixel_stoch(const RasterParams& p, int px, int py, const StochState& S) {
    const size_t o = (size_t)(p.height - 1 - py) * p.width + px;
    float4 c;
    if (S.best_id == 0xFFFFFFFFu) c = make_float4(p.bg, p.bg, p.bg, 0.0f);
    else c = make_float4(S.r, S.g, S.b, 1.0f);
    if (p.rgba8) {
        c.x = rintf(g_clamp(c.x, 0.0f, 1.0f) * 255.0f) / 255.0f;
        c.y = rintf(g_clamp(c.y, 0.0f, 1.0f) * 255.0f) / 255.0f;
        c.z = rintf(g_clamp(c.z, 0.0f, 1.0f) * 255.0f) / 255.0f;
        c.w = rintf(g_clamp(c.w, 0.0f, 1.0f) * 255.0f) / 255.0f;
    }
    if (p.out_rgba32f) p.out_rgba32f[o] = c;
    if (p.out_depth) p.out_depth[o] = (float)S.best_d24 / 16777215.0f;
    if (p.out_rgba16f) {
        __half2 h01 = __floats2half2_rn(c.x, c.y), h23 = __floats2half2_rn(c.z, c.w);
        uint2 packed;
        packed.x = *reinterpret_cast<uint32_t*>(&h01);
        packed.y = *reinterpret_cast<uint32_t*>(&h23);
        reinterpret_cast<uint2*>(p.out_rgba16f)[o] = packed;
    }
}

// One CTA of 128 threads per 16x16 tile; warp w owns the 8x8 block
// (w & 1, w >> 1); lane l shades pixels (l & 7, l >> 3) and (l & 7, (l >> 3) + 4)
// of it: the two pixels share a column, hence dx, the column test and the
// first term of the Gaussian exponent.
template <int kMode>  // 0 = alpha, 1 = stochastic
__global__ void __launch_bounds__(kRasterThreads) raster_kernel(RasterParams p) {
    __shared__ __align__(128) RasterRecord s_rec[2][kBatch];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint8_t s_mask[kBatch];

    const uint32_t tile = blockIdx.x;
    const int tx = (int)(tile % (uint32_t)p.tiles_x), ty = (int)(tile / (uint32_t)p.tiles_x);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bx0 = tx * kTileW + (warp & 1) * 8, by0 = ty * kTileH + (warp >> 1) * 8;
    const int px = bx0 + (lane & 7), py0 = by0 + (lane >> 3), py1 = py0 + 4;
    const bool in0 = px < p.width && py0 < p.height, in1 = px < p.width && py1 < p.height;
    const uint2 range = p.tile_ranges[tile];
    const uint32_t n = range.y > range.x ? range.y - range.x : 0u;
    const uint32_t* __restrict__ vals = p.tile_plan->vfinal;

    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();

    const float fcx = (float)px + 0.5f, fcy0 = (float)py0 + 0.5f, fcy1 = (float)py1 + 0.5f;
    AlphaState A0 = {1.0f, 0.0f, 0.0f, 0.0f}, A1 = A0;
    StochState S0 = {16777215u, 0xFFFFFFFFu, 0.0f, 0.0f, 0.0f}, S1 = S0;
    bool done0 = !in0, done1 = !in1;
    bool failed = false;
    const uint32_t nb = (n + kBatch - 1) / kBatch;
    uint32_t phase0 = 0, phase1 = 0;

    auto issue = [&](uint32_t b) {
        const uint32_t first = b * kBatch;
        const uint32_t cnt = min((uint32_t)kBatch, n - first);
        uint64_t* bar = &s_bar[b & 1];
        if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, cnt * (uint32_t)sizeof(RasterRecord));
        if (threadIdx.x < cnt) {
            const uint32_t s = min(vals[range.y - 1 - (first + threadIdx.x)], p.record_cap - 1u);
            bulk_g2s(&s_rec[b & 1][threadIdx.x], p.records + s, (uint32_t)sizeof(RasterRecord), bar);
        }
    };

    if (nb > 0) issue(0);
    for (uint32_t b = 0; b < nb; ++b) {
        if (b + 1 < nb) issue(b + 1);
        const uint32_t ph = (b & 1) ? phase1 : phase0;
        if (!mbar_wait_bounded(&s_bar[b & 1], ph)) failed = true;
        if (b & 1) phase1 ^= 1u; else phase0 ^= 1u;
        const uint32_t cnt = min((uint32_t)kBatch, n - b * kBatch);
        const RasterRecord* recs = s_rec[b & 1];
        // Which of the four 8x8 warp blocks each staged splat's rectangle
        // touches (one thread per record); warps then visit only their own.
        if (threadIdx.x < cnt) {
            const uint4 q2 = reinterpret_cast<const uint4*>(recs + threadIdx.x)[2];
            const int i0 = (int)(q2.z & 0xFFFFu), i1 = (int)(q2.z >> 16);
            const int j0 = (int)(q2.w & 0xFFFFu), j1 = (int)(q2.w >> 16);
            const int x0 = tx * kTileW, y0 = ty * kTileH;
            const uint32_t cols = (uint32_t)(i0 < x0 + 8 && i1 > x0) | ((uint32_t)(i0 < x0 + 16 && i1 > x0 + 8) << 1);
            const uint32_t rows = (uint32_t)(j0 < y0 + 8 && j1 > y0) | ((uint32_t)(j0 < y0 + 16 && j1 > y0 + 8) << 1);
            // block w = (w & 1, w >> 1): bit w set iff its column and row halves are covered
            s_mask[threadIdx.x] = (uint8_t)((cols & (rows & 1u ? 3u : 0u)) | ((cols & (rows & 2u ? 3u : 0u)) << 2));
        }
        __syncthreads();
        // Warp-uniform control flow only; per-pixel work is predicated.
        bool warp_done = __all_sync(0xffffffffu, (done0 && done1) || failed);
        for (uint32_t c = 0; c < cnt && !warp_done; c += 32) {
            const bool mine = c + lane < cnt && ((s_mask[c + lane] >> warp) & 1u);
            uint32_t todo = __ballot_sync(0xffffffffu, mine);
            while (todo) {
                const uint32_t j = c + (uint32_t)(__ffs(todo) - 1);
                todo &= todo - 1u;
                const uint4 q2 = reinterpret_cast<const uint4*>(recs + j)[2];
                const float4 q0 = reinterpret_cast<const float4*>(recs + j)[0];
                const float4 q1 = reinterpret_cast<const float4*>(recs + j)[1];
                const int i0 = (int)(q2.z & 0xFFFFu), i1 = (int)(q2.z >> 16);
                const int j0 = (int)(q2.w & 0xFFFFu), j1 = (int)(q2.w >> 16);
                const bool colx = px >= i0 && px < i1;
                // splat_power() evaluated for both pixels with the shared first term
                const float dx = sub(fcx, q0.x);
                const float t0 = mul(mul(q0.z, dx), dx);
                const float dy0 = sub(fcy0, q0.y), dy1 = sub(fcy1, q0.y);
                const float pw0 = mul(-0.5f, add(add(t0, mul(mul(q0.w, dx), dy0)), mul(mul(q1.x, dy0), dy0)));
                const float pw1 = mul(-0.5f, add(add(t0, mul(mul(q0.w, dx), dy1)), mul(mul(q1.x, dy1), dy1)));
                const bool live0 = !done0 && colx && py0 >= j0 && py0 < j1 && (pw0 <= 0.0f) && !(pw0 < q1.z);
                const bool live1 = !done1 && colx && py1 >= j0 && py1 < j1 && (pw1 <= 0.0f) && !(pw1 < q1.z);
                if (kMode == 0) {
                    const float g = __uint_as_float(q2.x), bb = __uint_as_float(q2.y);
                    if (live0) alpha_step(A0, done0, pw0, q1.y, q1.w, g, bb);
                    if (live1) alpha_step(A1, done1, pw1, q1.y, q1.w, g, bb);
                    if (__all_sync(0xffffffffu, (done0 && done1) || failed)) { warp_done = true; break; }
                } else {
                    const uint4 q3 = reinterpret_cast<const uint4*>(recs + j)[3];
                    const uint32_t z24 = q3.x, id = q3.y;
                    // a pixel stops once splats are beyond its kept depth (+ margin)
                    if (S0.best_id != 0xFFFFFFFFu && z24 > S0.best_d24 + kDepthMargin) done0 = true;
                    if (S1.best_id != 0xFFFFFFFFu && z24 > S1.best_d24 + kDepthMargin) done1 = true;
                    if (__all_sync(0xffffffffu, (done0 && done1) || failed)) { warp_done = true; break; }
                    const bool b0 = z24 < S0.best_d24 || (z24 == S0.best_d24 && id < S0.best_id);
                    const bool b1 = z24 < S1.best_d24 || (z24 == S1.best_d24 && id < S1.best_id);
                    const float g = __uint_as_float(q2.x), bb = __uint_as_float(q2.y);
                    const float hz = __uint_as_float(q3.z);
                    if (live0 && !done0 && b0) stoch_step(S0, pw0, q1.y, fcx, fcy0, hz, z24, id, q1.w, g, bb);
                    if (live1 && !done1 && b1) stoch_step(S1, pw1, q1.y, fcx, fcy1, hz, z24, id, q1.w, g, bb);
                }
            }
        }
        const int all_done = __syncthreads_and(warp_done || (done0 && done1) || failed);
        if (all_done) {
            if (b + 1 < nb) {
                const uint32_t ph2 = ((b + 1) & 1) ? phase1 : phase0;
                if (!mbar_wait_bounded(&s_bar[(b + 1) & 1], ph2)) failed = true;
            }
            break;
        }
    }
    if (failed) atomicOr(&p.fc->error_flags, kErrRasterWait);
    if (kMode == 0) {
        if (in0) write_pixel_alpha(p, px, py0, A0);
        if (in1) write_pixel_alpha(p, px, py1, A1);
    } else {
        if (in0) write_pixel_stoch(p, px, py0, S0);
        if (in1) write_pixel_stoch(p, px, py1, S1);
    }
}

int launch_raster_alpha(const RasterParams& p, cudaStream_t s) {
    const uint32_t tiles = (uint32_t)p.tiles_x * (uint32_t)p.tiles_y;
    if (tiles == 0) return 0;
    raster_kernel<0><<<tiles, kRasterThreads, 0, s>>>(p);
    return 1;
}

int launch_raster_stochastic(const RasterParams& p, cudaStream_t s) {
    const uint32_t tiles = (uint32_t)p.tiles_x * (uint32_t)p.tiles_y;
    if (tiles == 0) return 0;
    raster_kernel<1><<<tiles, kRasterThreads, 0, s>>>(p);
    return 1;
}

}  // namespace gs
