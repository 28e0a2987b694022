// Tile rasterizer: replaces the reference's GL instanced-quad draw, fragment
// shader and fixed-function blender (shaders/splat.glsl:39-145,
// src/renderer.cpp:266-320, 1687-1720).
//
// One CTA per 16x16 pixel tile, two pixels per thread, each warp an 8x8 pixel
// block (GL window coordinates, row 0 at the bottom; the image is written
// top row first).  Control flow is warp-uniform: lanes never diverge around
// the per-splat loop (per-pixel work is predicated or selected), a warp skips
// splats whose rectangle misses its block and leaves the loop when all its
// pixels are done.  The tile's splat list (descending sorted position) is
// walked front to back (reverse of the reference's back-to-front draw order,
// so equal depth keys are visited in descending splat index, which
// reproduces "later instance on top").  Batches of 128 64-byte RasterRecords
// are staged into shared memory by TMA 1-D bulk copies (cp.async.bulk,
// completion on an mbarrier), double buffered so the next batch lands while
// the current one is composited.  When a batch lands, one thread per record turns its pixel
// rectangle into tile-relative column and row bit masks, so a pixel's
// coverage test is one AND and one compare (in alpha mode the mask is also
// written into the staged record next to g, b: one 16-byte load per splat).
//
// The two pixels of a thread share a column; their arithmetic runs as packed
// f32x2 operations (add/mul/fma .rn on float pairs, each element rounded like
// the scalar operation), which halves the issue slots of the per-pixel math.
// In alpha mode a warp takes its splats two per loop trip (one loop test and
// one "all pixels done" vote per pair).  CTA b rasterizes tile
// tile_order[b]: the heaviest tiles first, so they do not form the last wave.
//
// Alpha mode: premultiplied "over" in FP32, front to back:
//   C += T * alpha * rgb,  T -= T * alpha,  output (C + T*bg, 1 - T),
// which equals the reference's back-to-front ONE / ONE_MINUS_SRC_ALPHA
// blend into a (bg,bg,bg,0) target up to FP32 rounding.  A warp stops once
// T < 2^-13 for all its pixels: the skipped remainder is below T * max(rgb, bg).
// Coverage (quad rectangle) and the two discards (power > 0, power < cutoff)
// are evaluated bit-exactly like the CPU oracle, on the quadratic form s with
// the bounds of RasterRecord; alpha = min(2^(s * -0.5 log2(e) + log2(opacity)),
// 0.99) uses the hardware exp2.
//
// Two-sample mode (the input of the denoised mode): the stochastic sample
// rule below for two seeds at once, on un-jittered records (the alpha
// binning), alpha evaluated once per (pixel, splat) and hashed per seed; a
// pixel stops when both samples are decided.  Writes the mean colour of the
// two samples (background where none kept), the fraction that kept a
// fragment and the mean window depth (1 where none kept), all in float.
//
// Stochastic mode: a fragment is kept iff hash13(fragcoord, id + seed) <
// alpha; the depth test (LESS, writes on) keeps the kept fragment with the
// smallest (D24 depth, instance index).  Walking front to back, a pixel stops
// once a splat's D24 exceeds the kept one's by more than 8 (the float
// depth-to-D24 mapping is monotone to within 5 units).  Deterministic exp and
// hash, so the kept set matches the oracle bit for bit.
#include <cuda_fp16.h>

#include <type_traits>

#include "gs_common.cuh"
#include "gs_internal.h"
#include "gs_tma.cuh"

namespace gs {

constexpr int kRasterThreads = kTileW * kTileH / 2;   // two pixels per thread
constexpr int kBatch = 128;
constexpr float kTransmittanceMin = 1.0f / 8192.0f;
constexpr uint32_t kDepthMargin = 8;
constexpr float kNegHalfLog2e = -0.72134752044448170368f;   // -0.5 / ln(2)

// hash13(x, y, z) (shaders/splat.glsl:121-125), split by what its terms
// depend on: p0 = fract(0.1031 x), p1 = fract(0.1031 y) and the products that
// hold only them belong to the pixel (computed once per tile), p2 =
// fract(0.1031 z) to the splat and sample (once per splat for all the pixels of
// a warp); the rest, per (pixel, splat, sample), is the same operations in the
// same order:  d = p0 (p1 + 33.33) + p1 (p2 + 33.33) + p2 (p0 + 33.33),
// hash = fract((p0 + d + p1 + d) (p2 + d)).
struct PixelHash {
    float p0, p1, t1, p0c;   // p0, p1, p0 (p1 + 33.33), p0 + 33.33
};

__device__ __forceinline__ PixelHash pixel_hash(float x, float y) {
    PixelHash h;
    h.p0 = g_fract(mul(x, 0.1031f));
    h.p1 = g_fract(mul(y, 0.1031f));
    h.t1 = mul(h.p0, add(h.p1, 33.33f));
    h.p0c = add(h.p0, 33.33f);
    return h;
}

__device__ __forceinline__ float hash_z(float z) { return g_fract(mul(z, 0.1031f)); }

__device__ __forceinline__ float hash13(const PixelHash& h, float p2) {
    const float d = add(add(h.t1, mul(h.p1, add(p2, 33.33f))), mul(p2, h.p0c));
    return g_fract(mul(add(add(h.p0, d), add(h.p1, d)), add(p2, d)));
}

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }

struct StochState {
    uint32_t best_d24, best_id;
    float r, g, b;
};

// alpha = min(opacity * exp(power), 0.99) with power <= 0 (exp <= 1 there, also
// for the deterministic exp) never exceeds min(opacity, 0.99): a fragment whose
// hash is at or above that bound is rejected without evaluating exp.
// ph: the pixel's hash terms, hz: hash_z(splat id + sample seed).
__device__ __forceinline__ void stoch_step(StochState& S, float s, float opacity, const PixelHash& ph, float hz,
                                           uint32_t z24, uint32_t id, float r, float g, float b) {
    const float rnd = hash13(ph, hz);
    if (!(rnd < g_min(opacity, 0.99f))) return;
    const float alpha = g_min(mul(opacity, det_expf(mul(-0.5f, s))), 0.99f);
    if (rnd < alpha) {
        S.best_d24 = z24;
        S.best_id = id;
        S.r = r;
        S.g = g;
        S.b = b;
    }
}

// Two samples of one pixel (denoised mode): the kept fragment of each seed.
struct Stoch2 {
    StochState s[2];
    bool done[2];
};

__device__ __forceinline__ void stoch2_init(Stoch2& P, bool inside) {
    for (int k = 0; k < 2; ++k) {
        P.s[k] = {16777215u, 0xFFFFFFFFu, 0.0f, 0.0f, 0.0f};
        P.done[k] = !inside;
    }
}

// One splat into both samples of a pixel: alpha once, one hash per seed.
__device__ __forceinline__ void stoch2_step(Stoch2& P, bool live, float sq, float opacity, const PixelHash& ph,
                                            float hz0, float hz1, uint32_t z24, uint32_t id, float r, float g,
                                            float b) {
    bool want[2];
#pragma unroll
    for (int k = 0; k < 2; ++k)
        want[k] = live && !P.done[k] &&
                  (z24 < P.s[k].best_d24 || (z24 == P.s[k].best_d24 && id < P.s[k].best_id));
    if (!(want[0] || want[1])) return;
    // hashes first: exp only when one of them is below alpha's bound (see stoch_step)
    const float bound = g_min(opacity, 0.99f);
    float rnd[2];
    bool cand[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        rnd[k] = want[k] ? hash13(ph, k ? hz1 : hz0) : 1.0f;
        cand[k] = want[k] && rnd[k] < bound;
    }
    if (!(cand[0] || cand[1])) return;
    const float alpha = g_min(mul(opacity, det_expf(mul(-0.5f, sq))), 0.99f);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (cand[k] && rnd[k] < alpha) {
            P.s[k].best_d24 = z24;
            P.s[k].best_id = id;
            P.s[k].r = r;
            P.s[k].g = g;
            P.s[k].b = b;
        }
    }
}

__device__ __forceinline__ void stoch2_retire(Stoch2& P, uint32_t z24, uint32_t margin) {
#pragma unroll
    for (int k = 0; k < 2; ++k)
        if (P.s[k].best_id != 0xFFFFFFFFu && z24 > P.s[k].best_d24 + margin) P.done[k] = true;
}

__device__ __forceinline__ void write_pixel_stoch2(const RasterParams& p, int px, int py, const Stoch2& P) {
    const size_t o = (size_t)(p.height - 1 - py) * p.width + px;
    float c[2][3], a[2], d[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool kept = P.s[k].best_id != 0xFFFFFFFFu;
        c[k][0] = kept ? P.s[k].r : p.bg;
        c[k][1] = kept ? P.s[k].g : p.bg;
        c[k][2] = kept ? P.s[k].b : p.bg;
        a[k] = kept ? 1.0f : 0.0f;
        d[k] = __fdiv_rn((float)P.s[k].best_d24, 16777215.0f);
    }
    p.out_rgba32f[o] = make_float4(mul(add(c[0][0], c[1][0]), 0.5f), mul(add(c[0][1], c[1][1]), 0.5f),
                                   mul(add(c[0][2], c[1][2]), 0.5f), mul(add(a[0], a[1]), 0.5f));
    p.out_depth[o] = mul(add(d[0], d[1]), 0.5f);
}

__device__ __forceinline__ void write_rgba16f(uint16_t* out, size_t o, float r, float g, float b, float a) {
    __half2 h01 = __floats2half2_rn(r, g), h23 = __floats2half2_rn(b, a);
    uint2 packed;
    packed.x = *reinterpret_cast<uint32_t*>(&h01);
    packed.y = *reinterpret_cast<uint32_t*>(&h23);
    reinterpret_cast<uint2*>(out)[o] = packed;
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
    if (p.accum_out) {   // the frame's running mean, as accum_kernel computes it from the sample
        const float nn = g_max(p.accum_n, 1.0f);
        const float4 h = p.accum_in ? p.accum_in[o] : c;
        p.accum_out[o] = make_float4(add(h.x, dv(sub(c.x, h.x), nn)), add(h.y, dv(sub(c.y, h.y), nn)),
                                     add(h.z, dv(sub(c.z, h.z), nn)), add(h.w, dv(sub(c.w, h.w), nn)));
    }
    if (p.out_rgba16f) write_rgba16f(p.out_rgba16f, o, c.x, c.y, c.z, c.w);
}

// Tile shapes: kTw x kTh pixels, four 8x8 warp blocks (16x16, 32x8, 8x32).
// Coverage masks: column bits from bit 0, row bits from bit RowShift (16 for
// 16x16 tiles, whose masks fit 32 bits; 32 for the others, in 64 bits).
template <int kTw, int kTh>
struct TileShape {
    static_assert(kTw * kTh == 256 && kTw % 8 == 0 && kTh % 8 == 0, "four 8x8 blocks");
    static constexpr int kBx = kTw / 8;          // blocks per row
    static constexpr int kRowShift = kTw == 16 && kTh == 16 ? 16 : 32;
    using Mask = typename std::conditional<kRowShift == 16, uint32_t, unsigned long long>::type;
};

// Tile-relative coverage of a record's pixel rectangle: column bits
// [0, kTw), row bits [RowShift, RowShift + kTh) (bit k = tile column / GL row
// k).  Empty rectangles give 0.
template <int kTw, int kTh>
__device__ __forceinline__ typename TileShape<kTw, kTh>::Mask rect_bits(uint32_t rect_x, uint32_t rect_y, int x0,
                                                                        int y0) {
    using S = TileShape<kTw, kTh>;
    using M = typename S::Mask;
    const int i0 = min(max((int)(rect_x & 0xFFFFu) - x0, 0), kTw), i1 = min(max((int)(rect_x >> 16) - x0, 0), kTw);
    const int j0 = min(max((int)(rect_y & 0xFFFFu) - y0, 0), kTh), j1 = min(max((int)(rect_y >> 16) - y0, 0), kTh);
    if (i1 <= i0 || j1 <= j0) return (M)0;
    const unsigned long long cols = (1ull << i1) - (1ull << i0);
    const unsigned long long rows = (1ull << j1) - (1ull << j0);
    return (M)(cols | (rows << S::kRowShift));
}

// Lower bound of the splat's quadratic form q(d) = A dx^2 + B dx dy + C dy^2
// over the box [X0,X1] x [Y0,Y1] of pixel-centre offsets.  With A, C > 0, q is
// convex along every box edge, and when the box does not hold the origin its
// minimum lies on an edge (a convex q has its only interior stationary point
// at the origin; an indefinite one has none that is a minimum), at the
// clamped stationary point of that edge's 1-D quadratic.
__device__ __forceinline__ float min_q_box(float A, float B, float C, float X0, float X1, float Y0, float Y1) {
    if (X0 <= 0.0f && X1 >= 0.0f && Y0 <= 0.0f && Y1 >= 0.0f) return 0.0f;
    const float ia = -0.5f * B / A, ic = -0.5f * B / C;
    float m = 3.0e38f;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float X = e ? X1 : X0, Y = e ? Y1 : Y0;
        const float dy = fminf(fmaxf(ic * X, Y0), Y1);
        m = fminf(m, fmaf(fmaf(C, dy, B * X), dy, A * X * X));
        const float dx = fminf(fmaxf(ia * Y, X0), X1);
        m = fminf(m, fmaf(fmaf(A, dx, B * Y), dx, C * Y * Y));
    }
    return m;
}

// One CTA of 128 threads per 16x16 tile; warp w owns the 8x8 block
// (w & 1, w >> 1); lane l shades pixels (l & 7, l >> 3) and (l & 7, (l >> 3) + 4)
// of it: the two pixels share a column, hence dx, the column test and the
// first term of the Gaussian exponent.
// Shared memory of one CTA's tile: two staging buffers of records, their
// barriers, the records' coverage bits and warp-block masks.
// A staged record and 16 bytes of padding: at an 80-byte stride the 16-byte
// loads of 8 consecutive records (one record per thread in the staging pass)
// fall in distinct banks, and a 32-bit field of 32 consecutive records spreads
// over 8 banks instead of 2.
struct __align__(16) StagedRecord {
    RasterRecord r;
    uint4 pad;
};

template <int kMode, int kTw = 16, int kTh = 16>
struct __align__(128) RasterShared {
    StagedRecord rec[2][kBatch];
    uint64_t bar[2];
    typename TileShape<kTw, kTh>::Mask bits[kBatch];
    uint8_t mask[kBatch];
    float4 cen[kMode == 1 ? kBatch : 1];   // stochastic: jittered centre and hash z of the sample
};

// One 16x16 tile, the whole CTA (used by the per-frame kernel, one tile per
// CTA, and by the batch kernel, many frames' tiles per CTA in turn).
template <int kMode, int kTw = 16, int kTh = 16>  // kMode: 0 alpha, 1 stochastic, 2 two stochastic samples
__device__ __forceinline__ void raster_tile(const RasterParams& p, const uint32_t tile,
                                            RasterShared<kMode, kTw, kTh>& sh) {
    using Shape = TileShape<kTw, kTh>;
    using Mask = typename Shape::Mask;
    constexpr int kRs = Shape::kRowShift;
    static_assert(kMode == 0 || (kTw == 16 && kTh == 16), "the stochastic modes rasterize 16x16 tiles");
    const int tx = (int)(tile % (uint32_t)p.tiles_x), ty = (int)(tile / (uint32_t)p.tiles_x);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x0 = tx * kTw, y0 = ty * kTh;
    const int lx = (warp % Shape::kBx) * 8 + (lane & 7), ly0 = (warp / Shape::kBx) * 8 + (lane >> 3), ly1 = ly0 + 4;
    const int px = x0 + lx, py0 = y0 + ly0, py1 = y0 + ly1;
    const bool in0 = px < p.width && py0 < p.height, in1 = px < p.width && py1 < p.height;
    // coverage bits a pixel needs: its tile column and its tile row
    const Mask need0 = ((Mask)1 << lx) | ((Mask)1 << (kRs + ly0)), need1 = ((Mask)1 << lx) | ((Mask)1 << (kRs + ly1));
    const uint2 range = p.tile_ranges[tile];
    const uint32_t n = range.y > range.x ? range.y - range.x : 0u;
    const uint32_t* __restrict__ vals = p.tile_plan->vfinal;

    if (threadIdx.x == 0) {
        mbar_init(&sh.bar[0], 1);
        mbar_init(&sh.bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();

    const float fcx = (float)px + 0.5f, fcy0 = (float)py0 + 0.5f, fcy1 = (float)py1 + 0.5f;
    const float2 fcy = make_float2(fcy0, fcy1);
    // the stochastic modes' hash terms of the two pixels
    const PixelHash ph0 = pixel_hash(fcx, fcy0), ph1 = pixel_hash(fcx, fcy1);
    // alpha state of the two pixels (x: pixel 0, y: pixel 1); pixels outside
    // the image start "done" (T = 0) and are never written
    float2 T = make_float2(in0 ? 1.0f : 0.0f, in1 ? 1.0f : 0.0f);
    float2 C0 = f2(0.0f), C1 = f2(0.0f), C2 = f2(0.0f);
    StochState S0 = {16777215u, 0xFFFFFFFFu, 0.0f, 0.0f, 0.0f}, S1 = S0;
    bool sdone0 = !in0, sdone1 = !in1;
    Stoch2 P0, P1;
    if (kMode == 2) {
        stoch2_init(P0, in0);
        stoch2_init(P1, in1);
    }
    bool failed = false;
    const uint32_t nb = (n + kBatch - 1) / kBatch;
    uint32_t phase0 = 0, phase1 = 0;

    auto issue = [&](uint32_t b) {
        const uint32_t first = b * kBatch;
        const uint32_t cnt = min((uint32_t)kBatch, n - first);
        uint64_t* bar = &sh.bar[b & 1];
        if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, cnt * (uint32_t)sizeof(RasterRecord));
        for (uint32_t i = threadIdx.x; i < cnt; i += kRasterThreads) {
            const uint32_t s = min(vals[range.x + first + i], p.record_cap - 1u);
            bulk_g2s(&sh.rec[b & 1][i].r, p.records + s, (uint32_t)sizeof(RasterRecord), bar);
        }
    };
    auto pixels_done = [&]() -> bool {
        if (kMode == 0) return fmaxf(T.x, T.y) < kTransmittanceMin;
        if (kMode == 2) return P0.done[0] && P0.done[1] && P1.done[0] && P1.done[1];
        return sdone0 && sdone1;
    };

    if (nb > 0) issue(0);
    for (uint32_t b = 0; b < nb; ++b) {
        if (b + 1 < nb) issue(b + 1);
        const uint32_t ph = (b & 1) ? phase1 : phase0;
        if (!mbar_wait_bounded(&sh.bar[b & 1], ph)) failed = true;
        if (b & 1) phase1 ^= 1u; else phase0 ^= 1u;
        const uint32_t cnt = min((uint32_t)kBatch, n - b * kBatch);
        const StagedRecord* recs = sh.rec[b & 1];
        // Coverage bits of each staged record and which of the four 8x8 warp
        // blocks it can shade (one thread per record): blocks its rectangle
        // touches, minus those where the splat's ellipse q(d) <= s_max misses
        // every covered pixel centre (tested with a 2 % + 0.02 margin over
        // s_max, far above the rounding of q and of the exact per-pixel sum).
        for (uint32_t i = threadIdx.x; i < cnt; i += kRasterThreads) {
            const RasterRecord* R = &recs[i].r;
            if (p.colours) {
                // per-frame colours (gsanim state batches): the record's r, g, b replaced
                const uint32_t si = min(vals[range.x + b * kBatch + i], p.record_cap - 1u);
                const float4 col = __ldg(p.colours + si);
                RasterRecord* Rw = const_cast<RasterRecord*>(R);
                Rw->r = col.x;
                Rw->g = col.y;
                Rw->b = col.z;
                if (kMode != 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            const uint2 rr = reinterpret_cast<const uint2*>(R)[5];
            Mask bits;
            float cen_x, cen_y;
            if (kMode == 1) {
                // envelope record: this sample's quad (same computation as
                // the per-sample binning of the oracle) and jittered centre
                PixelRect q;
                const bool qok = quad_rect(R->cx, R->cy, R->log2_opacity, __uint_as_float(rr.y), __uint_as_float(rr.x),
                                           p.jitter_x, p.jitter_y, p.vp_w, p.vp_h, p.clip_y_sign, p.width, p.height,
                                           &q);
                bits = qok ? rect_bits<kTw, kTh>((uint32_t)q.i0 | ((uint32_t)q.i1 << 16),
                                                 (uint32_t)q.j0 | ((uint32_t)q.j1 << 16), x0, y0)
                           : (Mask)0;
                cen_x = add(R->cx, p.jitter_x);
                cen_y = add(R->cy, p.jitter_y);
                sh.cen[i] = make_float4(cen_x, cen_y, add((float)R->splat_id, p.frame_seed), 0.0f);
            } else {
                bits = rect_bits<kTw, kTh>(rr.x, rr.y, x0, y0);
                cen_x = R->cx;
                cen_y = R->cy;
            }
            sh.bits[i] = bits;
            if (kMode == 0) {
                // coverage bits next to g, b: one 16-byte load per splat in the loop
                const_cast<RasterRecord*>(R)->rect_x = (uint32_t)bits;
                if (kRs == 32) const_cast<RasterRecord*>(R)->rect_y = (uint32_t)((unsigned long long)bits >> 32);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            // block w = (w % kBx, w / kBx): bit w set iff its 8 columns and 8 rows are covered
            uint32_t blocks = 0u;
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const int bxw = w % Shape::kBx, byw = w / Shape::kBx;
                if (((bits >> (8 * bxw)) & 0xFFu) != 0u && ((bits >> (kRs + 8 * byw)) & 0xFFu) != 0u) blocks |= 1u << w;
            }
            const float4 q0 = reinterpret_cast<const float4*>(R)[0];
            const float2 q1 = reinterpret_cast<const float2*>(R)[2];
            const float A = q0.z, B = q0.w, C = q1.x;
            if (blocks && A > 0.0f && C > 0.0f) {
                const float thr = fmaf(R->s_max, 1.02f, 0.02f);
                for (uint32_t todo_w = blocks; todo_w; todo_w &= todo_w - 1u) {
                    const int w = __ffs(todo_w) - 1;
                    const int bxw = w % Shape::kBx, byw = w / Shape::kBx;
                    const uint32_t cb = (uint32_t)(bits >> (8 * bxw)) & 0xFFu;
                    const uint32_t rb = (uint32_t)(bits >> (kRs + 8 * byw)) & 0xFFu;
                    const float bx = (float)(x0 + 8 * bxw) + 0.5f - cen_x;
                    const float by = (float)(y0 + 8 * byw) + 0.5f - cen_y;
                    const float m = min_q_box(A, B, C, bx + (float)(__ffs(cb) - 1), bx + (float)(31 - __clz(cb)),
                                              by + (float)(__ffs(rb) - 1), by + (float)(31 - __clz(rb)));
                    if (m > thr) blocks &= ~(1u << w);
                }
            }
            sh.mask[i] = (uint8_t)blocks;
        }
        __syncthreads();
        // Warp-uniform control flow only; per-pixel work is predicated.
        bool warp_done = __any_sync(0xffffffffu, failed) || __all_sync(0xffffffffu, pixels_done());
        for (uint32_t c = 0; c < cnt && !warp_done; c += 32) {
            const bool mine = c + lane < cnt && ((sh.mask[c + lane] >> warp) & 1u);
            uint32_t todo = __ballot_sync(0xffffffffu, mine);
            if (kMode == 0) {
                // one splat of the warp's list into both pixels' state
                auto alpha_one = [&](uint32_t j) {
                    const float4 q0 = reinterpret_cast<const float4*>(&recs[j].r)[0];
                    const float4 q1 = reinterpret_cast<const float4*>(&recs[j].r)[1];
                    const uint4 q2u = reinterpret_cast<const uint4*>(&recs[j].r)[2];
                    Mask bits;
                    if (kRs == 32) bits = (Mask)((unsigned long long)q2u.z | ((unsigned long long)q2u.w << 32));
                    else bits = (Mask)q2u.z;
                    const float dx = sub(fcx, q0.x);
                    const float t0 = mul(mul(q0.z, dx), dx);
                    const float m = mul(q0.w, dx);
                    const float2 dy = __fadd2_rn(fcy, f2(-q0.y));
                    const float2 sq = __fadd2_rn(__fadd2_rn(f2(t0), __fmul2_rn(f2(m), dy)),
                                                 __fmul2_rn(__fmul2_rn(f2(q1.x), dy), dy));
                    const bool live0 = (bits & need0) == need0 && sq.x >= -__int_as_float(1) && sq.x <= q1.z;
                    const bool live1 = (bits & need1) == need1 && sq.y >= -__int_as_float(1) && sq.y <= q1.z;
                    const float2 q2 = make_float2(__uint_as_float(q2u.x), __uint_as_float(q2u.y));
                    const float2 arg = __ffma2_rn(sq, f2(kNegHalfLog2e), f2(q1.y));
                    const float a0 = live0 ? fminf(ex2_approx(arg.x), 0.99f) : 0.0f;
                    const float a1 = live1 ? fminf(ex2_approx(arg.y), 0.99f) : 0.0f;
                    const float2 w = __fmul2_rn(make_float2(a0, a1), T);
                    C0 = __ffma2_rn(w, f2(q1.w), C0);
                    C1 = __ffma2_rn(w, f2(q2.x), C1);
                    C2 = __ffma2_rn(w, f2(q2.y), C2);
                    T = __ffma2_rn(w, f2(-1.0f), T);
                };
                // two splats per trip: one loop test and one warp vote per pair
                while (todo) {
                    const uint32_t j = c + (uint32_t)(__ffs(todo) - 1);
                    todo &= todo - 1u;
                    alpha_one(j);
                    if (todo) {
                        const uint32_t j2 = c + (uint32_t)(__ffs(todo) - 1);
                        todo &= todo - 1u;
                        alpha_one(j2);
                    }
                    if (__all_sync(0xffffffffu, pixels_done())) { warp_done = true; break; }
                }
                continue;
            }
            while (todo) {
                const uint32_t j = c + (uint32_t)(__ffs(todo) - 1);
                todo &= todo - 1u;
                float4 q0 = reinterpret_cast<const float4*>(&recs[j].r)[0];
                const float4 q1 = reinterpret_cast<const float4*>(&recs[j].r)[1];
                const Mask bits = sh.bits[j];
                float hz = 0.0f;
                if (kMode == 1) {
                    const float4 cz = sh.cen[j];
                    q0.x = cz.x;
                    q0.y = cz.y;
                    hz = cz.z;
                }
                // splat_power()'s sum for both pixels with the shared first term
                const float dx = sub(fcx, q0.x);
                const float t0 = mul(mul(q0.z, dx), dx);
                const float m = mul(q0.w, dx);
                const float2 dy = __fadd2_rn(fcy, f2(-q0.y));
                const float2 sq = __fadd2_rn(__fadd2_rn(f2(t0), __fmul2_rn(f2(m), dy)),
                                             __fmul2_rn(__fmul2_rn(f2(q1.x), dy), dy));
                const bool live0 = (bits & need0) == need0 && sq.x >= -__int_as_float(1) && sq.x <= q1.z;
                const bool live1 = (bits & need1) == need1 && sq.y >= -__int_as_float(1) && sq.y <= q1.z;
                if (kMode == 0) {
                    const float2 q2 = reinterpret_cast<const float2*>(&recs[j].r)[4];
                    const float2 arg = __ffma2_rn(sq, f2(kNegHalfLog2e), f2(q1.y));
                    const float a0 = live0 ? fminf(ex2_approx(arg.x), 0.99f) : 0.0f;
                    const float a1 = live1 ? fminf(ex2_approx(arg.y), 0.99f) : 0.0f;
                    const float2 w = __fmul2_rn(make_float2(a0, a1), T);
                    C0 = __ffma2_rn(w, f2(q1.w), C0);
                    C1 = __ffma2_rn(w, f2(q2.x), C1);
                    C2 = __ffma2_rn(w, f2(q2.y), C2);
                    T = __ffma2_rn(w, f2(-1.0f), T);
                    if (__all_sync(0xffffffffu, pixels_done())) { warp_done = true; break; }
                } else if (kMode == 2) {
                    const uint4 q3 = reinterpret_cast<const uint4*>(&recs[j].r)[3];
                    const uint32_t z24 = q3.x, id = q3.y;
                    stoch2_retire(P0, z24, kDepthMargin);
                    stoch2_retire(P1, z24, kDepthMargin);
                    if (__all_sync(0xffffffffu, pixels_done())) { warp_done = true; break; }
                    const float2 q2 = reinterpret_cast<const float2*>(&recs[j].r)[4];
                    const float op = __uint_as_float(q3.w);
                    const float hz0 = hash_z(add((float)id, p.frame_seed)), hz1 = hash_z(add((float)id, p.frame_seed2));
                    stoch2_step(P0, live0, sq.x, op, ph0, hz0, hz1, z24, id, q1.w, q2.x, q2.y);
                    stoch2_step(P1, live1, sq.y, op, ph1, hz0, hz1, z24, id, q1.w, q2.x, q2.y);
                } else {
                    const uint4 q3 = reinterpret_cast<const uint4*>(&recs[j].r)[3];
                    const uint32_t z24 = q3.x, id = q3.y;
                    // a pixel stops once splats are beyond its kept depth (+ margin)
                    if (S0.best_id != 0xFFFFFFFFu && z24 > S0.best_d24 + kDepthMargin) sdone0 = true;
                    if (S1.best_id != 0xFFFFFFFFu && z24 > S1.best_d24 + kDepthMargin) sdone1 = true;
                    if (__all_sync(0xffffffffu, pixels_done())) { warp_done = true; break; }
                    const bool b0 = z24 < S0.best_d24 || (z24 == S0.best_d24 && id < S0.best_id);
                    const bool b1 = z24 < S1.best_d24 || (z24 == S1.best_d24 && id < S1.best_id);
                    const float2 q2 = reinterpret_cast<const float2*>(&recs[j].r)[4];
                    const float op = __uint_as_float(q3.w);
                    const float hzf = hash_z(hz);
                    if (live0 && !sdone0 && b0) stoch_step(S0, sq.x, op, ph0, hzf, z24, id, q1.w, q2.x, q2.y);
                    if (live1 && !sdone1 && b1) stoch_step(S1, sq.y, op, ph1, hzf, z24, id, q1.w, q2.x, q2.y);
                }
            }
        }
        const int all_done = __syncthreads_and(warp_done || pixels_done() || failed);
        if (all_done) {
            if (b + 1 < nb) {
                const uint32_t ph2 = ((b + 1) & 1) ? phase1 : phase0;
                if (!mbar_wait_bounded(&sh.bar[(b + 1) & 1], ph2)) failed = true;
            }
            break;
        }
    }
    if (failed) atomicOr(&p.fc->error_flags, kErrRasterWait);
    if (kMode == 0) {
        const size_t o0 = (size_t)(p.height - 1 - py0) * p.width + px;
        const size_t o1 = (size_t)(p.height - 1 - py1) * p.width + px;
        const float2 bg = f2(p.bg);
        const float2 r = __ffma2_rn(T, bg, C0), g = __ffma2_rn(T, bg, C1), bb = __ffma2_rn(T, bg, C2);
        if (in0) write_rgba16f(p.out_rgba16f, o0, r.x, g.x, bb.x, 1.0f - T.x);
        if (in1) write_rgba16f(p.out_rgba16f, o1, r.y, g.y, bb.y, 1.0f - T.y);
    } else if (kMode == 2) {
        if (in0) write_pixel_stoch2(p, px, py0, P0);
        if (in1) write_pixel_stoch2(p, px, py1, P1);
    } else {
        if (in0) write_pixel_stoch(p, px, py0, S0);
        if (in1) write_pixel_stoch(p, px, py1, S1);
    }
}

template <int kMode, int kTw = 16, int kTh = 16>
__global__ void __launch_bounds__(kRasterThreads) raster_kernel(RasterParams p) {
    pdl_wait();
    __shared__ RasterShared<kMode, kTw, kTh> sh;
    if (p.tile_count && blockIdx.x >= *p.tile_count) return;
    raster_tile<kMode, kTw, kTh>(p, p.tile_order[blockIdx.x], sh);
}

// Many frames in one persistent launch: work item w is tile
// frames[f].tile_order[w - first[f]] of the frame f with first[f] <= w <
// first[f + 1]; CTAs take items by ticket until all are done.  Every frame of
// a launch has the launch's tile shape.
template <int kMode, int kTw = 16, int kTh = 16>
__global__ void __launch_bounds__(kRasterThreads) raster_batch_kernel(const RasterParams* __restrict__ frames,
                                                                      const uint32_t* __restrict__ first,
                                                                      uint32_t nframes, uint32_t* __restrict__ ticket) {
    __shared__ RasterShared<kMode, kTw, kTh> sh;
    __shared__ uint32_t s_item;
    const uint32_t total = first[nframes];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t w = s_item;
        if (w >= total) break;
        uint32_t lo = 0, hi = nframes;   // last f with first[f] <= w
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (first[mid] <= w) lo = mid;
            else hi = mid;
        }
        const RasterParams p = frames[lo];
        raster_tile<kMode, kTw, kTh>(p, p.tile_order[w - first[lo]], sh);
        __syncthreads();
    }
}

void raster_batch_occupancy(int* blocks_per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, raster_batch_kernel<0, 16, 16>, kRasterThreads, 0);
}

int launch_raster_batch_alpha(const RasterParams* frames, const uint32_t* first, uint32_t nframes, uint32_t* ticket,
                              uint32_t grid, int tile_w, cudaStream_t s) {
    if (nframes == 0) return 0;
    if (tile_w == 32) raster_batch_kernel<0, 32, 8><<<grid, kRasterThreads, 0, s>>>(frames, first, nframes, ticket);
    else if (tile_w == 8) raster_batch_kernel<0, 8, 32><<<grid, kRasterThreads, 0, s>>>(frames, first, nframes, ticket);
    else raster_batch_kernel<0, 16, 16><<<grid, kRasterThreads, 0, s>>>(frames, first, nframes, ticket);
    return 1;
}

int launch_raster_alpha(const RasterParams& p, cudaStream_t s) {
    const uint32_t tiles = (uint32_t)p.tiles_x * (uint32_t)p.tiles_y;
    if (tiles == 0) return 0;
    if (p.tile_w == 32) raster_kernel<0, 32, 8><<<tiles, kRasterThreads, 0, s>>>(p);
    else if (p.tile_w == 8) raster_kernel<0, 8, 32><<<tiles, kRasterThreads, 0, s>>>(p);
    else launch_pdl(raster_kernel<0, 16, 16>, dim3(tiles), dim3(kRasterThreads), 0, s, p);
    return 1;
}

int launch_raster_stochastic2(const RasterParams& p, cudaStream_t s) {
    const uint32_t tiles = (uint32_t)p.tiles_x * (uint32_t)p.tiles_y;
    if (tiles == 0) return 0;
    launch_pdl(raster_kernel<2>, dim3(tiles), dim3(kRasterThreads), 0, s, p);
    return 1;
}

int launch_raster_stochastic(const RasterParams& p, cudaStream_t s) {
    const uint32_t tiles = (uint32_t)p.tiles_x * (uint32_t)p.tiles_y;
    if (tiles == 0) return 0;
    launch_pdl(raster_kernel<1>, dim3(tiles), dim3(kRasterThreads), 0, s, p);
    return 1;
}

}  // namespace gs
