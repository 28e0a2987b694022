// Shared device-side helpers for the gamesplat B200 splatting path.
//
// Arithmetic that must reproduce the reference shaders' results bit for bit is
// written with explicit round-to-nearest intrinsics (__fmul_rn, __fadd_rn, ...)
// so that the compiler never contracts it into FMAs; the operand order follows
// the GLSL source named at each use.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gs {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;

// Spin budget for every device-side wait (decoupled look-back, mbarriers).
// Far above any legitimate wait; after it the kernel records an error flag
// and carries on instead of hanging the GPU.
constexpr uint32_t kSpinLimit = 1u << 20;

// ---------------------------------------------------------------------------
// Exact single-rounding operations (never fused).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dv(float a, float b) { return __fdiv_rn(a, b); }

// GLSL built-ins with their specified definitions.
__device__ __forceinline__ float g_min(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float g_max(float x, float y) { return (x < y) ? y : x; }
__device__ __forceinline__ float g_clamp(float x, float lo, float hi) { return g_min(g_max(x, lo), hi); }
// mix(x, y, a) = x * (1 - a) + y * a
__device__ __forceinline__ float g_mix(float x, float y, float a) {
    return add(mul(x, sub(1.0f, a)), mul(y, a));
}
__device__ __forceinline__ float g_fract(float x) { return sub(x, floorf(x)); }
// float -> uint with saturation (cvt.rzi.u32.f32 semantics, NaN -> 0).
__device__ __forceinline__ uint32_t g_f2u_sat(float x) { return __float2uint_rz(x); }

// ---------------------------------------------------------------------------
// Deterministic transcendental functions, made only of correctly rounded
// +,-,*,/ and exact bit operations (same method and operation order as the
// CPU oracle):
//   log: x = m 2^e, m in [sqrt(1/2), sqrt(2)], ln m = 2 atanh((m-1)/(m+1)) by
//        the atanh Taylor series to s^9; ln 2 split into a 15-bit head and tail.
//   exp: Cody-Waite reduction by ln 2, Taylor series of e^r to degree 7.
//   sin/cos: reduction by pi/2 (17-bit head + tail), Taylor series to degree
//        9 / 10, quadrant selection.
// ---------------------------------------------------------------------------
constexpr float kLn2Hi = 0.693145751953125f;
constexpr float kLn2Lo = 1.428606765330187e-06f;
constexpr float kInvLn2 = 1.4426950216293335f;
constexpr float kLn2f = 0.6931471805599453f;
constexpr float kPio2Hi = 1.5707855224609375f;
constexpr float kPio2Lo = 1.0804334124259185e-05f;
constexpr float kTwoOverPi = 0.6366197466850281f;

__device__ __forceinline__ float det_logf(float x) {
    if (x != x) return x;
    if (x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (x == __int_as_float(0x7f800000)) return x;
    uint32_t ix = __float_as_uint(x);
    int e = 0;
    if (ix < 0x00800000u) { x = mul(x, 16777216.0f); ix = __float_as_uint(x); e = -24; }
    e += (int)(ix >> 23) - 127;
    float m = __uint_as_float((ix & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421354f) { m = mul(m, 0.5f); e += 1; }
    float f = sub(m, 1.0f);
    float s = dv(f, add(m, 1.0f));
    float z = mul(s, s);
    float p = mul(add(mul(add(mul(add(mul(z, 0.1111111119389534f), 0.1428571492433548f), z),
                              0.20000000298023224f), z), 0.3333333432674408f), z);
    float two_s = add(s, s);
    float lm = add(two_s, mul(two_s, p));
    float ef = (float)e;
    return add(mul(ef, kLn2Hi), add(lm, mul(ef, kLn2Lo)));
}

__device__ __forceinline__ float det_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283f) return __int_as_float(0x7f800000);
    if (x < -103.97208f) return 0.0f;
    float n = rintf(mul(x, kInvLn2));
    float r = sub(sub(x, mul(n, kLn2Hi)), mul(n, kLn2Lo));
    float p = 0.00019841270113829523f;
    p = add(0.0013888889225199819f, mul(r, p));
    p = add(0.008333333767950535f, mul(r, p));
    p = add(0.0416666679084301f, mul(r, p));
    p = add(0.1666666716337204f, mul(r, p));
    p = add(0.5f, mul(r, p));
    p = add(1.0f, mul(r, p));
    p = add(1.0f, mul(r, p));
    int k = (int)n;
    if (k > 127) { p = mul(p, 2.0f); k -= 1; }
    if (k < -126) { p = mul(p, 5.421010862427522e-20f); k += 64; }
    return mul(p, __uint_as_float((uint32_t)(k + 127) << 23));
}

__device__ __forceinline__ void det_sincosf(float x, float* s_out, float* c_out) {
    float n = rintf(mul(x, kTwoOverPi));
    float r = sub(sub(x, mul(n, kPio2Hi)), mul(n, kPio2Lo));
    float z = mul(r, r);
    float sp = add(-0.00019841270113829523f, mul(z, 2.7557318844628753e-06f));
    sp = add(0.008333333767950535f, mul(z, sp));
    sp = add(-0.1666666716337204f, mul(z, sp));
    float sr = add(r, mul(mul(r, z), sp));
    float cp = add(2.4801587642286904e-05f, mul(z, -2.755731998149713e-07f));
    cp = add(-0.0013888889225199819f, mul(z, cp));
    cp = add(0.0416666679084301f, mul(z, cp));
    cp = add(-0.5f, mul(z, cp));
    float cr = add(1.0f, mul(z, cp));
    int q = ((int)n) & 3;
    float s, c;
    if (q == 0) { s = sr; c = cr; }
    else if (q == 1) { s = cr; c = -sr; }
    else if (q == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
    *s_out = s;
    *c_out = c;
}

// shaders/cull.glsl:116-123
__device__ __forceinline__ float det_dilog(float x) {
    float s = sub(1.0f, x);
    float y = add(mul(-1.068681974f, x), 3.334685126f);
    y = sub(mul(y, x), 4.173996483f);
    y = add(mul(y, x), 2.567860600f);
    y = sub(mul(y, x), 0.884150470f);
    y = sub(mul(y, x), 0.123550674f);
    y = add(mul(y, x), 1.992765336f);
    y = add(mul(y, x), 6.74195669e-05f);
    y = add(y, (s > 0.0f) ? mul(s, det_logf(s)) : 0.0f);
    return y;
}

// shaders/gps.glsl:225-230
__device__ __forceinline__ float det_inv_dilog(float x) {
    float y = add(mul(-0.322192871f, x), 2.562830719f);
    y = sub(mul(y, x), 8.669815892f);
    y = add(mul(y, x), 16.243561492f);
    y = sub(mul(y, x), 18.394710417f);
    y = add(mul(y, x), 12.891925084f);
    y = sub(mul(y, x), 5.501796628f);
    y = add(mul(y, x), 1.361194673f);
    y = sub(mul(y, x), 0.417517201f);
    y = add(mul(y, x), 1.008071981f);
    y = sub(mul(y, x), 6.39879974e-05f);
    return y;
}

// log((1/255) / max(opacity, 1e-8)): the per-splat alpha cut-off of
// shaders/splat.glsl:70 (frag_alpha_power_cutoff).
__device__ __forceinline__ float alpha_cutoff(float opacity) {
    return det_logf(dv(1.0f / 255.0f, g_max(opacity, 1.0e-8f)));
}

// ---------------------------------------------------------------------------
// Quad coverage of one splat (shaders/splat.glsl:61-67): corners centre ±
// radius (+ jitter), NDC, viewport transform x_w = ndc * (w/2) + w/2, 8-bit
// sub-pixel snapping, pixel centres at k + 0.5, left/top edges inclusive
// (top = larger GL window y).  Returns false when clipped in z or empty.
// Rect is [i0,i1) x [j0,j1) in GL window coordinates (row 0 at the bottom).
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long floor_div256(long long a) { return a >> 8; }
__device__ __forceinline__ long long ceil_div256(long long a) { return -((-a) >> 8); }
__device__ __forceinline__ long long snap256(float w) {
    float s = mul(w, 256.0f);
    s = fminf(fmaxf(s, -1.0e15f), 1.0e15f);
    return __float2ll_rn(s);
}

struct PixelRect { int i0, i1, j0, j1; };

__device__ __forceinline__ bool quad_rect(float cx, float cy, float rx, float ry, float ndc_z, float jx,
                                          float jy, float vp_w, float vp_h, float clip_y_sign, int width,
                                          int height, PixelRect* r) {
    if (!(ndc_z >= -1.0f && ndc_z <= 1.0f)) return false;
    float hw = mul((float)width, 0.5f), hh = mul((float)height, 0.5f);
    float xa = add(add(cx, -rx), jx), xb = add(add(cx, rx), jx);
    float ya = add(add(cy, -ry), jy), yb = add(add(cy, ry), jy);
    float nxa = sub(dv(mul(2.0f, xa), vp_w), 1.0f), nxb = sub(dv(mul(2.0f, xb), vp_w), 1.0f);
    float nya = mul(sub(dv(mul(2.0f, ya), vp_h), 1.0f), clip_y_sign);
    float nyb = mul(sub(dv(mul(2.0f, yb), vp_h), 1.0f), clip_y_sign);
    long long Xa = snap256(add(mul(nxa, hw), hw)), Xb = snap256(add(mul(nxb, hw), hw));
    long long Ya = snap256(add(mul(nya, hh), hh)), Yb = snap256(add(mul(nyb, hh), hh));
    long long X0 = Xa < Xb ? Xa : Xb, X1 = Xa < Xb ? Xb : Xa;
    long long Y0 = Ya < Yb ? Ya : Yb, Y1 = Ya < Yb ? Yb : Ya;
    long long i0 = ceil_div256(X0 - 128), i1 = ceil_div256(X1 - 128);
    long long j0 = floor_div256(Y0 - 128) + 1, j1 = floor_div256(Y1 - 128) + 1;
    if (i0 < 0) i0 = 0;
    if (j0 < 0) j0 = 0;
    if (i1 > width) i1 = width;
    if (j1 > height) j1 = height;
    if (i1 <= i0 || j1 <= j0) return false;
    r->i0 = (int)i0; r->i1 = (int)i1; r->j0 = (int)j0; r->j1 = (int)j1;
    return true;
}

// shaders/splat.glsl:88-92: power = -0.5 (cx dx^2 + 2 cy dx dy + cz dy^2),
// evaluated in GLSL operand order; conic_2y holds 2*conic.y (exact).
__device__ __forceinline__ float splat_power(float dx, float dy, float conic_x, float conic_2y, float conic_z) {
    float t0 = mul(mul(conic_x, dx), dx);
    float t1 = mul(mul(conic_2y, dx), dy);
    float t2 = mul(mul(conic_z, dy), dy);
    return mul(-0.5f, add(add(t0, t1), t2));
}

// ---------------------------------------------------------------------------
// Decoupled look-back status words (64 bit): [63:32] epoch, [31:30] flag,
// [29:0] value.  A word counts only when its epoch matches the current
// launch's, so status arrays are zeroed once at allocation, never per frame.
// ---------------------------------------------------------------------------
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1u;
typedef unsigned long long u64;

// Programmatic dependent launch: a kernel launched with launch_pdl() may be
// scheduled while its predecessor in the stream still runs, and must wait
// here before touching anything the predecessor writes; a kernel triggers
// early scheduling of its dependent once all of its CTAs have called
// pdl_trigger() (or exited).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Status words carry their whole message (flag + value); the data a tile
// writes is read only by later kernels, so publishing needs no release
// ordering, and a relaxed GPU-scope store avoids a memory barrier per tile.
__device__ __forceinline__ void st_relaxed64(u64* p, u64 v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Look-backs only read the status words themselves (no data published with
// them), so relaxed GPU-scope loads of the atomically written 64-bit words
// suffice and several can be in flight at once.
__device__ __forceinline__ u64 ld_relaxed64(const u64* p) {
    u64 v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ u64 status_word(uint32_t epoch, uint32_t flag, uint32_t value) {
    return ((u64)epoch << 32) | (u64)(flag | (value & kValMask));
}

// Single-thread look-back that reads W predecessor words per step
// (independent loads), then consumes them nearest first until an inclusive
// prefix; an unpublished word is re-polled (bounded) before continuing.
// Sets *timed_out if a wait exceeded kSpinLimit (the result is then
// incomplete but the kernel ends).
template <int W>
__device__ __forceinline__ uint32_t lookback_vec(const u64* status, size_t stride, uint32_t tile, uint32_t epoch,
                                                 bool* timed_out) {
    uint32_t excl = 0;
    long long j = (long long)tile - 1;
    uint32_t spins = 0;
    while (j >= 0) {
        u64 w[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            w[k] = (j - k >= 0) ? ld_relaxed64(status + (size_t)(j - k) * stride) : status_word(epoch, kFlagInc, 0);
        int k = 0;
        bool found = false;
#pragma unroll
        for (int q = 0; q < W; ++q) {
            if (k != q || found) continue;
            const uint32_t lo = (uint32_t)w[q];
            const uint32_t flag = lo & ~kValMask;
            if ((uint32_t)(w[q] >> 32) != epoch || flag == 0u) continue;  // not published yet
            excl += lo & kValMask;
            ++k;
            if (flag == kFlagInc) found = true;
        }
        if (found) return excl;
        j -= k;
        if (k < W) {  // word j is not published yet: wait for it
            if (++spins > kSpinLimit) { *timed_out = true; return excl; }
            if (spins > 64) __nanosleep(32);
        }
    }
    return excl;
}

// Warp-cooperative look-back: all 32 lanes read a window of 32 predecessors
// at once, the nearest inclusive word is found by ballot and the aggregates
// after it are summed with a warp reduction.  Every lane returns the same
// exclusive prefix, and every lane sees *timed_out if any lane's wait ran
// out.  Bounded like lookback_vec().
__device__ __forceinline__ uint32_t lookback_warp(const u64* status, uint32_t tile, uint32_t epoch,
                                                  bool* timed_out, uint32_t spin_limit = kSpinLimit) {
    const int lane = threadIdx.x & 31;
    uint32_t excl = 0;
    long long end = (long long)tile;  // window = [end - 32, end)
    uint32_t spins = 0;
    bool ran_out = false;   // this lane's wait gave up (made warp-uniform at the end)
    while (end > 0) {
        const long long j = end - 32 + lane;
        uint32_t flag = kFlagInc, val = 0;   // before tile 0: an inclusive zero
        if (j >= 0) {
            for (;;) {
                const u64 w = ld_relaxed64(status + j);
                flag = (uint32_t)w & ~kValMask;
                val = (uint32_t)w & kValMask;
                if ((uint32_t)(w >> 32) == epoch && flag != 0u) break;
                if (++spins > spin_limit) { ran_out = true; flag = kFlagInc; val = 0; break; }
                if (spins > 64) __nanosleep(32);
            }
        }
        const uint32_t inc = __ballot_sync(0xffffffffu, flag == kFlagInc);
        if (inc) {
            const int h = 31 - __clz(inc);   // nearest inclusive in the window
            excl += __reduce_add_sync(0xffffffffu, lane >= h ? val : 0u);
            break;
        }
        excl += __reduce_add_sync(0xffffffffu, val);
        end -= 32;
    }
    if (__any_sync(0xffffffffu, ran_out)) *timed_out = true;
    return excl;
}

// Block-wide exclusive scan of one uint32 per thread (blockDim.x <= 1024,
// multiple of 32).  `warp_tmp` holds >= 33 words of shared memory.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tmp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nwarps ? warp_tmp[lane] : 0u;
        uint32_t ws = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        if (lane < nwarps) warp_tmp[lane] = ws - w;
        if (lane == nwarps - 1) warp_tmp[32] = ws;
    }
    __syncthreads();
    uint32_t r = warp_tmp[warp] + x - v;
    *total = warp_tmp[32];
    __syncthreads();
    return r;
}

// Block-wide exclusive prefix maximum of signed values (identity -1);
// warp_tmp holds 33 words.  Every thread of the block must call it.
__device__ __forceinline__ int32_t block_excl_max(int32_t v, int32_t* warp_tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    if (lane == 31) warp_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int32_t w = lane < nwarps ? warp_tmp[lane] : -1;
        int32_t ws = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws = max(ws, y);
        }
        // exclusive over warps: shift by one
        const int32_t prev = __shfl_up_sync(0xffffffffu, ws, 1);
        if (lane < nwarps) warp_tmp[lane] = lane == 0 ? -1 : prev;
    }
    __syncthreads();
    const int32_t xin = __shfl_up_sync(0xffffffffu, x, 1);
    const int32_t r = max(warp_tmp[warp], lane == 0 ? -1 : xin);
    __syncthreads();
    return r;
}

}  // namespace gs
