// Cull / project / SH kernels: shaders/cull.glsl:166-424 (+ cull_reset,
// :456-473, folded in) for the B200.
//
// Memory plan (HBM-bound, 256-byte GpuGaussian rows), two kernels:
//   * cull_visible_kernel reads the first 16 bytes (position, opacity) of
//     every row from the heads array (a contiguous copy of them written once
//     per upload by gather_heads_kernel: reading them out of the rows would
//     fetch at least one 32-byte sector, in practice 128 bytes, per 16 bytes
//     used), runs the near/frustum test, computes the depth keys and
//     compacts the visible (key, id) pairs in index order with a decoupled
//     look-back over 2048-row CTA tiles, so the depth sort runs on N_vis
//     pairs instead of N (the culled tail of the reference's all-N sort is
//     all-equal (0xFFFFFFFF, 0xFFFFFFFF) pairs, so the result is identical);
//   * cull_project_kernel walks the compacted ids in groups of 32 and stages
//     each visible row whole into a padded shared-memory row (272-byte
//     stride: conflict-free 128-bit shared loads) with one TMA bulk copy,
//     then projects it; culled rows cost one 32-byte sector, visible rows
//     256 bytes (fewer for sh_degree < 3).
// Arithmetic follows the GLSL operand order with unfused intrinsics so the
// keys, cull mask and projected records match the CPU oracle bit for bit.

#include <cuda_fp16.h>

#include <atomic>

#include "gs_common.cuh"
#include "gs_internal.h"
#include "gs_tma.cuh"

namespace gs {

constexpr int kStageStride = 17;  // float4 per staged row (16 + 1 pad)
constexpr int kHalfStageStride = 9;   // float4 per staged 144-byte FP16-SH row
constexpr int kCullWarps = kCullThreads / 32;
constexpr size_t kCullSmem = (size_t)kCullWarps * 32 * kStageStride * sizeof(float4);  // one stage per warp
constexpr size_t kCullHalfSmem = (size_t)kCullWarps * 32 * kHalfStageStride * sizeof(float4);

struct CamRegs {
    float V[16];
    float P0, P5, P10, P14;
    float vpx, vpy, ortho, fxp, fxo, ysign, z01;
    float camw[3];
};

__device__ __forceinline__ void load_cam(const gs_camera& c, CamRegs& r) {
#pragma unroll
    for (int k = 0; k < 16; ++k) r.V[k] = c.view[k];
    r.P0 = c.proj[0];
    r.P5 = c.proj[5];
    r.P10 = c.proj[10];
    r.P14 = c.proj[14];
    r.vpx = c.viewport[0];
    r.vpy = c.viewport[1];
    r.ortho = c.orthographic;
    r.fxp = c.persp_focal;
    r.fxo = c.ortho_focal;
    r.ysign = c.clip_y_sign;
    r.z01 = c.clip_z_01;
    // cam_pos_world = -transpose(W) * view[3].xyz (shaders/cull.glsl:323)
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) {
        float t = add(add(mul(r.V[rr * 4 + 0], r.V[12]), mul(r.V[rr * 4 + 1], r.V[13])), mul(r.V[rr * 4 + 2], r.V[14]));
        r.camw[rr] = -t;
    }
}

#define SH_C0 0.28209479177387814f
#define SH_C1 0.4886025119029199f
#define SH_C2_0 1.0925484305920792f
#define SH_C2_1 (-1.0925484305920792f)
#define SH_C2_2 0.31539156525252005f
#define SH_C2_3 (-1.0925484305920792f)
#define SH_C2_4 0.5462742152960396f
#define SH_C3_0 (-0.5900435899266435f)
#define SH_C3_1 2.890611442640554f
#define SH_C3_2 (-0.4570457994644658f)
#define SH_C3_3 0.3731763325901154f
#define SH_C3_4 (-0.4570457994644658f)
#define SH_C3_5 1.445305721320277f
#define SH_C3_6 (-0.5900435899266435f)

__device__ __forceinline__ void sh_acc(float* res, float w, float a, float b, float c) {
    res[0] = add(res[0], mul(w, a));
    res[1] = add(res[1], mul(w, b));
    res[2] = add(res[2], mul(w, c));
}

// Full projection of one visible Gaussian (shaders/cull.glsl:234-423).
// row: staged chunks 1..15 of the row in shared memory; c0 = chunk 0.
// SH colour before the bias (shaders/cull.glsl:355-408): DC at row[3].xyz,
// SH(k) = floats 16 + 3k .. 18 + 3k (chunks 4..15).
__device__ __forceinline__ void sh_eval(const float4* row, float x, float y, float z, int eff, float* res) {
    const float4 c3 = row[3];
    res[0] = mul(SH_C0, c3.x);
    res[1] = mul(SH_C0, c3.y);
    res[2] = mul(SH_C0, c3.z);
    if (eff >= 1) {
        float4 q4 = row[4], q5 = row[5], q6 = row[6];
        sh_acc(res, mul(-SH_C1, y), q4.x, q4.y, q4.z);
        sh_acc(res, mul(SH_C1, z), q4.w, q5.x, q5.y);
        sh_acc(res, mul(-SH_C1, x), q5.z, q5.w, q6.x);
        if (eff >= 2) {
            float4 q7 = row[7], q8 = row[8], q9 = row[9];
            float xx = mul(x, x), yy = mul(y, y), zz = mul(z, z);
            float xy = mul(x, y), yz = mul(y, z), xz = mul(z, x);
            sh_acc(res, mul(SH_C2_0, xy), q6.y, q6.z, q6.w);
            sh_acc(res, mul(SH_C2_1, yz), q7.x, q7.y, q7.z);
            sh_acc(res, mul(SH_C2_2, sub(sub(mul(2.0f, zz), xx), yy)), q7.w, q8.x, q8.y);
            sh_acc(res, mul(SH_C2_3, xz), q8.z, q8.w, q9.x);
            sh_acc(res, mul(SH_C2_4, sub(xx, yy)), q9.y, q9.z, q9.w);
            if (eff >= 3) {
                float4 qa = row[10], qb = row[11], qc = row[12], qd = row[13], qe = row[14], qf = row[15];
                sh_acc(res, mul(mul(SH_C3_0, y), sub(mul(3.0f, xx), yy)), qa.x, qa.y, qa.z);
                sh_acc(res, mul(mul(SH_C3_1, xy), z), qa.w, qb.x, qb.y);
                sh_acc(res, mul(mul(SH_C3_2, y), sub(sub(mul(4.0f, zz), xx), yy)), qb.z, qb.w, qc.x);
                sh_acc(res, mul(mul(SH_C3_3, z), sub(sub(mul(2.0f, zz), mul(3.0f, xx)), mul(3.0f, yy))), qc.y, qc.z, qc.w);
                sh_acc(res, mul(mul(SH_C3_4, x), sub(sub(mul(4.0f, zz), xx), yy)), qd.x, qd.y, qd.z);
                sh_acc(res, mul(mul(SH_C3_5, z), sub(xx, yy)), qd.w, qe.x, qe.y);
                sh_acc(res, mul(mul(SH_C3_6, x), sub(xx, mul(3.0f, yy))), qe.z, qe.w, qf.x);
            }
        }
    }
}

// kGivenColour: the SH colour before the bias comes in sh_colour (FP16-SH rows)
template <bool kGivenColour = false>
__device__ __forceinline__ void project_visible(const float4* row, float4 c0, float vx, float vy, float vz,
                                                const CamRegs& cam, int sh_degree, float sh_lod, float4* out,
                                                float* quad_area, float* gps_points, float sc0 = 0.0f,
                                                float sc1 = 0.0f, float sc2 = 0.0f) {
    const float t = cam.ortho;
    float4 c1 = row[1], c2 = row[2];
    float sx = c1.x, sy = c1.y, sz = c1.z;
    float qw = c2.x, qx = c2.y, qy = c2.z, qz = c2.w;

    float R[3][3];
    R[0][0] = sub(1.0f, mul(2.0f, add(mul(qy, qy), mul(qz, qz))));
    R[0][1] = mul(2.0f, add(mul(qx, qy), mul(qw, qz)));
    R[0][2] = mul(2.0f, sub(mul(qx, qz), mul(qw, qy)));
    R[1][0] = mul(2.0f, sub(mul(qx, qy), mul(qw, qz)));
    R[1][1] = sub(1.0f, mul(2.0f, add(mul(qx, qx), mul(qz, qz))));
    R[1][2] = mul(2.0f, add(mul(qy, qz), mul(qw, qx)));
    R[2][0] = mul(2.0f, add(mul(qx, qz), mul(qw, qy)));
    R[2][1] = mul(2.0f, sub(mul(qy, qz), mul(qw, qx)));
    R[2][2] = sub(1.0f, mul(2.0f, add(mul(qx, qx), mul(qy, qy))));
    const float s3[3] = {sx, sy, sz};
    float M[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) M[c][r] = mul(R[c][r], s3[c]);
    float cov[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r)
            cov[c][r] = add(add(mul(M[0][r], M[0][c]), mul(M[1][r], M[1][c])), mul(M[2][r], M[2][c]));

    const float fxp = cam.fxp, fxo = cam.fxo;
    float J00 = g_mix(dv(fxp, vz), -fxo, t);
    float J11 = g_mix(dv(fxp, vz), -fxo, t);
    float vz2 = mul(vz, vz);
    float J02 = g_mix(dv(mul(-fxp, vx), vz2), 0.0f, t);
    float J12 = g_mix(dv(mul(-fxp, vy), vz2), 0.0f, t);

    float W[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) W[c][r] = cam.V[c * 4 + r];
    float A[3][3], B[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r)
            A[c][r] = add(add(mul(W[0][r], cov[c][0]), mul(W[1][r], cov[c][1])), mul(W[2][r], cov[c][2]));
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r)
            B[c][r] = add(add(mul(A[0][r], W[0][c]), mul(A[1][r], W[1][c])), mul(A[2][r], W[2][c]));

    float a = add(add(mul(mul(J00, J00), B[0][0]), mul(mul(mul(2.0f, J00), J02), B[0][2])), mul(mul(J02, J02), B[2][2]));
    float b = add(add(add(mul(mul(J00, J11), B[0][1]), mul(mul(J00, J12), B[0][2])), mul(mul(J02, J11), B[1][2])),
                  mul(mul(J02, J12), B[2][2]));
    float c = add(add(mul(mul(J11, J11), B[1][1]), mul(mul(mul(2.0f, J11), J12), B[1][2])), mul(mul(J12, J12), B[2][2]));
    a = add(a, 0.3f);
    c = add(c, 0.3f);
    float det = sub(mul(a, c), mul(b, b));
    if (det < 1e-6f) det = 1e-6f;
    float conic_x = dv(c, det), conic_y = dv(-b, det), conic_z = dv(a, det);

    float pcx = add(dv(mul(fxp, vx), vz), mul(cam.vpx, 0.5f));
    float pcy = add(mul(cam.vpy, 0.5f), dv(mul(fxp, vy), vz));
    float ocx = add(mul(-fxo, vx), mul(cam.vpx, 0.5f));
    float ocy = sub(mul(cam.vpy, 0.5f), mul(fxo, vy));
    float cx = g_mix(pcx, ocx, t), cy = g_mix(pcy, ocy, t);
    float y_flip = mul(sub(1.0f, cam.ysign), 0.5f);
    float rcy = g_mix(cy, sub(cam.vpy, cy), y_flip);
    float rconic_y = mul(conic_y, cam.ysign);
    float radius_x = ceilf(mul(3.0f, __fsqrt_rn(a)));
    float radius_y = ceilf(mul(3.0f, __fsqrt_rn(c)));
    *quad_area = mul(mul(4.0f, radius_x), radius_y);
    *gps_points = mul(mul(6.28318530718f, __fsqrt_rn(g_max(det, 0.0f))), det_dilog(g_clamp(c0.w, 0.0f, 1.0f)));

    float ndc_z = dv(add(mul(cam.P10, vz), cam.P14), -vz);
    ndc_z = g_mix(ndc_z, add(mul(ndc_z, 0.5f), 0.5f), cam.z01);

    float ddx = sub(c0.x, cam.camw[0]), ddy = sub(c0.y, cam.camw[1]), ddz = sub(c0.z, cam.camw[2]);
    float len = __fsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
    float x = dv(ddx, len), y = dv(ddy, len), z = dv(ddz, len);

    int eff = sh_degree;
    if (sh_lod > 0.0f && (-vz) > sh_lod) eff = 0;
    float res[3];
    if (kGivenColour) {
        res[0] = sc0;
        res[1] = sc1;
        res[2] = sc2;
    } else {
        sh_eval(row, x, y, z, eff, res);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) res[k] = g_max(add(res[k], 0.5f), 0.0f);

    out[0] = make_float4(res[0], res[1], res[2], c0.w);
    out[1] = make_float4(cx, rcy, radius_x, radius_y);
    out[2] = make_float4(conic_x, rconic_y, conic_z, ndc_z);
    out[3] = make_float4(a, mul(b, cam.ysign), c, det);
}

// Stage one group of 32 compacted visible rows: lane l copies the first
// kChunks 16-byte chunks of row ids[first + l] (if first + l < count) to
// stage row l with one TMA bulk copy; completion is counted on `bar`.
// Returns the lane's row id, or kSentinel past the end.
template <int kChunks, int kRowChunks = 16, int kStride = kStageStride>
__device__ __forceinline__ uint32_t stage_group(const float4* rows, const uint32_t* ids, uint32_t first,
                                                uint32_t count, float4* stage, uint64_t* bar, int lane,
                                                uint64_t policy) {
    const uint32_t idx = first + (uint32_t)lane;
    const uint32_t id = idx < count ? ids[idx] : kSentinel;
    const uint32_t mask = __ballot_sync(0xffffffffu, id != kSentinel);
    if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)__popc(mask) * (uint32_t)(kChunks * 16));
    __syncwarp();
    // order this lane's earlier generic accesses to its stage row (reads, and
    // the in-place gsanim deltas) before the async-proxy refill
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (id != kSentinel)
        bulk_g2s_hint(stage + lane * kStride, rows + (size_t)id * kRowChunks, (uint32_t)(kChunks * 16), bar, policy);
    return id;
}

// gsanim int8 appearance deltas applied in place to a staged row
// (shaders/cull.glsl:125-164): DC slots 12..14 are j = 0..2, the SH slot
// 16 + 3k + c is j = 3 + 15c + k; state s >= 1 adds q * scale[j] with q the
// int8 at ((s-1) * n + row) * 48 + j; two states blend with the weight.
__device__ __forceinline__ float anim_coeff(const CullParams& p, float base, uint32_t row, int j, int state) {
    if (state == 0) return base;
    const size_t off = ((size_t)(state - 1) * p.n + row) * 48u + (size_t)j;
    return add(base, mul((float)p.anim_deltas[off], __ldg(p.anim_scales + j)));
}

__device__ void animate_row(const CullParams& p, uint32_t row, float4* staged, float4& c3) {
    float* f = reinterpret_cast<float*>(staged);
    float dc[3] = {c3.x, c3.y, c3.z};
    for (int slot = 12; slot < 61; ++slot) {
        if (slot == 15) continue;
        const int j = slot < 15 ? slot - 12 : 3 + ((slot - 16) % 3) * 15 + (slot - 16) / 3;
        const float base = slot < 15 ? dc[slot - 12] : f[slot];
        float v = anim_coeff(p, base, row, j, p.anim_state_a);
        if (p.anim_weight > 0.0f) {
            const float bb = anim_coeff(p, base, row, j, p.anim_state_b);
            v = add(mul(sub(1.0f, p.anim_weight), v), mul(p.anim_weight, bb));
        }
        if (slot < 15) dc[slot - 12] = v;
        else f[slot] = v;
    }
    c3 = make_float4(dc[0], dc[1], dc[2], c3.w);
    staged[3] = c3;
}

// Copies the first 16 bytes of every row into the contiguous heads array
// (run once per upload; the rows are written nowhere else).
__global__ void gather_heads_kernel(const float4* __restrict__ rows, float4* __restrict__ heads, uint32_t n,
                                    uint32_t stride) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        heads[i] = __ldg(rows + (size_t)i * stride);
}

int launch_gather_heads(const float4* rows, float4* heads, uint32_t n, uint32_t num_sms, cudaStream_t s,
                        uint32_t row_chunks) {
    if (n == 0) return 0;
    uint32_t grid = (n + 255) / 256;
    if (grid > num_sms * 8) grid = num_sms * 8;
    gather_heads_kernel<<<grid, 256, 0, s>>>(rows, heads, n, row_chunks);
    return 1;
}

// 256-byte GpuGaussian rows -> 144-byte rows with FP16 SH: chunks 0..2
// (position, opacity, scale, rotation) copied, then the 48 SH coefficients
// (DC at floats 12..14, SH k = 1..15 at 16 + 3(k-1) + c) as IEEE half, one
// channel after the other: half 16c + k (k = 0 the DC term), so that the
// coefficients k, k + 1 of a channel are one 32-bit word (round to nearest even).
__global__ void pack_half_rows_kernel(const float4* __restrict__ rows, float4* __restrict__ half_rows,
                                      uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = reinterpret_cast<const float*>(rows + (size_t)i * 16);
        float4* o = half_rows + (size_t)i * kHalfRowChunks;
        o[0] = __ldg(rows + (size_t)i * 16);
        o[1] = __ldg(rows + (size_t)i * 16 + 1);
        o[2] = __ldg(rows + (size_t)i * 16 + 2);
        __align__(16) __half h[48];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            h[16 * c] = __float2half_rn(r[12 + c]);
#pragma unroll
            for (int k = 1; k < 16; ++k) h[16 * c + k] = __float2half_rn(r[16 + 3 * (k - 1) + c]);
        }
        const float4* hv = reinterpret_cast<const float4*>(h);
#pragma unroll
        for (int q = 0; q < 6; ++q) o[3 + q] = hv[q];
    }
}

int launch_pack_half_rows(const float4* rows, float4* half_rows, uint32_t n, uint32_t num_sms, cudaStream_t s) {
    if (n == 0) return 0;
    uint32_t grid = (n + 255) / 256;
    if (grid > num_sms * 8) grid = num_sms * 8;
    pack_half_rows_kernel<<<grid, 256, 0, s>>>(rows, half_rows, n);
    return 1;
}

// Pass 1 (visibility and compaction): each CTA takes one 2048-row tile by
// ticket (tickets follow CTA start order, so every tile a look-back waits on
// belongs to a CTA that is already running), loads 8 heads per thread
// (coalesced, all in flight at once), tests visibility
// (shaders/cull.glsl:209-220), computes the depth keys (:230-232) and places
// the tile's visible (key, id) pairs in index order: a block scan of the
// per-(row group, warp) counts, then one warp-level decoupled look-back per
// tile.  The 4 x 256 key-digit histograms of the depth sort are accumulated in
// shared memory; the top digit (sign and high exponent bits, a handful of
// values in a scene) is aggregated per warp first, since 32 lanes adding to
// one shared word would serialize.
__global__ void __launch_bounds__(kCullVisThreads) cull_visible_kernel(CullParams p) {
    pdl_wait();
    constexpr int kWarps = kCullVisThreads / 32;
    static_assert(kCullVisItems * kWarps == 64, "the count scan gives each lane two (row group, warp) counts");
    __shared__ uint32_t s_hist[4][256];
    __shared__ uint32_t s_cnt[kCullVisItems * kWarps];   // (row group, warp) order = index order
    __shared__ uint32_t s_tile, s_excl;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (int i = t; i < 4 * 256; i += kCullVisThreads) (&s_hist[0][0])[i] = 0u;
    if (t == 0) s_tile = atomicAdd(&p.fc->cull_ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t num_tiles = (p.n + kCullVisTile - 1) / kCullVisTile;
    if (tile >= num_tiles) return;   // uniform over the CTA
    const uint32_t base = tile * kCullVisTile;
    const float* V = p.cam.view;
    const float P0 = p.cam.proj[0], P5 = p.cam.proj[5], ortho = p.cam.orthographic;
    float4 c0[kCullVisItems];
#pragma unroll
    for (int k = 0; k < kCullVisItems; ++k) {
        const uint32_t g = base + k * kCullVisThreads + t;
        c0[k] = g < p.n ? __ldg(p.heads + g) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    uint32_t mask[kCullVisItems], key[kCullVisItems];
#pragma unroll
    for (int k = 0; k < kCullVisItems; ++k) {
        const uint32_t g = base + k * kCullVisThreads + t;
        // p_view = view * vec4(position, 1.0)
        const float vx = add(add(add(mul(V[0], c0[k].x), mul(V[4], c0[k].y)), mul(V[8], c0[k].z)), V[12]);
        const float vy = add(add(add(mul(V[1], c0[k].x), mul(V[5], c0[k].y)), mul(V[9], c0[k].z)), V[13]);
        const float vz = add(add(add(mul(V[2], c0[k].x), mul(V[6], c0[k].y)), mul(V[10], c0[k].z)), V[14]);
        bool visible = g < p.n && (vz <= -0.2f);
        if (visible) {
            float inv_z = dv(-1.0f, vz);
            float ndc_x = add(mul(mul(mul(P0, vx), inv_z), sub(1.0f, ortho)), mul(mul(P0, vx), ortho));
            float ndc_y = add(mul(mul(mul(P5, vy), inv_z), sub(1.0f, ortho)), mul(mul(P5, vy), ortho));
            visible = fabsf(ndc_x) <= 1.3f && fabsf(ndc_y) <= 1.3f;
        }
        key[k] = 0xFFFFFFFFu - __float_as_uint(g_max(-vz, 0.0f));
        mask[k] = __ballot_sync(0xffffffffu, visible);
        if (lane == 0) s_cnt[k * kWarps + warp] = (uint32_t)__popc(mask[k]);
        if (!visible && g < p.n && p.write_invisible) {   // shaders/cull.glsl:222-228
            float4* dst = p.projected + (size_t)g * 4;
            dst[0] = make_float4(0.f, 0.f, 0.f, 0.f);
            dst[1] = make_float4(0.f, 0.f, 0.f, 0.f);
            dst[2] = make_float4(1.f, 0.f, 1.f, 1.f);
            dst[3] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    __syncthreads();
    if (warp == 0) {
        // exclusive scan of the 64 counts in index order, two per lane
        const uint32_t a = s_cnt[2 * lane], b = s_cnt[2 * lane + 1];
        uint32_t incl = a + b;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        s_cnt[2 * lane] = incl - a - b;
        s_cnt[2 * lane + 1] = incl - b;
        if (lane == 0)
            st_relaxed64(p.status + tile, status_word(p.epoch, tile == 0 ? kFlagInc : kFlagAgg, total));
        uint32_t excl = 0;
        if (tile > 0) {
            bool to = false;
            excl = lookback_warp(p.status, tile, p.epoch, &to);
            if (lane == 0) {
                if (to) atomicOr(&p.fc->error_flags, kErrCullLookback);
                st_relaxed64(p.status + tile, status_word(p.epoch, kFlagInc, excl + total));
            }
        }
        if (lane == 0) {
            s_excl = excl;
            if (tile == num_tiles - 1) p.fc->visible_count = excl + total;
        }
    }
    __syncthreads();
    const uint32_t excl = s_excl;
#pragma unroll
    for (int k = 0; k < kCullVisItems; ++k) {
        const bool v = (mask[k] >> lane) & 1u;
        const uint32_t kk = key[k];
        if (v) {
            const uint32_t o = excl + s_cnt[k * kWarps + warp] + (uint32_t)__popc(mask[k] & lt);
            p.keys_out[o] = kk;
            p.ids_out[o] = base + k * kCullVisThreads + t;
            atomicAdd(&s_hist[0][kk & 255u], 1u);
            atomicAdd(&s_hist[1][(kk >> 8) & 255u], 1u);
            atomicAdd(&s_hist[2][(kk >> 16) & 255u], 1u);
        }
        // invisible lanes match among themselves (256 is no digit) and add nothing
        const uint32_t d3 = v ? (kk >> 24) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d3);
        if (v && lane == __ffs(peers) - 1) atomicAdd(&s_hist[3][d3], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int i = t; i < 4 * 256; i += kCullVisThreads) {
        const uint32_t c = (&s_hist[0][0])[i];
        if (c) atomicAdd(p.key_hist + i, c);
    }
}

// Pass 2 (projection): warps take groups of 32 compacted visible rows
// (statically: group = warp + k * warps), stage a group's rows into their
// shared-memory rows (TMA bulk copies), project them and write the projected
// records (shaders/cull.glsl:234-423).  Every lane holds a visible row, so no
// projection issue slot is spent on culled rows.  One stage per warp lets 6
// CTAs (24 warps) share an SM; the other warps' math hides a warp's staging
// wait (measured faster than two stages per warp at 3 CTAs per SM).
template <int kChunks>  // 16-byte chunks of a row the SH degree needs: 4, 7, 10 or 16
__global__ void __launch_bounds__(kCullThreads, 6) cull_project_kernel(CullParams p) {
    pdl_wait();
    extern __shared__ float4 smem4[];
    __shared__ __align__(8) uint64_t s_bar[kCullWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        mbar_init(&s_bar[warp], 1);
        mbar_fence_init();
    }
    __syncthreads();
    float4* const stage0 = smem4 + (size_t)warp * 32 * kStageStride;
    const uint32_t n_vis = p.fc->visible_count;
    const uint32_t groups = (n_vis + 31) / 32;
    const uint32_t wg = blockIdx.x * kCullWarps + warp, nw = gridDim.x * kCullWarps;
    CamRegs cam;
    load_cam(p.cam, cam);
    // the shader blends whenever the weight is positive, states 0 and 0
    // included (gsanim_sample returns {0, 0, w} between two linear keys of
    // the base state), and (1 - w) x + w x need not round to x
    const bool animated = p.anim_deltas != nullptr && (p.anim_state_a != 0 || p.anim_weight > 0.0f);
    const uint64_t stream_policy = l2_policy_evict_first();
    bool stage_failed = false;
    uint32_t phase = 0;   // parity of the next completion of the warp's barrier
    uint32_t d0 = 0, d2 = 0, d3 = 0, d4 = 0, d6 = 0, d7 = 0, m1 = 0, m5 = 0;
    for (uint32_t g = wg; g < groups; g += nw) {
        const uint32_t id = stage_group<kChunks>(p.rows, p.ids_out, g * 32u, n_vis, stage0, &s_bar[warp], lane,
                                                 stream_policy);
        if (!mbar_wait_bounded(&s_bar[warp], phase)) stage_failed = true;
        phase ^= 1u;
        if (id != kSentinel) {
            float4* row = stage0 + lane * kStageStride;
            const float4 c0 = row[0];
            const float vx = add(add(add(mul(cam.V[0], c0.x), mul(cam.V[4], c0.y)), mul(cam.V[8], c0.z)), cam.V[12]);
            const float vy = add(add(add(mul(cam.V[1], c0.x), mul(cam.V[5], c0.y)), mul(cam.V[9], c0.z)), cam.V[13]);
            const float vz = add(add(add(mul(cam.V[2], c0.x), mul(cam.V[6], c0.y)), mul(cam.V[10], c0.z)), cam.V[14]);
            if (animated) {
                float4 c3 = row[3];
                animate_row(p, id, row, c3);
            }
            float4 rec[4];
            float qa, gp;
            project_visible(row, c0, vx, vy, vz, cam, p.sh_degree, p.sh_lod_distance, rec, &qa, &gp);
            float4* dst = p.projected + (size_t)id * 4;
            dst[0] = rec[0];
            dst[1] = rec[1];
            dst[2] = rec[2];
            dst[3] = rec[3];
            if (p.collect_stats) {
                // shaders/cull.glsl:296-318
                const uint32_t qpx = g_f2u_sat(g_min(g_max(0.0f, qa), 4294967295.0f));
                const uint32_t gpx = g_f2u_sat(g_min(ceilf(gp), 4294967295.0f));
                d0 += (uint32_t)(qpx + 1023u) >> 10u;
                m1 = max(m1, qpx);
                d2 += qpx > 1024u;
                d3 += qpx > 16384u;
                d4 += (uint32_t)(gpx + 1023u) >> 10u;
                m5 = max(m5, gpx);
                d6 += gpx > 1024u;
                d7 += gpx > 16384u;
            }
        }
        // every lane is done with the stage before the next group refills it
        __syncwarp();
    }
    if (stage_failed) atomicOr(&p.fc->error_flags, kErrCullStage);
    if (p.collect_stats) {
        const uint32_t s0 = __reduce_add_sync(0xffffffffu, d0), s2 = __reduce_add_sync(0xffffffffu, d2);
        const uint32_t s3 = __reduce_add_sync(0xffffffffu, d3), s4 = __reduce_add_sync(0xffffffffu, d4);
        const uint32_t s6 = __reduce_add_sync(0xffffffffu, d6), s7 = __reduce_add_sync(0xffffffffu, d7);
        const uint32_t x1 = __reduce_max_sync(0xffffffffu, m1), x5 = __reduce_max_sync(0xffffffffu, m5);
        if (lane == 0) {
            if (s0) atomicAdd(&p.fc->diag[0], s0);
            if (x1) atomicMax(&p.fc->diag[1], x1);
            if (s2) atomicAdd(&p.fc->diag[2], s2);
            if (s3) atomicAdd(&p.fc->diag[3], s3);
            if (s4) atomicAdd(&p.fc->diag[4], s4);
            if (x5) atomicMax(&p.fc->diag[5], x5);
            if (s6) atomicAdd(&p.fc->diag[6], s6);
            if (s7) atomicAdd(&p.fc->diag[7], s7);
        }
    }
}

// ---------------------------------------------------------------------------
// FP16-SH rows (144 bytes: chunks 0..2 as the GpuGaussian row, then 48 IEEE
// half SH coefficients in the order 3k + c).  The SH colour of a warp's 32
// visible rows is evaluated on the tensor cores: per row the 16 SH basis
// values Y_k(dir) (FP32, the weights of shaders/cull.glsl:355-408) split into
// two FP16 terms (Y = hi + lo, so Y keeps ~22 bits) times the row's FP16
// coefficients, accumulated in FP32.  Every row has its own coefficients,
// so the product is a batch of 1 x 16 by 16 x 3 products: one
// mma.m16n8k16 takes 16 rows' basis vectors (A, 16 x 16) against 8
// (row, channel) columns of coefficients (B, 16 x 8) and keeps the 8 outputs
// on its diagonal blocks; 2 x 6 x 2 instructions per 32 rows.  The warp-level
// MMA fits the per-warp staging of this kernel; a CTA-wide tcgen05 MMA would
// need 128-row tiles staged through shared memory and TMEM for the same
// 48 useful outputs per 16 rows.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sh_basis(float x, float y, float z, int eff, bool valid, float* Y) {
#pragma unroll
    for (int k = 0; k < 16; ++k) Y[k] = 0.0f;
    if (!valid) return;
    Y[0] = SH_C0;
    if (eff >= 1) {
        Y[1] = mul(-SH_C1, y);
        Y[2] = mul(SH_C1, z);
        Y[3] = mul(-SH_C1, x);
        if (eff >= 2) {
            const float xx = mul(x, x), yy = mul(y, y), zz = mul(z, z);
            const float xy = mul(x, y), yz = mul(y, z), xz = mul(z, x);
            Y[4] = mul(SH_C2_0, xy);
            Y[5] = mul(SH_C2_1, yz);
            Y[6] = mul(SH_C2_2, sub(sub(mul(2.0f, zz), xx), yy));
            Y[7] = mul(SH_C2_3, xz);
            Y[8] = mul(SH_C2_4, sub(xx, yy));
            if (eff >= 3) {
                Y[9] = mul(mul(SH_C3_0, y), sub(mul(3.0f, xx), yy));
                Y[10] = mul(mul(SH_C3_1, xy), z);
                Y[11] = mul(mul(SH_C3_2, y), sub(sub(mul(4.0f, zz), xx), yy));
                Y[12] = mul(mul(SH_C3_3, z), sub(sub(mul(2.0f, zz), mul(3.0f, xx)), mul(3.0f, yy)));
                Y[13] = mul(mul(SH_C3_4, x), sub(sub(mul(4.0f, zz), xx), yy));
                Y[14] = mul(mul(SH_C3_5, z), sub(xx, yy));
                Y[15] = mul(mul(SH_C3_6, x), sub(xx, mul(3.0f, yy)));
            }
        }
    }
}

__device__ __forceinline__ uint32_t pack_h2(__half a, __half b) {
    return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

__device__ __forceinline__ void mma_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                          uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// SH colour (before the +0.5 bias) of the warp's 32 staged half rows; lane l
// passes the direction of its row and receives that row's colour.  s_y: 2 x
// 32 x 16 halves of scratch, s_out: 32 x 3 floats of scratch (per warp).
__device__ __forceinline__ void sh_eval_tc(const float4* stage, int lane, float x, float y, float z, int eff,
                                           bool valid, __half* s_y, float* s_out, float* res) {
    float Y[16];
    sh_basis(x, y, z, eff, valid, Y);
    uint32_t hw[8], lw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const __half h0 = __float2half_rn(Y[2 * k]), h1 = __float2half_rn(Y[2 * k + 1]);
        hw[k] = pack_h2(h0, h1);
        lw[k] = pack_h2(__float2half_rn(Y[2 * k] - __half2float(h0)), __float2half_rn(Y[2 * k + 1] - __half2float(h1)));
    }
    uint4* yh = reinterpret_cast<uint4*>(s_y) + lane * 2;
    uint4* yl = reinterpret_cast<uint4*>(s_y + 512) + lane * 2;
    yh[0] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    yh[1] = make_uint4(hw[4], hw[5], hw[6], hw[7]);
    yl[0] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    yl[1] = make_uint4(lw[4], lw[5], lw[6], lw[7]);
    __syncwarp();
    const int gid = lane >> 2, tig = lane & 3;
    const uint32_t* wy = reinterpret_cast<const uint32_t*>(s_y);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int r0 = 16 * t + gid, r1 = r0 + 8;
        uint32_t ah[4], al[4];
        ah[0] = wy[r0 * 8 + tig];
        ah[1] = wy[r1 * 8 + tig];
        ah[2] = wy[r0 * 8 + tig + 4];
        ah[3] = wy[r1 * 8 + tig + 4];
        al[0] = wy[256 + r0 * 8 + tig];
        al[1] = wy[256 + r1 * 8 + tig];
        al[2] = wy[256 + r0 * 8 + tig + 4];
        al[3] = wy[256 + r1 * 8 + tig + 4];
#pragma unroll
        for (int b = 0; b < 6; ++b) {
            // column gid of this 8-column block: coefficients of channel c of row g
            const int q = 8 * b + gid, g = q / 3, c = q - 3 * g;
            const uint32_t* shw =
                reinterpret_cast<const uint32_t*>(stage + (16 * t + g) * kHalfStageStride + 3) + 8 * c;
            const uint32_t b0 = shw[tig], b1 = shw[tig + 4];
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            mma_16816(d, ah[0], ah[1], ah[2], ah[3], b0, b1);
            mma_16816(d, al[0], al[1], al[2], al[3], b0, b1);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = gid + (e >> 1) * 8, col = 2 * tig + (e & 1);
                const int qq = 8 * b + col;
                if (qq / 3 == row) s_out[(16 * t + row) * 3 + (qq - 3 * row)] = d[e];
            }
        }
    }
    __syncwarp();
    res[0] = s_out[lane * 3 + 0];
    res[1] = s_out[lane * 3 + 1];
    res[2] = s_out[lane * 3 + 2];
    __syncwarp();
}

// The projection pass for FP16-SH rows: as cull_project_kernel, staging 144
// bytes per visible row, with the SH colour from sh_eval_tc and everything
// else (covariance, conic, radius, centre, depth) in FP32 as for full rows.
__global__ void __launch_bounds__(kCullThreads, 6) cull_project_half_kernel(CullParams p) {
    extern __shared__ float4 smem4[];
    __shared__ __align__(8) uint64_t s_bar[kCullWarps];
    __shared__ __align__(16) __half s_y[kCullWarps][1024];
    __shared__ float s_out[kCullWarps][96];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        mbar_init(&s_bar[warp], 1);
        mbar_fence_init();
    }
    __syncthreads();
    float4* const stage0 = smem4 + (size_t)warp * 32 * kHalfStageStride;
    const uint32_t n_vis = p.fc->visible_count;
    const uint32_t groups = (n_vis + 31) / 32;
    const uint32_t wg = blockIdx.x * kCullWarps + warp, nw = gridDim.x * kCullWarps;
    CamRegs cam;
    load_cam(p.cam, cam);
    const uint64_t stream_policy = l2_policy_evict_first();
    bool stage_failed = false;
    uint32_t phase = 0;
    uint32_t d0 = 0, d2 = 0, d3 = 0, d4 = 0, d6 = 0, d7 = 0, m1 = 0, m5 = 0;
    for (uint32_t g = wg; g < groups; g += nw) {
        const uint32_t id = stage_group<kHalfRowChunks, kHalfRowChunks, kHalfStageStride>(
            p.rows, p.ids_out, g * 32u, n_vis, stage0, &s_bar[warp], lane, stream_policy);
        if (!mbar_wait_bounded(&s_bar[warp], phase)) stage_failed = true;
        phase ^= 1u;
        const bool valid = id != kSentinel;
        float4* row = stage0 + lane * kHalfStageStride;
        const float4 c0 = row[0];
        float vx = 0.0f, vy = 0.0f, vz = 0.0f, dx = 0.0f, dy = 0.0f, dz = 0.0f;
        int eff = 0;
        if (valid) {
            vx = add(add(add(mul(cam.V[0], c0.x), mul(cam.V[4], c0.y)), mul(cam.V[8], c0.z)), cam.V[12]);
            vy = add(add(add(mul(cam.V[1], c0.x), mul(cam.V[5], c0.y)), mul(cam.V[9], c0.z)), cam.V[13]);
            vz = add(add(add(mul(cam.V[2], c0.x), mul(cam.V[6], c0.y)), mul(cam.V[10], c0.z)), cam.V[14]);
            // view direction and SH degree as in project_visible (shaders/cull.glsl:323-351)
            const float ddx = sub(c0.x, cam.camw[0]), ddy = sub(c0.y, cam.camw[1]), ddz = sub(c0.z, cam.camw[2]);
            const float len = __fsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
            dx = dv(ddx, len);
            dy = dv(ddy, len);
            dz = dv(ddz, len);
            eff = p.sh_degree;
            if (p.sh_lod_distance > 0.0f && (-vz) > p.sh_lod_distance) eff = 0;
        }
        float colour[3];
        sh_eval_tc(stage0, lane, dx, dy, dz, eff, valid, s_y[warp], s_out[warp], colour);
        if (valid) {
            float4 rec[4];
            float qa, gp;
            project_visible<true>(row, c0, vx, vy, vz, cam, p.sh_degree, p.sh_lod_distance, rec, &qa, &gp, colour[0],
                                  colour[1], colour[2]);
            float4* dst = p.projected + (size_t)id * 4;
            dst[0] = rec[0];
            dst[1] = rec[1];
            dst[2] = rec[2];
            dst[3] = rec[3];
            if (p.collect_stats) {
                const uint32_t qpx = g_f2u_sat(g_min(g_max(0.0f, qa), 4294967295.0f));
                const uint32_t gpx = g_f2u_sat(g_min(ceilf(gp), 4294967295.0f));
                d0 += (uint32_t)(qpx + 1023u) >> 10u;
                m1 = max(m1, qpx);
                d2 += qpx > 1024u;
                d3 += qpx > 16384u;
                d4 += (uint32_t)(gpx + 1023u) >> 10u;
                m5 = max(m5, gpx);
                d6 += gpx > 1024u;
                d7 += gpx > 16384u;
            }
        }
        __syncwarp();
    }
    if (stage_failed) atomicOr(&p.fc->error_flags, kErrCullStage);
    if (p.collect_stats) {
        const uint32_t s0 = __reduce_add_sync(0xffffffffu, d0), s2 = __reduce_add_sync(0xffffffffu, d2);
        const uint32_t s3 = __reduce_add_sync(0xffffffffu, d3), s4 = __reduce_add_sync(0xffffffffu, d4);
        const uint32_t s6 = __reduce_add_sync(0xffffffffu, d6), s7 = __reduce_add_sync(0xffffffffu, d7);
        const uint32_t x1 = __reduce_max_sync(0xffffffffu, m1), x5 = __reduce_max_sync(0xffffffffu, m5);
        if (lane == 0) {
            if (s0) atomicAdd(&p.fc->diag[0], s0);
            if (x1) atomicMax(&p.fc->diag[1], x1);
            if (s2) atomicAdd(&p.fc->diag[2], s2);
            if (s3) atomicAdd(&p.fc->diag[3], s3);
            if (s4) atomicAdd(&p.fc->diag[4], s4);
            if (x5) atomicMax(&p.fc->diag[5], x5);
            if (s6) atomicAdd(&p.fc->diag[6], s6);
            if (s7) atomicAdd(&p.fc->diag[7], s7);
        }
    }
}

// Colours of a frame's binned records for another gsanim appearance state
// (a frame of a state batch: the geometry, order and tiles of the frame stay,
// the colours change).  Record i (sorted position) gets the colour the
// projection pass would give its splat under the state of `p`: the same row,
// deltas, view direction, SH degree and operations (animate_row, sh_eval,
// shaders/cull.glsl:125-164, 323-417), bias and clamp.
__global__ void __launch_bounds__(128) recolour_kernel(CullParams p, const RasterRecord* __restrict__ records,
                                                       float4* __restrict__ colours) {
    const uint32_t n_vis = p.fc->visible_count;
    CamRegs cam;
    load_cam(p.cam, cam);
    // the shader blends whenever the weight is positive, states 0 and 0
    // included (gsanim_sample returns {0, 0, w} between two linear keys of
    // the base state), and (1 - w) x + w x need not round to x
    const bool animated = p.anim_deltas != nullptr && (p.anim_state_a != 0 || p.anim_weight > 0.0f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_vis; i += gridDim.x * blockDim.x) {
        const uint32_t id = records[i].splat_id;
        if (id >= p.n) continue;
        float4 row[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) row[k] = __ldg(p.rows + (size_t)id * 16 + k);
        const float4 c0 = row[0];
        const float vz = add(add(add(mul(cam.V[2], c0.x), mul(cam.V[6], c0.y)), mul(cam.V[10], c0.z)), cam.V[14]);
        if (animated) {
            float4 c3 = row[3];
            animate_row(p, id, row, c3);
        }
        const float ddx = sub(c0.x, cam.camw[0]), ddy = sub(c0.y, cam.camw[1]), ddz = sub(c0.z, cam.camw[2]);
        const float len = __fsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
        const float x = dv(ddx, len), y = dv(ddy, len), z = dv(ddz, len);
        int eff = p.sh_degree;
        if (p.sh_lod_distance > 0.0f && (-vz) > p.sh_lod_distance) eff = 0;
        float res[3];
        sh_eval(row, x, y, z, eff, res);
        colours[i] = make_float4(g_max(add(res[0], 0.5f), 0.0f), g_max(add(res[1], 0.5f), 0.0f),
                                 g_max(add(res[2], 0.5f), 0.0f), 0.0f);
    }
}

int launch_recolour(const CullParams& p, const RasterRecord* records, float4* colours, uint32_t num_sms,
                    cudaStream_t s) {
    uint32_t grid = (p.n + 127) / 128;
    if (grid > num_sms * 8) grid = num_sms * 8;
    if (grid == 0) return 0;
    recolour_kernel<<<grid, 128, 0, s>>>(p, records, colours);
    return 1;
}

// Pass 3, gsanim 0.3 assets only (shaders/cull.glsl:141-148, 354-416): the
// colour of every compacted visible row is the sum over the layers of
// max(SH colour, 0) * the layer's RGB weight, without the +0.5 bias, where
// layer l's 48 half coefficients replace the row's DC (slots 12..14) and SH
// (slot 16 + 3k + c holds j = 3 + 15c + k).  The view direction, the SH
// degree and its distance LOD are those of the projection pass, computed
// with the same operations; the record's other fields stay as projected.
__global__ void __launch_bounds__(256) cull_layers_kernel(CullParams p) {
    const uint32_t n_vis = p.fc->visible_count;
    CamRegs cam;
    load_cam(p.cam, cam);
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n_vis; v += gridDim.x * blockDim.x) {
        const uint32_t id = p.ids_out[v];
        const float4 c0 = __ldg(p.heads + id);
        const float vz = add(add(add(mul(cam.V[2], c0.x), mul(cam.V[6], c0.y)), mul(cam.V[10], c0.z)), cam.V[14]);
        const float ddx = sub(c0.x, cam.camw[0]), ddy = sub(c0.y, cam.camw[1]), ddz = sub(c0.z, cam.camw[2]);
        const float len = __fsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
        const float x = dv(ddx, len), y = dv(ddy, len), z = dv(ddz, len);
        int eff = p.sh_degree;
        if (p.sh_lod_distance > 0.0f && (-vz) > p.sh_lod_distance) eff = 0;
        float4 row[16];
        float* f = reinterpret_cast<float*>(row);
        float col[3] = {0.0f, 0.0f, 0.0f};
        for (int l = 0; l < p.layer_count; ++l) {
            const unsigned short* h =
                reinterpret_cast<const unsigned short*>(p.layer_halves) + ((size_t)l * p.n + id) * 48u;
            for (int j = 0; j < 3; ++j) f[12 + j] = __half2float(__ushort_as_half(__ldg(h + j)));
            for (int slot = 16; slot < 61; ++slot)
                f[slot] = __half2float(__ushort_as_half(__ldg(h + 3 + ((slot - 16) % 3) * 15 + (slot - 16) / 3)));
            float r3[3];
            sh_eval(row, x, y, z, eff, r3);
            for (int k = 0; k < 3; ++k) col[k] = add(col[k], mul(g_max(r3[k], 0.0f), __ldg(p.layer_weights + l * 3 + k)));
        }
        p.projected[(size_t)id * 4] = make_float4(col[0], col[1], col[2], c0.w);
    }
}

int launch_cull(const CullParams& p, uint32_t num_sms, cudaStream_t s) {
    // the shared-memory limit is a per-device function attribute: raise it
    // once on every device this process launches on
    static std::atomic<uint64_t> attr_devices{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
    if (!bit || !(attr_devices.load() & bit)) {
        cudaFuncSetAttribute(cull_project_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCullSmem);
        cudaFuncSetAttribute(cull_project_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCullSmem);
        cudaFuncSetAttribute(cull_project_kernel<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCullSmem);
        cudaFuncSetAttribute(cull_project_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCullSmem);
        cudaFuncSetAttribute(cull_project_half_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kCullHalfSmem);
        attr_devices.fetch_or(bit);
    }
    int deg = p.sh_degree < 0 ? 0 : (p.sh_degree > 3 ? 3 : p.sh_degree);
    if (p.anim_deltas) deg = 3;   // the delta pass touches every SH slot of the staged row
    const uint32_t tiles = (p.n + kCullVisTile - 1) / kCullVisTile;
    if (tiles == 0) return 0;
    launch_pdl(cull_visible_kernel, dim3(tiles), dim3(kCullVisThreads), 0, s, p);
    // projection: persistent, as many CTAs as fit (6 per SM) for the largest possible visible count
    const uint32_t groups_cap = (p.n + 31) / 32;
    uint32_t pgrid = num_sms * 6;
    if (pgrid * kCullWarps > groups_cap) pgrid = (groups_cap + kCullWarps - 1) / kCullWarps;
    if (p.half_rows) {
        cull_project_half_kernel<<<pgrid, kCullThreads, kCullHalfSmem, s>>>(p);
        return 2;
    }
    switch (deg) {
        case 0: launch_pdl(cull_project_kernel<4>, dim3(pgrid), dim3(kCullThreads), kCullSmem, s, p); break;
        case 1: launch_pdl(cull_project_kernel<7>, dim3(pgrid), dim3(kCullThreads), kCullSmem, s, p); break;
        case 2: launch_pdl(cull_project_kernel<10>, dim3(pgrid), dim3(kCullThreads), kCullSmem, s, p); break;
        default: launch_pdl(cull_project_kernel<16>, dim3(pgrid), dim3(kCullThreads), kCullSmem, s, p); break;
    }
    if (p.layer_count > 0) {
        uint32_t lgrid = (p.n + 255) / 256;
        if (lgrid > num_sms * 8) lgrid = num_sms * 8;
        cull_layers_kernel<<<lgrid, 256, 0, s>>>(p);
        return 3;
    }
    return 2;
}

}  // namespace gs
