// Cull / project / SH kernel: shaders/cull.glsl:166-424 (+ cull_reset,
// :456-473, folded in) for the B200.
//
// Memory plan (HBM-bound, 256-byte GpuGaussian rows):
//   * each lane reads the first 16 bytes (position, opacity) of its row and
//     runs the near/frustum test;
//   * the warp then fetches only the visible rows' remaining 16-byte chunks
//     with coalesced 128-bit loads (consecutive lanes -> consecutive chunks)
//     into a padded shared-memory stage (272-byte row stride: conflict-free
//     128-bit shared loads);
//   * culled rows cost one 32-byte sector, visible rows 256 bytes (fewer for
//     sh_degree < 3);
//   * visible (key, id) pairs are compacted in index order with a
//     decoupled look-back over CTA tiles, so the depth sort runs on N_vis
//     pairs instead of N (the culled tail of the reference's all-N sort is
//     all-equal (0xFFFFFFFF, 0xFFFFFFFF) pairs, so the result is identical).
// Arithmetic follows the GLSL operand order with unfused intrinsics so the
// keys, cull mask and projected records match the CPU oracle bit for bit.
#include "gs_common.cuh"
#include "gs_internal.h"

namespace gs {

constexpr int kStageStride = 17;  // float4 per staged row (16 + 1 pad)
constexpr int kCullWarps = kCullThreads / 32;
constexpr size_t kCullSmem = (size_t)kCullWarps * 32 * kStageStride * sizeof(float4) +
                             2 * (size_t)kCullTile * sizeof(uint32_t);

struct CamRegs {
    float V[16];
    float P0, P5, P10, P14;
    float vpx, vpy, ortho, fxp, fxo, ysign, z01;
    float camw[3];
};

__device__ __forceinline__ void load_cam(const gs_camera* c, CamRegs& r) {
    const float* f = reinterpret_cast<const float*>(c);
#pragma unroll
    for (int k = 0; k < 16; ++k) r.V[k] = __ldg(f + k);
    r.P0 = __ldg(f + 16 + 0);
    r.P5 = __ldg(f + 16 + 5);
    r.P10 = __ldg(f + 16 + 10);
    r.P14 = __ldg(f + 16 + 14);
    r.vpx = __ldg(f + 32);
    r.vpy = __ldg(f + 33);
    r.ortho = __ldg(f + 34);
    r.fxp = __ldg(f + 35);
    r.fxo = __ldg(f + 36);
    r.ysign = __ldg(f + 37);
    r.z01 = __ldg(f + 38);
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
__device__ __forceinline__ void project_visible(const float4* row, float4 c0, float vx, float vy, float vz,
                                                const CamRegs& cam, int sh_degree, float sh_lod, float4* out,
                                                float* quad_area, float* gps_points) {
    const float t = cam.ortho;
    float4 c1 = row[1], c2 = row[2], c3 = row[3];
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
    float res[3] = {mul(SH_C0, c3.x), mul(SH_C0, c3.y), mul(SH_C0, c3.z)};
    if (eff >= 1) {
        // SH(k) = floats 16 + 3k .. 18 + 3k  (chunks 4..15)
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
#pragma unroll
    for (int k = 0; k < 3; ++k) res[k] = g_max(add(res[k], 0.5f), 0.0f);

    out[0] = make_float4(res[0], res[1], res[2], c0.w);
    out[1] = make_float4(cx, rcy, radius_x, radius_y);
    out[2] = make_float4(conic_x, rconic_y, conic_z, ndc_z);
    out[3] = make_float4(a, mul(b, cam.ysign), c, det);
}

__global__ void __launch_bounds__(kCullThreads, 2) cull_kernel(CullParams p, int nchunks) {
    extern __shared__ float4 smem4[];
    float4* stage = smem4;
    uint32_t* s_keys = reinterpret_cast<uint32_t*>(stage + kCullWarps * 32 * kStageStride);
    uint32_t* s_ids = s_keys + kCullTile;
    __shared__ int vis_list[kCullWarps][32];
    __shared__ uint32_t seg_count[kCullRounds * kCullWarps];
    __shared__ uint32_t seg_off[kCullRounds * kCullWarps];
    __shared__ uint32_t s_tile, s_excl, s_total;
    static_assert(kCullRounds * kCullWarps == 32, "one warp scans the segments");

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t num_tiles = (p.n + kCullTile - 1) / kCullTile;
    CamRegs cam;
    load_cam(p.cam, cam);
    float4* warp_stage = stage + warp * 32 * kStageStride;
    float4* my_stage = warp_stage + lane * kStageStride;

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&p.fc->cull_ticket, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= num_tiles) break;
        const uint32_t base = tile * kCullTile;

        for (int round = 0; round < kCullRounds; ++round) {
            const uint32_t wbase = base + round * kCullThreads + warp * 32;
            const uint32_t g = wbase + lane;
            const bool valid = g < p.n;
            float4 c0 = valid ? __ldg(p.rows + (size_t)g * 16) : make_float4(0.f, 0.f, 0.f, 0.f);
            // p_view = view * vec4(position, 1.0)
            float vx = add(add(add(mul(cam.V[0], c0.x), mul(cam.V[4], c0.y)), mul(cam.V[8], c0.z)), cam.V[12]);
            float vy = add(add(add(mul(cam.V[1], c0.x), mul(cam.V[5], c0.y)), mul(cam.V[9], c0.z)), cam.V[13]);
            float vz = add(add(add(mul(cam.V[2], c0.x), mul(cam.V[6], c0.y)), mul(cam.V[10], c0.z)), cam.V[14]);
            bool visible = valid && (vz <= -0.2f);
            if (visible) {
                float inv_z = dv(-1.0f, vz);
                float ndc_x = add(mul(mul(mul(cam.P0, vx), inv_z), sub(1.0f, cam.ortho)), mul(mul(cam.P0, vx), cam.ortho));
                float ndc_y = add(mul(mul(mul(cam.P5, vy), inv_z), sub(1.0f, cam.ortho)), mul(mul(cam.P5, vy), cam.ortho));
                visible = fabsf(ndc_x) <= 1.3f && fabsf(ndc_y) <= 1.3f;
            }
            const uint32_t mask = __ballot_sync(0xffffffffu, visible);
            const int nvis = __popc(mask);
            const int pos = __popc(mask & ((1u << lane) - 1u));
            if (visible) vis_list[warp][pos] = lane;
            __syncwarp();
            // Coalesced 128-bit loads of the visible rows' chunks 1..nchunks-1.
            const int per = nchunks - 1;
            const int total = nvis * per;
            for (int u = lane; u < total; u += 32) {
                int v = u / per;
                int ch = 1 + (u - v * per);
                int rl = vis_list[warp][v];
                warp_stage[rl * kStageStride + ch] = __ldg(p.rows + (size_t)(wbase + rl) * 16 + ch);
            }
            __syncwarp();
            float qa = 0.0f, gp = 0.0f;
            if (visible) {
                float4 rec[4];
                project_visible(my_stage, c0, vx, vy, vz, cam, p.sh_degree, p.sh_lod_distance, rec, &qa, &gp);
                float4* dst = p.projected + (size_t)g * 4;
                dst[0] = rec[0];
                dst[1] = rec[1];
                dst[2] = rec[2];
                dst[3] = rec[3];
                const int seg = round * kCullWarps + warp;
                s_keys[seg * 32 + pos] = 0xFFFFFFFFu - __float_as_uint(g_max(-vz, 0.0f));
                s_ids[seg * 32 + pos] = g;
            } else if (valid && p.write_invisible) {
                float4* dst = p.projected + (size_t)g * 4;
                dst[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                dst[1] = make_float4(0.f, 0.f, 0.f, 0.f);
                dst[2] = make_float4(1.f, 0.f, 1.f, 1.f);
                dst[3] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if (p.collect_stats && mask) {
                // shaders/cull.glsl:296-318, warp-aggregated.
                uint32_t qpx = visible ? g_f2u_sat(g_min(g_max(0.0f, qa), 4294967295.0f)) : 0u;
                uint32_t gpx = visible ? g_f2u_sat(g_min(ceilf(gp), 4294967295.0f)) : 0u;
                uint32_t d0 = visible ? ((uint32_t)(qpx + 1023u) >> 10u) : 0u;
                uint32_t d4 = visible ? ((uint32_t)(gpx + 1023u) >> 10u) : 0u;
                uint32_t s0 = __reduce_add_sync(0xffffffffu, d0);
                uint32_t m1 = __reduce_max_sync(0xffffffffu, qpx);
                uint32_t s2 = __reduce_add_sync(0xffffffffu, (uint32_t)(visible && qpx > 1024u));
                uint32_t s3 = __reduce_add_sync(0xffffffffu, (uint32_t)(visible && qpx > 16384u));
                uint32_t s4 = __reduce_add_sync(0xffffffffu, d4);
                uint32_t m5 = __reduce_max_sync(0xffffffffu, gpx);
                uint32_t s6 = __reduce_add_sync(0xffffffffu, (uint32_t)(visible && gpx > 1024u));
                uint32_t s7 = __reduce_add_sync(0xffffffffu, (uint32_t)(visible && gpx > 16384u));
                if (lane == 0) {
                    atomicAdd(&p.fc->diag[0], s0);
                    atomicMax(&p.fc->diag[1], m1);
                    atomicAdd(&p.fc->diag[2], s2);
                    atomicAdd(&p.fc->diag[3], s3);
                    atomicAdd(&p.fc->diag[4], s4);
                    atomicMax(&p.fc->diag[5], m5);
                    atomicAdd(&p.fc->diag[6], s6);
                    atomicAdd(&p.fc->diag[7], s7);
                }
            }
            if (lane == 0) seg_count[round * kCullWarps + warp] = (uint32_t)nvis;
            __syncwarp();
        }
        __syncthreads();
        if (warp == 0) {
            uint32_t cnt = seg_count[lane];
            uint32_t x = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            seg_off[lane] = x - cnt;
            uint32_t total = __shfl_sync(0xffffffffu, x, 31);
            if (lane == 0) {
                u64* st = p.status + tile;
                uint32_t excl = 0;
                if (tile == 0) {
                    st_release64(st, status_word(p.epoch, kFlagInc, total));
                } else {
                    st_release64(st, status_word(p.epoch, kFlagAgg, total));
                    bool to = false;
                    excl = lookback(p.status, 1, tile, p.epoch, &to);
                    if (to) atomicOr(&p.fc->error_flags, kErrCullLookback);
                    st_release64(st, status_word(p.epoch, kFlagInc, excl + total));
                }
                s_excl = excl;
                s_total = total;
                if (tile == num_tiles - 1) p.fc->visible_count = excl + total;
            }
        }
        __syncthreads();
        const uint32_t excl = s_excl;
        for (int slot = threadIdx.x; slot < kCullTile; slot += kCullThreads) {
            int seg = slot >> 5, k = slot & 31;
            if ((uint32_t)k < seg_count[seg]) {
                uint32_t o = excl + seg_off[seg] + (uint32_t)k;
                p.keys_out[o] = s_keys[slot];
                p.ids_out[o] = s_ids[slot];
            }
        }
        __syncthreads();
    }
}

int launch_cull(const CullParams& p, uint32_t num_sms, cudaStream_t s) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(cull_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCullSmem);
        attr_set = true;
    }
    static const int chunks_for_degree[4] = {4, 7, 10, 16};
    int deg = p.sh_degree < 0 ? 0 : (p.sh_degree > 3 ? 3 : p.sh_degree);
    uint32_t tiles = (p.n + kCullTile - 1) / kCullTile;
    uint32_t grid = num_sms * 2;
    if (grid > tiles) grid = tiles;
    if (grid == 0) return 0;
    cull_kernel<<<grid, kCullThreads, kCullSmem, s>>>(p, chunks_for_degree[deg]);
    return 1;
}

}  // namespace gs
