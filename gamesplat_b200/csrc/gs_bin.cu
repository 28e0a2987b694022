// Tile binning of depth-sorted splats for the tile rasterizer.
//
// The reference rasterizes one instanced quad per sorted splat through the GL
// pipeline (shaders/splat.glsl:39-75, src/renderer.cpp:1687-1720).  Here each
// sorted splat s (a) computes its covered pixel rectangle with the same quad
// geometry and fill rule as the CPU oracle (gs::quad_rect), (b) writes a
// 64-byte RasterRecord at position s, and (c) emits one (tile, s) entry per
// 16x16 tile that can receive a non-discarded fragment.  Entries are written
// in s order at offsets found by a decoupled look-back over CTA tiles, so a
// stable sort on the tile id alone keeps each tile's list in depth order.
//
// Tile selection is conservative: the covered rectangle is intersected with
// the bounding box of the ellipse where the Gaussian's alpha reaches 1/255
// (power >= cutoff), widened by a pixel; per-pixel coverage and discards are
// still evaluated exactly in the rasterizer.
#include "gs_common.cuh"
#include "gs_internal.h"

namespace gs {

__global__ void __launch_bounds__(kBinThreads) bin_kernel(BinParams p) {
    __shared__ uint32_t scan_tmp[33];
    __shared__ uint32_t s_tile, s_excl;
    const uint32_t n_vis = p.fc->visible_count;
    const uint32_t num_tiles = (n_vis + kBinThreads - 1) / kBinThreads;
    const uint32_t* __restrict__ sorted_ids = p.depth_plan->vfinal;
    const float* camf = reinterpret_cast<const float*>(p.cam);
    const float vp_w = __ldg(camf + 32), vp_h = __ldg(camf + 33), ysign = __ldg(camf + 37);

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&p.fc->bin_ticket, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= num_tiles) break;
        const uint32_t s = tile * kBinThreads + threadIdx.x;
        uint32_t count = 0;
        int tx0 = 0, tx1 = -1, ty0 = 0, ty1 = -1;
        if (s < n_vis) {
            const uint32_t id = sorted_ids[s];
            const float4* P = p.projected + (size_t)id * 4;
            const float4 co = P[0], cr = P[1], cd = P[2];
            PixelRect rc;
            const float cutoff = alpha_cutoff(co.w);
            bool ok = quad_rect(cr.x, cr.y, cr.z, cr.w, cd.w, p.jitter_x, p.jitter_y, vp_w, vp_h, ysign, p.width,
                                p.height, &rc);
            ok = ok && cutoff <= 0.0f;
            const float ccx = add(cr.x, p.jitter_x), ccy = add(cr.y, p.jitter_y);
            if (ok) {
                // Bounding box of {d : conic(d) <= -2 cutoff}.
                const float cx = cd.x, cy = cd.y, cz = cd.z;
                const float k = -2.0f * cutoff;
                const float dt = cx * cz - cy * cy;
                if (dt > 0.0f) {
                    float hx = sqrtf(k * cz / dt) * 1.001f + 1.0f;
                    float hy = sqrtf(k * cx / dt) * 1.001f + 1.0f;
                    // pixel i is a candidate if |i + 0.5 - ccx| <= hx
                    float fi0 = ceilf(ccx - hx - 0.5f), fi1 = floorf(ccx + hx - 0.5f);
                    float fj0 = ceilf(ccy - hy - 0.5f), fj1 = floorf(ccy + hy - 0.5f);
                    int ei0 = (int)fmaxf(fi0, -1.0f), ei1 = (int)fminf(fi1, 32767.0f);
                    int ej0 = (int)fmaxf(fj0, -1.0f), ej1 = (int)fminf(fj1, 32767.0f);
                    rc.i0 = max(rc.i0, ei0);
                    rc.i1 = min(rc.i1, ei1 + 1);
                    rc.j0 = max(rc.j0, ej0);
                    rc.j1 = min(rc.j1, ej1 + 1);
                }
                ok = rc.i0 < rc.i1 && rc.j0 < rc.j1;
            }
            if (ok) {
                tx0 = rc.i0 / kTileW;
                tx1 = (rc.i1 - 1) / kTileW;
                ty0 = rc.j0 / kTileH;
                ty1 = (rc.j1 - 1) / kTileH;
                count = (uint32_t)((tx1 - tx0 + 1) * (ty1 - ty0 + 1));
                // Record with the exact (untightened) quad coverage.
                PixelRect q;
                quad_rect(cr.x, cr.y, cr.z, cr.w, cd.w, p.jitter_x, p.jitter_y, vp_w, vp_h, ysign, p.width,
                          p.height, &q);
                RasterRecord rec;
                rec.cx = ccx;
                rec.cy = ccy;
                rec.conic_x = cd.x;
                rec.conic_2y = mul(2.0f, cd.y);
                rec.conic_z = cd.z;
                rec.opacity = co.w;
                rec.cutoff = cutoff;
                rec.r = co.x;
                rec.g = co.y;
                rec.b = co.z;
                rec.rect_x = (uint32_t)q.i0 | ((uint32_t)q.i1 << 16);
                rec.rect_y = (uint32_t)q.j0 | ((uint32_t)q.j1 << 16);
                float zw = add(mul(cd.w, 0.5f), 0.5f);
                rec.depth24 = (uint32_t)__float2int_rn(mul(g_clamp(zw, 0.0f, 1.0f), 16777215.0f));
                rec.splat_id = id;
                rec.hash_z = add((float)id, p.frame_seed);
                rec.pad = 0u;
                float4* dst = reinterpret_cast<float4*>(p.records + s);
                const float4* src = reinterpret_cast<const float4*>(&rec);
                dst[0] = src[0];
                dst[1] = src[1];
                dst[2] = src[2];
                dst[3] = src[3];
            }
        }
        uint32_t total;
        const uint32_t local = block_excl_scan(count, scan_tmp, &total);
        if (threadIdx.x == 0) {
            u64* st = p.status + tile;
            uint32_t excl = 0;
            if (tile == 0) {
                st_release64(st, status_word(p.epoch, kFlagInc, total));
            } else {
                st_release64(st, status_word(p.epoch, kFlagAgg, total));
                bool to = false;
                excl = lookback(p.status, 1, tile, p.epoch, &to);
                if (to) atomicOr(&p.fc->error_flags, kErrBinLookback);
                st_release64(st, status_word(p.epoch, kFlagInc, excl + total));
            }
            s_excl = excl;
            if (tile == num_tiles - 1) {
                uint32_t e = excl + total;
                p.fc->tile_entries = e < p.entry_cap ? e : p.entry_cap;
                p.fc->tile_overflow = e > p.entry_cap ? e - p.entry_cap : 0u;
                if (e > p.entry_cap) atomicOr(&p.fc->error_flags, kErrTileOverflow);
            }
        }
        __syncthreads();
        uint32_t o = s_excl + local;
        for (int ty = ty0; ty <= ty1; ++ty) {
            for (int tx = tx0; tx <= tx1; ++tx) {
                if (o < p.entry_cap) {
                    p.entry_keys[o] = (uint32_t)(ty * p.tiles_x + tx);
                    p.entry_vals[o] = s;
                }
                ++o;
            }
        }
        __syncthreads();
    }
}

__global__ void tile_ranges_kernel(const SortPlan* plan, const FrameCounters* fc, uint2* ranges,
                                   uint32_t num_tiles) {
    const uint32_t E = fc->tile_entries;
    const uint32_t* keys = plan->kfinal;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        uint32_t k = keys[e];
        if (k >= num_tiles) continue;  // only after a failed (timed-out) sort
        if (e == 0 || keys[e - 1] != k) ranges[k].x = e;
        if (e == E - 1 || keys[e + 1] != k) ranges[k].y = e + 1;
    }
}

int launch_bin(const BinParams& p, uint32_t n_cap, uint32_t num_sms, cudaStream_t s) {
    uint32_t tiles = (n_cap + kBinThreads - 1) / kBinThreads;
    uint32_t grid = num_sms * 4;
    if (grid > tiles) grid = tiles;
    if (grid == 0) grid = 1;
    bin_kernel<<<grid, kBinThreads, 0, s>>>(p);
    return 1;
}

int launch_tile_ranges(const SortPlan* tile_plan, const FrameCounters* fc, uint32_t entry_cap, uint2* ranges,
                       uint32_t num_tiles, uint32_t num_sms, cudaStream_t s) {
    uint32_t grid = (entry_cap + 255) / 256;
    if (grid > num_sms * 8) grid = num_sms * 8;
    if (grid == 0) grid = 1;
    tile_ranges_kernel<<<grid, 256, 0, s>>>(tile_plan, fc, ranges, num_tiles);
    return 1;
}

}  // namespace gs
