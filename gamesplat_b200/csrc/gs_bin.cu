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

struct BinItem {
    uint32_t count;
    int tx0, tx1, ty0, ty1;
};

// One sorted splat: raster record + the range of tiles it can touch.
__device__ __forceinline__ BinItem bin_one(const BinParams& p, uint32_t s, uint32_t id, float vp_w, float vp_h,
                                           float ysign) {
    BinItem it = {0u, 0, -1, 0, -1};
    const float4* P = p.projected + (size_t)id * 4;
    const float4 co = P[0], cr = P[1], cd = P[2];
    PixelRect q;
    const float cutoff = alpha_cutoff(co.w);
    bool ok = quad_rect(cr.x, cr.y, cr.z, cr.w, cd.w, p.jitter_x, p.jitter_y, vp_w, vp_h, ysign, p.width, p.height,
                        &q);
    ok = ok && cutoff <= 0.0f;
    if (!ok) return it;
    const float ccx = add(cr.x, p.jitter_x), ccy = add(cr.y, p.jitter_y);
    PixelRect rc = q;
    // Bounding box of {d : conic(d) <= -2 cutoff}, widened by a pixel.
    const float cx = cd.x, cy = cd.y, cz = cd.z;
    const float k = -2.0f * cutoff;
    const float dt = cx * cz - cy * cy;
    if (dt > 0.0f) {
        float hx = sqrtf(k * cz / dt) * 1.001f + 1.0f;
        float hy = sqrtf(k * cx / dt) * 1.001f + 1.0f;
        float fi0 = ceilf(ccx - hx - 0.5f), fi1 = floorf(ccx + hx - 0.5f);
        float fj0 = ceilf(ccy - hy - 0.5f), fj1 = floorf(ccy + hy - 0.5f);
        rc.i0 = max(rc.i0, (int)fmaxf(fi0, -1.0f));
        rc.i1 = min(rc.i1, (int)fminf(fi1, 32767.0f) + 1);
        rc.j0 = max(rc.j0, (int)fmaxf(fj0, -1.0f));
        rc.j1 = min(rc.j1, (int)fminf(fj1, 32767.0f) + 1);
    }
    if (rc.i0 >= rc.i1 || rc.j0 >= rc.j1) return it;
    it.tx0 = rc.i0 / kTileW;
    it.tx1 = (rc.i1 - 1) / kTileW;
    it.ty0 = rc.j0 / kTileH;
    it.ty1 = (rc.j1 - 1) / kTileH;
    it.count = (uint32_t)((it.tx1 - it.tx0 + 1) * (it.ty1 - it.ty0 + 1));
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
    // Quad coverage intersected with the alpha-ellipse box: every pixel the
    // box drops has power < cutoff and is discarded anyway, so the
    // rasterizer's per-pixel result is unchanged.
    rec.rect_x = (uint32_t)rc.i0 | ((uint32_t)rc.i1 << 16);
    rec.rect_y = (uint32_t)rc.j0 | ((uint32_t)rc.j1 << 16);
    const float zw = add(mul(cd.w, 0.5f), 0.5f);
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
    return it;
}

__device__ __forceinline__ void emit(const BinParams& p, uint32_t o, uint32_t s, int tx0, int tx1, int ty0, int ty1,
                                     uint32_t first, uint32_t step) {
    const int w = tx1 - tx0 + 1;
    const uint32_t cnt = (uint32_t)(w * (ty1 - ty0 + 1));
    for (uint32_t k = first; k < cnt; k += step) {
        const uint32_t e = o + k;
        if (e < p.entry_cap) {
            const int ty = ty0 + (int)(k / (uint32_t)w), tx = tx0 + (int)(k % (uint32_t)w);
            const uint32_t t = (uint32_t)(ty * p.tiles_x + tx);
            p.entry_keys[e] = t;
            p.entry_vals[e] = s;
            atomicAdd(&p.tile_count[t], 1u);
        }
    }
}

__global__ void __launch_bounds__(kBinThreads) bin_kernel(BinParams p) {
    __shared__ uint32_t scan_tmp[33];
    __shared__ uint32_t s_tile, s_excl;
    const uint32_t n_vis = p.fc->visible_count;
    const uint32_t num_tiles = (n_vis + kBinTile - 1) / kBinTile;
    const uint32_t* __restrict__ sorted_ids = p.depth_plan->vfinal;
    const float* camf = reinterpret_cast<const float*>(p.cam);
    const float vp_w = __ldg(camf + 32), vp_h = __ldg(camf + 33), ysign = __ldg(camf + 37);
    const int lane = threadIdx.x & 31;

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&p.fc->bin_ticket, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= num_tiles) break;
        // Items are blocked per thread (s = base + 4t + i) so that each
        // thread's entries are contiguous and in s order.
        const uint32_t sbase = tile * kBinTile + threadIdx.x * kBinItems;
        uint32_t ids[kBinItems];
#pragma unroll
        for (int i = 0; i < kBinItems; ++i) ids[i] = sbase + i < n_vis ? sorted_ids[sbase + i] : kSentinel;
        BinItem it[kBinItems];
        uint32_t count = 0;
#pragma unroll
        for (int i = 0; i < kBinItems; ++i) {
            it[i] = ids[i] != kSentinel ? bin_one(p, sbase + i, ids[i], vp_w, vp_h, ysign)
                                        : BinItem{0u, 0, -1, 0, -1};
            count += it[i].count;
        }
        uint32_t total;
        const uint32_t local = block_excl_scan(count, scan_tmp, &total);
        if (threadIdx.x < 32) {
            // warp 0: publish the tile count, resolve the prefix by a
            // warp-cooperative look-back, publish the inclusive prefix
            u64* st = p.status + tile;
            uint32_t excl = 0;
            if (tile == 0) {
                if (threadIdx.x == 0) st_release64(st, status_word(p.epoch, kFlagInc, total));
            } else {
                if (threadIdx.x == 0) st_release64(st, status_word(p.epoch, kFlagAgg, total));
                bool to = false;
                excl = lookback_warp(p.status, tile, p.epoch, &to);
                if (threadIdx.x == 0) {
                    if (to) atomicOr(&p.fc->error_flags, kErrBinLookback);
                    st_release64(st, status_word(p.epoch, kFlagInc, excl + total));
                }
            }
            if (threadIdx.x == 0) {
                s_excl = excl;
                if (tile == num_tiles - 1) {
                    const uint32_t e = excl + total;
                    p.fc->tile_entries = e < p.entry_cap ? e : p.entry_cap;
                    p.fc->tile_overflow = e > p.entry_cap ? e - p.entry_cap : 0u;
                    if (e > p.entry_cap) atomicOr(&p.fc->error_flags, kErrTileOverflow);
                }
            }
        }
        __syncthreads();
        // Entries: small splats by their own thread, splats covering many
        // tiles by the whole warp.
        uint32_t o = s_excl + local;
        constexpr uint32_t kBig = 8;
#pragma unroll
        for (int i = 0; i < kBinItems; ++i) {
            const bool big = it[i].count > kBig;
            if (!big && it[i].count) emit(p, o, sbase + i, it[i].tx0, it[i].tx1, it[i].ty0, it[i].ty1, 0u, 1u);
            uint32_t bigmask = __ballot_sync(0xffffffffu, big);
            while (bigmask) {
                const int l = __ffs(bigmask) - 1;
                bigmask &= bigmask - 1;
                const uint32_t lo = __shfl_sync(0xffffffffu, o, l);
                const uint32_t ls = __shfl_sync(0xffffffffu, sbase + i, l);
                const int a = __shfl_sync(0xffffffffu, it[i].tx0, l), b = __shfl_sync(0xffffffffu, it[i].tx1, l);
                const int c = __shfl_sync(0xffffffffu, it[i].ty0, l), d = __shfl_sync(0xffffffffu, it[i].ty1, l);
                emit(p, lo, ls, a, b, c, d, (uint32_t)lane, 32u);
            }
            o += it[i].count;
        }
        __syncthreads();
    }
}

// From the per-tile entry counts (one CTA): each tile's [start, end) in the
// tile-sorted entry array (exclusive scan over tiles) and the digit
// histograms of the tile-sort passes.  After an entry-buffer overflow the
// frame is invalid: every range is left empty.
constexpr int kPlanThreads = 1024;
__global__ void __launch_bounds__(kPlanThreads) tile_plan_kernel(const uint32_t* __restrict__ tile_count,
                                                                 uint32_t num_tiles, int npasses,
                                                                 const FrameCounters* fc, uint2* ranges,
                                                                 uint32_t* tile_hist) {
    __shared__ uint32_t s_hist[4][256];
    __shared__ uint32_t warp_tmp[33];
    for (int i = threadIdx.x; i < 4 * 256; i += kPlanThreads) (&s_hist[0][0])[i] = 0u;
    __syncthreads();
    const bool overflow = fc->tile_overflow != 0u;
    const uint32_t per = (num_tiles + kPlanThreads - 1) / kPlanThreads;
    const uint32_t t0 = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t t = t0; t < t0 + per && t < num_tiles; ++t) {
        const uint32_t c = tile_count[t];
        sum += c;
        for (int ps = 0; ps < npasses; ++ps)
            if (c) atomicAdd(&s_hist[ps][(t >> (8 * ps)) & 255u], c);
    }
    uint32_t total;
    uint32_t run = block_excl_scan(sum, warp_tmp, &total);
    for (uint32_t t = t0; t < t0 + per && t < num_tiles; ++t) {
        const uint32_t c = tile_count[t];
        ranges[t] = overflow ? make_uint2(0u, 0u) : make_uint2(run, run + c);
        run += c;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * 256; i += kPlanThreads) tile_hist[i] = (&s_hist[0][0])[i];
}

int launch_bin(const BinParams& p, uint32_t n_cap, uint32_t num_sms, cudaStream_t s) {
    uint32_t tiles = (n_cap + kBinTile - 1) / kBinTile;
    uint32_t grid = num_sms * 4;
    if (grid > tiles) grid = tiles;
    if (grid == 0) grid = 1;
    bin_kernel<<<grid, kBinThreads, 0, s>>>(p);
    return 1;
}

int launch_tile_plan(const uint32_t* tile_count, uint32_t num_tiles, int tile_bits, const FrameCounters* fc,
                     uint2* ranges, uint32_t* tile_hist, cudaStream_t s) {
    const int npasses = (tile_bits + 7) / 8;
    tile_plan_kernel<<<1, kPlanThreads, 0, s>>>(tile_count, num_tiles, npasses, fc, ranges, tile_hist);
    return 1;
}

}  // namespace gs
