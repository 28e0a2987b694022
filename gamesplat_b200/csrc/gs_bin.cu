// Tile binning of depth-sorted splats for the tile rasterizer.
//
// The reference rasterizes one instanced quad per sorted splat through the GL
// pipeline (shaders/splat.glsl:39-75, src/renderer.cpp:1687-1720).  Here each
// sorted splat s (a) computes its covered pixel rectangle with the same quad
// geometry and fill rule as the CPU oracle (gs::quad_rect), (b) writes a
// 64-byte RasterRecord at position s, and (c) emits one (tile, s) entry per
// 16x16 tile that can receive a non-discarded fragment.  Entries are written
// in descending s order (nearest splat first) at offsets found by a
// decoupled look-back over CTA tiles, so a stable sort on the tile id alone
// leaves each tile's list in front-to-back order, the order the rasterizer
// walks.
//
// Two kernels: bin_kernel does (a) and (b), counts each splat's entries and
// finds the entry offsets; expand_kernel writes the entries, one chunk of the
// global entry range per CTA round (entry e finds its splat through an owner
// map: marks at each splat's first entry, then a block prefix maximum), so
// the work is balanced however many tiles one splat covers and the stores are
// coalesced; the tile ids' digit histograms for the tile sort are accumulated
// on the way.  Two more small kernels follow the tile sort: the [start, end)
// range of each tile, and the rasterization order (heaviest tiles first).
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
    bool ok;
    if (p.envelope) {
        // every quad of a jitter in [-0.5, 0.5]^2 lies inside the quad of
        // radius + 0.5 without jitter; a pixel more on each side absorbs the
        // snapping of the two rectangles' edges
        ok = quad_rect(cr.x, cr.y, add(cr.z, 0.5f), add(cr.w, 0.5f), cd.w, 0.0f, 0.0f, vp_w, vp_h, ysign, p.width,
                       p.height, &q);
        if (ok) {
            q.i0 = max(q.i0 - 1, 0);
            q.j0 = max(q.j0 - 1, 0);
            q.i1 = min(q.i1 + 1, p.width);
            q.j1 = min(q.j1 + 1, p.height);
        }
    } else {
        ok = quad_rect(cr.x, cr.y, cr.z, cr.w, cd.w, p.jitter_x, p.jitter_y, vp_w, vp_h, ysign, p.width, p.height, &q);
    }
    ok = ok && cutoff <= 0.0f;
    if (!ok) return it;
    const float ccx = add(cr.x, p.jitter_x), ccy = add(cr.y, p.jitter_y);
    PixelRect rc = q;
    // Bounding box of {d : conic(d) <= -2 cutoff}, widened by a pixel (and by
    // the jitter's half pixel in envelope mode).
    const float cx = cd.x, cy = cd.y, cz = cd.z;
    const float k = -2.0f * cutoff;
    const float dt = cx * cz - cy * cy;
    const float margin = p.envelope ? 1.5f : 1.0f;
    if (dt > 0.0f) {
        float hx = sqrtf(k * cz / dt) * 1.001f + margin;
        float hy = sqrtf(k * cx / dt) * 1.001f + margin;
        float fi0 = ceilf(ccx - hx - 0.5f), fi1 = floorf(ccx + hx - 0.5f);
        float fj0 = ceilf(ccy - hy - 0.5f), fj1 = floorf(ccy + hy - 0.5f);
        rc.i0 = max(rc.i0, (int)fmaxf(fi0, -1.0f));
        rc.i1 = min(rc.i1, (int)fminf(fi1, 32767.0f) + 1);
        rc.j0 = max(rc.j0, (int)fmaxf(fj0, -1.0f));
        rc.j1 = min(rc.j1, (int)fminf(fj1, 32767.0f) + 1);
    }
    if (rc.i0 >= rc.i1 || rc.j0 >= rc.j1) return it;
    it.tx0 = rc.i0 >> p.tile_shift_x;
    it.tx1 = (rc.i1 - 1) >> p.tile_shift_x;
    it.ty0 = rc.j0 >> p.tile_shift_y;
    it.ty1 = (rc.j1 - 1) >> p.tile_shift_y;
    it.count = (uint32_t)((it.tx1 - it.tx0 + 1) * (it.ty1 - it.ty0 + 1));
    RasterRecord rec;
    rec.cx = ccx;
    rec.cy = ccy;
    rec.conic_x = cd.x;
    rec.conic_2y = mul(2.0f, cd.y);
    rec.conic_z = cd.z;
    rec.log2_opacity = log2f(co.w);
    // cutoff <= 0 here; s_max = -2 cutoff is exact (cutoff is a normal float)
    rec.s_max = cutoff == 0.0f ? __int_as_float(1) : mul(-2.0f, cutoff);
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
    rec.opacity = co.w;
    if (p.envelope) {   // the rasterizer derives each sample's quad from these
        rec.cx = cr.x;
        rec.cy = cr.y;
        rec.log2_opacity = cr.z;
        rec.rect_x = __float_as_uint(cd.w);
        rec.rect_y = __float_as_uint(cr.w);
    }
    float4* dst = reinterpret_cast<float4*>(p.records + s);
    const float4* src = reinterpret_cast<const float4*>(&rec);
    dst[0] = src[0];
    dst[1] = src[1];
    dst[2] = src[2];
    dst[3] = src[3];
    return it;
}

// Per-item entry information for the expansion kernel (item q = CTA tile *
// kBinTile + position in the tile): global offset of its first entry, tile
// rectangle origin tx0 | ty0 << 16, and width in tiles (0 when it has no
// entries).

__global__ void __launch_bounds__(kBinThreads) bin_kernel(BinParams p) {
    pdl_wait();
    __shared__ uint32_t scan_tmp[33];
    __shared__ uint32_t s_tile, s_excl, s_total;
    __shared__ uint32_t s_off[kBinTile];    // exclusive entry offset of each splat in the CTA tile
    __shared__ uint32_t s_org[kBinTile];    // tx0 | ty0 << 16 of its tile rectangle
    __shared__ uint16_t s_w[kBinTile];      // its width in tiles (0: no entries)
    const uint32_t n_vis = p.fc->visible_count;
    const uint32_t num_tiles = (n_vis + kBinTile - 1) / kBinTile;
    const uint32_t* __restrict__ sorted_ids = p.depth_plan->vfinal;
    const float vp_w = p.vp_w, vp_h = p.vp_h, ysign = p.clip_y_sign;
    const int t = threadIdx.x;

    for (;;) {
        if (t == 0) s_tile = atomicAdd(&p.fc->bin_ticket, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= num_tiles) break;
        // CTA tile b holds sorted positions top - 1, top - 2, ..., down to
        // top - kBinTile (nearest splats first).
        const uint32_t top = n_vis - tile * kBinTile;
        const uint32_t cnt = min((uint32_t)kBinTile, top);
        // Splats striped over threads (coalesced id loads and record writes).
        uint32_t ids[kBinItems];
#pragma unroll
        for (int i = 0; i < kBinItems; ++i) {
            const uint32_t j = (uint32_t)(i * kBinThreads + t);
            ids[i] = j < cnt ? sorted_ids[top - 1u - j] : kSentinel;
        }
#pragma unroll
        for (int i = 0; i < kBinItems; ++i) {
            const uint32_t s = top - 1u - (uint32_t)(i * kBinThreads + t);
            const BinItem it = ids[i] != kSentinel ? bin_one(p, s, ids[i], vp_w, vp_h, ysign)
                                                   : BinItem{0u, 0, -1, 0, -1};
            const int slot = i * kBinThreads + t;
            s_off[slot] = it.count;
            s_org[slot] = it.count ? (uint32_t)it.tx0 | ((uint32_t)it.ty0 << 16) : 0u;
            s_w[slot] = it.count ? (uint16_t)(it.tx1 - it.tx0 + 1) : (uint16_t)0;
        }
        __syncthreads();
        // Exclusive scan of the counts in splat order (blocked: 4 per thread).
        uint32_t c[kBinItems], sum = 0;
#pragma unroll
        for (int k = 0; k < kBinItems; ++k) {
            c[k] = s_off[t * kBinItems + k];
            sum += c[k];
        }
        uint32_t total;
        uint32_t run = block_excl_scan(sum, scan_tmp, &total);
#pragma unroll
        for (int k = 0; k < kBinItems; ++k) {
            s_off[t * kBinItems + k] = run;
            run += c[k];
        }
        if (t < 32) {
            // warp 0: publish the tile count, resolve the prefix by a
            // warp-cooperative look-back, publish the inclusive prefix
            u64* st = p.status + tile;
            uint32_t excl = 0;
            if (tile == 0) {
                if (t == 0) st_relaxed64(st, status_word(p.epoch, kFlagInc, total));
            } else {
                if (t == 0) st_relaxed64(st, status_word(p.epoch, kFlagAgg, total));
                bool to = false;
                excl = lookback_warp(p.status, tile, p.epoch, &to);
                if (t == 0) {
                    if (to) atomicOr(&p.fc->error_flags, kErrBinLookback);
                    st_relaxed64(st, status_word(p.epoch, kFlagInc, excl + total));
                }
            }
            if (t == 0) {
                s_excl = excl;
                s_total = total;
                if (tile == num_tiles - 1) {
                    const uint32_t e = excl + total;
                    p.fc->tile_entries = e < p.entry_cap ? e : p.entry_cap;
                    p.fc->tile_overflow = e > p.entry_cap ? e - p.entry_cap : 0u;
                    if (e > p.entry_cap) atomicOr(&p.fc->error_flags, kErrTileOverflow);
                }
            }
        }
        __syncthreads();
        const uint32_t excl = s_excl, cta_total = s_total;
        // Per-item information for the expansion kernel (coalesced).
        for (int j = t; j < (int)cnt; j += kBinThreads)
            p.item_info[(size_t)tile * kBinTile + j] = make_uint4(excl + s_off[j], s_org[j], s_w[j], 0u);
        // Owner of every expansion chunk that starts inside this CTA tile: the
        // last item whose first entry is at or before the chunk start.
        if (cta_total) {
            const uint32_t c0 = (excl + kBinChunk - 1) / kBinChunk, c1 = (excl + cta_total - 1) / kBinChunk;
            for (uint32_t ch = c0 + t; ch <= c1; ch += kBinThreads) {
                if (ch >= p.chunk_cap) break;
                const uint32_t rel = ch * kBinChunk - excl;
                int lo = 0, hi = (int)cnt - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s_off[mid] <= rel) lo = mid;
                    else hi = mid - 1;
                }
                p.chunk_first[ch] = tile * kBinTile + (uint32_t)lo;
            }
        }
        __syncthreads();
    }
}

// Load-balanced expansion of the (tile id, sorted position) entries: chunk c
// covers entries [c * kBinChunk, (c + 1) * kBinChunk); its items run from
// chunk_first[c] to chunk_first[c + 1].  Each non-empty item marks its first
// entry with its index and a block-wide prefix maximum gives every entry its
// owner (the chunk's first entries belong to chunk_first[c]).  Entries are
// written in the order the binning defined, so the result is the same
// whichever CTA expands a chunk; the tile ids' digit histograms for the tile
// sort are accumulated here.
__global__ void __launch_bounds__(kBinThreads) expand_kernel(BinParams p) {
    pdl_wait();
    __shared__ uint32_t scan_tmp[33];
    __shared__ uint32_t s_hist[3][256];
    __shared__ __align__(16) int32_t s_own[kBinChunk];
    const int t = threadIdx.x;
    for (int i = t; i < 3 * 256; i += kBinThreads) (&s_hist[0][0])[i] = 0u;
    const uint32_t n_vis = p.fc->visible_count;
    const uint32_t entries = min(p.fc->tile_entries, p.entry_cap);
    const uint32_t nchunks = (entries + kBinChunk - 1) / kBinChunk;
    __syncthreads();
    for (uint32_t ch = blockIdx.x; ch < nchunks && ch < p.chunk_cap; ch += gridDim.x) {
        const uint32_t e0 = ch * kBinChunk, e1 = min(e0 + kBinChunk, entries);
        const uint32_t qa = p.chunk_first[ch];
        const uint32_t qb = (ch + 1 < nchunks && ch + 1 < p.chunk_cap) ? p.chunk_first[ch + 1] : n_vis - 1u;
        for (int i = t; i < kBinChunk; i += kBinThreads) s_own[i] = -1;
        __syncthreads();
        for (uint32_t q = qa + 1u + (uint32_t)t; q <= qb && q < n_vis; q += kBinThreads) {
            const uint4 inf = p.item_info[q];
            if (inf.z && inf.x >= e0 && inf.x < e1) s_own[inf.x - e0] = (int32_t)(q - qa);
        }
        __syncthreads();
        static_assert(kBinChunk == 8 * kBinThreads, "eight entries per thread in the prefix maximum");
        int4* own4 = reinterpret_cast<int4*>(s_own) + 2 * t;
        int4 a = own4[0], bq = own4[1];
        a.x = max(a.x, 0);   // entries before the first mark belong to item qa
        a.y = max(a.y, a.x);
        a.z = max(a.z, a.y);
        a.w = max(a.w, a.z);
        bq.x = max(bq.x, a.w);
        bq.y = max(bq.y, bq.x);
        bq.z = max(bq.z, bq.y);
        bq.w = max(bq.w, bq.z);
        const int32_t pre = max(block_excl_max(bq.w, reinterpret_cast<int32_t*>(scan_tmp)), 0);
        own4[0] = make_int4(max(a.x, pre), max(a.y, pre), max(a.z, pre), max(a.w, pre));
        own4[1] = make_int4(max(bq.x, pre), max(bq.y, pre), max(bq.z, pre), max(bq.w, pre));
        __syncthreads();
        // the owners' item records first (all in flight at once), then the entries
        static_assert(kBinChunk == 8 * kBinThreads, "eight entries per thread");
        const uint32_t ne = e1 - e0;
        uint4 infs[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const uint32_t i = (uint32_t)(t + r * kBinThreads);
            if (i < ne) infs[r] = __ldg(p.item_info + qa + (uint32_t)s_own[i]);
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const uint32_t i = (uint32_t)(t + r * kBinThreads);
            if (i >= ne) break;
            const uint32_t q = qa + (uint32_t)s_own[i];
            const uint4 inf = infs[r];
            const uint32_t k = e0 + i - inf.x;
            const uint32_t w = max(inf.z, 1u);
            const uint32_t ty = (inf.y >> 16) + k / w, tx = (inf.y & 0xFFFFu) + k % w;
            const uint32_t tid = ty * (uint32_t)p.tiles_x + tx;
            p.entry_keys[e0 + i] = tid;
            p.entry_vals[e0 + i] = n_vis - 1u - q;
            atomicAdd(&s_hist[0][tid & 255u], 1u);
            atomicAdd(&s_hist[1][(tid >> 8) & 255u], 1u);
            atomicAdd(&s_hist[2][(tid >> 16) & 255u], 1u);
        }
        __syncthreads();
    }
    __syncthreads();
    for (int i = t; i < 3 * 256; i += kBinThreads) {
        const uint32_t c = (&s_hist[0][0])[i];
        if (c) atomicAdd(p.tile_hist + i, c);
    }
}

// [start, end) of every tile's run in the tile-sorted entries: a thread
// takes 8 consecutive keys (two 16-byte loads) and the keys either side.
__global__ void tile_ranges_kernel(const SortPlan* plan, const FrameCounters* fc, uint2* ranges,
                                   uint32_t num_tiles) {
    pdl_wait();
    pdl_trigger();
    const uint32_t E = fc->tile_entries;
    const uint32_t* keys = plan->kfinal;
    const uint32_t groups = (E + 7) / 8;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x) {
        const uint32_t e0 = g * 8;
        uint32_t k[10];   // k[0] = key e0 - 1, k[1..8] = keys e0..e0+7, k[9] = key e0 + 8
        k[0] = e0 > 0 ? keys[e0 - 1] : 0xFFFFFFFFu;
        if (e0 + 8 <= E) {
            const uint4 a = reinterpret_cast<const uint4*>(keys + e0)[0];
            const uint4 b = reinterpret_cast<const uint4*>(keys + e0)[1];
            k[1] = a.x; k[2] = a.y; k[3] = a.z; k[4] = a.w;
            k[5] = b.x; k[6] = b.y; k[7] = b.z; k[8] = b.w;
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) k[1 + j] = e0 + j < E ? keys[e0 + j] : 0xFFFFFFFFu;
        }
        k[9] = e0 + 8 < E ? keys[e0 + 8] : 0xFFFFFFFFu;
#pragma unroll
        for (int j = 1; j <= 8; ++j) {
            const uint32_t e = e0 + (uint32_t)(j - 1);
            if (e >= E || k[j] >= num_tiles) continue;   // >= num_tiles only after a failed (timed-out) sort
            if (e == 0 || k[j - 1] != k[j]) ranges[k[j]].x = e;
            if (e == E - 1 || k[j + 1] != k[j]) ranges[k[j]].y = e + 1;
        }
    }
}

// Rasterization order: tiles by descending entry count (quarter-octave
// classes), so the heaviest tiles start in the first wave instead of
// stretching the last one.  One CTA; the order within a class is immaterial
// (each tile's CTA writes only its own pixels).
__global__ void __launch_bounds__(1024) tile_order_kernel(const uint2* __restrict__ ranges, uint32_t num_tiles,
                                                          uint32_t* __restrict__ order) {
    pdl_wait();
    pdl_trigger();
    __shared__ uint32_t s_cnt[129], s_start[129];
    const int t = threadIdx.x;
    if (t < 129) s_cnt[t] = 0u;
    __syncthreads();
    auto cls = [&](uint32_t tl) -> uint32_t {   // quarter-octave classes, heaviest first
        const uint2 r = ranges[tl];
        const uint32_t w = r.y > r.x ? r.y - r.x : 0u;
        if (!w) return 128u;
        const uint32_t lz = (uint32_t)__clz(w);
        const uint32_t frac = lz >= 30 ? 0u : (w << (lz + 1)) >> 30;   // two bits after the leading one
        return lz * 4u + (3u - frac);
    };
    for (uint32_t tl = t; tl < num_tiles; tl += blockDim.x) atomicAdd(&s_cnt[cls(tl)], 1u);
    __syncthreads();
    if (t == 0) {
        uint32_t run = 0;
        for (int k = 0; k < 129; ++k) {
            s_start[k] = run;
            run += s_cnt[k];
        }
    }
    __syncthreads();
    for (uint32_t tl = t; tl < num_tiles; tl += blockDim.x) order[atomicAdd(&s_start[cls(tl)], 1u)] = tl;
}

int launch_tile_order(const uint2* ranges, uint32_t num_tiles, uint32_t* order, cudaStream_t s) {
    if (num_tiles == 0) return 0;
    // programmatic dependent launch (as the ranges and the raster after it): the kernel is scheduled while its
    // predecessor drains and waits for it (griddepcontrol.wait) before it reads anything
    launch_pdl(tile_order_kernel, dim3(1), dim3(1024), 0, s, ranges, num_tiles, order);
    return 1;
}

int launch_bin(const BinParams& p, uint32_t n_cap, uint32_t num_sms, cudaStream_t s) {
    uint32_t tiles = (n_cap + kBinTile - 1) / kBinTile;
    uint32_t grid = num_sms * (1024 / kBinThreads);
    if (grid > tiles) grid = tiles;
    if (grid == 0) grid = 1;
    launch_pdl(bin_kernel, dim3(grid), dim3(kBinThreads), 0, s, p);
    launch_pdl(expand_kernel, dim3(num_sms * (1024 / kBinThreads)), dim3(kBinThreads), 0, s, p);
    return 2;
}

int launch_tile_ranges(const SortPlan* tile_plan, const FrameCounters* fc, uint32_t entry_cap, uint2* ranges,
                       uint32_t num_tiles, uint32_t num_sms, cudaStream_t s) {
    uint32_t grid = (entry_cap / 8 + 255) / 256;
    if (grid > num_sms * 8) grid = num_sms * 8;
    if (grid == 0) grid = 1;
    launch_pdl(tile_ranges_kernel, dim3(grid), dim3(256), 0, s, tile_plan, (const FrameCounters*)fc, ranges, num_tiles);
    return 1;
}

}  // namespace gs
