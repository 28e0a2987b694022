// Onesweep LSD radix sort of (uint32 key, uint32 value) pairs for the B200.
//
// Same result as the reference's 4 x (histogram, single-workgroup prefix,
// bitmask-rank scatter) passes (shaders/sort.glsl:26-163,
// src/renderer.cpp:1873-1962): a stable ascending sort, equal keys in input
// order.  Structure:
//   1. sort_hist_kernel   - one read of the keys builds the digit histograms
//                           of every pass (warp-private shared histograms);
//      (skipped when the producer of the keys already accumulated them);
//   2. sort_pass_kernel   - every CTA derives the pass plan from the
//                           histograms (passes whose digit is the same for all
//                           keys are skipped: identity for a stable sort;
//                           ping-pong assignment of the active passes), then
//                           persistent CTAs (3 per SM) take 4096-key tiles in
//                           ticket order, copy the tile's values into shared
//                           memory (cp.async: registers hold only keys and
//                           ranks, which is what lets 3 CTAs share an SM),
//                           rank keys within each warp (lanes
//                           of equal digit found by per-bit ballots), publish
//                           per-digit counts,
//                           reorder the tile by digit in shared memory, then
//                           resolve their global offsets by decoupled
//                           look-back (bounded spin) and write runs coalesced;
//   3. sort_copy_kernel   - only when the caller needs the result in a given
//                           buffer and every pass was skipped.
// Element counts are read on the device, so nothing here synchronises with
// the host.
#include "gs_common.cuh"
#include "gs_internal.h"
#include "gs_tma.cuh"

namespace gs {

constexpr int kSortWarps = kSortThreads / 32;
static_assert(kSortThreads == kRadix, "one thread per digit in the pass kernel");

int sort_passes(int begin_bit, int end_bit) { return (end_bit - begin_bit + kRadixBits - 1) / kRadixBits; }

size_t sort_status_words(uint32_t count_cap) {
    size_t tiles = ((size_t)count_cap + kSortTile - 1) / kSortTile;
    if (tiles == 0) tiles = 1;
    return tiles * kRadix;
}

// Asynchronous global -> shared copies of 4 and 16 bytes (zero-filled past src_bytes).
__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

// Dynamic shared memory of the pass kernel: the reordered keys and values and
// the tile's values in input order.
constexpr int kPassSmem = 3 * kSortTile * 4;

__device__ __forceinline__ uint32_t digit_of(uint32_t key, int shift, uint32_t dmask) { return (key >> shift) & dmask; }

__global__ void __launch_bounds__(kSortThreads) sort_hist_kernel(SortParams p, int npasses) {
    __shared__ uint32_t wh[kSortWarps][4][kRadix];  // warp-private histograms, 32 KB
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * 4 * kRadix; i += kSortThreads) (&wh[0][0][0])[i] = 0u;
    __syncthreads();
    const uint32_t n = p.count_ptr ? *p.count_ptr : p.count_cap;
    const uint32_t stride = gridDim.x * blockDim.x;
    // Vector loads only when the caller's key pointer is 16-byte aligned.
    const uint32_t n4 = (((uintptr_t)p.keys_in & 15u) == 0u) ? (n >> 2) : 0u;
    const uint4* k4 = reinterpret_cast<const uint4*>(p.keys_in);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        uint4 k = __ldg(k4 + i);
        for (int ps = 0; ps < npasses; ++ps) {
            int shift = p.begin_bit + ps * kRadixBits;
            uint32_t dmask = (1u << min(kRadixBits, p.end_bit - shift)) - 1u;
            atomicAdd(&wh[warp][ps][digit_of(k.x, shift, dmask)], 1u);
            atomicAdd(&wh[warp][ps][digit_of(k.y, shift, dmask)], 1u);
            atomicAdd(&wh[warp][ps][digit_of(k.z, shift, dmask)], 1u);
            atomicAdd(&wh[warp][ps][digit_of(k.w, shift, dmask)], 1u);
        }
    }
    for (uint32_t i = (n4 << 2) + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t k = __ldg(p.keys_in + i);
        for (int ps = 0; ps < npasses; ++ps) {
            int shift = p.begin_bit + ps * kRadixBits;
            uint32_t dmask = (1u << min(kRadixBits, p.end_bit - shift)) - 1u;
            atomicAdd(&wh[warp][ps][digit_of(k, shift, dmask)], 1u);
        }
    }
    __syncthreads();
    for (int ps = 0; ps < npasses; ++ps) {
        uint32_t sum = 0;
        for (int w = 0; w < kSortWarps; ++w) sum += wh[w][ps][threadIdx.x];
        if (sum) atomicAdd(&p.hist[ps * kRadix + threadIdx.x], sum);
    }
}

// Pass plan, recomputed by every CTA of every pass kernel from the digit
// histograms: a pass is skipped when one digit holds every key (a stable sort
// by a constant digit is the identity); active passes ping-pong between the
// writable buffers (with land_in_buf0 the last one writes buffer 0).
struct PassIO {
    const uint32_t* kin;
    const uint32_t* vin;
    uint32_t* kout;
    uint32_t* vout;
    const uint32_t* kfinal;
    const uint32_t* vfinal;
    bool active;
    bool copy_needed;
};

__device__ PassIO plan_passes(const SortParams& p, int npasses, int pass, uint32_t n, uint32_t* s_act) {
    for (int ps = 0; ps < npasses; ++ps) {
        const int trivial = __syncthreads_or(p.hist[ps * kRadix + threadIdx.x] == n);
        if (threadIdx.x == 0) s_act[ps] = trivial ? 0u : 1u;
    }
    __syncthreads();
    int m = 0;
    for (int ps = 0; ps < npasses; ++ps) m += (int)s_act[ps];
    PassIO io{};
    const uint32_t* kcur = p.keys_in;
    const uint32_t* vcur = p.vals_in;
    int j = 0;
    for (int ps = 0; ps < npasses; ++ps) {
        if (!s_act[ps]) continue;
        const int dst = p.land_in_buf0 ? ((m - 1 - j) & 1) : (j & 1);
        if (ps == pass) {
            io.kin = kcur;
            io.vin = vcur;
            io.kout = p.keys_buf[dst];
            io.vout = p.vals_buf[dst];
        }
        kcur = p.keys_buf[dst];
        vcur = p.vals_buf[dst];
        ++j;
    }
    io.active = s_act[pass] != 0u;
    io.copy_needed = p.land_in_buf0 && m == 0;
    io.kfinal = io.copy_needed ? p.keys_buf[0] : kcur;
    io.vfinal = io.copy_needed ? p.vals_buf[0] : vcur;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        SortPlan* pl = p.plan;
        for (int ps = 0; ps < 4; ++ps) pl->active[ps] = ps < npasses ? s_act[ps] : 0u;
        pl->kfinal = io.kfinal;
        pl->vfinal = io.vfinal;
        pl->copy_needed = io.copy_needed ? 1u : 0u;
        pl->count = n;
    }
    return io;
}

__global__ void __launch_bounds__(kSortThreads, 3) sort_pass_kernel(SortParams p, int pass, int npasses) {
    pdl_wait();
    pdl_trigger();
    extern __shared__ __align__(16) uint32_t s_dyn[];
    uint32_t* s_keys = s_dyn;                    // the tile reordered by digit
    uint32_t* s_vals = s_dyn + kSortTile;
    uint32_t* s_vstage = s_dyn + 2 * kSortTile;  // the tile's values in input order
    __shared__ uint32_t warp_hist[kSortWarps][kRadix];
    __shared__ uint32_t s_global_base[kRadix];
    __shared__ uint32_t scan_tmp[33];
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_act[4];

    const uint32_t n = p.count_ptr ? *p.count_ptr : p.count_cap;
    const PassIO io = plan_passes(p, npasses, pass, n, s_act);
    if (!io.active) return;
    const uint32_t* __restrict__ kin = io.kin;
    const uint32_t* __restrict__ vin = io.vin;
    uint32_t* __restrict__ kout = io.kout;
    uint32_t* __restrict__ vout = io.vout;
    const int shift = p.begin_bit + pass * kRadixBits;
    const int nbits = min(kRadixBits, p.end_bit - shift);
    const uint32_t dmask = (1u << nbits) - 1u;
    u64* status = p.status + (size_t)pass * p.status_stride;
    const uint32_t num_tiles = (n + kSortTile - 1) / kSortTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    // global start of this thread's digit (exclusive scan of the histogram)
    uint32_t digit_total;
    const uint32_t gdigit = block_excl_scan(p.hist[pass * kRadix + threadIdx.x], scan_tmp, &digit_total);

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&p.plan->ticket[pass], 1u);
        for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&warp_hist[0][0])[i] = 0u;
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= num_tiles) break;
        const uint32_t base = tile * kSortTile;
        const uint32_t wbase = base + warp * (kSortItems * 32);

        uint32_t key[kSortItems], rank[kSortItems];
        // The warp's 512 values go to shared memory in input order (item k of
        // lane l at k * 32 + l), 16 bytes per copy when the values are
        // 16-byte aligned; they are read once, at the reorder.
        uint32_t* vst = s_vstage + warp * (kSortItems * 32);
        if ((reinterpret_cast<uintptr_t>(vin) & 15u) == 0u) {
#pragma unroll
            for (int q = 0; q < kSortItems / 4; ++q) {
                const uint32_t e = (uint32_t)(q * 128 + lane * 4);
                const uint32_t idx = wbase + e;
                const uint32_t left = idx < n ? min(n - idx, 4u) : 0u;
                cp_async16(vst + e, left ? vin + idx : vin, left * 4u);
            }
        } else {
#pragma unroll
            for (int k = 0; k < kSortItems; ++k) {
                const uint32_t idx = wbase + k * 32 + lane;
                cp_async4(vst + k * 32 + lane, idx < n ? vin + idx : vin, idx < n ? 4u : 0u);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
#pragma unroll
        for (int k = 0; k < kSortItems; ++k) {
            uint32_t idx = wbase + k * 32 + lane;
            key[k] = idx < n ? kin[idx] : 0u;
        }
        // Warp ranking in index order (item k, then lane): the lanes holding a
        // digit find each other; their leader reads and advances the warp's
        // running count of that digit.
#pragma unroll
        for (int k = 0; k < kSortItems; ++k) {
            uint32_t idx = wbase + k * 32 + lane;
            uint32_t d = (idx < n) ? digit_of(key[k], shift, dmask) : (uint32_t)kRadix;
            // Lanes with the same digit: one ballot per digit bit (plus one
            // for validity).  Measured faster than __match_any_sync here.
            const bool valid = d < (uint32_t)kRadix;
            const uint32_t vb = __ballot_sync(0xffffffffu, valid);
            uint32_t peers = valid ? vb : ~vb;
#pragma unroll
            for (int bit = 0; bit < kRadixBits; ++bit) {
                if (bit < nbits) {
                    const uint32_t bb = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
                    peers &= ((d >> bit) & 1u) ? bb : ~bb;
                }
            }
            int leader = __ffs(peers) - 1;
            uint32_t before = 0;
            if (lane == leader && d < (uint32_t)kRadix) {
                before = warp_hist[warp][d];
                warp_hist[warp][d] = before + __popc(peers);
            }
            before = __shfl_sync(0xffffffffu, before, leader);
            rank[k] = before + __popc(peers & lt_mask);
            __syncwarp();
        }
        asm volatile("cp.async.wait_all;" ::: "memory");   // this thread's value copies
        __syncthreads();                                      // ... and every other thread's
        // One thread per digit: tile count, published at once; then every
        // warp's start of the digit's run in the reordered tile.
        const uint32_t d = threadIdx.x;
        uint32_t c[kSortWarps], tile_count = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            c[w] = warp_hist[w][d];
            tile_count += c[w];
        }
        u64* st = status + (size_t)tile * kRadix + d;
        if (tile == 0) st_relaxed64(st, status_word(p.epoch, kFlagInc, gdigit + tile_count));
        else st_relaxed64(st, status_word(p.epoch, kFlagAgg, tile_count));
        uint32_t total;
        const uint32_t lstart = block_excl_scan(tile_count, scan_tmp, &total);
        uint32_t run = lstart;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            warp_hist[w][d] = run;
            run += c[w];
        }
        __syncthreads();
        // Reorder the tile by digit in shared memory while predecessors publish.
#pragma unroll
        for (int k = 0; k < kSortItems; ++k) {
            uint32_t idx = wbase + k * 32 + lane;
            if (idx < n) {
                const uint32_t lp = warp_hist[warp][digit_of(key[k], shift, dmask)] + rank[k];
                s_keys[lp] = key[k];
                s_vals[lp] = vst[k * 32 + lane];
            }
        }
        // Global offset of each digit's run: decoupled look-back.
        uint32_t gexcl = gdigit;
        if (tile > 0) {
            bool to = false;
            gexcl = lookback_vec<kSortLookback>(status + d, kRadix, tile, p.epoch, &to);
            if (to) atomicOr(p.error_flags, kErrSortLookback);
            st_relaxed64(st, status_word(p.epoch, kFlagInc, gexcl + tile_count));
        }
        s_global_base[d] = gexcl - lstart;
        __syncthreads();
        const uint32_t nvalid = min((uint32_t)kSortTile, n - base);
        for (uint32_t i = threadIdx.x; i < nvalid; i += kSortThreads) {
            const uint32_t k = s_keys[i];
            const uint32_t o = s_global_base[digit_of(k, shift, dmask)] + i;
            if (o < n) {  // always true unless a look-back wait ran out
                kout[o] = k;
                vout[o] = s_vals[i];
            }
        }
        __syncthreads();
    }
}

__global__ void sort_copy_kernel(SortParams p) {
    pdl_wait();
    pdl_trigger();
    const SortPlan* pl = p.plan;
    if (!pl->copy_needed) return;
    const uint32_t n = pl->count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        p.keys_buf[0][i] = p.keys_in[i];
        p.vals_buf[0][i] = p.vals_in[i];
    }
}

// Per device: the pass kernel's shared-memory opt-in, then its occupancy.
constexpr int kMaxDevices = 64;
static int g_pass_blocks_per_sm[kMaxDevices] = {};

int launch_sort(const SortParams& p, uint32_t num_sms, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    int& blocks_per_sm = g_pass_blocks_per_sm[dev >= 0 && dev < kMaxDevices ? dev : 0];
    if (blocks_per_sm == 0 || dev >= kMaxDevices) {
        cudaFuncSetAttribute(sort_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPassSmem);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, sort_pass_kernel, kSortThreads, kPassSmem);
        blocks_per_sm = b > 0 ? b : 1;
    }
    const int npasses = sort_passes(p.begin_bit, p.end_bit);
    int launches = 0;
    uint32_t tiles_cap = (p.count_cap + kSortTile - 1) / kSortTile;
    if (!p.hist_ready) {
        uint32_t hist_grid = num_sms * 2;
        uint32_t hist_need = (p.count_cap / 4 + kSortThreads - 1) / kSortThreads;
        if (hist_grid > hist_need) hist_grid = hist_need > 0 ? hist_need : 1;
        sort_hist_kernel<<<hist_grid, kSortThreads, 0, s>>>(p, npasses);
        ++launches;
    }
    uint32_t pass_grid = num_sms * (uint32_t)blocks_per_sm;
    if (pass_grid > tiles_cap) pass_grid = tiles_cap > 0 ? tiles_cap : 1;
    for (int ps = 0; ps < npasses; ++ps) {
        // Passes after the first overlap their launch with the previous pass's
        // tail (programmatic dependent launch); so does the first pass when the
        // caller asks (the frame's sorts: every kernel of a frame starts with
        // griddepcontrol.wait).  The stage-level entry points launch it
        // ordinarily behind the caller's work.
        if (ps == 0 && !p.first_pdl) sort_pass_kernel<<<pass_grid, kSortThreads, kPassSmem, s>>>(p, ps, npasses);
        else launch_pdl(sort_pass_kernel, dim3(pass_grid), dim3(kSortThreads), kPassSmem, s, p, ps, npasses);
        ++launches;
    }
    if (p.land_in_buf0) {
        uint32_t g = (p.count_cap + 1023) / 1024;
        if (g > num_sms * 4) g = num_sms * 4;
        if (g == 0) g = 1;
        launch_pdl(sort_copy_kernel, dim3(g), dim3(256), 0, s, p);
        ++launches;
    }
    return launches;
}

}  // namespace gs

// ---------------------------------------------------------------------------
// Stage-level C entry point: sort caller-owned device buffers.
// Scratch layout: SortPlan | 4x256 histograms | error word | 4 passes of
// look-back words | temporary keys | temporary values (256-byte aligned).
// ---------------------------------------------------------------------------
namespace {
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
struct SortScratch {
    size_t plan, hist, err, status, tkeys, tvals, total, control_bytes;
};
SortScratch sort_scratch_layout(uint32_t n) {
    SortScratch l{};
    size_t off = 0;
    l.plan = off; off += align256(sizeof(gs::SortPlan));
    l.hist = off; off += align256(4 * 256 * 4);
    l.err = off; off += align256(4);
    l.status = off; off += align256(gs::sort_status_words(n) * 4 * sizeof(unsigned long long));
    l.control_bytes = off;
    l.tkeys = off; off += align256((size_t)n * 4);
    l.tvals = off; off += align256((size_t)n * 4);
    l.total = off;
    return l;
}
}  // namespace

extern "C" size_t gs_sort_pairs_scratch_bytes(uint32_t n) { return sort_scratch_layout(n).total; }

extern "C" int gs_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                             uint32_t n, int begin_bit, int end_bit, void* scratch, size_t scratch_bytes,
                             void* stream) {
    if (begin_bit < 0 || end_bit > 32 || end_bit <= begin_bit) return GS_ERR_BAD_ARG;
    if (n == 0) return GS_OK;
    if (n > (1u << 30) - 1) return GS_ERR_TOO_LARGE;
    if (!keys_in || !vals_in || !keys_out || !vals_out || !scratch) return GS_ERR_BAD_ARG;
    if ((const void*)keys_in == (const void*)keys_out || (const void*)vals_in == (const void*)vals_out)
        return GS_ERR_BAD_ARG;
    const SortScratch l = sort_scratch_layout(n);
    if (scratch_bytes < l.total) return GS_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(scratch);
    if (cudaMemsetAsync(base, 0, l.control_bytes, s) != cudaSuccess) return GS_ERR_CUDA;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    gs::SortParams p{};
    p.keys_in = keys_in;
    p.vals_in = vals_in;
    p.keys_buf[0] = keys_out;
    p.vals_buf[0] = vals_out;
    p.keys_buf[1] = reinterpret_cast<uint32_t*>(base + l.tkeys);
    p.vals_buf[1] = reinterpret_cast<uint32_t*>(base + l.tvals);
    p.land_in_buf0 = 1;
    p.count_ptr = nullptr;
    p.count_cap = n;
    p.begin_bit = begin_bit;
    p.end_bit = end_bit;
    p.hist = reinterpret_cast<uint32_t*>(base + l.hist);
    p.plan = reinterpret_cast<gs::SortPlan*>(base + l.plan);
    p.status = reinterpret_cast<unsigned long long*>(base + l.status);
    p.status_stride = gs::sort_status_words(n);
    p.epoch = 1;
    p.error_flags = reinterpret_cast<uint32_t*>(base + l.err);
    gs::launch_sort(p, sms > 0 ? (uint32_t)sms : 148u, s);
    return cudaGetLastError() == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}
