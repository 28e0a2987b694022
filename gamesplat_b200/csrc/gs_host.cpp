// Host orchestration of the B200 splatting path behind the C ABI
// (include/gs_api.h).  Mirrors the reference renderer's per-frame sequence
// (renderer_draw_frame, src/renderer.cpp:2139-2600) for the splatting
// modes, with the GL passes replaced by CUDA kernels:
//
//   alpha       cull -> depth sort -> bin -> tile sort -> tile ranges -> raster
//   stochastic  cull -> depth sort -> per sample (bin -> tile sort -> ranges ->
//               stochastic raster -> accumulation / frame average) -> TAA
//   gps         cull -> clear -> expand -> splat -> resolve -> accumulation
//
// All device buffers are owned by the context; the scene is copied in and the
// caller keeps its host memory (src/renderer.cpp:736-1074).  Work is issued
// on one stream without host synchronisation; element counts that depend on
// the camera (visible splats, tile entries, GPS work) stay on the device.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <atomic>
#include <vector>

#include "gs_internal.h"
#include "gs_extra.h"
#include "gs_display.h"
#include "gs_denoise.h"
#include "gs_denoiser.h"

using gs::FrameCounters;
using gs::RasterRecord;
using gs::SortPlan;

namespace {

enum Stage { ST_CULL = 0, ST_SORT, ST_BIN, ST_TILE_SORT, ST_RASTER, ST_ACCUM, ST_GPS, ST_DENOISE, ST_COUNT };
const char* kStageNames = "cull,sort,bin,tile_sort,raster,accum,gps,denoise";

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// The buffers one frame's stages leave for its raster pass.  A batch keeps
// one slot per frame and swaps it into the context while that frame's cull,
// sort and binning run, so the stages need no batch-specific code.
struct FrameSlot {
    int width = 0, height = 0, tiles_x = 0, tiles_y = 0;
    int tile_w = 16, tile_h = 16;
    uint32_t tiles_cap = 0;
    void* ctrl = nullptr;
    size_t ctrl_bytes = 0;
    FrameCounters* fc = nullptr;
    SortPlan* depth_plan = nullptr;
    SortPlan* tile_plan = nullptr;
    uint32_t* depth_hist = nullptr;
    uint32_t* tile_hist = nullptr;
    uint2* tile_ranges = nullptr;
    uint32_t* tile_order = nullptr;
    RasterRecord* records = nullptr;
    uint32_t entry_cap = 0;
    uint32_t* ekeys[2] = {nullptr, nullptr};
    uint32_t* evals[2] = {nullptr, nullptr};
    uint32_t* chunk_first = nullptr;
    uint32_t chunk_cap = 0;
    unsigned long long* tsort_status = nullptr;
    size_t tsort_status_stride = 0;
    uint32_t record_cap = 0;
};

}  // namespace

struct gs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t num_sms = 148;
    gs_knobs knobs{};
    std::string last_error;

    // display transform LUT (gsanim 0.3 "layers" scenes)
    uint16_t* display_lut = nullptr;
    int lut_size = 0;
    float lut_log2_min = 0.0f, lut_log2_max = 0.0f;

    // scene
    uint32_t n = 0;
    int row_format = 0;                  // of the next upload: 0 GpuGaussian (256 B), 1 FP16 SH (144 B)
    int half_rows = 0;                   // of the resident scene
    float4* rows = nullptr;
    float4* heads = nullptr;             // first 16 bytes of every row, contiguous (cull visibility pass)
    float4* projected = nullptr;
    uint32_t* keys[2] = {nullptr, nullptr};
    uint32_t* ids[2] = {nullptr, nullptr};
    RasterRecord* records = nullptr;
    uint4* item_info = nullptr;          // binning -> expansion, one per visible splat
    uint32_t* chunk_first = nullptr;     // binning -> expansion, one per entry chunk
    uint32_t chunk_cap = 0;
    unsigned long long* cull_status = nullptr;
    unsigned long long* sort_status = nullptr;
    unsigned long long* bin_status = nullptr;
    size_t sort_status_stride = 0;

    // tile entries
    uint32_t entry_cap = 0;
    uint32_t* ekeys[2] = {nullptr, nullptr};
    uint32_t* evals[2] = {nullptr, nullptr};
    unsigned long long* tsort_status = nullptr;
    size_t tsort_status_stride = 0;

    // per-frame control block (zeroed each frame)
    void* ctrl = nullptr;
    size_t ctrl_bytes = 0;
    FrameCounters* fc = nullptr;
    SortPlan* depth_plan = nullptr;
    SortPlan* tile_plan = nullptr;
    uint32_t* depth_hist = nullptr;
    uint32_t* tile_hist = nullptr;
    uint2* tile_ranges = nullptr;
    uint32_t* tile_order = nullptr;      // raster CTA -> tile (heaviest first)
    uint32_t tiles_cap = 0;
    // the last host read of this block's counters (on fc_stream) is queued:
    // the block is zeroed again only after it (a device-side wait)
    cudaEvent_t ctrl_read = nullptr;
    bool ctrl_read_pending = false;
    // The other control block of the frames drawn by gs_render (same layout):
    // consecutive frames take the two blocks in turn, so a frame's counters are
    // copied to the host on fc_stream while the next frame runs, instead of a
    // copy between two kernels of the render stream.
    struct CtrlBlock {
        void* ctrl = nullptr;
        FrameCounters* fc = nullptr;
        SortPlan* depth_plan = nullptr;
        SortPlan* tile_plan = nullptr;
        uint32_t* depth_hist = nullptr;
        uint32_t* tile_hist = nullptr;
        uint2* tile_ranges = nullptr;
        cudaEvent_t read = nullptr;
        bool read_pending = false;
    };
    CtrlBlock alt;

    // gsanim appearance deltas (renderer animation buffer, src/renderer.cpp:824-841)
    int8_t* anim_deltas = nullptr;
    float* anim_scales = nullptr;
    uint32_t anim_states = 0;     // delta states (state 0 = the uploaded rows)
    int anim_a = 0, anim_b = 0;
    float anim_w = 0.0f;
    // gsanim 0.3 appearance layers (renderer animation buffer of version 3 assets)
    uint16_t* layer_halves = nullptr;
    uint32_t layers_uploaded = 0;
    float* layer_weights = nullptr;      // 256 x 3 floats (device)
    uint32_t layer_count = 0;            // layers weighted in the next frames (0: layer path off)
    std::vector<float> layer_weights_host;

    // camera
    gs_camera cam{};                 // the frame's camera (kernels take it by value)
    FrameCounters* h_fc = nullptr;  // pinned readback
    cudaEvent_t fc_event = nullptr;
    bool fc_pending = false;
    // the frame's counters read back right after binning, while the rest of
    // the frame is still queued: gs_render checks the tile entries there
    FrameCounters* h_bin_fc = nullptr;
    cudaEvent_t bin_event = nullptr;
    bool bin_recorded = false;
    // small device-to-host copies of the frame counters, off the render stream
    cudaStream_t fc_stream = nullptr;
    cudaEvent_t binned = nullptr, frame_done = nullptr;
    FrameCounters* fc_extra = nullptr;   // a second destination of the next end-of-frame copy
    uint32_t epoch = 0;

    // image targets
    int width = 0, height = 0, tiles_x = 0, tiles_y = 0;
    int tile_w = 16, tile_h = 16;            // tile shape of the targets
    int alpha_tile_w = 16, alpha_tile_h = 16;   // tile shape of alpha frames (gs_set_tile_shape)
    uint32_t batch_depth = 0;                // frames per persistent raster launch in batches (0: all)
    uint16_t* out16 = nullptr;     // internal RGBA16F (gs_render_host)
    uint16_t* h_out16 = nullptr;   // pinned
    size_t h_out16_bytes = 0;
    cudaEvent_t chunk_events[8] = {};   // gs_render_host: readback chunks of a pageable destination
    // streamed readback (gs_render_host_submit / gs_render_host_wait): two
    // device images; each frame's image is copied to its caller's page-locked
    // buffer on copy_stream while the next frame renders on `stream`
    struct StreamSlot {
        uint16_t* image = nullptr;          // device RGBA16F
        size_t bytes = 0;                   // its capacity
        const uint16_t* host = nullptr;     // destination of the frame in flight (null: slot free)
        FrameCounters* h_fc = nullptr;      // pinned: that frame's counters
        cudaEvent_t rendered = nullptr, copied = nullptr;
    };
    StreamSlot sslot[2];
    int sslot_next = 0;                     // the slot the next frame takes (the older one when both are busy)
    cudaStream_t copy_stream = nullptr;
    gs::StochasticTargets st{};
    gs::GpsTargets gps{};
    uint32_t gps_max_work_items = 16u * 1024u * 1024u;

    // denoised mode: the attached denoiser (not owned), its input features
    // (W x H x 16 bf16), the tiles over the error budget and its knobs
    gs_denoiser* denoiser = nullptr;
    __nv_bfloat16* features = nullptr;
    size_t features_pix = 0;
    uint32_t* fallback_tiles = nullptr;   // tiles_cap entries
    float* tile_error = nullptr;          // tiles_cap estimated MSE per tile
    float denoise_budget = 1.0e-4f;       // tile MSE budget: 40 dB PSNR
    int denoise_fallback = 1;

    // stochastic / accumulation state (src/renderer.h:230-246)
    uint32_t frame_seed = 0;
    uint32_t sample_count = 0;
    uint32_t accum_write_index = 0;
    gs_camera prev_cam{};
    bool prev_cam_valid = false;
    bool taa_prev_valid = false;

    // batches (gs_render_batch, gs_render_anim_batch): one slot per frame
    std::vector<FrameSlot> slots;
    FrameCounters* h_slot_fc = nullptr;   // pinned, one per slot
    uint32_t h_slot_fc_cap = 0;
    gs::RasterParams* h_batch_params = nullptr;   // pinned
    gs::RasterParams* batch_params = nullptr;     // device
    uint32_t* batch_first = nullptr;              // device: prefix sums of tiles (+ the ticket word)
    uint32_t* h_batch_first = nullptr;            // pinned
    uint32_t batch_cap = 0;
    float4* state_colours = nullptr;              // anim batches: n x states colours
    size_t state_colours_cap = 0;
    cudaEvent_t batch_event = nullptr;
    cudaEvent_t params_event = nullptr;           // after the last copy out of h_batch_params / h_batch_first
    bool params_pending = false;

    // profiling
    bool profiling = false;
    struct Pending { cudaEvent_t a, b; int stage; uint32_t launches; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double stage_ms[ST_COUNT] = {};
    uint32_t stage_launches[ST_COUNT] = {};
    uint32_t last_launches = 0;
    uint32_t frame_launches = 0;
};

namespace {

int fail(gs_ctx* c, int status, const std::string& msg) {
    if (c) c->last_error = msg;
    return status;
}

int cuda_fail(gs_ctx* c, cudaError_t e, const char* what) {
    return fail(c, e == cudaErrorMemoryAllocation ? GS_ERR_OOM : GS_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define GS_CUDA(ctx, call)                                  \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
    } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    return gs::device_malloc(reinterpret_cast<void**>(p), bytes);
}

// Tile-entry capacity of a scene of n Gaussians before any frame overflowed it.
uint32_t default_entry_cap(uint32_t n) {
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(8ull * n, 1u << 20), 0x3FFFFFFFull);
}

// Device bytes of a scene of n Gaussians with a GPS budget of work_items:
// what an upload allocates (rows, heads, projected records, sort pairs,
// raster records, binning state, look-back words, tile entries at their
// initial capacity) plus the GPS prepared records and work items.  The
// counterpart of renderer_scene_buffer_bytes (src/renderer.cpp:705-709) for
// this layout.  Frame targets (sized by the viewport) are not counted there
// either.
uint64_t scene_device_bytes(uint32_t n, uint32_t work_items) {
    uint64_t b = (uint64_t)work_items * sizeof(uint2);
    if (!n) return b;
    b += (uint64_t)n * (256u + 16u + 64u + 16u + sizeof(RasterRecord) + sizeof(uint4) + 48u);
    b += ((uint64_t)n + gs::kCullVisTile - 1) / gs::kCullVisTile * 8u;
    b += (uint64_t)gs::sort_status_words(n) * 4u * 8u;
    b += ((uint64_t)n + gs::kBinTile - 1) / gs::kBinTile * 8u;
    const uint32_t cap = default_entry_cap(n);
    b += (uint64_t)cap * 16u + ((uint64_t)cap / gs::kBinChunk + 2u) * 4u;
    b += (uint64_t)gs::sort_status_words(cap) * 4u * 8u;
    return b;
}

template <class T>
void dfree(T*& p) {
    if (p) cudaFree(reinterpret_cast<void*>(p));
    p = nullptr;
}

void release_slot(FrameSlot& f) {
    dfree(f.ctrl);
    dfree(f.tile_order);
    dfree(f.records);
    for (int k = 0; k < 2; ++k) {
        dfree(f.ekeys[k]);
        dfree(f.evals[k]);
    }
    dfree(f.chunk_first);
    dfree(f.tsort_status);
    f = FrameSlot{};
}

void release_slots(gs_ctx* c) {
    for (auto& f : c->slots) release_slot(f);
    c->slots.clear();
    dfree(c->state_colours);
    c->state_colours_cap = 0;
}

// Exchange the per-frame buffers of the context with those of a slot.
void swap_slot(gs_ctx* c, FrameSlot& f) {
    std::swap(c->width, f.width);
    std::swap(c->height, f.height);
    std::swap(c->tiles_x, f.tiles_x);
    std::swap(c->tiles_y, f.tiles_y);
    std::swap(c->tile_w, f.tile_w);
    std::swap(c->tile_h, f.tile_h);
    std::swap(c->tiles_cap, f.tiles_cap);
    std::swap(c->ctrl, f.ctrl);
    std::swap(c->ctrl_bytes, f.ctrl_bytes);
    std::swap(c->fc, f.fc);
    std::swap(c->depth_plan, f.depth_plan);
    std::swap(c->tile_plan, f.tile_plan);
    std::swap(c->depth_hist, f.depth_hist);
    std::swap(c->tile_hist, f.tile_hist);
    std::swap(c->tile_ranges, f.tile_ranges);
    std::swap(c->tile_order, f.tile_order);
    std::swap(c->records, f.records);
    std::swap(c->entry_cap, f.entry_cap);
    for (int k = 0; k < 2; ++k) {
        std::swap(c->ekeys[k], f.ekeys[k]);
        std::swap(c->evals[k], f.evals[k]);
    }
    std::swap(c->chunk_first, f.chunk_first);
    std::swap(c->chunk_cap, f.chunk_cap);
    std::swap(c->tsort_status, f.tsort_status);
    std::swap(c->tsort_status_stride, f.tsort_status_stride);
}

void release_scene(gs_ctx* c) {
    dfree(c->rows);
    dfree(c->heads);
    dfree(c->projected);
    for (int k = 0; k < 2; ++k) {
        dfree(c->keys[k]);
        dfree(c->ids[k]);
        dfree(c->ekeys[k]);
        dfree(c->evals[k]);
    }
    dfree(c->records);
    dfree(c->item_info);
    dfree(c->cull_status);
    dfree(c->sort_status);
    dfree(c->bin_status);
    dfree(c->tsort_status);
    dfree(c->chunk_first);
    c->chunk_cap = 0;
    gs::release_gps_scene(c->gps);
    dfree(c->anim_deltas);
    dfree(c->anim_scales);
    c->anim_states = 0;
    c->anim_a = c->anim_b = 0;
    c->anim_w = 0.0f;
    dfree(c->layer_halves);
    dfree(c->layer_weights);
    c->layers_uploaded = 0;
    c->layer_count = 0;
    c->layer_weights_host.clear();
    c->n = 0;
    c->entry_cap = 0;
    release_slots(c);
}

void release_targets(gs_ctx* c) {
    // copies of the counters may still read the blocks
    if (c->fc_stream) cudaStreamSynchronize(c->fc_stream);
    dfree(c->out16);
    dfree(c->ctrl);
    if (c->alt.ctrl) {
        void* p = c->alt.ctrl;
        dfree(p);
        c->alt.ctrl = nullptr;
        c->alt.fc = nullptr;
    }
    c->ctrl_read_pending = c->alt.read_pending = false;
    dfree(c->tile_order);
    dfree(c->features);
    dfree(c->fallback_tiles);
    dfree(c->tile_error);
    c->features_pix = 0;
    c->fc = nullptr;
    gs::release_stochastic_targets(c->st);
    gs::release_gps_targets(c->gps);
    c->width = c->height = 0;
    c->tiles_cap = 0;
}

cudaEvent_t take_event(gs_ctx* c) {
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// NVTX range names of the stages (the reference's profiler zones,
// src/renderer.cpp:1890-1937,1984-2088): visible to nsys / ncu --nvtx.
const char* const kStageRanges[ST_COUNT] = {"gs cull/project", "gs depth sort", "gs bin", "gs tile sort",
                                            "gs raster", "gs accumulate", "gs gps splat", "gs denoise"};

struct StageScope {
    gs_ctx* c;
    int stage;
    cudaEvent_t a = nullptr;
    uint32_t launches = 0;
    StageScope(gs_ctx* ctx, int s) : c(ctx), stage(s) {
        nvtxRangePushA(kStageRanges[s]);
        if (c->profiling) {
            a = take_event(c);
            cudaEventRecord(a, c->stream);
        }
    }
    void add(int k) { launches += (uint32_t)k; }
    ~StageScope() {
        c->frame_launches += launches;
        if (c->profiling) {
            cudaEvent_t b = take_event(c);
            cudaEventRecord(b, c->stream);
            c->pending.push_back({a, b, stage, launches});
        }
        nvtxRangePop();
    }
};

// renderer_gpu_buffer_limits (src/renderer.cpp:713-732), the NVIDIA branch:
// new allocations stay within 4/5 of the device's free memory, and the
// retained scene buffers within gpu_budget_mb when it is set.
struct MemoryLimits {
    uint64_t scene_cap;
    uint64_t allocation_budget;
};

MemoryLimits memory_limits(const gs_ctx* c) {
    MemoryLimits m{UINT64_MAX, UINT64_MAX};
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) m.allocation_budget = (uint64_t)free_b * 4u / 5u;
    else cudaGetLastError();   // the allocations themselves will report the failure
    if (c->knobs.gpu_budget_mb) m.scene_cap = (uint64_t)c->knobs.gpu_budget_mb << 20;
    return m;
}

uint64_t anim_device_bytes(uint32_t n, uint32_t states) {
    return states ? (uint64_t)states * n * 48u + 48u * sizeof(float) : 0u;
}

uint64_t layer_device_bytes(uint32_t n, uint32_t layers) {
    return layers ? (uint64_t)layers * n * 48u * sizeof(uint16_t) + 256u * 3u * sizeof(float) : 0u;
}

std::string mib(uint64_t bytes) {
    if (bytes == UINT64_MAX) return "unlimited";
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%.1f MiB", (double)bytes / 1048576.0);
    return buf;
}

int entry_bits(uint32_t tiles) {
    int bits = 1;
    while (bits < 32 && (1u << bits) < tiles) ++bits;
    return bits;
}

// Tile-entry buffers: (tile, splat) pairs.  Grown on overflow.
int ensure_entries(gs_ctx* c, uint32_t cap) {
    if (cap <= c->entry_cap) return GS_OK;
    for (int k = 0; k < 2; ++k) {
        dfree(c->ekeys[k]);
        dfree(c->evals[k]);
    }
    dfree(c->tsort_status);
    dfree(c->chunk_first);
    c->entry_cap = 0;
    c->chunk_cap = 0;
    for (int k = 0; k < 2; ++k) {
        GS_CUDA(c, dalloc(&c->ekeys[k], (size_t)cap * 4));
        GS_CUDA(c, dalloc(&c->evals[k], (size_t)cap * 4));
    }
    const uint32_t chunks = cap / (uint32_t)gs::kBinChunk + 2u;
    GS_CUDA(c, dalloc(&c->chunk_first, (size_t)chunks * 4));
    c->chunk_cap = chunks;
    c->tsort_status_stride = gs::sort_status_words(cap);
    GS_CUDA(c, dalloc(&c->tsort_status, c->tsort_status_stride * 4 * sizeof(unsigned long long)));
    GS_CUDA(c, cudaMemsetAsync(c->tsort_status, 0, c->tsort_status_stride * 4 * sizeof(unsigned long long), c->stream));
    c->entry_cap = cap;
    return GS_OK;
}

// The per-frame control block of a w x h frame in the context's fields:
// FrameCounters | SortPlan x2 | hist x2 (4x256) | tile ranges, and the tile order.
// Control block layout: FrameCounters | SortPlan x2 | hist x2 (4x256) | tile
// ranges; each part 256-byte aligned.
struct CtrlLayout {
    size_t fc, dp, tp, dh, th, tr, bytes;
};

CtrlLayout ctrl_layout(uint32_t tiles) {
    CtrlLayout L{};
    size_t off = 0;
    auto place = [&](size_t bytes) {
        size_t o = off;
        off = (off + bytes + 255) & ~(size_t)255;
        return o;
    };
    L.fc = place(sizeof(FrameCounters));
    L.dp = place(sizeof(SortPlan));
    L.tp = place(sizeof(SortPlan));
    L.dh = place(4 * 256 * 4);
    L.th = place(4 * 256 * 4);
    L.tr = place((size_t)tiles * sizeof(uint2));
    L.bytes = off;
    return L;
}

template <typename B> void carve_ctrl(B& b, void* ctrl, const CtrlLayout& L) {
    char* base = static_cast<char*>(ctrl);
    b.ctrl = ctrl;
    b.fc = reinterpret_cast<FrameCounters*>(base + L.fc);
    b.depth_plan = reinterpret_cast<SortPlan*>(base + L.dp);
    b.tile_plan = reinterpret_cast<SortPlan*>(base + L.tp);
    b.depth_hist = reinterpret_cast<uint32_t*>(base + L.dh);
    b.tile_hist = reinterpret_cast<uint32_t*>(base + L.th);
    b.tile_ranges = reinterpret_cast<uint2*>(base + L.tr);
}

// The context's control block (and, with_alt, the second block of gs_render's
// frames) for a w x h viewport of tw x th tiles.
int alloc_control(gs_ctx* c, int w, int h, int tw, int th, bool with_alt = true) {
    const int tx = (w + tw - 1) / tw, ty = (h + th - 1) / th;
    c->tile_w = tw;
    c->tile_h = th;
    c->tiles_cap = (uint32_t)(tx * ty);
    const CtrlLayout L = ctrl_layout(c->tiles_cap);
    c->ctrl_bytes = L.bytes;
    void* block = nullptr;
    GS_CUDA(c, dalloc(reinterpret_cast<char**>(&block), c->ctrl_bytes));
    carve_ctrl(*c, block, L);
    GS_CUDA(c, cudaMemsetAsync(c->ctrl, 0, c->ctrl_bytes, c->stream));
    if (with_alt) {
        void* other = nullptr;
        GS_CUDA(c, dalloc(reinterpret_cast<char**>(&other), c->ctrl_bytes));
        carve_ctrl(c->alt, other, L);
        GS_CUDA(c, cudaMemsetAsync(c->alt.ctrl, 0, c->ctrl_bytes, c->stream));
    }
    GS_CUDA(c, dalloc(&c->tile_order, (size_t)c->tiles_cap * sizeof(uint32_t)));
    c->width = w;
    c->height = h;
    c->tiles_x = tx;
    c->tiles_y = ty;
    return GS_OK;
}

// gs_render's frames alternate between the two control blocks: this one's
// counters may still be on their way to the host while the next frame runs.
void swap_ctrl(gs_ctx* c) {
    if (!c->alt.ctrl) return;
    gs_ctx::CtrlBlock cur;
    cur.ctrl = c->ctrl;
    cur.fc = c->fc;
    cur.depth_plan = c->depth_plan;
    cur.tile_plan = c->tile_plan;
    cur.depth_hist = c->depth_hist;
    cur.tile_hist = c->tile_hist;
    cur.tile_ranges = c->tile_ranges;
    cur.read = c->ctrl_read;
    cur.read_pending = c->ctrl_read_pending;
    const gs_ctx::CtrlBlock nxt = c->alt;
    c->alt = cur;
    c->ctrl = nxt.ctrl;
    c->fc = nxt.fc;
    c->depth_plan = nxt.depth_plan;
    c->tile_plan = nxt.tile_plan;
    c->depth_hist = nxt.depth_hist;
    c->tile_hist = nxt.tile_hist;
    c->tile_ranges = nxt.tile_ranges;
    c->ctrl_read = nxt.read;
    c->ctrl_read_pending = nxt.read_pending;
}

// Tile shape of the context's frames: the alpha knob in alpha mode, 16x16 otherwise.
void frame_tile_shape(const gs_ctx* c, int* tw, int* th) {
    const bool alpha = c->knobs.render_mode == GS_MODE_ALPHA;
    *tw = alpha ? c->alpha_tile_w : 16;
    *th = alpha ? c->alpha_tile_h : 16;
}

int ensure_targets(gs_ctx* c, int w, int h) {
    if (w <= 0 || h <= 0) return fail(c, GS_ERR_BAD_ARG, "viewport must be positive");
    if (w > 32767 || h > 32767) return fail(c, GS_ERR_TOO_LARGE, "viewport beyond 32767 pixels");
    int tw = 16, th = 16;
    frame_tile_shape(c, &tw, &th);
    if (c->width == w && c->height == h && c->ctrl && c->tile_w == tw && c->tile_h == th) return GS_OK;
    release_targets(c);
    int rc = alloc_control(c, w, h, tw, th);
    if (rc) return rc;
    const cudaError_t e = dalloc(&c->out16, (size_t)w * h * 8);
    if (e != cudaSuccess) {
        c->width = c->height = 0;   // the next frame allocates the targets again
        return cuda_fail(c, e, "dalloc(out16)");
    }
    c->sample_count = 0;
    c->accum_write_index = 0;
    c->taa_prev_valid = false;
    return GS_OK;
}

// Grow the entry buffers if the last completed frame overflowed them.
int check_previous_frame(gs_ctx* c) {
    if (!c->fc_pending) return GS_OK;
    if (cudaEventQuery(c->fc_event) != cudaSuccess) return GS_OK;
    c->fc_pending = false;
    if (c->h_fc->tile_overflow) {
        uint64_t need = (uint64_t)c->h_fc->tile_entries + c->h_fc->tile_overflow;
        uint64_t cap = std::min<uint64_t>(need + need / 4 + 1024, 0x3FFFFFFFull);
        return ensure_entries(c, (uint32_t)cap);
    }
    return GS_OK;
}

void begin_frame(gs_ctx* c, const gs_camera* cam, bool zero_ctrl = true) {
    c->cam = *cam;
    if (zero_ctrl) cudaMemsetAsync(c->ctrl, 0, c->ctrl_bytes, c->stream);
    ++c->epoch;
    if (c->epoch == 0) ++c->epoch;
    c->frame_launches = 0;
}

// A frame of gs_render / gs_render_features: it takes the other control
// block, zeroed on fc_stream after its last counters went to the host (the
// render stream waits for that, long done by now), and the block it leaves
// is zeroed the same way while this frame runs.  The last frame's block stays
// intact until the next frame begins, for gs_debug_read.
void begin_render_frame(gs_ctx* c, const gs_camera* cam) {
    if (!c->alt.ctrl) {
        begin_frame(c, cam);
        return;
    }
    swap_ctrl(c);
    if (c->ctrl_read_pending) cudaStreamWaitEvent(c->stream, c->ctrl_read, 0);
    c->ctrl_read_pending = false;
    if (c->alt.read_pending) {   // queued behind the copy of its counters on fc_stream
        cudaMemsetAsync(c->alt.ctrl, 0, c->ctrl_bytes, c->fc_stream);
        cudaEventRecord(c->alt.read, c->fc_stream);
    }
    begin_frame(c, cam, /*zero_ctrl*/ false);
}

// The frame's counters go to the host on fc_stream, behind the frame's last
// operation but off the render stream (and, when set, to fc_extra as well).
void end_frame(gs_ctx* c) {
    cudaEventRecord(c->frame_done, c->stream);
    cudaStreamWaitEvent(c->fc_stream, c->frame_done, 0);
    cudaMemcpyAsync(c->h_fc, c->fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, c->fc_stream);
    if (c->fc_extra)
        cudaMemcpyAsync(c->fc_extra, c->fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, c->fc_stream);
    cudaEventRecord(c->fc_event, c->fc_stream);
    cudaEventRecord(c->ctrl_read, c->fc_stream);
    c->ctrl_read_pending = true;
    c->fc_pending = true;
    c->last_launches = c->frame_launches;
}

gs::CullParams cull_params(gs_ctx* c) {
    gs::CullParams p{};
    p.rows = c->rows;
    p.heads = c->heads;
    p.n = c->n;
    p.cam = c->cam;
    p.sh_degree = std::max(0, std::min(3, c->knobs.sh_degree));
    p.sh_lod_distance = c->knobs.sh_lod_distance;
    p.collect_stats = c->knobs.splat_diagnostics_enabled ? 1 : 0;
    p.write_invisible = c->knobs.write_invisible_records ? 1 : 0;
    p.projected = c->projected;
    p.keys_out = c->keys[1];
    p.ids_out = c->ids[1];
    p.status = c->cull_status;
    p.epoch = c->epoch;
    p.key_hist = c->depth_hist;
    if (c->anim_deltas) {
        p.anim_deltas = c->anim_deltas;
        p.anim_scales = c->anim_scales;
        p.anim_state_a = c->anim_a;
        p.anim_state_b = c->anim_b;
        p.anim_weight = c->anim_w;
    }
    if (c->layer_count) {
        p.layer_halves = c->layer_halves;
        p.layer_weights = c->layer_weights;
        p.layer_count = (int)c->layer_count;
    }
    p.half_rows = c->half_rows;
    p.fc = c->fc;
    return p;
}

void run_cull(gs_ctx* c) {
    StageScope sc(c, ST_CULL);
    sc.add(gs::launch_cull(cull_params(c), c->num_sms, c->stream));
}

void run_depth_sort(gs_ctx* c) {
    StageScope sc(c, ST_SORT);
    gs::SortParams p{};
    p.keys_in = c->keys[1];
    p.vals_in = c->ids[1];
    p.keys_buf[0] = c->keys[0];
    p.keys_buf[1] = c->keys[1];
    p.vals_buf[0] = c->ids[0];
    p.vals_buf[1] = c->ids[1];
    p.land_in_buf0 = 0;
    p.count_ptr = &c->fc->visible_count;
    p.count_cap = c->n;
    p.begin_bit = 0;
    p.end_bit = 32;
    p.hist = c->depth_hist;   // accumulated by the cull kernel
    p.hist_ready = 1;
    p.plan = c->depth_plan;
    p.status = c->sort_status;
    p.status_stride = c->sort_status_stride;
    p.epoch = c->epoch;
    p.error_flags = &c->fc->error_flags;
    p.first_pdl = 1;
    sc.add(gs::launch_sort(p, c->num_sms, c->stream));
}

// Binning, tile sort and tile ranges for one raster pass.
// readback: copy the counters to h_bin_fc on fc_stream once the tile sort has
// run (the entry count is final after the expansion).
void run_binning(gs_ctx* c, float jx, float jy, float seed, bool envelope = false, bool readback = true) {
    {
        StageScope sc(c, ST_BIN);
        gs::BinParams p{};
        p.depth_plan = c->depth_plan;
        p.projected = c->projected;
        p.vp_w = c->cam.viewport[0];
        p.vp_h = c->cam.viewport[1];
        p.clip_y_sign = c->cam.clip_y_sign;
        p.jitter_x = jx;
        p.jitter_y = jy;
        p.frame_seed = seed;
        p.width = c->width;
        p.height = c->height;
        p.tiles_x = c->tiles_x;
        p.tiles_y = c->tiles_y;
        p.tile_shift_x = c->tile_w == 32 ? 5 : c->tile_w == 8 ? 3 : 4;
        p.tile_shift_y = c->tile_h == 32 ? 5 : c->tile_h == 8 ? 3 : 4;
        p.records = c->records;
        p.entry_keys = c->ekeys[1];
        p.entry_vals = c->evals[1];
        p.entry_cap = c->entry_cap;
        p.item_info = c->item_info;
        p.chunk_first = c->chunk_first;
        p.chunk_cap = c->chunk_cap;
        p.tile_hist = c->tile_hist;
        p.status = c->bin_status;
        p.epoch = c->epoch;
        p.fc = c->fc;
        p.envelope = envelope ? 1 : 0;
        sc.add(gs::launch_bin(p, c->n, c->num_sms, c->stream));
    }
    {
        StageScope sc(c, ST_TILE_SORT);
        gs::SortParams p{};
        p.keys_in = c->ekeys[1];
        p.vals_in = c->evals[1];
        p.keys_buf[0] = c->ekeys[0];
        p.keys_buf[1] = c->ekeys[1];
        p.vals_buf[0] = c->evals[0];
        p.vals_buf[1] = c->evals[1];
        p.land_in_buf0 = 0;
        p.count_ptr = &c->fc->tile_entries;
        p.count_cap = c->entry_cap;
        p.begin_bit = 0;
        p.end_bit = entry_bits(c->tiles_cap);
        p.hist = c->tile_hist;    // accumulated by the bin kernel
        p.hist_ready = 1;
        p.plan = c->tile_plan;
        p.status = c->tsort_status;
        p.status_stride = c->tsort_status_stride;
        p.epoch = c->epoch;
        p.error_flags = &c->fc->error_flags;
        p.first_pdl = 1;
        sc.add(gs::launch_sort(p, c->num_sms, c->stream));
        // The entry count is final once the expansion ran; the readback is
        // queued behind the tile sort so that the expansion and the sort's
        // first pass stay adjacent (programmatic dependent launch between them).
        if (readback) {
            cudaEventRecord(c->binned, c->stream);
            cudaStreamWaitEvent(c->fc_stream, c->binned, 0);
            cudaMemcpyAsync(c->h_bin_fc, c->fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, c->fc_stream);
            cudaEventRecord(c->bin_event, c->fc_stream);
            c->bin_recorded = true;
        }
        sc.add(gs::launch_tile_ranges(c->tile_plan, c->fc, c->entry_cap, c->tile_ranges, c->tiles_cap, c->num_sms,
                                       c->stream));
        sc.add(gs::launch_tile_order(c->tile_ranges, c->tiles_cap, c->tile_order, c->stream));
    }
}

gs::RasterParams raster_params(gs_ctx* c, float bg) {
    gs::RasterParams r{};
    r.records = c->records;
    r.record_cap = c->n;
    r.tile_plan = c->tile_plan;
    r.tile_ranges = c->tile_ranges;
    r.tile_order = c->tile_order;
    r.width = c->width;
    r.height = c->height;
    r.tiles_x = c->tiles_x;
    r.tiles_y = c->tiles_y;
    r.tile_w = c->tile_w;
    r.tile_h = c->tile_h;
    r.bg = bg;
    r.fc = c->fc;
    return r;
}

float background(const gs_ctx* c) { return c->knobs.black_background ? 0.0f : 0.1f; }  // src/renderer.cpp:2146

int render_alpha(gs_ctx* c, uint16_t* out) {
    run_cull(c);
    run_depth_sort(c);
    run_binning(c, 0.0f, 0.0f, 0.0f);
    StageScope sc(c, ST_RASTER);
    gs::RasterParams r = raster_params(c, background(c));
    r.out_rgba16f = out;
    sc.add(gs::launch_raster_alpha(r, c->stream));
    return GS_OK;
}

// src/renderer.cpp:246-255
float halton(uint32_t index, uint32_t base) {
    float f = 1.0f, r = 0.0f;
    while (index > 0) {
        f /= (float)base;
        r += f * (float)(index % base);
        index /= base;
    }
    return r;
}

int render_stochastic(gs_ctx* c, const gs_camera* cam, uint16_t* out) {
    int rc = gs::ensure_stochastic_targets(c->st, c->width, c->height, c->stream);
    if (rc) return fail(c, rc, "stochastic target allocation failed");
    const size_t npix = (size_t)c->width * c->height;
    const float bg = background(c);
    // src/renderer.cpp:2300-2330
    bool prev_cam_valid = c->prev_cam_valid;
    const bool cam_changed = c->prev_cam_valid && std::memcmp(&c->prev_cam, cam, sizeof(gs_camera)) != 0;
    const gs_camera prev_cam = c->prev_cam;
    if (!c->knobs.stochastic_taa_enabled && cam_changed) {
        c->sample_count = 0;
        c->taa_prev_valid = false;
        prev_cam_valid = false;
    }
    c->prev_cam = *cam;
    c->prev_cam_valid = true;
    const uint32_t spf = std::max(1u, std::min(16u, c->knobs.stochastic_samples_per_frame));
    const bool use_taa = c->knobs.stochastic_taa_enabled != 0;
    uint32_t render_samples = use_taa ? std::max(1u, std::min(16u, c->knobs.stochastic_taa_current_samples)) : spf;
    float inv_view[16];
    if (use_taa && !gs::mat4_inverse(cam->view, inv_view)) {
        c->sample_count = 0;
        c->taa_prev_valid = false;
        std::memcpy(inv_view, cam->view, sizeof(inv_view));
        prev_cam_valid = false;
    }

    run_cull(c);
    run_depth_sort(c);
    // One binning for every sample of the frame: tiles for any jitter, the
    // rasterizer derives each sample's quad coverage.
    run_binning(c, 0.0f, 0.0f, 0.0f, /*envelope*/ true);
    uint32_t write_index = c->accum_write_index & 1u;
    bool display_accum = false;
    for (uint32_t i = 0; i < render_samples; ++i) {
        c->frame_seed++;
        float jx = 0.0f, jy = 0.0f;
        if (use_taa) {
            uint32_t jitter_index = (c->frame_seed % 1024u) + 1u;
            jx = halton(jitter_index, 2u) - 0.5f;
            jy = halton(jitter_index, 3u) - 0.5f;
        }
        {
            StageScope sc(c, ST_RASTER);
            gs::RasterParams r = raster_params(c, bg);
            r.jitter_x = jx;
            r.jitter_y = jy;
            r.frame_seed = (float)c->frame_seed;
            r.vp_w = c->cam.viewport[0];
            r.vp_h = c->cam.viewport[1];
            r.clip_y_sign = c->cam.clip_y_sign;
            // TAA with several samples: the rasterizer folds each sample into
            // the frame average itself; only the last sample's colour and
            // depth are kept (the TAA pass and the debug reads use those)
            const bool fold = use_taa && render_samples > 1, last = i + 1 == render_samples;
            r.out_rgba32f = !fold || last ? c->st.sample : nullptr;
            r.out_depth = !fold || last ? c->st.depth : nullptr;
            if (fold) {
                const uint32_t w = i & 1u, rd = w ^ 1u;
                r.accum_in = i == 0 ? nullptr : c->st.frame_avg[rd];
                r.accum_out = c->st.frame_avg[w];
                r.accum_n = (float)(i + 1);
            }
            r.rgba8 = c->knobs.linear_color ? 0 : 1;
            sc.add(gs::launch_raster_stochastic(r, c->stream));
        }
        StageScope sa(c, ST_ACCUM);
        if (use_taa && render_samples > 1) {
            // folded into the rasterizer above
        } else if (!use_taa && (c->knobs.stochastic_accumulation_enabled || render_samples > 1)) {
            const bool acc = c->knobs.stochastic_accumulation_enabled != 0;
            uint32_t next = acc ? c->sample_count + 1 : i + 1;
            write_index = acc ? (c->accum_write_index & 1u) : (i & 1u);
            uint32_t rd = write_index ^ 1u;
            sa.add(gs::launch_accum(c->st.sample, next == 1 ? c->st.sample : c->st.accum[rd], (float)next,
                                    c->st.accum[write_index], npix, c->stream));
            display_accum = true;
            if (acc) {
                c->sample_count = next;
                c->accum_write_index = write_index ^ 1u;
            }
        }
    }
    if (use_taa) {
        StageScope sa(c, ST_ACCUM);
        write_index = c->accum_write_index & 1u;
        uint32_t rd = write_index ^ 1u;
        const float4* current = render_samples > 1 ? c->st.frame_avg[(render_samples - 1) & 1u] : c->st.sample;
        const bool has_history = c->taa_prev_valid && prev_cam_valid;
        gs::TaaUniforms u{};
        std::memcpy(u.inv_view, inv_view, sizeof(u.inv_view));
        std::memcpy(u.prev_view, has_history ? prev_cam.view : cam->view, sizeof(u.prev_view));
        u.viewport_orthographic[0] = cam->viewport[0];
        u.viewport_orthographic[1] = cam->viewport[1];
        u.viewport_orthographic[2] = cam->orthographic;
        u.viewport_orthographic[3] = has_history ? prev_cam.orthographic : cam->orthographic;
        u.focal_clip[0] = cam->persp_focal;
        u.focal_clip[1] = cam->ortho_focal;
        u.focal_clip[2] = cam->clip_y_sign;
        u.focal_clip[3] = cam->clip_z_01;
        u.prev_focal_clip[0] = has_history ? prev_cam.persp_focal : cam->persp_focal;
        u.prev_focal_clip[1] = has_history ? prev_cam.ortho_focal : cam->ortho_focal;
        u.prev_focal_clip[2] = has_history ? prev_cam.clip_y_sign : cam->clip_y_sign;
        u.proj_z[0] = cam->proj[10];
        u.proj_z[1] = cam->proj[14];
        u.history_valid = has_history ? 1.0f : 0.0f;
        u.view_changed = cam_changed ? 1.0f : 0.0f;
        sa.add(gs::launch_taa(current, c->st.depth, c->st.accum[rd], c->st.xyz[rd], c->width, c->height, u,
                              c->st.accum[write_index], c->st.xyz[write_index], c->stream));
        c->taa_prev_valid = true;
        c->sample_count++;
        c->accum_write_index = write_index ^ 1u;
        display_accum = true;
    }
    StageScope sd(c, ST_ACCUM);
    c->st.display = display_accum ? c->st.accum[write_index] : c->st.sample;
    sd.add(gs::launch_to_half(c->st.display, out, npix, c->stream));
    return GS_OK;
}

// TAA uniforms of a frame (shaders/accum.glsl:65-76; src/renderer.cpp:2426-2485).
gs::TaaUniforms taa_uniforms(const gs_camera* cam, const gs_camera& prev_cam, const float inv_view[16],
                             bool has_history, bool cam_changed) {
    gs::TaaUniforms u{};
    std::memcpy(u.inv_view, inv_view, sizeof(u.inv_view));
    std::memcpy(u.prev_view, has_history ? prev_cam.view : cam->view, sizeof(u.prev_view));
    u.viewport_orthographic[0] = cam->viewport[0];
    u.viewport_orthographic[1] = cam->viewport[1];
    u.viewport_orthographic[2] = cam->orthographic;
    u.viewport_orthographic[3] = has_history ? prev_cam.orthographic : cam->orthographic;
    u.focal_clip[0] = cam->persp_focal;
    u.focal_clip[1] = cam->ortho_focal;
    u.focal_clip[2] = cam->clip_y_sign;
    u.focal_clip[3] = cam->clip_z_01;
    u.prev_focal_clip[0] = has_history ? prev_cam.persp_focal : cam->persp_focal;
    u.prev_focal_clip[1] = has_history ? prev_cam.ortho_focal : cam->ortho_focal;
    u.prev_focal_clip[2] = has_history ? prev_cam.clip_y_sign : cam->clip_y_sign;
    u.proj_z[0] = cam->proj[10];
    u.proj_z[1] = cam->proj[14];
    u.history_valid = has_history ? 1.0f : 0.0f;
    u.view_changed = cam_changed ? 1.0f : 0.0f;
    return u;
}

int ensure_denoise_targets(gs_ctx* c) {
    int rc = gs::ensure_stochastic_targets(c->st, c->width, c->height, c->stream);
    if (rc) return fail(c, rc, "stochastic target allocation failed");
    const size_t npix = (size_t)c->width * c->height;
    if (c->features_pix != npix || !c->features) {
        dfree(c->features);
        dfree(c->fallback_tiles);
        dfree(c->tile_error);
        c->features_pix = 0;
        GS_CUDA(c, dalloc(&c->features, npix * gs::dn::kInC * sizeof(__nv_bfloat16)));
        GS_CUDA(c, dalloc(&c->fallback_tiles, (size_t)c->tiles_cap * sizeof(uint32_t)));
        GS_CUDA(c, dalloc(&c->tile_error, (size_t)c->tiles_cap * sizeof(float)));
        c->features_pix = npix;
    }
    return GS_OK;
}

// The stochastic half of a denoised frame: two un-jittered stochastic samples
// per pixel (seeds frame_seed + 1, + 2) from the sorted tile lists, their TAA
// history (shaders/accum.glsl:148-178) and the denoiser's input features.
int render_denoise_inputs(gs_ctx* c, const gs_camera* cam) {
    int rc = ensure_denoise_targets(c);
    if (rc) return rc;
    const size_t npix = (size_t)c->width * c->height;
    const bool cam_changed = c->prev_cam_valid && std::memcmp(&c->prev_cam, cam, sizeof(gs_camera)) != 0;
    const gs_camera prev_cam = c->prev_cam;
    bool prev_valid = c->prev_cam_valid;
    c->prev_cam = *cam;
    c->prev_cam_valid = true;
    float inv_view[16];
    if (!gs::mat4_inverse(cam->view, inv_view)) {
        c->taa_prev_valid = false;
        std::memcpy(inv_view, cam->view, sizeof(inv_view));
        prev_valid = false;
    }
    run_cull(c);
    run_depth_sort(c);
    run_binning(c, 0.0f, 0.0f, 0.0f);
    {
        StageScope sc(c, ST_RASTER);
        gs::RasterParams r = raster_params(c, background(c));
        r.frame_seed = (float)(c->frame_seed + 1u);
        r.frame_seed2 = (float)(c->frame_seed + 2u);
        c->frame_seed += 2u;
        r.out_rgba32f = c->st.sample;
        r.out_depth = c->st.depth;
        sc.add(gs::launch_raster_stochastic2(r, c->stream));
    }
    StageScope sa(c, ST_ACCUM);
    const uint32_t w = c->accum_write_index & 1u, rd = w ^ 1u;
    const bool has_history = c->taa_prev_valid && prev_valid;
    const gs::TaaUniforms u = taa_uniforms(cam, prev_cam, inv_view, has_history, cam_changed);
    // the TAA pass also writes the denoiser's input features
    sa.add(gs::launch_taa(c->st.sample, c->st.depth, c->st.accum[rd], c->st.xyz[rd], c->width, c->height, u,
                          c->st.accum[w], c->st.xyz[w], c->stream, c->features));
    c->taa_prev_valid = true;
    c->sample_count++;
    c->accum_write_index = w ^ 1u;
    return GS_OK;
}

// Denoised stochastic mode: the denoiser's estimate of the sorted-alpha
// frame; tiles whose estimated error exceeds the budget are rendered again
// by the sorted-alpha rasterizer from the same tile lists.
int render_denoised(gs_ctx* c, const gs_camera* cam, uint16_t* out) {
    if (!c->denoiser) return fail(c, GS_ERR_BAD_ARG, "denoised mode needs a denoiser (gs_set_denoiser)");
    if ((c->width & 1) || (c->height & 1)) return fail(c, GS_ERR_BAD_ARG, "denoised mode needs an even viewport");
    int rc = render_denoise_inputs(c, cam);
    if (rc) return rc;
    {
        StageScope sd(c, ST_DENOISE);
        // the network, its last layer writing the frame and the tiles' error estimates
        rc = gs::dn::forward_frame(c->denoiser, c->features, c->height, c->width, out, c->tiles_x,
                                   c->denoise_fallback ? c->denoise_budget : 3.0e38f, &c->fc->fallback_tiles,
                                   c->fallback_tiles, c->tile_error, c->stream);
        if (rc) return fail(c, rc, "denoiser forward failed");
        sd.add(5);
    }
    if (c->denoise_fallback) {
        StageScope sc(c, ST_RASTER);
        gs::RasterParams r = raster_params(c, background(c));
        r.tile_order = c->fallback_tiles;
        r.tile_count = &c->fc->fallback_tiles;
        r.out_rgba16f = out;
        sc.add(gs::launch_raster_alpha(r, c->stream));
    }
    return GS_OK;
}

int render_gps(gs_ctx* c, const gs_camera* cam, uint16_t* out) {
    int rc = gs::ensure_stochastic_targets(c->st, c->width, c->height, c->stream);
    if (rc) return fail(c, rc, "stochastic target allocation failed");
    uint32_t ss = std::max(1u, std::min(4u, c->knobs.gps_supersample_factor));
    rc = gs::ensure_gps_targets(c->gps, c->width, c->height, ss, c->n, c->gps_max_work_items, c->stream);
    if (rc) return fail(c, rc, "GPS target allocation failed");
    const size_t npix = (size_t)c->width * c->height;
    // src/renderer.cpp:2206-2211
    if (c->prev_cam_valid && std::memcmp(&c->prev_cam, cam, sizeof(gs_camera)) != 0) {
        c->sample_count = 0;
        c->taa_prev_valid = false;
    }
    c->prev_cam = *cam;
    c->prev_cam_valid = true;
    c->frame_seed++;
    run_cull(c);
    {
        StageScope sc(c, ST_GPS);
        gs::GpsParams g{};
        g.projected = c->projected;
        g.vis_ids = c->ids[1];
        g.fc = c->fc;
        g.width = c->width;
        g.height = c->height;
        g.supersample = ss;
        g.max_work_items = c->gps_max_work_items;
        g.clip_z_01 = cam->clip_z_01;
        g.linear_color = c->knobs.linear_color;
        g.frame_seed = (float)c->frame_seed;
        g.bg = background(c);
        g.out_color = c->st.sample;
        g.out_depth = c->st.depth;
        sc.add(gs::launch_gps(c->gps, g, c->n, c->num_sms, c->stream));
    }
    StageScope sa(c, ST_ACCUM);
    if (!c->knobs.stochastic_accumulation_enabled) {
        c->sample_count = 0;
        c->st.display = c->st.sample;
    } else {
        uint32_t w = c->accum_write_index & 1u, rd = w ^ 1u;
        uint32_t next = c->sample_count + 1;
        sa.add(gs::launch_accum(c->st.sample, next == 1 ? c->st.sample : c->st.accum[rd], (float)next, c->st.accum[w],
                                npix, c->stream));
        c->sample_count = next;
        c->accum_write_index = w ^ 1u;
        c->st.display = c->st.accum[w];
    }
    sa.add(gs::launch_to_half(c->st.display, out, npix, c->stream));
    return GS_OK;
}

}  // namespace

namespace {
std::atomic<int64_t> g_fail_alloc_countdown{-1};   // allocations to let pass before one fails; -1: off
}  // namespace

namespace gs {
cudaError_t device_malloc(void** p, size_t bytes) {
    *p = nullptr;
    int64_t left = g_fail_alloc_countdown.load();
    while (left >= 0 && !g_fail_alloc_countdown.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 0) return cudaErrorMemoryAllocation;   // injected failure (once)
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();   // reported through the return value only
        *p = nullptr;
    }
    return e;
}
}  // namespace gs

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int gs_debug_fail_alloc(int64_t after) {
    g_fail_alloc_countdown.store(after < 0 ? -1 : after);
    return GS_OK;
}

const char* gs_status_str(int s) {
    switch (s) {
        case GS_OK: return "ok";
        case GS_ERR_BAD_ARG: return "bad argument";
        case GS_ERR_OOM: return "out of memory";
        case GS_ERR_CUDA: return "CUDA error";
        case GS_ERR_DEVICE_TIMEOUT: return "device wait limit reached";
        case GS_ERR_NO_SCENE: return "no scene uploaded";
        case GS_ERR_BUDGET_REFUSED: return "GPS budget resize refused";
        case GS_ERR_NO_DEVICE: return "no CUDA device";
        case GS_ERR_TOO_LARGE: return "size beyond limit";
        case GS_ERR_FORMAT: return "not a valid asset";
        default: return "unknown status";
    }
}

const char* gs_last_error(const gs_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

const char* gs_stage_names(void) { return kStageNames; }

int gs_create(gs_ctx** out, int device, void* stream) {
    if (!out) return GS_ERR_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return GS_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return GS_ERR_BAD_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GS_ERR_NO_DEVICE;
    gs_ctx* c = new (std::nothrow) gs_ctx();
    if (!c) return GS_ERR_OOM;
    c->device = device;
    c->stream = static_cast<cudaStream_t>(stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    c->num_sms = sms > 0 ? (uint32_t)sms : 148u;
    // renderer_init defaults (src/renderer.cpp:588-599)
    c->knobs.render_mode = GS_MODE_GPS;
    c->knobs.sh_degree = 3;
    c->knobs.sh_lod_distance = 0.0f;
    c->knobs.gps_supersample_factor = 2;
    c->knobs.stochastic_samples_per_frame = 1;
    c->knobs.stochastic_taa_current_samples = 4;
    c->knobs.stochastic_accumulation_enabled = 1;
    c->knobs.stochastic_taa_enabled = 1;
    c->knobs.black_background = 0;
    c->knobs.splat_diagnostics_enabled = 0;
    c->knobs.linear_color = 0;
    c->knobs.write_invisible_records = 0;
    if (cudaMallocHost(reinterpret_cast<void**>(&c->h_fc), sizeof(FrameCounters)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&c->h_bin_fc), sizeof(FrameCounters)) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->fc_event, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->bin_event, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->binned, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->frame_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ctrl_read, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->alt.read, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->fc_stream, cudaStreamNonBlocking) != cudaSuccess) {
        gs_destroy(c);
        return GS_ERR_OOM;
    }
    std::memset(c->h_fc, 0, sizeof(FrameCounters));
    std::memset(c->h_bin_fc, 0, sizeof(FrameCounters));
    *out = c;
    return GS_OK;
}

void gs_destroy(gs_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->fc_stream) cudaStreamSynchronize(c->fc_stream);
    release_scene(c);
    release_targets(c);
    dfree(c->display_lut);
    if (c->h_fc) cudaFreeHost(c->h_fc);
    if (c->h_bin_fc) cudaFreeHost(c->h_bin_fc);
    if (c->h_slot_fc) cudaFreeHost(c->h_slot_fc);
    if (c->h_batch_params) cudaFreeHost(c->h_batch_params);
    if (c->h_batch_first) cudaFreeHost(c->h_batch_first);
    dfree(c->batch_params);
    dfree(c->batch_first);
    if (c->batch_event) cudaEventDestroy(c->batch_event);
    if (c->params_event) cudaEventDestroy(c->params_event);
    if (c->h_out16) cudaFreeHost(c->h_out16);
    for (auto e : c->chunk_events)
        if (e) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    for (auto& ss : c->sslot) {
        dfree(ss.image);
        if (ss.h_fc) cudaFreeHost(ss.h_fc);
        if (ss.rendered) cudaEventDestroy(ss.rendered);
        if (ss.copied) cudaEventDestroy(ss.copied);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->fc_event) cudaEventDestroy(c->fc_event);
    if (c->bin_event) cudaEventDestroy(c->bin_event);
    for (cudaEvent_t e : {c->binned, c->frame_done, c->ctrl_read, c->alt.read})
        if (e) cudaEventDestroy(e);
    if (c->fc_stream) cudaStreamDestroy(c->fc_stream);
    for (auto& p : c->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    delete c;
}

int gs_get_knobs(const gs_ctx* c, gs_knobs* out) {
    if (!c || !out) return GS_ERR_BAD_ARG;
    *out = c->knobs;
    return GS_OK;
}

int gs_set_knobs(gs_ctx* c, const gs_knobs* k) {
    if (!c || !k) return GS_ERR_BAD_ARG;
    if (k->render_mode < 0 || k->render_mode > 3 || k->sh_degree < 0 || k->sh_degree > 3)
        return fail(c, GS_ERR_BAD_ARG, "knob out of range");
    const bool reset = k->render_mode != c->knobs.render_mode ||
                       k->gps_supersample_factor != c->knobs.gps_supersample_factor ||
                       k->black_background != c->knobs.black_background || k->sh_degree != c->knobs.sh_degree ||
                       k->stochastic_taa_enabled != c->knobs.stochastic_taa_enabled ||
                       k->linear_color != c->knobs.linear_color;
    c->knobs = *k;
    if (reset) gs_reset_accumulation(c);
    return GS_OK;
}

int gs_set_mode(gs_ctx* c, int mode) {
    if (!c || mode < 0 || mode > 3) return GS_ERR_BAD_ARG;
    gs_knobs k = c->knobs;
    k.render_mode = mode;
    return gs_set_knobs(c, &k);
}

int gs_set_denoiser(gs_ctx* c, gs_denoiser* d) {
    if (!c) return GS_ERR_BAD_ARG;
    c->denoiser = d;
    return GS_OK;
}

int gs_set_denoise_budget(gs_ctx* c, float tile_mse, int fallback) {
    if (!c || !(tile_mse >= 0.0f)) return GS_ERR_BAD_ARG;
    c->denoise_budget = tile_mse;
    c->denoise_fallback = fallback ? 1 : 0;
    return GS_OK;
}

int gs_reset_accumulation(gs_ctx* c) {
    if (!c) return GS_ERR_BAD_ARG;
    // src/renderer.cpp renderer_reset_stochastic_accumulation
    c->sample_count = 0;
    c->accum_write_index = 0;
    c->prev_cam_valid = false;
    c->taa_prev_valid = false;
    return GS_OK;
}

static int upload_common(gs_ctx* c, const float* rows, uint64_t count, cudaMemcpyKind kind) {
    if (!c || (!rows && count)) return GS_ERR_BAD_ARG;
    if (count == 0) return fail(c, GS_ERR_BAD_ARG, "empty scene");  // src/renderer.cpp:757
    if (count > (1ull << 30) - 1) return fail(c, GS_ERR_TOO_LARGE, "more than 2^30-1 Gaussians");
    cudaSetDevice(c->device);
    const uint32_t n = (uint32_t)count;
    {   // src/renderer.cpp:739-763: refuse before touching the resident scene
        const MemoryLimits lim = memory_limits(c);
        const uint64_t need = scene_device_bytes(n, std::max(c->gps_max_work_items, 1u));
        const uint64_t budget = std::min(lim.scene_cap, lim.allocation_budget);
        if (need > budget)
            return fail(c, GS_ERR_TOO_LARGE, "scene needs " + mib(need) + " of device memory; budget " + mib(budget));
    }
    cudaStreamSynchronize(c->stream);
    release_scene(c);
    const bool half = c->row_format == 1;
    const size_t row_bytes = half ? (size_t)gs::kHalfRowChunks * 16 : 256;
    c->half_rows = half ? 1 : 0;
    GS_CUDA(c, dalloc(&c->rows, (size_t)n * row_bytes));
    GS_CUDA(c, dalloc(&c->heads, (size_t)n * 16));
    GS_CUDA(c, dalloc(&c->projected, (size_t)n * 64));
    for (int k = 0; k < 2; ++k) {
        GS_CUDA(c, dalloc(&c->keys[k], (size_t)n * 4));
        GS_CUDA(c, dalloc(&c->ids[k], (size_t)n * 4));
    }
    GS_CUDA(c, dalloc(&c->records, (size_t)n * sizeof(RasterRecord)));
    GS_CUDA(c, dalloc(&c->item_info, (size_t)n * sizeof(uint4)));
    const size_t cull_tiles = ((size_t)n + gs::kCullVisTile - 1) / gs::kCullVisTile;
    GS_CUDA(c, dalloc(&c->cull_status, cull_tiles * sizeof(unsigned long long)));
    c->sort_status_stride = gs::sort_status_words(n);
    GS_CUDA(c, dalloc(&c->sort_status, c->sort_status_stride * 4 * sizeof(unsigned long long)));
    const size_t bin_tiles = ((size_t)n + gs::kBinTile - 1) / gs::kBinTile;
    GS_CUDA(c, dalloc(&c->bin_status, bin_tiles * sizeof(unsigned long long)));
    GS_CUDA(c, cudaMemsetAsync(c->cull_status, 0, cull_tiles * 8, c->stream));
    GS_CUDA(c, cudaMemsetAsync(c->sort_status, 0, c->sort_status_stride * 4 * 8, c->stream));
    GS_CUDA(c, cudaMemsetAsync(c->bin_status, 0, bin_tiles * 8, c->stream));
    GS_CUDA(c, cudaMemsetAsync(c->projected, 0, (size_t)n * 64, c->stream));
    if (half) {
        // the 256-byte rows pass through a temporary device copy into the FP16-SH rows
        float4* full = nullptr;
        GS_CUDA(c, dalloc(&full, (size_t)n * 256));
        cudaError_t e = cudaMemcpyAsync(full, rows, (size_t)n * 256, kind, c->stream);
        if (e == cudaSuccess) gs::launch_pack_half_rows(full, c->rows, n, c->num_sms, c->stream);
        cudaStreamSynchronize(c->stream);
        dfree(full);
        GS_CUDA(c, e);
    } else {
        GS_CUDA(c, cudaMemcpyAsync(c->rows, rows, (size_t)n * 256, kind, c->stream));
    }
    gs::launch_gather_heads(c->rows, c->heads, n, c->num_sms, c->stream, half ? gs::kHalfRowChunks : 16);
    GS_CUDA(c, cudaGetLastError());
    int rc = ensure_entries(c, default_entry_cap(n));
    if (rc) return rc;   // the scene stays unloaded: every buffer must exist before n is set
    c->n = n;
    GS_CUDA(c, cudaStreamSynchronize(c->stream));
    gs_reset_accumulation(c);
    return GS_OK;
}

int gs_upload_rows(gs_ctx* c, const float* rows, uint64_t count) {
    return upload_common(c, rows, count, cudaMemcpyHostToDevice);
}

int gs_upload_rows_device(gs_ctx* c, const float* rows, uint64_t count) {
    return upload_common(c, rows, count, cudaMemcpyDeviceToDevice);
}

int gs_upload_rows_range(gs_ctx* c, const float* rows, uint64_t first, uint64_t count) {
    if (!c || (!rows && count)) return GS_ERR_BAD_ARG;
    if (!c->n) return fail(c, GS_ERR_NO_SCENE, "upload the scene before replacing rows of it");
    if (first > c->n || count > c->n - first) return fail(c, GS_ERR_BAD_ARG, "row range beyond the scene");
    if (!count) return GS_OK;
    cudaSetDevice(c->device);
    // stream-ordered after the frames already queued, which read the old rows
    if (c->half_rows) {
        float4* full = nullptr;
        GS_CUDA(c, dalloc(&full, (size_t)count * 256));
        cudaError_t e = cudaMemcpyAsync(full, rows, count * 256, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            gs::launch_pack_half_rows(full, c->rows + first * gs::kHalfRowChunks, (uint32_t)count, c->num_sms,
                                      c->stream);
        cudaStreamSynchronize(c->stream);
        dfree(full);
        GS_CUDA(c, e);
        gs::launch_gather_heads(c->rows + first * gs::kHalfRowChunks, c->heads + first, (uint32_t)count, c->num_sms,
                                c->stream, gs::kHalfRowChunks);
    } else {
        GS_CUDA(c, cudaMemcpyAsync(c->rows + first * 16, rows, count * 256, cudaMemcpyHostToDevice, c->stream));
        gs::launch_gather_heads(c->rows + first * 16, c->heads + first, (uint32_t)count, c->num_sms, c->stream);
    }
    GS_CUDA(c, cudaGetLastError());
    GS_CUDA(c, cudaStreamSynchronize(c->stream));   // the caller may reuse `rows` on return
    gs_reset_accumulation(c);
    return GS_OK;
}

int gs_set_row_format(gs_ctx* c, int format) {
    if (!c || format < 0 || format > 1) return GS_ERR_BAD_ARG;
    c->row_format = format;
    return GS_OK;
}

int gs_upload_anim(gs_ctx* c, const int8_t* deltas, uint32_t num_states, const float* scales) {
    if (!c || (num_states && (!deltas || !scales))) return GS_ERR_BAD_ARG;
    if (!c->n) return fail(c, GS_ERR_NO_SCENE, "upload the Gaussians before their animation");
    if (c->half_rows && num_states) return fail(c, GS_ERR_BAD_ARG, "animation needs GpuGaussian (FP32) rows");
    cudaSetDevice(c->device);
    if (num_states) {   // the old animation stays when the new one is refused
        const MemoryLimits lim = memory_limits(c);
        const uint64_t add = anim_device_bytes(c->n, num_states);
        const uint64_t kept = scene_device_bytes(c->n, std::max(c->gps_max_work_items, 1u)) +
                              layer_device_bytes(c->n, c->layers_uploaded);
        if (add > lim.allocation_budget || kept + add > lim.scene_cap)
            return fail(c, GS_ERR_TOO_LARGE, "animation needs " + mib(add) + " of device memory beyond the budget");
    }
    cudaStreamSynchronize(c->stream);
    dfree(c->anim_deltas);
    dfree(c->anim_scales);
    c->anim_states = 0;
    c->anim_a = c->anim_b = 0;
    c->anim_w = 0.0f;
    if (num_states == 0) return GS_OK;
    const size_t bytes = (size_t)num_states * c->n * 48u;
    cudaError_t e = dalloc(&c->anim_deltas, bytes);
    if (e == cudaSuccess) e = dalloc(&c->anim_scales, 48 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->anim_deltas, deltas, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->anim_scales, scales, 48 * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {   // all or nothing: no half-uploaded animation stays behind
        dfree(c->anim_deltas);
        dfree(c->anim_scales);
        return cuda_fail(c, e, "animation upload");
    }
    c->anim_states = num_states;
    gs_reset_accumulation(c);
    return GS_OK;
}

int gs_set_anim_state(gs_ctx* c, int state_a, int state_b, float weight) {
    if (!c) return GS_ERR_BAD_ARG;
    if (state_a < 0 || state_b < 0 || (uint32_t)state_a > c->anim_states || (uint32_t)state_b > c->anim_states ||
        !(weight >= 0.0f && weight <= 1.0f))
        return fail(c, GS_ERR_BAD_ARG, "animation state out of range");
    // src/renderer.cpp:2148-2161: a changed sample resets accumulation
    if (state_a != c->anim_a || state_b != c->anim_b || weight != c->anim_w) gs_reset_accumulation(c);
    c->anim_a = state_a;
    c->anim_b = state_b;
    c->anim_w = weight;
    return GS_OK;
}

int gs_upload_layers(gs_ctx* c, const uint16_t* halves, uint32_t layer_count) {
    if (!c || (layer_count && !halves)) return GS_ERR_BAD_ARG;
    if (!c->n) return fail(c, GS_ERR_NO_SCENE, "upload the Gaussians before their layers");
    if (layer_count > 256) return fail(c, GS_ERR_TOO_LARGE, "more than 256 layers");
    if (c->half_rows && layer_count) return fail(c, GS_ERR_BAD_ARG, "appearance layers need GpuGaussian (FP32) rows");
    cudaSetDevice(c->device);
    if (layer_count) {   // the old layers stay when the new ones are refused
        const MemoryLimits lim = memory_limits(c);
        const uint64_t add = layer_device_bytes(c->n, layer_count);
        const uint64_t kept = scene_device_bytes(c->n, std::max(c->gps_max_work_items, 1u)) +
                              anim_device_bytes(c->n, c->anim_states);
        if (add > lim.allocation_budget || kept + add > lim.scene_cap)
            return fail(c, GS_ERR_TOO_LARGE, "layers need " + mib(add) + " of device memory beyond the budget");
    }
    cudaStreamSynchronize(c->stream);
    dfree(c->layer_halves);
    c->layers_uploaded = 0;
    c->layer_count = 0;
    c->layer_weights_host.clear();
    gs_reset_accumulation(c);
    if (layer_count == 0) return GS_OK;
    const size_t bytes = (size_t)layer_count * c->n * 48u * sizeof(uint16_t);
    cudaError_t e = dalloc(&c->layer_halves, bytes);
    if (e == cudaSuccess && !c->layer_weights) e = dalloc(&c->layer_weights, 256 * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->layer_halves, halves, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {   // all or nothing
        dfree(c->layer_halves);
        return cuda_fail(c, e, "layer upload");
    }
    c->layers_uploaded = layer_count;
    return GS_OK;
}

int gs_set_layer_weights(gs_ctx* c, const float* weights, uint32_t count) {
    if (!c || (count && !weights)) return GS_ERR_BAD_ARG;
    if (count > c->layers_uploaded) return fail(c, GS_ERR_BAD_ARG, "more layer weights than uploaded layers");
    std::vector<float> w(weights, weights + (size_t)count * 3);
    // src/renderer.cpp:2153-2155: a new playback position of a layered asset resets accumulation
    if (w != c->layer_weights_host) gs_reset_accumulation(c);
    c->layer_weights_host = w;
    c->layer_count = count;
    if (count) {
        cudaSetDevice(c->device);
        // from pageable memory: the source is copied before the call returns
        GS_CUDA(c, cudaMemcpyAsync(c->layer_weights, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice,
                                   c->stream));
    }
    return GS_OK;
}

int gs_set_gps_budget(gs_ctx* c, uint32_t max_work_items) {
    if (!c) return GS_ERR_BAD_ARG;
    if (max_work_items == 0) return fail(c, GS_ERR_BUDGET_REFUSED, "GPS budget must be >= 1");
    if (max_work_items == c->gps_max_work_items) return GS_OK;
    {   // src/renderer.cpp:1080-1092: the replacement against free memory, the scene against the cap
        cudaSetDevice(c->device);
        const MemoryLimits lim = memory_limits(c);
        const uint64_t add = (uint64_t)max_work_items * sizeof(uint2);
        const uint64_t total = scene_device_bytes(c->n, max_work_items) + anim_device_bytes(c->n, c->anim_states) +
                               layer_device_bytes(c->n, c->layers_uploaded);
        if (add > lim.allocation_budget || total > lim.scene_cap)
            return fail(c, GS_ERR_BUDGET_REFUSED, "GPS work buffer of " + mib(add) + " refused by the memory budget");
    }
    int rc = gs::resize_gps_work(c->gps, max_work_items, c->stream);
    if (rc) return fail(c, GS_ERR_BUDGET_REFUSED, "GPS work buffer resize refused; old budget kept");
    c->gps_max_work_items = max_work_items;
    gs_reset_accumulation(c);
    return GS_OK;
}

int gs_set_display_lut(gs_ctx* c, const uint16_t* lut, uint32_t lut_size, float log2_min, float log2_max) {
    if (!c) return GS_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    // a queued gs_display may still read the old table
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return cuda_fail(c, cudaGetLastError(), "stream sync");
    dfree(c->display_lut);
    c->lut_size = 0;
    if (!lut) return GS_OK;
    // src/gaussian_loader_gsanim.cpp:237,244
    if (lut_size < 2 || lut_size > 256) return fail(c, GS_ERR_BAD_ARG, "display LUT size must be 2..256");
    if (!(log2_min < log2_max)) return fail(c, GS_ERR_BAD_ARG, "display LUT needs log2_min < log2_max");
    const size_t count = (size_t)lut_size * lut_size * lut_size * 3;
    GS_CUDA(c, dalloc(&c->display_lut, count * sizeof(uint16_t)));
    GS_CUDA(c, cudaMemcpy(c->display_lut, lut, count * sizeof(uint16_t), cudaMemcpyHostToDevice));
    c->lut_size = (int)lut_size;
    c->lut_log2_min = log2_min;
    c->lut_log2_max = log2_max;
    return GS_OK;
}

int gs_display(gs_ctx* c, const uint16_t* rgba16f_in, float* rgba32f_out, int width, int height, float exposure_ev) {
    if (!c || !rgba16f_in || !rgba32f_out || width <= 0 || height <= 0) return GS_ERR_BAD_ARG;
    if (((uintptr_t)rgba16f_in & 7u) || ((uintptr_t)rgba32f_out & 15u))
        return fail(c, GS_ERR_BAD_ARG, "gs_display buffers must be 8-byte (input) and 16-byte (output) aligned");
    cudaSetDevice(c->device);
    gs::DisplayParams p{};
    p.in_rgba16f = rgba16f_in;
    p.out_rgba32f = reinterpret_cast<float4*>(rgba32f_out);
    p.width = width;
    p.height = height;
    p.lut = c->lut_size ? c->display_lut : nullptr;
    p.lut_size = c->lut_size;
    p.log2_min = c->lut_log2_min;
    p.log2_max = c->lut_log2_max;
    p.exposure_ev = exposure_ev;
    gs::launch_display(p, c->num_sms, c->stream);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GS_OK : cuda_fail(c, e, "display kernel launch");
}

int gs_debug_wait_probe(gs_ctx* c, int which, uint32_t spin_limit) {
    if (!c || which < 0 || which > 1 || spin_limit == 0) return GS_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    // private words: the frame's counters and status arrays stay untouched
    void* mem = nullptr;
    const size_t status_bytes = 64 * sizeof(unsigned long long);
    GS_CUDA(c, gs::device_malloc(&mem, status_bytes + sizeof(FrameCounters)));
    auto* status = static_cast<unsigned long long*>(mem);
    auto* fc = reinterpret_cast<FrameCounters*>(static_cast<char*>(mem) + status_bytes);
    cudaError_t e = cudaMemsetAsync(mem, 0, status_bytes + sizeof(FrameCounters), c->stream);
    if (e == cudaSuccess) {
        gs::launch_wait_probe(status, fc, /*epoch*/ 1u, which, spin_limit, c->stream);
        e = cudaGetLastError();
    }
    FrameCounters h{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, fc, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(mem);
    if (e != cudaSuccess) return cuda_fail(c, e, "wait probe");
    if (h.error_flags) return fail(c, GS_ERR_DEVICE_TIMEOUT, "a device-side wait ran out (probe)");
    return GS_OK;
}

// The image rules are GL's: window y from the bottom, depth clipped to
// [-1, 1] (src/main.cpp:1275-1281, the non-WGPU branch).  The WGPU branch
// (clip_y_sign -1, clip_z_01 1) rasterises with a top-left fragment origin,
// which no kernel here follows, so such a camera is refused instead of
// drawn wrongly.
static bool gl_clip_convention(const gs_camera* cam) {
    return cam->clip_y_sign == 1.0f && cam->clip_z_01 == 0.0f;
}

// Target size: the viewport rounded to whole pixels (src/renderer.cpp:2193-2196),
// range-checked as a float first so that NaN or huge viewports never reach
// the integer conversion.
static int viewport_dims(gs_ctx* c, const gs_camera* cam, int* w, int* h) {
    const float vw = cam->viewport[0] + 0.5f, vh = cam->viewport[1] + 0.5f;
    if (!(vw >= 1.0f && vh >= 1.0f)) return fail(c, GS_ERR_BAD_ARG, "viewport must be positive");
    if (vw >= 32768.0f || vh >= 32768.0f) return fail(c, GS_ERR_TOO_LARGE, "viewport beyond 32767 pixels");
    *w = (int)vw;
    *h = (int)vh;
    return GS_OK;
}

uint64_t gs_scene_device_bytes(uint64_t count, uint32_t gps_work_items) {
    if (count == 0 || count > (1ull << 30) - 1) return 0;
    return scene_device_bytes((uint32_t)count, std::max(gps_work_items, 1u));
}

int gs_render(gs_ctx* c, const gs_camera* cam, void* out) {
    if (!c || !cam || !out) return GS_ERR_BAD_ARG;
    if (!gl_clip_convention(cam)) return fail(c, GS_ERR_BAD_ARG, "only the GL clip convention is drawn");
    if (!c->n) return fail(c, GS_ERR_NO_SCENE, "no scene uploaded");
    cudaSetDevice(c->device);
    int w = 0, h = 0;
    int rc = viewport_dims(c, cam, &w, &h);
    if (rc) return rc;
    rc = ensure_targets(c, w, h);
    if (rc) return rc;
    rc = check_previous_frame(c);
    if (rc) return rc;
    if (!c->entry_cap) {   // a failed growth freed the entry buffers: no frame runs without them
        rc = ensure_entries(c, default_entry_cap(c->n));
        if (rc) return rc;
    }
    uint16_t* o = static_cast<uint16_t*>(out);
    // The (tile, splat) entries of a frame are counted on the device.  The
    // host reads the count back as soon as the binning has run (the rest of
    // the frame stays queued behind it) and, if the entries did not fit,
    // grows the buffers and renders the frame again, restoring the state a
    // frame advances; so a frame that returns GS_OK is never truncated.
    for (int attempt = 0;; ++attempt) {
        const uint32_t seed = c->frame_seed, samples = c->sample_count, widx = c->accum_write_index;
        const gs_camera pcam = c->prev_cam;
        const bool pvalid = c->prev_cam_valid, tvalid = c->taa_prev_valid;
        nvtxRangePushA("gs_render");
        begin_render_frame(c, cam);
        c->bin_recorded = false;
        switch (c->knobs.render_mode) {
            case GS_MODE_ALPHA: rc = render_alpha(c, o); break;
            case GS_MODE_STOCHASTIC: rc = render_stochastic(c, cam, o); break;
            case GS_MODE_DENOISED: rc = render_denoised(c, cam, o); break;
            default: rc = render_gps(c, cam, o); break;
        }
        end_frame(c);
        nvtxRangePop();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
        if (rc || !c->bin_recorded) return rc;
        GS_CUDA(c, cudaEventSynchronize(c->bin_event));
        const uint32_t over = c->h_bin_fc->tile_overflow;
        if (!over) return GS_OK;
        GS_CUDA(c, cudaStreamSynchronize(c->stream));
        c->fc_pending = false;
        const uint64_t need = (uint64_t)c->h_bin_fc->tile_entries + over;
        if (attempt >= 3 || c->entry_cap >= 0x3FFFFFFFu)
            return fail(c, GS_ERR_TOO_LARGE, "tile entries beyond the largest entry buffer: frame truncated");
        rc = ensure_entries(c, (uint32_t)std::min<uint64_t>(need + need / 4 + 1024, 0x3FFFFFFFull));
        if (rc) return rc;
        c->frame_seed = seed;
        c->sample_count = samples;
        c->accum_write_index = widx;
        c->prev_cam = pcam;
        c->prev_cam_valid = pvalid;
        c->taa_prev_valid = tvalid;
    }
}

int gs_render_host(gs_ctx* c, const gs_camera* cam, uint16_t* host_out) {
    if (!c || !cam || !host_out) return GS_ERR_BAD_ARG;
    if (!gl_clip_convention(cam)) return fail(c, GS_ERR_BAD_ARG, "only the GL clip convention is drawn");
    int w = 0, h = 0;
    int rc = viewport_dims(c, cam, &w, &h);
    if (rc) return rc;
    rc = ensure_targets(c, w, h);
    if (rc) return rc;
    const size_t bytes = (size_t)w * h * 8;
    // A page-locked destination is written by the copy engine directly;
    // a pageable one goes through the context's pinned staging buffer.
    cudaPointerAttributes pa{};
    const bool pinned_out = cudaPointerGetAttributes(&pa, host_out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();   // a pageable pointer may leave an error to clear on older drivers
    if (!pinned_out && c->h_out16_bytes < bytes) {
        if (c->h_out16) cudaFreeHost(c->h_out16);
        c->h_out16 = nullptr;
        c->h_out16_bytes = 0;
        GS_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(&c->h_out16), bytes));
        c->h_out16_bytes = bytes;
    }
    // Alpha frames into page-locked memory: the rasterizer writes the pixels
    // straight into the host buffer (mapped, over PCIe), so the transfer
    // overlaps the raster instead of following it.  gs_render grows the tile
    // entries and re-renders the frame itself when they overflow.
    void* mapped = nullptr;
    const bool direct = pinned_out && c->knobs.render_mode == GS_MODE_ALPHA &&
                        cudaHostGetDevicePointer(&mapped, host_out, 0) == cudaSuccess && mapped;
    cudaGetLastError();
    rc = gs_render(c, cam, direct ? mapped : static_cast<void*>(c->out16));
    if (rc) return rc;
    if (direct) {
        GS_CUDA(c, cudaStreamSynchronize(c->stream));   // written by the frame's kernels
    } else if (pinned_out) {
        GS_CUDA(c, cudaMemcpyAsync(host_out, c->out16, bytes, cudaMemcpyDeviceToHost, c->stream));
        GS_CUDA(c, cudaStreamSynchronize(c->stream));
    } else {
        // eight chunks, each with an event, so the host copies chunk i out of
        // the staging buffer while the copy engine brings in chunk i + 1
        for (int k = 0; k < 8; ++k) {
            if (!c->chunk_events[k])
                GS_CUDA(c, cudaEventCreateWithFlags(&c->chunk_events[k], cudaEventDisableTiming));
            const size_t b0 = bytes * k / 8, b1 = bytes * (k + 1) / 8;
            GS_CUDA(c, cudaMemcpyAsync(reinterpret_cast<char*>(c->h_out16) + b0,
                                       reinterpret_cast<const char*>(c->out16) + b0, b1 - b0,
                                       cudaMemcpyDeviceToHost, c->stream));
            GS_CUDA(c, cudaEventRecord(c->chunk_events[k], c->stream));
        }
        for (int k = 0; k < 8; ++k) {
            const size_t b0 = bytes * k / 8, b1 = bytes * (k + 1) / 8;
            GS_CUDA(c, cudaEventSynchronize(c->chunk_events[k]));
            std::memcpy(reinterpret_cast<char*>(host_out) + b0, reinterpret_cast<const char*>(c->h_out16) + b0,
                        b1 - b0);
        }
    }
    GS_CUDA(c, cudaEventSynchronize(c->fc_event));
    c->fc_pending = false;
    if (c->h_fc->error_flags & ~(uint32_t)gs::kErrTileOverflow)
        return fail(c, GS_ERR_DEVICE_TIMEOUT, "a device-side wait ran out");
    return GS_OK;
}

// Waits for the copy of a streamed frame and frees its slot; the frame's
// device-side waits are checked on the counters it read back.
static int retire_stream_slot(gs_ctx* c, gs_ctx::StreamSlot& ss) {
    if (!ss.host) return GS_OK;
    ss.host = nullptr;
    GS_CUDA(c, cudaEventSynchronize(ss.copied));
    if (ss.h_fc->error_flags & ~(uint32_t)gs::kErrTileOverflow)
        return fail(c, GS_ERR_DEVICE_TIMEOUT, "a device-side wait ran out");
    return GS_OK;
}

int gs_render_host_submit(gs_ctx* c, const gs_camera* cam, uint16_t* host_out) {
    if (!c || !cam || !host_out) return GS_ERR_BAD_ARG;
    if (!gl_clip_convention(cam)) return fail(c, GS_ERR_BAD_ARG, "only the GL clip convention is drawn");
    cudaSetDevice(c->device);
    int w = 0, h = 0;
    int rc = viewport_dims(c, cam, &w, &h);
    if (rc) return rc;
    const size_t bytes = (size_t)w * h * 8;
    cudaPointerAttributes pa{};
    const bool pinned_out = cudaPointerGetAttributes(&pa, host_out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (!pinned_out) return fail(c, GS_ERR_BAD_ARG, "gs_render_host_submit needs a page-locked destination");
    if (!c->copy_stream) GS_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    // a destination still in flight is delivered before it is written again
    int first_err = GS_OK;
    for (auto& o : c->sslot)
        if (o.host == host_out) {
            rc = retire_stream_slot(c, o);
            if (rc && !first_err) first_err = rc;
        }
    gs_ctx::StreamSlot& ss = c->sslot[c->sslot_next];
    rc = retire_stream_slot(c, ss);   // the older frame: at most two in flight
    if (rc && !first_err) first_err = rc;
    if (first_err) return first_err;
    if (!ss.h_fc) {
        GS_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(&ss.h_fc), sizeof(FrameCounters)));
        std::memset(ss.h_fc, 0, sizeof(FrameCounters));
    }
    if (!ss.rendered) GS_CUDA(c, cudaEventCreateWithFlags(&ss.rendered, cudaEventDisableTiming));
    if (!ss.copied) GS_CUDA(c, cudaEventCreateWithFlags(&ss.copied, cudaEventDisableTiming));
    if (ss.bytes < bytes) {
        dfree(ss.image);
        ss.image = nullptr;
        ss.bytes = 0;
        const cudaError_t e = dalloc(&ss.image, bytes);
        if (e != cudaSuccess) return cuda_fail(c, e, "dalloc(stream image)");
        ss.bytes = bytes;
    }
    c->fc_extra = ss.h_fc;   // the frame's counters, copied on fc_stream by end_frame
    rc = gs_render(c, cam, ss.image);
    c->fc_extra = nullptr;
    if (rc) return rc;
    GS_CUDA(c, cudaEventRecord(ss.rendered, c->stream));
    GS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ss.rendered, 0));
    GS_CUDA(c, cudaMemcpyAsync(host_out, ss.image, bytes, cudaMemcpyDeviceToHost, c->copy_stream));
    GS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, c->fc_event, 0));   // ss.copied covers the counters too
    GS_CUDA(c, cudaEventRecord(ss.copied, c->copy_stream));
    ss.host = host_out;
    c->sslot_next ^= 1;
    return GS_OK;
}

int gs_render_host_wait(gs_ctx* c, const uint16_t* host_out) {
    if (!c) return GS_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    int first_err = GS_OK;
    for (int k = 0; k < 2; ++k) {   // oldest first
        gs_ctx::StreamSlot& ss = c->sslot[(c->sslot_next + k) & 1];
        if (!ss.host || (host_out && ss.host != host_out)) continue;
        const int rc = retire_stream_slot(c, ss);
        if (rc && !first_err) first_err = rc;
    }
    return first_err;
}

int gs_render_features(gs_ctx* c, const gs_camera* cam, void* features_out) {
    if (!c || !cam || !features_out) return GS_ERR_BAD_ARG;
    if (!gl_clip_convention(cam)) return fail(c, GS_ERR_BAD_ARG, "only the GL clip convention is drawn");
    if (!c->n) return fail(c, GS_ERR_NO_SCENE, "no scene uploaded");
    cudaSetDevice(c->device);
    int w = 0, h = 0;
    int rc = viewport_dims(c, cam, &w, &h);
    if (rc) return rc;
    if ((w & 1) || (h & 1)) return fail(c, GS_ERR_BAD_ARG, "the denoiser input needs an even viewport");
    if ((rc = ensure_targets(c, w, h))) return rc;
    if ((rc = check_previous_frame(c))) return rc;
    if (!c->entry_cap && (rc = ensure_entries(c, default_entry_cap(c->n)))) return rc;
    for (int attempt = 0;; ++attempt) {
        const uint32_t seed = c->frame_seed, samples = c->sample_count, widx = c->accum_write_index;
        const gs_camera pcam = c->prev_cam;
        const bool pvalid = c->prev_cam_valid, tvalid = c->taa_prev_valid;
        begin_render_frame(c, cam);
        c->bin_recorded = false;
        rc = render_denoise_inputs(c, cam);
        end_frame(c);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
        if (rc) return rc;
        GS_CUDA(c, cudaEventSynchronize(c->bin_event));
        const uint32_t over = c->h_bin_fc->tile_overflow;
        if (!over) break;
        GS_CUDA(c, cudaStreamSynchronize(c->stream));
        if (attempt >= 3 || c->entry_cap >= 0x3FFFFFFFu)
            return fail(c, GS_ERR_TOO_LARGE, "tile entries beyond the largest entry buffer: frame truncated");
        const uint64_t need = (uint64_t)c->h_bin_fc->tile_entries + over;
        if ((rc = ensure_entries(c, (uint32_t)std::min<uint64_t>(need + need / 4 + 1024, 0x3FFFFFFFull)))) return rc;
        c->frame_seed = seed;
        c->sample_count = samples;
        c->accum_write_index = widx;
        c->prev_cam = pcam;
        c->prev_cam_valid = pvalid;
        c->taa_prev_valid = tvalid;
    }
    GS_CUDA(c, cudaMemcpyAsync(features_out, c->features, c->features_pix * gs::dn::kInC * sizeof(__nv_bfloat16),
                               cudaMemcpyDeviceToDevice, c->stream));
    return GS_OK;
}

// ---- batches ---------------------------------------------------------------
namespace {

constexpr uint32_t kMaxBatch = 256;

int ensure_batch(gs_ctx* c, uint32_t count) {
    if (c->slots.size() < count) c->slots.resize(count);
    if (c->batch_cap >= count) return GS_OK;
    if (c->h_slot_fc) cudaFreeHost(c->h_slot_fc);
    if (c->h_batch_params) cudaFreeHost(c->h_batch_params);
    if (c->h_batch_first) cudaFreeHost(c->h_batch_first);
    c->h_slot_fc = nullptr;
    c->h_batch_params = nullptr;
    c->h_batch_first = nullptr;
    dfree(c->batch_params);
    dfree(c->batch_first);
    c->batch_cap = 0;
    GS_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(&c->h_slot_fc), kMaxBatch * sizeof(FrameCounters)));
    GS_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(&c->h_batch_params), kMaxBatch * sizeof(gs::RasterParams)));
    GS_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(&c->h_batch_first), (kMaxBatch + 2) * sizeof(uint32_t)));
    GS_CUDA(c, dalloc(&c->batch_params, kMaxBatch * sizeof(gs::RasterParams)));
    GS_CUDA(c, dalloc(&c->batch_first, (kMaxBatch + 2) * sizeof(uint32_t)));
    if (!c->batch_event) GS_CUDA(c, cudaEventCreateWithFlags(&c->batch_event, cudaEventDisableTiming));
    if (!c->params_event) GS_CUDA(c, cudaEventCreateWithFlags(&c->params_event, cudaEventDisableTiming));
    c->batch_cap = kMaxBatch;
    return GS_OK;
}

// Make slot f (swapped into the context) ready for a w x h frame of the scene.
int prepare_slot(gs_ctx* c, int w, int h, int tw, int th, bool fresh_records) {
    if (c->width != w || c->height != h || !c->ctrl || c->tile_w != tw || c->tile_h != th) {
        dfree(c->ctrl);
        dfree(c->tile_order);
        c->width = c->height = 0;
        int rc = alloc_control(c, w, h, tw, th, /*with_alt*/ false);
        if (rc) return rc;
    }
    if (fresh_records || !c->records) {
        dfree(c->records);
        GS_CUDA(c, dalloc(&c->records, (size_t)c->n * sizeof(RasterRecord)));
    }
    if (!c->entry_cap) return ensure_entries(c, default_entry_cap(c->n));
    return GS_OK;
}

// The cull, depth sort and binning of frame k into slot k, and its raster
// parameters; the slot's counters are read back into h_slot_fc[k].
int stage_frame(gs_ctx* c, uint32_t k, const gs_camera* cam, void* out) {
    if (c->params_pending) {   // the pinned parameters of the last launch are copied before they are rewritten
        GS_CUDA(c, cudaEventSynchronize(c->params_event));
        c->params_pending = false;
    }
    FrameSlot& f = c->slots[k];
    const int tw = c->alpha_tile_w, th = c->alpha_tile_h;
    swap_slot(c, f);
    int w = 0, h = 0;
    int rc = viewport_dims(c, cam, &w, &h);
    if (!rc) rc = prepare_slot(c, w, h, tw, th, false);
    if (!rc) {
        begin_frame(c, cam);
        run_cull(c);
        run_depth_sort(c);
        run_binning(c, 0.0f, 0.0f, 0.0f, false, /*readback*/ false);
        // on fc_stream: a copy between two kernels would idle the render stream
        cudaEventRecord(c->binned, c->stream);
        cudaStreamWaitEvent(c->fc_stream, c->binned, 0);
        cudaMemcpyAsync(&c->h_slot_fc[k], c->fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, c->fc_stream);
        gs::RasterParams r = raster_params(c, background(c));
        r.out_rgba16f = static_cast<uint16_t*>(out);
        c->h_batch_params[k] = r;
    }
    swap_slot(c, f);
    return rc;
}

// Grow the entries of every slot whose binning overflowed; returns the
// number of such slots (< 0: error).
int grow_overflowed(gs_ctx* c, uint32_t count, std::vector<uint32_t>& redo) {
    GS_CUDA(c, cudaEventRecord(c->batch_event, c->stream));
    GS_CUDA(c, cudaEventSynchronize(c->batch_event));
    GS_CUDA(c, cudaStreamSynchronize(c->fc_stream));   // the slots' counters
    redo.clear();
    for (uint32_t k = 0; k < count; ++k) {
        const FrameCounters& fc = c->h_slot_fc[k];
        if (!fc.tile_overflow) continue;
        FrameSlot& f = c->slots[k];
        if (f.entry_cap >= 0x3FFFFFFFu) return fail(c, GS_ERR_TOO_LARGE, "tile entries beyond the largest buffer");
        const uint64_t need = (uint64_t)fc.tile_entries + fc.tile_overflow;
        swap_slot(c, f);
        const int rc = ensure_entries(c, (uint32_t)std::min<uint64_t>(need + need / 4 + 1024, 0x3FFFFFFFull));
        swap_slot(c, f);
        if (rc) return rc;
        redo.push_back(k);
    }
    return GS_OK;
}

int raster_batch(gs_ctx* c, uint32_t count) {
    uint32_t total = 0;
    for (uint32_t k = 0; k < count; ++k) {
        c->h_batch_first[k] = total;
        total += (uint32_t)c->h_batch_params[k].tiles_x * (uint32_t)c->h_batch_params[k].tiles_y;
    }
    c->h_batch_first[count] = total;
    c->h_batch_first[count + 1] = 0;   // the work ticket
    GS_CUDA(c, cudaMemcpyAsync(c->batch_params, c->h_batch_params, count * sizeof(gs::RasterParams),
                               cudaMemcpyHostToDevice, c->stream));
    GS_CUDA(c, cudaMemcpyAsync(c->batch_first, c->h_batch_first, (count + 2) * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, c->stream));
    GS_CUDA(c, cudaEventRecord(c->params_event, c->stream));
    c->params_pending = true;
    static int blocks_per_sm = 0;
    if (!blocks_per_sm) {
        int b = 0;
        gs::raster_batch_occupancy(&b);
        blocks_per_sm = b > 0 ? b : 1;
    }
    StageScope sc(c, ST_RASTER);
    sc.add(gs::launch_raster_batch_alpha(c->batch_params, c->batch_first, count, c->batch_first + count + 1,
                                         c->num_sms * (uint32_t)blocks_per_sm, c->h_batch_params[0].tile_w,
                                         c->stream));
    return GS_OK;
}

int batch_checks(gs_ctx* c, uint32_t count) {
    if (!c->n) return fail(c, GS_ERR_NO_SCENE, "no scene uploaded");
    if (count > kMaxBatch) return fail(c, GS_ERR_TOO_LARGE, "more than 256 frames in a batch");
    if (c->knobs.render_mode != GS_MODE_ALPHA) return fail(c, GS_ERR_BAD_ARG, "batches render the alpha mode");
    return GS_OK;
}

}  // namespace

int gs_render_batch(gs_ctx* c, const gs_camera* cams, uint32_t count, void* const* outs) {
    if (!c || (count && (!cams || !outs))) return GS_ERR_BAD_ARG;
    for (uint32_t k = 0; k < count; ++k) {
        if (!outs[k]) return GS_ERR_BAD_ARG;
        if (!gl_clip_convention(&cams[k])) return fail(c, GS_ERR_BAD_ARG, "only the GL clip convention is drawn");
    }
    int rc = batch_checks(c, count);
    if (rc || !count) return rc;
    cudaSetDevice(c->device);
    const uint32_t depth = c->batch_depth ? std::min(c->batch_depth, count) : count;
    if ((rc = ensure_batch(c, depth))) return rc;
    nvtxRangePushA("gs_render_batch");
    c->frame_launches = 0;
    std::vector<uint32_t> redo;
    // frames in chunks of `depth`: the stages of a chunk's frames into its
    // slots, then one persistent raster launch for the chunk
    for (uint32_t k0 = 0; k0 < count && !rc; k0 += depth) {
        const uint32_t m = std::min(depth, count - k0);
        redo.resize(m);
        for (uint32_t k = 0; k < m; ++k) redo[k] = k;
        for (int attempt = 0; !redo.empty() && !rc; ++attempt) {
            if (attempt > 3) {
                rc = fail(c, GS_ERR_TOO_LARGE, "tile entries still overflowing");
                break;
            }
            for (uint32_t k : redo)
                if ((rc = stage_frame(c, k, &cams[k0 + k], outs[k0 + k]))) break;
            if (!rc) rc = grow_overflowed(c, m, redo);
        }
        if (!rc) rc = raster_batch(c, m);
        if (!rc) {
            // the statistics of the batch's last frame
            cudaStreamWaitEvent(c->stream, c->fc_event, 0);   // after gs_render's copy of h_fc
            cudaMemcpyAsync(c->h_fc, c->slots[m - 1].fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, c->stream);
            cudaEventRecord(c->fc_event, c->stream);
        }
    }
    c->fc_pending = false;
    c->last_launches = c->frame_launches;
    nvtxRangePop();
    if (rc) return rc;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return GS_OK;
}

int gs_set_tile_shape(gs_ctx* c, int tile_w, int tile_h) {
    if (!c) return GS_ERR_BAD_ARG;
    const bool ok = (tile_w == 16 && tile_h == 16) || (tile_w == 32 && tile_h == 8) || (tile_w == 8 && tile_h == 32);
    if (!ok) return fail(c, GS_ERR_BAD_ARG, "tile shapes: 16x16, 32x8, 8x32");
    c->alpha_tile_w = tile_w;
    c->alpha_tile_h = tile_h;
    return GS_OK;
}

int gs_set_batch_depth(gs_ctx* c, uint32_t depth) {
    if (!c || depth > kMaxBatch) return GS_ERR_BAD_ARG;
    c->batch_depth = depth;
    return GS_OK;
}

int gs_autotune_batch(gs_ctx* c, const gs_camera* cams, uint32_t count, void* const* outs, gs_tune_result* res) {
    if (!c || !cams || !outs || !count) return GS_ERR_BAD_ARG;
    int rc = batch_checks(c, count);
    if (rc) return rc;
    static const int shapes[3][2] = {{16, 16}, {32, 8}, {8, 32}};
    static const uint32_t depths[6] = {4, 8, 16, 32, 64, 128};
    const int keep_w = c->alpha_tile_w, keep_h = c->alpha_tile_h;
    const uint32_t keep_d = c->batch_depth;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GS_CUDA(c, cudaEventCreate(&e0));
    GS_CUDA(c, cudaEventCreate(&e1));
    gs_tune_result r{};
    r.best_ms = 3.0e38f;
    int tried = 0;
    for (int si = 0; si < 3 && !rc; ++si) {
        for (int di = 0; di < 6 && !rc; ++di) {
            const uint32_t d = depths[di];
            if (d > count && di > 0 && depths[di - 1] >= count) break;
            c->alpha_tile_w = shapes[si][0];
            c->alpha_tile_h = shapes[si][1];
            c->batch_depth = std::min(d, count);
            if ((rc = gs_render_batch(c, cams, count, outs))) break;   // warm-up (and slot allocation)
            cudaEventRecord(e0, c->stream);
            for (int rep = 0; rep < 2 && !rc; ++rep) rc = gs_render_batch(c, cams, count, outs);
            cudaEventRecord(e1, c->stream);
            if (rc) break;
            GS_CUDA(c, cudaEventSynchronize(e1));
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms *= 0.5f;
            if (tried < 32) {
                r.tried_tile_w[tried] = shapes[si][0];
                r.tried_tile_h[tried] = shapes[si][1];
                r.tried_depth[tried] = c->batch_depth;
                r.tried_ms[tried] = ms;
            }
            ++tried;
            if (ms < r.best_ms) {
                r.best_ms = ms;
                r.tile_w = shapes[si][0];
                r.tile_h = shapes[si][1];
                r.batch_depth = c->batch_depth;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        c->alpha_tile_w = keep_w;
        c->alpha_tile_h = keep_h;
        c->batch_depth = keep_d;
        return rc;
    }
    r.tried = (uint32_t)std::min(tried, 32);
    c->alpha_tile_w = r.tile_w;
    c->alpha_tile_h = r.tile_h;
    c->batch_depth = r.batch_depth;
    if (res) *res = r;
    return GS_OK;
}

int gs_render_anim_batch(gs_ctx* c, const gs_camera* cam, const int32_t* states_a, const int32_t* states_b,
                         const float* weights, uint32_t count, void* const* outs) {
    if (!c || !cam || (count && (!states_a || !outs))) return GS_ERR_BAD_ARG;
    if (!gl_clip_convention(cam)) return fail(c, GS_ERR_BAD_ARG, "only the GL clip convention is drawn");
    int rc = batch_checks(c, count);
    if (rc || !count) return rc;
    if (!c->anim_deltas) return fail(c, GS_ERR_BAD_ARG, "no gsanim appearance states uploaded");
    for (uint32_t k = 0; k < count; ++k) {
        const int a = states_a[k], b = states_b ? states_b[k] : 0;
        const float wgt = weights ? weights[k] : 0.0f;
        if (!outs[k] || a < 0 || a > (int)c->anim_states || b < 0 || b > (int)c->anim_states || !(wgt >= 0.0f) ||
            wgt > 1.0f)
            return fail(c, GS_ERR_BAD_ARG, "bad appearance state in the batch");
    }
    cudaSetDevice(c->device);
    if ((rc = ensure_batch(c, count))) return rc;
    const size_t need = (size_t)count * c->n;
    if (c->state_colours_cap < need) {
        dfree(c->state_colours);
        c->state_colours_cap = 0;
        GS_CUDA(c, dalloc(&c->state_colours, need * sizeof(float4)));
        c->state_colours_cap = need;
    }
    nvtxRangePushA("gs_render_anim_batch");
    c->frame_launches = 0;
    // the geometry, order and tiles of the frame, once (slot 0)
    std::vector<uint32_t> redo;
    for (int attempt = 0;; ++attempt) {
        if ((rc = stage_frame(c, 0, cam, outs[0]))) break;
        if ((rc = grow_overflowed(c, 1, redo))) break;
        if (redo.empty()) break;
        if (attempt >= 3) {
            rc = fail(c, GS_ERR_TOO_LARGE, "tile entries still overflowing");
            break;
        }
    }
    if (rc) {
        nvtxRangePop();
        return rc;
    }
    // per state: the colours of the frame's records, and the raster parameters
    FrameSlot& f0 = c->slots[0];
    swap_slot(c, f0);
    const int sa = c->anim_a, sb = c->anim_b;
    const float sw = c->anim_w;
    const gs::RasterParams base = c->h_batch_params[0];
    {
        StageScope sc(c, ST_CULL);
        for (uint32_t k = 0; k < count; ++k) {
            c->anim_a = states_a[k];
            c->anim_b = states_b ? states_b[k] : 0;
            c->anim_w = weights ? weights[k] : 0.0f;
            gs::CullParams p = cull_params(c);
            float4* colours = c->state_colours + (size_t)k * c->n;
            sc.add(gs::launch_recolour(p, c->records, colours, c->num_sms, c->stream));
            gs::RasterParams r = base;
            r.colours = colours;
            r.out_rgba16f = static_cast<uint16_t*>(outs[k]);
            c->h_batch_params[k] = r;
        }
    }
    c->anim_a = sa;
    c->anim_b = sb;
    c->anim_w = sw;
    swap_slot(c, f0);
    rc = raster_batch(c, count);
    cudaStreamWaitEvent(c->stream, c->fc_event, 0);   // after gs_render's copy of h_fc
    cudaMemcpyAsync(c->h_fc, c->slots[0].fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, c->stream);
    cudaEventRecord(c->fc_event, c->stream);
    c->fc_pending = false;
    c->last_launches = c->frame_launches;
    nvtxRangePop();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return rc;
}

int gs_read_stats(gs_ctx* c, gs_stats* s) {
    if (!c || !s) return GS_ERR_BAD_ARG;
    GS_CUDA(c, cudaStreamSynchronize(c->stream));
    GS_CUDA(c, cudaStreamSynchronize(c->fc_stream));   // gs_render's counters come on fc_stream
    c->fc_pending = false;
    std::memset(s, 0, sizeof(*s));
    const FrameCounters& f = *c->h_fc;
    s->gaussian_count = c->n;
    s->visible_count = f.visible_count;
    s->tile_entries = f.tile_entries;
    s->tile_overflow = f.tile_overflow;
    for (int k = 0; k < 8; ++k) s->diagnostics[k] = f.diag[k];
    s->gps_requested_work_items = f.gps_work[0];
    s->gps_budget_exhausted = f.gps_work[1];
    s->gps_max_work_items = c->gps_max_work_items;
    s->sample_count = c->sample_count;
    s->frame_seed = c->frame_seed;
    s->error_flags = f.error_flags;
    s->kernel_launches = c->last_launches;
    s->denoise_fallback_tiles = f.fallback_tiles;
    return (f.error_flags & ~(uint32_t)gs::kErrTileOverflow) ? GS_ERR_DEVICE_TIMEOUT : GS_OK;
}

int gs_debug_read(gs_ctx* c, int which, void* dst, uint64_t bytes) {
    if (!c || !dst) return GS_ERR_BAD_ARG;
    GS_CUDA(c, cudaStreamSynchronize(c->stream));
    GS_CUDA(c, cudaStreamSynchronize(c->fc_stream));   // h_fc of the last frame
    const uint64_t n = c->n;
    const uint32_t vis = c->h_fc->visible_count;
    const size_t npix = (size_t)c->width * c->height;
    switch (which) {
        case GS_DEBUG_IDS:
        case GS_DEBUG_KEYS: {
            // The reference keeps all-N arrays (culled = 0xFFFFFFFF); ours are
            // compacted in index order, so expand them here.
            if (bytes < n * 4) return GS_ERR_BAD_ARG;
            std::vector<uint32_t> k(vis), id(vis);
            GS_CUDA(c, cudaMemcpy(k.data(), c->keys[1], (size_t)vis * 4, cudaMemcpyDeviceToHost));
            GS_CUDA(c, cudaMemcpy(id.data(), c->ids[1], (size_t)vis * 4, cudaMemcpyDeviceToHost));
            uint32_t* o = static_cast<uint32_t*>(dst);
            std::fill(o, o + n, 0xFFFFFFFFu);
            for (uint32_t i = 0; i < vis; ++i) o[id[i]] = which == GS_DEBUG_IDS ? id[i] : k[i];
            return GS_OK;
        }
        case GS_DEBUG_PROJECTED:
            if (bytes < n * 64) return GS_ERR_BAD_ARG;
            GS_CUDA(c, cudaMemcpy(dst, c->projected, n * 64, cudaMemcpyDeviceToHost));
            return GS_OK;
        case GS_DEBUG_SORTED_IDS:
        case GS_DEBUG_SORTED_KEYS: {
            if (bytes < n * 4) return GS_ERR_BAD_ARG;
            SortPlan pl;
            GS_CUDA(c, cudaMemcpy(&pl, c->depth_plan, sizeof(pl), cudaMemcpyDeviceToHost));
            const uint32_t* src = which == GS_DEBUG_SORTED_IDS ? pl.vfinal : pl.kfinal;
            uint32_t* o = static_cast<uint32_t*>(dst);
            if (!src) return fail(c, GS_ERR_BAD_ARG, "no sort in the last frame");
            GS_CUDA(c, cudaMemcpy(o, src, (size_t)vis * 4, cudaMemcpyDeviceToHost));
            std::fill(o + vis, o + n, 0xFFFFFFFFu);
            return GS_OK;
        }
        case GS_DEBUG_ACCUM:
        case GS_DEBUG_SAMPLE: {
            if (bytes < npix * 16) return GS_ERR_BAD_ARG;
            const float4* src = which == GS_DEBUG_SAMPLE ? c->st.sample : c->st.display;
            if (!src) return fail(c, GS_ERR_BAD_ARG, "no stochastic/GPS frame rendered");
            GS_CUDA(c, cudaMemcpy(dst, src, npix * 16, cudaMemcpyDeviceToHost));
            return GS_OK;
        }
        case GS_DEBUG_DEPTH:
            if (bytes < npix * 4) return GS_ERR_BAD_ARG;
            if (!c->st.depth) return fail(c, GS_ERR_BAD_ARG, "no stochastic/GPS frame rendered");
            GS_CUDA(c, cudaMemcpy(dst, c->st.depth, npix * 4, cudaMemcpyDeviceToHost));
            return GS_OK;
        default:
            return GS_ERR_BAD_ARG;
    }
}

int gs_profile_enable(gs_ctx* c, int enable) {
    if (!c) return GS_ERR_BAD_ARG;
    c->profiling = enable != 0;
    return GS_OK;
}

int gs_stage_times(gs_ctx* c, float* ms, uint32_t* launches, int max_stages, int reset) {
    if (!c) return GS_ERR_BAD_ARG;
    GS_CUDA(c, cudaStreamSynchronize(c->stream));
    for (auto& p : c->pending) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, p.a, p.b);
        c->stage_ms[p.stage] += t;
        c->stage_launches[p.stage] += p.launches;
        c->event_pool.push_back(p.a);
        c->event_pool.push_back(p.b);
    }
    c->pending.clear();
    for (int k = 0; k < ST_COUNT && k < max_stages; ++k) {
        if (ms) ms[k] = (float)c->stage_ms[k];
        if (launches) launches[k] = c->stage_launches[k];
    }
    if (reset) {
        std::fill(c->stage_ms, c->stage_ms + ST_COUNT, 0.0);
        std::fill(c->stage_launches, c->stage_launches + ST_COUNT, 0u);
    }
    return ST_COUNT;
}

}  // extern "C"
