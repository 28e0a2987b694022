// Internal interfaces between the C++ host orchestration (gs_host.cpp) and the
// CUDA kernels.  Not part of the public C ABI (include/gs_api.h).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gs_api.h"

namespace gs {

// Device error flags (gs_stats.error_flags).
enum : uint32_t {
    kErrCullLookback = 1u << 0,
    kErrSortLookback = 1u << 1,
    kErrBinLookback = 1u << 2,
    kErrRasterWait = 1u << 3,
    kErrTileOverflow = 1u << 4,
    kErrGpsWait = 1u << 5,
    kErrCullStage = 1u << 6,
};

// Small per-frame device control block.  Zeroed at the start of each frame
// (one memset), except where noted.
struct FrameCounters {
    uint32_t visible_count;      // cull output (shaders/cull.glsl:230)
    uint32_t diag[8];            // SplatDiagnostics (shaders/cull.glsl:296-318)
    uint32_t error_flags;        // gs::kErr* bits
    uint32_t cull_ticket;        // tile tickets for persistent kernels
    uint32_t bin_ticket;
    uint32_t tile_entries;       // (tile, splat) pairs produced by binning
    uint32_t tile_overflow;      // entries that did not fit
    uint32_t gps_work[2];        // [0] requested work items, [1] overflow (gps.glsl work_count)
    uint32_t raster_ticket;
    uint32_t fallback_tiles;     // denoised mode: tiles over the error budget
    uint32_t pad[1];
};

// Device-resident plan of one radix sort, written by its plan kernel from the
// digit histograms: which passes do work (a pass whose digit is the same for
// every key is the identity permutation of a stable sort and is skipped),
// and the ping-pong buffers of each active pass.  Zeroed before each sort.
struct SortPlan {
    const uint32_t* kin[4];
    const uint32_t* vin[4];
    uint32_t* kout[4];
    uint32_t* vout[4];
    uint32_t active[4];
    uint32_t ticket[4];
    const uint32_t* kfinal;      // where the sorted keys are
    const uint32_t* vfinal;      // where the sorted values are
    uint32_t copy_needed;        // land_in_buf0 with no active pass
    uint32_t count;
    uint32_t pad[2];
};

// Onesweep radix sort configuration.
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per CTA tile
constexpr int kSortLookback = 8;                       // look-back words read per step
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

// Cull configuration.  Visibility pass: 256-thread CTAs, 8 rows per thread;
// its 2048-row CTA tiles are the units of the look-back.  Projection pass:
// 128-thread CTAs, each warp stages and projects 32 visible rows at a time.
constexpr int kCullVisThreads = 256;
constexpr int kCullVisItems = 8;
constexpr int kCullVisTile = kCullVisThreads * kCullVisItems;
constexpr int kCullThreads = 128;
constexpr int kHalfRowChunks = 9;   // 144-byte FP16-SH row: position/opacity, scale, rotation, 48 half SH

// Binning configuration: 8 sorted splats per thread, 1024 per CTA tile; the
// expansion takes the global entry range in chunks of 1024 entries.
constexpr int kBinThreads = 128;
constexpr int kBinItems = 8;
constexpr int kBinTile = kBinThreads * kBinItems;
constexpr int kBinChunk = 8 * kBinThreads;     // entries expanded per round
constexpr int kTileW = 16;
constexpr int kTileH = 16;

// Raster record: one per visible splat in depth-sorted order, 64 bytes,
// staged into shared memory by TMA bulk copies.
//
// The rasterizer tests the splat's quadratic form s = conic(d) (the power is
// -0.5 s) instead of the power: "power <= 0 && !(power < cutoff)" holds
// exactly when -kSMin <= s <= s_max, with s_max = -2 cutoff, or the smallest
// subnormal when cutoff == 0 (multiplying by -0.5 is exact except for
// subnormal s, and those cases are what the two bounds absorb).
//
// Stochastic envelope records (BinParams::envelope) reuse three slots:
// log2_opacity holds radius_x, rect_x holds the bits of ndc_z and rect_y the
// bits of radius_y; cx, cy are un-jittered and hash_z is unused.
struct __align__(16) RasterRecord {
    float cx, cy, conic_x, conic_2y;     // centre (+jitter), conic.x, 2*conic.y
    float conic_z, log2_opacity, s_max, r;
    float g, b;
    uint32_t rect_x;                     // i0 | i1 << 16  (candidate pixel columns: quad coverage
    uint32_t rect_y;                     // j0 | j1 << 16   intersected with the alpha >= 1/255 box, GL rows)
    uint32_t depth24;                    // window depth as D24 (stochastic depth test)
    uint32_t splat_id;                   // original Gaussian index
    float hash_z;                        // float(splat_id) + frame_seed
    float opacity;
};
static_assert(sizeof(RasterRecord) == 64, "RasterRecord must be 64 bytes");

struct CullParams {
    const float4* rows;          // N x 16 float4 (GpuGaussian)
    const float4* heads;         // N float4: the first 16 bytes of every row (position, opacity), kept beside the rows
    uint32_t n;
    gs_camera cam;               // the frame's CameraUniforms, by value (constant-bank operands)
    int sh_degree;
    float sh_lod_distance;
    int collect_stats;
    int write_invisible;         // also write the reference's invisible record
    float4* projected;           // N x 4 float4 (CullProjectedSplatData)
    uint32_t* keys_out;          // compacted visible keys, index order
    uint32_t* ids_out;           // compacted visible ids
    unsigned long long* status;  // per-tile look-back words (epoch-tagged)
    uint32_t epoch;
    uint32_t* key_hist;          // 4 x 256 digit histograms of the emitted keys (zeroed per frame)
    // gsanim int8 appearance deltas (shaders/cull.glsl:125-164); null = none
    const int8_t* anim_deltas;   // [(state-1) * n + row] * 48 + j
    const float* anim_scales;    // 48 (device)
    int anim_state_a, anim_state_b;
    float anim_weight;
    // gsanim 0.3 appearance layers (shaders/cull.glsl:141-148, 354-416); layer_count 0 = none
    const uint16_t* layer_halves;   // [(l * n + row) * 48 + j] IEEE half bits
    const float* layer_weights;     // [l * 3 + c] (device)
    int layer_count;
    int half_rows;               // rows are 144-byte FP16-SH rows (kHalfRowChunks float4 each)
    FrameCounters* fc;
};

struct SortParams {
    const uint32_t* keys_in;     // input pairs (never written)
    const uint32_t* vals_in;
    uint32_t* keys_buf[2];       // writable ping-pong buffers (keys_buf[1] may alias keys_in
    uint32_t* vals_buf[2];       //  when land_in_buf0 == 0)
    int land_in_buf0;            // 1: the result must end in keys_buf[0]/vals_buf[0]
    const uint32_t* count_ptr;   // device-side element count
    uint32_t count_cap;          // capacity (grid sizing)
    int begin_bit, end_bit;
    uint32_t* hist;              // 4 x 256 digit histograms (zeroed before the sort)
    int hist_ready;              // 1: the producer of the keys already filled `hist`
    SortPlan* plan;              // zeroed before the sort
    unsigned long long* status;  // per pass: tiles x 256 look-back words (epoch-tagged)
    size_t status_stride;        // words per pass
    uint32_t epoch;
    uint32_t* error_flags;
    int first_pdl = 0;           // 1: the first pass too is a programmatic dependent launch
};

struct BinParams {
    const SortPlan* depth_plan;      // sorted ids at depth_plan->vfinal
    const float4* projected;
    float vp_w, vp_h, clip_y_sign;   // CameraUniforms viewport and clip_y_sign of the frame
    float jitter_x, jitter_y;
    float frame_seed;
    int width, height, tiles_x, tiles_y;
    int tile_shift_x, tile_shift_y;  // log2 of the tile width and height
    RasterRecord* records;           // N_vis records (sorted order)
    uint32_t* entry_keys;            // tile id per entry
    uint32_t* entry_vals;            // sorted position per entry
    uint32_t entry_cap;
    uint4* item_info;                // per binned item: first entry, tx0 | ty0 << 16, width in tiles (0: none)
    uint32_t* chunk_first;           // per expansion chunk: the item owning its first entry
    uint32_t chunk_cap;              // chunk_first capacity (entry_cap / kBinChunk + 2)
    uint32_t* tile_hist;             // 3 x 256 digit histograms of the tile ids (zeroed per pass)
    unsigned long long* status;      // per-CTA-tile look-back words (epoch-tagged)
    uint32_t epoch;
    FrameCounters* fc;
    // 1: stochastic envelope mode.  Tiles are chosen for every sub-pixel
    // jitter in [-0.5, 0.5]^2 at once and the records keep the un-jittered
    // quad (centre, radii, ndc_z), so one binning serves all samples of a
    // frame; the rasterizer derives each sample's coverage.
    int envelope;
};

struct RasterParams {
    const RasterRecord* records;
    uint32_t record_cap;             // records allocated (bounds every record index)
    const SortPlan* tile_plan;       // tile-sorted entry values at tile_plan->vfinal
    const uint2* tile_ranges;        // [start, end) per tile
    const uint32_t* tile_order;      // tiles by descending work (CTA b rasterizes tile_order[b])
    const uint32_t* tile_count;      // optional: CTAs b >= *tile_count do nothing (a tile list of the frame)
    const float4* colours;           // optional: r, g, b per record, replacing the records' colour
    int width, height, tiles_x, tiles_y;
    int tile_w, tile_h;              // tile shape: 16x16, or 32x8 / 8x32 (alpha mode)
    float bg;
    // stochastic mode (envelope records): the sample's jitter and seed, and
    // the viewport of the quad computation
    float jitter_x, jitter_y, frame_seed;
    float frame_seed2;               // two-sample mode: the second sample's seed (frame_seed is the first's)
    float vp_w, vp_h, clip_y_sign;
    uint16_t* out_rgba16f;           // width*height*4 halves, top row first
    float4* out_rgba32f;             // optional float copy (stochastic sample), top row first
    float* out_depth;                // optional window depth (stochastic), top row first
    // optional running mean of the samples (stochastic): accum_out = h + (sample - h) / max(accum_n, 1)
    // with h = accum_in, or the sample itself when accum_in is null (accum_kernel's arithmetic)
    const float4* accum_in;
    float4* accum_out;
    float accum_n;
    int rgba8;                       // quantise stochastic sample like RGBA8 UNORM
    FrameCounters* fc;
};

// Launch with programmatic stream serialization: the kernel may be scheduled
// while its predecessor in the stream finishes, and calls pdl_wait() before
// it reads or writes anything the predecessor touches.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Every device allocation of the library goes through here: cudaMalloc, with
// a failed call's error cleared (it is reported through the return value),
// and the allocation-failure injection of gs_debug_fail_alloc.
cudaError_t device_malloc(void** p, size_t bytes);

// Launchers (each returns the number of kernels it launched).
int launch_cull(const CullParams& p, uint32_t num_sms, cudaStream_t s);
int launch_gather_heads(const float4* rows, float4* heads, uint32_t n, uint32_t num_sms, cudaStream_t s,
                        uint32_t row_chunks = 16);
int launch_pack_half_rows(const float4* rows, float4* half_rows, uint32_t n, uint32_t num_sms, cudaStream_t s);
int launch_recolour(const CullParams& p, const RasterRecord* records, float4* colours, uint32_t num_sms,
                    cudaStream_t s);
int launch_sort(const SortParams& p, uint32_t num_sms, cudaStream_t s);
int launch_bin(const BinParams& p, uint32_t n_cap, uint32_t num_sms, cudaStream_t s);
int launch_tile_ranges(const SortPlan* tile_plan, const FrameCounters* fc, uint32_t entry_cap, uint2* ranges,
                       uint32_t num_tiles, uint32_t num_sms, cudaStream_t s);
int launch_tile_order(const uint2* ranges, uint32_t num_tiles, uint32_t* order, cudaStream_t s);
int launch_raster_alpha(const RasterParams& p, cudaStream_t s);
int launch_raster_stochastic(const RasterParams& p, cudaStream_t s);
int launch_raster_stochastic2(const RasterParams& p, cudaStream_t s);
// alpha frames[f] for f < nframes in one persistent launch (first: nframes + 1
// prefix sums of the frames' tile counts, device; ticket: a zeroed device word)
int launch_raster_batch_alpha(const RasterParams* frames, const uint32_t* first, uint32_t nframes, uint32_t* ticket,
                              uint32_t grid, int tile_w, cudaStream_t s);
void raster_batch_occupancy(int* blocks_per_sm);

int launch_wait_probe(const unsigned long long* status, FrameCounters* fc, uint32_t epoch, int which, uint32_t limit,
                      cudaStream_t s);

size_t sort_status_words(uint32_t count_cap);   // look-back words per pass
int sort_passes(int begin_bit, int end_bit);
}  // namespace gs
