/* gs_api.h - C ABI of libgs_cuda.so, the B200 (sm_100a) splatting path of
 * gamesplat.
 *
 * The entry points replace the renderer interface of the reference
 * (src/renderer.h:249-266) for the per-frame splatting path: cull/SH/project
 * (shaders/cull.glsl), radix depth sort (shaders/sort.glsl), sorted alpha
 * compositing (shaders/splat.glsl + GL blend), stochastic splatting and the
 * Gaussian Point Splatting passes (shaders/gps.glsl, shaders/accum.glsl).
 *
 * Conventions
 *  - Plain C types only; no CUDA or C++ types cross the boundary.  A CUDA
 *    stream is passed as an opaque pointer (cudaStream_t value, NULL = legacy
 *    default stream).
 *  - Every function returns a gs_status (0 = GS_OK, < 0 = error) and never
 *    aborts or traps; the reference reports failures as bool + log line
 *    (src/renderer.cpp:860-1073).
 *  - All calls on one gs_ctx must be serialised by the caller, as the
 *    reference renderer is used from one thread (src/main.cpp:1963).
 *  - Work is stream-ordered; only gs_render_host, gs_render_host_wait (and a
 *    gs_render_host_submit that retires an older frame), gs_read_stats and
 *    gs_debug_read synchronise, and gs_render waits for its frame's tile
 *    entry count (see there) while the rest of the frame stays queued.
 *  - Images are RGBA16F (IEEE half, 4 channels), row-major, top row first
 *    (the orientation of the reference harness's linear_capture,
 *    tests/gsanim_render.cpp:161-163).
 */
#ifndef GS_API_H
#define GS_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_API_VERSION 1

typedef enum gs_status {
    GS_OK = 0,
    GS_ERR_BAD_ARG = -1,          /* invalid argument or state */
    GS_ERR_OOM = -2,              /* device or pinned-host allocation failed */
    GS_ERR_CUDA = -3,             /* a CUDA runtime call failed */
    GS_ERR_DEVICE_TIMEOUT = -4,   /* a bounded device-side wait ran out (gs_stats.error_flags) */
    GS_ERR_NO_SCENE = -5,         /* render before upload */
    GS_ERR_BUDGET_REFUSED = -6,   /* GPS budget resize refused; the old budget is kept */
    GS_ERR_NO_DEVICE = -7,        /* no usable CUDA device */
    GS_ERR_TOO_LARGE = -8,        /* size beyond a documented limit */
    GS_ERR_FORMAT = -9            /* file missing, unreadable or not a valid asset */
} gs_status;

/* src/renderer.h:58-64 SplatRenderMode */
typedef enum gs_render_mode {
    GS_MODE_ALPHA = 0,            /* AlphaBlendSorted */
    GS_MODE_STOCHASTIC = 1,       /* StochasticSplats */
    GS_MODE_GPS = 2,              /* GaussianPointSplatting */
    GS_MODE_DENOISED = 3          /* two-sample stochastic frame + denoiser (gs_set_denoiser), tiles over
                                     the error budget rendered sorted-alpha; no counterpart in the reference */
} gs_render_mode;

/* CameraUniforms, byte for byte (src/camera.h:23-38): 40 floats, 160 bytes. */
typedef struct gs_camera {
    float view[16];
    float proj[16];
    float viewport[2];
    float orthographic;
    float persp_focal;
    float ortho_focal;
    float clip_y_sign;
    float clip_z_01;
    float pad[1];
} gs_camera;

/* Renderer knobs of the splatting path: the Renderer fields of
 * src/renderer.h:121-247 that the path reads, with the defaults of
 * renderer_init (src/renderer.cpp:588-599). */
typedef struct gs_knobs {
    int32_t render_mode;                      /* gs_render_mode; default GS_MODE_GPS */
    int32_t sh_degree;                        /* 0..3; default 3 */
    float sh_lod_distance;                    /* <= 0 disables; default 0 */
    uint32_t gps_supersample_factor;          /* 1..4; default 2 */
    uint32_t stochastic_samples_per_frame;    /* 1..16; default 1 */
    uint32_t stochastic_taa_current_samples;  /* 1..16; default 4 */
    int32_t stochastic_accumulation_enabled;  /* default 1 */
    int32_t stochastic_taa_enabled;           /* default 1 */
    int32_t black_background;                 /* default 0 (background 0.1) */
    int32_t splat_diagnostics_enabled;        /* default 0 */
    int32_t linear_color;                     /* 1: float sample target and linear GPS colour
                                                 (gsanim 0.3 path); 0: RGBA8 sample target */
    int32_t write_invisible_records;          /* 1: also write the reference's record for culled
                                                 Gaussians (debug/parity); default 0 */
    uint32_t gpu_budget_mb;                   /* cap on the scene's device memory in MiB (Renderer
                                                 gpu_budget_bytes = MiB << 20, src/renderer.h:175,
                                                 src/main.cpp:352-359); 0: none beyond 4/5 of the
                                                 free device memory; default 0 */
    int32_t reserved[3];
} gs_knobs;

/* Per-frame statistics (the reference's SplatDiagnostics, src/renderer.h:28-38,
 * and GPS work statistics, src/renderer.cpp:2038-2055). */
typedef struct gs_stats {
    uint32_t gaussian_count;
    uint32_t visible_count;
    uint32_t tile_entries;               /* (16x16 tile, splat) pairs of the last frame */
    uint32_t tile_overflow;              /* entries that did not fit in the frame's last pass (gs_render grows
                                            the buffers and re-renders, so 0 after a GS_OK frame) */
    uint32_t diagnostics[8];             /* shaders/cull.glsl:296-318 counters, if enabled */
    uint32_t gps_requested_work_items;
    uint32_t gps_budget_exhausted;
    uint32_t gps_max_work_items;
    uint32_t sample_count;               /* accumulated samples (stochastic / GPS) */
    uint32_t frame_seed;
    uint32_t error_flags;                /* device error bits (bounded waits that ran out) */
    uint32_t kernel_launches;            /* kernels launched by the last gs_render */
    uint32_t denoise_fallback_tiles;     /* denoised mode: 16x16 tiles rendered again sorted-alpha */
    uint32_t reserved[4];
} gs_stats;

/* gs_debug_read selectors (reference buffers, src/renderer.cpp:922-1058). */
typedef enum gs_debug_buffer {
    GS_DEBUG_IDS = 0,        /* uint32[N] unsorted ids (idx or 0xFFFFFFFF), after cull */
    GS_DEBUG_KEYS = 1,       /* uint32[N] depth keys (0xFFFFFFFF for culled), after cull */
    GS_DEBUG_PROJECTED = 2,  /* float[N*16] CullProjectedSplatData */
    GS_DEBUG_SORTED_IDS = 3, /* uint32[N] ids after the depth sort (culled tail = 0xFFFFFFFF) */
    GS_DEBUG_SORTED_KEYS = 4,/* uint32[N] keys after the depth sort */
    GS_DEBUG_ACCUM = 5,      /* float[W*H*4] accumulation image (stochastic / GPS), top row first */
    GS_DEBUG_SAMPLE = 6,     /* float[W*H*4] last stochastic/GPS sample, top row first */
    GS_DEBUG_DEPTH = 7       /* float[W*H] last sample's window depth, top row first */
} gs_debug_buffer;

typedef struct gs_ctx gs_ctx;
typedef struct gs_denoiser gs_denoiser;   /* the stochastic-splat denoiser, see gs_denoiser_create */

/* renderer_init (src/renderer.h:249): create a context on `device`, issuing
 * work on `stream` (cudaStream_t, may be NULL).  Knobs get the reference
 * defaults. */
int gs_create(gs_ctx** out, int device, void* stream);

/* renderer_destroy (src/renderer.h:266). Accepts NULL. */
void gs_destroy(gs_ctx* ctx);

/* Renderer fields set by the caller (src/main.cpp:341-387). */
int gs_get_knobs(const gs_ctx* ctx, gs_knobs* out);
int gs_set_knobs(gs_ctx* ctx, const gs_knobs* knobs);
int gs_set_mode(gs_ctx* ctx, int render_mode);

/* renderer_upload_gaussians (src/renderer.h:250): copy `count` GpuGaussian
 * rows (64 floats = 256 bytes each, src/gaussian.h:63-73) from host memory.
 * The caller keeps ownership of `rows`.  Replaces any previous scene. */
int gs_upload_rows(gs_ctx* ctx, const float* rows, uint64_t count);

/* Row format of the next upload (no counterpart in the reference, whose rows
 * are always the FP32 GpuGaussian): 0 = GpuGaussian rows kept as uploaded
 * (256 bytes, the default); 1 = 144-byte rows with the SH coefficients in
 * IEEE half (position, opacity, scale and rotation stay FP32, as do the
 * projected records and all arithmetic after the cull): the upload converts
 * the GpuGaussian rows on the device, and the cull evaluates SH3 on the tensor
 * cores (FP16 operands, FP32 accumulation).  Scenes in format 1 take no
 * gsanim deltas or layers (GS_ERR_BAD_ARG). */
int gs_set_row_format(gs_ctx* ctx, int format);

/* As gs_upload_rows, from device memory (stream-ordered copy). */
int gs_upload_rows_device(gs_ctx* ctx, const float* rows_dev, uint64_t count);

/* Replace rows [first, first + count) of the resident scene with `count`
 * GpuGaussian rows from host memory (the per-chunk copy of
 * renderer_upload_gaussians, src/renderer.cpp:896-919, applied to a range of
 * a scene already uploaded): for hosts that edit or stream part of a scene
 * without re-uploading all of it.  Queued after the frames already issued,
 * returns once the copy is done, and resets accumulation.  GS_ERR_NO_SCENE
 * without a scene, GS_ERR_BAD_ARG for a range beyond it. */
int gs_upload_rows_range(gs_ctx* ctx, const float* rows, uint64_t first, uint64_t count);

/* gsanim appearance states (the renderer's animation buffer,
 * src/renderer.cpp:824-841, decoded by shaders/cull.glsl:125-164):
 * `deltas` holds num_states x N x 48 int8 values (state-major, row, then
 * coefficient j: 0..2 = DC, 3 + 15c + k = SH coefficient k of channel c);
 * state s >= 1 adds deltas[s-1][row][j] * scales[j] to the uploaded row's
 * coefficient, state 0 is the row itself.  Upload after gs_upload_rows;
 * num_states = 0 removes the animation.  Copies; the caller keeps ownership. */
int gs_upload_anim(gs_ctx* ctx, const int8_t* deltas, uint32_t num_states, const float* scales);

/* The renderer's animation_state_a / animation_state_b / animation_weight
 * (src/renderer.cpp:2148-2161, from gsanim_sample): the coefficients are
 * (1 - weight) * state_a + weight * state_b.  A change resets accumulation. */
int gs_set_anim_state(gs_ctx* ctx, int state_a, int state_b, float weight);

/* gsanim 0.3 appearance layers: the renderer's animation buffer for version 3
 * assets (src/renderer.cpp:840-864, GSAnim::layer_data), layer_count x N x 48
 * IEEE half bits, [(layer * N + row) * 48 + j] with j = DC 0..2, then
 * 3 + channel * 15 + k.  Upload after gs_upload_rows (at most 256 layers);
 * layer_count = 0 removes them.  Copies; the caller keeps ownership. */
int gs_upload_layers(gs_ctx* ctx, const uint16_t* halves, uint32_t layer_count);

/* The layer weights of the next frames: gsanim_layer_weights at the playback
 * time (src/renderer.cpp:1829-1835), weights[count * 3] RGB per layer, count
 * at most the uploaded layers (1 for the renderer's first_layer_only).  With
 * count > 0 the cull colours each splat as the sum over the layers of
 * max(SH colour of the layer's coefficients, 0) * weight, without the +0.5
 * bias (shaders/cull.glsl:141-148, 354-416); count = 0 turns the layer path
 * off.  Changed weights reset accumulation. */
int gs_set_layer_weights(gs_ctx* ctx, const float* weights, uint32_t count);

/* renderer_set_gps_work_budget (src/renderer.h:252): replace only the GPS work
 * buffer; on failure the old budget and buffer are kept
 * (src/renderer.cpp:1076-1123). */
int gs_set_gps_budget(gs_ctx* ctx, uint32_t max_work_items);

/* Denoised mode (GS_MODE_DENOISED; no counterpart in the reference): the
 * denoiser the context uses (not owned; NULL detaches), and the error
 * budget: a 16x16 tile whose estimated mean squared error (over RGBA)
 * reaches tile_mse (>= 0; default 1e-4, i.e. 40 dB PSNR) is rendered again by
 * the sorted-alpha rasterizer when fallback != 0 (default); tile_mse 0 sends
 * every tile to the sorted-alpha rasterizer. */
int gs_set_denoiser(gs_ctx* ctx, gs_denoiser* denoiser);
int gs_set_denoise_budget(gs_ctx* ctx, float tile_mse, int fallback);

/* The denoiser's input of the next frame, without the denoiser: two
 * un-jittered stochastic samples per pixel (seeds frame_seed + 1 and + 2,
 * the kept-fragment rule of shaders/splat.glsl:127-145 on the sorted tile
 * lists), their TAA history (shaders/accum.glsl:148-178, advanced as a
 * denoised frame advances it) and the features, written to features_out
 * (device, height x width x 16 bf16, top row first; even viewport).  For
 * generating training pairs. */
int gs_render_features(gs_ctx* ctx, const gs_camera* cam, void* features_out);

/* renderer_reset_stochastic_accumulation (src/renderer.h:261). */
int gs_reset_accumulation(gs_ctx* ctx);

/* Device bytes of a scene of `count` Gaussians with a GPS budget of
 * `gps_work_items` (renderer_scene_buffer_bytes, src/renderer.cpp:705-709, for
 * this library's layout): what gs_upload_rows allocates plus the GPS
 * prepared records and work items; frame targets not included.  0 for a count
 * outside 1..2^30-1.  Host only.  gs_upload_rows refuses a scene with
 * GS_ERR_TOO_LARGE, before it touches the resident one, when this exceeds
 * gpu_budget_mb or 4/5 of the device's free memory (src/renderer.cpp:739-763);
 * gs_upload_anim and gs_upload_layers check their own bytes the same way, and
 * gs_set_gps_budget its new work buffer (GS_ERR_BUDGET_REFUSED). */
uint64_t gs_scene_device_bytes(uint64_t count, uint32_t gps_work_items);

/* renderer_draw_frame (src/renderer.h:265), splatting path only: cull,
 * (alpha) sort, then composite / stochastic / GPS according to the mode, into
 * caller-owned device memory `rgba16f_out` (width*height*4 halves, top row
 * first; width/height = round(cam->viewport)).  `cam` is host memory.
 * Only the GL clip convention (clip_y_sign 1, clip_z_01 0; the non-WGPU
 * branch of src/main.cpp:1275-1281) is drawn: other cameras return
 * GS_ERR_BAD_ARG, since the WGPU backend's top-left fragment origin is not
 * what the kernels rasterise.
 * Alpha and stochastic frames count their (tile, splat) entries on the
 * device; the call waits for that count (read back once the binning and the
 * tile sort have run, on a stream of the context's own, with the rest of the
 * frame still queued, as the reference's draw_frame reads back inside the
 * frame) and, when the entries did not fit, grows the
 * buffers and renders the frame again before returning.  A GS_OK frame is
 * therefore complete; GS_ERR_TOO_LARGE if the entries exceed the largest
 * buffer (2^30 - 1 entries), GS_ERR_OOM if growing fails. */
int gs_render(gs_ctx* ctx, const gs_camera* cam, void* rgba16f_out);

/* Batches (no counterpart in the reference, which draws one frame per call):
 * `count` alpha-mode frames (at most 256) rendered as gs_render would render
 * them one after another, each into its own device image outs[k]; cameras may
 * differ in position and viewport size.  Every frame's cull, depth sort and
 * binning run in turn into buffers the context keeps per frame slot, then one
 * persistent rasterizer launch composites all frames' tiles, taking
 * (frame, tile) work items by ticket.  Each image is identical to the
 * frame's gs_render image.  Waits once for the frames' tile-entry counts
 * (growing and re-binning overflowed frames, as gs_render does).  The slots
 * hold each frame's raster records and tile entries (about 0.2 KB per
 * Gaussian per frame), kept until the scene changes. */
int gs_render_batch(gs_ctx* ctx, const gs_camera* cams, uint32_t count, void* const* outs);

/* Tile shape of alpha frames (the other modes use 16 x 16): 16 x 16 (default),
 * 32 x 8 or 8 x 32 pixels; images are the same for every shape. */
int gs_set_tile_shape(gs_ctx* ctx, int tile_w, int tile_h);

/* Frames per persistent raster launch in gs_render_batch (0: the whole
 * batch, the default); each launch's frames are staged, checked for
 * tile-entry overflow and rasterized before the next ones. */
int gs_set_batch_depth(gs_ctx* ctx, uint32_t depth);

typedef struct gs_tune_result {
    int32_t tile_w, tile_h;          /* the fastest configuration, now set on the context */
    uint32_t batch_depth;
    float best_ms;                   /* its time for the whole batch */
    uint32_t tried;                  /* configurations measured (at most 32 listed) */
    int32_t tried_tile_w[32], tried_tile_h[32];
    uint32_t tried_depth[32];
    float tried_ms[32];
} gs_tune_result;

/* Autotuner of the batched path (no counterpart in the reference): renders
 * the batch (gs_render_batch, images into outs) with every tile shape
 * (16x16, 32x8, 8x32) and batch depth (4, 8, ..., 128, up to the batch),
 * times each on the device (CUDA events, two runs after a warm-up), and sets
 * the fastest on the context; res (may be NULL) receives every timing. */
int gs_autotune_batch(gs_ctx* ctx, const gs_camera* cams, uint32_t count, void* const* outs, gs_tune_result* res);

/* A batch of `count` gsanim appearance states of one camera (at most 256):
 * frame k is what gs_render draws after gs_set_anim_state(states_a[k],
 * states_b[k], weights[k]) (states_b / weights may be NULL for 0), into
 * outs[k].  The states share the frame's geometry, depth order and tiles,
 * computed once; per state only the colours of the visible splats are
 * evaluated again (the SH of shaders/cull.glsl:125-164, 323-417 with that
 * state's deltas), and one persistent rasterizer launch composites all
 * states.  Needs gs_upload_anim; alpha mode. */
int gs_render_anim_batch(gs_ctx* ctx, const gs_camera* cam, const int32_t* states_a, const int32_t* states_b,
                         const float* weights, uint32_t count, void* const* outs);

/* gs_render into host memory: includes the host->device camera copy and the
 * device->host image copy, and waits for them. */
int gs_render_host(gs_ctx* ctx, const gs_camera* cam, uint16_t* rgba16f_out_host);

/* Streamed readback, for a frame loop that displays or stores every frame on
 * the host (the reference's renderer_draw_frame + present, src/main.cpp's
 * frame loop): gs_render_host_submit queues the frame of `cam` (gs_render
 * into one of two device images of the context), then the copy of its image
 * into rgba16f_out_host on a copy stream of the context, and returns once
 * both are queued; the copy of frame i overlaps the kernels of frame i + 1.
 * rgba16f_out_host must be page-locked (cudaMallocHost / cudaHostRegister),
 * else GS_ERR_BAD_ARG.  Two frames are in flight at most: a submit first
 * waits for the copy of the older one, and for an earlier frame to the same
 * buffer.  The image is in the buffer once gs_render_host_wait(ctx, buffer)
 * returns (NULL: every frame in flight); a device-side wait that ran out in a
 * frame is reported (GS_ERR_DEVICE_TIMEOUT) by the call that retires it.
 * Same image as gs_render_host. */
int gs_render_host_submit(gs_ctx* ctx, const gs_camera* cam, uint16_t* rgba16f_out_host);
int gs_render_host_wait(gs_ctx* ctx, const uint16_t* rgba16f_out_host);

/* gsanim 0.3 display LUT: the scene's display_lut, lut_size, log2_min and
 * log2_max (src/gsanim.h:33-35), uploaded by the renderer at
 * src/renderer.cpp:870-881.  `lut` holds lut_size^3 x RGB uint16 values (x
 * fastest, then y, then z), lut_size 2..256, log2_min < log2_max
 * (src/gaussian_loader_gsanim.cpp:237,244).  Copies; waits for queued work on
 * the context's stream.  lut = NULL removes it. */
int gs_set_display_lut(gs_ctx* ctx, const uint16_t* lut, uint32_t lut_size, float log2_min, float log2_max);

/* renderer_display_appearance (src/renderer.cpp:2120-2137): the display pass
 * of a linear frame, shaders/accum.glsl:201-240 with the LUT, else the blit
 * (:181-192).  rgba16f_in: a gs_render frame in device memory (width*height*4
 * halves, 8-byte aligned); rgba32f_out: device memory for width*height*4
 * floats (16-byte aligned); both top row first.  exposure_ev is the
 * renderer's exposure_ev (src/renderer.h:168).  Stream-ordered. */
int gs_display(gs_ctx* ctx, const uint16_t* rgba16f_in, float* rgba32f_out, int width, int height,
               float exposure_ev);

/* Diagnostics, no counterpart in the reference (its GL path has no device
 * waits): runs one of the library's bounded device waits against a word that
 * nothing publishes (which = 0: decoupled look-back; 1: mbarrier / TMA
 * completion) with at most spin_limit polls, on private memory, and returns
 * what a frame would: GS_ERR_DEVICE_TIMEOUT once the wait runs out.  The
 * context stays usable.  Synchronises; allocates a few hundred bytes. */
int gs_debug_wait_probe(gs_ctx* ctx, int which, uint32_t spin_limit);

/* Statistics of the last frame (synchronises). */
int gs_read_stats(gs_ctx* ctx, gs_stats* out);

/* Copy a reference-layout buffer of the last frame to host memory (synchronises). */
int gs_debug_read(gs_ctx* ctx, int which, void* host_dst, uint64_t bytes);

/* Per-stage device timing.  enable != 0 records CUDA events around each stage
 * of every following frame on the context's stream and accumulates them;
 * gs_stage_times reads (and with reset != 0 clears) the totals in ms, one per
 * stage in the order of gs_stage_names().  Returns the number of stages. */
int gs_profile_enable(gs_ctx* ctx, int enable);
int gs_stage_times(gs_ctx* ctx, float* ms_out, uint32_t* launches_out, int max_stages, int reset);
const char* gs_stage_names(void);   /* comma-separated */

const char* gs_status_str(int status);
const char* gs_last_error(const gs_ctx* ctx);

/* ---- host helpers (no GPU) ---------------------------------------------- */

/* CameraUniforms of the reference fly camera: camera_get_view_matrix /
 * camera_get_proj_matrix (src/camera.cpp:137-245) and the uniform setup of
 * src/main.cpp:1264-1281 (persp_focal = H/2/tan(fov/2), ortho_focal =
 * H/(2 ortho_size), GL clip conventions unless webgpu != 0; gs_render
 * draws the GL ones only). */
int gs_camera_uniforms(const float position[3], float yaw, float pitch, float fov_y, float near_plane,
                       float far_plane, int z_up, float ortho_size, float ortho_blend, int width,
                       int height, int webgpu, gs_camera* out);

/* Load a binary little-endian 3DGS PLY into GpuGaussian rows with the
 * reference loader's header rules and transforms
 * (src/gaussian_loader_ply.cpp:14-228 and pack_gpu_gaussians,
 * src/gaussian.cpp:53-73).  With rows == NULL returns the vertex count (the
 * body must hold that many vertices); otherwise fills min(count, capacity)
 * rows.  < 0 on error.  A file naming scale_0, rot_0 or f_dc_0 without the
 * rest of its group is rejected: the reference reads outside the row for the
 * missing members, so it has no defined result to match. */
int64_t gs_load_ply(const char* path, float* rows, uint64_t capacity);

/* The same transforms on raw PLY-layout attributes already in memory:
 * raw is count x 59 floats in the order x y z, f_dc_0..2, f_rest_0..44,
 * opacity, scale_0..2, rot_0..3 (the 3DGS property order). */
int gs_pack_raw(const float* raw, uint64_t count, float* rows);

/* gs_pack_raw on the device (the loader transforms of
 * src/gaussian_loader_ply.cpp:148-203 and pack_gpu_gaussians,
 * src/gaussian.cpp:53-73): raw_dev and rows_dev are device memory (rows
 * 16-byte aligned), stream-ordered on `stream` (a cudaStream_t, NULL = the
 * default stream).  exp is correctly rounded here, while the reference's
 * loader calls expf: where expf is not correctly rounded (about 0.008 % of
 * float arguments) a scale can differ by one ulp and an opacity by up to two
 * (through 1 / (1 + exp(-x))); every other field is identical.  Feed the
 * rows to gs_upload_rows_device. */
int gs_pack_raw_device(const float* raw_dev, uint64_t count, float* rows_dev, void* stream);

/* Allocation-failure injection (no counterpart in the reference, whose
 * renderer refuses oversized scenes before allocating, src/renderer.cpp:717-763):
 * the device allocation after `after` more successful ones fails once with
 * GS_ERR_OOM, as a full GPU would make it fail; after < 0 turns it off.
 * Process-wide.  Every entry point that allocates leaves its context usable
 * after such a failure: a failed upload leaves no scene (GS_ERR_NO_SCENE
 * until the next successful one), a failed frame allocation fails that frame
 * only, and nothing half-uploaded stays behind. */
int gs_debug_fail_alloc(int64_t after);

/* load_gaussian_scene (src/gaussian.cpp:27-40): a scene file by its
 * extension, case-insensitively (.gsanim, .ply, .sog), as GpuGaussian rows
 * (for .gsanim the base Gaussians; its animation through gs_gsanim_load).
 * With rows == NULL returns the Gaussian count; otherwise fills
 * min(count, capacity) rows.  < 0 on error; GS_ERR_FORMAT for other
 * extensions. */
int64_t gs_load_scene(const char* path, float* rows, uint64_t capacity);

/* Load a SOG archive (version 2: meta.json and lossless WebP images) into
 * GpuGaussian rows with the reference loader's decode (gaussian_load_sog,
 * src/gaussian_loader_sog.cpp:126-551, and pack_gpu_gaussians,
 * src/gaussian.cpp:53-73).  With rows == NULL returns the Gaussian count;
 * otherwise fills min(count, capacity) rows.  GS_ERR_FORMAT (< 0) for files
 * the reference loader rejects, and for lossy WebP images and meta texts
 * that are not valid JSON, which it may accept. */
int64_t gs_load_sog(const char* path, float* rows, uint64_t capacity);

/* Decode a lossless WebP image (RIFF container or raw VP8L bitstream), the
 * image format of SOG archives, to RGBA8 rows top first: the WebPGetInfo +
 * WebPDecodeRGBA pair of the SOG loader (src/gaussian_loader_sog.cpp:98-124)
 * for lossless images.  Writes the size, and the pixels when `capacity` holds
 * width * height * 4 bytes.  GS_ERR_FORMAT for invalid, lossy or animated
 * images. */
int gs_webp_decode_rgba(const uint8_t* data, uint64_t size, int32_t* width, int32_t* height, uint8_t* rgba,
                        uint64_t capacity);

/* ---- gsanim assets (host, no GPU) ---------------------------------------- */

typedef struct gs_gsanim gs_gsanim;

typedef struct gs_gsanim_info {
    uint32_t version;          /* 1, 2, 3: manifest version "0.1", "0.2", "0.3" */
    uint32_t gaussian_count;
    uint32_t state_count;      /* appearance states incl. the base state 0 (0.1 / 0.2; 0 for 0.3) */
    uint32_t layer_count;      /* appearance layers (0.3) */
    uint32_t key_count;        /* state keys (0.1 / 0.2) */
    uint32_t lut_size;         /* display LUT edge (0.3) */
    int32_t linear;            /* manifest interpolation "linear" (0.1 / 0.2) */
    float log2_min, log2_max;  /* display LUT domain (0.3) */
    double duration_seconds;
} gs_gsanim_info;

/* gaussian_load_gsanim (src/gaussian_loader_gsanim.cpp:386-495): read and
 * validate a .gsanim archive (manifest.json, base.ply and scales.bin +
 * deltas.bin, or layers.bin + display_lut.bin).  Accepts exactly what the
 * reference loader accepts; GS_ERR_FORMAT otherwise (*out = NULL).  The
 * handle owns the decoded asset until gs_gsanim_free. */
int gs_gsanim_load(const char* path, gs_gsanim** out);
void gs_gsanim_free(gs_gsanim* asset);
int gs_gsanim_get_info(const gs_gsanim* asset, gs_gsanim_info* out);

/* The base Gaussians as GpuGaussian rows, gaussian_count x 64 floats (the
 * loader's Gaussian decode + pack_gpu_gaussians, src/gaussian.cpp:53-73):
 * the input of gs_upload_rows. */
int gs_gsanim_rows(const gs_gsanim* asset, float* rows);

/* GSAnim::deltas ((state_count - 1) x gaussian_count x 48 int8) and
 * GSAnim::scales (48 floats), src/gsanim.h:47-49: the inputs of
 * gs_upload_anim.  Either pointer may be NULL. */
int gs_gsanim_deltas(const gs_gsanim* asset, int8_t* deltas, float* scales);

/* GSAnim::layer_data (layer_count x gaussian_count x 48 IEEE half bits) and
 * GSAnim::display_lut (lut_size^3 x 3 uint16, red fastest), src/gsanim.h:38-41;
 * the LUT is the input of gs_set_display_lut. */
int gs_gsanim_layer_data(const gs_gsanim* asset, uint16_t* halves);
int gs_gsanim_display_lut(const gs_gsanim* asset, uint16_t* rgb);

/* Layer `layer`'s decoded UTF-8 name (GSAnimLayer::name; may hold NUL bytes):
 * copies min(length, capacity) bytes and returns the length. */
int64_t gs_gsanim_layer_name(const gs_gsanim* asset, uint32_t layer, char* buf, uint64_t capacity);

/* gsanim_sample (src/gaussian_loader_gsanim.cpp:497-509): the appearance
 * states and blend weight at `seconds` (wrapped into [0, duration)); state 0
 * for both and weight 0 for non-finite times or 0.3 assets.  The input of
 * gs_set_anim_state. */
int gs_gsanim_sample(const gs_gsanim* asset, double seconds, int32_t* state_a, int32_t* state_b, float* weight);

/* gsanim_layer_weights (src/gaussian_loader_gsanim.cpp:511-531): the RGB
 * weight of each layer at `seconds` into weights[layer_count * 3]; returns
 * the number of layers weighted, 0 (the reference's empty result) for 0.1 /
 * 0.2 assets and non-finite times. */
int gs_gsanim_layer_weights(const gs_gsanim* asset, double seconds, float* weights);

/* ---- stage-level entry points (device pointers, stream-ordered) ---------- */

/* Scratch bytes gs_sort_pairs needs for n pairs. */
size_t gs_sort_pairs_scratch_bytes(uint32_t n);

/* Stable ascending radix sort of (key, value) pairs on key bits
 * [begin_bit, end_bit): the order of the reference's 8-bit LSD passes
 * (shaders/sort.glsl:26-163, driven by src/renderer.cpp:1873-1962).
 * keys_in/vals_in are left unchanged; results go to keys_out/vals_out.
 * scratch: device memory of gs_sort_pairs_scratch_bytes(n) bytes.
 * Stream-ordered and never synchronising, so a bounded device wait that ran
 * out (a look-back that gave up, which needs a stalled GPU) is not reported
 * here; renders report theirs through gs_stats.error_flags. */
int gs_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                  uint32_t* vals_out, uint32_t n, int begin_bit, int end_bit, void* scratch,
                  size_t scratch_bytes, void* stream);

/* ---- stochastic-splat denoiser (the learned half of the render modes) ---- */

/* A 5-layer, 32-channel convolutional denoiser with a U-Net skip that turns
 * a two-sample stochastic frame (shaders/splat.glsl:127-145 without the
 * sort) plus its reprojected history (shaders/accum.glsl:148-178) into an
 * estimate of the sorted-alpha frame.  No counterpart in the reference,
 * which has no denoiser; its stochastic and sorted-alpha modes are the input
 * and the training target.
 *
 * Tensors are NHWC in device memory.  Input x: n x h x w x 16 bf16 (noisy RGB,
 * alpha, expected depth, reprojected history RGB, 8 zero channels); output:
 * n x h x w x 16 f32 (RGBA residual over (history RGB, alpha), then the
 * error estimate in channel 4, 1000 x the expected squared error); h, w even.
 * Layers, each a 3x3 "same" convolution on the tensor cores (BF16 operands,
 * FP32 accumulation):
 *   e1 = relu(conv1(x)) 16->32;  p1 = avgpool2(e1);  e2 = relu(conv2(p1));
 *   e3 = relu(conv3(e2));  d4 = relu(conv4(up2(e3) + e1));  o = conv5(d4) 32->16.
 * Parameters (gs_denoiser_param_count floats): per layer the weights as
 * [ky][kx][cin][cout] then the bias [cout].  All calls are stream-ordered
 * on the denoiser's stream unless they return host data. */
uint64_t gs_denoiser_param_count(void);
int gs_denoiser_create(gs_denoiser** out, int device, void* stream);   /* seeded initial parameters */
void gs_denoiser_destroy(gs_denoiser* d);
int gs_denoiser_init_params(gs_denoiser* d, uint64_t seed);            /* He initialisation, zero bias */
int gs_denoiser_set_params(gs_denoiser* d, const float* host, uint64_t count);   /* resets Adam's moments */
int gs_denoiser_get_params(gs_denoiser* d, float* host, uint64_t count);
int gs_denoiser_get_grads(gs_denoiser* d, float* host, uint64_t count);
/* Forward pass; `out` (device, may be NULL) receives the 16-channel output. */
int gs_denoiser_forward(gs_denoiser* d, const void* x_bf16, int n, int h, int w, float* out);
/* Parameter gradients (gs_denoiser_get_grads) of sum(out * dout) for the last
 * forward pass, which must have been on the same x; dout: n x h x w x 16 bf16.
 * The error estimate (output channel 4) is a head of the last layer alone: its
 * gradient trains conv5 and stops there (the trunk's features would otherwise
 * grow to chase their own error). */
int gs_denoiser_backward(gs_denoiser* d, const void* x_bf16, const void* dout_bf16, int n, int h, int w);
/* Training loss of an output against a target RGBA (n x h x w x 4 f32):
 *   L = mean |rgba - target| + ssim_weight (1 - mean SSIM(rgb)) + err_weight mean (o4 - 1000 e)^2,
 * SSIM with an 11-tap Gaussian window (sigma 1.5) over pixels at least 5 from the border,
 * e = mean over RGBA of (rgba - target)^2 (not differentiated).  Writes dL/dout
 * (bf16, 16 channels) to dout_bf16; with parts != NULL waits and stores
 * {mean L1, mean SSIM, error-head mean square, L}. */
int gs_denoiser_loss(gs_denoiser* d, const void* x_bf16, const float* out, const float* target, int n, int h,
                     int w, float ssim_weight, float err_weight, void* dout_bf16, float* parts);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected) with the last gradients. */
int gs_denoiser_adam(gs_denoiser* d, float lr);
/* forward + loss (ssim_weight 0.2, err_weight 0.01) + backward + Adam; with
 * loss_parts != NULL waits and stores the loss parts as gs_denoiser_loss. */
int gs_denoiser_train_step(gs_denoiser* d, const void* x_bf16, const float* target, int n, int h, int w, float lr,
                           float* loss_parts);
/* Waits; GS_ERR_DEVICE_TIMEOUT if a bounded device wait of a denoiser kernel ran out. */
int gs_denoiser_status(gs_denoiser* d);

/* One 3x3 "same" convolution of the denoiser on the tensor cores, NHWC bf16:
 * out[c] = epilogue(sum_{ky,kx,ci} in[y+ky-1][x+kx-1][ci] * weights[ky][kx][ci][c] + bias[c]),
 * epilogue = ReLU if relu, then 0 where mask <= 0 (mask: a tensor shaped like
 * the output, or NULL).  weights: device f32 [3][3][cin][cout]; with
 * transposed != 0 the convolution is the input gradient of that layer (input
 * of cout channels, output of cin channels).  x_half != NULL: the input is
 * x + the 2x nearest upsampling of x_half (n x h/2 x w/2, h and w >= 2; an
 * odd size's last row / column takes the last half-resolution one).  Supported
 * (input, output) channels: (16, 32), (32, 32), (32, 16), the last two with
 * x_half only for (32, 32).  image_scratch: gs_conv3x3_scratch_bytes(cin, cout)
 * device bytes; err: a device word, bit 0 set if a bounded wait ran out. */
size_t gs_conv3x3_scratch_bytes(int cin, int cout);
int gs_conv3x3_bf16(const void* x, const void* x_half, int n, int h, int w, int cin, int cout, const float* weights,
                    const float* bias, int relu, int transposed, const void* mask, void* out_bf16, float* out_f32,
                    void* image_scratch, uint32_t* err, void* stream);
/* Weight gradient of that convolution: dw[ky][kx][ci][c] += sum over pixels of
 * in[p + (ky-1, kx-1)][ci] * dy[p][c]; db[c] += sum of dy[p][c] (db may be NULL). */
int gs_conv3x3_wgrad_bf16(const void* x, const void* x_half, int n, int h, int w, int cin, int cout, const void* dy,
                          float* dw, float* db, uint32_t* err, void* stream);

/* gs_sort_pairs without any allocation; no counterpart in the reference.
 * For callers that cannot allocate device memory through this library: a
 * real-time render loop where cudaMalloc/cudaFree would synchronise the device
 * mid-frame, or a host engine whose memory manager owns every device
 * allocation.  The caller passes inputs and outputs; the scratch is a fixed
 * array of about 10 MiB in the library's device memory, held on every GPU that
 * loads the library until exit, so n is limited to 1,048,576 pairs
 * (GS_ERR_TOO_LARGE beyond).  The first call on a device, with that device
 * current, looks up the array's device address; make it before any stream
 * capture.  After a reset of the device's context (cudaDeviceReset) the next
 * call looks the address up again, in the new context.  Every call shares the array (each clears what must start at zero);
 * calls that overlap on the GPU race, so serialise them. */
int gs_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                          uint32_t* vals_out, uint32_t n, int begin_bit, int end_bit, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GS_API_H */
