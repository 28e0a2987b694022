// Host side of the stochastic-splat denoiser: parameters, activations, the
// forward and backward passes, the L1 + SSIM loss and Adam, behind the C ABI
// of include/gs_api.h (gs_denoiser_*, gs_conv3x3_*).  Kernels: gs_conv.cu
// (tensor-core convolutions), gs_denoise.cu (everything else).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "gs_conv.h"
#include "gs_denoise.h"
#include "gs_denoiser.h"
#include "gs_internal.h"

namespace {

using bf16 = __nv_bfloat16;

struct Layer {
    int cin, cout, relu, load;
};
// conv1 .. conv5 (see gs_denoise.cu for the network)
constexpr Layer kNet[gs::dn::kLayers] = {
    {gs::dn::kInC, gs::dn::kHidC, 1, 0}, {gs::dn::kHidC, gs::dn::kHidC, 1, 0}, {gs::dn::kHidC, gs::dn::kHidC, 1, 0},
    {gs::dn::kHidC, gs::dn::kHidC, 1, 1}, {gs::dn::kHidC, gs::dn::kOutC, 0, 0}};

constexpr int kErrChannel = 4;   // output channel of the error estimate

constexpr size_t w_count(int l) { return (size_t)9 * kNet[l].cin * kNet[l].cout; }
size_t w_offset(int l) {
    size_t o = 0;
    for (int k = 0; k < l; ++k) o += w_count(k) + (size_t)kNet[k].cout;
    return o;
}
size_t b_offset(int l) { return w_offset(l) + w_count(l); }
size_t param_count() { return b_offset(gs::dn::kLayers - 1) + (size_t)kNet[gs::dn::kLayers - 1].cout; }

template <class T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    return gs::device_malloc(reinterpret_cast<void**>(p), std::max<size_t>(count * sizeof(T), 16));
}
template <class T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

}  // namespace

struct gs_denoiser {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t num_sms = 148;
    float* params = nullptr;
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int adam_t = 0;
    uint8_t* wimg[gs::dn::kLayers] = {};
    uint8_t* wimg_t[gs::dn::kLayers] = {};
    bool images_valid = false;
    uint32_t* err = nullptr;
    float* acc = nullptr;       // loss accumulators
    float* h_acc = nullptr;     // pinned
    // activations (capacity in full-resolution pixels)
    size_t cap = 0;
    bf16 *e1 = nullptr, *p1 = nullptr, *e2 = nullptr, *e3 = nullptr, *d4 = nullptr;
    float* out = nullptr;
    // training
    size_t tcap = 0;
    float4* pred = nullptr;
    float *mom = nullptr, *tmp = nullptr, *bmom = nullptr, *part = nullptr, *bpart = nullptr;
    bf16 *dout = nullptr, *dz4 = nullptr, *du = nullptr, *dz3 = nullptr, *dz2 = nullptr, *dp1 = nullptr,
         *dz1 = nullptr;
    int last_n = 0, last_h = 0, last_w = 0;
    const void* last_x = nullptr;
};

namespace gs {
namespace dn {

uint64_t parameter_count() { return param_count(); }
const float* output(const gs_denoiser* d) { return d->out; }

static void release_acts(gs_denoiser* d) {
    dfree(d->e1);
    dfree(d->p1);
    dfree(d->e2);
    dfree(d->e3);
    dfree(d->d4);
    dfree(d->out);
    d->cap = 0;
}

static void release_train(gs_denoiser* d) {
    dfree(d->pred);
    dfree(d->mom);
    dfree(d->tmp);
    dfree(d->bmom);
    dfree(d->part);
    dfree(d->bpart);
    dfree(d->dout);
    dfree(d->dz4);
    dfree(d->du);
    dfree(d->dz3);
    dfree(d->dz2);
    dfree(d->dp1);
    dfree(d->dz1);
    d->tcap = 0;
}

static int ensure_acts(gs_denoiser* d, size_t pix) {
    if (pix <= d->cap) return GS_OK;
    release_acts(d);
    const size_t half = pix / 4 + 1;
    if (dalloc(&d->e1, pix * kHidC) || dalloc(&d->p1, half * kHidC) || dalloc(&d->e2, half * kHidC) ||
        dalloc(&d->e3, half * kHidC) || dalloc(&d->d4, pix * kHidC) || dalloc(&d->out, pix * kOutC)) {
        release_acts(d);
        return GS_ERR_OOM;
    }
    d->cap = pix;
    return GS_OK;
}

static int ensure_train(gs_denoiser* d, size_t pix) {
    if (pix <= d->tcap) return GS_OK;
    release_train(d);
    const size_t half = pix / 4 + 1;
    if (dalloc(&d->pred, pix) || dalloc(&d->mom, pix * 15) || dalloc(&d->tmp, pix * 15) ||
        dalloc(&d->bmom, pix * 15) || dalloc(&d->part, pix * 9) || dalloc(&d->bpart, pix * 9) ||
        dalloc(&d->dout, pix * kOutC) || dalloc(&d->dz4, pix * kHidC) || dalloc(&d->du, pix * kHidC) ||
        dalloc(&d->dz3, half * kHidC) || dalloc(&d->dz2, half * kHidC) || dalloc(&d->dp1, half * kHidC) ||
        dalloc(&d->dz1, pix * kHidC)) {
        release_train(d);
        return GS_ERR_OOM;
    }
    d->tcap = pix;
    return GS_OK;
}

static void pack_images(gs_denoiser* d, cudaStream_t s) {
    for (int l = 0; l < gs::dn::kLayers; ++l) {
        conv::launch_pack_weights(d->params + w_offset(l), kNet[l].cin, kNet[l].cout, 0, d->wimg[l], s);
        // the error estimate (channel 4 of the last layer) trains the last layer only: its gradient
        // does not reach the trunk, whose features would otherwise chase their own growing error
        conv::launch_pack_weights(d->params + w_offset(l), kNet[l].cin, kNet[l].cout, 1, d->wimg_t[l], s,
                                  l == gs::dn::kLayers - 1 ? kErrChannel : -1);
    }
    d->images_valid = true;
}

static int rows_per_cta(const gs_denoiser* d, int n, int h, int w) {
    const long strips = (long)n * ((w + 127) / 128);
    const long want = (long)d->num_sms * 8;   // enough CTAs for every SM's occupancy, a few rows each
    long rows = (strips * h + want - 1) / want;
    return (int)std::max(2L, std::min(64L, rows));
}

static int conv_fwd(gs_denoiser* d, int l, bool transposed, const bf16* x, const bf16* xh, int n, int h, int w,
                    const bf16* mask, bf16* out_bf16, float* out_f32, cudaStream_t s) {
    const Layer& L = kNet[l];
    conv::ConvArgs a{};
    a.x = x;
    a.xh = xh;
    a.n = n;
    a.h = h;
    a.w = w;
    a.wimage = transposed ? d->wimg_t[l] : d->wimg[l];
    a.bias = transposed ? nullptr : d->params + b_offset(l);
    a.relu = transposed ? 0 : L.relu;
    a.mask = mask;
    a.out_bf16 = out_bf16;
    a.out_f32 = out_f32;
    a.rows_per_cta = rows_per_cta(d, n, h, w);
    a.err = d->err;
    if (l == 0 && !transposed) {   // conv1 also writes p1 = avgpool2(e1): row bands of an even number of rows
        a.pool_out = d->p1;
        a.rows_per_cta = (a.rows_per_cta + 1) & ~1;
    }
    const int cin = transposed ? L.cout : L.cin, cout = transposed ? L.cin : L.cout;
    return conv::launch_fwd(cin, cout, transposed ? 0 : L.load, a, s) < 0 ? GS_ERR_BAD_ARG : GS_OK;
}

static int conv_wgrad(gs_denoiser* d, int l, const bf16* x, const bf16* xh, int n, int h, int w, const bf16* dy) {
    const Layer& L = kNet[l];
    conv::WgradArgs a{};
    a.x = x;
    a.xh = xh;
    a.n = n;
    a.h = h;
    a.w = w;
    a.dy = dy;
    a.dw = d->grads + w_offset(l);
    a.db = d->grads + b_offset(l);
    a.err = d->err;
    const long blocks = (long)n * h * ((w + 63) / 64);
    const int grid = (int)std::max(1L, std::min<long>(blocks, (long)d->num_sms * 2));
    return conv::launch_wgrad(L.cin, L.cout, L.load, a, grid, d->stream) < 0 ? GS_ERR_BAD_ARG : GS_OK;
}

int forward(gs_denoiser* d, const bf16* x, int n, int h, int w, cudaStream_t s) {
    if (n <= 0 || h <= 0 || w <= 0 || (h & 1) || (w & 1)) return GS_ERR_BAD_ARG;
    const size_t pix = (size_t)n * h * w;
    int rc = ensure_acts(d, pix);
    if (rc) return rc;
    if (!d->images_valid) pack_images(d, s);
    const int hh = h / 2, hw = w / 2;
    if ((rc = conv_fwd(d, 0, false, x, nullptr, n, h, w, nullptr, d->e1, nullptr, s))) return rc;   // e1 and p1
    if ((rc = conv_fwd(d, 1, false, d->p1, nullptr, n, hh, hw, nullptr, d->e2, nullptr, s))) return rc;
    if ((rc = conv_fwd(d, 2, false, d->e2, nullptr, n, hh, hw, nullptr, d->e3, nullptr, s))) return rc;
    if ((rc = conv_fwd(d, 3, false, d->e1, d->e3, n, h, w, nullptr, d->d4, nullptr, s))) return rc;
    if ((rc = conv_fwd(d, 4, false, d->d4, nullptr, n, h, w, nullptr, nullptr, d->out, s))) return rc;
    d->last_n = n;
    d->last_h = h;
    d->last_w = w;
    d->last_x = x;
    return GS_OK;
}

int forward_frame(gs_denoiser* d, const bf16* x, int h, int w, uint16_t* out16, int tiles_x, float err_budget,
                  uint32_t* fallback_count, uint32_t* fallback_tiles, float* tile_err, cudaStream_t s) {
    if (h <= 0 || w <= 0 || (h & 1) || (w & 1) || !out16 || !fallback_count || !fallback_tiles) return GS_ERR_BAD_ARG;
    int rc = ensure_acts(d, (size_t)h * w);
    if (rc) return rc;
    d->last_x = nullptr;   // the activations are this frame's now: no backward pass follows
    d->last_n = 0;
    if (!d->images_valid) pack_images(d, s);
    const int hh = h / 2, hw = w / 2;
    if ((rc = conv_fwd(d, 0, false, x, nullptr, 1, h, w, nullptr, d->e1, nullptr, s))) return rc;   // e1 and p1
    if ((rc = conv_fwd(d, 1, false, d->p1, nullptr, 1, hh, hw, nullptr, d->e2, nullptr, s))) return rc;
    if ((rc = conv_fwd(d, 2, false, d->e2, nullptr, 1, hh, hw, nullptr, d->e3, nullptr, s))) return rc;
    if ((rc = conv_fwd(d, 3, false, d->e1, d->e3, 1, h, w, nullptr, d->d4, nullptr, s))) return rc;
    // the last layer with the output step in its epilogue: row bands of 16 rows aligned with the tiles
    const Layer& L = kNet[4];
    conv::ConvArgs a{};
    a.x = d->d4;
    a.n = 1;
    a.h = h;
    a.w = w;
    a.wimage = d->wimg[4];
    a.bias = d->params + b_offset(4);
    a.relu = L.relu;
    a.rows_per_cta = 16;
    a.row_offset = (16 - h % 16) % 16;
    a.err = d->err;
    a.head_x = x;
    a.head_out16 = out16;
    a.tile_err = tile_err;
    a.fallback_count = fallback_count;
    a.fallback_tiles = fallback_tiles;
    a.err_budget = err_budget;
    a.tiles_x = tiles_x;
    return conv::launch_fwd(L.cin, L.cout, L.load, a, s) < 0 ? GS_ERR_BAD_ARG : GS_OK;
}

int backward(gs_denoiser* d, const bf16* x, const bf16* dout, int n, int h, int w) {
    if (d->last_x != x || d->last_n != n || d->last_h != h || d->last_w != w) return GS_ERR_BAD_ARG;
    const size_t pix = (size_t)n * h * w;
    int rc = ensure_train(d, pix);
    if (rc) return rc;
    const int hh = h / 2, hw = w / 2;
    cudaMemsetAsync(d->grads, 0, param_count() * sizeof(float), d->stream);
    // conv5
    if ((rc = conv_wgrad(d, 4, d->d4, nullptr, n, h, w, dout))) return rc;
    if ((rc = conv_fwd(d, 4, true, dout, nullptr, n, h, w, d->d4, d->dz4, nullptr, d->stream))) return rc;
    // conv4 (input up2(e3) + e1)
    if ((rc = conv_wgrad(d, 3, d->e1, d->e3, n, h, w, d->dz4))) return rc;
    if ((rc = conv_fwd(d, 3, true, d->dz4, nullptr, n, h, w, nullptr, d->du, nullptr, d->stream))) return rc;
    launch_upsample_grad(d->du, d->e3, n, h, w, d->dz3, d->stream);
    // conv3, conv2 at half resolution
    if ((rc = conv_wgrad(d, 2, d->e2, nullptr, n, hh, hw, d->dz3))) return rc;
    if ((rc = conv_fwd(d, 2, true, d->dz3, nullptr, n, hh, hw, d->e2, d->dz2, nullptr, d->stream))) return rc;
    if ((rc = conv_wgrad(d, 1, d->p1, nullptr, n, hh, hw, d->dz2))) return rc;
    if ((rc = conv_fwd(d, 1, true, d->dz2, nullptr, n, hh, hw, nullptr, d->dp1, nullptr, d->stream))) return rc;
    launch_skip_pool_grad(d->du, d->dp1, d->e1, n, h, w, d->dz1, d->stream);
    // conv1
    return conv_wgrad(d, 0, x, nullptr, n, h, w, d->dz1);
}

int loss(gs_denoiser* d, const bf16* x, const float* out, const float4* target, int n, int h, int w, bf16* dout,
         float ssim_weight, float err_weight) {
    const size_t pix = (size_t)n * h * w;
    int rc = ensure_train(d, pix);
    if (rc) return rc;
    cudaMemsetAsync(d->acc, 0, 4 * sizeof(float), d->stream);
    const bool ssim = ssim_weight > 0.0f && h > 10 && w > 10;
    launch_head_moments(out, x, target, (int)pix, d->pred, ssim ? d->mom : nullptr, d->stream);
    float ssim_scale = 0.0f;
    if (ssim) {
        launch_blur(d->mom, n, h, w, 15, 0, d->tmp, d->stream);
        launch_blur(d->tmp, n, h, w, 15, 1, d->bmom, d->stream);
        launch_ssim_partials(d->bmom, n, h, w, d->part, d->acc, d->stream);
        launch_blur(d->part, n, h, w, 9, 0, d->tmp, d->stream);
        launch_blur(d->tmp, n, h, w, 9, 1, d->bpart, d->stream);
        ssim_scale = ssim_weight / (3.0f * (float)n * (float)(h - 10) * (float)(w - 10));
    }
    launch_loss_grad(out, d->pred, target, ssim ? d->bpart : nullptr, (int)pix, 1.0f / (4.0f * (float)pix),
                     ssim_scale, err_weight / (float)pix, dout, d->acc, d->stream);
    return GS_OK;
}

}  // namespace dn
}  // namespace gs

using namespace gs::dn;

namespace {

int check_err(gs_denoiser* d) {
    uint32_t e = 0;
    if (cudaMemcpyAsync(&e, d->err, 4, cudaMemcpyDeviceToHost, d->stream) != cudaSuccess ||
        cudaStreamSynchronize(d->stream) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    return e ? GS_ERR_DEVICE_TIMEOUT : GS_OK;
}

int launched(gs_denoiser* d, int rc) {
    if (rc) return rc;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? GS_ERR_OOM : GS_ERR_CUDA;
    (void)d;
    return GS_OK;
}

// Deterministic normal draws for the initial weights (SplitMix64 + Box-Muller).
struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() { return std::sqrt(-2.0 * std::log(uniform())) * std::cos(6.283185307179586 * uniform()); }
};

}  // namespace

extern "C" {

uint64_t gs_denoiser_param_count(void) { return param_count(); }

int gs_denoiser_create(gs_denoiser** out, int device, void* stream) {
    if (!out) return GS_ERR_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GS_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return GS_ERR_BAD_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GS_ERR_NO_DEVICE;
    gs_denoiser* d = new (std::nothrow) gs_denoiser();
    if (!d) return GS_ERR_OOM;
    d->device = device;
    d->stream = static_cast<cudaStream_t>(stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    d->num_sms = sms > 0 ? (uint32_t)sms : 148u;
    const size_t pc = param_count();
    bool ok = !dalloc(&d->params, pc) && !dalloc(&d->grads, pc) && !dalloc(&d->adam_m, pc) &&
              !dalloc(&d->adam_v, pc) && !dalloc(&d->err, 4) && !dalloc(&d->acc, 4) &&
              cudaMallocHost(reinterpret_cast<void**>(&d->h_acc), 4 * sizeof(float)) == cudaSuccess;
    for (int l = 0; ok && l < gs::dn::kLayers; ++l) {
        const size_t b = gs::conv::weight_image_bytes(kNet[l].cin, kNet[l].cout);
        ok = !dalloc(&d->wimg[l], b) && !dalloc(&d->wimg_t[l], b);
    }
    if (!ok) {
        gs_denoiser_destroy(d);
        return GS_ERR_OOM;
    }
    cudaMemsetAsync(d->err, 0, 16, d->stream);
    set_gauss_window(d->stream);
    const int rc = gs_denoiser_init_params(d, 1);
    if (rc) {
        gs_denoiser_destroy(d);
        return rc;
    }
    *out = d;
    return GS_OK;
}

void gs_denoiser_destroy(gs_denoiser* d) {
    if (!d) return;
    cudaSetDevice(d->device);
    cudaStreamSynchronize(d->stream);
    release_acts(d);
    release_train(d);
    dfree(d->params);
    dfree(d->grads);
    dfree(d->adam_m);
    dfree(d->adam_v);
    dfree(d->err);
    dfree(d->acc);
    for (int l = 0; l < gs::dn::kLayers; ++l) {
        dfree(d->wimg[l]);
        dfree(d->wimg_t[l]);
    }
    if (d->h_acc) cudaFreeHost(d->h_acc);
    delete d;
}

int gs_denoiser_init_params(gs_denoiser* d, uint64_t seed) {
    if (!d) return GS_ERR_BAD_ARG;
    const size_t pc = param_count();
    float* h = new (std::nothrow) float[pc];
    if (!h) return GS_ERR_OOM;
    Rng r{seed * 0x2545F4914F6CDD1Dull + 1};
    for (int l = 0; l < gs::dn::kLayers; ++l) {
        // He initialisation; the last layer starts small so the first output
        // is close to the reprojected history
        const double sd = std::sqrt(2.0 / (9.0 * kNet[l].cin)) * (l == gs::dn::kLayers - 1 ? 0.1 : 1.0);
        for (size_t i = 0; i < w_count(l); ++i) h[w_offset(l) + i] = (float)(sd * r.normal());
        for (int c = 0; c < kNet[l].cout; ++c) h[b_offset(l) + c] = 0.0f;
    }
    const int rc = gs_denoiser_set_params(d, h, pc);
    delete[] h;
    return rc;
}

int gs_denoiser_set_params(gs_denoiser* d, const float* host, uint64_t count) {
    if (!d || !host || count != param_count()) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    if (cudaMemcpyAsync(d->params, host, count * sizeof(float), cudaMemcpyHostToDevice, d->stream) != cudaSuccess ||
        cudaMemsetAsync(d->adam_m, 0, count * sizeof(float), d->stream) != cudaSuccess ||
        cudaMemsetAsync(d->adam_v, 0, count * sizeof(float), d->stream) != cudaSuccess ||
        cudaStreamSynchronize(d->stream) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    d->adam_t = 0;
    pack_images(d, d->stream);
    // a renderer may run the network on its own stream next
    if (cudaStreamSynchronize(d->stream) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    return launched(d, GS_OK);
}

static int read_buffer(gs_denoiser* d, const float* src, float* host, uint64_t count) {
    if (!d || !host || count != param_count()) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    if (cudaMemcpyAsync(host, src, count * sizeof(float), cudaMemcpyDeviceToHost, d->stream) != cudaSuccess ||
        cudaStreamSynchronize(d->stream) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    return GS_OK;
}

int gs_denoiser_get_params(gs_denoiser* d, float* host, uint64_t count) {
    return read_buffer(d, d ? d->params : nullptr, host, count);
}

int gs_denoiser_get_grads(gs_denoiser* d, float* host, uint64_t count) {
    return read_buffer(d, d ? d->grads : nullptr, host, count);
}

int gs_denoiser_forward(gs_denoiser* d, const void* x, int n, int h, int w, float* out) {
    if (!d || !x) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    int rc = launched(d, forward(d, static_cast<const bf16*>(x), n, h, w, d->stream));
    if (rc) return rc;
    if (out) {
        if (cudaMemcpyAsync(out, d->out, (size_t)n * h * w * kOutC * sizeof(float), cudaMemcpyDeviceToDevice,
                            d->stream) != cudaSuccess)
            return GS_ERR_CUDA;
    }
    return GS_OK;
}

int gs_denoiser_backward(gs_denoiser* d, const void* x, const void* dout, int n, int h, int w) {
    if (!d || !x || !dout) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    return launched(d, backward(d, static_cast<const bf16*>(x), static_cast<const bf16*>(dout), n, h, w));
}

int gs_denoiser_loss(gs_denoiser* d, const void* x, const float* out, const float* target, int n, int h, int w,
                     float ssim_weight, float err_weight, void* dout, float* parts) {
    if (!d || !x || !out || !target || !dout || n <= 0 || h <= 0 || w <= 0) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    int rc = launched(d, loss(d, static_cast<const bf16*>(x), out, reinterpret_cast<const float4*>(target), n, h, w,
                              static_cast<bf16*>(dout), ssim_weight, err_weight));
    if (rc || !parts) return rc;
    if (cudaMemcpyAsync(d->h_acc, d->acc, 4 * sizeof(float), cudaMemcpyDeviceToHost, d->stream) != cudaSuccess ||
        cudaStreamSynchronize(d->stream) != cudaSuccess)
        return GS_ERR_CUDA;
    const double pix = (double)n * h * w;
    parts[0] = (float)(d->h_acc[2] / (4.0 * pix));                          // mean |pred - target|
    parts[1] = d->h_acc[1] > 0.0f ? d->h_acc[0] / d->h_acc[1] : 1.0f;      // mean SSIM
    parts[2] = (float)(d->h_acc[3] / pix);                                 // error-head mean square
    parts[3] = parts[0] + ssim_weight * (1.0f - parts[1]) + err_weight * parts[2];
    return GS_OK;
}

int gs_denoiser_adam(gs_denoiser* d, float lr) {
    if (!d || !(lr > 0.0f)) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    d->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - (float)std::pow(b1, d->adam_t), bc2 = 1.0f - (float)std::pow(b2, d->adam_t);
    launch_adam(d->params, d->grads, d->adam_m, d->adam_v, (int)param_count(), lr, b1, b2, 1e-8f, bc1, bc2,
                d->stream);
    pack_images(d, d->stream);
    return launched(d, GS_OK);
}

int gs_denoiser_train_step(gs_denoiser* d, const void* x, const float* target, int n, int h, int w, float lr,
                           float* loss_parts) {
    if (!d || !x || !target) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    int rc = gs_denoiser_forward(d, x, n, h, w, nullptr);
    if (rc) return rc;
    if ((rc = ensure_train(d, (size_t)n * h * w))) return rc;
    rc = gs_denoiser_loss(d, x, d->out, target, n, h, w, kTrainSsimWeight, kTrainErrWeight, d->dout, loss_parts);
    if (rc) return rc;
    if ((rc = gs_denoiser_backward(d, x, d->dout, n, h, w))) return rc;
    if ((rc = gs_denoiser_adam(d, lr))) return rc;
    return loss_parts ? check_err(d) : GS_OK;
}

int gs_denoiser_status(gs_denoiser* d) {
    if (!d) return GS_ERR_BAD_ARG;
    cudaSetDevice(d->device);
    return check_err(d);
}

// ---- stage-level convolutions ----------------------------------------------
int gs_conv3x3_bf16(const void* x, const void* x_half, int n, int h, int w, int cin, int cout, const float* weights,
                    const float* bias, int relu, int transposed, const void* mask, void* out_bf16, float* out_f32,
                    void* image_scratch, uint32_t* err, void* stream) {
    if (!x || !weights || !image_scratch || !err || n <= 0 || h <= 0 || w <= 0) return GS_ERR_BAD_ARG;
    if (x_half && (h < 2 || w < 2)) return GS_ERR_BAD_ARG;   // the half-resolution input has no pixels
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // weights are [tap][cin][cout] of the layer; transposed: the input gradient
    // of that layer (an input of cout channels, an output of cin channels)
    gs::conv::launch_pack_weights(weights, cin, cout, transposed ? 1 : 0, static_cast<uint8_t*>(image_scratch), s);
    gs::conv::ConvArgs a{};
    a.x = static_cast<const bf16*>(x);
    a.xh = static_cast<const bf16*>(x_half);
    a.n = n;
    a.h = h;
    a.w = w;
    a.wimage = static_cast<const uint8_t*>(image_scratch);
    a.bias = bias;
    a.relu = relu;
    a.mask = static_cast<const bf16*>(mask);
    a.out_bf16 = static_cast<bf16*>(out_bf16);
    a.out_f32 = out_f32;
    a.rows_per_cta = 8;
    a.err = err;
    const int ci = transposed ? cout : cin, co = transposed ? cin : cout;
    if (gs::conv::launch_fwd(ci, co, x_half ? 1 : 0, a, s) < 0) return GS_ERR_BAD_ARG;
    return cudaGetLastError() == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}

int gs_conv3x3_wgrad_bf16(const void* x, const void* x_half, int n, int h, int w, int cin, int cout, const void* dy,
                          float* dw, float* db, uint32_t* err, void* stream) {
    if (!x || !dy || !dw || !err || n <= 0 || h <= 0 || w <= 0) return GS_ERR_BAD_ARG;
    if (x_half && (h < 2 || w < 2)) return GS_ERR_BAD_ARG;
    gs::conv::WgradArgs a{};
    a.x = static_cast<const bf16*>(x);
    a.xh = static_cast<const bf16*>(x_half);
    a.n = n;
    a.h = h;
    a.w = w;
    a.dy = static_cast<const bf16*>(dy);
    a.dw = dw;
    a.db = db;
    a.err = err;
    if (gs::conv::launch_wgrad(cin, cout, x_half ? 1 : 0, a, 296, static_cast<cudaStream_t>(stream)) < 0)
        return GS_ERR_BAD_ARG;
    return cudaGetLastError() == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}

size_t gs_conv3x3_scratch_bytes(int cin, int cout) { return gs::conv::weight_image_bytes(cin, cout); }

}  // extern "C"
