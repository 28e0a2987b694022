// Host-side use of the asset entry points of gs_api.h: load a .gsanim archive,
// upload its base Gaussians and appearance data, and set the appearance for
// playback time t every frame (what load_gaussian_scene + the renderer's
// animation upload and per-frame sampling do in the reference,
// src/gaussian.cpp:27-40, src/renderer.cpp:824-881, 2148-2161).  Compiled by
// tests/test_abi.py against the public header.
#include <cstdint>
#include <vector>

#include "gs_api.h"

bool load_asset(gs_ctx* ctx, const char* path, double t) {
    gs_gsanim* anim = nullptr;
    if (gs_gsanim_load(path, &anim) != GS_OK) return false;   // GS_ERR_FORMAT: rejected like the reference
    gs_gsanim_info info;
    gs_gsanim_get_info(anim, &info);
    std::vector<float> rows((size_t)info.gaussian_count * 64);
    gs_gsanim_rows(anim, rows.data());
    gs_upload_rows(ctx, rows.data(), info.gaussian_count);
    if (info.version == 3) {   // half-float appearance layers
        std::vector<uint16_t> halves((size_t)info.layer_count * info.gaussian_count * 48);
        std::vector<uint16_t> lut((size_t)info.lut_size * info.lut_size * info.lut_size * 3);
        gs_gsanim_layer_data(anim, halves.data());
        gs_gsanim_display_lut(anim, lut.data());
        gs_upload_layers(ctx, halves.data(), info.layer_count);
        gs_set_display_lut(ctx, lut.data(), info.lut_size, info.log2_min, info.log2_max);
    } else {                   // int8 appearance states
        std::vector<int8_t> deltas((size_t)(info.state_count - 1) * info.gaussian_count * 48);
        float scales[48];
        gs_gsanim_deltas(anim, deltas.data(), scales);
        gs_upload_anim(ctx, deltas.data(), info.state_count - 1, scales);
    }
    // every frame, at playback time t:
    if (info.version == 3) {
        std::vector<float> w((size_t)info.layer_count * 3);
        gs_set_layer_weights(ctx, w.data(), (uint32_t)gs_gsanim_layer_weights(anim, t, w.data()));
    } else {
        int32_t a, b;
        float wgt;
        gs_gsanim_sample(anim, t, &a, &b, &wgt);
        gs_set_anim_state(ctx, a, b, wgt);
    }
    gs_gsanim_free(anim);
    return true;
}
