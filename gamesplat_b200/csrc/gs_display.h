// Internal interface of the display transform (gs_display.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gs {

struct DisplayParams {
    const uint16_t* in_rgba16f;   // width*height*4 halves (a gs_render frame), top row first
    float4* out_rgba32f;          // width*height display colours, top row first
    int width, height;
    const uint16_t* lut;          // lut_size^3 x RGB uint16 (x fastest), or null for the plain blit
    int lut_size;
    float log2_min, log2_max;
    float exposure_ev;
};

int launch_display(const DisplayParams& p, uint32_t num_sms, cudaStream_t s);

}  // namespace gs
