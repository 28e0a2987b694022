// Launchers of the denoiser's tensor-core convolutions (gs_conv.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace gs {
namespace conv {

// One 3x3 "same" convolution, NHWC bf16 in, per output pixel
//   out[c] = epilogue(sum over taps and input channels + bias[c]).
struct ConvArgs {
    const __nv_bfloat16* x;     // input (Cin channels), or the full-resolution term of load mode 1
    const __nv_bfloat16* xh;    // load mode 1: half-resolution term, upsampled 2x (nearest) and added to x
    int n, h, w;                // batch and spatial size (input = output; h, w even in load mode 1)
    const uint8_t* wimage;      // packed weights (launch_pack_weights)
    const float* bias;          // Cout floats or null
    int relu;                   // max(., 0) after the bias
    const __nv_bfloat16* mask;  // Cout-channel tensor: outputs where mask <= 0 become 0 (ReLU backward); or null
    __nv_bfloat16* out_bf16;    // Cout channels, or null
    float* out_f32;             // Cout channels, or null
    int rows_per_cta;
    uint32_t* err;              // bit 0 set if a bounded wait ran out
    int row_offset;             // the row bands of the CTAs start at -row_offset (0: at row 0)
    // (Cin = 16, Cout = 32, forward): also the 2x2 average of the bf16 output, n x h/2 x w/2 (h, w
    // and rows_per_cta even), summed and rounded as the denoiser's pooling kernel does
    __nv_bfloat16* pool_out;
    // Denoised-mode head (Cout = 16, forward, head_x set): the epilogue writes head_out16 =
    // RGBA16F (head_x[5..7] + o[0..2], head_x[3] + o[3]) instead of the outputs above and,
    // per 16x16 tile of GL rows (rows_per_cta = 16 and row_offset aligning the bands with
    // them), tile_err = mean(max(o[4], 0)) * 0.001, listing tiles at or above err_budget.
    const __nv_bfloat16* head_x;   // the network input (16 channels per pixel)
    uint16_t* head_out16;
    float* tile_err;
    uint32_t* fallback_count;
    uint32_t* fallback_tiles;
    float err_budget;
    int tiles_x;
};

// dw[tap * Cin + cin][cout] += sum over pixels of X[p + tap][cin] * dy[p][cout],
// db[cout] += sum over pixels of dy[p][cout].
struct WgradArgs {
    const __nv_bfloat16* x;     // layer input (as ConvArgs::x)
    const __nv_bfloat16* xh;    // load mode 1 (as ConvArgs::xh)
    int n, h, w;
    const __nv_bfloat16* dy;    // gradient of the layer output (Cout channels)
    float* dw;                  // 9 * Cin * Cout floats, accumulated
    float* db;                  // Cout floats, accumulated, or null
    uint32_t* err;
};

// Supported (cin, cout, load mode): (16, 32, 0), (32, 32, 0), (32, 16, 0), (32, 32, 1).
// Return the number of kernels launched, or -1 for an unsupported shape.
int launch_fwd(int cin, int cout, int load_mode, const ConvArgs& a, cudaStream_t s);
int launch_wgrad(int cin, int cout, int load_mode, const WgradArgs& a, int grid, cudaStream_t s);
// transposed: the image of the layer's input gradient; cut_cout >= 0 leaves that
// output channel out of it (its gradient stops at the layer)
int launch_pack_weights(const float* w, int cin, int cout, int transposed, uint8_t* image, cudaStream_t s,
                        int cut_cout = -1);
size_t weight_image_bytes(int cin, int cout);

}  // namespace conv
}  // namespace gs
