// Device-side GpuGaussian packing of raw 3DGS attributes: the PLY loader's
// transforms (src/gaussian_loader_ply.cpp:148-203: exp of the log-scales,
// sigmoid of the opacity logit, quaternion normalisation, f_rest reordered
// from channel-major to RGB triples) and the row layout of
// pack_gpu_gaussians (src/gaussian.cpp:53-73), so a scene can be decoded
// where it will be rendered instead of on the host.
//
// Same operation order as the host packer (gs_pack_raw, compiled without
// FMA contraction).  exp is evaluated in double precision and rounded to
// float (correctly rounded except in double-rounding ties); the host uses
// glibc's expf, which is not correctly rounded for about 0.008 % of float
// arguments, so there a scale can differ from the host row by one ulp and an
// opacity by up to two (a one-ulp change of 1 + exp(-x) can move the
// quotient two ulps).  Every other field is bit-identical.
#include "gs_common.cuh"
#include "gs_internal.h"

namespace gs {

__device__ __forceinline__ float exp_cr(float x) { return __double2float_rn(exp((double)x)); }

// One thread per Gaussian: raw row of 59 floats (x y z, f_dc 0..2,
// f_rest 0..44, opacity, scale 0..2, rot 0..3) -> 64-float GpuGaussian row.
__global__ void pack_raw_kernel(const float* __restrict__ raw, uint64_t count, float4* __restrict__ rows) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float* r = raw + i * 59;
        float d[64];
#pragma unroll
        for (int k = 0; k < 64; ++k) d[k] = 0.0f;
        d[0] = __ldg(r + 0);
        d[1] = __ldg(r + 1);
        d[2] = __ldg(r + 2);
        d[4] = exp_cr(__ldg(r + 52));
        d[5] = exp_cr(__ldg(r + 53));
        d[6] = exp_cr(__ldg(r + 54));
        float rw = __ldg(r + 55), rx = __ldg(r + 56), ry = __ldg(r + 57), rz = __ldg(r + 58);
        const float len = __fsqrt_rn(add(add(add(mul(rw, rw), mul(rx, rx)), mul(ry, ry)), mul(rz, rz)));
        if (len > 1e-8f) {
            rw = dv(rw, len);
            rx = dv(rx, len);
            ry = dv(ry, len);
            rz = dv(rz, len);
        }
        d[8] = rw;
        d[9] = rx;
        d[10] = ry;
        d[11] = rz;
        d[3] = dv(1.0f, add(1.0f, exp_cr(-__ldg(r + 51))));   // sigmoid
        d[12] = __ldg(r + 3);
        d[13] = __ldg(r + 4);
        d[14] = __ldg(r + 5);
#pragma unroll
        for (int k = 0; k < 15; ++k) {
            d[16 + k * 3 + 0] = __ldg(r + 6 + k);
            d[16 + k * 3 + 1] = __ldg(r + 6 + 15 + k);
            d[16 + k * 3 + 2] = __ldg(r + 6 + 30 + k);
        }
        float4* o = rows + i * 16;
#pragma unroll
        for (int k = 0; k < 16; ++k) o[k] = make_float4(d[4 * k], d[4 * k + 1], d[4 * k + 2], d[4 * k + 3]);
    }
}

}  // namespace gs

extern "C" int gs_pack_raw_device(const float* raw_dev, uint64_t count, float* rows_dev, void* stream) {
    if (count == 0) return GS_OK;
    if (!raw_dev || !rows_dev || ((uintptr_t)rows_dev & 15u)) return GS_ERR_BAD_ARG;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t grid = (count + 127) / 128;
    const uint64_t cap = (uint64_t)(sms > 0 ? sms : 148) * 16;
    if (grid > cap) grid = cap;
    gs::pack_raw_kernel<<<(unsigned)grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        raw_dev, count, reinterpret_cast<float4*>(rows_dev));
    return cudaGetLastError() == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}
