// 3x3 "same" convolutions of the denoiser on the fifth-generation tensor
// cores (tcgen05.mma, BF16 operands, FP32 accumulators in TMEM).
//
// Tensors are NHWC bf16.  Weights are kept as FP32 masters in [tap][cin][cout]
// order (tap = ky * 3 + kx, ky = 0 the row above); each step packs them into
// the byte image of the shared-memory operand the kernels copy verbatim.
//
// conv_fwd_kernel (also the input gradient, with the transposed weights):
// implicit GEMM with M = 128 output pixels of one image row, N = Cout,
// K = 9 taps x Cin.  A CTA walks a column strip of 128 pixels down a run of
// rows; three input rows (the row above, the row, the row below, 130 pixels
// with the halo) sit in shared memory in the K-major core-matrix layout,
// rows of 16 bytes one pixel apart, so the A operand of tap (ky, kx) is the
// same buffer started kx pixels (kx * 16 bytes) further: no im2col copy.
// Per output row the CTA loads one new input row, one thread issues
// 9 * Cin / 16 MMAs into a TMEM accumulator, and the four warps read it back
// (thread t = TMEM lane t = pixel t) for the epilogue (bias, ReLU, ReLU
// mask, bf16 / f32 store).
//
// conv_wgrad_kernel: dW[tap, cin][cout] = sum over pixels of
// X[p + tap][cin] * dY[p][cout], a GEMM with M = 9 * Cin (tiles of 128 rows),
// N = Cout, K = pixels, both operands MN-major (channels contiguous per
// pixel, as NHWC stores them).  Each CTA accumulates its share of 64-pixel
// row segments in TMEM and adds the result to dW with FP32 atomics.  The
// first padding row of the M range holds the constant 1, so its row of dW is
// the bias gradient (sum over pixels of dY).
//
// Every wait is bounded; a wait that runs out sets err[0] and the kernel
// frees its TMEM and returns.
#include <cuda_bf16.h>

#include "gs_conv.h"
#include "gs_umma.cuh"

namespace gs {
namespace conv {

constexpr int kThreads = 128;
constexpr int kHaloRows = 136;                  // 130 used (pixels x0-1 .. x0+128)
// One 8-channel column of a halo row (kHaloRows pixels of 16 bytes) plus
// padding.  Consecutive threads copy the kG columns of a pixel, then the next
// pixel's; a quarter warp's eight 16-byte copies hit distinct banks when the
// columns are 8 banks apart for kG = 4 (stride = 32 mod 128 bytes) and 16
// banks apart for kG = 2 (64 mod 128).  It is also the MMA descriptors'
// K-direction stride.
__host__ __device__ constexpr int col_bytes(int cin) { return kHaloRows * 16 + (cin / 8 == 2 ? 64 : 32); }
constexpr uint32_t kWaitLimit = 1u << 22;

__host__ __device__ constexpr int wimage_bytes(int cin, int cout) { return 9 * cin * cout * 2; }

constexpr int kSlots = 4;   // halo rows resident: the three a row needs and the one being loaded

constexpr int kHalfPix = 66;   // half-resolution pixels under a 130-pixel halo row

// Dynamic shared memory of the forward kernel: the halo rows, the weight
// image, and (load mode 1) the half-resolution rows staged beside them.
__host__ __device__ constexpr int fwd_smem_bytes(int cin, int cout, int load = 0) {
    return kSlots * (cin / 8) * col_bytes(cin) + wimage_bytes(cin, cout) + (load ? kSlots * kHalfPix * cin * 2 : 0);
}

// 16-byte asynchronous global -> shared copy (zero-filled when src_bytes is 0).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_but_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Byte offset of weight (k = tap * cin + ci, n = co) in the K-major B image.
__host__ __device__ constexpr int wimage_offset(int k, int n, int cout) {
    return (k >> 3) * (cout * 16) + (n >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint4 bf16x8_add(uint4 a, uint4 b) {
    uint4 r;
    const __nv_bfloat162* pa = reinterpret_cast<const __nv_bfloat162*>(&a);
    const __nv_bfloat162* pb = reinterpret_cast<const __nv_bfloat162*>(&b);
    __nv_bfloat162* pr = reinterpret_cast<__nv_bfloat162*>(&r);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 fa = __bfloat1622float2(pa[i]), fb = __bfloat1622float2(pb[i]);
        pr[i] = __floats2bfloat162_rn(fa.x + fb.x, fa.y + fb.y);
    }
    return r;
}

// 8 channels (16 bytes) of input pixel (n, y, x), zero outside the image.
// kLoad 1: the decoder input, nearest 2x upsampling of `xh` (half
// resolution) plus `x` at full resolution.
template <int kCin, int kLoad>
__device__ __forceinline__ uint4 load_granule(const ConvArgs& a, int n, int y, int x, int g) {
    if (y < 0 || y >= a.h || x < 0 || x >= a.w) return make_uint4(0u, 0u, 0u, 0u);
    const size_t pix = ((size_t)n * a.h + y) * a.w + x;
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.x + pix * kCin) + g);
    if (kLoad == 0) return v;
    const int hh = a.h >> 1, hw = a.w >> 1;
    const size_t hp = ((size_t)n * hh + min(y >> 1, hh - 1)) * hw + min(x >> 1, hw - 1);
    return bf16x8_add(v, __ldg(reinterpret_cast<const uint4*>(a.xh + hp * kCin) + g));
}

template <int kCin, int kCout, int kLoad>
__global__ void __launch_bounds__(kThreads) conv_fwd_kernel(ConvArgs a) {
    static_assert(kCin % 16 == 0 && (kCout == 16 || kCout == 32), "channel counts");
    constexpr int kG = kCin / 8;                         // 16-byte columns per pixel
    constexpr int kColBytes = col_bytes(kCin);
    constexpr int kSlot = kG * kColBytes;                // one halo row
    constexpr int kW = wimage_bytes(kCin, kCout);
    constexpr uint32_t kIdesc = umma::idesc_bf16(128, kCout, 0, 0);
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* s_halo = smem;                              // kSlots rows: row yy in slot (yy + 4) & 3
    uint8_t* s_w = smem + kSlots * kSlot;
    constexpr int kHalfSlot = kHalfPix * kG * 16;
    uint8_t* s_hstage = s_w + kW;                        // load mode 1: kSlots half rows
    __shared__ __align__(8) uint64_t s_bar[2];   // MMA completion, one per accumulator
    __shared__ uint32_t s_taddr;
    __shared__ float s_bias[kCout];
    constexpr bool kPool = kCin == 16 && kCout == 32;   // the pooled output (conv1 of the denoiser)
    __shared__ __align__(16) uint4 s_pool[kPool ? kThreads * 4 : 1];   // an even row's bf16 outputs

    const int strips_x = (a.w + 127) / 128;
    const int segs = (a.h + a.row_offset + a.rows_per_cta - 1) / a.rows_per_cta;
    const int item = blockIdx.x;
    if (item >= a.n * strips_x * segs) return;
    const int seg = item % segs, strip = item / segs;
    const int n = strip / strips_x, x0 = (strip % strips_x) * 128;
    const int y0 = max(0, seg * a.rows_per_cta - a.row_offset);
    const int y1 = min(a.h, seg * a.rows_per_cta - a.row_offset + a.rows_per_cta);
    const int tid = threadIdx.x, warp = tid >> 5;

    // weights: the packed image, copied verbatim; the bias
    for (int i = tid; i < kW / 16; i += kThreads)
        reinterpret_cast<uint4*>(s_w)[i] = __ldg(reinterpret_cast<const uint4*>(a.wimage) + i);
    if (tid < kCout) s_bias[tid] = a.bias ? __ldg(a.bias + tid) : 0.0f;
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
    }
    if (warp == 0) umma::tmem_alloc(&s_taddr, 64);   // two accumulators of 32 columns

    // Rows come in by cp.async, one row ahead of the MMAs (the copy of row
    // y + 2 is in flight while row y is multiplied).  Load mode 1 also copies
    // the half-resolution row under the halo into a staging buffer, and a
    // pass over the landed row adds it in (FP32 sum rounded to bf16).
    auto slot_of = [&](int yy) { return s_halo + ((yy + 4) & 3) * kSlot; };
    auto hstage_of = [&](int yy) { return s_hstage + ((yy + 4) & 3) * kHalfSlot; };
    auto issue_row = [&](int yy) {
        uint8_t* slot = slot_of(yy);
        const bool row_in = yy >= 0 && yy < a.h;
        const __nv_bfloat16* rowp = a.x + ((size_t)n * a.h + (row_in ? yy : 0)) * a.w * kCin;
        for (int q = tid; q < 130 * kG; q += kThreads) {
            const int hp = q / kG, g = q - hp * kG;
            const int x = x0 - 1 + hp;
            const bool in = row_in && x >= 0 && x < a.w;
            cp_async16(slot + g * kColBytes + hp * 16, in ? rowp + (size_t)x * kCin + g * 8 : a.x, in ? 16u : 0u);
        }
        if (kLoad == 1) {
            const int hh = a.h >> 1, hw = a.w >> 1, hx0 = (x0 - 1) >> 1;
            uint8_t* hs = hstage_of(yy);
            const __nv_bfloat16* hrow = a.xh + ((size_t)n * hh + (row_in ? min(yy >> 1, hh - 1) : 0)) * hw * kCin;
            for (int q = tid; q < kHalfPix * kG; q += kThreads) {
                const int hp = q / kG, g = q - hp * kG;
                // clamped like the row: an odd width's last pixel takes the last half pixel
                const int hx = min(max(hx0 + hp, 0), hw - 1);
                cp_async16(hs + q * 16, row_in ? hrow + (size_t)hx * kCin + g * 8 : a.xh, row_in ? 16u : 0u);
            }
        }
        cp_async_commit();
    };
    // load mode 1: row yy's landed halo += its upsampled half-resolution row
    auto combine_row = [&](int yy) {
        if (yy < 0 || yy >= a.h) return;
        uint8_t* slot = slot_of(yy);
        const uint8_t* hs = hstage_of(yy);
        const int hx0 = (x0 - 1) >> 1;
        for (int q = tid; q < 130 * kG; q += kThreads) {
            const int hp = q / kG, g = q - hp * kG;
            const int x = x0 - 1 + hp;
            if (x < 0 || x >= a.w) continue;
            uint4* dst = reinterpret_cast<uint4*>(slot + g * kColBytes + hp * 16);
            *dst = bf16x8_add(*dst, *reinterpret_cast<const uint4*>(hs + (((x >> 1) - hx0) * kG + g) * 16));
        }
    };
    issue_row(y0 - 1);
    issue_row(y0);
    issue_row(y0 + 1);
    if (kLoad == 1) {
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // rows y0 - 1 and y0
        __syncthreads();
        combine_row(y0 - 1);
        combine_row(y0);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = s_taddr;
    const uint32_t halo_base = smem_u32(s_halo), w_base = smem_u32(s_w);
    uint32_t phase0 = 0, phase1 = 0;
    bool failed = false;
    float err_sum = 0.0f, err_cnt = 0.0f;   // head mode: this thread's column of the band, in row order
    // Two TMEM accumulators: the MMAs of row y (accumulator y & 1) run while
    // the epilogue of row y - 1 reads the other one.
    auto wait_mma = [&](int y) {   // row y's MMAs are done (every thread waits)
        if (!mbar_wait_bounded(&s_bar[y & 1], (y & 1) ? phase1 : phase0, kWaitLimit)) failed = true;
        if (y & 1) phase1 ^= 1u; else phase0 ^= 1u;
    };
    auto mma_row = [&](int y) {
        if (tid == 0) {
            umma::fence_after_sync();
            const uint32_t acc_addr = taddr + (uint32_t)((y & 1) * 32);
            uint32_t acc = 0;
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                const uint32_t slot = halo_base + (uint32_t)(((y - 1 + ky + 4) & 3) * kSlot);
#pragma unroll
                for (int kx = 0; kx < 3; ++kx) {
#pragma unroll
                    for (int kb = 0; kb < kCin / 16; ++kb) {
                        const uint64_t ad = umma::smem_desc(slot + (uint32_t)(2 * kb * kColBytes + kx * 16),
                                                            (uint32_t)kColBytes, 128u);
                        const int k0 = (ky * 3 + kx) * kCin + kb * 16;
                        const uint64_t bd =
                            umma::smem_desc(w_base + (uint32_t)((k0 >> 3) * kCout * 16), (uint32_t)(kCout * 16), 128u);
                        umma::mma_bf16(acc_addr, ad, bd, kIdesc, acc);
                        acc = 1;
                    }
                }
            }
            umma::commit(&s_bar[y & 1]);
        }
    };
    auto epilogue = [&](int y) {   // row y's MMAs waited for
        umma::fence_after_sync();
        const uint32_t acc_addr = taddr + (uint32_t)((y & 1) * 32) + ((uint32_t)(warp * 32) << 16);
        const int x = x0 + tid;
        const size_t o = ((size_t)n * a.h + y) * a.w + x;
        float v[32];
        if (kCout == 32) {
            umma::tmem_ld32(acc_addr, *reinterpret_cast<float(*)[32]>(v));
        } else {
            umma::tmem_ld16(acc_addr, *reinterpret_cast<float(*)[16]>(v));
        }
        if (x < a.w && !failed) {
            if (a.bias) {
#pragma unroll
                for (int c = 0; c < kCout; ++c) v[c] += s_bias[c];
            }
            if (a.relu) {
#pragma unroll
                for (int c = 0; c < kCout; ++c) v[c] = fmaxf(v[c], 0.0f);
            }
            if (a.mask) {
                const uint4* mp = reinterpret_cast<const uint4*>(a.mask + o * kCout);
#pragma unroll
                for (int q = 0; q < kCout / 8; ++q) {
                    const uint4 mv = __ldg(mp + q);
                    const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        if (!(__bfloat162float(mb[e]) > 0.0f)) v[q * 8 + e] = 0.0f;
                }
            }
            if (kCout == 16 && a.head_x) {
                // the denoised frame's pixel (head_rgba of the output step) and its error estimate
                const uint4 xv = __ldg(reinterpret_cast<const uint4*>(a.head_x + o * 16));
                const __nv_bfloat16* xb = reinterpret_cast<const __nv_bfloat16*>(&xv);
                const float4 px = make_float4(__bfloat162float(xb[5]) + v[0], __bfloat162float(xb[6]) + v[1],
                                              __bfloat162float(xb[7]) + v[2], __bfloat162float(xb[3]) + v[3]);
                __half2 h01 = __floats2half2_rn(px.x, px.y), h23 = __floats2half2_rn(px.z, px.w);
                uint2 pk;
                pk.x = *reinterpret_cast<uint32_t*>(&h01);
                pk.y = *reinterpret_cast<uint32_t*>(&h23);
                reinterpret_cast<uint2*>(a.head_out16)[o] = pk;
                err_sum += fmaxf(v[4], 0.0f);
                err_cnt += 1.0f;
            }
            if (a.out_bf16) {
                uint4* op = reinterpret_cast<uint4*>(a.out_bf16 + o * kCout);
#pragma unroll
                for (int q = 0; q < kCout / 8; ++q) {
                    uint4 pk;
                    __nv_bfloat162* pb = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
                    for (int e = 0; e < 4; ++e) pb[e] = __floats2bfloat162_rn(v[q * 8 + 2 * e], v[q * 8 + 2 * e + 1]);
                    op[q] = pk;
                }
            }
            if (a.out_f32) {
                float4* op = reinterpret_cast<float4*>(a.out_f32 + o * kCout);
#pragma unroll
                for (int q = 0; q < kCout / 4; ++q)
                    op[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
        if (kPool && a.pool_out) {
            // 2x2 average of the bf16 outputs: (0 + (y, x) + (y, x + 1) + (y + 1, x) + (y + 1, x + 1)) * 0.25,
            // the even row parked in shared memory, the right neighbour's by a lane shuffle
            uint32_t pk[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
                pk[e] = *reinterpret_cast<uint32_t*>(&b2);
            }
            if ((y & 1) == 0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) s_pool[tid * 4 + q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
            } else {
                uint32_t nb[16];
#pragma unroll
                for (int e = 0; e < 16; ++e) nb[e] = __shfl_xor_sync(0xffffffffu, pk[e], 1);
                if ((x & 1) == 0 && x < a.w && !failed) {
                    const uint32_t* up = reinterpret_cast<const uint32_t*>(&s_pool[tid * 4]);
                    const uint32_t* un = reinterpret_cast<const uint32_t*>(&s_pool[(tid + 1) * 4]);
                    uint32_t res[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const uint32_t t4[4] = {up[e], un[e], pk[e], nb[e]};
                        float acc0 = 0.0f, acc1 = 0.0f;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&t4[k]));
                            acc0 += f.x;
                            acc1 += f.y;
                        }
                        __nv_bfloat162 r2 = __floats2bfloat162_rn(0.25f * acc0, 0.25f * acc1);
                        res[e] = *reinterpret_cast<uint32_t*>(&r2);
                    }
                    const int hw2 = a.w >> 1;
                    uint4* dp = reinterpret_cast<uint4*>(a.pool_out + (((size_t)n * (a.h >> 1) + (y >> 1)) * hw2 + (x >> 1)) * kCout);
#pragma unroll
                    for (int q = 0; q < 4; ++q) dp[q] = make_uint4(res[4 * q], res[4 * q + 1], res[4 * q + 2], res[4 * q + 3]);
                }
            }
        }
        umma::fence_before_sync();
    };

    bool broke = false;   // uniform over the CTA (from __syncthreads_or)
    for (int y = y0; y < y1; ++y) {
        if (y > y0) wait_mma(y - 1);    // its MMAs were the last readers of row y - 2's slot
        issue_row(y + 2);               // into that slot
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // rows up to y + 1 have landed
        if (kLoad == 1) {
            __syncthreads();            // every thread's copies of row y + 1 are visible
            combine_row(y + 1);
        }
        umma::fence_smem_to_async();
        if (__syncthreads_or(failed)) {
            failed = broke = true;
            break;
        }
        mma_row(y);
        if (y > y0) epilogue(y - 1);
    }
    if (!broke) {   // the whole CTA: the epilogue's TMEM loads are warp-collective
        wait_mma(y1 - 1);
        if (kPool && a.pool_out) __syncthreads();   // the even row parked by the previous epilogue
        epilogue(y1 - 1);
    }
    if (kCout == 16 && a.head_x && !broke) {
        // per tile (16 threads = 16 columns of the band): the sum of the error estimates and the
        // pixel count, each over 16 lanes in a fixed order, then the tile's mean
#pragma unroll
        for (int off = 8; off; off >>= 1) {
            err_sum += __shfl_xor_sync(0xffffffffu, err_sum, off);
            err_cnt += __shfl_xor_sync(0xffffffffu, err_cnt, off);
        }
        const int tx = (x0 >> 4) + (tid >> 4);
        if ((tid & 15) == 0 && tx < a.tiles_x && err_cnt > 0.0f) {
            const int ty = (a.h + a.row_offset) / 16 - 1 - seg;   // GL tile row of this band
            const uint32_t tile = (uint32_t)(ty * a.tiles_x + tx);
            const float mse = err_sum / err_cnt * 0.001f;
            if (a.tile_err) a.tile_err[tile] = mse;
            if (mse >= a.err_budget) a.fallback_tiles[atomicAdd(a.fallback_count, 1u)] = tile;
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");   // the prefetched rows past the run
    if (failed && tid == 0) atomicOr(a.err, 1u);
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, 64);
}

// ---------------------------------------------------------------------------
// Weight gradient.
// ---------------------------------------------------------------------------
constexpr int kKBlock = 64;                       // pixels per K block
constexpr int kGroupBytes = kKBlock * 16 + 16;    // one 8-channel group of a K block (+16: bank spread)

__host__ __device__ constexpr int wgrad_mtiles(int cin) { return (9 * cin + 1 + 127) / 128; }
__host__ __device__ constexpr int tmem_cols_for(int c) { return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : 256; }

template <int kCin, int kCout, int kLoad>
__global__ void __launch_bounds__(kThreads) conv_wgrad_kernel(WgradArgs a) {
    constexpr int kMT = wgrad_mtiles(kCin);
    constexpr int kA = 16 * kGroupBytes;           // one M tile: 16 groups of 8 rows
    constexpr int kCols = tmem_cols_for(kMT * kCout);
    constexpr uint32_t kIdesc = umma::idesc_bf16(128, kCout, 1, 1);
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* s_a = smem;
    uint8_t* s_b = smem + kMT * kA;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_taddr;
    const int tid = threadIdx.x, warp = tid >> 5;

    if (tid == 0) {
        mbar_init(&s_bar, 1);
        mbar_fence_init();
    }
    if (warp == 0) umma::tmem_alloc(&s_taddr, kCols);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = s_taddr;
    const uint32_t a_base = smem_u32(s_a), b_base = smem_u32(s_b);
    const int blocks_x = (a.w + kKBlock - 1) / kKBlock;
    const int total = a.n * a.h * blocks_x;
    uint32_t phase = 0;
    bool failed = false, any = false;
    const ConvArgs ca{a.x, a.xh, a.n, a.h, a.w};

    for (int blk = blockIdx.x; blk < total && !failed; blk += gridDim.x) {
        const int xb = blk % blocks_x, row = blk / blocks_x;
        const int y = row % a.h, n = row / a.h, x0 = xb * kKBlock;
        // A: rows m = tap * cin + ci (8-row groups never straddle a tap), K = pixels
        for (int q = tid; q < kMT * 16 * kKBlock; q += kThreads) {
            const int k = q % kKBlock, grp = q / kKBlock;      // grp = tile * 16 + group
            const int m0 = grp * 8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m0 < 9 * kCin) {
                const int tap = m0 / kCin, cg = (m0 % kCin) >> 3;
                v = load_granule<kCin, kLoad>(ca, n, y + tap / 3 - 1, x0 + k + tap % 3 - 1, cg);
            } else if (m0 == 9 * kCin && x0 + k < a.w) {
                v.x = 0x3F80u;   // bf16 1.0 in row m0 (the bias row), zero in rows m0+1..m0+7
            }
            *reinterpret_cast<uint4*>(s_a + (grp >> 4) * kA + (grp & 15) * kGroupBytes + k * 16) = v;
        }
        // B: dY, rows = output channels, K = pixels
        for (int q = tid; q < (kCout / 8) * kKBlock; q += kThreads) {
            const int k = q % kKBlock, g = q / kKBlock;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (x0 + k < a.w) {
                const size_t pix = ((size_t)n * a.h + y) * a.w + x0 + k;
                v = __ldg(reinterpret_cast<const uint4*>(a.dy + pix * kCout) + g);
            }
            *reinterpret_cast<uint4*>(s_b + g * kGroupBytes + k * 16) = v;
        }
        umma::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after_sync();
#pragma unroll
            for (int t = 0; t < kMT; ++t) {
#pragma unroll
                for (int kk = 0; kk < kKBlock / 16; ++kk) {
                    const uint64_t ad = umma::smem_desc(a_base + (uint32_t)(t * kA + kk * 256), 128u,
                                                        (uint32_t)kGroupBytes);
                    const uint64_t bd = umma::smem_desc(b_base + (uint32_t)(kk * 256), 128u, (uint32_t)kGroupBytes);
                    umma::mma_bf16(taddr + (uint32_t)(t * kCout), ad, bd, kIdesc, (any || kk > 0) ? 1u : 0u);
                }
            }
            umma::commit(&s_bar);
        }
        any = true;
        if (!mbar_wait_bounded(&s_bar, phase, kWaitLimit)) failed = true;
        phase ^= 1u;
        umma::fence_after_sync();
        if (__syncthreads_or(failed)) failed = true;
    }
    if (any && !failed) {
        // warp w holds rows 32w..32w+31 of every M tile
        const int r = warp * 32 + (tid & 31);
#pragma unroll
        for (int t = 0; t < kMT; ++t) {
            float v[32];
            if (kCout == 32)
                umma::tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * kCout),
                                *reinterpret_cast<float(*)[32]>(v));
            else
                umma::tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * kCout),
                                *reinterpret_cast<float(*)[16]>(v));
            const int m = t * 128 + r;
            if (m < 9 * kCin) {
#pragma unroll
                for (int c = 0; c < kCout; ++c) atomicAdd(a.dw + (size_t)m * kCout + c, v[c]);
            } else if (m == 9 * kCin && a.db) {
#pragma unroll
                for (int c = 0; c < kCout; ++c) atomicAdd(a.db + c, v[c]);
            }
        }
    }
    if (failed && tid == 0) atomicOr(a.err, 1u);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, kCols);
}

// ---------------------------------------------------------------------------
// Weight packing: FP32 masters [tap][cin][cout] -> the bf16 B-operand image of
// the forward convolution, or of the transposed convolution that gives the
// input gradient (cin' = cout, cout' = cin, tap' = 8 - tap).
// ---------------------------------------------------------------------------
__global__ void pack_weights_kernel(const float* __restrict__ w, int cin, int cout, int transposed, int cut_cout,
                                    uint8_t* __restrict__ image) {
    const int total = 9 * cin * cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int co = i % cout, ci = (i / cout) % cin, tap = i / (cin * cout);
        // cut_cout: the output channel whose gradient stops at this layer (zero in the transposed image)
        const float v = (transposed && co == cut_cout) ? 0.0f : w[i];
        int k, nn, cdim;
        if (!transposed) {
            k = tap * cin + ci;
            nn = co;
            cdim = cout;
        } else {
            k = (8 - tap) * cout + co;
            nn = ci;
            cdim = cin;
        }
        *reinterpret_cast<__nv_bfloat16*>(image + wimage_offset(k, nn, cdim)) = __float2bfloat16_rn(v);
    }
}

template <int kCin, int kCout, int kLoad>
static int launch_fwd_t(const ConvArgs& a, cudaStream_t s) {
    const int strips = a.n * ((a.w + 127) / 128);
    const int segs = (a.h + a.row_offset + a.rows_per_cta - 1) / a.rows_per_cta;
    const size_t smem = (size_t)fwd_smem_bytes(kCin, kCout, kLoad);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(conv_fwd_kernel<kCin, kCout, kLoad>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        attr = true;
    }
    conv_fwd_kernel<kCin, kCout, kLoad><<<strips * segs, kThreads, smem, s>>>(a);
    return 1;
}

template <int kCin, int kCout, int kLoad>
static int launch_wgrad_t(const WgradArgs& a, int grid, cudaStream_t s) {
    // + 2 groups: every address a descriptor can name, with either stride
    // reading as either, stays inside the allocation
    const size_t smem = (size_t)wgrad_mtiles(kCin) * 16 * kGroupBytes + (size_t)(kCout / 8 + 2) * kGroupBytes;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(conv_wgrad_kernel<kCin, kCout, kLoad>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        attr = true;
    }
    conv_wgrad_kernel<kCin, kCout, kLoad><<<grid, kThreads, smem, s>>>(a);
    return 1;
}

int launch_fwd(int cin, int cout, int load_mode, const ConvArgs& a, cudaStream_t s) {
    if (a.n <= 0 || a.h <= 0 || a.w <= 0) return 0;
    if (load_mode == 0) {
        if (cin == 16 && cout == 32) return launch_fwd_t<16, 32, 0>(a, s);
        if (cin == 32 && cout == 32) return launch_fwd_t<32, 32, 0>(a, s);
        if (cin == 32 && cout == 16) return launch_fwd_t<32, 16, 0>(a, s);
    } else {
        if (cin == 32 && cout == 32) return launch_fwd_t<32, 32, 1>(a, s);
    }
    return -1;
}

int launch_wgrad(int cin, int cout, int load_mode, const WgradArgs& a, int grid, cudaStream_t s) {
    if (a.n <= 0 || a.h <= 0 || a.w <= 0) return 0;
    if (load_mode == 0) {
        if (cin == 16 && cout == 32) return launch_wgrad_t<16, 32, 0>(a, grid, s);
        if (cin == 32 && cout == 32) return launch_wgrad_t<32, 32, 0>(a, grid, s);
        if (cin == 32 && cout == 16) return launch_wgrad_t<32, 16, 0>(a, grid, s);
    } else {
        if (cin == 32 && cout == 32) return launch_wgrad_t<32, 32, 1>(a, grid, s);
    }
    return -1;
}

int launch_pack_weights(const float* w, int cin, int cout, int transposed, uint8_t* image, cudaStream_t s,
                        int cut_cout) {
    const int total = 9 * cin * cout;
    pack_weights_kernel<<<(total + 255) / 256, 256, 0, s>>>(w, cin, cout, transposed, cut_cout, image);
    return 1;
}

size_t weight_image_bytes(int cin, int cout) { return (size_t)wimage_bytes(cin, cout); }

}  // namespace conv
}  // namespace gs
