// gs_sort_pairs_noalloc: the stable radix sort of gs_sort_pairs for callers
// that cannot allocate device memory through this library.
//
// Who cannot allocate: a real-time render loop that must not stall, where
// cudaMalloc / cudaFree would synchronise the whole device in the middle of a
// frame; and host engines whose memory manager owns and budgets every device
// allocation up front and forbids libraries from allocating behind its back.
// Such callers still pass their own input and output buffers; only the sort's
// scratch comes from here.
//
// The scratch is one file-scope __device__ array of kNoAllocScratchBytes
// (about 10 MiB, enough for kNoAllocMaxPairs = 2^20 pairs).  Every GPU that
// loads this library holds it until the process exits.  Larger sorts are
// rejected with GS_ERR_TOO_LARGE.
//
// In host code `g_sort_scratch` is only a host-side stand-in for the array,
// not a device address: handing it to a kernel would fault (or, where the GPU
// can reach host memory, silently use the wrong memory).  The device address
// is looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on that device; that first call should
// therefore come before any stream capture.  The address is kept together
// with the id of the CUDA context it belongs to: if the device's primary
// context has been reset since (cudaDeviceReset), the module and its array
// were loaded anew in a new context, so the next call looks the address up
// again instead of using a stale one.
//
// All calls share the one array and it keeps the previous call's contents:
// each call clears the parts that must start at zero (sort plan, histograms,
// look-back words) on its stream before using them.  Calls that overlap on
// the GPU (different streams or host threads) race on the array and corrupt
// each other's results; callers must serialise them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "gs_internal.h"

namespace {

constexpr uint32_t kNoAllocMaxPairs = 1u << 20;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Same layout as the scratch gs_sort_pairs expects for n pairs.
constexpr size_t kNoAllocStatusWords =
    (((size_t)kNoAllocMaxPairs + gs::kSortTile - 1) / gs::kSortTile) * gs::kRadix;
constexpr size_t kNoAllocScratchBytes = align256(sizeof(gs::SortPlan)) + align256(4 * 256 * 4) + align256(4) +
                                        align256(kNoAllocStatusWords * 4 * sizeof(unsigned long long)) +
                                        2 * align256((size_t)kNoAllocMaxPairs * 4);

static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};   // id of the context each address was looked up in
std::mutex g_setup_mutex;

// Driver entry points reached through the runtime (no link against libcuda).
void* driver_entry(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

// The unique id (cuCtxGetId; never reused within a process) of the context
// current on this thread; 0 if there is none.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = reinterpret_cast<GetCurrent>(driver_entry("cuCtxGetCurrent"));
    static GetId get_id = reinterpret_cast<GetId>(driver_entry("cuCtxGetId"));
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

}  // namespace

extern "C" int gs_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, uint32_t n, int begin_bit, int end_bit, void* stream) {
    if (n > kNoAllocMaxPairs) return GS_ERR_TOO_LARGE;
    if (gs_sort_pairs_scratch_bytes(n) > kNoAllocScratchBytes) return GS_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return GS_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return GS_ERR_BAD_ARG;
    // Make the device's primary context current (cudaSetDevice initialises
    // it), so that the context read below is the one the sort will run in.
    if (cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return GS_ERR_CUDA;
    }
    const unsigned long long ctx = current_context_id();
    if (!ctx) return GS_ERR_CUDA;
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
            void* addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_sort_scratch);
            if (e != cudaSuccess || !addr) {
                cudaGetLastError();
                return GS_ERR_CUDA;
            }
            g_scratch_addr[dev] = addr;
            g_scratch_ctx[dev] = ctx;
        }
        scratch = g_scratch_addr[dev];
    }
    return gs_sort_pairs(keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit, scratch,
                         kNoAllocScratchBytes, stream);
}
