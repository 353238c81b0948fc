// Allocation-free variant of the tile-count prefix scan (r2s_scan_tile_counts).
//
// The scan's scratch (the per-block totals of each recursion level) lives in a
// file-scope __device__ array instead of a caller workspace, so a call needs no
// device allocation from anyone: not from this library, the caller, or torch.
// The array holds the scratch for up to kNoAllocScanMaxElems elements; larger
// inputs are rejected with R2S_ERR_UNSUPPORTED before anything is launched.
//
// Nothing in the scratch has to start at zero: every block total is written by
// scan_reduce_kernel before the next kernel on the same stream reads it.
//
// The array is one per device and is shared by all calls on that device, so
// calls that overlap in time (on different streams or host threads) race on it
// and must be serialised by the caller. The first call on a device resolves the
// array's address with cudaGetSymbolAddress (which may load the module); make
// that first call before any stream capture on the device. The address is
// cached per device ordinal for the life of the process: after a
// cudaDeviceReset (or any other teardown of the device's primary context) the
// cached address would be stale, so this entry point does not support a reset
// of a device it has already been called on.
#include <mutex>

#include "scan.cuh"

namespace r2s {

constexpr int64_t kNoAllocScanMaxElems = int64_t(1) << 25;  // 33,554,432 tile counts
constexpr size_t kNoAllocScanScratchBytes = 72 * 1024;
static_assert(scan_workspace_bytes<int64_t>(kNoAllocScanMaxElems) <= kNoAllocScanScratchBytes,
              "no-alloc scan scratch too small for its stated maximum");

static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[kNoAllocScanScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Resolves (once per device) the device address of g_noalloc_scan_scratch.
int noalloc_scratch(void** out) {
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return fail(R2S_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
    R2S_REQUIRE(device >= 0 && device < kMaxDevices, R2S_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_ptr[device] == nullptr) {
        void* ptr = nullptr;
        err = cudaGetSymbolAddress(&ptr, g_noalloc_scan_scratch);
        if (err != cudaSuccess || ptr == nullptr) {
            return fail(R2S_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scan scratch): ") +
                                          cudaGetErrorString(err));
        }
        g_scratch_ptr[device] = ptr;
    }
    *out = g_scratch_ptr[device];
    return R2S_OK;
}

}  // namespace
}  // namespace r2s

using namespace r2s;

extern "C" {

uint64_t r2s_scan_tile_counts_noalloc_max(void) { return uint64_t(kNoAllocScanMaxElems); }

int r2s_scan_tile_counts_noalloc(const int32_t* counts, uint64_t n, int64_t* cum, void* stream) {
    if (n > uint64_t(kNoAllocScanMaxElems)) {
        return fail(R2S_ERR_UNSUPPORTED, "scan_tile_counts_noalloc: n = " + std::to_string(n) +
                                             " exceeds the static scratch limit of " +
                                             std::to_string(kNoAllocScanMaxElems) + " elements");
    }
    if (n == 0) return R2S_OK;
    R2S_REQUIRE(counts != nullptr && cum != nullptr, R2S_ERR_ARGUMENT, "counts and cum must be non-null");
    void* scratch = nullptr;
    R2S_TRY(noalloc_scratch(&scratch));
    return device_scan<int32_t, int64_t, true>(counts, cum, int64_t(n), scratch, kNoAllocScanScratchBytes,
                                               as_stream(stream));
}

}  // extern "C"
