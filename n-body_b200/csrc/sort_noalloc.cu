// Morton-code sort that allocates nothing: nb_sort_codes_noalloc (include/nbody_gpu.h).
//
// Some callers cannot allocate device memory when they sort: applications that hand every byte
// of device memory to their own pool allocator and forbid other allocations, and step loops that
// cannot afford cudaMalloc / cudaFree, which may synchronise the whole device. For them this
// entry point runs the same one-sweep radix sort as the force path, with its scratch memory
// (ping-pong key/index buffers, digit histograms, look-back flags) in one file-scope device array.
//
// Properties a caller must know:
//   - capacity: at most kNoAllocMaxKeys (2^20) codes per call; larger inputs are rejected with
//     NB_ERR_INVALID_ARGUMENT before any work is queued;
//   - the array holds kNoAllocScratchBytes (about 16 MiB) on every GPU that loads this library,
//     from the first use of the library on that GPU until the process exits;
//   - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current; make that first call before any stream capture;
//   - each call returns only once the sort has finished: it copies a status word to the host and
//     synchronises the stream (pageable copy + cudaStreamSynchronize);
//   - every call shares the one array and it keeps the previous call's contents: each call clears
//     what must start at zero, but two calls that overlap on the GPU (different streams, or
//     different host threads) race on the scratch and corrupt each other's results.
#include <algorithm>
#include <mutex>

#include "../../include/nbody_gpu.h"
#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int64_t kNoAllocMaxKeys = int64_t(1) << 20;
constexpr int64_t kMaxTiles = (kNoAllocMaxKeys + kSortTileKeys - 1) / kSortTileKeys;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffKeys = 0;
constexpr size_t kOffVals = align256(kOffKeys + sizeof(uint64_t) * kNoAllocMaxKeys);
constexpr size_t kOffHist = align256(kOffVals + sizeof(uint32_t) * kNoAllocMaxKeys);
constexpr size_t kOffOffsets = align256(kOffHist + sizeof(uint32_t) * kSortPasses * 256);
constexpr size_t kOffLookback = align256(kOffOffsets + sizeof(uint32_t) * (kSortPasses * 256 + kSortPasses));
constexpr size_t kLookbackWords = (size_t) kSortPasses * kMaxTiles * 256;
constexpr size_t kOffTiles = align256(kOffLookback + sizeof(uint32_t) * kLookbackWords);
constexpr size_t kOffErr = align256(kOffTiles + sizeof(uint32_t) * kSortPasses);
constexpr size_t kNoAllocScratchBytes = align256(kOffErr + sizeof(uint32_t));
// The sort's launcher clears sort_lookback_words(n) look-back words: at the largest n accepted they
// must fit before the tile tickets.
static_assert(kOffLookback + sizeof(uint32_t) * kLookbackWords <= kOffTiles, "look-back region overlaps");

static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// The symbol's device address for the current device, looked up once per device.
cudaError_t scratch_for(int device, unsigned char **out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = (unsigned char *) p;
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

// The eight 8-bit digit histograms of 64-bit keys (what the Morton kernel produces on the way).
__global__ void __launch_bounds__(256) digit_hist_kernel(const uint64_t *__restrict__ keys, int64_t n,
                                                         uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
#pragma unroll
        for (int d = 0; d < 8; ++d) atomicAdd(&sh[d * 256 + (uint32_t) ((k >> (8 * d)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
        const uint32_t c = sh[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

}  // namespace

}  // namespace nbg

using namespace nbg;

extern "C" int nb_sort_codes_noalloc(const uint64_t *d_codes, uint64_t *d_sorted_codes, uint32_t *d_sorted_ids,
                                     int64_t n, void *cuda_stream) {
    if (n < 0 || n > kNoAllocMaxKeys) return NB_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!d_codes || !d_sorted_codes || !d_sorted_ids)) return NB_ERR_INVALID_ARGUMENT;
    if (n == 0) return NB_OK;
    if (sort_lookback_words(n) > kLookbackWords) return NB_ERR_INVALID_ARGUMENT;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return NB_ERR_CUDA;
    unsigned char *base = nullptr;
    if (scratch_for(device, &base) != cudaSuccess) return NB_ERR_CUDA;
    cudaStream_t s = (cudaStream_t) cuda_stream;

    SortWorkspace ws;
    ws.keys_alt = (uint64_t *) (base + kOffKeys);
    ws.vals_alt = (uint32_t *) (base + kOffVals);
    ws.hist = (uint32_t *) (base + kOffHist);
    ws.offsets = (uint32_t *) (base + kOffOffsets);
    ws.lookback = (uint32_t *) (base + kOffLookback);
    ws.tile_counter = (uint32_t *) (base + kOffTiles);
    ws.capacity = kNoAllocMaxKeys;
    uint32_t *err = (uint32_t *) (base + kOffErr);

    // The scratch keeps the previous call's contents: clear what must start at zero.
    if (cudaMemsetAsync(ws.hist, 0, sizeof(uint32_t) * kSortPasses * 256, s) != cudaSuccess) return NB_ERR_CUDA;
    if (cudaMemsetAsync(err, 0, sizeof(uint32_t), s) != cudaSuccess) return NB_ERR_CUDA;
    if (cudaMemcpyAsync(d_sorted_codes, d_codes, (size_t) n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess)
        return NB_ERR_CUDA;
    const int64_t blocks = std::min<int64_t>((n + 256 * 8 - 1) / (256 * 8), (int64_t) current_sm_count() * 4);
    digit_hist_kernel<<<(unsigned) std::max<int64_t>(blocks, 1), 256, 0, s>>>(d_codes, n, ws.hist);
    if (cudaPeekAtLastError() != cudaSuccess) return NB_ERR_CUDA;
    // Sorts in place in (d_sorted_codes, d_sorted_ids) with the scratch as the other buffer; the
    // launcher clears the look-back flags and tile tickets itself.
    if (launch_radix_sort(d_sorted_codes, d_sorted_ids, n, ws, err, s) != cudaSuccess) return NB_ERR_CUDA;
    uint32_t e = 0;
    if (cudaMemcpyAsync(&e, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess) return NB_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return NB_ERR_CUDA;
    return (e & kErrLookbackTimeout) ? NB_ERR_DEVICE_TIMEOUT : NB_OK;
}
