// One-sweep LSD radix sort of 64-bit Morton codes with 32-bit slot indices.
//
// Replaces the reference's recursiveParallelMortonSort / mortonSort
// (src/NBody/Simulation/Solvers/MortonSort.h:75-88, 141-183: MSB partition then boost spreadsort).
// The reference leaves the order of equal codes unspecified; this sort is stable, so equal codes
// keep their input order (input index order on a fresh set of bodies).
//
// Design (one-sweep, decoupled look-back):
//   - the Morton kernel already counted all eight 8-bit digit histograms;
//   - scan_hist turns them into global digit offsets and flags passes whose digit is constant;
//   - each of the 8 passes is ONE kernel: a block takes the next tile (atomic ticket), ranks its
//     2048 keys by digit with warp-level match (stable), publishes its per-digit counts, looks
//     back over earlier tiles' published counts for its global digit offsets, stages the tile
//     in shared memory in digit order and writes it out in runs of equal digits.
// Per pass each key is read once and written once: 12 B read + 12 B written per body.
// Every look-back wait is bounded by a 2 s timer; on expiry the kernel sets an error bit that the
// host reports, and carries on without hanging the device.
#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kSortTileKeys;
static_assert(kThreads * kItems == kTile, "one tile is kItems keys per thread");
constexpr int kWarps = kThreads / 32;
constexpr int kPasses = kSortPasses;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t load_volatile(const uint32_t *p) { return *(const volatile uint32_t *) p; }
__device__ __forceinline__ void store_volatile(uint32_t *p, uint32_t v) { *(volatile uint32_t *) p = v; }

// Exclusive prefix of each 256-bin digit histogram; offsets[8*256 + p] = 1 if pass p is trivial
// (every key has the same digit), in which case the pass is a plain copy.
__global__ void __launch_bounds__(256) scan_hist_kernel(const uint32_t *__restrict__ hist, uint32_t *__restrict__ offsets,
                                                        int64_t n) {
    __shared__ uint32_t warp_tot[8];
    __shared__ int trivial;
    const int p = blockIdx.x, d = threadIdx.x, lane = d & 31, warp = d >> 5;
    if (d == 0) trivial = 0;
    uint32_t v = hist[p * 256 + d];
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    offsets[p * 256 + d] = before + incl - v;
    if ((int64_t) v == n) trivial = 1;
    __syncthreads();
    if (d == 0) offsets[kPasses * 256 + p] = (uint32_t) trivial;
}

__global__ void __launch_bounds__(kThreads) onesweep_kernel(const uint64_t *__restrict__ keys_in,
                                                            const uint32_t *__restrict__ vals_in,
                                                            uint64_t *__restrict__ keys_out,
                                                            uint32_t *__restrict__ vals_out, int64_t n, int pass,
                                                            const uint32_t *__restrict__ offsets,
                                                            uint32_t *__restrict__ lookback,
                                                            uint32_t *__restrict__ tile_counter,
                                                            uint32_t *__restrict__ err,
                                                            unsigned long long wait_limit_ns) {
    __shared__ uint64_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];
    __shared__ uint32_t s_whist[kWarps][256];
    __shared__ uint32_t s_start[256];
    __shared__ int32_t s_base[256];
    __shared__ uint32_t s_warp_tot[kWarps];
    __shared__ uint32_t s_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int num_tiles = gridDim.x;
    const bool first = (pass == 0);
    const int shift = 8 * pass;

    if (tid == 0) s_tile = atomicAdd(&tile_counter[pass], 1u);
    for (int i = tid; i < kWarps * 256; i += kThreads) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t base = tile * kTile;

    if (offsets[kPasses * 256 + pass]) {
        // Every key has the same digit in this pass: the stable result is the input order.
        for (int i = tid; i < kTile; i += kThreads) {
            int64_t idx = base + i;
            if (idx < n) {
                keys_out[idx] = keys_in[idx];
                vals_out[idx] = first ? (uint32_t) idx : vals_in[idx];
            }
        }
        return;
    }

    // Warp-striped load: item it of lane l in warp w is key base + w*256 + it*32 + l, so that
    // ranking items in (it, lane) order within a warp and warps in order keeps the sort stable.
    uint64_t k[kItems];
    uint32_t v[kItems], rank[kItems], dig[kItems];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        int64_t idx = base + warp * 32 * kItems + it * 32 + lane;
        bool valid = idx < n;
        k[it] = valid ? keys_in[idx] : ~0ull;
        v[it] = valid ? (first ? (uint32_t) idx : vals_in[idx]) : 0u;
        dig[it] = valid ? (uint32_t) ((k[it] >> shift) & 255u) : 256u;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const uint32_t d = dig[it];
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const int leader = 31 - __clz(peers);
        uint32_t before = 0;
        if (lane == leader && d < 256u) {
            before = s_whist[warp][d];
            s_whist[warp][d] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        rank[it] = before + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();

    // Per digit: exclusive prefix over warps, tile count.
    const int d = tid;
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        uint32_t c = s_whist[w][d];
        s_whist[w][d] = count;
        count += c;
    }
    uint32_t *my_lb = lookback + ((int64_t) pass * num_tiles + tile) * 256;
    const uint32_t global_off = offsets[pass * 256 + d];
    if (tile == 0) store_volatile(&my_lb[d], kFlagInc | (global_off + count));
    else store_volatile(&my_lb[d], kFlagAgg | count);

    // Exclusive scan of the tile's digit counts -> where each digit starts within the tile.
    uint32_t incl = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp_tot[warp] = incl;
    __syncthreads();
    uint32_t wbefore = 0;
    for (int w = 0; w < warp; ++w) wbefore += s_warp_tot[w];
    const uint32_t start = wbefore + incl - count;
    s_start[d] = start;

    // Decoupled look-back for this digit.
    uint32_t excl;
    if (tile == 0) {
        excl = global_off;
    } else {
        excl = 0;
        int64_t t = tile - 1;
        const unsigned long long t0 = global_timer_ns();
        while (true) {
            uint32_t w = load_volatile(lookback + ((int64_t) pass * num_tiles + t) * 256 + d);
            uint32_t f = w & kFlagMask;
            if (f == 0u) {
                if (global_timer_ns() - t0 > wait_limit_ns) {
                    atomicOr(err, (uint32_t) kErrLookbackTimeout);
                    break;
                }
                continue;
            }
            excl += w & kValueMask;
            if (f == kFlagInc) break;
            --t;
        }
        store_volatile(&my_lb[d], kFlagInc | ((excl + count) & kValueMask));
    }
    s_base[d] = (int32_t) excl - (int32_t) start;
    __syncthreads();

    // Stage the tile in digit order.
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const uint32_t dd = dig[it];
        if (dd < 256u) {
            const uint32_t pos = s_start[dd] + s_whist[warp][dd] + rank[it];
            s_keys[pos] = k[it];
            s_vals[pos] = v[it];
        }
    }
    __syncthreads();

    const int tile_n = (int) ((n - base) < kTile ? (n - base) : kTile);
    for (int i = tid; i < tile_n; i += kThreads) {
        const uint64_t key = s_keys[i];
        const uint32_t dd = (uint32_t) ((key >> shift) & 255u);
        const int64_t o = (int64_t) s_base[dd] + i;
        keys_out[o] = key;
        vals_out[o] = s_vals[i];
    }
}

}  // namespace

int64_t sort_tiles(int64_t n) { return (n + kTile - 1) / kTile; }

size_t sort_lookback_words(int64_t n) { return (size_t) kPasses * (size_t) (sort_tiles(n) > 0 ? sort_tiles(n) : 1) * 256; }

void launch_radix_pass(const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out, uint32_t *vals_out,
                       int64_t n, int pass, const uint32_t *offsets, uint32_t *lookback, uint32_t *tile_counter,
                       uint32_t *err, cudaStream_t s) {
    if (n <= 0) return;
    onesweep_kernel<<<(unsigned) sort_tiles(n), kThreads, 0, s>>>(keys_in, vals_in, keys_out, vals_out, n, pass,
                                                                   offsets, lookback, tile_counter, err, kWaitLimitNs);
}

cudaError_t launch_radix_sort(uint64_t *keys, uint32_t *vals, int64_t n, SortWorkspace &ws, uint32_t *err,
                              cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int64_t tiles = sort_tiles(n);
    cudaError_t e = cudaMemsetAsync(ws.lookback, 0, sort_lookback_words(n) * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(ws.tile_counter, 0, kPasses * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    scan_hist_kernel<<<kPasses, 256, 0, s>>>(ws.hist, ws.offsets, n);
    if ((e = cudaPeekAtLastError()) != cudaSuccess) return e;
    uint64_t *kin = keys, *kout = ws.keys_alt;
    uint32_t *vin = vals, *vout = ws.vals_alt;
    for (int p = 0; p < kPasses; ++p) {
        onesweep_kernel<<<(unsigned) tiles, kThreads, 0, s>>>(kin, vin, kout, vout, n, p, ws.offsets, ws.lookback,
                                                               ws.tile_counter, err, kWaitLimitNs);
        if ((e = cudaPeekAtLastError()) != cudaSuccess) return e;
        uint64_t *tk = kin; kin = kout; kout = tk;
        uint32_t *tv = vin; vin = vout; vout = tv;
    }
    // An even number of passes leaves the result in (keys, vals).
    static_assert(kPasses % 2 == 0, "the sorted data must end in the caller's buffers");
    return cudaSuccess;
}

}  // namespace nbg

namespace nbg {

// One pass whose look-back can never complete, to check that the bounded wait ends: a single block
// is launched with its tile ticket preset to 1, so it takes tile 1 of a two-tile input and waits on
// tile 0's flags, which nothing ever publishes. Every index stays in bounds: keys and values hold
// two tiles, the look-back buffer two tiles of 256 flags (the kernel indexes it with gridDim = 1),
// and the tile's scatter writes within the first tile's positions. Returns the error word.
cudaError_t lookback_timeout_selftest(unsigned long long wait_limit_ns, uint32_t *err_word) {
    const int64_t n = 2 * kTile;
    uint64_t *keys = nullptr, *keys_out = nullptr;
    uint32_t *vals = nullptr, *vals_out = nullptr, *offsets = nullptr, *lookback = nullptr, *ticket = nullptr,
             *err = nullptr;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    alloc((void **) &keys, n * sizeof(uint64_t));
    alloc((void **) &keys_out, n * sizeof(uint64_t));
    alloc((void **) &vals, n * sizeof(uint32_t));
    alloc((void **) &vals_out, n * sizeof(uint32_t));
    alloc((void **) &offsets, (kPasses * 256 + kPasses) * sizeof(uint32_t));  // no pass is trivial
    alloc((void **) &lookback, 2 * 256 * sizeof(uint32_t));
    alloc((void **) &ticket, kPasses * sizeof(uint32_t));
    alloc((void **) &err, sizeof(uint32_t));
    if (e == cudaSuccess) {
        const uint32_t one = 1;
        e = cudaMemcpy(ticket, &one, sizeof(one), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        onesweep_kernel<<<1, kThreads>>>(keys, vals, keys_out, vals_out, n, 0, offsets, lookback, ticket, err,
                                         wait_limit_ns);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(err_word, err, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    for (void *p: {(void *) keys, (void *) keys_out, (void *) vals, (void *) vals_out, (void *) offsets,
                   (void *) lookback, (void *) ticket, (void *) err})
        if (p) cudaFree(p);
    return e;
}

}  // namespace nbg
