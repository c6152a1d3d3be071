// Global bounding box and 64-bit Morton codes.
//
// Semantics follow the reference exactly (bit-exact codes):
//   outerBoundingBox  src/NBody/Physics/Summaries/SummaryType.h:73-81 (FP32 min/max of positions)
//   setMortonCodes    src/NBody/Simulation/Solvers/MortonSort.h:63-73 (scale = max side length)
//   toMortonCode      MortonSort.h:46-60 (v = (p - min) / scale; clamp(v * 2^21, 0, 2^21 - 1);
//                     truncate; interleave x*4 + y*2 + z with 21 bits per axis)
// Min and max are exact in any order, so the parallel reduction gives the same box. The
// subtraction, division and multiplication are single IEEE round-to-nearest operations
// (__fsub_rn, __fdiv_rn, __fmul_rn), as in the reference's FP32 build without FMA.
//
// The Morton kernel also builds the eight 8-bit digit histograms the one-sweep radix sort needs,
// so the sort's up-front counting pass costs no extra read of the codes.
//
// Both kernels are HBM-bound: bbox reads 16 B/body; Morton reads 16 B/body and writes 8 B/body.
#include <cfloat>

#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) bbox_reduce_kernel(const float4 *__restrict__ pos, int64_t n,
                                                               BBoxAccum *__restrict__ acc) {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float4 p = __ldg(pos + i);
        mn[0] = gmin(mn[0], p.x); mn[1] = gmin(mn[1], p.y); mn[2] = gmin(mn[2], p.z);
        mx[0] = gmax(mx[0], p.x); mx[1] = gmax(mx[1], p.y); mx[2] = gmax(mx[2], p.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = gmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = gmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    __shared__ float smn[3][kThreads / 32], smx[3][kThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { smn[k][warp] = mn[k]; smx[k][warp] = mx[k]; }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int k = threadIdx.x;
        float a = smn[k][0], b = smx[k][0];
        for (int w = 1; w < kThreads / 32; ++w) { a = gmin(a, smn[k][w]); b = gmax(b, smx[k][w]); }
        atomicMin(&acc->v[k], float_to_ordered(a));
        atomicMin(&acc->v[3 + k], ~float_to_ordered(b));
    }
}

__global__ void __launch_bounds__(kThreads) morton_hist_kernel(const float4 *__restrict__ pos, int64_t n,
                                                               const BBoxAccum *__restrict__ acc,
                                                               uint64_t *__restrict__ codes,
                                                               uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) sh[i] = 0;
    float mn[3], mx[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        mn[k] = ordered_to_float(acc->v[k]);
        mx[k] = ordered_to_float(~acc->v[3 + k]);
    }
    const float dx = fsub(mx[0], mn[0]), dy = fsub(mx[1], mn[1]), dz = fsub(mx[2], mn[2]);
    const float scale = gmax(gmax(dx, dy), dz);  // std::max(std::max(x, y), z)
    __syncthreads();
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t code = morton_code(__ldg(pos + i), mn, scale);
        codes[i] = code;
#pragma unroll
        for (int d = 0; d < 8; ++d) atomicAdd(&sh[d * 256 + (uint32_t) ((code >> (8 * d)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
        uint32_t c = sh[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

int grid_for(int64_t n, int per_thread) {
    int64_t blocks = (n + (int64_t) kThreads * per_thread - 1) / ((int64_t) kThreads * per_thread);
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 8) blocks = 148 * 8;
    return (int) blocks;
}

}  // namespace

void launch_bbox_reset(BBoxAccum *acc, cudaStream_t s) { cudaMemsetAsync(acc, 0xFF, sizeof(BBoxAccum), s); }

void launch_bbox_reduce(const float4 *pos, int64_t n, BBoxAccum *acc, cudaStream_t s) {
    if (n <= 0) return;
    bbox_reduce_kernel<<<grid_for(n, 8), kThreads, 0, s>>>(pos, n, acc);
}

void launch_morton_hist(const float4 *pos, int64_t n, const BBoxAccum *acc, uint64_t *codes, uint32_t *hist,
                        cudaStream_t s) {
    if (n <= 0) return;
    cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(uint32_t), s);
    morton_hist_kernel<<<grid_for(n, 4), kThreads, 0, s>>>(pos, n, acc, codes, hist);
}

}  // namespace nbg
