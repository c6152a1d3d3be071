// Kernels of the batched pipeline: many independent instances (each its own Morton box, tree and
// theta) laid out back to back in one body array and advanced by one launch per phase.
//
// Per force pass:
//   seg_bbox_kernel      slices of up to 8192 bodies of each instance: exact FP32 min/max of its
//                        positions (outerBoundingBox, SummaryType.h:73-81, per instance),
//                        combined with order-preserving integer atomics as bbox_reduce does
//   seg_morton_kernel    Morton code of every body in its instance's box (MortonSort.h:46-73) and
//                        the eight digit histograms of all codes
//   8 one-sweep passes   over all codes (radix_sort.cu), then 1-2 stable passes on the instance id
//                        (inst_key_kernel builds the keys, compose_kernel maps the result back), so
//                        bodies end grouped by instance, sorted by code within it, ties by position
//   the Karras build     over the keys (instance, code, index): each instance's subtree is exactly
//                        its standalone tree (lbvh_build.cu)
//   the traversal        driven by a table of 32-target groups that never straddle instances
// Since every instance sees exactly the operations of a standalone run, in the same order,
// its codes, tree and accelerations are bit-identical to running it alone.
#include <cfloat>

#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;

// Block (k, j) reduces slice j of `slices` of instance k. inst_box holds 6 ordered uints per
// instance (min.xyz, then ~max.xyz; see float_to_ordered), all reduced with atomicMin from all
// ones, so the result does not depend on the order of the slices.
__global__ void __launch_bounds__(kThreads) seg_bbox_kernel(const float4 *__restrict__ pos,
                                                            const int2 *__restrict__ inst_range, int slices,
                                                            uint32_t *__restrict__ inst_box) {
    const int k = blockIdx.x / slices, j = blockIdx.x - k * slices;
    const int2 r = inst_range[k];
    const int64_t len = (int64_t) r.y - r.x + 1;
    const int lo = r.x + (int) (len * j / slices), hi = r.x + (int) (len * (j + 1) / slices);
    if (lo >= hi) return;  // uniform across the block
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const float4 p = __ldg(pos + i);
        mn[0] = gmin(mn[0], p.x); mn[1] = gmin(mn[1], p.y); mn[2] = gmin(mn[2], p.z);
        mx[0] = gmax(mx[0], p.x); mx[1] = gmax(mx[1], p.y); mx[2] = gmax(mx[2], p.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            mn[c] = gmin(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
            mx[c] = gmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
        }
    }
    __shared__ float smn[3][kThreads / 32], smx[3][kThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { smn[c][warp] = mn[c]; smx[c][warp] = mx[c]; }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int c = threadIdx.x;
        float a = smn[c][0], b = smx[c][0];
        for (int w = 1; w < kThreads / 32; ++w) { a = gmin(a, smn[c][w]); b = gmax(b, smx[c][w]); }
        atomicMin(&inst_box[6 * k + c], float_to_ordered(a));
        atomicMin(&inst_box[6 * k + 3 + c], ~float_to_ordered(b));
    }
}

__global__ void __launch_bounds__(kThreads) seg_morton_kernel(const float4 *__restrict__ pos, int64_t n,
                                                              const int *__restrict__ inst_of,
                                                              const uint32_t *__restrict__ inst_box,
                                                              uint64_t *__restrict__ codes,
                                                              uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t *ob = inst_box + 6 * inst_of[i];
        const float b[6] = {ordered_to_float(ob[0]), ordered_to_float(ob[1]), ordered_to_float(ob[2]),
                            ordered_to_float(~ob[3]), ordered_to_float(~ob[4]), ordered_to_float(~ob[5])};
        const float mn[3] = {b[0], b[1], b[2]};
        const float dx = fsub(b[3], b[0]), dy = fsub(b[4], b[1]), dz = fsub(b[5], b[2]);
        const float scale = gmax(gmax(dx, dy), dz);
        const uint64_t code = morton_code(__ldg(pos + i), mn, scale);
        codes[i] = code;
#pragma unroll
        for (int d = 0; d < 8; ++d) atomicAdd(&sh[d * 256 + (uint32_t) ((code >> (8 * d)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
        const uint32_t c = sh[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// Instance id of the body at each code-sorted position (positions never leave their instance's
// segment, so inst_of indexed by the sort's slot value is that body's instance).
__global__ void __launch_bounds__(kThreads) inst_key_kernel(const uint32_t *__restrict__ slot, int64_t n,
                                                            const int *__restrict__ inst_of,
                                                            uint64_t *__restrict__ ikeys) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t s = slot[k];
    ikeys[k] = (s < (uint64_t) n) ? (uint64_t) inst_of[s] : 0ull;
}

// perm[j] = slot[order[j]], codes_out[j] = codes[order[j]]: the instance-major permutation.
__global__ void __launch_bounds__(kThreads) compose_kernel(const uint32_t *__restrict__ order, int64_t n,
                                                           const uint32_t *__restrict__ slot,
                                                           const uint64_t *__restrict__ codes,
                                                           uint32_t *__restrict__ perm,
                                                           uint64_t *__restrict__ codes_out) {
    const int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t k = order[j];
    if (k >= (uint64_t) n) return;
    perm[j] = slot[k];
    codes_out[j] = codes[k];
}

unsigned blocks_for(int64_t n) { return (unsigned) ((n + kThreads - 1) / kThreads); }

// One block per instance: the instance id of each of its body positions, and its 32-target
// traversal groups (first target, count, instance) starting at group_first[k].
__global__ void __launch_bounds__(kThreads) fill_tables_kernel(const int2 *__restrict__ inst_range,
                                                               const int *__restrict__ group_first,
                                                               int *__restrict__ inst_of, int4 *__restrict__ groups) {
    const int k = blockIdx.x;
    const int2 r = inst_range[k];
    for (int i = r.x + threadIdx.x; i <= r.y; i += blockDim.x) inst_of[i] = k;
    const int n = r.y - r.x + 1;
    const int g0 = group_first[k];
    for (int j = threadIdx.x; j * 32 < n; j += blockDim.x)
        groups[g0 + j] = make_int4(r.x + 32 * j, min(32, n - 32 * j), k, 0);
}

}  // namespace

void launch_fill_tables(const int2 *inst_range, const int *group_first, int num_inst, int *inst_of, int4 *groups,
                        cudaStream_t s) {
    if (num_inst <= 0) return;
    fill_tables_kernel<<<num_inst, kThreads, 0, s>>>(inst_range, group_first, inst_of, groups);
}

void launch_seg_bbox(const float4 *pos, const int2 *inst_range, int num_inst, int slices, uint32_t *inst_box,
                     cudaStream_t s) {
    if (num_inst <= 0) return;
    slices = slices < 1 ? 1 : slices;
    cudaMemsetAsync(inst_box, 0xFF, (size_t) num_inst * 6 * sizeof(uint32_t), s);
    seg_bbox_kernel<<<(unsigned) ((int64_t) num_inst * slices), kThreads, 0, s>>>(pos, inst_range, slices, inst_box);
}

void launch_seg_morton(const float4 *pos, int64_t n, const int *inst_of, const uint32_t *inst_box, uint64_t *codes,
                       uint32_t *hist, cudaStream_t s) {
    if (n <= 0) return;
    cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(uint32_t), s);
    int64_t blocks = (n + kThreads * 4 - 1) / (kThreads * 4);
    blocks = blocks < 1 ? 1 : (blocks > 148 * 8 ? 148 * 8 : blocks);
    seg_morton_kernel<<<(unsigned) blocks, kThreads, 0, s>>>(pos, n, inst_of, inst_box, codes, hist);
}

void launch_inst_keys(const uint32_t *slot, int64_t n, const int *inst_of, uint64_t *ikeys, cudaStream_t s) {
    if (n <= 0) return;
    inst_key_kernel<<<blocks_for(n), kThreads, 0, s>>>(slot, n, inst_of, ikeys);
}

void launch_compose(const uint32_t *order, int64_t n, const uint32_t *slot, const uint64_t *codes, uint32_t *perm,
                    uint64_t *codes_out, cudaStream_t s) {
    if (n <= 0) return;
    compose_kernel<<<blocks_for(n), kThreads, 0, s>>>(order, n, slot, codes, perm, codes_out);
}

}  // namespace nbg
