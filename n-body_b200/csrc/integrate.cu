// State permutation and the kick-drift integrator.
//
// Solver::step (src/NBody/Simulation/Solver.h:103-139) advances bodies with v = v + a*dt followed
// by p = p + v*dt; the multiply and add are separate IEEE operations here as in the reference's
// FP32 build. The drift kernel also reduces the bounding box of the new positions, so the next
// step's Morton quantisation needs no separate pass over the bodies.
//
// Bodies live in the order of the last Morton sort; gather_state permutes positions, velocities
// and input ids after each sort so the traversal reads its targets and leaf bodies contiguously.
// All kernels here are HBM-bound streaming kernels.
#include <cfloat>

#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;

unsigned blocks_for(int64_t n) { return (unsigned) ((n + kThreads - 1) / kThreads); }

__global__ void __launch_bounds__(kThreads) gather_state_kernel(const uint32_t *__restrict__ perm, int64_t n,
                                                                 const float4 *__restrict__ pos,
                                                                 const float4 *__restrict__ vel,
                                                                 const uint32_t *__restrict__ id,
                                                                 float4 *__restrict__ pos_out,
                                                                 float4 *__restrict__ vel_out,
                                                                 uint32_t *__restrict__ id_out) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t src = perm[k];
    if (src >= (uint64_t) n) return;  // defensive: a failed sort never makes this read out of bounds
    pos_out[k] = __ldg(pos + src);
    if (vel) vel_out[k] = __ldg(vel + src);
    id_out[k] = __ldg(id + src);
}

__global__ void __launch_bounds__(kThreads) scatter_by_id_kernel(const uint32_t *__restrict__ id, int64_t n,
                                                                 const float4 *__restrict__ src,
                                                                 float4 *__restrict__ dst) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t d = id[k];
    if (d < (uint64_t) n) dst[d] = src[k];
}

__global__ void __launch_bounds__(kThreads) iota_kernel(uint32_t *__restrict__ id, int64_t n, uint32_t first) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) id[k] = first + (uint32_t) k;
}

__global__ void __launch_bounds__(kThreads) add_offset_kernel(uint32_t *__restrict__ id, int64_t n, int64_t delta) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) id[k] = (uint32_t) ((int64_t) id[k] + delta);
}

__global__ void __launch_bounds__(kThreads) kick_drift_kernel(float4 *__restrict__ pos, float4 *__restrict__ vel,
                                                              const float4 *__restrict__ acc, int64_t n, float dt,
                                                              BBoxAccum *__restrict__ next_bbox) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    if (k < n) {
        float4 p = pos[k], v = vel[k];
        const float4 a = acc[k];
        v.x = fadd(v.x, fmul(a.x, dt));
        v.y = fadd(v.y, fmul(a.y, dt));
        v.z = fadd(v.z, fmul(a.z, dt));
        p.x = fadd(p.x, fmul(v.x, dt));
        p.y = fadd(p.y, fmul(v.y, dt));
        p.z = fadd(p.z, fmul(v.z, dt));
        vel[k] = v;
        pos[k] = p;
        mn[0] = p.x; mn[1] = p.y; mn[2] = p.z;
        mx[0] = p.x; mx[1] = p.y; mx[2] = p.z;
    }
    if (!next_bbox) return;
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
        if (a <= b) {
            atomicMin(&next_bbox->v[c], float_to_ordered(a));
            atomicMin(&next_bbox->v[3 + c], ~float_to_ordered(b));
        }
    }
}

}  // namespace

void launch_gather_state(const uint32_t *perm, int64_t n, const float4 *pos, const float4 *vel, const uint32_t *id,
                         float4 *pos_out, float4 *vel_out, uint32_t *id_out, cudaStream_t s) {
    if (n <= 0) return;
    gather_state_kernel<<<blocks_for(n), kThreads, 0, s>>>(perm, n, pos, vel, id, pos_out, vel_out, id_out);
}

void launch_scatter_by_id(const uint32_t *id, int64_t n, const float4 *src, float4 *dst, cudaStream_t s) {
    if (n <= 0) return;
    scatter_by_id_kernel<<<blocks_for(n), kThreads, 0, s>>>(id, n, src, dst);
}

void launch_iota(uint32_t *id, int64_t n, cudaStream_t s, uint32_t first) {
    if (n <= 0) return;
    iota_kernel<<<blocks_for(n), kThreads, 0, s>>>(id, n, first);
}

void launch_add_offset(uint32_t *id, int64_t n, int64_t delta, cudaStream_t s) {
    if (n <= 0 || delta == 0) return;
    add_offset_kernel<<<blocks_for(n), kThreads, 0, s>>>(id, n, delta);
}

void launch_kick_drift(float4 *pos, float4 *vel, const float4 *acc, int64_t n, float dt, BBoxAccum *next_bbox,
                       cudaStream_t s) {
    if (n <= 0) return;
    kick_drift_kernel<<<blocks_for(n), kThreads, 0, s>>>(pos, vel, acc, n, dt, next_bbox);
}

}  // namespace nbg
