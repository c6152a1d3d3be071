// Shared-memory-tiled direct sum: the NaiveSolver path (src/NBody/Simulation/Solvers/NaiveSolver.h:22-52)
// in FP32, and an FP64 variant that serves as the accuracy reference for the tree solvers.
//
// Each thread owns one target; the block stages 256 source bodies at a time in shared memory
// (coalesced float4 loads) and every thread sweeps the tile from shared memory (broadcast reads).
// Pair term as Gravity::particleParticle (Gravity.h:199-209): a += -R m / (|R|^2 + eps)^{3/2},
// R = target - source, identical positions skipped.
#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;

template<bool EPS0>
__global__ void __launch_bounds__(kThreads) direct_f32_kernel(const float4 *__restrict__ bodies, int64_t n,
                                                              const float4 *__restrict__ targets, int64_t nt,
                                                              float G, float eps, float4 *__restrict__ acc) {
    __shared__ float4 tile[kThreads];
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    const float4 p = i < nt ? targets[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t j = base + threadIdx.x;
        tile[threadIdx.x] = j < n ? bodies[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        const int cnt = (int) ((n - base) < kThreads ? (n - base) : kThreads);
#pragma unroll 8
        for (int k = 0; k < cnt; ++k) {
            const float4 b = tile[k];
            const float rx = p.x - b.x, ry = p.y - b.y, rz = p.z - b.z;
            const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps)));
            if (EPS0 && r2 == 0.f) continue;
            const float inv = rsqrtf(r2);
            const float s = b.w * (inv * inv * inv);
            ax = fmaf(-rx, s, ax);
            ay = fmaf(-ry, s, ay);
            az = fmaf(-rz, s, az);
        }
        __syncthreads();
    }
    if (i < nt) acc[i] = make_float4(G * ax, G * ay, G * az, 0.f);
}

__global__ void __launch_bounds__(kThreads) direct_f64_kernel(const float4 *__restrict__ bodies, int64_t n,
                                                              const float4 *__restrict__ targets, int64_t nt,
                                                              double G, double eps, double *__restrict__ acc3) {
    __shared__ float4 tile[kThreads];
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    const float4 p = i < nt ? targets[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const double px = p.x, py = p.y, pz = p.z;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t j = base + threadIdx.x;
        tile[threadIdx.x] = j < n ? bodies[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        const int cnt = (int) ((n - base) < kThreads ? (n - base) : kThreads);
        for (int k = 0; k < cnt; ++k) {
            const float4 b = tile[k];
            const double dx = (double) b.x - px, dy = (double) b.y - py, dz = (double) b.z - pz;
            if (dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
            const double r2 = dx * dx + dy * dy + dz * dz + eps;
            const double s = (double) b.w / (r2 * sqrt(r2));
            ax += dx * s;
            ay += dy * s;
            az += dz * s;
        }
        __syncthreads();
    }
    if (i < nt) {
        acc3[3 * i + 0] = G * ax;
        acc3[3 * i + 1] = G * ay;
        acc3[3 * i + 2] = G * az;
    }
}

}  // namespace

void launch_direct_f32(const float4 *bodies, int64_t n, const float4 *targets, int64_t nt, float G, float eps,
                       float4 *acc, cudaStream_t s) {
    if (nt <= 0) return;
    const unsigned blocks = (unsigned) ((nt + kThreads - 1) / kThreads);
    if (eps == 0.f) direct_f32_kernel<true><<<blocks, kThreads, 0, s>>>(bodies, n, targets, nt, G, eps, acc);
    else direct_f32_kernel<false><<<blocks, kThreads, 0, s>>>(bodies, n, targets, nt, G, eps, acc);
}

void launch_direct_f64(const float4 *bodies, int64_t n, const float4 *targets, int64_t nt, double G, double eps,
                       double *acc3, cudaStream_t s) {
    if (nt <= 0) return;
    const unsigned blocks = (unsigned) ((nt + kThreads - 1) / kThreads);
    direct_f64_kernel<<<blocks, kThreads, 0, s>>>(bodies, n, targets, nt, G, eps, acc3);
}

}  // namespace nbg
