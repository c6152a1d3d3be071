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
            const float inv = rsqrt_hw(r2);
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

// Energy diagnostics in FP64: per block, the kinetic energy 1/2 m v^2 of its bodies and the sum
// over its bodies i of m_i * sum_j m_j / sqrt(|r_ij|^2 + eps) (pairs at equal positions skipped,
// as the force skips them), reduced in a fixed order.
__global__ void __launch_bounds__(kThreads) energy_f64_kernel(const float4 *__restrict__ bodies,
                                                              const float4 *__restrict__ vel, int64_t n, double eps,
                                                              double *__restrict__ parts) {
    __shared__ float4 tile[kThreads];
    __shared__ double red[2][kThreads];
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    const float4 p = i < n ? bodies[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 v = i < n ? vel[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const double px = p.x, py = p.y, pz = p.z;
    double phi = 0.0;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t j = base + threadIdx.x;
        tile[threadIdx.x] = j < n ? bodies[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        const int cnt = (int) ((n - base) < kThreads ? (n - base) : kThreads);
        for (int k = 0; k < cnt; ++k) {
            const float4 b = tile[k];
            const double dx = (double) b.x - px, dy = (double) b.y - py, dz = (double) b.z - pz;
            if (dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
            phi += (double) b.w / sqrt(dx * dx + dy * dy + dz * dz + eps);
        }
        __syncthreads();
    }
    const double m = p.w;
    red[0][threadIdx.x] = i < n ? 0.5 * m * ((double) v.x * v.x + (double) v.y * v.y + (double) v.z * v.z) : 0.0;
    red[1][threadIdx.x] = i < n ? m * phi : 0.0;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if ((int) threadIdx.x < o) {
            red[0][threadIdx.x] += red[0][threadIdx.x + o];
            red[1][threadIdx.x] += red[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = red[0][0];
        parts[2 * blockIdx.x + 1] = red[1][0];
    }
}

// Sums the per-block parts in block order: out = (kinetic, -G/2 * sum m_i phi_i).
__global__ void energy_sum_kernel(const double *__restrict__ parts, int blocks, double G, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double k = 0.0, u = 0.0;
    for (int b = 0; b < blocks; ++b) {
        k += parts[2 * b];
        u += parts[2 * b + 1];
    }
    out[0] = k;
    out[1] = -0.5 * G * u;
}

}  // namespace

int64_t energy_parts(int64_t n) { return 2 * ((n + kThreads - 1) / kThreads) + 2; }

void launch_energy_f64(const float4 *bodies, const float4 *vel, int64_t n, double G, double eps, double *parts,
                       double *out, cudaStream_t s) {
    const int blocks = (int) ((n + kThreads - 1) / kThreads);
    if (blocks > 0) energy_f64_kernel<<<blocks, kThreads, 0, s>>>(bodies, vel, n, eps, parts);
    energy_sum_kernel<<<1, 1, 0, s>>>(parts, blocks, G, out);
}

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
