// Barnes-Hut traversal of the preorder linear BVH: one warp walks the tree for 32 Morton-adjacent
// targets in lock step, without a stack.
//
// Semantics are those of Descent::activeTree (src/NBody/Simulation/Solvers/Descent/activeTree.h:24-79)
// under DiagonalOverCenterDistance (DiagonalOverCenterDistance.h:18-22) with the Gravity rule
// (src/NBody/Physics/Rules/Gravity.h:199-259), decided per target:
//   - a node is approximated for a target iff diag^2 / |centre - p|^2 < theta^2; the node record
//     carries the exact threshold on |centre - p|^2, and the squared distance is formed with the
//     reference's IEEE operation order, so every target takes exactly the reference's decisions
//     (and the interaction counts match the reference's SimpleTrackingRule counts exactly);
//   - an opened leaf interacts pairwise with its bodies (including the target itself, which
//     contributes zero);
//   - otherwise the children are visited.
//
// Lock-step without a stack: nodes are stored in preorder with a "skip" index (first node after
// the subtree). Each lane keeps the next preorder node it needs; the warp processes the smallest
// such node (one redux.sync), so every lane sees its own visit sequence in order, node records
// are broadcast loads shared by the whole warp, and leaf bodies are loaded once per warp.
//
// Arithmetic: FP32, one MUFU rsqrt per interaction, G applied once per target. The pair term is
// 12 FP32 instructions (20 flops by the usual direct-sum convention); the quadrupole node term
// (non-traceless moments about the centre of mass, as in Gravity.h:239-259 with D<3> contracted
// analytically: (D3:Q)_i = g3 R_i (R.Q.R) + g2 (2 (Q R)_i + R_i tr Q)) is 56 flops.
#include <climits>

#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;

template<bool EPS0>
__device__ __forceinline__ void pair_term(float px, float py, float pz, float4 b, float eps, float &ax, float &ay,
                                          float &az) {
    const float rx = px - b.x, ry = py - b.y, rz = pz - b.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps)));
    if (EPS0 && r2 == 0.f) return;  // equal positions contribute nothing (Gravity.h:203)
    const float inv = rsqrtf(r2);
    const float s = b.w * (inv * inv * inv);
    ax = fmaf(-rx, s, ax);
    ay = fmaf(-ry, s, ay);
    az = fmaf(-rz, s, az);
}

template<bool EPS0>
__device__ __forceinline__ void quad_term(float px, float py, float pz, float4 com, const float q[6], float eps,
                                          float &ax, float &ay, float &az) {
    const float rx = px - com.x, ry = py - com.y, rz = pz - com.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps)));
    if (EPS0 && r2 == 0.f) return;
    const float inv = rsqrtf(r2);
    const float inv2 = inv * inv;
    const float inv3 = inv2 * inv;
    const float inv5 = inv3 * inv2;
    const float inv7 = inv5 * inv2;
    const float qx = fmaf(q[0], rx, fmaf(q[1], ry, q[2] * rz));
    const float qy = fmaf(q[1], rx, fmaf(q[3], ry, q[4] * rz));
    const float qz = fmaf(q[2], rx, fmaf(q[4], ry, q[5] * rz));
    const float rqr = fmaf(rx, qx, fmaf(ry, qy, rz * qz));
    const float tr = q[0] + q[3] + q[5];
    const float sr = fmaf(-7.5f * inv7, rqr, fmaf(1.5f * inv5, tr, -com.w * inv3));
    const float sq = 3.0f * inv5;
    ax = fmaf(rx, sr, fmaf(qx, sq, ax));
    ay = fmaf(ry, sr, fmaf(qy, sq, ay));
    az = fmaf(rz, sr, fmaf(qz, sq, az));
}

template<int ORDER, bool EPS0>
__global__ void __launch_bounds__(kThreads) bh_kernel(const float4 *__restrict__ nodes,
                                                      const int *__restrict__ num_nodes_p,
                                                      const float4 *__restrict__ bodies, int n_bodies,
                                                      const float4 *__restrict__ targets, int64_t n_targets, float G,
                                                      float eps, float4 *__restrict__ acc,
                                                      unsigned long long *__restrict__ counts) {
    constexpr int REC = NodeLayout<ORDER>::REC;
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x);
    if ((i - lane) >= n_targets) return;  // whole warp out of range
    const int num_nodes = *num_nodes_p;
    const bool valid = i < n_targets;
    const float4 p = valid ? targets[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    float ax = 0.f, ay = 0.f, az = 0.f;
    unsigned npp = 0, nnp = 0;
    int next = valid ? 0 : INT_MAX;

    while (true) {
        const int c = __reduce_min_sync(0xffffffffu, next);
        if (c >= num_nodes) break;
        const float4 *r = nodes + (int64_t) c * REC;
        const float4 mac = __ldg(r);
        const float4 com = __ldg(r + 1);
        float q[6];
        int link0, link1;
        if constexpr (ORDER == 1) {
            const float4 l = __ldg(r + 2);
            link0 = __float_as_int(l.x);
            link1 = __float_as_int(l.y);
        } else {
            const float4 q0 = __ldg(r + 2), q1 = __ldg(r + 3);
            q[0] = q0.x; q[1] = q0.y; q[2] = q0.z; q[3] = q0.w; q[4] = q1.x; q[5] = q1.y;
            link0 = __float_as_int(q1.z);
            link1 = __float_as_int(q1.w);
        }
        const bool leaf = link1 >= 0;
        if (leaf) {  // defensive clamp: a leaf never reaches outside the body array
            link0 = max(link0, 0);
            link1 = min(link1, n_bodies);
        }
        bool open = false;
        if (next == c) {
            const float dx = fsub(p.x, mac.x), dy = fsub(p.y, mac.y), dz = fsub(p.z, mac.z);
            const float d2 = fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
            if (d2 >= mac.w) {
                if constexpr (ORDER == 1) pair_term<EPS0>(p.x, p.y, p.z, com, eps, ax, ay, az);
                else quad_term<EPS0>(p.x, p.y, p.z, com, q, eps, ax, ay, az);
                ++nnp;
                next = leaf ? c + 1 : max(link0, c + 1);  // the cursor only moves forward
            } else {
                next = c + 1;
                open = leaf;
            }
        }
        if (leaf && __any_sync(0xffffffffu, open)) {
            for (int j = link0; j < link1; ++j) {
                const float4 b = __ldg(bodies + j);
                if (open) pair_term<EPS0>(p.x, p.y, p.z, b, eps, ax, ay, az);
            }
            if (open) npp += (unsigned) (link1 - link0);
        }
    }
    if (valid) acc[i] = make_float4(G * ax, G * ay, G * az, 0.f);
    if (counts) {
        const unsigned spp = __reduce_add_sync(0xffffffffu, npp);
        const unsigned snp = __reduce_add_sync(0xffffffffu, nnp);
        if (lane == 0) {
            atomicAdd(counts + 0, (unsigned long long) spp);
            atomicAdd(counts + 1, (unsigned long long) snp);
        }
    }
}

template<int ORDER>
void launch_order(const float4 *nodes, const int *num_nodes, const float4 *bodies, int n_bodies,
                  const float4 *targets, int64_t nt, float G, float eps, float4 *acc, unsigned long long *counts,
                  cudaStream_t s) {
    const int64_t blocks = (nt + kThreads - 1) / kThreads;
    if (eps == 0.f)
        bh_kernel<ORDER, true><<<(unsigned) blocks, kThreads, 0, s>>>(nodes, num_nodes, bodies, n_bodies, targets, nt,
                                                                       G, eps, acc, counts);
    else
        bh_kernel<ORDER, false><<<(unsigned) blocks, kThreads, 0, s>>>(nodes, num_nodes, bodies, n_bodies, targets, nt,
                                                                        G, eps, acc, counts);
}

}  // namespace

void launch_bh_traverse(int order, const float4 *nodes, const int *num_nodes, const float4 *bodies, int64_t n_bodies,
                        const float4 *targets, int64_t n_targets, float G, float eps, float4 *acc,
                        unsigned long long *counts, cudaStream_t s) {
    if (n_targets <= 0) return;
    const int nb = (int) n_bodies;
    if (order == 1) launch_order<1>(nodes, num_nodes, bodies, nb, targets, n_targets, G, eps, acc, counts, s);
    else launch_order<2>(nodes, num_nodes, bodies, nb, targets, n_targets, G, eps, acc, counts, s);
}

}  // namespace nbg
