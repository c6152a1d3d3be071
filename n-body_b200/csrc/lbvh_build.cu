// Linear BVH construction and bottom-up summaries.
//
// The reference builds its LinearBVH top-down (src/NBody/Simulation/Solvers/Trees/LinearBVH.h:47-76,
// 106-133): a node holding a range of Morton-sorted bodies splits at the first body whose code has
// the most significant differing bit of the range's end codes set, and stops splitting when it
// holds at most maxLeafSize bodies or its end codes are equal. That split rule is the binary
// radix tree rule, so the same tree comes out of a fully parallel Karras (HPG 2012) build over
// the sorted codes (ties broken by index), collapsed wherever the reference stops splitting:
//   - a Karras internal node is a final internal node iff it is "splittable"
//     (more than maxLeafSize bodies and different end codes); splittability is monotone, so all
//     its ancestors are final internal nodes too;
//   - a final leaf is a non-splittable child of a final internal node (or the root itself).
//
// Kernels:
//   karras_kernel     one thread per Karras internal node: children, range, parent, the final
//                     internal / final leaf flags (reads ~2 log n codes per node, L2-resident),
//                     and the number of final nodes starting at each body position
//   scan kernels      exclusive prefix over body positions of those counts: the preorder index of
//                     the final leaf starting at each position
//   summarize_kernel  one thread per final internal node with leaf children: sequential leaf
//                     summaries over the leaf's bodies, then an atomic climb in which the second
//                     child to arrive summarises the parent (CenterOfMassSummary.h:30-55,
//                     BoundingBoxSummary.h:30-68, MultipoleMassSummary.h:37-97; the leaf moment
//                     sum follows libstdc++'s 4-way std::transform_reduce). All float operations
//                     are single IEEE operations in the reference's order, so summaries are
//                     bit-identical to the CPU restatement. Every node's record (the arrays the
//                     traversal reads: MAC data, links, payload) is written by the thread that
//                     finishes the node, at the node's preorder index. That index is closed-form:
//                     for a node whose range starts at body f, the final nodes before it in
//                     preorder are those starting before f and, among the internal nodes starting
//                     at f (a chain of left children), the larger ones; a leaf starting at f comes
//                     after that whole chain.
#include <algorithm>
#include <cfloat>

#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;

// Length of the common prefix of the keys (instance, code, index) at sorted positions i and j;
// -1 outside the array. Without instances the instance field is equal everywhere.
__device__ __forceinline__ int prefix_delta(const uint64_t *__restrict__ codes, const int *__restrict__ inst_of, int n,
                                            int i, int j) {
    if (j < 0 || j >= n) return -1;
    if (inst_of) {
        const int a = inst_of[i], b = inst_of[j];
        if (a != b) return __clz(a ^ b);
    }
    const uint64_t a = codes[i], b = codes[j];
    return 32 + ((a != b) ? __clzll(a ^ b) : 64 + __clz(i ^ j));
}

// A node covering sorted positions [a, b] is split by the reference (a final internal node) iff it
// holds more than `leaf` bodies with different end codes; a node spanning several instances only
// connects their trees and is always split.
__device__ __forceinline__ bool range_splittable(const uint64_t *__restrict__ codes, const int *__restrict__ inst_of,
                                                 int leaf, int a, int b) {
    if (inst_of && inst_of[a] != inst_of[b]) return true;
    return (b - a + 1 > leaf) && (codes[a] != codes[b]);
}

// Karras node flags: bit 0 a final internal node (the reference splits it); bits 1 and 2 its left /
// right child is a final leaf (set for final internal nodes only).
constexpr uint8_t kFinal = 1, kLeftLeaf = 2, kRightLeaf = 4;

__global__ void __launch_bounds__(kThreads) karras_kernel(const uint64_t *__restrict__ codes,
                                                          const int *__restrict__ inst_of, int n, int leaf,
                                                          TreeWorkspace tw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int dn = prefix_delta(codes, inst_of, n, i, i + 1);
    const int dp = prefix_delta(codes, inst_of, n, i, i - 1);
    const int d = (dn > dp) ? 1 : -1;
    const int dmin = (d > 0) ? dp : dn;
    int lmax = 2;
    while (prefix_delta(codes, inst_of, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (prefix_delta(codes, inst_of, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = prefix_delta(codes, inst_of, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (prefix_delta(codes, inst_of, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    const int first = min(i, j), last = max(i, j);
    const int lc = (first == gamma) ? ~gamma : gamma;
    const int rc = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    tw.topo[i] = make_int4(lc, rc, first, last);
    tw.visit[i] = 0;
    if (lc >= 0) tw.parent[lc] = i;
    if (rc >= 0) tw.parent[rc] = i;
    const bool split = range_splittable(codes, inst_of, leaf, first, last);
    uint8_t f = (uint8_t) split;
    if (split) {
        // a final internal node starts at `first`; a child that is not split is a final leaf
        atomicAdd(tw.start + first, 2);
        const bool lleaf = lc < 0 || !range_splittable(codes, inst_of, leaf, first, gamma);
        const bool rleaf = rc < 0 || !range_splittable(codes, inst_of, leaf, gamma + 1, last);
        if (lleaf) atomicAdd(tw.start + first, 1);
        if (rleaf) atomicAdd(tw.start + gamma + 1, 1);
        if (lleaf || rleaf) tw.leaf_parents[atomicAdd(tw.leaf_parents_count, 1)] = i;
        f |= (uint8_t) ((lleaf ? kLeftLeaf : 0) | (rleaf ? kRightLeaf : 0));
    }
    tw.flags[i] = f;
}

// Exclusive prefix over positions 0..n of the number of final nodes starting at each position,
// in three steps: tile totals, a prefix over the tiles (one block), and the per-tile scan.
constexpr int kScanTile = 2048;

__device__ __forceinline__ int starts_at(const int *__restrict__ start, int64_t b) {
    const int w = start[b];
    return (w >> 1) + (w & 1);
}

__global__ void __launch_bounds__(kThreads) scan_tiles_kernel(const int *__restrict__ start, int64_t m,
                                                              int *__restrict__ part) {
    __shared__ int red[kThreads / 32];
    const int64_t base = (int64_t) blockIdx.x * kScanTile;
    int sum = 0;
    for (int k = threadIdx.x; k < kScanTile; k += kThreads)
        if (base + k < m) sum += starts_at(start, base + k);
    sum = __reduce_add_sync(0xffffffffu, sum);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

// One block: part[t] becomes the exclusive prefix of the tile totals; the total is the node count.
__global__ void __launch_bounds__(1024) scan_parts_kernel(int *__restrict__ part, int tiles, int *__restrict__ total) {
    __shared__ int warp_sum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < tiles; base += 1024) {
        const int t = base + threadIdx.x;
        const int v = t < tiles ? part[t] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sum[warp] = incl;
        __syncthreads();
        int before = carry;
        for (int w = 0; w < warp; ++w) before += warp_sum[w];
        if (t < tiles) part[t] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Writes pre_base[f] = (final nodes starting before f) + (final internal nodes starting at f): the
// preorder index of the final leaf starting at f, one past the smallest internal node starting there.
__global__ void __launch_bounds__(kThreads) scan_apply_kernel(const int *__restrict__ start, int64_t m,
                                                              const int *__restrict__ part, int *__restrict__ pre_base) {
    constexpr int kPer = kScanTile / kThreads;  // consecutive positions per thread
    __shared__ int warp_sum[kThreads / 32];
    const int64_t base = (int64_t) blockIdx.x * kScanTile + (int64_t) threadIdx.x * kPer;
    int v[kPer], w[kPer];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        w[k] = base + k < m ? start[base + k] : 0;
        v[k] = (w[k] >> 1) + (w[k] & 1);
        sum += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    int run = part[blockIdx.x] + incl - sum;
    for (int w = 0; w < warp; ++w) run += warp_sum[w];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (base + k < m) pre_base[base + k] = run + (w[k] >> 1);
        run += v[k];
    }
}

// Preorder index of a final node whose range starts at body f: after the final nodes starting
// before f; an internal node follows the larger internal nodes of its chain at f (chain = final
// internal nodes below it that share f), a leaf follows the whole chain.
__device__ __forceinline__ int preorder_internal(const TreeWorkspace &tw, int f, int chain) {
    return tw.pre_base[f] - 1 - chain;
}
__device__ __forceinline__ int preorder_leaf(const TreeWorkspace &tw, int f) { return tw.pre_base[f]; }

template<int ORDER>
struct Summ {
    float bmin[3], bmax[3], com[3], M;
    float q[6];
    float q3[ORDER >= 3 ? 10 : 1];
};

// Summary slots, one record per node (Karras internal index, or n - 1 + body index for a leaf):
// 4 float4 (64 bytes) for orders 1 and 2, 8 float4 (128 bytes) for order 3:
//   [0] bmin.xyz, bmax.x  [1] bmax.yz, com.xy  [2] com.z, M, Q2[0..1]  [3] Q2[2..5]
//   [4] Q3[0..3]  [5] Q3[4..7]  [6] Q3[8..9]
template<int ORDER>
__device__ __forceinline__ float4 *slot_ptr(const TreeWorkspace &tw, int slot) {
    return ORDER >= 3 ? tw.slot3 + (int64_t) slot * 8 : tw.slot + (int64_t) slot * 4;
}

template<int ORDER>
__device__ __forceinline__ void store_slot(const TreeWorkspace &tw, int slot, const Summ<ORDER> &s) {
    float4 *d = slot_ptr<ORDER>(tw, slot);
    d[0] = make_float4(s.bmin[0], s.bmin[1], s.bmin[2], s.bmax[0]);
    d[1] = make_float4(s.bmax[1], s.bmax[2], s.com[0], s.com[1]);
    if constexpr (ORDER >= 2) {
        d[2] = make_float4(s.com[2], s.M, s.q[0], s.q[1]);
        d[3] = make_float4(s.q[2], s.q[3], s.q[4], s.q[5]);
    } else {
        d[2] = make_float4(s.com[2], s.M, 0.f, 0.f);
    }
    if constexpr (ORDER >= 3) {
        d[4] = make_float4(s.q3[0], s.q3[1], s.q3[2], s.q3[3]);
        d[5] = make_float4(s.q3[4], s.q3[5], s.q3[6], s.q3[7]);
        d[6] = make_float4(s.q3[8], s.q3[9], 0.f, 0.f);
    }
}

// Loads bypass L1: the slot was written by another thread, possibly of another block, moments ago.
template<int ORDER>
__device__ __forceinline__ Summ<ORDER> load_slot(const TreeWorkspace &tw, int slot) {
    Summ<ORDER> s;
    const float4 *d = slot_ptr<ORDER>(tw, slot);
    const float4 a = __ldcg(d), b = __ldcg(d + 1), c = __ldcg(d + 2);
    s.bmin[0] = a.x; s.bmin[1] = a.y; s.bmin[2] = a.z; s.bmax[0] = a.w;
    s.bmax[1] = b.x; s.bmax[2] = b.y; s.com[0] = b.z; s.com[1] = b.w;
    s.com[2] = c.x; s.M = c.y;
    if constexpr (ORDER >= 2) {
        const float4 e = __ldcg(d + 3);
        s.q[0] = c.z; s.q[1] = c.w; s.q[2] = e.x; s.q[3] = e.y; s.q[4] = e.z; s.q[5] = e.w;
    }
    if constexpr (ORDER >= 3) {
        const float4 f = __ldcg(d + 4), g = __ldcg(d + 5), h = __ldcg(d + 6);
        s.q3[0] = f.x; s.q3[1] = f.y; s.q3[2] = f.z; s.q3[3] = f.w;
        s.q3[4] = g.x; s.q3[5] = g.y; s.q3[6] = g.z; s.q3[7] = g.w;
        s.q3[8] = h.x; s.q3[9] = h.y;
    }
    return s;
}

// Packed quadrupole of an offset: [xx, xy, xz, yy, yz, zz], each times the mass.
__device__ __forceinline__ void offset_quadrupole(float ox, float oy, float oz, float m, float q[6]) {
    q[0] = fmul(fmul(ox, ox), m);
    q[1] = fmul(fmul(ox, oy), m);
    q[2] = fmul(fmul(ox, oz), m);
    q[3] = fmul(fmul(oy, oy), m);
    q[4] = fmul(fmul(oy, oz), m);
    q[5] = fmul(fmul(oz, oz), m);
}

// Unique-slot dimensions of the order-3 packed tensor (XXX, XXY, XXZ, XYY, XYZ, XZZ, YYY, YYZ,
// YZZ, ZZZ) and the order-2 slot of a sorted pair, as in SymmetricTensor3.h:372-395.
__device__ __forceinline__ int slot2(int a, int b) { return a == 0 ? b : 3 + (a == 2) + (b == 2); }
__device__ __forceinline__ void dims3(int L, int d[3]) {
    const int t[10][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 1, 1}, {0, 1, 2},
                          {0, 2, 2}, {1, 1, 1}, {1, 1, 2}, {1, 2, 2}, {2, 2, 2}};
    d[0] = t[L][0]; d[1] = t[L][1]; d[2] = t[L][2];
}
__device__ __forceinline__ int slot2u(int a, int b) { return a <= b ? slot2(a, b) : slot2(b, a); }

// Octupole term of one offset: outerProduct(outerProduct(d, d), d) (MultipoleMoment.h:46-62),
// times the mass; t2 is the unscaled packed d (x) d.
__device__ __forceinline__ void offset_octupole(const float t2[6], const float d[3], float m, float q3[10]) {
#pragma unroll
    for (int L = 0; L < 10; ++L) {
        int dd[3];
        dims3(L, dd);
        q3[L] = fmul(fmul(t2[slot2(dd[0], dd[1])], d[dd[2]]), m);
    }
}

// sumOfOuterProducts(T2, d) at each order-3 slot: right fold over the three left rotations of
// the index (SymmetricTensor3.h:235-244, 483-488).
__device__ __forceinline__ void sum_outer3(const float t2[6], const float d[3], float out[10]) {
#pragma unroll
    for (int L = 0; L < 10; ++L) {
        int a[3];
        dims3(L, a);
        const float e0 = fmul(t2[slot2u(a[0], a[1])], d[a[2]]);
        const float e1 = fmul(t2[slot2u(a[1], a[2])], d[a[0]]);
        const float e2 = fmul(t2[slot2u(a[2], a[0])], d[a[1]]);
        out[L] = fadd(e0, fadd(e1, e2));
    }
}

template<int ORDER>
__device__ Summ<ORDER> leaf_summary(const float4 *__restrict__ bodies, int b, int e /* inclusive */) {
    Summ<ORDER> s;
    float M = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    for (int i = b; i <= e; ++i) {
        const float4 p = bodies[i];
        M = fadd(M, p.w);
        cx = fadd(cx, fmul(p.w, p.x));
        cy = fadd(cy, fmul(p.w, p.y));
        cz = fadd(cz, fmul(p.w, p.z));
    }
    cx = fdiv(cx, M); cy = fdiv(cy, M); cz = fdiv(cz, M);
    s.com[0] = cx; s.com[1] = cy; s.com[2] = cz; s.M = M;
    if constexpr (ORDER >= 2) {
        // moments of order 2 (and 3) of each body about the centre of mass, times its mass
        constexpr int NQ = ORDER >= 3 ? 16 : 6;
        float acc[NQ];
#pragma unroll
        for (int k = 0; k < NQ; ++k) acc[k] = 0.f;
        auto term = [&](int i, float q[NQ]) {
            const float4 p = bodies[i];
            const float d[3] = {fsub(p.x, cx), fsub(p.y, cy), fsub(p.z, cz)};
            offset_quadrupole(d[0], d[1], d[2], p.w, q);
            if constexpr (ORDER >= 3) {
                const float t2[6] = {fmul(d[0], d[0]), fmul(d[0], d[1]), fmul(d[0], d[2]),
                                     fmul(d[1], d[1]), fmul(d[1], d[2]), fmul(d[2], d[2])};
                offset_octupole(t2, d, p.w, q + 6);
            }
        };
        int i = b;
        for (; e + 1 - i >= 4; i += 4) {
            float f0[NQ], f1[NQ], f2[NQ], f3[NQ];
            term(i, f0); term(i + 1, f1); term(i + 2, f2); term(i + 3, f3);
#pragma unroll
            for (int k = 0; k < NQ; ++k) acc[k] = fadd(acc[k], fadd(fadd(f0[k], f1[k]), fadd(f2[k], f3[k])));
        }
        for (; i <= e; ++i) {
            float f[NQ];
            term(i, f);
#pragma unroll
            for (int k = 0; k < NQ; ++k) acc[k] = fadd(acc[k], f[k]);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) s.q[k] = acc[k];
        if constexpr (ORDER >= 3) {
#pragma unroll
            for (int k = 0; k < 10; ++k) s.q3[k] = acc[6 + k];
        }
    }
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = b; i <= e; ++i) {
        const float4 p = bodies[i];
        mn[0] = gmin(p.x, mn[0]); mn[1] = gmin(p.y, mn[1]); mn[2] = gmin(p.z, mn[2]);
        mx[0] = gmax(p.x, mx[0]); mx[1] = gmax(p.y, mx[1]); mx[2] = gmax(p.z, mx[2]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) { s.bmin[k] = mn[k]; s.bmax[k] = mx[k]; }
    return s;
}

template<int ORDER>
__device__ Summ<ORDER> internal_summary(const Summ<ORDER> &a, const Summ<ORDER> &b) {
    Summ<ORDER> s;
    float M = fadd(fadd(0.f, a.M), b.M);
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) c[k] = fdiv(fadd(fadd(0.f, fmul(a.com[k], a.M)), fmul(b.com[k], b.M)), M);
    s.M = M;
#pragma unroll
    for (int k = 0; k < 3; ++k) s.com[k] = c[k];
    if constexpr (ORDER >= 2) {
        float qa[6], qb[6];
        offset_quadrupole(fsub(a.com[0], c[0]), fsub(a.com[1], c[1]), fsub(a.com[2], c[2]), a.M, qa);
        offset_quadrupole(fsub(b.com[0], c[0]), fsub(b.com[1], c[1]), fsub(b.com[2], c[2]), b.M, qb);
#pragma unroll
        for (int k = 0; k < 6; ++k) s.q[k] = fadd(fadd(0.f, fadd(qa[k], a.q[k])), fadd(qb[k], b.q[k]));
        if constexpr (ORDER >= 3) {
            // per child: (moment of the offset) * mass + child moment, plus sumOfOuterProducts(child
            // quadrupole, offset) (MultipoleMassSummary.h:63-73)
            float m3[2][10];
            const Summ<ORDER> *cs[2] = {&a, &b};
#pragma unroll
            for (int ci = 0; ci < 2; ++ci) {
                const Summ<ORDER> &ch = *cs[ci];
                const float d[3] = {fsub(ch.com[0], c[0]), fsub(ch.com[1], c[1]), fsub(ch.com[2], c[2])};
                const float t2[6] = {fmul(d[0], d[0]), fmul(d[0], d[1]), fmul(d[0], d[2]),
                                     fmul(d[1], d[1]), fmul(d[1], d[2]), fmul(d[2], d[2])};
                float o3[10], sop[10];
                offset_octupole(t2, d, ch.M, o3);
                sum_outer3(ch.q, d, sop);
#pragma unroll
                for (int k = 0; k < 10; ++k) m3[ci][k] = fadd(fadd(o3[k], ch.q3[k]), sop[k]);
            }
#pragma unroll
            for (int k = 0; k < 10; ++k) s.q3[k] = fadd(fadd(0.f, m3[0][k]), m3[1][k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s.bmin[k] = gmin(b.bmin[k], gmin(a.bmin[k], FLT_MAX));
        s.bmax[k] = gmax(b.bmax[k], gmax(a.bmax[k], -FLT_MAX));
    }
    return s;
}

// internal_summary's formulas (MultipoleMassSummary.h:37-97) evaluated in FP64 from the children's
// FP32 summaries and rounded once: the precision option for the top levels of the tree. The
// bounding box is exact in any precision (min / max do not round).
template<int ORDER>
__device__ Summ<ORDER> internal_summary_f64(const Summ<ORDER> &a, const Summ<ORDER> &b) {
    Summ<ORDER> s;
    const double M = (double) a.M + (double) b.M;
    double c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) c[k] = ((double) a.com[k] * (double) a.M + (double) b.com[k] * (double) b.M) / M;
    s.M = (float) M;
#pragma unroll
    for (int k = 0; k < 3; ++k) s.com[k] = (float) c[k];
    if constexpr (ORDER >= 2) {
        double q2[6] = {0, 0, 0, 0, 0, 0}, q3[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        const Summ<ORDER> *cs[2] = {&a, &b};
#pragma unroll
        for (int ci = 0; ci < 2; ++ci) {
            const Summ<ORDER> &ch = *cs[ci];
            const double m = ch.M;
            const double d[3] = {(double) ch.com[0] - c[0], (double) ch.com[1] - c[1], (double) ch.com[2] - c[2]};
            const double t2[6] = {d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]};
#pragma unroll
            for (int k = 0; k < 6; ++k) q2[k] += t2[k] * m + (double) ch.q[k];
            if constexpr (ORDER >= 3) {
#pragma unroll
                for (int L = 0; L < 10; ++L) {
                    int i[3];
                    dims3(L, i);
                    // (d (x) d (x) d) m + child octupole + sumOfOuterProducts(child quadrupole, d)
                    const double sop = (double) ch.q[slot2u(i[0], i[1])] * d[i[2]] +
                                       (double) ch.q[slot2u(i[1], i[2])] * d[i[0]] +
                                       (double) ch.q[slot2u(i[2], i[0])] * d[i[1]];
                    q3[L] += t2[slot2(i[0], i[1])] * d[i[2]] * m + (double) ch.q3[L] + sop;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) s.q[k] = (float) q2[k];
        if constexpr (ORDER >= 3) {
#pragma unroll
            for (int k = 0; k < 10; ++k) s.q3[k] = (float) q3[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s.bmin[k] = gmin(b.bmin[k], gmin(a.bmin[k], FLT_MAX));
        s.bmax[k] = gmax(b.bmax[k], gmax(a.bmax[k], -FLT_MAX));
    }
    return s;
}

// Smallest float b such that RN(a / b) < t, i.e. d2 >= b <=> the reference's
// diag^2 / d2 < theta^2 (DiagonalOverCenterDistance.h:18-22). RN(a / b) is monotone in b, so the
// threshold is exact; NaN means "never approximate" (every comparison with NaN is false).
__device__ float mac_threshold(float a, float t) {
    if (!(t > 0.f) || !(a >= 0.f) || isinf(a)) return __int_as_float(0x7fc00000);
    if (a == 0.f) return __int_as_float(1);  // 0 / b < t for every b > 0
    auto pred = [&](float b) { return fdiv(a, b) < t; };
    float b = fdiv(a, t);
    if (isinf(b)) b = FLT_MAX;
    if (pred(b)) {
        for (int k = 0; k < 64; ++k) {
            float pb = nextafterf(b, 0.f);
            if (pb > 0.f && pred(pb)) b = pb;
            else break;
        }
    } else {
        for (int k = 0; k < 64 && !pred(b); ++k) b = nextafterf(b, __int_as_float(0x7f800000));
    }
    return b;
}

template<int ORDER>
__device__ void write_record(const NodeArrays &nodes, int pre, const Summ<ORDER> &s, float t, int link0, int link1,
                             uint32_t *err) {
    if (pre < 0 || pre >= nodes.capacity) {
        atomicOr(err, (uint32_t) kErrNodeOverflow);
        return;
    }
    constexpr int PAY = NodeLayout<ORDER>::PAY;
    float cx = fdiv(fadd(s.bmax[0], s.bmin[0]), 2.0f);
    float cy = fdiv(fadd(s.bmax[1], s.bmin[1]), 2.0f);
    float cz = fdiv(fadd(s.bmax[2], s.bmin[2]), 2.0f);
    float dx = fsub(s.bmax[0], s.bmin[0]), dy = fsub(s.bmax[1], s.bmin[1]), dz = fsub(s.bmax[2], s.bmin[2]);
    float diag2 = fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
    nodes.mac[pre] = make_float4(cx, cy, cz, mac_threshold(diag2, t));
    nodes.link[pre] = make_int2(link0, link1);
    float4 *p = nodes.pay + (int64_t) pre * PAY;
    p[0] = make_float4(s.com[0], s.com[1], s.com[2], s.M);
    if constexpr (ORDER >= 2) {
        p[1] = make_float4(s.q[0], s.q[1], s.q[2], s.q[3]);
        // third slot: 1.5 * trace(Q), the traversal's quadrupole term uses it per interaction
        p[2] = make_float4(s.q[4], s.q[5], fmul(1.5f, fadd(fadd(s.q[0], s.q[3]), s.q[5])), 0.f);
    }
}

// The MAC threshold parameter of the node covering bodies [first, last], and the registration
// of an instance root (a node whose range is exactly one instance).
__device__ __forceinline__ float node_theta2(const BatchSegments &seg, float t, int first) {
    return seg.inst_theta2 ? seg.inst_theta2[seg.inst_of[first]] : t;
}
__device__ __forceinline__ void register_root(const BatchSegments &seg, int pre, int first, int last) {
    if (!seg.inst_root) return;
    const int k = seg.inst_of ? seg.inst_of[first] : 0;
    const int2 r = seg.inst_range[k];
    if (r.x == first && r.y == last) seg.inst_root[k] = pre;
}

// Smallest float s >= 0 with RN(sqrt(s)) >= b (sqrt is monotone, so the set is an up-set).
__device__ float sqrt_threshold(float b) {
    if (isnan(b)) return b;
    if (isinf(b)) return b;
    auto pred = [&](float v) { return __fsqrt_rn(v) >= b; };
    float v = fmul(b, b);
    if (isinf(v)) v = FLT_MAX;
    if (pred(v)) {
        for (int k = 0; k < 64; ++k) {
            const float pv = nextafterf(v, 0.f);
            if (pv >= 0.f && pv < v && pred(pv)) v = pv;
            else break;
        }
    } else {
        for (int k = 0; k < 64 && !pred(v); ++k) v = nextafterf(v, __int_as_float(0x7f800000));
    }
    return v;
}

// Dual-tree node arrays (order 3 summaries): bounding box, centre of mass and mass, packed
// quadrupole and octupole, links, and the criterion thresholds for theta.
__device__ void write_dual_record(const DualNodes &nodes, int pre, const Summ<3> &s, int first, int last,
                                  int link0, int link1, float theta, uint32_t *err) {
    if (pre < 0 || pre >= nodes.capacity) {
        atomicOr(err, (uint32_t) kErrNodeOverflow);
        return;
    }
    // diagonal length as BoundingBox::diagonalLength: sqrt((dx*dx + dy*dy) + dz*dz), IEEE operations
    const float dx = fsub(s.bmax[0], s.bmin[0]), dy = fsub(s.bmax[1], s.bmin[1]), dz = fsub(s.bmax[2], s.bmin[2]);
    const float diag = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
    nodes.bmin[pre] = make_float4(s.bmin[0], s.bmin[1], s.bmin[2], __int_as_float(last - first + 1));
    nodes.bmax[pre] = make_float4(s.bmax[0], s.bmax[1], s.bmax[2], diag);
    // DiagonalOverSeparation (DiagonalOverSeparation.h:29-49): RN(diag / sep) < theta for the
    // active node, RN(RN(3 diag) / sep) < theta for the passive node
    const float b_near = mac_threshold(diag, theta), b_far = mac_threshold(fmul(3.0f, diag), theta);
    nodes.thr[pre] = make_float4(b_near, sqrt_threshold(b_near), b_far, sqrt_threshold(b_far));
    nodes.com[pre] = make_float4(s.com[0], s.com[1], s.com[2], s.M);
    float4 *q = nodes.q + (int64_t) pre * 4;
    q[0] = make_float4(s.q[0], s.q[1], s.q[2], s.q[3]);
    q[1] = make_float4(s.q[4], s.q[5], s.q3[0], s.q3[1]);
    q[2] = make_float4(s.q3[2], s.q3[3], s.q3[4], s.q3[5]);
    q[3] = make_float4(s.q3[6], s.q3[7], s.q3[8], s.q3[9]);
    nodes.link[pre] = make_int2(link0, link1);
}

__device__ __forceinline__ int slot_of(int c, int n) { return c >= 0 ? c : (n - 1) + ~c; }

// Arrival counter of the bottom-up climb with release-acquire ordering: the caller's summary
// stores are visible before its arrival, and the second arriver sees the first one's stores.
__device__ __forceinline__ int arrive_acq_rel(int *p) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
    return old;
}

// Node record writers of the two node formats, called by the thread that finishes a node.
template<int ORDER>
struct BhRecords {
    NodeArrays nodes;
    float t;  // RN(theta * theta)
    BatchSegments seg;
    __device__ void leaf(int pre, const Summ<ORDER> &s, int first, int last, uint32_t *err) const {
        write_record<ORDER>(nodes, pre, s, node_theta2(seg, t, first), first, last + 1, err);
        register_root(seg, pre, first, last);
    }
    __device__ void internal(int pre, const Summ<ORDER> &s, int first, int last, int right_pre, uint32_t *err) const {
        write_record<ORDER>(nodes, pre, s, node_theta2(seg, t, first), right_pre, -1, err);
        register_root(seg, pre, first, last);
    }
};

struct DualRecords {
    DualNodes nodes;
    float theta;
    __device__ void leaf(int pre, const Summ<3> &s, int first, int last, uint32_t *err) const {
        write_dual_record(nodes, pre, s, first, last, first, last + 1, theta, err);
    }
    __device__ void internal(int pre, const Summ<3> &s, int first, int last, int right_pre, uint32_t *err) const {
        write_dual_record(nodes, pre, s, first, last, right_pre, -1 - first, theta, err);
    }
};

// Summary of a final internal node covering bodies [first, last] from its children's.
template<int ORDER>
__device__ __forceinline__ Summ<ORDER> combine(const TreeWorkspace &tw, const Summ<ORDER> &l, const Summ<ORDER> &r,
                                               int first, int last) {
    return (tw.fp64_min_bodies > 0 && last - first + 1 >= tw.fp64_min_bodies) ? internal_summary_f64<ORDER>(l, r)
                                                                              : internal_summary<ORDER>(l, r);
}

// Final internal node i's final-leaf children: leaf summaries and records, then the climb. A node
// whose children are both final leaves is finished at once, without an arrival. The topology of
// the next node up is loaded while the current level computes, so a level waits for its arrival
// and the sibling's summary only.
template<int ORDER, class Records>
__device__ void summarize_from(const float4 *__restrict__ bodies, int n, const TreeWorkspace &tw, uint32_t *err,
                               const Records &rec, int i) {
    int4 tp = tw.topo[i];  // (left child, right child, first body, last body) of the node p below
    uint8_t fl = tw.flags[i];
    int par = tw.parent[i];  // not written for the root, and read only below a non-root node
    const int gamma = tp.x >= 0 ? tp.x : ~tp.x;  // the left child's last body
    Summ<ORDER> mine;
    int from, p, chain_from;  // the finished child and its chain (-1: a leaf), the node above it
    if ((fl & kLeftLeaf) && (fl & kRightLeaf)) {
        const Summ<ORDER> l = leaf_summary<ORDER>(bodies, tp.z, gamma);
        const Summ<ORDER> r = leaf_summary<ORDER>(bodies, gamma + 1, tp.w);
        rec.leaf(preorder_leaf(tw, tp.z), l, tp.z, gamma, err);
        const int right_pre = preorder_leaf(tw, gamma + 1);
        rec.leaf(right_pre, r, gamma + 1, tp.w, err);
        mine = combine<ORDER>(tw, l, r, tp.z, tp.w);
        store_slot<ORDER>(tw, i, mine);
        tw.chain[i] = 0;
        rec.internal(preorder_internal(tw, tp.z, 0), mine, tp.z, tp.w, right_pre, err);
        if (i == 0) return;
        from = i;
        chain_from = 0;
        p = par;
        if (p < 0 || p >= n - 1) {
            atomicOr(err, (uint32_t) kErrTreeDepth);
            return;
        }
        tp = tw.topo[p];
        fl = tw.flags[p];
        par = tw.parent[p];
    } else {
        const bool left = (fl & kLeftLeaf) != 0;  // exactly one child is a final leaf
        const int b = left ? tp.z : gamma + 1, e = left ? gamma : tp.w;
        mine = leaf_summary<ORDER>(bodies, b, e);
        from = left ? tp.x : tp.y;
        store_slot<ORDER>(tw, slot_of(from, n), mine);
        rec.leaf(preorder_leaf(tw, b), mine, b, e, err);
        chain_from = -1;
        p = i;
    }
    for (int level = 0;; ++level) {
        if (level >= kMaxTreeDepth || p < 0 || p >= n - 1) {
            atomicOr(err, (uint32_t) kErrTreeDepth);
            return;
        }
        if (arrive_acq_rel(&tw.visit[p]) == 0) return;  // the sibling's thread finishes p
        const int lc = tp.x, rc = tp.y;
        const bool from_left = (lc == from);
        const bool lfin = (fl & kLeftLeaf) != 0, rfin = (fl & kRightLeaf) != 0;
        const int sib = from_left ? rc : lc;
        const Summ<ORDER> other = load_slot<ORDER>(tw, slot_of(sib, n));
        const int sib_chain = (from_left ? rfin : lfin) ? -1 : __ldcg(tw.chain + sib);
        int4 ntp = make_int4(0, 0, 0, 0);
        uint8_t nfl = 0;
        int npar = -1;
        if (p != 0 && par >= 0 && par < n - 1) {
            ntp = tw.topo[par];
            nfl = tw.flags[par];
            npar = tw.parent[par];
        }
        const Summ<ORDER> up = from_left ? combine<ORDER>(tw, mine, other, tp.z, tp.w)
                                         : combine<ORDER>(tw, other, mine, tp.z, tp.w);
        store_slot<ORDER>(tw, p, up);
        // final internal nodes below p that share its first body: its left child's chain
        const int lchain = lfin ? -1 : (from_left ? chain_from : sib_chain);
        const int rchain = rfin ? -1 : (from_left ? sib_chain : chain_from);
        const int ch = lchain + 1;
        tw.chain[p] = ch;
        const int rfirst = (lc >= 0 ? lc : ~lc) + 1;
        const int right_pre = rfin ? preorder_leaf(tw, rfirst) : preorder_internal(tw, rfirst, rchain);
        rec.internal(preorder_internal(tw, tp.z, ch), up, tp.z, tp.w, right_pre, err);
        if (p == 0) return;
        mine = up;
        chain_from = ch;
        from = p;
        p = par;
        tp = ntp;
        fl = nfl;
        par = npar;
    }
}

// One thread per final internal node with leaf children (the compact list karras_kernel built), on
// a grid of a few waves at most.
template<int ORDER, class Records>
__global__ void __launch_bounds__(kThreads) summarize_kernel(const float4 *__restrict__ bodies, int n, TreeWorkspace tw,
                                                             uint32_t *err, Records rec) {
    const int count = *tw.leaf_parents_count;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x)
        summarize_from<ORDER, Records>(bodies, n, tw, err, rec, tw.leaf_parents[idx]);
}

__global__ void root_leaf_dual_kernel(const float4 *__restrict__ bodies, int n, TreeWorkspace tw, DualNodes nodes,
                                      float theta, uint32_t *err) {
    if (n > 1 && (tw.flags[0] & kFinal)) return;
    write_dual_record(nodes, 0, leaf_summary<3>(bodies, 0, n - 1), 0, n - 1, 0, n, theta, err);
    *tw.num_nodes = 1;
}

// The whole tree is one leaf when n == 1, or when the root is not splittable (n <= maxLeafSize
// or every code equal).
template<int ORDER>
__global__ void root_leaf_kernel(const float4 *__restrict__ bodies, int n, TreeWorkspace tw, float t,
                                 NodeArrays nodes, uint32_t *err, BatchSegments seg) {
    if (n > 1 && (tw.flags[0] & kFinal)) return;
    write_record<ORDER>(nodes, 0, leaf_summary<ORDER>(bodies, 0, n - 1), node_theta2(seg, t, 0), 0, n, err);
    register_root(seg, 0, 0, n - 1);
    *tw.num_nodes = 1;
}

// Grid of the summary climb: enough threads for every possible leaf parent, capped at a few waves
// (the kernel loops over the compact list).
int summarize_blocks(int n) {
    const int64_t need = ((int64_t) n - 1 + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t) current_sm_count() * 8;
    return (int) std::max<int64_t>(1, std::min(need, cap));
}

// Karras topology, the final nodes per start position and their exclusive prefix (which also
// gives the node count); the topology kernel also clears the climb's arrival counters.
void launch_topology(const uint64_t *sorted_codes, const int *inst_of, int n, int leaf, TreeWorkspace &tw,
                     cudaStream_t s) {
    const int internal = n - 1;
    const int blocks = (internal + kThreads - 1) / kThreads;
    const int64_t m = (int64_t) n + 1;
    const int tiles = (int) build_scan_tiles(n);
    cudaMemsetAsync(tw.start, 0, (size_t) m * sizeof(int), s);
    cudaMemsetAsync(tw.leaf_parents_count, 0, sizeof(int), s);
    karras_kernel<<<blocks, kThreads, 0, s>>>(sorted_codes, inst_of, n, leaf, tw);
    scan_tiles_kernel<<<tiles, kThreads, 0, s>>>(tw.start, m, tw.scan_part);
    scan_parts_kernel<<<1, 1024, 0, s>>>(tw.scan_part, tiles, tw.num_nodes);
    scan_apply_kernel<<<tiles, kThreads, 0, s>>>(tw.start, m, tw.scan_part, tw.pre_base);
}

}  // namespace

int64_t build_scan_tiles(int64_t n) { return (n + 1 + kScanTile - 1) / kScanTile; }

void launch_build_dual_tree(const uint64_t *sorted_codes, const float4 *bodies, int64_t n64, int leaf, float theta,
                            TreeWorkspace &tw, const DualNodes &nodes, uint32_t *err, cudaStream_t s) {
    const int n = (int) n64;
    if (n <= 0) {
        cudaMemsetAsync(tw.num_nodes, 0, sizeof(int), s);
        return;
    }
    if (n > 1) {
        launch_topology(sorted_codes, nullptr, n, leaf, tw, s);
        summarize_kernel<3, DualRecords>
            <<<summarize_blocks(n), kThreads, 0, s>>>(bodies, n, tw, err, DualRecords{nodes, theta});
    }
    root_leaf_dual_kernel<<<1, 1, 0, s>>>(bodies, n, tw, nodes, theta, err);
}

void launch_build_tree(const uint64_t *sorted_codes, const float4 *bodies, int64_t n64, int leaf, int order,
                       float theta, TreeWorkspace &tw, const NodeArrays &nodes, uint32_t *err, cudaStream_t s,
                       const BatchSegments &seg) {
    const int n = (int) n64;
    if (n <= 0) {
        cudaMemsetAsync(tw.num_nodes, 0, sizeof(int), s);
        return;
    }
    const float t = theta * theta;  // the reference compares against theta * theta in float
    if (n > 1) launch_topology(sorted_codes, seg.inst_of, n, leaf, tw, s);
    if (order == 1) {
        if (n > 1)
            summarize_kernel<1, BhRecords<1>>
                <<<summarize_blocks(n), kThreads, 0, s>>>(bodies, n, tw, err, BhRecords<1>{nodes, t, seg});
        root_leaf_kernel<1><<<1, 1, 0, s>>>(bodies, n, tw, t, nodes, err, seg);
    } else {
        if (n > 1)
            summarize_kernel<2, BhRecords<2>>
                <<<summarize_blocks(n), kThreads, 0, s>>>(bodies, n, tw, err, BhRecords<2>{nodes, t, seg});
        root_leaf_kernel<2><<<1, 1, 0, s>>>(bodies, n, tw, t, nodes, err, seg);
    }
}

}  // namespace nbg
