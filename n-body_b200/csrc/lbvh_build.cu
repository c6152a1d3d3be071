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
//   karras_kernel     one thread per Karras internal node: range, split, children, parent,
//                     splittable flag (reads ~2 log n codes per node, L2-resident)
//   summarize_kernel  one thread per final internal node with leaf children: sequential leaf
//                     summaries over the leaf's bodies, then an atomic climb in which the second
//                     child to arrive summarises the parent (CenterOfMassSummary.h:30-55,
//                     BoundingBoxSummary.h:30-68, MultipoleMassSummary.h:37-97; the leaf moment
//                     sum follows libstdc++'s 4-way std::transform_reduce). All float operations
//                     are single IEEE operations in the reference's order, so summaries are
//                     bit-identical to the CPU restatement.
//   emit_kernel       preorder index of every final node (walk to the root adding left-sibling
//                     subtree sizes) and the node arrays the traversal reads: MAC data (centre and
//                     exact MAC threshold), links (right child / leaf body range) and payload
//                     (centre of mass, mass, quadrupole).
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

__global__ void __launch_bounds__(kThreads) karras_kernel(const uint64_t *__restrict__ codes,
                                                          const int *__restrict__ inst_of, int n, int leaf,
                                                          int2 *__restrict__ range, int *__restrict__ left,
                                                          int *__restrict__ right, int *__restrict__ parent,
                                                          uint8_t *__restrict__ splittable) {
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
    left[i] = lc;
    right[i] = rc;
    range[i] = make_int2(first, last);
    if (lc >= 0) parent[lc] = i;
    if (rc >= 0) parent[rc] = i;
    // A node spanning several instances only connects their trees: it is always split.
    const bool spans = inst_of && inst_of[first] != inst_of[last];
    splittable[i] = (uint8_t) (spans || ((last - first + 1 > leaf) && (codes[first] != codes[last])));
}

template<int ORDER>
struct Summ {
    float bmin[3], bmax[3], com[3], M;
    float q[6];
};

template<int ORDER>
__device__ __forceinline__ void store_slot(const TreeWorkspace &tw, int slot, const Summ<ORDER> &s) {
    tw.sbmin[slot] = make_float4(s.bmin[0], s.bmin[1], s.bmin[2], 0.f);
    tw.sbmax[slot] = make_float4(s.bmax[0], s.bmax[1], s.bmax[2], 0.f);
    tw.scom[slot] = make_float4(s.com[0], s.com[1], s.com[2], s.M);
    if constexpr (ORDER >= 2) {
        tw.sq0[slot] = make_float4(s.q[0], s.q[1], s.q[2], s.q[3]);
        tw.sq1[slot] = make_float4(s.q[4], s.q[5], 0.f, 0.f);
    }
}

// Loads bypass L1: the slot may have been written by another block moments ago.
template<int ORDER>
__device__ __forceinline__ Summ<ORDER> load_slot(const TreeWorkspace &tw, int slot) {
    Summ<ORDER> s;
    float4 a = __ldcg(tw.sbmin + slot), b = __ldcg(tw.sbmax + slot), c = __ldcg(tw.scom + slot);
    s.bmin[0] = a.x; s.bmin[1] = a.y; s.bmin[2] = a.z;
    s.bmax[0] = b.x; s.bmax[1] = b.y; s.bmax[2] = b.z;
    s.com[0] = c.x; s.com[1] = c.y; s.com[2] = c.z; s.M = c.w;
    if constexpr (ORDER >= 2) {
        float4 q0 = __ldcg(tw.sq0 + slot), q1 = __ldcg(tw.sq1 + slot);
        s.q[0] = q0.x; s.q[1] = q0.y; s.q[2] = q0.z; s.q[3] = q0.w; s.q[4] = q1.x; s.q[5] = q1.y;
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
        float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        auto term = [&](int i, float q[6]) {
            const float4 p = bodies[i];
            offset_quadrupole(fsub(p.x, cx), fsub(p.y, cy), fsub(p.z, cz), p.w, q);
        };
        int i = b;
        for (; e + 1 - i >= 4; i += 4) {
            float f0[6], f1[6], f2[6], f3[6];
            term(i, f0); term(i + 1, f1); term(i + 2, f2); term(i + 3, f3);
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[k] = fadd(acc[k], fadd(fadd(f0[k], f1[k]), fadd(f2[k], f3[k])));
        }
        for (; i <= e; ++i) {
            float f[6];
            term(i, f);
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[k] = fadd(acc[k], f[k]);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) s.q[k] = acc[k];
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
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s.bmin[k] = gmin(b.bmin[k], gmin(a.bmin[k], FLT_MAX));
        s.bmax[k] = gmax(b.bmax[k], gmax(a.bmax[k], -FLT_MAX));
    }
    return s;
}

__device__ __forceinline__ bool is_final_leaf(const uint8_t *splittable, int c) { return c < 0 || !splittable[c]; }
__device__ __forceinline__ int slot_of(int c, int n) { return c >= 0 ? c : (n - 1) + ~c; }

template<int ORDER>
__global__ void __launch_bounds__(kThreads) summarize_kernel(const float4 *__restrict__ bodies, int n, TreeWorkspace tw,
                                                             uint32_t *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1 || !tw.splittable[i]) return;
    for (int side = 0; side < 2; ++side) {
        const int c = side ? tw.right[i] : tw.left[i];
        if (!is_final_leaf(tw.splittable, c)) continue;
        int b, e;
        if (c < 0) { b = e = ~c; } else { int2 r = tw.range[c]; b = r.x; e = r.y; }
        const int slot = slot_of(c, n);
        store_slot<ORDER>(tw, slot, leaf_summary<ORDER>(bodies, b, e));
        tw.cnt[slot] = 1;
        int p = i;
        for (int level = 0;; ++level) {
            if (level >= kMaxTreeDepth || p < 0 || p >= n - 1) {
                atomicOr(err, (uint32_t) kErrTreeDepth);
                break;
            }
            __threadfence();
            if (atomicAdd(&tw.visit[p], 1) == 0) break;  // the sibling's thread finishes p
            __threadfence();
            const int sl = slot_of(tw.left[p], n), sr = slot_of(tw.right[p], n);
            store_slot<ORDER>(tw, p, internal_summary<ORDER>(load_slot<ORDER>(tw, sl), load_slot<ORDER>(tw, sr)));
            tw.cnt[p] = 1 + __ldcg(tw.cnt + sl) + __ldcg(tw.cnt + sr);
            if (p == 0) break;
            p = tw.parent[p];
        }
    }
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

template<int ORDER>
__global__ void __launch_bounds__(kThreads) emit_kernel(int n, TreeWorkspace tw, float t, NodeArrays nodes,
                                                        uint32_t *err, BatchSegments seg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1 || !tw.splittable[i]) return;
    int pre = 0;
    int depth = 0;
    for (int u = i; u != 0; ++depth) {
        const int p = tw.parent[u];
        if (depth >= kMaxTreeDepth || p < 0 || p >= n - 1) {
            atomicOr(err, (uint32_t) kErrTreeDepth);
            return;
        }
        pre += 1;
        if (tw.right[p] == u) pre += tw.cnt[slot_of(tw.left[p], n)];
        u = p;
    }
    const int lc = tw.left[i], rc = tw.right[i];
    const int lslot = slot_of(lc, n);
    const int right_pre = pre + 1 + tw.cnt[lslot];
    const int2 ri = tw.range[i];
    write_record<ORDER>(nodes, pre, load_slot<ORDER>(tw, i), node_theta2(seg, t, ri.x), right_pre, -1, err);
    register_root(seg, pre, ri.x, ri.y);
    if (is_final_leaf(tw.splittable, lc)) {
        int2 r = lc < 0 ? make_int2(~lc, ~lc) : tw.range[lc];
        write_record<ORDER>(nodes, pre + 1, load_slot<ORDER>(tw, lslot), node_theta2(seg, t, r.x), r.x, r.y + 1, err);
        register_root(seg, pre + 1, r.x, r.y);
    }
    if (is_final_leaf(tw.splittable, rc)) {
        int2 r = rc < 0 ? make_int2(~rc, ~rc) : tw.range[rc];
        write_record<ORDER>(nodes, right_pre, load_slot<ORDER>(tw, slot_of(rc, n)), node_theta2(seg, t, r.x), r.x,
                            r.y + 1, err);
        register_root(seg, right_pre, r.x, r.y);
    }
    if (i == 0) *tw.num_nodes = tw.cnt[i];
}

// The whole tree is one leaf when n == 1, or when the root is not splittable (n <= maxLeafSize
// or every code equal).
template<int ORDER>
__global__ void root_leaf_kernel(const float4 *__restrict__ bodies, int n, TreeWorkspace tw, float t,
                                 NodeArrays nodes, uint32_t *err, BatchSegments seg) {
    if (n > 1 && tw.splittable[0]) return;
    write_record<ORDER>(nodes, 0, leaf_summary<ORDER>(bodies, 0, n - 1), node_theta2(seg, t, 0), 0, n, err);
    register_root(seg, 0, 0, n - 1);
    *tw.num_nodes = 1;
}

}  // namespace

void launch_build_tree(const uint64_t *sorted_codes, const float4 *bodies, int64_t n64, int leaf, int order,
                       float theta, TreeWorkspace &tw, const NodeArrays &nodes, uint32_t *err, cudaStream_t s,
                       const BatchSegments &seg) {
    const int n = (int) n64;
    if (n <= 0) {
        cudaMemsetAsync(tw.num_nodes, 0, sizeof(int), s);
        return;
    }
    const float t = theta * theta;  // the reference compares against theta * theta in float
    const int internal = n - 1;
    const int blocks = internal > 0 ? (internal + kThreads - 1) / kThreads : 1;
    if (internal > 0) {
        karras_kernel<<<blocks, kThreads, 0, s>>>(sorted_codes, seg.inst_of, n, leaf, tw.range, tw.left, tw.right,
                                                  tw.parent, tw.splittable);
        cudaMemsetAsync(tw.visit, 0, (size_t) internal * sizeof(int), s);
    }
    if (order == 1) {
        if (internal > 0) {
            summarize_kernel<1><<<blocks, kThreads, 0, s>>>(bodies, n, tw, err);
            emit_kernel<1><<<blocks, kThreads, 0, s>>>(n, tw, t, nodes, err, seg);
        }
        root_leaf_kernel<1><<<1, 1, 0, s>>>(bodies, n, tw, t, nodes, err, seg);
    } else {
        if (internal > 0) {
            summarize_kernel<2><<<blocks, kThreads, 0, s>>>(bodies, n, tw, err);
            emit_kernel<2><<<blocks, kThreads, 0, s>>>(n, tw, t, nodes, err, seg);
        }
        root_leaf_kernel<2><<<1, 1, 0, s>>>(bodies, n, tw, t, nodes, err, seg);
    }
}

}  // namespace nbg
