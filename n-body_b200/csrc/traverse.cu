// Barnes-Hut traversal of the preorder linear BVH for groups of 32 Morton-adjacent targets, one
// warp per group, in a persistent grid.
//
// Semantics are those of Descent::activeTree (src/NBody/Simulation/Solvers/Descent/activeTree.h:24-79)
// under DiagonalOverCenterDistance (DiagonalOverCenterDistance.h:18-22) with the Gravity rule
// (src/NBody/Physics/Rules/Gravity.h:199-259), decided per target: a node is approximated for a
// target iff diag^2 / |centre - p|^2 < theta^2 (the node carries the exact threshold on
// |centre - p|^2, and squared distances are formed in the reference's IEEE operation order), an
// opened leaf interacts pairwise with all its bodies, otherwise the children are visited. Every
// target therefore takes exactly the reference's decisions, and the interaction counts equal the
// reference's SimpleTrackingRule counts.
//
// Work organisation (per warp, 32 targets, 32-bit target masks):
//   1. Chunked traversal: up to 32 (node, mask) entries are popped from the warp's stack, one per
//      lane. Each lane classifies its node against the bounding box of the group's targets:
//        accept-all  if even the box point nearest the centre passes the MAC,
//        open-all    if even the farthest box corner fails it,
//        mixed       otherwise.
//      Rounding is monotone, so the rounded squared distance of every target lies between the
//      nearest and farthest values computed with the same operation sequence: the group decision
//      is exact for every target, not a heuristic.
//   2. Mixed nodes are batched and resolved lane-parallel: each lane takes one node and tests the
//      32 targets (broadcast from shared memory), producing accept and open masks.
//   3. Nodes accepted by every target go to a shared list evaluated by all lanes with broadcast
//      loads; nodes accepted by some targets only go to per-target private lists in shared memory,
//      evaluated target-major (each lane walks its own list). Opened leaves go to a (leaf, mask)
//      list evaluated with broadcast body loads. Opened internal nodes push both children.
// The expensive terms thus run without traversal bookkeeping between them, and the per-node
// traversal cost is spread over 32 nodes per instruction.
//
// Arithmetic: FP32, one MUFU rsqrt per interaction, G applied once per target. Pair term:
// 20 flops by the usual direct-sum convention (12 FP32 instructions + rsqrt). Quadrupole node
// term (non-traceless moments about the centre of mass, Gravity.h:239-259, with D<3> contracted
// analytically: (D3:Q)_i = g3 R_i (R.Q.R) + g2 (2 (Q R)_i + R_i tr Q)): 56 flops.
#include <algorithm>
#include <cfloat>
#include <climits>

#include "nb_internal.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kList = 64;          // capacity of each per-warp list; rounds append at most 32
// Stack: kTraverseStack entries per warp. No bound below that size is proven for every tree, so a
// round whose pushes would not fit abandons its group and sets kErrStackOverflow (the host turns it
// into an error); every entry on the stack has been written, so no stale entry is ever popped.
constexpr int kPriv = 32;          // per-target private list of partially accepted nodes
constexpr unsigned kFull = 0xffffffffu;

enum : int { kNone = 0, kAcceptAll = 1, kOpenAll = 2, kMixed = 3 };

struct WarpLists {
    float4 tpos[32];
    int approx_node[kList];       // nodes accepted by every target of the group
    int pp_begin[kList], pp_end[kList];
    uint32_t pp_mask[kList];
    int mixed_node[kList];
    uint32_t mixed_mask[kList];
    int priv[kPriv][32];          // [slot][lane]: nodes accepted by some targets only
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Squared distance in the reference's IEEE order: (dx*dx + dy*dy) + dz*dz, d = p - c.
__device__ __forceinline__ float ref_dist2(float px, float py, float pz, float4 c) {
    const float dx = fsub(px, c.x), dy = fsub(py, c.y), dz = fsub(pz, c.z);
    return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
}

template<bool EPS0>
__device__ __forceinline__ void pair_term(float4 p, float4 b, float eps, float &ax, float &ay, float &az) {
    const float rx = p.x - b.x, ry = p.y - b.y, rz = p.z - b.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps)));
    if (EPS0 && r2 == 0.f) return;  // equal positions contribute nothing (Gravity.h:203)
    const float inv = rsqrtf(r2);
    const float s = b.w * (inv * inv * inv);
    ax = fmaf(-rx, s, ax);
    ay = fmaf(-ry, s, ay);
    az = fmaf(-rz, s, az);
}

template<bool EPS0>
__device__ __forceinline__ void quad_term(float4 p, float4 com, float4 q0, float4 q1, float eps, float &ax,
                                          float &ay, float &az) {
    const float rx = p.x - com.x, ry = p.y - com.y, rz = p.z - com.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps)));
    if (EPS0 && r2 == 0.f) return;
    const float inv = rsqrtf(r2);
    const float inv2 = inv * inv;
    const float inv3 = inv2 * inv;
    const float inv5 = inv3 * inv2;
    const float inv7 = inv5 * inv2;
    const float qx = fmaf(q0.x, rx, fmaf(q0.y, ry, q0.z * rz));
    const float qy = fmaf(q0.y, rx, fmaf(q0.w, ry, q1.x * rz));
    const float qz = fmaf(q0.z, rx, fmaf(q1.x, ry, q1.y * rz));
    const float rqr = fmaf(rx, qx, fmaf(ry, qy, rz * qz));
    // q1.z holds 1.5 * (Qxx + Qyy + Qzz), precomputed per node
    const float sr = fmaf(-7.5f * inv7, rqr, fmaf(inv5, q1.z, -com.w * inv3));
    const float sq = 3.0f * inv5;
    ax = fmaf(rx, sr, fmaf(qx, sq, ax));
    ay = fmaf(ry, sr, fmaf(qy, sq, ay));
    az = fmaf(rz, sr, fmaf(qz, sq, az));
}

// Warp-wide ordered append: returns this lane's slot (valid where pred) and advances count.
__device__ __forceinline__ int warp_append(bool pred, int &count, uint32_t lt) {
    const uint32_t b = __ballot_sync(kFull, pred);
    const int pos = count + __popc(b & lt);
    count += __popc(b);
    return pos;
}

template<int ORDER, bool EPS0>
__device__ __forceinline__ void node_term(const float4 *__restrict__ pay, int c, float4 p, float eps, float &ax,
                                          float &ay, float &az) {
    constexpr int PAY = NodeLayout<ORDER>::PAY;
    const float4 *pc = pay + (int64_t) c * PAY;
    if constexpr (ORDER == 1) {
        pair_term<EPS0>(p, __ldg(pc), eps, ax, ay, az);
    } else {
        quad_term<EPS0>(p, __ldg(pc), __ldg(pc + 1), __ldg(pc + 2), eps, ax, ay, az);
    }
}

// Nodes accepted by the whole group: every lane evaluates every entry (broadcast loads).
template<int ORDER, bool EPS0>
__device__ __forceinline__ void flush_approx(WarpLists &L, int &napprox, const float4 *__restrict__ pay, float4 p,
                                             float eps, float &ax, float &ay, float &az, unsigned &cnp) {
    int j = 0;
    for (; j + 1 < napprox; j += 2) {
        const int c0 = L.approx_node[j], c1 = L.approx_node[j + 1];
        node_term<ORDER, EPS0>(pay, c0, p, eps, ax, ay, az);
        node_term<ORDER, EPS0>(pay, c1, p, eps, ax, ay, az);
    }
    if (j < napprox) node_term<ORDER, EPS0>(pay, L.approx_node[j], p, eps, ax, ay, az);
    cnp += (unsigned) napprox;
    napprox = 0;
    __syncwarp();
}

// Nodes accepted by some targets only: each lane walks its own list (target-major).
template<int ORDER, bool EPS0>
__device__ __forceinline__ void flush_private(WarpLists &L, int &npriv, const float4 *__restrict__ pay, float4 p,
                                              float eps, int lane, float &ax, float &ay, float &az, unsigned &cnp) {
    const int most = __reduce_max_sync(kFull, npriv);
    for (int k = 0; k < most; ++k) {
        if (k < npriv) node_term<ORDER, EPS0>(pay, L.priv[k][lane], p, eps, ax, ay, az);
    }
    cnp += (unsigned) npriv;
    npriv = 0;
    __syncwarp();
}

// Partially accepted entries (node c_i with target mask A_i in lane i) go to the private lists
// of the targets in A_i; a full list is evaluated before it would overflow.
template<int ORDER, bool EPS0>
__device__ __forceinline__ void append_private(WarpLists &L, int &npriv, bool partial, int c, uint32_t A,
                                               const float4 *__restrict__ pay, float4 p, float eps, int lane,
                                               float &ax, float &ay, float &az, unsigned &cnp) {
    uint32_t pend = __ballot_sync(kFull, partial);
    while (pend) {
        const int src = __ffs(pend) - 1;
        pend &= pend - 1;
        const int node = __shfl_sync(kFull, c, src);
        const uint32_t mask = __shfl_sync(kFull, A, src);
        if (__any_sync(kFull, npriv == kPriv)) flush_private<ORDER, EPS0>(L, npriv, pay, p, eps, lane, ax, ay, az, cnp);
        if ((mask >> lane) & 1u) L.priv[npriv++][lane] = node;
    }
    __syncwarp();
}

template<bool EPS0>
__device__ __forceinline__ void flush_pp(WarpLists &L, int &npp, const float4 *__restrict__ bodies, float4 p,
                                         float eps, int lane, float &ax, float &ay, float &az, unsigned &cpp) {
    for (int j = 0; j < npp; ++j) {
        const int b = L.pp_begin[j], e = L.pp_end[j];
        const bool on = (L.pp_mask[j] >> lane) & 1u;
        int k = b;
        for (; k + 3 < e; k += 4) {
            const float4 s0 = __ldg(bodies + k), s1 = __ldg(bodies + k + 1);
            const float4 s2 = __ldg(bodies + k + 2), s3 = __ldg(bodies + k + 3);
            if (on) {
                pair_term<EPS0>(p, s0, eps, ax, ay, az);
                pair_term<EPS0>(p, s1, eps, ax, ay, az);
                pair_term<EPS0>(p, s2, eps, ax, ay, az);
                pair_term<EPS0>(p, s3, eps, ax, ay, az);
            }
        }
        for (; k < e; ++k) {
            const float4 s0 = __ldg(bodies + k);
            if (on) pair_term<EPS0>(p, s0, eps, ax, ay, az);
        }
        if (on) cpp += (unsigned) (e - b);
    }
    npp = 0;
    __syncwarp();
}

template<int ORDER, bool EPS0>
__global__ void __launch_bounds__(kThreads) bh_kernel(NodeArrays nodes, const int *__restrict__ num_nodes_p,
                                                      const float4 *__restrict__ bodies, int n_bodies,
                                                      const float4 *__restrict__ targets, int n_targets, float G,
                                                      float eps, float4 *__restrict__ acc,
                                                      unsigned long long *__restrict__ counts,
                                                      int2 *__restrict__ stack_base, unsigned *__restrict__ group_counter,
                                                      uint32_t *__restrict__ err, const int4 *__restrict__ groups,
                                                      int num_group_tasks, const int *__restrict__ inst_root,
                                                      unsigned long long *__restrict__ inst_counts) {
    __shared__ WarpLists lists[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpLists &L = lists[warp];
    int2 *stack = stack_base + ((int64_t) blockIdx.x * kWarps + warp) * kTraverseStack;
    const float4 *__restrict__ mac = nodes.mac;
    const int2 *__restrict__ link = nodes.link;
    const float4 *__restrict__ pay = nodes.pay;
    const int num_nodes = *num_nodes_p;
    const int num_groups = groups ? num_group_tasks : (n_targets + 31) / 32;
    const uint32_t lt = lanemask_lt();
    // A valid tree needs fewer chunk rounds than it has nodes for one group; the cap only bounds
    // the work on a corrupted tree.
    const int64_t round_limit = 4 * (int64_t) num_nodes + 64;
    unsigned cpp = 0, cnp = 0;

    while (true) {
        int g = 0;
        if (lane == 0) g = (int) atomicAdd(group_counter, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= num_groups) break;
        int first = g * 32, count = min(32, n_targets - g * 32), root = 0, inst = -1;
        if (groups) {
            const int4 ge = groups[g];
            first = ge.x;
            count = ge.y;
            inst = ge.z;
            root = inst_root[inst];
        }
        const int i = first + lane;
        const bool valid = lane < count && i < n_targets;
        const float4 p = valid ? targets[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const uint32_t full = __ballot_sync(kFull, valid);
        float lo[3] = {valid ? p.x : FLT_MAX, valid ? p.y : FLT_MAX, valid ? p.z : FLT_MAX};
        float hi[3] = {valid ? p.x : -FLT_MAX, valid ? p.y : -FLT_MAX, valid ? p.z : -FLT_MAX};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                lo[k] = fminf(lo[k], __shfl_xor_sync(kFull, lo[k], o));
                hi[k] = fmaxf(hi[k], __shfl_xor_sync(kFull, hi[k], o));
            }
        }
        L.tpos[lane] = p;
        int top = 0, napprox = 0, npp = 0, nmixed = 0, npriv = 0;
        if (num_nodes > 0 && root >= 0 && root < num_nodes) {
            if (lane == 0) stack[0] = make_int2(root, (int) full);
            top = 1;
        } else if (num_nodes > 0 && lane == 0) {
            atomicOr(err, (uint32_t) kErrTraverseLimit);  // a group without a valid tree root
        }
        __syncwarp();
        float ax = 0.f, ay = 0.f, az = 0.f;
        unsigned gnp = 0, gpp = 0;  // this group's interaction counts (kept for valid targets only)
        int64_t rounds = 0;

        while (top > 0 || nmixed > 0) {
            if (++rounds > round_limit) {
                if (lane == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
                break;
            }
            if (top > 0) {
                // ---- 1. pop up to 32 entries and classify them lane-parallel ----
                const int k = min(32, top);
                const int base = top - k;
                top = base;
                int c = 0, l0 = 0, l1 = -1, cls = kNone;
                uint32_t m = 0;
                if (lane < k) {
                    const int2 e = stack[base + lane];
                    c = e.x;
                    m = (uint32_t) e.y;
                    const float4 mc = __ldg(mac + c);
                    const int2 lk = __ldg(link + c);
                    l0 = lk.x;
                    l1 = lk.y;
                    // nearest box point and farthest box corner, per axis, with the reference's rounding
                    const float nx = fsub(fminf(fmaxf(mc.x, lo[0]), hi[0]), mc.x);
                    const float ny = fsub(fminf(fmaxf(mc.y, lo[1]), hi[1]), mc.y);
                    const float nz = fsub(fminf(fmaxf(mc.z, lo[2]), hi[2]), mc.z);
                    const float fx = fmaxf(fabsf(fsub(lo[0], mc.x)), fabsf(fsub(hi[0], mc.x)));
                    const float fy = fmaxf(fabsf(fsub(lo[1], mc.y)), fabsf(fsub(hi[1], mc.y)));
                    const float fz = fmaxf(fabsf(fsub(lo[2], mc.z)), fabsf(fsub(hi[2], mc.z)));
                    const float dmin2 = fadd(fadd(fmul(nx, nx), fmul(ny, ny)), fmul(nz, nz));
                    const float dmax2 = fadd(fadd(fmul(fx, fx), fmul(fy, fy)), fmul(fz, fz));
                    if (!(mc.w == mc.w)) cls = kOpenAll;  // NaN threshold: never approximated
                    else if (dmin2 >= mc.w) cls = kAcceptAll;
                    else if (dmax2 < mc.w) cls = kOpenAll;
                    else cls = kMixed;
                }
                __syncwarp();  // popped entries are read before children overwrite them
                const bool is_acc = cls == kAcceptAll && m == full;
                const bool is_acc_part = cls == kAcceptAll && m != full;
                const bool is_leaf_open = cls == kOpenAll && l1 >= 0;
                const bool is_int_open = cls == kOpenAll && l1 < 0 && l0 > c + 1 && l0 < num_nodes;
                if (cls == kOpenAll && l1 < 0 && !is_int_open) atomicOr(err, (uint32_t) kErrTraverseLimit);
                const bool is_mix = cls == kMixed;
                int pos = warp_append(is_acc, napprox, lt);
                if (is_acc) L.approx_node[pos] = c;
                append_private<ORDER, EPS0>(L, npriv, is_acc_part, c, m, pay, p, eps, lane, ax, ay, az, gnp);
                pos = warp_append(is_leaf_open, npp, lt);
                if (is_leaf_open) {
                    L.pp_begin[pos] = max(l0, 0);
                    L.pp_end[pos] = min(l1, n_bodies);
                    L.pp_mask[pos] = m;
                }
                pos = warp_append(is_mix, nmixed, lt);
                if (is_mix) { L.mixed_node[pos] = c; L.mixed_mask[pos] = m; }
                const uint32_t bi = __ballot_sync(kFull, is_int_open);
                if (top + 2 * __popc(bi) > kTraverseStack) {
                    // warp-uniform: a push would not fit, so the group is abandoned with an error
                    // (every entry on the stack was written; nothing unwritten is ever popped)
                    if (lane == 0) atomicOr(err, (uint32_t) kErrStackOverflow);
                    top = 0;
                    nmixed = 0;
                } else {
                    if (is_int_open) {
                        const int sp = top + 2 * __popc(bi & lt);
                        stack[sp] = make_int2(l0, (int) m);         // right child
                        stack[sp + 1] = make_int2(c + 1, (int) m);  // left child, popped first
                    }
                    top += 2 * __popc(bi);
                }
                __syncwarp();
                // each round appends at most 32 entries per list: evaluate before the next one
                if (napprox > kList - 32) flush_approx<ORDER, EPS0>(L, napprox, pay, p, eps, ax, ay, az, gnp);
                if (npp > kList - 32) flush_pp<EPS0>(L, npp, bodies, p, eps, lane, ax, ay, az, gpp);
            }
            if (nmixed >= 32 || (top == 0 && nmixed > 0)) {
                // ---- 2. resolve up to 32 mixed nodes: per-target MAC, lane-parallel over nodes ----
                const int k = min(32, nmixed);
                const int base = nmixed - k;
                nmixed = base;
                int c = 0, l0 = 0, l1 = -1;
                uint32_t A = 0, O = 0;
                if (lane < k) {
                    c = L.mixed_node[base + lane];
                    const uint32_t m = L.mixed_mask[base + lane];
                    const float4 mc = __ldg(mac + c);
                    const int2 lk = __ldg(link + c);
                    l0 = lk.x;
                    l1 = lk.y;
                    uint32_t bits = 0;
#pragma unroll 8
                    for (int t = 0; t < 32; ++t) {
                        const float4 tp = L.tpos[t];
                        bits |= (ref_dist2(tp.x, tp.y, tp.z, mc) >= mc.w) ? (1u << t) : 0u;
                    }
                    A = bits & m;
                    O = m & ~A;
                }
                __syncwarp();
                const bool is_acc = A != 0 && A == full;
                const bool is_acc_part = A != 0 && A != full;
                const bool is_leaf_open = O != 0 && l1 >= 0;
                const bool is_int_open = O != 0 && l1 < 0 && l0 > c + 1 && l0 < num_nodes;
                if (O != 0 && l1 < 0 && !is_int_open) atomicOr(err, (uint32_t) kErrTraverseLimit);
                int pos = warp_append(is_acc, napprox, lt);
                if (is_acc) L.approx_node[pos] = c;
                append_private<ORDER, EPS0>(L, npriv, is_acc_part, c, A, pay, p, eps, lane, ax, ay, az, gnp);
                pos = warp_append(is_leaf_open, npp, lt);
                if (is_leaf_open) {
                    L.pp_begin[pos] = max(l0, 0);
                    L.pp_end[pos] = min(l1, n_bodies);
                    L.pp_mask[pos] = O;
                }
                const uint32_t bi = __ballot_sync(kFull, is_int_open);
                if (top + 2 * __popc(bi) > kTraverseStack) {
                    if (lane == 0) atomicOr(err, (uint32_t) kErrStackOverflow);
                    top = 0;
                    nmixed = 0;
                } else {
                    if (is_int_open) {
                        const int sp = top + 2 * __popc(bi & lt);
                        stack[sp] = make_int2(l0, (int) O);
                        stack[sp + 1] = make_int2(c + 1, (int) O);
                    }
                    top += 2 * __popc(bi);
                }
                __syncwarp();
                if (napprox > kList - 32) flush_approx<ORDER, EPS0>(L, napprox, pay, p, eps, ax, ay, az, gnp);
                if (npp > kList - 32) flush_pp<EPS0>(L, npp, bodies, p, eps, lane, ax, ay, az, gpp);
            }
        }
        flush_approx<ORDER, EPS0>(L, napprox, pay, p, eps, ax, ay, az, gnp);
        flush_private<ORDER, EPS0>(L, npriv, pay, p, eps, lane, ax, ay, az, gnp);
        flush_pp<EPS0>(L, npp, bodies, p, eps, lane, ax, ay, az, gpp);
        if (valid) acc[i] = make_float4(G * ax, G * ay, G * az, 0.f);
        if (valid) {
            cnp += gnp;
            cpp += gpp;
        }
        if (inst_counts && inst >= 0) {
            const unsigned ipp = __reduce_add_sync(kFull, valid ? gpp : 0u);
            const unsigned inp = __reduce_add_sync(kFull, valid ? gnp : 0u);
            if (lane == 0) {
                atomicAdd(inst_counts + 2 * (int64_t) inst, (unsigned long long) ipp);
                atomicAdd(inst_counts + 2 * (int64_t) inst + 1, (unsigned long long) inp);
            }
        }
        __syncwarp();
    }
    if (counts) {
        const unsigned spp = __reduce_add_sync(kFull, cpp);
        const unsigned snp = __reduce_add_sync(kFull, cnp);
        if (lane == 0) {
            atomicAdd(counts + 0, (unsigned long long) spp);
            atomicAdd(counts + 1, (unsigned long long) snp);
        }
    }
}

// Occupancy and SM count are fixed per device and kernel: queried once (B200 parts are identical).
template<int ORDER, bool EPS0>
int blocks_per_sm() {
    static int cached = 0;
    if (cached == 0) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, bh_kernel<ORDER, EPS0>, kThreads, 0);
        cached = b > 0 ? b : 1;
    }
    return cached;
}

template<int ORDER, bool EPS0>
void launch_variant(const NodeArrays &nodes, const int *num_nodes, const float4 *bodies, int n_bodies,
                    const float4 *targets, int nt, float G, float eps, float4 *acc, unsigned long long *counts,
                    TraverseWorkspace &ws, uint32_t *err, cudaStream_t s, const int4 *gtab, int64_t ngroups,
                    const int *inst_root, unsigned long long *inst_counts) {
    int device = 0;
    cudaGetDevice(&device);
    int64_t blocks = (int64_t) sm_count(device) * blocks_per_sm<ORDER, EPS0>();
    blocks = std::min<int64_t>(blocks, ws.warps / kWarps);
    const int64_t groups = gtab ? ngroups : (nt + 31) / 32;
    blocks = std::min<int64_t>(blocks, (groups + kWarps - 1) / kWarps);
    if (blocks < 1) blocks = 1;
    cudaMemsetAsync(ws.group_counter, 0, sizeof(unsigned), s);
    bh_kernel<ORDER, EPS0><<<(unsigned) blocks, kThreads, 0, s>>>(nodes, num_nodes, bodies, n_bodies, targets, nt, G,
                                                                   eps, acc, counts, ws.stack, ws.group_counter, err,
                                                                   gtab, (int) ngroups, inst_root, inst_counts);
}

}  // namespace

int sm_count(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (cached[device] == 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cached[device] = sms > 0 ? sms : 1;
    }
    return cached[device];
}

int current_sm_count() {
    int device = 0;
    cudaGetDevice(&device);
    return sm_count(device);
}

int64_t traverse_resident_warps(int device) {
    int b = std::max(std::max(blocks_per_sm<1, false>(), blocks_per_sm<1, true>()),
                     std::max(blocks_per_sm<2, false>(), blocks_per_sm<2, true>()));
    return (int64_t) sm_count(device) * b * kWarps;
}

void launch_bh_traverse(int order, const NodeArrays &nodes, const int *num_nodes, const float4 *bodies, int64_t n_bodies,
                        const float4 *targets, int64_t n_targets, float G, float eps, float4 *acc,
                        unsigned long long *counts, TraverseWorkspace &ws, uint32_t *err, cudaStream_t s,
                        const int4 *gtab, int64_t ngroups, const int *inst_root, unsigned long long *inst_counts) {
    if (n_targets <= 0) return;
    const int nb = (int) n_bodies, nt = (int) n_targets;
    if (order == 1) {
        if (eps == 0.f) launch_variant<1, true>(nodes, num_nodes, bodies, nb, targets, nt, G, eps, acc, counts, ws, err, s, gtab, ngroups, inst_root, inst_counts);
        else launch_variant<1, false>(nodes, num_nodes, bodies, nb, targets, nt, G, eps, acc, counts, ws, err, s, gtab, ngroups, inst_root, inst_counts);
    } else {
        if (eps == 0.f) launch_variant<2, true>(nodes, num_nodes, bodies, nb, targets, nt, G, eps, acc, counts, ws, err, s, gtab, ngroups, inst_root, inst_counts);
        else launch_variant<2, false>(nodes, num_nodes, bodies, nb, targets, nt, G, eps, acc, counts, ws, err, s, gtab, ngroups, inst_root, inst_counts);
    }
}

}  // namespace nbg
