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
//   3. Accepted nodes are staged in per-warp shared-memory slabs: the lane that accepted a node
//      copies its payload there asynchronously (cp.async), so the payload crosses L2 once per
//      group instead of once per target. Nodes accepted by every target go to the full slab and
//      are evaluated by all lanes with broadcast reads; nodes accepted by some targets go to the
//      partial slab with their target masks, and at evaluation a warp bit-matrix transpose of
//      the masks gives every lane the set of slab entries it owns, which it walks on its own.
//      Opened leaves go to a (leaf, mask) list evaluated with broadcast body loads; opened
//      internal nodes push both children.
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

// Launch shapes (autotuned per workload, see nb_set_traversal_shape): THREADS threads per block
// (128 or 256) and PART entries in the partial-accept slab (32 or 64). The launch bounds keep
// 1024 threads per SM resident (64 registers per thread).
constexpr int kResidentThreads = 1024;
constexpr int kList = 64;      // leaf and mixed lists: each round appends at most 32, evaluated above 32
constexpr int kFullSlab = 32;  // staged nodes accepted by the whole group
// Stack: kTraverseStack entries per warp. No bound below that size is proven for every tree, so a
// round whose pushes would not fit abandons its group and sets kErrStackOverflow (the host turns it
// into an error); every entry on the stack has been written, so no stale entry is ever popped.
constexpr unsigned kFull = 0xffffffffu;

enum : int { kNone = 0, kAcceptAll = 1, kOpenAll = 2, kMixed = 3 };

template<int PAY, int PART>
struct WarpSmem {
    float4 tpos[32];
    float4 full_pay[kFullSlab * PAY];  // payloads of group-wide accepted nodes
    float4 part_pay[(PART + 1) * PAY]; // payloads of partially accepted nodes, then the null payload
    uint32_t part_mask[PART];          // their target masks
    int pp_begin[kList], pp_end[kList];
    uint32_t pp_mask[kList];
    int mixed_node[kList];
    uint32_t mixed_mask[kList];
};

template<int ORDER, int THREADS, int PART>
constexpr size_t block_smem_bytes() {
    return sizeof(WarpSmem<NodeLayout<ORDER>::PAY, PART>) * (THREADS / 32);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// 16-byte asynchronous global -> shared copy (completes at cp_async_wait_all).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Transpose of the 32 x 32 bit matrix whose row r is lane r's word: afterwards bit r of lane c's
// word is bit c of row r (five butterfly stages exchanging off-diagonal blocks).
__device__ __forceinline__ uint32_t transpose32(uint32_t x, int lane) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const uint32_t hi = s == 16 ? 0xFFFF0000u : s == 8 ? 0xFF00FF00u : s == 4 ? 0xF0F0F0F0u
                          : s == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;
        const uint32_t y = __shfl_xor_sync(kFull, x, s);
        x = (lane & s) ? ((x & hi) | ((y & hi) >> s)) : ((x & ~hi) | ((y & ~hi) << s));
    }
    return x;
}

// Squared distance in the reference's IEEE order: (dx*dx + dy*dy) + dz*dz, d = p - c.
__device__ __forceinline__ float ref_dist2(float px, float py, float pz, float4 c) {
    const float dx = fsub(px, c.x), dy = fsub(py, c.y), dz = fsub(pz, c.z);
    return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
}

// on = false makes the term exactly zero (a select, not a branch, so that lanes whose target does
// not take the term run the same instructions).
template<bool EPS0>
__device__ __forceinline__ void pair_term(float4 p, float4 b, float eps, float &ax, float &ay, float &az,
                                          bool on = true) {
    const float rx = p.x - b.x, ry = p.y - b.y, rz = p.z - b.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps)));
    if (EPS0 && r2 == 0.f) return;  // equal positions contribute nothing (Gravity.h:203)
    const float inv = rsqrt_hw(r2);
    const float s = on ? b.w * (inv * inv * inv) : 0.f;
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
    const float inv = rsqrt_hw(r2);
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

// Node term from a staged payload (PAY float4 in shared memory).
template<int ORDER, bool EPS0>
__device__ __forceinline__ void staged_term(const float4 *pc, float4 p, float eps, float &ax, float &ay, float &az) {
    if constexpr (ORDER == 1) {
        pair_term<EPS0>(p, pc[0], eps, ax, ay, az);
    } else {
        quad_term<EPS0>(p, pc[0], pc[1], pc[2], eps, ax, ay, az);
    }
}

template<int PAY>
__device__ __forceinline__ void stage_node(float4 *dst, const float4 *__restrict__ pay, int c) {
    const float4 *src = pay + (int64_t) c * PAY;
#pragma unroll
    for (int k = 0; k < PAY; ++k) cp_async16(dst + k, src + k);
}

// Nodes accepted by the whole group: every lane evaluates every staged entry (broadcast reads).
template<int ORDER, bool EPS0, int PART>
__device__ __forceinline__ void flush_full(WarpSmem<NodeLayout<ORDER>::PAY, PART> &S, int &nfull, float4 p, float eps,
                                           float &ax, float &ay, float &az, unsigned &cnp) {
    constexpr int PAY = NodeLayout<ORDER>::PAY;
    cp_async_wait_all();
    __syncwarp();
    int j = 0;
    for (; j + 1 < nfull; j += 2) {
        staged_term<ORDER, EPS0>(S.full_pay + j * PAY, p, eps, ax, ay, az);
        staged_term<ORDER, EPS0>(S.full_pay + (j + 1) * PAY, p, eps, ax, ay, az);
    }
    if (j < nfull) staged_term<ORDER, EPS0>(S.full_pay + j * PAY, p, eps, ax, ay, az);
    cnp += (unsigned) nfull;
    nfull = 0;
    __syncwarp();
}

// Nodes accepted by some targets only: the masks are transposed so that each lane holds the set
// of entries it evaluates, then every lane walks its own set.
template<int ORDER, bool EPS0, int PART>
__device__ __forceinline__ void flush_part(WarpSmem<NodeLayout<ORDER>::PAY, PART> &S, int &npart, float4 p, float eps,
                                           int lane, float &ax, float &ay, float &az, unsigned &cnp) {
    constexpr int PAY = NodeLayout<ORDER>::PAY;
    cp_async_wait_all();
    __syncwarp();
    uint32_t b0 = transpose32(lane < npart ? S.part_mask[lane] : 0u, lane);
    uint32_t b1 = 0u;
    if constexpr (PART > 32)
        b1 = npart > 32 ? transpose32(lane + 32 < npart ? S.part_mask[lane + 32] : 0u, lane) : 0u;
    cnp += (unsigned) (__popc(b0) + __popc(b1));
    // a lane whose set is used up evaluates the null payload instead of branching around the term
    while (__any_sync(kFull, (b0 | b1) != 0u)) {
        int j = PART;
        if (b0) {
            j = __ffs(b0) - 1;
            b0 &= b0 - 1;
        } else if (b1) {
            j = 31 + __ffs(b1);
            b1 &= b1 - 1;
        }
        staged_term<ORDER, EPS0>(S.part_pay + j * PAY, p, eps, ax, ay, az);
    }
    npart = 0;
    __syncwarp();
}

template<bool EPS0, int PAY, int PART>
__device__ __forceinline__ void flush_pp(WarpSmem<PAY, PART> &S, int &npp, const float4 *__restrict__ bodies, float4 p,
                                         float eps, int lane, float &ax, float &ay, float &az, unsigned &cpp) {
    for (int j = 0; j < npp; ++j) {
        const int b = S.pp_begin[j], e = S.pp_end[j];
        const bool on = (S.pp_mask[j] >> lane) & 1u;
        int k = b;
        for (; k + 3 < e; k += 4) {
            const float4 s0 = __ldg(bodies + k), s1 = __ldg(bodies + k + 1);
            const float4 s2 = __ldg(bodies + k + 2), s3 = __ldg(bodies + k + 3);
            pair_term<EPS0>(p, s0, eps, ax, ay, az, on);
            pair_term<EPS0>(p, s1, eps, ax, ay, az, on);
            pair_term<EPS0>(p, s2, eps, ax, ay, az, on);
            pair_term<EPS0>(p, s3, eps, ax, ay, az, on);
        }
        for (; k < e; ++k) {
            const float4 s0 = __ldg(bodies + k);
            pair_term<EPS0>(p, s0, eps, ax, ay, az, on);
        }
        if (on) cpp += (unsigned) (e - b);
    }
    npp = 0;
    __syncwarp();
}

// Classified entries of one round, appended to the slabs and lists (warp-uniform control flow):
// acc / part are accepted nodes (target mask mk for part), leaf is an opened leaf (body range
// l0..l1, mask mk), open an opened internal node (children c + 1 and l0, mask mk), mixed a node
// still to be resolved per target.
template<int ORDER, bool EPS0, int PART>
__device__ __forceinline__ bool dispatch(WarpSmem<NodeLayout<ORDER>::PAY, PART> &S, const float4 *__restrict__ pay,
                                         const float4 *__restrict__ bodies, int2 *stack, bool acc, bool part,
                                         bool leaf, bool open, bool mixed, int c, uint32_t mk, int l0, int l1,
                                         int n_bodies, uint32_t lt, int lane, int &nfull, int &npart, int &npp,
                                         int &nmixed, int &top, float4 p, float eps, float &ax, float &ay, float &az,
                                         unsigned &gnp, unsigned &gpp, uint32_t *err) {
    constexpr int PAY = NodeLayout<ORDER>::PAY;
    uint32_t b = __ballot_sync(kFull, acc);
    if (b) {
        if (nfull + __popc(b) > kFullSlab) flush_full<ORDER, EPS0, PART>(S, nfull, p, eps, ax, ay, az, gnp);
        if (acc) stage_node<PAY>(S.full_pay + (nfull + __popc(b & lt)) * PAY, pay, c);
        nfull += __popc(b);
    }
    b = __ballot_sync(kFull, part);
    if (b) {
        if (npart + __popc(b) > PART) flush_part<ORDER, EPS0, PART>(S, npart, p, eps, lane, ax, ay, az, gnp);
        if (part) {
            const int slot = npart + __popc(b & lt);
            stage_node<PAY>(S.part_pay + slot * PAY, pay, c);
            S.part_mask[slot] = mk;
        }
        npart += __popc(b);
    }
    b = __ballot_sync(kFull, leaf);
    if (leaf) {
        const int pos = npp + __popc(b & lt);
        S.pp_begin[pos] = max(l0, 0);
        S.pp_end[pos] = min(l1, n_bodies);
        S.pp_mask[pos] = mk;
    }
    npp += __popc(b);
    b = __ballot_sync(kFull, mixed);
    if (mixed) {
        const int pos = nmixed + __popc(b & lt);
        S.mixed_node[pos] = c;
        S.mixed_mask[pos] = mk;
    }
    nmixed += __popc(b);
    b = __ballot_sync(kFull, open);
    bool abandoned = false;
    if (top + 2 * __popc(b) > kTraverseStack) {
        // a push would not fit: the group is abandoned with an error (warp-uniform)
        if (lane == 0) atomicOr(err, (uint32_t) kErrStackOverflow);
        abandoned = true;
    } else {
        if (open) {
            const int sp = top + 2 * __popc(b & lt);
            stack[sp] = make_int2(l0, (int) mk);         // right child
            stack[sp + 1] = make_int2(c + 1, (int) mk);  // left child, popped first
        }
        top += 2 * __popc(b);
    }
    __syncwarp();
    // each round appends at most 32 leaves: evaluate before the next one could overflow the list
    if (npp > kList - 32) flush_pp<EPS0, NodeLayout<ORDER>::PAY, PART>(S, npp, bodies, p, eps, lane, ax, ay, az, gpp);
    return abandoned;
}

template<int ORDER, bool EPS0, int THREADS, int PART>
__global__ void __launch_bounds__(THREADS, kResidentThreads / THREADS) bh_kernel(NodeArrays nodes, const int *__restrict__ num_nodes_p,
                                                         const float4 *__restrict__ bodies, int n_bodies,
                                                         const float4 *__restrict__ targets, int n_targets, float G,
                                                         float eps, float4 *__restrict__ acc,
                                                         unsigned long long *__restrict__ counts,
                                                         int2 *__restrict__ stack_base,
                                                         unsigned *__restrict__ group_counter,
                                                         uint32_t *__restrict__ err, const int4 *__restrict__ groups,
                                                         int num_group_tasks, const int *__restrict__ inst_root,
                                                         unsigned long long *__restrict__ inst_counts) {
    constexpr int PAY = NodeLayout<ORDER>::PAY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpSmem<PAY, PART> &S = reinterpret_cast<WarpSmem<PAY, PART> *>(smem_raw)[warp];
    int2 *stack = stack_base + ((int64_t) blockIdx.x * (THREADS / 32) + warp) * kTraverseStack;
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
        S.tpos[lane] = p;
        // the null payload: no mass and no moments at 1e30 on every axis, where the squared
        // distance from any target with coordinates below 1e29 in magnitude overflows to
        // infinity, so that every factor of the term is exactly zero and it adds nothing
        if (lane < PAY) S.part_pay[PART * PAY + lane] = lane == 0 ? make_float4(1e30f, 1e30f, 1e30f, 0.f)
                                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
        int top = 0, nfull = 0, npart = 0, npp = 0, nmixed = 0;
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
                const bool is_leaf_open = cls == kOpenAll && l1 >= 0;
                const bool is_int_open = cls == kOpenAll && l1 < 0 && l0 > c + 1 && l0 < num_nodes;
                if (cls == kOpenAll && l1 < 0 && !is_int_open) atomicOr(err, (uint32_t) kErrTraverseLimit);
                if (dispatch<ORDER, EPS0, PART>(S, pay, bodies, stack, cls == kAcceptAll && m == full,
                                          cls == kAcceptAll && m != full, is_leaf_open, is_int_open, cls == kMixed,
                                          c, m, l0, l1, n_bodies, lt, lane, nfull, npart, npp, nmixed, top, p, eps,
                                          ax, ay, az, gnp, gpp, err)) {
                    top = 0;
                    nmixed = 0;
                }
            }
            if (nmixed >= 32 || (top == 0 && nmixed > 0)) {
                // ---- 2. resolve up to 32 mixed nodes: per-target MAC, lane-parallel over nodes ----
                const int k = min(32, nmixed);
                const int base = nmixed - k;
                nmixed = base;
                int c = 0, l0 = 0, l1 = -1;
                uint32_t A = 0, O = 0;
                if (lane < k) {
                    c = S.mixed_node[base + lane];
                    const uint32_t m = S.mixed_mask[base + lane];
                    const float4 mc = __ldg(mac + c);
                    const int2 lk = __ldg(link + c);
                    l0 = lk.x;
                    l1 = lk.y;
                    uint32_t bits = 0;
#pragma unroll 8
                    for (int t = 0; t < 32; ++t) {
                        const float4 tp = S.tpos[t];
                        bits |= (ref_dist2(tp.x, tp.y, tp.z, mc) >= mc.w) ? (1u << t) : 0u;
                    }
                    A = bits & m;
                    O = m & ~A;
                }
                __syncwarp();
                const bool is_int_open = O != 0 && l1 < 0 && l0 > c + 1 && l0 < num_nodes;
                if (O != 0 && l1 < 0 && !is_int_open) atomicOr(err, (uint32_t) kErrTraverseLimit);
                const bool is_acc = A != 0 && A == full;
                const bool is_part = A != 0 && A != full;
                // an entry can be accepted by some targets and opened by others: append both parts
                if (dispatch<ORDER, EPS0, PART>(S, pay, bodies, stack, is_acc, is_part, false, false, false, c, A, l0,
                                          l1, n_bodies, lt, lane, nfull, npart, npp, nmixed, top, p, eps, ax, ay,
                                          az, gnp, gpp, err) ||
                    dispatch<ORDER, EPS0, PART>(S, pay, bodies, stack, false, false, O != 0 && l1 >= 0, is_int_open, false,
                                          c, O, l0, l1, n_bodies, lt, lane, nfull, npart, npp, nmixed, top, p, eps,
                                          ax, ay, az, gnp, gpp, err)) {
                    top = 0;
                    nmixed = 0;
                }
            }
        }
        flush_full<ORDER, EPS0, PART>(S, nfull, p, eps, ax, ay, az, gnp);
        flush_part<ORDER, EPS0, PART>(S, npart, p, eps, lane, ax, ay, az, gnp);
        flush_pp<EPS0, PAY, PART>(S, npp, bodies, p, eps, lane, ax, ay, az, gpp);
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
// The kernel's dynamic shared memory (the warps' slabs and lists) is enabled on first use.
template<int ORDER, bool EPS0, int THREADS, int PART>
int blocks_per_sm(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (cached[device] == 0) {
        const size_t smem = block_smem_bytes<ORDER, THREADS, PART>();
        auto kernel = bh_kernel<ORDER, EPS0, THREADS, PART>;
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, THREADS, smem);
        cached[device] = b > 0 ? b : 1;
    }
    return cached[device];
}

template<int ORDER, bool EPS0, int THREADS, int PART>
int resident_warps(int device) {
    return sm_count(device) * blocks_per_sm<ORDER, EPS0, THREADS, PART>(device) * (THREADS / 32);
}

struct LaunchArgs {
    const NodeArrays *nodes;
    const int *num_nodes;
    const float4 *bodies;
    int n_bodies;
    const float4 *targets;
    int nt;
    float G, eps;
    float4 *acc;
    unsigned long long *counts;
    TraverseWorkspace *ws;
    uint32_t *err;
    cudaStream_t s;
    const int4 *gtab;
    int64_t ngroups;
    const int *inst_root;
    unsigned long long *inst_counts;
};

template<int ORDER, bool EPS0, int THREADS, int PART>
void launch_variant(const LaunchArgs &a) {
    constexpr int kWarps = THREADS / 32;
    int device = 0;
    cudaGetDevice(&device);
    int64_t blocks = (int64_t) sm_count(device) * blocks_per_sm<ORDER, EPS0, THREADS, PART>(device);
    blocks = std::min<int64_t>(blocks, a.ws->warps / kWarps);
    const int64_t groups = a.gtab ? a.ngroups : (a.nt + 31) / 32;
    blocks = std::min<int64_t>(blocks, (groups + kWarps - 1) / kWarps);
    if (blocks < 1) blocks = 1;
    cudaMemsetAsync(a.ws->group_counter, 0, sizeof(unsigned), a.s);
    bh_kernel<ORDER, EPS0, THREADS, PART><<<(unsigned) blocks, THREADS, block_smem_bytes<ORDER, THREADS, PART>(), a.s>>>(
        *a.nodes, a.num_nodes, a.bodies, a.n_bodies, a.targets, a.nt, a.G, a.eps, a.acc, a.counts, a.ws->stack,
        a.ws->group_counter, a.err, a.gtab, (int) a.ngroups, a.inst_root, a.inst_counts);
}

template<int ORDER, bool EPS0>
void launch_shape(const LaunchArgs &a, int threads, int part) {
    if (threads == 128) {
        if (part == 32) launch_variant<ORDER, EPS0, 128, 32>(a);
        else launch_variant<ORDER, EPS0, 128, 64>(a);
    } else {
        if (part == 32) launch_variant<ORDER, EPS0, 256, 32>(a);
        else launch_variant<ORDER, EPS0, 256, 64>(a);
    }
}

template<int ORDER, bool EPS0>
int max_resident_warps(int device) {
    return std::max(std::max(resident_warps<ORDER, EPS0, 128, 32>(device), resident_warps<ORDER, EPS0, 128, 64>(device)),
                    std::max(resident_warps<ORDER, EPS0, 256, 32>(device), resident_warps<ORDER, EPS0, 256, 64>(device)));
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
    return std::max(std::max(max_resident_warps<1, false>(device), max_resident_warps<1, true>(device)),
                    std::max(max_resident_warps<2, false>(device), max_resident_warps<2, true>(device)));
}

bool traversal_shape_valid(int threads, int slab) { return (threads == 128 || threads == 256) && (slab == 32 || slab == 64); }

void launch_bh_traverse(int order, const NodeArrays &nodes, const int *num_nodes, const float4 *bodies, int64_t n_bodies,
                        const float4 *targets, int64_t n_targets, float G, float eps, float4 *acc,
                        unsigned long long *counts, TraverseWorkspace &ws, uint32_t *err, cudaStream_t s,
                        const int4 *gtab, int64_t ngroups, const int *inst_root, unsigned long long *inst_counts) {
    if (n_targets <= 0) return;
    const LaunchArgs a{&nodes, num_nodes, bodies, (int) n_bodies, targets, (int) n_targets, G, eps, acc, counts, &ws,
                       err, s, gtab, ngroups, inst_root, inst_counts};
    const bool ok = traversal_shape_valid(ws.threads, ws.slab);
    const int threads = ok ? ws.threads : 256, part = ok ? ws.slab : 64;
    if (order == 1) {
        if (eps == 0.f) launch_shape<1, true>(a, threads, part);
        else launch_shape<1, false>(a, threads, part);
    } else {
        if (eps == 0.f) launch_shape<2, true>(a, threads, part);
        else launch_shape<2, false>(a, threads, part);
    }
}

}  // namespace nbg
