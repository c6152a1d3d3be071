// Implicit-field dual-tree traversal on the device: the reference's
// MultipoleImplicitLinearBVHFMMSolver<3> (octupole node moments, local field of order 4) under the
// DiagonalOverSeparation criterion.
//
// Decisions follow the reference, evaluated with the same IEEE operations, so the set of
// interactions (and the interaction counts) equals the reference's:
//   ImplicitDualTraversalSolver::updateAccelerations   ImplicitDualTraversalSolver.h:42-69
//   Tree::loadBalancedBreak(256)                       Tree.h:84-107
//   balancedLockstepDualTreeImplicitField              balancedLockstepDualTreeImplicitField.h:14-46
//   lockstepDualTreeImplicitField                      lockstepDualTreeImplicitField.h:21-168
//   passiveTreeImplicitField                           passiveTreeImplicitField.h:13-78
//   activeTree (point form of the criterion)           activeTree.h:24-79
//   DiagonalOverSeparation                             DiagonalOverSeparation.h:17-49
//   separation                                         BoundingBox.h:84-94 (std::pow(float, int) is a
//                                                      double pow, so the sum and root are in double)
//   M2L / P2L / M2P / L2L / L2P                        Gravity.h:239-259, 282-306, 352-392;
//                                                      MultipoleAcceleration.h:33-84
//
// Work organisation, two kernels:
//   dual_kernel  one thread block per starting passive node (the <= 256 nodes of
//                loadBalancedBreak, found on the device). Each block runs the reference's
//                recursion as a depth-first stack of tasks (lock-step and passive-tree tasks)
//                whose lists and local fields live in a per-block arena of global memory. Every
//                step is block-parallel: lists are classified one entry per thread with a stable
//                block-wide compaction (ballots and warp counts); the far entries' M2L / P2L terms
//                are then evaluated uniformly, one per thread, and reduced into the task's local
//                field in a fixed order; L2L translates it to the children; at a passive leaf the
//                block applies L2P. The leaf's near field is not evaluated here: the block appends
//                it to the leaf's item list (the activeTree roots of a lock-step leaf, or the close
//                bodies of a passive-tree leaf) in a global pool.
//   near_kernel  a persistent grid over all SMs. Each warp takes 32 targets of one passive leaf
//                and runs the leaf's items in list order: close bodies as pair tiles staged in
//                shared memory; activeTree roots as a warp walk with one lane per target and a
//                lane mask per stack entry, pairs at opened leaves as shared-memory tiles, and
//                M2P terms queued per lane and evaluated target-major.
// The near field, about nine tenths of the work, is thereby balanced over the whole GPU, and the
// uneven passive subtrees only bound the much shorter traversal. Every sum has a fixed order, so
// results are deterministic run to run; the accumulation order differs from the reference's
// serial recursion, the interactions evaluated are the same.
#include <algorithm>
#include <cfloat>
#include <climits>

#include "nb_internal.cuh"
#include "stensor.cuh"

namespace nbg {

namespace {

constexpr int kThreads = 256;  // traversal block: the whole block works on one task at a time
constexpr int kWarps = kThreads / 32;
constexpr int kTaskInts = 6;  // type, passive node, list offset, list length, field offset, arena top
constexpr int kLockstep = 0, kPassive = 1;
constexpr int F = st::kFieldFloats;

// Dual-tree node as stored (nb_internal.cuh, DualNodes). Internal nodes keep ~first body in link.y.
struct DNode {
    float mn[3], mx[3], diag;
    int size;
    float com[3], M;
    int link0, link1;
    __device__ bool leaf() const { return link1 >= 0; }
    __device__ int first() const { return link1 >= 0 ? link0 : -1 - link1; }
};

__device__ __forceinline__ DNode load_node(const DualNodes &N, int k) {
    DNode d;
    const float4 a = __ldg(N.bmin + k), b = __ldg(N.bmax + k), c = __ldg(N.com + k);
    const int2 l = __ldg(N.link + k);
    d.mn[0] = a.x; d.mn[1] = a.y; d.mn[2] = a.z; d.size = __float_as_int(a.w);
    d.mx[0] = b.x; d.mx[1] = b.y; d.mx[2] = b.z; d.diag = b.w;
    d.com[0] = c.x; d.com[1] = c.y; d.com[2] = c.z; d.M = c.w;
    d.link0 = l.x; d.link1 = l.y;
    return d;
}

// BoundingBox::center: (max + min) / 2
__device__ __forceinline__ void center(const DNode &n, float c[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) c[k] = fdiv(fadd(n.mx[k], n.mn[k]), 2.0f);
}

__device__ __forceinline__ float max0(float x) { return (x < 0.f) ? 0.f : x; }
// glm::length: sqrt((x*x + y*y) + z*z)
__device__ __forceinline__ float len3(float a, float b, float c) {
    return __fsqrt_rn(fadd(fadd(fmul(a, a), fmul(b, b)), fmul(c, c)));
}
// (float) sqrt(pow(|u|, 2) + pow(|v|, 2)) with the pow, sum and root in double. When one length
// is zero the result is the other one exactly (a float's square is exact in double, and so is the
// root of an exact square), which is the common case and needs no double arithmetic.
__device__ __forceinline__ float sep_from(float lu, float lv) {
    if (lv == 0.f) return lu;
    if (lu == 0.f) return lv;
    const double du = (double) lu, dv = (double) lv;
    return __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(du, du), __dmul_rn(dv, dv))));
}
__device__ __forceinline__ float sep_box(const DNode &a, const DNode &b) {
    const float lu = len3(max0(fsub(a.mn[0], b.mx[0])), max0(fsub(a.mn[1], b.mx[1])), max0(fsub(a.mn[2], b.mx[2])));
    const float lv = len3(max0(fsub(b.mn[0], a.mx[0])), max0(fsub(b.mn[1], a.mx[1])), max0(fsub(b.mn[2], a.mx[2])));
    return sep_from(lu, lv);
}

// sep(node, p) >= B, exactly, with the node's thresholds (B, S): when one of the two separation
// vectors is zero, sep is RN(sqrt(|v|^2)) and the test is |v|^2 >= S; otherwise the double path.
// sep >= B from the squared lengths su, sv of the two separation vectors (non-decreasing in both).
//
// With both vectors nonzero, the exact sum lu^2 + lv^2 of the rounded lengths lies within a
// relative 1.5 * 2^-23 of q = RN(su + sv), and sep (its double root rounded to float) is >= B
// whenever that sum is >= B^2 (1 + 2^-21) and < B^2 whenever it is <= B^2 (1 - 2^-21). So
// q >= RN(B^2) (1 + 2^-18) decides "yes" and q < RN(B^2) (1 - 2^-18) decides "no" exactly (for
// RN(B^2) in [1e-30, 1e30], where no term is denormal or overflows); only the cases in between
// take the double path.
__device__ __forceinline__ bool sep_test(float su, float sv, float B, float S) {
    if (sv == 0.f) return su >= S;
    if (su == 0.f) return sv >= S;
    const float b2 = B * B, q = su + sv;
    if (b2 >= 1e-30f && b2 <= 1e30f) {
        if (q >= b2 * (1.0f + 0x1p-18f)) return true;
        if (q < b2 * (1.0f - 0x1p-18f)) return false;
    }
    return sep_from(__fsqrt_rn(su), __fsqrt_rn(sv)) >= B;
}
// Squared length of the per-axis gaps (max0(a - b))_k, in the reference's operation order.
__device__ __forceinline__ float gap2(float a0, float a1, float a2, float b0, float b1, float b2) {
    const float x = max0(fsub(a0, b0)), y = max0(fsub(a1, b1)), z = max0(fsub(a2, b2));
    return fadd(fadd(fmul(x, x), fmul(y, y)), fmul(z, z));
}
__device__ __forceinline__ bool sep_at_least(const DNode &n, const float p[3], float B, float S) {
    return sep_test(gap2(n.mn[0], n.mn[1], n.mn[2], p[0], p[1], p[2]), gap2(p[0], p[1], p[2], n.mx[0], n.mx[1], n.mx[2]),
                    B, S);
}

// DiagonalOverSeparation (DiagonalOverSeparation.h:29-49), (active node, point): approximate the
// node for the point iff RN(diag / sep) < theta and it has more than 32 bodies; chunk_walk decides
// it per target (sep_at_least with the node's thresholds) and for boxes of targets (classify_group).
// (point, passive node): the active point is far from the passive node, RN(3 diag / sep) < theta
__device__ __forceinline__ bool point_is_far(const float p[3], const DNode &P, float4 thr) {
    return sep_at_least(P, p, thr.z, thr.w);
}
// (active node, passive node): 0 = approximate, else DescendActive (1) | DescendPassive (2)
__device__ __forceinline__ int node_node(const DNode &A, const DNode &P, float theta) {
    if (A.size > 32 && fdiv(fadd(A.diag, P.diag), sep_box(A, P)) < theta) return 0;
    int r = 0;
    if (A.diag <= fmul(P.diag, 2.0f)) r |= 2;
    if (P.diag <= fmul(A.diag, 2.0f)) r |= 1;
    return r;
}

struct Ctx {
    DualNodes nodes;
    const float4 *bodies;
    float G, eps, theta;
    int nn, n;  // node and body counts
    // Preorder links only point forward: a child's index exceeds its parent's and the left child's
    // (parent + 1); a leaf's bodies lie in [0, n). A link that breaks this is not followed (error
    // bit kErrTraverseLimit), so every descent terminates and stays in bounds.
    __device__ bool right_ok(int k, int right) const { return right > k + 1 && right < nn; }
    __device__ bool left_ok(int k) const { return k + 1 < nn; }
    __device__ bool range_ok(int first, int end) const { return 0 <= first && first <= end && end <= n; }
};

__device__ __forceinline__ void load_q(const DualNodes &N, int k, float q2[6], float q3[10]) {
    const float4 *q = N.q + (int64_t) k * 4;
    const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
    q2[0] = a.x; q2[1] = a.y; q2[2] = a.z; q2[3] = a.w; q2[4] = b.x; q2[5] = b.y;
    q3[0] = b.z; q3[1] = b.w; q3[2] = c.x; q3[3] = c.y; q3[4] = c.z; q3[5] = c.w;
    q3[6] = d.x; q3[7] = d.y; q3[8] = d.z; q3[9] = d.w;
}

// 1 / sqrt(|R|^2 + eps) (the reference's r is sqrt(|R|^2 + eps), Gravity.h:207)
__device__ __forceinline__ float soft_inv_r(const float R[3], float eps) {
    return rsqrt_hw(fmaf(R[0], R[0], fmaf(R[1], R[1], fmaf(R[2], R[2], eps))));
}

// Gravity::nodeNode for MultipoleMassSummary<3> -> MultipoleAccelerationSummary<4> (M2L,
// Gravity.h:352-392), added into the local field f about pc. As in the reference, the moment
// terms carry no factor G.
__device__ void m2l(const Ctx &x, int k, const DNode &n, const float pc[3], float *f) {
    const float R[3] = {pc[0] - n.com[0], pc[1] - n.com[1], pc[2] - n.com[2]};
    if (R[0] == 0.f && R[1] == 0.f && R[2] == 0.f) return;
    const float inv = soft_inv_r(R, x.eps);
    const st::Coef c = st::Coef::from_inverse(inv);
    float q2[6], q3[10], d2[6], d3[10], d4[15], v3[3], v4[3], t2q[6];
    load_q(x.nodes, k, q2, q3);
    st::D2(R, c, d2);
    st::D3(R, c, d3);
    st::D4(R, c, d4);
    st::t3_dot_t2(d3, q2, v3);
    st::t4_dot_t3(d4, q3, v4);
    st::t4_dot_t2(d4, q2, t2q);
    const float mg = n.M * x.G;
    const float mono = mg * (inv * inv * inv);
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] += -R[i] * mono + v3[i] / 2.0f + v4[i] / 6.0f;
#pragma unroll
    for (int a = 0; a < 6; ++a) f[3 + a] += d2[a] * mg - t2q[a] * 0.5f;
#pragma unroll
    for (int a = 0; a < 10; ++a) f[9 + a] += d3[a] * mg * 0.5f;
#pragma unroll
    for (int a = 0; a < 15; ++a) f[19 + a] += d4[a] * mg * (1.0f / 6.0f);
}

// Gravity::particleNode into MultipoleAccelerationSummary<4> (P2L, Gravity.h:282-306). The
// expansion factors (m G for D2, m G / 2 for D3, m G / 6 for D4) are folded into the derivative
// coefficients, so each field component takes one product sum.
__device__ __forceinline__ st::Coef scaled(const st::Coef &c, float s) {
    st::Coef o;
    o.g1 = c.g1 * s;
    o.g2 = c.g2 * s;
    o.g3 = c.g3 * s;
    o.g4 = c.g4 * s;
    return o;
}
__device__ void p2l(const Ctx &x, float4 b, const float pc[3], float *f) {
    const float R[3] = {pc[0] - b.x, pc[1] - b.y, pc[2] - b.z};
    if (R[0] == 0.f && R[1] == 0.f && R[2] == 0.f) return;
    const float inv = soft_inv_r(R, x.eps);
    const st::Coef c = st::Coef::from_inverse(inv);
    const float mg = b.w * x.G;
    float d[15];
    const float m1 = c.g1 * mg;  // -m G / r^3
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] = fmaf(R[i], m1, f[i]);
    st::D2(R, scaled(c, mg), d);
#pragma unroll
    for (int a = 0; a < 6; ++a) f[3 + a] += d[a];
    st::D3(R, scaled(c, mg * 0.5f), d);
#pragma unroll
    for (int a = 0; a < 10; ++a) f[9 + a] += d[a];
    st::D4(R, scaled(c, mg * (1.0f / 6.0f)), d);
#pragma unroll
    for (int a = 0; a < 15; ++a) f[19 + a] += d[a];
}

struct Scan3 {
    int wcnt[3][kWarps];
    int base[3];
};

// Stable block-wide rank of a class label (0..2, or -1 for none) in thread order; returns the
// element's position within its class, the running bases in s.base carrying across calls.
// Every thread of the block must call it.
__device__ int stable_rank(int cls, Scan3 &s) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m0 = __ballot_sync(0xffffffffu, cls == 0);
    const unsigned m1 = __ballot_sync(0xffffffffu, cls == 1);
    const unsigned m2 = __ballot_sync(0xffffffffu, cls == 2);
    if (lane == 0) {
        s.wcnt[0][warp] = __popc(m0);
        s.wcnt[1][warp] = __popc(m1);
        s.wcnt[2][warp] = __popc(m2);
    }
    __syncthreads();
    int pos = -1;
    if (cls >= 0) {
        const unsigned mine = cls == 0 ? m0 : (cls == 1 ? m1 : m2);
        int off = s.base[cls];
        for (int w = 0; w < warp; ++w) off += s.wcnt[cls][w];
        pos = off + __popc(mine & ((1u << lane) - 1u));
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        int t = 0;
        for (int w = 0; w < kWarps; ++w) t += s.wcnt[threadIdx.x][w];
        s.base[threadIdx.x] += t;
    }
    __syncthreads();
    return pos;
}

// Stable block-wide partition of list[0..len) into classes 0, 1, 2 (c0, c1, c2; -1 drops the
// entry), appending after the counts already in s.base. A round covers kPartK x kThreads entries:
// warp w takes the w-th run of 32 kPartK consecutive entries, lane l its entries l, l + 32, ...
// (coalesced loads, kPartK classifications in flight per thread). Ranks come from ballots within
// the warp and one prefix over the warps' class totals: two block barriers per round. Every thread
// of the block must call it.
constexpr int kPartK = 4;
template<typename Classify>
__device__ void stable_partition(const int *list, int len, int *c0, int *c1, int *c2, Scan3 &s, Classify classify) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int i0 = 0; i0 < len; i0 += kPartK * kThreads) {
        const int wb = i0 + warp * (32 * kPartK) + lane;
        int e[kPartK], cls[kPartK];
#pragma unroll
        for (int j = 0; j < kPartK; ++j) e[j] = wb + 32 * j < len ? list[wb + 32 * j] : -1;
#pragma unroll
        for (int j = 0; j < kPartK; ++j) cls[j] = wb + 32 * j < len ? classify(e[j]) : -1;
        int tot[3] = {0, 0, 0};
#pragma unroll
        for (int j = 0; j < kPartK; ++j) {
            tot[0] += __popc(__ballot_sync(0xffffffffu, cls[j] == 0));
            tot[1] += __popc(__ballot_sync(0xffffffffu, cls[j] == 1));
            tot[2] += __popc(__ballot_sync(0xffffffffu, cls[j] == 2));
        }
        if (lane == 0) {
            s.wcnt[0][warp] = tot[0];
            s.wcnt[1][warp] = tot[1];
            s.wcnt[2][warp] = tot[2];
        }
        __syncthreads();
        int off[3], next[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int pre = s.base[k], all = s.base[k];
            for (int w = 0; w < kWarps; ++w) {
                const int c = s.wcnt[k][w];
                if (w < warp) pre += c;
                all += c;
            }
            off[k] = pre;
            next[k] = all;
        }
        // every thread has read the bases and the counts before the bases change and before the
        // next round's counts overwrite them; the next round reads the new bases after its first
        // barrier
        __syncthreads();
        if (threadIdx.x < 3) s.base[threadIdx.x] = threadIdx.x == 0 ? next[0] : (threadIdx.x == 1 ? next[1] : next[2]);
#pragma unroll
        for (int j = 0; j < kPartK; ++j) {
            const unsigned b0 = __ballot_sync(0xffffffffu, cls[j] == 0);
            const unsigned b1 = __ballot_sync(0xffffffffu, cls[j] == 1);
            const unsigned b2 = __ballot_sync(0xffffffffu, cls[j] == 2);
            if (cls[j] == 0) c0[off[0] + __popc(b0 & lt)] = e[j];
            else if (cls[j] == 1) c1[off[1] + __popc(b1 & lt)] = e[j];
            else if (cls[j] == 2) c2[off[2] + __popc(b2 & lt)] = e[j];
            off[0] += __popc(b0);
            off[1] += __popc(b1);
            off[2] += __popc(b2);
        }
    }
}

// Block-wide exclusive prefix sum of v; every thread gets the block total.
__device__ int block_exclusive_scan(int v, int *s_w, int &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    int off = 0, tot = 0;
    for (int w = 0; w < kWarps; ++w) {
        if (w < warp) off += s_w[w];
        tot += s_w[w];
    }
    __syncthreads();
    total = tot;
    return off + x - v;
}

// Adds the per-thread partial fields into the block's shared field (fixed order: lanes by
// butterfly, then warps in index order).
__device__ void block_add_field(const float part[F], float *s_field, float (*s_red)[F]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < F; ++a) {
        float v = part[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_red[warp][a] = v;
    }
    __syncthreads();
    if (threadIdx.x < F) {
        float s = 0.f;
        for (int w = 0; w < kWarps; ++w) s += s_red[w][threadIdx.x];
        s_field[threadIdx.x] += s;
    }
    __syncthreads();
}

constexpr int kItemRoots = 0, kItemBodies = 1;

// Appends a near-field item for passive leaf `leaf` (bodies [first, first + size)): the payload is
// a[0..na) then b[0..nb) (activeTree roots), or for close bodies the runs of consecutive indices as
// (first index, length) pairs. The owning block is the only writer of the leaf's list head, so the
// list order is the block's task order. The first item of a leaf also registers its 32-target
// units for the near kernel. Called by every thread of the block.
__device__ void append_item(const NearPool &pool, int leaf, int first, int size, int kind, const int *a, int na,
                            const int *b, int nb, uint32_t *err, int *s_slot) {
    const int count = na + nb;
    if (count == 0) return;  // uniform
    if (threadIdx.x == 0) {
        int slot = -1;
        const unsigned long long it = atomicAdd(&pool.counters[0], 1ull);
        const unsigned long long off = atomicAdd(&pool.counters[1], (unsigned long long) count);
        bool ok = it < (unsigned long long) pool.item_cap && off + count <= (unsigned long long) pool.word_cap &&
                  leaf < pool.head_cap;
        const int old = ok ? pool.head[leaf] : -1;
        if (ok && old < 0) {
            const int nunits = (size + 31) / 32;
            const unsigned long long u = atomicAdd(&pool.counters[2], (unsigned long long) nunits);
            ok = u + nunits <= (unsigned long long) pool.unit_cap;
            if (ok)
                for (int j = 0; j < nunits; ++j) pool.units[u + j] = make_int2(leaf, first + 32 * j);
        }
        if (ok) {
            pool.items[it] = make_int4(old, kind, (int) off, count);
            pool.head[leaf] = (int) it;
            slot = (int) off;
        } else {
            atomicOr(err, (uint32_t) kErrNearPool);
        }
        *s_slot = slot;
    }
    __syncthreads();
    const int off = *s_slot;
    if (off >= 0) {
        for (int i = threadIdx.x; i < na; i += kThreads) pool.words[off + i] = a[i];
        for (int i = threadIdx.x; i < nb; i += kThreads) pool.words[off + na + i] = b[i];
    }
}

// Hands the tasks of children `right` / `left` (where spill_r / spill_l) to the frontier kernel:
// one copy of their shared list and one field each, linked to the child's record list. Only the
// block that owns a frontier node's ancestors appends to its list, so the order is that block's
// task order. The first record of a node registers it in the work list. Called by every thread.
__device__ void spill_children(const SpillPool &sp, int type, const int *list, int len, const float *field_r,
                               const float *field_l, int right, int left, bool spill_r, bool spill_l, uint32_t *err,
                               int *s_slot) {
    const int nrec = (spill_r ? 1 : 0) + (spill_l ? 1 : 0);
    if (nrec == 0) return;  // uniform
    if (threadIdx.x == 0) {
        int slot = -1;
        const unsigned long long words = (unsigned long long) len + (unsigned long long) F * nrec;
        const unsigned long long rec = atomicAdd(&sp.counters[0], (unsigned long long) nrec);
        const unsigned long long off = atomicAdd(&sp.counters[1], words);
        if (rec + nrec <= (unsigned long long) sp.rec_cap && off + words <= (unsigned long long) sp.word_cap &&
            right < sp.head_cap && left < sp.head_cap) {
            int k = 0;
            for (int side = 0; side < 2; ++side) {
                const bool on = side == 0 ? spill_r : spill_l;
                if (!on) continue;
                const int c = side == 0 ? right : left;
                const int r = (int) rec + k;
                const int old = sp.head[c];
                sp.recs[r] = make_int4(old, type, (int) off, len);
                sp.rec_field[r] = (int) off + len + F * k;
                sp.head[c] = r;
                if (old < 0) {
                    const unsigned long long w = atomicAdd(&sp.counters[2], 1ull);
                    if (w < (unsigned long long) sp.work_cap) sp.work[w] = c;
                    else atomicOr(err, (uint32_t) kErrNearPool);
                }
                ++k;
            }
            slot = (int) off;
        } else {
            atomicOr(err, (uint32_t) kErrNearPool);
        }
        s_slot[0] = slot;
    }
    __syncthreads();
    const int off = s_slot[0];
    if (off < 0) return;
    for (int i = threadIdx.x; i < len; i += kThreads) sp.words[off + i] = list[i];
    int k = 0;
    for (int side = 0; side < 2; ++side) {
        const bool on = side == 0 ? spill_r : spill_l;
        if (!on) continue;
        const float *f = side == 0 ? field_r : field_l;
        for (int a = threadIdx.x; a < F; a += kThreads) sp.words[off + len + F * k + a] = __float_as_int(f[a]);
        ++k;
    }
}

__device__ __forceinline__ int node_size(const DualNodes &N, int k) { return __float_as_int(__ldg(N.bmin + k).w); }

__device__ __forceinline__ void push_task(int *t, int type, int node, int list, int len, int field, int top) {
    t[0] = type; t[1] = node; t[2] = list; t[3] = len; t[4] = field; t[5] = top;
}

// FRONTIER = false: one block per start node; tasks of frontier nodes (at most `frontier` bodies,
// parent above) are spilled. FRONTIER = true: blocks take frontier nodes from the work list and
// run their spilled tasks, in record order, to completion. Only targets in [t_lo, t_hi) are
// evaluated: a task whose passive node holds none of them is dropped with everything below it,
// and the tasks that remain run exactly as in an unrestricted pass.
// Four blocks per SM (64 registers; the per-thread field accumulators spill a little): the task
// loop is latency- and barrier-bound, so resident blocks matter more than the spills.
template<bool FRONTIER>
__global__ void __launch_bounds__(kThreads, 4) dual_kernel(DualNodes nodes, const int *__restrict__ num_nodes,
                                                        const float4 *__restrict__ bodies, int n, float G,
                                                        float eps, float theta, float4 *__restrict__ acc,
                                                        unsigned long long *__restrict__ counts,
                                                        const int *__restrict__ roots, const int *__restrict__ num_roots,
                                                        int *__restrict__ arena_all, int arena_words,
                                                        int *__restrict__ tasks_all, NearPool pool, SpillPool spill,
                                                        int frontier, int t_lo, int t_hi,
                                                        uint32_t *__restrict__ err) {
    __shared__ float s_field[F];
    __shared__ float s_child[2][F];
    __shared__ float s_red[kWarps][F];
    __shared__ int s_task[kTaskInts];
    __shared__ Scan3 s_scan;
    __shared__ int s_w[kWarps];
    __shared__ int s_ntask, s_fail, s_slot, s_work;

    if (!FRONTIER && (int) blockIdx.x >= *num_roots) return;  // uniform across the block
    const int tid = threadIdx.x;
    const Ctx x{nodes, bodies, G, eps, theta, *num_nodes, n};
    int *arena = arena_all + (int64_t) blockIdx.x * arena_words;
    float *farena = reinterpret_cast<float *>(arena);
    int *tasks = tasks_all + (int64_t) blockIdx.x * kDualTasks * kTaskInts;
    unsigned long long npn = 0, nnn = 0;
    // spill children at the frontier (first kernel only)
    const int spill_size = FRONTIER ? -1 : frontier;

    auto run_tasks = [&]() {

    // ---- depth-first task loop ----
    for (;;) {
        __syncthreads();
        const int nt = s_ntask;
        if (nt == 0) break;
        __syncthreads();
        if (tid == 0) {
            const int *t = tasks + (nt - 1) * kTaskInts;
            for (int k = 0; k < kTaskInts; ++k) s_task[k] = t[k];
            s_ntask = nt - 1;
        }
        if (tid < 3) s_scan.base[tid] = 0;
        __syncthreads();
        const int type = s_task[0], pk = s_task[1], loff = s_task[2], len = s_task[3], foff = s_task[4];
        const int scratch = s_task[5];
        const DNode P = load_node(nodes, pk);
        const float4 pthr = __ldg(nodes.thr + pk);
        float pc[3];
        center(P, pc);
        const int pfirst = P.first(), pend = pfirst + P.size;
        if (!x.range_ok(pfirst, pend) || (!P.leaf() && !(x.left_ok(pk) && x.right_ok(pk, P.link0)))) {
            if (tid == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
            continue;
        }
        if (pend <= t_lo || pfirst >= t_hi) continue;  // no target of this pass below the passive node
        if (tid < F) s_field[tid] = foff >= 0 ? farena[foff + tid] : 0.f;
        __syncthreads();

        if (type == kLockstep && len == 0) {
            // no active nodes remain: evaluate the local field at every body of the passive node
            for (int b = pfirst + tid; b < pend; b += kThreads) {
                const float4 q = __ldg(bodies + b);
                const float o[3] = {fsub(q.x, pc[0]), fsub(q.y, pc[1]), fsub(q.z, pc[2])};
                float a[3];
                st::field_at(s_field, o, a);
                float4 v = acc[b];
                v.x += a[0]; v.y += a[1]; v.z += a[2];
                acc[b] = v;
            }
            continue;
        }

        // arena needed by this task above `scratch`: the three class lists, the deeper list (or the
        // close-body runs) and two child fields (the leaf-body list is checked once its length is known)
        const int64_t need = 5 * (int64_t) len + 2 * F;
        if ((int64_t) scratch + need >= arena_words) {
            if (tid == 0) atomicOr(err, (uint32_t) kErrDualArena);
            continue;
        }
        const int *list = arena + loff;
        int *c1 = arena + scratch + len, *c2 = c1 + len;
        int *c0 = arena + scratch;  // scratch for leaf-body offsets (far entries are not stored)

        // ---- classify the list (stable compaction): far c0, leaf / close c1, non-leaf c2 ----
        if (type == kLockstep) {
            stable_partition(list, len, c0, c1, c2, s_scan, [&](int e) {
                const DNode A = load_node(nodes, e);
                int cls;
                if (node_node(A, P, theta) == 0) cls = 0;
                else if (A.leaf()) cls = x.range_ok(A.link0, A.link1) ? 1 : -1;
                else cls = (x.left_ok(e) && x.right_ok(e, A.link0)) ? 2 : -1;
                if (cls < 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
                return cls;
            });
        } else {
            stable_partition(list, len, c0, c1, c2, s_scan, [&](int e) {
                const float4 q = __ldg(bodies + e);
                const float pe[3] = {q.x, q.y, q.z};
                return point_is_far(pe, P, pthr) ? 0 : 1;
            });
        }
        __syncthreads();  // the compacted lists are read by other threads below
        const int nfar = s_scan.base[0], nleaf = s_scan.base[1], nnon = s_scan.base[2];

        // ---- far entries into the local field: M2L (lock-step) or P2L (passive tree) ----
        if (type == kLockstep) {
            float part[F];
#pragma unroll
            for (int a = 0; a < F; ++a) part[a] = 0.f;
            for (int i = tid; i < nfar; i += kThreads) {
                const int e = c0[i];
                m2l(x, e, load_node(nodes, e), pc, part);
                ++nnn;
            }
            block_add_field(part, s_field, s_red);
        } else {
            float part[F];
#pragma unroll
            for (int a = 0; a < F; ++a) part[a] = 0.f;
            for (int i = tid; i < nfar; i += kThreads) {
                p2l(x, __ldg(bodies + c0[i]), pc, part);
                ++npn;
            }
            block_add_field(part, s_field, s_red);
        }

        if (P.leaf()) {
            // ---- passive leaf: L2P of this task's field; the near field goes to the leaf's items ----
            for (int b = pfirst + tid; b < pend; b += kThreads) {
                const float4 q = __ldg(bodies + b);
                const float o[3] = {fsub(q.x, pc[0]), fsub(q.y, pc[1]), fsub(q.z, pc[2])};
                float a[3];
                st::field_at(s_field, o, a);
                float4 w = acc[b];
                w.x += a[0];
                w.y += a[1];
                w.z += a[2];
                acc[b] = w;
            }
            if (type == kLockstep) {
                append_item(pool, pk, pfirst, P.size, kItemRoots, c1, nleaf, c2, nnon, err, &s_slot);
            } else {
                // close bodies as runs of consecutive indices: run starts in c0 (free once the far
                // terms are summed), then (first body, length) pairs in c2 (room for 2 len words)
                for (int i0 = 0; i0 < nleaf; i0 += kThreads) {
                    const int i = i0 + tid;
                    const bool start = i < nleaf && (i == 0 || c1[i] != c1[i - 1] + 1);
                    const int pos = stable_rank(start ? 0 : -1, s_scan);
                    if (start) c0[pos - nfar] = i;  // base[0] already counted the far entries
                }
                __syncthreads();
                const int runs = s_scan.base[0] - nfar;
                for (int r = tid; r < runs; r += kThreads) {
                    const int i = c0[r];
                    const int next = r + 1 < runs ? c0[r + 1] : nleaf;
                    c2[2 * r] = c1[i];
                    c2[2 * r + 1] = next - i;
                }
                __syncthreads();
                append_item(pool, pk, pfirst, P.size, kItemBodies, c2, 2 * runs, c2, 0, err, &s_slot);
            }
            continue;
        }

        // ---- internal passive node: translate the field to both children ----
        const int left = pk + 1, right = P.link0;
        if (tid == 0 || tid == 32) {
            const DNode C = load_node(nodes, tid == 0 ? left : right);
            float cc[3];
            center(C, cc);
            const float o[3] = {fsub(cc[0], pc[0]), fsub(cc[1], pc[1]), fsub(cc[2], pc[2])};
            st::field_translated(s_field, o, s_child[tid == 0 ? 0 : 1]);
        }
        __syncthreads();
        const int top = scratch + 3 * len;
        if (type == kPassive) {
            // children see the close bodies with their translated fields; left runs first
            const int fr = top, fl = top + F;
            for (int a = tid; a < F; a += kThreads) {
                farena[fr + a] = s_child[1][a];
                farena[fl + a] = s_child[0][a];
            }
            const bool sp_r = spill_size >= 0 && P.size > spill_size && node_size(nodes, right) <= spill_size;
            const bool sp_l = spill_size >= 0 && P.size > spill_size && node_size(nodes, left) <= spill_size;
            spill_children(spill, kPassive, c1, nleaf, s_child[1], s_child[0], right, left, sp_r, sp_l, err, &s_slot);
            if (tid == 0) {
                const int pushes = (sp_r ? 0 : 1) + (sp_l ? 0 : 1);
                if (nt - 1 + pushes <= kDualTasks) {
                    int *t = tasks + (nt - 1) * kTaskInts;
                    if (!sp_r) {
                        push_task(t, kPassive, right, scratch + len, nleaf, fr, fr + F);
                        t += kTaskInts;
                    }
                    if (!sp_l) push_task(t, kPassive, left, scratch + len, nleaf, fl, fl + F);
                    s_ntask = nt - 1 + pushes;
                } else {
                    atomicOr(err, (uint32_t) kErrDualArena);
                }
            }
            continue;
        }

        // lock-step at an internal passive node: the children of the non-leaf active nodes form the
        // deeper list shared by both passive children; the bodies of the leaf active nodes go
        // through passiveTree over this passive node first (with an empty field)
        const int dp = top;
        for (int i = tid; i < nnon; i += kThreads) {
            const int a = c2[i];
            arena[dp + 2 * i] = a + 1;
            arena[dp + 2 * i + 1] = __ldg(nodes.link + a).x;
        }
        const int fr = dp + 2 * nnon, fl = fr + F, lb = fl + F;
        for (int a = tid; a < F; a += kThreads) {
            farena[fr + a] = s_child[1][a];
            farena[fl + a] = s_child[0][a];
        }
        int total = 0;
        for (int i0 = 0; i0 < nleaf; i0 += kThreads) {
            const int i = i0 + tid;
            int sz = 0;
            if (i < nleaf) {
                const int2 l = __ldg(nodes.link + c1[i]);
                sz = l.y - l.x;
            }
            int chunk = 0;
            const int off = block_exclusive_scan(sz, s_w, chunk);
            if (i < nleaf) c0[i] = total + off;
            total += chunk;
        }
        const bool fits = (int64_t) lb + total < arena_words;
        if (fits) {
            for (int i = tid; i < nleaf; i += kThreads) {
                const int2 l = __ldg(nodes.link + c1[i]);
                int *dst = arena + lb + c0[i];
                for (int b = l.x; b < l.y; ++b) dst[b - l.x] = b;
            }
        }
        const bool sp_r = spill_size >= 0 && P.size > spill_size && node_size(nodes, right) <= spill_size;
        const bool sp_l = spill_size >= 0 && P.size > spill_size && node_size(nodes, left) <= spill_size;
        spill_children(spill, kLockstep, arena + dp, 2 * nnon, s_child[1], s_child[0], right, left, sp_r, sp_l, err,
                       &s_slot);
        if (tid == 0) {
            const int pushes = (sp_r ? 0 : 1) + (sp_l ? 0 : 1) + (total > 0 ? 1 : 0);
            if (!fits || nt - 1 + pushes > kDualTasks) {
                atomicOr(err, (uint32_t) kErrDualArena);
            } else {
                int *t = tasks + (nt - 1) * kTaskInts;
                if (!sp_r) {
                    push_task(t, kLockstep, right, dp, 2 * nnon, fr, fr + F);
                    t += kTaskInts;
                }
                if (!sp_l) {
                    push_task(t, kLockstep, left, dp, 2 * nnon, fl, fl + F);
                    t += kTaskInts;
                }
                if (total > 0) push_task(t, kPassive, pk, lb, total, -1, lb + total);
                s_ntask = nt - 1 + pushes;
            }
        }
    }

    };  // run_tasks

    if (!FRONTIER) {
        const int root = roots[blockIdx.x];
        if (root < 0 || root >= x.nn || x.nn <= 0) {
            if (tid == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
            return;
        }
        const DNode Rt = load_node(nodes, root);
        // ---- balancedLockstepDualTreeImplicitField: breadth-first over the active tree from its root;
        // a node joins the starting list unless the criterion says "descend the active node" only and
        // it is not a leaf, in which case its children join the next level ----
        const int eq_cap = arena_words / 4;
        int cur = eq_cap, curlen = 1;
        if (tid == 0) {
            arena[cur] = 0;
            s_fail = 0;
        }
        if (tid < 3) s_scan.base[tid] = 0;
        __syncthreads();
        while (curlen > 0) {
            const int nxt = cur + curlen;
            for (int i0 = 0; i0 < curlen; i0 += kThreads) {
                const int i = i0 + tid;
                int a = -1, cls = -1, right = -1;
                if (i < curlen) {
                    a = arena[cur + i];
                    const DNode A = load_node(nodes, a);
                    const int rec = node_node(A, Rt, theta);
                    cls = (rec != 1 || A.leaf()) ? 0 : 1;
                    right = A.link0;
                    if (cls == 1 && !(x.left_ok(a) && x.right_ok(a, right))) {
                        atomicOr(err, (uint32_t) kErrTraverseLimit);
                        cls = -1;
                    }
                }
                const int pos = stable_rank(cls, s_scan);
                if (cls == 0) {
                    if (pos < eq_cap) arena[pos] = a;
                    else s_fail = 1;
                } else if (cls == 1) {
                    if ((int64_t) nxt + 2 * (int64_t) pos + 1 < arena_words) {
                        arena[nxt + 2 * pos] = a + 1;
                        arena[nxt + 2 * pos + 1] = right;
                    } else {
                        s_fail = 1;
                    }
                }
            }
            __syncthreads();
            const int nextlen = 2 * s_scan.base[1];
            const bool failed = s_fail != 0;
            __syncthreads();
            if (tid == 1) s_scan.base[1] = 0;
            cur = nxt;
            curlen = failed ? 0 : nextlen;
        }
        __syncthreads();
        if (tid == 0) {
            const int eq = min(s_scan.base[0], eq_cap);
            push_task(tasks, kLockstep, root, 0, eq, -1, eq);
            s_ntask = 1;
            if (s_fail) atomicOr(err, (uint32_t) kErrDualArena);
        }
        run_tasks();
    } else {
        const unsigned long long nwork = min(spill.counters[2], (unsigned long long) spill.work_cap);
        const unsigned long long nrecs = min(spill.counters[0], (unsigned long long) spill.rec_cap);
        for (;;) {
            __syncthreads();
            if (tid == 0) s_work = (int) min(atomicAdd(&spill.counters[3], 1ull), (unsigned long long) INT_MAX);
            __syncthreads();
            const int w = s_work;
            if ((unsigned long long) w >= nwork) break;
            const int c = spill.work[w];
            if (c < 0 || c >= x.nn) {
                if (tid == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
                continue;
            }
            int guard = 0;
            for (int r = spill.head[c]; r >= 0; ++guard) {
                if ((unsigned long long) r >= nrecs || guard > (1 << 20)) {
                    if (tid == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
                    break;
                }
                const int4 rec = spill.recs[r];
                const int fo = spill.rec_field[r];
                const int len = rec.w;
                if (len < 0 || (int64_t) len + F >= arena_words) {
                    if (tid == 0) atomicOr(err, (uint32_t) kErrDualArena);
                    r = rec.x;
                    continue;
                }
                for (int i = tid; i < len; i += kThreads) arena[i] = spill.words[rec.z + i];
                for (int a = tid; a < F; a += kThreads) arena[len + a] = spill.words[fo + a];
                if (tid == 0) {
                    push_task(tasks, rec.y, c, 0, len, len, len + F);
                    s_ntask = 1;
                }
                __syncthreads();
                run_tasks();
                // every thread has read the empty task count before thread 0 sets up the next record
                __syncthreads();
                r = rec.x;
            }
        }
    }

    // interaction counts {particle-node, node-node} (the near kernel counts the other two)
    const unsigned long long c[2] = {npn, nnn};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        unsigned long long v = c[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0 && v) atomicAdd(counts + 2 + k, v);
    }
}

// Tree::loadBalancedBreak(256) (Tree.h:84-107): split the node with the most bodies until 256
// starting nodes exist or the largest is a leaf. The heap steps restate libstdc++'s
// std::pop_heap / std::push_heap (__adjust_heap, __push_heap) so that ties between equal sizes
// resolve as on the host. One thread; (size, node) pairs in shared memory.
__global__ void load_balanced_break_kernel(DualNodes nodes, const int *__restrict__ num_nodes, int *__restrict__ roots,
                                           int *__restrict__ num_roots, uint32_t *__restrict__ err) {
    __shared__ int hs[kDualRoots + 2], hn[kDualRoots + 2];
    if (threadIdx.x != 0) return;
    const int nn = *num_nodes;
    if (nn <= 0) {
        *num_roots = 0;
        return;
    }
    auto push_up = [&](int hole, int top, int vs, int vn) {
        int parent = (hole - 1) / 2;
        while (hole > top && hs[parent] < vs) {
            hs[hole] = hs[parent];
            hn[hole] = hn[parent];
            hole = parent;
            parent = (hole - 1) / 2;
        }
        hs[hole] = vs;
        hn[hole] = vn;
    };
    auto pop_heap = [&](int len) {
        if (len <= 1) return;
        const int L = len - 1;
        const int vs = hs[L], vn = hn[L];
        hs[L] = hs[0];
        hn[L] = hn[0];
        int hole = 0, child = 0;
        while (child < (L - 1) / 2) {
            child = 2 * (child + 1);
            if (hs[child] < hs[child - 1]) child--;
            hs[hole] = hs[child];
            hn[hole] = hn[child];
            hole = child;
        }
        if ((L & 1) == 0 && child == (L - 2) / 2) {
            child = 2 * (child + 1);
            hs[hole] = hs[child - 1];
            hn[hole] = hn[child - 1];
            hole = child - 1;
        }
        push_up(hole, 0, vs, vn);
    };
    auto size_of = [&](int k) { return __float_as_int(__ldg(nodes.bmin + k).w); };
    int len = 1;
    hs[0] = size_of(0);
    hn[0] = 0;
    while (len < kDualRoots) {
        pop_heap(len);
        const int k = hn[len - 1];
        const int2 l = __ldg(nodes.link + k);
        if (l.y >= 0) break;  // the largest node is a leaf
        if (!(k + 1 < nn && l.x > k + 1 && l.x < nn)) {
            atomicOr(err, (uint32_t) kErrTraverseLimit);
            break;
        }
        len -= 1;
        for (int c: {k + 1, l.x}) {
            hs[len] = size_of(c);
            hn[len] = c;
            len += 1;
            push_up(len - 1, 0, hs[len - 1], hn[len - 1]);
        }
    }
    for (int i = 0; i < len; ++i) roots[i] = hn[i];
    *num_roots = len;
}


// ---------------------------------------------------------------------------------------------
// Near field of the passive leaves (second kernel).
//
// A unit is up to 32 targets of one passive leaf. With T targets, the warp runs G = 32 / T
// replicas of each: lane l serves target l % T as replica l / T. Decisions are per target (every
// replica of a target computes the same criterion); pair tiles and queued M2P terms are split
// between the replicas, whose partial sums are added in replica order at the end of the unit. So
// short leaves still keep the whole warp busy. Terms are summed without G; G is applied once.

constexpr int kNearThreads = 128;  // 4 warps: their slabs and lists fit in 48 KB of static shared memory
constexpr int kNearWarps = kNearThreads / 32;
// A round of the walk adds at most 32 entries to each slab and list, which therefore hold 32.
constexpr int kM2pFull = 32;  // staged nodes approximated for every target of the unit
constexpr int kM2pPart = 32;  // staged nodes approximated for some targets (one 32-entry mask block)
constexpr int kM2pRec = 5;    // float4 per staged node: (com, mass), quadrupole and octupole

constexpr int kNearLeaves = 32;  // opened leaves of a walk waiting for their pair tiles

static_assert(kM2pFull >= 32 && kM2pPart >= 32 && kNearLeaves >= 32, "a round adds up to 32 entries");

struct NearWarp {
    float4 m2p_full[kM2pFull * kM2pRec];  // node records approximated for every target
    float4 m2p_part[(kM2pPart + 1) * kM2pRec];  // node records approximated for some targets, then a null record
    unsigned part_mask[kM2pPart];         // their target masks
    float4 tile[32];      // staged source bodies (16 interleaved pairs), then the replicas' partial sums
    float4 tpos[32];      // the unit's targets (replica-0 lanes)
    int4 leaf[kNearLeaves];  // opened leaves: (first body, end body, target mask, 0)
};

struct Lane {
    int t, r, T, G;     // target, replica, targets in the unit, replicas
    bool active;        // r < G
    bool counted;       // replica 0 of a target of this pass (its interactions are counted)
};

// Gravity::nodeParticle for MultipoleMassSummary<3> (Gravity.h:239-259) without G, added into a:
//   a += -M R / r^3 + (D3 : Q2) / 2 - (D4 : Q3) / 6,
// with the two full contractions (SymmetricTensor3.h:281-292) written out for symmetric moments:
//   (D3 : Q2)_i = g3 R_i (R.Q2.R) + g2 (2 (Q2 R)_i + R_i tr Q2)
//   (D4 : Q3)_i = g4 R_i (Q3 : RRR) + 3 g3 ((Q3 : RR)_i + R_i (t.R)) + 3 g2 t_i,  t_i = Q3_ikk,
// which is the same sum over index tuples, grouped (about 100 flops instead of about 550).
// c4 = (centre of mass, mass), qa..qd = packed quadrupole (6) and octupole (10), as stored.
__device__ __forceinline__ void m2p_term(float4 c4, float4 qa, float4 qb, float4 qc, float4 qd, float eps,
                                         const float p[3], float a[3]) {
    const float rx = p[0] - c4.x, ry = p[1] - c4.y, rz = p[2] - c4.z;
    if (rx == 0.f && ry == 0.f && rz == 0.f) return;
    const float inv = rsqrt_hw(fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps))));
    const float i2 = inv * inv, i3 = inv * i2, i5 = i3 * i2, i7 = i5 * i2, i9 = i7 * i2;
    const float g2 = 3.0f * i5, g3 = -15.0f * i7, g4 = 105.0f * i9;
    // quadrupole xx xy xz yy yz zz; octupole xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz
    const float Qxx = qa.x, Qxy = qa.y, Qxz = qa.z, Qyy = qa.w, Qyz = qb.x, Qzz = qb.y;
    const float Oxxx = qb.z, Oxxy = qb.w, Oxxz = qc.x, Oxyy = qc.y, Oxyz = qc.z, Oxzz = qc.w;
    const float Oyyy = qd.x, Oyyz = qd.y, Oyzz = qd.z, Ozzz = qd.w;
    // (D3 : Q2) / 2
    const float qrx = fmaf(Qxx, rx, fmaf(Qxy, ry, Qxz * rz));
    const float qry = fmaf(Qxy, rx, fmaf(Qyy, ry, Qyz * rz));
    const float qrz = fmaf(Qxz, rx, fmaf(Qyz, ry, Qzz * rz));
    const float rqr = fmaf(rx, qrx, fmaf(ry, qry, rz * qrz));
    const float trq = Qxx + Qyy + Qzz;
    const float s2r = 0.5f * fmaf(g3, rqr, g2 * trq), s2q = g2;  // R_i s2r + (Q2 R)_i s2q
    // (D4 : Q3) / 6
    const float xx = rx * rx, xy = rx * ry, xz = rx * rz, yy = ry * ry, yz = ry * rz, zz = rz * rz;
    const float ox = fmaf(Oxxx, xx, fmaf(2.0f * Oxxy, xy, fmaf(2.0f * Oxxz, xz, fmaf(Oxyy, yy, fmaf(2.0f * Oxyz, yz, Oxzz * zz)))));
    const float oy = fmaf(Oxxy, xx, fmaf(2.0f * Oxyy, xy, fmaf(2.0f * Oxyz, xz, fmaf(Oyyy, yy, fmaf(2.0f * Oyyz, yz, Oyzz * zz)))));
    const float oz = fmaf(Oxxz, xx, fmaf(2.0f * Oxyz, xy, fmaf(2.0f * Oxzz, xz, fmaf(Oyyz, yy, fmaf(2.0f * Oyzz, yz, Ozzz * zz)))));
    const float orrr = fmaf(rx, ox, fmaf(ry, oy, rz * oz));
    const float tx = Oxxx + Oxyy + Oxzz, ty = Oxxy + Oyyy + Oyzz, tz = Oxxz + Oyyz + Ozzz;
    const float tr = fmaf(tx, rx, fmaf(ty, ry, tz * rz));
    const float s4r = fmaf(g4, orrr, 3.0f * g3 * tr) * (1.0f / 6.0f);  // R_i s4r + O_i s4o + t_i s4t
    const float s4o = 0.5f * g3, s4t = 0.5f * g2;
    const float sr = fmaf(-c4.w, i3, s2r - s4r);
    a[0] += fmaf(rx, sr, fmaf(qrx, s2q, -fmaf(ox, s4o, tx * s4t)));
    a[1] += fmaf(ry, sr, fmaf(qry, s2q, -fmaf(oy, s4o, ty * s4t)));
    a[2] += fmaf(rz, sr, fmaf(qrz, s2q, -fmaf(oz, s4o, tz * s4t)));
}

// The node term from a node record staged in shared memory: (com, mass) then the four moment float4.
__device__ __forceinline__ void m2p_staged(const float4 *pc, float eps, const float p[3], float a[3]) {
    m2p_term(pc[0], pc[1], pc[2], pc[3], pc[4], eps, p, a);
}

// Pairs of the unit's targets with sources src(0..m) for lanes in `mine`. 32 sources at a time are
// staged in shared memory as 16 interleaved pairs (sources 2j and 2j+1 in one 32-byte record, so
// that each 16-byte load yields two register pairs); replica r takes pairs r, r + G, ...
// Pairs of the unit's targets with the c sources staged in the warp's tile, for lanes in `mine`;
// replica r takes pairs r, r + G, ...
template<bool EPS0>
__device__ __forceinline__ void tile_pairs(NearWarp &w, const Lane &L, int c, bool mine, float2 npx, float2 npy,
                                           float2 npz, float2 eps2, float2 &ax, float2 &ay, float2 &az) {
    if (!mine) return;
    const int np = (c + 1) >> 1;
    const int G = L.G;
    int k = L.r;
    for (; k + 3 * G < np; k += 4 * G) {
        const float4 u0 = w.tile[2 * k], v0 = w.tile[2 * k + 1];
        const float4 u1 = w.tile[2 * (k + G)], v1 = w.tile[2 * (k + G) + 1];
        const float4 u2 = w.tile[2 * (k + 2 * G)], v2 = w.tile[2 * (k + 2 * G) + 1];
        const float4 u3 = w.tile[2 * (k + 3 * G)], v3 = w.tile[2 * (k + 3 * G) + 1];
        pair2_term<EPS0>(npx, npy, npz, eps2, u0, v0, ax, ay, az);
        pair2_term<EPS0>(npx, npy, npz, eps2, u1, v1, ax, ay, az);
        pair2_term<EPS0>(npx, npy, npz, eps2, u2, v2, ax, ay, az);
        pair2_term<EPS0>(npx, npy, npz, eps2, u3, v3, ax, ay, az);
    }
    for (; k < np; k += G) pair2_term<EPS0>(npx, npy, npz, eps2, w.tile[2 * k], w.tile[2 * k + 1], ax, ay, az);
}

// Padding of a partly filled tile: no mass, at 1e30 on every axis, where the squared distance from
// any target with coordinates below 1e29 in magnitude overflows to infinity; its reciprocal root
// and every factor of its term are then exactly zero (a source at the origin would give 0 * inf
// for a target within about 1e-13 of the origin when the softening is zero).
__device__ __constant__ const float4 kNullSource = {1e30f, 1e30f, 1e30f, 0.f};

// Stages one source per lane (the null source past the end) as 16 interleaved
// pairs: sources 2j and 2j+1 in one 32-byte record, so that each 16-byte load yields two register
// pairs.
__device__ __forceinline__ void stage_tile(NearWarp &w, float4 b) {
    const int lane = threadIdx.x & 31;
    float *tf = reinterpret_cast<float *>(w.tile);
    const int slot = (lane >> 1) * 8 + (lane & 1);
    tf[slot] = b.x;
    tf[slot + 2] = b.y;
    tf[slot + 4] = b.z;
    tf[slot + 6] = b.w;
}

// Pairs of the unit's targets with sources src(0..m) for lanes in `mine`, 32 sources per tile.
template<bool EPS0, typename Src>
__device__ __forceinline__ void pair_tile(NearWarp &w, const Lane &L, int m, Src src, bool mine, const float p[3],
                                          float eps, float a[3]) {
    const int lane = threadIdx.x & 31;
    const float2 npx = make_float2(-p[0], -p[0]), npy = make_float2(-p[1], -p[1]), npz = make_float2(-p[2], -p[2]);
    const float2 eps2 = make_float2(eps, eps);
    float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax;
    for (int j0 = 0; j0 < m; j0 += 32) {
        const int c = min(32, m - j0);
        stage_tile(w, lane < c ? src(j0 + lane) : kNullSource);
        __syncwarp();
        tile_pairs<EPS0>(w, L, c, mine, npx, npy, npz, eps2, ax, ay, az);
        __syncwarp();
    }
    a[0] += ax.x + ax.y;
    a[1] += ay.x + ay.y;
    a[2] += az.x + az.y;
}

// Pairs of the unit's targets with the close bodies of one item, given as runs of consecutive
// bodies ((first body, length) pairs): the runs are packed back to back into 32-source tiles, so a
// short run does not cost a whole tile. Invalid runs are skipped with kErrTraverseLimit.
template<bool EPS0>
__device__ void run_tiles(const Ctx &x, NearWarp &w, const Lane &L, const int *words, int nwords, const float p[3],
                          float a[3], unsigned long long &npp, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const float2 npx = make_float2(-p[0], -p[0]), npy = make_float2(-p[1], -p[1]), npz = make_float2(-p[2], -p[2]);
    const float2 eps2 = make_float2(x.eps, x.eps);
    float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax;
    int r = 0, first = 0, len = 0, o = 0;  // next word, current run, offset in it
    for (;;) {
        int fill = 0;
        float4 b = kNullSource;
        while (fill < 32) {
            if (o == len) {  // the current run is used up: take the next valid one
                if (r + 1 >= nwords) break;
                first = words[r];
                len = words[r + 1];
                r += 2;
                o = 0;
                if (len < 0 || len > x.n || !x.range_ok(first, first + len)) {
                    if (lane == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
                    len = 0;
                    continue;
                }
                if (L.counted) npp += (unsigned long long) len;
                continue;
            }
            const int take = min(len - o, 32 - fill);
            if (lane >= fill && lane < fill + take) b = __ldg(x.bodies + first + o + (lane - fill));
            fill += take;
            o += take;
        }
        if (fill == 0) break;
        stage_tile(w, b);
        __syncwarp();
        tile_pairs<EPS0>(w, L, fill, L.active, npx, npy, npz, eps2, ax, ay, az);
        __syncwarp();
    }
    a[0] += ax.x + ax.y;
    a[1] += ay.x + ay.y;
    a[2] += az.x + az.y;
}

__device__ __forceinline__ void near_cp_async16(void *smem, const void *gmem) {
    const uint32_t a = (uint32_t) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void near_cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copies node k's record (centre of mass and mass, then the four moment float4) into a slab slot.
__device__ __forceinline__ void stage_m2p(float4 *dst, const DualNodes &N, int k) {
    near_cp_async16(dst, N.com + k);
    const float4 *q = N.q + (int64_t) k * 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) near_cp_async16(dst + 1 + i, q + i);
}

// Transpose of the 32 x 32 bit matrix whose row r is lane r's word: afterwards bit r of lane c's
// word is bit c of row r.
__device__ __forceinline__ uint32_t near_transpose32(uint32_t v, int lane) {
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
        const uint32_t hi = sh == 16 ? 0xFFFF0000u : sh == 8 ? 0xFF00FF00u : sh == 4 ? 0xF0F0F0F0u
                          : sh == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;
        const uint32_t y = __shfl_xor_sync(0xffffffffu, v, sh);
        v = (lane & sh) ? ((v & hi) | ((y & hi) >> sh)) : ((v & ~hi) | ((y & ~hi) << sh));
    }
    return v;
}

// M2P of the nodes approximated for every target: each target's replicas split the entries.
__device__ void flush_m2p_full(const Ctx &x, NearWarp &w, const Lane &L, int &nfull, const float p[3], float a[3],
                               unsigned long long &nnp) {
    near_cp_async_wait_all();
    __syncwarp();
    if (L.active)
        for (int j = L.r; j < nfull; j += L.G) m2p_staged(w.m2p_full + j * kM2pRec, x.eps, p, a);
    if (L.counted) nnp += (unsigned long long) nfull;
    nfull = 0;
    __syncwarp();
}

// M2P of the nodes approximated for some targets: the masks are transposed so that each target
// holds the set of entries it takes; its replicas split that set.
__device__ void flush_m2p_part(const Ctx &x, NearWarp &w, const Lane &L, int &npart, const float p[3], float a[3],
                               unsigned long long &nnp) {
    const int lane = threadIdx.x & 31;
    near_cp_async_wait_all();
    __syncwarp();
    const uint32_t mine_t = near_transpose32(lane < npart ? w.part_mask[lane] : 0u, lane);  // lane = target
    uint32_t bits = __shfl_sync(0xffffffffu, mine_t, L.t);
    if (!L.active) bits = 0u;
    if (L.counted) nnp += (unsigned long long) __popc(bits);
    if (L.G > 1) {  // replica r takes every G-th entry of its target's set, starting at the r-th
        uint32_t own = 0u;
        int idx = 0;
        for (uint32_t t = bits; t; t &= t - 1, ++idx)
            if (idx % L.G == L.r) own |= t & (0u - t);
        bits = own;
    }
    // a lane whose entries are used up evaluates the null record instead of branching
    while (__any_sync(0xffffffffu, bits != 0u)) {
        int j = kM2pPart;
        if (bits) {
            j = __ffs(bits) - 1;
            bits &= bits - 1;
        }
        m2p_staged(w.m2p_part + j * kM2pRec, x.eps, p, a);
    }
    npart = 0;
    __syncwarp();
}

enum : int { kGroupAccept = 1, kGroupOpen = 2, kGroupMixed = 3 };

// The point criterion decided for every target in the box [lo, hi] at once: a target's separation
// gaps are bounded below by the gaps to the box's nearest corner and above by those to its
// farthest one, computed with the same IEEE operations, and sep_test is non-decreasing in both
// squared lengths; so "all approximate" / "none approximates" are exact. A node of at most 32
// bodies is never approximated.
__device__ __forceinline__ int classify_group(const DNode &nd, float4 thr, const float lo[3], const float hi[3]) {
    if (nd.size <= 32) return kGroupOpen;
    const float su_lo = gap2(nd.mn[0], nd.mn[1], nd.mn[2], hi[0], hi[1], hi[2]);
    const float sv_lo = gap2(lo[0], lo[1], lo[2], nd.mx[0], nd.mx[1], nd.mx[2]);
    if (sep_test(su_lo, sv_lo, thr.x, thr.y)) return kGroupAccept;
    const float su_hi = gap2(nd.mn[0], nd.mn[1], nd.mn[2], lo[0], lo[1], lo[2]);
    const float sv_hi = gap2(hi[0], hi[1], hi[2], nd.mx[0], nd.mx[1], nd.mx[2]);
    if (!sep_test(su_hi, sv_hi, thr.x, thr.y)) return kGroupOpen;
    return kGroupMixed;
}

__device__ __forceinline__ uint32_t near_lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Pairs of the listed opened leaves with the targets that opened them (pair tiles, replicas split).
template<bool EPS0>
__device__ void flush_leaves(const Ctx &x, NearWarp &w, const Lane &L, int &nleaf, const float p[3], float a[3],
                             unsigned long long &npp) {
    for (int j = 0; j < nleaf; ++j) {
        const int4 lf = w.leaf[j];
        const bool mine = L.active && (((unsigned) lf.z >> L.t) & 1u);
        const int first = lf.x;
        pair_tile<EPS0>(w, L, lf.y - lf.x, [&](int jj) { return __ldg(x.bodies + first + jj); }, mine, p, x.eps, a);
        if (mine && L.counted) npp += (unsigned long long) (lf.y - lf.x);
    }
    nleaf = 0;
    __syncwarp();
}

// activeTree (activeTree.h:24-79) for the unit's targets from the `top` roots on the warp's stack,
// walked 32 entries per round: each lane classifies one (node, target mask) entry for the whole
// box of targets (classify_group), nodes left mixed are decided per target, approximated nodes are
// queued per target (M2P), opened leaves are listed for pair tiles, and opened internal nodes push
// both children with the targets that opened them. Every target takes exactly the reference's
// decisions; a round whose pushes would not fit the stack ends the walk with kErrStackOverflow.
template<bool EPS0>
__device__ void chunk_walk(const Ctx &x, NearWarp &w, const Lane &L, int2 *stack, int top, const float lo[3],
                           const float hi[3], const float p[3], float a[3], unsigned long long &npp,
                           unsigned long long &nnp, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = near_lanemask_lt();
    const unsigned tmask = L.T >= 32 ? 0xffffffffu : ((1u << L.T) - 1u);
    int nleaf = 0, nfull = 0, npart = 0;
    int64_t rounds = 0;
    const int64_t round_limit = 4 * (int64_t) x.nn + 64;
    while (top > 0) {
        if (++rounds > round_limit) {
            if (lane == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
            break;
        }
        const int k = min(32, top);
        const int base = top - k;
        top = base;
        int c = 0, l0 = 0, l1 = -1;
        unsigned A = 0, O = 0, m = 0;
        bool mixed = false;
        DNode nd;
        float4 thr = make_float4(0.f, 0.f, 0.f, 0.f);
        if (lane < k) {
            const int2 e = stack[base + lane];
            c = e.x;
            m = (unsigned) e.y;
            nd = load_node(x.nodes, c);
            thr = __ldg(x.nodes.thr + c);
            l0 = nd.link0;
            l1 = nd.link1;
            const int cls = classify_group(nd, thr, lo, hi);
            if (cls == kGroupAccept) A = m;
            else if (cls == kGroupOpen) O = m;
            else mixed = true;
        }
        // nodes left mixed: decided per target, one node at a time, every lane testing its own
        // target (lane t < T holds target t)
        for (unsigned mb = __ballot_sync(0xffffffffu, mixed); mb; mb &= mb - 1) {
            const int src = __ffs(mb) - 1;
            DNode q;
            q.mn[0] = __shfl_sync(0xffffffffu, nd.mn[0], src);
            q.mn[1] = __shfl_sync(0xffffffffu, nd.mn[1], src);
            q.mn[2] = __shfl_sync(0xffffffffu, nd.mn[2], src);
            q.mx[0] = __shfl_sync(0xffffffffu, nd.mx[0], src);
            q.mx[1] = __shfl_sync(0xffffffffu, nd.mx[1], src);
            q.mx[2] = __shfl_sync(0xffffffffu, nd.mx[2], src);
            const float B = __shfl_sync(0xffffffffu, thr.x, src), S = __shfl_sync(0xffffffffu, thr.y, src);
            const bool yes = lane < L.T && sep_at_least(q, p, B, S);
            const unsigned bits = __ballot_sync(0xffffffffu, yes);
            if (lane == src) {
                A = bits & m;
                O = m & ~A;
            }
        }
        __syncwarp();  // popped entries are read before children overwrite them
        const bool is_leaf = O != 0 && l1 >= 0, is_inner = O != 0 && l1 < 0;
        const bool leaf_ok = is_leaf && x.range_ok(l0, l1);
        const bool inner_ok = is_inner && x.left_ok(c) && x.right_ok(c, l0);
        if ((is_leaf && !leaf_ok) || (is_inner && !inner_ok)) atomicOr(err, (uint32_t) kErrTraverseLimit);
        // approximated: node records staged once per unit (cp.async); every target's, or some
        // targets' with their mask
        const bool acc_all = A != 0 && A == tmask, acc_some = A != 0 && A != tmask;
        uint32_t b = __ballot_sync(0xffffffffu, acc_all);
        if (b) {
            if (nfull + __popc(b) > kM2pFull) flush_m2p_full(x, w, L, nfull, p, a, nnp);
            if (acc_all) stage_m2p(w.m2p_full + (nfull + __popc(b & lt)) * kM2pRec, x.nodes, c);
            nfull += __popc(b);
        }
        b = __ballot_sync(0xffffffffu, acc_some);
        if (b) {
            if (npart + __popc(b) > kM2pPart) flush_m2p_part(x, w, L, npart, p, a, nnp);
            if (acc_some) {
                const int slot = npart + __popc(b & lt);
                stage_m2p(w.m2p_part + slot * kM2pRec, x.nodes, c);
                w.part_mask[slot] = A;
            }
            npart += __popc(b);
        }
        // opened leaves: listed, pair tiles when the list could overflow
        b = __ballot_sync(0xffffffffu, leaf_ok);
        if (nleaf + __popc(b) > kNearLeaves) flush_leaves<EPS0>(x, w, L, nleaf, p, a, npp);
        if (leaf_ok) w.leaf[nleaf + __popc(b & lt)] = make_int4(l0, l1, (int) O, 0);
        nleaf += __popc(b);
        // opened internal nodes: both children, left popped first
        b = __ballot_sync(0xffffffffu, inner_ok);
        if (top + 2 * __popc(b) > kNearWalkStack) {
            if (lane == 0) atomicOr(err, (uint32_t) kErrStackOverflow);
            top = 0;
        } else {
            if (inner_ok) {
                const int sp = top + 2 * __popc(b & lt);
                stack[sp] = make_int2(l0, (int) O);
                stack[sp + 1] = make_int2(c + 1, (int) O);
            }
            top += 2 * __popc(b);
        }
        __syncwarp();
    }
    flush_leaves<EPS0>(x, w, L, nleaf, p, a, npp);
    flush_m2p_full(x, w, L, nfull, p, a, nnp);
    flush_m2p_part(x, w, L, npart, p, a, nnp);
}

template<bool EPS0>
__global__ void __launch_bounds__(kNearThreads, 8) near_kernel(DualNodes nodes, const int *__restrict__ num_nodes,
                                                               const float4 *__restrict__ bodies, int n, float G,
                                                               float eps, float theta, float4 *__restrict__ acc,
                                                               unsigned long long *__restrict__ counts, NearPool pool,
                                                               int t_lo, int t_hi, uint32_t *__restrict__ err) {
    __shared__ NearWarp s_warps[kNearWarps];
    const int lane = threadIdx.x & 31;
    NearWarp &w = s_warps[threadIdx.x >> 5];
    int2 *wstack = pool.walk_stack + ((int64_t) blockIdx.x * kNearWarps + (threadIdx.x >> 5)) * kNearWalkStack;
    const Ctx x{nodes, bodies, G, eps, theta, *num_nodes, n};
    const unsigned long long nunits = min(pool.counters[2], (unsigned long long) pool.unit_cap);
    const unsigned long long nitems = min(pool.counters[0], (unsigned long long) pool.item_cap);
    unsigned long long npp = 0, nnp = 0;
    for (;;) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(&pool.counters[3], 1ull);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= nunits) break;
        const int2 unit = pool.units[u];
        const int leaf = unit.x;
        if (leaf < 0 || leaf >= x.nn) {
            if (lane == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
            continue;
        }
        const int2 lr = __ldg(nodes.link + leaf);
        const int tend = min(lr.y, unit.y + 32);
        if (lr.y < 0 || !x.range_ok(unit.y, tend) || tend == unit.y) {
            if (lane == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
            continue;
        }
        // a unit is evaluated whole (the same replica split as in an unrestricted pass), and only
        // its targets in [t_lo, t_hi) are written
        if (tend <= t_lo || unit.y >= t_hi) continue;
        Lane L;
        L.T = tend - unit.y;
        L.G = 32 / L.T;
        L.t = lane % L.T;
        L.r = lane / L.T;
        L.active = L.r < L.G;
        const int t = unit.y + L.t;
        L.counted = L.r == 0 && t >= t_lo && t < t_hi;
        const float4 q = __ldg(bodies + t);
        const float p[3] = {q.x, q.y, q.z};
        const unsigned tmask = L.T >= 32 ? 0xffffffffu : ((1u << L.T) - 1u);
        // the box of the unit's targets (every lane holds one of them) and their positions
        float lo[3] = {p[0], p[1], p[2]}, hi[3] = {p[0], p[1], p[2]};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
        }
        if (lane < L.T) w.tpos[lane] = q;
        // the null M2P record: no mass and no moments at 1e18 on every axis; for targets with
        // coordinates below 1e17 in magnitude every product of offsets in the term stays finite,
        // so each one meets a zero moment or mass and the term adds exactly zero
        if (lane < kM2pRec) w.m2p_part[kM2pPart * kM2pRec + lane] = lane == 0 ? make_float4(1e18f, 1e18f, 1e18f, 0.f)
                                                                              : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
        float a[3] = {0.f, 0.f, 0.f};
        int guard = 0;
        int top = 0;  // activeTree roots of the unit's items, walked together after the close bodies
        bool overflow = false;
        for (int it = pool.head[leaf]; it >= 0; ++guard) {
            if ((unsigned long long) it >= nitems || guard > (1 << 24)) {
                if (lane == 0) atomicOr(err, (uint32_t) kErrTraverseLimit);
                break;
            }
            const int4 item = pool.items[it];
            const int *words = pool.words + item.z;
            if (item.y == kItemBodies) {
                // runs of consecutive close bodies: (first body, length) pairs, packed into tiles
                run_tiles<EPS0>(x, w, L, words, item.w, p, a, npp, err);
            } else {
                for (int r0 = 0; r0 < item.w; r0 += 32) {
                    const int r = r0 + lane;
                    const int root = r < item.w ? words[r] : -1;
                    const bool ok = r < item.w && root >= 0 && root < x.nn;
                    if (r < item.w && !ok) atomicOr(err, (uint32_t) kErrTraverseLimit);
                    const uint32_t b = __ballot_sync(0xffffffffu, ok);
                    if (top + __popc(b) > kNearWalkStack) {
                        overflow = true;
                        continue;
                    }
                    if (ok) wstack[top + __popc(b & near_lanemask_lt())] = make_int2(root, (int) tmask);
                    top += __popc(b);
                }
            }
            it = item.x;
        }
        if (overflow && lane == 0) atomicOr(err, (uint32_t) kErrStackOverflow);
        __syncwarp();
        if (top > 0) chunk_walk<EPS0>(x, w, L, wstack, top, lo, hi, p, a, npp, nnp, err);
        // replicas' partial sums, added in replica order
        w.tile[lane] = make_float4(a[0], a[1], a[2], 0.f);
        __syncwarp();
        if (L.r == 0 && t >= t_lo && t < t_hi) {
            float s0 = a[0], s1 = a[1], s2 = a[2];
            for (int r = 1; r < L.G; ++r) {
                const float4 v = w.tile[r * L.T + L.t];
                s0 += v.x;
                s1 += v.y;
                s2 += v.z;
            }
            float4 o = acc[t];
            o.x += G * s0;
            o.y += G * s1;
            o.z += G * s2;
            acc[t] = o;
        }
        __syncwarp();
    }
    const unsigned long long c[2] = {npp, nnp};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        unsigned long long v = c[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(counts + k, v);
    }
}

}  // namespace

// Near-field grid: the resident blocks, never more than the walk stacks allocated (one per warp).
unsigned near_grid(const DualWorkspace &ws) {
    const int64_t by_stacks = ws.near.walk_warps / kNearWarps;
    return (unsigned) std::max<int64_t>(1, std::min<int64_t>(ws.near_blocks, by_stacks));
}

void launch_dual_traverse(const DualNodes &nodes, const int *num_nodes, const float4 *bodies, int64_t n, float G,
                          float eps, float theta, float4 *acc, unsigned long long *counts, DualWorkspace &ws,
                          uint32_t *err, cudaStream_t s, int64_t t_lo, int64_t t_hi) {
    if (n <= 0) return;
    const int lo = (int) std::max<int64_t>(0, std::min(t_lo, n)), hi = (int) std::max<int64_t>(lo, std::min(t_hi, n));
    cudaMemsetAsync(acc, 0, (size_t) n * sizeof(float4), s);
    cudaMemsetAsync(ws.near.head, 0xFF, (size_t) ws.near.head_cap * sizeof(int), s);
    cudaMemsetAsync(ws.near.counters, 0, 4 * sizeof(unsigned long long), s);
    cudaMemsetAsync(ws.spill.head, 0xFF, (size_t) ws.spill.head_cap * sizeof(int), s);
    cudaMemsetAsync(ws.spill.counters, 0, 4 * sizeof(unsigned long long), s);
    load_balanced_break_kernel<<<1, 32, 0, s>>>(nodes, num_nodes, ws.roots, ws.num_roots, err);
    // passive nodes of at most `frontier` bodies below a larger parent are handed to the second
    // kernel, which balances them over the whole GPU
    const int frontier = (int) std::max<int64_t>(64, n / 4096);
    dual_kernel<false><<<kDualRoots, kThreads, 0, s>>>(nodes, num_nodes, bodies, (int) n, G, eps, theta, acc,
                                                       counts, ws.roots, ws.num_roots, ws.arena, (int) ws.arena_words,
                                                       ws.tasks, ws.near, ws.spill, frontier, lo, hi, err);
    dual_kernel<true><<<ws.frontier_blocks, kThreads, 0, s>>>(nodes, num_nodes, bodies, (int) n, G, eps, theta, acc,
                                                              counts, ws.roots, ws.num_roots, ws.arena,
                                                              (int) ws.arena_words, ws.tasks, ws.near, ws.spill, -1,
                                                              lo, hi, err);
    if (eps == 0.f)
        near_kernel<true><<<near_grid(ws), kNearThreads, 0, s>>>(nodes, num_nodes, bodies, (int) n, G, eps, theta,
                                                                  acc, counts, ws.near, lo, hi, err);
    else
        near_kernel<false><<<near_grid(ws), kNearThreads, 0, s>>>(nodes, num_nodes, bodies, (int) n, G, eps, theta,
                                                                   acc, counts, ws.near, lo, hi, err);
}

void dual_near_sizes(int64_t n, int64_t *item_cap, int64_t *word_cap) {
    *item_cap = 4 * n + 65536;
    *word_cap = std::min<int64_t>(64 * n + (int64_t(1) << 22), (int64_t(1) << 31) - 1);
}

void dual_spill_sizes(int64_t n, int64_t *rec_cap, int64_t *word_cap) {
    *rec_cap = n / 8 + 65536;
    *word_cap = std::min<int64_t>(16 * n + (int64_t(1) << 22), (int64_t(1) << 31) - 1);
}

int dual_frontier_blocks(int device) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dual_kernel<true>, kThreads, 0);
    return std::max(1, sms * std::max(per_sm, 1));
}

int dual_near_warps_per_block() { return kNearWarps; }

int dual_near_blocks(int device) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, near_kernel<false>, kNearThreads, 0);
    return std::max(1, sms * std::max(per_sm, 1));
}

int64_t dual_arena_words(int64_t n) {
    // lists along one root-to-leaf path of the passive tree; grows with the body count. The largest
    // use measured on two 2^21-body Hernquist spheres at theta 0.4 is 1.5 Mi words (a start-node
    // block); a pass that runs out doubles the arenas and runs again.
    const int64_t w = 64 * n + (int64_t(1) << 16);
    return std::min<int64_t>(std::max<int64_t>(w, int64_t(1) << 16), int64_t(1) << 22);
}

}  // namespace nbg
