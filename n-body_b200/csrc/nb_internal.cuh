// Internal declarations shared by the sm_100a kernels of the force path.
//
// Device data layout (all in HBM, structure of arrays, 16-byte aligned):
//   bodies      float4 (x, y, z, m)     one per body, in Morton order after each sort
//   velocities  float4 (vx, vy, vz, 0)
//   ids         uint32                  input index of the body held in each slot
//   codes       uint64                  Morton codes, sorted together with a uint32 slot index
//   nodes       float4[REC] per node    preorder linear BVH, see NodeLayout below
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nbg {

// ---- bit-exact float helpers (no FMA contraction, IEEE round-to-nearest) ----
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// Reciprocal square root of the hardware special-function unit without the denormal-input fixup
// that rsqrtf carries (a compare and two multiplies per call). At the interaction sites the
// argument is |R|^2 + epsilon, a normal float for every pair that is evaluated (an exact zero is
// skipped first), and for a normal argument the result equals rsqrtf's; a denormal argument is
// flushed to zero (1/sqrt then overflows to infinity either way).
__device__ __forceinline__ float rsqrt_hw(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Gravity::particleParticle (Gravity.h:199-209) without G for one target and two sources at once,
// in paired FP32 arithmetic (sm_100 FADD2 / FFMA2 / FMUL2: one instruction for both halves):
// u = (x_a, x_b, y_a, y_b), v = (z_a, z_b, m_a, m_b), np = -p in both halves. Per half:
// d = b - p, r2 = d.d + eps (z term first, as the scalar form), a += d m / r2^(3/2). With eps > 0 a
// source at the target's own position adds 0 * s = 0; with eps = 0 a source at zero distance is
// skipped. A massless padding source far away (r2 overflowing to infinity) adds exactly 0.
template<bool EPS0>
__device__ __forceinline__ void pair2_term(float2 npx, float2 npy, float2 npz, float2 eps2, float4 u, float4 v,
                                           float2 &ax, float2 &ay, float2 &az) {
    const float2 dx = __fadd2_rn(make_float2(u.x, u.y), npx);
    const float2 dy = __fadd2_rn(make_float2(u.z, u.w), npy);
    const float2 dz = __fadd2_rn(make_float2(v.x, v.y), npz);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
    float2 inv;
    inv.x = rsqrt_hw(r2.x);
    inv.y = rsqrt_hw(r2.y);
    float2 s = __fmul2_rn(make_float2(v.z, v.w), __fmul2_rn(__fmul2_rn(inv, inv), inv));
    if (EPS0) {
        if (r2.x == 0.f) s.x = 0.f;
        if (r2.y == 0.f) s.y = 0.f;
    }
    ax = __ffma2_rn(dx, s, ax);
    ay = __ffma2_rn(dy, s, ay);
    az = __ffma2_rn(dz, s, az);
}

// glm::min / glm::max semantics: min(x, y) = (y < x) ? y : x, max(x, y) = (x < y) ? y : x
__device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return (x < y) ? y : x; }

// Order-preserving map float -> uint32 (for atomicMin/atomicMax on floats).
__host__ __device__ __forceinline__ uint32_t float_to_ordered(float f) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ordered_to_float(uint32_t o) {
    uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

// Morton code of one position (MortonSort.h:46-73): v = (p - min) / scale, clamp(v * 2^21, 0,
// 2^21 - 1) per axis, truncated and interleaved x*4 + y*2 + z. NaN (zero scale) maps to cell 0.
__device__ __forceinline__ uint64_t expand_bits21(uint64_t i) {
    i &= 0x1fffff;
    i = (i | i << 32) & 0x1f00000000ffffULL;
    i = (i | i << 16) & 0x1f0000ff0000ffULL;
    i = (i | i << 8) & 0x100f00f00f00f00fULL;
    i = (i | i << 4) & 0x10c30c30c30c30c3ULL;
    i = (i | i << 2) & 0x1249249249249249ULL;
    return i;
}
__device__ __forceinline__ uint64_t axis_cell(float v) {
    const float c = gmin(gmax(fmul(v, 2097152.f), 0.f), 2097151.f);
    return (c == c) ? __float2ull_rz(c) : 0ull;
}
__device__ __forceinline__ uint64_t morton_code(float4 p, const float mn[3], float scale) {
    const uint64_t cx = axis_cell(fdiv(fsub(p.x, mn[0]), scale));
    const uint64_t cy = axis_cell(fdiv(fsub(p.y, mn[1]), scale));
    const uint64_t cz = axis_cell(fdiv(fsub(p.z, mn[2]), scale));
    return expand_bits21(cx) * 4u + expand_bits21(cy) * 2u + expand_bits21(cz);
}

// Global bounding box accumulator: 6 ordered uints, all reduced with atomicMin.
// [0..2] = ordered(min.xyz), [3..5] = ~ordered(max.xyz). Reset by filling with 0xFF bytes.
struct BBoxAccum {
    uint32_t v[6];
};

// ---- node records (preorder linear BVH), three arrays indexed by preorder position ----
// mac[c]  = (centre.xyz, mac_threshold): centre = (max + min) / 2 of the node's bounding box;
//           a target at squared distance d2 from the centre takes the node's approximation iff
//           d2 >= mac_threshold (bit-identical to diag^2 / d2 < theta^2 of the reference MAC)
// link[c] = internal node: (preorder index of the right child, -1); the left child is c + 1
//           leaf:          (first body, end body) of its range in Morton order
// pay[c * PAY + k]: k = 0: (centre_of_mass.xyz, mass); order 2 adds k = 1: (Qxx, Qxy, Qxz, Qyy),
//           k = 2: (Qyz, Qzz, 1.5 * trace(Q), 0) - moments about the centre of mass, not traceless.
template<int ORDER>
struct NodeLayout;
template<>
struct NodeLayout<1> {
    static constexpr int PAY = 1;
};
template<>
struct NodeLayout<2> {
    static constexpr int PAY = 3;
};
struct NodeArrays {
    float4 *mac = nullptr;
    int2 *link = nullptr;
    float4 *pay = nullptr;
    int64_t capacity = 0;
};

constexpr int kMaxOrder = 2;
// Deepest possible binary radix tree over 64-bit codes with 32-bit index tie-breaks.
constexpr int kMaxTreeDepth = 128;

// ---- device-side error reporting ----
enum DeviceError : uint32_t {
    kErrNone = 0,
    kErrLookbackTimeout = 1u << 0,   // onesweep look-back wait exceeded its limit
    kErrTreeDepth = 1u << 1,         // a walk up the tree exceeded the maximum depth
    kErrNodeOverflow = 1u << 2,      // more tree nodes than the node buffer holds
    kErrStackOverflow = 1u << 3,     // traversal stack full (a push was dropped)
    kErrTraverseLimit = 1u << 4,     // traversal met an invalid link or exceeded its round limit
    kErrDualArena = 1u << 5,         // dual-tree list or task storage exhausted
    kErrNearPool = 1u << 6,          // dual-tree near-field pool too small (the host grows it and retries)
};

// ---- launchers (stream-ordered; defined in the .cu files) ----

// bbox_morton.cu
void launch_bbox_reset(BBoxAccum *acc, cudaStream_t s);
void launch_bbox_reduce(const float4 *pos, int64_t n, BBoxAccum *acc, cudaStream_t s);
void launch_morton_hist(const float4 *pos, int64_t n, const BBoxAccum *acc, uint64_t *codes, uint32_t *hist,
                        cudaStream_t s);

// radix_sort.cu
constexpr int kSortTileKeys = 2048;  // keys ranked per block (tile) of one one-sweep pass
constexpr int kSortPasses = 8;       // 8-bit digits of the 64-bit keys
struct SortWorkspace {
    uint64_t *keys_alt = nullptr;
    uint32_t *vals_alt = nullptr;
    uint32_t *hist = nullptr;      // 8 x 256 digit counts, filled by launch_morton_hist
    uint32_t *offsets = nullptr;   // 8 x 256 exclusive prefixes + 8 trivial-pass flags
    uint32_t *lookback = nullptr;  // 8 x tiles x 256
    uint32_t *tile_counter = nullptr;  // 8
    int64_t capacity = 0;
};
int64_t sort_tiles(int64_t n);
size_t sort_lookback_words(int64_t n);
// Sorts (keys, iota) by key; the sorted keys and slot indices end in keys/vals (ping-pong inside).
// Returns the first error reported while queuing its memsets and launches (checked with
// cudaPeekAtLastError, which clears nothing).
cudaError_t launch_radix_sort(uint64_t *keys, uint32_t *vals, int64_t n, SortWorkspace &ws, uint32_t *err,
                              cudaStream_t s);
// Self-test of the bounded look-back wait: one pass that can never complete its look-back runs
// with the given wait limit; the error word it leaves is returned (kErrLookbackTimeout expected).
cudaError_t lookback_timeout_selftest(unsigned long long wait_limit_ns, uint32_t *err_word);
// One stable one-sweep pass on digit `pass` (bits 8*pass .. 8*pass+7) of the keys. offsets holds
// the exclusive digit prefixes at [pass*256 + d] and a trivial-pass flag at [8*256 + pass];
// lookback (pass x tiles x 256 words) and tile_counter[pass] must be zero. Pass 0 ignores vals_in
// and emits the input positions as values.
void launch_radix_pass(const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out, uint32_t *vals_out,
                       int64_t n, int pass, const uint32_t *offsets, uint32_t *lookback, uint32_t *tile_counter,
                       uint32_t *err, cudaStream_t s);

// Several independent instances laid out back to back in one body array (device pointers).
// With inst_of == nullptr the body array is a single instance.
struct BatchSegments {
    const int *inst_of = nullptr;        // instance of each body position (positions stay in their segment)
    const float *inst_theta2 = nullptr;  // RN(theta * theta) per instance
    const int2 *inst_range = nullptr;    // first and last (inclusive) body position per instance
    int *inst_root = nullptr;            // written by the build: preorder index of each instance's root
};

// lbvh_build.cu
struct TreeWorkspace {
    int4 *topo = nullptr;           // n-1 Karras internal nodes: (left child, right child, first body, last body);
                                    // child encoding: internal i >= 0, Karras leaf j as ~j
    int *parent = nullptr;          // parent of internal node
    uint8_t *flags = nullptr;       // n-1: final internal node, left / right child a final leaf (lbvh_build.cu)
    int *visit = nullptr;           // n-1 arrival counters of the summary climb
    float4 *slot = nullptr;         // 2n summary slots of 4 float4 (orders 1 and 2)
    float4 *slot3 = nullptr;        // 2n summary slots of 8 float4 (order 3, dual tree)
    int *chain = nullptr;           // per final internal node: final internal nodes below it that share its first body
    int *start = nullptr;           // per body position (n + 1): 2 x (final internal nodes whose range starts
                                    // there) + 1 if a final leaf starts there
    int *pre_base = nullptr;        // per body position (n + 1): preorder index of the final leaf starting there
                                    // (final nodes starting before it plus final internal nodes starting at it)
    int *scan_part = nullptr;       // per scan tile: its total, then its exclusive prefix
    int *leaf_parents = nullptr;    // final internal nodes with at least one final-leaf child (n - 1),
                                    // in no particular order; the count is leaf_parents_count[0]
    int *leaf_parents_count = nullptr;
    int *num_nodes = nullptr;       // device scalar: final node count
    int64_t capacity = 0;
    // Precision option (0: off, the reference's FP32 operations everywhere): internal nodes of at
    // least this many bodies combine their children's summaries in FP64, rounded once to FP32.
    int fp64_min_bodies = 0;
};
// Scan tiles of the preorder prefix over n + 1 body positions (sizes tw.scan_part).
int64_t build_scan_tiles(int64_t n);
void launch_build_tree(const uint64_t *sorted_codes, const float4 *bodies, int64_t n, int leaf, int order, float theta,
                       TreeWorkspace &tw, const NodeArrays &nodes, uint32_t *err, cudaStream_t s,
                       const BatchSegments &seg = BatchSegments());

// Dual-tree node arrays (preorder): bmin = (min.xyz, body count as int bits), bmax = (max.xyz,
// diagonal length as BoundingBox::diagonalLength computes it),
// com = (centre of mass, mass), q = 4 float4 per node: Q2 (6) then Q3 (10);
// link = (first body, end body) at a leaf, (right child, -1 - first body) at an internal node.
// thr = exact criterion thresholds for the configured theta: (B, S) with
// RN(diag / sep) < theta  <=>  sep >= B  <=>  (when one separation vector is zero) |v|^2 >= S,
// and the same pair for the passive test RN(3 diag / sep) < theta.
struct DualNodes {
    float4 *bmin = nullptr, *bmax = nullptr, *com = nullptr, *q = nullptr, *thr = nullptr;
    int2 *link = nullptr;
    int64_t capacity = 0;
};
void launch_build_dual_tree(const uint64_t *sorted_codes, const float4 *bodies, int64_t n, int leaf, float theta,
                            TreeWorkspace &tw, const DualNodes &nodes, uint32_t *err, cudaStream_t s);

// dualtree.cu
constexpr int kDualRoots = 256;   // starting passive nodes (Tree::loadBalancedBreak(256))
constexpr int kDualTasks = 4096;  // task records per block
// Near-field work handed from the traversal to the near-field kernel: per passive leaf, a list
// of items (activeTree roots, or close bodies) whose payload lives in one word pool.
struct NearPool {
    int *head = nullptr;                  // per node: newest item of the passive leaf, -1 if none
    int4 *items = nullptr;                // (next item, kind, payload offset, payload count)
    int *words = nullptr;                 // payload: node or body indices
    int2 *units = nullptr;                // (passive leaf, first target) per 32-target unit
    unsigned long long *counters = nullptr;  // items, words, units, unit cursor
    int64_t head_cap = 0, item_cap = 0, word_cap = 0, unit_cap = 0;
    int2 *walk_stack = nullptr;           // per warp of the near-field grid: kNearWalkStack (node, mask)
    int64_t walk_warps = 0;               // warps the walk stacks were sized for
};
constexpr int kNearWalkStack = 4608;
// Tasks handed from the first traversal kernel (above the frontier of passive nodes with at
// most `frontier` bodies) to the second one, which takes frontier nodes from a work list.
struct SpillPool {
    int *head = nullptr;                  // per node: newest task record of a frontier node, -1 if none
    int4 *recs = nullptr;                 // (next record, task type, list offset, list length)
    int *rec_field = nullptr;             // field offset per record
    int *words = nullptr;                 // list copies and fields (float bits)
    int *work = nullptr;                  // frontier nodes with tasks, in registration order
    unsigned long long *counters = nullptr;  // records, words, work items, work cursor
    int64_t head_cap = 0, rec_cap = 0, word_cap = 0, work_cap = 0;
};
struct DualWorkspace {
    int *roots = nullptr;           // starting passive nodes (at most kDualRoots)
    int *num_roots = nullptr;
    int *arena = nullptr;           // per block: arena_words words of lists and local fields
    int *tasks = nullptr;           // per block: kDualTasks task records of 6 ints
    int64_t arena_words = 0;
    NearPool near;
    int near_blocks = 0;            // resident blocks of the near-field kernel
    SpillPool spill;
    int frontier_blocks = 0;        // resident blocks of the frontier-task kernel
    int blocks = 0;                 // arenas and task stacks allocated (one per traversal block)
};
// Arena words per block, near-pool sizes and the near kernel's resident grid for n bodies.
int64_t dual_arena_words(int64_t n);
void dual_near_sizes(int64_t n, int64_t *item_cap, int64_t *word_cap);
void dual_spill_sizes(int64_t n, int64_t *rec_cap, int64_t *word_cap);
int dual_near_blocks(int device);
int dual_near_warps_per_block();
int dual_frontier_blocks(int device);
// Accelerations of the targets in [t_lo, t_hi) of the Morton-ordered bodies (all sources act);
// [0, n) for an unsharded pass.
void launch_dual_traverse(const DualNodes &nodes, const int *num_nodes, const float4 *bodies, int64_t n, float G,
                          float eps, float theta, float4 *acc, unsigned long long *counts, DualWorkspace &ws,
                          uint32_t *err, cudaStream_t s, int64_t t_lo, int64_t t_hi);

// traverse.cu
struct TraverseWorkspace {
    int2 *stack = nullptr;            // per resident warp: kTraverseStack entries of (node, target mask)
    unsigned *group_counter = nullptr;
    int64_t warps = 0;                // resident warps the stack memory was sized for
    int threads = 256;                // launch shape: threads per block (128 or 256)
    int slab = 64;                    // launch shape: partial-accept slab entries per warp (32 or 64)
};
// Whether (threads, slab) is one of the traversal's compiled launch shapes.
bool traversal_shape_valid(int threads, int slab);
constexpr int kTraverseStack = 4608;
// Resident warps of the persistent traversal grid on `device` (for sizing TraverseWorkspace).
int64_t traverse_resident_warps(int device);
// groups (optional): one int4 (first target, target count <= 32, instance, 0) per warp task; the
// traversal of a group starts at inst_root[instance]. Without groups, targets are cut into
// consecutive groups of 32 that start at node 0. inst_counts (optional, with groups): per instance,
// (particle-particle, node-particle) interaction counts are added at [2 * instance + {0, 1}].
void launch_bh_traverse(int order, const NodeArrays &nodes, const int *num_nodes, const float4 *bodies, int64_t n_bodies,
                        const float4 *targets, int64_t n_targets, float G, float eps, float4 *acc,
                        unsigned long long *counts, TraverseWorkspace &ws, uint32_t *err, cudaStream_t s,
                        const int4 *groups = nullptr, int64_t num_groups = 0, const int *inst_root = nullptr,
                        unsigned long long *inst_counts = nullptr);

// direct_sum.cu
// FP64 energy diagnostics: (kinetic, potential) of n bodies into out[0..1]; parts needs
// energy_parts(n) doubles.
int64_t energy_parts(int64_t n);
void launch_energy_f64(const float4 *bodies, const float4 *vel, int64_t n, double G, double eps, double *parts,
                       double *out, cudaStream_t s);
void launch_direct_f32(const float4 *bodies, int64_t n, const float4 *targets, int64_t nt, float G, float eps,
                       float4 *acc, cudaStream_t s);
void launch_direct_f64(const float4 *bodies, int64_t n, const float4 *targets, int64_t nt, double G, double eps,
                       double *acc3, cudaStream_t s);

// integrate.cu
void launch_gather_state(const uint32_t *perm, int64_t n, const float4 *pos, const float4 *vel, const uint32_t *id,
                         float4 *pos_out, float4 *vel_out, uint32_t *id_out, cudaStream_t s);
void launch_scatter_by_id(const uint32_t *id, int64_t n, const float4 *src, float4 *dst, cudaStream_t s);
void launch_kick_drift(float4 *pos, float4 *vel, const float4 *acc, int64_t n, float dt, BBoxAccum *next_bbox,
                       cudaStream_t s);
void launch_iota(uint32_t *id, int64_t n, cudaStream_t s, uint32_t first = 0);
void launch_add_offset(uint32_t *id, int64_t n, int64_t delta, cudaStream_t s);

// batch.cu
// inst_box: 6 order-preserving uints per instance (min.xyz, ~max.xyz); slices: blocks per instance
void launch_seg_bbox(const float4 *pos, const int2 *inst_range, int num_inst, int slices, uint32_t *inst_box,
                     cudaStream_t s);
void launch_seg_morton(const float4 *pos, int64_t n, const int *inst_of, const uint32_t *inst_box, uint64_t *codes,
                       uint32_t *hist, cudaStream_t s);
void launch_inst_keys(const uint32_t *slot, int64_t n, const int *inst_of, uint64_t *ikeys, cudaStream_t s);
void launch_compose(const uint32_t *order, int64_t n, const uint32_t *slot, const uint64_t *codes, uint32_t *perm,
                    uint64_t *codes_out, cudaStream_t s);
void launch_fill_tables(const int2 *inst_range, const int *group_first, int num_inst, int *inst_of, int4 *groups,
                        cudaStream_t s);

// SM count of a device, queried once per device (cached).
int sm_count(int device);
// SM count of the current device.
int current_sm_count();

// Largest number of bodies one context accepts (30-bit counts in the sort's look-back words,
// 31-bit body indices in the tree).
constexpr int64_t kMaxBodies = (int64_t(1) << 30) - 1;

}  // namespace nbg
