// C ABI of the force path (declared in include/nbody_gpu.h): context, device memory and the
// per-step pipeline.
//
// One force pass (Solver::updateAccelerations, ActiveTreeSolver.h:33-72) on the device:
//   bbox reduce (skipped when the previous drift already reduced it)
//   -> Morton codes + digit histograms -> one-sweep radix sort (8 passes)
//   -> gather positions/velocities/ids into Morton order
//   -> Karras build + collapse + bottom-up summaries + preorder records
//   -> lock-step warp traversal
// and Solver::step adds the kick-drift kernel (which also reduces the next bounding box).
// No phase has a host fallback: without a usable device nb_create fails.
#include <algorithm>
#include <cmath>
#include <array>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/nbody_gpu.h"
#include "nb_internal.cuh"

using namespace nbg;

namespace {

template<typename T>
cudaError_t dev_alloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void **) p, count * sizeof(T));
}

template<typename T>
void dev_free(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

enum Phase { kBBox = 0, kMorton, kSort, kGather, kBuild, kTraverse, kIntegrate, kEnd, kNumMarks };

}  // namespace

struct nb_ctx {
    nb_config cfg{};
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string error;

    int64_t n = 0, cap = 0;
    float4 *pos = nullptr, *vel = nullptr, *acc = nullptr, *pos2 = nullptr, *vel2 = nullptr;
    uint32_t *id = nullptr, *id2 = nullptr;
    uint64_t *keys = nullptr;
    uint32_t *vals = nullptr;
    SortWorkspace sw;
    TreeWorkspace tw;
    NodeArrays nodes;
    TraverseWorkspace trav;
    DualNodes dnodes;          // dual solver: octupole node arrays
    DualWorkspace dws;         // dual solver: starting nodes, per-block arenas and task stacks
    int64_t dual_cap = 0;      // body capacity the dual buffers were sized for
    unsigned long long *host_scratch = nullptr;  // pinned: near-pool counters and the error word
    BBoxAccum *bbox = nullptr;
    unsigned long long *counts = nullptr;
    uint32_t *err = nullptr;
    double *acc64 = nullptr;
    int64_t acc64_cap = 0;

    // batch of independent instances (0: one instance set by nb_set_bodies)
    int32_t num_inst = 0;
    std::vector<int64_t> inst_start, inst_size;
    int *inst_of = nullptr, *inst_root = nullptr;
    float *inst_theta2 = nullptr;
    uint32_t *inst_box = nullptr;  // 6 order-preserving uints per instance (min.xyz, ~max.xyz)
    int inst_bbox_slices = 1;      // blocks per instance of the box reduction
    int2 *inst_range = nullptr;
    int4 *groups = nullptr;
    int64_t ngroups = 0;
    unsigned long long *inst_counts = nullptr;  // (particle-particle, node-particle) per instance
    uint64_t *ikeys = nullptr, *ikeys2 = nullptr;
    uint32_t *ivals = nullptr, *ivals2 = nullptr;
    uint32_t *inst_offsets = nullptr, *inst_lookback = nullptr, *inst_tiles = nullptr;
    int inst_passes = 0;
    int64_t batch_body_cap = 0, batch_inst_cap = 0, batch_group_cap = 0;  // grow-only batch buffers
    int *group_first = nullptr;
    const uint64_t *sorted_codes = nullptr;  // buffer holding the last pass's sorted codes

    // CUDA graph of two consecutive steps (bodies ping-pong between two buffers each step)
    bool use_graphs = false;
    cudaGraphExec_t graph2 = nullptr;
    float4 *graph_pos = nullptr;   // the body buffer the captured pair starts from
    int64_t steps_since_set = 0;   // plain or captured steps since the body set was replaced

    // target sharding of one instance over `shard_world` processes (1: not sharded)
    int32_t shard_rank = 0, shard_world = 1;

    bool bbox_valid = false;  // bbox already holds the box of the current positions
    bool have_tree = false;
    bool have_acc = false;
    bool acc_is_bh = false;
    bool acc_is_dual = false;

    bool timing = false;
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::array<cudaEvent_t, kNumMarks>> pending;  // marks of passes not yet read
    nb_phase_times times{};
    std::string id_str, name_str;
};

namespace {

int fail(nb_ctx *c, int code, const std::string &msg) {
    if (c) c->error = msg;
    return code;
}

int check_cuda(nb_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return NB_OK;
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(c, e == cudaErrorMemoryAllocation ? NB_ERR_OUT_OF_MEMORY : NB_ERR_CUDA, m);
}

#define NB_TRY(expr, what)                                  \
    do {                                                    \
        int _rc = check_cuda(ctx, (expr), what);            \
        if (_rc != NB_OK) return _rc;                       \
    } while (0)

// Exported record: mac (4 floats), link (2 ints + 2 zero), payload (4 floats per PAY entry).
int pay_float4s(int order) { return order == 1 ? NodeLayout<1>::PAY : NodeLayout<2>::PAY; }
int rec_floats(int order) { return 8 + 4 * pay_float4s(order); }

// Slice of Morton-ordered bodies owned by `rank`: chunks of ceil(n / world) rounded up to whole
// 32-target traversal groups; the last chunks may be short or empty.
void shard_slice(int64_t n, int32_t rank, int32_t world, int64_t *chunk, int64_t *first, int64_t *count) {
    int64_t c = world > 0 ? (n + world - 1) / world : n;
    c = (c + 31) / 32 * 32;
    const int64_t f = std::min<int64_t>(n, (int64_t) rank * c);
    *chunk = c;
    *first = f;
    *count = std::min<int64_t>(n, f + c) - f;
}

void refresh_names(nb_ctx *ctx) {
    if (ctx->cfg.solver == NB_SOLVER_DUAL_LINEAR_BVH) {
        ctx->id_str = "implicit-linear-bvh-fmm-8p";
        ctx->name_str = "Implicit Linear-BVH Fast Multipole Method (Octupole)";
    } else if (ctx->cfg.solver == NB_SOLVER_NAIVE) {
        ctx->id_str = "naive";
        ctx->name_str = "Naive";
    } else if (ctx->cfg.order == 1) {
        ctx->id_str = "linear-bvh";
        ctx->name_str = "Linear-BVH";
    } else {
        ctx->id_str = "linear-bvh-4p";
        ctx->name_str = "Linear BVH (Quadrupole)";
    }
}

int validate(nb_ctx *ctx, const nb_config *cfg) {
    if (!cfg) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "config is NULL");
    if (cfg->solver != NB_SOLVER_LINEAR_BVH && cfg->solver != NB_SOLVER_NAIVE &&
        cfg->solver != NB_SOLVER_DUAL_LINEAR_BVH)
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "unknown solver");
    if (cfg->solver == NB_SOLVER_DUAL_LINEAR_BVH) {
        if (cfg->order != 3) return fail(ctx, NB_ERR_UNSUPPORTED, "the dual-tree solver runs at order 3 (octupole)");
    } else if (cfg->order < 1 || cfg->order > kMaxOrder) {
        return fail(ctx, NB_ERR_UNSUPPORTED, "order must be 1 (centre of mass) or 2 (quadrupole)");
    }
    if (cfg->max_leaf_size < 1) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "max_leaf_size must be >= 1");
    if (!(cfg->theta >= 0.f)) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "theta must be >= 0");
    if (!(cfg->epsilon >= 0.f)) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "epsilon must be >= 0");
    return NB_OK;
}

void free_batch(nb_ctx *ctx) {
    dev_free(ctx->inst_of); dev_free(ctx->inst_root); dev_free(ctx->inst_theta2); dev_free(ctx->inst_box);
    dev_free(ctx->inst_range); dev_free(ctx->groups); dev_free(ctx->ikeys); dev_free(ctx->ikeys2);
    dev_free(ctx->ivals); dev_free(ctx->ivals2); dev_free(ctx->inst_offsets); dev_free(ctx->inst_lookback);
    dev_free(ctx->inst_tiles); dev_free(ctx->group_first); dev_free(ctx->inst_counts);
    ctx->batch_body_cap = ctx->batch_inst_cap = ctx->batch_group_cap = 0;
    ctx->num_inst = 0;
    ctx->ngroups = 0;
    ctx->inst_start.clear();
    ctx->inst_size.clear();
}

void drop_graph(nb_ctx *ctx) {
    if (ctx->graph2) cudaGraphExecDestroy(ctx->graph2);
    ctx->graph2 = nullptr;
}

void free_dual(nb_ctx *ctx) {
    dev_free(ctx->tw.slot3);
    dev_free(ctx->dnodes.bmin); dev_free(ctx->dnodes.bmax); dev_free(ctx->dnodes.com); dev_free(ctx->dnodes.q);
    dev_free(ctx->dnodes.link); dev_free(ctx->dnodes.thr);
    ctx->dnodes.capacity = 0;
    dev_free(ctx->dws.roots); dev_free(ctx->dws.num_roots); dev_free(ctx->dws.arena); dev_free(ctx->dws.tasks);
    ctx->dws.arena_words = 0;
    NearPool &np = ctx->dws.near;
    dev_free(np.head); dev_free(np.items); dev_free(np.words); dev_free(np.units); dev_free(np.counters);
    dev_free(np.walk_stack);
    np.head_cap = np.item_cap = np.word_cap = np.unit_cap = 0;
    np.walk_warps = 0;
    SpillPool &sp = ctx->dws.spill;
    dev_free(sp.head); dev_free(sp.recs); dev_free(sp.rec_field); dev_free(sp.words); dev_free(sp.work);
    dev_free(sp.counters);
    sp.head_cap = sp.rec_cap = sp.word_cap = sp.work_cap = 0;
    ctx->dual_cap = 0;
}

// Buffers of the dual solver, sized for the current body capacity (allocated before any capture).
int ensure_dual(nb_ctx *ctx) {
    if (ctx->cfg.solver != NB_SOLVER_DUAL_LINEAR_BVH || ctx->cap == 0) return NB_OK;
    if (ctx->dual_cap == ctx->cap) return NB_OK;
    free_dual(ctx);
    const int64_t c = ctx->cap;
    const size_t slots = (size_t) (2 * c);
    NB_TRY(dev_alloc(&ctx->tw.slot3, 8 * slots), "alloc octupole summaries");
    NB_TRY(dev_alloc(&ctx->dnodes.bmin, slots), "alloc dual nodes");
    NB_TRY(dev_alloc(&ctx->dnodes.bmax, slots), "alloc dual nodes");
    NB_TRY(dev_alloc(&ctx->dnodes.com, slots), "alloc dual nodes");
    NB_TRY(dev_alloc(&ctx->dnodes.q, 4 * slots), "alloc dual nodes");
    NB_TRY(dev_alloc(&ctx->dnodes.link, slots), "alloc dual nodes");
    NB_TRY(dev_alloc(&ctx->dnodes.thr, slots), "alloc dual nodes");
    ctx->dnodes.capacity = (int64_t) slots;
    NB_TRY(dev_alloc(&ctx->dws.roots, kDualRoots), "alloc dual roots");
    NB_TRY(dev_alloc(&ctx->dws.num_roots, 1), "alloc dual roots");
    ctx->dws.arena_words = dual_arena_words(c);
    // one arena and task stack per traversal block: the start-node blocks and the frontier blocks
    if (ctx->dws.frontier_blocks == 0) ctx->dws.frontier_blocks = dual_frontier_blocks(ctx->cfg.device);
    ctx->dws.blocks = std::max(kDualRoots, ctx->dws.frontier_blocks);
    NB_TRY(dev_alloc(&ctx->dws.arena, (size_t) ctx->dws.blocks * (size_t) ctx->dws.arena_words), "alloc dual arena");
    NB_TRY(dev_alloc(&ctx->dws.tasks, (size_t) ctx->dws.blocks * kDualTasks * 6), "alloc dual tasks");
    NearPool &np = ctx->dws.near;
    np.head_cap = (int64_t) slots;
    dual_near_sizes(c, &np.item_cap, &np.word_cap);
    np.unit_cap = c + 64;
    NB_TRY(dev_alloc(&np.head, (size_t) np.head_cap), "alloc near-field pool");
    NB_TRY(dev_alloc(&np.items, (size_t) np.item_cap), "alloc near-field pool");
    NB_TRY(dev_alloc(&np.words, (size_t) np.word_cap), "alloc near-field pool");
    NB_TRY(dev_alloc(&np.units, (size_t) np.unit_cap), "alloc near-field pool");
    NB_TRY(dev_alloc(&np.counters, 4), "alloc near-field pool");
    if (ctx->dws.near_blocks == 0) ctx->dws.near_blocks = dual_near_blocks(ctx->cfg.device);
    np.walk_warps = (int64_t) ctx->dws.near_blocks * dual_near_warps_per_block();
    NB_TRY(dev_alloc(&np.walk_stack, (size_t) np.walk_warps * kNearWalkStack), "alloc near-field walk stacks");
    SpillPool &sp = ctx->dws.spill;
    sp.head_cap = (int64_t) slots;
    sp.work_cap = (int64_t) slots;
    dual_spill_sizes(c, &sp.rec_cap, &sp.word_cap);
    NB_TRY(dev_alloc(&sp.head, (size_t) sp.head_cap), "alloc frontier pool");
    NB_TRY(dev_alloc(&sp.work, (size_t) sp.work_cap), "alloc frontier pool");
    NB_TRY(dev_alloc(&sp.recs, (size_t) sp.rec_cap), "alloc frontier pool");
    NB_TRY(dev_alloc(&sp.rec_field, (size_t) sp.rec_cap), "alloc frontier pool");
    NB_TRY(dev_alloc(&sp.words, (size_t) sp.word_cap), "alloc frontier pool");
    NB_TRY(dev_alloc(&sp.counters, 4), "alloc frontier pool");
    ctx->dual_cap = c;
    return NB_OK;
}

void free_buffers(nb_ctx *ctx) {
    free_dual(ctx);
    dev_free(ctx->pos); dev_free(ctx->vel); dev_free(ctx->acc); dev_free(ctx->pos2); dev_free(ctx->vel2);
    dev_free(ctx->id); dev_free(ctx->id2); dev_free(ctx->keys); dev_free(ctx->vals);
    dev_free(ctx->sw.keys_alt); dev_free(ctx->sw.vals_alt); dev_free(ctx->sw.lookback);
    dev_free(ctx->tw.topo); dev_free(ctx->tw.parent); dev_free(ctx->tw.flags); dev_free(ctx->tw.visit);
    dev_free(ctx->tw.slot); dev_free(ctx->tw.chain);
    dev_free(ctx->tw.start); dev_free(ctx->tw.pre_base); dev_free(ctx->tw.scan_part);
    dev_free(ctx->tw.leaf_parents); dev_free(ctx->tw.leaf_parents_count);
    dev_free(ctx->nodes.mac); dev_free(ctx->nodes.link); dev_free(ctx->nodes.pay);
    ctx->nodes.capacity = 0;
    ctx->cap = 0;
}

int ensure_capacity(nb_ctx *ctx, int64_t n) {
    if (n <= ctx->cap) return NB_OK;
    free_buffers(ctx);
    const int64_t c = std::max<int64_t>(n, 1);
    const size_t slots = (size_t) (2 * c);
    NB_TRY(dev_alloc(&ctx->pos, c), "alloc positions");
    NB_TRY(dev_alloc(&ctx->vel, c), "alloc velocities");
    NB_TRY(dev_alloc(&ctx->acc, c), "alloc accelerations");
    NB_TRY(dev_alloc(&ctx->pos2, c), "alloc positions");
    NB_TRY(dev_alloc(&ctx->vel2, c), "alloc velocities");
    NB_TRY(dev_alloc(&ctx->id, c), "alloc ids");
    NB_TRY(dev_alloc(&ctx->id2, c), "alloc ids");
    NB_TRY(dev_alloc(&ctx->keys, c), "alloc codes");
    NB_TRY(dev_alloc(&ctx->vals, c), "alloc sort values");
    NB_TRY(dev_alloc(&ctx->sw.keys_alt, c), "alloc codes");
    NB_TRY(dev_alloc(&ctx->sw.vals_alt, c), "alloc sort values");
    NB_TRY(dev_alloc(&ctx->sw.lookback, sort_lookback_words(c)), "alloc sort look-back");
    ctx->sw.capacity = c;
    NB_TRY(dev_alloc(&ctx->tw.topo, c), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.parent, c), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.flags, c), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.visit, c), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.slot, 4 * slots), "alloc summaries");
    NB_TRY(dev_alloc(&ctx->tw.chain, c), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.leaf_parents, c), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.leaf_parents_count, 1), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.start, c + 1), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.pre_base, c + 1), "alloc tree");
    NB_TRY(dev_alloc(&ctx->tw.scan_part, build_scan_tiles(c)), "alloc tree");
    ctx->tw.capacity = c;
    const int64_t node_cap = 2 * c;
    NB_TRY(dev_alloc(&ctx->nodes.mac, (size_t) node_cap), "alloc tree nodes");
    NB_TRY(dev_alloc(&ctx->nodes.link, (size_t) node_cap), "alloc tree nodes");
    NB_TRY(dev_alloc(&ctx->nodes.pay, (size_t) node_cap * NodeLayout<2>::PAY), "alloc tree nodes");
    ctx->nodes.capacity = node_cap;
    ctx->cap = c;
    return ensure_dual(ctx);
}

cudaEvent_t take_event(nb_ctx *ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Phase boundaries of one pass: CUDA events on the context's stream when timing is enabled, and
// an NVTX range per phase (host side, for timeline profilers; near free without one attached).
struct Marks {
    nb_ctx *ctx;
    std::array<cudaEvent_t, kNumMarks> ev{};
    bool on;
    bool range_open = false;
    explicit Marks(nb_ctx *c) : ctx(c), on(c->timing) {
        if (on)
            for (auto &e: ev) e = take_event(c);
    }
    ~Marks() {
        if (range_open) nvtxRangePop();
    }
    void mark(int phase) {
        static const char *const names[kNumMarks] = {"nb.bbox", "nb.morton", "nb.sort", "nb.gather", "nb.build",
                                                     "nb.traverse", "nb.integrate", "nb.end"};
        if (on) cudaEventRecord(ev[phase], ctx->stream);
        if (range_open) nvtxRangePop();
        range_open = phase != kEnd;
        if (range_open) nvtxRangePushA(names[phase]);
    }
    void commit() {
        if (on) ctx->pending.push_back(ev);
    }
};

// Reads finished passes' events into the phase totals (after a synchronise).
void collect_times(nb_ctx *ctx) {
    for (auto &ev: ctx->pending) {
        float ms[kNumMarks - 1];
        for (int p = 0; p < kNumMarks - 1; ++p) {
            ms[p] = 0.f;
            cudaEventElapsedTime(&ms[p], ev[p], ev[p + 1]);
        }
        ctx->times.bbox_ms += ms[kBBox];
        ctx->times.morton_ms += ms[kMorton];
        ctx->times.sort_ms += ms[kSort];
        ctx->times.gather_ms += ms[kGather];
        ctx->times.build_ms += ms[kBuild];
        ctx->times.traverse_ms += ms[kTraverse];
        ctx->times.integrate_ms += ms[kIntegrate];
        ctx->times.passes += 1;
        for (auto e: ev) ctx->event_pool.push_back(e);
    }
    ctx->pending.clear();
}

// Kernel launches of one force pass + drift (for the launch count the bench reports).
int64_t launches_per_pass(const nb_ctx *ctx, bool with_bbox, bool with_drift) {
    if (ctx->cfg.solver == NB_SOLVER_NAIVE) return 1 + (with_drift ? 1 : 0);
    // the dual path adds loadBalancedBreak to the same pipeline
    // morton(1) + scan(1) + 8 sort passes + gather(1) + karras(1) + summarize(1) + emit(1)
    // + root-leaf(1) + traverse(1)
    int64_t k = 1 + 1 + 8 + 1 + 1 + 1 + 1 + 1 + 1;
    if (ctx->n <= 1) k -= 3;  // no Karras internal nodes
    if (ctx->cfg.solver == NB_SOLVER_DUAL_LINEAR_BVH) k += 2;  // loadBalancedBreak and the near-field kernel
    return k + (with_bbox ? 1 : 0) + (with_drift ? 1 : 0);
}

// The dual-tree traversal and near field. The near-field pool and the per-block arenas are sized
// from the body count; when a pass finds them too small (error bits kErrNearPool / kErrDualArena),
// the host grows them to the sizes the pass asked for and runs the traversal again.
int dual_traverse(nb_ctx *ctx, int64_t n, int64_t first, int64_t count, cudaStream_t s) {
    NearPool &np = ctx->dws.near;
    for (int attempt = 0;; ++attempt) {
        launch_dual_traverse(ctx->dnodes, ctx->tw.num_nodes, ctx->pos, n, ctx->cfg.G, ctx->cfg.epsilon,
                             ctx->cfg.theta, ctx->acc, ctx->counts, ctx->dws, ctx->err, s, first, first + count);
        unsigned long long *h = ctx->host_scratch;
        SpillPool &sp = ctx->dws.spill;
        NB_TRY(cudaMemcpyAsync(h, np.counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
               "read near-field pool");
        NB_TRY(cudaMemcpyAsync(h + 5, sp.counters, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
               "read frontier pool");
        NB_TRY(cudaMemcpyAsync(h + 4, ctx->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "read status");
        NB_TRY(cudaStreamSynchronize(s), "dual-tree traversal");
        uint32_t e = 0;
        std::memcpy(&e, h + 4, sizeof(uint32_t));
        const bool pool = (e & kErrNearPool) != 0, arena = (e & kErrDualArena) != 0;
        if ((!pool && !arena) || attempt == 3) return NB_OK;
        if (pool && ((int64_t) h[5] > sp.rec_cap || (int64_t) h[6] > sp.word_cap)) {
            const int64_t recs = (int64_t) h[5], words = (int64_t) h[6];
            dev_free(sp.recs);
            dev_free(sp.rec_field);
            dev_free(sp.words);
            sp.rec_cap = std::max<int64_t>(sp.rec_cap, recs + recs / 4 + 1024);
            sp.word_cap = std::min<int64_t>(std::max<int64_t>(sp.word_cap, words + words / 4 + 4096),
                                            (int64_t(1) << 31) - 1);
            NB_TRY(dev_alloc(&sp.recs, (size_t) sp.rec_cap), "grow frontier pool");
            NB_TRY(dev_alloc(&sp.rec_field, (size_t) sp.rec_cap), "grow frontier pool");
            NB_TRY(dev_alloc(&sp.words, (size_t) sp.word_cap), "grow frontier pool");
        }
        if (pool && ((int64_t) h[0] > np.item_cap || (int64_t) h[1] > np.word_cap)) {
            const int64_t items = (int64_t) h[0], words = (int64_t) h[1];
            dev_free(np.items);
            dev_free(np.words);
            np.item_cap = std::max<int64_t>(np.item_cap, items + items / 4 + 1024);
            np.word_cap = std::min<int64_t>(std::max<int64_t>(np.word_cap, words + words / 4 + 4096),
                                            (int64_t(1) << 31) - 1);
            NB_TRY(dev_alloc(&np.items, (size_t) np.item_cap), "grow near-field pool");
            NB_TRY(dev_alloc(&np.words, (size_t) np.word_cap), "grow near-field pool");
        }
        if (arena) {
            dev_free(ctx->dws.arena);
            ctx->dws.arena_words = std::min<int64_t>(2 * ctx->dws.arena_words, int64_t(1) << 28);
            NB_TRY(dev_alloc(&ctx->dws.arena, (size_t) ctx->dws.blocks * (size_t) ctx->dws.arena_words),
                   "grow dual arena");
        }
        e &= ~(uint32_t) (kErrNearPool | kErrDualArena);
        std::memcpy(h + 4, &e, sizeof(uint32_t));
        NB_TRY(cudaMemcpyAsync(ctx->err, h + 4, sizeof(uint32_t), cudaMemcpyHostToDevice, s), "reset status");
        NB_TRY(cudaMemsetAsync(ctx->counts, 0, 4 * sizeof(unsigned long long), s), "reset counts");
    }
}

// Force pass over a batch of instances: per-instance boxes and codes, a global code sort followed
// by a stable sort on the instance id, one build over (instance, code, index) keys, and one
// traversal over a group table whose 32-target groups never straddle instances.
int force_pass_batch(nb_ctx *ctx, Marks &mk) {
    const int64_t n = ctx->n;
    cudaStream_t s = ctx->stream;
    launch_seg_bbox(ctx->pos, ctx->inst_range, ctx->num_inst, ctx->inst_bbox_slices, ctx->inst_box, s);
    mk.mark(kMorton);
    launch_seg_morton(ctx->pos, n, ctx->inst_of, ctx->inst_box, ctx->keys, ctx->sw.hist, s);
    mk.mark(kSort);
    NB_TRY(launch_radix_sort(ctx->keys, ctx->vals, n, ctx->sw, ctx->err, s), "radix sort");
    launch_inst_keys(ctx->vals, n, ctx->inst_of, ctx->ikeys, s);
    const int64_t tiles = sort_tiles(n);
    cudaMemsetAsync(ctx->inst_lookback, 0, (size_t) ctx->inst_passes * tiles * 256 * sizeof(uint32_t), s);
    cudaMemsetAsync(ctx->inst_tiles, 0, 8 * sizeof(uint32_t), s);
    launch_radix_pass(ctx->ikeys, nullptr, ctx->ikeys2, ctx->ivals, n, 0, ctx->inst_offsets, ctx->inst_lookback,
                      ctx->inst_tiles, ctx->err, s);
    const uint32_t *order = ctx->ivals;
    if (ctx->inst_passes == 2) {
        launch_radix_pass(ctx->ikeys2, ctx->ivals, ctx->ikeys, ctx->ivals2, n, 1, ctx->inst_offsets,
                          ctx->inst_lookback, ctx->inst_tiles, ctx->err, s);
        order = ctx->ivals2;
    }
    launch_compose(order, n, ctx->vals, ctx->keys, ctx->sw.vals_alt, ctx->sw.keys_alt, s);
    mk.mark(kGather);
    launch_gather_state(ctx->sw.vals_alt, n, ctx->pos, ctx->vel, ctx->id, ctx->pos2, ctx->vel2, ctx->id2, s);
    std::swap(ctx->pos, ctx->pos2);
    std::swap(ctx->vel, ctx->vel2);
    std::swap(ctx->id, ctx->id2);
    mk.mark(kBuild);
    BatchSegments seg;
    seg.inst_of = ctx->inst_of;
    seg.inst_theta2 = ctx->inst_theta2;
    seg.inst_range = ctx->inst_range;
    seg.inst_root = ctx->inst_root;
    cudaMemsetAsync(ctx->inst_root, 0xFF, (size_t) ctx->num_inst * sizeof(int), s);
    launch_build_tree(ctx->sw.keys_alt, ctx->pos, n, ctx->cfg.max_leaf_size, ctx->cfg.order, ctx->cfg.theta, ctx->tw,
                      ctx->nodes, ctx->err, s, seg);
    ctx->sorted_codes = ctx->sw.keys_alt;
    mk.mark(kTraverse);
    cudaMemsetAsync(ctx->inst_counts, 0, (size_t) 2 * ctx->num_inst * sizeof(unsigned long long), s);
    launch_bh_traverse(ctx->cfg.order, ctx->nodes, ctx->tw.num_nodes, ctx->pos, n, ctx->pos, n, ctx->cfg.G,
                       ctx->cfg.epsilon, ctx->acc, ctx->counts, ctx->trav, ctx->err, s, ctx->groups, ctx->ngroups,
                       ctx->inst_root, ctx->inst_counts);
    ctx->have_tree = true;
    ctx->acc_is_bh = true;
    if (ctx->timing) ctx->times.launches += launches_per_pass(ctx, false, false) + 4 + ctx->inst_passes;
    return check_cuda(ctx, cudaGetLastError(), "batched force pass");
}

// One force pass over the current state. Leaves accelerations in ctx->acc (current order).
int force_pass(nb_ctx *ctx, Marks &mk) {
    const int64_t n = ctx->n;
    cudaStream_t s = ctx->stream;
    cudaMemsetAsync(ctx->counts, 0, 4 * sizeof(unsigned long long), s);
    ctx->acc_is_dual = false;
    const bool need_bbox = !ctx->bbox_valid;
    mk.mark(kBBox);
    int64_t chunk = n, first = 0, count = n;
    shard_slice(n, ctx->shard_rank, ctx->shard_world, &chunk, &first, &count);
    if (ctx->cfg.solver == NB_SOLVER_NAIVE) {
        mk.mark(kMorton); mk.mark(kSort); mk.mark(kGather); mk.mark(kBuild); mk.mark(kTraverse);
        launch_direct_f32(ctx->pos, n, ctx->pos + first, count, ctx->cfg.G, ctx->cfg.epsilon, ctx->acc + first, s);
        ctx->have_tree = false;
        ctx->acc_is_bh = false;
        if (ctx->timing) ctx->times.launches += 1;
        return check_cuda(ctx, cudaGetLastError(), "naive direct sum");
    }
    if (ctx->num_inst > 0) return force_pass_batch(ctx, mk);
    if (need_bbox) {
        launch_bbox_reset(ctx->bbox, s);
        launch_bbox_reduce(ctx->pos, n, ctx->bbox, s);
    }
    mk.mark(kMorton);
    launch_morton_hist(ctx->pos, n, ctx->bbox, ctx->keys, ctx->sw.hist, s);
    mk.mark(kSort);
    NB_TRY(launch_radix_sort(ctx->keys, ctx->vals, n, ctx->sw, ctx->err, s), "radix sort");
    mk.mark(kGather);
    launch_gather_state(ctx->vals, n, ctx->pos, ctx->vel, ctx->id, ctx->pos2, ctx->vel2, ctx->id2, s);
    std::swap(ctx->pos, ctx->pos2);
    std::swap(ctx->vel, ctx->vel2);
    std::swap(ctx->id, ctx->id2);
    mk.mark(kBuild);
    ctx->sorted_codes = ctx->keys;
    if (ctx->cfg.solver == NB_SOLVER_DUAL_LINEAR_BVH) {
        if (ctx->dual_cap != ctx->cap) return fail(ctx, NB_ERR_CUDA, "dual-tree buffers missing");
        launch_build_dual_tree(ctx->keys, ctx->pos, n, ctx->cfg.max_leaf_size, ctx->cfg.theta, ctx->tw, ctx->dnodes,
                               ctx->err, s);
        mk.mark(kTraverse);
        // a sharded context evaluates only its slice of the Morton-ordered targets
        const int rc = dual_traverse(ctx, n, first, count, s);
        if (rc != NB_OK) return rc;
        ctx->have_tree = true;
        ctx->acc_is_bh = true;
        ctx->acc_is_dual = true;
        if (ctx->timing) ctx->times.launches += launches_per_pass(ctx, need_bbox, false);
        return check_cuda(ctx, cudaGetLastError(), "dual-tree force pass");
    }
    launch_build_tree(ctx->keys, ctx->pos, n, ctx->cfg.max_leaf_size, ctx->cfg.order, ctx->cfg.theta, ctx->tw,
                      ctx->nodes, ctx->err, s);
    mk.mark(kTraverse);
    // a sharded context evaluates only its slice of the Morton-ordered targets
    launch_bh_traverse(ctx->cfg.order, ctx->nodes, ctx->tw.num_nodes, ctx->pos, n, ctx->pos + first, count,
                       ctx->cfg.G, ctx->cfg.epsilon, ctx->acc + first, ctx->counts, ctx->trav, ctx->err, s);
    ctx->have_tree = true;
    ctx->acc_is_bh = true;
    if (ctx->timing) ctx->times.launches += launches_per_pass(ctx, need_bbox, false);
    return check_cuda(ctx, cudaGetLastError(), "force pass");
}

int device_status(nb_ctx *ctx) {
    uint32_t e = 0;
    NB_TRY(cudaMemcpyAsync(&e, ctx->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream), "read status");
    NB_TRY(cudaStreamSynchronize(ctx->stream), "synchronize");
    if (ctx->timing) collect_times(ctx);
    if (e & kErrLookbackTimeout)
        return fail(ctx, NB_ERR_DEVICE_TIMEOUT, "radix sort look-back wait exceeded its limit");
    if (e & kErrNodeOverflow) return fail(ctx, NB_ERR_DEVICE_CHECK, "tree node buffer overflow");
    if (e & kErrTreeDepth) return fail(ctx, NB_ERR_DEVICE_CHECK, "tree walk exceeded the maximum depth");
    if (e & kErrStackOverflow) return fail(ctx, NB_ERR_DEVICE_CHECK, "traversal stack overflow");
    if (e & kErrTraverseLimit) return fail(ctx, NB_ERR_DEVICE_CHECK, "traversal met an invalid tree link");
    if (e & kErrDualArena) return fail(ctx, NB_ERR_DEVICE_CHECK, "dual-tree list or task storage exhausted");
    if (e & kErrNearPool) return fail(ctx, NB_ERR_DEVICE_CHECK, "dual-tree near-field pool exhausted");
    return NB_OK;
}

int begin(nb_ctx *ctx) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    return check_cuda(ctx, cudaSetDevice(ctx->cfg.device), "cudaSetDevice");
}

}  // namespace

extern "C" {

void nb_config_default(nb_config *cfg) {
    if (!cfg) return;
    cfg->solver = NB_SOLVER_LINEAR_BVH;
    cfg->order = 1;
    cfg->G = 1.0f;
    cfg->epsilon = 0.00001f;
    cfg->theta = 0.3f;
    cfg->max_leaf_size = 64;
    cfg->time_step = 0.001f;
    cfg->device = 0;
}

int nb_create(const nb_config *cfg, nb_ctx **out) {
    if (!out) return NB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    nb_ctx *ctx = new nb_ctx();
    int rc = validate(ctx, cfg);
    if (rc != NB_OK) { delete ctx; return rc; }
    ctx->cfg = *cfg;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= cfg->device || cfg->device < 0) {
        cudaGetLastError();
        delete ctx;
        return NB_ERR_CUDA;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major < 10) {
        delete ctx;
        return NB_ERR_UNSUPPORTED;
    }
    if (cudaSetDevice(cfg->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return NB_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    if (dev_alloc(&ctx->bbox, 1) != cudaSuccess || dev_alloc(&ctx->counts, 4) != cudaSuccess ||
        dev_alloc(&ctx->err, 1) != cudaSuccess || dev_alloc(&ctx->sw.hist, 8 * 256) != cudaSuccess ||
        dev_alloc(&ctx->sw.offsets, 8 * 256 + 8) != cudaSuccess || dev_alloc(&ctx->sw.tile_counter, 8) != cudaSuccess ||
        dev_alloc(&ctx->tw.num_nodes, 1) != cudaSuccess) {
        nb_destroy(ctx);
        return NB_ERR_OUT_OF_MEMORY;
    }
    if (cudaMallocHost((void **) &ctx->host_scratch, 8 * sizeof(unsigned long long)) != cudaSuccess) {
        nb_destroy(ctx);
        return NB_ERR_OUT_OF_MEMORY;
    }
    ctx->trav.warps = traverse_resident_warps(cfg->device);
    if (dev_alloc(&ctx->trav.stack, (size_t) ctx->trav.warps * kTraverseStack) != cudaSuccess ||
        dev_alloc(&ctx->trav.group_counter, 1) != cudaSuccess) {
        nb_destroy(ctx);
        return NB_ERR_OUT_OF_MEMORY;
    }
    cudaMemsetAsync(ctx->err, 0, sizeof(uint32_t), ctx->stream);
    cudaMemsetAsync(ctx->counts, 0, 4 * sizeof(unsigned long long), ctx->stream);
    cudaMemsetAsync(ctx->tw.num_nodes, 0, sizeof(int), ctx->stream);
    refresh_names(ctx);
    *out = ctx;
    return NB_OK;
}

int nb_destroy(nb_ctx *ctx) {
    if (!ctx) return NB_OK;
    cudaSetDevice(ctx->cfg.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);
    free_batch(ctx);
    free_buffers(ctx);
    dev_free(ctx->bbox); dev_free(ctx->counts); dev_free(ctx->err); dev_free(ctx->sw.hist);
    dev_free(ctx->sw.offsets); dev_free(ctx->sw.tile_counter); dev_free(ctx->tw.num_nodes); dev_free(ctx->acc64);
    dev_free(ctx->trav.stack); dev_free(ctx->trav.group_counter);
    if (ctx->host_scratch) cudaFreeHost(ctx->host_scratch);
    for (auto &ev: ctx->pending) ctx->event_pool.insert(ctx->event_pool.end(), ev.begin(), ev.end());
    for (auto e: ctx->event_pool) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return NB_OK;
}

const char *nb_last_error(const nb_ctx *ctx) { return ctx ? ctx->error.c_str() : "no context"; }

const char *nb_solver_id(const nb_ctx *ctx) { return ctx ? ctx->id_str.c_str() : ""; }

const char *nb_solver_name(const nb_ctx *ctx) { return ctx ? ctx->name_str.c_str() : ""; }

int nb_set_config(nb_ctx *ctx, const nb_config *cfg) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    int rc = validate(ctx, cfg);
    if (rc != NB_OK) return rc;
    if (cfg->device != ctx->cfg.device) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "the device cannot change");
    if (cfg->solver == NB_SOLVER_DUAL_LINEAR_BVH && ctx->num_inst > 0)
        return fail(ctx, NB_ERR_UNSUPPORTED, "the dual-tree solver runs one instance (no batches)");
    ctx->cfg = *cfg;
    ctx->have_tree = false;
    drop_graph(ctx);
    refresh_names(ctx);
    return ensure_dual(ctx);
}

int nb_get_config(const nb_ctx *ctx, nb_config *cfg) {
    if (!ctx || !cfg) return NB_ERR_INVALID_ARGUMENT;
    *cfg = ctx->cfg;
    return NB_OK;
}

int nb_set_stream(nb_ctx *ctx, void *cuda_stream) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    ctx->stream = cuda_stream ? (cudaStream_t) cuda_stream : ctx->own_stream;
    return NB_OK;
}

void *nb_get_stream(const nb_ctx *ctx) { return ctx ? (void *) ctx->stream : nullptr; }

int64_t nb_body_count(const nb_ctx *ctx) { return ctx ? ctx->n : -1; }

static int set_bodies_impl(nb_ctx *ctx, int64_t n, const void *pm, const void *vel, cudaMemcpyKind kind) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (n < 0 || n > kMaxBodies) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "body count out of range");
    if (n > 0 && !pm) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "positions are NULL");
    int64_t chunk = n, first = 0, count = n;
    shard_slice(n, ctx->shard_rank, ctx->shard_world, &chunk, &first, &count);
    // a sharded context all-gathers whole chunks in place: room for world * chunk bodies
    rc = ensure_capacity(ctx, std::max<int64_t>(n, chunk * ctx->shard_world));
    if (rc != NB_OK) return rc;
    free_batch(ctx);
    drop_graph(ctx);
    ctx->steps_since_set = 0;
    ctx->n = n;
    const size_t bytes = (size_t) n * sizeof(float4);
    if (n > 0) {
        NB_TRY(cudaMemcpyAsync(ctx->pos, pm, bytes, kind, ctx->stream), "copy positions");
        if (vel) NB_TRY(cudaMemcpyAsync(ctx->vel, vel, bytes, kind, ctx->stream), "copy velocities");
        else NB_TRY(cudaMemsetAsync(ctx->vel, 0, bytes, ctx->stream), "zero velocities");
        NB_TRY(cudaMemsetAsync(ctx->acc, 0, bytes, ctx->stream), "zero accelerations");
        launch_iota(ctx->id, n, ctx->stream);
    }
    ctx->bbox_valid = false;
    ctx->have_tree = false;
    ctx->have_acc = false;
    return check_cuda(ctx, cudaGetLastError(), "set bodies");
}

int nb_set_bodies(nb_ctx *ctx, int64_t n, const float *pos_mass, const float *velocity) {
    int rc = set_bodies_impl(ctx, n, pos_mass, velocity, cudaMemcpyHostToDevice);
    if (rc != NB_OK) return rc;
    // The caller may reuse its host buffers as soon as this returns.
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "set bodies");
}

int nb_set_bodies_device(nb_ctx *ctx, int64_t n, const void *d_pos_mass, const void *d_velocity) {
    return set_bodies_impl(ctx, n, d_pos_mass, d_velocity, cudaMemcpyDeviceToDevice);
}

static int get_state_impl(nb_ctx *ctx, void *pm, void *vel, cudaMemcpyKind kind, bool host) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    const int64_t n = ctx->n;
    const size_t bytes = (size_t) n * sizeof(float4);
    if (n > 0) {
        // pos2/vel2 are free between passes; use them to restore the caller's order.
        if (pm) {
            launch_scatter_by_id(ctx->id, n, ctx->pos, ctx->pos2, ctx->stream);
            NB_TRY(cudaMemcpyAsync(pm, ctx->pos2, bytes, kind, ctx->stream), "copy positions out");
        }
        if (vel) {
            launch_scatter_by_id(ctx->id, n, ctx->vel, ctx->vel2, ctx->stream);
            NB_TRY(cudaMemcpyAsync(vel, ctx->vel2, bytes, kind, ctx->stream), "copy velocities out");
        }
    }
    rc = check_cuda(ctx, cudaGetLastError(), "get bodies");
    if (rc != NB_OK) return rc;
    return host ? device_status(ctx) : NB_OK;
}

int nb_get_bodies(nb_ctx *ctx, float *pos_mass, float *velocity) {
    return get_state_impl(ctx, pos_mass, velocity, cudaMemcpyDeviceToHost, true);
}

int nb_get_bodies_device(nb_ctx *ctx, void *d_pos_mass, void *d_velocity) {
    return get_state_impl(ctx, d_pos_mass, d_velocity, cudaMemcpyDeviceToDevice, false);
}

static int copy_acc_out(nb_ctx *ctx, void *out, cudaMemcpyKind kind, bool host) {
    const int64_t n = ctx->n;
    if (!ctx->have_acc) return fail(ctx, NB_ERR_NO_BODIES, "no accelerations computed yet");
    if (n > 0) {
        launch_scatter_by_id(ctx->id, n, ctx->acc, ctx->pos2, ctx->stream);
        NB_TRY(cudaMemcpyAsync(out, ctx->pos2, (size_t) n * sizeof(float4), kind, ctx->stream), "copy accelerations");
    }
    int rc = check_cuda(ctx, cudaGetLastError(), "accelerations out");
    if (rc != NB_OK) return rc;
    return host ? device_status(ctx) : NB_OK;
}

int nb_update_accelerations(nb_ctx *ctx, float *acc_out) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    Marks mk(ctx);
    if (ctx->n > 0) {
        rc = force_pass(ctx, mk);
        if (rc != NB_OK) return rc;
    }
    mk.mark(kIntegrate);
    mk.mark(kEnd);
    mk.commit();
    ctx->have_acc = true;
    if (acc_out) return copy_acc_out(ctx, acc_out, cudaMemcpyDeviceToHost, true);
    return NB_OK;
}

int nb_get_accelerations(nb_ctx *ctx, float *acc_out) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!acc_out) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    return copy_acc_out(ctx, acc_out, cudaMemcpyDeviceToHost, true);
}

int nb_get_accelerations_device(nb_ctx *ctx, void *d_acc_out) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!d_acc_out) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    return copy_acc_out(ctx, d_acc_out, cudaMemcpyDeviceToDevice, false);
}

static int one_step(nb_ctx *ctx) {
    Marks mk(ctx);
    int rc;
    if (ctx->n > 0) {
        rc = force_pass(ctx, mk);
        if (rc != NB_OK) return rc;
        mk.mark(kIntegrate);
        // a sharded context drifts only its slice; the box is recomputed after the all-gather
        const bool reduce_box = ctx->cfg.solver != NB_SOLVER_NAIVE && ctx->num_inst == 0 && ctx->shard_world == 1;
        int64_t chunk = ctx->n, first = 0, count = ctx->n;
        shard_slice(ctx->n, ctx->shard_rank, ctx->shard_world, &chunk, &first, &count);
        if (reduce_box) launch_bbox_reset(ctx->bbox, ctx->stream);
        launch_kick_drift(ctx->pos + first, ctx->vel + first, ctx->acc + first, count, ctx->cfg.time_step,
                          reduce_box ? ctx->bbox : nullptr, ctx->stream);
        ctx->bbox_valid = reduce_box;
        if (ctx->timing) ctx->times.launches += 1;
        rc = check_cuda(ctx, cudaGetLastError(), "kick-drift");
        if (rc != NB_OK) return rc;
    } else {
        mk.mark(kMorton); mk.mark(kSort); mk.mark(kGather); mk.mark(kBuild); mk.mark(kTraverse);
        mk.mark(kIntegrate);
    }
    mk.mark(kEnd);
    mk.commit();
    ctx->have_acc = true;
    ctx->steps_since_set += 1;
    return NB_OK;
}

// Two steps captured once and replayed: after two steps the bodies are back in the same buffers,
// so the graph's pointers stay valid. Timing marks are not captured.
static int graph_pair(nb_ctx *ctx) {
    if (!ctx->graph2) {
        // captured steps see the steady-state shape: the previous drift already reduced the box
        // and every lazily initialised launch setting is in place
        cudaGraph_t g = nullptr;
        ctx->graph_pos = ctx->pos;
        NB_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = one_step(ctx);
        if (rc == NB_OK) rc = one_step(ctx);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        ctx->steps_since_set -= 2;  // recorded, not executed
        if (rc != NB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        NB_TRY(e, "end capture");
        e = cudaGraphInstantiate(&ctx->graph2, g, 0);
        cudaGraphDestroy(g);
        NB_TRY(e, "instantiate graph");
    }
    NB_TRY(cudaGraphLaunch(ctx->graph2, ctx->stream), "launch graph");
    ctx->steps_since_set += 2;
    ctx->have_acc = true;
    return NB_OK;
}

int nb_step(nb_ctx *ctx, int32_t steps) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (steps < 0) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "negative step count");
    if (ctx->shard_world > 1 && steps > 1)
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "a sharded context steps once per call (all-gather between steps)");
    int32_t k = 0;
    while (k < steps) {
        // the dual-tree pass reads its pool usage back on the host, so it is never captured
        const bool pair = ctx->use_graphs && !ctx->timing && ctx->n > 0 && steps - k >= 2 && ctx->steps_since_set > 0 &&
                          ctx->cfg.solver != NB_SOLVER_DUAL_LINEAR_BVH;
        // The captured pair reads and writes the buffers it was recorded with; each plain force
        // pass swaps the ping-pong buffers, so replay only when the bodies sit where it expects.
        if (pair && (!ctx->graph2 || ctx->pos == ctx->graph_pos)) {
            rc = graph_pair(ctx);
            if (rc != NB_OK) return rc;
            k += 2;
            continue;
        }
        rc = one_step(ctx);
        if (rc != NB_OK) return rc;
        k += 1;
    }
    return NB_OK;
}

int nb_synchronize(nb_ctx *ctx) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    return device_status(ctx);
}

int nb_get_instance_counts(nb_ctx *ctx, int32_t count, uint64_t *particle_particle, uint64_t *node_particle) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (ctx->num_inst == 0) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "the context holds no batch of instances");
    if (count != ctx->num_inst) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "count must equal the number of instances");
    if (!particle_particle || !node_particle) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    if (!ctx->acc_is_bh) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "no force pass has run on this batch");
    std::vector<unsigned long long> c((size_t) 2 * count);
    NB_TRY(cudaMemcpyAsync(c.data(), ctx->inst_counts, c.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           ctx->stream), "read instance counts");
    rc = device_status(ctx);
    if (rc != NB_OK) return rc;
    for (int32_t k = 0; k < count; ++k) {
        particle_particle[k] = c[2 * (size_t) k];
        node_particle[k] = c[2 * (size_t) k + 1];
    }
    return NB_OK;
}

int nb_get_counts(nb_ctx *ctx, nb_counts *out) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!out) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    unsigned long long c[4] = {0, 0, 0, 0};
    NB_TRY(cudaMemcpyAsync(c, ctx->counts, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream), "read counts");
    rc = device_status(ctx);
    if (rc != NB_OK) return rc;
    // device counters: {particle-particle, node-particle, particle-node, node-node}
    if (ctx->acc_is_bh) {
        out->particle_particle = c[0];
        out->node_particle = c[1];
    } else {
        out->particle_particle = (uint64_t) ctx->n * (uint64_t) ctx->n;
        out->node_particle = 0;
    }
    out->particle_node = ctx->acc_is_dual ? c[2] : 0;
    out->node_node = ctx->acc_is_dual ? c[3] : 0;
    return NB_OK;
}

int nb_enable_timing(nb_ctx *ctx, int enable) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    rc = device_status(ctx);
    ctx->timing = enable != 0;
    ctx->times = nb_phase_times{};
    return rc;
}

int nb_get_phase_times(nb_ctx *ctx, nb_phase_times *out) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!out) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    rc = device_status(ctx);
    *out = ctx->times;
    return rc;
}

int nb_get_tree(nb_ctx *ctx, int64_t *num_nodes, int32_t *record_floats, uint64_t *sorted_codes, uint32_t *sorted_ids,
                float *records, float *bbox) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!ctx->have_tree) return fail(ctx, NB_ERR_NO_BODIES, "no tree has been built");
    int nn = 0;
    NB_TRY(cudaMemcpyAsync(&nn, ctx->tw.num_nodes, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "read tree");
    uint32_t box[6];
    NB_TRY(cudaMemcpyAsync(box, ctx->bbox, sizeof(box), cudaMemcpyDeviceToHost, ctx->stream), "read bbox");
    rc = device_status(ctx);
    if (rc != NB_OK) return rc;
    const bool dual = ctx->acc_is_dual;
    const int rf = dual ? 32 : rec_floats(ctx->cfg.order);
    if (num_nodes) *num_nodes = nn;
    if (record_floats) *record_floats = rf;
    if (bbox) {
        for (int k = 0; k < 3; ++k) {
            bbox[k] = ordered_to_float(box[k]);
            bbox[3 + k] = ordered_to_float(~box[3 + k]);
        }
    }
    const int64_t n = ctx->n;
    if (sorted_codes && n > 0)
        NB_TRY(cudaMemcpyAsync(sorted_codes, ctx->sorted_codes, (size_t) n * 8, cudaMemcpyDeviceToHost, ctx->stream),
               "codes");
    if (sorted_ids && n > 0)
        NB_TRY(cudaMemcpyAsync(sorted_ids, ctx->id, (size_t) n * 4, cudaMemcpyDeviceToHost, ctx->stream), "ids");
    if (records && nn > 0 && dual) {
        std::vector<float4> a((size_t) nn), b((size_t) nn), c((size_t) nn), q((size_t) nn * 4);
        std::vector<int2> link((size_t) nn);
        const size_t f4 = (size_t) nn * sizeof(float4);
        NB_TRY(cudaMemcpyAsync(a.data(), ctx->dnodes.bmin, f4, cudaMemcpyDeviceToHost, ctx->stream), "records");
        NB_TRY(cudaMemcpyAsync(b.data(), ctx->dnodes.bmax, f4, cudaMemcpyDeviceToHost, ctx->stream), "records");
        NB_TRY(cudaMemcpyAsync(c.data(), ctx->dnodes.com, f4, cudaMemcpyDeviceToHost, ctx->stream), "records");
        NB_TRY(cudaMemcpyAsync(q.data(), ctx->dnodes.q, 4 * f4, cudaMemcpyDeviceToHost, ctx->stream), "records");
        NB_TRY(cudaMemcpyAsync(link.data(), ctx->dnodes.link, (size_t) nn * sizeof(int2), cudaMemcpyDeviceToHost,
                               ctx->stream), "records");
        rc = device_status(ctx);
        if (rc != NB_OK) return rc;
        for (int64_t k = 0; k < nn; ++k) {
            float *r = records + k * rf;
            std::memcpy(r, &a[k], 16);
            std::memcpy(r + 4, &b[k], 16);
            std::memcpy(r + 8, &c[k], 16);
            std::memcpy(r + 12, &link[k], 8);
            r[14] = 0.f;
            r[15] = 0.f;
            std::memcpy(r + 16, &q[4 * k], 64);
        }
    } else if (records && nn > 0) {
        const int pf = pay_float4s(ctx->cfg.order);
        std::vector<float4> mac((size_t) nn), pay((size_t) nn * pf);
        std::vector<int2> link((size_t) nn);
        NB_TRY(cudaMemcpyAsync(mac.data(), ctx->nodes.mac, (size_t) nn * sizeof(float4), cudaMemcpyDeviceToHost,
                               ctx->stream), "records");
        NB_TRY(cudaMemcpyAsync(link.data(), ctx->nodes.link, (size_t) nn * sizeof(int2), cudaMemcpyDeviceToHost,
                               ctx->stream), "records");
        NB_TRY(cudaMemcpyAsync(pay.data(), ctx->nodes.pay, (size_t) nn * pf * sizeof(float4), cudaMemcpyDeviceToHost,
                               ctx->stream), "records");
        rc = device_status(ctx);
        if (rc != NB_OK) return rc;
        for (int64_t k = 0; k < nn; ++k) {
            float *r = records + k * rf;
            std::memcpy(r, &mac[k], 16);
            std::memcpy(r + 4, &link[k], 8);
            r[6] = 0.f;
            r[7] = 0.f;
            std::memcpy(r + 8, &pay[k * pf], (size_t) pf * 16);
        }
    }
    return device_status(ctx);
}

int nb_energy(nb_ctx *ctx, double *kinetic, double *potential) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!kinetic || !potential) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    const int64_t need = energy_parts(ctx->n) + 2;
    if (ctx->acc64_cap < need) {
        dev_free(ctx->acc64);
        ctx->acc64_cap = 0;
        NB_TRY(dev_alloc(&ctx->acc64, (size_t) need), "alloc energy buffer");
        ctx->acc64_cap = need;
    }
    double *out = ctx->acc64 + need - 2;
    launch_energy_f64(ctx->pos, ctx->vel, ctx->n, (double) ctx->cfg.G, (double) ctx->cfg.epsilon, ctx->acc64, out,
                      ctx->stream);
    NB_TRY(cudaGetLastError(), "energy");
    double h[2] = {0.0, 0.0};
    NB_TRY(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "read energy");
    rc = device_status(ctx);
    if (rc != NB_OK) return rc;
    *kinetic = h[0];
    *potential = h[1];
    return NB_OK;
}

int nb_direct_device(nb_ctx *ctx, int64_t n, const void *d_bodies, int64_t nt, const void *d_targets, void *d_acc,
                     int32_t precision) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (n < 0 || nt < 0 || (n > 0 && !d_bodies) || (nt > 0 && (!d_targets || !d_acc)))
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "bad direct-sum arguments");
    if (precision == 32)
        launch_direct_f32((const float4 *) d_bodies, n, (const float4 *) d_targets, nt, ctx->cfg.G, ctx->cfg.epsilon,
                          (float4 *) d_acc, ctx->stream);
    else if (precision == 64)
        launch_direct_f64((const float4 *) d_bodies, n, (const float4 *) d_targets, nt, (double) ctx->cfg.G,
                          (double) ctx->cfg.epsilon, (double *) d_acc, ctx->stream);
    else
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "precision must be 32 or 64");
    return check_cuda(ctx, cudaGetLastError(), "direct sum");
}

// Builds the batch tables for `count` instances whose bodies already sit back to back in the
// context's state arrays (ctx->n bodies in total).
static int build_batch_tables(nb_ctx *ctx, int32_t count, const int64_t *sizes, const float *thetas) {
    const int64_t n = ctx->n;
    drop_graph(ctx);
    std::vector<int2> range((size_t) count);
    std::vector<int> group_first((size_t) count);
    std::vector<float> theta2((size_t) count);
    std::vector<uint32_t> offsets(8 * 256 + 8, 0), hist(2 * 256, 0);
    ctx->inst_start.resize(count);
    ctx->inst_size.assign(sizes, sizes + count);
    int64_t start = 0, ngroups = 0;
    for (int32_t k = 0; k < count; ++k) {
        ctx->inst_start[k] = start;
        range[k] = make_int2((int) start, (int) (start + sizes[k] - 1));
        group_first[k] = (int) ngroups;
        ngroups += (sizes[k] + 31) / 32;
        const float th = thetas ? thetas[k] : ctx->cfg.theta;
        theta2[k] = th * th;  // the reference compares against theta * theta in float
        hist[k & 255] += (uint32_t) sizes[k];
        hist[256 + (k >> 8)] += (uint32_t) sizes[k];
        start += sizes[k];
    }
    const int64_t largest = count > 0 ? *std::max_element(sizes, sizes + count) : 1;
    ctx->inst_bbox_slices = (int) std::min<int64_t>(std::max<int64_t>((largest + 8191) / 8192, 1), 64);
    const int passes = count > 256 ? 2 : 1;
    for (int p = 0; p < passes; ++p) {
        uint32_t acc = 0;
        bool trivial = false;
        for (int d = 0; d < 256; ++d) {
            offsets[p * 256 + d] = acc;
            acc += hist[p * 256 + d];
            if ((int64_t) hist[p * 256 + d] == n) trivial = true;
        }
        offsets[8 * 256 + p] = trivial ? 1u : 0u;
    }
    const int64_t tiles = sort_tiles(n);
    if (n > ctx->batch_body_cap) {  // per-body buffers grow only
        dev_free(ctx->inst_of); dev_free(ctx->ikeys); dev_free(ctx->ikeys2); dev_free(ctx->ivals);
        dev_free(ctx->ivals2); dev_free(ctx->inst_lookback);
        ctx->batch_body_cap = 0;
        const int64_t cap = std::max<int64_t>(n, 1);
        NB_TRY(dev_alloc(&ctx->inst_of, (size_t) cap), "alloc batch");
        NB_TRY(dev_alloc(&ctx->ikeys, (size_t) cap), "alloc batch");
        NB_TRY(dev_alloc(&ctx->ikeys2, (size_t) cap), "alloc batch");
        NB_TRY(dev_alloc(&ctx->ivals, (size_t) cap), "alloc batch");
        NB_TRY(dev_alloc(&ctx->ivals2, (size_t) cap), "alloc batch");
        NB_TRY(dev_alloc(&ctx->inst_lookback, (size_t) 2 * sort_tiles(cap) * 256), "alloc batch");
        ctx->batch_body_cap = cap;
    }
    if (count > ctx->batch_inst_cap) {
        dev_free(ctx->inst_root); dev_free(ctx->inst_theta2); dev_free(ctx->inst_box); dev_free(ctx->inst_range);
        dev_free(ctx->group_first); dev_free(ctx->inst_counts);
        ctx->batch_inst_cap = 0;
        NB_TRY(dev_alloc(&ctx->inst_root, (size_t) count), "alloc batch");
        NB_TRY(dev_alloc(&ctx->inst_theta2, (size_t) count), "alloc batch");
        NB_TRY(dev_alloc(&ctx->inst_box, (size_t) count * 6), "alloc batch");
        NB_TRY(dev_alloc(&ctx->inst_range, (size_t) count), "alloc batch");
        NB_TRY(dev_alloc(&ctx->group_first, (size_t) count), "alloc batch");
        NB_TRY(dev_alloc(&ctx->inst_counts, (size_t) 2 * count), "alloc batch");
        ctx->batch_inst_cap = count;
    }
    if (ngroups > ctx->batch_group_cap) {
        dev_free(ctx->groups);
        ctx->batch_group_cap = 0;
        NB_TRY(dev_alloc(&ctx->groups, (size_t) ngroups), "alloc batch");
        ctx->batch_group_cap = ngroups;
    }
    if (!ctx->inst_offsets) NB_TRY(dev_alloc(&ctx->inst_offsets, offsets.size()), "alloc batch");
    if (!ctx->inst_tiles) NB_TRY(dev_alloc(&ctx->inst_tiles, 8), "alloc batch");
    (void) tiles;
    int *group_first_dev = ctx->group_first;
    cudaStream_t s = ctx->stream;
    NB_TRY(cudaMemcpyAsync(ctx->inst_theta2, theta2.data(), theta2.size() * sizeof(float), cudaMemcpyHostToDevice, s),
           "copy");
    NB_TRY(cudaMemcpyAsync(ctx->inst_range, range.data(), range.size() * sizeof(int2), cudaMemcpyHostToDevice, s), "copy");
    NB_TRY(cudaMemcpyAsync(group_first_dev, group_first.data(), group_first.size() * sizeof(int), cudaMemcpyHostToDevice,
                           s), "copy");
    launch_fill_tables(ctx->inst_range, group_first_dev, count, ctx->inst_of, ctx->groups, s);
    NB_TRY(cudaMemcpyAsync(ctx->inst_offsets, offsets.data(), offsets.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
           "copy");
    ctx->num_inst = count;
    ctx->ngroups = ngroups;
    ctx->inst_passes = passes;
    // host vectors are released on return: wait for the copies out of them
    return check_cuda(ctx, cudaStreamSynchronize(s), "batch tables");
}

static int check_instances(nb_ctx *ctx, int32_t count, const int64_t *sizes, const float *thetas, int64_t *total) {
    if (count < 1 || count > 65535 || !sizes) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "1..65535 instances required");
    int64_t n = 0;
    for (int32_t k = 0; k < count; ++k) {
        if (sizes[k] < 1) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "every instance needs at least one body");
        n += sizes[k];
    }
    if (n > kMaxBodies) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "body count out of range");
    if (thetas)
        for (int32_t k = 0; k < count; ++k)
            if (!(thetas[k] >= 0.f)) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "theta must be >= 0");
    *total = n;
    return NB_OK;
}

int nb_set_instances(nb_ctx *ctx, int32_t count, const int64_t *sizes, const float *thetas, const float *pos_mass,
                     const float *velocity) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (ctx->cfg.solver == NB_SOLVER_DUAL_LINEAR_BVH)
        return fail(ctx, NB_ERR_UNSUPPORTED, "the dual-tree solver runs one instance");
    if (ctx->shard_world > 1)
        return fail(ctx, NB_ERR_UNSUPPORTED, "batched instances are not sharded (run independent batches per rank)");
    int64_t n = 0;
    rc = check_instances(ctx, count, sizes, thetas, &n);
    if (rc != NB_OK) return rc;
    rc = set_bodies_impl(ctx, n, pos_mass, velocity, cudaMemcpyHostToDevice);
    if (rc != NB_OK) return rc;
    return build_batch_tables(ctx, count, sizes, thetas);
}

int32_t nb_instance_count(const nb_ctx *ctx) { return ctx ? (ctx->num_inst > 0 ? ctx->num_inst : 1) : -1; }

int nb_get_instance_roots(nb_ctx *ctx, int32_t *roots) {
    int rc = begin(ctx);
    if (rc != NB_OK) return rc;
    if (!roots) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "output is NULL");
    if (ctx->num_inst == 0) {
        roots[0] = 0;
        return NB_OK;
    }
    NB_TRY(cudaMemcpyAsync(roots, ctx->inst_root, (size_t) ctx->num_inst * sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream), "read roots");
    return device_status(ctx);
}

int nb_enable_graphs(nb_ctx *ctx, int enable) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    ctx->use_graphs = enable != 0;
    if (!ctx->use_graphs) drop_graph(ctx);
    return NB_OK;
}

int nb_set_fp64_summaries(nb_ctx *ctx, int64_t min_bodies) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    if (min_bodies < 0) return fail(ctx, NB_ERR_INVALID_ARGUMENT, "negative body count");
    ctx->tw.fp64_min_bodies = (int) std::min<int64_t>(min_bodies, INT32_MAX);
    ctx->have_tree = false;
    drop_graph(ctx);  // captured builds hold the old setting
    return NB_OK;
}

int nb_selftest_bounded_wait(int32_t device, int32_t wait_ms) {
    if (wait_ms < 1 || wait_ms > 2000) return NB_ERR_INVALID_ARGUMENT;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return NB_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return NB_ERR_CUDA;
    uint32_t e = 0;
    if (lookback_timeout_selftest((unsigned long long) wait_ms * 1000000ull, &e) != cudaSuccess) return NB_ERR_CUDA;
    return (e & kErrLookbackTimeout) ? NB_ERR_DEVICE_TIMEOUT : NB_OK;
}

int nb_set_traversal_shape(nb_ctx *ctx, int32_t block_threads, int32_t slab_entries) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    if (block_threads == 0) block_threads = 256;
    if (slab_entries == 0) slab_entries = 64;
    if (!traversal_shape_valid(block_threads, slab_entries))
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "traversal shape: block of 128 or 256 threads, slab of 32 or 64");
    ctx->trav.threads = block_threads;
    ctx->trav.slab = slab_entries;
    drop_graph(ctx);  // captured passes hold the old launch shape
    return NB_OK;
}

int nb_get_traversal_shape(const nb_ctx *ctx, int32_t *block_threads, int32_t *slab_entries) {
    if (!ctx || !block_threads || !slab_entries) return NB_ERR_INVALID_ARGUMENT;
    *block_threads = ctx->trav.threads;
    *slab_entries = ctx->trav.slab;
    return NB_OK;
}

int nb_shard_range(int64_t n, int32_t rank, int32_t world, int64_t *chunk, int64_t *first, int64_t *count) {
    if (n < 0 || world < 1 || rank < 0 || rank >= world || !chunk || !first || !count)
        return NB_ERR_INVALID_ARGUMENT;
    shard_slice(n, rank, world, chunk, first, count);
    return NB_OK;
}

int nb_set_shard(nb_ctx *ctx, int32_t rank, int32_t world) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    if (world < 1 || world > 4096 || rank < 0 || rank >= world)
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "shard rank out of range");
    if (world > 1 && ctx->num_inst > 0)
        return fail(ctx, NB_ERR_UNSUPPORTED, "batched instances are not sharded");
    int64_t chunk = 0, first = 0, count = 0;
    shard_slice(ctx->n, rank, world, &chunk, &first, &count);
    if (ctx->n > 0 && chunk * world > ctx->cap)
        return fail(ctx, NB_ERR_INVALID_ARGUMENT, "call nb_set_shard before nb_set_bodies (buffers lack gather room)");
    ctx->shard_rank = rank;
    ctx->shard_world = world;
    ctx->bbox_valid = false;
    drop_graph(ctx);
    return NB_OK;
}

int nb_shard_buffers(nb_ctx *ctx, void **d_pos_mass, void **d_velocity, int64_t *capacity) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    if (d_pos_mass) *d_pos_mass = ctx->pos;
    if (d_velocity) *d_velocity = ctx->vel;
    if (capacity) *capacity = ctx->cap;
    return NB_OK;
}

int nb_shard_gathered(nb_ctx *ctx) {
    if (!ctx) return NB_ERR_INVALID_ARGUMENT;
    ctx->bbox_valid = false;
    return NB_OK;
}

void *nb_host_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    return p;
}

void nb_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Serving: continuous batching of independent simulations on one device.
//
// Requests (a body set, theta and a step count) queue on the host until the resident-memory
// budget admits them. Every tick retires finished requests (their final bodies are copied out),
// admits queued ones in arrival order while they fit, re-lays out the device state when the set
// changed (survivors move device-to-device, newcomers are copied in once), and advances every
// running request by one step in ONE batched force pass (nb_set_instances' pipeline). Each
// request keeps its bodies and its per-step tree on the device from admission to completion.
// A request's arithmetic is exactly that of running it alone, so its result does not depend on
// what else is in the batch.
// ---------------------------------------------------------------------------------------------

namespace {

// Device bytes one resident body costs the context (state, sort, tree and batch buffers, with
// the growth headroom of a re-layout); admission charges this per body against the budget.
constexpr uint64_t kResidentBytesPerBody = 544;

struct ServedRequest {
    int64_t id = 0;
    int64_t n = 0;
    float theta = 0.f;
    int32_t steps = 0, done = 0;
    int32_t state = 0;   // 0 queued, 1 running, 2 done
    bool cancel = false; // running request to drop at the next tick
    int64_t start = -1;  // first body position in the batch (or in the staged layout) while resident
    std::vector<float> pm, vel;  // input until admitted, result once done
};

}  // namespace

struct nb_server {
    nb_ctx *ctx = nullptr;
    uint64_t budget = 0;
    std::string error;
    int64_t next_id = 1;
    std::deque<ServedRequest *> queue;
    std::vector<ServedRequest *> active;
    std::map<int64_t, ServedRequest *> all;
    float4 *tpos = nullptr, *tvel = nullptr;
    uint32_t *tid = nullptr;
    int64_t tcap = 0;
    bool staged = false;          // the staging buffers hold the running set's layout; the context does not
    bool dirty = false;           // the context's layout still holds requests that left the running set
    int32_t fail_next[2] = {0, 0};  // injected allocation failures: staging buffers, context buffers
    nb_server_stats stats{};
};

// An injected allocation failure at `point` (fault-injection tests), consumed once.
static bool injected(nb_server *sv, int point) {
    if (sv->fail_next[point] <= 0) return false;
    sv->fail_next[point] -= 1;
    return true;
}

static int server_fail(nb_server *sv, int rc) {
    if (sv && sv->ctx) sv->error = sv->ctx->error;
    return rc;
}

// Lays the running set out anew. Two stages, so that a failure leaves a consistent server:
//   1. staging: the staging buffers are grown if needed and every running request is copied into
//      them (resident ones from the context, newcomers from their host copies). A failure here
//      changes nothing; the caller puts the newcomers back in the queue.
//   2. loading: the context's buffers are grown if needed and the staged layout is copied in,
//      with the batch tables. A failure here leaves the layout staged (`staged`); the next tick
//      finishes it before stepping.
static int server_relayout(nb_server *sv) {
    nb_ctx *ctx = sv->ctx;
    cudaStream_t s = ctx->stream;
    int64_t total = 0;
    for (auto *r: sv->active) total += r->n;
    if (!sv->staged) {
        if (total > sv->tcap) {
            if (injected(sv, 0)) {
                sv->error = "out of device memory for the re-layout (injected)";
                return NB_ERR_OUT_OF_MEMORY;
            }
            dev_free(sv->tpos); dev_free(sv->tvel); dev_free(sv->tid);
            sv->tcap = 0;
            if (dev_alloc(&sv->tpos, (size_t) total) != cudaSuccess ||
                dev_alloc(&sv->tvel, (size_t) total) != cudaSuccess ||
                dev_alloc(&sv->tid, (size_t) total) != cudaSuccess) {
                cudaGetLastError();
                dev_free(sv->tpos); dev_free(sv->tvel); dev_free(sv->tid);
                sv->error = "out of device memory for the re-layout";
                return NB_ERR_OUT_OF_MEMORY;
            }
            sv->tcap = total;
        }
        int64_t off = 0;
        for (auto *r: sv->active) {
            const size_t bytes = (size_t) r->n * sizeof(float4);
            if (r->start >= 0) {  // resident: move device-to-device, rebase the caller indices
                if (cudaMemcpyAsync(sv->tpos + off, ctx->pos + r->start, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                    cudaMemcpyAsync(sv->tvel + off, ctx->vel + r->start, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                    cudaMemcpyAsync(sv->tid + off, ctx->id + r->start, (size_t) r->n * 4, cudaMemcpyDeviceToDevice, s) !=
                        cudaSuccess) {
                    sv->error = "re-layout copy failed";
                    return NB_ERR_CUDA;
                }
                launch_add_offset(sv->tid + off, r->n, off - r->start, s);
            } else {  // newcomer: one copy in
                if (cudaMemcpyAsync(sv->tpos + off, r->pm.data(), bytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                    cudaMemcpyAsync(sv->tvel + off, r->vel.data(), bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) {
                    sv->error = "copy-in failed";
                    return NB_ERR_CUDA;
                }
                launch_iota(sv->tid + off, r->n, s, (uint32_t) off);
            }
            off += r->n;
        }
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            sv->error = "re-layout failed";
            return NB_ERR_CUDA;
        }
        off = 0;
        for (auto *r: sv->active) {
            r->start = off;
            off += r->n;
        }
        sv->staged = true;
    }
    // 2. loading
    if (total > ctx->cap && injected(sv, 1)) {
        sv->error = "out of device memory for the context buffers (injected)";
        return NB_ERR_OUT_OF_MEMORY;
    }
    int rc = ensure_capacity(ctx, total);
    if (rc != NB_OK) return server_fail(sv, rc);
    drop_graph(ctx);
    ctx->num_inst = 0;  // the batch buffers stay allocated; the tables are rebuilt below
    ctx->n = total;
    ctx->steps_since_set = 0;
    ctx->bbox_valid = false;
    ctx->have_tree = false;
    ctx->have_acc = false;
    sv->stats.relayouts += 1;
    if (total > 0) {
        const size_t bytes = (size_t) total * sizeof(float4);
        if (cudaMemcpyAsync(ctx->pos, sv->tpos, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(ctx->vel, sv->tvel, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(ctx->id, sv->tid, (size_t) total * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
            sv->error = "re-layout copy failed";
            return NB_ERR_CUDA;
        }
        std::vector<int64_t> sizes;
        std::vector<float> thetas;
        for (auto *r: sv->active) {
            sizes.push_back(r->n);
            thetas.push_back(r->theta);
        }
        rc = build_batch_tables(ctx, (int32_t) sizes.size(), sizes.data(), thetas.data());
        if (rc != NB_OK) return server_fail(sv, rc);
    }
    sv->staged = false;
    for (auto *r: sv->active) {  // host input copies are no longer needed
        std::vector<float>().swap(r->pm);
        std::vector<float>().swap(r->vel);
    }
    return NB_OK;
}

// Copies a running request's bodies out, in its caller order.
static int server_collect(nb_server *sv, ServedRequest *r) {
    nb_ctx *ctx = sv->ctx;
    std::vector<float4> pos((size_t) r->n), vel((size_t) r->n);
    std::vector<uint32_t> ids((size_t) r->n);
    cudaStream_t s = ctx->stream;
    if (cudaMemcpyAsync(pos.data(), ctx->pos + r->start, (size_t) r->n * 16, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(vel.data(), ctx->vel + r->start, (size_t) r->n * 16, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(ids.data(), ctx->id + r->start, (size_t) r->n * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        sv->error = "copy-out failed";
        return NB_ERR_CUDA;
    }
    r->pm.assign((size_t) r->n * 4, 0.f);
    r->vel.assign((size_t) r->n * 4, 0.f);
    for (int64_t k = 0; k < r->n; ++k) {
        const int64_t local = (int64_t) ids[k] - r->start;
        if (local < 0 || local >= r->n) {
            sv->error = "corrupt body ids in a served request";
            return NB_ERR_DEVICE_CHECK;
        }
        std::memcpy(&r->pm[4 * local], &pos[k], 16);
        std::memcpy(&r->vel[4 * local], &vel[k], 16);
    }
    return NB_OK;
}

extern "C" {

int nb_server_create(const nb_config *cfg, uint64_t hbm_budget_bytes, nb_server **out) {
    if (!out) return NB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    nb_ctx *ctx = nullptr;
    int rc = nb_create(cfg, &ctx);
    if (rc != NB_OK) return rc;
    if (cfg->solver != NB_SOLVER_LINEAR_BVH) {
        nb_destroy(ctx);
        return NB_ERR_UNSUPPORTED;
    }
    nb_server *sv = new nb_server();
    sv->ctx = ctx;
    sv->budget = hbm_budget_bytes;
    *out = sv;
    return NB_OK;
}

int nb_server_destroy(nb_server *sv) {
    if (!sv) return NB_OK;
    for (auto &kv: sv->all) delete kv.second;
    cudaSetDevice(sv->ctx->cfg.device);
    dev_free(sv->tpos); dev_free(sv->tvel); dev_free(sv->tid);
    nb_destroy(sv->ctx);
    delete sv;
    return NB_OK;
}

const char *nb_server_last_error(const nb_server *sv) { return sv ? sv->error.c_str() : "no server"; }

void *nb_server_context(nb_server *sv) { return sv ? (void *) sv->ctx : nullptr; }

int nb_server_submit(nb_server *sv, int64_t n, const float *pos_mass, const float *velocity, float theta,
                     int32_t steps, int64_t *request_id) {
    if (!sv || !request_id) return NB_ERR_INVALID_ARGUMENT;
    if (n < 1 || !pos_mass || steps < 0 || !(theta >= 0.f)) {
        sv->error = "a request needs at least one body, theta >= 0 and steps >= 0";
        return NB_ERR_INVALID_ARGUMENT;
    }
    if ((uint64_t) n * kResidentBytesPerBody > sv->budget) {
        sv->error = "request larger than the whole memory budget";
        return NB_ERR_OUT_OF_MEMORY;
    }
    for (int64_t k = 0; k < 4 * n; ++k) {
        if (!std::isfinite(pos_mass[k]) || (velocity && !std::isfinite(velocity[k]))) {
            sv->error = "non-finite position, mass or velocity";
            return NB_ERR_INVALID_ARGUMENT;
        }
    }
    auto *r = new ServedRequest();
    r->id = sv->next_id++;
    r->n = n;
    r->theta = theta;
    r->steps = steps;
    r->pm.assign(pos_mass, pos_mass + 4 * n);
    if (velocity) r->vel.assign(velocity, velocity + 4 * n);
    else r->vel.assign((size_t) 4 * n, 0.f);
    sv->all[r->id] = r;
    sv->queue.push_back(r);
    sv->stats.submitted += 1;
    *request_id = r->id;
    return NB_OK;
}

int nb_server_tick(nb_server *sv, int32_t *completed_now) {
    if (!sv) return NB_ERR_INVALID_ARGUMENT;
    nb_ctx *ctx = sv->ctx;
    if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) return NB_ERR_CUDA;
    if (completed_now) *completed_now = 0;
    // 0. a layout left staged by a failed tick is loaded before anything else
    if (sv->staged) {
        int rc = server_relayout(sv);
        if (rc != NB_OK) {
            sv->stats.failed_ticks += 1;
            return rc;
        }
    }
    int32_t completed = 0;
    bool changed = sv->dirty;
    // 1. retire requests whose steps are done, drop cancelled ones
    std::vector<ServedRequest *> keep;
    for (auto *r: sv->active) {
        if (r->cancel) {
            sv->all.erase(r->id);
            delete r;
            sv->stats.cancelled += 1;
            changed = true;
        } else if (r->done >= r->steps) {
            int rc = server_collect(sv, r);
            if (rc != NB_OK) return rc;
            r->state = 2;
            r->start = -1;
            ++completed;
            changed = true;
        } else {
            keep.push_back(r);
        }
    }
    sv->active.swap(keep);
    // 2. admit queued requests in arrival order while they fit the budget
    uint64_t resident = 0;
    for (auto *r: sv->active) resident += (uint64_t) r->n * kResidentBytesPerBody;
    std::vector<ServedRequest *> admitted;
    while (!sv->queue.empty()) {
        ServedRequest *r = sv->queue.front();
        const uint64_t need = (uint64_t) r->n * kResidentBytesPerBody;
        if (resident + need > sv->budget) break;
        sv->queue.pop_front();
        if (r->steps == 0) {  // nothing to run: the result is the input
            r->state = 2;
            ++completed;
            continue;
        }
        r->state = 1;
        r->start = -1;
        sv->active.push_back(r);
        admitted.push_back(r);
        resident += need;
        changed = true;
    }
    sv->stats.completed += completed;
    if (completed_now) *completed_now = completed;
    if (changed) {
        int rc = server_relayout(sv);
        if (rc != NB_OK) {
            sv->stats.failed_ticks += 1;
            if (!sv->staged) {
                // nothing was laid out: the newcomers go back to the front of the queue, in order
                for (auto it = admitted.rbegin(); it != admitted.rend(); ++it) {
                    (*it)->state = 0;
                    sv->queue.push_front(*it);
                }
                sv->active.resize(sv->active.size() - admitted.size());
                resident = 0;
                for (auto *r: sv->active) resident += (uint64_t) r->n * kResidentBytesPerBody;
                // the context keeps its previous layout (retired or cancelled requests included,
                // stepped but unused) until the next tick lays the running set out again
                sv->dirty = true;
            }
            sv->stats.queued = (int64_t) sv->queue.size();
            sv->stats.running = (int64_t) sv->active.size();
            sv->stats.resident_bytes = resident;
            return rc;
        }
    }
    sv->dirty = false;
    // 3. one batched step for every running request
    if (!sv->active.empty()) {
        int rc = nb_step(ctx, 1);
        if (rc != NB_OK) return server_fail(sv, rc);
        for (auto *r: sv->active) {
            r->done += 1;
            sv->stats.body_steps += r->n;
        }
    }
    sv->stats.ticks += 1;
    sv->stats.queued = (int64_t) sv->queue.size();
    sv->stats.running = (int64_t) sv->active.size();
    sv->stats.resident_bytes = resident;
    return NB_OK;
}

int nb_server_cancel(nb_server *sv, int64_t request_id) {
    if (!sv) return NB_ERR_INVALID_ARGUMENT;
    auto it = sv->all.find(request_id);
    if (it == sv->all.end()) {
        sv->error = "unknown request";
        return NB_ERR_INVALID_ARGUMENT;
    }
    ServedRequest *r = it->second;
    if (r->state == 1) {  // running: dropped from the layout at the next tick
        r->cancel = true;
        return NB_OK;
    }
    if (r->state == 0) {
        for (auto q = sv->queue.begin(); q != sv->queue.end(); ++q) {
            if (*q == r) {
                sv->queue.erase(q);
                break;
            }
        }
    }
    sv->all.erase(it);
    delete r;
    sv->stats.cancelled += 1;
    return NB_OK;
}

int nb_server_inject_alloc_failures(nb_server *sv, int32_t point, int32_t count) {
    if (!sv || point < 0 || point > 1 || count < 0) return NB_ERR_INVALID_ARGUMENT;
    sv->fail_next[point] = count;
    return NB_OK;
}

int nb_server_status(nb_server *sv, int64_t request_id, int32_t *state, int32_t *steps_done) {
    if (!sv) return NB_ERR_INVALID_ARGUMENT;
    auto it = sv->all.find(request_id);
    if (it == sv->all.end()) {
        sv->error = "unknown request";
        return NB_ERR_INVALID_ARGUMENT;
    }
    if (state) *state = it->second->state;
    if (steps_done) *steps_done = it->second->done;
    return NB_OK;
}

int nb_server_take_result(nb_server *sv, int64_t request_id, float *pos_mass, float *velocity) {
    if (!sv) return NB_ERR_INVALID_ARGUMENT;
    auto it = sv->all.find(request_id);
    if (it == sv->all.end() || it->second->state != 2) {
        sv->error = "request unknown or not done";
        return NB_ERR_INVALID_ARGUMENT;
    }
    ServedRequest *r = it->second;
    if (pos_mass) std::memcpy(pos_mass, r->pm.data(), r->pm.size() * sizeof(float));
    if (velocity) std::memcpy(velocity, r->vel.data(), r->vel.size() * sizeof(float));
    sv->all.erase(it);
    delete r;
    return NB_OK;
}

int nb_server_get_stats(nb_server *sv, nb_server_stats *out) {
    if (!sv || !out) return NB_ERR_INVALID_ARGUMENT;
    sv->stats.queued = (int64_t) sv->queue.size();
    sv->stats.running = (int64_t) sv->active.size();
    *out = sv->stats;
    return NB_OK;
}

}  // extern "C"
