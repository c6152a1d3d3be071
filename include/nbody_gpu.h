/*
 * nbody_gpu.h - C ABI of the B200 (sm_100a) force-evaluation path of the n-body simulator.
 *
 * One opaque context stands in for one reference solver instance (Solver<Rule>,
 * src/NBody/Simulation/Solver.h:26-187) together with its rule (Gravity, src/NBody/Physics/Rules/Gravity.h)
 * and its tree (LinearBVH, src/NBody/Simulation/Solvers/Trees/LinearBVH.h). The context owns the
 * bodies' device-resident state; host buffers are copied in and out at the calls that take them.
 *
 * Conventions
 *   - Every function returns an int status: NB_OK (0) or a negative NB_ERR_* code; the message of
 *     the last failure is available from nb_last_error(). (The reference reports errors through
 *     assert and spdlog only, MultiSolver.h:86, 104-105.)
 *   - Bodies cross the boundary as 4 floats each: positions+masses as (x, y, z, m), velocities
 *     as (vx, vy, vz, unused), accelerations as (ax, ay, az, 0), always in the caller's order.
 *     The reference keeps Position/Velocity/Acceleration as glm::vec3 and Mass as float
 *     components in an EnTT registry (src/NBody/Simulation/Simulation.h:45); a caller gathers
 *     those views into these arrays (one pass over view<Position, Mass>, one over
 *     view<Velocity>) and scatters the accelerations back the same way.
 *   - "_device" variants take device pointers (16-byte aligned) on the context's device.
 *   - Work is ordered on the context's CUDA stream (nb_set_stream to share the caller's stream).
 *     Calls that return host data synchronise that stream.
 *   - A context is not re-entrant: one thread at a time per context. Different contexts are
 *     independent.
 */
#ifndef NBODY_GPU_H
#define NBODY_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NB_OK 0
#define NB_ERR_INVALID_ARGUMENT (-1)
#define NB_ERR_CUDA (-2)
#define NB_ERR_OUT_OF_MEMORY (-3)
#define NB_ERR_NO_BODIES (-4)
#define NB_ERR_DEVICE_TIMEOUT (-5)
#define NB_ERR_UNSUPPORTED (-6)
#define NB_ERR_DEVICE_CHECK (-7)

/* Solver selection: the reference's Solver::id() strings (Solver.h:89-91). */
typedef enum nb_solver {
    /* ActiveTreeSolver<LinearBVH<S>, DiagonalOverCenterDistance, Gravity>
     * (src/NBody/Simulation/Solvers/ActiveTreeSolver.h:16-82, LinearBVHSolver.h:18-53):
     * order 1 = LinearBVHSolver ("linear-bvh"), order 2 = QuadrupoleLinearBVHSolver ("linear-bvh-4p"). */
    NB_SOLVER_LINEAR_BVH = 0,
    /* NaiveSolver (src/NBody/Simulation/Solvers/NaiveSolver.h:12-53, "naive"): FP32 direct sum. */
    NB_SOLVER_NAIVE = 1,
    /* MultipoleImplicitLinearBVHFMMSolver<3> (ImplicitLinearBVHFMMSolver.h:15-33 over
     * ImplicitDualTraversalSolver.h:17-82, "implicit-linear-bvh-fmm-8p"): dual-tree traversal under
     * DiagonalOverSeparation, octupole node moments, local fields of order 4. Requires order 3. */
    NB_SOLVER_DUAL_LINEAR_BVH = 2
} nb_solver;

typedef struct nb_config {
    int32_t solver;        /* nb_solver */
    int32_t order;         /* multipole order of the node summaries: 1 (centre of mass) or 2 (quadrupole);
                            * 3 (octupole) with NB_SOLVER_DUAL_LINEAR_BVH */
    float G;               /* Gravity::g()        (Gravity.h:195, 407) */
    float epsilon;         /* Gravity::epsilon(): added to r^2 (Gravity.h:207) */
    float theta;           /* ActiveTreeSolver::theta() (ActiveTreeSolver.h:78-80); the dual solver's
                            * DiagonalOverSeparation::theta() (DiagonalOverSeparation.h:19-27) */
    int32_t max_leaf_size; /* LinearBVH::maxLeafSize() (LinearBVH.h:135-137) */
    float time_step;       /* Solver::timeStep() (Solver.h:101) */
    int32_t device;        /* CUDA device ordinal */
} nb_config;

/* Interaction counts of the last force pass, SimpleTrackingRule's convention
 * (src/NBody/Physics/Rules/SimpleTrackingRule.h:29-51): one per Gravity call. */
typedef struct nb_counts {
    uint64_t particle_particle;
    uint64_t particle_node;
    uint64_t node_particle;
    uint64_t node_node;
} nb_counts;

/* Device time per phase, summed over the force passes since timing was enabled (CUDA events on
 * the context's stream). Kernel launches of each phase are counted in `launches`. */
typedef struct nb_phase_times {
    double bbox_ms, morton_ms, sort_ms, gather_ms, build_ms, traverse_ms, integrate_ms;
    int64_t passes;
    int64_t launches;
} nb_phase_times;

typedef struct nb_ctx nb_ctx;

/* Reference defaults: Gravity(G = 1, epsilon = 1e-5) (Gravity.h:195), theta 0.3
 * (ActiveTreeSolver.h:21), maxLeafSize 64 (LinearBVH.h:88), dt 0.001 (Solver.h:34), order 1. */
void nb_config_default(nb_config *cfg);

/* Construct a solver (Solver(Simulation&, Rule&), Solver.h:51). Fails with NB_ERR_CUDA when no
 * usable sm_100 device is present: there is no CPU fallback. */
int nb_create(const nb_config *cfg, nb_ctx **out);
int nb_destroy(nb_ctx *ctx);
const char *nb_last_error(const nb_ctx *ctx);

/* Solver::id() / Solver::name() of the configured solver (Solver.h:89-91, LinearBVHSolver.h:28-44). */
const char *nb_solver_id(const nb_ctx *ctx);
const char *nb_solver_name(const nb_ctx *ctx);

/* Change theta, leaf size, G, epsilon, dt or the solver between steps
 * (ActiveTreeSolver::theta(), LinearBVH::maxLeafSize(), Gravity::g()/epsilon(), Solver::timeStep()). */
int nb_set_config(nb_ctx *ctx, const nb_config *cfg);
int nb_get_config(const nb_ctx *ctx, nb_config *cfg);

/* Order the context's work on a caller-owned cudaStream_t (NULL: the context's own stream). */
int nb_set_stream(nb_ctx *ctx, void *cuda_stream);
void *nb_get_stream(const nb_ctx *ctx);

/* Replace the body set (the Simulation's Position/Mass/Velocity components). velocity may be NULL
 * (zero velocities). n may be 0. Coordinates are expected well inside float range: the traversals
 * pad partly filled work with massless records far away (1e30, and 1e18 in the dual tree's M2P),
 * whose terms are exactly zero for targets with coordinates below 1e29 (1e17 for the dual tree)
 * in magnitude. */
int nb_set_bodies(nb_ctx *ctx, int64_t n, const float *pos_mass, const float *velocity);
int nb_set_bodies_device(nb_ctx *ctx, int64_t n, const void *d_pos_mass, const void *d_velocity);
int64_t nb_body_count(const nb_ctx *ctx);

/* Read the current bodies back in the caller's order. Either pointer may be NULL. */
int nb_get_bodies(nb_ctx *ctx, float *pos_mass, float *velocity);
int nb_get_bodies_device(nb_ctx *ctx, void *d_pos_mass, void *d_velocity);

/* Solver::updateAccelerations() (Solver.h:115; ActiveTreeSolver.h:33-72; NaiveSolver.h:22-52):
 * compute every body's acceleration from the current positions. acc_out (n x 4 floats, caller's
 * order) may be NULL to leave the result on the device. */
int nb_update_accelerations(nb_ctx *ctx, float *acc_out);
int nb_get_accelerations(nb_ctx *ctx, float *acc_out);
int nb_get_accelerations_device(nb_ctx *ctx, void *d_acc_out);

/* Solver::step() repeated `steps` times (Solver.h:103-139): accelerations, then v += a dt,
 * then x += v dt. Device-resident between steps; asynchronous on the context's stream. */
int nb_step(nb_ctx *ctx, int32_t steps);

/* Wait for the context's work; reports device-side check failures (e.g. a bounded wait that
 * expired) as NB_ERR_DEVICE_TIMEOUT / NB_ERR_DEVICE_CHECK. */
int nb_synchronize(nb_ctx *ctx);

/* SimpleTrackingRule counts of the last force pass (synchronises). */
int nb_get_counts(nb_ctx *ctx, nb_counts *out);

/* Per-phase device timing (CUDA events), off by default. */
int nb_enable_timing(nb_ctx *ctx, int enable);
int nb_get_phase_times(nb_ctx *ctx, nb_phase_times *out);

/* Parity taps on the last tree built (synchronise). Any output pointer may be NULL.
 *   num_nodes     node count of the linear BVH (preorder)
 *   record_floats floats per node record (12 for order 1, 16 for order 2; 32 for the dual solver:
 *                 box min xyz + body count (int bits), box max xyz + diagonal length, centre of
 *                 mass + mass, link (2 ints, 2 zero), quadrupole (6), octupole (10));
 *                 see nb_tree_record
 *   sorted_codes  n Morton codes in sorted order (MortonSort.h:46-73)
 *   sorted_ids    n caller indices of the sorted bodies (the Morton sort's permutation)
 *   records       num_nodes * record_floats floats
 *   bbox          6 floats: global box min xyz, max xyz (SummaryType.h:73-81) */
int nb_get_tree(nb_ctx *ctx, int64_t *num_nodes, int32_t *record_floats, uint64_t *sorted_codes,
                uint32_t *sorted_ids, float *records, float *bbox);

/* Batched independent instances (one launch per phase over all of them). Replaces the body set
 * with `count` instances laid out back to back: instance k holds sizes[k] bodies (at least one)
 * starting after instance k-1 in pos_mass / velocity (4 floats per body; velocity may be NULL).
 * thetas[k] is instance k's opening angle (NULL: the config's theta); G, epsilon, leaf size, order
 * and dt are shared. Each instance is an independent simulation: its own bounding box, Morton
 * codes and tree (ActiveTreeSolver.h:33-72 per instance), and its results are bit-identical to
 * running it alone. nb_update_accelerations / nb_step / nb_get_bodies then act on the whole batch,
 * in the concatenated caller order. At most 65535 instances. */
int nb_set_instances(nb_ctx *ctx, int32_t count, const int64_t *sizes, const float *thetas, const float *pos_mass,
                     const float *velocity);
int32_t nb_instance_count(const nb_ctx *ctx);
/* Preorder index of each instance's root in the last tree built (count entries; synchronises). */
int nb_get_instance_roots(nb_ctx *ctx, int32_t *roots);
/* SimpleTrackingRule counts (SimpleTrackingRule.h:29-51) of the last force pass, per instance of
 * the batch: particle_particle[k] and node_particle[k] for instance k, exactly what a standalone
 * solver over instance k counts (count must equal nb_instance_count; synchronises). */
int nb_get_instance_counts(nb_ctx *ctx, int32_t count, uint64_t *particle_particle, uint64_t *node_particle);

/* Capture pairs of steps in a CUDA graph and replay it in nb_step (off by default; per-phase
 * timing, when enabled, runs the steps uncaptured). */
int nb_enable_graphs(nb_ctx *ctx, int enable);

/* Precision option, off by default (min_bodies = 0): internal tree nodes of at least min_bodies
 * bodies combine their children's centre of mass and moments in FP64 and round once to FP32
 * (MultipoleMassSummary.h:37-97 evaluated in double). Bounding boxes, and therefore every
 * approximation decision and interaction count, are unchanged; with the option on, the summaries
 * of those nodes are no longer bit-identical to the reference's FP32 ones. */
int nb_set_fp64_summaries(nb_ctx *ctx, int64_t min_bodies);

/* Self-test of the device-side bounded waits (no counterpart in the reference, which has no device
 * waits): runs one radix-sort pass on `device` whose look-back can never complete (every index in
 * bounds), with its wait limited to wait_ms (1..2000) milliseconds. Returns NB_ERR_DEVICE_TIMEOUT
 * when the wait ended at its limit and reported it, as designed; the device stays usable. */
int nb_selftest_bounded_wait(int32_t device, int32_t wait_ms);

/* Launch shape of the Barnes-Hut traversal (no counterpart in the reference, whose TBB loop has no
 * such knob; LinearBVH::maxLeafSize, LinearBVH.h:135-137, is the one it has): block_threads
 * threads per block (128 or 256) and slab_entries staged partially accepted nodes per warp (32 or
 * 64); 0 selects the default (256, 64). Decisions and interaction counts do not depend on it;
 * accelerations sum the same terms, possibly in another order. The autotuner
 * (nbody_b200/autotune.py) picks it per workload. */
int nb_set_traversal_shape(nb_ctx *ctx, int32_t block_threads, int32_t slab_entries);
int nb_get_traversal_shape(const nb_ctx *ctx, int32_t *block_threads, int32_t *slab_entries);

/* Target sharding of one instance over `world` processes, one GPU each (the path shards over
 * targets; every rank needs all sources). Every rank holds the same state.
 * A force pass still sorts and builds over all bodies, but evaluates accelerations, and nb_step
 * applies the kick-drift, only for this rank's slice of the Morton-ordered bodies:
 *   chunk = ceil(n / world) rounded up to a multiple of 32, slice = [rank * chunk, (rank+1) * chunk) ∩ [0, n).
 * After each nb_step(ctx, 1) the caller all-gathers the chunks of positions and velocities in place
 * (recv = the buffers of nb_shard_buffers, rank r's chunk at offset r * chunk; an NCCL in-place
 * all-gather) and calls nb_shard_gathered. Sharded contexts step once per nb_step call;
 * accelerations are valid for the own slice only. Call nb_set_shard before nb_set_bodies, so the
 * buffers get room for world * chunk bodies. Not for batches. The dual-tree solver drops every
 * task whose passive node holds none of the slice's targets, so its far-field and near-field work
 * both split over the ranks. */
int nb_shard_range(int64_t n, int32_t rank, int32_t world, int64_t *chunk, int64_t *first, int64_t *count);
int nb_set_shard(nb_ctx *ctx, int32_t rank, int32_t world);
/* Current state buffers (Morton slot order, float4 per body; they alternate between passes, so
 * query them after every step) and their capacity in bodies. */
int nb_shard_buffers(nb_ctx *ctx, void **d_pos_mass, void **d_velocity, int64_t *capacity);
int nb_shard_gathered(nb_ctx *ctx);

/* Serving: continuous batching of independent simulations on one device (no reference
 * counterpart beyond Solver::step per simulation). A request is a body set with its own theta and
 * step count. nb_server_tick retires finished requests (copying their final bodies out), admits
 * queued ones in arrival order while their resident memory fits the budget, and advances every
 * running request by one step in one batched force pass. Each request's result equals running it
 * alone (bit-identical). */
typedef struct nb_server nb_server;
typedef struct nb_server_stats {
    int64_t submitted, queued, running, completed;
    int64_t body_steps;      /* body-steps advanced so far */
    int64_t ticks, relayouts;
    uint64_t resident_bytes; /* budget charge of the running requests */
    int64_t cancelled;       /* requests dropped by nb_server_cancel */
    int64_t failed_ticks;    /* ticks that returned an error (the server stayed consistent) */
} nb_server_stats;
int nb_server_create(const nb_config *cfg, uint64_t hbm_budget_bytes, nb_server **out);
int nb_server_destroy(nb_server *sv);
const char *nb_server_last_error(const nb_server *sv);
/* The server's solver context (for nb_set_stream, nb_enable_timing, nb_get_counts). */
void *nb_server_context(nb_server *sv);
/* Queue a request (bodies copied; velocity may be NULL). Fails with NB_ERR_OUT_OF_MEMORY when
 * the request alone exceeds the budget, and with NB_ERR_INVALID_ARGUMENT for non-finite input. */
int nb_server_submit(nb_server *sv, int64_t n, const float *pos_mass, const float *velocity, float theta,
                     int32_t steps, int64_t *request_id);
/* One tick. A failed tick leaves the server consistent: if the new layout could not be staged,
 * the newly admitted requests return to the front of the queue; if it was staged but could not be
 * loaded, the next tick loads it before stepping. */
int nb_server_tick(nb_server *sv, int32_t *completed_now);
/* Drop a request: queued or done ones at once, running ones from the layout at the next tick.
 * A cancelled request is forgotten. */
int nb_server_cancel(nb_server *sv, int64_t request_id);
/* Fault injection for tests: the next `count` device allocations at `point` fail
 * (0: the re-layout's staging buffers, 1: the context's buffers when they must grow). */
int nb_server_inject_alloc_failures(nb_server *sv, int32_t point, int32_t count);
/* state: 0 queued, 1 running, 2 done. */
int nb_server_status(nb_server *sv, int64_t request_id, int32_t *state, int32_t *steps_done);
/* Final bodies of a done request in its caller order (then the request is forgotten). */
int nb_server_take_result(nb_server *sv, int64_t request_id, float *pos_mass, float *velocity);
int nb_server_get_stats(nb_server *sv, nb_server_stats *out);

/* Energy diagnostics of the current bodies in FP64 (synchronises): kinetic = sum 1/2 m |v|^2 and
 * potential = -G/2 sum_i sum_j m_i m_j / sqrt(|r_ij|^2 + epsilon), pairs at equal positions
 * excluded as the force excludes them (Gravity.h:203). O(n^2) on the device. */
int nb_energy(nb_ctx *ctx, double *kinetic, double *potential);

/* Direct sum on device pointers: accelerations of nt targets (4 floats each) from n bodies.
 * precision 32: FP32, acc 4 floats per target (NaiveSolver arithmetic).
 * precision 64: FP64 accumulation, acc 3 doubles per target (accuracy reference). */
int nb_direct_device(nb_ctx *ctx, int64_t n, const void *d_bodies, int64_t nt, const void *d_targets,
                     void *d_acc, int32_t precision);

/* Morton-code sort that allocates no device memory (no counterpart in the reference: it serves
 * callers that cannot call cudaMalloc, such as applications whose own pool owns all device memory
 * or step loops that must not take cudaMalloc's implicit device synchronisation).
 * Sorts n 64-bit codes (device pointer d_codes) into d_sorted_codes, with d_sorted_ids[k] = the
 * input index of the k-th smallest code; equal codes keep their input order. All three are
 * caller-owned device buffers. Scratch comes from one static device array of about 16 MiB that
 * every GPU loading this library holds until exit: n must be at most 2^20 (larger n is rejected
 * with NB_ERR_INVALID_ARGUMENT). The first call on a device looks up that array with the device
 * current; make it before any stream capture. Calls share the array: calls that overlap on the
 * GPU race. Runs on cuda_stream (NULL: the legacy default stream) and waits for it. */
int nb_sort_codes_noalloc(const uint64_t *d_codes, uint64_t *d_sorted_codes, uint32_t *d_sorted_ids, int64_t n,
                          void *cuda_stream);

/* Page-locked host buffers for fast copies in and out (cudaMallocHost / cudaFreeHost). */
void *nb_host_alloc(size_t bytes);
void nb_host_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* NBODY_GPU_H */
