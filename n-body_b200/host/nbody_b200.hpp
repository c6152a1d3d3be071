// C++ host interface of the B200 force path: the reference's Solver / Gravity / Simulation
// surface (NBody::Solver<Rule>, src/NBody/Simulation/Solver.h:26-187; NBody::Physics::Gravity,
// src/NBody/Physics/Rules/Gravity.h:187-410; NBody::Simulation, src/NBody/Simulation/Simulation.h)
// over the C ABI in include/nbody_gpu.h. Header-only; link with libnbody_b200.so.
//
// Differences from the reference, by design:
//   - Simulation holds plain arrays (positions, velocities, masses, accelerations in particle
//     order) instead of an EnTT registry; the reference's views map onto them one to one.
//   - Errors raise nbody_b200::Error (the reference asserts or logs, MultiSolver.h:86, 104-105).
//   - step() keeps the bodies on the device between calls and copies them back once per call;
//     step(n) runs n steps on the device with a single copy back (the device-resident fast path).
//   - There is no CPU fallback: constructing a solver without an sm_100 device throws.
//   - The reference's sigc signals (signal_status, signal_computeTime, signal_finished) are plain
//     std::function callbacks, and slot_step is stepAsync() on a std::thread.
#pragma once

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nbody_gpu.h"

namespace nbody_b200 {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string &what) : std::runtime_error(what), _status(status) {}
    int status() const { return _status; }

private:
    int _status;
};

struct vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
    friend bool operator==(const vec3 &a, const vec3 &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
    friend vec3 operator+(const vec3 &a, const vec3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
    friend vec3 operator-(const vec3 &a, const vec3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
    friend vec3 operator*(const vec3 &a, float s) { return {a.x * s, a.y * s, a.z * s}; }
    friend vec3 operator/(const vec3 &a, float s) { return {a.x / s, a.y / s, a.z / s}; }
};

// BoundingBox (src/NBody/Physics/BoundingBox.h:17-72): an empty box is (+max, -max), so the
// first position extends it to a point.
struct BoundingBox {
    vec3 min{FLT_MAX, FLT_MAX, FLT_MAX}, max{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    vec3 center() const { return (max + min) / 2.0f; }
    vec3 diagonal() const { return max - min; }
    float maxSideLength() const {
        const vec3 d = diagonal();
        return std::max({d.x, d.y, d.z});
    }
    // half-open in every axis, as the reference's contains()
    bool contains(const vec3 &p) const {
        return min.x <= p.x && min.y <= p.y && min.z <= p.z && p.x < max.x && p.y < max.y && p.z < max.z;
    }
};

// Gravity rule: G and the softening epsilon added to r^2 (Gravity.h:195, 207, 407-409).
class Gravity {
public:
    explicit Gravity(float G = 1.0f, float epsilon = 0.00001f) : _G(G), _epsilon(epsilon) {}
    float &g() { return _G; }
    const float &g() const { return _G; }
    float &epsilon() { return _epsilon; }
    const float &epsilon() const { return _epsilon; }

private:
    float _G, _epsilon;
};

// The bodies of a simulation in particle order. Particles without an acceleration component in
// the reference (inactive as passive) are not modelled: every particle is active and passive.
class Simulation {
public:
    std::vector<vec3> position, velocity, acceleration;
    std::vector<float> mass;

    std::size_t particleCount() const { return position.size(); }

    std::size_t newParticle(vec3 p, vec3 v, float m) {
        position.push_back(p);
        velocity.push_back(v);
        mass.push_back(m);
        acceleration.push_back({});
        return position.size() - 1;
    }

    void clear() {
        position.clear();
        velocity.clear();
        acceleration.clear();
        mass.clear();
    }

    // Simulation::removeParticle (Simulation.cpp:73-79); the other particles keep their order.
    void removeParticle(std::size_t i) {
        if (i >= particleCount()) throw std::out_of_range("no such particle");
        position.erase(position.begin() + (std::ptrdiff_t) i);
        velocity.erase(velocity.begin() + (std::ptrdiff_t) i);
        acceleration.erase(acceleration.begin() + (std::ptrdiff_t) i);
        mass.erase(mass.begin() + (std::ptrdiff_t) i);
    }

    // Simulation::averagePosition / totalMass / centerOfMass / interactionCount / boundingBox
    // (Simulation.cpp:85-132): float sums over the particles in order. Every particle is active
    // and passive here, so the interaction count is N^2 and all three boxes are the same.
    vec3 averagePosition() const {
        vec3 sum;
        for (const vec3 &p: position) sum = sum + p;
        return sum / (float) particleCount();
    }
    float totalMass() const {
        float m = 0.f;
        for (float v: mass) m += v;
        return m;
    }
    vec3 centerOfMass() const {
        vec3 sum;
        float m = 0.f;
        for (std::size_t i = 0; i < particleCount(); ++i) {
            sum = sum + position[i] * mass[i];
            m += mass[i];
        }
        return sum / m;
    }
    std::size_t interactionCount() const { return particleCount() * particleCount(); }
    BoundingBox boundingBox() const {
        BoundingBox b;
        for (const vec3 &p: position) {
            b.min = {std::min(b.min.x, p.x), std::min(b.min.y, p.y), std::min(b.min.z, p.z)};
            b.max = {std::max(b.max.x, p.x), std::max(b.max.y, p.y), std::max(b.max.z, p.z)};
        }
        return b;
    }
    BoundingBox activeBoundingBox() const { return boundingBox(); }
    BoundingBox passiveBoundingBox() const { return boundingBox(); }

    // 4 floats per body, as the C ABI takes them
    std::vector<float> packedPositionMass() const {
        std::vector<float> out(4 * particleCount());
        for (std::size_t i = 0; i < particleCount(); ++i) {
            out[4 * i] = position[i].x;
            out[4 * i + 1] = position[i].y;
            out[4 * i + 2] = position[i].z;
            out[4 * i + 3] = mass[i];
        }
        return out;
    }
    std::vector<float> packedVelocity() const {
        std::vector<float> out(4 * particleCount(), 0.f);
        for (std::size_t i = 0; i < particleCount(); ++i) {
            out[4 * i] = velocity[i].x;
            out[4 * i + 1] = velocity[i].y;
            out[4 * i + 2] = velocity[i].z;
        }
        return out;
    }
    void unpackPositionMass(const std::vector<float> &pm) {
        for (std::size_t i = 0; i < particleCount(); ++i) {
            position[i] = {pm[4 * i], pm[4 * i + 1], pm[4 * i + 2]};
            mass[i] = pm[4 * i + 3];
        }
    }
    void unpackVelocity(const std::vector<float> &v) {
        for (std::size_t i = 0; i < particleCount(); ++i) velocity[i] = {v[4 * i], v[4 * i + 1], v[4 * i + 2]};
    }
    void unpackAcceleration(const std::vector<float> &a) {
        for (std::size_t i = 0; i < particleCount(); ++i) acceleration[i] = {a[4 * i], a[4 * i + 1], a[4 * i + 2]};
    }
};

// Interaction counts (SimpleTrackingRule's convention, SimpleTrackingRule.h:29-51).
struct InteractionCounts {
    uint64_t particleParticle = 0, particleNode = 0, nodeParticle = 0, nodeNode = 0;
};

// Solver<Rule> (Solver.h:26-187) over one device context. The subclasses fix the algorithm.
class Solver {
public:
    Solver(const Solver &) = delete;
    Solver &operator=(const Solver &) = delete;
    virtual ~Solver() {
        if (_thread.joinable()) _thread.join();
        if (_ctx) nb_destroy(_ctx);
    }

    // Solver::id / name (Solver.h:89-91), as the reference formats them
    std::string id() const { return nb_solver_id(_ctx); }
    std::string name() const { return nb_solver_name(_ctx); }

    // ActiveTreeSolver::theta (ActiveTreeSolver.h:78-80) / DiagonalOverSeparation::theta
    float theta() const { return config().theta; }
    void setTheta(float t) { update([&](nb_config &c) { c.theta = t; }); }
    // LinearBVH::maxLeafSize (LinearBVH.h:135-137)
    int maxLeafSize() const { return config().max_leaf_size; }
    void setMaxLeafSize(int l) { update([&](nb_config &c) { c.max_leaf_size = l; }); }
    // Solver::timeStep (Solver.h:101); per solver here rather than a static
    float timeStep() const { return config().time_step; }
    void setTimeStep(float dt) { update([&](nb_config &c) { c.time_step = dt; }); }

    Simulation &simulation() { return _sim; }
    Gravity &rule() { return _rule; }
    // Solver::maxThreadCount (Solver.h:38, 97-99) caps the reference's TBB workers. The device path
    // has no host worker pool, so the value is kept for source compatibility and not used.
    std::size_t &maxThreadCount() { return _max_threads; }
    const std::size_t &maxThreadCount() const { return _max_threads; }

    // Solver::updateAccelerations (ActiveTreeSolver.h:33-72 / ImplicitDualTraversalSolver.h:42-69):
    // accelerations of the simulation's current bodies, written to simulation().acceleration.
    void updateAccelerations() {
        upload();
        std::vector<float> acc(4 * _sim.particleCount());
        check(nb_update_accelerations(_ctx, acc.empty() ? nullptr : acc.data()));
        _sim.unpackAcceleration(acc);
    }

    // Solver::step (Solver.h:103-113): accelerations, then v += a dt and x += v dt.
    // step(n) runs n steps on the device and copies the bodies back once. Status callbacks see
    // "Starting step" and "Finished step"; the compute-time callback gets the call's wall time
    // (host copies included), as the reference's on_step reports it (Solver.h:155-185).
    void step(int n = 1) {
        status("Starting step");
        const auto t0 = std::chrono::steady_clock::now();
        upload();
        check(nb_step(_ctx, n));
        download();
        const std::chrono::duration<double> took = std::chrono::steady_clock::now() - t0;
        status("Finished step");
        if (_on_compute_time) _on_compute_time(took);
    }

    // signal_status / signal_computeTime / signal_finished (Solver.h:143-149). Set them before
    // stepping; with stepAsync they run on the stepping thread.
    void onStatus(std::function<void(const std::string &)> f) { _on_status = std::move(f); }
    void onComputeTime(std::function<void(std::chrono::duration<double>)> f) { _on_compute_time = std::move(f); }
    void onFinished(std::function<void()> f) { _on_finished = std::move(f); }

    // slot_step / on_step (Solver.h:151-185): one step on a background thread. A call while a step
    // is still running is ignored (returns false), as the reference ignores a second spawn.
    // wait() joins the thread and rethrows an error the step raised. Do not touch the simulation
    // while a step runs.
    bool stepAsync() {
        std::lock_guard<std::mutex> lock(_thread_mutex);
        if (_thread.joinable()) {
            if (_running.load()) return false;
            _thread.join();
        }
        _error = nullptr;
        _running.store(true);
        _thread = std::thread([this] {
            try {
                step(1);
            } catch (...) {
                _error = std::current_exception();
            }
            _running.store(false);
            if (_on_finished) _on_finished();
        });
        return true;
    }
    bool stepping() const { return _running.load(); }
    void wait() {
        std::lock_guard<std::mutex> lock(_thread_mutex);
        if (_thread.joinable()) _thread.join();
        if (_error) {
            std::exception_ptr e = _error;
            _error = nullptr;
            std::rethrow_exception(e);
        }
    }

    InteractionCounts counts() const {
        nb_counts c{};
        check(nb_get_counts(_ctx, &c));
        return {c.particle_particle, c.particle_node, c.node_particle, c.node_node};
    }

    // Forces the next call to copy the simulation's bodies to the device (call after editing them).
    void invalidate() { _uploaded_count = SIZE_MAX; }

    nb_ctx *handle() const { return _ctx; }

protected:
    Solver(Simulation &sim, Gravity &rule, int32_t solver, int32_t order, float theta)
        : _sim(sim), _rule(rule) {
        nb_config c;
        nb_config_default(&c);
        c.solver = solver;
        c.order = order;
        c.theta = theta;
        c.G = rule.g();
        c.epsilon = rule.epsilon();
        int rc = nb_create(&c, &_ctx);
        if (rc != NB_OK) throw Error(rc, "nb_create failed: no usable sm_100 device or invalid configuration");
    }

private:
    template<typename F>
    void update(F &&f) {
        nb_config c = config();
        f(c);
        check(nb_set_config(_ctx, &c));
    }
    nb_config config() const {
        nb_config c{};
        check(nb_get_config(_ctx, &c));
        return c;
    }
    void check(int rc) const {
        if (rc != NB_OK) throw Error(rc, nb_last_error(_ctx));
    }
    // The rule's constants and the bodies go to the device when they changed on the host.
    void upload() {
        nb_config c = config();
        if (c.G != _rule.g() || c.epsilon != _rule.epsilon()) {
            c.G = _rule.g();
            c.epsilon = _rule.epsilon();
            check(nb_set_config(_ctx, &c));
        }
        if (_uploaded_count == _sim.particleCount() && !changed()) return;
        std::vector<float> pm = _sim.packedPositionMass(), v = _sim.packedVelocity();
        check(nb_set_bodies(_ctx, (int64_t) _sim.particleCount(), pm.empty() ? nullptr : pm.data(),
                            v.empty() ? nullptr : v.data()));
        _uploaded_count = _sim.particleCount();
        _shadow_pm = std::move(pm);
        _shadow_v = std::move(v);
    }
    void download() {
        const std::size_t n = _sim.particleCount();
        std::vector<float> pm(4 * n), v(4 * n), a(4 * n);
        check(nb_get_bodies(_ctx, n ? pm.data() : nullptr, n ? v.data() : nullptr));
        check(nb_get_accelerations(_ctx, n ? a.data() : nullptr));
        _sim.unpackPositionMass(pm);
        _sim.unpackVelocity(v);
        _sim.unpackAcceleration(a);
        _shadow_pm = std::move(pm);
        _shadow_v = std::move(v);
    }
    // Host edits since the last transfer (positions, masses or velocities)
    bool changed() const { return _sim.packedPositionMass() != _shadow_pm || _sim.packedVelocity() != _shadow_v; }
    void status(const char *what) {
        if (_on_status) _on_status(what);
    }

    Simulation &_sim;
    Gravity &_rule;
    nb_ctx *_ctx = nullptr;
    std::size_t _uploaded_count = SIZE_MAX;
    std::vector<float> _shadow_pm, _shadow_v;
    std::function<void(const std::string &)> _on_status;
    std::function<void(std::chrono::duration<double>)> _on_compute_time;
    std::function<void()> _on_finished;
    std::thread _thread;
    std::mutex _thread_mutex;
    std::atomic<bool> _running{false};
    std::exception_ptr _error;
    std::size_t _max_threads = std::thread::hardware_concurrency();
};

// LinearBVHSolver (LinearBVHSolver.h:18-31): centre-of-mass summaries, "linear-bvh"
class LinearBVHSolver : public Solver {
public:
    LinearBVHSolver(Simulation &sim, Gravity &rule) : Solver(sim, rule, NB_SOLVER_LINEAR_BVH, 1, 0.3f) {}
};

// MultipoleLinearBVHSolver<Order> (LinearBVHSolver.h:33-44); order 2 runs on the GPU
template<int Order>
class MultipoleLinearBVHSolver : public Solver {
    static_assert(Order == 2, "the device path implements the quadrupole (order 2) linear BVH");

public:
    MultipoleLinearBVHSolver(Simulation &sim, Gravity &rule) : Solver(sim, rule, NB_SOLVER_LINEAR_BVH, Order, 0.3f) {}
};
using QuadrupoleLinearBVHSolver = MultipoleLinearBVHSolver<2>;

// NaiveSolver (NaiveSolver.h:12-53): FP32 direct sum, "naive"
class NaiveSolver : public Solver {
public:
    NaiveSolver(Simulation &sim, Gravity &rule) : Solver(sim, rule, NB_SOLVER_NAIVE, 1, 0.3f) {}
};

// MultipoleImplicitLinearBVHFMMSolver<Order> (ImplicitLinearBVHFMMSolver.h:15-38); order 3 runs on the GPU
template<int Order>
class MultipoleImplicitLinearBVHFMMSolver : public Solver {
    static_assert(Order == 3, "the device dual-tree path implements octupole moments (order 3)");

public:
    // theta defaults to ThetaDescentCriterion's 0.5 (DescentCriterionType.h:53)
    MultipoleImplicitLinearBVHFMMSolver(Simulation &sim, Gravity &rule)
        : Solver(sim, rule, NB_SOLVER_DUAL_LINEAR_BVH, Order, 0.5f) {}
};
using OctupoleImplicitLinearBVHFMMSolver = MultipoleImplicitLinearBVHFMMSolver<3>;

// MultiSolver::select (MultiSolver.h:79-87): a solver by its id.
inline std::unique_ptr<Solver> makeSolver(const std::string &id, Simulation &sim, Gravity &rule) {
    if (id == "linear-bvh") return std::make_unique<LinearBVHSolver>(sim, rule);
    if (id == "linear-bvh-4p") return std::make_unique<QuadrupoleLinearBVHSolver>(sim, rule);
    if (id == "naive") return std::make_unique<NaiveSolver>(sim, rule);
    if (id == "implicit-linear-bvh-fmm-8p") return std::make_unique<OctupoleImplicitLinearBVHFMMSolver>(sim, rule);
    throw Error(NB_ERR_INVALID_ARGUMENT, "unknown solver id: " + id);
}

inline std::vector<std::string> solverIds() {
    return {"linear-bvh", "linear-bvh-4p", "naive", "implicit-linear-bvh-fmm-8p"};
}

// MultiSolver (MultiSolver.h:20-114): the solvers of solverIds() behind one object, one selected
// at a time, so a caller can switch algorithms by id as the reference's application does. The
// reference constructs every solver up front; here a solver (and its device context) is created
// on its first selection and kept, so unused algorithms hold no device memory. The first solver
// (by default "linear-bvh-4p") is selected on construction. An unknown id throws (the reference
// logs an error and keeps its selection, MultiSolver.h:79-87).
class MultiSolver {
public:
    MultiSolver(Simulation &sim, Gravity &rule, const std::string &initial = "linear-bvh-4p")
        : _sim(sim), _rule(rule) {
        select(initial);
    }

    void select(const std::string &id) {
        const auto ids = solverIds();
        for (std::size_t i = 0; i < ids.size(); ++i)
            if (ids[i] == id) return select(i);
        throw Error(NB_ERR_INVALID_ARGUMENT, "unknown solver id: " + id);
    }
    void select(std::size_t index) {
        const auto ids = solverIds();
        if (index >= ids.size()) throw Error(NB_ERR_INVALID_ARGUMENT, "solver index out of range");
        if (_solvers.size() < ids.size()) _solvers.resize(ids.size());
        if (!_solvers[index]) _solvers[index] = makeSolver(ids[index], _sim, _rule);
        // a newly selected solver starts from the simulation's current bodies
        _solvers[index]->invalidate();
        _selected = index;
    }
    std::size_t selected() const { return _selected; }

    Solver &get() { return *_solvers[_selected]; }
    const Solver &get() const { return *_solvers[_selected]; }

    std::string id() const { return get().id(); }
    std::string name() const { return get().name(); }
    void updateAccelerations() { get().updateAccelerations(); }
    void step(int n = 1) { get().step(n); }
    InteractionCounts counts() const { return get().counts(); }

private:
    Simulation &_sim;
    Gravity &_rule;
    std::vector<std::unique_ptr<Solver>> _solvers;
    std::size_t _selected = 0;
};

}  // namespace nbody_b200
