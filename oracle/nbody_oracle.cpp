// Oracle (test infrastructure only; never linked into the product library).
//
// CPU restatement of the reference's Barnes-Hut force path on a linear BVH, in FP32 with the
// reference's operation order, built with -ffp-contract=off so that every float operation is
// a single IEEE-rounded operation like the reference's default (no -march, no FMA) build.
// Callers: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
//
// Restated pieces and their sources (paths inside the reference project):
//   outerBoundingBox               src/NBody/Physics/Summaries/SummaryType.h:73-81
//   expandBits21 / toMortonCode    src/NBody/Simulation/Solvers/MortonSort.h:35-60
//   setMortonCodes                 MortonSort.h:63-73
//   Morton sort                    MortonSort.h:75-88, 141-183 (ties ordered by input index)
//   LinearBVHNode::split / build   src/NBody/Simulation/Solvers/Trees/LinearBVH.h:47-76, 106-133
//   NodeBase::refine / summarize   src/NBody/Simulation/Solvers/Trees/NodeBase.h:43-75
//   CenterOfMassSummary            src/NBody/Physics/Summaries/CenterOfMassSummary.h:30-55
//   BoundingBoxSummary             src/NBody/Physics/Summaries/BoundingBoxSummary.h:30-68
//   MultipoleMassSummary           src/NBody/Physics/Summaries/MultipoleMassSummary.h:37-97
//   DiagonalOverCenterDistance     src/NBody/Simulation/Solvers/Descent/DescentCriterion/DiagonalOverCenterDistance.h:18-22
//   Descent::activeTree            src/NBody/Simulation/Solvers/Descent/activeTree.h:24-79
//   ActiveTreeSolver               src/NBody/Simulation/Solvers/ActiveTreeSolver.h:33-72
//   NaiveSolver                    src/NBody/Simulation/Solvers/NaiveSolver.h:22-52
//   Solver::step                   src/NBody/Simulation/Solver.h:103-139
//   SimpleTrackingRule counts      src/NBody/Physics/Rules/SimpleTrackingRule.h:29-51
#include <algorithm>
#include <bit>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include <omp.h>

#include "dualtree.h"
#include "physics.h"

using namespace oracle;

namespace {

inline vec3 load3(const float *pm, int64_t i) { return {pm[4 * i + 0], pm[4 * i + 1], pm[4 * i + 2]}; }

// glm::min / glm::max per component: min(x, y) = (y < x) ? y : x, max(x, y) = (x < y) ? y : x.
inline float gmin(float x, float y) { return (y < x) ? y : x; }
inline float gmax(float x, float y) { return (x < y) ? y : x; }

uint64_t expand_bits21(uint64_t i) {
    i &= 0x1fffff;
    i = (i | i << 32) & 0x1f00000000ffffULL;
    i = (i | i << 16) & 0x1f0000ff0000ffULL;
    i = (i | i << 8) & 0x100f00f00f00f00fULL;
    i = (i | i << 4) & 0x10c30c30c30c30c3ULL;
    i = (i | i << 2) & 0x1249249249249249ULL;
    return i;
}

// toMortonCode for 64-bit codes: clamp(v * 2^21, 0, 2^21 - 1), truncate, interleave x*4 + y*2 + z.
// A NaN coordinate (zero scale, when every position is equal) maps to 0 here; the reference's
// float->uint64 conversion of NaN is undefined, and such a tree is a single leaf either way.
uint64_t morton_code(vec3 v) {
    float c[3] = {v.x * 2097152.f, v.y * 2097152.f, v.z * 2097152.f};
    uint64_t u[3];
    for (int k = 0; k < 3; ++k) {
        float t = gmin(gmax(c[k], 0.f), 2097151.f);
        u[k] = (t == t) ? (uint64_t) t : 0;
    }
    return expand_bits21(u[0]) * 4u + expand_bits21(u[1]) * 2u + expand_bits21(u[2]);
}

struct Tree {
    std::vector<int32_t> begin, end, left, right;  // preorder; left/right = -1 for leaves
};

// Top-down build with the reference's split rule: a node splits while it holds more than
// maxLeafSize bodies and its first and last codes differ; the split point is the first body
// whose code has the most significant differing bit set (std::upper_bound, LinearBVH.h:59-65).
int32_t build_node(Tree &t, const uint64_t *codes, int32_t b, int32_t e, int leaf) {
    int32_t id = (int32_t) t.begin.size();
    t.begin.push_back(b);
    t.end.push_back(e);
    t.left.push_back(-1);
    t.right.push_back(-1);
    if ((e - b) > leaf && codes[b] != codes[e - 1]) {
        int msb = 63 - std::countl_zero(codes[b] ^ codes[e - 1]);
        uint64_t boundary = uint64_t(1) << msb;
        const uint64_t *s = std::upper_bound(codes + b, codes + e, boundary,
                                             [](uint64_t v, uint64_t c) { return (v & c) != 0; });
        int32_t split = (int32_t) (s - codes);
        int32_t l = build_node(t, codes, b, split, leaf);
        int32_t r = build_node(t, codes, split, e, leaf);
        t.left[id] = l;
        t.right[id] = r;
    }
    return id;
}

template<int Order>
struct Summary {
    vec3 bmin{FLT_MAX, FLT_MAX, FLT_MAX};
    vec3 bmax{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    vec3 com{};
    float mass = 0.f;
    Multipole<Order> mp;
};

// Leaf summary over bodies [b, e) of the sorted arrays (CenterOfMassSummary.h:30-42,
// MultipoleMassSummary.h:37-52 with libstdc++'s 4-way std::transform_reduce, BoundingBoxSummary.h:30-57).
template<int Order>
void summarize_leaf(Summary<Order> &s, const float *pm, int32_t b, int32_t e) {
    s.mass = 0.0f;
    s.com = {0.0f, 0.0f, 0.0f};
    for (int32_t i = b; i < e; ++i) {
        float m = pm[4 * i + 3];
        s.mass += m;
        s.com = s.com + (m * load3(pm, i));
    }
    s.com = s.com / s.mass;
    if constexpr (Order >= 2) {
        auto f = [&](int32_t i) {
            vec3 off = load3(pm, i) - s.com;
            return moment_of_offset<Order>(off) * pm[4 * i + 3];
        };
        Multipole<Order> init{};
        int32_t i = b;
        for (; e - i >= 4; i += 4) {
            Multipole<Order> v1 = f(i) + f(i + 1);
            Multipole<Order> v2 = f(i + 2) + f(i + 3);
            Multipole<Order> v3 = v1 + v2;
            init = init + v3;
        }
        for (; i < e; ++i) init = init + f(i);
        s.mp = init;
    }
    s.bmin = {FLT_MAX, FLT_MAX, FLT_MAX};
    s.bmax = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int32_t i = b; i < e; ++i) {
        vec3 p = load3(pm, i);
        s.bmin = {gmin(p.x, s.bmin.x), gmin(p.y, s.bmin.y), gmin(p.z, s.bmin.z)};
        s.bmax = {gmax(p.x, s.bmax.x), gmax(p.y, s.bmax.y), gmax(p.z, s.bmax.z)};
    }
}

// Internal summary from children 0 then 1 (CenterOfMassSummary.h:44-55, MultipoleMassSummary.h:54-97,
// BoundingBoxSummary.h:59-68). Two children go through transform_reduce's sequential tail.
template<int Order>
void summarize_internal(Summary<Order> &s, const Summary<Order> &c0, const Summary<Order> &c1) {
    const Summary<Order> *cs[2] = {&c0, &c1};
    s.mass = 0.0f;
    s.com = {0.0f, 0.0f, 0.0f};
    for (auto *c: cs) {
        s.mass += c->mass;
        s.com = s.com + (c->com * c->mass);
    }
    s.com = s.com / s.mass;
    if constexpr (Order >= 2) {
        Multipole<Order> init{};
        for (auto *c: cs) {
            vec3 off = c->com - s.com;
            Multipole<Order> m = (moment_of_offset<Order>(off) * c->mass) + c->mp;
            if constexpr (Order >= 3) m.t3 += sum_of_outer_products<3>(c->mp.t2, off);
            if constexpr (Order >= 4) {
                m.t4 += sum_of_outer_products<4>(c->mp.t3, off);
                m.t4 += sum_of_outer_products<4>(outer_product<3>(c->mp.t2, off), off);
            }
            init = init + m;
        }
        s.mp = init;
    }
    s.bmin = {FLT_MAX, FLT_MAX, FLT_MAX};
    s.bmax = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (auto *c: cs) {
        s.bmin = {gmin(c->bmin.x, s.bmin.x), gmin(c->bmin.y, s.bmin.y), gmin(c->bmin.z, s.bmin.z)};
        s.bmax = {gmax(c->bmax.x, s.bmax.x), gmax(c->bmax.y, s.bmax.y), gmax(c->bmax.z, s.bmax.z)};
    }
}

template<int Order>
std::vector<Summary<Order>> summarize_tree(const Tree &t, const float *pm_sorted) {
    int64_t nn = (int64_t) t.begin.size();
    std::vector<Summary<Order>> s(nn);
    // Preorder puts every child after its parent, so a reverse sweep is a valid post-order.
    for (int64_t k = nn - 1; k >= 0; --k) {
        if (t.left[k] < 0) summarize_leaf<Order>(s[k], pm_sorted, t.begin[k], t.end[k]);
        else summarize_internal<Order>(s[k], s[t.left[k]], s[t.right[k]]);
    }
    return s;
}

struct Counts {
    uint64_t pp = 0, np = 0;
};

// DiagonalOverCenterDistance(node, p): diag^2 / |centre - p|^2 < theta^2
template<int Order>
inline bool mac_diag_over_center(const Summary<Order> &s, vec3 p, float theta) {
    vec3 center = (s.bmax + s.bmin) / 2.0f;
    float distance2 = length2(p - center);
    float diag2 = length2(s.bmax - s.bmin);
    return (diag2 / distance2) < (theta * theta);
}

template<int Order>
vec3 active_tree(const Tree &t, const std::vector<Summary<Order>> &s, const float *pm_sorted, int32_t k,
                 vec3 p, float theta, const Gravity &g, Counts &cnt) {
    if (t.end[k] == t.begin[k]) return {};
    const Summary<Order> &sk = s[k];
    if (mac_diag_over_center<Order>(sk, p, theta)) {
        cnt.np++;
        if constexpr (Order == 1) return g.node_particle_mono(sk.com, sk.mass, p);
        else return g.node_particle<Order>(sk.com, sk.mass, sk.mp, p);
    }
    if (t.left[k] < 0) {
        vec3 a{};
        for (int32_t i = t.begin[k]; i < t.end[k]; ++i) a += g.particle_particle(load3(pm_sorted, i), pm_sorted[4 * i + 3], p);
        cnt.pp += (uint64_t) (t.end[k] - t.begin[k]);
        return a;
    }
    vec3 a{};
    a = a + active_tree<Order>(t, s, pm_sorted, t.left[k], p, theta, g, cnt);
    a = a + active_tree<Order>(t, s, pm_sorted, t.right[k], p, theta, g, cnt);
    return a;
}

template<int Order>
void bh_all(const Tree &t, const float *pm_sorted, int64_t nt, const float *targets, float G, float eps,
            float theta, float *acc, uint64_t *counts, int threads) {
    std::vector<Summary<Order>> s = summarize_tree<Order>(t, pm_sorted);
    Gravity g{G, eps};
    uint64_t pp = 0, np = 0;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : pp, np)
    for (int64_t i = 0; i < nt; ++i) {
        Counts c;
        vec3 p = load3(targets, i);
        vec3 a = t.begin.empty() ? vec3{} : active_tree<Order>(t, s, pm_sorted, 0, p, theta, g, c);
        acc[4 * i + 0] = a.x;
        acc[4 * i + 1] = a.y;
        acc[4 * i + 2] = a.z;
        acc[4 * i + 3] = 0.f;
        pp += c.pp;
        np += c.np;
    }
    if (counts) {
        counts[0] = pp;
        counts[1] = np;
    }
}

void sort_codes(int64_t n, const uint64_t *codes, uint32_t *perm) {
    std::vector<std::pair<uint64_t, uint32_t>> kv((size_t) n);
    for (int64_t i = 0; i < n; ++i) kv[i] = {codes[i], (uint32_t) i};
    std::sort(kv.begin(), kv.end());
    for (int64_t i = 0; i < n; ++i) perm[i] = kv[i].second;
}

}  // namespace

extern "C" {

// outerBoundingBox over all bodies: out = {min.x, min.y, min.z, max.x, max.y, max.z}
void or_bbox(int64_t n, const float *pm, float *out) {
    vec3 mn{FLT_MAX, FLT_MAX, FLT_MAX}, mx{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; ++i) {
        vec3 p = load3(pm, i);
        mn = {gmin(mn.x, p.x), gmin(mn.y, p.y), gmin(mn.z, p.z)};
        mx = {gmax(mx.x, p.x), gmax(mx.y, p.y), gmax(mx.z, p.z)};
    }
    out[0] = mn.x; out[1] = mn.y; out[2] = mn.z;
    out[3] = mx.x; out[4] = mx.y; out[5] = mx.z;
}

// setMortonCodes: code_i = toMortonCode((p_i - bbox.min) / maxSideLength)
void or_morton(int64_t n, const float *pm, const float *bbox, uint64_t *codes) {
    vec3 mn{bbox[0], bbox[1], bbox[2]}, mx{bbox[3], bbox[4], bbox[5]};
    vec3 dims = mx - mn;
    float scale = std::max(std::max(dims.x, dims.y), dims.z);
    for (int64_t i = 0; i < n; ++i) codes[i] = morton_code((load3(pm, i) - mn) / scale);
}

// Morton sort, ties broken by input index: perm[k] = input index of the k-th smallest code.
void or_sort(int64_t n, const uint64_t *codes, uint32_t *perm) { sort_codes(n, codes, perm); }

// LinearBVH topology in preorder over sorted codes. Output arrays must hold 2n entries.
// Returns the node count (0 for n == 0).
int64_t or_build(int64_t n, const uint64_t *sorted_codes, int32_t leaf, int32_t *begin, int32_t *end,
                 int32_t *left, int32_t *right) {
    if (n <= 0) return 0;
    Tree t;
    t.begin.reserve(2 * n);
    build_node(t, sorted_codes, 0, (int32_t) n, leaf);
    int64_t nn = (int64_t) t.begin.size();
    std::memcpy(begin, t.begin.data(), nn * 4);
    std::memcpy(end, t.end.data(), nn * 4);
    std::memcpy(left, t.left.data(), nn * 4);
    std::memcpy(right, t.right.data(), nn * 4);
    return nn;
}

// Node summaries of a preorder tree over the sorted bodies. Per node: bbox[6] = min, max;
// com_m[4] = centre of mass, total mass; moments[31] = unique tensor values of orders 2, 3, 4
// (6 + 10 + 15) in the reference's packed layout, zero above `order`.
int or_summarize(int64_t nn, const int32_t *begin, const int32_t *end, const int32_t *left, const int32_t *right,
                 const float *pm_sorted, int32_t order, float *bbox, float *com_m, float *moments) {
    Tree t;
    t.begin.assign(begin, begin + nn);
    t.end.assign(end, end + nn);
    t.left.assign(left, left + nn);
    t.right.assign(right, right + nn);
    auto emit = [&](auto &s) {
        for (int64_t k = 0; k < nn; ++k) {
            const auto &sk = s[k];
            float *b = bbox + 6 * k;
            b[0] = sk.bmin.x; b[1] = sk.bmin.y; b[2] = sk.bmin.z;
            b[3] = sk.bmax.x; b[4] = sk.bmax.y; b[5] = sk.bmax.z;
            float *c = com_m + 4 * k;
            c[0] = sk.com.x; c[1] = sk.com.y; c[2] = sk.com.z; c[3] = sk.mass;
            float *m = moments + 31 * k;
            std::fill(m, m + 31, 0.f);
            for (int i = 0; i < 6; ++i) m[i] = sk.mp.t2.v[i];
            for (int i = 0; i < 10; ++i) m[6 + i] = sk.mp.t3.v[i];
            for (int i = 0; i < 15; ++i) m[16 + i] = sk.mp.t4.v[i];
        }
    };
    switch (order) {
        case 1: { auto s = summarize_tree<1>(t, pm_sorted); emit(s); return 0; }
        case 2: { auto s = summarize_tree<2>(t, pm_sorted); emit(s); return 0; }
        case 3: { auto s = summarize_tree<3>(t, pm_sorted); emit(s); return 0; }
        case 4: { auto s = summarize_tree<4>(t, pm_sorted); emit(s); return 0; }
        default: return -1;
    }
}

// ActiveTreeSolver<LinearBVH, DiagonalOverCenterDistance, Gravity>::updateAccelerations for every
// body (all bodies are both active and passive). Inputs and outputs are in input order, 4 floats
// per body. counts = {particle-particle, node-particle} calls. Returns the tree's node count.
int64_t or_bh_accelerations(int64_t n, const float *pm, float G, float eps, float theta, int32_t leaf,
                            int32_t order, float *acc, uint64_t *counts, int32_t threads) {
    if (n <= 0) {
        if (counts) counts[0] = counts[1] = 0;
        return 0;
    }
    float bbox[6];
    or_bbox(n, pm, bbox);
    std::vector<uint64_t> codes((size_t) n), sorted((size_t) n);
    std::vector<uint32_t> perm((size_t) n);
    or_morton(n, pm, bbox, codes.data());
    sort_codes(n, codes.data(), perm.data());
    std::vector<float> pms((size_t) n * 4);
    for (int64_t k = 0; k < n; ++k) {
        sorted[k] = codes[perm[k]];
        std::memcpy(&pms[4 * k], pm + 4 * (int64_t) perm[k], 16);
    }
    Tree t;
    t.begin.reserve(2 * n);
    build_node(t, sorted.data(), 0, (int32_t) n, leaf);
    switch (order) {
        case 1: bh_all<1>(t, pms.data(), n, pm, G, eps, theta, acc, counts, threads); break;
        case 2: bh_all<2>(t, pms.data(), n, pm, G, eps, theta, acc, counts, threads); break;
        case 3: bh_all<3>(t, pms.data(), n, pm, G, eps, theta, acc, counts, threads); break;
        case 4: bh_all<4>(t, pms.data(), n, pm, G, eps, theta, acc, counts, threads); break;
        default: return -1;
    }
    return (int64_t) t.begin.size();
}

// Same traversal for an arbitrary list of target positions (4 floats each) against the tree
// of `pm`; used to time a bounded sample of targets.
int64_t or_bh_targets(int64_t n, const float *pm, int64_t nt, const float *targets, float G, float eps,
                      float theta, int32_t leaf, int32_t order, float *acc, uint64_t *counts, int32_t threads) {
    if (n <= 0) return 0;
    float bbox[6];
    or_bbox(n, pm, bbox);
    std::vector<uint64_t> codes((size_t) n), sorted((size_t) n);
    std::vector<uint32_t> perm((size_t) n);
    or_morton(n, pm, bbox, codes.data());
    sort_codes(n, codes.data(), perm.data());
    std::vector<float> pms((size_t) n * 4);
    for (int64_t k = 0; k < n; ++k) {
        sorted[k] = codes[perm[k]];
        std::memcpy(&pms[4 * k], pm + 4 * (int64_t) perm[k], 16);
    }
    Tree t;
    t.begin.reserve(2 * n);
    build_node(t, sorted.data(), 0, (int32_t) n, leaf);
    switch (order) {
        case 1: bh_all<1>(t, pms.data(), nt, targets, G, eps, theta, acc, counts, threads); break;
        case 2: bh_all<2>(t, pms.data(), nt, targets, G, eps, theta, acc, counts, threads); break;
        case 3: bh_all<3>(t, pms.data(), nt, targets, G, eps, theta, acc, counts, threads); break;
        case 4: bh_all<4>(t, pms.data(), nt, targets, G, eps, theta, acc, counts, threads); break;
        default: return -1;
    }
    return (int64_t) t.begin.size();
}

// NaiveSolver: FP32 direct sum in body order for the listed targets (idx == NULL: all bodies).
void or_direct_f32(int64_t n, const float *pm, int64_t nt, const int64_t *idx, float G, float eps, float *acc,
                   int32_t threads) {
    Gravity g{G, eps};
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nt; ++t) {
        int64_t i = idx ? idx[t] : t;
        vec3 p = load3(pm, i);
        vec3 a{};
        for (int64_t j = 0; j < n; ++j) a += g.particle_particle(load3(pm, j), pm[4 * j + 3], p);
        acc[4 * t + 0] = a.x; acc[4 * t + 1] = a.y; acc[4 * t + 2] = a.z; acc[4 * t + 3] = 0.f;
    }
}

// FP64 direct sum (accuracy reference): a_i = G sum_j m_j (x_j - x_i) / (|x_j - x_i|^2 + eps)^(3/2),
// pairs at identical positions skipped as in Gravity.h:203.
void or_direct_f64(int64_t n, const float *pm, int64_t nt, const int64_t *idx, double G, double eps, double *acc,
                   int32_t threads) {
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nt; ++t) {
        int64_t i = idx ? idx[t] : t;
        double px = pm[4 * i], py = pm[4 * i + 1], pz = pm[4 * i + 2];
        double ax = 0, ay = 0, az = 0;
        for (int64_t j = 0; j < n; ++j) {
            double dx = (double) pm[4 * j] - px, dy = (double) pm[4 * j + 1] - py, dz = (double) pm[4 * j + 2] - pz;
            if (dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
            double r2 = dx * dx + dy * dy + dz * dz + eps;
            double s = (double) pm[4 * j + 3] / (r2 * std::sqrt(r2));
            ax += dx * s; ay += dy * s; az += dz * s;
        }
        acc[3 * t + 0] = G * ax; acc[3 * t + 1] = G * ay; acc[3 * t + 2] = G * az;
    }
}

// Solver::updateVelocities then updatePositions: v = v + a*dt; p = p + v*dt (Solver.h:117-139).
void or_kick_drift(int64_t n, float *pm, float *vel, const float *acc, float dt) {
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) vel[4 * i + k] = vel[4 * i + k] + (acc[4 * i + k] * dt);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) pm[4 * i + k] = pm[4 * i + k] + (vel[4 * i + k] * dt);
}


// ---- Rule-level entry points (for the reference's own known-answer tests) ----

// Gravity::particleParticle; out = 3 floats.
void or_particle_particle(float G, float eps, const float *active, float m, const float *passive, float *out) {
    Gravity g{G, eps};
    vec3 a = g.particle_particle({active[0], active[1], active[2]}, m, {passive[0], passive[1], passive[2]});
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
}

// Leaf summary of bodies (4 floats each) at the given order; outputs as or_summarize.
int or_leaf_summary(int64_t n, const float *pm, int32_t order, float *bbox, float *com_m, float *moments) {
    int32_t b = 0, e = (int32_t) n, l = -1;
    return or_summarize(1, &b, &e, &l, &l, pm, order, bbox, com_m, moments);
}

// Gravity::nodeParticle for a summary (order 1: centre of mass only); moments as or_summarize.
int or_node_particle(int32_t order, float G, float eps, const float *com_m, const float *moments, const float *passive,
                     float *out) {
    Gravity g{G, eps};
    vec3 c{com_m[0], com_m[1], com_m[2]}, p{passive[0], passive[1], passive[2]};
    float M = com_m[3];
    auto load = [&](auto &mp) {
        for (int i = 0; i < 6; ++i) mp.t2.v[i] = moments[i];
        for (int i = 0; i < 10; ++i) mp.t3.v[i] = moments[6 + i];
        for (int i = 0; i < 15; ++i) mp.t4.v[i] = moments[16 + i];
    };
    vec3 a;
    switch (order) {
        case 1: a = g.node_particle_mono(c, M, p); break;
        case 2: { Multipole<2> mp; load(mp); a = g.node_particle<2>(c, M, mp, p); break; }
        case 3: { Multipole<3> mp; load(mp); a = g.node_particle<3>(c, M, mp, p); break; }
        case 4: { Multipole<4> mp; load(mp); a = g.node_particle<4>(c, M, mp, p); break; }
        default: return -1;
    }
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
    return 0;
}

}  // extern "C"

namespace {
// Field expansions cross the C boundary as 55 floats: vector(3), t2(6), t3(10), t4(15), t5(21).
template<int Order>
void field_in(FieldExpansion<Order> &f, const float *s) {
    f.vector = {s[0], s[1], s[2]};
    for (int i = 0; i < 6; ++i) f.t2.v[i] = s[3 + i];
    for (int i = 0; i < 10; ++i) f.t3.v[i] = s[9 + i];
    for (int i = 0; i < 15; ++i) f.t4.v[i] = s[19 + i];
    for (int i = 0; i < 21; ++i) f.t5.v[i] = s[34 + i];
}
template<int Order>
void field_out(const FieldExpansion<Order> &f, float *s) {
    s[0] = f.vector.x; s[1] = f.vector.y; s[2] = f.vector.z;
    for (int i = 0; i < 6; ++i) s[3 + i] = f.t2.v[i];
    for (int i = 0; i < 10; ++i) s[9 + i] = f.t3.v[i];
    for (int i = 0; i < 15; ++i) s[19 + i] = f.t4.v[i];
    for (int i = 0; i < 21; ++i) s[34 + i] = f.t5.v[i];
}
template<typename F>
int with_order(int32_t order, F &&f) {
    switch (order) {
        case 2: f(std::integral_constant<int, 2>{}); return 0;
        case 3: f(std::integral_constant<int, 3>{}); return 0;
        case 4: f(std::integral_constant<int, 4>{}); return 0;
        case 5: f(std::integral_constant<int, 5>{}); return 0;
        default: return -1;
    }
}
}  // namespace

extern "C" {

// Gravity::particleNode into a field expansion of the given passive order (accumulates in place).
int or_particle_node(int32_t order, float G, float eps, const float *active, float m, const float *center, float *field) {
    Gravity g{G, eps};
    return with_order(order, [&](auto O) {
        FieldExpansion<O.value> f;
        field_in(f, field);
        g.particle_node<O.value>({active[0], active[1], active[2]}, m, {center[0], center[1], center[2]}, f);
        field_out(f, field);
    });
}

// MultipoleAcceleration::at
int or_field_at(int32_t order, const float *field, const float *off, float *out) {
    return with_order(order, [&](auto O) {
        FieldExpansion<O.value> f;
        field_in(f, field);
        vec3 a = f.at({off[0], off[1], off[2]});
        out[0] = a.x; out[1] = a.y; out[2] = a.z;
    });
}

// MultipoleAcceleration::translated
int or_field_translated(int32_t order, const float *field, const float *off, float *out) {
    return with_order(order, [&](auto O) {
        FieldExpansion<O.value> f;
        field_in(f, field);
        field_out(f.translated({off[0], off[1], off[2]}), out);
    });
}

}  // extern "C"

// ---- symmetric tensor index maps and products (SymmetricTensor3.h), for the index KATs ----
namespace {
template<typename F>
int with_tensor_order(int32_t order, F &&f) {
    switch (order) {
        case 1: f(std::integral_constant<int, 1>{}); return 0;
        case 2: f(std::integral_constant<int, 2>{}); return 0;
        case 3: f(std::integral_constant<int, 3>{}); return 0;
        case 4: f(std::integral_constant<int, 4>{}); return 0;
        case 5: f(std::integral_constant<int, 5>{}); return 0;
        default: return -1;
    }
}
}  // namespace

extern "C" {

int32_t or_tensor_linear_index(int32_t order, const int32_t *dims) {
    int32_t out = -1;
    with_tensor_order(order, [&](auto K) {
        Dims<K.value> d{};
        for (int i = 0; i < K.value; ++i) d[i] = dims[i];
        out = linear_index<K.value>(d);
    });
    return out;
}

int or_tensor_dimensional_index(int32_t order, int32_t L, int32_t *dims) {
    return with_tensor_order(order, [&](auto K) {
        Dims<K.value> d = dimensional_index<K.value>(L);
        for (int i = 0; i < K.value; ++i) dims[i] = d[i];
    });
}

int or_tensor_lexicographic_index(int32_t order, int32_t I, int32_t *dims) {
    return with_tensor_order(order, [&](auto K) {
        Dims<K.value> d = lexicographic_index<K.value>(I);
        for (int i = 0; i < K.value; ++i) dims[i] = d[i];
    });
}

int or_tensor_cartesian_power(int32_t order, const float *v, float *out) {
    if (order < 2) return -1;
    return with_tensor_order(order, [&](auto K) {
        if constexpr (K.value >= 2) {
            ST<K.value> t = cartesian_power<K.value>({v[0], v[1], v[2]});
            for (int i = 0; i < ST<K.value>::U; ++i) out[i] = t.v[i];
        }
    });
}

// T_2 * v (SymmetricTensor3.h:253-260)
void or_tensor2_times_vector(const float *t2, const float *v, float *out) {
    ST<2> t;
    for (int i = 0; i < 6; ++i) t.v[i] = t2[i];
    vec3 r = contract_down(t, {v[0], v[1], v[2]});
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

}  // extern "C"

namespace {
template<int Order>
int64_t dual_accelerations(int64_t n, const float *pm, float G, float eps, float theta, int32_t leaf, float *acc,
                           uint64_t *counts, int32_t threads) {
    float box[6];
    or_bbox(n, pm, box);
    std::vector<uint64_t> codes((size_t) n), sorted((size_t) n);
    std::vector<uint32_t> perm((size_t) n);
    or_morton(n, pm, box, codes.data());
    sort_codes(n, codes.data(), perm.data());
    std::vector<float> pms((size_t) n * 4);
    for (int64_t k = 0; k < n; ++k) {
        sorted[k] = codes[perm[k]];
        std::memcpy(&pms[4 * k], pm + 4 * (int64_t) perm[k], 16);
    }
    Tree t;
    t.begin.reserve(2 * n);
    build_node(t, sorted.data(), 0, (int32_t) n, leaf);
    std::vector<Summary<Order>> s = summarize_tree<Order>(t, pms.data());
    const int64_t nn = (int64_t) t.begin.size();
    std::vector<dual::Node<Order>> nodes((size_t) nn);
    for (int64_t k = 0; k < nn; ++k) {
        auto &d = nodes[k];
        d.begin = t.begin[k]; d.end = t.end[k]; d.left = t.left[k]; d.right = t.right[k];
        d.box = {s[k].bmin, s[k].bmax};
        d.com = s[k].com; d.mass = s[k].mass; d.mp = s[k].mp;
    }
    std::vector<float> accs((size_t) n * 4, 0.f);
    std::vector<int32_t> roots = dual::load_balanced_break<Order>(nodes, 256);
    uint64_t tot[4] = {0, 0, 0, 0};
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        uint64_t local[4] = {0, 0, 0, 0};
        dual::DualSolver<Order> solver{nodes, pms.data(), accs.data(), Gravity{G, eps}, dual::Criterion{theta}, local};
#pragma omp for schedule(dynamic, 1)
        for (int64_t r = 0; r < (int64_t) roots.size(); ++r) solver.balanced(roots[r]);
#pragma omp critical
        for (int k = 0; k < 4; ++k) tot[k] += local[k];
    }
    for (int64_t k = 0; k < n; ++k) std::memcpy(acc + 4 * (int64_t) perm[k], &accs[4 * k], 16);
    if (counts) for (int k = 0; k < 4; ++k) counts[k] = tot[k];
    return nn;
}
}  // namespace

extern "C" {

// MultipoleImplicitLinearBVHFMMSolver<order> accelerations (order 1..3; the local field has order
// order+1), in input order. counts = {particle-particle, node-particle, particle-node, node-node}.
int64_t or_dual_accelerations(int64_t n, const float *pm, float G, float eps, float theta, int32_t leaf, int32_t order,
                              float *acc, uint64_t *counts, int32_t threads) {
    if (n <= 0) return 0;
    switch (order) {
        case 2: return dual_accelerations<2>(n, pm, G, eps, theta, leaf, acc, counts, threads);
        case 3: return dual_accelerations<3>(n, pm, G, eps, theta, leaf, acc, counts, threads);
        default: return -1;
    }
}

int32_t or_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
