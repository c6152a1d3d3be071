// Oracle (test infrastructure only): the reference's implicit-field dual-tree solver restated,
// MultipoleImplicitLinearBVHFMMSolver<Order> = ImplicitDualTraversalSolver<
//     LinearBVH<MultipoleDualEmptySummary<Order>>, DiagonalOverSeparation, Gravity>.
//
//   ImplicitDualTraversalSolver::updateAccelerations
//                                   src/NBody/Simulation/Solvers/ImplicitDualTraversalSolver.h:42-69
//   Tree::loadBalancedBreak         src/NBody/Simulation/Solvers/Trees/Tree.h:84-107
//   balancedLockstepDualTreeImplicitField
//                                   src/NBody/Simulation/Solvers/Descent/balancedLockstepDualTreeImplicitField.h:14-46
//   partitionByDescentCriterionLockstep, lockstepDualTreeImplicitField
//                                   src/NBody/Simulation/Solvers/Descent/lockstepDualTreeImplicitField.h:21-168
//   passiveTreeImplicitField        src/NBody/Simulation/Solvers/Descent/passiveTreeImplicitField.h:13-78
//   activeTree                      src/NBody/Simulation/Solvers/Descent/activeTree.h:24-79
//   DiagonalOverSeparation          src/NBody/Simulation/Solvers/Descent/DescentCriterion/DiagonalOverSeparation.h:17-49
//   separation                      src/NBody/Physics/BoundingBox.h:84-94 (std::pow(float, int) is a double pow)
// The local field has order Order + 1 (MultipoleDualEmptySummary, EmptySummary.h:38-49).
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <functional>
#include <queue>
#include <vector>

#include "physics.h"

namespace oracle::dual {

struct Box {
    vec3 mn, mx;
};

// glm::max(v, 0.0f) per component
inline vec3 max0(vec3 a) { return {(a.x < 0.f) ? 0.f : a.x, (a.y < 0.f) ? 0.f : a.y, (a.z < 0.f) ? 0.f : a.z}; }
inline float length(vec3 a) { return std::sqrt(dot(a, a)); }
inline float diagonal_length(const Box &b) { return length(b.mx - b.mn); }
inline vec3 center(const Box &b) { return (b.mx + b.mn) / 2.0f; }

// separation(box, point) and separation(box, box), BoundingBox.h:84-94
inline float separation(const Box &b, vec3 p) {
    vec3 u = max0(b.mn - p), v = max0(p - b.mx);
    return (float) std::sqrt(std::pow((double) length(u), 2) + std::pow((double) length(v), 2));
}
inline float separation(const Box &b1, const Box &b2) {
    vec3 u = max0(b1.mn - b2.mx), v = max0(b2.mn - b1.mx);
    return (float) std::sqrt(std::pow((double) length(u), 2) + std::pow((double) length(v), 2));
}

enum Recommendation : int { Approximate = 0, DescendActive = 1, DescendPassive = 2 };

struct Criterion {
    float theta;
    // (activeNode, point): approximate the active node for a point
    bool active_point(const Box &b, int64_t size, vec3 p) const {
        return (diagonal_length(b) / separation(b, p)) < theta && size > 32;
    }
    // (point, passiveNode): an active point is far from a passive node
    bool point_passive(vec3 p, const Box &b) const { return (3 * diagonal_length(b) / separation(b, p)) < theta; }
    int node_node(const Box &a, int64_t asize, const Box &p) const {
        float ad = diagonal_length(a), pd = diagonal_length(p);
        if ((ad + pd) / separation(a, p) < theta && asize > 32) return Approximate;
        int r = 0;
        if (ad <= pd * 2.0f) r |= DescendPassive;
        if (pd <= ad * 2.0f) r |= DescendActive;
        return r;
    }
};

template<int Order>
struct Node {
    int32_t begin, end, left, right;
    Box box;
    vec3 com;
    float mass;
    Multipole<Order> mp;
    bool leaf() const { return left < 0; }
    int64_t size() const { return end - begin; }
};

template<int Order>
struct DualSolver {
    using Field = FieldExpansion<Order + 1>;
    const std::vector<Node<Order>> &nodes;
    const float *pm;  // sorted bodies, 4 floats each
    float *acc;       // sorted-order accelerations, 4 floats each
    Gravity g;
    Criterion crit;
    uint64_t *counts;  // optional per-thread counters: pp, np, pn, nn

    vec3 pos(int32_t i) const { return {pm[4 * i], pm[4 * i + 1], pm[4 * i + 2]}; }
    float mass(int32_t i) const { return pm[4 * i + 3]; }
    void add(int32_t i, vec3 a) {
        acc[4 * i] = acc[4 * i] + a.x;
        acc[4 * i + 1] = acc[4 * i + 1] + a.y;
        acc[4 * i + 2] = acc[4 * i + 2] + a.z;
    }

    // activeTree under the point form of DiagonalOverSeparation (activeTree.h:24-79)
    vec3 active_tree(int32_t k, vec3 p) {
        const Node<Order> &n = nodes[k];
        if (n.end == n.begin) return {};
        if (crit.active_point(n.box, n.size(), p)) {
            if (counts) counts[1]++;
            if constexpr (Order == 1) return g.node_particle_mono(n.com, n.mass, p);
            else return g.node_particle<Order>(n.com, n.mass, n.mp, p);
        }
        if (n.leaf()) {
            vec3 a{};
            for (int32_t i = n.begin; i < n.end; ++i) a += g.particle_particle(pos(i), mass(i), p);
            if (counts) counts[0] += (uint64_t) n.size();
            return a;
        }
        vec3 a{};
        a = a + active_tree(n.left, p);
        a = a + active_tree(n.right, p);
        return a;
    }

    // passiveTreeImplicitField (passiveTreeImplicitField.h:13-78); `active` is rearranged in place.
    void passive_tree(int32_t *first, int32_t *last, int32_t k, Field field) {
        const Node<Order> &n = nodes[k];
        if (n.end == n.begin) return;
        vec3 c = center(n.box);
        int32_t *middle = std::partition(first, last, [&](int32_t e) { return crit.point_passive(pos(e), n.box); });
        for (int32_t *e = first; e != middle; ++e) {
            g.particle_node<Order + 1>(pos(*e), mass(*e), c, field);
            if (counts) counts[2]++;
        }
        if (n.leaf()) {
            for (int32_t i = n.begin; i < n.end; ++i) {
                vec3 p = pos(i);
                vec3 a{acc[4 * i], acc[4 * i + 1], acc[4 * i + 2]};
                for (int32_t *e = middle; e != last; ++e) a += g.particle_particle(pos(*e), mass(*e), p);
                if (counts) counts[0] += (uint64_t) (last - middle);
                a += field.at(p - c);
                acc[4 * i] = a.x; acc[4 * i + 1] = a.y; acc[4 * i + 2] = a.z;
            }
        } else {
            for (int32_t ch: {n.left, n.right})
                passive_tree(middle, last, ch, field.translated(center(nodes[ch].box) - c));
        }
    }

    // lockstepDualTreeImplicitField (lockstepDualTreeImplicitField.h:60-168). The active list is a
    // span the callee partitions in place: both passive children of a node see the same vector,
    // the second one in the order the first one left it, as in the reference.
    void lockstep(int32_t *first, int32_t *last, int32_t pk, Field field) {
        const Node<Order> &P = nodes[pk];
        if (P.end == P.begin) return;
        vec3 pc = center(P.box);
        if (first == last) {
            for (int32_t i = P.begin; i < P.end; ++i) add(i, field.at(pos(i) - pc));
            return;
        }
        // partitionByDescentCriterionLockstep (L21-58): far first, non-leaves last, leaves between
        int32_t *endFar = first;
        int32_t *beginNonLeaf = last;
        for (int32_t *i = first; i < beginNonLeaf; ++i) {
            const Node<Order> &A = nodes[*i];
            int rec = crit.node_node(A.box, A.size(), P.box);
            if (rec == Approximate) {
                std::iter_swap(i, endFar);
                ++endFar;
            } else if (!A.leaf()) {
                --beginNonLeaf;
                std::iter_swap(i, beginNonLeaf);
                i--;
            }
        }
        for (int32_t *i = first; i != endFar; ++i) {
            const Node<Order> &A = nodes[*i];
            if constexpr (Order >= 2) g.node_node<Order, Order + 1>(A.com, A.mass, A.mp, pc, field);
            if (counts) counts[3]++;
        }
        if (P.leaf()) {
            for (int32_t *i = endFar; i != beginNonLeaf; ++i)
                for (int32_t b = P.begin; b < P.end; ++b) add(b, active_tree(*i, pos(b)));
            for (int32_t b = P.begin; b < P.end; ++b) {
                for (int32_t *i = beginNonLeaf; i != last; ++i) add(b, active_tree(*i, pos(b)));
                add(b, field.at(pos(b) - pc));
            }
        } else {
            std::vector<int32_t> leafBodies;
            for (int32_t *i = endFar; i != beginNonLeaf; ++i)
                for (int32_t b = nodes[*i].begin; b < nodes[*i].end; ++b) leafBodies.push_back(b);
            passive_tree(leafBodies.data(), leafBodies.data() + leafBodies.size(), pk, Field{});
            std::vector<int32_t> deeper;
            for (int32_t *i = beginNonLeaf; i != last; ++i) {
                deeper.push_back(nodes[*i].left);
                deeper.push_back(nodes[*i].right);
            }
            for (int32_t ch: {P.left, P.right})
                lockstep(deeper.data(), deeper.data() + deeper.size(), ch,
                         field.translated(center(nodes[ch].box) - pc));
        }
    }

    // balancedLockstepDualTreeImplicitField (balancedLockstepDualTreeImplicitField.h:14-46)
    void balanced(int32_t passive_root) {
        std::queue<int32_t> q;
        q.push(0);
        std::vector<int32_t> equal;
        while (!q.empty()) {
            int32_t a = q.front();
            const Node<Order> &A = nodes[a];
            int rec = crit.node_node(A.box, A.size(), nodes[passive_root].box);
            q.pop();
            if (rec != DescendActive || A.leaf()) equal.push_back(a);
            else {
                q.push(A.left);
                q.push(A.right);
            }
        }
        lockstep(equal.data(), equal.data() + equal.size(), passive_root, Field{});
    }
};

// Tree::loadBalancedBreak (Tree.h:84-107): split the largest node until n starting nodes exist
// or the largest is a leaf.
template<int Order>
std::vector<int32_t> load_balanced_break(const std::vector<Node<Order>> &nodes, size_t n) {
    std::vector<int32_t> q{0};
    auto cmp = [&](int32_t a, int32_t b) { return nodes[a].size() < nodes[b].size(); };
    while (q.size() < n) {
        std::pop_heap(q.begin(), q.end(), cmp);
        int32_t k = q.back();
        if (nodes[k].leaf()) break;
        q.pop_back();
        for (int32_t c: {nodes[k].left, nodes[k].right}) {
            q.push_back(c);
            std::push_heap(q.begin(), q.end(), cmp);
        }
    }
    return q;
}

}  // namespace oracle::dual
