// Oracle (test infrastructure only): the Gravity rule, multipole moments and local-field
// expansions of the reference, restated in FP32 with the reference's operation order.
//
//   Gravity::particleParticle        src/NBody/Physics/Rules/Gravity.h:199-209
//   Gravity::nodeParticle (COM)      Gravity.h:213-236
//   Gravity::nodeParticle (multipole) Gravity.h:239-259
//   Gravity::particleNode            Gravity.h:282-306
//   Gravity::nodeNode                Gravity.h:310-403
//   D<1..5>                          Gravity.h:43-180
//   MultipoleMoment::init            src/NBody/Physics/MultipoleMoment.h:46-62
//   MultipoleAcceleration::at        src/NBody/Physics/MultipoleAcceleration.h:33-49
//   MultipoleAcceleration::translated MultipoleAcceleration.h:51-84
#pragma once

#include <cmath>

#include "stensor.h"

namespace oracle {

template<int P>
inline float powi(float v) {
    if constexpr (P == 0) return 1.0f;
    else return v * powi<P - 1>(v);
}

// Multipole<Order>: tensors of order 2..Order (src/NBody/Physics/Multipole.h:34-126).
template<int Order>
struct Multipole {
    ST<2> t2;
    ST<3> t3;
    ST<4> t4;
    Multipole &operator+=(const Multipole &o) {
        if constexpr (Order >= 2) t2 += o.t2;
        if constexpr (Order >= 3) t3 += o.t3;
        if constexpr (Order >= 4) t4 += o.t4;
        return *this;
    }
    Multipole &operator*=(float s) {
        if constexpr (Order >= 2) t2 *= s;
        if constexpr (Order >= 3) t3 *= s;
        if constexpr (Order >= 4) t4 *= s;
        return *this;
    }
    friend Multipole operator+(const Multipole &a, const Multipole &b) { Multipole r = a; r += b; return r; }
    friend Multipole operator*(const Multipole &a, float s) { Multipole r = a; r *= s; return r; }
};

// MultipoleMoment{offset}: repeated outer products of the offset (MultipoleMoment.h:46-62).
template<int Order>
inline Multipole<Order> moment_of_offset(vec3 d) {
    Multipole<Order> m;
    if constexpr (Order >= 2) m.t2 = outer_product<2>(d, d);
    if constexpr (Order >= 3) m.t3 = outer_product<3>(m.t2, d);
    if constexpr (Order >= 4) m.t4 = outer_product<4>(m.t3, d);
    return m;
}

// MultipoleAcceleration<Order>: vector plus field tensors of order 2..Order.
template<int Order>
struct FieldExpansion {
    vec3 vector{};
    ST<2> t2;
    ST<3> t3;
    ST<4> t4;
    ST<5> t5;

    // MultipoleAcceleration::at (MultipoleAcceleration.h:33-49)
    vec3 at(vec3 off) const {
        vec3 a = vector;
        if constexpr (Order >= 2) a += contract_down(t2, off);
        if constexpr (Order >= 3) a += fully_contract<3>(t3, off) / 2.0f;
        if constexpr (Order >= 4) a += fully_contract<4>(t4, off) / 6.0f;
        if constexpr (Order >= 5) a += fully_contract<5>(t5, off) / 24.0f;
        return a;
    }

    // MultipoleAcceleration::translated (MultipoleAcceleration.h:51-84)
    FieldExpansion translated(vec3 off) const {
        FieldExpansion t = *this;
        if constexpr (Order >= 2) {
            vec3 delta = contract_down(t2, off);
            t.vector += delta;
        }
        if constexpr (Order >= 3) {
            ST<2> delta2 = contract_down<3>(t3, off);
            vec3 delta = contract_down(delta2, off);
            t.t2 += delta2;
            t.vector += delta / 2.0f;
        }
        if constexpr (Order >= 4) {
            ST<3> delta3 = contract_down<4>(t4, off);
            ST<2> delta2 = contract_down<3>(delta3, off);
            vec3 delta = contract_down(delta2, off);
            t.t3 += delta3;
            t.t2 += delta2 / 2.0f;
            t.vector += delta / 6.0f;
        }
        if constexpr (Order >= 5) {
            ST<4> delta4 = contract_down<5>(t5, off);
            ST<3> delta3 = contract_down<4>(delta4, off);
            ST<2> delta2 = contract_down<3>(delta3, off);
            vec3 delta = contract_down(delta2, off);
            t.t4 += delta4;
            t.t3 += delta3 / 2.0f;
            t.t2 += delta2 / 6.0f;
            t.vector += delta / 24.0f;
        }
        return t;
    }

    FieldExpansion &operator+=(const FieldExpansion &o) {
        vector += o.vector;
        if constexpr (Order >= 2) t2 += o.t2;
        if constexpr (Order >= 3) t3 += o.t3;
        if constexpr (Order >= 4) t4 += o.t4;
        if constexpr (Order >= 5) t5 += o.t5;
        return *this;
    }
};

// Coefficients f_k = (-1)^k (2k-1)!! / r^(k+1) and g_k = f_k / r^k shared by every D<k>.
struct DerivCoefficients {
    float g1, g2, g3, g4, g5;
    explicit DerivCoefficients(float r) {
        float f1 = -1.0f / powi<2>(r);
        float f2 = 3.0f / powi<3>(r);
        float f3 = -15.0f / powi<4>(r);
        float f4 = 105.0f / powi<5>(r);
        float f5 = -945.0f / powi<6>(r);
        g1 = f1 / r;
        g2 = f2 / powi<2>(r);
        g3 = f3 / powi<3>(r);
        g4 = f4 / powi<4>(r);
        g5 = f5 / powi<5>(r);
    }
};

// Derivative tensors of the softened 1/r (Gravity.h:43-180), term by term.
inline vec3 D1(vec3 R, float r) { DerivCoefficients c(r); return c.g1 * R; }

inline ST<2> D2(vec3 R, float r) {
    DerivCoefficients c(r);
    return (c.g2 * cartesian_power<2>(R)) + (c.g1 * ST<2>::identity());
}

inline ST<3> D3(vec3 R, float r) {
    DerivCoefficients c(r);
    ST<3> A = c.g3 * cartesian_power<3>(R);
    ST<3> B;
    B.at(0, 1, 1) = R.x;
    B.at(0, 2, 2) = R.x;
    B.at(1, 0, 0) = R.y;
    B.at(1, 2, 2) = R.y;
    B.at(2, 0, 0) = R.z;
    B.at(2, 1, 1) = R.z;
    B += 3.0f * ST<3>::diagonal(R);
    B *= c.g2;
    return A + B;
}

inline ST<4> D4(vec3 R, float r) {
    DerivCoefficients c(r);
    ST<4> A = c.g4 * cartesian_power<4>(R);
    ST<4> B;
    B.at(0, 0, 1, 1) = 1;
    B.at(0, 0, 2, 2) = 1;
    B.at(1, 1, 2, 2) = 1;
    B += ST<4>::diagonal({3, 3, 3});
    B *= c.g2;
    ST<4> C;
    ST<2> R2 = cartesian_power<2>(R);
    C += 6.0f * ST<4>::diagonal(R2.diagonal());
    C.at(0, 0, 0, 1) = 3.0f * R2.at(0, 1);
    C.at(0, 1, 1, 1) = 3.0f * R2.at(0, 1);
    C.at(0, 0, 0, 2) = 3.0f * R2.at(0, 2);
    C.at(0, 2, 2, 2) = 3.0f * R2.at(0, 2);
    C.at(1, 1, 1, 2) = 3.0f * R2.at(1, 2);
    C.at(1, 2, 2, 2) = 3.0f * R2.at(1, 2);
    C.at(0, 0, 1, 1) = R2.at(0, 0) + R2.at(1, 1);
    C.at(0, 0, 2, 2) = R2.at(0, 0) + R2.at(2, 2);
    C.at(1, 1, 2, 2) = R2.at(1, 1) + R2.at(2, 2);
    C.at(0, 0, 1, 2) = R2.at(1, 2);
    C.at(0, 1, 1, 2) = R2.at(0, 2);
    C.at(0, 1, 2, 2) = R2.at(0, 1);
    C *= c.g3;
    return A + B + C;
}

inline ST<5> D5(vec3 R, float r) {
    DerivCoefficients c(r);
    ST<3> R3 = cartesian_power<3>(R);
    ST<5> A = c.g5 * cartesian_power<5>(R);
    const float g3 = c.g3, g4 = c.g4;
    ST<5> B;
    B.at(0, 0, 0, 0, 0) += 15 * g3 * R.x;
    B.at(1, 1, 1, 1, 1) += 15 * g3 * R.y;
    B.at(2, 2, 2, 2, 2) += 15 * g3 * R.z;
    B.at(0, 0, 0, 0, 1) += 3 * g3 * R.y;
    B.at(0, 0, 0, 0, 2) += 3 * g3 * R.z;
    B.at(0, 1, 1, 1, 1) += 3 * g3 * R.x;
    B.at(0, 2, 2, 2, 2) += 3 * g3 * R.x;
    B.at(1, 1, 1, 1, 2) += 3 * g3 * R.z;
    B.at(1, 2, 2, 2, 2) += 3 * g3 * R.y;
    B.at(0, 0, 0, 1, 1) += 3 * g3 * R.x;
    B.at(0, 0, 0, 2, 2) += 3 * g3 * R.x;
    B.at(0, 0, 1, 1, 1) += 3 * g3 * R.y;
    B.at(0, 0, 2, 2, 2) += 3 * g3 * R.z;
    B.at(1, 1, 1, 2, 2) += 3 * g3 * R.y;
    B.at(1, 1, 2, 2, 2) += 3 * g3 * R.z;
    B.at(0, 0, 1, 2, 2) += g3 * R.y;
    B.at(0, 0, 1, 1, 2) += g3 * R.z;
    B.at(0, 1, 1, 2, 2) += g3 * R.x;
    B.at(0, 0, 0, 1, 2) += 0;
    B.at(0, 1, 1, 1, 2) += 0;
    B.at(0, 1, 2, 2, 2) += 0;
    ST<5> C;
    C.at(0, 0, 0, 0, 0) += 10 * g4 * R3.at(0, 0, 0);
    C.at(1, 1, 1, 1, 1) += 10 * g4 * R3.at(1, 1, 1);
    C.at(2, 2, 2, 2, 2) += 10 * g4 * R3.at(2, 2, 2);
    C.at(0, 0, 0, 0, 1) += 6 * g4 * R3.at(0, 0, 1);
    C.at(0, 0, 0, 0, 2) += 6 * g4 * R3.at(0, 0, 2);
    C.at(0, 1, 1, 1, 1) += 6 * g4 * R3.at(1, 1, 0);
    C.at(0, 2, 2, 2, 2) += 6 * g4 * R3.at(2, 2, 0);
    C.at(1, 1, 1, 1, 2) += 6 * g4 * R3.at(1, 1, 2);
    C.at(1, 2, 2, 2, 2) += 6 * g4 * R3.at(2, 2, 1);
    C.at(0, 0, 0, 1, 1) += g4 * R3.at(0, 0, 0) + 3 * g4 * R3.at(0, 1, 1);
    C.at(0, 0, 0, 2, 2) += g4 * R3.at(0, 0, 0) + 3 * g4 * R3.at(0, 2, 2);
    C.at(0, 0, 1, 1, 1) += g4 * R3.at(1, 1, 1) + 3 * g4 * R3.at(1, 0, 0);
    C.at(0, 0, 2, 2, 2) += g4 * R3.at(2, 2, 2) + 3 * g4 * R3.at(2, 0, 0);
    C.at(1, 1, 1, 2, 2) += g4 * R3.at(1, 1, 1) + 3 * g4 * R3.at(1, 2, 2);
    C.at(1, 1, 2, 2, 2) += g4 * R3.at(2, 2, 2) + 3 * g4 * R3.at(2, 1, 1);
    C.at(0, 0, 1, 2, 2) += g4 * R3.at(1, 2, 2) + g4 * R3.at(0, 0, 1);
    C.at(0, 0, 1, 1, 2) += g4 * R3.at(1, 1, 2) + g4 * R3.at(0, 0, 2);
    C.at(0, 1, 1, 2, 2) += g4 * R3.at(0, 2, 2) + g4 * R3.at(0, 1, 1);
    C.at(0, 0, 0, 1, 2) += 3 * g4 * R3.at(0, 1, 2);
    C.at(0, 1, 1, 1, 2) += 3 * g4 * R3.at(0, 1, 2);
    C.at(0, 1, 2, 2, 2) += 3 * g4 * R3.at(0, 1, 2);
    return A + B + C;
}

struct Gravity {
    float G = 1.0f;
    float epsilon = 0.00001f;  // added to r^2 (Gravity.h:195, 207)

    // Gravity::particleParticle (Gravity.h:199-209)
    vec3 particle_particle(vec3 active, float m, vec3 passive) const {
        if (active == passive) return {};
        vec3 R = passive - active;
        float r = std::sqrt(length2(R) + epsilon);
        return -R * m * G / powi<3>(r);
    }

    // Gravity::nodeParticle for a CenterOfMassSummary (Gravity.h:227-236)
    vec3 node_particle_mono(vec3 com, float M, vec3 passive) const { return particle_particle(com, M, passive); }

    // Gravity::nodeParticle for a MultipoleMassSummary<Order> (Gravity.h:239-259)
    template<int Order>
    vec3 node_particle(vec3 com, float M, const Multipole<Order> &mp, vec3 passive) const {
        if (com == passive) return {};
        vec3 R = passive - com;
        float r = std::sqrt(length2(R) + epsilon);
        vec3 dPhi = R * -M / powi<3>(r);
        if constexpr (Order >= 2) dPhi += contract_to_vector<3>(D3(R, r), mp.t2) / 2.0f;
        if constexpr (Order >= 3) dPhi -= contract_to_vector<4>(D4(R, r), mp.t3) / 6.0f;
        if constexpr (Order >= 4) dPhi += contract_to_vector<5>(D5(R, r), mp.t4) / 24.0f;
        return G * dPhi;
    }

    // Gravity::particleNode into a MultipoleAccelerationSummary<PassiveOrder> (Gravity.h:282-306)
    template<int PassiveOrder>
    void particle_node(vec3 active, float m, vec3 passive, FieldExpansion<PassiveOrder> &f) const {
        if (active == passive) return;
        vec3 R = passive - active;
        float r = std::sqrt(length2(R) + epsilon);
        f.vector -= (R / powi<3>(r)) * m * G;
        if constexpr (PassiveOrder >= 2) f.t2 += D2(R, r) * m * G;
        if constexpr (PassiveOrder >= 3) f.t3 += D3(R, r) * m * G / 2.0f;
        if constexpr (PassiveOrder >= 4) f.t4 += D4(R, r) * m * G / 6.0f;
        if constexpr (PassiveOrder >= 5) f.t5 += D5(R, r) * m * G / 24.0f;
    }

    // Gravity::nodeNode for MultipoleMassSummary<P-1> -> MultipoleAccelerationSummary<P> (Gravity.h:352-392).
    // Terms beyond passive order 4 are empty in the reference ("todo", L388-391).
    template<int ActiveOrder, int PassiveOrder>
    void node_node(vec3 com, float M, const Multipole<ActiveOrder> &mp, vec3 passive,
                   FieldExpansion<PassiveOrder> &f) const {
        static_assert(ActiveOrder == PassiveOrder - 1);
        if (com == passive) return;
        vec3 R = passive - com;
        float r = std::sqrt(length2(R) + epsilon);
        f.vector -= R * M * G / powi<3>(r);
        if constexpr (PassiveOrder >= 2) {
            f.t2 += D2(R, r) * M * G;
        }
        if constexpr (PassiveOrder >= 3) {
            f.t3 += D3(R, r) * M * G / 2.0f;
            f.vector += (contract_to_vector<3>(D3(R, r), mp.t2)) / 2.0f;
        }
        if constexpr (PassiveOrder >= 4) {
            f.t4 += D4(R, r) * M * G / 6.0f;
            f.t2 -= (contract_general<4, 2>(D4(R, r), mp.t2)) / 2.0f;
            f.vector += (contract_to_vector<4>(D4(R, r), mp.t3)) / 6.0f;
        }
    }
};

}  // namespace oracle
