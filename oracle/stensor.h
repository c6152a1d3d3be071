// Oracle (test infrastructure only): packed symmetric 3-tensors restated from the reference's
// SymmetricTensor3 (src/NBody/Physics/SymmetricTensor3.h). Used by the CPU restatement of the
// force path; never linked into the product library.
//
// Storage follows the reference's unique-value layout exactly, because the multipole moments
// and the field tensors are compared element by element between the oracle and the GPU:
//   - unique values of order k: 3, 6, 10, 15, 21 for k = 1..5          (SymmetricTensor3.h:36-40)
//   - unique index L of order k -> sorted dimensions                    (SymmetricTensor3.h:372-395)
//       L <  U(k-1): X followed by the order-(k-1) index of L
//       L >= U(k-1): Ys then Zs, with (L - U(k-1)) Zs
//   - lexicographic index I of order k: last dimension = I % 3, rest = index I / 3 (L397-410)
// Every product below evaluates its float operations in the same order as the reference's
// fold expressions, so that results are bit-identical with an IEEE FP32 build without FMA
// contraction (the reference is built with default flags: no -march, so no FMA).
#pragma once

#include <algorithm>
#include <array>
#include <cstddef>
#include <utility>

namespace oracle {

struct vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

inline vec3 operator+(vec3 a, vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(vec3 a, vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator-(vec3 a) { return {-a.x, -a.y, -a.z}; }
inline vec3 operator*(vec3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline vec3 operator*(float s, vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline vec3 operator/(vec3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline vec3 &operator+=(vec3 &a, vec3 b) { a = a + b; return a; }
inline vec3 &operator-=(vec3 &a, vec3 b) { a = a - b; return a; }
inline bool operator==(vec3 a, vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
// glm::dot for vec3: component products first, then (x + y) + z.
inline float dot(vec3 a, vec3 b) {
    float tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z;
    return tx + ty + tz;
}
inline float length2(vec3 a) { return dot(a, a); }

constexpr int unique_count(int order) { return order == 1 ? 3 : unique_count(order - 1) + order + 1; }
constexpr int full_count(int order) { return order == 1 ? 3 : 3 * full_count(order - 1); }

template<int K>
using Dims = std::array<int, K>;

// Compile-time loop: f(integral_constant<int, 0>), f(...1), ... in order, so that every index
// map below is folded to a constant like the reference's index_sequence folds.
template<int N, typename F>
inline void static_for(F &&f) {
    [&]<int... I>(std::integer_sequence<int, I...>) {
        (f(std::integral_constant<int, I>{}), ...);
    }(std::make_integer_sequence<int, N>{});
}

template<int K>
constexpr Dims<K> dimensional_index(int L) {
    Dims<K> d{};
    if constexpr (K == 1) {
        d[0] = L;
    } else {
        if (L < unique_count(K - 1)) {
            Dims<K - 1> lower = dimensional_index<K - 1>(L);
            d[0] = 0;
            for (int i = 0; i < K - 1; ++i) d[i + 1] = lower[i];
        } else {
            int zs = L - unique_count(K - 1);
            int ys = K - zs;
            for (int i = 0; i < K; ++i) d[i] = (i < ys) ? 1 : 2;
        }
    }
    return d;
}

template<int K>
constexpr int linear_index(Dims<K> d) {
    std::sort(d.begin(), d.end());
    if constexpr (K == 1) {
        return d[0];
    } else {
        if (d[0] == 0) {
            Dims<K - 1> tail{};
            for (int i = 0; i < K - 1; ++i) tail[i] = d[i + 1];
            return linear_index<K - 1>(tail);
        }
        int zs = 0;
        for (int i = 0; i < K; ++i) zs += (d[i] == 2);
        return unique_count(K - 1) + zs;
    }
}

template<int K>
constexpr Dims<K> lexicographic_index(int I) {
    Dims<K> d{};
    if constexpr (K == 1) {
        d[0] = I;
    } else {
        Dims<K - 1> lower = lexicographic_index<K - 1>(I / 3);
        for (int i = 0; i < K - 1; ++i) d[i] = lower[i];
        d[K - 1] = I % 3;
    }
    return d;
}

template<int K, int N>
constexpr Dims<N> head(Dims<K> d) {
    Dims<N> h{};
    for (int i = 0; i < N; ++i) h[i] = d[i];
    return h;
}

template<int K, int N>
constexpr Dims<N> tail(Dims<K> d) {
    Dims<N> t{};
    for (int i = 0; i < N; ++i) t[i] = d[K - N + i];
    return t;
}

// std::rotate(begin, begin + n, end): left rotation by n.
template<int K>
constexpr Dims<K> rotated(Dims<K> d, int n) {
    Dims<K> r{};
    for (int i = 0; i < K; ++i) r[i] = d[(i + n) % K];
    return r;
}

template<int K>
struct ST {
    static constexpr int U = unique_count(K);
    static constexpr int F = full_count(K);
    std::array<float, U> v{};

    template<typename... I>
    float &at(I... dims) { return v[linear_index<K>(Dims<K>{int(dims)...})]; }
    template<typename... I>
    float at(I... dims) const { return v[linear_index<K>(Dims<K>{int(dims)...})]; }

    ST &operator+=(const ST &o) { for (int i = 0; i < U; ++i) v[i] += o.v[i]; return *this; }
    ST &operator-=(const ST &o) { for (int i = 0; i < U; ++i) v[i] -= o.v[i]; return *this; }
    ST &operator*=(float s) { for (int i = 0; i < U; ++i) v[i] *= s; return *this; }
    ST &operator/=(float s) { for (int i = 0; i < U; ++i) v[i] /= s; return *this; }
    friend ST operator+(const ST &a, const ST &b) { ST r; for (int i = 0; i < U; ++i) r.v[i] = a.v[i] + b.v[i]; return r; }
    friend ST operator-(const ST &a, const ST &b) { ST r; for (int i = 0; i < U; ++i) r.v[i] = a.v[i] - b.v[i]; return r; }
    friend ST operator*(const ST &a, float s) { ST r; for (int i = 0; i < U; ++i) r.v[i] = a.v[i] * s; return r; }
    friend ST operator*(float s, const ST &a) { return a * s; }
    // tensor / scalar is evaluated as tensor * (1 / scalar) in the reference (SymmetricTensor3.h:307-309)
    friend ST operator/(const ST &a, float s) { return a * (1 / s); }
    bool operator==(const ST &o) const { return v == o.v; }

    vec3 diagonal() const { return {v[0], v[unique_count(K - 1)], v[U - 1]}; }

    static ST diagonal(vec3 d) {
        ST t;
        t.v[0] = d.x;
        t.v[unique_count(K - 1)] = d.y;
        t.v[U - 1] = d.z;
        return t;
    }

    static ST identity() {
        ST t;
        for (int L = 0; L < U; ++L) {
            Dims<K> d = dimensional_index<K>(L);
            bool same = true;
            for (int i = 1; i < K; ++i) same = same && d[i] == d[0];
            t.v[L] = same ? 1.0f : 0.0f;
        }
        return t;
    }
};

// Right fold v[d0] * (v[d1] * (... * v[dk-1])) as in productOfDimensions (SymmetricTensor3.h:470-475).
template<int K>
inline float product_of_dimensions(const Dims<K> &d, vec3 a) {
    float p = a[d[K - 1]];
    for (int i = K - 2; i >= 0; --i) p = a[d[i]] * p;
    return p;
}

template<int K>
inline ST<K> cartesian_power(vec3 a) {
    ST<K> t;
    static_for<ST<K>::U>([&](auto L) {
        constexpr Dims<K> d = dimensional_index<K>(L.value);
        t.v[L.value] = product_of_dimensions<K>(d, a);
    });
    return t;
}

// Reference helper for lower-order access: an order-1 "tensor" is the vec3 itself.
template<int K>
struct LowerT { using type = ST<K>; };
template<>
struct LowerT<1> { using type = vec3; };

template<int K, Dims<K> D>
inline float get_lower(const typename LowerT<K>::type &t) {
    if constexpr (K == 1) return t[D[0]];
    else return t.v[linear_index<K>(D)];
}

// outerProduct(T_{k-1}, v) at unique index d: T[head(d)] * v[d_last]   (SymmetricTensor3.h:478-481, 345-353)
template<int K>
inline ST<K> outer_product(const typename LowerT<K - 1>::type &t, vec3 a) {
    ST<K> r;
    static_for<ST<K>::U>([&](auto L) {
        constexpr Dims<K> d = dimensional_index<K>(L.value);
        r.v[L.value] = get_lower<K - 1, head<K, K - 1>(d)>(t) * a[d[K - 1]];
    });
    return r;
}

// sumOfOuterProducts: right fold over the K left rotations of the index (SymmetricTensor3.h:235-244, 483-488).
template<int K>
inline ST<K> sum_of_outer_products(const typename LowerT<K - 1>::type &t, vec3 a) {
    ST<K> r;
    static_for<ST<K>::U>([&](auto L) {
        constexpr Dims<K> d = dimensional_index<K>(L.value);
        float terms[K];
        static_for<K>([&](auto n) {
            constexpr Dims<K> rd = rotated<K>(d, n.value);
            terms[n.value] = get_lower<K - 1, head<K, K - 1>(rd)>(t) * a[rd[K - 1]];
        });
        float s = terms[K - 1];
        for (int n = K - 2; n >= 0; --n) s = terms[n] + s;
        r.v[L.value] = s;
    });
    return r;
}

// T_K * T_{K-1} -> vec3 (SymmetricTensor3.h:281-292): product[lex0] += A[lex] * B[tail(lex)], lex order.
template<int K>
inline vec3 contract_to_vector(const ST<K> &a, const typename LowerT<K - 1>::type &b) {
    vec3 p{};
    static_for<ST<K>::F>([&](auto I) {
        constexpr Dims<K> d = lexicographic_index<K>(I.value);
        p[d[0]] += a.v[linear_index<K>(d)] * get_lower<K - 1, tail<K, K - 1>(d)>(b);
    });
    return p;
}

// T_2 * v -> vec3 (SymmetricTensor3.h:253-260)
inline vec3 contract_down(const ST<2> &t, vec3 a) {
    return {(t.at(0, 0) * a.x) + (t.at(0, 1) * a.y) + (t.at(0, 2) * a.z),
            (t.at(1, 0) * a.x) + (t.at(1, 1) * a.y) + (t.at(1, 2) * a.z),
            (t.at(2, 0) * a.x) + (t.at(2, 1) * a.y) + (t.at(2, 2) * a.z)};
}

// T_K * v -> T_{K-1} for K >= 3 (SymmetricTensor3.h:262-272): product[head(lex)] += T[lex] * v[lex_last].
template<int K>
inline ST<K - 1> contract_down(const ST<K> &t, vec3 a) {
    ST<K - 1> p;
    static_for<ST<K>::F>([&](auto I) {
        constexpr Dims<K> d = lexicographic_index<K>(I.value);
        constexpr int lo = linear_index<K - 1>(head<K, K - 1>(d));
        constexpr int hi = linear_index<K>(d);
        p.v[lo] += t.v[hi] * a[d[K - 1]];
    });
    return p;
}

// T_K * T_M -> T_{K-M} for M < K - 1 (SymmetricTensor3.h:295-307).
template<int K, int M>
inline ST<K - M> contract_general(const ST<K> &a, const ST<M> &b) {
    ST<K - M> p;
    static_for<ST<K>::F>([&](auto I) {
        constexpr Dims<K> d = lexicographic_index<K>(I.value);
        constexpr int lo = linear_index<K - M>(head<K, K - M>(d));
        constexpr int hi = linear_index<K>(d);
        constexpr int rb = linear_index<M>(tail<K, M>(d));
        p.v[lo] += a.v[hi] * b.v[rb];
    });
    return p;
}

// fullyContract (SymmetricTensor3.h:327-331)
template<int K>
inline vec3 fully_contract(const ST<K> &t, vec3 a) {
    if constexpr (K == 2) return contract_down(t, a);
    else return fully_contract<K - 1>(contract_down<K>(t, a), a);
}

}  // namespace oracle
