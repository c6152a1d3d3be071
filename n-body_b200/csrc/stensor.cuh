// Packed symmetric 3-tensors for the dual-tree path (device code).
//
// Storage and products follow the reference's SymmetricTensor3 (src/NBody/Physics/SymmetricTensor3.h):
//   - unique values of order k: 3, 6, 10, 15 for k = 1..4, in the reference's unique-index order
//     (an index starting with X defers to the order k-1 layout; the rest hold Ys then Zs,
//     position = count of Zs);
//   - T_k * v -> T_(k-1) (L262-272) and T_k * T_m -> T_(k-m) (L295-307) accumulate every one of
//     the 3^k index tuples into the unique slot of its (sorted) head, so off-diagonal slots
//     collect one term per permutation of the head: these are the reference's semantics, restated
//     as they are because field expansions are compared against the reference's arithmetic;
//   - T_k * T_(k-1) -> vector (L281-292) is the full sum over all index tuples.
#pragma once

#include <cuda_runtime.h>

namespace nbg {
namespace st {

template<int K>
struct Count;
template<> struct Count<1> { static constexpr int U = 3; };
template<> struct Count<2> { static constexpr int U = 6; };
template<> struct Count<3> { static constexpr int U = 10; };
template<> struct Count<4> { static constexpr int U = 15; };
template<> struct Count<5> { static constexpr int U = 21; };

// Unique-slot index of a (not necessarily sorted) index tuple.
__host__ __device__ constexpr int idx1(int a) { return a; }
__host__ __device__ constexpr int idx2s(int a, int b) { return a == 0 ? idx1(b) : 3 + (a == 2) + (b == 2); }
__host__ __device__ constexpr int idx2(int a, int b) { return a <= b ? idx2s(a, b) : idx2s(b, a); }
__host__ __device__ constexpr int idx3s(int a, int b, int c) {
    return a == 0 ? idx2s(b, c) : 6 + (a == 2) + (b == 2) + (c == 2);
}
__host__ __device__ constexpr int idx3(int a, int b, int c) {
    // sort three
    return (a <= b) ? ((b <= c) ? idx3s(a, b, c) : (a <= c ? idx3s(a, c, b) : idx3s(c, a, b)))
                    : ((a <= c) ? idx3s(b, a, c) : (b <= c ? idx3s(b, c, a) : idx3s(c, b, a)));
}
__host__ __device__ constexpr int idx4s(int a, int b, int c, int d) {
    return a == 0 ? idx3s(b, c, d) : 10 + (a == 2) + (b == 2) + (c == 2) + (d == 2);
}
__host__ __device__ constexpr int idx4(int a, int b, int c, int d) {
    // the slot only depends on how many of each dimension the tuple holds
    const int nx = (a == 0) + (b == 0) + (c == 0) + (d == 0);
    const int nz = (a == 2) + (b == 2) + (c == 2) + (d == 2);
    const int ny = 4 - nx - nz;
    return nx == 4 ? 0 : idx4s(nx > 0 ? 0 : (ny > 0 ? 1 : 2), nx > 1 ? 0 : (nx + ny > 1 ? 1 : 2),
                               nx > 2 ? 0 : (nx + ny > 2 ? 1 : 2), nx + ny > 3 ? 1 : 2);
}

__device__ __forceinline__ float comp(const float v[3], int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }

// g_k coefficients of the softened 1/r derivatives: f_k = (-1)^k (2k-1)!! / r^(k+1), g_k = f_k / r^k
// (Gravity.h:43-58).
struct Coef {
    float g1, g2, g3, g4;
    Coef() = default;
    __device__ explicit Coef(float r) {
        const float r2 = r * r, r3 = r * r2, r4 = r * r3, r5 = r * r4;
        g1 = (-1.0f / r2) / r;
        g2 = (3.0f / r3) / r2;
        g3 = (-15.0f / r4) / r3;
        g4 = (105.0f / r5) / r4;
    }
    // the same coefficients from 1 / r: g_k = (-1)^k (2k-1)!! / r^(2k+1)
    __device__ static Coef from_inverse(float inv) {
        Coef c;
        const float i2 = inv * inv, i3 = inv * i2, i5 = i3 * i2, i7 = i5 * i2, i9 = i7 * i2;
        c.g1 = -i3;
        c.g2 = 3.0f * i5;
        c.g3 = -15.0f * i7;
        c.g4 = 105.0f * i9;
        return c;
    }
};

__device__ __forceinline__ float kd(int a, int b) { return a == b ? 1.f : 0.f; }

// D<2>, D<3>, D<4> of the softened potential at offset R (Gravity.h:60-110), unique slots.
__device__ __forceinline__ void D2(const float R[3], const Coef &c, float out[6]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) out[idx2(i, j)] = c.g2 * (R[i] * R[j]) + c.g1 * kd(i, j);
}
__device__ __forceinline__ void D3(const float R[3], const Coef &c, float out[10]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
#pragma unroll
            for (int k = j; k < 3; ++k)
                out[idx3(i, j, k)] = c.g3 * (R[i] * R[j] * R[k]) +
                                     c.g2 * (kd(i, j) * R[k] + kd(j, k) * R[i] + kd(i, k) * R[j]);
}
__device__ __forceinline__ void D4(const float R[3], const Coef &c, float out[15]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
#pragma unroll
            for (int k = j; k < 3; ++k)
#pragma unroll
                for (int l = k; l < 3; ++l) {
                    const float pairs = kd(i, j) * R[k] * R[l] + kd(i, k) * R[j] * R[l] + kd(i, l) * R[j] * R[k] +
                                        kd(j, k) * R[i] * R[l] + kd(j, l) * R[i] * R[k] + kd(k, l) * R[i] * R[j];
                    const float dd = kd(i, j) * kd(k, l) + kd(i, k) * kd(j, l) + kd(i, l) * kd(j, k);
                    out[idx4(i, j, k, l)] = c.g4 * (R[i] * R[j] * R[k] * R[l]) + c.g3 * pairs + c.g2 * dd;
                }
}

// T_k * T_(k-1) -> vector (full sum over index tuples)
__device__ __forceinline__ void t3_dot_t2(const float t3[10], const float t2[6], float out[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) s = fmaf(t3[idx3(i, j, k)], t2[idx2(j, k)], s);
        out[i] = s;
    }
}
__device__ __forceinline__ void t4_dot_t3(const float t4[15], const float t3[10], float out[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l = 0; l < 3; ++l) s = fmaf(t4[idx4(i, j, k, l)], t3[idx3(j, k, l)], s);
        out[i] = s;
    }
}

// T_2 * v -> vector (explicit product, SymmetricTensor3.h:253-260)
__device__ __forceinline__ void t2_dot_v(const float t2[6], const float v[3], float out[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) s = fmaf(t2[idx2(i, j)], v[j], s);
        out[i] = s;
    }
}

// T_3 * v -> T_2 and T_4 * v -> T_3, accumulating every tuple into its head's unique slot.
__device__ __forceinline__ void t3_dot_v(const float t3[10], const float v[3], float out[6]) {
#pragma unroll
    for (int a = 0; a < 6; ++a) out[a] = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) out[idx2(i, j)] = fmaf(t3[idx3(i, j, k)], v[k], out[idx2(i, j)]);
}
__device__ __forceinline__ void t4_dot_v(const float t4[15], const float v[3], float out[10]) {
#pragma unroll
    for (int a = 0; a < 10; ++a) out[a] = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l = 0; l < 3; ++l)
                    out[idx3(i, j, k)] = fmaf(t4[idx4(i, j, k, l)], v[l], out[idx3(i, j, k)]);
}
// T_4 * T_2 -> T_2 (head pair <- tail pair), SymmetricTensor3.h:295-307
__device__ __forceinline__ void t4_dot_t2(const float t4[15], const float t2[6], float out[6]) {
#pragma unroll
    for (int a = 0; a < 6; ++a) out[a] = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l = 0; l < 3; ++l)
                    out[idx2(i, j)] = fmaf(t4[idx4(i, j, k, l)], t2[idx2(k, l)], out[idx2(i, j)]);
}

// Local field of order 4 (MultipoleAcceleration<4>): vector + field tensors of order 2, 3, 4.
struct Field4 {
    float v[3], t2[6], t3[10], t4[15];
    __device__ void zero() {
#pragma unroll
        for (int a = 0; a < 3; ++a) v[a] = 0.f;
#pragma unroll
        for (int a = 0; a < 6; ++a) t2[a] = 0.f;
#pragma unroll
        for (int a = 0; a < 10; ++a) t3[a] = 0.f;
#pragma unroll
        for (int a = 0; a < 15; ++a) t4[a] = 0.f;
    }
};
constexpr int kFieldFloats = 34;

// MultipoleAcceleration::at (MultipoleAcceleration.h:33-49)
__device__ __forceinline__ void field_at(const float *f, const float o[3], float out[3]) {
    const float *v = f, *t2 = f + 3, *t3 = f + 9, *t4 = f + 19;
    float a[3], b2[6], b[3], c3[10], c2[6], c[3];
    t2_dot_v(t2, o, a);
    t3_dot_v(t3, o, b2);
    t2_dot_v(b2, o, b);
    t4_dot_v(t4, o, c3);
    t3_dot_v(c3, o, c2);
    t2_dot_v(c2, o, c);
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i] = v[i] + a[i] + b[i] / 2.0f + c[i] / 6.0f;
}

// MultipoleAcceleration::translated (MultipoleAcceleration.h:51-84), in -> out (may alias? no)
__device__ __forceinline__ void field_translated(const float *f, const float o[3], float *out) {
    const float *v = f, *t2 = f + 3, *t3 = f + 9, *t4 = f + 19;
    float d1[3], d2[6], d2v[3], e3[10], e2[6], e1[3];
    t2_dot_v(t2, o, d1);
    t3_dot_v(t3, o, d2);
    t2_dot_v(d2, o, d2v);
    t4_dot_v(t4, o, e3);
    t3_dot_v(e3, o, e2);
    t2_dot_v(e2, o, e1);
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i] = v[i] + d1[i] + d2v[i] / 2.0f + e1[i] / 6.0f;
#pragma unroll
    for (int a = 0; a < 6; ++a) out[3 + a] = t2[a] + d2[a] + e2[a] * 0.5f;
#pragma unroll
    for (int a = 0; a < 10; ++a) out[9 + a] = t3[a] + e3[a];
#pragma unroll
    for (int a = 0; a < 15; ++a) out[19 + a] = t4[a];
}

}  // namespace st
}  // namespace nbg
