// vmath.cuh — float3 / column-major mat3 arithmetic of physics.comp.
//
// Every expression keeps the GLSL evaluation order of physics.comp and the
// library is compiled with -fmad=false, so each product and sum rounds on
// its own (no FMA contraction) and results are reproducible bit for bit:
//   dot(a,b)   = (a.x*b.x + a.y*b.y) + a.z*b.z
//   R*v        = (c0*v.x + c1*v.y) + c2*v.z            (GLSL mat3, columns)
//   Rᵀ*v       = (dot(c0,v), dot(c1,v), dot(c2,v))
//   normalize  = v / length(v), componentwise IEEE division
//   min(x,y)   = y<x ? y : x ; max(x,y) = x<y ? y : x  (GLSL definitions)
#pragma once
#include <cstdint>

namespace seevr {

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 neg(f3 a) { return f3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 scale(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 hadamard(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ f3 divs(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 normalize(f3 a) { return divs(a, length(a)); }
__device__ __forceinline__ float gmin(float x, float y) { return y < x ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return x < y ? y : x; }
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return f3{gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)}; }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return f3{gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }

__device__ __forceinline__ f3 ld3(const float* p, uint32_t i) {
    return f3{p[size_t(i) * 3], p[size_t(i) * 3 + 1], p[size_t(i) * 3 + 2]};
}
__device__ __forceinline__ void st3(float* p, uint32_t i, f3 v) {
    p[size_t(i) * 3] = v.x;
    p[size_t(i) * 3 + 1] = v.y;
    p[size_t(i) * 3 + 2] = v.z;
}

// GLSL mat3 as three columns.
struct m3 {
    f3 c0, c1, c2;
};

// quat_to_mat (physics.comp:74-81), quaternion xyzw.
__device__ __forceinline__ m3 quat_to_mat(float x, float y, float z, float w) {
    m3 m;
    m.c0 = f3{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + w * z), 2.0f * (x * z - w * y)};
    m.c1 = f3{2.0f * (x * y - w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + w * x)};
    m.c2 = f3{2.0f * (x * z + w * y), 2.0f * (y * z - w * x), 1.0f - 2.0f * (x * x + y * y)};
    return m;
}
__device__ __forceinline__ m3 quat_to_mat(const float* q, uint32_t i) {
    return quat_to_mat(q[size_t(i) * 4], q[size_t(i) * 4 + 1], q[size_t(i) * 4 + 2],
                       q[size_t(i) * 4 + 3]);
}
__device__ __forceinline__ f3 mul(const m3& m, f3 v) {
    return f3{m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z,
              m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
              m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z};
}
__device__ __forceinline__ f3 mulT(const m3& m, f3 v) { return f3{dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }
// apply_inv_I (physics.comp:90-94): R * (inv_i ⊙ (Rᵀ v))
__device__ __forceinline__ f3 apply_inv_I(const m3& R, f3 inv_i, f3 v) {
    return mul(R, hadamard(inv_i, mulT(R, v)));
}
__device__ __forceinline__ void st_m3(float* p, uint32_t i, const m3& m) {
    float* q = p + size_t(i) * 9;
    q[0] = m.c0.x; q[1] = m.c0.y; q[2] = m.c0.z;
    q[3] = m.c1.x; q[4] = m.c1.y; q[5] = m.c1.z;
    q[6] = m.c2.x; q[7] = m.c2.y; q[8] = m.c2.z;
}
__device__ __forceinline__ m3 ld_m3(const float* p, uint32_t i) {
    const float* q = p + size_t(i) * 9;
    m3 m;
    m.c0 = f3{q[0], q[1], q[2]};
    m.c1 = f3{q[3], q[4], q[5]};
    m.c2 = f3{q[6], q[7], q[8]};
    return m;
}

// Arctangent of y/x in (-pi, pi], replacing GLSL atan(y,x)
// (physics.comp:136-140).  After folding to t = min/max in [0,1], values
// above tan(pi/8) use atan(t) = pi/4 + atan((t-1)/(t+1)), leaving
// |u| <= 0.4142 for the Maclaurin series sum (-1)^k u^(2k+1)/(2k+1)
// truncated after u^19 (truncation error < 1e-9).  atan2(0,0) = 0.
__device__ __forceinline__ float seevr_atan2f(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = ax < ay ? ay : ax;
    const float mn = ax < ay ? ax : ay;
    if (mx == 0.0f) return 0.0f;
    float t = mn / mx;
    float base = 0.0f;
    if (t > 0.41421356237309503f) {
        t = (t - 1.0f) / (t + 1.0f);
        base = 0.78539816339744831f;
    }
    const float u2 = t * t;
    float p = 1.0f / 19.0f;
    p = 1.0f / 17.0f - u2 * p;
    p = 1.0f / 15.0f - u2 * p;
    p = 1.0f / 13.0f - u2 * p;
    p = 1.0f / 11.0f - u2 * p;
    p = 1.0f / 9.0f - u2 * p;
    p = 1.0f / 7.0f - u2 * p;
    p = 1.0f / 5.0f - u2 * p;
    p = 1.0f / 3.0f - u2 * p;
    p = 1.0f - u2 * p;
    float r = base + t * p;
    if (ay > ax) r = 1.5707963267948966f - r;
    if (x < 0.0f) r = 3.1415926535897931f - r;
    if (y < 0.0f) r = -r;
    return r;
}

}  // namespace seevr
