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

// The support lookup's bin of an axis angle (physics.comp:136-147: atan(y,x),
// plus 2 pi when negative, / 2 pi * 64, truncated, mod 64), found without
// the angle.  The quadrant comes from the signs; (u, v), the direction
// rotated into the first quadrant (u > 0, v >= 0), has angle atan(v/u) in
// [0, pi/2), which is at least j pi/32 exactly when v >= u tan(j pi/32), so
// a binary search over the tangents of the 15 inner boundaries gives the
// bin within the quadrant.  The same bin as the angle's except within
// rounding of a boundary (where the reference's own GLSL atan and division
// are of implementation-defined precision); (0,0) -> bin 0, as atan(0,0)
// = 0.  Four multiplies and compares instead of an arctangent and two
// divisions.  The thresholds are tan(j pi/32) rounded to float.
__device__ __forceinline__ uint32_t angle_bin64(float y, float x) {
    float u, v;
    uint32_t q;
    if (x > 0.0f && y >= 0.0f) {
        q = 0, u = x, v = y;
    } else if (x <= 0.0f && y > 0.0f) {
        q = 16, u = y, v = -x;
    } else if (x < 0.0f && y <= 0.0f) {
        q = 32, u = -x, v = -y;
    } else if (x >= 0.0f && y < 0.0f) {
        q = 48, u = -y, v = x;
    } else {
        return 0;
    }
    // tan(j pi/32) for j = 4, 8, 12; then j + 2 in {2, 6, 10, 14}; then the odd j
    const bool h8 = v >= u * 1.0f;
    const bool h4 = v >= u * (h8 ? 2.4142137f : 0.41421357f);
    const uint32_t j4 = (h8 ? 8u : 0u) + (h4 ? 4u : 0u);
    const float t2 = h8 ? (h4 ? 5.0273395f : 1.4966058f) : (h4 ? 0.6681786f : 0.19891237f);
    const bool h2 = v >= u * t2;
    const uint32_t j2 = j4 + (h2 ? 2u : 0u);
    float t1;
    switch (j2) {  // tan((j2 + 1) pi/32)
        case 0: t1 = 0.0984914f; break;
        case 2: t1 = 0.3033467f; break;
        case 4: t1 = 0.53451115f; break;
        case 6: t1 = 0.8206788f; break;
        case 8: t1 = 1.2185035f; break;
        case 10: t1 = 1.8708684f; break;
        case 12: t1 = 3.2965581f; break;
        default: t1 = 10.153171f; break;
    }
    return q + j2 + (v >= u * t1 ? 1u : 0u);
}

}  // namespace seevr
