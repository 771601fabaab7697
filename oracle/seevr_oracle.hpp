// seevr_oracle.hpp — TEST INFRASTRUCTURE, not product code.
//
// CPU restatement of seeVR's physics step (src/shaders/physics.comp as
// dispatched by src/physics.zig) and of the LBVH build (src/shaders/bvh.comp
// as dispatched by src/bvh.zig).  It is the checker for the CUDA library:
// only tests, the smoke check and the CPU baseline of bench.py use it.
//
// Parity status: the reference has no tests, golden vectors or fixtures and
// cannot run here (Zig toolchain and a Vulkan ICD are absent), so parity is
// UNPINNED against reference outputs.  This file follows the shader line by
// line (citations below) and is pinned against analytic known-answer cases
// derived from the code (tests/test_oracle.py).
//
// Semantics kept from the reference, with the two documented changes:
//  1. canonical order: broadphase pairs are emitted in lexicographic (i,j)
//     order and contacts in pair order (the reference appends both with
//     atomicAdd, physics.comp:465 and 404, so its own order varies run to
//     run);
//  2. the support lookup's bin of each axis angle, uint(atan(y,x) (+2 pi if
//     negative) / 2 pi * 64) % 64 (physics.comp:136-147), is found without
//     the angle: by quadrant and by comparing against the tangents of the
//     bin boundaries (angle_bin64 below).  It is the same bin except for
//     directions within rounding of a bin boundary, where the reference's
//     own choice depends on its GLSL atan and division, both of
//     implementation-defined precision.
// FP32 instantiation compiled with -ffp-contract=off (no FMA), so every
// expression rounds exactly as written; FP64 instantiation = error reference.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

template <class R>
struct V3 {
    R x, y, z;
};
template <class R> inline V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> mulv(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline V3<R> divs(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> normalize(V3<R> a) { return divs(a, length(a)); }
// GLSL min/max: min(x,y) = y<x ? y : x ; max(x,y) = x<y ? y : x
template <class R> inline R gmin(R x, R y) { return y < x ? y : x; }
template <class R> inline R gmax(R x, R y) { return x < y ? y : x; }
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) { return {gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) { return {gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }

// GLSL mat3 stored as three columns.
template <class R>
struct M3 {
    V3<R> c0, c1, c2;
};
// R * v = c0*v.x + c1*v.y + c2*v.z
template <class R> inline V3<R> mul(const M3<R>& m, V3<R> v) {
    return {m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z,
            m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
            m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z};
}
// transpose(R) * v = (dot(c0,v), dot(c1,v), dot(c2,v))
template <class R> inline V3<R> mulT(const M3<R>& m, V3<R> v) {
    return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)};
}

// tan(j*pi/32), j = 0..15, rounded to float: the boundaries of the 16 bins
// of one quadrant.  The CUDA kernel holds the same float values.
constexpr float kTanBin[16] = {0.0f,       0.0984914f, 0.19891237f, 0.3033467f,
                               0.41421357f, 0.53451115f, 0.6681786f,  0.8206788f,
                               1.0f,        1.2185035f,  1.4966058f,  1.8708684f,
                               2.4142137f,  3.2965581f,  5.0273395f,  10.153171f};

// Bin k of 64 equal bins of the angle atan2(y, x) taken in [0, 2 pi) (bin k
// covers [k pi/32, (k+1) pi/32)), found without the angle.  The quadrant
// comes from the signs; (u, v), the direction rotated into the first
// quadrant (u > 0, v >= 0), has angle phi = atan(v/u) in [0, pi/2), and
// phi >= j pi/32 exactly when v >= u tan(j pi/32), so a binary search over
// the 15 tangents gives the bin within the quadrant.  (0,0) -> bin 0, as
// the reference's atan(0,0) = 0.
template <class R>
inline uint32_t angle_bin64(R y, R x) {
    R u, v;
    uint32_t q;
    if (x > R(0) && y >= R(0)) {
        q = 0, u = x, v = y;
    } else if (x <= R(0) && y > R(0)) {
        q = 16, u = y, v = -x;
    } else if (x < R(0) && y <= R(0)) {
        q = 32, u = -x, v = -y;
    } else if (x >= R(0) && y < R(0)) {
        q = 48, u = -y, v = x;
    } else {
        return 0;
    }
    uint32_t j = v >= u * R(kTanBin[8]) ? 8u : 0u;
    if (v >= u * R(kTanBin[j + 4])) j += 4;
    if (v >= u * R(kTanBin[j + 2])) j += 2;
    if (v >= u * R(kTanBin[j + 1])) j += 1;
    return q + j;
}

// Input arrays, indexed like the physics.comp bindings (physics.comp:16-57).
struct SceneIn {
    uint32_t num_bodies = 0, num_geoms = 0, num_hull_verts = 0, num_vertices = 0;
    uint32_t num_scenes = 1;
    const float *body_pos, *body_quat, *body_vel, *body_omega, *body_inv_mass, *body_inv_inertia;
    const uint32_t *body_vert_start, *body_vert_count, *geom_body_idx;
    const float *geom_data, *geom_friction, *geom_restitution, *hull_verts, *orig_verts;
    const uint32_t *support_offset, *support_lookup;
    const uint32_t* scene_body_offset = nullptr;  // [num_scenes+1] or NULL
    const uint32_t* hull_range = nullptr;         // [G*2] or NULL (replaces geom_data[0..1])
};

struct Params {
    uint32_t pgs_iterations = 4;  // physics.comp:68
    double baumgarte = 0.2;       // physics.comp:66
    double slop = 0.005;          // physics.comp:67
    double lin_damp = 0.999;      // physics.comp:422
    double ang_damp = 0.998;      // physics.comp:425
    double eps = 1e-6;            // physics.comp:174
    double tol = 1e-6;            // physics.comp:175
    uint32_t mpr_iterations = 50; // physics.comp:176
    uint32_t discover_trials = 15;// physics.comp:290
    uint32_t max_pairs = 10000;   // physics.comp:70
    uint32_t max_contacts = 4000; // physics.comp:69
    uint32_t narrowphase = 0;     // 0: MPR (physics.comp:171-399), 1: GJK + EPA
};

// Work counters for the algorithmic flop count of one run.
struct OpCounts {
    uint64_t support_brute = 0, support_brute_verts = 0, support_lookup = 0;
    uint64_t mpr_calls = 0, mpr_support_calls = 0;
    uint64_t pgs_contact_iters = 0, pgs_friction_iters = 0;
    uint64_t aabb_verts = 0, broad_tests = 0, bodies = 0;
};

template <class R>
class Physics {
   public:
    // state (mutable) and constants converted to R
    std::vector<R> pos, quat, vel, omega, inv_mass, inv_inertia, hull, orig, verts;
    std::vector<R> friction, restitution;
    std::vector<uint32_t> hull_start, hull_count, vert_start, geom_body, sup_off;
    const uint32_t* sup_lut = nullptr;  // shared lookup table (absolute offsets)
    std::vector<uint32_t> scene_of;  // body -> scene
    // Test instrumentation (off while empty): per scene, a hash of the
    // step's structural decisions (every support vertex chosen, every pair
    // and whether it made a contact), so that two runs can be checked to
    // have produced the same contact sets from the same MPR portals.
    std::vector<uint64_t> branch;
    void mix(uint32_t body, uint64_t v) {
        if (branch.empty()) return;
        uint64_t& h = branch[scene_of[body]];
        h = (h ^ v) * 1099511628211ull;
    }
    // Test instrumentation: branch locking.  In Record mode every
    // data-dependent decision of the step (each float comparison that picks
    // a branch, each support vertex chosen) is appended to `lock`; in Replay
    // mode the decisions are read back instead of computed, so that a run in
    // another precision, or from perturbed inputs, follows exactly the
    // recorded branches.  Finite differences of replayed FP64 runs are then
    // the derivative of the recorded branch: what an adjoint computes.
    enum class Lock { Off, Record, Replay };
    Lock lock_mode = Lock::Off;
    std::vector<uint32_t> lock;
    size_t lock_pos = 0;
    bool lock_error = false;  // replay ran past the recorded decisions
    uint32_t decide(uint32_t v) {
        if (lock_mode == Lock::Record) {
            lock.push_back(v);
        } else if (lock_mode == Lock::Replay) {
            if (lock_pos < lock.size()) return lock[lock_pos++];
            lock_error = true;
        }
        return v;
    }
    bool decide(bool b) { return decide(b ? 1u : 0u) != 0u; }
    std::vector<uint32_t> scene_end; // scene -> one past its last body
    uint32_t nb = 0, nv = 0, nhv = 0;
    Params P;
    // step outputs (last substep)
    std::vector<R> aabb_min, aabb_max;
    std::vector<uint32_t> pairs;  // canonical, truncated to max_pairs
    uint32_t pairs_total = 0, contacts_total = 0;
    std::vector<R> c_pos, c_normal, c_pen, lambda;
    std::vector<uint32_t> c_a, c_b;
    OpCounts ops;

    // Bodies [b0, b1) of `in` (geom g == body g, physics.comp:99).  With
    // b0 = 0, b1 = num_bodies the whole batch is one instance whose
    // broadphase respects in.scene_body_offset; any other range must be one
    // whole scene.  Hull and render-vertex indices are rebased to the range.
    Physics(const SceneIn& in, const Params& p, uint32_t b0 = 0, uint32_t b1 = 0xFFFFFFFFu)
        : P(p) {
        if (b1 == 0xFFFFFFFFu) b1 = in.num_bodies;
        nb = b1 - b0;
        auto cvt = [](const float* src, size_t n) {
            std::vector<R> v(n);
            for (size_t i = 0; i < n; ++i) v[i] = R(src[i]);
            return v;
        };
        hull_start.resize(nb);
        hull_count.resize(nb);
        for (uint32_t g = 0; g < nb; ++g) {
            if (in.hull_range) {
                hull_start[g] = in.hull_range[(b0 + g) * 2];
                hull_count[g] = in.hull_range[(b0 + g) * 2 + 1];
            } else {  // uint(geom_data[gi*8+0]) (physics.comp:100-101)
                hull_start[g] = uint32_t(in.geom_data[(b0 + g) * 8 + 0]);
                hull_count[g] = uint32_t(in.geom_data[(b0 + g) * 8 + 1]);
            }
        }
        const bool whole = (b0 == 0 && b1 == in.num_bodies);
        const uint32_t h0 = whole ? 0 : hull_start[0];
        const uint32_t h1 = whole ? in.num_hull_verts : hull_start[nb - 1] + hull_count[nb - 1];
        for (auto& h : hull_start) h -= h0;
        nhv = h1 - h0;
        const uint32_t r0 = whole ? 0 : in.body_vert_start[b0];
        const uint32_t r1 = whole ? in.num_vertices
                                  : in.body_vert_start[b1 - 1] + in.body_vert_count[b1 - 1];
        nv = in.orig_verts ? r1 - r0 : 0;
        pos = cvt(in.body_pos + size_t(b0) * 3, size_t(nb) * 3);
        quat = cvt(in.body_quat + size_t(b0) * 4, size_t(nb) * 4);
        vel = cvt(in.body_vel + size_t(b0) * 3, size_t(nb) * 3);
        omega = cvt(in.body_omega + size_t(b0) * 3, size_t(nb) * 3);
        inv_mass = cvt(in.body_inv_mass + b0, nb);
        inv_inertia = cvt(in.body_inv_inertia + size_t(b0) * 3, size_t(nb) * 3);
        hull = cvt(in.hull_verts + size_t(h0) * 3, size_t(nhv) * 3);
        if (nv) {
            orig = cvt(in.orig_verts + size_t(r0) * 3, size_t(nv) * 3);
            verts.assign(size_t(nv) * 3, R(0));
        }
        friction = cvt(in.geom_friction + b0, nb);
        restitution = cvt(in.geom_restitution + b0, nb);
        vert_start.resize(nb);
        for (uint32_t b = 0; b < nb; ++b) vert_start[b] = in.body_vert_start[b0 + b] - r0;
        geom_body.resize(nb);
        for (uint32_t g = 0; g < nb; ++g) geom_body[g] = in.geom_body_idx[b0 + g] - b0;
        sup_off.assign(in.support_offset + b0, in.support_offset + b1);
        sup_lut = in.support_lookup;
        scene_of.assign(nb, 0);
        if (whole && in.scene_body_offset && in.num_scenes > 0) {
            for (uint32_t s = 0; s < in.num_scenes; ++s) {
                for (uint32_t b = in.scene_body_offset[s]; b < in.scene_body_offset[s + 1]; ++b)
                    scene_of[b] = s;
                scene_end.push_back(in.scene_body_offset[s + 1]);
            }
        } else {
            scene_end.push_back(nb);
        }
        aabb_min.assign(size_t(nb) * 3, R(0));
        aabb_max.assign(size_t(nb) * 3, R(0));
        lambda.assign(P.max_contacts, R(0));
    }

    // ---- helpers (physics.comp:74-102) ----
    M3<R> quat_to_mat(uint32_t bi) const {
        const R x = quat[bi * 4], y = quat[bi * 4 + 1], z = quat[bi * 4 + 2], w = quat[bi * 4 + 3];
        const R one(1), two(2);
        M3<R> m;
        m.c0 = {one - two * (y * y + z * z), two * (x * y + w * z), two * (x * z - w * y)};
        m.c1 = {two * (x * y - w * z), one - two * (x * x + z * z), two * (y * z + w * x)};
        m.c2 = {two * (x * z + w * y), two * (y * z - w * x), one - two * (x * x + y * y)};
        return m;
    }
    V3<R> get3(const std::vector<R>& a, uint32_t i) const { return {a[i * 3], a[i * 3 + 1], a[i * 3 + 2]}; }
    void set3(std::vector<R>& a, uint32_t i, V3<R> v) {
        a[i * 3] = v.x;
        a[i * 3 + 1] = v.y;
        a[i * 3 + 2] = v.z;
    }
    V3<R> apply_inv_I(uint32_t bi, V3<R> v) const {  // physics.comp:90-94
        const M3<R> Rm = quat_to_mat(bi);
        return mul(Rm, mulv(get3(inv_inertia, bi), mulT(Rm, v)));
    }

    // ---- support (physics.comp:107-162) ----
    V3<R> support(uint32_t bi, V3<R> d) {
        const M3<R> Rm = quat_to_mat(bi);
        const V3<R> p = get3(pos, bi);
        const V3<R> ld = mulT(Rm, d);
        const uint32_t vs = hull_start[bi], vc = hull_count[bi];
        const uint32_t lk = sup_off[bi];
        if (lk == 0) {
            ops.support_brute++;
            ops.support_brute_verts += vc;
            R best = R(-1e10);
            V3<R> bv = {R(0), R(0), R(0)};
            uint32_t chosen = 0xFFFFFFFFu;
            for (uint32_t i = 0; i < vc; ++i) {
                const V3<R> v = get3(hull, vs + i);
                const R dd = dot(v, ld);
                if (dd > best) {
                    best = dd;
                    bv = v;
                    chosen = i;
                }
            }
            chosen = decide(chosen);
            bv = chosen < vc ? get3(hull, vs + chosen) : V3<R>{R(0), R(0), R(0)};
            mix(bi, chosen);
            return p + mul(Rm, bv);
        }
        ops.support_lookup++;
        // the bins of atan(z,y), atan(z,x), atan(y,x) (X, Y, Z axes)
        const uint32_t bins[3] = {angle_bin64(ld.z, ld.y), angle_bin64(ld.z, ld.x),
                                  angle_bin64(ld.y, ld.x)};
        R best = R(-1e10);
        V3<R> bv = {R(0), R(0), R(0)};
        uint32_t chosen = 0xFFFFFFFFu;
        for (uint32_t ax = 0; ax < 3; ++ax) {
            const uint32_t b0 = bins[ax];
            const uint32_t b1 = (b0 + 1) % 64u;
            const V3<R> v0 = get3(hull, vs + sup_lut[lk + ax * 64 + b0]);
            const R d0 = dot(v0, ld);
            if (d0 > best) {
                best = d0;
                bv = v0;
                chosen = sup_lut[lk + ax * 64 + b0];
            }
            const V3<R> v1 = get3(hull, vs + sup_lut[lk + ax * 64 + b1]);
            const R d1 = dot(v1, ld);
            if (d1 > best) {
                best = d1;
                bv = v1;
                chosen = sup_lut[lk + ax * 64 + b1];
            }
        }
        chosen = decide(chosen);
        bv = chosen < vc ? get3(hull, vs + chosen) : V3<R>{R(0), R(0), R(0)};
        mix(bi, chosen);
        return p + mul(Rm, bv);
    }
    void mink(uint32_t a, uint32_t b, V3<R> d, V3<R>& v, V3<R>& sa, V3<R>& sb) {  // 165-169
        ops.mpr_support_calls++;
        sa = support(a, d);
        sb = support(b, -d);
        v = sa - sb;
    }

    // ---- MPR (physics.comp:171-399) ----
    R eps() const { return R(P.eps); }
    V3<R> portal_dir(V3<R> v1, V3<R> v2, V3<R> v3) const { return normalize(cross(v2 - v1, v3 - v1)); }
    bool reach_tol(V3<R> v1, V3<R> v2, V3<R> v3, V3<R> v4, V3<R> dir) const {
        const R dv1 = dot(v1, dir), dv2 = dot(v2, dir), dv3 = dot(v3, dir), dv4 = dot(v4, dir);
        const R dot1 = gmin(gmin(dv4 - dv1, dv4 - dv2), dv4 - dv3);
        return dot1 < R(P.tol) + eps() * gmax(R(1), dot1);
    }
    void expand(V3<R>& v0, V3<R>& v1, V3<R>& v2, V3<R>& v3, V3<R> v4, V3<R>& s1a,
                V3<R>& s2a, V3<R>& s3a, V3<R> s4a, V3<R>& s1b, V3<R>& s2b, V3<R>& s3b,
                V3<R> s4b) {  // 200-221
        const V3<R> v4v0 = cross(v4, v0);
        R d = dot(v1, v4v0);
        if (decide(d > R(0))) {
            d = dot(v2, v4v0);
            if (decide(d > R(0))) { v1 = v4; s1a = s4a; s1b = s4b; }
            else { v3 = v4; s3a = s4a; s3b = s4b; }
        } else {
            d = dot(v3, v4v0);
            if (decide(d > R(0))) { v2 = v4; s2a = s4a; s2b = s4b; }
            else { v1 = v4; s1a = s4a; s1b = s4b; }
        }
    }
    V3<R> find_pos(V3<R> v0, V3<R> v1, V3<R> v2, V3<R> v3, V3<R> s0a, V3<R> s1a, V3<R> s2a,
                   V3<R> s3a, V3<R> s0b, V3<R> s1b, V3<R> s2b, V3<R> s3b) {  // 224-247
        R b0 = dot(cross(v1, v2), v3);
        R b1 = -dot(cross(v0, v2), v3);
        R b2 = dot(cross(v0, v1), v3);
        R b3 = -dot(cross(v0, v1), v2);
        R sum = b0 + b1 + b2 + b3;
        if (decide(std::fabs(sum) < eps())) {
            const V3<R> dir = portal_dir(v1, v2, v3);
            b0 = R(0);
            b1 = dot(cross(v2, v3), dir);
            b2 = dot(cross(v3, v1), dir);
            b3 = dot(cross(v1, v2), dir);
            sum = b0 + b1 + b2 + b3;
        }
        const V3<R> p1 = b0 * s0a + b1 * s1a + b2 * s2a + b3 * s3a;
        const V3<R> p2 = b0 * s0b + b1 * s1b + b2 * s2b + b3 * s3b;
        return (R(0.5) / sum) * (p1 + p2);
    }
    int discover(uint32_t a, uint32_t b, V3<R>& v0, V3<R>& v1, V3<R>& v2, V3<R>& v3, V3<R>& s0a,
                 V3<R>& s1a, V3<R>& s2a, V3<R>& s3a, V3<R>& s0b, V3<R>& s1b, V3<R>& s2b,
                 V3<R>& s3b) {  // 250-320
        s0a = get3(pos, a);
        s0b = get3(pos, b);
        v0 = s0a - s0b;
        if (decide(std::fabs(v0.x) < eps() && std::fabs(v0.y) < eps() && std::fabs(v0.z) < eps()))
            v0.x += R(10) * eps();
        V3<R> dir = normalize(-v0);
        mink(a, b, dir, v1, s1a, s1b);
        R d = dot(v1, dir);
        if (decide(d < eps())) return -1;
        dir = cross(v0, v1);
        if (decide(dot(dir, dir) < eps())) {
            if (decide(std::fabs(v1.x) < eps() && std::fabs(v1.y) < eps() && std::fabs(v1.z) < eps()))
                return 1;
            return 2;
        }
        dir = normalize(dir);
        mink(a, b, dir, v2, s2a, s2b);
        d = dot(v2, dir);
        if (decide(d < eps())) return -1;
        V3<R> va = v1 - v0, vb = v2 - v0;
        dir = normalize(cross(va, vb));
        if (decide(dot(dir, v0) > R(0))) {
            std::swap(v1, v2);
            std::swap(s1a, s2a);
            std::swap(s1b, s2b);
            dir = -dir;
        }
        uint32_t trials = 0;
        while (trials < P.discover_trials) {
            V3<R> v3c, s3ca, s3cb;
            mink(a, b, dir, v3c, s3ca, s3cb);
            d = dot(v3c, dir);
            if (decide(d < eps())) return -1;
            va = cross(v1, v3c);
            d = dot(va, v0);
            if (decide(d < -eps())) {
                v2 = v3c; s2a = s3ca; s2b = s3cb;
                va = v1 - v0; vb = v2 - v0;
                dir = normalize(cross(va, vb));
                trials++;
                continue;
            }
            va = cross(v3c, v2);
            d = dot(va, v0);
            if (decide(d < -eps())) {
                v1 = v3c; s1a = s3ca; s1b = s3cb;
                va = v1 - v0; vb = v2 - v0;
                dir = normalize(cross(va, vb));
                trials++;
                continue;
            }
            v3 = v3c; s3a = s3ca; s3b = s3cb;
            return 0;
        }
        return -1;
    }
    bool mpr(uint32_t a, uint32_t b, V3<R>& normal, R& depth, V3<R>& cp) {  // 368-399
        ops.mpr_calls++;
        V3<R> v0{}, v1{}, v2{}, v3{}, s0a{}, s1a{}, s2a{}, s3a{}, s0b{}, s1b{}, s2b{}, s3b{};
        int res = discover(a, b, v0, v1, v2, v3, s0a, s1a, s2a, s3a, s0b, s1b, s2b, s3b);
        if (res == 1) {
            normal = normalize(v0);
            depth = R(0);
            cp = R(0.5) * (s1a + s1b);
            return true;
        }
        if (res == 2) {
            depth = length(v1);
            normal = normalize(v1);
            cp = R(0.5) * (s1a + s1b);
            return true;
        }
        if (res != 0) return false;
        // refine (323-343)
        res = 1;
        for (uint32_t it = 0; it < P.mpr_iterations; ++it) {
            const V3<R> dir = portal_dir(v1, v2, v3);
            if (decide(dot(v1, dir) > -eps())) { res = 0; break; }
            V3<R> v4, s4a, s4b;
            mink(a, b, dir, v4, s4a, s4b);
            if (decide(!(dot(v4, dir) > -eps()) || reach_tol(v1, v2, v3, v4, dir))) { res = -1; break; }
            expand(v0, v1, v2, v3, v4, s1a, s2a, s3a, s4a, s1b, s2b, s3b, s4b);
        }
        if (res < 0) return false;
        // penetration (346-365)
        bool found = false;
        for (uint32_t it = 0; it < P.mpr_iterations; ++it) {
            const V3<R> dir = portal_dir(v1, v2, v3);
            V3<R> v4, s4a, s4b;
            mink(a, b, dir, v4, s4a, s4b);
            if (decide(reach_tol(v1, v2, v3, v4, dir) || it >= P.mpr_iterations - 1)) {
                depth = dot(dir, v1);
                normal = dir;
                found = true;
                break;
            }
            expand(v0, v1, v2, v3, v4, s1a, s2a, s3a, s4a, s1b, s2b, s3b, s4b);
        }
        if (found) cp = find_pos(v0, v1, v2, v3, s0a, s1a, s2a, s3a, s0b, s1b, s2b, s3b);
        return found;
    }


    // ---- GJK + EPA (no counterpart in the reference, whose narrowphase is
    // MPR only; the alternative narrowphase of seevr_params.narrowphase) ----
    // Gilbert-Johnson-Keerthi finds a tetrahedron of Minkowski points (A-B
    // support points) enclosing the origin; the expanding polytope algorithm
    // then grows it toward the boundary of A-B until the face closest to the
    // origin is within tolerance of the boundary: its normal and distance
    // are the contact normal and depth, and the barycentric coordinates of
    // the origin's projection on it weight the witness points into the
    // contact point.  Same contract as mpr(): normal n (A is pushed along -n),
    // depth, contact point.
    struct SPt {
        V3<R> v, sa, sb;
    };
    static constexpr uint32_t kGjkIters = 64, kEpaIters = 64, kEpaMaxV = 32, kEpaMaxF = 64,
                              kEpaMaxE = 96;
    // Reduce the simplex s[0..n) (newest last) toward the origin; returns
    // true when a tetrahedron encloses it.  d: the next search direction.
    bool gjk_line(SPt* s, uint32_t& n, V3<R>& d) {
        const V3<R> a = s[n - 1].v, b = s[n - 2].v;
        const V3<R> ab = b - a, ao = -a;
        if (dot(ab, ao) > R(0)) {
            s[0] = s[n - 2];
            s[1] = s[n - 1];
            n = 2;
            d = cross(cross(ab, ao), ab);
        } else {
            s[0] = s[n - 1];
            n = 1;
            d = ao;
        }
        return false;
    }
    bool gjk_triangle(SPt* s, uint32_t& n, V3<R>& d) {  // s = [c, b, a]
        const V3<R> a = s[2].v, b = s[1].v, c = s[0].v;
        const V3<R> ab = b - a, ac = c - a, ao = -a;
        const V3<R> abc = cross(ab, ac);
        if (dot(cross(abc, ac), ao) > R(0)) {
            if (dot(ac, ao) > R(0)) {
                s[1] = s[2];  // [c, a]
                n = 2;
                d = cross(cross(ac, ao), ac);
                return false;
            }
            s[0] = s[1];  // [b, a]
            s[1] = s[2];
            n = 2;
            return gjk_line(s, n, d);
        }
        if (dot(cross(ab, abc), ao) > R(0)) {
            s[0] = s[1];  // [b, a]
            s[1] = s[2];
            n = 2;
            return gjk_line(s, n, d);
        }
        if (dot(abc, ao) > R(0)) {
            d = abc;
        } else {
            const SPt t = s[0];  // [b, c, a]
            s[0] = s[1];
            s[1] = t;
            d = -abc;
        }
        return false;
    }
    bool gjk_tetra(SPt* s, uint32_t& n, V3<R>& d) {  // s = [d, c, b, a]
        const V3<R> a = s[3].v, b = s[2].v, c = s[1].v, dd = s[0].v;
        const V3<R> ab = b - a, ac = c - a, ad = dd - a, ao = -a;
        if (dot(cross(ab, ac), ao) > R(0)) {  // outside face abc: [c, b, a]
            s[0] = s[1];
            s[1] = s[2];
            s[2] = s[3];
            n = 3;
            return gjk_triangle(s, n, d);
        }
        if (dot(cross(ac, ad), ao) > R(0)) {  // outside face acd: [d, c, a]
            s[2] = s[3];
            n = 3;
            return gjk_triangle(s, n, d);
        }
        if (dot(cross(ad, ab), ao) > R(0)) {  // outside face adb: [b, d, a]
            const SPt t = s[0];
            s[0] = s[2];
            s[1] = t;
            s[2] = s[3];
            n = 3;
            return gjk_triangle(s, n, d);
        }
        return true;
    }
    bool gjk(uint32_t a, uint32_t b, SPt* s) {
        const R e2 = eps() * eps();
        V3<R> d = get3(pos, a) - get3(pos, b);
        if (dot(d, d) < e2) d = v3(R(1), R(0), R(0));
        mink(a, b, d, s[0].v, s[0].sa, s[0].sb);
        uint32_t n = 1;
        d = -s[0].v;
        for (uint32_t it = 0; it < kGjkIters; ++it) {
            if (dot(d, d) < e2) return false;  // the origin lies on the simplex: touching
            SPt p;
            mink(a, b, d, p.v, p.sa, p.sb);
            if (dot(p.v, d) <= R(0)) return false;  // A-B does not reach past the origin
            s[n++] = p;
            const bool in = n == 2   ? gjk_line(s, n, d)
                            : n == 3 ? gjk_triangle(s, n, d)
                                     : gjk_tetra(s, n, d);
            if (in) return true;
        }
        return false;
    }
    struct Face {
        uint32_t i, j, k;
        V3<R> n;
        R dist;
    };
    Face make_face(const SPt* v, uint32_t i, uint32_t j, uint32_t k) const {
        Face f{i, j, k, v3(R(0), R(0), R(0)), R(1e30)};
        const V3<R> n = cross(v[j].v - v[i].v, v[k].v - v[i].v);
        const R l = length(n);
        if (l > R(0)) {
            f.n = divs(n, l);
            f.dist = dot(f.n, v[i].v);
        }
        return f;
    }
    bool gjk_epa(uint32_t a, uint32_t b, V3<R>& normal, R& depth, V3<R>& cp) {
        SPt v[kEpaMaxV];
        if (!gjk(a, b, v)) return false;
        uint32_t nv = 4, nf = 0;
        Face f[kEpaMaxF];
        const uint32_t tri[4][4] = {{3, 2, 1, 0}, {3, 1, 0, 2}, {3, 0, 2, 1}, {2, 0, 1, 3}};
        for (uint32_t t = 0; t < 4; ++t) {
            Face g = make_face(v, tri[t][0], tri[t][1], tri[t][2]);
            if (dot(g.n, v[tri[t][3]].v - v[tri[t][0]].v) > R(0)) {  // the fourth point in front
                g = make_face(v, tri[t][0], tri[t][2], tri[t][1]);
            }
            f[nf++] = g;
        }
        Face g{};
        for (uint32_t it = 0;; ++it) {
            uint32_t best = 0;  // the closest face (the first of equals)
            for (uint32_t i = 1; i < nf; ++i)
                if (f[i].dist < f[best].dist) best = i;
            g = f[best];
            if (it >= kEpaIters || nv == kEpaMaxV) break;
            SPt p;
            mink(a, b, g.n, p.v, p.sa, p.sb);
            const R dp = dot(p.v, g.n);
            if (dp - g.dist < R(P.tol) + eps() * gmax(R(1), dp)) break;
            // faces the new point sees are removed; their unshared edges
            // (the horizon) are joined to it
            uint32_t e[kEpaMaxE][2], ne = 0;
            bool full = false;
            uint32_t keep = 0;
            for (uint32_t i = 0; i < nf; ++i) {
                if (dot(f[i].n, p.v - v[f[i].i].v) > R(0)) {
                    const uint32_t ed[3][2] = {{f[i].i, f[i].j}, {f[i].j, f[i].k}, {f[i].k, f[i].i}};
                    for (uint32_t q = 0; q < 3; ++q) {
                        uint32_t r = 0;
                        while (r < ne && !(e[r][0] == ed[q][1] && e[r][1] == ed[q][0])) ++r;
                        if (r < ne) {  // shared with another removed face
                            for (uint32_t t = r; t + 1 < ne; ++t) {
                                e[t][0] = e[t + 1][0];
                                e[t][1] = e[t + 1][1];
                            }
                            --ne;
                        } else if (ne < kEpaMaxE) {
                            e[ne][0] = ed[q][0];
                            e[ne][1] = ed[q][1];
                            ++ne;
                        } else {
                            full = true;
                        }
                    }
                } else {
                    f[keep++] = f[i];
                }
            }
            if (full || keep + ne > kEpaMaxF) break;  // out of room: the last closest face
            nf = keep;
            v[nv] = p;
            for (uint32_t r = 0; r < ne; ++r) f[nf++] = make_face(v, e[r][0], e[r][1], nv);
            ++nv;
        }
        if (!(g.dist < R(1e30))) return false;  // no face with a normal
        normal = g.n;
        depth = g.dist;
        // barycentric coordinates of the origin's projection g.n * g.dist
        const V3<R> A = v[g.i].v, B = v[g.j].v, C = v[g.k].v;
        const V3<R> e0 = B - A, e1 = C - A, e2 = g.dist * g.n - A;
        const R d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1);
        const R d20 = dot(e2, e0), d21 = dot(e2, e1);
        const R den = d00 * d11 - d01 * d01;
        R wb = R(1) / R(3), wc = R(1) / R(3);
        if (std::fabs(den) > eps() * eps()) {
            wb = (d11 * d20 - d01 * d21) / den;
            wc = (d00 * d21 - d01 * d20) / den;
        }
        const R wa = R(1) - wb - wc;
        const V3<R> pa = wa * v[g.i].sa + wb * v[g.j].sa + wc * v[g.k].sa;
        const V3<R> pb = wa * v[g.i].sb + wb * v[g.j].sb + wc * v[g.k].sb;
        cp = R(0.5) * (pa + pb);
        return true;
    }

    // ---- steps ----
    void step_gravity(R dt, const R g[3]) {  // physics.comp:418-428
        const R ld = R(P.lin_damp), ad = R(P.ang_damp);
        for (uint32_t i = 0; i < nb; ++i) {
            if (inv_mass[i] <= R(0)) continue;
            for (int k = 0; k < 3; ++k) vel[i * 3 + k] = vel[i * 3 + k] * ld + g[k] * dt;
            for (int k = 0; k < 3; ++k) omega[i * 3 + k] *= ad;
        }
    }
    // AABB cascade (physics.comp:686-844): min/max over each body's hull
    // vertices, the owner of hull vertex gid being the last body whose
    // hull_start <= gid (binary search, physics.comp:695-703).
    void step_aabb() {
        const R big = R(1e30);
        std::vector<V3<R>> mn(nb, v3(big, big, big)), mx(nb, v3(-big, -big, -big));
        std::vector<char> seen(nb, 0);
        for (uint32_t gid = 0; gid < nhv; ++gid) {
            uint32_t lo = 0, hi = nb;
            while (lo + 1 < hi) {
                const uint32_t mid = (lo + hi) / 2;
                if (hull_start[mid] <= gid) lo = mid;
                else hi = mid;
            }
            const uint32_t b = lo;
            const V3<R> wv = get3(pos, b) + mul(quat_to_mat(b), get3(hull, gid));
            if (!seen[b]) {
                mn[b] = wv;
                mx[b] = wv;
                seen[b] = 1;
            } else {
                mn[b] = vmin(mn[b], wv);
                mx[b] = vmax(mx[b], wv);
            }
            ops.aabb_verts++;
        }
        for (uint32_t b = 0; b < nb; ++b)
            if (seen[b]) {
                set3(aabb_min, b, mn[b]);
                set3(aabb_max, b, mx[b]);
            }
    }
    // physics.comp:451-472, rows in order, j ascending (canonical order);
    // pairs never cross scenes.
    void step_broad() {
        pairs.clear();
        pairs_total = 0;
        for (uint32_t i = 0; i < nb; ++i) {
            const V3<R> mna = get3(aabb_min, i), mxa = get3(aabb_max, i);
            const uint32_t end = scene_end[scene_of[i]];
            for (uint32_t j = i + 1; j < end; ++j) {
                ops.broad_tests++;
                if (inv_mass[i] <= R(0) && inv_mass[j] <= R(0)) continue;
                const V3<R> mnb = get3(aabb_min, j), mxb = get3(aabb_max, j);
                if (decide(!(mxa.x < mnb.x || mxb.x < mna.x || mxa.y < mnb.y || mxb.y < mna.y ||
                             mxa.z < mnb.z || mxb.z < mna.z))) {
                    if (pairs_total < P.max_pairs) {
                        pairs.push_back(i);
                        pairs.push_back(j);
                    }
                    pairs_total++;
                }
            }
        }
    }
    void step_narrow() {  // physics.comp:475-491 + add_contact 403-412
        c_pos.clear(); c_normal.clear(); c_pen.clear(); c_a.clear(); c_b.clear();
        contacts_total = 0;
        const uint32_t np = std::min(pairs_total, P.max_pairs);
        for (uint32_t pi = 0; pi < np; ++pi) {
            const uint32_t a = pairs[pi * 2], b = pairs[pi * 2 + 1];
            V3<R> n{}, cp{};
            R depth = R(0);
            const bool found = P.narrowphase == 1 ? gjk_epa(a, b, n, depth, cp)
                                                  : mpr(a, b, n, depth, cp);
            const bool hit = decide(found && depth > R(0));
            mix(a, (uint64_t(b - a) << 8) ^ (hit ? 0x5Aull : 0ull));
            if (hit) {
                if (contacts_total < P.max_contacts) {
                    c_pos.insert(c_pos.end(), {cp.x, cp.y, cp.z});
                    c_normal.insert(c_normal.end(), {n.x, n.y, n.z});
                    c_pen.push_back(depth);
                    c_a.push_back(a);
                    c_b.push_back(b);
                }
                contacts_total++;
            }
        }
    }
    void step_clear() { std::fill(lambda.begin(), lambda.end(), R(0)); }  // 494-497
    void step_solve(R dt) {  // physics.comp:500-583
        const uint32_t nc = std::min(contacts_total, P.max_contacts);
        const R baum = R(P.baumgarte), slop = R(P.slop);
        std::vector<R> bias(nc);
        for (uint32_t ci = 0; ci < nc; ++ci) {
            const uint32_t ga = c_a[ci], gb = c_b[ci];
            const uint32_t a = geom_body[ga], b = geom_body[gb];
            const V3<R> n = get3(c_normal, ci), cp = get3(c_pos, ci);
            const V3<R> ra = cp - get3(pos, a), rb = cp - get3(pos, b);
            const V3<R> va = get3(vel, a) + cross(get3(omega, a), ra);
            const V3<R> vb = get3(vel, b) + cross(get3(omega, b), rb);
            const R vn = dot(vb - va, n);
            const R pen = c_pen[ci];
            const R e = gmax(restitution[ga], restitution[gb]);
            const R over = decide(pen - slop < R(0)) ? R(0) : pen - slop;  // gmax(pen - slop, 0)
            const R sep = decide(-vn < R(0)) ? R(0) : -vn;                  // gmax(-vn, 0)
            bias[ci] = baum * over / dt + e * sep;
        }
        for (uint32_t it = 0; it < P.pgs_iterations; ++it) {
            for (uint32_t ci = 0; ci < nc; ++ci) {
                const uint32_t ga = c_a[ci], gb = c_b[ci];
                const uint32_t a = geom_body[ga], b = geom_body[gb];
                const R ima = inv_mass[a], imb = inv_mass[b];
                if (ima == R(0) && imb == R(0)) continue;
                ops.pgs_contact_iters++;
                const V3<R> n = get3(c_normal, ci), cp = get3(c_pos, ci);
                const V3<R> ra = cp - get3(pos, a), rb = cp - get3(pos, b);
                V3<R> va = get3(vel, a) + cross(get3(omega, a), ra);
                V3<R> vb = get3(vel, b) + cross(get3(omega, b), rb);
                const R vn = dot(vb - va, n);
                const V3<R> ran = cross(ra, n), rbn = cross(rb, n);
                const R k = ima + imb + dot(ran, apply_inv_I(a, ran)) + dot(rbn, apply_inv_I(b, rbn));
                R d_ln = (-vn + bias[ci]) / k;
                const R old_ln = lambda[ci];
                const R new_ln = decide(old_ln + d_ln < R(0)) ? R(0) : old_ln + d_ln;  // gmax(., 0)
                d_ln = new_ln - old_ln;
                lambda[ci] = new_ln;
                const V3<R> imp = d_ln * n;
                set3(vel, a, get3(vel, a) - ima * imp);
                set3(vel, b, get3(vel, b) + imb * imp);
                set3(omega, a, get3(omega, a) - apply_inv_I(a, cross(ra, imp)));
                set3(omega, b, get3(omega, b) + apply_inv_I(b, cross(rb, imp)));
                const R mu = std::sqrt(friction[ga] * friction[gb]);
                va = get3(vel, a) + cross(get3(omega, a), ra);
                vb = get3(vel, b) + cross(get3(omega, b), rb);
                const V3<R> dv = vb - va;
                const V3<R> vt = dv - dot(dv, n) * n;
                const R vt_len = length(vt);
                if (decide(vt_len > R(1e-6))) {
                    ops.pgs_friction_iters++;
                    const V3<R> td = divs(vt, vt_len);
                    const V3<R> rat = cross(ra, td), rbt = cross(rb, td);
                    const R kt = ima + imb + dot(rat, apply_inv_I(a, rat)) + dot(rbt, apply_inv_I(b, rbt));
                    const R q1 = vt_len / kt, q2 = mu * lambda[ci];
                    const R d_lt = decide(q2 < q1) ? q2 : q1;  // gmin(q1, q2)
                    const V3<R> imp_t = d_lt * td;
                    set3(vel, a, get3(vel, a) + ima * imp_t);
                    set3(vel, b, get3(vel, b) - imb * imp_t);
                    set3(omega, a, get3(omega, a) + apply_inv_I(a, cross(ra, imp_t)));
                    set3(omega, b, get3(omega, b) - apply_inv_I(b, cross(rb, imp_t)));
                }
            }
        }
    }
    void step_integrate(R dt) {  // physics.comp:586-604
        for (uint32_t i = 0; i < nb; ++i) {
            if (inv_mass[i] <= R(0)) continue;
            for (int k = 0; k < 3; ++k) pos[i * 3 + k] += vel[i * 3 + k] * dt;
            const R ox = omega[i * 3], oy = omega[i * 3 + 1], oz = omega[i * 3 + 2];
            R qx = quat[i * 4], qy = quat[i * 4 + 1], qz = quat[i * 4 + 2], qw = quat[i * 4 + 3];
            const R dx = ox * qw + oy * qz - oz * qy;
            const R dy = -ox * qz + oy * qw + oz * qx;
            const R dz = ox * qy - oy * qx + oz * qw;
            const R dw = -ox * qx - oy * qy - oz * qz;
            const R h(0.5);
            qx += h * dx * dt;
            qy += h * dy * dt;
            qz += h * dz * dt;
            qw += h * dw * dt;
            const R l = std::sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
            if (decide(l > R(1e-8))) {
                qx /= l;
                qy /= l;
                qz /= l;
                qw /= l;
            }
            quat[i * 4] = qx;
            quat[i * 4 + 1] = qy;
            quat[i * 4 + 2] = qz;
            quat[i * 4 + 3] = qw;
        }
    }
    void step_update_verts() {  // physics.comp:607-627
        for (uint32_t vid = 0; vid < nv; ++vid) {
            uint32_t lo = 0, hi = nb;
            while (lo + 1 < hi) {
                const uint32_t mid = (lo + hi) / 2;
                if (vert_start[mid] <= vid) lo = mid;
                else hi = mid;
            }
            const V3<R> wp = get3(pos, lo) + mul(quat_to_mat(lo), get3(orig, vid));
            set3(verts, vid, wp);
        }
    }

    // Physics.step (physics.zig:80-165): dispatch order 8,0,9..11,2,3,4,5,6
    // per substep, then 7 once.
    void step(uint32_t substeps, R dt, const R g[3], bool update_verts = true) {
        if (nb == 0 || substeps == 0) return;  // physics.zig:81
        const R sub_dt = dt / R(substeps);      // physics.zig:90
        for (uint32_t s = 0; s < substeps; ++s) {
            pairs_total = contacts_total = 0;  // step 8
            step_gravity(sub_dt, g);          // step 0
            step_aabb();                      // steps 9, 10, 11
            step_broad();                     // step 2
            step_narrow();                    // step 3
            step_clear();                     // step 4
            step_solve(sub_dt);               // step 5
            step_integrate(sub_dt);           // step 6
            ops.bodies += nb;
        }
        if (update_verts) step_update_verts();  // step 7
    }
};

// ---- LBVH spec (bvh.comp) ----
// expand_bits / morton3d (bvh.comp:32-46)
inline uint32_t expand_bits(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
inline uint32_t quantize10(float x) {
    float t = x * 1024.0f;
    t = t < 0.f ? 0.f : (t > 1023.f ? 1023.f : t);  // clamp(x*1024, 0, 1023)
    return uint32_t(t);
}
inline uint32_t morton3d(float x, float y, float z) {
    return (expand_bits(quantize10(x)) << 2) | (expand_bits(quantize10(y)) << 1) |
           expand_bits(quantize10(z));
}
inline int clz32(uint32_t x) {  // bvh.comp:48-57
    if (x == 0u) return 32;
    int n = 0;
    if ((x & 0xFFFF0000u) == 0u) { n += 16; x <<= 16; }
    if ((x & 0xFF000000u) == 0u) { n += 8; x <<= 8; }
    if ((x & 0xF0000000u) == 0u) { n += 4; x <<= 4; }
    if ((x & 0xC0000000u) == 0u) { n += 2; x <<= 2; }
    if ((x & 0x80000000u) == 0u) { n += 1; }
    return n;
}

// Morton codes of centroids normalised by their bounds (bvh.comp:101-183).
inline void morton_codes(const float* c, uint32_t n, uint32_t* out, float bounds[6]) {
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = gmin(mn[k], c[i * 3 + k]);
            mx[k] = gmax(mx[k], c[i * 3 + k]);
        }
    float inv[3];
    for (int k = 0; k < 3; ++k) {
        const float ext = mx[k] - mn[k];
        inv[k] = ext > 1e-6f ? 1.0f / ext : 0.0f;
        bounds[k] = mn[k];
        bounds[k + 3] = mx[k];
    }
    for (uint32_t i = 0; i < n; ++i)
        out[i] = morton3d((c[i * 3] - mn[0]) * inv[0], (c[i * 3 + 1] - mn[1]) * inv[1],
                          (c[i * 3 + 2] - mn[2]) * inv[2]);
}

// 4-bit LSD radix sort, 8 passes, per-256 group histograms laid out
// digit-major and scanned globally (bvh.comp:192-295, bvh.zig:85-89).
inline void radix_sort_lsd4(std::vector<uint32_t>& key, std::vector<uint32_t>& idx) {
    const uint32_t n = uint32_t(key.size());
    const uint32_t groups = (n + 255) / 256;
    std::vector<uint32_t> hist(size_t(16) * groups), k2(n), i2(n);
    for (uint32_t shift = 0; shift < 32; shift += 4) {
        std::fill(hist.begin(), hist.end(), 0u);
        for (uint32_t g = 0; g < n; ++g) hist[((key[g] >> shift) & 0xF) * groups + g / 256]++;
        uint32_t run = 0;
        for (auto& h : hist) {
            const uint32_t v = h;
            h = run;
            run += v;
        }
        for (uint32_t g = 0; g < n; ++g) {
            const uint32_t d = (key[g] >> shift) & 0xF;
            const uint32_t dest = hist[d * groups + g / 256]++;
            k2[dest] = key[g];
            i2[dest] = idx[g];
        }
        key.swap(k2);
        idx.swap(i2);
    }
}

// Karras 2012 hierarchy over sorted codes (bvh.comp:59-65, 299-348).
// Internal nodes 0..n-2, leaves n-1..2n-2; parent[0] = 0xFFFFFFFF.
inline void karras(const std::vector<uint32_t>& m, std::vector<uint32_t>& left,
                   std::vector<uint32_t>& right, std::vector<uint32_t>& parent) {
    const int n = int(m.size());
    left.assign(size_t(2 * n - 1), 0);
    right.assign(size_t(2 * n - 1), 0);
    parent.assign(size_t(2 * n - 1), 0);
    auto delta = [&](int i, int j) -> int {
        if (j < 0 || j >= n) return -1;
        if (m[i] == m[j]) return 32 + clz32(uint32_t(i) ^ uint32_t(j));
        return clz32(m[i] ^ m[j]);
    };
    for (int i = 0; i < n; ++i) left[size_t(n - 1 + i)] = uint32_t(i);
    for (int i = 0; i < n - 1; ++i) {
        const int d = delta(i, i + 1) > delta(i, i - 1) ? 1 : -1;
        const int dmin = delta(i, i - d);
        int lmax = 2;
        while (delta(i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (delta(i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int first = std::min(i, j), last = std::max(i, j);
        const int dn = delta(first, last);
        int split = first, stride = last - first;
        while (stride > 1) {
            stride = (stride + 1) / 2;
            const int mid = split + stride;
            if (mid < last && delta(first, mid) > dn) split = mid;
        }
        uint32_t lc = uint32_t(split), rc = uint32_t(split + 1);
        if (first == split) lc = uint32_t(split + n - 1);
        if (last == split + 1) rc = uint32_t(split + 1 + n - 1);
        left[size_t(i)] = lc;
        right[size_t(i)] = rc;
        parent[lc] = uint32_t(i);
        parent[rc] = uint32_t(i);
    }
    if (n > 0) parent[0] = 0xFFFFFFFFu;
}

}  // namespace oracle
