// narrowphase.cu — MPR narrowphase (step 3, physics.comp:475-491) with the
// support function (physics.comp:107-169) and Minkowski Portal Refinement
// (physics.comp:171-399), plus deterministic contact compaction.
//
// One thread per candidate pair.  Each body's rotation matrix, position,
// hull range and lookup offset are loaded once per pair and kept in
// registers (the reference recomputes quat_to_mat in every support call;
// the values are identical).  The contact found for pair p is staged at
// slot p; a scan over the found flags then writes contacts in pair order,
// where the reference appends with atomicAdd (physics.comp:404).
#include "common.cuh"

namespace seevr {

struct Shape {
    m3 R;
    f3 p;
    uint32_t vs, vc, lk;
};

__device__ __forceinline__ Shape load_shape(const World& w, uint32_t b) {
    Shape s;
    s.R = quat_to_mat(w.quat, b);
    s.p = ld3(w.pos, b);
    s.vs = w.hull_range[size_t(b) * 2];
    s.vc = w.hull_range[size_t(b) * 2 + 1];
    s.lk = w.sup_off[b];
    return s;
}

// support (physics.comp:107-162)
__device__ f3 support(const World& w, const Shape& s, f3 d) {
    const f3 ld = mulT(s.R, d);
    float best = -1e10f;
    f3 bv = mk(0.f, 0.f, 0.f);
    if (s.lk == 0) {
        for (uint32_t i = 0; i < s.vc; ++i) {
            const f3 v = ld3(w.hull, s.vs + i);
            const float dd = dot(v, ld);
            if (dd > best) {
                best = dd;
                bv = v;
            }
        }
        return add(s.p, mul(s.R, bv));
    }
    const float angles[3] = {seevr_atan2f(ld.z, ld.y), seevr_atan2f(ld.z, ld.x),
                             seevr_atan2f(ld.y, ld.x)};
#pragma unroll
    for (uint32_t ax = 0; ax < 3; ++ax) {
        float a = angles[ax];
        if (a < 0.0f) a += 6.2831853f;
        const float bin_f = a / 6.2831853f * 64.0f;
        const uint32_t b0 = uint32_t(bin_f) % 64u;
        const uint32_t b1 = (b0 + 1u) % 64u;
        const uint32_t* lut = w.sup_lut + s.lk + ax * 64u;
        const f3 v0 = ld3(w.hull, s.vs + lut[b0]);
        const float d0 = dot(v0, ld);
        if (d0 > best) {
            best = d0;
            bv = v0;
        }
        const f3 v1 = ld3(w.hull, s.vs + lut[b1]);
        const float d1 = dot(v1, ld);
        if (d1 > best) {
            best = d1;
            bv = v1;
        }
    }
    return add(s.p, mul(s.R, bv));
}

struct Mink {
    f3 v, sa, sb;
};
__device__ __forceinline__ Mink mink(const World& w, const Shape& A, const Shape& B, f3 d) {
    Mink m;
    m.sa = support(w, A, d);
    m.sb = support(w, B, neg(d));
    m.v = sub(m.sa, m.sb);
    return m;
}

__device__ __forceinline__ f3 portal_dir(f3 v1, f3 v2, f3 v3) {
    return normalize(cross(sub(v2, v1), sub(v3, v1)));
}
__device__ __forceinline__ bool reach_tol(const Consts& k, f3 v1, f3 v2, f3 v3, f3 v4, f3 dir) {
    const float dv1 = dot(v1, dir), dv2 = dot(v2, dir), dv3 = dot(v3, dir), dv4 = dot(v4, dir);
    const float dot1 = gmin(gmin(dv4 - dv1, dv4 - dv2), dv4 - dv3);
    return dot1 < k.tol + k.eps * gmax(1.0f, dot1);
}

// portal vertex i: Minkowski point v and the support points on A and B
struct Portal {
    Mink m[4];
};

// mpr_expand_portal (physics.comp:200-221)
__device__ __forceinline__ void expand(Portal& P, const Mink& m4) {
    const f3 v4v0 = cross(m4.v, P.m[0].v);
    float d = dot(P.m[1].v, v4v0);
    if (d > 0.0f) {
        d = dot(P.m[2].v, v4v0);
        if (d > 0.0f) P.m[1] = m4;
        else P.m[3] = m4;
    } else {
        d = dot(P.m[3].v, v4v0);
        if (d > 0.0f) P.m[2] = m4;
        else P.m[1] = m4;
    }
}

// mpr_find_pos (physics.comp:224-247)
__device__ f3 find_pos(const Consts& k, const Portal& P) {
    const f3 v0 = P.m[0].v, v1 = P.m[1].v, v2 = P.m[2].v, v3 = P.m[3].v;
    float b0 = dot(cross(v1, v2), v3);
    float b1 = -dot(cross(v0, v2), v3);
    float b2 = dot(cross(v0, v1), v3);
    float b3 = -dot(cross(v0, v1), v2);
    float sum = b0 + b1 + b2 + b3;
    if (fabsf(sum) < k.eps) {
        const f3 dir = portal_dir(v1, v2, v3);
        b0 = 0.0f;
        b1 = dot(cross(v2, v3), dir);
        b2 = dot(cross(v3, v1), dir);
        b3 = dot(cross(v1, v2), dir);
        sum = b0 + b1 + b2 + b3;
    }
    const f3 p1 = add(add(add(scale(b0, P.m[0].sa), scale(b1, P.m[1].sa)), scale(b2, P.m[2].sa)),
                      scale(b3, P.m[3].sa));
    const f3 p2 = add(add(add(scale(b0, P.m[0].sb), scale(b1, P.m[1].sb)), scale(b2, P.m[2].sb)),
                      scale(b3, P.m[3].sb));
    return scale(0.5f / sum, add(p1, p2));
}

// mpr (physics.comp:368-399) with discover (250-320), refine (323-343) and
// penetration (346-365).  Returns found; fills normal, depth, contact point.
__device__ bool mpr(const World& w, const Consts& k, uint32_t a, uint32_t b, f3& normal,
                    float& depth, f3& cp) {
    const Shape A = load_shape(w, a), B = load_shape(w, b);
    Portal P;
    // ---- discover portal ----
    P.m[0].sa = A.p;
    P.m[0].sb = B.p;
    P.m[0].v = sub(A.p, B.p);
    if (fabsf(P.m[0].v.x) < k.eps && fabsf(P.m[0].v.y) < k.eps && fabsf(P.m[0].v.z) < k.eps)
        P.m[0].v.x += 10.0f * k.eps;
    f3 dir = normalize(neg(P.m[0].v));
    P.m[1] = mink(w, A, B, dir);
    float d = dot(P.m[1].v, dir);
    if (d < k.eps) return false;
    dir = cross(P.m[0].v, P.m[1].v);
    if (dot(dir, dir) < k.eps) {
        const f3 v1 = P.m[1].v;
        if (fabsf(v1.x) < k.eps && fabsf(v1.y) < k.eps && fabsf(v1.z) < k.eps) {
            normal = normalize(P.m[0].v);  // res == 1
            depth = 0.0f;
        } else {
            depth = length(v1);  // res == 2
            normal = normalize(v1);
        }
        cp = scale(0.5f, add(P.m[1].sa, P.m[1].sb));
        return true;
    }
    dir = normalize(dir);
    P.m[2] = mink(w, A, B, dir);
    d = dot(P.m[2].v, dir);
    if (d < k.eps) return false;
    f3 va = sub(P.m[1].v, P.m[0].v), vb = sub(P.m[2].v, P.m[0].v);
    dir = normalize(cross(va, vb));
    if (dot(dir, P.m[0].v) > 0.0f) {
        const Mink t = P.m[1];
        P.m[1] = P.m[2];
        P.m[2] = t;
        dir = neg(dir);
    }
    bool discovered = false;
    for (uint32_t trials = 0; trials < k.discover_trials;) {
        const Mink c = mink(w, A, B, dir);
        d = dot(c.v, dir);
        if (d < k.eps) return false;
        va = cross(P.m[1].v, c.v);
        d = dot(va, P.m[0].v);
        if (d < -k.eps) {
            P.m[2] = c;
            va = sub(P.m[1].v, P.m[0].v);
            vb = sub(P.m[2].v, P.m[0].v);
            dir = normalize(cross(va, vb));
            ++trials;
            continue;
        }
        va = cross(c.v, P.m[2].v);
        d = dot(va, P.m[0].v);
        if (d < -k.eps) {
            P.m[1] = c;
            va = sub(P.m[1].v, P.m[0].v);
            vb = sub(P.m[2].v, P.m[0].v);
            dir = normalize(cross(va, vb));
            ++trials;
            continue;
        }
        P.m[3] = c;
        discovered = true;
        break;
    }
    if (!discovered) return false;
    // ---- refine portal ----
    bool inside = false;
    for (uint32_t it = 0; it < k.mpr_iterations; ++it) {
        const f3 pd = portal_dir(P.m[1].v, P.m[2].v, P.m[3].v);
        if (dot(P.m[1].v, pd) > -k.eps) {
            inside = true;
            break;
        }
        const Mink m4 = mink(w, A, B, pd);
        if (!(dot(m4.v, pd) > -k.eps) || reach_tol(k, P.m[1].v, P.m[2].v, P.m[3].v, m4.v, pd))
            return false;
        expand(P, m4);
    }
    // refine returning 1 (iterations exhausted) continues like 0
    (void)inside;
    // ---- find penetration ----
    for (uint32_t it = 0; it < k.mpr_iterations; ++it) {
        const f3 pd = portal_dir(P.m[1].v, P.m[2].v, P.m[3].v);
        const Mink m4 = mink(w, A, B, pd);
        if (reach_tol(k, P.m[1].v, P.m[2].v, P.m[3].v, m4.v, pd) || it >= k.mpr_iterations - 1) {
            depth = dot(pd, P.m[1].v);
            normal = pd;
            cp = find_pos(k, P);
            return true;
        }
        expand(P, m4);
    }
    return false;
}

__global__ void __launch_bounds__(128) k_narrow(World w, Consts k, float4* __restrict__ res0,
                                                float4* __restrict__ res1,
                                                uint32_t* __restrict__ flag) {
    const uint32_t np = min(w.counters[0], w.max_pairs);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        const uint32_t a = w.pairs[size_t(p) * 2], b = w.pairs[size_t(p) * 2 + 1];
        f3 n = mk(0, 0, 0), cp = mk(0, 0, 0);
        float depth = 0.0f;
        const bool found = mpr(w, k, a, b, n, depth, cp);
        const bool keep = found && depth > 0.0f;
        flag[p] = keep ? 1u : 0u;
        if (keep) {
            res0[p] = make_float4(cp.x, cp.y, cp.z, depth);
            res1[p] = make_float4(n.x, n.y, n.z, 0.0f);
        }
    }
}

// add_contact (physics.comp:403-412) at the scanned slot.
__global__ void k_contact_scatter(World w, const float4* __restrict__ res0,
                                  const float4* __restrict__ res1,
                                  const uint32_t* __restrict__ flag,
                                  const uint32_t* __restrict__ coff) {
    const uint32_t np = min(w.counters[0], w.max_pairs);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        if (!flag[p]) continue;
        const uint32_t c = coff[p];
        if (c >= w.max_contacts) continue;
        const float4 r0 = res0[p], r1 = res1[p];
        st3(w.c_pos, c, mk(r0.x, r0.y, r0.z));
        st3(w.c_normal, c, mk(r1.x, r1.y, r1.z));
        w.c_pen[c] = r0.w;
        w.c_a[c] = w.pairs[size_t(p) * 2];
        w.c_b[c] = w.pairs[size_t(p) * 2 + 1];
    }
}

static uint32_t grid_for(uint32_t cap, uint32_t threads, uint32_t max_blocks) {
    uint32_t g = (cap + threads - 1) / threads;
    if (g > max_blocks) g = max_blocks;
    return g ? g : 1;
}

int launch_narrowphase(const World& w, const Consts& k, const Scratch& s, cudaStream_t st) {
    if (w.max_pairs == 0) return 0;
    k_narrow<<<grid_for(w.max_pairs, 128, 148 * 32), 128, 0, st>>>(w, k, s.pair_res0,
                                                                   s.pair_res1, s.pair_flag);
    launch_exclusive_scan(s.pair_flag, s.pair_coff, &w.counters[0], w.max_pairs,
                          &w.counters[1], w.max_contacts, kFlagContactOverflow, s, st);
    k_contact_scatter<<<grid_for(w.max_pairs, 256, 148 * 16), 256, 0, st>>>(
        w, s.pair_res0, s.pair_res1, s.pair_flag, s.pair_coff);
    return 3;
}

}  // namespace seevr
