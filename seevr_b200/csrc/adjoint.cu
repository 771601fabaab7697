// adjoint.cu — reverse mode of one physics substep, for gradients of a
// rollout with respect to initial velocities, angular velocities and
// friction coefficients.
//
// The substep is gravity (physics.comp:418-428), contacts from MPR
// (physics.comp:171-399, 475-491), the PGS solve (500-583) and integration
// (586-604).  Its adjoint, run once per substep in reverse order with the
// state restored from a checkpoint:
//   1. the contacts are recomputed by the regular kernels, the narrowphase
//      taping which hull vertices support each contact's final portal;
//   2. per solver bundle (one warp), the PGS sweep is recomputed in the
//      reference order, recording the inputs of every contact update;
//   3. integration, the PGS sweep (unrolled, reverse order), the contact
//      constants (effective mass, bias, friction coefficient, lever arms),
//      the contact normal, depth and point (as functions of the taped
//      support points), rotation matrices and gravity are differentiated by
//      hand, statement by statement.
// Contact selection (AABBs, broadphase, which pairs touch, MPR's discrete
// portal choices) and the clamps max(., 0), min(., .) and the friction test
// are piecewise constant: the adjoint follows the branches the forward took.
// The sequential parts run on lane 0 of the bundle's warp, so every sum is
// accumulated in a fixed order and the gradients are deterministic.
#include "adjoint.cuh"

namespace seevr {
namespace {

__device__ __forceinline__ f3 z3() { return mk(0.f, 0.f, 0.f); }
__device__ __forceinline__ void acc(f3& a, f3 b) { a = add(a, b); }
__device__ __forceinline__ void acc_s(f3& a, float s, f3 b) { a = add(a, scale(s, b)); }
__device__ __forceinline__ void add3(float* p, uint32_t i, f3 v) {
    p[size_t(i) * 3] += v.x;
    p[size_t(i) * 3 + 1] += v.y;
    p[size_t(i) * 3 + 2] += v.z;
}
__device__ __forceinline__ m3 m3zero() {
    m3 m;
    m.c0 = m.c1 = m.c2 = z3();
    return m;
}
__device__ __forceinline__ void add_m3(float* p, uint32_t i, const m3& g) {
    float* q = p + size_t(i) * 9;
    q[0] += g.c0.x; q[1] += g.c0.y; q[2] += g.c0.z;
    q[3] += g.c1.x; q[4] += g.c1.y; q[5] += g.c1.z;
    q[6] += g.c2.x; q[7] += g.c2.y; q[8] += g.c2.z;
}

// y = R (I ⊙ (Rᵀ x)) (apply_inv_I, physics.comp:90-94): accumulates dL/dR
// into gR (columns) and returns dL/dx (the map is symmetric in x).
__device__ __forceinline__ f3 inv_I_bwd(const m3& R, f3 I, f3 x, f3 gy, m3& gR) {
    const f3 w = mulT(R, x);
    const f3 u = hadamard(I, w);
    const f3 gw = hadamard(I, mulT(R, gy));
    gR.c0 = add(gR.c0, add(scale(u.x, gy), scale(gw.x, x)));
    gR.c1 = add(gR.c1, add(scale(u.y, gy), scale(gw.y, x)));
    gR.c2 = add(gR.c2, add(scale(u.z, gy), scale(gw.z, x)));
    return mul(R, gw);
}

// dL/d(x,y,z,w) of quat_to_mat (physics.comp:74-81) from dL/dR by columns
__device__ __forceinline__ void quat_bwd(float x, float y, float z, float w, const float* g,
                                         float out[4]) {
    out[0] = 2.f * (g[1] * y + g[2] * z + g[3] * y - 2.f * g[4] * x + g[5] * w + g[6] * z -
                    g[7] * w - 2.f * g[8] * x);
    out[1] = 2.f * (-2.f * g[0] * y + g[1] * x - g[2] * w + g[3] * x + g[5] * z + g[6] * w +
                    g[7] * z - 2.f * g[8] * y);
    out[2] = 2.f * (-2.f * g[0] * z + g[1] * w + g[2] * x - g[3] * w - 2.f * g[4] * z + g[5] * y +
                    g[6] * x + g[7] * y);
    out[3] = 2.f * (g[1] * z - g[2] * y - g[3] * z + g[5] * x + g[6] * y - g[7] * x);
}

struct Body {
    float ima;
    f3 I;
    m3 R;
    bool fixed;
};
__device__ __forceinline__ Body load_body(const World& w, uint32_t b) {
    Body o;
    o.ima = w.inv_mass[b];
    o.I = ld3(w.inv_inertia, b);
    o.R = quat_to_mat(w.quat, b);
    o.fixed = o.ima == 0.0f && o.I.x == 0.0f && o.I.y == 0.0f && o.I.z == 0.0f;
    return o;
}

struct CParams {
    f3 n, ra, rb;
    float bias, kn, mu;
};
struct CGrad {
    f3 n, ra, rb;
    float bias, kn, mu;
};
__device__ __forceinline__ CParams ld_par(const float* p, uint32_t c) {
    const float* q = p + size_t(c) * 12;
    return CParams{mk(q[0], q[1], q[2]), mk(q[3], q[4], q[5]), mk(q[6], q[7], q[8]), q[9], q[10],
                   q[11]};
}
__device__ __forceinline__ void st_par(float* p, uint32_t c, const CParams& v) {
    float* q = p + size_t(c) * 12;
    q[0] = v.n.x; q[1] = v.n.y; q[2] = v.n.z;
    q[3] = v.ra.x; q[4] = v.ra.y; q[5] = v.ra.z;
    q[6] = v.rb.x; q[7] = v.rb.y; q[8] = v.rb.z;
    q[9] = v.bias; q[10] = v.kn; q[11] = v.mu;
}
__device__ __forceinline__ CGrad ld_grad(const float* p, uint32_t c) {
    const float* q = p + size_t(c) * 12;
    return CGrad{mk(q[0], q[1], q[2]), mk(q[3], q[4], q[5]), mk(q[6], q[7], q[8]), q[9], q[10],
                 q[11]};
}
__device__ __forceinline__ void st_grad(float* p, uint32_t c, const CGrad& v) {
    float* q = p + size_t(c) * 12;
    q[0] = v.n.x; q[1] = v.n.y; q[2] = v.n.z;
    q[3] = v.ra.x; q[4] = v.ra.y; q[5] = v.ra.z;
    q[6] = v.rb.x; q[7] = v.rb.y; q[8] = v.rb.z;
    q[9] = v.bias; q[10] = v.kn; q[11] = v.mu;
}

// One contact update (physics.comp:525-580), the solver's arithmetic.
__device__ __forceinline__ void update_fwd(const Body& A, const Body& B, const CParams& c, f3& va,
                                          f3& wa, f3& vb, f3& wb, float& lam) {
    f3 ua = add(va, cross(wa, c.ra)), ub = add(vb, cross(wb, c.rb));
    const float vn = dot(sub(ub, ua), c.n);
    float d = (-vn + c.bias) / c.kn;
    const float nl = gmax(lam + d, 0.0f);
    d = nl - lam;
    lam = nl;
    const f3 imp = scale(d, c.n);
    f3 va1 = sub(va, scale(A.ima, imp)), vb1 = add(vb, scale(B.ima, imp));
    f3 wa1 = sub(wa, apply_inv_I(A.R, A.I, cross(c.ra, imp)));
    f3 wb1 = add(wb, apply_inv_I(B.R, B.I, cross(c.rb, imp)));
    ua = add(va1, cross(wa1, c.ra));
    ub = add(vb1, cross(wb1, c.rb));
    const f3 dv = sub(ub, ua);
    const f3 vt = sub(dv, scale(dot(dv, c.n), c.n));
    const float s = length(vt);
    if (s > 1e-6f) {
        const f3 td = divs(vt, s);
        const f3 rat = cross(c.ra, td), rbt = cross(c.rb, td);
        const float kt = A.ima + B.ima + dot(rat, apply_inv_I(A.R, A.I, rat)) +
                         dot(rbt, apply_inv_I(B.R, B.I, rbt));
        const float dt_ = gmin(s / kt, c.mu * nl);
        const f3 it = scale(dt_, td);
        va1 = add(va1, scale(A.ima, it));
        vb1 = sub(vb1, scale(B.ima, it));
        wa1 = add(wa1, apply_inv_I(A.R, A.I, cross(c.ra, it)));
        wb1 = sub(wb1, apply_inv_I(B.R, B.I, cross(c.rb, it)));
    }
    if (!A.fixed) {
        va = va1;
        wa = wa1;
    }
    if (!B.fixed) {
        vb = vb1;
        wb = wb1;
    }
}

// Reverse of update_fwd, from its inputs.  On entry G* hold dL/d(body state
// after the update) and glam dL/d(λ after); on return dL/d(before).
// Parameter gradients accumulate into gc, gRa, gRb.
__device__ void update_bwd(const Body& A, const Body& B, const CParams& c, f3 va, f3 wa, f3 vb,
                           f3 wb, float lam, f3& Gva, f3& Gwa, f3& Gvb, f3& Gwb, float& glam,
                           CGrad& gc, m3& gRa, m3& gRb) {
    // forward intermediates
    const f3 ua = add(va, cross(wa, c.ra)), ub = add(vb, cross(wb, c.rb));
    const f3 dvn = sub(ub, ua);
    const float vn = dot(dvn, c.n);
    const float d0 = (-vn + c.bias) / c.kn;
    const float s1 = lam + d0;
    const float l1 = gmax(s1, 0.0f);
    const float d = l1 - lam;
    const f3 imp = scale(d, c.n);
    const f3 va1 = sub(va, scale(A.ima, imp)), vb1 = add(vb, scale(B.ima, imp));
    const f3 xa = cross(c.ra, imp), xb = cross(c.rb, imp);
    const f3 wa1 = sub(wa, apply_inv_I(A.R, A.I, xa));
    const f3 wb1 = add(wb, apply_inv_I(B.R, B.I, xb));
    const f3 ua1 = add(va1, cross(wa1, c.ra)), ub1 = add(vb1, cross(wb1, c.rb));
    const f3 dv = sub(ub1, ua1);
    const float dn = dot(dv, c.n);
    const f3 vt = sub(dv, scale(dn, c.n));
    const float s = length(vt);
    // gradients of the outputs: a fixed body's outputs are discarded
    const f3 gva2 = A.fixed ? z3() : Gva, gwa2 = A.fixed ? z3() : Gwa;
    const f3 gvb2 = B.fixed ? z3() : Gvb, gwb2 = B.fixed ? z3() : Gwb;
    f3 gva1 = gva2, gwa1 = gwa2, gvb1 = gvb2, gwb1 = gwb2;
    float g_l1 = glam;
    f3 g_vt = z3();
    float g_s = 0.f;
    if (s > 1e-6f) {
        const f3 td = divs(vt, s);
        const f3 rat = cross(c.ra, td), rbt = cross(c.rb, td);
        const f3 pa = apply_inv_I(A.R, A.I, rat), pb = apply_inv_I(B.R, B.I, rbt);
        const float kt = A.ima + B.ima + dot(rat, pa) + dot(rbt, pb);
        const float q1 = s / kt, q2 = c.mu * l1;
        const bool take2 = q2 < q1;  // GLSL min(q1, q2)
        const float dt_ = take2 ? q2 : q1;
        const f3 it = scale(dt_, td);
        const f3 xa2 = cross(c.ra, it), xb2 = cross(c.rb, it);
        f3 g_it = z3();
        // wa2 = wa1 + A(xa2); wb2 = wb1 - A(xb2)
        const f3 g_xa2 = inv_I_bwd(A.R, A.I, xa2, gwa2, gRa);
        const f3 g_xb2 = inv_I_bwd(B.R, B.I, xb2, neg(gwb2), gRb);
        acc(gc.ra, cross(it, g_xa2));
        acc(g_it, cross(g_xa2, c.ra));
        acc(gc.rb, cross(it, g_xb2));
        acc(g_it, cross(g_xb2, c.rb));
        // va2 = va1 + ima it; vb2 = vb1 - imb it
        acc_s(g_it, A.ima, gva2);
        acc_s(g_it, -B.ima, gvb2);
        // it = dt_ td
        const float g_dt = dot(g_it, td);
        f3 g_td = scale(dt_, g_it);
        float g_kt = 0.f;
        if (take2) {
            gc.mu += g_dt * l1;
            g_l1 += g_dt * c.mu;
        } else {
            g_s += g_dt / kt;
            g_kt = -g_dt * s / (kt * kt);
        }
        // kt = ... + rat·A(rat) + rbt·A(rbt): d/drat = 2 A(rat)
        const f3 g_rat = scale(2.f * g_kt, pa), g_rbt = scale(2.f * g_kt, pb);
        inv_I_bwd(A.R, A.I, rat, scale(g_kt, rat), gRa);
        inv_I_bwd(B.R, B.I, rbt, scale(g_kt, rbt), gRb);
        // rat = ra x td
        acc(gc.ra, cross(td, g_rat));
        acc(g_td, cross(g_rat, c.ra));
        acc(gc.rb, cross(td, g_rbt));
        acc(g_td, cross(g_rbt, c.rb));
        // td = vt / s
        acc_s(g_vt, 1.f / s, g_td);
        g_s += -dot(g_td, vt) / (s * s);
    }
    if (s > 0.f) acc_s(g_vt, g_s / s, vt);
    // vt = dv - dn n; dn = dv·n
    f3 g_dv = g_vt;
    const float g_dn = -dot(g_vt, c.n);
    acc_s(gc.n, -dn, g_vt);
    acc_s(g_dv, g_dn, c.n);
    acc_s(gc.n, g_dn, dv);
    // dv = ub1 - ua1; ua1 = va1 + wa1 x ra
    const f3 g_ua1 = neg(g_dv), g_ub1 = g_dv;
    acc(gva1, g_ua1);
    acc(gwa1, cross(c.ra, g_ua1));
    acc(gc.ra, cross(g_ua1, wa1));
    acc(gvb1, g_ub1);
    acc(gwb1, cross(c.rb, g_ub1));
    acc(gc.rb, cross(g_ub1, wb1));
    // wa1 = wa - A(xa); wb1 = wb + A(xb); xa = ra x imp
    f3 gi_va = gva1, gi_wa = gwa1, gi_vb = gvb1, gi_wb = gwb1, g_imp = z3();
    const f3 g_xa = inv_I_bwd(A.R, A.I, xa, neg(gwa1), gRa);
    const f3 g_xb = inv_I_bwd(B.R, B.I, xb, gwb1, gRb);
    acc(gc.ra, cross(imp, g_xa));
    acc(g_imp, cross(g_xa, c.ra));
    acc(gc.rb, cross(imp, g_xb));
    acc(g_imp, cross(g_xb, c.rb));
    // va1 = va - ima imp; vb1 = vb + imb imp
    acc_s(g_imp, -A.ima, gva1);
    acc_s(g_imp, B.ima, gvb1);
    // imp = d n
    const float g_d = dot(g_imp, c.n);
    acc_s(gc.n, d, g_imp);
    // d = l1 - lam; l1 = max(s1, 0); s1 = lam + d0
    g_l1 += g_d;
    float gi_lam = -g_d;
    const float g_s1 = s1 < 0.f ? 0.f : g_l1;
    gi_lam += g_s1;
    // d0 = (-vn + bias) / kn
    const float g_vn = -g_s1 / c.kn;
    gc.bias += g_s1 / c.kn;
    gc.kn += -g_s1 * d0 / c.kn;
    // vn = dvn·n; dvn = ub - ua; ua = va + wa x ra
    acc_s(gc.n, g_vn, dvn);
    const f3 g_ub = scale(g_vn, c.n), g_ua = neg(g_ub);
    acc(gi_va, g_ua);
    acc(gi_wa, cross(c.ra, g_ua));
    acc(gc.ra, cross(g_ua, wa));
    acc(gi_vb, g_ub);
    acc(gi_wb, cross(c.rb, g_ub));
    acc(gc.rb, cross(g_ub, wb));
    // a fixed body's state persists: its incoming gradient passes through
    Gva = A.fixed ? add(Gva, gi_va) : gi_va;
    Gwa = A.fixed ? add(Gwa, gi_wa) : gi_wa;
    Gvb = B.fixed ? add(Gvb, gi_vb) : gi_vb;
    Gwb = B.fixed ? add(Gwb, gi_wb) : gi_wb;
    glam = gi_lam;
}

__device__ __forceinline__ f3 hull_vert(const World& w, uint32_t vs, uint32_t i) {
    return i == kNone ? z3() : ld3(w.hull, vs + i);
}

// dL/d (positions, rotations) of one contact's normal, depth and point,
// through the taped supporting vertices (physics.comp:224-247, 346-365,
// 376-387).
__device__ void contact_geom_bwd(const World& w, const Consts& k, const AdjScratch& a, uint32_t c,
                                 uint32_t ba, uint32_t bb, f3 g_n, float g_pen, f3 g_cp) {
    const uint4 t0 = a.ctape[size_t(c) * 2], t1 = a.ctape[size_t(c) * 2 + 1];
    const f3 pA = ld3(w.pos, ba), pB = ld3(w.pos, bb);
    const m3 RA = quat_to_mat(w.quat, ba), RB = quat_to_mat(w.quat, bb);
    const uint32_t vsA = w.hull_range[size_t(ba) * 2], vsB = w.hull_range[size_t(bb) * 2];
    f3 hA[4], hB[4], sa[4], sb[4], gsa[4], gsb[4], v[4], gv[4];
    const uint32_t ia[4] = {kNone, t0.y, t0.w, t1.y};
    const uint32_t ib[4] = {kNone, t0.z, t1.x, t1.z};
    for (int i = 0; i < 4; ++i) {
        hA[i] = hull_vert(w, vsA, ia[i]);
        hB[i] = hull_vert(w, vsB, ib[i]);
        sa[i] = add(pA, mul(RA, hA[i]));
        sb[i] = add(pB, mul(RB, hB[i]));
        v[i] = sub(sa[i], sb[i]);
        gsa[i] = gsb[i] = gv[i] = z3();
    }
    f3 gpA = z3(), gpB = z3();
    if (t0.x == 2u) {  // segment case: depth = |v1|, n = v1/|v1|, cp = (s1a + s1b)/2
        const float l = length(v[1]);
        const f3 n = divs(v[1], l);
        f3 g1 = scale(g_pen, n);
        acc_s(g1, 1.f / l, sub(g_n, scale(dot(n, g_n), n)));
        gsa[1] = add(scale(0.5f, g_cp), g1);
        gsb[1] = sub(scale(0.5f, g_cp), g1);
    } else {  // portal: n = normalize((v2-v1)x(v3-v1)), depth = n·v1, cp = find_pos
        f3 v0 = sub(pA, pB);
        if (fabsf(v0.x) < k.eps && fabsf(v0.y) < k.eps && fabsf(v0.z) < k.eps) v0.x += 10.0f * k.eps;
        v[0] = v0;
        sa[0] = pA;
        sb[0] = pB;
        const f3 e1 = sub(v[2], v[1]), e2 = sub(v[3], v[1]);
        const f3 cr = cross(e1, e2);
        const float cl = length(cr);
        const f3 n = divs(cr, cl);
        f3 g_nn = g_n;
        acc_s(g_nn, g_pen, v[1]);
        acc_s(gv[1], g_pen, n);
        // contact point
        float b[4];
        b[0] = dot(cross(v[1], v[2]), v[3]);
        b[1] = -dot(cross(v[0], v[2]), v[3]);
        b[2] = dot(cross(v[0], v[1]), v[3]);
        b[3] = -dot(cross(v[0], v[1]), v[2]);
        float sum = b[0] + b[1] + b[2] + b[3];
        const bool fallback = fabsf(sum) < k.eps;
        if (fallback) {
            b[0] = 0.f;
            b[1] = dot(cross(v[2], v[3]), n);
            b[2] = dot(cross(v[3], v[1]), n);
            b[3] = dot(cross(v[1], v[2]), n);
            sum = b[0] + b[1] + b[2] + b[3];
        }
        f3 P = z3();
        for (int i = 0; i < 4; ++i) P = add(P, scale(b[i], add(sa[i], sb[i])));
        const float kk = 0.5f / sum;
        const f3 gP = scale(kk, g_cp);
        const float g_sum = -0.5f / (sum * sum) * dot(g_cp, P);
        float gb[4];
        for (int i = 0; i < 4; ++i) {
            gb[i] = dot(gP, sa[i]) + dot(gP, sb[i]) + g_sum;
            acc_s(gsa[i], b[i], gP);
            acc_s(gsb[i], b[i], gP);
        }
        if (!fallback) {
            // triple products [a,b,c] = (a x b)·c: d/da = b x c, d/db = c x a, d/dc = a x b
            acc_s(gv[1], gb[0], cross(v[2], v[3]));
            acc_s(gv[2], gb[0], cross(v[3], v[1]));
            acc_s(gv[3], gb[0], cross(v[1], v[2]));
            acc_s(gv[0], -gb[1], cross(v[2], v[3]));
            acc_s(gv[2], -gb[1], cross(v[3], v[0]));
            acc_s(gv[3], -gb[1], cross(v[0], v[2]));
            acc_s(gv[0], gb[2], cross(v[1], v[3]));
            acc_s(gv[1], gb[2], cross(v[3], v[0]));
            acc_s(gv[3], gb[2], cross(v[0], v[1]));
            acc_s(gv[0], -gb[3], cross(v[1], v[2]));
            acc_s(gv[1], -gb[3], cross(v[2], v[0]));
            acc_s(gv[2], -gb[3], cross(v[0], v[1]));
        } else {
            // b1 = (v2 x v3)·n, b2 = (v3 x v1)·n, b3 = (v1 x v2)·n
            acc_s(gv[2], gb[1], cross(v[3], n));
            acc_s(gv[3], gb[1], cross(n, v[2]));
            acc_s(g_nn, gb[1], cross(v[2], v[3]));
            acc_s(gv[3], gb[2], cross(v[1], n));
            acc_s(gv[1], gb[2], cross(n, v[3]));
            acc_s(g_nn, gb[2], cross(v[3], v[1]));
            acc_s(gv[1], gb[3], cross(v[2], n));
            acc_s(gv[2], gb[3], cross(n, v[1]));
            acc_s(g_nn, gb[3], cross(v[1], v[2]));
        }
        // n = cr / |cr|; cr = e1 x e2
        const f3 g_cr = scale(1.f / cl, sub(g_nn, scale(dot(n, g_nn), n)));
        const f3 g_e1 = cross(e2, g_cr), g_e2 = cross(g_cr, e1);
        acc(gv[2], g_e1);
        acc(gv[3], g_e2);
        gv[1] = sub(gv[1], add(g_e1, g_e2));
        // v0 = pA - pB; s0a = pA; s0b = pB
        acc(gpA, add(gv[0], gsa[0]));
        acc(gpB, sub(gsb[0], gv[0]));
        for (int i = 1; i < 4; ++i) {
            acc(gsa[i], gv[i]);
            gsb[i] = sub(gsb[i], gv[i]);
        }
    }
    // s_ia = pA + RA h_ia; s_ib = pB + RB h_ib (i = 1..3)
    m3 gRA = m3zero(), gRB = m3zero();
    for (int i = 1; i < 4; ++i) {
        acc(gpA, gsa[i]);
        acc(gpB, gsb[i]);
        gRA.c0 = add(gRA.c0, scale(hA[i].x, gsa[i]));
        gRA.c1 = add(gRA.c1, scale(hA[i].y, gsa[i]));
        gRA.c2 = add(gRA.c2, scale(hA[i].z, gsa[i]));
        gRB.c0 = add(gRB.c0, scale(hB[i].x, gsb[i]));
        gRB.c1 = add(gRB.c1, scale(hB[i].y, gsb[i]));
        gRB.c2 = add(gRB.c2, scale(hB[i].z, gsb[i]));
    }
    add3(a.gp, ba, gpA);
    add3(a.gp, bb, gpB);
    add_m3(a.gR, ba, gRA);
    add_m3(a.gR, bb, gRB);
}

constexpr uint32_t kAdjWarps = 4;

__global__ void __launch_bounds__(kAdjWarps * 32)
    k_adjoint(World w, Consts k, Scratch s, AdjScratch a, Grads g, float dt) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t bundle = blockIdx.x * kAdjWarps + (threadIdx.x >> 5);
    if (bundle >= w.nbundles) return;
    const uint32_t b0 = w.bundle_off[bundle], b1 = w.bundle_off[bundle + 1];
    const uint32_t c0 = s.bundle_c0[bundle], c1 = s.bundle_c0[bundle + 1];
    const uint32_t ncb = c1 - c0;
    const uint32_t iters = k.pgs_iterations;

    // ---- working velocities (post-gravity) and cleared accumulators ----
    for (uint32_t b = b0 + lane; b < b1; b += 32) {
        for (int j = 0; j < 3; ++j) {
            a.vw[size_t(b) * 6 + j] = w.vel[size_t(b) * 3 + j];
            a.vw[size_t(b) * 6 + 3 + j] = w.omega[size_t(b) * 3 + j];
            a.gp[size_t(b) * 3 + j] = 0.f;
        }
        for (int j = 0; j < 9; ++j) a.gR[size_t(b) * 9 + j] = 0.f;
    }
    // ---- contact constants (physics.comp:504-521, 533-546) ----
    for (uint32_t c = c0 + lane; c < c1; c += 32) {
        const uint32_t ga = w.c_a[c], gb = w.c_b[c];
        const uint32_t ba = w.geom_body[ga], bb = w.geom_body[gb];
        const Body A = load_body(w, ba), B = load_body(w, bb);
        CParams p;
        p.n = ld3(w.c_normal, c);
        const f3 cp = ld3(w.c_pos, c);
        p.ra = sub(cp, ld3(w.pos, ba));
        p.rb = sub(cp, ld3(w.pos, bb));
        const f3 va = add(ld3(w.vel, ba), cross(ld3(w.omega, ba), p.ra));
        const f3 vb = add(ld3(w.vel, bb), cross(ld3(w.omega, bb), p.rb));
        const float vn = dot(sub(vb, va), p.n);
        const float e = gmax(w.restitution[ga], w.restitution[gb]);
        p.bias = k.baumgarte * gmax(w.c_pen[c] - k.slop, 0.0f) / dt + e * gmax(-vn, 0.0f);
        const f3 ran = cross(p.ra, p.n), rbn = cross(p.rb, p.n);
        p.kn = A.ima + B.ima + dot(ran, apply_inv_I(A.R, A.I, ran)) + dot(rbn, apply_inv_I(B.R, B.I, rbn));
        p.mu = sqrtf(w.friction[ga] * w.friction[gb]);
        st_par(a.par, c, p);
        a.lam[c] = 0.f;
        a.glam[c] = 0.f;
        st_grad(a.gc, c, CGrad{z3(), z3(), z3(), 0.f, 0.f, 0.f});
    }
    __syncwarp();

    // ---- the PGS sweep recomputed in the reference order, taped ----
    if (lane == 0 && ncb > 0) {
        for (uint32_t it = 0; it < iters; ++it)
            for (uint32_t c = c0; c < c1; ++c) {
                const uint32_t ba = w.geom_body[w.c_a[c]], bb = w.geom_body[w.c_b[c]];
                const Body A = load_body(w, ba), B = load_body(w, bb);
                if (A.ima == 0.0f && B.ima == 0.0f) continue;  // physics.comp:531
                f3 va = mk(a.vw[size_t(ba) * 6], a.vw[size_t(ba) * 6 + 1], a.vw[size_t(ba) * 6 + 2]);
                f3 wa = mk(a.vw[size_t(ba) * 6 + 3], a.vw[size_t(ba) * 6 + 4], a.vw[size_t(ba) * 6 + 5]);
                f3 vb = mk(a.vw[size_t(bb) * 6], a.vw[size_t(bb) * 6 + 1], a.vw[size_t(bb) * 6 + 2]);
                f3 wb = mk(a.vw[size_t(bb) * 6 + 3], a.vw[size_t(bb) * 6 + 4], a.vw[size_t(bb) * 6 + 5]);
                float lam = a.lam[c];
                float* t = a.tape + (size_t(c0) * iters + size_t(it) * ncb + (c - c0)) * 13;
                t[0] = va.x; t[1] = va.y; t[2] = va.z;
                t[3] = wa.x; t[4] = wa.y; t[5] = wa.z;
                t[6] = vb.x; t[7] = vb.y; t[8] = vb.z;
                t[9] = wb.x; t[10] = wb.y; t[11] = wb.z;
                t[12] = lam;
                update_fwd(A, B, ld_par(a.par, c), va, wa, vb, wb, lam);
                a.lam[c] = lam;
                for (int j = 0; j < 3; ++j) {
                    a.vw[size_t(ba) * 6 + j] = (&va.x)[j];
                    a.vw[size_t(ba) * 6 + 3 + j] = (&wa.x)[j];
                    a.vw[size_t(bb) * 6 + j] = (&vb.x)[j];
                    a.vw[size_t(bb) * 6 + 3 + j] = (&wb.x)[j];
                }
            }
    }
    __syncwarp();

    // ---- integration (physics.comp:586-604), reversed ----
    for (uint32_t b = b0 + lane; b < b1; b += 32) {
        const f3 Gp1 = ld3(g.pos, b), Gv1 = ld3(g.vel, b), Gw1 = ld3(g.omega, b);
        float Gq1[4] = {g.quat[size_t(b) * 4], g.quat[size_t(b) * 4 + 1], g.quat[size_t(b) * 4 + 2],
                        g.quat[size_t(b) * 4 + 3]};
        f3 Gv = Gv1, Gw = Gw1;
        float Gq[4] = {Gq1[0], Gq1[1], Gq1[2], Gq1[3]};
        if (w.inv_mass[b] > 0.0f) {
            acc_s(Gv, dt, Gp1);  // pos += vel dt
            const float ox = a.vw[size_t(b) * 6 + 3], oy = a.vw[size_t(b) * 6 + 4],
                        oz = a.vw[size_t(b) * 6 + 5];
            const float qx = w.quat[size_t(b) * 4], qy = w.quat[size_t(b) * 4 + 1],
                        qz = w.quat[size_t(b) * 4 + 2], qw = w.quat[size_t(b) * 4 + 3];
            const float dx = ox * qw + oy * qz - oz * qy;
            const float dy = -ox * qz + oy * qw + oz * qx;
            const float dz = ox * qy - oy * qx + oz * qw;
            const float dw = -ox * qx - oy * qy - oz * qz;
            const float ux = qx + 0.5f * dx * dt, uy = qy + 0.5f * dy * dt, uz = qz + 0.5f * dz * dt,
                        uw = qw + 0.5f * dw * dt;
            const float l = sqrtf(ux * ux + uy * uy + uz * uz + uw * uw);
            float gu[4] = {Gq1[0], Gq1[1], Gq1[2], Gq1[3]};
            if (l > 1e-8f) {  // q' = u / |u|
                const float nq[4] = {ux / l, uy / l, uz / l, uw / l};
                const float dp = nq[0] * Gq1[0] + nq[1] * Gq1[1] + nq[2] * Gq1[2] + nq[3] * Gq1[3];
                for (int j = 0; j < 4; ++j) gu[j] = (Gq1[j] - nq[j] * dp) / l;
            }
            const float h = 0.5f * dt;
            const float gdx = h * gu[0], gdy = h * gu[1], gdz = h * gu[2], gdw = h * gu[3];
            Gq[0] = gu[0] + gdy * oz - gdz * oy - gdw * ox;
            Gq[1] = gu[1] - gdx * oz + gdz * ox - gdw * oy;
            Gq[2] = gu[2] + gdx * oy - gdy * ox - gdw * oz;
            Gq[3] = gu[3] + gdx * ox + gdy * oy + gdz * oz;
            Gw.x += gdx * qw - gdy * qz + gdz * qy - gdw * qx;
            Gw.y += gdx * qz + gdy * qw - gdz * qx - gdw * qy;
            Gw.z += -gdx * qy + gdy * qx + gdz * qw - gdw * qz;
        }
        st3(a.gv, b, Gv);
        st3(a.gw, b, Gw);
        for (int j = 0; j < 4; ++j) a.gq[size_t(b) * 4 + j] = Gq[j];
        for (int j = 0; j < 3; ++j) a.gp[size_t(b) * 3 + j] = (&Gp1.x)[j];
    }
    __syncwarp();

    if (lane == 0 && ncb > 0) {
        // ---- the sweep, reversed ----
        for (int it = int(iters) - 1; it >= 0; --it)
            for (uint32_t c = c1; c-- > c0;) {
                const uint32_t ba = w.geom_body[w.c_a[c]], bb = w.geom_body[w.c_b[c]];
                const Body A = load_body(w, ba), B = load_body(w, bb);
                if (A.ima == 0.0f && B.ima == 0.0f) continue;
                const float* t = a.tape + (size_t(c0) * iters + size_t(it) * ncb + (c - c0)) * 13;
                f3 Gva = ld3(a.gv, ba), Gwa = ld3(a.gw, ba), Gvb = ld3(a.gv, bb), Gwb = ld3(a.gw, bb);
                float glam = a.glam[c];
                CGrad gc = ld_grad(a.gc, c);
                m3 gRa = m3zero(), gRb = m3zero();
                update_bwd(A, B, ld_par(a.par, c), mk(t[0], t[1], t[2]), mk(t[3], t[4], t[5]),
                           mk(t[6], t[7], t[8]), mk(t[9], t[10], t[11]), t[12], Gva, Gwa, Gvb, Gwb,
                           glam, gc, gRa, gRb);
                st3(a.gv, ba, Gva);
                st3(a.gw, ba, Gwa);
                st3(a.gv, bb, Gvb);
                st3(a.gw, bb, Gwb);
                a.glam[c] = glam;
                st_grad(a.gc, c, gc);
                add_m3(a.gR, ba, gRa);
                add_m3(a.gR, bb, gRb);
            }
        // ---- contact constants and contact geometry, reversed ----
        for (uint32_t c = c0; c < c1; ++c) {
            const uint32_t ga = w.c_a[c], gb = w.c_b[c];
            const uint32_t ba = w.geom_body[ga], bb = w.geom_body[gb];
            const Body A = load_body(w, ba), B = load_body(w, bb);
            const CParams p = ld_par(a.par, c);
            CGrad gc = ld_grad(a.gc, c);
            m3 gRa = m3zero(), gRb = m3zero();
            // kn = ima + imb + ran·A(ran) + rbn·A(rbn); ran = ra x n
            const f3 ran = cross(p.ra, p.n), rbn = cross(p.rb, p.n);
            const f3 g_ran = scale(2.f * gc.kn, apply_inv_I(A.R, A.I, ran));
            const f3 g_rbn = scale(2.f * gc.kn, apply_inv_I(B.R, B.I, rbn));
            inv_I_bwd(A.R, A.I, ran, scale(gc.kn, ran), gRa);
            inv_I_bwd(B.R, B.I, rbn, scale(gc.kn, rbn), gRb);
            acc(gc.ra, cross(p.n, g_ran));
            acc(gc.n, cross(g_ran, p.ra));
            acc(gc.rb, cross(p.n, g_rbn));
            acc(gc.n, cross(g_rbn, p.rb));
            // bias = baum max(pen - slop, 0)/dt + e max(-vn0, 0)
            const float pen = w.c_pen[c];
            const float g_pen = (pen - k.slop < 0.f) ? 0.f : gc.bias * k.baumgarte / dt;
            const float e = gmax(w.restitution[ga], w.restitution[gb]);
            const f3 va0 = add(ld3(w.vel, ba), cross(ld3(w.omega, ba), p.ra));
            const f3 vb0 = add(ld3(w.vel, bb), cross(ld3(w.omega, bb), p.rb));
            const float vn0 = dot(sub(vb0, va0), p.n);
            const float g_vn0 = (-vn0 < 0.f) ? 0.f : -e * gc.bias;
            acc_s(gc.n, g_vn0, sub(vb0, va0));
            const f3 g_ub0 = scale(g_vn0, p.n), g_ua0 = neg(g_ub0);
            add3(a.gv, ba, g_ua0);
            add3(a.gw, ba, cross(p.ra, g_ua0));
            acc(gc.ra, cross(g_ua0, ld3(w.omega, ba)));
            add3(a.gv, bb, g_ub0);
            add3(a.gw, bb, cross(p.rb, g_ub0));
            acc(gc.rb, cross(g_ub0, ld3(w.omega, bb)));
            // mu = sqrt(fa fb)
            if (p.mu > 0.f) {
                const float fa = w.friction[ga], fb = w.friction[gb];
                g.friction[ga] += gc.mu * fb / (2.f * p.mu);
                g.friction[gb] += gc.mu * fa / (2.f * p.mu);
            }
            // ra = cp - pos_a; rb = cp - pos_b
            const f3 g_cp = add(gc.ra, gc.rb);
            add3(a.gp, ba, neg(gc.ra));
            add3(a.gp, bb, neg(gc.rb));
            add_m3(a.gR, ba, gRa);
            add_m3(a.gR, bb, gRb);
            contact_geom_bwd(w, k, a, c, ba, bb, gc.n, g_pen, g_cp);
        }
    }
    __syncwarp();

    // ---- rotations -> quaternions, gravity (physics.comp:418-428), reversed
    for (uint32_t b = b0 + lane; b < b1; b += 32) {
        float gq[4];
        quat_bwd(w.quat[size_t(b) * 4], w.quat[size_t(b) * 4 + 1], w.quat[size_t(b) * 4 + 2],
                 w.quat[size_t(b) * 4 + 3], a.gR + size_t(b) * 9, gq);
        for (int j = 0; j < 4; ++j) g.quat[size_t(b) * 4 + j] = a.gq[size_t(b) * 4 + j] + gq[j];
        f3 Gv = ld3(a.gv, b), Gw = ld3(a.gw, b);
        if (w.inv_mass[b] > 0.0f) {
            Gv = scale(k.lin_damp, Gv);
            Gw = scale(k.ang_damp, Gw);
        }
        st3(g.vel, b, Gv);
        st3(g.omega, b, Gw);
        st3(g.pos, b, ld3(a.gp, b));
    }
}

}  // namespace

int launch_adjoint(const World& w, const Consts& k, const Scratch& s, const AdjScratch& a,
                   const Grads& g, float dt, cudaStream_t st) {
    if (w.nbundles == 0) return 0;
    const uint32_t blocks = (w.nbundles + kAdjWarps - 1) / kAdjWarps;
    k_adjoint<<<blocks, kAdjWarps * 32, 0, st>>>(w, k, s, a, g, dt);
    return 1;
}

}  // namespace seevr
