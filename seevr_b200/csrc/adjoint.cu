// adjoint.cu — reverse mode of one physics substep, for gradients of a
// rollout with respect to initial positions, orientations, velocities,
// angular velocities and friction coefficients.
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
//
// Precision: every forward quantity is recomputed in FP32 with the forward's
// arithmetic, so branch decisions and values are the forward's own; the
// reverse-mode arithmetic on them runs in FP64 (type d3 below).  The PGS
// sweep's per-iteration sensitivities nearly cancel (later iterations undo
// most of an earlier impulse), so FP32 accumulation loses digits, most
// visibly in the friction gradient, while FP64 keeps the result to the
// FP32 forward's own accuracy.
//
// Parallelism: one warp per solver bundle.  The sweep's contacts get the
// solver's wavefront levels (contacts of one level touch disjoint dynamic
// bodies), so the recomputed sweep, its reverse and the constants' reverse
// run a level at a time across the lanes.  Every dynamic body still
// receives its gradient contributions in the serial order; contributions to
// fixed bodies (shared by contacts of one level) are kept per contact and
// summed in contact order at the end, so the result stays deterministic.
#include "adjoint.cuh"

namespace seevr {
namespace {

// ---- FP64 vectors for the reverse pass (operators only on d3, so an FP32
// f3 can never enter a derivative expression without an explicit D()) ----
struct d3 {
    double x, y, z;
};
struct dm3 {
    d3 c0, c1, c2;
};
__device__ __forceinline__ d3 D(f3 a) { return d3{a.x, a.y, a.z}; }
__device__ __forceinline__ dm3 DM(const m3& m) { return dm3{D(m.c0), D(m.c1), D(m.c2)}; }
__device__ __forceinline__ d3 dz() { return d3{0.0, 0.0, 0.0}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator-(d3 a) { return d3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return d3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ d3& operator+=(d3& a, d3 b) {
    a = a + b;
    return a;
}
__device__ __forceinline__ double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 dcross(d3 a, d3 b) {
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 dhad(d3 a, d3 b) { return d3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ d3 dmul(const dm3& m, d3 v) { return v.x * m.c0 + v.y * m.c1 + v.z * m.c2; }
__device__ __forceinline__ d3 dmulT(const dm3& m, d3 v) {
    return d3{ddot(m.c0, v), ddot(m.c1, v), ddot(m.c2, v)};
}
// R (I ⊙ (Rᵀ v)) (apply_inv_I, physics.comp:90-94) in FP64
__device__ __forceinline__ d3 dapply(const dm3& R, d3 I, d3 v) { return dmul(R, dhad(I, dmulT(R, v))); }
__device__ __forceinline__ dm3 dm3zero() { return dm3{dz(), dz(), dz()}; }
__device__ __forceinline__ void addd3(double* p, uint32_t i, d3 v) {
    p[size_t(i) * 3] += v.x;
    p[size_t(i) * 3 + 1] += v.y;
    p[size_t(i) * 3 + 2] += v.z;
}
__device__ __forceinline__ d3 ldd3(const double* p, uint32_t i) {
    return d3{p[size_t(i) * 3], p[size_t(i) * 3 + 1], p[size_t(i) * 3 + 2]};
}
__device__ __forceinline__ void std3(double* p, uint32_t i, d3 v) {
    p[size_t(i) * 3] = v.x;
    p[size_t(i) * 3 + 1] = v.y;
    p[size_t(i) * 3 + 2] = v.z;
}
__device__ __forceinline__ void add_dm3(double* p, uint32_t i, const dm3& g) {
    double* q = p + size_t(i) * 9;
    q[0] += g.c0.x; q[1] += g.c0.y; q[2] += g.c0.z;
    q[3] += g.c1.x; q[4] += g.c1.y; q[5] += g.c1.z;
    q[6] += g.c2.x; q[7] += g.c2.y; q[8] += g.c2.z;
}

// y = R (I ⊙ (Rᵀ x)): accumulates dL/dR into gR (columns) and returns dL/dx
// (the map is symmetric in x).
__device__ __forceinline__ d3 inv_I_bwd(const dm3& R, d3 I, d3 x, d3 gy, dm3& gR) {
    const d3 u = dhad(I, dmulT(R, x));
    const d3 gw = dhad(I, dmulT(R, gy));
    gR.c0 += u.x * gy + gw.x * x;
    gR.c1 += u.y * gy + gw.y * x;
    gR.c2 += u.z * gy + gw.z * x;
    return dmul(R, gw);
}

// dL/d(x,y,z,w) of quat_to_mat (physics.comp:74-81) from dL/dR by columns
__device__ __forceinline__ void quat_bwd(double x, double y, double z, double w, const double* g,
                                         double out[4]) {
    out[0] = 2.0 * (g[1] * y + g[2] * z + g[3] * y - 2.0 * g[4] * x + g[5] * w + g[6] * z -
                    g[7] * w - 2.0 * g[8] * x);
    out[1] = 2.0 * (-2.0 * g[0] * y + g[1] * x - g[2] * w + g[3] * x + g[5] * z + g[6] * w +
                    g[7] * z - 2.0 * g[8] * y);
    out[2] = 2.0 * (-2.0 * g[0] * z + g[1] * w + g[2] * x - g[3] * w - 2.0 * g[4] * z + g[5] * y +
                    g[6] * x + g[7] * y);
    out[3] = 2.0 * (g[1] * z - g[2] * y - g[3] * z + g[5] * x + g[6] * y - g[7] * x);
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

// Contact constants (FP32, the forward's values) and their gradients (FP64).
struct CParams {
    f3 n, ra, rb;
    float bias, kn, mu;
};
struct CGrad {
    d3 n, ra, rb;
    double bias, kn, mu;
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
__device__ __forceinline__ CGrad ld_grad(const double* p, uint32_t c) {
    const double* q = p + size_t(c) * 12;
    return CGrad{d3{q[0], q[1], q[2]}, d3{q[3], q[4], q[5]}, d3{q[6], q[7], q[8]}, q[9], q[10],
                 q[11]};
}
__device__ __forceinline__ void st_grad(double* p, uint32_t c, const CGrad& v) {
    double* q = p + size_t(c) * 12;
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
                           f3 wb, float lam, d3& Gva, d3& Gwa, d3& Gvb, d3& Gwb, double& glam,
                           CGrad& gc, dm3& gRa, dm3& gRb) {
    // forward intermediates, FP32 as in the forward: the same values and branches
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
    // the reverse pass, FP64
    const dm3 RA = DM(A.R), RB = DM(B.R);
    const d3 IA = D(A.I), IB = D(B.I);
    const double ima = A.ima, imb = B.ima;
    const d3 n = D(c.n), ra = D(c.ra), rb = D(c.rb);
    // gradients of the outputs: a fixed body's outputs are discarded
    const d3 gva2 = A.fixed ? dz() : Gva, gwa2 = A.fixed ? dz() : Gwa;
    const d3 gvb2 = B.fixed ? dz() : Gvb, gwb2 = B.fixed ? dz() : Gwb;
    d3 gva1 = gva2, gwa1 = gwa2, gvb1 = gvb2, gwb1 = gwb2;
    double g_l1 = glam;
    d3 g_vt = dz();
    double g_s = 0.0;
    if (s > 1e-6f) {
        const f3 tdf = divs(vt, s);
        const f3 ratf = cross(c.ra, tdf), rbtf = cross(c.rb, tdf);
        const float kt = A.ima + B.ima + dot(ratf, apply_inv_I(A.R, A.I, ratf)) +
                         dot(rbtf, apply_inv_I(B.R, B.I, rbtf));
        const float q1 = s / kt, q2 = c.mu * l1;
        const bool take2 = q2 < q1;  // GLSL min(q1, q2)
        const float dtf = take2 ? q2 : q1;
        const f3 itf = scale(dtf, tdf);
        const d3 td = D(tdf), it = D(itf), rat = D(ratf), rbt = D(rbtf);
        const double ktd = kt, sd = s, dtd = dtf;
        d3 g_it = dz();
        // wa2 = wa1 + A(ra x it); wb2 = wb1 - B(rb x it)
        const d3 g_xa2 = inv_I_bwd(RA, IA, D(cross(c.ra, itf)), gwa2, gRa);
        const d3 g_xb2 = inv_I_bwd(RB, IB, D(cross(c.rb, itf)), -gwb2, gRb);
        gc.ra += dcross(it, g_xa2);
        g_it += dcross(g_xa2, ra);
        gc.rb += dcross(it, g_xb2);
        g_it += dcross(g_xb2, rb);
        // va2 = va1 + ima it; vb2 = vb1 - imb it
        g_it += ima * gva2;
        g_it += (-imb) * gvb2;
        // it = dt_ td
        const double g_dt = ddot(g_it, td);
        d3 g_td = dtd * g_it;
        double g_kt = 0.0;
        if (take2) {
            gc.mu += g_dt * double(l1);
            g_l1 += g_dt * double(c.mu);
        } else {
            g_s += g_dt / ktd;
            g_kt = -g_dt * sd / (ktd * ktd);
        }
        // kt = ... + rat·A(rat) + rbt·B(rbt): d/drat = 2 A(rat)
        const d3 g_rat = (2.0 * g_kt) * dapply(RA, IA, rat);
        const d3 g_rbt = (2.0 * g_kt) * dapply(RB, IB, rbt);
        inv_I_bwd(RA, IA, rat, g_kt * rat, gRa);
        inv_I_bwd(RB, IB, rbt, g_kt * rbt, gRb);
        // rat = ra x td
        gc.ra += dcross(td, g_rat);
        g_td += dcross(g_rat, ra);
        gc.rb += dcross(td, g_rbt);
        g_td += dcross(g_rbt, rb);
        // td = vt / s
        g_vt += (1.0 / sd) * g_td;
        g_s += -ddot(g_td, D(vt)) / (sd * sd);
    }
    if (s > 0.f) g_vt += (g_s / double(s)) * D(vt);
    // vt = dv - dn n; dn = dv·n
    d3 g_dv = g_vt;
    const double g_dn = -ddot(g_vt, n);
    gc.n += (-double(dn)) * g_vt;
    g_dv += g_dn * n;
    gc.n += g_dn * D(dv);
    // dv = ub1 - ua1; ua1 = va1 + wa1 x ra
    const d3 g_ua1 = -g_dv, g_ub1 = g_dv;
    gva1 += g_ua1;
    gwa1 += dcross(ra, g_ua1);
    gc.ra += dcross(g_ua1, D(wa1));
    gvb1 += g_ub1;
    gwb1 += dcross(rb, g_ub1);
    gc.rb += dcross(g_ub1, D(wb1));
    // wa1 = wa - A(xa); wb1 = wb + B(xb); xa = ra x imp
    d3 gi_va = gva1, gi_wa = gwa1, gi_vb = gvb1, gi_wb = gwb1, g_imp = dz();
    const d3 g_xa = inv_I_bwd(RA, IA, D(xa), -gwa1, gRa);
    const d3 g_xb = inv_I_bwd(RB, IB, D(xb), gwb1, gRb);
    const d3 impd = D(imp);
    gc.ra += dcross(impd, g_xa);
    g_imp += dcross(g_xa, ra);
    gc.rb += dcross(impd, g_xb);
    g_imp += dcross(g_xb, rb);
    // va1 = va - ima imp; vb1 = vb + imb imp
    g_imp += (-ima) * gva1;
    g_imp += imb * gvb1;
    // imp = d n
    const double g_d = ddot(g_imp, n);
    gc.n += double(d) * g_imp;
    // d = l1 - lam; l1 = max(s1, 0); s1 = lam + d0
    g_l1 += g_d;
    double gi_lam = -g_d;
    const double g_s1 = s1 < 0.f ? 0.0 : g_l1;
    gi_lam += g_s1;
    // d0 = (-vn + bias) / kn
    const double knd = c.kn;
    const double g_vn = -g_s1 / knd;
    gc.bias += g_s1 / knd;
    gc.kn += -g_s1 * double(d0) / knd;
    // vn = dvn·n; dvn = ub - ua; ua = va + wa x ra
    gc.n += g_vn * D(dvn);
    const d3 g_ub = g_vn * n, g_ua = -g_ub;
    gi_va += g_ua;
    gi_wa += dcross(ra, g_ua);
    gc.ra += dcross(g_ua, D(wa));
    gi_vb += g_ub;
    gi_wb += dcross(rb, g_ub);
    gc.rb += dcross(g_ub, D(wb));
    // a fixed body's state persists: its incoming gradient passes through
    Gva = A.fixed ? Gva + gi_va : gi_va;
    Gwa = A.fixed ? Gwa + gi_wa : gi_wa;
    Gvb = B.fixed ? Gvb + gi_vb : gi_vb;
    Gwb = B.fixed ? Gwb + gi_wb : gi_wb;
    glam = gi_lam;
}

__device__ __forceinline__ f3 hull_vert(const World& w, uint32_t vs, uint32_t i) {
    return i == kNone ? mk(0.f, 0.f, 0.f) : ld3(w.hull, vs + i);
}

// dL/d (positions, rotations) of one contact's normal, depth and point,
// through the taped supporting vertices (physics.comp:224-247, 346-365,
// 376-387).  The support points are recomputed in FP32 as the narrowphase
// computed them; the derivatives are FP64.
__device__ void contact_geom_bwd(const World& w, const Consts& k, const AdjScratch& a, uint32_t c,
                                 uint32_t ba, uint32_t bb, d3 g_n, double g_pen, d3 g_cp,
                                 d3& gpA, d3& gpB, dm3& gRA, dm3& gRB) {
    const uint4 t0 = a.ctape[size_t(c) * 2], t1 = a.ctape[size_t(c) * 2 + 1];
    const f3 pAf = ld3(w.pos, ba), pBf = ld3(w.pos, bb);
    const m3 RAf = quat_to_mat(w.quat, ba), RBf = quat_to_mat(w.quat, bb);
    const uint32_t vsA = w.hull_range[size_t(ba) * 2], vsB = w.hull_range[size_t(bb) * 2];
    f3 hA[4], hB[4], saf[4], sbf[4], vf[4];
    d3 gsa[4], gsb[4], gv[4];
    const uint32_t ia[4] = {kNone, t0.y, t0.w, t1.y};
    const uint32_t ib[4] = {kNone, t0.z, t1.x, t1.z};
    for (int i = 0; i < 4; ++i) {
        hA[i] = hull_vert(w, vsA, ia[i]);
        hB[i] = hull_vert(w, vsB, ib[i]);
        saf[i] = add(pAf, mul(RAf, hA[i]));
        sbf[i] = add(pBf, mul(RBf, hB[i]));
        vf[i] = sub(saf[i], sbf[i]);
        gsa[i] = gsb[i] = gv[i] = dz();
    }
    gpA = dz();
    gpB = dz();
    if (t0.x == 2u) {  // segment case: depth = |v1|, n = v1/|v1|, cp = (s1a + s1b)/2
        const d3 v1 = D(vf[1]);
        const double l = sqrt(ddot(v1, v1));
        const d3 n = (1.0 / l) * v1;
        d3 g1 = g_pen * n;
        g1 += (1.0 / l) * (g_n - ddot(n, g_n) * n);
        gsa[1] = 0.5 * g_cp + g1;
        gsb[1] = 0.5 * g_cp - g1;
    } else {  // portal: n = normalize((v2-v1)x(v3-v1)), depth = n·v1, cp = find_pos
        f3 v0f = sub(pAf, pBf);
        if (fabsf(v0f.x) < k.eps && fabsf(v0f.y) < k.eps && fabsf(v0f.z) < k.eps)
            v0f.x += 10.0f * k.eps;
        vf[0] = v0f;
        saf[0] = pAf;
        sbf[0] = pBf;
        d3 v[4], sa[4], sb[4];
        for (int i = 0; i < 4; ++i) {
            v[i] = D(vf[i]);
            sa[i] = D(saf[i]);
            sb[i] = D(sbf[i]);
        }
        const d3 e1 = v[2] - v[1], e2 = v[3] - v[1];
        const d3 cr = dcross(e1, e2);
        const double cl = sqrt(ddot(cr, cr));
        const d3 n = (1.0 / cl) * cr;
        d3 g_nn = g_n;
        g_nn += g_pen * v[1];
        gv[1] += g_pen * n;
        // contact point: the forward's fallback test (FP32, find_pos)
        const float fsum = dot(cross(vf[1], vf[2]), vf[3]) + -dot(cross(vf[0], vf[2]), vf[3]) +
                           dot(cross(vf[0], vf[1]), vf[3]) + -dot(cross(vf[0], vf[1]), vf[2]);
        const bool fallback = fabsf(fsum) < k.eps;
        double b[4];
        if (!fallback) {
            b[0] = ddot(dcross(v[1], v[2]), v[3]);
            b[1] = -ddot(dcross(v[0], v[2]), v[3]);
            b[2] = ddot(dcross(v[0], v[1]), v[3]);
            b[3] = -ddot(dcross(v[0], v[1]), v[2]);
        } else {
            b[0] = 0.0;
            b[1] = ddot(dcross(v[2], v[3]), n);
            b[2] = ddot(dcross(v[3], v[1]), n);
            b[3] = ddot(dcross(v[1], v[2]), n);
        }
        const double sum = b[0] + b[1] + b[2] + b[3];
        d3 P = dz();
        for (int i = 0; i < 4; ++i) P += b[i] * (sa[i] + sb[i]);
        const d3 gP = (0.5 / sum) * g_cp;
        const double g_sum = -0.5 / (sum * sum) * ddot(g_cp, P);
        double gb[4];
        for (int i = 0; i < 4; ++i) {
            gb[i] = ddot(gP, sa[i]) + ddot(gP, sb[i]) + g_sum;
            gsa[i] += b[i] * gP;
            gsb[i] += b[i] * gP;
        }
        if (!fallback) {
            // triple products [a,b,c] = (a x b)·c: d/da = b x c, d/db = c x a, d/dc = a x b
            gv[1] += gb[0] * dcross(v[2], v[3]);
            gv[2] += gb[0] * dcross(v[3], v[1]);
            gv[3] += gb[0] * dcross(v[1], v[2]);
            gv[0] += (-gb[1]) * dcross(v[2], v[3]);
            gv[2] += (-gb[1]) * dcross(v[3], v[0]);
            gv[3] += (-gb[1]) * dcross(v[0], v[2]);
            gv[0] += gb[2] * dcross(v[1], v[3]);
            gv[1] += gb[2] * dcross(v[3], v[0]);
            gv[3] += gb[2] * dcross(v[0], v[1]);
            gv[0] += (-gb[3]) * dcross(v[1], v[2]);
            gv[1] += (-gb[3]) * dcross(v[2], v[0]);
            gv[2] += (-gb[3]) * dcross(v[0], v[1]);
        } else {
            // b1 = (v2 x v3)·n, b2 = (v3 x v1)·n, b3 = (v1 x v2)·n
            gv[2] += gb[1] * dcross(v[3], n);
            gv[3] += gb[1] * dcross(n, v[2]);
            g_nn += gb[1] * dcross(v[2], v[3]);
            gv[3] += gb[2] * dcross(v[1], n);
            gv[1] += gb[2] * dcross(n, v[3]);
            g_nn += gb[2] * dcross(v[3], v[1]);
            gv[1] += gb[3] * dcross(v[2], n);
            gv[2] += gb[3] * dcross(n, v[1]);
            g_nn += gb[3] * dcross(v[1], v[2]);
        }
        // n = cr / |cr|; cr = e1 x e2
        const d3 g_cr = (1.0 / cl) * (g_nn - ddot(n, g_nn) * n);
        const d3 g_e1 = dcross(e2, g_cr), g_e2 = dcross(g_cr, e1);
        gv[2] += g_e1;
        gv[3] += g_e2;
        gv[1] = gv[1] - (g_e1 + g_e2);
        // v0 = pA - pB; s0a = pA; s0b = pB
        gpA += gv[0] + gsa[0];
        gpB += gsb[0] - gv[0];
        for (int i = 1; i < 4; ++i) {
            gsa[i] += gv[i];
            gsb[i] = gsb[i] - gv[i];
        }
    }
    // s_ia = pA + RA h_ia; s_ib = pB + RB h_ib (i = 1..3)
    gRA = dm3zero();
    gRB = dm3zero();
    for (int i = 1; i < 4; ++i) {
        gpA += gsa[i];
        gpB += gsb[i];
        const d3 ha = D(hA[i]), hb = D(hB[i]);
        gRA.c0 += ha.x * gsa[i];
        gRA.c1 += ha.y * gsa[i];
        gRA.c2 += ha.z * gsa[i];
        gRB.c0 += hb.x * gsb[i];
        gRB.c1 += hb.y * gsb[i];
        gRB.c2 += hb.z * gsb[i];
    }
}

constexpr uint32_t kAdjWarps = 4;
constexpr uint32_t kFixStride = 20;  // v3 w3 p3 R9 friction1

// A contact side's contribution to a fixed body's gradients, kept with the
// contact (fixed bodies are shared by contacts of one level).
__device__ __forceinline__ double* fix_slot(const AdjScratch& a, uint32_t c, int side) {
    return a.fix + (size_t(c) * 2 + side) * kFixStride;
}
__device__ __forceinline__ void fix_add3(double* f, int off, d3 v) {
    f[off] += v.x;
    f[off + 1] += v.y;
    f[off + 2] += v.z;
}
__device__ __forceinline__ void fix_addR(double* f, const dm3& g) {
    f[9] += g.c0.x; f[10] += g.c0.y; f[11] += g.c0.z;
    f[12] += g.c1.x; f[13] += g.c1.y; f[14] += g.c1.z;
    f[15] += g.c2.x; f[16] += g.c2.y; f[17] += g.c2.z;
}

__global__ void __launch_bounds__(kAdjWarps * 32)
    k_adjoint(World w, Consts k, Scratch s, AdjScratch a, Grads g, float dt) {
    if (halted(w.status)) return;  // the recomputed contacts are not valid
    const unsigned full = 0xFFFFFFFFu;
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
            a.gp[size_t(b) * 3 + j] = 0.0;
        }
        for (int j = 0; j < 9; ++j) a.gR[size_t(b) * 9 + j] = 0.0;
        a.last[b] = 0;
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
        a.glam[c] = 0.0;
        st_grad(a.gc, c, CGrad{dz(), dz(), dz(), 0.0, 0.0, 0.0});
        double* f = fix_slot(a, c, 0);
        for (uint32_t j = 0; j < 2 * kFixStride; ++j) f[j] = 0.0;
    }
    __syncwarp();

    // ---- wavefront levels: a contact comes after every earlier contact
    // sharing a dynamic body with it, so contacts of one level touch disjoint
    // dynamic bodies (the solver's rule; skipped contacts get no level) ----
    uint32_t maxl = 0;
    for (uint32_t cb = c0; cb < c1; cb += 32) {
        const uint32_t c = cb + lane;
        const bool valid = c < c1;
        uint32_t ba = 0, bb = 0;
        bool use = false, da = false, db = false;
        if (valid) {
            ba = w.geom_body[w.c_a[c]];
            bb = w.geom_body[w.c_b[c]];
            use = !(w.inv_mass[ba] == 0.0f && w.inv_mass[bb] == 0.0f);  // physics.comp:531
            da = use && !load_body(w, ba).fixed;
            db = use && !load_body(w, bb).fixed;
        }
        const uint32_t xa = da ? ba : (0x80000000u | (lane * 2u));
        const uint32_t xb = db ? bb : (0x80000000u | (lane * 2u + 1u));
        uint32_t L = use ? max(da ? a.last[ba] : 0u, db ? a.last[bb] : 0u) + 1u : 0u;
        for (uint32_t j = 0; j < 32; ++j) {
            const uint32_t aj = __shfl_sync(full, xa, j), bj = __shfl_sync(full, xb, j);
            const uint32_t Lj = __shfl_sync(full, L, j);
            if (use && j < lane && (aj == xa || aj == xb || bj == xa || bj == xb)) L = max(L, Lj + 1u);
        }
        if (da) atomicMax(&a.last[ba], L);
        if (db) atomicMax(&a.last[bb], L);
        if (valid) a.level[c] = use ? L - 1u : kNone;
        maxl = max(maxl, L);
        __syncwarp();
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) maxl = max(maxl, __shfl_xor_sync(full, maxl, off));
    uint32_t* lvl = a.lvl + c0 + bundle;  // [maxl + 1], within [c0 + bundle, c1 + bundle]
    uint32_t pos = 0;
    for (uint32_t l = 0; l < maxl; ++l) {
        if (lane == 0) lvl[l] = pos;
        for (uint32_t cb = c0; cb < c1; cb += 32) {
            const uint32_t c = cb + lane;
            const bool hit = c < c1 && a.level[c] == l;
            const unsigned m = __ballot_sync(full, hit);
            if (hit) a.order[c0 + pos + __popc(m & ((1u << lane) - 1u))] = c;
            pos += __popc(m);
        }
    }
    if (lane == 0) lvl[maxl] = pos;
    __syncwarp();

    // ---- the PGS sweep recomputed level by level, taped ----
    for (uint32_t it = 0; it < iters; ++it)
        for (uint32_t l = 0; l < maxl; ++l) {
            for (uint32_t j = lvl[l] + lane; j < lvl[l + 1]; j += 32) {
                const uint32_t c = a.order[c0 + j];
                const uint32_t ba = w.geom_body[w.c_a[c]], bb = w.geom_body[w.c_b[c]];
                const Body A = load_body(w, ba), B = load_body(w, bb);
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
                if (!A.fixed)
                    for (int q = 0; q < 3; ++q) {
                        a.vw[size_t(ba) * 6 + q] = (&va.x)[q];
                        a.vw[size_t(ba) * 6 + 3 + q] = (&wa.x)[q];
                    }
                if (!B.fixed)
                    for (int q = 0; q < 3; ++q) {
                        a.vw[size_t(bb) * 6 + q] = (&vb.x)[q];
                        a.vw[size_t(bb) * 6 + 3 + q] = (&wb.x)[q];
                    }
            }
            __syncwarp();
        }

    // ---- integration (physics.comp:586-604), reversed ----
    for (uint32_t b = b0 + lane; b < b1; b += 32) {
        const d3 Gp1 = ldd3(g.pos, b), Gv1 = ldd3(g.vel, b), Gw1 = ldd3(g.omega, b);
        const double Gq1[4] = {g.quat[size_t(b) * 4], g.quat[size_t(b) * 4 + 1],
                               g.quat[size_t(b) * 4 + 2], g.quat[size_t(b) * 4 + 3]};
        d3 Gv = Gv1, Gw = Gw1;
        double Gq[4] = {Gq1[0], Gq1[1], Gq1[2], Gq1[3]};
        if (w.inv_mass[b] > 0.0f) {
            Gv += double(dt) * Gp1;  // pos += vel dt
            const float ox = a.vw[size_t(b) * 6 + 3], oy = a.vw[size_t(b) * 6 + 4],
                        oz = a.vw[size_t(b) * 6 + 5];
            const float qx = w.quat[size_t(b) * 4], qy = w.quat[size_t(b) * 4 + 1],
                        qz = w.quat[size_t(b) * 4 + 2], qw = w.quat[size_t(b) * 4 + 3];
            const float dx = ox * qw + oy * qz - oz * qy;
            const float dy = -ox * qz + oy * qw + oz * qx;
            const float dzq = ox * qy - oy * qx + oz * qw;
            const float dw = -ox * qx - oy * qy - oz * qz;
            const float ux = qx + 0.5f * dx * dt, uy = qy + 0.5f * dy * dt,
                        uz = qz + 0.5f * dzq * dt, uw = qw + 0.5f * dw * dt;
            const float l = sqrtf(ux * ux + uy * uy + uz * uz + uw * uw);
            double gu[4] = {Gq1[0], Gq1[1], Gq1[2], Gq1[3]};
            if (l > 1e-8f) {  // q' = u / |u|
                const double ld = l;
                const double nq[4] = {ux / ld, uy / ld, uz / ld, uw / ld};
                const double dp = nq[0] * Gq1[0] + nq[1] * Gq1[1] + nq[2] * Gq1[2] + nq[3] * Gq1[3];
                for (int j = 0; j < 4; ++j) gu[j] = (Gq1[j] - nq[j] * dp) / ld;
            }
            const double h = 0.5 * double(dt);
            const double gdx = h * gu[0], gdy = h * gu[1], gdz = h * gu[2], gdw = h * gu[3];
            const double Ox = ox, Oy = oy, Oz = oz, Qx = qx, Qy = qy, Qz = qz, Qw = qw;
            Gq[0] = gu[0] + gdy * Oz - gdz * Oy - gdw * Ox;
            Gq[1] = gu[1] - gdx * Oz + gdz * Ox - gdw * Oy;
            Gq[2] = gu[2] + gdx * Oy - gdy * Ox - gdw * Oz;
            Gq[3] = gu[3] + gdx * Ox + gdy * Oy + gdz * Oz;
            Gw.x += gdx * Qw - gdy * Qz + gdz * Qy - gdw * Qx;
            Gw.y += gdx * Qz + gdy * Qw - gdz * Qx - gdw * Qy;
            Gw.z += -gdx * Qy + gdy * Qx + gdz * Qw - gdw * Qz;
        }
        std3(a.gv, b, Gv);
        std3(a.gw, b, Gw);
        for (int j = 0; j < 4; ++j) a.gq[size_t(b) * 4 + j] = Gq[j];
        std3(a.gp, b, Gp1);
    }
    __syncwarp();

    // ---- the sweep, reversed: levels in reverse order, the contacts of a
    // level in parallel; a fixed side's gradient goes to the contact's slot ----
    for (int it = int(iters) - 1; it >= 0; --it)
        for (int l = int(maxl) - 1; l >= 0; --l) {
            for (uint32_t j = lvl[l] + lane; j < lvl[l + 1]; j += 32) {
                const uint32_t c = a.order[c0 + j];
                const uint32_t ba = w.geom_body[w.c_a[c]], bb = w.geom_body[w.c_b[c]];
                const Body A = load_body(w, ba), B = load_body(w, bb);
                const float* t = a.tape + (size_t(c0) * iters + size_t(it) * ncb + (c - c0)) * 13;
                d3 Gva = A.fixed ? dz() : ldd3(a.gv, ba), Gwa = A.fixed ? dz() : ldd3(a.gw, ba);
                d3 Gvb = B.fixed ? dz() : ldd3(a.gv, bb), Gwb = B.fixed ? dz() : ldd3(a.gw, bb);
                double glam = a.glam[c];
                CGrad gc = ld_grad(a.gc, c);
                dm3 gRa = dm3zero(), gRb = dm3zero();
                update_bwd(A, B, ld_par(a.par, c), mk(t[0], t[1], t[2]), mk(t[3], t[4], t[5]),
                           mk(t[6], t[7], t[8]), mk(t[9], t[10], t[11]), t[12], Gva, Gwa, Gvb, Gwb,
                           glam, gc, gRa, gRb);
                if (A.fixed) {
                    double* f = fix_slot(a, c, 0);
                    fix_add3(f, 0, Gva);
                    fix_add3(f, 3, Gwa);
                    fix_addR(f, gRa);
                } else {
                    std3(a.gv, ba, Gva);
                    std3(a.gw, ba, Gwa);
                    add_dm3(a.gR, ba, gRa);
                }
                if (B.fixed) {
                    double* f = fix_slot(a, c, 1);
                    fix_add3(f, 0, Gvb);
                    fix_add3(f, 3, Gwb);
                    fix_addR(f, gRb);
                } else {
                    std3(a.gv, bb, Gvb);
                    std3(a.gw, bb, Gwb);
                    add_dm3(a.gR, bb, gRb);
                }
                a.glam[c] = glam;
                st_grad(a.gc, c, gc);
            }
            __syncwarp();
        }

    // ---- contact constants and contact geometry, reversed (level order,
    // which is contact order for the contacts of any one dynamic body) ----
    for (uint32_t l = 0; l < maxl; ++l) {
        for (uint32_t j = lvl[l] + lane; j < lvl[l + 1]; j += 32) {
            const uint32_t c = a.order[c0 + j];
            const uint32_t ga = w.c_a[c], gb = w.c_b[c];
            const uint32_t ba = w.geom_body[ga], bb = w.geom_body[gb];
            const Body A = load_body(w, ba), B = load_body(w, bb);
            const CParams p = ld_par(a.par, c);
            CGrad gc = ld_grad(a.gc, c);
            dm3 gRa = dm3zero(), gRb = dm3zero();
            const dm3 RA = DM(A.R), RB = DM(B.R);
            const d3 IA = D(A.I), IB = D(B.I), n = D(p.n), ra = D(p.ra), rb = D(p.rb);
            // kn = ima + imb + ran·A(ran) + rbn·B(rbn); ran = ra x n
            const d3 ran = D(cross(p.ra, p.n)), rbn = D(cross(p.rb, p.n));
            const d3 g_ran = (2.0 * gc.kn) * dapply(RA, IA, ran);
            const d3 g_rbn = (2.0 * gc.kn) * dapply(RB, IB, rbn);
            inv_I_bwd(RA, IA, ran, gc.kn * ran, gRa);
            inv_I_bwd(RB, IB, rbn, gc.kn * rbn, gRb);
            gc.ra += dcross(n, g_ran);
            gc.n += dcross(g_ran, ra);
            gc.rb += dcross(n, g_rbn);
            gc.n += dcross(g_rbn, rb);
            // bias = baum max(pen - slop, 0)/dt + e max(-vn0, 0)
            const float pen = w.c_pen[c];
            const double g_pen =
                (pen - k.slop < 0.f) ? 0.0 : gc.bias * double(k.baumgarte) / double(dt);
            const float e = gmax(w.restitution[ga], w.restitution[gb]);
            const f3 va0 = add(ld3(w.vel, ba), cross(ld3(w.omega, ba), p.ra));
            const f3 vb0 = add(ld3(w.vel, bb), cross(ld3(w.omega, bb), p.rb));
            const float vn0 = dot(sub(vb0, va0), p.n);
            const double g_vn0 = (-vn0 < 0.f) ? 0.0 : -double(e) * gc.bias;
            gc.n += g_vn0 * D(sub(vb0, va0));
            const d3 g_ub0 = g_vn0 * n, g_ua0 = -g_ub0;
            gc.ra += dcross(g_ua0, D(ld3(w.omega, ba)));
            gc.rb += dcross(g_ub0, D(ld3(w.omega, bb)));
            // mu = sqrt(fa fb)
            double gfa = 0.0, gfb = 0.0;
            if (p.mu > 0.f) {
                const double fa = w.friction[ga], fb = w.friction[gb], mu = p.mu;
                gfa = gc.mu * fb / (2.0 * mu);
                gfb = gc.mu * fa / (2.0 * mu);
            }
            // ra = cp - pos_a; rb = cp - pos_b; the contact point, normal and
            // depth through the taped support vertices
            const d3 g_cp = gc.ra + gc.rb;
            d3 gpA, gpB;
            dm3 gRA, gRB;
            contact_geom_bwd(w, k, a, c, ba, bb, gc.n, g_pen, g_cp, gpA, gpB, gRA, gRB);
            const d3 gva = g_ua0, gwa = dcross(ra, g_ua0), gvb = g_ub0, gwb = dcross(rb, g_ub0);
            if (A.fixed) {
                double* f = fix_slot(a, c, 0);
                fix_add3(f, 0, gva);
                fix_add3(f, 3, gwa);
                fix_add3(f, 6, -gc.ra);
                fix_add3(f, 6, gpA);
                fix_addR(f, gRa);
                fix_addR(f, gRA);
                f[18] += gfa;
            } else {  // the serial order of the additions, kept for bit-identical sums
                addd3(a.gv, ba, gva);
                addd3(a.gw, ba, gwa);
                g.friction[ga] += gfa;
                addd3(a.gp, ba, -gc.ra);
                add_dm3(a.gR, ba, gRa);
                addd3(a.gp, ba, gpA);
                add_dm3(a.gR, ba, gRA);
            }
            if (B.fixed) {
                double* f = fix_slot(a, c, 1);
                fix_add3(f, 0, gvb);
                fix_add3(f, 3, gwb);
                fix_add3(f, 6, -gc.rb);
                fix_add3(f, 6, gpB);
                fix_addR(f, gRb);
                fix_addR(f, gRB);
                f[18] += gfb;
            } else {
                addd3(a.gv, bb, gvb);
                addd3(a.gw, bb, gwb);
                g.friction[gb] += gfb;
                addd3(a.gp, bb, -gc.rb);
                add_dm3(a.gR, bb, gRb);
                addd3(a.gp, bb, gpB);
                add_dm3(a.gR, bb, gRB);
            }
        }
        __syncwarp();
    }

    // ---- fixed bodies: the kept contributions, in contact order ----
    if (lane == 0)
        for (uint32_t c = c0; c < c1; ++c) {
            if (a.level[c] == kNone) continue;
            for (int side = 0; side < 2; ++side) {
                const uint32_t gi = side == 0 ? w.c_a[c] : w.c_b[c];
                const uint32_t b = w.geom_body[gi];
                if (!load_body(w, b).fixed) continue;
                const double* f = fix_slot(a, c, side);
                addd3(a.gv, b, d3{f[0], f[1], f[2]});
                addd3(a.gw, b, d3{f[3], f[4], f[5]});
                addd3(a.gp, b, d3{f[6], f[7], f[8]});
                double* R = a.gR + size_t(b) * 9;
                for (int q = 0; q < 9; ++q) R[q] += f[9 + q];
                g.friction[gi] += f[18];
            }
        }
    __syncwarp();

    // ---- rotations -> quaternions, gravity (physics.comp:418-428), reversed
    for (uint32_t b = b0 + lane; b < b1; b += 32) {
        double gq[4];
        quat_bwd(w.quat[size_t(b) * 4], w.quat[size_t(b) * 4 + 1], w.quat[size_t(b) * 4 + 2],
                 w.quat[size_t(b) * 4 + 3], a.gR + size_t(b) * 9, gq);
        for (int j = 0; j < 4; ++j) g.quat[size_t(b) * 4 + j] = a.gq[size_t(b) * 4 + j] + gq[j];
        d3 Gv = ldd3(a.gv, b), Gw = ldd3(a.gw, b);
        if (w.inv_mass[b] > 0.0f) {
            Gv = double(k.lin_damp) * Gv;
            Gw = double(k.ang_damp) * Gw;
        }
        std3(g.vel, b, Gv);
        std3(g.omega, b, Gw);
        std3(g.pos, b, ldd3(a.gp, b));
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
