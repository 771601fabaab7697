// solver.cuh — one PGS contact update (physics.comp:525-580) over a view of
// the body state, shared by the bundle (solver.cu) and island (islands.cu)
// solvers.
#pragma once
#include "common.cuh"

namespace seevr {

struct BodyView {
    float* v;           // [n*3]
    float* w;           // [n*3]
    const float* R;     // [n*9]
    const float* invI;  // [n*3]
    const float* invm;  // [n]
};

__device__ __forceinline__ bool is_fixed(const BodyView& B, uint32_t i) {
    return B.invm[i] == 0.0f && B.invI[i * 3] == 0.0f && B.invI[i * 3 + 1] == 0.0f &&
           B.invI[i * 3 + 2] == 0.0f;
}

// One normal + friction update of contact c (physics.comp:525-580), given
// the two bodies' constant data; v, w: velocities and angular velocities,
// indexed by la / lb; a fixed body's velocities are not written.
__device__ __forceinline__ void solve_core(float* V, float* W, uint32_t la, uint32_t lb, bool fixed_a,
                                           bool fixed_b, float ima, float imb, const m3& Ra,
                                           const m3& Rb, f3 Ia, f3 Ib, f3 n, f3 ra, f3 rb,
                                           float bias, float kn, float mu, float* lam) {
    f3 va = ld3(V, la), wa = ld3(W, la), vb = ld3(V, lb), wb = ld3(W, lb);
    f3 ua = add(va, cross(wa, ra)), ub = add(vb, cross(wb, rb));
    const float vn = dot(sub(ub, ua), n);
    float d_ln = (-vn + bias) / kn;
    const float old_ln = *lam;
    const float new_ln = gmax(old_ln + d_ln, 0.0f);
    d_ln = new_ln - old_ln;
    *lam = new_ln;
    const f3 imp = scale(d_ln, n);
    va = sub(va, scale(ima, imp));
    vb = add(vb, scale(imb, imp));
    wa = sub(wa, apply_inv_I(Ra, Ia, cross(ra, imp)));
    wb = add(wb, apply_inv_I(Rb, Ib, cross(rb, imp)));
    // Coulomb friction along the current slip direction
    ua = add(va, cross(wa, ra));
    ub = add(vb, cross(wb, rb));
    const f3 dv = sub(ub, ua);
    const f3 vt = sub(dv, scale(dot(dv, n), n));
    const float vt_len = length(vt);
    if (vt_len > 1e-6f) {
        const f3 td = divs(vt, vt_len);
        const f3 rat = cross(ra, td), rbt = cross(rb, td);
        const float kt = ima + imb + dot(rat, apply_inv_I(Ra, Ia, rat)) + dot(rbt, apply_inv_I(Rb, Ib, rbt));
        const float d_lt = gmin(vt_len / kt, mu * new_ln);
        const f3 it = scale(d_lt, td);
        va = add(va, scale(ima, it));
        vb = sub(vb, scale(imb, it));
        wa = add(wa, apply_inv_I(Ra, Ia, cross(ra, it)));
        wb = sub(wb, apply_inv_I(Rb, Ib, cross(rb, it)));
    }
    if (!fixed_a) {
        st3(V, la, va);
        st3(W, la, wa);
    }
    if (!fixed_b) {
        st3(V, lb, vb);
        st3(W, lb, wb);
    }
}

__device__ __forceinline__ void solve_one(const BodyView& B, uint32_t la, uint32_t lb, f3 n, f3 ra,
                                          f3 rb, float bias, float kn, float mu, float* lam) {
    solve_core(B.v, B.w, la, lb, is_fixed(B, la), is_fixed(B, lb), B.invm[la], B.invm[lb],
               ld_m3(B.R, la), ld_m3(B.R, lb), ld3(B.invI, la), ld3(B.invI, lb), n, ra, rb, bias,
               kn, mu, lam);
}

}  // namespace seevr
