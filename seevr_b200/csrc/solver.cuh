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
// indexed by la / lb; a fixed body's velocities are not written.  The
// vector arithmetic runs on packed FP32 pairs (the p3 forms of vmath.cuh),
// equal to the scalar expressions bit for bit: a warp's update issues fewer
// instructions, which the warps sharing an SM sub-partition compete for.
__device__ __forceinline__ void solve_core(float* V, float* W, uint32_t la, uint32_t lb, bool fixed_a,
                                           bool fixed_b, float ima, float imb, const m3& Ra_,
                                           const m3& Rb_, f3 Ia_, f3 Ib_, f3 n_, f3 ra_, f3 rb_,
                                           float bias, float kn, float mu, float* lam) {
    const pm3 Ra = pkm(Ra_), Rb = pkm(Rb_);
    const p3 Ia = pk(Ia_), Ib = pk(Ib_), n = pk(n_), ra = pk(ra_), rb = pk(rb_);
    p3 va = pk(ld3(V, la)), wa = pk(ld3(W, la)), vb = pk(ld3(V, lb)), wb = pk(ld3(W, lb));
    p3 ua = padd(va, pcross(wa, ra)), ub = padd(vb, pcross(wb, rb));
    const float vn = pdot(psub(ub, ua), n);
    float d_ln = (-vn + bias) / kn;
    const float old_ln = *lam;
    const float new_ln = gmax(old_ln + d_ln, 0.0f);
    d_ln = new_ln - old_ln;
    *lam = new_ln;
    const p3 imp = pscale(d_ln, n);
    va = psub(va, pscale(ima, imp));
    vb = padd(vb, pscale(imb, imp));
    wa = psub(wa, papply_inv_I(Ra, Ia, pcross(ra, imp)));
    wb = padd(wb, papply_inv_I(Rb, Ib, pcross(rb, imp)));
    // Coulomb friction along the current slip direction
    ua = padd(va, pcross(wa, ra));
    ub = padd(vb, pcross(wb, rb));
    const p3 dv = psub(ub, ua);
    const p3 vt = psub(dv, pscale(pdot(dv, n), n));
    const float vt_len = sqrtf(pdot(vt, vt));
    if (vt_len > 1e-6f) {
        const p3 td = p3{make_float2(vt.xy.x / vt_len, vt.xy.y / vt_len), vt.z / vt_len};
        const p3 rat = pcross(ra, td), rbt = pcross(rb, td);
        const float kt = ima + imb + pdot(rat, papply_inv_I(Ra, Ia, rat)) +
                         pdot(rbt, papply_inv_I(Rb, Ib, rbt));
        const float d_lt = gmin(vt_len / kt, mu * new_ln);
        const p3 it = pscale(d_lt, td);
        va = padd(va, pscale(ima, it));
        vb = psub(vb, pscale(imb, it));
        wa = padd(wa, papply_inv_I(Ra, Ia, pcross(ra, it)));
        wb = psub(wb, papply_inv_I(Rb, Ib, pcross(rb, it)));
    }
    if (!fixed_a) {
        st3(V, la, up(va));
        st3(W, la, up(wa));
    }
    if (!fixed_b) {
        st3(V, lb, up(vb));
        st3(W, lb, up(wb));
    }
}

__device__ __forceinline__ void solve_one(const BodyView& B, uint32_t la, uint32_t lb, f3 n, f3 ra,
                                          f3 rb, float bias, float kn, float mu, float* lam) {
    solve_core(B.v, B.w, la, lb, is_fixed(B, la), is_fixed(B, lb), B.invm[la], B.invm[lb],
               ld_m3(B.R, la), ld_m3(B.R, lb), ld3(B.invI, la), ld3(B.invI, lb), n, ra, rb, bias,
               kn, mu, lam);
}

}  // namespace seevr
