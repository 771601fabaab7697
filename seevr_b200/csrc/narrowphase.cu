// narrowphase.cu — MPR narrowphase (step 3, physics.comp:475-491) with the
// support function (physics.comp:107-169) and Minkowski Portal Refinement
// (physics.comp:171-399), plus deterministic contact compaction.
//
// MPR's cost per pair varies by an order of magnitude (separated pairs stop
// after one or two support calls; touching pairs refine and search the
// penetration for tens).  With one pair per thread, a warp waits for its
// slowest lane.  Here every lane runs MPR as a state machine whose steps
// each make exactly one Minkowski support call:
//   D1   first support along -v0           (physics.comp:254-271)
//   D2   second support                     (272-287)
//   DT   portal discovery trials            (289-319)
//   R    portal refinement                  (323-343)
//   P    penetration search                 (346-365)
// and a lane whose pair finishes takes the next pair from a global counter
// (warp-aggregated atomics), so all lanes stay busy until the pair list is
// exhausted and converge on the support call, the expensive part of a step.
// The arithmetic and the order of every test are those of the reference
// loops, so each pair's result is the same bit for bit.
//
// The contact found for pair p is staged at slot p; a scan over the found
// flags then writes contacts in pair order, where the reference appends with
// atomicAdd (physics.comp:404).
#include "common.cuh"

namespace seevr {

constexpr uint32_t kNarrowThreads = 128;
constexpr uint32_t kNarrowThreadsW = kNarrowThreads;  // witness slots per thread row

// A pair's two shapes: hull range and lookup offset in registers; rotation
// and position in shared memory (Pose), read at each support call, so that
// the state a lane carries from step to step fits its register budget.
struct Shape {
    uint32_t vs, vc, lk;
};

struct Pose {
    float (*q)[12][kNarrowThreadsW];  // [shape][R by columns, p][thread]
    uint32_t t;
    __device__ __forceinline__ void put(uint32_t i, const m3& R, f3 p) const {
        q[i][0][t] = R.c0.x; q[i][1][t] = R.c0.y; q[i][2][t] = R.c0.z;
        q[i][3][t] = R.c1.x; q[i][4][t] = R.c1.y; q[i][5][t] = R.c1.z;
        q[i][6][t] = R.c2.x; q[i][7][t] = R.c2.y; q[i][8][t] = R.c2.z;
        q[i][9][t] = p.x; q[i][10][t] = p.y; q[i][11][t] = p.z;
    }
    __device__ __forceinline__ m3 R(uint32_t i) const {
        m3 m;
        m.c0 = mk(q[i][0][t], q[i][1][t], q[i][2][t]);
        m.c1 = mk(q[i][3][t], q[i][4][t], q[i][5][t]);
        m.c2 = mk(q[i][6][t], q[i][7][t], q[i][8][t]);
        return m;
    }
    __device__ __forceinline__ f3 p(uint32_t i) const { return mk(q[i][9][t], q[i][10][t], q[i][11][t]); }
};

__device__ __forceinline__ Shape load_shape(const World& w, uint32_t b, const Pose& P, uint32_t i) {
    P.put(i, quat_to_mat(w.quat, b), ld3(w.pos, b));
    return Shape{w.hull_range[size_t(b) * 2], w.hull_range[size_t(b) * 2 + 1], lut_of(w, b)};
}

// support (physics.comp:107-162).  Both paths of the reference visit a list
// of candidate vertices in order and keep the first strict maximum: all
// hull vertices when lk == 0 (brute force), else for each of the 3 axes the
// two lookup bins around the direction's angle.  The lookup path issues its
// six entry loads, then its six vertex loads, each level at once (two
// dependent memory latencies per call instead of twelve); pairs are ordered
// by path (k_pair_classes), so a warp's lanes mostly take the same one.
__device__ __forceinline__ f3 support_rp(const World& w, const Shape& s, const m3& R, f3 pos,
                                         f3 d, uint32_t& chosen) {
    const f3 ld = mulT(R, d);
    float best = -1e10f;
    f3 bv = mk(0.f, 0.f, 0.f);
    chosen = kNone;  // no vertex beat -1e10: the support point is the body position
    if (s.lk != 0) {
        // the angle bins of the X, Y, Z axes (atan(z,y), atan(z,x),
        // atan(y,x)); then the six lookup entries, then the six candidate
        // vertices, all loads of a level in flight together; compared in
        // the reference's order
        const uint32_t bins[3] = {angle_bin64(ld.z, ld.y), angle_bin64(ld.z, ld.x),
                                  angle_bin64(ld.y, ld.x)};
        uint32_t idx[6];
#pragma unroll
        for (uint32_t ax = 0; ax < 3; ++ax) {
            const uint32_t b0 = bins[ax];
            idx[2 * ax] = w.sup_lut[s.lk + ax * 64u + b0];
            idx[2 * ax + 1] = w.sup_lut[s.lk + ax * 64u + (b0 + 1u) % 64u];
        }
        f3 v[6];
#pragma unroll
        for (uint32_t k = 0; k < 6; ++k) v[k] = ld3(w.hull, s.vs + idx[k]);
#pragma unroll
        for (uint32_t k = 0; k < 6; ++k) {
            const float dd = dot(v[k], ld);
            if (dd > best) {
                best = dd;
                bv = v[k];
                chosen = idx[k];
            }
        }
        return add(pos, mul(R, bv));
    }
    for (uint32_t k = 0; k < s.vc; ++k) {
        const f3 v = ld3(w.hull, s.vs + k);
        const float dd = dot(v, ld);
        if (dd > best) {
            best = dd;
            bv = v;
            chosen = k;
        }
    }
    return add(pos, mul(R, bv));
}

__device__ __forceinline__ f3 support(const World& w, const Shape& s, const Pose& P, uint32_t i,
                                      f3 d, uint32_t& chosen) {
    return support_rp(w, s, P.R(i), P.p(i), d, chosen);
}

// A Minkowski support point (mink_support_pts, physics.comp:165-169): its
// value v = sa - sb stays in registers, while the supporting points sa, sb
// (and, for the adjoint's tape, the hull-relative indices of the supporting
// vertices) are kept in one of four shared-memory slots per lane, named by
// `slot`.  The portal's three points and the step's fresh point always hold
// four different slots, so a point entering the portal frees the slot of
// the one it replaces.  Only the contact point (find_pos) and the segment
// case read sa and sb, so keeping them out of registers costs one store per
// support call and lets the lane's state fit the register budget of seven
// resident blocks per SM.
struct Mink {
    f3 v;
    uint32_t slot;
};

template <bool kTape>
struct Witness {
    static constexpr uint32_t kWords = kTape ? 8 : 6;  // sa xyz, sb xyz (, ia, ib)
    float (*w)[kWords][kNarrowThreadsW];               // [slot][word][thread]
    uint32_t t;
    __device__ __forceinline__ void put(uint32_t slot, f3 sa, f3 sb, uint32_t ia, uint32_t ib) const {
        w[slot][0][t] = sa.x; w[slot][1][t] = sa.y; w[slot][2][t] = sa.z;
        w[slot][3][t] = sb.x; w[slot][4][t] = sb.y; w[slot][5][t] = sb.z;
        if (kTape) {
            w[slot][kWords - 2][t] = __uint_as_float(ia);
            w[slot][kWords - 1][t] = __uint_as_float(ib);
        }
    }
    __device__ __forceinline__ f3 sa(uint32_t slot) const {
        return mk(w[slot][0][t], w[slot][1][t], w[slot][2][t]);
    }
    __device__ __forceinline__ f3 sb(uint32_t slot) const {
        return mk(w[slot][3][t], w[slot][4][t], w[slot][5][t]);
    }
    __device__ __forceinline__ uint32_t ia(uint32_t slot) const {
        return __float_as_uint(w[slot][kWords - 2][t]);
    }
    __device__ __forceinline__ uint32_t ib(uint32_t slot) const {
        return __float_as_uint(w[slot][kWords - 1][t]);
    }
};

// dst takes the fresh point m (held in slot `free`): dst's old slot becomes
// the free one.
__device__ __forceinline__ void take(Mink& dst, const Mink& m, uint32_t& free) {
    free = dst.slot;
    dst = m;
}

__device__ __forceinline__ f3 portal_dir(f3 v1, f3 v2, f3 v3) {
    return normalize(cross(sub(v2, v1), sub(v3, v1)));
}
__device__ __forceinline__ bool reach_tol(const Consts& k, f3 v1, f3 v2, f3 v3, f3 v4, f3 dir) {
    const float dv1 = dot(v1, dir), dv2 = dot(v2, dir), dv3 = dot(v3, dir), dv4 = dot(v4, dir);
    const float dot1 = gmin(gmin(dv4 - dv1, dv4 - dv2), dv4 - dv3);
    return dot1 < k.tol + k.eps * gmax(1.0f, dot1);
}

// mpr_expand_portal (physics.comp:200-221)
__device__ __forceinline__ void expand(const f3& v0, Mink& m1, Mink& m2, Mink& m3, const Mink& m4,
                                       uint32_t& free) {
    const f3 v4v0 = cross(m4.v, v0);
    float d = dot(m1.v, v4v0);
    if (d > 0.0f) {
        d = dot(m2.v, v4v0);
        if (d > 0.0f) take(m1, m4, free);
        else take(m3, m4, free);
    } else {
        d = dot(m3.v, v4v0);
        if (d > 0.0f) take(m2, m4, free);
        else take(m1, m4, free);
    }
}

// mpr_find_pos (physics.comp:224-247); s0a, s0b are the body positions
template <bool kTape>
__device__ f3 find_pos(const Consts& k, f3 v0, f3 s0a, f3 s0b, const Mink& m1, const Mink& m2,
                       const Mink& m3, const Witness<kTape>& W) {
    const f3 v1 = m1.v, v2 = m2.v, v3 = m3.v;
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
    const f3 p1 = add(add(add(scale(b0, s0a), scale(b1, W.sa(m1.slot))), scale(b2, W.sa(m2.slot))),
                      scale(b3, W.sa(m3.slot)));
    const f3 p2 = add(add(add(scale(b0, s0b), scale(b1, W.sb(m1.slot))), scale(b2, W.sb(m2.slot))),
                      scale(b3, W.sb(m3.slot)));
    return scale(0.5f / sum, add(p1, p2));
}

enum MprState : uint32_t { kD1 = 0, kD2 = 1, kDT = 2, kR = 3, kP = 4 };

// Record pair p's outcome (physics.comp:486-489: a contact when found and
// depth > 0).
__device__ __forceinline__ void finish(float4* res0, float4* res1, uint32_t* flag, uint32_t p,
                                       bool found, f3 cp, f3 n, float depth) {
    const bool keep = found && depth > 0.0f;
    flag[p] = keep ? 1u : 0u;
    if (keep) {
        res0[p] = make_float4(cp.x, cp.y, cp.z, depth);
        res1[p] = make_float4(n.x, n.y, n.z, 0.0f);
    }
}

// kTape: also record, per pair, which hull vertices support the final
// portal (tape[2p] = {case, m1.ia, m1.ib, m2.ia}, tape[2p+1] = {m2.ib,
// m3.ia, m3.ib, 0}; case 1 = penetration portal, 2 = the segment case of
// physics.comp:267-271), from which the adjoint differentiates the contact.
// kMinBlocks: resident blocks per SM the register allocation is capped for
// (7: 72 registers with a few spilled values; 6: about 80, no spills).
template <bool kTape, uint32_t kMinBlocks>
__global__ void __launch_bounds__(kNarrowThreads, kMinBlocks)
    k_narrow(World w, Consts k, float4* __restrict__ res0, float4* __restrict__ res1,
             uint32_t* __restrict__ flag, uint32_t* __restrict__ ticket,
             uint4* __restrict__ tape, const uint32_t* __restrict__ order) {
    __shared__ float wit[4][Witness<kTape>::kWords][kNarrowThreadsW];
    __shared__ float pose[2][12][kNarrowThreadsW];
    if (halted(w.status)) return;  // pairs from a scan that gave up
    const uint32_t np = min(w.counters[0], w.max_pairs);
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned full = 0xFFFFFFFFu;
    const Witness<kTape> W{wit, threadIdx.x};
    const Pose P{pose, threadIdx.x};

    bool active = false, drained = false;
    uint32_t p = 0, state = kD1, iter = 0;
    Shape A, B;
    f3 v0 = mk(0, 0, 0), dir = mk(0, 0, 0);
    Mink m1{mk(0, 0, 0), 0}, m2{mk(0, 0, 0), 1}, m3{mk(0, 0, 0), 2};
    uint32_t free = 3;

    while (true) {
        // ---- refill idle lanes with the next pairs ----
        if (!drained) {
            const unsigned need = __ballot_sync(full, !active);
            if (need) {
                const uint32_t leader = __ffs(need) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(ticket, uint32_t(__popc(need)));
                base = __shfl_sync(full, base, leader);
                if (base + __popc(need) >= np) drained = true;
                if (!active) {
                    const uint32_t q = base + __popc(need & ((1u << lane) - 1u));
                    if (q < np) {
                        p = order ? order[q] : q;
                        const uint32_t a = w.pairs[size_t(p) * 2], b = w.pairs[size_t(p) * 2 + 1];
                        A = load_shape(w, a, P, 0);
                        B = load_shape(w, b, P, 1);
                        v0 = sub(ld3(w.pos, a), ld3(w.pos, b));  // s0a - s0b (physics.comp:254-258)
                        if (fabsf(v0.x) < k.eps && fabsf(v0.y) < k.eps && fabsf(v0.z) < k.eps)
                            v0.x += 10.0f * k.eps;
                        dir = normalize(neg(v0));
                        state = kD1;
                        iter = 0;
                        active = true;
                    }
                }
            }
        }
        if (__ballot_sync(full, active) == 0u) break;
        if (!active) continue;

        // ---- prelude: the direction of this step's support call ----
        if (state == kR) {
            dir = portal_dir(m1.v, m2.v, m3.v);
            if (dot(m1.v, dir) > -k.eps) {  // origin inside: refine returns 0
                state = kP;
                iter = 0;
                if (k.mpr_iterations == 0) {
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                    continue;
                }
            }
        } else if (state == kP) {
            dir = portal_dir(m1.v, m2.v, m3.v);
        }

        // ---- the one Minkowski support call of the step ----
        Mink m;
        {
            uint32_t ia, ib;
            const f3 sa = support(w, A, P, 0, dir, ia);
            const f3 sb = support(w, B, P, 1, neg(dir), ib);
            m.v = sub(sa, sb);
            m.slot = free;
            W.put(free, sa, sb, ia, ib);
        }

        // ---- postlude ----
        switch (state) {
            case kD1: {
                if (dot(m.v, dir) < k.eps) {
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                    break;
                }
                take(m1, m, free);
                const f3 c = cross(v0, m1.v);
                if (dot(c, c) < k.eps) {
                    const f3 v1 = m1.v;
                    f3 n;
                    float depth;
                    if (fabsf(v1.x) < k.eps && fabsf(v1.y) < k.eps && fabsf(v1.z) < k.eps) {
                        n = normalize(v0);  // touching: res == 1
                        depth = 0.0f;
                    } else {
                        depth = length(v1);  // origin on segment v0-v1: res == 2
                        n = normalize(v1);
                    }
                    if (kTape) {
                        tape[size_t(p) * 2] = make_uint4(2u, W.ia(m1.slot), W.ib(m1.slot), 0u);
                        tape[size_t(p) * 2 + 1] = make_uint4(0u, 0u, 0u, 0u);
                    }
                    finish(res0, res1, flag, p, true,
                           scale(0.5f, add(W.sa(m1.slot), W.sb(m1.slot))), n, depth);
                    active = false;
                    break;
                }
                dir = normalize(c);
                state = kD2;
                break;
            }
            case kD2: {
                if (dot(m.v, dir) < k.eps) {
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                    break;
                }
                take(m2, m, free);
                dir = normalize(cross(sub(m1.v, v0), sub(m2.v, v0)));
                if (dot(dir, v0) > 0.0f) {
                    const Mink t = m1;
                    m1 = m2;
                    m2 = t;
                    dir = neg(dir);
                }
                iter = 0;  // discovery trials
                state = kDT;
                if (k.discover_trials == 0) {
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                }
                break;
            }
            case kDT: {
                if (dot(m.v, dir) < k.eps) {
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                    break;
                }
                bool retry = false;
                if (dot(cross(m1.v, m.v), v0) < -k.eps) {
                    take(m2, m, free);
                    retry = true;
                } else if (dot(cross(m.v, m2.v), v0) < -k.eps) {
                    take(m1, m, free);
                    retry = true;
                }
                if (retry) {
                    dir = normalize(cross(sub(m1.v, v0), sub(m2.v, v0)));
                    if (++iter >= k.discover_trials) {
                        finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                        active = false;
                    }
                    break;
                }
                take(m3, m, free);  // portal found: refine
                iter = 0;
                state = kR;
                if (k.mpr_iterations == 0) {  // refine returns 1, penetration finds nothing
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                }
                break;
            }
            case kR: {
                if (!(dot(m.v, dir) > -k.eps) || reach_tol(k, m1.v, m2.v, m3.v, m.v, dir)) {
                    finish(res0, res1, flag, p, false, v0, v0, 0.0f);
                    active = false;
                    break;
                }
                expand(v0, m1, m2, m3, m, free);
                if (++iter >= k.mpr_iterations) {  // refine returns 1: go on to penetration
                    iter = 0;
                    state = kP;
                }
                break;
            }
            default: {  // kP
                if (reach_tol(k, m1.v, m2.v, m3.v, m.v, dir) || iter >= k.mpr_iterations - 1) {
                    const float depth = dot(dir, m1.v);
                    if (kTape) {
                        tape[size_t(p) * 2] =
                            make_uint4(1u, W.ia(m1.slot), W.ib(m1.slot), W.ia(m2.slot));
                        tape[size_t(p) * 2 + 1] =
                            make_uint4(W.ib(m2.slot), W.ia(m3.slot), W.ib(m3.slot), 0u);
                    }
                    finish(res0, res1, flag, p, true,
                           find_pos(k, v0, P.p(0), P.p(1), m1, m2, m3, W), dir, depth);
                    active = false;
                    break;
                }
                expand(v0, m1, m2, m3, m, free);
                ++iter;
                break;
            }
        }
    }
}

// ---- GJK + EPA -----------------------------------------------------------------
// The alternative narrowphase (seevr_params.narrowphase = GJK_EPA; no
// counterpart in the reference, whose shader has MPR only).  Gilbert-Johnson-
// Keerthi finds a tetrahedron of Minkowski points enclosing the origin; the
// expanding polytope algorithm grows it toward the boundary of A-B until the
// face nearest the origin is within tolerance: its normal and distance are the
// contact normal and depth, and the barycentric coordinates of the origin's
// projection weight the witness points into the contact point.  One thread
// per pair, the polytope in local memory (32 points, 64 faces); the
// arithmetic and the order of every test are those of the oracle's gjk_epa,
// so results are equal bit for bit.
struct SPt {
    f3 v, sa, sb;
};
constexpr uint32_t kGjkIters = 64, kEpaIters = 64, kEpaMaxV = 32, kEpaMaxF = 64, kEpaMaxE = 96;

struct PairShapes {
    Shape A, B;
    m3 Ra, Rb;
    f3 pa, pb;
};

__device__ __forceinline__ SPt mink_pt(const World& w, const PairShapes& q, f3 d) {
    uint32_t ia, ib;
    SPt p;
    p.sa = support_rp(w, q.A, q.Ra, q.pa, d, ia);
    p.sb = support_rp(w, q.B, q.Rb, q.pb, neg(d), ib);
    p.v = sub(p.sa, p.sb);
    return p;
}

__device__ __forceinline__ bool gjk_line(SPt* s, uint32_t& n, f3& d) {
    const f3 a = s[n - 1].v, b = s[n - 2].v;
    const f3 ab = sub(b, a), ao = neg(a);
    if (dot(ab, ao) > 0.0f) {
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

__device__ __forceinline__ bool gjk_triangle(SPt* s, uint32_t& n, f3& d) {  // s = [c, b, a]
    const f3 a = s[2].v, b = s[1].v, c = s[0].v;
    const f3 ab = sub(b, a), ac = sub(c, a), ao = neg(a);
    const f3 abc = cross(ab, ac);
    if (dot(cross(abc, ac), ao) > 0.0f) {
        if (dot(ac, ao) > 0.0f) {
            s[1] = s[2];
            n = 2;
            d = cross(cross(ac, ao), ac);
            return false;
        }
        s[0] = s[1];
        s[1] = s[2];
        n = 2;
        return gjk_line(s, n, d);
    }
    if (dot(cross(ab, abc), ao) > 0.0f) {
        s[0] = s[1];
        s[1] = s[2];
        n = 2;
        return gjk_line(s, n, d);
    }
    if (dot(abc, ao) > 0.0f) {
        d = abc;
    } else {
        const SPt t = s[0];
        s[0] = s[1];
        s[1] = t;
        d = neg(abc);
    }
    return false;
}

__device__ __forceinline__ bool gjk_tetra(SPt* s, uint32_t& n, f3& d) {  // s = [d, c, b, a]
    const f3 a = s[3].v, b = s[2].v, c = s[1].v, dd = s[0].v;
    const f3 ab = sub(b, a), ac = sub(c, a), ad = sub(dd, a), ao = neg(a);
    if (dot(cross(ab, ac), ao) > 0.0f) {
        s[0] = s[1];
        s[1] = s[2];
        s[2] = s[3];
        n = 3;
        return gjk_triangle(s, n, d);
    }
    if (dot(cross(ac, ad), ao) > 0.0f) {
        s[2] = s[3];
        n = 3;
        return gjk_triangle(s, n, d);
    }
    if (dot(cross(ad, ab), ao) > 0.0f) {
        const SPt t = s[0];
        s[0] = s[2];
        s[1] = t;
        s[2] = s[3];
        n = 3;
        return gjk_triangle(s, n, d);
    }
    return true;
}

struct Face {
    uint32_t i, j, k;
    f3 n;
    float dist;
};

__device__ __forceinline__ Face make_face(const SPt* v, uint32_t i, uint32_t j, uint32_t k) {
    Face f{i, j, k, mk(0.f, 0.f, 0.f), 1e30f};
    const f3 n = cross(sub(v[j].v, v[i].v), sub(v[k].v, v[i].v));
    const float l = length(n);
    if (l > 0.0f) {
        f.n = divs(n, l);
        f.dist = dot(f.n, v[i].v);
    }
    return f;
}

// GJK + EPA for one pair; false: no contact.
__device__ bool gjk_epa(const World& w, const Consts& k, const PairShapes& q, f3& normal,
                        float& depth, f3& cp) {
    SPt v[kEpaMaxV];
    const float e2 = k.eps * k.eps;
    // ---- GJK ----
    f3 d = sub(q.pa, q.pb);
    if (dot(d, d) < e2) d = mk(1.f, 0.f, 0.f);
    v[0] = mink_pt(w, q, d);
    uint32_t n = 1;
    d = neg(v[0].v);
    bool in = false;
    for (uint32_t it = 0; it < kGjkIters && !in; ++it) {
        if (dot(d, d) < e2) return false;  // the origin lies on the simplex: touching
        const SPt p = mink_pt(w, q, d);
        if (dot(p.v, d) <= 0.0f) return false;  // A-B does not reach past the origin
        v[n++] = p;
        in = n == 2 ? gjk_line(v, n, d) : n == 3 ? gjk_triangle(v, n, d) : gjk_tetra(v, n, d);
    }
    if (!in) return false;
    // ---- EPA ----
    Face f[kEpaMaxF];
    uint32_t nv = 4, nf = 0;
    const uint32_t tri[4][4] = {{3, 2, 1, 0}, {3, 1, 0, 2}, {3, 0, 2, 1}, {2, 0, 1, 3}};
    for (uint32_t t = 0; t < 4; ++t) {
        Face g = make_face(v, tri[t][0], tri[t][1], tri[t][2]);
        if (dot(g.n, sub(v[tri[t][3]].v, v[tri[t][0]].v)) > 0.0f)
            g = make_face(v, tri[t][0], tri[t][2], tri[t][1]);
        f[nf++] = g;
    }
    Face g{};
    for (uint32_t it = 0;; ++it) {
        uint32_t best = 0;
        for (uint32_t i = 1; i < nf; ++i)
            if (f[i].dist < f[best].dist) best = i;
        g = f[best];
        if (it >= kEpaIters || nv == kEpaMaxV) break;
        const SPt p = mink_pt(w, q, g.n);
        const float dp = dot(p.v, g.n);
        if (dp - g.dist < k.tol + k.eps * gmax(1.0f, dp)) break;
        uint32_t e[kEpaMaxE][2], ne = 0, keep = 0;
        bool full = false;
        for (uint32_t i = 0; i < nf; ++i) {
            if (dot(f[i].n, sub(p.v, v[f[i].i].v)) > 0.0f) {
                const uint32_t ed[3][2] = {{f[i].i, f[i].j}, {f[i].j, f[i].k}, {f[i].k, f[i].i}};
                for (uint32_t t = 0; t < 3; ++t) {
                    uint32_t r = 0;
                    while (r < ne && !(e[r][0] == ed[t][1] && e[r][1] == ed[t][0])) ++r;
                    if (r < ne) {
                        for (uint32_t u = r; u + 1 < ne; ++u) {
                            e[u][0] = e[u + 1][0];
                            e[u][1] = e[u + 1][1];
                        }
                        --ne;
                    } else if (ne < kEpaMaxE) {
                        e[ne][0] = ed[t][0];
                        e[ne][1] = ed[t][1];
                        ++ne;
                    } else {
                        full = true;
                    }
                }
            } else {
                f[keep++] = f[i];
            }
        }
        if (full || keep + ne > kEpaMaxF) break;
        nf = keep;
        v[nv] = p;
        for (uint32_t r = 0; r < ne; ++r) f[nf++] = make_face(v, e[r][0], e[r][1], nv);
        ++nv;
    }
    if (!(g.dist < 1e30f)) return false;
    normal = g.n;
    depth = g.dist;
    const f3 A = v[g.i].v, B = v[g.j].v, C = v[g.k].v;
    const f3 e0 = sub(B, A), e1 = sub(C, A), e2v = sub(scale(g.dist, g.n), A);
    const float d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1);
    const float d20 = dot(e2v, e0), d21 = dot(e2v, e1);
    const float den = d00 * d11 - d01 * d01;
    float wb = 1.0f / 3.0f, wc = 1.0f / 3.0f;
    if (fabsf(den) > e2) {
        wb = (d11 * d20 - d01 * d21) / den;
        wc = (d00 * d21 - d01 * d20) / den;
    }
    const float wa = 1.0f - wb - wc;
    const f3 pa = add(add(scale(wa, v[g.i].sa), scale(wb, v[g.j].sa)), scale(wc, v[g.k].sa));
    const f3 pb = add(add(scale(wa, v[g.i].sb), scale(wb, v[g.j].sb)), scale(wc, v[g.k].sb));
    cp = scale(0.5f, add(pa, pb));
    return true;
}

__global__ void __launch_bounds__(128)
    k_gjk_epa(World w, Consts k, float4* __restrict__ res0, float4* __restrict__ res1,
              uint32_t* __restrict__ flag, const uint32_t* __restrict__ order) {
    if (halted(w.status)) return;
    const uint32_t np = min(w.counters[0], w.max_pairs);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x) {
        const uint32_t p = order ? order[t] : t;
        const uint32_t a = w.pairs[size_t(p) * 2], b = w.pairs[size_t(p) * 2 + 1];
        PairShapes q;
        q.A = Shape{w.hull_range[size_t(a) * 2], w.hull_range[size_t(a) * 2 + 1], lut_of(w, a)};
        q.B = Shape{w.hull_range[size_t(b) * 2], w.hull_range[size_t(b) * 2 + 1], lut_of(w, b)};
        q.Ra = quat_to_mat(w.quat, a);
        q.Rb = quat_to_mat(w.quat, b);
        q.pa = ld3(w.pos, a);
        q.pb = ld3(w.pos, b);
        f3 n = mk(0.f, 0.f, 0.f), cp = n;
        float depth = 0.0f;
        const bool found = gjk_epa(w, k, q, n, depth, cp);
        finish(res0, res1, flag, p, found, cp, n, depth);
    }
}

// ---- pair order by support path ---------------------------------------------
// A warp's lanes run their pairs' support calls together; a shape with a
// support lookup (lk != 0) takes three angle bins and six candidates, one
// without walks all its hull vertices.  Taking the pairs grouped by the two
// shapes' paths (4 classes) keeps a warp's lanes on one path, and within a
// class the broadphase's order, in which neighbouring pairs share a body
// (and its hull in cache).  Each pair's result is staged at its own index,
// so the order changes no result.  Scene groups' handles take it (their
// partial-size launches run beside other groups' kernels: 12.15 against
// 12.52 ms per frame with 8 groups); a single handle takes the pairs in the
// broadphase's order, which keeps every pair beside the neighbours that
// share its bodies (12.62 against 13.52 ms per frame).  (Reordering only
// within chunks of 256 pairs fell between the two in both settings;
// putting pairs whose bounding spheres overlap first, as longer MPR runs,
// measured 11% slower.)
__device__ __forceinline__ uint32_t pair_class(const World& w, uint32_t p) {
    const uint32_t a = w.pairs[size_t(p) * 2], b = w.pairs[size_t(p) * 2 + 1];
    return (w.sup_off[a] != 0u ? 2u : 0u) | (w.sup_off[b] != 0u ? 1u : 0u);
}

// cls[0..3]: pairs per class; cls[4..7]: placement cursors (zeroed before)
template <bool kScatter>
__global__ void k_pair_classes(World w, uint32_t* __restrict__ cls, uint32_t* __restrict__ order) {
    if (halted(w.status)) return;
    const uint32_t np = min(w.counters[0], w.max_pairs);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t pre[kPairClasses];
    pre[0] = 0;
#pragma unroll
    for (uint32_t k = 1; k < kPairClasses; ++k) pre[k] = kScatter ? pre[k - 1] + cls[k - 1] : 0u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t p0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); p0 < np; p0 += stride) {
        const uint32_t p = p0 + lane;
        const uint32_t c = p < np ? pair_class(w, p) : kPairClasses;
#pragma unroll
        for (uint32_t k = 0; k < kPairClasses; ++k) {
            const unsigned m = __ballot_sync(0xFFFFFFFFu, c == k);
            if (!m) continue;
            const uint32_t leader = __ffs(m) - 1;
            uint32_t base = 0;
            if (lane == leader)
                base = atomicAdd(&cls[kScatter ? kPairClasses + k : k], uint32_t(__popc(m)));
            if (kScatter) {
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (c == k) order[pre[k] + base + __popc(m & ((1u << lane) - 1u))] = p;
            }
        }
    }
}

static uint32_t grid_for(uint32_t cap, uint32_t threads, uint32_t max_blocks) {
    uint32_t g = (cap + threads - 1) / threads;
    if (g > max_blocks) g = max_blocks;
    return g ? g : 1;
}

// ---- shared lookup tables ------------------------------------------------------
// Scene builders give every geom with a lookup its own table (data.zig:299-353),
// though all UV spheres of one segment count have identical ones: the bench
// batch holds about 250,000 copies of one 768-byte table, which the support
// calls would read from 190 MB.  Per frame, the first body with a lookup of
// each hull size is found, and a body whose table equals that body's entry
// for entry reads it instead: the same indices, one copy in cache.
__global__ void k_lut_reps(World w, uint32_t* __restrict__ rep) {
    if (check_failed(w.status)) return;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.nb; b += gridDim.x * blockDim.x) {
        if (w.sup_off[b] == 0u) continue;
        const uint32_t hc = w.hull_range[size_t(b) * 2 + 1];
        // most bodies find a smaller one already there: a plain read first
        // keeps them off the contended word
        if (hc < kLutHullMax && b < *reinterpret_cast<volatile uint32_t*>(&rep[hc]))
            atomicMin(&rep[hc], b);
    }
}

__global__ void k_lut_alias(World w, const uint32_t* __restrict__ rep, uint32_t* __restrict__ out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    if (check_failed(w.status)) return;
    for (uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < w.nb; b += nwarps) {
        const uint32_t lk = w.sup_off[b];
        uint32_t res = lk;
        if (lk != 0u) {
            const uint32_t hc = w.hull_range[size_t(b) * 2 + 1];
            const uint32_t r = hc < kLutHullMax ? rep[hc] : kNone;
            if (r != kNone && r != b) {
                const uint32_t lr = w.sup_off[r];
                bool same = true;
                for (uint32_t k = lane; k < 192u; k += 32u) same &= w.sup_lut[lk + k] == w.sup_lut[lr + k];
                if (__all_sync(0xFFFFFFFFu, same)) res = lr;
            }
        }
        if (lane == 0) out[b] = res;
    }
}

int launch_lut_alias(const World& w, const Scratch& s, cudaStream_t st) {
    if (!s.lut_off || w.nb == 0) return 0;
    cudaMemsetAsync(s.lut_rep, 0xFF, sizeof(uint32_t) * kLutHullMax, st);
    const uint32_t blocks = grid_for(w.nb, 256, 148 * 8);
    k_lut_reps<<<blocks, 256, 0, st>>>(w, s.lut_rep);
    // a warp per body, 8 per block
    k_lut_alias<<<grid_for(w.nb, 8, 148 * 16), 256, 0, st>>>(w, s.lut_rep, s.lut_off);
    return 2;
}

// add_contact (physics.comp:403-412) at the scanned slot.
__global__ void k_contact_scatter(World w, const float4* __restrict__ res0,
                                  const float4* __restrict__ res1,
                                  const uint32_t* __restrict__ flag,
                                  const uint32_t* __restrict__ coff,
                                  const uint4* __restrict__ pair_tape,
                                  uint4* __restrict__ contact_tape) {
    if (halted(w.status)) return;  // offsets from a scan that gave up
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
        w.lambda[c] = 0.0f;  // step 4 (physics.comp:494-497) for the contacts of this substep
        if (contact_tape) {
            contact_tape[size_t(c) * 2] = pair_tape[size_t(p) * 2];
            contact_tape[size_t(c) * 2 + 1] = pair_tape[size_t(p) * 2 + 1];
        }
    }
}

int launch_narrowphase_taped(const World& w, const Consts& k, const Scratch& s, uint4* pair_tape,
                             uint4* contact_tape, cudaStream_t st) {
    if (w.max_pairs == 0) return 0;
    // persistent grid: a few resident blocks per SM; the pair ticket lives
    // in status[1] and is cleared here
    cudaMemsetAsync(&s.status[1], 0, sizeof(uint32_t), st);
    const uint32_t blocks = grid_for(w.max_pairs, kNarrowThreads,
                                     s.narrow_blocks ? s.narrow_blocks : 148 * kNarrowBlocksPerSm);
    // the register budget of seven blocks per SM when that many are resident,
    // else the larger one of six
    const bool seven = (s.narrow_per_sm ? s.narrow_per_sm : kNarrowBlocksPerSm) >= 7;
    // pair order by support path, in pair_coff (free until the scan below)
    const uint32_t* order = nullptr;
    int n = 3;
    if (s.pair_class && s.order_pairs) {
        cudaMemsetAsync(s.pair_class, 0, 2 * kPairClasses * sizeof(uint32_t), st);
        const uint32_t cb = grid_for(w.max_pairs, 256, 148 * 8);
        k_pair_classes<false><<<cb, 256, 0, st>>>(w, s.pair_class, nullptr);
        k_pair_classes<true><<<cb, 256, 0, st>>>(w, s.pair_class, s.pair_coff);
        order = s.pair_coff;
        n += 2;
    }
    if (k.narrowphase == 1u && !pair_tape) {  // GJK + EPA (the adjoint tapes MPR only)
        k_gjk_epa<<<grid_for(w.max_pairs, 128, uint32_t(148 * 16)), 128, 0, st>>>(
            w, k, s.pair_res0, s.pair_res1, s.pair_flag, order);
    } else if (pair_tape) {
        if (seven)
            k_narrow<true, 7><<<blocks, kNarrowThreads, 0, st>>>(
                w, k, s.pair_res0, s.pair_res1, s.pair_flag, &s.status[1], pair_tape, order);
        else
            k_narrow<true, 6><<<blocks, kNarrowThreads, 0, st>>>(
                w, k, s.pair_res0, s.pair_res1, s.pair_flag, &s.status[1], pair_tape, order);
    } else {
        if (seven)
            k_narrow<false, 7><<<blocks, kNarrowThreads, 0, st>>>(
                w, k, s.pair_res0, s.pair_res1, s.pair_flag, &s.status[1], nullptr, order);
        else
            k_narrow<false, 6><<<blocks, kNarrowThreads, 0, st>>>(
                w, k, s.pair_res0, s.pair_res1, s.pair_flag, &s.status[1], nullptr, order);
    }
    launch_exclusive_scan(s.pair_flag, s.pair_coff, &w.counters[0], w.max_pairs,
                          &w.counters[1], w.max_contacts, kFlagContactOverflow, s, st);
    k_contact_scatter<<<grid_for(w.max_pairs, 256, 148 * 16), 256, 0, st>>>(
        w, s.pair_res0, s.pair_res1, s.pair_flag, s.pair_coff, pair_tape,
        pair_tape ? contact_tape : nullptr);
    return n;
}

int launch_narrowphase(const World& w, const Consts& k, const Scratch& s, cudaStream_t st) {
    return launch_narrowphase_taped(w, k, s, nullptr, nullptr, st);
}

}  // namespace seevr
