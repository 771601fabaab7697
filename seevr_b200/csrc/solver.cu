// solver.cu — PGS contact solver (step 5, physics.comp:500-583) and the
// impulse clear (step 4, physics.comp:494-497).
//
// Work is split into bundles: runs of whole consecutive scenes.  Scenes share
// no body, so a bundle is solved exactly like one scene whose contacts are
// the union of its scenes' (each scene's contacts keep their order, and the
// wavefront levels of different scenes simply merge); small scenes are
// bundled so that a warp's lanes have work.
//
// One CTA per bundle.  Phase 1 stages the bundle's bodies (velocity, angular
// velocity, rotation matrix, inverse inertia, inverse mass) in shared memory
// (global scratch when the scene is too large).  Phase 2 computes, for every
// contact in parallel, the values the reference recomputes on every
// iteration but which cannot change during the solve: the lever arms
// ra, rb (positions and contact points are constant), the normal effective
// mass k, the friction coefficient and the restitution/Baumgarte bias
// (taken from the pre-solve velocities, as physics.comp:504-521 does).
// Phase 3 runs the Gauss-Seidel sweeps:
//  - SEQUENTIAL: one thread, contacts in index order (physics.comp:523-582);
//  - WAVEFRONT: contacts are assigned levels so that a contact comes after
//    every earlier contact sharing a dynamic body with it; contacts of one
//    level touch disjoint dynamic bodies and run in parallel.  Each contact
//    then sees exactly the body state it sees in the sequential sweep, so the
//    result is bit-identical to SEQUENTIAL.
// A body is "fixed" when inv_mass == 0 and inv_inertia == 0: its velocities
// cannot change (the reference writes v - 0*impulse, the same value), so
// fixed bodies create no ordering constraint and are never written.
#include "common.cuh"
#include "solver.cuh"

namespace seevr {

constexpr uint32_t kSolverThreads = 128;
constexpr uint32_t kBodySmemWords = 20;  // v3 w3 R9 invI3 invm1 last1

__global__ void __launch_bounds__(kSolverThreads)
    k_solver(World w, Consts k, Scratch s, uint32_t mode, float dt, uint32_t smem_bodies) {
    extern __shared__ float sm[];
    __shared__ uint32_t sh_levels;
    if (halted(w.status)) return;  // contacts from a scan that gave up
    const uint32_t scene = blockIdx.x;  // bundle index
    const uint32_t b0 = w.bundle_off[scene], b1 = w.bundle_off[scene + 1];
    const uint32_t nbs = b1 - b0;
    const uint32_t c0 = s.bundle_c0[scene], c1 = s.bundle_c0[scene + 1];
    if (c0 >= c1) return;
    const uint32_t tid = threadIdx.x;

    // ---- phase 1: bodies ----
    const bool in_smem = nbs <= smem_bodies;
    BodyView B;
    uint32_t* last;
    if (in_smem) {
        float* p = sm;
        B.v = p; p += nbs * 3;
        B.w = p; p += nbs * 3;
        float* R = p; p += nbs * 9;
        float* invI = p; p += nbs * 3;
        float* invm = p; p += nbs;
        last = reinterpret_cast<uint32_t*>(p);
        for (uint32_t i = tid; i < nbs; i += blockDim.x) {
            const uint32_t g = b0 + i;
            st3(B.v, i, ld3(w.vel, g));
            st3(B.w, i, ld3(w.omega, g));
            st_m3(R, i, quat_to_mat(w.quat, g));
            st3(invI, i, ld3(w.inv_inertia, g));
            invm[i] = w.inv_mass[g];
            last[i] = 0;
        }
        B.R = R;
        B.invI = invI;
        B.invm = invm;
    } else {
        B.v = w.vel + size_t(b0) * 3;
        B.w = w.omega + size_t(b0) * 3;
        float* R = s.s_R + size_t(b0) * 9;
        for (uint32_t i = tid; i < nbs; i += blockDim.x) {
            st_m3(R, i, quat_to_mat(w.quat, b0 + i));
            s.s_last[b0 + i] = 0;
        }
        B.R = R;
        B.invI = w.inv_inertia + size_t(b0) * 3;
        B.invm = w.inv_mass + b0;
        last = s.s_last + b0;
        if (tid == 0) atomicOr(&s.status[0], kFlagSolverGlobal);
    }
    __syncthreads();

    // ---- phase 2: per-contact constants (physics.comp:504-521, 533-546) ----
    for (uint32_t c = c0 + tid; c < c1; c += blockDim.x) {
        const uint32_t ga = w.c_a[c], gb = w.c_b[c];
        const uint32_t a = w.geom_body[ga], b = w.geom_body[gb];
        const uint32_t la = a - b0, lb = b - b0;
        const f3 n = ld3(w.c_normal, c), cp = ld3(w.c_pos, c);
        const f3 ra = sub(cp, ld3(w.pos, a)), rb = sub(cp, ld3(w.pos, b));
        const f3 va = add(ld3(B.v, la), cross(ld3(B.w, la), ra));
        const f3 vb = add(ld3(B.v, lb), cross(ld3(B.w, lb), rb));
        const float vn = dot(sub(vb, va), n);
        const float e = gmax(w.restitution[ga], w.restitution[gb]);
        const float bias = k.baumgarte * gmax(w.c_pen[c] - k.slop, 0.0f) / dt + e * gmax(-vn, 0.0f);
        const float ima = B.invm[la], imb = B.invm[lb];
        const m3 Ra = ld_m3(B.R, la), Rb = ld_m3(B.R, lb);
        const f3 ran = cross(ra, n), rbn = cross(rb, n);
        const float kn = ima + imb + dot(ran, apply_inv_I(Ra, ld3(B.invI, la), ran)) +
                         dot(rbn, apply_inv_I(Rb, ld3(B.invI, lb), rbn));
        st3(s.s_ra, c, ra);
        st3(s.s_rb, c, rb);
        s.s_bias[c] = bias;
        s.s_kn[c] = kn;
        s.s_mu[c] = sqrtf(w.friction[ga] * w.friction[gb]);
        const bool skip = (ima == 0.0f && imb == 0.0f);  // physics.comp:531
        s.s_ab[size_t(c) * 2] = skip ? kNone : la;
        s.s_ab[size_t(c) * 2 + 1] = lb;
        w.lambda[c] = 0.0f;
    }
    __syncthreads();

    if (mode == 0) {
        // ---- SEQUENTIAL: the reference order on one thread ----
        if (tid == 0) {
            for (uint32_t it = 0; it < k.pgs_iterations; ++it)
                for (uint32_t c = c0; c < c1; ++c) {
                    const uint32_t la = s.s_ab[size_t(c) * 2];
                    if (la == kNone) continue;
                    solve_one(B, la, s.s_ab[size_t(c) * 2 + 1], ld3(w.c_normal, c), ld3(s.s_ra, c),
                              ld3(s.s_rb, c), s.s_bias[c], s.s_kn[c], s.s_mu[c], &w.lambda[c]);
                }
        }
    } else {
        // ---- WAVEFRONT: levels, counting sort by level, parallel sweeps ----
        uint32_t* lvl = s.s_lvl_start + c0 + scene;  // [levels+1], fits in [c0+scene, c1+scene]
        if (tid == 0) {
            uint32_t maxl = 0;
            for (uint32_t c = c0; c < c1; ++c) {
                const uint32_t la = s.s_ab[size_t(c) * 2];
                if (la == kNone) {
                    s.s_level[c] = kNone;
                    continue;
                }
                const uint32_t lb = s.s_ab[size_t(c) * 2 + 1];
                const bool fa = is_fixed(B, la), fb = is_fixed(B, lb);
                const uint32_t l = max(fa ? 0u : last[la], fb ? 0u : last[lb]) + 1u;
                if (!fa) last[la] = l;
                if (!fb) last[lb] = l;
                s.s_level[c] = l - 1u;
                maxl = max(maxl, l);
            }
            for (uint32_t l = 0; l <= maxl; ++l) lvl[l] = 0;
            for (uint32_t c = c0; c < c1; ++c)
                if (s.s_level[c] != kNone) lvl[s.s_level[c] + 1]++;
            for (uint32_t l = 1; l <= maxl; ++l) lvl[l] += lvl[l - 1];
            // stable fill: order[c0 + slot]; lvl[l] is used as a cursor and
            // restored afterwards
            for (uint32_t c = c0; c < c1; ++c) {
                const uint32_t l = s.s_level[c];
                if (l != kNone) s.s_order[c0 + lvl[l]++] = c;
            }
            for (uint32_t l = maxl; l > 0; --l) lvl[l] = lvl[l - 1];
            lvl[0] = 0;
            sh_levels = maxl;
        }
        __syncthreads();
        const uint32_t levels = sh_levels;
        for (uint32_t it = 0; it < k.pgs_iterations; ++it) {
            for (uint32_t l = 0; l < levels; ++l) {
                const uint32_t beg = lvl[l], end = lvl[l + 1];
                for (uint32_t i = beg + tid; i < end; i += blockDim.x) {
                    const uint32_t c = s.s_order[c0 + i];
                    solve_one(B, s.s_ab[size_t(c) * 2], s.s_ab[size_t(c) * 2 + 1],
                              ld3(w.c_normal, c), ld3(s.s_ra, c), ld3(s.s_rb, c), s.s_bias[c],
                              s.s_kn[c], s.s_mu[c], &w.lambda[c]);
                }
                __syncthreads();
            }
        }
    }
    __syncthreads();
    if (in_smem) {
        for (uint32_t i = tid; i < nbs; i += blockDim.x) {
            st3(w.vel, b0 + i, ld3(B.v, i));
            st3(w.omega, b0 + i, ld3(B.w, i));
        }
    }
}

// ---- contact range of every bundle ----------------------------------------
// Contacts are in (a, b) order and bundles own consecutive body ranges, so
// each bundle's contacts form one run; bundle_c0[k] = first contact of bundle
// k (bundle_c0[nbundles] = the contact count).  Marked in one pass instead of
// a binary search at the start of every solver block.
__global__ void k_bundle_ranges(World w, uint32_t* __restrict__ bundle_c0) {
    if (halted(w.status)) return;  // contacts from a scan that gave up
    const uint32_t nc = min(w.counters[1], w.max_contacts);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= nc; c += gridDim.x * blockDim.x) {
        const uint32_t cur = c < nc ? w.body_bundle[w.geom_body[w.c_a[c]]] : w.nbundles;
        const int prev = c > 0 ? int(w.body_bundle[w.geom_body[w.c_a[c - 1]]]) : -1;
        for (int k = prev + 1; k <= int(cur); ++k) bundle_c0[k] = c;
    }
}

// ---- block per bundle -------------------------------------------------------
// Bundles of up to kWarpMaxBodies bodies: one block of W warps per bundle;
// one warp builds the levels and records, then the block sweeps passes of up
// to 32 W same-level contacts, a barrier between passes.
// What a solve round waits on lives in shared memory: the
// bundle's velocities and angular velocities, the impulses and the level
// boundaries.  The per-contact constants are computed directly in level
// order, so the lanes of a round read consecutive entries.  Levels are
// assigned 32 contacts at a time: each lane starts from the latest level of
// its bodies in earlier chunks, then lanes are visited in order and every
// later lane sharing a dynamic body with lane j moves past lane j's level.
// One bundle per block: the SM places a bundle's 19 KB of shared memory
// wherever it fits beside other kernels (14.05 -> 13.80 ms per frame
// against four bundles per block on the 4,096-scene batch).
// W = 1 for a handle stepped alone; W = 2 for scene groups' handles, whose
// solver chains are the frame's critical path while other groups' collision
// stages fill the GPU: 64-wide passes cut the largest bundles' passes per
// iteration by about a tenth (frame 12.68 -> 12.13 ms with 8 groups on the
// 4,096-scene batch), while alone the doubled warps per SM sub-partition
// slow every pass more than that (12.52 -> 12.89 ms ungrouped).
constexpr uint32_t kMaxSweepWarps = 2;
constexpr uint32_t kWarpLamCap = 1024;   // impulses per bundle held in smem
constexpr uint32_t kWarpLevelCap = 128;  // passes held in smem
// pass entry: start position | count << kPassShift (count <= 128)
constexpr uint32_t kPassShift = 24, kPassMask = (1u << kPassShift) - 1u;
static_assert(32 * kMaxSweepWarps < (1u << (32 - kPassShift)), "pass count field too narrow");
constexpr uint32_t kRegChunks = 8;  // contacts per lane kept in registers by the setup

// A contact's record (kRecWords float4, 160 bytes): n ra rb bias kn mu,
// both bodies' rotation matrix (columns), inverse inertia and inverse mass,
// and the bundle-local body indices with each body's fixed flag in bit 31.
// The matrices are those quat_to_mat gives at every update of the sweep,
// built once here instead of at each of the 30 updates (a third fewer
// instructions than rebuilding them from quaternions in the sweep).
__device__ __forceinline__ void load_rec(const float4* __restrict__ src, float4 (&r)[kRecWords]) {
#pragma unroll
    for (uint32_t j = 0; j < kRecWords; ++j) r[j] = src[j];
}
// Contact c's record at slot q (physics.comp:504-521, 533-546): the
// constants, computed from the pre-solve velocities, and both bodies' data.
__device__ __forceinline__ void write_rec(const World& w, const Consts& k, const Scratch& s,
                                          const BodyView& B, uint32_t b0, uint32_t c, uint32_t la,
                                          uint32_t lb, uint32_t q, float dt) {
    const uint32_t ga = w.c_a[c], gb = w.c_b[c];
    const uint32_t a = b0 + la, b = b0 + lb;
    const f3 n = ld3(w.c_normal, c), cp = ld3(w.c_pos, c);
    const f3 ra = sub(cp, ld3(w.pos, a)), rb = sub(cp, ld3(w.pos, b));
    const f3 va = add(ld3(B.v, la), cross(ld3(B.w, la), ra));
    const f3 vb = add(ld3(B.v, lb), cross(ld3(B.w, lb), rb));
    const float vn = dot(sub(vb, va), n);
    const float e = gmax(w.restitution[ga], w.restitution[gb]);
    const float bias = k.baumgarte * gmax(w.c_pen[c] - k.slop, 0.0f) / dt + e * gmax(-vn, 0.0f);
    const float ima = B.invm[la], imb = B.invm[lb];
    const float4 qa = make_float4(w.quat[size_t(a) * 4], w.quat[size_t(a) * 4 + 1],
                                  w.quat[size_t(a) * 4 + 2], w.quat[size_t(a) * 4 + 3]);
    const float4 qb = make_float4(w.quat[size_t(b) * 4], w.quat[size_t(b) * 4 + 1],
                                  w.quat[size_t(b) * 4 + 2], w.quat[size_t(b) * 4 + 3]);
    const m3 Ra = quat_to_mat(qa.x, qa.y, qa.z, qa.w), Rb = quat_to_mat(qb.x, qb.y, qb.z, qb.w);
    const f3 Ia = ld3(B.invI, la), Ib = ld3(B.invI, lb);
    const f3 ran = cross(ra, n), rbn = cross(rb, n);
    const float kn = ima + imb + dot(ran, apply_inv_I(Ra, Ia, ran)) + dot(rbn, apply_inv_I(Rb, Ib, rbn));
    float4* r = s.s_rec + size_t(q) * kRecWords;
    r[0] = make_float4(n.x, n.y, n.z, ra.x);
    r[1] = make_float4(ra.y, ra.z, rb.x, rb.y);
    r[2] = make_float4(rb.z, bias, kn, sqrtf(w.friction[ga] * w.friction[gb]));
    r[3] = make_float4(Ra.c0.x, Ra.c0.y, Ra.c0.z, Ra.c1.x);
    r[4] = make_float4(Ra.c1.y, Ra.c1.z, Ra.c2.x, Ra.c2.y);
    r[5] = make_float4(Ra.c2.z, Rb.c0.x, Rb.c0.y, Rb.c0.z);
    r[6] = make_float4(Rb.c1.x, Rb.c1.y, Rb.c1.z, Rb.c2.x);
    r[7] = make_float4(Rb.c2.y, Rb.c2.z, Ia.x, Ia.y);
    r[8] = make_float4(Ia.z, Ib.x, Ib.y, Ib.z);
    r[9] = make_float4(ima, imb, __uint_as_float(la | (is_fixed(B, la) ? 0x80000000u : 0u)),
                       __uint_as_float(lb | (is_fixed(B, lb) ? 0x80000000u : 0u)));
}

// Passes of the positions [beg, pos) of one level, from entry npass on.
// kPassWidth: contacts a pass solves at once (the block's threads).
template <uint32_t kPassWidth>
__device__ __forceinline__ uint32_t write_passes(uint32_t* gpass, uint32_t npass, uint32_t beg,
                                                 uint32_t pos, uint32_t lane) {
    for (uint32_t q = beg + lane * kPassWidth; q < pos; q += 32 * kPassWidth)
        gpass[npass + (q - beg) / kPassWidth] = q | (min(kPassWidth, pos - q) << kPassShift);
    return npass + (pos - beg + kPassWidth - 1) / kPassWidth;
}

__device__ __forceinline__ void solve_rec(float* V, float* W, const float4 (&r)[kRecWords], float* lam) {
    const uint32_t xa = __float_as_uint(r[9].z), xb = __float_as_uint(r[9].w);
    const m3 Ra{mk(r[3].x, r[3].y, r[3].z), mk(r[3].w, r[4].x, r[4].y), mk(r[4].z, r[4].w, r[5].x)};
    const m3 Rb{mk(r[5].y, r[5].z, r[5].w), mk(r[6].x, r[6].y, r[6].z), mk(r[6].w, r[7].x, r[7].y)};
    solve_core(V, W, xa & 0x7FFFFFFFu, xb & 0x7FFFFFFFu, (xa >> 31) != 0, (xb >> 31) != 0, r[9].x,
               r[9].y, Ra, Rb, mk(r[7].z, r[7].w, r[8].x), mk(r[8].y, r[8].z, r[8].w),
               mk(r[0].x, r[0].y, r[0].z), mk(r[0].w, r[1].x, r[1].y), mk(r[1].z, r[1].w, r[2].x),
               r[2].y, r[2].z, r[2].w, lam);
}

__host__ __device__ constexpr uint32_t warp_smem_words(uint32_t nbmax) {
    return 7 * nbmax + kWarpLamCap + kWarpLevelCap;
}

// Levels, solve positions, pass table and contact records of one bundle,
// built by one warp (lane = its lane): returns the positions (contacts
// solved) and the passes written to gpass.
template <uint32_t kPassWidth>
__device__ __forceinline__ void bundle_setup(const World& w, const Consts& k, const Scratch& s,
                                             const BodyView& B, uint32_t mode, float dt,
                                             uint32_t b0, uint32_t c0, uint32_t c1, uint32_t nbs,
                                             uint32_t ncb, uint32_t* last, float* lam,
                                             uint32_t* gpass, uint32_t lane, uint32_t& pos_out,
                                             uint32_t& npass_out) {
    const unsigned full = 0xFFFFFFFFu;
    uint32_t maxl = 0, pos = 0, npass = 0;
    if (mode != 2 && ncb <= 32 * kRegChunks && nbs <= 0x10000u) {
        // ---- register path: each lane keeps its contacts (c0 + lane + 32 k)
        // with their bodies (two 16-bit bundle-local indices, hence at most
        // 65,536 bodies per bundle), levels and positions in registers
        const uint32_t K = (ncb + 31) / 32;
        uint32_t ab[kRegChunks], lv[kRegChunks], pk[kRegChunks];
#pragma unroll
        for (uint32_t j = 0; j < kRegChunks; ++j) {
            const uint32_t c = c0 + 32 * j + lane;
            ab[j] = 0xFFFFFFFFu;
            if (j < K && c < c1)
                ab[j] = (w.geom_body[w.c_a[c]] - b0) | ((w.geom_body[w.c_b[c]] - b0) << 16);
        }
#pragma unroll
        for (uint32_t j = 0; j < kRegChunks; ++j) {
            lv[j] = kNone;
            if (j >= K) continue;  // warp-uniform
            const bool valid = ab[j] != 0xFFFFFFFFu;
            const uint32_t la = ab[j] & 0xFFFFu, lb = ab[j] >> 16;
            // both inverse masses zero -> skipped (physics.comp:531)
            const bool use = valid && !(B.invm[la] == 0.0f && B.invm[lb] == 0.0f);
            uint32_t L = use ? 1u : 0u;
            if (mode != 0) {
                const bool da = use && !is_fixed(B, la), db = use && !is_fixed(B, lb);
                const uint32_t xa = da ? la : (0x80000000u | (lane * 2u));
                const uint32_t xb = db ? lb : (0x80000000u | (lane * 2u + 1u));
                if (use) L = max(da ? last[la] : 0u, db ? last[lb] : 0u) + 1u;
                for (uint32_t i = 0; i < 32; ++i) {
                    const uint32_t ai = __shfl_sync(full, xa, i), bi = __shfl_sync(full, xb, i);
                    const uint32_t Li = __shfl_sync(full, L, i);
                    if (use && i < lane && (ai == xa || ai == xb || bi == xa || bi == xb))
                        L = max(L, Li + 1u);
                }
                if (da) atomicMax(&last[la], L);
                if (db) atomicMax(&last[lb], L);
                __syncwarp();
            }
            if (use) lv[j] = L - 1u;
            maxl = max(maxl, L);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) maxl = max(maxl, __shfl_xor_sync(full, maxl, off));
        const unsigned below = (1u << lane) - 1u;
        for (uint32_t l = 0; l < maxl; ++l) {
            const uint32_t beg = pos;
#pragma unroll
            for (uint32_t j = 0; j < kRegChunks; ++j) {
                const bool hit = lv[j] == l;
                const unsigned m = __ballot_sync(full, hit);
                if (hit) pk[j] = pos + __popc(m & below);
                pos += __popc(m);
            }
            npass = write_passes<kPassWidth>(gpass, npass, beg, pos, lane);
        }
#pragma unroll
        for (uint32_t j = 0; j < kRegChunks; ++j) {
            if (lv[j] == kNone) continue;
            const uint32_t c = c0 + 32 * j + lane;
            s.s_order[c0 + pk[j]] = c;
            write_rec(w, k, s, B, b0, c, ab[j] & 0xFFFFu, ab[j] >> 16, c0 + pk[j], dt);
            lam[pk[j]] = 0.0f;
        }
    } else {
        // ---- memory path (colouring, or more contacts than the registers hold)
        // ---- bodies of each contact; both inverse masses zero -> skipped (531)
        for (uint32_t c = c0 + lane; c < c1; c += 32) {
            const uint32_t la = w.geom_body[w.c_a[c]] - b0, lb = w.geom_body[w.c_b[c]] - b0;
            const bool skip = B.invm[la] == 0.0f && B.invm[lb] == 0.0f;
            s.s_ab[size_t(c) * 2] = skip ? kNone : la;
            s.s_ab[size_t(c) * 2 + 1] = lb;
        }
        __syncwarp();

        // ---- levels: colours (COLORED), wavefront levels (WAVEFRONT) or one
        // level in index order (SEQUENTIAL)
        bool coloured = mode == 2;
        if (coloured) {
            // greedy colouring in contact order: the smallest colour not used by
            // an earlier contact at either of its dynamic bodies (per-body colour
            // masks in `last`); more than 32 colours at a body falls back to the
            // wavefront levels
            uint32_t ok = 1u, mx = 0u;
            if (lane == 0) {
                for (uint32_t c = c0; c < c1; ++c) {
                    const uint32_t la = s.s_ab[size_t(c) * 2], lb = s.s_ab[size_t(c) * 2 + 1];
                    if (la == kNone) {
                        s.s_level[c] = kNone;
                        continue;
                    }
                    const bool da = !is_fixed(B, la), db = !is_fixed(B, lb);
                    const uint32_t used = (da ? last[la] : 0u) | (db ? last[lb] : 0u);
                    if (used == 0xFFFFFFFFu) {
                        ok = 0u;
                        break;
                    }
                    const uint32_t col = uint32_t(__ffs(int(~used))) - 1u;
                    if (da) last[la] |= 1u << col;
                    if (db) last[lb] |= 1u << col;
                    s.s_level[c] = col;
                    mx = max(mx, col + 1u);
                }
            }
            ok = __shfl_sync(full, ok, 0);
            maxl = __shfl_sync(full, mx, 0);
            if (!ok) {
                coloured = false;
                maxl = 0;
                for (uint32_t i = lane; i < nbs; i += 32) last[i] = 0;
            }
            __syncwarp();
        }
        for (uint32_t cb = c0; !coloured && cb < c1; cb += 32) {
            const uint32_t c = cb + lane;
            const bool valid = c < c1;
            const uint32_t la = valid ? s.s_ab[size_t(c) * 2] : kNone;
            const uint32_t lb = valid ? s.s_ab[size_t(c) * 2 + 1] : 0u;
            const bool use = valid && la != kNone;
            uint32_t L = use ? 1u : 0u;
            if (mode != 0) {
                const bool da = use && !is_fixed(B, la), db = use && !is_fixed(B, lb);
                // dynamic bodies, or a sentinel unique to this lane and role
                const uint32_t xa = da ? la : (0x80000000u | (lane * 2u));
                const uint32_t xb = db ? lb : (0x80000000u | (lane * 2u + 1u));
                if (use) L = max(da ? last[la] : 0u, db ? last[lb] : 0u) + 1u;
                for (uint32_t j = 0; j < 32; ++j) {
                    const uint32_t aj = __shfl_sync(full, xa, j), bj = __shfl_sync(full, xb, j);
                    const uint32_t Lj = __shfl_sync(full, L, j);
                    if (use && j < lane && (aj == xa || aj == xb || bj == xa || bj == xb))
                        L = max(L, Lj + 1u);
                }
                if (da) atomicMax(&last[la], L);
                if (db) atomicMax(&last[lb], L);
            }
            if (valid) s.s_level[c] = use ? L - 1u : kNone;
            maxl = max(maxl, L);
            __syncwarp();
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) maxl = max(maxl, __shfl_xor_sync(full, maxl, off));

        // ---- positions: contacts grouped by level, index order within a level;
        // passes: runs of at most kPassWidth positions of one level,
        // the unit the lanes solve together.  A pass holds at least one contact,
        // so the passes fit in [c0 + bundle, c1 + bundle] of s_lvl_start.
        for (uint32_t l = 0; l < maxl; ++l) {
            const uint32_t beg = pos;
            for (uint32_t cb = c0; cb < c1; cb += 32) {
                const uint32_t c = cb + lane;
                const bool hit = c < c1 && s.s_level[c] == l;
                const unsigned m = __ballot_sync(full, hit);
                if (hit) s.s_order[c0 + pos + __popc(m & ((1u << lane) - 1u))] = c;
                pos += __popc(m);
            }
            npass = write_passes<kPassWidth>(gpass, npass, beg, pos, lane);
        }
        __syncwarp();
        for (uint32_t i = lane; i < pos; i += 32) {
            const uint32_t c = s.s_order[c0 + i];
            write_rec(w, k, s, B, b0, c, s.s_ab[size_t(c) * 2], s.s_ab[size_t(c) * 2 + 1], c0 + i, dt);
            lam[i] = 0.0f;
        }
    }
    pos_out = pos;
    npass_out = npass;
}

// Barrier of a W-warp block.
template <uint32_t W>
__device__ __forceinline__ void block_sync() {
    if (W == 1)
        __syncwarp();
    else
        __syncthreads();
}

template <uint32_t W>
__global__ void __launch_bounds__(32 * W)
    k_solver_warp(World w, Consts k, Scratch s, uint32_t mode, float dt, uint32_t nbmax) {
    constexpr uint32_t kSweepThreads = 32 * W;
    // nbmax: bodies per warp held in shared memory; a bundle with more
    // bodies (a single scene above the bundle size) solves on the bound
    // velocity buffers in place
    extern __shared__ float sm[];
    if (halted(w.status)) return;  // contacts from a scan that gave up
    const uint32_t t = threadIdx.x, lane = t & 31u, wid = t >> 5;
    const uint32_t bundle = blockIdx.x;
    if (bundle >= w.nbundles) return;
    const uint32_t b0 = w.bundle_off[bundle], b1 = w.bundle_off[bundle + 1];
    const uint32_t c0 = s.bundle_c0[bundle], c1 = s.bundle_c0[bundle + 1];
    if (c0 >= c1) return;
    const uint32_t nbs = b1 - b0, ncb = c1 - c0;
    // pass entries hold a position in kPassShift bits: a bundle with more
    // contacts runs the sequential sweep, which has no pass table and gives
    // the same result bit for bit
    if (ncb > kPassMask) mode = 0;

    float* base = sm;
    const bool in_smem = nbs <= nbmax;
    float* V = in_smem ? base : w.vel + size_t(b0) * 3;
    float* Wv = in_smem ? base + 3 * nbmax : w.omega + size_t(b0) * 3;
    uint32_t* last = in_smem ? reinterpret_cast<uint32_t*>(base + 6 * nbmax) : s.s_last + b0;
    float* lam = ncb <= kWarpLamCap ? base + 7 * nbmax : s.s_lam + c0;
    uint32_t* lvl_sm = reinterpret_cast<uint32_t*>(base + 7 * nbmax + kWarpLamCap);
    for (uint32_t i = t; i < nbs; i += kSweepThreads) {
        if (in_smem) {
            st3(V, i, ld3(w.vel, b0 + i));
            st3(Wv, i, ld3(w.omega, b0 + i));
        }
        last[i] = 0;
    }
    block_sync<W>();
    BodyView B{V, Wv, nullptr, w.inv_inertia + size_t(b0) * 3, w.inv_mass + b0};

    uint32_t* gpass = s.s_lvl_start + c0 + bundle;
    uint32_t pos = 0, npass = 0;
    if (W == 1) {
        bundle_setup<kSweepThreads>(w, k, s, B, mode, dt, b0, c0, c1, nbs, ncb, last, lam, gpass,
                                    lane, pos, npass);
        __syncwarp();
    } else {
        __shared__ uint32_t sh_counts[2];
        if (wid == 0) {
            bundle_setup<kSweepThreads>(w, k, s, B, mode, dt, b0, c0, c1, nbs, ncb, last, lam,
                                        gpass, lane, pos, npass);
            if (lane == 0) {
                sh_counts[0] = pos;
                sh_counts[1] = npass;
            }
        }
        __syncthreads();
        pos = sh_counts[0];
        npass = sh_counts[1];
    }
    const bool pass_sm = npass <= kWarpLevelCap;
    if (pass_sm)
        for (uint32_t j = t; j < npass; j += kSweepThreads) lvl_sm[j] = gpass[j];
    block_sync<W>();
    const uint32_t* pass = pass_sm ? lvl_sm : gpass;

    // ---- Gauss-Seidel sweeps ----
    if (mode == 0) {
        if (t == 0) {
            float4 r[kRecWords];
            for (uint32_t it = 0; it < k.pgs_iterations; ++it)
                for (uint32_t i = 0; i < pos; ++i) {
                    load_rec(s.s_rec + size_t(c0 + i) * kRecWords, r);
                    solve_rec(V, Wv, r, &lam[i]);
                }
        }
    } else if (npass > 0) {
        // the next pass's records are loaded while this pass solves
        float4 cur[kRecWords], nxt[kRecWords];
        uint32_t pe = pass[0];
        if (t < (pe >> kPassShift))
            load_rec(s.s_rec + size_t(c0 + (pe & kPassMask) + t) * kRecWords, nxt);
        const uint32_t total = k.pgs_iterations * npass;
        uint32_t p = 0;
        for (uint32_t q = 0; q < total; ++q) {
#pragma unroll
            for (uint32_t j = 0; j < kRecWords; ++j) cur[j] = nxt[j];
            const uint32_t ce = pe;
            p = p + 1 == npass ? 0u : p + 1;
            pe = pass[p];
            if (q + 1 < total && t < (pe >> kPassShift))
                load_rec(s.s_rec + size_t(c0 + (pe & kPassMask) + t) * kRecWords, nxt);
            if (t < (ce >> kPassShift)) solve_rec(V, Wv, cur, &lam[(ce & kPassMask) + t]);
            block_sync<W>();
        }
    }
    block_sync<W>();
    // ---- results back to the bound buffers ----
    if (in_smem)
        for (uint32_t i = t; i < nbs; i += kSweepThreads) {
            st3(w.vel, b0 + i, ld3(V, i));
            st3(w.omega, b0 + i, ld3(Wv, i));
        }
    for (uint32_t i = t; i < pos; i += kSweepThreads) w.lambda[s.s_order[c0 + i]] = lam[i];
}

constexpr uint32_t kSolverMaxSmem = 160 * 1024;

cudaError_t init_solver() {
    const int bytes = int(warp_smem_words(kWarpMaxBodies) * sizeof(float));
    cudaError_t e = cudaFuncSetAttribute(k_solver_warp<1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_solver_warp<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    // opt in to more than 48 KB of dynamic shared memory; done at handle
    // creation so that no attribute call happens during graph capture
    return cudaFuncSetAttribute(k_solver, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(kSolverMaxSmem));
}

int launch_bundle_ranges(const World& w, const Scratch& s, cudaStream_t st) {
    uint32_t rb = (w.max_contacts + 1 + 255) / 256;
    if (rb > 148u * 8u) rb = 148u * 8u;
    k_bundle_ranges<<<rb, 256, 0, st>>>(w, s.bundle_c0);
    return 1;
}

int launch_solver(const World& w, const Consts& k, const Scratch& s, uint32_t mode, float dt,
                  uint32_t max_scene_bodies, uint32_t smem_bodies, cudaStream_t st) {
    if (w.nbundles == 0 || w.max_contacts == 0) return 0;
    launch_bundle_ranges(w, s, st);
    if (max_scene_bodies <= kWarpMaxBodies) {
        uint32_t nbmax = smem_bodies < max_scene_bodies ? smem_bodies : max_scene_bodies;
        if (nbmax == 0) nbmax = 1;
        const size_t smem = warp_smem_words(nbmax) * sizeof(float);
        if (s.sweep_warps >= 2)
            k_solver_warp<2><<<w.nbundles, 64, smem, st>>>(w, k, s, mode, dt, nbmax);
        else
            k_solver_warp<1><<<w.nbundles, 32, smem, st>>>(w, k, s, mode, dt, nbmax);
        return 2;
    }
    if (s.isl.parent) return 1 + launch_solver_islands(w, k, s, mode, dt, st);
    uint32_t cta_bodies = max_scene_bodies;
    if (cta_bodies * kBodySmemWords * 4 > kSolverMaxSmem)
        cta_bodies = kSolverMaxSmem / (kBodySmemWords * 4);
    const size_t smem = size_t(cta_bodies) * kBodySmemWords * 4;
    k_solver<<<w.nbundles, kSolverThreads, smem, st>>>(w, k, s, mode, dt, cta_bodies);
    return 2;
}

}  // namespace seevr
