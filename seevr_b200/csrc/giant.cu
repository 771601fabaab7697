// giant.cu — grid-wide coloured PGS for giant islands.
//
// The island solver (islands.cu) gives each island one warp.  When stacks
// collapse into one heap, a single island can hold hundreds of thousands of
// contacts, and its warp then runs the sweep alone while the rest of the GPU
// idles (about a second per frame for 262,144 boxes).  In the coloured mode
// (SEEVR_SOLVER_COLORED, where the Gauss-Seidel order is the colour order,
// not the reference's contact order) islands above kGiantContacts contacts
// are solved here instead, by every SM at once, in one cooperative launch:
//   1. collect the giant islands' contacts;
//   2. colour them in parallel (Jones-Plassmann rounds: a contact takes a
//      colour once its priority is the highest among the uncoloured
//      contacts at each of its dynamic bodies; the colour is the smallest
//      one unused at both bodies).  Priorities are a hash of the contact's
//      index, so colours do not depend on the schedule;
//   3. group the contacts by colour;
//   4. per-contact constants (physics.comp:504-521, 533-546);
//   5. PGS_ITERATIONS sweeps, one colour at a time across the whole grid:
//      contacts of one colour share no dynamic body, so they run in parallel
//      and the result does not depend on which thread takes which contact.
// A grid barrier separates the phases; every wait is bounded by the
// handle's wait limit and gives up (raising kFlagTimeout) when another
// block has already done so.  Body state lives in global memory and is read
// past L1 (ld.global.cg), since other SMs write it between barriers.
#include "common.cuh"
#include "solver.cuh"

namespace seevr {

constexpr uint32_t kGiantThreads = 256;
constexpr uint32_t kMaskColours = 64;  // colours tracked per body; more: one per round
constexpr uint32_t kMaxRounds = 1024;
constexpr uint32_t kMaxColours = kMaskColours + kMaxRounds;
static_assert(kMaxColours == kGiantMaxColours, "colour table size");

namespace {

__device__ __forceinline__ uint32_t ldcg(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ f3 ld3cg(const float* p, uint32_t i) {
    return mk(__ldcg(p + size_t(i) * 3), __ldcg(p + size_t(i) * 3 + 1), __ldcg(p + size_t(i) * 3 + 2));
}

// Grid barrier of a cooperative launch: arrival count bar[0] and a
// generation word bar[kGenWord], a cache line apart so that the polls of
// the waiting blocks do not contend with the arrivals.  Returns false, after
// raising kFlagTimeout, when the wait exceeds `limit` polls or another
// block has given up (checked every 64 polls).
constexpr uint32_t kGenWord = 32;
__device__ bool grid_sync(uint32_t* bar, uint32_t* status, uint32_t limit) {
    __shared__ uint32_t sh_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ok = 1u;
        volatile uint32_t* gen = bar + kGenWord;
        const uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == gridDim.x - 1u) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(&bar[kGenWord], 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g) {
                if (++spins > limit || ((spins & 63u) == 0u && halted(status))) {
                    atomicOr(status, kFlagTimeout);
                    ok = 0u;
                    break;
                }
            }
        }
        __threadfence();
        sh_ok = ok;
    }
    __syncthreads();
    return sh_ok != 0u;
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {  // a 32-bit integer mix
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ bool fixed_body(const World& w, uint32_t b) {
    return w.inv_mass[b] == 0.0f && w.inv_inertia[size_t(b) * 3] == 0.0f &&
           w.inv_inertia[size_t(b) * 3 + 1] == 0.0f && w.inv_inertia[size_t(b) * 3 + 2] == 0.0f;
}

// One normal + friction update (solve_core's arithmetic) with the bodies'
// velocities read past L1.
__device__ __forceinline__ void solve_global(const World& w, const Scratch& s, uint32_t q) {
    const uint32_t a = s.s_abp[size_t(q) * 2], b = s.s_abp[size_t(q) * 2 + 1];
    const bool fa = fixed_body(w, a), fb = fixed_body(w, b);
    // solve_core works on body views: the two bodies' fresh velocities as
    // local bodies 0 (a) and 1 (b), which stay in registers
    const f3 Va = ld3cg(w.vel, a), Wa = ld3cg(w.omega, a), Vb = ld3cg(w.vel, b),
             Wb = ld3cg(w.omega, b);
    float V[6] = {Va.x, Va.y, Va.z, Vb.x, Vb.y, Vb.z};
    float W[6] = {Wa.x, Wa.y, Wa.z, Wb.x, Wb.y, Wb.z};
    float lam = __ldcg(&s.s_lam[q]);
    solve_core(V, W, 0u, 1u, fa, fb, w.inv_mass[a], w.inv_mass[b], ld_m3(s.s_R, a), ld_m3(s.s_R, b),
               ld3(w.inv_inertia, a), ld3(w.inv_inertia, b), ld3(s.s_n, q), ld3(s.s_ra, q),
               ld3(s.s_rb, q), s.s_bias[q], s.s_kn[q], s.s_mu[q], &lam);
    s.s_lam[q] = lam;
    if (!fa) {
        st3(w.vel, a, mk(V[0], V[1], V[2]));
        st3(w.omega, a, mk(W[0], W[1], W[2]));
    }
    if (!fb) {
        st3(w.vel, b, mk(V[3], V[4], V[5]));
        st3(w.omega, b, mk(W[3], W[4], W[5]));
    }
}

__global__ void __launch_bounds__(kGiantThreads)
    k_solver_giant(World w, Consts k, Scratch s, float dt, uint32_t threshold) {
    if (halted(w.status)) return;
    GiantScratch& g = s.isl.giant;
    uint32_t* bar = g.ctr;        // [0] and [kGenWord]: barrier
    uint32_t* n_giant = g.ctr + 2;
    uint32_t* n_coloured = g.ctr + 3;
    uint32_t* n_colours = g.ctr + 4;
    const uint32_t limit = s.wait_limit;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t count = *s.isl.count;
    const uint32_t npos = s.isl.start[count];

    // ---- 1. the giant islands' contact positions ----
    for (uint32_t i = tid; i < npos; i += stride) {
        const uint32_t isl = s.isl.idx[i] + s.isl.head[i] - 1u;
        if (s.isl.start[isl + 1] - s.isl.start[isl] <= threshold) continue;
        g.list[atomicAdd(n_giant, 1u)] = i;
        const uint32_t c = s.isl.perm[i];
        const uint32_t a = w.geom_body[w.c_a[c]], b = w.geom_body[w.c_b[c]];
        s.s_abp[size_t(i) * 2] = a;
        s.s_abp[size_t(i) * 2 + 1] = b;
        g.used[a] = 0ull;
        g.used[b] = 0ull;
        g.prio[a] = 0ull;
        g.prio[b] = 0ull;
        g.colour[i] = kNone;
    }
    if (!grid_sync(bar, w.status, limit)) return;
    const uint32_t ng = ldcg(n_giant);
    if (ng == 0) return;
    if (tid == 0) atomicOr(w.status, kFlagGiantIslands);

    // ---- 2. Jones-Plassmann colouring ----
    for (uint32_t r = 0;; ++r) {
        if (r >= kMaxRounds) {
            if (tid == 0) atomicOr(w.status, kFlagTimeout);
            return;
        }
        const uint64_t tag = uint64_t(r + 1) << 48;
        for (uint32_t e = tid; e < ng; e += stride) {
            const uint32_t i = ldcg(&g.list[e]);
            if (ldcg(&g.colour[i]) != kNone) continue;
            const uint32_t c = s.isl.perm[i];
            const uint64_t v = tag | (uint64_t(hash32(c) & 0xFFFFFFu) << 24) | (c & 0xFFFFFFu);
            const uint32_t a = s.s_abp[size_t(i) * 2], b = s.s_abp[size_t(i) * 2 + 1];
            if (!fixed_body(w, a)) atomicMax(reinterpret_cast<unsigned long long*>(&g.prio[a]), v);
            if (!fixed_body(w, b)) atomicMax(reinterpret_cast<unsigned long long*>(&g.prio[b]), v);
        }
        if (!grid_sync(bar, w.status, limit)) return;
        for (uint32_t e = tid; e < ng; e += stride) {
            const uint32_t i = ldcg(&g.list[e]);
            if (ldcg(&g.colour[i]) != kNone) continue;
            const uint32_t c = s.isl.perm[i];
            const uint64_t v = tag | (uint64_t(hash32(c) & 0xFFFFFFu) << 24) | (c & 0xFFFFFFu);
            const uint32_t a = s.s_abp[size_t(i) * 2], b = s.s_abp[size_t(i) * 2 + 1];
            const bool da = !fixed_body(w, a), db = !fixed_body(w, b);
            const unsigned long long* P = reinterpret_cast<const unsigned long long*>(g.prio);
            if (da && __ldcg(P + a) != v) continue;
            if (db && __ldcg(P + b) != v) continue;
            // the highest-priority uncoloured contact at both bodies: no
            // other contact at a or b takes a colour this round
            const unsigned long long* U = reinterpret_cast<const unsigned long long*>(g.used);
            const uint64_t ua = da ? __ldcg(U + a) : 0ull, ub = db ? __ldcg(U + b) : 0ull;
            const uint64_t used = ua | ub;
            uint32_t col;
            if (~used != 0ull) {
                col = uint32_t(__ffsll(static_cast<long long>(~used))) - 1u;
                if (da) g.used[a] = ua | (1ull << col);
                if (db) g.used[b] = ub | (1ull << col);
            } else {
                col = kMaskColours + r;  // every mask colour taken: a colour of this round's own
            }
            g.colour[i] = col;
            atomicMax(n_colours, col + 1u);
            atomicAdd(n_coloured, 1u);
        }
        if (!grid_sync(bar, w.status, limit)) return;
        if (ldcg(n_coloured) >= ng) break;
    }

    // ---- 3. contacts grouped by colour ----
    const uint32_t nc = ldcg(n_colours);
    for (uint32_t e = tid; e < ng; e += stride)
        atomicAdd(&g.hist[ldcg(&g.colour[ldcg(&g.list[e])])], 1u);
    if (!grid_sync(bar, w.status, limit)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t col = 0; col < nc; ++col) {
            const uint32_t h = ldcg(&g.hist[col]);
            g.hist[col] = run;            // cursor
            g.first[col] = run;           // first slot of the colour
            run += h;
        }
        g.first[nc] = run;
    }
    if (!grid_sync(bar, w.status, limit)) return;
    for (uint32_t e = tid; e < ng; e += stride) {
        const uint32_t i = ldcg(&g.list[e]);
        g.order[atomicAdd(&g.hist[ldcg(&g.colour[i])], 1u)] = i;
    }

    // ---- 4. per-contact constants from the pre-solve velocities ----
    for (uint32_t e = tid; e < ng; e += stride) {
        const uint32_t i = ldcg(&g.list[e]), c = s.isl.perm[i];
        const uint32_t ga = w.c_a[c], gb = w.c_b[c];
        const uint32_t a = s.s_abp[size_t(i) * 2], b = s.s_abp[size_t(i) * 2 + 1];
        const f3 n = ld3(w.c_normal, c), cp = ld3(w.c_pos, c);
        const f3 ra = sub(cp, ld3(w.pos, a)), rb = sub(cp, ld3(w.pos, b));
        const f3 va = add(ld3cg(w.vel, a), cross(ld3cg(w.omega, a), ra));
        const f3 vb = add(ld3cg(w.vel, b), cross(ld3cg(w.omega, b), rb));
        const float vn = dot(sub(vb, va), n);
        const float e_r = gmax(w.restitution[ga], w.restitution[gb]);
        const float bias = k.baumgarte * gmax(w.c_pen[c] - k.slop, 0.0f) / dt + e_r * gmax(-vn, 0.0f);
        const m3 Ra = ld_m3(s.s_R, a), Rb = ld_m3(s.s_R, b);
        const f3 ran = cross(ra, n), rbn = cross(rb, n);
        const float kn = w.inv_mass[a] + w.inv_mass[b] +
                         dot(ran, apply_inv_I(Ra, ld3(w.inv_inertia, a), ran)) +
                         dot(rbn, apply_inv_I(Rb, ld3(w.inv_inertia, b), rbn));
        st3(s.s_n, i, n);
        st3(s.s_ra, i, ra);
        st3(s.s_rb, i, rb);
        s.s_bias[i] = bias;
        s.s_kn[i] = kn;
        s.s_mu[i] = sqrtf(w.friction[ga] * w.friction[gb]);
        s.s_lam[i] = 0.0f;
    }
    if (!grid_sync(bar, w.status, limit)) return;

    // ---- 5. sweeps, colour by colour ----
    for (uint32_t it = 0; it < k.pgs_iterations; ++it)
        for (uint32_t col = 0; col < nc; ++col) {
            const uint32_t j0 = ldcg(&g.first[col]), j1 = ldcg(&g.first[col + 1]);
            if (j0 == j1) continue;
            for (uint32_t j = j0 + tid; j < j1; j += stride) solve_global(w, s, ldcg(&g.order[j]));
            if (!grid_sync(bar, w.status, limit)) return;
        }
    for (uint32_t e = tid; e < ng; e += stride) {
        const uint32_t i = ldcg(&g.list[e]);
        w.lambda[s.isl.perm[i]] = __ldcg(&s.s_lam[i]);
    }
}

}  // namespace

int launch_solver_giant(const World& w, const Consts& k, const Scratch& s, float dt,
                        cudaStream_t st) {
    const GiantScratch& g = s.isl.giant;
    if (!g.list || w.max_contacts > (1u << 24)) return 0;  // priorities hold 24-bit indices
    // one block per SM: each grid barrier waits for as few arrivals as the
    // grid can have while every SM works (towers after their collapse: 45
    // against 49 ms per frame with two blocks per SM)
    const int per_sm = 1;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaMemsetAsync(g.ctr, 0, kGiantCtrWords * sizeof(uint32_t), st);
    cudaMemsetAsync(g.hist, 0, sizeof(uint32_t) * kMaxColours, st);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(uint32_t(sms) * uint32_t(per_sm));
    cfg.blockDim = dim3(kGiantThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_solver_giant, w, k, s, dt, s.giant_min ? s.giant_min : kGiantContacts);
    return 1;
}

}  // namespace seevr
