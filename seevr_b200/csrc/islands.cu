// islands.cu — island-parallel PGS for scenes too large for one warp.
//
// Two contacts interact in the Gauss-Seidel sweep only through a dynamic
// body they share, so the contact graph's connected components (islands,
// static bodies excluded) can be solved independently: every contact of an
// island sees exactly the body state it would see in the sequential sweep
// over the whole scene, so WAVEFRONT stays bit-identical to SEQUENTIAL.  A
// pile of 262,144 boxes in 1,024 towers is 1,024 islands; one warp per
// island replaces one block per scene.
//
// Per substep:
//   1. union-find over the dynamic bodies of every contact (lock-free
//      hooking of the larger root under the smaller, so the final root of a
//      component is its smallest body index, whatever the schedule);
//   2. key = island root per contact (skipped contacts sort last), and a
//      stable radix sort of (key, contact), which keeps each island's
//      contacts in index order;
//   3. island starts from the key changes (one exclusive scan);
//   4. a persistent grid of warps takes islands in turn: levels (WAVEFRONT),
//      greedy colours (COLORED) or one level (SEQUENTIAL), then the sweep
//      with the body state in place in global memory.
#include "common.cuh"
#include "lbvh.cuh"
#include "solver.cuh"

namespace seevr {
namespace {

constexpr uint32_t kIslandThreads = 128;
constexpr uint32_t kNoKey = 0xFFFFFFFFu;

__device__ __forceinline__ bool body_fixed(const World& w, uint32_t b) {
    return w.inv_mass[b] == 0.0f && w.inv_inertia[size_t(b) * 3] == 0.0f &&
           w.inv_inertia[size_t(b) * 3 + 1] == 0.0f && w.inv_inertia[size_t(b) * 3 + 2] == 0.0f;
}

// Root of x.  Links always point to a smaller index, so the walk ends;
// path halving shortens it for later calls (a benign race: every value
// written is an ancestor).
__device__ __forceinline__ uint32_t find_root(uint32_t* parent, uint32_t x) {
    volatile uint32_t* p = parent;
    uint32_t cur = p[x];
    if (cur != x) {
        uint32_t prev = x, next;
        while (cur > (next = p[cur])) {
            p[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

// Every island kernel runs on contacts from the narrowphase's scan (and the
// later ones on the island sort): none runs after a wait gave up.
__global__ void k_island_prep(World w, Scratch s) {
    if (halted(w.status)) return;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.nb; b += gridDim.x * blockDim.x) {
        s.isl.parent[b] = b;
        s.s_last[b] = 0;
        st_m3(s.s_R, b, quat_to_mat(w.quat, b));
    }
}

// Hook the roots of a contact's two dynamic bodies: a failed CAS returns a
// smaller root, so every retry makes progress.
__global__ void k_island_union(World w, Scratch s) {
    if (halted(w.status)) return;
    const uint32_t nc = min(w.counters[1], w.max_contacts);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const uint32_t a = w.geom_body[w.c_a[c]], b = w.geom_body[w.c_b[c]];
        if (w.inv_mass[a] == 0.0f && w.inv_mass[b] == 0.0f) continue;  // skipped (physics.comp:531)
        if (body_fixed(w, a) || body_fixed(w, b)) continue;
        uint32_t ra = find_root(s.isl.parent, a), rb = find_root(s.isl.parent, b);
        while (ra != rb) {
            if (ra > rb) {
                const uint32_t t = ra;
                ra = rb;
                rb = t;
            }
            const uint32_t old = atomicCAS(&s.isl.parent[rb], rb, ra);
            if (old == rb) break;
            rb = find_root(s.isl.parent, old);
        }
    }
}

__global__ void k_island_keys(World w, Scratch s) {
    if (halted(w.status)) return;
    const uint32_t nc = min(w.counters[1], w.max_contacts);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < w.max_contacts;
         c += gridDim.x * blockDim.x) {
        uint32_t key = kNoKey;
        if (c < nc) {
            const uint32_t a = w.geom_body[w.c_a[c]], b = w.geom_body[w.c_b[c]];
            if (!(w.inv_mass[a] == 0.0f && w.inv_mass[b] == 0.0f))
                key = find_root(s.isl.parent, body_fixed(w, a) ? b : a);
        }
        s.isl.keys_in[c] = key;
        s.isl.vals_in[c] = c;
    }
}

__global__ void k_island_heads(World w, Scratch s) {
    if (halted(w.status)) return;
    const uint32_t* k = s.isl.keys_out;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.max_contacts;
         i += gridDim.x * blockDim.x)
        s.isl.head[i] = (k[i] != kNoKey && (i == 0 || k[i - 1] != k[i])) ? 1u : 0u;
}

__global__ void k_island_starts(World w, Scratch s) {
    if (halted(w.status)) return;
    const uint32_t* k = s.isl.keys_out;
    const uint32_t n = w.max_contacts;
    const uint32_t count = *s.isl.count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (s.isl.head[i]) s.isl.start[s.isl.idx[i]] = i;
        if (k[i] != kNoKey && (i + 1 == n || k[i + 1] == kNoKey)) s.isl.start[count] = i + 1;
    }
    if (count == 0 && blockIdx.x == 0 && threadIdx.x == 0) s.isl.start[0] = 0;
}

// Warp per island (persistent).  Positions p in [start, start+1) index the
// island's contacts in index order (perm[p] = contact).
__global__ void __launch_bounds__(kIslandThreads)
    k_solver_island(World w, Consts k, Scratch s, uint32_t mode, float dt, uint32_t giant) {
    if (halted(w.status)) return;
    const unsigned full = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t count = *s.isl.count;
    const uint32_t* perm = s.isl.perm;
    uint32_t* last = s.s_last;
    for (uint32_t isl = gwarp; isl < count; isl += nwarps) {
        const uint32_t p0 = s.isl.start[isl], p1 = s.isl.start[isl + 1];
        if (p1 - p0 > giant) continue;  // solved grid-wide (giant.cu)
        for (uint32_t i = p0 + lane; i < p1; i += 32) {
            const uint32_t c = perm[i];
            s.s_ab[size_t(i) * 2] = w.geom_body[w.c_a[c]];
            s.s_ab[size_t(i) * 2 + 1] = w.geom_body[w.c_b[c]];
        }
        __syncwarp();

        // ---- levels ----
        uint32_t maxl = 0;
        bool coloured = mode == 2;
        if (coloured) {
            // greedy colouring in contact order (per-body colour masks in
            // `last`); more than 32 colours at a body falls back to levels
            uint32_t ok = 1u, mx = 0u;
            if (lane == 0) {
                for (uint32_t i = p0; i < p1; ++i) {
                    const uint32_t a = s.s_ab[size_t(i) * 2], b = s.s_ab[size_t(i) * 2 + 1];
                    const bool da = !body_fixed(w, a), db = !body_fixed(w, b);
                    const uint32_t used = (da ? last[a] : 0u) | (db ? last[b] : 0u);
                    if (used == 0xFFFFFFFFu) {
                        ok = 0u;
                        break;
                    }
                    const uint32_t col = uint32_t(__ffs(int(~used))) - 1u;
                    if (da) last[a] |= 1u << col;
                    if (db) last[b] |= 1u << col;
                    s.s_level[i] = col;
                    mx = max(mx, col + 1u);
                }
            }
            ok = __shfl_sync(full, ok, 0);
            maxl = __shfl_sync(full, mx, 0);
            if (!ok) {
                coloured = false;
                maxl = 0;
                for (uint32_t i = p0 + lane; i < p1; i += 32) {
                    last[s.s_ab[size_t(i) * 2]] = 0;
                    last[s.s_ab[size_t(i) * 2 + 1]] = 0;
                }
            }
            __syncwarp();
        }
        for (uint32_t ib = p0; !coloured && ib < p1; ib += 32) {
            const uint32_t i = ib + lane;
            const bool valid = i < p1;
            const uint32_t a = valid ? s.s_ab[size_t(i) * 2] : 0u;
            const uint32_t b = valid ? s.s_ab[size_t(i) * 2 + 1] : 0u;
            uint32_t L = valid ? 1u : 0u;
            if (mode != 0) {
                const bool da = valid && !body_fixed(w, a), db = valid && !body_fixed(w, b);
                const uint32_t xa = da ? a : (0x80000000u | (lane * 2u));
                const uint32_t xb = db ? b : (0x80000000u | (lane * 2u + 1u));
                if (valid) L = max(da ? last[a] : 0u, db ? last[b] : 0u) + 1u;
                for (uint32_t j = 0; j < 32; ++j) {
                    const uint32_t aj = __shfl_sync(full, xa, j), bj = __shfl_sync(full, xb, j);
                    const uint32_t Lj = __shfl_sync(full, L, j);
                    if (valid && j < lane && (aj == xa || aj == xb || bj == xa || bj == xb))
                        L = max(L, Lj + 1u);
                }
                if (da) atomicMax(&last[a], L);
                if (db) atomicMax(&last[b], L);
            }
            if (valid) s.s_level[i] = L - 1u;
            maxl = max(maxl, L);
            __syncwarp();
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) maxl = max(maxl, __shfl_xor_sync(full, maxl, off));

        // ---- positions by level, island order within a level ----
        uint32_t* lvl = s.isl.lvl + p0 + isl;  // [levels+1] within [p0+isl, p1+isl]
        uint32_t pos = 0;
        for (uint32_t l = 0; l < maxl; ++l) {
            if (lane == 0) lvl[l] = pos;
            for (uint32_t ib = p0; ib < p1; ib += 32) {
                const uint32_t i = ib + lane;
                const bool hit = i < p1 && s.s_level[i] == l;
                const unsigned m = __ballot_sync(full, hit);
                if (hit) s.s_order[p0 + pos + __popc(m & ((1u << lane) - 1u))] = i;
                pos += __popc(m);
            }
        }
        if (lane == 0) lvl[maxl] = pos;
        __syncwarp();

        // ---- per-contact constants in solve order (physics.comp:504-521,
        // 533-546), from the pre-solve velocities ----
        for (uint32_t j = lane; j < pos; j += 32) {
            const uint32_t q = p0 + j, i = s.s_order[q], c = perm[i];
            const uint32_t ga = w.c_a[c], gb = w.c_b[c];
            const uint32_t a = s.s_ab[size_t(i) * 2], b = s.s_ab[size_t(i) * 2 + 1];
            const f3 n = ld3(w.c_normal, c), cp = ld3(w.c_pos, c);
            const f3 ra = sub(cp, ld3(w.pos, a)), rb = sub(cp, ld3(w.pos, b));
            const f3 va = add(ld3(w.vel, a), cross(ld3(w.omega, a), ra));
            const f3 vb = add(ld3(w.vel, b), cross(ld3(w.omega, b), rb));
            const float vn = dot(sub(vb, va), n);
            const float e = gmax(w.restitution[ga], w.restitution[gb]);
            const float bias =
                k.baumgarte * gmax(w.c_pen[c] - k.slop, 0.0f) / dt + e * gmax(-vn, 0.0f);
            const m3 Ra = ld_m3(s.s_R, a), Rb = ld_m3(s.s_R, b);
            const f3 ran = cross(ra, n), rbn = cross(rb, n);
            const float kn = w.inv_mass[a] + w.inv_mass[b] +
                             dot(ran, apply_inv_I(Ra, ld3(w.inv_inertia, a), ran)) +
                             dot(rbn, apply_inv_I(Rb, ld3(w.inv_inertia, b), rbn));
            st3(s.s_n, q, n);
            st3(s.s_ra, q, ra);
            st3(s.s_rb, q, rb);
            s.s_bias[q] = bias;
            s.s_kn[q] = kn;
            s.s_mu[q] = sqrtf(w.friction[ga] * w.friction[gb]);
            s.s_abp[size_t(q) * 2] = a;
            s.s_abp[size_t(q) * 2 + 1] = b;
            s.s_lam[q] = 0.0f;
        }
        __syncwarp();

        // ---- Gauss-Seidel sweeps ----
        const BodyView B{w.vel, w.omega, s.s_R, w.inv_inertia, w.inv_mass};
        auto solve = [&](uint32_t q) {
            solve_one(B, s.s_abp[size_t(q) * 2], s.s_abp[size_t(q) * 2 + 1], ld3(s.s_n, q),
                      ld3(s.s_ra, q), ld3(s.s_rb, q), s.s_bias[q], s.s_kn[q], s.s_mu[q],
                      &s.s_lam[q]);
        };
        if (mode == 0) {
            if (lane == 0)
                for (uint32_t it = 0; it < k.pgs_iterations; ++it)
                    for (uint32_t j = 0; j < pos; ++j) solve(p0 + j);
        } else {
            for (uint32_t it = 0; it < k.pgs_iterations; ++it)
                for (uint32_t l = 0; l < maxl; ++l) {
                    const uint32_t beg = lvl[l], end = lvl[l + 1];
                    for (uint32_t j = beg + lane; j < end; j += 32) solve(p0 + j);
                    __syncwarp();
                }
        }
        __syncwarp();
        for (uint32_t j = lane; j < pos; j += 32)
            w.lambda[perm[s.s_order[p0 + j]]] = s.s_lam[p0 + j];
        __syncwarp();
    }
}

inline uint32_t blocks_of(uint32_t n, uint32_t t) { return n ? (n + t - 1) / t : 1u; }

}  // namespace

int launch_solver_islands(const World& w, const Consts& k, const Scratch& s, uint32_t mode,
                          float dt, cudaStream_t st) {
    if (w.max_contacts == 0) return 0;
    const uint32_t cap = 148u * 8u;
    const uint32_t nbb = min(blocks_of(w.nb, 256), cap), ncb = min(blocks_of(w.max_contacts, 256), cap);
    k_island_prep<<<nbb, 256, 0, st>>>(w, s);
    k_island_union<<<ncb, 256, 0, st>>>(w, s);
    k_island_keys<<<ncb, 256, 0, st>>>(w, s);
    LbvhScratch ls{};
    ls.hist = s.isl.sort_hist;
    ls.status = s.isl.sort_status;
    ls.wait_limit = s.wait_limit;
    int n = 3 + lbvh_sort(s.isl.keys_in, s.isl.vals_in, s.isl.keys_tmp, s.isl.vals_tmp,
                          s.isl.keys_out, s.isl.perm, w.max_contacts, ls, &s.status[0], st);
    k_island_heads<<<ncb, 256, 0, st>>>(w, s);
    n += 1 + launch_exclusive_scan(s.isl.head, s.isl.idx, nullptr, w.max_contacts, s.isl.count,
                                   w.max_contacts + 1, 0u, s, st);
    k_island_starts<<<ncb, 256, 0, st>>>(w, s);
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solver_island, kIslandThreads, 0);
        if (per_sm <= 0) per_sm = 1;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // coloured mode: islands above kGiantContacts contacts are solved by the
    // whole grid, the others by a warp each
    const int giant = mode == 2 ? launch_solver_giant(w, k, s, dt, st) : 0;
    k_solver_island<<<uint32_t(sms) * uint32_t(per_sm), kIslandThreads, 0, st>>>(
        w, k, s, mode, dt, giant ? (s.giant_min ? s.giant_min : kGiantContacts) : 0xFFFFFFFFu);
    return n + 2 + giant;
}

}  // namespace seevr
