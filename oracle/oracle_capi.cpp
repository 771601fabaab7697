// oracle_capi.cpp — TEST INFRASTRUCTURE, not product code.
// C ABI over seevr_oracle.hpp for the tests (ctypes) and for the CPU
// baseline leg of bench.py.  Parity unpinned: see seevr_oracle.hpp.
#include <chrono>
#include <cstdint>
#include <vector>

#include "seevr_oracle.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Same fields as oracle::SceneIn, C layout.
typedef struct oracle_scene {
    uint32_t num_bodies, num_geoms, num_hull_verts, num_vertices, num_scenes;
    const float *body_pos, *body_quat, *body_vel, *body_omega, *body_inv_mass, *body_inv_inertia;
    const uint32_t *body_vert_start, *body_vert_count, *geom_body_idx;
    const float *geom_data, *geom_friction, *geom_restitution, *hull_verts, *orig_verts;
    const uint32_t *support_offset, *support_lookup, *scene_body_offset, *hull_range;
} oracle_scene;

typedef struct oracle_params {
    uint32_t pgs_iterations;
    float baumgarte, slop, lin_damp, ang_damp, eps, tol;
    uint32_t mpr_iterations, discover_trials, max_pairs, max_contacts;
} oracle_params;

// Outputs (any pointer may be NULL).  Values of the last substep.
typedef struct oracle_out {
    double *pos, *quat, *vel, *omega;  // N*3, N*4, N*3, N*3
    double *aabb_min, *aabb_max;       // N*3
    double* verts;                     // V*3 (render vertices, step 7)
    uint32_t* pairs;                   // max_pairs*2, canonical order
    double *c_pos, *c_normal, *c_pen, *lambda;  // max_contacts*{3,3,1,1}
    uint32_t *c_a, *c_b;
    uint32_t counters[2];  // pairs, contacts (true totals)
    uint64_t ops[10];      // OpCounts fields, in declaration order
} oracle_out;

}  // extern "C"

namespace {

oracle::SceneIn to_in(const oracle_scene* s) {
    oracle::SceneIn in;
    in.num_bodies = s->num_bodies;
    in.num_geoms = s->num_geoms;
    in.num_hull_verts = s->num_hull_verts;
    in.num_vertices = s->num_vertices;
    in.num_scenes = s->num_scenes;
    in.body_pos = s->body_pos;
    in.body_quat = s->body_quat;
    in.body_vel = s->body_vel;
    in.body_omega = s->body_omega;
    in.body_inv_mass = s->body_inv_mass;
    in.body_inv_inertia = s->body_inv_inertia;
    in.body_vert_start = s->body_vert_start;
    in.body_vert_count = s->body_vert_count;
    in.geom_body_idx = s->geom_body_idx;
    in.geom_data = s->geom_data;
    in.geom_friction = s->geom_friction;
    in.geom_restitution = s->geom_restitution;
    in.hull_verts = s->hull_verts;
    in.orig_verts = s->orig_verts;
    in.support_offset = s->support_offset;
    in.support_lookup = s->support_lookup;
    in.scene_body_offset = s->scene_body_offset;
    in.hull_range = s->hull_range;
    return in;
}

oracle::Params to_params(const oracle_params* p) {
    oracle::Params P;
    P.pgs_iterations = p->pgs_iterations;
    P.baumgarte = p->baumgarte;
    P.slop = p->slop;
    P.lin_damp = p->lin_damp;
    P.ang_damp = p->ang_damp;
    P.eps = p->eps;
    P.tol = p->tol;
    P.mpr_iterations = p->mpr_iterations;
    P.discover_trials = p->discover_trials;
    P.max_pairs = p->max_pairs;
    P.max_contacts = p->max_contacts;
    return P;
}

template <class R>
void copy_out(const std::vector<R>& src, double* dst, size_t offset) {
    if (!dst) return;
    for (size_t i = 0; i < src.size(); ++i) dst[offset + i] = double(src[i]);
}

struct Totals {
    uint32_t pairs = 0, contacts = 0;
};

// Write one instance's results at body offset b0 / vertex offset v0 /
// pair+contact offsets held in *t.
template <class R>
void emit(const oracle::Physics<R>& ph, uint32_t b0, uint32_t v0, uint32_t max_pairs,
          uint32_t max_contacts, oracle_out* o, Totals* t) {
    copy_out(ph.pos, o->pos, size_t(b0) * 3);
    copy_out(ph.quat, o->quat, size_t(b0) * 4);
    copy_out(ph.vel, o->vel, size_t(b0) * 3);
    copy_out(ph.omega, o->omega, size_t(b0) * 3);
    copy_out(ph.aabb_min, o->aabb_min, size_t(b0) * 3);
    copy_out(ph.aabb_max, o->aabb_max, size_t(b0) * 3);
    copy_out(ph.verts, o->verts, size_t(v0) * 3);
    const uint32_t np = std::min(ph.pairs_total, ph.P.max_pairs);
    for (uint32_t i = 0; i < np && t->pairs + i < max_pairs; ++i)
        if (o->pairs) {
            o->pairs[(t->pairs + i) * 2] = ph.pairs[i * 2] + b0;
            o->pairs[(t->pairs + i) * 2 + 1] = ph.pairs[i * 2 + 1] + b0;
        }
    const uint32_t nc = std::min(ph.contacts_total, ph.P.max_contacts);
    for (uint32_t i = 0; i < nc && t->contacts + i < max_contacts; ++i) {
        const size_t c = t->contacts + i;
        for (int k = 0; k < 3; ++k) {
            if (o->c_pos) o->c_pos[c * 3 + k] = double(ph.c_pos[i * 3 + k]);
            if (o->c_normal) o->c_normal[c * 3 + k] = double(ph.c_normal[i * 3 + k]);
        }
        if (o->c_pen) o->c_pen[c] = double(ph.c_pen[i]);
        if (o->lambda) o->lambda[c] = double(ph.lambda[i]);
        if (o->c_a) o->c_a[c] = ph.c_a[i] + b0;
        if (o->c_b) o->c_b[c] = ph.c_b[i] + b0;
    }
    t->pairs += ph.pairs_total;
    t->contacts += ph.contacts_total;
}

template <class R>
void add_ops(const oracle::OpCounts& c, uint64_t* ops) {
    const uint64_t v[10] = {c.support_brute, c.support_brute_verts, c.support_lookup,
                            c.mpr_calls,     c.mpr_support_calls,   c.pgs_contact_iters,
                            c.pgs_friction_iters, c.aabb_verts,     c.broad_tests,
                            c.bodies};
    for (int i = 0; i < 10; ++i) ops[i] += v[i];
}

constexpr uint64_t kBranchSeed = 1469598103934665603ull;

// Decision tapes of the last recording run, one per instance (the whole
// batch, or one per scene); replay runs read them.  Test infrastructure:
// callers are single-threaded.
std::vector<std::vector<uint32_t>> g_tapes;

// Instrumentation options of a run: per-scene branch hashes and branch
// locking (lock_mode 0 off, 1 record, 2 replay).
struct Instr {
    uint64_t* branch_sig;
    int lock_mode;
};

// Set up instance `k` (covering `nsig` scenes) before its run.
template <class R>
bool instr_begin(oracle::Physics<R>& ph, const Instr& in, size_t k, uint32_t nsig) {
    using L = typename oracle::Physics<R>::Lock;
    if (in.branch_sig) ph.branch.assign(nsig, kBranchSeed);
    if (in.lock_mode == 1) ph.lock_mode = L::Record;
    if (in.lock_mode == 2) {
        if (k >= g_tapes.size()) return false;
        ph.lock_mode = L::Replay;
        ph.lock = g_tapes[k];
    }
    return true;
}

// Collect instance `k`'s outputs: hashes at scene offset sig0; the tape
// (record); false when a replay did not consume its tape exactly.
template <class R>
bool instr_end(oracle::Physics<R>& ph, const Instr& in, size_t k, uint32_t sig0) {
    if (in.branch_sig) std::copy(ph.branch.begin(), ph.branch.end(), in.branch_sig + sig0);
    if (in.lock_mode == 1) g_tapes[k] = std::move(ph.lock);
    if (in.lock_mode == 2) return !ph.lock_error && ph.lock_pos == ph.lock.size();
    return true;
}

template <class R>
int run(const oracle_scene* s, const oracle_params* p, uint32_t frames, uint32_t substeps,
        float dt, const float g[3], int update_verts, int threads, oracle_out* o,
        const Instr& ins, const double* const st[5]) {
    const oracle::SceneIn in = to_in(s);
    const oracle::Params P = to_params(p);
    const R gr[3] = {R(g[0]), R(g[1]), R(g[2])};
    o->counters[0] = o->counters[1] = 0;
    for (auto& x : o->ops) x = 0;
    // optional double-precision initial state (pos, quat, vel, omega, friction)
    auto put = [&](oracle::Physics<R>& ph, uint32_t b0, uint32_t nb) {
        if (!st) return;
        auto cp = [](std::vector<R>& dst, const double* src, size_t off, size_t n) {
            if (src)
                for (size_t i = 0; i < n; ++i) dst[i] = R(src[off + i]);
        };
        cp(ph.pos, st[0], size_t(b0) * 3, size_t(nb) * 3);
        cp(ph.quat, st[1], size_t(b0) * 4, size_t(nb) * 4);
        cp(ph.vel, st[2], size_t(b0) * 3, size_t(nb) * 3);
        cp(ph.omega, st[3], size_t(b0) * 3, size_t(nb) * 3);
        cp(ph.friction, st[4], b0, nb);
    };
    if (threads <= 0 || s->num_scenes <= 1 || !s->scene_body_offset) {
        // whole batch in one instance: global caps, global canonical order
        oracle::Physics<R> ph(in, P);
        if (ins.lock_mode == 1) g_tapes.assign(1, {});
        const uint32_t nsig = s->scene_body_offset && s->num_scenes > 0 ? s->num_scenes : 1u;
        if (!instr_begin(ph, ins, 0, nsig)) return 3;
        put(ph, 0, s->num_bodies);
        for (uint32_t f = 0; f < frames; ++f) ph.step(substeps, R(dt), gr, update_verts != 0);
        Totals t;
        emit(ph, 0, 0, P.max_pairs, P.max_contacts, o, &t);
        o->counters[0] = t.pairs;
        o->counters[1] = t.contacts;
        add_ops<R>(ph.ops, o->ops);
        return instr_end(ph, ins, 0, 0) ? 0 : 3;
    }
    // one instance per scene, scenes in parallel; identical results to the
    // whole-batch instance as long as no cap overflows (scenes share no body)
    const uint32_t ns = s->num_scenes;
    std::vector<oracle::Physics<R>*> inst(ns, nullptr);
    if (ins.lock_mode == 1) g_tapes.assign(ns, {});
    int bad = 0;
#ifdef _OPENMP
    omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int64_t sc = 0; sc < int64_t(ns); ++sc) {
        const uint32_t b0 = s->scene_body_offset[sc], b1 = s->scene_body_offset[sc + 1];
        if (b1 <= b0) continue;
        auto* ph = new oracle::Physics<R>(in, P, b0, b1);
        if (!instr_begin(*ph, ins, size_t(sc), 1u)) bad = 1;
        put(*ph, b0, b1 - b0);
        for (uint32_t f = 0; f < frames; ++f) ph->step(substeps, R(dt), gr, update_verts != 0);
        if (!instr_end(*ph, ins, size_t(sc), uint32_t(sc))) bad = 1;
        inst[size_t(sc)] = ph;
    }
    Totals t;
    for (uint32_t sc = 0; sc < ns; ++sc) {
        if (!inst[sc]) continue;
        const uint32_t b0 = s->scene_body_offset[sc];
        emit(*inst[sc], b0, s->body_vert_start[b0], P.max_pairs, P.max_contacts, o, &t);
        add_ops<R>(inst[sc]->ops, o->ops);
        delete inst[sc];
    }
    o->counters[0] = t.pairs;
    o->counters[1] = t.contacts;
    return bad ? 3 : 0;
}

}  // namespace

extern "C" {

// Run `frames` calls of Physics.step on a copy of the scene.  precision 32
// or 64; threads <= 0 runs the batch as one instance, otherwise one
// instance per scene on `threads` OpenMP threads.  Test instrumentation:
// branch_sig (NULL = off) receives per scene a hash of the run's structural
// decisions (support vertices, pairs, contacts); lock_mode 1 records every
// branch decision, 2 replays the last recording (same instance layout)
// instead of deciding.  Returns 0 on success, 3 when a replay did not match
// its recording's length.
int oracle_run(const oracle_scene* s, const oracle_params* p, int precision, uint32_t frames,
               uint32_t substeps, float dt, const float g[3], int update_verts, int threads,
               oracle_out* o, uint64_t* branch_sig, int lock_mode) {
    if (!s || !p || !o) return 1;
    const Instr ins{branch_sig, lock_mode};
    if (precision == 64)
        return run<double>(s, p, frames, substeps, dt, g, update_verts, threads, o, ins, nullptr);
    return run<float>(s, p, frames, substeps, dt, g, update_verts, threads, o, ins, nullptr);
}

// FP64 run from a double-precision initial state: pos/quat/vel/omega/
// friction override the scene's float values (any may be NULL).  Central
// finite differences of the adjoint tests perturb these inputs by far less
// than a float ulp.  Other arguments as oracle_run.
int oracle_run_f64_state(const oracle_scene* s, const oracle_params* p, uint32_t frames,
                         uint32_t substeps, float dt, const float g[3], const double* pos,
                         const double* quat, const double* vel, const double* omega,
                         const double* friction, int threads, oracle_out* o,
                         uint64_t* branch_sig, int lock_mode) {
    if (!s || !p || !o) return 1;
    const double* st[5] = {pos, quat, vel, omega, friction};
    return run<double>(s, p, frames, substeps, dt, g, 0, threads, o, Instr{branch_sig, lock_mode},
                       st);
}

// Morton codes (bvh.comp:169-183) of n centroids; bounds[6] = min, max.
void oracle_morton(const float* centroids, uint32_t n, uint32_t* codes, float* bounds) {
    oracle::morton_codes(centroids, n, codes, bounds);
}

// 4-bit LSD radix sort of codes (bvh.comp:192-295): sorted keys and the
// permutation (original index of each sorted slot).
void oracle_radix_sort(const uint32_t* codes, uint32_t n, uint32_t* sorted, uint32_t* perm) {
    std::vector<uint32_t> k(codes, codes + n), idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    oracle::radix_sort_lsd4(k, idx);
    std::copy(k.begin(), k.end(), sorted);
    std::copy(idx.begin(), idx.end(), perm);
}

// Karras hierarchy (bvh.comp:299-348) over sorted codes; arrays of 2n-1.
void oracle_karras(const uint32_t* sorted, uint32_t n, uint32_t* left, uint32_t* right,
                   uint32_t* parent) {
    std::vector<uint32_t> m(sorted, sorted + n), l, r, p;
    oracle::karras(m, l, r, p);
    std::copy(l.begin(), l.end(), left);
    std::copy(r.begin(), r.end(), right);
    std::copy(p.begin(), p.end(), parent);
}

float oracle_atan2f(float y, float x) { return oracle::seevr_atan2<float>(y, x); }
double oracle_atan2d(double y, double x) { return oracle::seevr_atan2<double>(y, x); }

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
