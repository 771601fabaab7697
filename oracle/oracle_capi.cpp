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
    uint32_t narrowphase;  // 0: MPR, 1: GJK + EPA
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
    P.narrowphase = p->narrowphase;
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

uint32_t oracle_angle_bin64f(float y, float x) { return oracle::angle_bin64<float>(y, x); }

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"

// ---- path tracer (raytrace.comp), test infrastructure ------------------------
// A restatement of raytrace.comp:37-282 in the shader's evaluation order,
// with the same pinned definitions as the library (its own sin/cos
// polynomials, pow(x, 5) as a product, the float literal 4294967295.0 as
// 2^32).  Images are float RGBA, row-major.
namespace rt {

struct V {
    float x, y, z;
};
inline V mk(float x, float y, float z) { return V{x, y, z}; }
inline V add(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V sub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V neg(V a) { return V{-a.x, -a.y, -a.z}; }
inline V scale(float s, V a) { return V{s * a.x, s * a.y, s * a.z}; }
inline V mul(V a, V b) { return V{a.x * b.x, a.y * b.y, a.z * b.z}; }
inline float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(V a, V b) {
    return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V normalize(V a) {
    const float l = std::sqrt(dot(a, a));
    return V{a.x / l, a.y / l, a.z / l};
}
inline float gmin(float x, float y) { return y < x ? y : x; }  // GLSL min
inline float gmax(float x, float y) { return x < y ? y : x; }  // GLSL max
inline V ld(const float* p, uint32_t i) { return V{p[size_t(i) * 3], p[size_t(i) * 3 + 1], p[size_t(i) * 3 + 2]}; }

inline uint32_t pcg(uint32_t seed) {  // raytrace.comp:43-47
    const uint32_t state = seed * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
inline float rand_f(uint32_t seed) { return float(pcg(seed)) / 4294967296.0f; }

inline void sincos_pinned(float x, float& s, float& c) {
    const float hi = 1.57079637050628662109375f, lo = -4.37113900018624283e-8f;
    const float q = float(int(x * 0.636619772f + 0.5f));
    const float r = (x - q * hi) - q * lo;
    const float r2 = r * r;
    const float sp = r * (1.0f + r2 * (-1.0f / 6.0f + r2 * (1.0f / 120.0f + r2 * (-1.0f / 5040.0f +
                                                                                  r2 * (1.0f / 362880.0f)))));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (1.0f / 24.0f + r2 * (-1.0f / 720.0f +
                                                                    r2 * (1.0f / 40320.0f +
                                                                          r2 * (-1.0f / 3628800.0f)))));
    switch (int(q) & 3) {
        case 0: s = sp; c = cp; break;
        case 1: s = cp; c = -sp; break;
        case 2: s = -sp; c = -cp; break;
        default: s = -cp; c = sp; break;
    }
}
inline V mix3(V x, V y, float a) { return add(scale(1.0f - a, x), scale(a, y)); }
inline V reflect3(V i, V n) { return sub(i, scale(2.0f * dot(n, i), n)); }
inline V refract3(V i, V n, float eta) {
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return mk(0.f, 0.f, 0.f);
    return sub(scale(eta, i), scale(eta * d + std::sqrt(k), n));
}
inline float schlick(float cos_theta, float r0) {
    const float x = 1.0f - cos_theta;
    return r0 + (1.0f - r0) * (((x * x) * (x * x)) * x);
}

struct Scene {
    const float *verts, *node_min, *node_max, *albedo, *roughness, *metallic, *emission, *ior;
    const uint32_t *idx, *left, *right, *count, *prim, *tri_geom, *geom_material;
};

inline float ray_tri(V ro, V rd, V v0, V v1, V v2) {  // raytrace.comp:55-69
    const V e1 = sub(v1, v0), e2 = sub(v2, v0);
    const V h = cross(rd, e2);
    const float a = dot(e1, h);
    if (std::fabs(a) < 1e-8f) return -1.0f;
    const float f = 1.0f / a;
    const V s = sub(ro, v0);
    const float u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const V q = cross(s, e1);
    const float v = f * dot(rd, q);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = f * dot(e2, q);
    return t > 0.001f ? t : -1.0f;
}

inline bool ray_aabb(V ro, V inv_d, V bmin, V bmax, float closest) {  // 73-81
    const V t1 = mul(sub(bmin, ro), inv_d), t2 = mul(sub(bmax, ro), inv_d);
    const V tmin{gmin(t1.x, t2.x), gmin(t1.y, t2.y), gmin(t1.z, t2.z)};
    const V tmax{gmax(t1.x, t2.x), gmax(t1.y, t2.y), gmax(t1.z, t2.z)};
    const float enter = gmax(gmax(tmin.x, tmin.y), tmin.z);
    const float exit_ = gmin(gmin(tmax.x, tmax.y), tmax.z);
    return exit_ >= enter && enter < closest && exit_ > 0.0f;
}

inline void trace(const Scene& g, V ro, V rd, float& closest, V& normal, uint32_t& hit, bool& front) {
    closest = 1e10f;
    normal = mk(0.f, 1.f, 0.f);
    hit = 0xFFFFFFFFu;
    front = true;
    const V inv_d = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    int stack[32];
    stack[0] = 0;
    int sp = 1;
    while (sp > 0) {
        --sp;
        const int node = stack[sp];
        if (!ray_aabb(ro, inv_d, ld(g.node_min, node), ld(g.node_max, node), closest)) continue;
        const uint32_t cnt = g.count[node], lf = g.left[node];
        if (cnt > 0) {
            for (uint32_t i = 0; i < cnt; ++i) {
                const uint32_t ti = g.prim[lf + i];
                const V v0 = ld(g.verts, g.idx[size_t(ti) * 3]);
                const V v1 = ld(g.verts, g.idx[size_t(ti) * 3 + 1]);
                const V v2 = ld(g.verts, g.idx[size_t(ti) * 3 + 2]);
                const float t = ray_tri(ro, rd, v0, v1, v2);
                if (t > 0.0f && t < closest) {
                    closest = t;
                    const V n = normalize(cross(sub(v1, v0), sub(v2, v0)));
                    front = dot(n, rd) < 0.0f;
                    normal = front ? n : neg(n);
                    hit = ti;
                }
            }
        } else {
            const uint32_t r = g.right[node];
            if (sp < 31) stack[sp++] = int(lf);
            if (sp < 31) stack[sp++] = int(r);
        }
    }
}

inline V sky_color(V rd) {
    const float t = 0.5f * (rd.y + 1.0f);
    return scale(0.8f, mix3(mk(1.f, 1.f, 1.f), mk(0.5f, 0.7f, 1.0f), t));
}

inline V sample_hemisphere(V n, uint32_t s1, uint32_t s2) {
    const float r1 = rand_f(s1), r2 = rand_f(s2);
    const float phi = 2.0f * 3.14159265f * r1;
    const float cos_t = std::sqrt(r2), sin_t = std::sqrt(1.0f - r2);
    const V up = std::fabs(n.y) > 0.99f ? mk(1.f, 0.f, 0.f) : mk(0.f, 1.f, 0.f);
    const V tan1 = normalize(cross(up, n));
    const V tan2 = cross(n, tan1);
    float sp, cp;
    sincos_pinned(phi, sp, cp);
    return normalize(add(add(scale(cp, scale(sin_t, tan1)), scale(cos_t, n)), scale(sp, scale(sin_t, tan2))));
}

void pixel(const Scene& g, const float* cam, uint32_t w, uint32_t h, uint32_t frame, float fov,
           uint32_t px, uint32_t py, float* out) {  // raytrace.comp:163-282
    const V cam_pos{cam[0], cam[1], cam[2]}, cam_dir{cam[3], cam[4], cam[5]};
    const V cam_right{cam[6], cam[7], cam[8]}, cam_up{cam[9], cam[10], cam[11]};
    const float aspect = float(w) / float(h);
    V pix = mk(0.f, 0.f, 0.f);
    for (int si = 0; si < 16; ++si) {
        uint32_t seed = px + py * w + frame * w * h + uint32_t(si) * 12345u;
        const float jx = rand_f(seed) - 0.5f;
        const float jy = rand_f(seed + 1u) - 0.5f;
        const float u = (2.0f * (float(px) + 0.5f + jx) / float(w) - 1.0f) * aspect * fov;
        const float v = -(2.0f * (float(py) + 0.5f + jy) / float(h) - 1.0f) * fov;
        V rd = normalize(add(add(cam_dir, scale(u, cam_right)), scale(v, cam_up)));
        V ro = cam_pos;
        V thr = mk(1.f, 1.f, 1.f), color = mk(0.f, 0.f, 0.f);
        for (int bounce = 0; bounce < 16; ++bounce) {
            float t;
            V normal;
            uint32_t hit;
            bool front;
            trace(g, ro, rd, t, normal, hit, front);
            if (t >= 1e9f) {
                color = add(color, mul(thr, sky_color(rd)));
                break;
            }
            const uint32_t mi = g.geom_material[g.tri_geom[hit]];
            const V albedo = ld(g.albedo, mi), emission = ld(g.emission, mi);
            const float rough = g.roughness[mi], metal = g.metallic[mi], ior = g.ior[mi];
            color = add(color, mul(thr, emission));
            if (emission.x + emission.y + emission.z > 0.0f) break;
            const V hp = add(ro, scale(t, rd));
            if (bounce > 0) {
                const float p = gmax(thr.x, gmax(thr.y, thr.z));
                if (rand_f(seed + uint32_t(bounce) * 7u) > p) break;
                thr = mk(thr.x / p, thr.y / p, thr.z / p);
            }
            seed = pcg(seed);
            if (ior > 0.0f) {
                const float eta = front ? (1.0f / ior) : ior;
                const float cos_i = std::fabs(dot(rd, normal));
                const float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
                float r0 = (1.0f - ior) / (1.0f + ior);
                r0 = r0 * r0;
                const float fresnel = schlick(cos_i, r0);
                const bool tir = sin2_t > 1.0f;
                if (rand_f(seed + 5u) < fresnel || tir) {
                    rd = reflect3(rd, normal);
                    ro = add(hp, scale(0.001f, normal));
                } else {
                    rd = refract3(rd, normal, eta);
                    ro = sub(hp, scale(0.001f, normal));
                }
                thr = mul(thr, albedo);
            } else if (metal > 0.5f) {
                const V refl = reflect3(rd, normal);
                const V diff = sample_hemisphere(normal, seed, seed + 1u);
                rd = normalize(mix3(refl, diff, rough * rough));
                thr = mul(thr, albedo);
                ro = add(hp, scale(0.001f, normal));
            } else {
                const V refl = reflect3(rd, normal);
                const V diff = sample_hemisphere(normal, seed, seed + 1u);
                const float cos_theta = gmax(dot(neg(rd), normal), 0.0f);
                const float fresnel = schlick(cos_theta, 0.04f);
                if (rand_f(seed + 3u) < fresnel) {
                    rd = normalize(mix3(refl, diff, rough * rough));
                } else {
                    rd = diff;
                    thr = mul(thr, albedo);
                }
                ro = add(hp, scale(0.001f, normal));
            }
        }
        pix = add(pix, color);
    }
    out[0] = pix.x / 16.0f;
    out[1] = pix.y / 16.0f;
    out[2] = pix.z / 16.0f;
    out[3] = 1.0f;
}

}  // namespace rt

extern "C" {

// cam: pos, dir, right, up (12 floats); fov = tan(30 degrees) as the library
// computes it; image: w*h*4 floats.  OpenMP over rows when threads > 0.
void oracle_raytrace(const float* verts, const uint32_t* idx, const float* node_min,
                     const float* node_max, const uint32_t* left, const uint32_t* right,
                     const uint32_t* count, const uint32_t* prim, const uint32_t* tri_geom,
                     const uint32_t* geom_material, const float* albedo, const float* roughness,
                     const float* metallic, const float* emission, const float* ior,
                     const float* cam, uint32_t w, uint32_t h, uint32_t frame, float fov,
                     int threads, float* image) {
    const rt::Scene g{verts, node_min, node_max, albedo, roughness, metallic, emission, ior,
                      idx,   left,     right,    count,  prim,      tri_geom, geom_material};
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1) if (threads > 0)
    for (int64_t py = 0; py < int64_t(h); ++py)
        for (uint32_t px = 0; px < w; ++px)
            rt::pixel(g, cam, w, h, frame, fov, px, uint32_t(py), image + (size_t(py) * w + px) * 4);
}

}  // extern "C"
