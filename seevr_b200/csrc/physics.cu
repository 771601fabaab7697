// physics.cu — libseevr_cuda C ABI: handle, scratch, and the step driver
// that replaces Physics.init/step/readCounters/deinit (src/physics.zig).
//
// One substep issues, in the reference's order (physics.zig:130-158):
//   body stage  = integrate(prev substep) + gravity + AABB   (steps 6, 0, 9-11)
//   broadphase  = count, scan, write                         (steps 8, 2)
//   narrowphase = MPR, scan, scatter                         (step 3)
//   impulse clear (memset)                                   (step 4)
//   PGS solver                                               (step 5)
// and the frame ends with integrate + render-vertex update (steps 6, 7).
// Every kernel sizes its grid from capacities and reads live counts from
// device memory, so a frame needs no host round trip and can be captured
// into a CUDA graph.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/seevr.h"
#include "adjoint.cuh"
#include "common.cuh"
#include "lbvh.cuh"

using namespace seevr;

namespace {

thread_local std::string g_last_error;

seevr_status fail(seevr_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

}  // namespace

void seevr::set_last_error(const char* msg) { g_last_error = msg; }

namespace {

#define SEEVR_CUDA(call)                                                              \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(SEEVR_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

enum Stage {
    kStGravity = 0,
    kStAabb = 1,
    kStBroad = 2,
    kStNarrow = 3,
    kStClear = 4,
    kStSolve = 5,
    kStIntegrate = 6,
    kStRender = 7,
    kStClearCounters = 8
};

// The arguments a captured frame graph was built for (the graph itself can
// be launched on any stream).
struct GraphKey {
    uint32_t nb, nv, nhv, substeps;
    float dt, g[3];
    // host arrays whose copies the frame holds (seevr_physics_step_io), or
    // none
    const void* io[8];
    bool operator==(const GraphKey& o) const {
        for (int i = 0; i < 8; ++i)
            if (io[i] != o.io[i]) return false;
        return nb == o.nb && nv == o.nv && nhv == o.nhv && substeps == o.substeps && dt == o.dt &&
               g[0] == o.g[0] && g[1] == o.g[1] && g[2] == o.g[2];
    }
};

}  // namespace

struct seevr_physics {
    int device = 0;
    seevr_bindings b{};
    seevr_caps caps{};
    seevr_params params{};
    cudaStream_t stream = nullptr;
    World w{};
    Consts k{};
    Scratch s{};
    uint32_t* body_scene = nullptr;
    uint32_t* scene_off = nullptr;
    uint32_t* bundle_off = nullptr;  // solver bundles (runs of whole scenes)
    uint32_t* body_bundle = nullptr;  // body -> bundle
    uint32_t num_bundles = 1;
    uint32_t max_bundle_bodies = 0;
    // bodies per bundle the warp solver keeps in shared memory: the bundle
    // size, so that single scenes above it (solved in place) do not cut
    // the number of resident warps
    uint32_t smem_bundle_bodies = 0;
    uint32_t num_scenes = 1;
    bool scenes_set = false;
    uint32_t single_scene_nb = 0xFFFFFFFFu;
    uint32_t max_scene_bodies = 0;
    std::vector<void*> allocations;
    uint64_t launches = 0;
    uint32_t host_flags = 0;
    // bounds-check mode: SEEVR_CHECK=1 in the environment at creation
    bool check = false;
    // CUDA graph of one frame
    cudaGraphExec_t graph_exec = nullptr;
    GraphKey graph_key{};
    uint64_t graph_kernels = 0;
    // profiling events
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // LBVH broadphase work arrays (broadphase == SEEVR_BROADPHASE_LBVH)
    LbvhScratch lb{};
    // adjoint work arrays, allocated by the first adjoint call
    AdjScratch adj{};
    bool adj_ready = false;
    // broadphase overlap words (s.bp_mask), sized for the scene layout
    size_t bp_mask_cap = 0;
    // broadphase tile table (s.bp_tiles) capacity, in tiles
    uint32_t bp_tiles_cap = 0;
    // streaming multiprocessors of the device (launch shapes are per SM)
    int sm_count = 148;
    uint32_t narrow_blocks_per_sm = kNarrowBlocksPerSm;
    // the caller's scene layout, kept to rebuild bundles and tiles on retuning
    std::vector<uint32_t> scene_offsets_host;
    // Scene groups (seevr_tuning.scene_groups > 1): sub-handles over
    // contiguous scene ranges, each stepping its scenes on its own stream
    // with its own pair and contact lists, merged into the bound buffers at
    // the end of every frame.
    struct Group {
        seevr_physics* h = nullptr;
        uint32_t b0 = 0, nb = 0;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        std::vector<void*> allocs;  // the group's own pair/contact lists
        GroupOut out{};
    };
    std::vector<Group> groups;
    uint32_t scene_groups = 1;
    cudaEvent_t fork = nullptr;
};

namespace {

template <class T>
seevr_status dev_alloc(seevr_physics* h, T** p, size_t count) {
    void* q = nullptr;
    const size_t bytes = count ? count * sizeof(T) : 16;
    if (cudaMalloc(&q, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(SEEVR_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    h->allocations.push_back(q);
    *p = static_cast<T*>(q);
    return SEEVR_OK;
}

void free_groups(seevr_physics* h) {
    for (auto& g : h->groups) {
        if (g.stream) cudaStreamSynchronize(g.stream);
        if (g.h) seevr_physics_destroy(g.h);
        for (void* p : g.allocs) cudaFree(p);
        if (g.done) cudaEventDestroy(g.done);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    h->groups.clear();
}

void free_all(seevr_physics* h) {
    free_groups(h);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    if (h->s.bp_mask) cudaFree(h->s.bp_mask);
    h->s.bp_mask = nullptr;
    if (h->s.bp_tiles) cudaFree(h->s.bp_tiles);
    h->s.bp_tiles = nullptr;
    for (void* p : h->allocations) cudaFree(p);
    h->allocations.clear();
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// Required byte size of each binding for the given capacities (0 = optional).
uint64_t required_bytes(int i, const seevr_caps& c) {
    const uint64_t N = c.max_bodies, HV = c.max_hull_verts, P = c.max_pairs, C = c.max_contacts;
    switch (i) {
        case SEEVR_B_BODY_POS: case SEEVR_B_BODY_VEL: case SEEVR_B_BODY_OMEGA:
        case SEEVR_B_BODY_INV_INERTIA: case SEEVR_B_BODY_AABB_MIN: case SEEVR_B_BODY_AABB_MAX:
            return N * 12;
        case SEEVR_B_BODY_QUAT: return N * 16;
        case SEEVR_B_BODY_INV_MASS: case SEEVR_B_BODY_VERT_START: case SEEVR_B_BODY_VERT_COUNT:
        case SEEVR_B_GEOM_BODY_IDX: case SEEVR_B_GEOM_FRICTION: case SEEVR_B_GEOM_RESTITUTION:
        case SEEVR_B_SUPPORT_OFFSET:
            return N * 4;
        case SEEVR_B_GEOM_DATA: return N * 32;
        case SEEVR_B_HULL_VERTS: return HV * 12;
        case SEEVR_B_CONTACT_POS: case SEEVR_B_CONTACT_NORMAL: return C * 12;
        case SEEVR_B_CONTACT_PEN: case SEEVR_B_CONTACT_GEOM_A: case SEEVR_B_CONTACT_GEOM_B:
        case SEEVR_B_LAMBDA_N:
            return C * 4;
        case SEEVR_B_COUNTERS: return 8;
        case SEEVR_B_COLLISION_PAIRS: return P * 8;
        case SEEVR_B_SUPPORT_LOOKUP: return 4;
        default: return 0;  // 13, 14 checked at step time; 25-27 unused; 30 optional
    }
}

void setup_world(seevr_physics* h) {
    World& w = h->w;
    auto P = [&](int i) { return h->b.ptr[i]; };
    w.pos = static_cast<float*>(P(SEEVR_B_BODY_POS));
    w.quat = static_cast<float*>(P(SEEVR_B_BODY_QUAT));
    w.vel = static_cast<float*>(P(SEEVR_B_BODY_VEL));
    w.omega = static_cast<float*>(P(SEEVR_B_BODY_OMEGA));
    w.inv_mass = static_cast<const float*>(P(SEEVR_B_BODY_INV_MASS));
    w.inv_inertia = static_cast<const float*>(P(SEEVR_B_BODY_INV_INERTIA));
    w.vert_start = static_cast<const uint32_t*>(P(SEEVR_B_BODY_VERT_START));
    w.vert_count = static_cast<const uint32_t*>(P(SEEVR_B_BODY_VERT_COUNT));
    w.geom_body = static_cast<const uint32_t*>(P(SEEVR_B_GEOM_BODY_IDX));
    w.friction = static_cast<const float*>(P(SEEVR_B_GEOM_FRICTION));
    w.restitution = static_cast<const float*>(P(SEEVR_B_GEOM_RESTITUTION));
    w.hull = static_cast<const float*>(P(SEEVR_B_HULL_VERTS));
    w.verts = static_cast<float*>(P(SEEVR_B_VERTICES));
    w.orig = static_cast<const float*>(P(SEEVR_B_ORIG_VERTICES));
    w.c_pos = static_cast<float*>(P(SEEVR_B_CONTACT_POS));
    w.c_normal = static_cast<float*>(P(SEEVR_B_CONTACT_NORMAL));
    w.c_pen = static_cast<float*>(P(SEEVR_B_CONTACT_PEN));
    w.c_a = static_cast<uint32_t*>(P(SEEVR_B_CONTACT_GEOM_A));
    w.c_b = static_cast<uint32_t*>(P(SEEVR_B_CONTACT_GEOM_B));
    w.lambda = static_cast<float*>(P(SEEVR_B_LAMBDA_N));
    w.counters = static_cast<uint32_t*>(P(SEEVR_B_COUNTERS));
    w.status = h->s.status;
    w.aabb_min = static_cast<float*>(P(SEEVR_B_BODY_AABB_MIN));
    w.aabb_max = static_cast<float*>(P(SEEVR_B_BODY_AABB_MAX));
    w.pairs = static_cast<uint32_t*>(P(SEEVR_B_COLLISION_PAIRS));
    w.sup_off = static_cast<const uint32_t*>(P(SEEVR_B_SUPPORT_OFFSET));
    w.sup_lut = static_cast<const uint32_t*>(P(SEEVR_B_SUPPORT_LOOKUP));
    w.lut_off = h->s.lut_off;
    w.hull_range = P(SEEVR_B_HULL_RANGE) ? static_cast<const uint32_t*>(P(SEEVR_B_HULL_RANGE))
                                         : h->s.derived_hull_range;
    w.body_scene = h->body_scene;
    w.scene_off = h->scene_off;
    w.bundle_off = h->bundle_off;
    w.body_bundle = h->body_bundle;
    w.max_pairs = h->caps.max_pairs;
    w.max_contacts = h->caps.max_contacts;
    const seevr_params& p = h->params;
    h->k.baumgarte = p.baumgarte;
    h->k.slop = p.slop;
    h->k.lin_damp = p.linear_damping;
    h->k.ang_damp = p.angular_damping;
    h->k.eps = p.mpr_eps;
    h->k.tol = p.mpr_tolerance;
    h->k.pgs_iterations = p.pgs_iterations;
    h->k.mpr_iterations = p.mpr_iterations;
    h->k.discover_trials = p.mpr_discover_trials;
    h->k.narrowphase = p.narrowphase;
}

__global__ void k_single_scene(uint32_t* body_scene, uint32_t* body_bundle, uint32_t* scene_off,
                               uint32_t* bundle_off, uint32_t nb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) body_scene[i] = body_bundle[i] = 0;
    if (i == 0) {
        scene_off[0] = bundle_off[0] = 0;
        scene_off[1] = bundle_off[1] = nb;
    }
}

// Greedy bundling of consecutive scenes: a bundle grows while its bodies stay
// within `target` (a scene larger than `target` is a bundle by itself).
std::vector<uint32_t> make_bundles(const uint32_t* body_offset, uint32_t num_scenes,
                                   uint32_t target, uint32_t* max_bodies) {
    std::vector<uint32_t> off{0};
    uint32_t start = 0, mx = 0;
    for (uint32_t s = 0; s < num_scenes; ++s) {
        const uint32_t end = body_offset[s + 1];
        if (end - body_offset[start] > target && s > start) {
            off.push_back(body_offset[s]);
            mx = std::max(mx, body_offset[s] - body_offset[start]);
            start = s;
        }
    }
    off.push_back(body_offset[num_scenes]);
    mx = std::max(mx, body_offset[num_scenes] - body_offset[start]);
    *max_bodies = mx;
    return off;
}

// Timed region helper: in profiling mode, brackets the launches of one
// stage with events on the handle's stream and accumulates milliseconds.
struct StageTimer {
    seevr_physics* h;
    seevr_profile* prof;
    cudaStream_t st;
    void begin() {
        if (prof) cudaEventRecord(h->ev[0], st);
    }
    void end(int stage) {
        if (!prof) return;
        cudaEventRecord(h->ev[1], st);
        cudaEventSynchronize(h->ev[1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
        prof->ms[stage] += ms;
    }
};

// NVTX range of one stage, named as the reference's profiler sections
// (Physics.step_names, physics.zig:22-32); free when no tool is attached.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

// One frame (Physics.step body) in four phases, so that scene groups can
// interleave their substeps: begin (hull ranges, input checks, shared
// lookups), per substep collide (gravity + AABB, broadphase, narrowphase,
// impulse clear) and solve (PGS), and end (frame-end integrate and render
// vertices).  Kernels go to stream st; n counts them.
struct FrameIssue {
    seevr_physics* h;
    uint32_t nv, substeps;
    float sub_dt;
    const float* g;
    cudaStream_t st;
    StageTimer T;
    bool render;
    uint64_t n = 0;

    FrameIssue(seevr_physics* h_, uint32_t nb, uint32_t nv_, uint32_t nhv, uint32_t substeps_,
               float dt, const float g_[3], cudaStream_t st_, seevr_profile* prof)
        : h(h_), nv(nv_), substeps(substeps_), sub_dt(dt / float(substeps_)),  // physics.zig:90
          g(g_), st(st_), T{h_, prof, st_},
          render(nv_ > 0 && !(h_->params.flags & SEEVR_FLAG_SKIP_RENDER_VERTS)) {
        World& w = h->w;
        w.nb = nb;
        w.nv = nv;
        w.nhv = nhv;
        w.ns = h->num_scenes;
        w.nbundles = h->num_bundles;
    }

    void begin() {
        World& w = h->w;
        if (!h->b.ptr[SEEVR_B_HULL_RANGE])
            n += launch_hull_range_from_geom_data(
                static_cast<const float*>(h->b.ptr[SEEVR_B_GEOM_DATA]), h->s.derived_hull_range,
                w.nb, st);
        if (h->check) {  // bounds-check mode: the caller's index arrays first
            const Range r("phys/check_inputs");
            World wc = w;
            wc.nv = render ? nv : 0u;
            n += launch_check_inputs(wc, uint32_t(h->b.bytes[SEEVR_B_SUPPORT_LOOKUP] / 4), st);
        }
        const Range r("phys/lut_alias");
        n += launch_lut_alias(w, h->s, st);
    }

    void collide(uint32_t s) {
        const World& w = h->w;
        T.begin();
        {
            const Range r("phys/aabb");  // with integrate and gravity
            n += launch_body_stage(w, h->k, (s > 0 ? kIntegrate : 0u) | kGravity | kAabb, sub_dt,
                                   g[0], g[1], g[2], st);
        }
        T.end(kStAabb);
        T.begin();
        {
            const Range r("phys/broad_phase");
            n += h->params.broadphase == SEEVR_BROADPHASE_LBVH
                     ? launch_broadphase_lbvh(w, h->s, h->lb, st)
                     : launch_broadphase_n2(w, h->s, h->max_scene_bodies, st);
            if (h->check) n += launch_check_pairs(w, st);
        }
        T.end(kStBroad);
        T.begin();
        {
            const Range r("phys/narrow_phase");
            n += launch_narrowphase(w, h->k, h->s, st);
            if (h->check) n += launch_check_contacts(w, st);
        }
        T.end(kStNarrow);
        // step 4 (clear impulses) is done by the contact scatter, which
        // zeroes the impulse of every contact it writes
    }

    void solve(uint32_t) {
        T.begin();
        {
            const Range r("phys/pgs_solve");
            n += launch_solver(h->w, h->k, h->s, h->params.solver, sub_dt, h->max_bundle_bodies,
                               h->smem_bundle_bodies, st);
        }
        T.end(kStSolve);
    }

    void end() {
        T.begin();
        {
            const Range r(render ? "phys/render_verts" : "phys/integrate");
            n += launch_body_stage(h->w, h->k, kIntegrate | (render ? kRenderVerts : 0u), sub_dt,
                                   g[0], g[1], g[2], st);
        }
        T.end(render ? kStRender : kStIntegrate);
    }
};

// Issue one frame (Physics.step body) on stream st; returns kernels launched.
uint64_t issue_frame(seevr_physics* h, uint32_t nb, uint32_t nv, uint32_t nhv, uint32_t substeps,
                     float dt, const float g[3], cudaStream_t st, seevr_profile* prof) {
    const Range frame("phys/step");
    FrameIssue f(h, nb, nv, nhv, substeps, dt, g, st, prof);
    f.begin();
    for (uint32_t s = 0; s < substeps; ++s) {
        f.collide(s);
        f.solve(s);
    }
    f.end();
    return f.n;
}

// ---- scene groups --------------------------------------------------------
// The groups' lists concatenated in group order are the canonical lists of
// the whole batch (a group's bodies all come after the previous group's), so
// the merge copies group g's entry i to the group's prefix + i, adding the
// group's first body to every body and geom index.  Counters are the true
// totals; entries beyond the caps are dropped and the overflow bit raised, as
// in the ungrouped step.  Each group's status bits are moved into the
// handle's status word.
__global__ void k_merge_groups(World w, GroupTable t) {
    uint32_t pp[kMaxGroups + 1], cp[kMaxGroups + 1];
    pp[0] = cp[0] = 0;
    for (uint32_t g = 0; g < t.n; ++g) {
        pp[g + 1] = pp[g] + t.g[g].counters[0];
        cp[g + 1] = cp[g] + t.g[g].counters[1];
    }
    const uint32_t np = min(pp[t.n], w.max_pairs), nc = min(cp[t.n], w.max_contacts);
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t d = tid; d < np; d += stride) {
        uint32_t g = 0;
        while (g + 1 < t.n && pp[g + 1] <= d) ++g;
        const GroupOut& o = t.g[g];
        const uint32_t i = d - pp[g];
        w.pairs[size_t(d) * 2] = o.pairs[size_t(i) * 2] + o.b0;
        w.pairs[size_t(d) * 2 + 1] = o.pairs[size_t(i) * 2 + 1] + o.b0;
    }
    for (uint32_t d = tid; d < nc; d += stride) {
        uint32_t g = 0;
        while (g + 1 < t.n && cp[g + 1] <= d) ++g;
        const GroupOut& o = t.g[g];
        const uint32_t i = d - cp[g];
        st3(w.c_pos, d, ld3(o.c_pos, i));
        st3(w.c_normal, d, ld3(o.c_normal, i));
        w.c_pen[d] = o.c_pen[i];
        w.c_a[d] = o.c_a[i] + o.b0;
        w.c_b[d] = o.c_b[i] + o.b0;
        w.lambda[d] = o.lambda[i];
    }
    if (tid == 0) {
        uint32_t f = 0;
        for (uint32_t g = 0; g < t.n; ++g) {
            f |= t.g[g].status[0];
            t.g[g].status[0] = 0u;
        }
        if (pp[t.n] > w.max_pairs) f |= kFlagPairOverflow;
        if (cp[t.n] > w.max_contacts) f |= kFlagContactOverflow;
        if (f) atomicOr(&w.status[0], f);
        w.counters[0] = pp[t.n];
        w.counters[1] = cp[t.n];
    }
}

// One frame of every group: forked from `st` onto the groups' streams (or,
// with per-stage profiling, group after group on `st`), joined back, merged.
// The state rows [b0, b0 + n) between the host arrays of `io` and the bound
// buffers (pos, vel, omega: 12 bytes a body; quat: 16), ordered on st.
void copy_state_in(const seevr_physics* h, uint32_t b0, uint32_t n, const seevr_host_state* io,
                   cudaStream_t st) {
    if (!io || n == 0) return;
    const size_t o3 = size_t(b0) * 3, o4 = size_t(b0) * 4;
    const auto H2D = cudaMemcpyHostToDevice;
    if (io->pos_in) cudaMemcpyAsync(h->w.pos + o3, io->pos_in + o3, size_t(n) * 12, H2D, st);
    if (io->quat_in) cudaMemcpyAsync(h->w.quat + o4, io->quat_in + o4, size_t(n) * 16, H2D, st);
    if (io->vel_in) cudaMemcpyAsync(h->w.vel + o3, io->vel_in + o3, size_t(n) * 12, H2D, st);
    if (io->omega_in) cudaMemcpyAsync(h->w.omega + o3, io->omega_in + o3, size_t(n) * 12, H2D, st);
}
void copy_state_out(const seevr_physics* h, uint32_t b0, uint32_t n, const seevr_host_state* io,
                    cudaStream_t st) {
    if (!io || n == 0) return;
    const size_t o3 = size_t(b0) * 3, o4 = size_t(b0) * 4;
    const auto D2H = cudaMemcpyDeviceToHost;
    if (io->pos_out) cudaMemcpyAsync(io->pos_out + o3, h->w.pos + o3, size_t(n) * 12, D2H, st);
    if (io->quat_out) cudaMemcpyAsync(io->quat_out + o4, h->w.quat + o4, size_t(n) * 16, D2H, st);
    if (io->vel_out) cudaMemcpyAsync(io->vel_out + o3, h->w.vel + o3, size_t(n) * 12, D2H, st);
    if (io->omega_out) cudaMemcpyAsync(io->omega_out + o3, h->w.omega + o3, size_t(n) * 12, D2H, st);
}

// io (seevr_physics_step_io, not with prof): each group's state rows are
// copied in on the group's stream before its frame and out after it.
uint64_t issue_frame_groups(seevr_physics* h, uint32_t nv, uint32_t nhv, uint32_t substeps,
                            float dt, const float g[3], cudaStream_t st, seevr_profile* prof,
                            const seevr_host_state* io = nullptr) {
    uint64_t n = 0;
    if (prof) {
        for (auto& G : h->groups)
            if (G.h) n += issue_frame(G.h, G.nb, nv, nhv, substeps, dt, g, st, prof);
    } else {
        // Each group's whole frame on its own stream; the GPU's scheduler
        // interleaves them.  (Serialising the groups' collision stages in
        // round-robin order, so that each solver runs beside another group's
        // collision stages, measured slower: 15.7 against 12.8 ms per frame
        // with 4 groups, 13.9 against 13.4 with 2; a group's collision
        // kernels alone do not fill the GPU.)
        const Range frame("phys/step");
        cudaEventRecord(h->fork, st);
        for (auto& G : h->groups) {
            if (!G.h) continue;  // a group of empty scenes
            cudaStreamWaitEvent(G.stream, h->fork, 0);
            copy_state_in(h, G.b0, G.nb, io, G.stream);
            FrameIssue f(G.h, G.nb, nv, nhv, substeps, dt, g, G.stream, nullptr);
            f.begin();
            for (uint32_t s = 0; s < substeps; ++s) {
                f.collide(s);
                f.solve(s);
            }
            f.end();
            n += f.n;
            copy_state_out(h, G.b0, G.nb, io, G.stream);
            cudaEventRecord(G.done, G.stream);
            cudaStreamWaitEvent(st, G.done, 0);
        }
    }
    GroupTable t{};
    t.n = uint32_t(h->groups.size());
    for (uint32_t i = 0; i < t.n; ++i) t.g[i] = h->groups[i].out;
    const uint32_t cap = std::max(h->caps.max_pairs, h->caps.max_contacts);
    const uint32_t blocks = std::min((cap + 255) / 256, uint32_t(h->sm_count) * 8u);
    k_merge_groups<<<std::max(blocks, 1u), 256, 0, st>>>(h->w, t);
    return n + 1;
}

__global__ void k_local_geom_body(const uint32_t* __restrict__ geom_body, uint32_t b0, uint32_t n,
                                  uint32_t* __restrict__ out, uint32_t* bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = geom_body[b0 + i];
    const bool inside = b >= b0 && b - b0 < n;
    out[i] = inside ? b - b0 : i;
    if (!inside) atomicOr(bad, 1u);
}

// Split the scenes into h->scene_groups contiguous ranges of about equal
// bodies and create one sub-handle per range: bound to the handle's arrays
// at the range's offset (state, masses, geoms, AABBs, render and hull
// ranges), to the shared hull vertices, lookup table and render vertices,
// and to its own pair and contact lists and geom -> body map in local
// indices.  Each group keeps the handle's capacities, so no group overflows
// where the whole batch would not.
seevr_status build_groups(seevr_physics* h) {
    free_groups(h);
    const std::vector<uint32_t>& off = h->scene_offsets_host;
    const uint32_t ns = h->num_scenes, G = std::min(h->scene_groups, ns);
    if (G <= 1) return SEEVR_OK;
    if (h->params.broadphase != SEEVR_BROADPHASE_N2 || h->check)
        return fail(SEEVR_ERR_NOT_SUPPORTED,
                    "scene groups need the all-pairs broadphase and no bounds-check mode");
    if (!h->fork && cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(SEEVR_ERR_CUDA, "cudaEventCreate failed");
    const uint32_t nb = off[ns];
    std::vector<uint32_t> cut{0};
    for (uint32_t s = 1, k = 1; s < ns && k < G; ++s)
        if (uint64_t(off[s]) * G >= uint64_t(nb) * k) {
            cut.push_back(s);
            ++k;
        }
    cut.push_back(ns);
    const seevr_caps& pc = h->caps;
    uint32_t* bad = nullptr;
    if (cudaMalloc(&bad, sizeof(uint32_t)) != cudaSuccess || cudaMemset(bad, 0, 4) != cudaSuccess) {
        cudaGetLastError();
        return fail(SEEVR_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    }
    seevr_status st = SEEVR_OK;
    for (size_t gi = 0; gi + 1 < cut.size() && st == SEEVR_OK; ++gi) {
        h->groups.emplace_back();
        auto& g = h->groups.back();
        const uint32_t s0 = cut[gi], s1 = cut[gi + 1];
        g.b0 = off[s0];
        g.nb = off[s1] - off[s0];
        auto alloc = [&](size_t bytes) -> void* {
            void* p = nullptr;
            if (st != SEEVR_OK) return nullptr;
            if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
                cudaGetLastError();
                st = fail(SEEVR_ERR_OUT_OF_MEMORY, "cudaMalloc of a scene group's lists failed");
                return nullptr;
            }
            g.allocs.push_back(p);
            return p;
        };
        seevr_bindings b = h->b;
        auto shift = [&](int i, size_t elem) {
            if (!b.ptr[i]) return;
            b.ptr[i] = static_cast<char*>(h->b.ptr[i]) + size_t(g.b0) * elem;
            b.bytes[i] = size_t(g.nb) * elem;
        };
        shift(SEEVR_B_BODY_POS, 12);
        shift(SEEVR_B_BODY_QUAT, 16);
        shift(SEEVR_B_BODY_VEL, 12);
        shift(SEEVR_B_BODY_OMEGA, 12);
        shift(SEEVR_B_BODY_INV_MASS, 4);
        shift(SEEVR_B_BODY_INV_INERTIA, 12);
        shift(SEEVR_B_BODY_VERT_START, 4);
        shift(SEEVR_B_BODY_VERT_COUNT, 4);
        shift(SEEVR_B_GEOM_DATA, 32);
        shift(SEEVR_B_GEOM_FRICTION, 4);
        shift(SEEVR_B_GEOM_RESTITUTION, 4);
        shift(SEEVR_B_BODY_AABB_MIN, 12);
        shift(SEEVR_B_BODY_AABB_MAX, 12);
        shift(SEEVR_B_SUPPORT_OFFSET, 4);
        shift(SEEVR_B_HULL_RANGE, 8);
        const size_t P = pc.max_pairs, C = pc.max_contacts;
        auto own = [&](int i, size_t bytes) {
            b.ptr[i] = alloc(bytes);
            b.bytes[i] = bytes;
        };
        own(SEEVR_B_GEOM_BODY_IDX, size_t(g.nb) * 4);
        own(SEEVR_B_COLLISION_PAIRS, P * 8);
        own(SEEVR_B_CONTACT_POS, C * 12);
        own(SEEVR_B_CONTACT_NORMAL, C * 12);
        own(SEEVR_B_CONTACT_PEN, C * 4);
        own(SEEVR_B_CONTACT_GEOM_A, C * 4);
        own(SEEVR_B_CONTACT_GEOM_B, C * 4);
        own(SEEVR_B_LAMBDA_N, C * 4);
        own(SEEVR_B_COUNTERS, 16);
        if (st != SEEVR_OK) break;
        cudaMemset(b.ptr[SEEVR_B_COUNTERS], 0, 16);
        g.out = GroupOut{static_cast<const uint32_t*>(b.ptr[SEEVR_B_COUNTERS]), nullptr,
                         static_cast<const uint32_t*>(b.ptr[SEEVR_B_COLLISION_PAIRS]),
                         static_cast<const float*>(b.ptr[SEEVR_B_CONTACT_POS]),
                         static_cast<const float*>(b.ptr[SEEVR_B_CONTACT_NORMAL]),
                         static_cast<const float*>(b.ptr[SEEVR_B_CONTACT_PEN]),
                         static_cast<const uint32_t*>(b.ptr[SEEVR_B_CONTACT_GEOM_A]),
                         static_cast<const uint32_t*>(b.ptr[SEEVR_B_CONTACT_GEOM_B]),
                         static_cast<const float*>(b.ptr[SEEVR_B_LAMBDA_N]), g.b0};
        if (g.nb == 0) {  // empty scenes only: nothing to step, counters stay 0
            uint32_t* word = static_cast<uint32_t*>(alloc(16));
            if (word) cudaMemset(word, 0, 16);
            g.out.status = word;
            continue;
        }
        const uint32_t n = g.nb;
        k_local_geom_body<<<(n + 255) / 256, 256>>>(
            static_cast<const uint32_t*>(h->b.ptr[SEEVR_B_GEOM_BODY_IDX]), g.b0, g.nb,
            static_cast<uint32_t*>(b.ptr[SEEVR_B_GEOM_BODY_IDX]), bad);
        seevr_caps c = pc;
        c.max_bodies = n;
        c.max_scenes = s1 - s0;
        seevr_params p = h->params;
        p.flags &= ~uint32_t(SEEVR_FLAG_NO_SYNC | SEEVR_FLAG_CUDA_GRAPH);
        st = seevr_physics_create(&b, &c, &p, &g.h);
        if (st != SEEVR_OK) break;
        std::vector<uint32_t> lo(s1 - s0 + 1);
        for (uint32_t s = s0; s <= s1; ++s) lo[s - s0] = off[s] - g.b0;
        g.h->narrow_blocks_per_sm = h->narrow_blocks_per_sm;
        g.h->s.narrow_blocks = h->s.narrow_blocks;
        g.h->s.narrow_per_sm = h->s.narrow_per_sm;
        g.h->s.bp_tile_rows = h->s.bp_tile_rows;
        g.h->s.wait_limit = h->s.wait_limit;
        g.h->s.giant_min = h->s.giant_min;
        g.h->s.order_pairs = 1;  // pairs by support path (narrowphase.cu)
        g.h->s.sweep_warps = 2;  // 64-wide solver passes (solver.cu)
        st = seevr_physics_set_scenes(g.h, lo.data(), s1 - s0);
        if (st != SEEVR_OK) break;
        if (cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming) != cudaSuccess)
            st = fail(SEEVR_ERR_CUDA, "cudaStreamCreate for a scene group failed");
        g.out.status = g.h->s.status;
    }
    uint32_t bad_host = 0;
    if (st == SEEVR_OK && cudaMemcpy(&bad_host, bad, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        st = fail(SEEVR_ERR_CUDA, "cudaMemcpy failed");
    cudaFree(bad);
    if (st == SEEVR_OK && bad_host)
        st = fail(SEEVR_ERR_INVALID_ARGUMENT,
                  "scene groups need every geom's body inside its own scene (geom_body_idx)");
    if (st != SEEVR_OK) free_groups(h);
    return st;
}

seevr_status check_step_args(seevr_physics* h, uint32_t nb, uint32_t nv, uint32_t nhv) {
    if (nb > h->caps.max_bodies)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_bodies exceeds caps.max_bodies");
    if (nhv > h->caps.max_hull_verts)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_hull_verts exceeds caps.max_hull_verts");
    if (nv > h->caps.max_vertices)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_vertices exceeds caps.max_vertices");
    if (nv > 0 && !(h->params.flags & SEEVR_FLAG_SKIP_RENDER_VERTS) &&
        (!h->b.ptr[SEEVR_B_VERTICES] || !h->b.ptr[SEEVR_B_ORIG_VERTICES]))
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "render vertices requested but bindings 13/14 are NULL");
    if (h->scenes_set) {
        // scene offsets were validated against max_bodies at set time; the
        // last offset must equal num_bodies
        if (nb != h->single_scene_nb)
            return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_bodies differs from the declared scenes' total");
    }
    return SEEVR_OK;
}

// Overlap-word rows of the all-pairs broadphase for nb bodies in scenes of
// at most maxs bodies: one 32-bit word per 32 columns of the largest scene.
// Layouts needing more than 1 GiB go without (the write pass re-tests).
seevr_status ensure_bp_mask(seevr_physics* h, uint32_t nb, uint32_t maxs) {
    // (maxs + 31) / 32 words: column-aligned words of the shared-memory
    // kernel; the global-memory kernel's row-relative words need no more
    const uint32_t stride = maxs > 0 ? (maxs + 31) / 32 : 1u;
    const size_t words = size_t(nb ? nb : 1) * stride;
    if (words * sizeof(uint32_t) > (size_t(1) << 30)) {
        if (h->s.bp_mask) cudaFree(h->s.bp_mask);
        h->s.bp_mask = nullptr;
        h->s.bp_stride = 0;
        h->bp_mask_cap = 0;
        return SEEVR_OK;
    }
    if (words > h->bp_mask_cap) {
        if (h->s.bp_mask) cudaFree(h->s.bp_mask);
        h->s.bp_mask = nullptr;
        h->bp_mask_cap = 0;
        void* q = nullptr;
        if (cudaMalloc(&q, words * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            return fail(SEEVR_ERR_OUT_OF_MEMORY, "cudaMalloc of the broadphase overlap words failed");
        }
        h->s.bp_mask = static_cast<uint32_t*>(q);
        h->bp_mask_cap = words;
    }
    h->s.bp_stride = stride;
    return SEEVR_OK;
}

// Tile table of the all-pairs broadphase: ceil(n / kTileRows) blocks for a
// scene of n bodies, so that large scenes are spread over as many warps as
// their rows need (only for layouts the shared-memory kernel takes).
seevr_status set_bp_tiles(seevr_physics* h, const uint32_t* body_offset, uint32_t num_scenes,
                          uint32_t maxs) {
    h->s.bp_ntiles = 0;
    if (maxs > kTileBodies) return SEEVR_OK;
    std::vector<uint2> tiles;
    for (uint32_t s = 0; s < num_scenes; ++s) {
        const uint32_t n = body_offset[s + 1] - body_offset[s];
        const uint32_t rows = h->s.bp_tile_rows ? h->s.bp_tile_rows : kTileRows;
        const uint32_t k = std::max(1u, (n + rows - 1) / rows);
        for (uint32_t j = 0; j < k; ++j) tiles.push_back(make_uint2(s, j | (k << 16)));
    }
    if (tiles.size() > h->bp_tiles_cap) {
        if (h->s.bp_tiles) cudaFree(h->s.bp_tiles);
        h->s.bp_tiles = nullptr;
        h->bp_tiles_cap = 0;
        void* q = nullptr;
        if (cudaMalloc(&q, tiles.size() * sizeof(uint2)) != cudaSuccess) {
            cudaGetLastError();
            return fail(SEEVR_ERR_OUT_OF_MEMORY, "cudaMalloc of the broadphase tile table failed");
        }
        h->s.bp_tiles = static_cast<uint2*>(q);
        h->bp_tiles_cap = uint32_t(tiles.size());
    }
    SEEVR_CUDA(cudaMemcpy(h->s.bp_tiles, tiles.data(), tiles.size() * sizeof(uint2),
                          cudaMemcpyHostToDevice));
    h->s.bp_ntiles = uint32_t(tiles.size());
    return SEEVR_OK;
}

seevr_status ensure_single_scene(seevr_physics* h, uint32_t nb, cudaStream_t st) {
    if (h->scenes_set || h->single_scene_nb == nb) return SEEVR_OK;
    const seevr_status ms = ensure_bp_mask(h, nb, nb);
    if (ms != SEEVR_OK) return ms;
    const uint32_t n = nb > 0 ? nb : 1;
    k_single_scene<<<(n + 255) / 256, 256, 0, st>>>(h->body_scene, h->body_bundle, h->scene_off,
                                                     h->bundle_off, nb);
    SEEVR_CUDA(cudaGetLastError());
    h->launches += 1;
    h->single_scene_nb = nb;
    h->max_scene_bodies = nb;
    h->max_bundle_bodies = nb;
    h->smem_bundle_bodies = nb;
    h->num_scenes = 1;
    h->num_bundles = 1;
    return SEEVR_OK;
}

seevr_status collect_flags(seevr_physics* h, cudaStream_t st, bool* overflow) {
    uint32_t f[4] = {0, 0, 0, 0};
    SEEVR_CUDA(cudaMemcpyAsync(f, h->s.status, sizeof f, cudaMemcpyDeviceToHost, st));
    SEEVR_CUDA(cudaMemsetAsync(h->s.status, 0, sizeof(uint32_t), st));
    SEEVR_CUDA(cudaMemsetAsync(h->s.status + 2, 0, 2 * sizeof(uint32_t), st));
    SEEVR_CUDA(cudaStreamSynchronize(st));
    h->host_flags |= f[0];
    *overflow = (f[0] & (kFlagPairOverflow | kFlagContactOverflow)) != 0;
    if (f[0] & kFlagCheckFailed)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, std::string("bounds check: ") + check_name(f[2]) +
                                                    " (index " + std::to_string(f[3]) + ")");
    if (f[0] & kFlagTimeout) return fail(SEEVR_ERR_TIMEOUT, "a device-side wait exceeded its limit");
    return SEEVR_OK;
}

}  // namespace

extern "C" {

void seevr_params_default(seevr_params* p) {
    if (!p) return;
    p->pgs_iterations = 4;
    p->baumgarte = 0.2f;
    p->slop = 0.005f;
    p->linear_damping = 0.999f;
    p->angular_damping = 0.998f;
    p->mpr_eps = 1e-6f;
    p->mpr_tolerance = 1e-6f;
    p->mpr_iterations = 50;
    p->mpr_discover_trials = 15;
    p->broadphase = SEEVR_BROADPHASE_N2;
    p->solver = SEEVR_SOLVER_WAVEFRONT;
    p->flags = 0;
    p->bundle_bodies = 0;
    p->narrowphase = SEEVR_NARROWPHASE_MPR;
}

seevr_status seevr_physics_create(const seevr_bindings* b, const seevr_caps* caps,
                                  const seevr_params* params, seevr_physics** out) {
    if (!out) return fail(SEEVR_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!b || !caps) return fail(SEEVR_ERR_INVALID_ARGUMENT, "bindings or caps is NULL");
    if (caps->max_bodies == 0) return fail(SEEVR_ERR_INVALID_ARGUMENT, "caps.max_bodies is 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SEEVR_ERR_NO_DEVICE, "no CUDA device");
    }
    for (int i = 0; i < SEEVR_NUM_BINDINGS; ++i) {
        const uint64_t need = required_bytes(i, *caps);
        if (need == 0) continue;
        if (!b->ptr[i])
            return fail(SEEVR_ERR_INVALID_ARGUMENT, "binding " + std::to_string(i) + " is NULL");
        if (b->bytes[i] < need)
            return fail(SEEVR_ERR_INVALID_ARGUMENT, "binding " + std::to_string(i) + " holds " +
                                                        std::to_string(b->bytes[i]) + " bytes, needs " +
                                                        std::to_string(need));
    }
    if (b->ptr[SEEVR_B_HULL_RANGE] && b->bytes[SEEVR_B_HULL_RANGE] < uint64_t(caps->max_bodies) * 8)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "binding 30 (hull range) is undersized");
    seevr_params p;
    seevr_params_default(&p);
    if (params) p = *params;
    if (p.broadphase > SEEVR_BROADPHASE_LBVH || p.solver > SEEVR_SOLVER_COLORED ||
        p.narrowphase > SEEVR_NARROWPHASE_GJK_EPA)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "unknown broadphase, solver or narrowphase");

    auto* h = new seevr_physics();
    cudaGetDevice(&h->device);
    h->b = *b;
    h->caps = *caps;
    if (h->caps.max_scenes == 0) h->caps.max_scenes = 1;
    h->params = p;
    seevr_status st = SEEVR_OK;
    const seevr_caps& c = h->caps;
    const uint32_t scan_n = std::max(std::max(std::max(c.max_bodies, c.max_pairs), c.max_contacts), 1u);
    h->s.scan_tiles_cap = (scan_n + 2047) / 2048 + 2;
    h->s.wait_limit = kSpinLimit;
    h->lb.wait_limit = kSpinLimit;
    if (const char* e = std::getenv("SEEVR_CHECK")) h->check = std::strcmp(e, "1") == 0;
#define ALLOC(ptr, n)                                   \
    if (st == SEEVR_OK) st = dev_alloc(h, &(ptr), (n));
    ALLOC(h->s.status, 4);
    ALLOC(h->s.row_count, c.max_bodies);
    ALLOC(h->s.row_off, c.max_bodies);
    ALLOC(h->s.scan_tiles, h->s.scan_tiles_cap);
    ALLOC(h->s.pair_res0, c.max_pairs);
    ALLOC(h->s.pair_res1, c.max_pairs);
    ALLOC(h->s.pair_flag, c.max_pairs);
    ALLOC(h->s.pair_coff, c.max_pairs);
    ALLOC(h->s.pair_class, 2 * kPairClasses);
    ALLOC(h->s.lut_rep, kLutHullMax);
    ALLOC(h->s.lut_off, c.max_bodies);
    ALLOC(h->s.s_ra, size_t(c.max_contacts) * 3);
    ALLOC(h->s.s_rb, size_t(c.max_contacts) * 3);
    ALLOC(h->s.s_bias, c.max_contacts);
    ALLOC(h->s.s_kn, c.max_contacts);
    ALLOC(h->s.s_mu, c.max_contacts);
    ALLOC(h->s.s_ab, size_t(c.max_contacts) * 2);
    ALLOC(h->s.s_level, c.max_contacts);
    ALLOC(h->s.s_order, c.max_contacts);
    ALLOC(h->s.s_lvl_start, size_t(c.max_contacts) + c.max_scenes + 1);
    ALLOC(h->s.s_n, size_t(c.max_contacts) * 3);
    ALLOC(h->s.s_lam, c.max_contacts);
    ALLOC(h->s.s_abp, size_t(c.max_contacts) * 2);
    ALLOC(h->s.s_rec, size_t(c.max_contacts) * kRecWords);
    ALLOC(h->s.bundle_c0, size_t(c.max_scenes) + 2);
    ALLOC(h->body_bundle, c.max_bodies);
    ALLOC(h->s.s_R, size_t(c.max_bodies) * 9);
    ALLOC(h->s.s_last, c.max_bodies);
    ALLOC(h->s.derived_hull_range, size_t(c.max_bodies) * 2);
    ALLOC(h->body_scene, c.max_bodies);
    ALLOC(h->scene_off, size_t(c.max_scenes) + 1);
    ALLOC(h->bundle_off, size_t(c.max_scenes) + 1);
    if (c.max_bodies > kWarpMaxBodies) {  // scenes large enough for the island solver
        IslandScratch& is = h->s.isl;
        const size_t nc = c.max_contacts;
        ALLOC(is.parent, c.max_bodies);
        ALLOC(is.keys_in, nc);
        ALLOC(is.vals_in, nc);
        ALLOC(is.keys_tmp, nc);
        ALLOC(is.vals_tmp, nc);
        ALLOC(is.keys_out, nc);
        ALLOC(is.perm, nc);
        ALLOC(is.head, nc);
        ALLOC(is.idx, nc);
        ALLOC(is.start, nc + 1);
        ALLOC(is.count, 1);
        ALLOC(is.lvl, 2 * nc + 2);
        ALLOC(is.sort_hist, 4 * 256);
        ALLOC(is.sort_status, lbvh_status_words(c.max_contacts));
        GiantScratch& gs = is.giant;
        ALLOC(gs.list, nc);
        ALLOC(gs.colour, nc);
        ALLOC(gs.order, nc);
        ALLOC(gs.used, c.max_bodies);
        ALLOC(gs.prio, c.max_bodies);
        ALLOC(gs.hist, kGiantMaxColours);
        ALLOC(gs.first, kGiantMaxColours + 1);
        ALLOC(gs.ctr, kGiantCtrWords);
    }
    if (p.broadphase == SEEVR_BROADPHASE_LBVH) {
        LbvhScratch& lb = h->lb;
        const size_t n = c.max_bodies;
        lb.cap = c.max_bodies;
        ALLOC(lb.centroid, n * 3);
        ALLOC(lb.bounds_o, 6);
        ALLOC(lb.bounds_f, 6);
        ALLOC(lb.keys_a, n);
        ALLOC(lb.vals_a, n);
        ALLOC(lb.keys_b, n);
        ALLOC(lb.vals_b, n);
        ALLOC(lb.keys_sorted, n);
        ALLOC(lb.vals_sorted, n);
        ALLOC(lb.hist, 4 * 256);
        ALLOC(lb.status, lbvh_status_words(c.max_bodies));
        ALLOC(lb.left, 2 * n);
        ALLOC(lb.right, 2 * n);
        ALLOC(lb.parent, 2 * n);
        ALLOC(lb.flags, n);
        ALLOC(lb.node_min, 6 * n);
        ALLOC(lb.node_max, 6 * n);
        ALLOC(lb.static_list, n);
        ALLOC(lb.static_count, 1);
        ALLOC(lb.bfs, size_t(kStaticBlocks) * 3 * 2 * n);
        ALLOC(lb.row_cache, size_t(kRowCache) * n);
        ALLOC(lb.packed, size_t(4) * n);
    }
#undef ALLOC
    if (st == SEEVR_OK && cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        st = fail(SEEVR_ERR_CUDA, "cudaStreamCreate failed");
    if (st == SEEVR_OK && (cudaEventCreate(&h->ev[0]) != cudaSuccess ||
                           cudaEventCreate(&h->ev[1]) != cudaSuccess))
        st = fail(SEEVR_ERR_CUDA, "cudaEventCreate failed");
    if (st == SEEVR_OK && cudaMemset(h->s.status, 0, 16) != cudaSuccess)
        st = fail(SEEVR_ERR_CUDA, "cudaMemset failed");
    if (st == SEEVR_OK && init_solver() != cudaSuccess)
        st = fail(SEEVR_ERR_CUDA, "cudaFuncSetAttribute for the solver failed");
    if (st == SEEVR_OK) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) == cudaSuccess &&
            sms > 0)
            h->sm_count = sms;
        h->s.narrow_blocks = uint32_t(h->sm_count) * h->narrow_blocks_per_sm;
        h->s.narrow_per_sm = h->narrow_blocks_per_sm;
        h->s.bp_tile_rows = kTileRows;
    }
    if (st == SEEVR_OK && init_broadphase() != cudaSuccess)
        st = fail(SEEVR_ERR_CUDA, "cudaFuncSetAttribute for the broadphase failed");
    if (st != SEEVR_OK) {
        cudaGetLastError();
        free_all(h);
        delete h;
        return st;
    }
    setup_world(h);
    *out = h;
    return SEEVR_OK;
}

seevr_status seevr_physics_set_scenes(seevr_physics* h, const uint32_t* body_offset,
                                      uint32_t num_scenes) {
    if (!h || !body_offset || num_scenes == 0)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "bad scene arguments");
    if (num_scenes > h->caps.max_scenes)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_scenes exceeds caps.max_scenes");
    if (body_offset[0] != 0) return fail(SEEVR_ERR_INVALID_ARGUMENT, "body_offset[0] must be 0");
    uint32_t maxs = 0;
    for (uint32_t s = 0; s < num_scenes; ++s) {
        if (body_offset[s + 1] < body_offset[s])
            return fail(SEEVR_ERR_INVALID_ARGUMENT, "body_offset must be non-decreasing");
        maxs = std::max(maxs, body_offset[s + 1] - body_offset[s]);
    }
    const uint32_t nb = body_offset[num_scenes];
    if (nb > h->caps.max_bodies)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "scenes hold more bodies than caps.max_bodies");
    h->scene_offsets_host.assign(body_offset, body_offset + num_scenes + 1);
    std::vector<uint32_t> bs(nb ? nb : 1, 0);
    for (uint32_t s = 0; s < num_scenes; ++s)
        for (uint32_t i = body_offset[s]; i < body_offset[s + 1]; ++i) bs[i] = s;
    SEEVR_CUDA(cudaSetDevice(h->device));
    SEEVR_CUDA(cudaMemcpy(h->body_scene, bs.data(), sizeof(uint32_t) * nb, cudaMemcpyHostToDevice));
    SEEVR_CUDA(cudaMemcpy(h->scene_off, body_offset, sizeof(uint32_t) * (num_scenes + 1),
                          cudaMemcpyHostToDevice));
    if (h->params.broadphase == SEEVR_BROADPHASE_LBVH && num_scenes > 1)
        return fail(SEEVR_ERR_NOT_SUPPORTED,
                    "the LBVH broadphase steps a single scene; use the all-pairs broadphase for "
                    "batches");
    const seevr_status ms = ensure_bp_mask(h, nb, maxs);
    if (ms != SEEVR_OK) return ms;
    const seevr_status ts = set_bp_tiles(h, body_offset, num_scenes, maxs);
    if (ts != SEEVR_OK) return ts;
    uint32_t max_bundle = 0;
    const uint32_t target = h->params.bundle_bodies ? h->params.bundle_bodies : 512u;
    const std::vector<uint32_t> bundles = make_bundles(body_offset, num_scenes, target, &max_bundle);
    SEEVR_CUDA(cudaMemcpy(h->bundle_off, bundles.data(), sizeof(uint32_t) * bundles.size(),
                          cudaMemcpyHostToDevice));
    for (size_t k = 0; k + 1 < bundles.size(); ++k)
        for (uint32_t i = bundles[k]; i < bundles[k + 1]; ++i) bs[i] = uint32_t(k);
    SEEVR_CUDA(cudaMemcpy(h->body_bundle, bs.data(), sizeof(uint32_t) * nb, cudaMemcpyHostToDevice));
    h->num_bundles = uint32_t(bundles.size() - 1);
    h->max_bundle_bodies = max_bundle;
    h->smem_bundle_bodies = h->num_bundles > 1 ? std::min(max_bundle, target) : max_bundle;
    h->num_scenes = num_scenes;
    h->scenes_set = true;
    h->single_scene_nb = nb;
    h->max_scene_bodies = maxs;
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    if (h->scene_groups > 1 || !h->groups.empty()) return build_groups(h);
    return SEEVR_OK;
}

seevr_status seevr_physics_step(seevr_physics* h, uint32_t num_bodies, uint32_t num_vertices,
                                uint32_t num_hull_verts, uint32_t substeps, float dt,
                                const float gravity[3], seevr_profile* prof) {
    if (!h || !gravity) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle or gravity is NULL");
    if (num_bodies == 0 || substeps == 0) return SEEVR_OK;  // physics.zig:81
    seevr_status st = check_step_args(h, num_bodies, num_vertices, num_hull_verts);
    if (st != SEEVR_OK) return st;
    SEEVR_CUDA(cudaSetDevice(h->device));
    st = ensure_single_scene(h, num_bodies, h->stream);
    if (st != SEEVR_OK) return st;
    if (prof) {
        prof->calls += 1;
    }
    if (!prof && (h->params.flags & SEEVR_FLAG_CUDA_GRAPH)) {
        // the frame replayed from its captured graph on the handle's stream
        // (one launch instead of one per kernel), then the same wait
        st = seevr_physics_step_async(h, num_bodies, num_vertices, num_hull_verts, substeps, dt,
                                      gravity, 1, h->stream);
        if (st != SEEVR_OK) return st;
    } else {
        h->launches += h->groups.empty()
                           ? issue_frame(h, num_bodies, num_vertices, num_hull_verts, substeps, dt,
                                         gravity, h->stream, prof)
                           : issue_frame_groups(h, num_vertices, num_hull_verts, substeps, dt,
                                                gravity, h->stream, prof);
    }
    SEEVR_CUDA(cudaGetLastError());
    if (h->params.flags & SEEVR_FLAG_NO_SYNC) return SEEVR_OK;
    bool overflow = false;
    st = collect_flags(h, h->stream, &overflow);
    if (st != SEEVR_OK) return st;
    if (overflow) return fail(SEEVR_ERR_CAPACITY, "pairs or contacts exceeded the caps");
    return SEEVR_OK;
}

namespace {

// One frame's kernels, with io's copies (ungrouped: all rows before and
// after the frame on st; grouped: per group, on the group's stream).
uint64_t issue_frame_io(seevr_physics* h, uint32_t nb, uint32_t nv, uint32_t nhv,
                        uint32_t substeps, float dt, const float g[3], cudaStream_t st,
                        const seevr_host_state* io) {
    if (!h->groups.empty()) return issue_frame_groups(h, nv, nhv, substeps, dt, g, st, nullptr, io);
    copy_state_in(h, 0, nb, io, st);
    const uint64_t n = issue_frame(h, nb, nv, nhv, substeps, dt, g, st, nullptr);
    copy_state_out(h, 0, nb, io, st);
    return n;
}

seevr_status run_frames(seevr_physics* h, uint32_t num_bodies, uint32_t num_vertices,
                        uint32_t num_hull_verts, uint32_t substeps, float dt,
                        const float gravity[3], uint32_t frames, cudaStream_t s,
                        const seevr_host_state* io) {
    if (!(h->params.flags & SEEVR_FLAG_CUDA_GRAPH)) {
        for (uint32_t f = 0; f < frames; ++f)
            h->launches += issue_frame_io(h, num_bodies, num_vertices, num_hull_verts, substeps, dt,
                                          gravity, s, io);
        SEEVR_CUDA(cudaGetLastError());
        return SEEVR_OK;
    }
    GraphKey key{num_bodies, num_vertices, num_hull_verts, substeps, dt,
                 {gravity[0], gravity[1], gravity[2]}, {}};
    if (io) {
        const void* p[8] = {io->pos_in,  io->quat_in,  io->vel_in,  io->omega_in,
                            io->pos_out, io->quat_out, io->vel_out, io->omega_out};
        for (int i = 0; i < 8; ++i) key.io[i] = p[i];
    }
    if (!h->graph_exec || !(h->graph_key == key)) {
        if (h->graph_exec) {
            cudaGraphExecDestroy(h->graph_exec);
            h->graph_exec = nullptr;
        }
        // captured on the handle's own stream (the legacy default stream
        // cannot be captured), launched on the caller's
        const cudaStream_t cap = h->stream;
        cudaGraph_t g = nullptr;
        SEEVR_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const uint64_t n = issue_frame_io(h, num_bodies, num_vertices, num_hull_verts, substeps, dt,
                                          gravity, cap, io);
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        if (e != cudaSuccess) return fail(SEEVR_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&h->graph_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(SEEVR_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        h->graph_key = key;
        h->graph_kernels = n;
    }
    for (uint32_t f = 0; f < frames; ++f) SEEVR_CUDA(cudaGraphLaunch(h->graph_exec, s));
    h->launches += h->graph_kernels * frames;
    return SEEVR_OK;
}

bool page_locked(const void* p) {
    if (!p) return true;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

seevr_status seevr_physics_step_async(seevr_physics* h, uint32_t num_bodies, uint32_t num_vertices,
                                      uint32_t num_hull_verts, uint32_t substeps, float dt,
                                      const float gravity[3], uint32_t frames, void* stream) {
    if (!h || !gravity) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle or gravity is NULL");
    if (num_bodies == 0 || substeps == 0 || frames == 0) return SEEVR_OK;
    seevr_status st = check_step_args(h, num_bodies, num_vertices, num_hull_verts);
    if (st != SEEVR_OK) return st;
    SEEVR_CUDA(cudaSetDevice(h->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    st = ensure_single_scene(h, num_bodies, s);
    if (st != SEEVR_OK) return st;
    return run_frames(h, num_bodies, num_vertices, num_hull_verts, substeps, dt, gravity, frames, s,
                      nullptr);
}

seevr_status seevr_physics_step_io(seevr_physics* h, uint32_t num_bodies, uint32_t num_vertices,
                                   uint32_t num_hull_verts, uint32_t substeps, float dt,
                                   const float gravity[3], const seevr_host_state* io,
                                   void* stream) {
    if (!h || !gravity || !io) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle, gravity or io is NULL");
    if (num_bodies == 0 || substeps == 0) return SEEVR_OK;
    seevr_status st = check_step_args(h, num_bodies, num_vertices, num_hull_verts);
    if (st != SEEVR_OK) return st;
    SEEVR_CUDA(cudaSetDevice(h->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    const void* p[8] = {io->pos_in,  io->quat_in,  io->vel_in,  io->omega_in,
                        io->pos_out, io->quat_out, io->vel_out, io->omega_out};
    bool locked = true;
    for (const void* q : p) locked = locked && page_locked(q);
    if (!locked) {
        // pageable memory: one copy after another, each waited for
        st = seevr_physics_upload_state(h, num_bodies, io->pos_in, io->quat_in, io->vel_in,
                                        io->omega_in);
        if (st != SEEVR_OK) return st;
        st = seevr_physics_step_async(h, num_bodies, num_vertices, num_hull_verts, substeps, dt,
                                      gravity, 1, s);
        if (st != SEEVR_OK) return st;
        SEEVR_CUDA(cudaStreamSynchronize(s));
        return seevr_physics_download_state(h, num_bodies, io->pos_out, io->quat_out, io->vel_out,
                                            io->omega_out);
    }
    st = ensure_single_scene(h, num_bodies, s);
    if (st != SEEVR_OK) return st;
    return run_frames(h, num_bodies, num_vertices, num_hull_verts, substeps, dt, gravity, 1, s, io);
}

seevr_status seevr_physics_read_counters(seevr_physics* h, uint32_t out[2]) {
    if (!h || !out) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle or out is NULL");
    SEEVR_CUDA(cudaSetDevice(h->device));
    SEEVR_CUDA(cudaMemcpyAsync(out, h->w.counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    SEEVR_CUDA(cudaStreamSynchronize(h->stream));
    return SEEVR_OK;
}

seevr_status seevr_physics_read_flags(seevr_physics* h, uint32_t* flags) {
    if (!h || !flags) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle or flags is NULL");
    SEEVR_CUDA(cudaSetDevice(h->device));
    bool overflow = false;
    seevr_status st = collect_flags(h, h->stream, &overflow);
    *flags = h->host_flags;
    h->host_flags = 0;
    return st;
}

seevr_status seevr_physics_get_tuning(seevr_physics* h, seevr_tuning* out) {
    if (!h || !out) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle or out is NULL");
    out->bundle_bodies = h->params.bundle_bodies ? h->params.bundle_bodies : 512u;
    out->narrow_blocks_per_sm = h->narrow_blocks_per_sm;
    out->broad_tile_rows = h->s.bp_tile_rows ? h->s.bp_tile_rows : kTileRows;
    out->scene_groups = h->scene_groups;
    out->giant_island_contacts = h->s.giant_min ? h->s.giant_min : kGiantContacts;
    return SEEVR_OK;
}

seevr_status seevr_physics_set_tuning(seevr_physics* h, const seevr_tuning* t) {
    if (!h || !t) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle or tuning is NULL");
    const uint32_t nbps = t->narrow_blocks_per_sm ? t->narrow_blocks_per_sm : kNarrowBlocksPerSm;
    const uint32_t rows = t->broad_tile_rows ? t->broad_tile_rows : kTileRows;
    if (nbps > kNarrowBlocksPerSm)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "narrow_blocks_per_sm above " +
                                                    std::to_string(kNarrowBlocksPerSm) +
                                                    " (the blocks that fit on an SM)");
    if (rows < 8 || rows > kTileBodies)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "broad_tile_rows outside [8, " +
                                                    std::to_string(kTileBodies) + "]");
    if (t->bundle_bodies > (1u << 24))
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "bundle_bodies above 2^24");
    if (t->scene_groups > kMaxGroups)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "scene_groups above " + std::to_string(kMaxGroups));
    SEEVR_CUDA(cudaSetDevice(h->device));
    h->narrow_blocks_per_sm = nbps;
    h->s.narrow_blocks = uint32_t(h->sm_count) * nbps;
    h->s.narrow_per_sm = nbps;
    h->s.bp_tile_rows = rows;
    h->params.bundle_bodies = t->bundle_bodies;
    h->scene_groups = t->scene_groups ? t->scene_groups : 1u;
    h->s.giant_min = t->giant_island_contacts;
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    if (h->scenes_set) {  // rebuild the bundles and the broadphase tiles
        const std::vector<uint32_t> off = h->scene_offsets_host;
        return seevr_physics_set_scenes(h, off.data(), uint32_t(off.size() - 1));
    }
    return SEEVR_OK;
}

seevr_status seevr_physics_set_wait_limit(seevr_physics* h, uint32_t polls) {
    if (!h) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle is NULL");
    h->s.wait_limit = polls;
    h->lb.wait_limit = polls;
    for (auto& g : h->groups)
        if (g.h) seevr_physics_set_wait_limit(g.h, polls);
    if (h->graph_exec) {  // kernel arguments are baked into a captured frame
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    return SEEVR_OK;
}

seevr_status seevr_physics_upload_state(seevr_physics* h, uint32_t nb, const float* pos,
                                        const float* quat, const float* vel, const float* omega) {
    if (!h) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle is NULL");
    if (nb > h->caps.max_bodies) return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_bodies exceeds caps");
    SEEVR_CUDA(cudaSetDevice(h->device));
    const cudaStream_t s = h->stream;
    if (pos) SEEVR_CUDA(cudaMemcpyAsync(h->w.pos, pos, size_t(nb) * 12, cudaMemcpyHostToDevice, s));
    if (quat) SEEVR_CUDA(cudaMemcpyAsync(h->w.quat, quat, size_t(nb) * 16, cudaMemcpyHostToDevice, s));
    if (vel) SEEVR_CUDA(cudaMemcpyAsync(h->w.vel, vel, size_t(nb) * 12, cudaMemcpyHostToDevice, s));
    if (omega) SEEVR_CUDA(cudaMemcpyAsync(h->w.omega, omega, size_t(nb) * 12, cudaMemcpyHostToDevice, s));
    SEEVR_CUDA(cudaStreamSynchronize(s));
    return SEEVR_OK;
}

seevr_status seevr_physics_download_state(seevr_physics* h, uint32_t nb, float* pos, float* quat,
                                          float* vel, float* omega) {
    if (!h) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle is NULL");
    if (nb > h->caps.max_bodies) return fail(SEEVR_ERR_INVALID_ARGUMENT, "num_bodies exceeds caps");
    SEEVR_CUDA(cudaSetDevice(h->device));
    const cudaStream_t s = h->stream;
    if (pos) SEEVR_CUDA(cudaMemcpyAsync(pos, h->w.pos, size_t(nb) * 12, cudaMemcpyDeviceToHost, s));
    if (quat) SEEVR_CUDA(cudaMemcpyAsync(quat, h->w.quat, size_t(nb) * 16, cudaMemcpyDeviceToHost, s));
    if (vel) SEEVR_CUDA(cudaMemcpyAsync(vel, h->w.vel, size_t(nb) * 12, cudaMemcpyDeviceToHost, s));
    if (omega) SEEVR_CUDA(cudaMemcpyAsync(omega, h->w.omega, size_t(nb) * 12, cudaMemcpyDeviceToHost, s));
    SEEVR_CUDA(cudaStreamSynchronize(s));
    return SEEVR_OK;
}

void seevr_physics_destroy(seevr_physics* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
}

uint64_t seevr_physics_kernel_launches(const seevr_physics* h) { return h ? h->launches : 0; }

seevr_status seevr_physics_read_lbvh(seevr_physics* h, uint32_t n, uint32_t* morton_sorted,
                                     uint32_t* order, float bounds[6]) {
    if (!h) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle is NULL");
    if (h->params.broadphase != SEEVR_BROADPHASE_LBVH)
        return fail(SEEVR_ERR_NOT_SUPPORTED, "handle does not use the LBVH broadphase");
    if (n > h->lb.cap) return fail(SEEVR_ERR_INVALID_ARGUMENT, "n exceeds the handle's bodies");
    SEEVR_CUDA(cudaSetDevice(h->device));
    const cudaStream_t s = h->stream;
    if (morton_sorted)
        SEEVR_CUDA(cudaMemcpyAsync(morton_sorted, h->lb.keys_sorted, size_t(n) * 4, cudaMemcpyDeviceToHost, s));
    if (order)
        SEEVR_CUDA(cudaMemcpyAsync(order, h->lb.vals_sorted, size_t(n) * 4, cudaMemcpyDeviceToHost, s));
    if (bounds) SEEVR_CUDA(cudaMemcpyAsync(bounds, h->lb.bounds_f, 24, cudaMemcpyDeviceToHost, s));
    SEEVR_CUDA(cudaStreamSynchronize(s));
    return SEEVR_OK;
}

seevr_status seevr_physics_adjoint_substep(seevr_physics* h, uint32_t num_bodies,
                                           uint32_t num_hull_verts, float dt,
                                           const float gravity[3],
                                           const seevr_adjoint_grads* grads) {
    if (!h || !gravity || !grads) return fail(SEEVR_ERR_INVALID_ARGUMENT, "handle, gravity or grads is NULL");
    if (!grads->pos || !grads->quat || !grads->vel || !grads->omega || !grads->friction)
        return fail(SEEVR_ERR_INVALID_ARGUMENT, "a gradient buffer is NULL");
    if (num_bodies == 0) return SEEVR_OK;
    if (h->params.narrowphase != SEEVR_NARROWPHASE_MPR)
        return fail(SEEVR_ERR_NOT_SUPPORTED, "the adjoint differentiates the MPR narrowphase only");
    seevr_status st = check_step_args(h, num_bodies, 0, num_hull_verts);
    if (st != SEEVR_OK) return st;
    SEEVR_CUDA(cudaSetDevice(h->device));
    const cudaStream_t s = h->stream;
    st = ensure_single_scene(h, num_bodies, s);
    if (st != SEEVR_OK) return st;
    AdjScratch& a = h->adj;
    if (!h->adj_ready) {
        const size_t nb = h->caps.max_bodies, nc = h->caps.max_contacts, np = h->caps.max_pairs;
        const size_t iters = h->params.pgs_iterations;
        st = dev_alloc(h, &a.tape, nc * iters * 13);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.ptape, np * 2);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.ctape, nc * 2);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.vw, nb * 6);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.gv, nb * 3);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.gw, nb * 3);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.gR, nb * 9);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.gp, nb * 3);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.gq, nb * 4);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.gc, nc * 12);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.glam, nc);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.lam, nc);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.par, nc * 12);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.last, nb);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.level, nc);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.order, nc);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.lvl, nc + size_t(h->caps.max_scenes) + 2);
        if (st == SEEVR_OK) st = dev_alloc(h, &a.fix, nc * 40);
        if (st != SEEVR_OK) return st;
        h->adj_ready = true;
    }
    World& w = h->w;
    w.nb = num_bodies;
    w.nv = 0;
    w.nhv = num_hull_verts;
    w.ns = h->num_scenes;
    w.nbundles = h->num_bundles;
    uint64_t n = 0;
    if (!h->b.ptr[SEEVR_B_HULL_RANGE])
        n += launch_hull_range_from_geom_data(static_cast<const float*>(h->b.ptr[SEEVR_B_GEOM_DATA]),
                                              h->s.derived_hull_range, num_bodies, s);
    // the substep's forward up to its contacts, in the order of issue_frame
    n += launch_body_stage(w, h->k, kGravity | kAabb, dt, gravity[0], gravity[1], gravity[2], s);
    n += h->params.broadphase == SEEVR_BROADPHASE_LBVH ? launch_broadphase_lbvh(w, h->s, h->lb, s)
                                                       : launch_broadphase_n2(w, h->s, h->max_scene_bodies, s);
    n += launch_lut_alias(w, h->s, s);
    n += launch_narrowphase_taped(w, h->k, h->s, a.ptape, a.ctape, s);
    n += launch_bundle_ranges(w, h->s, s);
    const Grads g{grads->pos, grads->quat, grads->vel, grads->omega, grads->friction};
    n += launch_adjoint(w, h->k, h->s, a, g, dt, s);
    h->launches += n;
    SEEVR_CUDA(cudaGetLastError());
    bool overflow = false;
    st = collect_flags(h, s, &overflow);
    if (st != SEEVR_OK) return st;
    if (overflow) return fail(SEEVR_ERR_CAPACITY, "pairs or contacts exceeded the caps");
    return SEEVR_OK;
}

const char* seevr_status_string(seevr_status s) {
    switch (s) {
        case SEEVR_OK: return "ok";
        case SEEVR_ERR_INVALID_ARGUMENT: return "invalid argument";
        case SEEVR_ERR_CAPACITY: return "capacity exceeded";
        case SEEVR_ERR_CUDA: return "CUDA error";
        case SEEVR_ERR_TIMEOUT: return "device wait timed out";
        case SEEVR_ERR_NO_DEVICE: return "no CUDA device";
        case SEEVR_ERR_OUT_OF_MEMORY: return "out of device memory";
        case SEEVR_ERR_NOT_SUPPORTED: return "not supported";
    }
    return "unknown status";
}

const char* seevr_last_error(void) { return g_last_error.c_str(); }
int seevr_abi_version(void) { return SEEVR_ABI_VERSION; }

}  // extern "C"
