// noalloc.cu — seevr_physics_step_noalloc: the single-scene physics step
// without any device allocation.
//
// seevr_physics_create allocates its scratch with cudaMalloc.  Some hosts
// cannot do that: a renderer that owns every byte of device memory and sizes
// it once at start-up (seeVR's Data.init creates all buffers up front and
// shares them with Vulkan), real-time loops that must not allocate after
// initialisation, and code that enqueues the step while a stream is being
// captured in global capture mode, where cudaMalloc is prohibited.  This
// entry point runs the same kernels on scratch carved from one file-scope
// device array, so the caller provides only the bound buffers and a stream.
//
// The array holds SEEVR_NOALLOC_SCRATCH_BYTES (5,489,920 bytes, about 5.5 MB)
// on every device that loads the library, until the process exits.  All calls share it: calls whose GPU
// work overlaps (different streams, or different host threads on one
// device) race on it and must be serialised by the caller.  Each call
// clears the parts that must start at zero (the status word, scan and
// solver state are reset by the kernels themselves).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/seevr.h"
#include "common.cuh"

namespace seevr {
namespace {

constexpr uint32_t kNaBodies = SEEVR_NOALLOC_MAX_BODIES;
constexpr uint32_t kNaPairs = SEEVR_NOALLOC_MAX_PAIRS;
constexpr uint32_t kNaContacts = SEEVR_NOALLOC_MAX_CONTACTS;
constexpr uint32_t kNaScanTiles = (kNaPairs > kNaBodies ? kNaPairs : kNaBodies) / 2048 + 2;

// Byte layout of the scratch array (each region 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffStatus = 0;
constexpr size_t kOffRowCount = align256(kOffStatus + 16);
constexpr size_t kOffRowOff = align256(kOffRowCount + 4ull * kNaBodies);
constexpr size_t kOffScanTiles = align256(kOffRowOff + 4ull * kNaBodies);
constexpr size_t kOffRes0 = align256(kOffScanTiles + 8ull * kNaScanTiles);
constexpr size_t kOffRes1 = align256(kOffRes0 + 16ull * kNaPairs);
constexpr size_t kOffFlag = align256(kOffRes1 + 16ull * kNaPairs);
constexpr size_t kOffCoff = align256(kOffFlag + 4ull * kNaPairs);
constexpr size_t kOffRa = align256(kOffCoff + 4ull * kNaPairs);
constexpr size_t kOffRb = align256(kOffRa + 12ull * kNaContacts);
constexpr size_t kOffBias = align256(kOffRb + 12ull * kNaContacts);
constexpr size_t kOffKn = align256(kOffBias + 4ull * kNaContacts);
constexpr size_t kOffMu = align256(kOffKn + 4ull * kNaContacts);
constexpr size_t kOffAb = align256(kOffMu + 4ull * kNaContacts);
constexpr size_t kOffLevel = align256(kOffAb + 8ull * kNaContacts);
constexpr size_t kOffOrder = align256(kOffLevel + 4ull * kNaContacts);
constexpr size_t kOffLvlStart = align256(kOffOrder + 4ull * kNaContacts);
constexpr size_t kOffR = align256(kOffLvlStart + 4ull * (kNaContacts + 2));
constexpr size_t kOffLast = align256(kOffR + 36ull * kNaBodies);
constexpr size_t kOffHullRange = align256(kOffLast + 4ull * kNaBodies);
constexpr size_t kOffBodyScene = align256(kOffHullRange + 8ull * kNaBodies);
constexpr size_t kOffSceneOff = align256(kOffBodyScene + 4ull * kNaBodies);
constexpr size_t kOffN = align256(kOffSceneOff + 8);
constexpr size_t kOffLam = align256(kOffN + 12ull * kNaContacts);
constexpr size_t kOffAbp = align256(kOffLam + 4ull * kNaContacts);
constexpr size_t kOffBundleC0 = align256(kOffAbp + 8ull * kNaContacts);
constexpr size_t kOffRec = align256(kOffBundleC0 + 16);
constexpr size_t kNaBytes = align256(kOffRec + 16ull * kRecWords * kNaContacts);
static_assert(kNaBytes == SEEVR_NOALLOC_SCRATCH_BYTES, "header constant out of date");

// The scratch itself.  In host code this name is a host-side stand-in, not
// a device address: only the pointer from cudaGetSymbolAddress may be
// handed to kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
unsigned char* g_dev_ptr[kMaxDevices] = {};
cudaError_t g_setup_err[kMaxDevices] = {};
uint32_t g_narrow_blocks[kMaxDevices] = {};
// the status bits the calling thread's last synchronous call read back
thread_local uint32_t t_last_flags = 0;

// Once per device, with that device current: the device address of the
// scratch array, the solver's shared-memory opt-in and the persistent
// narrowphase grid for this device's SM count (as seevr_physics_create).
void setup_device(int dev) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e == cudaSuccess) e = init_solver();
    if (e == cudaSuccess) e = init_broadphase();
    int sms = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g_narrow_blocks[dev] = uint32_t(sms > 0 ? sms : 1) * kNarrowBlocksPerSm;
    g_setup_err[dev] = e;
    g_dev_ptr[dev] = e == cudaSuccess ? static_cast<unsigned char*>(p) : nullptr;
}

__global__ void k_noalloc_one_scene(uint32_t* body_scene, uint32_t* scene_off, uint32_t nb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) body_scene[i] = 0;
    if (i == 0) {
        scene_off[0] = 0;
        scene_off[1] = nb;
    }
}

uint64_t need_bytes(int i, uint32_t nb, uint32_t nhv, uint32_t np, uint32_t nc) {
    switch (i) {
        case SEEVR_B_BODY_POS: case SEEVR_B_BODY_VEL: case SEEVR_B_BODY_OMEGA:
        case SEEVR_B_BODY_INV_INERTIA: case SEEVR_B_BODY_AABB_MIN: case SEEVR_B_BODY_AABB_MAX:
            return 12ull * nb;
        case SEEVR_B_BODY_QUAT: return 16ull * nb;
        case SEEVR_B_BODY_INV_MASS: case SEEVR_B_BODY_VERT_START: case SEEVR_B_BODY_VERT_COUNT:
        case SEEVR_B_GEOM_BODY_IDX: case SEEVR_B_GEOM_FRICTION: case SEEVR_B_GEOM_RESTITUTION:
        case SEEVR_B_SUPPORT_OFFSET:
            return 4ull * nb;
        case SEEVR_B_GEOM_DATA: return 32ull * nb;
        case SEEVR_B_HULL_VERTS: return 12ull * nhv;
        case SEEVR_B_CONTACT_POS: case SEEVR_B_CONTACT_NORMAL: return 12ull * nc;
        case SEEVR_B_CONTACT_PEN: case SEEVR_B_CONTACT_GEOM_A: case SEEVR_B_CONTACT_GEOM_B:
        case SEEVR_B_LAMBDA_N:
            return 4ull * nc;
        case SEEVR_B_COUNTERS: return 8;
        case SEEVR_B_COLLISION_PAIRS: return 8ull * np;
        case SEEVR_B_SUPPORT_LOOKUP: return 4;
        default: return 0;
    }
}

// the message is reported by seevr_last_error(), as for every entry point
seevr_status na_fail(seevr_status s, const std::string& m) {
    set_last_error(m);
    return s;
}

}  // namespace
}  // namespace seevr

using namespace seevr;

extern "C" seevr_status seevr_physics_step_noalloc(
    const seevr_bindings* b, const seevr_params* params, uint32_t max_pairs, uint32_t max_contacts,
    uint32_t num_bodies, uint32_t num_vertices, uint32_t num_hull_verts, uint32_t substeps,
    float dt, const float gravity[3], void* stream) {
    if (!b || !gravity) return na_fail(SEEVR_ERR_INVALID_ARGUMENT, "bindings or gravity is NULL");
    if (num_bodies > kNaBodies || max_pairs > kNaPairs || max_contacts > kNaContacts)
        return na_fail(SEEVR_ERR_INVALID_ARGUMENT,
                       "seevr_physics_step_noalloc: at most " + std::to_string(kNaBodies) +
                           " bodies, " + std::to_string(kNaPairs) + " pairs and " +
                           std::to_string(kNaContacts) + " contacts (got " +
                           std::to_string(num_bodies) + ", " + std::to_string(max_pairs) + ", " +
                           std::to_string(max_contacts) + ")");
    seevr_params p;
    seevr_params_default(&p);
    if (params) p = *params;
    if (p.broadphase != SEEVR_BROADPHASE_N2 || p.solver > SEEVR_SOLVER_WAVEFRONT)
        return na_fail(SEEVR_ERR_NOT_SUPPORTED,
                       "seevr_physics_step_noalloc: all-pairs broadphase with the sequential or "
                       "wavefront solver only");
    for (int i = 0; i < SEEVR_NUM_BINDINGS; ++i) {
        const uint64_t need = need_bytes(i, num_bodies, num_hull_verts, max_pairs, max_contacts);
        if (need && (!b->ptr[i] || b->bytes[i] < need))
            return na_fail(SEEVR_ERR_INVALID_ARGUMENT,
                           "binding " + std::to_string(i) + " is NULL or smaller than " +
                               std::to_string(need) + " bytes");
    }
    const bool render = num_vertices > 0 && !(p.flags & SEEVR_FLAG_SKIP_RENDER_VERTS);
    if (render && (!b->ptr[SEEVR_B_VERTICES] || !b->ptr[SEEVR_B_ORIG_VERTICES] ||
                   b->bytes[SEEVR_B_VERTICES] < 12ull * num_vertices ||
                   b->bytes[SEEVR_B_ORIG_VERTICES] < 12ull * num_vertices))
        return na_fail(SEEVR_ERR_INVALID_ARGUMENT, "render vertex bindings 13/14 missing or short");
    if (num_bodies == 0 || substeps == 0) return SEEVR_OK;  // physics.zig:81

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return na_fail(SEEVR_ERR_NO_DEVICE, "no usable current CUDA device");
    }
    std::call_once(g_once[dev], setup_device, dev);
    if (g_setup_err[dev] != cudaSuccess)
        return na_fail(SEEVR_ERR_CUDA, std::string("cudaGetSymbolAddress of the step scratch: ") +
                                           cudaGetErrorString(g_setup_err[dev]));
    unsigned char* base = g_dev_ptr[dev];
    auto at = [&](size_t off) { return base + off; };

    Scratch s{};
    s.status = reinterpret_cast<uint32_t*>(at(kOffStatus));
    s.row_count = reinterpret_cast<uint32_t*>(at(kOffRowCount));
    s.row_off = reinterpret_cast<uint32_t*>(at(kOffRowOff));
    s.scan_tiles = reinterpret_cast<unsigned long long*>(at(kOffScanTiles));
    s.scan_tiles_cap = kNaScanTiles;
    s.wait_limit = kSpinLimit;
    s.narrow_blocks = g_narrow_blocks[dev];
    s.narrow_per_sm = kNarrowBlocksPerSm;
    s.pair_res0 = reinterpret_cast<float4*>(at(kOffRes0));
    s.pair_res1 = reinterpret_cast<float4*>(at(kOffRes1));
    s.pair_flag = reinterpret_cast<uint32_t*>(at(kOffFlag));
    s.pair_coff = reinterpret_cast<uint32_t*>(at(kOffCoff));
    s.s_ra = reinterpret_cast<float*>(at(kOffRa));
    s.s_rb = reinterpret_cast<float*>(at(kOffRb));
    s.s_bias = reinterpret_cast<float*>(at(kOffBias));
    s.s_kn = reinterpret_cast<float*>(at(kOffKn));
    s.s_mu = reinterpret_cast<float*>(at(kOffMu));
    s.s_ab = reinterpret_cast<uint32_t*>(at(kOffAb));
    s.s_level = reinterpret_cast<uint32_t*>(at(kOffLevel));
    s.s_order = reinterpret_cast<uint32_t*>(at(kOffOrder));
    s.s_lvl_start = reinterpret_cast<uint32_t*>(at(kOffLvlStart));
    s.s_R = reinterpret_cast<float*>(at(kOffR));
    s.s_last = reinterpret_cast<uint32_t*>(at(kOffLast));
    s.derived_hull_range = reinterpret_cast<uint32_t*>(at(kOffHullRange));
    s.s_n = reinterpret_cast<float*>(at(kOffN));
    s.s_lam = reinterpret_cast<float*>(at(kOffLam));
    s.s_abp = reinterpret_cast<uint32_t*>(at(kOffAbp));
    s.bundle_c0 = reinterpret_cast<uint32_t*>(at(kOffBundleC0));
    s.s_rec = reinterpret_cast<float4*>(at(kOffRec));
    uint32_t* body_scene = reinterpret_cast<uint32_t*>(at(kOffBodyScene));
    uint32_t* scene_off = reinterpret_cast<uint32_t*>(at(kOffSceneOff));

    World w{};
    auto P = [&](int i) { return b->ptr[i]; };
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
    w.status = s.status;
    w.aabb_min = static_cast<float*>(P(SEEVR_B_BODY_AABB_MIN));
    w.aabb_max = static_cast<float*>(P(SEEVR_B_BODY_AABB_MAX));
    w.pairs = static_cast<uint32_t*>(P(SEEVR_B_COLLISION_PAIRS));
    w.sup_off = static_cast<const uint32_t*>(P(SEEVR_B_SUPPORT_OFFSET));
    w.sup_lut = static_cast<const uint32_t*>(P(SEEVR_B_SUPPORT_LOOKUP));
    const bool ext_range = P(SEEVR_B_HULL_RANGE) != nullptr &&
                           b->bytes[SEEVR_B_HULL_RANGE] >= 8ull * num_bodies;
    w.hull_range = ext_range ? static_cast<const uint32_t*>(P(SEEVR_B_HULL_RANGE))
                             : s.derived_hull_range;
    w.body_scene = body_scene;
    w.scene_off = scene_off;
    w.bundle_off = scene_off;  // one scene, one solver bundle
    w.body_bundle = body_scene;
    w.nbundles = 1;
    w.nb = num_bodies;
    w.nv = render ? num_vertices : 0;
    w.nhv = num_hull_verts;
    w.ns = 1;
    w.max_pairs = max_pairs;
    w.max_contacts = max_contacts;
    Consts k{};
    k.baumgarte = p.baumgarte;
    k.slop = p.slop;
    k.lin_damp = p.linear_damping;
    k.ang_damp = p.angular_damping;
    k.eps = p.mpr_eps;
    k.tol = p.mpr_tolerance;
    k.pgs_iterations = p.pgs_iterations;
    k.mpr_iterations = p.mpr_iterations;
    k.discover_trials = p.mpr_discover_trials;
    k.narrowphase = p.narrowphase <= SEEVR_NARROWPHASE_GJK_EPA ? p.narrowphase : 0u;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // state the kernels expect to start from: a clear status word, the one
    // scene's body map and (without binding 30) the hull ranges
    cudaMemsetAsync(s.status, 0, 16, st);
    k_noalloc_one_scene<<<(num_bodies + 255) / 256, 256, 0, st>>>(body_scene, scene_off, num_bodies);
    if (!ext_range)
        launch_hull_range_from_geom_data(static_cast<const float*>(P(SEEVR_B_GEOM_DATA)),
                                         s.derived_hull_range, num_bodies, st);
    const float sub_dt = dt / float(substeps);
    const uint32_t mode = p.solver;
    for (uint32_t sub = 0; sub < substeps; ++sub) {
        launch_body_stage(w, k, (sub > 0 ? kIntegrate : 0u) | kGravity | kAabb, sub_dt, gravity[0],
                          gravity[1], gravity[2], st);
        launch_broadphase_n2(w, s, num_bodies, st);
        launch_narrowphase(w, k, s, st);  // zeroes the contacts' impulses (step 4)
        launch_solver(w, k, s, mode, sub_dt, num_bodies, num_bodies, st);
    }
    launch_body_stage(w, k, kIntegrate | (render ? kRenderVerts : 0u), sub_dt, gravity[0],
                      gravity[1], gravity[2], st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(SEEVR_ERR_CUDA, cudaGetErrorString(e));
    if (p.flags & SEEVR_FLAG_NO_SYNC) return SEEVR_OK;
    uint32_t flags = 0;
    e = cudaMemcpyAsync(&flags, s.status, sizeof flags, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(SEEVR_ERR_CUDA, cudaGetErrorString(e));
    t_last_flags = flags;
    if (flags & kFlagTimeout) return na_fail(SEEVR_ERR_TIMEOUT, "a device-side wait gave up");
    if (flags & (kFlagPairOverflow | kFlagContactOverflow))
        return na_fail(SEEVR_ERR_CAPACITY, "pairs or contacts exceeded max_pairs/max_contacts");
    return SEEVR_OK;
}

// The status bits of the calling thread's last synchronous no-allocation
// step (bit 3: the solver swept in global memory; the others as
// seevr_physics_read_flags).
extern "C" uint32_t seevr_physics_noalloc_flags(void) { return t_last_flags; }
