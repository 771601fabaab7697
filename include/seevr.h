/*
 * seevr.h — C ABI of libseevr_cuda, the sm_100a rigid-body physics step.
 *
 * This library replaces the Vulkan dispatches of seeVR's physics step.  The
 * entry points below are what the Zig host (src/physics.zig, src/bvh.zig)
 * binds in place of its compute pipeline; each declaration names the
 * reference interface it replaces.
 *
 * Conventions
 *  - Every function returns seevr_status (0 = OK) and never aborts.  A
 *    human-readable message for the last failure on the calling thread is
 *    available from seevr_last_error().
 *  - Device buffers are owned by the caller (CUDA device pointers).  The
 *    library owns only its scratch space (pair/contact staging, scans, sort
 *    and solver work arrays) and frees it in seevr_physics_destroy().
 *  - Buffer layout is the SoA layout of src/data.zig:31-121 (packed float3,
 *    quaternions xyzw, geom_data 8 floats per geom with [0]=hull_start and
 *    [1]=hull_count stored as float).
 *  - One handle per host thread; handles are not reentrant.
 */
#ifndef SEEVR_H
#define SEEVR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEEVR_ABI_VERSION 2

typedef enum seevr_status {
    SEEVR_OK = 0,
    SEEVR_ERR_INVALID_ARGUMENT = 1, /* NULL/undersized buffer, bad count      */
    SEEVR_ERR_CAPACITY = 2,         /* pairs or contacts overflowed the caps;
                                       the step completed with the first
                                       max_pairs/max_contacts in canonical
                                       order, counters hold the true totals  */
    SEEVR_ERR_CUDA = 3,             /* a CUDA runtime call failed            */
    SEEVR_ERR_TIMEOUT = 4,          /* a bounded device-side wait gave up    */
    SEEVR_ERR_NO_DEVICE = 5,        /* no usable CUDA device                 */
    SEEVR_ERR_OUT_OF_MEMORY = 6,    /* scratch allocation failed             */
    SEEVR_ERR_NOT_SUPPORTED = 7     /* option combination not implemented    */
} seevr_status;

/* Binding indices: identical to the `binding=` numbers of physics.comp:16-57
 * and to the buffer order of Physics.init (physics.zig:37-68). */
enum seevr_binding {
    SEEVR_B_BODY_POS = 0,          /* f32[N*3]            rw */
    SEEVR_B_BODY_QUAT = 1,         /* f32[N*4] xyzw       rw */
    SEEVR_B_BODY_VEL = 2,          /* f32[N*3]            rw */
    SEEVR_B_BODY_OMEGA = 3,        /* f32[N*3]            rw */
    SEEVR_B_BODY_INV_MASS = 4,     /* f32[N]              r  */
    SEEVR_B_BODY_INV_INERTIA = 5,  /* f32[N*3] local diag r  */
    SEEVR_B_BODY_VERT_START = 6,   /* u32[N]              r  */
    SEEVR_B_BODY_VERT_COUNT = 7,   /* u32[N]              r  */
    SEEVR_B_GEOM_BODY_IDX = 8,     /* u32[G]              r  */
    SEEVR_B_GEOM_DATA = 9,         /* f32[G*8]            r  */
    SEEVR_B_GEOM_FRICTION = 10,    /* f32[G]              r  */
    SEEVR_B_GEOM_RESTITUTION = 11, /* f32[G]              r  */
    SEEVR_B_HULL_VERTS = 12,       /* f32[HV*3] local     r  */
    SEEVR_B_VERTICES = 13,         /* f32[V*3] world      w  */
    SEEVR_B_ORIG_VERTICES = 14,    /* f32[V*3] local      r  */
    SEEVR_B_CONTACT_POS = 15,      /* f32[MAXC*3]         w  */
    SEEVR_B_CONTACT_NORMAL = 16,   /* f32[MAXC*3]         w  */
    SEEVR_B_CONTACT_PEN = 17,      /* f32[MAXC]           w  */
    SEEVR_B_CONTACT_GEOM_A = 18,   /* u32[MAXC]           w  */
    SEEVR_B_CONTACT_GEOM_B = 19,   /* u32[MAXC]           w  */
    SEEVR_B_LAMBDA_N = 20,         /* f32[MAXC]           w  */
    SEEVR_B_COUNTERS = 21,         /* u32[4] [0]=pairs [1]=contacts         */
    SEEVR_B_BODY_AABB_MIN = 22,    /* f32[N*3]            w  */
    SEEVR_B_BODY_AABB_MAX = 23,    /* f32[N*3]            w  */
    SEEVR_B_COLLISION_PAIRS = 24,  /* u32[MAXP*2]         w  */
    SEEVR_B_AABB_TEMP_MIN = 25,    /* unused: the segmented AABB reduce needs
                                      no cascade temp (may be NULL)          */
    SEEVR_B_AABB_TEMP_MAX = 26,    /* unused (may be NULL)                   */
    SEEVR_B_AABB_TEMP_BODY = 27,   /* unused (may be NULL)                   */
    SEEVR_B_SUPPORT_OFFSET = 28,   /* u32[G] 0 = brute force                 */
    SEEVR_B_SUPPORT_LOOKUP = 29,   /* u32[1+192*k]                           */
    /* Extension (no reference binding): u32[G*2] (hull_start, hull_count)
     * per geom.  geom_data stores hull_start as a float (data.zig:468-473),
     * exact only below 2^24 hull vertices; when this pointer is non-NULL it
     * replaces geom_data[0..1].  May be NULL. */
    SEEVR_B_HULL_RANGE = 30,
    SEEVR_NUM_BINDINGS = 31
};

/* The 30 storage buffers of Physics.init (physics.zig:37-68) plus the
 * optional hull-range extension: device pointer and size in bytes,
 * index == binding. */
typedef struct seevr_bindings {
    void* ptr[SEEVR_NUM_BINDINGS];
    uint64_t bytes[SEEVR_NUM_BINDINGS];
} seevr_bindings;

/* Capacities.  The reference hard-codes them (data.zig:11-18 and
 * physics.comp:69-70); here they are per handle. */
typedef struct seevr_caps {
    uint32_t max_bodies;     /* MAX_BODIES (data.zig:13)            */
    uint32_t max_hull_verts; /* MAX_HULL_VERTS (data.zig:17)        */
    uint32_t max_vertices;   /* MAX_VERTICES (data.zig:11)          */
    uint32_t max_pairs;      /* MAX_COLLISION_PAIRS (data.zig:16)   */
    uint32_t max_contacts;   /* MAX_CONTACTS (data.zig:15)          */
    uint32_t max_scenes;     /* independent scenes per handle (>=1) */
} seevr_caps;

enum seevr_broadphase {
    SEEVR_BROADPHASE_N2 = 0,   /* all-pairs per scene (physics.comp:451-472) */
    SEEVR_BROADPHASE_LBVH = 1  /* Morton/radix/Karras tree (bvh.comp spec)   */
};

enum seevr_solver {
    SEEVR_SOLVER_SEQUENTIAL = 0, /* one thread per scene, contacts in order
                                    (physics.comp:500-583)                   */
    SEEVR_SOLVER_WAVEFRONT = 1,  /* same contact order, independent contacts
                                    run in parallel waves: bit-identical to
                                    SEQUENTIAL                               */
    SEEVR_SOLVER_COLORED = 2     /* graph-coloured Gauss-Seidel: a different
                                    contact order, assessed by drift        */
};

enum seevr_narrowphase {
    SEEVR_NARROWPHASE_MPR = 0,     /* Minkowski portal refinement, the
                                      reference's (physics.comp:171-399)      */
    SEEVR_NARROWPHASE_GJK_EPA = 1  /* GJK then the expanding polytope
                                      algorithm: no counterpart in the
                                      reference's code (its README names
                                      GJK + EPA); same contract: normal,
                                      depth and contact point per pair; not
                                      available to the adjoint               */
};

enum seevr_flags {
    SEEVR_FLAG_NO_SYNC = 1u << 0,      /* do not synchronize before return  */
    SEEVR_FLAG_CUDA_GRAPH = 1u << 1,   /* capture the frame once, replay    */
    SEEVR_FLAG_SKIP_RENDER_VERTS = 1u << 2 /* omit step 7 (update_verts)    */
};

/* Solver and collision constants.  Defaults equal the reference constants. */
typedef struct seevr_params {
    uint32_t pgs_iterations;   /* PGS_ITERATIONS = 4 (physics.comp:68)      */
    float baumgarte;           /* BAUMGARTE = 0.2 (physics.comp:66)         */
    float slop;                /* SLOP = 0.005 (physics.comp:67)            */
    float linear_damping;      /* 0.999 (physics.comp:422-424)              */
    float angular_damping;     /* 0.998 (physics.comp:425-427)              */
    float mpr_eps;             /* CCD_EPS = 1e-6 (physics.comp:174)         */
    float mpr_tolerance;       /* CCD_TOLERANCE = 1e-6 (physics.comp:175)   */
    uint32_t mpr_iterations;   /* CCD_ITERATIONS = 50 (physics.comp:176)    */
    uint32_t mpr_discover_trials; /* 15 (physics.comp:290)                  */
    uint32_t broadphase;       /* enum seevr_broadphase                     */
    uint32_t solver;           /* enum seevr_solver                         */
    uint32_t flags;            /* enum seevr_flags                          */
    uint32_t bundle_bodies;    /* solver work unit: consecutive scenes are
                                  solved together up to this many bodies
                                  (0 = 512); any value gives the same
                                  results, only speed changes              */
    uint32_t narrowphase;      /* enum seevr_narrowphase (ABI version 2)    */
} seevr_params;

/* Per-stage device timings in milliseconds, summed over the substeps of one
 * call.  Section names follow Physics.step_names (physics.zig:22-32). */
#define SEEVR_NUM_STAGES 9
typedef struct seevr_profile {
    float ms[SEEVR_NUM_STAGES];
    uint32_t calls;
} seevr_profile;
/* Stage order inside seevr_profile.ms: gravity, aabb, broad_phase,
 * narrow_phase, clear_impulse, pgs_solve, integrate, render_verts,
 * clear_counters — the order of physics.zig:22-32.  Stages fused into
 * another report 0: gravity and integrate run in the aabb stage's kernel,
 * the impulse clear in the narrowphase's contact write (it zeroes the
 * impulse of each contact of the substep; entries past the contact count
 * are left as they were, where the reference zeroes all MAX_CONTACTS), and
 * the counters are written by the scans. */

typedef struct seevr_physics seevr_physics;

/* Fill *p with the reference constants. */
void seevr_params_default(seevr_params* p);

/* Replaces Physics.init(vk, data, allocator, prof) (physics.zig:34-78):
 * binds the caller's buffers and allocates scratch sized by *caps.
 * The handle is bound to the CUDA device current on the calling thread. */
seevr_status seevr_physics_create(const seevr_bindings* bindings,
                                  const seevr_caps* caps,
                                  const seevr_params* params,
                                  seevr_physics** out);

/* Declare independent scenes: scene s owns bodies
 * [body_offset[s], body_offset[s+1]) (host array of num_scenes+1 entries,
 * body_offset[0] = 0, non-decreasing).  Bodies of different scenes never
 * collide.  Without this call a handle steps one scene.  No counterpart in
 * the reference (it steps one scene, physics.zig:80). */
seevr_status seevr_physics_set_scenes(seevr_physics* h,
                                      const uint32_t* body_offset,
                                      uint32_t num_scenes);

/* Replaces Physics.step(num_bodies, num_vertices, num_hull_verts, substeps,
 * dt, gravity, prof) (physics.zig:80-165): `substeps` substeps of
 * sub_dt = dt/substeps, each running gravity, AABB, broadphase, MPR
 * narrowphase, impulse clear, PGS and integration, then one render-vertex
 * update.  Synchronous unless SEEVR_FLAG_NO_SYNC; `prof` may be NULL (fast
 * mode, physics.zig:118-164) or receive per-stage device timings
 * (profiling mode, physics.zig:97-117).  With SEEVR_FLAG_CUDA_GRAPH and no
 * `prof`, the frame is replayed from its captured graph (as
 * seevr_physics_step_async does) before the wait: the same results, one
 * launch per frame. */
seevr_status seevr_physics_step(seevr_physics* h,
                                uint32_t num_bodies,
                                uint32_t num_vertices,
                                uint32_t num_hull_verts,
                                uint32_t substeps,
                                float dt,
                                const float gravity[3],
                                seevr_profile* prof);

/* Same as seevr_physics_step, ordered on `stream` (a cudaStream_t; NULL =
 * the handle's own stream, pass cudaStreamLegacy for the legacy default
 * stream) and never synchronizing; `frames` consecutive calls are issued
 * back to back.  With
 * SEEVR_FLAG_CUDA_GRAPH the frame is captured into a CUDA graph on first
 * use and replayed (re-captured when an argument changes).  No counterpart
 * in the reference. */
seevr_status seevr_physics_step_async(seevr_physics* h,
                                      uint32_t num_bodies,
                                      uint32_t num_vertices,
                                      uint32_t num_hull_verts,
                                      uint32_t substeps,
                                      float dt,
                                      const float gravity[3],
                                      uint32_t frames,
                                      void* stream);

/* Replaces Physics.readCounters (physics.zig:213-217): out[0] = pairs found,
 * out[1] = contacts found, in the last substep (true totals, may exceed the
 * caps). */
seevr_status seevr_physics_read_counters(seevr_physics* h, uint32_t out[2]);

/* Overflow and error flags accumulated since the last call (bit 0: pairs
 * overflowed, bit 1: contacts overflowed, bit 2: a device wait timed out,
 * bit 3: a scene exceeded the solver's per-scene limits and took the
 * global-memory path, bit 4: a bounds check failed (SEEVR_CHECK=1), bit 5:
 * in the coloured mode, islands of more than 4,096 contacts were solved by
 * the whole grid).  Cleared by the call. */
seevr_status seevr_physics_read_flags(seevr_physics* h, uint32_t* flags);

/* Launch shapes of the batched step (no counterpart in the reference, whose
 * work-group sizes are fixed in the shader).  None of them changes any
 * result, only speed; seevr_b200.tune.autotune times candidates on the
 * caller's workload and sets the fastest.
 *  - bundle_bodies: solver bundle size (as seevr_params.bundle_bodies;
 *    0 = 512), at most 2^24;
 *  - narrow_blocks_per_sm: blocks per SM of the persistent narrowphase grid,
 *    1 to 7 (0 = 7, the register budget's maximum);
 *  - broad_tile_rows: rows of a scene per all-pairs broadphase block, 8 to
 *    2,048 (0 = 64);
 *  - scene_groups: 1 to 8 (0 = 1).  With more than one, the scenes are split
 *    into that many contiguous ranges of about equal bodies, each stepped
 *    through the whole frame on its own stream (one branch of the captured
 *    frame graph), so that one range's solver, whose time is its largest
 *    scene's dependent chain, overlaps the other ranges' collision stages.
 *    Each range keeps its own pair and contact lists (the handle's
 *    capacities each); they are merged into the bound buffers in canonical
 *    order at the end of every frame, so pairs, contacts, impulses, state
 *    and counters are bit for bit those of one group.  Needs scenes set,
 *    the all-pairs broadphase, no bounds-check mode, and every geom's body
 *    inside its own scene (geom_body_idx is read when the groups are
 *    built).  Which contacts a step that overflowed a cap keeps may differ;
 *  - giant_island_contacts: in the coloured mode, islands of more contacts
 *    than this are coloured and swept by the whole GPU (one cooperative
 *    launch, a grid barrier between colours) instead of by one warp; 0 =
 *    4,096.  Their colouring differs from the one-warp greedy colouring
 *    (it is computed in parallel), so this setting changes the coloured
 *    mode's results, never the sequential and wavefront modes'.
 * get returns the values in use (defaults resolved).  set applies them to
 * the following steps: a handle with scenes set rebuilds its solver bundles,
 * broadphase tiles and scene groups (as seevr_physics_set_scenes does), and
 * a captured frame graph is recaptured at the next graph step. */
typedef struct seevr_tuning {
    uint32_t bundle_bodies;
    uint32_t narrow_blocks_per_sm;
    uint32_t broad_tile_rows;
    uint32_t scene_groups;
    uint32_t giant_island_contacts;
} seevr_tuning;
seevr_status seevr_physics_get_tuning(seevr_physics* h, seevr_tuning* out);
seevr_status seevr_physics_set_tuning(seevr_physics* h, const seevr_tuning* t);

/* No counterpart in the reference, whose waits cannot fail.  Every bounded
 * device-side wait of this handle (the decoupled look-back of its scans and
 * radix sorts) gives up after `polls` polls of a tile that has not yet
 * published, raises the timeout bit and lets the step finish; the step then
 * returns SEEVR_ERR_TIMEOUT (seevr_physics_step) or reports bit 2 in
 * seevr_physics_read_flags (async steps; the bit stays set, and the stages
 * that consume scan or sort results stay skipped, until it is read).  A step
 * that timed out has advanced only the body state (gravity, damping,
 * integration) and wrote nothing outside its buffers; its pairs and contacts
 * are unspecified.  The default, 4,194,304 polls, is reached only if the GPU
 * stops scheduling a tile.  Small values exist so that tests can exercise
 * the error path without hanging or faulting the GPU (0: give up at the
 * first poll of an unpublished tile).  A captured frame graph is recaptured
 * at the next graph step. */
seevr_status seevr_physics_set_wait_limit(seevr_physics* h, uint32_t polls);

/* Copy the mutable body state between host memory and the bound device
 * buffers (pos, quat, vel, omega of num_bodies bodies), ordered on the
 * handle's stream and synchronous.  Mirrors Data.upload (data.zig:599-611)
 * and Vulkan.readBuffer (vulkan.zig:317-328) for the state the step
 * changes; any pointer may be NULL to skip that array. */
seevr_status seevr_physics_upload_state(seevr_physics* h, uint32_t num_bodies,
                                        const float* pos, const float* quat,
                                        const float* vel, const float* omega);
seevr_status seevr_physics_download_state(seevr_physics* h, uint32_t num_bodies,
                                          float* pos, float* quat,
                                          float* vel, float* omega);

/* Host arrays of one frame's state for seevr_physics_step_io: `*_in` are
 * copied into the bound device buffers before the frame, the bound buffers
 * into `*_out` after it (pos, vel, omega: 3 floats per body; quat: 4).  Any
 * pointer may be NULL to skip that copy; an input and an output may be the
 * same array. */
typedef struct seevr_host_state {
    const float* pos_in;
    const float* quat_in;
    const float* vel_in;
    const float* omega_in;
    float* pos_out;
    float* quat_out;
    float* vel_out;
    float* omega_out;
} seevr_host_state;

/* One frame (seevr_physics_step_async with frames = 1) with its state copied
 * in from and out to host arrays: Data.upload, Physics.step and
 * Vulkan.readBuffer of the state (data.zig:599-611, physics.zig:80,
 * vulkan.zig:317-328) in one call.  When every non-NULL array is page-locked
 * (cudaHostAlloc / cudaHostRegister), the copies are ordered on `stream`
 * without waiting (the outputs are valid once the stream has reached this
 * point), and with scene groups each group's bodies are copied on the
 * group's stream, just before and just after that group's frame, so that
 * one group's copies overlap the other groups' kernels; with
 * SEEVR_FLAG_CUDA_GRAPH the copies are part of the captured frame graph
 * (re-captured when an array pointer changes).  With a pageable array the
 * call copies in, steps and copies out one after another and returns after
 * the last copy.  Results equal seevr_physics_upload_state, the step and
 * seevr_physics_download_state.  No counterpart in the reference. */
seevr_status seevr_physics_step_io(seevr_physics* h,
                                   uint32_t num_bodies,
                                   uint32_t num_vertices,
                                   uint32_t num_hull_verts,
                                   uint32_t substeps,
                                   float dt,
                                   const float gravity[3],
                                   const seevr_host_state* io,
                                   void* stream);

/* Replaces Physics.deinit (physics.zig:219-221). */
void seevr_physics_destroy(seevr_physics* h);

/* No counterpart in the reference.  One physics step of a single scene that
 * allocates no device memory, for callers that cannot call cudaMalloc: a
 * renderer that owns and pre-sizes all device memory (as seeVR's Data.init
 * does for the buffers it shares with Vulkan), a real-time loop that must
 * not allocate after start-up, or code that enqueues the step while a stream
 * is captured in global capture mode.  It runs the same kernels as
 * seevr_physics_step (same results, bit for bit) on scratch held in one
 * static device array of SEEVR_NOALLOC_SCRATCH_BYTES that every device which
 * loads the library keeps until the process exits.
 *  - Limits: num_bodies <= SEEVR_NOALLOC_MAX_BODIES, max_pairs <=
 *    SEEVR_NOALLOC_MAX_PAIRS, max_contacts <= SEEVR_NOALLOC_MAX_CONTACTS
 *    (the capacities of the caller's pair and contact buffers); larger
 *    values return SEEVR_ERR_INVALID_ARGUMENT with a message.
 *  - All-pairs broadphase, sequential or wavefront solver.
 *  - Ordered on `stream` (a cudaStream_t, NULL = default stream) on the
 *    current device; synchronous unless params->flags has NO_SYNC.  To
 *    enqueue the step while `stream` is being captured, set NO_SYNC: the
 *    synchronous mode reads the status word back and waits, which capture
 *    forbids.  With NO_SYNC no status is reported: capacity overflow and
 *    timeouts are not returned, and the next call clears the status word.
 *  - The first call on a device looks up the scratch array's device address
 *    (cudaGetSymbolAddress) and configures the solver and broadphase
 *    kernels; make that first call before any stream capture.
 *  - Every call shares the one array: calls whose GPU work may overlap
 *    (other streams or host threads on the same device) race and must be
 *    serialised by the caller.  Each call clears what must start at zero. */
#define SEEVR_NOALLOC_MAX_BODIES 4096u
#define SEEVR_NOALLOC_MAX_PAIRS 32768u
#define SEEVR_NOALLOC_MAX_CONTACTS 16384u
#define SEEVR_NOALLOC_SCRATCH_BYTES 5489920u
seevr_status seevr_physics_step_noalloc(const seevr_bindings* bindings,
                                        const seevr_params* params,
                                        uint32_t max_pairs, uint32_t max_contacts,
                                        uint32_t num_bodies, uint32_t num_vertices,
                                        uint32_t num_hull_verts, uint32_t substeps,
                                        float dt, const float gravity[3], void* stream);
/* The device status bits the calling thread's last synchronous
 * seevr_physics_step_noalloc read back (the bits of seevr_physics_read_flags;
 * bit 3: a bundle too large for shared memory was swept in global memory). */
uint32_t seevr_physics_noalloc_flags(void);

/* Number of kernels the library launched on this handle since creation. */
uint64_t seevr_physics_kernel_launches(const seevr_physics* h);

/* LBVH state of the last substep of a handle created with
 * SEEVR_BROADPHASE_LBVH: sorted 30-bit Morton codes of the body centroids
 * (AABB centres), the body index of each sorted slot, and the centroid
 * bounds (min xyz, max xyz).  Synchronous.  Mirrors the bvh_morton /
 * bvh_sort_indices / bvh_scene_bounds buffers of bvh.comp:14-18 for the
 * body tree. */
seevr_status seevr_physics_read_lbvh(seevr_physics* h, uint32_t n, uint32_t* morton_sorted,
                                     uint32_t* order, float bounds[6]);

/* ---- adjoint ---------------------------------------------------------------- */

/* Gradient buffers of seevr_physics_adjoint_substep (device, FP64, indexed
 * like the body and geom bindings).  The forward is FP32; the reverse pass
 * runs in FP64 because the PGS sweep's per-iteration sensitivities nearly
 * cancel. */
typedef struct seevr_adjoint_grads {
    double* pos;      /* f64[N*3]  in: dL/d state after the substep; out: before */
    double* quat;     /* f64[N*4] */
    double* vel;      /* f64[N*3] */
    double* omega;    /* f64[N*3] */
    double* friction; /* f64[G]    dL/d geom_friction, accumulated (+=)        */
} seevr_adjoint_grads;

/* No counterpart in the reference.  Reverse mode of one substep of
 * Physics.step (gravity, contacts, PGS, integration; physics.comp:418-604)
 * for gradient-based rollouts: the bound state buffers must hold the state
 * at the start of the substep (pos, quat, vel, omega, e.g. restored from a
 * checkpoint); the call recomputes the substep's contacts, recomputes the
 * PGS sweep in the reference order and back-propagates through it.  On
 * return `grads` holds dL/d(state before the substep) and dL/d friction has
 * been accumulated.  The state buffers' velocities are left at their
 * post-gravity values and the contact outputs are overwritten.  Contact
 * selection and the solver's clamps follow the branches the forward took.
 * Synchronous; allocates its work arrays on first use. */
seevr_status seevr_physics_adjoint_substep(seevr_physics* h, uint32_t num_bodies,
                                           uint32_t num_hull_verts, float dt,
                                           const float gravity[3],
                                           const seevr_adjoint_grads* grads);

/* ---- path tracer (raytracer.zig / raytrace.comp) ------------------------- */

/* Binding indices of Raytracer.init (raytracer.zig:31-58), identical to
 * raytrace.comp's `binding=` numbers (raytrace.comp:15-35).  Binding 0 is a
 * storage image in the reference; here it is a headless device buffer of
 * f32[width*height*4] RGBA, row-major.  Bindings 3-8 are the triangle BVH's
 * node min/max, left, right, count and primitive indices as seevr_bvh_build
 * writes them. */
enum seevr_rt_binding {
    SEEVR_RT_IMAGE = 0,          /* f32[W*H*4]   w */
    SEEVR_RT_VERTICES = 1,       /* f32[V*3]     r */
    SEEVR_RT_INDICES = 2,        /* u32[T*3]     r */
    SEEVR_RT_NODE_MIN = 3,       /* f32[(2T-1)*3] r */
    SEEVR_RT_NODE_MAX = 4,       /* f32[(2T-1)*3] r */
    SEEVR_RT_LEFT = 5,           /* u32[2T-1]    r */
    SEEVR_RT_RIGHT = 6,          /* u32[2T-1]    r */
    SEEVR_RT_COUNT = 7,          /* u32[2T-1]    r */
    SEEVR_RT_PRIM = 8,           /* u32[T]       r */
    SEEVR_RT_TRI_GEOM = 9,       /* u32[T]       r */
    SEEVR_RT_GEOM_MATERIAL = 10, /* u32[G]       r */
    SEEVR_RT_MAT_ALBEDO = 11,    /* f32[M*3]     r */
    SEEVR_RT_MAT_ROUGHNESS = 12, /* f32[M]       r */
    SEEVR_RT_MAT_METALLIC = 13,  /* f32[M]       r */
    SEEVR_RT_MAT_EMISSION = 14,  /* f32[M*3]     r */
    SEEVR_RT_MAT_IOR = 15,       /* f32[M] 0 = opaque r */
    SEEVR_RT_NUM_BINDINGS = 16
};

typedef struct seevr_rt_bindings {
    void* ptr[SEEVR_RT_NUM_BINDINGS];
} seevr_rt_bindings;

/* The push constants of raytrace.comp:5-13 (PC, raytracer.zig:6-15). */
typedef struct seevr_rt_params {
    float cam_pos[3], cam_dir[3], cam_right[3], cam_up[3];
    uint32_t width, height;
    uint32_t frame_num;      /* seeds the per-pixel RNG (raytrace.comp:182) */
    uint32_t num_triangles;
} seevr_rt_params;

/* Raytracer.render (raytracer.zig:159-200): one frame, 16 samples per pixel
 * and up to 16 bounces per sample, written (not accumulated) to binding 0.
 * Ordered on `stream` (a cudaStream_t, NULL = the default stream) and
 * synchronous, as render() waits for its queue.  Where GLSL leaves precision
 * to the implementation the library pins it: sin/cos of the hemisphere
 * angle by its own polynomials, pow(x, 5) as a product, and tan(30 degrees)
 * rounded from double (seevr_raytrace_fov_scale). */
seevr_status seevr_raytrace(const seevr_rt_bindings* b, const seevr_rt_params* p, void* stream);
float seevr_raytrace_fov_scale(void);

/* ---- triangle LBVH (bvh.zig / bvh.comp) ---------------------------------- */

/* Binding indices of BVH.init (bvh.zig:32-51), identical to bvh.comp's
 * `binding=` numbers (bvh.comp:11-28); temp (16) and temp_u (17) are one
 * buffer in the reference and may alias here too. */
enum seevr_bvh_binding {
    SEEVR_BVH_VERTICES = 0,      /* f32[V*3]                r */
    SEEVR_BVH_INDICES = 1,       /* u32[T*3]                r */
    SEEVR_BVH_CENTROIDS = 2,     /* f32[T*3]                w */
    SEEVR_BVH_MORTON = 3,        /* u32[T] sorted codes     w */
    SEEVR_BVH_MORTON_TEMP = 4,   /* u32[T] sort ping-pong   w */
    SEEVR_BVH_SORT_INDICES = 5,  /* u32[T] triangle of each sorted slot w */
    SEEVR_BVH_SORT_TEMP = 6,     /* u32[T] sort ping-pong   w */
    SEEVR_BVH_SCENE_BOUNDS = 7,  /* f32[6] centroid bounds  w */
    SEEVR_BVH_NODE_MIN = 8,      /* f32[(2T-1)*3]           w */
    SEEVR_BVH_NODE_MAX = 9,      /* f32[(2T-1)*3]           w */
    SEEVR_BVH_LEFT = 10,         /* u32[2T-1]               w */
    SEEVR_BVH_RIGHT = 11,        /* u32[2T-1]               w */
    SEEVR_BVH_COUNT = 12,        /* u32[2T-1] 1 on leaves   w */
    SEEVR_BVH_PARENT = 13,       /* u32[2T-1] root = 0xFFFFFFFF w */
    SEEVR_BVH_PRIM_INDICES = 14, /* u32[T]                  w */
    SEEVR_BVH_FLAGS = 15,        /* u32[T] refit flags      w */
    SEEVR_BVH_TEMP = 16,         /* unused (may be NULL)      */
    SEEVR_BVH_TEMP_U = 17,       /* u32 work area: 8 + 1024 + 1 + ceil(T/2048)*256 words */
    SEEVR_BVH_NUM_BINDINGS = 18
};

typedef struct seevr_bvh_bindings {
    void* ptr[SEEVR_BVH_NUM_BINDINGS];
    uint64_t bytes[SEEVR_BVH_NUM_BINDINGS];
} seevr_bvh_bindings;

typedef struct seevr_bvh seevr_bvh;

/* Replaces BVH.init (bvh.zig:29-61): binds the 18 buffers for up to
 * max_tris triangles.  Allocates no device memory. */
seevr_status seevr_bvh_create(const seevr_bvh_bindings* bindings, uint32_t max_tris,
                              seevr_bvh** out);
/* Replaces BVH.build(num_tris) (bvh.zig:63-172): centroids, 30-bit Morton
 * codes, stable radix sort, Karras hierarchy, leaf boxes and bottom-up refit
 * over the triangles `indices` makes of `vertices`.  Synchronous. */
seevr_status seevr_bvh_build(seevr_bvh* h, uint32_t num_tris);
/* Replaces BVH.deinit (bvh.zig:208-210). */
void seevr_bvh_destroy(seevr_bvh* h);

const char* seevr_status_string(seevr_status s);
const char* seevr_last_error(void);
int seevr_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SEEVR_H */
