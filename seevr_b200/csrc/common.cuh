// common.cuh — kernel-side view of the bound buffers, library scratch, and
// the launchers each translation unit exports to the step driver.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "vmath.cuh"

namespace seevr {

// Device status word bits (seevr_physics_read_flags).
enum : uint32_t {
    kFlagPairOverflow = 1u << 0,
    kFlagContactOverflow = 1u << 1,
    kFlagTimeout = 1u << 2,
    kFlagSolverGlobal = 1u << 3,
    kFlagCheckFailed = 1u << 4,  // bounds-check mode found a bad index (check.cu)
    kFlagGiantIslands = 1u << 5,  // islands were solved grid-wide (giant.cu)
};

// Checks of the bounds-check mode; the failing one is kept in status[2]
// and its body, pair or contact index in status[3].
enum : uint32_t {
    kCheckHullRange = 1,
    kCheckRenderRange = 2,
    kCheckLookup = 3,
    kCheckGeomBody = 4,
    kCheckPairs = 5,
    kCheckContacts = 6,
};

// Bounded spin for decoupled look-back: after this many polls of an
// unpublished tile a wait gives up, raises kFlagTimeout and proceeds, so no
// kernel can hang.  The default of Scratch::wait_limit (per handle,
// seevr_physics_set_wait_limit).
constexpr uint32_t kSpinLimit = 1u << 22;

constexpr uint32_t kNone = 0xFFFFFFFFu;

// The caller's buffers (physics.comp:16-57) plus derived read-only arrays.
struct World {
    float* pos;
    float* quat;
    float* vel;
    float* omega;
    const float* inv_mass;
    const float* inv_inertia;
    const uint32_t* vert_start;
    const uint32_t* vert_count;
    const uint32_t* geom_body;
    const float* friction;
    const float* restitution;
    const float* hull;
    float* verts;
    const float* orig;
    float* c_pos;
    float* c_normal;
    float* c_pen;
    uint32_t* c_a;
    uint32_t* c_b;
    float* lambda;
    uint32_t* counters;
    // library status word (Scratch::status): kernels that consume scan or
    // sort results read its timeout bit first (timed_out)
    uint32_t* status;
    float* aabb_min;
    float* aabb_max;
    uint32_t* pairs;
    const uint32_t* sup_off;
    const uint32_t* sup_lut;
    // per body, the offset of a lookup table equal in content to its own
    // (launch_lut_alias; NULL: sup_off)
    const uint32_t* lut_off;
    const uint32_t* hull_range;  // (start,count) per geom: binding 30 or derived
    const uint32_t* body_scene;  // body -> scene
    const uint32_t* scene_off;   // scene -> first body, [num_scenes+1]
    // Solver bundles: runs of whole consecutive scenes solved together by
    // one warp or block, bundle -> first body, [nbundles+1]
    const uint32_t* bundle_off;
    const uint32_t* body_bundle;  // body -> bundle
    uint32_t nbundles;
    uint32_t nb, nv, nhv, ns;
    uint32_t max_pairs, max_contacts;
};

// Solver / collision constants (seevr_params), as kernels see them.
struct Consts {
    float baumgarte, slop, lin_damp, ang_damp, eps, tol;
    uint32_t pgs_iterations, mpr_iterations, discover_trials;
    uint32_t narrowphase;  // 0: MPR, 1: GJK + EPA (seevr_params.narrowphase)
};

// Grid-wide coloured solve of giant islands (giant.cu); list == NULL: not
// allocated.  Indexed by contact position in island order (i) or body.
struct GiantScratch {
    uint32_t* list;    // [max_contacts] positions of the giant islands' contacts
    uint32_t* colour;  // [max_contacts] colour per position
    uint32_t* order;   // [max_contacts] positions grouped by colour
    uint64_t* used;    // [max_bodies] colours taken at each body (bit mask)
    uint64_t* prio;    // [max_bodies] highest priority of an uncoloured contact
    uint32_t* hist;    // [kGiantMaxColours] contacts per colour, then cursors
    uint32_t* first;   // [kGiantMaxColours + 1] first slot of each colour
    uint32_t* ctr;     // [kGiantCtrWords] barrier (words 0 and 32), counts (2-4)
};
constexpr uint32_t kGiantCtrWords = 64;
constexpr uint32_t kGiantMaxColours = 64 + 1024;
// Islands of more contacts than this are solved grid-wide in the coloured
// mode (launch_solver_giant).
constexpr uint32_t kGiantContacts = 4096;

// Island solver work arrays (islands.cu); parent == NULL: not allocated.
struct IslandScratch {
    uint32_t* parent;       // [max_bodies] union-find links
    uint32_t* keys_in;      // [max_contacts] island root per contact (or none)
    uint32_t* vals_in;      // [max_contacts] contact index
    uint32_t* keys_tmp;     // [max_contacts] sort ping-pong
    uint32_t* vals_tmp;     // [max_contacts]
    uint32_t* keys_out;     // [max_contacts] sorted roots
    uint32_t* perm;         // [max_contacts] contact of each sorted slot
    uint32_t* head;         // [max_contacts] 1 at an island's first slot
    uint32_t* idx;          // [max_contacts] exclusive scan of head
    uint32_t* start;        // [max_contacts + 1] first slot of each island
    uint32_t* count;        // [1] islands
    uint32_t* lvl;          // [2 * max_contacts + 2] level boundaries per island
    uint32_t* sort_hist;    // [4 * 256]
    uint32_t* sort_status;  // look-back words of the sort
    GiantScratch giant;
};

// Library-owned scratch (device).
struct Scratch {
    uint32_t* status;       // [4]: flags, scratch counters
    uint32_t* row_count;    // [max_bodies]   broadphase pairs per row
    uint32_t* row_off;      // [max_bodies]   exclusive scan of row_count
    unsigned long long* scan_tiles;  // look-back tile status (+1 tile ticket)
    uint32_t scan_tiles_cap;
    float4* pair_res0;      // [max_pairs] contact point xyz, depth
    float4* pair_res1;      // [max_pairs] normal xyz, found flag
    uint32_t* pair_flag;    // [max_pairs] 1 if the pair makes a contact
    uint32_t* pair_coff;    // [max_pairs] exclusive scan of pair_flag (before it:
                            // the narrowphase's pair order)
    uint32_t* pair_class;   // [2*kPairClasses] pairs per class and cursors
                            // (NULL: pairs taken in index order)
    uint32_t order_pairs;   // 1: pairs taken grouped by class (scene groups'
                            // handles), 0: in index order
    uint32_t sweep_warps;   // warps per solver bundle: 2 in scene groups'
                            // handles (64-wide passes), else 1
    uint32_t* lut_rep;      // [kLutHullMax] first body with a lookup per hull size
    uint32_t* lut_off;      // [max_bodies] lookup offset read by the narrowphase
    // solver, per contact
    float* s_ra;            // [max_contacts*3]
    float* s_rb;            // [max_contacts*3]
    float* s_bias;          // [max_contacts]
    float* s_kn;            // [max_contacts]
    float* s_mu;            // [max_contacts]
    uint32_t* s_ab;         // [max_contacts*2] scene-local body indices, kNone = skip
    uint32_t* s_level;      // [max_contacts]
    uint32_t* s_order;      // [max_contacts]
    uint32_t* s_lvl_start;  // [max_contacts + max_scenes + 1]
    float* s_n;             // [max_contacts*3] normals in solve order
    float* s_lam;           // [max_contacts] impulses of large bundles
    uint32_t* s_abp;        // [max_contacts*2] body pair in solve order
    float4* s_rec;          // [max_contacts*kRecWords] per-contact solver records
    uint32_t* bundle_c0;    // [max_scenes + 1] first contact of each bundle
    // solver, per body (global-memory path for scenes too large for smem)
    float* s_R;             // [max_bodies*9]
    uint32_t* s_last;       // [max_bodies]
    uint32_t* derived_hull_range;  // [max_bodies*2]
    // all-pairs broadphase: per row, the 32-column overlap words of the
    // count pass (NULL: the write pass re-tests)
    uint32_t* bp_mask;      // [rows * bp_stride]
    uint32_t bp_stride;     // words per row
    // all-pairs broadphase blocks: (scene, slice | slices << 16) per block
    // (NULL: every scene gets the slices of the largest)
    uint2* bp_tiles;
    uint32_t bp_ntiles;
    // polls of an unpublished tile before a look-back gives up (kSpinLimit)
    uint32_t wait_limit;
    // coloured mode: islands above this many contacts are solved grid-wide
    // (0: kGiantContacts)
    uint32_t giant_min;
    // launch shapes (seevr_physics_set_tuning; 0 = the built-in default)
    uint32_t narrow_blocks;  // persistent narrowphase grid, in blocks
    uint32_t narrow_per_sm;  // of which per SM (selects the register budget)
    uint32_t bp_tile_rows;   // all-pairs broadphase rows per block
    IslandScratch isl;
};

// True once a bounded wait of the running step gave up or a bounds check
// failed.  Every kernel that consumes a scan's offsets or a sort's order
// returns at once when it is set: offsets from a look-back that gave up are
// too small, and the lists they would index (pairs, contacts, bundle
// ranges, tree nodes) are then neither complete nor ordered.  A step that
// timed out therefore only advances the body state and stays within every
// buffer.  The bits stay set until the host reads and clears the status
// word.
__device__ __forceinline__ bool halted(const uint32_t* status) {
    return (*reinterpret_cast<const volatile uint32_t*>(status) &
            (kFlagTimeout | kFlagCheckFailed)) != 0u;
}
// True once a bounds check failed: then the per-body stages stop as well,
// since the inputs they index are not valid.
__device__ __forceinline__ bool check_failed(const uint32_t* status) {
    return (*reinterpret_cast<const volatile uint32_t*>(status) & kFlagCheckFailed) != 0u;
}

// ---- launchers (one translation unit each) ------------------------------
enum BodyStageFlags : uint32_t {
    kIntegrate = 1u << 0,
    kGravity = 1u << 1,
    kAabb = 1u << 2,
    kRenderVerts = 1u << 3,
};
// Every launcher returns the number of kernels it launched.
int launch_hull_range_from_geom_data(const float* geom_data, uint32_t* out, uint32_t nb,
                                     cudaStream_t st);
int launch_body_stage(const World& w, const Consts& k, uint32_t flags, float dt, float gx,
                      float gy, float gz, cudaStream_t st);
// Exclusive scan of n_in[0..n) where n = min(*n_dev, n_cap) if n_dev else
// n_cap.  Writes the grand total (unclamped input count semantics: the sum)
// to *total_out when non-NULL, and sets `overflow_bit` in status[0] when the
// total exceeds `total_cap`.
int launch_exclusive_scan(const uint32_t* in, uint32_t* out, const uint32_t* n_dev,
                          uint32_t n_cap, uint32_t* total_out, uint32_t total_cap,
                          uint32_t overflow_bit, const Scratch& s, cudaStream_t st);
int launch_broadphase_n2(const World& w, const Scratch& s, uint32_t max_scene_bodies,
                         cudaStream_t st);
cudaError_t init_broadphase();
// all-pairs broadphase on shared-memory tiles: scenes up to kTileBodies
// bodies, one block per kTileRows rows of a scene
constexpr uint32_t kTileBodies = 2048;
constexpr uint32_t kTileRows = 64;
// narrowphase: resident blocks per SM of the persistent grid (its register
// cap; measured best of 4 to 8)
constexpr uint32_t kNarrowBlocksPerSm = 7;
int launch_narrowphase(const World& w, const Consts& k, const Scratch& s, cudaStream_t st);
// The support lookups of bodies whose table equals, entry for entry, the
// table of the first body with the same hull size are read through that one
// table (s.lut_off): the same values, from a copy that stays in cache.
constexpr uint32_t kLutHullMax = 4096;
// narrowphase pair order: 4 classes by the two shapes' support paths
constexpr uint32_t kPairClasses = 4;
int launch_lut_alias(const World& w, const Scratch& s, cudaStream_t st);
__device__ __forceinline__ uint32_t lut_of(const World& w, uint32_t b) {
    return w.lut_off ? w.lut_off[b] : w.sup_off[b];
}
// Narrowphase that also tapes the supporting hull vertices of each contact's
// final portal (2 uint4 per pair / contact) for the adjoint.
int launch_narrowphase_taped(const World& w, const Consts& k, const Scratch& s, uint4* pair_tape,
                             uint4* contact_tape, cudaStream_t st);
cudaError_t init_solver();
// bundle_c0: the first contact of every solver bundle (one marking pass)
int launch_bundle_ranges(const World& w, const Scratch& s, cudaStream_t st);
// Set the calling thread's message returned by seevr_last_error().
void set_last_error(const char* msg);
inline void set_last_error(const std::string& msg) { set_last_error(msg.c_str()); }
// max_scene_bodies: the largest bundle; smem_bodies: bodies per bundle kept
// in shared memory by the warp solver (larger bundles solve in place)
int launch_solver(const World& w, const Consts& k, const Scratch& s, uint32_t mode,
                  float dt, uint32_t max_scene_bodies, uint32_t smem_bodies, cudaStream_t st);
// Island-parallel solve of the whole contact list (needs s.isl); mode 0
// sequential, 1 wavefront, 2 coloured.
int launch_solver_islands(const World& w, const Consts& k, const Scratch& s, uint32_t mode,
                          float dt, cudaStream_t st);
// Grid-wide coloured solve of the islands above kGiantContacts contacts (a
// cooperative launch); returns 0 without launching when not available.
int launch_solver_giant(const World& w, const Consts& k, const Scratch& s, float dt,
                        cudaStream_t st);
// Scenes above this many bodies are solved by islands (when allocated).
constexpr uint32_t kWarpMaxBodies = 1024;
constexpr uint32_t kRecWords = 10;  // float4 words of a warp-solver contact record

// One scene group's outputs, merged into the bound buffers at frame end
// (physics.cu): its counters and status word, its pair and contact lists in
// group-local body and geom indices, and its first body.
struct GroupOut {
    const uint32_t* counters;
    uint32_t* status;
    const uint32_t* pairs;
    const float* c_pos;
    const float* c_normal;
    const float* c_pen;
    const uint32_t* c_a;
    const uint32_t* c_b;
    const float* lambda;
    uint32_t b0;
};
constexpr uint32_t kMaxGroups = 8;
struct GroupTable {
    GroupOut g[kMaxGroups];
    uint32_t n;
};

// Bounds-check mode (check.cu): validation of the caller's index arrays
// (lut_words: entries of the support-lookup binding) and of each substep's
// pair and contact lists; check_name describes a status[2] code.
int launch_check_inputs(const World& w, uint32_t lut_words, cudaStream_t st);
int launch_check_pairs(const World& w, cudaStream_t st);
int launch_check_contacts(const World& w, cudaStream_t st);
const char* check_name(uint32_t code);

}  // namespace seevr
