// lbvh.cuh — linear BVH scratch, views and launchers (lbvh.cu).
#pragma once
#include "common.cuh"

namespace seevr {

// Library-owned LBVH work arrays for up to `cap` primitives.
struct LbvhScratch {
    uint32_t cap;
    float* centroid;        // [cap*3]
    uint32_t* bounds_o;     // [6] order-preserving encoded min/max
    float* bounds_f;        // [6] decoded bounds of the last build
    uint32_t* keys_a;       // [cap] Morton codes, unsorted
    uint32_t* vals_a;       // [cap]
    uint32_t* keys_b;       // [cap] ping-pong
    uint32_t* vals_b;       // [cap]
    uint32_t* keys_sorted;  // [cap]
    uint32_t* vals_sorted;  // [cap] original index of each sorted slot
    uint32_t* hist;         // [4*256]
    uint32_t* status;       // [1 + tiles*256] look-back tile status
    uint32_t* left;         // [2*cap]
    uint32_t* right;        // [2*cap]
    uint32_t* parent;       // [2*cap]
    uint32_t* flags;        // [cap]
    float* node_min;        // [2*cap*3]
    float* node_max;        // [2*cap*3]
    // rows of static bodies (body broadphase): list, count and per-block
    // breadth-first work areas (kStaticBlocks x 3 x 2*cap)
    uint32_t* static_list;   // [cap]
    uint32_t* static_count;  // [1]
    uint32_t* bfs;
    // partners of each dynamic body's row found by the count traversal, in
    // ascending order, for rows of at most kRowCache partners
    uint32_t* row_cache;  // [cap * kRowCache]
    // the body tree packed for the traversals: node k at [2k, 2k+1]
    float4* packed;  // [2 * 2*cap]
    // polls of an unpublished sort tile before a look-back gives up
    uint32_t wait_limit = kSpinLimit;
};

// Blocks that traverse static bodies' rows.
constexpr uint32_t kStaticBlocks = 8;
// Partners per row the count traversal keeps for the write pass.
constexpr uint32_t kRowCache = 8;

struct LbvhView {
    const float* node_min;
    const float* node_max;
    const uint32_t* left;
    const uint32_t* right;
    const uint32_t* vals;
    // the same tree as one 32-byte record per node (lbvh.cu k_pack_nodes)
    const float4* packed;
};

// Output buffers of the triangle BVH, laid out as bvh.comp's bindings.
struct TriOut {
    float* centroids;      // binding 2
    uint32_t* morton;      // binding 3 (sorted codes)
    uint32_t* sort_idx;    // binding 5 (original triangle of each slot)
    float* scene_bounds;   // binding 7
    float* node_min;       // binding 8
    float* node_max;       // binding 9
    uint32_t* left;        // binding 10
    uint32_t* right;       // binding 11
    uint32_t* count;       // binding 12
    uint32_t* parent;      // binding 13
    uint32_t* prim_idx;    // binding 14
    uint32_t* flags;       // binding 15
};

inline uint32_t lbvh_status_words(uint32_t cap) { return 1 + ((cap + 2047) / 2048) * 256; }

int lbvh_sort(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_tmp,
              uint32_t* vals_tmp, uint32_t* keys_out, uint32_t* vals_out, uint32_t n,
              const LbvhScratch& s, uint32_t* err, cudaStream_t st);
int lbvh_build_bodies(const World& w, const LbvhScratch& s, uint32_t* err, cudaStream_t st);
int launch_broadphase_lbvh(const World& w, const Scratch& sc, const LbvhScratch& s,
                           cudaStream_t st);
int lbvh_build_triangles(const float* verts, const uint32_t* idx, uint32_t n, const LbvhScratch& s,
                         const TriOut& o, uint32_t* err, cudaStream_t st);

}  // namespace seevr
