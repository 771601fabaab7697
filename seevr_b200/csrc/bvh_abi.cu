// bvh_abi.cu — C ABI of the triangle LBVH build, replacing BVH.init /
// BVH.build / BVH.deinit (src/bvh.zig:29-210).  The 18 bindings are those of
// bvh.zig:32-51; the build writes the buffers bvh.comp writes: centroids,
// sorted Morton codes and sort indices (morton / sort_indices after an even
// number of passes, as bvh.comp:186-188 leaves them), scene bounds, node
// boxes, children, counts, parents and primitive indices.  The sort's
// ping-pong goes through morton_temp / sort_temp and its histograms and
// look-back state through temp_u, so the build allocates nothing.
#include <cuda_runtime.h>

#include <string>

#include "../../include/seevr.h"
#include "common.cuh"
#include "lbvh.cuh"

using namespace seevr;

struct seevr_bvh {
    int device = 0;
    seevr_bvh_bindings b{};
    uint32_t max_tris = 0;
    cudaStream_t stream = nullptr;
    uint64_t launches = 0;
};

namespace {

// words of temp_u the build needs: bounds (6, padded to 8) + digit
// histograms (4*256) + look-back status
uint64_t temp_words(uint32_t n) { return 8 + 4 * 256 + uint64_t(lbvh_status_words(n)); }

uint64_t bvh_need(int i, uint32_t n) {
    const uint64_t N = n, nodes = n ? 2ull * n - 1 : 0;
    switch (i) {
        case SEEVR_BVH_CENTROIDS: return 12 * N;
        case SEEVR_BVH_MORTON: case SEEVR_BVH_MORTON_TEMP: case SEEVR_BVH_SORT_INDICES:
        case SEEVR_BVH_SORT_TEMP: case SEEVR_BVH_PRIM_INDICES: case SEEVR_BVH_FLAGS:
            return 4 * N;
        case SEEVR_BVH_SCENE_BOUNDS: return 24;
        case SEEVR_BVH_NODE_MIN: case SEEVR_BVH_NODE_MAX: return 12 * nodes;
        case SEEVR_BVH_LEFT: case SEEVR_BVH_RIGHT: case SEEVR_BVH_COUNT: case SEEVR_BVH_PARENT:
            return 4 * nodes;
        case SEEVR_BVH_TEMP_U: return 4 * temp_words(n);
        default: return 0;  // vertices, indices: checked by the caller's counts
    }
}

}  // namespace

extern "C" {

seevr_status seevr_bvh_create(const seevr_bvh_bindings* b, uint32_t max_tris, seevr_bvh** out) {
    if (!out) return SEEVR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!b) {
        set_last_error("bindings is NULL");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return SEEVR_ERR_NO_DEVICE;
    }
    if (max_tris >= (1u << 30)) {
        set_last_error("max_tris must be below 2^30");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < SEEVR_BVH_NUM_BINDINGS; ++i) {
        const uint64_t need = bvh_need(i, max_tris);
        if ((i == SEEVR_BVH_VERTICES || i == SEEVR_BVH_INDICES || need) && !b->ptr[i]) {
            set_last_error("bvh binding " + std::to_string(i) + " is NULL");
            return SEEVR_ERR_INVALID_ARGUMENT;
        }
        if (need && b->bytes[i] < need) {
            set_last_error("bvh binding " + std::to_string(i) + " holds " +
                           std::to_string(b->bytes[i]) + " bytes, needs " + std::to_string(need));
            return SEEVR_ERR_INVALID_ARGUMENT;
        }
    }
    auto* h = new seevr_bvh();
    cudaGetDevice(&h->device);
    h->b = *b;
    h->max_tris = max_tris;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        set_last_error("cudaStreamCreate failed");
        return SEEVR_ERR_CUDA;
    }
    *out = h;
    return SEEVR_OK;
}

seevr_status seevr_bvh_build(seevr_bvh* h, uint32_t num_tris) {
    if (!h) {
        set_last_error("handle is NULL");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    if (num_tris == 0) return SEEVR_OK;  // bvh.zig:64
    if (num_tris > h->max_tris) {
        set_last_error("num_tris exceeds the handle's max_tris");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    cudaSetDevice(h->device);
    auto P = [&](int i) { return h->b.ptr[i]; };
    uint32_t* tu = static_cast<uint32_t*>(P(SEEVR_BVH_TEMP_U));
    LbvhScratch s{};
    s.cap = num_tris;
    s.bounds_o = tu;                 // [6]
    s.hist = tu + 8;                 // [4*256]
    s.status = tu + 8 + 4 * 256;     // look-back tiles
    s.keys_a = static_cast<uint32_t*>(P(SEEVR_BVH_MORTON));
    s.vals_a = static_cast<uint32_t*>(P(SEEVR_BVH_SORT_INDICES));
    s.keys_b = static_cast<uint32_t*>(P(SEEVR_BVH_MORTON_TEMP));
    s.vals_b = static_cast<uint32_t*>(P(SEEVR_BVH_SORT_TEMP));
    TriOut o{};
    o.centroids = static_cast<float*>(P(SEEVR_BVH_CENTROIDS));
    o.morton = static_cast<uint32_t*>(P(SEEVR_BVH_MORTON));
    o.sort_idx = static_cast<uint32_t*>(P(SEEVR_BVH_SORT_INDICES));
    o.scene_bounds = static_cast<float*>(P(SEEVR_BVH_SCENE_BOUNDS));
    o.node_min = static_cast<float*>(P(SEEVR_BVH_NODE_MIN));
    o.node_max = static_cast<float*>(P(SEEVR_BVH_NODE_MAX));
    o.left = static_cast<uint32_t*>(P(SEEVR_BVH_LEFT));
    o.right = static_cast<uint32_t*>(P(SEEVR_BVH_RIGHT));
    o.count = static_cast<uint32_t*>(P(SEEVR_BVH_COUNT));
    o.parent = static_cast<uint32_t*>(P(SEEVR_BVH_PARENT));
    o.prim_idx = static_cast<uint32_t*>(P(SEEVR_BVH_PRIM_INDICES));
    o.flags = static_cast<uint32_t*>(P(SEEVR_BVH_FLAGS));
    // a status word for bounded waits: the first padding word of temp_u
    uint32_t* err = tu + 6;
    cudaMemsetAsync(err, 0, sizeof(uint32_t), h->stream);
    h->launches += lbvh_build_triangles(static_cast<const float*>(P(SEEVR_BVH_VERTICES)),
                                        static_cast<const uint32_t*>(P(SEEVR_BVH_INDICES)),
                                        num_tris, s, o, err, h->stream);
    uint32_t flags = 0;
    cudaMemcpyAsync(&flags, err, sizeof flags, cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);  // BVH.build waits (bvh.zig:169)
    if (e != cudaSuccess) {
        set_last_error(std::string("bvh build: ") + cudaGetErrorString(e));
        return SEEVR_ERR_CUDA;
    }
    if (flags & kFlagTimeout) {
        set_last_error("a device-side wait of the bvh build gave up");
        return SEEVR_ERR_TIMEOUT;
    }
    return SEEVR_OK;
}

void seevr_bvh_destroy(seevr_bvh* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) {
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
    }
    delete h;
}

}  // extern "C"
