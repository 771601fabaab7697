// check.cu — bounds-check mode (SEEVR_CHECK=1): device-side validation of
// every index the step's kernels dereference, in place of a memory checker.
//
// The step's kernels trust their inputs: a hull range past the hull vertex
// buffer, a support-lookup offset past the table, a geom mapped to a body of
// another scene, or a pair list corrupted by a bug would make them read or
// write outside the bound buffers.  With SEEVR_CHECK=1 in the environment
// when a handle is created, each step validates the caller's index arrays
// before the first substep and the pair and contact lists each substep
// produces before they are consumed.  A violation sets kFlagCheckFailed and
// records the first failing check and index in status[2..3]; every later
// kernel of the step sees the bit (halted / check_failed) and returns
// without touching memory, and the step returns SEEVR_ERR_INVALID_ARGUMENT
// naming the check.  The reference has no such mode (it has no sanitizer
// and discards Vulkan result codes, physics.zig:173, 194-200); its own
// hazards are the cascade race of physics.comp:758-763 against 801, which
// the one-pass AABB reduce here does not have, and the 16 KB per-thread
// array of physics.comp:505.
#include "common.cuh"

namespace seevr {

__device__ __forceinline__ void check_fail(uint32_t* status, uint32_t code, uint32_t index) {
    if (atomicCAS(&status[2], 0u, code) == 0u) status[3] = index;
    atomicOr(&status[0], kFlagCheckFailed);
}

// Inputs, per body b: its hull range within the hull vertices, its render
// vertices within the vertex buffers, its support lookup within the table
// with every entry inside its hull, and its geom's body in its own scene.
__global__ void k_check_inputs(World w, uint32_t lut_words) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= w.nb) return;
    const uint32_t hs = w.hull_range[size_t(b) * 2], hc = w.hull_range[size_t(b) * 2 + 1];
    if (hs > w.nhv || hc > w.nhv - hs) check_fail(w.status, kCheckHullRange, b);
    if (w.nv > 0) {
        const uint32_t vs = w.vert_start[b], vc = w.vert_count[b];
        if (vs > w.nv || vc > w.nv - vs) check_fail(w.status, kCheckRenderRange, b);
    }
    const uint32_t lk = w.sup_off[b];
    if (lk != 0u) {
        if (lk > lut_words || 192u > lut_words - lk) {
            check_fail(w.status, kCheckLookup, b);
        } else {
            for (uint32_t k = 0; k < 192u; ++k)
                if (w.sup_lut[lk + k] >= hc) {
                    check_fail(w.status, kCheckLookup, b);
                    break;
                }
        }
    }
    const uint32_t g = w.geom_body[b];
    if (g >= w.nb || w.body_scene[g] != w.body_scene[b])
        check_fail(w.status, kCheckGeomBody, b);
}

// Pairs of this substep: i < j < nb, both in one scene.
__global__ void k_check_pairs(World w) {
    if (halted(w.status)) return;
    const uint32_t np = min(w.counters[0], w.max_pairs);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        const uint32_t i = w.pairs[size_t(p) * 2], j = w.pairs[size_t(p) * 2 + 1];
        if (!(i < j && j < w.nb) || w.body_scene[i] != w.body_scene[j])
            check_fail(w.status, kCheckPairs, p);
    }
}

// Contacts of this substep: geoms below nb whose bodies share a solver
// bundle, in non-decreasing bundle order (each bundle's contacts one run).
__global__ void k_check_contacts(World w) {
    if (halted(w.status)) return;
    const uint32_t nc = min(w.counters[1], w.max_contacts);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const uint32_t ga = w.c_a[c], gb = w.c_b[c];
        bool ok = ga < w.nb && gb < w.nb;
        if (ok) {
            const uint32_t a = w.geom_body[ga], b = w.geom_body[gb];
            ok = a < w.nb && b < w.nb && w.body_bundle[a] == w.body_bundle[b];
            if (ok && c > 0 && w.c_a[c - 1] < w.nb && w.geom_body[w.c_a[c - 1]] < w.nb)
                ok = w.body_bundle[w.geom_body[w.c_a[c - 1]]] <= w.body_bundle[a];
        }
        if (!ok) check_fail(w.status, kCheckContacts, c);
    }
}

static uint32_t grid(uint32_t n) {
    const uint32_t b = (n + 255) / 256;
    return b == 0 ? 1 : (b > 148u * 8u ? 148u * 8u : b);
}

int launch_check_inputs(const World& w, uint32_t lut_words, cudaStream_t st) {
    if (w.nb == 0) return 0;
    k_check_inputs<<<(w.nb + 255) / 256, 256, 0, st>>>(w, lut_words);
    return 1;
}

int launch_check_pairs(const World& w, cudaStream_t st) {
    k_check_pairs<<<grid(w.max_pairs), 256, 0, st>>>(w);
    return 1;
}

int launch_check_contacts(const World& w, cudaStream_t st) {
    k_check_contacts<<<grid(w.max_contacts), 256, 0, st>>>(w);
    return 1;
}

const char* check_name(uint32_t code) {
    switch (code) {
        case kCheckHullRange: return "hull range of a body exceeds num_hull_verts";
        case kCheckRenderRange: return "render vertex range of a body exceeds num_vertices";
        case kCheckLookup: return "support lookup of a body outside the table or its hull";
        case kCheckGeomBody: return "geom_body_idx maps a geom outside its scene";
        case kCheckPairs: return "pair list entry out of order, range or scene";
        case kCheckContacts: return "contact list entry out of range or bundle order";
    }
    return "unknown check";
}

}  // namespace seevr
