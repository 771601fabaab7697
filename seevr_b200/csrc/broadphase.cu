// broadphase.cu — all-pairs AABB broadphase within each scene
// (step 2, physics.comp:451-472).
//
// Same predicate as the reference: rows i, columns j > i of the same scene,
// skip when both bodies have inv_mass <= 0, closed-interval overlap test.
// The reference appends with atomicAdd (nondeterministic order); here a
// count pass, an exclusive scan and a write pass emit pairs in canonical
// (i, j) lexicographic order.  Pairs beyond max_pairs are dropped while the
// total keeps counting, as in the reference (physics.comp:465-466).
//
// One warp per row: lanes test 32 consecutive columns at a time and the
// ballot/popc prefix gives each hit its slot in ascending-j order.  The
// count pass keeps each 32-column ballot word in a per-row mask array (when
// the library could size it for the largest scene), so the write pass reads
// the words back instead of re-testing, and stops at the row's count.
#include "common.cuh"

namespace seevr {

__device__ __forceinline__ bool overlap(f3 mna, f3 mxa, f3 mnb, f3 mxb) {
    return !(mxa.x < mnb.x || mxb.x < mna.x || mxa.y < mnb.y || mxb.y < mna.y ||
             mxa.z < mnb.z || mxb.z < mna.z);
}

template <bool kWrite>
__global__ void __launch_bounds__(256) k_broad_n2(World w, const uint32_t* __restrict__ row_off,
                                                  uint32_t* __restrict__ row_count,
                                                  uint32_t* __restrict__ mask, uint32_t stride) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= w.nb) return;
    uint32_t total = 0;
    if (kWrite) {
        total = row_count[i];
        if (total == 0) return;
    }
    const uint32_t end = w.scene_off[w.body_scene[i] + 1];
    uint32_t* mrow = mask ? mask + size_t(i) * stride : nullptr;
    f3 mna = mk(0.f, 0.f, 0.f), mxa = mna;
    bool static_i = false;
    if (!kWrite || !mrow) {
        mna = ld3(w.aabb_min, i);
        mxa = ld3(w.aabb_max, i);
        static_i = w.inv_mass[i] <= 0.0f;
    }
    uint32_t count = 0;
    const uint32_t base = kWrite ? row_off[i] : 0u;
    for (uint32_t j0 = i + 1, ch = 0; j0 < end; j0 += 32, ++ch) {
        const uint32_t j = j0 + lane;
        unsigned m;
        if (kWrite && mrow) {
            m = mrow[ch];
        } else {
            bool hit = false;
            if (j < end && !(static_i && w.inv_mass[j] <= 0.0f))
                hit = overlap(mna, mxa, ld3(w.aabb_min, j), ld3(w.aabb_max, j));
            m = __ballot_sync(0xFFFFFFFFu, hit);
            if (!kWrite && mrow && lane == 0) mrow[ch] = m;
        }
        if (kWrite && ((m >> lane) & 1u)) {
            const uint32_t slot = base + count + __popc(m & ((1u << lane) - 1u));
            if (slot < w.max_pairs) {
                w.pairs[size_t(slot) * 2] = i;
                w.pairs[size_t(slot) * 2 + 1] = j;
            }
        }
        count += __popc(m);
        if (kWrite && count >= total) break;
    }
    if (!kWrite && lane == 0) row_count[i] = count;
}

int launch_broadphase_n2(const World& w, const Scratch& s, cudaStream_t st) {
    if (w.nb == 0) return 0;
    const uint32_t threads = 256;
    const uint32_t blocks = uint32_t((uint64_t(w.nb) * 32 + threads - 1) / threads);
    k_broad_n2<false><<<blocks, threads, 0, st>>>(w, nullptr, s.row_count, s.bp_mask, s.bp_stride);
    launch_exclusive_scan(s.row_count, s.row_off, nullptr, w.nb, &w.counters[0], w.max_pairs,
                          kFlagPairOverflow, s, st);
    k_broad_n2<true><<<blocks, threads, 0, st>>>(w, s.row_off, s.row_count, s.bp_mask, s.bp_stride);
    return 3;
}

}  // namespace seevr
