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
// Rows are processed by warps: lanes test 32 consecutive columns at a time
// and the ballot/popc prefix gives each hit its slot in ascending-j order.
// The count pass keeps each 32-column ballot word in a per-row mask array
// (when the library could size it for the largest scene), so the write pass
// reads the words back instead of re-testing.
//
// Scenes of at most kTileBodies bodies (k_broad_tile): each of a scene's
// blocks (one per kTileRows rows, or the tuned row count) stages the
// scene's AABBs and static flags in shared memory, so a column test reads
// shared memory only.  The count
// pass deals groups of kRowGroup consecutive rows to the warps of the
// scene's blocks in turn (row work shrinks with the row index); a warp reads
// 32 columns and tests them against every row of its group.  Its overlap
// words are column-aligned (word c of a row: scene columns 32c .. 32c+31).
// The write pass loads a row's words with one coalesced load and places the
// hits with a warp prefix sum over the words' population counts.  Larger
// scenes use one warp per row reading the AABBs from global memory
// (k_broad_n2).
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
    if (kWrite && halted(w.status)) return;  // row offsets from a scan that gave up
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

constexpr uint32_t kTileThreads = 256, kTileWarps = kTileThreads / 32;
constexpr uint32_t kRowGroup = 4;  // rows a warp tests against one column read

template <bool kWrite>
__global__ void __launch_bounds__(kTileThreads)
    k_broad_tile(World w, const uint2* __restrict__ tiles, uint32_t uniform_slices,
                 const uint32_t* __restrict__ row_off, uint32_t* __restrict__ row_count,
                 uint32_t* __restrict__ mask, uint32_t stride) {
    extern __shared__ float sm[];
    if (kWrite && halted(w.status)) return;  // row offsets from a scan that gave up
    uint32_t scene, slice, slices;
    if (tiles) {
        const uint2 t = tiles[blockIdx.x];
        scene = t.x;
        slice = t.y & 0xFFFFu;
        slices = t.y >> 16;
    } else {
        scene = blockIdx.x / uniform_slices;
        slice = blockIdx.x % uniform_slices;
        slices = uniform_slices;
    }
    const uint32_t s0 = w.scene_off[scene], s1 = w.scene_off[scene + 1];
    const uint32_t n = s1 - s0;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const bool test = !kWrite || !mask;  // this pass evaluates the overlap tests
    float* mn = sm;
    float* mx = sm + 3 * n;
    float* stat = sm + 6 * n;  // 1: inv_mass <= 0
    if (test) {
        for (uint32_t t = threadIdx.x; t < 3 * n; t += kTileThreads) {
            mn[t] = w.aabb_min[size_t(s0) * 3 + t];
            mx[t] = w.aabb_max[size_t(s0) * 3 + t];
        }
        for (uint32_t t = threadIdx.x; t < n; t += kTileThreads)
            stat[t] = w.inv_mass[s0 + t] <= 0.0f ? 1.0f : 0.0f;
        __syncthreads();
    }
    const uint32_t nwords = (n + 31) / 32;  // column words of the scene
    if (!kWrite) {
        // kRowGroup consecutive rows per warp step: a column's AABB is read
        // once and tested against every row of the group
        for (uint32_t g = slice * kTileWarps + wid; g * kRowGroup < n; g += slices * kTileWarps) {
            const uint32_t r0 = g * kRowGroup;
            f3 rmn[kRowGroup], rmx[kRowGroup];
            bool rst[kRowGroup];
            uint32_t cnt[kRowGroup];
#pragma unroll
            for (uint32_t q = 0; q < kRowGroup; ++q) {
                const uint32_t r = min(r0 + q, n - 1);
                rmn[q] = ld3(mn, r);
                rmx[q] = ld3(mx, r);
                rst[q] = stat[r] != 0.0f;
                cnt[q] = 0;
            }
            for (uint32_t c = (r0 + 1) / 32; c < nwords; ++c) {
                const uint32_t j = 32 * c + lane;
                const uint32_t jj = j < n ? j : n - 1;
                const f3 cmn = ld3(mn, jj), cmx = ld3(mx, jj);
                const bool cst = stat[jj] != 0.0f;
                unsigned mine = 0;
#pragma unroll
                for (uint32_t q = 0; q < kRowGroup; ++q) {
                    const bool hit = j < n && j > r0 + q && !(rst[q] && cst) &&
                                     overlap(rmn[q], rmx[q], cmn, cmx);
                    const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
                    cnt[q] += __popc(m);
                    if (lane == q) mine = m;
                }
                if (mask && lane < kRowGroup && r0 + lane < n)
                    mask[size_t(s0 + r0 + lane) * stride + c] = mine;
            }
            if (lane == 0)
#pragma unroll
                for (uint32_t q = 0; q < kRowGroup; ++q)
                    if (r0 + q < n) row_count[s0 + r0 + q] = cnt[q];
        }
        return;
    }
    const unsigned below = (1u << lane) - 1u;
    for (uint32_t r = slice * kTileWarps + wid; r < n; r += slices * kTileWarps) {
        const uint32_t i = s0 + r;
        const uint32_t total = row_count[i];
        if (total == 0) continue;
        const uint32_t* mrow = mask ? mask + size_t(i) * stride : nullptr;
        const f3 mna = test ? ld3(mn, r) : mk(0.f, 0.f, 0.f);
        const f3 mxa = test ? ld3(mx, r) : mna;
        const bool static_i = test && stat[r] != 0.0f;
        uint32_t slot0 = row_off[i];
        for (uint32_t c0 = (r + 1) / 32; c0 < nwords; c0 += 32) {
            // lane l holds column word c0 + l
            unsigned word = 0;
            if (mrow) {
                if (c0 + lane < nwords) word = mrow[c0 + lane];
            } else {
                for (uint32_t q = 0; q < 32 && c0 + q < nwords; ++q) {
                    const uint32_t j = 32 * (c0 + q) + lane;
                    const bool hit = j < n && j > r && !(static_i && stat[j] != 0.0f) &&
                                     overlap(mna, mxa, ld3(mn, j), ld3(mx, j));
                    const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
                    if (lane == q) word = m;
                }
            }
            // exclusive prefix of the words' population counts
            const uint32_t pc = __popc(word);
            uint32_t incl = pc;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
                if (int(lane) >= off) incl += v;
            }
            const uint32_t excl = incl - pc;
            unsigned nz = __ballot_sync(0xFFFFFFFFu, word != 0u);
            while (nz) {
                const uint32_t q = uint32_t(__ffs(int(nz))) - 1u;
                nz &= nz - 1u;
                const unsigned m = __shfl_sync(0xFFFFFFFFu, word, q);
                const uint32_t pre = __shfl_sync(0xFFFFFFFFu, excl, q);
                if ((m >> lane) & 1u) {
                    const uint32_t slot = slot0 + pre + __popc(m & below);
                    if (slot < w.max_pairs) {
                        w.pairs[size_t(slot) * 2] = i;
                        w.pairs[size_t(slot) * 2 + 1] = s0 + 32 * (c0 + q) + lane;
                    }
                }
            }
            slot0 += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
    }
}

int launch_broadphase_n2(const World& w, const Scratch& s, uint32_t max_scene_bodies,
                         cudaStream_t st) {
    if (w.nb == 0) return 0;
    if (max_scene_bodies <= kTileBodies && w.ns > 0) {
        // one block per `rows` rows of each scene (the tile table), or
        // without a table the largest scene's block count for every scene
        const uint32_t rows = s.bp_tile_rows ? s.bp_tile_rows : kTileRows;
        const uint32_t slices = max(1u, (max_scene_bodies + rows - 1) / rows);
        const uint2* tiles = s.bp_ntiles ? s.bp_tiles : nullptr;
        const uint32_t blocks = tiles ? s.bp_ntiles : w.ns * slices;
        const size_t smem = size_t(7) * max_scene_bodies * sizeof(float);
        k_broad_tile<false><<<blocks, kTileThreads, smem, st>>>(w, tiles, slices, nullptr,
                                                                s.row_count, s.bp_mask, s.bp_stride);
        launch_exclusive_scan(s.row_count, s.row_off, nullptr, w.nb, &w.counters[0], w.max_pairs,
                              kFlagPairOverflow, s, st);
        k_broad_tile<true><<<blocks, kTileThreads, s.bp_mask ? 0 : smem, st>>>(
            w, tiles, slices, s.row_off, s.row_count, s.bp_mask, s.bp_stride);
        return 3;
    }
    const uint32_t threads = 256;
    const uint32_t blocks = uint32_t((uint64_t(w.nb) * 32 + threads - 1) / threads);
    k_broad_n2<false><<<blocks, threads, 0, st>>>(w, nullptr, s.row_count, s.bp_mask, s.bp_stride);
    launch_exclusive_scan(s.row_count, s.row_off, nullptr, w.nb, &w.counters[0], w.max_pairs,
                          kFlagPairOverflow, s, st);
    k_broad_n2<true><<<blocks, threads, 0, st>>>(w, s.row_off, s.row_count, s.bp_mask, s.bp_stride);
    return 3;
}

cudaError_t init_broadphase() {
    const int bytes = int(7 * kTileBodies * sizeof(float));
    const cudaError_t e =
        cudaFuncSetAttribute(k_broad_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_broad_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace seevr
