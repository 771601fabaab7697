// lbvh.cu — linear BVH over AABBs, following the LBVH of bvh.comp:
// centroids (bvh.comp:69-79), centroid bounds (101-165), 30-bit Morton codes
// (32-46, 169-183), a stable LSD radix sort (185-295), the Karras 2012
// hierarchy with the index tiebreak for equal codes (59-65, 299-348), leaf
// boxes (352-368) and the bottom-up refit with arrival flags (372-397).
//
// The sort is a onesweep radix sort: 8-bit digits (4 passes for 32-bit
// keys), one upsweep that histograms all four digits, and per pass one
// kernel in which every tile ranks its keys stably (warp match_any
// multisplit), publishes its per-digit counts and resolves its global
// offsets by decoupled look-back.  A stable LSD sort of the same keys gives
// one permutation, so the order equals bvh.comp's 4-bit, 8-pass sort.
//
// The body broadphase traverses the tree once per body to count and once
// to write, emitting pairs (i, j>i) in canonical lexicographic order: the
// same set as the all-pairs test of physics.comp:451-472 (node boxes are
// exact unions of leaf boxes, so every overlapping leaf is reached).  Rows
// of static bodies, which can hold thousands of partners (a ground box), are
// traversed by whole blocks instead of one thread.
#include "common.cuh"
#include "lbvh.cuh"

namespace seevr {

// ---- Morton codes (bvh.comp:32-46) ---------------------------------------
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t quantize10(float x) {
    float t = x * 1024.0f;
    t = t < 0.0f ? 0.0f : (t > 1023.0f ? 1023.0f : t);
    return uint32_t(t);
}
__device__ __forceinline__ uint32_t morton3d(float x, float y, float z) {
    return (expand_bits(quantize10(x)) << 2) | (expand_bits(quantize10(y)) << 1) |
           expand_bits(quantize10(z));
}

// float <-> order-preserving uint (for exact atomic min/max of floats)
__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

// ---- centroids + bounds ----------------------------------------------------
// bounds_o[0..2] = ordered min, [3..5] = ordered max; initialised to
// (0xFFFFFFFF, 0) by the caller.
__global__ void k_body_centroids(const float* __restrict__ aabb_min,
                                 const float* __restrict__ aabb_max, uint32_t n,
                                 float* __restrict__ centroid, uint32_t* bounds_o) {
    __shared__ uint32_t smn[3], smx[3];
    if (threadIdx.x < 3) {
        smn[threadIdx.x] = 0xFFFFFFFFu;
        smx[threadIdx.x] = 0u;
    }
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        // body centroid = AABB centre
        const f3 c = scale(0.5f, add(ld3(aabb_min, i), ld3(aabb_max, i)));
        st3(centroid, i, c);
        atomicMin(&smn[0], f2o(c.x));
        atomicMin(&smn[1], f2o(c.y));
        atomicMin(&smn[2], f2o(c.z));
        atomicMax(&smx[0], f2o(c.x));
        atomicMax(&smx[1], f2o(c.y));
        atomicMax(&smx[2], f2o(c.z));
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&bounds_o[threadIdx.x], smn[threadIdx.x]);
        atomicMax(&bounds_o[3 + threadIdx.x], smx[threadIdx.x]);
    }
}

// triangle centroids (bvh.comp:69-79)
__global__ void k_tri_centroids(const float* __restrict__ verts, const uint32_t* __restrict__ idx,
                                uint32_t n, float* __restrict__ centroid, uint32_t* bounds_o) {
    __shared__ uint32_t smn[3], smx[3];
    if (threadIdx.x < 3) {
        smn[threadIdx.x] = 0xFFFFFFFFu;
        smx[threadIdx.x] = 0u;
    }
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint32_t i0 = idx[size_t(i) * 3], i1 = idx[size_t(i) * 3 + 1], i2 = idx[size_t(i) * 3 + 2];
        f3 c;
        c.x = (verts[size_t(i0) * 3] + verts[size_t(i1) * 3] + verts[size_t(i2) * 3]) / 3.0f;
        c.y = (verts[size_t(i0) * 3 + 1] + verts[size_t(i1) * 3 + 1] + verts[size_t(i2) * 3 + 1]) / 3.0f;
        c.z = (verts[size_t(i0) * 3 + 2] + verts[size_t(i1) * 3 + 2] + verts[size_t(i2) * 3 + 2]) / 3.0f;
        st3(centroid, i, c);
        atomicMin(&smn[0], f2o(c.x));
        atomicMin(&smn[1], f2o(c.y));
        atomicMin(&smn[2], f2o(c.z));
        atomicMax(&smx[0], f2o(c.x));
        atomicMax(&smx[1], f2o(c.y));
        atomicMax(&smx[2], f2o(c.z));
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&bounds_o[threadIdx.x], smn[threadIdx.x]);
        atomicMax(&bounds_o[3 + threadIdx.x], smx[threadIdx.x]);
    }
}

// step_morton (bvh.comp:169-183); also writes identity values and the
// decoded bounds (bounds_f) for the caller.
__global__ void k_morton(const float* __restrict__ centroid, uint32_t n,
                         const uint32_t* __restrict__ bounds_o, uint32_t* __restrict__ keys,
                         uint32_t* __restrict__ vals, float* bounds_f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const f3 bmin = mk(o2f(bounds_o[0]), o2f(bounds_o[1]), o2f(bounds_o[2]));
    const f3 bmax = mk(o2f(bounds_o[3]), o2f(bounds_o[4]), o2f(bounds_o[5]));
    if (i == 0 && bounds_f) {
        st3(bounds_f, 0, bmin);
        st3(bounds_f, 1, bmax);
    }
    if (i >= n) return;
    const f3 ext = sub(bmax, bmin);
    const f3 inv = mk(ext.x > 1e-6f ? 1.0f / ext.x : 0.0f, ext.y > 1e-6f ? 1.0f / ext.y : 0.0f,
                      ext.z > 1e-6f ? 1.0f / ext.z : 0.0f);
    const f3 c = hadamard(sub(ld3(centroid, i), bmin), inv);
    keys[i] = morton3d(c.x, c.y, c.z);
    vals[i] = i;
}

// ---- onesweep radix sort ---------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;  // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048
constexpr uint32_t kRadix = 256;

// global histogram of all four 8-bit digits
__global__ void k_sort_upsweep(const uint32_t* __restrict__ keys, uint32_t n,
                               uint32_t* __restrict__ hist /* [4][256] */) {
    __shared__ uint32_t sh[4][kRadix];
    for (uint32_t t = threadIdx.x; t < 4 * kRadix; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
#pragma unroll
        for (int p = 0; p < 4; ++p) atomicAdd(&sh[p][(k >> (8 * p)) & 0xFFu], 1u);
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < 4 * kRadix; t += blockDim.x)
        if ((&sh[0][0])[t]) atomicAdd(&hist[t], (&sh[0][0])[t]);
}

// exclusive scan of each digit histogram (one block of 4 warps x 256)
__global__ void k_sort_scan(uint32_t* __restrict__ hist) {
    const uint32_t p = threadIdx.x >> 8, d = threadIdx.x & 255u;
    __shared__ uint32_t sh[4][kRadix];
    sh[p][d] = hist[p * kRadix + d];
    __syncthreads();
    if (d == 0) {
        uint32_t run = 0;
        for (uint32_t i = 0; i < kRadix; ++i) {
            const uint32_t v = sh[p][i];
            sh[p][i] = run;
            run += v;
        }
    }
    __syncthreads();
    hist[p * kRadix + d] = sh[p][d];
}

// One LSD pass on digit (shift/8).  status: [1 + tiles*256] u32, zeroed;
// status[0] is the tile ticket.  Flag bits 30-31: 1 = tile aggregate,
// 2 = inclusive prefix; value in bits 0-29 (n < 2^30).
__global__ void __launch_bounds__(kSortThreads)
    k_sort_onesweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                    uint32_t shift, const uint32_t* __restrict__ bin_start, uint32_t* status,
                    uint32_t* err, uint32_t wait_limit) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_hist[kSortWarps][kRadix];
    __shared__ uint32_t s_bin_off[kRadix];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(status, 1u);
    for (uint32_t t = threadIdx.x; t < kSortWarps * kRadix; t += blockDim.x)
        (&s_warp_hist[0][0])[t] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    if (tile >= tiles) return;
    // warp w owns keys [base_w, base_w + 32*kSortItems), processed in order
    const uint32_t base_w = tile * kSortTile + warp * 32 * kSortItems;
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t i = base_w + k * 32 + lane;
        const bool valid = i < n;
        key[k] = valid ? keys_in[i] : 0xFFFFFFFFu;
        val[k] = valid ? vals_in[i] : 0u;
        const uint32_t d = (key[k] >> shift) & 0xFFu;
        const unsigned active = __ballot_sync(0xFFFFFFFFu, valid);
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, valid ? d : 0x100u) & active;
        uint32_t before = 0;
        if (valid) {
            const uint32_t leader = __ffs(peers) - 1;
            const uint32_t cnt = __popc(peers);
            const uint32_t lt = __popc(peers & ((1u << lane) - 1u));
            if (lane == leader) {
                before = s_warp_hist[warp][d];
                s_warp_hist[warp][d] = before + cnt;
            }
            before = __shfl_sync(peers, before, leader);
            rank[k] = before + lt;
        } else {
            rank[k] = 0;
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive offsets over warps and the tile aggregate
    uint32_t agg = 0;
    {
        const uint32_t d = threadIdx.x;  // kSortThreads == kRadix
        for (uint32_t w = 0; w < kSortWarps; ++w) {
            const uint32_t c = s_warp_hist[w][d];
            s_warp_hist[w][d] = agg;
            agg += c;
        }
        // decoupled look-back for digit d
        uint32_t* st = status + 1;
        uint32_t excl = 0;
        if (tile == 0) {
            atomicExch(&st[d], (2u << 30) | agg);
        } else {
            atomicExch(&st[size_t(tile) * kRadix + d], (1u << 30) | agg);
            int p = int(tile) - 1;
            uint32_t spins = 0;
            while (p >= 0) {
                const uint32_t s = *reinterpret_cast<volatile uint32_t*>(&st[size_t(p) * kRadix + d]);
                const uint32_t f = s >> 30;
                if (f == 0u) {
                    if (++spins > wait_limit) {
                        atomicOr(err, kFlagTimeout);
                        break;
                    }
                    continue;
                }
                excl += s & 0x3FFFFFFFu;
                if (f == 2u) break;
                --p;
            }
            atomicExch(&st[size_t(tile) * kRadix + d], (2u << 30) | (excl + agg));
        }
        s_bin_off[d] = bin_start[d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t i = base_w + k * 32 + lane;
        if (i < n) {
            const uint32_t d = (key[k] >> shift) & 0xFFu;
            const uint32_t dst = s_bin_off[d] + s_warp_hist[warp][d] + rank[k];
            keys_out[dst] = key[k];
            vals_out[dst] = val[k];
        }
    }
}

// ---- Karras hierarchy (bvh.comp:59-65, 299-348) ----------------------------
__device__ __forceinline__ int delta(const uint32_t* m, int i, int j, int n) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = m[i], b = m[j];
    if (a == b) return 32 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clz(a ^ b);
}

__global__ void k_karras(const uint32_t* __restrict__ m, uint32_t n, uint32_t* __restrict__ left,
                         uint32_t* __restrict__ right, uint32_t* __restrict__ parent,
                         uint32_t* __restrict__ count, const uint32_t* err) {
    if (halted(err)) return;  // the sort gave up: the keys are not ordered
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        left[n - 1 + i] = i;
        if (count) count[n - 1 + i] = 1;
    }
    if (n < 2 || i >= n - 1) {
        if (i == 0 && parent) parent[0] = kNone;
        return;
    }
    const int ii = int(i), nn = int(n);
    const int d = delta(m, ii, ii + 1, nn) > delta(m, ii, ii - 1, nn) ? 1 : -1;
    const int dmin = delta(m, ii, ii - d, nn);
    int lmax = 2;
    while (delta(m, ii, ii + lmax * d, nn) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(m, ii, ii + (l + t) * d, nn) > dmin) l += t;
    const int j = ii + l * d;
    const int first = min(ii, j), last = max(ii, j);
    const int dn = delta(m, first, last, nn);
    int split = first, stride = last - first;
    while (stride > 1) {
        stride = (stride + 1) / 2;
        const int mid = split + stride;
        if (mid < last && delta(m, first, mid, nn) > dn) split = mid;
    }
    uint32_t lc = uint32_t(split), rc = uint32_t(split + 1);
    if (first == split) lc = uint32_t(split) + n - 1;
    if (last == split + 1) rc = uint32_t(split + 1) + n - 1;
    left[i] = lc;
    right[i] = rc;
    if (count) count[i] = 0;
    parent[lc] = i;
    parent[rc] = i;
    if (i == 0) parent[0] = kNone;
}

// ---- leaves + refit (bvh.comp:352-397) --------------------------------------
__global__ void k_leaves_bodies(const float* __restrict__ aabb_min, const float* __restrict__ aabb_max,
                                const uint32_t* __restrict__ sorted_vals, uint32_t n,
                                float* __restrict__ node_min, float* __restrict__ node_max,
                                uint32_t* __restrict__ flags, const uint32_t* err) {
    if (halted(err)) return;  // slots of the sorted order may be unwritten
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 < n) flags[i] = 0;
    if (i >= n) return;
    const uint32_t b = sorted_vals[i];
    st3(node_min, n - 1 + i, ld3(aabb_min, b));
    st3(node_max, n - 1 + i, ld3(aabb_max, b));
}

__global__ void k_leaves_tris(const float* __restrict__ verts, const uint32_t* __restrict__ idx,
                              const uint32_t* __restrict__ sorted_vals, uint32_t n,
                              float* __restrict__ node_min, float* __restrict__ node_max,
                              uint32_t* __restrict__ prim_idx, uint32_t* __restrict__ flags,
                              const uint32_t* err) {
    if (halted(err)) return;  // slots of the sorted order may be unwritten
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 < n) flags[i] = 0;
    if (i >= n) return;
    const uint32_t pi = sorted_vals[i];
    if (prim_idx) prim_idx[i] = pi;
    const f3 v0 = ld3(verts, idx[size_t(pi) * 3]), v1 = ld3(verts, idx[size_t(pi) * 3 + 1]),
             v2 = ld3(verts, idx[size_t(pi) * 3 + 2]);
    st3(node_min, n - 1 + i, vmin(vmin(v0, v1), v2));
    st3(node_max, n - 1 + i, vmax(vmax(v0, v1), v2));
}

// Bottom-up: the second child to arrive at a node computes its box.
__global__ void k_refit(uint32_t n, const uint32_t* __restrict__ left,
                        const uint32_t* __restrict__ right, const uint32_t* __restrict__ parent,
                        float* node_min, float* node_max, uint32_t* flags, const uint32_t* err) {
    if (halted(err)) return;  // no valid hierarchy to refit
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || n < 2) return;
    uint32_t p = parent[n - 1 + i];
    uint32_t guard = 0;
    while (p != kNone && guard++ < 64u + n) {
        __threadfence();
        if (atomicAdd(&flags[p], 1u) == 0u) return;
        __threadfence();
        const uint32_t l = left[p], r = right[p];
        const f3 lmn = ld3(node_min, l), lmx = ld3(node_max, l);
        const f3 rmn = ld3(node_min, r), rmx = ld3(node_max, r);
        st3(node_min, p, vmin(lmn, rmn));
        st3(node_max, p, vmax(lmx, rmx));
        p = parent[p];
    }
}

// ---- body pairs by traversal ------------------------------------------------
constexpr int kStack = 64;
constexpr int kRowBuf = 32;

__device__ __forceinline__ bool overlap_box(f3 mna, f3 mxa, f3 mnb, f3 mxb) {
    return !(mxa.x < mnb.x || mxb.x < mna.x || mxa.y < mnb.y || mxb.y < mna.y || mxa.z < mnb.z ||
             mxb.z < mna.z);
}

// The body tree as one 32-byte record per node, written after the refit:
// lo = (min, left child or, for a leaf, its body), hi = (max, right child
// or kLeafBit).  A traversal step reads one sector instead of five arrays.
constexpr uint32_t kLeafBit = 0x80000000u;
__global__ void k_pack_nodes(uint32_t n, const float* __restrict__ node_min,
                             const float* __restrict__ node_max, const uint32_t* __restrict__ left,
                             const uint32_t* __restrict__ right, const uint32_t* __restrict__ vals,
                             float4* __restrict__ packed, uint32_t* err) {
    if (halted(err)) return;  // the tree was not built
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * n - 1; k += gridDim.x * blockDim.x) {
        const bool leaf = k >= n - 1;
        const f3 mn = ld3(node_min, k), mx = ld3(node_max, k);
        packed[2 * size_t(k)] = make_float4(mn.x, mn.y, mn.z, __uint_as_float(leaf ? vals[k - (n - 1)] : left[k]));
        packed[2 * size_t(k) + 1] = make_float4(mx.x, mx.y, mx.z, __uint_as_float(leaf ? kLeafBit : right[k]));
    }
}

// Visit every leaf j (original index) with j > lo_j whose box overlaps
// body i's box, excluding static-static; `emit(j)` is called for each.
template <class F>
__device__ __forceinline__ void traverse(const World& w, const LbvhView& t, uint32_t i,
                                         uint32_t lo_j, uint32_t* err, F emit) {
    const f3 mna = ld3(w.aabb_min, i), mxa = ld3(w.aabb_max, i);
    const bool static_i = w.inv_mass[i] <= 0.0f;
    uint32_t stack[kStack];
    int sp = 0;
    stack[sp++] = 0;  // root (n >= 2)
    while (sp > 0) {
        const uint32_t node = stack[--sp];
        const float4 lo = __ldg(&t.packed[2 * size_t(node)]), hi = __ldg(&t.packed[2 * size_t(node) + 1]);
        if (!overlap_box(mna, mxa, mk(lo.x, lo.y, lo.z), mk(hi.x, hi.y, hi.z))) continue;
        const uint32_t a = __float_as_uint(lo.w), b = __float_as_uint(hi.w);
        if (b == kLeafBit) {
            const uint32_t j = a;
            if (j > lo_j && !(static_i && w.inv_mass[j] <= 0.0f)) emit(j);
        } else {
            if (sp + 2 > kStack) {
                atomicOr(err, kFlagTimeout);
                return;
            }
            stack[sp++] = b;
            stack[sp++] = a;
        }
    }
}

// Rows of dynamic bodies, one thread each; static bodies' rows (a ground
// box overlapping thousands of bodies) are left to k_lbvh_static_rows and
// listed here.  A row of at most kRowCache partners is kept, sorted, in
// row_cache, so the write pass copies it instead of traversing again.
// Threads take bodies in Morton order (the tree's leaf order), so a warp's
// bodies are neighbours whose traversals visit the same nodes.
__global__ void k_lbvh_count(World w, LbvhView t, uint32_t* __restrict__ row_count, uint32_t* err,
                             uint32_t* static_list, uint32_t* static_count,
                             uint32_t* __restrict__ row_cache) {
    if (halted(err)) return;  // the tree was not built
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= w.nb) return;
    const uint32_t i = w.nb >= 2 ? t.vals[q] : q;
    if (w.inv_mass[i] <= 0.0f) {
        static_list[atomicAdd(static_count, 1u)] = i;
        return;
    }
    uint32_t c = 0;
    uint32_t buf[kRowCache];
    if (w.nb >= 2)
        traverse(w, t, i, i, err, [&](uint32_t j) {
            if (c < kRowCache) {  // insertion into the ascending buffer
                uint32_t pos = c;
                while (pos > 0 && buf[pos - 1] > j) {
                    buf[pos] = buf[pos - 1];
                    --pos;
                }
                buf[pos] = j;
            }
            ++c;
        });
    row_count[i] = c;
    if (c <= kRowCache)
        for (uint32_t k = 0; k < c; ++k) row_cache[size_t(i) * kRowCache + k] = buf[k];
}

// Rows of static bodies, one block each: a breadth-first traversal whose
// frontier the block's threads expand together.  Count pass: the row's
// length.  Write pass: the row's partners are collected unordered, then each
// is written at its rank (the number of smaller partners), which gives the
// ascending-j order of the canonical pair list.
template <bool kWrite>
__global__ void __launch_bounds__(256)
    k_lbvh_static_rows(World w, LbvhView t, uint32_t* row_count, const uint32_t* row_off,
                       const uint32_t* static_list, const uint32_t* static_count, uint32_t* bfs) {
    __shared__ uint32_t sh_next, sh_found, sh_cur;
    if (halted(w.status)) return;  // the tree (or the row offsets) are not valid
    const uint32_t n = w.nb;
    if (n < 2) return;
    uint32_t* fa = bfs + size_t(blockIdx.x) * 3 * 2 * n;
    uint32_t* fb = fa + 2 * n;
    uint32_t* found = fb + 2 * n;
    const uint32_t ns = *static_count;
    for (uint32_t r = blockIdx.x; r < ns; r += gridDim.x) {
        const uint32_t i = static_list[r];
        const f3 mna = ld3(w.aabb_min, i), mxa = ld3(w.aabb_max, i);
        if (threadIdx.x == 0) {
            fa[0] = 0;  // root
            sh_cur = 1;
            sh_found = 0;
        }
        __syncthreads();
        uint32_t* in = fa;
        uint32_t* out = fb;
        while (sh_cur > 0) {
            const uint32_t cur = sh_cur;
            if (threadIdx.x == 0) sh_next = 0;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < cur; k += blockDim.x) {
                const uint32_t node = in[k];
                const float4 lo = __ldg(&t.packed[2 * size_t(node)]);
                const float4 hi = __ldg(&t.packed[2 * size_t(node) + 1]);
                if (!overlap_box(mna, mxa, mk(lo.x, lo.y, lo.z), mk(hi.x, hi.y, hi.z))) continue;
                const uint32_t a = __float_as_uint(lo.w), b = __float_as_uint(hi.w);
                if (b == kLeafBit) {
                    const uint32_t j = a;
                    // the row owner is static: only dynamic partners count
                    if (j > i && w.inv_mass[j] > 0.0f) found[atomicAdd(&sh_found, 1u)] = j;
                } else {
                    const uint32_t o = atomicAdd(&sh_next, 2u);
                    out[o] = a;
                    out[o + 1] = b;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) sh_cur = sh_next;
            uint32_t* tmp = in;
            in = out;
            out = tmp;
            __syncthreads();
        }
        const uint32_t cnt = sh_found;
        if (!kWrite) {
            if (threadIdx.x == 0) row_count[i] = cnt;
        } else {
            const uint32_t base = row_off[i];
            for (uint32_t e = threadIdx.x; e < cnt; e += blockDim.x) {
                const uint32_t j = found[e];
                uint32_t rank = 0;
                for (uint32_t q = 0; q < cnt; ++q) rank += found[q] < j ? 1u : 0u;
                const uint32_t slot = base + rank;
                if (slot < w.max_pairs) {
                    w.pairs[size_t(slot) * 2] = i;
                    w.pairs[size_t(slot) * 2 + 1] = j;
                }
            }
        }
        __syncthreads();
    }
}

// Writes row i's pairs at row_off[i] in ascending j: a row the count pass
// kept is copied; longer rows are emitted in chunks of up to kRowBuf
// smallest remaining j, one traversal per chunk.
__global__ void k_lbvh_write(World w, LbvhView t, const uint32_t* __restrict__ row_count,
                             const uint32_t* __restrict__ row_off, uint32_t* err,
                             const uint32_t* __restrict__ row_cache) {
    if (halted(err)) return;  // the tree or the row offsets are not valid
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;  // Morton order, as the count
    if (q >= w.nb) return;
    const uint32_t i = w.nb >= 2 ? t.vals[q] : q;
    if (w.inv_mass[i] <= 0.0f) return;  // static rows: k_lbvh_static_rows
    uint32_t remaining = row_count[i];
    uint32_t slot = row_off[i];
    if (remaining <= kRowCache) {
        for (uint32_t k = 0; k < remaining && slot < w.max_pairs; ++k, ++slot) {
            w.pairs[size_t(slot) * 2] = i;
            w.pairs[size_t(slot) * 2 + 1] = row_cache[size_t(i) * kRowCache + k];
        }
        return;
    }
    uint32_t lo = i;
    while (remaining > 0 && slot < w.max_pairs) {
        uint32_t buf[kRowBuf];
        uint32_t nbuf = 0;
        // keep the kRowBuf smallest j > lo, sorted ascending (buf[kRowBuf - 1]
        // is read only once nbuf == kRowBuf, i.e. after every entry is set)
        traverse(w, t, i, lo, err, [&](uint32_t j) {
            if (nbuf == kRowBuf && j >= buf[kRowBuf - 1]) return;
            uint32_t pos = nbuf < kRowBuf ? nbuf++ : kRowBuf - 1;
            while (pos > 0 && buf[pos - 1] > j) {
                buf[pos] = buf[pos - 1];
                --pos;
            }
            buf[pos] = j;
        });
        if (nbuf == 0) break;
        for (uint32_t k = 0; k < nbuf && slot < w.max_pairs; ++k, ++slot) {
            w.pairs[size_t(slot) * 2] = i;
            w.pairs[size_t(slot) * 2 + 1] = buf[k];
        }
        remaining = remaining > nbuf ? remaining - nbuf : 0;
        lo = buf[nbuf - 1];
    }
}

// ---- launchers ---------------------------------------------------------------
static inline uint32_t blocks_for(uint32_t n, uint32_t t) {
    const uint32_t b = (n + t - 1) / t;
    return b ? b : 1;
}

int lbvh_sort(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_tmp,
              uint32_t* vals_tmp, uint32_t* keys_out, uint32_t* vals_out, uint32_t n,
              const LbvhScratch& s, uint32_t* err, cudaStream_t st) {
    // 4 passes ping-pong: in -> tmp -> out -> tmp -> out
    cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * 4 * kRadix, st);
    const uint32_t up_blocks = blocks_for(n, 256) < 148u * 4u ? blocks_for(n, 256) : 148u * 4u;
    k_sort_upsweep<<<up_blocks, 256, 0, st>>>(keys_in, n, s.hist);
    k_sort_scan<<<1, 4 * kRadix, 0, st>>>(s.hist);
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    const uint32_t* ki = keys_in;
    const uint32_t* vi = vals_in;
    int launches = 2;
    for (int p = 0; p < 4; ++p) {
        uint32_t* ko = (p % 2 == 0) ? keys_tmp : keys_out;
        uint32_t* vo = (p % 2 == 0) ? vals_tmp : vals_out;
        cudaMemsetAsync(s.status, 0, sizeof(uint32_t) * (1 + size_t(tiles) * kRadix), st);
        k_sort_onesweep<<<tiles ? tiles : 1, kSortThreads, 0, st>>>(ki, vi, ko, vo, n, 8u * p,
                                                                   s.hist + p * kRadix, s.status, err,
                                                                   s.wait_limit);
        ki = ko;
        vi = vo;
        ++launches;
    }
    return launches;
}

int lbvh_build_bodies(const World& w, const LbvhScratch& s, uint32_t* err, cudaStream_t st) {
    const uint32_t n = w.nb;
    if (n < 2) return 0;
    cudaMemsetAsync(s.bounds_o, 0xFF, sizeof(uint32_t) * 3, st);
    cudaMemsetAsync(s.bounds_o + 3, 0, sizeof(uint32_t) * 3, st);
    k_body_centroids<<<blocks_for(n, 256), 256, 0, st>>>(w.aabb_min, w.aabb_max, n, s.centroid,
                                                         s.bounds_o);
    k_morton<<<blocks_for(n, 256), 256, 0, st>>>(s.centroid, n, s.bounds_o, s.keys_a, s.vals_a,
                                                 s.bounds_f);
    int k = 2 + lbvh_sort(s.keys_a, s.vals_a, s.keys_b, s.vals_b, s.keys_sorted, s.vals_sorted, n,
                          s, err, st);
    k_karras<<<blocks_for(n, 256), 256, 0, st>>>(s.keys_sorted, n, s.left, s.right, s.parent,
                                                 nullptr, err);
    k_leaves_bodies<<<blocks_for(n, 256), 256, 0, st>>>(w.aabb_min, w.aabb_max, s.vals_sorted, n,
                                                        s.node_min, s.node_max, s.flags, err);
    k_refit<<<blocks_for(n, 256), 256, 0, st>>>(n, s.left, s.right, s.parent, s.node_min,
                                                s.node_max, s.flags, err);
    return k + 3;
}

int launch_broadphase_lbvh(const World& w, const Scratch& sc, const LbvhScratch& s,
                           cudaStream_t st) {
    const uint32_t n = w.nb;
    if (n == 0) return 0;
    int k = lbvh_build_bodies(w, s, &sc.status[0], st);
    LbvhView t{s.node_min, s.node_max, s.left, s.right, s.vals_sorted, s.packed};
    if (n >= 2) {
        k_pack_nodes<<<blocks_for(2 * n - 1, 256) < 148u * 8u ? blocks_for(2 * n - 1, 256) : 148u * 8u,
                       256, 0, st>>>(n, s.node_min, s.node_max, s.left, s.right, s.vals_sorted,
                                     s.packed, &sc.status[0]);
        ++k;
    }
    cudaMemsetAsync(s.static_count, 0, sizeof(uint32_t), st);
    k_lbvh_count<<<blocks_for(n, 128), 128, 0, st>>>(w, t, sc.row_count, &sc.status[0],
                                                     s.static_list, s.static_count, s.row_cache);
    k_lbvh_static_rows<false><<<kStaticBlocks, 256, 0, st>>>(w, t, sc.row_count, nullptr,
                                                            s.static_list, s.static_count, s.bfs);
    launch_exclusive_scan(sc.row_count, sc.row_off, nullptr, n, &w.counters[0], w.max_pairs,
                          kFlagPairOverflow, sc, st);
    k_lbvh_write<<<blocks_for(n, 128), 128, 0, st>>>(w, t, sc.row_count, sc.row_off, &sc.status[0],
                                                     s.row_cache);
    k_lbvh_static_rows<true><<<kStaticBlocks, 256, 0, st>>>(w, t, nullptr, sc.row_off,
                                                           s.static_list, s.static_count, s.bfs);
    return k + 5;
}

int lbvh_build_triangles(const float* verts, const uint32_t* idx, uint32_t n, const LbvhScratch& s,
                         const TriOut& o, uint32_t* err, cudaStream_t st) {
    if (n == 0) return 0;
    cudaMemsetAsync(s.bounds_o, 0xFF, sizeof(uint32_t) * 3, st);
    cudaMemsetAsync(s.bounds_o + 3, 0, sizeof(uint32_t) * 3, st);
    k_tri_centroids<<<blocks_for(n, 256), 256, 0, st>>>(verts, idx, n, o.centroids, s.bounds_o);
    k_morton<<<blocks_for(n, 256), 256, 0, st>>>(o.centroids, n, s.bounds_o, s.keys_a, s.vals_a,
                                                 o.scene_bounds);
    int k = 2 + lbvh_sort(s.keys_a, s.vals_a, s.keys_b, s.vals_b, o.morton, o.sort_idx, n, s, err,
                          st);
    k_karras<<<blocks_for(n, 256), 256, 0, st>>>(o.morton, n, o.left, o.right, o.parent, o.count,
                                                 err);
    k_leaves_tris<<<blocks_for(n, 256), 256, 0, st>>>(verts, idx, o.sort_idx, n, o.node_min,
                                                      o.node_max, o.prim_idx, o.flags, err);
    k_refit<<<blocks_for(n, 256), 256, 0, st>>>(n, o.left, o.right, o.parent, o.node_min,
                                                o.node_max, o.flags, err);
    return k + 3;
}

}  // namespace seevr
