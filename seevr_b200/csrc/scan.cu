// scan.cu — single-pass exclusive prefix sum with decoupled look-back.
//
// Used wherever the reference appends with atomicAdd (pairs,
// physics.comp:465; contacts, physics.comp:404): counting, scanning and
// writing at the scanned offsets gives the same totals in a deterministic
// canonical order.  Tiles take tickets from an atomic counter so every tile
// a block waits on has already started; each wait is bounded (the handle's
// wait limit, kSpinLimit polls by default) and raises kFlagTimeout instead
// of hanging.  Offsets written after a wait gave up are too small but stay
// within `out`; the kernels that would use them see the timeout bit and
// return (timed_out).
#include "common.cuh"

namespace seevr {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, const uint32_t* n_dev,
           uint32_t n_cap, uint32_t* total_out, uint32_t total_cap, uint32_t overflow_bit,
           unsigned long long* tiles, uint32_t* status, uint32_t wait_limit) {
    __shared__ uint32_t s_tile, s_excl;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const uint32_t n = n_dev ? min(*n_dev, n_cap) : n_cap;
    const uint32_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (threadIdx.x == 0) s_tile = atomicAdd(reinterpret_cast<unsigned int*>(tiles), 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) {
        if (n == 0 && tile == 0 && threadIdx.x == 0 && total_out) *total_out = 0;
        return;
    }
    const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        sum += v[i];
    }
    // block exclusive scan of per-thread sums
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if (lane >= uint32_t(off)) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t ws = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
        uint32_t wi = ws;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, off);
            if (lane >= uint32_t(off)) wi += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = wi - ws;  // exclusive warp offsets
        if (lane == kScanThreads / 32 - 1) {
            // lane 7 holds the block aggregate in wi; look back
            const uint32_t agg = wi;
            unsigned long long* st = tiles + 1;
            uint32_t excl = 0;
            if (tile == 0) {
                atomicExch(&st[0], (2ull << 32) | agg);
            } else {
                atomicExch(&st[tile], (1ull << 32) | agg);
                int p = int(tile) - 1;
                uint32_t spins = 0;
                while (p >= 0) {
                    const unsigned long long s = ld_volatile(&st[p]);
                    const uint32_t f = uint32_t(s >> 32);
                    if (f == 0u) {
                        if (++spins > wait_limit) {
                            atomicOr(status, kFlagTimeout);
                            break;
                        }
                        continue;
                    }
                    excl += uint32_t(s);
                    if (f == 2u) break;
                    --p;
                }
                atomicExch(&st[tile], (2ull << 32) | (excl + agg));
            }
            s_excl = excl;
            if (tile == ntiles - 1) {
                const uint32_t total = excl + agg;
                if (total_out) *total_out = total;
                if (total > total_cap) atomicOr(status, overflow_bit);
            }
        }
    }
    __syncthreads();
    uint32_t run = s_excl + s_warp[warp] + (incl - sum);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

int launch_exclusive_scan(const uint32_t* in, uint32_t* out, const uint32_t* n_dev,
                          uint32_t n_cap, uint32_t* total_out, uint32_t total_cap,
                          uint32_t overflow_bit, const Scratch& s, cudaStream_t st) {
    const uint32_t tiles = (n_cap + kScanTile - 1) / kScanTile;
    const uint32_t blocks = tiles > 0 ? tiles : 1;
    cudaMemsetAsync(s.scan_tiles, 0, sizeof(unsigned long long) * (blocks + 1), st);
    k_scan<<<blocks, kScanThreads, 0, st>>>(in, out, n_dev, n_cap, total_out, total_cap,
                                            overflow_bit, s.scan_tiles, s.status, s.wait_limit);
    return 1;
}

}  // namespace seevr
