// body.cu — per-body stages of physics.comp: one kernel fuses integrate
// (step 6, physics.comp:586-604) of the previous substep, gravity + damping
// (step 0, 418-428) and the world AABB of the body's hull (steps 9-11,
// 686-844); the render-vertex update (step 7, 607-627) runs at frame end in
// its own kernel after the state update.
//
// The stage streams every hull vertex once per substep (12 bytes each, the
// bulk of its HBM traffic).  A block takes 256 consecutive bodies: each
// thread updates its body's state with coalesced loads and handles a small
// hull itself; bodies whose hull has more than 32 vertices go to a
// per-block queue that the block's warps then drain, lanes striding over
// the vertices, so no warp waits on a single lane's state update.
//
// The reference reduces AABBs with a thread-0 serial loop per 256-vertex
// workgroup and a multi-launch cascade; min/max are exact in any order, so
// the reductions here give the same values in one pass.  They reduce R v
// and add the position once: rounding is monotone, so the least (greatest)
// of p + R v_i, each rounded, is p + the least (greatest) R v_i, rounded.
// fminf/fmaxf (one instruction) stand for GLSL min/max (y < x ? y : x):
// on numbers the two differ only in which zero they return for
// min(-0, +0), and every later test treats the two zeros alike; a NaN pose
// gives NaN bounds as the reference's reduction does (aabb_bound).  (A NaN
// among a hull's own vertices is skipped here, where the reference keeps
// it when it is the first vertex of its pass.)  Hull vertex
// ownership: body b owns [hull_start, hull_start+hull_count), which is what
// the reference's binary search (physics.comp:695-703) yields for
// contiguous hull ranges.
#include "common.cuh"

namespace seevr {

__global__ void k_hull_range(const float* __restrict__ geom_data, uint32_t* __restrict__ out,
                             uint32_t nb) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nb) return;
    // uint(geom_data[gi*8+0]), uint(geom_data[gi*8+1]) (physics.comp:100-101)
    out[g * 2] = uint32_t(geom_data[size_t(g) * 8]);
    out[g * 2 + 1] = uint32_t(geom_data[size_t(g) * 8 + 1]);
}

int launch_hull_range_from_geom_data(const float* geom_data, uint32_t* out, uint32_t nb,
                                     cudaStream_t st) {
    if (nb == 0) return 0;
    k_hull_range<<<(nb + 255) / 256, 256, 0, st>>>(geom_data, out, nb);
    return 1;
}

constexpr uint32_t kBodyThreads = 256;
// Hulls up to this many vertices are transformed by the body's own thread;
// larger ones by a warp in the block's second phase.
constexpr uint32_t kSmallVerts = 32;
// Vertices per lane per round of loads in the warp phase.
constexpr uint32_t kLaneVerts = 10;

// p + the reduced bound of one axis; NaN when the position or the
// rotation's row on that axis has a NaN.  Then every p + R v of the axis is
// NaN, and the reference's reduction, which starts from the first vertex's
// value and keeps it against NaN (min(x, y) = y < x ? y : x), ends at NaN.
__device__ __forceinline__ float aabb_axis(float p, float r0, float r1, float r2, float m) {
    return (p != p || r0 != r0 || r1 != r1 || r2 != r2) ? __int_as_float(0x7fffffff) : p + m;
}
__device__ __forceinline__ f3 aabb_bound(f3 p, const m3& R, f3 m) {
    return f3{aabb_axis(p.x, R.c0.x, R.c1.x, R.c2.x, m.x), aabb_axis(p.y, R.c0.y, R.c1.y, R.c2.y, m.y),
              aabb_axis(p.z, R.c0.z, R.c1.z, R.c2.z, m.z)};
}
__device__ __forceinline__ f3 fmin3(f3 a, f3 b) { return f3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ f3 fmax3(f3 a, f3 b) { return f3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }

// Integrate (physics.comp:586-604) and gravity (418-428) of body b, in the
// reference's arithmetic; returns the (possibly updated) pose.
__device__ __forceinline__ void body_state(const World& w, const Consts& k, uint32_t flags,
                                           uint32_t b, float dt, float gx, float gy, float gz,
                                           f3& p, float (&q)[4]) {
    float px = w.pos[size_t(b) * 3], py = w.pos[size_t(b) * 3 + 1], pz = w.pos[size_t(b) * 3 + 2];
    float qx = w.quat[size_t(b) * 4], qy = w.quat[size_t(b) * 4 + 1],
          qz = w.quat[size_t(b) * 4 + 2], qw = w.quat[size_t(b) * 4 + 3];
    const float im = w.inv_mass[b];
    if ((flags & (kIntegrate | kGravity)) && im > 0.0f) {
        float vx = w.vel[size_t(b) * 3], vy = w.vel[size_t(b) * 3 + 1], vz = w.vel[size_t(b) * 3 + 2];
        const float ox = w.omega[size_t(b) * 3], oy = w.omega[size_t(b) * 3 + 1],
                    oz = w.omega[size_t(b) * 3 + 2];
        if (flags & kIntegrate) {  // step 6 of the previous substep
            px += vx * dt;
            py += vy * dt;
            pz += vz * dt;
            const float dx = ox * qw + oy * qz - oz * qy;
            const float dy = -ox * qz + oy * qw + oz * qx;
            const float dz = ox * qy - oy * qx + oz * qw;
            const float dw = -ox * qx - oy * qy - oz * qz;
            qx += 0.5f * dx * dt;
            qy += 0.5f * dy * dt;
            qz += 0.5f * dz * dt;
            qw += 0.5f * dw * dt;
            const float l = sqrtf(qx * qx + qy * qy + qz * qz + qw * qw);
            if (l > 1e-8f) {
                qx /= l;
                qy /= l;
                qz /= l;
                qw /= l;
            }
            w.pos[size_t(b) * 3] = px;
            w.pos[size_t(b) * 3 + 1] = py;
            w.pos[size_t(b) * 3 + 2] = pz;
            w.quat[size_t(b) * 4] = qx;
            w.quat[size_t(b) * 4 + 1] = qy;
            w.quat[size_t(b) * 4 + 2] = qz;
            w.quat[size_t(b) * 4 + 3] = qw;
        }
        if (flags & kGravity) {  // step 0 of this substep
            vx = vx * k.lin_damp + gx * dt;
            vy = vy * k.lin_damp + gy * dt;
            vz = vz * k.lin_damp + gz * dt;
            w.vel[size_t(b) * 3] = vx;
            w.vel[size_t(b) * 3 + 1] = vy;
            w.vel[size_t(b) * 3 + 2] = vz;
            w.omega[size_t(b) * 3] = ox * k.ang_damp;
            w.omega[size_t(b) * 3 + 1] = oy * k.ang_damp;
            w.omega[size_t(b) * 3 + 2] = oz * k.ang_damp;
        }
    }
    p = mk(px, py, pz);
    q[0] = qx;
    q[1] = qy;
    q[2] = qz;
    q[3] = qw;
}

// Phase 1, one thread per body: state update, then the AABB of a small hull
// in vertex order.  Bodies with a large hull are queued in shared memory
// with their pose; phase 2 gives each a warp whose lanes stride over the
// vertices and reduce with shuffles (min/max are exact in any order).
__global__ void __launch_bounds__(kBodyThreads) k_body_stage(World w, Consts k, uint32_t flags,
                                                             float dt, float gx, float gy,
                                                             float gz) {
    __shared__ float sh_pose[kBodyThreads][12];  // p xyz, R by columns
    __shared__ uint32_t sh_body[kBodyThreads];
    __shared__ uint32_t sh_n;
    if (check_failed(w.status)) return;  // bounds-check mode: hull ranges not valid
    if (threadIdx.x == 0) sh_n = 0;
    __syncthreads();

    const uint32_t b = blockIdx.x * kBodyThreads + threadIdx.x;
    const float inf = __int_as_float(0x7f800000);
    if (b < w.nb) {
        uint32_t hs = 0, hc = 0;
        if (flags & kAabb) {
            hs = w.hull_range[size_t(b) * 2];
            hc = w.hull_range[size_t(b) * 2 + 1];
        }

        f3 p;
        float q[4];
        body_state(w, k, flags, b, dt, gx, gy, gz, p, q);
        const m3 R = quat_to_mat(q[0], q[1], q[2], q[3]);
        const bool big = hc > kSmallVerts;
        if ((flags & kAabb) && hc <= kSmallVerts) {
            f3 mn = mk(inf, inf, inf), mx = mk(-inf, -inf, -inf);
#pragma unroll 8
            for (uint32_t i = 0; i < hc; ++i) {
                const f3 rv = mul(R, ld3(w.hull, hs + i));
                mn = fmin3(mn, rv);
                mx = fmax3(mx, rv);
            }
            if (hc > 0) {
                st3(w.aabb_min, b, aabb_bound(p, R, mn));
                st3(w.aabb_max, b, aabb_bound(p, R, mx));
            }
        }

        if (big) {
            const uint32_t e = atomicAdd(&sh_n, 1u);
            sh_body[e] = b;
            float* o = sh_pose[e];
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
            o[3] = R.c0.x; o[4] = R.c0.y; o[5] = R.c0.z;
            o[6] = R.c1.x; o[7] = R.c1.y; o[8] = R.c1.z;
            o[9] = R.c2.x; o[10] = R.c2.y; o[11] = R.c2.z;
        }
    }
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned full = 0xFFFFFFFFu;
    for (uint32_t e = warp; e < sh_n; e += kBodyThreads / 32) {
        const uint32_t bb = sh_body[e];
        const float* o = sh_pose[e];
        const f3 p = mk(o[0], o[1], o[2]);
        m3 R;
        R.c0 = mk(o[3], o[4], o[5]);
        R.c1 = mk(o[6], o[7], o[8]);
        R.c2 = mk(o[9], o[10], o[11]);
        if (flags & kAabb) {
            const uint32_t hs = w.hull_range[size_t(bb) * 2], hc = w.hull_range[size_t(bb) * 2 + 1];
            if (hc > kSmallVerts) {
                f3 mn = mk(inf, inf, inf), mx = mk(-inf, -inf, -inf);
                // all loads of a chunk (kLaneVerts per lane) in flight at once:
                // a 16-segment sphere (289 vertices) is one memory latency
                for (uint32_t c0 = 0; c0 < hc; c0 += 32u * kLaneVerts) {
                    f3 v[kLaneVerts];
#pragma unroll
                    for (uint32_t j = 0; j < kLaneVerts; ++j) {
                        const uint32_t i = c0 + lane + 32u * j;
                        if (i < hc) {
                            const float* q = w.hull + size_t(hs + i) * 3;
                            v[j] = mk(__ldg(q), __ldg(q + 1), __ldg(q + 2));
                        }
                    }
#pragma unroll
                    for (uint32_t j = 0; j < kLaneVerts; ++j) {
                        if (c0 + lane + 32u * j < hc) {
                            const f3 rv = mul(R, v[j]);
                            mn = fmin3(mn, rv);
                            mx = fmax3(mx, rv);
                        }
                    }
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    mn.x = fminf(mn.x, __shfl_xor_sync(full, mn.x, off));
                    mn.y = fminf(mn.y, __shfl_xor_sync(full, mn.y, off));
                    mn.z = fminf(mn.z, __shfl_xor_sync(full, mn.z, off));
                    mx.x = fmaxf(mx.x, __shfl_xor_sync(full, mx.x, off));
                    mx.y = fmaxf(mx.y, __shfl_xor_sync(full, mx.y, off));
                    mx.z = fmaxf(mx.z, __shfl_xor_sync(full, mx.z, off));
                }
                if (lane == 0) {
                    st3(w.aabb_min, bb, aabb_bound(p, R, mn));
                    st3(w.aabb_max, bb, aabb_bound(p, R, mx));
                }
            }
        }
    }
}

// Render vertices (step 7, physics.comp:607-627) from the final pose: a warp
// per body, lanes striding over its vertices, kRenderBatch loads in flight
// per lane before the stores (the source and destination buffers may
// alias, so the compiler cannot move a load above an earlier store).  The
// same arithmetic as the per-body stage: R = quat_to_mat(q), v' = p + R v.
constexpr uint32_t kRenderBatch = 8;
constexpr uint32_t kRenderThreads = 256;

__global__ void __launch_bounds__(kRenderThreads) k_render_verts(World w) {
    if (check_failed(w.status)) return;  // bounds-check mode: vertex ranges not valid
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = gridDim.x * (kRenderThreads / 32);
    for (uint32_t b = (blockIdx.x * kRenderThreads + threadIdx.x) >> 5; b < w.nb; b += nwarps) {
        const uint32_t vs = w.vert_start[b];
        uint32_t ve = vs + w.vert_count[b];
        if (ve > w.nv) ve = w.nv;
        if (ve <= vs) continue;
        const f3 p = ld3(w.pos, b);
        const m3 R = quat_to_mat(w.quat, b);
        for (uint32_t c0 = vs; c0 < ve; c0 += 32u * kRenderBatch) {
            f3 v[kRenderBatch];
#pragma unroll
            for (uint32_t j = 0; j < kRenderBatch; ++j) {
                const uint32_t i = c0 + lane + 32u * j;
                if (i < ve) v[j] = ld3(w.orig, i);
            }
#pragma unroll
            for (uint32_t j = 0; j < kRenderBatch; ++j) {
                const uint32_t i = c0 + lane + 32u * j;
                if (i < ve) st3(w.verts, i, add(p, mul(R, v[j])));
            }
        }
    }
}

int launch_body_stage(const World& w, const Consts& k, uint32_t flags, float dt, float gx,
                      float gy, float gz, cudaStream_t st) {
    if (w.nb == 0) return 0;
    const uint32_t blocks = (w.nb + kBodyThreads - 1) / kBodyThreads;
    // render vertices in their own kernel, after the state update: the
    // per-body stage keeps its register budget (and occupancy) for the
    // substep launches
    k_body_stage<<<blocks, kBodyThreads, 0, st>>>(w, k, flags & ~kRenderVerts, dt, gx, gy, gz);
    if (!(flags & kRenderVerts)) return 1;
    const uint32_t rblocks = (w.nb + kRenderThreads / 32 - 1) / (kRenderThreads / 32);
    k_render_verts<<<rblocks < 148u * 64u ? rblocks : 148u * 64u, kRenderThreads, 0, st>>>(w);
    return 2;
}

}  // namespace seevr
