// body.cu — per-body stages of physics.comp, fused into one warp-per-body
// kernel:  integrate (step 6, physics.comp:586-604) of the previous substep,
// gravity + damping (step 0, 418-428), the world AABB of the body's hull
// (steps 9-11, 686-844) and the render-vertex update (step 7, 607-627).
//
// The reference reduces AABBs with a thread-0 serial loop per 256-vertex
// workgroup and a multi-launch cascade; min/max are exact in any order, so
// a warp-shuffle reduction over the body's contiguous hull range gives the
// same values in one pass.  Hull vertex ownership: body b owns
// [hull_start, hull_start+hull_count), which is what the reference's binary
// search (physics.comp:695-703) yields for contiguous hull ranges.
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

__global__ void __launch_bounds__(256) k_body_stage(World w, Consts k, uint32_t flags, float dt,
                                                    float gx, float gy, float gz) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= w.nb) return;

    float px = 0, py = 0, pz = 0, qx = 0, qy = 0, qz = 0, qw = 1;
    if (lane == 0) {
        px = w.pos[size_t(b) * 3];
        py = w.pos[size_t(b) * 3 + 1];
        pz = w.pos[size_t(b) * 3 + 2];
        qx = w.quat[size_t(b) * 4];
        qy = w.quat[size_t(b) * 4 + 1];
        qz = w.quat[size_t(b) * 4 + 2];
        qw = w.quat[size_t(b) * 4 + 3];
        const float im = w.inv_mass[b];
        if ((flags & (kIntegrate | kGravity)) && im > 0.0f) {
            float vx = w.vel[size_t(b) * 3], vy = w.vel[size_t(b) * 3 + 1],
                  vz = w.vel[size_t(b) * 3 + 2];
            float ox = w.omega[size_t(b) * 3], oy = w.omega[size_t(b) * 3 + 1],
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
    }
    if (!(flags & (kAabb | kRenderVerts))) return;
    const unsigned full = 0xFFFFFFFFu;
    px = __shfl_sync(full, px, 0);
    py = __shfl_sync(full, py, 0);
    pz = __shfl_sync(full, pz, 0);
    qx = __shfl_sync(full, qx, 0);
    qy = __shfl_sync(full, qy, 0);
    qz = __shfl_sync(full, qz, 0);
    qw = __shfl_sync(full, qw, 0);
    const m3 R = quat_to_mat(qx, qy, qz, qw);
    const f3 p = mk(px, py, pz);

    if (flags & kAabb) {
        const uint32_t hs = w.hull_range[size_t(b) * 2], hc = w.hull_range[size_t(b) * 2 + 1];
        const float inf = __int_as_float(0x7f800000);
        f3 mn = mk(inf, inf, inf), mx = mk(-inf, -inf, -inf);
        for (uint32_t i = lane; i < hc; i += 32) {
            const f3 wv = add(p, mul(R, ld3(w.hull, hs + i)));
            mn = vmin(mn, wv);
            mx = vmax(mx, wv);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            mn.x = gmin(mn.x, __shfl_xor_sync(full, mn.x, off));
            mn.y = gmin(mn.y, __shfl_xor_sync(full, mn.y, off));
            mn.z = gmin(mn.z, __shfl_xor_sync(full, mn.z, off));
            mx.x = gmax(mx.x, __shfl_xor_sync(full, mx.x, off));
            mx.y = gmax(mx.y, __shfl_xor_sync(full, mx.y, off));
            mx.z = gmax(mx.z, __shfl_xor_sync(full, mx.z, off));
        }
        if (lane == 0 && hc > 0) {
            st3(w.aabb_min, b, mn);
            st3(w.aabb_max, b, mx);
        }
    }
    if (flags & kRenderVerts) {
        const uint32_t vs = w.vert_start[b];
        uint32_t ve = vs + w.vert_count[b];
        if (ve > w.nv) ve = w.nv;
        for (uint32_t i = vs + lane; i < ve; i += 32) st3(w.verts, i, add(p, mul(R, ld3(w.orig, i))));
    }
}

int launch_body_stage(const World& w, const Consts& k, uint32_t flags, float dt, float gx,
                      float gy, float gz, cudaStream_t st) {
    if (w.nb == 0) return 0;
    const uint32_t threads = 256;
    const uint64_t blocks = (uint64_t(w.nb) * 32 + threads - 1) / threads;
    k_body_stage<<<uint32_t(blocks), threads, 0, st>>>(w, k, flags, dt, gx, gy, gz);
    return 1;
}

}  // namespace seevr
