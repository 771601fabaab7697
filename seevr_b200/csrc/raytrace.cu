// raytrace.cu — the path tracer of raytrace.comp (Raytracer.render,
// raytracer.zig:159-200) over the triangle LBVH, writing a headless RGBA32F
// buffer in place of the Vulkan storage image.
//
// Each sample path of raytrace.comp (16 samples per pixel, up to 16
// bounces, Russian roulette after the first, Lambert / metal / glass
// materials, sky colour on a miss; raytrace.comp:37-282) keeps the shader's
// arithmetic, but the work is laid out for the GPU rather than as the
// shader's thread per pixel:
//   - a pre-pass packs the BVH into one 32-byte record per node (bounds and
//     child or leaf words: one sector per visit instead of five scattered
//     loads) and the triangles into 48-byte records in leaf order (v0 and
//     the two edges the intersection test forms, with the triangle index),
//     so a leaf's triangles are one contiguous read;
//   - a persistent grid of lanes runs sample paths one bounce per loop
//     step, and a lane whose path ends takes the next (pixel, sample) from
//     a warp-aggregated ticket, so lanes do not idle while the longest path
//     of their warp finishes;
//   - each path's colour is stored per sample and a resolve pass sums a
//     pixel's 16 samples in sample order, as the shader's loop does.
// The traversal visits nodes in the shader's order (left pushed before
// right, the same stack bound), every expression keeps its evaluation
// order and the library is built without FMA contraction, so the image
// equals the CPU restatement's bit for bit.  Three functions whose GLSL
// precision is implementation-defined are pinned here, and the restatement
// uses the same definitions:
//   - sin/cos of the hemisphere angle: reduction by quadrant (pi/2 split in
//     two parts, Cody and Waite's method) and Maclaurin polynomials on
//     [-pi/4, pi/4] to x^9 / x^10 (truncation below 2e-9);
//   - pow(x, 5.0) in Schlick's Fresnel: ((x*x)*(x*x))*x;
//   - the field-of-view scale tan(30 degrees): computed on the host in
//     double and rounded to float.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "../../include/seevr.h"
#include "common.cuh"

namespace seevr {
namespace {

constexpr float kPi = 3.14159265f;
constexpr int kMaxBounces = 16;
constexpr int kSamples = 16;

struct RtArgs {
    float* image;
    const float* verts;
    const uint32_t* idx;
    const float* node_min;
    const float* node_max;
    const uint32_t* left;
    const uint32_t* right;
    const uint32_t* count;
    const uint32_t* prim;
    const uint32_t* tri_geom;
    const uint32_t* geom_material;
    const float* albedo;
    const float* roughness;
    const float* metallic;
    const float* emission;
    const float* ior;
    f3 cam_pos, cam_dir, cam_right, cam_up;
    uint32_t width, height, frame, num_tris;
    float fov_scale;
};

// PCG hash (raytrace.comp:43-47)
__device__ __forceinline__ uint32_t pcg(uint32_t seed) {
    const uint32_t state = seed * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
// rand_f (raytrace.comp:49-51): the literal 4294967295.0 is a float, 2^32
__device__ __forceinline__ float rand_f(uint32_t seed) { return float(pcg(seed)) / 4294967296.0f; }

// sin and cos of x >= 0 (see the header comment)
__device__ __forceinline__ void sincos_pinned(float x, float& s, float& c) {
    const float kHalfPiHi = 1.57079637050628662109375f;       // float(pi/2)
    const float kHalfPiLo = -4.37113900018624283e-8f;          // pi/2 - kHalfPiHi
    const float q = float(int(x * 0.636619772f + 0.5f));      // nearest quadrant
    const float r = (x - q * kHalfPiHi) - q * kHalfPiLo;
    const float r2 = r * r;
    const float sp = r * (1.0f + r2 * (-1.0f / 6.0f + r2 * (1.0f / 120.0f + r2 * (-1.0f / 5040.0f +
                                                                                  r2 * (1.0f / 362880.0f)))));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (1.0f / 24.0f + r2 * (-1.0f / 720.0f +
                                                                    r2 * (1.0f / 40320.0f +
                                                                          r2 * (-1.0f / 3628800.0f)))));
    switch (int(q) & 3) {
        case 0: s = sp; c = cp; break;
        case 1: s = cp; c = -sp; break;
        case 2: s = -sp; c = -cp; break;
        default: s = -cp; c = sp; break;
    }
}

// GLSL built-ins with their specified definitions
__device__ __forceinline__ f3 mix3(f3 x, f3 y, float a) { return add(scale(1.0f - a, x), scale(a, y)); }
__device__ __forceinline__ f3 reflect3(f3 i, f3 n) { return sub(i, scale(2.0f * dot(n, i), n)); }
__device__ __forceinline__ f3 refract3(f3 i, f3 n, float eta) {
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return mk(0.f, 0.f, 0.f);
    return sub(scale(eta, i), scale(eta * d + sqrtf(k), n));
}
__device__ __forceinline__ f3 mul3(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }

// ray_tri (raytrace.comp:55-69): Moller-Trumbore, t > 0.001; the edges
// e1 = v1 - v0 and e2 = v2 - v0 come precomputed from the packed triangle
__device__ __forceinline__ float ray_tri(f3 ro, f3 rd, f3 v0, f3 e1, f3 e2) {
    const f3 h = cross(rd, e2);
    const float a = dot(e1, h);
    if (fabsf(a) < 1e-8f) return -1.0f;
    const float f = 1.0f / a;
    const f3 s = sub(ro, v0);
    const float u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const f3 q = cross(s, e1);
    const float v = f * dot(rd, q);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = f * dot(e2, q);
    return t > 0.001f ? t : -1.0f;
}

// ray_aabb (raytrace.comp:73-81) with GLSL min/max
__device__ __forceinline__ bool ray_aabb(f3 ro, f3 inv_d, f3 bmin, f3 bmax, float closest) {
    const f3 t1 = mul3(sub(bmin, ro), inv_d), t2 = mul3(sub(bmax, ro), inv_d);
    const f3 tmin = vmin(t1, t2), tmax = vmax(t1, t2);
    const float enter = gmax(gmax(tmin.x, tmin.y), tmin.z);
    const float exit_ = gmin(gmin(tmax.x, tmax.y), tmax.z);
    return exit_ >= enter && enter < closest && exit_ > 0.0f;
}

// One BVH node: bounds, with the left child (or a leaf's first primitive
// slot) in lo.w and the right child (or 0x80000000 | a leaf's count) in hi.w.
struct NodeP {
    float4 lo, hi;
};
// One triangle in leaf order: v0 with the triangle index, e1, e2.
struct TriP {
    float4 a, b, c;
};
constexpr uint32_t kLeafBit = 0x80000000u;

__global__ void k_rt_pack_nodes(RtArgs g, uint32_t nnodes, NodeP* __restrict__ out) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < nnodes; n += gridDim.x * blockDim.x) {
        const f3 lo = ld3(g.node_min, n), hi = ld3(g.node_max, n);
        const uint32_t cnt = g.count[n];
        const uint32_t w = cnt > 0 ? (kLeafBit | cnt) : g.right[n];
        out[n].lo = make_float4(lo.x, lo.y, lo.z, __uint_as_float(g.left[n]));
        out[n].hi = make_float4(hi.x, hi.y, hi.z, __uint_as_float(w));
    }
}

__global__ void k_rt_pack_tris(RtArgs g, TriP* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.num_tris; i += gridDim.x * blockDim.x) {
        const uint32_t ti = g.prim[i];
        const f3 v0 = ld3(g.verts, g.idx[size_t(ti) * 3]);
        const f3 v1 = ld3(g.verts, g.idx[size_t(ti) * 3 + 1]);
        const f3 v2 = ld3(g.verts, g.idx[size_t(ti) * 3 + 2]);
        const f3 e1 = sub(v1, v0), e2 = sub(v2, v0);
        out[i].a = make_float4(v0.x, v0.y, v0.z, __uint_as_float(ti));
        out[i].b = make_float4(e1.x, e1.y, e1.z, 0.0f);
        out[i].c = make_float4(e2.x, e2.y, e2.z, 0.0f);
    }
}

// trace (raytrace.comp:85-131) over the packed records: the same visiting
// order (left pushed before right) and stack bound (32 entries, pushes
// guarded by sp < 31)
__device__ void trace(const NodeP* __restrict__ nodes, const TriP* __restrict__ tris, f3 ro, f3 rd,
                      float& closest, f3& normal, uint32_t& hit, bool& front) {
    closest = 1e10f;
    normal = mk(0.f, 1.f, 0.f);
    hit = 0xFFFFFFFFu;
    front = true;
    const f3 inv_d = mk(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    uint32_t stack[32];
    stack[0] = 0;
    int sp = 1;
    while (sp > 0) {
        --sp;
        const uint32_t node = stack[sp];
        const float4 lo = __ldg(&nodes[node].lo), hi = __ldg(&nodes[node].hi);
        if (!ray_aabb(ro, inv_d, mk(lo.x, lo.y, lo.z), mk(hi.x, hi.y, hi.z), closest)) continue;
        const uint32_t lf = __float_as_uint(lo.w), wd = __float_as_uint(hi.w);
        if (wd & kLeafBit) {
            const uint32_t cnt = wd & ~kLeafBit;
            for (uint32_t i = 0; i < cnt; ++i) {
                const float4 a = __ldg(&tris[lf + i].a), b = __ldg(&tris[lf + i].b),
                             c = __ldg(&tris[lf + i].c);
                const f3 e1 = mk(b.x, b.y, b.z), e2 = mk(c.x, c.y, c.z);
                const float t = ray_tri(ro, rd, mk(a.x, a.y, a.z), e1, e2);
                if (t > 0.0f && t < closest) {
                    closest = t;
                    const f3 n = normalize(cross(e1, e2));
                    front = dot(n, rd) < 0.0f;
                    normal = front ? n : neg(n);
                    hit = __float_as_uint(a.w);
                }
            }
        } else {
            if (sp < 31) stack[sp++] = lf;
            if (sp < 31) stack[sp++] = wd;
        }
    }
}

__device__ __forceinline__ f3 sky_color(f3 rd) {  // raytrace.comp:135-138
    const float t = 0.5f * (rd.y + 1.0f);
    return scale(0.8f, mix3(mk(1.f, 1.f, 1.f), mk(0.5f, 0.7f, 1.0f), t));
}

__device__ __forceinline__ f3 sample_hemisphere(f3 n, uint32_t seed1, uint32_t seed2) {  // 142-153
    const float r1 = rand_f(seed1), r2 = rand_f(seed2);
    const float phi = 2.0f * kPi * r1;
    const float cos_t = sqrtf(r2), sin_t = sqrtf(1.0f - r2);
    const f3 up = fabsf(n.y) > 0.99f ? mk(1.f, 0.f, 0.f) : mk(0.f, 1.f, 0.f);
    const f3 tan1 = normalize(cross(up, n));
    const f3 tan2 = cross(n, tan1);
    float sp, cp;
    sincos_pinned(phi, sp, cp);
    return normalize(add(add(scale(cp, scale(sin_t, tan1)), scale(cos_t, n)), scale(sp, scale(sin_t, tan2))));
}

__device__ __forceinline__ float schlick(float cos_theta, float r0) {  // 157-159
    const float x = 1.0f - cos_theta;
    return r0 + (1.0f - r0) * (((x * x) * (x * x)) * x);
}

constexpr uint32_t kRtThreads = 128;

// The camera ray of sample si of pixel (px, py) (raytrace.comp:176-190).
__device__ __forceinline__ void camera_ray(const RtArgs& g, uint32_t px, uint32_t py, uint32_t si,
                                           uint32_t& seed, f3& ro, f3& rd) {
    const float aspect = float(g.width) / float(g.height);
    seed = px + py * g.width + g.frame * g.width * g.height + si * 12345u;
    const float jx = rand_f(seed) - 0.5f;
    const float jy = rand_f(seed + 1u) - 0.5f;
    const float u = (2.0f * (float(px) + 0.5f + jx) / float(g.width) - 1.0f) * aspect * g.fov_scale;
    const float v = -(2.0f * (float(py) + 0.5f + jy) / float(g.height) - 1.0f) * g.fov_scale;
    rd = normalize(add(add(g.cam_dir, scale(u, g.cam_right)), scale(v, g.cam_up)));
    ro = g.cam_pos;
}

// Sample paths (raytrace.comp:192-270), one bounce per loop step.  Item q
// is sample q % 16 of pixel q / 16 (row-major), so a warp's first paths are
// two neighbouring pixels' samples; its colour goes to samples[3q..3q+2].
__global__ void __launch_bounds__(kRtThreads) k_rt_paths(RtArgs g, const NodeP* __restrict__ nodes,
                                                         const TriP* __restrict__ tris,
                                                         float* __restrict__ samples,
                                                         uint32_t* __restrict__ ticket,
                                                         uint32_t nitems) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned full = 0xFFFFFFFFu;
    bool active = false, drained = false;
    uint32_t item = 0, seed = 0, bounce = 0;
    f3 ro = mk(0.f, 0.f, 0.f), rd = ro, throughput = ro, color = ro;
    while (true) {
        if (!drained) {  // idle lanes take the next items
            const unsigned need = __ballot_sync(full, !active);
            if (need) {
                const uint32_t leader = __ffs(need) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(ticket, uint32_t(__popc(need)));
                base = __shfl_sync(full, base, leader);
                if (base + __popc(need) >= nitems) drained = true;
                if (!active) {
                    const uint32_t q = base + __popc(need & ((1u << lane) - 1u));
                    if (q < nitems) {
                        item = q;
                        const uint32_t pix = q >> 4;
                        camera_ray(g, pix % g.width, pix / g.width, q & 15u, seed, ro, rd);
                        throughput = mk(1.f, 1.f, 1.f);
                        color = mk(0.f, 0.f, 0.f);
                        bounce = 0;
                        active = true;
                    }
                }
            }
        }
        if (__ballot_sync(full, active) == 0u) break;
        if (!active) continue;

        float t;
        f3 normal;
        uint32_t hit;
        bool front;
        trace(nodes, tris, ro, rd, t, normal, hit, front);
        bool done = false;
        if (t >= 1e9f) {
            color = add(color, mul3(throughput, sky_color(rd)));
            done = true;
        } else {
            const uint32_t mi = g.geom_material[g.tri_geom[hit]];
            const f3 albedo = ld3(g.albedo, mi);
            const float rough = g.roughness[mi], metal = g.metallic[mi], ior = g.ior[mi];
            const f3 emission = ld3(g.emission, mi);
            color = add(color, mul3(throughput, emission));
            if (emission.x + emission.y + emission.z > 0.0f) done = true;
            const f3 hp = add(ro, scale(t, rd));
            if (!done && bounce > 0) {  // Russian roulette
                const float p = gmax(throughput.x, gmax(throughput.y, throughput.z));
                if (rand_f(seed + bounce * 7u) > p) done = true;
                else throughput = mk(throughput.x / p, throughput.y / p, throughput.z / p);
            }
            if (!done) {
                seed = pcg(seed);
                if (ior > 0.0f) {  // glass
                    const float eta = front ? (1.0f / ior) : ior;
                    const float cos_i = fabsf(dot(rd, normal));
                    const float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
                    float r0 = (1.0f - ior) / (1.0f + ior);
                    r0 = r0 * r0;
                    const float fresnel = schlick(cos_i, r0);
                    const bool tir = sin2_t > 1.0f;
                    if (rand_f(seed + 5u) < fresnel || tir) {
                        rd = reflect3(rd, normal);
                        ro = add(hp, scale(0.001f, normal));
                    } else {
                        rd = refract3(rd, normal, eta);
                        ro = sub(hp, scale(0.001f, normal));
                    }
                    throughput = mul3(throughput, albedo);
                } else if (metal > 0.5f) {  // metal
                    const f3 refl = reflect3(rd, normal);
                    const f3 diff = sample_hemisphere(normal, seed, seed + 1u);
                    rd = normalize(mix3(refl, diff, rough * rough));
                    throughput = mul3(throughput, albedo);
                    ro = add(hp, scale(0.001f, normal));
                } else {  // dielectric
                    const f3 refl = reflect3(rd, normal);
                    const f3 diff = sample_hemisphere(normal, seed, seed + 1u);
                    const float cos_theta = gmax(dot(neg(rd), normal), 0.0f);
                    const float fresnel = schlick(cos_theta, 0.04f);
                    if (rand_f(seed + 3u) < fresnel) {
                        rd = normalize(mix3(refl, diff, rough * rough));
                    } else {
                        rd = diff;
                        throughput = mul3(throughput, albedo);
                    }
                    ro = add(hp, scale(0.001f, normal));
                }
                if (++bounce >= uint32_t(kMaxBounces)) done = true;
            }
        }
        if (done) {
            st3(samples, item, color);
            active = false;
        }
    }
}

// A pixel's samples summed in sample order and averaged (raytrace.comp:272-281).
__global__ void k_rt_resolve(RtArgs g, const float* __restrict__ samples) {
    const uint32_t npix = g.width * g.height;
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        f3 pixel = mk(0.f, 0.f, 0.f);
        for (uint32_t si = 0; si < uint32_t(kSamples); ++si) pixel = add(pixel, ld3(samples, pix * 16u + si));
        const float inv = float(kSamples);
        float* o = g.image + size_t(pix) * 4;
        o[0] = pixel.x / inv;
        o[1] = pixel.y / inv;
        o[2] = pixel.z / inv;
        o[3] = 1.0f;
    }
}

// The work arrays come from a memory pool of the library's own per device,
// which keeps freed memory for the next frame (the device's default pool
// returns it to the system at every synchronisation, and mapping it again
// costs milliseconds per frame).
cudaMemPool_t work_pool(int dev) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = ~uint64_t(0);
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    return pools[dev];
}

}  // namespace
}  // namespace seevr

using namespace seevr;

extern "C" {

float seevr_raytrace_fov_scale(void) {
    // tan(30 degrees) as raytrace.comp:172 computes its argument in float
    const float arg = 30.0f * kPi / 180.0f;
    return float(std::tan(double(arg)));
}

seevr_status seevr_raytrace(const seevr_rt_bindings* b, const seevr_rt_params* p, void* stream) {
    if (!b || !p) {
        set_last_error("bindings or params is NULL");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    for (int i = 0; i < SEEVR_RT_NUM_BINDINGS; ++i)
        if (!b->ptr[i]) {
            set_last_error("raytrace binding " + std::to_string(i) + " is NULL");
            return SEEVR_ERR_INVALID_ARGUMENT;
        }
    if (p->width == 0 || p->height == 0) return SEEVR_OK;
    if (p->num_triangles == 0) {
        set_last_error("num_triangles is 0: the tree has no root");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    RtArgs g;
    g.image = static_cast<float*>(b->ptr[SEEVR_RT_IMAGE]);
    g.verts = static_cast<const float*>(b->ptr[SEEVR_RT_VERTICES]);
    g.idx = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_INDICES]);
    g.node_min = static_cast<const float*>(b->ptr[SEEVR_RT_NODE_MIN]);
    g.node_max = static_cast<const float*>(b->ptr[SEEVR_RT_NODE_MAX]);
    g.left = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_LEFT]);
    g.right = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_RIGHT]);
    g.count = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_COUNT]);
    g.prim = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_PRIM]);
    g.tri_geom = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_TRI_GEOM]);
    g.geom_material = static_cast<const uint32_t*>(b->ptr[SEEVR_RT_GEOM_MATERIAL]);
    g.albedo = static_cast<const float*>(b->ptr[SEEVR_RT_MAT_ALBEDO]);
    g.roughness = static_cast<const float*>(b->ptr[SEEVR_RT_MAT_ROUGHNESS]);
    g.metallic = static_cast<const float*>(b->ptr[SEEVR_RT_MAT_METALLIC]);
    g.emission = static_cast<const float*>(b->ptr[SEEVR_RT_MAT_EMISSION]);
    g.ior = static_cast<const float*>(b->ptr[SEEVR_RT_MAT_IOR]);
    g.cam_pos = f3{p->cam_pos[0], p->cam_pos[1], p->cam_pos[2]};
    g.cam_dir = f3{p->cam_dir[0], p->cam_dir[1], p->cam_dir[2]};
    g.cam_right = f3{p->cam_right[0], p->cam_right[1], p->cam_right[2]};
    g.cam_up = f3{p->cam_up[0], p->cam_up[1], p->cam_up[2]};
    g.width = p->width;
    g.height = p->height;
    g.frame = p->frame_num;
    g.num_tris = p->num_triangles;
    g.fov_scale = seevr_raytrace_fov_scale();
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t npix = uint64_t(p->width) * p->height;
    if (npix * kSamples >= (1ull << 32)) {
        set_last_error("width * height * 16 samples must stay below 2^32");
        return SEEVR_ERR_INVALID_ARGUMENT;
    }
    const uint32_t nitems = uint32_t(npix * kSamples);
    const uint32_t nnodes = 2 * p->num_triangles - 1;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rt_paths, kRtThreads, 0);
    // work arrays, stream-ordered: packed nodes and triangles, per-sample
    // colours, the path ticket
    const size_t node_bytes = size_t(nnodes) * sizeof(NodeP), tri_bytes = size_t(p->num_triangles) * sizeof(TriP);
    const size_t sample_bytes = size_t(nitems) * 3 * sizeof(float);
    void* work = nullptr;
    const cudaMemPool_t pool = work_pool(dev);
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&work, node_bytes + tri_bytes + sample_bytes + 16, pool, st)
                         : cudaMallocAsync(&work, node_bytes + tri_bytes + sample_bytes + 16, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_last_error(std::string("raytrace work arrays: ") + cudaGetErrorString(e));
        return SEEVR_ERR_OUT_OF_MEMORY;
    }
    char* w = static_cast<char*>(work);
    NodeP* nodes = reinterpret_cast<NodeP*>(w);
    TriP* tris = reinterpret_cast<TriP*>(w + node_bytes);
    float* samples = reinterpret_cast<float*>(w + node_bytes + tri_bytes);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(w + node_bytes + tri_bytes + sample_bytes);
    const uint32_t cap = uint32_t(std::max(sms, 1)) * 8u;
    cudaMemsetAsync(ticket, 0, sizeof(uint32_t), st);
    k_rt_pack_nodes<<<std::min((nnodes + 255) / 256, cap), 256, 0, st>>>(g, nnodes, nodes);
    k_rt_pack_tris<<<std::min((p->num_triangles + 255) / 256, cap), 256, 0, st>>>(g, tris);
    const uint32_t resident = uint32_t(std::max(sms, 1)) * uint32_t(std::max(per_sm, 1));
    const uint32_t blocks = std::min((nitems + kRtThreads - 1) / kRtThreads, resident);
    k_rt_paths<<<blocks, kRtThreads, 0, st>>>(g, nodes, tris, samples, ticket, nitems);
    k_rt_resolve<<<std::min(uint32_t((npix + 255) / 256), cap), 256, 0, st>>>(g, samples);
    e = cudaGetLastError();
    cudaFreeAsync(work, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_last_error(std::string("raytrace: ") + cudaGetErrorString(e));
        return SEEVR_ERR_CUDA;
    }
    return SEEVR_OK;
}

}  // extern "C"
