// Host-side scene builder: the CPU staging half of seeVR's Data
// (src/data.zig).  Builders keep the reference's float operation order so
// that masses, inertias, hull vertices and support lookups are the values
// the Zig host would upload.  Compiled without FP contraction.
#include "../../include/seevr_scene.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr uint32_t kSupportAxes = 3;       // data.zig:20
constexpr uint32_t kSupportBins = 64;      // data.zig:21
constexpr uint32_t kSupportThreshold = 32; // data.zig:22
constexpr uint32_t kSupportEntry = kSupportAxes * kSupportBins;  // 192

// splitmix64 stream: the one seeded generator of every workload.
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // U[0,1) with 53 random bits
    double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double lo, double hi) { return lo + (hi - lo) * uniform(); }
    // N(0,1) by Box-Muller (one of the pair)
    double normal() {
        double u1 = 1.0 - uniform();  // (0,1]
        double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    // Uniform unit quaternion (Shoemake), xyzw
    void quat(float q[4]) {
        double u1 = uniform(), u2 = uniform(), u3 = uniform();
        double a = std::sqrt(1.0 - u1), b = std::sqrt(u1);
        q[0] = float(a * std::sin(6.283185307179586 * u2));
        q[1] = float(a * std::cos(6.283185307179586 * u2));
        q[2] = float(b * std::sin(6.283185307179586 * u3));
        q[3] = float(b * std::cos(6.283185307179586 * u3));
    }
};

}  // namespace

struct seevr_scene {
    // render
    std::vector<float> vertices, colors, orig_verts;
    std::vector<uint32_t> indices;
    // body
    std::vector<float> body_pos, body_quat, body_vel, body_omega, body_inv_mass,
        body_inertia, body_inv_inertia;
    std::vector<uint32_t> body_vert_start, body_vert_count;
    // geom
    std::vector<int32_t> geom_type;
    std::vector<uint32_t> geom_body_idx, geom_material, geom_vert_start,
        geom_vert_count, geom_tri_start, geom_tri_count;
    std::vector<float> geom_data, geom_friction, geom_restitution;
    std::vector<uint32_t> hull_range;  // exact (hull_start, hull_count) per geom
    // materials
    std::vector<float> mat_albedo, mat_roughness, mat_metallic, mat_emission,
        mat_ior, mat_density;
    std::vector<uint32_t> tri_geom;  // built on request (seevr_scene_array)
    // hull + support lookup
    std::vector<float> hull_verts;
    std::vector<uint32_t> support_offset, support_lookup;
    uint32_t num_support_entries = 0;
    uint32_t placement_failures = 0;  // generator placements left overlapping
    // scenes
    std::vector<uint32_t> scene_starts{0};
    std::vector<uint32_t> scene_offsets_view;

    uint32_t num_bodies() const { return uint32_t(body_inv_mass.size()); }
    uint32_t num_geoms() const { return uint32_t(geom_body_idx.size()); }
    uint32_t num_hull_verts() const { return uint32_t(hull_verts.size() / 3); }
    uint32_t num_vertices() const { return uint32_t(orig_verts.size() / 3); }
    uint32_t num_triangles() const { return uint32_t(indices.size() / 3); }

    // Data.buildSupportLookup (data.zig:299-353)
    void build_support_lookup(uint32_t gi, uint32_t hull_start, uint32_t hull_count) {
        if (support_offset.size() <= gi) support_offset.resize(gi + 1, 0);
        if (hull_count <= kSupportThreshold) {
            support_offset[gi] = 0;
            return;
        }
        const uint32_t entry_start = num_support_entries == 0 ? 1u : num_support_entries;
        support_offset[gi] = entry_start;
        if (support_lookup.size() < entry_start + kSupportEntry)
            support_lookup.resize(entry_start + kSupportEntry, 0);
        static const float perps[3][2][3] = {
            {{0, 1, 0}, {0, 0, 1}},  // X axis
            {{1, 0, 0}, {0, 0, 1}},  // Y axis
            {{1, 0, 0}, {0, 1, 0}},  // Z axis
        };
        const float pi_f = 3.14159265358979323846f;  // std.math.pi as f32
        const float* hv = hull_verts.data() + size_t(hull_start) * 3;
        for (uint32_t ax = 0; ax < kSupportAxes; ++ax) {
            const float* p1 = perps[ax][0];
            const float* p2 = perps[ax][1];
            for (uint32_t bin = 0; bin < kSupportBins; ++bin) {
                const float angle = float(bin) / float(kSupportBins) * 2.0f * pi_f;
                const float cos_a = std::cos(angle);
                const float sin_a = std::sin(angle);
                const float dx = cos_a * p1[0] + sin_a * p2[0];
                const float dy = cos_a * p1[1] + sin_a * p2[1];
                const float dz = cos_a * p1[2] + sin_a * p2[2];
                float best_dot = -1e10f;
                uint32_t best_idx = 0;
                for (uint32_t v = 0; v < hull_count; ++v) {
                    const float d = dx * hv[v * 3 + 0] + dy * hv[v * 3 + 1] + dz * hv[v * 3 + 2];
                    if (d > best_dot) {
                        best_dot = d;
                        best_idx = v;
                    }
                }
                support_lookup[entry_start + ax * kSupportBins + bin] = best_idx;
            }
        }
        num_support_entries = entry_start + kSupportEntry;
    }

    void push_body(const float c[3], float inv_mass, const float inertia[3], const float inv_inertia[3]) {
        body_pos.insert(body_pos.end(), c, c + 3);
        const float q[4] = {0, 0, 0, 1};
        body_quat.insert(body_quat.end(), q, q + 4);
        for (int k = 0; k < 3; ++k) {
            body_vel.push_back(0.f);
            body_omega.push_back(0.f);
            body_inertia.push_back(inertia[k]);
            body_inv_inertia.push_back(inv_inertia[k]);
        }
        body_inv_mass.push_back(inv_mass);
        body_vert_start.push_back(0);
        body_vert_count.push_back(0);
    }

    void push_geom(int32_t type, uint32_t bi, uint32_t hv, uint32_t hc, float friction,
                   float restitution, uint32_t material, uint32_t vs, uint32_t vc,
                   uint32_t ts, uint32_t tc) {
        geom_type.push_back(type);
        geom_body_idx.push_back(bi);
        const float gd[8] = {float(hv), float(hc), 0, 0, 0, 0, 0, 0};
        geom_data.insert(geom_data.end(), gd, gd + 8);
        hull_range.push_back(hv);
        hull_range.push_back(hc);
        geom_friction.push_back(friction);
        geom_restitution.push_back(restitution);
        geom_material.push_back(material);
        geom_vert_start.push_back(vs);
        geom_vert_count.push_back(vc);
        geom_tri_start.push_back(ts);
        geom_tri_count.push_back(tc);
        // Data.upload derives body vert start/count from the first geom of
        // each body (data.zig:633-638)
        body_vert_start[bi] = vs;
        body_vert_count[bi] = vc;
    }

    float density(uint32_t material) const {
        return material < mat_density.size() ? mat_density[material] : 0.f;
    }

    // Data.addBox (data.zig:392-485)
    uint32_t add_box(const float center[3], const float half[3], const float color[3],
                     float friction, float restitution, uint32_t material) {
        const uint32_t vs = num_vertices(), ts = num_triangles(), bi = num_bodies(),
                       gi = num_geoms();
        const float box_v[8][3] = {
            {-half[0], -half[1], -half[2]}, {half[0], -half[1], -half[2]},
            {half[0], half[1], -half[2]},   {-half[0], half[1], -half[2]},
            {-half[0], -half[1], half[2]},  {half[0], -half[1], half[2]},
            {half[0], half[1], half[2]},    {-half[0], half[1], half[2]},
        };
        static const uint32_t box_f[12][3] = {
            {0, 2, 1}, {0, 3, 2}, {5, 7, 4}, {5, 6, 7}, {4, 3, 0}, {4, 7, 3},
            {1, 6, 5}, {1, 2, 6}, {3, 6, 2}, {3, 7, 6}, {4, 1, 5}, {4, 0, 1},
        };
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 3; ++j) {
                orig_verts.push_back(box_v[i][j]);
                vertices.push_back(center[j] + box_v[i][j]);
                colors.push_back(color[j]);
            }
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 3; ++j) indices.push_back(vs + box_f[i][j]);

        const float dens = density(material);
        const float volume = half[0] * 2 * half[1] * 2 * half[2] * 2;
        const float mass = dens * volume;
        float inertia[3] = {0, 0, 0}, inv_inertia[3] = {0, 0, 0};
        if (mass > 0) {
            const float wx = half[0] * 2, wy = half[1] * 2, wz = half[2] * 2;
            inertia[0] = mass / 12.0f * (wy * wy + wz * wz);
            inertia[1] = mass / 12.0f * (wx * wx + wz * wz);
            inertia[2] = mass / 12.0f * (wx * wx + wy * wy);
            for (int k = 0; k < 3; ++k) inv_inertia[k] = 1.0f / inertia[k];
        }
        push_body(center, mass > 0 ? 1.0f / mass : 0.f, inertia, inv_inertia);

        const uint32_t hv = num_hull_verts();
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 3; ++j) hull_verts.push_back(box_v[i][j]);
        push_geom(2, bi, hv, 8, friction, restitution, material, vs, 8, ts, 12);
        build_support_lookup(gi, hv, 8);
        return bi;
    }

    // Data.addSphere (data.zig:487-597)
    uint32_t add_sphere(const float center[3], float radius, const float color[3],
                        uint32_t segments, float friction, float restitution,
                        uint32_t material) {
        const uint32_t vs = num_vertices(), ts = num_triangles(), bi = num_bodies(),
                       gi = num_geoms();
        const float pi = 3.14159265f;
        const float two_pi = 6.2831853f;  // comptime 2.0*pi coerced to f32
        const uint32_t num_v = (segments + 1) * (segments + 1);
        const uint32_t num_t = segments * segments * 2;
        const float segs = float(segments);
        for (uint32_t i_ = 0; i_ <= segments; ++i_) {
            const float i = float(i_);
            const float lat = pi * i / segs;
            const float sin_lat = std::sin(lat);
            const float cos_lat = std::cos(lat);
            for (uint32_t j_ = 0; j_ <= segments; ++j_) {
                const float j = float(j_);
                const float lon = two_pi * j / segs;
                const float lx = radius * std::cos(lon) * sin_lat;
                const float ly = radius * cos_lat;
                const float lz = radius * std::sin(lon) * sin_lat;
                const float l[3] = {lx, ly, lz};
                for (int k = 0; k < 3; ++k) {
                    orig_verts.push_back(l[k]);
                    vertices.push_back(center[k] + l[k]);
                    colors.push_back(color[k]);
                }
            }
        }
        for (uint32_t i_ = 0; i_ < segments; ++i_)
            for (uint32_t j_ = 0; j_ < segments; ++j_) {
                const uint32_t cur = vs + i_ * (segments + 1) + j_;
                const uint32_t nxt = cur + segments + 1;
                const uint32_t t[6] = {cur, nxt, cur + 1, cur + 1, nxt, nxt + 1};
                indices.insert(indices.end(), t, t + 6);
            }
        const float dens = density(material);
        const float pi_val = 3.14159265f;
        const float four_thirds = float(4.0 / 3.0);
        const float volume = four_thirds * pi_val * radius * radius * radius;
        const float mass = dens * volume;
        float inertia[3] = {0, 0, 0}, inv_inertia[3] = {0, 0, 0};
        if (mass > 0) {
            const float in = 0.4f * mass * radius * radius;
            for (int k = 0; k < 3; ++k) {
                inertia[k] = in;
                inv_inertia[k] = 1.0f / in;
            }
        }
        push_body(center, mass > 0 ? 1.0f / mass : 0.f, inertia, inv_inertia);

        const uint32_t hv = num_hull_verts();
        hull_verts.insert(hull_verts.end(), orig_verts.begin() + size_t(vs) * 3,
                          orig_verts.begin() + size_t(vs + num_v) * 3);
        push_geom(1, bi, hv, num_v, friction, restitution, material, vs, num_v, ts, num_t);
        build_support_lookup(gi, hv, num_v);
        return bi;
    }

    // Convex hull body.  Faces: every triple whose plane has all other
    // points on one side (exact hull for points in general position).
    uint32_t add_hull(const float center[3], const float* pts, uint32_t n, const float color[3],
                      float friction, float restitution, uint32_t material) {
        const uint32_t vs = num_vertices(), ts = num_triangles(), bi = num_bodies(),
                       gi = num_geoms();
        for (uint32_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                orig_verts.push_back(pts[i * 3 + k]);
                vertices.push_back(center[k] + pts[i * 3 + k]);
                colors.push_back(color[k]);
            }
        std::vector<uint32_t> faces;
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = i + 1; j < n; ++j)
                for (uint32_t k = j + 1; k < n; ++k) {
                    const double ax = pts[j * 3] - pts[i * 3], ay = pts[j * 3 + 1] - pts[i * 3 + 1],
                                 az = pts[j * 3 + 2] - pts[i * 3 + 2];
                    const double bx = pts[k * 3] - pts[i * 3], by = pts[k * 3 + 1] - pts[i * 3 + 1],
                                 bz = pts[k * 3 + 2] - pts[i * 3 + 2];
                    const double nx = ay * bz - az * by, ny = az * bx - ax * bz,
                                 nz = ax * by - ay * bx;
                    int pos = 0, neg = 0;
                    for (uint32_t m = 0; m < n && !(pos && neg); ++m) {
                        if (m == i || m == j || m == k) continue;
                        const double d = nx * (pts[m * 3] - pts[i * 3]) +
                                         ny * (pts[m * 3 + 1] - pts[i * 3 + 1]) +
                                         nz * (pts[m * 3 + 2] - pts[i * 3 + 2]);
                        if (d > 1e-12) pos = 1;
                        else if (d < -1e-12) neg = 1;
                    }
                    if (pos && neg) continue;
                    if (!pos) faces.insert(faces.end(), {vs + i, vs + j, vs + k});
                    else faces.insert(faces.end(), {vs + i, vs + k, vs + j});
                }
        indices.insert(indices.end(), faces.begin(), faces.end());
        const uint32_t num_t = uint32_t(faces.size() / 3);
        // Data.meshVolume (data.zig:374-390)
        float vol = 0;
        for (uint32_t t = 0; t < num_t; ++t) {
            const float* v0 = pts + (faces[t * 3] - vs) * 3;
            const float* v1 = pts + (faces[t * 3 + 1] - vs) * 3;
            const float* v2 = pts + (faces[t * 3 + 2] - vs) * 3;
            const float cx = v1[1] * v2[2] - v1[2] * v2[1];
            const float cy = v1[2] * v2[0] - v1[0] * v2[2];
            const float cz = v1[0] * v2[1] - v1[1] * v2[0];
            vol += v0[0] * cx + v0[1] * cy + v0[2] * cz;
        }
        const float volume = std::fabs(vol) / 6.0f;
        const float mass = density(material) * volume;
        float inertia[3] = {0, 0, 0}, inv_inertia[3] = {0, 0, 0};
        if (mass > 0) {
            const float r_eq = std::cbrt(3.0f * volume / (4.0f * 3.14159265f));
            const float in = 0.4f * mass * r_eq * r_eq;
            for (int k = 0; k < 3; ++k) {
                inertia[k] = in;
                inv_inertia[k] = 1.0f / in;
            }
        }
        push_body(center, mass > 0 ? 1.0f / mass : 0.f, inertia, inv_inertia);
        const uint32_t hv = num_hull_verts();
        hull_verts.insert(hull_verts.end(), pts, pts + size_t(n) * 3);
        push_geom(3, bi, hv, n, friction, restitution, material, vs, n, ts, num_t);
        build_support_lookup(gi, hv, n);
        return bi;
    }

    // Append another builder's bodies as new scenes, rebasing every index
    // (materials of `o` must equal this builder's).
    void merge(const seevr_scene& o) {
        const uint32_t vs = num_vertices(), bi = num_bodies(), hv = num_hull_verts();
        const uint32_t gi0 = num_geoms();
        auto app = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
        app(vertices, o.vertices);
        app(colors, o.colors);
        app(orig_verts, o.orig_verts);
        for (uint32_t x : o.indices) indices.push_back(x + vs);
        app(body_pos, o.body_pos);
        app(body_quat, o.body_quat);
        app(body_vel, o.body_vel);
        app(body_omega, o.body_omega);
        app(body_inv_mass, o.body_inv_mass);
        app(body_inertia, o.body_inertia);
        app(body_inv_inertia, o.body_inv_inertia);
        for (uint32_t x : o.body_vert_start) body_vert_start.push_back(x + vs);
        app(body_vert_count, o.body_vert_count);
        app(geom_type, o.geom_type);
        for (uint32_t x : o.geom_body_idx) geom_body_idx.push_back(x + bi);
        app(geom_material, o.geom_material);
        for (uint32_t x : o.geom_vert_start) geom_vert_start.push_back(x + vs);
        app(geom_vert_count, o.geom_vert_count);
        const uint32_t ts = num_triangles() - o.num_triangles();
        for (uint32_t x : o.geom_tri_start) geom_tri_start.push_back(x + ts);
        app(geom_tri_count, o.geom_tri_count);
        for (size_t g = 0; g < o.hull_range.size() / 2; ++g) {
            const uint32_t st = o.hull_range[g * 2] + hv, ct = o.hull_range[g * 2 + 1];
            hull_range.push_back(st);
            hull_range.push_back(ct);
            const float gd[8] = {float(st), float(ct), 0, 0, 0, 0, 0, 0};
            geom_data.insert(geom_data.end(), gd, gd + 8);
        }
        app(geom_friction, o.geom_friction);
        app(geom_restitution, o.geom_restitution);
        app(hull_verts, o.hull_verts);
        // support lookup: o's entries live at [1, o.nse); rebase to `base`
        const uint32_t base = num_support_entries == 0 ? 1u : num_support_entries;
        support_offset.resize(gi0, 0);
        for (uint32_t x : o.support_offset) support_offset.push_back(x ? x - 1 + base : 0);
        if (o.num_support_entries > 1) {
            support_lookup.resize(base, 0);
            support_lookup.insert(support_lookup.end(), o.support_lookup.begin() + 1,
                                  o.support_lookup.begin() + o.num_support_entries);
            num_support_entries = base + (o.num_support_entries - 1);
        }
        for (uint32_t st : o.scene_starts)
            if (scene_starts.back() != st + bi) scene_starts.push_back(st + bi);
        placement_failures += o.placement_failures;
    }

    uint32_t add_material(const float albedo[3], float roughness, float metallic,
                          const float emission[3], float ior, float dens) {
        const uint32_t mi = uint32_t(mat_density.size());
        mat_albedo.insert(mat_albedo.end(), albedo, albedo + 3);
        mat_roughness.push_back(roughness);
        mat_metallic.push_back(metallic);
        mat_emission.insert(mat_emission.end(), emission, emission + 3);
        mat_ior.push_back(ior);
        mat_density.push_back(dens);
        return mi;
    }

    void begin() {
        if (scene_starts.back() != num_bodies()) scene_starts.push_back(num_bodies());
    }
    uint32_t num_scenes() const {
        return uint32_t(scene_starts.size());
    }
    void swap_out(seevr_scene& o) { std::swap(*this, o); }
    uint32_t num_dynamic() const {
        uint32_t n = 0;
        for (float im : body_inv_mass) n += im > 0.f;
        return n;
    }
};

namespace {

const float kGrey[3] = {0.35f, 0.35f, 0.30f};
const float kRed[3] = {0.85f, 0.15f, 0.15f};
const float kBlue[3] = {0.2f, 0.4f, 0.9f};
const float kZero3[3] = {0, 0, 0};

struct Mats {
    uint32_t ground, body;
};

Mats default_materials(seevr_scene* s) {
    Mats m;
    m.ground = s->add_material(kGrey, 0.95f, 0.f, kZero3, 0.f, 0.f);
    m.body = s->add_material(kRed, 0.4f, 0.f, kZero3, 0.f, 1000.f);
    return m;
}

void random_unit_points(SplitMix64& rng, uint32_t n, float scale, std::vector<float>& out) {
    out.resize(size_t(n) * 3);
    for (uint32_t i = 0; i < n; ++i) {
        double x, y, z, l;
        do {
            x = rng.normal();
            y = rng.normal();
            z = rng.normal();
            l = std::sqrt(x * x + y * y + z * z);
        } while (l < 1e-9);
        out[i * 3 + 0] = float(x / l * scale);
        out[i * 3 + 1] = float(y / l * scale);
        out[i * 3 + 2] = float(z / l * scale);
    }
}

// Rejection placement.  A new body may not overlap an earlier one (exact
// oriented-box / sphere tests with a 2 cm margin; hulls use their bounding
// sphere) nor reach below the ground top y = 0.  Up to 256 draws, then the
// last draw is kept.  Deep initial overlaps would otherwise be resolved by
// the unclamped Baumgarte bias of physics.comp:520 as an explosion.
struct PlacedShape {
    double c[3];
    double ax[3][3];  // local axes in world space (rotation columns)
    double h[3];      // box half extents
    double r;         // sphere radius (or bounding radius)
    bool box;
};

struct Placer {
    static constexpr double kMargin = 0.02;
    double cell;
    std::vector<PlacedShape> shapes;
    std::unordered_map<int64_t, std::vector<uint32_t>> grid;
    uint32_t& failures;  // draws that ended overlapping (volume too dense)
    Placer(double cell_size, uint32_t& fail_count) : cell(cell_size), failures(fail_count) {}
    static int64_t key(int64_t x, int64_t y, int64_t z) {
        return ((x & 0x1FFFFF) << 42) | ((y & 0x1FFFFF) << 21) | (z & 0x1FFFFF);
    }
    static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
    static bool box_sphere(const PlacedShape& b, const PlacedShape& s) {
        double d2 = 0;
        for (int k = 0; k < 3; ++k) {
            const double t[3] = {s.c[0] - b.c[0], s.c[1] - b.c[1], s.c[2] - b.c[2]};
            const double p = dot3(t, b.ax[k]);
            const double q = std::min(std::max(p, -b.h[k]), b.h[k]);
            d2 += (p - q) * (p - q);
        }
        const double rr = s.r + kMargin;
        return d2 < rr * rr;
    }
    // separating-axis test over the 15 candidate axes of two boxes
    static bool box_box(const PlacedShape& A, const PlacedShape& B) {
        const double T[3] = {B.c[0] - A.c[0], B.c[1] - A.c[1], B.c[2] - A.c[2]};
        auto separated = [&](const double* L) {
            const double l2 = dot3(L, L);
            if (l2 < 1e-12) return false;
            double ra = 0, rb = 0;
            for (int k = 0; k < 3; ++k) {
                ra += A.h[k] * std::fabs(dot3(A.ax[k], L));
                rb += B.h[k] * std::fabs(dot3(B.ax[k], L));
            }
            return std::fabs(dot3(T, L)) > ra + rb + kMargin * std::sqrt(l2);
        };
        for (int i = 0; i < 3; ++i)
            if (separated(A.ax[i]) || separated(B.ax[i])) return false;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double* a = A.ax[i];
                const double* b = B.ax[j];
                const double L[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                                     a[0] * b[1] - a[1] * b[0]};
                if (separated(L)) return false;
            }
        return true;
    }
    static bool overlap(const PlacedShape& a, const PlacedShape& b) {
        const double e[3] = {a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]};
        const double ra = a.box ? std::sqrt(dot3(a.h, a.h)) : a.r;
        const double rb = b.box ? std::sqrt(dot3(b.h, b.h)) : b.r;
        const double rr = ra + rb + kMargin;
        if (dot3(e, e) >= rr * rr) return false;
        if (a.box && b.box) return box_box(a, b);
        if (a.box) return box_sphere(a, b);
        if (b.box) return box_sphere(b, a);
        return true;
    }
    static double lowest_y(const PlacedShape& s) {
        if (!s.box) return s.c[1] - s.r;
        return s.c[1] - (s.h[0] * std::fabs(s.ax[0][1]) + s.h[1] * std::fabs(s.ax[1][1]) +
                         s.h[2] * std::fabs(s.ax[2][1]));
    }
    bool free(const PlacedShape& s) const {
        if (lowest_y(s) < 0.01) return false;
        const int64_t cx = int64_t(std::floor(s.c[0] / cell)), cy = int64_t(std::floor(s.c[1] / cell)),
                      cz = int64_t(std::floor(s.c[2] / cell));
        for (int64_t dx = -1; dx <= 1; ++dx)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dz = -1; dz <= 1; ++dz) {
                    auto it = grid.find(key(cx + dx, cy + dy, cz + dz));
                    if (it == grid.end()) continue;
                    for (uint32_t i : it->second)
                        if (overlap(shapes[i], s)) return false;
                }
        return true;
    }
    // Draw a center in [lo, hi) per axis for a box (half h) or sphere /
    // hull (bounding radius r) with orientation q (xyzw).
    void place(SplitMix64& rng, const double lo[3], const double hi[3], bool box, const float h[3],
               float r, const float q[4], float c[3]) {
        PlacedShape s{};
        s.box = box;
        s.r = r;
        for (int k = 0; k < 3; ++k) s.h[k] = box ? h[k] : 0.0;
        const double x = q[0], y = q[1], z = q[2], w = q[3];
        const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                                {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                                {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j) s.ax[k][j] = R[j][k];
        bool placed = false;
        for (int attempt = 0; attempt < 256 && !placed; ++attempt) {
            for (int k = 0; k < 3; ++k) c[k] = float(rng.uniform(lo[k], hi[k]));
            for (int k = 0; k < 3; ++k) s.c[k] = c[k];
            placed = free(s);
        }
        failures += placed ? 0u : 1u;
        shapes.push_back(s);
        grid[key(int64_t(std::floor(s.c[0] / cell)), int64_t(std::floor(s.c[1] / cell)),
                 int64_t(std::floor(s.c[2] / cell)))]
            .push_back(uint32_t(shapes.size() - 1));
    }
};

// One pile scene: static ground box, then bodies alternating box/sphere.
// Per body the stream draws: size, orientation, position(s), then the
// optional velocities and friction.
const double kPileLo[3] = {-5.0, 1.0, -5.0}, kPileHi[3] = {5.0, 21.0, 5.0};

void gen_pile_scene(seevr_scene* s, SplitMix64& rng, uint32_t n_boxes, uint32_t n_spheres,
                    uint32_t segments, const Mats& m, bool random_vel, bool random_mu,
                    const double lo[3] = kPileLo, const double hi[3] = kPileHi) {
    s->begin();
    const float gc[3] = {0.f, -0.25f, 0.f}, gh[3] = {50.f, 0.25f, 50.f};
    s->add_box(gc, gh, kGrey, 0.5f, 0.2f, m.ground);
    Placer placer(2.5, s->placement_failures);
    uint32_t nb = 0, ns = 0;
    while (nb < n_boxes || ns < n_spheres) {
        const bool box = (nb < n_boxes) && (ns >= n_spheres || nb <= ns);
        float c[3], q[4], h[3] = {0, 0, 0}, r = 0;
        uint32_t b;
        if (box) {
            for (int k = 0; k < 3; ++k) h[k] = float(rng.uniform(0.2, 0.6));
        } else {
            r = float(rng.uniform(0.2, 0.5));
        }
        rng.quat(q);
        placer.place(rng, lo, hi, box, h, r, q, c);
        if (box) {
            b = s->add_box(c, h, kRed, 0.5f, 0.2f, m.body);
            ++nb;
        } else {
            b = s->add_sphere(c, r, kBlue, segments, 0.5f, 0.2f, m.body);
            ++ns;
        }
        std::memcpy(&s->body_quat[size_t(b) * 4], q, sizeof q);
        if (random_vel) {
            for (int k = 0; k < 3; ++k) s->body_vel[size_t(b) * 3 + k] = float(rng.normal());
            for (int k = 0; k < 3; ++k) s->body_omega[size_t(b) * 3 + k] = float(rng.normal());
        }
        if (random_mu) s->geom_friction[b] = float(rng.uniform(0.2, 0.8));
    }
}

}  // namespace

extern "C" {

seevr_scene* seevr_scene_create(void) { return new seevr_scene(); }
void seevr_scene_destroy(seevr_scene* s) { delete s; }
void seevr_scene_begin(seevr_scene* s) { s->begin(); }

uint32_t seevr_scene_add_material(seevr_scene* s, const float albedo[3], float roughness,
                                  float metallic, const float emission[3], float ior,
                                  float density) {
    return s->add_material(albedo, roughness, metallic, emission, ior, density);
}

uint32_t seevr_scene_add_box(seevr_scene* s, const float center[3], const float half[3],
                             const float color[3], float friction, float restitution,
                             uint32_t material) {
    return s->add_box(center, half, color, friction, restitution, material);
}

uint32_t seevr_scene_add_sphere(seevr_scene* s, const float center[3], float radius,
                                const float color[3], uint32_t segments, float friction,
                                float restitution, uint32_t material) {
    return s->add_sphere(center, radius, color, segments, friction, restitution, material);
}

uint32_t seevr_scene_add_hull(seevr_scene* s, const float center[3], const float* points,
                              uint32_t count, const float color[3], float friction,
                              float restitution, uint32_t material) {
    return s->add_hull(center, points, count, color, friction, restitution, material);
}

void seevr_scene_set_body_quat(seevr_scene* s, uint32_t b, const float q[4]) {
    std::memcpy(&s->body_quat[size_t(b) * 4], q, 4 * sizeof(float));
}

void seevr_scene_set_body_vel(seevr_scene* s, uint32_t b, const float v[3], const float w[3]) {
    if (v) std::memcpy(&s->body_vel[size_t(b) * 3], v, 3 * sizeof(float));
    if (w) std::memcpy(&s->body_omega[size_t(b) * 3], w, 3 * sizeof(float));
}

void seevr_scene_set_geom_friction(seevr_scene* s, uint32_t g, float mu) {
    s->geom_friction[g] = mu;
}

void seevr_scene_gen_pile(seevr_scene* s, uint64_t seed, uint32_t n_boxes, uint32_t n_spheres,
                          uint32_t segments) {
    SplitMix64 rng(seed);
    const Mats m = default_materials(s);
    gen_pile_scene(s, rng, n_boxes, n_spheres, segments, m, false, false);
}

void seevr_scene_gen_pile_in(seevr_scene* s, uint64_t seed, uint32_t n_boxes, uint32_t n_spheres,
                             uint32_t segments, const float lo[3], const float hi[3]) {
    SplitMix64 rng(seed);
    const Mats m = default_materials(s);
    const double l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
    gen_pile_scene(s, rng, n_boxes, n_spheres, segments, m, false, false, l, h);
}

void seevr_scene_gen_large(seevr_scene* s, uint64_t seed, uint32_t n_bodies, uint32_t segments) {
    SplitMix64 rng(seed);
    const Mats m = default_materials(s);
    s->begin();
    const float gc[3] = {0.f, -0.25f, 0.f}, gh[3] = {40.f, 0.25f, 40.f};
    s->add_box(gc, gh, kGrey, 0.5f, 0.2f, m.ground);
    std::vector<float> pts;
    Placer placer(2.5, s->placement_failures);
    const double lo[3] = {-32.0, 1.0, -32.0}, hi[3] = {32.0, 65.0, 32.0};
    for (uint32_t i = 0; i < n_bodies; ++i) {
        const double kind = rng.uniform();
        float c[3], q[4], h[3] = {0, 0, 0}, r = 0;
        uint32_t b;
        if (kind < 0.4) {
            for (int k = 0; k < 3; ++k) h[k] = float(rng.uniform(0.2, 0.6));
            rng.quat(q);
            placer.place(rng, lo, hi, true, h, 0.f, q, c);
            b = s->add_box(c, h, kRed, 0.5f, 0.2f, m.body);
        } else if (kind < 0.8) {
            r = float(rng.uniform(0.2, 0.5));
            rng.quat(q);
            placer.place(rng, lo, hi, false, h, r, q, c);
            b = s->add_sphere(c, r, kBlue, segments, 0.5f, 0.2f, m.body);
        } else {
            const uint32_t n = 16 + uint32_t(rng.uniform() * 17.0);  // 16..32
            const float scale = float(rng.uniform(0.2, 0.6));
            random_unit_points(rng, n > 32 ? 32 : n, scale, pts);
            rng.quat(q);
            placer.place(rng, lo, hi, false, h, scale, q, c);
            b = s->add_hull(c, pts.data(), uint32_t(pts.size() / 3), kGrey, 0.5f, 0.2f, m.body);
        }
        std::memcpy(&s->body_quat[size_t(b) * 4], q, sizeof q);
        for (int k = 0; k < 3; ++k) s->body_vel[size_t(b) * 3 + k] = float(rng.normal());
    }
}

// Scenes are generated independently (one splitmix64 stream per scene,
// seeded seed_base + scene) into private builders, then merged in order, so
// the result does not depend on the thread count.
static void gen_many(seevr_scene* s, uint32_t num_scenes, uint64_t seed_base,
                     uint32_t min_bodies, uint32_t max_bodies, uint32_t segments,
                     bool rollout, const uint64_t* seeds = nullptr) {
    const Mats m = default_materials(s);
    std::vector<seevr_scene> parts(num_scenes);
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t sc = 0; sc < int64_t(num_scenes); ++sc) {
        seevr_scene& p = parts[size_t(sc)];
        default_materials(&p);
        SplitMix64 rng(seeds ? seeds[sc] : seed_base + uint64_t(sc));
        uint32_t n = max_bodies;
        if (!rollout) {
            const double lo = std::log(double(min_bodies)), hi = std::log(double(max_bodies));
            n = uint32_t(std::lround(std::exp(rng.uniform(lo, hi))));
            n = std::min(std::max(n, min_bodies), max_bodies);
        }
        gen_pile_scene(&p, rng, (n + 1) / 2, n / 2, segments, m, rollout, rollout);
    }
    for (uint32_t sc = 0; sc < num_scenes; ++sc) {
        s->begin();
        s->merge(parts[sc]);
        seevr_scene().swap_out(parts[sc]);
    }
}

void seevr_scene_gen_batch(seevr_scene* s, uint32_t num_scenes, uint32_t min_bodies,
                           uint32_t max_bodies, uint32_t segments, uint64_t seed_base) {
    gen_many(s, num_scenes, seed_base, min_bodies, max_bodies, segments, false);
}

void seevr_scene_gen_batch_seeds(seevr_scene* s, const uint64_t* seeds, uint32_t num_scenes,
                                 uint32_t min_bodies, uint32_t max_bodies, uint32_t segments) {
    if (!seeds || num_scenes == 0) return;
    gen_many(s, num_scenes, 0, min_bodies, max_bodies, segments, false, seeds);
}

void seevr_scene_gen_rollout(seevr_scene* s, uint32_t num_scenes, uint32_t bodies,
                             uint32_t segments, uint64_t seed_base) {
    gen_many(s, num_scenes, seed_base, bodies, bodies, segments, true);
}

void seevr_scene_gen_towers(seevr_scene* s, uint64_t seed, uint32_t towers, uint32_t height,
                            float spacing) {
    seevr_scene_gen_towers_stacked(s, seed, towers, height, spacing, 0.0f);
}

void seevr_scene_gen_towers_stacked(seevr_scene* s, uint64_t seed, uint32_t towers,
                                    uint32_t height, float spacing, float overlap) {
    SplitMix64 rng(seed);
    const Mats m = default_materials(s);
    s->begin();
    uint32_t side = 1;
    while (side * side < towers) ++side;
    const float extent = 0.5f * float(side) * spacing + 5.f;
    const float gc[3] = {0.f, -0.25f, 0.f}, gh[3] = {extent, 0.25f, extent};
    s->add_box(gc, gh, kGrey, 0.6f, 0.f, m.ground);
    const float half[3] = {0.5f, 0.5f, 0.5f};
    for (uint32_t t = 0; t < towers; ++t) {
        const float tx = (float(t % side) - 0.5f * float(side - 1)) * spacing;
        const float tz = (float(t / side) - 0.5f * float(side - 1)) * spacing;
        for (uint32_t k = 0; k < height; ++k) {
            float c[3];
            c[0] = tx + float(0.01 * rng.normal());
            c[1] = 0.5f - overlap + float(k) * (1.0f - overlap);
            c[2] = tz + float(0.01 * rng.normal());
            s->add_box(c, half, kRed, 0.6f, 0.f, m.body);
        }
    }
}

void* seevr_scene_array(seevr_scene* s, int id) {
    switch (id) {
        case SEEVR_S_BODY_POS: return s->body_pos.data();
        case SEEVR_S_BODY_QUAT: return s->body_quat.data();
        case SEEVR_S_BODY_VEL: return s->body_vel.data();
        case SEEVR_S_BODY_OMEGA: return s->body_omega.data();
        case SEEVR_S_BODY_INV_MASS: return s->body_inv_mass.data();
        case SEEVR_S_BODY_INV_INERTIA: return s->body_inv_inertia.data();
        case SEEVR_S_BODY_VERT_START: return s->body_vert_start.data();
        case SEEVR_S_BODY_VERT_COUNT: return s->body_vert_count.data();
        case SEEVR_S_GEOM_BODY_IDX: return s->geom_body_idx.data();
        case SEEVR_S_GEOM_DATA: return s->geom_data.data();
        case SEEVR_S_GEOM_FRICTION: return s->geom_friction.data();
        case SEEVR_S_GEOM_RESTITUTION: return s->geom_restitution.data();
        case SEEVR_S_HULL_VERTS: return s->hull_verts.data();
        case SEEVR_S_VERTICES: return s->vertices.data();
        case SEEVR_S_ORIG_VERTICES: return s->orig_verts.data();
        case SEEVR_S_SUPPORT_OFFSET: return s->support_offset.data();
        case SEEVR_S_SUPPORT_LOOKUP:
            if (s->support_lookup.empty()) s->support_lookup.assign(1, 0);
            return s->support_lookup.data();
        case SEEVR_S_INDICES: return s->indices.data();
        case SEEVR_S_BODY_INERTIA: return s->body_inertia.data();
        case SEEVR_S_GEOM_TYPE: return s->geom_type.data();
        case SEEVR_S_SCENE_BODY_OFFSET:
            s->scene_offsets_view = s->scene_starts;
            s->scene_offsets_view.push_back(s->num_bodies());
            return s->scene_offsets_view.data();
        case SEEVR_S_COLORS: return s->colors.data();
        case SEEVR_S_HULL_RANGE: return s->hull_range.data();
        case SEEVR_S_GEOM_MATERIAL: return s->geom_material.data();
        case SEEVR_S_TRI_GEOM: {
            // triangle -> geom, from each geom's triangle range (data.zig:642-652)
            s->tri_geom.assign(s->num_triangles(), 0u);
            for (uint32_t g = 0; g < s->geom_tri_start.size(); ++g)
                for (uint32_t t = 0; t < s->geom_tri_count[g]; ++t)
                    s->tri_geom[s->geom_tri_start[g] + t] = g;
            return s->tri_geom.data();
        }
        case SEEVR_S_MAT_ALBEDO: return s->mat_albedo.data();
        case SEEVR_S_MAT_ROUGHNESS: return s->mat_roughness.data();
        case SEEVR_S_MAT_METALLIC: return s->mat_metallic.data();
        case SEEVR_S_MAT_EMISSION: return s->mat_emission.data();
        case SEEVR_S_MAT_IOR: return s->mat_ior.data();
        default: return nullptr;
    }
}

uint64_t seevr_scene_count(const seevr_scene* s, int id) {
    switch (id) {
        case SEEVR_C_BODIES: return s->num_bodies();
        case SEEVR_C_GEOMS: return s->num_geoms();
        case SEEVR_C_HULL_VERTS: return s->num_hull_verts();
        case SEEVR_C_VERTICES: return s->num_vertices();
        case SEEVR_C_TRIANGLES: return s->num_triangles();
        case SEEVR_C_SUPPORT_ENTRIES:
            return s->num_support_entries ? s->num_support_entries : 1;
        case SEEVR_C_SCENES: return s->num_scenes();
        case SEEVR_C_MATERIALS: return s->mat_density.size();
        case SEEVR_C_DYNAMIC_BODIES: return s->num_dynamic();
        case SEEVR_C_PLACEMENT_FAILURES: return s->placement_failures;
        default: return 0;
    }
}

// ---- binary scene file --------------------------------------------------
// header: magic "SEEVRSC1", u32 array count, then per array: u32 id, u64
// byte length, bytes.  Arrays not listed load as empty.
}  // extern "C"
namespace {
template <class T>
void put_vec(FILE* f, uint32_t id, const std::vector<T>& v) {
    const uint64_t n = uint64_t(v.size()) * sizeof(T);
    std::fwrite(&id, 4, 1, f);
    std::fwrite(&n, 8, 1, f);
    if (n) std::fwrite(v.data(), 1, n, f);
}
template <class T>
bool get_vec(FILE* f, uint64_t n, std::vector<T>& v) {
    if (n % sizeof(T)) return false;
    v.resize(n / sizeof(T));
    return n == 0 || std::fread(v.data(), 1, n, f) == n;
}
}  // namespace
extern "C" {

int seevr_scene_save(const seevr_scene* s, const char* path) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return 1;
    std::fwrite("SEEVRSC1", 1, 8, f);
    const uint32_t count = 35;
    std::fwrite(&count, 4, 1, f);
    put_vec(f, 0, s->body_pos);
    put_vec(f, 1, s->body_quat);
    put_vec(f, 2, s->body_vel);
    put_vec(f, 3, s->body_omega);
    put_vec(f, 4, s->body_inv_mass);
    put_vec(f, 5, s->body_inv_inertia);
    put_vec(f, 6, s->body_vert_start);
    put_vec(f, 7, s->body_vert_count);
    put_vec(f, 8, s->geom_body_idx);
    put_vec(f, 9, s->geom_data);
    put_vec(f, 10, s->geom_friction);
    put_vec(f, 11, s->geom_restitution);
    put_vec(f, 12, s->hull_verts);
    put_vec(f, 13, s->vertices);
    put_vec(f, 14, s->orig_verts);
    put_vec(f, 15, s->support_offset);
    put_vec(f, 16, s->support_lookup);
    put_vec(f, 17, s->indices);
    put_vec(f, 18, s->body_inertia);
    put_vec(f, 19, s->geom_type);
    put_vec(f, 20, s->scene_starts);
    put_vec(f, 21, s->colors);
    put_vec(f, 22, s->geom_material);
    put_vec(f, 23, s->mat_density);
    put_vec(f, 24, s->geom_vert_start);
    put_vec(f, 25, s->geom_vert_count);
    const std::vector<uint32_t> nse{s->num_support_entries};
    put_vec(f, 26, nse);
    put_vec(f, 27, s->hull_range);
    put_vec(f, 28, s->geom_tri_start);
    put_vec(f, 29, s->geom_tri_count);
    put_vec(f, 30, s->mat_albedo);
    put_vec(f, 31, s->mat_roughness);
    put_vec(f, 32, s->mat_metallic);
    put_vec(f, 33, s->mat_emission);
    put_vec(f, 34, s->mat_ior);
    const int bad = std::ferror(f);
    std::fclose(f);
    return bad ? 1 : 0;
}

seevr_scene* seevr_scene_load(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return nullptr;
    char magic[8];
    uint32_t count = 0;
    seevr_scene* s = new seevr_scene();
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "SEEVRSC1", 8) == 0 &&
              std::fread(&count, 4, 1, f) == 1;
    std::vector<uint32_t> nse;
    for (uint32_t a = 0; ok && a < count; ++a) {
        uint32_t id;
        uint64_t n;
        ok = std::fread(&id, 4, 1, f) == 1 && std::fread(&n, 8, 1, f) == 1;
        if (!ok) break;
        switch (id) {
            case 0: ok = get_vec(f, n, s->body_pos); break;
            case 1: ok = get_vec(f, n, s->body_quat); break;
            case 2: ok = get_vec(f, n, s->body_vel); break;
            case 3: ok = get_vec(f, n, s->body_omega); break;
            case 4: ok = get_vec(f, n, s->body_inv_mass); break;
            case 5: ok = get_vec(f, n, s->body_inv_inertia); break;
            case 6: ok = get_vec(f, n, s->body_vert_start); break;
            case 7: ok = get_vec(f, n, s->body_vert_count); break;
            case 8: ok = get_vec(f, n, s->geom_body_idx); break;
            case 9: ok = get_vec(f, n, s->geom_data); break;
            case 10: ok = get_vec(f, n, s->geom_friction); break;
            case 11: ok = get_vec(f, n, s->geom_restitution); break;
            case 12: ok = get_vec(f, n, s->hull_verts); break;
            case 13: ok = get_vec(f, n, s->vertices); break;
            case 14: ok = get_vec(f, n, s->orig_verts); break;
            case 15: ok = get_vec(f, n, s->support_offset); break;
            case 16: ok = get_vec(f, n, s->support_lookup); break;
            case 17: ok = get_vec(f, n, s->indices); break;
            case 18: ok = get_vec(f, n, s->body_inertia); break;
            case 19: ok = get_vec(f, n, s->geom_type); break;
            case 20: ok = get_vec(f, n, s->scene_starts); break;
            case 21: ok = get_vec(f, n, s->colors); break;
            case 22: ok = get_vec(f, n, s->geom_material); break;
            case 23: ok = get_vec(f, n, s->mat_density); break;
            case 24: ok = get_vec(f, n, s->geom_vert_start); break;
            case 25: ok = get_vec(f, n, s->geom_vert_count); break;
            case 26: ok = get_vec(f, n, nse); break;
            case 27: ok = get_vec(f, n, s->hull_range); break;
            case 28: ok = get_vec(f, n, s->geom_tri_start); break;
            case 29: ok = get_vec(f, n, s->geom_tri_count); break;
            case 30: ok = get_vec(f, n, s->mat_albedo); break;
            case 31: ok = get_vec(f, n, s->mat_roughness); break;
            case 32: ok = get_vec(f, n, s->mat_metallic); break;
            case 33: ok = get_vec(f, n, s->mat_emission); break;
            case 34: ok = get_vec(f, n, s->mat_ior); break;
            default: ok = std::fseek(f, long(n), SEEK_CUR) == 0; break;
        }
    }
    std::fclose(f);
    const size_t nb = s->body_inv_mass.size();
    ok = ok && s->body_pos.size() == nb * 3 && s->body_quat.size() == nb * 4 &&
         s->geom_data.size() == s->geom_body_idx.size() * 8 && !s->scene_starts.empty();
    if (!ok) {
        delete s;
        return nullptr;
    }
    if (!nse.empty()) s->num_support_entries = nse[0];
    // files written before records 28-34 existed carry no triangle ranges
    if (s->geom_tri_start.size() != s->geom_body_idx.size() ||
        s->geom_tri_count.size() != s->geom_body_idx.size()) {
        s->geom_tri_start.assign(s->geom_body_idx.size(), 0);
        s->geom_tri_count.assign(s->geom_body_idx.size(), 0);
    }
    return s;
}

}  // extern "C"
