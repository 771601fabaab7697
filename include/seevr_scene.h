/*
 * seevr_scene.h — host-side scene builder of libseevr_cuda.
 *
 * Mirrors the CPU staging half of seeVR's Data (src/data.zig): the same SoA
 * arrays, filled by the same builders (addMaterial data.zig:356, addBox
 * data.zig:392, addSphere data.zig:487, buildSupportLookup data.zig:299),
 * plus addHull, which the reference lacks (convex hull of a point cloud).
 * Scenes can be concatenated into one batch; scene s owns bodies
 * [scene_body_offset[s], scene_body_offset[s+1]).
 *
 * The seeded generators build the benchmark workloads (ground box + boxes,
 * UV spheres and hulls) from one splitmix64 stream per scene.
 */
#ifndef SEEVR_SCENE_H
#define SEEVR_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct seevr_scene seevr_scene;

/* Array identifiers for seevr_scene_array(). */
enum seevr_scene_array_id {
    SEEVR_S_BODY_POS = 0,          /* f32 N*3 */
    SEEVR_S_BODY_QUAT = 1,         /* f32 N*4 */
    SEEVR_S_BODY_VEL = 2,          /* f32 N*3 */
    SEEVR_S_BODY_OMEGA = 3,        /* f32 N*3 */
    SEEVR_S_BODY_INV_MASS = 4,     /* f32 N   */
    SEEVR_S_BODY_INV_INERTIA = 5,  /* f32 N*3 */
    SEEVR_S_BODY_VERT_START = 6,   /* u32 N   */
    SEEVR_S_BODY_VERT_COUNT = 7,   /* u32 N   */
    SEEVR_S_GEOM_BODY_IDX = 8,     /* u32 G   */
    SEEVR_S_GEOM_DATA = 9,         /* f32 G*8 */
    SEEVR_S_GEOM_FRICTION = 10,    /* f32 G   */
    SEEVR_S_GEOM_RESTITUTION = 11, /* f32 G   */
    SEEVR_S_HULL_VERTS = 12,       /* f32 HV*3 */
    SEEVR_S_VERTICES = 13,         /* f32 V*3 */
    SEEVR_S_ORIG_VERTICES = 14,    /* f32 V*3 */
    SEEVR_S_SUPPORT_OFFSET = 15,   /* u32 G   */
    SEEVR_S_SUPPORT_LOOKUP = 16,   /* u32 num_support_entries */
    SEEVR_S_INDICES = 17,          /* u32 T*3 */
    SEEVR_S_BODY_INERTIA = 18,     /* f32 N*3 */
    SEEVR_S_GEOM_TYPE = 19,        /* i32 G (1 sphere, 2 box, 3 hull) */
    SEEVR_S_SCENE_BODY_OFFSET = 20,/* u32 num_scenes+1 */
    SEEVR_S_COLORS = 21,           /* f32 V*3 */
    SEEVR_S_HULL_RANGE = 22,       /* u32 G*2 exact (hull_start, hull_count) */
    /* path-tracer inputs (raytrace.comp bindings 9-15, data.zig:72, 104) */
    SEEVR_S_GEOM_MATERIAL = 23,    /* u32 G   material of each geom          */
    SEEVR_S_TRI_GEOM = 24,         /* u32 T   geom of each render triangle   */
    SEEVR_S_MAT_ALBEDO = 25,       /* f32 M*3 */
    SEEVR_S_MAT_ROUGHNESS = 26,    /* f32 M   */
    SEEVR_S_MAT_METALLIC = 27,     /* f32 M   */
    SEEVR_S_MAT_EMISSION = 28,     /* f32 M*3 */
    SEEVR_S_MAT_IOR = 29,          /* f32 M   0 = opaque, > 0 = glass        */
    SEEVR_S_NUM_ARRAYS = 30
};

enum seevr_scene_count_id {
    SEEVR_C_BODIES = 0,
    SEEVR_C_GEOMS = 1,
    SEEVR_C_HULL_VERTS = 2,
    SEEVR_C_VERTICES = 3,
    SEEVR_C_TRIANGLES = 4,
    SEEVR_C_SUPPORT_ENTRIES = 5,
    SEEVR_C_SCENES = 6,
    SEEVR_C_MATERIALS = 7,
    SEEVR_C_DYNAMIC_BODIES = 8,
    SEEVR_C_PLACEMENT_FAILURES = 9 /* generator draws left overlapping */
};

seevr_scene* seevr_scene_create(void);
void seevr_scene_destroy(seevr_scene* s);

/* Start a new independent scene; bodies added afterwards belong to it.  A
 * builder starts with one open scene. */
void seevr_scene_begin(seevr_scene* s);

/* Data.addMaterial (data.zig:356): returns the material index.  Density in
 * kg/m^3, 0 = static. */
uint32_t seevr_scene_add_material(seevr_scene* s, const float albedo[3],
                                  float roughness, float metallic,
                                  const float emission[3], float ior,
                                  float density);

/* Data.addBox (data.zig:392-485): returns the body index. */
uint32_t seevr_scene_add_box(seevr_scene* s, const float center[3],
                             const float half[3], const float color[3],
                             float friction, float restitution,
                             uint32_t material);

/* Data.addSphere (data.zig:487-597): UV sphere of (segments+1)^2 verts. */
uint32_t seevr_scene_add_sphere(seevr_scene* s, const float center[3],
                                float radius, const float color[3],
                                uint32_t segments, float friction,
                                float restitution, uint32_t material);

/* Convex hull of `count` local-space points (no reference counterpart; the
 * reference has only boxes and spheres).  Every point is kept as a hull
 * vertex; faces come from the exact convex hull.  Mass uses the hull
 * volume (tetrahedron fan, as Data.meshVolume data.zig:374-390), inertia
 * that of the sphere of equal volume. */
uint32_t seevr_scene_add_hull(seevr_scene* s, const float center[3],
                              const float* points, uint32_t count,
                              const float color[3], float friction,
                              float restitution, uint32_t material);

/* Overwrite a body's orientation (xyzw) or velocities after adding it. */
void seevr_scene_set_body_quat(seevr_scene* s, uint32_t body, const float q[4]);
void seevr_scene_set_body_vel(seevr_scene* s, uint32_t body, const float v[3],
                              const float w[3]);
void seevr_scene_set_geom_friction(seevr_scene* s, uint32_t geom, float mu);

/* Seeded workloads (splitmix64).  See seevr_b200/scenes.py for the
 * distributions.  Each call appends one or more scenes. */
void seevr_scene_gen_pile(seevr_scene* s, uint64_t seed, uint32_t n_boxes,
                          uint32_t n_spheres, uint32_t segments);
/* Same distributions, spawned in the box [lo, hi] instead of
 * x,z in [-5,5], y in [1,21]. */
void seevr_scene_gen_pile_in(seevr_scene* s, uint64_t seed, uint32_t n_boxes,
                             uint32_t n_spheres, uint32_t segments,
                             const float lo[3], const float hi[3]);
void seevr_scene_gen_large(seevr_scene* s, uint64_t seed, uint32_t n_bodies,
                           uint32_t segments);
void seevr_scene_gen_batch(seevr_scene* s, uint32_t num_scenes,
                           uint32_t min_bodies, uint32_t max_bodies,
                           uint32_t segments, uint64_t seed_base);
/* The scenes of seevr_scene_gen_batch whose seeds are listed: seeds
 * {k0, k1, ...} give scenes k0, k1, ... of the batch generated with
 * seed_base 0 (each scene has its own stream, seeded with its number). */
void seevr_scene_gen_batch_seeds(seevr_scene* s, const uint64_t* seeds,
                                 uint32_t num_scenes, uint32_t min_bodies,
                                 uint32_t max_bodies, uint32_t segments);
void seevr_scene_gen_rollout(seevr_scene* s, uint32_t num_scenes,
                             uint32_t bodies, uint32_t segments,
                             uint64_t seed_base);
void seevr_scene_gen_towers(seevr_scene* s, uint64_t seed, uint32_t towers,
                            uint32_t height, float spacing);
/* Towers of unit boxes (half-extent 0.5) on a static ground: `towers`
 * stacks of `height` boxes on a square grid `spacing` apart, x and z
 * jittered N(0, 0.01) m, friction 0.6, no restitution.  Each box sinks
 * `overlap` metres into the one below (the lowest into the ground), so every
 * stack contact exists from the first substep; overlap 0 gives boxes that
 * just touch (seevr_scene_gen_towers), whose contacts appear only as the
 * boxes below settle. */
void seevr_scene_gen_towers_stacked(seevr_scene* s, uint64_t seed, uint32_t towers,
                                    uint32_t height, float spacing, float overlap);

/* Views of the staging arrays (valid until the next add/gen call). */
void* seevr_scene_array(seevr_scene* s, int array_id);
uint64_t seevr_scene_count(const seevr_scene* s, int count_id);

/* Binary scene file (a dump of the arrays above with a small header). */
int seevr_scene_save(const seevr_scene* s, const char* path);
seevr_scene* seevr_scene_load(const char* path);

#ifdef __cplusplus
}
#endif
#endif /* SEEVR_SCENE_H */
