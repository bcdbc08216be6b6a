/* threert_b200 host prep: a scene description in, the reference's packed buffers out.
 *
 * What ThreeRT's `prepare_as` (renderer/src/lib.rs:530-789) makes of a scene under software traversal, restated in
 * C++: the mesh trees (renderer/src/bvh.rs:81-239 binned SAH; renderer/src/units.rs:231-248 `mesh_tree`), the units'
 * top tree (units.rs:140-224 `build_sah`, 303-326 `top_tree`, 288-300 `UnitBox::new`), the unit records
 * (scene.rs:239-247 `Instance::gpu`, units.rs:329-342 `unit_record`), shared vertices and leaves (indexed.rs:12-28),
 * the instances' rows (scene.rs:96-117), the emitter list, its CDF, guide table and header (lib.rs:190-214, 437-489),
 * the light tree (ltree.rs:405-470), the GGX energy table (lib.rs:1041-1104), the sky bake and its CDF (lib.rs:916-944,
 * sky.rs:941-975), the table / word heaps (heap.rs:127-135) and the 624-byte Params block (gpu.rs:127-186).
 *
 * The output is exactly what `trt_scene_upload` (threert_cuda.h) takes, so a caller that builds scenes some other way
 * (the reference's own Rust prep) hands over the same buffers.
 */
#ifndef THREERT_PREP_H
#define THREERT_PREP_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A mesh: triangles in model space, three corners each. */
typedef struct {
    uint32_t n_tris;
    const float* positions;  /* n_tris * 9 */
    const float* normals;    /* n_tris * 9, or NULL: each triangle's own normal at its corners */
    const float* uvs;        /* n_tris * 6, or NULL: zeros */
    const uint32_t* sections;/* n_tris section indices, or NULL: all in section 0 */
    uint32_t n_sections;     /* at least 1 */
    uint32_t like;           /* 1 + an earlier mesh this one repeats (its own vertices, leaves and tree, copied from
                              * that mesh's instead of built: the fields above are then not read); 0: none */
} trt_mesh_spec;

/* A metal-rough material (scene.rs:480-491 GpuMaterial's fields the pass reads). */
typedef struct {
    float base_color[4];
    float emissive[3];       /* nits */
    float metallic, roughness, specular;
    int32_t card;            /* 1: a rect light's card (MAT_EMITTER_CARD), lit on its front alone */
} trt_material_spec;

/* An instance: a mesh placed by a 3x4 row-major world matrix, with a material per section of the mesh. */
typedef struct {
    uint32_t mesh;
    uint32_t object;
    float world[12];
    const uint32_t* section_materials; /* the mesh's n_sections material indices */
    uint32_t cast_shadow;
} trt_instance_spec;

/* A directional light (scene.rs:1315-1331 gpu_light): the direction light travels, its colour x illuminance (lux). */
typedef struct {
    float dir[3];
    float color[3];
    float intensity;
    float angular_diameter_deg;
    uint32_t cast_shadow;
    float specular_scale;
} trt_dirlight_spec;

/* The sky: 0 none (black), 1 a uniform colour (nits), 2 a gradient bake (sky.rs:941-975: zenith, horizon, ground),
 * 3 the atmosphere (sky.rs:643), baked on the device: the prep reserves a black width x height map for it. */
typedef struct {
    uint32_t kind;
    float color[3];
    float zenith[3], horizon[3], ground[3];
    uint32_t width, height;  /* bake size for kind 2 (the reference bakes 1024 x 512) */
} trt_sky_spec;

typedef struct {
    float position[3], forward[3], right[3], up[3];
    float tan_half_fov;      /* of the vertical field of view */
    uint32_t width, height;
    float lens_radius, focus_distance;
} trt_camera_spec;

/* The render preset (the preset JSON files' "native" block; gpu.rs:1971-1976 set_preset). */
typedef struct {
    uint32_t max_bounces, rr_depth;
    float clamp_indirect;    /* the firefly clamp at the exposure used */
    float energy_compensation;
} trt_preset_spec;

typedef struct {
    uint32_t n_meshes;
    const trt_mesh_spec* meshes;
    uint32_t n_materials;
    const trt_material_spec* materials;
    uint32_t n_instances;
    const trt_instance_spec* instances;
    uint32_t n_objects;
    const float* object_power; /* n_objects, or NULL: 1 */
    uint32_t n_lights;
    const trt_dirlight_spec* lights;
    trt_sky_spec sky;
    trt_camera_spec camera;
    trt_preset_spec preset;
    uint32_t seed;             /* Params.size.w (lib.rs:312-315: 0x5eed by default) */
    uint32_t use_light_tree;   /* 1: as THREERT_LTREE unset; 0: the CDF alone */
} trt_scene_spec;

/* The packed buffers (the boundary's input; threert_cuda.h trt_scene_desc has the same fields). */
typedef struct {
    const float* vertices;   uint64_t vertices_bytes;
    const float* leaves;     uint64_t leaves_bytes;
    const uint32_t* nodes;   uint64_t nodes_bytes;
    const uint32_t* tables;  uint64_t tables_bytes;
    const uint32_t* words;   uint64_t words_bytes;
    const uint16_t* env_half; uint32_t env_w, env_h;
} trt_prepared_buffers;

typedef struct trt_prepared trt_prepared;

/* 0 on success; on failure a message in `trt_prep_last_error`. */
int trt_prep_build(const trt_scene_spec* spec, trt_prepared** out);
void trt_prep_free(trt_prepared* p);
/* A baked sky as the prep packs it (lib.rs:916-944 build_env_cdf, lib.rs:1013 sky_brightest): RGBA16F texels (w * h
 * * 4 halves, or NULL), the CDF (h + w * h floats, or NULL) and the brightest luminance (or NULL) of w * h RGBA f32
 * texels. 0 on success. */
int trt_prep_env(const float* texels, uint32_t w, uint32_t h, uint16_t* env_half, float* cdf, float* brightest);
void trt_prep_buffers(const trt_prepared* p, trt_prepared_buffers* out);
/* The 156-word Params block with `size.z` (the sample index) 0. */
void trt_prep_params(const trt_prepared* p, uint32_t out[156]);
/* Facts the tests check: units, mesh nodes, top tree's first node, emitters, light tree nodes. */
typedef struct {
    uint32_t n_units, top_first, n_nodes, n_tris, n_vertices, n_emitters, light_tree_nodes, env_sampled;
    uint32_t max_mesh_depth, top_depth;
    float emitter_total, env_nee_floor;
} trt_prep_info;
void trt_prep_get_info(const trt_prepared* p, trt_prep_info* out);
/* The light tree's per-entry codes and order (ltree.rs LightTree::code / order), for the prep's own tests. */
uint32_t trt_prep_light_tree(const trt_prepared* p, uint32_t* order, uint32_t* codes, uint32_t cap);
const char* trt_prep_last_error(void);

/* The binned-SAH tree over triangles (bvh.rs:81-98 build_tris), for the builder's tests: nodes (8 words each) and
 * the order; returns the node count (0 on failure), writes the depth. */
uint32_t trt_prep_bvh(const float* tris, uint32_t n_tris, uint32_t max_depth, uint32_t* nodes, uint32_t nodes_cap,
                      uint32_t* order, uint32_t* depth);
/* bvh.rs:246-285 check_tree over a tree's nodes with leaves of at most max_leaf items among n_items. 0 if it holds. */
int trt_prep_check_tree(const uint32_t* nodes, uint32_t n_nodes, uint32_t max_depth, uint32_t max_leaf,
                        uint32_t n_items, uint32_t* depth);
/* Unit records for instances placed anew (scene.rs:239-247 Instance::gpu with units.rs:329-342 unit_record), to write
 * over the tables' instance section with trt_scene_update before trt_deform: worlds n * 12 floats (3x4 row-major),
 * info n * 4 words (first triangle, object, first vertex, rows' first), roots n tree roots, cast_shadow n flags;
 * out n * 40 words. 0 on success. */
int trt_prep_unit_records(uint32_t n, const float* worlds, const uint32_t* info, const uint32_t* roots,
                          const uint32_t* cast_shadow, uint32_t* out);
/* The top tree over n units (units.rs:303-326 top_tree over units.rs:288-300 UnitBox::new of each unit's model-space
 * box, local_boxes n * 6 floats lo then hi, under its world rows): (2n - 1) * 8 words of nodes, a leaf's
 * left_or_first its unit's index. What trt_deform builds on the device. 0 on success; *depth the tree's depth. */
int trt_prep_units_top(uint32_t n, const float* worlds, const float* local_boxes, uint32_t* nodes, uint32_t* depth);
/* lib.rs:1041-1083 specular_albedo (f64), for the energy table's tests. */
void trt_prep_specular_albedo(double mu, double alpha, uint32_t nr, uint32_t nphi, double out[2]);

#ifdef __cplusplus
}
#endif
#endif
