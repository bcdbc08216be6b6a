/* Test infrastructure, not product code: the CPU oracle of the path-trace pass.
 *
 * A statement-by-statement C++ restatement of ThreeRT's offline path-trace kernel (renderer/shaders/pathtrace.wgsl
 * `main` with LIVE = false, APPROX = 0, FEAT = F_INST), its two-level software walk (renderer/shaders/trace_units.wgsl)
 * and its sampler (renderer/shaders/sample.wgsl). It reads exactly the buffers the CUDA pass is given (the reference's
 * vertices / leaves / nodes / tables / words heaps, the RGBA16F environment texels and the 624-byte Params block) and
 * writes the same 80-byte `Pixel` records (renderer/shaders/records.wgsl `Pixel`).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library, and only as the checker or
 * the timed CPU baseline. Nothing in the product links or calls it.
 */
#ifndef THREERT_ORACLE_H
#define THREERT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const float* vertices;   /* vec4s, 3 per vertex: (position, u), (normal, v), (tangent, hand) */
    uint64_t n_vertex_vec4;
    const float* leaves;     /* vec4s, 3 per triangle: (v0, section bits), (e1, rank bits), (e2, 0) */
    uint64_t n_leaf_vec4;
    const uint32_t* nodes;   /* GpuNode, 8 words each */
    uint64_t n_nodes;
    const uint32_t* tables;  /* vec4 heap (words) */
    uint64_t n_table_vec4;
    const uint32_t* words;   /* word heap */
    uint64_t n_words;
    const uint16_t* env_half; /* RGBA16F texels, env_w * env_h * 4 halves */
    uint32_t env_w, env_h;
} orc_scene;

typedef struct {
    uint64_t closest_rays;   /* closest-hit traces */
    uint64_t shadow_rays;    /* shadow / any-hit traces */
    uint64_t node_visits;    /* nodes read by the walk (both levels) */
    uint64_t tri_tests;      /* triangle tests */
    uint64_t unit_entries;   /* instance records read on entering a unit */
} orc_stats;

/* One ray cast: o, d, tmax, mode (0 closest, 1 shadow, 2 any). Output per ray: t, tri, u, v, inst, part. */
typedef struct { float o[3]; float tmax; float d[3]; uint32_t mode; } orc_ray;
typedef struct { float t; uint32_t tri; float u; float v; uint32_t inst; uint32_t part; } orc_hit;

/* Renders samples [first_sample, first_sample + spp) into `accum` (w * h Pixel records of 20 floats, accumulated onto
 * what is there). `params` is the 156-word Params block. `threads` <= 0: every hardware thread. */
int orc_render(const orc_scene* s, const uint32_t* params, uint32_t first_sample, uint32_t spp, float* accum,
               int threads, orc_stats* stats);
/* Renders only the pixels listed in `pixels` (pixel indices), for bounded-sample timing. */
int orc_render_pixels(const orc_scene* s, const uint32_t* params, uint32_t first_sample, uint32_t spp,
                      const uint32_t* pixels, uint64_t n_pixels, float* accum, int threads, orc_stats* stats);
/* The reference walk (trace_units) on each ray. */
int orc_trace(const orc_scene* s, const uint32_t* params, const orc_ray* rays, uint64_t n, orc_hit* hits,
              int threads, orc_stats* stats);
/* Brute force over every unit's triangles (what the walk must equal), closest or any. */
int orc_trace_brute(const orc_scene* s, const uint32_t* params, const orc_ray* rays, uint64_t n, orc_hit* hits,
                    int threads);
/* The t of one named triangle (of instance which[i].inst) along each ray, in the unit's space as the walk tests it. */
int orc_intersect(const orc_scene* s, const uint32_t* params, const orc_ray* rays, const orc_hit* which, uint64_t n,
                  float* t_out);
/* The per-frame deformation (deform.cpp), one job a mesh: 8 words (first vertex, vertices, first corner, palette's
 * first matrix, first triangle, triangles, tree root, tree nodes). Corners: 16 floats each (skin.wgsl Corner); palette:
 * 12 floats a matrix (three rows). skin.wgsl main over each job's vertices, in place: */
int orc_skin(const uint32_t* jobs, uint32_t n_jobs, const float* corners, const float* palette, float* vertices);
/* leaf_gather.wgsl main over each job's triangles, in place (w_indices: the Indices section's first word): */
int orc_leaf_gather(const uint32_t* jobs, uint32_t n_jobs, const float* vertices, const uint32_t* words,
                    uint32_t w_indices, float* leaves);
/* units.rs:251-275 refit of each job's tree from the vertices, in place: */
int orc_refit(const uint32_t* jobs, uint32_t n_jobs, const float* vertices, const uint32_t* words, uint32_t w_indices,
              uint32_t* nodes);
/* The denoiser fallback (denoise.cpp): denoise.rs over the Frame of w * h Pixel records (20 floats each), `iterations`
 * a-trous passes; w * h RGB floats out. */
int orc_denoise(const float* accum, uint32_t w, uint32_t h, uint32_t iterations, float* rgb);
/* sample.wgsl rng4 for a pixel seed, an index and a dimension id (tests pin the sampler with it). */
void orc_rng4(uint32_t pixel_seed, uint32_t index, uint32_t dim, float out[4]);
/* The Sobol direction numbers (3 dimensions x 32, bit-reversed) the sampler's tables hold. */
void orc_sobol_directions(uint32_t out[96]);
uint32_t orc_hash_hp(uint32_t x);
int orc_hardware_threads(void);

#ifdef __cplusplus
}
#endif
#endif
