/* threert_b200: the B200 path-trace pass behind a C ABI.
 *
 * The drop-in for ThreeRT's offline path-trace pass under software traversal: the buffers `Gpu::render` uploads
 * (renderer/src/gpu.rs:4116-4236, upload at gpu.rs:2613) go in as plain pointers and byte counts, the per-sample
 * dispatch loop of renderer/shaders/pathtrace.wgsl `main` (gpu.rs:4174-4196) runs as a wavefront of sm_100a kernels,
 * and the 80-byte `Pixel` records of `accum` (renderer/shaders/records.wgsl `Pixel`; gpu.rs:4211-4232 reads them)
 * come back. Every function returns 0 on success and a nonzero TRT_E* code otherwise; `trt_last_error` has the
 * message (the reference returns anyhow::Result, gpu.rs:4116).
 *
 * Threading: one context per host thread; a context owns one CUDA stream, and every call on a context and its
 * scenes is ordered on that stream.
 */
#ifndef THREERT_CUDA_H
#define THREERT_CUDA_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TRT_OK = 0,
    TRT_EINVAL = 1,    /* a bad argument: sizes, offsets, counts past their buffers */
    TRT_ECUDA = 2,     /* a CUDA call failed (out of device memory, no device) */
    TRT_EGUARD = 3,    /* a traversal gave up at its iteration limit: the scene's trees are not trees */
};

#define TRT_PARAMS_WORDS 156 /* Params: 39 vec4s, 624 bytes (gpu.rs:127-186) */
#define TRT_PIXEL_FLOATS 20  /* Pixel: color, albedo, normal, emit, spec (records.wgsl) */

typedef struct trt_ctx trt_ctx;
typedef struct trt_scene trt_scene;

typedef struct {
    int device;          /* CUDA device ordinal */
    uint32_t flags;      /* 0 */
} trt_options;

/* The scene's buffers as the reference binds them (pathtrace.wgsl:141-268): vertices (binding 1), leaves (2), nodes
 * (3), tables (4), words (5), the environment texels (9, RGBA16F, env_w x env_h). Copied to the device; the library
 * owns the copies. Replaces `Gpu::upload` (gpu.rs:2613). */
typedef struct {
    const void* vertices; uint64_t vertices_bytes;
    const void* leaves;   uint64_t leaves_bytes;
    const void* nodes;    uint64_t nodes_bytes;
    const void* tables;   uint64_t tables_bytes;
    const void* words;    uint64_t words_bytes;
    const uint16_t* env_half; uint32_t env_w, env_h;
} trt_scene_desc;

/* What one render did (gpu.rs:4197 trace_ms and the ray counts the reference does not keep). */
typedef struct {
    uint64_t closest_rays;   /* extend rays traced (camera + bounce) */
    uint64_t shadow_rays;    /* shadow / any-hit rays traced */
    uint64_t paths;          /* pixels x samples */
    float device_ms;         /* device time of the call, CUDA events on the context's stream */
    uint32_t launches;       /* kernels launched */
    uint32_t guard_trips;    /* traversals stopped at the iteration limit (pathtrace.wgsl's loop guard) */
} trt_stats;

/* Cumulative counters of a scene since `trt_scene_reset_totals` (reads them with one synchronisation). */
typedef struct {
    uint64_t closest_rays, shadow_rays, paths, renders, launches;
    /* Filled by renders (and traces) with TRT_RENDER_COUNT, for the closest-hit walks and the shadow walks: node
     * records read (a binary walk reads a node and, at an interior node, both children), triangles tested, unit
     * records entered. */
    uint64_t node_visits, tri_tests, unit_entries;
    uint64_t shadow_node_visits, shadow_tri_tests, shadow_unit_entries;
    double extend_ms, shadow_ms, shade_ms;          /* with trt_scene_set_profiling on: per-stage device time */
    uint64_t extend_launches, shadow_launches;
    uint64_t guard_trips;
    double sort_ms;                                 /* with profiling on: the coherence sorts' device time */
} trt_totals;

/* One ray for trt_trace: origin, tmax, direction, mode (0 closest, 1 shadow casters, 2 any surface). */
typedef struct { float o[3]; float tmax; float d[3]; uint32_t mode; } trt_ray;
typedef struct { float t; uint32_t tri; float u; float v; uint32_t inst; uint32_t part; } trt_hit;

/* Render flags. */
#define TRT_RENDER_ACCUMULATE 1u /* add to accum instead of clearing it first (resume at first_sample) */
#define TRT_RENDER_COUNT      2u /* also count node visits, triangle tests and unit entries (a slower walk) */
#define TRT_RENDER_WIDE       4u /* walk the 8-wide quantised BVH instead of the reference's binary trees */
/* Coherence sorts on the device, per depth; the image does not depend on them, bit for bit. trt_render sorts hits by
 * material before shading when the scene has more than TRT_SORT_HITS_MIN_MATERIALS materials (measured: the city's
 * 4,201 and the crowd's 217 gain 3-10 %, the Cornell box's 4 loses 14 %), unless this flag is given; a server sorts
 * every step's hits unless its options' flags hold it: */
#define TRT_RENDER_UNSORTED_HITS 16u
#define TRT_SORT_HITS_MIN_MATERIALS 32u
/* Optional, measured slower on the city scene: secondary rays by (queue chunk, direction octant) before the
 * closest-hit walk, shadow rays by (position chunk, direction octant) in each light class before the shadow walk. */
#define TRT_RENDER_SORT_RAYS      8u
/* Also sum each sample's first-hit distance (0 where the camera ray escapes) into x of the Pixel's fourth vec4, which
 * the offline reference leaves zero: the denoisers' depth guide (mean = x / count). */
#define TRT_RENDER_DEPTH         64u
#define TRT_RENDER_SORT_SHADOWS  32u
/* With accum_host: the call returns once the render is queued, and the accum's copy to accum_host (which must be
 * pinned memory, left untouched until then) runs on the context's copy stream while the next render, into the scene's
 * other accum, runs; trt_synchronize (or trt_timer_stop) waits for the copies too. Not with TRT_RENDER_ACCUMULATE. */
#define TRT_RENDER_ASYNC_READBACK 128u

int trt_create(const trt_options* opts, trt_ctx** out);
/* Frees the context and every scene still uploaded through it (their handles are then invalid). */
void trt_destroy(trt_ctx* ctx);
const char* trt_last_error(const trt_ctx* ctx);
/* The library's version and the device it runs on (name, SM count). */
int trt_device_info(const trt_ctx* ctx, char* name, size_t name_len, int* sm_count);

/* Uploads a scene (gpu.rs:2613 Gpu::upload). Its wide BVH is built from the uploaded trees at the first render or
 * trace that asks for it (TRT_RENDER_WIDE), and again after an update to the nodes, leaves or tables. */
int trt_scene_upload(trt_ctx* ctx, const trt_scene_desc* desc, trt_scene** out);
void trt_scene_free(trt_scene* scene);
/* Overwrites bytes [offset, offset + bytes) of one of the scene's buffers (0 vertices, 1 leaves, 2 nodes, 3 tables,
 * 4 words) from host memory: in-place record edits and refits (gpu.rs:4028 write_nodes). */
int trt_scene_update(trt_scene* scene, uint32_t which, uint64_t offset, const void* src, uint64_t bytes);

/* Copies bytes [offset, offset + bytes) of one of the scene's buffers (numbered as for trt_scene_update; 5: the
 * environment's RGBA16F texels, 8 bytes each) to host memory: what a deformation or a sky bake wrote, for checks. */
int trt_scene_read(trt_scene* scene, uint32_t which, uint64_t offset, void* dst, uint64_t bytes);

/* The denoiser fallback on the scene's last accum (renderer/src/denoise.rs `denoise`, what main.rs:548-557 runs
 * when OIDN is absent): the Frame of each Pixel (gpu.rs:4219-4232), demodulated by the albedo, `iterations` a-trous
 * passes (4 in the reference) guided by albedo, normal and the 3 x 3-filtered variance, modulated again. Writes
 * w * h RGB floats to rgb_host; ms (may be NULL): the device time of the filter. */
int trt_denoise_atrous(trt_scene* scene, uint32_t iterations, float* rgb_host, float* ms);

/* ---- The atmosphere's sky baked on the device (renderer/src/sky.rs:643-819 bake_atmosphere /
 * bake_atmosphere_tables, with the tables of Luts::build, sky.rs:386-433): the environment map the pass samples, for
 * prep without a CPU bake and for re-baking a scene's sky in place when its sun moves. */
typedef struct {
    float sun_dir[3];        /* toward the sun (world, Y up; any length) */
    float sun_lux[3];        /* the sun's illuminance above the atmosphere: colour x intensity (lux) */
    float rayleigh_scale, mie_scale, mie_g;
    float ground_albedo[3];
    float altitude_m;        /* the viewer's altitude: the camera's height, or the planet's (planet = 1) */
    uint32_t planet;         /* 0: a flat world's horizon (sky.rs Horizon::Level); 1: a planet's, dipped */
    float glow_uniform[3];   /* the night sky's glow (sky.rs Glow), nits */
    float glow_horizon[3];
    float glow_height;       /* radians to 1/e */
    float cloud_cover;       /* 0..1: the overcast blend (sky.rs:775-811) */
    uint32_t width, height;  /* the bake: 1024 x 512 (lib.rs:966), 256 x 128 for a moving sun (sky.rs:633) */
} trt_atmosphere;

typedef struct {
    float sun_illuminance[3];  /* lux at the ground: the atmosphere's sun light's colour (lib.rs:682-684) */
    float horizon_v;           /* a planet's limb row (Params.sky_color.w), 0 otherwise */
    float brightest;           /* the bake's brightest luminance (lib.rs:1013 sky_brightest); trt_scene_set_sky only */
    float tables_ms;           /* device time of the tables (0 when those of the same atmosphere were reused) */
    float bake_ms;             /* device time of the bake (and, for trt_scene_set_sky, of the texels and CDF) */
} trt_sky_result;

/* Bakes on the ctx's device. texels_host: NULL or width * height * 4 floats (RGBA f32, equirect, row 0 the zenith);
 * tables_host: NULL or TRT_SKY_TABLE_FLOATS floats (the sun's optical depth 128 x 257 x 3, the scattered light
 * 32 x 64 x 3, the ground's 64 x 3). The tables are kept and reused while the atmosphere (scales, anisotropy, ground
 * albedo) stays the same. */
#define TRT_SKY_TABLE_FLOATS (3 * (257 * 128 + 64 * 32 + 64))
int trt_sky_bake(trt_ctx* ctx, const trt_atmosphere* atm, float* texels_host, float* tables_host, trt_sky_result* out);
/* Bakes into a scene's environment in place: its RGBA16F texels, its CDF (the words' first section, lib.rs:916-941),
 * the colour of light `sun_light` (-1: none) in the tables, and in params: env (1, w, h), sky_color.w and
 * counts2.y (the sky light-sampled when its brightest luminance reaches env_nee_floor, lib.rs:1005-1021). The
 * scene's environment must already be width x height (its prep reserved it). */
int trt_scene_set_sky(trt_scene* scene, const trt_atmosphere* atm, int32_t sun_light, float env_nee_floor,
                      uint32_t params[TRT_PARAMS_WORDS], trt_sky_result* out);

/* The light list's weights made again on the device (renderer/shaders/emitter_weights.wgsl, run by gpu.rs:3219
 * weigh_emitters): each emitter's weight from its record, instance, material and object power as the tables hold
 * them now, the cumulative table and its guide, the light tree's node powers (tree_nodes of them, 0: no tree) and the
 * header. After edits of object powers, materials or emitter records (trt_scene_update). lod: NULL, or the light
 * LOD's reference point and d0 (on when d0 > 0); cull: NULL, or radius, far distance, cone cosine, cone direction
 * (6 floats). ms (may be NULL): device time. */
int trt_scene_weigh_emitters(trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t tree_nodes,
                             const float* lod, const float* cull, float* ms);

/* The light tree built again on the device (renderer/src/ltree.rs:405-470 build: the emitters of positive power that
 * are neither nominal nor moving, one a leaf, median splits along the widest axis of their centroids; lib.rs:393-418:
 * the emitter table put in the tree's leaf order, the others after it, each triangle's code) from the emitter records
 * as the tables hold them now: after emitters moved (their records written). params: its light-tree words are set
 * (the tree's entries; the candidates resampled at camera hits); *tree_nodes: the tree's nodes (0: no tree, below 256
 * such emitters). Then trt_scene_weigh_emitters(scene, params, *tree_nodes, ...) makes the nodes' powers, the CDF and
 * the header. At most 16,384 emitters in the tree; ms (may be NULL): device time. */
int trt_scene_build_light_tree(trt_scene* scene, uint32_t params[TRT_PARAMS_WORDS], uint32_t* tree_nodes, float* ms);

/* ---- The learned denoiser (no counterpart in the reference, whose learned denoiser is the external OIDN library,
 * renderer/src/denoise.rs:80-103): a 4-level U-Net (32 / 64 / 96 / 128 channels, 3 x 3 convolutions, 2 x 2 average
 * pooling, nearest upsampling, skip concatenations) on bf16 tensor cores with f32 accumulation; its training (forward,
 * backward, Adam) runs on the device too. Input a pixel: log1p(radiance * s), albedo, normal, log1p(depth * sd),
 * log1p(variance of the mean luminance * s^2) (11 floats; s = 1 / the image's mean luminance, sd = 1 / its mean
 * first-hit distance); output: log1p(radiance * s). */
typedef struct trt_unet trt_unet;
/* A network for batches of up to max_batch images of up to max_h x max_w (multiples of 8) on `device`. */
int trt_unet_create(int device, uint32_t max_batch, uint32_t max_h, uint32_t max_w, trt_unet** out);
void trt_unet_destroy(trt_unet* net);
const char* trt_unet_last_error(const trt_unet* net);
/* Parameters (f32) in the network's layout: per layer, weights [9][cin padded to 32][cout padded to 64] then the bias
 * (cout padded to 64); the layers in order e0a e0b e1a e1b e2a e2b e3a e3b d2a d2b d1a d1b d0a d0b out. Setting them
 * resets the optimiser. */
uint64_t trt_unet_param_count(void);
int trt_unet_set_params(trt_unet* net, const float* params);
int trt_unet_get_params(trt_unet* net, float* params);
/* features: b * h * w * 11 floats (NHWC); pred: b * h * w * 3. ms (may be NULL): device time of the network. */
int trt_unet_forward(trt_unet* net, const float* features, uint32_t b, uint32_t h, uint32_t w, float* pred, float* ms);
/* One step of training on (features, targets = log1p(reference radiance * s)): the L1 loss's gradient by the
 * backward pass, then (update != 0) an Adam step at rate lr. loss, grads (param_count floats), ms: may be NULL. */
int trt_unet_train_step(trt_unet* net, const float* features, const float* targets, uint32_t b, uint32_t h, uint32_t w,
                        float lr, int update, float* loss, float* grads, float* ms);
/* Denoises a rendered accum in device memory (w * h Pixel records with TRT_RENDER_DEPTH's depth; trt_accum_device_ptr)
 * into w * h RGB floats: features, network and output transform all on the device. */
int trt_unet_denoise_accum(trt_unet* net, const void* accum_device, uint32_t w, uint32_t h, float* rgb_host, float* ms);
/* For tests of the error path: the next convolution of the next trt_unet_forward or trt_unet_denoise_accum withholds
 * one of its copies, so that the pipeline's bounded wait (about a second) runs out. That call returns TRT_ECUDA with
 * the message of a wait that gave up, and the network stays usable. */
int trt_unet_hold_next_load(trt_unet* net);

/* ---- Scenes that move: the per-frame deformation, on the device ----
 * The reference poses skinned meshes with two shaders (renderer/shaders/skin.wgsl, leaf_gather.wgsl), refits their
 * mesh trees on the CPU (units.rs:251-275 refit, live/edits.rs:2395-2450) and builds the top tree on the CPU
 * (units.rs:303-326 top_tree through Kept::top, units.rs:771-830; written by gpu.rs:4014 Gpu::retop). Here all of it
 * runs on the scene's stream: skinning, leaf gather, a bottom-up refit of each deforming mesh's tree, the units' world
 * boxes (units.rs:288-300 UnitBox::new) and the top tree built again over all units by the same binned SAH
 * (units.rs:140-224 build_sah), laid out as that build lays it out.
 *
 * The units are the instances 0 .. Params.motion.w - 1 (one a top-tree leaf, as trt_prep_build lays scenes out) and
 * the top tree's 2 * units - 1 nodes start at Params.motion.z. A unit's world box comes from its record in the tables
 * (its world rows and its tree's root, n0.w) and its tree's root box: move units by writing their records
 * (trt_scene_update, trt_prep_unit_records) before trt_deform. */

/* A corner of a skinned model (skin.wgsl Corner): position, w the bits of its first two palette indices (16 bits
 * each, low first); normal, w the other two; tangent, w the bits of TRT_CORNER_* flags; the four weights. */
typedef struct { float p[4], n[4], t[4], w[4]; } trt_corner;
#define TRT_CORNER_NORMAL  1u
#define TRT_CORNER_TANGENT 2u

/* A mesh that deforms (skin.wgsl and leaf_gather.wgsl Job, with its tree): its vertices among the scene's and the
 * corner of the first (one corner a vertex, in the vertices' order), the first matrix of its palette, its triangles
 * (leaves; indices in the words' Indices section, counted from first_vertex), its tree's root node and node count. */
typedef struct {
    uint32_t first_vertex, n_vertices, first_corner, palette;
    uint32_t first_tri, n_tris, root, n_nodes;
} trt_deform_mesh;

typedef struct {
    const trt_corner* corners;
    uint64_t n_corners;
    const trt_deform_mesh* meshes;
    uint32_t n_meshes;
} trt_deform_desc;

/* Device times of one deformation (filled when stats is given: the call then waits for it) and the errors the device
 * found (a tree that is not one, a top tree that came out deeper than TOP_DEPTH; bit 16: the wide BVH's refit met an
 * index out of its buffers). wide_ms: the wide BVH's refit (0 when the scene has none built), after device_ms. */
typedef struct { float device_ms, skin_ms, gather_ms, refit_ms, top_ms, wide_ms; uint32_t errors; } trt_deform_stats;

/* Uploads the skinned models' corners and the deforming meshes, checks each mesh's tree (on the host copy taken at
 * upload) and links every node to its parent. Again replaces what was set up. */
int trt_deform_setup(trt_scene* scene, const trt_deform_desc* desc);
/* One frame: palette_rows holds n_matrices matrices of 3 rows (x, y, z, translation) each; every mesh's palette
 * indices must fall inside it. Asynchronous unless stats is given. A wide BVH (TRT_RENDER_WIDE) follows on the device:
 * its mesh trees' nodes quantised again over the refit boxes, its triangle copies gathered again, the rebuilt top tree
 * collapsed again (at once when one is built, else when the first wide walk builds it). flags: 0. */
int trt_deform(trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], const float* palette_rows,
               uint32_t n_matrices, uint32_t flags, trt_deform_stats* stats);

/* Renders samples [first_sample, first_sample + spp) at Params' size (gpu.rs:4116 Gpu::render; its per-dispatch
 * `size.z` is the sample index). Without TRT_RENDER_ACCUMULATE the scene's accum is cleared first, as the reference
 * clears it (gpu.rs:4170). accum_host: NULL, or w * h * 20 floats to copy the result to. stats: NULL (no
 * synchronisation), or filled after the call completes. */
int trt_render(trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t first_sample, uint32_t spp,
               uint32_t flags, float* accum_host, trt_stats* stats);
/* The scene's accum on the device (w * h Pixel records) for zero-copy consumers (a denoiser). */
int trt_accum_device_ptr(trt_scene* scene, void** ptr, uint64_t* bytes);
/* Copies the accum to host memory. */
int trt_accum_read(trt_scene* scene, float* accum_host, uint64_t bytes);
/* Copies the accum into device memory the caller owns (a buffer on the scene's device, bytes = w * h * 80) and waits
 * for the copy: for a collective that sums the accums of ranks that rendered disjoint sample ranges of one image. */
int trt_accum_copy(trt_scene* scene, void* dst_device, uint64_t bytes);

/* Casts rays against the scene (trace_units.wgsl:44-135's query) from host arrays: parity and cost tests. */
int trt_trace(trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], const trt_ray* rays, uint64_t n, uint32_t flags,
              trt_hit* hits);

/* ---- Serving: many requests on resident scenes, batched into shared waves ----
 * Replaces the reference's `serve` loop (renderer/src/main.rs:345-397: JSON-line jobs rendered one at a time through
 * Gpu::render). A server owns a worker thread, its own streams and one wave's device state. Requests (a resident
 * scene, a Params block, a sample count, a host buffer for the result) wait until the device has room for their
 * accum (free HBM less a reserve) and a slot among the active ones; each step then packs the next samples of the
 * active requests, oldest first, into one wave of up to `wave_slots` paths that every kernel of the pass runs at once
 * (a path finds its request through the wave's job table). A request that arrives while others are on the GPU joins
 * the next step. Each request's accum is the one trt_render makes alone, bit for bit: a path's random numbers and
 * sums are its own, and its samples are added in sample order. Scenes must stay uploaded and unchanged while they
 * have requests in flight; requests walk the binary trees. */
typedef struct trt_server trt_server;
typedef struct {
    uint32_t wave_slots;   /* path slots a step (0: 2,097,152); a request's image needs ceil(w/8)*ceil(h/4)*32 */
    uint32_t max_active;   /* requests in flight at most, 1-64 (0: 64) */
    uint64_t hbm_reserve;  /* device bytes admission leaves free (0: 1 GiB) */
    uint32_t flags;        /* TRT_RENDER_UNSORTED_HITS / TRT_RENDER_SORT_* for every step */
    uint32_t launch_mode;  /* 0: each step's launches replayed from a CUDA graph captured once per (depth, size
                            * class); 1: launched one by one */
    trt_unet* denoiser;    /* NULL, or the learned denoiser for requests of few samples (trt_server_submit_rgb); the
                            * server owns it until destroyed: no other call may use it meanwhile */
    uint32_t denoise_max_spp; /* the most samples a request may have to be denoised (0: 4) */
} trt_server_options;
typedef struct {
    uint64_t id;
    int32_t status;        /* TRT_OK, or the error the request ended with */
    uint32_t steps;        /* steps its samples were spread over */
    double submit_ms, start_ms, done_ms;  /* host monotonic clock, ms since the server was created */
} trt_request_done;
typedef struct {
    uint64_t steps, requests_done, paths, closest_rays, shadow_rays;
    double busy_ms;        /* device time of the steps (events around each) */
    uint32_t active, pending;
} trt_server_stats;

int trt_server_create(trt_ctx* ctx, const trt_server_options* opts, trt_server** out);
/* Stops the worker after the requests already admitted are done; pending ones end with TRT_EINVAL. */
void trt_server_destroy(trt_server* server);
/* Queues a request; accum_host (w * h * 20 floats) receives the result and must stay valid until the request is
 * reported done. The Params are checked here (TRT_EINVAL). Thread-safe. */
int trt_server_submit(trt_server* server, trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t spp,
                      float* accum_host, uint64_t* id);
/* A request whose result is also (or only) the denoised image (configs' serving mix: the denoiser on for spp <= 4):
 * rendered with the first-hit depth (TRT_RENDER_DEPTH), its accum denoised on the device by the server's network when
 * its samples are done, rgb_host (w * h * 3 floats) receiving the image. accum_host may be NULL. TRT_EINVAL without a
 * denoiser, above denoise_max_spp samples, or at a size the network does not take. */
int trt_server_submit_rgb(trt_server* server, trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t spp,
                          float* accum_host, float* rgb_host, uint64_t* id);
/* The server's clock: ms since it was created (the clock of trt_request_done's times). */
int trt_server_clock(trt_server* server, double* now_ms);
/* trt_server_submit_rgb (accum_host, rgb_host: either may be NULL, not both; rgb_host needs the denoiser) for a request
 * that arrives at at_ms on the server's clock: the worker admits it no earlier, and its submit_ms is at_ms, so that an
 * open-loop stream of arrivals is handed over at once, with no host thread timing it. A time not after now (or
 * negative: now) arrives at once. No counterpart in the reference, whose serve loop reads jobs as they come. */
int trt_server_submit_at(trt_server* server, trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t spp,
                         float* accum_host, float* rgb_host, double at_ms, uint64_t* id);
/* Up to cap finished requests since the last call, waiting up to wait_ms for one if none is ready. */
int trt_server_poll(trt_server* server, trt_request_done* done, uint32_t cap, uint32_t* n, uint32_t wait_ms);
int trt_server_stats_get(trt_server* server, trt_server_stats* out);

/* The render without allocations. It has no counterpart in the reference. It is for callers that may not call
 * cudaMalloc: a process whose device memory all belongs to one pool (an engine's caching allocator that reserved the
 * device up front, or a hard per-process memory budget), where an allocation from outside the pool fails or steals
 * memory the pool has counted on; and plugin hosts that forbid allocation inside their render callbacks. The caller
 * owns every buffer: `dev` holds DEVICE pointers to the scene's buffers (laid out as for trt_scene_upload),
 * `accum_device` w * h Pixel records, `stream` a cudaStream_t (NULL: the legacy default stream). The wave's working
 * state lives in one file-scope device array of 32 MiB (31.5 MiB used) that every GPU loading the library holds
 * until the process exits; the call allocates nothing: no cudaMalloc, no cudaFree, no allocating library routine.
 * Limits: images of at most 65,536 path slots (8 x 4 pixel tiles: 256 x 256), at most 4 directional lights, the
 * binary walk; larger sizes are refused with TRT_EINVAL before any CUDA call, with a message in `err` (err_len bytes,
 * may be NULL). The first call on a device sets it up with that device current (the array's device address, the
 * sampler's tables). The kernels run on `stream`; the call then waits for them and returns TRT_EGUARD if a walk
 * stopped at its iteration limit. Every call shares the array, which keeps the last call's contents (each call
 * clears the counters it needs): calls whose work overlaps on the GPU race for it, so run them on one stream, or one
 * at a time. Flags: TRT_RENDER_ACCUMULATE; TRT_RENDER_UNSORTED_HITS is accepted and changes nothing (the hits are
 * always shaded unsorted here). */
int trt_render_noalloc(const trt_scene_desc* dev, const uint32_t params[TRT_PARAMS_WORDS], uint32_t first_sample,
                       uint32_t spp, uint32_t flags, float* accum_device, void* stream, char* err, size_t err_len);

/* Diagnostics: the device's single-precision transcendentals, compiled as the pass's shading calls them (cosf, sinf
 * for sampled angles, acosf and atan2f for the environment's coordinates), over host arrays: out[i] = f(x[i]) or
 * atan2f(x[i], y[i]). The shading's results differ from a CPU libm's only by these functions' last bits; this lets a
 * test bound that difference in ulps (the reference leaves WGSL builtins' precision to the GPU driver). */
#define TRT_MATH_COS 0u
#define TRT_MATH_SIN 1u
#define TRT_MATH_ACOS 2u
#define TRT_MATH_ATAN2 3u
int trt_math_eval(trt_ctx* ctx, uint32_t fn, const float* x, const float* y, uint64_t n, float* out);

int trt_scene_totals(trt_scene* scene, trt_totals* out);
void trt_scene_reset_totals(trt_scene* scene);
/* 1: record per-stage CUDA events (extend_ms, shadow_ms in the totals). */
void trt_scene_set_profiling(trt_scene* scene, int on);

/* Device-time brackets on the context's stream: start records an event, stop records one, synchronises and returns
 * the milliseconds between them. */
int trt_timer_start(trt_ctx* ctx);
/* (waits for the asynchronous read-backs queued on the context's copy stream as well) */
int trt_timer_stop(trt_ctx* ctx, float* ms);
/* Waits for the context's stream and its copy stream. */
int trt_synchronize(trt_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
