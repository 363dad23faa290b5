/*
 * lux.h - C ABI of the B200 Split Radiance Cascades transport library (liblux).
 *
 * This is the drop-in boundary for the Split transport hot path of bevy_lux
 * (HyperExtendedReality/bevy_penumbra): closest-hit BVH traversal of cascade
 * interval rays, interval deposit, the split cascade merge, probe packing and
 * the world-space probe resolve.  In the reference these run as Slang compute
 * dispatches issued by `render` (src/render.rs:9553-9801); here each call
 * below replaces one group of those dispatches.
 *
 * Conventions
 *  - Every function returns lux_status; 0 (LUX_OK) is success.  No C++
 *    exception crosses this boundary.  The text of the last failure of a
 *    context is available from lux_last_error_message (the reference records
 *    failures as strings: RadianceCascadesStatus::record_failure,
 *    src/lib.rs:225-230).
 *  - Handles are opaque and owned by the library.  Calls on one context must
 *    be serialised by the caller; distinct contexts may run on distinct host
 *    threads.
 *  - Pointers documented as "device" are CUDA device pointers on the
 *    context's device; all device work is ordered on the context's stream.
 *  - Scene inputs are the reference's own packed word streams (uint4 words,
 *    little endian), so src/scene.rs output can be passed unchanged.
 */
#ifndef LUX_H
#define LUX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUX_ABI_VERSION 1u

typedef enum lux_status {
    LUX_OK = 0,
    LUX_ERR_INVALID_ARGUMENT = 1,
    LUX_ERR_CUDA = 2,
    LUX_ERR_OUT_OF_MEMORY = 3,
    LUX_ERR_CAPACITY = 4,        /* a view's fixed capacity was exceeded */
    LUX_ERR_MALFORMED_SCENE = 5, /* scene words failed validation */
    LUX_ERR_NO_DEVICE = 6,
    LUX_ERR_TIMEOUT = 7,         /* a bounded device wait gave up */
    LUX_ERR_INTERNAL = 8
} lux_status;

/* Hit.errors bits, same values as shaders/traversal.slang:16 and :500,:743. */
#define LUX_HIT_BLAS_FALLBACK 1u
#define LUX_HIT_TLAS_FALLBACK 2u
#define LUX_HIT_QUERY_UNSUPPORTED 4u
#define LUX_EMPTY 0xffffffffu

typedef struct LuxContext LuxContext;
typedef struct LuxScene LuxScene;
typedef struct LuxView LuxView;

typedef struct LuxDeviceDesc {
    int32_t device;  /* CUDA ordinal */
    void *stream;    /* cudaStream_t to order work on; NULL = library-owned stream */
} LuxDeviceDesc;

/* One ray of the traversal harness: the reference's `Ray` of
 * src/traversal_tests.rs (origin, direction, limit, any_hit). */
typedef struct LuxRay {
    float origin[3];
    float tmin;       /* hits must satisfy t > max(tmin, 2.5e-5) */
    float direction[3];
    float limit;      /* hits must satisfy t < limit */
} LuxRay;

/* Closest-hit record: the reference's Hit (shaders/traversal.slang:1). */
typedef struct LuxHit {
    float distance;
    uint32_t triangle;
    uint32_t instance;
    uint32_t errors;
    float barycentric[3];
    uint32_t visited;  /* nodes visited (statistics) */
} LuxHit;

/* Emitter / light record, the reference's `Light`
 * (shaders/common.slang:110): position, color, direction, edge1, edge2 as
 * float4 then source as uint4; 24 words.  Emissive triangle records follow
 * the conventional ones exactly as build_emissive_lights writes them
 * (src/scene.rs:2311-2372). */
typedef struct LuxLight {
    float position[4];
    float color[4];
    float direction[4];
    float edge1[4];
    float edge2[4];
    uint32_t source[4];
} LuxLight;

/* Probe layouts. */
#define LUX_LAYOUT_SPLIT 0u      /* receivers trace rays and deposit into every level (the reference's Split) */
#define LUX_LAYOUT_DENSE 1u      /* every (probe, direction) of every level traces its own interval */

/* Interval growth rules. */
#define LUX_INTERVAL_ENDS_GEOMETRIC 0u   /* end_L = length * ratio^L (reference: ratio 4, shaders/split.slang:224-227) */
#define LUX_INTERVAL_LENGTHS_GEOMETRIC 1u /* length_L = length * ratio^L, end_L = sum of lengths */

#define LUX_MAX_LEVELS 12u

/* Per-view transport settings.  Field names and clamps follow
 * RadianceCascades / SamplingSettings (src/lib.rs:343-518, sanitized at
 * src/lib.rs:731-759); the fields marked "extension" parameterise what the
 * reference hard-codes (CASCADES = 4, BASE_THETA = 4 and the x4 interval rule,
 * shaders/common.slang:10-11, shaders/split.slang:224-231). */
typedef struct LuxSettings {
    float probe_spacing;            /* RadianceCascades::probe_spacing (tuning.x) */
    float interval_length;          /* RadianceCascades::interval_length (tuning.y) */
    float normal_bias;              /* RadianceCascades::normal_bias (tuning.z) */
    float intensity;                /* RadianceCascades::intensity (tuning.w) */
    float environment[3];           /* RadianceCascades::environment: constant sky radiance seen by hit-surface NEE
                                       (environmentResponseTracked, shaders/environment.slang:154-230; black: no
                                       sky samples); escaped interval rays carry supported zero */
    float exposure;                 /* camera exposure (params.environment.w) */
    uint32_t emissive_samples;      /* RadianceCascades::emissive_samples, 1..=32; NEE draws max(1, n/2) */
    uint32_t levels;                /* extension: cascade count, 1..=LUX_MAX_LEVELS (reference 4) */
    uint32_t base_columns;          /* extension: azimuth bins at cascade 0 (reference 2*BASE_THETA = 8) */
    uint32_t base_rows;             /* extension: polar bins at cascade 0 (reference BASE_THETA = 4) */
    float interval_ratio;           /* extension: growth ratio (reference 4) */
    uint32_t interval_rule;         /* extension: LUX_INTERVAL_* (reference ENDS_GEOMETRIC) */
    uint32_t layout;                /* LUX_LAYOUT_* */
    uint32_t rays_per_receiver;     /* Split layout: rays traced per receiver per frame (reference 1) */
    uint32_t frame_index;           /* params.frame.x */
    uint32_t resolve_scale;         /* SamplingSettings::resolve_scale, 1..=8 */
    float temporal_blend;           /* RadianceCascades::temporal_blend (history.x): per-observation retention of
                                       interval radiance, 0..=0.99; mass limit 1 / (1 - blend) */
    float transmittance_blend;      /* RadianceCascades::split_transmittance_blend (intervalHistory.x), 0..=0.999 */
    uint32_t history_frames;        /* RadianceCascades::history_frames (history.w), 0..=64; 0 disables history */
    uint32_t multi_bounce;          /* RadianceCascades::multi_bounce: 1 adds the secondary cache's diffuse bounce
                                       light at interval-ray hits (Split layout, unbatched frames) */
    uint32_t cached_hit_sky;        /* RadianceCascades::cached_hit_sky (lightCounts.w, src/render.rs:8495): with
                                       multi_bounce, the secondary cache's escaped rays carry the environment and
                                       hits its previous frame covers take their sky light from it instead of
                                       tracing environment samples (cachedHitSky, shaders/common.slang:71-74) */
} LuxSettings;

/* Receivers (Split) or the cascade-0 probe set (Dense), device pointers.
 * position[i] = (x, y, z, unused), normal[i] = (geometric normal, unused).
 * For the dense layout normals are ignored and positions are cascade-0
 * probe centres. */
typedef struct LuxReceivers {
    const float *position;  /* device float4[count] */
    const float *normal;    /* device float4[count] */
    uint32_t count;
} LuxReceivers;

/* Device-side statistics of the last frame (the reference's head counters,
 * shaders/split.slang:517-533). */
typedef struct LuxStats {
    uint64_t interval_rays;     /* closest-hit interval rays traced */
    uint64_t shadow_rays;       /* NEE visibility rays traced */
    uint64_t nodes_visited;     /* BVH4 nodes visited by all rays */
    uint64_t triangles_tested;  /* triangle tests by all rays */
    uint64_t instances_visited; /* instance transforms applied */
    uint64_t deposits;          /* (level, entry) samples deposited */
    uint64_t unsupported;       /* rays whose query was unsupported */
    uint64_t shadow_nodes;      /* of nodes_visited: by visibility queries */
    uint64_t shadow_triangles;  /* of triangles_tested: by visibility queries */
    uint64_t shadow_instances;  /* of instances_visited: by visibility queries */
    uint32_t cells[LUX_MAX_LEVELS];
    uint64_t entries[LUX_MAX_LEVELS];
    uint32_t levels;
    uint32_t error_flags;       /* LUX_VIEW_ERR_* bits raised on the device */
} LuxStats;

#define LUX_VIEW_ERR_CELL_CAPACITY 1u
#define LUX_VIEW_ERR_ENTRY_CAPACITY 2u
#define LUX_VIEW_ERR_PROBE_LOOKUP 4u
#define LUX_VIEW_ERR_RAY_CAPACITY 8u
#define LUX_VIEW_ERR_TIMEOUT 16u   /* a batch's grid-barrier wait ran out (lux_batch_status) */

/* Capacities of a view (ViewBuffers, src/render.rs:5077-5160).  Device
 * memory grows with max_entries by 88 bytes per record (sums, counts, merged,
 * raw and mass records, the previous frame's raw and mass, the merge's list
 * of records that pass light on). */
typedef struct LuxViewDesc {
    uint32_t max_receivers;  /* receivers (Split) or cascade-0 probes (Dense) */
    uint32_t max_cells;      /* distinct world cells per level */
    uint64_t max_entries;    /* (cell, direction) records summed over levels */
    uint32_t max_rays;       /* interval rays per frame: receivers x rays_per_receiver (Split) or records (Dense) */
    uint32_t reserved;
} LuxViewDesc;

/* ---- library / context ---------------------------------------------- */
uint32_t lux_abi_version(void);
lux_status lux_context_create(const LuxDeviceDesc *desc, LuxContext **out);
lux_status lux_context_destroy(LuxContext *ctx);
const char *lux_last_error_message(const LuxContext *ctx);
lux_status lux_context_synchronize(LuxContext *ctx);

/* ---- settings (RadianceCascades mirror, src/lib.rs:671-759) ----------- */
void lux_settings_default(LuxSettings *out);   /* RadianceCascades::default() */
void lux_settings_low_end(LuxSettings *out);   /* RadianceCascades::low_end() */
void lux_settings_sanitize(LuxSettings *s);    /* RadianceCascades::sanitized() */
/* Interval end of `level` (shaders/split.slang:224-227 generalised). */
float lux_interval_end(const LuxSettings *s, uint32_t level);
uint32_t lux_direction_count(const LuxSettings *s, uint32_t level);

/* ---- scene (GiScene words, src/scene.rs:2096-2117, :809-823) ---------- */
/* Packs meshes and instances into the reference's word streams.  Restates
 * build_tree (binned SAH, 12 bins, leaves <= 4, depth <= 48,
 * src/scene.rs:2398-2554), node_words (src/scene.rs:1025-1038),
 * pack_instances (src/scene.rs:1071-1122), geometry_words
 * (src/scene.rs:809-823) and build_emissive_lights (src/scene.rs:2311-2372).
 * Inputs (host):
 *   positions[3*vertex_count], indices[3*triangle_count] (global vertex ids)
 *   mesh_first_triangle[mesh_count], mesh_triangle_count[mesh_count]
 *   per instance (host): mesh id, world_from_local 3x4 row-major (12 floats),
 *   flags (bits 0-1 cull mode, 2 mirror), material id
 *   materials: 8 uint4 words each (MATERIAL_WORDS, src/material.rs:16)
 * The library keeps the packed words; query sizes then copy them out. */
typedef struct LuxPackedScene LuxPackedScene;
lux_status lux_scene_pack(const float *positions, uint32_t vertex_count,
                          const uint32_t *indices, uint32_t triangle_count,
                          const uint32_t *mesh_first_triangle, const uint32_t *mesh_triangle_count,
                          uint32_t mesh_count,
                          const uint32_t *instance_mesh, const float *instance_world_from_local,
                          const uint32_t *instance_flags, const uint32_t *instance_material,
                          uint32_t instance_count,
                          const uint32_t *material_words, uint32_t material_count,
                          LuxPackedScene **out);
/* Word counts are in uint4 units; light count in LuxLight records. */
lux_status lux_packed_scene_sizes(const LuxPackedScene *p, size_t *scene_words,
                                  size_t *geometry_words, size_t *lights,
                                  uint32_t *tlas_nodes, uint32_t *blas_nodes);
lux_status lux_packed_scene_copy(const LuxPackedScene *p, uint32_t *scene_words,
                                 uint32_t *geometry_words, LuxLight *lights);
/* Packed instance i is caller instance order[i] (the TLAS build permutes
 * instances into leaf order, src/scene.rs:2052). */
lux_status lux_packed_scene_instance_order(const LuxPackedScene *p, uint32_t *order);
/* SAH cost of the packed TLAS and of all BLASes (tree_cost, src/scene.rs:2383-2396)
 * and the maximum leaf depth. */
lux_status lux_packed_scene_quality(const LuxPackedScene *p, double *blas_cost,
                                    uint32_t *max_depth);
void lux_packed_scene_destroy(LuxPackedScene *p);
/* Emissive light records after a rigid pose update (moving emitters, for
 * lux_scene_refit's `lights`): every record's triangle is re-transformed by
 * its instance's new world_from_local (host float[instance_count * 12] in
 * instance-record order) exactly as the packer transforms it
 * (build_emissive_lights, src/scene.rs:2311-2372); areas, power and the CDF
 * stay those of `lights`.  out: host LuxLight[light_count]. */
lux_status lux_emissive_lights_at(const uint32_t *geometry_words, size_t geometry_word_count,
                                  const LuxLight *lights, uint32_t light_count,
                                  const float *world_from_local, uint32_t instance_count, LuxLight *out);

/* Uploads word streams (host pointers) and builds the device BVH4 layout.
 * scene_words = [header, TLAS node words, BLAS node words, instance words,
 * materials...]; conventional_lights = how many leading light records are
 * conventional (lightCounts.x); the rest are emissive (lightCounts.y). */
lux_status lux_scene_upload(LuxContext *ctx,
                            const uint32_t *scene_words, size_t scene_word_count,
                            const uint32_t *geometry_words, size_t geometry_word_count,
                            const LuxLight *lights, uint32_t light_count,
                            uint32_t conventional_lights,
                            LuxScene **out);
/* The host half of lux_scene_upload without a device: the same validation of
 * the word streams and the same BVH4 collapse, returning the status the
 * upload would return (LUX_ERR_MALFORMED_SCENE for cycles, shared subtrees,
 * out-of-range indices or oversized leaves -- the reference's malformed BLAS
 * fixtures, src/traversal_tests.rs:1594-1636 -- in time linear in the node
 * count).  message: optional, receives the upload's error text. */
lux_status lux_scene_validate(const uint32_t *scene_words, size_t scene_word_count,
                              const uint32_t *geometry_words, size_t geometry_word_count,
                              const LuxLight *lights, uint32_t light_count,
                              uint32_t conventional_lights, char *message, size_t message_size);
lux_status lux_scene_destroy(LuxScene *scene);
/* Device BVH4 size facts: nodes (TLAS+BLAS) and node/triangle record bytes. */
lux_status lux_scene_layout(const LuxScene *scene, uint32_t *nodes, uint32_t *node_bytes,
                            uint32_t *triangles, uint32_t *triangle_bytes,
                            uint32_t *instances);

/* Rigid pose update of every instance: the host half writes each instance's
 * rows 0-5 (local_from_world, inverted in f64 like the packer, and
 * world_from_local) as the reference's instance upload does
 * (src/render.rs:3819-3915), then one device launch refits the TLAS bottom-up
 * by depth with refitTlas's conservative transformed boxes
 * (shaders/acceleration.slang:61-88) and rewrites the BVH4 child boxes.  The
 * tree topology is kept.  world_from_local: host float[count * 12], row-major
 * 3x4, in instance-record order (the packed scene's slot order); count must
 * equal the scene's instance count.  lights: NULL to keep the uploaded
 * records, else light_count (= the uploaded count) replacement records
 * (moved emitters).  Stream-ordered on the context stream. */
lux_status lux_scene_refit(LuxScene *scene, const float *world_from_local, uint32_t count,
                           const LuxLight *lights, uint32_t light_count);
/* Copies the scene's device words (scene_words as uploaded, with refit boxes
 * and instance rows) to host memory: out[word_count * 4]; word_count must
 * equal the uploaded scene word count.  Synchronises the context stream. */
lux_status lux_scene_read_words(const LuxScene *scene, uint32_t *out, size_t word_count);

/* ---- traversal (traceRay / traceOccluded, shaders/traversal.slang:696-1046) -- */
/* Closest hit (any_hit = 0) or occlusion (any_hit = 1) for `count` rays.
 * rays: device LuxRay[count]; hits: device LuxHit[count].  For any-hit rays
 * hits[i].triangle != LUX_EMPTY means blocked. */
lux_status lux_trace_rays(LuxContext *ctx, const LuxScene *scene, const LuxRay *rays,
                          uint32_t count, uint32_t any_hit, LuxHit *hits);

/* Interval radiance of caller rays: the closest hit of each ray and the
 * outgoing radiance there (hit emission + emissive next-event estimation with
 * visibility rays), the value traceTransport deposits
 * (shaders/split.slang:1122-1216, shaders/cascades.slang:196-268).
 * rays: device LuxRay[count]; out: device float4[count] = (radiance rgb, hit
 * distance, or the ray's limit on a miss), or (0, 0, 0, -1) when the query is
 * unsupported.  Trace scratch is owned by the context and grows with count. */
lux_status lux_interval_radiance(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings,
                                 const LuxRay *rays, uint32_t count, float *out);

/* lux_interval_radiance for callers that are not allowed to allocate device
 * memory.  No counterpart in the reference: it exists for hosts such as a
 * real-time render thread, where cudaMalloc / cudaFree can synchronise the
 * device and stall a frame, or an engine that reserves its whole device
 * budget up front through its own allocator and forbids allocations it does
 * not account for.  This entry point calls no cudaMalloc, cudaFree or other
 * allocating routine: its scratch is one fixed array of about 7.5 MiB built
 * into the library, which every device that loads the library keeps until the
 * process exits.
 *  - At most 8192 rays per call; larger counts fail with LUX_ERR_CAPACITY
 *    before any work is queued.  Split bigger batches.
 *  - The first call on a device looks up the array's device address (with
 *    that device made current, and the caller's current device restored
 *    afterwards); make that first call before any stream capture on the
 *    device.
 *  - All calls share the one array.  Each call resets the counters it needs
 *    and overwrites the rest, but calls whose GPU work overlaps (different
 *    streams or contexts on the same device) race: order them. */
lux_status lux_interval_radiance_noalloc(LuxContext *ctx, const LuxScene *scene,
                                         const LuxSettings *settings, const LuxRay *rays,
                                         uint32_t count, float *out);

/* ---- cascade view (render(), src/render.rs:9124-9830) ------------------ */
lux_status lux_view_create(LuxContext *ctx, const LuxViewDesc *desc, LuxView **out);
lux_status lux_view_destroy(LuxView *view);
/* seed -> trace (+NEE) -> deposit -> merge (levels L-1..0) -> pack.
 * Replaces the dispatch sequence clear..packProbes (src/render.rs:9553-9801). */
lux_status lux_view_trace_merge(LuxView *view, const LuxScene *scene, const LuxSettings *settings,
                                const LuxReceivers *receivers);
/* worldResolve (shaders/world_resolve.slang:281-313): for each point
 * (device float4 position, float4 shading normal) writes device float4
 * (irradiance / pi, alpha = 1 + 0.25 coverage | -1 | 0). */
lux_status lux_view_resolve(LuxView *view, const LuxSettings *settings, const float *points_position,
                            const float *points_normal, uint32_t count, float *out_irradiance);
/* The same frame with HOST buffers: copies receivers and resolve points to
 * the device, runs trace_merge and resolve, copies irradiance back, and
 * synchronises.  This is the call a host engine makes per frame. */
lux_status lux_view_frame_host(LuxView *view, const LuxScene *scene, const LuxSettings *settings,
                               const float *receiver_position, const float *receiver_normal,
                               uint32_t receiver_count, const float *points_position,
                               const float *points_normal, uint32_t point_count,
                               float *out_irradiance);
lux_status lux_view_stats(LuxView *view, LuxStats *out);
/* Per-stage CUDA-event timing of a view's frames (the reference's per-pass
 * timestamp spans, src/render.rs:9323-9333). */
typedef struct LuxTimings {
    float seed_ms;     /* clear + seed + record layout */
    float trace_ms;    /* closest hit + hit shading + deposit */
    float merge_ms;    /* corner tables + merge of every level */
    float pack_ms;     /* cascade-0 probe tables */
    float resolve_ms;  /* last lux_view_resolve */
} LuxTimings;
lux_status lux_view_set_timing(LuxView *view, uint32_t enable);

/* Launch-shape choices of a view's trace kernels (the autotuner's knobs).
 * closest_mode / shadow_mode: 0 = persistent warps taking 32 rays per fetch,
 * 1 = persistent warps refilling idle lanes between traversal steps.
 * *_blocks_per_sm: persistent blocks of 128 threads per SM (1..64). */
typedef struct LuxTuning {
    uint32_t closest_mode;
    uint32_t shadow_mode;
    uint32_t closest_blocks_per_sm;
    uint32_t shadow_blocks_per_sm;
    uint32_t sort_queries;        /* 1: order visibility queries by (emitter bucket of 8, origin cell of a 128^3
                                     grid over the scene box) before tracing */
    uint32_t sort_rays;           /* 1: order interval rays by (direction bin, origin cell) before tracing */
    uint32_t stack_depth;         /* traversal stack entries per thread: 32 or 64 (0 = 64); an overflowing
                                     walk continues with the reference's ordered scan, same answers */
    uint32_t fused_trace;         /* batches only: 1 = the trace stage (closest hits, shading, visibility,
                                     deposit) as one persistent cooperative launch with bounded grid
                                     barriers between the phases; 0 = four launches */
    uint32_t tile_rays;           /* rays (or visibility queries) a warp takes from the work queue per
                                     fetch: 32, 64, 128 or 256 (0 = 32); the persistent walkers of modes 0 */
    uint32_t reserved;
} LuxTuning;
lux_status lux_view_set_tuning(LuxView *view, const LuxTuning *tuning);
lux_status lux_view_get_tuning(const LuxView *view, LuxTuning *tuning);
lux_status lux_view_timings(LuxView *view, LuxTimings *out);
/* Camera of a view for distance LODs (splitLodBlendForParameters,
 * shaders/common.slang:431-461; LOD keys, spacing and interval ends,
 * shaders/common.slang:414-422, shaders/split.slang:224-236): with a camera
 * set, each Split receiver's probes coarsen by 2^lod with its Chebyshev
 * distance from a perspective camera (or by the projected spacing of an
 * orthographic one); in an LOD overlap both LODs' cells are seeded and the
 * receiver's rays deposit into one of them (seed, shaders/split.slang:
 * 747-786); lux_view_resolve blends the two LODs (resolveSplitDiffuse).
 * Dense, batched and learned-cache frames use LOD 0. */
typedef struct LuxCamera {
    float clip_from_world[16];  /* row-major */
    float position[3];          /* camera position (world) */
    uint32_t viewport_height;   /* pixels */
    uint32_t target_pixels;     /* probe footprint in pixels (split_lod_target_pixels: the resolve scale); 0 = 1 */
    uint32_t enabled;           /* 0: LOD 0 everywhere */
} LuxCamera;
/* NULL or enabled = 0 disables distance LODs. */
lux_status lux_view_set_camera(LuxView *view, const LuxCamera *camera);

/* The view's multi-bounce secondary cache (RadianceCascades::multi_bounce;
 * src/render.rs:5974-6118, :9662-9752): a view owned by `view`, created by
 * its first multi-bounce frame (NULL before), whose receivers are the
 * interval-ray hits of `view`.  Read it with lux_view_read_level /
 * read_probes / stats / timings; do not trace or destroy it. */
lux_status lux_view_secondary(LuxView *view, LuxView **secondary);
/* Copies one level's records to host memory (tests): cell keys int4[cells],
 * merged float4[cells*dirs] (I.rgb, support), raw float4[cells*dirs]
 * (J.rgb, beta) and sample counts uint32[cells*dirs].  Any pointer may be NULL. */
lux_status lux_view_read_level(LuxView *view, uint32_t level, int32_t *cell_keys,
                               float *merged, float *raw, uint32_t *samples);
/* Copies packed cascade-0 probe tables: keys int4[cells], tables float4[cells*36]. */
lux_status lux_view_read_probes(LuxView *view, int32_t *cell_keys, float *tables);

/* World history (mergeEntry, shaders/split.slang:1624-1725).  Each
 * unbatched lux_view_trace_merge blends every record's fresh observations
 * with the same record (cell key, direction, level) of the view's previous
 * frame: retention temporal_blend^n of the old radiance mass (limit
 * 1 / (1 - blend)), likewise the transmittance with transmittance_blend;
 * records without observations keep their history.  History applies when
 * history_frames > 0 and the previous frame had the same cascade shape.
 * Cells seen in neither frame carry no history (records live as long as
 * receivers keep seeding their cell).  Batched frames do not blend, but
 * their records serve as the next unbatched frame's history. */
/* Forgets the view's history (RadianceCascades::reset_history). */
lux_status lux_view_reset_history(LuxView *view);
/* Queues a world box for the next frame: records whose rays may have crossed
 * it (the cell grown by its level's interval end; any record of the last
 * level) take no history (dirty-bounds invalidation; moved geometry). */
lux_status lux_view_invalidate_bounds(LuxView *view, const float lo[3], const float hi[3]);

/* Interval-ray hits of the view's last Split frame, in ray order
 * (ray = receiver * rays_per_receiver + sample): out[count] LuxHit, count <=
 * the frame's interval rays.  visited is 0.  For comparing runs. */
lux_status lux_view_read_hits(LuxView *view, LuxHit *out, uint32_t count);

/* ---- FP64 reference and error reductions ----------------------------------
 * No reference counterpart: the oracle of the error reports.  For every point
 * (device float4 position, float4 unit normal) the mean over `spp`
 * cosine-weighted hemisphere rays from rayOffset(point, normal, normal_bias)
 * of the interval radiance the cascades resolve (emission seen plus
 * one-bounce next-event estimation; irradiance / pi before receiver albedo,
 * the raw output's units).  Rays are traced and shaded in FP32 by the same
 * kernels as lux_interval_radiance; only the per-point accumulation is FP64.
 * Samples run in rounds of lux_reference_round_samples(count, spp) per point
 * (frame index seed + round for the next-event samples).  out: device
 * double4[count] = (mean r, g, b, supported samples).  Allocates temporary
 * device memory; ordered on the context stream. */
uint32_t lux_reference_round_samples(uint32_t count, uint32_t spp);
lux_status lux_reference_irradiance(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings,
                                    const float *position, const float *normal, uint32_t count,
                                    uint32_t spp, uint32_t seed, double *out);
/* The path-traced reference (no reference counterpart in the C API; it
 * restates the reference project's offline path tracer, trace_sample,
 * examples/pathtrace_reference.rs:724-833, from the receivers): per point
 * (device float4 position, float4 unit normal) `spp` paths of up to `bounces`
 * diffuse vertices (1 = direct light only; the reference's default is 3),
 * emissive-triangle next-event estimation with power-heuristic MIS against
 * the cosine proposal, Russian roulette from the fourth vertex; the receiver
 * is Lambertian with unit albedo (irradiance / pi before receiver albedo, the
 * raw output's units) and later vertices use the hit's diffuse colour and
 * disneyDiffuseMultiplier.  FP32 rays, FP64 sums.  out: device
 * double4[count] = (mean r, g, b, supported samples); ordered on the context
 * stream, no allocation. */
lux_status lux_path_reference(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings,
                              const float *position, const float *normal, uint32_t count, uint32_t spp,
                              uint32_t bounces, uint32_t seed, double *out);
/* FP64 error of an FP32 estimate (device float4[count], alpha > 0 =
 * resolved) against a reference (device double4[count], w > 0 = sampled):
 * out[4] (host) = {sum of squared rgb error, sum of reference rgb, points
 * used, max |error|}; relative RMSE = sqrt(out[0] / (3 out[2])) /
 * (out[1] / (3 out[2])).  Synchronises the context stream. */
lux_status lux_error_stats(LuxContext *ctx, const float *estimate, const double *reference, uint32_t count,
                           double out[4]);
/* Measured read rate of the context's device (no reference counterpart; the
 * denominator of the traversal roofline): one launch reads a device buffer
 * of `bytes` bytes (a multiple of 16 in [1 MiB, 64 GiB]) `passes` times
 * (1..4096) with 16-byte loads that bypass L1; the shortest of five timed
 * launches after a warm-up.  A buffer well inside L2 (126 MB on B200) gives
 * the L2 read rate, the bound of the traversal kernels, whose scene stays in
 * L2; one well above it gives the HBM read rate.  *gb_per_s = bytes x passes
 * / time / 1e9.  Allocates and frees the buffer; synchronises the context
 * stream. */
lux_status lux_measure_read_rate(LuxContext *ctx, uint64_t bytes, uint32_t passes, double *gb_per_s);

/* ---- learned radiance cache ------------------------------------------------
 * No reference counterpart (the reference's README defers neural caching).
 * A multiresolution hash encoding (levels x 2 BF16 features, 2^log2_table
 * entries per level, base resolution x growth^level over the scene box)
 * feeding a fused MLP: 64 inputs (32 hash features, 16 spherical-harmonic
 * coefficients of the direction, normal, albedo, a constant 1, zeros), 4
 * hidden layers of 64 ReLU units, 3 linear outputs; BF16
 * weights and FP32 accumulation on the 5th-generation tensor cores
 * (tcgen05.mma with TMEM accumulators) for the forward pass and the
 * backward data gradients; Adam (FP32 master copies) for the table and the
 * weights.  Loss: relative L2, (y - t)^2 / (y^2 + 0.01).  Trained online on
 * interval radiance samples the transport produces and queried for the
 * radiance arriving at a point from a direction. */
typedef struct LuxCache LuxCache;
typedef struct LuxCacheDesc {
    uint32_t levels;          /* 16 */
    uint32_t log2_table;      /* 19 */
    uint32_t base_resolution; /* 16 */
    float growth;             /* 1.5 */
    float learning_rate;      /* 1e-3 */
    uint32_t batch;           /* samples per Adam step: 16384 */
    uint32_t seed;
    uint32_t reserved;
} LuxCacheDesc;
/* One training sample or query: the radiance arriving at `position` from
 * `direction` (unit; the ray's direction), at a receiver with `normal` and
 * `albedo`; radiance = target (samples) and weight (0 = ignore). 64 bytes. */
typedef struct LuxCacheSample {
    float position[3];
    float weight;
    float direction[3];
    float pad0;
    float normal[3];
    float pad1;
    float albedo[3];
    float pad2;
} LuxCacheSample;
typedef struct LuxCacheStats {
    uint64_t steps;           /* Adam steps taken */
    uint64_t samples;         /* training samples consumed */
    float last_loss;          /* mean relative L2 loss of the last step */
    uint32_t error_flags;     /* 1: a tensor-core wait gave up */
} LuxCacheStats;
void lux_cache_desc_default(LuxCacheDesc *desc);
lux_status lux_cache_create(LuxContext *ctx, const LuxCacheDesc *desc, LuxCache **out);
lux_status lux_cache_destroy(LuxCache *cache);
/* Scene box the hash grid covers (positions outside are clamped). */
lux_status lux_cache_set_bounds(LuxCache *cache, const float lo[3], const float hi[3]);
/* Trains on `count` device samples with device targets rgb (float4 per
 * sample, .w unused): ceil(count / batch) Adam steps in order. */
lux_status lux_cache_train(LuxCache *cache, const LuxCacheSample *samples, const float *targets, uint32_t count);
/* Predicts radiance (device float4 per query: rgb >= 0, w = 1). */
lux_status lux_cache_query(LuxCache *cache, const LuxCacheSample *queries, uint32_t count, float *out);
lux_status lux_cache_stats(LuxCache *cache, LuxCacheStats *out);
/* Tests: the 64-wide BF16 input encoding of `count` device samples
 * (device uint16 bf16 bits [count][64]), the MLP weights as FP32
 * (host float[64*64*4 + 16*64], layer-major, each [out][in]), and the raw
 * MLP output of given encodings (device float4 per row; no clamping). */
lux_status lux_cache_encode(LuxCache *cache, const LuxCacheSample *samples, uint32_t count, uint16_t *out);
lux_status lux_cache_read_weights(LuxCache *cache, float *out);
lux_status lux_cache_forward(LuxCache *cache, const uint16_t *encoded, uint32_t count, float *out);
/* Tests: one training pass of count (1..batch) device samples with device
 * targets without the Adam step -- the FP32 weight gradients (host
 * float[64*64*4 + 16*64], layout of lux_cache_read_weights) and hash-table
 * gradients (host float[levels * 2^log2_table * 2]) -- then clears both; and
 * the FP32 master hash table (same layout). */
lux_status lux_cache_gradients(LuxCache *cache, const LuxCacheSample *samples, const float *targets,
                               uint32_t count, float *grad_weights, float *grad_table);
lux_status lux_cache_read_table(LuxCache *cache, float *out);

/* Learned-cache form of a view's Split frame (no reference counterpart).
 * Interval rays of cascade-0 cells that are neither validated this frame nor
 * falling back trace only up to the end of level cutoff_level - 1; a ray
 * that meets nothing there takes the cache's radiance for its (origin,
 * direction) as its hit radiance at level cutoff_level, so the levels from
 * cutoff_level on are answered by the cache instead of traced.  Each frame
 * 1/validate_period of the cascade-0 cells (rotating) trace fully; their
 * rays past the cutoff are compared with the cache and a cell whose bias
 * |sum cache - sum traced| exceeds error_bound x its summed traced radiance
 * plus three standard deviations of that sum (single traced rays carry
 * next-event noise) traces fully for the next fallback_frames frames.  Up to train_samples rays per frame
 * (validated rays and rays that hit within cascade 1) train the cache, one
 * lux_cache_train inside the frame.  mode NULL or mode->cache NULL: plain. */
typedef struct LuxCacheMode {
    LuxCache *cache;
    uint32_t cutoff_level;     /* 3 */
    uint32_t validate_period;  /* 16 */
    float error_bound;         /* 0.25 */
    uint32_t train_samples;    /* 65536 */
    uint32_t fallback_frames;  /* 32 */
    uint32_t reserved[3];
} LuxCacheMode;
typedef struct LuxCacheFrameStats {
    uint64_t cached_rays;      /* rays answered by the cache */
    uint64_t validated_rays;   /* fully traced rays past the cutoff compared with the cache */
    uint64_t train_candidates; /* rays eligible as training samples */
    uint64_t trained_samples;  /* samples given to lux_cache_train */
    uint32_t validated_cells;
    uint32_t failed_cells;     /* cells sent to fallback this frame */
    uint32_t fallback_rays;    /* rays traced fully because their cell falls back */
    float validated_bias;      /* (sum cache - sum traced) / sum traced over the validated rays */
} LuxCacheFrameStats;
lux_status lux_view_set_cache(LuxView *view, const LuxCacheMode *mode);
lux_status lux_view_cache_stats(LuxView *view, LuxCacheFrameStats *out);

/* ---- batching: many scenes and views in one launch per trace stage -------
 * No reference counterpart (the reference renders one view per dispatch
 * sequence).  One lux_batch_trace_merge runs the Split frame of every job:
 * each view's seed/layout and merge/pack kernels, and for all jobs together
 * ONE persistent closest-hit launch, one shading launch, one visibility launch
 * and one deposit launch over the concatenated rays (every warp works on
 * one job; uneven ray counts balance across the GPU).  With graphs enabled
 * (the default) the whole multi-view frame is captured once per job
 * configuration as a CUDA graph and replayed; only frame_index may change
 * between replays.  Results per view are read with the lux_view_* calls and
 * equal an unbatched lux_view_trace_merge of the same view bit for bit on hit
 * ids (queue order, and so float sums, may differ).  Sorting tuning flags do
 * not apply to batched frames. */
typedef struct LuxBatch LuxBatch;
typedef struct LuxBatchJob {
    LuxView *view;            /* distinct per job, created on the batch's context */
    const LuxScene *scene;    /* may be shared between jobs */
    LuxReceivers receivers;   /* device pointers, as lux_view_trace_merge */
} LuxBatchJob;
typedef struct LuxBatchInfo {
    uint32_t jobs;
    uint32_t graph_captures;  /* CUDA graphs captured so far */
    uint64_t graph_launches;  /* frames replayed from a graph */
    uint64_t interval_rays;   /* interval rays of one frame */
    uint32_t kernels_per_frame; /* kernel launches one frame enqueues */
    uint32_t reserved;
} LuxBatchInfo;
lux_status lux_batch_create(LuxContext *ctx, LuxBatch **out);
lux_status lux_batch_destroy(LuxBatch *batch);
/* 1 (default): capture/replay a CUDA graph; 0: direct launches. */
lux_status lux_batch_set_graph(LuxBatch *batch, uint32_t enable);
/* closest/shadow blocks per SM of the batched persistent launches and
 * fused_trace (modes, sort flags and stack depth are ignored); the fused
 * launch takes min(closest_blocks_per_sm, resident blocks per SM). */
lux_status lux_batch_set_tuning(LuxBatch *batch, const LuxTuning *tuning);
/* One frame of every job with shared settings (layout must be Split). */
lux_status lux_batch_trace_merge(LuxBatch *batch, const LuxBatchJob *jobs, uint32_t job_count,
                                 const LuxSettings *settings);
lux_status lux_batch_info(const LuxBatch *batch, LuxBatchInfo *out);
/* Waits for the batch's last frame; LUX_ERR_TIMEOUT when a grid-barrier
 * wait of its fused trace launch ran out (the jobs' views then carry
 * LUX_VIEW_ERR_TIMEOUT and their passes after the trace were skipped; the
 * next frame starts clean). */
lux_status lux_batch_status(LuxBatch *batch);
/* Bound of each grid-barrier wait of the fused trace launch (1 ms .. 10 s,
 * default 1 s).  missing_arrivals > 0 is a test hook: every barrier then
 * waits for that many blocks that do not exist, so the first wait runs out. */
lux_status lux_batch_set_wait(LuxBatch *batch, uint64_t limit_ns, uint32_t missing_arrivals);

/* ---- Screen reconstruction after the world resolve --------------------
 * The reference's temporal and denoise passes (shaders/cascades.slang:310-690,
 * dispatched at src/render.rs:9836-9930) for the Split method's persistent
 * world intervals: reprojected screen history with neighbourhood clamping,
 * then `spatial_filter_steps` edge-stopping a-trous passes (strides 1, 2, 4,
 * 8).  Only the temporal result becomes history.  Per-pixel inputs are at the
 * resolve extent, row-major, device pointers. */
typedef struct LuxScreenFrame {
    const float *irradiance;     /* float4: lux_view_resolve output of the pixel (alpha = rawGiSupportAlpha) */
    const float *position;       /* float4: world position xyz; w = view depth, > 0 on a surface, 0 none */
    const float *normal;         /* float4: unit geometric normal xyz */
    const uint32_t *identity;    /* uint32 x 2: raster identity of the pixel's surface (receiverSame) */
    float previous_clip_from_world[16]; /* the previous frame's camera, row-major; reprojects history */
    float dirty_lo[3], dirty_hi[3];     /* dirtyMin / dirtyMax: no history is reused inside */
    uint32_t dirty;              /* 1: the dirty box applies */
    uint32_t scene_changed;      /* stability.y: a global change this frame (reactive blend, radiometric steps) */
    uint32_t spatial_filter_steps; /* RadianceCascades::spatial_filter_steps, 0..=4 */
    uint32_t reserved;
} LuxScreenFrame;
typedef struct LuxScreen LuxScreen;
lux_status lux_screen_create(LuxContext *ctx, uint32_t width, uint32_t height, LuxScreen **out);
lux_status lux_screen_destroy(LuxScreen *screen);
/* The next frame has no screen history (stability.x = 0). */
lux_status lux_screen_reset(LuxScreen *screen);
/* One frame: temporal (reads settings temporal_blend, history_frames,
 * probe_spacing, normal_bias), then the spatial passes; `out` is a device
 * float4[width * height] (rgb, depth or 0 without lighting support). */
lux_status lux_screen_filter(LuxScreen *screen, const LuxSettings *settings, const LuxScreenFrame *frame,
                             float *out);
/* Copies the screen history to host memory (tests): irradiance float4 (rgb,
 * depth or 0) and metadata float4 (retained length, variance, support mask,
 * surface flag) per pixel; either pointer may be NULL. */
lux_status lux_screen_read_history(LuxScreen *screen, float *irradiance, float *metadata);

#ifdef __cplusplus
}
#endif
#endif /* LUX_H */
