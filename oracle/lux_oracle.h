/*
 * lux_oracle.h - CPU restatement of the Split Radiance Cascades transport
 * path of bevy_lux (HyperExtendedReality/bevy_penumbra).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for liblux:
 * only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * load it.  The product never links, loads or calls it.
 *
 * Every function restates a reference function; the citation is given at the
 * definition in lux_oracle.c.  Parity is pinned against the reference's own
 * known-answer tests (tests/test_oracle_golden.py): the deposit KAT
 * (src/transport_tests.rs:3637-3829), the merge / support KATs
 * (src/split_merge_tests.rs:13-305, 1298-1430), the resolve references
 * (src/world_resolve_tests.rs:31-309), the dense-SDF direction mapping
 * (src/transport_tests.rs:179-248, 3830-4107) and the traversal brute force
 * (src/traversal_tests.rs:978-1125).
 *
 * Record layouts are the ones of include/lux.h (LuxRay, LuxHit, LuxLight,
 * LuxSettings), so a test can hand the same bytes to both libraries.
 */
#ifndef LUX_ORACLE_H
#define LUX_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#include "../include/lux.h"

#ifdef __cplusplus
extern "C" {
#endif

/* --- direction / key math (shaders/common.slang) --------------------- */
void orc_sincos_turns(float turns, float *c, float *s);
void orc_decode_direction(float u, float v, float out[3]);
void orc_bin_direction(uint32_t index, uint32_t columns, uint32_t rows, float out[3]);
uint32_t orc_direction_index_uv(float u, float v, uint32_t columns, uint32_t rows);
void orc_r2(uint32_t index, float out[2]);
uint32_t orc_transport_hash(uint32_t value);
uint32_t orc_hash_key(const int32_t key[4], uint32_t bucket_count);
void orc_ray_offset(const float position[3], const float normal[3], float bias, float out[3]);
void orc_encode_normal(const float n[3], float out[2]);
void orc_decode_normal(const float p[2], float out[3]);
float orc_interval_end(const LuxSettings *s, uint32_t level);
float orc_spacing(const LuxSettings *s, uint32_t level);

/* --- scene over the reference word streams ---------------------------- */
typedef struct OrcScene OrcScene;
OrcScene *orc_scene_create(const uint32_t *scene_words, size_t scene_word_count,
                           const uint32_t *geometry_words, size_t geometry_word_count,
                           const LuxLight *lights, uint32_t light_count,
                           uint32_t conventional_lights);
void orc_scene_destroy(OrcScene *scene);
int orc_scene_refit(OrcScene *scene, const float *world_from_local, uint32_t count);
void orc_scene_words(const OrcScene *scene, uint32_t *out);

typedef struct OrcCounters {
    uint64_t nodes;      /* binary BVH nodes whose box was tested */
    uint64_t triangles;  /* triangle tests */
    uint64_t instances;  /* instance transforms */
} OrcCounters;

/* traceRayTracked / traceRay (shaders/traversal.slang:696-819), closest hit. */
void orc_trace_closest(const OrcScene *scene, const float origin[3], const float direction[3],
                       float tmin, float limit, LuxHit *hit, OrcCounters *counters);
/* traceOccluded (shaders/traversal.slang:955-1046). Returns blocked; *supported. */
int orc_trace_occluded(const OrcScene *scene, const float origin[3], const float direction[3],
                       float limit, int *supported, OrcCounters *counters);
/* Same triangle test as the traversal, applied to every triangle (no BVH). */
void orc_brute_closest(const OrcScene *scene, const float origin[3], const float direction[3],
                       float tmin, float limit, LuxHit *hit);
/* The f64 Moller-Trumbore brute force of src/traversal_tests.rs:978-1038:
 * writes up to `capacity` (t, triangle, instance) candidates sorted by t and
 * returns how many exist. */
uint32_t orc_brute_f64(const OrcScene *scene, const float origin[3], const float direction[3],
                       float limit, double *t, uint32_t *triangle, uint32_t *instance,
                       uint32_t capacity);
/* Batched harness: one LuxHit per LuxRay, `threads` host threads. */
void orc_trace_rays(const OrcScene *scene, const LuxRay *rays, uint32_t count, int any_hit,
                    LuxHit *hits, int threads, OrcCounters *counters);

/* outgoingTransportRadianceTracked (shaders/cascades.slang:196-268) for the
 * synthetic-material subset.  Returns supported. */
int orc_outgoing_radiance(const OrcScene *scene, const LuxSettings *settings,
                          const float origin[3], const float direction[3], const LuxHit *hit,
                          float out[3], uint64_t *shadow_rays, OrcCounters *counters);

/* transportRandom and cosineDirection (shaders/common.slang:292-295,
 * 407-412), and the constant-environment estimator of
 * environmentResponseTracked (shaders/environment.slang:154-230): count
 * samples of sequence base `sequence_base`; `visibility` negative traces the
 * scene, 0/1/2 stub every query as visible/blocked/unsupported (scene may
 * then be NULL).  Returns supported. */
/* Each Split receiver's place in the sample sequence (receiver i's ray k
 * uses R2 index out[i] x R + k): LOD, then the Morton order of the cascade-0
 * cell, then the receiver index; absent receivers (sparse, position.w == 0)
 * last (shaders/split.slang:788-963). */
void orc_sequence_order(const LuxSettings *settings, const LuxCamera *camera, const float *pos, uint32_t n,
                        int sparse, uint32_t *out);
float orc_transport_random(uint32_t seed, uint32_t lane);
void orc_cosine_direction_frame(const float n[3], float u1, float u2, float out[3]);
int orc_environment_response(const OrcScene *scene, const float environment[3], float probe_spacing, float bias,
                             uint32_t count, uint32_t sequence_base, const float position[3], const float normal[3],
                             const float gnormal[3], const float view[3], float roughness, const float diffuse[3],
                             int visibility, float out[3], uint64_t *shadow_rays, OrcCounters *counters);

/* FP64 reference irradiance (lux_reference_irradiance restated; `round` =
 * lux_reference_round_samples(count, spp)); out double4[count]. */
void orc_reference_sample(uint32_t p, uint32_t s, uint32_t seed, float *u1, float *u2);
void orc_cosine_direction(const float n[3], float u1, float u2, float out[3]);
void orc_reference_irradiance(const OrcScene *scene, const LuxSettings *settings, const float *position,
                              const float *normal, uint32_t count, uint32_t spp, uint32_t seed, uint32_t round,
                              double *out);

/* --- one cascade frame ---------------------------------------------------- */
typedef struct OrcFrame OrcFrame;
/* A frame that takes history from `previous` (NULL: none; settings must be
 * sanitized): records of the previous frame with the same key blend in as
 * lux_view_trace_merge does; `dirty` holds dirty_count boxes (lo xyz, hi xyz)
 * whose nearby records take no history. */
OrcFrame *orc_frame_run_history(const OrcScene *scene, const LuxSettings *settings, const float *receiver_position,
                                const float *receiver_normal, uint32_t receiver_count, int threads,
                                const OrcFrame *previous, const float *dirty, uint32_t dirty_count);
/* orc_frame_run_history with the view capacities that bound the retained
 * cells of the previous frame (max_cells per level, max_entries records). */
OrcFrame *orc_frame_run_retain(const OrcScene *scene, const LuxSettings *settings, const float *receiver_position,
                               const float *receiver_normal, uint32_t receiver_count, int threads,
                               const OrcFrame *previous, const float *dirty, uint32_t dirty_count,
                               uint32_t max_cells, uint64_t max_entries);
/* Multi-bounce roles (RadianceCascades::multi_bounce): ORC_FRAME_SPARSE,
 * receivers with position.w == 0 are absent; ORC_FRAME_SKIP_EMISSION, hits
 * add no emission of their own (the secondary cache); ORC_FRAME_RECORD_HITS,
 * the surface of each receiver's ray frame % R (position, 1; geometric normal
 * facing the ray, 0) is written to hit_pos / hit_nrm (float4 per receiver,
 * untouched where there is none).  `feedback`: the secondary frame whose
 * cascade-0 probes add diffuse bounce light at every hit (NULL: none). */
#define ORC_FRAME_SPARSE 1u
#define ORC_FRAME_SKIP_EMISSION 2u
#define ORC_FRAME_RECORD_HITS 4u
/* cachedHitSky (RadianceCascades::cached_hit_sky): with ORC_FRAME_SKIP_EMISSION
 * escaped rays carry the environment; hits the feedback frame covers take no
 * environment samples. */
#define ORC_FRAME_CACHED_SKY 8u
OrcFrame *orc_frame_run_bounce(const OrcScene *scene, const LuxSettings *settings, const float *receiver_position,
                               const float *receiver_normal, uint32_t receiver_count, int threads,
                               const OrcFrame *previous, const float *dirty, uint32_t dirty_count,
                               uint32_t max_cells, uint64_t max_entries, const OrcFrame *feedback, uint32_t flags,
                               float *hit_pos, float *hit_nrm, const LuxCamera *camera);
/* splitLodBlendForParameters of one point (camera NULL or disabled: 0, 0, 0). */
void orc_lod_blend(const LuxSettings *settings, const LuxCamera *camera, const float position[3], uint32_t *low,
                   uint32_t *high, float *blend);
/* Screen reconstruction (temporal + denoise, shaders/cascades.slang:310-690):
 * inputs per pixel of a width x height image (row-major): irradiance float4
 * (resolve output), position float4 (xyz, view depth), normal float4, identity
 * uint32 x 2; `dirty` = 6 floats (lo, hi) or NULL.  history_in / history_out:
 * ORC_SCREEN_WORDS floats per pixel (irradiance rgb + depth; retained length,
 * variance, support mask, surface flag; position; normal; identity bits).
 * `out` float4 per pixel. */
#define ORC_SCREEN_WORDS 18
void orc_screen_filter(const LuxSettings *settings, uint32_t width, uint32_t height, const float *irradiance,
                       const float *position, const float *normal, const uint32_t *identity,
                       const float previous_clip_from_world[16], const float *dirty, uint32_t scene_changed,
                       uint32_t spatial_filter_steps, uint32_t history_valid, const float *history_in,
                       float *history_out, float *out);
void orc_history_blend(const LuxSettings *settings, uint32_t samples, const float fresh[4], const float *old,
                       const float *old_mass, float out[4], float mass[2]);
OrcFrame *orc_frame_run(const OrcScene *scene, const LuxSettings *settings,
                        const float *receiver_position, const float *receiver_normal,
                        uint32_t receiver_count, int threads);
void orc_frame_destroy(OrcFrame *frame);
/* The path-traced reference (lux_path_reference's restatement): one sample's
 * radiance (0 when a trace is unsupported), and per point the FP64 mean over
 * spp samples (out double4[count]: rgb, supported samples). */
float orc_path_random(uint32_t p, uint32_t s, uint32_t seed, uint32_t dim);
int orc_path_sample(const OrcScene *scene, const LuxSettings *settings, uint32_t bounces, uint32_t seed, uint32_t p,
                    const float position[3], const float normal[3], uint32_t s, float radiance[3]);
void orc_path_reference(const OrcScene *scene, const LuxSettings *settings, const float *position,
                        const float *normal, uint32_t count, uint32_t spp, uint32_t bounces, uint32_t seed,
                        int threads, double *out);

/* The oracle's scene packer (orc_pack.c): build_tree / node_words /
 * pack_instances / geometry_words / build_emissive_lights restated in C.
 * Inputs as lux_scene_pack; returns 0, or -1 for invalid input. */
typedef struct OrcPacked OrcPacked;
int orc_scene_pack(const float *positions, uint32_t vertex_count, const uint32_t *indices, uint32_t triangle_count,
                   const uint32_t *mesh_first_triangle, const uint32_t *mesh_triangle_count, uint32_t mesh_count,
                   const uint32_t *instance_mesh, const float *instance_world_from_local,
                   const uint32_t *instance_flags, const uint32_t *instance_material, uint32_t instance_count,
                   const uint32_t *material_words, uint32_t material_count, OrcPacked **out);
void orc_packed_sizes(const OrcPacked *p, size_t *scene_words, size_t *geometry_words, uint32_t *lights,
                      uint32_t *tlas_nodes, uint32_t *blas_nodes, uint32_t *max_depth, double *blas_cost);
void orc_packed_copy(const OrcPacked *p, uint32_t *scene_words, uint32_t *geometry_words, LuxLight *lights,
                     uint32_t *instance_order, uint32_t instance_count);
void orc_packed_destroy(OrcPacked *p);
/* Split frames: the closest hit of each interval ray (receiver i, ray k at
 * index i x rays_per_receiver + k); returns the records copied. */
uint64_t orc_frame_read_hits(const OrcFrame *frame, LuxHit *out, uint64_t count);
uint32_t orc_frame_cells(const OrcFrame *frame, uint32_t level);
/* cell keys int4[cells] sorted ascending; merged/raw float4[cells*dirs];
 * samples uint32[cells*dirs]; any pointer may be NULL. */
void orc_frame_read_level(const OrcFrame *frame, uint32_t level, int32_t *keys, float *merged,
                          float *raw, uint32_t *samples);
/* packed cascade-0 tables float4[cells*36], same cell order as level 0. */
void orc_frame_read_probes(const OrcFrame *frame, float *tables);
void orc_frame_stats(const OrcFrame *frame, LuxStats *stats);
void orc_frame_resolve(const OrcFrame *frame, const float *position, const float *normal,
                       uint32_t count, float *out);

/* Resolve over given cascade-0 tables: keys int4[cells] (any order), tables
 * float4[cells*36], cascade-0 spacing. */
void orc_resolve_tables(const int32_t *keys, uint32_t cells, const float *tables, float spacing,
                        const float *position, const float *normal, uint32_t count, float *out);

/* --- stand-alone KAT entry points ------------------------------------ */
/* deposit (shaders/split.slang:1056-1117) of one ray at `distance` with
 * radiance rgb into `levels` (J.rgb, beta) records; returns the number of
 * levels written (later levels untouched). */
uint32_t orc_deposit_levels(const LuxSettings *s, float distance, int hit, int unsupported,
                            const float radiance[3], float *out_interval);
/* mergeEntry without history (shaders/split.slang:1624-1725): J, beta of one
 * entry at `level` with its 4 children x 8 corners merged records supplied
 * as child_merged[4][8] float4 (w <= 0 = missing) and the spatial fraction. */
void orc_merge_entry(const float interval[4], uint32_t samples, const float fraction[3],
                     const float *child_merged, int has_children, float out[4]);
/* mergeEntry with history for one entry: orc_history_blend of the fresh
 * interval with the previous record (old / old_mass may be NULL), then the
 * children as orc_merge_entry. */
void orc_merge_history_entry(const LuxSettings *settings, const float interval[4], uint32_t samples,
                             const float *old, const float *old_mass, const float fraction[3],
                             const float *child_merged, int has_children, float out[4]);
/* interpolateMergedChildSources, one source (shaders/split.slang:389-479). */
void orc_interpolate_children(const float fraction[3], const float *corner_merged, float out[4]);
/* packProbes texel table from base-direction merged values float4[dirs]. */
void orc_pack_table(const float *merged, uint32_t columns, uint32_t rows, float *table36);
/* irradianceLookup + diffuseProbePage on one table (shaders/world_resolve.slang:27-89). */
void orc_probe_lookup(const float *table36, const float normal[3], float out[4]);
/* Dense 16^3 SDF interval reference (src/transport_tests.rs:179-248) record i:
 * interval float4 and direction float4 (xyz, index). */
void orc_dense_sdf_record(uint32_t index, float interval[4], float direction[4]);

#ifdef __cplusplus
}
#endif
#endif
