/*
 * lux_oracle.c - CPU restatement of bevy_lux's Split transport path.
 *
 * TEST INFRASTRUCTURE ONLY (see lux_oracle.h).  Build: oracle/Makefile
 * (gcc -O2 -ffp-contract=off -fno-fast-math): every floating-point expression
 * below is evaluated in IEEE single precision in the order written, without
 * contraction, which is the evaluation contract liblux's kernels follow too
 * (nvcc --fmad=false).  Citations are paths inside the reference project.
 */
#define _GNU_SOURCE
#include "lux_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define EMPTY 0xffffffffu
#define MAX_TRAVERSAL_STEPS 4096u   /* shaders/traversal.slang:8 */
#define MAX_LEAF_TRIANGLES 256u     /* shaders/traversal.slang:9 */
#define MAX_LEAF_INSTANCES 4096u    /* shaders/traversal.slang:10 */
#define HIT_QUERY_UNSUPPORTED 4u    /* shaders/traversal.slang:16 */
#define STACK 49u                   /* shaders/traversal.slang:490, :712 */
#define PI_F 3.14159265358979323846f

static inline float saturatef(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
static inline float fracf(float x) { return x - floorf(x); }
static inline float asf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t asu(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline int finite3(const float v[3]) { return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]); }
static inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const float a[3], const float b[3], float o[3]) {
    float x = a[1] * b[2] - a[2] * b[1];
    float y = a[2] * b[0] - a[0] * b[2];
    float z = a[0] * b[1] - a[1] * b[0];
    o[0] = x; o[1] = y; o[2] = z;
}
static inline float length3(const float v[3]) { return sqrtf(dot3(v, v)); }

/* ======================================================================
 * Direction and key math (shaders/common.slang)
 * ==================================================================== */

/* cos and sin of 2*pi*turns.  The reference calls the GPU's cos/sin on
 * phi = uv.x * 2 * PI (decodeDirection, shaders/common.slang:376-382).  The
 * restatement reduces exactly to the nearest quarter turn and evaluates the
 * Taylor series of sin(2 pi r) and cos(2 pi r), |r| <= 1/8, to degree 11/10
 * (truncation error < 3e-8), so CPU and GPU agree bit for bit. */
#define SC_S1 6.2831855f
#define SC_S3 41.3417f
#define SC_S5 81.60525f
#define SC_S7 76.70586f
#define SC_S9 42.058693f
#define SC_S11 15.094643f
#define SC_C2 19.739208f
#define SC_C4 64.93939f
#define SC_C6 85.45682f
#define SC_C8 60.24464f
#define SC_C10 26.426256f
void orc_sincos_turns(float turns, float *c, float *s) {
    float k = floorf(turns * 4.0f + 0.5f);
    float r = turns - k * 0.25f;
    int q = ((int)k) & 3;
    float r2 = r * r;
    float sp = SC_S9 - r2 * SC_S11;
    sp = SC_S7 - r2 * sp;
    sp = SC_S5 - r2 * sp;
    sp = SC_S3 - r2 * sp;
    sp = SC_S1 - r2 * sp;
    float sn = r * sp;
    float cp = SC_C8 - r2 * SC_C10;
    cp = SC_C6 - r2 * cp;
    cp = SC_C4 - r2 * cp;
    cp = SC_C2 - r2 * cp;
    float cs = 1.0f - r2 * cp;
    switch (q) {
    case 0: *c = cs; *s = sn; break;
    case 1: *c = -sn; *s = cs; break;
    case 2: *c = -cs; *s = -sn; break;
    default: *c = sn; *s = -cs; break;
    }
}

/* decodeDirection, shaders/common.slang:376-382 (+Y is the polar axis). */
void orc_decode_direction(float u, float v, float out[3]) {
    float y = v * 2.0f - 1.0f;
    float r = sqrtf(fmaxf(0.0f, 1.0f - y * y));
    float c, s;
    orc_sincos_turns(u, &c, &s);
    out[0] = r * c;
    out[1] = y;
    out[2] = r * s;
}

/* binDirection, shaders/common.slang:395-400, for a columns x rows grid. */
void orc_bin_direction(uint32_t index, uint32_t columns, uint32_t rows, float out[3]) {
    float u = ((float)(index % columns) + 0.5f) / (float)columns;
    float v = ((float)(index / columns) + 0.5f) / (float)rows;
    orc_decode_direction(u, v, out);
}

/* directionIndex, shaders/common.slang:388-394, applied to the (u, v) that
 * encodeDirection returns for a direction decoded from (u, v). */
uint32_t orc_direction_index_uv(float u, float v, uint32_t columns, uint32_t rows) {
    uint32_t x = (uint32_t)(u * (float)columns);
    uint32_t y = (uint32_t)(v * (float)rows);
    if (x > columns - 1u) x = columns - 1u;
    if (y > rows - 1u) y = rows - 1u;
    return x + y * columns;
}

/* r2, shaders/common.slang:401-406. */
void orc_r2(uint32_t index, float out[2]) {
    uint32_t px = index * 3242174889u;
    uint32_t py = index * 2447445414u;
    out[0] = (float)(px >> 8) / 16777216.0f;
    out[1] = (float)(py >> 8) / 16777216.0f;
}

/* transportHash, shaders/common.slang:281-289. */
uint32_t orc_transport_hash(uint32_t value) {
    value ^= value >> 16;
    value *= 0x7feb352du;
    value ^= value >> 15;
    value *= 0x846ca68bu;
    value ^= value >> 16;
    return value;
}

/* hashKey, shaders/common.slang:423-429. */
uint32_t orc_hash_key(const int32_t key[4], uint32_t bucket_count) {
    uint32_t h = (uint32_t)key[0] * 0x8da6b343u ^ (uint32_t)key[1] * 0xd8163841u ^
                 (uint32_t)key[2] * 0xcb1ab31fu ^ (uint32_t)key[3] * 0x165667b1u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h & (bucket_count - 1u);
}

/* rayOffset, shaders/common.slang:343-359. */
void orc_ray_offset(const float position[3], const float normal[3], float bias, float out[3]) {
    for (int i = 0; i < 3; ++i) {
        float origin = position[i] + normal[i] * bias;
        int32_t step = (int32_t)(normal[i] * 256.0f);
        int32_t bits;
        memcpy(&bits, &origin, 4);
        int32_t moved = bits + (origin < 0.0f ? -step : step);
        float integer_offset;
        memcpy(&integer_offset, &moved, 4);
        float shifted = fabsf(origin) < 0.03125f ? origin + normal[i] / 65536.0f : integer_offset;
        out[i] = isfinite(shifted) ? shifted : position[i];
    }
}

/* encodeNormal, shaders/common.slang:360-366. */
void orc_encode_normal(const float n_in[3], float out[2]) {
    float d = (fabsf(n_in[0]) + fabsf(n_in[1])) + fabsf(n_in[2]);
    float n[3] = {n_in[0] / d, n_in[1] / d, n_in[2] / d};
    float p[2] = {n[0], n[1]};
    if (n[2] < 0.0f) {
        float px = (1.0f - fabsf(n[1])) * (p[0] >= 0.0f ? 1.0f : -1.0f);
        float py = (1.0f - fabsf(n[0])) * (p[1] >= 0.0f ? 1.0f : -1.0f);
        p[0] = px;
        p[1] = py;
    }
    out[0] = p[0] * 0.5f + 0.5f;
    out[1] = p[1] * 0.5f + 0.5f;
}

/* decodeNormal, shaders/common.slang:367-374 (normalize = v / length(v)). */
void orc_decode_normal(const float p_in[2], float out[3]) {
    float p[2] = {p_in[0] * 2.0f - 1.0f, p_in[1] * 2.0f - 1.0f};
    float n[3] = {p[0], p[1], (1.0f - fabsf(p[0])) - fabsf(p[1])};
    float t = saturatef(-n[2]);
    n[0] = n[0] + (n[0] >= 0.0f ? -t : t);
    n[1] = n[1] + (n[1] >= 0.0f ? -t : t);
    float l = length3(n);
    out[0] = n[0] / l;
    out[1] = n[1] / l;
    out[2] = n[2] / l;
}

/* splitIntervalEnd, shaders/split.slang:224-227, with the growth ratio and
 * rule as parameters (reference: end_L = length * 4^L). */
float orc_interval_end(const LuxSettings *s, uint32_t level) {
    if (s->interval_rule == LUX_INTERVAL_LENGTHS_GEOMETRIC) {
        float sum = 0.0f, term = 1.0f;
        for (uint32_t k = 0; k <= level; ++k) {
            sum += term;
            term *= s->interval_ratio;
        }
        return s->interval_length * sum;
    }
    float scale = 1.0f;
    for (uint32_t k = 0; k < level; ++k) scale *= s->interval_ratio;
    return s->interval_length * scale;
}

static float interval_start(const LuxSettings *s, uint32_t level) {
    return level == 0u ? 0.0f : orc_interval_end(s, level - 1u);
}

/* spacing, shaders/common.slang:413-416 (LOD 0). */
float orc_spacing(const LuxSettings *s, uint32_t level) {
    return s->probe_spacing * (float)(1u << level);
}

static inline uint32_t level_columns(const LuxSettings *s, uint32_t level) { return s->base_columns << level; }
static inline uint32_t level_rows(const LuxSettings *s, uint32_t level) { return s->base_rows << level; }

/* ======================================================================
 * Scene words (src/scene.rs:809-823, :1025-1122, :2096-2117)
 * ==================================================================== */
struct OrcScene {
    uint32_t *sw;
    size_t sn;
    uint32_t *gw;
    size_t gn;
    LuxLight *lights;
    uint32_t light_count;
    uint32_t conventional;
};

typedef struct { uint32_t x, y, z, w; } U4;

/* sceneInlineWord / geometryInlineWord: clamped reads
 * (shaders/traversal.slang:58-62, :114-118). */
static inline U4 sword(const OrcScene *S, uint32_t index) {
    U4 r = {0, 0, 0, 0};
    if (S->sn == 0) return r;
    if (index > S->sn - 1) index = (uint32_t)(S->sn - 1);
    memcpy(&r, S->sw + 4 * (size_t)index, 16);
    return r;
}
static inline U4 gword(const OrcScene *S, uint32_t index) {
    U4 r = {0, 0, 0, 0};
    if (S->gn == 0) return r;
    if (index > S->gn - 1) index = (uint32_t)(S->gn - 1);
    memcpy(&r, S->gw + 4 * (size_t)index, 16);
    return r;
}

OrcScene *orc_scene_create(const uint32_t *scene_words, size_t scene_word_count,
                           const uint32_t *geometry_words, size_t geometry_word_count,
                           const LuxLight *lights, uint32_t light_count, uint32_t conventional) {
    OrcScene *S = (OrcScene *)calloc(1, sizeof(OrcScene));
    S->sn = scene_word_count;
    S->gn = geometry_word_count;
    S->sw = (uint32_t *)malloc(16 * (scene_word_count ? scene_word_count : 1));
    S->gw = (uint32_t *)malloc(16 * (geometry_word_count ? geometry_word_count : 1));
    if (scene_word_count) memcpy(S->sw, scene_words, 16 * scene_word_count);
    if (geometry_word_count) memcpy(S->gw, geometry_words, 16 * geometry_word_count);
    S->light_count = light_count;
    S->conventional = conventional;
    S->lights = (LuxLight *)malloc(sizeof(LuxLight) * (light_count ? light_count : 1));
    if (light_count) memcpy(S->lights, lights, sizeof(LuxLight) * light_count);
    return S;
}

void orc_scene_destroy(OrcScene *S) {
    if (!S) return;
    free(S->sw);
    free(S->gw);
    free(S->lights);
    free(S);
}

typedef struct { float mn[3]; uint32_t first; float mx[3]; uint32_t count; } Node;


/* sceneNode, shaders/traversal.slang:192-196. */
static inline Node scene_node(const OrcScene *S, uint32_t index) {
    U4 a = sword(S, 1 + index * 2), b = sword(S, 2 + index * 2);
    Node n;
    n.mn[0] = asf(a.x); n.mn[1] = asf(a.y); n.mn[2] = asf(a.z); n.first = a.w;
    n.mx[0] = asf(b.x); n.mx[1] = asf(b.y); n.mx[2] = asf(b.z); n.count = b.w;
    return n;
}
static inline uint32_t instance_count(const OrcScene *S) { return sword(S, 0).z; }
/* instanceBase, shaders/traversal.slang:197-201. */
static inline uint32_t instance_base(const OrcScene *S, uint32_t instance) {
    U4 h = sword(S, 0);
    return h.y + instance * h.w;
}

static inline float word_f(uint32_t w) { return asf(w); }

/* refitTlas's transformed box for one instance (shaders/acceleration.slang:
 * 73-84): BLAS root box centre/extent through world_from_local (rows 3-5),
 * error (|t| + |M| max(|a|,|b|)) * 9.536743164e-7. */
static void refit_instance_box(const OrcScene *S, uint32_t instance, float mn[3], float mx[3]) {
    uint32_t base = sword(S, 0).y + instance * sword(S, 0).w;
    uint32_t root = sword(S, base + 8).x;
    U4 la = sword(S, 1 + root * 2), ub = sword(S, 2 + root * 2);
    float a[3] = {word_f(la.x), word_f(la.y), word_f(la.z)};
    float b[3] = {word_f(ub.x), word_f(ub.y), word_f(ub.z)};
    float center[3], extent[3], absolute[3];
    for (int k = 0; k < 3; ++k) {
        center[k] = a[k] * 0.5f + b[k] * 0.5f;
        extent[k] = b[k] * 0.5f - a[k] * 0.5f;
        absolute[k] = fmaxf(fabsf(a[k]), fabsf(b[k]));
    }
    for (int r = 0; r < 3; ++r) {
        U4 w = sword(S, base + 3 + r);
        float x = word_f(w.x), y = word_f(w.y), z = word_f(w.z), t = word_f(w.w);
        float wc = ((x * center[0] + y * center[1]) + z * center[2]) + t * 1.0f;
        float we = (fabsf(x) * extent[0] + fabsf(y) * extent[1]) + fabsf(z) * extent[2];
        float err = (fabsf(t) + ((fabsf(x) * absolute[0] + fabsf(y) * absolute[1]) + fabsf(z) * absolute[2])) *
                    9.536743164e-7f;
        mn[r] = (wc - we) - err;
        mx[r] = (wc + we) + err;
    }
}

static void put_word(OrcScene *S, uint32_t index, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    uint32_t *p = S->sw + 4 * (size_t)index;
    p[0] = x; p[1] = y; p[2] = z; p[3] = w;
}

static uint32_t fbits_u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* Rigid pose update (host instance upload, src/render.rs:3819-3915, then
 * refitTlas by depth, shaders/acceleration.slang:61-88).  Rows 0-2 get
 * local_from_world (f64 inverse rounded to f32), rows 3-5 world_from_local;
 * TLAS nodes are refit deepest depth first.  Returns 0, or -1 for a count
 * mismatch / singular transform. */
int orc_scene_refit(OrcScene *S, const float *wfl, uint32_t count) {
    uint32_t n = instance_count(S);
    if (count != n) return -1;
    U4 h = sword(S, 0);
    for (uint32_t i = 0; i < n; ++i) {
        const float *m = wfl + 12 * (size_t)i;
        double w[3][4];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) w[r][c] = m[4 * r + c];
        double a = w[0][0], b = w[0][1], c = w[0][2], d = w[1][0], e = w[1][1], f = w[1][2], g = w[2][0],
               hh = w[2][1], k = w[2][2];
        double det = a * (e * k - f * hh) - b * (d * k - f * g) + c * (d * hh - e * g);
        if (!(fabs(det) > 0.0) || !isfinite(det)) return -1;
        double inv[3][3] = {{(e * k - f * hh) / det, (c * hh - b * k) / det, (b * f - c * e) / det},
                            {(f * g - d * k) / det, (a * k - c * g) / det, (c * d - a * f) / det},
                            {(d * hh - e * g) / det, (b * g - a * hh) / det, (a * e - b * d) / det}};
        uint32_t base = h.y + i * h.w;
        for (int r = 0; r < 3; ++r) {
            double t = -(inv[r][0] * w[0][3] + inv[r][1] * w[1][3] + inv[r][2] * w[2][3]);
            put_word(S, base + r, fbits_u((float)inv[r][0]), fbits_u((float)inv[r][1]), fbits_u((float)inv[r][2]),
                     fbits_u((float)t));
            put_word(S, base + 3 + r, fbits_u(m[4 * r]), fbits_u(m[4 * r + 1]), fbits_u(m[4 * r + 2]),
                     fbits_u(m[4 * r + 3]));
        }
    }
    if (n == 0) return 0;
    /* Depth of every TLAS node (DFS from node 0), then passes deepest first. */
    uint32_t node_total = (h.y - 1u) / 2u;
    uint32_t *depth = (uint32_t *)malloc(sizeof(uint32_t) * (node_total ? node_total : 1));
    uint8_t *in_tlas = (uint8_t *)calloc(node_total ? node_total : 1, 1);
    uint32_t *todo = (uint32_t *)malloc(sizeof(uint32_t) * (2 * (size_t)node_total + 2));
    uint32_t top = 0, max_depth = 0;
    todo[top++] = 0;
    depth[0] = 0;
    while (top) {
        uint32_t i = todo[--top];
        in_tlas[i] = 1;
        Node nd = scene_node(S, i);
        if (depth[i] > max_depth) max_depth = depth[i];
        if (nd.count == 0 && nd.first + 1 < node_total) {
            depth[nd.first] = depth[nd.first + 1] = depth[i] + 1;
            todo[top++] = nd.first;
            todo[top++] = nd.first + 1;
        }
    }
    for (int64_t dd = max_depth; dd >= 0; --dd)
        for (uint32_t i = 0; i < node_total; ++i) {
            if (!in_tlas[i] || depth[i] != (uint32_t)dd) continue;
            U4 lower = sword(S, 1 + i * 2), upper = sword(S, 2 + i * 2);
            float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
            float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
            if (upper.w == 0) {
                Node c0 = scene_node(S, lower.w), c1 = scene_node(S, lower.w + 1);
                for (int k = 0; k < 3; ++k) {
                    mn[k] = fminf(c0.mn[k], c1.mn[k]);
                    mx[k] = fmaxf(c0.mx[k], c1.mx[k]);
                }
            } else {
                for (uint32_t inst = lower.w; inst < lower.w + upper.w; ++inst) {
                    float a[3], b[3];
                    refit_instance_box(S, inst, a, b);
                    for (int k = 0; k < 3; ++k) {
                        mn[k] = fminf(mn[k], a[k]);
                        mx[k] = fmaxf(mx[k], b[k]);
                    }
                }
            }
            put_word(S, 1 + i * 2, fbits_u(mn[0]), fbits_u(mn[1]), fbits_u(mn[2]), lower.w);
            put_word(S, 2 + i * 2, fbits_u(mx[0]), fbits_u(mx[1]), fbits_u(mx[2]), upper.w);
        }
    free(depth);
    free(in_tlas);
    free(todo);
    return 0;
}

/* The scene words (after refits): out[sn * 4]. */
void orc_scene_words(const OrcScene *S, uint32_t *out) { memcpy(out, S->sw, 16 * S->sn); }

/* localTriangle, shaders/traversal.slang:158-173. */
static void local_triangle(const OrcScene *S, uint32_t triangle, U4 header, float a[3], float b[3],
                           float c[3], uint32_t idx[3]) {
    U4 t = gword(S, header.x + triangle);
    idx[0] = t.x; idx[1] = t.y; idx[2] = t.z;
    U4 va = gword(S, header.y + t.x * header.z);
    U4 vb = gword(S, header.y + t.y * header.z);
    U4 vc = gword(S, header.y + t.z * header.z);
    a[0] = asf(va.x); a[1] = asf(va.y); a[2] = asf(va.z);
    b[0] = asf(vb.x); b[1] = asf(vb.y); b[2] = asf(vb.z);
    c[0] = asf(vc.x); c[1] = asf(vc.y); c[2] = asf(vc.z);
}

/* ======================================================================
 * Traversal (shaders/traversal.slang)
 * ==================================================================== */

/* boxRayInterval, shaders/traversal.slang:349-369, with the slab entry
 * padded down by 7.2e-7 relative like the GPU's child tests.  The reference
 * pads only the exit, so once a surface is found the box of another surface
 * within one rounding of it can be culled, and which of the two a query
 * returns depends on the order boxes are visited in (binary here, four-wide
 * on the GPU); with both ends padded every box holding a triangle at or
 * before the current distance is visited and the closest hit is the
 * smallest (distance, instance, triangle) over all triangles. */
static int box_interval(const float o[3], const float d[3], const Node *n, float limit, float *entry,
                        float *exit) {
    float near_t = 0.0f, far_t = limit;
    for (int axis = 0; axis < 3; ++axis) {
        if (d[axis] == 0.0f) {
            if (o[axis] < n->mn[axis] || o[axis] > n->mx[axis]) {
                *entry = 0.0f;
                *exit = 0.0f;
                return 0;
            }
        } else {
            float a = (n->mn[axis] - o[axis]) / d[axis];
            float b = (n->mx[axis] - o[axis]) / d[axis];
            float axis_exit = fmaxf(a, b);
            near_t = fmaxf(near_t, fminf(a, b));
            far_t = fminf(far_t, axis_exit + fabsf(axis_exit) * 3.5762791e-7f);
        }
    }
    near_t = near_t - fabsf(near_t) * 7.2e-7f;
    *entry = near_t;
    *exit = far_t;
    return near_t <= far_t;
}
static inline float box_entry(const float o[3], const float d[3], const Node *n, float limit) {
    float e, x;
    return box_interval(o, d, n, limit, &e, &x) ? e : -1.0f;
}

/* orientedEdge, shaders/traversal.slang:379-392. */
static inline float oriented_edge(const float a[2], const float b[2]) {
    int reverse = a[0] > b[0] || (a[0] == b[0] && a[1] > b[1]);
    const float *first = reverse ? b : a, *second = reverse ? a : b;
    float pa = first[0] * second[1];
    float pb = first[1] * second[0];
    float edge = pa - pb;
    float error = (fabsf(pa) + fabsf(pb)) * 2.3841858e-7f;
    if (fabsf(edge) <= error) edge = 0.0f;
    return reverse ? -edge : edge;
}

typedef struct { uint32_t kx, ky, kz; float sx, sy; int valid; } TriRay;

/* triangleRay, shaders/traversal.slang:399-413. */
static TriRay triangle_ray(const float d[3]) {
    TriRay r;
    memset(&r, 0, sizeof r);
    float m[3] = {fabsf(d[0]), fabsf(d[1]), fabsf(d[2])};
    r.kz = m[0] > m[1] ? (m[0] > m[2] ? 0 : 2) : (m[1] > m[2] ? 1 : 2);
    r.valid = d[r.kz] != 0.0f;
    if (!r.valid) return r;
    r.kx = (r.kz + 1) % 3;
    r.ky = (r.kx + 1) % 3;
    if (d[r.kz] < 0.0f) {
        uint32_t t = r.kx;
        r.kx = r.ky;
        r.ky = t;
    }
    r.sx = d[r.kx] / d[r.kz];
    r.sy = d[r.ky] / d[r.kz];
    return r;
}

/* intersectTriangle, shaders/traversal.slang:415-443.  Returns distance or
 * -1; w1, w2 = barycentric y, z. */
static float intersect_triangle(const float o[3], const float d[3], const TriRay *ray, const float A[3],
                                const float B[3], const float C[3], float *w1, float *w2) {
    if (!ray->valid) return -1.0f;
    uint32_t kx = ray->kx, ky = ray->ky, kz = ray->kz;
    float a[3] = {A[0] - o[0], A[1] - o[1], A[2] - o[2]};
    float b[3] = {B[0] - o[0], B[1] - o[1], B[2] - o[2]};
    float c[3] = {C[0] - o[0], C[1] - o[1], C[2] - o[2]};
    float pa[2] = {a[kx] - ray->sx * a[kz], a[ky] - ray->sy * a[kz]};
    float pb[2] = {b[kx] - ray->sx * b[kz], b[ky] - ray->sy * b[kz]};
    float pc[2] = {c[kx] - ray->sx * c[kz], c[ky] - ray->sy * c[kz]};
    float largest = fmaxf(fmaxf(fmaxf(fabsf(pa[0]), fabsf(pa[1])), fmaxf(fabsf(pb[0]), fabsf(pb[1]))),
                          fmaxf(fabsf(pc[0]), fabsf(pc[1])));
    if (largest == 0.0f || !isfinite(largest)) return -1.0f;
    uint32_t exponent = (asu(largest) >> 23) & 255u;
    if (exponent < 1u) exponent = 1u;
    if (exponent > 253u) exponent = 253u;
    float scale = asf((254u - exponent) << 23);
    pa[0] *= scale; pa[1] *= scale;
    pb[0] *= scale; pb[1] *= scale;
    pc[0] *= scale; pc[1] *= scale;
    float e0 = oriented_edge(pb, pc), e1 = oriented_edge(pc, pa), e2 = oriented_edge(pa, pb);
    int any_neg = e0 < 0.0f || e1 < 0.0f || e2 < 0.0f;
    int any_pos = e0 > 0.0f || e1 > 0.0f || e2 > 0.0f;
    if (any_neg && any_pos) return -1.0f;
    float det = (e0 + e1) + e2;
    if (det == 0.0f || !isfinite(det)) return -1.0f;
    float wx = e0 / det, wy = e1 / det, wz = e2 / det;
    float dist = ((wx * a[kz] + wy * b[kz]) + wz * c[kz]) / d[kz];
    if (!isfinite(dist)) return -1.0f;
    *w1 = wy;
    *w2 = wz;
    return dist;
}

/* Deterministic closest-hit order: smaller distance, then (instance,
 * triangle).  The reference keeps the first of equal distances found by its
 * depth-first order (strict `<`, shaders/traversal.slang:457); an explicit
 * key makes the answer independent of the BVH shape. */
static inline int hit_better(float t, uint32_t instance, uint32_t triangle, const LuxHit *h) {
    if (t < h->distance) return 1;
    if (t > h->distance || h->triangle == EMPTY) return 0;
    if (instance != h->instance) return instance < h->instance;
    return triangle < h->triangle;
}

static inline int cull_reject(uint32_t flags, const float A[3], const float B[3], const float C[3],
                              const float d[3]) {
    if ((flags & 3u) == 0u) return 0;
    float e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    float e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
    float cr[3];
    cross3(e1, e2, cr);
    float facing = dot3(cr, d) * ((flags & 4u) != 0u ? -1.0f : 1.0f);
    return ((flags & 1u) != 0u && facing >= 0.0f) || ((flags & 2u) != 0u && facing <= 0.0f);
}

/* traceTriangle, shaders/traversal.slang:445-473 (opaque materials). */
static void trace_triangle(const OrcScene *S, const float lo[3], const float ld[3], const TriRay *ray,
                           uint32_t tri, uint32_t instance, uint32_t flags, U4 header, float tmin,
                           LuxHit *hit, OrcCounters *cn) {
    float A[3], B[3], C[3];
    uint32_t idx[3];
    local_triangle(S, tri, header, A, B, C, idx);
    if (cn) cn->triangles++;
    if (cull_reject(flags, A, B, C, ld)) return;
    float w1 = 0, w2 = 0;
    float t = intersect_triangle(lo, ld, ray, A, B, C, &w1, &w2);
    if (t > 0.000025f && t > tmin && hit_better(t, instance, tri, hit)) {
        hit->distance = t;
        hit->triangle = tri;
        hit->instance = instance;
        hit->barycentric[0] = (1.0f - w1) - w2;
        hit->barycentric[1] = w1;
        hit->barycentric[2] = w2;
    }
}

/* Local ray of an instance: rows 0-2 of the record (local_from_world),
 * shaders/traversal.slang:481-488. */
static void local_ray(const OrcScene *S, uint32_t base, const float o[3], const float d[3], float lo[3],
                      float ld[3]) {
    for (int r = 0; r < 3; ++r) {
        U4 w = sword(S, base + (uint32_t)r);
        float x = asf(w.x), y = asf(w.y), z = asf(w.z), t = asf(w.w);
        lo[r] = ((x * o[0] + y * o[1]) + z * o[2]) + t * 1.0f;
        ld[r] = ((x * d[0] + y * d[1]) + z * d[2]) + t * 0.0f;
    }
}

/* traceInstance, shaders/traversal.slang:474-566 (closest hit). */
static void trace_instance(const OrcScene *S, const float o[3], const float d[3], uint32_t instance,
                           U4 header, float tmin, LuxHit *hit, OrcCounters *cn) {
    uint32_t base = instance_base(S, instance);
    U4 record = sword(S, base + 6);
    float lo[3], ld[3];
    local_ray(S, base, o, d, lo, ld);
    if (cn) cn->instances++;
    uint32_t flags = record.w;
    uint32_t stack_node[STACK];
    float stack_t[STACK];
    uint32_t count = 0;
    U4 geometry = sword(S, base + 8);
    Node node = scene_node(S, geometry.x);
    if (cn) cn->nodes++;
    int ready = box_entry(lo, ld, &node, hit->distance) >= 0.0f;
    TriRay ray;
    memset(&ray, 0, sizeof ray);
    if (ready) ray = triangle_ray(ld);
    uint32_t steps = 0;
    while (ready || count != 0) {
        if (++steps > MAX_TRAVERSAL_STEPS) {
            hit->errors |= HIT_QUERY_UNSUPPORTED;
            break;
        }
        if (!ready) {
            --count;
            if (stack_t[count] > hit->distance) continue;
            node = scene_node(S, stack_node[count]);
        }
        ready = 0;
        if (node.count == 0) {
            if (count + 2 > STACK) {
                hit->errors |= 1u;
                node.first = geometry.y;
                node.count = geometry.z;
                count = 0;
            } else {
                uint32_t li = node.first, ri = li + 1;
                Node ln = scene_node(S, li), rn = scene_node(S, ri);
                if (cn) cn->nodes += 2;
                float le = box_entry(lo, ld, &ln, hit->distance);
                float re = box_entry(lo, ld, &rn, hit->distance);
                if (le >= 0.0f && re >= 0.0f) {
                    if (le <= re) {
                        stack_node[count] = ri; stack_t[count] = re; ++count;
                        node = ln;
                    } else {
                        stack_node[count] = li; stack_t[count] = le; ++count;
                        node = rn;
                    }
                    ready = 1;
                } else if (le >= 0.0f) {
                    node = ln;
                    ready = 1;
                } else if (re >= 0.0f) {
                    node = rn;
                    ready = 1;
                }
                continue;
            }
        }
        uint32_t begin = node.first > geometry.y ? node.first : geometry.y;
        uint32_t limit_tri = geometry.y + geometry.z;
        uint32_t requested_end = node.first + node.count;
        uint32_t end = requested_end < limit_tri ? requested_end : limit_tri;
        int truncated = node.first < geometry.y || requested_end < node.first ||
                        requested_end > limit_tri || node.count > MAX_LEAF_TRIANGLES;
        uint32_t bounded = end < begin + MAX_LEAF_TRIANGLES ? end : begin + MAX_LEAF_TRIANGLES;
        truncated = truncated || bounded < end;
        if (truncated) hit->errors |= HIT_QUERY_UNSUPPORTED;
        for (uint32_t i = begin; i < bounded; ++i)
            trace_triangle(S, lo, ld, &ray, i, instance, flags, header, tmin, hit, cn);
    }
}

/* traceRayTracked, shaders/traversal.slang:696-811 (software path, no
 * admission budget).  `tmin` extends the reference: hits must also satisfy
 * t > tmin (dense-layout intervals start there). */
void orc_trace_closest(const OrcScene *S, const float o[3], const float d[3], float tmin, float limit,
                       LuxHit *hit, OrcCounters *cn) {
    memset(hit, 0, sizeof *hit);
    hit->distance = limit;
    hit->triangle = EMPTY;
    hit->instance = EMPTY;
    uint32_t instances = instance_count(S);
    if (instances == 0) return;
    uint32_t stack_node[STACK];
    float stack_t[STACK];
    uint32_t count = 0;
    Node node = scene_node(S, 0);
    if (cn) cn->nodes++;
    float root_entry, root_exit;
    if (!box_interval(o, d, &node, hit->distance, &root_entry, &root_exit)) return;
    U4 header = gword(S, 0);
    int ready = root_entry >= 0.0f;
    uint32_t steps = 0;
    while (ready || count != 0) {
        if (++steps > MAX_TRAVERSAL_STEPS) {
            hit->errors |= HIT_QUERY_UNSUPPORTED;
            break;
        }
        if (!ready) {
            --count;
            if (stack_t[count] > hit->distance) continue;
            node = scene_node(S, stack_node[count]);
        }
        ready = 0;
        if (node.count == 0) {
            if (count + 2 > STACK) {
                hit->errors |= 2u;
                node.first = 0;
                node.count = instances;
                count = 0;
            } else {
                uint32_t li = node.first, ri = li + 1;
                Node ln = scene_node(S, li), rn = scene_node(S, ri);
                if (cn) cn->nodes += 2;
                float le = box_entry(o, d, &ln, hit->distance);
                float re = box_entry(o, d, &rn, hit->distance);
                if (le >= 0.0f && re >= 0.0f) {
                    if (le <= re) {
                        stack_node[count] = ri; stack_t[count] = re; ++count;
                        node = ln;
                    } else {
                        stack_node[count] = li; stack_t[count] = le; ++count;
                        node = rn;
                    }
                    ready = 1;
                } else if (le >= 0.0f) {
                    node = ln;
                    ready = 1;
                } else if (re >= 0.0f) {
                    node = rn;
                    ready = 1;
                }
                continue;
            }
        }
        uint32_t requested_end = node.first + node.count;
        int truncated = requested_end < node.first || node.first > instances || requested_end > instances ||
                        node.count > MAX_LEAF_INSTANCES;
        uint32_t begin = node.first < instances ? node.first : instances;
        uint32_t end = requested_end < instances ? requested_end : instances;
        uint32_t bounded = end < begin + MAX_LEAF_INSTANCES ? end : begin + MAX_LEAF_INSTANCES;
        truncated = truncated || bounded < end;
        if (truncated) hit->errors |= HIT_QUERY_UNSUPPORTED;
        for (uint32_t i = begin; i < bounded; ++i) trace_instance(S, o, d, i, header, tmin, hit, cn);
    }
}

/* occludedTriangle, shaders/traversal.slang:826-843 (opaque materials). */
static int occluded_triangle(const OrcScene *S, const float lo[3], const float ld[3], const TriRay *ray,
                             uint32_t tri, uint32_t flags, float limit, U4 header, OrcCounters *cn) {
    float A[3], B[3], C[3];
    uint32_t idx[3];
    local_triangle(S, tri, header, A, B, C, idx);
    if (cn) cn->triangles++;
    if (cull_reject(flags, A, B, C, ld)) return 0;
    float w1, w2;
    float t = intersect_triangle(lo, ld, ray, A, B, C, &w1, &w2);
    return t > 0.000025f && t < limit;
}

/* occludedInstance, shaders/traversal.slang:845-932. */
static int occluded_instance(const OrcScene *S, const float o[3], const float d[3], uint32_t instance,
                             float limit, U4 header, int *supported, OrcCounters *cn) {
    *supported = 1;
    uint32_t base = instance_base(S, instance);
    U4 record = sword(S, base + 6);
    float lo[3], ld[3];
    local_ray(S, base, o, d, lo, ld);
    if (cn) cn->instances++;
    uint32_t flags = record.w;
    uint32_t stack_node[STACK];
    uint32_t count = 0;
    U4 geometry = sword(S, base + 8);
    Node node = scene_node(S, geometry.x);
    if (cn) cn->nodes++;
    int ready = box_entry(lo, ld, &node, limit) >= 0.0f;
    TriRay ray;
    memset(&ray, 0, sizeof ray);
    if (ready) ray = triangle_ray(ld);
    uint32_t steps = 0;
    int incomplete = 0;
    while (ready || count != 0) {
        if (++steps > MAX_TRAVERSAL_STEPS) {
            *supported = 0;
            return 0;
        }
        if (!ready) node = scene_node(S, stack_node[--count]);
        ready = 0;
        if (node.count == 0) {
            if (count + 2 > STACK) {
                node.first = geometry.y;
                node.count = geometry.z;
                count = 0;
            } else {
                uint32_t li = node.first, ri = li + 1;
                Node ln = scene_node(S, li), rn = scene_node(S, ri);
                if (cn) cn->nodes += 2;
                float le = box_entry(lo, ld, &ln, limit);
                float re = box_entry(lo, ld, &rn, limit);
                if (le >= 0.0f && re >= 0.0f) {
                    if (le <= re) {
                        stack_node[count++] = ri;
                        node = ln;
                    } else {
                        stack_node[count++] = li;
                        node = rn;
                    }
                    ready = 1;
                } else if (le >= 0.0f) {
                    node = ln;
                    ready = 1;
                } else if (re >= 0.0f) {
                    node = rn;
                    ready = 1;
                }
                continue;
            }
        }
        uint32_t begin = node.first > geometry.y ? node.first : geometry.y;
        uint32_t limit_tri = geometry.y + geometry.z;
        uint32_t requested_end = node.first + node.count;
        uint32_t end = requested_end < limit_tri ? requested_end : limit_tri;
        int truncated = node.first < geometry.y || requested_end < node.first ||
                        requested_end > limit_tri || node.count > MAX_LEAF_TRIANGLES;
        uint32_t bounded = end < begin + MAX_LEAF_TRIANGLES ? end : begin + MAX_LEAF_TRIANGLES;
        truncated = truncated || bounded < end;
        incomplete = incomplete || truncated;
        for (uint32_t i = begin; i < bounded; ++i)
            if (occluded_triangle(S, lo, ld, &ray, i, flags, limit, header, cn)) return 1;
    }
    *supported = !incomplete;
    return 0;
}

/* traceOccluded, shaders/traversal.slang:955-1046. */
int orc_trace_occluded(const OrcScene *S, const float o[3], const float d[3], float limit, int *supported,
                       OrcCounters *cn) {
    *supported = 1;
    uint32_t instances = instance_count(S);
    if (instances == 0) return 0;
    uint32_t stack_node[STACK];
    uint32_t count = 0;
    Node node = scene_node(S, 0);
    if (cn) cn->nodes++;
    float root_entry, root_exit;
    int intersects = box_interval(o, d, &node, limit, &root_entry, &root_exit);
    int ready = intersects && root_entry >= 0.0f;
    if (!ready) return 0;
    U4 header = gword(S, 0);
    uint32_t steps = 0;
    int incomplete = 0;
    while (ready || count != 0) {
        if (++steps > MAX_TRAVERSAL_STEPS) {
            *supported = 0;
            return 0;
        }
        if (!ready) node = scene_node(S, stack_node[--count]);
        ready = 0;
        if (node.count == 0) {
            if (count + 2 > STACK) {
                node.first = 0;
                node.count = instances;
                count = 0;
            } else {
                uint32_t li = node.first, ri = li + 1;
                Node ln = scene_node(S, li), rn = scene_node(S, ri);
                if (cn) cn->nodes += 2;
                float le = box_entry(o, d, &ln, limit);
                float re = box_entry(o, d, &rn, limit);
                if (le >= 0.0f && re >= 0.0f) {
                    if (le <= re) {
                        stack_node[count++] = ri;
                        node = ln;
                    } else {
                        stack_node[count++] = li;
                        node = rn;
                    }
                    ready = 1;
                } else if (le >= 0.0f) {
                    node = ln;
                    ready = 1;
                } else if (re >= 0.0f) {
                    node = rn;
                    ready = 1;
                }
                continue;
            }
        }
        uint32_t requested_end = node.first + node.count;
        int truncated = requested_end < node.first || node.first > instances || requested_end > instances ||
                        node.count > MAX_LEAF_INSTANCES;
        uint32_t begin = node.first < instances ? node.first : instances;
        uint32_t end = requested_end < instances ? requested_end : instances;
        uint32_t bounded = end < begin + MAX_LEAF_INSTANCES ? end : begin + MAX_LEAF_INSTANCES;
        incomplete = incomplete || truncated || bounded < end;
        for (uint32_t i = begin; i < bounded; ++i) {
            int inst_supported;
            int blocked = occluded_instance(S, o, d, i, limit, header, &inst_supported, cn);
            incomplete = incomplete || !inst_supported;
            if (blocked) {
                *supported = 1;
                return 1;
            }
        }
    }
    *supported = !incomplete;
    return 0;
}

void orc_brute_closest(const OrcScene *S, const float o[3], const float d[3], float tmin, float limit,
                       LuxHit *hit) {
    memset(hit, 0, sizeof *hit);
    hit->distance = limit;
    hit->triangle = EMPTY;
    hit->instance = EMPTY;
    U4 header = gword(S, 0);
    uint32_t instances = instance_count(S);
    for (uint32_t inst = 0; inst < instances; ++inst) {
        uint32_t base = instance_base(S, inst);
        U4 record = sword(S, base + 6);
        U4 geometry = sword(S, base + 8);
        float lo[3], ld[3];
        local_ray(S, base, o, d, lo, ld);
        TriRay ray = triangle_ray(ld);
        for (uint32_t tri = geometry.y; tri < geometry.y + geometry.z; ++tri)
            trace_triangle(S, lo, ld, &ray, tri, inst, record.w, header, tmin, hit, NULL);
    }
}

/* brute_force, src/traversal_tests.rs:978-1038 (Moller-Trumbore in world
 * space, f64, componentwise f32 uncertainty band). */
typedef struct { double t; uint32_t tri, inst; } F64Hit;
static int f64_cmp(const void *a, const void *b) {
    double x = ((const F64Hit *)a)->t, y = ((const F64Hit *)b)->t;
    return x < y ? -1 : (x > y ? 1 : 0);
}
uint32_t orc_brute_f64(const OrcScene *S, const float o[3], const float d[3], float limit, double *t_out,
                       uint32_t *tri_out, uint32_t *inst_out, uint32_t capacity) {
    U4 header = gword(S, 0);
    uint32_t instances = instance_count(S);
    size_t cap = 64, n = 0;
    F64Hit *hits = (F64Hit *)malloc(cap * sizeof(F64Hit));
    const double eps = 8.0 * (double)FLT_EPSILON;
    for (uint32_t inst = 0; inst < instances; ++inst) {
        uint32_t base = instance_base(S, inst);
        U4 record = sword(S, base + 6);
        U4 geometry = sword(S, base + 8);
        double m[3][4];
        for (int r = 0; r < 3; ++r) {
            U4 w = sword(S, base + 3 + (uint32_t)r);
            m[r][0] = asf(w.x); m[r][1] = asf(w.y); m[r][2] = asf(w.z); m[r][3] = asf(w.w);
        }
        for (uint32_t tri = geometry.y; tri < geometry.y + geometry.z; ++tri) {
            float A[3], B[3], C[3];
            uint32_t idx[3];
            local_triangle(S, tri, header, A, B, C, idx);
            const float *lv[3] = {A, B, C};
            double w[3][3];
            for (int v = 0; v < 3; ++v)
                for (int r = 0; r < 3; ++r)
                    w[v][r] = m[r][0] * lv[v][0] + m[r][1] * lv[v][1] + m[r][2] * lv[v][2] + m[r][3];
            double dir[3] = {d[0], d[1], d[2]}, org[3] = {o[0], o[1], o[2]};
            double e1[3], e2[3], nrm[3], p[3], q[3], rel[3];
            for (int k = 0; k < 3; ++k) {
                e1[k] = w[1][k] - w[0][k];
                e2[k] = w[2][k] - w[0][k];
                rel[k] = org[k] - w[0][k];
            }
#define DCROSS(a, b, o_) do { o_[0] = a[1]*b[2]-a[2]*b[1]; o_[1] = a[2]*b[0]-a[0]*b[2]; o_[2] = a[0]*b[1]-a[1]*b[0]; } while (0)
#define DDOT(a, b) (a[0]*b[0]+a[1]*b[1]+a[2]*b[2])
            DCROSS(e1, e2, nrm);
            double facing = DDOT(nrm, dir);
            uint32_t cull = record.w & 3u;
            if ((cull == 1 && facing >= 0.0) || (cull == 2 && facing <= 0.0)) continue;
            DCROSS(dir, e2, p);
            double det = DDOT(e1, p);
            if (det == 0.0) continue;
            double u = DDOT(rel, p) / det;
            DCROSS(rel, e1, q);
            double v = DDOT(dir, q) / det;
            double t = DDOT(e2, q) / det;
            double nl2 = DDOT(nrm, nrm);
            double gu[3], gv[3];
            DCROSS(e2, nrm, gu);
            DCROSS(nrm, e1, gv);
            for (int k = 0; k < 3; ++k) { gu[k] /= nl2; gv[k] /= nl2; }
            double err[3];
            for (int k = 0; k < 3; ++k)
                err[k] = (fabs(org[k]) + fabs(dir[k]) * fabs(t) + fabs(w[0][k]) + fabs(w[1][k]) + fabs(w[2][k])) * eps;
            double bu = fabs(gu[0]) * err[0] + fabs(gu[1]) * err[1] + fabs(gu[2]) * err[2];
            double bv = fabs(gv[0]) * err[0] + fabs(gv[1]) * err[1] + fabs(gv[2]) * err[2];
            double buv = fabs(gu[0] + gv[0]) * err[0] + fabs(gu[1] + gv[1]) * err[1] + fabs(gu[2] + gv[2]) * err[2];
            if (u < -bu || v < -bv || u + v > 1.0 + buv) continue;
            if (t > 0.000025 && t < (double)limit) {
                if (n == cap) {
                    cap *= 2;
                    hits = (F64Hit *)realloc(hits, cap * sizeof(F64Hit));
                }
                hits[n].t = t;
                hits[n].tri = tri;
                hits[n].inst = inst;
                ++n;
            }
#undef DCROSS
#undef DDOT
        }
    }
    qsort(hits, n, sizeof(F64Hit), f64_cmp);
    for (size_t i = 0; i < n && i < capacity; ++i) {
        t_out[i] = hits[i].t;
        tri_out[i] = hits[i].tri;
        inst_out[i] = hits[i].inst;
    }
    free(hits);
    return (uint32_t)n;
}

/* ---- threaded batch harness ---- */
typedef struct {
    const OrcScene *S;
    const LuxRay *rays;
    LuxHit *hits;
    uint32_t begin, end;
    int any_hit;
    OrcCounters cn;
} RayJob;

static void *ray_job(void *arg) {
    RayJob *j = (RayJob *)arg;
    for (uint32_t i = j->begin; i < j->end; ++i) {
        const LuxRay *r = &j->rays[i];
        LuxHit *h = &j->hits[i];
        if (j->any_hit) {
            int supported;
            int blocked = orc_trace_occluded(j->S, r->origin, r->direction, r->limit, &supported, &j->cn);
            memset(h, 0, sizeof *h);
            h->distance = r->limit;
            h->triangle = blocked ? 0u : EMPTY;
            h->instance = blocked ? 0u : EMPTY;
            h->errors = supported ? 0u : HIT_QUERY_UNSUPPORTED;
        } else {
            orc_trace_closest(j->S, r->origin, r->direction, r->tmin, r->limit, h, &j->cn);
        }
    }
    return NULL;
}

void orc_trace_rays(const OrcScene *S, const LuxRay *rays, uint32_t count, int any_hit, LuxHit *hits,
                    int threads, OrcCounters *counters) {
    if (threads < 1) threads = 1;
    if ((uint32_t)threads > count) threads = count ? (int)count : 1;
    RayJob *jobs = (RayJob *)calloc((size_t)threads, sizeof(RayJob));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        jobs[t].S = S;
        jobs[t].rays = rays;
        jobs[t].hits = hits;
        jobs[t].any_hit = any_hit;
        jobs[t].begin = (uint32_t)((uint64_t)count * t / threads);
        jobs[t].end = (uint32_t)((uint64_t)count * (t + 1) / threads);
        pthread_create(&tid[t], NULL, ray_job, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) {
        pthread_join(tid[t], NULL);
        if (counters) {
            counters->nodes += jobs[t].cn.nodes;
            counters->triangles += jobs[t].cn.triangles;
            counters->instances += jobs[t].cn.instances;
        }
    }
    free(jobs);
    free(tid);
}

/* ======================================================================
 * Hit shading (shaders/cascades.slang:57-268, shaders/traversal.slang:174-316)
 * ==================================================================== */

/* unitVector, shaders/traversal.slang:183-190. */
static void unit_vector(const float v[3], const float fallback[3], float out[3]) {
    float scale = fmaxf(fabsf(v[0]), fmaxf(fabsf(v[1]), fabsf(v[2])));
    if (scale == 0.0f || !isfinite(scale)) {
        out[0] = fallback[0]; out[1] = fallback[1]; out[2] = fallback[2];
        return;
    }
    float div = fmaxf(scale * 0.25f, FLT_MIN);
    float w[3] = {v[0] / div, v[1] / div, v[2] / div};
    float l = length3(w);
    out[0] = w[0] / l; out[1] = w[1] / l; out[2] = w[2] / l;
}

/* transformDirection, shaders/traversal.slang:229-244. */
static void transform_direction(const OrcScene *S, uint32_t base, const float value[3], int transpose,
                                float out[3]) {
    float r[3][3];
    for (int k = 0; k < 3; ++k) {
        U4 w = sword(S, base + (uint32_t)k);
        r[k][0] = asf(w.x); r[k][1] = asf(w.y); r[k][2] = asf(w.z);
    }
    float mag[3];
    for (int k = 0; k < 3; ++k) mag[k] = fmaxf(fabsf(r[0][k]), fmaxf(fabsf(r[1][k]), fabsf(r[2][k])));
    float scale = fmaxf(mag[0], fmaxf(mag[1], mag[2]));
    if (scale == 0.0f) {
        out[0] = out[1] = out[2] = 0.0f;
        return;
    }
    scale = fmaxf(scale * 0.25f, FLT_MIN);
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) r[k][c] = r[k][c] / scale;
    static const float zero[3] = {0, 0, 0};
    float v[3];
    unit_vector(value, zero, v);
    if (transpose) {
        for (int c = 0; c < 3; ++c) out[c] = (r[0][c] * v[0] + r[1][c] * v[1]) + r[2][c] * v[2];
    } else {
        for (int k = 0; k < 3; ++k) out[k] = dot3(r[k], v);
    }
}

/* triangleGeometricNormal, shaders/traversal.slang:250-253. */
static void geometric_normal(const OrcScene *S, uint32_t base, uint32_t flags, const float A[3],
                             const float B[3], const float C[3], float out[3]) {
    float e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    float e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
    float cr[3], t[3];
    cross3(e1, e2, cr);
    transform_direction(S, base, cr, 1, t);
    static const float up[3] = {0.0f, 1.0f, 0.0f};
    unit_vector(t, up, out);
    float sign = (flags & 4u) != 0u ? -1.0f : 1.0f;
    out[0] *= sign; out[1] *= sign; out[2] *= sign;
}

/* hitVertexAttribute, shaders/traversal.slang:174-182. */
static void vertex_attribute(const OrcScene *S, U4 header, const uint32_t idx[3], const float bary[3],
                             uint32_t attribute, float out[4]) {
    float acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        U4 w = gword(S, header.y + idx[i] * header.z + attribute);
        float v[4] = {asf(w.x), asf(w.y), asf(w.z), asf(w.w)};
        for (int c = 0; c < 4; ++c) acc[c] = i == 0 ? v[c] * bary[i] : acc[c] + v[c] * bary[i];
    }
    memcpy(out, acc, sizeof acc);
}

typedef struct {
    float base_color[3];
    float emission[3];
    float metallic, roughness;
    uint32_t flags;
} Surface;

/* materialBaseColor / hitEmission (shaders/material.slang:139-141,
 * shaders/traversal.slang:287-300) for untextured materials. */
static void surface_at(const OrcScene *S, const LuxSettings *st, uint32_t instance, uint32_t triangle,
                       const float bary[3], Surface *sf) {
    uint32_t base = instance_base(S, instance);
    uint32_t flags = sword(S, base + 6).w;
    uint32_t material = sword(S, base + 7).w;
    U4 m0 = sword(S, material), m1 = sword(S, material + 1), m2 = sword(S, material + 2);
    U4 header = gword(S, 0);
    U4 t = gword(S, header.x + triangle);
    uint32_t idx[3] = {t.x, t.y, t.z};
    float color[4];
    vertex_attribute(S, header, idx, bary, 4, color);
    sf->base_color[0] = asf(m0.x) * color[0];
    sf->base_color[1] = asf(m0.y) * color[1];
    sf->base_color[2] = asf(m0.z) * color[2];
    if ((flags & 16u) != 0u) {
        memcpy(sf->emission, sf->base_color, sizeof sf->emission);
    } else {
        sf->emission[0] = asf(m1.x);
        sf->emission[1] = asf(m1.y);
        sf->emission[2] = asf(m1.z);
    }
    float weight = (flags & 16u) != 0u ? 0.0f : asf(m2.w);
    float exposure = fmaxf(st->exposure, 1e-20f);
    float inv = 1.0f / exposure;
    float factor = inv + weight * (1.0f - inv);
    for (int c = 0; c < 3; ++c) sf->emission[c] = sf->emission[c] * factor;
    sf->metallic = asf(m2.x);
    sf->roughness = asf(m2.y);
    sf->flags = flags;
}

/* disneyDiffuseMultiplier, shaders/common.slang:298-314 (rsqrt written as
 * 1/sqrt, pow(x, 5) as bsdfPow5). */
static float disney_multiplier(const float n[3], const float l[3], const float v[3], float pr) {
    float ndl = saturatef(dot3(n, l));
    float ndv = saturatef(dot3(n, v));
    float h[3] = {l[0] + v[0], l[1] + v[1], l[2] + v[2]};
    float hl2 = dot3(h, h);
    if (ndl <= 0.0f || ndv <= 0.0f || hl2 <= 1e-20f) return 0.0f;
    float hl = sqrtf(hl2);
    float hv[3] = {h[0] / hl, h[1] / hl, h[2] / hl};
    float rough = fmaxf(saturatef(pr), 0.089f);
    rough = rough * rough;
    float ldh = saturatef(dot3(l, hv));
    float f90 = 0.5f + ((2.0f * rough) * ldh) * ldh;
    float a = 1.0f - ndl, b = 1.0f - ndv;
    float a2 = a * a, b2 = b * b;
    float light_scatter = 1.0f + (f90 - 1.0f) * ((a2 * a2) * a);
    float view_scatter = 1.0f + (f90 - 1.0f) * ((b2 * b2) * b);
    return light_scatter * view_scatter;
}

/* emissiveResponseTracked, shaders/cascades.slang:57-134; the scattering
 * response is the diffuse colour times the Disney diffuse factor / pi
 * (shaders/environment.slang:2-6 non-full branch, times bsdfDiffuseColor). */
static int emissive_response(const OrcScene *S, const LuxSettings *st, const float position[3],
                             const float normal[3], const float gnormal[3], const float view[3],
                             float roughness, const float diffuse[3], float out[3], uint64_t *shadow_rays,
                             OrcCounters *cn) {
    out[0] = out[1] = out[2] = 0.0f;
    uint32_t emissive = S->light_count - S->conventional;
    uint32_t count = st->emissive_samples / 2u;
    if (count < 1u) count = 1u;
    if (emissive == 0u) return 1;
    float cell = st->probe_spacing * 0.05f;
    int32_t k1[4] = {(int32_t)floorf(position[0] / cell), (int32_t)floorf(position[1] / cell),
                     (int32_t)floorf(position[2] / cell), 0};
    uint32_t seed = orc_hash_key(k1, 16777216u);
    float rotation[2];
    orc_r2(seed, rotation);
    float s0 = orc_spacing(st, 0);
    int32_t k2[4] = {(int32_t)floorf(position[0] / s0), (int32_t)floorf(position[1] / s0),
                     (int32_t)floorf(position[2] / s0), 0};
    uint32_t selection_seed = orc_hash_key(k2, 65536u);
    uint32_t sample_frame = st->frame_index ^ 0xE11E0001u;
    float ra[2], rb[2];
    orc_r2(sample_frame, ra);
    orc_r2(selection_seed, rb);
    float phase = fracf(ra[0] + rb[0]);
    float sum[3] = {0, 0, 0};
    const float bias = st->normal_bias;
    for (uint32_t sample = 0; sample < count; ++sample) {
        float rr[2];
        orc_r2(sample + sample_frame * count + 1u, rr);
        float uv[2] = {fracf(rr[0] + rotation[0]), fracf(rr[1] + rotation[1])};
        float selection = fracf(((float)sample + 0.5f) / (float)count + phase);
        uint32_t low = 0, high = emissive - 1u;
        while (low < high) {
            uint32_t middle = (low + high) / 2u;
            if (S->lights[S->conventional + middle].direction[3] < selection)
                low = middle + 1u;
            else
                high = middle;
        }
        const LuxLight *L = &S->lights[S->conventional + low];
        float rel[3] = {position[0] - L->position[0], position[1] - L->position[1], position[2] - L->position[2]};
        if (L->edge1[3] <= 0.0f || (L->position[3] != -2.0f && dot3(L->direction, rel) <= 0.0f)) continue;
        float root = sqrtf(uv[0]);
        float w1 = root * (1.0f - uv[1]), w2 = root * uv[1];
        float target[3];
        for (int c = 0; c < 3; ++c) target[c] = (L->position[c] + L->edge1[c] * w1) + L->edge2[c] * w2;
        float to_light[3] = {target[0] - position[0], target[1] - position[1], target[2] - position[2]};
        float light_distance = length3(to_light);
        if (light_distance <= bias * 0.25f) continue;
        float ldir[3] = {to_light[0] / light_distance, to_light[1] / light_distance, to_light[2] / light_distance};
        float cosine = fmaxf(0.0f, dot3(normal, ldir));
        float neg[3] = {-ldir[0], -ldir[1], -ldir[2]};
        float c_emit = dot3(L->direction, neg);
        if (L->position[3] == -2.0f) c_emit = fabsf(c_emit);
        float emitter_cosine = fmaxf(0.0f, c_emit);
        if (cosine <= 0.0f || emitter_cosine <= 0.0f || dot3(gnormal, ldir) <= 0.0f) continue;
        float bary[3] = {1.0f - root, w1, w2};
        Surface es;
        surface_at(S, st, L->source[0], L->source[1], bary, &es);
        float emission[3] = {fmaxf(es.emission[0], 0.0f), fmaxf(es.emission[1], 0.0f), fmaxf(es.emission[2], 0.0f)};
        if (!(emission[0] > 0.0f || emission[1] > 0.0f || emission[2] > 0.0f)) continue;
        float pdf = ((L->edge1[3] * light_distance) * light_distance) / (L->color[3] * emitter_cosine);
        float plane = fabsf(dot3(L->direction, rel));
        float origin[3];
        orc_ray_offset(position, gnormal, fminf(bias, plane * 0.25f), origin);
        float delta[3] = {target[0] - origin[0], target[1] - origin[1], target[2] - origin[2]};
        float distance = length3(delta);
        if (distance <= bias * 0.25f) continue;
        float dir[3] = {delta[0] / distance, delta[1] / distance, delta[2] / distance};
        int supported;
        if (shadow_rays) (*shadow_rays)++;
        int blocked = orc_trace_occluded(S, origin, dir, distance - fminf(bias * 0.25f, distance * 0.001f),
                                         &supported, cn);
        if (!supported) {
            out[0] = out[1] = out[2] = 0.0f;
            return 0;
        }
        if (blocked) continue;
        float factor = disney_multiplier(normal, ldir, view, roughness) / PI_F;
        float p = fmaxf(pdf, 1e-20f);
        for (int c = 0; c < 3; ++c) {
            float response = diffuse[c] * factor;
            sum[c] = sum[c] + emission[c] * ((response * cosine) / p);
        }
    }
    for (int c = 0; c < 3; ++c) out[c] = sum[c] / (float)count;
    return 1;
}

/* transportRandom, shaders/common.slang:292-295. */
float orc_transport_random(uint32_t seed, uint32_t lane) {
    uint32_t bits = orc_transport_hash(seed + 0x9e3779b9u * (lane + 1u));
    return ((float)(bits >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

/* cosineDirection, shaders/common.slang:407-412: tangent
 * normalize(cross(|n.y| < 0.99 ? +y : +x, n)), bitangent cross(n, tangent),
 * radius sqrt(u1) at u2 turns (cosine and sine as orc_sincos_turns), height
 * sqrt(1 - u1). */
void orc_cosine_direction_frame(const float n[3], float u1, float u2, float out[3]) {
    float axis[3] = {0.0f, 1.0f, 0.0f};
    if (!(fabsf(n[1]) < 0.99f)) {
        axis[0] = 1.0f;
        axis[1] = 0.0f;
    }
    float t[3], b[3];
    cross3(axis, n, t);
    float tl = sqrtf(dot3(t, t));
    for (int k = 0; k < 3; ++k) t[k] = t[k] / tl;
    cross3(n, t, b);
    float c, s;
    orc_sincos_turns(u2, &c, &s);
    float r = sqrtf(u1), h = sqrtf(1.0f - u1);
    float rc = r * c, rs = r * s;
    for (int k = 0; k < 3; ++k) out[k] = (t[k] * rc + b[k] * rs) + n[k] * h;
}

/* environmentResponseTracked (shaders/environment.slang:154-230) for a
 * constant environment: `count` cosine proposals (no alias samples without
 * an environment map: pdf = 0 x 1/(4 pi) + 1 x cos/pi = cos/pi), sample
 * seed transportHash(seed ^ transportHash(sample + sequence_base x count +
 * 0x85ebca6b)) with seed = hashKey(floor(position / (0.05 probe spacings)),
 * w 37; 2^24); each sample above both normals traces a visibility query from
 * rayOffset(position, gnormal, bias) to 1e20 and adds environment x
 * (response x cos / pdf), response = diffuse x disneyDiffuseMultiplier / pi
 * (diffuse = 1 for environmentIrradiance).  `visibility` (negative: trace
 * the scene) stubs the query: 0 visible, 1 blocked, 2 unsupported.  Returns 0
 * when a query is unsupported (out = 0). */
int orc_environment_response(const OrcScene *S, const float environment[3], float probe_spacing, float bias,
                             uint32_t count, uint32_t sequence_base, const float position[3], const float normal[3],
                             const float gnormal[3], const float view[3], float roughness, const float diffuse[3],
                             int visibility, float out[3], uint64_t *shadow_rays, OrcCounters *cn) {
    out[0] = out[1] = out[2] = 0.0f;
    if (count == 0u || !(environment[0] > 0.0f || environment[1] > 0.0f || environment[2] > 0.0f)) return 1;
    float cell = probe_spacing * 0.05f;
    int32_t k[4] = {(int32_t)floorf(position[0] / cell), (int32_t)floorf(position[1] / cell),
                    (int32_t)floorf(position[2] / cell), 37};
    uint32_t seed = orc_hash_key(k, 16777216u);
    float origin[3];
    orc_ray_offset(position, gnormal, bias, origin);
    float sum[3] = {0, 0, 0};
    for (uint32_t sample = 0; sample < count; ++sample) {
        uint32_t sequence = sample + sequence_base * count;
        uint32_t sample_seed = orc_transport_hash(seed ^ orc_transport_hash(sequence + 0x85ebca6bu));
        float d[3];
        orc_cosine_direction_frame(normal, orc_transport_random(sample_seed, 0u), orc_transport_random(sample_seed, 1u),
                                   d);
        float cosine = fmaxf(0.0f, dot3(normal, d));
        if (cosine <= 0.0f || dot3(gnormal, d) <= 0.0f) continue;
        float pdf = cosine / PI_F;
        if (!(pdf > 0.0f) || !isfinite(pdf)) continue;
        int blocked = 0, supported = 1;
        if (shadow_rays) (*shadow_rays)++;
        if (visibility < 0)
            blocked = orc_trace_occluded(S, origin, d, 1e20f, &supported, cn);
        else {
            blocked = visibility == 1;
            supported = visibility != 2;
        }
        if (!supported) {
            out[0] = out[1] = out[2] = 0.0f;
            return 0;
        }
        if (blocked) continue;
        float factor = disney_multiplier(normal, d, view, roughness) / PI_F;
        for (int c = 0; c < 3; ++c) {
            float response = diffuse[c] * factor;
            sum[c] = sum[c] + environment[c] * ((response * cosine) / pdf);
        }
    }
    for (int c = 0; c < 3; ++c) out[c] = sum[c] / (float)count;
    return 1;
}

/* conventionalLightResponseTracked (shaders/cascades.slang:136-176): the
 * visible contributions of the conventional lights (point, spot: range fade
 * (1 - (d/range)^4)^2 / d^2 with (d/range)^4 as (x^2)^2, spot cone squared;
 * directional: direction in position.xyz at distance 1e20), summed in light
 * order; 0 when a visibility query is unsupported. */
static int conventional_response(const OrcScene *S, const LuxSettings *st, const float position[3],
                                 const float normal[3], const float gnormal[3], const float view[3], float roughness,
                                 const float diffuse[3], float out[3], uint64_t *shadow_rays, OrcCounters *cn) {
    out[0] = out[1] = out[2] = 0.0f;
    const float bias = st->normal_bias;
    float offset[3];
    orc_ray_offset(position, gnormal, bias, offset);
    for (uint32_t i = 0; i < S->conventional; ++i) {
        const LuxLight *L = &S->lights[i];
        float range = L->position[3];
        int finite = range > 0.0f;
        float to_light[3] = {L->position[0], L->position[1], L->position[2]};
        float distance = 1e20f, attenuation = 1.0f;
        if (finite) {
            for (int c = 0; c < 3; ++c) to_light[c] = L->position[c] - position[c];
            distance = length3(to_light);
            if (distance >= range || distance < bias) continue;
            for (int c = 0; c < 3; ++c) to_light[c] = to_light[c] / distance;
            float x = distance / range;
            float x2 = x * x;
            float fade = saturatef(1.0f - x2 * x2);
            attenuation = (fade * fade) / fmaxf(distance * distance, 0.0001f);
            if (L->direction[3] > 0.0f) {
                float neg[3] = {-to_light[0], -to_light[1], -to_light[2]};
                float cone = saturatef(dot3(L->direction, neg) * L->direction[3] + L->color[3]);
                attenuation *= cone * cone;
            }
        }
        float cosine = fmaxf(0.0f, dot3(normal, to_light));
        if (!(cosine > 0.0f && dot3(gnormal, to_light) > 0.0f && attenuation > 0.0f)) continue;
        int supported;
        if (shadow_rays) (*shadow_rays)++;
        int blocked = orc_trace_occluded(S, offset, to_light, distance - bias, &supported, cn);
        if (!supported) {
            out[0] = out[1] = out[2] = 0.0f;
            return 0;
        }
        if (blocked) continue;
        float factor = disney_multiplier(normal, to_light, view, roughness) / PI_F;
        float scale = attenuation * cosine;
        for (int c = 0; c < 3; ++c) out[c] = out[c] + L->color[c] * (scale * (diffuse[c] * factor));
    }
    return 1;
}

/* Multi-bounce roles of a frame (RadianceCascades::multi_bounce). */
typedef struct {
    const OrcFrame *feedback;  /* secondary frame whose cascade-0 probes add bounce light (NULL: none) */
    int skip_emission;         /* the secondary cache: no first-hit emission (environmentScale.z) */
    int cached_sky;            /* cachedHitSky: secondary escapes carry the environment, covered hits skip its samples */
} Bounce;

static void feedback_irradiance(const OrcFrame *fb, const float position[3], const float normal[3], float out[3],
                                float *coverage);

/* outgoingTransportRadianceTracked, shaders/cascades.slang:196-268, with
 * every active source group summed into one radiance in the order emission,
 * emissive next-event estimate, constant environment, conventional lights.  With a feedback frame
 * the secondary cache's irradiance times the diffuse colour is added last
 * (secondaryFeedback, shaders/world_resolve.slang:204-279).  `rec` receives
 * the surface a multi-bounce secondary receiver takes from this hit:
 * position xyz, geometric normal facing the ray xyz, valid flag. */
static int outgoing_radiance(const OrcScene *S, const LuxSettings *st, const Bounce *bn, const float origin[3],
                             const float direction[3], const LuxHit *hit, float out[3], float rec[7],
                             uint64_t *shadow_rays, OrcCounters *cn) {
    out[0] = out[1] = out[2] = 0.0f;
    if (rec) rec[6] = 0.0f;
    if ((hit->errors & HIT_QUERY_UNSUPPORTED) != 0u) return 0;
    if (hit->triangle == EMPTY) {
        /* outgoingEnvironmentEscape (shaders/environment.slang:145-152). */
        if (bn && bn->skip_emission && bn->cached_sky)
            for (int c = 0; c < 3; ++c) out[c] = fmaxf(st->environment[c], 0.0f);
        return 1;
    }
    Surface sf;
    surface_at(S, st, hit->instance, hit->triangle, hit->barycentric, &sf);
    float radiance[3] = {sf.emission[0], sf.emission[1], sf.emission[2]};
    if (bn && bn->skip_emission) radiance[0] = radiance[1] = radiance[2] = 0.0f;
    if ((sf.flags & 16u) == 0u) {
        uint32_t base = instance_base(S, hit->instance);
        U4 header = gword(S, 0);
        float A[3], B[3], C[3];
        uint32_t idx[3];
        local_triangle(S, hit->triangle, header, A, B, C, idx);
        float position[3];
        for (int c = 0; c < 3; ++c) position[c] = origin[c] + direction[c] * hit->distance;
        float gn[3];
        geometric_normal(S, base, sf.flags, A, B, C, gn);
        /* hitAttributes world normal, shaders/traversal.slang:258-282. */
        float world_normal[3] = {0, 0, 0};
        for (int i = 0; i < 3; ++i) {
            U4 vw = gword(S, header.y + idx[i] * header.z);
            float nrm[3] = {gn[0], gn[1], gn[2]};
            if ((vw.w & 1u) != 0u) {
                U4 nw = gword(S, header.y + idx[i] * header.z + 1);
                float vn[3] = {asf(nw.x), asf(nw.y), asf(nw.z)}, tn[3];
                transform_direction(S, base, vn, 1, tn);
                unit_vector(tn, gn, nrm);
            }
            for (int c = 0; c < 3; ++c) world_normal[c] = world_normal[c] + nrm[c] * hit->barycentric[i];
        }
        /* materialNormal without a normal texture, shaders/material.slang:171-177. */
        float normal[3];
        unit_vector(world_normal, gn, normal);
        int back = dot3(gn, direction) > 0.0f;
        if (back && (sf.flags & 8u) != 0u) {
            normal[0] = -normal[0]; normal[1] = -normal[1]; normal[2] = -normal[2];
        }
        float flipped[3] = {gn[0], gn[1], gn[2]};
        if (dot3(flipped, direction) > 0.0f) {
            flipped[0] = -flipped[0]; flipped[1] = -flipped[1]; flipped[2] = -flipped[2];
        }
        float neg[3] = {-direction[0], -direction[1], -direction[2]};
        if (!(dot3(normal, neg) <= 0.0f || dot3(normal, flipped) <= 0.0f)) {
            float nl = length3(neg);
            float view[3] = {neg[0] / nl, neg[1] / nl, neg[2] / nl};
            float metallic = saturatef(sf.metallic);
            float roughness = saturatef(sf.roughness);
            if (!isfinite(roughness)) roughness = 1.0f;
            float diffuse[3];
            int base_finite = finite3(sf.base_color);
            for (int c = 0; c < 3; ++c)
                diffuse[c] = (base_finite ? saturatef(sf.base_color[c]) : 0.0f) * (1.0f - metallic);
            if (rec) {
                memcpy(rec, position, 12);
                memcpy(rec + 3, flipped, 12);
                rec[6] = finite3(position) && finite3(flipped) && finite3(normal) && dot3(flipped, flipped) > 0.01f;
            }
            float nee[3];
            if (!emissive_response(S, st, position, normal, flipped, view, roughness, diffuse, nee, shadow_rays, cn)) {
                out[0] = out[1] = out[2] = 0.0f;
                return 0;
            }
            for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + nee[c];
            /* secondaryFeedback before the environment (shaders/cascades.slang:236-242):
             * with cached hit sky a covered hit takes its sky light from the cache. */
            float fb_e[3] = {0, 0, 0}, coverage = 0.0f;
            if (bn && bn->feedback) feedback_irradiance(bn->feedback, position, normal, fb_e, &coverage);
            int sky_from_cache = bn && bn->cached_sky && coverage > 0.0f;
            uint32_t count = st->emissive_samples / 2u < 1u ? 1u : st->emissive_samples / 2u;
            float env[3] = {0, 0, 0};
            if (!sky_from_cache &&
                !orc_environment_response(S, st->environment, st->probe_spacing, st->normal_bias, count,
                                          st->frame_index ^ 0xE17A0002u, position, normal, flipped, view, roughness,
                                          diffuse, -1, env, shadow_rays, cn)) {
                out[0] = out[1] = out[2] = 0.0f;
                return 0;
            }
            if (!sky_from_cache && (st->environment[0] > 0.0f || st->environment[1] > 0.0f || st->environment[2] > 0.0f))
                for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + env[c];
            if (S->conventional) {
                float conv[3];
                if (!conventional_response(S, st, position, normal, flipped, view, roughness, diffuse, conv,
                                           shadow_rays, cn)) {
                    out[0] = out[1] = out[2] = 0.0f;
                    return 0;
                }
                for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + conv[c];
            }
            if (bn && bn->feedback)
                for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + fb_e[c] * diffuse[c];
        }
    }
    /* clampOutgoingTransportRadiance, shaders/cascades.slang:179-188. */
    if (!finite3(radiance)) return 1;
    for (int c = 0; c < 3; ++c) out[c] = fmaxf(radiance[c], 0.0f);
    return 1;
}

int orc_outgoing_radiance(const OrcScene *S, const LuxSettings *st, const float origin[3],
                          const float direction[3], const LuxHit *hit, float out[3], uint64_t *shadow_rays,
                          OrcCounters *cn) {
    return outgoing_radiance(S, st, NULL, origin, direction, hit, out, NULL, shadow_rays, cn);
}

/* ======================================================================
 * Cascade frame: deposit, reduce, merge, pack, resolve (shaders/split.slang,
 * shaders/world_resolve.slang)
 * ==================================================================== */
/* A cell key: x, y, z and the probe LOD (cacheKey, shaders/common.slang:
 * 418-422); `aux` carries per-key scratch (a last-receiver frame, an index). */
typedef struct { int32_t k[4]; uint32_t aux; } Key;

static int key_cmp(const void *a, const void *b) {
    const int32_t *x = ((const Key *)a)->k, *y = ((const Key *)b)->k;
    for (int i = 0; i < 4; ++i)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}

/* Distance LODs (splitLodBlendForParameters, shaders/common.slang:431-461)
 * with the camera terms evaluated once per frame, as lux_view_trace_merge
 * does. */
#define MAX_LOD 24u
typedef struct {
    int enabled, perspective;
    float camera[3];
    float base, ortho_scale;
} LodParams;

static float lod_scale(uint32_t lod) {
    uint32_t bits = (127u + lod) << 23;
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static void lod_params(const LuxSettings *st, const LuxCamera *cam, LodParams *L) {
    memset(L, 0, sizeof *L);
    if (!cam || !cam->enabled || st->layout != LUX_LAYOUT_SPLIT) return;
    const float *m = cam->clip_from_world;
    float px = m[12], py = m[13], pz = m[14];
    int perspective = isfinite(px) && isfinite(py) && isfinite(pz) && (px * px + py * py) + pz * pz > 1e-12f;
    float focal = 0.5f * (float)cam->viewport_height * sqrtf((m[4] * m[4] + m[5] * m[5]) + m[6] * m[6]);
    float target = (float)(cam->target_pixels > 1u ? cam->target_pixels : 1u);
    L->enabled = 1;
    L->perspective = perspective;
    for (int a = 0; a < 3; ++a) L->camera[a] = cam->position[a];
    L->base = fmaxf(focal * st->probe_spacing / target, st->probe_spacing);
    L->ortho_scale = target / fmaxf(focal * st->probe_spacing, 1e-20f);
}

/* floor(log2(x)) for x >= 1 is the exponent (exact); 2^(low+1) is exact. */
static void point_lod(const LodParams *L, const float p[3], uint32_t *low, uint32_t *high, float *blend) {
    *low = *high = 0u;
    *blend = 0.0f;
    if (!L || !L->enabled) return;
    float scale;
    if (L->perspective) {
        float ox = fabsf(p[0] - L->camera[0]), oy = fabsf(p[1] - L->camera[1]), oz = fabsf(p[2] - L->camera[2]);
        scale = fmaxf(ox, fmaxf(oy, oz)) / L->base;
    } else {
        scale = L->ortho_scale;
    }
    float s1 = fmaxf(scale, 1.0f);
    uint32_t bits;
    memcpy(&bits, &s1, 4);
    uint32_t e = s1 < INFINITY ? (bits >> 23) - 127u : MAX_LOD;
    *low = e < MAX_LOD ? e : MAX_LOD;
    *high = *low;
    if (*low < MAX_LOD) {
        float next = lod_scale(*low + 1u);
        float overlap = 0.9f * next;
        if (scale >= overlap && scale < next) {
            *high = *low + 1u;
            *blend = saturatef((scale - overlap) / (next - overlap));
        }
    }
}

/* seed's variant choice in an LOD overlap (shaders/split.slang:747-752). */
static uint32_t receiver_lod(const LodParams *L, const float p[3], uint32_t sample, uint32_t frame) {
    uint32_t low, high;
    float blend;
    point_lod(L, p, &low, &high, &blend);
    if (high == low) return low;
    uint32_t bits = orc_transport_hash(sample ^ (frame * 0x9e3779b9u));
    float phase = (float)(bits >> 8) * (1.0f / 16777216.0f);
    return phase < blend ? high : low;
}

void orc_lod_blend(const LuxSettings *st, const LuxCamera *camera, const float position[3], uint32_t *low,
                   uint32_t *high, float *blend) {
    LodParams L;
    lod_params(st, camera, &L);
    point_lod(&L, position, low, high, blend);
}

typedef struct {
    uint32_t cells, dirs, columns, rows;
    Key *keys;
    float *jsum;     /* float4: J sum rgb, non-terminating count */
    uint32_t *count;
    float *merged;   /* float4 */
    float *raw;      /* float4 J, beta (history-blended) */
    float *mass;     /* float2 radiance mass, transmittance mass */
    uint32_t *last;  /* frame index of each cell's last receiver */
} Level;

struct OrcFrame {
    LuxSettings st;
    LodParams lod;
    uint32_t levels;
    Level level[LUX_MAX_LEVELS];
    float *tables;  /* c0 cells * 36 float4 */
    LuxStats stats;
    const struct OrcFrame *previous;  /* history source (NULL: none) */
    const float *dirty;               /* invalidation boxes, 6 floats each */
    uint32_t dirty_count;
    LuxHit *hits;                     /* split: the closest hit of every interval ray, ray order */
    uint64_t hit_count;
};

static int64_t find_cell(const Level *L, const int32_t key[4]) {
    int64_t lo = 0, hi = (int64_t)L->cells - 1;
    while (lo <= hi) {
        int64_t mid = (lo + hi) / 2;
        const int32_t *m = L->keys[mid].k;
        int c = 0;
        for (int i = 0; i < 4 && c == 0; ++i)
            if (m[i] != key[i]) c = m[i] < key[i] ? -1 : 1;
        if (c == 0) return mid;
        if (c < 0) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

/* cacheKey cell, shaders/common.slang:417-422: spacing x 2^lod. */
static void cell_key(const LuxSettings *st, uint32_t level, const float p[3], uint32_t lod, int32_t out[4]) {
    float s = orc_spacing(st, level) * lod_scale(lod);
    for (int i = 0; i < 3; ++i) out[i] = (int32_t)floorf(p[i] / s);
    out[3] = (int32_t)lod;
}

/* Sample sequence order (rank / parents / prefix, shaders/split.slang:788-963):
 * the receivers of one cascade-0 cell take consecutive places and sibling cells
 * of every coarser level adjacent runs.  Key: LOD, then the Morton code of the
 * cascade-0 cell (octant ordinal x + 2y + 4z at every level, 19 bits per axis
 * biased by 2^18); ties by receiver index; absent receivers last. */
static uint64_t sequence_key(const int32_t key[4]) {
    uint32_t b[3] = {(uint32_t)key[0] + (1u << 18), (uint32_t)key[1] + (1u << 18), (uint32_t)key[2] + (1u << 18)};
    uint64_t m = 0;
    for (int bit = 0; bit < 19; ++bit)
        for (int a = 0; a < 3; ++a) m |= (uint64_t)((b[a] >> bit) & 1u) << (3 * bit + a);
    return ((uint64_t)((uint32_t)key[3] & 31u) << 57) | m;
}
typedef struct {
    uint64_t key;
    uint32_t index;
} OrderItem;
static int order_cmp(const void *a, const void *b) {
    const OrderItem *x = (const OrderItem *)a, *y = (const OrderItem *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->index < y->index ? -1 : (x->index > y->index ? 1 : 0);
}

/* Each receiver's place in the sample sequence: out[i] = rank of receiver i. */
static void sequence_order(const LuxSettings *st, const LodParams *lod, const float *pos, uint32_t n, int sparse,
                           uint32_t *out) {
    OrderItem *order = (OrderItem *)malloc(sizeof(OrderItem) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) {
        const float *p = pos + 4 * (size_t)i;
        order[i].index = i;
        if (sparse && p[3] == 0.0f) {
            order[i].key = ~0ull;
            continue;
        }
        int32_t key[4];
        cell_key(st, 0, p, receiver_lod(lod, p, i, st->frame_index), key);
        order[i].key = sequence_key(key);
    }
    qsort(order, n, sizeof(OrderItem), order_cmp);
    for (uint32_t j = 0; j < n; ++j) out[order[j].index] = j;
    free(order);
}

void orc_sequence_order(const LuxSettings *settings, const LuxCamera *camera, const float *pos, uint32_t n,
                        int sparse, uint32_t *out) {
    LodParams lod;
    lod_params(settings, camera, &lod);
    sequence_order(settings, &lod, pos, n, sparse, out);
}

typedef struct {
    const OrcScene *S;
    const LuxSettings *st;
    const float *pos, *nrm;
    uint32_t n;
    /* multi-bounce */
    const Bounce *bounce;
    const LodParams *lod;     /* distance LODs of the frame (NULL: LOD 0) */
    int sparse;               /* receivers with position.w == 0 are absent */
    float *hit_pos, *hit_nrm; /* float4 per receiver: the surface of ray frame % R, or NULL */
    const uint32_t *ordinal;  /* split: each receiver's place in the sample sequence */
    /* split: per ray outputs */
    int32_t *term_level;  /* -1 = unsupported */
    float *radiance;      /* rgb per ray */
    LuxHit *hits;         /* closest hit per ray */
    uint32_t *ubin;       /* flipped (u, v) stored as bits */
    float *uv;
    /* dense */
    Level *levels;
    uint32_t level;
    uint64_t begin, end;
    uint64_t shadow;
    OrcCounters cn;
} FrameJob;

static void split_ray(const OrcScene *S, const LuxSettings *st, const float p[3], const float n[3], uint32_t sequence,
                      float uv_out[2], LuxHit *hit, float origin[3], float dir[3]) {
    float jitter[2], r[2];
    orc_r2(orc_transport_hash(st->frame_index ^ 0x5a17c9e3u), jitter);
    orc_r2(sequence + 1u, r);
    float u = fracf((0.5f + r[0]) + jitter[0]);
    float v = fracf((0.5f + r[1]) + jitter[1]);
    orc_decode_direction(u, v, dir);
    if (dot3(dir, n) < 0.0f) {
        dir[0] = -dir[0]; dir[1] = -dir[1]; dir[2] = -dir[2];
        u = fracf(u + 0.5f);
        v = 1.0f - v;
    }
    uv_out[0] = u;
    uv_out[1] = v;
    orc_ray_offset(p, n, st->normal_bias, origin);
    (void)S;
    (void)hit;
}

static void *split_job(void *arg) {
    FrameJob *j = (FrameJob *)arg;
    const LuxSettings *st = j->st;
    uint32_t R = st->rays_per_receiver;
    for (uint64_t ray = j->begin; ray < j->end; ++ray) {
        uint32_t i = (uint32_t)(ray / R), k = (uint32_t)(ray % R);
        const float *p = j->pos + 4 * (size_t)i, *n = j->nrm + 4 * (size_t)i;
        if (j->sparse && p[3] == 0.0f) {
            j->term_level[ray] = -2;  /* absent receiver: no ray */
            memset(&j->hits[ray], 0, sizeof(LuxHit));
            j->hits[ray].triangle = j->hits[ray].instance = EMPTY;
            j->hits[ray].errors = HIT_QUERY_UNSUPPORTED;
            continue;
        }
        float uv[2], origin[3], dir[3];
        LuxHit hit;
        split_ray(j->S, st, p, n, j->ordinal[i] * R + k, uv, &hit, origin, dir);
        orc_trace_closest(j->S, origin, dir, 0.0f, 1e20f, &hit, &j->cn);
        j->hits[ray] = hit;
        float rad[3], rec[7];
        int supported = outgoing_radiance(j->S, st, j->bounce, origin, dir, &hit, rad, rec, &j->shadow, &j->cn);
        if (j->hit_pos && rec[6] != 0.0f && k == st->frame_index % R) {
            float *hp = j->hit_pos + 4 * (size_t)i, *hn = j->hit_nrm + 4 * (size_t)i;
            hp[0] = rec[0]; hp[1] = rec[1]; hp[2] = rec[2]; hp[3] = 1.0f;
            hn[0] = rec[3]; hn[1] = rec[4]; hn[2] = rec[5]; hn[3] = 0.0f;
        }
        j->uv[2 * ray] = uv[0];
        j->uv[2 * ray + 1] = uv[1];
        memcpy(&j->radiance[3 * ray], rad, sizeof rad);
        if (!supported || (hit.errors & HIT_QUERY_UNSUPPORTED)) {
            j->term_level[ray] = -1;
            continue;
        }
        /* splitIntervalContainsHit at the receiver's LOD (ends x 2^lod). */
        float ls = j->lod && j->lod->enabled ? lod_scale(receiver_lod(j->lod, p, i, st->frame_index)) : 1.0f;
        int32_t term = (int32_t)st->levels - 1;
        for (uint32_t l = 0; l + 1 < st->levels; ++l) {
            if (hit.distance > interval_start(st, l) * ls && hit.distance <= orc_interval_end(st, l) * ls) {
                term = (int32_t)l;
                break;
            }
        }
        j->term_level[ray] = term;
    }
    return NULL;
}

static void *dense_job(void *arg) {
    FrameJob *j = (FrameJob *)arg;
    const LuxSettings *st = j->st;
    Level *L = &j->levels[j->level];
    uint32_t l = j->level;
    int terminal = l + 1 == st->levels;
    float start = interval_start(st, l), end = orc_interval_end(st, l);
    float limit = terminal ? 1e20f : nextafterf(end, INFINITY);
    float sp = orc_spacing(st, l);
    for (uint64_t e = j->begin; e < j->end; ++e) {
        uint32_t cell = (uint32_t)(e / L->dirs), d = (uint32_t)(e % L->dirs);
        float origin[3], dir[3];
        for (int c = 0; c < 3; ++c) origin[c] = ((float)L->keys[cell].k[c] + 0.5f) * sp;
        orc_bin_direction(d, L->columns, L->rows, dir);
        LuxHit hit;
        orc_trace_closest(j->S, origin, dir, start, limit, &hit, &j->cn);
        float rad[3];
        int supported = orc_outgoing_radiance(j->S, st, origin, dir, &hit, rad, &j->shadow, &j->cn);
        if (!supported || (hit.errors & HIT_QUERY_UNSUPPORTED)) continue;
        int terminates = terminal || hit.triangle != EMPTY;
        float *js = &L->jsum[4 * e];
        L->count[e] = 1;
        if (terminates) {
            js[0] = rad[0]; js[1] = rad[1]; js[2] = rad[2];
        } else {
            js[3] = 1.0f;
        }
    }
    return NULL;
}

static void run_jobs(FrameJob *proto, uint64_t total, int threads, void *(*fn)(void *), uint64_t *shadow,
                     OrcCounters *cn) {
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > total) threads = total ? (int)total : 1;
    FrameJob *jobs = (FrameJob *)calloc((size_t)threads, sizeof(FrameJob));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        jobs[t] = *proto;
        jobs[t].begin = total * (uint64_t)t / (uint64_t)threads;
        jobs[t].end = total * (uint64_t)(t + 1) / (uint64_t)threads;
        pthread_create(&tid[t], NULL, fn, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) {
        pthread_join(tid[t], NULL);
        *shadow += jobs[t].shadow;
        cn->nodes += jobs[t].cn.nodes;
        cn->triangles += jobs[t].cn.triangles;
        cn->instances += jobs[t].cn.instances;
    }
    free(jobs);
    free(tid);
}

/* interpolateMergedChildSources, shaders/split.slang:389-479, one source
 * group; corner_merged = float4[8] (w <= 0 or NaN: unsupported / missing). */
void orc_interpolate_children(const float fraction[3], const float *corner_merged, float out[4]) {
    float sum[3] = {0, 0, 0}, total = 0.0f, potential = 0.0f;
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        uint32_t bx = corner & 1u, by = (corner >> 1) & 1u, bz = corner >> 2;
        float ax = bx == 0u ? 1.0f - fraction[0] : fraction[0];
        float ay = by == 0u ? 1.0f - fraction[1] : fraction[1];
        float az = bz == 0u ? 1.0f - fraction[2] : fraction[2];
        float weight = (ax * ay) * az;
        if (!(weight > 0.0f)) continue;
        potential += weight;
        const float *s = corner_merged + 4 * corner;
        if (s[3] > 0.0f && isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3])) {
            float sw = weight * saturatef(s[3]);
            for (int c = 0; c < 3; ++c) sum[c] = sum[c] + s[c] * sw;
            total += sw;
        }
    }
    if (total > 0.0f) {
        for (int c = 0; c < 3; ++c) out[c] = sum[c] / total;
        out[3] = saturatef(total / fmaxf(potential, 1e-8f));
    } else {
        out[0] = out[1] = out[2] = out[3] = 0.0f;
    }
}

/* mergeEntry + mergeRadianceGroups + finishMergeGroup without history
 * (shaders/split.slang:1523-1725): interval = (J.rgb, beta) of the reduced
 * entry, child values = the 4 angular children already interpolated. */
/* base^n by squaring and multiplying (the GPU kernel rounds identically). */
static float pow_count(float base, uint32_t n) {
    float r = 1.0f, b = base;
    while (n) {
        if (n & 1u) r = r * b;
        b = b * b;
        n >>= 1;
    }
    return r;
}

/* mergeEntry's history blend (shaders/split.slang:1624-1725 with
 * mergeRawRadianceGroup, :1478-1521) of one record, for the summed radiance
 * group (blend temporal_blend) and the transmittance (transmittance_blend):
 * n fresh observations with mean `fresh` (J rgb, beta); `old` / `old_mass`
 * the previous frame's record (NULL: none).  With n > 0 the new mass is
 * (1 - blend^n) / (1 - blend) and the old mass is min(old, limit) * blend^n;
 * with n == 0 the old record is kept as it is; without either, J = 0,
 * beta = 1 and both masses are 0. */
void orc_history_blend(const LuxSettings *st, uint32_t n, const float fresh[4], const float *old,
                       const float *old_mass, float out[4], float mass[2]) {
    float jb = st->temporal_blend, tb = st->transmittance_blend;
    float jlimit = 1.0f / (1.0f - jb), tlimit = 1.0f / (1.0f - tb);
    float rm = old_mass ? old_mass[0] : 0.0f, tm = old_mass ? old_mass[1] : 0.0f;
    if (!isfinite(rm) || rm < 0.0f) rm = 0.0f;
    if (!isfinite(tm) || tm < 0.0f) tm = 0.0f;
    int reuse_r = old && jb > 0.0f, reuse_t = old && tb > 0.0f;
    float j[3] = {0.0f, 0.0f, 0.0f}, beta = 1.0f, rmass = 0.0f, tmass = 0.0f;
    if (n) {
        float ret = pow_count(jb, n);
        rmass = (1.0f - ret) * jlimit;
        for (int c = 0; c < 3; ++c) j[c] = fresh[c];
        float om = fminf(rm, jlimit) * ret;
        if (reuse_r && om > 0.0f) {
            for (int c = 0; c < 3; ++c) j[c] = (j[c] * rmass + old[c] * om) / (rmass + om);
            rmass = rmass + om;
        }
        float tret = pow_count(tb, n);
        tmass = (1.0f - tret) * tlimit;
        beta = fresh[3];
        float otm = fminf(tm, tlimit) * tret;
        if (reuse_t && otm > 0.0f) {
            beta = (beta * tmass + old[3] * otm) / (tmass + otm);
            tmass = tmass + otm;
        }
    } else {
        if (reuse_r && rm > 0.0f) {
            for (int c = 0; c < 3; ++c) j[c] = old[c];
            rmass = rm;
        }
        if (reuse_t && tm > 0.0f) {
            beta = old[3];
            tmass = tm;
        }
    }
    out[0] = j[0];
    out[1] = j[1];
    out[2] = j[2];
    out[3] = beta;
    mass[0] = rmass;
    mass[1] = tmass;
}

/* Eq. 7 on a blended record (mergeRadianceGroups / finishMergeGroup,
 * shaders/split.slang:1523-1622). */
static void merge_blended(const float raw[4], const float mass[2], const float *children, int has_children,
                          float out[4]) {
    float transmittance = mass[1] > 0.0f ? saturatef(raw[3]) : 0.0f;
    float support = mass[0] > 0.0f && mass[1] > 0.0f ? 1.0f - transmittance : 0.0f;
    float radiance[3] = {0, 0, 0};
    if (support > 0.0f) {
        radiance[0] = raw[0]; radiance[1] = raw[1]; radiance[2] = raw[2];
    }
    float child_sum[3] = {0, 0, 0}, child_support = 0.0f;
    if (transmittance > 0.0f && has_children) {
        for (int c = 0; c < 4; ++c) {
            const float *v = children + 4 * c;
            if (!(v[3] > 0.0f)) continue;
            for (int k = 0; k < 3; ++k) child_sum[k] = child_sum[k] + v[k] * v[3];
            child_support += v[3];
        }
    }
    if (child_support > 0.0f) {
        for (int k = 0; k < 3; ++k) radiance[k] = radiance[k] + (transmittance * child_sum[k]) * 0.25f;
        support = support + (transmittance * child_support) * 0.25f;
    }
    if (support > 0.0f) {
        for (int k = 0; k < 3; ++k) out[k] = radiance[k] / support;
        out[3] = saturatef(support);
    } else {
        out[0] = out[1] = out[2] = out[3] = 0.0f;
    }
}

static void merge_values(const LuxSettings *st, const float interval[4], uint32_t samples, const float *children,
                         int has_children, float out[4]) {
    float raw[4], mass[2];
    orc_history_blend(st, samples, interval, NULL, NULL, raw, mass);
    merge_blended(raw, mass, children, has_children, out);
}

void orc_merge_entry(const float interval[4], uint32_t samples, const float fraction[3], const float *child_merged,
                     int has_children, float out[4]) {
    float children[16];
    for (int c = 0; c < 4; ++c) orc_interpolate_children(fraction, child_merged + 32 * c, children + 4 * c);
    LuxSettings st;
    memset(&st, 0, sizeof st);  /* no history: blends 0 */
    merge_values(&st, interval, samples, children, has_children, out);
}

/* mergeEntry with history (shaders/split.slang:1478-1521, :1624-1725) for
 * one entry: the fresh (J, beta) of `samples` observations blended with the
 * previous frame's record (old raw, old mass; NULL: none) under the
 * settings' blends, then the children as orc_merge_entry takes them. */
void orc_merge_history_entry(const LuxSettings *st, const float interval[4], uint32_t samples, const float *old,
                             const float *old_mass, const float fraction[3], const float *child_merged,
                             int has_children, float out[4]) {
    float children[16], raw[4], mass[2];
    for (int c = 0; c < 4; ++c) orc_interpolate_children(fraction, child_merged + 32 * c, children + 4 * c);
    orc_history_blend(st, samples, interval, old, old_mass, raw, mass);
    merge_blended(raw, mass, children, has_children, out);
}

/* A record's history is invalid when its cell grown by the level's
 * interval end (unbounded at the last level) meets an invalidation box. */
static int record_dirty(const OrcFrame *F, uint32_t level, const int32_t key[4]) {
    if (F->dirty_count == 0) return 0;
    if (level + 1 >= F->levels) return 1;
    float ls = lod_scale((uint32_t)key[3]);
    float s = orc_spacing(&F->st, level) * ls, reach = orc_interval_end(&F->st, level) * ls;
    for (uint32_t b = 0; b < F->dirty_count; ++b) {
        const float *box = F->dirty + 6 * (size_t)b;
        int meet = 1;
        for (int a = 0; a < 3; ++a) {
            float lo = (float)key[a] * s - reach, hi = (float)(key[a] + 1) * s + reach;
            meet = meet && lo <= box[3 + a] && hi >= box[a];
        }
        if (meet) return 1;
    }
    return 0;
}

static void merge_level(OrcFrame *F, uint32_t l) {
    const LuxSettings *st = &F->st;
    Level *L = &F->level[l];
    int has_children = l + 1 < F->levels;
    Level *P = has_children ? &F->level[l + 1] : NULL;
    for (uint32_t cell = 0; cell < L->cells; ++cell) {
        int64_t corner_cell[8];
        float fraction[3];
        /* A cell's children are the next level's cells of the same LOD. */
        const uint32_t lod = (uint32_t)L->keys[cell].k[3];
        const float sp = orc_spacing(st, l) * lod_scale(lod);
        const float sp1 = has_children ? orc_spacing(st, l + 1) * lod_scale(lod) : 1.0f;
        if (has_children) {
            int32_t base[3];
            for (int c = 0; c < 3; ++c) {
                float origin = ((float)L->keys[cell].k[c] + 0.5f) * sp;
                float grid = origin / sp1 - 0.5f;
                float fl = floorf(grid);
                base[c] = (int32_t)fl;
                fraction[c] = grid - fl;
            }
            for (uint32_t corner = 0; corner < 8u; ++corner) {
                int32_t k[4] = {base[0] + (int32_t)(corner & 1u), base[1] + (int32_t)((corner >> 1) & 1u),
                                base[2] + (int32_t)(corner >> 2), (int32_t)lod};
                corner_cell[corner] = find_cell(P, k);
            }
        }
        /* The previous frame's cell of this key (history), unless an
         * invalidation box meets the region its rays may have crossed. */
        const Level *H = NULL;
        int64_t hcell = -1;
        if (F->previous && l < F->previous->levels && F->previous->level[l].dirs == L->dirs &&
            !record_dirty(F, l, L->keys[cell].k)) {
            H = &F->previous->level[l];
            hcell = find_cell(H, L->keys[cell].k);
        }
        for (uint32_t d = 0; d < L->dirs; ++d) {
            uint64_t e = (uint64_t)cell * L->dirs + d;
            uint32_t n = L->count[e];
            float interval[4] = {0, 0, 0, 0};
            if (n) {
                float fn = (float)n;
                for (int c = 0; c < 4; ++c) interval[c] = L->jsum[4 * e + c] / fn;
            }
            const float *old = NULL, *old_mass = NULL;
            if (hcell >= 0) {
                uint64_t he = (uint64_t)hcell * H->dirs + d;
                old = &H->raw[4 * he];
                old_mass = &H->mass[2 * he];
            }
            float raw[4], mass[2];
            orc_history_blend(st, n, interval, old, old_mass, raw, mass);
            if (n || mass[0] > 0.0f || mass[1] > 0.0f)
                memcpy(&L->raw[4 * e], raw, sizeof raw);
            else
                memset(&L->raw[4 * e], 0, sizeof raw);
            memcpy(&L->mass[2 * e], mass, sizeof mass);
            float transmittance = mass[1] > 0.0f ? saturatef(raw[3]) : 0.0f;
            float children[16];
            memset(children, 0, sizeof children);
            if (has_children && transmittance > 0.0f) {
                uint32_t x = d % L->columns, y = d / L->columns;
                for (uint32_t child = 0; child < 4u; ++child) {
                    uint32_t fx = x * 2u + (child & 1u), fy = y * 2u + (child >> 1);
                    uint32_t fine = fx + fy * P->columns;
                    float corners[32];
                    for (uint32_t corner = 0; corner < 8u; ++corner) {
                        if (corner_cell[corner] < 0) {
                            memset(corners + 4 * corner, 0, 16);
                        } else {
                            memcpy(corners + 4 * corner, &P->merged[4 * ((uint64_t)corner_cell[corner] * P->dirs + fine)], 16);
                        }
                    }
                    orc_interpolate_children(fraction, corners, children + 4 * child);
                }
            }
            merge_blended(raw, mass, children, has_children, &L->merged[4 * e]);
        }
    }
}

/* packProbes, shaders/split.slang:1786-1918 (one source group; D0 base
 * directions with scale nominal * 4 / D0). */
void orc_pack_table(const float *merged, uint32_t columns, uint32_t rows, float *table) {
    uint32_t dirs = columns * rows;
    float *dir = (float *)malloc(sizeof(float) * 3 * dirs);
    float *val = (float *)malloc(sizeof(float) * 4 * dirs);
    for (uint32_t d = 0; d < dirs; ++d) {
        orc_bin_direction(d, columns, rows, dir + 3 * d);
        const float *m = merged + 4 * d;
        int ok = m[3] > 0.0f && isfinite(m[0]) && isfinite(m[1]) && isfinite(m[2]) && isfinite(m[3]);
        for (int c = 0; c < 4; ++c) val[4 * d + c] = ok ? m[c] : 0.0f;
    }
    for (uint32_t texel = 0; texel < 36u; ++texel) {
        float p[2] = {((float)(texel % 6u) + 0.5f) / 6.0f, ((float)(texel / 6u) + 0.5f) / 6.0f};
        float normal[3];
        orc_decode_normal(p, normal);
        float sum[3] = {0, 0, 0}, nominal = 0.0f, observed = 0.0f;
        for (uint32_t d = 0; d < dirs; ++d) {
            float cosine = fmaxf(dot3(normal, dir + 3 * d), 0.0f);
            nominal += cosine;
            if (cosine <= 0.0f) continue;
            const float *v = val + 4 * d;
            if (v[3] > 0.0f) {
                float w = cosine * saturatef(v[3]);
                for (int c = 0; c < 3; ++c) sum[c] = sum[c] + v[c] * w;
                observed += w;
            }
        }
        float *out = table + 4 * texel;
        out[0] = out[1] = out[2] = out[3] = 0.0f;
        if (nominal > 0.0f) {
            float scale = nominal * (4.0f / (float)dirs);
            if (observed > 0.0f) {
                for (int c = 0; c < 3; ++c) out[c] = (sum[c] / observed) * scale;
                out[3] = saturatef(observed / nominal);
            }
        }
    }
    free(dir);
    free(val);
}

/* wrapIrradianceTexel / irradianceTexelIndex, shaders/world_resolve.slang:1-11. */
static uint32_t texel_index(int32_t x, int32_t y) {
    if (x < 0) { int32_t nx = -x - 1, ny = 5 - y; x = nx; y = ny; }
    else if (x >= 6) { int32_t nx = 11 - x, ny = 5 - y; x = nx; y = ny; }
    if (y < 0) { int32_t nx = 5 - x, ny = -y - 1; x = nx; y = ny; }
    else if (y >= 6) { int32_t nx = 5 - x, ny = 11 - y; x = nx; y = ny; }
    return (uint32_t)(y * 6 + x);
}

typedef struct { uint32_t texel[4]; float weight[4]; } Lookup;

/* irradianceLookup, shaders/world_resolve.slang:27-40. */
static Lookup irradiance_lookup(const float normal[3]) {
    Lookup lk;
    float e[2];
    orc_encode_normal(normal, e);
    float gx = e[0] * 6.0f - 0.5f, gy = e[1] * 6.0f - 0.5f;
    float bx = floorf(gx), by = floorf(gy);
    float fx = gx - bx, fy = gy - by;
    float cx = 1.0f - fx, cy = 1.0f - fy;
    lk.weight[0] = cx * cy;
    lk.weight[1] = fx * cy;
    lk.weight[2] = cx * fy;
    lk.weight[3] = fx * fy;
    int32_t ix = (int32_t)bx, iy = (int32_t)by;
    lk.texel[0] = texel_index(ix, iy);
    lk.texel[1] = texel_index(ix + 1, iy);
    lk.texel[2] = texel_index(ix, iy + 1);
    lk.texel[3] = texel_index(ix + 1, iy + 1);
    return lk;
}

/* diffuseProbePage, shaders/world_resolve.slang:51-89: out = rgb, coverage. */
static void probe_page(const float *table, const Lookup *lk, float out[4]) {
    float sum[3] = {0, 0, 0}, observed = 0.0f;
    for (int c = 0; c < 4; ++c) {
        float bw = lk->weight[c];
        if (!(bw > 0.0f)) continue;
        const float *s = table + 4 * lk->texel[c];
        if (!(s[3] > 0.0f) || !(isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3]))) continue;
        float w = bw * saturatef(s[3]);
        for (int k = 0; k < 3; ++k) sum[k] = sum[k] + s[k] * w;
        observed += w;
    }
    for (int k = 0; k < 3; ++k) out[k] = observed > 0.0f ? sum[k] / observed : 0.0f;
    out[3] = saturatef(observed);
}

void orc_probe_lookup(const float *table36, const float normal[3], float out[4]) {
    Lookup lk = irradiance_lookup(normal);
    probe_page(table36, &lk, out);
}

OrcFrame *orc_frame_run(const OrcScene *S, const LuxSettings *st_in, const float *pos, const float *nrm, uint32_t n,
                        int threads) {
    return orc_frame_run_history(S, st_in, pos, nrm, n, threads, NULL, NULL, 0);
}

OrcFrame *orc_frame_run_history(const OrcScene *S, const LuxSettings *st_in, const float *pos, const float *nrm,
                                uint32_t n, int threads, const OrcFrame *previous, const float *dirty,
                                uint32_t dirty_count) {
    return orc_frame_run_retain(S, st_in, pos, nrm, n, threads, previous, dirty, dirty_count, UINT32_MAX,
                                UINT64_MAX);
}

#define RETAIN_BINS 256u

/* retain (shaders/split.slang:991-1054) with a persistent world cache
 * (persistentWorldIntervals, shaders/common.slang:82-89; set for the Split
 * method at src/render.rs:8470): the previous frame's cells that no receiver
 * seeded stay, unless an invalidation box voids their history.  Capacity
 * keeps the youngest (commitCache, shaders/split.slang:1919-1961) as whole
 * age classes, levels in order, while cells fit max_cells and records fit
 * max_entries.  Keys carry each cell's last receiver frame in aux here. */
static void retain_cells(OrcFrame *F, Key **keys, uint32_t *cells, uint32_t max_cells, uint64_t max_entries) {
    const OrcFrame *P = F->previous;
    uint64_t used = 0;
    for (uint32_t l = 0; l < F->levels; ++l) used += (uint64_t)cells[l] * F->level[l].dirs;
    uint64_t remaining = used < max_entries ? max_entries - used : 0;
    for (uint32_t l = 0; l < F->levels; ++l) {
        const Level *H = &P->level[l];
        Level seeded;
        memset(&seeded, 0, sizeof seeded);
        seeded.cells = cells[l];
        seeded.keys = keys[l];
        uint32_t *bin = (uint32_t *)malloc(sizeof(uint32_t) * (H->cells ? H->cells : 1));
        uint64_t hist[RETAIN_BINS];
        memset(hist, 0, sizeof hist);
        for (uint32_t c = 0; c < H->cells; ++c) {
            bin[c] = RETAIN_BINS;
            if (find_cell(&seeded, H->keys[c].k) >= 0 || record_dirty(F, l, H->keys[c].k)) continue;
            uint32_t age = F->st.frame_index - H->last[c];
            bin[c] = age < RETAIN_BINS - 1u ? age : RETAIN_BINS - 1u;
            hist[bin[c]]++;
        }
        uint64_t room = max_cells > cells[l] ? (uint64_t)max_cells - cells[l] : 0;
        uint64_t by_entries = remaining / F->level[l].dirs;
        if (by_entries < room) room = by_entries;
        uint64_t kept = 0;
        uint32_t limit = 0;
        while (limit < RETAIN_BINS && kept + hist[limit] <= room) kept += hist[limit++];
        if (kept) {
            Key *all = (Key *)realloc(keys[l], sizeof(Key) * (cells[l] + kept));
            uint32_t m = cells[l];
            for (uint32_t c = 0; c < H->cells; ++c)
                if (bin[c] < limit) {
                    all[m] = H->keys[c];
                    all[m].aux = H->last[c];
                    ++m;
                }
            qsort(all, m, sizeof(Key), key_cmp);
            keys[l] = all;
            cells[l] = m;
        }
        remaining -= kept * F->level[l].dirs;
        free(bin);
    }
}

OrcFrame *orc_frame_run_retain(const OrcScene *S, const LuxSettings *st_in, const float *pos, const float *nrm,
                               uint32_t n, int threads, const OrcFrame *previous, const float *dirty,
                               uint32_t dirty_count, uint32_t max_cells, uint64_t max_entries) {
    return orc_frame_run_bounce(S, st_in, pos, nrm, n, threads, previous, dirty, dirty_count, max_cells, max_entries,
                                NULL, 0u, NULL, NULL, NULL);
}

/* secondaryFeedback at LOD 0 of the secondary frame: its cascade-0 probe of
 * the cell holding `position`, looked up with the shading normal;
 * resolveLodSource with a zero LOD blend gives (rgb * coverage) / coverage. */
static void feedback_irradiance(const OrcFrame *fb, const float position[3], const float normal[3], float out[3],
                                float *coverage) {
    out[0] = out[1] = out[2] = 0.0f;
    *coverage = 0.0f;
    if (!finite3(position)) return;
    float s = orc_spacing(&fb->st, 0);
    int32_t key[4] = {(int32_t)floorf(position[0] / s), (int32_t)floorf(position[1] / s),
                      (int32_t)floorf(position[2] / s), 0};
    int64_t cell = find_cell(&fb->level[0], key);
    if (cell < 0) return;
    Lookup lk = irradiance_lookup(normal);
    float e[4];
    probe_page(&fb->tables[(size_t)cell * 144], &lk, e);
    if (!(e[3] > 0.0f)) return;
    *coverage = e[3];
    for (int c = 0; c < 3; ++c) out[c] = (e[c] * e[3]) / e[3];
}

OrcFrame *orc_frame_run_bounce(const OrcScene *S, const LuxSettings *st_in, const float *pos, const float *nrm,
                               uint32_t n, int threads, const OrcFrame *previous, const float *dirty,
                               uint32_t dirty_count, uint32_t max_cells, uint64_t max_entries,
                               const OrcFrame *feedback, uint32_t flags, float *hit_pos, float *hit_nrm,
                               const LuxCamera *camera) {
    const int sparse = (flags & ORC_FRAME_SPARSE) != 0u;
    Bounce bounce = {feedback, (flags & ORC_FRAME_SKIP_EMISSION) != 0u, (flags & ORC_FRAME_CACHED_SKY) != 0u};
    OrcFrame *F = (OrcFrame *)calloc(1, sizeof(OrcFrame));
    F->st = *st_in;
    lod_params(st_in, camera, &F->lod);
    /* History applies with history_frames > 0, a blend above zero and a
     * previous frame of the same cascade shape. */
    int same_shape = previous && previous->levels == st_in->levels;
    for (uint32_t l = 0; same_shape && l < st_in->levels; ++l)
        same_shape = previous->level[l].dirs == level_columns(st_in, l) * level_rows(st_in, l);
    if (same_shape && st_in->history_frames > 0 && (st_in->temporal_blend > 0.0f || st_in->transmittance_blend > 0.0f)) {
        F->previous = previous;
        F->dirty = dirty;
        F->dirty_count = dirty ? dirty_count : 0;
    }
    const LuxSettings *st = &F->st;
    F->levels = st->levels;
    /* seed: the cells of every level that hold a receiver. */
    Key *level_keys[LUX_MAX_LEVELS];
    uint32_t level_cells[LUX_MAX_LEVELS];
    for (uint32_t l = 0; l < F->levels; ++l) {
        Level *L = &F->level[l];
        L->columns = level_columns(st, l);
        L->rows = level_rows(st, l);
        L->dirs = L->columns * L->rows;
        Key *tmp = (Key *)malloc(sizeof(Key) * (2 * (size_t)n + 1));
        uint32_t present = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (sparse && pos[4 * (size_t)i + 3] == 0.0f) continue;
            /* Both LOD variants' cells in an overlap (seed, shaders/split.slang:758-786). */
            uint32_t low, high;
            float blend;
            point_lod(&F->lod, pos + 4 * (size_t)i, &low, &high, &blend);
            cell_key(st, l, pos + 4 * (size_t)i, low, tmp[present].k);
            tmp[present++].aux = st->frame_index;
            if (high != low) {
                cell_key(st, l, pos + 4 * (size_t)i, high, tmp[present].k);
                tmp[present++].aux = st->frame_index;
            }
        }
        qsort(tmp, present, sizeof(Key), key_cmp);
        uint32_t cells = 0;
        for (uint32_t i = 0; i < present; ++i)
            if (cells == 0 || key_cmp(&tmp[i], &tmp[cells - 1]) != 0) tmp[cells++] = tmp[i];
        level_keys[l] = tmp;
        level_cells[l] = cells;
    }
    if (F->previous && st->layout == LUX_LAYOUT_SPLIT) retain_cells(F, level_keys, level_cells, max_cells, max_entries);
    for (uint32_t l = 0; l < F->levels; ++l) {
        Level *L = &F->level[l];
        uint32_t cells = level_cells[l];
        L->cells = cells;
        L->keys = level_keys[l];
        L->last = (uint32_t *)malloc(sizeof(uint32_t) * (cells ? cells : 1));
        for (uint32_t c = 0; c < cells; ++c) L->last[c] = L->keys[c].aux;
        uint64_t entries = (uint64_t)cells * L->dirs;
        L->jsum = (float *)calloc(4 * entries + 4, sizeof(float));
        L->count = (uint32_t *)calloc(entries + 1, sizeof(uint32_t));
        L->merged = (float *)calloc(4 * entries + 4, sizeof(float));
        L->raw = (float *)calloc(4 * entries + 4, sizeof(float));
        L->mass = (float *)calloc(2 * entries + 2, sizeof(float));
        F->stats.cells[l] = cells;
        F->stats.entries[l] = entries;
    }
    F->stats.levels = F->levels;
    uint64_t shadow = 0;
    OrcCounters cn = {0, 0, 0};
    if (st->layout == LUX_LAYOUT_SPLIT) {
        uint64_t rays = (uint64_t)n * st->rays_per_receiver;
        FrameJob proto;
        memset(&proto, 0, sizeof proto);
        proto.S = S;
        proto.st = st;
        proto.pos = pos;
        proto.nrm = nrm;
        proto.n = n;
        proto.bounce = &bounce;
        proto.lod = &F->lod;
        proto.sparse = sparse;
        proto.hit_pos = (flags & ORC_FRAME_RECORD_HITS) ? hit_pos : NULL;
        proto.hit_nrm = (flags & ORC_FRAME_RECORD_HITS) ? hit_nrm : NULL;
        uint32_t *ordinal = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
        sequence_order(st, &F->lod, pos, n, sparse, ordinal);
        proto.ordinal = ordinal;
        proto.term_level = (int32_t *)malloc(sizeof(int32_t) * (rays ? rays : 1));
        proto.radiance = (float *)malloc(sizeof(float) * 3 * (rays ? rays : 1));
        proto.uv = (float *)malloc(sizeof(float) * 2 * (rays ? rays : 1));
        F->hits = (LuxHit *)malloc(sizeof(LuxHit) * (rays ? rays : 1));
        F->hit_count = rays;
        proto.hits = F->hits;
        run_jobs(&proto, rays, threads, split_job, &shadow, &cn);
        uint64_t present_rays = rays;
        /* deposit, shaders/split.slang:1056-1117, then the per-key mean of
         * reduce (shaders/split.slang:1386-1476), in ray order. */
        for (uint64_t ray = 0; ray < rays; ++ray) {
            int32_t term = proto.term_level[ray];
            if (term == -2) {  /* absent receiver of a sparse set */
                --present_rays;
                continue;
            }
            if (term < 0) {
                F->stats.unsupported++;
                continue;
            }
            uint32_t i = (uint32_t)(ray / st->rays_per_receiver);
            uint32_t lod = receiver_lod(&F->lod, pos + 4 * (size_t)i, i, st->frame_index);
            for (uint32_t l = 0; l <= (uint32_t)term; ++l) {
                Level *L = &F->level[l];
                int32_t key[4];
                cell_key(st, l, pos + 4 * (size_t)i, lod, key);
                int64_t cell = find_cell(L, key);
                uint32_t bin = orc_direction_index_uv(proto.uv[2 * ray], proto.uv[2 * ray + 1], L->columns, L->rows);
                uint64_t e = (uint64_t)cell * L->dirs + bin;
                L->count[e] += 1;
                if (l == (uint32_t)term) {
                    for (int c = 0; c < 3; ++c) L->jsum[4 * e + c] += proto.radiance[3 * ray + c];
                } else {
                    L->jsum[4 * e + 3] += 1.0f;
                }
                F->stats.deposits++;
            }
        }
        F->stats.interval_rays = present_rays;
        free(proto.term_level);
        free(proto.radiance);
        free(proto.uv);
        free(ordinal);
    } else {
        for (uint32_t l = 0; l < F->levels; ++l) {
            FrameJob proto;
            memset(&proto, 0, sizeof proto);
            proto.S = S;
            proto.st = st;
            proto.levels = F->level;
            proto.level = l;
            uint64_t total = (uint64_t)F->level[l].cells * F->level[l].dirs;
            run_jobs(&proto, total, threads, dense_job, &shadow, &cn);
            F->stats.interval_rays += total;
            for (uint64_t e = 0; e < total; ++e) {
                if (F->level[l].count[e]) F->stats.deposits++;
                else F->stats.unsupported++;
            }
        }
    }
    F->stats.shadow_rays = shadow;
    F->stats.nodes_visited = cn.nodes;
    F->stats.triangles_tested = cn.triangles;
    F->stats.instances_visited = cn.instances;
    /* merge, levels L-1 .. 0 (src/render.rs:9767-9777). */
    for (int l = (int)F->levels - 1; l >= 0; --l) merge_level(F, (uint32_t)l);
    /* pack every cascade-0 cell. */
    Level *L0 = &F->level[0];
    F->tables = (float *)calloc((size_t)L0->cells * 36 * 4 + 4, sizeof(float));
    for (uint32_t cell = 0; cell < L0->cells; ++cell)
        orc_pack_table(&L0->merged[4 * (uint64_t)cell * L0->dirs], L0->columns, L0->rows, &F->tables[(size_t)cell * 144]);
    return F;
}

void orc_frame_destroy(OrcFrame *F) {
    if (!F) return;
    for (uint32_t l = 0; l < F->levels; ++l) {
        free(F->level[l].keys);
        free(F->level[l].jsum);
        free(F->level[l].count);
        free(F->level[l].merged);
        free(F->level[l].raw);
        free(F->level[l].mass);
        free(F->level[l].last);
    }
    free(F->tables);
    free(F->hits);
    free(F);
}

uint64_t orc_frame_read_hits(const OrcFrame *F, LuxHit *out, uint64_t count) {
    uint64_t n = count < F->hit_count ? count : F->hit_count;
    if (n) memcpy(out, F->hits, sizeof(LuxHit) * n);
    return n;
}

uint32_t orc_frame_cells(const OrcFrame *F, uint32_t level) { return level < F->levels ? F->level[level].cells : 0; }

void orc_frame_read_level(const OrcFrame *F, uint32_t level, int32_t *keys, float *merged, float *raw,
                          uint32_t *samples) {
    if (level >= F->levels) return;
    const Level *L = &F->level[level];
    uint64_t entries = (uint64_t)L->cells * L->dirs;
    if (keys)
        for (uint32_t c = 0; c < L->cells; ++c) {
            memcpy(keys + 4 * (size_t)c, L->keys[c].k, 12);
            keys[4 * (size_t)c + 3] = (int32_t)((level << 12) | ((uint32_t)L->keys[c].k[3] << 18));
        }
    if (merged) memcpy(merged, L->merged, sizeof(float) * 4 * entries);
    if (raw) memcpy(raw, L->raw, sizeof(float) * 4 * entries);
    if (samples) memcpy(samples, L->count, sizeof(uint32_t) * entries);
}

void orc_frame_read_probes(const OrcFrame *F, float *tables) {
    memcpy(tables, F->tables, sizeof(float) * 144 * F->level[0].cells);
}

void orc_frame_stats(const OrcFrame *F, LuxStats *stats) { *stats = F->stats; }

/* diffuseAtLod (shaders/world_resolve.slang:96-150) over cascade-0 probe
 * tables (keys sorted ascending). */
static void diffuse_at_lod(const Level *L0, const float *tables, float s0, const float *p, const Lookup *lk,
                           uint32_t lod, float out[3], float *cov) {
    float s = s0 * lod_scale(lod);
    float grid[3], base[3], fr[3];
    for (int c = 0; c < 3; ++c) {
        grid[c] = p[c] / s - 0.5f;
        base[c] = floorf(grid[c]);
        fr[c] = grid[c] - base[c];
    }
    float sum[3] = {0, 0, 0}, observed = 0.0f, potential = 0.0f;
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        uint32_t bx = corner & 1u, by = (corner >> 1) & 1u, bz = corner >> 2;
        float ax = bx == 0u ? 1.0f - fr[0] : fr[0];
        float ay = by == 0u ? 1.0f - fr[1] : fr[1];
        float az = bz == 0u ? 1.0f - fr[2] : fr[2];
        float w = (ax * ay) * az;
        if (!(w > 0.0f)) continue;
        potential += w;
        int32_t key[4] = {(int32_t)base[0] + (int32_t)bx, (int32_t)base[1] + (int32_t)by,
                          (int32_t)base[2] + (int32_t)bz, (int32_t)lod};
        int64_t cell = find_cell(L0, key);
        if (cell < 0) continue;
        float probe[4];
        probe_page(&tables[(size_t)cell * 144], lk, probe);
        float support = probe[3];
        if (!(support > 0.0f)) continue;
        float weight = w * support;
        for (int c = 0; c < 3; ++c) sum[c] = sum[c] + probe[c] * weight;
        observed += weight;
    }
    out[0] = out[1] = out[2] = 0.0f;
    *cov = 0.0f;
    if (potential > 0.0f) {
        *cov = saturatef(observed / potential);
        if (observed > 0.0f)
            for (int c = 0; c < 3; ++c) out[c] = sum[c] / observed;
    }
}

/* worldResolve -> resolveSplitDiffuse (shaders/world_resolve.slang:96-196,
 * :281-313) over cascade-0 probe tables: keys sorted ascending, tables
 * float4[cells*36]; the LOD pair and blend of each point from `lod`. */
static void resolve_tables(const Key *keys, uint32_t cells, const float *tables, float s0, const LodParams *lod,
                           const float *position, const float *normal_in, uint32_t count, float *out) {
    Level L0;
    memset(&L0, 0, sizeof L0);
    L0.cells = cells;
    L0.keys = (Key *)keys;
    for (uint32_t i = 0; i < count; ++i) {
        const float *p = position + 4 * (size_t)i, *nn = normal_in + 4 * (size_t)i;
        float *o = out + 4 * (size_t)i;
        float diffuse[3] = {0, 0, 0}, coverage = 0.0f;
        int supported = 0;
        float n3[3] = {nn[0], nn[1], nn[2]};
        if (finite3(n3) && dot3(n3, n3) > 0.01f) {
            float l = length3(n3);
            float normal[3] = {n3[0] / l, n3[1] / l, n3[2] / l};
            Lookup lk = irradiance_lookup(normal);
            uint32_t low, high;
            float blend;
            point_lod(lod, p, &low, &high, &blend);
            float lo[3], low_cov, hi[3] = {0, 0, 0}, high_cov = 1.0f;
            diffuse_at_lod(&L0, tables, s0, p, &lk, low, lo, &low_cov);
            if (high != low) diffuse_at_lod(&L0, tables, s0, p, &lk, high, hi, &high_cov);
            /* resolveLodSource (a single LOD takes high coverage 1, blend 0). */
            float low_weight = low_cov * (1.0f - blend);
            float high_weight = high_cov * blend;
            float total = low_weight + high_weight;
            coverage = saturatef(total);
            for (int c = 0; c < 3; ++c)
                diffuse[c] = total > 0.0f ? (lo[c] * low_weight + hi[c] * high_weight) / total : 0.0f;
            supported = coverage > 0.0f && finite3(diffuse);
        }
        o[0] = diffuse[0];
        o[1] = diffuse[1];
        o[2] = diffuse[2];
        /* rawGiSupportAlpha, shaders/common.slang:323-326. */
        o[3] = supported ? 1.0f + 0.25f * coverage : -1.0f;
    }
}

void orc_frame_resolve(const OrcFrame *F, const float *position, const float *normal_in, uint32_t count, float *out) {
    resolve_tables(F->level[0].keys, F->level[0].cells, F->tables, orc_spacing(&F->st, 0), &F->lod, position,
                   normal_in, count, out);
}

void orc_resolve_tables(const int32_t *keys, uint32_t cells, const float *tables, float spacing, const float *position,
                        const float *normal, uint32_t count, float *out) {
    Key *sorted = (Key *)malloc(sizeof(Key) * (cells ? cells : 1));
    uint32_t *order = (uint32_t *)malloc(sizeof(uint32_t) * (cells ? cells : 1));
    for (uint32_t i = 0; i < cells; ++i) {
        memcpy(sorted[i].k, keys + 4 * (size_t)i, 12);
        sorted[i].k[3] = (int32_t)(((uint32_t)keys[4 * (size_t)i + 3] >> 18) & 31u);
        sorted[i].aux = i;
    }
    qsort(sorted, cells, sizeof(Key), key_cmp);
    float *tab = (float *)malloc(sizeof(float) * 144 * (cells ? cells : 1));
    for (uint32_t i = 0; i < cells; ++i) {
        order[i] = sorted[i].aux;
        memcpy(&tab[(size_t)i * 144], &tables[(size_t)order[i] * 144], sizeof(float) * 144);
    }
    resolve_tables(sorted, cells, tab, spacing, NULL, position, normal, count, out);
    free(sorted);
    free(order);
    free(tab);
}

/* ---- KAT helpers ---- */
uint32_t orc_deposit_levels(const LuxSettings *s, float distance, int hit, int unsupported, const float radiance[3],
                            float *out) {
    if (unsupported) return 0;
    uint32_t written = 0;
    for (uint32_t l = 0; l < s->levels; ++l) {
        int terminal = l + 1 == s->levels;
        int terminates = terminal || (distance > interval_start(s, l) && distance <= orc_interval_end(s, l));
        float *o = out + 4 * l;
        o[0] = terminates ? radiance[0] : 0.0f;
        o[1] = terminates ? radiance[1] : 0.0f;
        o[2] = terminates ? radiance[2] : 0.0f;
        o[3] = terminates ? 0.0f : 1.0f;
        ++written;
        if (terminates) break;
    }
    (void)hit;
    return written;
}

/* checkDenseSdf, src/transport_tests.rs:179-248, on the CPU. */
static float dense_box(const float p[3], const float c[3], const float h[3]) {
    float q[3] = {fabsf(p[0] - c[0]) - h[0], fabsf(p[1] - c[1]) - h[1], fabsf(p[2] - c[2]) - h[2]};
    float m[3] = {fmaxf(q[0], 0.0f), fmaxf(q[1], 0.0f), fmaxf(q[2], 0.0f)};
    return length3(m) + fminf(fmaxf(q[0], fmaxf(q[1], q[2])), 0.0f);
}
static float dense_scene(const float p[3], uint32_t *material) {
    static const float c1[3] = {-3, 0, 0}, h1[3] = {0.9f, 0.9f, 0.9f};
    static const float c3[3] = {0, 3, 0}, h3[3] = {2, 0.04f, 2};
    static const float c4[3] = {0, 0, 4}, h4[3] = {2, 0.5f, 0.03f};
    float d = dense_box(p, c1, h1);
    *material = 1;
    float q[3] = {p[0] - 3.0f, p[1] - 1.0f, p[2]};
    float sphere = length3(q) - 1.0f;
    if (sphere < d) { d = sphere; *material = 2; }
    float f = dense_box(p, c3, h3);
    if (f < d) { d = f; *material = 3; }
    float b = dense_box(p, c4, h4);
    if (b < d) { d = b; *material = 4; }
    return d;
}
void orc_dense_sdf_record(uint32_t index, float interval[4], float direction[4]) {
    uint32_t level = 0, offset = 0, dimension = 1, dcount = 1;
    for (uint32_t c = 0; c < 4; ++c) {
        dimension = 16u >> c;
        dcount = 32u << (2u * c);
        uint32_t count = dimension * dimension * dimension * dcount;
        if (index < offset + count) { level = c; break; }
        offset += count;
    }
    uint32_t local = index - offset;
    uint32_t di = local % dcount, probe = local / dcount;
    uint32_t x = probe % dimension, y = (probe / dimension) % dimension, z = probe / (dimension * dimension);
    float cell = (float)(1u << level);
    float origin[3] = {-8.0f + ((float)x + 0.5f) * cell, -8.0f + ((float)y + 0.5f) * cell,
                       -8.0f + ((float)z + 0.5f) * cell};
    float dir[3];
    orc_bin_direction(di, 8u << level, 4u << level, dir);
    float start = (float)((1u << level) - 1u) + 0.001f;
    float end = (float)((1u << (level + 1u)) - 1u);
    interval[0] = interval[1] = interval[2] = 0.0f;
    interval[3] = 1.0f;
    for (uint32_t step = 0; step < 96u && start <= end; ++step) {
        uint32_t material;
        float p[3] = {origin[0] + dir[0] * start, origin[1] + dir[1] * start, origin[2] + dir[2] * start};
        float d = dense_scene(p, &material);
        if (d < 0.001f) {
            if (material == 3u) {
                interval[0] = 6.0f; interval[1] = 2.0f; interval[2] = 0.5f; interval[3] = 0.0f;
            } else {
                interval[0] = interval[1] = interval[2] = interval[3] = 0.0f;
            }
            break;
        }
        start += fmaxf(d, 0.005f);
    }
    direction[0] = dir[0];
    direction[1] = dir[1];
    direction[2] = dir[2];
    direction[3] = (float)di;
}

/* --- FP64 reference irradiance (the error-report oracle; no reference
 * counterpart).  Restates lux_reference_irradiance: cosine-weighted rays,
 * interval radiance per ray, per-point means accumulated in double in
 * sample order, rounds of `round` samples with frame index seed + round. */

static uint32_t orc_hash(uint32_t value) { return orc_transport_hash(value); }

void orc_reference_sample(uint32_t p, uint32_t s, uint32_t seed, float *u1, float *u2) {
    uint32_t h1 = orc_hash(p ^ orc_hash(s ^ orc_hash(seed + 0x2545f491u)));
    uint32_t h2 = orc_hash(h1 ^ 0x68bc21ebu);
    *u1 = (float)(h1 >> 8) / 16777216.0f;
    *u2 = (float)(h2 >> 8) / 16777216.0f;
}

/* Cosine-weighted direction in the orthonormal frame of Duff et al. (2017). */
void orc_cosine_direction(const float n[3], float u1, float u2, float out[3]) {
    float sign = n[2] >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sign + n[2]);
    float b = n[0] * n[1] * a;
    float t[3] = {1.0f + sign * n[0] * n[0] * a, sign * b, -sign * n[0]};
    float bt[3] = {b, sign + n[1] * n[1] * a, -n[1]};
    float c, s;
    orc_sincos_turns(u2, &c, &s);
    float r = sqrtf(u1);
    float z = sqrtf(fmaxf(1.0f - u1, 0.0f));
    float x = r * c, y = r * s;
    for (int k = 0; k < 3; ++k) out[k] = (t[k] * x + bt[k] * y) + n[k] * z;
}

void orc_reference_irradiance(const OrcScene *S, const LuxSettings *settings_in, const float *position,
                              const float *normal, uint32_t count, uint32_t spp, uint32_t seed, uint32_t round,
                              double *out) {
    LuxSettings st = *settings_in;
    for (uint32_t p = 0; p < count; ++p) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        const float *P = position + 4 * (size_t)p, *N = normal + 4 * (size_t)p;
        for (uint32_t k = 0, s0 = 0; s0 < spp; ++k, s0 += round) {
            uint32_t samples = round < spp - s0 ? round : spp - s0;
            st.frame_index = seed + k;
            for (uint32_t s = s0; s < s0 + samples; ++s) {
                float u1, u2, d[3], o[3];
                orc_reference_sample(p, s, seed, &u1, &u2);
                orc_cosine_direction(N, u1, u2, d);
                orc_ray_offset(P, N, st.normal_bias, o);
                LuxHit hit;
                orc_trace_closest(S, o, d, 0.0f, 1e20f, &hit, NULL);
                float rad[3];
                uint64_t shadow = 0;
                if (!orc_outgoing_radiance(S, &st, o, d, &hit, rad, &shadow, NULL)) continue;
                acc[0] += (double)rad[0];
                acc[1] += (double)rad[1];
                acc[2] += (double)rad[2];
                acc[3] += 1.0;
            }
        }
        double *q = out + 4 * (size_t)p;
        if (acc[3] > 0.0) {
            q[0] = acc[0] / acc[3];
            q[1] = acc[1] / acc[3];
            q[2] = acc[2] / acc[3];
            q[3] = acc[3];
        } else {
            q[0] = q[1] = q[2] = q[3] = 0.0;
        }
    }
}

/* ======================================================================
 * Path-traced reference (the reference's trace_sample,
 * examples/pathtrace_reference.rs:724-833, from the receivers): emissive
 * next-event estimation with power-heuristic MIS against the cosine
 * proposal at every diffuse vertex, the last vertex's sample alone, Russian
 * roulette from the fourth vertex; Lambertian unit-albedo receiver (the raw
 * output's irradiance / pi), hit vertices with the diffuse colour and the
 * Disney diffuse factor.  Each sample in FP32 as liblux's lux_path_reference,
 * the per-point sums in FP64 in sample order.
 * ==================================================================== */
float orc_path_random(uint32_t p, uint32_t s, uint32_t seed, uint32_t dim) {
    uint32_t h = orc_hash(p ^ orc_hash(s ^ orc_hash(seed + 0x7f4a7c15u + dim * 0x9e3779b9u)));
    return (float)(h >> 8) / 16777216.0f;
}

typedef struct {
    float position[3], normal[3], gnormal[3], view[3], diffuse[3];
    float roughness;
    int lambert;
} PathVertex;

static float power_heuristic(float a, float b) {
    float aa = a * a;
    return aa / fmaxf(aa + b * b, 1e-30f);
}

static void path_response(const PathVertex *v, const float l[3], float out[3]) {
    if (v->lambert) {
        out[0] = out[1] = out[2] = 1.0f / PI_F;
        return;
    }
    float factor = disney_multiplier(v->normal, l, v->view, v->roughness) / PI_F;
    for (int c = 0; c < 3; ++c) out[c] = v->diffuse[c] * factor;
}

static uint32_t light_of(const OrcScene *S, uint32_t inst, uint32_t tri) {
    const LuxLight *L = S->lights + S->conventional;
    uint32_t n = S->light_count - S->conventional, lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (L[mid].source[0] < inst || (L[mid].source[0] == inst && L[mid].source[1] < tri))
            lo = mid + 1u;
        else
            hi = mid;
    }
    if (lo < n && L[lo].source[0] == inst && L[lo].source[1] == tri) return lo;
    return EMPTY;
}

static int path_next_event(const OrcScene *S, const LuxSettings *st, const PathVertex *v, float u0, float u1,
                           float u2, int competitor, float out[3]) {
    out[0] = out[1] = out[2] = 0.0f;
    uint32_t emissive = S->light_count - S->conventional;
    if (emissive == 0u) return 1;
    const LuxLight *lights = S->lights + S->conventional;
    uint32_t low = 0, high = emissive - 1u;
    while (low < high) {
        uint32_t middle = (low + high) / 2u;
        if (lights[middle].direction[3] < u0)
            low = middle + 1u;
        else
            high = middle;
    }
    const LuxLight *L = lights + low;
    const float bias = st->normal_bias;
    float rel[3] = {v->position[0] - L->position[0], v->position[1] - L->position[1], v->position[2] - L->position[2]};
    if (L->edge1[3] <= 0.0f || (L->position[3] != -2.0f && dot3(L->direction, rel) <= 0.0f)) return 1;
    float root = sqrtf(u1);
    float w1 = root * (1.0f - u2), w2 = root * u2;
    float target[3];
    for (int c = 0; c < 3; ++c) target[c] = (L->position[c] + L->edge1[c] * w1) + L->edge2[c] * w2;
    float to_light[3] = {target[0] - v->position[0], target[1] - v->position[1], target[2] - v->position[2]};
    float light_distance = length3(to_light);
    if (light_distance <= bias * 0.25f) return 1;
    float ld[3] = {to_light[0] / light_distance, to_light[1] / light_distance, to_light[2] / light_distance};
    float cosine = fmaxf(0.0f, dot3(v->normal, ld));
    float neg[3] = {-ld[0], -ld[1], -ld[2]};
    float c_emit = dot3(L->direction, neg);
    if (L->position[3] == -2.0f) c_emit = fabsf(c_emit);
    float emitter_cosine = fmaxf(0.0f, c_emit);
    if (cosine <= 0.0f || emitter_cosine <= 0.0f || dot3(v->gnormal, ld) <= 0.0f) return 1;
    float bary[3] = {1.0f - root, w1, w2};
    Surface es;
    surface_at(S, st, L->source[0], L->source[1], bary, &es);
    float emission[3] = {fmaxf(es.emission[0], 0.0f), fmaxf(es.emission[1], 0.0f), fmaxf(es.emission[2], 0.0f)};
    if (!(emission[0] > 0.0f || emission[1] > 0.0f || emission[2] > 0.0f)) return 1;
    float pdf = ((L->edge1[3] * light_distance) * light_distance) / (L->color[3] * emitter_cosine);
    float plane = fabsf(dot3(L->direction, rel));
    float origin[3];
    orc_ray_offset(v->position, v->gnormal, fminf(bias, plane * 0.25f), origin);
    float delta[3] = {target[0] - origin[0], target[1] - origin[1], target[2] - origin[2]};
    float distance = length3(delta);
    if (distance <= bias * 0.25f) return 1;
    float dir[3] = {delta[0] / distance, delta[1] / distance, delta[2] / distance};
    int supported;
    int blocked = orc_trace_occluded(S, origin, dir, distance - fminf(bias * 0.25f, distance * 0.001f), &supported,
                                     NULL);
    if (blocked) return 1;
    if (!supported) return 0;
    float f[3];
    path_response(v, ld, f);
    float mis = competitor ? power_heuristic(pdf, cosine / PI_F) : 1.0f;
    float p = fmaxf(pdf, 1e-20f);
    for (int c = 0; c < 3; ++c) out[c] = emission[c] * (((f[c] * cosine) / p) * mis);
    return 1;
}

static int path_hit_vertex(const OrcScene *S, const LuxSettings *st, const float origin[3], const float d[3],
                           const LuxHit *hit, PathVertex *v, float emission[3]) {
    Surface sf;
    surface_at(S, st, hit->instance, hit->triangle, hit->barycentric, &sf);
    for (int c = 0; c < 3; ++c) emission[c] = fmaxf(sf.emission[c], 0.0f);
    if (!finite3(emission)) emission[0] = emission[1] = emission[2] = 0.0f;
    if ((sf.flags & 16u) != 0u) return 0;
    uint32_t base = instance_base(S, hit->instance);
    U4 header = gword(S, 0);
    float A[3], B[3], C[3];
    uint32_t idx[3];
    local_triangle(S, hit->triangle, header, A, B, C, idx);
    float position[3];
    for (int c = 0; c < 3; ++c) position[c] = origin[c] + d[c] * hit->distance;
    float gn[3];
    geometric_normal(S, base, sf.flags, A, B, C, gn);
    float world_normal[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        U4 vw = gword(S, header.y + idx[i] * header.z);
        float nrm[3] = {gn[0], gn[1], gn[2]};
        if ((vw.w & 1u) != 0u) {
            U4 nw = gword(S, header.y + idx[i] * header.z + 1);
            float vn[3] = {asf(nw.x), asf(nw.y), asf(nw.z)}, tn[3];
            transform_direction(S, base, vn, 1, tn);
            unit_vector(tn, gn, nrm);
        }
        for (int c = 0; c < 3; ++c) world_normal[c] = world_normal[c] + nrm[c] * hit->barycentric[i];
    }
    float normal[3];
    unit_vector(world_normal, gn, normal);
    if (dot3(gn, d) > 0.0f && (sf.flags & 8u) != 0u) {
        normal[0] = -normal[0]; normal[1] = -normal[1]; normal[2] = -normal[2];
    }
    float flipped[3] = {gn[0], gn[1], gn[2]};
    if (dot3(gn, d) > 0.0f) {
        flipped[0] = -flipped[0]; flipped[1] = -flipped[1]; flipped[2] = -flipped[2];
    }
    float neg[3] = {-d[0], -d[1], -d[2]};
    if (dot3(normal, neg) <= 0.0f || dot3(normal, flipped) <= 0.0f) return 0;
    float nl = length3(neg);
    float metallic = saturatef(sf.metallic);
    float roughness = saturatef(sf.roughness);
    if (!isfinite(roughness)) roughness = 1.0f;
    int bf = finite3(sf.base_color);
    for (int c = 0; c < 3; ++c) {
        v->position[c] = position[c];
        v->normal[c] = normal[c];
        v->gnormal[c] = flipped[c];
        v->view[c] = neg[c] / nl;
        v->diffuse[c] = (bf ? saturatef(sf.base_color[c]) : 0.0f) * (1.0f - metallic);
    }
    v->roughness = roughness;
    v->lambert = 0;
    return finite3(position) && (v->diffuse[0] > 0.0f || v->diffuse[1] > 0.0f || v->diffuse[2] > 0.0f);
}

int orc_path_sample(const OrcScene *S, const LuxSettings *st, uint32_t bounces, uint32_t seed, uint32_t p,
                    const float pos[3], const float nrm[3], uint32_t s, float radiance[3]) {
    radiance[0] = radiance[1] = radiance[2] = 0.0f;
    float throughput[3] = {1.0f, 1.0f, 1.0f};
    PathVertex v;
    for (int c = 0; c < 3; ++c) {
        v.position[c] = pos[c];
        v.normal[c] = nrm[c];
        v.gnormal[c] = nrm[c];
        v.view[c] = nrm[c];
        v.diffuse[c] = 1.0f;
    }
    v.roughness = 1.0f;
    v.lambert = 1;
    for (uint32_t bounce = 0; bounce < bounces; ++bounce) {
        uint32_t dim = bounce * 6u;
        int competitor = bounce + 1u < bounces;
        float c3[3];
        if (!path_next_event(S, st, &v, orc_path_random(p, s, seed, dim), orc_path_random(p, s, seed, dim + 1u),
                             orc_path_random(p, s, seed, dim + 2u), competitor, c3))
            return 0;
        for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + throughput[c] * c3[c];
        if (!competitor) break;
        float d[3];
        orc_cosine_direction(v.normal, orc_path_random(p, s, seed, dim + 3u), orc_path_random(p, s, seed, dim + 4u), d);
        float cosine = dot3(v.normal, d);
        if (!(cosine > 0.0f) || dot3(v.gnormal, d) <= 0.0f) break;
        float pdf = cosine / PI_F;
        float f[3];
        path_response(&v, d, f);
        for (int c = 0; c < 3; ++c) throughput[c] = throughput[c] * ((f[c] * cosine) / pdf);
        if (bounce >= 3u) {
            float survival = fminf(fmaxf(fmaxf(throughput[0], fmaxf(throughput[1], throughput[2])), 0.05f), 0.95f);
            if (orc_path_random(p, s, seed, dim + 5u) >= survival) break;
            for (int c = 0; c < 3; ++c) throughput[c] = throughput[c] / survival;
        }
        float origin[3];
        orc_ray_offset(v.position, v.gnormal, st->normal_bias, origin);
        LuxHit hit;
        orc_trace_closest(S, origin, d, 0.0f, 1e20f, &hit, NULL);
        if ((hit.errors & HIT_QUERY_UNSUPPORTED) != 0u) return 0;
        if (hit.triangle == EMPTY) {
            for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + throughput[c] * st->environment[c];
            break;
        }
        PathVertex next;
        float emission[3];
        int scatters = path_hit_vertex(S, st, origin, d, &hit, &next, emission);
        if (emission[0] > 0.0f || emission[1] > 0.0f || emission[2] > 0.0f) {
            float mis = 1.0f;
            uint32_t li = light_of(S, hit.instance, hit.triangle);
            if (li != EMPTY) {
                const LuxLight *L = S->lights + S->conventional + li;
                float neg[3] = {-d[0], -d[1], -d[2]};
                float c_emit = dot3(L->direction, neg);
                if (L->position[3] == -2.0f) c_emit = fabsf(c_emit);
                if (c_emit > 0.0f && L->color[3] > 0.0f && L->edge1[3] > 0.0f)
                    mis = power_heuristic(pdf, ((L->edge1[3] * hit.distance) * hit.distance) / (L->color[3] * c_emit));
            }
            for (int c = 0; c < 3; ++c) radiance[c] = radiance[c] + (throughput[c] * emission[c]) * mis;
        }
        if (!scatters) break;
        v = next;
    }
    if (!finite3(radiance)) radiance[0] = radiance[1] = radiance[2] = 0.0f;
    return 1;
}

typedef struct {
    const OrcScene *S;
    const LuxSettings *st;
    const float *position, *normal;
    uint32_t spp, bounces, seed, begin, end;
    double *out;
} PathJob;

static void *path_job(void *arg) {
    PathJob *j = (PathJob *)arg;
    for (uint32_t p = j->begin; p < j->end; ++p) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (uint32_t s = 0; s < j->spp; ++s) {
            float r[3];
            if (!orc_path_sample(j->S, j->st, j->bounces, j->seed, p, j->position + 4 * (size_t)p,
                                 j->normal + 4 * (size_t)p, s, r))
                continue;
            acc[0] += (double)r[0];
            acc[1] += (double)r[1];
            acc[2] += (double)r[2];
            acc[3] += 1.0;
        }
        double *q = j->out + 4 * (size_t)p;
        if (acc[3] > 0.0) {
            q[0] = acc[0] / acc[3]; q[1] = acc[1] / acc[3]; q[2] = acc[2] / acc[3]; q[3] = acc[3];
        } else {
            q[0] = q[1] = q[2] = q[3] = 0.0;
        }
    }
    return NULL;
}

void orc_path_reference(const OrcScene *S, const LuxSettings *settings, const float *position, const float *normal,
                        uint32_t count, uint32_t spp, uint32_t bounces, uint32_t seed, int threads, double *out) {
    if (threads < 1) threads = 1;
    if ((uint32_t)threads > count) threads = count ? (int)count : 1;
    PathJob *jobs = (PathJob *)calloc((size_t)threads, sizeof(PathJob));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (PathJob){S, settings, position, normal, spp, bounces, seed,
                            (uint32_t)((uint64_t)count * t / threads), (uint32_t)((uint64_t)count * (t + 1) / threads),
                            out};
        pthread_create(&tid[t], NULL, path_job, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    free(jobs);
    free(tid);
}

/* ======================================================================
 * Screen reconstruction: temporal + denoise (shaders/cascades.slang:310-690)
 * for persistent world intervals without motion vectors; positions are the
 * caller's (xyz, view depth in w) and the previous positions are kept in the
 * history.  History words per pixel (ORC_SCREEN_WORDS): irradiance rgb +
 * depth, metadata (retained length, variance, support mask, surface flag),
 * position xyzw, normal xyzw, identity (2 words of raw bits).
 * ==================================================================== */
typedef struct {
    uint32_t width, height;
    float temporal_blend, capacity, tolerance, plane_scale;
    uint32_t history_valid, scene_changed, dirty;
    float dirty_lo[3], dirty_hi[3];
    float prev[16];
} ScreenParams;

static float lum3(const float *c) { return (c[0] * 0.2126f + c[1] * 0.7152f) + c[2] * 0.0722f; }

static float sdot(const float *a, const float *b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

/* surfacePlaneDistance, shaders/common.slang:585-591. */
static float plane_distance(const float delta[3], const float *target, const float *sample) {
    float avg[3] = {target[0] + sample[0], target[1] + sample[1], target[2] + sample[2]};
    float len2 = sdot(avg, avg);
    if (!(len2 > 1e-20f) || !isfinite(len2)) return fabsf(sdot(delta, target));
    float inv = 1.0f / sqrtf(len2);
    float n[3] = {avg[0] * inv, avg[1] * inv, avg[2] * inv};
    return fabsf(sdot(delta, n));
}

static int screen_compatible(int a_surface, const uint32_t *a_id, const float *a_n, int b_surface,
                             const uint32_t *b_id, const float *b_n) {
    return a_surface && b_surface && a_id[0] == b_id[0] && a_id[1] == b_id[1] && sdot(a_n, b_n) > 0.97f;
}

static int screen_dirty(const ScreenParams *P, const float *p) {
    return P->dirty && p[0] >= P->dirty_lo[0] && p[1] >= P->dirty_lo[1] && p[2] >= P->dirty_lo[2] &&
           p[0] <= P->dirty_hi[0] && p[1] <= P->dirty_hi[1] && p[2] <= P->dirty_hi[2];
}

static float lerpf_(float a, float b, float t) { return a + t * (b - a); }

#define HW ORC_SCREEN_WORDS
static const float *hw_irr(const float *h, size_t p) { return h + HW * p; }
static const float *hw_meta(const float *h, size_t p) { return h + HW * p + 4; }
static const float *hw_pos(const float *h, size_t p) { return h + HW * p + 8; }
static const float *hw_nrm(const float *h, size_t p) { return h + HW * p + 12; }
static const uint32_t *hw_id(const float *h, size_t p) { return (const uint32_t *)(h + HW * p + 16); }

static void screen_temporal(const ScreenParams *P, const float *irr, const float *pos, const float *nrm,
                            const uint32_t *ids, const float *H, float *out) {
    for (int y = 0; y < (int)P->height; ++y)
        for (int x = 0; x < (int)P->width; ++x) {
            size_t p = (size_t)y * P->width + x;
            float *o = out + HW * p;
            float center[4];
            memcpy(center, irr + 4 * p, 16);
            const float *position = pos + 4 * p;
            float depth = position[3];
            if (!(depth > 0.0f)) {
                memset(o, 0, sizeof(float) * HW);
                continue;
            }
            const float *gn = nrm + 4 * p;
            const uint32_t *id = ids + 2 * p;
            int current_finite = isfinite(center[3]) && finite3(center);
            uint32_t current_mask = current_finite && center[3] > 0.0f ? ((uint32_t)floorf(center[3]) & 1u) : 0u;
            int current_supported = current_mask != 0u && current_finite;
            float freshness = current_supported ? saturatef((center[3] - floorf(center[3])) * 4.0f) : 0.0f;
            if (!current_supported) center[0] = center[1] = center[2] = 0.0f;
            uint32_t output_mask = current_mask;
            float mean[3] = {0, 0, 0}, sq[3] = {0, 0, 0}, count = 0.0f;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int qx = x + dx, qy = y + dy;
                    if (qx < 0 || qy < 0 || qx >= (int)P->width || qy >= (int)P->height) continue;
                    size_t q = (size_t)qy * P->width + qx;
                    const float *v = irr + 4 * q;
                    if (v[3] <= 0.0f) continue;
                    uint32_t nmask = (uint32_t)floorf(v[3]) & 1u;
                    if (current_mask != 0u && nmask != current_mask) continue;
                    const float *op = pos + 4 * q;
                    if (op[3] <= 0.0f) continue;
                    const float *on = nrm + 4 * q;
                    if (!screen_compatible(1, id, gn, 1, ids + 2 * q, on)) continue;
                    float delta[3] = {op[0] - position[0], op[1] - position[1], op[2] - position[2]};
                    if (sdot(gn, on) < 0.95f || plane_distance(delta, gn, on) > P->tolerance) continue;
                    for (int c = 0; c < 3; ++c) {
                        mean[c] += v[c];
                        sq[c] += v[c] * v[c];
                    }
                    count += 1.0f;
                }
            float cdiv = fmaxf(count, 1.0f);
            float var[3], dev[3];
            for (int c = 0; c < 3; ++c) {
                mean[c] /= cdiv;
                sq[c] /= cdiv;
            }
            for (int c = 0; c < 3; ++c) {
                var[c] = fmaxf(0.0f, sq[c] - mean[c] * mean[c]);
                dev[c] = sqrtf(var[c]);
            }
            float hist[4] = {0, 0, 0, 0}, meta[4] = {0, 0, 0, 0}, total = 0.0f;
            uint32_t history_mask = 0u;
            const float *M = P->prev;
            float cx = ((M[0] * position[0] + M[1] * position[1]) + M[2] * position[2]) + M[3];
            float cy = ((M[4] * position[0] + M[5] * position[1]) + M[6] * position[2]) + M[7];
            float cw = ((M[12] * position[0] + M[13] * position[1]) + M[14] * position[2]) + M[15];
            float u = (cx / cw) * 0.5f + 0.5f, v = 0.5f - (cy / cw) * 0.5f;
            int projected = cw > 0.0f && isfinite(u) && isfinite(v);
            float px = u * (float)P->width, py = v * (float)P->height;
            if (projected && P->history_valid && !screen_dirty(P, position) && P->temporal_blend > 0.0f &&
                P->capacity > 0.0f && px >= 0.0f && py >= 0.0f && px < (float)P->width && py < (float)P->height) {
                float lx = px - 0.5f, ly = py - 0.5f;
                int bx = (int)floorf(lx), by = (int)floorf(ly);
                float lastx = (float)(P->width - 1u), lasty = (float)(P->height - 1u);
                float leftx = fminf((float)bx, lastx), lefty = fminf((float)by, lasty);
                float rightx = fminf((float)(bx + 1), lastx), righty = fminf((float)(by + 1), lasty);
                float fx = saturatef((lx - leftx) / fmaxf(rightx - leftx, 1.0f));
                float fy = saturatef((ly - lefty) / fmaxf(righty - lefty, 1.0f));
                for (int corner = 0; corner < 4; ++corner) {
                    int ox = bx + (corner & 1), oy = by + (corner >> 1);
                    if (ox < 0 || oy < 0 || ox >= (int)P->width || oy >= (int)P->height) continue;
                    size_t q = (size_t)oy * P->width + ox;
                    const float *old = hw_irr(H, q), *om = hw_meta(H, q), *onrm = hw_nrm(H, q), *opos = hw_pos(H, q);
                    if (om[0] <= 0.0f || old[3] <= 0.0f || !finite3(old) || sdot(gn, onrm) < 0.95f ||
                        !screen_compatible(1, id, gn, om[3] > 0.0f, hw_id(H, q), onrm))
                        continue;
                    if (screen_dirty(P, opos)) continue;
                    float delta[3] = {opos[0] - position[0], opos[1] - position[1], opos[2] - position[2]};
                    if (plane_distance(delta, gn, onrm) > P->tolerance) continue;
                    float wx = (corner & 1) ? fx : 1.0f - fx, wy = (corner >> 1) ? fy : 1.0f - fy;
                    float weight = wx * wy;
                    if (weight <= 0.0f) continue;
                    if (om[2] <= 0.0f) continue;
                    history_mask = 1u;
                    for (int c = 0; c < 4; ++c) {
                        hist[c] = hist[c] + old[c] * weight;
                        meta[c] = meta[c] + om[c] * weight;
                    }
                    total += weight;
                }
            }
            float capacity = fmaxf(P->capacity, 0.0f);
            float retained = current_supported ? freshness : 0.0f;
            float out_var = current_supported ? lum3(var) : 0.0f;
            if (total > 0.00001f) {
                for (int c = 0; c < 4; ++c) {
                    hist[c] /= total;
                    meta[c] /= total;
                }
                output_mask = history_mask;
                float old_length = fminf(meta[0], capacity);
                if (current_supported) {
                    if (freshness <= 0.00001f) {
                        memcpy(center, hist, 12);
                        retained = old_length;
                        out_var = meta[1];
                    } else {
                        int complete = freshness >= 1.0f;
                        float clipped[3] = {hist[0], hist[1], hist[2]};
                        if (count >= 2.0f && complete) {
                            float d = lum3(hist) - lum3(center);
                            float tv = fmaxf(meta[1], d * d * 0.25f);
                            float st = sqrtf(tv);
                            for (int c = 0; c < 3; ++c) {
                                float r = 2.5f * fmaxf(dev[c], st) + 0.0001f;
                                clipped[c] = fminf(fmaxf(hist[c], fmaxf(0.0f, mean[c] - r)), mean[c] + r);
                            }
                        }
                        float hl = lum3(hist), cl = lum3(center);
                        float delta = hl - cl;
                        float ll = lum3(clipped);
                        float change = fabsf(ll - cl) / fmaxf(fmaxf(ll, cl), 0.001f);
                        float reactive = P->scene_changed && complete ? 1.0f - change * change : 1.0f;
                        float ref_l = fmaxf(fmaxf(hl, cl), 0.001f);
                        float noise = sqrtf(fmaxf(meta[1], 0.0f)) / ref_l;
                        float threshold = fminf(fmaxf(3.0f * noise, 0.05f), 0.25f);
                        int step = freshness > 0.0f && complete && P->scene_changed && change > threshold;
                        if (step) old_length = 0.0f;
                        float weight = fminf(P->temporal_blend, old_length / (old_length + 1.0f));
                        weight = weight / fmaxf(weight + freshness * (1.0f - weight), 1e-8f);
                        weight *= reactive;
                        if (step) weight = 0.0f;
                        for (int c = 0; c < 3; ++c) center[c] = lerpf_(center[c], clipped[c], weight);
                        retained = fminf(capacity, old_length + freshness);
                        out_var = lerpf_(lum3(var), meta[1], weight) + (weight * (1.0f - weight)) * (delta * delta);
                    }
                } else {
                    memcpy(center, hist, 12);
                    retained = old_length;
                    out_var = meta[1];
                }
            }
            center[3] = current_supported || retained > 0.0f ? depth : 0.0f;
            memcpy(o, center, 16);
            o[4] = retained;
            o[5] = out_var;
            o[6] = (float)output_mask;
            o[7] = 1.0f;
            memcpy(o + 8, position, 16);
            memcpy(o + 12, gn, 16);
            memcpy(o + 16, id, 8);
        }
}

static void screen_denoise(const ScreenParams *P, uint32_t step, const float *pos, const float *T,
                           const float *src, const float *src_mask, float *dst, float *dst_mask) {
    static const float kernel[5] = {1.0f, 4.0f, 6.0f, 4.0f, 1.0f};
    for (int y = 0; y < (int)P->height; ++y)
        for (int x = 0; x < (int)P->width; ++x) {
            size_t p = (size_t)y * P->width + x;
            const float *center = src + 4 * p;
            int has_light = center[3] > 0.0f && isfinite(center[3]) && finite3(center);
            const float *position = pos + 4 * p;
            float depth = has_light ? center[3] : position[3];
            if (depth <= 0.0f || !isfinite(depth)) {
                memset(dst + 4 * p, 0, 16);
                dst_mask[p] = 0.0f;
                continue;
            }
            const float *tm = hw_meta(T, p);
            int surface = tm[3] > 0.0f;
            const uint32_t *id = hw_id(T, p);
            const float *gn = hw_nrm(T, p);
            uint32_t center_mask = (uint32_t)src_mask[p];
            int center_supported = tm[0] > 0.0f;
            float variance = fmaxf(tm[1], 0.0f);
            float cl = lum3(center);
            float sum[3] = {0, 0, 0}, total = 0.0f;
            for (int dy = -2; dy <= 2; ++dy) {
                int xr = abs(dy) == 2 ? 1 : 2;
                for (int dx = -xr; dx <= xr; ++dx) {
                    int qx = x + dx * (int)step, qy = y + dy * (int)step;
                    if (qx < 0 || qy < 0 || qx >= (int)P->width || qy >= (int)P->height) continue;
                    size_t q = (size_t)qy * P->width + qx;
                    const float *value = src + 4 * q;
                    if (value[3] <= 0.0f) continue;
                    const float *om = hw_meta(T, q);
                    if (om[0] <= 0.0f) continue;
                    const float *on = hw_nrm(T, q);
                    if (!screen_compatible(surface, id, gn, om[3] > 0.0f, hw_id(T, q), on)) continue;
                    uint32_t other_mask = (uint32_t)src_mask[q];
                    if (center_mask != 0u && other_mask != center_mask) continue;
                    if (center_mask == 0u && other_mask == 0u) continue;
                    const float *op = pos + 4 * q;
                    if (sdot(gn, on) < 0.95f) continue;
                    float delta[3] = {op[0] - position[0], op[1] - position[1], op[2] - position[2]};
                    float pd = plane_distance(delta, gn, on);
                    if (pd > P->tolerance) continue;
                    float c = fmaxf(0.0f, sdot(gn, on));
                    float c2 = c * c, c4 = c2 * c2, c8 = c4 * c4, c16 = c8 * c8, c32 = c16 * c16;
                    float weight = ((kernel[dx + 2] * kernel[dy + 2]) * c32) * expf(-pd / P->plane_scale);
                    if (center_supported) {
                        float scale = fmaxf(0.02f, 2.0f * sqrtf(fmaxf(variance + om[1], 0.0f)));
                        weight *= expf(-fabsf(lum3(value) - cl) / scale);
                    }
                    for (int k = 0; k < 3; ++k) sum[k] += value[k] * weight;
                    total += weight;
                }
            }
            int filtered = total > 0.00001f;
            float *o = dst + 4 * p;
            if (filtered) {
                for (int k = 0; k < 3; ++k) o[k] = sum[k] / total;
            } else {
                memcpy(o, center, 12);
            }
            float out_depth = has_light || center_supported || filtered ? depth : 0.0f;
            o[3] = out_depth;
            dst_mask[p] = out_depth > 0.0f ? 1.0f : 0.0f;
        }
}

void orc_screen_filter(const LuxSettings *settings, uint32_t width, uint32_t height, const float *irradiance,
                       const float *position, const float *normal, const uint32_t *identity,
                       const float previous_clip_from_world[16], const float *dirty, uint32_t scene_changed,
                       uint32_t spatial_filter_steps, uint32_t history_valid, const float *history_in,
                       float *history_out, float *out) {
    LuxSettings st = *settings;
    ScreenParams P;
    memset(&P, 0, sizeof P);
    P.width = width;
    P.height = height;
    P.temporal_blend = st.temporal_blend;
    P.capacity = (float)st.history_frames;
    P.tolerance = fmaxf(st.normal_bias * 2.0f, st.probe_spacing * 0.02f);
    P.plane_scale = fmaxf(st.normal_bias * 2.0f, st.probe_spacing * 0.05f);
    P.history_valid = history_valid;
    P.scene_changed = scene_changed;
    if (dirty) {
        P.dirty = 1;
        memcpy(P.dirty_lo, dirty, 12);
        memcpy(P.dirty_hi, dirty + 3, 12);
    }
    memcpy(P.prev, previous_clip_from_world, sizeof P.prev);
    screen_temporal(&P, irradiance, position, normal, identity, history_in, history_out);
    size_t n = (size_t)width * height;
    if (spatial_filter_steps == 0) {
        for (size_t p = 0; p < n; ++p) memcpy(out + 4 * p, hw_irr(history_out, p), 16);
        return;
    }
    float *a = (float *)malloc(n * 16), *b = (float *)malloc(n * 16);
    float *ma = (float *)malloc(n * 4), *mb = (float *)malloc(n * 4);
    float *src = a, *src_mask = ma;
    for (size_t p = 0; p < n; ++p) {
        memcpy(a + 4 * p, hw_irr(history_out, p), 16);
        ma[p] = hw_meta(history_out, p)[2];
    }
    for (uint32_t level = 0; level < spatial_filter_steps; ++level) {
        uint32_t step = level == 0 ? 1u : (1u << level);
        float *dst = src == a ? b : a, *dst_mask = src_mask == ma ? mb : ma;
        screen_denoise(&P, step, position, history_out, src, src_mask, dst, dst_mask);
        src = dst;
        src_mask = dst_mask;
    }
    memcpy(out, src, n * 16);
    free(a);
    free(b);
    free(ma);
    free(mb);
}
#undef HW
