/* orc_pack.c - the oracle's own scene packer (test infrastructure only).
 *
 * A C restatement of how bevy_lux turns meshes and instances into its GPU
 * word streams, written from the reference independently of liblux's packer
 * so the two can pin each other (tests/test_oracle_pack.py) and so the CPU
 * baseline needs nothing from liblux:
 *   build_tree             src/scene.rs:2398-2554 (binned SAH, 12 bins, leaves
 *                          <= 4 elements, depth <= 48, median fallback)
 *   tree_cost              src/scene.rs:2383-2396
 *   node_words             src/scene.rs:1025-1038
 *   pack_instances         src/scene.rs:1071-1122 (no render layers: zero layer
 *                          words; the entity id is the caller's instance index)
 *   geometry_words         src/scene.rs:809-823 (positions only, white colour)
 *   build_emissive_lights  src/scene.rs:2311-2372 (coverage 1, opaque materials)
 * The median fallback orders the range by centroid with Rust's total order
 * (f32::total_cmp) and keeps equal centroids in their current order before
 * splitting at len / 2; with coincident centroids (the only case in which the
 * binned search finds no split) that is the identity order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lux_oracle.h"

#define PACK_BINS 12
#define INSTANCE_WORDS 9u
#define MATERIAL_WORDS 8u
#define VERTEX_WORDS 5u
#define CDF_STEPS (1u << 24)

typedef struct {
    float mn[3], mx[3];
    uint32_t id;
} Elem;

typedef struct {
    float mn[3], mx[3];
    uint32_t first, count;
} PNode;

typedef struct {
    PNode *v;
    size_t n, cap;
} PNodes;

static void nodes_push(PNodes *a, PNode x) {
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 64;
        a->v = (PNode *)realloc(a->v, a->cap * sizeof(PNode));
    }
    a->v[a->n++] = x;
}

static uint32_t fbits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

static float bitsf(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* bounds_area, src/scene.rs:2378-2381. */
static double area_of(const float mn[3], const float mx[3]) {
    double x = (double)mx[0] - (double)mn[0], y = (double)mx[1] - (double)mn[1], z = (double)mx[2] - (double)mn[2];
    return 2.0 * (x * y + y * z + z * x);
}

static float centroid(const Elem *e, int axis) { return e->mn[axis] * 0.5f + e->mx[axis] * 0.5f; }

/* f32::total_cmp as an integer key. */
static int32_t total_key(float f) {
    int32_t i;
    memcpy(&i, &f, 4);
    return i ^ (int32_t)((uint32_t)(i >> 31) >> 1);
}

typedef struct {
    int32_t key;
    uint32_t pos;
    Elem e;
} Keyed;

static int keyed_cmp(const void *a, const void *b) {
    const Keyed *x = (const Keyed *)a, *y = (const Keyed *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos ? 1 : 0);
}

typedef struct {
    float mn[3], mx[3];
    size_t count;
} PBin;

static void bin_empty(PBin *b) {
    for (int i = 0; i < 3; ++i) {
        b->mn[i] = INFINITY;
        b->mx[i] = -INFINITY;
    }
    b->count = 0;
}

static void bin_join(PBin *b, const float mn[3], const float mx[3], size_t count) {
    for (int i = 0; i < 3; ++i) {
        b->mn[i] = fminf(b->mn[i], mn[i]);
        b->mx[i] = fmaxf(b->mx[i], mx[i]);
    }
    b->count += count;
}

static double bin_cost(const PBin *b) { return b->count == 0 ? 0.0 : area_of(b->mn, b->mx) * (double)b->count; }

static size_t bin_index(float c, float cmin, double span) {
    double x = ((double)c - (double)cmin) / span * (double)PACK_BINS;
    size_t i = x <= 0.0 ? 0 : (size_t)x;  /* `as usize` saturates at zero */
    return i < PACK_BINS - 1 ? i : PACK_BINS - 1;
}

/* build in build_tree (src/scene.rs:2405-2548). */
static void build(PNodes *nodes, size_t index, Elem *e, size_t len, uint32_t first, uint32_t depth,
                  uint32_t *max_depth) {
    PNode nd;
    for (int i = 0; i < 3; ++i) {
        nd.mn[i] = INFINITY;
        nd.mx[i] = -INFINITY;
    }
    for (size_t k = 0; k < len; ++k)
        for (int i = 0; i < 3; ++i) {
            nd.mn[i] = fminf(nd.mn[i], e[k].mn[i]);
            nd.mx[i] = fmaxf(nd.mx[i], e[k].mx[i]);
        }
    nd.first = first;
    nd.count = (uint32_t)len;
    nodes->v[index] = nd;
    if (depth > *max_depth) *max_depth = depth;
    if (len <= 4 || depth == 48) return;
    float cmin[3] = {INFINITY, INFINITY, INFINITY}, cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t k = 0; k < len; ++k)
        for (int i = 0; i < 3; ++i) {
            float c = centroid(&e[k], i);
            cmin[i] = fminf(cmin[i], c);
            cmax[i] = fmaxf(cmax[i], c);
        }
    double best = INFINITY, best_span = 0.0;
    int best_axis = -1;
    size_t best_bin = 0;
    for (int axis = 0; axis < 3; ++axis) {
        double span = (double)cmax[axis] - (double)cmin[axis];
        if (span <= 0.0) continue;
        PBin bins[PACK_BINS], right[PACK_BINS], sum, left;
        for (int b = 0; b < PACK_BINS; ++b) bin_empty(&bins[b]);
        for (size_t k = 0; k < len; ++k)
            bin_join(&bins[bin_index(centroid(&e[k], axis), cmin[axis], span)], e[k].mn, e[k].mx, 1);
        bin_empty(&sum);
        for (int b = PACK_BINS - 1; b >= 0; --b) {
            bin_join(&sum, bins[b].mn, bins[b].mx, bins[b].count);
            right[b] = sum;
        }
        bin_empty(&left);
        for (int b = 0; b < PACK_BINS - 1; ++b) {
            bin_join(&left, bins[b].mn, bins[b].mx, bins[b].count);
            double cost = bin_cost(&left) + bin_cost(&right[b + 1]);
            if (left.count > 0 && right[b + 1].count > 0 && cost < best) {
                best = cost;
                best_axis = axis;
                best_bin = (size_t)b;
                best_span = span;
            }
        }
    }
    size_t mid;
    if (best_axis >= 0) {
        size_t l = 0, r = len;
        while (l < r) {
            if (bin_index(centroid(&e[l], best_axis), cmin[best_axis], best_span) <= best_bin) {
                ++l;
            } else {
                --r;
                Elem t = e[l];
                e[l] = e[r];
                e[r] = t;
            }
        }
        mid = l;
    } else {
        float size[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
        int axis = size[0] >= size[1] && size[0] >= size[2] ? 0 : (size[1] >= size[2] ? 1 : 2);
        Keyed *tmp = (Keyed *)malloc(sizeof(Keyed) * len);
        for (size_t k = 0; k < len; ++k) {
            tmp[k].key = total_key(centroid(&e[k], axis));
            tmp[k].pos = (uint32_t)k;
            tmp[k].e = e[k];
        }
        qsort(tmp, len, sizeof(Keyed), keyed_cmp);
        for (size_t k = 0; k < len; ++k) e[k] = tmp[k].e;
        free(tmp);
        mid = len / 2;
    }
    size_t children = nodes->n;
    PNode blank;
    memset(&blank, 0, sizeof blank);
    nodes_push(nodes, blank);
    nodes_push(nodes, blank);
    nodes->v[index].first = (uint32_t)children;
    nodes->v[index].count = 0;
    build(nodes, children, e, mid, first, depth + 1, max_depth);
    build(nodes, children + 1, e + mid, len - mid, first + (uint32_t)mid, depth + 1, max_depth);
}

static PNodes build_tree(Elem *e, size_t len, uint32_t *max_depth) {
    PNodes nodes = {NULL, 0, 0};
    if (len == 0) return nodes;
    PNode blank;
    memset(&blank, 0, sizeof blank);
    nodes_push(&nodes, blank);
    build(&nodes, 0, e, len, 0, 0, max_depth);
    return nodes;
}

/* tree_cost, src/scene.rs:2383-2396. */
static double tree_cost(const PNodes *nodes) {
    if (nodes->n == 0) return 0.0;
    double root = area_of(nodes->v[0].mn, nodes->v[0].mx);
    if (root <= 0.0) return 0.0;
    double sum = 0.0;
    for (size_t i = 0; i < nodes->n; ++i)
        sum += area_of(nodes->v[i].mn, nodes->v[i].mx) * (double)(nodes->v[i].count ? nodes->v[i].count : 1u);
    return sum / root;
}

typedef struct {
    uint32_t *v;
    size_t n, cap;
} Words;

static void words_push(Words *w, uint32_t x, uint32_t y, uint32_t z, uint32_t a) {
    if (w->n + 4 > w->cap) {
        w->cap = w->cap ? 2 * w->cap : 1024;
        while (w->n + 4 > w->cap) w->cap *= 2;
        w->v = (uint32_t *)realloc(w->v, w->cap * sizeof(uint32_t));
    }
    w->v[w->n++] = x;
    w->v[w->n++] = y;
    w->v[w->n++] = z;
    w->v[w->n++] = a;
}

/* node_words, src/scene.rs:1025-1038: inner nodes' first child index offset
 * by `child_offset` (the TLAS node count for BLAS nodes). */
static void node_words(Words *w, const PNode *n, uint32_t child_offset) {
    words_push(w, fbits(n->mn[0]), fbits(n->mn[1]), fbits(n->mn[2]), n->count == 0 ? n->first + child_offset : n->first);
    words_push(w, fbits(n->mx[0]), fbits(n->mx[1]), fbits(n->mx[2]), n->count);
}

/* local_from_world: the f64 inverse of the 3x4 affine map, rounded to f32. */
static int affine_inverse(const float m[12], float out[12]) {
    double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], k = m[10];
    double det = a * (e * k - f * h) - b * (d * k - f * g) + c * (d * h - e * g);
    if (!(fabs(det) > 0.0) || !isfinite(det)) return 0;
    double inv[3][3] = {{(e * k - f * h) / det, (c * h - b * k) / det, (b * f - c * e) / det},
                        {(f * g - d * k) / det, (a * k - c * g) / det, (c * d - a * f) / det},
                        {(d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det}};
    double t[3] = {m[3], m[7], m[11]};
    for (int r = 0; r < 3; ++r) {
        for (int col = 0; col < 3; ++col) out[4 * r + col] = (float)inv[r][col];
        out[4 * r + 3] = (float)-(inv[r][0] * t[0] + inv[r][1] * t[1] + inv[r][2] * t[2]);
    }
    return 1;
}

struct OrcPacked {
    Words sw, gw;
    LuxLight *lights;
    uint32_t light_count;
    uint32_t *order;  /* packed instance slot -> caller instance */
    uint32_t tlas_nodes, blas_nodes, max_depth;
    double blas_cost;
};

void orc_packed_destroy(OrcPacked *p) {
    if (!p) return;
    free(p->sw.v);
    free(p->gw.v);
    free(p->lights);
    free(p->order);
    free(p);
}

int orc_scene_pack(const float *pos, uint32_t vertex_count, const uint32_t *idx, uint32_t triangle_count,
                   const uint32_t *mesh_first, const uint32_t *mesh_count, uint32_t meshes, const uint32_t *inst_mesh,
                   const float *inst_wfl, const uint32_t *inst_flags, const uint32_t *inst_material,
                   uint32_t instances, const uint32_t *material_words, uint32_t materials, OrcPacked **out) {
    *out = NULL;
    for (uint64_t t = 0; t < 3ull * triangle_count; ++t)
        if (idx[t] >= vertex_count) return -1;
    for (uint32_t m = 0; m < meshes; ++m)
        if ((uint64_t)mesh_first[m] + mesh_count[m] > triangle_count) return -1;
    for (uint32_t i = 0; i < instances; ++i)
        if (inst_mesh[i] >= meshes || inst_material[i] >= materials) return -1;
    OrcPacked *P = (OrcPacked *)calloc(1, sizeof(OrcPacked));
    /* BLAS per mesh (MeshCache::pack, src/scene.rs:880-1013), concatenated;
     * triangles in leaf order. */
    uint32_t *tri_order = (uint32_t *)malloc(sizeof(uint32_t) * (triangle_count ? triangle_count : 1));
    uint32_t tri_total = 0;
    PNodes blas = {NULL, 0, 0};
    uint32_t *root = (uint32_t *)calloc(meshes ? meshes : 1, sizeof(uint32_t));
    uint32_t *first_out = (uint32_t *)calloc(meshes ? meshes : 1, sizeof(uint32_t));
    float (*mbox)[6] = (float (*)[6])malloc(sizeof(float[6]) * (meshes ? meshes : 1));
    for (uint32_t m = 0; m < meshes; ++m) {
        uint32_t n = mesh_count[m];
        Elem *e = (Elem *)malloc(sizeof(Elem) * (n ? n : 1));
        for (uint32_t k = 0; k < n; ++k) {
            uint32_t t = mesh_first[m] + k;
            e[k].id = t;
            for (int i = 0; i < 3; ++i) {
                e[k].mn[i] = INFINITY;
                e[k].mx[i] = -INFINITY;
            }
            for (int v = 0; v < 3; ++v) {
                const float *p = pos + 3 * (size_t)idx[3 * (size_t)t + v];
                for (int i = 0; i < 3; ++i) {
                    e[k].mn[i] = fminf(e[k].mn[i], p[i]);
                    e[k].mx[i] = fmaxf(e[k].mx[i], p[i]);
                }
            }
        }
        PNodes tree = build_tree(e, n, &P->max_depth);
        double cost = tree_cost(&tree);
        if (cost > P->blas_cost) P->blas_cost = cost;
        uint32_t node_base = (uint32_t)blas.n;
        root[m] = node_base;
        first_out[m] = tri_total;
        for (uint32_t k = 0; k < n; ++k) tri_order[tri_total + k] = e[k].id;
        for (size_t k = 0; k < tree.n; ++k) {
            PNode nd = tree.v[k];
            nd.first += nd.count == 0 ? node_base : tri_total;
            nodes_push(&blas, nd);
        }
        for (int i = 0; i < 3; ++i) {
            mbox[m][i] = tree.n ? tree.v[0].mn[i] : INFINITY;
            mbox[m][3 + i] = tree.n ? tree.v[0].mx[i] : -INFINITY;
        }
        tri_total += n;
        free(tree.v);
        free(e);
    }
    /* Instances: inverse transform and the world box of the mesh box's
     * corners, padded by 8 f32 epsilons of each coordinate (src/scene.rs:1911-1924). */
    float *lfw = (float *)malloc(sizeof(float) * 12 * (instances ? instances : 1));
    Elem *ie = (Elem *)malloc(sizeof(Elem) * (instances ? instances : 1));
    int bad = 0;
    for (uint32_t i = 0; i < instances && !bad; ++i) {
        const float *w = inst_wfl + 12 * (size_t)i;
        if (!affine_inverse(w, lfw + 12 * (size_t)i)) bad = 1;
        const float *mb = mbox[inst_mesh[i]];
        ie[i].id = i;
        for (int r = 0; r < 3; ++r) {
            ie[i].mn[r] = INFINITY;
            ie[i].mx[r] = -INFINITY;
        }
        for (int corner = 0; corner < 8; ++corner) {
            double p[3] = {(corner & 1) ? mb[3] : mb[0], (corner & 2) ? mb[4] : mb[1], (corner & 4) ? mb[5] : mb[2]};
            for (int r = 0; r < 3; ++r) {
                double v = (double)w[4 * r] * p[0] + (double)w[4 * r + 1] * p[1] + (double)w[4 * r + 2] * p[2] +
                           (double)w[4 * r + 3];
                double pad = fabs(v) * 9.5367431640625e-7;
                if (pad < 1e-30) pad = 1e-30;
                ie[i].mn[r] = fminf(ie[i].mn[r], (float)(v - pad));
                ie[i].mx[r] = fmaxf(ie[i].mx[r], (float)(v + pad));
            }
        }
    }
    if (bad) {
        free(tri_order); free(blas.v); free(root); free(first_out); free(mbox); free(lfw); free(ie);
        orc_packed_destroy(P);
        return -1;
    }
    /* TLAS over the instances (src/scene.rs:2052). */
    PNodes tlas = build_tree(ie, instances, &P->max_depth);
    P->tlas_nodes = (uint32_t)tlas.n;
    P->blas_nodes = (uint32_t)blas.n;
    P->order = (uint32_t *)malloc(sizeof(uint32_t) * (instances ? instances : 1));
    for (uint32_t s = 0; s < instances; ++s) P->order[s] = ie[s].id;
    /* Scene words: header, TLAS, BLAS, instances, materials. */
    uint32_t base = 1u + 2u * (P->tlas_nodes + P->blas_nodes);
    uint32_t material_base = base + instances * INSTANCE_WORDS;
    words_push(&P->sw, material_base + materials * MATERIAL_WORDS, base, instances, INSTANCE_WORDS);
    for (size_t k = 0; k < tlas.n; ++k) node_words(&P->sw, &tlas.v[k], 0);
    for (size_t k = 0; k < blas.n; ++k) node_words(&P->sw, &blas.v[k], P->tlas_nodes);
    for (uint32_t s = 0; s < instances; ++s) {
        uint32_t i = P->order[s];
        const float *l = lfw + 12 * (size_t)i, *w = inst_wfl + 12 * (size_t)i;
        for (int r = 0; r < 3; ++r) words_push(&P->sw, fbits(l[4 * r]), fbits(l[4 * r + 1]), fbits(l[4 * r + 2]), fbits(l[4 * r + 3]));
        for (int r = 0; r < 3; ++r) words_push(&P->sw, fbits(w[4 * r]), fbits(w[4 * r + 1]), fbits(w[4 * r + 2]), fbits(w[4 * r + 3]));
        const uint32_t *mw = material_words + 32 * (size_t)inst_material[i];
        /* hardware_opaque: no cull test and an opaque material (alpha cutoff -1). */
        uint32_t opaque = (inst_flags[i] & 3u) == 0u && bitsf(mw[7]) == -1.0f;
        words_push(&P->sw, 0u, 0u, opaque, inst_flags[i]);
        words_push(&P->sw, i, 0u, 0u, material_base + inst_material[i] * MATERIAL_WORDS);
        uint32_t m = inst_mesh[i];
        words_push(&P->sw, P->tlas_nodes + root[m], first_out[m], mesh_count[m], 0u);
    }
    for (uint32_t k = 0; k < materials * MATERIAL_WORDS; ++k)
        words_push(&P->sw, material_words[4 * k], material_words[4 * k + 1], material_words[4 * k + 2],
                   material_words[4 * k + 3]);
    /* Geometry words: header {1, vertex base, 5, vertices}, one index word per
     * triangle (leaf order), padding to a multiple of 5 words, then 5 words
     * per vertex (position + flags, normal, tangent, uv, colour). */
    uint32_t vertex_base = (1u + triangle_count + VERTEX_WORDS - 1u) / VERTEX_WORDS * VERTEX_WORDS;
    words_push(&P->gw, 1u, vertex_base, VERTEX_WORDS, vertex_count);
    for (uint32_t t = 0; t < triangle_count; ++t) {
        uint32_t src = t < tri_total ? tri_order[t] : t;
        words_push(&P->gw, idx[3 * (size_t)src], idx[3 * (size_t)src + 1], idx[3 * (size_t)src + 2], 0u);
    }
    while (P->gw.n < 4 * (size_t)vertex_base) words_push(&P->gw, 0u, 0u, 0u, 0u);
    uint32_t one = fbits(1.0f);
    for (uint32_t v = 0; v < vertex_count; ++v) {
        const float *p = pos + 3 * (size_t)v;
        words_push(&P->gw, fbits(p[0]), fbits(p[1]), fbits(p[2]), 0u);
        words_push(&P->gw, 0u, 0u, 0u, 0u);
        words_push(&P->gw, 0u, 0u, 0u, one);
        words_push(&P->gw, 0u, 0u, 0u, 0u);
        words_push(&P->gw, one, one, one, one);
    }
    /* build_emissive_lights: one record per emissive triangle with positive
     * power (area x luminance of max(emission, 0)), in instance slot order,
     * then the CDF boundaries on the 2^24 grid. */
    size_t cap = 64, count = 0;
    LuxLight *lights = (LuxLight *)malloc(sizeof(LuxLight) * cap);
    double *power = (double *)malloc(sizeof(double) * cap);
    for (uint32_t s = 0; s < instances; ++s) {
        uint32_t i = P->order[s];
        const uint32_t *mw = material_words + 32 * (size_t)inst_material[i];
        float em[3];
        for (int c = 0; c < 3; ++c) em[c] = fmaxf(bitsf(mw[4 + c]), 0.0f);
        double lum = 0.2126 * em[0] + 0.7152 * em[1] + 0.0722 * em[2];
        if (!(lum > 0.0)) continue;
        uint32_t m = inst_mesh[i], cull = inst_flags[i] & 3u;
        const float *w = inst_wfl + 12 * (size_t)i;
        for (uint32_t t = first_out[m]; t < first_out[m] + mesh_count[m]; ++t) {
            uint32_t src = tri_order[t];
            float q[3][3];
            for (int v = 0; v < 3; ++v) {
                const float *p = pos + 3 * (size_t)idx[3 * (size_t)src + v];
                for (int r = 0; r < 3; ++r)
                    q[v][r] = (float)((double)w[4 * r] * p[0] + (double)w[4 * r + 1] * p[1] +
                                      (double)w[4 * r + 2] * p[2] + (double)w[4 * r + 3]);
            }
            double e1[3], e2[3];
            for (int r = 0; r < 3; ++r) {
                e1[r] = (double)q[1][r] - (double)q[0][r];
                e2[r] = (double)q[2][r] - (double)q[0][r];
            }
            double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            double len = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            double area = len * 0.5;
            double pw = (double)(float)area * lum;
            if (!isfinite(pw) || pw <= 0.0) continue;
            if (count == cap) {
                cap *= 2;
                lights = (LuxLight *)realloc(lights, sizeof(LuxLight) * cap);
                power = (double *)realloc(power, sizeof(double) * cap);
            }
            LuxLight *L = &lights[count];
            memset(L, 0, sizeof *L);
            double sign = cull == 2u ? -1.0 : 1.0;
            for (int r = 0; r < 3; ++r) {
                L->position[r] = q[0][r];
                L->color[r] = em[r];
                L->direction[r] = (float)(cr[r] / len * sign);
                L->edge1[r] = (float)e1[r];
                L->edge2[r] = (float)e2[r];
            }
            L->position[3] = cull == 0u ? -2.0f : -1.0f;
            L->color[3] = (float)area;
            L->source[0] = s;
            L->source[1] = t;
            power[count++] = pw;
        }
    }
    int rc = 0;
    if (count > CDF_STEPS) rc = -1;
    double total = 0.0;
    for (size_t k = 0; k < count; ++k) total += power[k];
    double cumulative = 0.0;
    uint32_t previous = 0;
    for (size_t k = 0; k < count && rc == 0; ++k) {
        cumulative += power[k];
        uint32_t boundary;
        if (k + 1 == count) {
            boundary = CDF_STEPS;
        } else {
            double ideal = round(cumulative / total * (double)CDF_STEPS);
            uint32_t u = ideal <= 0.0 ? 0u : (ideal >= 4294967295.0 ? 0xffffffffu : (uint32_t)ideal);
            uint32_t hi = CDF_STEPS - (uint32_t)(count - k - 1);
            if (u < previous + 1u) u = previous + 1u;
            if (u > hi) u = hi;
            boundary = u;
        }
        lights[k].direction[3] = (float)boundary / (float)CDF_STEPS;
        lights[k].edge1[3] = (float)(boundary - previous) / (float)CDF_STEPS;
        previous = boundary;
    }
    P->lights = lights;
    P->light_count = (uint32_t)count;
    free(power);
    free(tri_order); free(blas.v); free(tlas.v); free(root); free(first_out); free(mbox); free(lfw); free(ie);
    if (rc) {
        orc_packed_destroy(P);
        return rc;
    }
    *out = P;
    return 0;
}

void orc_packed_sizes(const OrcPacked *p, size_t *scene_words, size_t *geometry_words, uint32_t *lights,
                      uint32_t *tlas_nodes, uint32_t *blas_nodes, uint32_t *max_depth, double *blas_cost) {
    *scene_words = p->sw.n / 4;
    *geometry_words = p->gw.n / 4;
    *lights = p->light_count;
    *tlas_nodes = p->tlas_nodes;
    *blas_nodes = p->blas_nodes;
    *max_depth = p->max_depth;
    *blas_cost = p->blas_cost;
}

void orc_packed_copy(const OrcPacked *p, uint32_t *scene_words, uint32_t *geometry_words, LuxLight *lights,
                     uint32_t *instance_order, uint32_t instance_count) {
    memcpy(scene_words, p->sw.v, p->sw.n * 4);
    memcpy(geometry_words, p->gw.v, p->gw.n * 4);
    if (p->light_count) memcpy(lights, p->lights, sizeof(LuxLight) * p->light_count);
    if (instance_count) memcpy(instance_order, p->order, sizeof(uint32_t) * instance_count);
}
