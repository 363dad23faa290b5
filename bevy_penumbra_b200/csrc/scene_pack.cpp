// scene_pack.cpp - packs meshes and instances into bevy_lux's GPU word
// streams (GiScene / SceneData, src/scene.rs:130-171).
//
// Restated pieces, each cited at its definition:
//   build_tree      binned SAH, 12 bins, leaves <= 4, depth <= 48
//   tree_cost       normalised SAH cost
//   node_words      two uint4 words per binary node
//   pack_instances  nine uint4 words per instance
//   geometry_words  header, triangle index words, 5 words per vertex
//   build_emissive_lights  power-weighted emitter CDF on a 2^24 grid
// The output is what lux_scene_upload and the CPU oracle both consume.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/lux.h"
#include "lux_internal.h"

namespace {

struct Box {
    float mn[3];
    float mx[3];
};

struct BinNode {
    float mn[3];
    float mx[3];
    uint32_t first;
    uint32_t count;
};

// bounds_area, src/scene.rs:2378-2381.
double bounds_area(const float mn[3], const float mx[3]) {
    double sx = (double)mx[0] - (double)mn[0];
    double sy = (double)mx[1] - (double)mn[1];
    double sz = (double)mx[2] - (double)mn[2];
    return 2.0 * (sx * sy + sy * sz + sz * sx);
}

// tree_cost, src/scene.rs:2383-2396.
double tree_cost(const std::vector<BinNode> &nodes) {
    if (nodes.empty()) return 0.0;
    double area = bounds_area(nodes[0].mn, nodes[0].mx);
    if (area <= 0.0) return 0.0;
    double sum = 0.0;
    for (const BinNode &n : nodes) sum += bounds_area(n.mn, n.mx) * (double)std::max<uint32_t>(n.count, 1u);
    return sum / area;
}

struct BuildElement {
    Box box;
    uint32_t id;
};

constexpr int kBins = 12;

struct Bin {
    float mn[3];
    float mx[3];
    size_t count;
    Bin() {
        for (int i = 0; i < 3; ++i) {
            mn[i] = INFINITY;
            mx[i] = -INFINITY;
        }
        count = 0;
    }
    void join(const Bin &o) {
        for (int i = 0; i < 3; ++i) {
            mn[i] = std::min(mn[i], o.mn[i]);
            mx[i] = std::max(mx[i], o.mx[i]);
        }
        count += o.count;
    }
    void add(const Box &b) {
        for (int i = 0; i < 3; ++i) {
            mn[i] = std::min(mn[i], b.mn[i]);
            mx[i] = std::max(mx[i], b.mx[i]);
        }
        count += 1;
    }
    double cost() const { return count == 0 ? 0.0 : bounds_area(mn, mx) * (double)count; }
};

inline float center_of(const Box &b, int axis) { return b.mn[axis] * 0.5f + b.mx[axis] * 0.5f; }

// build_tree, src/scene.rs:2398-2554.  Elements are permuted in place into
// leaf order; node 0 is the root and children of an inner node are adjacent.
void build_node(std::vector<BinNode> &nodes, size_t index, BuildElement *e, size_t len, uint32_t first,
                uint32_t depth, uint32_t &max_depth) {
    BinNode node;
    for (int i = 0; i < 3; ++i) {
        node.mn[i] = INFINITY;
        node.mx[i] = -INFINITY;
    }
    for (size_t k = 0; k < len; ++k)
        for (int i = 0; i < 3; ++i) {
            node.mn[i] = std::min(node.mn[i], e[k].box.mn[i]);
            node.mx[i] = std::max(node.mx[i], e[k].box.mx[i]);
        }
    node.first = first;
    node.count = (uint32_t)len;
    nodes[index] = node;
    max_depth = std::max(max_depth, depth);
    if (len <= 4 || depth == 48) return;
    float cmin[3] = {INFINITY, INFINITY, INFINITY}, cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t k = 0; k < len; ++k)
        for (int i = 0; i < 3; ++i) {
            float c = center_of(e[k].box, i);
            cmin[i] = std::min(cmin[i], c);
            cmax[i] = std::max(cmax[i], c);
        }
    double best = INFINITY;
    int split_axis = -1;
    size_t split_bin = 0;
    double split_span = 0.0;
    auto bin_of = [&](float c, int axis, double span) {
        double x = ((double)c - (double)cmin[axis]) / span * (double)kBins;
        size_t b = x <= 0.0 ? 0 : (size_t)x;
        return std::min<size_t>(b, kBins - 1);
    };
    for (int axis = 0; axis < 3; ++axis) {
        double span = (double)cmax[axis] - (double)cmin[axis];
        if (span <= 0.0) continue;
        Bin bins[kBins];
        for (size_t k = 0; k < len; ++k) bins[bin_of(center_of(e[k].box, axis), axis, span)].add(e[k].box);
        Bin right[kBins];
        Bin sum;
        for (int i = kBins - 1; i >= 0; --i) {
            sum.join(bins[i]);
            right[i] = sum;
        }
        Bin left;
        for (int i = 0; i < kBins - 1; ++i) {
            left.join(bins[i]);
            double cost = left.cost() + right[i + 1].cost();
            if (left.count > 0 && right[i + 1].count > 0 && cost < best) {
                best = cost;
                split_axis = axis;
                split_bin = (size_t)i;
                split_span = span;
            }
        }
    }
    size_t mid;
    if (split_axis >= 0) {
        size_t l = 0, r = len;
        while (l < r) {
            if (bin_of(center_of(e[l].box, split_axis), split_axis, split_span) <= split_bin) {
                ++l;
            } else {
                --r;
                std::swap(e[l], e[r]);
            }
        }
        mid = l;
    } else {
        float size[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
        int axis = (size[0] >= size[1] && size[0] >= size[2]) ? 0 : (size[1] >= size[2] ? 1 : 2);
        // select_nth_unstable_by(total_cmp) leaves the order inside each half
        // unspecified; a stable sort by the same total order fixes it (equal
        // centroids keep their current order), so the oracle's packer can
        // restate the result exactly.  The binned search above finds a split
        // whenever two centroids differ, so in practice this runs on
        // coincident centroids and keeps the range as it is.
        mid = len / 2;
        auto total = [](float f) {
            int32_t i;
            std::memcpy(&i, &f, 4);
            return i ^ (int32_t)((uint32_t)(i >> 31) >> 1);
        };
        std::stable_sort(e, e + len, [axis, &total](const BuildElement &a, const BuildElement &b) {
            return total(center_of(a.box, axis)) < total(center_of(b.box, axis));
        });
    }
    size_t children = nodes.size();
    nodes.resize(children + 2);
    nodes[index].first = (uint32_t)children;
    nodes[index].count = 0;
    build_node(nodes, children, e, mid, first, depth + 1, max_depth);
    build_node(nodes, children + 1, e + mid, len - mid, first + (uint32_t)mid, depth + 1, max_depth);
}

std::vector<BinNode> build_tree(std::vector<BuildElement> &elements, uint32_t &max_depth) {
    std::vector<BinNode> nodes;
    if (elements.empty()) return nodes;
    nodes.resize(1);
    build_node(nodes, 0, elements.data(), elements.size(), 0, 0, max_depth);
    return nodes;
}

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// node_words, src/scene.rs:1025-1038.
void push_node_words(std::vector<uint32_t> &out, const BinNode &n, uint32_t child_offset) {
    uint32_t first = n.first + (n.count == 0 ? child_offset : 0u);
    out.insert(out.end(), {fbits(n.mn[0]), fbits(n.mn[1]), fbits(n.mn[2]), first});
    out.insert(out.end(), {fbits(n.mx[0]), fbits(n.mx[1]), fbits(n.mx[2]), n.count});
}

}  // namespace

struct LuxPackedScene {
    std::vector<uint32_t> scene_words;     // uint4 words flattened
    std::vector<uint32_t> geometry_words;  // uint4 words flattened
    std::vector<LuxLight> lights;
    std::vector<uint32_t> instance_order;  // packed instance -> caller instance
    uint32_t tlas_nodes = 0, blas_nodes = 0;
    double blas_cost = 0.0;
    uint32_t max_depth = 0;
};

extern "C" lux_status lux_scene_pack(const float *positions, uint32_t vertex_count, const uint32_t *indices,
                                     uint32_t triangle_count, const uint32_t *mesh_first_triangle,
                                     const uint32_t *mesh_triangle_count, uint32_t mesh_count,
                                     const uint32_t *instance_mesh, const float *instance_world_from_local,
                                     const uint32_t *instance_flags, const uint32_t *instance_material,
                                     uint32_t instance_count, const uint32_t *material_words,
                                     uint32_t material_count, LuxPackedScene **out) {
    if (!out) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if ((vertex_count && !positions) || (triangle_count && !indices) || (mesh_count && (!mesh_first_triangle || !mesh_triangle_count)) ||
        (instance_count && (!instance_mesh || !instance_world_from_local || !instance_flags || !instance_material)) ||
        (material_count && !material_words))
        return LUX_ERR_INVALID_ARGUMENT;
    for (uint32_t t = 0; t < 3u * triangle_count; ++t)
        if (indices[t] >= vertex_count) return LUX_ERR_INVALID_ARGUMENT;
    for (uint32_t m = 0; m < mesh_count; ++m)
        if ((uint64_t)mesh_first_triangle[m] + mesh_triangle_count[m] > triangle_count) return LUX_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < instance_count; ++i)
        if (instance_mesh[i] >= mesh_count || instance_material[i] >= material_count) return LUX_ERR_INVALID_ARGUMENT;

    LuxPackedScene *P = new (std::nothrow) LuxPackedScene();
    if (!P) return LUX_ERR_OUT_OF_MEMORY;
    try {
        // --- BLAS per mesh (MeshCache::pack, src/scene.rs:880-1013) ---
        std::vector<uint32_t> tri_order;  // packed triangle -> caller triangle
        tri_order.reserve(triangle_count);
        std::vector<BinNode> blas;
        std::vector<uint32_t> mesh_root(mesh_count), mesh_first(mesh_count), mesh_count_out(mesh_count);
        std::vector<Box> mesh_box(mesh_count);
        for (uint32_t m = 0; m < mesh_count; ++m) {
            std::vector<BuildElement> elems(mesh_triangle_count[m]);
            for (uint32_t k = 0; k < mesh_triangle_count[m]; ++k) {
                uint32_t t = mesh_first_triangle[m] + k;
                BuildElement &be = elems[k];
                be.id = t;
                for (int i = 0; i < 3; ++i) {
                    be.box.mn[i] = INFINITY;
                    be.box.mx[i] = -INFINITY;
                }
                for (int v = 0; v < 3; ++v) {
                    const float *p = positions + 3 * (size_t)indices[3 * (size_t)t + v];
                    for (int i = 0; i < 3; ++i) {
                        be.box.mn[i] = std::min(be.box.mn[i], p[i]);
                        be.box.mx[i] = std::max(be.box.mx[i], p[i]);
                    }
                }
            }
            uint32_t depth = 0;
            std::vector<BinNode> nodes = build_tree(elems, depth);
            P->max_depth = std::max(P->max_depth, depth);
            P->blas_cost = std::max(P->blas_cost, tree_cost(nodes));
            uint32_t tri_base = (uint32_t)tri_order.size();
            uint32_t node_base = (uint32_t)blas.size();
            for (const BuildElement &be : elems) tri_order.push_back(be.id);
            for (BinNode n : nodes) {
                if (n.count == 0) n.first += node_base;
                else n.first += tri_base;
                blas.push_back(n);
            }
            mesh_root[m] = node_base;
            mesh_first[m] = tri_base;
            mesh_count_out[m] = mesh_triangle_count[m];
            if (!nodes.empty()) {
                std::memcpy(mesh_box[m].mn, nodes[0].mn, sizeof(mesh_box[m].mn));
                std::memcpy(mesh_box[m].mx, nodes[0].mx, sizeof(mesh_box[m].mx));
            } else {
                for (int i = 0; i < 3; ++i) {
                    mesh_box[m].mn[i] = INFINITY;
                    mesh_box[m].mx[i] = -INFINITY;
                }
            }
        }
        // --- instances: inverse transforms and world bounds ---
        struct Inst {
            double w[3][4];
            float lfw[3][4];
            float wfl[3][4];
            Box box;
        };
        std::vector<Inst> inst(instance_count);
        std::vector<BuildElement> ielems(instance_count);
        for (uint32_t i = 0; i < instance_count; ++i) {
            Inst &I = inst[i];
            const float *m = instance_world_from_local + 12 * (size_t)i;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 4; ++c) {
                    I.w[r][c] = m[4 * r + c];
                    I.wfl[r][c] = m[4 * r + c];
                }
            float lfw[12];
            if (!lux_affine_inverse(m, lfw)) {
                delete P;
                return LUX_ERR_INVALID_ARGUMENT;
            }
            for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc < 4; ++cc) I.lfw[r][cc] = lfw[4 * r + cc];
            const Box &mb = mesh_box[instance_mesh[i]];
            Box wb;
            for (int r = 0; r < 3; ++r) {
                wb.mn[r] = INFINITY;
                wb.mx[r] = -INFINITY;
            }
            for (int corner = 0; corner < 8; ++corner) {
                double p[3] = {(corner & 1) ? mb.mx[0] : mb.mn[0], (corner & 2) ? mb.mx[1] : mb.mn[1],
                               (corner & 4) ? mb.mx[2] : mb.mn[2]};
                for (int r = 0; r < 3; ++r) {
                    double v = I.w[r][0] * p[0] + I.w[r][1] * p[1] + I.w[r][2] * p[2] + I.w[r][3];
                    double pad = std::max(std::fabs(v) * 9.5367431640625e-7, 1e-30);
                    wb.mn[r] = std::min(wb.mn[r], (float)(v - pad));
                    wb.mx[r] = std::max(wb.mx[r], (float)(v + pad));
                }
            }
            I.box = wb;
            ielems[i].box = wb;
            ielems[i].id = i;
        }
        // --- TLAS over instances (src/scene.rs:2052) ---
        uint32_t tdepth = 0;
        std::vector<BinNode> tlas = build_tree(ielems, tdepth);
        P->max_depth = std::max(P->max_depth, tdepth);
        uint32_t tlas_count = (uint32_t)tlas.size();
        P->tlas_nodes = tlas_count;
        P->blas_nodes = (uint32_t)blas.size();
        P->instance_order.resize(instance_count);
        for (uint32_t i = 0; i < instance_count; ++i) P->instance_order[i] = ielems[i].id;

        // --- scene words: header, TLAS nodes, BLAS nodes, instances, materials ---
        const uint32_t kInstanceWords = 9, kMaterialWords = 8;
        size_t blas_words = 2 * blas.size();
        size_t base = 1 + 2 * (size_t)tlas_count + blas_words;
        size_t material_base = base + (size_t)instance_count * kInstanceWords;
        std::vector<uint32_t> &sw = P->scene_words;
        sw.reserve(4 * (material_base + (size_t)material_count * kMaterialWords));
        sw.insert(sw.end(), {(uint32_t)(material_base + (size_t)material_count * kMaterialWords), (uint32_t)base,
                             instance_count, kInstanceWords});
        for (const BinNode &n : tlas) push_node_words(sw, n, 0);
        for (const BinNode &n : blas) push_node_words(sw, n, tlas_count);
        // pack_instances, src/scene.rs:1071-1122.
        for (uint32_t slot = 0; slot < instance_count; ++slot) {
            uint32_t i = P->instance_order[slot];
            const Inst &I = inst[i];
            for (int r = 0; r < 3; ++r)
                sw.insert(sw.end(), {fbits(I.lfw[r][0]), fbits(I.lfw[r][1]), fbits(I.lfw[r][2]), fbits(I.lfw[r][3])});
            for (int r = 0; r < 3; ++r)
                sw.insert(sw.end(), {fbits(I.wfl[r][0]), fbits(I.wfl[r][1]), fbits(I.wfl[r][2]), fbits(I.wfl[r][3])});
            uint32_t flags = instance_flags[i];
            const uint32_t *mw = material_words + 32 * (size_t)instance_material[i];
            uint32_t opaque = (flags & 3u) == 0u && mw[7] == fbits(-1.0f) ? 1u : 0u;
            sw.insert(sw.end(), {0u, 0u, opaque, flags});
            sw.insert(sw.end(), {i, 0u, 0u, (uint32_t)(material_base + (size_t)instance_material[i] * kMaterialWords)});
            uint32_t mesh = instance_mesh[i];
            sw.insert(sw.end(), {tlas_count + mesh_root[mesh], mesh_first[mesh], mesh_count_out[mesh], 0u});
        }
        sw.insert(sw.end(), material_words, material_words + 32 * (size_t)material_count);

        // --- geometry words, src/scene.rs:809-823 ---
        const uint32_t kVertexWords = 5;
        uint32_t vertex_base = (1u + triangle_count + kVertexWords - 1u) / kVertexWords * kVertexWords;
        std::vector<uint32_t> &gw = P->geometry_words;
        gw.reserve(4 * ((size_t)vertex_base + (size_t)vertex_count * kVertexWords));
        gw.insert(gw.end(), {1u, vertex_base, kVertexWords, vertex_count});
        for (uint32_t t = 0; t < triangle_count; ++t) {
            uint32_t src = t < tri_order.size() ? tri_order[t] : t;
            gw.insert(gw.end(), {indices[3 * (size_t)src], indices[3 * (size_t)src + 1], indices[3 * (size_t)src + 2], 0u});
        }
        gw.resize(4 * (size_t)vertex_base, 0u);
        const uint32_t one = fbits(1.0f);
        for (uint32_t v = 0; v < vertex_count; ++v) {
            const float *p = positions + 3 * (size_t)v;
            gw.insert(gw.end(), {fbits(p[0]), fbits(p[1]), fbits(p[2]), 0u});  // position, flags (no normal)
            gw.insert(gw.end(), {0u, 0u, 0u, 0u});                             // normal
            gw.insert(gw.end(), {0u, 0u, 0u, one});                            // tangent
            gw.insert(gw.end(), {0u, 0u, 0u, 0u});                             // uv
            gw.insert(gw.end(), {one, one, one, one});                         // colour
        }

        // --- emissive lights, build_emissive_lights src/scene.rs:2311-2372 ---
        struct Cand {
            LuxLight light;
            double power;
        };
        std::vector<Cand> cands;
        for (uint32_t slot = 0; slot < instance_count; ++slot) {
            uint32_t i = P->instance_order[slot];
            const uint32_t *mw = material_words + 32 * (size_t)instance_material[i];
            float emission[3];
            for (int c = 0; c < 3; ++c) {
                float v;
                std::memcpy(&v, &mw[4 + c], 4);
                emission[c] = std::max(v, 0.0f);
            }
            double lum = 0.2126 * emission[0] + 0.7152 * emission[1] + 0.0722 * emission[2];
            if (!(lum > 0.0)) continue;
            uint32_t mesh = instance_mesh[i];
            const Inst &I = inst[i];
            uint32_t cull = instance_flags[i] & 3u;
            for (uint32_t t = mesh_first[mesh]; t < mesh_first[mesh] + mesh_count_out[mesh]; ++t) {
                uint32_t src = tri_order[t];
                float w[3][3];
                for (int v = 0; v < 3; ++v) {
                    const float *p = positions + 3 * (size_t)indices[3 * (size_t)src + v];
                    for (int r = 0; r < 3; ++r)
                        w[v][r] = (float)(I.w[r][0] * p[0] + I.w[r][1] * p[1] + I.w[r][2] * p[2] + I.w[r][3]);
                }
                double e1[3], e2[3];
                for (int r = 0; r < 3; ++r) {
                    e1[r] = (double)w[1][r] - w[0][r];
                    e2[r] = (double)w[2][r] - w[0][r];
                }
                double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
                double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
                double area = len * 0.5;
                double power = (double)(float)area * lum * 1.0;
                if (!std::isfinite(power) || power <= 0.0) continue;
                Cand cd;
                std::memset(&cd.light, 0, sizeof cd.light);
                double sign = cull == 2 ? -1.0 : 1.0;
                for (int r = 0; r < 3; ++r) {
                    cd.light.position[r] = w[0][r];
                    cd.light.color[r] = emission[r];
                    cd.light.direction[r] = (float)(cr[r] / len * sign);
                    cd.light.edge1[r] = (float)e1[r];
                    cd.light.edge2[r] = (float)e2[r];
                }
                cd.light.position[3] = cull == 0 ? -2.0f : -1.0f;
                cd.light.color[3] = (float)area;
                cd.light.source[0] = slot;
                cd.light.source[1] = t;
                cd.power = power;
                cands.push_back(cd);
            }
        }
        const uint32_t kSteps = 1u << 24;
        if (cands.size() > kSteps) {
            delete P;
            return LUX_ERR_INVALID_ARGUMENT;
        }
        double total = 0.0;
        for (const Cand &c : cands) total += c.power;
        double cumulative = 0.0;
        uint32_t previous = 0;
        for (size_t k = 0; k < cands.size(); ++k) {
            cumulative += cands[k].power;
            uint32_t boundary;
            if (k + 1 == cands.size()) {
                boundary = kSteps;
            } else {
                double ideal = std::round(cumulative / total * (double)kSteps);
                uint32_t ideal_u = ideal <= 0.0 ? 0u : (ideal >= 4294967295.0 ? 0xffffffffu : (uint32_t)ideal);
                uint32_t max_boundary = kSteps - (uint32_t)(cands.size() - k - 1);
                boundary = std::min(std::max(ideal_u, previous + 1u), max_boundary);
            }
            cands[k].light.direction[3] = (float)boundary / (float)kSteps;
            cands[k].light.edge1[3] = (float)(boundary - previous) / (float)kSteps;
            previous = boundary;
            P->lights.push_back(cands[k].light);
        }
    } catch (const std::bad_alloc &) {
        delete P;
        return LUX_ERR_OUT_OF_MEMORY;
    }
    *out = P;
    return LUX_OK;
}

extern "C" lux_status lux_packed_scene_sizes(const LuxPackedScene *p, size_t *scene_words, size_t *geometry_words,
                                             size_t *lights, uint32_t *tlas_nodes, uint32_t *blas_nodes) {
    if (!p) return LUX_ERR_INVALID_ARGUMENT;
    if (scene_words) *scene_words = p->scene_words.size() / 4;
    if (geometry_words) *geometry_words = p->geometry_words.size() / 4;
    if (lights) *lights = p->lights.size();
    if (tlas_nodes) *tlas_nodes = p->tlas_nodes;
    if (blas_nodes) *blas_nodes = p->blas_nodes;
    return LUX_OK;
}

extern "C" lux_status lux_packed_scene_copy(const LuxPackedScene *p, uint32_t *scene_words, uint32_t *geometry_words,
                                            LuxLight *lights) {
    if (!p) return LUX_ERR_INVALID_ARGUMENT;
    if (scene_words) std::memcpy(scene_words, p->scene_words.data(), p->scene_words.size() * 4);
    if (geometry_words) std::memcpy(geometry_words, p->geometry_words.data(), p->geometry_words.size() * 4);
    if (lights && !p->lights.empty()) std::memcpy(lights, p->lights.data(), p->lights.size() * sizeof(LuxLight));
    return LUX_OK;
}

extern "C" lux_status lux_packed_scene_instance_order(const LuxPackedScene *p, uint32_t *order) {
    if (!p || !order) return LUX_ERR_INVALID_ARGUMENT;
    if (!p->instance_order.empty())
        std::memcpy(order, p->instance_order.data(), p->instance_order.size() * 4);
    return LUX_OK;
}

extern "C" lux_status lux_packed_scene_quality(const LuxPackedScene *p, double *blas_cost, uint32_t *max_depth) {
    if (!p) return LUX_ERR_INVALID_ARGUMENT;
    if (blas_cost) *blas_cost = p->blas_cost;
    if (max_depth) *max_depth = p->max_depth;
    return LUX_OK;
}

extern "C" void lux_packed_scene_destroy(LuxPackedScene *p) { delete p; }

bool lux_affine_inverse(const float m[12], float out[12]) {
    double w[3][4];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) w[r][c] = m[4 * r + c];
    double a = w[0][0], b = w[0][1], c = w[0][2], d = w[1][0], e = w[1][1], f = w[1][2], g = w[2][0], h = w[2][1],
           k = w[2][2];
    double det = a * (e * k - f * h) - b * (d * k - f * g) + c * (d * h - e * g);
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
    double inv[3][3] = {{(e * k - f * h) / det, (c * h - b * k) / det, (b * f - c * e) / det},
                        {(f * g - d * k) / det, (a * k - c * g) / det, (c * d - a * f) / det},
                        {(d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det}};
    for (int r = 0; r < 3; ++r) {
        double t = -(inv[r][0] * w[0][3] + inv[r][1] * w[1][3] + inv[r][2] * w[2][3]);
        for (int cc = 0; cc < 3; ++cc) out[4 * r + cc] = (float)inv[r][cc];
        out[4 * r + 3] = (float)t;
    }
    return true;
}

// Emissive light records of a rigidly moved scene (build_emissive_lights,
// src/scene.rs:2311-2372, at new instance poses): each record's triangle
// (source.y, packed order) is re-transformed by its instance's new
// world_from_local (source.x, slot order) with the packer's arithmetic;
// position, edges and the facing normal change, while the area, power and
// CDF fields stay those of the given records (rigid motion keeps areas).
extern "C" lux_status lux_emissive_lights_at(const uint32_t *gw, size_t gn, const LuxLight *lights,
                                             uint32_t light_count, const float *world_from_local,
                                             uint32_t instance_count, LuxLight *out) {
    if ((light_count && (!lights || !out)) || !gw || gn < 1 || (instance_count && !world_from_local))
        return LUX_ERR_INVALID_ARGUMENT;
    uint32_t vertex_base = gw[1], vertex_stride = gw[2], vertex_count = gw[3];
    if (gw[0] != 1u || vertex_stride != 5u || (uint64_t)vertex_base + (uint64_t)vertex_count * 5u > gn)
        return LUX_ERR_MALFORMED_SCENE;
    for (uint32_t k = 0; k < light_count; ++k) {
        const LuxLight &L = lights[k];
        uint32_t slot = L.source[0], t = L.source[1];
        if (slot >= instance_count || 1u + (uint64_t)t >= vertex_base) return LUX_ERR_MALFORMED_SCENE;
        const float *m = world_from_local + 12 * (size_t)slot;
        double w64[3][4];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) w64[r][c] = m[4 * r + c];
        const uint32_t *idx = gw + 4 * (size_t)(1 + t);
        float w[3][3];
        for (int v = 0; v < 3; ++v) {
            if (idx[v] >= vertex_count) return LUX_ERR_MALFORMED_SCENE;
            const uint32_t *pw = gw + 4 * ((size_t)vertex_base + (size_t)idx[v] * 5u);
            float p[3];
            std::memcpy(p, pw, 12);
            for (int r = 0; r < 3; ++r)
                w[v][r] = (float)(w64[r][0] * p[0] + w64[r][1] * p[1] + w64[r][2] * p[2] + w64[r][3]);
        }
        double e1[3], e2[3];
        for (int r = 0; r < 3; ++r) {
            e1[r] = (double)w[1][r] - w[0][r];
            e2[r] = (double)w[2][r] - w[0][r];
        }
        double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        LuxLight o = L;
        // The facing sign the packer chose: the old normal's orientation
        // relative to the old edges' cross product.
        double old_cr[3] = {(double)L.edge1[1] * L.edge2[2] - (double)L.edge1[2] * L.edge2[1],
                            (double)L.edge1[2] * L.edge2[0] - (double)L.edge1[0] * L.edge2[2],
                            (double)L.edge1[0] * L.edge2[1] - (double)L.edge1[1] * L.edge2[0]};
        double sign = old_cr[0] * L.direction[0] + old_cr[1] * L.direction[1] + old_cr[2] * L.direction[2] < 0.0
                          ? -1.0
                          : 1.0;
        for (int r = 0; r < 3; ++r) {
            o.position[r] = w[0][r];
            o.direction[r] = len > 0.0 ? (float)(cr[r] / len * sign) : L.direction[r];
            o.edge1[r] = (float)e1[r];
            o.edge2[r] = (float)e2[r];
        }
        out[k] = o;
    }
    return LUX_OK;
}
