// Compressed 8-wide BVH builder.
//
// The reference hands its triangles to OptiX (Geometry::build_accel,
// src/base/mgr/geometry.cpp:36-52); B200 has no RT-core path here, so the
// acceleration structure is built on the host: a binned-SAH binary BVH with
// leaves of at most one to three triangles (by tree size) is collapsed into
// 8-wide nodes whose child boxes are quantised to 8 bits per plane against a
// per-node power-of-two grid (80-byte nodes, after Ylitie, Karras and Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs",
// HPG 2017).  Each wide node's children are chosen by that paper's
// SAH-optimal dynamic programme (the default) or greedily (open the largest
// internal child until there are eight).  Child slots are ordered by
// direction so that traversal visits children roughly front to back by
// flipping slot bits with the ray octant.
#include "vs_host.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <thread>

namespace vs {

namespace {

struct Box {
    f3 lo{FLT_MAX, FLT_MAX, FLT_MAX};
    f3 hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(f3 p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void grow(const Box &b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    float area() const {
        f3 d = hi - lo;
        if (d.x < 0) return 0.0f;
        return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
    f3 center() const { return (lo + hi) * 0.5f; }
};

struct Node2 {
    Box box;
    uint32_t left = 0, right = 0;  // children (internal) or first/count (leaf)
    uint32_t first = 0, count = 0;
    bool leaf = false;
};

constexpr int kBins = 32;
// Most primitives a leaf child may hold (the node format's limit; scenes
// choose 1 to 3, default 1).
constexpr uint32_t kMaxLeaf = 3;

// Subtrees at least this large are built on their own thread (down to
// kParallelDepth levels): the binary build is the bulk of the host work, and
// the two halves of a split touch disjoint ranges of `order`.
constexpr uint32_t kParallelPrims = 1u << 15;
constexpr uint32_t kParallelDepth = 5;

struct Builder2 {
    const std::vector<Box> &boxes;
    const std::vector<f3> &cent;
    std::vector<uint32_t> &order;
    uint32_t max_leaf;                 // subtrees of at most this many primitives are leaves
    std::vector<Node2> nodes;          // sized 2 n up front; ids handed out by `next`
    std::atomic<uint32_t> next{0};

    uint32_t build(uint32_t first, uint32_t count, uint32_t depth = 0) {
        uint32_t id = next.fetch_add(1);
        Box bb, cb;
        for (uint32_t i = first; i < first + count; ++i) {
            bb.grow(boxes[order[i]]);
            cb.grow(cent[order[i]]);
        }
        nodes[id].box = bb;
        if (count <= max_leaf) {
            nodes[id].leaf = true;
            nodes[id].first = first;
            nodes[id].count = count;
            return id;
        }
        // Binned SAH over centroids.  The bins of a large node are filled by
        // several threads over chunks of its range and merged (min / max and
        // counts: the same bins in any order).
        int best_axis = -1, best_split = -1;
        float best_cost = FLT_MAX;
        Box all_bins[3][kBins];
        uint32_t all_cnt[3][kBins] = {};
        auto fill = [&](uint32_t b0, uint32_t b1, Box (*bb)[kBins], uint32_t (*bc)[kBins]) {
            for (int axis = 0; axis < 3; ++axis) {
                float lo = comp(cb.lo, axis), hi = comp(cb.hi, axis);
                if (!(hi > lo)) continue;
                float k = kBins / (hi - lo);
                for (uint32_t i = b0; i < b1; ++i) {
                    int b = std::min(kBins - 1, static_cast<int>((comp(cent[order[i]], axis) - lo) * k));
                    bc[axis][b]++;
                    bb[axis][b].grow(boxes[order[i]]);
                }
            }
        };
        const uint32_t chunks = count >= (1u << 17) ? 8u : 1u;
        if (chunks == 1) {
            fill(first, first + count, all_bins, all_cnt);
        } else {
            std::vector<std::array<std::array<Box, kBins>, 3>> cbox(chunks);
            std::vector<std::array<std::array<uint32_t, kBins>, 3>> ccnt(chunks);
            std::vector<std::thread> th;
            for (uint32_t c = 0; c < chunks; ++c) {
                for (auto &a : ccnt[c]) a.fill(0u);
                th.emplace_back([&, c] {
                    const uint32_t b0 = first + static_cast<uint32_t>(static_cast<uint64_t>(count) * c / chunks);
                    const uint32_t b1 = first + static_cast<uint32_t>(static_cast<uint64_t>(count) * (c + 1) / chunks);
                    Box lb[3][kBins];
                    uint32_t lc[3][kBins] = {};
                    fill(b0, b1, lb, lc);
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < kBins; ++b) {
                            cbox[c][a][b] = lb[a][b];
                            ccnt[c][a][b] = lc[a][b];
                        }
                });
            }
            for (auto &t : th) t.join();
            for (uint32_t c = 0; c < chunks; ++c)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < kBins; ++b) {
                        all_bins[a][b].grow(cbox[c][a][b]);
                        all_cnt[a][b] += ccnt[c][a][b];
                    }
        }
        for (int axis = 0; axis < 3; ++axis) {
            float lo = comp(cb.lo, axis), hi = comp(cb.hi, axis);
            if (!(hi > lo)) continue;
            const Box *bin_box = all_bins[axis];
            const uint32_t *bin_cnt = all_cnt[axis];
            float right_area[kBins];
            uint32_t right_cnt[kBins];
            Box acc;
            uint32_t c = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bin_box[b]);
                c += bin_cnt[b];
                right_area[b] = acc.area();
                right_cnt[b] = c;
            }
            Box lacc;
            uint32_t lc = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                lacc.grow(bin_box[b]);
                lc += bin_cnt[b];
                if (lc == 0 || right_cnt[b + 1] == 0) continue;
                float cost = lacc.area() * lc + right_area[b + 1] * right_cnt[b + 1];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_split = b;
                }
            }
        }
        uint32_t mid;
        if (best_axis < 0) {
            mid = first + count / 2;  // all centroids coincide: split in the middle
        } else {
            float lo = comp(cb.lo, best_axis), hi = comp(cb.hi, best_axis);
            float k = kBins / (hi - lo);
            auto it = std::partition(order.begin() + first, order.begin() + first + count, [&](uint32_t p) {
                int b = std::min(kBins - 1, static_cast<int>((comp(cent[p], best_axis) - lo) * k));
                return b <= best_split;
            });
            mid = static_cast<uint32_t>(it - order.begin());
            if (mid == first || mid == first + count) mid = first + count / 2;
        }
        uint32_t l = 0, r = 0;
        if (count >= kParallelPrims && depth < kParallelDepth) {
            std::thread left([&] { l = build(first, mid - first, depth + 1); });
            r = build(mid, first + count - mid, depth + 1);
            left.join();
        } else {
            l = build(first, mid - first, depth + 1);
            r = build(mid, first + count - mid, depth + 1);
        }
        nodes[id].left = l;
        nodes[id].right = r;
        return id;
    }
};

struct Collapse {
    const std::vector<Node2> &n2;
    const std::vector<uint32_t> &order;
    // Writes the leaf entry of primitive `prim` (a triangle's 12 floats, or a
    // top-level leaf's instance id) and returns nothing; leaf_base() is the
    // index the next entry will get.
    std::function<void(uint32_t)> emit;
    std::function<uint32_t()> leaf_base;
    std::vector<Bvh8Node> &out;
    std::vector<uint32_t> subtree_count;
    uint32_t max_leaf = kMaxLeaf;
    uint32_t max_depth = 0;

    uint32_t count_tris(uint32_t id) {
        const Node2 &n = n2[id];
        uint32_t c = n.leaf ? n.count : count_tris(n.left) + count_tris(n.right);
        subtree_count[id] = c;
        return c;
    }

    void gather(uint32_t id, std::vector<uint32_t> &prims) const {
        const Node2 &n = n2[id];
        if (n.leaf) {
            for (uint32_t i = 0; i < n.count; ++i) prims.push_back(order[n.first + i]);
        } else {
            gather(n.left, prims);
            gather(n.right, prims);
        }
    }

    // SAH-optimal collapse (Ylitie, Karras and Laine 2017, section 3.1):
    // cost[n][i - 1] is the least SAH cost of binary subtree n spread over at
    // most i child slots of a wide node: n itself as one child (a leaf of at
    // most max_leaf triangles, or a wide node whose 8 slots are shared by
    // n's two subtrees), or i slots shared by its two subtrees.  split[n][i - 1]
    // is the left subtree's share (0: n as one child); as_leaf[n] says which
    // one-child form won; split8[n] shares the 8 slots of n as a wide node.
    static constexpr float kCostNode = 1.0f, kCostPrim = 0.3f;
    std::vector<std::array<float, 8>> cost;
    std::vector<std::array<uint8_t, 8>> split;
    std::vector<uint8_t> as_leaf, split8;

    void optimise() {
        const size_t m = n2.size();
        cost.assign(m, {});
        split.assign(m, {});
        as_leaf.assign(m, 0);
        split8.assign(m, 0);
        // Children get larger ids than their parent (ids are handed out on
        // entry to the binary build), so a reverse sweep sees them first.
        for (size_t id = m; id-- > 0;) {
            const Node2 &n = n2[id];
            const float area = n.box.area();
            const uint32_t cnt = subtree_count[id];
            const float c_leaf = cnt <= max_leaf ? area * kCostPrim * static_cast<float>(cnt) : FLT_MAX;
            if (n.leaf) {
                as_leaf[id] = 1;
                for (int i = 0; i < 8; ++i) cost[id][i] = c_leaf;
                continue;
            }
            const std::array<float, 8> &L = cost[n.left], &R = cost[n.right];
            // The best sharing of i slots between the two subtrees.
            auto share = [&](int i, int &best_k) {
                float best = FLT_MAX;
                best_k = 0;
                for (int k = 1; k < i; ++k) {
                    const float c = L[k - 1] + R[i - k - 1];
                    if (c < best) {
                        best = c;
                        best_k = k;
                    }
                }
                return best;
            };
            int k8 = 0;
            const float s8 = share(8, k8);
            split8[id] = static_cast<uint8_t>(k8);
            const float c_node = s8 < FLT_MAX ? area * kCostNode + s8 : FLT_MAX;
            as_leaf[id] = c_leaf <= c_node ? 1 : 0;
            const float c_one = std::min(c_leaf, c_node);
            cost[id][0] = c_one;
            split[id][0] = 0;
            for (int i = 2; i <= 8; ++i) {
                int k = 0;
                const float c = share(i, k);
                if (c < c_one) {
                    cost[id][i - 1] = c;
                    split[id][i - 1] = static_cast<uint8_t>(k);
                } else {
                    cost[id][i - 1] = c_one;
                    split[id][i - 1] = 0;
                }
            }
        }
    }

    // The children (binary node ids) that subtree n contributes to a wide
    // node when given at most i slots.
    void collect(uint32_t id, int i, std::vector<uint32_t> &ch) const {
        const int k = split[id][i - 1];
        if (k == 0) {
            ch.push_back(id);
            return;
        }
        collect(n2[id].left, k, ch);
        collect(n2[id].right, i - k, ch);
    }

    bool optimal = false;  // SAH-optimal children instead of the greedy expansion
    bool is_leaf_child(uint32_t id) const {
        return optimal ? as_leaf[id] != 0 : (n2[id].leaf || subtree_count[id] <= max_leaf);
    }

    // Writes node `slot_index` of `out` for binary node `id` and recurses.
    void build(uint32_t id, uint32_t out_index, uint32_t depth) {
        max_depth = std::max(max_depth, depth);
        std::vector<uint32_t> ch;
        if (is_leaf_child(id)) {
            ch.push_back(id);  // a tree of at most max_leaf primitives: one leaf child
        } else if (optimal) {
            const int k = split8[id];
            collect(n2[id].left, k, ch);
            collect(n2[id].right, 8 - k, ch);
        } else {
            ch.push_back(n2[id].left);
            ch.push_back(n2[id].right);
            while (ch.size() < 8) {
                int best = -1;
                float best_area = -1.0f;
                for (size_t i = 0; i < ch.size(); ++i) {
                    if (is_leaf_child(ch[i])) continue;
                    float a = n2[ch[i]].box.area();
                    if (a > best_area) {
                        best_area = a;
                        best = static_cast<int>(i);
                    }
                }
                if (best < 0) break;
                uint32_t c = ch[best];
                ch[best] = n2[c].left;
                ch.push_back(n2[c].right);
            }
        }
        // Assign children to slots: slot s prefers children lying toward the
        // corner whose coordinate signs are the bits of s (bit set = +).
        Box nb;
        for (uint32_t c : ch) nb.grow(n2[c].box);
        f3 nc = nb.center();
        int slot_of[8];
        bool used_slot[8] = {false};
        bool done[8] = {false};
        for (size_t step = 0; step < ch.size(); ++step) {
            float best_cost = FLT_MAX;
            int bc = -1, bs = -1;
            for (size_t i = 0; i < ch.size(); ++i) {
                if (done[i]) continue;
                f3 d = n2[ch[i]].box.center() - nc;
                for (int sl = 0; sl < 8; ++sl) {
                    if (used_slot[sl]) continue;
                    f3 dir = {(sl & 1) ? 1.0f : -1.0f, (sl & 2) ? 1.0f : -1.0f, (sl & 4) ? 1.0f : -1.0f};
                    float cost = -dot(d, dir);
                    if (cost < best_cost) {
                        best_cost = cost;
                        bc = static_cast<int>(i);
                        bs = sl;
                    }
                }
            }
            done[bc] = true;
            used_slot[bs] = true;
            slot_of[bc] = bs;
        }
        int child_at[8];
        for (int sl = 0; sl < 8; ++sl) child_at[sl] = -1;
        for (size_t i = 0; i < ch.size(); ++i) child_at[slot_of[i]] = static_cast<int>(i);

        Bvh8Node node;
        std::memset(&node, 0, sizeof(node));
        node.px = nb.lo.x;
        node.py = nb.lo.y;
        node.pz = nb.lo.z;
        // Per-axis grid step 2^e with 255 steps covering the node box.
        float step[3];
        for (int a = 0; a < 3; ++a) {
            float ext = comp(nb.hi, a) - comp(nb.lo, a);
            int e = -100;
            if (ext > 0.0f) e = static_cast<int>(std::ceil(std::log2(ext / 255.0f)));
            e = std::max(e, -120);
            while (true) {
                float s = std::ldexp(1.0f, e);
                float lo = comp(nb.lo, a);
                // The top of the grid must reach the node's upper bound.
                if (lo + 255.0f * s >= comp(nb.hi, a)) break;
                ++e;
            }
            node.e[a] = static_cast<uint8_t>(e + 127);
            step[a] = std::ldexp(1.0f, e);
        }
        float p[3] = {node.px, node.py, node.pz};
        uint32_t internal_count = 0;
        for (int sl = 0; sl < 8; ++sl)
            if (child_at[sl] >= 0 && !is_leaf_child(ch[child_at[sl]])) internal_count++;
        node.base_child = static_cast<uint32_t>(out.size());
        node.base_tri = leaf_base();
        out.resize(out.size() + internal_count);
        uint32_t tri_offset = 0;
        std::vector<std::pair<uint32_t, uint32_t>> recurse;  // (binary id, out index)
        uint32_t next_internal = node.base_child;
        for (int sl = 0; sl < 8; ++sl) {
            if (child_at[sl] < 0) continue;
            uint32_t c = ch[child_at[sl]];
            const Box &cb = n2[c].box;
            for (int a = 0; a < 3; ++a) {
                float s = step[a];
                float lo = comp(cb.lo, a), hi = comp(cb.hi, a);
                int ql = static_cast<int>(std::floor((lo - p[a]) / s));
                int qh = static_cast<int>(std::ceil((hi - p[a]) / s));
                ql = std::min(std::max(ql, 0), 255);
                qh = std::min(std::max(qh, 0), 255);
                // Conservative with the exact float ops the traversal uses.
                while (ql > 0 && p[a] + static_cast<float>(ql) * s > lo) --ql;
                while (qh < 255 && p[a] + static_cast<float>(qh) * s < hi) ++qh;
                if (p[a] + static_cast<float>(ql) * s > lo || p[a] + static_cast<float>(qh) * s < hi)
                    throw std::runtime_error("bvh8: quantisation cannot bound a child box");
                node.qlo[a][sl] = static_cast<uint8_t>(ql);
                node.qhi[a][sl] = static_cast<uint8_t>(qh);
            }
            if (is_leaf_child(c)) {
                std::vector<uint32_t> prims;
                gather(c, prims);
                if (prims.size() > max_leaf || tri_offset + prims.size() > 24)
                    throw std::runtime_error("bvh8: leaf too large");
                node.meta[sl] = static_cast<uint8_t>((((1u << prims.size()) - 1u) << 5) | tri_offset);
                for (uint32_t pr : prims) emit(pr);
                tri_offset += static_cast<uint32_t>(prims.size());
            } else {
                node.imask |= static_cast<uint8_t>(1u << sl);
                node.meta[sl] = static_cast<uint8_t>(0x20u | (24u + sl));
                recurse.push_back({c, next_internal++});
            }
        }
        out[out_index] = node;
        for (auto &r : recurse) build(r.first, r.second, depth + 1);
    }
};

}  // namespace

namespace {

// Binned-SAH binary tree over `n` primitive boxes, collapsed into BVH8 nodes
// appended to `out` (root at the returned index); leaf entries written by
// `emit` (see Collapse).  Returns the depth of the collapsed tree.
uint32_t build_tree(bool optimal, uint32_t max_leaf, const std::vector<Box> &boxes, std::vector<Bvh8Node> &out, uint32_t &root,
                    const std::function<void(uint32_t)> &emit, const std::function<uint32_t()> &leaf_base) {
    const uint32_t n = static_cast<uint32_t>(boxes.size());
    std::vector<f3> cent(n);
    for (uint32_t i = 0; i < n; ++i) cent[i] = boxes[i].center();
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    // Leaf size 0 picks by tree size: single-primitive leaves for trees of
    // 4096 primitives or more (fewer, less divergent triangle tests per ray:
    // +11 % on the 2.3 M-triangle scene, +16 % on the many-light frame),
    // three for smaller ones (whose few nodes stay in L1: the 36-triangle
    // room traces 4.5 % faster with three).
    if (max_leaf == 0) max_leaf = boxes.size() >= 4096 ? 1u : kMaxLeaf;
    if (max_leaf > kMaxLeaf) throw std::runtime_error("bvh8: leaf size outside 1..3");
    Builder2 b2{boxes, cent, order, max_leaf, {}};
    b2.nodes.resize(2 * static_cast<size_t>(n));
    b2.build(0, n);
    b2.nodes.resize(b2.next.load());
    Collapse col{b2.nodes, order, emit, leaf_base, out, std::vector<uint32_t>(b2.nodes.size(), 0)};
    col.count_tris(0);
    col.max_leaf = max_leaf;
    col.optimal = optimal;
    if (optimal) col.optimise();
    root = static_cast<uint32_t>(out.size());
    out.resize(out.size() + 1);
    col.build(0, root, 1);
    if (col.max_depth + 1 > 32) throw std::runtime_error("bvh8: tree deeper than the traversal stack");
    return col.max_depth;
}

std::vector<Box> triangle_boxes(const f3 *pos, const uint32_t *idx, uint32_t n) {
    std::vector<Box> boxes(n);
    const uint32_t nt = n >= (1u << 17) ? 8u : 1u;
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (uint32_t i = static_cast<uint32_t>(static_cast<uint64_t>(n) * t / nt);
                 i < static_cast<uint32_t>(static_cast<uint64_t>(n) * (t + 1) / nt); ++i) {
                Box b;
                for (int k = 0; k < 3; ++k) b.grow(pos[idx[3 * i + k]]);
                boxes[i] = b;
            }
        });
    for (auto &x : th) x.join();
    return boxes;
}

}  // namespace

void build_bvh8(HostScene &s) {
    const uint32_t n = static_cast<uint32_t>(s.prim_inst.size());
    s.nodes.clear();
    s.tri_v.clear();
    s.tlas_inst.clear();
    s.blas_root.clear();
    // Two levels when meshes are shared: always (instancing 2), or (1, auto)
    // when the scene is large (2^20 triangles or more) and its instances hold
    // at least 8 times the distinct meshes' triangles, where the smaller
    // structure and build pay for the extra level; otherwise one BVH8 over
    // world space traces faster.
    std::vector<uint32_t> uses(s.meshes.size(), 0);
    for (uint32_t m : s.inst_mesh) uses[m]++;
    uint64_t unique_tris = 0;
    for (const HostScene::MeshRec &r : s.meshes) unique_tris += r.tri_count;
    const bool shared = std::any_of(uses.begin(), uses.end(), [](uint32_t u) { return u > 1; });
    // The real-time ReSTIR kernels trace one world-space BVH8.
    s.two_level = !s.rt && s.inst_mesh.size() == s.instances.size() && shared &&
                  (s.instancing == 2 ||
                   (s.instancing == 1 && n >= (1u << 20) && static_cast<uint64_t>(n) >= 8 * unique_tris));
    if (!s.two_level) {
        // One BVH8 over the world-space triangles; tri_v w = global primitive id.
        std::vector<Box> boxes = triangle_boxes(s.pos.data(), s.idx.data(), n);
        s.tri_v.reserve(static_cast<size_t>(n) * 12);
        auto emit = [&](uint32_t prim) {
            for (int k = 0; k < 3; ++k) {
                f3 p = s.pos[s.idx[3 * prim + k]];
                s.tri_v.push_back(p.x);
                s.tri_v.push_back(p.y);
                s.tri_v.push_back(p.z);
                s.tri_v.push_back(k == 0 ? bits_float(prim) : 0.0f);
            }
        };
        uint32_t root = 0;
        s.bvh_depth = build_tree(s.bvh_sah_collapse, s.bvh_leaf_size, boxes, s.nodes, root, emit, [&] { return static_cast<uint32_t>(s.tri_v.size() / 12); });
        if (s.tri_v.size() != static_cast<size_t>(n) * 12) throw std::runtime_error("bvh8: primitive count mismatch");
        s.tlas_root = 0;
        return;
    }
    // Bottom level: one BVH8 per mesh over its object-space triangles
    // (tri_v w = the triangle's index in the mesh).  The top level's root goes
    // first so that node 0 bounds the whole scene.
    s.nodes.resize(1);
    uint32_t depth = 0;
    for (uint32_t m = 0; m < s.meshes.size(); ++m) {
        const HostScene::MeshRec &r = s.meshes[m];
        std::vector<Box> boxes = triangle_boxes(s.mesh_pos.data() + r.first_vertex, s.mesh_idx.data() + 3u * r.first_tri,
                                                r.tri_count);
        const f3 *mp = s.mesh_pos.data() + r.first_vertex;
        const uint32_t *mi = s.mesh_idx.data() + 3u * r.first_tri;
        auto emit = [&](uint32_t tri) {
            for (int k = 0; k < 3; ++k) {
                f3 p = mp[mi[3 * tri + k]];
                s.tri_v.push_back(p.x);
                s.tri_v.push_back(p.y);
                s.tri_v.push_back(p.z);
                s.tri_v.push_back(k == 0 ? bits_float(tri) : 0.0f);
            }
        };
        uint32_t root = 0;
        depth = std::max(depth, build_tree(s.bvh_sah_collapse, s.bvh_leaf_size, boxes, s.nodes, root, emit,
                                           [&] { return static_cast<uint32_t>(s.tri_v.size() / 12); }));
        s.blas_root.push_back(root);
    }
    // Top level over the instances' world boxes (the bounds of their
    // world-space vertices); leaf entries are instance ids.
    std::vector<Box> iboxes(s.instances.size());
    for (uint32_t i = 0; i < s.instances.size(); ++i) {
        const uint32_t first = s.instances[i].first_prim;
        Box wb;
        for (uint32_t t = 0; t < s.instances[i].prim_count; ++t)
            for (int k = 0; k < 3; ++k) wb.grow(s.pos[s.idx[3 * (first + t) + k]]);
        iboxes[i] = wb;
    }
    std::vector<Bvh8Node> top;
    uint32_t troot = 0;
    auto emit_inst = [&](uint32_t inst) { s.tlas_inst.push_back(inst); };
    depth = std::max(depth, build_tree(s.bvh_sah_collapse, s.bvh_leaf_size, iboxes, top, troot, emit_inst,
                                       [&] { return static_cast<uint32_t>(s.tlas_inst.size()); }));
    // Append the top level after the meshes, its root at node 0: child
    // indices of the top level move by the offset of its other nodes.
    const uint32_t off = static_cast<uint32_t>(s.nodes.size()) - 1u;
    for (size_t k = 0; k < top.size(); ++k) {
        Bvh8Node nd = top[k];
        if (nd.imask) nd.base_child += off;  // children of a node always follow the root
        if (k == troot) s.nodes[0] = nd;
        else s.nodes.push_back(nd);
    }
    s.tlas_root = 0;
    s.bvh_depth = depth;
}

}  // namespace vs
