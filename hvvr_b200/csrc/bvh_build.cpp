// bvh_build.cpp - hvvr_generate_topology: host BVH build for MeshData.
//
// Triangle IDs everywhere on the path are BVH-order IDs, so a drop-in must produce the
// same topology and the same triangle/vertex order as the reference's GenerateTopology
// (libraries/hvvr/shared/bvh.cpp:542-556). The steps are therefore the reference's:
//   1. top-down SAH binary BVH over triangle boxes with full sorts on the centroid sum
//      lower+upper per axis and the cost/termination rule of helpBuildBVH2 (bvh.cpp:167-249);
//   2. collapse to 4-wide nodes, evicting the 1-2 children that minimise the kept box's
//      surface area, leaves first then by surface area (helpBuildBVH4, bvh.cpp:343-467);
//   3. depth-first topology with leaf triangle ranges and relative child offsets, then the
//      vertex reorder in reverse triangle order (TopologyBuilder, bvh.cpp:474-540).
// The implementation is different: sort keys are precomputed per axis (the comparisons see
// the same float sums, so std::sort makes the same decisions on the same sequences), large
// subtrees are built in parallel into private node buffers and spliced in (BVH2 offsets are
// relative, so a subtree block can move), and the BVH4 cache uses node indices.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <future>
#include <vector>

#include "../../include/hvvr_c.h"

namespace {

struct Box {
    float lo[3], hi[3];
};
inline float fminr(float a, float b) { return a < b ? a : b; }
inline float fmaxr(float a, float b) { return a > b ? a : b; }
inline Box boxEmpty() { return Box{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
inline Box unite(const Box& a, const Box& b) {
    Box r;
    for (int i = 0; i < 3; i++) {
        r.lo[i] = fminr(a.lo[i], b.lo[i]);
        r.hi[i] = fmaxr(a.hi[i], b.hi[i]);
    }
    return r;
}
inline float area(const Box& b) {
    const float ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    return ex * (ey + ez) + ey * ez;
}

struct Node2 {
    Box box[2];
    uint32_t offset[2]; // relative node offset, 0 = leaf range
    uint32_t size[2];   // triangles below the child
};

struct Builder {
    const std::vector<Box>* leaf;
    std::vector<float> key[3]; // lo + hi per axis

    void sortAxis(uint32_t* idx, size_t n, int axis) const {
        const float* k = key[axis].data();
        std::sort(idx, idx + n, [k](uint32_t a, uint32_t b) { return k[a] < k[b]; });
    }

    bool scanAxis(size_t& bestIndex, float& bestCost, float* temp, uint32_t* idx, size_t n, int axis) const {
        sortAxis(idx, n, axis);
        Box b = boxEmpty();
        for (size_t i = 1; i < n; i++) {
            b = unite(b, (*leaf)[idx[n - i]]);
            temp[n - i] = area(b) * float(i);
        }
        bool better = false;
        b = boxEmpty();
        for (size_t i = 1; i < n; i++) {
            b = unite(b, (*leaf)[idx[i - 1]]);
            const float cost = temp[i] + area(b) * float(i);
            if (bestCost > cost) {
                bestCost = cost;
                bestIndex = i;
                better = true;
            }
        }
        return better;
    }

    Box rangeBox(const uint32_t* idx, size_t n) const {
        Box b = (*leaf)[idx[0]];
        for (size_t i = 1; i < n; i++) b = unite(b, (*leaf)[idx[i]]);
        return b;
    }

    // builds the subtree for idx[0..n) at nodes[0..); returns the node count or 0 for a leaf range
    size_t build(Node2* nodes, float* temp, uint32_t* idx, size_t n, int parallelDepth) const {
        if (n < 2) return 0;
        int axis = 0;
        size_t index = 0;
        float cost = INFINITY;
        scanAxis(index, cost, temp, idx, n, 0);
        if (scanAxis(index, cost, temp, idx, n, 1)) axis = 1;
        if (scanAxis(index, cost, temp, idx, n, 2)) axis = 2;
        sortAxis(idx, n, axis);
        Node2& node = nodes[0];
        size_t offset = 1;
        size_t countL = 0, countR = 0;
        std::vector<Node2> rightNodes;
        const bool par = parallelDepth > 0 && n > (1u << 15);
        if (par) {
            // right subtree into a private buffer, spliced in after the left subtree's size is known
            rightNodes.resize(std::max<size_t>(n - index, 1));
            auto fut = std::async(std::launch::async, [&]() {
                return build(rightNodes.data(), temp + index, idx + index, n - index, parallelDepth - 1);
            });
            countL = build(nodes + offset, temp, idx, index, parallelDepth - 1);
            countR = fut.get();
        } else {
            countL = build(nodes + offset, temp, idx, index, 0);
        }
        if (countL) {
            node.box[0] = unite(nodes[offset].box[0], nodes[offset].box[1]);
            node.offset[0] = uint32_t(offset);
            offset += countL;
        } else {
            node.box[0] = rangeBox(idx, index);
            node.offset[0] = 0;
        }
        node.size[0] = uint32_t(index);
        if (par) {
            if (countR) memcpy(nodes + offset, rightNodes.data(), countR * sizeof(Node2));
        } else {
            countR = build(nodes + offset, temp + index, idx + index, n - index, 0);
        }
        if (countR) {
            node.box[1] = unite(nodes[offset].box[0], nodes[offset].box[1]);
            node.offset[1] = uint32_t(offset);
            offset += countR;
        } else {
            node.box[1] = rangeBox(idx + index, n - index);
            node.offset[1] = 0;
        }
        node.size[1] = uint32_t(n - index);
        const float mult = 2.0f; // a node test costs two triangle tests
        return area(unite(node.box[0], node.box[1])) * (float(n) - mult) < cost ? 0 : offset;
    }
};

// one 4-wide slot; ofs encodes (absolute node index + 1) while pending, then the relative offset
struct Slot {
    Box box;
    uint32_t first, bound, ofs, depth;
};
struct Node4 {
    Slot s[4];
};

bool slotOrder(const Slot& a, const Slot& b) {
    return (a.ofs == 0 && b.ofs != 0) || ((a.ofs == 0 || b.ofs != 0) && area(a.box) > area(b.box));
}

struct Collapser {
    const std::vector<Node2>& n2;
    std::vector<Node4>& out;
    size_t next; // allocation cursor, counts down

    uint32_t visit(size_t ni, Slot* parentCache, uint32_t first) {
        const Node2& node = n2[ni];
        Slot cache[6];
        uint32_t cs = 0;
        if (node.offset[0]) cs += visit(ni + node.offset[0], cache + cs, first);
        else cache[cs++] = Slot{node.box[0], first, first + node.size[0], 0, 0};
        if (node.offset[1]) cs += visit(ni + node.offset[1], cache + cs, first + node.size[0]);
        else cache[cs++] = Slot{node.box[1], first + node.size[0], first + node.size[0] + node.size[1], 0, 0};
        if (cs < 4) {
            for (uint32_t i = 0; i < cs; i++) parentCache[i] = cache[i];
            return cs;
        }
        uint32_t j0 = 4, j1 = 5;
        if (cs > 4) {
            std::sort(cache, cache + cs, [](const Slot& a, const Slot& b) { return a.depth > b.depth; });
            float best = INFINITY;
            if (cs == 5) {
                for (uint32_t a = 0; a < 5; a++) {
                    Box b = boxEmpty();
                    for (uint32_t i = 0; i < 5; i++)
                        if (i != a) b = unite(b, cache[i].box);
                    if (best > area(b)) { best = area(b); j0 = a; }
                }
            } else {
                for (uint32_t c = 1; c < 6; c++)
                    for (uint32_t a = 0; a < c; a++) {
                        Box b = boxEmpty();
                        for (uint32_t i = 0; i < 6; i++)
                            if (i != a && i != c) b = unite(b, cache[i].box);
                        if (best > area(b)) { best = area(b); j0 = a; j1 = c; }
                    }
            }
        }
        const size_t me = --next;
        Slot* parent = parentCache++;
        *parent = Slot{boxEmpty(), 0, 0, uint32_t(me + 1), 0};
        uint32_t w = 0;
        for (uint32_t i = 0; i < cs; i++) {
            if (i == j0 || i == j1) {
                *parentCache++ = cache[i];
                continue;
            }
            if (cache[i].ofs) cache[i].ofs -= uint32_t(me + 1);
            if (cache[i].depth + 1 > parent->depth) parent->depth = cache[i].depth + 1;
            parent->box = unite(parent->box, cache[i].box);
            out[me].s[w++] = cache[i];
        }
        std::sort(out[me].s, out[me].s + 4, slotOrder);
        return cs - 3;
    }
};

struct Emitter {
    const std::vector<Node4>& n4;
    const hvvr_tri_shade* src;
    std::vector<hvvr_tri_shade> tris;
    std::vector<hvvr_topology_node> topo;

    uint32_t visit(size_t ni) {
        const uint32_t index = uint32_t(topo.size());
        topo.emplace_back();
        topo[index].leaf_mask = 0;
        topo[index].data[0] = uint32_t(tris.size());
        for (int k = 0; k < 4; k++) {
            const Slot& s = n4[ni].s[k];
            if (s.ofs) {
                const uint32_t child = visit(ni + s.ofs);
                topo[index].data[1 + k] = child - index;
                continue;
            }
            topo[index].leaf_mask |= 1u << k;
            for (uint32_t t = s.first; t != s.bound; t++) tris.push_back(src[t]);
            topo[index].data[1 + k] = uint32_t(tris.size());
        }
        return index;
    }
};

thread_local char gBvhError[160];

} // namespace

extern "C" int hvvr_generate_topology(hvvr_shading_vertex* verts, uint32_t vert_count, hvvr_tri_shade* tri_shade,
                                      uint32_t tri_count, hvvr_topology_node* nodes_out, uint32_t nodes_capacity,
                                      uint32_t* node_count) {
    if (!verts || !tri_shade || !nodes_out || !node_count || tri_count == 0) return HVVR_ERR_INVALID;
    for (uint32_t t = 0; t < tri_count; t++)
        for (int v = 0; v < 3; v++)
            if (tri_shade[t].indices[v] >= vert_count) return HVVR_ERR_INVALID;
    // leaf boxes (buildBVH2, bvh.cpp:251-294)
    std::vector<Box> leaf(tri_count);
    Builder bld;
    bld.leaf = &leaf;
    for (int a = 0; a < 3; a++) bld.key[a].resize(tri_count);
    for (uint32_t i = 0; i < tri_count; i++) {
        const hvvr_vec3& p0 = verts[tri_shade[i].indices[0]].pos;
        const hvvr_vec3& p1 = verts[tri_shade[i].indices[1]].pos;
        const hvvr_vec3& p2 = verts[tri_shade[i].indices[2]].pos;
        const float px[3] = {p0.x, p0.y, p0.z}, qx[3] = {p1.x, p1.y, p1.z}, rx[3] = {p2.x, p2.y, p2.z};
        for (int a = 0; a < 3; a++) {
            leaf[i].lo[a] = fminr(fminr(px[a], qx[a]), rx[a]);
            leaf[i].hi[a] = fmaxr(fmaxr(px[a], qx[a]), rx[a]);
            bld.key[a][i] = leaf[i].lo[a] + leaf[i].hi[a];
        }
    }
    std::vector<uint32_t> idx(tri_count);
    for (uint32_t i = 0; i < tri_count; i++) idx[i] = i;
    std::vector<float> scratch(tri_count);
    std::vector<Node2> n2(std::max<size_t>(tri_count - 1, 1));
    size_t count = bld.build(n2.data(), scratch.data(), idx.data(), tri_count, 3);
    if (!count) {
        Box all = leaf[0];
        for (uint32_t i = 1; i < tri_count; i++) all = unite(all, leaf[i]);
        n2[0].box[0] = boxEmpty();
        n2[0].offset[0] = 0;
        n2[0].size[0] = 0;
        n2[0].box[1] = all;
        n2[0].offset[1] = 0;
        n2[0].size[1] = tri_count;
        count = 1;
    }
    n2.resize(count);
    std::vector<hvvr_tri_shade> sortedTris(tri_count);
    for (uint32_t i = 0; i < tri_count; i++) sortedTris[i] = tri_shade[idx[i]];
    // buildBVH4 (bvh.cpp:427-467)
    std::vector<Node4> n4((n2.size() + 2) / 3);
    Collapser col{n2, n4, n4.size()};
    Slot cache[3];
    const uint32_t cs = col.visit(0, cache, 0);
    if (cs != 1) {
        const size_t me = --col.next;
        uint32_t w = 0;
        for (uint32_t extra = 4 - cs; extra; --extra) n4[me].s[w++] = Slot{Box{{0, 0, 0}, {0, 0, 0}}, 0, 0, 0, 0};
        for (uint32_t i = 0; i < cs; i++) {
            if (cache[i].ofs) cache[i].ofs -= uint32_t(me + 1);
            n4[me].s[w++] = cache[i];
        }
        std::sort(n4[me].s, n4[me].s + 4, slotOrder);
    }
    if (col.next != 0) {
        snprintf(gBvhError, sizeof(gBvhError), "BVH4 collapse left %zu unused nodes", col.next);
        return HVVR_ERR_STATE;
    }
    // TopologyBuilder (bvh.cpp:474-540)
    Emitter em{n4, sortedTris.data(), {}, {}};
    em.tris.reserve(tri_count);
    em.topo.reserve(n4.size());
    em.visit(0);
    if (em.tris.size() != tri_count || em.topo.size() > nodes_capacity) return HVVR_ERR_OVERFLOW;
    const uint32_t invalid = vert_count;
    uint32_t newIndex = invalid;
    std::vector<uint32_t> remap(vert_count, invalid);
    std::vector<hvvr_shading_vertex> outVerts(vert_count);
    for (int64_t t = int64_t(em.tris.size()) - 1; t >= 0; t--) {
        for (int v = 2; v >= 0; v--) {
            const uint32_t i = em.tris[t].indices[v];
            if (remap[i] == invalid) {
                remap[i] = --newIndex;
                outVerts[newIndex] = verts[i];
            }
            em.tris[t].indices[v] = remap[i];
        }
    }
    if (newIndex != 0) return HVVR_ERR_INVALID; // unreferenced vertices
    memcpy(tri_shade, em.tris.data(), size_t(tri_count) * sizeof(hvvr_tri_shade));
    memcpy(verts, outVerts.data(), size_t(vert_count) * sizeof(hvvr_shading_vertex));
    memcpy(nodes_out, em.topo.data(), em.topo.size() * sizeof(hvvr_topology_node));
    *node_count = uint32_t(em.topo.size());
    return HVVR_OK;
}
