// bvh_device.cu - hvvr_generate_topology_device: a linear BVH built on the GPU.
//
// No counterpart in the reference: its only build is the host SAH build of GenerateTopology
// (libraries/hvvr/shared/bvh.cpp:167-556), which this library restates in bvh_build.cpp. A scene
// admitted by a server pays for that build on the host (seconds at a million triangles); this is
// the fast alternative, with a different topology:
//   1. centroids of the triangles and their bounds (one pass, float min/max through ordered ints);
//   2. 30-bit Morton codes of the centroids over those bounds; a stable radix sort (CUB) of the
//      triangle indices by code, so equal codes keep the input order;
//   3. the binary radix tree of the sorted codes (one thread per internal node; equal codes are
//      told apart by their sorted position);
//   4. 4-wide nodes, level by level from the root: a node takes its two children and expands the
//      child with the most triangles (the first such in slot order) until it has four or none can
//      be expanded; a child of at most four triangles is a leaf slot. Leaf slots come before
//      internal slots, so that leaf slot k spans [data[k], data[k+1]) as the reference's
//      TopologyNode layout requires (libraries/hvvr/shared/graphics_types.h:126-151);
//   5. subtree sizes bottom-up, then depth-first node indices and leaf positions top-down, and the
//      nodes and the reordered triangles written in that order (vertices keep their order).
// Every step is exact integer or IEEE single-precision work in a fixed order, so the result is the
// same on every run; the oracle restates it step for step (oracle_lbvh_build).
#include <algorithm>
#include <cstdio>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/hvvr_c.h"
#include "dev_common.cuh"

namespace hvb {
namespace {

constexpr uint32_t kLeafTris = 4;
constexpr uint32_t kSingle = 0x80000000u; // a radix-tree child that is one sorted triangle

__device__ __forceinline__ uint32_t spreadBits10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t quantize10(float c, float lo, float scale) {
    float q = (c - lo) * scale;
    q = q > 0.0f ? q : 0.0f;
    q = q < 1023.0f ? q : 1023.0f;
    return uint32_t(q);
}

// order-preserving integer image of a float, for atomicMin / atomicMax on bounds
__device__ __forceinline__ uint32_t orderedBits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedFloat(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// centroid ((a + b) + c) * (1/3) per axis and the bounds of all centroids; bounds[0..2] min, [3..5] max
__global__ void __launch_bounds__(256) centroidKernel(const float4* __restrict__ verts, const uint4* __restrict__ tris,
                                                     uint32_t n, float* __restrict__ cen, uint32_t* bounds) {
    __shared__ uint32_t sb[6];
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint4 t = tris[i];
        const float4 a = verts[2 * size_t(t.x)], b = verts[2 * size_t(t.y)], c = verts[2 * size_t(t.z)];
        const float v[3] = {((a.x + b.x) + c.x) * (1.0f / 3.0f), ((a.y + b.y) + c.y) * (1.0f / 3.0f),
                            ((a.z + b.z) + c.z) * (1.0f / 3.0f)};
        for (int k = 0; k < 3; k++) {
            cen[size_t(i) * 3 + k] = v[k];
            atomicMin(&sb[k], orderedBits(v[k]));
            atomicMax(&sb[3 + k], orderedBits(v[k]));
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&bounds[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&bounds[threadIdx.x], sb[threadIdx.x]);
}

__global__ void __launch_bounds__(256) mortonKernel(const float* __restrict__ cen, uint32_t n,
                                                    const uint32_t* __restrict__ bounds, uint32_t* __restrict__ codes,
                                                    uint32_t* __restrict__ index) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], scale[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = orderedFloat(bounds[k]);
        const float ext = orderedFloat(bounds[3 + k]) - lo[k];
        scale[k] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    const float* c = cen + size_t(i) * 3;
    codes[i] = (spreadBits10(quantize10(c[0], lo[0], scale[0])) << 2) |
               (spreadBits10(quantize10(c[1], lo[1], scale[1])) << 1) | spreadBits10(quantize10(c[2], lo[2], scale[2]));
    index[i] = i;
}

__device__ __forceinline__ int delta(const uint32_t* __restrict__ keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clz(a ^ b);
}

// one internal node of the binary radix tree per thread (i in [0, n-2])
__global__ void __launch_bounds__(256) radixTreeKernel(const uint32_t* __restrict__ keys, int n, uint32_t* left,
                                                       uint32_t* right, uint32_t* first, uint32_t* last) {
    const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i + 1 >= n) return;
    const int d = delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1) > 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int s = lmax / 2; s >= 1; s /= 2)
        if (delta(keys, n, i, i + (l + s) * d) > dmin) l += s;
    const int j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
        const int step = (l + div - 1) / div;
        if (delta(keys, n, i, i + (s + step) * d) > dnode) s += step;
        if (step <= 1) break;
    }
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    left[i] = lo == gamma ? (kSingle | uint32_t(gamma)) : uint32_t(gamma);
    right[i] = hi == gamma + 1 ? (kSingle | uint32_t(gamma + 1)) : uint32_t(gamma + 1);
    first[i] = uint32_t(lo);
    last[i] = uint32_t(hi);
}

struct Tree {
    const uint32_t* left;
    const uint32_t* right;
    const uint32_t* first;
    const uint32_t* last;
};

struct Entry {
    uint32_t node, lo, hi;
    __device__ uint32_t count() const { return hi - lo + 1; }
    __device__ bool internal() const { return count() > kLeafTris; }
};

__device__ __forceinline__ Entry entryOf(const Tree& t, uint32_t c) {
    if (c & kSingle) return Entry{c, c & ~kSingle, c & ~kSingle};
    return Entry{c, t.first[c], t.last[c]};
}

// the 4-wide nodes of one level, one thread each: its entries (leaf slots first), and one node of
// the next level per internal entry (appended at *nextCount after nextBase)
struct Levels {
    uint32_t* src;        // [node] radix-tree node the 4-wide node expands (kSingle | 0: the whole set as a leaf)
    uint32_t* parent;     // [node] parent 4-wide node (root: itself)
    uint32_t* slots;      // [node * 4] entry node ids (kSingle | position for one triangle; ~0 empty)
    uint32_t* lo;         // [node * 4]
    uint32_t* hi;         // [node * 4]
    uint32_t* child;      // [node * 4] 4-wide node of an internal entry, else ~0
    uint32_t* nslots;     // [node] entries used (1..4)
    uint32_t* subtree;    // [node] nodes in its subtree
    uint32_t* dfs;        // [node] depth-first index
    uint32_t* triStart;   // [node] position of its first triangle in the output order
};

__global__ void __launch_bounds__(256) collapseKernel(Tree t, Levels L, uint32_t levelStart, uint32_t levelCount,
                                                      uint32_t nextBase, uint32_t* nextCount, uint32_t nTris,
                                                      uint32_t maxNodes, uint32_t* error) {
    const uint32_t m = levelStart + blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= levelStart + levelCount) return;
    Entry e[4];
    int n;
    const uint32_t x = L.src[m];
    if (x == kSingle) { // fewer triangles than one leaf holds: the root is one leaf slot
        e[0] = Entry{kSingle, 0u, nTris - 1};
        n = 1;
    } else {
        e[0] = entryOf(t, t.left[x]);
        e[1] = entryOf(t, t.right[x]);
        n = 2;
        while (n < 4) {
            int best = -1;
            for (int k = 0; k < n; k++)
                if (e[k].internal() && (best < 0 || e[k].count() > e[best].count())) best = k;
            if (best < 0) break;
            const uint32_t id = e[best].node;
            for (int k = n; k > best + 1; k--) e[k] = e[k - 1];
            e[best] = entryOf(t, t.left[id]);
            e[best + 1] = entryOf(t, t.right[id]);
            n++;
        }
    }
    int w = 0;
    for (int pass = 0; pass < 2; pass++)
        for (int k = 0; k < n; k++) {
            if (e[k].internal() != (pass == 1)) continue;
            L.slots[m * 4 + w] = e[k].node;
            L.lo[m * 4 + w] = e[k].lo;
            L.hi[m * 4 + w] = e[k].hi;
            uint32_t c = ~0u;
            if (pass == 1) {
                c = nextBase + atomicAdd(nextCount, 1u);
                if (c < maxNodes) { // always: a 4-wide node per radix-tree node at most
                    L.src[c] = e[k].node;
                    L.parent[c] = m;
                } else {
                    atomicOr(error, 1u);
                    c = ~0u;
                }
            }
            L.child[m * 4 + w] = c;
            w++;
        }
    for (; w < 4; w++) {
        L.slots[m * 4 + w] = ~0u;
        L.child[m * 4 + w] = ~0u;
    }
    L.nslots[m] = uint32_t(n);
}

// subtree node counts of one level, children (one level down) already counted
__global__ void __launch_bounds__(256) subtreeKernel(Levels L, uint32_t levelStart, uint32_t levelCount) {
    const uint32_t m = levelStart + blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= levelStart + levelCount) return;
    uint32_t s = 1;
    for (int k = 0; k < 4; k++)
        if (L.child[m * 4 + k] != ~0u) s += L.subtree[L.child[m * 4 + k]];
    L.subtree[m] = s;
}

// depth-first index and first triangle position of the children of one level's nodes, then the
// node itself and its leaf triangles written
__global__ void __launch_bounds__(256) layoutKernel(Levels L, uint32_t levelStart, uint32_t levelCount,
                                                    const uint32_t* __restrict__ order, const uint4* __restrict__ tris,
                                                    uint4* __restrict__ trisOut, hvvr_topology_node* __restrict__ nodes) {
    const uint32_t m = levelStart + blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= levelStart + levelCount) return;
    const uint32_t index = L.dfs[m];
    uint32_t pos = L.triStart[m];
    hvvr_topology_node out;
    out.leaf_mask = 0;
    out.data[0] = pos;
    uint32_t nextIndex = index + 1;
    for (int k = 0; k < 4; k++) {
        const uint32_t c = L.child[m * 4 + k];
        if (L.slots[m * 4 + k] == ~0u) { // empty leaf slot
            out.leaf_mask |= 1u << k;
            out.data[1 + k] = pos;
            continue;
        }
        if (c == ~0u) { // leaf slot: its triangles in sorted order
            out.leaf_mask |= 1u << k;
            for (uint32_t p = L.lo[m * 4 + k]; p <= L.hi[m * 4 + k]; p++) trisOut[pos++] = tris[order[p]];
            out.data[1 + k] = pos;
            continue;
        }
        out.data[1 + k] = nextIndex - index;
        L.dfs[c] = nextIndex;
        L.triStart[c] = pos;
        nextIndex += L.subtree[c];
        pos += L.hi[m * 4 + k] - L.lo[m * 4 + k] + 1;
    }
    for (int k = 5; k < 7; k++) out.data[k] = 0;
    nodes[index] = out;
}

template <class T>
struct Buf {
    T* p = nullptr;
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

int failBuild(int code, const char* msg, cudaError_t e = cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%s%s%s", msg, e == cudaSuccess ? "" : ": ", e == cudaSuccess ? "" : cudaGetErrorString(e));
    return setLastError(code, buf);
}

} // namespace
} // namespace hvb

using namespace hvb;

#define BUILD_TRY(x)                                                                                                  \
    do {                                                                                                             \
        const cudaError_t e_ = (x);                                                                                  \
        if (e_ != cudaSuccess) return failBuild(HVVR_ERR_CUDA, #x, e_);                                              \
    } while (0)

extern "C" int hvvr_generate_topology_device(const hvvr_shading_vertex* verts, uint32_t vert_count,
                                             hvvr_tri_shade* tri_shade, uint32_t tri_count, hvvr_topology_node* nodes_out,
                                             uint32_t capacity, uint32_t* node_count, void* stream) {
    if (!verts || !tri_shade || !nodes_out || !node_count) return failBuild(HVVR_ERR_INVALID, "NULL argument");
    if (tri_count == 0) return failBuild(HVVR_ERR_INVALID, "no triangles");
    if (tri_count >= (1u << 30)) return failBuild(HVVR_ERR_INVALID, "at most 2^30-1 triangles");
    for (uint32_t i = 0; i < tri_count; i++)
        for (int k = 0; k < 3; k++)
            if (tri_shade[i].indices[k] >= vert_count) return failBuild(HVVR_ERR_INVALID, "vertex index out of range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t n = tri_count;
    // at most one 4-wide node per radix-tree node (n - 1 of them), and one for a single-leaf root
    const size_t maxNodes = std::max<size_t>(1, n);
    Buf<float4> dVerts;
    Buf<uint4> dTris, dTrisOut;
    Buf<float> dCen;
    Buf<uint32_t> dBounds, dCodes, dCodesSorted, dIndex, dOrder, dLeft, dRight, dFirst, dLast, dCount;  // dCount: [0] next level, [1] error
    Buf<uint32_t> lSrc, lParent, lSlots, lLo, lHi, lChild, lN, lSub, lDfs, lTri;
    Buf<hvvr_topology_node> dNodes;
    BUILD_TRY(dVerts.alloc(size_t(vert_count) * 2));
    BUILD_TRY(dTris.alloc(n));
    BUILD_TRY(dTrisOut.alloc(n));
    BUILD_TRY(dCen.alloc(size_t(n) * 3));
    BUILD_TRY(dBounds.alloc(6));
    BUILD_TRY(dCodes.alloc(n));
    BUILD_TRY(dCodesSorted.alloc(n));
    BUILD_TRY(dIndex.alloc(n));
    BUILD_TRY(dOrder.alloc(n));
    for (Buf<uint32_t>* b : {&dLeft, &dRight, &dFirst, &dLast}) BUILD_TRY(b->alloc(n));
    BUILD_TRY(dCount.alloc(2));
    BUILD_TRY(cudaMemsetAsync(dCount.p, 0, 8, st));
    for (Buf<uint32_t>* b : {&lSrc, &lParent, &lN, &lSub, &lDfs, &lTri}) BUILD_TRY(b->alloc(maxNodes));
    for (Buf<uint32_t>* b : {&lSlots, &lLo, &lHi, &lChild}) BUILD_TRY(b->alloc(maxNodes * 4));
    BUILD_TRY(dNodes.alloc(maxNodes));
    BUILD_TRY(cudaMemcpyAsync(dVerts.p, verts, size_t(vert_count) * 32, cudaMemcpyHostToDevice, st));
    BUILD_TRY(cudaMemcpyAsync(dTris.p, tri_shade, size_t(n) * 16, cudaMemcpyHostToDevice, st));
    const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    BUILD_TRY(cudaMemcpyAsync(dBounds.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
    const uint32_t grid = (n + 255) / 256;
    centroidKernel<<<grid, 256, 0, st>>>(dVerts.p, dTris.p, n, dCen.p, dBounds.p);
    mortonKernel<<<grid, 256, 0, st>>>(dCen.p, n, dBounds.p, dCodes.p, dIndex.p);
    BUILD_TRY(cudaGetLastError());
    size_t tempBytes = 0;
    BUILD_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, dCodes.p, dCodesSorted.p, dIndex.p, dOrder.p, int(n),
                                              0, 30, st));
    Buf<unsigned char> temp;
    BUILD_TRY(temp.alloc(tempBytes));
    BUILD_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tempBytes, dCodes.p, dCodesSorted.p, dIndex.p, dOrder.p, int(n), 0,
                                              30, st));
    if (n > 1) radixTreeKernel<<<(n - 1 + 255) / 256, 256, 0, st>>>(dCodesSorted.p, int(n), dLeft.p, dRight.p,
                                                                     dFirst.p, dLast.p);
    BUILD_TRY(cudaGetLastError());
    const Tree tree{dLeft.p, dRight.p, dFirst.p, dLast.p};
    const Levels L{lSrc.p, lParent.p, lSlots.p, lLo.p, lHi.p, lChild.p, lN.p, lSub.p, lDfs.p, lTri.p};
    // the root: radix-tree node 0, or the whole set as one leaf
    const uint32_t rootSrc = n > kLeafTris ? 0u : kSingle;
    const uint32_t zero = 0;
    BUILD_TRY(cudaMemcpyAsync(lSrc.p, &rootSrc, 4, cudaMemcpyHostToDevice, st));
    BUILD_TRY(cudaMemcpyAsync(lParent.p, &zero, 4, cudaMemcpyHostToDevice, st));
    BUILD_TRY(cudaMemcpyAsync(lDfs.p, &zero, 4, cudaMemcpyHostToDevice, st));
    BUILD_TRY(cudaMemcpyAsync(lTri.p, &zero, 4, cudaMemcpyHostToDevice, st));
    std::vector<uint32_t> levelStart{0}, levelCount{1};
    for (;;) {
        const uint32_t s = levelStart.back(), c = levelCount.back();
        BUILD_TRY(cudaMemsetAsync(dCount.p, 0, 4, st));
        collapseKernel<<<(c + 255) / 256, 256, 0, st>>>(tree, L, s, c, s + c, dCount.p, n, uint32_t(maxNodes),
                                                         dCount.p + 1);
        BUILD_TRY(cudaGetLastError());
        uint32_t next[2] = {0, 0};
        BUILD_TRY(cudaMemcpyAsync(next, dCount.p, 8, cudaMemcpyDeviceToHost, st));
        BUILD_TRY(cudaStreamSynchronize(st));
        if (next[1] || size_t(s) + c + next[0] > maxNodes) return failBuild(HVVR_ERR_INVALID, "node count past the bound");
        if (next[0] == 0) break;
        levelStart.push_back(s + c);
        levelCount.push_back(next[0]);
    }
    const uint32_t total = levelStart.back() + levelCount.back();
    if (total > capacity) return failBuild(HVVR_ERR_OVERFLOW, "node capacity too small");
    for (size_t k = levelStart.size(); k-- > 0;)
        subtreeKernel<<<(levelCount[k] + 255) / 256, 256, 0, st>>>(L, levelStart[k], levelCount[k]);
    for (size_t k = 0; k < levelStart.size(); k++)
        layoutKernel<<<(levelCount[k] + 255) / 256, 256, 0, st>>>(L, levelStart[k], levelCount[k], dOrder.p, dTris.p,
                                                                  dTrisOut.p, dNodes.p);
    BUILD_TRY(cudaGetLastError());
    BUILD_TRY(cudaMemcpyAsync(nodes_out, dNodes.p, size_t(total) * sizeof(hvvr_topology_node), cudaMemcpyDeviceToHost, st));
    BUILD_TRY(cudaMemcpyAsync(tri_shade, dTrisOut.p, size_t(n) * 16, cudaMemcpyDeviceToHost, st));
    BUILD_TRY(cudaStreamSynchronize(st));
    *node_count = total;
    return HVVR_OK;
}
