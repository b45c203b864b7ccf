// traverse.cu - tile-frustum BVH traversal on the GPU.
//
// Two kernels restate the reference's two-level CPU traversal (cullThread,
// libraries/hvvr/raycaster/traversal.cpp:99-190) one warp per frustum:
//   blockCullKernel: traverseBlocks + BlockFrame::sort per 8192-sample block frustum
//                    (libraries/hvvr/raycaster/traverse_avx.h:293-410);
//   tileCullKernel:  traverseTiles per 128-sample tile frustum, starting from its block's
//                    sorted stack (traverse_avx.h:412-527), emitting the tile's triangle list.
// Both rebuild the world-space frustum of Frustum::Frustum (traverse_avx.cpp:22-211) from the
// camera-space corner rays and the camera matrix (frustumTransform, traversal.h:38-47).
//
// Lane layout of one node visit: lane l loads word l of the 128-byte node (one coalesced
// row); child c = l & 3 receives its six bounds by shuffle. Lanes 0-15 run the plane test
// of plane l>>2, lanes 16-27 the axis-projection test of axis (l-16)>>2, and every lane runs
// one or two of the 48 edge-axis tests (edge l>>2 and, for l < 16, edge 8+(l>>2)). Ballots
// fold the per-lane results into the reference's 4-bit child masks, so the arithmetic per
// test is exactly the reference's lane arithmetic (explicit fmaf where it uses
// _mm256_fmadd_ps, IEEE single ops elsewhere) and the stacks evolve identically.
#include <algorithm>
#include <mutex>

#include "../../include/hvvr_c.h"
#include "dev_common.cuh"

namespace hvb {

namespace {

constexpr unsigned kFull = 0xffffffffu;

#ifdef HVVR_VISIT_CLOCKS
// Profiling build only (make -C hvvr_b200/csrc visit-clocks): per global tile, the SM cycles of
// its tile-cull node visits split into phases, plus its visit count, read back through
// hvvr_dbg_visit_clocks. The counters cost registers and instructions of their own, so the
// phases' shares are what this build measures, not the production kernel's absolute times.
constexpr uint32_t kVisitClockTiles = 1u << 17;
enum : uint32_t {
    kVcRow,    // waiting for the node's row (loaded during the previous visit)
    kVcTest,   // child-row loads issued, child boxes shuffled, frustum plane/projection tests
    kVcLeaf,   // refine tests of passing leaf slots and recording their triangle ranges
    kVcInsert, // sorted insertion of two or more internal children
    kVcNext,   // choosing the next node (one child, an inserted child, or a pop)
    kVcTail,   // after the last visit: expanding the buffered ranges into the tile's list
    kVcPhases
};
__device__ unsigned long long gVisitClocks[kVisitClockTiles][kVcPhases + 1];
#define VISIT_MARK(phase, dep)                                                                                         \
    do {                                                                                                               \
        const long long t_ = phaseClock(dep);                                                                          \
        vcAcc[phase] += t_ - vcLast;                                                                                   \
        vcLast = t_;                                                                                                   \
    } while (0)
#else
#define VISIT_MARK(phase, dep) do { } while (0)
#endif

struct SmemFrustum {
    float tpLo[4][3], tpHi[4][3], w[4];
    float proj[3][8];
    float edge[12][3];
    float minF[12], maxF[12];
    int distIdx;
    int degenerate;
};

// Lane layout (child-major): lane l serves child c = l >> 3 and test slot j = l & 7. Slots
// 0-3 are the four frustum planes, 4-6 the x/y/z projection overlaps, 7 always passes; so
// child c passes testBVHNodeChildren when byte c of the ballot is 0xFF. For the refine, slot j
// tests edge axis j and, for j < 4, also edge axis 8 + j; child c is rejected when byte c of
// that ballot is nonzero.
struct LaneTest {
    float c0, c1, c2, c3, c4, c5, c6; // plane slots: lo xyz, hi xyz, w; projection slots: c0 = max side, c1 = -min side
    int kind;                         // 0 plane, 1 projection, 2 always pass
    int axis;                         // projection axis
    float e0x, e0y, e0z, mn0, mx0;
    float e1x, e1y, e1z, mn1, mx1;
    bool has1;
};

// Frustum::Frustum on world-space rays, computed cooperatively by one warp.
__device__ void buildFrustum(const Rays4& cr, const Mat4& M, SmemFrustum& f) {
    F3 o[4], d[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        o[i] = xformPoint(M, f3(cr.o[i][0], cr.o[i][1], cr.o[i][2]));
        d[i] = xformDir(M, f3(cr.d[i][0], cr.d[i][1], cr.d[i][2]));
    }
    const uint32_t lane = laneId();
    const bool inf0 = isinf(o[0].x);
    if (lane < 4) {
        const int p = int(lane);
        F3 n = f3(0.0f, 0.0f, 0.0f);
        float w = -INFINITY;
        if (!inf0) {
            n = cross3(d[p], d[(p + 1) & 3]);
            w = dot3(o[p], n);
        }
        const float c[3] = {n.x, n.y, n.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            f.tpLo[p][a] = c[a] < 0.0f ? c[a] : 0.0f;
            f.tpHi[p][a] = c[a] > 0.0f ? -c[a] : 0.0f;
        }
        f.w[p] = w;
        if (p == 0) f.degenerate = (w == -INFINITY) ? 1 : 0;
    } else if (lane < 16) {
        const int e = int(lane) - 4, i = e / 3, k = e % 3;
        const F3 axis = f3(k == 0 ? 1.0f : 0.0f, k == 1 ? 1.0f : 0.0f, k == 2 ? 1.0f : 0.0f);
        const F3 ed = cross3(d[i], axis);
        f.edge[e][0] = ed.x;
        f.edge[e][1] = ed.y;
        f.edge[e][2] = ed.z;
        float mn = FLT_MAX, mx = -FLT_MAX;
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const float d0 = fmaf(ed.x, o[p].x, fmaf(ed.y, o[p].y, ed.z * o[p].z));
            mn = mn < d0 ? mn : d0;
            mx = mx > d0 ? mx : d0;
            const float d1 = fmaf(ed.x, d[p].x, fmaf(ed.y, d[p].y, ed.z * d[p].z));
            const float a = d1 + .000001f, b = d1 - .000001f;
            const float amin = a < 0.0f ? a : 0.0f;
            const float bmax = b > 0.0f ? b : 0.0f;
            mn = amin * FLT_MAX + mn;
            mx = bmax * FLT_MAX + mx;
        }
        f.minF[e] = mn;
        f.maxF[e] = mx;
    } else if (lane < 19) {
        const int a = int(lane) - 16;
        float lanev[8];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float oc = a == 0 ? o[i].x : (a == 1 ? o[i].y : o[i].z);
            const float dc = a == 0 ? d[i].x : (a == 1 ? d[i].y : d[i].z);
            const float nd0 = -dc, nd1 = -(-dc);
            const float m0 = (0.0f > nd0) ? 0.0f : nd0;
            const float m1 = (0.0f > nd1) ? 0.0f : nd1;
            lanev[i] = -oc + FLT_MAX * m0;
            lanev[4 + i] = -(-oc) + FLT_MAX * m1;
        }
        float y[8];
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float p0 = lanev[4 * h + i], p1 = lanev[4 * h + (i ^ 2)];
                y[4 * h + i] = p0 > p1 ? p0 : p1;
            }
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float p0 = y[4 * h + i], p1 = y[4 * h + (i ^ 1)];
                f.proj[a][4 * h + i] = -(p0 > p1 ? p0 : p1);
            }
    } else if (lane == 19) {
        F3 avg = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int p = 0; p < 4; p++) avg = avg + d[p];
        int idx;
        if (fabsf(avg.x) > fabsf(avg.y)) {
            if (fabsf(avg.x) > fabsf(avg.z)) idx = avg.x < 0 ? 0 : 1;
            else idx = avg.z < 0 ? 4 : 5;
        } else {
            if (fabsf(avg.y) > fabsf(avg.z)) idx = avg.y < 0 ? 2 : 3;
            else idx = avg.z < 0 ? 4 : 5;
        }
        f.distIdx = idx;
    }
    __syncwarp();
}

// blockTransformAndCullTask's cull of a tile frustum (libraries/hvvr/raycaster/render.cpp:270-279,
// 314-338): culled when all four corner rays, at their origin and 10000 units out, lie beyond
// one of the planes. Evaluated by every lane on the same world-space rays.
__device__ bool tileCulled(const Rays4& cr, const Mat4& M, const float (&pl)[4][4]) {
    F3 o[4], d[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        o[i] = xformPoint(M, f3(cr.o[i][0], cr.o[i][1], cr.o[i][2]));
        d[i] = xformDir(M, f3(cr.d[i][0], cr.d[i][1], cr.d[i][2]));
    }
    bool culled = false;
#pragma unroll
    for (int p = 0; p < 4; p++) {
        const F3 n = f3(pl[p][0], pl[p][1], pl[p][2]);
        const float dist = pl[p][3];
        bool allout = true;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            allout = allout && dot3(n, o[i]) > dist;
            allout = allout && dot3(n, o[i] + d[i] * 10000.0f) > dist;
        }
        culled = culled || allout;
    }
    return culled;
}

__device__ LaneTest loadLaneTest(const SmemFrustum& f) {
    LaneTest t;
    const uint32_t lane = laneId();
    const int c = int(lane >> 3), j = int(lane & 7);
    t.c0 = t.c1 = t.c2 = t.c3 = t.c4 = t.c5 = t.c6 = 0.0f;
    t.axis = 0;
    if (j < 4) {
        t.kind = 0;
        t.c0 = f.tpLo[j][0]; t.c1 = f.tpLo[j][1]; t.c2 = f.tpLo[j][2];
        t.c3 = f.tpHi[j][0]; t.c4 = f.tpHi[j][1]; t.c5 = f.tpHi[j][2];
        t.c6 = f.w[j];
    } else if (j < 7) {
        t.kind = 1;
        t.axis = j - 4;
        t.c0 = f.proj[j - 4][c];
        t.c1 = f.proj[j - 4][4 + c];
    } else {
        t.kind = 2;
    }
    t.e0x = f.edge[j][0]; t.e0y = f.edge[j][1]; t.e0z = f.edge[j][2];
    t.mn0 = f.minF[j]; t.mx0 = f.maxF[j];
    t.has1 = j < 4;
    const int e1 = t.has1 ? 8 + j : j;
    t.e1x = f.edge[e1][0]; t.e1y = f.edge[e1][1]; t.e1z = f.edge[e1][2];
    t.mn1 = f.minF[e1]; t.mx1 = f.maxF[e1];
    return t;
}

struct ChildBox {
    float xM, xN, yM, yN, zM, zN;
};

__device__ __forceinline__ ChildBox childBox(float v) {
    const uint32_t c = laneId() >> 3;
    ChildBox b;
    b.xM = __shfl_sync(kFull, v, c);
    b.xN = __shfl_sync(kFull, v, 4 + c);
    b.yM = __shfl_sync(kFull, v, 8 + c);
    b.yN = __shfl_sync(kFull, v, 12 + c);
    b.zM = __shfl_sync(kFull, v, 16 + c);
    b.zN = __shfl_sync(kFull, v, 20 + c);
    return b;
}

// Bit c set where byte c of m is all ones / nonzero. Per byte, (b & 0x7f) + 0x7f sets the byte's
// high bit exactly when its low seven bits are not all zero and never carries into the next byte
// (at most 0xfe), so the byte tests are exact; the multiply gathers bits 7, 15, 23, 31 into bits
// 21-24 (the partial products land on distinct bits, so nothing carries).
__device__ __forceinline__ uint32_t gatherByteFlags(uint32_t z) { return (((z >> 7) * 0x204081u) >> 21) & 0xfu; }
__device__ __forceinline__ uint32_t bytesAllOnes(uint32_t m) {
    const uint32_t s = (~m & 0x7f7f7f7fu) + 0x7f7f7f7fu; // high bit: the byte of ~m has a low bit set
    return gatherByteFlags(~s & m & 0x80808080u);
}
__device__ __forceinline__ uint32_t bytesNonZero(uint32_t m) {
    const uint32_t s = (m & 0x7f7f7f7fu) + 0x7f7f7f7fu;
    return gatherByteFlags((s | m) & 0x80808080u);
}

// Frustum::testBVHNodeChildren (traverse_avx.h:104-164)
__device__ __forceinline__ uint32_t testChildren(const ChildBox& b, const LaneTest& t) {
    const float lo = fmaf(t.c0, b.xM, fmaf(t.c1, b.yM, t.c2 * b.zM));
    const float hi = fmaf(t.c3, b.xN, fmaf(t.c4, b.yN, t.c5 * b.zN));
    const bool planePass = (lo + hi) <= t.c6;
    const float am = t.axis == 0 ? b.xM : (t.axis == 1 ? b.yM : b.zM);
    const float an = t.axis == 0 ? b.xN : (t.axis == 1 ? b.yN : b.zN);
    const bool projPass = (am >= t.c0) && (an >= t.c1);
    const bool pass = t.kind == 0 ? planePass : (t.kind == 1 ? projPass : true);
    return bytesAllOnes(__ballot_sync(kFull, pass));
}

// The reference adds +0.0f to each selected bound (turning -0 into +0); that only changes the
// sign of a zero product or sum, which no comparison below can see, so it is left out.
__device__ __forceinline__ bool edgeReject(const ChildBox& b, float ex, float ey, float ez, float mn, float mx) {
    const bool px = ex > 0.0f, py = ey > 0.0f, pz = ez > 0.0f;
    const float pX = px ? b.xM : -b.xN, nX = px ? -b.xN : b.xM;
    const float pY = py ? b.yM : -b.yN, nY = py ? -b.yN : b.yM;
    const float pZ = pz ? b.zM : -b.zN, nZ = pz ? -b.zN : b.zM;
    const float maxBox = fmaf(ex, pX, fmaf(ey, pY, ez * pZ));
    const float minBox = fmaf(ex, nX, fmaf(ey, nY, ez * nZ));
    return (maxBox < mn) || (mx < minBox);
}

// Frustum::testBVHNodeChildrenRefine (traverse_avx.h:166-217): mask of rejected children
__device__ __forceinline__ uint32_t refineReject(const ChildBox& b, const LaneTest& t) {
    const bool rej0 = edgeReject(b, t.e0x, t.e0y, t.e0z, t.mn0, t.mx0);
    const bool rej1 = edgeReject(b, t.e1x, t.e1y, t.e1z, t.mn1, t.mx1);
    return bytesNonZero(__ballot_sync(kFull, rej0 || (t.has1 && rej1)));
}

// Number of consecutive stack entries, from position top-1 downwards, for which pred holds.
// Equivalent to the reference's serial shift loop; the guard band below position 0 stops it.
template <class Pred>
__device__ __forceinline__ uint32_t shiftCount(uint32_t top, Pred pred) {
    const uint32_t lane = laneId();
    uint32_t k = 0;
    for (;;) {
        const int p = int(top) - 1 - int(k) - int(lane);
        const bool pr = (p >= 0) && pred(uint32_t(p));
        const uint32_t b = __ballot_sync(kFull, pr);
        const uint32_t run = (b == kFull) ? 32u : uint32_t(__ffs(~b) - 1);
        k += run;
        if (run < 32u || k >= top) return k < top ? k : top;
    }
}

// move entries [top-k, top) up by one slot (three parallel arrays)
template <class T0, class T1, class T2>
__device__ __forceinline__ void shiftUp(T0* a, T1* b, T2* c, uint32_t top, uint32_t k) {
    const uint32_t lane = laneId();
    for (uint32_t base = 0; base < k; base += 32) {
        const uint32_t j = base + lane;
        T0 va{}; T1 vb{}; T2 vc{};
        uint32_t p = 0;
        const bool act = j < k;
        if (act) { p = top - 1 - j; va = a[p]; vb = b[p]; vc = c[p]; }
        __syncwarp();
        if (act) { a[p + 1] = va; b[p + 1] = vb; c[p + 1] = vc; }
        __syncwarp();
    }
}

constexpr int kBlockWarps = 4;

struct BlockSmem {
    SmemFrustum f;
    uint32_t delta[kBlockStack + 4];
    float tMinTemp[kBlockStack + 4];
    uint32_t node[kBlockStack + 4];
    float sTMin[kBlockStack];
    uint32_t sMask[kBlockStack];
    uint32_t sNode[kBlockStack];
};

// the view of a global block (blocks of one view are consecutive)
__device__ __forceinline__ const ViewDev& viewOfBlock(const ViewDev* __restrict__ views,
                                                      const uint32_t* __restrict__ blockView, uint32_t viewCount,
                                                      uint32_t blk) {
    return views[viewCount == 1 ? 0u : __ldg(blockView + blk)];
}

// A block walks up to a few hundred dependent node visits, each of which waits for its node's row
// if it misses L2; so the CTAs past the block-cull CTAs first bring every scene's node array into
// L2 (bulk prefetches of 4 KiB, issued at once; the traversing warps meet lines in flight or
// resident, and so do the tile culls that follow).
constexpr uint32_t kPrefetchCtas = 32, kPrefetchChunk = 4096;

__device__ void prefetchSceneNodes(const FrameDev& fr, uint32_t cta) {
    const uint32_t tid = cta * blockDim.x + threadIdx.x, threads = kPrefetchCtas * blockDim.x;
    for (uint32_t vi = 0; vi < fr.viewCount; vi++) {
        const ViewDev& V = fr.views[vi];
        // whole 128-byte nodes of a 128-byte-aligned array: every chunk starts 16-byte aligned and
        // its size is a multiple of 16
        const size_t bytes = size_t(V.prefetchNodes) * sizeof(Node);
        const char* base = reinterpret_cast<const char*>(V.nodes);
        for (size_t off = size_t(tid) * kPrefetchChunk; off < bytes; off += size_t(threads) * kPrefetchChunk) {
            const uint32_t n = uint32_t(bytes - off < kPrefetchChunk ? bytes - off : kPrefetchChunk);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + off), "r"(n) : "memory");
        }
    }
}

__global__ void __launch_bounds__(kBlockWarps * 32) blockCullKernel(FrameDev fr) {
    __shared__ BlockSmem smem[kBlockWarps];
    const uint32_t blockCtas = (fr.blocks + kBlockWarps - 1) / kBlockWarps;
    if (blockIdx.x >= blockCtas) {
        prefetchSceneNodes(fr, blockIdx.x - blockCtas);
        return;
    }
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    const uint32_t gblk = blockIdx.x * kBlockWarps + warp;
    if (gblk >= fr.blocks) return;
    const ViewDev& V = viewOfBlock(fr.views, fr.blockView, fr.viewCount, gblk);
    const uint32_t blk = gblk - V.blockStart;
    const Node* __restrict__ nodes = V.nodes;
    StackEntry* __restrict__ out = V.blockStacks;
    uint32_t* __restrict__ sizes = V.blockSizes;
    BlockSmem& s = smem[warp];
    buildFrustum(V.blockRays[blk], V.M, s.f);
    if (s.f.degenerate) {
        if (lane == 0) sizes[blk] = 0;
        return;
    }
    const LaneTest t = loadLaneTest(s.f);
    const int distIdx = s.f.distIdx, maxIdx = distIdx & ~1;
    uint32_t top = 0, node = 0;
    float tMin = 0.0f;
    for (;;) {
        const float v = reinterpret_cast<const float*>(nodes + node)[lane];
        const ChildBox cb = childBox(v);
        uint32_t mask = testChildren(cb, t);
        mask &= ~refineReject(cb, t);
        const uint32_t leafMask = __float_as_uint(__shfl_sync(kFull, v, 24));
        if (mask) {
            const uint32_t leaf = mask & leafMask;
            if (leaf) {
                mask &= ~leaf;
                // leaf entries go below every internal entry (tDelta > 0 under DAZ)
                const uint32_t k = shiftCount(top, [&](uint32_t p) { return dazf(__uint_as_float(s.delta[p])) > 0.0f; });
                shiftUp(s.delta, s.tMinTemp, s.node, top, k);
                if (lane == 0) { s.delta[top - k] = leaf; s.tMinTemp[top - k] = tMin; s.node[top - k] = node; }
                __syncwarp();
                ++top;
            }
            while (mask) {
                const int k = __ffs(mask) - 1;
                const float tm = __uint_as_float(__float_as_uint(__shfl_sync(kFull, v, distIdx * 4 + k)) ^ 0x80000000u);
                const float td = __shfl_sync(kFull, v, maxIdx * 4 + k) + __shfl_sync(kFull, v, (maxIdx + 1) * 4 + k);
                const uint32_t child = node + __float_as_uint(__shfl_sync(kFull, v, 26 + k));
                const float tdz = dazf(td);
                const uint32_t n = shiftCount(top, [&](uint32_t p) { return dazf(__uint_as_float(s.delta[p])) > tdz; });
                shiftUp(s.delta, s.tMinTemp, s.node, top, n);
                if (lane == 0) { s.delta[top - n] = __float_as_uint(td); s.tMinTemp[top - n] = tm; s.node[top - n] = child; }
                __syncwarp();
                ++top;
                mask &= mask - 1;
            }
        }
        if (top >= kBlockStack - 4 || top == 0 || s.delta[top - 1] <= 0xfu) break;
        --top;
        node = s.node[top];
        tMin = s.tMinTemp[top];
    }
    // BlockFrame::sort: insertion sort by distance estimate, closest on top
    const uint32_t stackSize = top;
    for (uint32_t i = 0; i < stackSize; i++) {
        const float tm = s.tMinTemp[i];
        const uint32_t dbits = s.delta[i];
        const uint32_t nd = s.node[i];
        const float tmz = dazf(tm);
        const uint32_t k = shiftCount(i, [&](uint32_t p) { return dazf(s.sTMin[p]) < tmz; });
        shiftUp(s.sTMin, s.sMask, s.sNode, i, k);
        if (lane == 0) { s.sTMin[i - k] = tm; s.sMask[i - k] = dbits > 0xfu ? 0u : dbits; s.sNode[i - k] = nd; }
        __syncwarp();
    }
    for (uint32_t i = lane; i < stackSize; i += 32)
        out[size_t(blk) * kBlockStack + i] = StackEntry{s.sTMin[i], s.sMask[i], s.sNode[i]};
    if (lane == 0) sizes[blk] = stackSize;
}


// per-warp tile traversal state; S = sorted-stack capacity
// passing leaf slots buffered per warp as triangle ranges before they are expanded into the list
constexpr uint32_t kRanges = 128;

template <uint32_t S>
struct TileSmemT {
    SmemFrustum f;
    float tMin[S];
    uint32_t mask[S];
    uint32_t node[S];
    alignas(16) uint32_t buf[kChunk];
    uint32_t rStart[kRanges], rLen[kRanges];
};

// End of a streamed tile's list: every lane's list writes are visible device-wide before lane 0
// releases the last chunk's link as kNoChunk.
__device__ __forceinline__ void endStream(uint32_t* lastLink) {
    __threadfence();
    __syncwarp();
    if (laneId() == 0) asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(lastLink), "r"(kNoChunk) : "memory");
    __syncwarp();
}

struct Emitter {
    uint32_t* pool;
    uint32_t* chunkNext;
    uint32_t poolChunks;
    uint32_t* counters;
    uint32_t first, prev, bufCount, stored, total;
    bool dead;
    uint32_t rc; // ranges buffered in rStart/rLen
    // streamed tile (stream): published with its first chunk; list = its TileList, ready = the
    // launch's ready slots, gt = the global tile index the slot carries
    bool stream, published;
    TileList* list;
    uint32_t* ready;
    uint32_t* readyTail;
    uint32_t gt;

    // last: the list's final (partial) chunk
    __device__ void flush(uint32_t* buf, bool last = false) {
        __syncwarp();
        uint32_t c = 0;
        if (laneId() == 0) c = atomicAdd(&counters[0], 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= poolChunks) {
            if (laneId() == 0) atomicOr(&counters[1], kStatusPoolOverflow);
            dead = true;
            return;
        }
        const uint4 w = reinterpret_cast<const uint4*>(buf)[laneId()];
        reinterpret_cast<uint4*>(pool + size_t(c) * kChunk)[laneId()] = w;
        if (stream && (prev != kNoChunk || !last)) {
            // The chunk's entries and its pending link are visible device-wide before the chunk is
            // linked to its predecessor, or, the first chunk, before the tile is published with a
            // streaming TileList. (A list that fits one chunk is published at the end as usual.)
            if (laneId() == 0) chunkNext[c] = kChunkPending;
            __threadfence();
            __syncwarp();
            if (laneId() == 0) {
                if (prev != kNoChunk) {
                    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(chunkNext + prev), "r"(c) : "memory");
                } else {
                    *list = TileList{c, kCountStreaming};
                    __threadfence();
                    const uint32_t pos = atomicAdd(readyTail, 1u);
                    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(ready + pos), "r"(gt) : "memory");
                }
            }
            if (prev == kNoChunk) published = true;
        } else if (laneId() == 0) {
            if (prev != kNoChunk) chunkNext[prev] = c;
        }
        if (prev == kNoChunk) first = c;
        prev = c;
        stored += bufCount;
        bufCount = 0;
        __syncwarp();
    }

    // Records the triangle ranges of the passing leaf slots of one node, in slot order (leaf
    // slot k covers [tri[k], tri[k+1]) = words 25+k, 26+k of the node; v holds word l of the
    // node in lane l). The entries are written out later by expand(), in the same order.
    template <uint32_t S>
    __device__ void addLeaves(TileSmemT<S>& s, float v, uint32_t leaf) {
        const uint32_t lane = laneId(), k = lane & 3u;
        const uint32_t t0 = __float_as_uint(__shfl_sync(kFull, v, 25 + k));
        const uint32_t t1 = __float_as_uint(__shfl_sync(kFull, v, 26 + k));
        const bool on = lane < 4 && ((leaf >> k) & 1u);
        if (on && t1 <= t0) atomicOr(&counters[1], kStatusBadLeaf);
        const bool emit = on && t1 > t0;
        const uint32_t b = __ballot_sync(kFull, emit);
        if (rc + 4 > kRanges) expand(s);
        if (emit) {
            const uint32_t pos = rc + __popc(b & ((1u << lane) - 1u));
            s.rStart[pos] = t0;
            s.rLen[pos] = t1 - t0;
        }
        rc += __popc(b);
        __syncwarp();
    }

    // Expands the buffered ranges into list entries (through buf, flushed to the pool per
    // chunk), 32 ranges at a time: lane r holds range r's start and the exclusive prefix of
    // the lengths, and each entry finds its range by a binary search over the lanes.
    template <uint32_t S>
    __device__ void expand(TileSmemT<S>& s) {
        const uint32_t lane = laneId();
        for (uint32_t r0 = 0; r0 < rc && !dead; r0 += 32) {
            const uint32_t r = r0 + lane;
            const uint32_t len = r < rc ? s.rLen[r] : 0u;
            const uint32_t start = r < rc ? s.rStart[r] : 0u;
            uint32_t inc = len;
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, inc, o);
                if (lane >= o) inc += y;
            }
            const uint32_t n = __shfl_sync(kFull, inc, 31);
            const uint32_t excl = inc - len; // lanes past the last range hold n
            uint32_t done = 0;
            while (done < n && !dead) {
                const uint32_t m = min(n - done, kChunk - bufCount);
                for (uint32_t base = 0; base < m; base += 32) {
                    const uint32_t j = base + lane;
                    const uint32_t p = done + j;
                    uint32_t lo = 0;
#pragma unroll
                    for (uint32_t step = 16; step; step >>= 1) {
                        const uint32_t e = __shfl_sync(kFull, excl, lo + step);
                        if (e <= p) lo += step;
                    }
                    const uint32_t st = __shfl_sync(kFull, start, lo);
                    const uint32_t pre = __shfl_sync(kFull, excl, lo);
                    if (j < m) s.buf[bufCount + j] = st + (p - pre);
                }
                bufCount += m;
                done += m;
                total += m;
                if (bufCount == kChunk) flush(s.buf);
            }
        }
        rc = 0;
        __syncwarp();
    }
};

struct TileCullArgs {
    const ViewDev* views;
    const uint32_t* blockView;
    uint32_t viewCount;
    uint32_t* pool;
    uint32_t* chunkNext;
    uint32_t poolChunks;
    uint32_t* counters;    // [0] chunk allocator, [1] status
    const uint32_t* order; // global tile order for the queue (nullptr = natural order)
    uint32_t first;        // this launch culls order[first, first + count)
    uint32_t count;
    uint32_t* queue;       // work-queue head of this launch, zero at launch
    uint32_t* retry;       // tiles whose stack outgrew kTileStack, at retry[first + i]
    uint32_t* retryCount;  // number of such tiles, zero at launch
    uint32_t* retryQueue;  // work-queue head of the retry pass, zero at launch
    uint32_t stackLimit;   // entries the main pass may use (<= kTileStack)
    uint32_t* ready;       // pipelined: ready slots, slot first + i for the i-th finished tile (else nullptr)
    uint32_t* readyTail;   // pipelined: finished tiles so far, zero at launch
    uint32_t persistent;   // 0: every warp culls one tile (the grid has a warp per tile), then exits
    uint32_t streamTiles;  // with ready: queue positions below this stream their lists (else 0)
};

// traverseTiles for one tile of view V (tile = view-local index); returns the node visits.
// overflow: the sorted stack needed more than S entries; the tile's list is left empty.
template <uint32_t S>
__device__ uint32_t cullTile(const TileCullArgs& a, const ViewDev& V, uint32_t tile, TileSmemT<S>& s,
                             bool& overflow, bool stream = false, uint32_t gt = 0, bool* published = nullptr) {
    overflow = false;
    const uint32_t lane = laneId();
    const Node* __restrict__ nodes = V.nodes;
    const uint32_t blk = tile / kTilesPerBlock;
    const uint32_t stackSize = V.blockSizes[blk];
    buildFrustum(V.tileRays[tile], V.M, s.f);
    if (V.hasCull && tileCulled(V.tileRays[tile], V.M, V.cull)) {
        if (lane == 0) V.tileLists[tile] = TileList{kNoChunk, 0};
        return 0;
    }
    if (stackSize == 0 || s.f.degenerate) {
        if (lane == 0) V.tileLists[tile] = TileList{kNoChunk, 0};
        return 0;
    }
    for (uint32_t i = lane; i < stackSize; i += 32) {
        const StackEntry e = V.blockStacks[size_t(blk) * kBlockStack + i];
        s.tMin[i] = e.tMin;
        s.mask[i] = e.mask;
        s.node[i] = e.node;
    }
    __syncwarp();
    const LaneTest t = loadLaneTest(s.f);
    const int distIdx = s.f.distIdx;
    Emitter em{a.pool, a.chunkNext, a.poolChunks, a.counters, kNoChunk, kNoChunk, 0, 0, 0, false, 0,
               stream && a.ready != nullptr, false, V.tileLists + tile, a.ready ? a.ready + a.first : nullptr,
               a.readyTail, gt};
    uint32_t top = stackSize - 1;
    uint32_t node = s.node[top];
    uint32_t visits = 0;
    const float* rows = reinterpret_cast<const float*>(nodes);
    float v = rows[size_t(node) * 32 + lane];
#ifdef HVVR_VISIT_CLOCKS
    long long vcAcc[kVcPhases] = {0, 0, 0, 0, 0, 0};
    long long vcLast = phaseClock(node);
#endif
    for (;;) {
        ++visits;
        // The next visit is always one of this node's internal children or the stack entry
        // below the current one (a pop, or a push whose children all sort below it), so their
        // rows are loaded now and consumed at the end of the visit, hiding the load latency.
        const uint32_t leafMask = __float_as_uint(__shfl_sync(kFull, v, 24));
        VISIT_MARK(kVcRow, leafMask);
        uint32_t childNode[4];
        float vc[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            childNode[k] = node + __float_as_uint(__shfl_sync(kFull, v, 26 + k));
            vc[k] = ((leafMask >> k) & 1u) ? 0.0f : rows[size_t(childNode[k]) * 32 + lane];
        }
        const bool hasPop = top > 0;
        const uint32_t popNode = hasPop ? s.node[top - 1] : 0u;
        const float vp = hasPop ? rows[size_t(popNode) * 32 + lane] : 0.0f;
        const ChildBox cb = childBox(v);
        uint32_t mask = testChildren(cb, t);
        VISIT_MARK(kVcTest, mask);
        if (mask) {
            uint32_t leaf = mask & leafMask;
            if (leaf) {
                mask &= ~refineReject(cb, t);
                leaf = mask & leafMask;
                if (leaf) em.addLeaves(s, v, leaf);
                VISIT_MARK(kVcLeaf, em.rc);
                if (em.dead) break;
            }
            mask &= ~leafMask;
            if (mask && s.mask[top] == 0u) {
                int k = __ffs(mask) - 1;
                if (!(mask & (mask - 1))) {
                    // (child indices by shuffle: a register array indexed at run time would live
                    // in local memory)
                    node = node + __float_as_uint(__shfl_sync(kFull, v, 26 + k));
                    v = vc[0];
#pragma unroll
                    for (int q = 1; q < 4; q++)
                        if (q == k) v = vc[q];
                    VISIT_MARK(kVcNext, node);
                    continue;
                }
                // Insert all m >= 2 children at once. Keys are never NaN (a child that passes the
                // plane test has finite bounds), so the stack stays sorted, non-increasing from
                // bottom to top under the DAZ comparison, and the reference's one-at-a-time
                // insertion (shift entries with a smaller key up, place the child, newest above
                // equal keys) is equivalent to: an old entry moves up by the number of children
                // with a larger key; child i lands at
                //   top - #{old < key_i} + #{children with a larger key}
                //       + #{earlier children with an equal key}.
                const uint32_t m = __popc(mask);
                if (top + m >= (S == kTileStack ? a.stackLimit : S)) {
                    overflow = true;
                    break;
                }
                // the children in slot order (bit i of mask: child i is inserted); the reference
                // inserts them in slot order, so "earlier" in the tie rule is the earlier slot
                float ck[4], ckz[4];
                float maxKey = -INFINITY, minKey = INFINITY;
                uint32_t kmin = 0;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    ck[i] = __uint_as_float(__float_as_uint(__shfl_sync(kFull, v, distIdx * 4 + i)) ^ 0x80000000u);
                    ckz[i] = dazf(ck[i]);
                    if ((mask >> i) & 1u) {
                        maxKey = fmaxf(maxKey, ckz[i]);
                        if (ckz[i] <= minKey) { minKey = ckz[i]; kmin = uint32_t(i); }
                    }
                }
                // old entries that move: those with a key below the largest child key (a top run).
                // Lane j holds entry top-1-j of a group of 32; the first group is read once both
                // to find the run and to move it, and the run continues into later groups only
                // when all 32 of the first move.
                uint32_t less[4] = {0u, 0u, 0u, 0u};
                auto moveGroup = [&](uint32_t j, bool act, float e, float ez, uint32_t em_, uint32_t en) {
                    const uint32_t p = top - 1 - j;
                    uint32_t d = 0;
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const bool valid = (mask >> i) & 1u;
                        d += (act && valid && ckz[i] > ez) ? 1u : 0u;
                        less[i] += __popc(__ballot_sync(kFull, act && valid && ez < ckz[i]));
                    }
                    __syncwarp();
                    if (act && d) { s.tMin[p + d] = e; s.mask[p + d] = em_; s.node[p + d] = en; }
                    __syncwarp();
                };
                uint32_t region;
                float oldTopKey; // key of the entry below the current one (when there is one)
                {
                    const bool inb = lane < top;
                    float e = 0.0f, ez = 0.0f;
                    uint32_t em_ = 0, en = 0;
                    if (inb) {
                        const uint32_t p = top - 1 - lane;
                        e = s.tMin[p]; em_ = s.mask[p]; en = s.node[p]; ez = dazf(e);
                    }
                    oldTopKey = __shfl_sync(kFull, ez, 0);
                    const uint32_t b = __ballot_sync(kFull, inb && ez < maxKey);
                    region = (b == kFull) ? 32u : uint32_t(__ffs(~b) - 1);
                    moveGroup(lane, lane < region, e, ez, em_, en);
                    if (region == 32u && top > 32u)
                        region = 32u + shiftCount(top - 32u, [&](uint32_t p) { return dazf(s.tMin[p]) < maxKey; });
                }
                for (uint32_t base = 32; base < region; base += 32) {
                    const uint32_t j = base + lane;
                    const bool act = j < region;
                    float e = 0.0f, ez = 0.0f;
                    uint32_t em_ = 0, en = 0;
                    if (act) { const uint32_t p = top - 1 - j; e = s.tMin[p]; em_ = s.mask[p]; en = s.node[p]; ez = dazf(e); }
                    moveGroup(j, act, e, ez, em_, en);
                }
                if ((mask >> lane) & 1u) { // lanes 0-3, one per inserted child
                    uint32_t pos = top - less[0];
                    float mine = ckz[0];
                    float rawk = ck[0];
                    uint32_t nd = childNode[0];
#pragma unroll
                    for (int i = 1; i < 4; i++)
                        if (uint32_t(i) == lane) { pos = top - less[i]; mine = ckz[i]; rawk = ck[i]; nd = childNode[i]; }
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        if (!((mask >> i) & 1u) || uint32_t(i) == lane) continue;
                        if (ckz[i] > mine || (ckz[i] == mine && uint32_t(i) < lane)) pos++;
                    }
                    s.tMin[pos] = rawk;
                    s.mask[pos] = 0u;
                    s.node[pos] = nd;
                }
                __syncwarp();
                const bool popNext = hasPop && oldTopKey < minKey;
                top += m - 1;
                VISIT_MARK(kVcInsert, top);
                // The new top entry is the next node: the old entry below the current one when its
                // key is below every child's (it moved up by m), else the child with the smallest
                // key, the last slot among equal ones (an old entry with an equal key stays below it).
                if (popNext) {
                    node = popNode;
                    v = vp;
                } else {
                    node = childNode[0];
                    v = vc[0];
#pragma unroll
                    for (uint32_t q = 1; q < 4; q++)
                        if (q == kmin) { node = childNode[q]; v = vc[q]; }
                }
                VISIT_MARK(kVcNext, node);
                continue;
            }
        }
        if (top == 0) break;
        --top;
        node = popNode;
        v = vp;
        VISIT_MARK(kVcNext, node);
    }
#ifdef HVVR_VISIT_CLOCKS
    vcLast = phaseClock(top);
#endif
    if (overflow) {
        // (a streamed tile's shade ends its chunk walk here; the retry passes cull and shade the
        // tile again after it)
        if (published) *published = em.published;
        if (em.published) endStream(a.chunkNext + em.prev);
        if (lane == 0) V.tileLists[tile] = TileList{kNoChunk, 0};
        return visits;
    }
    if (!em.dead && em.rc) em.expand(s);
    if (em.published && !em.dead && em.bufCount) {
        // a streamed list's last chunk: its unused entries say so
        for (uint32_t i = em.bufCount + lane; i < kChunk; i += 32) s.buf[i] = kNoTriangle;
        __syncwarp();
    }
    if (!em.dead && em.bufCount) em.flush(s.buf, true);
    // (after the last expansion, whose full chunks may have published the tile)
    if (published) *published = em.published;
    if (em.published) {
        // the last chunk's end-of-list link, then the complete TileList, each after what precedes it
        endStream(a.chunkNext + em.prev);
        if (lane == 0) {
            __threadfence();
            const unsigned long long l =
                uint64_t(em.first) | (uint64_t(em.dead ? em.stored : em.total) << 32);
            asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(V.tileLists + tile), "l"(l) : "memory");
        }
    } else if (lane == 0) {
        if (em.prev != kNoChunk) a.chunkNext[em.prev] = kNoChunk;
        V.tileLists[tile] = TileList{em.first, em.dead ? em.stored : em.total};
    }
#ifdef HVVR_VISIT_CLOCKS
    VISIT_MARK(kVcTail, em.total);
    if (lane == 0 && V.tileStart + tile < kVisitClockTiles) {
        for (uint32_t k = 0; k < kVcPhases; k++) gVisitClocks[V.tileStart + tile][k] = uint64_t(vcAcc[k]);
        gVisitClocks[V.tileStart + tile][kVcPhases] = visits;
    }
#endif
    return visits;
}

// Persistent warps pull tiles from a queue (longest-first when an order is given), so a
// few long horizon tiles overlap with the rest instead of holding a CTA slot each. Non-persistent
// (a.persistent == 0): the grid has a warp per tile and each warp takes one tile from the same
// queue, so the tiles still start longest-first and every CTA ends with its tile.
// (W = 1: one warp per CTA, so a warp that runs out of tiles frees its registers at once; the
// bound asks for the 20 resident warps per SM that the wider CTAs reach)
template <int W>
__global__ void __launch_bounds__(W * 32, W == 1 ? 20 : 1) tileCullKernel(TileCullArgs a) {
    __shared__ TileSmemT<kTileStack> smem[W];
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    TileSmemT<kTileStack>& s = smem[warp];
    // A launch that follows this one with programmatic serialization (the pipelined shade) may be
    // scheduled once every CTA of this grid has started: its CTAs wait for tiles that only this
    // grid's warps publish, so they must never keep a cull CTA from becoming resident.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    for (;;) {
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(a.queue, 1u);
        w = __shfl_sync(kFull, w, 0);
        if (w >= a.count) return;
        const uint32_t gt = a.order ? a.order[a.first + w] : a.first + w;
        const ViewDev& V = viewOfBlock(a.views, a.blockView, a.viewCount, gt / kTilesPerBlock);
        const uint32_t tile = gt - V.tileStart;
        __syncwarp();
        bool overflow, published = false;
        const uint32_t visits = cullTile(a, V, tile, s, overflow, w < a.streamTiles, gt, &published);
        if (lane == 0) {
            V.tileCost[tile] = visits;
            if (overflow) a.retry[a.first + atomicAdd(a.retryCount, 1u)] = gt;
        }
        if (a.ready && !published) {
            // publish: every lane's list writes (pool chunks, links, the tile's TileList) are made
            // visible device-wide before lane 0 releases the slot
            __threadfence();
            __syncwarp();
            if (lane == 0) {
                const uint32_t pos = atomicAdd(a.readyTail, 1u);
                const uint32_t val = gt | (overflow ? kReadyRetry : 0u);
                asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.ready + a.first + pos), "r"(val) : "memory");
            }
        }
        __syncwarp();
        if (!a.persistent) return;
    }
}

// The tiles whose sorted stack outgrew kTileStack, culled again from the start with the
// reference's TileFrame capacity (4096 entries, 48 KiB of shared memory per warp).
constexpr uint32_t kRetryStack = 4096;
__global__ void __launch_bounds__(32) tileCullRetryKernel(TileCullArgs a) {
    extern __shared__ __align__(16) unsigned char retrySmem[];
    TileSmemT<kRetryStack>& s = *reinterpret_cast<TileSmemT<kRetryStack>*>(retrySmem);
    const uint32_t lane = laneId();
    for (;;) {
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(a.retryQueue, 1u);
        w = __shfl_sync(kFull, w, 0);
        if (w >= *reinterpret_cast<volatile uint32_t*>(a.retryCount)) return;
        const uint32_t gt = a.retry[a.first + w];
        const ViewDev& V = viewOfBlock(a.views, a.blockView, a.viewCount, gt / kTilesPerBlock);
        const uint32_t tile = gt - V.tileStart;
        __syncwarp();
        bool overflow;
        const uint32_t visits = cullTile(a, V, tile, s, overflow);
        if (lane == 0) {
            V.tileCost[tile] = visits;
            if (overflow) atomicOr(&a.counters[1], kStatusStackOverflow);
        }
        __syncwarp();
    }
}

// Orders the global tiles by (rate class ascending, cost descending), cost in log2 buckets
// of last frame's visit counts. One block; positions within a bucket are in arrival order.
constexpr uint32_t kOrderBuckets = kRateClasses * 33;
__global__ void __launch_bounds__(1024) tileOrderKernel(FrameDev fr) {
    __shared__ uint32_t hist[kOrderBuckets];
    __shared__ uint32_t start[kOrderBuckets];
    for (uint32_t b = threadIdx.x; b < kOrderBuckets; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    auto bucket = [&](uint32_t t) {
        const ViewDev& V = viewOfBlock(fr.views, fr.blockView, fr.viewCount, t / kTilesPerBlock);
        const uint32_t c = V.tileCost[t - V.tileStart];
        return V.rateIdx * 33u + uint32_t(__clz(c + 1u)); // clz falls as the cost grows
    };
    for (uint32_t t = threadIdx.x; t < fr.tiles; t += blockDim.x) atomicAdd(&hist[bucket(t)], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t b = 0; b < kOrderBuckets; b++) {
            start[b] = run;
            run += hist[b];
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < fr.tiles; t += blockDim.x) fr.order[atomicAdd(&start[bucket(t)], 1u)] = t;
}

__global__ void writeViewKernel(ViewDev v, ViewDev* dst) { *dst = v; }

// The reference runs its intersect and resolve kernels over the compacted list of occupied tiles
// (tileIndexRemapOccupied, libraries/hvvr/raycaster/traversal.cpp:213-330) and indexes the lens
// table by that CTA index; this is each tile's rank among the view's non-empty tiles.
__global__ void __launch_bounds__(1024) occupiedRankKernel(FrameDev fr) {
    const ViewDev& V = fr.views[blockIdx.x];
    if (!(V.lensRadius > 0.0f)) return;
    __shared__ uint32_t warpSums[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const uint32_t lane = laneId(), warp = threadIdx.x >> 5;
    const uint32_t tiles = (blockIdx.x + 1 < fr.viewCount ? fr.views[blockIdx.x + 1].tileStart : fr.tiles) - V.tileStart;
    for (uint32_t base = 0; base < tiles; base += 1024) {
        const uint32_t t = base + threadIdx.x;
        const uint32_t occ = (t < tiles && V.tileLists[t].count > 0) ? 1u : 0u;
        const uint32_t bal = __ballot_sync(kFull, occ);
        if (lane == 0) warpSums[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = carry;
        for (uint32_t w = 0; w < warp; w++) before += warpSums[w];
        if (t < tiles) V.occRank[t] = before + __popc(bal & ((1u << lane) - 1u));
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t sum = 0;
            for (uint32_t w = 0; w < 32; w++) sum += warpSums[w];
            carry += sum;
        }
        __syncthreads();
    }
}

struct DeviceLimits {
    int sms = 0;
    int ctasPerSm[9] = {};  // indexed by warps per CTA
    bool retryReady = false;
};

// per-device launch limits, filled on first use; host threads rendering on different streams
// may get here together, so the first use of a device is serialised
std::mutex gLimitsMutex;

DeviceLimits& limits() {
    static DeviceLimits perDevice[64];
    int dev = 0;
    cudaGetDevice(&dev);
    DeviceLimits& d = perDevice[dev < 0 || dev >= 64 ? 0 : dev];
    std::lock_guard<std::mutex> lock(gLimitsMutex);
    if (!d.sms) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        d.sms = sms < 1 ? 1 : sms;
    }
    return d;
}

template <int W>
cudaError_t launchTileCullW(const TileCullArgs& a, uint32_t count, uint32_t capPerSm, cudaStream_t st) {
    if (!a.persistent) {
        tileCullKernel<W><<<(count + W - 1) / W, W * 32, 0, st>>>(a);
        return cudaGetLastError();
    }
    DeviceLimits& d = limits();
    {
        std::lock_guard<std::mutex> lock(gLimitsMutex);
        if (!d.ctasPerSm[W]) {
            int occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, tileCullKernel<W>, W * 32, 0);
            d.ctasPerSm[W] = occ < 1 ? 1 : occ;
        }
    }
    const uint32_t needed = (count + W - 1) / W;
    const uint32_t perSm = capPerSm ? std::min<uint32_t>(capPerSm, uint32_t(d.ctasPerSm[W])) : uint32_t(d.ctasPerSm[W]);
    const uint32_t grid = std::min<uint32_t>(needed, uint32_t(d.sms) * perSm);
    tileCullKernel<W><<<grid, W * 32, 0, st>>>(a);
    return cudaGetLastError();
}

// the retry pass: one warp per CTA, one CTA per SM; it reads the retry count on the device and
// exits at once when no tile overflowed
cudaError_t launchTileCullRetry(const TileCullArgs& a, cudaStream_t st) {
    DeviceLimits& d = limits();
    const size_t smem = sizeof(TileSmemT<kRetryStack>);
    {
        std::lock_guard<std::mutex> lock(gLimitsMutex);
        if (!d.retryReady) {
            const cudaError_t e =
                cudaFuncSetAttribute(tileCullRetryKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (e != cudaSuccess) return e;
            d.retryReady = true;
        }
    }
    tileCullRetryKernel<<<d.sms, 32, smem, st>>>(a);
    return cudaGetLastError();
}

} // namespace

cudaError_t launchBlockCull(const FrameDev& fr, cudaStream_t st) {
    if (fr.blocks == 0) return cudaSuccess;
    blockCullKernel<<<(fr.blocks + kBlockWarps - 1) / kBlockWarps + kPrefetchCtas, kBlockWarps * 32, 0, st>>>(fr);
    return cudaGetLastError();
}

cudaError_t launchTileOrder(const FrameDev& fr, cudaStream_t st) {
    if (fr.tiles == 0) return cudaSuccess;
    tileOrderKernel<<<1, 1024, 0, st>>>(fr);
    return cudaGetLastError();
}

cudaError_t launchTileCullMain(const FrameDev& fr, const uint32_t* order, uint32_t first, uint32_t count,
                               uint32_t* queues, uint32_t warps, uint32_t stackLimit, uint32_t* ready,
                               uint32_t* readyTail, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    if (stackLimit == 0 || stackLimit > kTileStack) stackLimit = kTileStack;
    if (stackLimit < 8) return cudaErrorInvalidValue;
    const TileCullArgs a{fr.views, fr.blockView, fr.viewCount, fr.pool, fr.chunkNext, fr.poolChunks, fr.counters,
                         order, first, count, queues, fr.retry, queues + 1, queues + 2, stackLimit, ready, readyTail,
                         fr.cullPersistent ? 1u : 0u, ready ? fr.streamTiles : 0u};
    switch (warps) {
    case 1: return launchTileCullW<1>(a, count, fr.cullCtasPerSm, st);
    case 2: return launchTileCullW<2>(a, count, fr.cullCtasPerSm, st);
    case 4: return launchTileCullW<4>(a, count, fr.cullCtasPerSm, st);
    case 8: return launchTileCullW<8>(a, count, fr.cullCtasPerSm, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launchTileCullRetryPass(const FrameDev& fr, const uint32_t* order, uint32_t first, uint32_t count,
                                    uint32_t* queues, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    const TileCullArgs a{fr.views, fr.blockView, fr.viewCount, fr.pool, fr.chunkNext, fr.poolChunks, fr.counters,
                         order, first, count, queues, fr.retry, queues + 1, queues + 2, kTileStack, nullptr, nullptr, 1u,
                         0u};
    return launchTileCullRetry(a, st);
}

cudaError_t launchTileCull(const FrameDev& fr, const uint32_t* order, uint32_t first, uint32_t count,
                           uint32_t* queues, uint32_t warps, uint32_t stackLimit, cudaStream_t st) {
    const cudaError_t e = launchTileCullMain(fr, order, first, count, queues, warps, stackLimit, nullptr, nullptr, st);
    if (e != cudaSuccess) return e;
    return launchTileCullRetryPass(fr, order, first, count, queues, st);
}

cudaError_t launchOccupiedRank(const FrameDev& fr, cudaStream_t st) {
    if (fr.viewCount == 0) return cudaSuccess;
    occupiedRankKernel<<<fr.viewCount, 1024, 0, st>>>(fr);
    return cudaGetLastError();
}

cudaError_t launchWriteView(const ViewDev& v, ViewDev* dst, cudaStream_t st) {
    writeViewKernel<<<1, 1, 0, st>>>(v, dst);
    return cudaGetLastError();
}

} // namespace hvb

#ifdef HVVR_VISIT_CLOCKS
// profiling build only: per global tile [0, tiles), kVcPhases phase cycle sums then the visit count
extern "C" int hvvr_dbg_visit_clocks(unsigned long long* out, uint32_t tiles) {
    if (!out || tiles > hvb::kVisitClockTiles) return HVVR_ERR_INVALID;
    return cudaMemcpyFromSymbol(out, hvb::gVisitClocks, size_t(tiles) * sizeof(hvb::gVisitClocks[0])) == cudaSuccess
               ? HVVR_OK
               : HVVR_ERR_CUDA;
}
#endif
