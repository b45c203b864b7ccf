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
#include "dev_common.cuh"

namespace hvb {

namespace {

constexpr unsigned kFull = 0xffffffffu;

struct SmemFrustum {
    float tpLo[4][3], tpHi[4][3], w[4];
    float proj[3][8];
    float edge[12][3];
    float minF[12], maxF[12];
    int distIdx;
    int degenerate;
};

struct LaneTest {
    float c0, c1, c2, c3, c4, c5, c6;  // plane lanes: lo xyz, hi xyz, w; projection lanes: max, -min
    bool always;                       // projection lanes 28-31 (no axis)
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

__device__ LaneTest loadLaneTest(const SmemFrustum& f) {
    LaneTest t;
    const uint32_t lane = laneId();
    if (lane < 16) {
        const int p = int(lane >> 2);
        t.c0 = f.tpLo[p][0]; t.c1 = f.tpLo[p][1]; t.c2 = f.tpLo[p][2];
        t.c3 = f.tpHi[p][0]; t.c4 = f.tpHi[p][1]; t.c5 = f.tpHi[p][2];
        t.c6 = f.w[p];
        t.always = false;
    } else {
        const int a = int(lane - 16) >> 2, c = int(lane & 3);
        t.always = (a == 3);
        t.c0 = a < 3 ? f.proj[a][c] : 0.0f;
        t.c1 = a < 3 ? f.proj[a][4 + c] : 0.0f;
        t.c2 = t.c3 = t.c4 = t.c5 = t.c6 = 0.0f;
    }
    const int e0 = int(lane >> 2);
    t.e0x = f.edge[e0][0]; t.e0y = f.edge[e0][1]; t.e0z = f.edge[e0][2];
    t.mn0 = f.minF[e0]; t.mx0 = f.maxF[e0];
    t.has1 = lane < 16;
    const int e1 = t.has1 ? 8 + int(lane >> 2) : e0;
    t.e1x = f.edge[e1][0]; t.e1y = f.edge[e1][1]; t.e1z = f.edge[e1][2];
    t.mn1 = f.minF[e1]; t.mx1 = f.maxF[e1];
    return t;
}

struct ChildBox {
    float xM, xN, yM, yN, zM, zN;
};

__device__ __forceinline__ ChildBox childBox(float v) {
    const uint32_t c = laneId() & 3u;
    ChildBox b;
    b.xM = __shfl_sync(kFull, v, c);
    b.xN = __shfl_sync(kFull, v, 4 + c);
    b.yM = __shfl_sync(kFull, v, 8 + c);
    b.yN = __shfl_sync(kFull, v, 12 + c);
    b.zM = __shfl_sync(kFull, v, 16 + c);
    b.zN = __shfl_sync(kFull, v, 20 + c);
    return b;
}

// Frustum::testBVHNodeChildren (traverse_avx.h:104-164)
__device__ __forceinline__ uint32_t testChildren(const ChildBox& b, const LaneTest& t) {
    const uint32_t lane = laneId();
    bool pass;
    if (lane < 16) {
        const float lo = fmaf(t.c0, b.xM, fmaf(t.c1, b.yM, t.c2 * b.zM));
        const float hi = fmaf(t.c3, b.xN, fmaf(t.c4, b.yN, t.c5 * b.zN));
        pass = (lo + hi) <= t.c6;
    } else {
        const int a = int(lane - 16) >> 2;
        const float am = a == 0 ? b.xM : (a == 1 ? b.yM : b.zM);
        const float an = a == 0 ? b.xN : (a == 1 ? b.yN : b.zN);
        pass = t.always || (am >= t.c0 && an >= t.c1);
    }
    const uint32_t m = __ballot_sync(kFull, pass);
    return (m & (m >> 4) & (m >> 8) & (m >> 12) & (m >> 16) & (m >> 20) & (m >> 24) & (m >> 28)) & 0xfu;
}

__device__ __forceinline__ bool edgeReject(const ChildBox& b, float ex, float ey, float ez, float mn, float mx) {
    const bool px = ex > 0.0f, py = ey > 0.0f, pz = ez > 0.0f;
    const float pX = (px ? b.xM : -b.xN) + 0.0f, nX = (px ? -b.xN : b.xM) + 0.0f;
    const float pY = (py ? b.yM : -b.yN) + 0.0f, nY = (py ? -b.yN : b.yM) + 0.0f;
    const float pZ = (pz ? b.zM : -b.zN) + 0.0f, nZ = (pz ? -b.zN : b.zM) + 0.0f;
    const float maxBox = fmaf(ex, pX, fmaf(ey, pY, ez * pZ));
    const float minBox = fmaf(ex, nX, fmaf(ey, nY, ez * nZ));
    return (maxBox < mn) || (mx < minBox);
}

// Frustum::testBVHNodeChildrenRefine (traverse_avx.h:166-217): mask of rejected children
__device__ __forceinline__ uint32_t refineReject(const ChildBox& b, const LaneTest& t) {
    bool rej = edgeReject(b, t.e0x, t.e0y, t.e0z, t.mn0, t.mx0);
    if (t.has1) rej = rej || edgeReject(b, t.e1x, t.e1y, t.e1z, t.mn1, t.mx1);
    const uint32_t m = __ballot_sync(kFull, rej);
    return (m | (m >> 4) | (m >> 8) | (m >> 12) | (m >> 16) | (m >> 20) | (m >> 24) | (m >> 28)) & 0xfu;
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

__global__ void __launch_bounds__(kBlockWarps * 32) blockCullKernel(const Node* __restrict__ nodes,
                                                                    const Rays4* __restrict__ blockRays,
                                                                    uint32_t blocks, Mat4 M,
                                                                    StackEntry* __restrict__ out,
                                                                    uint32_t* __restrict__ sizes) {
    __shared__ BlockSmem smem[kBlockWarps];
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    const uint32_t blk = blockIdx.x * kBlockWarps + warp;
    if (blk >= blocks) return;
    BlockSmem& s = smem[warp];
    buildFrustum(blockRays[blk], M, s.f);
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

constexpr int kTileWarps = 8;

struct TileSmem {
    SmemFrustum f;
    float tMin[kTileStack];
    uint32_t mask[kTileStack];
    uint32_t node[kTileStack];
    alignas(16) uint32_t buf[kChunk];
};

struct Emitter {
    uint32_t* pool;
    uint32_t* chunkNext;
    uint32_t poolChunks;
    uint32_t* counters;
    uint32_t first, prev, bufCount, stored, total;
    bool dead;

    __device__ void flush(uint32_t* buf) {
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
        if (laneId() == 0) {
            if (prev != kNoChunk) chunkNext[prev] = c;
        }
        if (prev == kNoChunk) first = c;
        prev = c;
        stored += bufCount;
        bufCount = 0;
        __syncwarp();
    }

    __device__ void emitRange(uint32_t* buf, uint32_t t0, uint32_t t1) {
        if (t1 <= t0) {
            if (laneId() == 0) atomicOr(&counters[1], kStatusBadLeaf);
            return;
        }
        uint32_t n = t1 - t0;
        while (n && !dead) {
            const uint32_t m = min(n, kChunk - bufCount);
            for (uint32_t j = laneId(); j < m; j += 32) buf[bufCount + j] = t0 + j;
            bufCount += m;
            t0 += m;
            n -= m;
            total += m;
            if (bufCount == kChunk) flush(buf);
        }
    }
};

__global__ void __launch_bounds__(kTileWarps * 32) tileCullKernel(const Node* __restrict__ nodes,
                                                                  const Rays4* __restrict__ tileRays, uint32_t tiles,
                                                                  Mat4 M, const StackEntry* __restrict__ blockStacks,
                                                                  const uint32_t* __restrict__ blockSizes,
                                                                  TileList* __restrict__ lists, uint32_t* pool,
                                                                  uint32_t* chunkNext, uint32_t poolChunks,
                                                                  uint32_t* counters) {
    __shared__ TileSmem smem[kTileWarps];
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    const uint32_t tile = blockIdx.x * kTileWarps + warp;
    if (tile >= tiles) return;
    TileSmem& s = smem[warp];
    const uint32_t blk = tile / kTilesPerBlock;
    const uint32_t stackSize = blockSizes[blk];
    buildFrustum(tileRays[tile], M, s.f);
    if (stackSize == 0 || s.f.degenerate) {
        if (lane == 0) lists[tile] = TileList{kNoChunk, 0};
        return;
    }
    for (uint32_t i = lane; i < stackSize; i += 32) {
        const StackEntry e = blockStacks[size_t(blk) * kBlockStack + i];
        s.tMin[i] = e.tMin;
        s.mask[i] = e.mask;
        s.node[i] = e.node;
    }
    __syncwarp();
    const LaneTest t = loadLaneTest(s.f);
    const int distIdx = s.f.distIdx;
    Emitter em{pool, chunkNext, poolChunks, counters, kNoChunk, kNoChunk, 0, 0, 0, false};
    uint32_t top = stackSize - 1;
    uint32_t node = s.node[top];
    for (;;) {
        const float v = reinterpret_cast<const float*>(nodes + node)[lane];
        const ChildBox cb = childBox(v);
        uint32_t mask = testChildren(cb, t);
        bool descend = false;
        if (mask) {
            const uint32_t leafMask = __float_as_uint(__shfl_sync(kFull, v, 24));
            uint32_t leaf = mask & leafMask;
            if (leaf) {
                mask &= ~refineReject(cb, t);
                leaf = mask & leafMask;
                while (leaf && !em.dead) {
                    const int k = __ffs(leaf) - 1;
                    const uint32_t t0 = __float_as_uint(__shfl_sync(kFull, v, 25 + k));
                    const uint32_t t1 = __float_as_uint(__shfl_sync(kFull, v, 26 + k));
                    em.emitRange(s.buf, t0, t1);
                    leaf &= leaf - 1;
                }
                if (em.dead) break;
            }
            mask &= ~leafMask;
            if (mask && s.mask[top] == 0u) {
                int k = __ffs(mask) - 1;
                if (!(mask & (mask - 1))) {
                    node = node + __float_as_uint(__shfl_sync(kFull, v, 26 + k));
                    continue;
                }
                bool first = true;
                bool overflow = false;
                while (mask) {
                    if (!first) ++top;
                    first = false;
                    if (top + 1 >= kTileStack) { overflow = true; break; }
                    k = __ffs(mask) - 1;
                    const float tm = __uint_as_float(__float_as_uint(__shfl_sync(kFull, v, distIdx * 4 + k)) ^ 0x80000000u);
                    const uint32_t child = node + __float_as_uint(__shfl_sync(kFull, v, 26 + k));
                    const float tmz = dazf(tm);
                    const uint32_t n = shiftCount(top, [&](uint32_t p) { return dazf(s.tMin[p]) < tmz; });
                    shiftUp(s.tMin, s.mask, s.node, top, n);
                    if (lane == 0) { s.tMin[top - n] = tm; s.mask[top - n] = 0u; s.node[top - n] = child; }
                    __syncwarp();
                    mask &= mask - 1;
                }
                if (overflow) {
                    if (lane == 0) atomicOr(&counters[1], kStatusStackOverflow);
                    break;
                }
                descend = true;
            }
        }
        if (descend) {
            node = s.node[top];
            continue;
        }
        if (top == 0) break;
        --top;
        node = s.node[top];
    }
    if (!em.dead && em.bufCount) em.flush(s.buf);
    if (lane == 0) {
        if (em.prev != kNoChunk) chunkNext[em.prev] = kNoChunk;
        lists[tile] = TileList{em.first, em.dead ? em.stored : em.total};
    }
}

} // namespace

cudaError_t launchBlockCull(const SceneDev& s, const CameraDev& c, const FrameParams& f, cudaStream_t st) {
    if (c.blocks == 0) return cudaSuccess;
    const uint32_t grid = (c.blocks + kBlockWarps - 1) / kBlockWarps;
    blockCullKernel<<<grid, kBlockWarps * 32, 0, st>>>(s.nodes, c.blockRays, c.blocks, f.cameraToWorld, c.blockStacks,
                                                        c.blockSizes);
    return cudaGetLastError();
}

cudaError_t launchTileCull(const SceneDev& s, const CameraDev& c, const FrameParams& f, cudaStream_t st) {
    if (c.tiles == 0) return cudaSuccess;
    const uint32_t grid = (c.tiles + kTileWarps - 1) / kTileWarps;
    tileCullKernel<<<grid, kTileWarps * 32, 0, st>>>(s.nodes, c.tileRays, c.tiles, f.cameraToWorld, c.blockStacks,
                                                      c.blockSizes, c.tileLists, c.pool, c.chunkNext, c.poolChunks,
                                                      c.counters);
    return cudaGetLastError();
}

} // namespace hvb
