// hvvr_internal.h - device data layouts and kernel launch interfaces shared by the host
// driver (raycaster.cpp) and the CUDA kernels (*.cu). Not part of the public ABI.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime.h>

namespace hvb {

// Sample hierarchy constants (TILE_SIZE, TILES_PER_BLOCK, BLOCK_SIZE in
// libraries/hvvr/raycaster/raycaster_common.h:17-20)
enum : uint32_t { kTileSize = 128, kTilesPerBlock = 64, kBlockSize = kTileSize * kTilesPerBlock };
// block cull stack capacity (BlockFrame::stackSize, libraries/hvvr/raycaster/traverse_avx.h:255)
enum : uint32_t { kBlockStack = 64 };
// per-warp tile traversal stack in shared memory; the reference's TileFrame holds 4096
// entries, but a stack deeper than this needs a BVH deeper than ~60 levels. Overflow sets
// kStatusStackOverflow and stops that tile instead of writing out of bounds.
enum : uint32_t { kTileStack = 256 };
// triangle indices move between traversal and intersection in chunks of one intersect batch
enum : uint32_t { kChunk = 128 };
enum : uint32_t { kNoChunk = 0xffffffffu };

// device status bits (OR-ed into a per-frame word)
enum : uint32_t {
    kStatusPoolOverflow = 1u,   // triangle-index pool exhausted
    kStatusStackOverflow = 2u,  // tile traversal stack exhausted
    kStatusBadLeaf = 4u,        // a passing leaf had an empty/inverted triangle range
    kStatusRefitTimeout = 8u,   // refit walked more levels than the tree has
};

// BVHNode (libraries/hvvr/raycaster/bvh_node.h:17-36), 128 bytes
struct alignas(128) Node {
    float b[6][4];    // xMax, xNegMin, yMax, yNegMin, zMax, zNegMin
    uint32_t leafMask;
    uint32_t tri[5];  // leaf.triIndex[5]; children.offset[k] aliases tri[k+1]
    uint32_t pad[2];
};
static_assert(sizeof(Node) == 128, "Node");

// Camera-space corner rays of a tile or block frustum (Frustum::pointOrigin/pointDir)
struct Rays4 {
    float o[4][3];
    float d[4][3];
};
static_assert(sizeof(Rays4) == 96, "Rays4");

// Sorted block stack entry (TileFrame::Entry without the pointer: node is an index)
struct StackEntry {
    float tMin;
    uint32_t mask;
    uint32_t node;
};

// per-tile triangle list: a chain of kChunk-entry chunks in the camera's pool
struct TileList {
    uint32_t first;  // first chunk, kNoChunk when empty
    uint32_t count;  // triangle index entries
};

struct Mat4 {
    float m[4][4];  // column-major: m[col][row], matching matrix4x4 {m0,m1,m2,m3}
};

struct LightEnvDev {
    int nd, np, ns, pad;
    float dir[1][6];     // direction xyz, power xyz
    float pt[4][8];      // position xyz, falloffEnd, color xyz, falloffScale
    float spot[4][13];   // position, falloffEnd, direction, falloffScale, color, cosOuter, cosScale
};

// scene state resident on the device
struct SceneDev {
    Node* nodes = nullptr;
    uint32_t nodeCount = 0;
    float4* tris = nullptr;          // 3 x float4 per triangle: v0.xyz e0.x | e0.yz e1.xy | e1.z
    uint4* triShade = nullptr;       // indices[3], material
    uint32_t triCount = 0;
    float4* vertsIn = nullptr;       // ShadingVertex, 2 x float4 each, model space
    float4* verts = nullptr;         // ShadingVertex, world space
    uint32_t* vertModel = nullptr;   // model index per vertex
    uint32_t vertCount = 0;
    Mat4* modelToWorld = nullptr;
    uint32_t modelCount = 0;
    float4* materials = nullptr;     // SimpleMaterial, 4 x float4 each
    uint32_t materialCount = 0;
    // bottom-up refit support (computed on the host once per topology)
    uint32_t* parentSlot = nullptr;  // (parent << 2) | slot, or ~0 for roots
    uint32_t* internalCount = nullptr; // number of internal children per node
    uint32_t* arrivals = nullptr;    // arrival counters, zeroed before each refit
    uint32_t* refitStarts = nullptr; // nodes with no internal children
    uint32_t refitStartCount = 0;
    uint32_t maxDepth = 0;
    LightEnvDev env;
};

// per-camera device state
struct CameraDev {
    uint32_t blocks = 0, tiles = 0, padded = 0, valid = 0;
    uint32_t msaa = 16;
    Rays4* tileRays = nullptr;       // camera space [tiles]
    Rays4* blockRays = nullptr;      // camera space [blocks]
    float4* beams = nullptr;         // camera space [padded * 3]
    int32_t* remap = nullptr;        // [width * height * split]
    uint32_t width = 0, height = 0, split = 1;
    // per frame
    StackEntry* blockStacks = nullptr; // [blocks * kBlockStack]
    uint32_t* blockSizes = nullptr;    // [blocks]
    TileList* tileLists = nullptr;     // [tiles]
    uint32_t* pool = nullptr;          // [poolChunks * kChunk]
    uint32_t* chunkNext = nullptr;     // [poolChunks]
    uint32_t poolChunks = 0;
    uint32_t* counters = nullptr;      // [0] chunk allocator, [1] status bits, [2], [3] tile queue heads
    uint32_t* tileCost = nullptr;      // [tiles] node visits of the last frame (scheduling only)
    uint32_t* tileOrder = nullptr;     // [tiles] longest-first tile order built from tileCost
    bool costValid = false;            // tileCost holds a previous frame's values
    uint32_t* colors = nullptr;        // [padded] RGBA8 per sorted sample
    uint32_t* hitIds = nullptr;        // [padded * msaa] when capturing
    float* depth = nullptr;            // [padded * msaa] when capturing
    uint32_t* image = nullptr;         // device image [height * stride]
    uint64_t imageStride = 0;
};

struct FrameParams {
    Mat4 cameraToWorld;
    uint32_t fpStrict;
    uint32_t capture;
};

// records the message returned by hvvr_last_error() on this thread and returns code
int setLastError(int code, const char* msg);

// kernel launchers (defined in the .cu files); each returns cudaGetLastError()
cudaError_t launchBlockCull(const SceneDev& s, const CameraDev& c, const FrameParams& f, cudaStream_t st);
// whole-camera tile cull (longest-first when c.costValid) on queue counters[2]
cudaError_t launchTileCull(const SceneDev& s, const CameraDev& c, const FrameParams& f, cudaStream_t st);
// c.tileOrder <- tiles sorted by descending c.tileCost (log2 buckets)
cudaError_t launchTileOrder(const CameraDev& c, cudaStream_t st);
// tile cull / intersect of the tiles order[first, first + count) (order == nullptr: tiles 0..count-1);
// concurrent tile-cull launches of one camera need distinct zeroed queue heads
cudaError_t launchTileCullRange(const SceneDev& s, const CameraDev& c, const FrameParams& f, const uint32_t* order,
                                uint32_t first, uint32_t count, uint32_t* queue, cudaStream_t st);
cudaError_t launchIntersectShade(const SceneDev& s, const CameraDev& c, const FrameParams& f, cudaStream_t st);
cudaError_t launchIntersectShadeRange(const SceneDev& s, const CameraDev& c, const FrameParams& f,
                                      const uint32_t* order, uint32_t first, uint32_t count, cudaStream_t st);
cudaError_t launchRemap(const CameraDev& c, cudaStream_t st);
cudaError_t launchRefit(const SceneDev& s, cudaStream_t st);
cudaError_t uploadMsaaTable(uint32_t n, const float* offsets, cudaStream_t st);

} // namespace hvb
