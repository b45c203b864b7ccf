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
// per-warp tile traversal stack in shared memory. The reference's TileFrame holds 4096
// entries; nearly every tile needs far fewer (at most 123 on the 1M-triangle stereo frame), so
// the main pass uses kTileStack and a tile that would outgrow it is culled again by a retry
// pass with 4096 entries. Outgrowing that sets kStatusStackOverflow and leaves the tile empty.
enum : uint32_t { kTileStack = 256 };
// triangle indices move between traversal and intersection in chunks of one intersect batch
enum : uint32_t { kChunk = 128 };
enum : uint32_t { kNoChunk = 0xffffffffu };
// Streamed tiles (the first tiles of a pipelined launch's queue, its longest): the list is
// published after its first chunk and its shade follows the chunks as they are linked. A chunk's
// link reads kChunkPending until the next chunk is linked (kNoChunk after the last one), the
// tile's TileList reads count kCountStreaming until the list is complete, and the last chunk's
// unused entries hold kNoTriangle.
enum : uint32_t { kChunkPending = 0xfffffffeu, kCountStreaming = 0xffffffffu, kNoTriangle = 0xffffffffu };

// device status bits (OR-ed into a per-frame word)
enum : uint32_t {
    kStatusPoolOverflow = 1u,   // triangle-index pool exhausted
    kStatusStackOverflow = 2u,  // tile traversal stack exhausted
    kStatusBadLeaf = 4u,        // a passing leaf had an empty/inverted triangle range
    kStatusRefitTimeout = 8u,   // refit walked more levels than the tree has
    kStatusPipelineTimeout = 16u, // a pipelined shade CTA gave up waiting for its tile's list
    kStatusBadInput = 32u,      // caller-supplied cull inputs out of range (hvvr_tile_cull_static)
};

// A pipelined rate class publishes each culled tile into a ready slot; the slot holds the global
// tile index, with kReadyRetry set when the tile's traversal stack overflowed and the retry pass
// culls and shades it instead. kReadyEmpty marks a slot not yet published.
enum : uint32_t { kReadyEmpty = 0xffffffffu, kReadyRetry = 0x80000000u };

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
    const unsigned long long* textures = nullptr; // texture object of each texture id (0: none)
    uint32_t textureCount = 0;
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
    TileList* tileLists = nullptr;     // [tiles], chunk indices into the rendering batch's pool
    uint32_t* tileCost = nullptr;      // [tiles] node visits of the last frame (scheduling only)
    uint32_t* colors = nullptr;        // [padded] RGBA8 per sorted sample
    uint32_t* hitIds = nullptr;        // [padded * msaa] when capturing
    float* depth = nullptr;            // [padded * msaa] when capturing
    uint32_t* image = nullptr;         // device image [height * stride]
    uint64_t imageStride = 0;
};

// The foveated resolve of one view (polar sample texture -> screen image, with temporal
// reprojection and eccentricity-dependent contrast enhancement). Every texture is a CUDA array
// with a texture object for reads and a surface object for writes:
//   polar textures [rings][samplesPerRing]: colour (RGBA8 sRGB), view depth (float), first and
//   second moments (RGBA16 unorm each)
//   screen textures [height][width] (RGBA8 sRGB): this frame's temporally filtered result and the
//   previous frame's (the filter passes and the contrast enhancement run fused, in shared memory)
struct FoveaDev {
    const uint2* remap;        // [valid] polar texel (azimuth index, ring) of each sample
    cudaTextureObject_t rawTex, depthTex, m1Tex, m2Tex;
    cudaSurfaceObject_t rawSurf, depthSurf, m1Surf, m2Surf;
    cudaTextureObject_t resultTex, prevTex; // result: written this frame
    cudaSurfaceObject_t resultSurf;
    const float4* srgbDecode;  // [256] the texture unit's read of an RGBA8 sRGB texel per 8-bit code
    uint32_t* image;           // nullptr: the view has no foveated resolve
    uint32_t imageStride, width, height;
    uint32_t spr, rings, valid;
    // EccentricityMap {m, w_0, S, invLogA, invW_0, invM} and the texture-coordinate mapping
    float eccM, eccW0, eccS, eccInvLogA, eccInvW0, eccInvM;
    float texMapSize, invTexMapSize, invMaxEcc;
    float sampleToEye[9];      // column-major 3x3
    float eyeToSamplePrev[16]; // column-major 4x4: eye space -> previous frame's sample space
};

// One view of a frame: a camera and the scene it renders. A frame is a table of views whose
// blocks and tiles are numbered consecutively ("global" indices); every stage runs one launch
// over all views, and a kernel finds its view through blockView[global block].
struct ViewDev {
    Mat4 M;                          // camera to world for this frame
    LightEnvDev env;
    const Node* nodes;
    const float4* tris;
    const uint4* triShade;
    const float4* verts;
    const float4* materials;
    const unsigned long long* textures; // texture objects by id (0: none); textureCount entries
    uint32_t textureCount;
    uint32_t prefetchNodes;          // nodes to bring into L2 at the top of the frame (0: an earlier
                                     // view of the frame renders the same scene, or none)
    const Rays4* tileRays;
    const Rays4* blockRays;
    const float4* beams;
    StackEntry* blockStacks;
    uint32_t* blockSizes;
    TileList* tileLists;
    uint32_t* tileCost;
    uint32_t* colors;
    uint32_t* hitIds;                // nullptr unless capturing
    float* depth;
    uint32_t tileStart, blockStart;  // first global tile / block
    uint32_t msaa, rateIdx;          // rate; its class: log2(msaa), + 6 for a thin-lens view, + 12 for the rotated grid
    // thin lens (depth of field) when lensRadius > 0
    float lensRadius, focalDistance;
    const float2* lensPos;           // [4 tiles][msaa][128] lens positions (the reference's lookup table)
    uint32_t* occRank;               // [tiles] rank of each tile among the view's non-empty tiles
    // foveated views: world-space cull planes {normal, dist} for the tile frusta, and the
    // per-sample view depth of subsample 0 (the reference's TMaxBuffer)
    float cull[4][4];
    uint32_t hasCull;
    float* tmaxOut;
    FoveaDev fov;                    // foveated resolve (fov.image == nullptr: none)
};

// frame-wide device state shared by the launches of one batch
struct FrameDev {
    const ViewDev* views = nullptr;    // [viewCount]
    const uint32_t* blockView = nullptr; // [blocks] view of each global block
    uint32_t viewCount = 0, tiles = 0, blocks = 0;
    uint32_t* pool = nullptr;          // [poolChunks * kChunk] triangle-list chunks
    uint32_t* chunkNext = nullptr;     // [poolChunks]
    uint32_t poolChunks = 0;
    uint32_t* counters = nullptr;      // [0] chunk allocator, [1] status bits, [2 + 3k ..] per-launch queues
    uint32_t* order = nullptr;         // [tiles] tile order: grouped by rate, then longest first
    uint32_t* retry = nullptr;         // [tiles] tiles whose traversal stack overflowed, per range
    uint32_t* ready = nullptr;         // [tiles] ready slots of the pipelined rate classes (kReadyEmpty at frame start)
    uint32_t cullCtasPerSm = 0;        // cap on the persistent tile cull's resident CTAs per SM (0: occupancy)
    uint32_t cullPersistent = 1;       // 0: each tile-cull warp culls one tile, and the grid covers all tiles
    uint32_t streamTiles = 0;          // pipelined launches: the first streamTiles tiles of the queue stream
};


// records the message returned by hvvr_last_error() on this thread and returns code
int setLastError(int code, const char* msg);

// rate classes: log2(msaa) for pinhole views (spiral pattern), 6 + log2(msaa) for thin-lens views,
// 12 + log2(msaa) for pinhole views with the rotated-grid pattern
enum : uint32_t { kRateClasses = 18 };
// counters: [0] chunk allocator, [1] status, then per tile-cull launch k (2 per rate class)
// three words at kQueueBase + 3k: work-queue head, retry count, retry-queue head
// then one word counting the list entries that survive the intersect's per-tile tests, one counting
// the (warp, surviving entry) pairs whose subsample tests ran (the rest were skipped by the per-warp
// depth bound), then per launch part k (2 per rate class) the ready-slot tail of its cull -> shade
// pipeline
enum : uint32_t {
    kQueueBase = 2,
    kQueueWords = 3,
    kSurvivorWord = kQueueBase + kQueueWords * 2 * kRateClasses,
    kTestedWord = kSurvivorWord + 1,
    kPipeBase = kTestedWord + 1,
    kCounterWords = kPipeBase + 2 * kRateClasses
};

// kernel launchers (defined in the .cu files); each returns cudaGetLastError()
cudaError_t launchBlockCull(const FrameDev& fr, cudaStream_t st);
// fr.order <- global tiles grouped by ascending rate index, longest first (log2 buckets of
// last frame's visit counts) within a rate
cudaError_t launchTileOrder(const FrameDev& fr, cudaStream_t st);
// tile cull / intersect-shade of the global tiles order[first, first + count) (order ==
// nullptr: tiles first..first+count-1). queues: kQueueWords zeroed words of this launch
// (concurrent launches need their own). warps = tile-cull warps per CTA (1, 2, 4 or 8). Tiles
// whose traversal stack outgrows stackLimit (0 = kTileStack; at least 8) are
// culled again by a second launch with a 4096-entry stack.
cudaError_t launchTileCull(const FrameDev& fr, const uint32_t* order, uint32_t first, uint32_t count,
                           uint32_t* queues, uint32_t warps, uint32_t stackLimit, cudaStream_t st);
// pattern: 0 the spiral, 1 the rotated grid (pinhole only; thin lens always uses the spiral)
cudaError_t launchIntersectShade(const FrameDev& fr, uint32_t msaa, uint32_t pattern, bool fpStrict, bool dof,
                                 const uint32_t* order, uint32_t first, uint32_t count, cudaStream_t st);
// The cull -> shade pipeline of one part of a pinhole rate class over the global tiles
// order[first, first + count), on one stream: the tile cull publishes every finished tile into fr.ready[first + i]
// (i = the order of completion; pipe[0] counts them), and the shade launch - started while the
// cull runs (programmatic dependent launch, once every cull CTA is resident) - shades slot i as
// soon as it is published (pipe[1] hands out the slots; a wait gives up after about a second and
// sets kStatusPipelineTimeout). Tiles whose stack outgrew stackLimit are then culled again with a
// 4096-entry stack and shaded by a third launch over the retry list. queues: kQueueWords zeroed
// words; pipe: 1 zeroed word; fr.ready[first, first + count) must hold kReadyEmpty.
// the two passes of launchTileCull on their own: the main pass (which, given ready and readyTail,
// publishes each finished tile as the pipeline describes) and the retry pass
cudaError_t launchTileCullMain(const FrameDev& fr, const uint32_t* order, uint32_t first, uint32_t count,
                               uint32_t* queues, uint32_t warps, uint32_t stackLimit, uint32_t* ready,
                               uint32_t* readyTail, cudaStream_t st);
cudaError_t launchTileCullRetryPass(const FrameDev& fr, const uint32_t* order, uint32_t first, uint32_t count,
                                    uint32_t* queues, cudaStream_t st);
cudaError_t launchCullShadePipeline(const FrameDev& fr, uint32_t msaa, uint32_t pattern, bool fpStrict, uint32_t first,
                                    uint32_t count, uint32_t* queues, uint32_t* pipe, uint32_t warps,
                                    uint32_t stackLimit, cudaStream_t st);
// occRank of every thin-lens view (one block per view; pinhole views are skipped)
cudaError_t launchOccupiedRank(const FrameDev& fr, cudaStream_t st);
cudaError_t launchRemap(const CameraDev& c, cudaStream_t st);
cudaError_t launchRefit(const SceneDev& s, bool fma, cudaStream_t st);
// the unit offsets of rate n for pattern 0 (spiral) or 1 (rotated grid)
cudaError_t uploadMsaaTable(uint32_t n, uint32_t pattern, const float* offsets, cudaStream_t st);
// the foveated resolve of view `view` of the frame (fov: the host copy of its FoveaDev, for
// the launch shapes): scatter to the polar textures, moments, polar -> screen with temporal
// reprojection, two eccentricity filter passes and contrast enhancement into fov.image
cudaError_t launchFoveatedResolve(const FrameDev& fr, uint32_t view, const FoveaDev& fov, cudaStream_t st);
// out[256] <- the texture unit's value of a texel holding (i, i, i, i), read at its centre from
// codes (a 256 x 1 RGBA8 texture made like the foveated screen textures)
cudaError_t launchSrgbDecodeTable(cudaTextureObject_t codes, float4* out, cudaStream_t st);
// writes v to *dst with a one-thread kernel (no host memory involved; capturable)
cudaError_t launchWriteView(const ViewDev& v, ViewDev* dst, cudaStream_t st);

} // namespace hvb
