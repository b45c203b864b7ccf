// host_objects.h - the library's host-side objects (raycaster, scene models, lights, cameras,
// frame batches) and the frame driver entry points shared by raycaster.cpp and server.cpp.
// Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <stdint.h>

#include <atomic>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hvvr_c.h"
#include "foveated.h"
#include "host_setup.h"
#include "hvvr_internal.h"

namespace hvb {

// records a printf-style message for hvvr_last_error() on this thread and returns code
int fail(int code, const char* fmt, ...);

#define CUDA_TRY(expr)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? HVVR_ERR_OOM : HVVR_ERR_CUDA, "%s: %s (%s:%d)", \
                        #expr, cudaGetErrorString(e_), __FILE__, __LINE__);                               \
    } while (0)

#define TRY(expr)                \
    do {                         \
        int r_ = (expr);         \
        if (r_ != HVVR_OK) return r_; \
    } while (0)

// owning device allocation
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        if (count == n && p) return HVVR_OK;
        release();
        if (count == 0) return HVVR_OK;
        cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(HVVR_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        n = count;
        return HVVR_OK;
    }
    // grows only (a smaller request keeps the buffer: no free, which would synchronise the device)
    int ensure(size_t count) {
        if (count <= n && (p || count == 0)) return HVVR_OK;
        return alloc(count);
    }
    int upload(const void* src, size_t count, cudaStream_t st) {
        TRY(alloc(count));
        if (count) CUDA_TRY(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
        return HVVR_OK;
    }
};

// A 2D CUDA array with a texture object (reads) and a surface object (writes), made as the
// reference's createEmptyTexture makes one (libraries/hvvr/raycaster/texture.cu:283-321):
// normalized coordinates, the given addressing per axis (clamp on the third) and filter.
struct TexArray {
    cudaArray_t array = nullptr;
    cudaTextureObject_t tex = 0;
    cudaSurfaceObject_t surf = 0;
    uint32_t width = 0, height = 0, texelBytes = 0;
    TexArray() = default;
    TexArray(const TexArray&) = delete;
    TexArray& operator=(const TexArray&) = delete;
    ~TexArray() { release(); }
    void release();
    int create(uint32_t w, uint32_t h, const cudaChannelFormatDesc& channels, uint32_t texelBytes,
               cudaTextureReadMode readMode, bool srgb, cudaTextureAddressMode addrX, cudaTextureAddressMode addrY,
               bool linear);
    // all texels zero
    int clear(cudaStream_t st);
    // the texels as rows of width * texelBytes bytes (synchronous)
    int download(void* dst, cudaStream_t st) const;
};

} // namespace hvb

// the object structs below are the C ABI's opaque types (global namespace)
using namespace hvb;

struct hvvr_model {
    hvvr_raycaster* rc = nullptr;
    std::vector<hvvr_shading_vertex> verts;
    std::vector<hvvr_tri_shade> triShade;
    std::vector<hvvr_topology_node> nodes;
    std::vector<hvvr_material> materials;
    hvvr_transform xf{};
};

struct hvvr_light {
    hvvr_raycaster* rc = nullptr;
    hvvr_light_union light{};
};

// A material texture: a mipmapped CUDA array and the texture object the shading reads
struct hvvr_texture {
    hvvr_raycaster* rc = nullptr;
    uint32_t id = 0;
    uint32_t format = 0, width = 0, height = 0, levels = 0, elementSize = 0;
    cudaMipmappedArray_t array = nullptr;
    cudaTextureObject_t object = 0;
    ~hvvr_texture();
};

struct hvvr_camera {
    hvvr_raycaster* rc = nullptr;
    bool enabled = true;
    hvvr_float_rect viewport{};
    hvvr_thin_lens lens{0.0f, 1.0f};
    hvvr_vec3 eyeDir{0.0f, 0.0f, -1.0f};
    float fovX = 0.0f, fovY = 0.0f;
    hvvr_image_desc target{};
    std::vector<hvvr_sample> samples;
    uint32_t split = 1;
    hvvr_transform xf{};
    uint32_t msaa = 16;
    uint32_t msaaPattern = 0;       // HVVR_MSAA_SPIRAL or HVVR_MSAA_ROTATED_GRID
    uint32_t capture = 0;
    bool setupDirty = true;
    bool setupOnHost = false;         // the current sample setup was built on the host
    bool rendered = false;
    bool hidden = false;              // a server's camera: rendered only by batches that name it
    uint64_t setupGen = 0;            // process-unique id of the current sample setup and buffers
    uint64_t costFrames = 0;          // frames rendered since the setup (tileCost is valid when > 0)
    hvvr_batch* lastBatch = nullptr;  // batch whose pool holds this camera's last tile lists
    std::vector<hvvr_batch*> batches; // camera-list batches that name this camera
    CameraDev dev;
    SampleSetup setup;
    // device storage behind dev
    DevBuf<Rays4> tileRays, blockRays;
    DevBuf<float4> beams;
    DevBuf<int32_t> remap;
    DevBuf<StackEntry> blockStacks;
    DevBuf<uint32_t> blockSizes;
    DevBuf<TileList> tileLists;
    DevBuf<uint32_t> colors, hitIds, image, tileCost, occRank;
    DevBuf<float> depth;
    DevBuf<float2> lensPos;           // thin-lens table of rate lensRate
    uint32_t lensRate = 0;
    // foveated polar mode: the polar sample set replaces the camera's own samples for traversal
    // and shading; the camera's samples give the screen bounds and the output image
    bool foveated = false;
    hvvr_float_rect sampleBounds{};
    DevBuf<uint2> polarRemap;         // [padded] polar texel of each sample
    DevBuf<float> tmax;               // [padded] view depth of subsample 0
    float eyeToWorld[16] = {};        // the last frame's batch-to-world matrix and cull planes
    float cullPlanes[4][4] = {};
    // foveated resolve: polar textures, screen textures (fovResult[fovCur] is written by the next
    // frame, the other one holds the previous frame's result), the temporal history matrices
    // and the last frame's resolve matrices
    TexArray polarRaw, polarDepth, moment1, moment2, fovResult[2];
    DevBuf<float4> fovDecode;      // [256] the texture unit's read of each RGBA8 sRGB code
    FoveaDev fovStatic{};             // buffers, sizes and mapping constants (no per-frame fields)
    uint32_t fovCur = 0;
    float worldToEyePrev[16] = {};
    float eyePrevToSamplePrev[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float lastSampleToEye[9] = {}, lastEyeToSamplePrev[16] = {};
    void* registered = nullptr;       // CPU render target page-locked by cudaHostRegister
};

// A frame batch: the enabled cameras of one or more raycasters (one scene each, same device)
// rendered as one frame - one launch per stage over all views, the tile cull as one
// persistent work queue, intersect/shade once per MSAA rate - optionally replayed from a
// CUDA graph. Every raycaster renders its own cameras through an internal batch.
struct hvvr_batch {
    std::vector<hvvr_raycaster*> rcs;
    bool fixedViews = false;          // renders exactly `cams` (else every enabled camera of rcs)
    std::vector<hvvr_camera*> cams;
    bool internal = false;            // a raycaster's own batch
    // side-stream priorities: 0 = the slowest tiles' parts at the greatest priority, the rest at the
    // default; 1 = every part at the greatest priority; 2 = every part at the least priority
    int streamPriorities = 0;
    bool detached = false;            // one of its raycasters was destroyed
    hvvr_batch_config cfg{};
    // layout of the current frame
    struct View {
        hvvr_camera* cam;
        uint32_t tileStart, blockStart;
    };
    std::vector<View> views;
    std::vector<uint64_t> layoutKey;
    uint32_t tiles = 0, blocks = 0;
    uint32_t rateTiles[kRateClasses] = {}, rateStart[kRateClasses] = {};
    bool anyLens = false;             // a thin-lens view is in the layout
    bool fpStrict = false;
    bool costValid = false;           // every view's tileCost holds a previous frame's counts
    DevBuf<ViewDev> viewsDev;
    DevBuf<uint32_t> blockView, order, retry, ready, pool, chunkNext, counters;
    uint32_t poolChunks = 0;
    ViewDev* hostViews[2] = {};       // pinned staging of the per-frame view table
    size_t hostViewsCap = 0;
    cudaEvent_t hostViewsEv[2] = {};
    bool hostViewsUsed[2] = {};
    int hostSlot = 0;
    uint32_t* hostCounters = nullptr; // pinned copy of counters after each frame
    bool counterValid = false;
    cudaStream_t side[2 * kRateClasses] = {}; // per rate class: [2r] heavy tiles (high priority), [2r+1] the rest
    cudaEvent_t forkEv = nullptr, rankEv = nullptr, doneEv[2 * kRateClasses] = {}, cullEv[2 * kRateClasses] = {};
    cudaEvent_t orderForkEv = nullptr, orderDoneEv = nullptr; // the tile order, beside the block cull
    cudaEvent_t ev[6] = {};
    cudaEvent_t kev[2 * kRateClasses][3] = {}; // per side stream: before tile cull, after it, after intersect
    bool kevUsed[2 * kRateClasses] = {};
    bool kevPipelined[2 * kRateClasses] = {}; // the part ran as a cull -> shade pipeline (kev[1] == kev[2])
    bool stageTimes = false;          // ev[1..4] and kev were recorded by the last frame
    cudaGraphExec_t graph = nullptr;
    std::vector<uint64_t> graphKey;
};

struct hvvr_raycaster {
    hvvr_spec spec{};
    cudaStream_t stream = nullptr;
    std::vector<std::unique_ptr<hvvr_model>> models;
    std::vector<std::unique_ptr<hvvr_light>> lights;
    std::vector<std::unique_ptr<hvvr_camera>> cameras;
    std::vector<std::unique_ptr<hvvr_texture>> textures;
    uint32_t nextTextureId = 0;           // texture ids are not reused
    DevBuf<unsigned long long> texTable;  // [nextTextureId] texture object by id, 0 for none
    bool sceneDirty = true;
    bool refitDirty = true;
    SceneDev scene;
    DevBuf<Node> nodes;
    DevBuf<float4> tris, vertsIn, verts, materials;
    DevBuf<uint4> triShade;
    DevBuf<uint32_t> vertModel, parentSlot, internalCount, arrivals, refitStarts;
    DevBuf<Mat4> modelToWorld;
    std::vector<Node> hostNodes;
    uint32_t refitStatus = 0;
    std::unique_ptr<hvvr_batch> own;      // renders this raycaster's cameras
    std::unique_ptr<PolarSetup> polar;    // foveated polar mode: the sample set of spec's pattern
    std::vector<hvvr_batch*> batches;     // user batches that include this raycaster
};

namespace hvb {

constexpr uint64_t kDefaultCapacity = 128ull << 20; // MAX_TRI_INDICES_TO_INTERSECT

int uploadScene(hvvr_raycaster* rc, cudaStream_t st);
int setupCamera(hvvr_camera* cam, cudaStream_t st);
void releaseCamera(hvvr_camera* cam);
void batchConfigDefault(hvvr_batch_config* c);
int checkConfig(const hvvr_batch_config& c);
void releaseBatch(hvvr_batch* b);
int checkStatus(const hvvr_batch* b);
uint32_t rateIndex(uint32_t rate);
// scene update and refit of the batch's raycasters (unless skipScenes), then one frame of its views on st
int renderBatch(hvvr_batch* b, cudaStream_t st, bool skipScenes = false);
// grows the batch's frame buffers to hold a frame of this many tiles, blocks and views
int reserveBatch(hvvr_batch* b, size_t tiles, size_t blocks, size_t views);
// uploads the MSAA offset table of `rate` to the current device once
int ensureMsaaTable(uint32_t rate, cudaStream_t st);
// a new camera of the same raycaster with cam's sample set and setup (device copies, no
// re-clustering); cam must have been set up (rendered once)
int cloneCamera(const hvvr_camera* cam, hvvr_camera** out);
// forget a foveated camera's temporal history: its next frame reads no previous result
void resetFoveatedHistory(hvvr_camera* cam);
// the raycaster's texture objects by id, uploaded for the scene
int uploadTextureTable(hvvr_raycaster* rc, cudaStream_t st);
// device bytes a camera holds for its setup and per-frame buffers at the given MSAA rate
size_t cameraBytes(const hvvr_camera* cam, uint32_t msaa);

} // namespace hvb
