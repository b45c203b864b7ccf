// tile_cull_static.cu - hvvr_tile_cull_static: the tile-frustum cull for callers that cannot
// allocate device memory.
//
// Who needs this: code that runs where cudaMalloc is not allowed or not wanted - a render
// thread with a hard frame deadline (an allocation can synchronise the device), a plugin
// whose host application owns and budgets every device allocation, or a caller that has
// already handed all device memory to its own pool allocator. Such a caller owns its input
// and output buffers, but the cull also needs working memory for the per-tile triangle
// lists while they are being discovered, before their sizes are known.
//
// That working memory lives in gScratch below: a file-scope __device__ array compiled into
// the library, so it exists on every GPU that loads the library, for the life of the
// process, whether or not this entry point is ever called. Its size bounds one call:
// at most kMaxTiles tiles and kMaxEntries triangle-list entries. All calls share it and it
// keeps the previous call's contents; the chunk allocator and status word are cleared at
// the start of every call, and every other word a call reads is written by that call.
// Two calls whose work overlaps on the GPU (different streams, or different host threads)
// race on the array and must be serialised by the caller.
//
// In host code gScratch names a host-side shadow, not device memory, so its device address
// is looked up with cudaGetSymbolAddress once per device, on the first call made with that
// device current. Make that first call on each device before any stream capture starts. The
// address is cached for the life of the process: a cudaDeviceReset (which also ends every other
// object of the library on that device) leaves the cache stale, so do not reset a device that the
// library is using. Every call is synchronous: it checks the caller's inputs and reads the status
// back, waiting for the stream each time.
//
// The cull itself is the tileCullKernel of the render path (traverse.cu), given a one-view
// table written into the scratch by a one-thread kernel and pointed at the scratch pool;
// a one-block scan and a per-tile gather then copy the chunked lists into the caller's
// flat output in tile order. Nothing here calls cudaMalloc, cudaFree or an allocating library.
#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/hvvr_c.h"
#include "dev_common.cuh"
#include "host_setup.h"

namespace hvb {

namespace {

constexpr uint32_t kMaxTiles = 65536;                  // 4,194,304 padded samples, 1024 blocks
constexpr uint32_t kMaxChunks = 61440;                 // kMaxChunks * kChunk entries
constexpr uint64_t kMaxEntries = uint64_t(kMaxChunks) * kChunk; // 7,864,320 entries (30 MiB)
// word layout of the scratch array
constexpr size_t kOffCounters = 0;                     // [0] chunk allocator, [1] status, [2..3] total (u64),
                                                       // [4..6] work queue, retry count, retry queue
constexpr size_t kOffView = 64;                        // the one-view table of the cull (ViewDev)
constexpr size_t kViewWords = (sizeof(ViewDev) + 255) / 256 * 64;
constexpr size_t kOffLists = kOffView + kViewWords;    // TileList[kMaxTiles]
constexpr size_t kOffCost = kOffLists + 2 * size_t(kMaxTiles); // per-tile visit counts (written, unused)
constexpr size_t kOffRetry = kOffCost + kMaxTiles;    // tiles re-culled with the large stack
constexpr size_t kOffNext = kOffRetry + kMaxTiles;
constexpr size_t kOffOffsets = kOffNext + kMaxChunks;  // exclusive prefix of counts, kMaxTiles + 1 words (u32 lo)
constexpr size_t kOffPool = (kOffOffsets + kMaxTiles + 1 + 63) / 64 * 64;
constexpr size_t kScratchWords = kOffPool + size_t(kMaxChunks) * kChunk;

static __device__ __align__(256) uint32_t gScratch[kScratchWords];

// exclusive scan of the per-tile counts (64-bit running total), one block
__global__ void __launch_bounds__(1024) scanCounts(uint32_t* scratch, uint32_t tiles) {
    __shared__ unsigned long long carry;
    __shared__ uint32_t warpSums[32];
    const TileList* lists = reinterpret_cast<const TileList*>(scratch + kOffLists);
    uint32_t* offsets = scratch + kOffOffsets;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += 1024) {
        const uint32_t t = base + threadIdx.x;
        const uint32_t v = t < tiles ? lists[t].count : 0u;
        // inclusive warp scan
        uint32_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if ((threadIdx.x & 31u) >= uint32_t(d)) x += y;
        }
        if ((threadIdx.x & 31u) == 31u) warpSums[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint32_t w = warpSums[threadIdx.x];
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
                if (threadIdx.x >= uint32_t(d)) w += y;
            }
            warpSums[threadIdx.x] = w;
        }
        __syncthreads();
        const uint32_t warpBase = (threadIdx.x >> 5) ? warpSums[(threadIdx.x >> 5) - 1] : 0u;
        const unsigned long long excl = carry + warpBase + x - v;
        // offsets past 2^32 entries cannot fit any output buffer; the gather checks the total
        if (t < tiles) offsets[t] = excl > 0xffffffffull ? 0xffffffffu : uint32_t(excl);
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        unsigned long long* total = reinterpret_cast<unsigned long long*>(scratch + kOffCounters + 2);
        *total = carry;
    }
}

// copy each tile's chunk chain to out[offset .. offset+count) and write counts
__global__ void gatherLists(const uint32_t* __restrict__ scratch, uint32_t tiles, uint32_t* __restrict__ counts,
                            uint32_t* __restrict__ out, unsigned long long capacity) {
    const uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (t >= tiles) return;
    const uint32_t lane = threadIdx.x & 31u;
    const TileList L = reinterpret_cast<const TileList*>(scratch + kOffLists)[t];
    const unsigned long long total = *reinterpret_cast<const unsigned long long*>(scratch + kOffCounters + 2);
    if (lane == 0) counts[t] = L.count;
    if (total > capacity) return;
    const uint32_t* next = scratch + kOffNext;
    const uint32_t* pool = scratch + kOffPool;
    uint32_t off = scratch[kOffOffsets + t];
    uint32_t c = L.first, left = L.count;
    while (left && c < kMaxChunks) {
        const uint32_t n = left < kChunk ? left : kChunk;
        for (uint32_t j = lane; j < n; j += 32) out[size_t(off) + j] = pool[size_t(c) * kChunk + j];
        off += n;
        left -= n;
        c = next[c];
    }
}

// The cull trusts its inputs (the render path builds them itself); this entry point takes them
// from the caller, so they are checked first, one thread per node and per block: every internal
// child of a node must lie after it and inside the node array (the depth-first layout the render
// path checks when it builds a scene), every block-stack size must be at most kBlockStack, and every
// block-stack entry must name a node inside the array. Any violation sets kStatusBadInput.
__global__ void checkInputs(const Node* __restrict__ nodes, uint32_t nodeCount, const StackEntry* __restrict__ stacks,
                            const uint32_t* __restrict__ sizes, uint32_t blocks, uint32_t* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (i < nodeCount) {
        const uint32_t leafMask = nodes[i].leafMask;
        for (uint32_t k = 0; k < 4; k++) {
            if ((leafMask >> k) & 1u) continue;
            const uint64_t c = uint64_t(i) + nodes[i].tri[k + 1];
            if (c <= i || c >= nodeCount) bad = true;
        }
    }
    if (i < blocks) {
        const uint32_t n = sizes[i];
        if (n > kBlockStack) {
            bad = true;
        } else {
            for (uint32_t j = 0; j < n; j++)
                if (stacks[size_t(i) * kBlockStack + j].node >= nodeCount) bad = true;
        }
    }
    if (bad) atomicOr(status, kStatusBadInput);
}

std::mutex gSetupMutex;
uint32_t* gScratchAddr[64] = {};

int failStatic(int code, const char* msg, cudaError_t e = cudaSuccess) {
    return setLastError(code, e == cudaSuccess ? msg : (std::string(msg) + ": " + cudaGetErrorString(e)).c_str());
}

} // namespace

} // namespace hvb

using namespace hvb;

extern "C" int hvvr_tile_cull_static(const hvvr_tile_cull_args* args, uint32_t* counts, uint32_t* indices,
                                     uint64_t capacity, uint64_t* total, void* stream) {
    if (!args || !counts || !total) return failStatic(HVVR_ERR_INVALID, "NULL argument");
    if (!args->nodes || !args->tile_rays || !args->block_stacks || !args->block_sizes || args->node_count == 0)
        return failStatic(HVVR_ERR_INVALID, "missing input buffer");
    if (args->tile_count == 0 || args->tile_count % kTilesPerBlock != 0)
        return failStatic(HVVR_ERR_INVALID, "tile_count must be a positive multiple of 64");
    if (args->tile_count > kMaxTiles)
        return failStatic(HVVR_ERR_INVALID, "tile_count exceeds the static scratch limit of 65536 tiles");
    if (capacity && !indices) return failStatic(HVVR_ERR_INVALID, "capacity given without an indices buffer");
    if (args->tile_stack_entries && (args->tile_stack_entries < 8 || args->tile_stack_entries > kTileStack))
        return failStatic(HVVR_ERR_INVALID, "tile_stack_entries must be 0 or in [8, 256]");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return failStatic(HVVR_ERR_CUDA, "cudaGetDevice failed", e);
    uint32_t* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(gSetupMutex);
        if (!gScratchAddr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, gScratch);
            if (e != cudaSuccess || !p) return failStatic(HVVR_ERR_CUDA, "cudaGetSymbolAddress(gScratch) failed", e);
            gScratchAddr[dev] = static_cast<uint32_t*>(p);
        }
        scratch = gScratchAddr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t tiles = args->tile_count;
    ViewDev v{};
    v.M = transformToMatrix(args->camera_to_world);
    v.nodes = static_cast<const Node*>(args->nodes);
    v.tileRays = static_cast<const Rays4*>(args->tile_rays);
    v.blockStacks = const_cast<StackEntry*>(static_cast<const StackEntry*>(args->block_stacks));
    v.blockSizes = const_cast<uint32_t*>(args->block_sizes);
    v.tileLists = reinterpret_cast<TileList*>(scratch + kOffLists);
    v.tileCost = scratch + kOffCost;
    FrameDev fr;
    fr.views = reinterpret_cast<const ViewDev*>(scratch + kOffView);
    fr.viewCount = 1;
    fr.tiles = tiles;
    fr.blocks = tiles / kTilesPerBlock;
    fr.pool = scratch + kOffPool;
    fr.chunkNext = scratch + kOffNext;
    fr.poolChunks = kMaxChunks;
    fr.counters = scratch + kOffCounters;
    fr.retry = scratch + kOffRetry;
    if ((e = cudaMemsetAsync(scratch + kOffCounters, 0, 8 * sizeof(uint32_t), st)) != cudaSuccess)
        return failStatic(HVVR_ERR_CUDA, "clearing the scratch counters failed", e);
    {
        const uint32_t n = std::max(args->node_count, fr.blocks);
        checkInputs<<<(n + 255) / 256, 256, 0, st>>>(v.nodes, args->node_count, v.blockStacks, v.blockSizes, fr.blocks,
                                                     scratch + kOffCounters + 1);
        uint32_t bad = 0;
        if ((e = cudaGetLastError()) != cudaSuccess) return failStatic(HVVR_ERR_CUDA, "input check launch failed", e);
        if ((e = cudaMemcpyAsync(&bad, scratch + kOffCounters + 1, sizeof(bad), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return failStatic(HVVR_ERR_CUDA, "input check failed", e);
        if (bad & kStatusBadInput)
            return failStatic(HVVR_ERR_INVALID, "malformed input: a block-stack size above 64, or a node index or child "
                                                "offset outside node_count");
    }
    if ((e = launchWriteView(v, reinterpret_cast<ViewDev*>(scratch + kOffView), st)) != cudaSuccess)
        return failStatic(HVVR_ERR_CUDA, "view setup launch failed", e);
    if ((e = launchTileCull(fr, nullptr, 0, tiles, scratch + kOffCounters + 4, 4, args->tile_stack_entries, st)) !=
        cudaSuccess)
        return failStatic(HVVR_ERR_CUDA, "tile cull launch failed", e);
    scanCounts<<<1, 1024, 0, st>>>(scratch, tiles);
    gatherLists<<<(tiles + 7) / 8, 256, 0, st>>>(scratch, tiles, counts, indices, capacity);
    if ((e = cudaGetLastError()) != cudaSuccess) return failStatic(HVVR_ERR_CUDA, "gather launch failed", e);
    uint32_t status[4] = {0, 0, 0, 0};
    if ((e = cudaMemcpyAsync(status, scratch + kOffCounters, sizeof(status), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return failStatic(HVVR_ERR_CUDA, "status read failed", e);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return failStatic(HVVR_ERR_CUDA, "cull failed", e);
    const uint64_t t64 = uint64_t(status[2]) | (uint64_t(status[3]) << 32);
    *total = t64;
    if (status[1] & kStatusPoolOverflow)
        return failStatic(HVVR_ERR_OVERFLOW, "triangle lists exceed the static scratch limit of 7,864,320 entries");
    if (status[1] & kStatusStackOverflow) return failStatic(HVVR_ERR_OVERFLOW, "tile traversal stack exhausted");
    if (t64 > capacity) return failStatic(HVVR_ERR_OVERFLOW, "output capacity smaller than the list total");
    return HVVR_OK;
}
