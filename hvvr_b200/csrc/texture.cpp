// texture.cpp - material textures: createTexture / destroyTexture (libraries/hvvr/raycaster/
// scene.cpp:28-40) and CreateTexture (libraries/hvvr/raycaster/texture.cu:201-272) as a
// per-raycaster table of texture objects, plus the parity read-backs.
#include "host_objects.h"
#include "texture_dev.h"

#include <string.h>

#include <algorithm>
#include <vector>

hvvr_texture::~hvvr_texture() {
    if (object) cudaDestroyTextureObject(object);
    if (array) cudaFreeMipmappedArray(array);
}

namespace hvb {
namespace {

struct FormatInfo {
    uint32_t elementSize;
    cudaChannelFormatDesc channels;
    cudaTextureReadMode readMode;
    bool srgb;
};

// formatToDescriptor (texture.cu:39-60) with getTextureSize's element sizes (texture.h:56-76)
bool formatInfo(uint32_t format, FormatInfo& f) {
    switch (format) {
    case kTexRgba8Srgb:
    case kTexRgba8:
        f = {4, cudaCreateChannelDesc(8, 8, 8, 8, cudaChannelFormatKindUnsigned), cudaReadModeNormalizedFloat,
             format == kTexRgba8Srgb};
        return true;
    case kTexRgba16:
        f = {8, cudaCreateChannelDesc(16, 16, 16, 16, cudaChannelFormatKindUnsigned), cudaReadModeNormalizedFloat,
             false};
        return true;
    case kTexRgba32f:
        f = {16, cudaCreateChannelDesc(32, 32, 32, 32, cudaChannelFormatKindFloat), cudaReadModeElementType, false};
        return true;
    case kTexRgba16f:
        f = {8, cudaCreateChannelDesc(16, 16, 16, 16, cudaChannelFormatKindFloat), cudaReadModeElementType, false};
        return true;
    case kTexR32f:
        f = {4, cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat), cudaReadModeElementType, false};
        return true;
    default:
        return false;
    }
}

// getMipMapLevels (texture.cu:188-198): one level per bit of the larger side
uint32_t mipLevels(uint32_t w, uint32_t h) {
    uint32_t sz = std::max(w, h), n = 0;
    while (sz) {
        sz /= 2;
        n++;
    }
    return n;
}

// generateMipMaps (texture.cu:106-186): each level from the one above through a clamp-addressed,
// linear-filtered, normalized-coordinate read of it
int generateMips(hvvr_texture* t, cudaStream_t st) {
    uint32_t w = t->width, h = t->height;
    for (uint32_t level = 0; level + 1 < t->levels; level++) {
        w = std::max(1u, w / 2);
        h = std::max(1u, h / 2);
        cudaArray_t from = nullptr, to = nullptr;
        CUDA_TRY(cudaGetMipmappedArrayLevel(&from, t->array, level));
        CUDA_TRY(cudaGetMipmappedArrayLevel(&to, t->array, level + 1));
        cudaResourceDesc res;
        memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = from;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.normalizedCoords = 1;
        td.filterMode = cudaFilterModeLinear;
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        FormatInfo fi;
        formatInfo(t->format, fi);
        td.readMode = fi.readMode;
        cudaTextureObject_t in = 0;
        CUDA_TRY(cudaCreateTextureObject(&in, &res, &td, nullptr));
        cudaResourceDesc sres;
        memset(&sres, 0, sizeof(sres));
        sres.resType = cudaResourceTypeArray;
        sres.res.array.array = to;
        cudaSurfaceObject_t out = 0;
        cudaError_t e = cudaCreateSurfaceObject(&out, &sres);
        if (e == cudaSuccess) e = launchMipLevel(t->format, out, in, w, h, st);
        // the objects are only referenced by the launch: wait for it before destroying them
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (out) cudaDestroySurfaceObject(out);
        cudaDestroyTextureObject(in);
        if (e != cudaSuccess) return fail(HVVR_ERR_CUDA, "mip level %u: %s", level + 1, cudaGetErrorString(e));
    }
    return HVVR_OK;
}

int uploadTableNow(hvvr_raycaster* rc) {
    TRY(uploadTextureTable(rc, rc->stream));
    CUDA_TRY(cudaStreamSynchronize(rc->stream));
    return HVVR_OK;
}

} // namespace

void TexArray::release() {
    if (tex) cudaDestroyTextureObject(tex);
    if (surf) cudaDestroySurfaceObject(surf);
    if (array) cudaFreeArray(array);
    tex = 0;
    surf = 0;
    array = nullptr;
    width = height = texelBytes = 0;
}

int TexArray::create(uint32_t w, uint32_t h, const cudaChannelFormatDesc& channels, uint32_t bytes,
                     cudaTextureReadMode readMode, bool srgb, cudaTextureAddressMode addrX,
                     cudaTextureAddressMode addrY, bool linear) {
    release();
    CUDA_TRY(cudaMallocArray(&array, &channels, w, h, cudaArraySurfaceLoadStore));
    width = w;
    height = h;
    texelBytes = bytes;
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = array;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = addrX;
    td.addressMode[1] = addrY;
    td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
    td.readMode = readMode;
    td.normalizedCoords = 1;
    td.sRGB = srgb ? 1 : 0;
    CUDA_TRY(cudaCreateTextureObject(&tex, &res, &td, nullptr));
    CUDA_TRY(cudaCreateSurfaceObject(&surf, &res));
    return HVVR_OK;
}

int TexArray::clear(cudaStream_t st) {
    if (!array) return HVVR_OK;
    const size_t row = size_t(width) * texelBytes;
    DevBuf<uint8_t> zeros;
    TRY(zeros.alloc(row * height));
    CUDA_TRY(cudaMemsetAsync(zeros.p, 0, row * height, st));
    CUDA_TRY(cudaMemcpy2DToArrayAsync(array, 0, 0, zeros.p, row, row, height, cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return HVVR_OK;
}

int TexArray::download(void* dst, cudaStream_t st) const {
    if (!array) return fail(HVVR_ERR_STATE, "no texture");
    const size_t row = size_t(width) * texelBytes;
    CUDA_TRY(cudaMemcpy2DFromArrayAsync(dst, row, array, 0, 0, row, height, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return HVVR_OK;
}

int uploadTextureTable(hvvr_raycaster* rc, cudaStream_t st) {
    std::vector<unsigned long long> table(rc->nextTextureId, 0ull);
    for (const auto& t : rc->textures) table[t->id] = t->object;
    TRY(rc->texTable.upload(table.data(), table.size(), st));
    rc->scene.textures = rc->texTable.p;
    rc->scene.textureCount = uint32_t(table.size());
    return HVVR_OK;
}

} // namespace hvb

extern "C" {

int hvvr_texture_create(hvvr_raycaster* rc, const hvvr_texture_data* data, hvvr_texture** out) {
    if (!rc || !data || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    FormatInfo fi;
    if (data->format == kTexR11G11B10f) return fail(HVVR_ERR_INVALID, "r11g11b10_float has no CUDA array format");
    if (!formatInfo(data->format, fi)) return fail(HVVR_ERR_INVALID, "unknown texture format %u", data->format);
    if (!data->data || data->width == 0 || data->height == 0)
        return fail(HVVR_ERR_INVALID, "texture needs texels and a non-zero size");
    if (data->stride_elements < data->width) return fail(HVVR_ERR_INVALID, "stride below width");
    if (data->width > 65536 || data->height > 65536) return fail(HVVR_ERR_INVALID, "texture larger than 65536");
    // SimpleMaterial keeps 16-bit ids with 0xffff meaning none (material.h:22-29)
    if (rc->nextTextureId >= 0xffffu) return fail(HVVR_ERR_OVERFLOW, "texture ids exhausted (65535)");
    CUDA_TRY(cudaSetDevice(rc->spec.device));
    auto t = std::make_unique<hvvr_texture>();
    t->rc = rc;
    t->format = data->format;
    t->width = data->width;
    t->height = data->height;
    t->elementSize = fi.elementSize;
    t->levels = mipLevels(data->width, data->height);
    const cudaExtent ext = make_cudaExtent(data->width, data->height, 0);
    CUDA_TRY(cudaMallocMipmappedArray(&t->array, &fi.channels, ext, t->levels));
    cudaArray_t level0 = nullptr;
    CUDA_TRY(cudaGetMipmappedArrayLevel(&level0, t->array, 0));
    const size_t row = size_t(data->width) * fi.elementSize;
    CUDA_TRY(cudaMemcpy2DToArrayAsync(level0, 0, 0, data->data, size_t(data->stride_elements) * fi.elementSize, row,
                                      data->height, cudaMemcpyHostToDevice, rc->stream));
    TRY(generateMips(t.get(), rc->stream));
    // the material texture object (texture.cu:234-265)
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeMipmappedArray;
    res.res.mipmap.mipmap = t->array;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = fi.readMode;
    td.sRGB = fi.srgb ? 1 : 0;
    td.normalizedCoords = 1;
    td.maxAnisotropy = 8;
    td.mipmapFilterMode = cudaFilterModeLinear;
    td.maxMipmapLevelClamp = float(t->levels - 1);
    CUDA_TRY(cudaCreateTextureObject(&t->object, &res, &td, nullptr));
    t->id = rc->nextTextureId++;
    hvvr_texture* raw = t.get();
    rc->textures.push_back(std::move(t));
    TRY(uploadTableNow(rc));
    *out = raw;
    return HVVR_OK;
}

int hvvr_texture_destroy(hvvr_raycaster* rc, hvvr_texture* texture) {
    if (!rc) return fail(HVVR_ERR_INVALID, "NULL raycaster");
    for (auto it = rc->textures.begin(); it != rc->textures.end(); ++it) {
        if (it->get() == texture) {
            CUDA_TRY(cudaSetDevice(rc->spec.device));
            // frames in flight may still read the texture object
            CUDA_TRY(cudaDeviceSynchronize());
            rc->textures.erase(it);
            return uploadTableNow(rc);
        }
    }
    return fail(HVVR_ERR_NOT_FOUND, "texture not owned by this raycaster");
}

int hvvr_texture_get_id(const hvvr_texture* texture, uint32_t* id) {
    if (!texture || !id) return fail(HVVR_ERR_INVALID, "NULL argument");
    *id = texture->id;
    return HVVR_OK;
}

int hvvr_texture_read_level(const hvvr_texture* texture, uint32_t level, void* data, uint64_t capacity,
                            uint32_t* width, uint32_t* height) {
    if (!texture || !width || !height) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (level >= texture->levels) return fail(HVVR_ERR_INVALID, "level %u of %u", level, texture->levels);
    const uint32_t w = std::max(1u, texture->width >> level), h = std::max(1u, texture->height >> level);
    *width = w;
    *height = h;
    if (!data) return HVVR_OK;
    const size_t row = size_t(w) * texture->elementSize;
    if (capacity < row * h) return fail(HVVR_ERR_INVALID, "capacity below %zu bytes", row * h);
    CUDA_TRY(cudaSetDevice(texture->rc->spec.device));
    cudaArray_t a = nullptr;
    CUDA_TRY(cudaGetMipmappedArrayLevel(&a, texture->array, level));
    CUDA_TRY(cudaMemcpy2DFromArrayAsync(data, row, a, 0, 0, row, h, cudaMemcpyDeviceToHost, texture->rc->stream));
    CUDA_TRY(cudaStreamSynchronize(texture->rc->stream));
    return HVVR_OK;
}

int hvvr_texture_sample(const hvvr_texture* texture, uint32_t count, const float* q, float* rgba) {
    if (!texture || (count && (!q || !rgba))) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (count == 0) return HVVR_OK;
    hvvr_raycaster* rc = texture->rc;
    CUDA_TRY(cudaSetDevice(rc->spec.device));
    DevBuf<float> dq;
    DevBuf<float4> dout;
    TRY(dq.upload(q, size_t(count) * 6, rc->stream));
    TRY(dout.alloc(count));
    CUDA_TRY(launchTextureSample(texture->object, count, dq.p, dout.p, rc->stream));
    CUDA_TRY(cudaMemcpyAsync(rgba, dout.p, size_t(count) * sizeof(float4), cudaMemcpyDeviceToHost, rc->stream));
    CUDA_TRY(cudaStreamSynchronize(rc->stream));
    return HVVR_OK;
}

} // extern "C"
