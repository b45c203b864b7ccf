// scene_file.cpp - the reference's binary scene and sample files (host only).
//
// Scene files restate model_import::loadBin / saveBin (libraries/hvvr/samples_shared/
// model_import_bin.cpp:15-168): a 16-byte header {version = 1, texture count, light count,
// mesh count}; per texture a 16-byte record {TextureFormat, width, height, stride in elements}
// followed by its texels (getTextureSize, libraries/hvvr/raycaster/texture.h:56-76); the lights
// as LightUnion records; per mesh a 48-byte record {transform, vertex, triangle, node and
// material counts} followed by those four arrays. Every record is the reference's struct byte
// for byte (the hvvr_* types of the C ABI have the same layouts), so files written by either
// side load in the other.
//
// Sample files restate loadSamples / saveSamples (libraries/hvvr/raycaster/samples.cpp:161-187,
// header libraries/hvvr/raycaster/samples.h:40-45): {magic 0x0CD1, version 0, reserved, count}
// followed by the samples.
//
// Unlike the reference, a short read, a wrong version or magic, or an unknown texture format is
// an error (HVVR_ERR_INVALID / HVVR_ERR_NOT_FOUND), never a silent partial load.
#include <stdio.h>
#include <string.h>

#include <memory>
#include <vector>

#include "host_objects.h"

namespace {

struct BinHeader {
    uint32_t version, textureCount, lightCount, meshCount;
};
struct BinTexture {
    uint32_t format, width, height, stride;
};
struct BinMesh {
    hvvr_transform transform;
    uint32_t vertexCount, triangleCount, nodeCount, materialCount;
};
struct SampleFileHeader {
    uint32_t magic, version, reserved0, sampleCount;
};
static_assert(sizeof(BinHeader) == 16 && sizeof(BinTexture) == 16 && sizeof(BinMesh) == 48, "bin records");
static_assert(sizeof(SampleFileHeader) == 16 && sizeof(hvvr_sample) == 28, "sample file records");
static_assert(sizeof(hvvr_light_union) == 56 && sizeof(hvvr_shading_vertex) == 32 && sizeof(hvvr_tri_shade) == 16 &&
                  sizeof(hvvr_material) == 64,
              "scene records");

constexpr uint32_t kBinVersion = 1;
constexpr uint32_t kSampleMagic = 0x0CD1, kSampleVersion = 0;

// bytes per texel of the reference's TextureFormat values 1..7 (0 = none)
uint64_t texelBytes(uint32_t format) {
    switch (format) {
    case 1: case 2: return 4;   // r8g8b8a8_unorm_srgb, r8g8b8a8_unorm
    case 3: return 8;           // r16g16b16a16_unorm
    case 4: return 16;          // r32g32b32a32_float
    case 5: return 8;           // r16g16b16a16_float
    case 6: case 7: return 4;   // r11g11b10_float, r32_float
    default: return 0;
    }
}

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
    bool read(void* dst, size_t bytes) { return bytes == 0 || fread(dst, 1, bytes, f) == bytes; }
    bool write(const void* src, size_t bytes) { return bytes == 0 || fwrite(src, 1, bytes, f) == bytes; }
};

} // namespace

struct hvvr_scene_file {
    struct Texture {
        BinTexture desc;
        std::vector<uint8_t> texels;
    };
    struct Mesh {
        hvvr_transform transform;
        std::vector<hvvr_shading_vertex> verts;
        std::vector<hvvr_tri_shade> triShade;
        std::vector<hvvr_topology_node> nodes;
        std::vector<hvvr_material> materials;
    };
    std::vector<Texture> textures;
    std::vector<hvvr_light_union> lights;
    std::vector<Mesh> meshes;
};

extern "C" {

int hvvr_scene_file_load(const char* path, hvvr_scene_file** out) {
    if (!path || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    *out = nullptr;
    File fl;
    fl.f = fopen(path, "rb");
    if (!fl.f) return fail(HVVR_ERR_NOT_FOUND, "cannot open scene file %s", path);
    BinHeader h{};
    if (!fl.read(&h, sizeof(h))) return fail(HVVR_ERR_INVALID, "%s: truncated header", path);
    if (h.version != kBinVersion) return fail(HVVR_ERR_INVALID, "%s: bin file version %u, expected %u", path, h.version, kBinVersion);
    auto sf = std::make_unique<hvvr_scene_file>();
    sf->textures.resize(h.textureCount);
    for (uint32_t n = 0; n < h.textureCount; n++) {
        auto& t = sf->textures[n];
        if (!fl.read(&t.desc, sizeof(t.desc))) return fail(HVVR_ERR_INVALID, "%s: truncated texture %u", path, n);
        const uint64_t tb = texelBytes(t.desc.format);
        if (!tb) return fail(HVVR_ERR_INVALID, "%s: texture %u has unknown format %u", path, n, t.desc.format);
        t.texels.resize(size_t(uint64_t(t.desc.stride) * t.desc.height * tb));
        if (!fl.read(t.texels.data(), t.texels.size())) return fail(HVVR_ERR_INVALID, "%s: truncated texels of texture %u", path, n);
    }
    sf->lights.resize(h.lightCount);
    if (!fl.read(sf->lights.data(), sf->lights.size() * sizeof(hvvr_light_union)))
        return fail(HVVR_ERR_INVALID, "%s: truncated lights", path);
    sf->meshes.resize(h.meshCount);
    for (uint32_t n = 0; n < h.meshCount; n++) {
        BinMesh bm{};
        if (!fl.read(&bm, sizeof(bm))) return fail(HVVR_ERR_INVALID, "%s: truncated mesh %u", path, n);
        auto& m = sf->meshes[n];
        m.transform = bm.transform;
        m.verts.resize(bm.vertexCount);
        m.triShade.resize(bm.triangleCount);
        m.nodes.resize(bm.nodeCount);
        m.materials.resize(bm.materialCount);
        if (!fl.read(m.verts.data(), m.verts.size() * sizeof(hvvr_shading_vertex)) ||
            !fl.read(m.triShade.data(), m.triShade.size() * sizeof(hvvr_tri_shade)) ||
            !fl.read(m.nodes.data(), m.nodes.size() * sizeof(hvvr_topology_node)) ||
            !fl.read(m.materials.data(), m.materials.size() * sizeof(hvvr_material)))
            return fail(HVVR_ERR_INVALID, "%s: truncated arrays of mesh %u", path, n);
    }
    *out = sf.release();
    return HVVR_OK;
}

int hvvr_scene_file_counts(const hvvr_scene_file* f, uint32_t* textures, uint32_t* lights, uint32_t* meshes) {
    if (!f) return fail(HVVR_ERR_INVALID, "NULL scene file");
    if (textures) *textures = uint32_t(f->textures.size());
    if (lights) *lights = uint32_t(f->lights.size());
    if (meshes) *meshes = uint32_t(f->meshes.size());
    return HVVR_OK;
}

int hvvr_scene_file_mesh(const hvvr_scene_file* f, uint32_t i, hvvr_mesh_data* mesh, hvvr_transform* xf) {
    if (!f) return fail(HVVR_ERR_INVALID, "NULL scene file");
    if (i >= f->meshes.size()) return fail(HVVR_ERR_INVALID, "mesh %u out of range", i);
    const auto& m = f->meshes[i];
    if (mesh) {
        mesh->verts = m.verts.data();
        mesh->vert_count = uint32_t(m.verts.size());
        mesh->tri_shade = m.triShade.data();
        mesh->tri_count = uint32_t(m.triShade.size());
        mesh->nodes = m.nodes.data();
        mesh->node_count = uint32_t(m.nodes.size());
        mesh->materials = m.materials.data();
        mesh->material_count = uint32_t(m.materials.size());
    }
    if (xf) *xf = m.transform;
    return HVVR_OK;
}

int hvvr_scene_file_light(const hvvr_scene_file* f, uint32_t i, hvvr_light_union* light) {
    if (!f || !light) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (i >= f->lights.size()) return fail(HVVR_ERR_INVALID, "light %u out of range", i);
    *light = f->lights[i];
    return HVVR_OK;
}

int hvvr_scene_file_texture(const hvvr_scene_file* f, uint32_t i, uint32_t* format, uint32_t* width, uint32_t* height,
                            uint32_t* stride, const void** texels, uint64_t* bytes) {
    if (!f) return fail(HVVR_ERR_INVALID, "NULL scene file");
    if (i >= f->textures.size()) return fail(HVVR_ERR_INVALID, "texture %u out of range", i);
    const auto& t = f->textures[i];
    if (format) *format = t.desc.format;
    if (width) *width = t.desc.width;
    if (height) *height = t.desc.height;
    if (stride) *stride = t.desc.stride;
    if (texels) *texels = t.texels.data();
    if (bytes) *bytes = t.texels.size();
    return HVVR_OK;
}

void hvvr_scene_file_close(hvvr_scene_file* f) { delete f; }

int hvvr_scene_file_save(const char* path, const hvvr_texture_data* textures, uint32_t texture_count,
                         const hvvr_mesh_data* meshes, const hvvr_transform* transforms, uint32_t mesh_count,
                         const hvvr_light_union* lights, uint32_t light_count) {
    if (!path || (texture_count && !textures) || (mesh_count && (!meshes || !transforms)) || (light_count && !lights))
        return fail(HVVR_ERR_INVALID, "NULL argument");
    for (uint32_t n = 0; n < texture_count; n++) {
        if (!texelBytes(textures[n].format)) return fail(HVVR_ERR_INVALID, "texture %u: unknown format", n);
        if (!textures[n].data && textures[n].stride_elements && textures[n].height)
            return fail(HVVR_ERR_INVALID, "texture %u: no texels", n);
    }
    File fl;
    fl.f = fopen(path, "wb");
    if (!fl.f) return fail(HVVR_ERR_NOT_FOUND, "cannot create scene file %s", path);
    const BinHeader h{kBinVersion, texture_count, light_count, mesh_count};
    bool ok = fl.write(&h, sizeof(h));
    // per texture its record and getTextureSize(stride, height, format) bytes of texels
    for (uint32_t n = 0; ok && n < texture_count; n++) {
        const hvvr_texture_data& t = textures[n];
        const BinTexture bt{t.format, t.width, t.height, t.stride_elements};
        ok = fl.write(&bt, sizeof(bt)) && fl.write(t.data, uint64_t(t.stride_elements) * t.height * texelBytes(t.format));
    }
    ok = ok && fl.write(lights, size_t(light_count) * sizeof(hvvr_light_union));
    for (uint32_t n = 0; ok && n < mesh_count; n++) {
        const hvvr_mesh_data& m = meshes[n];
        const BinMesh bm{transforms[n], m.vert_count, m.tri_count, m.node_count, m.material_count};
        ok = fl.write(&bm, sizeof(bm)) && fl.write(m.verts, size_t(m.vert_count) * sizeof(hvvr_shading_vertex)) &&
             fl.write(m.tri_shade, size_t(m.tri_count) * sizeof(hvvr_tri_shade)) &&
             fl.write(m.nodes, size_t(m.node_count) * sizeof(hvvr_topology_node)) &&
             fl.write(m.materials, size_t(m.material_count) * sizeof(hvvr_material));
    }
    if (!ok) return fail(HVVR_ERR_INVALID, "%s: write failed", path);
    return HVVR_OK;
}

int hvvr_samples_load(const char* path, hvvr_sample* samples, uint32_t capacity, uint32_t* count) {
    if (!path || !count) return fail(HVVR_ERR_INVALID, "NULL argument");
    File fl;
    fl.f = fopen(path, "rb");
    if (!fl.f) return fail(HVVR_ERR_NOT_FOUND, "cannot open sample file %s", path);
    SampleFileHeader h{};
    if (!fl.read(&h, sizeof(h))) return fail(HVVR_ERR_INVALID, "%s: truncated header", path);
    if (h.magic != kSampleMagic || h.version != kSampleVersion)
        return fail(HVVR_ERR_INVALID, "%s: not a sample file (magic 0x%x, version %u)", path, h.magic, h.version);
    *count = h.sampleCount;
    if (!samples) return HVVR_OK;
    if (capacity < h.sampleCount) return fail(HVVR_ERR_INVALID, "%s holds %u samples, capacity %u", path, h.sampleCount, capacity);
    if (!fl.read(samples, size_t(h.sampleCount) * sizeof(hvvr_sample))) return fail(HVVR_ERR_INVALID, "%s: truncated samples", path);
    return HVVR_OK;
}

int hvvr_samples_save(const char* path, const hvvr_sample* samples, uint32_t count) {
    if (!path || (count && !samples)) return fail(HVVR_ERR_INVALID, "NULL argument");
    File fl;
    fl.f = fopen(path, "wb");
    if (!fl.f) return fail(HVVR_ERR_NOT_FOUND, "cannot create sample file %s", path);
    const SampleFileHeader h{kSampleMagic, kSampleVersion, 0, count};
    if (!fl.write(&h, sizeof(h)) || !fl.write(samples, size_t(count) * sizeof(hvvr_sample)))
        return fail(HVVR_ERR_INVALID, "%s: write failed", path);
    return HVVR_OK;
}

} // extern "C"
