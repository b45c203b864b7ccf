/*
 * hvvr.hpp - C++ facade with the reference's class names and signatures, over the C ABI in
 * hvvr_c.h (header-only; link libhvvr_b200.so).
 *
 * A caller written against the reference's Raycaster / Camera / Model / Light / Texture classes
 * (libraries/hvvr/raycaster/raycaster.h:38-115, camera.h:51-146, model.h:26-57) compiles against
 * these declarations: same class names in namespace hvvr, same method names, argument order and
 * meaning, and the reference's value types (FloatRect, ThinLens, transform, Sample, MeshData,
 * LightUnion, TextureData, ImageResourceDescriptor, RayCasterSpecification) as layout-identical
 * aliases or thin structs. The raycaster owns every object it creates and hands out raw pointers,
 * as the reference does (libraries/hvvr/raycaster/raycaster.cpp:78-91).
 *
 * Differences, all from the boundary's error model and target:
 *   - where the reference exits the process (fail(), cutilSafeCall) or asserts, these methods
 *     throw hvvr::Error carrying the C status code and message;
 *   - ImageResourceDescriptor holds CPU_MEMORY or CUDA_MEMORY only (no graphics API here), and
 *     RayCasterSpecification::outputTo3DApi defaults to false;
 *   - Camera::setMsaa selects the MSAA rate at run time (the reference fixes it at compile time,
 *     libraries/hvvr/raycaster/raycaster_common.h:27); the default is 16 as there.
 */
#ifndef HVVR_HPP
#define HVVR_HPP

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "hvvr_c.h"

namespace hvvr {

// ------------------------------------------------------------------ errors
class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), _code(code) {}
    int code() const { return _code; }

private:
    int _code;
};

inline void check(int rc, const char* call) {
    if (rc != HVVR_OK) throw Error(rc, std::string(call) + ": " + hvvr_last_error());
}

// ------------------------------------------------------------------ value types
// (libraries/hvvr/shared/vector_math.h, graphics_types.h; layouts as in hvvr_c.h)
struct vector2 : hvvr_vec2 {
    vector2() : hvvr_vec2{0.0f, 0.0f} {}
    vector2(float x_, float y_) : hvvr_vec2{x_, y_} {}
};
struct vector3 : hvvr_vec3 {
    vector3() : hvvr_vec3{0.0f, 0.0f, 0.0f} {}
    vector3(float x_, float y_, float z_) : hvvr_vec3{x_, y_, z_} {}
};
struct vector4 : hvvr_vec4 {
    vector4() : hvvr_vec4{0.0f, 0.0f, 0.0f, 0.0f} {}
    vector4(float x_, float y_, float z_, float w_) : hvvr_vec4{x_, y_, z_, w_} {}
};
// quaternion (x, y, z, w)
struct quaternion : hvvr_vec4 {
    quaternion() : hvvr_vec4{0.0f, 0.0f, 0.0f, 1.0f} {}
    quaternion(float x_, float y_, float z_, float w_) : hvvr_vec4{x_, y_, z_, w_} {}
};
// transform {rotation, translation, scale} (vector_math.h:966-969)
struct transform : hvvr_transform {
    transform() : hvvr_transform{{0.0f, 0.0f, 0.0f, 1.0f}, {0.0f, 0.0f, 0.0f}, 1.0f} {}
    transform(const vector3& t, const quaternion& r, float s) : hvvr_transform{r, t, s} {}
    static transform identity() { return transform(); }
};
// FloatRect {lower, upper} (graphics_types.h:27-32)
struct FloatRect : hvvr_float_rect {
    FloatRect() : hvvr_float_rect{{0.0f, 0.0f}, {0.0f, 0.0f}} {}
    FloatRect(const vector2& lower_, const vector2& upper_) : hvvr_float_rect{lower_, upper_} {}
};
// ThinLens {radius, focalDistance} (graphics_types.h:170-173)
struct ThinLens {
    float radius;
    float focalDistance;
};
static_assert(sizeof(ThinLens) == sizeof(hvvr_thin_lens), "ThinLens layout");

using Sample = hvvr_sample;                     // samples.h:17-29
using ShadingVertex = hvvr_shading_vertex;      // graphics_types.h:83-88
using PrecomputedTriangleShade = hvvr_tri_shade; // graphics_types.h:208-211
using TopologyNode = hvvr_topology_node;        // graphics_types.h:126-151
using SimpleMaterial = hvvr_material;           // material.h:22-49

// LightType and the light structs with the reference's member names (light.h:17-59); LightUnion
// is byte-compatible with hvvr_light_union
enum class LightType : uint32_t {
    none = HVVR_LIGHT_NONE,
    directional = HVVR_LIGHT_DIRECTIONAL,
    point = HVVR_LIGHT_POINT,
    spot = HVVR_LIGHT_SPOT
};
struct LightDirectional {
    vector3 Direction;
    vector3 Power;
};
struct LightPoint {
    vector3 Position;
    float FalloffEnd;
    vector3 Color;
    float FalloffScale;
};
struct LightSpot {
    vector3 Position;
    float FalloffEnd;
    vector3 Direction;
    float FalloffScale;
    vector3 Color;
    float CosOuterAngle;
    float CosAngleScale;
};
struct LightUnion {
    LightType type;
    union {
        LightDirectional directional;
        LightPoint point;
        LightSpot spot;
    };
    LightUnion() : type(LightType::none), spot() {}
};
static_assert(sizeof(LightUnion) == sizeof(hvvr_light_union), "LightUnion layout");

// MeshData (model.h:26-31)
struct MeshData {
    std::vector<ShadingVertex> verts;
    std::vector<PrecomputedTriangleShade> triShade;
    std::vector<TopologyNode> nodes;
    std::vector<SimpleMaterial> materials;
};

// TextureFormat / TextureData (texture.h:16-34)
enum class TextureFormat : uint32_t {
    none = HVVR_TEXTURE_NONE,
    r8g8b8a8_unorm_srgb = HVVR_TEXTURE_RGBA8_UNORM_SRGB,
    r8g8b8a8_unorm = HVVR_TEXTURE_RGBA8_UNORM,
    r16g16b16a16_unorm = HVVR_TEXTURE_RGBA16_UNORM,
    r32g32b32a32_float = HVVR_TEXTURE_RGBA32_FLOAT,
    r16g16b16a16_float = HVVR_TEXTURE_RGBA16_FLOAT,
    r11g11b10_float = HVVR_TEXTURE_R11G11B10_FLOAT,
    r32_float = HVVR_TEXTURE_R32_FLOAT
};
struct TextureData {
    const uint8_t* data = nullptr;
    TextureFormat format = TextureFormat::none;
    uint32_t width = 0;
    uint32_t height = 0;
    uint32_t strideElements = 0;
};

// ImageResourceDescriptor (graphics_types.h:56-80): CPU or CUDA memory, RGBA8 sRGB
struct ImageResourceDescriptor {
    enum class MemoryType : uint32_t { CPU_MEMORY = HVVR_MEMORY_CPU, CUDA_MEMORY = HVVR_MEMORY_CUDA };
    MemoryType memoryType = MemoryType::CPU_MEMORY;
    void* data = nullptr;
    uint32_t width = 0;
    uint32_t height = 0;
    size_t stride = 0; // pixels; 0 = width
};

// RayCasterSpecification (raycaster_spec.h:22-50)
enum class RaycasterOutputFormat { COLOR_RGBA8 };
enum class RayCasterGPUMode {
    GPU_INTERSECT_AND_RECONSTRUCT_DEFERRED_MSAA_RESOLVE,
    GPU_FOVEATED_POLAR_SPACE_CUDA_RECONSTRUCT
};
struct RayCasterSpecification {
    RayCasterGPUMode mode = RayCasterGPUMode::GPU_INTERSECT_AND_RECONSTRUCT_DEFERRED_MSAA_RESOLVE;
    size_t threadCount = 0;
    struct FoveatedSamplePattern {
        float degreeTrackingError = 0.5f;
        float maxFOVDegrees = 110.0f;
        float marSlope = 0.022f;
        float fovealMARDegrees = 1.0f / 60.0f;
    } foveatedSamplePattern;
    RaycasterOutputFormat outputFormat = RaycasterOutputFormat::COLOR_RGBA8;
    bool outputTo3DApi = false;

    static RayCasterSpecification feb2017FoveatedDemoSettings() {
        RayCasterSpecification spec;
        spec.mode = RayCasterGPUMode::GPU_FOVEATED_POLAR_SPACE_CUDA_RECONSTRUCT;
        spec.foveatedSamplePattern.degreeTrackingError = 7.0f;
        spec.foveatedSamplePattern.fovealMARDegrees = 1.0f / 20.0f;
        spec.foveatedSamplePattern.marSlope = 0.015f;
        spec.foveatedSamplePattern.maxFOVDegrees = 90.0f;
        return spec;
    }
};

class Raycaster;

// ------------------------------------------------------------------ objects
// Model (model.h:33-57): owned by its Raycaster; keeps the mesh it was created from
class Model {
public:
    const MeshData& getMesh() const { return _meshData; }
    void setTransform(const transform& xf) {
        check(hvvr_model_set_transform(_handle, &xf), "Model::setTransform");
        _transform = xf;
    }
    const transform& getTransform() const { return _transform; }
    hvvr_model* handle() const { return _handle; }

    Model(const Model&) = delete;
    Model& operator=(const Model&) = delete;

private:
    friend class Raycaster;
    Model(hvvr_model* h, MeshData&& mesh) : _handle(h), _meshData(std::move(mesh)) {}
    hvvr_model* _handle;
    MeshData _meshData;
    transform _transform;
};

// Light (light.h:61-77)
class Light {
public:
    const LightUnion& getLightUnion() const { return _lightUnion; }
    hvvr_light* handle() const { return _handle; }

    Light(const Light&) = delete;
    Light& operator=(const Light&) = delete;

private:
    friend class Raycaster;
    Light(hvvr_light* h, const LightUnion& l) : _handle(h), _lightUnion(l) {}
    hvvr_light* _handle;
    LightUnion _lightUnion;
};

// Texture (texture.h:38-60)
class Texture {
public:
    uint32_t getID() const {
        uint32_t id = 0;
        check(hvvr_texture_get_id(_handle, &id), "Texture::getID");
        return id;
    }
    hvvr_texture* handle() const { return _handle; }

    Texture(const Texture&) = delete;
    Texture& operator=(const Texture&) = delete;

private:
    friend class Raycaster;
    explicit Texture(hvvr_texture* h) : _handle(h) {}
    hvvr_texture* _handle;
};

// Camera (camera.h:51-146): owned by its Raycaster
class Camera {
public:
    void setEnabled(bool enabled) {
        check(hvvr_camera_set_enabled(_handle, enabled ? 1 : 0), "Camera::setEnabled");
        _enabled = enabled;
    }
    bool getEnabled() const { return _enabled; }

    void setEyeDir(const vector3& eyeDir) {
        check(hvvr_camera_set_eye_dir(_handle, &eyeDir), "Camera::setEyeDir");
        _eyeDir = eyeDir;
    }
    const vector3& getEyeDir() const { return _eyeDir; }

    void setViewport(const FloatRect& viewport) {
        check(hvvr_camera_set_viewport(_handle, &viewport), "Camera::setViewport");
        _viewport = viewport;
    }
    const FloatRect& getViewport() const { return _viewport; }

    void setLens(const ThinLens& lens) {
        const hvvr_thin_lens l{lens.radius, lens.focalDistance};
        check(hvvr_camera_set_lens(_handle, &l), "Camera::setLens");
        _lens = lens;
    }
    const ThinLens& getLens() const { return _lens; }
    void setAperture(float radius) {
        check(hvvr_camera_set_aperture(_handle, radius), "Camera::setAperture");
        _lens.radius = radius;
    }
    float getAperture() const { return _lens.radius; }
    void setFocalDepth(float depth) {
        check(hvvr_camera_set_focal_depth(_handle, depth), "Camera::setFocalDepth");
        _lens.focalDistance = depth;
    }

    void setRenderTarget(const ImageResourceDescriptor& target) {
        hvvr_image_desc d{};
        d.pixel_format = HVVR_PIXEL_RGBA8_SRGB;
        d.memory_type = uint32_t(target.memoryType);
        d.data = target.data;
        d.width = target.width;
        d.height = target.height;
        d.stride = target.stride;
        check(hvvr_camera_set_render_target(_handle, &d), "Camera::setRenderTarget");
    }
    void setSamples(const Sample* rawSamples, uint32_t rawSampleCount, uint32_t splitColorSamples) {
        check(hvvr_camera_set_samples(_handle, rawSamples, rawSampleCount, splitColorSamples), "Camera::setSamples");
    }
    // a spherical section for ray generation instead of the perspective transform (0, 0: off)
    void setSphericalWarpSettings(float fovXDegrees, float fovYDegrees) {
        check(hvvr_camera_set_spherical_warp(_handle, fovXDegrees, fovYDegrees), "Camera::setSphericalWarpSettings");
    }
    uint32_t getSampleCount() const {
        uint32_t n = 0;
        check(hvvr_camera_get_sample_count(_handle, &n), "Camera::getSampleCount");
        return n;
    }

    void setCameraToWorld(const transform& cameraToWorld) {
        check(hvvr_camera_set_camera_to_world(_handle, &cameraToWorld), "Camera::setCameraToWorld");
        _cameraToWorld = cameraToWorld;
    }
    const vector3& getTranslation() const { return static_cast<const vector3&>(_cameraToWorld.translation); }

    // Camera::extractImage (camera.h:57): the reference copies the device image into a CPU_MEMORY
    // render target here; Raycaster::render already returns with CPU targets complete, so nothing
    // is left to do
    void extractImage() {}
    // Camera::advanceJitter (camera.cpp:205-209): the reference steps a per-frame jitter that only
    // spins the MSAA pattern under JITTER_SAMPLES, which its build sets to 0
    // (kernel_constants.h:17); the image does not depend on it
    void advanceJitter() {}

    // additions: the MSAA rate (1, 2, 4, 8, 16 or 32; default 16) and an eager sample setup
    void setMsaa(uint32_t rate) { check(hvvr_camera_set_msaa(_handle, rate), "Camera::setMsaa"); }
    void setMsaaPattern(uint32_t pattern) { check(hvvr_camera_set_msaa_pattern(_handle, pattern), "Camera::setMsaaPattern"); }
    void prepare() { check(hvvr_camera_prepare(_handle, nullptr), "Camera::prepare"); }
    hvvr_camera* handle() const { return _handle; }

    Camera(const Camera&) = delete;
    Camera& operator=(const Camera&) = delete;

private:
    friend class Raycaster;
    Camera(hvvr_camera* h, const FloatRect& viewport, float apertureRadius)
        : _handle(h), _viewport(viewport), _lens{apertureRadius, 1.0f} {}
    hvvr_camera* _handle;
    bool _enabled = true;
    vector3 _eyeDir;
    FloatRect _viewport;
    ThinLens _lens;
    transform _cameraToWorld;
};

// Raycaster (raycaster.h:38-115)
class Raycaster {
public:
    explicit Raycaster(const RayCasterSpecification& spec) {
        if (spec.outputTo3DApi)
            throw Error(HVVR_ERR_INVALID, "Raycaster: no graphics API here (outputTo3DApi must be false)");
        hvvr_spec s;
        hvvr_spec_default(&s);
        s.mode = spec.mode == RayCasterGPUMode::GPU_FOVEATED_POLAR_SPACE_CUDA_RECONSTRUCT ? HVVR_MODE_FOVEATED_POLAR
                                                                                        : HVVR_MODE_DEFERRED_MSAA_RESOLVE;
        s.thread_count = uint32_t(spec.threadCount);
        s.foveated_degree_tracking_error = spec.foveatedSamplePattern.degreeTrackingError;
        s.foveated_max_fov_degrees = spec.foveatedSamplePattern.maxFOVDegrees;
        s.foveated_mar_slope = spec.foveatedSamplePattern.marSlope;
        s.foveated_foveal_mar_degrees = spec.foveatedSamplePattern.fovealMARDegrees;
        s.output_to_3d_api = 0;
        check(hvvr_raycaster_create(&s, &_handle), "Raycaster::Raycaster");
    }
    ~Raycaster() {
        // objects go with the raycaster, as the reference's unique_ptr members do
        _cameras.clear();
        _models.clear();
        _lights.clear();
        _textures.clear();
        if (_handle) hvvr_raycaster_destroy(_handle);
    }
    Raycaster(const Raycaster&) = delete;
    Raycaster& operator=(const Raycaster&) = delete;

    //// scene management
    Camera* createCamera(const FloatRect& viewport, float apertureRadius) {
        hvvr_camera* h = nullptr;
        check(hvvr_camera_create(_handle, &viewport, apertureRadius, &h), "Raycaster::createCamera");
        _cameras.emplace_back(new Camera(h, viewport, apertureRadius));
        return _cameras.back().get();
    }
    void destroyCamera(Camera* camera) {
        check(hvvr_camera_destroy(_handle, camera ? camera->_handle : nullptr), "Raycaster::destroyCamera");
        erase(_cameras, camera);
    }

    Texture* createTexture(const TextureData& textureData) {
        const hvvr_texture_data d{textureData.data, uint32_t(textureData.format), textureData.width,
                                  textureData.height, textureData.strideElements};
        hvvr_texture* h = nullptr;
        check(hvvr_texture_create(_handle, &d, &h), "Raycaster::createTexture");
        _textures.emplace_back(new Texture(h));
        return _textures.back().get();
    }
    void destroyTexture(Texture* texture) {
        check(hvvr_texture_destroy(_handle, texture ? texture->_handle : nullptr), "Raycaster::destroyTexture");
        erase(_textures, texture);
    }

    Light* createLight(const LightUnion& lightUnion) {
        hvvr_light* h = nullptr;
        check(hvvr_light_create(_handle, reinterpret_cast<const hvvr_light_union*>(&lightUnion), &h),
              "Raycaster::createLight");
        _lights.emplace_back(new Light(h, lightUnion));
        return _lights.back().get();
    }
    void destroyLight(Light* light) {
        check(hvvr_light_destroy(_handle, light ? light->_handle : nullptr), "Raycaster::destroyLight");
        erase(_lights, light);
    }

    // MeshData with an empty nodes array gets its topology built by the library
    Model* createModel(MeshData&& meshData) {
        const hvvr_mesh_data md{meshData.verts.data(),     uint32_t(meshData.verts.size()),
                                meshData.triShade.data(),  uint32_t(meshData.triShade.size()),
                                meshData.nodes.data(),     uint32_t(meshData.nodes.size()),
                                meshData.materials.data(), uint32_t(meshData.materials.size())};
        hvvr_model* h = nullptr;
        check(hvvr_model_create(_handle, &md, &h), "Raycaster::createModel");
        _models.emplace_back(new Model(h, std::move(meshData)));
        return _models.back().get();
    }
    Model* createModel(const MeshData& meshData) { return createModel(MeshData(meshData)); }
    void destroyModel(Model* model) {
        check(hvvr_model_destroy(_handle, model ? model->_handle : nullptr), "Raycaster::destroyModel");
        erase(_models, model);
    }

    void setSceneDirty() { check(hvvr_raycaster_set_scene_dirty(_handle), "Raycaster::setSceneDirty"); }

    //// rendering: every enabled camera; CPU_MEMORY targets are complete on return
    void render(double elapsedTime) { check(hvvr_raycaster_render(_handle, elapsedTime, nullptr), "Raycaster::render"); }

    // additions: wait for the enqueued work; the C handle
    void synchronize() { check(hvvr_raycaster_synchronize(_handle), "Raycaster::synchronize"); }
    hvvr_raycaster* handle() const { return _handle; }

private:
    template <class T>
    static void erase(std::vector<std::unique_ptr<T>>& v, T* p) {
        for (auto it = v.begin(); it != v.end(); ++it)
            if (it->get() == p) {
                v.erase(it);
                return;
            }
    }
    hvvr_raycaster* _handle = nullptr;
    std::vector<std::unique_ptr<Camera>> _cameras;
    std::vector<std::unique_ptr<Texture>> _textures;
    std::vector<std::unique_ptr<Light>> _lights;
    std::vector<std::unique_ptr<Model>> _models;
};

} // namespace hvvr

#endif // HVVR_HPP
