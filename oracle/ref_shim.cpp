// ref_shim.cpp — TEST INFRASTRUCTURE (oracle): a C ABI over the reference engine's own CPU
// path, compiled from the reference sources in place.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load the library built from this file; the product never
// does.  Each entry point drives the reference's public classes exactly as its own code does:
//
//   ref_scene_*      Scene::addShape / addLight / setEnvironment / setShadowCatcher / tagShape,
//                    Light::setLightLink, Scene::buildAccelerator
//                    (src/engine/scene.cpp:18-185), own BVH forced (Scene::setPreferOwnBvh)
//   ref_render       Renderer::renderSamples (src/engine/renderer.cpp:392-531); seed 12345
//   ref_render_seeded  the same tile loop as renderSamples with a caller seed: tracePixel
//                    (renderer.cpp:139-160) → PathTracer::Li → Film::addSample
//   ref_trace_primary  tracePixel's camera ray + Scene::intersect (bvh.cpp:322-401)
//   ref_sobol        SobolSampler (src/samplers/sobol_sampler.cpp:111-146)
//   ref_bsdf_probe   Material::evalPdf / sampleFull (src/materials/*.cpp)
//   ref_light_*      LightSampler::prepare/sample/pmf (src/lights/light_sampler.cpp:150-284)
//   ref_render_guided  renderSamples with RenderSettings::pathGuiding (SD-tree guiding)
//   ref_dtree_probe  DirectionalTree::addSplat / buildFrom / pdf / sample
//                    (src/integrators/path_guiding.cpp:80-222)
#include "photon_cuda.h"

#include "camera/camera.h"
#include "camera/orthographic_camera.h"
#include "camera/perspective_camera.h"
#include "camera/thin_lens_camera.h"
#include "core/image/film.h"
#include "core/image/image.h"
#include "core/image/pixel_filter.h"
#include "engine/renderer.h"
#include "engine/scene.h"
#include "geometry/mesh.h"
#include "geometry/sphere.h"
#include "geometry/mesh_instance.h"
#include "geometry/triangle.h"
#include "integrators/path_guiding.h"
#include "integrators/path_tracer.h"
#include "lights/area_light.h"
#include "lights/environment_light.h"
#include "materials/dielectric.h"
#include "materials/disney.h"
#include "materials/lambertian.h"
#include "materials/mirror.h"
#include "samplers/sobol_sampler.h"
#include "scene/document.h"
#include "scene/project_io.h"
#include "scene/scene_graph.h"
#include <nlohmann/json.hpp>
#ifdef PE_WITH_ADAPTER
#include "engine/render_session.h"
#include "adapter/cuda_render_device.h"
#include <cstdio>
#endif

#include <atomic>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace photon;

namespace {

Vec3f v3(const float* p) { return Vec3f(p[0], p[1], p[2]); }
Color3f c3(const float* p) { return Color3f(p[0], p[1], p[2]); }

// Camera whose rays are exactly PerspectiveCamera::generateRay for the given GPU description
// (perspective_camera.cpp:36-40); cone helpers come from Camera (camera.h:95-110).
class DescCamera : public Camera {
public:
    explicit DescCamera(const pe_camera& c) {
        m_d.position = v3(c.position);
        m_d.lowerLeft = v3(c.lower_left);
        m_d.horizontal = v3(c.horizontal);
        m_d.vertical = v3(c.vertical);
        m_d.u = v3(c.u);
        m_d.v = v3(c.v);
        m_d.forward = v3(c.forward);
        m_d.lensRadius = 0.0f;
        m_d.orthographic = false;
        if (c.has_shutter_end) setShutterEnd(endDesc(c));
    }
    // Camera::setShutterEnd's description from the pe_camera's end fields.
    static CameraGpuDesc endDesc(const pe_camera& c) {
        CameraGpuDesc e;
        e.position = v3(c.end_position);
        e.lowerLeft = v3(c.end_lower_left);
        e.horizontal = v3(c.end_horizontal);
        e.vertical = v3(c.end_vertical);
        e.u = v3(c.end_u);
        e.v = v3(c.end_v);
        e.forward = v3(c.end_forward);
        e.lensRadius = c.end_lens_radius;
        e.orthographic = c.orthographic != 0;
        return e;
    }
    Ray generateRay(float u, float v, const Vec2f&) const override {
        Vec3f targetPoint = m_d.lowerLeft + u * m_d.horizontal + v * m_d.vertical;
        Vec3f direction = (targetPoint - m_d.position).normalized();
        return Ray(m_d.position, direction);
    }
    CameraGpuDesc describeGpu() const override { return m_d; }

private:
    CameraGpuDesc m_d;
};

struct RefScene;
struct RefBlas {
    std::shared_ptr<TriangleMesh> mesh;
};

struct RefScene {
    std::shared_ptr<Scene> holder;
    Scene& scene;
    RefScene() : holder(std::make_shared<Scene>()), scene(*holder) {}
    explicit RefScene(std::shared_ptr<Scene> s) : holder(std::move(s)), scene(*holder) {}
    std::vector<std::shared_ptr<Material>> materials;
    std::unordered_map<const void*, int> shapeIndex; // hitObject → insertion index
    int nextShape = 0;
    std::string envGroup; // the environment's light group, applied at build
    std::vector<std::shared_ptr<Image>> textures; // ref_scene_add_texture
    std::vector<std::shared_ptr<TriangleMesh>> blases; // ref_scene_add_blas
    uint64_t id = ++counter;                            // unique over the process's RefScenes
    static inline uint64_t counter = 0;
    void indexNewShapes() {
        const auto& shapes = scene.shapes();
        for (size_t i = static_cast<size_t>(nextShape); i < shapes.size(); ++i)
            shapeIndex[shapes[i].get()] = static_cast<int>(i);
        nextShape = static_cast<int>(shapes.size());
    }
};

std::shared_ptr<Material> makeMaterial(const pe_material& m) {
    switch (m.type) {
        case PE_MAT_LAMBERT: {
            auto l = std::make_shared<Lambertian>(c3(m.base_color), c3(m.emission));
            l->setRoundEdgeRadius(m.round_edge_radius);
            return l;
        }
        case PE_MAT_DISNEY: {
            auto d = std::make_shared<DisneyMaterial>(c3(m.base_color), m.metallic, m.roughness, m.specular);
            d->setClearCoat(m.clearcoat);
            d->setClearCoatRoughness(m.clearcoat_roughness);
            d->setIor(m.ior);
            d->setSpecularTransmission(m.spec_transmission);
            d->setCoatIor(m.coat_ior);
            d->setCoatTint(c3(m.coat_tint));
            if (m.has_sheen_color) d->setSheenColor(c3(m.sheen_color));
            d->setAnisotropy(m.anisotropy);
            d->setSheen(m.sheen);
            d->setSheenRoughness(m.sheen_roughness);
            d->setDiffuseRoughness(m.diffuse_roughness);
            d->setDiffuseTransmission(m.diffuse_transmission);
            d->setSubsurface(m.subsurface);
            d->setSubsurfaceRadius(c3(m.subsurface_radius));
            d->setSubsurfaceScale(m.subsurface_scale);
            d->setSubsurfaceAnisotropy(m.subsurface_anisotropy);
            d->setEdgeTint(c3(m.edge_tint));
            d->setThinFilm(m.thin_film_thickness, m.thin_film_ior);
            if (m.flake_density > 0.0f) d->setFlakes(m.flake_density, m.flake_size, m.flake_roughness, c3(m.flake_color));
            d->setEmission(c3(m.emission));
            d->setOpacity(m.opacity);
            d->setRoundEdgeRadius(m.round_edge_radius);
            return d;
        }
        case PE_MAT_DIELECTRIC: {
            auto g = std::make_shared<Dielectric>(m.ior, c3(m.base_color), m.glass_roughness);
            g->setAbbe(m.abbe);
            if (m.has_absorption) g->setAbsorption(c3(m.absorb_color), m.absorb_distance);
            if (m.has_scattering) g->setScattering(m.scatter_density, c3(m.scatter_color), m.scatter_anisotropy);
            g->setThinWalled(m.thin_walled != 0);
            g->setThinFilm(m.film_thickness);
            g->setRoundEdgeRadius(m.round_edge_radius);
            return g;
        }
        case PE_MAT_MIRROR: {
            auto mi = std::make_shared<Mirror>(c3(m.base_color));
            mi->setRoundEdgeRadius(m.round_edge_radius);
            return mi;
        }
        default:
            return nullptr;
    }
}

RenderSettings toSettings(const pe_settings& st, int threads) {
    RenderSettings s;
    s.width = st.width;
    s.height = st.height;
    s.samplesPerPixel = 1;
    s.maxBounces = st.max_bounces;
    s.shadowQuality = st.shadow_quality;
    s.filter.type = static_cast<PixelFilterType>(st.filter_type);
    s.filter.width = st.filter_width;
    s.clampIndirect = st.clamp_indirect;
    s.aoStrength = st.ao_strength;
    s.adaptiveSampling = st.adaptive_sampling != 0;
    s.noiseThreshold = st.noise_threshold;
    s.minAdaptiveSamples = st.min_adaptive_samples;
    s.motionBlur = st.motion_blur != 0;
    s.numThreads = threads;
    return s;
}

int hardwareThreads() {
    const unsigned n = std::thread::hardware_concurrency();
    return n > 0 ? static_cast<int>(n) : 1;
}

void exportFilm(const Film& film, int w, int h, float* sum, uint32_t* count) {
    // Film keeps sum/count private; resolvedPixel × count recovers the sum exactly when the
    // caller only needs the mean, so the mean image and the counts are exported instead.
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x);
            const Color3f c = film.resolvedPixel(x, y);
            if (sum) {
                sum[3 * i + 0] = c.r;
                sum[3 * i + 1] = c.g;
                sum[3 * i + 2] = c.b;
            }
            if (count) count[i] = static_cast<uint32_t>(film.sampleCount(x, y));
        }
}

} // namespace

extern "C" {

void* ref_scene_create() {
    Scene::setPreferOwnBvh(true);
    return new RefScene();
}

void ref_scene_destroy(void* s) { delete static_cast<RefScene*>(s); }

// An RGB float image (row 0 first) for the Disney image maps; returns its index.
int32_t ref_scene_add_texture(void* s, const float* rgb, int32_t w, int32_t h) {
    auto* rs = static_cast<RefScene*>(s);
    auto img = std::make_shared<Image>(w, h);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float* px = rgb + 3 * (static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x));
            img->setPixel(x, y, Color3f(px[0], px[1], px[2]));
        }
    rs->textures.push_back(img);
    return static_cast<int32_t>(rs->textures.size() - 1);
}

// Image::createCompact8 (8-bit, sRGB-encoded when srgb != 0) for the Disney image maps.
int32_t ref_scene_add_texture_u8(void* s, const uint8_t* rgb, int32_t w, int32_t h, int32_t srgb) {
    auto* rs = static_cast<RefScene*>(s);
    auto img = std::make_shared<Image>(Image::createCompact8(
        w, h, rgb, srgb ? Image::StorageFormat::U8Srgb : Image::StorageFormat::U8Linear));
    rs->textures.push_back(img);
    return static_cast<int32_t>(rs->textures.size() - 1);
}

// Image::buildMipmaps of texture `i`.
int32_t ref_scene_build_texture_mipmaps(void* s, int32_t i) {
    auto* rs = static_cast<RefScene*>(s);
    if (i < 0 || i >= static_cast<int32_t>(rs->textures.size())) return -1;
    rs->textures[static_cast<size_t>(i)]->buildMipmaps();
    return 0;
}

int32_t ref_scene_add_material(void* s, const pe_material* m) {
    auto* rs = static_cast<RefScene*>(s);
    auto mat = makeMaterial(*m);
    if (!mat) return -1;
    if (m->type == PE_MAT_DISNEY) {
        // image maps, mapping and scale (DisneyMaterial::set*Image / setTextureMapping / setTextureScale)
        auto* d = static_cast<DisneyMaterial*>(mat.get());
        auto tex = [&](int32_t i) -> std::shared_ptr<Image> {
            return i >= 0 && i < static_cast<int32_t>(rs->textures.size()) ? rs->textures[static_cast<size_t>(i)] : nullptr;
        };
        if (auto t = tex(m->albedo_texture)) d->setAlbedoImage(t);
        if (auto t = tex(m->roughness_texture)) d->setRoughnessImage(t);
        if (auto t = tex(m->metalness_texture)) d->setMetalnessImage(t);
        if (auto t = tex(m->normal_texture)) d->setNormalImage(t);
        if (auto t = tex(m->opacity_texture)) d->setOpacityImage(t);
        d->setTextureMapping(m->texture_mapping == 1 ? DisneyMaterial::TextureMapping::Box
                                                     : DisneyMaterial::TextureMapping::UV);
        d->setTextureScale(m->texture_scale);
    }
    rs->materials.push_back(mat);
    rs->scene.retainMaterial(mat);
    return static_cast<int32_t>(rs->materials.size() - 1);
}

int32_t ref_scene_add_mesh(void* s, const float* pos, uint32_t nv, const float* nrm, const float* uv,
                           const uint32_t* idx, uint32_t ntri, int32_t material) {
    auto* rs = static_cast<RefScene*>(s);
    if (material < 0 || material >= static_cast<int32_t>(rs->materials.size())) return -1;
    std::vector<Vec3f> p(nv), n;
    std::vector<Vec2f> t;
    for (uint32_t i = 0; i < nv; ++i) p[i] = v3(pos + 3 * i);
    if (nrm) {
        n.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) n[i] = v3(nrm + 3 * i);
    }
    if (uv) {
        t.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) t[i] = Vec2f(uv[2 * i], uv[2 * i + 1]);
    }
    std::vector<uint32_t> ind(idx, idx + 3 * static_cast<size_t>(ntri));
    auto mesh = std::make_shared<TriangleMesh>(p, n, t, ind, rs->materials[static_cast<size_t>(material)].get());
    rs->scene.addShape(mesh);
    rs->indexNewShapes();
    return 0;
}

// Scene::tagShape of the shape added `shape`-th.
// loadProject + buildRenderScene, the CLI's path for a .photon file (main.cpp:197-206, 214-260):
// the project's render scene; its orbit camera (cameraFromJson, main.cpp:88-110) as
// ref_camera_create parameters; the render block's max bounces and pixel filter.
void* ref_load_project(const char* path, float aspect, int32_t* camKind, float* cam, int32_t* maxBounces,
                       int32_t* filterType, float* filterWidth, char* err, size_t errLen) {
    SceneGraph graph;
    ProjectData data;
    std::string e;
    if (!loadProject(path, graph, data, &e)) {
        std::snprintf(err, errLen, "%s", e.c_str());
        return nullptr;
    }
    EnvironmentCache cache;
    auto scene = buildRenderScene(graph, data.lights, data.environment, cache, false);
    auto* rs = new RefScene(scene);
    rs->indexNewShapes();
    const nlohmann::json& c = data.camera;
    Vec3f target(0, 0.5f, 0);
    if (auto t = c.find("target"); t != c.end() && t->is_array() && t->size() == 3)
        target = Vec3f((*t)[0].get<float>(), (*t)[1].get<float>(), (*t)[2].get<float>());
    const float r = c.value("radius", 5.0f), th = c.value("theta", 1.15f), ph = c.value("phi", 0.45f);
    const float fov = c.value("fov", 35.0f);
    const Vec3f eye = target + Vec3f(std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph)) * r;
    const float head[9] = {eye.x, eye.y, eye.z, target.x, target.y, target.z, 0.0f, 1.0f, 0.0f};
    for (int i = 0; i < 9; ++i) cam[i] = head[i];
    cam[10] = aspect;
    if (c.value("orthographic", false)) {
        *camKind = 2;
        cam[9] = 2.0f * std::tan(fov * DEG_TO_RAD * 0.5f) * r;
    } else if (c.value("aperture", 0.0f) > 0.0f) {
        *camKind = 1;
        cam[9] = fov;
        cam[11] = c.value("aperture", 0.0f);
        cam[12] = c.value("focusExplicit", false) ? c.value("focusDistance", r) : r;
        cam[13] = static_cast<float>(c.value("apertureBlades", 0));
        cam[14] = c.value("bladeRotation", 0.0f);
    } else {
        *camKind = 0;
        cam[9] = fov;
    }
    *maxBounces = data.render.value("maxBounces", 8);
    PixelFilterType ft = PixelFilterType::Box;
    parsePixelFilter(data.render.value("pixelFilter", std::string("box")).c_str(), ft);
    *filterType = static_cast<int32_t>(ft);
    *filterWidth = data.render.value("filterWidth", ft == PixelFilterType::Box ? 1.0f : 1.5f);
    return rs;
}

// The shapes of a scene in order: kind (0 mesh instance or mesh, 1 sphere, 2 area-light triangle,
// 3 other) and, per shape, its triangle count, world bounds (6 floats) and sphere radius.
int32_t ref_scene_shapes(void* s, int32_t* kind, int32_t* tris, float* bounds, int32_t cap) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& shapes = rs->scene.shapes();
    const int32_t n = static_cast<int32_t>(shapes.size());
    for (int32_t i = 0; i < n && i < cap; ++i) {
        const Shape* sh = shapes[static_cast<size_t>(i)].get();
        int32_t k = 3, t = 0;
        if (auto* mi = dynamic_cast<const MeshInstance*>(sh)) {
            k = 0;
            t = mi->mesh() ? static_cast<int32_t>(mi->mesh()->numTriangles()) : 0;
        } else if (auto* m = dynamic_cast<const TriangleMesh*>(sh)) {
            k = 0;
            t = static_cast<int32_t>(m->numTriangles());
        } else if (dynamic_cast<const Sphere*>(sh)) {
            k = 1;
        } else if (dynamic_cast<const Triangle*>(sh)) {
            k = 2;
            t = 1;
        }
        kind[i] = k;
        tris[i] = t;
        const AABB b = sh->bounds();
        const float v[6] = {b.pMin.x, b.pMin.y, b.pMin.z, b.pMax.x, b.pMax.y, b.pMax.z};
        for (int j = 0; j < 6; ++j) bounds[6 * i + j] = v[j];
    }
    return n;
}

// A TriangleMesh kept for instancing (its material is the instance's).
int32_t ref_scene_add_blas(void* s, const float* pos, uint32_t nv, const float* nrm, const float* uv, const uint32_t* idx,
                           uint32_t ntri) {
    auto* rs = static_cast<RefScene*>(s);
    std::vector<Vec3f> p(nv), n;
    std::vector<Vec2f> t;
    for (uint32_t i = 0; i < nv; ++i) p[i] = v3(pos + 3 * i);
    if (nrm) {
        n.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) n[i] = v3(nrm + 3 * i);
    }
    if (uv) {
        t.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) t[i] = Vec2f(uv[2 * i], uv[2 * i + 1]);
    }
    std::vector<uint32_t> ix(idx, idx + 3ull * ntri);
    rs->blases.push_back(std::make_shared<TriangleMesh>(p, n, t, ix, nullptr));
    return static_cast<int32_t>(rs->blases.size() - 1);
}

// Scene::addShape of a MeshInstance of BLAS `blas` with Transform(l2w, w2l) and a material.
int32_t ref_scene_add_instance(void* s, int32_t blas, const float* l2w, const float* w2l, int32_t material) {
    auto* rs = static_cast<RefScene*>(s);
    if (blas < 0 || blas >= static_cast<int32_t>(rs->blases.size()) || material < 0 ||
        material >= static_cast<int32_t>(rs->materials.size()))
        return -1;
    Mat4f m, mi;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            m(r, c) = l2w[4 * r + c];
            if (w2l) mi(r, c) = w2l[4 * r + c];
        }
    const Transform xf = w2l ? Transform(m, mi) : Transform(m);
    rs->scene.addShape(std::make_shared<MeshInstance>(rs->blases[static_cast<size_t>(blas)], xf,
                                                      rs->materials[static_cast<size_t>(material)].get()));
    rs->indexNewShapes();
    return 0;
}

int32_t ref_scene_shape_count(void* s) {
    return static_cast<int32_t>(static_cast<RefScene*>(s)->scene.shapes().size());
}

// MeshInstance::setMotionTransform of instance shape `shape` (before ref_scene_build).
int32_t ref_scene_set_instance_motion(void* s, int32_t shape, const float* l2w, const float* w2l) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& shapes = rs->scene.shapes();
    if (shape < 0 || shape >= static_cast<int32_t>(shapes.size())) return -1;
    auto* mi = dynamic_cast<MeshInstance*>(shapes[static_cast<size_t>(shape)].get());
    if (!mi) return -1;
    Mat4f m, inv;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            m(r, c) = l2w[4 * r + c];
            if (w2l) inv(r, c) = w2l[4 * r + c];
        }
    mi->setMotionTransform(w2l ? Transform(m, inv) : Transform(m));
    return 0;
}

// Camera::setShutterEnd of one of the reference's own cameras (ref_camera_create) to another's pose.
void ref_camera_set_shutter_end(void* cam, void* end) {
    static_cast<Camera*>(cam)->setShutterEnd(*static_cast<const Camera*>(end));
}

// Moves MeshInstance `shape`: a MeshInstance's matrix is fixed at construction, so an application
// that animates one places a new MeshInstance of the same mesh and material in its scene (the
// document rebuild of buildRenderScene).  The shape slot is replaced in place and the scene's
// accelerator rebuilt; 0, or -1 when `shape` is not a MeshInstance.
int32_t ref_scene_move_instance(void* s, int32_t shape, const float* l2w, const float* w2l) {
    auto* rs = static_cast<RefScene*>(s);
    auto& shapes = const_cast<std::vector<std::shared_ptr<Shape>>&>(rs->scene.shapes());
    if (shape < 0 || shape >= static_cast<int32_t>(shapes.size())) return -1;
    auto* old = dynamic_cast<MeshInstance*>(shapes[static_cast<size_t>(shape)].get());
    if (!old) return -1;
    Mat4f m, mi;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            m(r, c) = l2w[4 * r + c];
            if (w2l) mi(r, c) = w2l[4 * r + c];
        }
    const Transform xf = w2l ? Transform(m, mi) : Transform(m);
    auto moved = std::make_shared<MeshInstance>(old->mesh(), xf, old->material());
    rs->shapeIndex.erase(old);
    rs->shapeIndex[moved.get()] = shape;
    shapes[static_cast<size_t>(shape)] = std::move(moved);
    rs->scene.buildAccelerator();
    return 0;
}

// Scene::addShape of a Sphere (src/geometry/sphere.h).
int32_t ref_scene_add_sphere(void* s, const float* center, float radius, int32_t material) {
    auto* rs = static_cast<RefScene*>(s);
    if (material < 0 || material >= static_cast<int32_t>(rs->materials.size())) return -1;
    rs->scene.addShape(std::make_shared<Sphere>(v3(center), radius, rs->materials[static_cast<size_t>(material)].get()));
    rs->indexNewShapes();
    return 0;
}

int32_t ref_scene_tag_shape(void* s, int32_t shape, uint64_t uid) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& shapes = rs->scene.shapes();
    if (shape < 0 || shape >= static_cast<int32_t>(shapes.size())) return -1;
    rs->scene.tagShape(shapes[static_cast<size_t>(shape)].get(), uid);
    return 0;
}

// Light::setLightLink of the scene's `light`-th light.
int32_t ref_scene_set_light_link(void* s, int32_t light, int32_t mode, const uint64_t* uids, int32_t n,
                                 int32_t shadowMode, const uint64_t* shadowUids, int32_t nShadow) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& lights = rs->scene.lights();
    if (light < 0 || light >= static_cast<int32_t>(lights.size())) return -1;
    LightLinkSet l;
    l.mode = static_cast<LightLinkSet::Mode>(mode);
    l.nodeUids.assign(uids, uids + n);
    l.shadowMode = static_cast<LightLinkSet::Mode>(shadowMode);
    l.shadowNodeUids.assign(shadowUids, shadowUids + nShadow);
    // the Scene owns non-const lights; it hands them out as const
    const_cast<Light*>(lights[static_cast<size_t>(light)])->setLightLink(std::move(l));
    return 0;
}

// Light::setLightGroup of light `light` (scene.lights() order), or of the environment (-1; applied
// when the scene is built).
int32_t ref_scene_set_light_group(void* s, int32_t light, const char* name) {
    auto* rs = static_cast<RefScene*>(s);
    if (light < 0) {
        rs->envGroup = name ? name : "";
        return 0;
    }
    const auto& lights = rs->scene.lights();
    if (light >= static_cast<int32_t>(lights.size())) return -1;
    const_cast<Light*>(lights[static_cast<size_t>(light)])->setLightGroup(name ? name : "");
    return 0;
}

// Scene::setShadowCatcher with the shape added `shape`-th (-1: none).
int32_t ref_scene_set_shadow_catcher(void* s, int32_t shape) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& shapes = rs->scene.shapes();
    if (shape < 0 || shape >= static_cast<int32_t>(shapes.size())) {
        rs->scene.setShadowCatcher(nullptr);
        return shape < 0 ? 0 : -1;
    }
    rs->scene.setShadowCatcher(shapes[static_cast<size_t>(shape)].get());
    return 0;
}

int32_t ref_scene_add_area_light(void* s, const float* p, const float* u, const float* v, const float* radiance,
                                 int32_t visible) {
    auto* rs = static_cast<RefScene*>(s);
    auto a = std::make_shared<AreaLight>(v3(p), v3(u), v3(v), c3(radiance));
    a->setVisibleToCamera(visible != 0);
    rs->scene.addLight(a);
    rs->indexNewShapes();
    return 0;
}

int32_t ref_scene_set_environment(void* s, const float* rgb, int32_t w, int32_t h, float rotation, float intensity,
                                  const float* sun_dir, float sun_cos_max, const float* sun_radiance) {
    auto* rs = static_cast<RefScene*>(s);
    std::shared_ptr<Image> img;
    if (rgb && w > 0 && h > 0) {
        img = std::make_shared<Image>(w, h);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const float* px = rgb + 3 * (static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x));
                img->setPixel(x, y, Color3f(px[0], px[1], px[2]));
            }
    }
    auto env = std::make_shared<EnvironmentLight>(img, rotation, intensity);
    if (sun_dir) env->setSun(v3(sun_dir), sun_cos_max, c3(sun_radiance));
    rs->scene.setEnvironment(env);
    return 0;
}

int32_t ref_scene_set_background(void* s, int32_t mode, const float* color) {
    auto* rs = static_cast<RefScene*>(s);
    Background bg;
    bg.mode = static_cast<Background::Mode>(mode);
    bg.color = c3(color);
    rs->scene.setBackground(bg);
    return 0;
}

int32_t ref_scene_build(void* s) {
    auto* rs = static_cast<RefScene*>(s);
    if (!rs->envGroup.empty() && rs->scene.environment())
        const_cast<EnvironmentLight*>(rs->scene.environment())->setLightGroup(rs->envGroup);
    rs->scene.buildAccelerator();
    return 0;
}

int32_t ref_scene_light_count(void* s) {
    return static_cast<int32_t>(static_cast<RefScene*>(s)->scene.lights().size());
}

int32_t ref_scene_light_mode(void* s) {
    const LightSampler& ls = static_cast<RefScene*>(s)->scene.lightSampler();
    return ls.usesBvh() ? 2 : 1;
}

void ref_camera_perspective(const float* pos, const float* target, const float* up, float vfov, float aspect,
                            pe_camera* out) {
    PerspectiveCamera cam(v3(pos), v3(target), v3(up), vfov, aspect);
    const CameraGpuDesc d = cam.describeGpu();
    auto put = [](float* o, const Vec3f& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; };
    put(out->position, d.position);
    put(out->lower_left, d.lowerLeft);
    put(out->horizontal, d.horizontal);
    put(out->vertical, d.vertical);
    put(out->u, d.u);
    put(out->v, d.v);
    put(out->forward, d.forward);
    out->lens_radius = d.lensRadius;
    out->orthographic = d.orthographic ? 1 : 0;
}

// Renderer::renderSamples — the reference's own CPU render path (seed fixed at 12345 there).
// Returns the mean image and counts.
int32_t ref_render(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                   int32_t threads, float* mean_rgb, uint32_t* counts) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    Film film(st->width, st->height);
    Renderer renderer;
    renderer.renderSamples(rs->scene, camera, settings, film, first, count, nullptr);
    exportFilm(film, st->width, st->height, mean_rgb, counts);
    return 0;
}

// Renderer::renderSamples through one of the reference's own camera objects (ref_camera_create):
// the stock CPU path end to end, as CpuDevice::render runs it.
int32_t ref_render_camera(void* s, void* cam, const pe_settings* st, int32_t first, int32_t count, int32_t threads,
                          float* mean_rgb, uint32_t* counts) {
    auto* rs = static_cast<RefScene*>(s);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    Film film(st->width, st->height);
    Renderer renderer;
    renderer.renderSamples(rs->scene, *static_cast<const Camera*>(cam), settings, film, first, count, nullptr);
    exportFilm(film, st->width, st->height, mean_rgb, counts);
    return 0;
}

// The documented starting values of a pe_material description (include/photon_cuda.h), so that a
// description can be filled without the product library: zeros, no image maps, texture scale 1,
// base 0.8 (1 for glass tints), white tints, subsurface radius (1, 0.2, 0.1), roughness and
// specular 0.5, coat roughness 0.03, IORs 1.5, sheen roughness 0.3, subsurface scale 0.05,
// thin-film IOR 1.4, flakes 0.004 / 0.3 / 0.9, opacity 1, absorption distance 1.
void ref_material_defaults(int32_t type, pe_material* m) {
    std::memset(m, 0, sizeof(pe_material));
    m->type = type;
    m->albedo_texture = m->roughness_texture = m->metalness_texture = m->normal_texture = m->opacity_texture = -1;
    m->texture_scale = 1.0f;
    const float sr[3] = {1.0f, 0.2f, 0.1f};
    for (int i = 0; i < 3; ++i) {
        m->base_color[i] = type == PE_MAT_DIELECTRIC ? 1.0f : 0.8f;
        m->coat_tint[i] = m->sheen_color[i] = m->edge_tint[i] = 1.0f;
        m->absorb_color[i] = m->scatter_color[i] = 1.0f;
        m->flake_color[i] = 0.9f;
        m->subsurface_radius[i] = sr[i];
    }
    m->roughness = m->specular = 0.5f;
    m->clearcoat_roughness = 0.03f;
    m->ior = m->coat_ior = 1.5f;
    m->sheen_roughness = 0.3f;
    m->subsurface_scale = 0.05f;
    m->thin_film_ior = 1.4f;
    m->flake_size = 0.004f;
    m->flake_roughness = 0.3f;
    m->opacity = 1.0f;
    m->absorb_distance = 1.0f;
}

// A Film kept across calls (adaptive sampling reads the accumulated film).
void* ref_film_create(int32_t w, int32_t h) { return new Film(w, h); }
void ref_film_destroy(void* f) { delete static_cast<Film*>(f); }
int32_t ref_film_export(void* f, int32_t w, int32_t h, float* mean_rgb, uint32_t* counts) {
    exportFilm(*static_cast<Film*>(f), w, h, mean_rgb, counts);
    return 0;
}

// Renderer::renderSamples (seed 12345) adding samples [first, first+count) to a kept film;
// returns SampleBatchResult::samplesTraced.
int64_t ref_render_film(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                        int32_t threads, void* film) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    Renderer renderer;
    const SampleBatchResult r =
        renderer.renderSamples(rs->scene, camera, settings, *static_cast<Film*>(film), first, count, nullptr);
    return static_cast<int64_t>(r.samplesTraced);
}

// Renderer::renderSamples with AovFilms (seed 12345): the mean beauty, albedo, normal and alpha
// images and their counts.
int32_t ref_render_aovs(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                        int32_t threads, float* mean_rgb, uint32_t* counts, float* albedo, float* normal, float* alpha,
                        uint32_t* aov_counts) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    Film film(st->width, st->height);
    AovFilms aovs;
    aovs.resize(st->width, st->height);
    Renderer renderer;
    renderer.renderSamples(rs->scene, camera, settings, film, first, count, nullptr, &aovs);
    exportFilm(film, st->width, st->height, mean_rgb, counts);
    exportFilm(aovs.albedo, st->width, st->height, albedo, aov_counts);
    exportFilm(aovs.normal, st->width, st->height, normal, nullptr);
    exportFilm(aovs.alpha, st->width, st->height, alpha, nullptr);
    return 0;
}

// Renderer::renderSamples with RenderPassFilms (seed 12345): the mean beauty and counts, the
// eight light passes (light: 8 images), the data passes (data: depth, position, object id,
// material id) and the light groups (groups: up to max_groups images).  Returns the number of
// light groups.
int32_t ref_render_passes(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                          int32_t threads, float* mean_rgb, uint32_t* counts, float* light, float* data, float* groups,
                          int32_t max_groups) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    Film film(st->width, st->height);
    RenderPassFilms passes;
    passes.resize(st->width, st->height);
    Renderer renderer;
    renderer.renderSamples(rs->scene, camera, settings, film, first, count, nullptr, nullptr, &passes);
    const size_t img = static_cast<size_t>(st->width) * static_cast<size_t>(st->height) * 3;
    exportFilm(film, st->width, st->height, mean_rgb, counts);
    for (int k = 0; k < static_cast<int>(LightPass::Count); ++k)
        exportFilm(passes.light[k], st->width, st->height, light + static_cast<size_t>(k) * img, nullptr);
    const Film* d[4] = {&passes.depth, &passes.position, &passes.objectId, &passes.materialId};
    for (int k = 0; k < 4; ++k) exportFilm(*d[k], st->width, st->height, data + static_cast<size_t>(k) * img, nullptr);
    const int n = static_cast<int>(passes.lightGroups.size());
    for (int g = 0; g < n && g < max_groups; ++g)
        exportFilm(passes.lightGroups[static_cast<size_t>(g)].second, st->width, st->height,
                   groups + static_cast<size_t>(g) * img, nullptr);
    return n;
}

// Renderer::renderSamples with RenderPassFilms and both CryptoFilms on (seed 12345): per pixel
// the first `k` entries of CryptoFilm::pixelRanks (id, coverage) of the object film, then of the
// material film, into out[2][h][w][k][2] (unused entries 0).
int32_t ref_render_crypto(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                          int32_t threads, float* out, int32_t k) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    Film film(st->width, st->height);
    RenderPassFilms passes;
    passes.resize(st->width, st->height);
    Renderer renderer;
    renderer.renderSamples(rs->scene, camera, settings, film, first, count, nullptr, nullptr, &passes);
    const CryptoFilm* films[2] = {&passes.cryptoObject, &passes.cryptoMaterial};
    for (int f = 0; f < 2; ++f)
        for (int y = 0; y < st->height; ++y)
            for (int x = 0; x < st->width; ++x) {
                const auto ranks = films[f]->pixelRanks(x, y);
                float* o = out + ((static_cast<size_t>(f) * st->height + y) * st->width + x) * static_cast<size_t>(k) * 2;
                for (int j = 0; j < k && j < static_cast<int>(ranks.size()); ++j) {
                    o[2 * j] = ranks[static_cast<size_t>(j)].first;
                    o[2 * j + 1] = ranks[static_cast<size_t>(j)].second;
                }
            }
    return 0;
}

// Scene::setShapeName / setMaterialName of the `i`-th shape / material added.
int32_t ref_scene_set_shape_name(void* s, int32_t shape, const char* name) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& shapes = rs->scene.shapes();
    if (shape < 0 || shape >= static_cast<int32_t>(shapes.size())) return -1;
    rs->scene.setShapeName(shapes[static_cast<size_t>(shape)].get(), name ? name : "");
    return 0;
}
// Shape::setVisibilityMask (shape.h:27-29) of shape `shape`.
int32_t ref_scene_set_shape_visibility(void* s, int32_t shape, uint32_t mask) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& shapes = rs->scene.shapes();
    if (shape < 0 || shape >= static_cast<int32_t>(shapes.size())) return -1;
    shapes[static_cast<size_t>(shape)]->setVisibilityMask(static_cast<uint8_t>(mask & VisAll));
    return 0;
}
int32_t ref_scene_set_material_name(void* s, int32_t material, const char* name) {
    auto* rs = static_cast<RefScene*>(s);
    if (material < 0 || material >= static_cast<int32_t>(rs->materials.size())) return -1;
    rs->scene.setMaterialName(rs->materials[static_cast<size_t>(material)].get(), name ? name : "");
    return 0;
}

int32_t ref_render_guided(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                          int32_t threads, float* mean_rgb, uint32_t* counts) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    RenderSettings settings = toSettings(*st, threads > 0 ? threads : hardwareThreads());
    settings.pathGuiding = true;
    Film film(st->width, st->height);
    Renderer renderer;
    renderer.renderSamples(rs->scene, camera, settings, film, first, count, nullptr);
    exportFilm(film, st->width, st->height, mean_rgb, counts);
    return 0;
}

// Two training passes of one directional tree as a field leaf sees them (splats, buildFrom,
// building = sampling, splats, buildFrom), then pdf and sample queries on the sampling tree.
int32_t ref_dtree_probe(const float* dirs1, const float* rad1, int32_t n1, const float* dirs2, const float* rad2,
                        int32_t n2, const float* qdirs, const float* qu, int32_t nq, float* pdf_out, float* sample_out) {
    DirectionalTree building, sampling;
    for (int32_t i = 0; i < n1; ++i) building.addSplat(guidingDirToCanonical(v3(dirs1 + 3 * i)), rad1[i]);
    sampling.buildFrom(building, 0.01f, 10);
    building = sampling;
    for (int32_t i = 0; i < n2; ++i) building.addSplat(guidingDirToCanonical(v3(dirs2 + 3 * i)), rad2[i]);
    sampling.buildFrom(building, 0.01f, 10);
    for (int32_t i = 0; i < nq; ++i) {
        pdf_out[i] = sampling.pdf(v3(qdirs + 3 * i));
        float pdf = 0.0f;
        const Vec3f w = sampling.sample(Vec2f(qu[2 * i], qu[2 * i + 1]), pdf);
        sample_out[4 * i + 0] = w.x;
        sample_out[4 * i + 1] = w.y;
        sample_out[4 * i + 2] = w.z;
        sample_out[4 * i + 3] = pdf;
    }
    return 0;
}

// tracePixel (renderer.cpp:139-160) with a caller-chosen Sobol seed over rows [y0, y1); rows
// are split over `threads` workers, each pixel accumulating its samples in index order (so the
// result equals renderSamples' when seed == 12345 and the background mode is Environment).
int32_t ref_render_rows(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                        int32_t threads, int32_t y0, int32_t y1, float* mean_rgb, uint32_t* counts);

int32_t ref_render_seeded(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                          int32_t threads, float* mean_rgb, uint32_t* counts) {
    return ref_render_rows(s, cam, st, first, count, threads, 0, st->height, mean_rgb, counts);
}

static int32_t renderRowsWith(RefScene* rs, const Camera& camera, const pe_settings* st, int32_t first, int32_t count,
                              int32_t threads, int32_t y0, int32_t y1, float* mean_rgb, uint32_t* counts);

int32_t ref_render_rows(void* s, const pe_camera* cam, const pe_settings* st, int32_t first, int32_t count,
                        int32_t threads, int32_t y0, int32_t y1, float* mean_rgb, uint32_t* counts) {
    DescCamera camera(*cam);
    return renderRowsWith(static_cast<RefScene*>(s), camera, st, first, count, threads, y0, y1, mean_rgb, counts);
}

// The reference's own cameras: kind 0 PerspectiveCamera(position, target, up, vfov, aspect),
// 1 ThinLensCamera(..., aperture, focus) + setApertureShape(blades, rotation degrees),
// 2 OrthographicCamera(position, target, up, vertical extent, aspect).
void* ref_camera_create(int32_t kind, const float* p) {
    const Vec3f pos = v3(p), tgt = v3(p + 3), up = v3(p + 6);
    if (kind == 0) return new PerspectiveCamera(pos, tgt, up, p[9], p[10]);
    if (kind == 1) {
        auto* c = new ThinLensCamera(pos, tgt, up, p[9], p[10], p[11], p[12]);
        c->setApertureShape(static_cast<int>(p[13]), p[14]);
        return c;
    }
    if (kind == 2) return new OrthographicCamera(pos, tgt, up, p[9], p[10]);
    return nullptr;
}

void ref_camera_destroy(void* c) { delete static_cast<Camera*>(c); }

void ref_camera_describe(void* c, pe_camera* out) {
    const CameraGpuDesc d = static_cast<Camera*>(c)->describeGpu();
    auto put = [](float* o, const Vec3f& a) { o[0] = a.x; o[1] = a.y; o[2] = a.z; };
    put(out->position, d.position);
    put(out->lower_left, d.lowerLeft);
    put(out->horizontal, d.horizontal);
    put(out->vertical, d.vertical);
    put(out->u, d.u);
    put(out->v, d.v);
    put(out->forward, d.forward);
    out->lens_radius = d.lensRadius;
    out->orthographic = d.orthographic ? 1 : 0;
    out->blades = d.blades;
    out->blade_rotation = d.bladeRotation;
}

// ref_render_rows with one of the reference's own camera objects.
int32_t ref_render_rows_camera(void* s, void* cam, const pe_settings* st, int32_t first, int32_t count, int32_t threads,
                               int32_t y0, int32_t y1, float* mean_rgb, uint32_t* counts) {
    return renderRowsWith(static_cast<RefScene*>(s), *static_cast<Camera*>(cam), st, first, count, threads, y0, y1,
                          mean_rgb, counts);
}

static int32_t renderRowsWith(RefScene* rs, const Camera& camera, const pe_settings* st, int32_t first, int32_t count,
                              int32_t threads, int32_t y0, int32_t y1, float* mean_rgb, uint32_t* counts) {
    const int w = st->width, h = st->height;
    Film film(w, h);
    PathTracer integrator(st->max_bounces, st->rr_depth, st->ao_strength, st->shadow_quality);
    integrator.setClampIndirect(st->clamp_indirect);
    PixelFilter pf;
    pf.type = static_cast<PixelFilterType>(st->filter_type);
    pf.width = st->filter_width;
    const PixelFilterSampler filter(pf);
    const int nt = threads > 0 ? threads : hardwareThreads();
    std::atomic<int> nextRow{y0 < 0 ? 0 : y0};
    const int yEnd = y1 > h ? h : y1;
    auto work = [&]() {
        SobolSampler sampler(st->seed);
        for (;;) {
            const int y = nextRow.fetch_add(1);
            if (y >= yEnd) break;
            for (int x = 0; x < w; ++x)
                for (int si = first; si < first + count; ++si) {
                    sampler.startPixel(x, y);
                    sampler.startSample(si);
                    const Vec2f offset = filter.sample(sampler.get2D());
                    const float sx = (static_cast<float>(x) + 0.5f + offset.x) / static_cast<float>(w);
                    const float sy = 1.0f - (static_cast<float>(y) + 0.5f + offset.y) / static_cast<float>(h);
                    const Vec2f lens = sampler.get2D();
                    Ray ray = st->motion_blur ? camera.generateRay(sx, sy, lens, sampler.get1D())
                                              : camera.generateRay(sx, sy, lens);
                    ray.coneWidth = camera.pixelConeWidth(h);
                    ray.coneSpread = camera.pixelConeSpread(h);
                    // as tracePixel: with a colour or transparent background the integrator gets
                    // the primary-hit record, through which camera misses see that background
                    if (rs->scene.background().mode == Background::Mode::Environment) {
                        film.addSample(x, y, integrator.Li(ray, rs->scene, sampler));
                    } else {
                        PathTracer::PrimaryHit primary;
                        film.addSample(x, y, integrator.Li(ray, rs->scene, sampler, &primary, nullptr));
                    }
                }
        }
    };
    std::vector<std::thread> pool;
    for (int i = 0; i < nt; ++i) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    exportFilm(film, w, h, mean_rgb, counts);
    return 0;
}

// The seeded tracePixel loop of ref_render_rows over one rectangle of the frame (x0, y0, cw, ch),
// through the reference's own camera object: mean (ch, cw, 3) and counts (ch, cw) of the crop.
int32_t ref_render_rect(void* s, void* cam, const pe_settings* st, int32_t first, int32_t count, int32_t threads,
                        int32_t x0, int32_t y0, int32_t cw, int32_t ch, float* mean_rgb, uint32_t* counts) {
    auto* rs = static_cast<RefScene*>(s);
    const Camera& camera = *static_cast<const Camera*>(cam);
    const int w = st->width, h = st->height;
    if (x0 < 0 || y0 < 0 || cw <= 0 || ch <= 0 || x0 + cw > w || y0 + ch > h) return -1;
    Film film(w, h);
    PathTracer integrator(st->max_bounces, st->rr_depth, st->ao_strength, st->shadow_quality);
    integrator.setClampIndirect(st->clamp_indirect);
    PixelFilter pf;
    pf.type = static_cast<PixelFilterType>(st->filter_type);
    pf.width = st->filter_width;
    const PixelFilterSampler filter(pf);
    const int nt = threads > 0 ? threads : hardwareThreads();
    std::atomic<int> next{0};
    auto work = [&]() {
        SobolSampler sampler(st->seed);
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= cw * ch) break;
            const int x = x0 + k % cw, y = y0 + k / cw;
            for (int si = first; si < first + count; ++si) {
                sampler.startPixel(x, y);
                sampler.startSample(si);
                const Vec2f offset = filter.sample(sampler.get2D());
                const float sx = (static_cast<float>(x) + 0.5f + offset.x) / static_cast<float>(w);
                const float sy = 1.0f - (static_cast<float>(y) + 0.5f + offset.y) / static_cast<float>(h);
                const Vec2f lens = sampler.get2D();
                Ray ray = st->motion_blur ? camera.generateRay(sx, sy, lens, sampler.get1D())
                                          : camera.generateRay(sx, sy, lens);
                ray.coneWidth = camera.pixelConeWidth(h);
                ray.coneSpread = camera.pixelConeSpread(h);
                if (rs->scene.background().mode == Background::Mode::Environment) {
                    film.addSample(x, y, integrator.Li(ray, rs->scene, sampler));
                } else {
                    PathTracer::PrimaryHit primary;
                    film.addSample(x, y, integrator.Li(ray, rs->scene, sampler, &primary, nullptr));
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int i = 0; i < nt; ++i) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    std::vector<float> mean(static_cast<size_t>(w) * h * 3);
    std::vector<uint32_t> cnt(static_cast<size_t>(w) * h);
    exportFilm(film, w, h, mean.data(), cnt.data());
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) {
            const size_t src = static_cast<size_t>(y0 + y) * w + x0 + x, dst = static_cast<size_t>(y) * cw + x;
            for (int c = 0; c < 3; ++c) mean_rgb[3 * dst + c] = mean[3 * src + c];
            counts[dst] = cnt[src];
        }
    return 0;
}

// Primary hit per pixel for one sample index: tracePixel's camera ray, then the first
// Scene::intersect of PathTracer::Li with the camera visibility mask (path_tracer.cpp:326,420).
int32_t ref_trace_primary(void* s, const pe_camera* cam, const pe_settings* st, int32_t sample_index,
                          int32_t* out_shape, int32_t* out_prim, float* out_t) {
    auto* rs = static_cast<RefScene*>(s);
    DescCamera camera(*cam);
    const int w = st->width, h = st->height;
    PixelFilter pf;
    pf.type = static_cast<PixelFilterType>(st->filter_type);
    pf.width = st->filter_width;
    const PixelFilterSampler filter(pf);
    const int nt = hardwareThreads();
    std::atomic<int> nextRow{0};
    auto work = [&]() {
        SobolSampler sampler(st->seed);
        for (;;) {
            const int y = nextRow.fetch_add(1);
            if (y >= h) break;
            for (int x = 0; x < w; ++x) {
                sampler.startPixel(x, y);
                sampler.startSample(sample_index);
                const Vec2f offset = filter.sample(sampler.get2D());
                const float sx = (static_cast<float>(x) + 0.5f + offset.x) / static_cast<float>(w);
                const float sy = 1.0f - (static_cast<float>(y) + 0.5f + offset.y) / static_cast<float>(h);
                const Vec2f lens = sampler.get2D();
                Ray ray = camera.generateRay(sx, sy, lens);
                ray.visibilityMask = VisCamera;
                SurfaceInteraction isect;
                const size_t i = static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x);
                if (rs->scene.intersect(ray, isect)) {
                    auto it = rs->shapeIndex.find(isect.hitObject);
                    out_shape[i] = it == rs->shapeIndex.end() ? -2 : it->second;
                    out_prim[i] = isect.primIndex < 0 ? 0 : isect.primIndex;
                    out_t[i] = isect.t;
                } else {
                    out_shape[i] = -1;
                    out_prim[i] = -1;
                    out_t[i] = 0.0f;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int i = 0; i < nt; ++i) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    return 0;
}

// Scene::intersect / intersectAny of n rays (t in [0, t_max[i]], the visibility mask, the shutter
// time): mode 0 closest hit (shape, triangle within it, t; shape -1 on a miss), 2 any hit
// (out_shape 1 when occluded).
int32_t ref_trace_rays(void* s, const float* o, const float* d, const float* tmax, int32_t n, int32_t mode,
                       uint32_t mask, float time, int32_t* out_shape, int32_t* out_prim, float* out_t) {
    auto* rs = static_cast<RefScene*>(s);
    for (int32_t i = 0; i < n; ++i) {
        Ray ray(v3(o + 3 * i), v3(d + 3 * i));
        ray.tMin = 0.0f;
        ray.tMax = tmax[i];
        ray.visibilityMask = static_cast<uint8_t>(mask);
        ray.time = time;
        if (mode == 2) {
            out_shape[i] = rs->scene.intersectAny(ray) ? 1 : 0;
            out_prim[i] = -1;
            out_t[i] = 0.0f;
            continue;
        }
        SurfaceInteraction isect;
        if (rs->scene.intersect(ray, isect)) {
            auto it = rs->shapeIndex.find(isect.hitObject);
            out_shape[i] = it == rs->shapeIndex.end() ? -2 : it->second;
            out_prim[i] = isect.primIndex < 0 ? 0 : isect.primIndex;
            out_t[i] = isect.t;
        } else {
            out_shape[i] = -1;
            out_prim[i] = -1;
            out_t[i] = 0.0f;
        }
    }
    return 0;
}

int32_t ref_sobol(uint64_t seed, const int32_t* px, const int32_t* py, const int32_t* index, size_t n, int32_t ndims,
                  float* out) {
    SobolSampler s(seed);
    for (size_t i = 0; i < n; ++i) {
        s.startPixel(px[i], py[i]);
        s.startSample(index[i]);
        for (int k = 0; k < ndims; ++k) {
            const Vec2f v = s.get2D();
            out[(i * static_cast<size_t>(ndims) + static_cast<size_t>(k)) * 2 + 0] = v.x;
            out[(i * static_cast<size_t>(ndims) + static_cast<size_t>(k)) * 2 + 1] = v.y;
        }
    }
    return 0;
}

int32_t ref_sobol_1d(uint64_t seed, int32_t px, int32_t py, int32_t index, int32_t ndims, float* out) {
    SobolSampler s(seed);
    s.startPixel(px, py);
    s.startSample(index);
    for (int k = 0; k < ndims; ++k) out[k] = s.get1D();
    return 0;
}

int32_t ref_bsdf_probe(void* s, int32_t material, const pe_bsdf_query* q, size_t n, pe_bsdf_result* out) {
    auto* rs = static_cast<RefScene*>(s);
    if (material < 0 || material >= static_cast<int32_t>(rs->materials.size())) return -1;
    const Material* m = rs->materials[static_cast<size_t>(material)].get();
    for (size_t i = 0; i < n; ++i) {
        SurfaceInteraction si;
        si.normal = v3(q[i].normal);
        si.ng = v3(q[i].ng);
        si.tangent = v3(q[i].tangent);
        si.point = v3(q[i].point);
        si.frontFace = q[i].front_face != 0;
        si.wavelength = q[i].wavelength;
        si.material = m;
        pe_bsdf_result r{};
        float pdf = 0.0f;
        const Color3f f = m->evalPdf(v3(q[i].wo), v3(q[i].wi), si, pdf);
        r.f[0] = f.r;
        r.f[1] = f.g;
        r.f[2] = f.b;
        r.pdf = pdf;
        BSDFSample bs;
        r.sampled = m->sampleFull(v3(q[i].wo), si, q[i].uc, Vec2f(q[i].u[0], q[i].u[1]), bs) ? 1 : 0;
        r.wi[0] = bs.wi.x;
        r.wi[1] = bs.wi.y;
        r.wi[2] = bs.wi.z;
        r.sf[0] = bs.f.r;
        r.sf[1] = bs.f.g;
        r.sf[2] = bs.f.b;
        r.spdf = bs.pdf;
        r.delta = bs.delta;
        r.pass_through = bs.passThrough;
        r.subsurface = bs.subsurface;
        r.weight[0] = bs.weight.r;
        r.weight[1] = bs.weight.g;
        r.weight[2] = bs.weight.b;
        out[i] = r;
    }
    return 0;
}

// LightSampler: for each shading point, prepare() then sample(u) and pmf(index).
int32_t ref_light_pick(void* s, const float* p, const float* nrm, const float* u, size_t n, int32_t* out_index,
                       float* out_pmf, float* out_pmf_check) {
    auto* rs = static_cast<RefScene*>(s);
    const LightSampler& ls = rs->scene.lightSampler();
    for (size_t i = 0; i < n; ++i) {
        const LightSampler::Context c = ls.prepare(v3(p + 3 * i), v3(nrm + 3 * i));
        float pmf = 0.0f;
        const int idx = c.sample(u[i], pmf);
        out_index[i] = idx;
        out_pmf[i] = pmf;
        out_pmf_check[i] = idx >= 0 ? c.pmf(idx) : 0.0f;
    }
    return 0;
}

// Light::sampleLi for light `light` (or the environment when light == count) at point p with
// shading normal n: direction, Li, pdf, distance.
int32_t ref_light_sample(void* s, int32_t light, const float* p, const float* nrm, const float* u, size_t n,
                         float* out_wi, float* out_li, float* out_pdf, float* out_dist) {
    auto* rs = static_cast<RefScene*>(s);
    const auto& lights = rs->scene.lights();
    const EnvironmentLight* env = rs->scene.environment();
    for (size_t i = 0; i < n; ++i) {
        SurfaceInteraction si;
        si.point = v3(p + 3 * i);
        si.normal = v3(nrm + 3 * i);
        LightSample lsmp;
        const Vec2f uu(u[2 * i], u[2 * i + 1]);
        if (light >= 0 && light < static_cast<int32_t>(lights.size())) lsmp = lights[static_cast<size_t>(light)]->sampleLi(si, uu);
        else if (env) lsmp = env->sampleLi(si, uu);
        out_wi[3 * i + 0] = lsmp.wi.x;
        out_wi[3 * i + 1] = lsmp.wi.y;
        out_wi[3 * i + 2] = lsmp.wi.z;
        out_li[3 * i + 0] = lsmp.Li.r;
        out_li[3 * i + 1] = lsmp.Li.g;
        out_li[3 * i + 2] = lsmp.Li.b;
        out_pdf[i] = lsmp.pdf;
        out_dist[i] = lsmp.distance;
    }
    return 0;
}

// EnvironmentLight::eval and pdfLi for directions.
int32_t ref_env_eval(void* s, const float* dirs, size_t n, float* out_rgb, float* out_pdf) {
    auto* rs = static_cast<RefScene*>(s);
    const EnvironmentLight* env = rs->scene.environment();
    if (!env) return -1;
    for (size_t i = 0; i < n; ++i) {
        const Vec3f d = v3(dirs + 3 * i);
        const Color3f c = env->eval(d);
        out_rgb[3 * i + 0] = c.r;
        out_rgb[3 * i + 1] = c.g;
        out_rgb[3 * i + 2] = c.b;
        out_pdf[i] = env->pdfLi(d);
    }
    return 0;
}

#ifdef PE_WITH_ADAPTER
// The B200 device through the drop-in adapter (photon-engine_b200/adapter), driven by the
// reference's own RenderSession (src/engine/render_session.cpp:17-101) on a reference Scene: the
// parity check of the adapter itself.  One device per process, created on first use.
static uint64_t g_adapterScene = 0; // RefScene::id of the scene the adapter device holds

static std::unique_ptr<RenderDevice>& cudaAdapterDevice(std::string* err) {
    static std::unique_ptr<RenderDevice> dev;
    if (!dev) dev = createCudaRenderDevice(0, err);
    return dev;
}

// Full RenderSession on the adapter: begin(camera, settings with `spp` samples, Final mode, maxBatch
// `batch`), advance() until finished.  Beauty mean and counts (h, w) come back; with aovs, the
// albedo film's mean too.  features = the device's (aovs, lightPasses, adaptive) as bits 0-2.
int32_t ref_session_cuda(void* s, void* cam, const pe_settings* st, int32_t spp, int32_t batch, int32_t aovs,
                         int32_t adaptive, float* mean_rgb, uint32_t* counts, float* albedo_mean, int32_t* features,
                         char* err, size_t errLen) {
    auto* rs = static_cast<RefScene*>(s);
    std::string e;
    auto& dev = cudaAdapterDevice(&e);
    if (!dev) {
        std::snprintf(err, errLen, "%s", e.c_str());
        return -1;
    }
    const DeviceFeatures f = dev->features();
    *features = (f.aovs ? 1 : 0) | (f.lightPasses ? 2 : 0) | (f.adaptiveSampling ? 4 : 0);
    // a session on the scene the adapter already holds keeps it (its updateScene edits included)
    if (g_adapterScene != rs->id || !dev->hasScene()) {
        dev->setScene(std::shared_ptr<const Scene>(std::shared_ptr<const Scene>{}, &rs->scene));
        g_adapterScene = rs->id;
    }
    if (!dev->hasScene()) {
        std::snprintf(err, errLen, "the adapter did not take the scene");
        return -2;
    }
    RenderSettings settings = toSettings(*st, hardwareThreads());
    settings.samplesPerPixel = spp;
    settings.adaptiveSampling = adaptive != 0;
    settings.noiseThreshold = st->noise_threshold;
    settings.minAdaptiveSamples = st->min_adaptive_samples;
    SessionConfig config;
    config.mode = RenderMode::Final;
    config.targetSpp = spp;
    config.aovs = aovs != 0;
    config.maxBatch = batch;
    RenderSession session(*dev);
    session.begin(std::shared_ptr<const Camera>(std::shared_ptr<const Camera>{}, static_cast<const Camera*>(cam)),
                  settings, config);
    int guard = 0;
    while (!session.finished() && guard++ < 100000)
        if (!session.advance(nullptr)) break;
    exportFilm(session.film(), st->width, st->height, mean_rgb, counts);
    if (aovs && albedo_mean && session.aovs()) {
        std::vector<uint32_t> c(static_cast<size_t>(st->width) * static_cast<size_t>(st->height));
        exportFilm(session.aovs()->albedo, st->width, st->height, albedo_mean, c.data());
    }
    return session.samples();
}

// SceneUpdateKind edits through the adapter: kind 1 sets material `index`'s base colour (a Disney
// material) or albedo-free Lambert is left alone; kind 2 sets AreaLight `index`'s radiance; then
// RenderDevice::updateScene(scene, kind).
int32_t ref_session_cuda_update(void* s, int32_t kind, int32_t index, const float* rgb) {
    auto* rs = static_cast<RefScene*>(s);
    std::string e;
    auto& dev = cudaAdapterDevice(&e);
    if (!dev) return -1;
    if (kind == 1) {
        if (index < 0 || index >= static_cast<int32_t>(rs->materials.size())) return -2;
        auto* d = dynamic_cast<DisneyMaterial*>(rs->materials[static_cast<size_t>(index)].get());
        if (!d) return -3;
        d->setBaseColor(c3(rgb));
        dev->updateScene(std::shared_ptr<const Scene>(std::shared_ptr<const Scene>{}, &rs->scene),
                         SceneUpdateKind::Materials);
    } else if (kind == 2) {
        int k = 0;
        for (const Light* l : rs->scene.lights())
            if (auto* a = dynamic_cast<const AreaLight*>(l)) {
                if (k++ == index) const_cast<AreaLight*>(a)->setRadiance(c3(rgb));
            }
        dev->updateScene(std::shared_ptr<const Scene>(std::shared_ptr<const Scene>{}, &rs->scene),
                         SceneUpdateKind::Lights);
    } else if (kind == 3) {
        // the scene's MeshInstances were moved (ref_scene_move_instance)
        dev->updateScene(std::shared_ptr<const Scene>(std::shared_ptr<const Scene>{}, &rs->scene),
                         SceneUpdateKind::Transforms);
    } else {
        return -4;
    }
    return dev->hasScene() ? 0 : -5;
}
#endif

} // extern "C"
