// cuda_render_device.cpp — RenderDevice (src/engine/render_device.h:65-86) over photon_cuda.h.
//
// setScene   the reference Scene → one pe_scene in the Scene's own shape and light order (a mesh
//            is one shape, an AreaLight's quad two, as scene.cpp:65-99 adds them), so shape, light
//            and material numbering — and with it tags, names, light groups and links, the shadow
//            catcher — are the reference's; then pe_scene_build and pe_device_set_scene.
// updateScene Materials / Lights / Transforms edit the kept pe_scene and re-send only that
//            (SceneUpdateKind, render_device.h:34; Transforms refits the top-level tree over the
//            instances' BLASes); anything else rebuilds.
// render     [firstSample, firstSample+count) in one device call into fresh batch arrays, added to
//            the caller's films with Film::addBatch (film.cpp:119-137) as a GPU readback is; AOVs
//            and render passes likewise; Cryptomatte ids per sample through CryptoFilm::addSample.
//            Adaptive sampling keeps the session's exact film sums (sum, count, squared luminance)
//            beside the caller's Film, because the device decides from them as Film::relativeError
//            does (film.cpp:100-109) and Film keeps no per-sample squares after addBatch.
//            The cancel flag is polled while the call runs and ends it between waves.
#include "cuda_render_device.h"

#include "camera/camera.h"
#include "core/image/cryptomatte.h"
#include "core/image/film.h"
#include "core/image/image.h"
#include "engine/scene.h"
#include "geometry/mesh.h"
#include "geometry/mesh_instance.h"
#include "geometry/sphere.h"
#include "geometry/surface_interaction.h"
#include "geometry/triangle.h"
#include "lights/area_light.h"
#include "lights/environment_light.h"
#include "materials/dielectric.h"
#include "materials/disney.h"
#include "materials/lambertian.h"
#include "materials/mirror.h"
#include "photon_cuda.h"

#include <atomic>
#include <chrono>
#include <cstring>
#include <iostream>
#include <thread>
#include <unordered_map>
#include <vector>

namespace photon {
namespace {

void put3(float* o, const Color3f& c) {
    o[0] = c.r;
    o[1] = c.g;
    o[2] = c.b;
}
void put3(float* o, const Vec3f& v) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
}

// The scene content as the C ABI's flat description, built once per setScene and kept for
// incremental updates.
// A Transform's matrix and inverse as the row-major arrays of the C ABI.
void putTransform(const Transform& xf, float* m, float* inv) {
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            m[4 * r + c] = xf.matrix()(r, c);
            inv[4 * r + c] = xf.inverseMatrix()(r, c);
        }
}

struct PeScene {
    pe_scene* s = nullptr;
    const Scene* source = nullptr;
    std::unordered_map<const Image*, int32_t> textures;
    std::unordered_map<const Material*, int32_t> materials;
    std::vector<std::pair<int32_t, const AreaLight*>> areaLights; // light index of each AreaLight
    std::unordered_map<const TriangleMesh*, int32_t> blases;      // meshes of MeshInstances
    // every shape as built: its pointer and, for a MeshInstance, its mesh and material (kept by
    // value so a Transforms update can compare a scene whose old shapes are gone)
    struct Placed {
        const Shape* shape;
        const TriangleMesh* mesh;
        const Material* material;
    };
    std::vector<Placed> placed;
    std::string error;

    ~PeScene() { pe_scene_destroy(s); }

    int32_t texture(const std::shared_ptr<const Image>& img) {
        if (!img) return -1;
        auto it = textures.find(img.get());
        if (it != textures.end()) return it->second;
        int32_t t;
        if (img->isCompact8()) {
            t = pe_scene_add_texture_u8(s, img->dataU8(), img->width(), img->height(),
                                        img->storageFormat() == Image::StorageFormat::U8Srgb ? 1 : 0);
        } else {
            t = pe_scene_add_texture(s, img->data(), img->width(), img->height());
        }
        if (t >= 0 && img->hasMipmaps() && pe_scene_build_texture_mipmaps(s, t) != PE_OK) t = -1;
        textures[img.get()] = t;
        return t;
    }

    // SceneUpdateKind::Transforms: `scene` holds the shapes as built except MeshInstances placed
    // anew (same mesh and material, another matrix; a MeshInstance's matrix is fixed at
    // construction, so a moved instance is a new object).  Sends their matrices; false when
    // anything else changed, an instance moves with motion blur or emits light.
    bool moveInstances(const Scene& scene) {
        const auto& shapes = scene.shapes();
        if (shapes.size() != placed.size()) return false;
        for (size_t i = 0; i < shapes.size(); ++i) {
            const Shape* now = shapes[i].get();
            const auto* mi = dynamic_cast<const MeshInstance*>(now);
            if (now == placed[i].shape && !mi) continue;
            if (!mi || !placed[i].mesh || mi->mesh().get() != placed[i].mesh || mi->material() != placed[i].material ||
                mi->hasMotion())
                return false;
            float l2w[16], w2l[16];
            putTransform(mi->transform0(), l2w, w2l);
            if (pe_scene_set_instance_transform(s, static_cast<int32_t>(i), l2w, w2l) != PE_OK) return false;
            placed[i].shape = now;
        }
        source = &scene;
        return true;
    }

    // Material::* parameters as pe_material (the device clamps them as the setters do).
    bool describe(const Material* m, pe_material& p) {
        const SurfaceInteraction none{};
        if (auto* d = dynamic_cast<const DisneyMaterial*>(m)) {
            pe_material_defaults(PE_MAT_DISNEY, &p);
            put3(p.base_color, d->baseColor());
            put3(p.emission, d->emitted(none));
            p.metallic = d->metallic();
            p.roughness = d->roughness();
            p.specular = d->specular();
            p.clearcoat = d->clearCoat();
            p.clearcoat_roughness = d->clearCoatRoughness();
            p.ior = d->ior();
            p.spec_transmission = d->specularTransmission();
            p.coat_ior = d->coatIor();
            put3(p.coat_tint, d->coatTint());
            put3(p.sheen_color, d->sheenColor());
            p.has_sheen_color = d->hasCustomSheenColor() ? 1 : 0;
            p.anisotropy = d->anisotropy();
            p.sheen = d->sheen();
            p.sheen_roughness = d->sheenRoughness();
            p.diffuse_roughness = d->diffuseRoughness();
            p.diffuse_transmission = d->diffuseTransmission();
            p.subsurface = d->subsurface();
            put3(p.subsurface_radius, d->subsurfaceRadius());
            p.subsurface_scale = d->subsurfaceScale();
            p.subsurface_anisotropy = d->subsurfaceAnisotropy();
            put3(p.edge_tint, d->edgeTint());
            p.thin_film_thickness = d->thinFilmThickness();
            p.thin_film_ior = d->thinFilmIor();
            p.flake_density = d->flakeDensity();
            p.flake_size = d->flakeSize();
            p.flake_roughness = d->flakeRoughness();
            put3(p.flake_color, d->flakeColor());
            p.opacity = d->baseOpacity();
            p.albedo_texture = texture(d->albedoImage());
            p.roughness_texture = texture(d->roughnessImage());
            p.metalness_texture = texture(d->metalnessImage());
            p.normal_texture = texture(d->normalImage());
            p.opacity_texture = texture(d->opacityImage());
            p.texture_mapping = d->textureMapping() == DisneyMaterial::TextureMapping::Box ? 1 : 0;
            p.texture_scale = d->textureScale();
        } else if (auto* g = dynamic_cast<const Dielectric*>(m)) {
            pe_material_defaults(PE_MAT_DIELECTRIC, &p);
            p.ior = g->ior();
            put3(p.base_color, g->tint());
            p.glass_roughness = g->roughness();
            p.abbe = g->abbe();
            p.thin_walled = g->thinWalled() ? 1 : 0;
            p.film_thickness = g->thinFilmThickness();
            const Color3f a = g->absorptionColor();
            if (a.r != 1.0f || a.g != 1.0f || a.b != 1.0f) {
                p.has_absorption = 1;
                put3(p.absorb_color, a);
                p.absorb_distance = g->absorptionDistance();
            }
            if (g->scatterDensity() > 0.0f) {
                p.has_scattering = 1;
                p.scatter_density = g->scatterDensity();
                put3(p.scatter_color, g->scatterColor());
                p.scatter_anisotropy = g->scatterAnisotropy();
            }
        } else if (auto* r = dynamic_cast<const Mirror*>(m)) {
            pe_material_defaults(PE_MAT_MIRROR, &p);
            put3(p.base_color, r->reflectance());
        } else if (auto* l = dynamic_cast<const Lambertian*>(m)) {
            pe_material_defaults(PE_MAT_LAMBERT, &p);
            put3(p.base_color, l->albedo());
            put3(p.emission, l->emitted(none));
        } else {
            error = "a material type the CUDA device does not implement";
            return false;
        }
        p.round_edge_radius = m->roundEdgeRadius();
        return true;
    }

    int32_t material(const Material* m) {
        auto it = materials.find(m);
        if (it != materials.end()) return it->second;
        pe_material p;
        if (!describe(m, p)) return -1;
        const int32_t i = pe_scene_add_material(s, &p);
        materials[m] = i;
        return i;
    }

    bool build(const Scene& scene) {
        s = pe_scene_create();
        source = &scene;
        if (!s) {
            error = "pe_scene_create failed";
            return false;
        }
        // AreaLights in light order: each owns the next two Triangle shapes (scene.cpp:65-99)
        std::vector<const AreaLight*> areas;
        const auto& lights = scene.lights();
        for (size_t li = 0; li < lights.size(); ++li)
            if (auto* a = dynamic_cast<const AreaLight*>(lights[li])) {
                areas.push_back(a);
                areaLights.emplace_back(static_cast<int32_t>(li), a);
            }
        size_t nextArea = 0;
        bool secondHalf = false;
        const auto& owners = scene.shapeOwners();
        const auto& names = scene.shapeNames();
        const auto& shapes = scene.shapes();
        for (size_t i = 0; i < shapes.size(); ++i) {
            const Shape* shape = shapes[i].get();
            const int32_t index = static_cast<int32_t>(i);
            const auto* inst = dynamic_cast<const MeshInstance*>(shape);
            placed.push_back({shape, inst ? inst->mesh().get() : nullptr, inst ? inst->material() : nullptr});
            if (auto* m = dynamic_cast<const TriangleMesh*>(shape)) {
                const int32_t mat = material(m->material());
                if (mat < 0) return false;
                const auto& P = m->positions();
                const auto& N = m->normals();
                const auto& UV = m->uvs();
                if (pe_scene_add_mesh(s, P.empty() ? nullptr : &P[0].x, static_cast<uint32_t>(P.size()),
                                      N.empty() ? nullptr : &N[0].x, UV.empty() ? nullptr : &UV[0].x,
                                      m->indices().data(), static_cast<uint32_t>(m->numTriangles()), mat) != PE_OK) {
                    error = pe_last_error();
                    return false;
                }
            } else if (auto* mi = dynamic_cast<const MeshInstance*>(shape)) {
                // a MeshInstance: its mesh once as a BLAS, then the instance with both matrices
                if (!mi->mesh()) {
                    error = "a mesh instance without a mesh";
                    return false;
                }
                const TriangleMesh* m = mi->mesh().get();
                auto it = blases.find(m);
                if (it == blases.end()) {
                    const auto& P = m->positions();
                    const auto& N = m->normals();
                    const auto& UV = m->uvs();
                    const int32_t b = pe_scene_add_blas(s, &P[0].x, static_cast<uint32_t>(P.size()),
                                                        N.empty() ? nullptr : &N[0].x, UV.empty() ? nullptr : &UV[0].x,
                                                        m->indices().data(), static_cast<uint32_t>(m->numTriangles()));
                    if (b < 0) {
                        error = pe_last_error();
                        return false;
                    }
                    it = blases.emplace(m, b).first;
                }
                const int32_t mat = material(mi->material());
                if (mat < 0) return false;
                float l2w[16], w2l[16];
                putTransform(mi->transform0(), l2w, w2l);
                if (pe_scene_add_instance(s, it->second, l2w, w2l, mat) != PE_OK) {
                    error = pe_last_error();
                    return false;
                }
                if (mi->hasMotion()) { // setMotionTransform: the pose at shutter close
                    putTransform(mi->transform1(), l2w, w2l);
                    if (pe_scene_set_instance_motion(s, index, l2w, w2l) != PE_OK) {
                        error = pe_last_error();
                        return false;
                    }
                }
            } else if (auto* sp = dynamic_cast<const Sphere*>(shape)) {
                const int32_t mat = material(sp->material());
                if (mat < 0) return false;
                float c[3];
                put3(c, sp->center());
                if (pe_scene_add_sphere(s, c, sp->radius(), mat) != PE_OK) {
                    error = pe_last_error();
                    return false;
                }
            } else if (dynamic_cast<const Triangle*>(shape) && (secondHalf || nextArea < areas.size())) {
                if (!secondHalf) {
                    const AreaLight* a = areas[nextArea++];
                    float p[3], u[3], v[3], r[3];
                    put3(p, a->position());
                    put3(u, a->u());
                    put3(v, a->v());
                    put3(r, a->radiance());
                    if (pe_scene_add_area_light(s, p, u, v, r, a->visibleToCamera() ? 1 : 0) != PE_OK) {
                        error = pe_last_error();
                        return false;
                    }
                }
                secondHalf = !secondHalf;
            } else {
                error = "shape " + std::to_string(i) + " is of a kind the CUDA device does not trace "
                        "(stand-alone triangles)";
                return false;
            }
            if (shape == scene.shadowCatcherShape()) pe_scene_set_shadow_catcher(s, index);
            if (auto it = owners.find(shape); it != owners.end() && it->second != 0)
                pe_scene_tag_shape(s, index, it->second);
            if (auto it = names.find(shape); it != names.end() && !it->second.empty())
                pe_scene_set_shape_name(s, index, it->second.c_str());
            // an AreaLight's triangles carry their own camera visibility (pe_scene_add_area_light)
            if (!dynamic_cast<const Triangle*>(shape) && shape->visibilityMask() != VisAll)
                pe_scene_set_shape_visibility(s, index, shape->visibilityMask());
        }
        for (const auto& [m, name] : scene.materialNames())
            if (auto it = materials.find(m); it != materials.end() && !name.empty())
                pe_scene_set_material_name(s, it->second, name.c_str());
        for (size_t li = 0; li < lights.size(); ++li) {
            const Light* l = lights[li];
            if (!l->lightGroup().empty()) pe_scene_set_light_group(s, static_cast<int32_t>(li), l->lightGroup().c_str());
            const LightLinkSet& link = l->lightLink();
            if (!link.isDefault())
                pe_scene_set_light_link(s, static_cast<int32_t>(li), static_cast<int32_t>(link.mode),
                                        link.nodeUids.data(), static_cast<int32_t>(link.nodeUids.size()),
                                        static_cast<int32_t>(link.shadowMode), link.shadowNodeUids.data(),
                                        static_cast<int32_t>(link.shadowNodeUids.size()));
        }
        if (const EnvironmentLight* env = scene.environment()) {
            const auto& img = env->image();
            std::vector<float> rgb;
            if (img) {
                rgb.resize(static_cast<size_t>(img->width()) * static_cast<size_t>(img->height()) * 3);
                for (int y = 0; y < img->height(); ++y)
                    for (int x = 0; x < img->width(); ++x)
                        put3(&rgb[3 * (static_cast<size_t>(y) * static_cast<size_t>(img->width()) + static_cast<size_t>(x))],
                             img->getPixel(x, y));
            }
            if (pe_scene_set_environment(s, img ? rgb.data() : nullptr, img ? img->width() : 0, img ? img->height() : 0,
                                         env->rotation(), env->intensity()) != PE_OK) {
                error = pe_last_error();
                return false;
            }
            if (env->hasSun() && env->intensity() > 0.0f) {
                // EnvironmentLight::setSun scales the radiance by the intensity (environment_light.cpp:168-171)
                float dir[3], rad[3];
                put3(dir, env->sunDirection());
                put3(rad, env->sunRadiance() * (1.0f / env->intensity()));
                pe_scene_set_sun(s, dir, env->sunCosMax(), rad);
            }
            if (!env->lightGroup().empty()) pe_scene_set_light_group(s, -1, env->lightGroup().c_str());
        }
        const Background& bg = scene.background();
        float bc[3];
        put3(bc, bg.color);
        pe_scene_set_background(s, static_cast<int32_t>(bg.mode), bc);
        if (pe_scene_build(s) != PE_OK) {
            error = pe_last_error();
            return false;
        }
        return true;
    }
};

// A Film's three arrays for one device call.
struct Arrays {
    std::vector<float> sum, sq;
    std::vector<uint32_t> cnt;
    void reset(size_t n) {
        sum.assign(3 * n, 0.0f);
        sq.assign(n, 0.0f);
        cnt.assign(n, 0u);
    }
    pe_film_arrays view() { return pe_film_arrays{sum.data(), cnt.data(), sq.data()}; }
    void addTo(Film& film, int w, bool allowSigned) const {
        const int h = static_cast<int>(cnt.size()) / w;
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const size_t i = static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x);
                film.addBatch(x, y, Color3f(sum[3 * i], sum[3 * i + 1], sum[3 * i + 2]), cnt[i], allowSigned);
            }
    }
};

class CudaRenderDevice final : public RenderDevice {
public:
    CudaRenderDevice(pe_device* d, DeviceInfo info) : m_dev(d), m_info(std::move(info)) {}
    ~CudaRenderDevice() override {
        m_scene.reset();
        pe_device_destroy(m_dev);
    }

    const DeviceInfo& info() const override { return m_info; }
    DeviceFeatures features() const override {
        DeviceFeatures f;
        f.aovs = true;
        f.lightPasses = true;
        f.adaptiveSampling = true;
        return f;
    }
    bool hasScene() const override { return m_scene && pe_device_has_scene(m_dev) != 0; }

    void setScene(std::shared_ptr<const Scene> scene) override {
        m_scene.reset();
        m_sceneRef.reset();
        if (!scene) return;
        auto built = std::make_unique<PeScene>();
        if (!built->build(*scene)) {
            std::cerr << "cuda device: " << built->error << "\n";
            return;
        }
        if (pe_device_set_scene(m_dev, built->s) != PE_OK) {
            std::cerr << "cuda device: " << pe_last_error() << "\n";
            return;
        }
        m_scene = std::move(built);
        m_sceneRef = std::move(scene);
    }

    void updateScene(std::shared_ptr<const Scene> scene, SceneUpdateKind kind) override {
        if (!scene || !m_scene) return setScene(std::move(scene));
        if (kind == SceneUpdateKind::Transforms) {
            // new instance matrices: the device refits its top-level tree, no BLAS is rebuilt
            if (m_scene->moveInstances(*scene) && pe_device_update_transforms(m_dev, m_scene->s) == PE_OK) {
                m_sceneRef = std::move(scene);
                return;
            }
            return setScene(std::move(scene));
        }
        if (scene.get() != m_scene->source) return setScene(std::move(scene));
        bool ok = false;
        if (kind == SceneUpdateKind::Materials) {
            ok = true;
            for (const auto& [m, index] : m_scene->materials) {
                pe_material p;
                if (index < 0 || !m_scene->describe(m, p) || pe_scene_set_material(m_scene->s, index, &p) != PE_OK) {
                    ok = false;
                    break;
                }
            }
            ok = ok && pe_device_update_materials(m_dev, m_scene->s) == PE_OK;
        } else if (kind == SceneUpdateKind::Lights) {
            ok = true;
            for (const auto& [li, a] : m_scene->areaLights) {
                float r[3];
                put3(r, a->radiance());
                if (pe_scene_set_area_light_radiance(m_scene->s, li, r) != PE_OK) {
                    ok = false;
                    break;
                }
            }
            ok = ok && pe_device_update_lights(m_dev, m_scene->s) == PE_OK;
        }
        if (!ok) setScene(std::move(scene)); // the change needs a rebuild
    }

    SampleBatchResult render(const Camera& camera, const RenderSettings& settings, RenderTargets& targets,
                             int firstSample, int count, const std::atomic<bool>* cancel) override {
        SampleBatchResult r;
        r.completed = false;
        if (!targets.beauty || !hasScene()) return r;
        Film& film = *targets.beauty;
        const int w = film.width(), h = film.height();
        const size_t n = static_cast<size_t>(w) * static_cast<size_t>(h);
        const CameraGpuDesc c = camera.describeGpu();
        pe_camera pc{};
        put3(pc.position, c.position);
        put3(pc.lower_left, c.lowerLeft);
        put3(pc.horizontal, c.horizontal);
        put3(pc.vertical, c.vertical);
        put3(pc.u, c.u);
        put3(pc.v, c.v);
        put3(pc.forward, c.forward);
        pc.lens_radius = c.lensRadius;
        pc.orthographic = c.orthographic ? 1 : 0;
        pc.blades = c.blades;
        pc.blade_rotation = c.bladeRotation;
        if (camera.hasShutterEnd()) { // Camera::setShutterEnd
            const CameraGpuDesc e = camera.describeGpuEnd();
            pc.has_shutter_end = 1;
            put3(pc.end_position, e.position);
            put3(pc.end_lower_left, e.lowerLeft);
            put3(pc.end_horizontal, e.horizontal);
            put3(pc.end_vertical, e.vertical);
            put3(pc.end_u, e.u);
            put3(pc.end_v, e.v);
            put3(pc.end_forward, e.forward);
            pc.end_lens_radius = e.lensRadius;
        }
        // Renderer::renderSamples: Sobol seed 12345, roulette after depth 3 (renderer.cpp:431-432)
        pe_settings ps{w, h, settings.maxBounces, 3, settings.shadowQuality,
                       static_cast<int32_t>(settings.filter.type), settings.filter.width, settings.clampIndirect,
                       12345u, settings.aoStrength, settings.adaptiveSampling ? 1 : 0, settings.noiseThreshold,
                       settings.minAdaptiveSamples, settings.motionBlur ? 1 : 0};
        // RenderSettings::pathGuiding: the SD-tree on the device (trained over samples 0-31)
        if (settings.pathGuiding != m_guiding) {
            if (pe_device_set_guiding(m_dev, settings.pathGuiding ? 2 : 0, 0, 0.0f) != PE_OK) return r;
            m_guiding = settings.pathGuiding;
        }
        // the cancel flag as the C ABI reads it, mirrored while the call runs
        volatile int32_t stop = 0;
        std::atomic<bool> running{true};
        std::thread watcher;
        if (cancel)
            watcher = std::thread([&] {
                while (running.load()) {
                    if (cancel->load()) stop = 1;
                    std::this_thread::sleep_for(std::chrono::milliseconds(1));
                }
            });
        int32_t rc;
        uint64_t traced = 0;
        if (settings.adaptiveSampling) {
            // the session's exact sums: reset when a new accumulation starts
            if (firstSample == 0 || m_adaptive.cnt.size() != n) m_adaptive.reset(n);
            Arrays before = m_adaptive;
            rc = pe_device_render(m_dev, &pc, &ps, firstSample, count, &stop, m_adaptive.sum.data(),
                                  m_adaptive.cnt.data(), m_adaptive.sq.data(), &traced);
            if (rc == PE_OK || rc == PE_ERR_CANCELLED) {
                Arrays batch;
                batch.reset(n);
                for (size_t i = 0; i < n; ++i) {
                    batch.cnt[i] = m_adaptive.cnt[i] - before.cnt[i];
                    for (int k = 0; k < 3; ++k) batch.sum[3 * i + k] = m_adaptive.sum[3 * i + k] - before.sum[3 * i + k];
                }
                batch.addTo(film, w, false);
            }
        } else {
            Arrays beauty;
            beauty.reset(n);
            Arrays albedo, normal, alpha;
            pe_aov_films aov{};
            if (targets.aovs) {
                albedo.reset(n);
                normal.reset(n);
                alpha.reset(n);
                aov = pe_aov_films{albedo.sum.data(), albedo.cnt.data(), albedo.sq.data(), normal.sum.data(),
                                   normal.cnt.data(), alpha.sum.data(), alpha.cnt.data(), alpha.sq.data()};
            }
            std::vector<Arrays> passes;
            std::vector<float> cryptoObj, cryptoMat;
            pe_pass_films pf{};
            if (targets.passes) {
                RenderPassFilms& P = *targets.passes;
                const int groups = static_cast<int>(P.lightGroups.size());
                passes.resize(static_cast<size_t>(PE_LIGHT_PASSES + 4 + groups));
                for (Arrays& a : passes) a.reset(n);
                for (int k = 0; k < PE_LIGHT_PASSES; ++k) pf.light[k] = passes[static_cast<size_t>(k)].view();
                pf.depth = passes[PE_LIGHT_PASSES + 0].view();
                pf.position = passes[PE_LIGHT_PASSES + 1].view();
                pf.object_id = passes[PE_LIGHT_PASSES + 2].view();
                pf.material_id = passes[PE_LIGHT_PASSES + 3].view();
                pf.n_groups = groups;
                for (int g = 0; g < groups && g < PE_MAX_LIGHT_GROUPS; ++g)
                    pf.groups[g] = passes[static_cast<size_t>(PE_LIGHT_PASSES + 4 + g)].view();
                if (P.cryptoObject.width() > 0) {
                    cryptoObj.assign(n * static_cast<size_t>(count), 0.0f);
                    cryptoMat.assign(n * static_cast<size_t>(count), 0.0f);
                    pf.crypto_object = cryptoObj.data();
                    pf.crypto_material = cryptoMat.data();
                }
            }
            if (targets.passes)
                rc = pe_device_render_passes(m_dev, &pc, &ps, firstSample, count, &stop, beauty.sum.data(),
                                             beauty.cnt.data(), beauty.sq.data(), targets.aovs ? &aov : nullptr, &pf,
                                             &traced);
            else if (targets.aovs)
                rc = pe_device_render_aovs(m_dev, &pc, &ps, firstSample, count, &stop, beauty.sum.data(),
                                           beauty.cnt.data(), beauty.sq.data(), &aov, &traced);
            else
                rc = pe_device_render(m_dev, &pc, &ps, firstSample, count, &stop, beauty.sum.data(), beauty.cnt.data(),
                                      beauty.sq.data(), &traced);
            if (rc == PE_OK || rc == PE_ERR_CANCELLED) {
                beauty.addTo(film, w, false);
                if (targets.aovs) {
                    albedo.addTo(targets.aovs->albedo, w, false);
                    normal.addTo(targets.aovs->normal, w, true);
                    alpha.addTo(targets.aovs->alpha, w, false);
                }
                if (targets.passes) {
                    RenderPassFilms& P = *targets.passes;
                    for (int k = 0; k < PE_LIGHT_PASSES; ++k) passes[static_cast<size_t>(k)].addTo(P.light[k], w, false);
                    passes[PE_LIGHT_PASSES + 0].addTo(P.depth, w, false);
                    passes[PE_LIGHT_PASSES + 1].addTo(P.position, w, true);
                    passes[PE_LIGHT_PASSES + 2].addTo(P.objectId, w, false);
                    passes[PE_LIGHT_PASSES + 3].addTo(P.materialId, w, false);
                    for (size_t g = 0; g < P.lightGroups.size(); ++g)
                        passes[PE_LIGHT_PASSES + 4 + g].addTo(P.lightGroups[g].second, w, false);
                    if (!cryptoObj.empty()) {
                        // the samples that ran, in sample order per pixel
                        for (int s = 0; s < count; ++s)
                            for (int y = 0; y < h; ++y)
                                for (int x = 0; x < w; ++x) {
                                    const size_t i = static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x);
                                    if (static_cast<uint32_t>(s) >= beauty.cnt[i]) continue;
                                    const size_t o = static_cast<size_t>(s) * n + i;
                                    P.cryptoObject.addSample(x, y, cryptoObj[o]);
                                    P.cryptoMaterial.addSample(x, y, cryptoMat[o]);
                                }
                    }
                }
            }
        }
        running.store(false);
        if (watcher.joinable()) watcher.join();
        r.samplesTraced = traced;
        r.completed = rc == PE_OK;
        if (rc != PE_OK && rc != PE_ERR_CANCELLED) std::cerr << "cuda device: " << pe_last_error() << "\n";
        return r;
    }

private:
    pe_device* m_dev;
    DeviceInfo m_info;
    std::unique_ptr<PeScene> m_scene;
    std::shared_ptr<const Scene> m_sceneRef;
    Arrays m_adaptive;
    bool m_guiding = false;
};

} // namespace

std::unique_ptr<RenderDevice> createCudaRenderDevice(int ordinal, std::string* error) {
    char err[256] = {};
    pe_device* d = pe_device_create(ordinal, err, sizeof(err));
    if (!d) {
        if (error) *error = err;
        return nullptr;
    }
    pe_device_info di{};
    DeviceInfo info;
    info.id = "cuda:" + std::to_string(ordinal);
    info.kind = DeviceKind::Cuda;
    if (pe_device_info_get(d, &di) == PE_OK) {
        info.name = di.name;
        info.memoryBytes = di.memory_bytes;
        info.computeMajor = di.compute_major;
        info.computeMinor = di.compute_minor;
    }
    info.usable = true;
    info.note = "B200 wavefront path tracer (sm_100a)";
    return std::make_unique<CudaRenderDevice>(d, std::move(info));
}

} // namespace photon
