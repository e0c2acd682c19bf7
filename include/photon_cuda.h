/*
 * photon_cuda.h — C ABI of the B200 (sm_100a) path-tracing device.
 *
 * This is the boundary a host renderer binds to: plain pointers, sizes and
 * status codes, no C++ or torch types.  It fills the empty CUDA slot of the
 * reference engine's render-device interface:
 *
 *   reference interface                                      replaced by
 *   ---------------------------------------------------------------------------
 *   RenderDevice::info / features (src/engine/render_device.h:69-70)
 *                                                            pe_device_info
 *   RenderDevice::setScene / updateScene (render_device.h:74-79)
 *                                                            pe_device_set_scene
 *   RenderDevice::render (render_device.h:84-85)             pe_device_render
 *   createDevice("cuda:N", &error) (src/engine/render_device.cpp:110-157)
 *                                                            pe_device_create
 *   probeCudaDevices() usable=false (src/engine/gpu_probe.cpp:85-127)
 *                                                            pe_device_count
 *   Scene::addShape / addLight / setEnvironment / buildAccelerator
 *     (src/engine/scene.cpp:18-185)                          pe_scene_*
 *   Film::addBatch (src/core/image/film.cpp:119-137)         accumulation done by
 *                                                            pe_device_render into
 *                                                            caller-owned arrays
 *
 * Errors: every call returns a pe_status (0 = PE_OK) or a NULL handle; the
 * message of the last failure on the calling thread is pe_last_error().
 * No exception crosses this boundary.  Device handles are independent, so
 * two threads may drive two devices concurrently (as the reference's hybrid
 * device does); one handle must not be driven by two threads at once.
 */
#ifndef PHOTON_CUDA_H
#define PHOTON_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PE_ABI_VERSION 10

typedef enum pe_status {
    PE_OK = 0,
    PE_ERR_INVALID = 1,   /* bad argument or handle */
    PE_ERR_CUDA = 2,      /* CUDA runtime error */
    PE_ERR_NO_SCENE = 3,  /* render before set_scene */
    PE_ERR_CANCELLED = 4, /* cancel flag seen; film holds whole samples only */
    PE_ERR_OOM = 5,       /* device memory exhausted */
    PE_ERR_DEVICE = 6,    /* kernel reported an error status (bounded wait, bounds) */
    PE_ERR_LIMIT = 7      /* request larger than a documented maximum */
} pe_status;

/* ---- materials (src/materials) ------------------------------------------- */
enum {
    PE_MAT_LAMBERT = 0,    /* Lambertian (src/materials/lambertian.h:17)          */
    PE_MAT_DISNEY = 1,     /* DisneyMaterial (src/materials/disney.h:24)          */
    PE_MAT_DIELECTRIC = 2, /* Dielectric (src/materials/dielectric.h)             */
    PE_MAT_MIRROR = 3      /* Mirror (src/materials/mirror.h)                     */
};

/* Resolved, texture-free material parameters.  Field meaning and clamping
 * follow the reference setters (disney.h:50-160, dielectric.h).  Fill with
 * pe_material_defaults() and override. */
typedef struct pe_material {
    int32_t type;
    float base_color[3]; /* lambert albedo | disney base | dielectric tint | mirror reflectance */
    float emission[3];
    /* Disney / OpenPBR */
    float metallic, roughness, specular;
    float clearcoat, clearcoat_roughness;
    float ior, spec_transmission, coat_ior;
    float coat_tint[3];
    float sheen_color[3];
    int32_t has_sheen_color;
    float anisotropy, sheen, sheen_roughness;
    float diffuse_roughness, diffuse_transmission;
    float subsurface;
    float subsurface_radius[3];
    float subsurface_scale, subsurface_anisotropy;
    float edge_tint[3];
    float thin_film_thickness, thin_film_ior;
    float flake_density, flake_size, flake_roughness;
    float flake_color[3];
    float opacity;
    /* Dielectric */
    float glass_roughness;
    float abbe;
    float absorb_color[3];
    float absorb_distance;
    float scatter_density;
    float scatter_color[3];
    float scatter_anisotropy;
    int32_t thin_walled;
    float film_thickness;
    int32_t has_absorption; /* setAbsorption called (builds the interior medium) */
    int32_t has_scattering; /* setScattering called */
    /* any type */
    float round_edge_radius; /* Material::setRoundEdgeRadius (material.h:136); 0 = off */
    /* Disney image maps (DisneyMaterial::set{Albedo,Roughness,Metalness,Normal}Image, disney.h:142-145):
     * indices from pe_scene_add_texture, -1 none; roughness reads green, metalness blue */
    int32_t albedo_texture, roughness_texture, metalness_texture, normal_texture;
    int32_t texture_mapping;  /* 0 UV, 1 box projection (DisneyMaterial::TextureMapping) */
    float texture_scale;      /* DisneyMaterial::setTextureScale (≥ 1e-4) */
    int32_t opacity_texture;  /* DisneyMaterial::setOpacityImage: opacity × the red channel, -1 none */
} pe_material;

/* Camera as the reference's Camera::describeGpu() (src/camera/camera.h:17-29). */
typedef struct pe_camera {
    float position[3];
    float lower_left[3];
    float horizontal[3];
    float vertical[3];
    float u[3];
    float v[3];
    float forward[3];
    float lens_radius;
    int32_t orthographic;
    int32_t blades;         /* thin lens: aperture polygon sides (0 = round disk) */
    float blade_rotation;   /* thin lens: polygon rotation, radians */
    /* Camera::setShutterEnd (camera.h:48-55): the pose at shutter close (t = 1) when has_shutter_end
     * is non-zero.  With motion blur a ray at time t > 0 mixes the two descriptions linearly, its
     * lens a round disk (Camera::generateRay(u, v, lens, time), camera.h:58-90). */
    int32_t has_shutter_end;
    float end_position[3];
    float end_lower_left[3];
    float end_horizontal[3];
    float end_vertical[3];
    float end_u[3];
    float end_v[3];
    float end_forward[3];
    float end_lens_radius;
} pe_camera;

enum { PE_FILTER_BOX = 0, PE_FILTER_TRIANGLE = 1, PE_FILTER_GAUSSIAN = 2, PE_FILTER_BLACKMAN_HARRIS = 3 };
enum { PE_BG_ENVIRONMENT = 0, PE_BG_COLOR = 1, PE_BG_TRANSPARENT = 2 };

/* RenderSettings subset that changes the estimator (src/engine/render_settings.h:19-47). */
typedef struct pe_settings {
    int32_t width, height;
    int32_t max_bounces;    /* PathTracer maxDepth */
    int32_t rr_depth;       /* Russian roulette after this depth (reference: 3) */
    int32_t shadow_quality; /* NEE samples per vertex */
    int32_t filter_type;    /* PE_FILTER_* */
    float filter_width;
    float clamp_indirect;   /* 0 = off */
    uint64_t seed;          /* Owen-Sobol seed (reference renderSamples: 12345) */
    float ao_strength;      /* RenderSettings::aoStrength: contact AO at camera hits; 0 = off */
    int32_t adaptive_sampling;    /* RenderSettings::adaptiveSampling: clean pixels stop early */
    float noise_threshold;        /* relative standard error target (reference default 0.02; >= 1e-4 used) */
    int32_t min_adaptive_samples; /* samples before any decision (reference default 16; >= 2 used) */
    int32_t motion_blur;    /* RenderSettings::motionBlur: each camera sample draws a shutter time
                               (one more Sobol dimension, renderer.cpp:152-153) that moves the
                               camera and mesh instances with a motion transform */
} pe_settings;

/* ---- scene builder --------------------------------------------------------- */
typedef struct pe_scene pe_scene;

typedef struct pe_scene_info {
    uint64_t triangles;
    uint64_t bvh_nodes;   /* interior nodes of the flattened BVH */
    uint64_t bvh_leaves;
    uint64_t lights;      /* explicit lights incl. one per emissive triangle */
    uint64_t light_bvh_nodes;
    uint64_t device_bytes;
    int32_t has_environment;
    int32_t light_sampler_mode; /* 0 uniform, 1 exhaustive, 2 light BVH */
} pe_scene_info;

void pe_material_defaults(int32_t type, pe_material* out);
pe_scene* pe_scene_create(void);
void pe_scene_destroy(pe_scene* s);
/* Returns the material index (>= 0) or -1. */
int32_t pe_scene_add_material(pe_scene* s, const pe_material* m);
/* Scene::addShape(TriangleMesh) — normals/uvs may be NULL (normals are then
 * computed as in TriangleMesh::calculateNormals, src/geometry/mesh.cpp:30-55).
 * An emissive material registers one triangle light per triangle. */
int32_t pe_scene_add_mesh(pe_scene* s, const float* positions, uint32_t n_vertices, const float* normals,
                          const float* uvs, const uint32_t* indices, uint32_t n_triangles, int32_t material);
/* Sphere (src/geometry/sphere.h): an analytic sphere of the given centre and radius (> 0), one
 * shape and one BVH primitive, hit by Sphere::intersect's quadratic (sphere.cpp:12-90).  Like the
 * reference it is never a light, even with an emissive material. */
int32_t pe_scene_add_sphere(pe_scene* s, const float center[3], float radius, int32_t material);

/* Mesh instancing (MeshInstance, src/geometry/mesh_instance.h; Scene::addShape, scene.cpp:23-41).
 * pe_scene_add_blas keeps a triangle mesh for instancing and returns its id (or -PE_*): it gets
 * its own BVH (a BLAS, built once, at most 2,097,151 triangles; a mesh of at most 16 triangles is
 * one leaf tested in index order) and is not a shape by itself.  pe_scene_add_instance places it
 * by a row-major local-to-world matrix (column vectors, translation in the last column) with the
 * inverse the caller composed (NULL: Mat4f::inverse's cofactor expansion) and a material; the
 * instance is one shape and one top-level primitive, rays are carried into its space and its
 * BLAS walked (mesh_instance.cpp:104-133).  At most 1023 instances a scene.  An emissive
 * instance gives one light per triangle, placed by the transform. */
int32_t pe_scene_add_blas(pe_scene* s, const float* positions, uint32_t nv, const float* normals, const float* uvs,
                          const uint32_t* indices, uint32_t ntri);
int32_t pe_scene_add_instance(pe_scene* s, int32_t blas, const float local_to_world[16], const float world_to_local[16],
                              int32_t material);
/* MeshInstance::setMotionTransform (mesh_instance.h:20-21): instance shape `shape`'s local-to-world
 * matrix at shutter close (t = 1; world_to_local its inverse, NULL = Mat4f::inverse).  A ray at
 * time t meets the instance under interpolateTransform(t0, t1, t) (quat.cpp: translation and scale
 * linear, rotation by SLERP); its top-level box merges five poses over the shutter.  Lights of an
 * emissive instance stay at t0, as Scene::addShape places them.  Call before pe_scene_build. */
int32_t pe_scene_set_instance_motion(pe_scene* s, int32_t shape, const float local_to_world_end[16],
                                     const float world_to_local_end[16]);
/* Shape::bounds of shape `shape` (world box: lo xyz, hi xyz): a mesh's vertices, a sphere's cube,
 * a mesh instance's BLAS box under its transform (Arvo), over the shutter for a moving instance. */
int32_t pe_scene_shape_bounds(const pe_scene* s, int32_t shape, float out[6]);
/* Transform(m)'s inverse as the reference computes it (Mat4f::inverse, mat.h:130-175: cofactors
 * of 2×2 minors, identity for a singular matrix), row-major; what pe_scene_add_instance uses when
 * world_to_local is NULL.  For composing Transform products (A·B)⁻¹ = B⁻¹·A⁻¹ on the host. */
void pe_mat4_inverse(const float m[16], float out[16]);
/* SceneUpdateKind::Transforms: new matrices for instance shape `shape` of a built scene; then
 * pe_device_update_transforms refits the top-level tree on the device without rebuilding any
 * BLAS.  An emissive instance (its lights move) returns PE_ERR_LIMIT: rebuild the scene. */
int32_t pe_scene_set_instance_transform(pe_scene* s, int32_t shape, const float local_to_world[16],
                                        const float world_to_local[16]);
/* Refits a built scene's top-level tree to its instances' current matrices: boxes recomputed
 * bottom up, the tree's shape and leaf order kept (pe_device_update_transforms calls it). */
int32_t pe_scene_refit(pe_scene* s);
/* Scene::tagShape (scene.h:108): the scene-node uid of a shape (counted as for
 * pe_scene_set_shadow_catcher), which light links name. */
int32_t pe_scene_tag_shape(pe_scene* s, int32_t shape, uint64_t node_uid);
/* Light::setLightLink (light.h:23-32, 80-81) of explicit light `light` (the scene's lights in the
 * order they were registered: one per area light, one per triangle of an emissive mesh): mode 0
 * all receivers, 1 only those whose node uid is listed, 2 all but those; shadow_mode likewise for
 * the blockers that shadow this light (others are passed through).  At most 63 distinct uids over
 * all links (PE_ERR_LIMIT at pe_scene_build otherwise). */
int32_t pe_scene_set_light_link(pe_scene* s, int32_t light, int32_t mode, const uint64_t* uids, int32_t n,
                                int32_t shadow_mode, const uint64_t* shadow_uids, int32_t n_shadow);
/* Scene::setShadowCatcher (scene.h:90): the shape that camera rays see as the background darkened
 * by the shadows falling on it (path_tracer.cpp:515-563); -1 = none.  Shapes count from 0 in the
 * order they were added: one per pe_scene_add_mesh, two per pe_scene_add_area_light (its two
 * triangles, as Scene::addLight adds them).  Call before pe_scene_build. */
int32_t pe_scene_set_shadow_catcher(pe_scene* s, int32_t shape);
/* Scene::setShapeName / setMaterialName: the names the Cryptomatte ids hash (unnamed shapes are
 * "object_<node uid>" or "shape_<n>", unnamed materials "material_<n>", renderer.cpp:75-118). */
int32_t pe_scene_set_shape_name(pe_scene* s, int32_t shape, const char* name);
int32_t pe_scene_set_material_name(pe_scene* s, int32_t material, const char* name);
/* Shape::setVisibilityMask (shape.h:27-29; VisibilityMask, ray.h:18-25): the ray classes that see
 * shape `shape`, bits camera 1, diffuse 2, glossy 4, transmission 8, shadow 16 (default 31).  A
 * mesh instance's mask is tested at the top level only.  Call before pe_scene_build. */
int32_t pe_scene_set_shape_visibility(pe_scene* s, int32_t shape, uint32_t mask);
/* Replaces material `index` of a scene (built or not) for an incremental update: its type,
 * emission and the media, shadow-transmission and subsurface switches must stay as they were,
 * else PE_ERR_LIMIT (rebuild the scene).  Then pe_device_update_materials sends it to a device. */
int32_t pe_scene_set_material(pe_scene* s, int32_t index, const pe_material* m);
/* AreaLight radiance of light `light` (a built scene's light sampler is rebuilt on the host). */
int32_t pe_scene_set_area_light_radiance(pe_scene* s, int32_t light, const float radiance[3]);
/* An RGB float image (w*h*3, row 0 first) for the Disney image maps; returns its index (>= 0)
 * or a negative status.  Lookups are Image::sampleBilinear's (src/core/image/image.cpp:98-225):
 * bilinear, wrapping, without mipmaps. */
int32_t pe_scene_add_texture(pe_scene* s, const float* rgb, int32_t width, int32_t height);
/* Image::buildMipmaps (src/core/image/image.cpp:102-155) of texture `texture`: lookups then
 * select a level from the ray cone's footprint (sampleTex, src/materials/disney.cpp:530-539). */
int32_t pe_scene_build_texture_mipmaps(pe_scene* s, int32_t texture);
/* An 8-bit RGB image (Image::createCompact8, src/core/image/image.cpp:49-60): sRGB-encoded when
 * srgb != 0, else linear; looked up as the reference decodes it (a 256-entry table; mip levels
 * quantised to 8 bits).  The device holds the decoded values as floats. */
int32_t pe_scene_add_texture_u8(pe_scene* s, const uint8_t* rgb, int32_t width, int32_t height, int32_t srgb);
/* Light::setLightGroup (src/lights/light.h:85) of light `light` (the numbering of
 * pe_scene_set_light_link), or of the environment when light == -1; "" or NULL clears it.
 * Scene::buildAccelerator forms the groups (src/engine/scene.cpp:144-174): none unless some
 * light names one; then every light joins its group or "Default", the environment its group or
 * "Env", at most PE_MAX_LIGHT_GROUPS groups. */
int32_t pe_scene_set_light_group(pe_scene* s, int32_t light, const char* name);
/* Scene::lightGroupNames after pe_scene_build: returns the number of groups and, when names is
 * not NULL, writes them NUL-separated into names[0, capacity). */
int32_t pe_scene_light_groups(const pe_scene* s, char* names, int32_t capacity);
/* Scene::addLight(AreaLight) — rectangle p + s*u + t*v, two-sided, plus its
 * two emissive triangles in the BVH (src/engine/scene.cpp:65-99). */
int32_t pe_scene_add_area_light(pe_scene* s, const float p[3], const float u[3], const float v[3],
                                const float radiance[3], int32_t visible_to_camera);
/* EnvironmentLight(image, rotation, intensity) (src/lights/environment_light.cpp:64).
 * rgb == NULL gives the constant grey environment of the reference. */
int32_t pe_scene_set_environment(pe_scene* s, const float* rgb, int32_t width, int32_t height, float rotation,
                                 float intensity);
/* EnvironmentLight::setSun (environment_light.cpp:211-227). */
int32_t pe_scene_set_sun(pe_scene* s, const float direction[3], float cos_max, const float radiance[3]);
/* Scene::setBackground (src/engine/scene.h:41). */
int32_t pe_scene_set_background(pe_scene* s, int32_t mode, const float color[3]);
/* Scene::buildAccelerator: SAH BVH, light sampler, environment CDFs. */
int32_t pe_scene_build(pe_scene* s);
int32_t pe_scene_get_info(const pe_scene* s, pe_scene_info* out);

/* PerspectiveCamera(position, target, up, vfov, aspect) → pe_camera
 * (src/camera/perspective_camera.cpp:12-32). */
void pe_camera_perspective(const float position[3], const float target[3], const float up[3], float vfov_deg,
                           float aspect, pe_camera* out);
/* ThinLensCamera (src/camera/thin_lens_camera.cpp:14-33, setApertureShape :31-34): depth of field
 * with an aperture of `aperture_radius` focused at `focus_distance`; blades >= 3 makes the
 * aperture a regular polygon rotated by rotation_deg. */
void pe_camera_thin_lens(const float position[3], const float target[3], const float up[3], float vfov_deg,
                         float aspect, float aperture_radius, float focus_distance, int32_t blades, float rotation_deg,
                         pe_camera* out);
/* OrthographicCamera (src/camera/orthographic_camera.cpp:11-41): parallel rays over a
 * vertical_extent-high image plane through `position`. */
void pe_camera_orthographic(const float position[3], const float target[3], const float up[3],
                            float vertical_extent, float aspect, pe_camera* out);

/* ---- device ---------------------------------------------------------------- */
typedef struct pe_device pe_device;

typedef struct pe_device_info {
    char name[128];
    uint64_t memory_bytes;
    int32_t compute_major, compute_minor;
    int32_t sm_count;
    int32_t usable;
    int32_t feature_aovs, feature_light_passes, feature_adaptive;
    char pci_bus_id[32];
} pe_device_info;

typedef struct pe_render_stats {
    uint64_t paths;            /* camera samples traced */
    uint64_t closest_rays;     /* closest-hit segments */
    uint64_t shadow_rays;      /* any-hit segments */
    uint64_t rejected;         /* non-finite / negative samples counted black */
    uint64_t waves;
    float ms_total;            /* device time of the last render call */
    float ms_intersect;        /* device time in closest-hit traversal */
    float ms_shadow;           /* device time in any-hit traversal */
    float ms_shade;
    uint64_t intersect_launches;
    uint64_t node_visits;      /* closest-hit BVH node visits (counting enabled only) */
    uint64_t tri_tests;        /* closest-hit triangle tests (counting enabled only) */
    uint32_t error_flags;      /* kernel error word (0 = none) */
    uint64_t kernel_launches;  /* kernels this library launched in the last render call */
    uint64_t shadow_node_visits; /* any-hit BVH node visits (counting enabled only) */
    uint64_t shadow_tri_tests;   /* any-hit triangle tests (counting enabled only) */
    uint64_t tail_paths;       /* paths finished by the per-thread tail kernel */
    float ms_tail;             /* device time in the tail kernel (timed renders only) */
    uint32_t pad0;
    uint64_t tail_closest_rays; /* closest-hit segments traced by the tail kernel (in closest_rays) */
    uint64_t tail_shadow_rays;  /* any-hit segments traced by the tail kernel (in shadow_rays) */
} pe_render_stats;

const char* pe_last_error(void);
int32_t pe_abi_version(void);
int32_t pe_device_count(void);
pe_device* pe_device_create(int32_t ordinal, char* err, size_t err_len);
void pe_device_destroy(pe_device* d);
int32_t pe_device_info_get(pe_device* d, pe_device_info* out);
int32_t pe_device_set_scene(pe_device* d, const pe_scene* s);
int32_t pe_device_has_scene(pe_device* d);
/* RenderDevice::updateScene with SceneUpdateKind::Materials (src/engine/render_device.h:77-79):
 * copies the material table of the scene last set (same build) to the device again, leaving its
 * geometry, BVH, lights and textures in place. */
int32_t pe_device_update_materials(pe_device* d, const pe_scene* s);
/* SceneUpdateKind::Lights: after pe_scene_set_area_light_radiance edits, the lights, their quads'
 * materials and the light sampler go to the device again (PE_ERR_LIMIT when the sampler's tree
 * changed shape: set the scene again). */
int32_t pe_device_update_lights(pe_device* d, const pe_scene* s);
/* SceneUpdateKind::Transforms: after pe_scene_set_instance_transform edits, refits the scene's
 * top-level tree and sends only it, the instance table and the root box; no BLAS is rebuilt or
 * sent.  The film is the one a rebuilt scene gives, except where two triangles give the
 * identical hit distance (the refitted tree may visit them in another order). */
int32_t pe_device_update_transforms(pe_device* d, pe_scene* s);

/* RenderDevice::render: adds samples [first_sample, first_sample+count) to every
 * pixel and accumulates into the caller's host arrays exactly as
 * Film::addBatch would (sum_rgb: w*h*3 floats, sample_count: w*h, sum_lum_sq:
 * w*h, may be NULL).  cancel (may be NULL) is polled between waves; a
 * cancelled call returns PE_ERR_CANCELLED after adding only whole waves. */
int32_t pe_device_render(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first_sample,
                         int32_t count, const volatile int32_t* cancel, float* sum_rgb, uint32_t* sample_count,
                         float* sum_lum_sq, uint64_t* samples_traced);

/* AOV films (AovFilms, src/engine/renderer.h:42-53): the first visible surface's albedo, its
 * normal, and coverage — each a Film's arrays (sum of RGB, sample count, sum of squared
 * luminance), merged like the beauty film; a NULL array is skipped. */
typedef struct pe_aov_films {
    float* albedo_sum;
    uint32_t* albedo_count;
    float* albedo_sum_sq;
    float* normal_sum;   /* signed (Film::addSampleSigned); no squares are kept */
    uint32_t* normal_count;
    float* alpha_sum;    /* coverage in all three channels */
    uint32_t* alpha_count;
    float* alpha_sum_sq;
} pe_aov_films;
/* pe_device_render plus the AOV films of the same samples (RenderDevice::render with
 * RenderTargets::aovs; tracePixel with wantAovs, renderer.cpp:139-204). */
int32_t pe_device_render_aovs(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first_sample,
                              int32_t count, const volatile int32_t* cancel, float* sum_rgb, uint32_t* sample_count,
                              float* sum_lum_sq, const pe_aov_films* aovs, uint64_t* traced);

/* Render passes (RenderPassFilms, src/engine/renderer.h:59-98).  Each film is a Film's arrays
 * (sum of RGB, sample count, sum of squared luminance; a NULL array is skipped), merged like
 * the beauty film. */
#define PE_MAX_LIGHT_GROUPS 16
#define PE_LIGHT_PASSES 8
typedef struct pe_film_arrays {
    float* sum;
    uint32_t* count;
    float* sum_sq;
} pe_film_arrays;
typedef struct pe_pass_films {
    /* LightPass order (src/integrators/path_tracer.h:21-24): diffuse direct, diffuse indirect,
     * glossy direct, glossy indirect, transmission direct, transmission indirect, emission,
     * background; their sum is the beauty film */
    pe_film_arrays light[PE_LIGHT_PASSES];
    pe_film_arrays depth;       /* distance from the camera ray's origin to the first hit */
    pe_film_arrays position;    /* first hit point, signed (no squares are kept) */
    pe_film_arrays object_id;   /* idColor of the hit shape's node uid (pe_scene_tag_shape) */
    pe_film_arrays material_id; /* idColor of the hit material's index + 1 */
    int32_t n_groups;           /* must equal pe_scene_light_groups of the device's scene */
    int32_t pad;
    pe_film_arrays groups[PE_MAX_LIGHT_GROUPS]; /* one per light group, in Scene::lightGroupNames order */
    /* Cryptomatte (CryptoFilm, src/core/image/cryptomatte.h): when not NULL, count·w·h floats
     * each, the object and material id of every sample (index (sample − first)·w·h + y·w + x;
     * 0 on a miss), for the caller's CryptoFilm::addSample */
    float* crypto_object;
    float* crypto_material;
} pe_pass_films;
/* pe_device_render plus the render passes and, when aovs is not NULL, the AOV films of the same
 * samples (RenderDevice::render with RenderTargets::passes; tracePixel with wantPasses,
 * renderer.cpp:139-204, addPasses 206-217). */
int32_t pe_device_render_passes(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first_sample,
                                int32_t count, const volatile int32_t* cancel, float* sum_rgb, uint32_t* sample_count,
                                float* sum_lum_sq, const pe_aov_films* aovs, const pe_pass_films* passes,
                                uint64_t* traced);

/* A render region: pe_device_render restricted to the pixels of the rectangle (x0, y0, w, h) of
 * the st->width x st->height frame.  No counterpart in the reference's RenderDevice; it serves
 * crop renders (a viewport's border region, fixed crop windows of a convergence check) without
 * tracing the rest of the frame.  The host films cover the whole frame as for pe_device_render;
 * only the region's pixels change, each exactly as a whole-frame render would change it (same
 * paths, same per-pixel sample order).  Adaptive sampling is rejected (PE_ERR_INVALID). */
int32_t pe_device_render_region(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t x0, int32_t y0,
                                int32_t w, int32_t h, int32_t first_sample, int32_t count,
                                const volatile int32_t* cancel, float* sum_rgb, uint32_t* sample_count,
                                float* sum_lum_sq, uint64_t* samples_traced);

/* Same, accumulating into the device-resident film (kept across calls until
 * pe_device_film_clear; resized/cleared when width/height change). */
int32_t pe_device_render_resident(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t first_sample,
                                  int32_t count, const volatile int32_t* cancel);
int32_t pe_device_film_clear(pe_device* d);

/* Tile render that allocates no device memory.  No counterpart in the reference engine.
 *
 * For hosts that may not call cudaMalloc/cudaFree while they render: a viewport or plugin
 * running inside another application that owns the GPU's memory budget and hands out device
 * buffers from its own pool, or a render thread that must not hit the driver's allocator (which
 * can block and fragment) in the middle of a frame.  The caller passes the inputs (camera,
 * settings, the scene already set with pe_device_set_scene) and the outputs: sum_rgb
 * (width*height*3 floats), sample_count and sum_lum_sq (width*height each), all DEVICE memory
 * the caller owns, covering the whole film of st->width x st->height.  Samples
 * [first_sample, first_sample+count) of the pixels in the rectangle (x0, y0, w, h) are added to
 * them exactly as pe_device_render would add them; other pixels are not touched.  Each film
 * pointer is checked to be memory of this device that holds the whole film (PE_ERR_INVALID
 * otherwise).  The call runs on the library's own non-blocking stream and does not wait for the
 * caller's streams: finish writing the film buffers before calling, and synchronize the device
 * (pe_device_synchronize) before reading them.
 *
 * It renders plain paths only: a device with guided sampling on (pe_device_set_guiding) and a
 * scene with mipmapped image maps (whose level of detail needs a per-path ray cone) are rejected
 * with PE_ERR_INVALID, as is adaptive sampling; render those with pe_device_render.
 *
 * The path state lives in one file-scope device array of 8.5 MB (room for 32768 paths), which
 * every GPU that loads this library holds until the process exits; its address on a device is
 * taken once, when the device is created.  A tile of more than 32768 pixels (w*h) is rejected
 * with PE_ERR_LIMIT.  Every call uses the same array and finds the previous call's contents in
 * it (the call clears what must start at zero), so calls that run on the GPU at the same time,
 * from two threads or two device handles on one GPU, race and corrupt each other's results. */
int32_t pe_device_render_tile_noalloc(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t x0, int32_t y0,
                                      int32_t w, int32_t h, int32_t first_sample, int32_t count, float* sum_rgb,
                                      uint32_t* sample_count, float* sum_lum_sq);
int32_t pe_device_film_read(pe_device* d, float* sum_rgb, uint32_t* sample_count, float* sum_lum_sq);
int32_t pe_device_synchronize(pe_device* d);
int32_t pe_device_last_stats(pe_device* d, pe_render_stats* out);
/* 1 = count BVH node visits and triangle tests in traversal kernels (slower). */
int32_t pe_device_set_counting(pe_device* d, int32_t enabled);
/* B200 tuning knob with no counterpart in the reference engine.  A wave's paths are traced
 * bounce by bounce (one closest-hit, shade and any-hit launch per bounce) until at most `paths`
 * remain live; those finish in one launch that runs each path to its end on one thread.  The
 * film is the same either way.  -1 (default) = the paths one resident grid holds, 0 = never. */
int32_t pe_device_set_tail_paths(pe_device* d, int64_t paths);
int64_t pe_device_tail_paths(pe_device* d);
/* Autotuner (no reference counterpart): renders probe_spp samples of the view with each of a few
 * tail thresholds (1/4, 1/2, 1 and 2 resident grids) into a scratch film, twice, and keeps the
 * fastest of the second round; chosen (may be NULL) receives it.  The caller's films are untouched. */
int32_t pe_device_autotune(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t probe_spp, int64_t* chosen);

/* B200 tuning knobs with no counterpart in the reference engine; none changes a film.  The
 * autotuner above sets all five by coordinate descent on probe renders of the caller's frame
 * (paths in flight per wave, closest-hit traversal, any-hit traversal, the shading register
 * budget, the tail threshold). */
typedef struct pe_tuning {
    int64_t tail_paths;        /* as pe_device_set_tail_paths */
    int32_t closest_traversal; /* bounce-by-bounce closest hits: 0 the binary tree, 1 the 4-wide tree,
                                  2 / 3 the 4-wide tree with the first 8 / 16 stack entries of each
                                  thread in shared memory (the rest in local memory), 4 / 5 with the
                                  top 4 / 8 stack entries in registers, 6 (default) the 4-wide tree
                                  capped at 64 registers (eight 128-thread blocks per SM), 7 / 8 that
                                  with the first 8 / 16 stack entries in shared memory, 9 that with
                                  leaf tests postponed until the warp holds a leaf in every lane.
                                  Mode 9 only on request (the autotuner leaves it out): which of two
                                  triangles at a bit-identical distance wins then depends on the
                                  rays that share the warp, so films are no longer bit-identical
                                  across batchings and switch points where such ties occur */
    int32_t shade_budget;      /* lean shading kernels: 0 the compiler's register count, 1 (default) at
                                  most 128 registers a thread (four 128-thread blocks per SM), 2 at
                                  most 96 (five blocks) */
    int32_t any_traversal;     /* plain any-hit shadows: 0 the stack in local memory, 1 its top 4
                                  entries in registers, 2 (default) capped at 64 registers */
    int64_t wave_slots;        /* paths in flight in a regenerating wave (unguided renders without
                                  AOV or pass targets): 2^20 … 2^23, default 2^23; 0 on input keeps
                                  the current value.  Each of the device's two lanes holds path
                                  state for that many paths (536 B a slot, 256 B of it the radiance
                                  of the paths the slots cycle through: 9 GB for both lanes at
                                  2^23), allocated at the next render and never shrunk */
} pe_tuning;
int32_t pe_device_get_tuning(pe_device* d, pe_tuning* out);
int32_t pe_device_set_tuning(pe_device* d, const pe_tuning* t);
/* The last pe_device_autotune's probe times, one "knob=value time ms" line each, into buf
 * (NUL-terminated, truncated to len); returns the full length. */
int32_t pe_device_autotune_log(pe_device* d, char* buf, size_t len);
/* Device-stream timer: events recorded on the stream the kernels run on; end waits for the
 * stop event and returns the elapsed device milliseconds. */
int32_t pe_device_timer_begin(pe_device* d);
int32_t pe_device_timer_end(pe_device* d, float* ms);

/* ---- diagnostics used by parity tests --------------------------------------- */
/* Camera ray of (x, y, sample_index) for every pixel, then closest hit:
 * shape index (mesh/area-light triangle order of insertion; -1 = miss),
 * triangle index within the shape, t.  Follows Renderer tracePixel +
 * BVH::intersect (src/engine/renderer.cpp:139-160, src/geometry/bvh.cpp:322-401),
 * through the 4-wide tree the render kernels traverse: t equals the reference's bit
 * for bit; where two triangles give the identical t the other of them may be reported. */
int32_t pe_device_trace_primary(pe_device* d, const pe_camera* cam, const pe_settings* st, int32_t sample_index,
                                int32_t* out_shape, int32_t* out_prim, float* out_t);
/* The same through the binary tree in the reference's own visiting order (near child first,
 * last tested triangle wins a tie), so ids are the reference's bit for bit, ties included. */
/* Ray queries against the device's scene (Scene::intersect / intersectAny, bvh.cpp:322-446;
 * a test probe): n rays (origins, directions xyz; t in [0, t_max[i]]) with visibility mask `mask`
 * at shutter time `time`.  mode 0: closest hit on the binary tree in the reference's visiting
 * order, 1: closest hit on the 4-wide tree — shape, triangle within the shape and t (shape -1 on
 * a miss); 2: any hit on the 4-wide tree — out_shape 1 when occluded, else 0. */
int32_t pe_device_trace_rays(pe_device* d, const float* origins, const float* directions, const float* t_max,
                             int32_t n, int32_t mode, uint32_t mask, float time, int32_t* out_shape,
                             int32_t* out_prim, float* out_t);
int32_t pe_device_trace_primary_ordered(pe_device* d, const pe_camera* cam, const pe_settings* st,
                                        int32_t sample_index, int32_t* out_shape, int32_t* out_prim, float* out_t);

/* Owen-scrambled Sobol values: for each i, (px[i], py[i], index[i]) and
 * n_dims consecutive 2-D dimensions → out[i*n_dims*2 + 2*k + {0,1}]. */
int32_t pe_device_sobol(pe_device* d, uint64_t seed, const int32_t* px, const int32_t* py, const int32_t* index,
                        size_t n, int32_t n_dims, float* out);

/* BSDF probe: evaluates or samples material m of the current scene at a
 * synthetic shading point. */
typedef struct pe_bsdf_query {
    float wo[3], wi[3];
    float normal[3], ng[3], tangent[3], point[3];
    int32_t front_face;
    float wavelength;
    float uc, u[2];
} pe_bsdf_query;

typedef struct pe_bsdf_result {
    float f[3];
    float pdf;
    int32_t sampled;  /* sample: success */
    float wi[3];      /* sample: direction */
    float sf[3];      /* sample: f */
    float spdf;       /* sample: pdf */
    int32_t delta, pass_through, subsurface;
    float weight[3];  /* sample: subsurface weight */
} pe_bsdf_result;

int32_t pe_device_bsdf_probe(pe_device* d, int32_t material, const pe_bsdf_query* q, size_t n, pe_bsdf_result* out);

/* ---- Learned directional proposal ---------------------------------------------------------------
 * A hash grid over the scene box (16 levels x 2 features) plus the shading normal and the view
 * direction feed a 3x64 MLP (FP16 weights, FP32 accumulation) whose 40 outputs are an 8-lobe von
 * Mises-Fisher mixture over incident directions: 5 per lobe (direction x, y, z before
 * normalisation, log kappa clamped to [-6, 7], weight logit).  The learned counterpart of the
 * reference's SD-tree guiding (src/integrators/path_guiding.cpp); no reference function computes
 * it.  Parameter block layout (FP32): W1[64][48], b1[64], W2[64][64], b2, W3[64][64], b3,
 * W4[64][64], b4[64] (15616 floats); grid 16 x 2^18 x 2 floats. */
enum { PE_GUIDE_MLP_PARAMS = 15616, PE_GUIDE_GRID_PARAMS = 16 * 262144 * 2, PE_GUIDE_OUTPUTS = 40 };
/* (Re)initialises the network from a seed over the box [box_min, box_max]; with both NULL, over
 * the current scene's box as pe_device_set_guiding chooses it (so a later set_guiding keeps it). */
int32_t pe_device_guide_reset(pe_device* d, uint64_t seed, const float box_min[3], const float box_max[3]);
int32_t pe_device_guide_get(pe_device* d, float* mlp, float* grid);
int32_t pe_device_guide_set(pe_device* d, const float* mlp, const float* grid);
/* Network outputs for n queries (9 floats each: position, shading normal, direction to the
 * viewer) → out (40 floats each).  tensor_cores = 1: the tcgen05 path the renderer uses; 0: the
 * same network in FP32 on the SIMT cores. */
int32_t pe_device_guide_eval(pe_device* d, const float* queries, int64_t n, int32_t tensor_cores, float* out);
/* Gradient of sum_i c_i * (-log q(w_i | x_i)) over n samples (13 floats each: position, normal,
 * view direction, sampled direction w, weight c) into mlp_grad / grid_grad (either may be NULL),
 * and the loss; lr > 0 then takes one Adam step with the batch-mean gradient. */
int32_t pe_device_guide_grad(pe_device* d, const float* samples, int64_t n, float lr, float* mlp_grad, float* grid_grad,
                             float* loss);
/* Rendering with the proposal: mode 1 trains the network after every wave on up to 64K of its
 * paths (each one's first guidable vertex: the radiance that arrived along the sampled direction,
 * over the sampling pdf) and, once warmup_steps Adam steps are done, draws every guidable vertex of the
 * first bounces (not the tail kernel's) by one-sample MIS of proposal and BSDF, 50/50, as the
 * reference's SD-tree guiding does.  The estimate stays unbiased; results depend on the
 * training history, so batches no longer equal single passes bit for bit.  Guided renders use
 * one wave lane.  mode 0 turns it off (the network is kept).
 * mode 2 is the reference's SD-tree guiding (RenderSettings::pathGuiding, renderer.cpp:413-429):
 * a render from sample 0, or the first one on a new scene, starts a new field over the scene's
 * bounds; the first 32 samples run in chunks of 2, 2, 4, 8, 16, each recording its paths'
 * vertices into the field and refining it after, and all later samples draw from the frozen field
 * (path_tracer.cpp:625-735, 823-883).  warmup_steps and lr are ignored. */
int32_t pe_device_set_guiding(pe_device* d, int32_t mode, int32_t warmup_steps, float lr);
typedef struct pe_guide_info {
    int32_t mode;
    int32_t ready;       /* sampling with the proposal */
    int64_t steps;       /* Adam steps taken */
    float last_loss;     /* sum of c * (-log q) of the last batch */
    float pad;
} pe_guide_info;
int32_t pe_device_guide_info(pe_device* d, pe_guide_info* out);

/* ---- SD-tree guiding (GuidingField / DirectionalTree, src/integrators/path_guiding.{h,cpp}) ---- */
typedef struct pe_sdtree_info {
    int32_t ready;           /* GuidingField::ready() */
    int32_t refinements;     /* GuidingField::refine calls since the field was built */
    int32_t samples;         /* samples per pixel the field was trained on (<= 32) */
    int32_t spatial_leaves;  /* GuidingField::spatialLeafCount() */
    int64_t quad_nodes;      /* nodes of all sampling quadtrees */
    double energy;           /* sum of the sampling trees' totals */
} pe_sdtree_info;
int32_t pe_device_sdtree_info(pe_device* d, pe_sdtree_info* out);
/* Host-only check of one directional quadtree (no device needed): splats n1 (direction,
 * radiance) pairs, refines (DirectionalTree::buildFrom with split fraction 0.01, depth 10),
 * splats n2 more into the refined topology, refines again, then evaluates pdf(qdirs[i]) → pdf_out[i]
 * and sample(qu[i]) → sample_out[4i..4i+3] = (direction, pdf) for nq queries. */
int32_t pe_sdtree_probe(const float* dirs1, const float* rad1, int32_t n1, const float* dirs2, const float* rad2,
                        int32_t n2, const float* qdirs, const float* qu, int32_t nq, float* pdf_out,
                        float* sample_out);

/* ---- Request server ---------------------------------------------------------------------------
 * The served form of the render path; no class of the reference engine serves requests (its
 * RenderSession drives one device for one view).  Scenes stay resident; each
 * request (scene, camera, settings, spp) gets a device film when the HBM budget has room for
 * it; a worker thread packs the pending sample ranges of the admitted requests of one scene into
 * shared waves (continuous batching: a request submitted while waves run joins the next wave),
 * highest priority first, then least remaining work.  A request's film equals, bit for bit, the
 * film of pe_device_render over samples [0, spp) alone.  While a server runs it owns its device:
 * render nothing else on that device until pe_server_destroy, after which the device has the
 * scene it had before. */
typedef struct pe_server pe_server;

enum { PE_REQ_QUEUED = 0, PE_REQ_ACTIVE = 1, PE_REQ_DONE = 2, PE_REQ_FAILED = 3, PE_REQ_RELEASED = 4 };

typedef struct pe_request_desc {
    int32_t scene;          /* id from pe_server_add_scene */
    pe_camera camera;
    pe_settings settings;   /* film size, depth, filter, seed, ... */
    int32_t spp;            /* samples [0, spp) per pixel */
    int32_t priority;       /* larger first */
} pe_request_desc;

typedef struct pe_request_status {
    int32_t state;          /* PE_REQ_* */
    int32_t samples_done;   /* samples finished on every pixel */
    double submit_ms;       /* server clock (ms since pe_server_create) */
    double start_ms;        /* admitted: film allocated */
    double done_ms;         /* last sample in the device film */
    uint64_t paths;
    int32_t error;          /* PE_* status of a failed request */
    int32_t pad;
} pe_request_status;

typedef struct pe_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t queued, active;
    uint64_t waves, paths, segments;
    double busy_ms;               /* device time of the waves, each counted whole (two may overlap) */
    uint64_t film_bytes, film_bytes_peak, budget_bytes, scene_bytes;
} pe_server_stats;

/* budget_bytes bounds the device memory of resident scenes plus admitted films. */
pe_server* pe_server_create(pe_device* d, uint64_t budget_bytes, char* err, size_t err_len);
void pe_server_destroy(pe_server* s);
/* Uploads a built scene and keeps it resident; returns its id (>= 0) or a negative PE_* status. */
int32_t pe_server_add_scene(pe_server* s, const pe_scene* scene);
/* Queues a request; returns its id (>= 0) or a negative PE_* status (a film larger than the
 * whole budget is PE_ERR_LIMIT). */
int64_t pe_server_submit(pe_server* s, const pe_request_desc* r);
int32_t pe_server_status(pe_server* s, int64_t id, pe_request_status* out);
/* Waits until the request is done or failed, at most timeout_ms (< 0: no limit).  PE_OK when
 * done, PE_ERR_CANCELLED on timeout, the request's error when it failed. */
int32_t pe_server_wait(pe_server* s, int64_t id, int32_t timeout_ms);
/* Copies a done request's film out (any pointer may be NULL) and releases its device memory. */
int32_t pe_server_take(pe_server* s, int64_t id, float* sum_rgb, uint32_t* sample_count, float* sum_lum_sq);
int32_t pe_server_get_stats(pe_server* s, pe_server_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* PHOTON_CUDA_H */
