// pe_scene.h — the flattened scene as the kernels read it from HBM.  Every array is a
// separate allocation (SoA), 16-byte aligned, built once on the host (pe_host.cpp) and kept
// resident until the next set_scene.
//
// Layout (per unit):
//   BVH interior node   64 B  4 x float4: child boxes interleaved (c0.x, c1.x | c0.y, c1.y |
//                             c0.z, c1.z) and child references; a leaf child is ~firstPrim with
//                             its count beside it.  Same binary tree, same child order and the
//                             same leaf triangle order as the reference's SAH BVH
//                             (src/geometry/bvh.cpp:100-255), so traversal visits nodes and
//                             tests triangles in the reference's order.
//   leaf triangle       48 B  (v0, parallelEps) (e1, visibility mask) (e2, global triangle id),
//                             the lean record of BVH::TriAccel (bvh.h:84-88) in leaf order
//   triangle shading    16 B  vertex indices + shape id; vertices 16 B (pos), 16 B (normal), 8 B (uv)
//   material           256 B  resolved parameters (pe_material plus derived constants)
//   light               80 B  triangle light or rectangle (src/lights/area_light.h)
#pragma once

#include "pe_math.h"
#include "pe_xform.h"

#if !defined(__CUDACC__)
// The host compiler's stand-ins for CUDA's vector types, with CUDA's alignment, so that every
// struct below has one layout in both compilers.
struct alignas(16) float4 { float x, y, z, w; };
struct alignas(8) float2 { float x, y; };
struct alignas(16) int4 { int x, y, z, w; };
#endif
static_assert(alignof(float4) == 16 && alignof(int4) == 16 && alignof(float2) == 8,
              "host and device must lay out the scene structs alike");

namespace pe {

constexpr int kTableN = 32;          // microfacet / sheen table resolution (microfacet.cpp:13)
constexpr int kFilterBins = 512;     // pixel filter inverse CDF bins (pixel_filter.cpp:13)
constexpr int kMaxExhaustive = 33;   // LightSampler::kMaxExhaustive (light_sampler.h:31)
constexpr int kMaxInfinite = 16;     // LightSampler::kMaxInfinite
constexpr int kMaxStack = 64;        // traversal stack entries; builder rejects deeper trees
constexpr int kWideStack = 96;       // 4-wide traversal stack entries (at most 3 per level + 1)

enum ShapeFlags : uint32_t {
    SF_AREA_TRIANGLE = 1u,   // one of the two triangles of an AreaLight (a Triangle shape)
    SF_CAMERA_INVISIBLE = 2u,
    SF_HAS_NORMALS = 4u,
    SF_HAS_UVS = 8u,
    SF_SPHERE = 16u,         // an analytic sphere
    SF_INSTANCE = 32u,       // a MeshInstance
};

// A leaf record whose b.w meta has this bit is an analytic sphere (Sphere, src/geometry/sphere.h):
// a = (centre, radius); the other words hold the meta and the global primitive id as for a triangle.
constexpr uint32_t PRIM_SPHERE = 1u << 16;
// ... or a MeshInstance: a.x holds the instance index; its BLAS's leaf records follow the top
// level's in the same array, its nodes the top level's nodes.
constexpr uint32_t PRIM_INSTANCE = 1u << 17;
// A closest hit inside an instance is reported as kInstanceHit | instance << 21 | BLAS-local
// record (negative, never -1): at most kMaxInstances instances, kMaxBlasRecords records a BLAS.
constexpr int32_t kMaxInstances = 1023;
constexpr int32_t kMaxBlasRecords = (1 << 21) - 1;

// A MeshInstance (mesh_instance.cpp): world-to-local and local-to-world (row-major rows 0-3), its
// BLAS's root in the binary and in the 4-wide tree (a node index or a leaf reference) and first
// leaf record, the global id of the BLAS's first triangle, the shape and the material.
struct InstGPU {
    float4 w2l[4];
    float4 l2w[4];
    int32_t rootBinary, rootWide, recBase, firstTri;
    int32_t shape, material;
    float uvScale;   // 1 / cbrt(|det|) of the 3×3 part (uvDensity, mesh_instance.cpp:95-98)
    int32_t motion;  // index into SceneGPU::motions of a moving instance, -1 none
};

// A moving MeshInstance (MeshInstance::setMotionTransform): the pose at shutter close as given and
// the time-independent half of interpolateTransform for the poses between.
struct InstMotionGPU {
    float4 l2w1[4], w2l1[4];
    MotionTRS trs;
    float uvScale1;
    int32_t pad[3];
};

struct ShapeInfo {
    int32_t material;
    int32_t emitter;      // light index of triangle 0 (emissive mesh) or of the area light; -1 none
    uint32_t flags;
    uint32_t firstTri;    // global index of the shape's first triangle
    int32_t linkNode;     // bit of its node uid in the light-link masks; kLinkNodeOther if no link names it
};

// Light linking (Light::setLightLink, Scene::isLightLinked / isShadowLinked, scene.cpp:121-141,
// 242-256): the node uids that light links name are numbered 0..62; a link is a mode (0 all,
// 1 include, 2 exclude) and a 64-bit mask over those numbers, for lit receivers and for blockers.
constexpr int kLinkNodeOther = 63;
struct LightLinkGPU {
    unsigned long long mask, shadowMask;
    int32_t mode, shadowMode;
};

// Resolved material (pe_material + constants derived on the host).
struct MatGPU {
    int32_t type;
    int32_t flags;            // MF_*
    float base[3];
    float emission[3];
    float metallic, roughness, specular, clearcoat, clearcoatRoughness;
    float ior, specTrans, coatIor;
    float coatTint[3];
    float sheenColor[3];
    int32_t hasSheenColor;
    float anisotropy, sheen, sheenRoughness, diffuseRoughness, diffuseTransmission, subsurface;
    float ssRadius[3];
    float ssScale, ssAniso;
    float edgeTint[3];
    float thinFilmThickness, thinFilmIor;
    float flakeDensity, flakeSize, flakeRoughness;
    float flakeColor[3];
    float opacity;
    float glassRoughness;
    float abbe;
    float sigmaA[3], sigmaS[3];  // interior medium of a Dielectric (rebuildMedium)
    float mediumG;
    int32_t thinWalled;
    float filmThickness;
    float roundEdge;          // Material::roundEdgeRadius (0 = off)
    // DisneyMaterial image textures (disney.h:133-145): texture indices (-1 none), mapping
    // (0 UV, 1 box), scale
    int32_t texAlbedo, texRoughness, texMetalness, texNormal;
    int32_t texMapping;
    float texScale;
    int32_t texOpacity;       // opacity map (DisneyMaterial::setOpacityImage), red channel
};

// An RGB float image (Image, Float32 storage) read by bilinear lookups with wrap; with mipmaps
// (Image::buildMipmaps) its levels follow level 0 in `texels`.
constexpr int kMaxMipLevels = 16;
struct TexGPU {
    const float* texels; // level 0 then levels 1.. (each width·height·3)
    int32_t width, height;
    int32_t levels;      // 1 without mipmaps
    int32_t levelW[kMaxMipLevels], levelH[kMaxMipLevels];
    int32_t levelOffset[kMaxMipLevels]; // in floats
};

enum MatFlags : int32_t {
    MF_EMISSIVE = 1,
    MF_DELTA = 2,             // Material::isDelta
    MF_VOLUME_BOUNDARY = 4,   // Material::isVolumeBoundary
    MF_TRANSMITS_SHADOWS = 8,
    MF_DISPERSIVE = 16,
    MF_HAS_MEDIUM = 32,
    MF_MEDIUM_SCATTERS = 64,
};

enum LightType : int32_t { LT_TRIANGLE = 0, LT_AREA = 1 };

struct LightGPU {
    int32_t type;
    int32_t rectangle;  // AreaLight: u ⟂ v (spherical-rectangle sampling allowed)
    float area;
    float pad0;
    float p0[3];        // triangle p0 | area position
    float radiance_r;
    float p1[3];        // triangle p1 | area u
    float radiance_g;
    float p2[3];        // triangle p2 | area v
    float radiance_b;
    float normal[3];
    float pad1;
};

// Light BVH node (LightSampler::Node with LightBounds, light_sampler.h:57-61, light_bounds.h:16-26).
struct LightNodeGPU {
    float bmin[3], bmax[3];
    float w[3];
    float phi, cosThetaO, cosThetaE;
    int32_t twoSided;
    int32_t child1;
    int32_t light;
    int32_t pad;
};

struct TablesGPU {
    float ggxE[kTableN * kTableN];
    float ggxEa[kTableN * kTableN];
    float ggxEb[kTableN * kTableN];
    float avg0[kTableN], avg1[kTableN], avg2[kTableN];
    float sheenE[kTableN * kTableN];
    uint32_t sobolTab[4][256];
    float spectralCdf[351];
    float spectralPdf[350];
    float spectralNorm[3];
    float pad;
};

// Environment light (src/lights/environment_light.h:52-153).  The image distribution used for
// light sampling and for pdfLi is the MIS-compensated one (m_mis).
struct EnvGPU {
    int32_t present;
    int32_t width, height;
    int32_t hasImage;
    float rotation, intensity;
    float meanLuminance;
    float sunPdfWeight;
    float sunDir[3];
    float sunCosMax;
    float sunRadiance[3];
    float funcInt;      // m_mis.funcInt
    int32_t valid;      // m_mis.valid()
    int32_t pad[3];
    const float* image; // w*h*3
    const float* func;  // w*h
    const float* marginalCdf; // h+1
    const float* condCdf;     // h*(w+1)
};

struct SceneGPU {
    // geometry
    const float4* nodes;     // 4 float4 per interior node
    const float4* wide;      // 8 float4 per 4-wide node (null when the root is a leaf)
    const float4* tris;      // 3 float4 per leaf-ordered triangle
    const int4* triVerts;    // per global triangle: i0, i1, i2, shape
    const float4* pos;       // per vertex
    const float4* nrm;       // per vertex
    const float2* uv;        // per vertex
    const ShapeInfo* shapes;
    const MatGPU* materials;
    int32_t rootIsLeaf;      // tiny scenes: the whole BVH is one leaf
    int32_t rootFirst, rootCount;
    int32_t nNodes;
    float rootMin[3], rootMax[3];
    uint32_t nTris;
    int32_t nShapes;
    // lights
    const LightGPU* lights;
    int32_t nLights;
    int32_t lightMode;       // 0 uniform, 1 exhaustive, 2 light BVH
    int32_t lightCount;      // candidates = nLights + env
    int32_t nInfinite;
    int32_t infinite[kMaxInfinite];
    const LightNodeGPU* lightNodes;
    int32_t nLightNodes;
    int32_t pad0;
    const int16_t* topSlot;          // per candidate
    const unsigned long long* trail; // per candidate
    const uint8_t* trailDepth;       // per candidate
    EnvGPU env;
    EnvGPU envFull;          // the same light with its uncompensated distribution (shadow catcher)
    const TablesGPU* tables;
    int32_t bgMode;
    float bgColor[3];
    int32_t hasShadowTransmitters;
    int32_t hasVolumes;      // some material is a volume boundary: paths carry a medium stack
    int32_t hasSubsurface;   // some Disney material has a subsurface lobe (random walks)
    int32_t exitMaterial;    // white Lambert of the subsurface exit vertex
    int32_t catcherShape;    // Scene::setShadowCatcher's shape, -1 none
    const LightLinkGPU* links; // per explicit light (null without light links)
    int32_t hasLightLinks, hasShadowLinks;
    // render passes: light group of each light (null without groups), their number, the
    // environment's group; data-pass colours (shapes, then materials)
    const int32_t* lightGroup;
    int32_t nLightGroups, envGroup;
    const float4* idColor;
    const TexGPU* textures;  // image textures (null without any)
    int32_t nTextures;
    int32_t hasMips;         // some texture has mipmaps: paths carry ray cones for its LOD
    // 1 when no material or scene setting needs the shading features a plain surface scene
    // leaves unused (volumes, subsurface walks, dispersion, cutouts, rounded edges, ray cones,
    // light or shadow links, a shadow catcher): its waves may shade with the lean kernels
    int32_t leanShading;
    int32_t materialTypes;   // bit t: some material has type t
    const InstGPU* instances; // MeshInstances (null without)
    int32_t nInstances;
    const InstMotionGPU* motions; // moving instances (null without)
};

// Scene::isLightLinked / isShadowLinked for light `li` (explicit) and a receiver or blocker node.
PE_HD bool linkAllows(int mode, unsigned long long mask, int node) {
    if (mode == 0) return true;
    const bool found = node < kLinkNodeOther && ((mask >> node) & 1ull) != 0ull;
    return mode == 1 ? found : !found;
}

} // namespace pe
