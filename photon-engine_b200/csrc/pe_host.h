// pe_host.h — host-side scene representation and the flattened build the device uploads.
#pragma once

#include "photon_cuda.h"
#include "pe_scene.h"

#include <string>
#include <vector>

namespace pe {

struct HostShape {
    std::vector<V3> pos, nrm;
    std::vector<V2> uv;
    std::vector<uint32_t> idx;
    int32_t material = -1;
    uint32_t flags = 0;
    int32_t emitter = -1;
    uint8_t mask = 0x1F;
    bool sphere = false;        // an analytic sphere (Sphere, src/geometry/sphere.h): one primitive
    V3 center{0.0f, 0.0f, 0.0f};
    float radius = 0.0f;
    int32_t blas = -1;          // a MeshInstance of this BLAS (src/geometry/mesh_instance.h): one primitive
    float l2w[16] = {}, w2l[16] = {}; // its local-to-world matrix and inverse, row-major
    bool motion = false;        // MeshInstance::setMotionTransform: the pose at shutter close
    float l2w1[16] = {}, w2l1[16] = {};
};

// A mesh kept for instancing: its own BVH (BLAS), shared by its instances.
struct HostBlas {
    std::vector<V3> pos, nrm;
    std::vector<V2> uv;
    std::vector<uint32_t> idx;
    uint32_t flags = 0;         // SF_HAS_NORMALS / SF_HAS_UVS
};

struct HostEnv {
    bool present = false;
    bool hasImage = false;
    int width = 0, height = 0;
    float rotation = 0.0f, intensity = 1.0f;
    std::vector<float> image;                 // w*h*3
    std::vector<float> fullFunc, misFunc;     // w*h
    std::vector<float> fullMarg, misMarg;     // h+1
    std::vector<float> fullCond, misCond;     // h*(w+1)
    float fullInt = 0.0f, misInt = 0.0f;
    bool fullValid = false, misValid = false;
    float meanLuminance = 0.0f;
    float sunPdfWeight = 0.0f;
    V3 sunDir{0, 1, 0};
    float sunCosMax = 1.0f;
    V3 sunRadiance{0, 0, 0};
    bool hasSun = false;
    V3 sunDirIn{0, 1, 0};
    float sunCosIn = 1.0f;
    V3 sunRadIn{0, 0, 0};
};

// Everything the device uploads, as flat host arrays.
struct HostBuild {
    std::vector<float4> nodes;       // 4 per interior node
    std::vector<float4> wide;        // 8 per 4-wide node (traversal kernels)
    int wideDepth = 0;
    std::vector<InstGPU> instances;  // per MeshInstance shape (in shape order)
    std::vector<InstMotionGPU> motions; // per moving instance
    uint32_t tlasPrims = 0;          // leaf records of the top-level tree; BLAS records follow
    // the top-level tree as built, for refitting its boxes after instance transforms change
    struct TreeNode {
        float lo[3], hi[3];
        int32_t offset, count;   // leaf: first leaf-order primitive and count; interior: second child, 0
    };
    std::vector<TreeNode> tlasRef;
    std::vector<size_t> tlasOrdered;
    std::vector<float> tlasPrimBounds; // 6 per primitive: lo, hi
    std::vector<int4> tlasWideKids;  // per top-level wide node, its children's binary node indices
    int32_t tlasInterior = 0;        // binary interior nodes of the top level (the first in `nodes`)
    std::vector<float4> tris;        // 3 per leaf-ordered triangle
    std::vector<int4> triVerts;      // per global triangle
    std::vector<float4> pos, nrm;    // per vertex (global)
    std::vector<float2> uv;
    std::vector<ShapeInfo> shapes;
    std::vector<MatGPU> materials;
    std::vector<LightGPU> lights;
    std::vector<LightNodeGPU> lightNodes;
    std::vector<int16_t> topSlot;
    std::vector<unsigned long long> trail;
    std::vector<uint8_t> trailDepth;
    std::vector<int32_t> infinite;
    int32_t lightMode = 0;
    int32_t lightCount = 0;
    int32_t rootIsLeaf = 0, rootFirst = 0, rootCount = 0;
    float rootMin[3] = {0, 0, 0}, rootMax[3] = {0, 0, 0};
    uint64_t leaves = 0;
    int maxDepth = 0;
    bool hasShadowTransmitters = false;
    bool hasVolumes = false;
    bool hasSubsurface = false;
    bool hasDispersion = false;
    int32_t exitMaterial = -1;   // white Lambert of the subsurface exit vertex
    int32_t catcherShape = -1;   // shadow-catcher shape
    std::vector<LightLinkGPU> links; // per explicit light, empty without links
    int32_t hasLightLinks = 0, hasShadowLinks = 0;
    // light groups (Scene::buildAccelerator, scene.cpp:144-174): names, group of each light, of
    // the environment; empty when no light names a group
    std::vector<std::string> groupNames;
    std::vector<int32_t> lightGroup;
    int32_t envGroup = -1;
    // data-pass colours: object id of each shape, then material id of each material
    std::vector<float4> idColor;
};

struct HostLightLink {
    int32_t mode = 0, shadowMode = 0;
    std::vector<uint64_t> uids, shadowUids;
};

} // namespace pe

struct pe_scene {
    struct Texture {
        std::vector<float> texels; // width·height·3
        int32_t width = 0, height = 0;
        std::vector<std::vector<float>> mips; // levels 1.. (pe_scene_build_texture_mipmaps)
        std::vector<int32_t> mipW, mipH;
        int32_t format = 0; // 0 float, 1 8-bit sRGB, 2 8-bit linear (texels hold the decoded values)
    };
    std::vector<Texture> textures;             // pe_scene_add_texture
    std::vector<pe_material> materialsIn;
    std::vector<pe::MatGPU> materials;
    std::vector<pe::HostShape> shapes;
    std::vector<pe::HostBlas> blases;          // pe_scene_add_blas
    std::vector<pe::LightGPU> lights;
    pe::HostEnv env;
    int32_t bgMode = PE_BG_ENVIRONMENT;
    float bgColor[3] = {0.18f, 0.18f, 0.18f};
    bool built = false;
    int32_t catcherShape = -1;   // Scene::setShadowCatcher
    std::vector<uint64_t> shapeUid;            // Scene::tagShape (0 = untagged)
    std::vector<pe::HostLightLink> lightLinks; // Light::setLightLink, by explicit light index
    std::vector<std::string> lightGroups;      // Light::setLightGroup, by light index ("" = none)
    std::string envLightGroup;                 // the environment's Light::setLightGroup
    std::vector<std::string> shapeNames;       // Scene::setShapeName ("" = unnamed)
    std::vector<std::string> materialNames;    // Scene::setMaterialName
    pe::HostBuild build;
    uint64_t version = 0;
    uint64_t materialVersion = 0; // pe_scene_set_material edits since the build
    uint64_t transformVersion = 0; // pe_scene_set_instance_transform edits since the build
    uint64_t refitVersion = 0;     // pe_scene_refit calls since the build
};

namespace pe {
// Thread-local last error shared by the host and device halves of the ABI.
void setError(const std::string& msg);
const TablesGPU& staticTables();           // GGX / sheen / Sobol / spectral tables
void fillFilterCdf(int type, float width, float* cdf); // 513 entries; cdf[0] = -1 for box
}
