// pe_host.cpp — host side of the scene boundary: accepts the reference engine's scene content
// (meshes, materials, lights, environment) through the pe_scene_* C ABI and flattens it into
// the resident GPU layout of pe_scene.h.  The acceleration structures are built with the same
// algorithms, float operations and tie rules as the reference so the device traverses the same
// tree:
//   SAH BVH          src/geometry/bvh.cpp:11-255 (12 buckets, leaf when cost >= N and N <= 255)
//   vertex normals   src/geometry/mesh.cpp:30-55
//   emitter lights   src/engine/scene.cpp:18-99 (one TriangleLight per emissive triangle,
//                    two BVH triangles per area light)
//   light sampler    src/lights/light_sampler.cpp:42-148 (exhaustive <= 33 candidates, else
//                    light BVH with PBRT-v4 cost and bit trails)
//   environment      src/lights/environment_light.cpp:64-227 (full and MIS-compensated CDFs)
//   energy tables    src/materials/microfacet.cpp:36-163 (deterministic stratified integration)
// Compiled with -ffp-contract=off so every float result matches the reference's parity build.
#include "pe_host.h"
#include "pe_bsdf.h"
#include "pe_light.h"
#include "pe_medium.h"
#include "pe_xform.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>

namespace pe {

namespace {
thread_local std::string tlsError;
}
void setError(const std::string& msg) { tlsError = msg; }

namespace {

// ---------------------------------------------------------------------------------------------
// AABB with the reference's empty box (+max, -max) and std::min/max merges (aabb.h).
struct Box {
    V3 lo, hi;
    Box() : lo(mk(std::numeric_limits<float>::max())), hi(mk(-std::numeric_limits<float>::max())) {}
    Box(V3 a, V3 b) : lo(vmin(a, b)), hi(vmax(a, b)) {}
    Box merged(const Box& o) const {
        Box r;
        r.lo = vmin(lo, o.lo);
        r.hi = vmax(hi, o.hi);
        return r;
    }
    void merge(V3 p) {
        lo = vmin(lo, p);
        hi = vmax(hi, p);
    }
    void merge(const Box& o) {
        lo = vmin(lo, o.lo);
        hi = vmax(hi, o.hi);
    }
    V3 centroid() const { return (lo + hi) * 0.5f; }
    V3 diagonal() const { return hi - lo; }
    float surfaceArea() const {
        const V3 d = diagonal();
        return 2.0f * (d.x * d.y + d.x * d.z + d.y * d.z);
    }
    int maxExtent() const {
        const V3 d = diagonal();
        if (d.x > d.y && d.x > d.z) return 0;
        if (d.y > d.z) return 1;
        return 2;
    }
    V3 offset(V3 p) const {
        V3 o = p - lo;
        const V3 d = diagonal();
        if (d.x > 0.0f) o.x /= d.x;
        if (d.y > 0.0f) o.y /= d.y;
        if (d.z > 0.0f) o.z /= d.z;
        return o;
    }
};

struct BuildPrim {
    size_t primIndex;
    Box bounds;
    V3 centroid;
    BuildPrim(size_t i, const Box& b) : primIndex(i), bounds(b), centroid(b.centroid()) {}
};

struct BuildNode {
    Box bounds;
    BuildNode* child[2] = {nullptr, nullptr};
    int axis = 0;
    int first = 0;
    int count = 0;
};

struct RefNode { // BVHNode (bvh.h:27-36): 32-byte depth-first node
    Box bounds;
    int offset;  // leaf: first prim; interior: second child
    int count;   // leaf prim count, 0 for interior
};

// ---- transforms (src/core/math/mat.h, transform.cpp), row-major 4×4 ------------------------------
constexpr uint32_t VIS_ALL_MASK = 0x1Fu; // a BLAS is traversed with every visibility bit (mesh_instance.cpp:110)
constexpr int32_t kNoRoot = static_cast<int32_t>(0x80000000u);


// Transform::transformPoint (transform.cpp:15-26).
V3 xfPoint(const float* m, V3 p) {
    const float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    const float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    const float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    const float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
    if (w != 1.0f && w != 0.0f) {
        const float iw = 1.0f / w;
        return mk(x * iw, y * iw, z * iw);
    }
    return mk(x, y, z);
}

// Transform::transformAABB (transform.cpp:83-110): Arvo's bound of the transformed box.
Box xfAABB(const float* m, const Box& b) {
    float lo[3] = {m[3], m[7], m[11]}, hi[3] = {m[3], m[7], m[11]};
    const float bl[3] = {b.lo.x, b.lo.y, b.lo.z}, bh[3] = {b.hi.x, b.hi.y, b.hi.z};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const float a = m[4 * i + j] * bl[j], c = m[4 * i + j] * bh[j];
            if (a < c) {
                lo[i] += a;
                hi[i] += c;
            } else {
                lo[i] += c;
                hi[i] += a;
            }
        }
    Box r;
    r.lo = mk(lo[0], lo[1], lo[2]);
    r.hi = mk(hi[0], hi[1], hi[2]);
    return r;
}


// decomposeTRS (quat.cpp): translation, unit rotation (Quatf::fromMat3 of the orthonormalised
// columns) and signed scale of an affine matrix.
void decomposeTRS(const float* m, float* pos, float* rot, float* scale) {
    pos[0] = m[3];
    pos[1] = m[7];
    pos[2] = m[11];
    const V3 c0 = mk(m[0], m[4], m[8]), c1 = mk(m[1], m[5], m[9]), c2 = mk(m[2], m[6], m[10]);
    const float sx = length(c0), sy = length(c1);
    float sz = length(c2);
    const float det = dot(c0, cross(c1, c2));
    if (det < 0.0f) sz = -sz;
    scale[0] = sx;
    scale[1] = sy;
    scale[2] = sz;
    const V3 x = sx > 1e-8f ? c0 / sx : mk(1.0f, 0.0f, 0.0f);
    V3 y = sy > 1e-8f ? c1 / sy : mk(0.0f, 1.0f, 0.0f);
    y = y - x * dot(x, y);
    if (len2(y) > 1e-12f) y = normalize(y);
    else y = std::fabs(x.y) < 0.9f ? normalize(cross(x, mk(0.0f, 1.0f, 0.0f))) : normalize(cross(x, mk(1.0f, 0.0f, 0.0f)));
    const V3 z = normalize(cross(x, y));
    // Quatf::fromMat3 of r = [x y z] (columns)
    const float r00 = x.x, r10 = x.y, r20 = x.z, r01 = y.x, r11 = y.y, r21 = y.z, r02 = z.x, r12 = z.y, r22 = z.z;
    const float trace = r00 + r11 + r22;
    float q[4];
    if (trace > 0.0f) {
        const float s = std::sqrt(trace + 1.0f) * 2.0f;
        q[3] = 0.25f * s;
        q[0] = (r21 - r12) / s;
        q[1] = (r02 - r20) / s;
        q[2] = (r10 - r01) / s;
    } else if (r00 > r11 && r00 > r22) {
        const float s = std::sqrt(std::max(1e-12f, 1.0f + r00 - r11 - r22)) * 2.0f;
        q[3] = (r21 - r12) / s;
        q[0] = 0.25f * s;
        q[1] = (r01 + r10) / s;
        q[2] = (r02 + r20) / s;
    } else if (r11 > r22) {
        const float s = std::sqrt(std::max(1e-12f, 1.0f + r11 - r00 - r22)) * 2.0f;
        q[3] = (r02 - r20) / s;
        q[0] = (r01 + r10) / s;
        q[1] = 0.25f * s;
        q[2] = (r12 + r21) / s;
    } else {
        const float s = std::sqrt(std::max(1e-12f, 1.0f + r22 - r00 - r11)) * 2.0f;
        q[3] = (r10 - r01) / s;
        q[0] = (r02 + r20) / s;
        q[1] = (r12 + r21) / s;
        q[2] = 0.25f * s;
    }
    quatNormalized(q, rot);
}

// The time-independent half of interpolateTransform(t0, t1, ·) (quat.cpp): both poses decomposed,
// the rotations normalised (Quatf::slerp), the second flipped onto the short arc, the arc's angle
// and sine by the C library.
MotionTRS motionTRS(const float* m0, const float* m1) {
    MotionTRS M;
    std::memset(&M, 0, sizeof(M));
    float r0[4], r1[4], a[4], b[4];
    decomposeTRS(m0, M.p0, r0, M.s0);
    decomposeTRS(m1, M.p1, r1, M.s1);
    quatNormalized(r0, a);
    quatNormalized(r1, b);
    for (int k = 0; k < 4; ++k) {
        M.qa[k] = static_cast<double>(a[k]);
        M.qb[k] = static_cast<double>(b[k]);
    }
    double d = M.qa[0] * M.qb[0] + M.qa[1] * M.qb[1] + M.qa[2] * M.qb[2] + M.qa[3] * M.qb[3];
    if (d < 0.0) {
        d = -d;
        for (int k = 0; k < 4; ++k) M.qb[k] = -M.qb[k];
    }
    M.linear = d > 0.9995 ? 1 : 0;
    M.theta = std::acos(d < -1.0 ? -1.0 : (d > 1.0 ? 1.0 : d));
    M.sinT = std::sin(M.theta);
    return M;
}

// MeshInstance::recomputeBounds (mesh_instance.cpp:36-53): the local box under the transform, or
// for a moving instance the union over five poses a = 0, 1/4, .., 1 of the shutter.
Box instanceBox(const HostShape& sh, const Box& local) {
    if (!sh.motion) return xfAABB(sh.l2w, local);
    const MotionTRS M = motionTRS(sh.l2w, sh.l2w1);
    Box merged;
    for (int i = 0; i <= 4; ++i) {
        const float a = static_cast<float>(i) / 4.0f;
        float m[16], inv[16];
        const float* use = m;
        if (a <= 0.0f) use = sh.l2w;
        else if (a >= 1.0f) use = sh.l2w1;
        else motionPoseAt(M, a, m, inv);
        const Box b = xfAABB(use, local);
        merged = merged.merged(b);
    }
    return merged;
}

class SahBuilder {
public:
    std::vector<BuildPrim> prims;
    std::vector<size_t> ordered; // leaf order → ref index
    int total = 0;
    std::vector<std::unique_ptr<BuildNode>> pool;

    BuildNode* newNode() {
        pool.emplace_back(new BuildNode());
        return pool.back().get();
    }
    void makeLeaf(BuildNode* n, int start, int end, const Box& b) {
        n->first = static_cast<int>(ordered.size());
        for (int i = start; i < end; ++i) ordered.push_back(prims[static_cast<size_t>(i)].primIndex);
        n->count = end - start;
        n->bounds = b;
    }
    void makeInterior(BuildNode* n, int axis, BuildNode* c0, BuildNode* c1) {
        n->child[0] = c0;
        n->child[1] = c1;
        n->bounds = c0->bounds.merged(c1->bounds);
        n->axis = axis;
        n->count = 0;
    }
    // BVH::recursiveBuild (bvh.cpp:100-238).
    BuildNode* build(int start, int end) {
        ++total;
        BuildNode* node = newNode();
        Box bounds;
        for (int i = start; i < end; ++i) bounds = bounds.merged(prims[static_cast<size_t>(i)].bounds);
        const int n = end - start;
        if (n == 1) {
            makeLeaf(node, start, end, bounds);
            return node;
        }
        Box cb;
        for (int i = start; i < end; ++i) cb.merge(prims[static_cast<size_t>(i)].centroid);
        const int dim = cb.maxExtent();
        if (get(cb.hi, dim) == get(cb.lo, dim)) {
            if (n > 4) {
                const int mid = (start + end) / 2;
                BuildNode* a = build(start, mid);
                BuildNode* b = build(mid, end);
                makeInterior(node, dim, a, b);
                return node;
            }
            makeLeaf(node, start, end, bounds);
            return node;
        }
        int mid = (start + end) / 2;
        if (n <= 2) {
            std::nth_element(prims.begin() + start, prims.begin() + mid, prims.begin() + end,
                             [dim](const BuildPrim& a, const BuildPrim& b) { return get(a.centroid, dim) < get(b.centroid, dim); });
        } else {
            constexpr int nB = 12;
            int cnt[nB] = {};
            Box bb[nB];
            for (int i = start; i < end; ++i) {
                int b = static_cast<int>(nB * get(cb.offset(prims[static_cast<size_t>(i)].centroid), dim));
                if (b == nB) b = nB - 1;
                cnt[b]++;
                bb[b] = bb[b].merged(prims[static_cast<size_t>(i)].bounds);
            }
            float cost[nB - 1];
            for (int i = 0; i < nB - 1; ++i) {
                Box b0, b1;
                int c0 = 0, c1 = 0;
                for (int j = 0; j <= i; ++j) {
                    b0 = b0.merged(bb[j]);
                    c0 += cnt[j];
                }
                for (int j = i + 1; j < nB; ++j) {
                    b1 = b1.merged(bb[j]);
                    c1 += cnt[j];
                }
                cost[i] = 1.0f + (c0 * b0.surfaceArea() + c1 * b1.surfaceArea()) / bounds.surfaceArea();
            }
            float minCost = cost[0];
            int split = 0;
            for (int i = 1; i < nB - 1; ++i)
                if (cost[i] < minCost) {
                    minCost = cost[i];
                    split = i;
                }
            const float leafCost = static_cast<float>(n);
            if (n > 255 || minCost < leafCost) {
                auto pm = std::partition(prims.begin() + start, prims.begin() + end, [=](const BuildPrim& bp) {
                    int b = static_cast<int>(nB * get(cb.offset(bp.centroid), dim));
                    if (b == nB) b = nB - 1;
                    return b <= split;
                });
                mid = static_cast<int>(pm - prims.begin());
                if (mid != start && mid != end) {
                    BuildNode* a = build(start, mid);
                    BuildNode* b = build(mid, end);
                    makeInterior(node, dim, a, b);
                    return node;
                }
            }
            makeLeaf(node, start, end, bounds);
            return node;
        }
        BuildNode* a = build(start, mid);
        BuildNode* b = build(mid, end);
        makeInterior(node, dim, a, b);
        return node;
    }
    // BVH::flattenBVHTree (bvh.cpp:240-255): depth-first, first child follows its parent.
    int flatten(BuildNode* node, std::vector<RefNode>& out, int* offset, int depth, int& maxDepth) {
        if (depth > maxDepth) maxDepth = depth;
        const int my = (*offset)++;
        out[static_cast<size_t>(my)].bounds = node->bounds;
        if (node->count > 0) {
            out[static_cast<size_t>(my)].offset = node->first;
            out[static_cast<size_t>(my)].count = node->count;
        } else {
            out[static_cast<size_t>(my)].count = 0;
            flatten(node->child[0], out, offset, depth + 1, maxDepth);
            out[static_cast<size_t>(my)].offset = flatten(node->child[1], out, offset, depth + 1, maxDepth);
        }
        return my;
    }
};

inline float4 f4(float x, float y, float z, float w) {
    float4 r;
    r.x = x;
    r.y = y;
    r.z = z;
    r.w = w;
    return r;
}

// 4-wide collapse of the flattened binary BVH for the traversal kernels.  A wide node holds the
// children left after repeatedly replacing its largest-area interior child by that child's two
// children (at most four; leaves are never opened), in the binary tree's left-to-right order, so
// every box and leaf is one of the binary tree's.  Layout per node, 8 float4 (128 bytes, one L2
// line): lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of the four children (SoA, one child per lane),
// then the child references (interior: wide node index; leaf: ~(first << 8 | count-1)), then
// the child count.  Nodes are written depth-first, a node before its children.
static int collapseWide(const std::vector<RefNode>& ref, std::vector<float4>& out, int& maxDepth, int node = 0,
                        int depth = 1, int recBase = 0, std::vector<int4>* kidsOut = nullptr) {
    maxDepth = std::max(maxDepth, depth);
    int kids[4] = {node + 1, ref[static_cast<size_t>(node)].offset, -1, -1};
    int n = 2;
    while (n < 4) {
        int best = -1;
        float bestArea = -1.0f;
        for (int k = 0; k < n; ++k) {
            const RefNode& c = ref[static_cast<size_t>(kids[k])];
            if (c.count == 0 && c.bounds.surfaceArea() > bestArea) {
                best = k;
                bestArea = c.bounds.surfaceArea();
            }
        }
        if (best < 0) break;
        const int c = kids[best];
        for (int k = n; k > best + 1; --k) kids[k] = kids[k - 1];
        kids[best] = c + 1;
        kids[best + 1] = ref[static_cast<size_t>(c)].offset;
        ++n;
    }
    const size_t me = out.size() / 8;
    out.resize(out.size() + 8, float4{0.0f, 0.0f, 0.0f, 0.0f});
    if (kidsOut) {
        // the binary nodes a wide node's children are (for refitting its boxes in place)
        if (kidsOut->size() <= me) kidsOut->resize(me + 1, int4{-1, -1, -1, -1});
        (*kidsOut)[me] = int4{kids[0], kids[1], kids[2], kids[3]};
    }
    float lo[3][4], hi[3][4];
    int32_t child[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) {
        for (int a = 0; a < 3; ++a) {
            lo[a][k] = 0.0f;
            hi[a][k] = 0.0f;
        }
    }
    for (int k = 0; k < n; ++k) {
        const RefNode& c = ref[static_cast<size_t>(kids[k])];
        lo[0][k] = c.bounds.lo.x;
        lo[1][k] = c.bounds.lo.y;
        lo[2][k] = c.bounds.lo.z;
        hi[0][k] = c.bounds.hi.x;
        hi[1][k] = c.bounds.hi.y;
        hi[2][k] = c.bounds.hi.z;
        child[k] = c.count > 0 ? ~(((c.offset + recBase) << 8) | (c.count - 1))
                               : collapseWide(ref, out, maxDepth, kids[k], depth + 1, recBase, kidsOut);
    }
    float4* w = out.data() + me * 8;
    for (int a = 0; a < 3; ++a) {
        w[2 * a] = f4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
        w[2 * a + 1] = f4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
    }
    w[6] = f4(bitsf(static_cast<uint32_t>(child[0])), bitsf(static_cast<uint32_t>(child[1])),
              bitsf(static_cast<uint32_t>(child[2])), bitsf(static_cast<uint32_t>(child[3])));
    w[7] = f4(bitsf(static_cast<uint32_t>(n)), 0.0f, 0.0f, 0.0f);
    return static_cast<int>(me);
}

// The binary tree's interior nodes as 64-byte child-box nodes appended to B.nodes (leaf
// references offset by recBase); returns the root's reference (kNoRoot for a leaf too large).
static int32_t emitBinaryNodes(const std::vector<RefNode>& ref, int recBase, HostBuild& B) {
    const int base = static_cast<int>(B.nodes.size() / 4);
    std::vector<int> gpuIndex(ref.size(), -1);
    int nInterior = 0;
    for (size_t i = 0; i < ref.size(); ++i) {
        if (ref[i].count == 0) gpuIndex[i] = base + nInterior++;
        else ++B.leaves;
        if (ref[i].count > 256) {
            setError("BVH leaf with more than 256 triangles");
            return kNoRoot;
        }
    }
    auto childRef = [&](int c) -> int {
        const RefNode& n = ref[static_cast<size_t>(c)];
        if (n.count > 0) return ~(((n.offset + recBase) << 8) | (n.count - 1));
        return gpuIndex[static_cast<size_t>(c)];
    };
    B.nodes.resize(static_cast<size_t>(base + nInterior) * 4);
    for (size_t i = 0; i < ref.size(); ++i) {
        if (ref[i].count != 0) continue;
        const int c0 = static_cast<int>(i) + 1, c1 = ref[i].offset;
        const Box& b0 = ref[static_cast<size_t>(c0)].bounds;
        const Box& b1 = ref[static_cast<size_t>(c1)].bounds;
        const size_t k = static_cast<size_t>(gpuIndex[i]) * 4;
        B.nodes[k + 0] = f4(b0.lo.x, b0.hi.x, b0.lo.y, b0.hi.y);
        B.nodes[k + 1] = f4(b1.lo.x, b1.hi.x, b1.lo.y, b1.hi.y);
        B.nodes[k + 2] = f4(b0.lo.z, b0.hi.z, b1.lo.z, b1.hi.z);
        B.nodes[k + 3] = f4(bitsf(static_cast<uint32_t>(childRef(c0))), bitsf(static_cast<uint32_t>(childRef(c1))), 0.0f, 0.0f);
    }
    return ref[0].count > 0 ? childRef(0) : gpuIndex[0];
}

// ---------------------------------------------------------------------------------------------
// light BVH (light_sampler.cpp:24-148, light_bounds.cpp:73-109)
struct LBounds {
    Box bounds;
    V3 w{0.0f, 0.0f, 1.0f};
    float phi = 0.0f;
    float cosThetaO = 1.0f;
    float cosThetaE = 0.0f;
    bool twoSided = false;
};
float safeAcos(float x) { return std::acos(sclamp(x, -1.0f, 1.0f)); }
V3 rotateAround(V3 v, V3 axis, float theta) {
    const float c = std::cos(theta), s = std::sin(theta);
    return v * c + cross(axis, v) * s + axis * (dot(axis, v) * (1.0f - c));
}
LBounds unionBounds(const LBounds& a, const LBounds& b) {
    if (!(a.phi > 0.0f)) return b;
    if (!(b.phi > 0.0f)) return a;
    LBounds u;
    u.bounds = a.bounds.merged(b.bounds);
    u.phi = a.phi + b.phi;
    u.cosThetaE = smin(a.cosThetaE, b.cosThetaE);
    u.twoSided = a.twoSided || b.twoSided;
    const float thetaA = safeAcos(a.cosThetaO), thetaB = safeAcos(b.cosThetaO);
    const float thetaD = safeAcos(dot(a.w, b.w));
    if (smin(thetaD + thetaB, kPi) <= thetaA) {
        u.w = a.w;
        u.cosThetaO = a.cosThetaO;
        return u;
    }
    if (smin(thetaD + thetaA, kPi) <= thetaB) {
        u.w = b.w;
        u.cosThetaO = b.cosThetaO;
        return u;
    }
    const float thetaO = 0.5f * (thetaA + thetaD + thetaB);
    const V3 axis = cross(a.w, b.w);
    if (thetaO >= kPi || len2(axis) < 1e-12f) {
        u.w = a.w;
        u.cosThetaO = -1.0f;
        return u;
    }
    u.w = normalize(rotateAround(a.w, normalize(axis), thetaO - thetaA));
    u.cosThetaO = std::cos(thetaO);
    return u;
}
float groupCost(const LBounds& b, const Box& parent, int dim) {
    const float thetaO = std::acos(sclamp(b.cosThetaO, -1.0f, 1.0f));
    const float thetaE = std::acos(sclamp(b.cosThetaE, -1.0f, 1.0f));
    const float thetaW = smin(thetaO + thetaE, kPi);
    const float sinO = std::sqrt(smax(0.0f, 1.0f - b.cosThetaO * b.cosThetaO));
    const float mOmega = kTwoPi * (1.0f - b.cosThetaO) +
                         0.5f * kPi * (2.0f * thetaW * sinO - std::cos(thetaO - 2.0f * thetaW) - 2.0f * thetaO * sinO + b.cosThetaO);
    const V3 d = parent.diagonal();
    const float maxD = smax3(d.x, d.y, d.z);
    const float kr = get(d, dim) > 0.0f ? maxD / get(d, dim) : 1.0f;
    return b.phi * mOmega * kr * b.bounds.surfaceArea();
}
struct LItem {
    int index;
    LBounds lb;
};
struct LightBvhBuilder {
    std::vector<LightNodeGPU> nodes;
    std::vector<LBounds> nodeBounds;
    std::vector<unsigned long long>* trail;
    std::vector<uint8_t>* depthOut;
    int build(std::vector<LItem>& items, int begin, int end, unsigned long long tr, int depth) {
        const int idx = static_cast<int>(nodes.size());
        nodes.emplace_back();
        nodeBounds.emplace_back();
        std::memset(&nodes.back(), 0, sizeof(LightNodeGPU));
        nodes.back().child1 = -1;
        nodes.back().light = -1;
        if (end - begin == 1) {
            const LItem& it = items[static_cast<size_t>(begin)];
            nodeBounds[static_cast<size_t>(idx)] = it.lb;
            nodes[static_cast<size_t>(idx)].light = it.index;
            (*trail)[static_cast<size_t>(it.index)] = tr;
            (*depthOut)[static_cast<size_t>(it.index)] = static_cast<uint8_t>(depth);
            return idx;
        }
        Box bounds, centroids;
        for (int i = begin; i < end; ++i) {
            bounds.merge(items[static_cast<size_t>(i)].lb.bounds);
            centroids.merge(items[static_cast<size_t>(i)].lb.bounds.centroid());
        }
        constexpr int kB = 12;
        float bestCost = std::numeric_limits<float>::infinity();
        int bestDim = -1, bestBucket = -1;
        if (depth < 63 - 8) {
            for (int dim = 0; dim < 3; ++dim) {
                const float lo = get(centroids.lo, dim), hi = get(centroids.hi, dim);
                if (!(hi > lo)) continue;
                LBounds bucket[kB];
                for (int i = begin; i < end; ++i) {
                    const LBounds& lb = items[static_cast<size_t>(i)].lb;
                    int b = static_cast<int>(kB * (get(lb.bounds.centroid(), dim) - lo) / (hi - lo));
                    b = iclamp(b, 0, kB - 1);
                    bucket[b] = unionBounds(bucket[b], lb);
                }
                for (int split = 0; split < kB - 1; ++split) {
                    LBounds below, above;
                    for (int b = 0; b <= split; ++b) below = unionBounds(below, bucket[b]);
                    for (int b = split + 1; b < kB; ++b) above = unionBounds(above, bucket[b]);
                    if (!(below.phi > 0.0f) || !(above.phi > 0.0f)) continue;
                    const float cost = groupCost(below, bounds, dim) + groupCost(above, bounds, dim);
                    if (cost > 0.0f && cost < bestCost) {
                        bestCost = cost;
                        bestDim = dim;
                        bestBucket = split;
                    }
                }
            }
        }
        int mid = -1;
        if (bestDim >= 0) {
            const float lo = get(centroids.lo, bestDim), hi = get(centroids.hi, bestDim);
            auto it = std::partition(items.begin() + begin, items.begin() + end, [&](const LItem& item) {
                int b = static_cast<int>(kB * (get(item.lb.bounds.centroid(), bestDim) - lo) / (hi - lo));
                return iclamp(b, 0, kB - 1) <= bestBucket;
            });
            mid = static_cast<int>(it - items.begin());
        }
        if (mid <= begin || mid >= end) {
            mid = (begin + end) / 2;
            const int dim = centroids.maxExtent();
            std::nth_element(items.begin() + begin, items.begin() + mid, items.begin() + end,
                             [dim](const LItem& a, const LItem& b) {
                                 return get(a.lb.bounds.centroid(), dim) < get(b.lb.bounds.centroid(), dim);
                             });
        }
        const int c0 = build(items, begin, mid, tr, depth + 1);
        const int c1 = build(items, mid, end, tr | (1ull << depth), depth + 1);
        nodeBounds[static_cast<size_t>(idx)] = unionBounds(nodeBounds[static_cast<size_t>(c0)], nodeBounds[static_cast<size_t>(c1)]);
        nodes[static_cast<size_t>(idx)].child1 = c1;
        return idx;
    }
};

bool lightBounds(const LightGPU& l, LBounds& out) {
    const V3 rad = lightRadiance(l);
    if (!(l.area > 0.0f) || isBlack(rad)) return false;
    if (l.type == LT_TRIANGLE) {
        const V3 p0 = m3f(l.p0), p1 = m3f(l.p1), p2 = m3f(l.p2);
        out.bounds = Box(vmin(vmin(p0, p1), p2), vmax(vmax(p0, p1), p2));
    } else {
        const V3 p = m3f(l.p0), u = m3f(l.p1), v = m3f(l.p2);
        Box b;
        b.lo = p;
        b.hi = p;
        b.merge(p + u);
        b.merge(p + v);
        b.merge(p + u + v);
        out.bounds = b;
    }
    out.w = m3f(l.normal);
    out.phi = smax(0.0f, luminance(rad)) * l.area * kPi;
    out.cosThetaO = 1.0f;
    out.cosThetaE = 0.0f;
    out.twoSided = true;
    return true;
}

// ---------------------------------------------------------------------------------------------
// environment distributions (environment_light.cpp:82-163)
void buildCdf(const HostEnv& e, const std::vector<float>& func, std::vector<float>& marg, std::vector<float>& cond,
              float& funcInt, bool& valid) {
    const int w = e.width, h = e.height;
    marg.assign(static_cast<size_t>(h) + 1, 0.0f);
    cond.assign(static_cast<size_t>(h) * static_cast<size_t>(w + 1), 0.0f);
    for (int y = 0; y < h; ++y) {
        float* row = cond.data() + static_cast<size_t>(y) * static_cast<size_t>(w + 1);
        row[0] = 0.0f;
        for (int x = 0; x < w; ++x) row[x + 1] = row[x] + func[static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x)];
        marg[static_cast<size_t>(y) + 1] = marg[static_cast<size_t>(y)] + row[w];
    }
    funcInt = marg[static_cast<size_t>(h)];
    if (!(funcInt > 0.0f)) {
        funcInt = 0.0f;
        marg.clear();
        valid = false;
        return;
    }
    const float inv = 1.0f / funcInt;
    for (float& c : marg) c *= inv;
    for (int y = 0; y < h; ++y) {
        float* row = cond.data() + static_cast<size_t>(y) * static_cast<size_t>(w + 1);
        const float rowSum = row[w];
        if (rowSum <= 0.0f) continue;
        const float invRow = 1.0f / rowSum;
        for (int x = 0; x <= w; ++x) row[x] *= invRow;
    }
    valid = true;
}

V3 envPixelHost(const HostEnv& e, int x, int y) {
    const float* p = e.image.data() + 3 * (static_cast<size_t>(y) * static_cast<size_t>(e.width) + static_cast<size_t>(x));
    return mk(p[0], p[1], p[2]);
}

void buildEnvironment(HostEnv& e) {
    e.fullValid = e.misValid = false;
    e.fullFunc.clear();
    e.misFunc.clear();
    e.fullMarg.clear();
    e.misMarg.clear();
    e.fullCond.clear();
    e.misCond.clear();
    e.fullInt = e.misInt = 0.0f;
    if (e.hasImage && e.width > 0 && e.height > 0) {
        const int w = e.width, h = e.height;
        e.fullFunc.assign(static_cast<size_t>(w) * static_cast<size_t>(h), 0.0f);
        std::vector<float> sinRow(static_cast<size_t>(h));
        double weighted = 0.0, weights = 0.0;
        for (int y = 0; y < h; ++y) {
            const float sinTheta = std::sin(kPi * (static_cast<float>(y) + 0.5f) / static_cast<float>(h));
            sinRow[static_cast<size_t>(y)] = sinTheta;
            for (int x = 0; x < w; ++x) {
                float L = luminance(envPixelHost(e, x, y));
                if (!(L > 0.0f)) L = 0.0f;
                e.fullFunc[static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x)] = L * sinTheta;
                weighted += static_cast<double>(L) * sinTheta;
                weights += sinTheta;
            }
        }
        buildCdf(e, e.fullFunc, e.fullMarg, e.fullCond, e.fullInt, e.fullValid);
        if (e.fullValid) {
            const float meanL = weights > 0.0 ? static_cast<float>(weighted / weights) : 0.0f;
            e.misFunc.resize(e.fullFunc.size());
            double misTotal = 0.0, fullTotal = 0.0;
            for (int y = 0; y < h; ++y) {
                const float s = sinRow[static_cast<size_t>(y)];
                for (int x = 0; x < w; ++x) {
                    const size_t i = static_cast<size_t>(y) * static_cast<size_t>(w) + static_cast<size_t>(x);
                    float L = luminance(envPixelHost(e, x, y));
                    if (!(L > 0.0f)) L = 0.0f;
                    const float excess = L - meanL;
                    e.misFunc[i] = excess > 1e-4f * meanL ? excess * s : 0.0f;
                    misTotal += e.misFunc[i];
                    fullTotal += e.fullFunc[i];
                }
            }
            bool comp = misTotal > 1e-3 * fullTotal;
            if (comp) buildCdf(e, e.misFunc, e.misMarg, e.misCond, e.misInt, e.misValid);
            comp = comp && e.misValid;
            if (!comp) {
                e.misFunc = e.fullFunc;
                e.misMarg = e.fullMarg;
                e.misCond = e.fullCond;
                e.misInt = e.fullInt;
                e.misValid = e.fullValid;
            }
        }
    }
    // power() (environment_light.cpp:305-322) and the mean luminance of the constructor.
    V3 pw;
    if (!e.hasImage || e.width <= 0) {
        pw = mk(0.5f) * e.intensity * 4.0f * kPi;
    } else {
        V3 sum = mk(0.0f);
        float wsum = 0.0f;
        for (int y = 0; y < e.height; y += 4) {
            const float s = std::sin(kPi * (static_cast<float>(y) + 0.5f) / static_cast<float>(e.height));
            for (int x = 0; x < e.width; x += 4) {
                sum += envPixelHost(e, x, y) * s;
                wsum += s;
            }
        }
        pw = (wsum > 0.0f ? sum / wsum : sum) * e.intensity * 4.0f * kPi;
    }
    e.meanLuminance = smax(0.0f, luminance(pw) / (4.0f * kPi));
    // setSun (environment_light.cpp:211-227)
    e.sunPdfWeight = 0.0f;
    if (e.hasSun) {
        e.sunDir = normalize(e.sunDirIn);
        e.sunCosMax = sclamp(e.sunCosIn, -0.999f, 0.9999999f);
        e.sunRadiance = e.sunRadIn * e.intensity;
        const float omega = kTwoPi * (1.0f - e.sunCosMax);
        const float sunPower = smax(0.0f, luminance(e.sunRadiance)) * omega;
        const float skyPower = 4.0f * kPi * e.meanLuminance;
        if (sunPower > 0.0f) {
            e.sunPdfWeight = sclamp(sunPower / (sunPower + skyPower), 0.15f, 0.85f);
            if (!e.fullValid) e.sunPdfWeight = 1.0f;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Material parameters with the reference setters' clamps.
MatGPU resolveMaterial(const pe_material& m) {
    MatGPU g;
    std::memset(&g, 0, sizeof(g));
    g.type = m.type;
    auto c3 = [](float* dst, const float* src) { dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2]; };
    auto cc3 = [](float* dst, const float* src, float lo, float hi) {
        for (int i = 0; i < 3; ++i) dst[i] = smax(lo, smin(src[i], hi));
    };
    c3(g.base, m.base_color);
    c3(g.emission, m.emission);
    g.roundEdge = m.round_edge_radius > 0.0f ? m.round_edge_radius : 0.0f; // setRoundEdgeRadius
    // image maps: Disney only (the other materials have none)
    const bool disney = m.type == PE_MAT_DISNEY;
    g.texAlbedo = disney ? m.albedo_texture : -1;
    g.texRoughness = disney ? m.roughness_texture : -1;
    g.texMetalness = disney ? m.metalness_texture : -1;
    g.texNormal = disney ? m.normal_texture : -1;
    g.texOpacity = disney ? m.opacity_texture : -1;
    g.texMapping = m.texture_mapping == 1 ? 1 : 0;
    g.texScale = m.texture_scale > 1e-4f ? m.texture_scale : 1e-4f; // setTextureScale
    if (m.type == PE_MAT_DISNEY) {
        g.metallic = m.metallic;
        g.roughness = smax(0.001f, m.roughness);
        g.specular = m.specular;
        g.clearcoat = sclamp(m.clearcoat, 0.0f, 1.0f);
        g.clearcoatRoughness = smax(0.001f, m.clearcoat_roughness);
        g.ior = sclamp(m.ior, 1.0001f, 3.0f);
        g.specTrans = sclamp(m.spec_transmission, 0.0f, 1.0f);
        g.coatIor = sclamp(m.coat_ior, 1.0001f, 3.0f);
        cc3(g.coatTint, m.coat_tint, 0.0f, 1.0f);
        if (m.has_sheen_color) {
            cc3(g.sheenColor, m.sheen_color, 0.0f, 1.0f);
            g.hasSheenColor = 1;
        } else {
            g.sheenColor[0] = g.sheenColor[1] = g.sheenColor[2] = 1.0f;
        }
        g.anisotropy = sclamp(m.anisotropy, 0.0f, 1.0f);
        g.sheen = sclamp(m.sheen, 0.0f, 1.0f);
        g.sheenRoughness = sclamp(m.sheen_roughness, 0.02f, 1.0f);
        g.diffuseRoughness = sclamp(m.diffuse_roughness, 0.0f, 1.0f);
        g.diffuseTransmission = sclamp(m.diffuse_transmission, 0.0f, 1.0f);
        g.subsurface = sclamp(m.subsurface, 0.0f, 1.0f);
        cc3(g.ssRadius, m.subsurface_radius, 1e-4f, 1e4f);
        g.ssScale = smax(m.subsurface_scale, 1e-6f);
        g.ssAniso = sclamp(m.subsurface_anisotropy, -0.9f, 0.9f);
        cc3(g.edgeTint, m.edge_tint, 0.0f, 1.0f);
        g.thinFilmThickness = sclamp(m.thin_film_thickness, 0.0f, 2000.0f);
        g.thinFilmIor = sclamp(m.thin_film_ior, 1.0f, 3.0f);
        if (m.flake_density > 0.0f) {
            g.flakeDensity = sclamp(m.flake_density, 0.0f, 1.0f);
            g.flakeSize = smax(m.flake_size, 1e-6f);
            g.flakeRoughness = sclamp(m.flake_roughness, 0.0f, 1.0f);
            cc3(g.flakeColor, m.flake_color, 0.0f, 1.0f);
        } else {
            g.flakeDensity = 0.0f;
            g.flakeSize = 0.004f;
            g.flakeRoughness = 0.3f;
            g.flakeColor[0] = g.flakeColor[1] = g.flakeColor[2] = 0.9f;
        }
        g.opacity = sclamp(m.opacity, 0.0f, 1.0f);
        if (g.specTrans > 0.0f) g.flags |= MF_VOLUME_BOUNDARY;
        if (g.opacity < 1.0f || m.opacity_texture >= 0) g.flags |= MF_TRANSMITS_SHADOWS; // disney.h:158
    } else if (m.type == PE_MAT_DIELECTRIC) {
        g.ior = m.ior;
        g.glassRoughness = m.glass_roughness;
        g.abbe = m.abbe > 0.0f ? smax(m.abbe, 10.0f) : 0.0f;
        g.thinWalled = m.thin_walled ? 1 : 0;
        g.filmThickness = m.film_thickness > 0.0f ? m.film_thickness : 0.0f;
        // rebuildMedium (dielectric.cpp:140-148), evaluated only when a setter called it.
        if (m.has_absorption || m.has_scattering) {
            float absorb[3] = {1.0f, 1.0f, 1.0f};
            float absorbDist = 1.0f;
            float density = 0.0f;
            float scol[3] = {1.0f, 1.0f, 1.0f};
            float aniso = 0.0f;
            if (m.has_absorption) {
                cc3(absorb, m.absorb_color, 0.0f, 1.0f);
                absorbDist = smax(m.absorb_distance, 1e-5f);
            }
            if (m.has_scattering) {
                density = smax(m.scatter_density, 0.0f);
                cc3(scol, m.scatter_color, 0.0f, 1.0f);
                aniso = sclamp(m.scatter_anisotropy, -0.95f, 0.95f);
            }
            for (int c = 0; c < 3; ++c) {
                g.sigmaA[c] = -std::log(smax(absorb[c], 1e-4f)) / absorbDist;
                g.sigmaS[c] = scol[c] * density;
                g.sigmaA[c] += (1.0f - scol[c]) * density;
            }
            g.mediumG = aniso;
        }
        if (g.thinWalled || g.glassRoughness <= 1e-3f) g.flags |= MF_DELTA;
        if (!g.thinWalled) g.flags |= MF_VOLUME_BOUNDARY;
        if (g.thinWalled) g.flags |= MF_TRANSMITS_SHADOWS;
        if (g.abbe > 0.0f) g.flags |= MF_DISPERSIVE;
        const bool emptyMedium = isBlack(m3f(g.sigmaA)) && isBlack(m3f(g.sigmaS));
        if (!g.thinWalled && !emptyMedium) g.flags |= MF_HAS_MEDIUM;
        if (!isBlack(m3f(g.sigmaS))) g.flags |= MF_MEDIUM_SCATTERS;
    } else if (m.type == PE_MAT_MIRROR) {
        g.flags |= MF_DELTA;
    }
    if ((m.type == PE_MAT_LAMBERT || m.type == PE_MAT_DISNEY) && !isBlack(m3f(g.emission))) g.flags |= MF_EMISSIVE;
    if (!(m.type == PE_MAT_LAMBERT || m.type == PE_MAT_DISNEY)) g.emission[0] = g.emission[1] = g.emission[2] = 0.0f;
    return g;
}

// ---------------------------------------------------------------------------------------------
// GGX / sheen energy tables (microfacet.cpp:36-133), Sobol byte tables, spectral tables.
float nodeMu(int im) { return smax(static_cast<float>(im) / (kTableN - 1), 1e-3f); }

void buildGgxTables(TablesGPU& T) {
    constexpr int kS = 24;
    for (int ia = 0; ia < kTableN; ++ia) {
        const float alpha = static_cast<float>(ia) / (kTableN - 1);
        for (int im = 0; im < kTableN; ++im) {
            const float mu = nodeMu(im);
            const V3 wo = mk(std::sqrt(smax(0.0f, 1.0f - mu * mu)), 0.0f, mu);
            const float g1 = ggxG1(wo, alpha, alpha);
            double sum = 0.0, sumA = 0.0, sumB = 0.0;
            for (int sy = 0; sy < kS; ++sy)
                for (int sx = 0; sx < kS; ++sx) {
                    const float u1 = (static_cast<float>(sx) + 0.5f) / kS;
                    const float u2 = (static_cast<float>(sy) + 0.5f) / kS;
                    const V3 h = ggxSampleVisibleNormal(wo, alpha, alpha, u1, u2);
                    const float c = dot(wo, h);
                    const V3 wi = h * (2.0f * c) - wo;
                    if (wi.z <= 0.0f) continue;
                    const double w = ggxG(wo, wi, alpha, alpha) / g1;
                    const double s5 = pow5(1.0f - sclamp(c, 0.0f, 1.0f));
                    sum += w;
                    sumA += w * (1.0 - s5);
                    sumB += w * s5;
                }
            const int k = ia * kTableN + im;
            T.ggxE[k] = static_cast<float>(sum / (kS * kS));
            T.ggxEa[k] = static_cast<float>(sumA / (kS * kS));
            T.ggxEb[k] = static_cast<float>(sumB / (kS * kS));
        }
    }
    constexpr int kM = 256;
    for (int ia = 0; ia < kTableN; ++ia) {
        const float alpha = static_cast<float>(ia) / (kTableN - 1);
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int i = 0; i < kM; ++i) {
            const float mu = (static_cast<float>(i) + 0.5f) / kM;
            const float E = sclamp(tableLookup2D(T.ggxE, mu, alpha), 1e-3f, 1.0f);
            const float m = 1.0f / E - 1.0f;
            const float A = tableLookup2D(T.ggxEa, mu, alpha), B = tableLookup2D(T.ggxEb, mu, alpha);
            const double w = 2.0 * mu / kM;
            a0 += w * B;
            a1 += w * (A + B * m);
            a2 += w * (A * m);
        }
        T.avg0[ia] = static_cast<float>(a0);
        T.avg1[ia] = static_cast<float>(a1);
        T.avg2[ia] = static_cast<float>(a2);
    }
    constexpr int kC = 96, kP = 48;
    for (int ir = 0; ir < kTableN; ++ir) {
        const float r = smax(static_cast<float>(ir) / (kTableN - 1), 0.02f);
        for (int im = 0; im < kTableN; ++im) {
            const float mu = nodeMu(im);
            const V3 wo = mk(std::sqrt(smax(0.0f, 1.0f - mu * mu)), 0.0f, mu);
            double sum = 0.0;
            for (int i = 0; i < kC; ++i) {
                const float cz = (static_cast<float>(i) + 0.5f) / kC;
                const float s = std::sqrt(smax(0.0f, 1.0f - cz * cz));
                for (int j = 0; j < kP; ++j) {
                    const float phi = kPi * (static_cast<float>(j) + 0.5f) / kP;
                    const V3 wi = mk(s * std::cos(phi), s * std::sin(phi), cz);
                    const V3 h = normalize(wo + wi);
                    sum += charlieD(h.z, r) * charlieV(cz, mu) * cz;
                }
            }
            T.sheenE[ir * kTableN + im] = static_cast<float>(sum * (1.0 / kC) * (kTwoPi / kP));
        }
    }
}

// Wavelength tables of sampleWavelength (spectral.cpp:33-62).
void buildSpectral(TablesGPU& T) {
    const float lmin = 380.0f, lmax = 730.0f;
    constexpr int kBins = 350;
    V3 sum = mk(0.0f);
    constexpr int kSteps = 3500;
    const float dl = (lmax - lmin) / static_cast<float>(kSteps);
    for (int i = 0; i < kSteps; ++i) sum += spectralRaw(lmin + (static_cast<float>(i) + 0.5f) * dl);
    const V3 mean = sum / static_cast<float>(kSteps);
    const V3 norm = mk(1.0f / mean.x, 1.0f / mean.y, 1.0f / mean.z);
    const float bw = (lmax - lmin) / static_cast<float>(kBins);
    float acc = 0.0f;
    T.spectralCdf[0] = 0.0f;
    float s[kBins];
    for (int i = 0; i < kBins; ++i) {
        const V3 c = spectralRaw(lmin + (static_cast<float>(i) + 0.5f) * bw) * norm;
        s[i] = c.x + c.y + c.z + 0.02f;
        acc += s[i];
        T.spectralCdf[i + 1] = acc;
    }
    for (int i = 0; i <= kBins; ++i) T.spectralCdf[i] /= acc;
    for (int i = 0; i < kBins; ++i) T.spectralPdf[i] = s[i] / (acc * bw);
    T.spectralNorm[0] = norm.x;
    T.spectralNorm[1] = norm.y;
    T.spectralNorm[2] = norm.z;
}

// The data passes' colour of an id (idColor, renderer.cpp:252-271): 0 is black; otherwise the
// splitmix64 finaliser of id + 0x9e3779b97f4a7c15 gives a hue, stepped by the golden-ratio
// conjugate, shown at saturation 0.75 and value 1.
V3 idColorOf(uint64_t id) {
    if (id == 0) return mk(0.0f);
    uint64_t z = id + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    const float hue = std::fmod(static_cast<float>(z >> 40) * 0x1p-24f + 0.618034f, 1.0f) * 6.0f;
    const float frac = hue - std::floor(hue);
    const float lo = 1.0f * (1.0f - 0.75f);
    const float falling = 1.0f * (1.0f - 0.75f * frac);
    const float rising = 1.0f * (1.0f - 0.75f * (1.0f - frac));
    switch (static_cast<int>(hue) % 6) {
        case 0: return mk(1.0f, rising, lo);
        case 1: return mk(falling, 1.0f, lo);
        case 2: return mk(lo, 1.0f, rising);
        case 3: return mk(lo, falling, 1.0f);
        case 4: return mk(rising, lo, 1.0f);
        default: return mk(1.0f, lo, falling);
    }
}

// MurmurHash3_x86_32 (Austin Appleby's public-domain hash, seed 0): the Cryptomatte 1.2 name
// hash (cryptomatte.cpp:36-78).
uint32_t murmur3(const std::string& key) {
    auto rotl = [](uint32_t x, int r) { return (x << r) | (x >> (32 - r)); };
    const size_t len = key.size();
    const auto* bytes = reinterpret_cast<const uint8_t*>(key.data());
    uint32_t h = 0u;
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    size_t i = 0;
    for (; i + 4 <= len; i += 4) {
        uint32_t k = static_cast<uint32_t>(bytes[i]) | (static_cast<uint32_t>(bytes[i + 1]) << 8) |
                     (static_cast<uint32_t>(bytes[i + 2]) << 16) | (static_cast<uint32_t>(bytes[i + 3]) << 24);
        k = rotl(k * c1, 15) * c2;
        h = rotl(h ^ k, 13) * 5u + 0xe6546b64u;
    }
    uint32_t k = 0u;
    for (size_t j = len - i; j > 0; --j) k = (k << 8) | bytes[i + j - 1];
    if (len - i > 0) h ^= rotl(k * c1, 15) * c2;
    h ^= static_cast<uint32_t>(len);
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// The hash as a float id (cryptoHashToFloat, cryptomatte.cpp:82-92): exponents 0 and 255 have
// their lowest bit flipped, so the id is a finite, normal float.
float cryptoId(const std::string& name) {
    if (name.empty()) return 0.0f;
    uint32_t h = murmur3(name);
    const uint32_t e = (h >> 23) & 0xFFu;
    if (e == 0u || e == 0xFFu) h = (h & 0x807FFFFFu) | ((e ^ 1u) << 23);
    float f;
    std::memcpy(&f, &h, sizeof(f));
    return f;
}

} // namespace

const TablesGPU& staticTables() {
    static const TablesGPU* t = [] {
        auto* T = new TablesGPU();
        std::memset(T, 0, sizeof(TablesGPU));
        buildGgxTables(*T);
        for (int k = 0; k < 4; ++k)
            for (uint32_t b = 0; b < 256; ++b) T->sobolTab[k][b] = sobolTableEntry(k, b);
        buildSpectral(*T);
        return T;
    }();
    return *t;
}

// PixelFilterSampler (pixel_filter.cpp:39-91): inverse CDF of the separable filter.
void fillFilterCdf(int type, float width, float* cdf) {
    width = sclamp(width, 0.25f, 8.0f);
    const float radius = 0.5f * width;
    for (int i = 0; i <= kFilterBins; ++i) cdf[i] = 0.0f;
    if (type == PE_FILTER_BOX) {
        cdf[0] = -1.0f; // marker: box
        return;
    }
    auto evaluate = [&](float x) -> float {
        if (std::fabs(x) > radius) return 0.0f;
        switch (type) {
            case PE_FILTER_TRIANGLE: return smax(0.0f, 1.0f - std::fabs(x) / radius);
            case PE_FILTER_GAUSSIAN: {
                const float s = width / 6.0f;
                const float k = 1.0f / (2.0f * s * s);
                return smax(0.0f, std::exp(-k * x * x) - std::exp(-k * radius * radius));
            }
            default: {
                const float a = kTwoPi * (x / width + 0.5f);
                return 0.35875f - 0.48829f * std::cos(a) + 0.14128f * std::cos(2.0f * a) - 0.01168f * std::cos(3.0f * a);
            }
        }
    };
    const float dx = width / kFilterBins;
    double acc = 0.0;
    for (int i = 0; i < kFilterBins; ++i) {
        acc += smax(0.0f, evaluate(-radius + (static_cast<float>(i) + 0.5f) * dx));
        cdf[i + 1] = static_cast<float>(acc);
    }
    if (!(acc > 0.0)) {
        cdf[0] = -1.0f;
        return;
    }
    for (int i = 0; i <= kFilterBins; ++i) cdf[i] = static_cast<float>(cdf[i] / acc);
    cdf[kFilterBins] = 1.0f;
}

// ---------------------------------------------------------------------------------------------
// The lights and the light sampler of a scene (LightSampler::build, light_sampler.cpp:42-115):
// exhaustive up to kMaxExhaustive candidates, else infinite lights on top of a light BVH.
static void buildLightSampler(const pe_scene* s, HostBuild& B) {
    B.infinite.clear();
    B.lightNodes.clear();
    B.lights = s->lights;
    const int nl = static_cast<int>(B.lights.size());
    const int count = nl + (s->env.present ? 1 : 0);
    B.lightCount = count;
    B.topSlot.assign(static_cast<size_t>(count), -1);
    B.trail.assign(static_cast<size_t>(count), 0ull);
    B.trailDepth.assign(static_cast<size_t>(count), 0);
    B.lightMode = count <= 1 ? 0 : 1;
    if (count > kMaxExhaustive) {
        std::vector<LItem> items;
        for (int i = 0; i < nl; ++i) {
            LBounds lb;
            if (lightBounds(B.lights[static_cast<size_t>(i)], lb) && lb.phi > 0.0f) items.push_back({i, lb});
            else B.infinite.push_back(i);
        }
        if (s->env.present) B.infinite.push_back(nl);
        if (static_cast<int>(B.infinite.size()) + 1 > kMaxInfinite) {
            B.infinite.clear();
            B.lightMode = 0; // uniform (light_sampler.cpp:71-75)
        } else {
            for (size_t k = 0; k < B.infinite.size(); ++k) B.topSlot[static_cast<size_t>(B.infinite[k])] = static_cast<int16_t>(k);
            if (!items.empty()) {
                LightBvhBuilder lb;
                lb.trail = &B.trail;
                lb.depthOut = &B.trailDepth;
                lb.nodes.reserve(2 * items.size());
                lb.build(items, 0, static_cast<int>(items.size()), 0ull, 0);
                B.lightNodes = lb.nodes;
                for (size_t i = 0; i < lb.nodes.size(); ++i) {
                    const LBounds& b = lb.nodeBounds[i];
                    LightNodeGPU& n = B.lightNodes[i];
                    n.bmin[0] = b.bounds.lo.x; n.bmin[1] = b.bounds.lo.y; n.bmin[2] = b.bounds.lo.z;
                    n.bmax[0] = b.bounds.hi.x; n.bmax[1] = b.bounds.hi.y; n.bmax[2] = b.bounds.hi.z;
                    n.w[0] = b.w.x; n.w[1] = b.w.y; n.w[2] = b.w.z;
                    n.phi = b.phi;
                    n.cosThetaO = b.cosThetaO;
                    n.cosThetaE = b.cosThetaE;
                    n.twoSided = b.twoSided ? 1 : 0;
                }
            }
            B.lightMode = 2;
        }
    }
}

static int32_t buildScene(pe_scene* s) {
    HostBuild& B = s->build;
    B = HostBuild{};
    B.materials = s->materials;
    B.catcherShape = s->catcherShape >= 0 && s->catcherShape < static_cast<int32_t>(s->shapes.size()) ? s->catcherShape : -1;
    if (B.materials.size() >= 0xFFFFu) {
        setError("scene has " + std::to_string(B.materials.size()) + " materials; at most 65534 are supported");
        return PE_ERR_LIMIT;
    }
    // Exit vertex of a random-walk subsurface path: a white Lambert surface whose normal faces
    // out of the object (path_tracer.cpp:56-59, 757-761); appended after the scene's materials.
    {
        pe_material wl;
        pe_material_defaults(PE_MAT_LAMBERT, &wl);
        wl.base_color[0] = wl.base_color[1] = wl.base_color[2] = 1.0f;
        B.exitMaterial = static_cast<int32_t>(B.materials.size());
        B.materials.push_back(resolveMaterial(wl));
    }
    // shapes and global triangle / vertex numbering
    uint32_t nTris = 0, nVerts = 0;
    for (const HostShape& sh : s->shapes) {
        nTris += (sh.sphere || sh.blas >= 0) ? 1u : static_cast<uint32_t>(sh.idx.size() / 3);
        nVerts += static_cast<uint32_t>(sh.pos.size());
    }
    const uint32_t nTlas = nTris;
    // BLAS triangles and vertices follow the top level's
    std::vector<uint32_t> blasFirstTri(s->blases.size()), blasFirstVert(s->blases.size());
    for (size_t b = 0; b < s->blases.size(); ++b) {
        blasFirstTri[b] = nTris;
        blasFirstVert[b] = nVerts;
        nTris += static_cast<uint32_t>(s->blases[b].idx.size() / 3);
        nVerts += static_cast<uint32_t>(s->blases[b].pos.size());
    }
    if (nTris >= (1u << 23)) {
        setError("scene has " + std::to_string(nTris) + " triangles; the flattened BVH encodes at most 8388607");
        return PE_ERR_LIMIT;
    }
    B.triVerts.resize(nTris);
    B.pos.resize(nVerts);
    B.nrm.resize(nVerts);
    B.uv.resize(nVerts);
    B.shapes.resize(s->shapes.size());
    // light links: number the node uids that links name (Scene::buildAccelerator, scene.cpp:121-141)
    std::vector<uint64_t> linkUids;
    auto linkIndex = [&](uint64_t uid) -> int {
        for (size_t k = 0; k < linkUids.size(); ++k)
            if (linkUids[k] == uid) return static_cast<int>(k);
        return -1;
    };
    B.links.clear();
    if (!s->lightLinks.empty()) {
        B.links.assign(s->lights.size(), LightLinkGPU{0ull, 0ull, 0, 0});
        for (size_t li = 0; li < s->lightLinks.size() && li < s->lights.size(); ++li) {
            const HostLightLink& hl = s->lightLinks[li];
            LightLinkGPU& g = B.links[li];
            g.mode = hl.mode;
            g.shadowMode = hl.shadowMode;
            auto addAll = [&](const std::vector<uint64_t>& uids, unsigned long long& mask) -> bool {
                for (uint64_t u : uids) {
                    int k = linkIndex(u);
                    if (k < 0) {
                        if (linkUids.size() >= static_cast<size_t>(kLinkNodeOther)) return false;
                        k = static_cast<int>(linkUids.size());
                        linkUids.push_back(u);
                    }
                    mask |= 1ull << k;
                }
                return true;
            };
            if ((hl.mode != 0 && !addAll(hl.uids, g.mask)) || (hl.shadowMode != 0 && !addAll(hl.shadowUids, g.shadowMask))) {
                setError("light links name more than 63 distinct node uids");
                return PE_ERR_LIMIT;
            }
            if (hl.mode != 0) B.hasLightLinks = 1;
            if (hl.shadowMode != 0) B.hasShadowLinks = 1;
        }
        if (!B.hasLightLinks && !B.hasShadowLinks) B.links.clear();
    }
    std::vector<Box> triBounds(nTris);
    std::vector<uint8_t> triMask(nTris);
    uint32_t t0 = 0, v0 = 0;
    for (size_t si = 0; si < s->shapes.size(); ++si) {
        const HostShape& sh = s->shapes[si];
        ShapeInfo& info = B.shapes[si];
        info.material = sh.material;
        info.emitter = sh.emitter;
        info.flags = sh.flags;
        info.firstTri = t0;
        {
            const uint64_t uid = si < s->shapeUid.size() ? s->shapeUid[si] : 0ull;
            const int k = linkIndex(uid);
            info.linkNode = k >= 0 ? k : kLinkNodeOther;
        }
        for (size_t v = 0; v < sh.pos.size(); ++v) {
            B.pos[v0 + v] = f4(sh.pos[v].x, sh.pos[v].y, sh.pos[v].z, 0.0f);
            const V3 n = v < sh.nrm.size() ? sh.nrm[v] : mk(0.0f);
            B.nrm[v0 + v] = f4(n.x, n.y, n.z, 0.0f);
            float2 uv;
            uv.x = v < sh.uv.size() ? sh.uv[v].x : 0.0f;
            uv.y = v < sh.uv.size() ? sh.uv[v].y : 0.0f;
            B.uv[v0 + v] = uv;
        }
        if (sh.blas >= 0) {
            // one top-level primitive; its bounds are the BLAS's box under the transform
            // (Transform::transformAABB, Arvo's method, transform.cpp:83-110)
            B.triVerts[t0] = int4{-2, sh.blas, 0, static_cast<int>(si)};
            const HostBlas& hb = s->blases[static_cast<size_t>(sh.blas)];
            Box lb;
            for (const V3& p : hb.pos) lb = lb.merged(Box{p, p});
            triBounds[t0] = instanceBox(sh, lb);
            triMask[t0] = sh.mask;
            info.firstTri = blasFirstTri[static_cast<size_t>(sh.blas)];
            t0 += 1;
            const MatGPU& mi = s->materials[static_cast<size_t>(sh.material)];
            if (mi.flags & MF_TRANSMITS_SHADOWS) B.hasShadowTransmitters = true;
            continue;
        }
        if (sh.sphere) {
            // one primitive, no vertices: its triVerts entry carries only the shape
            B.triVerts[t0] = int4{-1, -1, -1, static_cast<int>(si)};
            Box b;
            b.lo = sh.center - mk(sh.radius);
            b.hi = sh.center + mk(sh.radius);
            triBounds[t0] = b;
            triMask[t0] = sh.mask;
            t0 += 1;
            const MatGPU& ms = s->materials[static_cast<size_t>(sh.material)];
            if (ms.flags & MF_TRANSMITS_SHADOWS) B.hasShadowTransmitters = true;
            continue;
        }
        const size_t nt = sh.idx.size() / 3;
        for (size_t t = 0; t < nt; ++t) {
            int4 tv;
            tv.x = static_cast<int>(v0 + sh.idx[3 * t + 0]);
            tv.y = static_cast<int>(v0 + sh.idx[3 * t + 1]);
            tv.z = static_cast<int>(v0 + sh.idx[3 * t + 2]);
            tv.w = static_cast<int>(si);
            B.triVerts[t0 + t] = tv;
            const V3 p0 = sh.pos[sh.idx[3 * t]], p1 = sh.pos[sh.idx[3 * t + 1]], p2 = sh.pos[sh.idx[3 * t + 2]];
            Box b;
            b.lo = vmin(vmin(p0, p1), p2);
            b.hi = vmax(vmax(p0, p1), p2);
            triBounds[t0 + t] = b;
            triMask[t0 + t] = sh.mask;
        }
        t0 += static_cast<uint32_t>(nt);
        v0 += static_cast<uint32_t>(sh.pos.size());
        const MatGPU& mg = s->materials[static_cast<size_t>(sh.material)];
        if (mg.flags & MF_TRANSMITS_SHADOWS) B.hasShadowTransmitters = true;
    }
    for (size_t b = 0; b < s->blases.size(); ++b) {
        const HostBlas& hb = s->blases[b];
        const uint32_t vb = blasFirstVert[b], tb = blasFirstTri[b];
        for (size_t v = 0; v < hb.pos.size(); ++v) {
            B.pos[vb + v] = f4(hb.pos[v].x, hb.pos[v].y, hb.pos[v].z, 0.0f);
            const V3 n = v < hb.nrm.size() ? hb.nrm[v] : mk(0.0f);
            B.nrm[vb + v] = f4(n.x, n.y, n.z, 0.0f);
            float2 uv;
            uv.x = v < hb.uv.size() ? hb.uv[v].x : 0.0f;
            uv.y = v < hb.uv.size() ? hb.uv[v].y : 0.0f;
            B.uv[vb + v] = uv;
        }
        for (size_t t = 0; t < hb.idx.size() / 3; ++t)
            B.triVerts[tb + t] = int4{static_cast<int>(vb + hb.idx[3 * t]), static_cast<int>(vb + hb.idx[3 * t + 1]),
                                      static_cast<int>(vb + hb.idx[3 * t + 2]), -1};
    }
    for (const MatGPU& m : s->materials)
        if (m.flags & MF_TRANSMITS_SHADOWS) B.hasShadowTransmitters = true; // Scene::retainMaterial
    for (const MatGPU& m : s->materials) {
        if (m.flags & (MF_VOLUME_BOUNDARY)) B.hasVolumes = true;
        if (m.type == PE_MAT_DISNEY && m.subsurface > 0.0f) B.hasSubsurface = true;
        if (m.flags & MF_DISPERSIVE) B.hasDispersion = true;
    }

    // SAH BVH
    B.tlasPrims = nTlas;
    B.instances.clear();
    B.motions.clear();
    std::vector<int> instOfShape(s->shapes.size(), -1);
    for (size_t si = 0; si < s->shapes.size(); ++si)
        if (s->shapes[si].blas >= 0) {
            if (static_cast<int32_t>(B.instances.size()) >= kMaxInstances) {
                setError("scene has more than " + std::to_string(kMaxInstances) + " mesh instances");
                return PE_ERR_LIMIT;
            }
            instOfShape[si] = static_cast<int>(B.instances.size());
            B.instances.emplace_back();
        }
    // the BVH leaf record of a triangle (lean Möller–Trumbore data), in local or world space
    auto triRecord = [&](size_t i, uint32_t g, uint32_t meta) {
        const int4 tv = B.triVerts[g];
        const V3 p0 = mk(B.pos[tv.x].x, B.pos[tv.x].y, B.pos[tv.x].z);
        const V3 p1 = mk(B.pos[tv.y].x, B.pos[tv.y].y, B.pos[tv.y].z);
        const V3 p2 = mk(B.pos[tv.z].x, B.pos[tv.z].y, B.pos[tv.z].z);
        const V3 e1 = p1 - p0, e2 = p2 - p0;
        const float eps = 1e-14f * len2(e1) * len2(e2);
        B.tris[3 * i + 0] = f4(p0.x, p0.y, p0.z, eps);
        B.tris[3 * i + 1] = f4(e1.x, e1.y, e1.z, bitsf(meta));
        B.tris[3 * i + 2] = f4(e2.x, e2.y, e2.z, bitsf(g));
    };
    if (nTlas > 0) {
        SahBuilder sb;
        sb.prims.reserve(nTlas);
        for (uint32_t i = 0; i < nTlas; ++i) sb.prims.emplace_back(i, triBounds[i]);
        sb.ordered.reserve(nTlas);
        BuildNode* root = sb.build(0, static_cast<int>(nTlas));
        std::vector<RefNode> ref(static_cast<size_t>(sb.total));
        int offset = 0;
        sb.flatten(root, ref, &offset, 0, B.maxDepth);
        if (B.maxDepth + 2 > kMaxStack) {
            setError("BVH depth " + std::to_string(B.maxDepth) + " exceeds the traversal stack of " +
                     std::to_string(kMaxStack));
            return PE_ERR_LIMIT;
        }
        // lean triangles in leaf order
        B.tris.resize(static_cast<size_t>(nTris) * 3);
        for (size_t i = 0; i < sb.ordered.size(); ++i) {
            const uint32_t g = static_cast<uint32_t>(sb.ordered[i]);
            const int4 tv = B.triVerts[g];
            if (tv.x == -2) {
                // mesh instance: its index; the instance's visibility mask and material type
                const HostShape& sh = s->shapes[static_cast<size_t>(tv.w)];
                const uint32_t matType = static_cast<uint32_t>(s->materials[static_cast<size_t>(sh.material)].type);
                B.tris[3 * i + 0] = f4(bitsf(static_cast<uint32_t>(instOfShape[static_cast<size_t>(tv.w)])), 0.0f, 0.0f, 0.0f);
                B.tris[3 * i + 1] = f4(0.0f, 0.0f, 0.0f,
                                       bitsf(static_cast<uint32_t>(triMask[g]) | (matType << 8) | PRIM_INSTANCE));
                B.tris[3 * i + 2] = f4(0.0f, 0.0f, 0.0f, bitsf(g));
                continue;
            }
            if (tv.x < 0) {
                // analytic sphere: (centre, radius), meta with the sphere bit, global id
                const HostShape& sh = s->shapes[static_cast<size_t>(tv.w)];
                const uint32_t matType = static_cast<uint32_t>(s->materials[static_cast<size_t>(sh.material)].type);
                B.tris[3 * i + 0] = f4(sh.center.x, sh.center.y, sh.center.z, sh.radius);
                B.tris[3 * i + 1] = f4(0.0f, 0.0f, 0.0f,
                                       bitsf(static_cast<uint32_t>(triMask[g]) | (matType << 8) | PRIM_SPHERE));
                B.tris[3 * i + 2] = f4(0.0f, 0.0f, 0.0f, bitsf(g));
                continue;
            }
            // w: visibility mask (bits 0-7) and material type (bits 8-15; the shading key)
            const uint32_t matType = static_cast<uint32_t>(s->materials[static_cast<size_t>(
                s->shapes[static_cast<size_t>(tv.w)].material)].type);
            triRecord(i, g, static_cast<uint32_t>(triMask[g]) | (matType << 8));
        }
        // interior nodes → 64-byte child-box nodes
        if (emitBinaryNodes(ref, 0, B) == kNoRoot) return PE_ERR_LIMIT;
        // 4-wide nodes for the traversal kernels (the same leaves, boxes and leaf order)
        B.tlasRef.resize(ref.size());
        for (size_t i = 0; i < ref.size(); ++i) {
            const Box& b = ref[i].bounds;
            B.tlasRef[i] = HostBuild::TreeNode{{b.lo.x, b.lo.y, b.lo.z}, {b.hi.x, b.hi.y, b.hi.z}, ref[i].offset, ref[i].count};
        }
        B.tlasOrdered.assign(sb.ordered.begin(), sb.ordered.end());
        B.tlasPrimBounds.resize(6 * static_cast<size_t>(nTlas));
        for (uint32_t i = 0; i < nTlas; ++i) {
            const Box& b = triBounds[i];
            const float v[6] = {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z};
            std::copy(v, v + 6, &B.tlasPrimBounds[6 * i]);
        }
        B.tlasInterior = static_cast<int32_t>(B.nodes.size() / 4);
        B.tlasWideKids.clear();
        if (ref[0].count == 0) {
            int depth4 = 0;
            collapseWide(ref, B.wide, depth4, 0, 1, 0, &B.tlasWideKids);
            B.wideDepth = depth4;
            if (3 * depth4 + 1 > kWideStack) {
                setError("4-wide BVH depth " + std::to_string(depth4) + " exceeds the traversal stack of " +
                         std::to_string(kWideStack));
                return PE_ERR_LIMIT;
            }
        }
        B.rootIsLeaf = ref[0].count > 0 ? 1 : 0;
        B.rootFirst = ref[0].count > 0 ? ref[0].offset : 0;
        B.rootCount = ref[0].count;
        B.rootMin[0] = ref[0].bounds.lo.x;
        B.rootMin[1] = ref[0].bounds.lo.y;
        B.rootMin[2] = ref[0].bounds.lo.z;
        B.rootMax[0] = ref[0].bounds.hi.x;
        B.rootMax[1] = ref[0].bounds.hi.y;
        B.rootMax[2] = ref[0].bounds.hi.z;
    }
    // BLASes: each mesh kept for instancing gets its own tree over its triangles in local space
    // (BVH::buildMesh, bvh.cpp:58-90), or — at most 16 triangles — one leaf in index order, the
    // order TriangleMesh::intersectAccelerated tests small meshes in (mesh.cpp:151-155).  Their
    // leaf records follow the top level's; their nodes follow the top level's nodes.
    std::vector<int32_t> blasRootB(s->blases.size()), blasRootW(s->blases.size()), blasRec(s->blases.size());
    uint32_t rec = nTlas;
    if (!s->blases.empty()) B.tris.resize(static_cast<size_t>(nTris) * 3);
    for (size_t b = 0; b < s->blases.size(); ++b) {
        const HostBlas& hb = s->blases[b];
        const uint32_t n = static_cast<uint32_t>(hb.idx.size() / 3), tb = blasFirstTri[b];
        blasRec[b] = static_cast<int32_t>(rec);
        if (n <= 16) {
            for (uint32_t k = 0; k < n; ++k) triRecord(rec + k, tb + k, VIS_ALL_MASK);
            blasRootB[b] = blasRootW[b] = static_cast<int32_t>(~((rec << 8) | (n - 1)));
        } else {
            SahBuilder bb;
            bb.prims.reserve(n);
            for (uint32_t k = 0; k < n; ++k) {
                const V3 p0 = hb.pos[hb.idx[3 * k]], p1 = hb.pos[hb.idx[3 * k + 1]], p2 = hb.pos[hb.idx[3 * k + 2]];
                Box bx;
                bx.lo = vmin(vmin(p0, p1), p2);
                bx.hi = vmax(vmax(p0, p1), p2);
                bb.prims.emplace_back(k, bx);
            }
            bb.ordered.reserve(n);
            BuildNode* root = bb.build(0, static_cast<int>(n));
            std::vector<RefNode> bref(static_cast<size_t>(bb.total));
            int offset = 0, depth = 0;
            bb.flatten(root, bref, &offset, 0, depth);
            if (depth + 2 > kMaxStack) {
                setError("BLAS depth " + std::to_string(depth) + " exceeds the traversal stack of " + std::to_string(kMaxStack));
                return PE_ERR_LIMIT;
            }
            for (size_t i = 0; i < bb.ordered.size(); ++i)
                triRecord(rec + i, tb + static_cast<uint32_t>(bb.ordered[i]), VIS_ALL_MASK);
            const int32_t rb = emitBinaryNodes(bref, static_cast<int>(rec), B);
            if (rb == kNoRoot) return PE_ERR_LIMIT;
            blasRootB[b] = rb;
            if (bref[0].count == 0) {
                int depth4 = 0;
                blasRootW[b] = collapseWide(bref, B.wide, depth4, 0, 1, static_cast<int>(rec));
                if (3 * depth4 + 1 > kWideStack) {
                    setError("4-wide BLAS depth " + std::to_string(depth4) + " exceeds the traversal stack of " +
                             std::to_string(kWideStack));
                    return PE_ERR_LIMIT;
                }
            } else {
                blasRootW[b] = rb;
            }
        }
        rec += n;
    }
    for (size_t si = 0; si < s->shapes.size(); ++si) {
        const int ii = instOfShape[si];
        if (ii < 0) continue;
        const HostShape& sh = s->shapes[si];
        InstGPU& g = B.instances[static_cast<size_t>(ii)];
        std::memset(&g, 0, sizeof(g));
        for (int r = 0; r < 4; ++r) {
            g.w2l[r] = f4(sh.w2l[4 * r], sh.w2l[4 * r + 1], sh.w2l[4 * r + 2], sh.w2l[4 * r + 3]);
            g.l2w[r] = f4(sh.l2w[4 * r], sh.l2w[4 * r + 1], sh.l2w[4 * r + 2], sh.l2w[4 * r + 3]);
        }
        const size_t bl = static_cast<size_t>(sh.blas);
        g.rootBinary = blasRootB[bl];
        g.rootWide = blasRootW[bl];
        g.recBase = blasRec[bl];
        g.firstTri = static_cast<int32_t>(blasFirstTri[bl]);
        g.shape = static_cast<int32_t>(si);
        g.material = sh.material;
        g.uvScale = uvScaleOf(sh.l2w);
        g.motion = -1;
        if (sh.motion) {
            g.motion = static_cast<int32_t>(B.motions.size());
            InstMotionGPU mg;
            std::memset(&mg, 0, sizeof(mg));
            for (int r = 0; r < 4; ++r) {
                mg.l2w1[r] = f4(sh.l2w1[4 * r], sh.l2w1[4 * r + 1], sh.l2w1[4 * r + 2], sh.l2w1[4 * r + 3]);
                mg.w2l1[r] = f4(sh.w2l1[4 * r], sh.w2l1[4 * r + 1], sh.w2l1[4 * r + 2], sh.w2l1[4 * r + 3]);
            }
            mg.trs = motionTRS(sh.l2w, sh.l2w1);
            mg.uvScale1 = uvScaleOf(sh.l2w1);
            B.motions.push_back(mg);
        }
    }

    buildLightSampler(s, B);
    if (s->env.present) buildEnvironment(s->env);
    // light groups (scene.cpp:144-174): only when some light or the environment names one; then
    // every light joins its group or "Default", the environment its group or "Env", at most 16
    // groups (later names fall into group 0)
    B.groupNames.clear();
    B.lightGroup.clear();
    B.envGroup = -1;
    bool anyGroup = s->env.present && !s->envLightGroup.empty();
    for (size_t i = 0; i < s->lights.size() && i < s->lightGroups.size(); ++i)
        if (!s->lightGroups[i].empty()) anyGroup = true;
    if (anyGroup) {
        auto groupOf = [&](const std::string& name) -> int32_t {
            for (size_t g = 0; g < B.groupNames.size(); ++g)
                if (B.groupNames[g] == name) return static_cast<int32_t>(g);
            if (B.groupNames.size() >= static_cast<size_t>(PE_MAX_LIGHT_GROUPS)) return 0;
            B.groupNames.push_back(name);
            return static_cast<int32_t>(B.groupNames.size() - 1);
        };
        B.lightGroup.resize(s->lights.size());
        for (size_t i = 0; i < s->lights.size(); ++i) {
            const std::string& g = i < s->lightGroups.size() ? s->lightGroups[i] : std::string();
            B.lightGroup[i] = groupOf(g.empty() ? std::string("Default") : g);
        }
        if (s->env.present) B.envGroup = groupOf(s->envLightGroup.empty() ? std::string("Env") : s->envLightGroup);
    }
    // data-pass colours: shapes by their node uid, materials by their index + 1
    B.idColor.resize(B.shapes.size() + B.materials.size());
    for (size_t i = 0; i < B.shapes.size(); ++i) {
        const V3 c = idColorOf(i < s->shapeUid.size() ? s->shapeUid[i] : 0ull);
        B.idColor[i] = f4(c.x, c.y, c.z, 0.0f);
    }
    for (size_t m = 0; m < B.materials.size(); ++m) {
        const V3 c = idColorOf(static_cast<uint64_t>(m) + 1ull);
        B.idColor[B.shapes.size() + m] = f4(c.x, c.y, c.z, 0.0f);
    }
    // Cryptomatte ids in w (buildCryptoLookup, renderer.cpp:75-118): a shape by its name, else
    // "object_<node uid>", else "shape_<n>" counting the unnamed untagged shapes; a material by
    // its name, else "material_<n>" counting unnamed materials as the shapes first use them
    {
        size_t anonShape = 0, anonMat = 0;
        std::vector<int> matSeen(s->materials.size(), 0);
        for (size_t i = 0; i < B.shapes.size(); ++i) {
            const std::string& nm = i < s->shapeNames.size() ? s->shapeNames[i] : std::string();
            const uint64_t uid = i < s->shapeUid.size() ? s->shapeUid[i] : 0ull;
            const std::string name = !nm.empty() ? nm
                                   : uid != 0 ? "object_" + std::to_string(uid)
                                              : "shape_" + std::to_string(anonShape++);
            B.idColor[i].w = cryptoId(name);
            const int mi = B.shapes[i].material;
            if (mi >= 0 && static_cast<size_t>(mi) < s->materials.size() && !matSeen[static_cast<size_t>(mi)]) {
                matSeen[static_cast<size_t>(mi)] = 1;
                const std::string& mn = static_cast<size_t>(mi) < s->materialNames.size() ? s->materialNames[static_cast<size_t>(mi)]
                                                                                         : std::string();
                B.idColor[B.shapes.size() + static_cast<size_t>(mi)].w =
                    cryptoId(!mn.empty() ? mn : "material_" + std::to_string(anonMat++));
            }
        }
    }
    s->built = true;
    ++s->version;
    return PE_OK;
}



const char* lastErrorCStr() { return tlsError.c_str(); }

} // namespace pe

using namespace pe;

extern "C" {

const char* pe_last_error(void) { return pe::lastErrorCStr(); }
int32_t pe_abi_version(void) { return PE_ABI_VERSION; }

// Reference defaults: DisneyMaterial members (disney.h:213-250), Dielectric members
// (dielectric.h), specular 0.5.
void pe_material_defaults(int32_t type, pe_material* m) {
    if (!m) return;
    std::memset(m, 0, sizeof(pe_material));
    m->type = type;
    m->albedo_texture = m->roughness_texture = m->metalness_texture = m->normal_texture = -1;
    m->opacity_texture = -1;
    m->texture_scale = 1.0f;
    for (int i = 0; i < 3; ++i) {
        m->base_color[i] = 0.8f;
        m->coat_tint[i] = 1.0f;
        m->sheen_color[i] = 1.0f;
        m->edge_tint[i] = 1.0f;
        m->flake_color[i] = 0.9f;
        m->absorb_color[i] = 1.0f;
        m->scatter_color[i] = 1.0f;
    }
    m->subsurface_radius[0] = 1.0f;
    m->subsurface_radius[1] = 0.2f;
    m->subsurface_radius[2] = 0.1f;
    m->metallic = 0.0f;
    m->roughness = 0.5f;
    m->specular = 0.5f;
    m->clearcoat_roughness = 0.03f;
    m->ior = 1.5f;
    m->coat_ior = 1.5f;
    m->sheen_roughness = 0.3f;
    m->subsurface_scale = 0.05f;
    m->thin_film_ior = 1.4f;
    m->flake_size = 0.004f;
    m->flake_roughness = 0.3f;
    m->opacity = 1.0f;
    m->absorb_distance = 1.0f;
    if (type == PE_MAT_DIELECTRIC) {
        for (int i = 0; i < 3; ++i) m->base_color[i] = 1.0f;
    }
}

pe_scene* pe_scene_create(void) { return new (std::nothrow) pe_scene(); }
void pe_scene_destroy(pe_scene* s) { delete s; }

int32_t pe_scene_add_material(pe_scene* s, const pe_material* m) {
    if (!s || !m) {
        setError("pe_scene_add_material: null argument");
        return -1;
    }
    if (m->type < PE_MAT_LAMBERT || m->type > PE_MAT_MIRROR) {
        setError("pe_scene_add_material: unknown material type " + std::to_string(m->type));
        return -1;
    }
    for (int32_t t : {m->albedo_texture, m->roughness_texture, m->metalness_texture, m->normal_texture,
                      m->opacity_texture})
        if (t < -1 || t >= static_cast<int32_t>(s->textures.size())) {
            setError("pe_scene_add_material: texture index " + std::to_string(t) + " not added with pe_scene_add_texture");
            return -1;
        }
    s->materialsIn.push_back(*m);
    s->materials.push_back(resolveMaterial(*m));
    s->built = false;
    return static_cast<int32_t>(s->materials.size() - 1);
}

int32_t pe_scene_set_material(pe_scene* s, int32_t index, const pe_material* m) {
    if (!s || !m || index < 0 || index >= static_cast<int32_t>(s->materialsIn.size())) {
        setError("pe_scene_set_material: bad argument");
        return PE_ERR_INVALID;
    }
    for (int32_t t : {m->albedo_texture, m->roughness_texture, m->metalness_texture, m->normal_texture,
                      m->opacity_texture})
        if (t < -1 || t >= static_cast<int32_t>(s->textures.size())) {
            setError("pe_scene_set_material: texture index " + std::to_string(t) + " not added");
            return PE_ERR_INVALID;
        }
    const MatGPU g = resolveMaterial(*m);
    const MatGPU& old = s->materials[static_cast<size_t>(index)];
    // what the built scene derived from the material (its lights, the triangles' shading keys,
    // the media, shadow and walk switches) must stay as it is
    const int32_t structural = MF_EMISSIVE | MF_DELTA | MF_VOLUME_BOUNDARY | MF_TRANSMITS_SHADOWS | MF_DISPERSIVE |
                               MF_HAS_MEDIUM | MF_MEDIUM_SCATTERS;
    const bool walks = g.type == PE_MAT_DISNEY && g.subsurface > 0.0f;
    const bool walked = old.type == PE_MAT_DISNEY && old.subsurface > 0.0f;
    const bool emissionMoved = g.emission[0] != old.emission[0] || g.emission[1] != old.emission[1] ||
                               g.emission[2] != old.emission[2];
    if (g.type != old.type || (g.flags & structural) != (old.flags & structural) || walks != walked ||
        emissionMoved) {
        setError("pe_scene_set_material: the change needs a full rebuild (type, emission, media, shadow or walk "
                 "properties differ)");
        return PE_ERR_LIMIT;
    }
    s->materialsIn[static_cast<size_t>(index)] = *m;
    s->materials[static_cast<size_t>(index)] = g;
    if (s->built && static_cast<size_t>(index) < s->build.materials.size()) s->build.materials[static_cast<size_t>(index)] = g;
    ++s->materialVersion;
    return PE_OK;
}

int32_t pe_scene_set_area_light_radiance(pe_scene* s, int32_t light, const float radiance[3]) {
    if (!s || !radiance || light < 0 || light >= static_cast<int32_t>(s->lights.size()) ||
        s->lights[static_cast<size_t>(light)].type != LT_AREA) {
        setError("pe_scene_set_area_light_radiance: not an area light");
        return PE_ERR_INVALID;
    }
    if (!(radiance[0] > 0.0f || radiance[1] > 0.0f || radiance[2] > 0.0f)) {
        setError("pe_scene_set_area_light_radiance: a dark light changes the scene's emitters (rebuild)");
        return PE_ERR_LIMIT;
    }
    LightGPU& l = s->lights[static_cast<size_t>(light)];
    l.radiance_r = radiance[0];
    l.radiance_g = radiance[1];
    l.radiance_b = radiance[2];
    // the quad's own emissive material (its two triangles in the BVH)
    for (const HostShape& sh : s->shapes)
        if ((sh.flags & SF_AREA_TRIANGLE) && sh.emitter == light) {
            pe_material& m = s->materialsIn[static_cast<size_t>(sh.material)];
            for (int i = 0; i < 3; ++i) m.emission[i] = radiance[i];
            s->materials[static_cast<size_t>(sh.material)] = resolveMaterial(m);
            if (s->built) s->build.materials[static_cast<size_t>(sh.material)] = s->materials[static_cast<size_t>(sh.material)];
            break;
        }
    // the light sampler weighs lights by their power
    if (s->built) buildLightSampler(s, s->build);
    ++s->materialVersion;
    return PE_OK;
}

int32_t pe_scene_add_mesh(pe_scene* s, const float* positions, uint32_t nv, const float* normals, const float* uvs,
                          const uint32_t* indices, uint32_t ntri, int32_t material) {
    if (!s || (nv && !positions) || (ntri && !indices)) {
        setError("pe_scene_add_mesh: null argument");
        return PE_ERR_INVALID;
    }
    if (material < 0 || material >= static_cast<int32_t>(s->materials.size())) {
        setError("pe_scene_add_mesh: material index out of range");
        return PE_ERR_INVALID;
    }
    for (uint64_t i = 0; i < 3ull * ntri; ++i)
        if (indices[i] >= nv) {
            setError("pe_scene_add_mesh: vertex index out of range");
            return PE_ERR_INVALID;
        }
    HostShape sh;
    sh.material = material;
    sh.pos.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) sh.pos[i] = mk(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
    sh.idx.assign(indices, indices + 3ull * ntri);
    if (normals) {
        sh.nrm.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) sh.nrm[i] = mk(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
    } else if (nv > 0 && ntri > 0) {
        // TriangleMesh::calculateNormals (mesh.cpp:30-55)
        sh.nrm.assign(nv, mk(0.0f));
        for (size_t i = 0; i < sh.idx.size(); i += 3) {
            const uint32_t a = sh.idx[i], b = sh.idx[i + 1], c = sh.idx[i + 2];
            const V3 n = cross(sh.pos[b] - sh.pos[a], sh.pos[c] - sh.pos[a]);
            sh.nrm[a] += n;
            sh.nrm[b] += n;
            sh.nrm[c] += n;
        }
        for (V3& n : sh.nrm)
            if (len2(n) > 0.0f) n = normalize(n);
    }
    if (!sh.nrm.empty()) sh.flags |= SF_HAS_NORMALS;
    if (uvs) {
        sh.uv.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) sh.uv[i] = mk2(uvs[2 * i], uvs[2 * i + 1]);
        sh.flags |= SF_HAS_UVS;
    }
    // Emissive mesh → one TriangleLight per triangle (scene.cpp:46-62).
    const MatGPU& mg = s->materials[static_cast<size_t>(material)];
    if (mg.flags & MF_EMISSIVE) {
        sh.emitter = static_cast<int32_t>(s->lights.size());
        for (uint32_t t = 0; t < ntri; ++t) {
            const V3 p0 = sh.pos[sh.idx[3 * t]], p1 = sh.pos[sh.idx[3 * t + 1]], p2 = sh.pos[sh.idx[3 * t + 2]];
            LightGPU l;
            std::memset(&l, 0, sizeof(l));
            l.type = LT_TRIANGLE;
            const V3 n = cross(p1 - p0, p2 - p0);
            const float len = length(n);
            l.area = 0.5f * len;
            const V3 nn = len > 0.0f ? n / len : mk(0.0f, 1.0f, 0.0f);
            l.p0[0] = p0.x; l.p0[1] = p0.y; l.p0[2] = p0.z;
            l.p1[0] = p1.x; l.p1[1] = p1.y; l.p1[2] = p1.z;
            l.p2[0] = p2.x; l.p2[1] = p2.y; l.p2[2] = p2.z;
            l.normal[0] = nn.x; l.normal[1] = nn.y; l.normal[2] = nn.z;
            l.radiance_r = mg.emission[0];
            l.radiance_g = mg.emission[1];
            l.radiance_b = mg.emission[2];
            s->lights.push_back(l);
        }
    }
    s->shapes.push_back(std::move(sh));
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_add_blas(pe_scene* s, const float* positions, uint32_t nv, const float* normals, const float* uvs,
                          const uint32_t* indices, uint32_t ntri) {
    if (!s || !positions || !indices || nv == 0 || ntri == 0) {
        setError("pe_scene_add_blas: a mesh for instancing needs vertices and triangles");
        return -PE_ERR_INVALID;
    }
    if (ntri > static_cast<uint32_t>(kMaxBlasRecords)) {
        setError("pe_scene_add_blas: at most " + std::to_string(kMaxBlasRecords) + " triangles a mesh for instancing");
        return -PE_ERR_LIMIT;
    }
    for (uint64_t i = 0; i < 3ull * ntri; ++i)
        if (indices[i] >= nv) {
            setError("pe_scene_add_blas: vertex index out of range");
            return -PE_ERR_INVALID;
        }
    HostBlas hb;
    hb.pos.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) hb.pos[i] = mk(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
    hb.idx.assign(indices, indices + 3ull * ntri);
    if (normals) {
        hb.nrm.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) hb.nrm[i] = mk(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
    } else {
        // TriangleMesh::calculateNormals (mesh.cpp:30-55)
        hb.nrm.assign(nv, mk(0.0f));
        for (size_t i = 0; i < hb.idx.size(); i += 3) {
            const uint32_t a = hb.idx[i], b = hb.idx[i + 1], c = hb.idx[i + 2];
            const V3 n = cross(hb.pos[b] - hb.pos[a], hb.pos[c] - hb.pos[a]);
            hb.nrm[a] += n;
            hb.nrm[b] += n;
            hb.nrm[c] += n;
        }
        for (V3& n : hb.nrm)
            if (len2(n) > 0.0f) n = normalize(n);
    }
    hb.flags = SF_HAS_NORMALS;
    if (uvs) {
        hb.uv.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) hb.uv[i] = mk2(uvs[2 * i], uvs[2 * i + 1]);
        hb.flags |= SF_HAS_UVS;
    }
    s->blases.push_back(std::move(hb));
    s->built = false;
    return static_cast<int32_t>(s->blases.size() - 1);
}

int32_t pe_scene_add_instance(pe_scene* s, int32_t blas, const float localToWorld[16], const float worldToLocal[16],
                              int32_t material) {
    if (!s || !localToWorld) {
        setError("pe_scene_add_instance: null argument");
        return PE_ERR_INVALID;
    }
    if (blas < 0 || blas >= static_cast<int32_t>(s->blases.size())) {
        setError("pe_scene_add_instance: no such mesh for instancing");
        return PE_ERR_INVALID;
    }
    if (material < 0 || material >= static_cast<int32_t>(s->materials.size())) {
        setError("pe_scene_add_instance: material index out of range");
        return PE_ERR_INVALID;
    }
    HostShape sh;
    sh.blas = blas;
    sh.material = material;
    std::memcpy(sh.l2w, localToWorld, sizeof(sh.l2w));
    if (worldToLocal) std::memcpy(sh.w2l, worldToLocal, sizeof(sh.w2l));
    else mat4Inverse(sh.l2w, sh.w2l);
    const HostBlas& hb = s->blases[static_cast<size_t>(blas)];
    sh.flags = SF_INSTANCE | hb.flags;
    // An emissive instance: one TriangleLight per triangle of its mesh, placed by the transform
    // (Scene::addShape, scene.cpp:23-41).
    const MatGPU& mg = s->materials[static_cast<size_t>(material)];
    if (mg.flags & MF_EMISSIVE) {
        sh.emitter = static_cast<int32_t>(s->lights.size());
        for (size_t t = 0; t < hb.idx.size() / 3; ++t) {
            const V3 p0 = xfPoint(sh.l2w, hb.pos[hb.idx[3 * t]]), p1 = xfPoint(sh.l2w, hb.pos[hb.idx[3 * t + 1]]),
                     p2 = xfPoint(sh.l2w, hb.pos[hb.idx[3 * t + 2]]);
            LightGPU l;
            std::memset(&l, 0, sizeof(l));
            l.type = LT_TRIANGLE;
            const V3 n = cross(p1 - p0, p2 - p0);
            const float len = length(n);
            l.area = 0.5f * len;
            const V3 nn = len > 0.0f ? n / len : mk(0.0f, 1.0f, 0.0f);
            l.p0[0] = p0.x; l.p0[1] = p0.y; l.p0[2] = p0.z;
            l.p1[0] = p1.x; l.p1[1] = p1.y; l.p1[2] = p1.z;
            l.p2[0] = p2.x; l.p2[1] = p2.y; l.p2[2] = p2.z;
            l.normal[0] = nn.x; l.normal[1] = nn.y; l.normal[2] = nn.z;
            l.radiance_r = mg.emission[0];
            l.radiance_g = mg.emission[1];
            l.radiance_b = mg.emission[2];
            s->lights.push_back(l);
        }
    }
    s->shapes.push_back(std::move(sh));
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_instance_transform(pe_scene* s, int32_t shape, const float localToWorld[16],
                                        const float worldToLocal[16]) {
    if (!s || !localToWorld || shape < 0 || shape >= static_cast<int32_t>(s->shapes.size()) ||
        s->shapes[static_cast<size_t>(shape)].blas < 0) {
        setError("pe_scene_set_instance_transform: not a mesh instance");
        return PE_ERR_INVALID;
    }
    HostShape& sh = s->shapes[static_cast<size_t>(shape)];
    if (sh.emitter >= 0) {
        setError("pe_scene_set_instance_transform: an emissive instance moves its lights; rebuild the scene");
        return PE_ERR_LIMIT;
    }
    if (sh.motion) {
        setError("pe_scene_set_instance_transform: a moving instance; rebuild the scene");
        return PE_ERR_LIMIT;
    }
    std::memcpy(sh.l2w, localToWorld, sizeof(sh.l2w));
    if (worldToLocal) std::memcpy(sh.w2l, worldToLocal, sizeof(sh.w2l));
    else mat4Inverse(sh.l2w, sh.w2l);
    ++s->transformVersion;
    return PE_OK;
}

// Refits the built scene's top-level tree after pe_scene_set_instance_transform: each moved
// instance's box again (transformAABB of its BLAS box), leaf and interior boxes recomputed bottom
// up with the tree's shape and leaf order kept, the binary and 4-wide top-level nodes and the
// instance table rewritten in place.  No BLAS is touched.
int32_t pe_scene_refit(pe_scene* s) {
    if (!s || !s->built) {
        setError("pe_scene_refit: the scene is not built");
        return PE_ERR_INVALID;
    }
    HostBuild& B = s->build;
    if (B.tlasRef.empty()) return PE_OK;
    // primitive boxes: moved instances from their new matrices
    int ii = 0;
    std::vector<int> instShape; // instance shapes in shape order, as the instance table holds them
    for (size_t si = 0; si < s->shapes.size(); ++si)
        if (s->shapes[si].blas >= 0) instShape.push_back(static_cast<int>(si));
    for (uint32_t p = 0; p < B.tlasPrims; ++p) {
        const int4 tv = B.triVerts[p];
        if (tv.x != -2) continue;
        const HostShape& sh = s->shapes[static_cast<size_t>(tv.w)];
        const HostBlas& hb = s->blases[static_cast<size_t>(sh.blas)];
        Box lb;
        for (const V3& q : hb.pos) lb = lb.merged(Box{q, q});
        const Box wb = instanceBox(sh, lb);
        const float v[6] = {wb.lo.x, wb.lo.y, wb.lo.z, wb.hi.x, wb.hi.y, wb.hi.z};
        std::copy(v, v + 6, &B.tlasPrimBounds[6 * p]);
    }
    // bottom up: a node's children follow it in depth-first order
    std::vector<Box> nb(B.tlasRef.size());
    for (size_t k = B.tlasRef.size(); k-- > 0;) {
        const HostBuild::TreeNode& n = B.tlasRef[k];
        Box b;
        if (n.count > 0) {
            for (int j = 0; j < n.count; ++j) {
                const float* v = &B.tlasPrimBounds[6 * B.tlasOrdered[static_cast<size_t>(n.offset + j)]];
                b = b.merged(Box{mk(v[0], v[1], v[2]), mk(v[3], v[4], v[5])});
            }
        } else {
            b = nb[k + 1].merged(nb[static_cast<size_t>(n.offset)]);
        }
        nb[k] = b;
        HostBuild::TreeNode& w = B.tlasRef[k];
        w.lo[0] = b.lo.x; w.lo[1] = b.lo.y; w.lo[2] = b.lo.z;
        w.hi[0] = b.hi.x; w.hi[1] = b.hi.y; w.hi[2] = b.hi.z;
    }
    // binary interior nodes, in the order they were emitted
    int gi = 0;
    for (size_t k = 0; k < B.tlasRef.size(); ++k) {
        if (B.tlasRef[k].count != 0) continue;
        const Box& b0 = nb[k + 1];
        const Box& b1 = nb[static_cast<size_t>(B.tlasRef[k].offset)];
        float4* q = &B.nodes[static_cast<size_t>(gi++) * 4];
        q[0] = f4(b0.lo.x, b0.hi.x, b0.lo.y, b0.hi.y);
        q[1] = f4(b1.lo.x, b1.hi.x, b1.lo.y, b1.hi.y);
        q[2] = f4(b0.lo.z, b0.hi.z, b1.lo.z, b1.hi.z);
    }
    // 4-wide nodes of the top level
    for (size_t w = 0; w < B.tlasWideKids.size(); ++w) {
        const int kids[4] = {B.tlasWideKids[w].x, B.tlasWideKids[w].y, B.tlasWideKids[w].z, B.tlasWideKids[w].w};
        float lo[3][4] = {}, hi[3][4] = {};
        for (int c = 0; c < 4; ++c) {
            if (kids[c] < 0) continue;
            const Box& b = nb[static_cast<size_t>(kids[c])];
            lo[0][c] = b.lo.x; lo[1][c] = b.lo.y; lo[2][c] = b.lo.z;
            hi[0][c] = b.hi.x; hi[1][c] = b.hi.y; hi[2][c] = b.hi.z;
        }
        float4* q = &B.wide[w * 8];
        for (int a = 0; a < 3; ++a) {
            q[2 * a] = f4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
            q[2 * a + 1] = f4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
        }
    }
    B.rootMin[0] = nb[0].lo.x; B.rootMin[1] = nb[0].lo.y; B.rootMin[2] = nb[0].lo.z;
    B.rootMax[0] = nb[0].hi.x; B.rootMax[1] = nb[0].hi.y; B.rootMax[2] = nb[0].hi.z;
    for (int si : instShape) {
        const HostShape& sh = s->shapes[static_cast<size_t>(si)];
        InstGPU& g = B.instances[static_cast<size_t>(ii++)];
        for (int r = 0; r < 4; ++r) {
            g.w2l[r] = f4(sh.w2l[4 * r], sh.w2l[4 * r + 1], sh.w2l[4 * r + 2], sh.w2l[4 * r + 3]);
            g.l2w[r] = f4(sh.l2w[4 * r], sh.l2w[4 * r + 1], sh.l2w[4 * r + 2], sh.l2w[4 * r + 3]);
        }
        g.uvScale = uvScaleOf(sh.l2w);
    }
    ++s->refitVersion;
    return PE_OK;
}

int32_t pe_scene_add_sphere(pe_scene* s, const float center[3], float radius, int32_t material) {
    if (!s || !center) {
        setError("pe_scene_add_sphere: null argument");
        return PE_ERR_INVALID;
    }
    if (material < 0 || material >= static_cast<int32_t>(s->materials.size())) {
        setError("pe_scene_add_sphere: material index out of range");
        return PE_ERR_INVALID;
    }
    if (!(radius > 0.0f) || !std::isfinite(radius)) {
        setError("pe_scene_add_sphere: the radius must be positive and finite");
        return PE_ERR_INVALID;
    }
    HostShape sh;
    sh.sphere = true;
    sh.center = mk(center[0], center[1], center[2]);
    sh.radius = radius;
    sh.material = material;
    sh.flags = SF_SPHERE;
    s->shapes.push_back(std::move(sh));
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_tag_shape(pe_scene* s, int32_t shape, uint64_t nodeUid) {
    if (!s || shape < 0) {
        setError("pe_scene_tag_shape: bad argument");
        return PE_ERR_INVALID;
    }
    if (s->shapeUid.size() <= static_cast<size_t>(shape)) s->shapeUid.resize(static_cast<size_t>(shape) + 1, 0ull);
    s->shapeUid[static_cast<size_t>(shape)] = nodeUid;
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_light_link(pe_scene* s, int32_t light, int32_t mode, const uint64_t* uids, int32_t n,
                                int32_t shadowMode, const uint64_t* shadowUids, int32_t nShadow) {
    if (!s || light < 0 || mode < 0 || mode > 2 || shadowMode < 0 || shadowMode > 2 || n < 0 || nShadow < 0 ||
        (n > 0 && !uids) || (nShadow > 0 && !shadowUids)) {
        setError("pe_scene_set_light_link: bad argument");
        return PE_ERR_INVALID;
    }
    if (s->lightLinks.size() <= static_cast<size_t>(light)) s->lightLinks.resize(static_cast<size_t>(light) + 1);
    HostLightLink& l = s->lightLinks[static_cast<size_t>(light)];
    l.mode = mode;
    l.shadowMode = shadowMode;
    l.uids.assign(uids, uids + n);
    l.shadowUids.assign(shadowUids, shadowUids + nShadow);
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_light_group(pe_scene* s, int32_t light, const char* name) {
    if (!s || light < -1) {
        setError("pe_scene_set_light_group: bad argument");
        return PE_ERR_INVALID;
    }
    const std::string g = name ? std::string(name) : std::string();
    if (light < 0) {
        s->envLightGroup = g;
    } else {
        if (s->lightGroups.size() <= static_cast<size_t>(light)) s->lightGroups.resize(static_cast<size_t>(light) + 1);
        s->lightGroups[static_cast<size_t>(light)] = g;
    }
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_light_groups(const pe_scene* s, char* names, int32_t capacity) {
    if (!s || capacity < 0 || (capacity > 0 && !names)) {
        setError("pe_scene_light_groups: bad argument");
        return PE_ERR_INVALID;
    }
    if (!s->built) {
        setError("pe_scene_light_groups: scene not built");
        return PE_ERR_NO_SCENE;
    }
    const std::vector<std::string>& g = s->build.groupNames;
    if (names) {
        std::string all;
        for (const std::string& n : g) {
            all += n;
            all.push_back('\0');
        }
        const size_t k = std::min(all.size(), static_cast<size_t>(capacity));
        std::memcpy(names, all.data(), k);
        if (k < all.size() && capacity > 0) names[capacity - 1] = '\0';
    }
    return static_cast<int32_t>(g.size());
}

int32_t pe_scene_add_texture(pe_scene* s, const float* rgb, int32_t width, int32_t height) {
    if (!s || !rgb || width <= 0 || height <= 0) {
        setError("pe_scene_add_texture: bad argument");
        return PE_ERR_INVALID;
    }
    pe_scene::Texture t;
    t.width = width;
    t.height = height;
    t.texels.assign(rgb, rgb + static_cast<size_t>(width) * static_cast<size_t>(height) * 3);
    s->textures.push_back(std::move(t));
    s->built = false;
    return static_cast<int32_t>(s->textures.size() - 1);
}

// Image::buildMipmaps (image.cpp:102-155), Float32 storage: each level the 2×2 box mean of the
// one before (the last row / column repeated on odd sizes), down to 1×1.
// 8-bit storage (Image::StorageFormat U8Srgb / U8Linear, image.cpp:14-36): the sRGB transfer
// of IEC 61966-2-1, decoded through a 256-entry table, encoded with round-to-nearest.
static float srgbToLinear(float e) { return e <= 0.04045f ? e / 12.92f : std::pow((e + 0.055f) / 1.055f, 2.4f); }
static float linearToSrgb(float l) {
    l = std::min(std::max(l, 0.0f), 1.0f);
    return l <= 0.0031308f ? 12.92f * l : 1.055f * std::pow(l, 1.0f / 2.4f) - 0.055f;
}
static const float* decodeTable(int32_t format) {
    static float srgb[256], lin[256];
    static bool ready = false;
    if (!ready) {
        for (int i = 0; i < 256; ++i) {
            srgb[i] = srgbToLinear(static_cast<float>(i) / 255.0f);
            lin[i] = static_cast<float>(i) / 255.0f;
        }
        ready = true;
    }
    return format == 1 ? srgb : lin;
}
static uint8_t encode8(float v, int32_t format) {
    const float c = std::min(std::max(v, 0.0f), 1.0f);
    const float e = format == 1 ? linearToSrgb(c) : c;
    return static_cast<uint8_t>(std::lround(e * 255.0f));
}

int32_t pe_scene_add_texture_u8(pe_scene* s, const uint8_t* rgb, int32_t width, int32_t height, int32_t srgb) {
    if (!s || !rgb || width <= 0 || height <= 0) {
        setError("pe_scene_add_texture_u8: bad argument");
        return PE_ERR_INVALID;
    }
    pe_scene::Texture t;
    t.width = width;
    t.height = height;
    t.format = srgb ? 1 : 2;
    const float* lut = decodeTable(t.format);
    const size_t n = static_cast<size_t>(width) * static_cast<size_t>(height) * 3;
    t.texels.resize(n);
    for (size_t i = 0; i < n; ++i) t.texels[i] = lut[rgb[i]];
    s->textures.push_back(std::move(t));
    s->built = false;
    return static_cast<int32_t>(s->textures.size() - 1);
}

int32_t pe_scene_build_texture_mipmaps(pe_scene* s, int32_t texture) {
    if (!s || texture < 0 || texture >= static_cast<int32_t>(s->textures.size())) {
        setError("pe_scene_build_texture_mipmaps: bad texture index");
        return PE_ERR_INVALID;
    }
    pe_scene::Texture& t = s->textures[static_cast<size_t>(texture)];
    t.mips.clear();
    t.mipW.clear();
    t.mipH.clear();
    int pw = t.width, ph = t.height;
    const std::vector<float>* prev = &t.texels;
    while ((pw > 1 || ph > 1) && t.mips.size() + 1 < static_cast<size_t>(kMaxMipLevels)) {
        const int nw = std::max(1, pw / 2), nh = std::max(1, ph / 2);
        std::vector<float> next(static_cast<size_t>(nw) * static_cast<size_t>(nh) * 3, 0.0f);
        for (int y = 0; y < nh; ++y) {
            const int ya = std::min(2 * y, ph - 1), yb = std::min(2 * y + 1, ph - 1);
            for (int x = 0; x < nw; ++x) {
                const int xa = std::min(2 * x, pw - 1), xb = std::min(2 * x + 1, pw - 1);
                auto at = [&](int px, int py) {
                    return (static_cast<size_t>(py) * static_cast<size_t>(pw) + static_cast<size_t>(px)) * 3;
                };
                const size_t o = (static_cast<size_t>(y) * static_cast<size_t>(nw) + static_cast<size_t>(x)) * 3;
                for (int c = 0; c < 3; ++c)
                    next[o + static_cast<size_t>(c)] =
                        0.25f * ((*prev)[at(xa, ya) + c] + (*prev)[at(xb, ya) + c] + (*prev)[at(xa, yb) + c] +
                                 (*prev)[at(xb, yb) + c]);
            }
        }
        t.mips.push_back(std::move(next));
        t.mipW.push_back(nw);
        t.mipH.push_back(nh);
        prev = &t.mips.back();
        pw = nw;
        ph = nh;
    }
    if (t.format != 0) {
        // 8-bit images keep each level quantised (the chain itself runs in float)
        const float* lut = decodeTable(t.format);
        for (std::vector<float>& level : t.mips)
            for (float& v : level) v = lut[encode8(v, t.format)];
    }
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_shape_name(pe_scene* s, int32_t shape, const char* name) {
    if (!s || shape < 0) {
        setError("pe_scene_set_shape_name: bad argument");
        return PE_ERR_INVALID;
    }
    if (s->shapeNames.size() <= static_cast<size_t>(shape)) s->shapeNames.resize(static_cast<size_t>(shape) + 1);
    s->shapeNames[static_cast<size_t>(shape)] = name ? name : "";
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_instance_motion(pe_scene* s, int32_t shape, const float localToWorldEnd[16],
                                     const float worldToLocalEnd[16]) {
    if (!s || !localToWorldEnd || shape < 0 || shape >= static_cast<int32_t>(s->shapes.size()) ||
        s->shapes[static_cast<size_t>(shape)].blas < 0) {
        setError("pe_scene_set_instance_motion: not a mesh instance");
        return PE_ERR_INVALID;
    }
    HostShape& sh = s->shapes[static_cast<size_t>(shape)];
    sh.motion = true;
    std::memcpy(sh.l2w1, localToWorldEnd, sizeof(sh.l2w1));
    if (worldToLocalEnd) std::memcpy(sh.w2l1, worldToLocalEnd, sizeof(sh.w2l1));
    else mat4Inverse(sh.l2w1, sh.w2l1);
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_shape_bounds(const pe_scene* s, int32_t shape, float out[6]) {
    if (!s || !out || shape < 0 || shape >= static_cast<int32_t>(s->shapes.size())) {
        setError("pe_scene_shape_bounds: no such shape");
        return PE_ERR_INVALID;
    }
    const HostShape& sh = s->shapes[static_cast<size_t>(shape)];
    Box b;
    if (sh.blas >= 0) {
        Box local;
        for (const V3& p : s->blases[static_cast<size_t>(sh.blas)].pos) local = local.merged(Box{p, p});
        b = instanceBox(sh, local);
    } else if (sh.sphere) {
        b = Box{sh.center - mk(sh.radius), sh.center + mk(sh.radius)};
    } else {
        for (const V3& p : sh.pos) b = b.merged(Box{p, p});
    }
    const float v[6] = {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z};
    std::copy(v, v + 6, out);
    return PE_OK;
}

void pe_mat4_inverse(const float m[16], float out[16]) {
    if (m && out) mat4Inverse(m, out);
}

// Shape::setVisibilityMask (shape.h:27-29): the ray classes (camera, diffuse, glossy,
// transmission, shadow) that see shape `shape`; a mesh instance's mask is tested at the top level
// only (mesh_instance.cpp:106).
int32_t pe_scene_set_shape_visibility(pe_scene* s, int32_t shape, uint32_t mask) {
    if (!s || shape < 0 || shape >= static_cast<int32_t>(s->shapes.size())) {
        setError("pe_scene_set_shape_visibility: no such shape");
        return PE_ERR_INVALID;
    }
    s->shapes[static_cast<size_t>(shape)].mask = static_cast<uint8_t>(mask & 0x1Fu);
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_material_name(pe_scene* s, int32_t material, const char* name) {
    if (!s || material < 0) {
        setError("pe_scene_set_material_name: bad argument");
        return PE_ERR_INVALID;
    }
    if (s->materialNames.size() <= static_cast<size_t>(material))
        s->materialNames.resize(static_cast<size_t>(material) + 1);
    s->materialNames[static_cast<size_t>(material)] = name ? name : "";
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_shadow_catcher(pe_scene* s, int32_t shape) {
    if (!s || shape < -1) {
        setError("pe_scene_set_shadow_catcher: bad argument");
        return PE_ERR_INVALID;
    }
    s->catcherShape = shape;
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_add_area_light(pe_scene* s, const float p[3], const float u[3], const float v[3], const float radiance[3],
                                int32_t visible) {
    if (!s || !p || !u || !v || !radiance) {
        setError("pe_scene_add_area_light: null argument");
        return PE_ERR_INVALID;
    }
    const int32_t index = static_cast<int32_t>(s->lights.size());
    const V3 P = m3f(p), U = m3f(u), Vv = m3f(v);
    LightGPU l;
    std::memset(&l, 0, sizeof(l));
    l.type = LT_AREA;
    const V3 nrm = cross(U, Vv);
    l.area = length(nrm);
    const V3 N = normalize(nrm);
    const float lu = length(U), lv = length(Vv);
    l.rectangle = (lu > 0.0f && lv > 0.0f && std::fabs(dot(U, Vv)) <= 1e-4f * lu * lv) ? 1 : 0;
    for (int i = 0; i < 3; ++i) {
        l.p0[i] = p[i];
        l.p1[i] = u[i];
        l.p2[i] = v[i];
    }
    l.normal[0] = N.x; l.normal[1] = N.y; l.normal[2] = N.z;
    l.radiance_r = radiance[0];
    l.radiance_g = radiance[1];
    l.radiance_b = radiance[2];
    s->lights.push_back(l);
    // Emissive black Lambertian quad in the BVH (scene.cpp:76-98).
    pe_material em;
    pe_material_defaults(PE_MAT_LAMBERT, &em);
    em.base_color[0] = em.base_color[1] = em.base_color[2] = 0.0f;
    em.emission[0] = radiance[0];
    em.emission[1] = radiance[1];
    em.emission[2] = radiance[2];
    s->materialsIn.push_back(em);
    s->materials.push_back(resolveMaterial(em));
    const int32_t mat = static_cast<int32_t>(s->materials.size() - 1);
    const V3 p0 = P, p1 = P + U, p2 = p1 + Vv, p3 = P + Vv;
    const V2 uv0 = mk2(0, 0), uv1 = mk2(1, 0), uv2 = mk2(1, 1), uv3 = mk2(0, 1);
    const V3 tris[2][3] = {{p0, p1, p2}, {p0, p2, p3}};
    const V2 uvs[2][3] = {{uv0, uv1, uv2}, {uv0, uv2, uv3}};
    for (int t = 0; t < 2; ++t) {
        HostShape sh;
        sh.material = mat;
        sh.emitter = index;
        sh.flags = SF_AREA_TRIANGLE | SF_HAS_NORMALS | SF_HAS_UVS;
        for (int k = 0; k < 3; ++k) {
            sh.pos.push_back(tris[t][k]);
            sh.nrm.push_back(N);
            sh.uv.push_back(uvs[t][k]);
        }
        sh.idx = {0, 1, 2};
        if (!visible) {
            sh.flags |= SF_CAMERA_INVISIBLE;
            sh.mask = static_cast<uint8_t>(0x1F & ~1u);
        }
        s->shapes.push_back(std::move(sh));
    }
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_environment(pe_scene* s, const float* rgb, int32_t w, int32_t h, float rotation, float intensity) {
    if (!s) {
        setError("pe_scene_set_environment: null scene");
        return PE_ERR_INVALID;
    }
    HostEnv& e = s->env;
    const bool hadSun = e.hasSun;
    const V3 sd = e.sunDirIn, sr = e.sunRadIn;
    const float sc = e.sunCosIn;
    e = HostEnv{};
    e.present = true;
    e.rotation = rotation;
    e.intensity = intensity;
    if (rgb && w > 0 && h > 0) {
        e.hasImage = true;
        e.width = w;
        e.height = h;
        e.image.assign(rgb, rgb + 3ull * static_cast<size_t>(w) * static_cast<size_t>(h));
    }
    e.hasSun = hadSun;
    e.sunDirIn = sd;
    e.sunRadIn = sr;
    e.sunCosIn = sc;
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_sun(pe_scene* s, const float direction[3], float cos_max, const float radiance[3]) {
    if (!s || !direction || !radiance) {
        setError("pe_scene_set_sun: null argument");
        return PE_ERR_INVALID;
    }
    s->env.hasSun = true;
    s->env.sunDirIn = m3f(direction);
    s->env.sunCosIn = cos_max;
    s->env.sunRadIn = m3f(radiance);
    s->built = false;
    return PE_OK;
}

int32_t pe_scene_set_background(pe_scene* s, int32_t mode, const float color[3]) {
    if (!s || mode < PE_BG_ENVIRONMENT || mode > PE_BG_TRANSPARENT) {
        setError("pe_scene_set_background: bad argument");
        return PE_ERR_INVALID;
    }
    s->bgMode = mode;
    if (color)
        for (int i = 0; i < 3; ++i) s->bgColor[i] = color[i];
    return PE_OK;
}

int32_t pe_scene_build(pe_scene* s) {
    if (!s) {
        setError("pe_scene_build: null scene");
        return PE_ERR_INVALID;
    }
    try {
        return pe::buildScene(s);
    } catch (const std::bad_alloc&) {
        setError("pe_scene_build: host out of memory");
        return PE_ERR_OOM;
    }
}

int32_t pe_scene_get_info(const pe_scene* s, pe_scene_info* out) {
    if (!s || !out) {
        setError("pe_scene_get_info: null argument");
        return PE_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    const HostBuild& B = s->build;
    // triangles stored once: scene meshes and each instanced mesh's BLAS (sphere and instance
    // primitives are not triangles)
    out->triangles = static_cast<uint64_t>(
        std::count_if(B.triVerts.begin(), B.triVerts.end(), [](const int4& v) { return v.x >= 0; }));
    out->bvh_nodes = B.nodes.size() / 4;
    out->bvh_leaves = B.leaves;
    out->lights = B.lights.size();
    out->light_bvh_nodes = B.lightNodes.size();
    out->has_environment = s->env.present ? 1 : 0;
    out->light_sampler_mode = B.lightMode;
    out->device_bytes = B.nodes.size() * sizeof(float4) + B.tris.size() * sizeof(float4) +
                        B.triVerts.size() * sizeof(int4) + B.pos.size() * sizeof(float4) * 2 + B.uv.size() * sizeof(float2) +
                        B.wide.size() * sizeof(float4) + B.instances.size() * sizeof(InstGPU) +
                        B.motions.size() * sizeof(InstMotionGPU);
    return s->built ? PE_OK : PE_ERR_INVALID;
}

// PerspectiveCamera constructor + describeGpu (perspective_camera.cpp:12-57).
void pe_camera_perspective(const float position[3], const float target[3], const float up[3], float vfov, float aspect,
                           pe_camera* out) {
    if (!out) return;
    const V3 pos = m3f(position), tgt = m3f(target), upv = m3f(up);
    const float theta = vfov * (kPi / 180.0f);
    const float h = std::tan(theta * 0.5f);
    const float vh = 2.0f * h;
    const float vw = aspect * vh;
    const V3 w = normalize(pos - tgt);
    const V3 u = normalize(cross(upv, w));
    const V3 v = cross(w, u);
    const V3 horizontal = vw * u;
    const V3 vertical = vh * v;
    const V3 lowerLeft = pos - horizontal * 0.5f - vertical * 0.5f - w;
    auto put = [](float* o, V3 a) { o[0] = a.x; o[1] = a.y; o[2] = a.z; };
    put(out->position, pos);
    put(out->lower_left, lowerLeft);
    put(out->horizontal, horizontal);
    put(out->vertical, vertical);
    put(out->u, u);
    put(out->v, v);
    put(out->forward, -w);
    out->lens_radius = 0.0f;
    out->orthographic = 0;
    out->blades = 0;
    out->blade_rotation = 0.0f;
}

void pe_camera_thin_lens(const float position[3], const float target[3], const float up[3], float vfov, float aspect,
                         float aperture, float focus, int32_t blades, float rotationDeg, pe_camera* out) {
    if (!out) return;
    const V3 pos = m3f(position), tgt = m3f(target), upv = m3f(up);
    // the pinhole's frame with the image plane at the focus distance (thin_lens_camera.cpp:14-33)
    const float theta = vfov * (kPi / 180.0f);
    const float h = std::tan(theta * 0.5f);
    const float vh = 2.0f * h * focus;
    const float vw = aspect * vh;
    const V3 w = normalize(pos - tgt);
    const V3 u = normalize(cross(upv, w));
    const V3 v = cross(w, u);
    const V3 horizontal = vw * u;
    const V3 vertical = vh * v;
    const V3 lowerLeft = pos - horizontal * 0.5f - vertical * 0.5f - focus * w;
    auto put = [](float* o, V3 a) { o[0] = a.x; o[1] = a.y; o[2] = a.z; };
    put(out->position, pos);
    put(out->lower_left, lowerLeft);
    put(out->horizontal, horizontal);
    put(out->vertical, vertical);
    put(out->u, u);
    put(out->v, v);
    put(out->forward, -w);
    out->lens_radius = aperture;
    out->orthographic = 0;
    out->blades = blades >= 3 ? blades : 0;
    out->blade_rotation = rotationDeg * 0.017453292519943295f;
}

void pe_camera_orthographic(const float position[3], const float target[3], const float up[3], float extent,
                            float aspect, pe_camera* out) {
    if (!out) return;
    const V3 pos = m3f(position), tgt = m3f(target), upv = m3f(up);
    const V3 w = normalize(pos - tgt);
    const V3 u = normalize(cross(upv, w));
    const V3 v = cross(w, u);
    const float height = extent > 1e-4f ? extent : 1.0f;
    const float width = aspect * height;
    const V3 horizontal = width * u;
    const V3 vertical = height * v;
    const V3 lowerLeft = pos - horizontal * 0.5f - vertical * 0.5f;
    auto put = [](float* o, V3 a) { o[0] = a.x; o[1] = a.y; o[2] = a.z; };
    put(out->position, lowerLeft + horizontal * 0.5f + vertical * 0.5f);
    put(out->lower_left, lowerLeft);
    put(out->horizontal, horizontal);
    put(out->vertical, vertical);
    put(out->u, len2(horizontal) > 0.0f ? normalize(horizontal) : mk(1.0f, 0.0f, 0.0f));
    put(out->v, len2(vertical) > 0.0f ? normalize(vertical) : mk(0.0f, 1.0f, 0.0f));
    put(out->forward, -w);
    out->lens_radius = 0.0f;
    out->orthographic = 1;
    out->blades = 0;
    out->blade_rotation = 0.0f;
}

} // extern "C"
