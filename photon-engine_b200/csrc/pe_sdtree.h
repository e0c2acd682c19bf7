// pe_sdtree.h — SD-tree path guiding on the device (Müller et al. 2017, "Practical Path Guiding";
// the reference's GuidingField / DirectionalTree, src/integrators/path_guiding.{h,cpp}).
//
// A spatial binary tree over the padded scene box (axis = depth mod 3, split at the middle of the
// node's unit cell) ends in leaves; each leaf carries a directional quadtree over the cylindrical
// equal-area map [0,1]² of the sphere (u = (cosθ+1)/2 with θ from +y, v = φ/2π, φ = atan2(z, x),
// path_guiding.cpp:11-25).  The sampling trees are read-only during a render; training splats go
// into building trees whose topology was fixed at the last refinement.  Refinement runs on the
// host (pe_sdtree.cu).
#pragma once

#include "pe_math.h"

#include <cstdint>

namespace pe {

struct SdSpatial {
    int32_t axis;     // -1 = leaf
    int32_t child[2];
    int32_t leaf;     // leaf index when axis < 0
};

struct SdQuad {
    float sums[4];
    int32_t child[4]; // absolute index into the same node array, 0 = leaf
};

struct SdLeaf {
    int32_t sampRoot;  // root of the sampling quadtree
    int32_t buildRoot; // root of the building quadtree
    float sampSum;     // > 0: the sampling tree holds a distribution
    int32_t pad;
};

struct SdField {
    const SdSpatial* spatial;
    const SdLeaf* leaves;
    const SdQuad* samp;
    SdQuad* build;
    float* buildSum;          // per leaf
    uint32_t* sampleCount;    // per leaf
    float boxMin[3], boxExt[3];
    int32_t ready;            // sampling trees refined at least once and holding energy
};

PE_HD V2 sdDirToCanonical(V3 d) {
    const V3 n = normalize(d);
    const float cosT = sclamp(n.y, -1.0f, 1.0f);
    float phi = atan2f(n.z, n.x);
    if (phi < 0.0f) phi += kTwoPi;
    return mk2(sclamp(0.5f * (cosT + 1.0f), 0.0f, 0.9999999f), sclamp(phi * kInvTwoPi, 0.0f, 0.9999999f));
}

PE_HD V3 sdCanonicalToDir(V2 p) {
    const float cosT = sclamp(2.0f * p.x - 1.0f, -1.0f, 1.0f);
    const float sinT = sqrtf(smax(0.0f, 1.0f - cosT * cosT));
    const float phi = kTwoPi * p.y;
    return mk(sinT * cosf(phi), cosT, sinT * sinf(phi));
}

// Leaf of the spatial tree containing p (the unit cell is rescaled at each level).
PE_HD int sdFindLeaf(const SdField& F, V3 p) {
    float u[3];
    const float pp[3] = {p.x, p.y, p.z};
    for (int a = 0; a < 3; ++a)
        u[a] = F.boxExt[a] > 1e-8f ? sclamp((pp[a] - F.boxMin[a]) / F.boxExt[a], 0.0f, 1.0f) : 0.5f;
    int idx = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const SdSpatial n = F.spatial[idx];
        if (n.axis < 0) return n.leaf;
        const float c = u[n.axis];
        const int side = c < 0.5f ? 0 : 1;
        u[n.axis] = side == 0 ? c * 2.0f : c * 2.0f - 1.0f;
        idx = n.child[side];
    }
    return -1;
}

constexpr float kSdInvFourPi = 1.0f / (4.0f * kPi);

// Solid-angle pdf of direction d under the quadtree rooted at `root`.
PE_HD float sdTreePdf(const SdQuad* nodes, int root, V3 d) {
    V2 p = sdDirToCanonical(d);
    float size = 1.0f, prob = 1.0f;
    int idx = root;
    for (int depth = 0; depth < 16; ++depth) {
        const SdQuad& n = nodes[idx];
        const float total = n.sums[0] + n.sums[1] + n.sums[2] + n.sums[3];
        if (!(total > 0.0f)) break;
        const int qx = p.x >= 0.5f ? 1 : 0, qy = p.y >= 0.5f ? 1 : 0;
        const int q = qy * 2 + qx;
        const float qs = n.sums[q];
        if (!(qs > 0.0f)) return 0.0f;
        prob *= qs / total;
        size *= 0.5f;
        const int c = n.child[q];
        if (c <= 0) break;
        p.x = p.x * 2.0f - static_cast<float>(qx);
        p.y = p.y * 2.0f - static_cast<float>(qy);
        idx = c;
    }
    return (prob / smax(size * size, 1e-12f)) * kSdInvFourPi;
}

// A direction from the quadtree: per level the column (x) by its energy, then the row (y) within
// it; the sample lands uniformly in the final cell.
PE_HD V3 sdTreeSample(const SdQuad* nodes, int root, V2 uIn, float& pdf) {
    V2 u = mk2(sclamp(uIn.x, 0.0f, 0.9999999f), sclamp(uIn.y, 0.0f, 0.9999999f));
    float ox = 0.0f, oy = 0.0f, size = 1.0f, prob = 1.0f;
    int idx = root;
    for (int depth = 0; depth < 16; ++depth) {
        const SdQuad& n = nodes[idx];
        const float left = n.sums[0] + n.sums[2], right = n.sums[1] + n.sums[3];
        const float total = left + right;
        if (!(total > 0.0f)) break;
        int qx = 0;
        float px = left / total;
        if (u.x < px) {
            u.x = smin(u.x / smax(px, 1e-8f), 0.9999999f);
        } else {
            qx = 1;
            const float rx = smax(1.0f - px, 1e-8f);
            u.x = smin((u.x - px) / rx, 0.9999999f);
            px = rx;
        }
        const float bot = n.sums[qx], top = n.sums[2 + qx];
        const float col = bot + top;
        int qy = 0;
        float py = col > 0.0f ? bot / col : 0.5f;
        if (u.y < py) {
            u.y = smin(u.y / smax(py, 1e-8f), 0.9999999f);
        } else {
            qy = 1;
            const float ty = smax(1.0f - py, 1e-8f);
            u.y = smin((u.y - py) / ty, 0.9999999f);
            py = ty;
        }
        size *= 0.5f;
        ox += static_cast<float>(qx) * size;
        oy += static_cast<float>(qy) * size;
        prob *= px * py;
        const int c = n.child[qy * 2 + qx];
        if (c <= 0) break;
        idx = c;
    }
    pdf = (prob / smax(size * size, 1e-12f)) * kSdInvFourPi;
    return sdCanonicalToDir(mk2(ox + u.x * size, oy + u.y * size));
}

// Leaf whose sampling tree serves p, or −1 (GuidingField::hasLeafData).
PE_HD int sdLeafWithData(const SdField& F, V3 p) {
    if (!F.ready) return -1;
    const int leaf = sdFindLeaf(F, p);
    return (leaf >= 0 && F.leaves[leaf].sampSum > 0.0f) ? leaf : -1;
}

} // namespace pe
