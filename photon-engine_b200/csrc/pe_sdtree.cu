// pe_sdtree.cu — host side of SD-tree path guiding (pe_sdtree.h): the field's trees, their
// refinement between training passes, the flat device copies the shading kernels read, and the
// kernel that splats a wave's recorded radiance into the building trees.
//
//   GuidingField::reset / splitLeaf / refine        path_guiding.cpp:274-364 → SdHost::reset/split/refine
//   DirectionalTree::buildFrom (copyAndRefine)      path_guiding.cpp:97-143  → refineTopology
//   DirectionalTree::addSplat, GuidingField::record path_guiding.cpp:80-95, 327-334 → kSdRecord
//   training schedule: refine at 2, 4, 8, 16, 32 samples, then frozen (renderer.cpp:413-429, 476-526)
#include "pe_device_impl.h"
#include "pe_sdtree.h"

#include <cmath>
#include <cstring>

using namespace pe;
using namespace pe_dev;

namespace {

// Incident radiance of each recorded vertex: what the path gathered after it, over its
// throughput after the bounce, as luminance over the sampling pdf (the reference's
// lum(suffix) / max(pdf, 1e-4)); splatted into the building quadtree of the vertex's leaf.
__global__ void kSdRecord(Paths P, int nSlots) {
    const SdField& F = P.sd;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nSlots; s += gridDim.x * blockDim.x) {
        const uint32_t n = P.sdCount[s];
        if (n == 0) continue;
        P.sdCount[s] = 0;
        const float4 Lf = P.L[s];
        for (uint32_t k = 0; k < n; ++k) {
            const float4* rec = P.sdRec + (static_cast<size_t>(s) * kSdRecords + k) * 4;
            const float4 r0 = rec[0], r1 = rec[1], r2 = rec[2], r3 = rec[3];
            const V3 snap = r3.w == 2.0f ? mk(r3.x, r3.y, r3.z) : mk(Lf.x, Lf.y, Lf.z);
            const float dl[3] = {Lf.x - snap.x, Lf.y - snap.y, Lf.z - snap.z};
            const float tw[3] = {r2.x, r2.y, r2.z};
            V3 li = mk(0.0f);
            for (int c = 0; c < 3; ++c) set(li, c, tw[c] > 0.0f ? dl[c] / tw[c] : 0.0f);
            const float radiance = luminance(li) / smax(r0.w, 1e-4f);
            if (!(radiance > 0.0f) || !pe::finitef(radiance)) continue;
            const int leaf = sdFindLeaf(F, mk(r0.x, r0.y, r0.z));
            if (leaf < 0) continue;
            atomicAdd(&F.sampleCount[leaf], 1u);
            atomicAdd(&F.buildSum[leaf], radiance);
            V2 p = sdDirToCanonical(mk(r1.x, r1.y, r1.z));
            int idx = F.leaves[leaf].buildRoot;
            for (int depth = 0; depth < 16; ++depth) {
                const int qx = p.x >= 0.5f ? 1 : 0, qy = p.y >= 0.5f ? 1 : 0;
                const int q = qy * 2 + qx;
                atomicAdd(&F.build[idx].sums[q], radiance);
                const int c = F.build[idx].child[q];
                if (c <= 0) break;
                p.x = p.x * 2.0f - static_cast<float>(qx);
                p.y = p.y * 2.0f - static_cast<float>(qy);
                idx = c;
            }
        }
    }
}

} // namespace

namespace pe_dev {

// Next training pass's quadtree topology from a sampling tree: cells holding more than 1 % of the
// energy (at most depth 10, 4096 nodes) are split; sums start at zero.
std::vector<SdQuad> refineTopology(const std::vector<SdQuad>& samp, float sum, float frac, int maxDepth) {
    std::vector<SdQuad> out(1);
    std::memset(out.data(), 0, sizeof(SdQuad));
    const float threshold = sum * std::max(1e-4f, frac);
    // depth-first, children in quadrant order, as the reference's recursion
    auto rec = [&](auto&& self, int src, int dst, int depth) -> void {
        for (int q = 0; q < 4; ++q) {
            const float e = samp[static_cast<size_t>(src)].sums[q];
            const int srcChild = samp[static_cast<size_t>(src)].child[q];
            if (e > threshold && depth < maxDepth && out.size() < 4096) {
                const int nc = static_cast<int>(out.size());
                SdQuad z;
                std::memset(&z, 0, sizeof(z));
                out.push_back(z);
                out[static_cast<size_t>(dst)].child[q] = nc;
                if (srcChild > 0) self(self, srcChild, nc, depth + 1);
            } else {
                out[static_cast<size_t>(dst)].child[q] = 0;
            }
        }
    };
    rec(rec, 0, 0, 0);
    return out;
}

void SdHost::reset(const float bmin[3], const float bmax[3]) {
    for (int a = 0; a < 3; ++a) {
        const float pad = (bmax[a] - bmin[a]) * 0.01f + 1e-3f;
        boxMin[a] = bmin[a] - pad;
        boxMax[a] = bmax[a] + pad;
    }
    nodes.assign(1, Node{});
    leaves.assign(1, Leaf{});
    nodes[0].leaf = 0;
    // an initial 2×2×2 grid of leaves (path_guiding.cpp:287-297)
    auto initSplit = [&](auto&& self, int idx, int depth) -> void {
        if (depth >= 3) return;
        split(idx, depth);
        const int c0 = nodes[static_cast<size_t>(idx)].child[0], c1 = nodes[static_cast<size_t>(idx)].child[1];
        if (c0 >= 0) self(self, c0, depth + 1);
        if (c1 >= 0) self(self, c1, depth + 1);
    };
    initSplit(initSplit, 0, 0);
    ready = false;
    iteration = 0;
    samplesSeen = 0;
    nextRefine = 2;
}

// Splits a leaf in two along axis depth mod 3; both children start from the parent's trees.
void SdHost::split(int idx, int depth) {
    if (depth >= 12 || nodes.size() >= 4096) return;
    const int leafIdx = nodes[static_cast<size_t>(idx)].leaf;
    const Leaf parent = leaves[static_cast<size_t>(leafIdx)];
    const int c0 = static_cast<int>(nodes.size());
    Node a, b;
    a.leaf = leafIdx;                                  // first child reuses the parent's leaf slot
    b.leaf = static_cast<int>(leaves.size());
    leaves.push_back(parent);
    nodes.push_back(a);
    nodes.push_back(b);
    Node& p = nodes[static_cast<size_t>(idx)];
    p.axis = depth % 3;
    p.child[0] = c0;
    p.child[1] = c0 + 1;
    p.leaf = -1;
}

// One refinement (GuidingField::refine): every leaf's sampling tree becomes its building sums
// (kept when the pass brought none), its next building topology is refined from it, and leaves
// that received more than 512·√(2^k) records are split.
void SdHost::refine(const std::vector<SdQuad>& buildSums, const std::vector<float>& buildSum,
                    const std::vector<uint32_t>& counts) {
    iteration += 1;
    const uint64_t splitThreshold =
        static_cast<uint64_t>(512.0 * std::sqrt(std::pow(2.0, static_cast<double>(std::min(iteration, 16)))));
    bool anyValid = false;
    std::vector<std::pair<int, int>> toSplit;
    auto walk = [&](auto&& self, int idx, int depth) -> void {
        if (idx < 0) return;
        const Node& n = nodes[static_cast<size_t>(idx)];
        if (n.axis < 0) {
            Leaf& L = leaves[static_cast<size_t>(n.leaf)];
            const float newSum = buildSum[static_cast<size_t>(n.leaf)];
            if (newSum > 0.0f) {
                L.samp.assign(buildSums.begin() + L.buildOffset, buildSums.begin() + L.buildOffset + L.build.size());
                L.sampSum = newSum;
                L.build = refineTopology(L.samp, L.sampSum, 0.01f, 10);
            } else {
                if (!(L.sampSum > 0.0f)) {
                    L.samp.assign(1, SdQuad{});
                    L.sampSum = 0.0f;
                }
                L.build.assign(1, SdQuad{});
            }
            if (L.sampSum > 0.0f) anyValid = true;
            if (counts[static_cast<size_t>(n.leaf)] > splitThreshold && depth < 12) toSplit.emplace_back(idx, depth);
            return;
        }
        self(self, n.child[0], depth + 1);
        self(self, n.child[1], depth + 1);
    };
    walk(walk, 0, 0);
    for (const auto& s : toSplit) split(s.first, s.second);
    ready = anyValid;
}

// Flat device copies: spatial nodes, leaves, sampling trees and zeroed building trees.
int32_t SdHost::upload(cudaStream_t s) {
    freeList(bufs);
    std::vector<SdSpatial> sp(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        sp[i].axis = nodes[i].axis;
        sp[i].child[0] = nodes[i].child[0];
        sp[i].child[1] = nodes[i].child[1];
        sp[i].leaf = nodes[i].leaf;
    }
    std::vector<SdLeaf> lv(leaves.size());
    std::vector<SdQuad> samp, build;
    for (size_t i = 0; i < leaves.size(); ++i) {
        Leaf& L = leaves[i];
        const int so = static_cast<int>(samp.size()), bo = static_cast<int>(build.size());
        for (SdQuad q : L.samp) {
            for (int c = 0; c < 4; ++c) q.child[c] = q.child[c] > 0 ? q.child[c] + so : 0;
            samp.push_back(q);
        }
        for (SdQuad q : L.build) {
            for (int c = 0; c < 4; ++c) {
                q.child[c] = q.child[c] > 0 ? q.child[c] + bo : 0;
                q.sums[c] = 0.0f;
            }
            build.push_back(q);
        }
        L.buildOffset = bo;
        lv[i].sampRoot = so;
        lv[i].buildRoot = bo;
        lv[i].sampSum = L.sampSum;
        lv[i].pad = 0;
    }
    SdSpatial* dSp = nullptr;
    SdLeaf* dLv = nullptr;
    SdQuad* dSamp = nullptr;
    SdQuad* dBuild = nullptr;
    float* dSum = nullptr;
    uint32_t* dCnt = nullptr;
    int32_t rc = 0;
    if ((rc = devAlloc(bufs, dSp, sp.size())) || (rc = devAlloc(bufs, dLv, lv.size())) ||
        (rc = devAlloc(bufs, dSamp, samp.size())) || (rc = devAlloc(bufs, dBuild, build.size())) ||
        (rc = devAlloc(bufs, dSum, leaves.size())) || (rc = devAlloc(bufs, dCnt, leaves.size())))
        return rc;
    PE_CUDA(cudaMemcpyAsync(dSp, sp.data(), sp.size() * sizeof(SdSpatial), cudaMemcpyHostToDevice, s));
    PE_CUDA(cudaMemcpyAsync(dLv, lv.data(), lv.size() * sizeof(SdLeaf), cudaMemcpyHostToDevice, s));
    PE_CUDA(cudaMemcpyAsync(dSamp, samp.data(), samp.size() * sizeof(SdQuad), cudaMemcpyHostToDevice, s));
    PE_CUDA(cudaMemcpyAsync(dBuild, build.data(), build.size() * sizeof(SdQuad), cudaMemcpyHostToDevice, s));
    PE_CUDA(cudaMemsetAsync(dSum, 0, leaves.size() * sizeof(float), s));
    PE_CUDA(cudaMemsetAsync(dCnt, 0, leaves.size() * sizeof(uint32_t), s));
    PE_CUDA(cudaStreamSynchronize(s)); // the host vectors above are pageable and local
    buildNodes = build.size();
    SdField& F = field;
    F.spatial = dSp;
    F.leaves = dLv;
    F.samp = dSamp;
    F.build = dBuild;
    F.buildSum = dSum;
    F.sampleCount = dCnt;
    for (int a = 0; a < 3; ++a) {
        F.boxMin[a] = boxMin[a];
        F.boxExt[a] = boxMax[a] - boxMin[a];
    }
    F.ready = ready ? 1 : 0;
    return PE_OK;
}

// Reads back the pass's building sums, refines on the host and uploads the new trees.
int32_t SdHost::refineOnDevice(cudaStream_t s) {
    std::vector<SdQuad> build(buildNodes);
    std::vector<float> sums(leaves.size());
    std::vector<uint32_t> counts(leaves.size());
    PE_CUDA(cudaMemcpyAsync(build.data(), field.build, build.size() * sizeof(SdQuad), cudaMemcpyDeviceToHost, s));
    PE_CUDA(cudaMemcpyAsync(sums.data(), field.buildSum, sums.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
    PE_CUDA(cudaMemcpyAsync(counts.data(), field.sampleCount, counts.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    PE_CUDA(cudaStreamSynchronize(s));
    // building trees were flattened with absolute child indices: make them relative per leaf
    for (const Leaf& L : leaves)
        for (size_t i = 0; i < L.build.size(); ++i) {
            SdQuad& q = build[static_cast<size_t>(L.buildOffset) + i];
            for (int c = 0; c < 4; ++c) q.child[c] = q.child[c] > 0 ? q.child[c] - L.buildOffset : 0;
        }
    refine(build, sums, counts);
    return upload(s);
}

// Splats of a wave's recorded vertices into the building trees.
int32_t sdRecord(pe_device* d, cudaStream_t s, Paths& P, int nSlots) {
    kSdRecord<<<std::max(1, std::min(d->prop.multiProcessorCount * 8, (nSlots + 255) / 256)), 256, 0, s>>>(P, nSlots);
    PE_CUDA(cudaGetLastError());
    return PE_OK;
}

int32_t sdBuffers(pe_device* d) {
    SdHost& H = d->sd;
    Paths& P = d->lanes[0].paths;
    if (H.bufCapacity == d->capacity && P.sdRec) return PE_OK;
    freeList(H.laneBufs);
    int32_t rc = 0;
    if ((rc = devAlloc(H.laneBufs, P.sdRec, d->capacity * kSdRecords * 4)) ||
        (rc = devAlloc(H.laneBufs, P.sdCount, d->capacity))) {
        freeList(H.laneBufs);
        P.sdRec = nullptr;
        P.sdCount = nullptr;
        return rc;
    }
    PE_CUDA(cudaMemsetAsync(P.sdCount, 0, d->capacity * sizeof(uint32_t), d->stream));
    H.bufCapacity = d->capacity;
    return PE_OK;
}

int32_t sdBeginRender(pe_device* d, int first) {
    SdHost& H = d->sd;
    int32_t rc = sdBuffers(d);
    if (rc) return rc;
    const cudaStream_t s = d->lanes[0].stream;
    if (!H.initialised || H.sceneSerial != d->sceneSerial || first == 0) {
        // GuidingField(scene.bounds()); an empty scene gets the box [-1, 1]³
        float lo[3], hi[3];
        const bool empty = d->scene.rootMin[0] > d->scene.rootMax[0];
        for (int a = 0; a < 3; ++a) {
            lo[a] = empty ? -1.0f : d->scene.rootMin[a];
            hi[a] = empty ? 1.0f : d->scene.rootMax[a];
        }
        H.reset(lo, hi);
        if (empty)
            for (int a = 0; a < 3; ++a) {
                H.boxMin[a] = -1.0f;
                H.boxMax[a] = 1.0f;
            }
        H.sceneSerial = d->sceneSerial;
        H.initialised = true;
        if ((rc = H.upload(s))) return rc;
    }
    PE_CUDA(cudaMemsetAsync(d->lanes[0].paths.sdCount, 0, d->capacity * sizeof(uint32_t), s));
    H.waveMode = 0;
    return PE_OK;
}

int sdChunkEnd(pe_device* d, int cur, int end) {
    SdHost& H = d->sd;
    if (H.samplesSeen < 32) {
        H.waveMode = SD_RECORD | (H.ready ? SD_SAMPLE : 0);
        return std::min(end, cur + std::max(1, H.nextRefine - H.samplesSeen));
    }
    H.waveMode = H.ready ? SD_SAMPLE : 0;
    return end;
}

int32_t sdEndChunk(pe_device* d, int samples) {
    SdHost& H = d->sd;
    if (H.samplesSeen >= 32) return PE_OK;
    H.samplesSeen += samples;
    if (H.samplesSeen < H.nextRefine) return PE_OK;
    H.nextRefine = H.nextRefine < 32 ? H.nextRefine * 2 : 64;
    return H.refineOnDevice(d->lanes[0].stream);
}

} // namespace pe_dev

extern "C" {

int32_t pe_device_sdtree_info(pe_device* d, pe_sdtree_info* out) {
    if (!d || !out) {
        setError("pe_device_sdtree_info: null argument");
        return PE_ERR_INVALID;
    }
    std::memset(out, 0, sizeof(*out));
    const SdHost& H = d->sd;
    if (!H.initialised) return PE_OK;
    out->ready = H.ready ? 1 : 0;
    out->refinements = H.iteration;
    out->samples = std::min(H.samplesSeen, 32);
    for (const SdHost::Node& n : H.nodes)
        if (n.axis < 0) ++out->spatial_leaves;
    for (const SdHost::Leaf& L : H.leaves) {
        out->quad_nodes += static_cast<int64_t>(L.samp.size());
        out->energy += L.sampSum;
    }
    return PE_OK;
}

// Host-only check of the quadtree code against the reference's DirectionalTree: splats `n`
// (direction, radiance) pairs in two passes with a refinement in between, as a field leaf sees
// them, then evaluates pdf(dir_i) and sample(u_i) → (direction, pdf) on the final tree.
int32_t pe_sdtree_probe(const float* dirs1, const float* rad1, int32_t n1, const float* dirs2, const float* rad2,
                        int32_t n2, const float* qdirs, const float* qu, int32_t nq, float* pdfOut, float* sampleOut) {
    if ((n1 > 0 && (!dirs1 || !rad1)) || (n2 > 0 && (!dirs2 || !rad2)) || (nq > 0 && (!qdirs || !qu || !pdfOut || !sampleOut))) {
        setError("pe_sdtree_probe: null argument");
        return PE_ERR_INVALID;
    }
    std::vector<SdQuad> samp(1), build(1);
    std::memset(samp.data(), 0, sizeof(SdQuad));
    std::memset(build.data(), 0, sizeof(SdQuad));
    float sampSum = 0.0f;
    auto pass = [&](const float* dirs, const float* rad, int n) {
        float sum = 0.0f;
        for (int i = 0; i < n; ++i) {
            const float r = rad[i];
            if (!(r > 0.0f) || !std::isfinite(r)) continue;
            sum += r;
            V2 p = sdDirToCanonical(mk(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
            int idx = 0;
            for (int depth = 0; depth < 16; ++depth) {
                const int qx = p.x >= 0.5f ? 1 : 0, qy = p.y >= 0.5f ? 1 : 0;
                const int q = qy * 2 + qx;
                build[static_cast<size_t>(idx)].sums[q] += r;
                const int c = build[static_cast<size_t>(idx)].child[q];
                if (c <= 0) break;
                p.x = p.x * 2.0f - static_cast<float>(qx);
                p.y = p.y * 2.0f - static_cast<float>(qy);
                idx = c;
            }
        }
        if (sum > 0.0f) {
            samp = build;
            sampSum = sum;
            build = refineTopology(samp, sampSum, 0.01f, 10);
        } else {
            build.assign(1, SdQuad{});
        }
    };
    pass(dirs1, rad1, n1);
    pass(dirs2, rad2, n2);
    for (int i = 0; i < nq; ++i) {
        const V3 d = mk(qdirs[3 * i], qdirs[3 * i + 1], qdirs[3 * i + 2]);
        pdfOut[i] = sampSum > 0.0f ? sdTreePdf(samp.data(), 0, d) : kSdInvFourPi;
        float pdf = kSdInvFourPi;
        const V2 u = mk2(qu[2 * i], qu[2 * i + 1]);
        const V3 w = sampSum > 0.0f ? sdTreeSample(samp.data(), 0, u, pdf) : sdCanonicalToDir(u);
        sampleOut[4 * i + 0] = w.x;
        sampleOut[4 * i + 1] = w.y;
        sampleOut[4 * i + 2] = w.z;
        sampleOut[4 * i + 3] = pdf;
    }
    return PE_OK;
}

} // extern "C"
