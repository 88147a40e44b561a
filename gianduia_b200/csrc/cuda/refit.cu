// BVH refit on the GPU: a mesh of a resident scene takes new vertex positions (same
// triangle count and order) and its 4-wide tree keeps its topology while every child box
// is recomputed bottom-up, level by level; the instance bounds and the top-level tree are
// refitted the same way. The boxes are the ones the host builder would compute for the
// same topology (bvhBuilder.cpp:59-262 builds them as unions of triangle bounds; the
// top-level boxes are the eight corners of each primitive's object bounds through its
// transform, bvh.cpp:10-36, transform.h:356-363), so only the tree's split choices can
// differ from a fresh build.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "runtime.h"

namespace gnd {

namespace {

struct Box {
    float lo[3], hi[3];
};
__device__ __forceinline__ Box emptyBox() {
    return Box{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
}
__device__ __forceinline__ void growPoint(Box& b, float x, float y, float z) {
    b.lo[0] = fminf(b.lo[0], x); b.lo[1] = fminf(b.lo[1], y); b.lo[2] = fminf(b.lo[2], z);
    b.hi[0] = fmaxf(b.hi[0], x); b.hi[1] = fmaxf(b.hi[1], y); b.hi[2] = fmaxf(b.hi[2], z);
}
__device__ __forceinline__ void growBox(Box& b, const Box& o) {
    for (int a = 0; a < 3; ++a) { b.lo[a] = fminf(b.lo[a], o.lo[a]); b.hi[a] = fmaxf(b.hi[a], o.hi[a]); }
}
// Union of a node's non-empty child boxes
__device__ __forceinline__ Box nodeBox(const Node4& n) {
    Box b = emptyBox();
    for (int k = 0; k < 4; ++k)
        if (n.child[k] != kEmpty)
            growBox(b, Box{{n.lox[k], n.loy[k], n.loz[k]}, {n.hix[k], n.hiy[k], n.hiz[k]}});
    return b;
}

// New positions (object space, original triangle order, 9 floats each) into the
// leaf-ordered triangle records of the mesh.
__global__ void kRefitTris(const float* __restrict__ pos, int64_t n, const uint32_t* __restrict__ origToLeaf, Tri* tris) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float* p = pos + 9 * i;
        Tri& t = tris[origToLeaf[i]];
        t.v0x = p[0]; t.v0y = p[1]; t.v0z = p[2];
        t.v1x = p[3]; t.v1y = p[4]; t.v1z = p[5];
        t.v2x = p[6]; t.v2y = p[7]; t.v2z = p[8];
    }
}

// One breadth-first step: the inner children of the nodes in `cur` are appended to `next`.
__global__ void kExpandLevel(const Node4* __restrict__ nodes, const uint32_t* __restrict__ cur, uint32_t count,
                             uint32_t* next, uint32_t* nextCount, uint32_t capacity, uint32_t* overflow) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const Node4& nd = nodes[cur[i]];
        for (int k = 0; k < 4; ++k) {
            const uint32_t c = nd.child[k];
            if (c == kEmpty || isLeaf(c)) continue;
            const uint32_t at = atomicAdd(nextCount, 1u);
            if (at < capacity) next[at] = c;
            else atomicOr(overflow, 1u);
        }
    }
}

// Child boxes of the nodes of one level, from the level below (inner children) or from
// the leaf items: triangles (bottom level) or instance world bounds (top level).
__global__ void kRefitLevel(Node4* nodes, const uint32_t* __restrict__ list, uint32_t count, const Tri* __restrict__ tris,
                            const Box* __restrict__ instBounds, const uint32_t* __restrict__ tlasList) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        Node4& nd = nodes[list[i]];
        for (int k = 0; k < 4; ++k) {
            const uint32_t c = nd.child[k];
            if (c == kEmpty) continue;
            Box b = emptyBox();
            if (!isLeaf(c)) {
                b = nodeBox(nodes[c]);
            } else {
                const uint32_t first = leafFirst(c), cnt = leafCount(c);
                for (uint32_t j = 0; j < cnt; ++j) {
                    if (tris) {
                        const Tri& t = tris[first + j];
                        growPoint(b, t.v0x, t.v0y, t.v0z);
                        growPoint(b, t.v1x, t.v1y, t.v1z);
                        growPoint(b, t.v2x, t.v2y, t.v2z);
                    } else {
                        growBox(b, instBounds[tlasList[first + j]]);
                    }
                }
            }
            nd.lox[k] = b.lo[0]; nd.loy[k] = b.lo[1]; nd.loz[k] = b.lo[2];
            nd.hix[k] = b.hi[0]; nd.hiy[k] = b.hi[1]; nd.hiz[k] = b.hi[2];
        }
    }
}

// World bounds of every (static) instance: its object bounds (the mesh tree's root box,
// the sphere's radius, the cube's extents) with the eight corners through object-to-world
// in the order of Bounds::transformed.
__global__ void kInstanceBounds(const Node4* __restrict__ nodes, const InstTrav* __restrict__ it,
                                const InstShade* __restrict__ is, int n, Box* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t kind = it[i].kind & ~kInstAnimated;
        Box ob;
        if (kind == kShapeMesh) {
            ob = it[i].blasRoot == kEmpty ? emptyBox() : nodeBox(nodes[it[i].blasRoot]);
        } else if (kind == kShapeSphere) {
            const float r = is[i].radius;
            ob = Box{{-r, -r, -r}, {r, r, r}};
        } else {
            ob = Box{{-is[i].ext[0], -is[i].ext[1], -is[i].ext[2]}, {is[i].ext[0], is[i].ext[1], is[i].ext[2]}};
        }
        Box w = emptyBox();
        for (int c = 0; c < 8; ++c) {
            const V3 p = xfPoint(is[i].o2w, v3((c & 1) ? ob.hi[0] : ob.lo[0], (c & 2) ? ob.hi[1] : ob.lo[1],
                                              (c & 4) ? ob.hi[2] : ob.lo[2]));
            if (c == 0) w = Box{{p.x, p.y, p.z}, {p.x, p.y, p.z}};
            else growPoint(w, p.x, p.y, p.z);
        }
        out[i] = w;
    }
}

unsigned gridFor(int64_t n, int numSMs) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)numSMs * 8));
}

}  // namespace

// Levels of the tree under `root` (cached per scene): node indices level by level.
const RefitTopo& refitTopology(Context* c, DeviceScene& ds, uint32_t root) {
    auto it = ds.refitTopo.find(root);
    if (it != ds.refitTopo.end()) return it->second;
    RefitTopo t;
    const uint32_t cap = (uint32_t)std::max<int64_t>(ds.numNodes, 1);
    t.list = PoolBuf((size_t)cap * sizeof(uint32_t), c->stream);
    PoolBuf counters(16, c->stream);
    uint32_t* list = t.list.as<uint32_t>();
    GND_CUDA(cudaMemcpyAsync(list, &root, 4, cudaMemcpyHostToDevice, c->stream));
    t.offsets = {0, 1};
    while (true) {
        const uint32_t begin = (uint32_t)t.offsets[t.offsets.size() - 2], end = (uint32_t)t.offsets.back();
        GND_CUDA(cudaMemsetAsync(counters.ptr, 0, 16, c->stream));
        kExpandLevel<<<gridFor(end - begin, c->numSMs), 256, 0, c->stream>>>(ds.view.nodes, list + begin, end - begin, list + end,
                                                                            counters.as<uint32_t>(), cap - end,
                                                                            counters.as<uint32_t>() + 1);
        GND_CUDA(cudaGetLastError());
        uint32_t h[2];
        GND_CUDA(cudaMemcpyAsync(h, counters.ptr, 8, cudaMemcpyDeviceToHost, c->stream));
        GND_CUDA(cudaStreamSynchronize(c->stream));
        if (h[1] || h[0] > cap - end) throw Error(GND_ERR_INVALID, "refit: the tree reaches more nodes than the scene holds");
        if (h[0] == 0) break;
        t.offsets.push_back(end + h[0]);
    }
    return ds.refitTopo.emplace(root, std::move(t)).first->second;
}

}  // namespace gnd

using namespace gnd;

extern "C" {

gnd_status gnd_gpu_scene_refit_mesh(gnd_gpu_ctx* ctxh, gnd_scene_id id, int32_t mesh, const float* positions,
                                    int64_t num_tris, float* device_ms) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!positions && num_tris > 0) throw Error(GND_ERR_INVALID, "refit: null positions");
        for (int64_t i = 0; i < 9 * num_tris; ++i)
            if (!std::isfinite(positions[i])) throw Error(GND_ERR_INVALID, "refit: positions must be finite");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        DeviceScene& ds = c->scene(id);
        const SceneView& v = ds.view;
        // Renders hold the context lock and run on its stream, so they finish before the
        // refit starts; a served job may still be queued or running, and would see the
        // geometry change between its rounds.
        auto use = c->sceneUse.find(id);
        if (use != c->sceneUse.end() && use->second > 0)
            throw Error(GND_ERR_INVALID, "refit: the scene is used by queued or running jobs");
        if (mesh < 0 || mesh >= ds.numMeshes) throw Error(GND_ERR_INVALID, "refit: mesh index out of range");
        if (v.motion) throw Error(GND_ERR_INVALID, "refit: scenes with moving instances are not refitted");
        MeshRec rec;
        std::vector<InstTrav> it(std::max(ds.numInstances, 1));
        std::vector<InstShade> is(std::max(ds.numInstances, 1));
        GND_CUDA(cudaMemcpyAsync(&rec, v.meshes + mesh, sizeof(MeshRec), cudaMemcpyDeviceToHost, c->stream));
        if (ds.numInstances) {
            GND_CUDA(cudaMemcpyAsync(it.data(), v.instT, sizeof(InstTrav) * ds.numInstances, cudaMemcpyDeviceToHost, c->stream));
            GND_CUDA(cudaMemcpyAsync(is.data(), v.instS, sizeof(InstShade) * ds.numInstances, cudaMemcpyDeviceToHost, c->stream));
        }
        GND_CUDA(cudaStreamSynchronize(c->stream));
        if ((int64_t)rec.numTris != num_tris)
            throw Error(GND_ERR_INVALID, "refit: the mesh has " + std::to_string(rec.numTris) + " triangles, not " +
                                             std::to_string(num_tris));
        if (num_tris == 0) return;
        if ((int64_t)rec.origToLeaf + num_tris > ds.origToLeafLen) throw Error(GND_ERR_INVALID, "refit: bad mesh record");
        uint32_t root = kEmpty;
        for (int i = 0; i < ds.numInstances; ++i) {
            if ((it[i].kind & ~kInstAnimated) != kShapeMesh || is[i].meshId != (uint32_t)mesh) continue;
            if (is[i].emitter >= 0) throw Error(GND_ERR_INVALID, "refit: the mesh carries an area light (its sampling tables would change)");
            root = it[i].blasRoot;
        }
        if (root == kEmpty) throw Error(GND_ERR_INVALID, "refit: no primitive uses the mesh");
        const RefitTopo& blas = refitTopology(c, ds, root);
        const RefitTopo* tlas = v.tlasRoot != kEmpty ? &refitTopology(c, ds, v.tlasRoot) : nullptr;
        PoolBuf pos((size_t)num_tris * 9 * sizeof(float), c->stream);
        PoolBuf inst((size_t)std::max(ds.numInstances, 1) * sizeof(Box), c->stream);
        GND_CUDA(cudaMemcpyAsync(pos.ptr, positions, pos.bytes, cudaMemcpyHostToDevice, c->stream));
        // timing events, destroyed on every exit (a failing launch throws)
        struct Events {
            cudaEvent_t e[2] = {nullptr, nullptr};
            ~Events() {
                for (cudaEvent_t x : e)
                    if (x) cudaEventDestroy(x);
            }
        } ev;
        GND_CUDA(cudaEventCreate(&ev.e[0]));
        GND_CUDA(cudaEventCreate(&ev.e[1]));
        cudaEvent_t e0 = ev.e[0], e1 = ev.e[1];
        GND_CUDA(cudaEventRecord(e0, c->stream));
        Node4* nodes = const_cast<Node4*>(v.nodes);
        kRefitTris<<<gridFor(num_tris, c->numSMs), 256, 0, c->stream>>>(pos.as<float>(), num_tris, v.origToLeaf + rec.origToLeaf,
                                                                        const_cast<Tri*>(v.tris));
        auto refitLevels = [&](const RefitTopo& t, const Tri* tris, const Box* ib) {
            for (size_t l = t.offsets.size() - 1; l-- > 0;) {
                const uint32_t b = (uint32_t)t.offsets[l], n = (uint32_t)(t.offsets[l + 1] - t.offsets[l]);
                kRefitLevel<<<gridFor(n, c->numSMs), 256, 0, c->stream>>>(nodes, t.list.as<uint32_t>() + b, n, tris, ib, v.tlasList);
            }
        };
        refitLevels(blas, v.tris, nullptr);
        if (tlas) {
            kInstanceBounds<<<gridFor(ds.numInstances, c->numSMs), 256, 0, c->stream>>>(v.nodes, v.instT, v.instS, ds.numInstances,
                                                                                     inst.as<Box>());
            refitLevels(*tlas, nullptr, inst.as<Box>());
        }
        GND_CUDA(cudaGetLastError());
        GND_CUDA(cudaEventRecord(e1, c->stream));
        GND_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (device_ms) *device_ms = ms;
    });
}

}  // extern "C"
