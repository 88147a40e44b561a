// Contexts and resident scenes: gnd_gpu_create/destroy, gnd_gpu_scene_upload/free.
#include <cmath>
#include <cstring>

#include "bvhbuild.h"
#include "runtime.h"
#include "server.h"
#include "wavefront.h"

namespace gnd {

namespace {
thread_local std::string t_lastError = "no error";
}
void setLastError(const std::string& m) { t_lastError = m; }
const std::string& lastError() { return t_lastError; }

Context::~Context() {
    if (device >= 0) cudaSetDevice(device);
    server.reset();   // joins the serving thread before the engine goes away
    wave.reset();
    scenes.clear();
    if (stream) cudaStreamSynchronize(stream);
    if (uploadStream) cudaStreamSynchronize(uploadStream);
    cudaMemPool_t pool = nullptr;
    if (device >= 0 && cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    errWord.release();
    rayScratch.release();
    hitScratch.release();
    if (stream) cudaStreamDestroy(stream);
    if (uploadStream) cudaStreamDestroy(uploadStream);
}

void Context::checkKernelErrors(const char* what) {
    uint32_t w = 0;
    GND_CUDA(cudaMemcpyAsync(&w, errWord.ptr, 4, cudaMemcpyDeviceToHost, stream));
    GND_CUDA(cudaStreamSynchronize(stream));
    if (w) {
        GND_CUDA(cudaMemsetAsync(errWord.ptr, 0, 4, stream));
        std::string m = std::string(what) + ": device check failed (";
        if (w & 1) m += " traversal-stack-overflow";
        if (w & 2) m += " traversal-iteration-limit";
        if (w & 4) m += " bad-node-reference";
        if (w & 8) m += " path-queue-overflow";
        if (w & 16) m += " path-iteration-limit";
        m += " )";
        throw Error(GND_ERR_DEVICE_CHECK, m);
    }
}

// Texture trees of a scene description: every slot's node, every node's children and
// texels in range, and warps nested inside warp inputs at most kTexWarpNesting deep (the
// depth the kernels evaluate).
namespace {
int warpNesting(const TexNode* nodes, int64_t n, int64_t node, int depth) {
    if (depth > kTexWarpNesting) return depth;
    int need = 0;
    for (int64_t hop = 0; hop <= n; ++hop) {
        const TexNode& t = nodes[node];
        if (t.kind != kTnWarp) return need;
        need = std::max(need, 1 + warpNesting(nodes, n, t.b, depth + 1));
        node = t.a;
    }
    throw Error(GND_ERR_INVALID, "texture tree has a cycle");
}
void validateTextures(const gnd_scene_desc* d) {
    const int64_t n = d->num_tex_nodes;
    if (n < 0 || d->num_tex_texels < 0 || (n > 0 && !d->tex_nodes) || (d->num_tex_texels > 0 && !d->tex_texels))
        throw Error(GND_ERR_INVALID, "bad texture arrays");
    auto slot = [&](const ColorTex& t) {
        if (t.kind > kTexNode) throw Error(GND_ERR_INVALID, "unknown color texture kind");
        if (t.kind == kTexNode && (int64_t)t.node >= n) throw Error(GND_ERR_INVALID, "texture node out of range");
    };
    const Material* mats = reinterpret_cast<const Material*>(d->materials);
    for (int m = 0; m < d->num_materials; ++m) {
        slot(mats[m].a);
        slot(mats[m].b);
        for (uint32_t r : {mats[m].roughTex, mats[m].etaTex, mats[m].kTex, mats[m].normalTex, mats[m].bumpTex})
            if ((int64_t)r > n) throw Error(GND_ERR_INVALID, "material texture node out of range");
    }
    const Emitter* ems = reinterpret_cast<const Emitter*>(d->emitters);
    for (int k = 0; k < d->num_emitters; ++k) slot(ems[k].radiance);
    const TexNode* nodes = reinterpret_cast<const TexNode*>(d->tex_nodes);
    for (int64_t i = 0; i < n; ++i) {
        const TexNode& t = nodes[i];
        if (t.kind < kTnConstant || t.kind > kTnWarp) throw Error(GND_ERR_INVALID, "unknown texture node kind");
        if (t.kind == kTnWarp && (t.a < 0 || t.a >= n || t.b < 0 || t.b >= n)) throw Error(GND_ERR_INVALID, "warp input out of range");
        if (t.kind == kTnImage && (t.w <= 0 || t.h <= 0 || t.a < 0 || (int64_t)t.a + (int64_t)t.w * t.h > d->num_tex_texels))
            throw Error(GND_ERR_INVALID, "image texels out of range");
        if (t.kind == kTnCellular && ((t.flags >> kTnMetricShift) & 3) > 2) throw Error(GND_ERR_INVALID, "unknown cellular metric");
        // beyond ~128 octaves p * 2^i is infinite and every further octave adds NaN; the
        // bound keeps a shading thread's work finite
        if ((t.kind == kTnPerlin || t.kind == kTnMarble || t.kind == kTnWood) && t.octaves > kTexMaxOctaves)
            throw Error(GND_ERR_INVALID, "texture octaves above " + std::to_string(kTexMaxOctaves));
    }
    for (int64_t i = 0; i < n; ++i)
        if (nodes[i].kind == kTnWarp && warpNesting(nodes, n, i, 0) > kTexWarpNesting)
            throw Error(GND_ERR_INVALID, "warps nested in warp inputs deeper than supported");
}
}  // namespace

Context* ctxOf(gnd_gpu_ctx* c) {
    if (!c) throw Error(GND_ERR_INVALID, "null context");
    return reinterpret_cast<Context*>(c);
}

namespace {
constexpr uint32_t kNodeBadRef = 1u, kNodeBadLeaf = 2u, kNodeSlowBounds = 4u;

// Checks every node of an uploaded tree: inner references below n, leaf ranges below
// leafLimit (triangles or top-level entries), and whether the bounds allow the fast slab
// test (no NaN, lo <= hi on every non-empty child).
__global__ void kValidateNodes(const Node4* __restrict__ nodes, int64_t n, int64_t leafLimit, uint32_t* flags) {
    uint32_t f = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Node4& nd = nodes[i];
        for (int k = 0; k < 4; ++k) {
            const float lo[3] = {nd.lox[k], nd.loy[k], nd.loz[k]};
            const float hi[3] = {nd.hix[k], nd.hiy[k], nd.hiz[k]};
            const uint32_t r = nd.child[k];
            for (int a = 0; a < 3; ++a) {
                if (isnan(lo[a]) || isnan(hi[a])) f |= kNodeSlowBounds;
                if (r != kEmpty && !(lo[a] <= hi[a])) f |= kNodeSlowBounds;
            }
            if (r == kEmpty) continue;
            if (!isLeaf(r)) {
                if ((int64_t)r >= n) f |= kNodeBadRef;
            } else if ((int64_t)(leafFirst(r) + leafCount(r)) > leafLimit) {
                f |= kNodeBadLeaf;
            }
        }
    }
    f = __reduce_or_sync(0xffffffffu, f);
    if (f && (threadIdx.x & 31) == 0) atomicOr(flags, f);
}

template <typename T>
const T* upload(DeviceScene& ds, cudaStream_t st, const void* src, size_t count) {
    size_t bytes = count * sizeof(T);
    ds.bufs.emplace_back(bytes > 0 ? bytes : 16, st);
    if (bytes) GND_CUDA(cudaMemcpyAsync(ds.bufs.back().ptr, src, bytes, cudaMemcpyHostToDevice, st));
    ds.bytes += ds.bufs.back().bytes;
    return ds.bufs.back().as<T>();
}
}  // namespace

}  // namespace gnd

using namespace gnd;

extern "C" {

const char* gnd_last_error(void) { return lastError().c_str(); }
const char* gnd_version(void) { return "gianduia_b200 1.0 (sm_100a)"; }

gnd_status gnd_gpu_create(int device, gnd_gpu_ctx** out) {
    return guarded([&]() {
        if (!out) throw Error(GND_ERR_INVALID, "null output pointer");
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0)
            throw Error(GND_ERR_NO_DEVICE, std::string("no CUDA device available: ") + cudaGetErrorString(e));
        if (device < 0 || device >= n) throw Error(GND_ERR_INVALID, "device ordinal out of range");
        auto c = std::make_unique<Context>();
        c->device = device;
        c->bind();
        cudaDeviceProp prop;
        GND_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10)
            throw Error(GND_ERR_NO_DEVICE, std::string("device ") + prop.name + " is not sm_100 (this build targets sm_100a)");
        c->numSMs = prop.multiProcessorCount;
        GND_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        GND_CUDA(cudaStreamCreateWithFlags(&c->uploadStream, cudaStreamNonBlocking));
        // scene arrays come from the default memory pool; keep freed memory in the pool
        // (a process-local setting) so that scene uploads reuse it
        cudaMemPool_t pool = nullptr;
        GND_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = UINT64_MAX;
        GND_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        c->errWord.alloc(16);
        GND_CUDA(cudaMemset(c->errWord.ptr, 0, 16));
        c->traceTotals.alloc(kTraceTotals * sizeof(unsigned long long));
        GND_CUDA(cudaMemset(c->traceTotals.ptr, 0, kTraceTotals * sizeof(unsigned long long)));
        *out = reinterpret_cast<gnd_gpu_ctx*>(c.release());
    });
}

gnd_status gnd_gpu_destroy(gnd_gpu_ctx* ctx) {
    return guarded([&]() { delete ctxOf(ctx); });
}

gnd_status gnd_gpu_counters(gnd_gpu_ctx* ctxh, gnd_counters* out, int32_t reset) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!out) throw Error(GND_ERR_INVALID, "null output pointer");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        // batches may have been queued on the caller's streams: wait for all of them
        GND_CUDA(cudaDeviceSynchronize());
        unsigned long long t[kTraceTotals];
        GND_CUDA(cudaMemcpy(t, c->traceTotals.ptr, sizeof(t), cudaMemcpyDeviceToHost));
        gnd_counters r = c->counters;
        r.trace_rays = (int64_t)t[kTraceTotalRays];
        r.counted_rays = (int64_t)t[kTraceTotalCountedRays];
        r.counted_nodes = (int64_t)t[kTraceTotalNodes];
        r.counted_tris = (int64_t)t[kTraceTotalTris];
        *out = r;
        if (reset) {
            GND_CUDA(cudaMemset(c->traceTotals.ptr, 0, sizeof(t)));
            const gnd_render_stats last = c->counters.last;
            c->counters = gnd_counters{};
            c->counters.last = last;
        }
    });
}

gnd_status gnd_gpu_scene_upload(gnd_gpu_ctx* ctxh, const gnd_scene_desc* d, gnd_scene_id* out) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!d || !out) throw Error(GND_ERR_INVALID, "null scene description");
        if (d->num_instances < 0 || d->num_nodes < 0 || d->num_tris < 0) throw Error(GND_ERR_INVALID, "negative sizes");
        if (d->num_tris >= (int64_t)kLeafFirstMask) throw Error(GND_ERR_INVALID, "too many triangles");
        // host-side validation of every reference stored in the tree (a corrupted index
        // is refused here rather than read out of bounds on the device)
        // The node references and bounds are checked on the device after the upload
        // (kValidateNodes), before any kernel follows them.
        const Node4* nodes = reinterpret_cast<const Node4*>(d->nodes);
        if (d->num_nodes > 0 && !nodes) throw Error(GND_ERR_INVALID, "null node array");
        bool nanBounds = false;   // true: the traversal keeps the exact slab arithmetic
        if (d->tlas_root != kEmpty && (int64_t)d->tlas_root >= d->num_nodes) throw Error(GND_ERR_INVALID, "bad top-level root");
        // mesh trees built here: the mesh records must tile the triangles in order
        const bool deviceBlas = d->blas_on_device != 0;
        std::vector<uint32_t> meshBase;
        if (deviceBlas) {
            if (d->num_meshes < 0 || (d->num_meshes > 0 && !d->meshes)) throw Error(GND_ERR_INVALID, "device tree build needs the mesh records");
            if (d->orig_to_leaf_len != d->num_tris) throw Error(GND_ERR_INVALID, "device tree build: orig_to_leaf must have one entry per triangle");
            const MeshRec* mr = reinterpret_cast<const MeshRec*>(d->meshes);
            meshBase.resize((size_t)d->num_meshes + 1, 0);
            for (int m = 0; m < d->num_meshes; ++m) {
                if (mr[m].origToLeaf != meshBase[m]) throw Error(GND_ERR_INVALID, "device tree build: meshes are not contiguous in triangle order");
                meshBase[m + 1] = meshBase[m] + mr[m].numTris;
            }
            if ((int64_t)meshBase.back() != d->num_tris) throw Error(GND_ERR_INVALID, "device tree build: mesh triangle counts do not add up");
        }
        for (int64_t i = 0; i < d->tlas_list_len; ++i)
            if ((int64_t)d->tlas_list[i] >= d->num_instances) throw Error(GND_ERR_INVALID, "instance list out of range");
        const InstTrav* it = reinterpret_cast<const InstTrav*>(d->inst_trav);
        const InstShade* is = reinterpret_cast<const InstShade*>(d->inst_shade);
        for (int i = 0; i < d->num_instances; ++i) {
            const uint32_t kind = it[i].kind & ~kInstAnimated;
            if (!deviceBlas && kind == kShapeMesh && it[i].blasRoot != kEmpty && (int64_t)it[i].blasRoot >= d->num_nodes)
                throw Error(GND_ERR_INVALID, "instance root out of range");
            if (deviceBlas && kind == kShapeMesh && (int64_t)is[i].meshId >= d->num_meshes)
                throw Error(GND_ERR_INVALID, "instance mesh out of range");
            if (is[i].material < 0 || is[i].material >= d->num_materials) throw Error(GND_ERR_INVALID, "instance material out of range");
            if (is[i].emitter >= d->num_emitters) throw Error(GND_ERR_INVALID, "instance emitter out of range");
            if ((it[i].kind & kInstAnimated) && !d->inst_motion) throw Error(GND_ERR_INVALID, "animated instance without motion records");
            if ((it[i].kind & ~kInstAnimated) > kShapeCube) throw Error(GND_ERR_INVALID, "unknown shape kind");
            if (is[i].emitter >= 0 && reinterpret_cast<const Emitter*>(d->emitters)[is[i].emitter].type != kEmitArea)
                throw Error(GND_ERR_INVALID, "instance emitter is not an area light");
            if (is[i].mediumIn >= d->num_media || is[i].mediumOut >= d->num_media) throw Error(GND_ERR_INVALID, "instance medium out of range");
        }
        const Emitter* ems = reinterpret_cast<const Emitter*>(d->emitters);
        for (int k = 0; k < d->num_emitters; ++k) {
            if (ems[k].type < kEmitArea || ems[k].type > kEmitEnv) throw Error(GND_ERR_INVALID, "unknown emitter type");
            if (ems[k].type == kEmitArea && (ems[k].instance < 0 || ems[k].instance >= d->num_instances))
                throw Error(GND_ERR_INVALID, "area emitter instance out of range");
            if (ems[k].type == kEmitEnv && k != d->env_emitter) throw Error(GND_ERR_INVALID, "environment emitter without its map");
        }
        validateTextures(d);
        c->bind();
        // the copies, the tree build and the validation run on the upload stream without
        // the context lock (a render may be running); the lock publishes the scene
        std::lock_guard<std::mutex> ul(c->uploadMu);
        cudaStream_t st = c->uploadStream;
        auto ds = std::make_unique<DeviceScene>();
        SceneView& v = ds->view;
        PoolBuf rawTris, rawAttrs;   // original order, for the device tree build
        if (!deviceBlas) {
            v.nodes = upload<Node4>(*ds, st, d->nodes, d->num_nodes);
            v.tris = upload<Tri>(*ds, st, d->tris, d->num_tris);
            v.attrs = upload<TriAttr>(*ds, st, d->tri_attrs, d->num_tris);
        } else {
            rawTris = PoolBuf(std::max<size_t>((size_t)d->num_tris * sizeof(Tri), 16), st);
            rawAttrs = PoolBuf(std::max<size_t>((size_t)d->num_tris * sizeof(TriAttr), 16), st);
            if (d->num_tris) {
                GND_CUDA(cudaMemcpyAsync(rawTris.ptr, d->tris, (size_t)d->num_tris * sizeof(Tri), cudaMemcpyHostToDevice, st));
                GND_CUDA(cudaMemcpyAsync(rawAttrs.ptr, d->tri_attrs, (size_t)d->num_tris * sizeof(TriAttr), cudaMemcpyHostToDevice, st));
            }
        }
        v.instT = upload<InstTrav>(*ds, st, d->inst_trav, d->num_instances);
        v.instS = upload<InstShade>(*ds, st, d->inst_shade, d->num_instances);
        v.tlasList = upload<uint32_t>(*ds, st, d->tlas_list, d->tlas_list_len);
        v.materials = upload<Material>(*ds, st, d->materials, d->num_materials);
        v.emitters = upload<Emitter>(*ds, st, d->emitters, d->num_emitters);
        v.media = upload<Medium>(*ds, st, d->media, d->num_media);
        v.meshes = upload<MeshRec>(*ds, st, d->meshes, d->num_meshes);
        v.cdf = upload<float>(*ds, st, d->cdf, d->cdf_len);
        v.origToLeaf = upload<uint32_t>(*ds, st, d->orig_to_leaf, d->orig_to_leaf_len);
        v.motion = d->inst_motion ? upload<InstMotion>(*ds, st, d->inst_motion, d->num_instances) : nullptr;
        v.texNodes = upload<TexNode>(*ds, st, d->tex_nodes, d->num_tex_nodes);
        v.texels = upload<float>(*ds, st, d->tex_texels, (size_t)d->num_tex_texels * 4);
        v.numTexNodes = d->num_tex_nodes;
        // environment map (texels + the sampling tables of distribution.cpp)
        v.env = EnvView{};
        v.env.emitter = -1;
        if (d->env_emitter >= 0) {
            const int64_t w = d->env_width, h = d->env_height;
            const Emitter* ems = reinterpret_cast<const Emitter*>(d->emitters);
            if (d->env_emitter >= d->num_emitters || ems[d->env_emitter].type != kEmitEnv || w <= 0 || h <= 0 ||
                w * h > ((int64_t)1 << 28) || !d->env_texels || !d->env_dist)
                throw Error(GND_ERR_INVALID, "bad environment map description");
            v.env.texels = upload<float>(*ds, st, d->env_texels, (size_t)(w * h * 3));
            const float* dist = upload<float>(*ds, st, d->env_dist, (size_t)(h + (h + 1) + h * w + h * (w + 1) + h));
            v.env.margFunc = dist;
            v.env.margCdf = dist + h;
            v.env.condFunc = dist + h + (h + 1);
            v.env.condCdf = v.env.condFunc + h * w;
            v.env.condInt = v.env.condCdf + h * (w + 1);
            v.env.width = (int32_t)w;
            v.env.height = (int32_t)h;
            v.env.margInt = d->env_marginal_integral;
            v.env.strength = d->env_strength;
            v.env.emitter = d->env_emitter;
        }
        v.tlasRoot = d->tlas_root;
        // the ray-reordering grid: the union of the top-level root's child boxes (the
        // scene's bounds; unit cube for an empty or non-finite scene)
        {
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            if (d->tlas_root != kEmpty && nodes) {
                const Node4& r = nodes[d->tlas_root];
                for (int k = 0; k < 4; ++k) {
                    if (r.child[k] == kEmpty) continue;
                    const float l[3] = {r.lox[k], r.loy[k], r.loz[k]}, h[3] = {r.hix[k], r.hiy[k], r.hiz[k]};
                    for (int a = 0; a < 3; ++a) {
                        lo[a] = std::min(lo[a], l[a]);
                        hi[a] = std::max(hi[a], h[a]);
                    }
                }
            }
            for (int a = 0; a < 3; ++a) {
                if (!(std::isfinite(lo[a]) && std::isfinite(hi[a]) && hi[a] >= lo[a])) { lo[a] = 0.0f; hi[a] = 1.0f; }
                v.keyLo[a] = lo[a];
                v.keyScale[a] = 8.0f / std::max(hi[a] - lo[a], 1e-6f);
            }
        }
        v.numEmitters = d->num_emitters;
        v.numInstances = d->num_instances;
        ds->numNodes = d->num_nodes;
        if (deviceBlas) {
            MeshTreeInput mi{};
            mi.tlasNodes = nodes;
            mi.numTlasNodes = (uint32_t)d->num_nodes;
            mi.meshBase = meshBase.data();
            mi.numMeshes = d->num_meshes;
            mi.tris = rawTris.as<Tri>();
            mi.attrs = rawAttrs.as<TriAttr>();
            mi.numTris = d->num_tris;
            mi.instT = const_cast<InstTrav*>(v.instT);
            mi.instS = v.instS;
            mi.numInstances = d->num_instances;
            mi.origToLeaf = const_cast<uint32_t*>(v.origToLeaf);
            mi.leafMax = c->buildLeafMax;
            mi.numSMs = c->numSMs;
            MeshTreeOutput mo = buildMeshTrees(mi, st);
            nanBounds |= mo.nonFinite;
            ds->numNodes = mo.numNodes;
            ds->buildMs = mo.ms;
            ds->blasOnDevice = true;
            for (PoolBuf* b : {&mo.nodes, &mo.tris, &mo.attrs}) {
                ds->bytes += b->bytes;
                ds->bufs.push_back(std::move(*b));
            }
            v.nodes = ds->bufs[ds->bufs.size() - 3].as<Node4>();
            v.tris = ds->bufs[ds->bufs.size() - 2].as<Tri>();
            v.attrs = ds->bufs[ds->bufs.size() - 1].as<TriAttr>();
        }
        ds->numTris = d->num_tris;
        ds->origToLeafLen = d->orig_to_leaf_len;
        ds->numInstances = d->num_instances;
        ds->numMeshes = d->num_meshes;
        // every node reference in range; bounds fit for the fast slab test
        PoolBuf vflags(16, st);
        GND_CUDA(cudaMemsetAsync(vflags.ptr, 0, 16, st));
        if (ds->numNodes > 0) {
            const unsigned grid = (unsigned)std::min<int64_t>((ds->numNodes + 255) / 256, (int64_t)c->numSMs * 8);
            kValidateNodes<<<grid, 256, 0, st>>>(v.nodes, ds->numNodes, std::max<int64_t>(d->num_tris, d->tlas_list_len),
                                                        vflags.as<uint32_t>());
            GND_CUDA(cudaGetLastError());
        }
        uint32_t vf = 0;
        GND_CUDA(cudaMemcpyAsync(&vf, vflags.ptr, 4, cudaMemcpyDeviceToHost, st));
        GND_CUDA(cudaStreamSynchronize(st));
        if (vf & kNodeBadRef) throw Error(GND_ERR_INVALID, "node reference out of range");
        if (vf & kNodeBadLeaf) throw Error(GND_ERR_INVALID, "leaf range out of range");
        nanBounds |= (vf & kNodeSlowBounds) != 0;
        v.fastBoxes = nanBounds ? 0 : 1;
        if (d->camera) std::memcpy(&v.camera, d->camera, sizeof(Camera));
        // the rarer features select the kernels' EXT variants
        bool ext = v.motion != nullptr || v.env.emitter >= 0 || v.camera.kind == kCamThinLens || v.camera.animated != 0 ||
                   d->num_tex_nodes > 0;
        for (int k = 0; k < d->num_emitters; ++k) ext = ext || ems[k].type != kEmitArea;
        v.ext = ext ? 1 : 0;
        // null-BSDF mask and material type per instance
        std::vector<uint8_t> mask(std::max(1, d->num_instances), 0), cls(std::max(1, d->num_instances), kMatIndex);
        const Material* mats = reinterpret_cast<const Material*>(d->materials);
        for (int i = 0; i < d->num_instances; ++i) {
            const uint32_t t = mats[is[i].material].type;
            cls[i] = (uint8_t)(t < kMatIndex ? t : kMatIndex);
            if (t == kMatIndex) { mask[i] = 1; ds->hasNullMaterials = true; }
        }
        ds->nullMask.alloc(mask.size());
        GND_CUDA(cudaMemcpyAsync(ds->nullMask.ptr, mask.data(), mask.size(), cudaMemcpyHostToDevice, st));
        ds->instClass.alloc(cls.size());
        GND_CUDA(cudaMemcpyAsync(ds->instClass.ptr, cls.data(), cls.size(), cudaMemcpyHostToDevice, st));
        v.instClass = ds->instClass.as<uint8_t>();
        ds->viewDev.alloc(sizeof(SceneView));
        GND_CUDA(cudaMemcpyAsync(ds->viewDev.ptr, &v, sizeof(SceneView), cudaMemcpyHostToDevice, st));
        GND_CUDA(cudaStreamSynchronize(st));
        ds->bytes += ds->nullMask.bytes + ds->instClass.bytes + ds->viewDev.bytes;
        ds->width = d->width; ds->height = d->height; ds->spp = d->spp; ds->maxDepth = d->max_depth;
        ds->integrator = d->integrator; ds->filter = d->filter;
        ds->filterRadius[0] = d->filter_radius[0]; ds->filterRadius[1] = d->filter_radius[1];
        ds->filterAlpha = d->filter_alpha;
        ds->numMaterials = d->num_materials;
        // every copy and kernel above has completed (the synchronize above): from here on
        // the arrays are released in the order of the context's stream, like the work
        // that reads them
        for (PoolBuf& b : ds->bufs) b.stream = c->stream;
        std::lock_guard<FairMutex> lk(c->mu);
        uint64_t id = c->nextScene++;
        c->scenes[id] = std::move(ds);
        *out = id;
    });
}

gnd_status gnd_gpu_scene_free(gnd_gpu_ctx* ctxh, gnd_scene_id id) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        auto use = c->sceneUse.find(id);
        if (use != c->sceneUse.end() && use->second > 0)
            throw Error(GND_ERR_INVALID, "scene " + std::to_string(id) + " is used by " + std::to_string(use->second) +
                                             " queued or running job(s)");
        auto it = c->scenes.find(id);
        if (it == c->scenes.end()) throw Error(GND_ERR_INVALID, "unknown scene id");
        // work queued on callers' streams (the _dev ray-batch calls) may still read the
        // scene; the arrays go back to the pool in the order of the context's stream
        GND_CUDA(cudaDeviceSynchronize());
        c->scenes.erase(it);
    });
}

// The large arrays of a scene description (BVH nodes, triangles, triangle attributes):
// each is one heap allocation of its own, so page-locking them never overlaps another
// registration.
static void bigArrays(const gnd_scene_desc* d, const void* ptr[3], size_t bytes[3]) {
    ptr[0] = d->nodes; bytes[0] = (size_t)d->num_nodes * sizeof(Node4);
    ptr[1] = d->tris; bytes[1] = (size_t)d->num_tris * sizeof(Tri);
    ptr[2] = d->tri_attrs; bytes[2] = (size_t)d->num_tris * sizeof(TriAttr);
}

gnd_status gnd_gpu_host_register(const gnd_scene_desc* d, int32_t pin) {
    return guarded([&]() {
        if (!d) throw Error(GND_ERR_INVALID, "null scene description");
        const void* ptr[3];
        size_t bytes[3];
        bigArrays(d, ptr, bytes);
        for (int k = 0; k < 3; ++k) {
            if (!ptr[k] || bytes[k] == 0) continue;
            cudaError_t e = pin ? cudaHostRegister(const_cast<void*>(ptr[k]), bytes[k], cudaHostRegisterPortable)
                                : cudaHostUnregister(const_cast<void*>(ptr[k]));
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw Error(GND_ERR_CUDA, std::string(pin ? "cudaHostRegister: " : "cudaHostUnregister: ") + cudaGetErrorString(e));
            }
        }
    });
}

gnd_status gnd_gpu_scene_bytes(gnd_gpu_ctx* ctxh, gnd_scene_id id, uint64_t* bytes) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        std::lock_guard<FairMutex> lk(c->mu);
        *bytes = c->scene(id).bytes;
    });
}

gnd_status gnd_gpu_set_build_leaf_max(gnd_gpu_ctx* ctxh, int32_t leafMax) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (leafMax < 1 || leafMax > kLeafMax) throw Error(GND_ERR_INVALID, "leaf size out of range (1..16)");
        std::lock_guard<std::mutex> ul(c->uploadMu);   // the uploads read it
        c->buildLeafMax = leafMax;
    });
}

gnd_status gnd_gpu_scene_info(gnd_gpu_ctx* ctxh, gnd_scene_id id, gnd_scene_info* info) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!info) throw Error(GND_ERR_INVALID, "null output pointer");
        std::lock_guard<FairMutex> lk(c->mu);
        const DeviceScene& s = c->scene(id);
        gnd_scene_info r{};
        r.num_nodes = s.numNodes;
        r.num_tris = s.numTris;
        r.num_instances = s.numInstances;
        r.blas_on_device = s.blasOnDevice ? 1 : 0;
        r.fast_boxes = s.view.fastBoxes;
        r.num_meshes = s.numMeshes;
        r.build_ms = s.buildMs;
        r.bytes = s.bytes;
        *info = r;
    });
}

gnd_status gnd_gpu_scene_download(gnd_gpu_ctx* ctxh, gnd_scene_id id, int32_t array, void* dst, int64_t capacity) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!dst && capacity > 0) throw Error(GND_ERR_INVALID, "null destination");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        const DeviceScene& s = c->scene(id);
        const void* src = nullptr;
        int64_t bytes = 0;
        switch (array) {
            case GND_ARRAY_NODES: src = s.view.nodes; bytes = s.numNodes * (int64_t)sizeof(Node4); break;
            case GND_ARRAY_TRIS: src = s.view.tris; bytes = s.numTris * (int64_t)sizeof(Tri); break;
            case GND_ARRAY_TRI_ATTRS: src = s.view.attrs; bytes = s.numTris * (int64_t)sizeof(TriAttr); break;
            case GND_ARRAY_ORIG_TO_LEAF: src = s.view.origToLeaf; bytes = s.origToLeafLen * 4; break;
            case GND_ARRAY_INST_TRAV: src = s.view.instT; bytes = s.numInstances * (int64_t)sizeof(InstTrav); break;
            default: throw Error(GND_ERR_INVALID, "unknown scene array");
        }
        if (bytes > capacity) throw Error(GND_ERR_INVALID, "destination too small: the array has " + std::to_string(bytes) + " bytes");
        if (bytes) {
            GND_CUDA(cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost, c->stream));
            GND_CUDA(cudaStreamSynchronize(c->stream));
        }
    });
}

}  // extern "C"
