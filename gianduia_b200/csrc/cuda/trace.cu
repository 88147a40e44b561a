// Ray-batch queries: gnd_gpu_trace_closest / _any / _count (Scene::rayIntersect for a
// batch). One thread per ray, persistent grid sized to the SM count.
#include <mutex>
#include <string>

#include "raysort.cuh"
#include "runtime.h"
#include "traverse.cuh"

namespace gnd {

constexpr int kTraceBlock = 128;
constexpr int kTraceBlocksPerSM = 8;

// Ray batch source / sink for the persistent traversal loop. With `perm` (a batch
// reordered by ray key) the loop's i-th ray is ray perm[i] of the batch, and its result
// goes to slot perm[i].
template <bool ANY, bool COUNT>
struct BatchSrc {
    const SceneView* sv;
    const gnd_ray* rays;
    uint32_t n;
    gnd_hit* hits;
    uint8_t* occ;
    uint32_t* nodesOut;
    uint32_t* trisOut;
    TraceCounters* cnt;
    const uint32_t* perm;
    unsigned long long sumNodes = 0, sumTris = 0;   // COUNT: this lane's rays, for the context totals
    __device__ uint32_t count() const { return n; }
    __device__ bool load(uint32_t k, TRay& r, const SceneView*& s, const uint8_t*& nm) {
        const uint32_t i = perm ? __ldg(perm + k) : k;
        float4 a = __ldg(reinterpret_cast<const float4*>(rays + i));
        float4 b = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
        r.o = v3(a.x, a.y, a.z);
        r.tmin = a.w;
        r.d = v3(b.x, b.y, b.z);
        r.tmax = b.w;
        s = sv;
        nm = nullptr;
        if (COUNT) { cnt->nodes = 0; cnt->tris = 0; }
        return true;
    }
    __device__ void store(uint32_t k, const THit& h, const SceneView&) {
        const uint32_t i = perm ? __ldg(perm + k) : k;
        if (COUNT) {
            nodesOut[i] = cnt->nodes;
            trisOut[i] = cnt->tris;
            sumNodes += cnt->nodes;
            sumTris += cnt->tris;
        } else if (ANY) {
            occ[i] = h.inst >= 0 ? 1 : 0;
        } else {
            gnd_hit o;
            o.t = h.t;
            o.u = h.u;
            o.v = h.v;
            o.inst = h.inst;
            o.prim = (h.inst >= 0 && h.slot != 0xFFFFFFFFu) ? (int32_t)__ldg(&sv->tris[h.slot].prim) : -1;
            hits[i] = o;
        }
    }
};

// MINB: blocks per SM the kernel is compiled to fit (8: 64 registers; 9 and 10 trade
// registers, some spilled, for more resident warps; gnd_tune trace_blocks).
template <bool ANY, bool COUNT, int MINB = kTraceBlocksPerSM>
__global__ void __launch_bounds__(kTraceBlock, MINB)
    traceKernel(const SceneView* __restrict__ sv, const gnd_ray* __restrict__ rays, uint32_t n, gnd_hit* __restrict__ hits,
                uint8_t* __restrict__ occ, uint32_t* __restrict__ nodesOut, uint32_t* __restrict__ trisOut,
                uint32_t* fetch, uint32_t* errWord, unsigned long long* totals, const uint32_t* __restrict__ perm,
                uint32_t leafBatch) {
    __shared__ uint32_t stack[kSmemStack * kTraceBlock];
    TraceCounters cnt{0, 0, 0, 0, 0};
    BatchSrc<ANY, COUNT> src{sv, rays, n, hits, occ, nodesOut, trisOut, &cnt, perm};
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&totals[kTraceTotalRays], (unsigned long long)n);
        if (COUNT) atomicAdd(&totals[kTraceTotalCountedRays], (unsigned long long)n);
    }
    int err = persistentTrace<kTraceBlock, ANY, COUNT>(src, fetch, stack, &cnt, leafBatch);
    if (COUNT) {
        unsigned long long nn = src.sumNodes, nt = src.sumTris;
        for (int o = 16; o > 0; o >>= 1) {
            nn += __shfl_down_sync(0xffffffffu, nn, o);
            nt += __shfl_down_sync(0xffffffffu, nt, o);
        }
        if ((threadIdx.x & 31) == 0 && (nn | nt)) {
            atomicAdd(&totals[kTraceTotalNodes], nn);
            atomicAdd(&totals[kTraceTotalTris], nt);
        }
    }
    if (err) atomicOr(errWord, (uint32_t)err);
}

// Keys of a ray batch and their histogram (raysort.cuh).
__global__ void __launch_bounds__(256) kBatchKeys(const SceneView* __restrict__ sv, const gnd_ray* __restrict__ rays,
                                                  uint32_t n, uint32_t* __restrict__ keys, uint32_t* bins) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane;
        uint32_t key = 0xFFFFFFFFu;
        if (i < n) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(rays + i));
            const float4 b = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
            key = rayKey(*sv, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z));
            keys[i] = key;
        }
        const uint32_t grp = __match_any_sync(0xffffffffu, key);
        if (i < n && (int)lane == __ffs(grp) - 1) atomicAdd(&bins[key], (uint32_t)__popc(grp));
    }
}

// The batch's permutation in key order (rays of one warp with the same key keep their order).
__global__ void __launch_bounds__(256) kBatchScatter(const uint32_t* __restrict__ keys, uint32_t n, uint32_t* bins,
                                                     uint32_t* __restrict__ perm) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane;
        const uint32_t key = i < n ? keys[i] : 0xFFFFFFFFu;
        const uint32_t grp = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(grp) - 1;
        uint32_t pos = 0;
        if (i < n && (int)lane == leader) pos = atomicAdd(&bins[key], (uint32_t)__popc(grp));
        pos = __shfl_sync(grp, pos, leader);
        if (i < n) perm[pos + (uint32_t)__popc(grp & ((1u << lane) - 1u))] = i;
    }
}

namespace {
// Batches of at least this many rays are reordered when the scene's ray_sort has bit 2.
constexpr int64_t kBatchSortMin = 1 << 16;

void launchTrace(Context* c, DeviceScene& ds, const gnd_ray* dr, int64_t n, gnd_hit* dh, uint8_t* docc,
                 uint32_t* dn, uint32_t* dt, cudaStream_t st) {
    if (n <= 0) return;
    if (n >= (int64_t)0xF0000000LL) throw Error(GND_ERR_INVALID, "ray batch too large (limit 4e9 rays per call)");
    int64_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    // the counting kernel always fits 8 blocks per SM
    const int bps = dn ? kTraceBlocksPerSM : std::min(std::max(ds.tune.traceBlocks, 1), 10);
    int g = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)c->numSMs * bps));
    uint32_t* ew = c->errWord.as<uint32_t>();
    uint32_t* fetch = c->nextFetchCounter();
    GND_CUDA(cudaMemsetAsync(fetch, 0, sizeof(uint32_t), st));
    const SceneView* sv = ds.viewDev.as<SceneView>();
    uint32_t nn = (uint32_t)n;
    unsigned long long* tot = c->traceTotals.as<unsigned long long>();
    // Reordering: scratch from the stream-ordered pool on the batch's own stream, so
    // batches queued on different streams never share it; freed behind the traversal.
    PoolBuf keys, perm, bins;
    const uint32_t* order = nullptr;
    if ((ds.tune.raySort & 4) && n >= kBatchSortMin) {
        keys = PoolBuf((size_t)n * sizeof(uint32_t), st);
        perm = PoolBuf((size_t)n * sizeof(uint32_t), st);
        bins = PoolBuf(kRayBins * sizeof(uint32_t), st);
        GND_CUDA(cudaMemsetAsync(bins.ptr, 0, kRayBins * sizeof(uint32_t), st));
        const int kg = (int)std::min<int64_t>((n + 255) / 256, (int64_t)c->numSMs * 8);
        kBatchKeys<<<kg, 256, 0, st>>>(sv, dr, nn, keys.as<uint32_t>(), bins.as<uint32_t>());
        kRayScan<<<1, 1024, 0, st>>>(bins.as<uint32_t>());
        kBatchScatter<<<kg, 256, 0, st>>>(keys.as<uint32_t>(), nn, bins.as<uint32_t>(), perm.as<uint32_t>());
        GND_CUDA(cudaGetLastError());
        order = perm.as<uint32_t>();
    }
    const uint32_t lb = (uint32_t)ds.tune.traceLeafBatch;
    if (dn) traceKernel<false, true><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, nullptr, nullptr, dn, dt, fetch, ew, tot, order, lb);
    else if (docc && bps == 9) traceKernel<true, false, 9><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, nullptr, docc, nullptr, nullptr, fetch, ew, tot, order, lb);
    else if (docc && bps == 10) traceKernel<true, false, 10><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, nullptr, docc, nullptr, nullptr, fetch, ew, tot, order, lb);
    else if (docc) traceKernel<true, false><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, nullptr, docc, nullptr, nullptr, fetch, ew, tot, order, lb);
    else if (bps == 9) traceKernel<false, false, 9><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, dh, nullptr, nullptr, nullptr, fetch, ew, tot, order, lb);
    else if (bps == 10) traceKernel<false, false, 10><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, dh, nullptr, nullptr, nullptr, fetch, ew, tot, order, lb);
    else traceKernel<false, false><<<g, kTraceBlock, 0, st>>>(sv, dr, nn, dh, nullptr, nullptr, nullptr, fetch, ew, tot, order, lb);
    GND_CUDA(cudaGetLastError());
    c->counters.trace_batches += 1;
}

// Host-buffer variant: copies in, traces, copies out (pinned staging is the caller's
// concern; pageable memory works, at lower copy bandwidth).
void traceHost(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_ray* rays, int64_t n, gnd_hit* hits, uint8_t* occ) {
    Context* c = ctxOf(ctxh);
    if (n < 0 || (n > 0 && (!rays || (!hits && !occ)))) throw Error(GND_ERR_INVALID, "bad ray batch arguments");
    c->bind();
    std::lock_guard<FairMutex> lk(c->mu);
    DeviceScene& ds = c->scene(id);
    if (n == 0) return;
    size_t outBytes = hits ? sizeof(gnd_hit) * (size_t)n : (size_t)n;
    c->rayScratch.ensure(sizeof(gnd_ray) * (size_t)n);
    c->hitScratch.ensure(outBytes);
    GND_CUDA(cudaMemcpyAsync(c->rayScratch.ptr, rays, sizeof(gnd_ray) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    launchTrace(c, ds, c->rayScratch.as<gnd_ray>(), n, hits ? c->hitScratch.as<gnd_hit>() : nullptr,
                hits ? nullptr : c->hitScratch.as<uint8_t>(), nullptr, nullptr, c->stream);
    GND_CUDA(cudaMemcpyAsync(hits ? (void*)hits : (void*)occ, c->hitScratch.ptr, outBytes, cudaMemcpyDeviceToHost, c->stream));
    GND_CUDA(cudaStreamSynchronize(c->stream));
    c->checkKernelErrors("trace");
}
}  // namespace

// ---------------------------------------------------------------- allocation-free variant
// Fixed device scratch of gnd_gpu_trace_closest_fixed: the persistent grid's fetch
// counter (first 256 bytes; must be zero when the kernel starts, so every call clears
// it), then the rays and the hits of one batch of at most kFixedMaxRays rays. It is a
// module-scope array, one per device, shared by every context and thread of the
// process on that device: calls that overlap in time on one device race on it.
constexpr int64_t kFixedMaxRays = GND_TRACE_FIXED_MAX_RAYS;
constexpr size_t kFixedCounterBytes = 256;
constexpr size_t kFixedRayBytes = sizeof(gnd_ray) * (size_t)kFixedMaxRays;   // 2 MiB
constexpr size_t kFixedHitBytes = sizeof(gnd_hit) * (size_t)kFixedMaxRays;   // 1.25 MiB
static_assert(kFixedRayBytes % 256 == 0 && kFixedHitBytes % 256 == 0, "scratch regions stay 256-byte aligned");
static __device__ __align__(256) unsigned char gFixedScratch[kFixedCounterBytes + kFixedRayBytes + kFixedHitBytes];

namespace {
constexpr int kFixedMaxDevices = 64;
std::mutex gFixedMu;
void* gFixedAddr[kFixedMaxDevices] = {};

// Device address of gFixedScratch on the current device, looked up once per device. The
// first lookup may load the module onto the device.
unsigned char* fixedScratch(int device) {
    if (device < 0 || device >= kFixedMaxDevices) throw Error(GND_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lk(gFixedMu);
    if (!gFixedAddr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, gFixedScratch);
        if (e != cudaSuccess || !ptr)
            throw Error(GND_ERR_CUDA, std::string("cudaGetSymbolAddress(fixed trace scratch): ") + cudaGetErrorString(e));
        gFixedAddr[device] = ptr;
    }
    return static_cast<unsigned char*>(gFixedAddr[device]);
}
}  // namespace

}  // namespace gnd

using namespace gnd;

extern "C" {

gnd_status gnd_gpu_trace_closest(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* rays, int64_t n, gnd_hit* hits) {
    return guarded([&]() {
        if (!hits && n > 0) throw Error(GND_ERR_INVALID, "null hit buffer");
        traceHost(ctx, scene, rays, n, hits, nullptr);
    });
}

gnd_status gnd_gpu_trace_any(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* rays, int64_t n, uint8_t* occluded) {
    return guarded([&]() {
        if (!occluded && n > 0) throw Error(GND_ERR_INVALID, "null output buffer");
        traceHost(ctx, scene, rays, n, nullptr, occluded);
    });
}

gnd_status gnd_gpu_trace_closest_dev(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_ray* d_rays, int64_t n, gnd_hit* d_hits,
                                     void* stream) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (n < 0 || (n > 0 && (!d_rays || !d_hits))) throw Error(GND_ERR_INVALID, "bad ray batch arguments");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
        launchTrace(c, c->scene(id), d_rays, n, d_hits, nullptr, nullptr, nullptr, st);
    });
}

gnd_status gnd_gpu_trace_any_dev(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_ray* d_rays, int64_t n, uint8_t* d_occ,
                                 void* stream) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (n < 0 || (n > 0 && (!d_rays || !d_occ))) throw Error(GND_ERR_INVALID, "bad ray batch arguments");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
        launchTrace(c, c->scene(id), d_rays, n, nullptr, d_occ, nullptr, nullptr, st);
    });
}

gnd_status gnd_gpu_trace_count_dev(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_ray* d_rays, int64_t n, uint32_t* d_nodes,
                                   uint32_t* d_tris, void* stream) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (n < 0 || (n > 0 && (!d_rays || !d_nodes || !d_tris))) throw Error(GND_ERR_INVALID, "bad ray batch arguments");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
        launchTrace(c, c->scene(id), d_rays, n, nullptr, nullptr, d_nodes, d_tris, st);
    });
}

// Closest hits of at most 65536 host-memory rays with no device allocation: rays, hits
// and the fetch counter live in gFixedScratch. No counterpart in the reference.
gnd_status gnd_gpu_trace_closest_fixed(gnd_gpu_ctx* ctxh, gnd_scene_id id, const gnd_ray* rays, int64_t n,
                                       gnd_hit* hits) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (n < 0 || (n > 0 && (!rays || !hits))) throw Error(GND_ERR_INVALID, "bad ray batch arguments");
        if (n > kFixedMaxRays)
            throw Error(GND_ERR_INVALID, "gnd_gpu_trace_closest_fixed: " + std::to_string(n) +
                                             " rays exceed the fixed scratch limit of " + std::to_string(kFixedMaxRays) +
                                             " rays per call");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        DeviceScene& ds = c->scene(id);
        unsigned char* base = fixedScratch(c->device);
        if (n == 0) return;
        uint32_t* fetch = reinterpret_cast<uint32_t*>(base);
        gnd_ray* dr = reinterpret_cast<gnd_ray*>(base + kFixedCounterBytes);
        gnd_hit* dh = reinterpret_cast<gnd_hit*>(base + kFixedCounterBytes + kFixedRayBytes);
        cudaStream_t st = c->stream;
        GND_CUDA(cudaMemcpyAsync(dr, rays, sizeof(gnd_ray) * (size_t)n, cudaMemcpyHostToDevice, st));
        GND_CUDA(cudaMemsetAsync(fetch, 0, sizeof(uint32_t), st));
        int64_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
        int g = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)c->numSMs * kTraceBlocksPerSM));
        traceKernel<false, false><<<g, kTraceBlock, 0, st>>>(ds.viewDev.as<SceneView>(), dr, (uint32_t)n, dh, nullptr,
                                                             nullptr, nullptr, fetch, c->errWord.as<uint32_t>(),
                                                             c->traceTotals.as<unsigned long long>(), nullptr, 32u);
        GND_CUDA(cudaGetLastError());
        c->counters.trace_batches += 1;
        GND_CUDA(cudaMemcpyAsync(hits, dh, sizeof(gnd_hit) * (size_t)n, cudaMemcpyDeviceToHost, st));
        GND_CUDA(cudaStreamSynchronize(st));
        c->checkKernelErrors("trace_closest_fixed");
    });
}

}  // extern "C"
