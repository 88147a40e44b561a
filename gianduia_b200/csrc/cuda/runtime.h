// Device runtime: contexts, resident scenes, status/error plumbing shared by the
// C-ABI entry points.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "gnd/layout.h"
#include "gnd_gpu.h"

namespace gnd {

// Error carrying a gnd_status; converted to a status code at the ABI.
struct Error : std::runtime_error {
    gnd_status code;
    Error(gnd_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void setLastError(const std::string& msg);
const std::string& lastError();

#define GND_CUDA(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) {                                                                           \
            if (e_ == cudaErrorMemoryAllocation)                                                           \
                throw ::gnd::Error(GND_ERR_OOM, std::string("out of device memory: ") + #call);            \
            throw ::gnd::Error(GND_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
        }                                                                                                  \
    } while (0)

// Device sums of the trace kernels (Context::traceTotals, unsigned long long each).
enum TraceTotal : int { kTraceTotalRays = 0, kTraceTotalCountedRays = 1, kTraceTotalNodes = 2, kTraceTotalTris = 3, kTraceTotals = 4 };

// Runs an ABI body, mapping exceptions to a status.
template <typename F>
gnd_status guarded(F&& f) {
    try {
        f();
        return GND_OK;
    } catch (const Error& e) {
        setLastError(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        setLastError("host allocation failed");
        return GND_ERR_OOM;
    } catch (const std::exception& e) {
        setLastError(e.what());
        return GND_ERR_INVALID;
    }
}

// A device allocation with RAII ownership.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n) { alloc(n); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); ptr = o.ptr; bytes = o.bytes; o.ptr = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t n) {
        release();
        if (n == 0) return;
        GND_CUDA(cudaMalloc(&ptr, n));
        bytes = n;
    }
    void ensure(size_t n) { if (n > bytes) alloc(n); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T>
    T* as() const { return reinterpret_cast<T*>(ptr); }
};

// A stream-ordered allocation from the device's default memory pool, for scene arrays.
// The context raises the pool's release threshold, so memory freed here stays mapped in
// the pool and the next upload reuses it: freeing and uploading scenes does not unmap and
// map device memory (a plain cudaFree of a large buffer can stall the host for a long,
// unpredictable time).
struct PoolBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    PoolBuf() = default;
    PoolBuf(size_t n, cudaStream_t st) : stream(st) {
        if (n == 0) return;
        GND_CUDA(cudaMallocAsync(&ptr, n, st));
        bytes = n;
    }
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    PoolBuf(PoolBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes), stream(o.stream) { o.ptr = nullptr; o.bytes = 0; }
    PoolBuf& operator=(PoolBuf&& o) noexcept {
        if (this != &o) {
            if (ptr) cudaFreeAsync(ptr, stream);
            ptr = o.ptr; bytes = o.bytes; stream = o.stream;
            o.ptr = nullptr; o.bytes = 0;
        }
        return *this;
    }
    ~PoolBuf() {
        if (ptr) cudaFreeAsync(ptr, stream);
    }
    template <typename T>
    T* as() const { return reinterpret_cast<T*>(ptr); }
};

// Engine settings that change speed, never results (gnd_tune in the C ABI).
struct Tune {
    int poolLog2 = 22;        // path slots of a batched render: 2^poolLog2
    int roundIters = 8;       // wavefront iterations per host round of a batched render
    int travBlocks = 8;       // persistent traversal blocks (128 threads) per SM
    int sort = 1;             // 1: classify hits and shade per material class
    int smem = 32;            // traversal stack entries in shared memory (16 or 32)
    int graphs = 1;           // replay iteration pairs as CUDA graphs
    int sampleFilm = 1;       // batched box-filter renders: per-sample records, no film atomics
    int specExtend = 0;       // speculative node traversal in the extend kernel
    int specShadow = 0;       // speculative node traversal in the shadow kernel
    int raySort = 0;          // reorder each iteration's closest-hit queries by ray key
    int leafBatch = 32;       // closest-hit traversal of renders: lanes holding a leaf that end the node phase
    int traceLeafBatch = 12;  // the same for the scene's ray batches
    int shadowLeafBatch = 32; // the same for the path tracer's shadow queries
    int traceBlocks = 8;      // persistent blocks per SM of the scene's ray batches
    bool operator==(const Tune& o) const {
        return poolLog2 == o.poolLog2 && roundIters == o.roundIters && travBlocks == o.travBlocks && sort == o.sort &&
               smem == o.smem && graphs == o.graphs && sampleFilm == o.sampleFilm && specExtend == o.specExtend &&
               specShadow == o.specShadow && raySort == o.raySort && leafBatch == o.leafBatch &&
               traceLeafBatch == o.traceLeafBatch && shadowLeafBatch == o.shadowLeafBatch && traceBlocks == o.traceBlocks;
    }
    bool operator!=(const Tune& o) const { return !(*this == o); }
};

// A scene resident in HBM.
// The nodes of one tree level by level, for refits (refit.cu): breadth-first node
// indices, level l at [offsets[l], offsets[l + 1]).
struct RefitTopo {
    PoolBuf list;
    std::vector<int64_t> offsets;
};

struct DeviceScene {
    std::vector<PoolBuf> bufs;  // the large arrays (pool memory, freed stream-ordered)
    std::map<uint32_t, RefitTopo> refitTopo;   // per tree root, built by the first refit
    SceneView view{};
    DevBuf nullMask;          // per instance: 1 when the material has no BSDF (index)
    DevBuf instClass;         // per instance: material type (SceneView::instClass)
    DevBuf viewDev;           // SceneView copy in device memory
    uint64_t bytes = 0;
    int width = 0, height = 0, spp = 1, maxDepth = 1000, integrator = 0, filter = 0;
    float filterRadius[2] = {0.5f, 0.5f}, filterAlpha = 2.f;
    bool hasNullMaterials = false;
    int numMaterials = 0;
    Tune tune;                // engine settings for renders of this scene
    // array sizes (gnd_gpu_scene_info / gnd_gpu_scene_download)
    int64_t numNodes = 0, numTris = 0, origToLeafLen = 0;
    int numInstances = 0, numMeshes = 0;
    bool blasOnDevice = false;   // mesh trees built on the GPU at upload
    float buildMs = 0.0f;        // device time of that build
};

// First-come first-served mutex (ticket lock). The serving thread takes the context
// again right after each round; with a plain std::mutex it can starve API calls (submit,
// upload, free) that wait for the same context.
class FairMutex {
public:
    void lock() {
        std::unique_lock<std::mutex> lk(m_);
        const uint64_t ticket = next_++;
        cv_.wait(lk, [&]() { return serving_ == ticket; });
    }
    void unlock() {
        std::lock_guard<std::mutex> lk(m_);
        ++serving_;
        cv_.notify_all();
    }

private:
    std::mutex m_;
    std::condition_variable cv_;
    uint64_t next_ = 0, serving_ = 0;
};

class Wavefront;
class Server;

struct Context {
    int device = 0;
    int numSMs = 148;
    int buildLeafMax = 4;     // largest leaf of device-built mesh trees (guarded by uploadMu)
    cudaStream_t stream = nullptr;
    FairMutex mu;   // serialises every use of the context (stream, scenes, engine)
    // Scene uploads copy, build and validate on their own stream without holding mu, so
    // that they overlap renders; mu is taken only to publish the finished scene, and
    // uploadMu serialises the uploads among themselves.
    cudaStream_t uploadStream = nullptr;
    std::mutex uploadMu;
    std::map<uint64_t, std::unique_ptr<DeviceScene>> scenes;
    uint64_t nextScene = 1;
    DevBuf errWord;           // device error bitmask written by kernels
    DevBuf rayScratch, hitScratch;
    // gnd_gpu_counters: device sums of the trace kernels (kTraceTotal*), allocated with
    // the context, and the host sums of the renders
    DevBuf traceTotals;
    gnd_counters counters{};
    void countRender(const gnd_render_stats& s) {
        counters.renders += 1;
        counters.paths += s.paths;
        counters.extend_rays += s.extend_rays;
        counters.shadow_rays += s.shadow_rays;
        counters.extend_nodes += s.extend_nodes;
        counters.extend_tris += s.extend_tris;
        counters.iterations += s.iterations;
        counters.launches += s.launches;
        counters.render_ms += s.ms;
        counters.last = s;
    }
    // Work counters of persistent launches: each launch takes the next entry of a ring of
    // kFetchRing counters (reset on the launch's stream), so launches on different
    // streams do not share one.
    static constexpr int kFetchRing = 1024;
    DevBuf fetchRing;
    uint32_t fetchNext = 0;
    uint32_t* nextFetchCounter() {
        if (!fetchRing.ptr) fetchRing.alloc(kFetchRing * sizeof(uint32_t));
        uint32_t k = fetchNext++ % kFetchRing;
        return fetchRing.as<uint32_t>() + k;
    }
    std::unique_ptr<Wavefront> wave;
    volatile bool cancel = false;
    // serving: HBM admission budget (0 = the device's free memory), queued or running
    // jobs per scene (a scene in use cannot be freed), and the job server (created on
    // the first submit; serverMu guards its creation)
    uint64_t hbmBudget = 0;
    Tune serveTune = serveDefaults();   // engine settings of the serving thread (its own pool size)
    static Tune serveDefaults() {
        Tune t;
        t.roundIters = 4;   // short rounds: jobs are admitted and finished between rounds
        return t;
    }
    std::map<uint64_t, int> sceneUse;
    std::mutex serverMu;
    std::unique_ptr<Server> server;
    ~Context();
    DeviceScene& scene(uint64_t id) {
        auto it = scenes.find(id);
        if (it == scenes.end()) throw Error(GND_ERR_INVALID, "unknown scene id " + std::to_string(id));
        return *it->second;
    }
    void bind() { GND_CUDA(cudaSetDevice(device)); }
    // Reads and clears the kernel error word; throws on a tripped device check.
    void checkKernelErrors(const char* what);
};

Context* ctxOf(gnd_gpu_ctx* c);

}  // namespace gnd
