// Wavefront path-tracing engine: path state in HBM, per-bounce kernels (extend =
// closest hit, shade = one bounce of path / volpath, shadow = occlusion or
// transmittance, retire = film accumulation and slot refill), queues of path slots
// with warp-aggregated appends.
#pragma once
#include <vector>

#include "runtime.h"

namespace gnd {

// Path state, one 96-byte record per slot.
struct alignas(16) PathState {
    float ox, oy, oz, pdfPrev;
    float dx, dy, dz, lastX;
    float tpr, tpg, tpb, lastY;
    float Lr, Lg, Lb, lastZ;
    uint32_t rngLo, rngHi, pixel, pass;   // pixel = index in the job's window
    uint32_t bounces;                     // bounces | nullBounces << 16
    uint32_t vsBounces;                   // volumeBounces | surfaceBounces << 16 (saturating)
    int32_t medium;                       // -1: vacuum
    uint32_t flags;                       // bit0 specularBounce, bits 8..31 job index
};
static_assert(sizeof(PathState) == 96, "PathState must be 96 bytes");

struct alignas(16) HitRec {
    float t, u, v;
    int32_t inst;
    uint32_t slot;
    uint32_t pad[3];
};

// Shadow work item: an occlusion (path) or transmittance (volpath) query whose
// contribution is added to the owning path's radiance when the segment is clear.
struct alignas(16) ShadowRec {
    float ox, oy, oz, tmax;
    float dx, dy, dz;
    uint32_t slot;
    float cr, cg, cb;
    int32_t medium;
    float lx, ly, lz;
    uint32_t pad;
};

// One render job as the kernels see it.
struct JobDev {
    SceneView view;
    const uint8_t* nullMask;
    unsigned long long* filmSum;   // per pixel: sum wL (r, g, b) and sum w, fixed point 2^-24
    float* filmSq;                 // per pixel: sum w L^2 (r, g, b)
    int32_t W, H, maxDepth, integrator;
    int32_t wx0, wy0, wx1, wy1;    // pixel window
    int32_t filter;                // 0 box, 1 gaussian
    float frx, fry, falpha, fexpX, fexpY;
    int32_t hasNull;
    int32_t firstPass;
    uint64_t workBegin, workEnd;   // work items [begin, end): item -> (pass, window pixel)
    // Per-sample film records (batched renders), indexed by work item; null: finished
    // samples are splatted into the film with atomics. With the Gaussian filter each
    // record also keeps its film position within its pixel (sampleOff).
    float4* samples;
    float2* sampleOff;
};

// Queue counters (device): ints.
// kQOut and kQFreeOut are one aligned 64-bit pair (low, high) so that kRetire appends to
// both lists with a single atomic.
enum QCounter : int {
    kQIn = 0, kQShadow = 2, kQDone = 3, kQFetchA = 4, kQFetchB = 5, kQFree = 6,
    kQActive = 8, kQIter = 9, kQWork = 10, kQOut = 12, kQFreeOut = 13, kQClass0 = 16, kQCount = 32
};
static_assert(kQOut % 2 == 0 && kQFreeOut == kQOut + 1, "kQOut / kQFreeOut must form an aligned pair");

// Per-job work control on the device.
struct alignas(16) JobCtl {
    unsigned long long next;      // next work item to hand out (may run past the end)
    unsigned long long retired;   // finished samples
};

constexpr int kMaxJobs = 64;

// Host record of an admitted job.
struct HostJob {
    bool used = false;
    JobDev dev{};
    uint64_t total = 0;           // work items (samples)
    uint64_t released = 0;        // work items handed to the device so far (workEnd)
    uint64_t retired = 0;         // last value read back
    DevBuf filmSum, filmSq;
    uint64_t bytes = 0;           // film bytes held in HBM
    uint64_t seq = 0;             // admission order
    uint64_t prio = 0;            // hand-out order key: lower first, ties by admission
};

// The engine: one pool of path slots shared by every admitted job. Each iteration runs
// extend, shade, shadow and retire on the active list; retire splats finished samples
// and refills their slots (and idle slots) with work items of the active jobs, taken
// round-robin in warp-sized grabs.
struct KParams;

class Wavefront {
public:
    explicit Wavefront(Context* c);
    ~Wavefront();
    struct Result {
        int64_t paths = 0, rays = 0, extendRays = 0, shadowRays = 0, extendNodes = 0, extendTris = 0, iterations = 0;
        int64_t extendNodeWarpSteps = 0, extendLeafSteps = 0, extendLeafWarpSteps = 0;
        int64_t launches = 0;         // kernels launched
        int passesDone = 0;
        double ms = 0.0, extendMs = 0.0;
    };
    // One job to completion: plain = one pass in flight (the pool is one pass and each
    // pass is released when the previous retired), batched = all passes released at once.
    // The film is added into filmHost (H x W x 7 floats) or, when fixedSum is given, in its
    // fixed-point form into fixedSum (H x W x 4 uint64) and fixedSq (H x W x 3 floats).
    Result render(DeviceScene& ds, int W, int H, int spp, int firstPass, int maxDepth, int integrator,
                  const int window[4], bool batched, int profile, float* filmHost, gnd_progress_fn cb, void* user,
                  uint64_t* fixedSum = nullptr, float* fixedSq = nullptr);

    // ---- engine interface used by render() and by the server
    void reset(size_t slots);                         // (re)initialise the pool: every slot idle
    int admit(const DeviceScene& ds, int W, int H, int spp, int firstPass, int maxDepth, int integrator,
              const int window[4], uint64_t releaseItems);
    void release(int job, uint64_t upTo);             // hand out work items [.., upTo)
    void finish(int job, float* filmHost);            // adds the film to filmHost, frees the job
    // adds the job's fixed-point sums into sum (H x W x 4) and sq (H x W x 3), frees the job
    void finishFixed(int job, uint64_t* sum, float* sq);
    void resolve(int job, float* filmHost);           // writes the film (H x W x 7 floats) to filmHost
    // The job's film resolved into pinned host memory (valid until the next call).
    const float* resolvePinned(int job);
    void stop(int job);                               // hands out no further work items of the job
    void drop(int job);                               // frees the job without reading it
    // Runs `iters` iterations; returns the number of paths in flight afterwards.
    uint32_t step(int iters, int integratorMix, bool hasNull, int profile, Result& acc);
    // Pipelined rounds: enqueueRound queues `iters` iterations followed by an
    // asynchronous copy of the queue and job counters into pinned snapshot `slot` (0/1);
    // waitRound blocks until that snapshot has landed. Queueing round k+1 before waiting
    // for round k keeps the GPU busy while the host reads the counters.
    struct alignas(16) Snapshot {
        uint32_t inflight;            // active paths after the round
        uint32_t err;                 // the context's kernel error word after the round
        unsigned long long retiredAll;   // paths retired by the engine since its pool was reset
        JobCtl ctl[kMaxJobs];         // per job: work items handed out, samples retired
    };
    void enqueueRound(int iters, int integratorMix, bool hasNull, int profile, Result& acc, int slot);
    const Snapshot& waitRound(int slot);
    uint64_t retired(int job);                        // reads the job's retired count (sync)
    void readRetired(std::vector<uint64_t>& out);     // all jobs (one copy, sync)
    void readCtl(std::vector<JobCtl>& out);           // all jobs' hand-out and retired counts (sync)
    // Gives the job a per-sample record buffer for `items` work items (see JobDev::samples);
    // filmFromSamples() then adds the records into the job's film.
    void useSampleRecords(int job, uint64_t items);
    void filmFromSamples(int job, uint64_t items);
    // Hand-out order: false = every warp starts at a different active job (even shares),
    // true = oldest admitted job first (first-come first-served with the pool kept full).
    void setFifo(bool fifo) { fifo_ = fifo; }
    // Sets the hand-out order keys of the admitted jobs (index -> key) and updates the
    // device's active list when the order changed.
    void setPriorities(const std::vector<std::pair<int, uint64_t>>& keys);
    bool busy() const;                                // any job admitted
    // Engine settings for the following iterations (graphs captured under other settings
    // are dropped).
    void setTune(const Tune& t);
    const Tune& tune() const { return tune_; }
    size_t capacity() const { return cap_; }
    // Device bytes of one path slot (state, hit, shadow record, lists) and of the pool.
    static uint64_t slotBytes() {
        return sizeof(PathState) + sizeof(HitRec) + sizeof(ShadowRec) + 5 * sizeof(uint32_t) + 10 * sizeof(uint32_t) +
               2 * sizeof(uint32_t);   // ray keys and the reordered list
    }
    uint64_t poolBytes() const;   // path pool + film staging + film buffers kept for reuse
    HostJob& job(int j) { return jobs_[j]; }
    uint64_t jobBytes() const;

private:
    void ensureCapacity(size_t slots);
    void syncActive();
    // One wavefront iteration on the stream for the lists of parity `par`.
    void enqueueIteration(KParams kp, int par, int mix, bool hasNull, int profile, cudaStream_t st);
    // Executable graph of two iterations (parity restored) for these settings, captured on
    // first use; the per-iteration state it needs (queue counters, iteration number) is
    // in device memory, so one capture serves every later replay.
    cudaGraphExec_t pairGraph(const KParams& kp, int par, int mix, bool hasNull, cudaStream_t st);
    void clearGraphs();
    struct GraphEntry {
        int par, mix;
        bool hasNull, fifo, motion, ext;
        cudaGraphExec_t exec;
    };
    bool motion_ = false;   // an admitted job's scene has animated instances (MOTION traversal)
    bool ext_ = false;      // an admitted job's scene uses the EXT features (SceneView::ext)
    std::vector<GraphEntry> graphs_;
    Tune tune_;
    Context* ctx_;
    size_t cap_ = 0;
    int cur_ = 0;
    DevBuf paths_, hits_, listA_, listB_, freeA_, freeB_, shadow_, done_, counters_, totals_, classes_, times_;
    DevBuf jobTab_, ctl_, active_, filmOut_, samples_, sampleOff_;
    DevBuf rayKeys_, rayBins_, raySorted_;   // ray reordering (Tune::raySort)
    Snapshot* snaps_ = nullptr;       // pinned host memory, two slots
    cudaEvent_t snapEv_[2] = {nullptr, nullptr};
    bool fifo_ = false;
    uint64_t launches_ = 0;           // kernels launched by the engine so far
    uint64_t seqNext_ = 0;
    HostJob jobs_[kMaxJobs];
    std::vector<cudaEvent_t> evs_;    // profile: (start, end) of each extend launch, from evPool_
    std::vector<cudaEvent_t> evPool_; // timing events created once and reused
    size_t evUsed_ = 0;
    cudaEvent_t evStart_ = nullptr, evEnd_ = nullptr;
    cudaEvent_t nextEvent();
    float* pinnedFilm_ = nullptr;     // resolve staging (pinned), grown as needed
    size_t pinnedFilmBytes_ = 0;
    bool activeDirty_ = true;
};

}  // namespace gnd
