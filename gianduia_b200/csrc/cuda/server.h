// Render-job serving on one context: submitted jobs (scene, film size, spp, depth,
// integrator) are admitted first-come first-served into the wavefront engine's shared
// pool of path slots while the job table and the HBM budget allow, and a host thread
// steps the engine until each job's samples have all retired, then resolves its film to
// host memory. Freed slots take the oldest admitted job's next samples, so the pool stays
// full across job boundaries instead of draining at the end of every image.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"
#include "wavefront.h"

namespace gnd {

struct ServeJob {
    gnd_job_id id = 0;
    uint64_t scene = 0;
    int W = 0, H = 0, spp = 0, maxDepth = 0, integ = 0, firstPass = 0;
    int state = GND_JOB_QUEUED;
    int slot = -1;                   // engine job index while running
    uint64_t total = 0, done = 0;
    uint64_t filmBytes = 0;          // device film bytes while running
    bool cancelReq = false;
    int64_t firstRound = 0;          // first engine round whose counters include the job
    int64_t stopRound = -1;          // first round queued after its hand-out was stopped
    double tSubmit = 0, tAdmit = 0, tDone = 0;
    std::vector<float> film;         // H x W x 7 once finished
    gnd_status status = GND_OK;
    std::string error;
};

class Server {
public:
    static constexpr int64_t kStallIters = 20000;           // iterations without a retired sample

    // Path slots of the serving pool: 2^pool_log2 of the serving settings (gnd_gpu_serve_tune;
    // default 22, 4M slots, about 1 GB). Read with the context mutex held.
    size_t poolSlots() const;
    explicit Server(Context* c);
    ~Server();
    gnd_job_id submit(const gnd_job_desc& d);
    void poll(gnd_job_id id, gnd_job_status* st);
    gnd_status wait(gnd_job_id id, float* film, gnd_job_status* st, int64_t timeoutMs, std::string& err);
    void cancel(gnd_job_id id);
    uint64_t bytesInUseLocked() const;                       // caller holds the context mutex
    void setPolicy(int policy);                              // GND_SERVE_*

private:
    void loop();
    void fillStatus(const ServeJob& j, gnd_job_status* st) const;
    double nowMs() const;
    bool fitsLocked(const ServeJob& j) const;                // caller holds the context mutex
    void finishJob(ServeJob* j, int state);
    void failRunning(const std::string& why, gnd_status code);
    void drainPipeline();
    void applyPriorities(const std::vector<ServeJob*>& run);   // caller holds the context mutex

    Context* c_;
    std::thread thread_;
    std::mutex m_;                                           // guards the job records below
    std::condition_variable workCv_, doneCv_;
    std::deque<gnd_job_id> queue_;
    std::unordered_map<gnd_job_id, std::unique_ptr<ServeJob>> jobs_;
    std::vector<ServeJob*> running_;
    gnd_job_id nextId_ = 1;
    bool stop_ = false;
    // Rounds are queued one ahead: round q+1 runs while the host reads round q's counters.
    int64_t enqRound_ = 0;                                   // index of the next round to queue
    int64_t slotRound_[2] = {-1, -1};                        // round held by each snapshot slot
    int inflightSlot_ = 0;
    bool inflight_ = false;
    std::vector<JobCtl> lastCtl_;                            // job counters of the last snapshot read
    int64_t lastRound_ = -1;                                 // its round
    std::atomic<int> policy_{GND_SERVE_DEADLINE};
    static constexpr double kDeadlineSlack = 4.0;
    double rate_ = 1e5;                                      // samples per ms, running estimate
    double lastRoundMs_ = -1.0;
    unsigned long long lastRetiredAll_ = 0;
    int64_t itersSinceProgress_ = 0;
    uint64_t lastRetiredSum_ = 0;
    const std::chrono::steady_clock::time_point t0_;
};

}  // namespace gnd
