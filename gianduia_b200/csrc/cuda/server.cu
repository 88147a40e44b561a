// Render-job serving (gnd_gpu_serve_*): a host thread per context drives the wavefront
// engine over every running job at once. Each round it admits queued jobs that fit,
// runs a few engine iterations, reads every job's hand-out and retired counts, and
// resolves the film of each job whose samples have all retired.
#include <algorithm>

#include "server.h"
#include "wavefront.h"

namespace gnd {

Server::Server(Context* c) : c_(c), t0_(std::chrono::steady_clock::now()) {
    thread_ = std::thread([this]() { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(m_);
        stop_ = true;
    }
    workCv_.notify_all();
    if (thread_.joinable()) thread_.join();
    // jobs still admitted are dropped with the engine; wake any waiter
    std::lock_guard<std::mutex> lk(m_);
    for (auto& kv : jobs_) {
        ServeJob& j = *kv.second;
        if (j.state == GND_JOB_QUEUED || j.state == GND_JOB_RUNNING) {
            j.state = GND_JOB_FAILED;
            j.status = GND_ERR_CANCELLED;
            j.error = "server shut down";
        }
    }
    doneCv_.notify_all();
}

double Server::nowMs() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
}

uint64_t Server::bytesInUseLocked() const {
    uint64_t b = 0;
    for (const auto& kv : c_->scenes) b += kv.second->bytes;
    if (c_->wave) b += c_->wave->poolBytes() + c_->wave->jobBytes();
    return b;
}

size_t Server::poolSlots() const {
    return size_t(1) << std::min(std::max(c_->serveTune.poolLog2, 16), 26);
}

bool Server::fitsLocked(const ServeJob& j) const {
    const size_t slots = poolSlots();
    const uint64_t pool = c_->wave && c_->wave->capacity() >= slots ? 0 : Wavefront::slotBytes() * slots;
    const uint64_t staging = (uint64_t)j.W * j.H * 7 * sizeof(float);
    const uint64_t need = j.filmBytes + staging + pool;
    if (c_->hbmBudget) return bytesInUseLocked() + need <= c_->hbmBudget;
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return false;
    return need + (uint64_t(256) << 20) <= freeB;
}

gnd_job_id Server::submit(const gnd_job_desc& d) {
    auto j = std::make_unique<ServeJob>();
    {
        // resolve defaults from the scene and check the budget (context mutex)
        std::lock_guard<FairMutex> ck(c_->mu);
        DeviceScene& ds = c_->scene(d.scene);
        j->scene = d.scene;
        j->W = d.width > 0 ? d.width : ds.width;
        j->H = d.height > 0 ? d.height : ds.height;
        j->spp = d.spp > 0 ? d.spp : ds.spp;
        j->maxDepth = std::min(d.max_depth > 0 ? d.max_depth : ds.maxDepth, 65535);
        j->integ = d.integrator >= 0 ? d.integrator : ds.integrator;
        j->firstPass = d.first_pass;
        if (j->integ != 0 && j->integ != 1) throw Error(GND_ERR_INVALID, "integrator must be 0 (path_gpu) or 1 (volpath_gpu)");
        if (j->W <= 0 || j->H <= 0 || (uint64_t)j->W * j->H > (1ull << 31)) throw Error(GND_ERR_INVALID, "bad film size");
        if (ds.view.numEmitters <= 0) throw Error(GND_ERR_INVALID, "the path integrators need at least one emitter");
        j->total = (uint64_t)j->W * j->H * (uint64_t)j->spp;
        j->filmBytes = (uint64_t)j->W * j->H * (4 * sizeof(unsigned long long) + 3 * sizeof(float));
        if (c_->hbmBudget) {
            uint64_t scenes = 0;
            for (const auto& kv : c_->scenes) scenes += kv.second->bytes;
            const uint64_t alone = scenes + Wavefront::slotBytes() * poolSlots() + j->filmBytes + (uint64_t)j->W * j->H * 28;
            if (alone > c_->hbmBudget)
                throw Error(GND_ERR_BUDGET, "job needs " + std::to_string(alone) + " bytes of HBM with its scenes and the path pool; budget " +
                                                std::to_string(c_->hbmBudget));
        }
        c_->sceneUse[d.scene]++;
    }
    std::lock_guard<std::mutex> lk(m_);
    j->id = nextId_++;
    j->tSubmit = nowMs();
    const gnd_job_id id = j->id;
    queue_.push_back(id);
    jobs_.emplace(id, std::move(j));
    workCv_.notify_all();
    return id;
}

void Server::fillStatus(const ServeJob& j, gnd_job_status* st) const {
    if (!st) return;
    st->state = j.state;
    st->pad = 0;
    st->samples_total = (int64_t)j.total;
    st->samples_done = (int64_t)j.done;
    st->submit_ms = j.tSubmit;
    st->admit_ms = j.tAdmit;
    st->done_ms = j.tDone;
}

void Server::poll(gnd_job_id id, gnd_job_status* st) {
    std::lock_guard<std::mutex> lk(m_);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) throw Error(GND_ERR_INVALID, "unknown job id " + std::to_string(id));
    fillStatus(*it->second, st);
}

gnd_status Server::wait(gnd_job_id id, float* film, gnd_job_status* st, int64_t timeoutMs, std::string& err) {
    std::unique_lock<std::mutex> lk(m_);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) throw Error(GND_ERR_INVALID, "unknown job id " + std::to_string(id));
    ServeJob* j = it->second.get();
    auto finished = [&]() { return j->state >= GND_JOB_DONE; };
    if (timeoutMs < 0) doneCv_.wait(lk, finished);
    else if (!doneCv_.wait_for(lk, std::chrono::milliseconds(timeoutMs), finished)) {
        fillStatus(*j, st);
        err = "job " + std::to_string(id) + " still running after " + std::to_string(timeoutMs) + " ms";
        return GND_ERR_TIMEOUT;
    }
    fillStatus(*j, st);
    if (film && !j->film.empty()) std::copy(j->film.begin(), j->film.end(), film);
    gnd_status s = j->state == GND_JOB_DONE ? GND_OK : (j->state == GND_JOB_CANCELLED ? GND_ERR_CANCELLED : j->status);
    if (s != GND_OK) err = j->state == GND_JOB_CANCELLED ? "job cancelled" : j->error;
    jobs_.erase(it);
    return s;
}

void Server::cancel(gnd_job_id id) {
    std::lock_guard<std::mutex> lk(m_);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) throw Error(GND_ERR_INVALID, "unknown job id " + std::to_string(id));
    it->second->cancelReq = true;
    workCv_.notify_all();
}

// Called with the context mutex held. Resolves the film (done or cancelled) and frees
// the engine's job entry.
void Server::finishJob(ServeJob* j, int state) {
    Wavefront& wf = *c_->wave;
    std::vector<float> film((size_t)j->W * j->H * 7);
    wf.resolve(j->slot, film.data());
    wf.drop(j->slot);
    if (--c_->sceneUse[j->scene] <= 0) c_->sceneUse.erase(j->scene);
    std::lock_guard<std::mutex> lk(m_);
    j->film.swap(film);
    j->state = state;
    j->tDone = nowMs();
    j->slot = -1;
    running_.erase(std::find(running_.begin(), running_.end(), j));
    doneCv_.notify_all();
}

// Called with the context mutex held: every running job fails with `why`.
void Server::failRunning(const std::string& why, gnd_status code) {
    Wavefront& wf = *c_->wave;
    std::vector<ServeJob*> run;
    {
        std::lock_guard<std::mutex> lk(m_);
        run = running_;
    }
    for (ServeJob* j : run) {
        try {
            wf.drop(j->slot);
        } catch (...) {
        }
        if (--c_->sceneUse[j->scene] <= 0) c_->sceneUse.erase(j->scene);
    }
    std::lock_guard<std::mutex> lk(m_);
    for (ServeJob* j : run) {
        j->state = GND_JOB_FAILED;
        j->status = code;
        j->error = why;
        j->tDone = nowMs();
        j->slot = -1;
    }
    running_.clear();
    doneCv_.notify_all();
}

void Server::loop() {
    cudaSetDevice(c_->device);
    std::vector<JobCtl> ctl;
    bool backoff = false;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(m_);
            if (backoff) {
                workCv_.wait_for(lk, std::chrono::milliseconds(5));
                backoff = false;
            }
            workCv_.wait(lk, [&]() { return stop_ || !queue_.empty() || !running_.empty(); });
            if (stop_) return;
        }
        std::lock_guard<FairMutex> ck(c_->mu);
        try {
            if (!c_->wave) c_->wave = std::make_unique<Wavefront>(c_);
            Wavefront& wf = *c_->wave;
            // admission, first come first served
            std::vector<ServeJob*> admit;
            {
                std::lock_guard<std::mutex> lk(m_);
                while (!queue_.empty() && running_.size() + admit.size() < (size_t)kMaxJobs) {
                    ServeJob* j = jobs_.at(queue_.front()).get();
                    if (j->cancelReq) {
                        queue_.pop_front();
                        j->state = GND_JOB_CANCELLED;
                        j->tDone = nowMs();
                        if (--c_->sceneUse[j->scene] <= 0) c_->sceneUse.erase(j->scene);
                        doneCv_.notify_all();
                        continue;
                    }
                    if (!fitsLocked(*j)) break;
                    queue_.pop_front();
                    admit.push_back(j);
                }
            }
            if (!admit.empty() && !wf.busy()) wf.reset(poolSlots());
            wf.setFifo(true);
            wf.setTune(c_->serveTune);
            for (ServeJob* j : admit) {
                int slot = -1;
                std::string why;
                gnd_status code = GND_OK;
                try {
                    DeviceScene& ds = c_->scene(j->scene);
                    const int win[4] = {0, 0, 0, 0};
                    slot = wf.admit(ds, j->W, j->H, j->spp, j->firstPass, j->maxDepth, j->integ, win, j->total);
                } catch (const Error& e) {
                    why = e.what();
                    code = e.code;
                }
                std::lock_guard<std::mutex> lk(m_);
                if (slot < 0) {   // the job fails alone (e.g. its film did not fit)
                    j->state = GND_JOB_FAILED;
                    j->status = code;
                    j->error = why;
                    j->tDone = nowMs();
                    if (--c_->sceneUse[j->scene] <= 0) c_->sceneUse.erase(j->scene);
                    doneCv_.notify_all();
                    continue;
                }
                j->slot = slot;
                j->firstRound = enqRound_;   // the next round queued is the first to include it
                j->state = GND_JOB_RUNNING;
                j->tAdmit = nowMs();
                running_.push_back(j);
            }
            std::vector<ServeJob*> run;
            bool blocked = false;
            {
                std::lock_guard<std::mutex> lk(m_);
                run = running_;
                blocked = run.empty() && !queue_.empty();
            }
            if (blocked) {
                // the queue head does not fit although nothing runs (the budget was lowered
                // or other memory is in use): look again shortly
                backoff = true;
                continue;
            }
            if (run.empty()) continue;
            int mix = 0;
            bool hasNull = false;
            for (ServeJob* j : run) {
                mix |= j->integ == 1 ? 2 : 1;
                if (j->integ == 0 && c_->scene(j->scene).hasNullMaterials) hasNull = true;
            }
            const int iters = std::min(std::max(c_->serveTune.roundIters & ~1, 2), 64);
            applyPriorities(run);   // newly admitted jobs take their place before the next round
            Wavefront::Result acc;
            auto enqueue = [&]() {
                const int slot = inflight_ ? (inflightSlot_ ^ 1) : inflightSlot_;
                wf.enqueueRound(iters, mix, hasNull, 0, acc, slot);
                slotRound_[slot] = enqRound_++;
                inflightSlot_ = slot;
                inflight_ = true;
            };
            if (!inflight_) enqueue();
            const int readSlot = inflightSlot_;
            enqueue();   // the next round runs while this one's counters are read
            const Wavefront::Snapshot& sn = wf.waitRound(readSlot);
            const int64_t q = slotRound_[readSlot];
            if (sn.err) c_->checkKernelErrors("serve");
            std::vector<JobCtl> ctl(sn.ctl, sn.ctl + kMaxJobs);
            uint64_t retiredSum = 0;
            for (ServeJob* j : run) {
                if (q < j->firstRound) continue;   // a round queued before the job's admission
                const JobCtl& k = ctl[j->slot];
                retiredSum += k.retired;
                bool cancelNow = false;
                {
                    std::lock_guard<std::mutex> lk(m_);
                    j->done = k.retired;
                    cancelNow = j->cancelReq && j->stopRound < 0;
                }
                if (cancelNow) {
                    wf.stop(j->slot);        // stream-ordered after the round in flight
                    j->stopRound = enqRound_;   // rounds from here on see the final hand-out
                    continue;
                }
                if (j->stopRound >= 0) {
                    if (q >= j->stopRound) {
                        const uint64_t handed = std::min<uint64_t>(k.next, j->total);
                        if (k.retired >= handed) finishJob(j, GND_JOB_CANCELLED);
                    }
                } else if (k.retired >= j->total) {
                    finishJob(j, GND_JOB_DONE);
                }
            }
            // sample rate of the server (retired samples per ms of round), for deadlines
            const double now = nowMs();
            // from the engine's own count of retired paths over windows of at least 50 ms
            // (rounds read back to back would give meaningless rates); the count restarts
            // when the pool is reset, and an idle gap starts a new window
            if (lastRoundMs_ < 0.0 || sn.retiredAll < lastRetiredAll_ || now - lastRoundMs_ > 500.0) {
                lastRoundMs_ = now;
                lastRetiredAll_ = sn.retiredAll;
            } else if (now - lastRoundMs_ >= 50.0) {
                rate_ = 0.7 * rate_ + 0.3 * (double)(sn.retiredAll - lastRetiredAll_) / (now - lastRoundMs_);
                lastRoundMs_ = now;
                lastRetiredAll_ = sn.retiredAll;
            }
            lastCtl_ = ctl;
            lastRound_ = q;
            if (retiredSum != lastRetiredSum_) {
                lastRetiredSum_ = retiredSum;
                itersSinceProgress_ = 0;
            } else if ((itersSinceProgress_ += iters) > kStallIters) {
                failRunning("no sample retired in " + std::to_string(kStallIters) + " iterations", GND_ERR_DEVICE_CHECK);
                itersSinceProgress_ = 0;
            }
        } catch (const Error& e) {
            failRunning(e.what(), e.code);
            drainPipeline();
        } catch (const std::exception& e) {
            failRunning(e.what(), GND_ERR_CUDA);
            drainPipeline();
        }
    }
}

// Hand-out order of the running jobs for the rounds queued next (FIFO: admission order,
// set at admission). Counters come from the last snapshot that includes the job; a job
// admitted since has handed out nothing.
void Server::applyPriorities(const std::vector<ServeJob*>& run) {
    if (policy_ == GND_SERVE_FIFO) return;
    std::vector<std::pair<int, uint64_t>> keys;
    for (ServeJob* j : run) {
        if (policy_ == GND_SERVE_SRPT) {
            // the job with the fewest samples left to hand out first
            const bool seen = lastRound_ >= j->firstRound && j->slot >= 0 && (size_t)j->slot < lastCtl_.size();
            const uint64_t handed = seen ? std::min<uint64_t>(lastCtl_[j->slot].next, j->total) : 0;
            keys.emplace_back(j->slot, j->total - handed);
        } else {
            // earliest deadline first (microseconds of the server clock)
            const double deadline = j->tSubmit + kDeadlineSlack * (double)j->total / std::max(rate_, 1.0);
            keys.emplace_back(j->slot, (uint64_t)(deadline * 1000.0));
        }
    }
    c_->wave->setPriorities(keys);
}

// After a failure: wait for whatever is queued (ignoring its errors) and restart the
// round pipeline.
void Server::drainPipeline() {
    cudaStreamSynchronize(c_->stream);
    cudaGetLastError();
    inflight_ = false;
    slotRound_[0] = slotRound_[1] = -1;
}

void Server::setPolicy(int policy) {
    if (policy != GND_SERVE_FIFO && policy != GND_SERVE_SRPT && policy != GND_SERVE_DEADLINE)
        throw Error(GND_ERR_INVALID, "unknown serving policy");
    std::lock_guard<std::mutex> lk(m_);
    policy_ = policy;
}

Server& serverOf(Context* c) {
    if (!c->server) c->server = std::make_unique<Server>(c);
    return *c->server;
}

}  // namespace gnd

using namespace gnd;

extern "C" {

gnd_status gnd_gpu_set_hbm_budget(gnd_gpu_ctx* ctxh, uint64_t bytes) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        std::lock_guard<FairMutex> lk(c->mu);
        c->hbmBudget = bytes;
    });
}

gnd_status gnd_gpu_serve_policy(gnd_gpu_ctx* ctxh, int32_t policy) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        c->bind();
        std::lock_guard<std::mutex> lk(c->serverMu);
        serverOf(c).setPolicy(policy);
    });
}

gnd_status gnd_gpu_serve_submit(gnd_gpu_ctx* ctxh, const gnd_job_desc* job, gnd_job_id* id) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!job || !id) throw Error(GND_ERR_INVALID, "null job description or id");
        c->bind();
        Server* s;
        {
            std::lock_guard<std::mutex> lk(c->serverMu);
            s = &serverOf(c);
        }
        *id = s->submit(*job);
    });
}

gnd_status gnd_gpu_serve_poll(gnd_gpu_ctx* ctxh, gnd_job_id id, gnd_job_status* st) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        std::lock_guard<std::mutex> lk(c->serverMu);
        if (!c->server) throw Error(GND_ERR_INVALID, "unknown job id " + std::to_string(id));
        c->server->poll(id, st);
    });
}

gnd_status gnd_gpu_serve_wait(gnd_gpu_ctx* ctxh, gnd_job_id id, float* film, gnd_job_status* st, int64_t timeoutMs) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        Server* s;
        {
            std::lock_guard<std::mutex> lk(c->serverMu);
            if (!c->server) throw Error(GND_ERR_INVALID, "unknown job id " + std::to_string(id));
            s = c->server.get();
        }
        std::string err;
        gnd_status r = s->wait(id, film, st, timeoutMs, err);
        if (r != GND_OK) throw Error(r, err);
    });
}

gnd_status gnd_gpu_serve_cancel(gnd_gpu_ctx* ctxh, gnd_job_id id) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        std::lock_guard<std::mutex> lk(c->serverMu);
        if (!c->server) throw Error(GND_ERR_INVALID, "unknown job id " + std::to_string(id));
        c->server->cancel(id);
    });
}

}  // extern "C"
