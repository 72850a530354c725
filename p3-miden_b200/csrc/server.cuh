// Batched and served proving: a pool of workers on one device, each with its
// own context (stream, twiddle cache), pulling jobs from one queue.
//
// Admission: a job is admitted while its estimated HBM footprint fits in the
// budget still free (always when nothing else runs, so an oversized job
// cannot starve), and at most one heavy job (job_is_heavy) runs at a time
// (set_max_heavy changes the limit).
// Jobs are taken in arrival order, except that light jobs may pass a heavy
// job that waits for the running heavy one: they fill the GPU time the
// heavy job leaves idle in its latency-bound phases. A worker keeps its job's LDEs,
// trees and FRI layers on the device for the whole proof; the device
// interleaves the kernels of up to n_workers proofs, and one proof's host
// work (transcript, challenges) overlaps the others' device work.
// A failing job (validation or device error) reports its own status; the
// other jobs are unaffected.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

#include "prover.cuh"
#include "verifier.cuh"

namespace p3g {

// Upper bound of the device bytes prove() allocates for a job.
inline uint64_t job_footprint_bytes(const PcsParams &pcs, const Instance *inst, size_t n) {
    const uint64_t B = 1ull << pcs.log_blowup;
    uint64_t D = 1;
    for (size_t i = 0; i < n; i++) D = std::max<uint64_t>(D, 1ull << inst_log_qd(inst[i]));
    uint64_t words = 0, max_hw = 0, hmax = 0, cm_words = 0;
    for (size_t i = 0; i < n; i++) {
        const uint64_t hw = inst[i].height * inst[i].width, aw2 = 2 * inst_aux_width(inst[i]);
        if (inst[i].air == AIR_SYMBOLIC)  // column-major copies of gJ's rows for the generated kernels
            cm_words += (inst[i].height << inst_log_qd(inst[i])) * (inst[i].width + aw2);
        if (!inst[i].trace_on_device) words += hw;  // uploaded trace
        words += hw * B;                             // main LDE
        words += inst[i].height * aw2 * (B + 1);     // aux trace + LDE
        max_hw = std::max(max_hw, inst[i].height * std::max<uint64_t>(inst[i].width, aw2));
        hmax = std::max(hmax, inst[i].height);
    }
    max_hw = std::max(max_hw, hmax * 2 * D);
    const uint64_t nl = hmax * B;
    words += max_hw;             // iNTT scratch
    words += cm_words;           // symbolic AIRs: column-major LDE rows
    words += 2 * hmax * D;       // quotient accumulator
    words += nl * 2 * D;         // quotient LDE
    words += 4 * nl;             // DEEP point quotients
    words += 4 * nl * 4;         // tree digest layers (3 trees + FRI), upper bound
    words += 2 * nl * 3;         // DEEP row dots, layer, FRI layers
    words += 4 * nl / B;         // barycentric weights
    return words * 8 + (64ull << 20);  // plus tables and slack
}

// A job is heavy when its LDEs alone hold more than 2^26 words (512 MB):
// its transforms and hashes fill the GPU, so a second heavy job running at
// the same time only competes for the same integer pipes and L2.
constexpr uint64_t kHeavyLdeWords = 1ull << 26;
inline bool job_is_heavy(const PcsParams &pcs, const Instance *inst, size_t n) {
    uint64_t words = 0;
    for (size_t i = 0; i < n; i++) words += (inst[i].height << pcs.log_blowup) * inst[i].width;
    return words > kHeavyLdeWords;
}

struct ServerJob {
    PcsParams pcs;
    std::vector<Instance> inst;
    double arrival_s = 0;  // seconds after serve() starts
    // results
    int status = -1;
    ProofOut out;
    int verdict = -1;      // self-check verdict (vfy::Verdict), -1 when not checked
    double verify_ms = 0;  // self-check wall time
    double submit_s = 0, start_s = 0, end_s = 0;
    std::string error;
};

class Server {
   public:
    Server(int device, const uint64_t *p2, uint32_t n_workers, uint64_t hbm_budget)
        : device_(device), budget_(hbm_budget) {
        CK(cudaSetDevice(device));
        for (uint32_t w = 0; w < n_workers; w++) {
            auto c = std::make_unique<Ctx>();
            c->device = device;
            CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            c->make_pool();
            // a worker's pool keeps at most its share of the budget between
            // jobs; memory above it goes back to the device at the next
            // synchronisation, so the workers' pools together stay within
            // the budget the admission rule assumes
            uint64_t share = hbm_budget / n_workers;
            CK(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &share));
            memcpy(c->p2, p2, sizeof(c->p2));
            ctxs_.push_back(std::move(c));
        }
        bind_p2(*ctxs_[0]);
        t0_ = std::chrono::steady_clock::now();
        for (uint32_t w = 0; w < n_workers; w++) workers_.emplace_back([this, w] { worker(w); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
        for (auto &c : ctxs_) c->release();
    }
    double now_s() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }
    // Enqueue a job; the caller keeps `job` (and its traces) alive until done.
    void submit(ServerJob *job) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            job->submit_s = now_s();
            job->status = -1;
            queue_.push_back(job);
            pending_++;
        }
        cv_.notify_all();
    }
    void wait(ServerJob *job) {
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return job->status >= 0; });
    }
    void wait_all() {
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }
    uint64_t peak_bytes() const { return peak_; }
    // Verify each proof on the device before returning it (vfy::verify, on
    // the worker's own stream); a rejected proof ends its job with
    // ERR_REJECTED.
    void set_self_check(bool on) { self_check_ = on; }
    // Tuned launch shapes for every worker (p3g_autotune_*); call before
    // submitting jobs.
    void set_lde_split(uint32_t log_h, const std::vector<uint32_t> &sizes) {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto &c : ctxs_) {
            if (sizes.empty()) c->lde_split.erase(log_h);
            else c->lde_split[log_h] = sizes;
        }
    }
    void set_slab_columns(uint64_t cols) {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto &c : ctxs_) c->slab_cols = cols;
    }
    // At most n heavy jobs at a time (0: no limit; default 1).
    void set_max_heavy(uint32_t n) {
        std::lock_guard<std::mutex> lk(mu_);
        max_heavy_ = n ? n : UINT32_MAX;
    }

   private:
    void worker(uint32_t w) {
        cudaSetDevice(device_);
        Ctx &ctx = *ctxs_[w];
        for (;;) {
            ServerJob *job = nullptr;
            uint64_t fp = 0;
            bool heavy = false;
            {
                std::unique_lock<std::mutex> lk(mu_);
                // first admissible job in arrival order (see the admission rule above)
                auto pick = [&]() -> std::deque<ServerJob *>::iterator {
                    for (auto it = queue_.begin(); it != queue_.end(); ++it) {
                        ServerJob *j = *it;
                        const uint64_t f = job_footprint_bytes(j->pcs, j->inst.data(), j->inst.size());
                        const bool h = job_is_heavy(j->pcs, j->inst.data(), j->inst.size());
                        const bool fits = in_use_ == 0 || in_use_ + f <= budget_;
                        if (fits && !(h && heavy_running_ >= max_heavy_)) return it;
                        if (!fits && !h) break;  // keep arrival order among light jobs when memory is short
                    }
                    return queue_.end();
                };
                std::deque<ServerJob *>::iterator it;
                cv_.wait(lk, [&] {
                    if (stop_) return true;
                    it = pick();
                    return it != queue_.end();
                });
                if (stop_ && queue_.empty()) return;
                it = pick();
                if (it == queue_.end()) continue;
                job = *it;
                queue_.erase(it);
                fp = job_footprint_bytes(job->pcs, job->inst.data(), job->inst.size());
                heavy = job_is_heavy(job->pcs, job->inst.data(), job->inst.size());
                if (heavy) heavy_running_++;
                in_use_ += fp;
                peak_ = std::max(peak_, in_use_);
            }
            job->start_s = now_s();
            int st = OK;
            try {
                bind_p2(ctx);
                prove(ctx, job->pcs, job->inst.data(), job->inst.size(), job->out);
                if (self_check_) {
                    const auto v0 = std::chrono::steady_clock::now();
                    const ProofOut &o = job->out;
                    job->verdict = vfy::verify(ctx, job->pcs, job->inst.data(), job->inst.size(), o.fields.data(),
                                               o.fields.size(), o.commits.data(), o.commits.size() / 4, o.digest,
                                               nullptr);
                    job->verify_ms =
                        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - v0).count();
                    if (job->verdict != vfy::ACCEPT) {
                        st = ERR_REJECTED;
                        job->error = "self-check rejected the proof (verdict " + std::to_string(job->verdict) + ")";
                    }
                }
            } catch (const CudaError &e) {
                st = e.status;
                job->error = e.what;
                cudaStreamSynchronize(ctx.stream);
                cudaGetLastError();
            } catch (const std::bad_alloc &) {
                st = ERR_OOM;
                job->error = "host allocation failed";
            }
            // the workspace is part of the job's footprint: give it back to the
            // worker's pool, which keeps memory only within its budget share
            ctx.ws.release();
            job->end_s = now_s();
            {
                std::lock_guard<std::mutex> lk(mu_);
                in_use_ -= fp;
                if (heavy) heavy_running_--;
                job->status = st;
                pending_--;
            }
            cv_.notify_all();
            done_cv_.notify_all();
        }
    }

    int device_;
    uint64_t budget_;
    std::vector<std::unique_ptr<Ctx>> ctxs_;
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<ServerJob *> queue_;
    uint64_t in_use_ = 0, peak_ = 0;
    uint32_t heavy_running_ = 0, max_heavy_ = 1;
    uint64_t pending_ = 0;
    bool stop_ = false;
    std::atomic<bool> self_check_{false};
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace p3g
