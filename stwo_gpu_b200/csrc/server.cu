// Proof server: continuous batching of wide-Fibonacci proof jobs on one GPU.
//
// Jobs are submitted at any time and queue in arrival order. A job is admitted when a
// worker is free and its device-memory bound (stwo_wide_fib_prove_device_bytes) fits
// in what the budget has left; a job that does not fit lets later, smaller jobs pass
// (backfill), so one large job does not idle the device. Each worker is a host thread
// with its own CUDA stream; a job keeps its trace, twiddle references, trees and FRI
// layers on the device from the trace commitment to the last decommitment, and its
// kernels interleave on the device with the other admitted jobs' kernels while its
// thread waits on the channel. All jobs share one twiddle tree, built at creation for
// the largest domain the server accepts. A job's proof bytes do not depend on what
// else is running: each job's arithmetic is confined to its own buffers and stream.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "prover.cuh"

namespace stwo {

namespace {

double steady_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct PendingJob {
    uint64_t id = 0;
    stwo_wide_fib_job job{};
    std::vector<uint32_t> a0, a1;           // host copies, or
    const uint32_t *a0_dev = nullptr, *a1_dev = nullptr;  // caller-owned device inputs
    uint64_t bytes;
    double submit_ms;
};

}  // namespace
}  // namespace stwo

using namespace stwo;

struct stwo_prover_server {
    int device = 0;
    uint64_t budget = 0, in_use = 0;
    uint32_t max_domain_log = 0;
    uint32_t *tw = nullptr, *itw = nullptr;
    uint64_t tree_size = 0;
    bool stopping = false;
    bool paused = false;          // workers start no job while set (stwo_server_pause)
    double queue_timeout_ms = 0;  // 0: queued jobs wait without limit
    bool blocking_wait = true;  // workers yield their core while waiting on the device...
    uint32_t spin_us = 2000;    // ...after polling this long
    bool use_priorities = true; // per-job stream priority by job size
    bool use_graphs = true;     // same-shape jobs reuse a worker's slab and proof graph
    uint32_t batch_max = 32;       // queued jobs of one shape proved in one launch sequence
    uint32_t batch_max_log = 16;   // ...for jobs of at most 2^batch_max_log trace rows
    std::atomic<uint64_t> batches{0}, batched_jobs{0};
    std::atomic<uint64_t> slab_reuses{0}, graph_replays{0};
    cudaStream_t epoch_stream = nullptr;  // idle stream for the device epoch
    cudaEvent_t epoch = nullptr;          // timing event: device time zero of device_done_ms
    std::atomic<bool> epoch_set{false};
    uint32_t running = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<PendingJob> pending;
    std::deque<stwo_server_result> done;
    std::vector<std::thread> workers;

    // A finished result for a job that never ran (cancelled or timed out).
    void post_unrun(const PendingJob &j, int status, const char *msg) {
        stwo_server_result r{};
        r.job_id = j.id;
        r.status = status;
        strncpy(r.error, msg, sizeof(r.error) - 1);
        r.submit_ms = j.submit_ms;
        r.start_ms = r.done_ms = steady_ms();
        r.device_done_ms = -1.0;
        done.push_back(r);
    }

    // Queued jobs past the queue timeout leave the queue with STWO_ERR_TIMEOUT (mu held).
    bool expire() {
        if (queue_timeout_ms <= 0) return false;
        const double now = steady_ms();
        bool any = false;
        for (auto it = pending.begin(); it != pending.end();) {
            if (now - it->submit_ms > queue_timeout_ms) {
                post_unrun(*it, STWO_ERR_TIMEOUT, "job waited in the queue past the server's queue timeout");
                it = pending.erase(it);
                any = true;
            } else {
                ++it;
            }
        }
        return any;
    }

    // The first pending job (in arrival order) whose bound fits the budget's remainder.
    bool take(PendingJob &out) {
        if (expire()) cv_done.notify_all();
        for (auto it = pending.begin(); it != pending.end(); ++it) {
            if (in_use + it->bytes <= budget) {
                out = std::move(*it);
                pending.erase(it);
                in_use += out.bytes;
                return true;
            }
        }
        return false;
    }

    // Stream priority of a job: smaller jobs get higher priority, so that the short
    // kernel chains of small jobs take free SM slots ahead of the queued CTAs of large
    // transforms instead of waiting behind them. Class 0 (the highest) holds jobs of up
    // to 2^16 trace cells; each further class doubles the bound twice.
    static bool same_shape(const stwo_wide_fib_job &a, const stwo_wide_fib_job &b) {
        return a.log_n_rows == b.log_n_rows && a.n_columns == b.n_columns && a.log_blowup == b.log_blowup &&
               a.n_queries == b.n_queries && a.pow_bits == b.pow_bits;
    }

    static uint32_t priority_class(const stwo_wide_fib_job &j, uint32_t n_classes) {
        uint32_t ln = 0;
        while ((1u << ln) < j.n_columns) ln++;
        const uint32_t w = j.log_n_rows + ln;
        const uint32_t c = w <= 16 ? 0 : (w - 15) / 2;
        return std::min(c, n_classes - 1);
    }

    // Proves j and the jobs of `more` (one shape) in one launch sequence and posts a
    // result per job; every result carries the sequence's stats.
    void prove_batch(const PendingJob &j, const std::vector<PendingJob> &more, cudaStream_t st) {
        std::vector<const PendingJob *> jobs{&j};
        for (auto &b : more) jobs.push_back(&b);
        const uint32_t k = (uint32_t)jobs.size();
        std::vector<const uint32_t *> a0(k), a1(k);
        for (uint32_t i = 0; i < k; i++) {
            a0[i] = jobs[i]->a0_dev ? jobs[i]->a0_dev : jobs[i]->a0.data();
            a1[i] = jobs[i]->a1_dev ? jobs[i]->a1_dev : jobs[i]->a1.data();
        }
        const double start = steady_ms();
        clear_error();
        std::vector<std::vector<uint8_t>> proofs;
        std::vector<int> rc(k, STWO_OK);
        stwo_prove_stats stats{};
        const int brc = wide_fib_prove_batch(&j.job, k, a0.data(), a1.data(), tw, itw, tree_size, proofs, rc.data(),
                                             &stats, st);
        const std::string err = brc ? stwo_last_error() : "";
        batches++;
        batched_jobs += k;
        double device_done = -1.0;
        if (brc == STWO_OK && epoch_set.load()) {
            float ms = 0.f;
            cudaEvent_t ev = last_wait_event();
            if (ev && cudaEventElapsedTime(&ms, epoch, ev) == cudaSuccess) device_done = ms;
            else cudaGetLastError();
        }
        const double end = steady_ms();
        std::lock_guard<std::mutex> lock(mu);
        for (uint32_t i = 0; i < k; i++) {
            stwo_server_result r{};
            r.job_id = jobs[i]->id;
            r.submit_ms = jobs[i]->submit_ms;
            r.start_ms = start;
            r.done_ms = end;
            r.stats = stats;
            r.status = brc ? brc : rc[i];
            r.device_done_ms = r.status == STWO_OK ? device_done : -1.0;
            if (r.status == STWO_OK) {
                r.proof = static_cast<uint8_t *>(malloc(proofs[i].size()));
                if (r.proof) {
                    memcpy(r.proof, proofs[i].data(), proofs[i].size());
                    r.proof_len = proofs[i].size();
                } else {
                    r.status = STWO_ERR_OUT_OF_MEMORY;
                }
            }
            if (r.status != STWO_OK)
                strncpy(r.error, brc ? err.c_str() : "proof of the batch failed", sizeof(r.error) - 1);
            done.push_back(r);
        }
        expire();
    }

    void worker() {
        cudaSetDevice(device);
        t_blocking_wait = blocking_wait;
        t_spin_us = spin_us;
        // One stream per priority level, greatest priority first.
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (!use_priorities) greatest = least;
        std::vector<cudaStream_t> streams;
        cudaError_t se = cudaSuccess;
        for (int pr = greatest; pr <= least && se == cudaSuccess; pr++) {
            cudaStream_t s = nullptr;
            se = cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, pr);
            if (se == cudaSuccess) streams.push_back(s);
        }
        // The slab of this worker's last proof, kept while the next job it takes has the
        // same shape: that job reuses every buffer at the same address and, from the
        // second reuse on, replays the proof's launch sequence as one CUDA graph.
        ProveCache cache;
        cudaStream_t cache_st = nullptr;
        PendingJob j;
        bool have_next = false;
        for (;;) {
            if (!have_next) {
                bool got = false;
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait(lock, [&] { return stopping || (!paused && !pending.empty() && (got = take(j))); });
                if (!got) break;  // stopping, nothing taken
                running++;
            }
            have_next = false;
            // Queued jobs of this job's shape join it in one launch sequence while they
            // are the jobs that arrival-order admission would take next.
            std::vector<PendingJob> batch;
            if (se == cudaSuccess && batch_max > 1 && j.job.log_n_rows <= batch_max_log) {
                std::lock_guard<std::mutex> lock(mu);
                for (auto it = pending.begin(); it != pending.end() && batch.size() + 1 < batch_max;) {
                    if (in_use + it->bytes > budget) {  // admission would pass it as well
                        ++it;
                        continue;
                    }
                    if (!same_shape(it->job, j.job) || it->bytes != j.bytes) break;
                    in_use += it->bytes;
                    batch.push_back(std::move(*it));
                    it = pending.erase(it);
                }
            }
            if (!batch.empty()) {
                if (cache.valid) prove_cache_release(&cache, cache_st);  // the batch plans its own slabs
                prove_batch(j, batch, streams[priority_class(j.job, (uint32_t)streams.size())]);
                {
                    std::lock_guard<std::mutex> lock(mu);
                    in_use -= j.bytes;
                    for (auto &b : batch) in_use -= b.bytes;
                    running--;
                }
                cv_done.notify_all();
                cv_work.notify_all();
                continue;
            }
            stwo_server_result r{};
            r.job_id = j.id;
            r.submit_ms = j.submit_ms;
            r.start_ms = steady_ms();
            std::vector<uint8_t> proof;
            if (se != cudaSuccess) {
                r.status = set_error(STWO_ERR_CUDA, "worker stream creation failed: %s", cudaGetErrorString(se));
            } else {
                clear_error();
                const uint32_t *a0 = j.a0_dev ? j.a0_dev : j.a0.data(), *a1 = j.a1_dev ? j.a1_dev : j.a1.data();
                cudaStream_t st = streams[priority_class(j.job, (uint32_t)streams.size())];
                const bool reuse = cache.valid;  // set only while this job has the cached shape
                const uint64_t replays0 = cache.replays;
                r.status = wide_fib_prove(&j.job, a0, a1, tw, itw, tree_size, proof, &r.stats, st,
                                          use_graphs ? &cache : nullptr);
                cache_st = st;
                if (reuse && r.status == STWO_OK) {
                    slab_reuses++;
                    if (cache.replays > replays0) graph_replays++;
                }
            }
            if (r.status == STWO_OK) {
                r.proof = static_cast<uint8_t *>(malloc(proof.size()));
                if (r.proof) {
                    memcpy(r.proof, proof.data(), proof.size());
                    r.proof_len = proof.size();
                } else {
                    r.status = STWO_ERR_OUT_OF_MEMORY;
                }
            } else {
                strncpy(r.error, stwo_last_error(), sizeof(r.error) - 1);
            }
            r.done_ms = steady_ms();
            r.device_done_ms = -1.0;
            if (r.status == STWO_OK && epoch_set.load()) {
                // The prover's last wait recorded an event after its final device work.
                float ms = 0.f;
                cudaEvent_t ev = last_wait_event();
                if (ev && cudaEventElapsedTime(&ms, epoch, ev) == cudaSuccess) r.device_done_ms = ms;
                else cudaGetLastError();
            }
            // A queued job of the same shape takes this one's place (and budget) at once, if
            // it is the job that admission in arrival order would take next with this job's
            // budget released: a job queued ahead of it that would fit goes first, so a
            // run of same-shape arrivals cannot hold back an earlier job of another shape.
            PendingJob next;
            {
                std::lock_guard<std::mutex> lock(mu);
                done.push_back(r);
                expire();
                if (cache.valid && !stopping && !paused)
                    for (auto it = pending.begin(); it != pending.end(); ++it) {
                        if (in_use - j.bytes + it->bytes > budget) continue;  // admission would pass it
                        if (same_shape(it->job, j.job) && it->bytes == j.bytes) {
                            next = std::move(*it);
                            pending.erase(it);
                            have_next = true;
                        }
                        break;
                    }
            }
            cv_done.notify_all();
            if (have_next) {
                j = std::move(next);
                continue;
            }
            // Free the retained slab before its bytes go back to the budget.
            if (cache.valid) prove_cache_release(&cache, cache_st);
            {
                std::lock_guard<std::mutex> lock(mu);
                in_use -= j.bytes;
                running--;
            }
            cv_work.notify_all();  // freed budget may admit waiting jobs
        }
        if (cache.valid) prove_cache_release(&cache, cache_st);
        for (cudaStream_t s : streams) cudaStreamDestroy(s);
    }
};

extern "C" {

double stwo_server_now_ms(void) { return steady_ms(); }

stwo_prover_server *stwo_server_create(uint32_t n_workers, uint64_t device_budget_bytes, uint32_t max_domain_log) {
    clear_error();
    if (n_workers == 0 || n_workers > 256 || max_domain_log < 4 || max_domain_log > 28) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "server needs 1..256 workers and a domain log size in 4..28");
        return nullptr;
    }
    auto *s = new stwo_prover_server();
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        set_error(STWO_ERR_CUDA, "no CUDA device");
        delete s;
        return nullptr;
    }
    s->budget = device_budget_bytes;
    if (const char *w = getenv("STWO_SERVER_WAIT")) s->blocking_wait = strcmp(w, "spin") != 0;
    if (const char *w = getenv("STWO_SERVER_SPIN_US")) s->spin_us = (uint32_t)strtoul(w, nullptr, 10);
    if (const char *w = getenv("STWO_SERVER_PRIORITY")) s->use_priorities = strcmp(w, "0") != 0;
    if (const char *w = getenv("STWO_SERVER_GRAPHS")) s->use_graphs = strcmp(w, "0") != 0;
    if (const char *w = getenv("STWO_SERVER_BATCH"))
        s->batch_max = (uint32_t)std::min<unsigned long>(256, std::max<unsigned long>(1, strtoul(w, nullptr, 10)));
    if (const char *w = getenv("STWO_SERVER_BATCH_MAX_LOG")) s->batch_max_log = (uint32_t)strtoul(w, nullptr, 10);
    s->max_domain_log = max_domain_log;
    // One twiddle tree for CanonicCoset(max_domain_log).half_coset serves every smaller
    // canonic domain: its doublings are the smaller domains' half cosets.
    s->tree_size = 1ull << (max_domain_log - 1);
    if (cudaMalloc(&s->tw, s->tree_size * 4) != cudaSuccess || cudaMalloc(&s->itw, s->tree_size * 4) != cudaSuccess) {
        set_error(STWO_ERR_OUT_OF_MEMORY, "server twiddle tree allocation failed");
        cudaFree(s->tw);
        delete s;
        return nullptr;
    }
    const uint32_t init = 1u << (30 - max_domain_log);
    const uint32_t step = (uint32_t)((1ull << (32 - max_domain_log)) & 0x7fffffffu);
    if (stwo_precompute_twiddles(init, step, max_domain_log - 1, s->tw, s->itw, nullptr) != STWO_OK ||
        cudaStreamSynchronize(0) != cudaSuccess) {
        cudaFree(s->tw);
        cudaFree(s->itw);
        delete s;
        return nullptr;
    }
    // Map the budget into the library's pool now (bounded by the free memory), so
    // admitted jobs never wait on the driver to back new allocations.
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const uint64_t margin = 2ull << 30;
        const uint64_t want = std::min<uint64_t>(device_budget_bytes, free_b > margin ? free_b - margin : 0);
        if (reserve_pool(want) != STWO_OK) clear_error();  // a smaller pool only costs speed
    }
    if (cudaStreamCreateWithFlags(&s->epoch_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->epoch) != cudaSuccess) {
        set_error(STWO_ERR_CUDA, "server epoch event creation failed");
        if (s->epoch_stream) cudaStreamDestroy(s->epoch_stream);
        cudaFree(s->tw);
        cudaFree(s->itw);
        delete s;
        return nullptr;
    }
    for (uint32_t i = 0; i < n_workers; i++) s->workers.emplace_back([s] { s->worker(); });
    return s;
}

namespace {
// Checks a job against the server before anything is copied: its parameters, its
// domain against the shared twiddle tree, its device bound against the budget.
int validate_job(stwo_prover_server *s, const stwo_wide_fib_job &job, uint64_t *bytes_out) {
    STWO_REQUIRE(job.log_n_rows <= 30 && job.log_blowup <= 30 &&
                     job.log_n_rows + 1 + job.log_blowup <= s->max_domain_log,
                 STWO_ERR_UNSUPPORTED_SIZE, "job domain log size %u exceeds the server's %u",
                 job.log_n_rows + 1 + job.log_blowup, s->max_domain_log);
    const uint64_t bytes = wide_fib_job_device_bytes(&job, false);
    STWO_REQUIRE(bytes, STWO_ERR_UNSUPPORTED_SIZE, "job parameters unsupported");
    STWO_REQUIRE(bytes <= s->budget, STWO_ERR_OUT_OF_MEMORY, "job needs %llu device bytes, budget is %llu",
                 (unsigned long long)bytes, (unsigned long long)s->budget);
    *bytes_out = bytes;
    return STWO_OK;
}

int submit_job(stwo_prover_server *s, PendingJob &&j) {
    j.submit_ms = steady_ms();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        STWO_REQUIRE(!s->stopping, STWO_ERR_INVALID_ARGUMENT, "server is shutting down");
        s->pending.push_back(std::move(j));
    }
    s->cv_work.notify_one();
    return STWO_OK;
}
}  // namespace

int stwo_server_submit(stwo_prover_server *s, uint64_t job_id, const stwo_wide_fib_job *job, const uint32_t *a0,
                       const uint32_t *a1) {
    STWO_REQUIRE(s && job && a0 && a1, STWO_ERR_INVALID_ARGUMENT, "null argument");
    PendingJob j;
    int rc = validate_job(s, *job, &j.bytes);  // before copying 2^log_n_rows words of each input
    if (rc) return rc;
    j.id = job_id;
    j.job = *job;
    const size_t rows = 1ull << job->log_n_rows;
    j.a0.assign(a0, a0 + rows);
    j.a1.assign(a1, a1 + rows);
    return submit_job(s, std::move(j));
}

int stwo_server_submit_device(stwo_prover_server *s, uint64_t job_id, const stwo_wide_fib_job *job,
                              const uint32_t *a0_dev, const uint32_t *a1_dev) {
    STWO_REQUIRE(s && job && a0_dev && a1_dev, STWO_ERR_INVALID_ARGUMENT, "null argument");
    PendingJob j;
    int rc = validate_job(s, *job, &j.bytes);
    if (rc) return rc;
    j.id = job_id;
    j.job = *job;
    j.a0_dev = a0_dev;
    j.a1_dev = a1_dev;
    return submit_job(s, std::move(j));
}

uint32_t stwo_server_poll(stwo_prover_server *s, stwo_server_result *out, uint32_t max_results, int32_t timeout_ms) {
    if (!s || !out || max_results == 0) return 0;
    std::unique_lock<std::mutex> lock(s->mu);
    auto ready = [&] { return !s->done.empty() || (s->pending.empty() && s->running == 0); };
    if (s->queue_timeout_ms > 0) {
        // With a queue timeout, jobs may expire while every worker is busy: check every
        // few milliseconds while waiting.
        const double until = timeout_ms < 0 ? 1e300 : steady_ms() + timeout_ms;
        for (;;) {
            s->expire();
            if (ready() || steady_ms() >= until) break;
            s->cv_done.wait_for(lock, std::chrono::milliseconds(2));
        }
    } else if (timeout_ms < 0) {
        s->cv_done.wait(lock, ready);
    } else if (timeout_ms > 0) {
        s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready);
    }
    uint32_t n = 0;
    while (n < max_results && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    return n;
}

void stwo_server_stats(stwo_prover_server *s, uint32_t *pending, uint32_t *running, uint64_t *device_bytes_in_use) {
    if (!s) return;
    std::lock_guard<std::mutex> lock(s->mu);
    if (pending) *pending = (uint32_t)s->pending.size();
    if (running) *running = s->running;
    if (device_bytes_in_use) *device_bytes_in_use = s->in_use;
}

int stwo_server_mark_epoch(stwo_prover_server *s) {
    STWO_REQUIRE(s, STWO_ERR_INVALID_ARGUMENT, "null server");
    int prev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&prev));
    STWO_CUDA_TRY(cudaSetDevice(s->device));
    cudaError_t e = cudaEventRecord(s->epoch, s->epoch_stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(s->epoch);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return set_error(STWO_ERR_CUDA, "server epoch: %s", cudaGetErrorString(e));
    s->epoch_set.store(true);
    return STWO_OK;
}

void stwo_server_batch_stats(stwo_prover_server *s, uint64_t *batches, uint64_t *batched_jobs) {
    if (batches) *batches = s ? s->batches.load() : 0;
    if (batched_jobs) *batched_jobs = s ? s->batched_jobs.load() : 0;
}

void stwo_server_graph_stats(stwo_prover_server *s, uint64_t *slab_reuses, uint64_t *graph_replays) {
    if (!s) return;
    if (slab_reuses) *slab_reuses = s->slab_reuses.load();
    if (graph_replays) *graph_replays = s->graph_replays.load();
}

int stwo_server_cancel(stwo_prover_server *s, uint64_t job_id) {
    STWO_REQUIRE(s, STWO_ERR_INVALID_ARGUMENT, "null server");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = std::find_if(s->pending.begin(), s->pending.end(), [&](const PendingJob &j) { return j.id == job_id; });
        STWO_REQUIRE(it != s->pending.end(), STWO_ERR_INVALID_ARGUMENT,
                     "job %llu is not queued (running, finished or unknown)", (unsigned long long)job_id);
        s->post_unrun(*it, STWO_ERR_CANCELLED, "job cancelled before it started");
        s->pending.erase(it);
    }
    s->cv_done.notify_all();
    return STWO_OK;
}

int stwo_server_pause(stwo_prover_server *s, int paused) {
    STWO_REQUIRE(s, STWO_ERR_INVALID_ARGUMENT, "null server");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->paused = paused != 0;
    }
    if (!paused) s->cv_work.notify_all();
    return STWO_OK;
}

int stwo_server_set_queue_timeout(stwo_prover_server *s, double queue_timeout_ms) {
    STWO_REQUIRE(s && queue_timeout_ms >= 0, STWO_ERR_INVALID_ARGUMENT, "invalid queue timeout");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->queue_timeout_ms = queue_timeout_ms;
    }
    s->cv_work.notify_all();
    return STWO_OK;
}

void stwo_server_destroy(stwo_prover_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        s->pending.clear();
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    for (auto &r : s->done) free(r.proof);
    cudaFree(s->tw);
    cudaFree(s->itw);
    cudaEventDestroy(s->epoch);
    cudaStreamDestroy(s->epoch_stream);
    delete s;
}

}  // extern "C"
