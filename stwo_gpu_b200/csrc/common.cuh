// Shared plumbing for the C ABI: status codes, the per-thread last-error record,
// launch checks and small device helpers.
#pragma once
#include <atomic>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/stwo_b200.h"
#include "field.cuh"

namespace stwo {

// Records a failure for stwo_last_error() and returns its status.
int set_error(int status, const char *fmt, ...);
void clear_error();

// Counts of kernel launches made by the library: process-wide and per host thread.
extern std::atomic<uint64_t> g_kernel_launches;
extern thread_local uint64_t t_kernel_launches;
inline void count_launch(uint64_t n = 1) {
    g_kernel_launches.fetch_add(n, std::memory_order_relaxed);
    t_kernel_launches += n;
}

#define STWO_CUDA_TRY(expr)                                                               \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess)                                                            \
            return ::stwo::set_error(STWO_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,       \
                                     cudaGetErrorString(_e), __FILE__, __LINE__);         \
    } while (0)

// Follows every kernel launch: counts it (stwo_kernel_launches) and checks it.
#define STWO_LAUNCH_CHECK(name)                                                           \
    do {                                                                                  \
        ::stwo::count_launch();                                                           \
        cudaError_t _e = cudaGetLastError();                                              \
        if (_e != cudaSuccess)                                                            \
            return ::stwo::set_error(STWO_ERR_CUDA, "launch of %s failed: %s", name,      \
                                     cudaGetErrorString(_e));                             \
    } while (0)

#define STWO_REQUIRE(cond, status, ...)                                                   \
    do {                                                                                  \
        if (!(cond)) return ::stwo::set_error(status, __VA_ARGS__);                       \
    } while (0)

inline bool is_pow2(uint64_t n) { return n && !(n & (n - 1)); }
inline uint32_t log2_u64(uint64_t n) {
    uint32_t l = 0;
    while ((1ull << l) < n) l++;
    return l;
}

constexpr int NUM_SMS_B200 = 148;

// Number of SMs of the current device (cached per process; the library drives one device).
int device_sm_count();

// Runs f() (a status-returning setup step such as cudaFuncSetAttribute) once per device:
// bit d of `done` records device d. Concurrent first calls may both run f, so f must be
// idempotent.
template <class F>
int once_per_device(std::atomic<uint64_t> &done, F f) {
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return STWO_OK;
    int rc = f();
    if (rc == STWO_OK) done.fetch_or(bit, std::memory_order_release);
    return rc;
}

// The library's stream-ordered memory pool on the current device, created on first use
// with an unbounded release threshold: memory a job frees is reused by the next job
// instead of going back to the driver at every synchronisation.
int library_pool(cudaMemPool_t *pool);
// Grows the library pool to hold at least `bytes` (allocated and freed once), so
// later allocations up to that total map no new physical memory.
int reserve_pool(uint64_t bytes);
// cudaMallocFromPoolAsync from the library pool (free with cudaFreeAsync).
int pool_alloc(void **p, size_t bytes, cudaStream_t st);

// Waits for all work on `st`. A thread that sets t_blocking_wait first polls for up to
// t_spin_us microseconds (a wake-up from a blocking wait costs a few hundred
// microseconds, more than a small proof's remaining device work), then yields its CPU
// core on a blocking-sync event; the proof server's workers do, so many in-flight large
// jobs do not compete for host cores. Other threads spin (cudaStreamSynchronize).
// Every wait records a timing-capable event, so the device time at which the stream's
// work ended can be read afterwards (last_wait_event).
extern thread_local bool t_blocking_wait;
extern thread_local uint32_t t_spin_us;
int wait_stream(cudaStream_t st);
// The event of this thread's last wait_stream on the current device, or null.
cudaEvent_t last_wait_event();

// Pinned host memory of at least `bytes`, owned by the calling thread and reused by its
// next call: the staging area of the small device<->host copies (roots, sampled values,
// decommitment words), which from pageable memory serialise on the driver's staging
// buffer across threads. Valid until the thread's next host_stage call.
int host_stage(size_t bytes, void **out);

// Launch parameters that stwo_autotune measures and stwo_set_tunable sets
// (process-wide; every value of a tunable computes the same results).
enum Tunable {
    TUNE_FFT_EPT_CONTIG_SMALL,  // log2 elements per thread, contiguous passes, domains <= 2^20
    TUNE_FFT_EPT_CONTIG_LARGE,  // same, larger domains
    TUNE_FFT_EPT_STRIDED,       // same, strided passes
    TUNE_MERKLE_SUB_THREADS,    // CTA size of the multi-layer Merkle kernel (log2 + 1 layers per launch)
    TUNE_MERKLE_SUB_SPREAD,     // log2 bottom-level nodes per thread of that kernel (0..5)
    TUNE_EAP_GROUPS_LOG,        // eval_at_point: log2 groups of 8192 coefficients per CTA (2..4), 0 = per launch
    TUNE_FFT_MAX_STRIDED,       // FFT radix split: at most this many layers per strided pass (4..10)
    TUNE_QUOT_TENSOR,           // DEEP quotients on the tensor cores: 0 never, 1 2+ batches over >= 2^16 rows, 2 always
    TUNE_COMP_TENSOR,           // wide-Fibonacci composition on the tensor cores: 1 yes, 0 (default) no
    TUNE_COUNT
};
int tunable(Tunable t);
void set_tunable(Tunable t, int v);
// Counts set_tunable calls: a captured launch sequence is valid only for the settings
// it was captured under.
uint64_t tunables_generation();

// Stream handle conversion for the C ABI.
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Synchronous wrapper used by the reference-compatible entry points: run on the
// legacy default stream and wait, as the reference's host functions do.
int sync_default_stream(int status);

// Several proofs of one shape in one launch sequence: job k's device memory is job 0's
// moved by k * stride bytes (identical allocation sequences in equal slabs), so a
// kernel launched once over K jobs moves every pointer into job memory by
// job * stride. Pointers outside the jobs' slabs (a shared twiddle tree) do not move.
template <class T>
__host__ __device__ __forceinline__ T *job_ptr(T *p, size_t stride, uint32_t job) {
    return p ? reinterpret_cast<T *>(reinterpret_cast<uintptr_t>(p) + (size_t)job * stride) : p;
}

}  // namespace stwo
