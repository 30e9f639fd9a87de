// Error reporting, device memory and copy entry points.
//
// The reference's memory helpers (cuda/include/utils.cuh:39-78, cuda/src/utils.cu:14-80)
// print CUDA failures and carry on. Here every failure is recorded per thread and
// returned as a status by the native API; the reference-compatible entry points keep
// their void / pointer signatures and return NULL on failure.
#include <chrono>
#include <cstdarg>
#include <mutex>

#include "common.cuh"

namespace stwo {

static thread_local char g_last_error[512] = "";

int set_error(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

void clear_error() { g_last_error[0] = 0; }

std::atomic<uint64_t> g_kernel_launches{0};

namespace {
std::atomic<int> g_tunables[TUNE_COUNT] = {{6}, {6}, {6}, {256}, {3}, {0}, {10}, {1}, {0}};
}
int tunable(Tunable t) { return g_tunables[t].load(std::memory_order_relaxed); }
std::atomic<uint64_t> g_tunables_gen{0};
void set_tunable(Tunable t, int v) {
    g_tunables[t].store(v, std::memory_order_relaxed);
    g_tunables_gen.fetch_add(1, std::memory_order_relaxed);
}
uint64_t tunables_generation() { return g_tunables_gen.load(std::memory_order_relaxed); }
thread_local uint64_t t_kernel_launches = 0;

int device_sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            count = NUM_SMS_B200;
    }
    return count;
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

struct BlockingEvent {
    cudaEvent_t ev = nullptr;
    int device = -1;
    ~BlockingEvent() {
        if (ev) cudaEventDestroy(ev);
    }
};
thread_local BlockingEvent t_event;

struct HostStage {
    void *p = nullptr;
    size_t cap = 0;
    ~HostStage() {
        if (p) cudaFreeHost(p);
    }
};
thread_local HostStage t_stage;
}  // namespace

int host_stage(size_t bytes, void **out) {
    if (t_stage.cap < bytes) {
        size_t cap = 1 << 16;
        while (cap < bytes) cap <<= 1;
        if (t_stage.p) cudaFreeHost(t_stage.p);
        t_stage.p = nullptr;
        t_stage.cap = 0;
        STWO_CUDA_TRY(cudaMallocHost(&t_stage.p, cap));
        t_stage.cap = cap;
    }
    *out = t_stage.p;
    return STWO_OK;
}

thread_local bool t_blocking_wait = false;
thread_local uint32_t t_spin_us = 0;

int library_pool(cudaMemPool_t *pool) {
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    STWO_REQUIRE(dev >= 0 && dev < 64, STWO_ERR_CUDA, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        STWO_CUDA_TRY(cudaMemPoolCreate(&p, &props));
        uint64_t threshold = ~0ull;
        STWO_CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &threshold));
        // A stream may reuse memory another stream freed only once that free has
        // completed: the pool must not make one job's stream wait on another's.
        int no = 0;
        STWO_CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolReuseAllowInternalDependencies, &no));
        g_pools[dev] = p;
    }
    *pool = g_pools[dev];
    return STWO_OK;
}

namespace {
std::atomic<uint32_t> g_fail_allocs{0};  // stwo_debug_fail_allocations

bool take_injected_failure() {
    uint32_t n = g_fail_allocs.load();
    while (n > 0)
        if (g_fail_allocs.compare_exchange_weak(n, n - 1)) return true;
    return false;
}
}  // namespace

int pool_alloc(void **p, size_t bytes, cudaStream_t st) {
    if (take_injected_failure()) {
        *p = nullptr;
        return set_error(STWO_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: injected failure", bytes);
    }
    cudaMemPool_t pool;
    int rc = library_pool(&pool);
    if (rc) return rc;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_error(e == cudaErrorMemoryAllocation ? STWO_ERR_OUT_OF_MEMORY : STWO_ERR_CUDA,
                         "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return STWO_OK;
}

int reserve_pool(uint64_t bytes) {
    if (bytes == 0) return STWO_OK;
    cudaMemPool_t pool;
    int rc = library_pool(&pool);
    if (rc) return rc;
    cudaStream_t s = nullptr;
    STWO_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, s);
    if (e == cudaSuccess) e = cudaFreeAsync(p, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(e == cudaErrorMemoryAllocation ? STWO_ERR_OUT_OF_MEMORY : STWO_ERR_CUDA,
                         "reserving %llu pool bytes failed: %s", (unsigned long long)bytes, cudaGetErrorString(e));
    }
    return STWO_OK;
}

int wait_stream(cudaStream_t st) {
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    if (!t_event.ev || t_event.device != dev) {
        if (t_event.ev) cudaEventDestroy(t_event.ev);
        t_event.ev = nullptr;
        STWO_CUDA_TRY(cudaEventCreateWithFlags(&t_event.ev, cudaEventBlockingSync));
        t_event.device = dev;
    }
    STWO_CUDA_TRY(cudaEventRecord(t_event.ev, st));
    if (!t_blocking_wait) {
        STWO_CUDA_TRY(cudaStreamSynchronize(st));
        return STWO_OK;
    }
    if (t_spin_us) {
        const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(t_spin_us);
        for (;;) {
            const cudaError_t q = cudaEventQuery(t_event.ev);
            if (q == cudaSuccess) return STWO_OK;
            if (q != cudaErrorNotReady) STWO_CUDA_TRY(q);
            if (std::chrono::steady_clock::now() >= until) break;
        }
    }
    STWO_CUDA_TRY(cudaEventSynchronize(t_event.ev));
    return STWO_OK;
}

cudaEvent_t last_wait_event() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || t_event.device != dev) return nullptr;
    return t_event.ev;
}

int sync_default_stream(int status) {
    if (status != STWO_OK) return status;
    cudaError_t e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) return set_error(STWO_ERR_CUDA, "device error: %s", cudaGetErrorString(e));
    return STWO_OK;
}

template <typename T>
static T *dev_alloc(size_t count, bool zero) {
    void *p = nullptr;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = sizeof(T);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        set_error(STWO_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return nullptr;
    }
    if (zero && cudaMemset(p, 0, bytes) != cudaSuccess) {
        set_error(STWO_ERR_CUDA, "cudaMemset failed");
        cudaFree(p);
        return nullptr;
    }
    return static_cast<T *>(p);
}

static void copy_sync(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpy(dst, src, bytes, kind);
    if (e != cudaSuccess) set_error(STWO_ERR_CUDA, "cudaMemcpy(%zu) failed: %s", bytes, cudaGetErrorString(e));
}

}  // namespace stwo

using namespace stwo;

extern "C" {

const char *stwo_last_error(void) { return g_last_error; }

void stwo_clear_last_error(void) { clear_error(); }

void stwo_debug_fail_allocations(uint32_t n) { g_fail_allocs.store(n); }

uint64_t stwo_kernel_launches(void) { return g_kernel_launches.load(std::memory_order_relaxed); }

int stwo_reserve_device_memory(uint64_t bytes) { return reserve_pool(bytes); }

int stwo_stream_synchronize(void *stream) {
    cudaError_t e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess) return set_error(STWO_ERR_CUDA, "device error: %s", cudaGetErrorString(e));
    return STWO_OK;
}

void copy_uint32_t_vec_from_device_to_host(const uint32_t *device_ptr, uint32_t *host_ptr, uint32_t size) {
    copy_sync(host_ptr, device_ptr, (size_t)size * 4, cudaMemcpyDeviceToHost);
}

uint32_t *copy_uint32_t_vec_from_host_to_device(const uint32_t *host_ptr, uint32_t size) {
    uint32_t *d = dev_alloc<uint32_t>(size, false);
    if (d) copy_sync(d, host_ptr, (size_t)size * 4, cudaMemcpyHostToDevice);
    return d;
}

uint32_t *copy_uint32_t_vec_from_device_to_device(const uint32_t *from, uint32_t *dst, uint32_t size) {
    copy_sync(dst, from, (size_t)size * 4, cudaMemcpyDeviceToDevice);
    return dst;
}

uint32_t *cuda_malloc_uint32_t(uint32_t size) { return dev_alloc<uint32_t>(size, false); }

stwo_blake2s_hash *cuda_malloc_blake_2s_hash(size_t size) { return dev_alloc<stwo_blake2s_hash>(size, false); }

uint32_t *cuda_alloc_zeroes_uint32_t(uint32_t size) { return dev_alloc<uint32_t>(size, true); }

stwo_blake2s_hash *cuda_alloc_zeroes_blake_2s_hash(size_t size) { return dev_alloc<stwo_blake2s_hash>(size, true); }

void cuda_free_memory(void *device_ptr) {
    if (!device_ptr) return;
    cudaError_t e = cudaFree(device_ptr);
    if (e != cudaSuccess) set_error(STWO_ERR_CUDA, "cudaFree failed: %s", cudaGetErrorString(e));
}

stwo_blake2s_hash *copy_blake_2s_hash_vec_from_host_to_device(const stwo_blake2s_hash *from, size_t size) {
    stwo_blake2s_hash *d = dev_alloc<stwo_blake2s_hash>(size, false);
    if (d) copy_sync(d, from, size * sizeof(stwo_blake2s_hash), cudaMemcpyHostToDevice);
    return d;
}

void copy_blake_2s_hash_vec_from_device_to_host(const stwo_blake2s_hash *from, stwo_blake2s_hash *to, size_t size) {
    copy_sync(to, from, size * sizeof(stwo_blake2s_hash), cudaMemcpyDeviceToHost);
}

void copy_blake_2s_hash_vec_from_device_to_device(const stwo_blake2s_hash *from, stwo_blake2s_hash *dst, size_t size) {
    copy_sync(dst, from, size * sizeof(stwo_blake2s_hash), cudaMemcpyDeviceToDevice);
}

uint32_t **copy_device_pointer_vec_from_host_to_device(uint32_t *const *from, size_t size) {
    uint32_t **d = dev_alloc<uint32_t *>(size, false);
    if (d) copy_sync(d, from, size * sizeof(uint32_t *), cudaMemcpyHostToDevice);
    return d;
}

}  // extern "C"
