// Shared plumbing for the C ABI: status codes, the per-thread last-error record,
// launch checks and small device helpers.
#pragma once
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

#define STWO_CUDA_TRY(expr)                                                               \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess)                                                            \
            return ::stwo::set_error(STWO_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,       \
                                     cudaGetErrorString(_e), __FILE__, __LINE__);         \
    } while (0)

#define STWO_LAUNCH_CHECK(name)                                                           \
    do {                                                                                  \
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

// Stream handle conversion for the C ABI.
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Synchronous wrapper used by the reference-compatible entry points: run on the
// legacy default stream and wait, as the reference's host functions do.
int sync_default_stream(int status);

}  // namespace stwo
