// tcb_alloc.h — the library's device and pinned-host allocations.
//
// Every cudaMalloc / cudaMallocHost of the library goes through these two
// calls, so that a test can make one of them fail on the host
// (tcb_debug_fail_allocations_after) and check that the failure surfaces as
// NULL or TC_ERR_MEMORY from the public call that made it, with the object
// left releasable or retryable, and never as a launch on a missing buffer.
#pragma once
#include <stddef.h>

#include <atomic>

#include <cuda_runtime.h>

namespace tcb {

// Allocations that still succeed before the injected failure; negative:
// no failure pending.  Exactly one allocation fails per arming.
extern std::atomic<long long> g_alloc_countdown;

inline bool alloc_fault_now() {
    long long v = g_alloc_countdown.load(std::memory_order_relaxed);
    while (v >= 0)
        if (g_alloc_countdown.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return v == 0;
    return false;
}

inline cudaError_t dev_alloc(void **p, size_t n) {
    if (alloc_fault_now()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMalloc(p, n);
}
inline cudaError_t pinned_alloc(void **p, size_t n) {
    if (alloc_fault_now()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMallocHost(p, n);
}
template <typename T> inline cudaError_t dev_alloc(T **p, size_t n) { return dev_alloc((void **)p, n); }
template <typename T> inline cudaError_t pinned_alloc(T **p, size_t n) { return pinned_alloc((void **)p, n); }

}  // namespace tcb
