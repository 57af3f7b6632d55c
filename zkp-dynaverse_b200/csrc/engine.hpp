// Host-side plumbing shared by the kernels' launch code: error type,
// grow-only device workspace buffers, CUDA status checks.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace dv {

// Invalid caller input: reported as status -1, the owner stays healthy.
struct InvalidArgument : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// CUDA failure: reported as status -2, the owner is retired.
struct CudaFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t s, const char* what) {
    if (s != cudaSuccess) throw CudaFailure(std::string(what) + ": " + cudaGetErrorString(s));
}
// Number of this library's kernel launches since load (all owners).
uint64_t& launch_counter();
// Number of this library's device and pinned-host allocations since load,
// and the nanoseconds spent in them (freeing the old buffer included: both
// calls can wait for the device).
uint64_t& alloc_counter();
uint64_t& alloc_ns_counter();
// The slowest single allocation since load: its nanoseconds, its bytes and
// whether it was pinned host memory (1) or device memory (0).
uint64_t* slowest_alloc();
inline uint64_t steady_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}
inline void allocated(uint64_t t0, size_t bytes, bool pinned) {
    const uint64_t dt = steady_ns() - t0;
    __atomic_add_fetch(&alloc_counter(), 1, __ATOMIC_RELAXED);
    __atomic_add_fetch(&alloc_ns_counter(), dt, __ATOMIC_RELAXED);
    uint64_t* s = slowest_alloc();
    if (dt > __atomic_load_n(s, __ATOMIC_RELAXED)) {  // diagnostics: a race only mixes two records
        __atomic_store_n(s, dt, __ATOMIC_RELAXED);
        __atomic_store_n(s + 1, (uint64_t)bytes, __ATOMIC_RELAXED);
        __atomic_store_n(s + 2, (uint64_t)pinned, __ATOMIC_RELAXED);
    }
}
inline void launched() {
    cuda_check(cudaGetLastError(), "kernel launch");
    __atomic_add_fetch(&launch_counter(), 1, __ATOMIC_RELAXED);
}
#define DV_CUDA(call) ::dv::cuda_check((call), #call)
#define DV_LAUNCH() ::dv::launched()

// Grow-only device buffer.  Contents are scratch between calls.  A buffer
// that has to grow again takes 1.5x headroom, so a stream of slowly
// growing requests does not reallocate (and synchronise) every time.
struct DevBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    void* get(size_t bytes) {
        if (bytes <= cap && ptr) return ptr;
        const uint64_t t0 = steady_ns();
        const size_t regrow = cap ? cap + cap / 2 : 0;
        release();
        size_t want = bytes < 256 ? 256 : bytes;
        if (regrow > want) want = regrow;
        DV_CUDA(cudaMalloc(&ptr, want));
        allocated(t0, want, false);
        cap = want;
        return ptr;
    }
    template <class T>
    T* as(size_t count) {
        return static_cast<T*>(get(count * sizeof(T)));
    }
    template <class T>
    T* view() const {
        return static_cast<T*>(ptr);
    }
    void release() noexcept {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// Grow-only pinned host buffer, with the same 1.5x headroom (freeing pinned
// memory synchronises the device, so a stream of slowly growing requests
// must not reallocate every time).
struct PinnedBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    void* get(size_t bytes) {
        if (bytes <= cap && ptr) return ptr;
        const uint64_t t0 = steady_ns();
        const size_t regrow = cap ? cap + cap / 2 : 0;
        release();
        size_t want = bytes < 256 ? 256 : bytes;
        if (regrow > want) want = regrow;
        DV_CUDA(cudaMallocHost(&ptr, want));
        allocated(t0, want, true);
        cap = want;
        return ptr;
    }
    template <class T>
    T* as(size_t count) {
        return static_cast<T*>(get(count * sizeof(T)));
    }
    void release() noexcept {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        cap = 0;
    }
    ~PinnedBuf() { release(); }
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
};

// SM count of the device current at the first call (every device of a
// node is the same part), read once under thread-safe static initialisation.
inline int sm_count() {
    static const int n = [] {
        int dev = 0, v = 0;
        DV_CUDA(cudaGetDevice(&dev));
        DV_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        return v;
    }();
    return n;
}

}  // namespace dv
