// Status discipline shared by every extern "C" entry point of libdvgpu.
//
// Follows native/src/icicle_msm.cu:38-45,188-238,424-432: invalid arguments
// return -1 and leave the owner healthy; CUDA failures retire the owner
// (-2/-3) and later calls return -4; outputs are written only on success;
// C++ exceptions never cross the ABI.
#pragma once
#include <algorithm>
#include <cstring>
#include <string>

#include "backend.hpp"

namespace dv {

inline int fail(int status, const std::string& msg, char* error, size_t cap) {
    if (error && cap) {
        const size_t n = std::min(cap - 1, msg.size());
        memcpy(error, msg.data(), n);
        error[n] = '\0';
    }
    return status;
}

template <class Fn>
int guarded(void* opaque, char* error, size_t cap, Fn&& fn) {
    auto* b = static_cast<Backend*>(opaque);
    if (!b) return fail(-1, "null backend", error, cap);
    if (b->retired) return fail(-4, "backend retired after an error; create a new backend", error, cap);
    try {
        DV_CUDA(cudaSetDevice(b->device));
        fn(*b);
        return 0;
    } catch (const InvalidArgument& e) {
        return fail(-1, e.what(), error, cap);
    } catch (const std::exception& e) {
        b->retired = true;
        b->release_all();
        return fail(-2, e.what(), error, cap);
    } catch (...) {
        b->retired = true;
        b->release_all();
        return fail(-3, "unknown native exception", error, cap);
    }
}

inline cudaStream_t pick(Backend& b, void* s) { return s ? static_cast<cudaStream_t>(s) : b.stream; }

inline void require(bool ok, const char* msg) {
    if (!ok) throw InvalidArgument(msg);
}

inline uint32_t read_err_word(Backend& b, uint32_t* d_word, cudaStream_t st) {
    uint32_t* h = b.pin_err.as<uint32_t>(1);
    DV_CUDA(cudaMemcpyAsync(h, d_word, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    return *h;
}

}  // namespace dv
