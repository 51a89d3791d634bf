// Shared plumbing for the B200 PDHG engine: status codes, the thread-local error
// message behind nk_last_error(), CUDA error checks and a device buffer.
#pragma once
#include "nk_pdhg.h"
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace nk {

// Errors inside the library are C++ exceptions carrying a status; every C entry
// point catches them and turns them into a status code plus nk_last_error().
struct Error : std::runtime_error {
    nk_status status;
    Error(nk_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

void set_last_error(const char *what);

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        nk_status s = e == cudaErrorMemoryAllocation ? NK_ERR_MEMORY : NK_ERR_CUDA;
        throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <class F> nk_status guard(F &&f) {
    try {
        f();
        return NK_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return NK_ERR_MEMORY;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return NK_ERR_INVALID;
    } catch (...) {
        set_last_error("unknown native failure");
        return NK_ERR_INVALID;
    }
}

// Device memory owned by one engine object; released on destruction.
template <class T> struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    // Every buffer carries kSlack zeroed bytes past its end: bulk copies widen
    // their ranges to 16-byte boundaries and may read up to 15 bytes beyond.
    static constexpr size_t kSlack = 64;
    void alloc(size_t count) {
        release();
        n = count;
        if (count) {
            cuda_check(cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T) + kSlack),
                       "cudaMalloc");
            cuda_check(cudaMemset(reinterpret_cast<char *>(p) + count * sizeof(T), 0, kSlack),
                       "slack");
        }
    }
    void release() noexcept {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    size_t bytes() const { return n * sizeof(T); }
};

} // namespace nk
