// common.cuh -- shared host/device helpers of libsweep_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sweep_b200.h"

namespace sweep {

// Host-side error: thrown inside the library, caught at the C boundary and
// turned into (non-zero return, message), as the reference's guarded()
// (reference src/sweep/csrc/cuda/common/capi.cu:578-580).
struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define SWEEP_REQUIRE(cond, ...)                                                  \
    do {                                                                          \
        if (!(cond)) {                                                            \
            char _buf[512];                                                       \
            snprintf(_buf, sizeof(_buf), __VA_ARGS__);                            \
            throw ::sweep::Error(_buf);                                           \
        }                                                                         \
    } while (0)

#define SWEEP_CUDA(call)                                                          \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess)                                                    \
            throw ::sweep::Error(std::string(#call " failed: ") + cudaGetErrorString(_e)); \
    } while (0)

#define SWEEP_LAUNCH_CHECK()                                                      \
    do {                                                                          \
        cudaError_t _e = cudaGetLastError();                                      \
        if (_e != cudaSuccess)                                                    \
            throw ::sweep::Error(std::string("kernel launch failed: ") + cudaGetErrorString(_e)); \
    } while (0)

// Run `fn` and convert any exception into the C ABI's (rc, message) pair.
template <class F>
int guarded(char* err, int32_t cap, F&& fn)
{
    try {
        fn();
        if (err && cap > 0) err[0] = '\0';
        return 0;
    } catch (const std::exception& e) {
        if (err && cap > 0) {
            strncpy(err, e.what(), (size_t)cap - 1);
            err[cap - 1] = '\0';
        }
        return 1;
    } catch (...) {
        if (err && cap > 0) {
            strncpy(err, "unknown error", (size_t)cap - 1);
            err[cap - 1] = '\0';
        }
        return 2;
    }
}

// Bump allocator over a caller-owned byte range: every sub-buffer 256-byte
// aligned.  With base == nullptr it only measures (the sizes query and the
// carve then agree by construction).
struct Carve {
    char* base;
    int64_t off = 0;
    explicit Carve(void* b) : base(static_cast<char*>(b)) {}
    template <class T>
    T* take(int64_t count)
    {
        off = (off + 255) & ~int64_t(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * (int64_t)sizeof(T);
        return p;
    }
};

// Source / receiver events grouped by (shot, tile): a CSR table so that the
// CTA owning a tile finds its point sources and receivers without scanning the
// whole list.  `cell` is the tile-local linear cell index, `id` the global
// event index (b * n + s).
struct EventTable {
    const int32_t* off = nullptr;   // (B * ntiles + 1)
    const int2* ev = nullptr;       // (count)
};


}  // namespace sweep
