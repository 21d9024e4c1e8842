// Common definitions of the MDFT B200 engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace mdft {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kEpsDp = 2.220446049250313080847263336181640625e-16;  // epsilon(1._dp)
constexpr double kEpsSp = 1.1920928955078125e-07;                      // epsilon(1.)
constexpr int kMaxMmax = 5;   // c(k) tables exist up to mmax 5
constexpr int kMaxNp = 88;    // projections at mmax 5, mrso 2 (mrso 1 is larger: see below)
constexpr int kMaxRot = 286;  // sum_{l<=5} (2l+1)^2 packed rotation entries

// Thread-local error text of the last failing C-ABI call.
void set_error(const char *fmt, ...);
const char *last_error();

#define MDFT_CUDA_TRY(expr)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            ::mdft::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_)); \
            return MDFT_E_CUDA;                                                          \
        }                                                                                \
    } while (0)

// Device buffer owned by a handle.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { free(); }
    cudaError_t alloc(size_t count) {
        free();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(&p, count * sizeof(T));
    }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

__host__ __device__ inline int neg1pow(int k) { return (k & 1) ? -1 : 1; }

}  // namespace mdft
