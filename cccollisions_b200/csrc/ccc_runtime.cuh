// ccc_runtime.cuh — launch accounting shared by the library's translation units.
//
// Every kernel launch goes through CCC_LAUNCH, which counts it and, while per-kernel
// timing is on (ccc_timing_begin / ccc_timing_end) and the stream is not being captured
// into a graph, brackets it with CUDA events on the launching stream.  Definitions live in
// ccc_capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace ccc {

// launches since load (exact when one host thread launches at a time)
extern std::atomic<int64_t> g_launches;
// elementary functions of the continuous-collision solver (MathLib)
extern int g_math_lib;

void timing_before(const char* name, cudaStream_t s, int* slot);
void timing_after(int slot, cudaStream_t s);
// per-kernel timing is on: work that would overlap on a second stream runs in order
bool timing_active();
int num_sms();

inline int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
inline int grid_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace ccc

#define CCC_LAUNCH(name, s, ...)                  \
    do {                                          \
        int slot__;                               \
        ::ccc::timing_before(name, s, &slot__);   \
        __VA_ARGS__;                              \
        ::ccc::timing_after(slot__, s);           \
    } while (0)

// Run the statement(s) with LIBV bound to the current math library (MathLib) as a
// compile-time constant, for kernels templated on it.
#define CCC_WITH_LIB(...)                                              \
    do {                                                               \
        if (::ccc::g_math_lib == 0) {                                  \
            constexpr int LIBV = 0;                                    \
            __VA_ARGS__;                                               \
        } else {                                                       \
            constexpr int LIBV = 1;                                    \
            __VA_ARGS__;                                               \
        }                                                              \
    } while (0)

#define CCC_LAUNCH_CHECK()                                         \
    do {                                                           \
        cudaError_t e__ = cudaGetLastError();                      \
        if (e__ != cudaSuccess) return CCC_ERR_CUDA;               \
    } while (0)
