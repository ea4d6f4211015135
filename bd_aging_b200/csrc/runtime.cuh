// runtime.cuh -- host-side plumbing shared by the translation units of
// libbd_aging_b200: status mapping, per-device workspace, launch checks.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/bd_aging.h"
#include "common.cuh"

namespace bd {

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Identifier of the CUDA context current on the calling thread (initialising
// the current device's primary context if needed).  Context ids are unique
// for the life of the process, so a device reset, which destroys the primary
// context and every address in it, changes the id.  0 when none can be had.
unsigned long long current_context_id();

// Per-device workspace for the mirror entry points: a status word and the
// FP64 partial sums of the fixed-order reductions.  Allocated on first use in
// each device's context (again after a device reset) and kept until exit.
constexpr int kWorkAccum = 2048;  // FP64 slots: one per reduction block plus the result
struct DeviceWork {
    unsigned *status = nullptr;   // device status word (kStat* bits)
    double *accum = nullptr;      // kWorkAccum FP64 partial sums
    unsigned long long ctx = 0;   // context the pointers belong to
};

DeviceWork *device_work();  // nullptr on allocation failure

// Map the device status word to a BD_* code.  A non-finite position also
// piles particles into one cell, so it is reported before the overflow.
inline int status_from_bits(unsigned bits) {
    if (bits & kStatNumeric) return BD_ERR_NUMERIC;
    if (bits & kStatCellOverflow) return BD_ERR_CELL_OVERFLOW;
    if (bits & kStatTimeout) return BD_ERR_TIMEOUT;
    if (bits & kStatArg) return BD_ERR_ARG;
    return BD_OK;
}

#define BD_CUDA_TRY(expr)                                                                    \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) {                                                             \
            std::fprintf(stderr, "bd_aging_b200: %s failed: %s (%s:%d)\n", #expr,            \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                        \
            return BD_ERR_CUDA;                                                              \
        }                                                                                    \
    } while (0)

#define BD_LAUNCH_CHECK() BD_CUDA_TRY(cudaPeekAtLastError())

inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace bd
