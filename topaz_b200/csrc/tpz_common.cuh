// tpz_common.cuh -- shared helpers of the topaz_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/topaz_b200.h"

namespace tpz {

// Per-thread last error message (tpz_last_error).
void set_error(const std::string &msg);

// Returns TPZ_E_CUDA and records the message when e != cudaSuccess.
int cuda_fail(cudaError_t e, const char *what);

#define TPZ_CUDA(call)                                   \
    do {                                                 \
        cudaError_t _e = (call);                         \
        if (_e != cudaSuccess) return tpz::cuda_fail(_e, #call); \
    } while (0)

// Parses the NCBI-layout matrix text into 625 int8 (row = subject letter).
int matrix_by_name(const char *name, int8_t *out625);

// SMs of the current device (cached per device).
int sm_count();

// Sets the current device's default memory pool to keep freed memory
// instead of returning it at every synchronization, so the stream-ordered
// per-call buffers are reused rather than mapped again (once per thread and
// device).
void keep_pool_memory();

// Inline PTX byte permute, including the sign-replicate selector bit that
// the generic prmt form supports (bit 3 of each selector nibble).
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

}  // namespace tpz
