// Shared helpers for the frostspin_b200 CUDA sources (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/frostspin_b200.h"

namespace fsb {

// Records the CUDA error string for fs_last_cuda_error (thread local).
void set_last_cuda_error(cudaError_t err);

// Number of SMs of the current device (queried once per device, cached);
// grids are sized as multiples of it.  Falls back to 148 (B200) if the query
// fails, so a grid is never empty.
int num_sms();

// Sets the dynamic shared memory limit of a kernel on the current device once
// per device (the attribute is per device).  Returns FS_OK or FS_ERR_CUDA.
int configure_smem(const void* func, int bytes);

// Iteration bound of the abortable device waits of the tcgen05 kernels, in
// clock64 cycles (fs_set_spin_limit).
long long spin_limit();

inline int launch_status() {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_last_cuda_error(err);
        return FS_ERR_LAUNCH;
    }
    return FS_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Granlund-Montgomery division by an invariant 32-bit divisor d:
// q = (umulhi(n, m) + n) >> s with s = ceil(log2 d), m = floor(2^32 (2^s - d) / d) + 1.
// The add is done in 64 bits so the identity holds for every 32-bit n.
__device__ __forceinline__ uint32_t fast_div(uint32_t n, uint32_t m, uint32_t s) {
    return static_cast<uint32_t>((static_cast<uint64_t>(__umulhi(n, m)) + n) >> s);
}

// Sets *flag = code once (first writer wins); flag may be null.
__device__ __forceinline__ void raise_flag(int32_t* flag, int32_t code) {
    if (flag != nullptr) atomicCAS(flag, 0, code);
}

}  // namespace fsb
