// Library-level C ABI entry points: version, status strings, last CUDA error.
#include "common.cuh"

namespace fsb {
namespace {
thread_local const char* g_last_cuda_error = "no error";
}
void set_last_cuda_error(cudaError_t err) { g_last_cuda_error = cudaGetErrorString(err); }
}  // namespace fsb

extern "C" int fs_version(void) { return 10000; }

extern "C" const char* fs_status_string(int status) {
    switch (status) {
        case FS_OK: return "ok";
        case FS_ERR_INVALID_ARG: return "invalid argument";
        case FS_ERR_LAUNCH: return "kernel launch failed";
        case FS_ERR_BOUNDS: return "plan entry out of bounds";
        case FS_ERR_TIMEOUT: return "bounded device wait ran out";
        case FS_ERR_UNSUPPORTED: return "unsupported shape or mode";
        case FS_ERR_CUDA: return "CUDA runtime error";
        case FS_ERR_TOO_LARGE: return "request exceeds a fixed capacity";
        default: return "unknown status";
    }
}

extern "C" const char* fs_last_cuda_error(void) { return fsb::g_last_cuda_error; }
