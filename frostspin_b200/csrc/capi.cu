// Library-level C ABI entry points: version, status strings, last CUDA error,
// the device-wait bound; and the per-device queries the launchers share.
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace fsb {
namespace {
thread_local const char* g_last_cuda_error = "no error";

constexpr int kMaxDevices = 64;
constexpr int kDefaultSMs = 148;
// ~1 s of clock64 at 1.9 GHz
constexpr long long kDefaultSpinLimit = 2000000000LL;

std::atomic<int> g_sms[kMaxDevices] = {};
std::atomic<long long> g_spin_limit{kDefaultSpinLimit};

struct SmemConfig {
    std::mutex mutex;
    // (kernel, device) pairs already configured, with the bytes set
    static constexpr int kSlots = 64;
    const void* func[kSlots] = {};
    int device[kSlots] = {};
    int bytes[kSlots] = {};
    int used = 0;
};
SmemConfig g_smem;

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return -1;
    return d;
}
}  // namespace

void set_last_cuda_error(cudaError_t err) { g_last_cuda_error = cudaGetErrorString(err); }

int num_sms() {
    const int d = current_device();
    if (d < 0 || d >= kMaxDevices) return kDefaultSMs;
    int n = g_sms[d].load(std::memory_order_relaxed);
    if (n > 0) return n;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || n <= 0)
        n = kDefaultSMs;
    g_sms[d].store(n, std::memory_order_relaxed);
    return n;
}

int configure_smem(const void* func, int bytes) {
    const int d = current_device();
    std::lock_guard<std::mutex> lock(g_smem.mutex);
    for (int i = 0; i < g_smem.used; ++i)
        if (g_smem.func[i] == func && g_smem.device[i] == d && g_smem.bytes[i] >= bytes)
            return FS_OK;
    cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) {
        set_last_cuda_error(e);
        return FS_ERR_CUDA;
    }
    if (g_smem.used < SmemConfig::kSlots) {
        g_smem.func[g_smem.used] = func;
        g_smem.device[g_smem.used] = d;
        g_smem.bytes[g_smem.used] = bytes;
        ++g_smem.used;
    }
    return FS_OK;
}

long long spin_limit() { return g_spin_limit.load(std::memory_order_relaxed); }

}  // namespace fsb

extern "C" int fs_version(void) { return 10100; }

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

extern "C" int64_t fs_set_spin_limit(int64_t cycles) {
    const long long v = cycles > 0 ? cycles : fsb::kDefaultSpinLimit;
    return fsb::g_spin_limit.exchange(v);
}
