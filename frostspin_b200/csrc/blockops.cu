// Elementwise and reduction kernels over block lists (bandwidth-trivial ops of
// the SymmetricTensor API, kept on the device so that tensors stay resident).
#include <math.h>

#include "common.cuh"

namespace fsb {

constexpr int kOpThreads = 256;
// partial sums of the weighted reductions: a fixed count (two CTAs per SM of a
// 148-SM B200) so that the caller-owned scratch size does not depend on the GPU
constexpr int kReducePartials = 296;

__global__ void k_scale(double* __restrict__ x, int64_t n, double alpha) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[i] *= alpha;
}

__global__ void k_scale_by(double* __restrict__ x, int64_t n, const double* __restrict__ s,
                           int invert) {
    const double a = invert ? 1.0 / s[0] : s[0];
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[i] *= a;
}

__global__ void k_axpby(const double* __restrict__ x, double* __restrict__ y, int64_t n,
                        double a, double b) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        y[i] = (b == 0.0) ? a * x[i] : fma(a, x[i], b * y[i]);
}

__global__ void k_pow(const double* __restrict__ x, double* __restrict__ y, int64_t n,
                      double p) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = x[i];
        double r;
        if (p == -1.0)
            r = 1.0 / v;
        else if (p == 2.0)
            r = v * v;
        else if (p == 0.5)
            r = sqrt(v);
        else if (p == -0.5)
            r = 1.0 / sqrt(v);
        else if (p == 1.0)
            r = v;
        else
            r = pow(v, p);
        y[i] = r;
    }
}

// Block-wide sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double warp_part[kOpThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x % 32, wid = threadIdx.x / 32;
    __syncthreads();
    if (lane == 0) warp_part[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < kOpThreads / 32) ? warp_part[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// mode 0: sum of squares, mode 1: plain sum.  Every CTA walks every segment with
// a grid stride, so the partial of CTA b is a fixed function of the input: the
// two-pass reduction is deterministic for a given grid.
template <int MODE>
__global__ void __launch_bounds__(kOpThreads)
    k_weighted_reduce(const double* __restrict__ x, const FsSegment* __restrict__ segs,
                      int64_t n_segs, double* __restrict__ partial) {
    double acc = 0.0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t s = 0; s < n_segs; ++s) {
        const FsSegment sg = segs[s];
        double part = 0.0;
        for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
             i < sg.length; i += stride) {
            const double v = __ldg(x + sg.offset + i);
            part += (MODE == 0) ? v * v : v;
        }
        acc = fma(sg.weight, part, acc);
    }
    const double r = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kOpThreads)
    k_final_sum(const double* __restrict__ partial, int64_t n, double* __restrict__ out) {
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    const double r = block_sum(acc);
    if (threadIdx.x == 0) out[0] = r;
}

__global__ void __launch_bounds__(kOpThreads)
    k_pair_contract(const double* __restrict__ a, const double* __restrict__ b,
                    const FsPairBlock* __restrict__ pairs, int64_t n_pairs,
                    double* __restrict__ partial) {
    double acc = 0.0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t q = 0; q < n_pairs; ++q) {
        const FsPairBlock pb = pairs[q];
        double part = 0.0;
        const int64_t m = pb.m, n = pb.n;
        if (pb.b_off < 0) {  // trace
            const int64_t d = m < n ? m : n;
            for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
                 i < d; i += stride) {
                part += __ldg(a + pb.a_off + (pb.a_trans ? i * m + i : i * n + i));
            }
        } else {
            const int64_t total = m * n;
            for (int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
                 f < total; f += stride) {
                const int64_t i = f / n, j = f % n;
                const double av = __ldg(a + pb.a_off + (pb.a_trans ? j * m + i : f));
                // B has logical shape (n, m); entry (j, i).
                const double bv = __ldg(b + pb.b_off + (pb.b_trans ? i * n + j : j * m + i));
                part = fma(av, bv, part);
            }
        }
        acc = fma(pb.weight, part, acc);
    }
    const double r = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kOpThreads)
    k_diag_mul(const double* __restrict__ x, const double* __restrict__ diag,
               double* __restrict__ out, const FsDiagBlock* __restrict__ blocks,
               int64_t n_blocks) {
    for (int64_t q = blockIdx.y; q < n_blocks; q += gridDim.y) {
        const FsDiagBlock db = blocks[q];
        const int64_t m = db.m, n = db.n, total = m * n;
        for (int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
             f < total; f += static_cast<int64_t>(gridDim.x) * blockDim.x) {
            const int64_t i = f / n, j = f % n;
            const double v = __ldg(x + db.x_off + (db.x_trans ? j * m + i : f));
            const double d = __ldg(diag + db.d_off + (db.left ? i : j));
            out[db.out_off + f] = v * d;
        }
    }
}

inline int elementwise_grid(int64_t n) {
    int64_t g = (n + kOpThreads - 1) / kOpThreads;
    const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

}  // namespace fsb

extern "C" int fs_reduce_partials(void) { return fsb::kReducePartials; }

extern "C" int fs_scale(double* d_x, int64_t n, double alpha, void* stream) {
    if (n < 0) return FS_ERR_INVALID_ARG;
    if (n == 0) return FS_OK;
    if (d_x == nullptr) return FS_ERR_INVALID_ARG;
    fsb::k_scale<<<fsb::elementwise_grid(n), fsb::kOpThreads, 0, fsb::as_stream(stream)>>>(
        d_x, n, alpha);
    return fsb::launch_status();
}

extern "C" int fs_scale_by(double* d_x, int64_t n, const double* d_scalar, int32_t invert,
                           void* stream) {
    if (n < 0) return FS_ERR_INVALID_ARG;
    if (n == 0) return FS_OK;
    if (d_x == nullptr || d_scalar == nullptr) return FS_ERR_INVALID_ARG;
    fsb::k_scale_by<<<fsb::elementwise_grid(n), fsb::kOpThreads, 0, fsb::as_stream(stream)>>>(
        d_x, n, d_scalar, invert);
    return fsb::launch_status();
}

extern "C" int fs_axpby(const double* d_x, double* d_y, int64_t n, double a, double b,
                        void* stream) {
    if (n < 0) return FS_ERR_INVALID_ARG;
    if (n == 0) return FS_OK;
    if (d_x == nullptr || d_y == nullptr) return FS_ERR_INVALID_ARG;
    fsb::k_axpby<<<fsb::elementwise_grid(n), fsb::kOpThreads, 0, fsb::as_stream(stream)>>>(
        d_x, d_y, n, a, b);
    return fsb::launch_status();
}

extern "C" int fs_pow(const double* d_x, double* d_y, int64_t n, double p, void* stream) {
    if (n < 0) return FS_ERR_INVALID_ARG;
    if (n == 0) return FS_OK;
    if (d_x == nullptr || d_y == nullptr) return FS_ERR_INVALID_ARG;
    fsb::k_pow<<<fsb::elementwise_grid(n), fsb::kOpThreads, 0, fsb::as_stream(stream)>>>(
        d_x, d_y, n, p);
    return fsb::launch_status();
}

namespace {
template <int MODE>
int weighted_reduce(const double* d_x, const FsSegment* d_segs, int64_t n_segs,
                    double* d_partial, int64_t n_partial, double* d_out, void* stream) {
    if (n_segs < 0 || n_partial < fsb::kReducePartials) return FS_ERR_INVALID_ARG;
    if (d_partial == nullptr || d_out == nullptr) return FS_ERR_INVALID_ARG;
    if (n_segs > 0 && (d_x == nullptr || d_segs == nullptr)) return FS_ERR_INVALID_ARG;
    cudaStream_t s = fsb::as_stream(stream);
    fsb::k_weighted_reduce<MODE><<<fsb::kReducePartials, fsb::kOpThreads, 0, s>>>(
        d_x, d_segs, n_segs, d_partial);
    int st = fsb::launch_status();
    if (st != FS_OK) return st;
    fsb::k_final_sum<<<1, fsb::kOpThreads, 0, s>>>(d_partial, fsb::kReducePartials, d_out);
    return fsb::launch_status();
}
}  // namespace

extern "C" int fs_weighted_sumsq(const double* d_x, const FsSegment* d_segs, int64_t n_segs,
                                 double* d_partial, int64_t n_partial, double* d_out,
                                 void* stream) {
    return weighted_reduce<0>(d_x, d_segs, n_segs, d_partial, n_partial, d_out, stream);
}

extern "C" int fs_weighted_sum(const double* d_x, const FsSegment* d_segs, int64_t n_segs,
                               double* d_partial, int64_t n_partial, double* d_out,
                               void* stream) {
    return weighted_reduce<1>(d_x, d_segs, n_segs, d_partial, n_partial, d_out, stream);
}

extern "C" int fs_pair_contract(const double* d_a, const double* d_b,
                                const FsPairBlock* d_pairs, int64_t n_pairs,
                                double* d_partial, int64_t n_partial, double* d_out,
                                void* stream) {
    if (n_pairs < 0 || n_partial < fsb::kReducePartials) return FS_ERR_INVALID_ARG;
    if (d_partial == nullptr || d_out == nullptr) return FS_ERR_INVALID_ARG;
    if (n_pairs > 0 && (d_a == nullptr || d_pairs == nullptr)) return FS_ERR_INVALID_ARG;
    cudaStream_t s = fsb::as_stream(stream);
    fsb::k_pair_contract<<<fsb::kReducePartials, fsb::kOpThreads, 0, s>>>(d_a, d_b, d_pairs,
                                                                          n_pairs, d_partial);
    int st = fsb::launch_status();
    if (st != FS_OK) return st;
    fsb::k_final_sum<<<1, fsb::kOpThreads, 0, s>>>(d_partial, fsb::kReducePartials, d_out);
    return fsb::launch_status();
}

extern "C" int fs_diag_mul(const double* d_x, const double* d_diag, double* d_out,
                           const FsDiagBlock* d_blocks, int64_t n_blocks, void* stream) {
    if (n_blocks < 0) return FS_ERR_INVALID_ARG;
    if (n_blocks == 0) return FS_OK;
    if (d_x == nullptr || d_diag == nullptr || d_out == nullptr || d_blocks == nullptr)
        return FS_ERR_INVALID_ARG;
    dim3 grid(fsb::num_sms(), static_cast<unsigned>(n_blocks < 65535 ? n_blocks : 65535));
    fsb::k_diag_mul<<<grid, fsb::kOpThreads, 0, fsb::as_stream(stream)>>>(d_x, d_diag, d_out,
                                                                          d_blocks, n_blocks);
    return fsb::launch_status();
}
