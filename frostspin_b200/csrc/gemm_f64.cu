// Grouped FP64 GEMM over irrep sectors: the plain double-precision path.
//
// Reference behaviour: SymmetricTensor.__matmul__ (frostspin/symmetric_tensor/
// symmetric_tensor.py:453-489) calls numpy's dgemm once per shared irrep block.
// Here every sector product of one contraction is a problem in one launch; the
// host flattens all output tiles of all problems into a tile list and CTAs
// stride over it (a static persistent schedule), so sectors of very uneven
// sizes share the machine.  64x64 output tile, 16-deep k slices staged through
// shared memory with register double buffering, 4x4 outputs per thread.
#include "common.cuh"

namespace fsb {

constexpr int kTM = 64;
constexpr int kTN = 64;
constexpr int kTK = 16;
constexpr int kGemmThreads = 256;

struct __align__(16) GemmSmem {
    double a[2][kTK][kTM + 2];
    double b[2][kTK][kTN + 2];
};

__device__ __forceinline__ void load_a_regs(const FsGemmProblem& p, int m0, int k0,
                                            double (&r)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = threadIdx.x + u * kGemmThreads;
        int i, k;
        if (p.transA) {
            k = idx / kTM;
            i = idx % kTM;
        } else {
            i = idx / kTK;
            k = idx % kTK;
        }
        const int gi = m0 + i, gk = k0 + k;
        double v = 0.0;
        if (gi < p.M && gk < p.K) {
            v = p.transA ? __ldg(p.A + static_cast<int64_t>(gk) * p.lda + gi)
                         : __ldg(p.A + static_cast<int64_t>(gi) * p.lda + gk);
        }
        r[u] = v;
    }
}

__device__ __forceinline__ void store_a_smem(const FsGemmProblem& p, double (*sa)[kTM + 2],
                                             const double (&r)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = threadIdx.x + u * kGemmThreads;
        int i, k;
        if (p.transA) {
            k = idx / kTM;
            i = idx % kTM;
        } else {
            i = idx / kTK;
            k = idx % kTK;
        }
        sa[k][i] = r[u];
    }
}

__device__ __forceinline__ void load_b_regs(const FsGemmProblem& p, int n0, int k0,
                                            double (&r)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = threadIdx.x + u * kGemmThreads;
        int j, k;
        if (p.transB) {
            j = idx / kTK;
            k = idx % kTK;
        } else {
            k = idx / kTN;
            j = idx % kTN;
        }
        const int gj = n0 + j, gk = k0 + k;
        double v = 0.0;
        if (gj < p.N && gk < p.K) {
            v = p.transB ? __ldg(p.B + static_cast<int64_t>(gj) * p.ldb + gk)
                         : __ldg(p.B + static_cast<int64_t>(gk) * p.ldb + gj);
        }
        r[u] = v;
    }
}

__device__ __forceinline__ void store_b_smem(const FsGemmProblem& p, double (*sb)[kTN + 2],
                                             const double (&r)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = threadIdx.x + u * kGemmThreads;
        int j, k;
        if (p.transB) {
            j = idx / kTK;
            k = idx % kTK;
        } else {
            k = idx / kTN;
            j = idx % kTN;
        }
        sb[k][j] = r[u];
    }
}

__global__ void __launch_bounds__(kGemmThreads)
    k_grouped_dgemm(const FsGemmProblem* __restrict__ problems, int64_t n_problems,
                    const FsGemmTile* __restrict__ tiles, int64_t n_tiles) {
    __shared__ GemmSmem sm;
    const int tx = threadIdx.x % 16;
    const int ty = threadIdx.x / 16;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const FsGemmTile tile = tiles[t];
        if (tile.problem < 0 || tile.problem >= n_problems) continue;
        const FsGemmProblem p = problems[tile.problem];
        const int m0 = tile.tm * kTM;
        const int n0 = tile.tn * kTN;
        if (m0 >= p.M || n0 >= p.N) continue;

        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

        double ra[4], rb[4];
        const int nk = (p.K + kTK - 1) / kTK;
        __syncthreads();  // previous tile finished reading smem
        if (nk > 0) {
            load_a_regs(p, m0, 0, ra);
            load_b_regs(p, n0, 0, rb);
            store_a_smem(p, sm.a[0], ra);
            store_b_smem(p, sm.b[0], rb);
        }
        __syncthreads();
        for (int kt = 0; kt < nk; ++kt) {
            const int cur = kt & 1;
            if (kt + 1 < nk) {
                load_a_regs(p, m0, (kt + 1) * kTK, ra);
                load_b_regs(p, n0, (kt + 1) * kTK, rb);
            }
#pragma unroll
            for (int k = 0; k < kTK; ++k) {
                double av[4], bv[4];
                const double2 a01 = *reinterpret_cast<const double2*>(&sm.a[cur][k][ty * 4]);
                const double2 a23 = *reinterpret_cast<const double2*>(&sm.a[cur][k][ty * 4 + 2]);
                const double2 b01 = *reinterpret_cast<const double2*>(&sm.b[cur][k][tx * 4]);
                const double2 b23 = *reinterpret_cast<const double2*>(&sm.b[cur][k][tx * 4 + 2]);
                av[0] = a01.x; av[1] = a01.y; av[2] = a23.x; av[3] = a23.y;
                bv[0] = b01.x; bv[1] = b01.y; bv[2] = b23.x; bv[3] = b23.y;
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
            }
            if (kt + 1 < nk) {
                store_a_smem(p, sm.a[cur ^ 1], ra);
                store_b_smem(p, sm.b[cur ^ 1], rb);
            }
            __syncthreads();
        }

#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gi = m0 + ty * 4 + i;
            if (gi >= p.M) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int gj = n0 + tx * 4 + j;
                if (gj >= p.N) continue;
                double* c = p.C + static_cast<int64_t>(gi) * p.ldc + gj;
                const double v = p.alpha * acc[i][j];
                *c = (p.beta == 0.0) ? v : fma(p.beta, *c, v);
            }
        }
    }
}

}  // namespace fsb

extern "C" int fs_dgemm_tile_shape(int32_t* tile_m, int32_t* tile_n) {
    if (tile_m == nullptr || tile_n == nullptr) return FS_ERR_INVALID_ARG;
    *tile_m = fsb::kTM;
    *tile_n = fsb::kTN;
    return FS_OK;
}

extern "C" int fs_grouped_dgemm(const FsGemmProblem* d_problems, int64_t n_problems,
                                const FsGemmTile* d_tiles, int64_t n_tiles, void* stream) {
    if (n_tiles < 0 || n_problems < 0) return FS_ERR_INVALID_ARG;
    if (n_tiles == 0) return FS_OK;
    if (d_problems == nullptr || d_tiles == nullptr) return FS_ERR_INVALID_ARG;
    const int64_t max_grid = static_cast<int64_t>(fsb::kNumSM) * 4;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    fsb::k_grouped_dgemm<<<grid, fsb::kGemmThreads, 0, fsb::as_stream(stream)>>>(
        d_problems, n_problems, d_tiles, n_tiles);
    return fsb::launch_status();
}
