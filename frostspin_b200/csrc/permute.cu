// Abelian (U(1) / Z2) block-sparse permute as a batch of strided copies.
//
// Reference behaviour: frostspin/symmetric_tensor/abelian_symmetric_tensor.py
// :103-250 (_numba_abelian_transpose) scatters every entry of every old block to
// its new (block, row, col) with per-element divmod arithmetic.  Here the host
// plan splits the tensor into elementary blocks (one irrep segment per leg), in
// which both the source and destination offsets are affine in the leg indices.
// Legs are ordered by output stride, so the last leg is the output-innermost
// one.  A *row* of an elementary block is one run along that leg; the kernel
// decodes the outer multi-index once per row (Granlund-Montgomery division with
// host-computed constants, descriptor in shared memory) and copies the run with
// a lane group sized to it, so stores are coalesced along the output and, when
// the source keeps the same innermost leg, loads are too.  Absent source blocks
// produce zeros, as the reference's zero-initialised output blocks do.
#include "common.cuh"

namespace fsb {

constexpr int kPermThreads = 256;
constexpr int kPermInnerUnroll = 4;

__global__ void __launch_bounds__(kPermThreads, 4)
    k_perm_rows(const double* __restrict__ in, int64_t in_len, double* __restrict__ out,
                int64_t out_len, const FsPermEB* __restrict__ ebs, int64_t n_ebs,
                const FsPermTask* __restrict__ tasks, int64_t n_tasks, int32_t* flag) {
    __shared__ FsPermEB e;
    static_assert(sizeof(FsPermEB) % 8 == 0, "descriptor must be 8-byte granular");
    constexpr int kWords = sizeof(FsPermEB) / 8;
    const int lane = threadIdx.x % 32;
    for (int64_t t = blockIdx.x; t < n_tasks; t += gridDim.x) {
        const FsPermTask task = tasks[t];
        if (task.eb < 0 || task.eb >= n_ebs) {
            if (threadIdx.x == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
        __syncthreads();
        if (threadIdx.x < kWords) {
            reinterpret_cast<int64_t*>(&e)[threadIdx.x] =
                reinterpret_cast<const int64_t*>(ebs + task.eb)[threadIdx.x];
        }
        __syncthreads();
        const int nd = e.ndim;
        if (nd < 1 || nd > FS_PERM_MAXR) {
            if (threadIdx.x == 0) raise_flag(flag, FS_ERR_UNSUPPORTED);
            continue;
        }
        const uint32_t L = e.dims[nd - 1];
        const int64_t osL = e.ostride[nd - 1];
        const int64_t nsL = e.nstride[nd - 1];
        const bool zero_fill = e.obase < 0;
        // lane group: smallest power of two >= L, at most a warp
        const int g = (L >= 32) ? 32 : (L <= 1 ? 1 : (1 << (32 - __clz(L - 1))));
        const int lg = lane % g;
        const int grp = static_cast<int>(threadIdx.x) / g;
        const int ngrp = kPermThreads / g;
        const uint32_t end = task.start + task.count;
        for (uint32_t row = task.start + grp; row < end; row += ngrp) {
            uint32_t q = row;
            int64_t so = e.obase, dof = e.nbase;
            for (int k = nd - 2; k >= 0; --k) {
                const uint32_t qq = fast_div(q, e.divm[k], e.divs[k]);
                const uint32_t i = q - qq * e.dims[k];
                q = qq;
                so += static_cast<int64_t>(i) * e.ostride[k];
                dof += static_cast<int64_t>(i) * e.nstride[k];
            }
            for (uint32_t i0 = lg; i0 < L; i0 += g * kPermInnerUnroll) {
                double v[kPermInnerUnroll];
                int64_t dst[kPermInnerUnroll];
#pragma unroll
                for (int u = 0; u < kPermInnerUnroll; ++u) {
                    const uint32_t i = i0 + u * g;
                    dst[u] = -1;
                    v[u] = 0.0;
                    if (i < L) {
                        const int64_t d = dof + static_cast<int64_t>(i) * nsL;
                        if (d < 0 || d >= out_len) {
                            raise_flag(flag, FS_ERR_BOUNDS);
                            continue;
                        }
                        dst[u] = d;
                        if (!zero_fill) {
                            const int64_t s = so + static_cast<int64_t>(i) * osL;
                            if (s >= 0 && s < in_len) {
                                v[u] = __ldg(in + s);
                            } else {
                                raise_flag(flag, FS_ERR_BOUNDS);
                                dst[u] = -1;
                            }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < kPermInnerUnroll; ++u) {
                    if (dst[u] >= 0) out[dst[u]] = v[u];
                }
            }
        }
    }
}

}  // namespace fsb

extern "C" int fs_abelian_permute(const double* d_in, int64_t in_len, double* d_out,
                                  int64_t out_len, const FsPermEB* d_ebs, int64_t n_ebs,
                                  const FsPermTask* d_tasks, int64_t n_tasks,
                                  int32_t* d_flag, void* stream) {
    if (n_tasks < 0 || n_ebs < 0 || in_len < 0 || out_len < 0) return FS_ERR_INVALID_ARG;
    if (n_tasks == 0) return FS_OK;
    if (d_out == nullptr || d_ebs == nullptr || d_tasks == nullptr) return FS_ERR_INVALID_ARG;
    if (d_in == nullptr && in_len > 0) return FS_ERR_INVALID_ARG;
    const int64_t max_grid = static_cast<int64_t>(fsb::kNumSM) * 8;
    const int grid = static_cast<int>(n_tasks < max_grid ? n_tasks : max_grid);
    fsb::k_perm_rows<<<grid, fsb::kPermThreads, 0, fsb::as_stream(stream)>>>(
        d_in, in_len, d_out, out_len, d_ebs, n_ebs, d_tasks, n_tasks, d_flag);
    return fsb::launch_status();
}
