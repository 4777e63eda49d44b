// Abelian (U(1) / Z2) block-sparse permute as a batch of strided copies.
//
// Reference behaviour: frostspin/symmetric_tensor/abelian_symmetric_tensor.py
// :103-250 (_numba_abelian_transpose) scatters every entry of every old block to
// its new (block, row, col) with per-element divmod arithmetic.  Here the host
// plan splits the tensor into elementary blocks (one irrep segment per leg), in
// which both the source and destination offsets are affine in the leg indices.
// The kernel walks each elementary block in output order (coalesced stores along
// the output-innermost leg) and gathers the source entry; absent source blocks
// produce zeros, as the reference's zero-initialised output blocks do.
#include "common.cuh"

namespace fsb {

constexpr int kPermThreads = 256;
constexpr int kPermUnroll = 4;

// One task = a contiguous range of output-order positions inside one EB.
// ND is the EB's (merged) leg count; descriptor fields live in registers.
template <int ND>
__device__ __forceinline__ void perm_gather_range(const double* __restrict__ in,
                                                  int64_t in_len,
                                                  double* __restrict__ out,
                                                  int64_t out_len,
                                                  const FsPermEB& e, uint32_t start,
                                                  uint32_t count, int32_t* flag) {
    uint32_t dims[ND], dm[ND], ds[ND];
    int64_t os[ND], ns[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) {
        dims[k] = e.dims[k];
        dm[k] = e.divm[k];
        ds[k] = e.divs[k];
        os[k] = e.ostride[k];
        ns[k] = e.nstride[k];
    }
    const int64_t obase = e.obase;
    const int64_t nbase = e.nbase;
    const bool zero_fill = obase < 0;
    const uint32_t end = start + count;
    for (uint32_t p0 = start + threadIdx.x; p0 < end; p0 += kPermThreads * kPermUnroll) {
        double v[kPermUnroll];
        int64_t dst[kPermUnroll];
#pragma unroll
        for (int u = 0; u < kPermUnroll; ++u) {
            const uint32_t p = p0 + u * kPermThreads;
            dst[u] = -1;
            v[u] = 0.0;
            if (p < end) {
                uint32_t q = p;
                int64_t so = obase, dof = nbase;
#pragma unroll
                for (int k = ND - 1; k >= 0; --k) {
                    const uint32_t qq = fast_div(q, dm[k], ds[k]);
                    const uint32_t i = q - qq * dims[k];
                    q = qq;
                    so += static_cast<int64_t>(i) * os[k];
                    dof += static_cast<int64_t>(i) * ns[k];
                }
                if (dof < 0 || dof >= out_len) {
                    raise_flag(flag, FS_ERR_BOUNDS);
                    continue;
                }
                dst[u] = dof;
                if (!zero_fill) {
                    if (so >= 0 && so < in_len) {
                        v[u] = __ldg(in + so);
                    } else {
                        raise_flag(flag, FS_ERR_BOUNDS);
                        dst[u] = -1;
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kPermUnroll; ++u) {
            if (dst[u] >= 0) out[dst[u]] = v[u];
        }
    }
}

__global__ void __launch_bounds__(kPermThreads)
    k_perm_gather(const double* __restrict__ in, int64_t in_len,
                  double* __restrict__ out, int64_t out_len,
                  const FsPermEB* __restrict__ ebs, int64_t n_ebs,
                  const FsPermTask* __restrict__ tasks, int64_t n_tasks,
                  int32_t* flag) {
    __shared__ FsPermEB e;
    static_assert(sizeof(FsPermEB) % 8 == 0, "descriptor must be 8-byte granular");
    constexpr int kWords = sizeof(FsPermEB) / 8;
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
        switch (e.ndim) {
            case 1: perm_gather_range<1>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 2: perm_gather_range<2>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 3: perm_gather_range<3>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 4: perm_gather_range<4>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 5: perm_gather_range<5>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 6: perm_gather_range<6>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 7: perm_gather_range<7>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            case 8: perm_gather_range<8>(in, in_len, out, out_len, e, task.start, task.count, flag); break;
            default:
                if (threadIdx.x == 0) raise_flag(flag, FS_ERR_UNSUPPORTED);
                break;
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
    fsb::k_perm_gather<<<grid, fsb::kPermThreads, 0, fsb::as_stream(stream)>>>(
        d_in, in_len, d_out, out_len, d_ebs, n_ebs, d_tasks, n_tasks, d_flag);
    return fsb::launch_status();
}
