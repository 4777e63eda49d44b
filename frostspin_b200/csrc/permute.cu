// Abelian (U(1) / Z2) block-sparse permute as a batch of strided copies.
//
// Reference behaviour: frostspin/symmetric_tensor/abelian_symmetric_tensor.py
// :103-250 (_numba_abelian_transpose) scatters every entry of every old block to
// its new (block, row, col) with per-element divmod arithmetic.  Here the host
// plan splits the tensor into elementary blocks (one irrep segment per leg), in
// which both the source and destination offsets are affine in the leg indices.
// Legs are ordered by output stride, so the last leg is the output-innermost
// one; positions are decoded with Granlund-Montgomery division by the leg
// sizes (host-computed constants).  Absent source blocks produce zeros, as the
// reference's zero-initialised output blocks do.
#include "common.cuh"

namespace fsb {

constexpr int kPermThreads = 256;
constexpr int kPermUnroll = 4;
constexpr int kPermMaxRows = 1024;   // rows per task (shared-memory row table)

// One task = a range of rows of one elementary block, a row being one run along
// the output-innermost leg (length L).  Phase 1 decodes the outer multi-index
// of every row of the task once (Granlund-Montgomery division by the leg sizes)
// into a shared-memory table of source/destination row offsets, checking both
// ends of each row against the buffers.  Phase 2 walks the task's entries flat:
// entry idx -> (row, i) by one division by L, offsets from the table plus i
// times the innermost strides.  Consecutive threads write consecutive outputs
// (coalesced stores) and read consecutive inputs whenever the source keeps the
// same innermost leg; each thread keeps kPermUnroll loads in flight.
//
// kMulti: the EBs of several independent permutes in one launch; EB e reads
// and writes the buffer pair bufs[e.pad] (the permutes of many CTMRG runs
// advanced in lock step share one launch).
template <bool kMulti>
__global__ void __launch_bounds__(kPermThreads, 4)
    k_perm_gather_t(const double* __restrict__ in0, int64_t in_len0, double* __restrict__ out0,
                    int64_t out_len0, const FsPermBuffers* __restrict__ bufs, int64_t n_bufs,
                    const FsPermEB* __restrict__ ebs, int64_t n_ebs,
                    const FsPermTask* __restrict__ tasks, int64_t n_tasks, int32_t* flag) {
    __shared__ FsPermEB e;
    __shared__ int64_t row_src[kPermMaxRows];
    __shared__ int64_t row_dst[kPermMaxRows];
    static_assert(sizeof(FsPermEB) % 8 == 0, "descriptor must be 8-byte granular");
    constexpr int kWords = sizeof(FsPermEB) / 8;
    for (int64_t t = blockIdx.x; t < n_tasks; t += gridDim.x) {
        const FsPermTask task = tasks[t];
        __syncthreads();  // previous task done with the shared tables
        if (task.eb < 0 || task.eb >= n_ebs || task.count > kPermMaxRows) {
            if (threadIdx.x == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
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
        const double* in = in0;
        double* out = out0;
        int64_t in_len = in_len0, out_len = out_len0;
        if (kMulti) {
            if (e.pad < 0 || e.pad >= n_bufs) {
                if (threadIdx.x == 0) raise_flag(flag, FS_ERR_BOUNDS);
                continue;
            }
            const FsPermBuffers b = bufs[e.pad];
            in = b.in;
            out = b.out;
            in_len = b.in_len;
            out_len = b.out_len;
        }
        const uint32_t L = e.dims[nd - 1];
        const int64_t osL = e.ostride[nd - 1];
        const int64_t nsL = e.nstride[nd - 1];
        const bool zero_fill = e.obase < 0;
        const int nrows = static_cast<int>(task.count);
        for (int j = threadIdx.x; j < nrows; j += kPermThreads) {
            uint32_t q = task.start + static_cast<uint32_t>(j);
            int64_t so = e.obase, dof = e.nbase;
            for (int k = nd - 2; k >= 0; --k) {
                const uint32_t qq = fast_div(q, e.divm[k], e.divs[k]);
                const uint32_t i = q - qq * e.dims[k];
                q = qq;
                so += static_cast<int64_t>(i) * e.ostride[k];
                dof += static_cast<int64_t>(i) * e.nstride[k];
            }
            const int64_t dlast = dof + static_cast<int64_t>(L - 1) * nsL;
            const int64_t slast = so + static_cast<int64_t>(L - 1) * osL;
            bool ok = dof >= 0 && dlast < out_len;
            if (!zero_fill) ok = ok && so >= 0 && slast < in_len;
            if (!ok) {
                raise_flag(flag, FS_ERR_BOUNDS);
                dof = -1;
            }
            row_src[j] = so;
            row_dst[j] = dof;
        }
        __syncthreads();
        const uint32_t total = static_cast<uint32_t>(nrows) * L;
        const uint32_t mL = e.divm[nd - 1], sL = e.divs[nd - 1];
        for (uint32_t i0 = threadIdx.x; i0 < total; i0 += kPermThreads * kPermUnroll) {
            double v[kPermUnroll];
            int64_t dst[kPermUnroll];
#pragma unroll
            for (int u = 0; u < kPermUnroll; ++u) {
                const uint32_t idx = i0 + u * kPermThreads;
                dst[u] = -1;
                v[u] = 0.0;
                if (idx < total) {
                    const uint32_t row = fast_div(idx, mL, sL);
                    const uint32_t i = idx - row * L;
                    const int64_t rd = row_dst[row];
                    if (rd >= 0) {
                        dst[u] = rd + static_cast<int64_t>(i) * nsL;
                        if (!zero_fill) v[u] = __ldg(in + row_src[row] + static_cast<int64_t>(i) * osL);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kPermUnroll; ++u) {
                if (dst[u] >= 0) out[dst[u]] = v[u];
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
    // one wave of resident CTAs (4 per SM at the kernel's register budget)
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 4;
    const int grid = static_cast<int>(n_tasks < max_grid ? n_tasks : max_grid);
    fsb::k_perm_gather_t<false><<<grid, fsb::kPermThreads, 0, fsb::as_stream(stream)>>>(
        d_in, in_len, d_out, out_len, nullptr, 0, d_ebs, n_ebs, d_tasks, n_tasks, d_flag);
    return fsb::launch_status();
}

extern "C" int fs_abelian_permute_multi(const FsPermBuffers* d_bufs, int64_t n_bufs,
                                        const FsPermEB* d_ebs, int64_t n_ebs,
                                        const FsPermTask* d_tasks, int64_t n_tasks,
                                        int32_t* d_flag, void* stream) {
    if (n_tasks < 0 || n_ebs < 0 || n_bufs < 0) return FS_ERR_INVALID_ARG;
    if (n_tasks == 0) return FS_OK;
    if (d_bufs == nullptr || d_ebs == nullptr || d_tasks == nullptr) return FS_ERR_INVALID_ARG;
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 4;
    const int grid = static_cast<int>(n_tasks < max_grid ? n_tasks : max_grid);
    fsb::k_perm_gather_t<true><<<grid, fsb::kPermThreads, 0, fsb::as_stream(stream)>>>(
        nullptr, 0, nullptr, 0, d_bufs, n_bufs, d_ebs, n_ebs, d_tasks, n_tasks, d_flag);
    return fsb::launch_status();
}
