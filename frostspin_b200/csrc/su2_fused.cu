// Fused SU(2) permute for the thin simple blocks: gather, recoupling product and
// scatter in one pass over the data.
//
// Reference behaviour: LieGroupSymmetricTensor._lie_permute_data ->
// fill_blocks_out -> permute_simple_block (frostspin/symmetric_tensor/
// lie_group_symmetric_tensor.py:96-265, :735-835): for every simple block, the
// sub-blocks of every input sector are gathered (strided view with the
// external legs permuted), multiplied by the block's recoupling isometry
// (new += U_sector @ old) and scattered into the output sectors.
//
// Here a simple block is a group with K input rows (input sectors x
// structural multiplicities), M = K output rows and E columns (the external
// multi-index, output leg order).  A task is a run of columns of one group.
// The CTA stages the group's recoupling matrix U (M x K <= 32 x 32) and its
// piece descriptors in shared memory; each thread then takes one column at a
// time: it decodes the column into the external leg indices (Granlund-
// Montgomery division by invariant integers), gathers the K input values of
// that column from every input piece (its own slots of a shared array),
// multiplies by U from shared memory (broadcast reads) and writes the M
// results to the output pieces.  Consecutive threads take consecutive
// columns, i.e. consecutive values of the output-innermost leg, so the stores
// are coalesced; the loads are coalesced where the source keeps that leg
// innermost.  Every address is checked against its buffer (skipped and
// flagged, FS_ERR_BOUNDS); the host validates the tables before the call.
// Traffic: 8 bytes read and 8 written per coefficient (the three-launch form
// moves three times that).  As built it is slower than the three launches on
// the SU(2) chi = 256 workload (2.6 s against 1.6 s over three iterations):
// every column decodes its whole external multi-index and every piece's
// offset (about 12 integer operations per coefficient, against about 3 in the
// permute kernel, which decodes once per row of the output-innermost leg), so
// the library keeps it off by default.
#include "common.cuh"

namespace fsb {

constexpr int kSu2Threads = 128;
constexpr int kSu2MaxRows = 32;     // M, K of a fused group
constexpr int kSu2MaxPieces = 16;   // input and output pieces of a fused group

struct Su2Smem {
    double u[kSu2MaxRows * kSu2MaxRows];
    double x[kSu2MaxRows][kSu2Threads];
    FsSu2Piece in[kSu2MaxPieces];
    FsSu2Piece out[kSu2MaxPieces];
};

__device__ __forceinline__ int64_t ext_offset(const FsSu2Piece& p, const uint32_t (&e)[FS_SU2_MAXD],
                                              int ndim) {
    int64_t off = 0;
#pragma unroll
    for (int l = 0; l < FS_SU2_MAXD; ++l)
        if (l < ndim) off += static_cast<int64_t>(e[l]) * p.ext[l];
    return off;
}

__global__ void __launch_bounds__(kSu2Threads)
    k_su2_fused(const double* __restrict__ src, int64_t src_len, double* __restrict__ out,
                int64_t out_len, const FsSu2Group* __restrict__ groups, int64_t n_groups,
                const FsSu2Piece* __restrict__ pieces, int64_t n_pieces,
                const double* __restrict__ U, int64_t u_len, const FsPermTask* __restrict__ tasks,
                int64_t n_tasks, int32_t* flag) {
    __shared__ Su2Smem sm;
    const int tid = threadIdx.x;
    for (int64_t t = blockIdx.x; t < n_tasks; t += gridDim.x) {
        const FsPermTask tk = tasks[t];
        __syncthreads();  // the previous task is done with the shared arrays
        if (tk.eb < 0 || tk.eb >= n_groups) {
            if (tid == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
        const FsSu2Group g = groups[tk.eb];
        const bool ok = g.M >= 0 && g.M <= kSu2MaxRows && g.K >= 0 && g.K <= kSu2MaxRows &&
                        g.ndim >= 0 && g.ndim <= FS_SU2_MAXD && g.in_count >= 0 &&
                        g.in_count <= kSu2MaxPieces && g.out_count >= 0 &&
                        g.out_count <= kSu2MaxPieces && g.in_first >= 0 &&
                        g.in_first + g.in_count <= n_pieces && g.out_first >= 0 &&
                        g.out_first + g.out_count <= n_pieces && g.u_off >= 0 &&
                        g.u_off + static_cast<int64_t>(g.M) * g.K <= u_len;
        if (!ok) {
            if (tid == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
        for (int i = tid; i < g.M * g.K; i += kSu2Threads) sm.u[i] = __ldg(U + g.u_off + i);
        if (tid < g.in_count) sm.in[tid] = pieces[g.in_first + tid];
        if (tid >= 32 && tid - 32 < g.out_count) sm.out[tid - 32] = pieces[g.out_first + tid - 32];
        __syncthreads();
        const int64_t c_end = static_cast<int64_t>(tk.start) + tk.count;
        for (int64_t c = static_cast<int64_t>(tk.start) + tid; c < c_end && c < g.ncols;
             c += kSu2Threads) {
            // external leg indices of column c (output order, last leg fastest)
            uint32_t e[FS_SU2_MAXD];
            uint32_t rem = static_cast<uint32_t>(c);
#pragma unroll
            for (int l = FS_SU2_MAXD - 1; l >= 0; --l) {
                if (l < g.ndim) {
                    const uint32_t q = fast_div(rem, g.divm[l], g.divs[l]);
                    e[l] = rem - q * g.dims[l];
                    rem = q;
                } else {
                    e[l] = 0;
                }
            }
            // gather the K inputs of this column
            for (int p = 0; p < g.in_count; ++p) {
                const FsSu2Piece& pc = sm.in[p];
                const bool present = pc.base >= 0;
                const int64_t b = pc.base + ext_offset(pc, e, g.ndim);
                for (int sr = 0; sr < pc.sr; ++sr) {
                    for (int sc = 0; sc < pc.sc; ++sc) {
                        const int k = pc.row0 + sr * pc.sc + sc;
                        double v = 0.0;
                        if (present) {
                            const int64_t off = b + sr * pc.sr_stride + sc * pc.sc_stride;
                            if (off >= 0 && off < src_len && k < kSu2MaxRows)
                                v = __ldg(src + off);
                            else
                                raise_flag(flag, FS_ERR_BOUNDS);
                        }
                        if (k < kSu2MaxRows) sm.x[k][tid] = v;
                    }
                }
            }
            double x[kSu2MaxRows];
#pragma unroll
            for (int k = 0; k < kSu2MaxRows; ++k) x[k] = (k < g.K) ? sm.x[k][tid] : 0.0;
            // recouple and scatter the M outputs
            for (int q = 0; q < g.out_count; ++q) {
                const FsSu2Piece& pc = sm.out[q];
                const int64_t b = pc.base + ext_offset(pc, e, g.ndim);
                for (int sr = 0; sr < pc.sr; ++sr) {
                    for (int sc = 0; sc < pc.sc; ++sc) {
                        const int i = pc.row0 + sr * pc.sc + sc;
                        if (i >= g.M) {
                            raise_flag(flag, FS_ERR_BOUNDS);
                            continue;
                        }
                        const double* ui = sm.u + i * g.K;
                        double acc = 0.0;
#pragma unroll
                        for (int k = 0; k < kSu2MaxRows; ++k)
                            if (k < g.K) acc = fma(ui[k], x[k], acc);
                        const int64_t off = b + sr * pc.sr_stride + sc * pc.sc_stride;
                        if (off >= 0 && off < out_len)
                            out[off] = acc;
                        else
                            raise_flag(flag, FS_ERR_BOUNDS);
                    }
                }
            }
        }
    }
}

}  // namespace fsb

extern "C" int fs_su2_fused_limits(int32_t* max_rows, int32_t* max_pieces, int32_t* threads) {
    if (max_rows == nullptr || max_pieces == nullptr || threads == nullptr)
        return FS_ERR_INVALID_ARG;
    *max_rows = fsb::kSu2MaxRows;
    *max_pieces = fsb::kSu2MaxPieces;
    *threads = fsb::kSu2Threads;
    return FS_OK;
}

extern "C" int fs_su2_permute_fused(const double* d_src, int64_t src_len, double* d_out,
                                    int64_t out_len, const FsSu2Group* d_groups,
                                    int64_t n_groups, const FsSu2Piece* d_pieces,
                                    int64_t n_pieces, const double* d_u, int64_t u_len,
                                    const FsPermTask* d_tasks, int64_t n_tasks, int32_t* d_flag,
                                    void* stream) {
    if (src_len < 0 || out_len < 0 || n_groups < 0 || n_pieces < 0 || u_len < 0 || n_tasks < 0)
        return FS_ERR_INVALID_ARG;
    if (n_tasks == 0) return FS_OK;
    if (d_out == nullptr || d_groups == nullptr || d_pieces == nullptr || d_tasks == nullptr ||
        (d_u == nullptr && u_len > 0) || (d_src == nullptr && src_len > 0))
        return FS_ERR_INVALID_ARG;
    // resident CTAs: the shared arrays (~45 KB) allow 4 per SM
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 4;
    const int grid = static_cast<int>(n_tasks < max_grid ? n_tasks : max_grid);
    fsb::k_su2_fused<<<grid, fsb::kSu2Threads, 0, fsb::as_stream(stream)>>>(
        d_src, src_len, d_out, out_len, d_groups, n_groups, d_pieces, n_pieces, d_u, u_len,
        d_tasks, n_tasks, d_flag);
    return fsb::launch_status();
}
