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
// multi-index, output leg order).  The CTA stages the group's recoupling
// matrix U (M x K <= 32 x 32) in shared memory and applies it column by column:
// the K inputs of a column are gathered from the input pieces, multiplied by U
// (broadcast reads) and the M results scattered to the output pieces.  Every
// row of a task is checked against its buffer (skipped and flagged,
// FS_ERR_BOUNDS); the host validates the tables before the call.
// Traffic: 8 bytes read and 8 written per coefficient (the three-launch form
// moves three times that).
//
// Work split: a task is a range of columns of one group that covers at most
// kSu2TaskRows rows of the output-innermost leg (a row = one value of the outer
// external legs, L = its innermost dimension columns).  Phase 1 decodes each
// outer row once (Granlund-Montgomery division by the leg sizes) and writes,
// per group row k (input) and m (output), the element offset of that row's
// first column into shared tables, after checking both ends of the row against
// the buffer.  Phase 2 streams the columns: a thread carries S columns at once
// (S * K <= 32 operand doubles in registers) and issues every load of the pass
// before the FMAs, so each thread keeps up to 32 loads in flight; per
// coefficient it costs one shared-memory offset read and one multiply-add of
// address arithmetic.  Consecutive threads take consecutive columns, so the
// stores are coalesced and so are the loads wherever the source keeps the
// innermost output leg innermost.  (A first form decoded the whole multi-index
// of every column in every thread, one column at a time: latency bound, and
// slower than the three launches.)
#include "common.cuh"

namespace fsb {

constexpr int kSu2Threads = 256;
constexpr int kSu2MaxRows = 32;     // M, K of a fused group
constexpr int kSu2MaxPieces = 16;   // input and output pieces of a fused group
constexpr int kSu2TaskRows = FS_SU2_TASK_ROWS;   // outer rows of one task

struct Su2Smem {
    double u[kSu2MaxRows * kSu2MaxRows];
    int64_t kbase[kSu2MaxRows][kSu2TaskRows];   // input row k: offset of the row (-1: absent)
    int64_t mbase[kSu2MaxRows][kSu2TaskRows];   // output row m (-1: skipped)
    int64_t kext[kSu2MaxRows];                  // stride of the innermost leg, input row k
    int64_t mext[kSu2MaxRows];
    uint32_t e[kSu2TaskRows][FS_SU2_MAXD];      // decoded outer legs of the task's rows
    FsSu2Piece pc[2 * kSu2MaxPieces];
};

// Phase 2 for one task: columns [c_begin, c_end) of rows r0.. (local rows)
template <int KB, int S>
__device__ __forceinline__ void su2_stream(const Su2Smem& sm, const double* __restrict__ src,
                                           double* __restrict__ out, int M, int K, uint32_t L,
                                           uint32_t mL, uint32_t sL, int64_t r0, int64_t c_begin,
                                           int64_t c_end) {
    for (int64_t c0 = c_begin + threadIdx.x; c0 < c_end; c0 += static_cast<int64_t>(kSu2Threads) * S) {
        int rr[S];
        int64_t ii[S];
        bool ok[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int64_t c = c0 + static_cast<int64_t>(s) * kSu2Threads;
            ok[s] = c < c_end;
            const uint32_t cc = static_cast<uint32_t>(ok[s] ? c : c_begin);
            const uint32_t q = fast_div(cc, mL, sL);
            rr[s] = static_cast<int>(static_cast<int64_t>(q) - r0);
            ii[s] = static_cast<int64_t>(cc - q * L);
        }
        double x[S][KB];
#pragma unroll
        for (int k = 0; k < KB; ++k) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                double v = 0.0;
                if (k < K && ok[s]) {
                    const int64_t b = sm.kbase[k][rr[s]];
                    if (b >= 0) v = __ldg(src + b + ii[s] * sm.kext[k]);
                }
                x[s][k] = v;
            }
        }
        for (int m = 0; m < M; ++m) {
            const double* um = sm.u + m * K;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < KB; ++k)
                    if (k < K) acc = fma(um[k], x[s][k], acc);
                if (ok[s]) {
                    const int64_t b = sm.mbase[m][rr[s]];
                    if (b >= 0) out[b + ii[s] * sm.mext[m]] = acc;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kSu2Threads)
    k_su2_fused(const double* __restrict__ src, int64_t src_len, double* __restrict__ out,
                int64_t out_len, const FsSu2Group* __restrict__ groups, int64_t n_groups,
                const FsSu2Piece* __restrict__ pieces, int64_t n_pieces,
                const double* __restrict__ U, int64_t u_len, const FsPermTask* __restrict__ tasks,
                int64_t n_tasks, int32_t* flag) {
    extern __shared__ __align__(16) uint8_t su2_raw[];
    Su2Smem& sm = *reinterpret_cast<Su2Smem*>(su2_raw);
    const int tid = threadIdx.x;
    for (int64_t t = blockIdx.x; t < n_tasks; t += gridDim.x) {
        const FsPermTask tk = tasks[t];
        __syncthreads();  // the previous task is done with the shared tables
        if (tk.eb < 0 || tk.eb >= n_groups) {
            if (tid == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
        const FsSu2Group g = groups[tk.eb];
        const int nd = g.ndim;
        const bool ok = g.M >= 0 && g.M <= kSu2MaxRows && g.K >= 0 && g.K <= kSu2MaxRows &&
                        nd >= 0 && nd <= FS_SU2_MAXD && g.in_count >= 0 &&
                        g.in_count <= kSu2MaxPieces && g.out_count >= 0 &&
                        g.out_count <= kSu2MaxPieces && g.in_first >= 0 &&
                        g.in_first + g.in_count <= n_pieces && g.out_first >= 0 &&
                        g.out_first + g.out_count <= n_pieces && g.u_off >= 0 &&
                        g.u_off + static_cast<int64_t>(g.M) * g.K <= u_len;
        if (!ok) {
            if (tid == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
        // the innermost output leg and the task's rows of the outer ones
        const uint32_t L = nd > 0 ? g.dims[nd - 1] : 1u;
        const uint32_t mL = nd > 0 ? g.divm[nd - 1] : 0u, sL = nd > 0 ? g.divs[nd - 1] : 0u;
        const int64_t c_begin = tk.start;
        const int64_t c_end = min(static_cast<int64_t>(tk.start) + tk.count, g.ncols);
        if (c_end <= c_begin || L == 0) continue;
        const int64_t r0 = static_cast<int64_t>(fast_div(static_cast<uint32_t>(c_begin), mL, sL));
        const int64_t r1 = static_cast<int64_t>(fast_div(static_cast<uint32_t>(c_end - 1), mL, sL)) + 1;
        const int nr = static_cast<int>(r1 - r0);
        if (nr > kSu2TaskRows) {
            if (tid == 0) raise_flag(flag, FS_ERR_BOUNDS);
            continue;
        }
        const int npc = g.in_count + g.out_count;
        for (int i = tid; i < g.M * g.K; i += kSu2Threads) sm.u[i] = __ldg(U + g.u_off + i);
        if (tid < g.in_count) sm.pc[tid] = pieces[g.in_first + tid];
        if (tid >= 32 && tid - 32 < g.out_count) sm.pc[g.in_count + tid - 32] = pieces[g.out_first + tid - 32];
        for (int j = tid; j < kSu2MaxRows * nr; j += kSu2Threads) {
            sm.kbase[j / nr][j % nr] = -1;   // rows no piece covers read zeros
            sm.mbase[j / nr][j % nr] = -1;   // and are not written
        }
        // phase 1a: outer legs of every row
        for (int j = tid; j < nr; j += kSu2Threads) {
            uint32_t rem = static_cast<uint32_t>(r0 + j);
            for (int l = nd - 2; l >= 0; --l) {
                const uint32_t q = fast_div(rem, g.divm[l], g.divs[l]);
                sm.e[j][l] = rem - q * g.dims[l];
                rem = q;
            }
        }
        __syncthreads();
        // phase 1b: per (piece, row) the offset of every group row it holds
        for (int j = tid; j < npc * nr; j += kSu2Threads) {
            const int p = j / nr, row = j - p * nr;
            const FsSu2Piece& pc = sm.pc[p];
            const bool is_in = p < g.in_count;
            int64_t off = pc.base;
            for (int l = 0; l + 1 < nd; ++l) off += static_cast<int64_t>(sm.e[row][l]) * pc.ext[l];
            const int64_t ext = nd > 0 ? pc.ext[nd - 1] : 0;
            const int64_t len = is_in ? src_len : out_len;
            const int lim = is_in ? g.K : g.M;
            for (int a = 0; a < pc.sr; ++a) {
                for (int b = 0; b < pc.sc; ++b) {
                    const int k = pc.row0 + a * pc.sc + b;
                    if (k < 0 || k >= lim) {
                        raise_flag(flag, FS_ERR_BOUNDS);
                        continue;
                    }
                    int64_t o = -1;
                    if (!is_in || pc.base >= 0) {
                        o = off + a * pc.sr_stride + b * pc.sc_stride;
                        const int64_t last = o + static_cast<int64_t>(L - 1) * ext;
                        if (o < 0 || last < 0 || o >= len || last >= len) {
                            raise_flag(flag, FS_ERR_BOUNDS);
                            o = -1;
                        }
                    }
                    if (is_in) {
                        sm.kbase[k][row] = o;
                        if (row == 0) sm.kext[k] = ext;
                    } else {
                        sm.mbase[k][row] = o;
                        if (row == 0) sm.mext[k] = ext;
                    }
                }
            }
        }
        __syncthreads();
        if (g.K <= 4)
            su2_stream<4, 4>(sm, src, out, g.M, g.K, L, mL, sL, r0, c_begin, c_end);
        else if (g.K <= 8)
            su2_stream<8, 4>(sm, src, out, g.M, g.K, L, mL, sL, r0, c_begin, c_end);
        else if (g.K <= 16)
            su2_stream<16, 2>(sm, src, out, g.M, g.K, L, mL, sL, r0, c_begin, c_end);
        else
            su2_stream<32, 1>(sm, src, out, g.M, g.K, L, mL, sL, r0, c_begin, c_end);
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
    constexpr int smem = static_cast<int>(sizeof(fsb::Su2Smem));
    const int st = fsb::configure_smem(reinterpret_cast<const void*>(fsb::k_su2_fused), smem);
    if (st != FS_OK) return st;
    // resident CTAs: 256 threads and ~38 KB of shared tables, 4 per SM
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 4;
    const int grid = static_cast<int>(n_tasks < max_grid ? n_tasks : max_grid);
    fsb::k_su2_fused<<<grid, fsb::kSu2Threads, smem, fsb::as_stream(stream)>>>(
        d_src, src_len, d_out, out_len, d_groups, n_groups, d_pieces, n_pieces, d_u, u_len,
        d_tasks, n_tasks, d_flag);
    return fsb::launch_status();
}
