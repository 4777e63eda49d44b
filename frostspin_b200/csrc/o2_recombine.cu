// O(2) <-> U(1) change of basis of symmetric-tensor blocks.
//
// Reference behaviour (frostspin/symmetric_tensor/o2_symmetric_tensor.py): an
// O(2) tensor stores its 0odd and 0even blocks and the U(1) blocks of charge
// n > 0.  Its U(1) form adds the charge -n blocks, obtained from the charge n
// ones by the Sz reflection with a sign per row and per column
// (_generate_neg_sz_blocks :798-851, _numba_generate_refl_block :327-354),
// and the charge-0 block, an orthogonal mix of the 0odd and 0even blocks
// (_numba_merge_b0oe :269-288); back from U(1), the charge-0 block is split
// into 0odd and 0even again (_numba_split_b0 :291-310).
//
// Every one of these is a separable gather: output element (i, j) of a block is
// a sum over at most four terms t of rcoef_t[i] * src_t[ridx_t[i], cidx_t[j]] *
// ccoef_t[j].  The host builds the per-row and per-column tables; one launch
// covers every block of a cast.  A CTA walks output rows (grid-stride), loads
// the row's index and coefficient of each term once, and its threads stride
// over the columns, so output stores are coalesced.  Products are rounded
// step by step in the reference's order ((rcoef * x) * ccoef, terms summed in
// order, no fused multiply-add), so the results equal the reference's loops.
#include "common.cuh"

namespace fsb {

constexpr int kO2Threads = 128;

__global__ void __launch_bounds__(kO2Threads)
    k_o2_recombine(const double* __restrict__ src, int64_t src_len, double* __restrict__ out,
                   int64_t out_len, const FsO2Block* __restrict__ blocks,
                   const int64_t* __restrict__ index, const double* __restrict__ coef,
                   int32_t* flag) {
    const FsO2Block& blk = blocks[blockIdx.y];
    const int nt = blk.nterms < FS_O2_MAXTERMS ? blk.nterms : FS_O2_MAXTERMS;
    for (int64_t i = blockIdx.x; i < blk.nrows; i += gridDim.x) {
        int64_t rbase[FS_O2_MAXTERMS];
        double rc[FS_O2_MAXTERMS];
#pragma unroll
        for (int t = 0; t < FS_O2_MAXTERMS; ++t) {
            if (t < nt) {
                const FsO2Term& tm = blk.terms[t];
                rbase[t] = tm.src_off + index[tm.ridx_off + i] * tm.rs;
                rc[t] = coef[tm.rcoef_off + i];
            }
        }
        const int64_t orow = blk.out_off + i * blk.ncols;
        for (int64_t j = threadIdx.x; j < blk.ncols; j += kO2Threads) {
            double acc = 0.0;
#pragma unroll
            for (int t = 0; t < FS_O2_MAXTERMS; ++t) {
                if (t < nt) {
                    const FsO2Term& tm = blk.terms[t];
                    const int64_t pos = rbase[t] + index[tm.cidx_off + j] * tm.cs;
                    if (pos < 0 || pos >= src_len) {
                        raise_flag(flag, FS_ERR_BOUNDS);
                        continue;
                    }
                    acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(rc[t], src[pos]),
                                                   coef[tm.ccoef_off + j]));
                }
            }
            const int64_t o = orow + j;
            if (o < 0 || o >= out_len) {
                raise_flag(flag, FS_ERR_BOUNDS);
                continue;
            }
            out[o] = acc;
        }
    }
}

}  // namespace fsb

extern "C" int fs_o2_recombine(const double* d_src, int64_t src_len, double* d_out,
                               int64_t out_len, const FsO2Block* d_blocks, int64_t n_blocks,
                               const int64_t* d_index, const double* d_coef, int64_t max_rows,
                               int32_t* d_flag, void* stream) {
    if (n_blocks < 0 || max_rows < 0 || src_len < 0 || out_len < 0) return FS_ERR_INVALID_ARG;
    if (n_blocks == 0 || max_rows == 0) return FS_OK;
    if (d_blocks == nullptr || d_index == nullptr || d_coef == nullptr || d_out == nullptr)
        return FS_ERR_INVALID_ARG;
    if (d_src == nullptr && src_len > 0) return FS_ERR_INVALID_ARG;
    if (n_blocks > 65535) return FS_ERR_TOO_LARGE;
    const int64_t cap = static_cast<int64_t>(fsb::num_sms()) * 8;
    const int gx = static_cast<int>(max_rows < cap ? max_rows : cap);
    fsb::k_o2_recombine<<<dim3(gx, static_cast<unsigned>(n_blocks)), fsb::kO2Threads, 0,
                          fsb::as_stream(stream)>>>(d_src, src_len, d_out, out_len, d_blocks,
                                                    d_index, d_coef, d_flag);
    return fsb::launch_status();
}
