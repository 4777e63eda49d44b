// Grouped FP64 GEMM over irrep sectors: the plain double-precision path, on the
// FP64 tensor cores (DMMA, mma.sync m8n8k4 f64 -- Blackwell has no tcgen05 kind
// for f64, so this is the FP64 tensor path of sm_100a).
//
// Reference behaviour: SymmetricTensor.__matmul__ (frostspin/symmetric_tensor/
// symmetric_tensor.py:453-489) calls numpy's dgemm once per shared irrep block.
// Here every sector product of one contraction is a problem in one launch; the
// host flattens all output tiles of all problems into a tile list and CTAs
// stride over it (a static persistent schedule), so sectors of very uneven
// sizes share the machine.
//
// 64x64 output tile per CTA, 4 warps of 32x32 (4x4 m8n8 fragments), k staged
// 16 deep through a 3-stage cp.async pipeline, 3 CTAs per SM.  Sector blocks
// start at any element offset, so copies are 8-byte cp.async with zero fill at
// the edges.  Shared layouts follow the global layout of each operand (row- or
// column-major, per problem; the tile body is instantiated for the four
// combinations) with padding chosen so that every fragment load of a half warp
// touches 32 distinct banks.
#include "common.cuh"

namespace fsb {

constexpr int kTM = 64;
constexpr int kTN = 64;
constexpr int kTK = 16;
constexpr int kStages = 3;
constexpr int kGemmThreads = 128;
constexpr int kLdK = kTK + 4;   // stride of a [row][k] tile (20 doubles, 4 mod 16)
constexpr int kLdR = kTM + 4;   // stride of a [k][row] tile (68 doubles, 4 mod 16)
constexpr int kOpTile = kTM * kLdK;  // >= kTK * kLdR
static_assert(kTM == kTN, "square tiles: one stage size for A and B");
static_assert(kOpTile >= kTK * kLdR, "stage too small for the k-major layout");
constexpr int kStageDoubles = 2 * kOpTile;
constexpr size_t kGemmSmem = sizeof(double) * kStageDoubles * kStages;

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n));
}

__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::);
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// One k slice of op(A) (rows m0.., k0..) and op(B) (k0.., cols n0..) into a stage.
// A stage holds A in [m][k] (TA == 0) or [k][m] (TA == 1) and B in [k][n]
// (TB == 0) or [n][k] (TB == 1): always the global contiguous direction
// innermost, so the copies are coalesced.
template <bool TA, bool TB>
__device__ __forceinline__ void load_stage(const FsGemmProblem& p, int m0, int n0, int k0,
                                           double* stage) {
    double* sa = stage;
    double* sb = stage + kOpTile;
#pragma unroll
    for (int u = 0; u < (kTM * kTK) / kGemmThreads; ++u) {
        const int e = threadIdx.x + u * kGemmThreads;
        const int k = TA ? e / kTM : e % kTK;
        const int m = TA ? e % kTM : e / kTK;
        const bool ok = (m0 + m < p.M) && (k0 + k < p.K);
        const int64_t off = TA ? static_cast<int64_t>(k0 + k) * p.lda + (m0 + m)
                               : static_cast<int64_t>(m0 + m) * p.lda + (k0 + k);
        cp_async8(sa + (TA ? k * kLdR + m : m * kLdK + k), ok ? p.A + off : p.A, ok);
    }
#pragma unroll
    for (int u = 0; u < (kTN * kTK) / kGemmThreads; ++u) {
        const int e = threadIdx.x + u * kGemmThreads;
        const int k = TB ? e % kTK : e / kTN;
        const int n = TB ? e / kTK : e % kTN;
        const bool ok = (n0 + n < p.N) && (k0 + k < p.K);
        const int64_t off = TB ? static_cast<int64_t>(n0 + n) * p.ldb + (k0 + k)
                               : static_cast<int64_t>(k0 + k) * p.ldb + (n0 + n);
        cp_async8(sb + (TB ? n * kLdK + k : k * kLdR + n), ok ? p.B + off : p.B, ok);
    }
}

// The DMMAs of one staged k slice for one warp's 32x32 block: k steps at or
// beyond k_left, fragment rows at or beyond rows_left and fragment columns at
// or beyond cols_left (all warp-uniform) are skipped.
template <bool TA, bool TB>
__device__ __forceinline__ void mma_slice(double (&acc)[4][4][2], const double* sa,
                                          const double* sb, int k_left, int rows_left,
                                          int cols_left) {
    constexpr int a_step_i = TA ? 8 : 8 * kLdK;   // next fragment row block
    constexpr int a_step_k = TA ? 4 * kLdR : 4;   // next k-step
    constexpr int b_step_j = TB ? 8 * kLdK : 8;
    constexpr int b_step_k = TB ? 4 : 4 * kLdR;
#pragma unroll
    for (int ks = 0; ks < kTK / 4; ++ks) {
        if (ks * 4 >= k_left) break;
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = sa[ks * a_step_k + i * a_step_i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = sb[ks * b_step_k + j * b_step_j];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (i * 8 >= rows_left) break;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j * 8 >= cols_left) break;
                dmma(acc[i][j], a[i], b[j]);
            }
        }
    }
}

// One 64x64 output tile: the cp.async pipeline over k and the DMMA fragments.
template <bool TA, bool TB>
__device__ __forceinline__ void dgemm_tile(const FsGemmProblem& p, int m0, int n0,
                                           double* smem) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wm = (warp & 1) * 32;
    const int wn = (warp >> 1) * 32;
    const int fr = lane >> 2;  // fragment row (A, C) / column (B)
    const int fk = lane & 3;   // fragment k (A, B) / column pair (C)

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    // per-thread fragment offsets inside a stage (k = 0)
    const int a_off = TA ? fk * kLdR + wm + fr : (wm + fr) * kLdK + fk;
    const int b_off = TB ? (wn + fr) * kLdK + fk : fk * kLdR + wn + fr;

    const int nk = (p.K + kTK - 1) / kTK;
    __syncthreads();  // every warp is done with the previous tile's stages
#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) load_stage<TA, TB>(p, m0, n0, s * kTK, smem + s * kStageDoubles);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        {
            const int nxt = kt + kStages - 1;
            if (nxt < nk)
                load_stage<TA, TB>(p, m0, n0, nxt * kTK, smem + (nxt % kStages) * kStageDoubles);
            cp_async_commit();
        }
        const double* sa = smem + (kt % kStages) * kStageDoubles + a_off;
        const double* sb = smem + (kt % kStages) * kStageDoubles + kOpTile + b_off;
        // the full padded slice: at 168 registers this kernel has no room for
        // the edge tests (the streaming kernel skips padded fragments)
        mma_slice<TA, TB>(acc, sa, sb, kTK, kTM, kTN);
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = m0 + wm + i * 8 + fr;
        if (gi >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = n0 + wn + j * 8 + fk * 2 + h;
                if (gj >= p.N) continue;
                double* c = p.C + static_cast<int64_t>(gi) * p.ldc + gj;
                const double v = p.alpha * acc[i][j][h];
                *c = (p.beta == 0.0) ? v : fma(p.beta, *c, v);
            }
        }
    }
}

__global__ void __launch_bounds__(kGemmThreads, 3)
    k_grouped_dgemm(const FsGemmProblem* __restrict__ problems, int64_t n_problems,
                    const FsGemmTile* __restrict__ tiles, int64_t n_tiles) {
    extern __shared__ __align__(16) double smem[];
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const FsGemmTile tile = tiles[t];
        if (tile.problem < 0 || tile.problem >= n_problems) continue;
        const FsGemmProblem p = problems[tile.problem];
        const int m0 = tile.tm * kTM;
        const int n0 = tile.tn * kTN;
        if (m0 >= p.M || n0 >= p.N) continue;
        switch ((p.transA ? 2 : 0) | (p.transB ? 1 : 0)) {
            case 0: dgemm_tile<false, false>(p, m0, n0, smem); break;
            case 1: dgemm_tile<false, true>(p, m0, n0, smem); break;
            case 2: dgemm_tile<true, false>(p, m0, n0, smem); break;
            default: dgemm_tile<true, true>(p, m0, n0, smem); break;
        }
    }
}

// Streaming variant for launches whose problems share both transpose flags,
// used for short-K sector products (wide recouplings and projector
// applications with K of a few tens): one cp.async ring runs continuously
// across the CTA's tiles, so the first k slices of the next tile load while
// the current tile finishes and writes its outputs, and fragments or k steps
// wholly outside the problem (M, N, K padding of the 64x64x16 tiling) issue no
// DMMA.  Tiles of problems with K = 0 consume no stage (their output is
// beta * C).
struct TileCursor {
    int64_t t;
    FsGemmProblem p;
    int m0, n0, nk;
};

__device__ __forceinline__ bool cursor_seek(TileCursor& c, int64_t t,
                                            const FsGemmProblem* __restrict__ problems,
                                            int64_t n_problems,
                                            const FsGemmTile* __restrict__ tiles, int64_t n_tiles,
                                            bool need_k) {
    for (; t < n_tiles; t += gridDim.x) {
        const FsGemmTile tile = tiles[t];
        if (tile.problem < 0 || tile.problem >= n_problems) continue;
        c.p = problems[tile.problem];
        c.m0 = tile.tm * kTM;
        c.n0 = tile.tn * kTN;
        if (c.m0 >= c.p.M || c.n0 >= c.p.N) continue;
        c.nk = (c.p.K + kTK - 1) / kTK;
        if (need_k && c.nk == 0) continue;
        c.t = t;
        return true;
    }
    c.t = n_tiles;
    return false;
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(kGemmThreads, 3)
    k_grouped_dgemm_stream(const FsGemmProblem* __restrict__ problems, int64_t n_problems,
                           const FsGemmTile* __restrict__ tiles, int64_t n_tiles) {
    extern __shared__ __align__(16) double smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wm = (warp & 1) * 32;
    const int wn = (warp >> 1) * 32;
    const int fr = lane >> 2;
    const int fk = lane & 3;
    const int a_off = TA ? fk * kLdR + wm + fr : (wm + fr) * kLdK + fk;
    const int b_off = TB ? (wn + fr) * kLdK + fk : fk * kLdR + wn + fr;

    // loader: the next (tile, k slice) to fetch; tiles without k slices skipped
    TileCursor ld;
    bool ld_ok = cursor_seek(ld, blockIdx.x, problems, n_problems, tiles, n_tiles, true);
    int ld_k = 0;
    int64_t issued = 0;
    auto issue = [&]() {
        if (ld_ok) {
            load_stage<TA, TB>(ld.p, ld.m0, ld.n0, ld_k * kTK,
                               smem + (issued % kStages) * kStageDoubles);
            ++issued;
            if (++ld_k == ld.nk) {
                ld_k = 0;
                ld_ok = cursor_seek(ld, ld.t + gridDim.x, problems, n_problems, tiles, n_tiles,
                                    true);
            }
        }
        cp_async_commit();
    };

    // consumer: every tile of this CTA in order (K = 0 tiles included)
    TileCursor cs;
    bool cs_ok = cursor_seek(cs, blockIdx.x, problems, n_problems, tiles, n_tiles, false);
    int cs_k = 0;
    int64_t consumed = 0;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) issue();

    while (cs_ok) {
        if (cs_k < cs.nk) {
            // stage `consumed` is the consumed-th issued one: its group is
            // complete once at most kStages - 2 newer groups are pending
            cp_async_wait<kStages - 2>();
            __syncthreads();  // and every warp is done with the slot refilled next
            issue();
            const double* sa = smem + (consumed % kStages) * kStageDoubles + a_off;
            const double* sb = smem + (consumed % kStages) * kStageDoubles + kOpTile + b_off;
            mma_slice<TA, TB>(acc, sa, sb, cs.p.K - cs_k * kTK, cs.p.M - (cs.m0 + wm),
                              cs.p.N - (cs.n0 + wn));
            ++consumed;
            ++cs_k;
        }
        if (cs_k < cs.nk) continue;
        // tile done: write it while the next tile's first slices load
        const FsGemmProblem& p = cs.p;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gi = cs.m0 + wm + i * 8 + fr;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int gj = cs.n0 + wn + j * 8 + fk * 2 + h;
                    if (gi < p.M && gj < p.N) {
                        double* c = p.C + static_cast<int64_t>(gi) * p.ldc + gj;
                        const double v = p.alpha * acc[i][j][h];
                        *c = (p.beta == 0.0) ? v : fma(p.beta, *c, v);
                    }
                    acc[i][j][h] = 0.0;
                }
            }
        }
        cs_k = 0;
        cs_ok = cursor_seek(cs, cs.t + gridDim.x, problems, n_problems, tiles, n_tiles, false);
    }
    cp_async_wait<0>();
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
    const int cfg = fsb::configure_smem(reinterpret_cast<const void*>(fsb::k_grouped_dgemm),
                                        static_cast<int>(fsb::kGemmSmem));
    if (cfg != FS_OK) return cfg;
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 3;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    fsb::k_grouped_dgemm<<<grid, fsb::kGemmThreads, fsb::kGemmSmem, fsb::as_stream(stream)>>>(
        d_problems, n_problems, d_tiles, n_tiles);
    return fsb::launch_status();
}

namespace {

template <bool TA, bool TB>
int launch_stream(const FsGemmProblem* d_problems, int64_t n_problems, const FsGemmTile* d_tiles,
                  int64_t n_tiles, cudaStream_t s) {
    const int cfg = fsb::configure_smem(
        reinterpret_cast<const void*>(fsb::k_grouped_dgemm_stream<TA, TB>),
        static_cast<int>(fsb::kGemmSmem));
    if (cfg != FS_OK) return cfg;
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 3;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    fsb::k_grouped_dgemm_stream<TA, TB><<<grid, fsb::kGemmThreads, fsb::kGemmSmem, s>>>(
        d_problems, n_problems, d_tiles, n_tiles);
    return fsb::launch_status();
}

}  // namespace

extern "C" int fs_grouped_dgemm_uniform(const FsGemmProblem* d_problems, int64_t n_problems,
                                        const FsGemmTile* d_tiles, int64_t n_tiles,
                                        int32_t trans_a, int32_t trans_b, void* stream) {
    if (n_tiles < 0 || n_problems < 0) return FS_ERR_INVALID_ARG;
    if (n_tiles == 0) return FS_OK;
    if (d_problems == nullptr || d_tiles == nullptr) return FS_ERR_INVALID_ARG;
    cudaStream_t s = fsb::as_stream(stream);
    if (trans_a)
        return trans_b ? launch_stream<true, true>(d_problems, n_problems, d_tiles, n_tiles, s)
                       : launch_stream<true, false>(d_problems, n_problems, d_tiles, n_tiles, s);
    return trans_b ? launch_stream<false, true>(d_problems, n_problems, d_tiles, n_tiles, s)
                   : launch_stream<false, false>(d_problems, n_problems, d_tiles, n_tiles, s);
}

// ---------------------------------------------------------------- thin GEMMs
// C[MxN] = alpha A[MxK] B[KxN] + beta C for M, K <= 32 and N large: the
// recoupling products of a non-abelian permute (one small isometry applied to
// many external-degeneracy columns).  Bandwidth bound: each thread owns output
// columns, A is staged once per tile in shared memory and read as broadcasts,
// the accumulators live in registers (M rounded up to 4, 8, 16 or 32).  Both
// operands row-major (transA == transB == 0; the host checks).
namespace fsb {

constexpr int kThinMax = 32;
constexpr int kThinThreads = 128;
constexpr int kThinColsPerThread = 4;

// MB, KB: M and K rounded up to 4, 8, 16 or 32; NC: columns a thread carries
// at once (KB * NC <= 32 doubles of operands in registers).  Every load of a
// pass (KB per column, predicated on k < K) is issued before its FMAs, so each
// thread keeps up to 32 loads in flight: with the k loop rolled, one load per
// column at a time left the kernel latency bound at a third of the HBM
// bandwidth.
template <int MB, int KB, int NC>
__device__ __forceinline__ void thin_tile(const FsGemmProblem& p, const double* su, int n0) {
#pragma unroll
    for (int c0 = 0; c0 < kThinColsPerThread; c0 += NC) {
        int cols[NC];
        bool ok[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            cols[c] = n0 + threadIdx.x + (c0 + c) * kThinThreads;
            ok[c] = cols[c] < p.N;
        }
        double x[KB][NC];
#pragma unroll
        for (int k = 0; k < KB; ++k)
#pragma unroll
            for (int c = 0; c < NC; ++c)
                x[k][c] = (ok[c] && k < p.K)
                              ? __ldg(p.B + static_cast<int64_t>(k) * p.ldb + cols[c])
                              : 0.0;
#pragma unroll
        for (int m = 0; m < MB; ++m) {
            if (m >= p.M) break;
            double acc[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) acc[c] = 0.0;
#pragma unroll
            for (int k = 0; k < KB; ++k) {
                // su holds zeros for k >= K (the staging pads the rows)
                const double u = su[m * kThinMax + k];
#pragma unroll
                for (int c = 0; c < NC; ++c) acc[c] = fma(u, x[k][c], acc[c]);
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (!ok[c]) continue;
                double* dst = p.C + static_cast<int64_t>(m) * p.ldc + cols[c];
                const double v = p.alpha * acc[c];
                *dst = (p.beta == 0.0) ? v : fma(p.beta, *dst, v);
            }
        }
    }
}

template <int MB>
__device__ __forceinline__ void thin_tile_k(const FsGemmProblem& p, const double* su, int n0) {
    if (p.K <= 4)
        thin_tile<MB, 4, 4>(p, su, n0);
    else if (p.K <= 8)
        thin_tile<MB, 8, 4>(p, su, n0);
    else if (p.K <= 16)
        thin_tile<MB, 16, 2>(p, su, n0);
    else
        thin_tile<MB, 32, 1>(p, su, n0);
}

__global__ void __launch_bounds__(kThinThreads, 4)
    k_grouped_dgemm_thin(const FsGemmProblem* __restrict__ problems, int64_t n_problems,
                         const FsGemmTile* __restrict__ tiles, int64_t n_tiles) {
    __shared__ double su[kThinMax * kThinMax];
    constexpr int kCols = kThinThreads * kThinColsPerThread;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const FsGemmTile tile = tiles[t];
        if (tile.problem < 0 || tile.problem >= n_problems) continue;
        const FsGemmProblem p = problems[tile.problem];
        if (p.M > kThinMax || p.K > kThinMax || p.transA || p.transB) continue;
        const int n0 = tile.tn * kCols;
        if (n0 >= p.N) continue;
        __syncthreads();  // previous tile's reads of su are done
        // rows m < M of U, zero-padded to kThinMax columns (the unrolled k
        // loop reads up to K rounded up)
        const int mk = p.M * kThinMax;
        for (int i = threadIdx.x; i < mk; i += kThinThreads) {
            const int m = i / kThinMax, k = i - m * kThinMax;
            su[i] = (k < p.K) ? p.A[static_cast<int64_t>(m) * p.lda + k] : 0.0;
        }
        __syncthreads();
        if (p.M <= 4)
            thin_tile_k<4>(p, su, n0);
        else if (p.M <= 8)
            thin_tile_k<8>(p, su, n0);
        else if (p.M <= 16)
            thin_tile_k<16>(p, su, n0);
        else
            thin_tile_k<32>(p, su, n0);
    }
}

}  // namespace fsb

extern "C" int fs_thin_dgemm_shape(int32_t* max_m, int32_t* max_k, int32_t* tile_n) {
    if (max_m == nullptr || max_k == nullptr || tile_n == nullptr) return FS_ERR_INVALID_ARG;
    *max_m = fsb::kThinMax;
    *max_k = fsb::kThinMax;
    *tile_n = fsb::kThinThreads * fsb::kThinColsPerThread;
    return FS_OK;
}

extern "C" int fs_grouped_dgemm_thin(const FsGemmProblem* d_problems, int64_t n_problems,
                                     const FsGemmTile* d_tiles, int64_t n_tiles, void* stream) {
    if (n_tiles < 0 || n_problems < 0) return FS_ERR_INVALID_ARG;
    if (n_tiles == 0) return FS_OK;
    if (d_problems == nullptr || d_tiles == nullptr) return FS_ERR_INVALID_ARG;
    const int64_t max_grid = static_cast<int64_t>(fsb::num_sms()) * 8;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    fsb::k_grouped_dgemm_thin<<<grid, fsb::kThinThreads, 0, fsb::as_stream(stream)>>>(
        d_problems, n_problems, d_tiles, n_tiles);
    return fsb::launch_status();
}

// ------------------------------------------------------------ split-K reduce
// When a contraction has too few output tiles to fill the GPU, the host cuts
// long-K sector problems into K chunks whose partial products go to a
// workspace (slice j of an item at W + j * slice); this kernel sums the slices
// in order (deterministic, no atomics) and applies alpha / beta into C.
namespace fsb {

__global__ void __launch_bounds__(256)
    k_splitk_reduce(const FsSplitReduce* __restrict__ items, int64_t n_items) {
    const int64_t it = blockIdx.y;
    if (it >= n_items) return;
    const FsSplitReduce r = items[it];
    const int64_t n = static_cast<int64_t>(r.M) * r.N;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double v = 0.0;
        for (int j = 0; j < r.nslices; ++j) v += __ldg(r.W + j * r.slice + e);
        const int64_t i = e / r.N, c = e - i * r.N;
        double* dst = r.C + i * r.ldc + c;
        *dst = (r.beta == 0.0) ? r.alpha * v : fma(r.beta, *dst, r.alpha * v);
    }
}

}  // namespace fsb

extern "C" int fs_splitk_reduce(const FsSplitReduce* d_items, int64_t n_items,
                                int64_t max_elems, void* stream) {
    if (n_items < 0 || max_elems < 0) return FS_ERR_INVALID_ARG;
    if (n_items == 0 || max_elems == 0) return FS_OK;
    if (d_items == nullptr) return FS_ERR_INVALID_ARG;
    if (n_items > 65535) return FS_ERR_TOO_LARGE;
    const int64_t blocks = (max_elems + 255) / 256;
    const int gx = static_cast<int>(blocks < 4 * fsb::num_sms() ? blocks : 4 * fsb::num_sms());
    fsb::k_splitk_reduce<<<dim3(gx, static_cast<unsigned>(n_items)), 256, 0,
                           fsb::as_stream(stream)>>>(d_items, n_items);
    return fsb::launch_status();
}

// Tile table from runs (see FsTileRun): one thread per tile, binary search of
// its run over the sorted run starts.
namespace fsb {

__global__ void __launch_bounds__(256)
    k_expand_tiles(const FsTileRun* __restrict__ runs, int64_t n_runs, int64_t total,
                   FsGemmTile* __restrict__ tiles) {
    for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t lo = 0, hi = n_runs - 1;   // last run with start <= t
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (__ldg(&runs[mid].start) <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        const FsTileRun r = runs[lo];
        const int64_t k = t - r.start;
        if (r.col_major) {
            const int32_t nr = r.nrow > 0 ? r.nrow : 1;
            tiles[t] = FsGemmTile{r.problem, static_cast<int32_t>(k % nr),
                                  static_cast<int32_t>(k / nr), 0};
        } else {
            const int32_t nc = r.ncol > 0 ? r.ncol : 1;
            tiles[t] = FsGemmTile{r.problem, static_cast<int32_t>(k / nc),
                                  static_cast<int32_t>(k % nc), 0};
        }
    }
}

}  // namespace fsb

extern "C" int fs_expand_tiles(const FsTileRun* d_runs, int64_t n_runs, int64_t total,
                               FsGemmTile* d_tiles, void* stream) {
    if (n_runs < 0 || total < 0) return FS_ERR_INVALID_ARG;
    if (total == 0) return FS_OK;
    if (n_runs == 0 || d_runs == nullptr || d_tiles == nullptr) return FS_ERR_INVALID_ARG;
    const int64_t blocks = (total + 255) / 256;
    const int grid = static_cast<int>(blocks < 8 * fsb::num_sms() ? blocks : 8 * fsb::num_sms());
    fsb::k_expand_tiles<<<grid, 256, 0, fsb::as_stream(stream)>>>(d_runs, n_runs, total,
                                                                  d_tiles);
    return fsb::launch_status();
}
