// Grouped GEMM on the 5th-generation tensor cores (sm_100a, tcgen05) with
// FP64-class accuracy: the Ozaki error-free splitting (Ozaki, Ogita, Oishi,
// Rump, "Error-free transformations of matrix multiplication by using fast
// routines of matrix multiplication", Numer. Algorithms 59, 2012), in the
// integer form of Uchino, Ozaki and Imamura (2024): every row of A and every
// column of B is scaled by a power of two into (-1, 1) and cut into S signed
// 7-bit digits (int8 slices).  Products of slices are exact in int32, so
//
//   C = alpha * sum_{d=0}^{S-1} 2^(ea_i + eb_j - 7(d+2)) sum_{s+t=d} A_s B_t + beta * C
//
// is exact except for the dropped digits beyond S (relative error ~ 2^-7S of
// the row/column maxima).  Each diagonal d is one int32 accumulation in TMEM
// (tcgen05.mma kind::i8, M=128, N=256, K=32 per instruction), converted to
// FP64 and added into C by the epilogue warps while the next diagonal
// accumulates in the second TMEM buffer.
//
// The split kernels write the slices already in the 128-byte-swizzled K-major
// tile layout the UMMA shared-memory descriptors expect, so every pipeline
// stage is filled by two contiguous bulk copies (cp.async.bulk, the TMA unit)
// without tensor maps.  All device waits are bounded: on timeout the kernel
// raises FS_ERR_TIMEOUT in the caller's flag, drains its copies, frees TMEM
// and returns.
#include <cuda.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"

namespace fsb {
namespace oz {

constexpr int kTileM = 128;       // rows of A per tile (UMMA M)
constexpr int kTileN = 256;       // rows of B^T per tile (UMMA N)
constexpr int kTileK = 128;       // int8 elements (bytes) per k-step = one swizzle atom
constexpr int kStages = 4;
constexpr int kABytes = kTileM * kTileK;            // 16 KB
constexpr int kBBytes = kTileN * kTileK;            // 32 KB
constexpr int kStageBytes = kABytes + kBBytes;      // 48 KB
constexpr int kThreads = 192;                       // 6 warps
constexpr int kTmemCols = 512;                      // two 256-column accumulators
constexpr int kSplitRows = 128;                     // rows per slice tile
// bound of the waits that drain in-flight copies and MMAs on the way out
// (~1 s of clock64 at 1.9 GHz); the abortable waits use the runtime bound
// passed to each kernel (fs_set_spin_limit)
constexpr long long kDrainLimit = 2000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false on timeout or when another role already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          volatile int* abort_flag, long long limit) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > limit) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

// Time-bounded wait that ignores the abort flag (used to drain in-flight work).
__device__ __forceinline__ bool mbar_wait_drain(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > kDrainLimit) return false;
    }
    return true;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// K-major operand, 128-byte swizzle, 8-row core groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr & 0x3FFFF) >> 4);        // start address
    d |= static_cast<uint64_t>(1) << 16;                      // leading byte offset (unused)
    d |= static_cast<uint64_t>(1024 >> 4) << 32;              // stride byte offset
    d |= static_cast<uint64_t>(1) << 46;                      // descriptor version (sm_100)
    d |= static_cast<uint64_t>(2) << 61;                      // SWIZZLE_128B
    return d;
}

// kind::i8 instruction descriptor: S32 accumulate, signed A and B, K-major both.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) |
                            (static_cast<uint32_t>(kTileN >> 3) << 17) |
                            (static_cast<uint32_t>(kTileM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            bar)
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
          "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
          "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// --------------------------------------------------------------- split kernels

// exps[v] = e with max_k |x(v, k)| < 2^e (frexp exponent; 0 for a zero vector).
// One warp per vector.
__global__ void __launch_bounds__(256)
    k_oz_exponents(const FsOzOperand* __restrict__ ops, int64_t n_ops) {
    const int op_id = blockIdx.y;
    if (op_id >= n_ops) return;
    const FsOzOperand op = ops[op_id];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * 8 + warp; v < op.rows;
         v += static_cast<int64_t>(gridDim.x) * 8) {
        double m = 0.0;
        for (int64_t k = lane; k < op.K; k += 32)
            m = fmax(m, fabs(__ldg(op.src + v * op.s_row + k * op.s_k)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) {
            int e = 0;
            if (m > 0.0) frexp(m, &e);
            op.exps[v] = e;
        }
    }
}

// Writes the S digit slices of one operand in swizzled tile layout:
// tile (s, kt, rt) of 128 rows x 128 bytes at ((s * ktiles + kt) * rowtiles + rt) * 16 KB,
// row r at r * 128 bytes, 16-byte chunk c stored at chunk (c ^ (r & 7)).
__global__ void __launch_bounds__(1024)
    k_oz_split(const FsOzOperand* __restrict__ ops, int64_t n_ops, int nslices) {
    const int op_id = blockIdx.y;
    if (op_id >= n_ops) return;
    const FsOzOperand op = ops[op_id];
    const int r = threadIdx.x / 8;      // row in tile
    const int c = threadIdx.x % 8;      // 16-byte chunk (16 k values)
    const int64_t ntiles = static_cast<int64_t>(op.rowtiles) * op.ktiles;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int kt = static_cast<int>(tile / op.rowtiles);
        const int rt = static_cast<int>(tile % op.rowtiles);
        const int64_t row = static_cast<int64_t>(rt) * kSplitRows + r;
        const int64_t k0 = static_cast<int64_t>(kt) * kTileK + c * 16;
        const int e = (row < op.rows) ? op.exps[row] : 0;
        double x[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int64_t k = k0 + j;
            x[j] = (row < op.rows && k < op.K)
                       ? ldexp(__ldg(op.src + row * op.s_row + k * op.s_k), -e)
                       : 0.0;
        }
        const int64_t slice_stride = static_cast<int64_t>(op.ktiles) * op.rowtiles * kABytes;
        int8_t* dst = op.slices + (static_cast<int64_t>(kt) * op.rowtiles + rt) * kABytes +
                      r * 128 + ((c ^ (r & 7)) * 16);
        for (int s = 0; s < nslices; ++s) {
            uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const double t = x[j] * 128.0;
                const double dgt = trunc(t);
                x[j] = t - dgt;
                const uint32_t byte = static_cast<uint32_t>(static_cast<int32_t>(dgt)) & 0xFFu;
                w[j / 4] |= byte << (8 * (j % 4));
            }
            *reinterpret_cast<uint4*>(dst + s * slice_stride) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// ------------------------------------------------------------------ GEMM kernel

struct __align__(8) Barriers {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t acc_full[2];
    uint64_t acc_empty[2];
    uint64_t mma_drain;
    uint32_t tmem_base;
    int abort_flag;
};

// Iteration order shared by the producer and the MMA issuer: for every tile of
// this CTA, for every diagonal d (S-1 down to 0), for every K chunk, for every
// slice pair (s, d - s), for every k-tile of the chunk.
struct PassIter {
    int nslices, ktiles, chunk;
};

__global__ void __launch_bounds__(kThreads, 1)
    k_oz_gemm(const FsOzProblem* __restrict__ probs, int64_t n_probs,
              const FsOzTile* __restrict__ tiles, int64_t n_tiles, int nslices,
              int chunk_ktiles, int32_t* flag, long long spin) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* smem = smem_raw + (base - raw);
    Barriers* bars = reinterpret_cast<Barriers*>(smem + kStages * kStageBytes);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_addr(&bars->full[s]), 1);
            mbar_init(smem_addr(&bars->empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_addr(&bars->acc_full[b]), 1);
            mbar_init(smem_addr(&bars->acc_empty[b]), 4);
        }
        mbar_init(smem_addr(&bars->mma_drain), 1);
        bars->abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&bars->tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;
    volatile int* abort_flag = &bars->abort_flag;

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            uint32_t issued_mask = 0;          // stages with a copy issued
            uint32_t issued_parity = 0;        // full-barrier parity of that copy
            for (int64_t t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
                const FsOzTile tile = tiles[t];
                const FsOzProblem p = probs[tile.problem];
                const int64_t a_slice = static_cast<int64_t>(p.ktiles) * p.a_rowtiles * kABytes;
                const int64_t b_slice = static_cast<int64_t>(p.ktiles) * p.b_rowtiles * kABytes;
                for (int d = nslices - 1; ok && d >= 0; --d) {
                    for (int k0 = 0; ok && k0 < p.ktiles; k0 += chunk_ktiles) {
                        const int k1 = min(p.ktiles, k0 + chunk_ktiles);
                        for (int s = 0; ok && s <= d; ++s) {
                            const int tt = d - s;
                            for (int kt = k0; kt < k1; ++kt) {
                                if (!mbar_wait(smem_addr(&bars->empty[stage]), phase ^ 1,
                                               abort_flag, spin)) {
                                    ok = false;
                                    break;
                                }
                                const uint32_t full = smem_addr(&bars->full[stage]);
                                mbar_expect_tx(full, kStageBytes);
                                const int8_t* a = p.a_slices + s * a_slice +
                                                  (static_cast<int64_t>(kt) * p.a_rowtiles + tile.tm) * kABytes;
                                const int8_t* b = p.b_slices + tt * b_slice +
                                                  (static_cast<int64_t>(kt) * p.b_rowtiles + 2 * tile.tn) * kABytes;
                                const uint32_t dst = base + stage * kStageBytes;
                                bulk_g2s(dst, a, kABytes, full);
                                bulk_g2s(dst + kABytes, b, kBBytes, full);
                                issued_mask |= 1u << stage;
                                issued_parity = (issued_parity & ~(1u << stage)) | (phase << stage);
                                if (++stage == kStages) {
                                    stage = 0;
                                    phase ^= 1;
                                }
                            }
                        }
                    }
                }
            }
            // drain: every issued copy must have landed before the CTA exits
            for (int s = 0; s < kStages; ++s) {
                if (issued_mask & (1u << s)) {
                    if (!mbar_wait_drain(smem_addr(&bars->full[s]), (issued_parity >> s) & 1u))
                        *abort_flag = 1;
                }
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
                const FsOzTile tile = tiles[t];
                const FsOzProblem p = probs[tile.problem];
                for (int d = nslices - 1; ok && d >= 0; --d) {
                    for (int k0 = 0; ok && k0 < p.ktiles; k0 += chunk_ktiles) {
                        const int k1 = min(p.ktiles, k0 + chunk_ktiles);
                        if (!mbar_wait(smem_addr(&bars->acc_empty[acc]), acc_phase ^ 1,
                                       abort_flag, spin)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t tmem_d = tmem_base + acc * kTileN;
                        uint32_t accumulate = 0;
                        for (int s = 0; ok && s <= d; ++s) {
                            for (int kt = k0; kt < k1; ++kt) {
                                if (!mbar_wait(smem_addr(&bars->full[stage]), phase, abort_flag, spin)) {
                                    ok = false;
                                    break;
                                }
                                tc_fence_after();
                                const uint32_t a_addr = base + stage * kStageBytes;
                                const uint32_t b_addr = a_addr + kABytes;
#pragma unroll
                                for (int k = 0; k < kTileK / 32; ++k) {
                                    mma_i8(tmem_d, smem_desc_sw128(a_addr + 32 * k),
                                           smem_desc_sw128(b_addr + 32 * k), accumulate);
                                    accumulate = 1;
                                }
                                mma_commit(smem_addr(&bars->empty[stage]));
                                if (++stage == kStages) {
                                    stage = 0;
                                    phase ^= 1;
                                }
                            }
                        }
                        if (!ok) break;
                        mma_commit(smem_addr(&bars->acc_full[acc]));
                        if (++acc == 2) {
                            acc = 0;
                            acc_phase ^= 1;
                        }
                    }
                }
            }
            // drain: all issued MMAs complete before TMEM is released
            mma_commit(smem_addr(&bars->mma_drain));
            if (!mbar_wait_drain(smem_addr(&bars->mma_drain), 0)) *abort_flag = 1;
        }
    } else {
        // ---------------------------------------------------------- epilogue
        const int quad = warp % 4;           // TMEM lane quadrant this warp may read
        const int row_in_tile = quad * 32 + lane;
        int acc = 0;
        uint32_t acc_phase = 0;
        bool ok = true;
        for (int64_t t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
            const FsOzTile tile = tiles[t];
            const FsOzProblem p = probs[tile.problem];
            const int64_t row = static_cast<int64_t>(tile.tm) * kTileM + row_in_tile;
            const int col0 = tile.tn * kTileN;
            const bool row_ok = row < p.M;
            const int ea = row_ok ? p.a_exps[row] : 0;
            bool first = true;
            for (int d = nslices - 1; ok && d >= 0; --d) {
                for (int k0 = 0; ok && k0 < p.ktiles; k0 += chunk_ktiles) {
                    // one lane waits, the warp follows its verdict, so the
                    // warp-wide tcgen05.ld below is never reached by a subset
                    int got = 0;
                    if (lane == 0)
                        got = mbar_wait(smem_addr(&bars->acc_full[acc]), acc_phase, abort_flag, spin)
                                  ? 1
                                  : 0;
                    got = __shfl_sync(0xffffffffu, got, 0);
                    if (!got) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) +
                                           acc * kTileN;
                    const int shift = -7 * (d + 2);
                    // C is read only when it contributes (later diagonals, or
                    // beta != 0), and the 16 reads of a chunk are issued before
                    // any store so that they overlap instead of each waiting a
                    // full memory latency behind the previous store
                    const bool read_c = !first || p.beta != 0.0;
                    for (int cb = 0; cb < kTileN; cb += 16) {
                        uint32_t v[16];
                        tmem_ld16(taddr + cb, v);
                        if (!row_ok || col0 + cb >= p.N) continue;
                        double* crow = p.C + row * p.ldc + col0 + cb;
                        const int32_t* be = p.b_exps + col0 + cb;
                        const int ncol = min(16, p.N - col0 - cb);
                        double old[16];
                        int eb[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            eb[j] = (j < ncol) ? __ldg(be + j) : 0;
                            old[j] = (read_c && j < ncol) ? crow[j] : 0.0;
                        }
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const double val =
                                p.alpha * ldexp(static_cast<double>(static_cast<int32_t>(v[j])),
                                                ea + eb[j] + shift);
                            old[j] = first ? ((p.beta == 0.0) ? val : fma(p.beta, old[j], val))
                                           : old[j] + val;
                        }
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (j < ncol) crow[j] = old[j];
                    }
                    first = false;
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_addr(&bars->acc_empty[acc]));
                    if (++acc == 2) {
                        acc = 0;
                        acc_phase ^= 1;
                    }
                }
            }
        }
    }

    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) raise_flag(flag, FS_ERR_TIMEOUT);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

// ------------------------------------------------------- CTA-pair GEMM kernel
//
// 256 x 256 output tiles computed by a cluster of two CTAs with
// tcgen05.mma.cta_group::2 (M = 256, N = 256).  CTA r of the pair loads its
// own 128 rows of the A slice tile (row tile 2 tm + r) and its own 128 rows of
// the B^T slice tile (row tile 2 tn + r) into its own shared memory: half the
// bytes per SM of the single-CTA kernel for the same MMA work.  The even CTA
// issues the MMAs, which read A from each CTA and B from both, and accumulate
// rows [128 r, 128 r + 128) of the tile in CTA r's TMEM.
//
// One kernel body serves both arithmetics (template kCRT):
//   digits (Ozaki I): accumulator groups are (diagonal d, K chunk), each the
//     sum over the slice pairs (s, d - s); the epilogue adds
//     2^(ea + eb - 7(d+2)) * acc into C in FP64;
//   moduli (Ozaki II): one accumulator group per modulus p_m, the product of
//     the residue slices m of A and B over all of K; the epilogue reduces it
//     to the symmetric residue mod p_m and parks it (one byte per entry) in a
//     per-CTA scratch; after the last modulus the CRT reconstruction turns the
//     residues into FP64 and writes C.
//
// Operand tiles are fetched by TMA through a 2-D tensor map that views the
// slice workspace as rows of 128 bytes (box 128 x 128, no swizzle: the split
// kernels already wrote the swizzled layout).  The loads carry .cta_group::2,
// so both CTAs' copies complete on the even CTA's barrier.  Handshakes (all
// waits bounded):
//   full[s]      even CTA: both CTAs' 2 x 32 KB of stage s landed (the even
//                CTA arrives once with the expected byte count);
//   empty[s]     both CTAs: the MMAs reading stage s finished (the even CTA's
//                commit arrives on both CTAs' barriers);
//   acc_full[b]  both CTAs: accumulator b holds a finished group;
//   acc_empty[b] even CTA: the 8 epilogue warps of the pair drained buffer b
//                (4 local arrivals, 4 remote ones from the odd CTA).
// Teardown: the odd CTA publishes how many stage loads it issued; after a
// cluster barrier the even CTA's producer waits for the last load of every
// stage (both CTAs' copies land on its barriers), first settling the byte
// count of a stage that only one CTA loaded because the other one aborted
// (mbarrier.complete_tx for a missing half, an arrive with the expected bytes
// for a stage the even CTA never armed).  A second cluster barrier then keeps
// both CTAs (their shared memory and TMEM) alive until no copy or MMA can
// touch them.  No load uses multicast.

constexpr int kPairStages = 6;
constexpr int kPairStageBytes = 2 * kABytes;                // 16 KB A half + 16 KB B half
constexpr uint32_t kIdescPair = (2u << 4) | (1u << 7) | (1u << 10) |
                                (static_cast<uint32_t>(kTileN >> 3) << 17) |
                                (static_cast<uint32_t>(256 >> 4) << 24);
// CRT scratch per CTA and modulus: 16 column chunks x 128 rows x 16 bytes
constexpr int kCrtChunkBytes = 16 * 128;
constexpr int kCrtModulusBytes = (kTileN / 16) * kCrtChunkBytes;   // 32 KB

struct __align__(8) PairBarriers {
    uint64_t full[kPairStages];
    uint64_t empty[kPairStages];
    uint64_t acc_full[2];
    uint64_t acc_empty[2];
    uint64_t mma_drain;
    uint32_t tmem_base;
    int abort_flag;
    uint32_t odd_items;   // stage loads issued by the odd CTA (written remotely)
};

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the same shared variable in CTA `rank`
__device__ __forceinline__ uint32_t map_to_rank(uint32_t addr, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
    return out;
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(
                     cluster_addr)
                 : "memory");
}

__device__ __forceinline__ void mbar_complete_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void st_cluster_u32(uint32_t cluster_addr, uint32_t v) {
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(cluster_addr), "r"(v) : "memory");
}

// TMA load of one 128-row x 128-byte tile (rows y .. y+127 of the workspace
// view) into this CTA's shared memory, completing on the barrier at the
// shared::cluster address `bar` (the even CTA's)
__device__ __forceinline__ void tma_tile_pair(uint32_t dst, const CUtensorMap* map, int32_t y,
                                              uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdescPair), "r"(accumulate)
        : "memory");
}

// commit of the pair's MMAs to this CTA's barrier at `bar`
__device__ __forceinline__ void mma_commit_pair_local(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

// commit of the pair's MMAs arriving on the barrier at this shared offset in
// both CTAs of the pair (commit multicast; no load is multicast)
__device__ __forceinline__ void mma_commit_pair(uint32_t bar) {
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
        "[%0], %1;" ::"r"(bar),
        "h"(mask)
        : "memory");
}

// One accumulator group: the slice pairs (sa + i, sb - i), i < npairs, over
// k-tiles [k0, k1).
struct Group {
    int sa, sb, npairs, k0, k1, d;
};

template <bool kCRT>
__device__ __forceinline__ int n_groups(int ktiles, int nsl, int chunk) {
    return kCRT ? nsl : nsl * ((ktiles + chunk - 1) / chunk);
}

// digits: groups run over diagonals d = S-1 .. 0 and, inside, over K chunks;
// moduli: group m is modulus m over all of K
template <bool kCRT>
__device__ __forceinline__ Group group_at(int g, int ktiles, int nsl, int chunk) {
    Group r;
    if (kCRT) {
        r.sa = g;
        r.sb = g;
        r.npairs = 1;
        r.k0 = 0;
        r.k1 = ktiles;
        r.d = g;
    } else {
        const int nch = (ktiles + chunk - 1) / chunk;
        r.d = nsl - 1 - g / nch;
        r.sa = 0;
        r.sb = r.d;
        r.npairs = r.d + 1;
        r.k0 = (g % nch) * chunk;
        r.k1 = min(ktiles, r.k0 + chunk);
    }
    return r;
}

// 2^k as a double for -1022 <= k <= 1023
__device__ __forceinline__ double pow2i(int k) {
    return __hiloint2double((k + 1023) << 20, 0);
}

// x * 2^k, exact unless the result leaves the normal range (then rounded once,
// like ldexp)
__device__ __forceinline__ double scale2(double x, int k) {
    return (k >= -1022 && k <= 1023) ? x * pow2i(k) : ldexp(x, k);
}

// the exact double value of a 32-bit signed integer, without the conversion
// unit: 1.5 * 2^52 + 2^31 + v, minus the constant
__device__ __forceinline__ double int_to_double(int32_t v) {
    return __hiloint2double(0x43380000, v ^ static_cast<int32_t>(0x80000000)) -
           6755401588539392.0;
}

constexpr double kRoundMagic = 6755399441055744.0;   // 1.5 * 2^52: x + M rounds x to an integer

// symmetric residue r of the int32 accumulator acc modulo the odd modulus p,
// parked as the byte r + 128: the low byte of acc - p * rint(acc / p) + 128
// (the quotient is exact: |acc/p| < 2^24 and acc/p is at least 1/(2p) away
// from any half integer)
__device__ __forceinline__ uint32_t residue_byte(int32_t acc, int32_t p, double inv_p) {
    const int32_t q = __double2loint(fma(int_to_double(acc), inv_p, kRoundMagic));
    return static_cast<uint32_t>(acc - q * p + 128) & 0xFFu;
}

// the exact double value of a byte u (0..255) without the conversion unit
__device__ __forceinline__ double byte_to_double(uint32_t u) {
    return __hiloint2double(0x43380000, static_cast<int>(u)) - kRoundMagic;
}

// CRT constants of one modulus count (host computed, passed by value): the
// moduli, 1/p_m rounded, y_m / p_m (y_m = (P/p_m)^-1 mod p_m) as FP32, the CRT
// weights W_m = (P/p_m) y_m split as w1_m + w2_m + (dropped) on the grids 2^e1
// and 2^e2, P split the same way, the offsets that undo the +128 of the parked
// residue bytes, and 1/P.
struct CrtConsts {
    int32_t n, e1, e2, pad;
    int32_t p[FS_OZAKI2_MAX_MODULI];
    float f[FS_OZAKI2_MAX_MODULI];
    double inv_p[FS_OZAKI2_MAX_MODULI];
    double w1[FS_OZAKI2_MAX_MODULI];
    double w2[FS_OZAKI2_MAX_MODULI];
    double p1, p2;
    double c1, c2;      // -128 sum_m w1_m and -128 sum_m w2_m (the byte offsets)
    double inv_P;       // 1 / P rounded
};

// ------------------------------------------------ Ozaki II (CRT over moduli)
//
// The integer-modular form of the Ozaki scheme (Ozaki, Uchino, Imamura,
// "Ozaki Scheme II: a GEMM-oriented emulation of floating-point matrix
// multiplication using an integer modular technique", 2025): every row i of
// op(A) is scaled by 2^(a - e_i) (e_i the frexp exponent of the row maximum)
// and rounded to an integer A'_ik with |A'_ik| <= 2^a; likewise the columns of
// op(B) with b bits.  The exact integer product X = A' B' satisfies
// |X| <= K 2^(a+b) <= P / 4 for P = p_0 ... p_(n-1), the product of n pairwise
// coprime moduli <= 256, so X is recovered from its residues X mod p_m.  Each
// residue product is one int8 GEMM of the symmetric residues of A' and B'
// (entries in [-128, 127], exact int32 accumulation for K < 2^17).  The CRT
// then gives X = sum_m r_m W_m - k P with W_m = (P/p_m) ((P/p_m)^-1 mod p_m),
// k = rint(sum_m r_m W_m / P), evaluated exactly in FP64 by splitting every
// W_m (and P) into two doubles on fixed binary grids 2^E1 and 2^E2 so that
// every product and partial sum is representable; the dropped remainder is
// below 2^(E2 + 12), far under the rounding of A and B.  C = alpha X 2^(e_i +
// f_j - a - b) + beta C.  One int8 product per modulus replaces the
// S(S+1)/2 digit-slice products of the Ozaki I form.

constexpr int kCrtMaxModuli = FS_OZAKI2_MAX_MODULI;

// the moduli, largest first; pairwise coprime (256 = 2^8, 255 = 3*5*17,
// 253 = 11*23, 247 = 13*19, 217 = 7*31, the rest prime)
constexpr int32_t kModuli[kCrtMaxModuli] = {256, 255, 253, 251, 247, 241, 239,
                                            233, 229, 227, 223, 217, 211, 199};

template <class Prob>
__device__ __forceinline__ void crt_store_row(const Prob& p, const CrtConsts& cc,
                                              const uint8_t* scratch, int64_t row, int col0,
                                              int ea) {
    const int n = cc.n;
    double* crow = p.C + row * p.ldc + col0;
    const int sa = ea - p.a_bits - p.b_bits;
    const int ncols = min(kTileN, p.N - col0);
    for (int cb = 0; cb < ncols; cb += 16) {
        // every load of the chunk first (parked residues, column exponents,
        // and C when beta != 0), so that their latencies overlap
        uint32_t w[kCrtMaxModuli][4];
#pragma unroll
        for (int m = 0; m < kCrtMaxModuli; ++m) {
            if (m < n) {
                const uint4 q = *reinterpret_cast<const uint4*>(
                    scratch + m * kCrtModulusBytes + (cb / 16) * kCrtChunkBytes);
                w[m][0] = q.x;
                w[m][1] = q.y;
                w[m][2] = q.z;
                w[m][3] = q.w;
            }
        }
        const int ncol = min(16, ncols - cb);
        const int32_t* be = p.b_exps + col0 + cb;
        int eb[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) eb[j] = (j < ncol) ? __ldg(be + j) : 0;
        double old[16];
        if (p.beta != 0.0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) old[j] = (j < ncol) ? crow[cb + j] : 0.0;
        }
        double val[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            // the residues arrive as bytes u_m = r_m + 128; the constant terms
            // c1, c2 remove the offsets.  d1 = sum_m r_m w1_m and d2 = sum_m
            // r_m w2_m are exact on their grids; d1 / P is within 2^-29 of
            // S / P = k + X / P with |X / P| <= 1/4, which gives k, and then
            // X = (d1 - k p1) + (d2 - k p2)
            double d1 = cc.c1;
            double d2 = cc.c2;
#pragma unroll
            for (int m = 0; m < kCrtMaxModuli; ++m) {
                if (m < n) {
                    const double u = byte_to_double((w[m][j / 4] >> (8 * (j % 4))) & 0xFFu);
                    d1 = fma(u, cc.w1[m], d1);
                    d2 = fma(u, cc.w2[m], d2);
                }
            }
            const double kd = fma(d1, cc.inv_P, kRoundMagic) - kRoundMagic;
            d1 = fma(-kd, cc.p1, d1);
            d2 = fma(-kd, cc.p2, d2);
            val[j] = p.alpha * scale2(d1 + d2, sa + eb[j]);
        }
        if (p.beta != 0.0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) val[j] = fma(p.beta, old[j], val[j]);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (j < ncol) crow[cb + j] = val[j];
    }
}

template <class Prob, bool kCRT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    k_oz_pair(const Prob* __restrict__ probs, int64_t n_probs, const FsOzTile* __restrict__ tiles,
              int64_t n_tiles, int nslices, int chunk_ktiles, int32_t* flag,
              const __grid_constant__ CUtensorMap ws_map, const int8_t* ws_base, long long spin,
              uint8_t* crt_scratch, const __grid_constant__ CrtConsts cc) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* smem = smem_raw + (base - raw);
    PairBarriers* bars = reinterpret_cast<PairBarriers*>(smem + kPairStages * kPairStageBytes);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t rank = cluster_ctarank();
    const int64_t cluster_id = blockIdx.x / 2;
    const int64_t n_clusters = gridDim.x / 2;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kPairStages; ++s) {
            mbar_init(smem_addr(&bars->full[s]), 1);
            mbar_init(smem_addr(&bars->empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_addr(&bars->acc_full[b]), 1);
            mbar_init(smem_addr(&bars->acc_empty[b]), 8);
        }
        mbar_init(smem_addr(&bars->mma_drain), 1);
        bars->abort_flag = 0;
        bars->odd_items = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&bars->tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        tc_fence_before();
    }
    __syncthreads();
    cluster_sync_all();  // barriers of both CTAs initialised before any remote arrive
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;
    volatile int* abort_flag = &bars->abort_flag;
    uint32_t items = 0;   // stage loads issued by this CTA's producer

    if (warp == 0) {
        // ------------------------------------------ producer (both CTAs)
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            for (int64_t t = cluster_id; ok && t < n_tiles; t += n_clusters) {
                const FsOzTile tile = tiles[t];
                const Prob p = probs[tile.problem];
                if (kCRT && p.K > FS_OZAKI2_MAX_K) continue;
                const int64_t a_slice = static_cast<int64_t>(p.ktiles) * p.a_rowtiles * kABytes;
                const int64_t b_slice = static_cast<int64_t>(p.ktiles) * p.b_rowtiles * kABytes;
                const int a_rt = 2 * tile.tm + static_cast<int>(rank);
                const int b_rt = 2 * tile.tn + static_cast<int>(rank);
                const int ng = n_groups<kCRT>(p.ktiles, nslices, chunk_ktiles);
                for (int g = 0; ok && g < ng; ++g) {
                    const Group gr = group_at<kCRT>(g, p.ktiles, nslices, chunk_ktiles);
                    for (int i = 0; ok && i < gr.npairs; ++i) {
                        const int8_t* a_sl = p.a_slices + (gr.sa + i) * a_slice;
                        const int8_t* b_sl = p.b_slices + (gr.sb - i) * b_slice;
                        for (int kt = gr.k0; kt < gr.k1; ++kt) {
                            if (!mbar_wait(smem_addr(&bars->empty[stage]), phase ^ 1, abort_flag,
                                           spin)) {
                                ok = false;
                                break;
                            }
                            const uint32_t full = smem_addr(&bars->full[stage]);
                            if (rank == 0) mbar_expect_tx(full, 2 * kPairStageBytes);
                            const int8_t* a =
                                a_sl + (static_cast<int64_t>(kt) * p.a_rowtiles + a_rt) * kABytes;
                            const int8_t* b =
                                b_sl + (static_cast<int64_t>(kt) * p.b_rowtiles + b_rt) * kABytes;
                            const uint32_t dst = base + stage * kPairStageBytes;
                            const uint32_t full_even = map_to_rank(full, 0);
                            tma_tile_pair(dst, &ws_map, static_cast<int32_t>((a - ws_base) >> 7),
                                          full_even);
                            tma_tile_pair(dst + kABytes, &ws_map,
                                          static_cast<int32_t>((b - ws_base) >> 7), full_even);
                            ++items;
                            if (++stage == kPairStages) {
                                stage = 0;
                                phase ^= 1;
                            }
                        }
                    }
                }
            }
            if (rank == 1) st_cluster_u32(map_to_rank(smem_addr(&bars->odd_items), 0), items);
        }
    } else if (warp == 1 && rank == 1) {
        // the odd CTA's warp 1 only shares the TMEM allocation
    } else if (warp == 1) {
        // ------------------------------------------ MMA issuer (even CTA)
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool ok = true;
            for (int64_t t = cluster_id; ok && t < n_tiles; t += n_clusters) {
                const Prob p = probs[tiles[t].problem];
                if (kCRT && p.K > FS_OZAKI2_MAX_K) continue;
                const int ng = n_groups<kCRT>(p.ktiles, nslices, chunk_ktiles);
                for (int g = 0; ok && g < ng; ++g) {
                    const Group gr = group_at<kCRT>(g, p.ktiles, nslices, chunk_ktiles);
                    if (!mbar_wait(smem_addr(&bars->acc_empty[acc]), acc_phase ^ 1, abort_flag,
                                   spin)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t tmem_d = tmem_base + acc * kTileN;
                    uint32_t accumulate = 0;
                    for (int i = 0; ok && i < gr.npairs; ++i) {
                        for (int kt = gr.k0; kt < gr.k1; ++kt) {
                            if (!mbar_wait(smem_addr(&bars->full[stage]), phase, abort_flag,
                                           spin)) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const uint32_t a_addr = base + stage * kPairStageBytes;
                            const uint32_t b_addr = a_addr + kABytes;
#pragma unroll
                            for (int k = 0; k < kTileK / 32; ++k) {
                                mma_i8_pair(tmem_d, smem_desc_sw128(a_addr + 32 * k),
                                            smem_desc_sw128(b_addr + 32 * k), accumulate);
                                accumulate = 1;
                            }
                            mma_commit_pair(smem_addr(&bars->empty[stage]));
                            if (++stage == kPairStages) {
                                stage = 0;
                                phase ^= 1;
                            }
                        }
                    }
                    if (!ok) break;
                    mma_commit_pair(smem_addr(&bars->acc_full[acc]));
                    if (++acc == 2) {
                        acc = 0;
                        acc_phase ^= 1;
                    }
                }
            }
            mma_commit_pair_local(smem_addr(&bars->mma_drain));
            if (!mbar_wait_drain(smem_addr(&bars->mma_drain), 0)) *abort_flag = 1;
        }
    } else {
        // ------------------------------------------ epilogue (both CTAs)
        const int quad = warp % 4;
        const int lrow = quad * 32 + lane;                // TMEM lane = row within this CTA
        const int row_in_tile = static_cast<int>(rank) * 128 + lrow;
        const uint32_t acc_empty_leader[2] = {
            map_to_rank(smem_addr(&bars->acc_empty[0]), 0),
            map_to_rank(smem_addr(&bars->acc_empty[1]), 0)};
        uint8_t* my_scratch = nullptr;
        if (kCRT)
            my_scratch = crt_scratch + static_cast<int64_t>(blockIdx.x) * nslices * kCrtModulusBytes +
                         lrow * 16;
        int acc = 0;
        uint32_t acc_phase = 0;
        bool ok = true;
        for (int64_t t = cluster_id; ok && t < n_tiles; t += n_clusters) {
            const FsOzTile tile = tiles[t];
            const Prob p = probs[tile.problem];
            if (kCRT && p.K > FS_OZAKI2_MAX_K) {
                // the int32 residue products could overflow: skipped, reported
                if (threadIdx.x == 64) raise_flag(flag, FS_ERR_UNSUPPORTED);
                continue;
            }
            const int64_t row = static_cast<int64_t>(tile.tm) * 256 + row_in_tile;
            const int col0 = tile.tn * kTileN;
            const bool row_ok = row < p.M;
            const int ea = row_ok ? p.a_exps[row] : 0;
            const int ng = n_groups<kCRT>(p.ktiles, nslices, chunk_ktiles);
            bool first = true;
            for (int g = 0; ok && g < ng; ++g) {
                int got = 0;
                if (lane == 0)
                    got = mbar_wait(smem_addr(&bars->acc_full[acc]), acc_phase, abort_flag, spin)
                              ? 1
                              : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t taddr =
                    tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + acc * kTileN;
                if constexpr (kCRT) {
                    // residues of modulus g, one byte per entry, parked in this
                    // thread's slots of the CTA scratch
                    const int32_t pm = cc.p[g];
                    const double ipm = cc.inv_p[g];
                    uint8_t* dst = my_scratch + static_cast<int64_t>(g) * kCrtModulusBytes;
                    for (int cb = 0; cb < kTileN; cb += 16) {
                        uint32_t v[16];
                        tmem_ld16(taddr + cb, v);
                        uint32_t w[4] = {0, 0, 0, 0};
                        if (g == 0) {
                            // p = 256: the low byte of acc + 128 is the
                            // symmetric residue plus 128
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                w[j / 4] |= ((v[j] + 128u) & 0xFFu) << (8 * (j % 4));
                        } else {
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                w[j / 4] |= residue_byte(static_cast<int32_t>(v[j]), pm, ipm)
                                            << (8 * (j % 4));
                        }
                        *reinterpret_cast<uint4*>(dst + (cb / 16) * kCrtChunkBytes) =
                            make_uint4(w[0], w[1], w[2], w[3]);
                    }
                } else {
                    const int shift = -7 * (group_at<kCRT>(g, p.ktiles, nslices, chunk_ktiles).d + 2);
                    const bool read_c = !first || p.beta != 0.0;
                    for (int cb = 0; cb < kTileN; cb += 16) {
                        uint32_t v[16];
                        tmem_ld16(taddr + cb, v);
                        if (!row_ok || col0 + cb >= p.N) continue;
                        double* crow = p.C + row * p.ldc + col0 + cb;
                        const int32_t* be = p.b_exps + col0 + cb;
                        const int ncol = min(16, p.N - col0 - cb);
                        double old[16];
                        int eb[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            eb[j] = (j < ncol) ? __ldg(be + j) : 0;
                            old[j] = (read_c && j < ncol) ? crow[j] : 0.0;
                        }
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const double val =
                                p.alpha * ldexp(static_cast<double>(static_cast<int32_t>(v[j])),
                                                ea + eb[j] + shift);
                            old[j] = first ? ((p.beta == 0.0) ? val : fma(p.beta, old[j], val))
                                           : old[j] + val;
                        }
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (j < ncol) crow[j] = old[j];
                    }
                }
                first = false;
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    if (rank == 0)
                        mbar_arrive(smem_addr(&bars->acc_empty[acc]));
                    else
                        mbar_arrive_remote(acc_empty_leader[acc]);
                }
                if (++acc == 2) {
                    acc = 0;
                    acc_phase ^= 1;
                }
                if constexpr (kCRT) {
                    if (g == ng - 1 && row_ok) crt_store_row(p, cc, my_scratch, row, col0, ea);
                }
            }
        }
    }

    __syncthreads();
    cluster_sync_all();  // every role done; the odd CTA's load count is visible
    if (rank == 0 && threadIdx.x == 0) {
        // wait for the last load of every stage, settling stages that only one
        // CTA loaded (see the teardown note above)
        const uint32_t n_odd = bars->odd_items;
        const uint32_t n_even = items;
        const uint32_t n_max = n_even > n_odd ? n_even : n_odd;
        const uint32_t first = n_max > static_cast<uint32_t>(kPairStages) ? n_max - kPairStages : 0;
        for (uint32_t i = first; i < n_max; ++i) {
            const uint32_t bar = smem_addr(&bars->full[i % kPairStages]);
            if (i >= n_even)
                mbar_expect_tx(bar, kPairStageBytes);
            else if (i >= n_odd)
                mbar_complete_tx(bar, kPairStageBytes);
            if (!mbar_wait_drain(bar, (i / kPairStages) & 1u)) *abort_flag = 1;
        }
    }
    __syncthreads();
    cluster_sync_all();  // no copy or MMA of the pair can touch either CTA after this
    if (threadIdx.x == 0 && *abort_flag) raise_flag(flag, FS_ERR_TIMEOUT);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

// Residue slices of one Ozaki II operand: for every entry, A' = rint(x 2^(bits
// - e_row)) (|A'| <= 2^bits <= 2^50) and its symmetric residues modulo the n
// moduli, one int8 slice per modulus in the swizzled tile layout of the digit
// slices.  A' stays exact in FP64; adding 1.5 * 2^52 rounds to the integer and
// leaves A' mod 2^32 in the low word.  For an odd modulus p the quotient
// q = rint(A' / p) comes from one FMA (|A' / p| < 2^43, so the rounded 1/p
// moves A'/p by less than 2^-10, while A'/p lies at least 1/(2p) > 2^-9 from
// any half integer) and the residue is the low byte of A' - q p computed in
// 32-bit integers.  For p = 256 it is the low byte of A'.
//
// Thread mapping: a block handles a 32-row group of one k-tile (32 rows x 128
// k values); each thread 16 consecutive k of one row.  When the operand's rows
// are contiguous in memory (transposed storage) a warp spans 32 rows at one
// k-chunk and reads them directly, coalesced.  Otherwise (k contiguous) the
// block first copies the 32 x 128 tile into shared memory with consecutive
// threads on consecutive k (a thread's own 16 k would spread one warp load over
// 32 sectors), each 16-value chunk padded to 17 doubles so that the threads of
// a half warp read 16 distinct bank pairs.
constexpr int kSplitPad = 17;

__global__ void __launch_bounds__(256, 3)
    k_oz2_split(const FsOz2Operand* __restrict__ ops, int64_t n_ops,
                const __grid_constant__ CrtConsts cc) {
    __shared__ double stage[32 * 8 * kSplitPad];
    const int op_id = blockIdx.y;
    if (op_id >= n_ops) return;
    const FsOz2Operand op = ops[op_id];
    const bool rows_contiguous = (op.s_row == 1 && op.s_k != 1);
    const int t = threadIdx.x;
    const int r = rows_contiguous ? (t & 31) : (t >> 3);   // row within the 32-row group
    const int c = rows_contiguous ? (t >> 5) : (t & 7);    // 16-byte chunk of the k-tile
    const int groups = op.rowtiles * (kSplitRows / 32);
    const int64_t units = static_cast<int64_t>(groups) * op.ktiles;
    const int64_t slice_stride = static_cast<int64_t>(op.ktiles) * op.rowtiles * kABytes;
    const int n = cc.n;
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int kt = static_cast<int>(u / groups);
        const int rg = static_cast<int>(u % groups);
        const int rt = rg / (kSplitRows / 32);
        const int rr = (rg % (kSplitRows / 32)) * 32 + r;       // row within the tile
        const int64_t row = static_cast<int64_t>(rt) * kSplitRows + rr;
        const int64_t k0 = static_cast<int64_t>(kt) * kTileK + c * 16;
        const bool row_ok = row < op.rows;
        const int sh = op.bits - (row_ok ? op.exps[row] : 0);
        if (!rows_contiguous) {
            // coalesced copy of the block's 32 rows x 128 k into shared memory
            const int64_t row_base = static_cast<int64_t>(rt) * kSplitRows +
                                     (rg % (kSplitRows / 32)) * 32;
            const int64_t kb = static_cast<int64_t>(kt) * kTileK;
            __syncthreads();   // the previous unit's reads of the stage are done
#pragma unroll
            for (int it = 0; it < 16; ++it) {
                const int e = it * 256 + t;
                const int sr = e >> 7, sk = e & 127;
                const int64_t grow = row_base + sr, gk = kb + sk;
                stage[(sr * 8 + (sk >> 4)) * kSplitPad + (sk & 15)] =
                    (grow < op.rows && gk < op.K) ? __ldg(op.src + grow * op.s_row + gk * op.s_k)
                                                  : 0.0;
            }
            __syncthreads();
        }
        int8_t* dst = op.slices + (static_cast<int64_t>(kt) * op.rowtiles + rt) * kABytes +
                      rr * 128 + ((c ^ (rr & 7)) * 16);
        // the 16 k of this thread in two halves of 8 (8-byte stores per
        // modulus): half the live operand registers, so that three CTAs fit on
        // an SM without spills
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int32_t lo[8];
            double ad[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int64_t k = k0 + 8 * h + j;
                double x;
                if (rows_contiguous)
                    x = (row_ok && k < op.K) ? __ldg(op.src + row * op.s_row + k * op.s_k) : 0.0;
                else
                    x = stage[(r * 8 + c) * kSplitPad + 8 * h + j];
                const double tt = scale2(x, sh) + kRoundMagic;
                lo[j] = __double2loint(tt);
                ad[j] = tt - kRoundMagic;
            }
            {
                uint32_t w[2] = {0, 0};
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    w[j / 4] |= (static_cast<uint32_t>(lo[j]) & 0xFFu) << (8 * (j % 4));
                *reinterpret_cast<uint2*>(dst + 8 * h) = make_uint2(w[0], w[1]);
            }
            for (int m = 1; m < n; ++m) {
                const int32_t pm = cc.p[m];
                const double ipm = cc.inv_p[m];
                uint32_t w[2] = {0, 0};
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int32_t q = __double2loint(fma(ad[j], ipm, kRoundMagic));
                    w[j / 4] |= (static_cast<uint32_t>(lo[j] - q * pm) & 0xFFu) << (8 * (j % 4));
                }
                *reinterpret_cast<uint2*>(dst + m * slice_stride + 8 * h) = make_uint2(w[0], w[1]);
            }
        }
    }
}

// Row exponents of Ozaki II operands (exps[v] = e with max_k |x(v, k)| < 2^e,
// 0 for a zero row): one warp per row when k is contiguous, else a 32-row x
// 8-lane block per row group so that a warp reads 32 consecutive rows.
__global__ void __launch_bounds__(256)
    k_oz2_exponents(const FsOz2Operand* __restrict__ ops, int64_t n_ops) {
    const int op_id = blockIdx.y;
    if (op_id >= n_ops) return;
    const FsOz2Operand op = ops[op_id];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (!(op.s_row == 1 && op.s_k != 1)) {
        for (int64_t v = static_cast<int64_t>(blockIdx.x) * 8 + warp; v < op.rows;
             v += static_cast<int64_t>(gridDim.x) * 8) {
            double m = 0.0;
            for (int64_t k = lane; k < op.K; k += 32)
                m = fmax(m, fabs(__ldg(op.src + v * op.s_row + k * op.s_k)));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) {
                int e = 0;
                if (m > 0.0) frexp(m, &e);
                op.exps[v] = e;
            }
        }
        return;
    }
    __shared__ double part[8][33];
    for (int64_t v0 = static_cast<int64_t>(blockIdx.x) * 32; v0 < op.rows;
         v0 += static_cast<int64_t>(gridDim.x) * 32) {
        const int64_t v = v0 + lane;
        double m = 0.0;
        if (v < op.rows)
            for (int64_t k = warp; k < op.K; k += 8) m = fmax(m, fabs(__ldg(op.src + v + k * op.s_k)));
        part[warp][lane] = m;
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int w = 1; w < 8; ++w) m = fmax(m, part[w][lane]);
            if (v < op.rows) {
                int e = 0;
                if (m > 0.0) frexp(m, &e);
                op.exps[v] = e;
            }
        }
        __syncthreads();
    }
}

}  // namespace oz
}  // namespace fsb

extern "C" int fs_ozaki_geometry(int32_t* tile_m, int32_t* tile_n, int32_t* tile_k,
                                 int32_t* split_rows) {
    if (!tile_m || !tile_n || !tile_k || !split_rows) return FS_ERR_INVALID_ARG;
    *tile_m = fsb::oz::kTileM;
    *tile_n = fsb::oz::kTileN;
    *tile_k = fsb::oz::kTileK;
    *split_rows = fsb::oz::kSplitRows;
    return FS_OK;
}

extern "C" int fs_ozaki_split(const FsOzOperand* d_ops, int64_t n_ops, int32_t max_rows,
                              int32_t max_tiles, int32_t nslices, void* stream) {
    if (n_ops < 0 || max_rows < 0 || max_tiles < 0) return FS_ERR_INVALID_ARG;
    if (nslices < 1 || nslices > FS_OZAKI_MAX_SLICES) return FS_ERR_INVALID_ARG;
    if (n_ops == 0 || max_tiles == 0) return FS_OK;
    if (d_ops == nullptr) return FS_ERR_INVALID_ARG;
    if (n_ops > 65535) return FS_ERR_TOO_LARGE;
    cudaStream_t s = fsb::as_stream(stream);
    const int gx = static_cast<int>(
        ((max_rows + 7) / 8) < 4 * fsb::num_sms() ? ((max_rows + 7) / 8) : 4 * fsb::num_sms());
    fsb::oz::k_oz_exponents<<<dim3(gx > 0 ? gx : 1, static_cast<unsigned>(n_ops)), 256, 0, s>>>(
        d_ops, n_ops);
    int st = fsb::launch_status();
    if (st != FS_OK) return st;
    const int tx = max_tiles < 4 * fsb::num_sms() ? max_tiles : 4 * fsb::num_sms();
    fsb::oz::k_oz_split<<<dim3(tx, static_cast<unsigned>(n_ops)), 1024, 0, s>>>(d_ops, n_ops,
                                                                                nslices);
    return fsb::launch_status();
}

extern "C" int fs_ozaki_gemm(const FsOzProblem* d_probs, int64_t n_probs,
                             const FsOzTile* d_tiles, int64_t n_tiles, int32_t nslices,
                             int32_t chunk_ktiles, int32_t* d_flag, void* stream) {
    if (n_probs < 0 || n_tiles < 0 || chunk_ktiles < 1) return FS_ERR_INVALID_ARG;
    if (nslices < 1 || nslices > FS_OZAKI_MAX_SLICES) return FS_ERR_INVALID_ARG;
    if (n_tiles == 0) return FS_OK;
    if (d_probs == nullptr || d_tiles == nullptr) return FS_ERR_INVALID_ARG;
    // int32 accumulation bound: nslices * chunk * 128 * 127^2 < 2^31
    const long long bound = static_cast<long long>(nslices) * chunk_ktiles * fsb::oz::kTileK *
                            127LL * 127LL;
    if (bound >= (1LL << 31)) return FS_ERR_INVALID_ARG;
    const int smem = fsb::oz::kStages * fsb::oz::kStageBytes +
                     static_cast<int>(sizeof(fsb::oz::Barriers)) + 1024;
    const int cfg = fsb::configure_smem(reinterpret_cast<const void*>(fsb::oz::k_oz_gemm), smem);
    if (cfg != FS_OK) return cfg;
    const int grid = static_cast<int>(n_tiles < fsb::num_sms() ? n_tiles : fsb::num_sms());
    fsb::oz::k_oz_gemm<<<grid, fsb::oz::kThreads, smem, fsb::as_stream(stream)>>>(
        d_probs, n_probs, d_tiles, n_tiles, nslices, chunk_ktiles, d_flag, fsb::spin_limit());
    return fsb::launch_status();
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

}  // namespace

// ------------------------------------------------- Ozaki II host side

namespace {

using u128 = unsigned __int128;

int bitlen(u128 x) {
    int b = 0;
    while (x != 0) {
        ++b;
        x >>= 1;
    }
    return b;
}

// CRT constants for the first n moduli (exact integer arithmetic: P < 2^111)
bool make_crt_consts(int n, fsb::oz::CrtConsts* c) {
    using fsb::oz::kModuli;
    if (n < FS_OZAKI2_MIN_MODULI || n > FS_OZAKI2_MAX_MODULI) return false;
    std::memset(c, 0, sizeof(*c));
    u128 P = 1;
    for (int m = 0; m < n; ++m) P *= static_cast<u128>(kModuli[m]);
    // |sum_m r_m W_m| + |k| P <= 128 n P + 128 n P
    const u128 bound = P * static_cast<u128>(256 * n);
    int e1 = bitlen(bound) - 53;
    if (e1 < 0) e1 = 0;
    int e2 = e1 + bitlen(static_cast<u128>(256 * n)) - 53;
    if (e2 < 0) e2 = 0;
    c->n = n;
    c->e1 = e1;
    c->e2 = e2;
    for (int m = 0; m < n; ++m) {
        const int32_t p = kModuli[m];
        const u128 Q = P / static_cast<u128>(p);
        const int32_t qm = static_cast<int32_t>(Q % static_cast<u128>(p));
        int32_t y = 0;
        for (int32_t t = 1; t < p; ++t)
            if ((static_cast<int64_t>(qm) * t) % p == 1) {
                y = t;
                break;
            }
        if (y == 0) return false;
        const u128 W = Q * static_cast<u128>(y);
        const u128 w1 = (W >> e1) << e1;
        c->p[m] = p;
        c->inv_p[m] = 1.0 / static_cast<double>(p);
        c->f[m] = static_cast<float>(static_cast<double>(y) / static_cast<double>(p));
        c->w1[m] = std::ldexp(static_cast<double>(static_cast<uint64_t>(W >> e1)), e1);
        c->w2[m] = std::ldexp(static_cast<double>(static_cast<uint64_t>((W - w1) >> e2)), e2);
    }
    const u128 p1 = (P >> e1) << e1;
    c->p1 = std::ldexp(static_cast<double>(static_cast<uint64_t>(P >> e1)), e1);
    c->p2 = std::ldexp(static_cast<double>(static_cast<uint64_t>((P - p1) >> e2)), e2);
    // the offsets are exact: 128 sum_m w1_m stays on the 2^e1 grid below
    // 2^(53 + e1) (likewise for w2), and are added first
    double s1 = 0.0, s2 = 0.0;
    for (int m = 0; m < n; ++m) {
        s1 += c->w1[m];
        s2 += c->w2[m];
    }
    c->c1 = -128.0 * s1;
    c->c2 = -128.0 * s2;
    c->inv_P = 1.0 / std::ldexp(static_cast<double>(static_cast<uint64_t>(P >> e1)), e1);
    return true;
}

const fsb::oz::CrtConsts* crt_consts(int n) {
    static fsb::oz::CrtConsts table[FS_OZAKI2_MAX_MODULI + 1];
    static bool ok[FS_OZAKI2_MAX_MODULI + 1];
    static std::once_flag once;
    std::call_once(once, [] {
        for (int k = FS_OZAKI2_MIN_MODULI; k <= FS_OZAKI2_MAX_MODULI; ++k)
            ok[k] = make_crt_consts(k, &table[k]);
    });
    if (n < FS_OZAKI2_MIN_MODULI || n > FS_OZAKI2_MAX_MODULI || !ok[n]) return nullptr;
    return &table[n];
}

// tensor map viewing a workspace as rows of 128 bytes (box 128 x 128): a
// 16-byte aligned base, whole rows, and row indices that fit the 32-bit TMA
// coordinate
int workspace_map(const void* d_workspace, int64_t workspace_bytes, CUtensorMap* map) {
    if ((reinterpret_cast<uintptr_t>(d_workspace) & 127u) != 0 || workspace_bytes < 128 * 128 ||
        (workspace_bytes & 127) != 0 || (workspace_bytes >> 7) >= (1LL << 31))
        return FS_ERR_INVALID_ARG;
    EncodeTiledFn enc = encode_tiled();
    if (enc == nullptr) return FS_ERR_UNSUPPORTED;
    const cuuint64_t dims[2] = {128, static_cast<cuuint64_t>(workspace_bytes >> 7)};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {128, 128};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(d_workspace), dims, strides,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return FS_ERR_INVALID_ARG;
    return FS_OK;
}

constexpr int kPairSmem = fsb::oz::kPairStages * fsb::oz::kPairStageBytes +
                          static_cast<int>(sizeof(fsb::oz::PairBarriers)) + 1024;

}  // namespace

extern "C" int fs_ozaki2_bits(int32_t nmod, int64_t K, int32_t* a_bits, int32_t* b_bits) {
    if (a_bits == nullptr || b_bits == nullptr || K < 0) return FS_ERR_INVALID_ARG;
    if (nmod < FS_OZAKI2_MIN_MODULI || nmod > FS_OZAKI2_MAX_MODULI) return FS_ERR_INVALID_ARG;
    if (K > FS_OZAKI2_MAX_K) return FS_ERR_UNSUPPORTED;
    u128 P = 1;
    for (int m = 0; m < nmod; ++m) P *= static_cast<u128>(fsb::oz::kModuli[m]);
    int ck = 0;
    while ((int64_t{1} << ck) < (K > 1 ? K : 1)) ++ck;
    // |X| <= K 2^(a+b) <= P / 4
    const int L = (bitlen(P) - 1) - 2 - ck;
    int a = L / 2;
    int b = L - a;
    if (a > 50) a = 50;
    if (b > 50) b = 50;
    if (a < 1) return FS_ERR_UNSUPPORTED;
    *a_bits = a;
    *b_bits = b;
    return FS_OK;
}

extern "C" int fs_ozaki2_constants(int32_t nmod, int32_t* moduli, double* weights_hi,
                                   double* weights_lo, double* modulus_product, float* frac,
                                   int32_t* grids) {
    const fsb::oz::CrtConsts* c = crt_consts(nmod);
    if (c == nullptr) return FS_ERR_INVALID_ARG;
    if (!moduli || !weights_hi || !weights_lo || !modulus_product || !frac || !grids)
        return FS_ERR_INVALID_ARG;
    for (int m = 0; m < nmod; ++m) {
        moduli[m] = c->p[m];
        weights_hi[m] = c->w1[m];
        weights_lo[m] = c->w2[m];
        frac[m] = c->f[m];
    }
    modulus_product[0] = c->p1;
    modulus_product[1] = c->p2;
    grids[0] = c->e1;
    grids[1] = c->e2;
    return FS_OK;
}

extern "C" int fs_ozaki2_scratch_bytes(int32_t nmod, int64_t* bytes) {
    if (bytes == nullptr) return FS_ERR_INVALID_ARG;
    if (nmod < FS_OZAKI2_MIN_MODULI || nmod > FS_OZAKI2_MAX_MODULI) return FS_ERR_INVALID_ARG;
    const int64_t ctas = 2 * (fsb::num_sms() / 2);
    *bytes = ctas * nmod * static_cast<int64_t>(fsb::oz::kCrtModulusBytes);
    return FS_OK;
}

extern "C" int fs_ozaki2_split(const FsOz2Operand* d_ops, int64_t n_ops, int32_t max_rows,
                               int64_t max_units, int32_t nmod, void* stream) {
    if (n_ops < 0 || max_rows < 0 || max_units < 0) return FS_ERR_INVALID_ARG;
    const fsb::oz::CrtConsts* c = crt_consts(nmod);
    if (c == nullptr) return FS_ERR_INVALID_ARG;
    if (n_ops == 0 || max_units == 0) return FS_OK;
    if (d_ops == nullptr) return FS_ERR_INVALID_ARG;
    if (n_ops > 65535) return FS_ERR_TOO_LARGE;
    cudaStream_t s = fsb::as_stream(stream);
    const int sms = fsb::num_sms();
    const int64_t ge = std::min<int64_t>((max_rows + 7) / 8, 4 * sms);
    fsb::oz::k_oz2_exponents<<<dim3(static_cast<unsigned>(ge > 0 ? ge : 1),
                                    static_cast<unsigned>(n_ops)),
                               256, 0, s>>>(d_ops, n_ops);
    int st = fsb::launch_status();
    if (st != FS_OK) return st;
    const int64_t gs = std::min<int64_t>(max_units, 8 * sms);
    fsb::oz::k_oz2_split<<<dim3(static_cast<unsigned>(gs), static_cast<unsigned>(n_ops)), 256, 0,
                           s>>>(d_ops, n_ops, *c);
    return fsb::launch_status();
}

extern "C" int fs_ozaki2_gemm_pair(const FsOz2Problem* d_probs, int64_t n_probs,
                                   const FsOzTile* d_tiles, int64_t n_tiles, int32_t nmod,
                                   const void* d_workspace, int64_t workspace_bytes,
                                   void* d_scratch, int64_t scratch_bytes, int32_t* d_flag,
                                   void* stream) {
    if (n_probs < 0 || n_tiles < 0) return FS_ERR_INVALID_ARG;
    const fsb::oz::CrtConsts* c = crt_consts(nmod);
    if (c == nullptr) return FS_ERR_INVALID_ARG;
    if (n_tiles == 0) return FS_OK;
    if (d_probs == nullptr || d_tiles == nullptr || d_workspace == nullptr || d_scratch == nullptr)
        return FS_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_scratch) & 15u) != 0) return FS_ERR_INVALID_ARG;
    CUtensorMap map;
    int st = workspace_map(d_workspace, workspace_bytes, &map);
    if (st != FS_OK) return st;
    const int64_t max_clusters = fsb::num_sms() / 2;
    const int clusters = static_cast<int>(n_tiles < max_clusters ? n_tiles : max_clusters);
    if (scratch_bytes < 2LL * clusters * nmod * fsb::oz::kCrtModulusBytes) return FS_ERR_INVALID_ARG;
    const void* fn = reinterpret_cast<const void*>(fsb::oz::k_oz_pair<FsOz2Problem, true>);
    st = fsb::configure_smem(fn, kPairSmem);
    if (st != FS_OK) return st;
    fsb::oz::k_oz_pair<FsOz2Problem, true>
        <<<2 * clusters, fsb::oz::kThreads, kPairSmem, fsb::as_stream(stream)>>>(
            d_probs, n_probs, d_tiles, n_tiles, nmod, 1, d_flag, map,
            static_cast<const int8_t*>(d_workspace), fsb::spin_limit(),
            static_cast<uint8_t*>(d_scratch), *c);
    return fsb::launch_status();
}

extern "C" int fs_ozaki_gemm_pair(const FsOzProblem* d_probs, int64_t n_probs,
                                  const FsOzTile* d_tiles, int64_t n_tiles, int32_t nslices,
                                  int32_t chunk_ktiles, const void* d_workspace,
                                  int64_t workspace_bytes, int32_t* d_flag, void* stream) {
    if (n_probs < 0 || n_tiles < 0 || chunk_ktiles < 1) return FS_ERR_INVALID_ARG;
    if (nslices < 1 || nslices > FS_OZAKI_MAX_SLICES) return FS_ERR_INVALID_ARG;
    if (n_tiles == 0) return FS_OK;
    if (d_probs == nullptr || d_tiles == nullptr || d_workspace == nullptr)
        return FS_ERR_INVALID_ARG;
    CUtensorMap map;
    int st = workspace_map(d_workspace, workspace_bytes, &map);
    if (st != FS_OK) return st;
    const long long bound = static_cast<long long>(nslices) * chunk_ktiles * fsb::oz::kTileK *
                            127LL * 127LL;
    if (bound >= (1LL << 31)) return FS_ERR_INVALID_ARG;
    const void* fn = reinterpret_cast<const void*>(fsb::oz::k_oz_pair<FsOzProblem, false>);
    st = fsb::configure_smem(fn, kPairSmem);
    if (st != FS_OK) return st;
    const int64_t max_clusters = fsb::num_sms() / 2;
    const int clusters = static_cast<int>(n_tiles < max_clusters ? n_tiles : max_clusters);
    fsb::oz::CrtConsts unused;
    std::memset(&unused, 0, sizeof(unused));
    fsb::oz::k_oz_pair<FsOzProblem, false>
        <<<2 * clusters, fsb::oz::kThreads, kPairSmem, fsb::as_stream(stream)>>>(
            d_probs, n_probs, d_tiles, n_tiles, nslices, chunk_ktiles, d_flag, map,
            static_cast<const int8_t*>(d_workspace), fsb::spin_limit(), nullptr, unused);
    return fsb::launch_status();
}

// ------------------------------------------------------ no-allocation variant
//
// Some callers cannot allocate device memory: a host application whose own
// memory pool has already reserved the device (a cudaMalloc from a library
// inside it would fail or fragment that pool), or a C / Fortran driver with no
// device allocator of its own that only holds the input and output buffers.
// fs_ozaki_gemm_noalloc serves them: the digit slices, exponents and launch
// tables live in one fixed file-scope device array instead of a caller-provided
// workspace.  Every GPU that loads this library holds that array until the
// process exits.

namespace {

constexpr size_t kNoAllocScratchBytes = static_cast<size_t>(48) << 20;   // 48 MiB
constexpr int64_t kNoAllocStatusBytes = 256;   // status word, padded to keep slices aligned
constexpr int kNoAllocMaxDevices = 64;

std::mutex g_noalloc_mutex;
uint8_t* g_noalloc_base[kNoAllocMaxDevices] = {};

}  // namespace

static __device__ __align__(256) uint8_t g_ozaki_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with that device current.
int noalloc_scratch(uint8_t** base) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        fsb::set_last_cuda_error(e);
        return FS_ERR_CUDA;
    }
    if (device < 0 || device >= kNoAllocMaxDevices) return FS_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_base[device] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_ozaki_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            fsb::set_last_cuda_error(e);
            return FS_ERR_CUDA;
        }
        g_noalloc_base[device] = static_cast<uint8_t*>(p);
    }
    *base = g_noalloc_base[device];
    return FS_OK;
}

int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

}  // namespace

extern "C" int fs_ozaki_gemm_noalloc(const FsGemmProblem* h_problems, int64_t n_problems,
                                     int32_t nslices, void* stream) {
    using namespace fsb::oz;
    if (n_problems < 0 || nslices < 1 || nslices > FS_OZAKI_MAX_SLICES)
        return FS_ERR_INVALID_ARG;
    if (n_problems == 0) return FS_OK;
    if (h_problems == nullptr) return FS_ERR_INVALID_ARG;
    cudaStream_t s = fsb::as_stream(stream);
    // the launch tables are staged from host memory that is gone when this
    // call returns: a captured copy would replay from freed memory
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(s, &capturing);
    if (ce != cudaSuccess) {
        fsb::set_last_cuda_error(ce);
        return FS_ERR_CUDA;
    }
    if (capturing != cudaStreamCaptureStatusNone) return FS_ERR_UNSUPPORTED;

    // layout of the scratch: the status word, per problem slices and
    // exponents, then the tables
    std::vector<FsOzOperand> ops;
    std::vector<FsOzProblem> probs;
    std::vector<std::pair<int32_t, FsOzTile>> tiles;  // (K, tile) for ordering
    int64_t off = kNoAllocStatusBytes;
    int32_t max_rows = 0, max_tiles = 0;
    for (int64_t i = 0; i < n_problems; ++i) {
        const FsGemmProblem& g = h_problems[i];
        if (g.M < 0 || g.N < 0 || g.K < 0) return FS_ERR_INVALID_ARG;
        if (g.M == 0 || g.N == 0) continue;
        if (g.C == nullptr || (g.K > 0 && (g.A == nullptr || g.B == nullptr)))
            return FS_ERR_INVALID_ARG;
        const int32_t kt = g.K > 0 ? (g.K + kTileK - 1) / kTileK : 1;
        const int32_t art = (g.M + kSplitRows - 1) / kSplitRows;
        const int32_t ntn = (g.N + kTileN - 1) / kTileN;
        const int32_t brt = 2 * ntn;
        const int64_t a_sl = off;
        off += static_cast<int64_t>(nslices) * kt * art * kABytes;
        const int64_t b_sl = off;
        off += static_cast<int64_t>(nslices) * kt * brt * kABytes;
        const int64_t a_ex = off;
        off += round_up(4 * static_cast<int64_t>(g.M), 256);
        const int64_t b_ex = off;
        off += round_up(4 * static_cast<int64_t>(g.N), 256);
        off = round_up(off, 1024);
        if (off > static_cast<int64_t>(kNoAllocScratchBytes)) return FS_ERR_TOO_LARGE;
        // offsets are patched to device addresses once the layout is known
        FsOzOperand a{g.A, g.transA ? 1 : g.lda, g.transA ? g.lda : 1,
                      reinterpret_cast<int8_t*>(a_sl), reinterpret_cast<int32_t*>(a_ex),
                      g.M, g.K, art, kt};
        FsOzOperand b{g.B, g.transB ? g.ldb : 1, g.transB ? 1 : g.ldb,
                      reinterpret_cast<int8_t*>(b_sl), reinterpret_cast<int32_t*>(b_ex),
                      g.N, g.K, brt, kt};
        ops.push_back(a);
        ops.push_back(b);
        FsOzProblem p{reinterpret_cast<const int8_t*>(a_sl), reinterpret_cast<const int8_t*>(b_sl),
                      reinterpret_cast<const int32_t*>(a_ex), reinterpret_cast<const int32_t*>(b_ex),
                      g.C, g.ldc, g.M, g.N, g.K, art, brt, kt, g.alpha, g.beta};
        const int32_t pid = static_cast<int32_t>(probs.size());
        probs.push_back(p);
        for (int32_t tm = 0; tm < art; ++tm)
            for (int32_t tn = 0; tn < ntn; ++tn) tiles.push_back({g.K, FsOzTile{pid, tm, tn, 0}});
        max_rows = std::max(max_rows, std::max(g.M, g.N));
        max_tiles = std::max(max_tiles, std::max(art, brt) * kt);
    }
    if (tiles.empty()) return FS_OK;
    std::stable_sort(tiles.begin(), tiles.end(),
                     [](const auto& x, const auto& y) { return x.first > y.first; });

    const int64_t ops_off = off;
    const int64_t probs_off = round_up(ops_off + static_cast<int64_t>(ops.size() * sizeof(FsOzOperand)), 256);
    const int64_t tiles_off = round_up(probs_off + static_cast<int64_t>(probs.size() * sizeof(FsOzProblem)), 256);
    const int64_t end = tiles_off + static_cast<int64_t>(tiles.size() * sizeof(FsOzTile));
    if (end > static_cast<int64_t>(kNoAllocScratchBytes)) return FS_ERR_TOO_LARGE;

    uint8_t* base = nullptr;
    int st = noalloc_scratch(&base);
    if (st != FS_OK) return st;
    const uintptr_t b = reinterpret_cast<uintptr_t>(base);
    for (auto& o : ops) {
        o.slices = reinterpret_cast<int8_t*>(b + reinterpret_cast<uintptr_t>(o.slices));
        o.exps = reinterpret_cast<int32_t*>(b + reinterpret_cast<uintptr_t>(o.exps));
    }
    for (auto& p : probs) {
        p.a_slices = reinterpret_cast<const int8_t*>(b + reinterpret_cast<uintptr_t>(p.a_slices));
        p.b_slices = reinterpret_cast<const int8_t*>(b + reinterpret_cast<uintptr_t>(p.b_slices));
        p.a_exps = reinterpret_cast<const int32_t*>(b + reinterpret_cast<uintptr_t>(p.a_exps));
        p.b_exps = reinterpret_cast<const int32_t*>(b + reinterpret_cast<uintptr_t>(p.b_exps));
    }
    std::vector<uint8_t> staging(static_cast<size_t>(end - ops_off), 0);
    std::memcpy(staging.data(), ops.data(), ops.size() * sizeof(FsOzOperand));
    std::memcpy(staging.data() + (probs_off - ops_off), probs.data(),
                probs.size() * sizeof(FsOzProblem));
    FsOzTile* tdst = reinterpret_cast<FsOzTile*>(staging.data() + (tiles_off - ops_off));
    for (size_t i = 0; i < tiles.size(); ++i) tdst[i] = tiles[i].second;

    // the status word starts every call at zero; a bounded device wait that
    // runs out writes FS_ERR_TIMEOUT into it (fs_ozaki_noalloc_status)
    int32_t* d_status = reinterpret_cast<int32_t*>(base);
    cudaError_t e = cudaMemsetAsync(d_status, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) {
        fsb::set_last_cuda_error(e);
        return FS_ERR_CUDA;
    }
    // pageable source: the call returns once the bytes are staged, so the
    // host vectors may go out of scope afterwards
    e = cudaMemcpyAsync(base + ops_off, staging.data(), staging.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        fsb::set_last_cuda_error(e);
        return FS_ERR_CUDA;
    }
    const FsOzOperand* d_ops = reinterpret_cast<const FsOzOperand*>(base + ops_off);
    const int64_t n_ops = static_cast<int64_t>(ops.size());
    for (int64_t start = 0; start < n_ops; start += 65534) {
        const int64_t cnt = std::min<int64_t>(65534, n_ops - start);
        st = fs_ozaki_split(d_ops + start, cnt, max_rows, max_tiles, nslices, stream);
        if (st != FS_OK) return st;
    }
    const int32_t chunk = static_cast<int32_t>(std::max<long long>(
        1, ((1LL << 31) - 1) / (static_cast<long long>(nslices) * kTileK * 127 * 127)));
    return fs_ozaki_gemm(reinterpret_cast<const FsOzProblem*>(base + probs_off),
                         static_cast<int64_t>(probs.size()),
                         reinterpret_cast<const FsOzTile*>(base + tiles_off),
                         static_cast<int64_t>(tiles.size()), nslices, chunk, d_status, stream);
}

extern "C" int fs_ozaki_noalloc_status(void* stream, int32_t* status) {
    if (status == nullptr) return FS_ERR_INVALID_ARG;
    uint8_t* base = nullptr;
    int st = noalloc_scratch(&base);
    if (st != FS_OK) return st;
    cudaError_t e = cudaStreamSynchronize(fsb::as_stream(stream));
    if (e == cudaSuccess) e = cudaMemcpy(status, base, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        fsb::set_last_cuda_error(e);
        return FS_ERR_CUDA;
    }
    return FS_OK;
}
