/*
 * frostspin_b200 C ABI.
 *
 * Block-sparse symmetric-tensor kernels for NVIDIA B200 (sm_100a).  Every entry
 * point takes plain device pointers, sizes and a cudaStream_t passed as void*,
 * returns an int status (FS_OK == 0, negative on error) and never allocates or
 * frees device memory: the caller (PyTorch's caching allocator in the Python
 * package) owns every buffer, including plan tables and scratch space.  No
 * exception crosses this boundary.
 *
 * Data layout shared by all entry points: a symmetric tensor is one contiguous
 * float64 buffer holding its irrep blocks back to back, each block a dense
 * row-major (C-order) matrix at an element offset into the buffer.  A tensor
 * may instead carry all of its blocks transposed (F-order); the plans below
 * encode that in their strides.
 *
 * Each declaration names the reference (frostspin 1.0.0) interface it replaces.
 */
#ifndef FROSTSPIN_B200_H
#define FROSTSPIN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define FS_OK 0
#define FS_ERR_INVALID_ARG (-1)   /* null pointer, negative size, bad enum       */
#define FS_ERR_LAUNCH (-2)        /* kernel launch failed (cudaGetLastError)     */
#define FS_ERR_BOUNDS (-3)        /* a plan entry lies outside its buffer        */
#define FS_ERR_TIMEOUT (-4)       /* a bounded device wait ran out               */
#define FS_ERR_UNSUPPORTED (-5)   /* shape or mode this build does not handle    */
#define FS_ERR_CUDA (-6)          /* other CUDA runtime error                    */
#define FS_ERR_TOO_LARGE (-7)     /* request exceeds a fixed internal capacity   */

/* Library version (major*10000 + minor*100 + patch). */
int fs_version(void);

/* Human-readable text of a status code (static storage). */
const char* fs_status_string(int status);

/* Name of the last CUDA error seen by this library on the calling thread. */
const char* fs_last_cuda_error(void);

/*
 * Bound, in clock64 cycles, of every device wait of the tcgen05 kernels that
 * ends in FS_ERR_TIMEOUT (default 2e9, about one second); cycles <= 0 restores
 * the default.  Returns the previous bound.  Kernels launched afterwards use
 * the new bound; the waits that drain in-flight copies and MMAs before a
 * kernel returns keep the default.  No counterpart in the reference (which has
 * no device code); it exists so that the timeout path can be exercised.
 */
int64_t fs_set_spin_limit(int64_t cycles);

/* --------------------------------------------------------- abelian permute */
/*
 * An elementary block (EB) is the set of tensor entries whose legs each lie in
 * one fixed run of constant irrep ("segment") of their representation.  Inside
 * one EB the input and output element offsets are affine in the per-leg local
 * indices, so the whole permutation is a batch of strided copies.  Legs are
 * listed outer to inner in output order; dims[ndim-1] is the output-innermost
 * leg; a row is one run along it, and a task covers at most 1024 whole rows
 * of one EB.
 * divm/divs are the Granlund-Montgomery magic multiplier and shift for
 * dividing by dims[k] (host computed).  obase < 0 marks an EB whose source
 * block is absent: its output entries are written as zeros.
 */
#define FS_PERM_MAXR 8

typedef struct FsPermEB {
    int64_t obase;                   /* input element offset of local index 0   */
    int64_t nbase;                   /* output element offset of local index 0  */
    int64_t ostride[FS_PERM_MAXR];   /* input stride per leg (elements)         */
    int64_t nstride[FS_PERM_MAXR];   /* output stride per leg (elements)        */
    uint32_t dims[FS_PERM_MAXR];
    uint32_t divm[FS_PERM_MAXR];
    uint32_t divs[FS_PERM_MAXR];
    int32_t ndim;
    uint32_t volume;                 /* product of dims, < 2^31                 */
    int32_t tile_leg;                /* leg with ostride == 1 for a tiled
                                        transpose, -1 for a plain gather        */
    int32_t pad;                     /* fs_abelian_permute_multi: buffer pair   */
} FsPermEB;

typedef struct FsPermTask {
    int32_t eb;                      /* index into the EB table                 */
    uint32_t start;                  /* first row (run along the last leg)      */
    uint32_t count;                  /* number of rows, at most 1024            */
    uint32_t pad;
} FsPermTask;

/*
 * Replaces AbelianSymmetricTensor._permute_data -> _numba_abelian_transpose
 * (frostspin/symmetric_tensor/abelian_symmetric_tensor.py:395-430, :103-250)
 * for U(1) and Z2.  d_ebs / d_tasks are device tables built by the host plan
 * (frostspin_b200/symmetric_tensor/abelian_plan.py).  in_len / out_len are the
 * buffer lengths in elements; every EB is checked against them on the host
 * side of the plan builder, and the kernel skips (and flags) any access that
 * would fall outside, returning FS_ERR_BOUNDS after the stream synchronises
 * when d_flag is not null.
 */
int fs_abelian_permute(const double* d_in, int64_t in_len, double* d_out,
                       int64_t out_len, const FsPermEB* d_ebs, int64_t n_ebs,
                       const FsPermTask* d_tasks, int64_t n_tasks,
                       int32_t* d_flag, void* stream);

/* -------------------------------------------------- fused SU(2) permute */
/*
 * Replaces LieGroupSymmetricTensor._lie_permute_data -> fill_blocks_out ->
 * permute_simple_block (frostspin/symmetric_tensor/lie_group_symmetric_tensor.py
 * :96-265, :735-835) for the simple blocks whose recoupling matrix is at most
 * 32 x 32: gather, recoupling product and scatter in one pass.
 *
 * A group is one simple block: K input rows (input sectors x structural
 * multiplicities), M output rows, ncols columns = the external multi-index in
 * output leg order (dims, outer to inner, with Granlund-Montgomery divm / divs
 * per leg as in FsPermEB), and U (M x K, row-major) at u_off in the U buffer.
 * A piece is one sector's share of a group: rows row0 .. row0 + sr*sc - 1 of
 * the group (structural index sr outer), at element base + r*sr_stride +
 * c*sc_stride + sum_l e_l*ext[l] of its buffer for column multi-index e.  An
 * input piece with base < 0 is an absent source block (zeros).  Pieces
 * in_first .. in_first + in_count - 1 are the group's inputs, out_first .. its
 * outputs.  Tasks are FsPermTask with eb = group index, start = first column,
 * count = number of columns; the columns of a task span at most
 * FS_SU2_TASK_ROWS values of the outer legs (all legs but the innermost), a
 * task that spans more is skipped and flagged.  Limits: fs_su2_fused_limits.
 * Accesses outside a buffer are skipped and raise FS_ERR_BOUNDS in *d_flag (if
 * not null).
 */
#define FS_SU2_MAXD 8
#define FS_SU2_TASK_ROWS 48

typedef struct FsSu2Group {
    int64_t u_off;
    int64_t ncols;
    uint32_t dims[FS_SU2_MAXD];
    uint32_t divm[FS_SU2_MAXD];
    uint32_t divs[FS_SU2_MAXD];
    int32_t ndim, M, K;
    int32_t in_first, in_count, out_first, out_count;
    int32_t pad;
} FsSu2Group;

typedef struct FsSu2Piece {
    int64_t base;
    int64_t sr_stride, sc_stride;
    int64_t ext[FS_SU2_MAXD];
    int32_t sr, sc;
    int32_t row0;
    int32_t pad;
} FsSu2Piece;

int fs_su2_fused_limits(int32_t* max_rows, int32_t* max_pieces, int32_t* threads);

int fs_su2_permute_fused(const double* d_src, int64_t src_len, double* d_out, int64_t out_len,
                         const FsSu2Group* d_groups, int64_t n_groups,
                         const FsSu2Piece* d_pieces, int64_t n_pieces, const double* d_u,
                         int64_t u_len, const FsPermTask* d_tasks, int64_t n_tasks,
                         int32_t* d_flag, void* stream);

/*
 * Several independent abelian permutes in one launch (the permutes of many
 * CTMRG runs advanced in lock step; the reference runs them one by one through
 * AbelianSymmetricTensor._permute_data, abelian_symmetric_tensor.py:395-430).
 * Same EB and task tables as fs_abelian_permute, concatenated; the pad field
 * of every EB indexes the buffer pair it reads and writes in d_bufs.
 */
typedef struct FsPermBuffers {
    const double* in;
    int64_t in_len;
    double* out;
    int64_t out_len;
} FsPermBuffers;

int fs_abelian_permute_multi(const FsPermBuffers* d_bufs, int64_t n_bufs,
                             const FsPermEB* d_ebs, int64_t n_ebs, const FsPermTask* d_tasks,
                             int64_t n_tasks, int32_t* d_flag, void* stream);

/* ------------------------------------------------------- grouped FP64 GEMM */
/*
 * One problem: C[MxN] = alpha * op(A) * op(B) + beta * C, all row-major with
 * leading dimensions in elements.  transA == 0: A[i*lda + k]; transA == 1:
 * A[k*lda + i].  transB == 0: B[k*ldb + j]; transB == 1: B[j*ldb + k].
 * beta == 0 ignores the previous content of C (NaN-safe).
 */
typedef struct FsGemmProblem {
    const double* A;
    const double* B;
    double* C;
    int64_t lda, ldb, ldc;
    int32_t M, N, K;
    int32_t transA, transB;
    int32_t pad;
    double alpha, beta;
} FsGemmProblem;

typedef struct FsGemmTile {
    int32_t problem;
    int32_t tm;   /* tile row index    */
    int32_t tn;   /* tile column index */
    int32_t pad;
} FsGemmTile;

/* Output tile shape used by fs_grouped_dgemm (for building d_tiles). */
int fs_dgemm_tile_shape(int32_t* tile_m, int32_t* tile_n);

/*
 * Replaces the per-irrep-block loop of SymmetricTensor.__matmul__
 * (frostspin/symmetric_tensor/symmetric_tensor.py:453-489) and the sector
 * products of construct_projectors (frostspin/ctmrg/ctm_renormalize.py:92-94,
 * 122-123): every sector of one contraction in a single launch over a
 * device tile list.
 */
int fs_grouped_dgemm(const FsGemmProblem* d_problems, int64_t n_problems,
                     const FsGemmTile* d_tiles, int64_t n_tiles, void* stream);

/*
 * The same launch when every problem has transA == trans_a and transB ==
 * trans_b (the caller guarantees it): one cp.async ring runs across each CTA's
 * tiles, so the next tile's first k slices load while the current tile writes
 * its outputs.  Same call sites as fs_grouped_dgemm.
 */
int fs_grouped_dgemm_uniform(const FsGemmProblem* d_problems, int64_t n_problems,
                             const FsGemmTile* d_tiles, int64_t n_tiles, int32_t trans_a,
                             int32_t trans_b, void* stream);

/*
 * Thin problems of the same table format: M <= max_m, K <= max_k, both
 * operands row-major (transA == transB == 0), N large -- the recoupling
 * products of the SU(2) permute (frostspin/symmetric_tensor/
 * lie_group_symmetric_tensor.py:179, new += U_sector @ old).  Tiles are
 * (problem, tn) over tile_n columns (tm unused).  Problems outside those
 * limits are skipped; the host routes them to fs_grouped_dgemm.
 */
int fs_thin_dgemm_shape(int32_t* max_m, int32_t* max_k, int32_t* tile_n);
int fs_grouped_dgemm_thin(const FsGemmProblem* d_problems, int64_t n_problems,
                          const FsGemmTile* d_tiles, int64_t n_tiles, void* stream);

/*
 * Split-K completion: C = alpha * sum_{j < nslices} W[j * slice ...] + beta * C
 * for M x N row-major results (C leading dimension ldc, slices contiguous
 * M x N), summed in slice order.  The host cuts a long-K sector problem into
 * K chunks (each an FsGemmProblem writing slice j with alpha 1, beta 0) when a
 * contraction has too few output tiles to fill the GPU.
 */
typedef struct FsSplitReduce {
    const double* W;
    double* C;
    int64_t ldc;
    int64_t slice;      /* elements between consecutive slices */
    int32_t nslices;
    int32_t M, N;
    int32_t pad;
    double alpha, beta;
} FsSplitReduce;

int fs_splitk_reduce(const FsSplitReduce* d_items, int64_t n_items, int64_t max_elems,
                     void* stream);

/*
 * Tile table of a grouped GEMM launch, written on the device (a planning
 * helper with no reference counterpart: the reference loops over blocks on the
 * host).  Run r covers tiles [start_r, start_{r+1}) (the last run ends at
 * `total`), all of problem `problem`, over nrow x ncol tiles: tile start_r + k
 * is (problem, k / ncol, k % ncol) in row-major order, or (problem, k % nrow,
 * k / nrow) when col_major is set (wide problems: the few row tiles of a
 * column block run side by side and share its B tile in L2).  Runs are sorted
 * by start, start_0 = 0.  Replaces the host enumeration of every output tile
 * (millions for the wide sector GEMMs of a chi = 256 CTMRG move).
 */
typedef struct FsTileRun {
    int64_t start;
    int32_t problem;
    int32_t ncol;
    int32_t nrow;
    int32_t col_major;
} FsTileRun;

int fs_expand_tiles(const FsTileRun* d_runs, int64_t n_runs, int64_t total, FsGemmTile* d_tiles,
                    void* stream);

/* ------------------------------------- grouped GEMM on tcgen05 (Ozaki int8) */
/*
 * FP64-class GEMM on the int8 tensor cores (tcgen05.mma kind::i8): every row of
 * op(A) and column of op(B) is scaled by a power of two into (-1, 1) and cut
 * into nslices signed 7-bit digits; diagonal sums of slice products are exact
 * int32 accumulations in TMEM, recombined in FP64.  Relative error per entry is
 * ~2^(-7 nslices) of the product of the row/column maxima.
 *
 * Workspace (caller-owned device memory, computed by the host): per operand
 * nslices * ktiles * rowtiles tiles of 128 rows x 128 bytes, written by
 * fs_ozaki_split in the 128-byte-swizzled K-major layout, plus one int32
 * exponent per row.  B operands are stored transposed (rows = columns of op(B))
 * and their rowtiles must be even (256-row MMA tiles).
 */
#define FS_OZAKI_MAX_SLICES 8

typedef struct FsOzOperand {
    const double* src;     /* element (row, k) at src[row*s_row + k*s_k]      */
    int64_t s_row, s_k;
    int8_t* slices;        /* workspace, nslices*ktiles*rowtiles*16384 bytes */
    int32_t* exps;         /* workspace, rows entries                          */
    int32_t rows, K;
    int32_t rowtiles, ktiles;
} FsOzOperand;

typedef struct FsOzProblem {
    const int8_t* a_slices;
    const int8_t* b_slices;
    const int32_t* a_exps;
    const int32_t* b_exps;
    double* C;             /* row-major M x N, leading dimension ldc          */
    int64_t ldc;
    int32_t M, N, K;
    int32_t a_rowtiles, b_rowtiles, ktiles;
    double alpha, beta;
} FsOzProblem;

typedef struct FsOzTile {
    int32_t problem;
    int32_t tm;            /* 128-row tile index of C                         */
    int32_t tn;            /* 256-column tile index of C                      */
    int32_t pad;
} FsOzTile;

/* Tile geometry of the tcgen05 kernel (M tile, N tile, K bytes per stage,
 * rows per slice tile). */
int fs_ozaki_geometry(int32_t* tile_m, int32_t* tile_n, int32_t* tile_k,
                      int32_t* split_rows);

/* Exponents and digit slices of every operand (grid.y = operand, <= 65535). */
int fs_ozaki_split(const FsOzOperand* d_ops, int64_t n_ops, int32_t max_rows,
                   int32_t max_tiles, int32_t nslices, void* stream);

/*
 * The mixed-precision replacement of fs_grouped_dgemm for the same call sites
 * (symmetric_tensor.py:453-489, ctm_renormalize.py:92-94, 122-123).
 * chunk_ktiles bounds the k-tiles accumulated in int32 before conversion:
 * nslices * chunk_ktiles * 128 * 127^2 must stay below 2^31.  A bounded wait
 * that runs out writes FS_ERR_TIMEOUT to d_flag (if not null).
 */
int fs_ozaki_gemm(const FsOzProblem* d_probs, int64_t n_probs,
                  const FsOzTile* d_tiles, int64_t n_tiles, int32_t nslices,
                  int32_t chunk_ktiles, int32_t* d_flag, void* stream);

/*
 * The same GEMM on 256 x 256 output tiles computed by clusters of two CTAs
 * (tcgen05.mma.cta_group::2, each CTA loading half of every operand stage by
 * TMA through a tensor map over the workspace).  Tiles index 256-row blocks
 * of C (tm) and 256-column blocks (tn); every problem listed in d_tiles must
 * have an even a_rowtiles.  d_workspace / workspace_bytes: the buffer holding
 * every problem's slices (128-byte aligned, a multiple of 128 bytes).
 */
int fs_ozaki_gemm_pair(const FsOzProblem* d_probs, int64_t n_probs,
                       const FsOzTile* d_tiles, int64_t n_tiles, int32_t nslices,
                       int32_t chunk_ktiles, const void* d_workspace,
                       int64_t workspace_bytes, int32_t* d_flag, void* stream);

/* ----------------------------- Ozaki II: CRT over int8 moduli on tcgen05 */
/*
 * FP64-class GEMM with one int8 tensor-core product per modulus (the
 * integer-modular "Ozaki scheme II", Ozaki, Uchino and Imamura 2025): each row
 * i of op(A) is scaled by 2^(a - e_i) and rounded to an integer (|A'| <= 2^a,
 * e_i the frexp exponent of the row maximum), each column j of op(B) by
 * 2^(b - f_j); the exact integer product X = A'B' (|X| <= K 2^(a+b) <= P/4,
 * P the product of the nmod pairwise coprime moduli 256, 255, 253, 251, 247,
 * 241, 239, 233, 229, 227, 223, 217, 211, 199) is rebuilt from its residues
 * by the Chinese remainder theorem in exact FP64 arithmetic, and
 * C = alpha X 2^(e_i + f_j - a - b) + beta C.  Relative error per entry is
 * ~2^-min(a, b) of the product of the row/column maxima; fs_ozaki2_bits gives
 * a and b for a modulus count and K (14 moduli, K = 2048: a = 48, b = 49).
 * Non-finite inputs are not supported.
 *
 * Operands use the slice layout of the digit form: nmod residue slices of
 * rowtiles x ktiles tiles of 128 rows x 128 bytes (128-byte swizzled, K-major),
 * B stored transposed; every problem needs an even a_rowtiles (256-row tiles on
 * CTA pairs) and K <= FS_OZAKI2_MAX_K (exact int32 residue products).
 */
#define FS_OZAKI2_MIN_MODULI 8
#define FS_OZAKI2_MAX_MODULI 14
#define FS_OZAKI2_MAX_K 131071

typedef struct FsOz2Operand {
    const double* src;     /* element (row, k) at src[row*s_row + k*s_k]      */
    int64_t s_row, s_k;
    int8_t* slices;        /* nmod*ktiles*rowtiles*16384 bytes                */
    int32_t* exps;         /* rows entries                                    */
    int32_t rows, K;
    int32_t rowtiles, ktiles;
    int32_t bits;          /* a for op(A), b for op(B)                        */
    int32_t pad;
} FsOz2Operand;

typedef struct FsOz2Problem {
    const int8_t* a_slices;
    const int8_t* b_slices;
    const int32_t* a_exps;
    const int32_t* b_exps;
    double* C;             /* row-major M x N, leading dimension ldc          */
    int64_t ldc;
    int32_t M, N, K;
    int32_t a_rowtiles, b_rowtiles, ktiles;
    double alpha, beta;
    int32_t a_bits, b_bits;
} FsOz2Problem;

/* Operand bits a, b for nmod moduli and inner dimension K. */
int fs_ozaki2_bits(int32_t nmod, int64_t K, int32_t* a_bits, int32_t* b_bits);

/*
 * The CRT constants the kernels use, for checking: the moduli, the weights
 * W_m = (P/p_m) ((P/p_m)^-1 mod p_m) split into two doubles on the grids
 * 2^grids[0] and 2^grids[1] (weights_hi, weights_lo; the remainder below
 * 2^grids[1] is dropped), P split the same way (modulus_product[0..1]) and
 * frac[m] = ((P/p_m)^-1 mod p_m) / p_m in FP32.  Host arrays of nmod entries.
 */
int fs_ozaki2_constants(int32_t nmod, int32_t* moduli, double* weights_hi,
                        double* weights_lo, double* modulus_product, float* frac,
                        int32_t* grids);

/* Bytes of CRT scratch fs_ozaki2_gemm_pair needs (every CTA parks nmod
 * residue bytes per entry of its 128 x 256 tile half). */
int fs_ozaki2_scratch_bytes(int32_t nmod, int64_t* bytes);

/* Row exponents and residue slices of every operand (grid.y = operand,
 * <= 65535); max_units = the largest rowtiles * 4 * ktiles. */
int fs_ozaki2_split(const FsOz2Operand* d_ops, int64_t n_ops, int32_t max_rows,
                    int64_t max_units, int32_t nmod, void* stream);

/*
 * The Ozaki II replacement of fs_grouped_dgemm for the same call sites
 * (symmetric_tensor.py:453-489, ctm_renormalize.py:92-94, 122-123): 256 x 256
 * output tiles on CTA pairs (tcgen05.mma.cta_group::2 kind::i8), one TMEM
 * accumulation per modulus, the residue reduction and the CRT in the epilogue.
 * d_workspace holds every problem's slices (as for fs_ozaki_gemm_pair);
 * d_scratch (fs_ozaki2_scratch_bytes, 16-byte aligned) the parked residues.
 * A bounded wait that runs out writes FS_ERR_TIMEOUT to d_flag (if not null);
 * a problem with K > FS_OZAKI2_MAX_K is skipped with FS_ERR_UNSUPPORTED there.
 */
int fs_ozaki2_gemm_pair(const FsOz2Problem* d_probs, int64_t n_probs,
                        const FsOzTile* d_tiles, int64_t n_tiles, int32_t nmod,
                        const void* d_workspace, int64_t workspace_bytes, void* d_scratch,
                        int64_t scratch_bytes, int32_t* d_flag, void* stream);

/*
 * Grouped Ozaki GEMM that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: a host application whose own
 * pool already reserved the device (a cudaMalloc from a library inside it
 * would fail or fragment that pool), or a C / Fortran driver without a device
 * allocator that only holds its input and output buffers.  The caller passes
 * the problems as a HOST array of FsGemmProblem (same meaning as for
 * fs_grouped_dgemm; A, B and C are device pointers).  Digit slices, exponents,
 * launch tables and a status word go to a fixed 48 MiB file-scope device array
 * inside this library, which every GPU that loads the library holds until the
 * process exits; requests that do not fit return FS_ERR_TOO_LARGE before any
 * GPU work (one 1024^3 product with 7 slices needs about 15 MiB).
 *
 * The first call on a device looks up the array's device address (with that
 * device current).  The call copies its launch tables from host memory with
 * cudaMemcpyAsync and calls no cudaMalloc, cudaFree or allocating library
 * routine.  It must not be called while `stream` is being captured into a CUDA
 * graph (the staged host tables do not outlive the call): it returns
 * FS_ERR_UNSUPPORTED then.  All calls on a device share that device's array and
 * every call rewrites what it reads, so calls that overlap on the GPU (for
 * example on two streams of the same device) race; serialise them.
 *
 * A bounded device wait that runs out ends the kernel early and leaves C
 * partly written; it is reported through fs_ozaki_noalloc_status.
 */
int fs_ozaki_gemm_noalloc(const FsGemmProblem* h_problems, int64_t n_problems,
                          int32_t nslices, void* stream);

/*
 * Status of the last fs_ozaki_gemm_noalloc call on the current device: waits
 * for `stream` to finish, then copies the status word of the fixed array to
 * *status (FS_OK, or FS_ERR_TIMEOUT when a bounded device wait ran out).
 * Allocates nothing.  No counterpart in the reference.
 */
int fs_ozaki_noalloc_status(void* stream, int32_t* status);

/* -------------------------------------------------------------- block ops */
/* x[0:n] *= alpha.  Replaces SymmetricTensor.__imul__/__itruediv__
 * (symmetric_tensor.py:441-451) and scalar __mul__ (:377-424). */
int fs_scale(double* d_x, int64_t n, double alpha, void* stream);

/* x[0:n] *= s (invert == 0) or x[0:n] /= s (invert != 0) with s = d_scalar[0]
 * read on the device: normalisation by a device-computed norm without a host
 * round trip (the `t /= t.norm()` steps of ctm_renormalize.py:165, :192, :215). */
int fs_scale_by(double* d_x, int64_t n, const double* d_scalar, int32_t invert,
                void* stream);

/* y[0:n] = a*x + b*y.  Replaces the block sums of __add__/__sub__
 * (symmetric_tensor.py:326-352). */
int fs_axpby(const double* d_x, double* d_y, int64_t n, double a, double b,
             void* stream);

/*
 * Weighted reductions over block lists.  A segment is a contiguous run of the
 * buffer with a weight (the irrep dimension).
 */
typedef struct FsSegment {
    int64_t offset;
    int64_t length;
    double weight;
} FsSegment;

/*
 * out[0] = sum_s weight_s * sum_i x[offset_s + i]^2, the squared Frobenius
 * norm SymmetricTensor.norm computes (symmetric_tensor.py:624-631) and
 * DiagonalTensor.norm (diagonal_tensor.py:201-205).  d_partial is caller
 * scratch of n_partial >= fs_reduce_partials() doubles.
 */
int fs_reduce_partials(void);
int fs_weighted_sumsq(const double* d_x, const FsSegment* d_segs, int64_t n_segs,
                      double* d_partial, int64_t n_partial, double* d_out,
                      void* stream);

/* out[0] = sum_s weight_s * sum_i x[offset_s + i]  (DiagonalTensor.sum,
 * diagonal_tensor.py:195-199). Same scratch contract as fs_weighted_sumsq. */
int fs_weighted_sum(const double* d_x, const FsSegment* d_segs, int64_t n_segs,
                    double* d_partial, int64_t n_partial, double* d_out,
                    void* stream);

/*
 * Pairwise block contraction: out[0] = sum_p weight_p * sum_{ij} A_p[i,j] B_p[j,i]
 * (full_contract, symmetric_tensor.py:639-653) or, with b == NULL entries,
 * sum_p weight_p * sum_i A_p[i,i] (trace, :633-637).  a_trans / b_trans mark
 * F-order blocks.
 */
typedef struct FsPairBlock {
    int64_t a_off, b_off;   /* b_off < 0: trace of A */
    int32_t m, n;           /* logical shape of A_p  */
    int32_t a_trans, b_trans;
    double weight;
} FsPairBlock;

int fs_pair_contract(const double* d_a, const double* d_b,
                     const FsPairBlock* d_pairs, int64_t n_pairs,
                     double* d_partial, int64_t n_partial, double* d_out,
                     void* stream);

/*
 * Diagonal scaling of blocks by 1-D weight vectors: out_b[i,j] = x_b[i,j] * d[j]
 * (right) or d[i] (left).  Replaces SymmetricTensor._diagonal_mul
 * (symmetric_tensor.py:1189-1248).  x may be F-order (x_trans); out is C-order.
 */
typedef struct FsDiagBlock {
    int64_t x_off, out_off, d_off;
    int32_t m, n;
    int32_t x_trans, left;
} FsDiagBlock;

int fs_diag_mul(const double* d_x, const double* d_diag, double* d_out,
                const FsDiagBlock* d_blocks, int64_t n_blocks, void* stream);

/* Elementwise power of a weight vector, y = x^p, with p = -1, -0.5, 0.5 and
 * 2 exact special cases (DiagonalTensor.__pow__, diagonal_tensor.py:133-143). */
int fs_pow(const double* d_x, double* d_y, int64_t n, double p, void* stream);

/*
 * O(2) <-> U(1) change of basis of symmetric-tensor blocks, replacing the
 * reference's Sz-reflection and 0odd / 0even loops
 * (frostspin/symmetric_tensor/o2_symmetric_tensor.py: _generate_neg_sz_blocks
 * :798-851 with _numba_generate_refl_block :327-354, _numba_merge_b0oe
 * :269-288, _numba_split_b0 :291-310; used by toU1 :682-733, from_U1 :650-675,
 * _permute_data :853-936 and _transpose_data :938-942).
 *
 * Output block b (C-order, nrows x ncols at d_out + out_off) gets
 *   out[i, j] = sum_t (coef[rcoef_off + i] * src[p_t(i, j)]) * coef[ccoef_off + j],
 *   p_t(i, j) = src_off + index[ridx_off + i] * rs + index[cidx_off + j] * cs,
 * summed over its nterms (<= FS_O2_MAXTERMS) terms in order, each product
 * rounded separately.  Source and output positions outside [0, src_len) /
 * [0, out_len) are skipped and reported in *d_flag (FS_ERR_BOUNDS, if d_flag
 * is not null); the host tables are validated before the call.  max_rows is
 * the largest nrows; at most 65535 blocks per call.
 */
#define FS_O2_MAXTERMS 4

typedef struct FsO2Term {
    int64_t src_off;
    int64_t rs, cs;                  /* source row / column strides (elements) */
    int64_t ridx_off, cidx_off;      /* into the index table                   */
    int64_t rcoef_off, ccoef_off;    /* into the coefficient table             */
} FsO2Term;

typedef struct FsO2Block {
    int64_t out_off;
    int64_t nrows, ncols;
    int32_t nterms;
    int32_t pad;
    FsO2Term terms[FS_O2_MAXTERMS];
} FsO2Block;

int fs_o2_recombine(const double* d_src, int64_t src_len, double* d_out, int64_t out_len,
                    const FsO2Block* d_blocks, int64_t n_blocks, const int64_t* d_index,
                    const double* d_coef, int64_t max_rows, int32_t* d_flag, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FROSTSPIN_B200_H */
