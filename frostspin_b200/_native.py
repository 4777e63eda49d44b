"""ctypes binding of the frostspin_b200 C ABI (include/frostspin_b200.h).

The shared library is built in-tree by ``frostspin_b200.build``.  There is no
fallback: if the library is missing or a CUDA device is absent, every device
operation raises.  Plan tables are numpy structured arrays whose dtypes mirror
the C structs byte for byte (checked by tests/test_abi.py against the header
compiled with gcc); they are uploaded once into torch-owned device buffers.
"""

import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(__file__), "_lib", "libfrostspin_b200.so")

FS_OK = 0
FS_PERM_MAXR = 8

# ----------------------------------------------------------------- C struct dtypes
PERM_EB_DTYPE = np.dtype(
    [
        ("obase", "<i8"),
        ("nbase", "<i8"),
        ("ostride", "<i8", (FS_PERM_MAXR,)),
        ("nstride", "<i8", (FS_PERM_MAXR,)),
        ("dims", "<u4", (FS_PERM_MAXR,)),
        ("divm", "<u4", (FS_PERM_MAXR,)),
        ("divs", "<u4", (FS_PERM_MAXR,)),
        ("ndim", "<i4"),
        ("volume", "<u4"),
        ("tile_leg", "<i4"),
        ("pad", "<i4"),
    ]
)

PERM_BUFFERS_DTYPE = np.dtype(
    [("in", "<u8"), ("in_len", "<i8"), ("out", "<u8"), ("out_len", "<i8")]
)

PERM_TASK_DTYPE = np.dtype(
    [("eb", "<i4"), ("start", "<u4"), ("count", "<u4"), ("pad", "<u4")]
)

FS_SU2_MAXD = 8

SU2_GROUP_DTYPE = np.dtype(
    [
        ("u_off", "<i8"),
        ("ncols", "<i8"),
        ("dims", "<u4", (FS_SU2_MAXD,)),
        ("divm", "<u4", (FS_SU2_MAXD,)),
        ("divs", "<u4", (FS_SU2_MAXD,)),
        ("ndim", "<i4"),
        ("M", "<i4"),
        ("K", "<i4"),
        ("in_first", "<i4"),
        ("in_count", "<i4"),
        ("out_first", "<i4"),
        ("out_count", "<i4"),
        ("pad", "<i4"),
    ]
)

SU2_PIECE_DTYPE = np.dtype(
    [
        ("base", "<i8"),
        ("sr_stride", "<i8"),
        ("sc_stride", "<i8"),
        ("ext", "<i8", (FS_SU2_MAXD,)),
        ("sr", "<i4"),
        ("sc", "<i4"),
        ("row0", "<i4"),
        ("pad", "<i4"),
    ]
)

GEMM_PROBLEM_DTYPE = np.dtype(
    [
        ("A", "<u8"),
        ("B", "<u8"),
        ("C", "<u8"),
        ("lda", "<i8"),
        ("ldb", "<i8"),
        ("ldc", "<i8"),
        ("M", "<i4"),
        ("N", "<i4"),
        ("K", "<i4"),
        ("transA", "<i4"),
        ("transB", "<i4"),
        ("pad", "<i4"),
        ("alpha", "<f8"),
        ("beta", "<f8"),
    ]
)

GEMM_TILE_DTYPE = np.dtype(
    [("problem", "<i4"), ("tm", "<i4"), ("tn", "<i4"), ("pad", "<i4")]
)

TILE_RUN_DTYPE = np.dtype([("start", "<i8"), ("problem", "<i4"), ("ncol", "<i4"),
                           ("nrow", "<i4"), ("col_major", "<i4")])

SPLIT_REDUCE_DTYPE = np.dtype(
    [
        ("W", "<u8"),
        ("C", "<u8"),
        ("ldc", "<i8"),
        ("slice", "<i8"),
        ("nslices", "<i4"),
        ("M", "<i4"),
        ("N", "<i4"),
        ("pad", "<i4"),
        ("alpha", "<f8"),
        ("beta", "<f8"),
    ]
)

OZ_OPERAND_DTYPE = np.dtype(
    [
        ("src", "<u8"),
        ("s_row", "<i8"),
        ("s_k", "<i8"),
        ("slices", "<u8"),
        ("exps", "<u8"),
        ("rows", "<i4"),
        ("K", "<i4"),
        ("rowtiles", "<i4"),
        ("ktiles", "<i4"),
    ]
)

OZ_PROBLEM_DTYPE = np.dtype(
    [
        ("a_slices", "<u8"),
        ("b_slices", "<u8"),
        ("a_exps", "<u8"),
        ("b_exps", "<u8"),
        ("C", "<u8"),
        ("ldc", "<i8"),
        ("M", "<i4"),
        ("N", "<i4"),
        ("K", "<i4"),
        ("a_rowtiles", "<i4"),
        ("b_rowtiles", "<i4"),
        ("ktiles", "<i4"),
        ("alpha", "<f8"),
        ("beta", "<f8"),
    ]
)

OZ_TILE_DTYPE = np.dtype([("problem", "<i4"), ("tm", "<i4"), ("tn", "<i4"), ("pad", "<i4")])

FS_OZAKI_MAX_SLICES = 8

OZ2_OPERAND_DTYPE = np.dtype(
    [
        ("src", "<u8"),
        ("s_row", "<i8"),
        ("s_k", "<i8"),
        ("slices", "<u8"),
        ("exps", "<u8"),
        ("rows", "<i4"),
        ("K", "<i4"),
        ("rowtiles", "<i4"),
        ("ktiles", "<i4"),
        ("bits", "<i4"),
        ("pad", "<i4"),
    ]
)

OZ2_PROBLEM_DTYPE = np.dtype(
    [
        ("a_slices", "<u8"),
        ("b_slices", "<u8"),
        ("a_exps", "<u8"),
        ("b_exps", "<u8"),
        ("C", "<u8"),
        ("ldc", "<i8"),
        ("M", "<i4"),
        ("N", "<i4"),
        ("K", "<i4"),
        ("a_rowtiles", "<i4"),
        ("b_rowtiles", "<i4"),
        ("ktiles", "<i4"),
        ("alpha", "<f8"),
        ("beta", "<f8"),
        ("a_bits", "<i4"),
        ("b_bits", "<i4"),
    ]
)

FS_OZAKI2_MIN_MODULI = 8
FS_OZAKI2_MAX_MODULI = 14
FS_OZAKI2_MAX_K = 131071

SEGMENT_DTYPE = np.dtype([("offset", "<i8"), ("length", "<i8"), ("weight", "<f8")])

PAIR_BLOCK_DTYPE = np.dtype(
    [
        ("a_off", "<i8"),
        ("b_off", "<i8"),
        ("m", "<i4"),
        ("n", "<i4"),
        ("a_trans", "<i4"),
        ("b_trans", "<i4"),
        ("weight", "<f8"),
    ]
)

FS_O2_MAXTERMS = 4

O2_TERM_DTYPE = np.dtype(
    [
        ("src_off", "<i8"),
        ("rs", "<i8"),
        ("cs", "<i8"),
        ("ridx_off", "<i8"),
        ("cidx_off", "<i8"),
        ("rcoef_off", "<i8"),
        ("ccoef_off", "<i8"),
    ]
)

O2_BLOCK_DTYPE = np.dtype(
    [
        ("out_off", "<i8"),
        ("nrows", "<i8"),
        ("ncols", "<i8"),
        ("nterms", "<i4"),
        ("pad", "<i4"),
        ("terms", O2_TERM_DTYPE, (FS_O2_MAXTERMS,)),
    ]
)

DIAG_BLOCK_DTYPE = np.dtype(
    [
        ("x_off", "<i8"),
        ("out_off", "<i8"),
        ("d_off", "<i8"),
        ("m", "<i4"),
        ("n", "<i4"),
        ("x_trans", "<i4"),
        ("left", "<i4"),
    ]
)

# name -> (restype, argtypes); pointers and streams travel as c_void_p
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_D = ctypes.c_double
SIGNATURES = {
    "fs_version": (ctypes.c_int, []),
    "fs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "fs_last_cuda_error": (ctypes.c_char_p, []),
    "fs_abelian_permute": (
        ctypes.c_int,
        [_P, _I64, _P, _I64, _P, _I64, _P, _I64, _P, _P],
    ),
    "fs_abelian_permute_multi": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _I64, _P, _P]),
    "fs_su2_fused_limits": (ctypes.c_int, [_P, _P, _P]),
    "fs_su2_permute_fused": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _I64, _P, _I64, _P, _I64,
                                            _P, _I64, _P, _P]),
    "fs_dgemm_tile_shape": (ctypes.c_int, [_P, _P]),
    "fs_grouped_dgemm": (ctypes.c_int, [_P, _I64, _P, _I64, _P]),
    "fs_thin_dgemm_shape": (ctypes.c_int, [_P, _P, _P]),
    "fs_grouped_dgemm_thin": (ctypes.c_int, [_P, _I64, _P, _I64, _P]),
    "fs_grouped_dgemm_uniform": (ctypes.c_int, [_P, _I64, _P, _I64, _I32, _I32, _P]),
    "fs_splitk_reduce": (ctypes.c_int, [_P, _I64, _I64, _P]),
    "fs_expand_tiles": (ctypes.c_int, [_P, _I64, _I64, _P, _P]),
    "fs_ozaki_geometry": (ctypes.c_int, [_P, _P, _P, _P]),
    "fs_ozaki_split": (ctypes.c_int, [_P, _I64, _I32, _I32, _I32, _P]),
    "fs_ozaki_gemm": (ctypes.c_int, [_P, _I64, _P, _I64, _I32, _I32, _P, _P]),
    "fs_ozaki_gemm_pair": (ctypes.c_int, [_P, _I64, _P, _I64, _I32, _I32, _P, _I64, _P, _P]),
    "fs_ozaki2_bits": (ctypes.c_int, [_I32, _I64, _P, _P]),
    "fs_ozaki2_constants": (ctypes.c_int, [_I32, _P, _P, _P, _P, _P, _P]),
    "fs_ozaki2_scratch_bytes": (ctypes.c_int, [_I32, _P]),
    "fs_ozaki2_split": (ctypes.c_int, [_P, _I64, _I32, _I64, _I32, _P]),
    "fs_ozaki2_gemm_pair": (ctypes.c_int, [_P, _I64, _P, _I64, _I32, _P, _I64, _P, _I64, _P, _P]),
    "fs_ozaki_gemm_noalloc": (ctypes.c_int, [_P, _I64, _I32, _P]),
    "fs_ozaki_noalloc_status": (ctypes.c_int, [_P, _P]),
    "fs_set_spin_limit": (ctypes.c_int64, [_I64]),
    "fs_scale": (ctypes.c_int, [_P, _I64, _D, _P]),
    "fs_axpby": (ctypes.c_int, [_P, _P, _I64, _D, _D, _P]),
    "fs_scale_by": (ctypes.c_int, [_P, _I64, _P, _I32, _P]),
    "fs_pow": (ctypes.c_int, [_P, _P, _I64, _D, _P]),
    "fs_reduce_partials": (ctypes.c_int, []),
    "fs_weighted_sumsq": (ctypes.c_int, [_P, _P, _I64, _P, _I64, _P, _P]),
    "fs_weighted_sum": (ctypes.c_int, [_P, _P, _I64, _P, _I64, _P, _P]),
    "fs_pair_contract": (ctypes.c_int, [_P, _P, _P, _I64, _P, _I64, _P, _P]),
    "fs_diag_mul": (ctypes.c_int, [_P, _P, _P, _P, _I64, _P]),
    "fs_o2_recombine": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _I64, _P, _P, _I64, _P, _P]),
}

_lib = None


class NativeError(RuntimeError):
    """A frostspin_b200 C ABI call returned a non-zero status."""


def lib():
    """Load the shared library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            msg = (
                f"frostspin_b200 CUDA library not found at {LIB_PATH}; build it with "
                "`python -m frostspin_b200.build`"
            )
            raise NativeError(msg)
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status, what):
    if status != FS_OK:
        text = lib().fs_status_string(status).decode()
        cuda = lib().fs_last_cuda_error().decode()
        msg = f"{what} failed: status {status} ({text}); last CUDA error: {cuda}"
        raise NativeError(msg)


# number of calls per entry point (bench.py reports the kernel launches of its
# timed region from these counters)
CALL_COUNTS = {}

# kernels each entry point launches
LAUNCHES_PER_CALL = {
    "fs_abelian_permute": 1, "fs_abelian_permute_multi": 1, "fs_su2_permute_fused": 1, "fs_grouped_dgemm": 1, "fs_grouped_dgemm_thin": 1,
    "fs_grouped_dgemm_uniform": 1, "fs_splitk_reduce": 1, "fs_expand_tiles": 1, "fs_ozaki_split": 2,
    "fs_ozaki_gemm": 1, "fs_ozaki_gemm_pair": 1, "fs_ozaki2_split": 2, "fs_ozaki2_gemm_pair": 1,
    "fs_scale": 1, "fs_scale_by": 1, "fs_axpby": 1, "fs_pow": 1, "fs_weighted_sumsq": 2,
    "fs_weighted_sum": 2, "fs_pair_contract": 2, "fs_diag_mul": 1, "fs_o2_recombine": 1,
}


def kernel_launches():
    return sum(LAUNCHES_PER_CALL.get(k, 0) * v for k, v in CALL_COUNTS.items())


def call(name, *args):
    """Call a C ABI function by name and raise on a non-zero status."""
    st = getattr(lib(), name)(*args)
    check(st, name)
    CALL_COUNTS[name] = CALL_COUNTS.get(name, 0) + 1
    return st


def reduce_partials():
    return int(lib().fs_reduce_partials())


def dgemm_tile_shape():
    tm = ctypes.c_int32()
    tn = ctypes.c_int32()
    call("fs_dgemm_tile_shape", ctypes.byref(tm), ctypes.byref(tn))
    return tm.value, tn.value


def thin_dgemm_shape():
    mm = ctypes.c_int32()
    mk = ctypes.c_int32()
    tn = ctypes.c_int32()
    call("fs_thin_dgemm_shape", ctypes.byref(mm), ctypes.byref(mk), ctypes.byref(tn))
    return mm.value, mk.value, tn.value


def ozaki2_bits(nmod, K):
    """(a, b): operand bits the library uses for nmod moduli and inner size K."""
    a = ctypes.c_int32()
    b = ctypes.c_int32()
    call("fs_ozaki2_bits", nmod, int(K), ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def ozaki2_constants(nmod):
    """The library's CRT constants (for checking against an exact computation)."""
    moduli = np.zeros(nmod, dtype=np.int32)
    w1 = np.zeros(nmod)
    w2 = np.zeros(nmod)
    pp = np.zeros(2)
    frac = np.zeros(nmod, dtype=np.float32)
    grids = np.zeros(2, dtype=np.int32)
    call("fs_ozaki2_constants", nmod, moduli.ctypes.data, w1.ctypes.data, w2.ctypes.data,
         pp.ctypes.data, frac.ctypes.data, grids.ctypes.data)
    return {"moduli": moduli, "w1": w1, "w2": w2, "P": pp, "frac": frac, "grids": grids}


def ozaki2_scratch_bytes(nmod):
    n = ctypes.c_int64()
    call("fs_ozaki2_scratch_bytes", nmod, ctypes.byref(n))
    return n.value


def su2_fused_limits():
    """(max rows M = K, max pieces per side, threads per CTA) of the fused
    SU(2) permute kernel."""
    a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    call("fs_su2_fused_limits", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value
