"""The C-ABI library loads, exports every declared entry point, and its struct
layouts match the numpy dtypes the host uses to build plan tables."""

import os
import re
import subprocess

import numpy as np
import pytest

from frostspin_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "include")


def declared_functions():
    names = []
    for f in sorted(os.listdir(HEADER_DIR)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(fs_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_loads_and_exports_all_symbols():
    lib = _native.lib()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_status_strings():
    lib = _native.lib()
    assert lib.fs_version() >= 10000
    assert lib.fs_status_string(0) == b"ok"
    assert lib.fs_status_string(-3).startswith(b"plan entry")


def test_invalid_arguments_rejected_without_gpu_work():
    # negative sizes are rejected on the host before any launch
    lib = _native.lib()
    assert lib.fs_scale(None, -1, 1.0, None) == -1
    assert lib.fs_grouped_dgemm(None, 0, None, -5, None) == -1
    assert lib.fs_abelian_permute(None, 0, None, 0, None, 0, None, -1, None, None) == -1
    assert lib.fs_expand_tiles(None, -1, 4, None, None) == -1
    assert lib.fs_expand_tiles(None, 0, 4, None, None) == -1
    assert lib.fs_expand_tiles(None, 0, 0, None, None) == 0
    # zero work is a no-op success
    assert lib.fs_scale(None, 0, 1.0, None) == 0


LAYOUT_PROGRAM = r"""
#include <stddef.h>
#include <stdio.h>
#include "frostspin_b200.h"
#define F(T, f) printf("%s %s %zu\n", #T, #f, offsetof(T, f));
#define S(T) printf("%s __size__ %zu\n", #T, sizeof(T));
int main(void) {
  S(FsPermEB) F(FsPermEB, obase) F(FsPermEB, nbase) F(FsPermEB, ostride)
  F(FsPermEB, nstride) F(FsPermEB, dims) F(FsPermEB, divm) F(FsPermEB, divs)
  F(FsPermEB, ndim) F(FsPermEB, volume) F(FsPermEB, tile_leg)
  S(FsPermTask) F(FsPermTask, eb) F(FsPermTask, start) F(FsPermTask, count)
  S(FsPermBuffers) F(FsPermBuffers, in) F(FsPermBuffers, in_len) F(FsPermBuffers, out)
  F(FsPermBuffers, out_len)
  S(FsGemmProblem) F(FsGemmProblem, A) F(FsGemmProblem, B) F(FsGemmProblem, C)
  F(FsGemmProblem, lda) F(FsGemmProblem, ldb) F(FsGemmProblem, ldc)
  F(FsGemmProblem, M) F(FsGemmProblem, N) F(FsGemmProblem, K)
  F(FsGemmProblem, transA) F(FsGemmProblem, transB)
  F(FsGemmProblem, alpha) F(FsGemmProblem, beta)
  S(FsGemmTile) F(FsGemmTile, problem) F(FsGemmTile, tm) F(FsGemmTile, tn)
  S(FsSegment) F(FsSegment, offset) F(FsSegment, length) F(FsSegment, weight)
  S(FsPairBlock) F(FsPairBlock, a_off) F(FsPairBlock, b_off) F(FsPairBlock, m)
  F(FsPairBlock, n) F(FsPairBlock, a_trans) F(FsPairBlock, b_trans)
  F(FsPairBlock, weight)
  S(FsDiagBlock) F(FsDiagBlock, x_off) F(FsDiagBlock, out_off) F(FsDiagBlock, d_off)
  F(FsDiagBlock, m) F(FsDiagBlock, n) F(FsDiagBlock, x_trans) F(FsDiagBlock, left)
  S(FsOzOperand) F(FsOzOperand, src) F(FsOzOperand, s_row) F(FsOzOperand, s_k)
  F(FsOzOperand, slices) F(FsOzOperand, exps) F(FsOzOperand, rows) F(FsOzOperand, K)
  F(FsOzOperand, rowtiles) F(FsOzOperand, ktiles)
  S(FsOzProblem) F(FsOzProblem, a_slices) F(FsOzProblem, b_slices) F(FsOzProblem, a_exps)
  F(FsOzProblem, b_exps) F(FsOzProblem, C) F(FsOzProblem, ldc) F(FsOzProblem, M)
  F(FsOzProblem, N) F(FsOzProblem, K) F(FsOzProblem, a_rowtiles) F(FsOzProblem, b_rowtiles)
  F(FsOzProblem, ktiles) F(FsOzProblem, alpha) F(FsOzProblem, beta)
  S(FsOzTile) F(FsOzTile, problem) F(FsOzTile, tm) F(FsOzTile, tn)
  S(FsSu2Group) F(FsSu2Group, u_off) F(FsSu2Group, ncols) F(FsSu2Group, dims)
  F(FsSu2Group, divm) F(FsSu2Group, divs) F(FsSu2Group, ndim) F(FsSu2Group, M)
  F(FsSu2Group, K) F(FsSu2Group, in_first) F(FsSu2Group, in_count)
  F(FsSu2Group, out_first) F(FsSu2Group, out_count)
  S(FsSu2Piece) F(FsSu2Piece, base) F(FsSu2Piece, sr_stride) F(FsSu2Piece, sc_stride)
  F(FsSu2Piece, ext) F(FsSu2Piece, sr) F(FsSu2Piece, sc) F(FsSu2Piece, row0)
  S(FsOz2Operand) F(FsOz2Operand, src) F(FsOz2Operand, s_row) F(FsOz2Operand, s_k)
  F(FsOz2Operand, slices) F(FsOz2Operand, exps) F(FsOz2Operand, rows) F(FsOz2Operand, K)
  F(FsOz2Operand, rowtiles) F(FsOz2Operand, ktiles) F(FsOz2Operand, bits)
  S(FsOz2Problem) F(FsOz2Problem, a_slices) F(FsOz2Problem, b_slices)
  F(FsOz2Problem, a_exps) F(FsOz2Problem, b_exps) F(FsOz2Problem, C) F(FsOz2Problem, ldc)
  F(FsOz2Problem, M) F(FsOz2Problem, N) F(FsOz2Problem, K) F(FsOz2Problem, a_rowtiles)
  F(FsOz2Problem, b_rowtiles) F(FsOz2Problem, ktiles) F(FsOz2Problem, alpha)
  F(FsOz2Problem, beta) F(FsOz2Problem, a_bits) F(FsOz2Problem, b_bits)
  S(FsSplitReduce) F(FsSplitReduce, W) F(FsSplitReduce, C) F(FsSplitReduce, ldc)
  F(FsSplitReduce, slice) F(FsSplitReduce, nslices) F(FsSplitReduce, M)
  F(FsSplitReduce, N) F(FsSplitReduce, alpha) F(FsSplitReduce, beta)
  S(FsTileRun) F(FsTileRun, start) F(FsTileRun, problem) F(FsTileRun, ncol)
  F(FsTileRun, nrow) F(FsTileRun, col_major)
  S(FsO2Term) F(FsO2Term, src_off) F(FsO2Term, rs) F(FsO2Term, cs) F(FsO2Term, ridx_off)
  F(FsO2Term, cidx_off) F(FsO2Term, rcoef_off) F(FsO2Term, ccoef_off)
  S(FsO2Block) F(FsO2Block, out_off) F(FsO2Block, nrows) F(FsO2Block, ncols)
  F(FsO2Block, nterms) F(FsO2Block, terms)
  return 0;
}
"""

DTYPES = {
    "FsPermEB": _native.PERM_EB_DTYPE,
    "FsPermTask": _native.PERM_TASK_DTYPE,
    "FsPermBuffers": _native.PERM_BUFFERS_DTYPE,
    "FsGemmProblem": _native.GEMM_PROBLEM_DTYPE,
    "FsGemmTile": _native.GEMM_TILE_DTYPE,
    "FsSegment": _native.SEGMENT_DTYPE,
    "FsPairBlock": _native.PAIR_BLOCK_DTYPE,
    "FsDiagBlock": _native.DIAG_BLOCK_DTYPE,
    "FsOzOperand": _native.OZ_OPERAND_DTYPE,
    "FsOzProblem": _native.OZ_PROBLEM_DTYPE,
    "FsOzTile": _native.OZ_TILE_DTYPE,
    "FsSu2Group": _native.SU2_GROUP_DTYPE,
    "FsSu2Piece": _native.SU2_PIECE_DTYPE,
    "FsOz2Operand": _native.OZ2_OPERAND_DTYPE,
    "FsOz2Problem": _native.OZ2_PROBLEM_DTYPE,
    "FsSplitReduce": _native.SPLIT_REDUCE_DTYPE,
    "FsTileRun": _native.TILE_RUN_DTYPE,
    "FsO2Term": _native.O2_TERM_DTYPE,
    "FsO2Block": _native.O2_BLOCK_DTYPE,
}


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text(LAYOUT_PROGRAM)
    try:
        subprocess.run(
            ["gcc", "-std=c11", "-I", HEADER_DIR, str(src), "-o", str(exe)],
            check=True, capture_output=True,
        )
    except FileNotFoundError:
        pytest.skip("gcc not available")
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    seen = set()
    for line in out.strip().splitlines():
        struct, field, value = line.split()
        dt = DTYPES[struct]
        if field == "__size__":
            assert dt.itemsize == int(value), struct
        else:
            assert dt.fields[field][1] == int(value), (struct, field)
        seen.add(struct)
    assert seen == set(DTYPES)


def test_magic_division_exact():
    from frostspin_b200.symmetric_tensor.abelian_plan import magic_divisor

    rng = np.random.default_rng(0)
    ds = np.concatenate([np.arange(1, 300), rng.integers(1, 2**31, 200)]).astype(np.uint64)
    m, s = magic_divisor(ds)
    ns = np.concatenate([np.arange(0, 5000), rng.integers(0, 2**32, 5000)]).astype(np.uint64)
    for d, mm, ss in zip(ds, m.astype(np.uint64), s.astype(np.uint64), strict=True):
        hi = (ns * mm) >> np.uint64(32)
        q = (hi + ns) >> ss
        assert np.array_equal(q, ns // d), int(d)
