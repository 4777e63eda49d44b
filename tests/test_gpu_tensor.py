"""Device SymmetricTensor parity: CUDA path (through the C ABI) against the
reference fixtures and the CPU oracle.

Tolerances: permute / transpose / dagger / layout are pure data movement and
must be bit-exact; GEMM-based results use a different summation order than
numpy's BLAS and are compared at 1e-12 relative to the largest entry;
eigen/singular values at 1e-10 relative (LAPACK vs cuSOLVER)."""

import numpy as np
import pytest

from oracle import frostspin_oracle as fo
from tests.helpers import (
    assert_blocks_close,
    assert_blocks_equal,
    assert_same_structure,
    diag_from_dic,
    load,
    oracle_from_dic,
)

pytestmark = pytest.mark.gpu


def dev_from_dic(d, prefix):
    from frostspin_b200 import U1SymmetricTensor

    return U1SymmetricTensor.load_from_dic(d, prefix=prefix)


@pytest.mark.parametrize("name", ["u1_reference_test", "z2_rank6"])
def test_permute_bit_exact_vs_reference(name):
    d = load(name)
    t = dev_from_dic(d, "in")
    i = 0
    while f"perm{i}_axes" in d:
        axes = tuple(int(a) for a in d[f"perm{i}_axes"])
        nrr = int(d[f"perm{i}_nrr"])
        ref = oracle_from_dic(d, f"perm{i}")
        got = t.permute(axes[:nrr], axes[nrr:])
        assert_same_structure(got, ref)
        assert_blocks_equal(got, ref)
        # same permute reached from transposed (F-order) storage: leg a of t is
        # leg (a - nrr) % ndim of t.transpose()
        tt = t.transpose()
        mapped = tuple((a - t.n_row_reps) % t.ndim for a in axes)
        got2 = tt.permute(mapped[:nrr], mapped[nrr:])
        assert_same_structure(got2, ref)
        assert_blocks_equal(got2, ref)
        i += 1


def test_transpose_dagger_and_dense():
    d = load("u1_reference_test")
    t = dev_from_dic(d, "in")
    assert np.array_equal(t.toarray(), d["dense"])
    for key, got in (("transpose", t.transpose()), ("dagger", t.dagger())):
        ref = oracle_from_dic(d, key)
        assert_same_structure(got, ref)
        assert_blocks_equal(got, ref)
    # permute of a transposed tensor goes through the F-order strides
    tt = t.transpose()
    p = tt.permute((0, 3), (1, 2, 4))
    ref = fo.permute(fo.transpose(oracle_from_dic(d, "in")), (0, 3), (1, 2, 4))
    assert_blocks_equal(p, ref)


def test_matmul_and_reductions():
    d = load("u1_reference_test")
    t = dev_from_dic(d, "in")
    m = t @ t.dagger()
    ref = oracle_from_dic(d, "matmul")
    assert_same_structure(m, ref)
    assert_blocks_close(m, ref, 1e-12)
    assert abs(t.norm() - float(d["norm"])) <= 1e-13 * float(d["norm"])
    assert abs(m.trace() - float(d["matmul_trace"])) <= 1e-12 * abs(float(d["matmul_trace"]))
    fc = t.full_contract(t.dagger())
    assert abs(fc - float(d["full_contract_dagger"])) <= 1e-12 * abs(fc)


def test_microbench_small_permute_matmul():
    d = load("u1_microbench_small")
    t1 = dev_from_dic(d, "t1")
    t2 = dev_from_dic(d, "t2")
    p = t1.permute((0, 2), (1, 3))
    ref = oracle_from_dic(d, "perm")
    assert_same_structure(p, ref)
    assert_blocks_equal(p, ref)
    m = p @ t2
    ref = oracle_from_dic(d, "matmul")
    assert_same_structure(m, ref)
    assert_blocks_close(m, ref, 1e-12)


def test_elementwise_ops_and_diagonal_products():
    from frostspin_b200 import DiagonalTensor

    d = load("u1_reference_test")
    t = dev_from_dic(d, "in")
    o = oracle_from_dic(d, "in")
    assert_blocks_equal(t * 2.0, fo.scale(o, 2.0))
    assert_blocks_equal(-t, fo.scale(o, -1.0))
    assert_blocks_equal(t + t, fo.add(o, o))
    c = t.copy()
    c /= 4.0
    assert_blocks_equal(c, fo.scale(o, 0.25))
    # diagonal product on the last column leg and on the first row leg
    u, s, v = t.svd()
    us = u * s
    rng = np.random.default_rng(0)
    assert (t - us @ v).norm() < 1e-12 * t.norm()
    sv = s * v
    assert (t - u @ sv).norm() < 1e-12 * t.norm()
    s12 = s**0.5
    assert (t - (u * s12) @ (s12 * v)).norm() < 1e-12 * t.norm()
    sigma = type(t).from_diagonal_tensor(s)
    assert (t - u @ sigma @ v).norm() < 1e-12 * t.norm()
    ref_blocks, ref_irr = diag_from_dic(d, "svd_s")
    assert np.array_equal(s.block_irreps, ref_irr)
    for a, b in zip(s.host_blocks(), ref_blocks, strict=True):
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-14)
    w = DiagonalTensor([rng.random(k) for k in s.block_sizes], s.representation,
                       s.block_irreps, s.block_degen, "U1")
    assert abs(w.sum() - sum(b.sum() for b in w.host_blocks())) < 1e-12
    assert abs(w.norm() - np.sqrt(sum((b**2).sum() for b in w.host_blocks()))) < 1e-12


def test_truncated_svd_spectrum_vs_reference():
    d = load("u1_reference_test")
    t = dev_from_dic(d, "in")
    u, s, v = t.truncated_svd(6)
    ref_blocks, ref_irr = diag_from_dic(d, "tsvd_s")
    assert np.array_equal(s.block_irreps, ref_irr)
    for a, b in zip(s.host_blocks(), ref_blocks, strict=True):
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-14)
    usv = (u * s) @ v
    ref = oracle_from_dic(d, "tsvd_usv")
    assert_blocks_close(usv, ref, 1e-10)


def test_io_roundtrip_reference_format(tmp_path):
    from frostspin_b200 import U1SymmetricTensor

    d = load("z2_rank6")
    t = dev_from_dic(d, "in")
    f = tmp_path / "t.npz"
    t.save_to_file(f)
    t2 = U1SymmetricTensor.load_from_file(f)
    assert_same_structure(t, t2)
    assert_blocks_equal(t, t2)
    with np.load(f) as fin:
        # same keys as the reference writes (it used prefix "in" in the fixture)
        assert set(fin.files) == {k[2:] for k in d.files if k.startswith("in_")}


def test_ising_c4v_iterations_vs_reference():
    from frostspin_b200 import DiagonalTensor
    from frostspin_b200.ctmrg import energy_per_bond, ising_site_tensors, iterate_c4v

    d = load("ising_chi8")
    a, a2, a0d, mopd = ising_site_tensors(float(d["beta"]))
    s = DiagonalTensor.load_from_dic(d, prefix="s0")
    T = dev_from_dic(d, "T0")
    for it in range(1, 11):
        s, T = iterate_c4v(s, T, a, a2, int(d["chi"]))
        if f"s{it}_block_irreps" in d:
            ref_blocks, ref_irr = diag_from_dic(d, f"s{it}")
            assert np.array_equal(s.block_irreps, ref_irr)
            for x, y in zip(s.host_blocks(), ref_blocks, strict=True):
                np.testing.assert_allclose(x, y, rtol=1e-9, atol=1e-13)
            e = energy_per_bond(s, T, a0d, mopd)
            assert abs(e - float(d[f"energy{it}"])) < 1e-9


def test_ising_chi32_100_iterations_energy():
    from frostspin_b200 import DiagonalTensor
    from frostspin_b200.ctmrg import energy_per_bond, ising_site_tensors, iterate_c4v

    d = load("ising_chi32")
    a, a2, a0d, mopd = ising_site_tensors(float(d["beta"]))
    s = DiagonalTensor.load_from_dic(d, prefix="s0")
    T = dev_from_dic(d, "T0")
    for _ in range(100):
        s, T = iterate_c4v(s, T, a, a2, 32)
    e = energy_per_bond(s, T, a0d, mopd)
    assert abs(e - float(d["energy100"])) < 1e-9


def test_ising_chi32_correlation_length():
    """Correlation length of the C4v Ising run (beta = 0.44, chi = 32, 100
    iterations): xi of the device environment against xi of the reference's
    own edge tensor after 100 iterations (the oracle's dense FP64 edge transfer
    operator), and the device transfer spectrum of the reference's tensor
    against the oracle's."""
    from frostspin_b200 import DiagonalTensor
    from frostspin_b200.ctmrg import (correlation_length, edge_transfer_spectrum,
                                      ising_site_tensors, iterate_c4v)
    from tests.helpers import oracle_from_dic

    d = load("ising_chi32")
    xi_ref, lam_ref = fo.ising_correlation_length(oracle_from_dic(d, "T100"))
    lam_dev = edge_transfer_spectrum(dev_from_dic(d, "T100"), 4)
    np.testing.assert_allclose(np.sort(np.abs(lam_dev)), np.sort(np.abs(lam_ref)), rtol=1e-12)
    a, a2, _, _ = ising_site_tensors(float(d["beta"]))
    s = DiagonalTensor.load_from_dic(d, prefix="s0")
    T = dev_from_dic(d, "T0")
    for _ in range(100):
        s, T = iterate_c4v(s, T, a, a2, 32)
    xi = correlation_length(T)
    assert abs(xi - xi_ref) < 1e-6 * xi_ref, (xi, xi_ref)
