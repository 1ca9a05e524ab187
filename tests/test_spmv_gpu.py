"""SpMV / residual / norm on the GPU, through the C ABI, against the oracle.

Per-row arithmetic is defined by the reference (CRSMatrix.cpp:42-128), so
SpMV and every residual variant must match the oracle bit for bit. Norms
accumulate in FP64 in a different order: relative tolerance 1e-13.
"""
import numpy as np
import pytest

import graphene_b200 as gb
from tests.util import random_coo

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_case(name, oracle, vt=gb.FLOAT32):
    ovt = 0 if vt == gb.FLOAT32 else 1
    if name == "poisson32":
        h = gb.generate3DPoissonMatrix(vt, 32, 32, 32, 64)
        return h, oracle.poisson(32, 32, 32, 64, h.rowToTile(), ovt)
    if name == "poisson_odd_bfs":
        h = gb.generate3DPoissonMatrix(vt, 13, 7, 9, 5, gb.PART_BFS)
        return h, oracle.poisson(13, 7, 9, 5, h.rowToTile(), ovt)
    if name == "poisson_1tile":
        h = gb.generate3DPoissonMatrix(vt, 10, 10, 10, 1)
        return h, oracle.poisson(10, 10, 10, 1, None, ovt)
    if name == "tiny":
        h = gb.generate3DPoissonMatrix(vt, 3, 1, 1, 2)
        return h, oracle.poisson(3, 1, 1, 2, h.rowToTile(), ovt)
    if name == "random":
        n, r, c, v = random_coo(777, 0.01, 3)
        h = gb.HostMatrix.from_coo(n, r, c, v, 9, partitioner=gb.PART_BFS, valueType=vt)
        return h, oracle.matrix(n, r, c, v, 9, h.rowToTile(), ovt)
    raise KeyError(name)


NAMES = ["poisson32", "poisson_odd_bfs", "poisson_1tile", "tiny", "random"]


@pytest.mark.parametrize("name", NAMES)
def test_spmv_f32_bit_exact(oracle, name):
    h, om = make_case(name, oracle)
    A = h.copyToTile()
    x = np.random.default_rng(1).uniform(-1, 1, h.numRows).astype(np.float32)
    y = A * dev(x)
    np.testing.assert_array_equal(y.cpu().numpy(), om.spmv(x))


@pytest.mark.parametrize("name", ["poisson32", "random"])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
def test_spmv_f64_vectors_bit_exact(oracle, name, vt):
    h, om = make_case(name, oracle, vt)
    A = h.copyToTile()
    x = np.random.default_rng(2).standard_normal(h.numRows)
    y = A * dev(x)
    np.testing.assert_array_equal(y.cpu().numpy(), om.spmv(x))


def test_spmv_matches_scipy_fp64():
    """Independent check of the whole path, natural order in and out."""
    import scipy.sparse as sp
    n, r, c, v = random_coo(500, 0.02, 11)
    h = gb.HostMatrix.from_coo(n, r, c, v, 7, partitioner=gb.PART_BFS, valueType=gb.FLOAT64)
    A = h.copyToTile()
    x = np.random.default_rng(3).standard_normal(n)
    y = A.toNatural(A * A.vector(x, gb.FLOAT64))
    ref = sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsr() @ x
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("name", ["poisson32", "random", "tiny"])
@pytest.mark.parametrize("xt,bt,rt,it", [
    (0, 0, 0, 0),   # PBiCGStab working type float32
    (1, 1, 1, 1),   # float64
    (1, 0, 0, 1),   # MPIR: phi float64, b / r float32
    (0, 0, 0, 1),   # float32 x, float64 intermediate
    (2, 0, 0, 2),   # MPIR: phi double-word
    (0, 0, 0, 2),   # float32 x, double-word intermediate
])
def test_residual_bit_exact(oracle, name, xt, bt, rt, it):
    h, om = make_case(name, oracle)
    A = h.copyToTile()
    rng = np.random.default_rng(5)
    n = h.numRows
    if xt == 2:
        hi = rng.uniform(-1, 1, n).astype(np.float32)
        lo = (rng.uniform(-1, 1, n) * np.abs(hi) * 2.0 ** -25).astype(np.float32)
        x = np.stack([hi, lo], 1).reshape(-1)
    else:
        x = rng.uniform(-1, 1, n).astype(np.float32 if xt == 0 else np.float64)
    b = rng.uniform(-1, 1, n).astype(np.float32 if bt == 0 else np.float64)
    r = A.residual(dev(x), dev(b), destType=rt, intermediateType=it, xType=xt)
    np.testing.assert_array_equal(r.cpu().numpy(), om.residual(x, xt, b, rt, it))


def test_double_word_residual_is_fp64_accurate(oracle):
    """A double-word residual of an FP64-exact x agrees with the FP64 one to
    about 2^-44 relative (DW algorithms' error bounds, JMP 2017)."""
    h, om = make_case("poisson32", oracle)
    A = h.copyToTile()
    rng = np.random.default_rng(9)
    n = h.numRows
    xd = rng.uniform(-1, 1, n)
    hi = xd.astype(np.float32)
    lo = (xd - hi.astype(np.float64)).astype(np.float32)
    xdw = np.stack([hi, lo], 1).reshape(-1)
    xe = hi.astype(np.float64) + lo.astype(np.float64)
    b = (rng.uniform(-1, 1, n)).astype(np.float32)
    r_dw = A.residual(dev(xdw), dev(b), destType=1 - 1, intermediateType=2, xType=2).cpu().numpy()
    r_64 = A.residual(dev(xe), dev(b), destType=0, intermediateType=1).cpu().numpy()
    np.testing.assert_allclose(r_dw, r_64, rtol=2e-7, atol=1e-12)


@pytest.mark.parametrize("norm", [gb.NORM_L1, gb.NORM_L2, gb.NORM_LINF])
@pytest.mark.parametrize("t", [np.float32, np.float64])
def test_norms(oracle, norm, t):
    h, om = make_case("poisson32", oracle)
    A = h.copyToTile()
    x = np.random.default_rng(7).standard_normal(h.numRows).astype(t)
    got = A.vectorNorm(norm, dev(x))
    np.testing.assert_allclose(got, om.norm(x, norm), rtol=1e-13)


def test_reduction_golden_vectors():
    """dsl/tensor/tests/TensorTests.cpp:136-160: an 8x2 tensor of 0..15 summed
    over dimension 0 gives 56 and 64 (L1 norm = signed sum)."""
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 8, 1, 1, 4)
    A = h.copyToTile()
    data = np.arange(16, dtype=np.float32).reshape(8, 2)
    assert A.vectorNorm(gb.NORM_L1, dev(data[:, 0].copy())) == 56.0
    assert A.vectorNorm(gb.NORM_L1, dev(data[:, 1].copy())) == 64.0
    # TensorTests.cpp:377-425: |(1,2,3)|^2 = 14, ... via L2^2
    v = np.array([1, 2, 3, 0, 0, 0, 0, 0], np.float32)
    assert A.vectorNorm(gb.NORM_L2, dev(v)) ** 2 == pytest.approx(14.0, rel=1e-15)


def test_decompose_compose_on_device(oracle):
    h, _ = make_case("poisson_odd_bfs", oracle)
    A = h.copyToTile()
    import ctypes
    import torch
    v = np.random.default_rng(0).standard_normal(h.numRows)
    nat = dev(v)
    tile = torch.empty_like(nat)
    lib = gb._lib.lib()
    gb._lib.check(lib.gr_decompose_vector(A._m, ctypes.c_void_p(nat.data_ptr()),
                                          ctypes.c_void_p(tile.data_ptr()), gb.FLOAT64))
    np.testing.assert_array_equal(tile.cpu().numpy(), h.decomposeVector(v, gb.FLOAT64))
    back = torch.empty_like(nat)
    gb._lib.check(lib.gr_compose_vector(A._m, ctypes.c_void_p(tile.data_ptr()),
                                        ctypes.c_void_p(back.data_ptr()), gb.FLOAT64))
    np.testing.assert_array_equal(back.cpu().numpy(), v)


def test_unsupported_combination_raises():
    h = gb.generate3DPoissonMatrix(gb.FLOAT64, 4, 4, 4, 2)
    A = h.copyToTile()
    x = dev(np.zeros(64, np.float32))
    with pytest.raises(gb.GrapheneError) as e:
        A * x
    assert e.value.code == 8


@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
def test_spmv_autotuner_keeps_results(oracle, vt):
    """The autotuner picks a launch geometry; every geometry computes the
    same rows in the same order, so y is bit-identical before and after."""
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 40, 36, 30, (1.0,), 3, 32)
    if vt == gb.FLOAT64:
        h = h.astype(gb.FLOAT64)
    A = h.copyToTile()
    t = np.float32 if vt == gb.FLOAT32 else np.float64
    x = dev(np.random.default_rng(9).standard_normal(h.numRows).astype(t))
    before = (A * x).cpu().numpy()
    g = A.tuneSpmv(vt, reps=3)
    assert g["block"] in (128, 256, 512) and g["batch"] in (4, 8, 16) and g["ms"] > 0
    np.testing.assert_array_equal((A * x).cpu().numpy(), before)


@pytest.mark.parametrize("flush", [False, True])
def test_spmv_device_timing_writes_the_product(flush):
    """gr_matrix_time_spmv launches the SpMV kernel itself: it reports a
    positive device time and leaves y = A x, bit-identical to gr_spmv."""
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 24, 20, 18, (1.0,), 3, 16)
    A = h.copyToTile()
    x = dev(np.random.default_rng(10).standard_normal(h.numRows).astype(np.float32))
    y = A.createUninitializedVector(gb.FLOAT32)
    ms = A.timeSpmv(x, y, reps=3, flushL2=flush)
    assert 0 < ms < 1000
    np.testing.assert_array_equal(y.cpu().numpy(), (A * x).cpu().numpy())
    with pytest.raises(gb.GrapheneError):
        A.timeSpmv(x, y, reps=0)
