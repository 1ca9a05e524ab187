"""Parity at the bench's full size: the 192^3 variable-coefficient Poisson
system with 2368 tiles (7,077,888 rows). SpMV, the FP64-intermediate
residual and the ILU(0) substitution (ring kernel, default layout) are
compared bit for bit with the oracle on the same tile layout; the oracle
runs on all host threads, which takes seconds at this size."""
import os

import numpy as np
import pytest

import graphene_b200 as gb
from tests.oracle_py import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full():
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 192, 192, 192, (1.5,), 2, 2368)
    o = Oracle()
    o.threads(os.cpu_count() or 1)
    rows, cols, vals = h.coo()
    om = o.matrix(h.numRows, rows, cols, vals, h.numTiles, h.rowToTile(), 0)
    A = h.copyToTile()
    return h, om, A


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_spmv_full_size_bit_exact(full):
    h, om, A = full
    x = gb.randomVector(31, h.numRows).astype(np.float32)  # tile order
    y = (A * dev(x)).cpu().numpy()
    np.testing.assert_array_equal(y, om.spmv(x))


def test_residual_fp64_intermediate_full_size_bit_exact(full):
    h, om, A = full
    x = gb.randomVector(32, h.numRows).astype(np.float32)
    b = gb.randomVector(33, h.numRows).astype(np.float32)
    r = A.residual(dev(x), dev(b), destType=gb.FLOAT32, intermediateType=gb.FLOAT64).cpu().numpy()
    np.testing.assert_array_equal(r, om.residual(x, 0, b, 0, 1))


def test_ilu_ring_full_size_bit_exact(full):
    h, om, A = full
    b = gb.randomVector(34, h.numRows).astype(np.float32)
    x = A.createUninitializedVector(gb.FLOAT32)
    gb.Solver(A, {"type": "ILU", "kernel": "ring"}).solve(x, dev(b))
    off, inv = om.ilu_factorize(False)
    np.testing.assert_array_equal(x.cpu().numpy(), om.ilu_solve(off, inv, b, False))
