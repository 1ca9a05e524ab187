"""The SpMV layout's two column encodings on the device: SpMV, residuals (float,
double and double-word intermediates) and a preconditioned PBiCGStab solve
give bit-identical results with 32-bit columns and with 16-bit row offsets,
including chunks with the most far columns the 16-bit layout takes (64);
SpMV equals the oracle."""
import numpy as np
import pytest

import graphene_b200 as gb
from tests.oracle_py import Oracle

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def far_matrix(n=150000):
    """Two far columns a row (64 in every chunk, the most the 16-bit layout
    takes), on both sides of the row, between near ones."""
    r = np.arange(n)
    far = np.where(r % 3 == 0, (r + 40000) % n, (r + n - 50000) % n)
    far2 = (r + 70001) % n
    up, down = r[:-1], r[2:]
    rows = np.concatenate([r, up, r, down, r])
    cols = np.concatenate([r, up + 1, far, down - 2, far2])
    vals = np.concatenate([np.full(n, 8.0), np.full(rows.size - n, -1.0)])
    return rows, cols, vals


CASES = {
    "var_poisson": lambda vt: gb.generateMatrix(gb.GEN_VAR_POISSON, 48, 40, 44, (1.5,), 2, 96, gb.PART_RCB,
                                                valueType=vt),
    "convdiff": lambda vt: gb.generateMatrix(gb.GEN_CONVDIFF, 36, 36, 36, (0.5, 0.25, 0.125), 0, 24,
                                             valueType=vt),
    "far": lambda vt: gb.HostMatrix.from_coo(150000, *far_matrix(), 1, valueType=vt),
}


def pair(make, vt):
    h0, h1 = make(vt), make(vt)
    h0.setSpmvLayout(0)
    h1.setSpmvLayout(1)
    A0, A1 = h0.copyToTile(), h1.copyToTile()
    assert not A0.spmvLayout()["compact"] and A1.spmvLayout()["compact"]
    return h0, A0, A1


def same(a, b):
    a, b = host(a), host(b)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("case", sorted(CASES))
def test_spmv_and_residuals_identical(case):
    h, A0, A1 = pair(CASES[case], gb.FLOAT32)
    n = h.numRows
    x = gb.randomVector(5, n).astype(np.float32)
    b = gb.randomVector(6, n).astype(np.float32)
    xd, bd = A0.vector(x), A0.vector(b)
    same(A0 * xd, A1 * xd)
    xd64 = A0.vector(x.astype(np.float64))
    same(A0 * xd64, A1 * xd64)
    for dest, inter in ((gb.FLOAT32, gb.FLOAT32), (gb.FLOAT32, gb.FLOAT64), (gb.FLOAT64, gb.FLOAT64),
                        (gb.FLOAT32, gb.TWOFLOAT32)):
        same(A0.residual(xd, bd, dest, inter), A1.residual(xd, bd, dest, inter))
    far = A1.spmvLayout()["far"]
    if case == "far":
        assert far == 2 * n


def test_spmv_matches_oracle_16_bit():
    h = CASES["var_poisson"](gb.FLOAT32)
    h.setSpmvLayout(1)
    A = h.copyToTile()
    o = Oracle()
    om = o.grid_system(1, 48, 40, 44, (1.5,), 2, 96)
    assert np.array_equal(om.row_to_tile(), h.rowToTile())
    x = om.decompose(gb.randomVector(7, h.numRows).astype(np.float32))
    np.testing.assert_array_equal(host(A * dev(x)), om.spmv(x))


def test_float64_coefficients_identical():
    h, A0, A1 = pair(CASES["convdiff"], gb.FLOAT64)
    x = A0.vector(gb.randomVector(8, h.numRows))
    same(A0 * x, A1 * x)


@pytest.mark.parametrize("case", ["var_poisson", "convdiff"])
def test_solve_identical(case):
    h, A0, A1 = pair(CASES[case], gb.FLOAT32)
    cfg = {"type": "PBiCGStab", "maxIterations": 40, "relResidual": 1e-9, "preconditioner": {"type": "ILU"}}
    b = A0.vector(gb.randomVector(9, h.numRows).astype(np.float32))
    out = []
    for A in (A0, A1):
        x = A.vector(np.zeros(h.numRows, np.float32))
        st = gb.Solver(A, cfg).solve(x, b)
        out.append((x, st.iterations))
    assert out[0][1] == out[1][1]
    same(out[0][0], out[1][0])
