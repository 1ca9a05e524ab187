"""Value updates on a resident structure, against building from scratch.

Matrix.updateValues + Solver.refresh must leave the device in the state a
new Matrix + Solver for the new values would have: every later solve is
bit-identical (SpMV, ILU / DILU / Gauss-Seidel preconditioned PBiCGStab,
MPIR), including solves replayed from the iteration graphs captured before
the update. The solve server uses the same path for requests whose matrix
shares a resident pair's structure (cache_hit == 2)."""
import numpy as np
import pytest

import graphene_b200 as gb

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


CFGS = {
    "ilu": {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-7, "preconditioner": {"type": "ILU"}},
    "dilu": {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-7,
             "preconditioner": {"type": "ILU", "diagonalBased": True}},
    "gs": {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-7,
           "preconditioner": {"type": "GaussSeidel", "numFixedIterations": 2}},
    "ilu_levels": {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-7,
                   "preconditioner": {"type": "ILU", "kernel": "levels"}},
    "mpir": {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 30,
             "extendedPrecisionType": "float64",
             "innerSolver": {"type": "PBiCGStab", "maxIterations": 300, "relResidual": 1e-4,
                             "preconditioner": {"type": "ILU"}}},
}


@pytest.mark.parametrize("name", list(CFGS))
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
def test_update_values_equals_fresh(name, vt):
    if name == "mpir" and vt == gb.FLOAT64:
        pytest.skip("IterativeRefinement works on float32 vectors")
    dims, tiles = (18, 17, 16), 12
    h0 = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 5, tiles, valueType=vt)
    h1 = gb.generateMatrixLike(h0, gb.GEN_VAR_POISSON, *dims, (1.0,), 6)
    dt = np.float32 if vt == gb.FLOAT32 else np.float64
    b = gb.randomVector(7, h0.numRows).astype(dt)
    # Fresh matrix and solver for h1.
    A1 = h1.copyToTile()
    x1 = dev(np.zeros_like(b))
    st1 = gb.Solver(A1, CFGS[name]).solve(x1, dev(b))
    y1 = host(A1 * dev(b))
    # A matrix and solver built for h0, used once (graphs captured), then updated.
    A0 = h0.copyToTile()
    s0 = gb.Solver(A0, CFGS[name])
    s0.solve(dev(np.zeros_like(b)), dev(b))
    A0.updateValues(h1)
    s0.refresh()
    np.testing.assert_array_equal(host(A0 * dev(b)), y1)
    for _ in range(2):
        x = dev(np.zeros_like(b))
        st = s0.solve(x, dev(b))
        assert st.iterations == st1.iterations and st.converged == st1.converged
        np.testing.assert_array_equal(host(x), host(x1))


@pytest.mark.parametrize("name", ["ilu", "gs", "mpir"])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
@pytest.mark.parametrize("layout", [0, 1])
def test_update_global_values_equals_fresh(name, vt, layout):
    """Matrix.updateGlobalValues (values gathered on the device from the
    global CRS order) leaves the state a fresh matrix and solver would have,
    in both SpMV layouts."""
    if name == "mpir" and vt == gb.FLOAT64:
        pytest.skip("IterativeRefinement works on float32 vectors")
    dims, tiles = (17, 18, 19), 10
    h0 = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 5, tiles, valueType=vt)
    h0.setSpmvLayout(layout)
    gv, gd = gb.generateValues(h0, gb.GEN_VAR_POISSON, *dims, (1.0,), 6)
    h1 = gb.generateMatrixLike(h0, gb.GEN_VAR_POISSON, *dims, (1.0,), 6)
    h1.setSpmvLayout(layout)
    dt = np.float32 if vt == gb.FLOAT32 else np.float64
    b = gb.randomVector(7, h0.numRows).astype(dt)
    A1 = h1.copyToTile()
    x1 = dev(np.zeros_like(b))
    st1 = gb.Solver(A1, CFGS[name]).solve(x1, dev(b))
    A0 = h0.copyToTile()
    assert A0.spmvLayout()["compact"] == bool(layout)
    s0 = gb.Solver(A0, CFGS[name])
    s0.solve(dev(np.zeros_like(b)), dev(b))
    A0.updateGlobalValues(gv, gd)
    s0.refresh()
    np.testing.assert_array_equal(host(A0 * dev(b)), host(A1 * dev(b)))
    x = dev(np.zeros_like(b))
    st = s0.solve(x, dev(b))
    assert st.iterations == st1.iterations and st.converged == st1.converged
    np.testing.assert_array_equal(host(x), host(x1))


def test_update_values_rejects_other_structures():
    h0 = gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 1, 8)
    other = gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 1, 9)
    A0 = h0.copyToTile()
    with pytest.raises(gb.GrapheneError):
        A0.updateValues(other)


def test_server_reuses_structure():
    """Requests with fresh values on a resident structure: served through the
    value update (cache_hit 2), with results bit-identical to a server that
    builds every pair from scratch."""
    cfg = CFGS["ilu"]
    dims, tiles = (20, 20, 20), 8
    tmpl = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 10, tiles)
    hs = [gb.generateMatrixLike(tmpl, gb.GEN_VAR_POISSON, *dims, (1.0,), 11 + k) for k in range(6)]
    bs = [gb.randomVector(20 + k, tmpl.numRows).astype(np.float32) for k in range(6)]
    srv = gb.Server(slots=1)
    ids = [srv.submit(h, cfg, b) for h, b in zip(hs, bs)]
    res = [srv.wait(i) for i in ids]
    srv.close()
    assert res[0][2]["cache_hit"] == 0
    assert all(r[2]["cache_hit"] == 2 for r in res[1:])
    for k, (h, b) in enumerate(zip(hs, bs)):
        fresh = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 11 + k, tiles)
        x = np.zeros_like(b)
        st = gb.Solver(fresh.copyToTile(), cfg).solveHost(x, b)
        np.testing.assert_array_equal(res[k][0], x)
        assert res[k][1].iterations == st.iterations


@pytest.mark.parametrize("cfg", ["ilu", "mpir"])
def test_server_values_only_requests(cfg):
    """gr_server_submit_values: a request carrying only new values for a
    template's structure gives the result of the full matrix, bit for bit,
    whether its pair is new (the first request) or resident (cache_hit 2)."""
    c = CFGS[cfg]
    dims, tiles = (22, 21, 20), 12
    tmpl = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 30, tiles)
    srv = gb.Server(slots=2)
    ids, bs = [], []
    for k in range(5):
        gv, gd = gb.generateValues(tmpl, gb.GEN_VAR_POISSON, *dims, (1.0,), 31 + k)
        b = gb.randomVector(40 + k, tmpl.numRows).astype(np.float32)
        bs.append(b)
        ids.append(srv.submitValues(tmpl, gv, gd, c, b))
    res = [srv.wait(i) for i in ids]
    srv.close()
    assert res[0][2]["cache_hit"] == 0 and all(r[2]["cache_hit"] == 2 for r in res[2:])
    for k, b in enumerate(bs):
        fresh = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 31 + k, tiles)
        x = np.zeros_like(b)
        st = gb.Solver(fresh.copyToTile(), c).solveHost(x, b)
        np.testing.assert_array_equal(res[k][0], x)
        assert res[k][1].converged and st.converged
