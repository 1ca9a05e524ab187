"""Batched solves (gr_batch_*): many systems of uneven sizes in one PBiCGStab
whose every launch covers all of them.

Each system keeps its own Krylov state, its own convergence test and the
block partition of its reductions that a solve of it alone uses, so its
result in a batch is bit-identical to its result alone: x, the iteration
count and every norm. The batch is checked against solo solves through the
ordinary solver path (which the oracle checks elsewhere), and converged
solutions are checked against an FP64 ground truth.
"""
import numpy as np
import pytest

import graphene_b200 as gb

pytestmark = pytest.mark.gpu


def cfg(tol=1e-6, maxit=300, norm="L2", prec="ILU", extra=None):
    c = {"type": "PBiCGStab", "maxIterations": maxit, "relTolerance": tol, "norm": norm,
         "preconditioner": {"type": prec, "kernel": "ring"}}
    if extra:
        c.update(extra)
    return c


# (nx, ny, nz, tiles, seed): sizes that are not multiples of 32 rows, one-
# tile and many-tile systems, and one tiny system that converges early.
SYSTEMS = [(12, 11, 9, 4, 1), (20, 20, 20, 16, 2), (5, 4, 3, 1, 3), (17, 13, 10, 8, 4),
           (32, 32, 8, 24, 5), (7, 9, 11, 3, 6)]


def systems(vt, spec=SYSTEMS, sigma=1.0):
    return [gb.generateMatrix(gb.GEN_VAR_POISSON, nx, ny, nz, (sigma,), seed, tiles, gb.PART_AUTO, vt)
            for (nx, ny, nz, tiles, seed) in spec]


def rhs(hs, dt, seed=11):
    return [gb.randomVector(seed + k, h.numRows).astype(dt) for k, h in enumerate(hs)]


def solo(h, c, b):
    A = h.copyToTile()
    x = np.zeros(h.numRows, b.dtype)
    st = gb.Solver(A, c).solveHost(x, b)
    return x, st


@pytest.mark.parametrize("vt,dt", [(gb.FLOAT32, np.float32), (gb.FLOAT64, np.float64), (gb.FLOAT32, np.float64)])
def test_batch_equals_solo(vt, dt):
    hs = systems(vt)
    bs = rhs(hs, dt)
    c = cfg(tol=1e-6 if dt == np.float32 else 1e-10)
    B = gb.Batch(hs, c)
    xs, sts = B.solveHost(bs)
    iters = []
    for h, b, x, st in zip(hs, bs, xs, sts):
        xr, sr = solo(h, c, b)
        np.testing.assert_array_equal(x, xr)
        assert st.iterations == sr.iterations
        assert st.converged == sr.converged
        assert st.finalResidual == sr.finalResidual
        assert st.initialResidual == sr.initialResidual
        assert st.bNorm == sr.bNorm
        iters.append(st.iterations)
    # Uneven sizes converge after different numbers of iterations: the
    # early ones drop out while the others continue.
    assert len(set(iters)) > 1
    assert all(st.converged for st in sts)


@pytest.mark.parametrize("vt,dt", [(gb.FLOAT32, np.float32), (gb.FLOAT64, np.float64)])
def test_batch_gauss_seidel_equals_solo(vt, dt):
    """PBiCGStab with Gauss-Seidel (2 sweeps) over a batch: the sweeps'
    kernel looks up each tile's system like the ILU substitution does."""
    hs = systems(vt)
    bs = rhs(hs, dt, seed=21)
    c = cfg(tol=1e-6 if dt == np.float32 else 1e-10,
            extra={"preconditioner": {"type": "GaussSeidel", "numFixedIterations": 2, "kernel": "ring"}})
    xs, sts = gb.Batch(hs, c).solveHost(bs)
    for h, b, x, st in zip(hs, bs, xs, sts):
        xr, sr = solo(h, c, b)
        np.testing.assert_array_equal(x, xr)
        assert st.iterations == sr.iterations and st.converged == sr.converged
        assert st.finalResidual == sr.finalResidual
    assert all(st.converged for st in sts)


def mpir_cfg(ext="float64", pre=None):
    return {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 30, "extendedPrecisionType": ext,
            "innerSolver": {"type": "PBiCGStab", "maxIterations": 300, "relResidual": 1e-4,
                            "preconditioner": pre or {"type": "ILU", "kernel": "ring"}}}


@pytest.mark.parametrize("ext", ["float64", "twofloat32"])
def test_batch_mpir_equals_solo(ext):
    """IterativeRefinement over a batch: per-system residual norms (each
    reduced as alone), one batched inner solve for the systems still
    refining, phi updated on those systems only. Every system's x, outer and
    inner iteration counts and norms equal its solo solve's."""
    hs = systems(gb.FLOAT32, sigma=1.5)
    bs = rhs(hs, np.float32, seed=31)
    c = mpir_cfg(ext)
    xs, sts = gb.Batch(hs, c).solveHost(bs)
    outer = []
    for h, b, x, st in zip(hs, bs, xs, sts):
        xr, sr = solo(h, c, b)
        np.testing.assert_array_equal(x, xr)
        assert st.iterations == sr.iterations and st.innerIterations == sr.innerIterations
        assert st.finalResidual == sr.finalResidual and st.initialResidual == sr.initialResidual
        assert st.converged == sr.converged
        outer.append(st.iterations)
    assert all(st.converged for st in sts)


def test_batch_mpir_gauss_seidel_inner():
    hs = systems(gb.FLOAT32, SYSTEMS[:4])
    bs = rhs(hs, np.float32, seed=37)
    c = mpir_cfg(pre={"type": "GaussSeidel", "numFixedIterations": 2, "kernel": "ring"})
    xs, sts = gb.Batch(hs, c).solveHost(bs)
    for h, b, x, st in zip(hs, bs, xs, sts):
        xr, sr = solo(h, c, b)
        np.testing.assert_array_equal(x, xr)
        assert st.iterations == sr.iterations and st.innerIterations == sr.innerIterations


def test_batch_mpir_outer_cap():
    """Systems stop at the outer iteration cap independently."""
    hs = systems(gb.FLOAT32, SYSTEMS[:3])
    bs = rhs(hs, np.float32, seed=41)
    c = mpir_cfg()
    c["maxIterations"] = 1
    xs, sts = gb.Batch(hs, c).solveHost(bs)
    for h, b, x, st in zip(hs, bs, xs, sts):
        xr, sr = solo(h, c, b)
        np.testing.assert_array_equal(x, xr)
        assert st.iterations == sr.iterations == 1


def test_batch_solutions_accurate():
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    hs = systems(gb.FLOAT64)
    bs = rhs(hs, np.float64)
    xs, sts = gb.Batch(hs, cfg(tol=1e-10)).solveHost(bs)
    for h, b, x in zip(hs, bs, xs):
        n = h.numRows
        rows, cols, vals = h.coo()
        A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
        xt = spl.spsolve(A.tocsc(), b)
        assert np.max(np.abs(x - xt)) <= 1e-7 * np.max(np.abs(xt))


def test_batch_initial_guess_and_repeat():
    hs = systems(gb.FLOAT32, SYSTEMS[:3])
    bs = rhs(hs, np.float32, seed=40)
    x0 = [gb.randomVector(90 + k, h.numRows).astype(np.float32) for k, h in enumerate(hs)]
    c = cfg(tol=1e-5)
    B = gb.Batch(hs, c)
    xa, sa = B.solveHost(bs, x0)
    xb, sb = B.solveHost(bs, x0)  # the same batch object solves again
    for h, b, g, x, y, s in zip(hs, bs, x0, xa, xb, sa):
        A = h.copyToTile()
        xr = g.copy()
        sr = gb.Solver(A, c).solveHost(xr, b)
        np.testing.assert_array_equal(x, xr)
        np.testing.assert_array_equal(y, xr)
        assert s.iterations == sr.iterations


def test_batch_iteration_cap_and_single_system():
    hs = systems(gb.FLOAT32, [(16, 16, 16, 8, 7)])
    bs = rhs(hs, np.float32)
    c = cfg(tol=1e-12, maxit=5)
    xs, sts = gb.Batch(hs, c).solveHost(bs)
    xr, sr = solo(hs[0], c, bs[0])
    np.testing.assert_array_equal(xs[0], xr)
    assert sts[0].iterations == sr.iterations == 5
    assert not sts[0].converged


def test_batch_many_small_systems():
    spec = [(3 + k % 5, 4 + k % 3, 2 + k % 4, 1 + k % 3, 100 + k) for k in range(40)]
    hs = systems(gb.FLOAT32, spec)
    bs = rhs(hs, np.float32, seed=300)
    c = cfg(tol=1e-6)
    xs, sts = gb.Batch(hs, c).solveHost(bs)
    for h, b, x, st in zip(hs, bs, xs, sts):
        xr, sr = solo(h, c, b)
        np.testing.assert_array_equal(x, xr)
        assert st.iterations == sr.iterations


@pytest.mark.parametrize("bad", [
    {"type": "CG"},
    cfg(prec="GaussSeidel"),
    {"type": "PBiCGStab", "maxIterations": 10, "relTolerance": 1e-6},
    cfg(extra={"preconditioner": {"type": "ILU", "kernel": "warp"}}),
    cfg(extra={"preconditioner": {"type": "GaussSeidel", "numFixedIterations": 2, "kernel": "wring"}}),
    cfg(extra={"preconditioner": {"type": "GaussSeidel", "numFixedIterations": 2, "kernel": "levels"}}),
])
def test_batch_rejects_unsupported_configs(bad):
    hs = systems(gb.FLOAT32, SYSTEMS[:2])
    with pytest.raises(gb.GrapheneError):
        gb.Batch(hs, bad)


def test_batch_rejects_mixed_coefficient_types():
    hs = systems(gb.FLOAT32, SYSTEMS[:1]) + systems(gb.FLOAT64, SYSTEMS[1:2])
    with pytest.raises(gb.GrapheneError):
        gb.Batch(hs, cfg())
