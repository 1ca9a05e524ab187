"""Pins of the CPU oracle (CPU only, no GPU).

The reference's only result-pinning tests are the tensor reductions of
dsl/tensor/tests/TensorTests.cpp; their expected values are checked here
against the oracle's reductions. For SpMV, residual, ILU(0), DILU, the
Gauss-Seidel sweep and the solvers the reference has no golden vectors, so the
oracle is checked against a second, independent restatement in plain Python
(small sizes, P = 1 so that tile-local order is natural order) and against
scipy in FP64.
"""
import json

import numpy as np
import pytest

from tests.util import poisson_coo, random_coo

F32 = np.float32


def natural_matrix(oracle, n, rows, cols, vals, vt=0):
    return oracle.matrix(n, rows, cols, vals, 1, np.zeros(n, np.int32), vt)


def tile_order(om):
    """Global row of each tile-order position: every tile's local rows
    without its halo (local_to_global lists each tile's interior, separator
    and halo rows)."""
    sizes = om.tile_sizes().reshape(-1, 3)
    l2g = om.local_to_global()
    out, pos = [], 0
    for ni, ns, nh in sizes:
        out.append(l2g[pos:pos + ni + ns])
        pos += ni + ns + nh
    return np.concatenate(out)


def scipy_csr(n, rows, cols, vals, dtype=np.float64):
    import scipy.sparse as sp
    return sp.csr_matrix((vals.astype(dtype), (rows, cols)), shape=(n, n))


# ---- TensorTests.cpp golden values ---------------------------------------------------

def test_reduce_across_tiles_golden(oracle):
    """TensorTests.cpp:136-160 (ReduceAcrossTilesSingleIPU): an 8x2 float32
    tensor holding 0..15, linearly distributed over 4 tiles, reduced over
    dimension 0 with ADD gives 56 and 64."""
    data = np.arange(16, dtype=F32).reshape(8, 2)
    om = oracle.poisson(8, 1, 1, 4, np.repeat(np.arange(4, dtype=np.int32), 2))
    # The L1 "norm" of the reference is the signed sum (Tensor.cpp:425-439).
    assert om.norm(np.ascontiguousarray(data[:, 0]), 0) == 56.0
    assert om.norm(np.ascontiguousarray(data[:, 1]), 0) == 64.0
    # Per-tile worker split of Expression::reduce (Expression.cpp:729-769).
    assert oracle.L.or_reduce_sum(np.ascontiguousarray(data[:, 0]).ctypes.data, 8, 1) == 56.0
    assert oracle.L.or_reduce_sum(np.ascontiguousarray(data[:, 1]).ctypes.data, 8, 1) == 64.0


def test_reduce_same_tiles_golden(oracle):
    """TensorTests.cpp:190-222 (ReduceSameTiles): an 8x8 tensor holding 0..63
    reduced over dimension 1 gives 28, 92, ..., 476."""
    data = np.arange(64, dtype=F32).reshape(8, 8)
    expect = [28, 92, 156, 220, 284, 348, 412, 476]
    for row, e in zip(data, expect):
        row = np.ascontiguousarray(row)
        assert oracle.L.or_reduce_sum(row.ctypes.data, 8, 1) == e
        om = oracle.poisson(8, 1, 1, 1, np.zeros(8, np.int32))
        assert om.norm(row, 0) == e


def test_dot_and_squared_norm_golden(oracle):
    """TensorTests.cpp:225-261 (DotProductSameShape): row dots of
    {1,2,3}.{2,3,4} and {4,5,6}.{1,2,1} are 20 and 20; TensorTests.cpp:377-425
    (VectorProductReduction): squared magnitudes 14, 29, 50, 77. The dots go
    through the oracle's squared L2 norm by polarisation,
    a.b = (|a+b|^2 - |a-b|^2) / 4, exact for these small integers."""
    om = oracle.poisson(3, 1, 1, 1, np.zeros(3, np.int32))
    sq = lambda v: om.norm(np.asarray(v, F32), 1) ** 2  # noqa: E731
    for a, b in [((1, 2, 3), (2, 3, 4)), ((4, 5, 6), (1, 2, 1))]:
        a, b = np.array(a, F32), np.array(b, F32)
        assert (sq(a + b) - sq(a - b)) / 4 == pytest.approx(20.0, abs=1e-12)
    for v, e in [((1, 2, 3), 14), ((2, 3, 4), 29), ((3, 4, 5), 50), ((4, 5, 6), 77)]:
        assert sq(v) == pytest.approx(e, rel=1e-15)
    # LINF is reduce(MAX) of the signed values (Tensor.cpp:433-434), not the
    # largest magnitude.
    assert om.norm(np.array([1, -7, 3], F32), 2) == 3.0


# ---- independent Python restatements (P = 1) -----------------------------------------

def csr_parts(om):
    rp, ci, od, dg = om.local_crs()
    return rp.astype(np.int64), ci.astype(np.int64), od, dg


def py_spmv_f32(rp, ci, od, dg, x):
    """CRSMatrix::spmv (CRSMatrix.cpp:42-83): diagonal product first, then the
    off-diagonals in column order, every operation rounded to float32."""
    y = np.empty(len(dg), F32)
    for i in range(len(dg)):
        acc = F32(dg[i]) * x[i]
        for p in range(rp[i], rp[i + 1]):
            acc = F32(acc + F32(od[p]) * x[ci[p]])
        y[i] = acc
    return y


def py_ilu0(rp, ci, od, dg, dilu=False):
    """Block ILU(0) in IKJ order (ilu/Solver.cpp:134-292) in float32 scalars."""
    off = [F32(v) for v in od]
    a_off = list(off)
    d = [F32(v) for v in dg]
    n = len(d)

    def get(k, j, vals):
        for p in range(rp[k], rp[k + 1]):
            if ci[p] == j:
                return vals[p]
        return F32(0)

    for i in range(1, n):
        for ik in range(rp[i], rp[i + 1]):
            k = ci[ik]
            if k >= i:
                break
            if dilu:
                d[i] = F32(d[i] - F32(F32(a_off[ik] * get(k, i, a_off)) / d[k]))
                continue
            off[ik] = F32(off[ik] / d[k])
            for ij in range(ik + 1, rp[i + 1]):
                off[ij] = F32(off[ij] - F32(off[ik] * get(k, ci[ij], off)))
            d[i] = F32(d[i] - F32(off[ik] * get(k, i, off)))
    inv = [F32(F32(1) / v) for v in d]
    return np.array(off, np.float64), np.array(inv, np.float64)


def py_ilu_solve(rp, ci, off, inv, b, dilu=False):
    """Forward then backward substitution (ilu/Solver.cpp:367-550), float32."""
    n = len(b)
    x = np.zeros(n, F32)
    for i in range(n):
        t = F32(b[i])
        for p in range(rp[i], rp[i + 1]):
            if ci[p] >= i:
                break
            t = F32(t - F32(F32(off[p]) * x[ci[p]]))
        x[i] = F32(t * F32(inv[i])) if dilu else t
    for i in range(n - 1, -1, -1):
        t = F32(0)
        for p in range(rp[i + 1] - 1, rp[i] - 1, -1):
            if ci[p] <= i:
                break
            t = F32(t - F32(F32(off[p]) * x[ci[p]]))
        if dilu:
            x[i] = F32(x[i] + F32(t * F32(inv[i])))
        else:
            x[i] = F32(F32(x[i] + t) * F32(inv[i]))
    return x


def py_gs_sweep(rp, ci, od, dg, x, b):
    """One Gauss-Seidel sweep seeded with b (gauss-seidel codelet
    specification), ascending rows, float32."""
    x = x.copy()
    for i in range(len(dg)):
        s = F32(b[i])
        for p in range(rp[i], rp[i + 1]):
            s = F32(s - F32(F32(od[p]) * x[ci[p]]))
        x[i] = F32(s / F32(dg[i]))
    return x


@pytest.fixture(scope="module")
def small_case(oracle):
    n, r, c, v = random_coo(60, 0.08, seed=11)
    om = natural_matrix(oracle, n, r, c, v)
    return n, r, c, v, om


def test_oracle_spmv_matches_python_restatement(small_case):
    n, r, c, v, om = small_case
    x = np.random.default_rng(1).standard_normal(n).astype(F32)
    np.testing.assert_array_equal(om.spmv(x), py_spmv_f32(*csr_parts(om), x))


def test_oracle_spmv_and_residual_match_scipy_fp64(oracle):
    n, r, c, v = random_coo(80, 0.06, seed=5)
    om = natural_matrix(oracle, n, r, c, v, vt=1)
    A = scipy_csr(n, r, c, v)
    x = np.random.default_rng(2).standard_normal(n)
    b = np.random.default_rng(3).standard_normal(n)
    np.testing.assert_allclose(om.spmv(x), A @ x, rtol=1e-13, atol=1e-13)
    res = om.residual(x, 1, b, 1, 1)
    np.testing.assert_allclose(res, b - A @ x, rtol=1e-12, atol=1e-12)


def test_oracle_dw_residual_accuracy(oracle):
    """The double-word residual (x as {h, l} float pairs) of an FP32 matrix,
    rounded to float32 at the end, agrees with the exact residual to the
    final rounding plus a few units of 2^-44 of the row's magnitude
    (DWPlusFP / DWTimesFP error bounds), even where the row cancels."""
    n, r, c, v = random_coo(64, 0.08, seed=9)
    om = natural_matrix(oracle, n, r, c, v, vt=0)
    rng = np.random.default_rng(4)
    xh = rng.standard_normal(n).astype(F32)
    xl = (rng.standard_normal(n) * 2.0 ** -26).astype(F32)
    xdw = np.stack([xh, xl], axis=1).reshape(-1).copy()
    b = rng.standard_normal(n).astype(F32)
    got = om.residual(xdw, 2, b, 0, 2).astype(np.float64)
    A = scipy_csr(n, r, c, v.astype(F32).astype(np.float64))
    x64 = xh.astype(np.float64) + xl.astype(np.float64)
    exact = b.astype(np.float64) - A @ x64
    scale = np.abs(A) @ np.abs(x64) + np.abs(b)
    assert np.all(np.abs(got - exact) <= 2.0 ** -24 * np.abs(exact) + 2.0 ** -40 * scale)


@pytest.mark.parametrize("dilu", [False, True])
def test_oracle_ilu_matches_python_restatement(small_case, dilu):
    n, r, c, v, om = small_case
    rp, ci, od, dg = csr_parts(om)
    off, inv = om.ilu_factorize(dilu)
    poff, pinv = py_ilu0(rp, ci, od, dg, dilu)
    np.testing.assert_array_equal(off, poff)  # DILU leaves the off-diagonals as they are
    np.testing.assert_array_equal(inv, pinv)
    b = np.random.default_rng(6).standard_normal(n).astype(F32)
    np.testing.assert_array_equal(om.ilu_solve(off, inv, b, dilu),
                                  py_ilu_solve(rp, ci, off, inv, b, dilu))


def test_oracle_ilu_is_exact_lu_for_tridiagonal(oracle):
    """ILU(0) of a tridiagonal matrix has no fill-in, so it is the exact LU
    factorisation: one application solves the system (FP64 values)."""
    n = 50
    i = np.arange(n)
    rows = np.concatenate([i, i[1:], i[:-1]])
    cols = np.concatenate([i, i[1:] - 1, i[:-1] + 1])
    vals = np.concatenate([np.full(n, 4.0), np.full(n - 1, -1.0), np.full(n - 1, -1.5)])
    om = natural_matrix(oracle, n, rows, cols, vals, vt=1)
    off, inv = om.ilu_factorize(False)
    b = np.random.default_rng(8).standard_normal(n)
    x = om.ilu_solve(off, inv, b)
    A = scipy_csr(n, rows, cols, vals)
    np.testing.assert_allclose(A @ x, b, rtol=1e-12, atol=1e-12)


def test_oracle_gs_sweep_matches_python_restatement(small_case):
    n, r, c, v, om = small_case
    rng = np.random.default_rng(12)
    x = rng.standard_normal(n).astype(F32)
    b = rng.standard_normal(n).astype(F32)
    np.testing.assert_array_equal(om.gs_sweep(x, b, True),
                                  py_gs_sweep(*csr_parts(om), x, b))


@pytest.mark.parametrize("cfg,tol", [
    ({"type": "PBiCGStab", "maxIterations": 200, "relResidual": 1e-6,
      "preconditioner": {"type": "ILU"}}, 1e-4),
    ({"type": "PBiCGStab", "maxIterations": 200, "relResidual": 1e-6,
      "preconditioner": {"type": "GaussSeidel", "numFixedIterations": 2}}, 1e-4),
    ({"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 30,
      "extendedPrecisionType": "float64",
      "innerSolver": {"type": "PBiCGStab", "maxIterations": 100, "relResidual": 1e-4,
                      "preconditioner": {"type": "ILU"}}}, 1e-8),
])
def test_oracle_solvers_match_scipy(oracle, cfg, tol):
    import scipy.sparse.linalg as spla
    n, r, c, v = poisson_coo(8, 7, 6)
    tiles = np.arange(n, dtype=np.int32) * 4 // n
    om = oracle.matrix(n, r, c, v, 4, tiles, 0)
    xt = np.random.default_rng(0).uniform(-1, 1, n).astype(F32)
    l2g = tile_order(om)
    b_nat = (scipy_csr(n, r, c, v) @ xt.astype(np.float64))
    b = b_nat[l2g].astype(F32)
    x, st, phi, _ = om.solve(json.dumps(cfg), np.zeros(n, F32), b, want_phi=True)
    assert st.converged
    exact = spla.spsolve(scipy_csr(n, r, c, v).tocsc(), b.astype(np.float64)[np.argsort(l2g)])
    got = (phi if cfg["type"] == "IterativeRefinement" else x.astype(np.float64))
    sol = np.empty(n)
    sol[l2g] = got
    assert np.max(np.abs(sol - exact)) <= tol * max(1.0, np.max(np.abs(exact)))


# ---- the reference's FP32 reduction order (Expression::reduce) ------------------------

def _ref_reduce_py(tiles, square=False):
    """Expression::reduce restated stage by stage in numpy float32 scalars
    (dsl/tensor/Expression.cpp:472-481, :597-769; common/Shape.hpp:336-351):
    per-tile 6-worker chunks of floor(n/6/4)*4 (rest on worker 5), the 6
    partials, then runs of 368, 736, 1472 and all tiles."""
    f = np.float32

    def seq(vals, sq):
        acc = f(0)
        for v in vals:
            acc = f(acc + f(v * v)) if sq else f(acc + v)
        return acc

    def workers(vals, sq):
        cnt = len(vals)
        chunk = (cnt // 6 // 4) * 4
        parts = [seq(vals[chunk * w:(cnt if w == 5 else chunk * w + chunk)], sq) for w in range(6)]
        return seq(parts, False)

    total = sum(len(t) for t in tiles)
    vals = [workers(list(t), square) if total > 6 else seq(list(t), square) for t in tiles]
    at = list(range(len(tiles)))
    for G in (368, 736, 1472, None):
        if len(vals) <= 1:
            break
        keys, groups = [], []
        for k, v in enumerate(vals):
            g = 0 if G is None else at[k] // G * G
            if not keys or keys[-1] != g:
                keys.append(g)
                groups.append([])
            groups[-1].append(v)
        per_worker = any(len(g) > 6 for g in groups)
        vals = [workers(g, False) if per_worker else seq(g, False) for g in groups]
        at = keys
    return vals[0]


@pytest.mark.parametrize("dims,tiles", [((5, 1, 1), 1), ((6, 5, 4), 1), ((9, 8, 7), 5), ((20, 20, 20), 64),
                                        ((30, 30, 24), 400), ((40, 40, 30), 800), ((48, 40, 40), 1600)])
def test_reference_order_reduction(oracle, dims, tiles):
    """The oracle's reduction in the reference's order equals the stage-by-
    stage restatement bit for bit, for tile counts that exercise the 368 /
    736 / 1472 tile runs, for dot products, squared sums and signed sums."""
    from tests.oracle_py import Oracle
    import graphene_b200 as gb
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, *dims, tiles, gb.PART_RCB)
    om = oracle.poisson(*dims, tiles, h.rowToTile())
    starts = np.concatenate([[0], np.cumsum(om.tile_sizes().reshape(-1, 3)[:, :2].sum(1))])
    rng = np.random.default_rng(tiles)
    a = rng.uniform(-1, 1, om.n).astype(F32)
    b = rng.uniform(-1, 1, om.n).astype(F32)
    split = lambda v: [v[starts[t]:starts[t + 1]] for t in range(om.P)]  # noqa: E731
    want_dot = _ref_reduce_py(split((a * b).astype(F32)))
    assert om.ref_dot(a, b) == float(want_dot)
    want_sq = _ref_reduce_py(split(a), square=True)
    assert om.ref_norm(a, 1) == float(np.sqrt(want_sq))
    assert om.ref_norm(a, 0) == float(_ref_reduce_py(split(a)))
    assert om.ref_norm(a, 2) == float(a.max())
    # FP32 accumulation differs from the FP64 reduction by rounding only.
    assert abs(om.ref_dot(a, b) - float(np.dot(a.astype(np.float64), b.astype(np.float64)))) < 1e-3 * om.n ** 0.5


def test_reference_order_reduction_golden(oracle):
    """TensorTests.cpp:136-160 through the staged reduction: 0..15 in an 8x2
    tensor over 4 tiles, column sums 56 and 64 (exact in any order; the
    per-tile chunks are (2) on worker 5)."""
    data = np.arange(16, dtype=F32).reshape(8, 2)
    om = oracle.poisson(8, 1, 1, 4, np.repeat(np.arange(4, dtype=np.int32), 2))
    assert om.ref_norm(np.ascontiguousarray(data[:, 0]), 0) == 56.0
    assert om.ref_norm(np.ascontiguousarray(data[:, 1]), 0) == 64.0


def py_gs_sweep_working_f64(rp, ci, od, dg, x, b):
    """A Gauss-Seidel sweep with workingType float64 over float32 x
    (gauss-seidel/Solver.cpp:65-84): each row in double, stored as float."""
    x = x.copy()
    for i in range(len(dg)):
        s = np.float64(b[i])
        for p in range(rp[i], rp[i + 1]):
            s = s - np.float64(F32(od[p])) * np.float64(x[ci[p]])
        x[i] = F32(s / np.float64(F32(dg[i])))
    return x


def test_oracle_gs_float64_working_type(small_case):
    n, r, c, v, om = small_case
    rng = np.random.default_rng(15)
    x = rng.standard_normal(n).astype(F32)
    b = rng.standard_normal(n).astype(F32)
    cfg = json.dumps({"type": "GaussSeidel", "numFixedIterations": 2, "workingType": "float64"})
    got, _, _, _ = om.solve(cfg, x, b)
    parts = csr_parts(om)
    want = py_gs_sweep_working_f64(*parts, py_gs_sweep_working_f64(*parts, x, b), b)
    np.testing.assert_array_equal(got, want)


def test_oracle_reference_order_pbicgstab_converges(oracle):
    """The oracle's PBiCGStab with the reference's float reductions reaches
    the tolerance like the FP64-reduction one, with a similar count."""
    n, r, c, v = poisson_coo(10, 9, 8)
    tiles = np.arange(n, dtype=np.int32) * 6 // n
    om = oracle.matrix(n, r, c, v, 6, tiles, 0)
    b = om.spmv(np.random.default_rng(1).uniform(-1, 1, n).astype(F32))
    cfg = {"type": "PBiCGStab", "maxIterations": 300, "relResidual": 1e-6, "preconditioner": {"type": "ILU"}}
    _, st64, _, _ = om.solve(json.dumps(cfg), np.zeros(n, F32), b)
    _, st32, _, _ = om.solve(json.dumps(dict(cfg, reduce="f32_ref_order")), np.zeros(n, F32), b)
    assert st64.converged and st32.converged
    assert abs(st64.iterations - st32.iterations) <= 2
    assert np.float32(st32.final_residual) == st32.final_residual  # stored as float


def py_block_gs_drop(om, x, b):
    """One Gauss-Seidel sweep seeded with b whose halo cells read as 0
    ("halo": "drop"), tile by tile over the oracle's tile-local CRS (row
    pointers restart at 0 in every tile; columns at or past the tile's row
    count are halo cells), in float32."""
    rp, ci, od, dg = om.local_crs()
    sizes = om.tile_sizes()
    x = x.copy()
    base, rbase, ebase = 0, 0, 0  # row, row-pointer and entry offsets
    for t in range(sizes.shape[0]):
        nt = int(sizes[t, 0] + sizes[t, 1])
        for i in range(nt):
            s = F32(b[base + i])
            for p in range(ebase + rp[rbase + i], ebase + rp[rbase + i + 1]):
                c = int(ci[p])
                xv = x[base + c] if c < nt else F32(0)
                s = F32(s - F32(F32(od[p]) * xv))
            x[base + i] = F32(s / F32(dg[base + i]))
        base += nt
        ebase += int(rp[rbase + nt])
        rbase += nt + 1
    return x


@pytest.mark.parametrize("dims,tiles", [((8, 7, 6), 5), ((10, 10, 10), 12), ((9, 8, 7), 1)])
def test_oracle_gs_drop_halo_matches_restatement(oracle, dims, tiles):
    n = dims[0] * dims[1] * dims[2]
    om = oracle.poisson(*dims, tiles, np.arange(n, dtype=np.int32) * tiles // n)
    rng = np.random.default_rng(17)
    x = rng.uniform(-1, 1, n).astype(F32)
    b = rng.uniform(-1, 1, n).astype(F32)
    drop = om.gs_sweep(x, b, True, drop_halo=True)
    np.testing.assert_array_equal(drop, py_block_gs_drop(om, x, b))
    stale = om.gs_sweep(x, b, True)
    if tiles > 1:
        assert not np.array_equal(drop, stale)
    else:
        np.testing.assert_array_equal(drop, stale)
