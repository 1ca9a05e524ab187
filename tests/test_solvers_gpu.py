"""Solvers on the GPU through the C ABI, against the oracle.

* ILU(0) / DILU factorisation + substitution and Gauss-Seidel sweeps follow
  the reference's per-row operation order exactly: bit-exact.
* PBiCGStab / MPIR iterates differ from the oracle only through the order of
  the FP64 dot-product sums; after k <= 5 iterations x agrees to 1e-5
  (relative, max norm), and converged solves agree in iteration count to +-2
  and in the solution to the stated solver tolerance.
* Final accuracy is checked against an FP64 ground truth (scipy).
"""
import json

import numpy as np
import pytest

import graphene_b200 as gb
from tests.util import random_coo

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def case(name, oracle, vt=gb.FLOAT32):
    ovt = 0 if vt == gb.FLOAT32 else 1
    if name == "poisson16":
        h = gb.generate3DPoissonMatrix(vt, 16, 16, 16, 8)
        return h, oracle.poisson(16, 16, 16, 8, h.rowToTile(), ovt)
    if name == "poisson_odd_bfs":
        h = gb.generate3DPoissonMatrix(vt, 13, 11, 7, 6, gb.PART_BFS)
        return h, oracle.poisson(13, 11, 7, 6, h.rowToTile(), ovt)
    if name == "poisson_1tile":
        h = gb.generate3DPoissonMatrix(vt, 12, 10, 8, 1)
        return h, oracle.poisson(12, 10, 8, 1, None, ovt)
    if name == "random":
        n, r, c, v = random_coo(600, 0.01, 4)
        h = gb.HostMatrix.from_coo(n, r, c, v, 7, partitioner=gb.PART_BFS, valueType=vt)
        return h, oracle.matrix(n, r, c, v, 7, h.rowToTile(), ovt)
    if name == "many_tiles":
        h = gb.generate3DPoissonMatrix(vt, 20, 20, 20, 200)
        return h, oracle.poisson(20, 20, 20, 200, h.rowToTile(), ovt)
    raise KeyError(name)


NAMES = ["poisson16", "poisson_odd_bfs", "poisson_1tile", "random", "many_tiles"]


def ilu_config(kernel, **kw):
    """'ring_wide': the ring kernel with 32-bit row and column ids;
    'ring_rec': with 16-byte row records for levels of 3 entries a row;
    'ring_noprod': records, the waiting warp issuing the copies."""
    c = {"type": "ILU", "kernel": "ring" if kernel in ("ring_wide", "ring_rec", "ring_pair", "ring_cw4", "ring_cw1",
                                                        "ring_nowait", "ring_noprod") else kernel}
    if kernel == "ring_nowait":
        c["waitingWarp"] = False
    if kernel == "ring_noprod":
        c["producerWarp"] = False
    if kernel in ("ring_cw4", "ring_cw1"):
        c["computeWarps"] = int(kernel[-1])
    if kernel.startswith("wring"):
        c["kernel"] = "wring"
    if kernel == "ring_wide":
        c["compactRing"] = False
    # Record levels are the default; the plain names run without them.
    c["recordLevels"] = kernel in ("ring_rec", "ring_pair", "ring_cw4", "ring_cw1", "ring_nowait", "ring_noprod", "wring_rec",
                                   "wring_pair", "wring_w4")
    if kernel in ("ring_pair", "wring_pair"):
        c["pairRows"] = True
    if kernel == "wring_w4":
        c["warpsPerBlock"] = 4
    c.update(kw)
    return c


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dilu", [False, True])
@pytest.mark.parametrize("kernel", ["ring", "ring_rec", "ring_pair", "ring_wide", "ring_cw4", "ring_cw1", "ring_nowait",
                                    "ring_noprod", "wring", "wring_rec", "wring_pair",
                                    "wring_w4", "warp", "tma", "levels"])
def test_ilu_bit_exact(oracle, name, dilu, kernel):
    h, om = case(name, oracle)
    A = h.copyToTile()
    b = np.random.default_rng(3).uniform(-1, 1, h.numRows).astype(np.float32)
    x = A.createUninitializedVector(gb.FLOAT32)
    gb.Solver(A, ilu_config(kernel, diagonalBased=dilu)).solve(x, dev(b))
    off, inv = om.ilu_factorize(dilu)
    np.testing.assert_array_equal(host(x), om.ilu_solve(off, inv, b, dilu))


@pytest.mark.parametrize("name", ["poisson16", "random"])
@pytest.mark.parametrize("kernel", ["ring", "ring_rec", "ring_pair", "ring_wide", "wring", "wring_pair", "warp", "tma",
                                    "levels"])
def test_ilu_bit_exact_float64(oracle, name, kernel):
    h, om = case(name, oracle, gb.FLOAT64)
    A = h.copyToTile()
    b = np.random.default_rng(4).standard_normal(h.numRows)
    x = A.createUninitializedVector(gb.FLOAT64)
    gb.Solver(A, ilu_config(kernel)).solve(x, dev(b))
    off, inv = om.ilu_factorize(False)
    np.testing.assert_array_equal(host(x), om.ilu_solve(off, inv, b, False))


@pytest.mark.parametrize("name", ["poisson16", "many_tiles", "random", "poisson_odd_bfs"])
@pytest.mark.parametrize("group", [2, 3, 8])
@pytest.mark.parametrize("dilu", [False, True])
@pytest.mark.parametrize("warps", ["default", "cw4", "cw8", "cw4_noprod"])
def test_ilu_ring_tile_groups_bit_exact(oracle, name, group, dilu, warps):
    """Several tiles per thread block, run level by level in lockstep, with
    2, 4 or 8 compute warps, with or without the producer warp: same bits."""
    h, om = case(name, oracle)
    A = h.copyToTile()
    b = np.random.default_rng(7).uniform(-1, 1, h.numRows).astype(np.float32)
    x = A.createUninitializedVector(gb.FLOAT32)
    cfg = {"type": "ILU", "kernel": "ring", "tilesPerBlock": group, "diagonalBased": dilu}
    if warps != "default":
        cfg["computeWarps"] = int(warps[2])
    if warps.endswith("noprod"):
        cfg["producerWarp"] = False
    gb.Solver(A, cfg).solve(x, dev(b))
    off, inv = om.ilu_factorize(dilu)
    np.testing.assert_array_equal(host(x), om.ilu_solve(off, inv, b, dilu))


@pytest.mark.parametrize("name", ["poisson16", "many_tiles", "random"])
@pytest.mark.parametrize("frac", [0.0, 0.35, 0.6])
def test_ilu_ring_small_rings_bit_exact(oracle, name, frac):
    """Rings from a few level blocks up: wrap-around placement and barrier
    reuse in the host-scheduled ring kernel give the same bits."""
    import ctypes as C
    h, om = case(name, oracle)
    used = C.c_int64()
    gb._lib.check(gb._lib.lib().gr_host_matrix_check_ilu_ring(h._h, 0, gb.FLOAT32, 0, 1, 1, C.byref(used), None, None))
    rb = 0 if frac == 0.0 else max(16, int(used.value * frac) // 16 * 16)
    A = h.copyToTile()
    b = np.random.default_rng(6).uniform(-1, 1, h.numRows).astype(np.float32)
    x = A.createUninitializedVector(gb.FLOAT32)
    try:
        s = gb.Solver(A, {"type": "ILU", "kernel": "ring", "ringBytes": rb})
    except gb.GrapheneError as e:
        assert "too small" in str(e)
        return
    s.solve(x, dev(b))
    off, inv = om.ilu_factorize(False)
    np.testing.assert_array_equal(host(x), om.ilu_solve(off, inv, b, False))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("sweeps", [1, 2, 3])
@pytest.mark.parametrize("seed", ["b", "diag"])
@pytest.mark.parametrize("kernel", ["ring", "ring_rec", "wring", "wring_rec", "wring_pair", "wring_rec_pair",
                                    "levels"])
def test_gauss_seidel_bit_exact(oracle, name, sweeps, seed, kernel):
    """'_rec': record levels; '_pair': the warp ring with two rows a lane at
    once (pairRows)."""
    h, om = case(name, oracle)
    A = h.copyToTile()
    rng = np.random.default_rng(5)
    b = rng.uniform(-1, 1, h.numRows).astype(np.float32)
    x0 = rng.uniform(-1, 1, h.numRows).astype(np.float32)
    x = dev(x0)
    cfg = {"type": "GaussSeidel", "numFixedIterations": sweeps, "seed": seed,
           "kernel": kernel.split("_")[0], "recordLevels": "_rec" in kernel,
           "pairRows": kernel.endswith("_pair")}
    gb.Solver(A, cfg).solve(x, dev(b))
    ref = x0
    for _ in range(sweeps):
        ref = om.gs_sweep(ref, b, seed_b=(seed == "b"))
    np.testing.assert_array_equal(host(x), ref)


@pytest.mark.parametrize("name", ["poisson16", "poisson_odd_bfs", "many_tiles"])
@pytest.mark.parametrize("kernel", ["ring", "wring", "levels"])
@pytest.mark.parametrize("start", ["x0", "zero"])
def test_gauss_seidel_drop_halo_bit_exact(oracle, name, kernel, start):
    """"halo": "drop": the halo cells read as 0 in every sweep (block
    Gauss-Seidel); two sweeps, from a nonzero x and from x = 0, same bits as
    the oracle's sweep with the halo zeroed."""
    h, om = case(name, oracle)
    A = h.copyToTile()
    rng = np.random.default_rng(13)
    b = rng.uniform(-1, 1, h.numRows).astype(np.float32)
    x0 = rng.uniform(-1, 1, h.numRows).astype(np.float32) if start == "x0" else np.zeros(h.numRows, np.float32)
    x = dev(x0)
    cfg = {"type": "GaussSeidel", "numFixedIterations": 2, "kernel": kernel, "halo": "drop"}
    gb.Solver(A, cfg).solve(x, dev(b))
    ref = x0
    for _ in range(2):
        ref = om.gs_sweep(ref, b, drop_halo=True)
    np.testing.assert_array_equal(host(x), ref)
    if h.numTiles > 1 and start == "x0":
        stale = x0
        for _ in range(2):
            stale = om.gs_sweep(stale, b)
        assert not np.array_equal(ref, stale)


@pytest.mark.parametrize("name", ["poisson16", "random", "many_tiles"])
@pytest.mark.parametrize("vt", ["f32", "f64", "f32_matrix_f64_vectors"])
@pytest.mark.parametrize("kernel", ["ring", "wring"])
def test_gauss_seidel_ring_types_bit_exact(oracle, name, vt, kernel):
    """The level-ring sweep with float64 vectors (float32 or float64
    coefficients): same bits as the oracle."""
    mt = gb.FLOAT64 if vt == "f64" else gb.FLOAT32
    h, om = case(name, oracle, mt)
    A = h.copyToTile()
    rng = np.random.default_rng(9)
    dt = np.float32 if vt == "f32" else np.float64
    b = rng.uniform(-1, 1, h.numRows).astype(dt)
    x0 = rng.uniform(-1, 1, h.numRows).astype(dt)
    x = dev(x0)
    gb.Solver(A, {"type": "GaussSeidel", "numFixedIterations": 2, "kernel": kernel}).solve(x, dev(b))
    ref = om.gs_sweep(om.gs_sweep(x0, b), b)
    np.testing.assert_array_equal(host(x), ref)


@pytest.mark.parametrize("name", ["poisson16", "random", "many_tiles", "poisson_odd_bfs"])
@pytest.mark.parametrize("sweeps", [1, 2, 3])
@pytest.mark.parametrize("records", [False, True])
@pytest.mark.parametrize("kernel", ["ring", "wring", "wring_pair"])
def test_gauss_seidel_ring_from_zero_bit_exact(oracle, name, sweeps, records, kernel):
    """Sweeps from x = 0 (the first one through the lower-only ring), as a
    PBiCGStab preconditioner applies them: same bits as the oracle's full
    sweeps from zero."""
    h, om = case(name, oracle)
    A = h.copyToTile()
    b = np.random.default_rng(10).uniform(-1, 1, h.numRows).astype(np.float32)
    cfg = {"type": "GaussSeidel", "numFixedIterations": sweeps, "kernel": kernel.split("_")[0],
           "recordLevels": records, "pairRows": kernel == "wring_pair"}
    x = dev(np.zeros_like(b))
    gb.Solver(A, cfg).solve(x, dev(b))
    ref = np.zeros_like(b)
    for _ in range(sweeps):
        ref = om.gs_sweep(ref, b)
    np.testing.assert_array_equal(host(x), ref)


def test_gauss_seidel_converges_with_checks(oracle):
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    b = np.ones(h.numRows, np.float32)
    cfg = {"type": "GaussSeidel", "numSweeps": 3, "maxIterations": 300, "relResidual": 1e-3}
    x = dev(np.zeros(h.numRows, np.float32))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros(h.numRows, np.float32), b)
    assert st.converged and ost.converged
    assert st.iterations == ost.iterations
    np.testing.assert_array_equal(host(x), xo)
    assert st.finalResidual == pytest.approx(ost.final_residual, rel=1e-12)


PCFG = {
    "ilu": {"type": "ILU"},
    "ilu_levels": {"type": "ILU", "kernel": "levels"},
    "ilu_tma": {"type": "ILU", "kernel": "tma"},
    "ilu_ring": {"type": "ILU", "kernel": "ring"},
    "dilu": {"type": "ILU", "diagonalBased": True},
    "gs2": {"type": "GaussSeidel", "numFixedIterations": 2},
    "gs2_levels": {"type": "GaussSeidel", "numFixedIterations": 2, "kernel": "levels"},
    "gs3_diag": {"type": "GaussSeidel", "numFixedIterations": 3, "seed": "diag"},
    "none": None,
}


def pbicgstab(pre, maxit, tol=0.0, **kw):
    c = {"type": "PBiCGStab", "maxIterations": maxit, "relResidual": tol}
    c.update(kw)
    if PCFG[pre] is not None:
        c["preconditioner"] = PCFG[pre]
    return c


@pytest.mark.parametrize("pre", list(PCFG))
@pytest.mark.parametrize("k", [1, 2, 5])
def test_pbicgstab_first_iterations_match(oracle, pre, k):
    h, om = case("poisson_odd_bfs", oracle)
    A = h.copyToTile()
    xt = np.random.default_rng(0).uniform(-1, 1, h.numRows).astype(np.float32)
    b = om.spmv(xt)
    cfg = pbicgstab(pre, k)
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.iterations == ost.iterations == k
    scale = np.abs(xo).max()
    assert np.abs(host(x) - xo).max() <= 1e-5 * scale
    assert st.finalResidual == pytest.approx(ost.final_residual, rel=1e-3)


@pytest.mark.parametrize("name", ["poisson16", "random", "many_tiles", "poisson_1tile"])
@pytest.mark.parametrize("pre", ["ilu", "dilu", "gs2", "none"])
def test_pbicgstab_converges_like_oracle(oracle, name, pre):
    h, om = case(name, oracle)
    A = h.copyToTile()
    xt = np.random.default_rng(1).uniform(-1, 1, h.numRows).astype(np.float32)
    b = om.spmv(xt)
    cfg = pbicgstab(pre, 1000, 1e-6)
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.converged and ost.converged
    assert abs(st.iterations - ost.iterations) <= 2, (st.iterations, ost.iterations)
    assert st.finalResidual < 1e-6 * st.initialResidual
    err = np.abs(host(x) - xt).max() / np.abs(xt).max()
    assert err < 1e-3


def test_pbicgstab_float64(oracle):
    h, om = case("poisson16", oracle, gb.FLOAT64)
    A = h.copyToTile()
    xt = np.random.default_rng(2).uniform(-1, 1, h.numRows)
    b = om.spmv(xt)
    cfg = pbicgstab("ilu", 1000, 1e-12)
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.converged and ost.converged
    assert abs(st.iterations - ost.iterations) <= 1
    np.testing.assert_allclose(host(x), xt, rtol=0, atol=1e-9)


def test_pbicgstab_float32_matrix_float64_vectors(oracle):
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    xt = np.random.default_rng(2).uniform(-1, 1, h.numRows)
    b = om.spmv(xt)
    cfg = pbicgstab("ilu", 1000, 1e-12)
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    assert st.converged
    np.testing.assert_allclose(host(x), xt, rtol=0, atol=1e-9)


@pytest.mark.parametrize("ext", ["float64", "twofloat32", "float32"])
def test_mpir_matches_oracle_and_fp64_truth(oracle, ext):
    import scipy.sparse as sp
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    n = h.numRows
    xt = np.random.default_rng(3).uniform(-1, 1, n).astype(np.float32)
    b = om.spmv(xt)
    target = 1e-10 if ext != "float32" else 1e-6
    cfg = {"type": "IterativeRefinement", "relResidual": target, "maxIterations": 30,
           "extendedPrecisionType": ext,
           "innerSolver": pbicgstab("ilu", 200, 1e-4)}
    solver = gb.Solver(A, cfg)
    x = dev(np.zeros(n, np.float32))
    st = solver.solve(x, dev(b))
    xo, ost, phio, _ = om.solve(json.dumps(cfg), np.zeros(n, np.float32), b, want_phi=True)
    assert st.converged and ost.converged, (st, ost)
    assert abs(st.iterations - ost.iterations) <= 1
    phi = host(solver.phi(gb.FLOAT64))
    # FP64 residual of phi on the stored (float32) matrix; the FP64 residual
    # kernel is itself bit-exact against the oracle (test_spmv_gpu).
    r = A.residual(dev(phi), dev(b), destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
    rel = np.linalg.norm(host(r)) / np.linalg.norm(b.astype(np.float64))
    if ext != "float32":
        assert rel < 1e-9
        np.testing.assert_allclose(phi, phio, rtol=0, atol=1e-8)
    np.testing.assert_allclose(host(x), phi.astype(np.float32), rtol=0, atol=0)


def test_restarter(oracle):
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    xt = np.random.default_rng(4).uniform(-1, 1, h.numRows).astype(np.float32)
    b = om.spmv(xt)
    cfg = {"type": "restarter", "maxRestarts": 20, "innerSolver": pbicgstab("ilu", 3, 1e-6)}
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.converged == ost.converged
    assert abs(st.innerIterations - ost.inner_iterations) <= 3


def test_zero_rhs_is_singular(oracle):
    """b = 0 and x0 = 0: rho = 0 is singular before the first iteration
    (pbicgstab/Solver.cpp:91-96)."""
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    b = np.zeros(h.numRows, np.float32)
    x = dev(b)
    st = gb.Solver(A, pbicgstab("ilu", 100, 1e-6)).solve(x, dev(b))
    _, ost, _, _ = om.solve(json.dumps(pbicgstab("ilu", 100, 1e-6)), b.copy(), b)
    assert st.singular and ost.singular
    assert st.iterations == ost.iterations == 0


def test_solve_host_natural_order(oracle):
    h, om = case("poisson_odd_bfs", oracle)
    A = h.copyToTile()
    xt_nat = np.random.default_rng(5).uniform(-1, 1, h.numRows).astype(np.float32)
    b_nat = h.composeVector(om.spmv(h.decomposeVector(xt_nat)))
    solver = gb.Solver(A, pbicgstab("ilu", 500, 1e-7))
    x = np.zeros_like(b_nat)
    st = solver.solveHost(x, b_nat)
    assert st.converged
    assert np.abs(x - xt_nat).max() < 1e-4


def test_solver_reuse_is_deterministic(oracle):
    h, om = case("many_tiles", oracle)
    A = h.copyToTile()
    b = dev(np.random.default_rng(6).uniform(-1, 1, h.numRows).astype(np.float32))
    solver = gb.Solver(A, pbicgstab("ilu", 1000, 1e-6))
    outs = []
    for _ in range(3):
        x = dev(np.zeros(h.numRows, np.float32))
        st = solver.solve(x, b)
        outs.append((host(x), st.iterations, st.finalResidual))
    for o in outs[1:]:
        np.testing.assert_array_equal(o[0], outs[0][0])
        assert o[1:] == outs[0][1:]


def test_launch_counter_counts_graph_replays():
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 12, 12, 12, 4)
    A = h.copyToTile()
    b = dev(np.ones(h.numRows, np.float32))
    solver = gb.Solver(A, pbicgstab("ilu", 1000, 1e-6))
    x = dev(np.zeros(h.numRows, np.float32))
    c0 = gb.launch_count()
    st = solver.solve(x, b)
    used = gb.launch_count() - c0
    assert st.converged
    assert used >= 5 * st.iterations


def test_time_repeated_runs_the_same_application(oracle):
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    b = np.random.default_rng(8).uniform(-1, 1, h.numRows).astype(np.float32)
    s = gb.Solver(A, {"type": "ILU"})
    x = A.createUninitializedVector(gb.FLOAT32)
    ms = s.timeRepeated(x, dev(b), 5)
    assert ms > 0
    off, inv = om.ilu_factorize(False)
    np.testing.assert_array_equal(host(x), om.ilu_solve(off, inv, b, False))
    with pytest.raises(gb.GrapheneError):
        gb.Solver(A, pbicgstab("ilu", 5)).timeRepeated(x, dev(b), 2)


@pytest.mark.parametrize("name", ["poisson16", "poisson_odd_bfs", "random", "many_tiles", "poisson_1tile"])
@pytest.mark.parametrize("pre", ["ilu", "gs2", "dilu", "none"])
def test_pbicgstab_reference_order_bit_exact(oracle, name, pre):
    """"reduce": "f32_ref_order": dot products and norms in the reference's
    float reduction order (Expression.cpp:472-481, :597-769), alpha, beta,
    omega and the convergence test in float. Every other step is already
    bit-exact, so whole solves agree with the oracle bit for bit: same
    iteration count, same solution, same residual norms."""
    h, om = case(name, oracle)
    A = h.copyToTile()
    xt = np.random.default_rng(11).uniform(-1, 1, h.numRows).astype(np.float32)
    b = om.spmv(xt)
    cfg = pbicgstab(pre, 1000, 1e-6, reduce="f32_ref_order")
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.converged and ost.converged
    assert st.iterations == ost.iterations
    np.testing.assert_array_equal(host(x), xo)
    assert st.finalResidual == ost.final_residual and st.initialResidual == ost.initial_residual


@pytest.mark.parametrize("norm", ["L1", "LINF"])
def test_pbicgstab_reference_order_other_norms(oracle, norm):
    h, om = case("many_tiles", oracle)
    A = h.copyToTile()
    b = om.spmv(np.random.default_rng(12).uniform(-1, 1, h.numRows).astype(np.float32))
    cfg = pbicgstab("ilu", 1000, 1e-5, reduce="f32_ref_order", norm=norm, relTolerance=1e-6)
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.iterations == ost.iterations
    np.testing.assert_array_equal(host(x), xo)


def test_reference_order_rejects_float64_vectors(oracle):
    h, _ = case("poisson16", oracle, gb.FLOAT64)
    A = h.copyToTile()
    b = dev(np.ones(h.numRows))
    with pytest.raises(gb.GrapheneError):
        gb.Solver(A, pbicgstab("ilu", 10, 1e-6, reduce="f32_ref_order")).solve(dev(np.zeros(h.numRows)), b)


@pytest.mark.parametrize("name", ["poisson16", "random", "many_tiles"])
@pytest.mark.parametrize("sweeps", [1, 3])
def test_gauss_seidel_float64_working_type_bit_exact(oracle, name, sweeps):
    """GaussSeidel "workingType": "float64" over float32 x and b: each row
    computed in double and stored as float (gauss-seidel/Solver.cpp:65-84)."""
    h, om = case(name, oracle)
    A = h.copyToTile()
    rng = np.random.default_rng(13)
    b = rng.uniform(-1, 1, h.numRows).astype(np.float32)
    x0 = rng.uniform(-1, 1, h.numRows).astype(np.float32)
    cfg = {"type": "GaussSeidel", "numFixedIterations": sweeps, "workingType": "float64"}
    x = dev(x0)
    gb.Solver(A, cfg).solve(x, dev(b))
    xo, _, _, _ = om.solve(json.dumps(cfg), x0.copy(), b)
    np.testing.assert_array_equal(host(x), xo)
    # It differs from the float32 sweep (the working type matters).
    xf, _, _, _ = om.solve(json.dumps({"type": "GaussSeidel", "numFixedIterations": sweeps}), x0.copy(), b)
    assert not np.array_equal(xo, xf)


def test_gauss_seidel_float64_working_type_with_checks(oracle):
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    b = np.ones(h.numRows, np.float32)
    cfg = {"type": "GaussSeidel", "numSweeps": 2, "maxIterations": 300, "relResidual": 1e-4,
           "workingType": "float64"}
    x = dev(np.zeros(h.numRows, np.float32))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros(h.numRows, np.float32), b)
    assert st.converged and ost.converged and st.iterations == ost.iterations
    np.testing.assert_array_equal(host(x), xo)


@pytest.mark.parametrize("pre", ["ilu", "gs2", "none"])
def test_pbicgstab_float64_working_type(oracle, pre):
    """PBiCGStab "workingType": "float64" over float32 x and b
    (pbicgstab/Solver.cpp:63-79): the Krylov vectors in double, x rounded to
    float at every update; iterates as close to the oracle's as the FP64
    reductions allow, and a solution closer to the FP64 truth than a float32
    working type can reach."""
    h, om = case("poisson16", oracle)
    A = h.copyToTile()
    xt = np.random.default_rng(14).uniform(-1, 1, h.numRows).astype(np.float32)
    b = om.spmv(xt)
    for k in (1, 3):
        cfg = pbicgstab(pre, k, 0.0, workingType="float64")
        x = dev(np.zeros_like(b))
        st = gb.Solver(A, cfg).solve(x, dev(b))
        xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
        assert st.iterations == ost.iterations == k
        assert np.abs(host(x) - xo).max() <= 1e-6 * np.abs(xo).max()
    cfg = pbicgstab(pre, 1000, 1e-9, workingType="float64")
    x = dev(np.zeros_like(b))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, _ = om.solve(json.dumps(cfg), np.zeros_like(b), b)
    assert st.converged and ost.converged
    assert abs(st.iterations - ost.iterations) <= 2
    assert host(x).dtype == np.float32
    np.testing.assert_allclose(host(x), xo, rtol=0, atol=2e-6 * np.abs(xo).max())
