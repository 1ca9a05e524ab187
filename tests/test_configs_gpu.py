"""Parity at the benchmark configurations' stated sizes, GPU against the
oracle, with the tolerances each comparison is held to.

* C1: 32^3 Poisson, 64 tiles, x_true ~ U[-1, 1) seed 0, FP32
  PBiCGStab-ILU(0) to 1e-6.
* C2: 128^3 upwind convection-diffusion, 1024 tiles, x_true ~ N(0, 1)
  seed 1, PBiCGStab with Gauss-Seidel (2 sweeps) and with ILU(0), FP32 and
  FP64, to 1e-8.
* C3: 192^3 variable-coefficient Poisson (sigma 1.5, seed 2), 2368 tiles,
  x_true seed 3: MPIR (FP64 residual and update, FP32 PBiCGStab-ILU(0)
  inner solves to 1e-4) to 1e-10.
* C4: the 100^3 jittered, permuted LDU mesh, 1024 tiles: LDU SpMV, a
  Gauss-Seidel sweep and the first PBiCGStab-GS iterations.

The oracle builds C1-C3 with its own generator and coordinate bisection
(oracle/generators.cpp; the tile maps are asserted equal to the library's);
C4's faces come from the library's mesh generator, which
tests/test_generators.py pins against an independent restatement.

Why iterates are compared within a tolerance and not bit for bit: every
kernel on the path is bit-exact against the oracle (SpMV, residual, ILU(0)
factorisation and substitution, Gauss-Seidel sweeps), but the PBiCGStab
dot products accumulate in FP64 in a different association order (per
block, then blocks, against the oracle's per tile, then tiles), so alpha and
omega differ in their last bits and the iterates drift apart slowly.
Stated tolerances:

* first k iterates (k <= 5): max |x - x_oracle| <= 1e-5 max |x_oracle|;
* converged solves: iteration counts within max(2, 4 %) of the oracle's,
  both final residuals at the target, and ||x - x_oracle|| / ||x_oracle||
  at most 1e-4 in FP32 and 1e-5 (1000 x the solver tolerance) in FP64: two
  solutions that both meet the 1e-8 residual lie up to about cond(A) x 1e-8
  apart, and C2's FP64 ILU(0) solve stops at 81 iterations against the
  oracle's 79, 1.7e-6 apart;
* MPIR (C3): the same outer count, inner counts within 4 %, both FP64
  relative residuals of phi <= 1e-10, ||phi - phi_oracle|| / ||phi_oracle||
  <= 1e-8.
"""
import json
import os

import numpy as np
import pytest

import graphene_b200 as gb
from tests.oracle_py import Oracle

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def orc():
    o = Oracle()
    o.threads(THREADS)
    return o


def pbicgstab(pre, maxit, tol):
    p = {"ILU": {"type": "ILU"},
         "GS": {"type": "GaussSeidel", "numSweeps": 2, "numFixedIterations": 2}}[pre]
    return {"type": "PBiCGStab", "maxIterations": maxit, "relResidual": tol, "preconditioner": p}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def its_close(a, b):
    return abs(a - b) <= max(2, 0.04 * max(a, b))


def report(name, **kv):
    print(f"[parity] {name}: " + ", ".join(f"{k}={v}" for k, v in kv.items()))


def solve_both(A, om, cfg, b, x0=None):
    x = dev(np.zeros_like(b) if x0 is None else x0)
    st = gb.Solver(A, cfg).solve(x, dev(b))
    xo, ost, _, hist = om.solve(json.dumps(cfg), np.zeros_like(b) if x0 is None else x0.copy(), b,
                                history_len=4096)
    return host(x), st, xo, ost, hist


# ---- C1 -------------------------------------------------------------------
def test_c1_exact_config(orc):
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 32, 32, 32, 64)
    om = orc.grid_system(0, 32, 32, 32, (), 0, 64)
    assert np.array_equal(om.row_to_tile(), h.rowToTile())
    A = h.copyToTile()
    xt = om.decompose(orc.random_vector(0, h.numRows).astype(np.float32))
    b = om.spmv(xt)
    np.testing.assert_array_equal(host(A * dev(xt)), b)  # b = A x_true, bit-exact
    cfg = pbicgstab("ILU", 1000, 1e-6)
    x, st, xo, ost, _ = solve_both(A, om, cfg, b)
    report("C1", gpu_it=st.iterations, oracle_it=ost.iterations, rel_x=rel(x, xo),
           gpu_res=st.finalResidual / st.initialResidual, oracle_res=ost.final_residual / ost.initial_residual)
    assert st.converged and ost.converged
    assert abs(st.iterations - ost.iterations) <= 1
    assert st.finalResidual <= 1e-6 * st.initialResidual
    assert rel(x, xo) <= 1e-4
    # The reference's own float reductions: the whole solve bit for bit.
    cfg_ref = dict(cfg, reduce="f32_ref_order")
    x, st, xo, ost, _ = solve_both(A, om, cfg_ref, b)
    report("C1 f32_ref_order", gpu_it=st.iterations, oracle_it=ost.iterations)
    assert st.iterations == ost.iterations and st.converged
    np.testing.assert_array_equal(x, xo)
    # First iterations, as iterates.
    for k in (1, 3, 5):
        x, st, xo, ost, _ = solve_both(A, om, pbicgstab("ILU", k, 0.0), b)
        assert st.iterations == ost.iterations == k
        assert np.abs(x - xo).max() <= 1e-5 * np.abs(xo).max()


# ---- C2 -------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2(orc):
    h = gb.generateMatrix(gb.GEN_CONVDIFF, 128, 128, 128, (0.5, 0.25, 0.125), 0, 1024)
    om32 = orc.grid_system(2, 128, 128, 128, (0.5, 0.25, 0.125), 0, 1024, 0)
    assert np.array_equal(om32.row_to_tile(), h.rowToTile())
    xt = orc.random_vector(1, h.numRows, "normal")
    return h, om32, xt


@pytest.mark.parametrize("vt", ["f32", "f64"])
@pytest.mark.parametrize("pre", ["GS", "ILU"])
def test_c2_convection_diffusion(orc, c2, pre, vt):
    h, om32, xt = c2
    if vt == "f32":
        hv, om, dt = h, om32, np.float32
    else:
        hv = h.astype(gb.FLOAT64)
        om = orc.grid_system(2, 128, 128, 128, (0.5, 0.25, 0.125), 0, 1024, 1)
        dt = np.float64
    A = hv.copyToTile()
    xtt = om.decompose(xt.astype(dt))
    b = om.spmv(xtt)
    np.testing.assert_array_equal(host(A * dev(xtt)), b)
    x, st, xo, ost, _ = solve_both(A, om, pbicgstab(pre, 2000, 1e-8), b)
    report(f"C2 {pre} {vt}", gpu_it=st.iterations, oracle_it=ost.iterations, rel_x=rel(x, xo),
           gpu_res=st.finalResidual / st.initialResidual, oracle_res=ost.final_residual / ost.initial_residual,
           conv=(st.converged, ost.converged))
    assert st.converged == ost.converged
    if st.converged:
        assert its_close(st.iterations, ost.iterations), (st.iterations, ost.iterations)
        assert st.finalResidual <= 1e-8 * st.initialResidual
    assert rel(x, xo) <= (1000 * 1e-8 if vt == "f64" else 1e-4)
    for k in (1, 5):
        x, st, xo, ost, _ = solve_both(A, om, pbicgstab(pre, k, 0.0), b)
        assert st.iterations == ost.iterations == k
        assert np.abs(x - xo).max() <= 1e-5 * np.abs(xo).max()


# ---- C3 -------------------------------------------------------------------
def test_c3_mpir_full_size(orc):
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 192, 192, 192, (1.5,), 2, 2368)
    om = orc.grid_system(1, 192, 192, 192, (1.5,), 2, 2368)
    assert np.array_equal(om.row_to_tile(), h.rowToTile())
    A = h.copyToTile()
    n = h.numRows
    b = om.spmv(om.decompose(orc.random_vector(3, n).astype(np.float32)))
    cfg = {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 50,
           "extendedPrecisionType": "float64",
           "innerSolver": {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-4,
                           "preconditioner": {"type": "ILU"}}}
    solver = gb.Solver(A, cfg)
    x = dev(np.zeros(n, np.float32))
    st = solver.solve(x, dev(b))
    phi = host(solver.phi(gb.FLOAT64))
    xo, ost, phio, _ = om.solve(json.dumps(cfg), np.zeros(n, np.float32), b, want_phi=True)
    bn = np.linalg.norm(b.astype(np.float64))
    r_gpu = np.linalg.norm(om.residual(phi, 1, b, 1, 1)) / bn  # FP64 residual by the oracle
    r_or = np.linalg.norm(om.residual(phio, 1, b, 1, 1)) / bn
    report("C3 MPIR", gpu=(st.iterations, st.innerIterations), oracle=(ost.iterations, ost.inner_iterations),
           r_gpu=r_gpu, r_oracle=r_or, rel_phi=rel(phi, phio))
    assert st.converged and ost.converged
    assert st.iterations == ost.iterations
    assert abs(st.innerIterations - ost.inner_iterations) <= 0.04 * ost.inner_iterations
    assert r_gpu <= 1e-10 and r_or <= 1e-10
    assert rel(phi, phio) <= 1e-8
    np.testing.assert_array_equal(host(x), phi.astype(np.float32))


# ---- C4 -------------------------------------------------------------------
@pytest.fixture(scope="module")
def c4(orc):
    h = gb.generateLduMesh(100, 100, 100, 4, 5, 6, numTiles=1024)
    o, nb, lo, up, dg = h.ldu()
    om = orc.ldu(h.numRows, o, nb, dg, lo, up, h.numTiles, h.rowToTile(), 0)
    return h, om


def test_c4_ldu_spmv_and_sweep_full_size(c4):
    h, om = c4
    A = h.copyToTile()
    x = om.decompose(gb.randomVector(41, h.numRows, "normal").astype(np.float32))
    np.testing.assert_array_equal(host(A * dev(x)), om.spmv(x))
    b = om.spmv(x)
    y = dev(np.zeros_like(b))
    gb.Solver(A, {"type": "GaussSeidel", "numFixedIterations": 2}).solve(y, dev(b))
    ref = np.zeros_like(b)
    for _ in range(2):
        ref = om.gs_sweep(ref, b, seed_b=True)
    np.testing.assert_array_equal(host(y), ref)


def test_c4_ldu_gs_pbicgstab_iterates(c4):
    h, om = c4
    A = h.copyToTile()
    xt = om.decompose(gb.randomVector(1, h.numRows, "normal").astype(np.float32))
    b = om.spmv(xt)
    for k in (1, 5):
        x, st, xo, ost, _ = solve_both(A, om, pbicgstab("GS", k, 0.0), b)
        assert st.iterations == ost.iterations == k
        assert np.abs(x - xo).max() <= 1e-5 * np.abs(xo).max()
    # 60 iterations: the residual histories stay together (relative 1e-3).
    cfg = pbicgstab("GS", 60, 0.0)
    x, st, xo, ost, hist = solve_both(A, om, cfg, b)
    report("C4 GS 60 it", gpu_res=st.finalResidual, oracle_res=ost.final_residual, rel_x=rel(x, xo))
    assert st.finalResidual == pytest.approx(ost.final_residual, rel=1e-3)
    assert rel(x, xo) <= 1e-4
