"""Solve server (gr_server_*): continuous batching on one GPU.

Each result must be identical whether the request runs alone or in a mix of
concurrent requests (the kernels are deterministic and every request has
its own buffers); requests overlap on the device; resident pairs are reused;
admission respects the memory budget; a failing request does not disturb
the others.
"""
import time

import numpy as np
import pytest

import graphene_b200 as gb

pytestmark = pytest.mark.gpu

ILU = {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-6, "preconditioner": {"type": "ILU"}}
MPIR = {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 30,
        "extendedPrecisionType": "float64",
        "innerSolver": {"type": "PBiCGStab", "maxIterations": 300, "relResidual": 1e-4,
                        "preconditioner": {"type": "ILU"}}}


def workload():
    out = []
    # Tiles of 16,000 and 23,328 rows need different dynamic shared memory
    # above the 48 KB default: concurrent launches must not undo each
    # other's limit.
    for i, (L, tiles, cfg) in enumerate([(20, 8, ILU), (28, 16, MPIR), (16, 4, ILU), (40, 4, ILU),
                                         (32, 32, MPIR), (36, 2, ILU), (18, 6, ILU)]):
        h = gb.generateMatrix(gb.GEN_VAR_POISSON, L, L, L, (1.0,), 10 + i, tiles)
        b = gb.randomVector(100 + i, h.numRows).astype(np.float32)
        out.append((h, cfg, b))
    return out


def alone(h, cfg, b):
    A = h.copyToTile()
    x = np.zeros(h.numRows, np.float32)
    st = gb.Solver(A, cfg).solveHost(x, b)
    return x, st


def test_results_in_the_mix_equal_results_alone():
    work = workload()
    ref = [alone(*w) for w in work]
    srv = gb.Server(slots=4)
    ids = [srv.submit(h, cfg, b) for h, cfg, b in work]
    res = [srv.wait(i) for i in ids]
    for (x, st, tm), (xr, str_) in zip(res, ref):
        np.testing.assert_array_equal(x, xr)
        assert st.converged and st.iterations == str_.iterations
    # Work overlapped: some request was admitted before another finished.
    spans = sorted((tm["admitted_ms"], tm["finished_ms"]) for _, _, tm in res)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    assert len({tm["slot"] for _, _, tm in res}) > 1
    srv.close()


def test_requests_admitted_while_others_run_and_resident_reuse():
    work = workload()
    srv = gb.Server(slots=2)
    first = [srv.submit(h, cfg, b) for h, cfg, b in work[:2]]
    time.sleep(0.005)
    later = [srv.submit(h, cfg, b) for h, cfg, b in work[2:4]]
    r1 = [srv.wait(i) for i in first + later]
    assert all(tm["cache_hit"] == 0 for _, _, tm in r1)
    # The same pairs again: resident, no upload or factorisation, same result.
    again = [srv.submit(h, cfg, b) for h, cfg, b in work[:4]]
    r2 = [srv.wait(i) for i in again]
    for (x1, _, _), (x2, _, tm) in zip(r1, r2):
        assert tm["cache_hit"] == 1
        np.testing.assert_array_equal(x1, x2)
    c = srv.counters()
    assert c["completed"] == 8 and c["queued"] == 0 and c["running"] == 0 and c["resident"] == 4
    srv.close()


def test_tiny_budget_runs_one_request_at_a_time():
    work = workload()[:4]
    srv = gb.Server(slots=4, budgetBytes=1)
    ids = [srv.submit(h, cfg, b) for h, cfg, b in work]
    res = [srv.wait(i) for i in ids]
    spans = sorted((tm["admitted_ms"], tm["finished_ms"]) for _, _, tm in res)
    assert all(spans[k + 1][0] >= spans[k][1] for k in range(len(spans) - 1))
    for (x, _, _), w in zip(res, work):
        np.testing.assert_array_equal(x, alone(*w)[0])
    assert srv.counters()["resident"] == 1  # each admission evicted the idle pair before it
    srv.close()


def test_failing_request_leaves_the_others_intact():
    work = workload()[:3]
    srv = gb.Server(slots=2)
    bad_cfg = {"type": "PBiCGStab", "preconditioner": {"type": "GaussSeidel"}}  # needs numFixedIterations
    ids = [srv.submit(work[0][0], bad_cfg, work[0][2])] + [srv.submit(h, cfg, b) for h, cfg, b in work[1:]]
    with pytest.raises(gb.GrapheneError):
        srv.wait(ids[0])
    for i, w in zip(ids[1:], work[1:]):
        x, st, _ = srv.wait(i)
        np.testing.assert_array_equal(x, alone(*w)[0])
    with pytest.raises(gb.GrapheneError):
        srv.submit(work[0][0], {"type": "NoSuchSolver"}, work[0][2])
    srv.close()
