"""Failure paths exercised from the host, with no device fault.

* A status stored in the matrix's device error word
  (gr_matrix_inject_status) stands for a kernel whose bounded wait ran out:
  the next solve stops at its first convergence check, reports the status
  and is not converged; MPIR stops its outer loop; the word is cleared, so
  the solve after it is normal.
* A queued request of the solve server is cancelled before admission
  (gr_server_cancel): its wait reports GR_ECANCELED and the other requests
  are unaffected; a request that has already run cannot be cancelled.
"""
import numpy as np
import pytest

import graphene_b200 as gb
from graphene_b200 import _lib

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def inject(A, status):
    _lib.check(_lib.lib().gr_matrix_inject_status(A._m, status))


@pytest.fixture(scope="module")
def system():
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 16)
    A = h.copyToTile()
    b = A * A.vector(gb.randomVector(0, h.numRows).astype(np.float32))
    return h, A, b


PB = {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-7, "preconditioner": {"type": "ILU"}}


def test_injected_timeout_stops_pbicgstab(system):
    h, A, b = system
    s = gb.Solver(A, PB)
    inject(A, _lib.GR_ETIMEOUT)
    x = dev(np.zeros(h.numRows, np.float32))
    st = s.solve(x, b)
    assert st.status == _lib.GR_ETIMEOUT and not st.converged
    assert st.iterations <= 8  # stopped at the first check (one graph of 8 iterations)
    # The word was cleared: the same solver now converges normally.
    x = dev(np.zeros(h.numRows, np.float32))
    st = s.solve(x, b)
    assert st.status == 0 and st.converged and st.iterations > 8


def test_injected_timeout_stops_mpir(system):
    h, A, b = system
    cfg = {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 30,
           "extendedPrecisionType": "float64",
           "innerSolver": {"type": "PBiCGStab", "maxIterations": 300, "relResidual": 1e-4,
                           "preconditioner": {"type": "ILU"}}}
    s = gb.Solver(A, cfg)
    inject(A, _lib.GR_ETIMEOUT)
    st = s.solve(dev(np.zeros(h.numRows, np.float32)), b)
    assert st.status == _lib.GR_ETIMEOUT and not st.converged
    assert st.iterations == 1  # no outer step after the failed inner solve
    st = s.solve(dev(np.zeros(h.numRows, np.float32)), b)
    assert st.status == 0 and st.converged


def test_injected_status_on_ilu_application(system):
    h, A, b = system
    s = gb.Solver(A, {"type": "ILU"})
    inject(A, _lib.GR_ETIMEOUT)
    st = s.solve(A.createUninitializedVector(gb.FLOAT32), b)
    assert st.status == _lib.GR_ETIMEOUT
    st = s.solve(A.createUninitializedVector(gb.FLOAT32), b)
    assert st.status == 0


def test_inject_rejects_negative_status(system):
    _, A, _ = system
    with pytest.raises(gb.GrapheneError):
        inject(A, -1)


def test_server_cancel_queued_request():
    srv = gb.Server(slots=1)
    big = gb.generateMatrix(gb.GEN_VAR_POISSON, 64, 64, 64, (1.0,), 1, 64)
    small = gb.generateMatrix(gb.GEN_VAR_POISSON, 12, 12, 12, (1.0,), 2, 4)
    cfg = {"type": "PBiCGStab", "maxIterations": 1000, "relResidual": 1e-8, "preconditioner": {"type": "ILU"}}
    bb = gb.randomVector(1, big.numRows).astype(np.float32)
    bs = gb.randomVector(2, small.numRows).astype(np.float32)
    first = srv.submit(big, cfg, bb)
    queued = [srv.submit(small, cfg, bs) for _ in range(4)]
    # One slot: the big request runs, the others wait (the cancelled one
    # must still be queued when cancel is called).
    assert srv.cancel(queued[2]) is True
    with pytest.raises(gb.GrapheneError) as e:
        srv.wait(queued[2])
    assert e.value.code == _lib.GR_ECANCELED
    x0, st0, _ = srv.wait(first)
    assert st0.converged
    xs = [srv.wait(q)[0] for i, q in enumerate(queued) if i != 2]
    for x in xs[1:]:
        np.testing.assert_array_equal(x, xs[0])  # same system, same result
    # Already finished and collected: unknown id.
    with pytest.raises(gb.GrapheneError):
        srv.cancel(first)
    # Finished but not yet collected: cannot be cancelled, its result stands.
    late = srv.submit(small, cfg, bs)
    import time
    for _ in range(200):
        if srv.counters()["queued"] == 0 and srv.counters()["running"] == 0:
            break
        time.sleep(0.01)
    assert srv.cancel(late) is False
    x, st, _ = srv.wait(late)
    assert st.converged
    np.testing.assert_array_equal(x, xs[0])
    srv.close()
