"""The bounded mbarrier wait of the pipelined kernels (gr_selftest_wait_timeout):
a wait on a barrier that nothing arrives on gives up after about a second,
the kernel reports GR_ETIMEOUT, and the device keeps working (an SpMV right
after it is exact). No fault, trap or hang is involved."""
import ctypes as C

import numpy as np
import pytest

import graphene_b200 as gb
import graphene_b200._lib as L

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_reports_timeout():
    status, ns = C.c_int32(-1), C.c_int64(0)
    assert L.lib().gr_selftest_wait_timeout(C.byref(status), C.byref(ns)) == L.GR_OK, L.lib().gr_last_error()
    assert status.value == L.GR_ETIMEOUT
    assert 0.9e9 <= ns.value <= 10e9  # the 1 s bound, with the last sleep's slack
    # The context is still usable.
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 8, 8, 8, 4)
    A = h.copyToTile()
    x = np.ones(h.numRows, np.float32)
    y = A * A.vector(x)
    rp, col, off, dg = h.globalCrs()
    ref = dg.astype(np.float32) + np.add.reduceat(off.astype(np.float32), rp[:-1]) * (np.diff(rp) > 0)
    np.testing.assert_allclose(np.asarray(A.toNatural(y)), ref, rtol=1e-6)
