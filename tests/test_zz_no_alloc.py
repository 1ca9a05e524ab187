"""gr_vector_norms_noalloc: norms through a static device scratch, no
device allocation. Compared with the matrix-bound gr_vector_norm on two
consecutive calls, which also shows that the scratch's arrival counters are
back at zero after a call: identical values while both use the same block
count (8 per SM up to the scratch's 148 x 8 partials, i.e. up to 148 SMs),
within 1e-13 relative beyond that. Collected last so that it also runs
after every other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

import graphene_b200 as gb
import graphene_b200._lib as L

pytestmark = pytest.mark.gpu


def noalloc(x, n, count, ld, t, norm, out):
    return L.lib().gr_vector_norms_noalloc(C.c_void_p(x.data_ptr()), n, count, ld, t, norm,
                                           C.c_void_p(out.data_ptr()), None)


@pytest.mark.parametrize("t", [gb.FLOAT32, gb.FLOAT64])
def test_noalloc_norms_equal_matrix_norms_twice(t):
    import torch
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 40, 40, 40, (1.0,), 2, 64)
    A = h.copyToTile()
    n = h.numRows
    dt = torch.float32 if t == gb.FLOAT32 else torch.float64
    g = torch.Generator(device="cuda").manual_seed(5)
    ld = n + 7
    xs = torch.randn(3, ld, generator=g, device="cuda", dtype=torch.float64).to(dt)
    same_blocks = torch.cuda.get_device_properties(0).multi_processor_count <= 148
    for norm in (gb.NORM_L1, gb.NORM_L2, gb.NORM_LINF):
        ref = [A.vectorNorm(norm, xs[j, :n]) for j in range(3)]
        for _ in range(2):
            out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
            assert noalloc(xs, n, 3, ld, t, norm, out) == L.GR_OK, L.lib().gr_last_error()
            torch.cuda.synchronize()
            if same_blocks:
                assert out.tolist() == ref
            else:
                np.testing.assert_allclose(out.tolist(), ref, rtol=1e-13)
        host = xs[:, :n].double().cpu().numpy()
        exp = {gb.NORM_L1: host.sum(1), gb.NORM_L2: np.linalg.norm(host, axis=1),
               gb.NORM_LINF: host.max(1)}[norm]
        np.testing.assert_allclose(ref, exp, rtol=1e-11)


def test_noalloc_norms_leave_free_memory_unchanged():
    import torch
    n = 1 << 20
    x = torch.randn(2, n, device="cuda")
    out = torch.empty(2, dtype=torch.float64, device="cuda")
    assert noalloc(x, n, 2, n, gb.FLOAT32, gb.NORM_L2, out) == L.GR_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert noalloc(x, n, 2, n, gb.FLOAT32, gb.NORM_L2, out) == L.GR_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    np.testing.assert_allclose(out.cpu().numpy(), np.linalg.norm(x.double().cpu().numpy(), axis=1),
                               rtol=1e-12)


def test_noalloc_norms_reject_oversize_and_host_pointers():
    import torch
    x = torch.zeros(16, device="cuda")
    out = torch.zeros(9, dtype=torch.float64, device="cuda")
    assert noalloc(x, 1, 9, 1, gb.FLOAT32, gb.NORM_L2, out) == L.GR_EINVAL
    assert b"count must be 1..8" in L.lib().gr_last_error()
    assert noalloc(x, 1 << 31, 1, 1 << 31, gb.FLOAT32, gb.NORM_L2, out) == L.GR_EINVAL
    assert noalloc(x, 8, 2, 4, gb.FLOAT32, gb.NORM_L2, out) == L.GR_EINVAL  # ld < n
    host = torch.zeros(16)
    assert noalloc(host, 16, 1, 16, gb.FLOAT32, gb.NORM_L2, out) == L.GR_EINVAL
    assert b"device-accessible" in L.lib().gr_last_error()


def test_noalloc_norms_reject_ranges_past_the_allocation():
    """A read range that leaves its allocation is refused before anything
    runs (nothing is launched, nothing faults); the same shape inside the
    allocation works. The allocation is a cudaMalloc of its own, and its
    extent is the driver's own answer."""
    import torch
    from cuda.bindings import driver, runtime
    torch.cuda.init()
    err, ptr = runtime.cudaMalloc(1 << 16)
    assert err == runtime.cudaError_t.cudaSuccess
    try:
        err, base, size = driver.cuMemGetAddressRange(ptr)
        assert err == driver.CUresult.CUDA_SUCCESS
        elems = int(size) // 4 - (int(ptr) - int(base)) // 4   # floats from ptr to the end
        runtime.cudaMemset(ptr, 0, 4 * elems)
        out = torch.zeros(2, dtype=torch.float64, device="cuda")
        f = L.lib().gr_vector_norms_noalloc
        o = C.c_void_p(out.data_ptr())
        half = elems // 2
        # Two vectors of half + 1 at stride half + 1 overrun by 2 elements or more.
        assert f(C.c_void_p(int(ptr)), half + 1, 2, half + 1, gb.FLOAT32, gb.NORM_L2, o, None) == L.GR_EINVAL
        assert b"past the end" in L.lib().gr_last_error()
        # One vector of exactly the allocation is fine.
        assert f(C.c_void_p(int(ptr)), elems, 1, elems, gb.FLOAT32, gb.NORM_L2, o, None) == L.GR_OK
        torch.cuda.synchronize()
        assert out[0].item() == 0.0
    finally:
        runtime.cudaFree(ptr)
