"""The streamed ILU substitution's byte stream, replayed on the host (CPU):
every row / column index in range, entries only reference rows computed in
earlier levels of the same sweep, and the shared-memory ring always holds the
chunks a level needs under the kernel's refill rule."""
import ctypes as C

import pytest

import graphene_b200 as gb
from tests.util import random_coo


def check(h, dilu, vt=gb.FLOAT32):
    lg = C.c_int32()
    nbytes = C.c_int64()
    gb._lib.check(gb._lib.lib().gr_host_matrix_check_ilu_stream(h._h, int(dilu), vt, C.byref(lg),
                                                                 C.byref(nbytes)))
    return lg.value, nbytes.value


@pytest.mark.parametrize("dims,tiles,part", [
    ((16, 16, 16), 8, gb.PART_RCB),
    ((13, 11, 7), 6, gb.PART_BFS),
    ((12, 10, 8), 1, gb.PART_AUTO),
    ((20, 20, 20), 200, gb.PART_RCB),
    ((5, 4, 3), 60, gb.PART_RCB),
    ((33, 17, 9), 5, gb.PART_CONTIGUOUS),
])
@pytest.mark.parametrize("dilu", [False, True])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
def test_stream_replay(dims, tiles, part, dilu, vt):
    h = gb.generate3DPoissonMatrix(vt, *dims, tiles, part)
    lg, nbytes = check(h, dilu, vt)
    assert 13 <= lg <= 20 and nbytes % 16 == 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_stream_replay_random(seed):
    n, r, c, v = random_coo(400, 0.03, seed)
    h = gb.HostMatrix.from_coo(n, r, c, v, 7, partitioner=gb.PART_BFS)
    check(h, False)
    check(h, True)
    h1 = gb.HostMatrix.from_coo(*random_coo(200, 0.05, seed, symmetric=False), 1)
    check(h1, False)


def test_stream_replay_bench_problem():
    """The 192^3 variable-coefficient system at the bench's 1024 tiles."""
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 192, 192, 192, (1.5,), 2, 1024)
    lg, nbytes = check(h, False)
    assert lg <= 16


# ---- host-scheduled level ring (kernels_ring.cu) ----------------------------------------

def check_ring(h, dilu, vt=gb.FLOAT32, ring_bytes=0, group=1, compact=True):
    used, nbytes, lv = C.c_int64(), C.c_int64(), C.c_int32()
    gb._lib.check(gb._lib.lib().gr_host_matrix_check_ilu_ring(h._h, int(dilu), vt, ring_bytes, group, int(compact),
                                                               C.byref(used), C.byref(nbytes), C.byref(lv)))
    return used.value, nbytes.value, lv.value


@pytest.mark.parametrize("dims,tiles,part", [
    ((16, 16, 16), 8, gb.PART_RCB),
    ((13, 11, 7), 6, gb.PART_BFS),
    ((12, 10, 8), 1, gb.PART_AUTO),
    ((20, 20, 20), 200, gb.PART_RCB),
    ((5, 4, 3), 60, gb.PART_RCB),
    ((33, 17, 9), 5, gb.PART_CONTIGUOUS),
])
@pytest.mark.parametrize("dilu", [False, True])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
@pytest.mark.parametrize("group", [1, 3])
@pytest.mark.parametrize("compact", [True, False, 2])
def test_ring_replay(dims, tiles, part, dilu, vt, group, compact):
    h = gb.generate3DPoissonMatrix(vt, *dims, tiles, part)
    used, nbytes, lv = check_ring(h, dilu, vt, 0, group, compact)
    assert used > 0 and used % 16 == 0 and nbytes % 16 == 0 and lv >= 2


def test_ring_compact_layout_is_smaller():
    """16-bit row and column ids: a 7-point lower-sweep row takes 2 + 3 x 6
    bytes instead of 4 + 3 x 8."""
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 8, gb.PART_RCB)
    _, wide, _ = check_ring(h, False, gb.FLOAT32, 0, 1, False)
    _, compact, _ = check_ring(h, False, gb.FLOAT32, 0, 1, True)
    assert compact < 0.8 * wide


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_ring_replay_random_and_ldu(seed):
    n, r, c, v = random_coo(400, 0.03, seed)
    check_ring(gb.HostMatrix.from_coo(n, r, c, v, 7, partitioner=gb.PART_BFS), seed == 1, group=seed + 1)
    check_ring(gb.generateLduMesh(9, 8, 7, numTiles=5, partitioner=gb.PART_RCB), seed == 2)


def test_ring_small_rings_wrap_and_reuse_barriers():
    """Rings of a few level blocks force wrap-around placement and more than
    16 levels in flight per barrier cycle; the replay must still pass, and a
    ring smaller than two consecutive levels must be rejected."""
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 4, gb.PART_RCB)
    used, _, lv = check_ring(h, False)
    assert lv > 2 * 16
    passed = 0
    for rb in range(used // 4, 2 * used + 1, 1024):
        try:
            check_ring(h, False, gb.FLOAT32, rb)
            passed += 1
        except gb.GrapheneError as e:
            assert "too small" in str(e) and rb < used
    assert passed > (2 * used - used) // 1024
    with pytest.raises(gb.GrapheneError):
        check_ring(h, False, gb.FLOAT32, 256)


@pytest.mark.parametrize("tiles", [2048, 2368])
def test_ring_replay_192_workload(tiles):
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, 192, 192, 192, (1.5,), 2, tiles)
    for group in (1, 2, 4):
        used, nbytes, lv = check_ring(h, False, gb.FLOAT32, 0, group)
        assert used >= 8192 and lv < 128


# ---- Gauss-Seidel level ring -------------------------------------------------------------

def check_gs_ring(h, lower_only, vt=gb.FLOAT32, ring_bytes=0, compact=True, want_in_place=False):
    used, nbytes, lv, ip = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
    gb._lib.check(gb._lib.lib().gr_host_matrix_check_gs_ring(h._h, int(lower_only), vt, ring_bytes, int(compact),
                                                              C.byref(used), C.byref(nbytes), C.byref(lv),
                                                              C.byref(ip)))
    if want_in_place:
        return used.value, nbytes.value, lv.value, bool(ip.value)
    return used.value, nbytes.value, lv.value


@pytest.mark.parametrize("dims,tiles,part", [
    ((16, 16, 16), 8, gb.PART_RCB),
    ((13, 11, 7), 6, gb.PART_BFS),
    ((12, 10, 8), 1, gb.PART_AUTO),
    ((20, 20, 20), 200, gb.PART_RCB),
    ((5, 4, 3), 60, gb.PART_RCB),
    ((33, 17, 9), 5, gb.PART_CONTIGUOUS),
])
@pytest.mark.parametrize("lower_only", [False, True])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
@pytest.mark.parametrize("compact", [True, False, 2])
def test_gs_ring_replay(dims, tiles, part, lower_only, vt, compact):
    h = gb.generate3DPoissonMatrix(vt, *dims, tiles, part)
    used, nbytes, lv = check_gs_ring(h, lower_only, vt, 0, compact)
    assert used > 0 and used % 16 == 0 and nbytes % 16 == 0 and lv >= 1
    # One sweep: the tile's lower levels only.
    _, _, lv_ilu = check_ring(h, False, vt)
    assert lv <= lv_ilu


def test_gs_ring_lower_only_is_smaller():
    """A sweep from x = 0 reads only the entries of earlier rows: about half
    the level bytes of a full sweep on a 7-point matrix."""
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 8, gb.PART_RCB)
    _, full, _ = check_gs_ring(h, False)
    _, lower, _ = check_gs_ring(h, True)
    assert lower < 0.7 * full


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_gs_ring_replay_random_and_ldu(seed):
    n, r, c, v = random_coo(400, 0.03, seed)
    h = gb.HostMatrix.from_coo(n, r, c, v, 7, partitioner=gb.PART_BFS)
    check_gs_ring(h, False)
    check_gs_ring(h, True)
    h1 = gb.HostMatrix.from_coo(*random_coo(300, 0.04, seed, symmetric=False), 1)
    check_gs_ring(h1, False)
    check_gs_ring(gb.generateLduMesh(9, 8, 7, numTiles=5, partitioner=gb.PART_RCB), seed == 2)


def test_gs_ring_replay_convdiff_workload():
    """The 128^3 convection-diffusion system at its 1024 tiles: boxes of a
    7-point grid, so the sweep runs in place (no sweep-start copy)."""
    h = gb.generateMatrix(gb.GEN_CONVDIFF, 128, 128, 128, (0.5, 0.25, 0.125), 0, 1024)
    for lower_only in (False, True):
        used, nbytes, lv, ip = check_gs_ring(h, lower_only, want_in_place=True)
        assert used >= 4096 and lv < 64 and ip


def test_gs_ring_in_place_only_when_safe():
    """In place needs every in-tile upper entry in a later level than its
    row: true whenever the pattern is structurally symmetric (entry (r, c)
    above the diagonal has (c, r) below it, so c's level exceeds r's), false
    for a nonsymmetric random pattern whose upper neighbours can sit in
    earlier levels; the replay checks both."""
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 16, 16, 16, 8, gb.PART_RCB)
    assert check_gs_ring(h, False, want_in_place=True)[3]
    n, r, c, v = random_coo(400, 0.03, 1)
    assert check_gs_ring(gb.HostMatrix.from_coo(n, r, c, v, 3, partitioner=gb.PART_BFS), False,
                         want_in_place=True)[3]
    n, r, c, v = random_coo(300, 0.04, 1, symmetric=False)
    hr = gb.HostMatrix.from_coo(n, r, c, v, 1)
    assert not check_gs_ring(hr, False, want_in_place=True)[3]
    assert check_gs_ring(hr, True, want_in_place=True)[3]  # lower-only rings have no upper entries


def test_ring_record_levels_same_bytes():
    """Row records (levels of 3 entries a row): 16 + 4 bytes a row without an
    inverse diagonal, 16 + 8 with one - the column-major compact layout's
    bytes (2 + 3 x 2 + 3 x 4, plus 4), up to 16-byte padding."""
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 8, gb.PART_RCB)
    _, compact, _ = check_ring(h, False, gb.FLOAT32, 0, 1, True)
    _, record, _ = check_ring(h, False, gb.FLOAT32, 0, 1, 2)
    assert abs(record - compact) <= 0.02 * compact
