"""Host pipeline parity (CPU): the product's CRS conversion, partition map,
tile layout, tile-local CRS and level sets against the oracle's restatement
of CRSHostMatrix.cpp / DistributedTileLayout.cpp. All comparisons are
bit-exact (integer and index work, coefficient values copied)."""
import numpy as np
import pytest

import graphene_b200 as gb
from tests.util import poisson_coo, random_coo


def compare_layout(h: gb.HostMatrix, om):
    assert h.numRows == om.n
    assert h.numTiles == om.P
    assert h.numOffDiag == om.m
    np.testing.assert_array_equal(h.rowToTile(), om.row_to_tile())
    np.testing.assert_array_equal(h.tileSizes(), om.tile_sizes())
    np.testing.assert_array_equal(h.localToGlobal(), om.local_to_global())
    rp, ci, od, dg = h.localCrs()
    orp, oci, ood, odg = om.local_crs()
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    np.testing.assert_array_equal(od, ood)
    np.testing.assert_array_equal(dg, odg)


@pytest.mark.parametrize("dims,tiles,part", [
    ((8, 6, 5), 1, gb.PART_AUTO),
    ((8, 6, 5), 3, gb.PART_CONTIGUOUS),
    ((8, 6, 5), 8, gb.PART_RCB),
    ((8, 6, 5), 7, gb.PART_BFS),
    ((16, 16, 16), 64, gb.PART_RCB),
    ((5, 4, 3), 60, gb.PART_RCB),   # one row per tile
])
def test_poisson_layout_matches_oracle(oracle, dims, tiles, part):
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, *dims, tiles, part)
    om = oracle.poisson(*dims, tiles, h.rowToTile())
    compare_layout(h, om)
    lo, up = h.levels()
    # Level sets equal the reference's colours on structurally symmetric tiles.
    np.testing.assert_array_equal(lo, om.colors())
    assert h.multicolorRecommended() == om.multicolor_recommended()


def test_poisson_triplets_match_reference_generator(oracle):
    """The product's generator and the oracle's restatement of Poisson.cpp
    yield identical global matrices (checked via a single-tile layout)."""
    dims = (7, 5, 4)
    h = gb.generate3DPoissonMatrix(gb.FLOAT64, *dims, 1)
    om = oracle.poisson(*dims, 1, None, value_type=1)
    compare_layout(h, om)


@pytest.mark.parametrize("seed", [0, 2])
@pytest.mark.parametrize("tiles", [2, 5, 13])
def test_random_matrix_explicit_partition(oracle, seed, tiles):
    n, rows, cols, vals = random_coo(300, 0.02, seed, symmetric=True)
    rng = np.random.default_rng(100 + seed)
    rtt = rng.integers(0, tiles, size=n).astype(np.int32)
    rtt[rtt == 1] = tiles + 2  # leaves empty tiles in [0, tiles + 3)
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, tiles + 3, rowToTile=rtt)
    om = oracle.matrix(n, rows, cols, vals, tiles + 3, rtt)
    compare_layout(h, om)
    lo, _ = h.levels()
    np.testing.assert_array_equal(lo, om.colors())


def test_unsymmetric_structure_inside_one_tile(oracle):
    """One-sided couplings are fine inside a tile (levels stay valid)."""
    n, rows, cols, vals = random_coo(120, 0.05, 1, symmetric=False)
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, 1)
    om = oracle.matrix(n, rows, cols, vals, 1, None)
    compare_layout(h, om)
    lo, up = h.levels()
    rp, ci, _, _ = h.localCrs()
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            j = ci[k]
            if j < i:
                assert lo[j] < lo[i]
            elif j > i:
                assert up[j] < up[i]


def test_unsymmetric_structure_across_tiles_rejected(oracle):
    """A coupling that only one side of a tile boundary references has no
    halo cell; the reference throws (globalToLocalRow.at), so do we."""
    n, rows, cols, vals = random_coo(120, 0.05, 1, symmetric=False)
    rtt = (np.arange(n) % 4).astype(np.int32)
    with pytest.raises(gb.GrapheneError) as e:
        gb.HostMatrix.from_coo(n, rows, cols, vals, 4, rowToTile=rtt)
    assert e.value.code == 8
    with pytest.raises(RuntimeError):
        oracle.matrix(n, rows, cols, vals, 4, rtt)


def test_empty_tiles_are_removed(oracle):
    n, rows, cols, vals = poisson_coo(4, 4, 2)
    rtt = np.where(np.arange(n) < n // 2, 5, 1).astype(np.int32)  # only tiles 1 and 5 used
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, 8, rowToTile=rtt)
    assert h.numTiles == 2
    np.testing.assert_array_equal(h.rowToTile(), np.where(rtt == 5, 1, 0))
    compare_layout(h, oracle.matrix(n, rows, cols, vals, 8, rtt))


def test_unsorted_triplets_and_missing_diagonal(oracle):
    # entries in scrambled order, row 2 without diagonal, row 5 empty
    rows = np.array([3, 0, 1, 0, 2, 4, 3, 1, 4, 6, 6, 0, 3], np.int64)
    cols = np.array([0, 1, 0, 0, 3, 4, 3, 1, 6, 6, 4, 3, 2], np.int64)
    vals = np.arange(1, 14, dtype=np.float64) * 0.5
    rtt = np.array([0, 1, 1, 0, 2, 2, 1], np.int32)
    h = gb.HostMatrix.from_coo(7, rows, cols, vals, 3, rowToTile=rtt)
    om = oracle.matrix(7, rows, cols, vals, 3, rtt)
    compare_layout(h, om)
    _, _, _, dg = h.localCrs()
    assert (dg == 0).sum() == 2  # rows 2 and 5 have no diagonal


def test_float32_rounding_of_coefficients(oracle):
    n, rows, cols, vals = random_coo(50, 0.1, 7)
    vals = vals * (1 + 1e-9)  # not representable in float32
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, 3, partitioner=gb.PART_CONTIGUOUS)
    om = oracle.matrix(n, rows, cols, vals, 3, h.rowToTile())
    compare_layout(h, om)
    _, _, od, _ = h.localCrs()
    np.testing.assert_array_equal(od, od.astype(np.float32).astype(np.float64))


def test_duplicates_rejected():
    rows = np.array([0, 0, 1], np.int64)
    cols = np.array([1, 1, 1], np.int64)
    with pytest.raises(gb.GrapheneError) as e:
        gb.HostMatrix.from_coo(2, rows, cols, np.ones(3), 1)
    assert e.value.code == 1


def test_invalid_arguments():
    with pytest.raises(gb.GrapheneError):
        gb.generate3DPoissonMatrix(gb.FLOAT32, 0, 4, 4, 2)
    with pytest.raises(gb.GrapheneError):
        gb.HostMatrix.from_coo(3, [0], [5], [1.0], 1)
    with pytest.raises(gb.GrapheneError):
        gb.HostMatrix.from_coo(3, [0], [1], [1.0], 2, rowToTile=[0, 1, 2])


def test_partitioners_cover_rows_and_balance():
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 64, gb.PART_RCB)
    assert h.numTiles == 64
    sizes = h.tileSizes()
    rows = sizes[:, 0] + sizes[:, 1]
    assert rows.sum() == 24 ** 3
    assert rows.max() <= 1.1 * rows.min()
    hb = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 64, gb.PART_BFS)
    rb = hb.tileSizes()[:, :2].sum(1)
    assert rb.sum() == 24 ** 3 and rb.max() <= 1.2 * rb.min()
    # deterministic
    h2 = gb.generate3DPoissonMatrix(gb.FLOAT32, 24, 24, 24, 64, gb.PART_BFS)
    np.testing.assert_array_equal(hb.rowToTile(), h2.rowToTile())


def test_decompose_compose_roundtrip():
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 9, 7, 5, 6)
    v = np.random.default_rng(0).standard_normal(h.numRows).astype(np.float32)
    t = h.decomposeVector(v)
    l2g = h.localToGlobal()
    # tile order = localToGlobal without halo cells
    sizes = h.tileSizes()
    own = []
    o = 0
    for ni, ns, nh in sizes:
        own.append(l2g[o:o + ni + ns])
        o += ni + ns + nh
    np.testing.assert_array_equal(t, v[np.concatenate(own)])
    np.testing.assert_array_equal(h.composeVector(t), v)


def test_matrix_market_reader(tmp_path, oracle):
    p = tmp_path / "m.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n% comment\n"
                 "4 4 6\n1 1 4.0\n2 1 -1.5\n2 2 4.0\n3 3 4.0\n4 3 -1.0\n4 4 4.0\n")
    h = gb.loadMatrixFromFile(gb.FLOAT32, str(p), 2, gb.PART_CONTIGUOUS)
    rows = [0, 1, 0, 1, 2, 3, 2, 3]
    cols = [0, 0, 1, 1, 2, 2, 3, 3]
    vals = [4.0, -1.5, -1.5, 4.0, 4.0, -1.0, -1.0, 4.0]
    om = oracle.matrix(4, rows, cols, vals, 2, h.rowToTile())
    compare_layout(h, om)
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(gb.GrapheneError):
        gb.loadMatrixFromFile(gb.FLOAT32, str(bad), 1)
    with pytest.raises(gb.GrapheneError) as e:
        gb.loadMatrixFromFile(gb.FLOAT32, str(tmp_path / "missing.mtx"), 1)
    assert e.value.code == 9
