"""The library's seeded generators against an independent numpy restatement
(tests/generators_ref.py), bit for bit, for every seed the benchmark uses.

The benchmark configurations' matrices (variable-coefficient Poisson,
convection-diffusion, the LDU mesh) and right-hand sides feed both the
device path and the oracle, so a mistake in a generator would pass every
parity test; these tests pin the generators to their definitions instead.
"""
import numpy as np
import pytest

import graphene_b200 as gb
from tests import generators_ref as ref


def _split(rows, cols, vals, n):
    """Global CRS with split diagonal from sorted triplets."""
    d = rows == cols
    diag = np.zeros(n)
    diag[rows[d]] = vals[d]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows[~d] + 1, 1)
    return np.cumsum(rp), cols[~d], vals[~d], diag


def _same_crs(h, rows, cols, vals):
    rp, col, off, dg = h.globalCrs()
    erp, ecol, eoff, edg = _split(rows, cols, vals, h.numRows)
    assert np.array_equal(rp, erp)
    assert np.array_equal(col, ecol)
    assert np.array_equal(off.view(np.int64), eoff.view(np.int64)), "off-diagonal values differ"
    assert np.array_equal(dg.view(np.int64), edg.view(np.int64)), "diagonal values differ"


# (grid, sigma, seed): the 192^3 headline's seed 2 (sigma 1.5), the serving
# stream's 1000 + k and the batch's 3000 + k (sigma 1).
@pytest.mark.parametrize("dims,sigma,seed", [
    ((11, 9, 7), 1.5, 2), ((16, 16, 16), 1.5, 2), ((12, 12, 12), 1.0, 1000),
    ((17, 17, 17), 1.0, 1005), ((9, 10, 11), 1.0, 3000), ((5, 5, 5), 1.0, 3063)])
def test_var_poisson_bit_exact(dims, sigma, seed):
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (sigma,), seed, 1, valueType=gb.FLOAT64)
    _same_crs(h, *ref.var_poisson(*dims, sigma, seed))


def test_var_poisson_float32_storage_rounds_once():
    dims = (8, 7, 6)
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.5,), 2, 1, valueType=gb.FLOAT32)
    r, c, v = ref.var_poisson(*dims, 1.5, 2)
    rp, col, off, dg = h.globalCrs()
    _, _, eoff, edg = _split(r, c, v, h.numRows)
    assert np.array_equal(off, eoff.astype(np.float32).astype(np.float64))
    assert np.array_equal(dg, edg.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("dims", [(10, 9, 8), (16, 16, 16)])
def test_conv_diff_bit_exact(dims):
    h = gb.generateMatrix(gb.GEN_CONVDIFF, *dims, (0.5, 0.25, 0.125), 0, 1, valueType=gb.FLOAT64)
    r, c, v = ref.conv_diff(*dims, 0.5, 0.25, 0.125)
    _same_crs(h, r, c, v)
    # The stated stencil: W -1.5, S -1.25, B -1.125, E/N/T -1, diagonal 6.875.
    rp, col, off, dg = h.globalCrs()
    assert set(np.unique(off)) == {-1.5, -1.25, -1.125, -1.0}
    assert np.all(dg == 6.875)


@pytest.mark.parametrize("dims,seeds", [((7, 6, 5), (4, 5, 6)), ((9, 8, 10), (4, 5, 6)),
                                        ((6, 6, 6), (14, 15, 16))])
def test_ldu_mesh_bit_exact(dims, seeds):
    h = gb.generateLduMesh(*dims, *seeds, numTiles=1, valueType=gb.FLOAT64)
    o, nb, lo, up, dg = h.ldu()
    eo, enb, elo, edg, _ = ref.ldu_mesh(*dims, *seeds)
    assert np.array_equal(o, eo) and np.array_equal(nb, enb)
    assert np.array_equal(lo.view(np.int64), elo.view(np.int64))
    assert np.array_equal(up, lo)  # symmetric
    assert np.array_equal(dg.view(np.int64), edg.view(np.int64))
    # Faces sorted by (owner, neighbour), owner < neighbour.
    assert np.all(o < nb)
    key = o * (o.max() + nb.max() + 2) + nb
    assert np.all(np.diff(key) > 0)


@pytest.mark.parametrize("seed,dist", [(0, "uniform"), (3, "uniform"), (1, "normal"), (2000, "uniform"),
                                       (4005, "uniform")])
def test_random_vectors_bit_exact(seed, dist):
    n = 3001
    got = gb.randomVector(seed, n, dist)
    want = ref.uniform(seed, n) if dist == "uniform" else ref.normal(seed, n)
    assert np.array_equal(got.view(np.int64), want.view(np.int64))


def test_stream_statistics():
    """The stream itself: uniform mean / variance and normal moments at the
    sizes the benchmark draws (a gross error in the finaliser would show)."""
    u = ref.uniform01(7, np.arange(200000, dtype=np.uint64))
    assert abs(u.mean() - 0.5) < 5e-3 and abs(u.var() - 1 / 12) < 5e-3
    assert u.min() >= 0.0 and u.max() < 1.0
    g = ref.normal(9, 50000)
    assert abs(g.mean()) < 2e-2 and abs(g.std() - 1) < 2e-2


# ---- the oracle's own copy (the reference arm of the benchmark uses it) ----
@pytest.fixture(scope="module")
def oracle():
    from tests.oracle_py import Oracle
    return Oracle()


@pytest.mark.parametrize("kind,params,seed,dims", [
    (1, (1.5,), 2, (11, 9, 7)), (1, (1.0,), 1003, (12, 13, 14)), (2, (0.5, 0.25, 0.125), 0, (10, 9, 8)),
    (0, (), 0, (6, 7, 8))])
def test_oracle_generators_bit_exact(oracle, kind, params, seed, dims):
    r, c, v, xyz = oracle.generate(kind, *dims, params, seed)
    if kind == 1:
        er, ec, ev = ref.var_poisson(*dims, params[0], seed)
    elif kind == 2:
        er, ec, ev = ref.conv_diff(*dims, *params)
    else:
        h = gb.generate3DPoissonMatrix(gb.FLOAT64, *dims, 1)
        er, ec, ev = (np.asarray(a) for a in h.coo())
        o = np.lexsort((ec, er))
        er, ec, ev = er[o], ec[o], ev[o]
    assert np.array_equal(r, er) and np.array_equal(c, ec)
    assert np.array_equal(v.view(np.int64), ev.view(np.int64))
    n = int(np.prod(dims))
    i = np.arange(n)
    assert np.array_equal(xyz, np.stack([i % dims[0], (i // dims[0]) % dims[1], i // (dims[0] * dims[1])], 1))


@pytest.mark.parametrize("seed,dist", [(0, "uniform"), (3, "uniform"), (1, "normal")])
def test_oracle_random_vectors_bit_exact(oracle, seed, dist):
    got = oracle.random_vector(seed, 2049, dist)
    want = ref.uniform(seed, 2049) if dist == "uniform" else ref.normal(seed, 2049)
    assert np.array_equal(got.view(np.int64), want.view(np.int64))


@pytest.mark.parametrize("dims,tiles", [((32, 32, 32), 64), ((24, 20, 18), 37), ((40, 40, 40), 512),
                                        ((7, 5, 3), 4)])
def test_oracle_bisection_matches_library(oracle, dims, tiles):
    """The oracle's coordinate bisection gives the library's RCB tile map,
    and the oracle matrix built on it has the library's tile order."""
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.5,), 2, tiles, gb.PART_RCB)
    om = oracle.grid_system(1, *dims, (1.5,), 2, tiles)
    assert np.array_equal(om.row_to_tile(), h.rowToTile())
    x = np.arange(h.numRows, dtype=np.float64)
    assert np.array_equal(om.decompose(x), h.decomposeVector(x, gb.FLOAT64))
