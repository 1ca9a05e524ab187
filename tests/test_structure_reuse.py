"""Matrices that share a sparsity pattern (CPU only): generateMatrixLike
copies a template's partition, tile layout and level sets and takes fresh
values, and must equal a matrix generated from scratch with the same seed
in every layout array and value; the structure key identifies the pattern."""
import numpy as np
import pytest

import graphene_b200 as gb


def layout(h):
    return [h.rowToTile(), h.tileSizes(), h.localToGlobal(), *h.localCrs(), *h.levels(), *h.globalCrs()]


@pytest.mark.parametrize("dims,tiles", [((12, 11, 10), 8), ((20, 20, 20), 64), ((7, 9, 5), 1)])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
def test_generate_like_equals_fresh(dims, tiles, vt):
    tmpl = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 100, tiles, valueType=vt)
    like = gb.generateMatrixLike(tmpl, gb.GEN_VAR_POISSON, *dims, (1.0,), 101)
    fresh = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 101, tiles, valueType=vt)
    for a, b in zip(layout(like), layout(fresh)):
        np.testing.assert_array_equal(a, b)
    assert like.structureKey == fresh.structureKey == tmpl.structureKey
    # New values: the template's differ.
    assert not np.array_equal(tmpl.globalCrs()[2], like.globalCrs()[2])


def test_structure_key_distinguishes_patterns():
    a = gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 1, 8)
    keys = {a.structureKey,
            gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 11, (1.0,), 1, 8).structureKey,
            gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 1, 9).structureKey,
            gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 1, 8, valueType=gb.FLOAT64).structureKey}
    assert len(keys) == 4
    assert gb.generateMatrix(gb.GEN_CONVDIFF, 10, 10, 10, (0.5, 0.25, 0.1), 0, 8).structureKey == a.structureKey


def test_generate_like_rejects_other_grids():
    tmpl = gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 1, 8)
    with pytest.raises(gb.GrapheneError):
        gb.generateMatrixLike(tmpl, gb.GEN_VAR_POISSON, 10, 10, 11, (1.0,), 2)
    with pytest.raises(gb.GrapheneError):
        gb.generateMatrixLike(tmpl, gb.GEN_VAR_POISSON, 20, 10, 5, (1.0,), 2)  # same n, other pattern
    ldu = gb.generateLduMesh(5, 5, 5, numTiles=2)
    with pytest.raises(gb.GrapheneError):
        gb.generateMatrixLike(ldu, gb.GEN_VAR_POISSON, 5, 5, 5, (1.0,), 2)


@pytest.mark.parametrize("kind,params", [(gb.GEN_VAR_POISSON, (1.3,)), (gb.GEN_CONVDIFF, (0.5, 0.25, 0.125)),
                                         (gb.GEN_POISSON, ())])
def test_generate_values_equals_generator(kind, params):
    """The values alone, in the template's global CRS order, are the full
    generator's values bit for bit (FP64 template: no rounding)."""
    dims, tiles = (13, 12, 11), 9
    tmpl = gb.generateMatrix(gb.GEN_VAR_POISSON, *dims, (1.0,), 3, tiles, valueType=gb.FLOAT64)
    gv, gd = gb.generateValues(tmpl, kind, *dims, params, 42)
    full = gb.generateMatrix(kind, *dims, params, 42, tiles, valueType=gb.FLOAT64)
    rp, col, off, dg = full.globalCrs()
    assert np.array_equal(gv.view(np.int64), off.view(np.int64))
    assert np.array_equal(gd.view(np.int64), dg.view(np.int64))


def test_generate_values_checks_the_grid():
    tmpl = gb.generateMatrix(gb.GEN_VAR_POISSON, 10, 10, 10, (1.0,), 3, 4)
    with pytest.raises(gb.GrapheneError):
        gb.generateValues(tmpl, gb.GEN_VAR_POISSON, 10, 10, 11, (1.0,), 1)
    with pytest.raises(gb.GrapheneError):
        gb.generateValues(tmpl, gb.GEN_VAR_POISSON, 20, 10, 5, (1.0,), 1)
