"""The SpMV layout's 16-bit column encoding, decoded on the host.

Every slot of the 16-bit layout (column - row, or a far column taken from
the chunk's side list in the order the device's warp votes hand them out)
must decode to the 32-bit layout's column; the far counts and the 64-column
limit per chunk follow the stated rule, and the automatic layout is the
32-bit one.
"""
import numpy as np
import pytest

import graphene_b200 as gb


def far_fraction(info):
    return info["far"] / max(1, info["slots"])


@pytest.mark.parametrize("make", [
    lambda: gb.generate3DPoissonMatrix(gb.FLOAT32, 40, 40, 40, 32),
    lambda: gb.generateMatrix(gb.GEN_VAR_POISSON, 33, 29, 31, (1.5,), 2, 48, gb.PART_RCB),
    lambda: gb.generateMatrix(gb.GEN_CONVDIFF, 24, 24, 24, (0.5, 0.25, 0.125), 0, 16),
    lambda: gb.generate3DPoissonMatrix(gb.FLOAT64, 7, 5, 3, 1),
])
def test_grid_matrices_decode(make):
    h = make()
    auto = h.checkSpmvLayout(-1)
    forced = h.checkSpmvLayout(1)
    plain = h.checkSpmvLayout(0)
    assert forced["compact"] and not plain["compact"] and not auto["compact"]  # automatic: 32-bit
    assert auto["slots"] == plain["slots"] == forced["slots"]
    assert far_fraction(forced) <= 0.125 and forced["max_chunk_far"] <= 64
    assert plain["far"] == 0


def test_permuted_mesh_keeps_32_bit_automatically():
    # Cells in a random order: most couplings are far from their row.
    h = gb.generateLduMesh(48, 48, 48, 4, 5, 6, numTiles=1)
    assert not h.checkSpmvLayout(-1)["compact"]
    with pytest.raises(gb.GrapheneError):  # more than 64 far columns in a chunk
        h.checkSpmvLayout(1)


def test_far_entries_per_chunk_limit():
    """Two far columns a row give chunks of exactly 64 far columns, the most
    the device hands out of the warp's lanes (two registers each); more are
    refused for the 16-bit layout and make the automatic choice keep 32-bit
    columns."""
    n = 150000
    r = np.arange(n)
    rows = np.concatenate([r, r, r, r[:-1]])
    cols = np.concatenate([r, (r + 40000) % n, (r + 90000) % n, r[:-1] + 1])
    vals = np.concatenate([np.full(n, 8.0), np.full(3 * n - 1, -1.0)])
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, 1)
    info = h.checkSpmvLayout(1)
    assert info["compact"] and info["max_chunk_far"] == 64 and info["far"] == 2 * n
    assert h.checkSpmvLayout(-1)["compact"] is False
    rows = np.concatenate([rows, r])
    cols = np.concatenate([cols, (r + 120000) % n])
    vals = np.concatenate([vals, np.full(n, -1.0)])
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, 1)
    with pytest.raises(gb.GrapheneError):
        h.checkSpmvLayout(1)
    assert not h.checkSpmvLayout(-1)["compact"]
    h.setSpmvLayout(1)  # accepted here; the device copy refuses it


def test_ragged_rows_and_empty_rows():
    rng = np.random.default_rng(3)
    n = 5003  # not a multiple of 32
    deg = rng.integers(0, 12, n)
    deg[::97] = 0
    rows = np.repeat(np.arange(n), deg)
    off = rng.integers(1, 40000, rows.size) * rng.choice([-1, 1], rows.size)
    cols = np.clip(rows + off, 0, n - 1)
    keep = cols != rows
    rows, cols = rows[keep], cols[keep]
    _, first = np.unique(rows * n + cols, return_index=True)
    rows, cols = rows[first], cols[first]
    rows = np.concatenate([rows, np.arange(n)])
    cols = np.concatenate([cols, np.arange(n)])
    vals = rng.uniform(-1, 1, rows.size)
    h = gb.HostMatrix.from_coo(n, rows, cols, vals, 1)  # nonsymmetric: one tile
    for layout in (-1, 0, 1):
        h.checkSpmvLayout(layout)


def test_layout_argument_checked():
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 4, 4, 4, 1)
    with pytest.raises(gb.GrapheneError):
        h.setSpmvLayout(2)
    with pytest.raises(gb.GrapheneError):
        h.checkSpmvLayout(-2)
    h.setSpmvLayout(0)
    h.setSpmvLayout(-1)
