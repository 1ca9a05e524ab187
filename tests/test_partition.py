"""The multilevel partitioner (GR_PART_MULTILEVEL, the default for matrices
without row coordinates), in the role METIS_PartGraphRecursive plays in the
reference (CRSHostMatrix.cpp:139-271): balance of the row weights (row
entries + 1), edge cut against the other coordinate-free partitioners,
determinism, degenerate graphs, and the block-ILU(0) iteration counts the
partitions give (oracle PBiCGStab on the CPU)."""
import json

import numpy as np
import pytest

import graphene_b200 as gb
from tests.oracle_py import Oracle


def poisson_coo(L):
    h = gb.generate3DPoissonMatrix(gb.FLOAT64, L, L, L, 1)
    return h.numRows, *(np.asarray(a) for a in h.coo())


def part_weights(h):
    rp, col, off, dg = h.globalCrs()
    w = np.diff(rp) + 1
    return np.bincount(h.rowToTile(), weights=w, minlength=h.numTiles)


@pytest.mark.parametrize("L,P", [(20, 2), (24, 16), (32, 64), (30, 37)])
def test_balance_and_cut(L, P):
    n, r, c, v = poisson_coo(L)
    ml = gb.HostMatrix.from_coo(n, r, c, v, P, gb.PART_MULTILEVEL)
    bfs = gb.HostMatrix.from_coo(n, r, c, v, P, gb.PART_BFS)
    contig = gb.HostMatrix.from_coo(n, r, c, v, P, gb.PART_CONTIGUOUS)
    assert ml.numTiles == P
    w = part_weights(ml)
    # 0.2 % per bisection plus one vertex, over ceil(log2 P) levels.
    levels = int(np.ceil(np.log2(P)))
    assert w.max() <= w.mean() * (1.002 + 8 / w.mean()) ** levels * 1.0001
    assert ml.edgeCut() < 0.8 * bfs.edgeCut()
    if P >= 16:  # natural-order slabs are planar cuts only for few parts
        assert ml.edgeCut() < 0.6 * contig.edgeCut()


def test_near_plane_cut_for_two_parts():
    n, r, c, v = poisson_coo(32)
    ml = gb.HostMatrix.from_coo(n, r, c, v, 2, gb.PART_MULTILEVEL)
    assert ml.edgeCut() <= 1.1 * 2 * 32 * 32  # a plane cuts 32^2 edges, counted both ways


def test_deterministic_and_default_without_coordinates():
    n, r, c, v = poisson_coo(16)
    a = gb.HostMatrix.from_coo(n, r, c, v, 8, gb.PART_MULTILEVEL).rowToTile()
    b = gb.HostMatrix.from_coo(n, r, c, v, 8, gb.PART_MULTILEVEL).rowToTile()
    auto = gb.HostMatrix.from_coo(n, r, c, v, 8).rowToTile()
    assert np.array_equal(a, b) and np.array_equal(a, auto)


def test_disconnected_and_isolated_rows():
    # Two Poisson blocks side by side plus rows with no off-diagonals.
    n1, r1, c1, v1 = poisson_coo(10)
    iso = 77
    n = 2 * n1 + iso
    r = np.concatenate([r1, r1 + n1, np.arange(2 * n1, n)])
    c = np.concatenate([c1, c1 + n1, np.arange(2 * n1, n)])
    v = np.concatenate([v1, v1, np.ones(iso)])
    h = gb.HostMatrix.from_coo(n, r, c, v, 6, gb.PART_MULTILEVEL)
    assert h.numTiles == 6
    w = part_weights(h)
    assert w.max() <= 1.05 * w.mean()


def test_more_parts_than_rows():
    n, r, c, v = poisson_coo(2)  # 8 rows
    h = gb.HostMatrix.from_coo(n, r, c, v, 20, gb.PART_MULTILEVEL)
    assert 1 <= h.numTiles <= 8
    assert np.array_equal(np.unique(h.rowToTile()), np.arange(h.numTiles))


def test_block_ilu_iterations_follow_the_cut():
    """PBiCGStab-ILU(0) iterations (oracle, FP64) on the variable-coefficient
    Poisson system: the multilevel partition needs fewer than the BFS and
    contiguous ones, within a few of coordinate bisection's boxes."""
    o = Oracle()
    L, P = 24, 16
    r, c, v, xyz = o.generate(1, L, L, L, (1.5,), 2)
    n = L ** 3
    b = o.random_vector(5, n)
    cfg = json.dumps({"type": "PBiCGStab", "maxIterations": 2000, "relResidual": 1e-8,
                      "preconditioner": {"type": "ILU"}})
    its = {}
    for name, part, coords in (("contiguous", gb.PART_CONTIGUOUS, None), ("bfs", gb.PART_BFS, None),
                               ("multilevel", gb.PART_MULTILEVEL, None), ("rcb", gb.PART_RCB, xyz)):
        h = gb.HostMatrix.from_coo(n, r, c, v, P, part, coords=coords, valueType=gb.FLOAT64)
        om = o.matrix(n, r, c, v, h.numTiles, h.rowToTile(), 1)
        _, st, _, _ = om.solve(cfg, np.zeros(n), om.decompose(b))
        its[name] = st.iterations
    assert its["multilevel"] < its["bfs"] and its["multilevel"] < its["contiguous"]
    assert its["multilevel"] <= its["rcb"] + 5
