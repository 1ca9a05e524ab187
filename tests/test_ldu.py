"""LDU (owner / neighbour face) matrices.

CPU: the mesh generator's structure, the host layout against the oracle, the
input checks, and the oracle's LDU row loops (LDUMatrix.cpp:42-168) against
an independent Python restatement and scipy.
GPU: SpMV and residual through the C ABI bit-exact against the oracle for
every partitioning, and Gauss-Seidel-preconditioned PBiCGStab on an LDU
matrix against the oracle.
"""
import json

import numpy as np
import pytest

import graphene_b200 as gb
from tests.test_layout import compare_layout

F32 = np.float32


def random_ldu(n, faces_per_cell, seed, symmetric=False):
    """Random LDU matrix: faces owner < neighbour, sorted by owner only (the
    neighbours of one owner in random order), diagonally dominant."""
    rng = np.random.default_rng(seed)
    pairs = set()
    while len(pairs) < faces_per_cell * n:
        a, b = rng.integers(0, n, 2)
        if a != b:
            pairs.add((min(a, b), max(a, b)))
    pairs = list(pairs)
    rng.shuffle(pairs)
    pairs.sort(key=lambda p: p[0])  # stable: neighbours of an owner stay shuffled
    owner = np.array([p[0] for p in pairs], np.int64)
    nb = np.array([p[1] for p in pairs], np.int64)
    lower = -rng.uniform(0.1, 1.0, len(pairs))
    upper = lower.copy() if symmetric else -rng.uniform(0.1, 1.0, len(pairs))
    diag = np.full(n, 1.0)
    np.add.at(diag, owner, np.abs(upper))
    np.add.at(diag, nb, np.abs(lower))
    return owner, nb, diag, lower, upper


def py_ldu_spmv_f32(n, owner, nb, lower, upper, diag, x):
    """LDUMatrix::spmv (LDUMatrix.cpp:64-86) in float32, natural order:
    diag * x, owned faces in face order, then losort order (faces sorted by
    neighbour, ties by face index)."""
    own = [[] for _ in range(n)]
    nbr = [[] for _ in range(n)]
    for f in range(len(owner)):
        own[owner[f]].append(f)
    for f in sorted(range(len(owner)), key=lambda f: (nb[f], f)):
        nbr[nb[f]].append(f)
    y = np.empty(n, F32)
    for c in range(n):
        acc = F32(diag[c]) * x[c]
        for f in own[c]:
            acc = F32(acc + F32(upper[f]) * x[nb[f]])
        for f in nbr[c]:
            acc = F32(acc + F32(lower[f]) * x[owner[f]])
        y[c] = acc
    return y


def scipy_ldu(n, owner, nb, diag, lower, upper):
    import scipy.sparse as sp
    r = np.concatenate([np.arange(n), owner, nb])
    c = np.concatenate([np.arange(n), nb, owner])
    v = np.concatenate([diag, upper, lower])
    return sp.csr_matrix((v, (r, c)), shape=(n, n))


# ---- CPU ------------------------------------------------------------------------------

def test_mesh_generator_structure():
    nx, ny, nz = 7, 6, 5
    h = gb.generateLduMesh(nx, ny, nz, numTiles=1)
    n = nx * ny * nz
    o, nb, lo, up, dg = h.ldu()
    assert h.isLdu and h.numRows == n
    assert len(o) == 3 * n - (ny * nz + nx * nz + nx * ny)
    assert np.all(o < nb) and np.all(np.diff(o) >= 0)
    keys = o * n + nb
    assert np.all(np.diff(keys) > 0)  # sorted by (owner, neighbour), no duplicates
    np.testing.assert_array_equal(lo, up)
    c = -lo
    assert c.min() >= 1e-2 * (1 - 1e-6) and c.max() <= 1e2 * (1 + 1e-6)
    s = np.full(n, 1e-3)
    np.add.at(s, o, c)
    np.add.at(s, nb, c)
    np.testing.assert_allclose(dg, s, rtol=1e-6)
    # Cell ids are permuted: neighbours in the mesh are not id +- 1, nx, nx*ny.
    assert np.mean(np.isin(nb - o, [1, nx, nx * ny])) < 0.5


@pytest.mark.parametrize("tiles,part", [(1, gb.PART_AUTO), (4, gb.PART_RCB), (5, gb.PART_BFS),
                                        (6, gb.PART_CONTIGUOUS)])
def test_ldu_layout_matches_oracle(oracle, tiles, part):
    h = gb.generateLduMesh(6, 5, 4, numTiles=tiles, partitioner=part)
    o, nb, lo, up, dg = h.ldu()
    om = oracle.ldu(h.numRows, o, nb, dg, lo, up, tiles, h.rowToTile())
    compare_layout(h, om)


def test_ldu_input_checks():
    n = 4
    d = np.ones(n)
    ok = gb.HostMatrix.from_ldu(n, [0, 1], [1, 3], d, [-0.5, -0.5])
    assert ok.numOffDiag == 4
    for owner, nb in [([1, 0], [1, 3]),      # owner == neighbour
                      ([2, 0], [3, 1]),      # not sorted by owner
                      ([0, 0], [1, 1]),      # duplicate face
                      ([0, 1], [1, 4])]:     # out of range
        with pytest.raises(gb.GrapheneError):
            gb.HostMatrix.from_ldu(n, owner, nb, d, [-0.5, -0.5])


def test_oracle_ldu_spmv_matches_python_restatement(oracle):
    n = 40
    owner, nb, diag, lower, upper = random_ldu(n, 3, seed=1)
    om = oracle.ldu(n, owner, nb, diag, lower, upper, 1, np.zeros(n, np.int32))
    x = np.random.default_rng(2).standard_normal(n).astype(F32)
    np.testing.assert_array_equal(om.spmv(x), py_ldu_spmv_f32(n, owner, nb, lower, upper, diag, x))


def test_oracle_ldu_matches_scipy_fp64(oracle):
    n = 60
    owner, nb, diag, lower, upper = random_ldu(n, 2, seed=3)
    om = oracle.ldu(n, owner, nb, diag, lower, upper, 1, np.zeros(n, np.int32), value_type=1)
    A = scipy_ldu(n, owner, nb, diag, lower, upper)
    x = np.random.default_rng(4).standard_normal(n)
    b = np.random.default_rng(5).standard_normal(n)
    np.testing.assert_allclose(om.spmv(x), A @ x, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(om.residual(x, 1, b, 1, 1), b - A @ x, rtol=1e-12, atol=1e-12)


def test_oracle_ldu_row_sums_do_not_depend_on_the_partition(oracle):
    """The LDU summation order of a row is fixed by the faces, so the SpMV is
    bit-identical for every partitioning."""
    h1 = gb.generateLduMesh(6, 5, 4, numTiles=1)
    o, nb, lo, up, dg = h1.ldu()
    n = h1.numRows
    x = np.random.default_rng(6).standard_normal(n).astype(F32)
    ref = oracle.ldu(n, o, nb, dg, lo, up, 1, np.zeros(n, np.int32)).spmv(x)
    h = gb.generateLduMesh(6, 5, 4, numTiles=7, partitioner=gb.PART_BFS)
    om = oracle.ldu(n, o, nb, dg, lo, up, 7, h.rowToTile())
    y = h.composeVector(om.spmv(h.decomposeVector(x)))
    np.testing.assert_array_equal(y, ref)


# ---- GPU ------------------------------------------------------------------------------

def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ldu_cases():
    yield "mesh_p1", lambda: gb.generateLduMesh(8, 7, 6, numTiles=1)
    yield "mesh_rcb", lambda: gb.generateLduMesh(8, 7, 6, numTiles=6, partitioner=gb.PART_RCB)
    yield "mesh_bfs", lambda: gb.generateLduMesh(8, 7, 6, numTiles=5, partitioner=gb.PART_BFS)

    def rnd():
        o, nb, d, lo, up = random_ldu(300, 3, seed=9)
        return gb.HostMatrix.from_ldu(300, o, nb, d, lo, up, numTiles=4, partitioner=gb.PART_BFS)
    yield "random_nonsym", rnd


@pytest.mark.gpu
@pytest.mark.parametrize("name", [c[0] for c in ldu_cases()])
@pytest.mark.parametrize("vt", [gb.FLOAT32, gb.FLOAT64])
def test_ldu_spmv_bit_exact(oracle, name, vt):
    make = dict(ldu_cases())[name]
    h = make()
    if vt == gb.FLOAT64:
        h = h.astype(gb.FLOAT64)
    o, nb, lo, up, dg = h.ldu()
    om = oracle.ldu(h.numRows, o, nb, dg, lo, up, h.numTiles, h.rowToTile(), value_type=vt)
    A = h.copyToTile()
    t = np.float32 if vt == gb.FLOAT32 else np.float64
    x = np.random.default_rng(1).standard_normal(h.numRows).astype(t)
    y = (A * dev(x)).cpu().numpy()
    np.testing.assert_array_equal(y, om.spmv(x))


@pytest.mark.gpu
@pytest.mark.parametrize("name", [c[0] for c in ldu_cases()])
def test_ldu_residual_bit_exact(oracle, name):
    h = dict(ldu_cases())[name]()
    o, nb, lo, up, dg = h.ldu()
    om = oracle.ldu(h.numRows, o, nb, dg, lo, up, h.numTiles, h.rowToTile())
    A = h.copyToTile()
    rng = np.random.default_rng(2)
    n = h.numRows
    x32 = rng.standard_normal(n).astype(F32)
    x64 = rng.standard_normal(n)
    b = rng.standard_normal(n).astype(F32)
    got = A.residual(dev(x64), dev(b), destType=gb.FLOAT32, intermediateType=gb.FLOAT64).cpu().numpy()
    np.testing.assert_array_equal(got, om.residual(x64, 1, b, 0, 1))
    got = A.residual(dev(x32), dev(b), destType=gb.FLOAT32, intermediateType=gb.FLOAT32).cpu().numpy()
    np.testing.assert_array_equal(got, om.residual(x32, 0, b, 0, 0))
    xdw = np.stack([x32, (x64 * 2.0 ** -26).astype(F32)], axis=1).reshape(-1).copy()
    got = A.residual(dev(xdw), dev(b), destType=gb.FLOAT32, intermediateType=gb.TWOFLOAT32,
                     xType=gb.TWOFLOAT32).cpu().numpy()
    np.testing.assert_array_equal(got, om.residual(xdw, 2, b, 0, 2))


@pytest.mark.gpu
def test_ldu_gs_pbicgstab_matches_oracle(oracle):
    h = gb.generateLduMesh(10, 9, 8, numTiles=8, partitioner=gb.PART_RCB)
    o, nb, lo, up, dg = h.ldu()
    om = oracle.ldu(h.numRows, o, nb, dg, lo, up, h.numTiles, h.rowToTile())
    A = h.copyToTile()
    n = h.numRows
    xt = np.random.default_rng(4).standard_normal(n).astype(F32)
    b = om.spmv(xt)
    for k in (1, 3):
        cfg = {"type": "PBiCGStab", "maxIterations": k,
               "preconditioner": {"type": "GaussSeidel", "numSweeps": 2, "numFixedIterations": 2}}
        x = dev(np.zeros(n, F32))
        gb.Solver(A, cfg).solve(x, dev(b))
        ox, _, _, _ = om.solve(json.dumps(cfg), np.zeros(n, F32), b)
        g = x.cpu().numpy()
        assert np.max(np.abs(g - ox)) <= 1e-5 * max(1.0, np.max(np.abs(ox)))
    cfg = {"type": "PBiCGStab", "maxIterations": 2000, "relResidual": 1e-6,
           "preconditioner": {"type": "GaussSeidel", "numSweeps": 2, "numFixedIterations": 2}}
    x = dev(np.zeros(n, F32))
    st = gb.Solver(A, cfg).solve(x, dev(b))
    _, ost, _, _ = om.solve(json.dumps(cfg), np.zeros(n, F32), b)
    assert st.converged and ost.converged
    assert abs(st.iterations - ost.iterations) <= 2
