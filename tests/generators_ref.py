"""Independent restatement of the seeded benchmark generators (test
infrastructure only).

The benchmark configurations' matrices come from seeded generators that
the reference does not have (it reads SuiteSparse files, benchmark.py:104-109,
or builds the constant-coefficient Poisson stencil, Poisson.cpp:26-69). This
module restates their definitions from scratch in numpy, so that the
library's generators (and the oracle's copy used by the reference arm of the
benchmark) are pinned by code that shares nothing with them:

* the counter-based stream: splitmix64 finaliser (Steele, Lea, Flood,
  OOPSLA 2014) of ``mix64(seed) ^ (i * 0xD1B54A32D192ED03)``, top 53 bits
  scaled to [0, 1); standard normals by Box-Muller on outputs 2i and 2i+1;
* variable-coefficient Poisson: cell conductivity ``exp(sigma * N(0,1))``,
  face coefficient the harmonic mean ``2 k_a k_b / (k_a + k_b)``,
  off-diagonal ``-face``, diagonal the sum of the six face terms in the order
  -z, -y, -x, +x, +y, +z with ``2 k`` for a boundary face;
* upwind convection-diffusion: ``-(1 + v_d)`` upstream, ``-1`` downstream,
  diagonal ``((6 + vx) + vy) + vz`` everywhere;
* the LDU hexahedral mesh: Fisher-Yates cell permutation, faces (min id,
  max id) sorted, coefficients ``10^U(-2, 2)``, diagonal the face sum in face
  order plus 1e-3, centroids of the jittered nodes.

Transcendental functions go through Python's ``math`` module, i.e. the C
library's exp / log / cos / pow, the same routines the C++ generators call,
so results are comparable bit for bit (numpy's own SIMD exp and log may
round differently). Rows are in natural order ``i + nx (j + ny k)``.
"""
from __future__ import annotations

import math

import numpy as np

_U = np.uint64


def mix64(z: np.ndarray) -> np.ndarray:
    z = z + _U(0x9E3779B97F4A7C15)
    z = (z ^ (z >> _U(30))) * _U(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U(27))) * _U(0x94D049BB133111EB)
    return z ^ (z >> _U(31))


def uniform01(seed: int, idx) -> np.ndarray:
    i = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = mix64(mix64(np.array([seed], dtype=np.uint64))[0] ^ (i * _U(0xD1B54A32D192ED03)))
    return (z >> _U(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform(seed: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    return lo + (hi - lo) * uniform01(seed, np.arange(n, dtype=np.uint64))


def normal(seed: int, n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.uint64)
    u1 = 1.0 - uniform01(seed, 2 * i)
    u2 = uniform01(seed, 2 * i + _U(1))
    two_pi = 6.283185307179586476925
    return np.array([math.sqrt(-2.0 * math.log(a)) * math.cos(two_pi * b) for a, b in zip(u1, u2)])


def _grid(nx, ny, nz):
    r = np.arange(nx * ny * nz, dtype=np.int64)
    return r, r % nx, (r // nx) % ny, r // (nx * ny)


def _seven_point(nx, ny, nz, coef, diag):
    """Triplets of a 7-point matrix, each row sorted by column: -z, -y, -x,
    diagonal, +x, +y, +z. coef(d) -> values for the rows that have neighbour
    d (direction 0..5 = -z, -y, -x, +x, +y, +z), diag -> all diagonal values."""
    r, i, j, k = _grid(nx, ny, nz)
    off = [-nx * ny, -nx, -1, 1, nx, nx * ny]
    has = [k > 0, j > 0, i > 0, i < nx - 1, j < ny - 1, k < nz - 1]
    parts = []  # (rows, cols, vals, slot) with slot giving the in-row order
    for slot, d in zip([0, 1, 2, 4, 5, 6], range(6)):
        m = has[d]
        parts.append((r[m], r[m] + off[d], coef(d)[m], np.full(m.sum(), slot)))
    parts.append((r, r, diag, np.full(len(r), 3)))
    rows = np.concatenate([p[0] for p in parts])
    cols = np.concatenate([p[1] for p in parts])
    vals = np.concatenate([p[2] for p in parts])
    slot = np.concatenate([p[3] for p in parts])
    order = np.lexsort((slot, rows))
    return rows[order], cols[order], vals[order]


def var_poisson(nx, ny, nz, sigma, seed):
    """(rows, cols, vals) of the variable-coefficient 7-point Poisson matrix."""
    n = nx * ny * nz
    kc = np.array([math.exp(sigma * g) for g in normal(seed, n)])
    r, i, j, k = _grid(nx, ny, nz)
    off = [-nx * ny, -nx, -1, 1, nx, nx * ny]
    has = [k > 0, j > 0, i > 0, i < nx - 1, j < ny - 1, k < nz - 1]

    def face(d):
        nb = np.clip(r + off[d], 0, n - 1)
        a, b = kc, kc[nb]
        return 2.0 * a * b / (a + b)
    faces = [face(d) for d in range(6)]
    s = np.zeros(n)
    for d in range(6):
        s = s + np.where(has[d], faces[d], 2.0 * kc)
    return _seven_point(nx, ny, nz, lambda d: -faces[d], s)


def conv_diff(nx, ny, nz, vx, vy, vz):
    """(rows, cols, vals) of the upwind convection-diffusion matrix."""
    n = nx * ny * nz
    up = [-(1.0 + vz), -(1.0 + vy), -(1.0 + vx), -1.0, -1.0, -1.0]
    dg = 6.0 + vx + vy + vz
    return _seven_point(nx, ny, nz, lambda d: np.full(n, up[d]), np.full(n, dg))


def ldu_mesh(nx, ny, nz, jitter_seed, perm_seed, coef_seed):
    """(owner, neighbour, lower, diag, coords[n, 3]) of the jittered,
    cell-permuted hexahedral mesh with log-uniform face coefficients."""
    n = nx * ny * nz
    ids = list(range(n))
    u = uniform(perm_seed, max(n - 1, 1), 0.0, 1.0)
    for i in range(n - 1, 0, -1):
        jj = min(int(u[n - 1 - i] * float(i + 1)), i)
        ids[i], ids[jj] = ids[jj], ids[i]
    faces = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                g = i + nx * (j + ny * k)
                for ok, g2 in ((i + 1 < nx, g + 1), (j + 1 < ny, g + nx), (k + 1 < nz, g + nx * ny)):
                    if ok:
                        a, b = ids[g], ids[g2]
                        faces.append((min(a, b), max(a, b)))
    faces.sort()
    F = len(faces)
    owner = np.array([f[0] for f in faces], dtype=np.int64)
    neigh = np.array([f[1] for f in faces], dtype=np.int64)
    uc = uniform(coef_seed, F, -2.0, 2.0)
    c = np.array([math.pow(10.0, v) for v in uc])
    s = [0.0] * n
    for f in range(F):
        s[owner[f]] += c[f]
        s[neigh[f]] += c[f]
    diag = np.array(s) + 1e-3
    mx, my, mz = nx + 1, ny + 1, nz + 1
    jit = uniform(jitter_seed, 3 * mx * my * mz, -0.2, 0.2)
    coords = np.zeros((n, 3))
    for g in range(n):
        i, j, k = g % nx, (g // nx) % ny, g // (nx * ny)
        acc = [0.0, 0.0, 0.0]
        for dz in range(2):
            for dy in range(2):
                for dx in range(2):
                    node = (i + dx) + mx * ((j + dy) + my * (k + dz))
                    acc[0] += float(i + dx) + jit[3 * node]
                    acc[1] += float(j + dy) + jit[3 * node + 1]
                    acc[2] += float(k + dz) + jit[3 * node + 2]
        coords[ids[g]] = [a / 8.0 for a in acc]
    return owner, neigh, -c, diag, coords
