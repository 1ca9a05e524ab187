"""Shared helpers for the tests: seeded synthetic matrices."""
from __future__ import annotations

import numpy as np


def poisson_coo(nx, ny, nz):
    """7-point Poisson triplets in the reference's emission order
    (matrix/host/details/Poisson.cpp:38-63)."""
    rows, cols, vals = [], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                r = k * nx * ny + j * nx + i
                ent = [(r, 6.0)]
                if i > 0: ent.append((r - 1, -1.0))
                if i < nx - 1: ent.append((r + 1, -1.0))
                if j > 0: ent.append((r - nx, -1.0))
                if j < ny - 1: ent.append((r + nx, -1.0))
                if k > 0: ent.append((r - nx * ny, -1.0))
                if k < nz - 1: ent.append((r + nx * ny, -1.0))
                for c, v in ent:
                    rows.append(r); cols.append(c); vals.append(v)
    return nx * ny * nz, np.array(rows, np.int64), np.array(cols, np.int64), np.array(vals)


def random_coo(n, density, seed, symmetric=True, diag_dominant=True):
    """Random sparse matrix with a full diagonal; symmetric structure when
    `symmetric` (values differ), triplets shuffled."""
    rng = np.random.default_rng(seed)
    mask = rng.random((n, n)) < density
    np.fill_diagonal(mask, False)
    if symmetric:
        mask = mask | mask.T
    r, c = np.nonzero(mask)
    v = -rng.uniform(0.1, 1.0, size=len(r))
    rowsum = np.zeros(n)
    np.add.at(rowsum, r, np.abs(v))
    d = rowsum + (1.0 if diag_dominant else 0.0) + rng.uniform(0, 0.5, size=n)
    rows = np.concatenate([r, np.arange(n)])
    cols = np.concatenate([c, np.arange(n)])
    vals = np.concatenate([v, d])
    perm = rng.permutation(len(rows))
    return n, rows[perm].astype(np.int64), cols[perm].astype(np.int64), vals[perm]
