"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

Test infrastructure only: tests and bench.py's CPU baseline use it as the
checker / baseline; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "oracle" / "liboracle.so"

vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int32


class OrStats(C.Structure):
    _fields_ = [("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("b_norm", C.c_double), ("iterations", i32), ("converged", i32),
                ("singular", i32), ("inner_iterations", i32)]


def _p(a):
    return C.c_void_p(None) if a is None else C.c_void_p(a.ctypes.data)


def build_oracle() -> Path:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return LIB


class Oracle:
    def __init__(self):
        if not LIB.exists():
            build_oracle()
        L = C.CDLL(str(LIB))
        sig = {
            "or_build": (vp, [i64, i64, vp, vp, vp, i64, vp, C.c_int]),
            "or_build_ldu": (vp, [i64, i64, vp, vp, vp, vp, vp, i64, vp, C.c_int]),
            "or_poisson": (vp, [i64, i64, i64, i64, vp, C.c_int]),
            "or_free": (None, [vp]),
            "or_last_error": (C.c_char_p, []),
            "or_set_threads": (None, [C.c_int]),
            "or_num_rows": (i64, [vp]), "or_num_tiles": (i64, [vp]),
            "or_num_off_diag": (i64, [vp]), "or_num_halo": (i64, [vp]),
            "or_row_to_tile": (C.c_int, [vp, vp]),
            "or_tile_sizes": (C.c_int, [vp, vp]),
            "or_local_to_global": (C.c_int, [vp, vp]),
            "or_local_crs": (C.c_int, [vp, vp, vp, vp, vp]),
            "or_colors": (C.c_int, [vp, vp]),
            "or_multicolor_recommended": (C.c_int, [vp]),
            "or_spmv": (C.c_int, [vp, vp, vp, C.c_int]),
            "or_residual": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int]),
            "or_norm": (C.c_double, [vp, vp, C.c_int, C.c_int]),
            "or_reduce_sum": (C.c_double, [vp, i64, C.c_int]),
            "or_ref_dot": (C.c_double, [vp, vp, vp, C.c_int]),
            "or_ref_norm": (C.c_double, [vp, vp, C.c_int, C.c_int]),
            "or_ilu_factorize": (C.c_int, [vp, C.c_int, vp, vp]),
            "or_ilu_solve": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, C.c_int]),
            "or_gs_sweep": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int]),
            "or_solve": (C.c_int, [vp, C.c_char_p, vp, C.c_int, vp, C.c_int, C.POINTER(OrStats),
                                   vp, vp, C.c_int]),
            "or_generate_nnz": (i64, [i64, i64, i64]),
            "or_generate": (C.c_int, [C.c_int, i64, i64, i64, vp, C.c_uint64, vp, vp, vp, vp]),
            "or_random_vector": (C.c_int, [C.c_uint64, i64, C.c_int, C.c_double, C.c_double, vp]),
            "or_partition_rcb": (C.c_int, [i64, vp, vp, i32, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L

    def err(self):
        return self.L.or_last_error().decode()

    def check(self, rc):
        if rc != 0:
            raise RuntimeError(self.err())

    def threads(self, n: int):
        self.L.or_set_threads(n)

    def matrix(self, n, rows, cols, vals, num_tiles, row_to_tile, value_type=0) -> "OMatrix":
        r = np.ascontiguousarray(rows, np.int64)
        c = np.ascontiguousarray(cols, np.int64)
        v = np.ascontiguousarray(vals, np.float64)
        rt = None if row_to_tile is None else np.ascontiguousarray(row_to_tile, np.int32)
        h = self.L.or_build(n, len(v), _p(r), _p(c), _p(v), num_tiles, _p(rt), value_type)
        if not h:
            raise RuntimeError(self.err())
        return OMatrix(self, h, value_type)

    def ldu(self, n, owner, neighbour, diag, lower, upper, num_tiles, row_to_tile,
            value_type=0) -> "OMatrix":
        a = [np.ascontiguousarray(v, t) for v, t in ((owner, np.int64), (neighbour, np.int64),
                                                     (diag, np.float64), (lower, np.float64))]
        up = None if upper is None else np.ascontiguousarray(upper, np.float64)
        rt = None if row_to_tile is None else np.ascontiguousarray(row_to_tile, np.int32)
        h = self.L.or_build_ldu(n, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(up),
                                num_tiles, _p(rt), value_type)
        if not h:
            raise RuntimeError(self.err())
        return OMatrix(self, h, value_type)

    # -- seeded benchmark inputs (oracle/generators.cpp) -------------------
    def generate(self, kind, nx, ny, nz, params=(), seed=0):
        """(rows, cols, vals, coords[n, 3]) of a 7-point matrix: kind 0
        constant Poisson, 1 variable-coefficient (params = (sigma,)), 2
        convection-diffusion (params = velocity)."""
        nnz = self.L.or_generate_nnz(nx, ny, nz)
        if nnz < 0:
            raise ValueError("grid dimensions must be positive")
        r = np.empty(nnz, np.int64)
        c = np.empty(nnz, np.int64)
        v = np.empty(nnz, np.float64)
        xyz = np.empty((nx * ny * nz, 3), np.float64)
        p = np.array(list(params) + [0.0] * (3 - len(params)), np.float64)
        self.check(self.L.or_generate(kind, nx, ny, nz, _p(p), seed, _p(r), _p(c), _p(v), _p(xyz)))
        return r, c, v, xyz

    def random_vector(self, seed, n, dist="uniform", lo=-1.0, hi=1.0):
        out = np.empty(n, np.float64)
        self.check(self.L.or_random_vector(seed, n, 0 if dist == "uniform" else 1, lo, hi, _p(out)))
        return out

    def partition_rcb(self, coords, weights, parts):
        coords = np.ascontiguousarray(coords, np.float64)
        w = np.ascontiguousarray(weights, np.int64)
        out = np.empty(len(w), np.int32)
        self.check(self.L.or_partition_rcb(len(w), _p(coords), _p(w), parts, _p(out)))
        return out

    def grid_system(self, kind, nx, ny, nz, params, seed, num_tiles, value_type=0):
        """A generated 7-point matrix partitioned by coordinate bisection
        into num_tiles tiles (vertex weight: row off-diagonals + 1), built as
        an oracle matrix: the benchmark's systems without the product
        library."""
        r, c, v, xyz = self.generate(kind, nx, ny, nz, params, seed)
        n = nx * ny * nz
        w = np.bincount(r, minlength=n).astype(np.int64)  # row entries = off-diagonals + 1
        rt = self.partition_rcb(xyz, w, num_tiles) if num_tiles > 1 else None
        return self.matrix(n, r, c, v, num_tiles, rt, value_type)

    def poisson(self, nx, ny, nz, num_tiles, row_to_tile, value_type=0) -> "OMatrix":
        rt = None if row_to_tile is None else np.ascontiguousarray(row_to_tile, np.int32)
        h = self.L.or_poisson(nx, ny, nz, num_tiles, _p(rt), value_type)
        if not h:
            raise RuntimeError(self.err())
        return OMatrix(self, h, value_type)


class OMatrix:
    def __init__(self, o: Oracle, h, vt):
        self.o, self.h, self.vt = o, h, vt
        L = o.L
        self.n = L.or_num_rows(h)
        self.P = L.or_num_tiles(h)
        self.m = L.or_num_off_diag(h)
        self.nhalo = L.or_num_halo(h)

    def __del__(self):
        if getattr(self, "h", None):
            self.o.L.or_free(self.h)
            self.h = None

    def tile_order(self):
        """Natural row index of every tile-order position."""
        sizes = self.tile_sizes()
        l2g = self.local_to_global()
        out, o = [], 0
        for ni, ns, nh in sizes:
            out.append(l2g[o:o + ni + ns])
            o += ni + ns + nh
        return np.concatenate(out) if out else np.empty(0, np.int64)

    def decompose(self, natural):
        """Natural-order vector to tile order."""
        return np.ascontiguousarray(np.asarray(natural)[self.tile_order()])

    def row_to_tile(self):
        out = np.empty(self.n, np.int32)
        self.o.check(self.o.L.or_row_to_tile(self.h, _p(out)))
        return out

    def tile_sizes(self):
        out = np.empty((self.P, 3), np.int64)
        self.o.check(self.o.L.or_tile_sizes(self.h, _p(out)))
        return out

    def local_to_global(self):
        out = np.empty(self.n + self.nhalo, np.int64)
        self.o.check(self.o.L.or_local_to_global(self.h, _p(out)))
        return out

    def local_crs(self):
        rp = np.empty(self.n + self.P, np.int64)
        ci = np.empty(self.m, np.int32)
        od = np.empty(self.m, np.float64)
        dg = np.empty(self.n, np.float64)
        self.o.check(self.o.L.or_local_crs(self.h, _p(rp), _p(ci), _p(od), _p(dg)))
        return rp, ci, od, dg

    def colors(self):
        out = np.empty(self.n, np.int32)
        self.o.check(self.o.L.or_colors(self.h, _p(out)))
        return out

    def multicolor_recommended(self):
        return bool(self.o.L.or_multicolor_recommended(self.h))

    def spmv(self, x):
        t = 0 if x.dtype == np.float32 else 1
        x = np.ascontiguousarray(x)
        y = np.empty_like(x)
        self.o.check(self.o.L.or_spmv(self.h, _p(x), _p(y), t))
        return y

    def residual(self, x, xt, b, rt, it):
        """xt/rt/it: 0 f32, 1 f64, 2 double-word (x as float32 pairs)."""
        bt = 0 if b.dtype == np.float32 else 1
        r = np.empty(self.n, np.float32 if rt == 0 else np.float64)
        self.o.check(self.o.L.or_residual(self.h, _p(np.ascontiguousarray(x)), xt,
                                          _p(np.ascontiguousarray(b)), bt, _p(r), rt, it))
        return r

    def norm(self, x, norm):
        t = 0 if x.dtype == np.float32 else 1
        return self.o.L.or_norm(self.h, _p(np.ascontiguousarray(x)), t, norm)

    def ref_dot(self, a, b):
        """a . b in the reference's reduction order and operand type."""
        t = 0 if a.dtype == np.float32 else 1
        return self.o.L.or_ref_dot(self.h, _p(np.ascontiguousarray(a)), _p(np.ascontiguousarray(b)), t)

    def ref_norm(self, x, norm=1):
        t = 0 if x.dtype == np.float32 else 1
        return self.o.L.or_ref_norm(self.h, _p(np.ascontiguousarray(x)), t, norm)

    def ilu_factorize(self, dilu=False):
        off = np.empty(self.m, np.float64)
        inv = np.empty(self.n, np.float64)
        self.o.check(self.o.L.or_ilu_factorize(self.h, int(dilu), _p(off), _p(inv)))
        return off, inv

    def ilu_solve(self, off, inv, b, dilu=False):
        t = 0 if b.dtype == np.float32 else 1
        x = np.empty_like(b)
        self.o.check(self.o.L.or_ilu_solve(self.h, int(dilu), _p(off), _p(inv),
                                           _p(np.ascontiguousarray(b)), _p(x), t))
        return x

    def gs_sweep(self, x, b, seed_b=True, drop_halo=False):
        t = 0 if x.dtype == np.float32 else 1
        x = np.array(x, copy=True)
        self.o.check(self.o.L.or_gs_sweep(self.h, _p(x), _p(np.ascontiguousarray(b)), t,
                                          int(seed_b), int(drop_halo)))
        return x

    def solve(self, config: str, x, b, history_len=0, want_phi=False):
        xt = 0 if x.dtype == np.float32 else 1
        bt = 0 if b.dtype == np.float32 else 1
        x = np.array(x, copy=True)
        st = OrStats()
        phi = np.empty(self.n, np.float64) if want_phi else None
        hist = np.empty(history_len, np.float64) if history_len else None
        self.o.check(self.o.L.or_solve(self.h, config.encode(), _p(x), xt,
                                       _p(np.ascontiguousarray(b)), bt, C.byref(st), _p(phi),
                                       _p(hist), history_len))
        return x, st, phi, hist
