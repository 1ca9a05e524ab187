"""graphene_b200: B200-native sparse-solver hot path of the Graphene framework.

Python mirror of the reference's matrix / solver surface
(libgraphene/matrix, esa-tu-darmstadt/graphene) over the C ABI in
``include/graphene_gpu.h``:

* ``generate3DPoissonMatrix`` / ``loadMatrixFromFile`` / ``HostMatrix.from_coo``
  -> ``HostMatrix`` (matrix/host/HostMatrix.hpp:31-96)
* ``HostMatrix.copyToTile()`` -> ``Matrix`` on the current CUDA device
  (matrix/Matrix.hpp:29-131): ``A * x``, ``A.residual``, ``A.vectorNorm``,
  ``A.solve(x, b, config)``, ``A.createUninitializedVector``
* ``Configuration.fromJSON`` + ``Solver.createSolver`` (matrix/solver/)

Device vectors are ``torch`` tensors in tile order (the reference's
decomposed vector layout without halo cells); ``HostMatrix.decomposeVector``
and ``composeVector`` convert from / to natural row order. All numerical work
runs in the CUDA kernels of ``lib/libgraphene_b200.so``; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import json as _json
from dataclasses import dataclass
from typing import Any, Optional, Union

import numpy as np

from . import _lib
from ._lib import (FLOAT32, FLOAT64, NORM_L1, NORM_L2, NORM_LINF, NORM_NONE, PART_AUTO, PART_BFS,
                   PART_CONTIGUOUS, PART_EXPLICIT, PART_MULTILEVEL, PART_RCB, TWOFLOAT32, GrapheneError, check)

__all__ = [
    "FLOAT32", "FLOAT64", "TWOFLOAT32", "NORM_L1", "NORM_L2", "NORM_LINF",
    "PART_AUTO", "PART_CONTIGUOUS", "PART_RCB", "PART_BFS", "PART_EXPLICIT", "PART_MULTILEVEL",
    "GrapheneError", "HostMatrix", "Matrix", "Configuration", "Solver", "SolverStats",
    "generate3DPoissonMatrix", "loadMatrixFromFile", "parseType", "launch_count",
    "generateMatrix", "generateMatrixLike", "generateValues", "generateLduMesh", "randomVector", "Server", "Batch",
]

_NP = {FLOAT32: np.float32, FLOAT64: np.float64}
_NAMES = {"float32": FLOAT32, "float": FLOAT32, "float64": FLOAT64, "double": FLOAT64,
          "twofloat32": TWOFLOAT32}


def parseType(name: Union[str, int]) -> int:
    """common/Type.cpp parseType: "float32" | "float64" | "twofloat32"."""
    if isinstance(name, int):
        return name
    if name not in _NAMES:
        raise ValueError(f"Unknown type: {name}")
    return _NAMES[name]


def launch_count() -> int:
    """Kernel launches issued by the native library so far."""
    return int(_lib.lib().gr_launch_count())


def _torch():
    import torch  # plumbing for device memory only
    return torch


def _torch_dtype(t: int):
    torch = _torch()
    if t == FLOAT32:
        return torch.float32
    if t == FLOAT64:
        return torch.float64
    raise ValueError("twofloat32 vectors are stored as float32 pairs; use FLOAT32 with 2*n")


def _dtype_of(tensor) -> int:
    torch = _torch()
    if tensor.dtype == torch.float32:
        return FLOAT32
    if tensor.dtype == torch.float64:
        return FLOAT64
    raise TypeError(f"unsupported vector dtype {tensor.dtype}")


def _ptr(a) -> C.c_void_p:
    if a is None:
        return C.c_void_p(None)
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())


@dataclass
class SolverStats:
    """matrix/solver/SolverStats.hpp:29-69 (norms accumulated in FP64)."""
    initialResidual: float
    finalResidual: float
    bNorm: float
    iterations: int
    converged: bool
    singular: bool
    status: int
    innerIterations: int
    solveMs: float

    @staticmethod
    def _from(s: _lib.Stats) -> "SolverStats":
        return SolverStats(s.initial_residual, s.final_residual, s.b_norm, s.iterations,
                           bool(s.converged), bool(s.singular), s.status, s.inner_iterations,
                           s.solve_ms)


class HostMatrix:
    """Host-side matrix with its tile layout (matrix/host/HostMatrix.hpp)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        info = _lib.MatrixInfo()
        check(_lib.lib().gr_host_matrix_get_info(self._h, C.byref(info)))
        self.info = info

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            try:
                _lib.lib().gr_host_matrix_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- constructors ------------------------------------------------------
    @staticmethod
    def from_coo(n: int, rows, cols, vals, numTiles: int, partitioner: int = PART_AUTO,
                 rowToTile=None, coords=None, valueType: int = FLOAT32) -> "HostMatrix":
        """HostMatrix(MatrixFormat::CRS, TripletMatrix, numTiles)."""
        r = np.ascontiguousarray(rows, dtype=np.int64)
        c = np.ascontiguousarray(cols, dtype=np.int64)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        rt = None if rowToTile is None else np.ascontiguousarray(rowToTile, dtype=np.int32)
        cd = None if coords is None else np.ascontiguousarray(coords, dtype=np.float64)
        if rt is not None:
            partitioner = PART_EXPLICIT
        h = C.c_void_p()
        check(_lib.lib().gr_host_matrix_from_coo(n, len(v), _ptr(r), _ptr(c), _ptr(v), numTiles,
                                                  partitioner, _ptr(rt), _ptr(cd), valueType,
                                                  C.byref(h)))
        return HostMatrix(h)

    @staticmethod
    def from_ldu(numCells: int, owner, neighbour, diag, lower, upper=None, numTiles: int = 1,
                 partitioner: int = PART_AUTO, rowToTile=None, coords=None,
                 valueType: int = FLOAT32) -> "HostMatrix":
        """LDU matrix (matrix/details/ldu/LDUMatrix.hpp): faces owner <
        neighbour sorted by owner, coefficients in face order (upper None:
        symmetric)."""
        o = np.ascontiguousarray(owner, dtype=np.int64)
        nb = np.ascontiguousarray(neighbour, dtype=np.int64)
        d = np.ascontiguousarray(diag, dtype=np.float64)
        lo = np.ascontiguousarray(lower, dtype=np.float64)
        up = None if upper is None else np.ascontiguousarray(upper, dtype=np.float64)
        rt = None if rowToTile is None else np.ascontiguousarray(rowToTile, dtype=np.int32)
        cd = None if coords is None else np.ascontiguousarray(coords, dtype=np.float64)
        if rt is not None:
            partitioner = PART_EXPLICIT
        h = C.c_void_p()
        check(_lib.lib().gr_host_matrix_from_ldu(numCells, len(o), _ptr(o), _ptr(nb), _ptr(d), _ptr(lo),
                                                  _ptr(up), numTiles, partitioner, _ptr(rt), _ptr(cd),
                                                  valueType, C.byref(h)))
        return HostMatrix(h)

    @property
    def isLdu(self) -> bool:
        return self.info.format == FORMAT_LDU

    def ldu(self):
        """(owner, neighbour, lower, upper, diag) of an LDU matrix, natural
        numbering, values rounded to the stored type."""
        nf = C.c_int64()
        check(_lib.lib().gr_host_matrix_get_ldu(self._h, C.byref(nf), None, None, None, None, None))
        F, n = nf.value, self.numRows
        o, nb = np.empty(F, np.int64), np.empty(F, np.int64)
        lo, up, dg = np.empty(F), np.empty(F), np.empty(n)
        check(_lib.lib().gr_host_matrix_get_ldu(self._h, C.byref(nf), _ptr(o), _ptr(nb), _ptr(lo),
                                                _ptr(up), _ptr(dg)))
        return o, nb, lo, up, dg

    # -- layout queries ----------------------------------------------------
    @property
    def numRows(self) -> int:
        return self.info.num_rows

    @property
    def numTiles(self) -> int:
        return self.info.num_tiles

    @property
    def numOffDiag(self) -> int:
        return self.info.num_off_diag

    def multicolorRecommended(self) -> bool:
        return bool(self.info.multicolor_recommended)

    def rowToTile(self) -> np.ndarray:
        out = np.empty(self.numRows, dtype=np.int32)
        check(_lib.lib().gr_host_matrix_row_to_tile(self._h, _ptr(out)))
        return out

    def tileSizes(self) -> np.ndarray:
        out = np.empty((self.numTiles, 3), dtype=np.int64)
        check(_lib.lib().gr_host_matrix_tile_sizes(self._h, _ptr(out)))
        return out

    def localToGlobal(self) -> np.ndarray:
        out = np.empty(self.numRows + self.info.num_halo_total, dtype=np.int64)
        check(_lib.lib().gr_host_matrix_local_to_global(self._h, _ptr(out)))
        return out

    def localCrs(self):
        rp = np.empty(self.numRows + self.numTiles, dtype=np.int64)
        ci = np.empty(self.numOffDiag, dtype=np.int32)
        od = np.empty(self.numOffDiag, dtype=np.float64)
        dg = np.empty(self.numRows, dtype=np.float64)
        check(_lib.lib().gr_host_matrix_local_crs(self._h, _ptr(rp), _ptr(ci), _ptr(od), _ptr(dg)))
        return rp, ci, od, dg

    def levels(self):
        lo = np.empty(self.numRows, dtype=np.int32)
        up = np.empty(self.numRows, dtype=np.int32)
        check(_lib.lib().gr_host_matrix_levels(self._h, _ptr(lo), _ptr(up)))
        return lo, up

    # -- vectors -----------------------------------------------------------
    def decomposeVector(self, vec, t: int = FLOAT32) -> np.ndarray:
        """DistributedTileLayout::decomposeVector without halo cells."""
        a = np.ascontiguousarray(vec, dtype=_NP[t])
        out = np.empty_like(a)
        check(_lib.lib().gr_host_matrix_decompose_vector(self._h, _ptr(a), _ptr(out), t))
        return out

    def loadVectorFromFile(self, t: int, path: str) -> np.ndarray:
        """DistributedTileLayout::loadVectorFromFile (DistributedTileLayout.cpp:185-206)
        without halo cells: a MatrixMarket vector, in tile order."""
        t = parseType(t)
        out = np.empty(self.numRows, dtype=_NP[t])
        check(_lib.lib().gr_host_matrix_load_vector_mm(self._h, str(path).encode(), t, _ptr(out)))
        return out

    def composeVector(self, vec, t: int = FLOAT32) -> np.ndarray:
        a = np.ascontiguousarray(vec, dtype=_NP[t])
        out = np.empty_like(a)
        check(_lib.lib().gr_host_matrix_compose_vector(self._h, _ptr(a), _ptr(out), t))
        return out

    def edgeCut(self) -> int:
        """Off-diagonal entries whose column lies in another tile
        (gr_host_matrix_edge_cut; a symmetric pattern's cut edges count twice)."""
        c = C.c_int64()
        check(_lib.lib().gr_host_matrix_edge_cut(self._h, C.byref(c)))
        return c.value

    def setSpmvLayout(self, layout: int) -> None:
        """SpMV column encoding of later device copies: -1 automatic, 0 32-bit
        columns, 1 16-bit row offsets (gr_host_matrix_set_spmv_layout)."""
        check(_lib.lib().gr_host_matrix_set_spmv_layout(self._h, layout))

    def checkSpmvLayout(self, layout: int = -1) -> dict:
        """Builds and decodes the SpMV layout on the host
        (gr_host_matrix_check_spmv_layout); raises on a mismatch."""
        c, sl, far, mx = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
        check(_lib.lib().gr_host_matrix_check_spmv_layout(self._h, layout, C.byref(c), C.byref(sl), C.byref(far),
                                                           C.byref(mx)))
        return {"compact": bool(c.value), "slots": sl.value, "far": far.value, "max_chunk_far": mx.value}

    def copyToTile(self) -> "Matrix":
        """HostMatrix::copyToTile: upload to the current CUDA device."""
        return Matrix(self)


def generate3DPoissonMatrix(valueType: int, nx: int, ny: int, nz: int, numTiles: int,
                            partitioner: int = PART_AUTO) -> HostMatrix:
    """matrix/host/HostMatrix.hpp:94-96 (7-point Poisson, Dirichlet)."""
    h = C.c_void_p()
    check(_lib.lib().gr_host_matrix_poisson(nx, ny, nz, numTiles, partitioner, parseType(valueType),
                                            C.byref(h)))
    return HostMatrix(h)


GEN_POISSON, GEN_VAR_POISSON, GEN_CONVDIFF = 0, 1, 2
FORMAT_CRS, FORMAT_LDU = 0, 1


def generateLduMesh(nx: int, ny: int, nz: int, jitterSeed: int = 4, permSeed: int = 5,
                    coefSeed: int = 6, numTiles: int = 1, partitioner: int = PART_AUTO,
                    valueType: int = FLOAT32) -> HostMatrix:
    """Jittered, cell-permuted hexahedral mesh in LDU form with log-uniform
    face coefficients (gr_host_matrix_ldu_mesh)."""
    h = C.c_void_p()
    check(_lib.lib().gr_host_matrix_ldu_mesh(nx, ny, nz, jitterSeed, permSeed, coefSeed, numTiles,
                                             partitioner, parseType(valueType), C.byref(h)))
    return HostMatrix(h)


def generateMatrix(kind: int, nx: int, ny: int, nz: int, params=(), seed: int = 0,
                   numTiles: int = 1, partitioner: int = PART_AUTO,
                   valueType: int = FLOAT32) -> HostMatrix:
    """Synthetic 7-point matrices (gr_host_matrix_generate): GEN_POISSON,
    GEN_VAR_POISSON (params = (sigma,)), GEN_CONVDIFF (params = velocity)."""
    p = (C.c_double * 3)(*(list(params) + [0.0] * (3 - len(params))))
    h = C.c_void_p()
    check(_lib.lib().gr_host_matrix_generate(kind, nx, ny, nz, p, seed, numTiles, partitioner,
                                             parseType(valueType), C.byref(h)))
    return HostMatrix(h)


def generateMatrixLike(like: HostMatrix, kind: int, nx: int, ny: int, nz: int, params=(),
                       seed: int = 0) -> HostMatrix:
    """generateMatrix with `like`'s structure (gr_host_matrix_generate_like):
    fresh values from (kind, params, seed), partition / layout / levels copied
    from `like`, which must come from the same generator and grid."""
    p = (C.c_double * 3)(*(list(params) + [0.0] * (3 - len(params))))
    h = C.c_void_p()
    check(_lib.lib().gr_host_matrix_generate_like(like._h, kind, nx, ny, nz, p, seed, C.byref(h)))
    return HostMatrix(h)


def generateValues(like: HostMatrix, kind: int, nx: int, ny: int, nz: int, params=(), seed: int = 0):
    """(gVal, gDiag): the generator's values in like's global CRS order
    (gr_host_matrix_generate_values), FP64."""
    p = (C.c_double * 3)(*(list(params) + [0.0] * (3 - len(params))))
    gv = np.empty(like.numOffDiag, np.float64)
    gd = np.empty(like.numRows, np.float64)
    check(_lib.lib().gr_host_matrix_generate_values(like._h, kind, nx, ny, nz, p, seed, _ptr(gv), _ptr(gd)))
    return gv, gd


def _structure_key(self: HostMatrix) -> int:
    k = C.c_uint64()
    check(_lib.lib().gr_host_matrix_structure_key(self._h, C.byref(k)))
    return k.value


HostMatrix.structureKey = property(_structure_key)


def randomVector(seed: int, n: int, dist: str = "uniform", lo: float = -1.0,
                 hi: float = 1.0) -> np.ndarray:
    """Seeded vector from the generators' counter-based stream (float64)."""
    out = np.empty(n, dtype=np.float64)
    check(_lib.lib().gr_random_vector(seed, n, 0 if dist == "uniform" else 1, lo, hi,
                                      _ptr(out)))
    return out


def _astype(self: HostMatrix, t: int) -> HostMatrix:
    """Same layout, coefficients stored as type t (gr_host_matrix_astype)."""
    h = C.c_void_p()
    check(_lib.lib().gr_host_matrix_astype(self._h, parseType(t), C.byref(h)))
    return HostMatrix(h)


def _global_crs(self: HostMatrix):
    """Global CRS with split diagonal, natural order."""
    n, m = self.numRows, self.numOffDiag
    rp = np.empty(n + 1, np.int64)
    col = np.empty(m, np.int64)
    off = np.empty(m, np.float64)
    dg = np.empty(n, np.float64)
    check(_lib.lib().gr_host_matrix_global_crs(self._h, _ptr(rp), _ptr(col), _ptr(off), _ptr(dg)))
    return rp, col, off, dg


def _coo(self: HostMatrix):
    """Global triplets (rows, cols, vals) including the diagonal."""
    rp, col, off, dg = self.globalCrs()
    n = self.numRows
    rows = np.concatenate([np.repeat(np.arange(n, dtype=np.int64), np.diff(rp)),
                           np.arange(n, dtype=np.int64)])
    return rows, np.concatenate([col, np.arange(n, dtype=np.int64)]), np.concatenate([off, dg])


HostMatrix.astype = _astype
HostMatrix.globalCrs = _global_crs
HostMatrix.coo = _coo


def loadMatrixFromFile(valueType: int, path: str, numTiles: int,
                       partitioner: int = PART_AUTO) -> HostMatrix:
    """matrix/host/HostMatrix.hpp:88-91 (MatrixMarket coordinate files)."""
    h = C.c_void_p()
    check(_lib.lib().gr_host_matrix_load_mm(str(path).encode(), numTiles, partitioner,
                                            parseType(valueType), C.byref(h)))
    return HostMatrix(h)


class Configuration:
    """Solver configuration tree (matrix/solver/Configuration.hpp:40).

    Parsed and validated by the native library at construction; the
    reference's schema is accepted (comments allowed, unknown keys ignored
    and listed in ``unknownKeys``)."""

    def __init__(self, text: str):
        self.text = text
        name = C.create_string_buffer(512)
        unk = C.create_string_buffer(1024)
        check(_lib.lib().gr_config_parse(text.encode(), name, 512, unk, 1024))
        self.solverName = name.value.decode()
        self.unknownKeys = [k for k in unk.value.decode().split(",") if k]

    @staticmethod
    def fromJSON(cfg: Union[str, dict]) -> "Configuration":
        return Configuration(cfg if isinstance(cfg, str) else _json.dumps(cfg))


class Solver:
    """Solver::createSolver(A, config) and Solver::solve(x, b)."""

    def __init__(self, A: "Matrix", config: Union[Configuration, str, dict]):
        if not isinstance(config, Configuration):
            config = Configuration.fromJSON(config)
        self.A = A
        self._s = C.c_void_p()
        check(_lib.lib().gr_solver_create(A._m, config.text.encode(), C.byref(self._s)))

    @staticmethod
    def createSolver(A: "Matrix", config) -> "Solver":
        return Solver(A, config)

    def __del__(self):
        s = getattr(self, "_s", None)
        if s and _lib is not None:
            try:
                _lib.lib().gr_solver_destroy(s)
            except Exception:
                pass
            self._s = None

    def name(self) -> str:
        buf = C.create_string_buffer(256)
        check(_lib.lib().gr_solver_name(self._s, buf, 256))
        return buf.value.decode()

    def solve(self, x, b) -> SolverStats:
        """x (in/out) and b: device tensors in tile order."""
        st = _lib.Stats()
        check(_lib.lib().gr_solve(self._s, _ptr(x), _dtype_of(x), _ptr(b), _dtype_of(b),
                                  C.byref(st)))
        return SolverStats._from(st)

    def solveHost(self, x: np.ndarray, b: np.ndarray) -> SolverStats:
        """Host arrays in natural order; copies are part of the call."""
        t = FLOAT32 if x.dtype == np.float32 else FLOAT64
        st = _lib.Stats()
        check(_lib.lib().gr_solve_host(self._s, _ptr(x), t, _ptr(b), t, C.byref(st)))
        return SolverStats._from(st)

    def timeRepeated(self, x, b, reps: int = 20) -> float:
        """Mean device ms per run of reps back-to-back runs (ILU, fixed GS)."""
        ms = C.c_float()
        check(_lib.lib().gr_solver_time_repeated(self._s, _ptr(x), _dtype_of(x), _ptr(b), _dtype_of(b), reps,
                                                 C.byref(ms)))
        return ms.value

    def refresh(self) -> None:
        """Recomputes the factors after Matrix.updateValues (gr_solver_refresh)."""
        check(_lib.lib().gr_solver_refresh(self._s))

    def phi(self, t: int = FLOAT64):
        """Extended-precision solution of the last IterativeRefinement solve."""
        torch = _torch()
        out = torch.empty(self.A.numRows, dtype=_torch_dtype(t), device=self.A.device)
        check(_lib.lib().gr_solver_phi(self._s, _ptr(out), t))
        return out


class Matrix:
    """Device matrix (matrix/Matrix.hpp:29-131)."""

    def __init__(self, host: HostMatrix):
        torch = _torch()
        self.host = host
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._m = C.c_void_p()
        check(_lib.lib().gr_matrix_create(host._h, C.byref(self._m)))

    def __del__(self):
        m = getattr(self, "_m", None)
        if m and _lib is not None:
            try:
                _lib.lib().gr_matrix_destroy(m)
            except Exception:
                pass
            self._m = None

    @property
    def numRows(self) -> int:
        return self.host.numRows

    @property
    def numTiles(self) -> int:
        return self.host.numTiles

    def createUninitializedVector(self, t: int = FLOAT32):
        torch = _torch()
        return torch.empty(self.numRows, dtype=_torch_dtype(parseType(t)), device=self.device)

    def vector(self, natural, t: int = None):
        """Device vector in tile order from a natural-order host array (type t,
        default: float64 for a float64 array, else float32)."""
        torch = _torch()
        if t is None:
            t = FLOAT64 if np.asarray(natural).dtype == np.float64 else FLOAT32
        return torch.from_numpy(self.host.decomposeVector(natural, t)).to(self.device)

    def toNatural(self, x) -> np.ndarray:
        t = _dtype_of(x)
        return self.host.composeVector(x.detach().cpu().numpy(), t)

    def __mul__(self, x):
        """Matrix::operator* -> CRSMatrix::spmv."""
        y = _torch().empty_like(x)
        check(_lib.lib().gr_spmv(self._m, _ptr(x), _ptr(y), _dtype_of(x)))
        return y

    def spmv(self, x, y) -> None:
        check(_lib.lib().gr_spmv(self._m, _ptr(x), _ptr(y), _dtype_of(x)))

    def residual(self, x, b, destType: Optional[int] = None, intermediateType: Optional[int] = None,
                 xType: Optional[int] = None):
        """Matrix::residual(x, b, destType, intermediateType)."""
        torch = _torch()
        xt = _dtype_of(x) if xType is None else xType
        if destType is None:
            destType = xt
        if intermediateType is None:
            intermediateType = destType
        r = torch.empty(self.numRows, dtype=_torch_dtype(destType), device=self.device)
        check(_lib.lib().gr_residual(self._m, _ptr(x), xt, _ptr(b), _dtype_of(b), _ptr(r),
                                     destType, intermediateType))
        return r

    def spmvLayout(self) -> dict:
        """The device SpMV layout (gr_matrix_spmv_layout)."""
        c, sl, far = C.c_int32(), C.c_int64(), C.c_int64()
        check(_lib.lib().gr_matrix_spmv_layout(self._m, C.byref(c), C.byref(sl), C.byref(far)))
        return {"compact": bool(c.value), "slots": sl.value, "far": far.value}

    def timeSpmv(self, x, y, reps: int = 20, flushL2: bool = True) -> float:
        """Mean device time in ms of y = A x (gr_matrix_time_spmv): each launch
        timed alone with CUDA events, L2 flushed before it when flushL2."""
        ms = C.c_float()
        check(_lib.lib().gr_matrix_time_spmv(self._m, _ptr(x), _ptr(y), _dtype_of(x), int(reps), int(flushL2),
                                             C.byref(ms)))
        return float(ms.value)

    def tuneSpmv(self, t: int = FLOAT32, reps: int = 5) -> dict:
        """Runs the SpMV autotuner (gr_matrix_tune_spmv) for vectors of type t."""
        v = [C.c_int32() for _ in range(3)]
        ms = C.c_float()
        check(_lib.lib().gr_matrix_tune_spmv(self._m, t, reps, *[C.byref(a) for a in v], C.byref(ms)))
        return {"block": v[0].value, "chunks_per_warp": v[1].value, "batch": v[2].value, "ms": ms.value}

    def updateValues(self, h: HostMatrix) -> None:
        """Takes h's coefficients (h has this matrix's structure); solvers on
        this matrix then need Solver.refresh() (gr_matrix_update_values)."""
        check(_lib.lib().gr_matrix_update_values(self._m, h._h))
        self.host = h

    def updateGlobalValues(self, gVal, gDiag) -> None:
        """New coefficients from global CRS values (natural order, FP64),
        gathered on the device (gr_matrix_update_global_values); solvers on
        this matrix then need Solver.refresh()."""
        gv = np.ascontiguousarray(gVal, dtype=np.float64)
        gd = np.ascontiguousarray(gDiag, dtype=np.float64)
        check(_lib.lib().gr_matrix_update_global_values(self._m, _ptr(gv), _ptr(gd)))

    def vectorNorm(self, norm: int, x) -> float:
        out = C.c_double()
        check(_lib.lib().gr_vector_norm(self._m, norm, _ptr(x), _dtype_of(x), C.byref(out)))
        return out.value

    def solve(self, x, b, config) -> SolverStats:
        """Matrix::solve(x, b, config) (matrix/Matrix.cpp:26-30)."""
        return Solver(self, config).solve(x, b)


class Server:
    """Continuous-batching solve server (gr_server_*): requests are admitted
    in arrival order as worker slots and device memory free up, run
    concurrently on separate CUDA streams, and (matrix, configuration) pairs
    stay resident for later requests."""

    def __init__(self, slots: int = 4, budgetBytes: int = 0, device: int = -1):
        cfg = _lib.ServerConfig(slots, device, budgetBytes)
        h = C.c_void_p()
        check(_lib.lib().gr_server_create(C.byref(cfg), C.byref(h)))
        self._s = h
        self._hosts = {}

    def submit(self, h: HostMatrix, config, b: np.ndarray) -> int:
        """Queues h x = b (natural order, float32 or float64), x0 = 0."""
        js = config if isinstance(config, str) else _json.dumps(config)
        bb = np.ascontiguousarray(b)
        t = FLOAT32 if bb.dtype == np.float32 else FLOAT64
        rid = C.c_uint64()
        check(_lib.lib().gr_server_submit(self._s, h._h, js.encode(), _ptr(bb), t, C.byref(rid)))
        self._hosts[rid.value] = (h, bb.dtype)
        return rid.value

    def wait(self, rid: int, timeoutMs: float = -1.0):
        """(x, SolverStats, times dict) of a finished request."""
        h, dt = self._hosts[rid]
        x = np.empty(h.numRows, dtype=dt)
        st = _lib.Stats()
        tm = _lib.RequestTimes()
        rc = _lib.lib().gr_server_wait(self._s, rid, timeoutMs, _ptr(x), C.byref(st), C.byref(tm))
        if rc != _lib.GR_ETIMEOUT:  # finished (or cancelled): the server forgot it
            self._hosts.pop(rid, None)
        check(rc)
        times = {k: getattr(tm, k) for k, _ in _lib.RequestTimes._fields_}
        return x, SolverStats._from(st), times

    def submitValues(self, like: HostMatrix, gVal: np.ndarray, gDiag: np.ndarray, config, b: np.ndarray) -> int:
        """Queues a solve of the matrix with like's structure and the global
        CRS values gVal / gDiag (gr_server_submit_values), x0 = 0."""
        js = config if isinstance(config, str) else _json.dumps(config)
        bb = np.ascontiguousarray(b)
        gv = np.ascontiguousarray(gVal, dtype=np.float64)
        gd = np.ascontiguousarray(gDiag, dtype=np.float64)
        if len(gv) != like.numOffDiag or len(gd) != like.numRows or len(bb) != like.numRows:
            raise ValueError("values, diagonal or b do not fit the template matrix")
        t = FLOAT32 if bb.dtype == np.float32 else FLOAT64
        rid = C.c_uint64()
        check(_lib.lib().gr_server_submit_values(self._s, like._h, _ptr(gv), _ptr(gd), js.encode(), _ptr(bb), t,
                                                 C.byref(rid)))
        self._hosts[rid.value] = (like, bb.dtype)
        return rid.value

    def cancel(self, rid: int) -> bool:
        """Cancels a request that has not been admitted yet (True; its wait
        then raises GrapheneError with code GR_ECANCELED); False when it is
        already running or finished."""
        c = C.c_int32()
        check(_lib.lib().gr_server_cancel(self._s, rid, C.byref(c)))
        return bool(c.value)

    def counters(self) -> dict:
        v = [C.c_int64() for _ in range(5)]
        check(_lib.lib().gr_server_counters(self._s, *[C.byref(a) for a in v]))
        return dict(zip(["queued", "running", "completed", "bytes_in_use", "resident"], [a.value for a in v]))

    def close(self):
        s = getattr(self, "_s", None)
        if s and _lib is not None:
            try:
                _lib.lib().gr_server_destroy(s)
            except Exception:
                pass
            self._s = None

    def __del__(self):
        self.close()


class Batch:
    """Many independent systems solved together (gr_batch_*): one PBiCGStab
    whose kernel launches cover all systems, each with its own device-side
    convergence test; each system's result equals its result alone."""

    def __init__(self, systems, config):
        self._hosts = list(systems)
        js = config if isinstance(config, str) else _json.dumps(config)
        arr = (C.c_void_p * len(self._hosts))(*[h._h for h in self._hosts])
        h = C.c_void_p()
        check(_lib.lib().gr_batch_create(arr, len(self._hosts), js.encode(), C.byref(h)))
        self._b = h

    def solveHost(self, bs, xs=None):
        """bs: natural-order host vectors (all float32 or all float64); x0 = 0
        unless xs is given. Returns (list of x, list of SolverStats)."""
        bs = [np.ascontiguousarray(b) for b in bs]
        dt = bs[0].dtype
        t = FLOAT32 if dt == np.float32 else FLOAT64
        xs = [np.zeros(h.numRows, dt) for h in self._hosts] if xs is None else \
            [np.array(x, dtype=dt, copy=True) for x in xs]
        xa = (C.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
        ba = (C.c_void_p * len(bs))(*[b.ctypes.data for b in bs])
        st = (_lib.Stats * len(bs))()
        check(_lib.lib().gr_batch_solve_host(self._b, xa, ba, t, st))
        return xs, [SolverStats._from(s) for s in st]

    def close(self):
        b = getattr(self, "_b", None)
        if b and _lib is not None:
            try:
                _lib.lib().gr_batch_destroy(b)
            except Exception:
                pass
            self._b = None

    def __del__(self):
        self.close()
