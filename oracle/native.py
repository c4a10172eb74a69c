"""Multi-threaded C Krylov solves for the CPU oracle (test and baseline
infrastructure only).

``oracle/krylov.c`` restates the same CG and BiCGStab as
``oracle/solvers.py`` (reference ``solvers/cg.py:237-336``,
``solvers/bicgstab.py:76-272``) with OpenMP loops over rows and fixed-chunk
reductions.  ``enable()`` routes ``oracle.solvers.solve`` through it, so a
multi-million-cell oracle run uses every host core; the arithmetic differs
from the numpy path only in the order of the row and dot-product sums.
``build()`` compiles the library with gcc into ``oracle/_build``.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
import weakref

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "krylov.c"
LIB = HERE / "_build" / "liboracle_krylov.so"

_lib = None


def build(force: bool = False) -> pathlib.Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(tmp), "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        P = ctypes.c_void_p
        lib.oracle_cg.argtypes = [ctypes.c_int64, P, P, P, P, P, P, P, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_int, P]
        lib.oracle_bicgstab.argtypes = [ctypes.c_int64, P, P, P, P, P, P, P, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        lib.oracle_cg.restype = ctypes.c_int
        lib.oracle_bicgstab.restype = ctypes.c_int
        lib.oracle_num_threads.restype = ctypes.c_int
        lib.oracle_segment_sum.argtypes = [ctypes.c_int64, P, P, ctypes.c_int64, P, P]
        lib.oracle_segment_sum.restype = None
        _lib = lib
    return _lib


def num_threads() -> int:
    return int(load().oracle_num_threads())


class RowPattern:
    """Rows of the off-diagonal LDU entries of a case (built once per mesh):
    row ``c`` holds ``upper[f] x[neighbour[f]]`` for faces it owns and
    ``lower[f] x[owner[f]]`` for faces where it is the neighbour."""

    def __init__(self, case):
        n, F = case.num_cells, case.num_internal_faces
        rows = np.concatenate([case.owner, case.neighbour])
        cols = np.concatenate([case.neighbour, case.owner]).astype(np.int32)
        order = np.argsort(rows, kind="stable")
        self.col = np.ascontiguousarray(cols[order])
        self.src = order.astype(np.int64)
        self.rowptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=self.rowptr[1:])
        self.F = F

    def coefficients(self, A) -> np.ndarray:
        return np.ascontiguousarray(np.concatenate([A.upper, A.lower])[self.src])


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def solve(A, rhs: np.ndarray, x0: np.ndarray, cfg: dict):
    """Drop-in for ``oracle.solvers.solve`` (krylov.py:34-82 plus the
    CG/BiCGStab dispatch of solvers/factory.py)."""
    from oracle.solvers import SolveStats, jacobi_inv_diag

    case = A.case
    pat = getattr(case, "_row_pattern", None)
    if pat is None:
        pat = RowPattern(case)
        case._row_pattern = pat
    coef = pat.coefficients(A)
    diag = np.ascontiguousarray(A.diag, dtype=np.float64)
    inv = jacobi_inv_diag(A, cfg["preconditioner"])
    inv = None if inv is None else np.ascontiguousarray(inv)
    lib = load()
    method = cfg["method"]
    cols = [rhs] if rhs.ndim == 1 else [rhs[:, k] for k in range(rhs.shape[1])]
    x0s = [x0] if rhs.ndim == 1 else [x0[:, k] for k in range(rhs.shape[1])]
    outs, stats = [], []
    for b, x in zip(cols, x0s):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x, dtype=np.float64, copy=True)
        st = np.zeros(4)
        args = [case.num_cells, _p(pat.rowptr), _p(pat.col), _p(coef), _p(diag), _p(b), _p(x),
                None if inv is None else _p(inv), float(cfg["tolerance"]), float(cfg["rel_tolerance"]),
                int(cfg["norm_type"] == "l_inf"), int(cfg["max_iter"])]
        if method == "cg":
            rc = lib.oracle_cg(*args, _p(st))
        elif method == "bicgstab":
            rc = lib.oracle_bicgstab(*args, int(cfg["max_restart"]), _p(st))
        else:
            raise ValueError(method)
        if rc != 0:
            raise MemoryError("oracle Krylov solve could not allocate its vectors")
        outs.append(x)
        stats.append(SolveStats(method, float(st[0]), float(st[1]), int(st[2]), bool(st[3])))
    if rhs.ndim == 1:
        return outs[0], (stats[0],)
    return np.stack(outs, axis=1), tuple(stats)


class _Segments:
    """Stable-sorted rows of one index array (kept while the array lives)."""

    def __init__(self, index: np.ndarray, n: int):
        self.ref = weakref.ref(index)
        self.n = n
        self.perm = np.argsort(index, kind="stable").astype(np.int64)
        self.rowptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(index, minlength=n)[:n], out=self.rowptr[1:])


_SEGMENTS: dict[int, _Segments] = {}
_SEEN: dict[int, weakref.ref] = {}
_SMALL = 1 << 12


def scatter_add(n: int, index: np.ndarray, values: np.ndarray, numpy_path) -> np.ndarray:
    """``oracle.case.scatter_add`` on every core for index arrays that are
    used repeatedly (case topology); one-off and small ones take numpy."""
    values = np.asarray(values, dtype=np.float64)
    m = index.shape[0]
    if m < _SMALL or index.ndim != 1 or values.shape[0] != m:
        return numpy_path(n, index, values)
    key = id(index)
    seg = _SEGMENTS.get(key)
    if seg is None or seg.ref() is not index or seg.n != n:
        seen = _SEEN.get(key)
        if seen is None or seen() is not index:
            _SEEN[key] = weakref.ref(index)
            return numpy_path(n, index, values)
        if index.min(initial=0) < 0 or index.max(initial=0) >= n:
            return numpy_path(n, index, values)
        seg = _Segments(index, n)
        _SEGMENTS[key] = seg
    flat = np.ascontiguousarray(values.reshape(m, -1))
    out = np.empty((n, flat.shape[1]))
    load().oracle_segment_sum(n, _p(seg.rowptr), _p(seg.perm), flat.shape[1], _p(flat), _p(out))
    return out.reshape((n,) + values.shape[1:])


def enable() -> None:
    """Route the oracle's Krylov solves and repeated scatter-adds through
    the C library."""
    import oracle.case as case
    import oracle.solvers as solvers

    load()
    solvers._NATIVE = solve
    case._NATIVE_SCATTER = scatter_add


def disable() -> None:
    import oracle.case as case
    import oracle.solvers as solvers

    solvers._NATIVE = None
    case._NATIVE_SCATTER = None
