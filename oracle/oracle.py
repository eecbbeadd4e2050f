"""ctypes view of the CPU oracle (oracle/hpccg_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker; the product never imports it.
Parity status: unpinned against reference outputs (see hpccg_oracle.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_libs: dict[str, ctypes.CDLL] = {}


def build() -> None:
    """Compile liboracle.so and liboracle_omp.so with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(omp: bool = False) -> ctypes.CDLL:
    name = "liboracle_omp.so" if omp else "liboracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    lib.orc_generate_matrix.restype = ctypes.c_int64
    lib.orc_generate_matrix.argtypes = [ctypes.c_int32] * 3 + [_i32p, _i32p, _f64p, _f64p, _f64p, _f64p]
    lib.orc_spmv.restype = None
    lib.orc_spmv.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p]
    lib.orc_ddot.restype = ctypes.c_double
    lib.orc_ddot.argtypes = [ctypes.c_int32, _f64p, _f64p]
    lib.orc_ddot1.restype = ctypes.c_double
    lib.orc_ddot1.argtypes = [ctypes.c_int32, _f64p]
    lib.orc_waxpby.restype = None
    lib.orc_waxpby.argtypes = [ctypes.c_int32, ctypes.c_double, _f64p, ctypes.c_double, _f64p, _f64p]
    lib.orc_wwpby.restype = None
    lib.orc_wwpby.argtypes = [ctypes.c_int32, ctypes.c_double, _f64p, _f64p]
    lib.orc_wxbw.restype = None
    lib.orc_wxbw.argtypes = [ctypes.c_int32, _f64p, ctypes.c_double, _f64p]
    lib.orc_vcopy.restype = None
    lib.orc_vcopy.argtypes = [ctypes.c_int32, _f64p, _f64p]
    lib.orc_cg.restype = ctypes.c_int
    lib.orc_cg.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p, ctypes.c_int32,
                           ctypes.c_double, ctypes.POINTER(ctypes.c_int32),
                           ctypes.POINTER(ctypes.c_double), _f64p]
    lib.orc_cg_work.restype = ctypes.c_int
    lib.orc_cg_work.argtypes = lib.orc_cg.argtypes + [_f64p]
    lib.orc_compute_residual.restype = ctypes.c_double
    lib.orc_compute_residual.argtypes = [ctypes.c_int32, _f64p, _f64p]
    lib.orc_true_relres.restype = ctypes.c_double
    lib.orc_true_relres.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p]
    lib.orc_splitmix64_at.restype = ctypes.c_uint64
    lib.orc_splitmix64_at.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    lib.orc_uniform_pm1.restype = None
    lib.orc_uniform_pm1.argtypes = [ctypes.c_uint64, ctypes.c_int64, _f64p]
    lib.orc_set_dot_mode.restype = None
    lib.orc_set_dot_mode.argtypes = [ctypes.c_int]
    lib.orc_grid_spmv.restype = None
    lib.orc_grid_spmv.argtypes = [ctypes.c_int32] * 3 + [_f64p, _f64p]
    lib.orc_cg_grid.restype = ctypes.c_int
    lib.orc_cg_grid.argtypes = [ctypes.c_int32] * 3 + [_f64p, _f64p, ctypes.c_int32, ctypes.c_double,
                                                       ctypes.POINTER(ctypes.c_int32),
                                                       ctypes.POINTER(ctypes.c_double), _f64p]
    lib.orc_grid_true_relres.restype = ctypes.c_double
    lib.orc_grid_true_relres.argtypes = [ctypes.c_int32] * 3 + [_f64p, _f64p]
    lib.orc_generate_matrix_rank.restype = ctypes.c_int64
    lib.orc_generate_matrix_rank.argtypes = [ctypes.c_int32] * 5 + [_i32p, _i32p, _f64p, _f64p, _f64p, _f64p]
    lib.orc_slab_plan_create.restype = ctypes.c_void_p
    lib.orc_slab_plan_create.argtypes = [ctypes.c_int32] * 5
    lib.orc_slab_plan_destroy.restype = None
    lib.orc_slab_plan_destroy.argtypes = [ctypes.c_void_p]
    lib.orc_slab_plan_get.restype = ctypes.c_int32
    lib.orc_slab_plan_get.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    lib.orc_cg_slabs.restype = ctypes.c_int
    lib.orc_cg_slabs.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_int32, ctypes.c_double,
                                 ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double), _f64p]
    lib.orc_batch_sizes.restype = None
    lib.orc_batch_sizes.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p]
    _libs[name] = lib
    return lib


class Matrix:
    """1-based CSR exactly as MPI/src/SparseMatrix.F90:44-64 stores it (trimmed to nnz)."""

    def __init__(self, nx: int, ny: int, nz: int, rowindex, colindex, values, nnz: int):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nrow = nx * ny * nz
        self.nnz = nnz
        self.rowindex, self.colindex, self.values = rowindex, colindex, values


def generate_matrix(nx: int, ny: int, nz: int, omp: bool = False):
    """MPI/src/SparseMatrix.F90:68-185.  Returns (A, x, b, xexact)."""
    n = nx * ny * nz
    rowindex = np.zeros(n + 1, np.int32)
    colindex = np.zeros(27 * n, np.int32)
    values = np.zeros(27 * n, np.float64)
    x = np.empty(n, np.float64)
    b = np.empty(n, np.float64)
    xexact = np.empty(n, np.float64)
    nnz = _lib(omp).orc_generate_matrix(nx, ny, nz, rowindex, colindex, values, x, b, xexact)
    A = Matrix(nx, ny, nz, rowindex, colindex[:nnz].copy(), values[:nnz].copy(), int(nnz))
    return A, x, b, xexact


def spmv(A: Matrix, x, omp: bool = False):
    y = np.empty(A.nrow, np.float64)
    _lib(omp).orc_spmv(A.nrow, A.rowindex, A.colindex, A.values, np.ascontiguousarray(x, np.float64), y)
    return y


def ddot(x, y) -> float:
    return _lib().orc_ddot(len(x), x, y)


def ddot1(x) -> float:
    return _lib().orc_ddot1(len(x), x)


def waxpby(alpha, x, beta, y):
    w = np.empty_like(x)
    _lib().orc_waxpby(len(x), alpha, x, beta, y, w)
    return w


def wwpby(beta, y, w):
    w = w.copy()
    _lib().orc_wwpby(len(w), beta, y, w)
    return w


def wxbw(x, beta, w):
    w = w.copy()
    _lib().orc_wxbw(len(w), x, beta, w)
    return w


def vcopy(x):
    y = np.empty_like(x)
    _lib().orc_vcopy(len(x), x, y)
    return y


def cg(A: Matrix, b, x0, max_iter: int, tolerance: float, omp: bool = False):
    """MPI/src/numerics.F90:41-162.  Returns (x, niters, normr, hist[0..niters])."""
    x = np.ascontiguousarray(x0, np.float64).copy()
    hist = np.zeros(max_iter + 1, np.float64)
    niters = ctypes.c_int32(0)
    normr = ctypes.c_double(0.0)
    _lib(omp).orc_cg(A.nrow, A.rowindex, A.colindex, A.values, np.ascontiguousarray(b, np.float64),
                     x, max_iter, tolerance, ctypes.byref(niters), ctypes.byref(normr), hist)
    return x, niters.value, normr.value, hist[: niters.value + 1].copy()


def grid_spmv(nx: int, ny: int, nz: int, x, omp: bool = False):
    """generate_matrix(nx,ny,nz)'s operator applied without a stored CSR; bit-identical to
    spmv() on the generated CSR (same terms, same order)."""
    y = np.empty(nx * ny * nz, np.float64)
    _lib(omp).orc_grid_spmv(nx, ny, nz, np.ascontiguousarray(x, np.float64), y)
    return y


def cg_grid(nx: int, ny: int, nz: int, b, x0, max_iter: int, tolerance: float, omp: bool = False):
    """cg() with the grid operator: same arithmetic, no host CSR.  Returns (x, niters, normr, hist)."""
    x = np.ascontiguousarray(x0, np.float64).copy()
    hist = np.zeros(max_iter + 1, np.float64)
    niters = ctypes.c_int32(0)
    normr = ctypes.c_double(0.0)
    _lib(omp).orc_cg_grid(nx, ny, nz, np.ascontiguousarray(b, np.float64), x, max_iter, tolerance,
                          ctypes.byref(niters), ctypes.byref(normr), hist)
    return x, niters.value, normr.value, hist[: niters.value + 1].copy()


def grid_true_relres(nx: int, ny: int, nz: int, b, x) -> float:
    """||b - A x|| / ||b|| with the grid operator (sequential sums, as true_relres)."""
    return _lib().orc_grid_true_relres(nx, ny, nz, np.ascontiguousarray(b, np.float64),
                                       np.ascontiguousarray(x, np.float64))


def generate_matrix_rank(nx: int, ny: int, nz: int, rank: int, nranks: int):
    """MPI/src/SparseMatrix.F90:68-185 on rank `rank` of `nranks` (z slabs of the
    nx x ny x nz*nranks grid; global 1-based columns).  Returns (A, x, b, xexact)."""
    n = nx * ny * nz
    rowindex = np.zeros(n + 1, np.int32)
    colindex = np.zeros(27 * n, np.int32)
    values = np.zeros(27 * n, np.float64)
    x, b, xexact = np.empty(n), np.empty(n), np.empty(n)
    nnz = _lib().orc_generate_matrix_rank(nx, ny, nz, rank, nranks, rowindex, colindex, values, x, b, xexact)
    A = Matrix(nx, ny, nz, rowindex, colindex[:nnz].copy(), values[:nnz].copy(), int(nnz))
    return A, x, b, xexact


HALO_MPI, HALO_GET = 0, 1


class SlabPlan:
    """Every rank's halo set-up for nranks z slabs of nx x ny x nz, simulated in one process:
    mode HALO_MPI follows MPI/src/SparseMatrix.F90:235-627 (make_local_matrix), HALO_GET
    CAF-V2/src/SparseMatrix.F90:205-331.  Indices keep the reference's 1-based convention;
    ranks are 0-based."""

    FIELDS = {"nnz": 0, "colindex": 1, "rowindex": 2, "externals": 3, "external_owners": 4, "neighbors": 5,
              "recv_length": 6, "recv_length_literal": 7, "send_length": 8, "elements_to_send": 9,
              "blocks": 10, "remote_index": 11}

    def __init__(self, nx: int, ny: int, nz: int, nranks: int, mode: int = HALO_MPI):
        self.nx, self.ny, self.nz, self.nranks, self.mode = nx, ny, nz, nranks, mode
        self.local_nrow = nx * ny * nz
        self._h = _lib().orc_slab_plan_create(nx, ny, nz, nranks, mode)

    def __del__(self):
        if getattr(self, "_h", None):
            _lib().orc_slab_plan_destroy(self._h)
            self._h = None

    def get(self, rank: int, what: str):
        code = self.FIELDS[what]
        n = _lib().orc_slab_plan_get(self._h, rank, code, None)
        if what == "nnz":
            return int(n)
        out = np.zeros(max(1, 4 * n if what == "blocks" else n), np.int32)
        _lib().orc_slab_plan_get(self._h, rank, code, out.ctypes.data)
        return out[:4 * n].reshape(n, 4) if what == "blocks" else out[:n]

    def cg(self, b, x0, max_iter: int, tolerance: float):
        """MPI/src/numerics.F90:41-162 on all ranks in step.  b, x0: the ranks' vectors one after
        another.  Returns (x, niters, normr, hist[0..niters])."""
        x = np.ascontiguousarray(x0, np.float64).copy()
        hist = np.zeros(max_iter + 1, np.float64)
        niters, normr = ctypes.c_int32(0), ctypes.c_double(0.0)
        _lib().orc_cg_slabs(self._h, np.ascontiguousarray(b, np.float64), x, max_iter, tolerance,
                            ctypes.byref(niters), ctypes.byref(normr), hist)
        return x, niters.value, normr.value, hist[: niters.value + 1].copy()


class CgWork:
    """Work arrays (r, p, Ap) for repeated timed solves: allocated once and first-touched by
    the same OpenMP static schedule the solve uses, so a timed solve neither allocates nor
    faults pages in.  `solve` is cg() on them."""

    def __init__(self, A: Matrix, omp: bool = False):
        self.A, self.omp = A, omp
        self.work = np.empty(3 * A.nrow, np.float64)
        _lib(omp).orc_vcopy(3 * A.nrow, np.zeros(3 * A.nrow), self.work)
        self.hist = np.zeros(100001, np.float64)

    def solve(self, b, x, max_iter: int, tolerance: float):
        """x (float64, contiguous) is updated in place.  Returns (niters, normr)."""
        assert max_iter < len(self.hist)
        niters = ctypes.c_int32(0)
        normr = ctypes.c_double(0.0)
        A = self.A
        _lib(self.omp).orc_cg_work(A.nrow, A.rowindex, A.colindex, A.values, b, x, max_iter, tolerance,
                                   ctypes.byref(niters), ctypes.byref(normr), self.hist, self.work)
        return niters.value, normr.value


class compensated_dots:
    """Context manager: the oracle's dot products use compensated summation inside."""

    def __init__(self, omp: bool = False):
        self.omp = omp

    def __enter__(self):
        _lib(self.omp).orc_set_dot_mode(1)
        return self

    def __exit__(self, *exc):
        _lib(self.omp).orc_set_dot_mode(0)


def compute_residual(v1, v2) -> float:
    return _lib().orc_compute_residual(len(v1), v1, v2)


def true_relres(A: Matrix, b, x) -> float:
    return _lib().orc_true_relres(A.nrow, A.rowindex, A.colindex, A.values,
                                  np.ascontiguousarray(b, np.float64), np.ascontiguousarray(x, np.float64))


def uniform_pm1(seed: int, n: int):
    out = np.empty(n, np.float64)
    _lib().orc_uniform_pm1(seed, n, out)
    return out


def splitmix64_at(seed: int, i: int) -> int:
    return int(_lib().orc_splitmix64_at(seed, i))


def batch_sizes(seed: int, nsys: int, lo: int, hi: int):
    out = np.empty(3 * nsys, np.int32)
    _lib().orc_batch_sizes(seed, nsys, lo, hi, out)
    return out.reshape(nsys, 3)
