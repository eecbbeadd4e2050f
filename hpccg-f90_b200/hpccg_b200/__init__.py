"""Python host mirror of the reference HPCCG interface over the B200 C-ABI.

Every call goes through ``libhpccg_b200.so`` (include/hpccg_gpu.h) with
ctypes; there is no CPU fallback.  If the library is missing, importing this
package raises.  Names follow the reference (MPI/src): ``generate_matrix``
(SparseMatrix.F90:68-185), ``Matrix.cg`` (numerics.F90:41-162), ``spmv``
(SparseMatrix.F90:213-232) and the BLAS-1 routines of vector_operations.F90.

Device arrays are torch CUDA tensors (torch is used for device memory only);
host arrays are numpy arrays.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(PKG_DIR), "libhpccg_b200.so")

HPCCG_OK = 0
HPCCG_ERR_INVALID_ARG = 1
HPCCG_ERR_CUDA = 2
HPCCG_ERR_OOM = 3
HPCCG_ERR_BREAKDOWN = 4
HPCCG_ERR_TIMEOUT = 5
HPCCG_ERR_NOT_CONVERGED = 6
HPCCG_ERR_UNSUPPORTED = 7
HPCCG_ERR_NO_DEVICE = 8
HPCCG_ERR_TOO_LARGE = 9

SPMV_AUTO, SPMV_ELL, SPMV_ELL2, SPMV_CSR_VECTOR, SPMV_STENCIL = 0, 1, 2, 3, 4
PREC_FP64, PREC_FP32, PREC_BF16 = 0, 1, 2


class MixedInfo(ctypes.Structure):
    """hpccg_mixed_info: refinement cycles, inner iterations, FP64 relres, status."""
    _fields_ = [("outer_iters", ctypes.c_int32), ("inner_iters", ctypes.c_int32), ("relres", ctypes.c_double),
                ("status", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class HpccgError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {strerror(code)} (code {code})")


if not os.path.exists(LIB_PATH):
    raise ImportError(f"libhpccg_b200.so not built ({LIB_PATH}); run `make -C hpccg-f90_b200`")

_lib = ctypes.CDLL(LIB_PATH)
_c = ctypes
_vp = _c.c_void_p
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = _c.c_int32
_i64 = _c.c_int64
_f64 = _c.c_double

_SIGS = {
    "hpccg_strerror": (_c.c_char_p, [_c.c_int]),
    "hpccg_generate_matrix": (_c.c_int, [_i32, _i32, _i32, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p,
                                          _c.POINTER(_i64)]),
    "hpccg_gpu_create": (_c.c_int, [_i32, _i64, _i32p, _i32p, _f64p, _c.POINTER(_vp)]),
    "hpccg_gpu_create_generated": (_c.c_int, [_i32, _i32, _i32, _vp, _vp, _vp, _c.POINTER(_vp)]),
    "hpccg_gpu_destroy": (None, [_vp]),
    "hpccg_gpu_info": (_c.c_int, [_vp, _c.POINTER(_i32), _c.POINTER(_i64), _c.POINTER(_i32)]),
    "hpccg_gpu_download_csr": (_c.c_int, [_vp, _i32p, _i32p, _f64p]),
    "hpccg_gpu_set_spmv": (_c.c_int, [_vp, _i32, _i32]),
    "hpccg_gpu_set_geometry": (_c.c_int, [_vp, _i32, _i32, _i32]),
    "hpccg_gpu_get_spmv": (_c.c_int, [_vp, _c.POINTER(_i32), _c.POINTER(_i32)]),
    "hpccg_gpu_cg": (_c.c_int, [_vp, _f64p, _f64p, _i32, _f64, _c.POINTER(_i32), _c.POINTER(_f64), _vp]),
    "hpccg_gpu_cg_device": (_c.c_int, [_vp, _vp, _vp, _i32, _f64, _c.POINTER(_i32), _c.POINTER(_f64), _vp]),
    "hpccg_gpu_spmv": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_gpu_ddot": (_c.c_int, [_vp, _i32, _vp, _vp, _c.POINTER(_f64)]),
    "hpccg_gpu_ddot1": (_c.c_int, [_vp, _i32, _vp, _c.POINTER(_f64)]),
    "hpccg_gpu_waxpby": (_c.c_int, [_vp, _i32, _f64, _vp, _f64, _vp, _vp]),
    "hpccg_gpu_wwpby": (_c.c_int, [_vp, _i32, _f64, _vp, _vp]),
    "hpccg_gpu_wxbw": (_c.c_int, [_vp, _i32, _vp, _f64, _vp]),
    "hpccg_gpu_vcopy": (_c.c_int, [_vp, _i32, _vp, _vp]),
    "hpccg_gpu_time_spmv": (_c.c_int, [_vp, _vp, _vp, _i32, _c.POINTER(_c.c_float)]),
    "hpccg_gpu_uniform_pm1": (_c.c_int, [_vp, _c.c_uint64, _i64, _i64, _vp]),
    "hpccg_gpu_last_solve_ms": (_c.c_int, [_vp, _c.POINTER(_c.c_float)]),
    "hpccg_gpu_time_cg_kernels": (_c.c_int, [_vp, _i32, _c.POINTER(_c.c_float)]),
    "hpccg_gpu_ddot_noalloc": (_c.c_int, [_i32, _vp, _vp, _c.POINTER(_f64), _vp]),
    "hpccg_batch_create_generated": (_c.c_int, [_i32, _i32p, _c.POINTER(_vp)]),
    "hpccg_batch_create": (_c.c_int, [_i32, _i32p, _vp, _vp, _vp, _c.POINTER(_vp)]),
    "hpccg_batch_destroy": (None, [_vp]),
    "hpccg_batch_info": (_c.c_int, [_vp, _c.POINTER(_i32), _c.POINTER(_i64), _vp]),
    "hpccg_batch_set_schedule": (_c.c_int, [_vp, _i32, _i32]),
    "hpccg_batch_set_spmv": (_c.c_int, [_vp, _i32]),
    "hpccg_batch_get_schedule": (_c.c_int, [_vp, _c.POINTER(_i32), _c.POINTER(_i32)]),
    "hpccg_batch_spmv": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_batch_solve": (_c.c_int, [_vp, _vp, _vp, _i32, _f64, _i32, _vp, _vp, _vp]),
    "hpccg_batch_solve_host": (_c.c_int, [_vp, _f64p, _f64p, _i32, _f64, _i32, _vp, _vp, _vp]),
    "hpccg_batch_last_solve_ms": (_c.c_int, [_vp, _c.POINTER(_c.c_float)]),
    "hpccg_unet_create": (_c.c_int, [_c.c_uint64, _c.POINTER(_vp)]),
    "hpccg_unet_destroy": (None, [_vp]),
    "hpccg_unet_num_params": (_c.c_int, [_vp, _c.POINTER(_i64)]),
    "hpccg_unet_get_params": (_c.c_int, [_vp, _vp]),
    "hpccg_unet_set_params": (_c.c_int, [_vp, _vp]),
    "hpccg_unet_forward": (_c.c_int, [_vp, _i32, _i32, _i32, _i32, _vp, _vp]),
    "hpccg_unet_loss_grad": (_c.c_int, [_vp, _i32, _i32, _i32, _i32, _vp, _vp, _c.POINTER(_c.c_float), _vp]),
    "hpccg_unet_set_loss": (_c.c_int, [_vp, _i32]),
    "hpccg_unet_adam_step": (_c.c_int, [_vp, _c.c_float, _c.c_float, _c.c_float, _c.c_float]),
    "hpccg_unet_time_forward": (_c.c_int, [_vp, _i32, _i32, _i32, _i32, _vp, _vp, _c.POINTER(_c.c_float)]),
    "hpccg_unet_conv3_layer": (_c.c_int, [_i32, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _vp]),
    "hpccg_gpu_solve_mixed": (_c.c_int, [_vp, _f64p, _f64p, _i32, _f64, _i32, _i32, _f64, _vp]),
    "hpccg_gpu_solve_mixed_device": (_c.c_int, [_vp, _vp, _vp, _i32, _f64, _i32, _i32, _f64, _vp]),
    "hpccg_gpu_spmv_lowp": (_c.c_int, [_vp, _i32, _vp, _vp]),
    "hpccg_gpu_set_mixed_rows_per_thread": (_c.c_int, [_vp, _i32, _i32]),
    "hpccg_gpu_time_mixed_kernels": (_c.c_int, [_vp, _i32, _i32, _c.POINTER(_c.c_float)]),
    "hpccg_gpu_set_mixed_fused": (_c.c_int, [_vp, _i32]),
    "hpccg_gpu_mixed_fused": (_c.c_int, [_vp, _c.POINTER(_i32)]),
    "hpccg_gpu_mixed_pass": (_c.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _c.c_double, _c.c_double, _i32,
                                        _c.POINTER(_c.c_double)]),
    "hpccg_generate_matrix_rank": (_c.c_int, [_i32, _i32, _i32, _i32, _i32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                              _f64p, _c.POINTER(_i64)]),
    "hpccg_slab_plan_create": (_c.c_int, [_i32, _i64, _i32p, _i32p, _i32, _i32, _i32p, _i32, _c.POINTER(_vp)]),
    "hpccg_slab_plan_destroy": (None, [_vp]),
    "hpccg_slab_plan_info": (_c.c_int, [_vp, _c.POINTER(_i32), _c.POINTER(_i32), _c.POINTER(_i32),
                                        _c.POINTER(_i32)]),
    "hpccg_slab_plan_neighbors": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_plan_externals": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_plan_set_sends": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_plan_sends": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_plan_colindex": (_c.c_int, [_vp, _vp]),
    "hpccg_slab_plan_blocks": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_create": (_c.c_int, [_vp, _f64p, _c.POINTER(_vp)]),
    "hpccg_slab_destroy": (None, [_vp]),
    "hpccg_slab_info": (_c.c_int, [_vp, _c.POINTER(_i32), _c.POINTER(_i32), _c.POINTER(_i32), _c.POINTER(_i32)]),
    "hpccg_slab_spmv": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_pack": (_c.c_int, [_vp, _vp, _vp]),
    "hpccg_slab_scatter_block": (_c.c_int, [_vp, _i32, _vp, _vp]),
    "hpccg_slab_cg_step": (_c.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpccg_slab_group_cg": (_c.c_int, [_vp, _i32, _vp, _vp, _i32, _f64, _c.POINTER(_i32), _c.POINTER(_f64), _vp]),
}
for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(_lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def strerror(code: int) -> str:
    return _lib.hpccg_strerror(code).decode()


def _check(rc: int, what: str, allow=(HPCCG_OK,)) -> int:
    if rc not in allow:
        raise HpccgError(rc, what)
    return rc


def exported_symbols() -> list[str]:
    """Names of the C-ABI entry points this binding resolved from the library."""
    return sorted(_SIGS)


def splitmix64_at(seed: int, i) -> np.ndarray:
    """The project's counter-based generator (splitmix64 finaliser of seed + (i+1)*golden),
    the same sequence hpccg_gpu_uniform_pm1 draws on the device; i is an index array."""
    i = np.asarray(i, np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (i + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform_pm1_host(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n doubles in [-1, 1) from the generator (host copy of hpccg_gpu_uniform_pm1)."""
    u = (splitmix64_at(seed, np.arange(offset, offset + n, dtype=np.uint64)) >> np.uint64(11)).astype(np.float64)
    return 2.0 * (u * 2.0 ** -53) - 1.0


def batch_sizes(seed: int, nsys: int, lo: int, hi: int) -> np.ndarray:
    """Grid sizes of a batch workload: (nx, ny, nz) per system, each uniform in [lo, hi]."""
    z = splitmix64_at(seed, np.arange(3 * nsys, dtype=np.uint64)) % np.uint64(hi - lo + 1)
    return (lo + z.astype(np.int64)).astype(np.int32).reshape(nsys, 3)


def _dptr(t) -> int:
    """Device pointer of a torch CUDA tensor (contiguous float64 expected)."""
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return t.data_ptr()


def _sync_torch():
    import torch

    torch.cuda.synchronize()


def ddot_noalloc(d_x, d_y, stream=None) -> float:
    """x.y through hpccg_gpu_ddot_noalloc: no context and no device allocation
    (partial sums in a fixed array inside the library; n <= 134,217,728)."""
    _sync_torch()
    r = _f64(0.0)
    _check(_lib.hpccg_gpu_ddot_noalloc(d_x.numel(), _dptr(d_x), _dptr(d_y), _c.byref(r), stream),
           "ddot_noalloc")
    return r.value


# ---- host generator ------------------------------------------------------------

def generate_matrix(nx: int, ny: int, nz: int):
    """SparseMatrix.F90:68-185 on the host.  Returns (rowindex, colindex, values, x, b, xexact),
    1-based int32 indices exactly as the reference stores them (colindex/values trimmed to nnz)."""
    n = nx * ny * nz
    rowindex = np.empty(n + 1, np.int32)
    colindex = np.empty(27 * n, np.int32)
    values = np.empty(27 * n, np.float64)
    x = np.empty(n, np.float64)
    b = np.empty(n, np.float64)
    xexact = np.empty(n, np.float64)
    nnz = _i64(0)
    _check(_lib.hpccg_generate_matrix(nx, ny, nz, rowindex, colindex, values, x, b, xexact, _c.byref(nnz)),
           "generate_matrix")
    k = nnz.value
    return rowindex, colindex[:k].copy(), values[:k].copy(), x, b, xexact


class Matrix:
    """A matrix resident on the GPU (the SparseMatrixT of the reference)."""

    def __init__(self, handle: int):
        self._h = _vp(handle)
        nr, nnz, w = _i32(0), _i64(0), _i32(0)
        _check(_lib.hpccg_gpu_info(self._h, _c.byref(nr), _c.byref(nnz), _c.byref(w)), "info")
        self.nrow, self.nnz, self.ell_width = nr.value, nnz.value, w.value

    # -- construction --
    @classmethod
    def from_csr(cls, rowindex, colindex, values) -> "Matrix":
        rowindex = np.ascontiguousarray(rowindex, np.int32)
        colindex = np.ascontiguousarray(colindex, np.int32)
        values = np.ascontiguousarray(values, np.float64)
        h = _vp()
        _check(_lib.hpccg_gpu_create(len(rowindex) - 1, len(colindex), rowindex, colindex, values,
                                     _c.byref(h)), "create")
        return cls(h.value)

    @classmethod
    def generated(cls, nx: int, ny: int, nz: int, d_x=None, d_b=None, d_xexact=None) -> "Matrix":
        h = _vp()
        ptr = lambda t: None if t is None else _dptr(t)  # noqa: E731
        if d_x is not None or d_b is not None or d_xexact is not None:
            _sync_torch()
        _check(_lib.hpccg_gpu_create_generated(nx, ny, nz, ptr(d_x), ptr(d_b), ptr(d_xexact), _c.byref(h)),
               "create_generated")
        return cls(h.value)

    def close(self):
        if self._h:
            _lib.hpccg_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def download_csr(self):
        rowindex = np.empty(self.nrow + 1, np.int32)
        colindex = np.empty(self.nnz, np.int32)
        values = np.empty(self.nnz, np.float64)
        _check(_lib.hpccg_gpu_download_csr(self._h, rowindex, colindex, values), "download_csr")
        return rowindex, colindex, values

    # -- kernel selection --
    def set_geometry(self, nx: int, ny: int, nz: int):
        """Check on the device that A is generate_matrix(nx,ny,nz); enables SPMV_STENCIL.
        Raises HpccgError (HPCCG_ERR_UNSUPPORTED) when the matrix differs."""
        _check(_lib.hpccg_gpu_set_geometry(self._h, nx, ny, nz), "set_geometry")

    def set_spmv(self, kind: int, param: int = 0):
        _check(_lib.hpccg_gpu_set_spmv(self._h, kind, param), "set_spmv")

    def get_spmv(self):
        k, p = _i32(0), _i32(0)
        _check(_lib.hpccg_gpu_get_spmv(self._h, _c.byref(k), _c.byref(p)), "get_spmv")
        return k.value, p.value

    # -- the CG entry point (numerics.F90:41-162) --
    def cg(self, b, x, max_iter: int = 150, tolerance: float = 0.0, history: bool = True):
        """Host arrays.  Returns (x, niters, normr, hist, status); x is updated in place."""
        b = np.ascontiguousarray(b, np.float64)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise ValueError("x must be a contiguous float64 numpy array (updated in place)")
        hist = np.zeros(max_iter + 1, np.float64)
        niters, normr = _i32(0), _f64(0.0)
        rc = _lib.hpccg_gpu_cg(self._h, b, x, max_iter, tolerance, _c.byref(niters), _c.byref(normr),
                               hist.ctypes.data if history else None)
        _check(rc, "cg", allow=(HPCCG_OK, HPCCG_ERR_BREAKDOWN))
        return x, niters.value, normr.value, hist[: niters.value + 1], rc

    def cg_device(self, d_b, d_x, max_iter: int = 150, tolerance: float = 0.0, history: bool = True):
        """Device arrays (torch CUDA float64).  Returns (niters, normr, hist, status)."""
        _sync_torch()
        hist = np.zeros(max_iter + 1, np.float64)
        niters, normr = _i32(0), _f64(0.0)
        rc = _lib.hpccg_gpu_cg_device(self._h, _dptr(d_b), _dptr(d_x), max_iter, tolerance,
                                      _c.byref(niters), _c.byref(normr), hist.ctypes.data if history else None)
        _check(rc, "cg_device", allow=(HPCCG_OK, HPCCG_ERR_BREAKDOWN))
        return niters.value, normr.value, hist[: niters.value + 1], rc

    # -- op-level drop-ins on device tensors --
    def spmv(self, d_x, d_y):
        _sync_torch()
        _check(_lib.hpccg_gpu_spmv(self._h, _dptr(d_x), _dptr(d_y)), "spmv")

    def ddot(self, d_x, d_y) -> float:
        _sync_torch()
        r = _f64(0.0)
        _check(_lib.hpccg_gpu_ddot(self._h, d_x.numel(), _dptr(d_x), _dptr(d_y), _c.byref(r)), "ddot")
        return r.value

    def ddot1(self, d_x) -> float:
        _sync_torch()
        r = _f64(0.0)
        _check(_lib.hpccg_gpu_ddot1(self._h, d_x.numel(), _dptr(d_x), _c.byref(r)), "ddot1")
        return r.value

    def waxpby(self, alpha, d_x, beta, d_y, d_w):
        _sync_torch()
        _check(_lib.hpccg_gpu_waxpby(self._h, d_x.numel(), alpha, _dptr(d_x), beta, _dptr(d_y), _dptr(d_w)),
               "waxpby")

    def wwpby(self, beta, d_y, d_w):
        _sync_torch()
        _check(_lib.hpccg_gpu_wwpby(self._h, d_w.numel(), beta, _dptr(d_y), _dptr(d_w)), "wwpby")

    def wxbw(self, d_x, beta, d_w):
        _sync_torch()
        _check(_lib.hpccg_gpu_wxbw(self._h, d_w.numel(), _dptr(d_x), beta, _dptr(d_w)), "wxbw")

    def vcopy(self, d_x, d_y):
        _sync_torch()
        _check(_lib.hpccg_gpu_vcopy(self._h, d_x.numel(), _dptr(d_x), _dptr(d_y)), "vcopy")

    # -- mixed precision (FP64 iterative refinement, low-precision inner CG) --
    def solve_mixed(self, b, x, precision: int, rel_tol: float = 1e-8, max_outer: int = 20,
                    max_inner: int = 1000, inner_rtol: float = 0.0):
        """Host arrays.  Returns (x, MixedInfo, status); x is updated in place."""
        b = np.ascontiguousarray(b, np.float64)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise ValueError("x must be a contiguous float64 numpy array (updated in place)")
        info = MixedInfo()
        rc = _lib.hpccg_gpu_solve_mixed(self._h, b, x, precision, rel_tol, max_outer, max_inner, inner_rtol,
                                        ctypes.byref(info))
        _check(rc, "solve_mixed", allow=(HPCCG_OK, HPCCG_ERR_NOT_CONVERGED, HPCCG_ERR_BREAKDOWN))
        return x, info, rc

    def solve_mixed_device(self, d_b, d_x, precision: int, rel_tol: float = 1e-8, max_outer: int = 20,
                           max_inner: int = 1000, inner_rtol: float = 0.0):
        _sync_torch()
        info = MixedInfo()
        rc = _lib.hpccg_gpu_solve_mixed_device(self._h, _dptr(d_b), _dptr(d_x), precision, rel_tol, max_outer,
                                               max_inner, inner_rtol, ctypes.byref(info))
        _check(rc, "solve_mixed_device", allow=(HPCCG_OK, HPCCG_ERR_NOT_CONVERGED, HPCCG_ERR_BREAKDOWN))
        return info, rc

    def spmv_lowp(self, precision: int, d_x, d_y):
        _sync_torch()
        _check(_lib.hpccg_gpu_spmv_lowp(self._h, precision, _dptr(d_x), _dptr(d_y)), "spmv_lowp")

    def set_mixed_rows_per_thread(self, precision: int, rpt: int):
        _check(_lib.hpccg_gpu_set_mixed_rows_per_thread(self._h, precision, rpt), "set_mixed_rows_per_thread")

    def time_mixed_kernels(self, precision: int, reps: int = 10):
        """[p update, SpMV + p.Ap, r update] ms; [FP64 residual, pass, 0] with the fused iteration."""
        ms = (_c.c_float * 3)()
        _check(_lib.hpccg_gpu_time_mixed_kernels(self._h, precision, reps, ms), "time_mixed_kernels")
        return [ms[0], ms[1], ms[2]]

    def set_mixed_fused(self, on: bool):
        """Select the one-pass fused inner iteration (default) or the three-kernel one."""
        _check(_lib.hpccg_gpu_set_mixed_fused(self._h, 1 if on else 0), "set_mixed_fused")

    def mixed_fused(self) -> bool:
        f = _i32(0)
        _check(_lib.hpccg_gpu_mixed_fused(self._h, _c.byref(f)), "mixed_fused")
        return bool(f.value)

    def mixed_pass(self, d_r, d_p, d_d, d_r_out, d_p_out, alpha: float, beta: float, first: bool):
        """One fused inner-CG pass on FP32 device vectors; returns (p'.Ap', r'.Ap', Ap'.Ap', r'.r')."""
        _sync_torch()
        dots = (_c.c_double * 4)()
        _check(_lib.hpccg_gpu_mixed_pass(self._h, _dptr(d_r), _dptr(d_p), _dptr(d_d), _dptr(d_r_out),
                                         _dptr(d_p_out), alpha, beta, 1 if first else 0, dots), "mixed_pass")
        return tuple(dots)

    def uniform_pm1(self, seed: int, d_out, offset: int = 0):
        """Fill a device tensor with the project's counter-based U[-1,1) stream."""
        _sync_torch()
        _check(_lib.hpccg_gpu_uniform_pm1(self._h, seed, offset, d_out.numel(), _dptr(d_out)), "uniform_pm1")

    def last_solve_ms(self) -> float:
        ms = _c.c_float(0.0)
        _check(_lib.hpccg_gpu_last_solve_ms(self._h, _c.byref(ms)), "last_solve_ms")
        return ms.value

    def time_cg_kernels(self, reps: int = 10):
        """Average ms of (p/x update, SpMV+p.Ap, r update+r.r) launched back to back."""
        ms = (_c.c_float * 3)()
        _check(_lib.hpccg_gpu_time_cg_kernels(self._h, reps, ms), "time_cg_kernels")
        return [ms[0], ms[1], ms[2]]

    def time_spmv(self, d_x, d_y, reps: int = 10) -> float:
        _sync_torch()
        ms = _c.c_float(0.0)
        _check(_lib.hpccg_gpu_time_spmv(self._h, _dptr(d_x), _dptr(d_y), reps, _c.byref(ms)), "time_spmv")
        return ms.value


class Batch:
    """Many independent systems solved together (hpccg_batch_* in the C-ABI).

    Vectors are "stacked": system s occupies rows offsets[s] .. offsets[s]+nrows[s]
    of one device vector of length stacked_rows (gaps between systems are zero)."""

    def __init__(self, handle):
        self._h = _vp(handle)
        ns, rows = _i32(0), _i64(0)
        _check(_lib.hpccg_batch_info(self._h, _c.byref(ns), _c.byref(rows), None), "batch_info")
        self.nsys, self.stacked_rows = ns.value, rows.value
        offs = np.zeros(2 * self.nsys, np.int64)
        _check(_lib.hpccg_batch_info(self._h, None, None, offs.ctypes.data), "batch_info")
        self.offsets, self.nrows = offs[0::2].copy(), offs[1::2].copy()

    @classmethod
    def generated(cls, sizes) -> "Batch":
        sizes = np.ascontiguousarray(np.asarray(sizes, np.int32).reshape(-1))
        h = _vp()
        _check(_lib.hpccg_batch_create_generated(len(sizes) // 3, sizes, _c.byref(h)), "batch_create_generated")
        return cls(h.value)

    @classmethod
    def from_csr(cls, systems) -> "Batch":
        """systems: list of (rowindex, colindex, values) in the reference's 1-based layout."""
        rows = [np.ascontiguousarray(r, np.int32) for r, _, _ in systems]
        cols = [np.ascontiguousarray(c, np.int32) for _, c, _ in systems]
        vals = [np.ascontiguousarray(v, np.float64) for _, _, v in systems]
        n = len(systems)
        nrows = np.array([len(r) - 1 for r in rows], np.int32)
        P = _vp * n
        h = _vp()
        _check(_lib.hpccg_batch_create(n, nrows, P(*[r.ctypes.data for r in rows]), P(*[c.ctypes.data for c in cols]),
                                       P(*[v.ctypes.data for v in vals]), _c.byref(h)), "batch_create")
        return cls(h.value)

    def close(self):
        if self._h:
            _lib.hpccg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stack(self, vectors):
        out = np.zeros(self.stacked_rows, np.float64)
        for s, v in enumerate(vectors):
            out[self.offsets[s]:self.offsets[s] + self.nrows[s]] = v
        return out

    def unstack(self, stacked):
        return [np.asarray(stacked[self.offsets[s]:self.offsets[s] + self.nrows[s]]) for s in range(self.nsys)]

    def set_schedule(self, tile_chunks: int, blocks_per_sm: int):
        _check(_lib.hpccg_batch_set_schedule(self._h, tile_chunks, blocks_per_sm), "batch_set_schedule")

    def set_spmv(self, kind: int):
        """SPMV_ELL (stacked matrix) or SPMV_STENCIL (matrix-free; generated batches only)."""
        _check(_lib.hpccg_batch_set_spmv(self._h, kind), "batch_set_spmv")

    def get_schedule(self):
        t, b = _i32(0), _i32(0)
        _check(_lib.hpccg_batch_get_schedule(self._h, _c.byref(t), _c.byref(b)), "batch_get_schedule")
        return t.value, b.value

    def spmv(self, d_x, d_y):
        _sync_torch()
        _check(_lib.hpccg_batch_spmv(self._h, _dptr(d_x), _dptr(d_y)), "batch_spmv")

    def solve(self, d_b, d_x, precision: int = PREC_FP64, rel_tol: float = 1e-8, max_iter: int = 1000):
        """Stacked device vectors.  Returns (iters, relres, outer, status) per system."""
        _sync_torch()
        iters = np.zeros(self.nsys, np.int32)
        relres = np.zeros(self.nsys, np.float64)
        outer = np.zeros(self.nsys, np.int32)
        rc = _lib.hpccg_batch_solve(self._h, _dptr(d_b), _dptr(d_x), precision, rel_tol, max_iter,
                                    iters.ctypes.data, relres.ctypes.data, outer.ctypes.data)
        _check(rc, "batch_solve", allow=(HPCCG_OK, HPCCG_ERR_NOT_CONVERGED, HPCCG_ERR_BREAKDOWN))
        return iters, relres, outer, rc

    def solve_host(self, b, x, precision: int = PREC_FP64, rel_tol: float = 1e-8, max_iter: int = 1000):
        """Stacked HOST arrays (float64, length stacked_rows); x is updated in place.
        Returns (iters, relres, outer, status) per system."""
        b = np.ascontiguousarray(b, np.float64)
        if x.dtype != np.float64 or not x.flags.c_contiguous or b.shape != x.shape or b.size != self.stacked_rows:
            raise ValueError("b and x must be contiguous float64 arrays of the stacked length")
        iters = np.zeros(self.nsys, np.int32)
        relres = np.zeros(self.nsys, np.float64)
        outer = np.zeros(self.nsys, np.int32)
        rc = _lib.hpccg_batch_solve_host(self._h, b, x, precision, rel_tol, max_iter, iters.ctypes.data,
                                         relres.ctypes.data, outer.ctypes.data)
        _check(rc, "batch_solve_host", allow=(HPCCG_OK, HPCCG_ERR_NOT_CONVERGED, HPCCG_ERR_BREAKDOWN))
        return iters, relres, outer, rc

    def last_solve_ms(self) -> float:
        ms = _c.c_float(0.0)
        _check(_lib.hpccg_batch_last_solve_ms(self._h, _c.byref(ms)), "batch_last_solve_ms")
        return ms.value


def conv3_layer(d_in0, d_in1, d_w, d_bias, d_proj, epi: int, path: int, d_out, nx, ny, nz, nb=1, nin=None):
    """One 3x3x3 conv with 16 outputs (test entry): torch device tensors, BF16 inputs;
    nin = 0: the 1-channel input layer on an FP32 grid."""
    _sync_torch()
    if nin is None:
        nin = 1 if d_in1 is None else 2
    p = lambda t: None if t is None else _dptr(t)  # noqa: E731
    _check(_lib.hpccg_unet_conv3_layer(nx, ny, nz, nb, nin, p(d_in0), p(d_in1), p(d_w), p(d_bias), p(d_proj), epi,
                                       path, p(d_out)), "conv3_layer")


class Unet:
    """The learned preconditioner network (hpccg_unet_* in the C-ABI)."""

    def __init__(self, seed: int = 1):
        h = _vp()
        _check(_lib.hpccg_unet_create(seed, _c.byref(h)), "unet_create")
        self._h = h
        n = _i64(0)
        _check(_lib.hpccg_unet_num_params(self._h, _c.byref(n)), "unet_num_params")
        self.nparams = n.value

    def close(self):
        if self._h:
            _lib.hpccg_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def get_params(self):
        out = np.empty(self.nparams, np.float32)
        _check(_lib.hpccg_unet_get_params(self._h, out.ctypes.data), "unet_get_params")
        return out

    def set_params(self, params):
        params = np.ascontiguousarray(params, np.float32)
        assert params.size == self.nparams
        _check(_lib.hpccg_unet_set_params(self._h, params.ctypes.data), "unet_set_params")

    def forward(self, d_in, d_out, nx, ny, nz, nb=1):
        _sync_torch()
        _check(_lib.hpccg_unet_forward(self._h, nx, ny, nz, nb, _dptr(d_in), _dptr(d_out)), "unet_forward")

    def loss_grad(self, d_in, d_target, nx, ny, nz, nb=1, want_grad=False):
        _sync_torch()
        loss = _c.c_float(0.0)
        g = np.empty(self.nparams, np.float32) if want_grad else None
        _check(_lib.hpccg_unet_loss_grad(self._h, nx, ny, nz, nb, _dptr(d_in), _dptr(d_target), _c.byref(loss),
                                         g.ctypes.data if want_grad else None), "unet_loss_grad")
        return (loss.value, g) if want_grad else loss.value

    def set_loss(self, kind: int):
        """0 = mean squared error, 1 = energy norm of the HPCCG operator."""
        _check(_lib.hpccg_unet_set_loss(self._h, kind), "unet_set_loss")

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        _check(_lib.hpccg_unet_adam_step(self._h, lr, beta1, beta2, eps), "unet_adam_step")

    def time_forward(self, d_in, d_out, nx, ny, nz, reps=10) -> float:
        _sync_torch()
        ms = _c.c_float(0.0)
        _check(_lib.hpccg_unet_time_forward(self._h, nx, ny, nz, reps, _dptr(d_in), _dptr(d_out), _c.byref(ms)),
               "unet_time_forward")
        return ms.value
