"""hpccg_gpu_ddot_noalloc: the dot product that allocates no device memory.

Some callers cannot let this library call cudaMalloc: their own memory
manager owns all device memory, or they may not allocate once set-up is over
(cudaMalloc can synchronise the device and can fail on a fragmented heap).
For them the library keeps the partial sums of this one dot product in a
fixed array compiled into the library.  These tests call the entry point
through the C-ABI and check it against the context-based hpccg_gpu_ddot and
the CPU oracle's ddot, twice in a row, because successive calls share that
array, and check that calls leave the device's free memory unchanged.  The
file is named to run last; it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import hpccg_b200 as hp

    lib = ctypes.CDLL(hp.LIB_PATH)
    fn = lib.hpccg_gpu_ddot_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                   ctypes.c_void_p]
    rows, cols, vals, *_ = hp.generate_matrix(3, 3, 3)
    M = hp.Matrix.from_csr(rows, cols, vals)  # context for the existing hpccg_gpu_ddot
    return torch, hp, fn, M


def _noalloc(torch, fn, dx, dy):
    torch.cuda.synchronize()
    r = ctypes.c_double(np.nan)
    rc = fn(dx.numel(), dx.data_ptr(), dy.data_ptr(), ctypes.byref(r), None)
    return rc, r.value


@pytest.mark.parametrize("n", [1, 1000, 2048, 2049, 1 << 20, 3_000_001])
def test_noalloc_matches_ctx_ddot_twice(env, n):
    torch, hp, fn, M = env
    rng = np.random.default_rng(n)
    for call in range(2):  # the second call reuses the scratch the first one left behind
        x = rng.uniform(-1, 1, n)
        y = rng.uniform(-1, 1, n)
        dx = torch.from_numpy(x).cuda()
        dy = torch.from_numpy(y).cuda()
        rc, got = _noalloc(torch, fn, dx, dy)
        assert rc == hp.HPCCG_OK
        want = M.ddot(dx, dy)
        # both are reassociated sums of the same terms: the dot-product bound of the suite
        assert abs(got - want) <= 1e-15 * np.abs(x * y).sum(), (call, got, want)
        ref = oracle.ddot(x, y)  # MPI/src/vector_operations.F90:40-71, sequential order
        assert abs(got - ref) <= 1e-15 * np.abs(x * y).sum(), (call, got, ref)


def test_noalloc_allocates_no_device_memory(env):
    """After one warm-up call (which may load the library's kernels on the device), calls with
    several sizes leave the device's free memory exactly as it was."""
    torch, hp, fn, M = env
    n_max = 3_000_001
    x = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, n_max)).cuda()
    y = torch.from_numpy(np.random.default_rng(6).uniform(-1, 1, n_max)).cuda()
    assert _noalloc(torch, fn, x, y)[0] == hp.HPCCG_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for n in (1, 777, 2048, 65537, 1 << 20, n_max):
        assert _noalloc(torch, fn, x[:n], y[:n])[0] == hp.HPCCG_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_sizes_beyond_capacity(env):
    torch, hp, fn, M = env
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    r = ctypes.c_double(0.0)
    # the size check runs on the host before any device access
    assert fn(134_217_729, d.data_ptr(), d.data_ptr(), ctypes.byref(r), None) == hp.HPCCG_ERR_TOO_LARGE
    assert fn(-1, d.data_ptr(), d.data_ptr(), ctypes.byref(r), None) == hp.HPCCG_ERR_INVALID_ARG
    assert fn(0, d.data_ptr(), d.data_ptr(), ctypes.byref(r), None) == hp.HPCCG_OK and r.value == 0.0
