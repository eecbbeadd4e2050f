"""Host-side checks that need no GPU: the product's host generator, the C-ABI
surface of libhpccg_b200.so, and the driver build."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from conftest import PKG, ROOT, gpu_available

import hpccg_b200 as hp

HEADER = os.path.join(ROOT, "include", "hpccg_gpu.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hpccg_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(hp.LIB_PATH)
    declared = _declared_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    nm = subprocess.run(["nm", "-D", "--defined-only", hp.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hpccg_\w+)", nm))
    assert set(declared) <= exported
    assert set(hp.exported_symbols()) <= set(declared)


def test_integration_table_names_every_entry_point():
    """The integration guide's entry-point table names every function the header
    declares: by its exact name, as a call, or through a `prefix*` group."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    table = text[text.index("## Which reference interface"):text.index("## Fortran 90 host")]
    named = set(re.findall(r"`(hpccg_\w+)[`(]", table))
    groups = set(re.findall(r"`(hpccg_\w+?)\*`", table))
    missing = [d for d in _declared_functions() if d not in named and not any(d.startswith(g) for g in groups)]
    assert not missing, missing


def test_library_is_sm100a_only():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", hp.LIB_PATH], capture_output=True,
                         text=True).stdout
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


@pytest.mark.parametrize("nx,ny,nz", [(1, 1, 1), (2, 1, 1), (1, 2, 3), (3, 5, 7), (4, 4, 4), (7, 1, 3),
                                      (16, 16, 16), (9, 2, 11), (33, 17, 5)])
def test_host_generator_bit_exact(nx, ny, nz):
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    rowindex, colindex, values, hx, hb, hxe = hp.generate_matrix(nx, ny, nz)
    assert np.array_equal(rowindex, A.rowindex)
    assert np.array_equal(colindex, A.colindex)
    assert np.array_equal(values, A.values)
    assert np.array_equal(hb, b) and np.array_equal(hx, x) and np.array_equal(hxe, xe)


def test_host_generator_rejects_bad_sizes():
    with pytest.raises(hp.HpccgError) as e:
        hp.generate_matrix(0, 4, 4)
    assert e.value.code == hp.HPCCG_ERR_INVALID_ARG


def test_strerror_names():
    assert hp.strerror(hp.HPCCG_OK) == "ok"
    assert "breakdown" in hp.strerror(hp.HPCCG_ERR_BREAKDOWN)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_cleanly():
    rowindex, colindex, values, *_ = hp.generate_matrix(3, 3, 3)
    with pytest.raises(hp.HpccgError) as e:
        hp.Matrix.from_csr(rowindex, colindex, values)
    assert e.value.code == hp.HPCCG_ERR_NO_DEVICE


def test_driver_built_and_prints_usage():
    exe = os.path.join(PKG, "HPCCG-B200")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and "USAGE" in out.stdout


@pytest.mark.parametrize("args,msg", [
    (["--batch", "random:0,8,20,7"], "bad --batch spec"),
    (["--batch", "4,4"], "bad --batch spec"),
    (["--batch", "4,4,4/5,x,5"], "bad --batch spec"),
    (["--batch", "random:3,9,8,1"], "bad --batch spec"),
    (["8", "8", "8", "--precision", "fp16"], "--precision takes fp64, fp32 or bf16"),
    (["8", "8", "8", "--rel-tol", "0"], "--rel-tol must be positive"),
    (["8", "8", "8", "--frobnicate"], "unknown option"),
    (["8", "8", "8", "--ranks", "0"], "--ranks must be positive"),
    (["8", "8", "8", "--ranks", "2", "--halo", "shmem"], "--halo takes mpi or get"),
])
def test_driver_rejects_bad_options_before_any_device_work(args, msg):
    """The driver's option errors exit with status 2 on the host (no GPU needed)."""
    exe = os.path.join(PKG, "HPCCG-B200")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    out = subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)
    assert out.returncode == 2 and msg in out.stderr, (out.returncode, out.stderr)


def test_host_generator_matches_oracle():
    """The package's host copy of the generator (workload synthesis in bench.py)
    draws the same numbers as the oracle's restatement."""
    import hpccg_b200 as hp
    import oracle

    assert np.array_equal(hp.uniform_pm1_host(1234, 1000), oracle.uniform_pm1(1234, 1000))
    assert np.array_equal(hp.uniform_pm1_host(9, 50, offset=0), oracle.uniform_pm1(9, 50))
    assert np.array_equal(hp.batch_sizes(7, 64, 16, 96).reshape(-1), np.asarray(oracle.batch_sizes(7, 64, 16, 96)).reshape(-1))


def test_fortran_interfaces_bind_exported_symbols():
    """The Fortran 90 host sources (not compiled: no Fortran compiler in this image) bind only
    names the library exports and the header declares, and the drop-in `cg` keeps the
    reference's argument list (MPI/src/numerics.F90:41-53)."""
    drv = os.path.join(os.path.dirname(hp.LIB_PATH), "driver")
    names = set()
    for f in ("hpccg_gpu.F90", "numerics_gpu.F90", "main.F90"):
        names |= set(re.findall(r'bind\(C,\s*name="(hpccg_\w+)"\)', open(os.path.join(drv, f)).read()))
    assert {"hpccg_generate_matrix", "hpccg_gpu_create", "hpccg_gpu_cg", "hpccg_gpu_destroy"} <= names
    assert names <= set(_declared_functions())
    lib = ctypes.CDLL(hp.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    src = open(os.path.join(drv, "numerics_gpu.F90")).read()
    assert re.search(r"subroutine cg\(A, b, x, max_iter, tolerance, niters, normr\)", src)
