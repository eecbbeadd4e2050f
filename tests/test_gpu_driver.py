"""The C++ host driver (HPCCG-B200), the reference's main.F90 over the C-ABI.

Checks the report against the reference's formats (MPI/src/main.F90:33-75,
numerics.F90:103-156): printInfo lines with total_nnz = 27 N, the initial
residual, the ITER lines at print_freq = clamp(max_iter/10, 1, 50) and at
k + 1 = max_iter in e20.10, the TIMER lines of each timing level and
MFLOPS SPARSEMV; the printed residuals equal the oracle's history to the 10
digits printed; the matrix-free SpMV prints the identical history.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from conftest import PKG

pytestmark = pytest.mark.gpu

EXE = os.path.join(PKG, "HPCCG-B200")


def _run(*args):
    if not os.path.exists(EXE):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    out = subprocess.run([EXE, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return out.stdout


def _iters(text):
    return {int(m.group(1)): float(m.group(2)) for m in re.finditer(r"^ITER\s*(\d+)\s+Residual\s+(\S+)$", text, re.M)}


def test_driver_report_matches_reference_format_and_oracle():
    n = 32
    A, x, b, xe = oracle.generate_matrix(n, n, n)
    _, it, normr, hist = oracle.cg(A, b, x, 150, 0.0)
    out = _run(n, n, n, "--timing-level", 3)
    assert re.search(r"^ HPCCG Benchmark$", out, re.M)
    assert re.search(r"Total size \(N x N\):\s+32768$", out, re.M)
    assert re.search(r"Total nonzeroes:\s+884736$", out, re.M)  # the reference's 27 N
    r0 = float(re.search(r"Initial Residual =\s+(\S+)", out).group(1))
    assert r0 == pytest.approx(hist[0], rel=1e-14)
    got = _iters(out)
    assert sorted(got) == sorted(set(range(15, 151, 15)) | {149})
    for k, v in got.items():
        assert re.search(r"^ITER%5d  Residual\s+-?0\.\d{10}E[+-]\d\d$" % k, out, re.M)
        assert v == pytest.approx(hist[k], rel=1e-9, abs=1e-12 * hist[0])
    assert len(re.findall(r"^ TIMER: Iteration\s+\S+ sec$", out, re.M)) == 150
    assert re.search(r"^ TIMER: Total\s+\S+ sec$", out, re.M)
    mflops = float(re.search(r"MFLOPS SPARSEMV\s+(\S+)", out).group(1))
    assert mflops > 0
    # default level 1: only the Total timer
    out1 = _run(n, n, n)
    assert "TIMER: Total" in out1 and "TIMER: Iteration" not in out1 and "MFLOPS" not in out1


def test_driver_stencil_prints_identical_history():
    """Host CSR + matrix-free SpMV and device-generated + matrix-free print the
    same digits; against the stored-matrix run (no grid declared, so its dot
    products associate differently) they agree to the printed precision."""
    base = _run(17, 9, 6, "--max-iter", 60)
    st = _run(17, 9, 6, "--max-iter", 60, "--spmv", 4)
    gen = _run(17, 9, 6, "--max-iter", 60, "--spmv", 4, "--device-generate")
    assert _iters(st) and _iters(st) == _iters(gen)
    for k, v in _iters(base).items():
        assert _iters(st)[k] == pytest.approx(v, rel=1.1e-9)
