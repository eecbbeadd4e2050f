"""The C++ host driver (HPCCG-B200), the reference's main.F90 over the C-ABI.

Checks the report against the reference's formats (MPI/src/main.F90:33-75,
numerics.F90:103-156): printInfo lines with total_nnz = 27 N, the initial
residual, the ITER lines at print_freq = clamp(max_iter/10, 1, 50) and at
k + 1 = max_iter in e20.10, the TIMER lines of each timing level and
MFLOPS SPARSEMV; the printed residuals equal the oracle's history to the 10
digits printed; the matrix-free SpMV prints the identical history.  The
options beyond the reference (--precision, --rel-tol, --batch) against the
library's own calls and the oracle, the host-array batch call, and host-side
fault injection (a NaN in b, a zero on the diagonal).
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


def _field(pattern, text, cast=float):
    m = re.search(pattern, text, re.M)
    assert m, (pattern, text[-2000:])
    return cast(m.group(1))


@pytest.mark.parametrize("extra", [(), ("--spmv", 4, "--device-generate")])
def test_driver_mixed_precision_reaches_fp64_target(extra):
    """--precision fp32: FP64 refinement around the FP32 inner CG on the reference's problem (b = A 1),
    to the FP64 relative residual --rel-tol; the same cycles and inner iterations as the library call
    on the same system, and the oracle's own residual of x = 1 bounds the error."""
    import hpccg_b200 as hp

    n = 24
    out = _run(n, n, n, "--precision", "fp32", "--rel-tol", "1e-9", *extra)
    relres = _field(r"FP64 rel-res: (\S+)$", out)
    outer = _field(r"Refinement cycles: (\d+)", out, int)
    inner = _field(r"inner iterations: (\d+)", out, int)
    err = _field(r"max\|x - xexact\|: (\S+)$", out)
    assert relres <= 1e-9 and err <= 1e-7, (relres, err)
    A, x, b, xe = oracle.generate_matrix(n, n, n)
    M = hp.Matrix.generated(n, n, n) if extra else hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    if extra:
        M.set_spmv(hp.SPMV_STENCIL)
    gx, info, st = M.solve_mixed(b, x.copy(), hp.PREC_FP32, 1e-9, 30, 150)
    M.close()
    assert st == hp.HPCCG_OK and (info.outer_iters, info.inner_iters) == (outer, inner)
    assert oracle.true_relres(A, b, gx) <= 1e-9 * (1 + 1e-6)


def test_driver_batch_random_spec_matches_oracle():
    """--batch random:COUNT,LO,HI,SEED draws the sizes from the project's generator (the bench's batch
    workload uses the same draw); every system of the reference's problem is solved in FP64 CG to
    --rel-tol with the oracle CG's iteration count (one more or less for a stop on the border)."""
    spec = (6, 6, 20, 7)
    out = _run("--batch", "random:%d,%d,%d,%d" % spec)
    sizes = oracle.batch_sizes(spec[3], spec[0], spec[1], spec[2])
    lines = re.findall(r"^ System (\d+) \((\d+) x (\d+) x (\d+)\): iterations (\d+), refinement cycles (\d+), "
                       r"FP64 rel-res (\S+), max\|x - xexact\| (\S+)$", out, re.M)
    assert len(lines) == spec[0]
    for s, (idx, nx, ny, nz, it, _, rel, err) in enumerate(lines):
        assert int(idx) == s and [int(nx), int(ny), int(nz)] == list(sizes[s])
        A, x, b, _ = oracle.generate_matrix(*sizes[s])
        _, ref_it, _, _ = oracle.cg(A, b, x, 1000, 1e-8 * float(np.linalg.norm(b)))
        assert abs(int(it) - ref_it) <= 1, (s, it, ref_it)
        assert float(rel) <= 1e-8 and float(err) <= 1e-6
    assert re.search(r"^ TIMER: Device\s+\S+ sec$", out, re.M)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_driver_batch_list_spec_mixed(prec):
    """An explicit size list, FP64 refinement around the low-precision inner CG per system, with the
    stored-matrix rows and the matrix-free ones."""
    for extra in ((), ("--spmv", 4)):
        out = _run("--batch", "5,6,7/16,16,16/1,1,40", "--precision", prec, *extra)
        rel = [float(v) for v in re.findall(r"FP64 rel-res (\S+),", out)]
        assert len(rel) == 3 and max(rel) <= 1e-8, (extra, rel)


def test_batch_host_arrays_equal_device_vectors():
    """hpccg_batch_solve_host (host arrays in and out) gives the device-vector call's iterates."""
    import torch

    import hpccg_b200 as hp

    sizes = [(5, 6, 7), (12, 9, 8), (3, 3, 33)]
    B = hp.Batch.generated(sizes)
    xs = B.stack([oracle.uniform_pm1(3 + s, int(B.nrows[s])) for s in range(B.nsys)])
    d_xs = torch.from_numpy(xs).cuda()
    d_b = torch.empty_like(d_xs)
    B.spmv(d_xs, d_b)
    b = d_b.cpu().numpy()
    for prec in (hp.PREC_FP64, hp.PREC_FP32):
        d_x = torch.zeros_like(d_b)
        it_d, rel_d, out_d, rc_d = B.solve(d_b, d_x, prec, 1e-9)
        x = np.zeros_like(b)
        it_h, rel_h, out_h, rc_h = B.solve_host(b, x, prec, 1e-9)
        assert rc_d == rc_h == hp.HPCCG_OK
        assert np.array_equal(it_d, it_h) and np.array_equal(out_d, out_h) and np.array_equal(rel_d, rel_h)
        assert np.array_equal(d_x.cpu().numpy(), x)


def test_nan_in_b_is_reported_not_hung():
    """Fault injection on the host: a NaN in b makes the first alpha non-finite; the CG graph exits
    and the call returns HPCCG_ERR_BREAKDOWN at once, and the mixed solver stops with a non-OK status
    within its cycle cap; the context stays usable for the next solve."""
    import hpccg_b200 as hp

    A, x, b, xe = oracle.generate_matrix(8, 8, 8)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    bad = b.copy()
    bad[17] = np.nan
    _, it, normr, hist, st = M.cg(bad, x.copy(), 150, 0.0)
    assert st == hp.HPCCG_ERR_BREAKDOWN and it < 150
    _, info, mst = M.solve_mixed(bad, x.copy(), hp.PREC_FP32, 1e-8, 3, 50)
    assert mst in (hp.HPCCG_ERR_BREAKDOWN, hp.HPCCG_ERR_NOT_CONVERGED)
    gx, it, normr, hist, st = M.cg(b, x.copy(), 150, 0.0)  # the same context, a clean right-hand side
    assert st == hp.HPCCG_OK and np.abs(gx - xe).max() <= 1e-10
    M.close()


def test_zero_diagonal_ends_within_caps():
    """Fault injection on the host: a zero on the diagonal makes A indefinite.  The reference's CG has
    no test for that and runs to max_iter; so does this one (or it stops with HPCCG_ERR_BREAKDOWN if a
    scalar turns non-finite), the mixed solver ends within its cycle cap, and the next context solves
    the intact matrix."""
    import hpccg_b200 as hp

    A, x, b, xe = oracle.generate_matrix(6, 5, 4)
    vals = A.values.copy()
    row = 37
    for k in range(A.rowindex[row] - 1, A.rowindex[row + 1] - 1):
        if A.colindex[k] - 1 == row:
            vals[k] = 0.0
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, vals)
    _, it, normr, hist, st = M.cg(b, x.copy(), 150, 0.0)
    assert st in (hp.HPCCG_OK, hp.HPCCG_ERR_BREAKDOWN) and it <= 150
    _, info, mst = M.solve_mixed(b, x.copy(), hp.PREC_FP32, 1e-8, 3, 50)
    assert mst in (hp.HPCCG_OK, hp.HPCCG_ERR_NOT_CONVERGED, hp.HPCCG_ERR_BREAKDOWN) and info.outer_iters <= 3
    M.close()
    M2 = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    gx, it, normr, hist, st = M2.cg(b, x.copy(), 150, 0.0)
    assert st in (hp.HPCCG_OK, hp.HPCCG_ERR_BREAKDOWN) and np.abs(gx - xe).max() <= 1e-10
    M2.close()


def test_zero_rhs_edge_cases():
    """b = 0.  From x0 = 0 the mixed solver and the batch report convergence at once (r = 0 too); from
    x0 != 0 the relative target ||r|| <= tol ||b|| = 0 cannot be met, so they stop at their caps with
    HPCCG_ERR_NOT_CONVERGED (never a false success), having driven x towards 0.  The reference's CG
    (tolerance 0) computes 0/0 on r = 0; the C-ABI stops there with HPCCG_ERR_BREAKDOWN and x0 unchanged."""
    import torch

    import hpccg_b200 as hp

    A, x, b, xe = oracle.generate_matrix(6, 6, 6)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    zero = np.zeros_like(b)
    _, info, st = M.solve_mixed(zero, zero.copy(), hp.PREC_FP32, 1e-8, 3, 50)
    assert st == hp.HPCCG_OK and info.relres == 0.0
    x1 = np.ones_like(b)
    _, info, st = M.solve_mixed(zero, x1, hp.PREC_FP32, 1e-8, 3, 50)
    assert st == hp.HPCCG_ERR_NOT_CONVERGED and info.outer_iters == 3 and np.abs(x1).max() < 1e-3
    gx, it, normr, hist, st = M.cg(zero, zero.copy(), 150, 0.0)
    assert st == hp.HPCCG_ERR_BREAKDOWN and normr == 0.0 and not np.any(gx)
    M.close()
    B = hp.Batch.generated([(6, 6, 6), (5, 4, 3)])
    d_b = torch.zeros(B.stacked_rows, dtype=torch.float64, device="cuda")
    for prec in (hp.PREC_FP64, hp.PREC_FP32):
        d_x = torch.zeros_like(d_b)
        iters, relres, outer, rc = B.solve(d_b, d_x, prec, 1e-8)
        assert rc == hp.HPCCG_OK and not np.any(relres), (prec, relres)
        d_x = torch.from_numpy(B.stack([np.ones(int(n)) for n in B.nrows])).cuda()  # zero gaps
        iters, relres, outer, rc = B.solve(d_b, d_x, prec, 1e-8, 40)
        assert rc == hp.HPCCG_ERR_NOT_CONVERGED and np.all(relres > 1e300), (prec, relres)


@pytest.mark.parametrize("halo,mode", [("mpi", 0), ("get", 1)])
@pytest.mark.parametrize("nx,ny,nz,P", [(8, 6, 4, 2), (6, 5, 4, 3)])
def test_driver_ranks_prints_the_oracle_multi_rank_history(halo, mode, nx, ny, nz, P):
    """--ranks P: the reference's P-rank run (z slabs of nx x ny x nz*P, make_local_matrix's plan in
    the MPI or CAF-V2 form, rank-order sums), all ranks in one process; the report's sizes are the
    reference's totals and the printed residuals are the oracle's multi-rank CG history."""
    iters = 60
    out = _run(nx, ny, nz, "--ranks", P, "--halo", halo, "--max-iter", iters)
    N = nx * ny * nz * P
    assert re.search(r"Total size \(N x N\):\s+%d$" % N, out, re.M)
    assert re.search(r"Total nonzeroes:\s+%d$" % (27 * N), out, re.M)
    _, x0, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
    rx, rit, rnr, rh = oracle.SlabPlan(nx, ny, nz, P, mode).cg(bg, x0, iters, 0.0)
    got = _iters(out)
    assert sorted(got) == sorted(set(range(6, iters + 1, 6)) | {iters - 1})
    for k, v in got.items():
        assert v == pytest.approx(rh[k], rel=1e-9, abs=1e-12 * rh[0]), (k, v, rh[k])
    assert _field(r"Iterations: (\d+)", out, int) == rit
    assert _field(r"max\|x - xexact\|: (\S+)$", out) <= 1e-10
