"""Mixed precision: FP64 iterative refinement around FP32 / BF16-value inner CG.

Bars: the low-precision SpMV matches an FP32 row sum within 2^-20 of
sum_k |a_ik x_k| (FP32 accumulation; BF16 values of this matrix are exact);
every solve's FP64 true residual, recomputed by the CPU oracle from the
returned x, meets rel_tol = 1e-8; the error against the FP64 oracle's solution
and against x* is reported and bounded.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

FP32, BF16 = 1, 2


@pytest.fixture(scope="module")
def hp():
    import hpccg_b200
    return hpccg_b200


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def _problem(n, seed=1234):
    A, x, b1, xe = oracle.generate_matrix(n, n, n)
    xstar = oracle.uniform_pm1(seed, A.nrow)
    b = oracle.spmv(A, xstar)
    return A, b, xstar


@pytest.mark.parametrize("prec", [FP32, BF16])
@pytest.mark.parametrize("rpt", [1, 2, 4])
def test_spmv_lowp(hp, torch, prec, rpt):
    A, b, xstar = _problem(24)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    M.set_mixed_rows_per_thread(prec, rpt)
    x32 = xstar.astype(np.float32)
    dx = torch.from_numpy(x32).cuda()
    dy = torch.empty_like(dx)
    M.spmv_lowp(prec, dx, dy)
    ref = oracle.spmv(A, x32.astype(np.float64))
    absref = oracle.spmv(oracle.Matrix(A.nx, A.ny, A.nz, A.rowindex, A.colindex, np.abs(A.values), A.nnz),
                         np.abs(x32).astype(np.float64))
    assert np.all(np.abs(dy.cpu().numpy() - ref) <= 2.0 ** -20 * absref + 1e-30)


@pytest.mark.parametrize("prec", [FP32, BF16])
@pytest.mark.parametrize("n", [16, 40, 64])
def test_mixed_solve_meets_fp64_target(hp, prec, n):
    A, b, xstar = _problem(n)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    x = np.zeros_like(b)
    x, info, status = M.solve_mixed(b, x, prec, rel_tol=1e-8)
    assert status == hp.HPCCG_OK
    rel = oracle.true_relres(A, b, x)
    assert rel <= 1e-8 and info.relres <= 1e-8
    assert abs(rel - info.relres) <= 1e-3 * 1e-8  # the device FP64 residual is the oracle's
    assert 1 <= info.outer_iters <= 6
    # error against the FP64 oracle CG run to the same FP64 target
    xo, it, _, _ = oracle.cg(A, b, np.zeros_like(b), 1000, 1e-8 * np.linalg.norm(b))
    assert np.abs(x - xo).max() <= 1e-7
    assert np.abs(x - xstar).max() <= 1e-7


def test_mixed_fixed_inner_tolerance_and_cycle_cap(hp):
    A, b, xstar = _problem(32)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    x, info, status = M.solve_mixed(b, np.zeros_like(b), FP32, rel_tol=1e-8, inner_rtol=1e-2)
    assert status == hp.HPCCG_OK and info.outer_iters >= 4
    x, info, status = M.solve_mixed(b, np.zeros_like(b), FP32, rel_tol=1e-12, max_outer=1, inner_rtol=1e-3)
    assert status == hp.HPCCG_ERR_NOT_CONVERGED and info.outer_iters == 1
    assert 1e-12 < info.relres < 1e-2


def test_mixed_zero_rhs_and_exact_start(hp):
    A, b, xstar = _problem(8)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    x, info, status = M.solve_mixed(np.zeros_like(b), np.zeros_like(b), BF16, rel_tol=1e-8)
    assert status == hp.HPCCG_OK and info.outer_iters == 0 and np.all(x == 0)
    x, info, status = M.solve_mixed(b, xstar.copy(), BF16, rel_tol=1e-8)  # x0 = x*: r = 0 already
    assert status == hp.HPCCG_OK and info.outer_iters == 0


def test_mixed_device_matches_host(hp, torch):
    A, b, xstar = _problem(20)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    xh, info_h, st_h = M.solve_mixed(b, np.zeros_like(b), BF16, rel_tol=1e-8)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros_like(db)
    info_d, st_d = M.solve_mixed_device(db, dx, BF16, rel_tol=1e-8)
    assert st_h == st_d == hp.HPCCG_OK
    assert np.array_equal(dx.cpu().numpy(), xh)
    assert (info_h.outer_iters, info_h.inner_iters) == (info_d.outer_iters, info_d.inner_iters)


def test_mixed_eager_equals_graph(hp, monkeypatch):
    A, b, xstar = _problem(18)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    xg, ig, sg = M.solve_mixed(b, np.zeros_like(b), FP32, rel_tol=1e-8)
    monkeypatch.setenv("HPCCG_EAGER", "1")
    xe, ie, se = M.solve_mixed(b, np.zeros_like(b), FP32, rel_tol=1e-8)
    assert np.array_equal(xg, xe) and ig.inner_iters == ie.inner_iters
