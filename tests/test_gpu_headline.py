"""Parity at the configurations the benchmark is quoted on, checked by the CPU oracle.

Every solver the benchmark times is run here at its own size, and the oracle
recomputes what the solver claims from the solver's output alone:

- 256^3 (16,777,216 rows, 449,455,096 nonzeros), x* U[-1,1) seed 1234,
  b = A x*, x0 = 0, stop at FP64 ||b - A x|| <= 1e-8 ||b||.  For FP64 CG on the
  stored matrix and matrix-free, FP32 and BF16-value refinement on the stored
  matrix, and FP32 refinement with the fused matrix-free inner pass (the
  headline method), the oracle's own operator and sequential sums give the
  true residual of the returned x (bar: <= 1e-8) and max|x - x*| (bar: 1e-6).
  The FP64 CG residual history is compared with the oracle's CG run with
  compensated dot products (the reference's iteration with near-exact sums;
  its own sequential sums err by ~N u = 1.9e-9 at this size) within the
  two-band 1e-12 bar of the 150-iteration tests, and the iteration counts
  must agree.
- The 64-system batch workload (nx, ny, nz each uniform in [16, 96], seed 7;
  11,216,985 rows): every system's true residual by the oracle, FP64 and FP32
  refinement, stored-matrix and matrix-free rows; FP64 iteration counts equal
  the oracle CG's (+-1 for a borderline stop); FP64 matrix-free iterates are
  bit-identical to the stored-matrix ones.
- 128^3 FP64 CG, 500 iterations: the whole history against the compensated
  oracle.

The oracle's grid form (generate_matrix's operator applied without storing
the CSR) repeats the CSR oracle's arithmetic bit for bit
(tests/test_oracle.py::test_grid_operator_equals_csr_oracle), so no 5.4 GB host
CSR is needed.  Reference: MPI/src/SparseMatrix.F90:68-232,
MPI/src/numerics.F90:41-162.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8
N256 = 256


@pytest.fixture(scope="module")
def hp():
    import hpccg_b200
    return hpccg_b200


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def assert_history_parity(h_gpu, h_ref, rtol=1e-12, band=1e-8):
    assert len(h_gpu) == len(h_ref)
    r0 = h_ref[0]
    for k in range(len(h_ref)):
        bound = rtol * h_ref[k] if h_ref[k] >= band * r0 else rtol * r0
        assert abs(h_gpu[k] - h_ref[k]) <= bound, (k, h_gpu[k], h_ref[k])


@pytest.fixture(scope="module")
def c256(hp, torch):
    """The 256^3 system on the device and its oracle data (x*, b)."""
    n = N256
    N = n ** 3
    d_x = torch.zeros(N, dtype=torch.float64, device="cuda")
    M = hp.Matrix.generated(n, n, n, d_x, None, None)
    assert M.nnz == 449455096
    d_xs = torch.empty_like(d_x)
    M.uniform_pm1(1234, d_xs)
    xs = oracle.uniform_pm1(1234, N)
    assert np.array_equal(d_xs.cpu().numpy(), xs)
    d_b = torch.empty_like(d_x)
    M.spmv(d_xs, d_b)
    b = oracle.grid_spmv(n, n, n, xs, omp=True)
    assert np.array_equal(d_b.cpu().numpy(), b)  # the reference's spmv, bit for bit
    yield M, d_x, d_b, xs, b
    M.close()


def _check_solution(n, b, xs, x):
    rel = oracle.grid_true_relres(n, n, n, b, x)
    err = float(np.abs(x - xs).max())
    assert rel <= REL_TOL * (1 + 1e-6), rel  # device and oracle sums differ in order (~1e-15 relative)
    assert err <= 1e-6, err
    return rel, err


def test_256_fp64_cg_history_and_solution(hp, torch, c256):
    M, d_x, d_b, xs, b = c256
    n = N256
    tol = REL_TOL * float(np.linalg.norm(b))
    with oracle.compensated_dots(omp=True):
        _, ref_it, ref_normr, ref_hist = oracle.cg_grid(n, n, n, b, np.zeros_like(b), 200, tol, omp=True)
    results = {}
    for kind in (hp.SPMV_AUTO, hp.SPMV_STENCIL):
        M.set_spmv(kind)
        d_x.zero_()
        it, normr, hist, st = M.cg_device(d_b, d_x, 200, tol, history=True)
        assert st == hp.HPCCG_OK
        assert it == ref_it, (kind, it, ref_it)
        assert_history_parity(hist, ref_hist)
        x = d_x.cpu().numpy()
        _check_solution(n, b, xs, x)
        results[kind] = (x, hist)
    # the matrix-free operator repeats the stored matrix's sums: identical iterates
    assert np.array_equal(results[hp.SPMV_AUTO][0], results[hp.SPMV_STENCIL][0])
    assert np.array_equal(results[hp.SPMV_AUTO][1], results[hp.SPMV_STENCIL][1])


@pytest.mark.parametrize("name", ["fp32_ir", "bf16_ir", "fp32_ir_stencil"])
def test_256_mixed_solution(hp, torch, c256, name):
    M, d_x, d_b, xs, b = c256
    n = N256
    prec = hp.PREC_BF16 if name.startswith("bf16") else hp.PREC_FP32
    M.set_spmv(hp.SPMV_STENCIL if name.endswith("stencil") else hp.SPMV_AUTO)
    if name.endswith("stencil"):
        assert M.mixed_fused()  # the headline's fused one-pass inner iteration
    d_x.zero_()
    info, st = M.solve_mixed_device(d_b, d_x, prec, REL_TOL)
    assert st == hp.HPCCG_OK
    rel, err = _check_solution(n, b, xs, d_x.cpu().numpy())
    # the device's own FP64 residual agrees with the oracle's
    assert info.relres == pytest.approx(rel, rel=1e-6)
    assert info.outer_iters >= 1 and info.inner_iters >= 1


def test_256_headline_host_array_call(hp, torch, c256):
    """The host-array call the end-to-end figure is measured through."""
    M, d_x, d_b, xs, b = c256
    n = N256
    M.set_spmv(hp.SPMV_STENCIL)
    x, info, st = M.solve_mixed(b, np.zeros_like(b), hp.PREC_FP32, REL_TOL)
    assert st == hp.HPCCG_OK
    _check_solution(n, b, xs, x)


def test_batch_workload_64_systems(hp, torch):
    sizes = hp.batch_sizes(7, 64, 16, 96)
    assert np.array_equal(sizes, oracle.batch_sizes(7, 64, 16, 96))
    B = hp.Batch.generated(sizes)
    assert int(B.nrows.sum()) == 11216985
    xs = [oracle.uniform_pm1(7 + s, int(B.nrows[s])) for s in range(B.nsys)]
    bs = [oracle.grid_spmv(int(nx), int(ny), int(nz), xs[s], omp=True) for s, (nx, ny, nz) in enumerate(sizes)]
    d_xs = torch.from_numpy(B.stack(xs)).cuda()
    d_b = torch.empty_like(d_xs)
    B.spmv(d_xs, d_b)
    got_b = B.unstack(d_b.cpu().numpy())
    for s in range(B.nsys):
        assert np.array_equal(got_b[s], bs[s]), s
    want_iters = []
    for s, (nx, ny, nz) in enumerate(sizes):
        tol = REL_TOL * float(np.linalg.norm(bs[s]))
        _, it, _, _ = oracle.cg_grid(int(nx), int(ny), int(nz), bs[s], np.zeros_like(bs[s]), 500, tol, omp=True)
        want_iters.append(it)
    d_x = torch.zeros_like(d_b)
    fp64_x = {}
    for kind in (hp.SPMV_ELL, hp.SPMV_STENCIL):
        B.set_spmv(kind)
        for prec in (hp.PREC_FP64, hp.PREC_FP32):
            d_x.zero_()
            iters, relres, outer, st = B.solve(d_b, d_x, prec, REL_TOL, 1000)
            assert st == hp.HPCCG_OK, (kind, prec)
            x = B.unstack(d_x.cpu().numpy())
            for s, (nx, ny, nz) in enumerate(sizes):
                rel = oracle.grid_true_relres(int(nx), int(ny), int(nz), bs[s], x[s])
                assert rel <= REL_TOL * (1 + 1e-6), (kind, prec, s, rel)
                assert relres[s] == pytest.approx(rel, rel=1e-6, abs=1e-15)
                assert np.abs(x[s] - xs[s]).max() <= 1e-6, (kind, prec, s)
                if prec == hp.PREC_FP64:
                    assert abs(int(iters[s]) - want_iters[s]) <= 1, (kind, s, iters[s], want_iters[s])
            if prec == hp.PREC_FP64:
                fp64_x[kind] = d_x.cpu().numpy()
    assert np.array_equal(fp64_x[hp.SPMV_ELL], fp64_x[hp.SPMV_STENCIL])
    B.close()


def test_128_cg_full_500_history(hp, torch):
    """C2: 128^3, 500 iterations, the whole residual history against the oracle
    with compensated dot products (two-band 1e-12 bar), and x -> 1."""
    n = 128
    N = n ** 3
    dx = torch.zeros(N, dtype=torch.float64, device="cuda")
    db = torch.zeros_like(dx)
    M = hp.Matrix.generated(n, n, n, dx, db, None)
    b = db.cpu().numpy()
    with oracle.compensated_dots(omp=True):
        ref_x, ref_it, _, ref_hist = oracle.cg_grid(n, n, n, b, np.zeros(N), 500, 0.0, omp=True)
    it, normr, hist, status = M.cg_device(db, dx, 500, 0.0)
    assert status == hp.HPCCG_OK and it == ref_it == 500
    assert_history_parity(hist, ref_hist)
    x = dx.cpu().numpy()
    assert np.abs(x - ref_x).max() <= 1e-10
    assert np.abs(x - 1.0).max() <= 1e-10
    M.close()
