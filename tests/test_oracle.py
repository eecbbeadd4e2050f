"""The CPU oracle against the golden fixtures and the analytic known answers.

The reference ships no tests or golden vectors, so the oracle is pinned by facts
that follow from its definitions (MPI/src/SparseMatrix.F90:68-185,
MPI/src/numerics.F90:41-162) and by the committed fixtures.
"""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KNOWN = json.load(open(os.path.join(GOLDEN, "known_answers.json")))

SIZES = [(1, 1, 1), (2, 1, 1), (1, 2, 3), (2, 2, 2), (3, 5, 7), (4, 4, 4), (7, 1, 3), (16, 16, 16),
         (5, 9, 2)]


def _expected_nnz(nx, ny, nz):
    t = lambda n: 3 * n - 2 if n >= 2 else 1  # noqa: E731
    return t(nx) * t(ny) * t(nz)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_generate_matrix_structure(nx, ny, nz):
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    n = nx * ny * nz
    assert A.nnz == _expected_nnz(nx, ny, nz)
    assert A.rowindex[0] == 1 and A.rowindex[-1] == A.nnz + 1
    lens = np.diff(A.rowindex)
    assert lens.min() >= 1 and lens.max() <= 27
    assert A.colindex.min() >= 1 and A.colindex.max() <= n
    for i in range(n):  # columns ascend inside each row; diagonal is 27
        cols = A.colindex[A.rowindex[i] - 1:A.rowindex[i + 1] - 1]
        vals = A.values[A.rowindex[i] - 1:A.rowindex[i + 1] - 1]
        assert np.all(np.diff(cols) > 0)
        assert vals[cols == i + 1].tolist() == [27.0]
        assert np.all(vals[cols != i + 1] == -1.0)
    assert np.all(x == 0.0) and np.all(xe == 1.0)
    assert np.array_equal(oracle.spmv(A, xe), b)  # b = A*1 exactly (small integers)
    assert np.array_equal(b, 28.0 - lens)


def test_interior_row_columns():
    nx, ny, nz = 5, 6, 7
    A, *_ = oracle.generate_matrix(nx, ny, nz)
    ix, iy, iz = 3, 4, 5  # 1-based interior point
    row = (iz - 1) * nx * ny + (iy - 1) * nx + (ix - 1)
    cols = A.colindex[A.rowindex[row] - 1:A.rowindex[row + 1] - 1]
    want = [row + 1 + sz * nx * ny + sy * nx + sx for sz in (-1, 0, 1) for sy in (-1, 0, 1) for sx in (-1, 0, 1)]
    assert cols.tolist() == want


@pytest.mark.parametrize("name", ["csr_3x5x7", "csr_4x4x4", "csr_1x2x3", "csr_2x1x1"])
def test_oracle_matches_csr_fixture(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    nx, ny, nz = map(int, name.split("_")[1].split("x"))
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    assert np.array_equal(A.rowindex, d["rowindex"])
    assert np.array_equal(A.colindex, d["colindex"])
    assert np.array_equal(A.values, d["values"])
    assert np.array_equal(b, d["b"])


@pytest.mark.parametrize("key", ["16x16x16", "3x5x7", "2x2x2", "1x1x1", "7x1x3"])
def test_oracle_cg_matches_fixture(key):
    nx, ny, nz = map(int, key.split("x"))
    d = np.load(os.path.join(GOLDEN, f"cg_{key}.npz"))
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    xs, niters, normr, hist = oracle.cg(A, b, x, 150, 0.0)
    assert niters == int(d["niters"])
    np.testing.assert_array_equal(hist, d["hist"])  # same code, same order: bit-exact
    assert hist[0] == pytest.approx(KNOWN["initial_residual"][key], rel=1e-15)
    assert A.nnz == KNOWN["nnz"][key]


@pytest.mark.parametrize("key,iters", [("16x16x16", 24), ("32x32x32", 38)])
def test_iterations_to_1e8(key, iters):
    assert KNOWN["iters_to_1e-8"][key] == iters
    nx, ny, nz = map(int, key.split("x"))
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    xs, niters, normr, hist = oracle.cg(A, b, x, iters + 2, 0.0)
    rel = hist / hist[0]
    assert rel[iters] <= 1e-8 < rel[iters - 1]


def test_cg_converges_to_ones():
    A, x, b, xe = oracle.generate_matrix(16, 16, 16)
    xs, niters, normr, hist = oracle.cg(A, b, x, 150, 0.0)
    assert niters == 150
    assert hist[0] == pytest.approx(np.linalg.norm(b), rel=1e-14)  # Initial Residual = ||b||
    assert oracle.compute_residual(xs, xe) < 1e-13
    assert oracle.true_relres(A, b, xs) < 1e-14


def test_cg_tolerance_stop_semantics():
    """The stop test uses the normr of the previous iteration (numerics.F90:109)."""
    A, x, b, xe = oracle.generate_matrix(8, 8, 8)
    _, full_it, _, full_hist = oracle.cg(A, b, x, 150, 0.0)
    tol = 1e-6 * full_hist[0]
    xs, niters, normr, hist = oracle.cg(A, b, x, 150, tol)
    k_first = int(np.nonzero(full_hist < tol)[0][0])  # first k whose normr < tol
    assert niters == k_first  # iteration k_first+1 sees normr(k_first) < tol and exits
    assert normr == full_hist[k_first]
    np.testing.assert_array_equal(hist, full_hist[: niters + 1])


def test_omp_build_agrees():
    A, x, b, xe = oracle.generate_matrix(12, 10, 9)
    Ao, *_ = oracle.generate_matrix(12, 10, 9, omp=True)
    assert np.array_equal(A.colindex, Ao.colindex)
    xs, it, nr, h = oracle.cg(A, b, x, 40, 0.0)
    xo, ito, nro, ho = oracle.cg(A, b, x, 40, 0.0, omp=True)
    np.testing.assert_allclose(ho[:20], h[:20], rtol=1e-12)


def test_rng_counter_based():
    a = oracle.uniform_pm1(1234, 1000)
    assert a.min() >= -1.0 and a.max() < 1.0
    assert abs(a.mean()) < 0.1
    b = oracle.uniform_pm1(1234, 10)
    np.testing.assert_array_equal(a[:10], b)
    assert oracle.splitmix64_at(0, 0) == 0xE220A8397B1DCDAF  # splitmix64 from state 0: first output
    s = oracle.batch_sizes(7, 64, 16, 96)
    assert s.shape == (64, 3) and s.min() >= 16 and s.max() <= 96


@pytest.mark.parametrize("nx,ny,nz", SIZES + [(33, 17, 5), (24, 24, 24)])
def test_grid_operator_equals_csr_oracle(nx, ny, nz):
    """The grid forms of spmv, cg and the true residual (used where a host CSR would be
    gigabytes) repeat the CSR oracle's arithmetic bit for bit."""
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    v = oracle.uniform_pm1(99, A.nrow)
    want = oracle.spmv(A, v)
    assert np.array_equal(oracle.grid_spmv(nx, ny, nz, v), want)
    assert np.array_equal(oracle.grid_spmv(nx, ny, nz, v, omp=True), want)
    same = lambda u, w: np.array_equal(np.asarray(u), np.asarray(w), equal_nan=True)  # noqa: E731
    r1 = oracle.cg(A, b, x, 40, 0.0)  # tiny grids converge exactly and then carry NaN, as the reference
    r2 = oracle.cg_grid(nx, ny, nz, b, x, 40, 0.0)
    r3 = oracle.cg_grid(nx, ny, nz, b, x, 40, 0.0, omp=True)
    assert same(r1[0], r2[0]) and same(r1[3], r2[3]) and r1[1] == r2[1] and same(r1[2], r2[2])
    with oracle.compensated_dots(omp=True), oracle.compensated_dots():
        c1 = oracle.cg(A, b, x, 40, 0.0)
        c3 = oracle.cg_grid(nx, ny, nz, b, x, 40, 0.0, omp=True)
    assert same(c1[3], c3[3]) and same(c1[0], c3[0])
    assert r3[1] == r1[1]
    xs = oracle.uniform_pm1(5, A.nrow)
    bs = oracle.spmv(A, xs)
    assert oracle.grid_true_relres(nx, ny, nz, bs, v) == oracle.true_relres(A, bs, v)


@pytest.mark.parametrize("case", ["4x3x2x2", "4x3x2x3", "3x3x1x3"])
@pytest.mark.parametrize("tag", ["mpi", "get"])
def test_slab_oracle_against_fixtures(case, tag):
    """The multi-rank oracle (make_local_matrix in both forms, the multi-rank CG) against the
    committed fixtures, list by list."""
    nx, ny, nz, P = map(int, case.split("x"))
    gold = np.load(os.path.join(GOLDEN, f"slab_{case}_{tag}.npz"))
    plan = oracle.SlabPlan(nx, ny, nz, P, oracle.HALO_MPI if tag == "mpi" else oracle.HALO_GET)
    for key in gold.files:
        if key == "hist":
            continue
        r, field = key.split("_", 1)
        np.testing.assert_array_equal(plan.get(int(r[1:]), field), gold[key], err_msg=key)
    G, x0, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
    np.testing.assert_array_equal(plan.cg(bg, x0, 30, 0.0)[3], gold["hist"])
