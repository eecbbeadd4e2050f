"""Matrix-free SpMV (HPCCG_SPMV_STENCIL) against the CSR it replaces.

Bars: the device check accepts exactly the generate_matrix CSR (any changed
column, value or row length is rejected); the stencil SpMV is bit-identical
to the ELL SpMV and to the oracle's spmv; a whole FP64 CG run (x, iteration
count and residual history) is bit-identical to the ELL run; the FP32
matrix-free inner solve of the iterative refinement meets the FP64 target.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SIZES = [(1, 1, 1), (2, 1, 1), (1, 2, 3), (2, 2, 2), (3, 5, 7), (7, 1, 3), (9, 2, 11), (33, 17, 5),
         (16, 16, 16), (64, 64, 64), (128, 4, 2)]


@pytest.fixture(scope="module")
def hp():
    import hpccg_b200
    return hpccg_b200


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_stencil_spmv_bit_identical(hp, torch, nx, ny, nz):
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    n = nx * ny * nz
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    with pytest.raises(hp.HpccgError):
        M.set_spmv(hp.SPMV_STENCIL)  # geometry not declared yet
    M.set_geometry(nx, ny, nz)
    rng = np.random.default_rng(nx * 10007 + ny * 101 + nz)
    xv = rng.uniform(-1, 1, n) * np.exp2(rng.integers(-20, 20, n))
    want = oracle.spmv(A, xv)
    dx = torch.from_numpy(xv).cuda()
    y_ell = torch.empty_like(dx)
    y_st = torch.empty_like(dx)
    M.set_spmv(hp.SPMV_ELL, 4)
    M.spmv(dx, y_ell)
    M.set_spmv(hp.SPMV_STENCIL)
    assert M.get_spmv()[0] == hp.SPMV_STENCIL
    M.spmv(dx, y_st)
    assert np.array_equal(_bits(y_st.cpu().numpy()), _bits(y_ell.cpu().numpy()))
    assert np.array_equal(_bits(y_st.cpu().numpy()), _bits(want))
    G = hp.Matrix.generated(nx, ny, nz)  # generated contexts are checked at creation
    G.set_spmv(hp.SPMV_STENCIL)
    y_g = torch.empty_like(dx)
    G.spmv(dx, y_g)
    assert np.array_equal(_bits(y_g.cpu().numpy()), _bits(want))


def test_stencil_check_rejects_other_matrices(hp):
    nx, ny, nz = 6, 5, 4
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    with pytest.raises(hp.HpccgError) as e:
        hp.Matrix.from_csr(A.rowindex, A.colindex, A.values).set_geometry(nx, ny, nz + 1)
    assert e.value.code == hp.HPCCG_ERR_INVALID_ARG
    with pytest.raises(hp.HpccgError) as e:  # same row count, other shape
        hp.Matrix.from_csr(A.rowindex, A.colindex, A.values).set_geometry(nz, ny, nx)
    assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
    v = A.values.copy()
    v[37] = -2.0
    with pytest.raises(hp.HpccgError) as e:
        hp.Matrix.from_csr(A.rowindex, A.colindex, v).set_geometry(nx, ny, nz)
    assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
    # a row with its last term dropped (row pointers shifted after it)
    r = A.rowindex.copy()
    c = np.delete(A.colindex, r[11] - 2)
    vv = np.delete(A.values, r[11] - 2)
    r[11:] -= 1
    M = hp.Matrix.from_csr(r, c, vv)
    with pytest.raises(hp.HpccgError) as e:
        M.set_geometry(nx, ny, nz)
    assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
    with pytest.raises(hp.HpccgError):
        M.set_spmv(hp.SPMV_STENCIL)


@pytest.mark.parametrize("key", ["32x32x32", "3x5x7", "17x9x6"])
def test_stencil_cg_bit_identical_to_ell(hp, key):
    nx, ny, nz = map(int, key.split("x"))
    A, x, b, xe = oracle.generate_matrix(nx, ny, nz)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    M.set_geometry(nx, ny, nz)
    M.set_spmv(hp.SPMV_ELL, 4)
    x1, it1, nr1, h1, s1 = M.cg(b, x.copy(), 150, 0.0)
    M.set_spmv(hp.SPMV_STENCIL)
    x2, it2, nr2, h2, s2 = M.cg(b, x.copy(), 150, 0.0)
    assert (it1, s1) == (it2, s2)
    assert np.array_equal(_bits(x1), _bits(x2)) and np.array_equal(_bits(h1), _bits(h2))
    assert _bits(np.array([nr1]))[0] == _bits(np.array([nr2]))[0]
    assert np.abs(x2 - 1.0).max() <= 1e-10


def test_stencil_cg_128_matches_ell(hp, torch):
    n = 128
    dx = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    db = torch.zeros_like(dx)
    M = hp.Matrix.generated(n, n, n, dx, db, None)
    M.set_spmv(hp.SPMV_ELL, 4)
    it1, nr1, h1, s1 = M.cg_device(db, dx, 120, 0.0)
    x1 = dx.cpu().numpy()
    dx.zero_()
    M.set_spmv(hp.SPMV_STENCIL)
    it2, nr2, h2, s2 = M.cg_device(db, dx, 120, 0.0)
    assert (it1, s1) == (it2, s2) == (120, hp.HPCCG_OK)
    assert np.array_equal(_bits(h1), _bits(h2)) and np.array_equal(_bits(x1), _bits(dx.cpu().numpy()))


@pytest.mark.parametrize("precision", [1, 2])
def test_stencil_mixed_refinement(hp, torch, precision):
    n = 48
    dx = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    db = torch.zeros_like(dx)
    M = hp.Matrix.generated(n, n, n)
    xs = torch.empty_like(dx)
    M.uniform_pm1(1234, xs)
    M.spmv(xs, db)
    M.set_spmv(hp.SPMV_STENCIL)
    info, rc = M.solve_mixed_device(db, dx, precision, rel_tol=1e-8)
    assert rc == hp.HPCCG_OK and info.relres <= 1e-8
    r = torch.empty_like(dx)
    M.set_spmv(hp.SPMV_ELL, 4)
    M.spmv(dx, r)
    true_rel = float(torch.linalg.vector_norm(db - r) / torch.linalg.vector_norm(db))
    assert true_rel <= 1e-8
    assert float((dx - xs).abs().max()) <= 1e-6
    y32 = torch.empty(n ** 3, dtype=torch.float32, device="cuda")
    M.set_spmv(hp.SPMV_STENCIL)
    M.spmv_lowp(precision, xs.float(), y32)
    ref = torch.empty_like(dx)
    M.spmv(xs.float().double(), ref)
    assert float((y32.double() - ref).abs().max()) <= 1e-5 * float(ref.abs().max())


@pytest.mark.parametrize("nx,ny,nz", [(3, 5, 7), (9, 2, 11), (4, 4, 4), (16, 16, 16), (33, 17, 5), (128, 4, 2),
                                      (12, 20, 7), (1, 1, 1)])
def test_stencil_fp32_spmv(hp, torch, nx, ny, nz):
    """The FP32 matrix-free SpMV of the inner solves (box sums; four columns per
    thread when nx is a multiple of 4) against the FP64 SpMV of the same
    FP32-rounded input, within FP32 accumulation error."""
    n = nx * ny * nz
    M = hp.Matrix.generated(nx, ny, nz)
    M.set_spmv(hp.SPMV_STENCIL)
    rng = np.random.default_rng(n + 3)
    x32 = torch.from_numpy(rng.uniform(-1, 1, n).astype(np.float32)).cuda()
    y32 = torch.empty_like(x32)
    M.spmv_lowp(hp.PREC_FP32, x32, y32)
    ref = torch.empty(n, dtype=torch.float64, device="cuda")
    M.spmv(x32.double(), ref)
    err = float((y32.double() - ref).abs().max())
    assert err <= 2e-5 * max(1.0, float(ref.abs().max())), err


def _stencil64(x, nx, ny, nz):
    """A x of the generate_matrix operator (27 on the diagonal, -1 for each
    neighbour inside the grid) in FP64: 28 x - (sum of the 3x3x3 box)."""
    g = np.asarray(x, np.float64).reshape(nz, ny, nx)
    pad = np.pad(g, 1)
    box = np.zeros_like(g)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                box += pad[dz:dz + nz, dy:dy + ny, dx:dx + nx]
    return (28.0 * g - box).ravel()


FUSED_SIZES = [(4, 4, 4), (8, 8, 1), (16, 1, 16), (12, 20, 7), (32, 64, 3), (48, 70, 9), (36, 5, 40),
               (96, 130, 5)]


@pytest.mark.parametrize("nx,ny,nz", FUSED_SIZES)
@pytest.mark.parametrize("first", [True, False])
def test_fused_pass_matches_fp64(hp, torch, nx, ny, nz, first):
    """One fused inner-CG pass (r' = r - alpha A p, p' = r' + beta p,
    d += alpha p, the four dots of A p') against the same algebra in FP64 on
    the FP32 inputs; partial tiles in x and y, a single plane, a single row."""
    n = nx * ny * nz
    M = hp.Matrix.generated(nx, ny, nz)
    M.set_spmv(hp.SPMV_STENCIL)
    assert M.mixed_fused()
    rng = np.random.default_rng(n * 7 + int(first))
    r, p, d = (rng.uniform(-1, 1, n).astype(np.float32) for _ in range(3))
    alpha, beta = 0.37, 0.81
    dr, dp, dd = (torch.from_numpy(v.copy()).cuda() for v in (r, p, d))
    ro, po = torch.full_like(dr, np.nan), torch.full_like(dr, np.nan)
    dots = M.mixed_pass(dr, dp, dd, ro, po, alpha, beta, first)
    a32, b32 = float(np.float32(alpha)), float(np.float32(beta))
    r64, p64, d64 = (v.astype(np.float64) for v in (r, p, d))
    if first:  # the first pass of an inner solve (scale 1 here) also clears d
        rn, pn, dn = r64, r64, np.zeros_like(d64)
    else:
        rn = r64 - a32 * _stencil64(p64, nx, ny, nz)
        pn = rn + b32 * p64
        dn = d64 + a32 * p64
    apn = _stencil64(pn, nx, ny, nz)
    assert float(np.abs(ro.cpu().numpy() - rn).max()) <= 1e-4
    assert float(np.abs(po.cpu().numpy() - pn).max()) <= 1e-4
    assert float(np.abs(dd.cpu().numpy() - dn).max()) <= 1e-6
    want = [pn @ apn, rn @ apn, apn @ apn, rn @ rn]
    scale = [np.abs(pn * apn).sum(), np.abs(rn * apn).sum(), apn @ apn, rn @ rn]
    for got, w, s in zip(dots, want, scale):
        assert abs(got - w) <= 1e-5 * s, (got, w)


@pytest.mark.parametrize("n", [48, 64, 100])
def test_fused_inner_solve_matches_three_kernel(hp, torch, n):
    """The mixed FP32 stencil solve with the fused one-pass iteration meets the
    FP64 target with about the iteration count of the three-kernel iteration."""
    dx = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    db = torch.zeros_like(dx)
    M = hp.Matrix.generated(n, n, n)
    xs = torch.empty_like(dx)
    M.uniform_pm1(99, xs)
    M.spmv(xs, db)
    M.set_spmv(hp.SPMV_STENCIL)
    assert M.mixed_fused()
    ms = M.time_mixed_kernels(hp.PREC_FP32, 3)
    assert ms[0] > 0.0 and ms[2] == 0.0 and ms[1] > 0.0  # FP64 refinement residual, fused pass
    info_f, rc_f = M.solve_mixed_device(db, dx, hp.PREC_FP32, rel_tol=1e-8)
    assert rc_f == hp.HPCCG_OK and info_f.relres <= 1e-8
    r = torch.empty_like(dx)
    M.spmv(dx, r)
    assert float(torch.linalg.vector_norm(db - r) / torch.linalg.vector_norm(db)) <= 1e-8
    M.set_mixed_fused(False)
    assert not M.mixed_fused()
    dx.zero_()
    info_3, rc_3 = M.solve_mixed_device(db, dx, hp.PREC_FP32, rel_tol=1e-8)
    assert rc_3 == hp.HPCCG_OK
    assert abs(info_f.inner_iters - info_3.inner_iters) <= max(3, info_3.inner_iters // 10)
    assert info_f.outer_iters <= info_3.outer_iters + 1


def _fused_problem(hp, n, seed=1234):
    A, x, b1, xe = oracle.generate_matrix(n, n, n)
    xstar = oracle.uniform_pm1(seed, A.nrow)
    b = oracle.spmv(A, xstar)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    M.set_geometry(n, n, n)
    M.set_spmv(hp.SPMV_STENCIL)
    assert M.mixed_fused()
    return A, b, xstar, M


@pytest.mark.parametrize("prec", [1, 2])
def test_fused_solve_meets_target_against_oracle(hp, prec):
    """The fused inner iteration inside FP64 refinement: the CPU oracle's FP64
    residual of the returned x meets 1e-8 and x is within 1e-7 of the oracle's
    FP64 CG solution and of x*."""
    A, b, xstar, M = _fused_problem(hp, 20)
    x, info, status = M.solve_mixed(b, np.zeros_like(b), prec, rel_tol=1e-8)
    assert status == hp.HPCCG_OK
    rel = oracle.true_relres(A, b, x)
    assert rel <= 1e-8 and abs(rel - info.relres) <= 1e-3 * 1e-8
    xo, it, _, _ = oracle.cg(A, b, np.zeros_like(b), 1000, 1e-8 * np.linalg.norm(b))
    assert np.abs(x - xo).max() <= 1e-7 and np.abs(x - xstar).max() <= 1e-7


def test_fused_eager_equals_graph_and_is_deterministic(hp, monkeypatch):
    A, b, xstar, M = _fused_problem(hp, 24)
    xg, ig, sg = M.solve_mixed(b, np.zeros_like(b), 1, rel_tol=1e-8)
    xg2, ig2, _ = M.solve_mixed(b, np.zeros_like(b), 1, rel_tol=1e-8)
    monkeypatch.setenv("HPCCG_EAGER", "1")
    xe, ie, se = M.solve_mixed(b, np.zeros_like(b), 1, rel_tol=1e-8)
    assert sg == se == hp.HPCCG_OK
    assert np.array_equal(_bits(xg), _bits(xg2)) and np.array_equal(_bits(xg), _bits(xe))
    assert (ig.outer_iters, ig.inner_iters) == (ie.outer_iters, ie.inner_iters) == (ig2.outer_iters, ig2.inner_iters)


def test_fused_zero_rhs_exact_start_and_caps(hp):
    A, b, xstar, M = _fused_problem(hp, 16)
    x, info, status = M.solve_mixed(np.zeros_like(b), np.zeros_like(b), 1, rel_tol=1e-8)
    assert status == hp.HPCCG_OK and info.outer_iters == 0 and np.all(x == 0)
    x, info, status = M.solve_mixed(b, xstar.copy(), 1, rel_tol=1e-8)  # r = 0 already
    assert status == hp.HPCCG_OK and info.outer_iters == 0
    # a loose fixed inner target needs more refinement cycles; a cycle cap stops early
    x, info, status = M.solve_mixed(b, np.zeros_like(b), 1, rel_tol=1e-8, inner_rtol=1e-2)
    assert status == hp.HPCCG_OK and info.outer_iters >= 4
    x, info, status = M.solve_mixed(b, np.zeros_like(b), 1, rel_tol=1e-12, max_outer=1, inner_rtol=1e-3)
    assert status == hp.HPCCG_ERR_NOT_CONVERGED and info.outer_iters == 1 and 1e-12 < info.relres < 1e-2
    # the inner iteration cap: at most max_inner x updates per cycle
    x, info, status = M.solve_mixed(b, np.zeros_like(b), 1, rel_tol=1e-8, max_outer=30, max_inner=3)
    assert status == hp.HPCCG_OK and info.inner_iters <= 3 * info.outer_iters


def test_fused_pass_entry_point_errors(hp, torch):
    """The fused-pass entry points reject what they cannot run: a stored-matrix
    context (no grid) has no fused iteration, a grid with nx % 4 != 0 neither;
    bad arguments are HPCCG_ERR_INVALID_ARG."""
    A, x, b, xe = oracle.generate_matrix(6, 5, 4)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    assert not M.mixed_fused()
    v = torch.zeros(A.nrow, dtype=torch.float32, device="cuda")
    with pytest.raises(hp.HpccgError) as e:
        M.mixed_pass(v, v.clone(), v.clone(), v.clone(), v.clone(), 0.5, 0.5, False)
    assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
    G = hp.Matrix.generated(6, 5, 4)  # nx % 4 != 0: the three-kernel iteration
    G.set_spmv(hp.SPMV_STENCIL)
    assert not G.mixed_fused()
    with pytest.raises(hp.HpccgError) as e:
        G.mixed_pass(v, v.clone(), v.clone(), v.clone(), v.clone(), 0.5, 0.5, False)
    assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
    H = hp.Matrix.generated(8, 5, 4)
    H.set_spmv(hp.SPMV_STENCIL)
    assert H.mixed_fused()
    with pytest.raises(hp.HpccgError) as e:
        hp._check(hp._lib.hpccg_gpu_set_mixed_fused(H._h, 2), "set_mixed_fused")
    assert e.value.code == hp.HPCCG_ERR_INVALID_ARG
    H.set_mixed_fused(False)
    assert not H.mixed_fused()
    H.set_mixed_fused(True)
    assert H.mixed_fused()


def test_fused_solve_non_cubic_partial_tiles(hp):
    """The fused inner iteration on a grid that fills no tile completely in x
    or y (40 x 70 x 9: tiles of 32 x 64), FP32 and BF16, against the oracle."""
    nx, ny, nz = 40, 70, 9
    A, x, b1, xe = oracle.generate_matrix(nx, ny, nz)
    xstar = oracle.uniform_pm1(77, A.nrow)
    b = oracle.spmv(A, xstar)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    M.set_geometry(nx, ny, nz)
    M.set_spmv(hp.SPMV_STENCIL)
    assert M.mixed_fused()
    for prec in (1, 2):
        xs, info, status = M.solve_mixed(b, np.zeros_like(b), prec, rel_tol=1e-8)
        assert status == hp.HPCCG_OK
        assert oracle.true_relres(A, b, xs) <= 1e-8
        assert np.abs(xs - xstar).max() <= 1e-7
