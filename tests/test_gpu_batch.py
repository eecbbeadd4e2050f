"""Batched solves of independent systems (stacked, one persistent kernel per phase).

Bars: per system, the FP64 true residual recomputed by the CPU oracle meets
rel_tol; the FP64 batch takes the same iteration count as the oracle's CG to
the same residual (+-1 for a borderline stop); the iterates do not depend on
the tile schedule (bit-identical); CSR input equals generated input.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

FP64, FP32, BF16 = 0, 1, 2
SIZES = [(3, 5, 7), (16, 16, 16), (1, 1, 1), (20, 9, 13), (12, 12, 12), (2, 2, 2), (31, 17, 5)]


@pytest.fixture(scope="module")
def hp():
    import hpccg_b200
    return hpccg_b200


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def _systems(sizes, seed=7):
    out = []
    for s, (nx, ny, nz) in enumerate(sizes):
        A, x, b1, xe = oracle.generate_matrix(nx, ny, nz)
        xs = oracle.uniform_pm1(seed + s, A.nrow)
        out.append((A, oracle.spmv(A, xs), xs))
    return out


def _oracle_iters(A, b, rel_tol):
    """Iterations plain CG needs for ||r_j|| <= rel_tol ||b|| (the reference's hist[j+1] = ||r_j||)."""
    _, it, _, hist = oracle.cg(A, b, np.zeros_like(b), 500, 0.0)
    tol = rel_tol * np.linalg.norm(b)
    r = hist[1:]  # r[j] = ||r_j||
    hit = np.nonzero(~(r > tol))[0]
    return int(hit[0]) if len(hit) else None


@pytest.mark.parametrize("prec", [FP64, FP32, BF16])
def test_batch_solve_per_system(hp, torch, prec):
    sysl = _systems(SIZES)
    B = hp.Batch.generated(SIZES)
    assert B.nsys == len(SIZES) and list(B.nrows) == [a * b * c for a, b, c in SIZES]
    assert all(o % 512 == 0 for o in B.offsets)
    db = torch.from_numpy(B.stack([b for _, b, _ in sysl])).cuda()
    dx = torch.zeros_like(db)
    iters, relres, outer, st = B.solve(db, dx, prec, 1e-8, 1000)
    assert st == hp.HPCCG_OK
    xs = B.unstack(dx.cpu().numpy())
    for s, (A, b, xstar) in enumerate(sysl):
        rel = oracle.true_relres(A, b, xs[s])
        assert rel <= 1e-8, (s, rel)
        assert relres[s] == pytest.approx(rel, rel=1e-6, abs=1e-15)
        assert np.abs(xs[s] - xstar).max() <= 1e-6
        if prec == FP64:
            want = _oracle_iters(A, b, 1e-8)
            assert want is not None and abs(int(iters[s]) - want) <= 1, (s, iters[s], want)
        else:
            assert outer[s] >= 1


def test_batch_schedule_independent(hp, torch):
    sysl = _systems(SIZES)
    B = hp.Batch.generated(SIZES)
    db = torch.from_numpy(B.stack([b for _, b, _ in sysl])).cuda()
    ref = None
    for sched in [(1, 2), (4, 4), (8, 8), (2, 3)]:
        B.set_schedule(*sched)
        assert B.get_schedule() == sched
        for prec in (FP64, BF16):
            dx = torch.zeros_like(db)
            iters, relres, outer, st = B.solve(db, dx, prec, 1e-8, 1000)
            got = (dx.cpu().numpy(), iters.copy())
            if ref is None:
                ref = {}
            if prec in ref:
                assert np.array_equal(got[0], ref[prec][0]) and np.array_equal(got[1], ref[prec][1]), sched
            else:
                ref[prec] = got
    B.set_schedule(0, 0)  # back to the autotuner
    dx = torch.zeros_like(db)
    B.solve(db, dx, FP64, 1e-8, 1000)
    assert np.array_equal(dx.cpu().numpy(), ref[FP64][0])


def test_batch_from_csr_equals_generated(hp, torch):
    sizes = SIZES[:4]
    sysl = _systems(sizes)
    G = hp.Batch.generated(sizes)
    C = hp.Batch.from_csr([(A.rowindex, A.colindex, A.values) for A, _, _ in sysl])
    assert list(C.offsets) == list(G.offsets)
    db = torch.from_numpy(G.stack([b for _, b, _ in sysl])).cuda()
    out = []
    for B in (G, C):
        dx = torch.zeros_like(db)
        B.solve(db, dx, FP64, 1e-8, 1000)
        out.append(dx.cpu().numpy())
    assert np.array_equal(out[0], out[1])


def test_batch_spmv_bit_exact(hp, torch):
    sysl = _systems(SIZES)
    B = hp.Batch.generated(SIZES)
    dx = torch.from_numpy(B.stack([xs for _, _, xs in sysl])).cuda()
    dy = torch.empty_like(dx)
    B.spmv(dx, dy)
    ys = B.unstack(dy.cpu().numpy())
    for s, (A, b, xs) in enumerate(sysl):
        assert np.array_equal(ys[s], b)


def test_batch_iteration_cap_reports_not_converged(hp, torch):
    sysl = _systems(SIZES[:2])
    B = hp.Batch.generated(SIZES[:2])
    db = torch.from_numpy(B.stack([b for _, b, _ in sysl])).cuda()
    dx = torch.zeros_like(db)
    iters, relres, outer, st = B.solve(db, dx, FP64, 1e-8, 3)
    assert st == hp.HPCCG_ERR_NOT_CONVERGED
    assert iters.max() <= 3 and relres.max() > 1e-8


def test_batch_eager_equals_graph(hp, torch, monkeypatch):
    sysl = _systems(SIZES[:3])
    B = hp.Batch.generated(SIZES[:3])
    db = torch.from_numpy(B.stack([b for _, b, _ in sysl])).cuda()
    res = []
    for eager in ("0", "1"):
        monkeypatch.setenv("HPCCG_EAGER", eager)
        for prec in (FP64, FP32):
            dx = torch.zeros_like(db)
            B.solve(db, dx, prec, 1e-8, 1000)
            res.append(dx.cpu().numpy())
    assert np.array_equal(res[0], res[2]) and np.array_equal(res[1], res[3])


def test_batch_stencil_bit_identical_to_ell(hp, torch):
    """Matrix-free rows (generated batches) give the ELL batch's FP64 iterates
    bit for bit; the FP32 refinement meets the FP64 target per system; a batch
    built from CSR refuses the stencil.  The column walks split z into 32-plane
    chunks: systems with nz > 32 and nz not a multiple of 32 (70, 65, 40, 33)
    run the chunks that start past plane 0 and the ragged last chunk, and
    40 x 36 planes have interior warps (32 columns off every face)."""
    sizes = [(3, 5, 7), (16, 16, 16), (1, 1, 1), (20, 9, 13), (2, 2, 2), (31, 17, 5),
             (20, 9, 70), (3, 2, 65), (1, 1, 40), (40, 36, 33)]
    B = hp.Batch.generated(sizes)
    xs = B.stack([oracle.uniform_pm1(11 + s, int(B.nrows[s])) for s in range(B.nsys)])
    d_xs = torch.from_numpy(xs).cuda()
    y_ell, y_st = torch.empty_like(d_xs), torch.empty_like(d_xs)
    B.spmv(d_xs, y_ell)
    B.set_spmv(hp.SPMV_STENCIL)
    B.spmv(d_xs, y_st)
    for u, v in zip(B.unstack(y_ell.cpu().numpy()), B.unstack(y_st.cpu().numpy())):  # real rows only
        assert np.array_equal(u.view(np.int64), v.view(np.int64))
    d_b = torch.from_numpy(B.stack(B.unstack(y_ell.cpu().numpy()))).cuda()  # zero gaps
    runs = {}
    for kind in (hp.SPMV_ELL, hp.SPMV_STENCIL):
        B.set_spmv(kind)
        d_x = torch.zeros_like(d_b)
        iters, relres, outer, rc = B.solve(d_b, d_x, FP64, 1e-10)
        assert rc == hp.HPCCG_OK
        runs[kind] = (iters.copy(), relres.copy(), d_x.cpu().numpy())
    assert np.array_equal(runs[hp.SPMV_ELL][0], runs[hp.SPMV_STENCIL][0])
    for u, v in zip(B.unstack(runs[hp.SPMV_ELL][2]), B.unstack(runs[hp.SPMV_STENCIL][2])):
        assert np.array_equal(u.view(np.int64), v.view(np.int64))
    B.set_spmv(hp.SPMV_STENCIL)
    d_x = torch.zeros_like(d_b)
    iters, relres, outer, rc = B.solve(d_b, d_x, FP32, 1e-8)
    assert rc == hp.HPCCG_OK and np.all(relres <= 1e-8)
    for s in range(B.nsys):
        A, _, _, _ = oracle.generate_matrix(*sizes[s])
        xs_s = d_x.cpu().numpy()[B.offsets[s]:B.offsets[s] + B.nrows[s]]
        bs = d_b.cpu().numpy()[B.offsets[s]:B.offsets[s] + B.nrows[s]]
        assert oracle.true_relres(A, bs, xs_s) <= 1e-8 * (1 + 1e-6), s  # device and oracle sums differ ~1e-15
    A4 = oracle.generate_matrix(4, 4, 4)[0]
    Bc = hp.Batch.from_csr([(A4.rowindex, A4.colindex, A4.values)])
    with pytest.raises(hp.HpccgError) as e:
        Bc.set_spmv(hp.SPMV_STENCIL)
    assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
