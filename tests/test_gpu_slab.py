"""Several ranks over z slabs on the GPU, checked against the oracle's multi-rank CG.

Every call in this suite has one GPU, so the ranks share it:
- ``group_cg``: all P ranks in one process (hpccg_slab_group_cg), the exchange
  by device copies between the ranks' buffers, sums folded in rank order;
- ``DistCG``: two processes on the same GPU joined by a gloo group, halos and
  dot products moving through torch.distributed (staged through host
  memory).  No kernel waits on another rank: the host orders every step.

Bars: the local SpMV (columns over own rows and externals) bit-exact against
the oracle's spmv on the renumbered CSR and against the single-rank matrix of
the stacked grid; pack and scatter bit-exact; CG residual histories within the
two-band 1e-12 bar of the single-rank tests, iteration counts equal, x within
1e-10 of the oracle's and of 1.  The oracle restates MPI/src/numerics.F90:41-162
with exchange_externals (MPI/src/SparseMatrix.F90:630-680 or
CAF-V2/src/SparseMatrix.F90:333-370) and rank-order sums.
"""
import os
import socket

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def zs():
    from hpccg_b200 import zslab
    return zslab


def _build(zs, nx, ny, nz, P, mode):
    plans, vals = [], []
    for r in range(P):
        rows, cols, v, *_ = zs.generate_matrix_rank(nx, ny, nz, r, P)
        plans.append(zs.SlabPlan(rows, cols, P, r, zs.first_rows_equal(nx * ny * nz, P), mode))
        vals.append(v)
    zs.exchange_plans_local(plans)
    return plans, [zs.Slab(p, v) for p, v in zip(plans, vals)]


def assert_history_parity(h_gpu, h_ref, rtol=1e-12, band=1e-8):
    assert len(h_gpu) == len(h_ref)
    r0 = h_ref[0]
    for k in range(len(h_ref)):
        bound = rtol * h_ref[k] if h_ref[k] >= band * r0 else rtol * r0
        assert abs(h_gpu[k] - h_ref[k]) <= bound, (k, h_gpu[k], h_ref[k])


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("nx,ny,nz,P", [(6, 5, 4, 3), (4, 4, 1, 3), (8, 3, 2, 2)])
def test_slab_spmv_pack_scatter(torch, zs, nx, ny, nz, P, mode):
    plans, slabs = _build(zs, nx, ny, nz, P, mode)
    G, _, _, _ = oracle.generate_matrix(nx, ny, nz * P)
    n = nx * ny * nz
    xg = oracle.uniform_pm1(5, n * P)
    yg = oracle.spmv(G, xg)
    ref = oracle.SlabPlan(nx, ny, nz, P, mode)
    for r, (plan, slab) in enumerate(zip(plans, slabs)):
        ids, _ = plan.externals()
        p = np.concatenate([xg[r * n:(r + 1) * n], xg[ids - 1]])
        dp = torch.from_numpy(p).cuda()
        dy = torch.zeros(n, dtype=torch.float64, device="cuda")
        slab.spmv(dp, dy)
        y = dy.cpu().numpy()
        A = oracle.Matrix(nx, ny, nz, ref.get(r, "rowindex"), ref.get(r, "colindex"),
                          oracle.generate_matrix_rank(nx, ny, nz, r, P)[0].values, ref.get(r, "nnz"))
        assert np.array_equal(y, oracle.spmv(A, p))  # the reference's spmv on the renumbered CSR
        assert np.array_equal(y, yg[r * n:(r + 1) * n])  # = the stacked single-rank matrix
        if mode == 0:
            _, ets = plan.sends()
            buf = torch.zeros(max(1, len(ets)), dtype=torch.float64, device="cuda")
            slab.pack(dp, buf)
            assert np.array_equal(buf.cpu().numpy()[:len(ets)], p[ets - 1])
        else:
            blk, rem = plan.blocks()
            dq = torch.from_numpy(np.concatenate([p[:n], np.zeros(len(ids))])).cuda()
            for b, (owner, start, lo, hi) in enumerate(blk):
                rng = torch.from_numpy(xg[owner * n + lo - 1: owner * n + hi].copy()).cuda()
                slab.scatter_block(b, rng, dq)
            assert np.array_equal(dq.cpu().numpy(), p)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("nx,ny,nz,P,iters", [(8, 6, 4, 2, 60), (6, 5, 4, 3, 60), (5, 4, 2, 4, 60),
                                              (6, 5, 1, 3, 40)])
def test_group_cg_matches_oracle(torch, zs, nx, ny, nz, P, iters, mode):
    """(6, 5, 1, 3): one plane per rank, so every row reaches both neighbours and the two
    halo forms order the externals differently; 40 iterations stay clear of the exact
    convergence of so small a system (after it the reference divides 0/0)."""
    plans, slabs = _build(zs, nx, ny, nz, P, mode)
    G, x0, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
    n = nx * ny * nz
    ref = oracle.SlabPlan(nx, ny, nz, P, mode)
    rx, rit, rnr, rh = ref.cg(bg, x0, iters, 0.0)
    assert np.all(np.isfinite(rh)) and rh[-1] > 0
    d_b = [torch.from_numpy(bg[r * n:(r + 1) * n].copy()).cuda() for r in range(P)]
    d_x = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(P)]
    it, nr, h, st = zs.group_cg(slabs, d_b, d_x, iters, 0.0)
    assert it == rit
    assert_history_parity(h, rh)
    x = np.concatenate([t.cpu().numpy() for t in d_x])
    assert np.abs(x - rx).max() <= 1e-10 and np.abs(x - 1.0).max() <= 1e-10
    # a tolerance stop (the reference's normr < tolerance at the top of an iteration)
    tol = 1e-8 * np.linalg.norm(bg)
    rx, rit, rnr, rh = ref.cg(bg, x0, iters, tol)
    for t in d_x:
        t.zero_()
    it, nr, h, st = zs.group_cg(slabs, d_b, d_x, iters, tol)
    assert it == rit and it < iters
    assert_history_parity(h, rh)
    assert nr == pytest.approx(rnr, rel=1e-12)
    for s in slabs:
        s.close()


def test_group_cg_one_rank_equals_single_context(torch, zs):
    """P = 1: no externals, no exchange; the same iterates as hpccg_gpu_cg."""
    import hpccg_b200 as hp

    plans, slabs = _build(zs, 7, 6, 5, 1, 0)
    A, x0, b, _ = oracle.generate_matrix(7, 6, 5)
    M = hp.Matrix.from_csr(A.rowindex, A.colindex, A.values)
    gx, it1, nr1, h1, _ = M.cg(b, x0.copy(), 50, 0.0)
    d_b, d_x = [torch.from_numpy(b).cuda()], [torch.zeros(len(b), dtype=torch.float64, device="cuda")]
    it, nr, h, st = zs.group_cg(slabs, d_b, d_x, 50, 0.0)
    assert it == it1
    assert_history_parity(h, h1)
    assert np.abs(d_x[0].cpu().numpy() - gx).max() <= 1e-12


# ---- two processes, one GPU, gloo -------------------------------------------------

def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dist_main(rank, P, port, nx, ny, nz, mode, max_iter, tol, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    from hpccg_b200 import zslab as zs

    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=P,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rows, cols, vals, x, b, xe = zs.generate_matrix_rank(nx, ny, nz, rank, P)
        plan = zs.SlabPlan(rows, cols, P, rank, zs.first_rows_equal(nx * ny * nz, P), mode)
        ranges = zs.exchange_plans_dist(plan)
        slab = zs.Slab(plan, vals)
        cg = zs.DistCG(slab, plan, get_ranges=ranges)
        d_b = torch.from_numpy(b).cuda()
        d_x = torch.zeros_like(d_b)
        it, nr, h = cg.solve(d_b, d_x, max_iter, tol)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), x=d_x.cpu().numpy(), it=it, nr=nr, h=h)
        slab.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", [0, 1])
def test_dist_cg_two_processes(tmp_path, zs, mode):
    import torch.multiprocessing as mp

    nx, ny, nz, P = 6, 5, 4, 2
    mp.start_processes(_dist_main, args=(P, _free_port(), nx, ny, nz, mode, 60, 0.0, str(tmp_path)), nprocs=P,
                       join=True, start_method="spawn")
    G, x0, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
    rx, rit, rnr, rh = oracle.SlabPlan(nx, ny, nz, P, mode).cg(bg, x0, 60, 0.0)
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(P)]
    for r in res:
        assert int(r["it"]) == rit
        assert_history_parity(r["h"], rh)
    x = np.concatenate([r["x"] for r in res])
    assert np.abs(x - rx).max() <= 1e-10
