"""Several ranks over z slabs: the host half, on the CPU.

- The rank generator (MPI/src/SparseMatrix.F90:68-185 with start_row, :112)
  matches the oracle's, and the ranks' rows stacked are the single-rank
  matrix of the nx x ny x (nz*P) grid.
- Every rank's halo plan (make_local_matrix, MPI/src/SparseMatrix.F90:235-627;
  CAF-V2/src/SparseMatrix.F90:205-331) matches the oracle's restatement list
  by list: renumbered columns, externals and owners, neighbours, block
  lengths, send lists; blocks and owner-local rows in the GET form.  Built in
  one process, and on gloo ranks (world sizes 2 and 3) whose plans exchange
  their requests through torch.distributed as the reference's ranks do
  through MPI.
- The oracle's multi-rank CG against its single-rank CG on the stacked grid.
- DistCG's transport (halo messages, rank-order sums of the dot products) on
  gloo ranks of world sizes 2 and 3, each rank's CG steps in host memory
  (HostSlab, a restatement of the step contract): the whole solve equals the
  oracle's multi-rank CG bit for bit.
- The reference's block-length count (:533-545), restated literally, is one
  too large for every block but the last: right for two ranks, off by one for
  the middle ranks of three -- the reason the plans use the block sizes.

Integer and index results are compared exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import hpccg_b200 as hp
import oracle
from hpccg_b200 import zslab

CASES = [(4, 3, 2, 2), (4, 3, 2, 3), (5, 4, 3, 4), (3, 3, 1, 3), (1, 1, 4, 2), (6, 2, 1, 2), (2, 5, 3, 1)]


def _plans(nx, ny, nz, P, mode):
    plans = []
    for r in range(P):
        rows, cols, vals, *_ = zslab.generate_matrix_rank(nx, ny, nz, r, P)
        plans.append(zslab.SlabPlan(rows, cols, P, r, zslab.first_rows_equal(nx * ny * nz, P), mode))
    zslab.exchange_plans_local(plans)
    return plans


def _compare(plan, ref, r, mode):
    np.testing.assert_array_equal(plan.colindex_local(), ref.get(r, "colindex"))
    ids, owners = plan.externals()
    np.testing.assert_array_equal(ids, ref.get(r, "externals"))
    np.testing.assert_array_equal(owners, ref.get(r, "external_owners"))
    if mode == zslab.HALO_MPI:
        nb, rl = plan.neighbors()
        np.testing.assert_array_equal(nb, ref.get(r, "neighbors"))
        np.testing.assert_array_equal(rl, ref.get(r, "recv_length"))
        sl, ets = plan.sends()
        np.testing.assert_array_equal(sl, ref.get(r, "send_length"))
        np.testing.assert_array_equal(ets, ref.get(r, "elements_to_send"))
    else:
        blk, rem = plan.blocks()
        np.testing.assert_array_equal(blk, ref.get(r, "blocks"))
        np.testing.assert_array_equal(rem, ref.get(r, "remote_index"))


@pytest.mark.parametrize("nx,ny,nz,P", CASES)
def test_rank_generator_matches_oracle_and_stacks(nx, ny, nz, P):
    G, _, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
    cols, vals, bs, rows_off = [], [], [], 0
    for r in range(P):
        rows, c, v, x, b, xe = zslab.generate_matrix_rank(nx, ny, nz, r, P)
        A, ox, ob, oxe = oracle.generate_matrix_rank(nx, ny, nz, r, P)
        np.testing.assert_array_equal(rows, A.rowindex)
        np.testing.assert_array_equal(c, A.colindex)
        np.testing.assert_array_equal(v, A.values)
        np.testing.assert_array_equal(b, ob)
        assert np.all(x == 0) and np.all(xe == 1)
        cols.append(c), vals.append(v), bs.append(b)
    np.testing.assert_array_equal(np.concatenate(cols), G.colindex)
    np.testing.assert_array_equal(np.concatenate(vals), G.values)
    np.testing.assert_array_equal(np.concatenate(bs), bg)


@pytest.mark.parametrize("mode", [zslab.HALO_MPI, zslab.HALO_GET])
@pytest.mark.parametrize("nx,ny,nz,P", CASES)
def test_plans_match_oracle(nx, ny, nz, P, mode):
    ref = oracle.SlabPlan(nx, ny, nz, P, mode)
    for r, plan in enumerate(_plans(nx, ny, nz, P, mode)):
        _compare(plan, ref, r, mode)


def test_reference_block_length_count():
    """The literal count of MPI/src/SparseMatrix.F90:533-545 against the block sizes."""
    two = oracle.SlabPlan(4, 3, 2, 2, oracle.HALO_MPI)
    for r in range(2):
        np.testing.assert_array_equal(two.get(r, "recv_length_literal"), two.get(r, "recv_length"))
    three = oracle.SlabPlan(4, 3, 2, 3, oracle.HALO_MPI)
    np.testing.assert_array_equal(three.get(1, "recv_length"), [12, 12])
    np.testing.assert_array_equal(three.get(1, "recv_length_literal"), [13, 12])  # first block one too long
    for r in (0, 2):
        np.testing.assert_array_equal(three.get(r, "recv_length_literal"), three.get(r, "recv_length"))


def test_plan_rejects_bad_input():
    rows, cols, vals, *_ = zslab.generate_matrix_rank(3, 3, 2, 0, 2)
    fr = zslab.first_rows_equal(18, 2)
    bad = cols.copy()
    bad[0] = 37  # beyond the 36 rows of two slabs
    with pytest.raises(hp.HpccgError):
        zslab.SlabPlan(rows, bad, 2, 0, fr)
    plan = zslab.SlabPlan(rows, cols, 2, 0, fr)
    with pytest.raises(hp.HpccgError):
        plan.set_sends({1: np.array([19], np.int32)})  # rank 0 owns rows 1..18 only


@pytest.mark.parametrize("nx,ny,nz,P", [(4, 3, 2, 2), (4, 3, 2, 3), (3, 3, 1, 4), (5, 2, 3, 1)])
def test_oracle_slab_cg_matches_single_rank(nx, ny, nz, P):
    G, x0, b, _ = oracle.generate_matrix(nx, ny, nz * P)
    _, it1, nr1, h1 = oracle.cg(G, b, x0, 30, 0.0)
    runs = []
    for mode in (oracle.HALO_MPI, oracle.HALO_GET):
        x, it, nr, h = oracle.SlabPlan(nx, ny, nz, P, mode).cg(b, x0, 30, 0.0)
        runs.append((x, h))
        assert it == it1
        r0 = h1[0]
        for k in range(len(h1)):  # only the dot products' association differs
            bound = 1e-12 * (h1[k] if h1[k] >= 1e-8 * r0 else r0)
            assert abs(h[k] - h1[k]) <= bound or (np.isnan(h[k]) and np.isnan(h1[k])), (mode, k)
        if P == 1:
            np.testing.assert_array_equal(h, h1)
    # the two halo forms fetch the same values: identical iterates
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


# ---- gloo ranks ----------------------------------------------------------------

def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, P, port, nx, ny, nz, mode, out_dir):
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=P,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rows, cols, vals, *_ = zslab.generate_matrix_rank(nx, ny, nz, rank, P)
        # global_index_offsets by an allreduce of each rank's first row (:318-324)
        import torch

        t = torch.zeros(P, dtype=torch.int64)
        t[rank] = nx * ny * nz * rank + 1
        dist.all_reduce(t)
        fr = np.append(t.numpy(), nx * ny * nz * P + 1).astype(np.int32)
        plan = zslab.SlabPlan(rows, cols, P, rank, fr, mode)
        ranges = zslab.exchange_plans_dist(plan)
        res = {"colindex": plan.colindex_local(), "externals": plan.externals()[0],
               "owners": plan.externals()[1]}
        if mode == zslab.HALO_MPI:
            res["neighbors"], res["recv_length"] = plan.neighbors()
            res["send_length"], res["elements_to_send"] = plan.sends()
        else:
            res["blocks"], res["remote_index"] = plan.blocks()
            served = sorted((q, lo, hi) for q, rr in ranges.items() for lo, hi in rr)
            res["served"] = np.array(served, np.int32).reshape(-1, 3)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **res)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", [zslab.HALO_MPI, zslab.HALO_GET])
@pytest.mark.parametrize("nx,ny,nz,P", [(4, 3, 2, 2), (3, 2, 2, 3), (3, 3, 1, 3)])
def test_plans_over_gloo_ranks(tmp_path, nx, ny, nz, P, mode):
    mp.start_processes(_rank_main, args=(P, _free_port(), nx, ny, nz, mode, str(tmp_path)), nprocs=P,
                       join=True, start_method="spawn")
    ref = oracle.SlabPlan(nx, ny, nz, P, mode)
    for r in range(P):
        got = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_array_equal(got["colindex"], ref.get(r, "colindex"))
        np.testing.assert_array_equal(got["externals"], ref.get(r, "externals"))
        np.testing.assert_array_equal(got["owners"], ref.get(r, "external_owners"))
        if mode == zslab.HALO_MPI:
            for k in ("neighbors", "recv_length", "send_length", "elements_to_send"):
                np.testing.assert_array_equal(got[k], ref.get(r, k))
        else:
            np.testing.assert_array_equal(got["blocks"], ref.get(r, "blocks"))
            np.testing.assert_array_equal(got["remote_index"], ref.get(r, "remote_index"))
            # each rank serves exactly the ranges the other ranks' blocks name
            want = sorted((q, int(lo), int(hi)) for q in range(P) for own, _s, lo, hi in ref.get(q, "blocks")
                          if own == r)
            np.testing.assert_array_equal(got["served"], np.array(want, np.int32).reshape(-1, 3))


# ---- DistCG's transport on gloo ranks, with the CG steps in host memory -------

class HostSlab:
    """One rank's CG steps in host memory, restating the contract of hpccg_slab_cg_step,
    hpccg_slab_pack and hpccg_slab_scatter_block (include/hpccg_gpu.h) with the operations of
    MPI/src/numerics.F90:41-162 and vector_operations.F90:40-169: separately rounded products
    and sums, row sums in CSR order and dot products in index order, both from 0.0.  With it,
    DistCG's exchanges and rank-order sums run on gloo ranks without a GPU, and the whole
    solve must equal the oracle's multi-rank CG bit for bit.  Test infrastructure only."""

    def __init__(self, plan, rowindex, values):
        info = plan.info()
        self.nranks, self.mode = plan.nranks, plan.mode
        self.nrow = len(rowindex) - 1
        self.ncol = self.nrow + info["num_external"]
        self.nsend = info["total_to_send"]
        self.neighbors, self.recv_length = plan.neighbors()
        if plan.mode == zslab.HALO_MPI:
            self.send_length, idx = plan.sends()
            self.send_idx = idx.astype(np.int64) - 1  # elements_to_send, 1-based local rows
            self.blocks = np.zeros((0, 4), np.int32)
        else:
            self.send_length = np.zeros(0, np.int32)
            self.blocks, remote = plan.blocks()
            self.remote = remote.astype(np.int64)  # owner-local rows, 1-based
        # the local CSR as rows padded at their ends with zero terms (which leave a row sum unchanged)
        cl = plan.colindex_local().astype(np.int64) - 1
        lens = np.diff(rowindex)
        w = int(lens.max())
        self.col = np.zeros((self.nrow, w), np.int64)
        self.val = np.zeros((self.nrow, w))
        for i in range(self.nrow):
            a, e = rowindex[i] - 1, rowindex[i + 1] - 1
            self.col[i, :e - a], self.val[i, :e - a] = cl[a:e], values[a:e]

    def _spmv(self, x):
        y = np.zeros(self.nrow)
        for j in range(self.col.shape[1]):
            y = y + self.val[:, j] * x[self.col[:, j]]
        return y

    @staticmethod
    def _dot(a, b):
        return float(np.add.accumulate(np.concatenate(([0.0], a * b)))[-1])

    def pack(self, d_x, d_sendbuf):
        d_sendbuf.numpy()[:self.nsend] = d_x.numpy()[self.send_idx]

    def scatter_block(self, block, d_range, d_x):
        _owner, first, inmin, _inmax = (int(v) for v in self.blocks[block])
        end = int(self.blocks[block + 1][1]) if block + 1 < len(self.blocks) else self.ncol - self.nrow + 1
        d_x.numpy()[self.nrow + first - 1:self.nrow + end - 1] = d_range.numpy()[self.remote[first - 1:end - 1] - inmin]

    def step(self, step, k, d_b, d_x, d_p, d_r, d_Ap, d_state, d_hist=None):
        st, x, p, r, Ap = d_state.numpy(), d_x.numpy(), d_p.numpy(), d_r.numpy(), d_Ap.numpy()
        h = d_hist.numpy() if d_hist is not None else None
        n = self.nrow
        L, G, RT, NR, BE, DN, TL = (zslab.LOCAL, zslab.GLOBAL, zslab.RTRANS, zslab.NORMR, zslab.BETA, zslab.DONE,
                                    zslab.TOL)
        if step == zslab.START:
            p[:n] = x
        elif step == zslab.PREPARE:  # Ap = A p, r = 1 b + (-1) Ap (:96), local r.r
            Ap[:] = self._spmv(p)
            r[:] = 1.0 * d_b.numpy() + (-1.0) * Ap
            st[L] = self._dot(r, r)
        elif step == zslab.PREPARED:
            st[RT] = st[G]
            st[NR] = np.sqrt(st[RT])
            st[DN] = 0.0
            if h is not None:
                h[0] = st[NR]
        elif step == zslab.BEGIN:  # stop test on the previous normr; p = r, or beta and p = r + beta p
            if st[DN] != 0.0:
                return
            if st[NR] < st[TL]:
                st[DN] = 1.0
                return
            beta, rtrans = 0.0, st[RT]
            if k > 1:
                rtrans = st[G]
                beta = rtrans / st[RT]
            p[:n] = r if k == 1 else r + beta * p[:n]
            st[BE] = beta
            if h is not None:
                h[k] = np.sqrt(rtrans)
            if k > 1:
                st[RT] = st[G]
            st[NR] = np.sqrt(st[RT])
        elif step == zslab.SPMV:
            if st[DN] == 0.0:
                Ap[:] = self._spmv(p)
                st[L] = self._dot(p[:n], Ap)
        elif step == zslab.UPDATE:  # alpha = rtrans / p.Ap; r -= alpha Ap; x += alpha p; local r.r
            if st[DN] == 0.0:
                alpha = st[RT] / st[G]
                r[:] = r + (-alpha) * Ap
                x[:] = x + alpha * p[:n]
                st[L] = self._dot(r, r)


def _dist_cg_main(rank, P, rdv, nx, ny, nz, mode, max_iter, tol, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"file://{rdv}", rank=rank, world_size=P,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rows, cols, vals, x, b, _ = zslab.generate_matrix_rank(nx, ny, nz, rank, P)
        plan = zslab.SlabPlan(rows, cols, P, rank, zslab.first_rows_equal(nx * ny * nz, P), mode)
        ranges = zslab.exchange_plans_dist(plan)
        cg = zslab.DistCG(HostSlab(plan, rows, vals), plan, get_ranges=ranges, device="cpu")
        d_b, d_x = torch.from_numpy(b.copy()), torch.zeros(len(b), dtype=torch.float64)
        it, nr, h = cg.solve(d_b, d_x, max_iter, tol)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), x=d_x.numpy(), it=it, nr=nr, h=h)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", [zslab.HALO_MPI, zslab.HALO_GET])
@pytest.mark.parametrize("nx,ny,nz,P,max_iter,tol", [(4, 3, 2, 2, 40, 0.0), (3, 4, 2, 3, 40, 0.0),
                                                     (3, 3, 1, 4, 40, 0.0), (5, 3, 2, 3, 150, 1e-6)])
def test_dist_cg_transport_over_gloo_ranks(tmp_path, nx, ny, nz, P, max_iter, tol, mode):
    """DistCG (one rank per process, halos by point-to-point messages, dot products by an
    all-gather folded in rank order) on 2-4 gloo ranks (one-plane slabs among them), every rank's CG steps in host memory:
    the iterates, iteration count, final normr and residual history equal the oracle's
    multi-rank CG exactly, in the MPI and the CAF-V2 halo form, with tolerance 0 and with a
    tolerance that stops the loop early."""
    mp.start_processes(_dist_cg_main, args=(P, str(tmp_path / "rdv"), nx, ny, nz, mode, max_iter, tol, str(tmp_path)),
                       nprocs=P, join=True, start_method="spawn")
    _, x0, bg, _ = oracle.generate_matrix(nx, ny, nz * P)
    rx, rit, rnr, rh = oracle.SlabPlan(nx, ny, nz, P, mode).cg(bg, x0, max_iter, tol)
    if tol > 0:
        assert rit < max_iter  # the tolerance ends the loop
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(P)]
    for r in res:
        assert int(r["it"]) == rit and float(r["nr"]) == rnr
        np.testing.assert_array_equal(r["h"], rh)
    np.testing.assert_array_equal(np.concatenate([r["x"] for r in res]), rx)


# ---- a rank that leaves between steps --------------------------------------------

class _LeftEarly(Exception):
    pass


def _dist_cg_leaver_main(rank, P, rdv, how, out_dir):
    import datetime
    import json
    import time

    import torch
    import torch.distributed as dist

    timeout_s = 5
    dist.init_process_group("gloo", init_method=f"file://{rdv}", rank=rank, world_size=P,
                            timeout=datetime.timedelta(seconds=timeout_s))
    nx, ny, nz = 4, 3, 2
    rows, cols, vals, x, b, _ = zslab.generate_matrix_rank(nx, ny, nz, rank, P)
    plan = zslab.SlabPlan(rows, cols, P, rank, zslab.first_rows_equal(nx * ny * nz, P), zslab.HALO_MPI)
    ranges = zslab.exchange_plans_dist(plan)
    slab = HostSlab(plan, rows, vals)
    if rank == P - 1:  # the last rank leaves at the top of iteration 3, between two steps
        inner = slab.step

        def step(s, k, *a, **kw):
            if s == zslab.BEGIN and k == 3:
                raise _LeftEarly()
            return inner(s, k, *a, **kw)

        slab.step = step
    cg = zslab.DistCG(slab, plan, get_ranges=ranges, device="cpu")
    d_b, d_x = torch.from_numpy(b.copy()), torch.zeros(len(b), dtype=torch.float64)
    t0, status = time.time(), "finished"
    try:
        cg.solve(d_b, d_x, 40, 0.0)
    except _LeftEarly:
        status = "left"
        if how == "stay":  # alive, but takes no further part until the others' timeout has passed
            time.sleep(timeout_s + 2)
    except RuntimeError as e:
        status = "error: " + str(e)[:200]
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"status": status, "seconds": time.time() - t0}, f)
    if status != "left" or how == "exit":
        dist.destroy_process_group()


@pytest.mark.parametrize("how", ["exit", "stay"])
def test_dist_cg_rank_leaving_between_steps_raises_on_the_others(tmp_path, how):
    """Failure detection on the host: one of three gloo ranks leaves DistCG at the top of
    iteration 3, between two steps, and either exits or stays alive without taking part.  The
    other ranks (its z neighbour and the rank beyond it) get an error from their next transfer
    -- at once when the peer's connection closes; when it stays silent, the first of them to
    give up does so on the process group's 5 s timeout, and the rest then on that timeout or
    on the closed connection of the rank that gave up -- instead of waiting for ever."""
    import json

    P = 3
    mp.start_processes(_dist_cg_leaver_main, args=(P, str(tmp_path / "rdv"), how, str(tmp_path)), nprocs=P, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(P)]
    assert res[P - 1]["status"] == "left"
    for r in res[:P - 1]:
        assert r["status"].startswith("error"), r
        assert r["seconds"] < 5 + 20, r
        if how == "stay":
            assert r["seconds"] >= 4.5, r
    if how == "stay":
        assert any("Timed out" in r["status"] for r in res[:P - 1]), res
