"""Several ranks over z slabs of the weak-scaled HPCCG problem, over the C-ABI.

Rank r of P owns the rows local_nrow*r+1 .. local_nrow*(r+1) of the
nx x ny x (nz*P) grid (MPI/src/SparseMatrix.F90:68-185), renumbers its columns
into own rows followed by externals (make_local_matrix, :235-627), fills p's
externals before every SpMV (exchange_externals, :630-680) and sums every dot
product over the ranks (MPI/src/vector_operations.F90:64-65, 96-97).

- ``SlabPlan``: one rank's halo plan (host only), in the MPI form (send lists)
  or the CAF-V2 form (one contiguous range per block of one owner,
  CAF-V2/src/SparseMatrix.F90:205-370).
- ``exchange_plans_local`` / ``exchange_plans_dist``: the messages of
  make_local_matrix -- each rank tells each neighbour which of its rows it
  needs -- between plans in this process, or between processes through
  torch.distributed.
- ``Slab`` + ``group_cg``: every rank in this process, the whole CG in the
  library (device copies for the exchange, rank-order sums).
- ``DistCG``: one rank per process; the library's CG steps with
  torch.distributed moving halos and summing dots (NCCL moves device tensors;
  gloo stages them through host memory).

Sums over ranks are left folds in rank order, so they match the oracle's for
any P (for P = 2 there is only one order).
"""
from __future__ import annotations

import ctypes as _c

import numpy as np

from . import HPCCG_OK, HPCCG_ERR_BREAKDOWN, _check, _dptr, _lib, _sync_torch

HALO_MPI, HALO_GET = 0, 1
START, PREPARE, PREPARED, BEGIN, SPMV, UPDATE = range(6)
# d_state layout of hpccg_slab_cg_step
LOCAL, GLOBAL, RTRANS, NORMR, ALPHA, BETA, DONE, TOL = range(8)


def generate_matrix_rank(nx: int, ny: int, nz: int, rank: int, nranks: int):
    """generate_matrix on rank `rank` of `nranks`: (rowindex, colindex, values, x, b, xexact),
    1-based with global columns."""
    n = nx * ny * nz
    rowindex = np.zeros(n + 1, np.int32)
    colindex = np.zeros(27 * n, np.int32)
    values = np.zeros(27 * n, np.float64)
    x, b, xexact = np.empty(n), np.empty(n), np.empty(n)
    nnz = _c.c_int64(0)
    _check(_lib.hpccg_generate_matrix_rank(nx, ny, nz, rank, nranks, rowindex, colindex, values, x, b, xexact,
                                           _c.byref(nnz)), "generate_matrix_rank")
    k = nnz.value
    return rowindex, colindex[:k].copy(), values[:k].copy(), x, b, xexact


def first_rows_equal(local_nrow: int, nranks: int) -> np.ndarray:
    """first_rows for equal slabs: rank q starts at local_nrow*q + 1 (:112)."""
    return (np.arange(nranks + 1, dtype=np.int64) * local_nrow + 1).astype(np.int32)


def _i32buf(n):
    return np.zeros(max(1, n), np.int32)


class SlabPlan:
    """One rank's halo plan (hpccg_slab_plan_*): host memory only."""

    def __init__(self, rowindex, colindex, nranks: int, rank: int, first_rows, mode: int = HALO_MPI):
        self.rowindex = np.ascontiguousarray(rowindex, np.int32)
        colindex = np.ascontiguousarray(colindex, np.int32)
        self.nrow = len(self.rowindex) - 1
        self.nnz = len(colindex)
        self.nranks, self.rank, self.mode = nranks, rank, mode
        self.first_rows = np.ascontiguousarray(first_rows, np.int32)
        h = _c.c_void_p()
        _check(_lib.hpccg_slab_plan_create(self.nrow, self.nnz, self.rowindex, colindex, nranks, rank,
                                           self.first_rows, mode, _c.byref(h)), "slab_plan_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.hpccg_slab_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        v = [_c.c_int32(0) for _ in range(4)]
        _check(_lib.hpccg_slab_plan_info(self._h, *[_c.byref(a) for a in v]), "slab_plan_info")
        return {"num_external": v[0].value, "num_neighbors": v[1].value, "num_blocks": v[2].value,
                "total_to_send": v[3].value}

    def neighbors(self):
        n = self.info()["num_neighbors"]
        nb, ln = _i32buf(n), _i32buf(n)
        _check(_lib.hpccg_slab_plan_neighbors(self._h, nb.ctypes.data, ln.ctypes.data), "slab_plan_neighbors")
        return nb[:n], ln[:n]

    def externals(self):
        n = self.info()["num_external"]
        g, o = _i32buf(n), _i32buf(n)
        _check(_lib.hpccg_slab_plan_externals(self._h, g.ctypes.data, o.ctypes.data), "slab_plan_externals")
        return g[:n], o[:n]

    def requests(self):
        """MPI form: {neighbour: global ids it must send here, in the order they land}."""
        ids, owners = self.externals()
        nb, _ = self.neighbors()
        return {int(q): ids[owners == q].copy() for q in nb}

    def set_sends(self, requested):
        """MPI form: requested = {neighbour: global ids it asked this rank for}."""
        nb, _ = self.neighbors()
        lens = np.array([len(requested.get(int(q), ())) for q in nb], np.int32)
        ids = (np.concatenate([np.asarray(requested.get(int(q), ()), np.int32) for q in nb])
               if len(nb) else np.zeros(0, np.int32))
        ids = np.ascontiguousarray(ids, np.int32)
        _check(_lib.hpccg_slab_plan_set_sends(self._h, _i32buf(0).ctypes.data if not len(lens) else lens.ctypes.data,
                                              _i32buf(0).ctypes.data if not len(ids) else ids.ctypes.data),
               "slab_plan_set_sends")

    def sends(self):
        inf = self.info()
        nb, _ = self.neighbors()
        lens, idx = _i32buf(len(nb)), _i32buf(inf["total_to_send"])
        _check(_lib.hpccg_slab_plan_sends(self._h, lens.ctypes.data, idx.ctypes.data), "slab_plan_sends")
        return lens[:len(nb)], idx[:inf["total_to_send"]]

    def colindex_local(self):
        out = _i32buf(self.nnz)
        _check(_lib.hpccg_slab_plan_colindex(self._h, out.ctypes.data), "slab_plan_colindex")
        return out[:self.nnz]

    def blocks(self):
        inf = self.info()
        nb, ne = inf["num_blocks"], inf["num_external"]
        blk, rem = _i32buf(4 * nb), _i32buf(ne)
        _check(_lib.hpccg_slab_plan_blocks(self._h, blk.ctypes.data, rem.ctypes.data), "slab_plan_blocks")
        return blk[:4 * nb].reshape(nb, 4), rem[:ne]


def exchange_plans_local(plans):
    """The make_local_matrix messages between plans of one process: every rank gets, from
    each neighbour, the ids that neighbour needs from it (MPI form; a no-op for GET)."""
    for p in plans:
        if p.mode != HALO_MPI:
            continue
        asked = {}
        for q in p.neighbors()[0]:
            asked[int(q)] = plans[int(q)].requests().get(p.rank, np.zeros(0, np.int32))
        p.set_sends(asked)


def exchange_plans_dist(plan: SlabPlan, group=None):
    """The make_local_matrix messages through torch.distributed (MPI/src/SparseMatrix.F90:
    563-604): each rank sends every neighbour the global ids it needs from it and receives
    theirs.  GET form: each rank sends each owner the [inmin, inmax] ranges it will fetch,
    so the owner can serve them (a two-sided transport has no one-sided get).  Counts are
    sent first, as the reference does.  Returns, for GET, {requester: [(inmin, inmax), ..]}."""
    import torch
    import torch.distributed as dist

    def swap(peers, payload):  # payload: {peer: int32 array}; returns {peer: int32 array}
        ops, counts_in = [], {}
        for q in peers:
            c = torch.tensor([len(payload[q])], dtype=torch.int64)
            counts_in[q] = torch.zeros(1, dtype=torch.int64)
            ops.append(dist.P2POp(dist.isend, c, q, group))
            ops.append(dist.P2POp(dist.irecv, counts_in[q], q, group))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        ops, got = [], {}
        for q in peers:
            got[q] = torch.zeros(int(counts_in[q].item()), dtype=torch.int32)
            if len(payload[q]):
                ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(payload[q], np.int32)), q,
                                      group))
            if len(got[q]):
                ops.append(dist.P2POp(dist.irecv, got[q], q, group))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        return {q: got[q].numpy() for q in peers}

    if plan.mode == HALO_MPI:
        req = plan.requests()
        peers = [int(q) for q in plan.neighbors()[0]]
        got = swap(peers, {q: req[q] for q in peers})
        plan.set_sends(got)
        return None
    blk, _ = plan.blocks()
    mine = {}
    for owner, _start, lo, hi in blk:
        mine.setdefault(int(owner), []).extend([int(lo), int(hi)])
    # every rank learns who fetches from it: the owners of a rank's blocks are its neighbours
    # in z; the stencil couples only adjacent slabs, so the peers are the ranks within one
    peers = [q for q in (plan.rank - 1, plan.rank + 1) if 0 <= q < plan.nranks]
    got = swap(peers, {q: np.asarray(mine.get(q, []), np.int32) for q in peers})
    return {q: [(int(v[2 * i]), int(v[2 * i + 1])) for i in range(len(v) // 2)] for q, v in got.items()}


class Slab:
    """A rank's device part (hpccg_slab_*) on the current GPU."""

    def __init__(self, plan: SlabPlan, values):
        h = _c.c_void_p()
        _check(_lib.hpccg_slab_create(plan._h, np.ascontiguousarray(values, np.float64), _c.byref(h)),
               "slab_create")
        self._h = h
        self.rank, self.nranks, self.mode = plan.rank, plan.nranks, plan.mode
        v = [_c.c_int32(0) for _ in range(4)]
        _check(_lib.hpccg_slab_info(h, *[_c.byref(a) for a in v]), "slab_info")
        self.nrow, self.ncol, self.nsend, self.nblocks = (a.value for a in v)
        self.neighbors, self.recv_length = plan.neighbors()
        self.send_length = plan.sends()[0] if plan.mode == HALO_MPI else np.zeros(0, np.int32)
        self.blocks = plan.blocks()[0] if plan.mode == HALO_GET else np.zeros((0, 4), np.int32)

    def close(self):
        if getattr(self, "_h", None):
            _lib.hpccg_slab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def spmv(self, d_x, d_y):
        _sync_torch()
        _check(_lib.hpccg_slab_spmv(self._h, _dptr(d_x), _dptr(d_y)), "slab_spmv")

    def pack(self, d_x, d_sendbuf):
        _sync_torch()
        _check(_lib.hpccg_slab_pack(self._h, _dptr(d_x), _dptr(d_sendbuf) if d_sendbuf is not None else None),
               "slab_pack")

    def scatter_block(self, block: int, d_range, d_x):
        _sync_torch()
        _check(_lib.hpccg_slab_scatter_block(self._h, block, _dptr(d_range), _dptr(d_x)), "slab_scatter_block")

    def step(self, step: int, k: int, d_b, d_x, d_p, d_r, d_Ap, d_state, d_hist=None):
        _sync_torch()
        _check(_lib.hpccg_slab_cg_step(self._h, step, k, _dptr(d_b) if d_b is not None else None, _dptr(d_x),
                                       _dptr(d_p), _dptr(d_r), _dptr(d_Ap), _dptr(d_state),
                                       _dptr(d_hist) if d_hist is not None else None), "slab_cg_step")


def group_cg(slabs, d_bs, d_xs, max_iter: int = 150, tolerance: float = 0.0, history: bool = True):
    """MPI/src/numerics.F90:41-162 on every rank of the communicator, all in this process
    (hpccg_slab_group_cg).  Returns (niters, normr, hist, status); x updated in place."""
    _sync_torch()
    P = len(slabs)
    hs = (_c.c_void_p * P)(*[s._h for s in slabs])
    bs = (_c.c_void_p * P)(*[_dptr(t) for t in d_bs])
    xs = (_c.c_void_p * P)(*[_dptr(t) for t in d_xs])
    hist = np.zeros(max_iter + 1, np.float64)
    it, nr = _c.c_int32(0), _c.c_double(0.0)
    rc = _lib.hpccg_slab_group_cg(hs, P, bs, xs, max_iter, tolerance, _c.byref(it), _c.byref(nr),
                                  hist.ctypes.data if history else None)
    _check(rc, "slab_group_cg", allow=(HPCCG_OK, HPCCG_ERR_BREAKDOWN))
    return it.value, nr.value, hist[: it.value + 1], rc


class DistCG:
    """One rank's CG (MPI/src/numerics.F90:41-162) driven from this process, with
    torch.distributed as the transport: exchange_externals by point-to-point messages, the
    dot products by an all-gather folded in rank order.  With the gloo backend the device
    vectors are staged through host memory."""

    def __init__(self, slab: Slab, plan: SlabPlan, group=None, get_ranges=None, device=None):
        """device: where the slab's vectors live, by default the current CUDA device (the
        library's Slab).  The transport works on any torch device: a slab object whose steps
        keep their vectors in host memory passes device="cpu"."""
        import torch
        import torch.distributed as dist

        self.torch, self.dist = torch, dist
        self.slab, self.group = slab, group
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.host_staged = self.dev.type == "cuda" and dist.get_backend(group) != "nccl"
        self.get_ranges = get_ranges or {}  # GET form: {requester: [(inmin, inmax), ..]}
        self.P = slab.nranks
        if slab.mode == HALO_MPI:
            self.sendbuf = torch.zeros(max(1, slab.nsend), dtype=torch.float64, device=self.dev)

    def _sync(self):
        if self.dev.type == "cuda":
            self.torch.cuda.synchronize()

    def _xfer(self, sends, recvs):
        """sends: [(peer, tensor)], recvs: [(peer, tensor)]; device tensors, staged if needed."""
        dist, torch = self.dist, self.torch
        ops, post = [], []
        for q, t in sends:
            ops.append(dist.P2POp(dist.isend, t.cpu() if self.host_staged else t.contiguous(), q, self.group))
        for q, t in recvs:
            buf = torch.empty(t.shape, dtype=t.dtype) if self.host_staged else t
            ops.append(dist.P2POp(dist.irecv, buf, q, self.group))
            if self.host_staged:
                post.append((t, buf))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for t, buf in post:
            t.copy_(buf)
        self._sync()

    def exchange(self, d_p):
        s = self.slab
        if s.mode == HALO_MPI:
            s.pack(d_p, self.sendbuf)
            sends, off = [], 0
            for q, n in zip(s.neighbors, s.send_length):
                sends.append((int(q), self.sendbuf[off:off + n]))
                off += n
            recvs, off = [], s.nrow
            for q, n in zip(s.neighbors, s.recv_length):
                recvs.append((int(q), d_p[off:off + n]))
                off += n
            self._xfer(sends, recvs)
        else:
            sends = [(q, d_p[lo - 1:hi]) for q, rngs in sorted(self.get_ranges.items()) for lo, hi in rngs]
            stages = [self.torch.empty(int(hi - lo + 1), dtype=self.torch.float64, device=self.dev)
                      for _owner, _st, lo, hi in s.blocks]
            recvs = [(int(blk[0]), st) for blk, st in zip(s.blocks, stages)]
            self._xfer(sends, recvs)
            for b, st in enumerate(stages):
                s.scatter_block(b, st, d_p)

    def allreduce(self, d_state):
        torch, dist = self.torch, self.dist
        loc = d_state[LOCAL:LOCAL + 1].clone()
        if self.host_staged:
            loc = loc.cpu()
        out = [torch.zeros_like(loc) for _ in range(self.P)]
        dist.all_gather(out, loc, group=self.group)
        s = out[0].clone()
        for q in range(1, self.P):
            s = s + out[q]
        d_state[GLOBAL:GLOBAL + 1].copy_(s.to(self.dev))
        self._sync()

    def solve(self, d_b, d_x, max_iter: int = 150, tolerance: float = 0.0):
        """Returns (niters, normr, hist); d_x is updated in place."""
        torch = self.torch
        s = self.slab
        f64 = dict(dtype=torch.float64, device=self.dev)
        p = torch.zeros(s.ncol, **f64)
        r, Ap = torch.zeros(s.nrow, **f64), torch.zeros(s.nrow, **f64)
        state = torch.zeros(8, **f64)
        state[TOL] = tolerance
        hist = torch.zeros(max_iter + 1, **f64)
        s.step(START, 0, d_b, d_x, p, r, Ap, state, hist)
        self.exchange(p)
        s.step(PREPARE, 0, d_b, d_x, p, r, Ap, state, hist)
        self.allreduce(state)
        s.step(PREPARED, 0, d_b, d_x, p, r, Ap, state, hist)
        niters = 0
        for k in range(1, max_iter + 1):
            s.step(BEGIN, k, d_b, d_x, p, r, Ap, state, hist)
            if float(state[DONE].item()) != 0.0:
                break
            self.exchange(p)
            s.step(SPMV, k, d_b, d_x, p, r, Ap, state, hist)
            self.allreduce(state)
            s.step(UPDATE, k, d_b, d_x, p, r, Ap, state, hist)
            self.allreduce(state)
            niters = k
        h = hist[: niters + 1].cpu().numpy()
        return niters, float(state[NORMR].item()), h
