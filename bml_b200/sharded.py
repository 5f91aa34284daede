"""Row-sharded SP2 on several GPUs: one process per GPU, torch.distributed.

The reference distributes the rows of its matrices over MPI ranks and
all-gathers the iterate after each product (`ellpack/bml_parallel_ellpack_typed.c:58-70`).
Here each rank forms its block of rows of X^2 from the whole iterate (rows
of X^2 are independent), the partial traces are summed over ranks (one
16-byte all-reduce), every rank takes the same branch, updates its rows, and
the new iterate's row blocks are all-gathered in place (NCCL over NVLink on
GPUs) before the next product.  Every rank therefore holds the same X after
each iteration, as in the single-GPU solve, and the trajectory is the same
up to the order in which the partial traces are summed.

With exchange="halo" the iterate is not all-gathered.  A row of X^2 reads
only the rows of X named by its columns, so after each update every rank
publishes the range [lo, hi) of the columns of its own rows (two integers,
all-gathered), and each rank sends to every other the rows of its block that
fall in that rank's range (point-to-point).  Rows outside a rank's range go
stale on it and are never read; one all-gather at the end gives every rank
the whole result.  On a banded iterate (the 1-D chain, or the first
iterations on a lattice) this moves a band of rows per neighbour instead of
the whole matrix; the trajectory is the same as with the all-gather.

The loop is written against a small set of operations so that its
collective logic can be exercised on CPU ranks (gloo) with a host
implementation of those operations; `GpuOps` is the implementation that
runs the library's kernels.
"""
import ctypes as C
import math

import numpy as np


def row_blocks(n, world):
    """Contiguous row blocks [r0, r1) per rank (the first n % world get one more)."""
    base, extra = divmod(n, world)
    out, r = [], 0
    for k in range(world):
        m = base + (1 if k < extra else 0)
        out.append((r, r + m))
        r += m
    return out


def _overlap(a, b):
    """Intersection of the half-open ranges a and b, or None."""
    lo, hi = max(a[0], b[0]), min(a[1], b[1])
    return (lo, hi) if lo < hi else None


class ShardedSP2:
    """SP2 with rows split over the ranks of `dist` (torch.distributed).

    ops must provide: n (rows), start() (X0 on this rank, whole), x2_rows(r0,
    r1) -> (trX, trX2) partial traces, update_rows(branch, r0, r1),
    gather(blocks) (every rank receives every block of X), reduce_sum(array)
    (sum over ranks), trace() (tr X, whole); for exchange="halo" also
    column_range(r0, r1) -> (lo, hi) (the columns of rows r0..r1 of X, hi
    exclusive; (0, 0) for no entries), allgather_ints(list) -> array of one
    row per rank, and exchange(sends, recvs) with (peer, row0, row1)
    entries (rows row0..row1 of X sent to or received from peer).
    """

    def __init__(self, ops, dist, rank, world, exchange="gather"):
        if exchange not in ("gather", "halo"):
            raise ValueError("exchange must be 'gather' or 'halo'")
        self.ops, self.dist, self.rank, self.world = ops, dist, rank, world
        self.exchange = exchange
        self.blocks = row_blocks(ops.n, world)
        self.rows_received = 0

    def _halo(self):
        """Send every rank the rows of this block that its next X^2 reads,
        receive the rows this block's X^2 reads from the others."""
        ops, me = self.ops, self.rank
        r0, r1 = self.blocks[me]
        lo, hi = ops.column_range(r0, r1)
        ranges = np.asarray(ops.allgather_ints([lo, hi]), dtype=np.int64).reshape(self.world, 2)
        sends, recvs = [], []
        for peer in range(self.world):
            if peer == me:
                continue
            out = _overlap(self.blocks[me], ranges[peer])
            if out:
                sends.append((peer, out[0], out[1]))
            inc = _overlap(self.blocks[peer], ranges[me])
            if inc:
                recvs.append((peer, inc[0], inc[1]))
        ops.exchange(sends, recvs)
        self.rows_received += sum(b - a for _, a, b in recvs)

    def run(self, occupation, maxiter, tol=-1.0, stall=0):
        ops = self.ops
        r0, r1 = self.blocks[self.rank]
        ops.start()
        it, rule, best, since, last = 0, 3, math.inf, 0, 0.0
        branches = []
        while it < maxiter:
            part = np.asarray(ops.x2_rows(r0, r1), dtype=np.float64)
            t, t2 = ops.reduce_sum(part)
            last = abs(t - t2)
            branch = 0 if abs(t2 - occupation) <= abs(2.0 * t - t2 - occupation) else 1
            branches.append(branch)
            ops.update_rows(branch, r0, r1)
            if self.exchange == "halo":
                self._halo()
            else:
                ops.gather(self.blocks)
                self.rows_received += ops.n - (r1 - r0)
            it += 1
            if last < tol:
                rule = 1
                break
            if stall > 0:
                if last < best:
                    best, since = last, 0
                else:
                    since += 1
                    if since >= stall:
                        rule = 2
                        break
        if self.exchange == "halo":
            ops.gather(self.blocks)  # every rank ends with the whole iterate
        return {"iterations": it, "rule": rule, "trace": ops.trace(), "idempotency": last,
                "branches": branches, "rows_received": self.rows_received}


class _CudaArrayView:
    """A device array described by __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class GpuOps:
    """The library's kernels on this rank's GPU; the iterate's device arrays
    are exchanged with NCCL through torch tensors that alias them."""

    def __init__(self, lib, H, M, threshold, dist, torch):
        self.lib, self.H, self.M, self.thr = lib, H, M, threshold
        self.dist, self.torch = dist, torch
        self.n = lib.bml_get_N(H)
        self.X = lib.bml_zero_matrix(2, 2, self.n, M, 0)
        self.X2 = lib.bml_zero_matrix(2, 2, self.n, M, 0)
        if not self.X or not self.X2:
            raise RuntimeError("sharded SP2: allocation failed")
        self._views = None

    def _check(self, st):
        if st:
            raise RuntimeError("libbml_b200 status %d: %s" % (st, self.lib.bml_b200_error_string(st)))

    def start(self):
        lib = self.lib
        lib.bml_copy(self.H, self.X)
        eb = lib.bml_gershgorin(self.H)
        e = C.cast(eb, C.POINTER(C.c_double))
        emin, emax = e[0], e[1]
        lib.bml_free_memory(eb)
        lib.bml_normalize(self.X, emin, emax)
        self._check(lib.bml_b200_last_error())
        self._views = None

    def _device_views(self):
        if self._views is None:
            pv, pi, pn, ld = C.c_void_p(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.c_int()
            self._check(self.lib.bml_b200_ellpack_device_arrays(self.X, C.byref(pv), C.byref(pi), C.byref(pn),
                                                                C.byref(ld)))
            t = self.torch
            n, ld = self.n, ld.value
            self.ld = ld
            self._views = (
                t.as_tensor(_CudaArrayView(pv.value, n * ld, "<f8"), device="cuda"),
                t.as_tensor(_CudaArrayView(C.cast(pi, C.c_void_p).value, n * ld, "<i4"), device="cuda"),
                t.as_tensor(_CudaArrayView(C.cast(pn, C.c_void_p).value, n, "<i4"), device="cuda"),
            )
        return self._views

    def x2_rows(self, r0, r1):
        tr = (C.c_double * 2)()
        self._check(self.lib.bml_b200_multiply_x2_rows(self.X, self.X2, self.thr, r0, r1, tr))
        return tr[0], tr[1]

    def update_rows(self, branch, r0, r1):
        self._check(self.lib.bml_b200_sp2_update_rows(self.X, self.X2, self.thr, branch, r0, r1))

    def reduce_sum(self, arr):
        t = self.torch.tensor(arr, dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t)
        return t.cpu().numpy()

    def gather(self, blocks):
        # the library's stream must be done with X before NCCL reads it, and
        # NCCL done before the library's next kernels read the gathered rows
        self._check(self.lib.bml_b200_synchronize())
        val, idx, nnz = self._device_views()
        ld = self.ld
        rank = self.dist.get_rank()
        equal = len({b - a for a, b in blocks}) == 1
        for full, width in ((val, ld), (idx, ld), (nnz, 1)):
            if equal:
                r0, r1 = blocks[rank]
                self.dist.all_gather_into_tensor(full, full[r0 * width:r1 * width].clone())
            else:
                for src, (a, b) in enumerate(blocks):
                    chunk = full[a * width:b * width]
                    self.dist.broadcast(chunk, src=src)
        self.torch.cuda.synchronize()

    def column_range(self, r0, r1):
        self._check(self.lib.bml_b200_synchronize())
        if r1 <= r0:
            return 0, 0
        t = self.torch
        _, idx, nnz = self._device_views()
        ld = self.ld
        cols = idx[r0 * ld:r1 * ld].view(r1 - r0, ld)
        live = t.arange(ld, device=cols.device)[None, :] < nnz[r0:r1, None]
        if not bool(live.any()):
            return 0, 0
        lo = int(t.where(live, cols, t.full_like(cols, self.n)).min())
        hi = int(t.where(live, cols, t.full_like(cols, -1)).max()) + 1
        return lo, hi

    def allgather_ints(self, vals):
        t = self.torch
        mine = t.tensor(vals, dtype=t.int64, device="cuda")
        parts = [t.empty_like(mine) for _ in range(self.dist.get_world_size())]
        self.dist.all_gather(parts, mine)
        return t.stack(parts).cpu().numpy()

    def exchange(self, sends, recvs):
        # the library's stream must be done with X before NCCL reads it, and
        # NCCL done before the library's next kernels read the received rows
        self._check(self.lib.bml_b200_synchronize())
        val, idx, nnz = self._device_views()
        ld, d = self.ld, self.dist
        p2p = []
        for peer, a, b in sends:
            for full, width in ((val, ld), (idx, ld), (nnz, 1)):
                p2p.append(d.P2POp(d.isend, full[a * width:b * width], peer))
        for peer, a, b in recvs:
            for full, width in ((val, ld), (idx, ld), (nnz, 1)):
                p2p.append(d.P2POp(d.irecv, full[a * width:b * width], peer))
        if p2p:
            for req in d.batch_isend_irecv(p2p):
                req.wait()
        self.torch.cuda.synchronize()

    def trace(self):
        return self.lib.bml_trace(self.X)

    def free(self):
        for h in (self.X, self.X2):
            hh = C.c_void_p(h)
            self.lib.bml_deallocate(C.byref(hh))
