"""Row-sharded SP2 (bml_b200/sharded.py) on CPU ranks: two gloo processes run
the sharded loop with host operations that follow the reference's row
semantics through the oracle, and the result must equal the single-process
oracle SP2 bit for bit (the partial traces are summed in another order, so
the trace agrees to 1e-12).  This covers the collective logic (row blocks,
trace all-reduce, branch agreement, all-gather) without a GPU; the GPU
operations are covered at world size 1 in test_sharded_gpu.py."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

N, M, THR, ITERS = 512, 512, 1e-5, 14


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _chain(n, m):
    import bml_b200 as B
    return B.gen_chain(n, m, 0)


class HostOps:
    """The sharded loop's operations on host arrays, through the oracle."""

    def __init__(self, O, v, ix, nz):
        self.O, self.lib = O, O.rest()
        self.n = N
        self.H = (v.copy(), ix.copy(), nz.copy())

    def _p(self, a, t):
        return a.ctypes.data_as(C.POINTER(t))

    def start(self):
        v, ix, nz = (a.copy() for a in self.H)
        b = np.zeros(2)
        lib = self.lib
        lib.oracle_ellpack_gershgorin_d(N, M, self._p(v, C.c_double), self._p(ix, C.c_int), self._p(nz, C.c_int),
                                        self._p(b, C.c_double))
        mm = b[1] - b[0]
        s = -1.0 / mm
        for i in range(N):
            v[i * M:i * M + nz[i]] = s * v[i * M:i * M + nz[i]]
        lib.oracle_ellpack_add_identity_d(N, M, self._p(v, C.c_double), self._p(ix, C.c_int), self._p(nz, C.c_int),
                                          C.c_double(b[1] / mm), C.c_double(0.0))
        self.X = [v, ix, nz]
        self.X2 = [np.zeros(N * M), np.zeros(N * M, np.int32), np.zeros(N, np.int32)]

    def x2_rows(self, r0, r1):
        v, ix, nz = self.X
        (v2, ix2, nz2), tr, w = self.O.rest_x2(v, ix, nz, N, M, THR, M)
        assert w <= M
        for a, b, wd in ((self.X2[0], v2, M), (self.X2[1], ix2, M), (self.X2[2], nz2, 1)):
            a[r0 * wd:r1 * wd] = b[r0 * wd:r1 * wd]
        t = t2 = 0.0
        for i in range(r0, r1):
            row = slice(i * M, i * M + nz[i])
            t += float(v[row][ix[row] == i].sum())
            row2 = slice(i * M, i * M + nz2[i])
            t2 += float(v2[row2][ix2[row2] == i].sum())
        return t, t2

    def update_rows(self, branch, r0, r1):
        if branch == 0:
            for a, b, wd in zip(self.X, self.X2, (M, M, 1)):
                a[r0 * wd:r1 * wd] = b[r0 * wd:r1 * wd]
            return
        v, ix, nz = (a.copy() for a in self.X)
        v2, ix2, nz2 = self.X2
        self.lib.oracle_ellpack_add_d(N, M, self._p(v, C.c_double), self._p(ix, C.c_int), self._p(nz, C.c_int), M,
                                      self._p(v2, C.c_double), self._p(ix2, C.c_int), self._p(nz2, C.c_int),
                                      C.c_double(2.0), C.c_double(-1.0), C.c_double(THR))
        for a, b, wd in zip(self.X, (v, ix, nz), (M, M, 1)):
            a[r0 * wd:r1 * wd] = b[r0 * wd:r1 * wd]

    def reduce_sum(self, arr):
        t = torch.tensor(arr, dtype=torch.float64)
        dist.all_reduce(t)
        return t.numpy()

    def gather(self, blocks):
        for a, wd in zip(self.X, (M, M, 1)):
            # blocks of unequal length (gloo's all_gather wants equal ones):
            # one broadcast per block
            for src, (s0, s1) in enumerate(blocks):
                buf = torch.from_numpy(a[s0 * wd:s1 * wd].copy())
                dist.broadcast(buf, src=src)
                a[s0 * wd:s1 * wd] = buf.numpy()

    def column_range(self, r0, r1):
        _, ix, nz = self.X
        cols = np.concatenate([ix[i * M:i * M + nz[i]] for i in range(r0, r1)] + [np.zeros(0, np.int32)])
        return (int(cols.min()), int(cols.max()) + 1) if cols.size else (0, 0)

    def allgather_ints(self, vals):
        mine = torch.tensor(vals, dtype=torch.int64)
        parts = [torch.empty_like(mine) for _ in range(dist.get_world_size())]
        dist.all_gather(parts, mine)
        return torch.stack(parts).numpy()

    def exchange(self, sends, recvs):
        reqs, inbox = [], []
        # one tag per array (gloo matches a message by peer and tag), far
        # from the small tags gloo's own collectives count up through
        for peer, a, b in sends:
            for k, (arr, wd) in enumerate(zip(self.X, (M, M, 1))):
                reqs.append(dist.isend(torch.from_numpy(arr[a * wd:b * wd].copy()), peer, tag=1000000 + k))
        for peer, a, b in recvs:
            for k, (arr, wd) in enumerate(zip(self.X, (M, M, 1))):
                buf = torch.from_numpy(np.empty((b - a) * wd, arr.dtype))
                reqs.append(dist.irecv(buf, peer, tag=1000000 + k))
                inbox.append((arr, a * wd, b * wd, buf))
        for r in reqs:
            r.wait()
        for arr, a, b, buf in inbox:
            arr[a:b] = buf.numpy()

    def trace(self):
        v, ix, nz = self.X
        return float(sum(v[i * M:i * M + nz[i]][ix[i * M:i * M + nz[i]] == i].sum() for i in range(N)))


def _rank_main(rank, world, port, out_dir, exchange="gather"):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from oracle import oracle as O
    from bml_b200.sharded import ShardedSP2
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        v, ix, nz = _chain(N, M)
        ops = HostOps(O, v, ix, nz)
        res = ShardedSP2(ops, dist, rank, world, exchange).run(N / 2.0, ITERS)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), v=ops.X[0], ix=ops.X[1], nz=ops.X[2],
                 trace=res["trace"], iterations=res["iterations"], branches=np.array(res["branches"]),
                 rows_received=res["rows_received"])
    finally:
        dist.destroy_process_group()


def test_sharded_sp2_two_ranks_matches_oracle(oracle_mod, tmp_path):
    O = oracle_mod
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r = [np.load(tmp_path / ("rank%d.npz" % k)) for k in range(2)]
    # both ranks hold the same iterate
    for key in ("v", "ix", "nz", "branches"):
        assert np.array_equal(r[0][key], r[1][key]), key
    v, ix, nz = _chain(N, M)
    (dv, dix, dnz), info = O.rest_sp2(v, ix, nz, N, M, THR, N / 2.0, ITERS, -1.0, 0)
    assert int(r[0]["iterations"]) == int(info[0]) == ITERS
    assert O.same_rows_exact((r[0]["v"], r[0]["ix"], r[0]["nz"]), (dv, dix, dnz), M, M)
    assert float(r[0]["trace"]) == pytest.approx(info[2], rel=1e-12)


def test_sharded_sp2_halo_three_ranks_matches_oracle(oracle_mod, tmp_path):
    """The halo exchange (point-to-point rows within each rank's column
    range, one all-gather at the end) on three gloo ranks, the middle one
    with two neighbours: the same density matrix, bit for bit, as the
    single-process oracle SP2, with far fewer rows moved than all-gathers
    of the whole iterate would move."""
    O = oracle_mod
    port = _free_port()
    world = 3
    mp.spawn(_rank_main, args=(world, port, str(tmp_path), "halo"), nprocs=world, join=True)
    r = [np.load(tmp_path / ("rank%d.npz" % k)) for k in range(world)]
    for k in range(1, world):
        for key in ("v", "ix", "nz", "branches"):
            assert np.array_equal(r[0][key], r[k][key]), key
    v, ix, nz = _chain(N, M)
    (dv, dix, dnz), info = O.rest_sp2(v, ix, nz, N, M, THR, N / 2.0, ITERS, -1.0, 0)
    assert int(r[0]["iterations"]) == int(info[0]) == ITERS
    assert O.same_rows_exact((r[0]["v"], r[0]["ix"], r[0]["nz"]), (dv, dix, dnz), M, M)
    assert float(r[0]["trace"]) == pytest.approx(info[2], rel=1e-12)
    # rows received by the middle rank: its two bands, against the
    # all-gather's N - N/3 rows per iteration
    from bml_b200.sharded import row_blocks
    b0, b1 = row_blocks(N, world)[1]
    got = int(r[1]["rows_received"])
    assert 0 < got < 0.5 * ITERS * (N - (b1 - b0))


def test_halo_ranges_are_symmetric():
    """What rank s sends to rank d is exactly what d receives from s."""
    from bml_b200.sharded import ShardedSP2

    class Fake:
        n = 100

        def __init__(self, me, ranges):
            self.me, self.ranges, self.sent = me, ranges, None

        def column_range(self, r0, r1):
            return self.ranges[self.me]

        def allgather_ints(self, vals):
            return np.array(self.ranges)

        def exchange(self, sends, recvs):
            self.sent, self.recv = sends, recvs

    ranges = [(0, 40), (20, 75), (60, 100), (0, 0)]
    fakes = [Fake(k, ranges) for k in range(4)]
    for k, f in enumerate(fakes):
        ShardedSP2(f, None, k, 4, "halo")._halo()
    for s_, fs in enumerate(fakes):
        for peer, a, b in fs.sent:
            assert (s_, a, b) in fakes[peer].recv
    for d_, fd in enumerate(fakes):
        for peer, a, b in fd.recv:
            assert (d_, a, b) in fakes[peer].sent
    # rank 3 (no entries) receives nothing; rank 1 receives rows 20..25 and 50..75
    assert fakes[3].recv == []
    assert sorted(fakes[1].recv) == [(0, 20, 25), (2, 50, 75)]


def test_row_blocks_cover_rows():
    from bml_b200.sharded import row_blocks
    for n in (1, 7, 64, 64000):
        for w in (1, 2, 3, 8):
            b = row_blocks(n, w)
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[k][1] == b[k + 1][0] for k in range(w - 1))
            assert max(y - x for x, y in b) - min(y - x for x, y in b) <= 1
