"""Row-sharded SP2 on the GPU through NCCL, at world size 1 (this run has
one GPU): the driver of bml_b200/sharded.py with the library's row-range
kernels and the iterate's device arrays gathered through NCCL must give the
same density matrix, bit for bit, as the single-call bml_b200_sp2.  The
multi-rank collective logic is covered on CPU ranks in test_sharded_sp2.py."""
import ctypes as C
import socket

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("exchange", ["gather", "halo"])
def test_sharded_world1_matches_single_call(oracle_mod, exchange):
    import torch
    import torch.distributed as dist
    from bml_b200.sharded import GpuOps, ShardedSP2
    L = 12
    N, M, thr, iters = L ** 3, L ** 3, 1e-5, 5
    v, ix, nz = B.gen_lattice(L, 3, N, 160, 0)
    pad = lambda a: np.pad(a.reshape(N, 160), ((0, 0), (0, M - 160))).reshape(-1)
    H = B.Ellpack.from_arrays(pad(v), pad(ix), nz, N, M)
    D = B.Ellpack(N, M)
    info = (C.c_double * 6)()
    assert B.lib.bml_b200_sp2(H.h, D.h, thr, N / 2.0, iters, -1.0, 0, info) == B.OK
    ref = D.download()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1)
    try:
        ops = GpuOps(B.lib, H.h, M, thr, dist, torch)
        res = ShardedSP2(ops, dist, 0, 1, exchange).run(N / 2.0, iters)
        if exchange == "halo":
            # the column range of all rows of the iterate: the whole lattice
            assert ops.column_range(0, N) == (0, N)
            assert res["rows_received"] == 0
        X = B.Ellpack(N, M, handle=ops.X)
        got = X.download()
        assert res["iterations"] == iters
        assert oracle_mod.same_rows_exact(got, ref, M, M)
        assert res["trace"] == pytest.approx(info[2], rel=1e-12)
        hh = C.c_void_p(ops.X2)
        B.lib.bml_deallocate(C.byref(hh))
    finally:
        dist.destroy_process_group()
