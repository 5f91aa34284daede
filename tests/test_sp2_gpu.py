"""SP2 purification on the GPU against the CPU oracle.

The oracle's SP2 (oracle/bml_oracle.c) runs the same loop with the reference's
arithmetic; since every X^2, copy and add of libbml_b200 is bit-identical to
the reference, the whole trajectory (branch choices, final density matrix)
must come out identical.  Traces are sums in a different order, so the
returned trace and idempotency error are compared to 1e-12 relative."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu


def run_gpu_sp2(v, ix, nz, N, M, thr, occ, maxiter, tol, stall):
    H = B.Ellpack.from_arrays(v, ix, nz, N, M)
    D = B.Ellpack(N, M)
    info = (C.c_double * 6)()
    st = B.lib.bml_b200_sp2(H.h, D.h, thr, occ, maxiter, tol, stall, info)
    return st, D.download(), list(info)


def test_sp2_chain_trajectory_identical(oracle_mod):
    O = oracle_mod
    N, M = 4096, 512
    v, ix, nz = B.gen_chain(N, M, 0)
    thr, occ = 1e-5, N / 2.0
    st, g, ginfo = run_gpu_sp2(v, ix, nz, N, M, thr, occ, 60, 1e-8, 0)
    assert st == B.OK
    o, oinfo = O.rest_sp2(v, ix, nz, N, M, thr, occ, 60, 1e-8, 0)
    assert ginfo[0] == oinfo[0] and ginfo[1] == oinfo[1], (ginfo, oinfo)
    assert O.same_rows_exact(g, o, M, M), "density matrix differs from the oracle"
    assert ginfo[2] == pytest.approx(oinfo[2], rel=1e-12)
    assert ginfo[4] == oinfo[4]


def test_sp2_lattice_small_trajectory_identical(oracle_mod):
    O = oracle_mod
    L = 8
    N, M = L ** 3, L ** 3
    v, ix, nz = B.gen_lattice(L, 2, N, M, 0)
    st, g, ginfo = run_gpu_sp2(v, ix, nz, N, M, 1e-5, N / 2.0, 25, 1e-8, 0)
    assert st == B.OK
    o, oinfo = O.rest_sp2(v, ix, nz, N, M, 1e-5, N / 2.0, 25, 1e-8, 0)
    assert ginfo[0] == oinfo[0]
    assert O.same_rows_exact(g, o, M, M)


def test_sp2_overflow_stops_with_status():
    N, M = 4096, 64
    v, ix, nz = B.gen_chain(N, M, 0)
    B.lib.bml_b200_set_verbose(0)
    st, _, info = run_gpu_sp2(v, ix, nz, N, M, 1e-5, N / 2.0, 10, 1e-8, 0)
    B.lib.bml_b200_set_verbose(1)
    B.clear_error()
    assert st == B.ERR_ROW_OVERFLOW and info[1] == 4
