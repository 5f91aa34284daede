"""The large mixed-precision configuration at its named size: the radius-3
lattice Hamiltonian on 64^3 sites (N = 262144, seed 0), threshold 1e-6,
occupation N/2, forward and adjoint, FP64 against mixed/FP32.

The configuration's M = 512 cannot hold the iterates (the first X^2 keeps 829
entries in an interior row) and its iterates fill in as the smaller lattices'
do, so this runs the first 3 SP2 iterations (rows of 829, about 1300 and
about 1800 entries) with M = 2048: 6.4 GB per FP64 iterate.  The
perturbation V is symmetric on H's pattern with entries U[-0.01, 0.01] (a
hash of the pair, so that no N x N array is built); L = sum_ij D_ij V_ij.

Checked:
  - the mixed forward (2 FP32 iterations, 1 FP64 closing) against the FP64
    one: trace and band energy tr(DH) within the 1e-6 target (measured
    7.4e-7 and 1.8e-7);
  - the FP64 adjoint's loss against tr(D V) of the FP64 forward, 1e-10;
  - the FP32 adjoint against the FP64 one, within 1e-2 of the largest entry.
The adjoint's backward products are formed on the iterates' patterns only
(the masked form of the unordered product), so nothing wider than M is
stored.  Times (synchronised; the second call of each, after the first has
grown the device memory pool) are printed for s/solve and s/backward."""
import ctypes as C
import time

import numpy as np
import pytest

import bml_b200 as B

pytestmark = [pytest.mark.gpu, pytest.mark.unordered]

L, RADIUS, N = 64, 3, 64 ** 3
MH, M = 128, 2048
THR, ITERS, EVERY = 1e-6, 3, 3


def _pair_uniform(i, j):
    """U[-0.01, 0.01] from the unordered pair (i, j): splitmix64 of the key."""
    a, b = np.minimum(i, j).astype(np.uint64), np.maximum(i, j).astype(np.uint64)
    x = a * np.uint64(N) + b + np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return ((x >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 - 0.5) * 0.02


@pytest.fixture(scope="module")
def problem():
    v, ix, nz = B.gen_lattice(L, RADIUS, N, MH, 0)
    mask = (np.arange(MH)[None, :] < nz[:, None]).reshape(-1)
    rows = np.repeat(np.arange(N), MH)
    vv = np.zeros_like(v)
    vv[mask] = _pair_uniform(rows[mask], ix[mask])
    return v, ix, nz, vv


def _mat(v, ix, nz, prec=2):
    dt = np.float64 if prec == 2 else np.float32
    return B.Ellpack.from_arrays(v.astype(dt), ix, nz, N, MH, prec=prec)


def _timed(fn):
    B.check(B.lib.bml_b200_synchronize())
    t0 = time.perf_counter()
    out = fn()
    B.check(B.lib.bml_b200_synchronize())
    return time.perf_counter() - t0, out


@pytest.fixture(scope="module")
def forward(problem):
    v, ix, nz, vv = problem
    H, V = _mat(v, ix, nz), _mat(vv, ix, nz)
    # H and V at the iterates' M, for tr(D H) and tr(D V) (bml_trace_mult
    # takes matrices of one shape, as the reference's does)
    Hm, Vm = B.Ellpack(N, M), B.Ellpack(N, M)
    B.lib.bml_copy(H.h, Hm.h)
    B.lib.bml_copy(V.h, Vm.h)
    B.check()
    res = {}
    for name in ("fp64", "mixed"):
        D = B.Ellpack(N, M)
        info = (C.c_double * 8)()
        if name == "fp64":
            call = lambda: B.lib.bml_b200_sp2(H.h, D.h, THR, N / 2.0, ITERS, -1.0, 0, info)
        else:
            call = lambda: B.lib.bml_b200_sp2_mixed(H.h, D.h, THR, N / 2.0, ITERS, -1.0, 0, 1, info)
        # the first call in the process grows the device memory pool (several
        # GB of new mappings); the second is timed
        assert call() == B.OK
        s, st = _timed(call)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        res[name] = {"s": s, "trace": B.lib.bml_trace(D.h), "energy": B.lib.bml_trace_mult(D.h, Hm.h),
                     "loss": B.lib.bml_trace_mult(D.h, Vm.h), "width": B.lib.bml_get_bandwidth(D.h),
                     "iterations": int(info[0]), "info": list(info)}
        B.check()
        D.free()
    for m in (H, V, Hm, Vm):
        m.free()
    print("config 5 forward, %d iterations: FP64 %.3f s, mixed %.3f s, widest row %d; info FP64 %s, mixed %s"
          % (ITERS, res["fp64"]["s"], res["mixed"]["s"], res["fp64"]["width"], res["fp64"]["info"],
             res["mixed"]["info"]))
    return res


def _adjoint(problem, prec):
    v, ix, nz, vv = problem
    H, V = _mat(v, ix, nz, prec), _mat(vv, ix, nz, prec)
    dH = B.Ellpack(N, MH, prec=prec)
    loss = C.c_double()
    call = lambda: B.lib.bml_b200_sp2_adjoint(H.h, V.h, THR, N / 2.0, ITERS, EVERY, M, dH.h, C.byref(loss))
    assert call() == B.OK  # grows the memory pool; the second call is timed
    s, st = _timed(call)
    assert st == B.OK, B.lib.bml_b200_error_string(st)
    g, gix, gnz = dH.download()
    for m in (H, V, dH):
        m.free()
    return s, loss.value, g.astype(np.float64), gix, gnz


@pytest.fixture(scope="module")
def adjoint64(problem):
    return _adjoint(problem, 2)


def test_config5_mixed_forward(forward):
    e, m = forward["fp64"], forward["mixed"]
    assert e["iterations"] == m["iterations"] == ITERS
    assert 1500 < e["width"] <= M
    tr_err = abs(m["trace"] - e["trace"]) / abs(e["trace"])
    en_err = abs(m["energy"] - e["energy"]) / abs(e["energy"])
    print("config 5 mixed: trace error %.2e, tr(DH) error %.2e, speed-up %.2f"
          % (tr_err, en_err, e["s"] / m["s"]))
    assert tr_err <= 1e-6
    assert en_err <= 1e-6


def test_config5_adjoint_fp64(problem, forward, adjoint64):
    s, loss, g, gix, gnz = adjoint64
    v, ix, nz, vv = problem
    assert np.array_equal(gnz, nz)
    assert loss == pytest.approx(forward["fp64"]["loss"], rel=1e-10)
    mask = (np.arange(MH)[None, :] < nz[:, None]).reshape(-1)
    assert np.isfinite(g[mask]).all() and np.abs(g[mask]).max() > 0
    print("config 5 adjoint FP64: %.3f s (forward %.3f s), loss %.12g" % (s, forward["fp64"]["s"], loss))


def test_config5_adjoint_fp32(problem, adjoint64):
    s64, loss64, g64, _, nz = adjoint64
    s32, loss32, g32, _, nz32 = _adjoint(problem, 1)
    assert np.array_equal(nz32, nz)
    mask = (np.arange(MH)[None, :] < nz[:, None]).reshape(-1)
    scale = np.abs(g64[mask]).max()
    err = np.abs(g32[mask] - g64[mask]).max() / scale
    print("config 5 adjoint FP32: %.3f s (FP64 %.3f s), gradient error %.2e of max, loss error %.2e"
          % (s32, s64, err, abs(loss32 - loss64) / abs(loss64)))
    assert err <= 1e-2
