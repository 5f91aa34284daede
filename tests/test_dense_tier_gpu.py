"""The dense tier of the unordered product and the wide-row operations,
against the reference library on identical inputs.

Operands whose rows fill at least 40 % of N take the dense tier (a GEMM on
dense images, then the reference's keep rule), and rows too wide for the
shared-memory hashes take the dense-image forms of add, trace_mult and
fnorm2 (and of restrict, which the adjoint uses).  Checked as in
test_unordered_gpu.py: products within 1e-12 of S = sum |a_ij b_jk| (FP32:
2 n 2^-24), patterns identical except at the threshold; add bit-identical to
the reference as a dense matrix (its rows in ascending column order); sums
within 1e-12."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B
import x2check

pytestmark = [pytest.mark.gpu, pytest.mark.unordered]
SINGLE, DOUBLE = 1, 2


def _ell_from_dense(D, M):
    """ELLPACK arrays of a dense matrix (nonzeros, ascending columns)."""
    N = D.shape[0]
    v = np.zeros(N * M, D.dtype)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    for i in range(N):
        cols = np.flatnonzero(D[i])
        assert len(cols) <= M
        v[i * M:i * M + len(cols)] = D[i, cols]
        ix[i * M:i * M + len(cols)] = cols
        nz[i] = len(cols)
    return v, ix, nz


def _random_dense(N, density, seed, symmetric=True, dtype=np.float64):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((N, N)) * (rng.random((N, N)) < density) / np.sqrt(N * density)
    if symmetric:
        D = np.triu(D) + np.triu(D, 1).T
    np.fill_diagonal(D, rng.standard_normal(N))
    return D.astype(dtype)


def _ref_product(O, a, b, N, M, thr, M2, prec, x2):
    A = O.ref_ellpack(*a, N, M, prec)
    Bm = A if x2 else O.ref_ellpack(*b, N, M, prec)
    R = O.ref().bml_zero_matrix(2, prec, N, M2, 0)
    if x2:
        tr = O.ref_x2(A, R, thr)
    else:
        O.ref().bml_multiply_AB(A, Bm, R, thr)
        tr = None
    out = O.ref_ellpack_arrays(R)
    for h in ([A, R] if x2 else [A, Bm, R]):
        O.ref_free(h)
    return out, tr


def _absum(a, b, N, M, M2):
    """S = |A| |B| on the structural pattern of the product, dense (numpy)."""
    def dense(arr):
        v, ix, nz = arr
        D = np.zeros((N, N))
        for i in range(N):
            D[i, ix[i * M:i * M + nz[i]]] = np.abs(v[i * M:i * M + nz[i]])
        return D
    Sd = dense(a) @ dense(b)
    return _ell_from_dense(Sd, M2)


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE], ids=["fp64", "fp32"])
def test_dense_tier_x2(oracle_mod, prec):
    O = oracle_mod
    N, M, thr = 2000, 2000, 1e-4
    dt = np.float64 if prec == DOUBLE else np.float32
    D = _random_dense(N, 0.6, 1, dtype=dt)
    a = _ell_from_dense(D, M)
    ref, tr_ref = _ref_product(O, a, a, N, M, thr, N, prec, True)
    S = _absum(a, a, N, M, N)
    X = B.Ellpack.from_arrays(*a, N, M, prec=prec)
    X2 = B.Ellpack(N, N, prec=prec)
    st, tr = B.multiply_x2(X, X2, thr)
    assert st == B.OK
    assert B.lib.bml_b200_last_x2_dense() == 1
    got = X2.download()
    eps = 1e-12 if prec == DOUBLE else 2.0 * N * 2.0 ** -24
    x2check.compare(got, ref, S, N, N, N, thr, eps)
    assert x2check.rows_sorted(got, N)
    assert tr[0] == pytest.approx(tr_ref[0], rel=1e-12 if prec == DOUBLE else 1e-5)
    # the same product on the sparse kernels agrees within the bound
    old = B.lib.bml_b200_set_dense_tier(0)
    try:
        st, _ = B.multiply_x2(X, X2, thr)
        assert st == B.OK and B.lib.bml_b200_last_x2_dense() == 0
        x2check.compare(X2.download(), got, S, N, N, N, thr, eps)
    finally:
        B.lib.bml_b200_set_dense_tier(old)
    X.free()
    X2.free()


def test_dense_tier_ab_and_diagonal_rule(oracle_mod):
    """A*B with A != B (not symmetric): values within the bound, and the
    diagonal rule on the structure: row 3 of A meets no row of B holding
    column 3 (C[3,3] untouched, not kept), row 5's diagonal products cancel
    to an exact zero (touched, kept with value 0)."""
    O = oracle_mod
    N, M, thr = 1500, 1500, 0.0
    Da = _random_dense(N, 0.5, 2, symmetric=False)
    Db = _random_dense(N, 0.5, 3, symmetric=False)
    # row 3 of A: only columns j whose row j of B lacks column 3
    Da[3, :] = 0.0
    js = np.flatnonzero(Db[:, 3] == 0.0)[:40]
    Da[3, js] = 1.0
    # row 5 of A: two products into column 5 that cancel exactly
    Da[5, :] = 0.0
    Db[:, 5] = 0.0
    Da[5, [10, 11]] = [1.0, 1.0]
    Db[10, 5], Db[11, 5] = 0.5, -0.5
    a, b = _ell_from_dense(Da, M), _ell_from_dense(Db, M)
    ref, _ = _ref_product(O, a, b, N, M, thr, N, DOUBLE, False)
    S = _absum(a, b, N, M, N)
    GA = B.Ellpack.from_arrays(*a, N, M)
    GB = B.Ellpack.from_arrays(*b, N, M)
    GC = B.Ellpack(N, N)
    B.lib.bml_multiply_AB(GA.h, GB.h, GC.h, thr)
    B.check()
    assert B.lib.bml_b200_last_x2_dense() == 1
    got = GC.download()
    x2check.compare(got, ref, S, N, N, N, thr, 1e-12)
    v, ix, nz = got
    row3 = ix[3 * N:3 * N + nz[3]]
    row5 = dict(zip(ix[5 * N:5 * N + nz[5]].tolist(), v[5 * N:5 * N + nz[5]].tolist()))
    assert 3 not in row3.tolist()
    assert row5.get(5) == 0.0
    for m in (GA, GB, GC):
        m.free()


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE], ids=["fp64", "fp32"])
def test_wide_row_operations(oracle_mod, prec):
    """Rows of about 4000 entries (N = 9000): add 2A - B at threshold 1e-3,
    trace_mult and fnorm2, against the reference (add as dense matrices, bit
    for bit) and numpy (the sums, to 1e-12; FP32 sums of products formed in
    float, to 1e-6).  (restrict's wide form runs in the adjoint at config 4.)"""
    O = oracle_mod
    N, M = 9000, 9000
    dt = np.float64 if prec == DOUBLE else np.float32
    Da = _random_dense(N, 0.5, 4, dtype=dt)
    Db = _random_dense(N, 0.4, 5, dtype=dt)
    a, b = _ell_from_dense(Da, M), _ell_from_dense(Db, M)
    GA = B.Ellpack.from_arrays(*a, N, M, prec=prec)
    GB = B.Ellpack.from_arrays(*b, N, M, prec=prec)
    # trace_mult: the reference's rule, sum_ij A_ij B_ij
    T = Da.astype(np.float64) * Db.astype(np.float64)
    tm = B.lib.bml_trace_mult(GA.h, GB.h)
    B.check()
    Sabs = np.abs(T).sum()
    assert abs(tm - T.sum()) <= (1e-12 if prec == DOUBLE else 1e-6) * Sabs
    # fnorm2 = ||A - B||_F
    fn = B.lib.bml_fnorm2(GA.h, GB.h)
    B.check()
    want = np.sqrt(((Da.astype(np.float64) - Db.astype(np.float64)) ** 2).sum())
    assert fn == pytest.approx(want, rel=1e-12 if prec == DOUBLE else 1e-6)
    # add, against the reference library
    RA = O.ref_ellpack(*a, N, M, prec)
    RB = O.ref_ellpack(*b, N, M, prec)
    O.ref().bml_add(RA, RB, 2.0, -1.0, 1e-3)
    B.lib.bml_add(GA.h, GB.h, 2.0, -1.0, 1e-3)
    B.check()
    ref = O.ref_ellpack_arrays(RA)
    got = GA.download()
    to_dense = lambda arr: _dense_of(arr, N, M, dt)
    assert np.array_equal(to_dense(got).view(np.uint8), to_dense(ref).view(np.uint8))
    assert np.array_equal(got[2], ref[2])
    assert x2check.rows_sorted(got, M)
    for h in (RA, RB):
        O.ref_free(h)
    for m in (GA, GB):
        m.free()


def _dense_of(arrs, N, M, dt):
    v, ix, nz = arrs
    D = np.zeros((N, N), dt)
    for i in range(N):
        D[i, ix[i * M:i * M + nz[i]]] = v[i * M:i * M + nz[i]]
    return D
