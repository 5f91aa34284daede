"""Every X^2 tier against the reference CPU library, bit for bit.

The multiply routes each row to a tier from an estimate of its width: the
product bound on a first call, the previous call's width after that.  These
tests enable one tier at a time (the dense tier C is always on, as the
fallback) and multiply twice, so the second call routes by the first call's
widths.  The inputs are wide enough to reach every tier.  Both calls must
match the reference exactly, and the second must have sent rows through the
tier under test.  A matrix whose columns are all multiples of 32 puts a
whole row on one warp of the column-partitioned tiers, which then hand the row on
to the next tier; that path must match the reference too."""
import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu

DOUBLE, SINGLE = 2, 1


def _reference_x2(O, v, ix, nz, N, M, thr, M2, prec=DOUBLE):
    A = O.ref_ellpack(v, ix, nz, N, M, prec)
    R = O.ref().bml_zero_matrix(2, prec, N, M2, 0)
    tr = O.ref_x2(A, R, thr)
    out = O.ref_ellpack_arrays(R)
    O.ref_free(A)
    O.ref_free(R)
    return out, tr


@pytest.fixture(scope="module")
def wide(oracle_mod):
    """H, the 14^3 lattice Hamiltonian (radius 3), and X1 = H^2 (thr 1e-5),
    with the reference H^2 and X1^2: rows of H^2 hold up to 621 distinct
    columns, rows of X1^2 about 900 to 2744."""
    O = oracle_mod
    L = 14
    N = L ** 3
    v, ix, nz = B.gen_lattice(L, 3, N, 160, 0)
    (v1, ix1, nz1), tr1 = _reference_x2(O, v, ix, nz, N, 160, 1e-5, 1024)
    M2 = N
    ref2, tr2 = _reference_x2(O, v1, ix1, nz1, N, 1024, 1e-5, M2)
    return dict(N=N, M=1024, M2=M2, x=(v1, ix1, nz1), ref=ref2, tr=tr2,
                h=(v, ix, nz), href=_reference_x2(O, v, ix, nz, N, 160, 1e-5, M2))


def _gpu_x2(x, N, M, M2, thr, prec=DOUBLE):
    X = B.Ellpack.from_arrays(*x, N, M, prec=prec)
    X2 = B.Ellpack(N, M2, prec=prec)
    out = []
    for _ in range(2):
        st, tr = B.multiply_x2(X, X2, thr)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        out.append((X2.download(), tr, B.last_tier_counts()))
    X.free()
    X2.free()
    return out


@pytest.mark.parametrize("tier", ["A", "W8", "B1", "W16", "K4", "K8", "C"])
def test_each_tier_bit_exact(oracle_mod, wide, tier):
    O = oracle_mod
    used = 0
    for x, M, (ref, tr_ref) in ((wide["h"], 160, wide["href"]), (wide["x"], wide["M"], (wide["ref"], wide["tr"]))):
        B.set_x2_tiers(tier)
        try:
            runs = _gpu_x2(x, wide["N"], M, wide["M2"], 1e-5)
        finally:
            B.set_x2_tiers()
        for got, tr, _ in runs:
            assert O.same_rows_exact(got, ref, wide["M2"], wide["M2"]), "rows differ from the reference"
            assert tr[0] == pytest.approx(tr_ref[0], rel=1e-12)
            assert tr[1] == pytest.approx(tr_ref[1], rel=1e-12)
        used += runs[1][2][B.X2_TIERS.index(tier)]
    assert used > 0


def test_partitioned_tiers_single_precision(oracle_mod, wide):
    O = oracle_mod
    v1, ix1, nz1 = wide["x"]
    x32 = (v1.astype(np.float32), ix1, nz1)
    ref, tr_ref = _reference_x2(O, *x32, wide["N"], wide["M"], 1e-5, wide["M2"], prec=SINGLE)
    B.set_x2_tiers("W8", "W16", "K4", "K8")
    try:
        runs = _gpu_x2(x32, wide["N"], wide["M"], wide["M2"], 1e-5, prec=SINGLE)
    finally:
        B.set_x2_tiers()
    for got, tr, _ in runs:
        assert O.same_rows_exact(got, ref, wide["M2"], wide["M2"])
        assert tr[0] == pytest.approx(tr_ref[0], rel=1e-5)
        assert tr[1] == pytest.approx(tr_ref[1], rel=1e-5)
    counts = runs[1][2]
    assert sum(counts[B.X2_TIERS.index(t)] for t in ("W8", "W16", "K4", "K8")) > 0


def _one_class_columns(N, per_row, seed):
    """Random rows whose columns are all multiples of 32: every product
    column falls in one class k % 32, so one warp of a wide tier holds all of
    a row's columns."""
    rng = np.random.default_rng(seed)
    M = per_row + 1
    v = np.zeros(N * M)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    pool = np.arange(0, N, 32)
    for i in range(N):
        cols = rng.choice(pool, size=per_row, replace=False)
        v[i * M:i * M + per_row] = rng.uniform(-1, 1, per_row)
        ix[i * M:i * M + per_row] = cols
        nz[i] = per_row
    return v, ix, nz, M


@pytest.mark.parametrize("tier", ["W8", "W16"])
def test_rows_handed_on_from_a_full_warp(oracle_mod, tier):
    O = oracle_mod
    N = 12800  # 400 columns in class 0
    v, ix, nz, M = _one_class_columns(N, 30 if tier == "W8" else 44, 7)
    M2 = 1024
    ref, tr_ref = _reference_x2(O, v, ix, nz, N, M, 0.0, M2)
    B.set_x2_tiers(tier)
    try:
        X = B.Ellpack.from_arrays(v, ix, nz, N, M)
        X2 = B.Ellpack(N, M2)
        st, tr = B.multiply_x2(X, X2, 0.0)
        counts = B.last_tier_counts()
        got = X2.download()
        X.free()
        X2.free()
    finally:
        B.set_x2_tiers()
    assert st == B.OK
    assert O.same_rows_exact(got, ref, M2, M2)
    assert tr[1] == pytest.approx(tr_ref[1], rel=1e-12)
    # the rows entered the tier and were handed on to the dense tier
    assert counts[B.X2_TIERS.index(tier)] > 0 and counts[B.X2_TIERS.index("C")] > 0, counts


def _wide_random_rows(N, lo, hi, empty, seed):
    """Rows of lo..hi random distinct columns in random order (the diagonal
    among them), values U(-1, 1)/32, and the listed rows empty: rows of B
    wider than the dense tier's 1024-entry staging unit, so one jp spans
    several units, and jps that reference an empty row."""
    rng = np.random.default_rng(seed)
    M = hi
    v = np.zeros(N * M)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    for i in range(N):
        if i in empty:
            continue
        w = int(rng.integers(lo, hi + 1))
        cols = rng.choice(np.delete(np.arange(N), i), size=w - 1, replace=False)
        cols = np.insert(cols, int(rng.integers(0, w)), i)
        v[i * M:i * M + w] = rng.uniform(-1, 1, w) / 32
        ix[i * M:i * M + w] = cols
        nz[i] = w
    return v, ix, nz, M


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE])
def test_dense_tier_multi_unit_rows(oracle_mod, prec):
    O = oracle_mod
    N = 1100
    v, ix, nz, M = _wide_random_rows(N, 1025, 1090, {3, 17, 600}, 11)
    if prec == SINGLE:
        v = v.astype(np.float32)
    M2 = N
    ref, tr_ref = _reference_x2(O, v, ix, nz, N, M, 1e-6, M2, prec=prec)
    runs = _gpu_x2((v, ix, nz), N, M, M2, 1e-6, prec=prec)
    for got, tr, counts in runs:
        assert O.same_rows_exact(got, ref, M2, M2), "rows differ from the reference"
        tol = 1e-12 if prec == DOUBLE else 1e-5
        assert tr[0] == pytest.approx(tr_ref[0], rel=tol)
        assert tr[1] == pytest.approx(tr_ref[1], rel=tol)
        assert counts[B.X2_TIERS.index("C")] > 0, counts
