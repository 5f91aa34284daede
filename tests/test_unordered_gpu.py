"""The unordered ELLPACK product (the library's default form) against the
reference CPU library (oracle/_ref/libbml_ref.so) on identical inputs.

The unordered kernel forms the reference's products and applies its keep
rule, but adds the products of one entry in no fixed order and writes each
row in ascending column order.  Checked here, with the bound stated in
tests/x2check.py:
  * values: |C - C_ref| <= eps S, S = sum_j |A_ij B_jk|, eps = 1e-12 (FP64),
    2 n 2^-24 (FP32, n = widest row of A);
  * pattern: identical except entries within that bound of the threshold;
  * traces: tr A within 1e-12 relative, tr C within eps sum_i S_ii;
  * rows strictly ascending.
"""
import numpy as np
import pytest

import bml_b200 as B
import x2check

pytestmark = [pytest.mark.gpu, pytest.mark.unordered]

DOUBLE, SINGLE = 2, 1


def _cases():
    out = []
    out.append(("chain4096", lambda: (*B.gen_chain(4096, 128, 0), 4096, 128)))
    out.append(("lattice12", lambda: (*B.gen_lattice(12, 3, 12 ** 3, 160, 0), 12 ** 3, 160)))
    out.append(("lattice_trunc", lambda: (*B.gen_lattice(10, 2, 777, 64, 3), 777, 64)))
    return out


def _ref_x2(O, v, ix, nz, N, M, thr, M2, prec=DOUBLE):
    A = O.ref_ellpack(v, ix, nz, N, M, prec)
    R = O.ref().bml_zero_matrix(2, prec, N, M2, 0)
    tr = O.ref_x2(A, R, thr)
    out = O.ref_ellpack_arrays(R)
    O.ref_free(A)
    O.ref_free(R)
    return out, tr


def _absum(O, v, ix, nz, N, M, M2):
    """S = |X| |X| over the structural pattern of X^2 (every touched column)."""
    out, _, w = O.rest_x2(np.abs(v), ix, nz, N, M, -1.0, M2)
    assert w <= M2
    return out


def _gpu_x2(v, ix, nz, N, M, M2, thr, prec=DOUBLE):
    X = B.Ellpack.from_arrays(v, ix, nz, N, M, prec=prec)
    X2 = B.Ellpack(N, M2, prec=prec)
    st, tr = B.multiply_x2(X, X2, thr)
    assert st == B.OK, B.lib.bml_b200_error_string(st)
    got = X2.download()
    X.free()
    X2.free()
    return got, tr


def _diag_S(absum, M, N):
    v, ix, nz = absum
    tot = 0.0
    for i in range(N):
        r = ix[i * M:i * M + nz[i]]
        hit = np.nonzero(r == i)[0]
        if len(hit):
            tot += v[i * M + hit[0]]
    return tot


@pytest.mark.parametrize("name,builder", _cases(), ids=[c[0] for c in _cases()])
@pytest.mark.parametrize("thr", [0.0, 1e-5, 1e-2])
def test_x2_unordered_fp64(oracle_mod, name, builder, thr):
    O = oracle_mod
    v, ix, nz, N, M = builder()
    M2 = min(N, 2048)
    ref, tr_ref = _ref_x2(O, v, ix, nz, N, M, thr, M2)
    S = _absum(O, v, ix, nz, N, M, M2)
    got, tr = _gpu_x2(v, ix, nz, N, M, M2, thr)
    st = x2check.compare(got, ref, S, M2, M2, M2, thr, 1e-12)
    assert x2check.rows_sorted(got, M2)
    assert tr[0] == pytest.approx(tr_ref[0], rel=1e-12, abs=1e-12)
    assert abs(tr[1] - tr_ref[1]) <= 1e-12 * _diag_S(S, M2, N)
    assert st["only_result"] + st["only_reference"] <= max(2, st["entries"] // 100000)


@pytest.mark.parametrize("name,builder", _cases(), ids=[c[0] for c in _cases()])
def test_x2_unordered_fp32(oracle_mod, name, builder):
    O = oracle_mod
    v, ix, nz, N, M = builder()
    v = v.astype(np.float32)
    thr = 1e-5
    M2 = min(N, 2048)
    ref, tr_ref = _ref_x2(O, v, ix, nz, N, M, thr, M2, prec=SINGLE)
    S = _absum(O, v.astype(np.float64), ix, nz, N, M, M2)
    got, tr = _gpu_x2(v, ix, nz, N, M, M2, thr, prec="single_real")
    eps = 2.0 * int(nz.max()) * 2.0 ** -24
    x2check.compare(got, ref, S, M2, M2, M2, thr, eps)
    assert x2check.rows_sorted(got, M2)
    # the reference sums its FP32 traces in float, row after row
    assert tr[1] == pytest.approx(tr_ref[1], rel=1e-5)


def _random_sparse(N, per_row, span, seed, shuffle):
    """Symmetric random pattern: row i holds the diagonal and columns drawn
    from [i - span, i + span]; values N(0, 1)/per_row.  shuffle: store
    each row in a random order (not ascending)."""
    rng = np.random.default_rng(seed)
    cols = [set([i]) for i in range(N)]
    for i in range(N):
        for c in rng.integers(max(0, i - span), min(N, i + span + 1), per_row // 2):
            cols[i].add(int(c))
            cols[int(c)].add(i)
    M = max(len(c) for c in cols)
    M = (M + 31) // 32 * 32
    v = np.zeros(N * M)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    vals = {}
    for i in range(N):
        row = sorted(cols[i])
        if shuffle:
            rng.shuffle(row)
        for p, c in enumerate(row):
            key = (min(i, c), max(i, c))
            if key not in vals:
                vals[key] = rng.standard_normal() / per_row
            v[i * M + p] = vals[key]
            ix[i * M + p] = c
        nz[i] = len(row)
    return v, ix, nz, M


@pytest.mark.parametrize("shuffle", [False, True], ids=["sorted_rows", "unsorted_rows"])
def test_x2_unordered_wide_span_tiles(oracle_mod, shuffle):
    """Rows whose product columns span far more than one accumulator tile
    (the window then runs in tiles with per-row cursors), with B's rows
    stored sorted or shuffled (the prep kernel sorts a copy)."""
    O = oracle_mod
    N = 60000
    v, ix, nz, M = _random_sparse(N, 24, 40000, 5, shuffle)
    M2 = 1024
    thr = 1e-4
    ref, tr_ref = _ref_x2(O, v, ix, nz, N, M, thr, M2)
    S = _absum(O, v, ix, nz, N, M, M2)
    got, tr = _gpu_x2(v, ix, nz, N, M, M2, thr)
    x2check.compare(got, ref, S, M2, M2, M2, thr, 1e-12)
    assert x2check.rows_sorted(got, M2)
    assert tr[0] == pytest.approx(tr_ref[0], rel=1e-12)


def test_x2_unordered_negative_threshold_keeps_all_touched(oracle_mod):
    """thr < 0 keeps every touched column, zeros included (the touched
    bitmap form of the kernel)."""
    O = oracle_mod
    v, ix, nz = B.gen_lattice(10, 2, 1000, 64, 1)
    N, M = 1000, 64
    v = v.reshape(N, M)
    v[:, 1::3] = 0.0  # structural zeros: products that sum to exactly 0
    v = v.reshape(-1)
    M2 = 512
    ref, _ = _ref_x2(O, v, ix, nz, N, M, -1.0, M2)
    S = _absum(O, v, ix, nz, N, M, M2)
    got, _ = _gpu_x2(v, ix, nz, N, M, M2, -1.0)
    st = x2check.compare(got, ref, S, M2, M2, M2, -1.0, 1e-12)
    assert st["only_result"] == 0 and st["only_reference"] == 0
    assert np.array_equal(got[2], ref[2])


def test_x2_unordered_empty_rows(oracle_mod):
    O = oracle_mod
    N, M = 3000, 64
    v, ix, nz = B.gen_lattice(15, 2, N, M, 2)
    nz = nz.copy()
    nz[::7] = 0      # empty rows of X
    M2 = 512
    ref, tr_ref = _ref_x2(O, v, ix, nz, N, M, 1e-6, M2)
    S = _absum(O, v, ix, nz, N, M, M2)
    got, tr = _gpu_x2(v, ix, nz, N, M, M2, 1e-6)
    x2check.compare(got, ref, S, M2, M2, M2, 1e-6, 1e-12)
    assert np.all(got[2][::7] == 0)
    assert tr[0] == pytest.approx(tr_ref[0], rel=1e-12)


def test_x2_unordered_overflow_and_bad_input():
    """A result row wider than M is reported without writing past M; an
    out-of-range column is rejected."""
    N, M = 1728, 160
    v, ix, nz = B.gen_lattice(12, 3, N, M, 0)
    X = B.Ellpack.from_arrays(v, ix, nz, N, M)
    X2 = B.Ellpack(N, 200)
    st, _ = B.multiply_x2(X, X2, 0.0)
    assert st == B.ERR_ROW_OVERFLOW
    got = X2.download()
    assert got[2].max() <= 200
    need = B.lib.bml_b200_last_required_M()
    assert need > 200
    ix2 = ix.copy()
    ix2[5 * M + 3] = N + 7
    Y = B.Ellpack.from_arrays(v, ix2, nz, N, M)
    Y2 = B.Ellpack(N, 1024)
    st, _ = B.multiply_x2(Y, Y2, 0.0)
    assert st == B.ERR_INVALID
    B.lib.bml_b200_clear_error()  # the status is sticky until cleared
    for m in (X, X2, Y, Y2):
        m.free()


def test_multiply_general_unordered(oracle_mod):
    """C = alpha A B + beta C (alpha 1.2, beta 0.8, the reference test's
    values) with A != B: the unordered A*B followed by the add."""
    O = oracle_mod
    N, M = 1000, 64
    a = B.gen_lattice(10, 2, N, M, 11)
    b = B.gen_lattice(10, 2, N, M, 12)
    c = B.gen_lattice(10, 2, N, M, 13)
    thr, M2 = 1e-6, 512
    pad = lambda arr: (np.pad(arr[0].reshape(N, M), ((0, 0), (0, M2 - M))).reshape(-1),
                       np.pad(arr[1].reshape(N, M), ((0, 0), (0, M2 - M))).reshape(-1), arr[2])
    RA = O.ref_ellpack(*a, N, M)
    RB = O.ref_ellpack(*b, N, M)
    RC = O.ref_ellpack(*pad(c), N, M2)
    O.ref().bml_multiply(RA, RB, RC, 1.2, 0.8, thr)
    ref = O.ref_ellpack_arrays(RC)
    for h in (RA, RB, RC):
        O.ref_free(h)
    GA = B.Ellpack.from_arrays(*a, N, M)
    GB = B.Ellpack.from_arrays(*b, N, M)
    GC = B.Ellpack.from_arrays(*pad(c), N, M2)
    B.lib.bml_multiply(GA.h, GB.h, GC.h, 1.2, 0.8, thr)
    B.check()
    got = GC.download()
    # S of alpha A B + beta C: |alpha| |A| |B| + |beta| |C| on every column
    d = lambda arr, m: _dense(arr, N, m)
    Sd = 1.2 * np.abs(d(a, M)) @ np.abs(d(b, M)) + 0.8 * np.abs(d(c, M))
    gd, rd = d(got, M2), d(ref, M2)
    err = np.abs(gd - rd)
    assert np.all(err <= 1e-12 * Sd + 1e-300)
    only = (gd != 0) ^ (rd != 0)
    assert np.all(np.abs(np.abs(np.where(gd != 0, gd, rd)[only]) - thr) <= 1e-12 * Sd[only])
    for m in (GA, GB, GC):
        m.free()


def _dense(arr, N, M):
    v, ix, nz = arr
    D = np.zeros((N, N))
    for i in range(N):
        n = nz[i]
        np.add.at(D[i], ix[i * M:i * M + n], v[i * M:i * M + n])
    return D


def _dense_of(arrs, N, M):
    v, ix, nz = arrs
    D = np.zeros((N, N))
    for i in range(N):
        n = nz[i]
        D[i, ix[i * M:i * M + n]] = v[i * M:i * M + n]
    return D


def test_x2_symmetric_form(oracle_mod):
    """A symmetric X takes the symmetric form (upper half formed, mirrored):
    the result is exactly symmetric, within the bound of the reference's,
    and within the bound of the full form's."""
    O = oracle_mod
    N, M = 12 ** 3, 160
    v, ix, nz = B.gen_lattice(12, 3, N, M, 0)
    M2 = N
    ref, tr_ref = _ref_x2(O, v, ix, nz, N, M, 1e-5, M2)
    S = _absum(O, v, ix, nz, N, M, M2)
    got, tr = _gpu_x2(v, ix, nz, N, M, M2, 1e-5)
    assert B.lib.bml_b200_last_x2_symmetric() == 1
    D = _dense_of(got, N, M2)
    assert np.array_equal(D, D.T), "the symmetric form's X^2 is not exactly symmetric"
    x2check.compare(got, ref, S, M2, M2, M2, 1e-5, 1e-12)
    assert x2check.rows_sorted(got, M2)
    old = B.lib.bml_b200_set_x2_symmetric(0)
    try:
        full, trf = _gpu_x2(v, ix, nz, N, M, M2, 1e-5)
        assert B.lib.bml_b200_last_x2_symmetric() == 0
    finally:
        B.lib.bml_b200_set_x2_symmetric(old)
    x2check.compare(got, full, S, M2, M2, M2, 1e-5, 1e-12)
    assert tr[1] == pytest.approx(trf[1], rel=1e-12)


def test_x2_nonsymmetric_input_takes_full_form(oracle_mod):
    """One entry off its mirror by one ulp: the check finds it and the full
    product runs, still within the bound of the reference's."""
    O = oracle_mod
    N, M = 12 ** 3, 160
    v, ix, nz = B.gen_lattice(12, 3, N, M, 0)
    v = v.copy()
    v[100 * M + 5] = np.nextafter(v[100 * M + 5], np.inf)
    M2 = N
    ref, _ = _ref_x2(O, v, ix, nz, N, M, 1e-5, M2)
    S = _absum(O, v, ix, nz, N, M, M2)
    got, _ = _gpu_x2(v, ix, nz, N, M, M2, 1e-5)
    assert B.lib.bml_b200_last_x2_symmetric() == 0
    x2check.compare(got, ref, S, M2, M2, M2, 1e-5, 1e-12)


def test_sp2_unordered_against_ordered():
    """SP2 on the 12^3 lattice (threshold 1e-5, 12 iterations): the iterates
    stay exactly symmetric, every X^2 takes the symmetric form (the dense tier
    once the rows fill in), and the result
    agrees with the ordered (reference-identical) solve: trace and band
    energy to 1e-10 relative, ||D - D_ordered||_F / ||D_ordered||_F to 1e-9
    (entries at the threshold may fall either way)."""
    import ctypes as C
    N, M = 12 ** 3, 12 ** 3
    v, ix, nz = B.gen_lattice(12, 3, N, 160, 0)
    pad = lambda a: np.pad(a.reshape(N, 160), ((0, 0), (0, M - 160))).reshape(-1)
    H = B.Ellpack.from_arrays(pad(v), pad(ix), nz, N, M)
    out = {}
    for exact in (1, 0):
        old = B.lib.bml_b200_set_x2_exact(exact)
        try:
            D = B.Ellpack(N, M)
            info = (C.c_double * 6)()
            assert B.lib.bml_b200_sp2(H.h, D.h, 1e-5, N / 2.0, 12, -1.0, 0, info) == B.OK
            # the last X^2 of the unordered solve: the symmetric form, or the
            # dense tier once the iterates have filled in (its GEMM keeps a
            # symmetric X^2 exactly symmetric too)
            out[exact] = (D, list(info),
                          B.lib.bml_b200_last_x2_symmetric() or B.lib.bml_b200_last_x2_dense())
        finally:
            B.lib.bml_b200_set_x2_exact(old)
    (Do, io, _), (Du, iu, symu) = out[1], out[0]
    assert symu == 1
    Dd = _dense_of(Du.download(), N, M)
    assert np.array_equal(Dd, Dd.T)
    assert iu[2] == pytest.approx(io[2], rel=1e-10)
    eo, eu = B.lib.bml_trace_mult(Do.h, H.h), B.lib.bml_trace_mult(Du.h, H.h)
    assert eu == pytest.approx(eo, rel=1e-10)
    assert B.lib.bml_fnorm2(Du.h, Do.h) <= 1e-9 * B.lib.bml_fnorm(Do.h)
    B.check()
