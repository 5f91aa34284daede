"""The CPU oracle is pinned before it is trusted: the C restatement
(oracle/bml_oracle.c) must reproduce, bit for bit, the golden fixtures made
from the reference library (tests/golden/make_golden.py) and, where the
reference library is built here (oracle/_ref/libbml_ref.so), the reference
itself on further inputs.  CPU only."""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

import bml_b200 as B
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name))


def test_generators_match_digests():
    dig = json.load(open(os.path.join(GOLD, "generators.json")))
    for name, args in (("chain_4096_128", lambda: B.gen_chain(4096, 128, 0)),
                       ("lattice_40_r3_256", lambda: B.gen_lattice(40, 3, 64000, 256, 0))):
        h = hashlib.sha256()
        for a in args():
            h.update(np.ascontiguousarray(a).tobytes())
        assert h.hexdigest() == dig[name], name


def test_oracle_generators_match_digests():
    """The oracle's own generators (used where the library must not be
    loaded, as in bench.py's reference arm) give the same bytes."""
    dig = json.load(open(os.path.join(GOLD, "generators.json")))
    for name, args in (("chain_4096_128", lambda: O.gen_chain(4096, 128, 0)),
                       ("lattice_40_r3_256", lambda: O.gen_lattice(40, 3, 64000, 256, 0))):
        h = hashlib.sha256()
        for a in args():
            h.update(np.ascontiguousarray(a).tobytes())
        assert h.hexdigest() == dig[name], name
    # a truncated lattice and another seed agree with the library too
    a = O.gen_lattice(26, 3, 16384, 128, 7)
    b = B.gen_lattice(26, 3, 16384, 128, 7)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_restatement_x2_matches_golden_chain():
    g = gold("x2_chain.npz")
    N, M, M2 = 256, 64, int(g["M2"])
    v, ix, nz = B.gen_chain(N, M, 0)
    (ov, oix, onz), tr, _ = O.rest_x2(v, ix, nz, N, M, 1e-5, M2)
    assert O.same_rows_exact((ov, oix, onz), (g["value"], g["index"], g["nnz"]), M2, M2)
    assert np.array_equal(tr, g["trace"])  # single-threaded reference sums in row order


def test_restatement_x2_matches_reference_test_matrix():
    g = gold("x2_random.npz")
    (ov, oix, onz), tr, _ = O.rest_x2(g["value"], g["index"], g["nnz"], 13, 13, 0.0, 13)
    assert O.same_rows_exact((ov, oix, onz), (g["value2"], g["index2"], g["nnz2"]), 13, 13)
    # the reference test's own check: X^2 equals the dense product to 1e-12
    d = np.zeros((13, 13))
    for i in range(13):
        for p in range(g["nnz"][i]):
            d[i, g["index"][i * 13 + p]] = g["value"][i * 13 + p]
    d2 = np.zeros((13, 13))
    for i in range(13):
        for p in range(onz[i]):
            d2[i, oix[i * 13 + p]] = ov[i * 13 + p]
    assert np.abs(d2 - d @ d).max() < 1e-12


def test_restatement_sp2_matches_golden():
    g = gold("sp2_chain.npz")
    N, M = 256, int(g["M"])
    v, ix, nz = B.gen_chain(N, 64, 0)
    pad = lambda a: np.pad(a.reshape(N, 64), ((0, 0), (0, M - 64))).reshape(-1)
    (dv, dix, dnz), info = O.rest_sp2(pad(v), pad(ix), nz, N, M, 1e-5, N / 2.0, 12, 0.0, 0)
    assert info[0] == 12
    assert O.same_rows_exact((dv, dix, dnz), (g["value"], g["index"], g["nnz"]), M, M)


def test_restatement_ellblock_matches_golden():
    g = gold("ellblock_x2.npz")
    d2, tr, _ = O.rest_ellblock_x2(g["bsize"], g["indexb"], g["nnzb"], int(g["MB"]), g["dense"], 0.0,
                                   int(g["MB"]), trace_quirk=1)
    assert np.array_equal(d2, g["dense2"])
    assert tr[0] == g["trace"][0] and tr[1] == g["trace"][1]
    # the true trace of X^2 (what libbml_b200 returns) differs where block sizes vary
    _, tr_true, _ = O.rest_ellblock_x2(g["bsize"], g["indexb"], g["nnzb"], int(g["MB"]), g["dense"], 0.0,
                                       int(g["MB"]), trace_quirk=0)
    assert tr_true[1] == pytest.approx(np.trace(g["dense2"]), rel=1e-12)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(O.REF_PATH):
        pytest.skip("reference library not built (needs the reference sources)")
    return O


@pytest.mark.parametrize("thr", [0.0, 1e-5, 1e-2])
@pytest.mark.parametrize("prec", [O.DOUBLE, O.SINGLE])
def test_restatement_x2_matches_reference(ref, thr, prec):
    # (M2 = N: a row wider than M2 makes the reference exit the process,
    # bml_multiply_ellpack_typed.c:325-330 and bml_logger.c:111-115)
    for (v, ix, nz), N, M in ((B.gen_lattice(9, 3, 729, 128, 1), 729, 128), (B.gen_chain(500, 40, 2), 500, 40)):
        M2 = N
        A = ref.ref_ellpack(v, ix, nz, N, M, prec)
        R2 = ref.ref().bml_zero_matrix(2, prec, N, M2, 0)
        tr = ref.ref_x2(A, R2, thr)
        r = ref.ref_ellpack_arrays(R2)
        o, otr, _ = ref.rest_x2(v, ix, nz, N, M, thr, M2, prec)
        assert ref.same_rows_exact(r, o, M2, M2)
        assert otr[1] == pytest.approx(tr[1], rel=1e-5 if prec == O.SINGLE else 1e-12)
        ref.ref_free(A)
        ref.ref_free(R2)


@pytest.mark.parametrize("thr", [0.0, 0.5])
@pytest.mark.parametrize("prec", [O.DOUBLE, O.SINGLE])
def test_restatement_ellblock_x2_matches_reference(ref, prec, thr):
    """The ELLBLOCK X^2 restatement, in both precisions, against the
    reference's bml_multiply_x2 on block sizes 1..6 (the sizes its micro
    kernels cover): identical products and block lists."""
    N = 48
    bs, count = [], 0
    while count < N:
        b = min((5 + len(bs)) % 6 + 1, N - count)
        bs.append(b)
        count += b
    nb = len(bs)
    lib = ref.ref()
    lib.bml_set_block_sizes((C.c_int * nb)(*bs), nb, nb)
    off = np.concatenate([[0], np.cumsum(bs)])
    rng = np.random.default_rng(5)
    D = np.zeros((N, N))
    for a in range(nb):
        for b in range(nb):
            if a == b or rng.random() < 0.4:
                D[off[a]:off[a + 1], off[b]:off[b + 1]] = rng.standard_normal((bs[a], bs[b]))
    D = D.astype(O._dt(prec))
    R = lib.bml_import_from_dense(3, prec, 0, N, N, D.ctypes.data_as(C.c_void_p), 0.0, 0)
    R2 = lib.bml_zero_matrix(3, prec, N, N, 0)
    p = lib.bml_multiply_x2(R, R2, thr)
    rtr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2,)).copy()
    lib.bml_free_memory(p)
    st = C.cast(R, C.POINTER(O.EllblockStruct)).contents
    ix = np.ctypeslib.as_array(st.indexb, shape=(st.NB * st.MB,)).copy()
    nz = np.ctypeslib.as_array(st.nnzb, shape=(st.NB,)).copy()
    d2, tr, _, oix, onz = O.rest_ellblock_x2(bs, ix, nz, st.MB, D, thr, nb, trace_quirk=1, prec=prec, lists=True)
    q = lib.bml_export_to_dense(R2, 0)
    got = np.ctypeslib.as_array(C.cast(q, C.POINTER(O._ct(prec))), shape=(N * N,)).copy().reshape(N, N)
    lib.bml_free_memory(q)
    s2 = C.cast(R2, C.POINTER(O.EllblockStruct)).contents
    rix = np.ctypeslib.as_array(s2.indexb, shape=(s2.NB * s2.MB,)).copy()
    rnz = np.ctypeslib.as_array(s2.nnzb, shape=(s2.NB,)).copy()
    for h in (R, R2):
        ref.ref_free(h)
    assert np.array_equal(got.view(np.uint8), d2.view(np.uint8))
    assert np.array_equal(rnz, onz)
    for ib in range(nb):
        assert np.array_equal(rix[ib * s2.MB:ib * s2.MB + rnz[ib]], oix[ib * nb:ib * nb + onz[ib]])
    # the reference sums the traces in an OpenMP reduction, whose order
    # follows the thread count: compare within the rounding of the sum,
    # relative to the sum of the magnitudes (tr X can cancel)
    eps = 1e-12 if prec == O.DOUBLE else 1e-6
    assert abs(tr[0] - rtr[0]) <= eps * np.abs(np.diag(D).astype(np.float64)).sum()
    assert abs(tr[1] - rtr[1]) <= eps * np.abs(np.diag(d2).astype(np.float64)).sum()


def test_restatement_on_example_hamiltonian(oracle_mod):
    """The reference's example Hamiltonian (fixture from make_golden.py):
    the restatement's X^2 equals the reference's bit for bit."""
    O = oracle_mod
    g = gold("hamiltonian600.npz")
    v, ix, nz, N, M = g["value"], g["index"], g["nnz"], int(g["N"]), int(g["M"])
    assert int(nz.sum()) == 12246 and int(nz.max()) <= M
    for thr in (0.0, 1e-3, 1e-1):
        A = O.ref_ellpack(v, ix, nz, N, M)
        R = O.ref().bml_zero_matrix(2, 2, N, N, 0)
        tr_ref = O.ref_x2(A, R, thr)
        ref = O.ref_ellpack_arrays(R)
        O.ref_free(A)
        O.ref_free(R)
        got, tr, _ = O.rest_x2(v, ix, nz, N, M, thr, N)
        assert O.same_rows_exact(got, ref, N, N)
        assert tr[1] == pytest.approx(tr_ref[1], rel=1e-12)
