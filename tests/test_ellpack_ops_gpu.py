"""Parity of every ELLPACK operation on the path, libbml_b200 (GPU) against the
reference library built from its own sources (oracle/_ref/libbml_ref.so),
on identical inputs.  Integer/index results and the order of entries within
rows must be identical; floating-point values are bit-identical wherever the
reference's arithmetic is a fixed sequence of rounded operations, and traces
(sums whose order differs) agree to 1e-12 relative."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu

DOUBLE, SINGLE = 2, 1
libc = C.CDLL(None)


def lattice(L=12, radius=3, seed=0, M=160):
    N = L ** 3
    v, ix, nz = B.gen_lattice(L, radius, N, M, seed)
    return v, ix, nz, N, M


def both(O, v, ix, nz, N, M, prec=DOUBLE):
    R = O.ref_ellpack(v, ix, nz, N, M, prec)
    G = B.Ellpack.from_arrays(v, ix, nz, N, M, prec)
    return R, G


def assert_same(O, R, G, M):
    r = O.ref_ellpack_arrays(R)
    g = G.download()
    assert np.array_equal(r[2], g[2]), "row widths differ"
    assert O.same_rows_exact(r, g, M, M), "rows differ"


def test_multiply_AB_bit_exact(oracle_mod):
    O = oracle_mod
    v1, ix1, nz1, N, M = lattice(seed=0)
    v2, ix2, nz2, _, _ = lattice(seed=7)
    Mc = 1024
    RA, GA = both(O, v1, ix1, nz1, N, M)
    RB, GB = both(O, v2, ix2, nz2, N, M)
    for thr in (0.0, 1e-4):
        RC = O.ref().bml_zero_matrix(2, DOUBLE, N, Mc, 0)
        O.ref().bml_multiply_AB(RA, RB, RC, thr)
        GC = B.Ellpack(N, Mc)
        B.lib.bml_multiply_AB(GA.h, GB.h, GC.h, thr)
        B.check()
        assert_same(O, RC, GC, Mc)
        O.ref_free(RC)


@pytest.mark.parametrize("alpha,beta,thr", [(1.2, 0.8, 0.0), (1.0, -1.0, 1e-4)])
def test_multiply_general_bit_exact(oracle_mod, alpha, beta, thr):
    """C <- alpha*A*B + beta*C, the reference's bml_multiply (the reference
    test multiply_matrix_typed.c uses alpha 1.2, beta 0.8): a product into a
    temporary, then the add."""
    O = oracle_mod
    v1, ix1, nz1, N, M = lattice(seed=0)
    v2, ix2, nz2, _, _ = lattice(seed=7)
    v3, ix3, nz3, _, _ = lattice(seed=11)
    Mc = 1024
    pad = lambda a: np.pad(a.reshape(N, M), ((0, 0), (0, Mc - M))).reshape(-1)
    RA, GA = both(O, v1, ix1, nz1, N, M)
    RB, GB = both(O, v2, ix2, nz2, N, M)
    RC, GC = both(O, pad(v3), pad(ix3), nz3, N, Mc)
    O.ref().bml_multiply(RA, RB, RC, alpha, beta, thr)
    B.lib.bml_multiply(GA.h, GB.h, GC.h, alpha, beta, thr)
    B.check()
    assert_same(O, RC, GC, Mc)
    for R in (RA, RB, RC):
        O.ref_free(R)


@pytest.mark.parametrize("alpha,beta,thr", [(2.0, -1.0, 1e-5), (1.0, 1.0, 0.0), (0.0, 0.5, 1e-3),
                                            (1.2, 0.0, 1e-2), (-0.7, 0.3, 0.0)])
def test_add_bit_exact(oracle_mod, alpha, beta, thr):
    O = oracle_mod
    v1, ix1, nz1, N, M = lattice(seed=1, M=256)
    v2, ix2, nz2, _, _ = lattice(L=12, radius=2, seed=2, M=256)
    RA, GA = both(O, v1, ix1, nz1, N, M)
    RB, GB = both(O, v2, ix2, nz2, N, M)
    O.ref().bml_add(RA, RB, alpha, beta, thr)
    B.lib.bml_add(GA.h, GB.h, alpha, beta, thr)
    B.check()
    assert_same(O, RA, GA, M)


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE])
def test_normalize_and_identity_bit_exact(oracle_mod, prec):
    O = oracle_mod
    v, ix, nz, N, M = lattice(seed=3, M=200)
    RA, GA = both(O, v, ix, nz, N, M, prec)
    rb = O.ref().bml_gershgorin(RA)
    rbounds = np.ctypeslib.as_array(C.cast(rb, C.POINTER(C.c_double)), shape=(2,)).copy()
    gb = B.lib.bml_gershgorin(GA.h)
    B.check()
    gbounds = np.ctypeslib.as_array(C.cast(gb, C.POINTER(C.c_double)), shape=(2,)).copy()
    assert np.array_equal(rbounds, gbounds)
    O.ref().bml_normalize(RA, rbounds[0], rbounds[1])
    B.lib.bml_normalize(GA.h, gbounds[0], gbounds[1])
    B.check()
    assert_same(O, RA, GA, M)
    O.ref().bml_add_identity(RA, -0.25, 1e-3)
    B.lib.bml_add_identity(GA.h, -0.25, 1e-3)
    B.check()
    assert_same(O, RA, GA, M)
    if prec == DOUBLE:
        # (for single_real the reference passes &alpha of a double to a routine
        # that reads a float, ellpack/bml_add_ellpack_typed.c:562-573, so only
        # the double form has a well-defined reference result)
        O.ref().bml_scale_add_identity(RA, 1.5, 0.125, 1e-4)
        B.lib.bml_scale_add_identity(GA.h, 1.5, 0.125, 1e-4)
        B.check()
        assert_same(O, RA, GA, M)


def test_threshold_and_traces(oracle_mod):
    O = oracle_mod
    v, ix, nz, N, M = lattice(seed=4, M=160)
    RA, GA = both(O, v, ix, nz, N, M)
    v2, ix2, nz2, _, _ = lattice(seed=5, M=160)
    RB, GB = both(O, v2, ix2, nz2, N, M)
    assert B.lib.bml_trace(GA.h) == pytest.approx(O.ref().bml_trace(RA), rel=1e-12)
    assert B.lib.bml_trace_mult(GA.h, GB.h) == pytest.approx(O.ref().bml_trace_mult(RA, RB), rel=1e-12)
    RT = O.ref().bml_threshold_new(RA, 0.02)
    GT = B.Ellpack(N, M, handle=B.lib.bml_threshold_new(GA.h, 0.02))
    assert_same(O, RT, GT, M)
    O.ref().bml_threshold(RA, 0.05)
    B.lib.bml_threshold(GA.h, 0.05)
    B.check()
    assert_same(O, RA, GA, M)


def test_transpose_same_entries(oracle_mod):
    O = oracle_mod
    # a non-symmetric input: product of two different symmetric matrices
    v1, ix1, nz1, N, M = lattice(L=10, radius=2, seed=8, M=64)
    v2, ix2, nz2, _, _ = lattice(L=10, radius=2, seed=9, M=64)
    Mc = 256
    GA, GB2 = B.Ellpack.from_arrays(v1, ix1, nz1, N, M), B.Ellpack.from_arrays(v2, ix2, nz2, N, M)
    GC = B.Ellpack(N, Mc)
    B.lib.bml_multiply_AB(GA.h, GB2.h, GC.h, 1e-6)
    B.check()
    cv, cix, cnz = GC.download()
    RC = O.ref_ellpack(cv, cix, cnz, N, Mc)
    RT = O.ref().bml_transpose_new(RC)
    GT = B.Ellpack(N, Mc, handle=B.lib.bml_transpose_new(GC.h))
    r = O.ref_ellpack_arrays(RT)
    g = GT.download()
    assert np.array_equal(r[2], g[2])
    # the reference's OpenMP transpose_new orders rows nondeterministically:
    # compare each row as a set of (column, value) pairs, values bit-exact
    for i in range(N):
        n = int(r[2][i])
        ro = np.argsort(r[1][i * Mc:i * Mc + n], kind="stable")
        go = np.argsort(g[1][i * Mc:i * Mc + n], kind="stable")
        assert np.array_equal(r[1][i * Mc:i * Mc + n][ro], g[1][i * Mc:i * Mc + n][go])
        assert np.array_equal(r[0][i * Mc:i * Mc + n][ro], g[0][i * Mc:i * Mc + n][go])
    # in-place transpose equals transpose_new as sets; twice gives back the input
    B.lib.bml_transpose(GC.h)
    B.check()
    assert np.array_equal(GC.to_dense(), GT.to_dense())
    B.lib.bml_transpose(GC.h)
    assert np.array_equal(GC.to_dense(), B.Ellpack.from_arrays(cv, cix, cnz, N, Mc).to_dense())


@pytest.mark.parametrize("thr", [0.0, 1e-5])
def test_x2_single_precision_bit_exact(oracle_mod, thr):
    O = oracle_mod
    v, ix, nz, N, M = lattice(seed=6, M=160)
    M2 = 1024
    RA, GA = both(O, v, ix, nz, N, M, SINGLE)
    R2 = O.ref().bml_zero_matrix(2, SINGLE, N, M2, 0)
    tr_ref = O.ref_x2(RA, R2, thr)
    G2 = B.Ellpack(N, M2, SINGLE)
    st, tr = B.multiply_x2(GA, G2, thr)
    assert st == B.OK
    assert_same(O, R2, G2, M2)
    # the reference sums the traces in float; this library in double
    assert tr[1] == pytest.approx(tr_ref[1], rel=1e-5)


def test_random_banded_identity_match_reference(oracle_mod):
    O = oracle_mod
    # The reference fills banded matrices inside an OpenMP parallel loop that
    # calls rand() (ellpack/bml_allocate_ellpack_typed.c:282-295), so its result
    # depends on thread scheduling; with one thread it is the serial sequence.
    gomp = C.CDLL("libgomp.so.1")
    nthreads = gomp.omp_get_max_threads()
    gomp.omp_set_num_threads(1)
    try:
        for kind, N, M in (("random", 200, 13), ("banded", 180, 9), ("identity", 64, 4)):
            libc.srand(1234)
            r = getattr(O.ref(), "bml_%s_matrix" % kind)(2, DOUBLE, N, M, 0)
            libc.srand(1234)
            g = B.Ellpack(N, M, handle=getattr(B.lib, "bml_%s_matrix" % kind)(2, DOUBLE, N, M, 0))
            assert_same(O, r, g, M)
    finally:
        gomp.omp_set_num_threads(nthreads)


def test_row_overflow_reported_not_written(oracle_mod):
    v, ix, nz, N, M = lattice(seed=0, M=160)
    X = B.Ellpack.from_arrays(v, ix, nz, N, M)
    X2 = B.Ellpack(N, 128)
    B.lib.bml_b200_set_verbose(0)
    st, _ = B.multiply_x2(X, X2, 1e-5)
    B.lib.bml_b200_set_verbose(1)
    B.clear_error()
    assert st == B.ERR_ROW_OVERFLOW
    assert B.lib.bml_b200_last_required_M() > 128
    _, _, nz2 = X2.download()
    assert nz2.max() <= 128


def test_bad_index_rejected_without_fault():
    N, M = 100, 8
    v = np.ones(N * M)
    ix = np.zeros(N * M, np.int32)
    nz = np.full(N, 2, np.int32)
    ix[5 * M + 1] = 10 ** 6  # out of range column
    X = B.Ellpack.from_arrays(v, ix, nz, N, M)
    X2 = B.Ellpack(N, M)
    B.lib.bml_b200_set_verbose(0)
    st, _ = B.multiply_x2(X, X2, 0.0)
    B.lib.bml_b200_set_verbose(1)
    B.clear_error()
    assert st == B.ERR_INVALID


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE])
def test_norms_match_reference(oracle_mod, prec):
    """bml_sum_squares, bml_fnorm and bml_fnorm2 against the reference (FP64
    sums in a different order: 1e-12 relative; the reference sums FP32
    matrices in FP32: 1e-5)."""
    O = oracle_mod
    v1, ix1, nz1, N, M = lattice(seed=2)
    v2, ix2, nz2, _, _ = lattice(seed=3, radius=2)
    # entries of B that A holds as exactly 0 count in full, as in the reference
    v1 = v1.copy()
    v1[::7] = 0.0
    RA, GA = both(O, v1, ix1, nz1, N, M, prec)
    RB, GB = both(O, v2, ix2, nz2, N, M, prec)
    ref = O.ref()
    for f in ("bml_sum_squares", "bml_fnorm", "bml_fnorm2"):
        getattr(ref, f).restype = C.c_double
    ref.bml_fnorm2.argtypes = [C.c_void_p, C.c_void_p]
    ref.bml_sum_squares.argtypes = [C.c_void_p]
    ref.bml_fnorm.argtypes = [C.c_void_p]
    tol = 1e-12 if prec == DOUBLE else 1e-5
    assert B.lib.bml_sum_squares(GA.h) == pytest.approx(ref.bml_sum_squares(RA), rel=tol)
    assert B.lib.bml_fnorm(GA.h) == pytest.approx(ref.bml_fnorm(RA), rel=tol)
    assert B.lib.bml_fnorm2(GA.h, GB.h) == pytest.approx(ref.bml_fnorm2(RA, RB), rel=tol)
    assert B.lib.bml_fnorm2(GB.h, GA.h) == pytest.approx(ref.bml_fnorm2(RB, RA), rel=tol)
    assert B.lib.bml_fnorm2(GA.h, GA.h) == 0.0
    B.check()
    for R in (RA, RB):
        O.ref_free(R)


def test_convert_between_precisions():
    """ELLPACK to ELLPACK across precisions keeps every entry in place and
    rounds its value to the new precision."""
    v, ix, nz, N, M = lattice(seed=4)
    G = B.Ellpack.from_arrays(v, ix, nz, N, M)
    F = B.Ellpack(N, M, prec=SINGLE, handle=B.lib.bml_convert(G.h, 2, SINGLE, M, 0))
    B.check()
    fv, fix, fnz = F.download()
    assert np.array_equal(fnz, nz)
    mask = (np.arange(M)[None, :] < nz[:, None]).reshape(-1)
    assert np.array_equal(fix[mask], ix[mask])
    assert np.array_equal(fv[mask], v[mask].astype(np.float32))
    D = B.Ellpack(N, M, handle=B.lib.bml_convert(F.h, 2, DOUBLE, M, 0))
    B.check()
    dv, dix, dnz = D.download()
    assert np.array_equal(dnz, nz) and np.array_equal(dix[mask], ix[mask])
    assert np.array_equal(dv[mask], fv[mask].astype(np.float64))
