"""ELLBLOCK parity on the GPU against the reference library built from its
sources: block sizes irregular (1..6, the pattern of the reference's own
tests, tests/C-tests/multiply_matrix_x2_typed.c:85-111) and uniform.  Block
lists and block contents must be identical; traces agree to 1e-12."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu
DOUBLE = 2
libc = C.CDLL(None)


def partition(N, pattern_offset=5, uniform=None):
    if uniform:
        return [uniform] * (N // uniform)
    bs, count = [], 0
    for i in range(N):
        b = (pattern_offset + i) % 6 + 1
        if count + b > N:
            b = N - count
        bs.append(b)
        count += b
        if count == N:
            break
    return bs


def set_partition(O, bs, MB):
    arr = (C.c_int * len(bs))(*bs)
    B.lib.bml_b200_reset_block_sizes()
    B.lib.bml_set_block_sizes(arr, len(bs), MB)
    O.ref().bml_set_block_sizes(arr, len(bs), MB)


def dense(lib_export, h, N):
    p = lib_export(h, 0)
    d = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(N * N,)).copy()
    return d.reshape(N, N)


def random_pair(O, N, M):
    libc.srand(77)
    R = O.ref().bml_random_matrix(3, DOUBLE, N, M, 0)
    libc.srand(77)
    G = B.lib.bml_random_matrix(3, DOUBLE, N, M, 0)
    B.check()
    return R, G


def ref_export(O):
    f = O.ref().bml_export_to_dense
    return f


@pytest.mark.parametrize("uniform", [None, 4])
def test_ellblock_x2_and_traces(oracle_mod, uniform):
    O = oracle_mod
    N = 48
    bs = partition(N, uniform=uniform)
    nb = len(bs)
    set_partition(O, bs, nb)
    R, G = random_pair(O, N, N)
    assert np.array_equal(dense(ref_export(O), R, N), dense(B.lib.bml_export_to_dense, G, N))
    R2 = O.ref().bml_zero_matrix(3, DOUBLE, N, N, 0)
    G2 = B.lib.bml_zero_matrix(3, DOUBLE, N, N, 0)
    for thr in (0.0, 0.5):
        p = O.ref().bml_multiply_x2(R, R2, thr)
        rtr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2,)).copy()
        q = B.lib.bml_multiply_x2(G, G2, thr)
        B.check()
        gtr = np.ctypeslib.as_array(C.cast(q, C.POINTER(C.c_double)), shape=(2,)).copy()
        assert np.array_equal(dense(ref_export(O), R2, N), dense(B.lib.bml_export_to_dense, G2, N))
        assert gtr[0] == pytest.approx(rtr[0], rel=1e-12)
        if uniform:
            # (with irregular block sizes the reference steps the X^2 diagonal
            # with the block size of a list position, bml_multiply_ellblock_typed.c:410-414)
            assert gtr[1] == pytest.approx(rtr[1], rel=1e-12)
        else:
            assert gtr[1] == pytest.approx(np.trace(dense(ref_export(O), R2, N)), rel=1e-12)


def test_ellblock_ops(oracle_mod):
    O = oracle_mod
    N = 40
    bs = partition(N, pattern_offset=3)
    nb = len(bs)
    set_partition(O, bs, nb)
    RA, GA = random_pair(O, N, N)
    libc.srand(99)
    RB = O.ref().bml_random_matrix(3, DOUBLE, N, N, 0)
    libc.srand(99)
    GB = B.lib.bml_random_matrix(3, DOUBLE, N, N, 0)
    same = lambda r, g: np.array_equal(dense(ref_export(O), r, N), dense(B.lib.bml_export_to_dense, g, N))
    # multiply_AB, general multiply
    RC = O.ref().bml_zero_matrix(3, DOUBLE, N, N, 0)
    GC = B.lib.bml_zero_matrix(3, DOUBLE, N, N, 0)
    O.ref().bml_multiply_AB(RA, RB, RC, 0.3)
    B.lib.bml_multiply_AB(GA, GB, GC, 0.3)
    B.check()
    assert same(RC, GC)
    O.ref().bml_multiply(RA, RB, RC, 1.2, 0.8, 0.0)
    B.lib.bml_multiply(GA, GB, GC, 1.2, 0.8, 0.0)
    B.check()
    assert same(RC, GC)
    # add, add_identity, threshold, scale_add_identity
    O.ref().bml_add(RA, RB, 2.0, -1.0, 0.1)
    B.lib.bml_add(GA, GB, 2.0, -1.0, 0.1)
    B.check()
    assert same(RA, GA)
    O.ref().bml_add_identity(RA, 0.5, 0.0)
    B.lib.bml_add_identity(GA, 0.5, 0.0)
    assert same(RA, GA)
    O.ref().bml_threshold(RA, 0.4)
    B.lib.bml_threshold(GA, 0.4)
    B.check()
    assert same(RA, GA)
    # traces
    assert B.lib.bml_trace(GA) == pytest.approx(O.ref().bml_trace(RA), rel=1e-12)
    assert B.lib.bml_trace_mult(GA, GB) == pytest.approx(O.ref().bml_trace_mult(RA, RB), rel=1e-12)
    # transpose
    RT = O.ref().bml_transpose_new(RA)
    GT = B.lib.bml_transpose_new(GA)
    B.check()
    assert same(RT, GT)
    # gershgorin + normalize
    rb = O.ref().bml_gershgorin(RB)
    gb = B.lib.bml_gershgorin(GB)
    rbb = np.ctypeslib.as_array(C.cast(rb, C.POINTER(C.c_double)), shape=(2,)).copy()
    gbb = np.ctypeslib.as_array(C.cast(gb, C.POINTER(C.c_double)), shape=(2,)).copy()
    assert np.array_equal(rbb, gbb)
    O.ref().bml_normalize(RB, rbb[0], rbb[1])
    B.lib.bml_normalize(GB, gbb[0], gbb[1])
    B.check()
    assert same(RB, GB)


def test_ellblock_import_export_identity(oracle_mod):
    O = oracle_mod
    N = 32
    set_partition(O, [4] * 8, 8)
    rng = np.random.default_rng(3)
    D = rng.standard_normal((N, N))
    D[np.abs(D) < 1.0] = 0.0
    G = B.lib.bml_import_from_dense(3, DOUBLE, 0, N, N, D.ctypes.data_as(C.c_void_p), 0.5, 0)
    R = O.ref().bml_import_from_dense(3, DOUBLE, 0, N, N, D.ctypes.data_as(C.c_void_p), 0.5, 0)
    B.check()
    assert np.array_equal(dense(ref_export(O), R, N), dense(B.lib.bml_export_to_dense, G, N))
    I = B.lib.bml_identity_matrix(3, DOUBLE, N, N, 0)
    assert np.array_equal(dense(B.lib.bml_export_to_dense, I, N), np.eye(N))
