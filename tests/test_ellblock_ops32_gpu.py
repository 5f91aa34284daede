"""ELLBLOCK one-pass operations on uniform 32x32 and 64x64 block partitions,
against the reference library built from its sources.  The reference runs
these operations at any block size (only its multiply is limited to block
sizes up to 6, ellblock/bml_multiply_ellblock_typed.c:292-305,380), so the
comparison is direct and bit for bit: add (where B brings new blocks),
add_identity, scale_add_identity, in-place threshold (blocks dropped
between kept ones), scale, transpose, trace and trace_mult, in FP64 and FP32.
A block row wider than 1024 blocks checks the add's merge of long block
lists."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu
SINGLE, DOUBLE = 1, 2


def set_partition(O, bs, MB):
    arr = (C.c_int * len(bs))(*bs)
    B.lib.bml_b200_reset_block_sizes()
    B.lib.bml_set_block_sizes(arr, len(bs), MB)
    O.ref().bml_set_block_sizes(arr, len(bs), MB)


def dense(export, h, N, prec):
    p = export(h, 0)
    ct = C.c_double if prec == DOUBLE else C.c_float
    d = np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(N * N,)).copy()
    return d.reshape(N, N)


def block_matrix(nb, bs, density, seed, small_frac=0.3, dtype=np.float64):
    """Dense N x N array with a random symmetric block pattern (diagonal
    blocks always present); a fraction of the blocks scaled by 1e-4 so that
    a threshold drops whole blocks, and entries of mixed magnitude so that it
    zeroes elements inside kept blocks."""
    rng = np.random.default_rng(seed)
    N = nb * bs
    D = np.zeros((N, N))
    for a in range(nb):
        for b in range(a, nb):
            if a == b or rng.random() < density:
                blk = rng.standard_normal((bs, bs)) * np.exp(-4.0 * rng.random((bs, bs)))
                if a != b and rng.random() < small_frac:
                    blk *= 1e-4
                D[a * bs:(a + 1) * bs, b * bs:(b + 1) * bs] = blk
                D[b * bs:(b + 1) * bs, a * bs:(a + 1) * bs] = blk.T
    return D.astype(dtype)


def check_trace_mult(got, ref, DA, DB, prec):
    """tr(A B) of this library against the reference.  FP64: 1e-12
    relative.  FP32: the reference sums FP32 products in float over every
    stored block element (ellblock/bml_trace_ellblock_typed.c:69-122), so
    both are checked against the FP64 value of the same products: this
    library's within 1e-6 of S = sum |A_ij B_ji|, the reference's within
    its float summation bound n 2^-24 S."""
    if prec == DOUBLE:
        assert got == pytest.approx(ref, rel=1e-12)
        return
    T = DA.astype(np.float64) * DB.astype(np.float64).T
    exact, S, n = T.sum(), np.abs(T).sum(), np.count_nonzero(T)
    assert abs(got - exact) <= 1e-6 * S
    assert abs(ref - exact) <= n * 2.0 ** -24 * S


def both(O, D, prec, N):
    ptr = D.ctypes.data_as(C.c_void_p)
    R = O.ref().bml_import_from_dense(3, prec, 0, N, N, ptr, 0.0, 0)
    G = B.lib.bml_import_from_dense(3, prec, 0, N, N, ptr, 0.0, 0)
    B.check()
    return R, G


def free(O, *pairs):
    for R, G in pairs:
        rr, gg = C.c_void_p(R), C.c_void_p(G)
        O.ref().bml_deallocate(C.byref(rr))
        B.lib.bml_deallocate(C.byref(gg))


@pytest.mark.parametrize("bs", [32, 64])
@pytest.mark.parametrize("prec", [DOUBLE, SINGLE], ids=["fp64", "fp32"])
def test_ellblock_one_pass_ops_wide_blocks(oracle_mod, bs, prec):
    O = oracle_mod
    nb = 24 if bs == 32 else 12
    N = nb * bs
    dt = np.float64 if prec == DOUBLE else np.float32
    set_partition(O, [bs] * nb, nb)
    try:
        DA = block_matrix(nb, bs, 0.25, 1, dtype=dt)
        DB = block_matrix(nb, bs, 0.35, 2, dtype=dt)   # blocks A does not have
        (RA, GA), (RB, GB) = both(O, DA, prec, N), both(O, DB, prec, N)
        same = lambda r, g: np.array_equal(dense(O.ref().bml_export_to_dense, r, N, prec).view(np.uint8),
                                           dense(B.lib.bml_export_to_dense, g, N, prec).view(np.uint8))
        assert same(RA, GA) and same(RB, GB)
        # traces and trace_mult before the in-place operations
        assert B.lib.bml_trace(GA) == pytest.approx(O.ref().bml_trace(RA), rel=1e-12 if prec == DOUBLE else 1e-6)
        check_trace_mult(B.lib.bml_trace_mult(GA, GB), O.ref().bml_trace_mult(RA, RB), DA, DB, prec)
        # transpose (new)
        RT, GT = O.ref().bml_transpose_new(RA), B.lib.bml_transpose_new(GA)
        B.check()
        assert same(RT, GT)
        # add: A = 2 A - B, threshold 1e-3 (B's new blocks appended; small blocks dropped)
        O.ref().bml_add(RA, RB, 2.0, -1.0, 1e-3)
        B.lib.bml_add(GA, GB, 2.0, -1.0, 1e-3)
        B.check()
        assert same(RA, GA)
        # add_identity, scale_add_identity
        O.ref().bml_add_identity(RA, 0.5, 0.0)
        B.lib.bml_add_identity(GA, 0.5, 0.0)
        B.check()
        assert same(RA, GA)
        O.ref().bml_scale_add_identity(RB, 0.7, 0.25, 1e-6)
        B.lib.bml_scale_add_identity(GB, 0.7, 0.25, 1e-6)
        B.check()
        if prec == DOUBLE:
            # (the reference's single_real form reads a double's bytes as a
            # float, bml_add_ellpack_typed.c:569; only FP64 is compared)
            assert same(RB, GB)
        # in-place threshold: whole blocks dropped between kept ones, small
        # elements zeroed inside kept blocks
        O.ref().bml_threshold(RA, 5e-3)
        B.lib.bml_threshold(GA, 5e-3)
        B.check()
        assert same(RA, GA)
        # scale in place
        if prec == DOUBLE:
            s = C.c_double(-0.375)
        else:
            s = C.c_float(-0.375)
        O.ref().bml_scale_inplace(C.byref(s), RA)
        B.lib.bml_scale_inplace(C.byref(s), GA)
        B.check()
        assert same(RA, GA)
        check_trace_mult(B.lib.bml_trace_mult(GA, GT), O.ref().bml_trace_mult(RA, RT),
                         dense(B.lib.bml_export_to_dense, GA, N, prec), dense(B.lib.bml_export_to_dense, GT, N, prec),
                         prec)
        free(O, (RA, GA), (RB, GB), (RT, GT))
    finally:
        B.lib.bml_b200_reset_block_sizes()


def test_ellblock_add_block_row_wider_than_1024(oracle_mod):
    """Block row 0 of A holds all 1500 block columns, and B's rows bring
    block columns A lacks: the merged lists are longer than 1024 blocks."""
    O = oracle_mod
    nb, bs = 1500, 1
    N = nb
    set_partition(O, [bs] * nb, nb)
    try:
        rng = np.random.default_rng(4)
        DA = np.zeros((N, N))
        DB = np.zeros((N, N))
        DA[0, :] = rng.standard_normal(N)
        DA[:, 0] = DA[0, :]
        DA[np.arange(N), np.arange(N)] = 1.0
        DB[1, ::2] = rng.standard_normal((N + 1) // 2)     # 750 new blocks in row 1
        DB[2, :1200] = rng.standard_normal(1200)          # row 2: 1200 new blocks
        DB[0, ::3] = rng.standard_normal((N + 2) // 3)     # row 0: merged with A's 1500
        (RA, GA), (RB, GB) = both(O, DA, DOUBLE, N), both(O, DB, DOUBLE, N)
        O.ref().bml_add(RA, RB, 1.5, -0.5, 1e-3)
        B.lib.bml_add(GA, GB, 1.5, -0.5, 1e-3)
        B.check()
        a = dense(O.ref().bml_export_to_dense, RA, N, DOUBLE)
        g = dense(B.lib.bml_export_to_dense, GA, N, DOUBLE)
        assert np.array_equal(a.view(np.uint8), g.view(np.uint8))
        assert np.count_nonzero(g[2]) > 1024
        free(O, (RA, GA), (RB, GB))
    finally:
        B.lib.bml_b200_reset_block_sizes()
