"""bml_convert between ELLPACK and ELLBLOCK on the device, against the
reference library (ellblock/bml_convert_ellblock_typed.c:16-73, which builds
every one of the NB x NB blocks through bml_get_element).  The dense forms
must be bit-identical; this library stores only the blocks that hold
entries (ascending block column).  ELLBLOCK -> ELLPACK gives back the
original matrix."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu
SINGLE, DOUBLE = 1, 2
ELLPACK, ELLBLOCK = 2, 3


def _dense(export, h, N, prec):
    p = export(h, 0)
    ct = C.c_double if prec == DOUBLE else C.c_float
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(N * N,)).copy().reshape(N, N)


def _free(O, *pairs):
    for R, G in pairs:
        if R:
            r = C.c_void_p(R)
            O.ref().bml_deallocate(C.byref(r))
        if G:
            g = C.c_void_p(G)
            B.lib.bml_deallocate(C.byref(g))


@pytest.mark.parametrize("bs,L", [(4, 7), (6, 8), (32, 10)], ids=["bs4", "bs6", "bs32"])
@pytest.mark.parametrize("pin,pout", [(DOUBLE, DOUBLE), (SINGLE, SINGLE), (DOUBLE, SINGLE)],
                         ids=["fp64", "fp32", "fp64_to_fp32"])
def test_convert_ellpack_to_ellblock(oracle_mod, bs, L, pin, pout):
    O = oracle_mod
    N = L ** 3
    N -= N % bs
    M = 64
    v, ix, nz = B.gen_lattice(L, 2, N, M, 3)
    nb = N // bs
    arr = (C.c_int * nb)(*([bs] * nb))
    B.lib.bml_b200_reset_block_sizes()
    B.lib.bml_set_block_sizes(arr, nb, nb)
    O.ref().bml_set_block_sizes(arr, nb, nb)
    try:
        dt = np.float64 if pin == DOUBLE else np.float32
        RA = O.ref_ellpack(v.astype(dt), ix, nz, N, M, pin)
        GA = B.Ellpack.from_arrays(v.astype(dt), ix, nz, N, M, prec=pin)
        RB = O.ref().bml_convert(RA, ELLBLOCK, pout, N, 0) if pin == pout else None
        GB = B.lib.bml_convert(GA.h, ELLBLOCK, pout, N, 0)
        B.check()
        dg = _dense(B.lib.bml_export_to_dense, GB, N, pout)
        want = _dense(B.lib.bml_export_to_dense, GA.h, N, pin).astype(dg.dtype)
        assert np.array_equal(dg.view(np.uint8), want.view(np.uint8))
        if RB:
            dr = _dense(O.ref().bml_export_to_dense, RB, N, pout)
            assert np.array_equal(dr.view(np.uint8), dg.view(np.uint8))
        # only the blocks that hold entries are stored
        assert B.lib.bml_b200_nnz(GB) < nb * nb * bs * bs or nb <= 4
        # back to ELLPACK: the original matrix
        GE = B.lib.bml_convert(GB, ELLPACK, pout, M, 0)
        B.check()
        assert np.array_equal(_dense(B.lib.bml_export_to_dense, GE, N, pout).view(np.uint8), dg.view(np.uint8))
        # and the converted matrix computes: its X^2 is the ELLPACK one's
        if pout == DOUBLE and bs <= 6:
            X2b = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
            p = B.lib.bml_multiply_x2(GB, X2b, C.c_double(0.0))
            B.lib.bml_free_memory(C.c_void_p(p))
            B.check()
            Dx = dg.astype(np.float64)
            np.testing.assert_allclose(_dense(B.lib.bml_export_to_dense, X2b, N, DOUBLE), Dx @ Dx,
                                       rtol=0, atol=1e-12 * np.abs(Dx).sum(1).max() ** 2)
            _free(O, (None, X2b))
        _free(O, (RA, None), (RB, GB), (None, GE))
        GA.free()
    finally:
        B.lib.bml_b200_reset_block_sizes()


def test_convert_rejects_bad_columns():
    N, M = 64, 8
    v, ix, nz = B.gen_lattice(4, 1, N, M, 0)
    ix = ix.copy()
    ix[3 * M + 1] = N + 5
    B.lib.bml_b200_reset_block_sizes()
    arr = (C.c_int * 16)(*([4] * 16))
    B.lib.bml_set_block_sizes(arr, 16, 16)
    try:
        GA = B.Ellpack.from_arrays(v, ix, nz, N, M)
        B.lib.bml_b200_set_verbose(0)
        GB = B.lib.bml_convert(GA.h, ELLBLOCK, DOUBLE, N, 0)
        B.lib.bml_b200_set_verbose(1)
        assert not GB and B.lib.bml_b200_last_error() == B.ERR_INVALID
        B.lib.bml_b200_clear_error()
        GA.free()
    finally:
        B.lib.bml_b200_reset_block_sizes()
