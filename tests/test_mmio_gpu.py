"""Matrix Market I/O (bml_write_bml_matrix / bml_read_bml_matrix) for ELLPACK
and ELLBLOCK against the reference library, and the products of the
reference's example Hamiltonian (examples/example1/hamiltonian.dat, through
the fixture tests/golden/hamiltonian600.npz).

  * the files this library writes are byte-identical to the reference's;
  * reading the reference's files gives the reference's matrix (dense forms
    bit-identical), for both formats and both real precisions;
  * a write-read round trip keeps the matrix (to the 15 significant digits
    of the reference's format);
  * a "symmetric" header mirrors off-diagonal entries (ELLPACK, as the
    reference does);
  * X^2 of the example Hamiltonian: bit-identical to the reference in the
    ordered form, within 1e-12 of the product magnitudes in the unordered
    one.
"""
import ctypes as C
import os

import numpy as np
import pytest

import bml_b200 as B
import x2check

pytestmark = pytest.mark.gpu
SINGLE, DOUBLE = 1, 2
ELLPACK, ELLBLOCK = 2, 3
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dense(export, h, N, prec):
    p = export(h, 0)
    ct = C.c_double if prec == DOUBLE else C.c_float
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(N * N,)).copy().reshape(N, N)


def _pair_from_dense(O, D, mtype, prec, M):
    N = D.shape[0]
    ptr = D.ctypes.data_as(C.c_void_p)
    R = O.ref().bml_import_from_dense(mtype, prec, 0, N, M, ptr, 0.0, 0)
    G = B.lib.bml_import_from_dense(mtype, prec, 0, N, M, ptr, 0.0, 0)
    B.check()
    return R, G


def _free(O, R=None, G=None):
    if R:
        r = C.c_void_p(R)
        O.ref().bml_deallocate(C.byref(r))
    if G:
        g = C.c_void_p(G)
        B.lib.bml_deallocate(C.byref(g))


def _set_blocks(O, bs, nb):
    arr = (C.c_int * nb)(*([bs] * nb))
    B.lib.bml_b200_reset_block_sizes()
    B.lib.bml_set_block_sizes(arr, nb, nb)
    O.ref().bml_set_block_sizes(arr, nb, nb)


def _sparse_dense(N, seed, dtype):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((N, N)) * (rng.random((N, N)) < 0.08)
    D = D + D.T + np.diag(rng.standard_normal(N))
    return D.astype(dtype)


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mtype", [ELLPACK, ELLBLOCK], ids=["ellpack", "ellblock"])
def test_write_read_match_reference(oracle_mod, tmp_path, mtype, prec):
    O = oracle_mod
    N = 96
    dt = np.float64 if prec == DOUBLE else np.float32
    if mtype == ELLBLOCK:
        _set_blocks(O, 4, N // 4)
    try:
        D = _sparse_dense(N, 3, dt)
        R, G = _pair_from_dense(O, D, mtype, prec, N)
        fr, fg = str(tmp_path / "ref.mtx"), str(tmp_path / "b200.mtx")
        O.ref().bml_write_bml_matrix(R, fr.encode())
        B.lib.bml_write_bml_matrix(G, fg.encode())
        B.check()
        assert open(fr, "rb").read() == open(fg, "rb").read(), "written files differ from the reference's"
        # read the reference's file with both libraries, into empty matrices
        R2 = O.ref().bml_zero_matrix(mtype, prec, N, N, 0)
        G2 = B.lib.bml_zero_matrix(mtype, prec, N, N, 0)
        O.ref().bml_read_bml_matrix(R2, fr.encode())
        B.lib.bml_read_bml_matrix(G2, fr.encode())
        B.check()
        dr = _dense(O.ref().bml_export_to_dense, R2, N, prec)
        dg = _dense(B.lib.bml_export_to_dense, G2, N, prec)
        assert np.array_equal(dr.view(np.uint8), dg.view(np.uint8))
        # round trip: 15 significant digits
        np.testing.assert_allclose(dg, D, rtol=1e-14 if prec == DOUBLE else 0, atol=0)
        _free(O, R, G)
        _free(O, R2, G2)
    finally:
        if mtype == ELLBLOCK:
            B.lib.bml_b200_reset_block_sizes()


def test_read_symmetric_header_ellpack(oracle_mod, tmp_path):
    """A coordinate file with a "symmetric" header holds one triangle; both
    libraries mirror its off-diagonal entries."""
    O = oracle_mod
    N = 50
    D = _sparse_dense(N, 5, np.float64)
    f = tmp_path / "sym.mtx"
    lines = ["%%MatrixMarket matrix coordinate real symmetric"]
    ent = [(i, j, D[i, j]) for i in range(N) for j in range(i + 1) if D[i, j] != 0.0]
    lines.append("%d %d %d" % (N, N, len(ent)))
    lines += ["%d %d %.17g" % (i + 1, j + 1, v) for i, j, v in ent]
    f.write_text("\n".join(lines) + "\n")
    R = O.ref().bml_zero_matrix(ELLPACK, DOUBLE, N, N, 0)
    G = B.lib.bml_zero_matrix(ELLPACK, DOUBLE, N, N, 0)
    O.ref().bml_read_bml_matrix(R, str(f).encode())
    B.lib.bml_read_bml_matrix(G, str(f).encode())
    B.check()
    dr = _dense(O.ref().bml_export_to_dense, R, N, DOUBLE)
    dg = _dense(B.lib.bml_export_to_dense, G, N, DOUBLE)
    assert np.array_equal(dr, dg)
    assert np.array_equal(dg, D)
    _free(O, R, G)


def test_read_rejects_a_size_mismatch(tmp_path):
    f = tmp_path / "m.mtx"
    f.write_text("%%MatrixMarket matrix coordinate real general\n10 10 1\n1 1 2.0\n")
    G = B.lib.bml_zero_matrix(ELLPACK, DOUBLE, 12, 12, 0)
    B.lib.bml_b200_set_verbose(0)
    B.lib.bml_read_bml_matrix(G, str(f).encode())
    B.lib.bml_b200_set_verbose(1)
    assert B.lib.bml_b200_last_error() == B.ERR_INVALID
    B.lib.bml_b200_clear_error()
    g = C.c_void_p(G)
    B.lib.bml_deallocate(C.byref(g))


def _hamiltonian():
    g = np.load(os.path.join(GOLD, "hamiltonian600.npz"))
    return g["value"], g["index"], g["nnz"], int(g["N"]), int(g["M"])


@pytest.mark.parametrize("thr", [0.0, 1e-3, 1e-1])
def test_example_hamiltonian_x2_ordered(oracle_mod, thr):
    """The reference's example Hamiltonian (thresholded at 0.05 as its
    example converts it): X^2 bit-identical to the reference library."""
    O = oracle_mod
    v, ix, nz, N, M = _hamiltonian()
    M2 = N
    A = O.ref_ellpack(v, ix, nz, N, M)
    R2 = O.ref().bml_zero_matrix(ELLPACK, DOUBLE, N, M2, 0)
    tr_ref = O.ref_x2(A, R2, thr)
    ref = O.ref_ellpack_arrays(R2)
    O.ref_free(A)
    O.ref_free(R2)
    X = B.Ellpack.from_arrays(v, ix, nz, N, M)
    X2 = B.Ellpack(N, M2)
    st, tr = B.multiply_x2(X, X2, thr)
    assert st == B.OK
    assert O.same_rows_exact(X2.download(), ref, M2, M2)
    assert tr[1] == pytest.approx(tr_ref[1], rel=1e-12)
    X.free()
    X2.free()


@pytest.mark.unordered
@pytest.mark.parametrize("thr", [0.0, 1e-3, 1e-1])
def test_example_hamiltonian_x2_unordered(oracle_mod, thr):
    O = oracle_mod
    v, ix, nz, N, M = _hamiltonian()
    M2 = N
    A = O.ref_ellpack(v, ix, nz, N, M)
    R2 = O.ref().bml_zero_matrix(ELLPACK, DOUBLE, N, M2, 0)
    tr_ref = O.ref_x2(A, R2, thr)
    ref = O.ref_ellpack_arrays(R2)
    O.ref_free(A)
    O.ref_free(R2)
    S, _, _ = O.rest_x2(np.abs(v), ix, nz, N, M, -1.0, M2)
    X = B.Ellpack.from_arrays(v, ix, nz, N, M)
    X2 = B.Ellpack(N, M2)
    st, tr = B.multiply_x2(X, X2, thr)
    assert st == B.OK
    x2check.compare(X2.download(), ref, S, M2, M2, M2, thr, 1e-12)
    assert tr[1] == pytest.approx(tr_ref[1], rel=1e-12)
    X.free()
    X2.free()
