"""CPU oracle loader.  TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/, both built by oracle/Makefile into
oracle/_ref/:

* libbml_ref.so    -- the reference bml C library itself, compiled from its own
                      sources (the ground truth where it runs);
* libbml_oracle.so -- bml_oracle.c, a serial C restatement of the same loops,
                      pinned against libbml_ref.so by tests/test_oracle.py and
                      used where the reference cannot run (ELLBLOCK blocks
                      larger than 6, see ellblock/bml_multiply_ellblock_typed.c:
                      292-305,380).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this
module.  The library under test never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_PATH = os.path.join(HERE, "_ref", "libbml_ref.so")
ORACLE_PATH = os.path.join(HERE, "_ref", "libbml_oracle.so")

ELLPACK, ELLBLOCK = 2, 3
SINGLE, DOUBLE = 1, 2


class EllpackStruct(C.Structure):
    """Leading fields of the reference's bml_matrix_ellpack_t
    (ellpack/bml_types_ellpack.h:11-46, built without MPI or cuSPARSE)."""
    _fields_ = [("matrix_type", C.c_int), ("matrix_precision", C.c_int),
                ("distribution_mode", C.c_int), ("N", C.c_int), ("M", C.c_int),
                ("value", C.c_void_p), ("index", C.POINTER(C.c_int)), ("nnz", C.POINTER(C.c_int)),
                ("domain", C.c_void_p), ("domain2", C.c_void_p)]


class EllblockStruct(C.Structure):
    """Leading fields of the reference's bml_matrix_ellblock_t
    (ellblock/bml_types_ellblock.h:11-54, built without the mempool or MPI)."""
    _fields_ = [("matrix_type", C.c_int), ("matrix_precision", C.c_int),
                ("distribution_mode", C.c_int), ("N", C.c_int), ("M", C.c_int),
                ("NB", C.c_int), ("MB", C.c_int),
                ("ptr_value", C.POINTER(C.c_void_p)), ("indexb", C.POINTER(C.c_int)),
                ("nnzb", C.POINTER(C.c_int)), ("bsize", C.POINTER(C.c_int)),
                ("domain", C.c_void_p), ("domain2", C.c_void_p)]


def available():
    return os.path.exists(REF_PATH) and os.path.exists(ORACLE_PATH)


_ref = None
_rest = None


def ref():
    """The reference library (ctypes), prototypes declared."""
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        protos = {
            "bml_zero_matrix": (vp, [i, i, i, i, i]),
            "bml_random_matrix": (vp, [i, i, i, i, i]),
            "bml_banded_matrix": (vp, [i, i, i, i, i]),
            "bml_identity_matrix": (vp, [i, i, i, i, i]),
            "bml_import_from_dense": (vp, [i, i, i, i, i, vp, d, i]),
            "bml_export_to_dense": (vp, [vp, i]),
            "bml_deallocate": (None, [C.POINTER(vp)]),
            "bml_copy_new": (vp, [vp]),
            "bml_copy": (None, [vp, vp]),
            "bml_multiply_x2": (vp, [vp, vp, d]),
            "bml_multiply": (None, [vp, vp, vp, d, d, d]),
            "bml_multiply_AB": (None, [vp, vp, vp, d]),
            "bml_add": (None, [vp, vp, d, d, d]),
            "bml_add_identity": (None, [vp, d, d]),
            "bml_scale_add_identity": (None, [vp, d, d, d]),
            "bml_scale_inplace": (None, [vp, vp]),
            "bml_threshold": (None, [vp, d]),
            "bml_threshold_new": (vp, [vp, d]),
            "bml_trace": (d, [vp]),
            "bml_trace_mult": (d, [vp, vp]),
            "bml_transpose_new": (vp, [vp]),
            "bml_transpose": (None, [vp]),
            "bml_gershgorin": (vp, [vp]),
            "bml_normalize": (None, [vp, d, d]),
            "bml_free_memory": (None, [vp]),
            "bml_set_block_sizes": (None, [C.POINTER(i), i, i]),
            "bml_get_N": (i, [vp]),
            "bml_get_M": (i, [vp]),
            "bml_convert": (vp, [vp, i, i, i, i]),
            "bml_write_bml_matrix": (None, [vp, C.c_char_p]),
            "bml_read_bml_matrix": (None, [vp, C.c_char_p]),
        }
        for name, (res, args) in protos.items():
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        _ref = lib
    return _ref


def rest():
    """The C restatement (ctypes)."""
    global _rest
    if _rest is None:
        _rest = C.CDLL(ORACLE_PATH)
    return _rest


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _dt(prec):
    return np.float64 if prec == DOUBLE else np.float32


def _ct(prec):
    return C.c_double if prec == DOUBLE else C.c_float


# ---------------------------------------------------------------------------
# reference ELLPACK matrices <-> numpy
# ---------------------------------------------------------------------------
def ref_ellpack(value, index, nnz, N, M, prec=DOUBLE):
    """A reference ELLPACK matrix holding the given host arrays."""
    lib = ref()
    A = lib.bml_zero_matrix(ELLPACK, prec, N, M, 0)
    s = C.cast(A, C.POINTER(EllpackStruct)).contents
    v = np.ascontiguousarray(value, dtype=_dt(prec)).reshape(-1)
    ix = np.ascontiguousarray(index, dtype=np.int32).reshape(-1)
    nz = np.ascontiguousarray(nnz, dtype=np.int32).reshape(-1)
    C.memmove(s.value, v.ctypes.data, v.nbytes)
    C.memmove(s.index, ix.ctypes.data, ix.nbytes)
    C.memmove(s.nnz, nz.ctypes.data, nz.nbytes)
    return A


def ref_ellpack_arrays(A):
    s = C.cast(A, C.POINTER(EllpackStruct)).contents
    N, M, prec = s.N, s.M, s.matrix_precision
    v = np.ctypeslib.as_array(C.cast(s.value, C.POINTER(_ct(prec))), shape=(N * M,)).copy()
    ix = np.ctypeslib.as_array(s.index, shape=(N * M,)).copy()
    nz = np.ctypeslib.as_array(s.nnz, shape=(N,)).copy()
    return v, ix, nz


def ref_free(A):
    h = C.c_void_p(A)
    ref().bml_deallocate(C.byref(h))


def ref_x2(X, X2, thr):
    lib = ref()
    p = lib.bml_multiply_x2(X, X2, thr)
    tr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2,)).copy()
    lib.bml_free_memory(p)
    return tr


def ref_to_dense(A, n):
    lib = ref()
    prec = C.cast(A, C.POINTER(EllpackStruct)).contents.matrix_precision
    p = lib.bml_export_to_dense(A, 0)
    d = np.ctypeslib.as_array(C.cast(p, C.POINTER(_ct(prec))), shape=(n * n,)).copy()
    lib.bml_free_memory(p)
    return d.reshape(n, n)


# ---------------------------------------------------------------------------
# restatement wrappers (double precision unless noted)
# ---------------------------------------------------------------------------
def rest_x2(v, ix, nz, N, M, thr, M2, prec=DOUBLE):
    lib = rest()
    dt, ct = _dt(prec), _ct(prec)
    v = np.ascontiguousarray(v, dt)
    ix = np.ascontiguousarray(ix, np.int32)
    nz = np.ascontiguousarray(nz, np.int32)
    v2 = np.zeros(N * M2, dt)
    ix2 = np.zeros(N * M2, np.int32)
    nz2 = np.zeros(N, np.int32)
    tr = np.zeros(2)
    f = lib.oracle_ellpack_x2_d if prec == DOUBLE else lib.oracle_ellpack_x2_f
    f.restype = C.c_int
    w = f(N, M, _p(v, ct), _p(ix, C.c_int), _p(nz, C.c_int), C.c_double(thr), M2, _p(v2, ct),
          _p(ix2, C.c_int), _p(nz2, C.c_int), _p(tr, C.c_double))
    return (v2, ix2, nz2), tr, w


def rest_sp2(v, ix, nz, N, M, thr, occ, maxiter, tol, stall):
    lib = rest()
    dv = np.zeros(N * M)
    dix = np.zeros(N * M, np.int32)
    dnz = np.zeros(N, np.int32)
    info = np.zeros(6)
    v = np.ascontiguousarray(v, np.float64)
    ix = np.ascontiguousarray(ix, np.int32)
    nz = np.ascontiguousarray(nz, np.int32)
    lib.oracle_ellpack_sp2_d.restype = C.c_int
    lib.oracle_ellpack_sp2_d(N, M, _p(v, C.c_double), _p(ix, C.c_int), _p(nz, C.c_int),
                             C.c_double(thr), C.c_double(occ), maxiter, C.c_double(tol), stall,
                             _p(dv, C.c_double), _p(dix, C.c_int), _p(dnz, C.c_int),
                             _p(info, C.c_double))
    return (dv, dix, dnz), info


# ---------------------------------------------------------------------------
# seeded inputs without the library under test (bml_oracle_gen.c)
# ---------------------------------------------------------------------------
def gen_chain(N, M, seed=0):
    """The 1-D chain Hamiltonian, reference ELLPACK host layout."""
    v = np.zeros(N * M, np.float64)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    f = rest().oracle_gen_chain
    f.restype = C.c_int
    if f(N, M, C.c_ulonglong(seed), _p(v, C.c_double), _p(ix, C.c_int), _p(nz, C.c_int)) < 0:
        raise ValueError("chain generator: a row needs more than M=%d entries" % M)
    return v, ix, nz


def gen_lattice(L, radius, N, M, seed=0):
    """The L^3 lattice Hamiltonian (first N sites), reference ELLPACK host layout."""
    v = np.zeros(N * M, np.float64)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    f = rest().oracle_gen_lattice
    f.restype = C.c_int
    if f(L, radius, N, M, C.c_ulonglong(seed), _p(v, C.c_double), _p(ix, C.c_int), _p(nz, C.c_int)) < 0:
        raise ValueError("lattice generator: a row needs more than M=%d entries" % M)
    return v, ix, nz


# ---------------------------------------------------------------------------
# comparison helpers
# ---------------------------------------------------------------------------
def rows(v, ix, nz, M):
    """List of per-row (index array, value array) in stored order."""
    out = []
    for i in range(len(nz)):
        n = int(nz[i])
        out.append((ix[i * M:i * M + n].copy(), v[i * M:i * M + n].copy()))
    return out


def same_rows_exact(a, b, Ma, Mb):
    """True when both ELLPACK matrices hold identical rows: same nnz, same
    column order, bit-identical values."""
    va, ia, na = a
    vb, ib, nb = b
    if not np.array_equal(na, nb):
        return False
    for i in range(len(na)):
        n = int(na[i])
        if not np.array_equal(ia[i * Ma:i * Ma + n], ib[i * Mb:i * Mb + n]):
            return False
        if not np.array_equal(va[i * Ma:i * Ma + n].view(np.uint8), vb[i * Mb:i * Mb + n].view(np.uint8)):
            return False
    return True


def rest_ellblock_x2(bsize, indexb, nnzb, MB, dense, thr, MB2, trace_quirk=0, prec=DOUBLE, lists=False):
    """ELLBLOCK X^2 by the restatement; blocks of `dense` at the positions the
    block lists name, in the matrix precision `prec`.  Returns (dense X^2,
    traces, widest block row), and with lists=True also the output block
    lists (indexb[NB*MB2], nnzb[NB])."""
    lib = rest()
    dt, ct = _dt(prec), _ct(prec)
    bsize = np.asarray(bsize, np.int32)
    NB = len(bsize)
    off = np.concatenate([[0], np.cumsum(bsize)])
    maxbs = int(bsize.max())
    pool = np.zeros((NB * MB, maxbs * maxbs), dt)
    for ib in range(NB):
        for jp in range(int(nnzb[ib])):
            jb = int(indexb[ib * MB + jp])
            blk = dense[off[ib]:off[ib + 1], off[jb]:off[jb + 1]]
            pool[ib * MB + jp, :blk.size] = blk.reshape(-1)
    out = np.zeros((NB * MB2, maxbs * maxbs), dt)
    ptrs = (C.POINTER(ct) * (NB * MB))(*[pool[q].ctypes.data_as(C.POINTER(ct)) for q in range(NB * MB)])
    optrs = (C.POINTER(ct) * (NB * MB2))(*[out[q].ctypes.data_as(C.POINTER(ct)) for q in range(NB * MB2)])
    oix = np.zeros(NB * MB2, np.int32)
    onz = np.zeros(NB, np.int32)
    tr = np.zeros(2)
    ib_ = np.ascontiguousarray(indexb, np.int32)
    nb_ = np.ascontiguousarray(nnzb, np.int32)
    fn = lib.oracle_ellblock_x2_d if prec == DOUBLE else lib.oracle_ellblock_x2_s
    fn.restype = C.c_int
    w = fn(NB, MB, _p(bsize, C.c_int), ptrs, _p(ib_, C.c_int), _p(nb_, C.c_int), C.c_double(thr), MB2, optrs,
           _p(oix, C.c_int), _p(onz, C.c_int), _p(tr, C.c_double), trace_quirk)
    N = int(off[-1])
    d2 = np.zeros((N, N), dt)
    for ib in range(NB):
        for jp in range(int(onz[ib])):
            jb = int(oix[ib * MB2 + jp])
            r, c = bsize[ib], bsize[jb]
            d2[off[ib]:off[ib + 1], off[jb]:off[jb + 1]] = out[ib * MB2 + jp, :r * c].reshape(r, c)
    if lists:
        return d2, tr, w, oix, onz
    return d2, tr, w
