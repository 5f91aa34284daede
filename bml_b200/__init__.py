"""Python view of libbml_b200.so, the B200 ELLPACK/ELLBLOCK bml path.

The product is the C ABI declared in include/bml_b200.h.  This module only
loads that shared library with ctypes and declares its prototypes, so that
tests and the benchmark call exactly what a C caller links against.  There is
no Python or CPU implementation behind it: if the library is missing, import
fails.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# BML_B200_LIB names another build of the same library (e.g. one compiled with
# different tuning switches); by default the in-tree build is loaded.
LIB_PATH = os.environ.get("BML_B200_LIB") or os.path.join(HERE, "libbml_b200.so")

# enumerators of the reference's bml_types.h (same order)
TYPE = {"dense": 1, "ellpack": 2, "ellblock": 3, "csr": 4}
PREC = {"single_real": 1, "double_real": 2}
DTYPE = {1: np.float32, 2: np.float64}
SEQUENTIAL = 0
ROW_MAJOR, COL_MAJOR = 0, 1

OK = 0
ERR_NO_DEVICE, ERR_CUDA, ERR_INVALID, ERR_UNSUPPORTED, ERR_ROW_OVERFLOW, ERR_ALLOC, ERR_TIMEOUT = range(1, 8)

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "libbml_b200.so is not built (run `python bml_b200/build.py` or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

_vp, _i, _d, _ip, _dp, _sz = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t

_PROTOS = {
    # allocation / introspection
    "bml_zero_matrix": (_vp, [_i, _i, _i, _i, _i]),
    "bml_noinit_matrix": (_vp, [_i, _i, _i, _i, _i]),
    "bml_random_matrix": (_vp, [_i, _i, _i, _i, _i]),
    "bml_banded_matrix": (_vp, [_i, _i, _i, _i, _i]),
    "bml_identity_matrix": (_vp, [_i, _i, _i, _i, _i]),
    "bml_deallocate": (None, [C.POINTER(_vp)]),
    "bml_clear": (None, [_vp]),
    "bml_get_N": (_i, [_vp]),
    "bml_get_M": (_i, [_vp]),
    "bml_get_NB": (_i, [_vp]),
    "bml_get_type": (_i, [_vp]),
    "bml_get_precision": (_i, [_vp]),
    "bml_get_bandwidth": (_i, [_vp]),
    "bml_get_row_bandwidth": (_i, [_vp, _i]),
    "bml_get_sparsity": (_d, [_vp, _d]),
    "bml_allocate_memory": (_vp, [_sz]),
    "bml_free_memory": (None, [_vp]),
    # copy / import / export / elements
    "bml_copy_new": (_vp, [_vp]),
    "bml_copy": (None, [_vp, _vp]),
    "bml_convert": (_vp, [_vp, _i, _i, _i, _i]),
    "bml_import_from_dense": (_vp, [_i, _i, _i, _i, _i, _vp, _d, _i]),
    "bml_export_to_dense": (_vp, [_vp, _i]),
    "bml_get_element": (_vp, [_vp, _i, _i]),
    "bml_get_row": (_vp, [_vp, _i]),
    "bml_get_diagonal": (_vp, [_vp]),
    "bml_set_element_new": (None, [_vp, _i, _i, _vp]),
    "bml_set_element": (None, [_vp, _i, _i, _vp]),
    "bml_set_row": (None, [_vp, _i, _vp, _d]),
    "bml_set_diagonal": (None, [_vp, _vp, _d]),
    # the path
    "bml_multiply": (None, [_vp, _vp, _vp, _d, _d, _d]),
    "bml_multiply_x2": (_vp, [_vp, _vp, _d]),
    "bml_multiply_AB": (None, [_vp, _vp, _vp, _d]),
    "bml_multiply_adjust_AB": (None, [_vp, _vp, _vp, _d]),
    "bml_add": (None, [_vp, _vp, _d, _d, _d]),
    "bml_add_identity": (None, [_vp, _d, _d]),
    "bml_scale_add_identity": (None, [_vp, _d, _d, _d]),
    "bml_threshold_new": (_vp, [_vp, _d]),
    "bml_threshold": (None, [_vp, _d]),
    "bml_trace": (_d, [_vp]),
    "bml_trace_mult": (_d, [_vp, _vp]),
    "bml_sum_squares": (_d, [_vp]),
    "bml_fnorm": (_d, [_vp]),
    "bml_fnorm2": (_d, [_vp, _vp]),
    "bml_transpose_new": (_vp, [_vp]),
    "bml_transpose": (None, [_vp]),
    "bml_scale_new": (_vp, [_vp, _vp]),
    "bml_scale": (None, [_vp, _vp, _vp]),
    "bml_scale_inplace": (None, [_vp, _vp]),
    "bml_gershgorin": (_vp, [_vp]),
    "bml_normalize": (None, [_vp, _d, _d]),
    "bml_set_block_sizes": (None, [_ip, _i, _i]),
    "bml_get_block_sizes": (_ip, [_i, _i]),
    "bml_get_nb": (_i, []),
    "bml_get_mb": (_i, []),
    "bml_init": (None, []),
    "bml_shutdown": (None, []),
    "bml_write_bml_matrix": (None, [_vp, C.c_char_p]),
    "bml_read_bml_matrix": (None, [_vp, C.c_char_p]),
    # extensions
    "bml_b200_last_error": (_i, []),
    "bml_b200_error_string": (C.c_char_p, [_i]),
    "bml_b200_clear_error": (None, []),
    "bml_b200_set_verbose": (None, [_i]),
    "bml_b200_multiply_x2": (_i, [_vp, _vp, _d, _dp]),
    "bml_b200_last_required_M": (_i, []),
    "bml_b200_ellpack_upload": (_i, [_vp, _vp, _ip, _ip]),
    "bml_b200_ellpack_download": (_i, [_vp, _vp, _ip, _ip]),
    "bml_b200_ellpack_device_arrays": (_i, [_vp, C.POINTER(_vp), C.POINTER(_ip), C.POINTER(_ip), _ip]),
    "bml_b200_nnz": (C.c_longlong, [_vp]),
    "bml_b200_synchronize": (_i, []),
    "bml_b200_device_info": (_i, [_ip, _ip]),
    "bml_b200_sp2": (_i, [_vp, _vp, _d, _d, _i, _d, _i, _dp]),
    "bml_b200_sp2_mixed": (_i, [_vp, _vp, _d, _d, _i, _d, _i, _i, _dp]),
    "bml_b200_sp2_adjoint": (_i, [_vp, _vp, _d, _d, _i, _i, _i, _vp, _dp]),
    "bml_b200_multiply_x2_rows": (_i, [_vp, _vp, _d, _i, _i, _dp]),
    "bml_b200_sp2_update_rows": (_i, [_vp, _vp, _d, _i, _i, _i]),
    "bml_b200_ellblock_multiply_x2_tc": (_i, [_vp, _vp, _d, _dp]),
    "bml_b200_set_tc_split": (_i, [_i]),
    "bml_b200_gen_block_lattice": (_vp, [_i, _d, _i, C.c_ulonglong, _i]),
    "bml_b200_ellblock_sp2_mixed": (_i, [_vp, _vp, _d, _d, _i, _d, _i, _i, _dp]),
    "bml_b200_gen_chain": (_i, [_i, _i, C.c_ulonglong, _dp, _ip, _ip]),
    "bml_b200_gen_lattice": (_i, [_i, _i, _i, _i, C.c_ulonglong, _dp, _ip, _ip]),
    "bml_b200_reset_block_sizes": (None, []),
    "bml_b200_last_tier_counts": (_i, [_ip, _i]),
    "bml_b200_set_x2_tiers": (_i, [_i]),
    "bml_b200_set_x2_exact": (_i, [_i]),
    "bml_b200_set_x2_symmetric": (_i, [_i]),
    "bml_b200_last_x2_symmetric": (_i, []),
    "bml_b200_set_kernel_timing": (_i, [_i]),
    "bml_b200_set_dense_tier": (_i, [_i]),
    "bml_b200_last_x2_dense": (_i, []),
    "bml_b200_last_x2_kernel_ms": (_d, []),
    "bml_getNRanks": (_i, []),
    "bml_getMyRank": (_i, []),
    "bml_printRank": (_i, []),
    "bml_b200_set_ellblock_slab_budget": (C.c_longlong, [C.c_longlong]),
    "bml_b200_set_device": (_i, [_i]),
    "bml_b200_launch_count": (C.c_ulonglong, []),
    "bml_b200_event_record": (_i, [_i]),
    "bml_b200_event_elapsed": (_i, [_i, _i, C.POINTER(C.c_float)]),
    "bml_b200_ellpack_trace_noalloc": (_i, [_vp, _ip, _ip, _i, _i, _i, _dp, _vp]),
}

for _name, (_res, _args) in _PROTOS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_PROTOS)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def last_error():
    return lib.bml_b200_last_error()


def clear_error():
    lib.bml_b200_clear_error()


def check(status=None):
    """Raise RuntimeError if the last call failed (or `status` is non-zero)."""
    st = lib.bml_b200_last_error() if status is None else status
    if st != OK:
        msg = lib.bml_b200_error_string(st).decode()
        lib.bml_b200_clear_error()
        raise RuntimeError("bml_b200 status %d: %s" % (st, msg))


# ---------------------------------------------------------------------------
# generators (host arrays in the reference ELLPACK layout)
# ---------------------------------------------------------------------------
def gen_chain(N, M, seed=0):
    v = np.zeros(N * M, np.float64)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    r = lib.bml_b200_gen_chain(N, M, seed, _ptr(v, C.c_double), _ptr(ix, C.c_int), _ptr(nz, C.c_int))
    if r < 0:
        raise ValueError("chain generator: a row needs more than M=%d entries" % M)
    return v, ix, nz


def gen_lattice(L, radius, N, M, seed=0):
    v = np.zeros(N * M, np.float64)
    ix = np.zeros(N * M, np.int32)
    nz = np.zeros(N, np.int32)
    r = lib.bml_b200_gen_lattice(L, radius, N, M, seed, _ptr(v, C.c_double), _ptr(ix, C.c_int),
                                 _ptr(nz, C.c_int))
    if r < 0:
        raise ValueError("lattice generator: a row needs more than M=%d entries" % M)
    return v, ix, nz


# ---------------------------------------------------------------------------
# ELLPACK matrices from/to numpy
# ---------------------------------------------------------------------------
class Ellpack:
    """Owning handle on a libbml_b200 ELLPACK matrix."""

    def __init__(self, N, M, prec="double_real", handle=None):
        self.prec = PREC[prec] if isinstance(prec, str) else prec
        self.h = handle if handle is not None else lib.bml_zero_matrix(TYPE["ellpack"], self.prec, N, M, SEQUENTIAL)
        if not self.h:
            check()
            raise RuntimeError("allocation failed")
        self.N = lib.bml_get_N(self.h)
        self.M = lib.bml_get_M(self.h)

    @property
    def dtype(self):
        return DTYPE[self.prec]

    @classmethod
    def from_arrays(cls, value, index, nnz, N, M, prec="double_real"):
        A = cls(N, M, prec)
        A.upload(value, index, nnz)
        return A

    def upload(self, value, index, nnz):
        v = np.ascontiguousarray(value, dtype=self.dtype).reshape(-1)
        ix = np.ascontiguousarray(index, dtype=np.int32).reshape(-1)
        nz = np.ascontiguousarray(nnz, dtype=np.int32).reshape(-1)
        assert v.size == self.N * self.M and ix.size == self.N * self.M and nz.size == self.N
        check(lib.bml_b200_ellpack_upload(self.h, v.ctypes.data_as(C.c_void_p), _ptr(ix, C.c_int),
                                          _ptr(nz, C.c_int)))

    def download(self):
        v = np.zeros(self.N * self.M, self.dtype)
        ix = np.zeros(self.N * self.M, np.int32)
        nz = np.zeros(self.N, np.int32)
        check(lib.bml_b200_ellpack_download(self.h, v.ctypes.data_as(C.c_void_p), _ptr(ix, C.c_int),
                                            _ptr(nz, C.c_int)))
        return v, ix, nz

    def to_dense(self):
        p = lib.bml_export_to_dense(self.h, ROW_MAJOR)
        if not p:
            check()
        n = self.N * self.N
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double if self.prec == 2 else C.c_float)),
                                    shape=(n,)).copy()
        lib.bml_free_memory(p)
        return arr.reshape(self.N, self.N)

    def free(self):
        if self.h:
            h = C.c_void_p(self.h)
            lib.bml_deallocate(C.byref(h))
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def multiply_x2(X, X2, threshold):
    tr = (C.c_double * 2)()
    st = lib.bml_b200_multiply_x2(X.h, X2.h, threshold, tr)
    return st, (tr[0], tr[1])


# Multiply tiers in the order of bml_b200_last_tier_counts.
X2_TIERS = ("A", "W8", "B1", "W16", "K4", "K8", "C")


def last_tier_counts():
    out = (C.c_int * 8)()
    n = lib.bml_b200_last_tier_counts(out, 8)
    return list(out[:n])


def set_x2_tiers(*names):
    """Restrict later multiplies to the named tiers (C is always on); no
    names restores the default.  Returns the previous mask."""
    mask = 0
    for n in names:
        mask |= 1 << X2_TIERS.index(n)
    return lib.bml_b200_set_x2_tiers(mask)


def event_ms(a, b):
    ms = C.c_float()
    check(lib.bml_b200_event_elapsed(a, b, C.byref(ms)))
    return ms.value


def device_info():
    sms, dev = C.c_int(), C.c_int()
    st = lib.bml_b200_device_info(C.byref(sms), C.byref(dev))
    return st, sms.value, dev.value
