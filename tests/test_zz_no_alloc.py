"""The allocation-free trace entry point (bml_b200_ellpack_trace_noalloc),
called through the C ABI on device arrays, agrees with bml_trace (the
library's regular, allocating trace) to the 1e-12 relative tolerance the
trace tests use, on two calls in a row (the second reuses the fixed scratch
array the first one filled).  It is for callers that cannot let the library
allocate device memory.  This file is collected last so that a failure here
stops a `-x` run only after every other test has run."""
import ctypes as C

import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu


def test_noalloc_trace_matches_bml_trace():
    import torch
    L = 20
    N, M = L ** 3, 200
    for prec in ("double_real", "single_real"):
        v, ix, nz = B.gen_lattice(L, 3, N, M, 11)
        A = B.Ellpack.from_arrays(v, ix, nz, N, M, prec)
        expected = B.lib.bml_trace(A.h)
        B.check()
        dv, di, dn, ld = C.c_void_p(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.c_int()
        B.check(B.lib.bml_b200_ellpack_device_arrays(A.h, C.byref(dv), C.byref(di), C.byref(dn), C.byref(ld)))
        out = torch.zeros(2, dtype=torch.float64, device="cuda")
        for call in range(2):
            out.zero_()
            torch.cuda.synchronize()
            st = B.lib.bml_b200_ellpack_trace_noalloc(dv, di, dn, N, ld.value, B.PREC[prec],
                                                      C.cast(C.c_void_p(out.data_ptr()), C.POINTER(C.c_double)),
                                                      None)
            assert st == B.OK, B.lib.bml_b200_error_string(st)
            torch.cuda.synchronize()
            got = out[0].item()
            assert got == pytest.approx(expected, rel=1e-12, abs=1e-12), (prec, call, got, expected)
            assert out[1].item() == 0.0  # nothing written past the output


def test_noalloc_trace_rejects_too_many_rows():
    B.lib.bml_b200_set_verbose(0)
    dummy = C.c_void_p(16)
    st = B.lib.bml_b200_ellpack_trace_noalloc(dummy, C.cast(dummy, C.POINTER(C.c_int)),
                                              C.cast(dummy, C.POINTER(C.c_int)), (1 << 19) + 1, 32, 2,
                                              C.cast(dummy, C.POINTER(C.c_double)), None)
    B.lib.bml_b200_set_verbose(1)
    B.clear_error()
    assert st == B.ERR_INVALID
