"""Parity at the headline size.

SP2 runs for 4 iterations on the 40^3 lattice Hamiltonian (N = 64000,
radius 3, M = 2048, threshold 1e-5, occupation N/2, FP64, seed 0). Two
implementations run it on the same input:

- libbml_b200 on the GPU;
- the reference library's own OpenMP CPU path (oracle/_ref, built from its
  sources).

The density matrix must match bit for bit: values, column order and row
widths. The trace must match to 1e-12 relative."""
import ctypes as C
import os

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu

L, RADIUS, MH, MX, THR, ITERS = 40, 3, 256, 2048, 1e-5, 4

# the reference's OpenMP threads hold N-long scratch arrays on their stacks
# (read when the reference library loads, after test collection)
os.environ.setdefault("OMP_STACKSIZE", "64M")


def test_sp2_40cubed_bit_exact(oracle_mod):
    O = oracle_mod
    N = L ** 3
    occ = N / 2.0
    v, ix, nz = B.gen_lattice(L, RADIUS, N, MH, 0)

    H = B.Ellpack.from_arrays(v, ix, nz, N, MH)
    D = B.Ellpack(N, MX)
    info = (C.c_double * 6)()
    st = B.lib.bml_b200_sp2(H.h, D.h, THR, occ, ITERS, -1.0, 0, info)
    assert st == B.OK, B.lib.bml_b200_error_string(st)
    got = D.download()
    H.free()
    D.free()

    # the reference's SP2 loop (bml_copy, bml_gershgorin, bml_normalize,
    # bml_multiply_x2, bml_copy / bml_add), whole padded rows of width MX
    lib = O.ref()
    pad = lambda a: np.pad(a.reshape(N, MH), ((0, 0), (0, MX - MH))).reshape(-1)
    RH = O.ref_ellpack(pad(v), pad(ix), nz, N, MX)
    RD = lib.bml_zero_matrix(2, 2, N, MX, 0)
    RX2 = lib.bml_zero_matrix(2, 2, N, MX, 0)
    lib.bml_copy(RH, RD)
    b = lib.bml_gershgorin(RH)
    bb = (C.c_double * 2).from_address(b)
    emin, emax = bb[0], bb[1]
    lib.bml_free_memory(b)
    lib.bml_normalize(RD, emin, emax)
    for _ in range(ITERS):
        tr = O.ref_x2(RD, RX2, THR)
        if abs(tr[1] - occ) <= abs(2 * tr[0] - tr[1] - occ):
            lib.bml_copy(RX2, RD)
        else:
            lib.bml_add(RD, RX2, 2.0, -1.0, THR)
    ref = O.ref_ellpack_arrays(RD)
    ref_trace = lib.bml_trace(RD)
    for m in (RH, RD, RX2):
        O.ref_free(m)

    assert int(info[0]) == ITERS
    assert np.array_equal(got[2], ref[2]), "row widths differ"
    assert int(ref[2].max()) <= MX
    assert O.same_rows_exact(got, ref, MX, MX), "density matrix differs from the reference"
    assert info[2] == pytest.approx(ref_trace, rel=1e-12)
