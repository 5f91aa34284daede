"""ELLPACK parity on the GPU: libbml_b200 against the reference CPU library
(oracle/_ref/libbml_ref.so) on identical inputs.  The X^2 and A*B results
must be bit-identical, rows in the same (first-touch) order."""
import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu

DOUBLE, SINGLE = 2, 1


def _cases():
    # (name, builder) -> (value, index, nnz, N, M)
    out = []
    out.append(("chain4096", lambda: (*B.gen_chain(4096, 128, 0), 4096, 128)))
    out.append(("lattice12", lambda: (*B.gen_lattice(12, 3, 12 ** 3, 160, 0), 12 ** 3, 160)))
    out.append(("lattice_trunc", lambda: (*B.gen_lattice(10, 2, 777, 64, 3), 777, 64)))
    return out


@pytest.mark.parametrize("name,builder", _cases(), ids=[c[0] for c in _cases()])
@pytest.mark.parametrize("thr", [0.0, 1e-5, 1e-2])
def test_x2_bit_exact(oracle_mod, name, builder, thr):
    O = oracle_mod
    v, ix, nz, N, M = builder()
    M2 = 1024
    A = O.ref_ellpack(v, ix, nz, N, M)
    R2 = O.ref().bml_zero_matrix(2, DOUBLE, N, M2, 0)
    tr_ref = O.ref_x2(A, R2, thr)
    ref_out = O.ref_ellpack_arrays(R2)
    X = B.Ellpack.from_arrays(v, ix, nz, N, M)
    X2 = B.Ellpack(N, M2)
    st, tr = B.multiply_x2(X, X2, thr)
    assert st == B.OK, B.lib.bml_b200_error_string(st)
    got = X2.download()
    assert np.array_equal(got[2], ref_out[2]), "row widths differ"
    assert O.same_rows_exact(got, ref_out, M2, M2), "rows differ from the reference"
    # traces: per-row values are identical; only the summation order differs
    assert tr[0] == pytest.approx(tr_ref[0], rel=1e-12, abs=1e-12)
    assert tr[1] == pytest.approx(tr_ref[1], rel=1e-12, abs=1e-12)
    O.ref_free(A)
    O.ref_free(R2)
