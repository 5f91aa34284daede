"""Comparison of ELLPACK products whose sums run in different orders.

Two evaluations of C[i,k] = sum_j A[i,j] B[j,k] that form the same separately
rounded products and add them in different orders differ by at most
2 (n-1) u S[i,k], where S[i,k] = sum_j |A[i,j]| |B[j,k]| (the product
magnitudes) and n the number of products (Higham, Accuracy and Stability of
Numerical Algorithms, 2nd ed., eq. 4.4).  The tolerances below are written in
that form: |C - C_ref| <= eps S with eps = 1e-12 in FP64 (the bar for the
plain form; above the bound for n below 4500) and eps = 2 n u for FP32.
An entry kept by one side only must lie within that tolerance of the
threshold (a value on the boundary may fall either way).
"""
import numpy as np


def coo(arrs, M):
    """(keys, values) of an ELLPACK matrix: key = row * 2^32 + column, sorted."""
    v, ix, nz = arrs
    N = len(nz)
    nz = np.asarray(nz, np.int64)
    mask = np.arange(M)[None, :] < nz[:, None]
    rows = np.repeat(np.arange(N, dtype=np.int64), nz)
    cols = np.asarray(ix).reshape(N, M)[mask].astype(np.int64)
    vals = np.asarray(v).reshape(N, M)[mask].astype(np.float64)
    keys = rows * (1 << 32) + cols
    order = np.argsort(keys, kind="stable")
    return keys[order], vals[order]


def rows_sorted(arrs, M):
    """True when every row's columns are strictly ascending."""
    v, ix, nz = arrs
    N = len(nz)
    ix = np.asarray(ix).reshape(N, M)
    d = np.diff(ix, axis=1)
    ok = np.arange(M - 1)[None, :] < (np.asarray(nz)[:, None] - 1)
    return bool(np.all(d[ok] > 0))


def compare(got, ref, absum, M_got, M_ref, M_abs, thr, eps):
    """Asserts that `got` matches `ref` to eps * S entrywise (S from `absum`,
    the product |A| |B| over the same pattern, thresholded at -1) and that
    the retained patterns differ only at the threshold.  Returns a dict of
    statistics."""
    kg, vg = coo(got, M_got)
    kr, vr = coo(ref, M_ref)
    ka, sa = coo(absum, M_abs)
    assert np.all(np.diff(kg) > 0), "duplicate columns in a row of the result"
    assert np.all(np.diff(kr) > 0)

    def S(keys):
        pos = np.searchsorted(ka, keys)
        pos = np.minimum(pos, len(ka) - 1)
        assert np.all(ka[pos] == keys), "an entry outside the structural pattern of the product"
        return sa[pos]

    both, ig, ir = np.intersect1d(kg, kr, assume_unique=True, return_indices=True)
    s_both = S(both)
    err = np.abs(vg[ig] - vr[ir])
    tol = eps * s_both
    bad = err > tol
    assert not np.any(bad), "%d entries outside eps*S: worst err %.3e at S %.3e, value %.3e" % (
        int(bad.sum()), float(err[bad].max()), float(s_both[bad][np.argmax(err[bad])]),
        float(vr[ir][bad][np.argmax(err[bad])]))
    only_g = np.setdiff1d(np.arange(len(kg)), ig, assume_unique=True)
    only_r = np.setdiff1d(np.arange(len(kr)), ir, assume_unique=True)
    for keys, vals, side in ((kg[only_g], vg[only_g], "result"), (kr[only_r], vr[only_r], "reference")):
        if len(keys):
            near = np.abs(np.abs(vals) - thr) <= eps * S(keys)
            assert np.all(near), "%d entries kept only by the %s are not at the threshold" % (
                int((~near).sum()), side)
    rel = err / np.maximum(np.abs(vr[ir]), 1e-300)
    return {"entries": int(len(kr)), "common": int(len(both)), "only_result": int(len(only_g)),
            "only_reference": int(len(only_r)), "max_err_over_S": float((err / np.maximum(s_both, 1e-300)).max())
            if len(err) else 0.0, "max_rel": float(rel.max()) if len(rel) else 0.0,
            "frac_rel_le_1e-12": float(np.mean(rel <= 1e-12)) if len(rel) else 1.0}
