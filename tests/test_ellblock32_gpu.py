"""ELLBLOCK X^2 and A*B with uniform 32 x 32 blocks (the register-tiled
kernel) against the C restatement of bml_multiply_x2_ellblock
(ellblock/bml_multiply_ellblock_typed.c:246-442), which is pinned to the
reference at block sizes <= 6 (the reference itself cannot run 32-wide
blocks without libxsmm).

Bit-exact: every element of the product, in both precisions, and the block
lists in first-touch order.  The second stage takes the product as its left
input, so a list order that differed would change the sums.  A*B is checked
through the square of the block matrix [[0, A], [0, B]], whose upper right
part is A*B summed in the same order."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu
ELLBLOCK, DOUBLE, SINGLE = 3, 2, 1
BS = 32


def block_lattice(L, radius, seed=0, bs=BS):
    """Dense symmetric matrix of L^3 blocks of bs x bs: block (a, b) nonzero
    when the block sites are within `radius`, entries N(0,1) exp(-d)."""
    rng = np.random.default_rng(seed)
    nb = L ** 3
    pos = np.array([(x, y, z) for z in range(L) for y in range(L) for x in range(L)])
    BS = bs
    H = np.zeros((nb * BS, nb * BS))
    for a in range(nb):
        for b in range(a, nb):
            d = np.sqrt(((pos[a] - pos[b]) ** 2).sum())
            if d <= radius:
                blk = rng.standard_normal((BS, BS)) * np.exp(-d)
                if a == b:
                    blk = (blk + blk.T) / 2
                H[a * BS:(a + 1) * BS, b * BS:(b + 1) * BS] = blk
                H[b * BS:(b + 1) * BS, a * BS:(a + 1) * BS] = blk.T
    return H


def set_partition(nb, MB=None, bs=BS):
    arr = (C.c_int * nb)(*([bs] * nb))
    B.lib.bml_b200_reset_block_sizes()
    B.lib.bml_set_block_sizes(arr, nb, MB or nb)


def dt(prec):
    return np.float64 if prec == DOUBLE else np.float32


def from_dense(D, prec):
    N = D.shape[0]
    a = np.ascontiguousarray(D, dtype=dt(prec))
    h = B.lib.bml_import_from_dense(ELLBLOCK, prec, 0, N, N, a.ctypes.data_as(C.c_void_p), 0.0, 0)
    B.check()
    return h


def to_dense(h, N, prec):
    p = B.lib.bml_export_to_dense(h, 0)
    B.check()
    ct = C.c_double if prec == DOUBLE else C.c_float
    d = np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(N * N,)).copy()
    B.lib.bml_free_memory(C.c_void_p(p))
    return d.reshape(N, N)


def lists(O, h):
    """(indexb, nnzb, MB) of a matrix of this library, read from its host
    mirror (the leading struct fields are the reference's)."""
    assert B.lib.bml_get_bandwidth(h) >= 0  # brings the host mirror up to date
    st = C.cast(h, C.POINTER(O.EllblockStruct)).contents
    nnzb = np.ctypeslib.as_array(st.nnzb, shape=(st.NB,)).copy()
    indexb = np.ctypeslib.as_array(st.indexb, shape=(st.NB * st.MB,)).copy()
    return indexb, nnzb, st.MB


def rows(indexb, nnzb, MB):
    return [list(indexb[ib * MB:ib * MB + nnzb[ib]]) for ib in range(len(nnzb))]


def free(*hs):
    for h in hs:
        hh = C.c_void_p(h)
        B.lib.bml_deallocate(C.byref(hh))


def same_bits(a, b):
    return a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE])
@pytest.mark.parametrize("L,radius,thr", [(3, 1.0, 0.0), (4, 1.0, 0.05), (3, 1.8, 1e-3)])
def test_x2_blocks32_bit_exact(oracle_mod, prec, L, radius, thr):
    O = oracle_mod
    nb = L ** 3
    N = nb * BS
    H = block_lattice(L, radius).astype(dt(prec))
    set_partition(nb)
    try:
        X = from_dense(H, prec)
        X2 = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
        X4 = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
        B.check()
        p = B.lib.bml_multiply_x2(X, X2, C.c_double(thr))
        B.check()
        tr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2,)).copy()
        B.lib.bml_free_memory(C.c_void_p(p))
        ix, nz, MB = lists(O, X)
        d2, rtr, _, oix, onz = O.rest_ellblock_x2([BS] * nb, ix, nz, MB, H, thr, nb, prec=prec, lists=True)
        got2 = to_dense(X2, N, prec)
        assert same_bits(got2, d2), "X^2 differs from the restatement"
        gix, gnz, gMB = lists(O, X2)
        assert rows(gix, gnz, gMB) == rows(oix, onz, nb), "block lists differ"
        rel = 1e-12 if prec == DOUBLE else 1e-5
        assert tr[0] == pytest.approx(rtr[0], rel=rel)
        assert tr[1] == pytest.approx(rtr[1], rel=rel)

        # the transpose: blocks transposed, block rows in ascending source row
        Xt = B.lib.bml_transpose_new(X2)
        B.check()
        assert same_bits(to_dense(Xt, N, prec), np.ascontiguousarray(got2.T))
        tix, tnz, tMB = lists(O, Xt)
        src_rows = rows(gix, gnz, gMB)
        assert rows(tix, tnz, tMB) == [[ib for ib in range(nb) if jb in src_rows[ib]] for jb in range(nb)]
        free(Xt)

        # X^2 as the left input: its list order sets the order of the sums
        B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(X2, X4, C.c_double(thr))))
        B.check()
        d4, _, _ = O.rest_ellblock_x2([BS] * nb, gix, gnz, gMB, got2, thr, nb, prec=prec)
        assert same_bits(to_dense(X4, N, prec), d4), "(X^2)^2 differs from the restatement"
        free(X, X2, X4)
    finally:
        B.lib.bml_b200_reset_block_sizes()


def test_multiply_ab_blocks32_bit_exact(oracle_mod):
    O = oracle_mod
    L, thr = 3, 0.0
    nb = L ** 3
    N = nb * BS
    Ad = block_lattice(L, 1.5, seed=1)
    Bd = block_lattice(L, 1.0, seed=2)
    set_partition(nb)
    try:
        A = from_dense(Ad, DOUBLE)
        Bm = from_dense(Bd, DOUBLE)
        Cm = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
        B.check()
        B.lib.bml_multiply_AB(A, Bm, Cm, C.c_double(thr))
        B.check()
        got = to_dense(Cm, N, DOUBLE)
        ra = rows(*lists(O, A))
        rb = rows(*lists(O, Bm))
        gc = rows(*lists(O, Cm))
        free(A, Bm, Cm)
    finally:
        B.lib.bml_b200_reset_block_sizes()

    # M = [[0, A], [0, B]]: row ib of M^2 (ib < nb) sums A[ib,jb] B[jb,kb] in
    # the order of A's row, then B's row, exactly as A*B does
    M = np.zeros((2 * N, 2 * N))
    M[:N, N:] = Ad
    M[N:, N:] = Bd
    mrows = [[nb + j for j in r] for r in ra] + [[nb + k for k in r] for r in rb]
    MB = max(len(r) for r in mrows)
    indexb = np.zeros(2 * nb * MB, np.int32)
    nnzb = np.array([len(r) for r in mrows], np.int32)
    for ib, r in enumerate(mrows):
        indexb[ib * MB:ib * MB + len(r)] = r
    d2, _, _, oix, onz = O.rest_ellblock_x2([BS] * (2 * nb), indexb, nnzb, MB, M, thr, 2 * nb, lists=True)
    assert same_bits(got, np.ascontiguousarray(d2[:N, N:]))
    want = [[k - nb for k in r] for r in rows(oix, onz, 2 * nb)[:nb]]
    assert gc == want


@pytest.mark.parametrize("budget", [0, 1 << 16])
@pytest.mark.parametrize("bs", [32, 4])
def test_x2_more_block_columns_than_mb_before_threshold(oracle_mod, bs, budget):
    """Rows of X^2 that touch more block columns than the output's MB before
    thresholding, but keep at most MB (the reference's accumulator spans all
    NB): with the default slab budget every CTA has room for all NB at once;
    with a 64 KiB budget the first launch has MB + 1 slots, stops early, and
    the call runs again with NB slots on fewer CTAs.  Both give the
    restatement's blocks and lists."""
    O = oracle_mod
    L, MB = 3, 12
    nb = L ** 3
    N = nb * bs
    H = block_lattice(L, 1.0, seed=4, bs=bs)
    # a threshold that leaves at most MB blocks in every row of X^2
    d2, _, w, _, _ = O.rest_ellblock_x2([bs] * nb, *full_lists(H, nb, bs), H, 0.0, nb, lists=True)
    assert w > MB + 1  # wider than the first attempt's room before thresholding
    thr = 0.0
    for ib in range(nb):
        norms = sorted((np.abs(d2[ib * bs:(ib + 1) * bs, kb * bs:(kb + 1) * bs]).max()
                        for kb in range(nb) if kb != ib), reverse=True)
        thr = max(thr, norms[MB - 2])
    set_partition(nb, MB, bs)
    old_budget = B.lib.bml_b200_set_ellblock_slab_budget(budget)
    try:
        X = from_dense(H, DOUBLE)
        X2 = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
        B.check()
        B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(X, X2, C.c_double(thr))))
        B.check()
        ix, nz, xMB = lists(O, X)
        r2, _, _, oix, onz = O.rest_ellblock_x2([bs] * nb, ix, nz, xMB, H, thr, MB, lists=True)
        assert int(onz.max()) <= MB
        assert same_bits(to_dense(X2, N, DOUBLE), r2)
        gix, gnz, gMB = lists(O, X2)
        assert rows(gix, gnz, gMB) == rows(oix, onz, MB)
        free(X, X2)
    finally:
        B.lib.bml_b200_set_ellblock_slab_budget(old_budget)
        B.lib.bml_b200_reset_block_sizes()


def full_lists(H, nb, bs):
    """Block lists (ascending) of the nonzero blocks of H, with MB = nb."""
    indexb = np.zeros(nb * nb, np.int32)
    nnzb = np.zeros(nb, np.int32)
    for ib in range(nb):
        cols = [jb for jb in range(nb) if np.any(H[ib * bs:(ib + 1) * bs, jb * bs:(jb + 1) * bs])]
        indexb[ib * nb:ib * nb + len(cols)] = cols
        nnzb[ib] = len(cols)
    return indexb, nnzb, nb


@pytest.mark.unordered
@pytest.mark.parametrize("prec", [DOUBLE, SINGLE], ids=["fp64", "fp32"])
@pytest.mark.parametrize("L,radius", [(4, 2.0), (6, 2.24)])
def test_x2_blocks32_fused_within_bound(prec, L, radius):
    """The unordered form of the 32 x 32 block product, whose inner sums are
    fused multiply-adds, against the FP64 dense product: every entry of a
    block kept by both within 1e-12 of its product magnitude sum S (FP32:
    2 n 2^-24 S, n = 32 x the widest block row), blocks kept by one side
    only at the threshold; the same block pattern and traces otherwise."""
    import torch
    from test_ellblock_tc_gpu import _fp64_block_x2, free, from_dense, set_partition, to_dense
    thr = 1e-6
    H = block_lattice(L, radius)
    nb, N = L ** 3, H.shape[0]
    set_partition(nb, nb)
    try:
        X = from_dense(H, prec)
        X2 = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
        B.check()
        p = B.lib.bml_multiply_x2(X, X2, C.c_double(thr))
        B.check()
        tr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2,)).copy()
        B.lib.bml_free_memory(C.c_void_p(p))
        Hq = H.astype(np.float32).astype(np.float64) if prec == SINGLE else H
        want, S, keep = _fp64_block_x2(Hq, nb, thr)
        got = torch.from_numpy(to_dense(X2, N, prec)).to(want.device)
        widest = int((Hq.reshape(nb, 32, nb, 32) != 0).any(axis=(1, 3)).sum(axis=1).max())
        eps = 1e-12 if prec == DOUBLE else 2.0 * 32 * widest * 2.0 ** -24
        gkeep = got.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3)) > 0
        both = (gkeep & keep)[:, None, :, None].expand(nb, 32, nb, 32).reshape(N, N)
        err = torch.where(both, (got - want).abs(), torch.zeros((), dtype=torch.float64, device=want.device))
        ratio = float((err / S.clamp_min(1e-300)).max())
        print("fused block X^2 %d^3 %s: max |err|/S %.2e (bound %.2e)"
              % (L, "fp64" if prec == DOUBLE else "fp32", ratio, eps))
        assert ratio <= eps
        differ = gkeep ^ keep
        if bool(differ.any()):
            norm = want.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3))
            smax = S.reshape(nb, 32, nb, 32).amax(dim=(1, 3))
            assert bool(((norm[differ] - thr).abs() <= eps * smax[differ]).all())
        assert tr[1] == pytest.approx(float(torch.trace(want)), rel=eps)
        for h in (X, X2):
            free(h)
        del want, S, got, err
        torch.cuda.empty_cache()
    finally:
        B.lib.bml_b200_reset_block_sizes()
