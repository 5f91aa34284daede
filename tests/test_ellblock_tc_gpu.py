"""ELLBLOCK X^2 on the tensor cores (scaled FP16 hi/lo split, FP32 accumulation)
against the matrix-precision block product of bml_multiply_x2.

Bounds: the split represents each entry to about 2^-17 of its size, and the
products are summed in FP32, so entries of X^2 agree to 2e-5 of the largest
entry and the traces to 2e-5 relative.  Blocks of 32 x 32 on a block lattice
(entries N(0,1) exp(-d), neighbours within a radius), as in the mixed
ELLBLOCK configuration."""
import ctypes as C

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu
ELLBLOCK, DOUBLE, SINGLE = 3, 2, 1


def block_lattice(L, radius, seed=0, bs=32):
    """Dense symmetric matrix of L^3 blocks of bs x bs: block (a, b) nonzero
    when the block sites are within `radius`, entries N(0,1) exp(-d)."""
    rng = np.random.default_rng(seed)
    nb = L ** 3
    pos = np.array([(x, y, z) for z in range(L) for y in range(L) for x in range(L)])
    N = nb * bs
    H = np.zeros((N, N))
    for a in range(nb):
        for b in range(a, nb):
            d = np.sqrt(((pos[a] - pos[b]) ** 2).sum())
            if d <= radius:
                blk = rng.standard_normal((bs, bs)) * np.exp(-d)
                if a == b:
                    blk = (blk + blk.T) / 2
                H[a * bs:(a + 1) * bs, b * bs:(b + 1) * bs] = blk
                H[b * bs:(b + 1) * bs, a * bs:(a + 1) * bs] = blk.T
    return H


def set_partition(nb, MB, bs=32):
    arr = (C.c_int * nb)(*([bs] * nb))
    B.lib.bml_b200_reset_block_sizes()
    B.lib.bml_set_block_sizes(arr, nb, MB)


def from_dense(D, prec=DOUBLE):
    N = D.shape[0]
    a = np.ascontiguousarray(D, dtype=np.float64 if prec == DOUBLE else np.float32)
    h = B.lib.bml_import_from_dense(ELLBLOCK, prec, 0, N, N, a.ctypes.data_as(C.c_void_p), 0.0, 0)
    B.check()
    return h


def to_dense(h, N, prec=DOUBLE):
    p = B.lib.bml_export_to_dense(h, 0)
    B.check()
    d = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double if prec == DOUBLE else C.c_float)),
                              shape=(N * N,)).copy()
    B.lib.bml_free_memory(C.c_void_p(p))
    return d.reshape(N, N).astype(np.float64)


def free(h):
    hh = C.c_void_p(h)
    B.lib.bml_deallocate(C.byref(hh))


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE])
# (6, 2.24): 57 block neighbours, about 7000 block products per group of four
# block rows
@pytest.mark.parametrize("L,radius", [(3, 1.0), (4, 2.0), (6, 2.24)])
def test_tc_x2_matches_block_product(prec, L, radius):
    H = block_lattice(L, radius)
    nb, N = L ** 3, H.shape[0]
    set_partition(nb, nb)
    try:
        X = from_dense(H, prec)
        Xe = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
        Xt = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
        B.check()
        tre = B.lib.bml_multiply_x2(X, Xe, C.c_double(1e-6))
        tre = np.ctypeslib.as_array(C.cast(tre, C.POINTER(C.c_double)), shape=(2,)).copy()
        trt = (C.c_double * 2)()
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X, Xt, 1e-6, trt)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        de, dt = to_dense(Xe, N, prec), to_dense(Xt, N, prec)
        scale = np.abs(de).max()
        assert np.abs(dt - de).max() <= 2e-5 * scale
        assert trt[0] == pytest.approx(tre[0], rel=1e-6)
        assert trt[1] == pytest.approx(tre[1], rel=2e-5)
        # a second call on the same inputs gives the same result
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X, Xt, 1e-6, trt)
        assert st == B.OK
        assert np.array_equal(to_dense(Xt, N, prec), dt)
        for h in (X, Xe, Xt):
            free(h)
    finally:
        B.lib.bml_b200_reset_block_sizes()


def _fp64_block_x2(H, nb, thr, bs=32):
    """FP64 oracle of the ELLBLOCK X^2: the dense product H H in FP64 (torch,
    on the GPU), restricted to the structural block pattern of the product
    and to the reference's block keep rule (block (ib, kb) kept when kb == ib
    or its max-norm exceeds thr, ellblock/bml_multiply_ellblock_typed.c:
    406-408).  Also returns S = |H| |H|, the product magnitudes."""
    import torch
    dev = torch.device("cuda")
    Ht = torch.from_numpy(H).to(dev)
    P = (Ht.reshape(nb, bs, nb, bs).abs().amax(dim=(1, 3)) > 0).to(torch.float64)
    pattern = (P @ P) > 0
    X2 = Ht @ Ht
    S = Ht.abs() @ Ht.abs()
    del Ht
    norm = X2.reshape(nb, bs, nb, bs).abs().amax(dim=(1, 3))
    keep = pattern & ((norm > thr) | torch.eye(nb, dtype=torch.bool, device=dev))
    mask = keep[:, None, :, None].expand(nb, bs, nb, bs).reshape(nb * bs, nb * bs)
    X2 = torch.where(mask, X2, torch.zeros((), dtype=torch.float64, device=dev))
    return X2, S, keep


# Bound: the FP16 hi/lo split holds every entry to about 2^-22 of its size,
# and the tensor cores accumulate in FP32, so an entry of X^2 carries an error
# of a few 2^-24 of its product magnitude sum S = (|H| |H|)_ik for each of the
# up to 32 * 57 terms summed; asserted: |X2_tc - X2_fp64| <= 2e-5 * S.  A block
# that one side keeps and the other drops has its max-norm within that error of
# the threshold.
TC_EPS = 2e-5


@pytest.mark.parametrize("L,radius", [(3, 1.0), (4, 2.0), (6, 2.24), (10, 2.0)])
def test_tc_x2_against_fp64_dense(L, radius):
    import torch
    thr = 1e-6
    H = block_lattice(L, radius)
    nb, N = L ** 3, H.shape[0]
    set_partition(nb, 257 if L == 10 else nb)
    try:
        X = from_dense(H)
        Xt = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
        B.check()
        trt = (C.c_double * 2)()
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X, Xt, thr, trt)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        want, S, keep = _fp64_block_x2(H, nb, thr)
        got = torch.from_numpy(to_dense(Xt, N)).to(want.device)
        gkeep = got.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3)) > 0
        both = (gkeep & keep)[:, None, :, None].expand(nb, 32, nb, 32).reshape(N, N)
        err = torch.where(both, (got - want).abs(), torch.zeros((), dtype=torch.float64, device=want.device))
        ratio = float((err / S.clamp_min(1e-300)).max())
        rel_to_max = float(err.max() / want.abs().max())
        print("tc X^2 %d^3: max |err|/S %.2e, max |err|/max|X2| %.2e" % (L, ratio, rel_to_max))
        assert ratio <= TC_EPS
        differ = gkeep ^ keep
        if bool(differ.any()):
            # blocks kept by one side only: their max-norm sits at the threshold
            norm = want.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3))
            smax = S.reshape(nb, 32, nb, 32).amax(dim=(1, 3))
            assert bool(((norm[differ] - thr).abs() <= TC_EPS * smax[differ]).all())
        assert trt[1] == pytest.approx(float(torch.trace(want)), rel=TC_EPS)
        for h in (X, Xt):
            free(h)
        del want, S, got, err
        torch.cuda.empty_cache()
    finally:
        B.lib.bml_b200_reset_block_sizes()


@pytest.mark.parametrize("L,radius", [(6, 2.0), (8, 2.0)])
def test_tc_x2_of_a_filled_iterate(L, radius):
    """X^2 of X1 = H^2 (the exact block product at 1e-6), whose rows hold up
    to every block of a radius-4 neighbourhood: groups of four block rows
    with hundreds of block columns and tens of thousands of block pairs, as
    in the later SP2 iterations.  Against the FP64 dense product of X1, with
    the bound grown with the number of FP32 accumulation steps per tile
    (measured at 6^3: 4.4e-5 of S with rows of 152 blocks)."""
    import torch
    thr = 1e-6
    H = block_lattice(L, radius, seed=5)
    nb, N = L ** 3, H.shape[0]
    set_partition(nb, nb)
    try:
        X = from_dense(H)
        X1 = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
        Xt = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
        B.check()
        B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(X, X1, C.c_double(thr))))
        B.check()
        X1d = to_dense(X1, N)
        widest = int((X1d.reshape(nb, 32, nb, 32).any(axis=(1, 3))).sum(axis=1).max())
        trt = (C.c_double * 2)()
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X1, Xt, thr, trt)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        want, S, keep = _fp64_block_x2(X1d, nb, thr)
        got = torch.from_numpy(to_dense(Xt, N)).to(want.device)
        gkeep = got.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3)) > 0
        both = (gkeep & keep)[:, None, :, None].expand(nb, 32, nb, 32).reshape(N, N)
        err = torch.where(both, (got - want).abs(), torch.zeros((), dtype=torch.float64, device=want.device))
        ratio = float((err / S.clamp_min(1e-300)).max())
        # an output tile accumulates up to `widest` pairs, six FP32 steps
        # each (two K = 16 halves of hi*hi, hi*lo and lo*hi), each step
        # within one unit in the last place (2^-23) of the running sum <= S
        eps = 6 * widest * 2.0 ** -23
        print("tc X^2 of X1 at %d^3 (widest row of X1: %d blocks): max |err|/S %.2e (bound %.2e)"
              % (L, widest, ratio, eps))
        assert widest > 100
        assert ratio <= eps
        differ = gkeep ^ keep
        if bool(differ.any()):
            norm = want.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3))
            smax = S.reshape(nb, 32, nb, 32).amax(dim=(1, 3))
            assert bool(((norm[differ] - thr).abs() <= eps * smax[differ]).all())
        assert trt[1] == pytest.approx(float(torch.trace(want)), rel=eps)
        for h in (X, X1, Xt):
            free(h)
        del want, S, got, err
        torch.cuda.empty_cache()
    finally:
        B.lib.bml_b200_reset_block_sizes()


def test_tc_rejects_other_block_sizes():
    set_partition(16, 16, bs=8)
    try:
        X = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, 128, 128, 0)
        X2 = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, 128, 128, 0)
        B.lib.bml_b200_set_verbose(0)
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X, X2, 1e-6, None)
        B.lib.bml_b200_set_verbose(1)
        assert st == B.ERR_UNSUPPORTED
        B.clear_error()
        free(X)
        free(X2)
    finally:
        B.lib.bml_b200_reset_block_sizes()


def test_ellblock_sp2_mixed_against_fp64():
    """bml_b200_ellblock_sp2_mixed: bulk SP2 iterations on the tensor-core X^2,
    the last two on the matrix-precision block product, against the same
    solve with every iteration exact (nclose = maxiter).  On the 4^3 block
    lattice (N = 2048, radius 2), all eight bulk iterations run on the
    tensor cores.  Tolerances: trace,
    band energy tr(DH) and ||D - D_exact||_F / ||D_exact||_F within 1e-4
    (the split carries about 1e-5 relative per X^2)."""
    L, radius, iters, nclose, thr = 4, 2.0, 10, 2, 1e-6
    Hd = block_lattice(L, radius, seed=3)
    nb, N = L ** 3, Hd.shape[0]
    set_partition(nb, nb)
    try:
        H = from_dense(Hd)
        out = {}
        for name, nc in (("exact", iters), ("mixed", nclose)):
            D = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
            info = (C.c_double * 8)()
            st = B.lib.bml_b200_ellblock_sp2_mixed(H, D, thr, N / 2.0, iters, -1.0, 0, nc, info)
            assert st == B.OK, B.lib.bml_b200_error_string(st)
            out[name] = (to_dense(D, N), list(info))
            free(D)
        (De, ie), (Dm, im) = out["exact"], out["mixed"]
        assert ie[0] == im[0] == iters
        assert ie[6] == 0 and im[6] == iters - nclose  # iterations on the tensor cores
        tr_e, tr_m = np.trace(De), np.trace(Dm)
        en_e, en_m = np.sum(De * Hd.T), np.sum(Dm * Hd.T)
        fro = np.linalg.norm(Dm - De) / np.linalg.norm(De)
        print("ellblock mixed SP2: trace err %.2e, energy err %.2e, ||dD||/||D|| %.2e"
              % (abs(tr_m - tr_e) / abs(tr_e), abs(en_m - en_e) / abs(en_e), fro))
        assert abs(tr_m - tr_e) <= 1e-4 * abs(tr_e)
        assert abs(en_m - en_e) <= 1e-4 * abs(en_e)
        assert fro <= 1e-4
        free(H)
    finally:
        B.lib.bml_b200_reset_block_sizes()


@pytest.mark.xfail(reason="the FP16 split accumulates in FP32 in tensor memory: the mixed ELLBLOCK SP2 is about "
                          "3e-5 from the exact solve in trace (5e-6 in band energy); the 8-bit split meets the target "
                          "(test_ellblock_sp2_mixed_8bit_meets_the_1e6_target)",
                   strict=False)
def test_ellblock_sp2_mixed_meets_the_1e6_target():
    """The mixed form's target (trace and band energy within 1e-6 of the
    exact solve) on the 4^3 block lattice, 8 tensor-core + 2 exact
    iterations, with the FP16 split: an expected failure, its accumulation
    is FP32."""
    L, radius, iters, nclose, thr = 4, 2.0, 10, 2, 1e-6
    Hd = block_lattice(L, radius, seed=3)
    nb, N = L ** 3, Hd.shape[0]
    set_partition(nb, nb)
    try:
        H = from_dense(Hd)
        res = {}
        for name, nc in (("exact", iters), ("mixed", nclose)):
            D = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
            info = (C.c_double * 8)()
            assert B.lib.bml_b200_ellblock_sp2_mixed(H, D, thr, N / 2.0, iters, -1.0, 0, nc, info) == B.OK
            res[name] = to_dense(D, N)
            free(D)
        free(H)
        De, Dm = res["exact"], res["mixed"]
        assert abs(np.trace(Dm) - np.trace(De)) <= 1e-6 * abs(np.trace(De))
        assert abs(np.sum(Dm * Hd.T) - np.sum(De * Hd.T)) <= 1e-6 * abs(np.sum(De * Hd.T))
    finally:
        B.lib.bml_b200_reset_block_sizes()


def _split_scales(D, nb, bs=32):
    """Per scalar row and column, the power of two just above the largest
    |entry| (1 for an empty row): the 8-bit split's sigma_r and tau_c."""
    def p2(m):
        e = np.frexp(m)[1].astype(np.float64)
        return np.where(m > 0, np.ldexp(1.0, e.astype(int)), 1.0)
    return p2(np.abs(D).max(axis=1)), p2(np.abs(D).max(axis=0))


@pytest.mark.parametrize("prec", [DOUBLE, SINGLE], ids=["fp64", "fp32"])
@pytest.mark.parametrize("L,radius,wide", [(4, 2.0, False), (6, 2.24, False), (6, 2.0, True)])
def test_tc_x2_8bit_split_against_fp64_dense(prec, L, radius, wide):
    """The 8-bit split (bml_b200_set_tc_split(1)): five slices leave each
    product term within about 2^-33 sigma_r tau_c (2^-35 per operand, plus
    the dropped slice products of order >= 7), and the INT32 sums are exact,
    so |X2_tc - X2_fp64| <= 32 P_IK 2^-31 sigma_r tau_c + 1e-15 S, with P_IK
    the block pairs of output block (I, K) and a factor 4 of margin.  On H
    and (wide) on X1 = H^2."""
    import torch
    thr = 1e-6
    H = block_lattice(L, radius, seed=7)
    nb, N = L ** 3, H.shape[0]
    set_partition(nb, nb)
    old = B.lib.bml_b200_set_tc_split(1)
    try:
        X = from_dense(H, prec)
        if wide:
            X1 = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
            B.check()
            B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(X, X1, C.c_double(thr))))
            B.check()
            free(X)
            X = X1
        Xd = to_dense(X, N, prec)
        Xt = B.lib.bml_zero_matrix(ELLBLOCK, prec, N, N, 0)
        B.check()
        trt = (C.c_double * 2)()
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X, Xt, thr, trt)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        want, S, keep = _fp64_block_x2(Xd, nb, thr)
        got = torch.from_numpy(to_dense(Xt, N, prec)).to(want.device)
        sig, tau = _split_scales(Xd, nb)
        P = torch.from_numpy((Xd.reshape(nb, 32, nb, 32) != 0).any(axis=(1, 3)).astype(np.float64)).to(want.device)
        pairs = (P @ P)[:, None, :, None].expand(nb, 32, nb, 32).reshape(N, N)
        bound = 32 * pairs * 2.0 ** -31 * torch.outer(torch.from_numpy(sig), torch.from_numpy(tau)).to(want.device)
        bound = bound + 1e-15 * S
        if prec == SINGLE:
            bound = bound + 2.0 ** -24 * want.abs()  # the result's rounding to FP32
        gkeep = got.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3)) > 0
        both = (gkeep & keep)[:, None, :, None].expand(nb, 32, nb, 32).reshape(N, N)
        err = torch.where(both, (got - want).abs(), torch.zeros((), dtype=torch.float64, device=want.device))
        ratio = float(torch.where(bound > 0, err / bound.clamp_min(1e-300), err).max())
        rel_s = float((err / S.clamp_min(1e-300)).max())
        print("tc 8-bit X^2 %d^3%s %s: max err/bound %.2e, max |err|/S %.2e"
              % (L, " (X1)" if wide else "", "fp64" if prec == DOUBLE else "fp32", ratio, rel_s))
        assert ratio <= 1.0
        differ = gkeep ^ keep
        if bool(differ.any()):
            norm = want.reshape(nb, 32, nb, 32).abs().amax(dim=(1, 3))
            bmax = bound.reshape(nb, 32, nb, 32).amax(dim=(1, 3))
            assert bool(((norm[differ] - thr).abs() <= bmax[differ]).all())
        assert abs(trt[1] - float(torch.trace(want))) <= float(torch.diagonal(bound).sum())
        for h in (X, Xt):
            free(h)
        del want, S, got, err, bound, pairs
        torch.cuda.empty_cache()
    finally:
        B.lib.bml_b200_set_tc_split(old)
        B.lib.bml_b200_reset_block_sizes()


@pytest.mark.parametrize("nclose", [2, 1])
def test_ellblock_sp2_mixed_8bit_meets_the_1e6_target(nclose):
    """The mixed ELLBLOCK SP2 with the 8-bit split in its bulk iterations
    (exact INT32 accumulation) and 2 or 1 exact closing ones, 10 in all, on
    the 4^3 block lattice: trace and band energy within 1e-6 of the
    all-exact solve."""
    L, radius, iters, thr = 4, 2.0, 10, 1e-6
    Hd = block_lattice(L, radius, seed=3)
    nb, N = L ** 3, Hd.shape[0]
    set_partition(nb, nb)
    old = B.lib.bml_b200_set_tc_split(1)
    try:
        H = from_dense(Hd)
        res = {}
        for name, nc in (("exact", iters), ("mixed", nclose)):
            D = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
            info = (C.c_double * 8)()
            assert B.lib.bml_b200_ellblock_sp2_mixed(H, D, thr, N / 2.0, iters, -1.0, 0, nc, info) == B.OK
            res[name] = (to_dense(D, N), list(info))
            free(D)
        free(H)
        (De, ie), (Dm, im) = res["exact"], res["mixed"]
        assert im[6] == iters - nclose
        tr_err = abs(np.trace(Dm) - np.trace(De)) / abs(np.trace(De))
        en_err = abs(np.sum(Dm * Hd.T) - np.sum(De * Hd.T)) / abs(np.sum(De * Hd.T))
        print("ellblock mixed SP2, 8-bit split, %d closing: trace err %.2e, energy err %.2e"
              % (nclose, tr_err, en_err))
        assert tr_err <= 1e-6
        assert en_err <= 1e-6
    finally:
        B.lib.bml_b200_set_tc_split(old)
        B.lib.bml_b200_reset_block_sizes()


@pytest.mark.parametrize("split", [0, 1], ids=["fp16", "8bit"])
def test_tc_x2_empty_block_rows_and_ragged_groups(split):
    """Block rows with no blocks at all (rows and columns 5, 6 and the last
    of a 3^3 block lattice emptied) and NB = 27, not a multiple of the four
    block rows a group takes: the empty rows come out empty, the others as
    the FP64 dense product (FP16 split within 2e-5 of S; 8-bit split, whose
    bound is relative to the row and column scales, within 1e-7 of S:
    measured 1e-8 on these lattices)."""
    import torch
    thr = 1e-6
    H = block_lattice(3, 1.8, seed=11)
    nb, N = 27, H.shape[0]
    for b in (5, 6, 26):
        H[b * 32:(b + 1) * 32, :] = 0.0
        H[:, b * 32:(b + 1) * 32] = 0.0
    set_partition(nb, nb)
    old = B.lib.bml_b200_set_tc_split(split)
    try:
        X = from_dense(H)
        Xt = B.lib.bml_zero_matrix(ELLBLOCK, DOUBLE, N, N, 0)
        B.check()
        st = B.lib.bml_b200_ellblock_multiply_x2_tc(X, Xt, thr, None)
        assert st == B.OK, B.lib.bml_b200_error_string(st)
        want, S, keep = _fp64_block_x2(H, nb, thr)
        got = torch.from_numpy(to_dense(Xt, N)).to(want.device)
        for b in (5, 6, 26):
            assert float(got[b * 32:(b + 1) * 32, :].abs().max()) == 0.0
        eps = 2e-5 if split == 0 else 1e-7
        err = (got - want).abs()
        assert float((err / S.clamp_min(1e-300)).max()) <= eps
        for h in (X, Xt):
            free(h)
    finally:
        B.lib.bml_b200_set_tc_split(old)
        B.lib.bml_b200_reset_block_sizes()
