"""The SP2 adjoint (bml_b200_sp2_adjoint): dL/dH for L = sum_ij D_ij V_ij,
D after a fixed number of SP2 iterations from H.

A thin torch.autograd.Function (here, in the tests only) exposes the C-ABI
call as a differentiable function of H's stored values.  Its gradient is
checked against
  - an FP64 dense reference: the same SP2 map written with dense torch
    tensors (Gershgorin bounds, thresholds and branch choices as in the
    library) and differentiated by torch autograd; compared on H's pattern
    to 1e-8 relative to the largest entry;
  - central finite differences (step 1e-6) of the library's own forward
    solve, on 32 entries, to 1e-6 (of the entry for the largest ones, of the
    largest entry for the rest).
Checkpoint intervals of 1, 4 and the full count must give the same gradient."""
import ctypes as C

import numpy as np
import pytest
import torch

import bml_b200 as B

pytestmark = pytest.mark.gpu

THR = 1e-5


def _problem(L=6, radius=2, seed=0, M=None):
    N = L ** 3
    MH = 64
    v, ix, nz = B.gen_lattice(L, radius, N, MH, seed)
    M = M or N
    pad = lambda a: np.pad(a.reshape(N, MH), ((0, 0), (0, M - MH))).reshape(-1)
    v, ix = pad(v), pad(ix)
    rng = np.random.default_rng(seed + 11)
    # V: symmetric, on H's pattern, U[-0.01, 0.01]
    dense_v = np.zeros((N, N))
    for i in range(N):
        for p in range(nz[i]):
            j = ix[i * M + p]
            if j >= i:
                x = rng.uniform(-0.01, 0.01)
                dense_v[i, j] = dense_v[j, i] = x
    vv = np.zeros(N * M)
    for i in range(N):
        for p in range(nz[i]):
            vv[i * M + p] = dense_v[i, ix[i * M + p]]
    return N, M, v, ix, nz, vv, dense_v


def _loss_and_grad(hv, ix, nz, vv, N, M, iters, every):
    H = B.Ellpack.from_arrays(hv, ix, nz, N, M)
    V = B.Ellpack.from_arrays(vv, ix, nz, N, M)
    dH = B.Ellpack(N, M)
    loss = C.c_double()
    st = B.lib.bml_b200_sp2_adjoint(H.h, V.h, THR, N / 2.0, iters, every, M, dH.h, C.byref(loss))
    assert st == B.OK, B.lib.bml_b200_error_string(st)
    g = dH.download()
    for m in (H, V, dH):
        m.free()
    return loss.value, g


def _loss_only(hv, ix, nz, vv, N, M, iters):
    H = B.Ellpack.from_arrays(hv, ix, nz, N, M)
    V = B.Ellpack.from_arrays(vv, ix, nz, N, M)
    D = B.Ellpack(N, M)
    info = (C.c_double * 6)()
    assert B.lib.bml_b200_sp2(H.h, D.h, THR, N / 2.0, iters, -1.0, 0, info) == B.OK
    val = B.lib.bml_trace_mult(D.h, V.h)
    for m in (H, V, D):
        m.free()
    return val


class SP2Response(torch.autograd.Function):
    """L(H) = sum_ij D(H)_ij V_ij as a function of H's stored values."""

    @staticmethod
    def forward(ctx, hvals, ix, nz, vv, N, M, iters, every):
        loss, (gv, gix, gnz) = _loss_and_grad(hvals.detach().cpu().numpy(), ix, nz, vv, N, M, iters, every)
        assert np.array_equal(gnz, nz) and np.array_equal(gix, ix)
        ctx.save_for_backward(torch.from_numpy(gv))
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        (g,) = ctx.saved_tensors
        return gout * g, None, None, None, None, None, None, None


def _dense_reference_grad(H, Vd, iters):
    """FP64 dense SP2 with the library's rules, differentiated by autograd."""
    Ht = torch.tensor(H, dtype=torch.float64, requires_grad=True)
    n = Ht.shape[0]
    eye = torch.eye(n, dtype=torch.float64)
    d = torch.diagonal(Ht)
    r = Ht.abs().sum(1) - d.abs()
    emax = torch.max(d + r)
    emin = torch.min(d - r)
    X = (emax * eye - Ht) / (emax - emin)
    occ = n / 2.0
    for _ in range(iters):
        X2 = X @ X
        with torch.no_grad():
            keep = ((X2.abs() > THR) | (eye > 0)).double()
        X2 = X2 * keep
        t, t2 = torch.trace(X).item(), torch.trace(X2).item()
        if abs(t2 - occ) <= abs(2 * t - t2 - occ):
            X = X2
        else:
            Y = 2 * X - X2
            with torch.no_grad():
                keep2 = (Y.abs() > THR).double()
            X = Y * keep2
    loss = (X * torch.tensor(Vd)).sum()
    loss.backward()
    return loss.item(), Ht.grad.numpy()


def _dense(v, ix, nz, N, M):
    H = np.zeros((N, N))
    for i in range(N):
        for p in range(nz[i]):
            H[i, ix[i * M + p]] = v[i * M + p]
    return H


@pytest.mark.parametrize("iters,every", [(12, 4), (12, 1), (12, 12)])
def test_adjoint_matches_dense_autograd(iters, every):
    N, M, v, ix, nz, vv, Vd = _problem()
    h = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    loss = SP2Response.apply(h, ix, nz, vv, N, M, iters, every)
    loss.backward()
    g = h.grad.numpy()
    ref_loss, ref_grad = _dense_reference_grad(_dense(v, ix, nz, N, M), Vd, iters)
    assert loss.item() == pytest.approx(ref_loss, rel=1e-10)
    mask = (np.arange(M)[None, :] < nz[:, None]).reshape(-1)
    rows = np.repeat(np.arange(N), M)
    ref_on_pattern = ref_grad[rows[mask], ix[mask]]
    scale = np.abs(ref_on_pattern).max()
    assert scale > 0
    assert np.abs(g[mask] - ref_on_pattern).max() <= 1e-8 * scale


@pytest.mark.unordered
@pytest.mark.parametrize("every", [4, 1])
def test_adjoint_unordered_matches_dense_autograd(every):
    """The unordered form, whose backward products are formed only on the
    iterates' patterns (the masked products): against the dense FP64
    autograd reference to the same 1e-8, and against the ordered form's
    gradient to 1e-10 of the largest entry (the two add products in other
    orders)."""
    iters = 12
    N, M, v, ix, nz, vv, Vd = _problem()
    loss_u, (g_u, _, _) = _loss_and_grad(v, ix, nz, vv, N, M, iters, every)
    old = B.lib.bml_b200_set_x2_exact(1)
    try:
        loss_o, (g_o, _, _) = _loss_and_grad(v, ix, nz, vv, N, M, iters, every)
    finally:
        B.lib.bml_b200_set_x2_exact(old)
    ref_loss, ref_grad = _dense_reference_grad(_dense(v, ix, nz, N, M), Vd, iters)
    assert loss_u == pytest.approx(ref_loss, rel=1e-10)
    mask = (np.arange(M)[None, :] < nz[:, None]).reshape(-1)
    rows = np.repeat(np.arange(N), M)
    ref_on_pattern = ref_grad[rows[mask], ix[mask]]
    scale = np.abs(ref_on_pattern).max()
    assert np.abs(g_u[mask] - ref_on_pattern).max() <= 1e-8 * scale
    assert np.abs(g_u[mask] - g_o[mask]).max() <= 1e-10 * scale


def _loss_and_pattern(hv, ix, nz, vv, N, M, iters):
    H = B.Ellpack.from_arrays(hv, ix, nz, N, M)
    V = B.Ellpack.from_arrays(vv, ix, nz, N, M)
    D = B.Ellpack(N, M)
    info = (C.c_double * 6)()
    assert B.lib.bml_b200_sp2(H.h, D.h, THR, N / 2.0, iters, -1.0, 0, info) == B.OK
    val = B.lib.bml_trace_mult(D.h, V.h)
    _, dix, dnz = D.download()
    for m in (H, V, D):
        m.free()
    keys = set()
    for i in range(N):
        keys.update(i * N + c for c in dix[i * M:i * M + dnz[i]].tolist())
    return val, keys


def test_adjoint_matches_finite_differences():
    """Central differences (step 1e-6, the differentiable configuration's
    step) of the library's forward SP2 against the adjoint on 32 entries of
    H's pattern: the 16 largest gradient entries, each to 1e-6 of itself,
    and 16 drawn at random, to 1e-6 of the largest entry.  The adjoint holds
    the thresholds fixed, so an entry whose +-h perturbation moves the
    retained pattern of D (an entry crossing the threshold, which makes L
    jump) is not compared; at most 4 of the 32 may be skipped so."""
    N, M, v, ix, nz, vv, _ = _problem(seed=1)
    iters, h = 10, 1e-6
    _, (g, _, _) = _loss_and_grad(v, ix, nz, vv, N, M, iters, 3)
    mask = np.flatnonzero((np.arange(M)[None, :] < nz[:, None]).reshape(-1))
    top = mask[np.argsort(-np.abs(g[mask]))[:16]]
    rest = np.setdiff1d(mask, top)
    picks = np.concatenate([top, np.random.default_rng(5).choice(rest, 16, replace=False)])
    _, base = _loss_and_pattern(v, ix, nz, vv, N, M, iters)
    gscale = np.abs(g[mask]).max()
    skipped, worst = 0, 0.0
    for q in picks:
        vp, vm = v.copy(), v.copy()
        vp[q] += h
        vm[q] -= h
        lp, pp = _loss_and_pattern(vp, ix, nz, vv, N, M, iters)
        lm, pm = _loss_and_pattern(vm, ix, nz, vv, N, M, iters)
        if pp != base or pm != base:
            skipped += 1
            continue
        fd = (lp - lm) / (2 * h)
        # within 1e-6 of the gradient's scale (its largest entry): the
        # differences carry a rounding error of about 1e-16 |L| / h, which
        # is above 1e-6 of the smallest entries themselves
        err = abs(fd - g[q]) / gscale
        worst = max(worst, err)
        assert err <= 1e-6, (q, fd, g[q])
        if q in top:
            assert abs(fd - g[q]) <= 1e-6 * abs(g[q]), (q, fd, g[q])
    assert skipped <= 4, skipped
    print("finite differences: worst relative error %.2e, %d of %d skipped" % (worst, skipped, len(picks)))


def test_adjoint_single_precision_close_to_double():
    """The FP32 adjoint (every step in FP32) against the FP64 one: the same
    pattern, values within 1e-3 of the largest gradient entry."""
    N, M, v, ix, nz, vv, _ = _problem(seed=2)
    iters = 8
    _, (g64, _, _) = _loss_and_grad(v, ix, nz, vv, N, M, iters, 4)
    H = B.Ellpack.from_arrays(v.astype(np.float32), ix, nz, N, M, prec=1)
    V = B.Ellpack.from_arrays(vv.astype(np.float32), ix, nz, N, M, prec=1)
    dH = B.Ellpack(N, M, prec=1)
    loss = C.c_double()
    assert B.lib.bml_b200_sp2_adjoint(H.h, V.h, THR, N / 2.0, iters, 4, M, dH.h, C.byref(loss)) == B.OK
    g32, ix32, nz32 = dH.download()
    assert np.array_equal(nz32, nz)
    mask = (np.arange(M)[None, :] < nz[:, None]).reshape(-1)
    scale = np.abs(g64[mask]).max()
    assert np.abs(g32[mask].astype(np.float64) - g64[mask]).max() <= 1e-3 * scale
