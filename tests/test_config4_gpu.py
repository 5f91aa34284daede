"""The differentiable SP2 configuration at its named size: N = 16384 (the
radius-3 lattice Hamiltonian on 26^3 sites, the first 16384 in lexicographic
order, seed 0), perturbation V symmetric on H's pattern with entries
U[-0.01, 0.01], loss L = tr(D V) = sum_ij D_ij V_ij after 40 SP2 iterations
(threshold 1e-5, occupation N/2), adjoint with a checkpoint every 8
iterations.  The iterates fill in to dense rows within a few iterations (the
lattice is metallic), so the products run on the dense tier.

Checked against
  - an FP64 dense reference: the same SP2 map in torch on the GPU
    (thresholds and branch choices as in the library, masks held fixed),
    checkpointed every 8 iterations, differentiated by autograd: loss within
    1e-9 relative, gradient on H's pattern within 1e-6 of its largest entry
    (measured: 6e-13);
  - the FP32 adjoint against the FP64 one, within 5e-2 of the largest entry.
Central differences are asserted at N = 216 (tests/test_adjoint_gpu.py),
where a step of 1e-6 leaves the retained pattern in place.  Here it does
not: among 2.7e8 entries some lie within the step's effect of the 1e-5
threshold, so the differences of the thresholded map measure jumps (one
measured entry: -4.13 against the adjoint's -0.895), while the adjoint, like
the reference above, is the derivative with the retained pattern held fixed.
"""
import ctypes as C
import time

import numpy as np
import pytest

import bml_b200 as B

pytestmark = pytest.mark.gpu

L, RADIUS, N = 26, 3, 16384
MH, M = 128, 16384
THR, ITERS, EVERY = 1e-5, 40, 8


@pytest.fixture(scope="module")
def problem():
    v, ix, nz = B.gen_lattice(L, RADIUS, N, MH, 0)
    mask = (np.arange(MH)[None, :] < nz[:, None]).reshape(-1)
    rows = np.repeat(np.arange(N), MH)[mask]
    cols = ix[mask]
    # V: one U[-0.01, 0.01] draw per pair i <= j, mirrored
    upper = cols >= rows
    Vd = np.zeros((N, N))
    Vd[rows[upper], cols[upper]] = np.random.default_rng(4).uniform(-0.01, 0.01, int(upper.sum()))
    Vd[cols[upper], rows[upper]] = Vd[rows[upper], cols[upper]]
    vv = np.zeros_like(v)
    vv[mask] = Vd[rows, cols]
    del Vd
    pad = lambda a: np.pad(a.reshape(N, MH), ((0, 0), (0, M - MH))).reshape(-1)
    return pad(v), pad(ix), nz, pad(vv)


def _dense(v, ix, nz):
    D = np.zeros((N, N))
    for i in range(N):
        D[i, ix[i * M:i * M + nz[i]]] = v[i * M:i * M + nz[i]]
    return D


@pytest.fixture(scope="module")
def reference(problem):
    """FP64 dense SP2 and its autograd gradient (torch, on the GPU)."""
    import torch
    from torch.utils.checkpoint import checkpoint
    v, ix, nz, vv = problem
    dev = torch.device("cuda")
    H = torch.tensor(_dense(v, ix, nz), dtype=torch.float64, device=dev, requires_grad=True)
    Vd = torch.tensor(_dense(vv, ix, nz), dtype=torch.float64, device=dev)
    eye = torch.eye(N, dtype=torch.bool, device=dev)
    occ = N / 2.0

    def segment(X):
        for _ in range(EVERY):
            X2 = X @ X
            keep = (X2.abs() > THR) | eye
            X2 = torch.where(keep, X2, torch.zeros((), dtype=X2.dtype, device=dev))
            t, t2 = float(torch.trace(X.detach())), float(torch.trace(X2.detach()))
            if abs(t2 - occ) <= abs(2 * t - t2 - occ):
                X = X2
            else:
                Y = 2 * X - X2
                X = torch.where(Y.abs() > THR, Y, torch.zeros((), dtype=Y.dtype, device=dev))
        return X

    t0 = time.perf_counter()
    d = torch.diagonal(H)
    r = H.abs().sum(1) - d.abs()
    emax, emin = torch.max(d + r), torch.min(d - r)
    X = (emax * torch.eye(N, dtype=torch.float64, device=dev) - H) / (emax - emin)
    for _ in range(ITERS // EVERY):
        X = checkpoint(segment, X, use_reentrant=False)
    loss = (X * Vd).sum()
    loss.backward()
    grad = H.grad.cpu().numpy()
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    out = (loss.item(), grad, elapsed)
    del H, Vd, X, loss, eye
    torch.cuda.empty_cache()
    return out


def _adjoint(v, ix, nz, vv, prec):
    H = B.Ellpack.from_arrays(v, ix, nz, N, M, prec=prec)
    V = B.Ellpack.from_arrays(vv, ix, nz, N, M, prec=prec)
    dH = B.Ellpack(N, M, prec=prec)
    loss = C.c_double()
    B.check(B.lib.bml_b200_synchronize())
    t0 = time.perf_counter()
    st = B.lib.bml_b200_sp2_adjoint(H.h, V.h, THR, N / 2.0, ITERS, EVERY, M, dH.h, C.byref(loss))
    B.check(B.lib.bml_b200_synchronize())
    dt = time.perf_counter() - t0
    assert st == B.OK, B.lib.bml_b200_error_string(st)
    g = dH.download()
    for m in (H, V, dH):
        m.free()
    return loss.value, g, dt


@pytest.fixture(scope="module")
def adjoint64(problem):
    v, ix, nz, vv = problem
    old = B.lib.bml_b200_set_x2_exact(0)
    try:
        return _adjoint(v, ix, nz, vv, 2)
    finally:
        B.lib.bml_b200_set_x2_exact(old)


@pytest.mark.unordered
def test_config4_adjoint_fp64(problem, reference, adjoint64):
    v, ix, nz, vv = problem
    ref_loss, ref_grad, t_ref = reference
    loss, (g, gix, gnz), t = adjoint64
    assert np.array_equal(gnz, nz)
    mask = (np.arange(M)[None, :] < nz[:, None]).reshape(-1)
    rows = np.repeat(np.arange(N), M)[mask]
    ref_on = ref_grad[rows, ix[mask]]
    scale = np.abs(ref_on).max()
    err = np.abs(g[mask] - ref_on).max() / scale
    print("config 4 FP64: loss %.15g (reference %.15g), gradient error %.2e of max, adjoint %.1f s, "
          "dense torch reference %.1f s" % (loss, ref_loss, err, t, t_ref))
    assert loss == pytest.approx(ref_loss, rel=1e-9)
    assert err <= 1e-6


@pytest.mark.unordered
def test_config4_adjoint_fp32(problem, adjoint64):
    v, ix, nz, vv = problem
    _, (g64, _, _), _ = adjoint64
    _, (g32, _, gnz), t = _adjoint(v.astype(np.float32), ix, nz, vv.astype(np.float32), 1)
    assert np.array_equal(gnz, nz)
    mask = (np.arange(M)[None, :] < nz[:, None]).reshape(-1)
    scale = np.abs(g64[mask]).max()
    err = np.abs(g32[mask].astype(np.float64) - g64[mask]).max() / scale
    print("config 4 FP32: gradient error against FP64 %.2e of max, adjoint %.1f s" % (err, t))
    # 40 iterations in FP32: each product sums up to 16384 terms in FP32 on
    # the dense tier (about 16384 * 2^-24 = 1e-3 of the magnitudes), and the
    # FP32 run keeps a slightly different set of entries at the 1e-5
    # threshold; measured 2.6e-2 of the largest entry
    assert err <= 5e-2
