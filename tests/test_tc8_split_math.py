"""The arithmetic of the tensor-core X^2's 8-bit split, restated in numpy
(the kernel is `tc8_slices`, `tc8_split_kernel` and the level epilogue of
`tc_x2_kernel` in bml_b200/csrc/ellblock_tc.cu), on the host:

  - every entry x of a scalar row with scale sigma = 2^e (the power of two
    just above the row's largest magnitude) is
    sigma 2^-6 (a1 + 2^-7 a2 + 2^-14 a3 + 2^-21 a4 + 2^-28 a5) + r with
    integer slices |a_s| <= 64 and |r| <= 2^-35 sigma;
  - a block product formed from the slice products with s + t <= 6, each
    level summed exactly in integers (as the INT32 accumulators do) and the
    levels combined in FP64, is within 32 K 2^-31 sigma_r tau_c of the FP64
    product for K terms per entry (the bound the GPU tests assert per block
    pair), and each level's sum stays below 2^31 for up to 3276 block pairs.
"""
import numpy as np

SLICES = 5


def scale_exp(m):
    """e with 2^e > m >= 0 (0 for m = 0): frexp's exponent."""
    return np.where(m > 0, np.frexp(m)[1], 0)


def slices(u):
    """The five slices of u (|u| < 1), each rint of the scaled remainder."""
    y = u * 64.0
    out = []
    for _ in range(SLICES):
        q = np.rint(y)
        out.append(q.astype(np.int64))
        y = (y - q) * 128.0
    return out


def split_rows(x):
    """Slices of every entry against its row's scale, and the scales."""
    e = scale_exp(np.abs(x).max(axis=1))
    u = np.ldexp(x, -e[:, None])
    return slices(u), np.ldexp(1.0, e)


def test_slices_and_residual():
    rng = np.random.default_rng(7)
    x = rng.standard_normal((64, 32)) * np.exp(rng.uniform(-30, 5, (64, 1)))
    x[3] = 0.0
    a, sig = split_rows(x)
    back = sum(np.ldexp(a[s].astype(np.float64), -6 - 7 * s) for s in range(SLICES)) * sig[:, None]
    assert all(np.abs(a[s]).max() <= 64 for s in range(SLICES))
    assert np.all(np.abs(x - back) <= np.ldexp(1.0, -35) * sig[:, None])
    assert np.all(back[3] == 0.0)


def level_product(x, y):
    """x (32 x K) times y (K x 32) from the slice products with s + t <= 6
    (s, t = 1..5): each level L = s + t summed in integers, the levels
    combined in FP64 as the epilogue does, scaled by sigma_r tau_c 2^-12."""
    a, sig = split_rows(x)
    bt, tau = split_rows(y.T)  # columns of y as rows
    lev = [np.zeros((x.shape[0], y.shape[1]), np.int64) for _ in range(SLICES)]
    for s in range(SLICES):
        for t in range(SLICES - s):
            lev[s + t] += a[s] @ bt[t].T
    v = np.zeros(lev[0].shape)
    for L in range(SLICES - 1, -1, -1):
        v = (0.0 if L == SLICES - 1 else v * 2.0 ** -7) + lev[L].astype(np.float64)
    return v * np.ldexp(np.outer(sig, tau), -12), sig, tau, lev


def test_level_product_bound_and_headroom():
    rng = np.random.default_rng(11)
    for K in (32, 32 * 40):
        x = rng.standard_normal((32, K)) * np.exp(rng.uniform(-8, 2, (1, K)))
        y = rng.standard_normal((K, 32)) * np.exp(rng.uniform(-8, 2, (K, 1)))
        got, sig, tau, lev = level_product(x, y)
        want = x @ y
        bound = 32 * (K // 32) * 2.0 ** -31 * np.outer(sig, tau)
        assert np.all(np.abs(got - want) <= bound + 1e-15 * (np.abs(x) @ np.abs(y)))
        # per level and block pair at most 5 terms of 64 * 64 * 32: 3276 pairs fit 2^31
        assert max(np.abs(l).max() for l in lev) <= (K // 32) * 5 * 64 * 64 * 32
    assert 3276 * 5 * 64 * 64 * 32 < 2 ** 31
