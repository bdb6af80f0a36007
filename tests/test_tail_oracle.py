"""CPU checks of the learned-tail oracle (oracle/tail_mlp.py), the checker of the
gx_tail_* kernels: its backward pass against finite differences, its bf16 rounding
against torch's, and the subsampling rules."""

import numpy as np
import pytest

import tail_mlp as T


def _params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in T.SHAPES:
        fan = shp[-1] if len(shp) == 2 else 1
        d[name] = rng.uniform(-1, 1, size=shp) * scale / np.sqrt(fan) if len(shp) == 2 else rng.normal(0, 0.1, shp)
    return T.pack(d)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = _params(1)
    X = rng.normal(0, 1, size=(6, T.NIN))
    Y = rng.normal(0, 1, size=(6, 2))
    norm = np.array([0.3, 2.0, -1.0, 0.5])
    w = (1.0, 0.7)
    loss, G = T.loss_and_grads(P, X, Y, norm, w, emulate=False)
    idx = np.concatenate([rng.choice(np.arange(n0, n0 + n), min(12, n), replace=False)
                          for n0, n in _offsets()])
    eps = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        fd = (T.loss_and_grads(Pp, X, Y, norm, w, emulate=False)[0] -
              T.loss_and_grads(Pm, X, Y, norm, w, emulate=False)[0]) / (2 * eps)
        assert abs(fd - G[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, G[i])


def _offsets():
    o = 0
    for _, shp in T.SHAPES:
        n = int(np.prod(shp))
        yield o, n
        o += n


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.normal(0, 1, 20000), rng.normal(0, 1e-3, 2000), [0.0, -0.0, 1.0, 65504.0, 1e-30]])
    # float32 values exactly halfway between two bf16 neighbours (ties to even)
    halves = ((np.arange(1000, dtype=np.uint32) << 16) | 0x8000).view(np.float32).astype(np.float64)
    x = np.concatenate([x, halves, -halves])
    ours = T.bf16_bits(x)
    theirs = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(ours, theirs)


def test_subsample_rules():
    rng = np.random.default_rng(3)
    h = np.zeros(T.HIST, np.int64)
    h[200:420] = rng.integers(0, 60, 220)
    hyp = 600
    h[hyp] = 1
    tot = int(h.sum())
    for keep in (1, 2, 17, 100, 512):
        sub, cs = T.subsample(h, hyp, keep, seed=99 + keep)
        assert cs == keep and sub.sum() == keep
        assert sub[hyp] == 1 and np.all(sub <= h)
        again, _ = T.subsample(h, hyp, keep, seed=99 + keep)
        assert np.array_equal(sub, again)
    full, cs = T.subsample(h, hyp, 0, seed=5)
    assert cs == tot and np.array_equal(full, h)
    big, cs = T.subsample(h, hyp, tot + 3, seed=5)
    assert cs == tot and np.array_equal(big, h)


def test_subsample_is_uniform_without_replacement():
    # every candidate equally likely: the kept share of each bin tracks its count
    h = np.zeros(T.HIST, np.int64)
    h[100], h[101], h[102], h[500] = 3000, 1000, 6000, 1
    acc = np.zeros(T.HIST)
    for s in range(200):
        sub, _ = T.subsample(h, 500, 401, seed=s)
        acc += sub
    share = acc[100:103] / acc[100:103].sum()
    np.testing.assert_allclose(share, [0.3, 0.1, 0.6], atol=0.01)


def test_feature_row_layout():
    h = np.zeros(T.HIST, np.int64)
    h[10:60] = 9
    h[300] = 1
    bits = T.feature_bits(h, cs=451, hyp=300, prec=1234.5, charge=3)
    v = T.bf16_value(bits)
    # window = bins 10..137, from the first non-empty bin
    np.testing.assert_allclose(v[:50], np.log10(10.0), rtol=4e-3)
    assert np.all(v[50:128] == 0.0)
    np.testing.assert_allclose(v[128:], [np.log10(451), 1.2345, 3.0, 2.9], rtol=4e-3)
    # a window reaching past the last bin reads zeros there
    h2 = np.zeros(T.HIST, np.int64)
    h2[760] = 4
    h2[801] = 1
    v2 = T.bf16_value(T.feature_bits(h2, cs=5, hyp=801, prec=500.0, charge=2))
    np.testing.assert_allclose(v2[[0, 41]], [np.log10(5.0), np.log10(2.0)], rtol=4e-3)
    assert np.all(v2[42:128] == 0.0) and v2[131] == T.bf16(0.41)[()]


def test_adam_matches_closed_form_first_step():
    P = np.ones(5)
    G = np.array([0.5, -2.0, 0.0, 1e-3, 3.0])
    P1, m, v = T.adam(P, G, np.zeros(5), np.zeros(5), step=1, lr=0.01)
    # first step: m/bc1 = g, v/bc2 = g^2, so the move is lr * sign(g) (up to eps)
    np.testing.assert_allclose(P1, 1 - 0.01 * np.sign(G) * np.abs(G) / (np.abs(G) + 1e-8), rtol=1e-12)


def test_choose_sparse_below_takes_the_largest_winning_threshold():
    """The fallback threshold: the largest candidate count below which the learned line
    beats the plain fit on both the median and the 90th percentile; 0 when it never does."""
    import gicops_b200.tail as T
    rng = np.random.default_rng(0)
    cands = rng.integers(20, 500, 4000)
    ep = rng.exponential(5.0, 4000)
    el = np.where(cands < 150, 0.5 * ep, 2.0 * ep)          # learned wins below 150 only
    t = T.choose_sparse_below(ep, el, cands)
    ths = (25, 50, 75, 100, 150, 200, 300, 500)
    wins = lambda x: (np.median(el[cands < x]) < np.median(ep[cands < x]) and  # noqa: E731
                      np.quantile(el[cands < x], 0.9) < np.quantile(ep[cands < x], 0.9))
    assert t >= 150 and wins(t) and not any(wins(x) for x in ths if x > t)
    assert T.choose_sparse_below(ep, 2.0 * ep, cands) == 0   # never wins
    assert T.choose_sparse_below(ep, 0.5 * ep, cands) == 500
    # too few rows below a threshold: that threshold is not judged
    assert T.choose_sparse_below(ep[:50], 0.5 * ep[:50], cands[:50]) == 0
