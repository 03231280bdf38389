"""The symmetric scan's threshold argument, restated in NumPy (no GPU).

The symmetric 16-bit scan (tc_scan.cu symmetric mode, sym.cu) keeps for row
c only the keys whose score reaches a threshold U_c derived from a sampled
pre-scan: T_c is the (C+1)-th best raw value over a strided sample, and
U_c = -(T_c + 2 A_c) rounded towards -inf, with A_c = (L/4 + 2) 2^-21
|x~_c| max|y~| the accumulation bound shared by the two scans.  Both the
mailbox (keys from earlier blocks) and the row's own heap (seeded) use U_c,
so the row's candidates are the top C of {self} and the keys reaching U_c.
Here the two scans' scores are the exact dot products of the 16-bit rows,
each perturbed independently by up to A_c (as two accumulations of the same
products may differ), and the test checks that this pool always holds the
top C by (raw, index) of the main scan's scores: the plain scan's candidates.
"""
import numpy as np
import pytest

MIN_POSITIVE = np.float32(1.17549435e-38)


def _raw(scores):
    return np.where(scores > 0, -scores, MIN_POSITIVE).astype(np.float64)


def _rows(n, d, seed, dup=False):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((12, d))
    x = c[rng.integers(0, 12, n)] + 0.2 * rng.standard_normal((n, d))
    if dup:
        x[n // 2:] = x[: n - n // 2]  # every row has an exact duplicate
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return x.astype(np.float32)


def _check(x, C, stride=16, seed=0):
    n, d = x.shape
    rng = np.random.default_rng(seed)
    xh = x.astype(np.float16).astype(np.float64)
    L = (d + 63) // 64 * 64
    hn = np.linalg.norm(xh, axis=1)
    hm = hn.max()
    A = (L / 4 + 2) * 2.0 ** -21 * hn * hm  # per row c: bounds the error of any pair of c
    exact = xh @ xh.T
    # two independent accumulations of the same products, each within the pair's own bound
    bound = (L / 4 + 2) * 2.0 ** -21 * np.outer(hn, hn)
    main = exact + rng.uniform(-1, 1, exact.shape) * bound
    pre = exact + rng.uniform(-1, 1, exact.shape) * bound
    sample = np.arange(0, n, stride)[: n // stride]
    idx = np.arange(n)
    for c in range(n):
        raw_main = _raw(main[c])
        raw_main[c] = -1.0  # the self rule
        plain = np.lexsort((idx, raw_main))[:C]
        raw_pre = _raw(pre[c, sample])  # the pre-scan has no self rule
        T = np.sort(raw_pre)[C]  # (C+1)-th best
        t = T + 2.0 * A[c]
        U = np.nextafter(np.float32(-t), np.float32(-np.inf)) if t < 0 else -np.inf  # rounded down
        passing = main[c] >= U
        passing[c] = True  # self offered directly
        pool = idx[passing]
        sym = pool[np.lexsort((pool, raw_main[pool]))][:C]
        assert np.array_equal(sym, plain), c


@pytest.mark.parametrize("n,d,C", [(1500, 32, 38), (2000, 64, 60), (1200, 768, 25)])
def test_threshold_pool_holds_plain_candidates(n, d, C):
    _check(_rows(n, d, n + d), C)


def test_duplicates_and_ties():
    _check(_rows(1600, 48, 3, dup=True), 30, seed=1)
