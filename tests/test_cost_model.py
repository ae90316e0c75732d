"""The cost model's per-plan estimate (fmcs_estimate_plan) and the effective
cardinality of skewed columns; no GPU needed.  The reference estimates plans
in StitchComposer::cost_estimation (src/stitch_composer.cpp:2929-3166) from
per-column cardinalities alone (src/stitch_composer.h:16-43)."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi

N = 1 << 24


def test_estimate_matches_the_search():
    """The optimizer's reported estimate is the estimate of the plan it picked,
    and no other two-bank split of 17B33 is estimated cheaper."""
    bw, card, cb = [17, 33], [8192, 1 << 24], [4, 8]
    split, order, est = capi.optimize_plan(bw, card, cb, N)
    assert capi.estimate_plan(bw, card, cb, N, split, order) == pytest.approx(est, rel=1e-12)
    for k in range(1, 50):
        assert capi.estimate_plan(bw, card, cb, N, [k, 50 - k]) >= est - 1e-12


def test_estimate_column_order_and_rejections():
    bw, card, cb = [2, 1, 12, 12, 32, 7], [3, 2, 2526, 2526, 60_000_000, 100], [2, 2, 2, 2, 4, 2]
    n = 60_000_000
    split, order, est = capi.optimize_plan(bw, card, cb, n, ordered=False)
    assert capi.estimate_plan(bw, card, cb, n, split, order) == pytest.approx(est, rel=1e-12)
    with pytest.raises(capi.FmcsError):
        capi.estimate_plan(bw, card, cb, n, [60])            # does not cover the 66 bits
    with pytest.raises(capi.FmcsError):
        capi.estimate_plan(bw, card, cb, n, [33, 33], [0, 0, 1, 2, 3, 4])   # not a permutation
    with pytest.raises(capi.FmcsError):
        capi.estimate_plan(bw, card, cb, n, [65, 1])         # a bank wider than 64 bits


def test_effective_cardinality():
    assert capi.effective_cardinality([5] * 1000) == 1000               # equal groups: the distinct count
    assert capi.effective_cardinality([10 ** 6] + [1] * 10 ** 6) in (3, 4)   # one giant group dominates
    assert capi.effective_cardinality([]) == 1
    # Zipf(1.0) over 2^20 codes: the row-weighted view sees a few hundred
    # groups where a million values are present
    r = np.arange(1, (1 << 20) + 1, dtype=np.float64)
    counts = np.floor(67_108_864 / (r * np.sum(1.0 / r)))
    eff = capi.effective_cardinality(counts)
    assert 50 < eff < 1000 < int((counts > 0).sum())


def test_skew_moves_the_zipf_plan():
    """Equal groups of a million distinct values make a 32-bit first round look
    as cheap as a 64-bit one (a tie); the effective cardinality of the skewed
    column makes the wide first round the clear choice, which is the faster
    plan on the GPU (5.5 against 6.9 ms at 67,108,864 rows)."""
    n = 67_108_864
    bw, cb = [20, 24, 40], [4, 4, 8]
    skewed = [127, 1 << 24, n]
    a = capi.estimate_plan(bw, skewed, cb, n, [64, 20])
    b = capi.estimate_plan(bw, skewed, cb, n, [32, 52])
    assert a < 0.9 * b
    split, _, _ = capi.optimize_plan(bw, skewed, cb, n)
    assert split[0] > 32
