"""The premise of split pose clustering, on the CPU: float32 sums of integer
weights whose absolute total stays below 2^24 are exact in every order and in
any split into partial sums added together; above that bound, order matters.
"""
import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st


def seq_sum(start, ws):
    c = np.float32(start)
    for w in ws:
        c = np.float32(c + np.float32(w))
    return c


@settings(max_examples=60, deadline=None)
@given(st.integers(0, 2**32 - 1), st.integers(2, 400))
def test_integer_sums_below_2_24_are_order_free(seed, n):
    rng = np.random.default_rng(seed)
    w = rng.integers(-5000, 5000, n).astype(np.float32)
    while np.abs(w).sum() >= 2**24 - 1:
        w = np.floor(w / 2)
    ordered = seq_sum(1, w)
    assert ordered == 1 + int(w.astype(np.int64).sum())
    assert seq_sum(1, rng.permutation(w)) == ordered
    cuts = np.sort(rng.choice(n, size=min(n - 1, 5), replace=False))
    parts = [seq_sum(0, p) for p in np.split(rng.permutation(w), cuts)]
    assert seq_sum(1, rng.permutation(np.array(parts, np.float32))) == ordered


def test_order_matters_above_2_24():
    w = np.array([2.0**24, 1.0, 1.0], np.float32)
    assert seq_sum(0, w) != seq_sum(0, w[::-1])
