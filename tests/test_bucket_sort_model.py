"""The sort inside a bucket (k_bucket_sort) restated on the host: a counting sort on
(first - min) >> shift, the shift leaving at most 4096 sub-ranges, then insertion sort by
(first, input index) inside each sub-range, equals the stable sort by `first` that the oracle uses
(Sorter.hpp:15-36 sorts by `first`; ties keep input order). Random buckets, duplicates, spans
below 4096 and the full 64-bit span (no GPU)."""
import numpy as np
import pytest

SUBS = 4096


def counting_sort_order(first, idx):
    m = len(first)
    if m < 2:
        return list(range(m))
    f = [int(x) for x in first]
    lo, hi = min(f), max(f)
    span = hi - lo
    bits = span.bit_length()
    shift = bits - 12 if bits > 12 else 0
    sub = [(x - lo) >> shift for x in f]
    assert max(sub) < SUBS
    count = [0] * SUBS
    for s in sub:
        count[s] += 1
    start = [0] * (SUBS + 1)
    for s in range(SUBS):
        start[s + 1] = start[s] + count[s]
    cursor = start[:SUBS]
    out = [None] * m
    for i, s in enumerate(sub):  # any order inside a sub-range
        out[cursor[s]] = i
        cursor[s] += 1
    for s in range(SUBS):
        a, e = start[s], start[s + 1]
        for i in range(a + 1, e):
            cur = out[i]
            j = i
            while j > a and (f[out[j - 1]], idx[out[j - 1]]) > (f[cur], idx[cur]):
                out[j] = out[j - 1]
                j -= 1
            out[j] = cur
    return out


CASES = ["random", "duplicates", "narrow", "full_span", "bucket_range"]


@pytest.mark.parametrize("case", CASES)
def test_counting_sort_equals_stable_sort(case):
    rng = np.random.default_rng(100 + CASES.index(case))
    for _ in range(20):
        m = int(rng.integers(0, 3000))
        if case == "random":
            first = rng.integers(0, 2**64, size=m, dtype=np.uint64)
        elif case == "duplicates":
            first = rng.choice(rng.integers(0, 2**64, size=max(1, m // 20), dtype=np.uint64), size=m)
        elif case == "narrow":
            first = (np.uint64(2**63) + rng.integers(0, 1000, size=m).astype(np.uint64)).astype(np.uint64)
        elif case == "full_span":
            first = rng.integers(0, 2**64, size=m, dtype=np.uint64)
            if m >= 2:
                first[0], first[1] = np.uint64(0), np.uint64(2**64 - 1)
        else:  # one bucket of remap128(first, 5000): a 2^64 / 5000 wide range
            b = int(rng.integers(0, 5000))
            lo = -(-(b << 64) // 5000)
            width = ((b + 1) << 64) // 5000 - lo
            first = np.array([lo + int(x) for x in rng.integers(0, width, size=m, dtype=np.uint64)], dtype=np.uint64)
        idx = rng.permutation(m).tolist()  # input positions, distinct
        got = counting_sort_order(first, idx)
        want = np.lexsort((np.array(idx, dtype=np.int64), first)).tolist() if m else []
        assert got == want
