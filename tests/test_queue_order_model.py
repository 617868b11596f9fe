"""The work-queue kernel's item order (k_qorder_count / k_qorder_scan / k_qorder_scatter) restated on
the host: time slot t holds the level-lv split nodes of bucket t - lv * lag for every level, then
the leaf group of bucket t - nlevels * lag. Over random plans (per-bucket node counts per level,
buckets with and without leaves) the sequence holds every split node once and one leaf group per
bucket with leaves, and every item comes after everything it waits for (the split nodes of its
bucket on the levels above it, or all of them for a leaf group), which is what lets the persistent
kernel's bounded waits end (no GPU)."""
import numpy as np
import pytest


def queue_order(level_counts, leaf_counts, lag):
    """level_counts[lv][b]: split nodes of bucket b on level lv; leaf_counts[b]: leaves of bucket b.
    Returns the item sequence: ids-array indices of split nodes (levels concatenated, buckets in
    order inside a level), nsplit + b for the leaves of bucket b."""
    nl, nb = len(level_counts), len(leaf_counts)
    cols = [np.concatenate([[0], np.cumsum(c)]).astype(np.int64) for c in level_counts]
    lcol = np.concatenate([[0], np.cumsum(leaf_counts)]).astype(np.int64)
    level_start = np.concatenate([[0], np.cumsum([c[-1] for c in cols])]).astype(np.int64)
    nsplit = int(level_start[-1])
    T = nb + nl * lag
    cnt = np.zeros(T, np.int64)
    for t in range(T):  # k_qorder_count
        for lv in range(nl + 1):
            sh = lv * lag
            if t < sh or t - sh >= nb:
                continue
            b = t - sh
            cnt[t] += cols[lv][b + 1] - cols[lv][b] if lv < nl else int(lcol[b + 1] > lcol[b])
    pos = np.concatenate([[0], np.cumsum(cnt)])  # k_qorder_scan (pos[T] = item count)
    seq = np.full(nsplit + nb, -1, np.int64)
    for t in range(T):  # k_qorder_scatter
        p = pos[t]
        for lv in range(nl + 1):
            sh = lv * lag
            if t < sh or t - sh >= nb:
                continue
            b = t - sh
            if lv < nl:
                for j in range(cols[lv][b], cols[lv][b + 1]):
                    seq[p] = level_start[lv] + j
                    p += 1
            elif lcol[b + 1] > lcol[b]:
                seq[p] = nsplit + b
                p += 1
    return seq[:pos[T]], cols, lcol, level_start, nsplit


@pytest.mark.parametrize("seed", range(40))
def test_queue_order_is_a_permutation_with_dependencies_first(seed):
    rng = np.random.default_rng(seed)
    nb, nl, lag = int(rng.integers(1, 200)), int(rng.integers(1, 7)), int(rng.integers(1, 40))
    level_counts = rng.integers(0, 5, size=(nl, nb))
    leaf_counts = rng.integers(0, 4, size=nb)
    items, cols, lcol, level_start, nsplit = queue_order(level_counts, leaf_counts, lag)
    assert sorted(items[items < nsplit].tolist()) == list(range(nsplit))
    assert sorted((items[items >= nsplit] - nsplit).tolist()) == [b for b in range(nb) if leaf_counts[b]]
    where = {int(x): i for i, x in enumerate(items)}
    for b in range(nb):
        seen = []  # positions of bucket b's split nodes on the levels so far
        for lv in range(nl):
            mine = [where[int(level_start[lv] + j)] for j in range(cols[lv][b], cols[lv][b + 1])]
            assert all(s < m for s in seen for m in mine)
            seen += mine
        if leaf_counts[b]:
            assert all(s < where[nsplit + b] for s in seen)


def test_lag_larger_than_the_buckets_gives_the_level_order():
    level_counts = np.array([[1, 1, 1], [2, 2, 2]])
    items, *_ = queue_order(level_counts, np.array([3, 0, 3]), lag=10)
    # levels one after another, then the leaf groups of the buckets that have leaves
    assert items.tolist() == [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 11]
