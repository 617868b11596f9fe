"""The build service's host logic without a GPU (shockhash_b200.serve): fake engines stand in for
the device, so these tests check admission in arrival order, the batch cap, requests larger than
a batch, per-request delivery of results and errors, shutdown, and the request stream."""
import threading

import numpy as np
import pytest

import shockhash_b200.serve as serve


class _FakeResult:
    def __init__(self, keys):
        self.n = len(keys)
        self.freed = False

    def free(self):
        self.freed = True


class _FakeEngine:
    batches = []
    lock = threading.Lock()
    gate = None      # when set, builds wait for it (keeps requests queued)
    entered = None   # set when a build starts
    fail_on = None   # a key value that makes the batch raise

    def __init__(self, device=0):
        self.closed = False

    def build_batch_u64(self, variant, leaf, key_arrays, bucket):
        _FakeEngine.entered.set()
        if _FakeEngine.gate is not None:
            _FakeEngine.gate.wait(5)
        with _FakeEngine.lock:
            _FakeEngine.batches.append([len(k) for k in key_arrays])
        if _FakeEngine.fail_on is not None and any((k == _FakeEngine.fail_on).any() for k in key_arrays):
            raise RuntimeError("device build failed")
        return [_FakeResult(k) for k in key_arrays]

    def build_batch_items(self, variant, leaf, items, bucket):
        _FakeEngine.entered.set()
        if _FakeEngine.gate is not None:
            _FakeEngine.gate.wait(5)
        sizes = [len(d["keys"]) if d.get("keys") is not None else len(d["first"]) for d in items]
        with _FakeEngine.lock:
            _FakeEngine.batches.append(sizes)
        return [_FakeResult(np.zeros(n)) for n in sizes]

    def partition_u64(self, keys, nb, parts):  # the device partition's host twin
        import shockhash_b200 as shg
        first, second = shg.hash_u64_host(keys)
        pairs = np.empty((len(keys), 2), np.uint64)
        counts = np.zeros(parts, np.uint64)
        shg._check(shg.lib().shg_shard_partition(shg._ptr(first), shg._ptr(second), len(keys), nb, parts,
                                                 shg._ptr(pairs), shg._ptr(counts)))
        return pairs, counts

    def close(self):
        self.closed = True


@pytest.fixture
def fake(monkeypatch):
    _FakeEngine.batches = []
    _FakeEngine.gate = None
    _FakeEngine.entered = threading.Event()
    _FakeEngine.fail_on = None
    monkeypatch.setattr(serve, "Engine", _FakeEngine)
    monkeypatch.setattr(serve, "device_memory", lambda device=0: (96 * 1000 * 4, 10 ** 12))
    return _FakeEngine


def _keys(n, base=1):
    return np.arange(base, base + n, dtype=np.uint64)


def test_batch_cap_from_memory_share_and_limit(fake):
    # free 384000 B, half kept, 2 workers: 96000 B each -> 1000 keys of 96 B
    srv = serve.BuildServer(workers=2, warm=False)
    assert srv.batch_keys == 1000
    srv.close()
    srv = serve.BuildServer(workers=2, warm=False, max_batch_keys=300)
    assert srv.batch_keys == 300
    srv.close()


def test_warm_up_builds_a_full_batch_per_worker(fake):
    srv = serve.BuildServer(workers=3, warm=True, max_batch_keys=500)
    srv.close()
    assert fake.batches == [[500]] * 3


def test_arrival_order_batches_and_results(fake):
    fake.gate = threading.Event()
    srv = serve.BuildServer(workers=1, warm=False, max_batch_keys=1000)
    first = srv.submit(0, _keys(10))          # taken at once; blocks on the gate
    assert fake.entered.wait(5)
    sizes = [400, 500, 300, 2500, 100]
    reqs = [srv.submit(i + 1, _keys(n, 100 * i + 1)) for i, n in enumerate(sizes)]
    fake.gate.set()
    for r in [first] + reqs:
        res = r.wait(5)
        assert res.n == len(r.keys)
        assert r.latency is not None and r.latency >= 0
    srv.close()
    # queue prefixes in arrival order, each within 1000 keys unless a single request exceeds it
    assert fake.batches == [[10], [400, 500], [300], [2500], [100]]
    assert [r.batch_size for r in reqs] == [2, 2, 1, 1, 1]


def test_errors_reach_every_request_of_the_batch(fake):
    fake.gate = threading.Event()
    fake.fail_on = 7
    srv = serve.BuildServer(workers=1, warm=False, max_batch_keys=1000)
    blocker = srv.submit(0, _keys(5, 1000))
    assert fake.entered.wait(5)
    bad = srv.submit(1, _keys(10, 1))         # holds key 7
    good_same_batch = srv.submit(2, _keys(10, 500))
    fake.gate.set()
    assert blocker.wait(5).n == 5
    for r in (bad, good_same_batch):
        with pytest.raises(RuntimeError):
            r.wait(5)
    after = srv.submit(3, _keys(10, 900))     # the service keeps going
    assert after.wait(5).n == 10
    srv.close()


def test_results_freed_when_not_kept_and_wait_timeout(fake):
    fake.gate = threading.Event()
    srv = serve.BuildServer(workers=1, warm=False, max_batch_keys=1000, keep_results=False)
    r = srv.submit(0, _keys(10))
    with pytest.raises(TimeoutError):
        r.wait(0.05)
    fake.gate.set()
    assert r.wait(5) is None and r.keys is None
    srv.close()
    assert all(e.closed for e in srv._engines)


def test_poisson_stream_is_deterministic_and_in_range():
    a = serve.poisson_stream(500, rate=200.0, seed=31)
    b = serve.poisson_stream(500, rate=200.0, seed=31)
    assert a == b
    arrivals = [t for t, _, _ in a]
    sizes = [n for _, n, _ in a]
    assert all(x < y for x, y in zip(arrivals, arrivals[1:]))
    assert min(sizes) >= 10 ** 3 and max(sizes) <= 10 ** 7
    assert 1.0 < arrivals[-1] < 5.0  # 500 arrivals at a mean of 200/s
    assert len({s for _, _, s in a}) == 500


def test_admission_reads_free_memory_per_batch(fake):
    free = {"bytes": 96 * 1000 * 2}  # half kept, one worker: a warm capacity of 1000 keys
    srv = serve.BuildServer(workers=1, warm=False, max_batch_keys=0, free_memory=lambda: free["bytes"])
    assert srv.batch_keys == 1000
    # the device's free memory is gone: batches stay within the worker's capacity
    fake.gate = threading.Event()
    free["bytes"] = 0
    blocker = srv.submit(0, _keys(10))
    assert fake.entered.wait(5)
    a = [srv.submit(1, _keys(600, 100)), srv.submit(2, _keys(600, 1000))]
    fake.gate.set()
    for r in [blocker] + a:
        r.wait(5)
    assert fake.batches == [[10], [600], [600]]
    assert srv.grown == 0
    # memory frees up: the next batch may grow the worker's buffers, once, by what is free now
    fake.gate = threading.Event()
    fake.entered = threading.Event()
    free["bytes"] = 96 * 2000 * 2
    blocker = srv.submit(3, _keys(10, 5000))
    assert fake.entered.wait(5)
    b = [srv.submit(4, _keys(600, 6000)), srv.submit(5, _keys(600, 7000))]
    fake.gate.set()
    for r in [blocker] + b:
        r.wait(5)
    srv.close()
    assert fake.batches[3:] == [[10], [600, 600]]
    assert srv.grown == 1 and srv._cap == [1200] and srv._reserved == 0


def test_stream_draws_keys_at_submission(fake):
    stream = serve.poisson_stream(20, rate=2000.0, seed=5, lo_exp=2.0, hi_exp=3.0)
    out = serve.run_stream(stream, workers=2, max_batch_keys=2000)
    assert out["requests"] == 20 and out["total_keys"] == sum(s for _, s, _ in stream)
    served = fake.batches[2:]  # after one warm-up batch per worker
    assert sorted(n for b in served for n in b) == sorted(s for _, s, _ in stream)
    assert out["p99_ms"] >= out["p50_ms"] >= 0


def test_request_keys_are_distinct_and_deterministic():
    import shockhash_b200 as shg
    a = shg.keys_mix(12345, 300_000, threads=4)
    assert len(np.unique(a)) == len(a)
    assert np.array_equal(a, shg.keys_mix(12345, 300_000, threads=1))
    j = np.arange(5, dtype=np.uint64)
    z = np.uint64(12345) ^ (j * np.uint64(0x9E3779B97F4A7C15))
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
    assert np.array_equal(a[:5], z ^ (z >> np.uint64(31)))


def test_split_request_covers_every_key_by_bucket_range():
    from shockhash_b200 import shard
    keys = serve.keys_mix(5, 250_000)
    pieces = serve.split_request(keys, 2000, 60_000, threads=4)
    nb = shard.nbuckets(len(keys), 2000)
    assert len(pieces) == 5 and pieces[0][3] == 0 and pieces[-1][4] == nb
    assert all(a[4] == b[3] for a, b in zip(pieces, pieces[1:]))  # contiguous bucket ranges
    import shockhash_b200 as shg
    f_all, s_all = shg.hash_u64_host(keys)
    got = set()
    for first, second, nbg, b0, b1 in pieces:
        assert nbg == nb
        b = shard.remap128(first, nb)
        assert b.min() >= b0 and b.max() < b1
        got.update(zip(first.tolist(), second.tolist()))
    assert got == set(zip(f_all.tolist(), s_all.tolist()))
    assert sum(len(p[0]) for p in pieces) == len(keys)


def test_chunked_request_joins_its_pieces(fake, monkeypatch):
    merged = []

    def fake_merge(variant, leaf, parts, bucket):
        merged.append([p.n for p in parts])
        return _FakeResult(np.zeros(sum(p.n for p in parts)))

    monkeypatch.setattr(serve, "merge_shards", fake_merge)
    srv = serve.BuildServer(workers=1, max_batch_keys=100_000, chunk_keys=40_000, warm=False)
    try:
        small = srv.submit("a", _keys(10))
        big = srv.submit("b", serve.keys_mix(3, 130_000))
        tail = srv.submit("c", _keys(20, 100))
        for r in (small, big, tail):
            r.wait(timeout=30)
            assert r.error is None
    finally:
        srv.close()
    assert big.result.n == 130_000 and len(merged) == 1 and len(merged[0]) == 4
    assert sum(merged[0]) == 130_000 and small.result.n == 10 and tail.result.n == 20
    # pieces were admitted like requests: batches never exceed the cap unless a single item does
    assert all(sum(b) <= 100_000 or len(b) == 1 for b in fake.batches)
    assert big.t_done >= big.t_start and big.batch_size >= 1
