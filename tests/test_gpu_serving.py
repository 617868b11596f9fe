"""Continuous batching: every request's products are identical alone and inside a batch/mix."""
import numpy as np
import pytest

import shockhash_b200 as shg
from shockhash_b200 import serve

pytestmark = pytest.mark.gpu


def same(a, b):
    return (np.array_equal(a.descriptors, b.descriptors) and np.array_equal(a.bucket_size_acc, b.bucket_size_acc)
            and np.array_equal(a.bucket_pos_acc, b.bucket_pos_acc) and np.array_equal(a.ribbon_keys, b.ribbon_keys)
            and np.array_equal(a.ribbon_bits, b.ribbon_bits))


def test_batch_equals_alone(engine):
    sizes = [1, 2, 777, 2000, 2001, 50_000, 3, 123_457]
    sets = [shg.keys_mt19937_64(900 + i, n) for i, n in enumerate(sizes)]
    batch = engine.build_batch_u64(2, 64, sets, 2000)
    for keys, got in zip(sets, batch):
        assert same(got, engine.build_u64(2, 64, keys, 2000))
    batch1 = engine.build_batch_u64(1, 30, sets[2:6], 2000)
    for keys, got in zip(sets[2:6], batch1):
        assert same(got, engine.build_u64(1, 30, keys, 2000))


def test_server_results_equal_alone_builds(engine):
    stream = serve.poisson_stream(40, rate=2000.0, seed=7, lo_exp=3.0, hi_exp=5.3)
    srv = serve.BuildServer(workers=2, max_batch_keys=300_000)
    try:
        reqs = [srv.submit(i, shg.keys_mt19937_64(kseed, size)) for i, (_, size, kseed) in enumerate(stream)]
        for r in reqs:
            r.wait(timeout=120)
        batched = sum(1 for r in reqs if r.batch_size > 1)
        for (_, size, kseed), r in zip(stream, reqs):
            alone = engine.build_u64(2, 64, shg.keys_mt19937_64(kseed, size), 2000)
            assert same(r.result, alone), r.rid
            alone.free()
    finally:
        srv.close()
    assert batched > 0  # the stream is fast enough that some requests were built in a mix
    # results outlive their server's engines: releasing them afterwards is safe
    for r in reqs:
        r.result.free()


def test_batch_items_equal_alone_and_shard_builds(engine):
    keys_a = shg.keys_mt19937_64(41, 30_000)
    keys_b = shg.keys_mt19937_64(42, 200_000)
    pieces = serve.split_request(keys_b, 2000, 70_000)
    items = [dict(keys=keys_a)] + [dict(first=f, second=s, nb_global=nb, b0=b0, b1=b1) for f, s, nb, b0, b1 in pieces]
    items.append(dict(keys=keys_a[:5]))
    got = engine.build_batch_items(2, 64, items, 2000)
    assert same(got[0], engine.build_u64(2, 64, keys_a, 2000))
    assert same(got[-1], engine.build_u64(2, 64, keys_a[:5], 2000))
    for (f, s, nb, b0, b1), r in zip(pieces, got[1:-1]):
        assert same(r, engine.build_shard_hash128(2, 64, f, s, nb, b0, b1, 2000))
    whole = shg.merge_shards(2, 64, got[1:-1], 2000)
    assert same(whole, engine.build_u64(2, 64, keys_b, 2000))


def test_device_split_equals_host_split(engine):
    keys = shg.keys_mt19937_64(43, 333_333)
    host = serve.split_request(keys, 2000, 50_000)
    dev = serve.split_request(keys, 2000, 50_000, engine=engine)
    assert len(host) == len(dev) == 7
    for a, b in zip(host, dev):
        assert a[2:] == b[2:] and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_chunked_server_results_equal_alone_builds(engine):
    sizes = [3_000, 260_000, 40_000, 1, 180_001, 9_999]
    srv = serve.BuildServer(workers=2, max_batch_keys=150_000, chunk_keys=60_000)
    try:
        reqs = [srv.submit(i, shg.keys_mt19937_64(500 + i, n)) for i, n in enumerate(sizes)]
        for r in reqs:
            r.wait(timeout=120)
            assert r.error is None, r.error
        for i, (n, r) in enumerate(zip(sizes, reqs)):
            alone = engine.build_u64(2, 64, shg.keys_mt19937_64(500 + i, n), 2000)
            assert same(r.result, alone), r.rid
            alone.free()
            r.result.free()
    finally:
        srv.close()


def test_serving_stream_reports_latency():
    out = serve.run_stream(serve.poisson_stream(30, rate=500.0, seed=31, hi_exp=5.0), workers=2)
    assert out["requests"] == 30 and out["p99_ms"] >= out["p50_ms"] > 0 and out["aggregate_keys_per_s"] > 0
