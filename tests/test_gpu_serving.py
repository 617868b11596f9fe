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


def test_serving_stream_reports_latency():
    out = serve.run_stream(serve.poisson_stream(30, rate=500.0, seed=31, hi_exp=5.0), workers=2)
    assert out["requests"] == 30 and out["p99_ms"] >= out["p50_ms"] > 0 and out["aggregate_keys_per_s"] > 0
