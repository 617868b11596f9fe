"""Continuous-batching construction service for ShockHash2 (and ShockHash) build requests.

A request is one independent key set (uint64 keys, each hashed as its 8-byte string) to be built
into its own minimal perfect hash function, e.g. ShockHash2<64> with bucket size 2000. The server
runs `workers` threads; each owns an Engine (its own CUDA stream and resident device buffers).
Whenever a worker is free it takes, in arrival order, as many queued requests as fit its batch
capacity and builds them in ONE batched call (shg_build_batch_u64): their buckets, split nodes and
leaves share the same kernel launches, one persistent leaf launch for the whole batch. Requests
that arrive while batches run wait for the next free worker; with two or more workers, the
batches of different workers overlap on the device.

Admission is by free device memory: at start the server reads the free HBM, keeps `mem_fraction`
of it, and gives every worker an equal share, which caps its batch at share / bytes_per_key keys
and at `max_batch_keys` (a larger request is built alone). Each worker then builds one batch of
that size before serving, so that its device buffers and its pinned result block exist before the
first request arrives: growing them later would allocate and free device and pinned memory, which
synchronises the whole device and stalls the other workers. Each result is bit-identical to
building that request alone.

    python -m shockhash_b200.serve --requests 400
prints one JSON line with p50/p99 build latency, aggregate keys/s and device utilisation for a
Poisson stream (mean 200 requests/s) of log-uniform sizes between 10^3 and 10^7 keys.
"""
import argparse
import json
import math
import threading
import time
from collections import deque

import numpy as np

from . import SHOCKHASH2, Engine, device_memory, keys_mt19937_64


class Request:
    __slots__ = ("rid", "keys", "t_arrival", "t_start", "t_done", "result", "error", "_event", "batch_size")

    def __init__(self, rid, keys, t_arrival):
        self.rid, self.keys, self.t_arrival = rid, keys, t_arrival
        self.t_start = self.t_done = None
        self.result = self.error = None
        self.batch_size = 0
        self._event = threading.Event()

    def wait(self, timeout=None):
        if not self._event.wait(timeout):
            raise TimeoutError(f"request {self.rid} not built within {timeout} s")
        if self.error:
            raise self.error
        return self.result

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_arrival


class BuildServer:
    def __init__(self, variant=SHOCKHASH2, leaf=64, bucket=2000, workers=2, device=0, mem_fraction=0.5,
                 bytes_per_key=96, max_batch_keys=32_000_000, keep_results=True, warm=True):
        self.variant, self.leaf, self.bucket = variant, leaf, bucket
        self.keep_results = keep_results
        free, _ = device_memory(device)
        share = free * mem_fraction / workers
        self.batch_keys = int(min(max_batch_keys or share // bytes_per_key, share // bytes_per_key))
        self._q = deque()
        self._cv = threading.Condition()
        self._stop = False
        self.busy_s = 0.0
        self.batches = []
        self._engines = [Engine(device) for _ in range(workers)]
        if warm:  # size every worker's buffers for a full batch before serving
            sample = keys_mt19937_64(0x5EED, self.batch_keys)
            for e in self._engines:
                for r in e.build_batch_u64(variant, leaf, [sample], bucket):
                    r.free()
            del sample
        self._threads = [threading.Thread(target=self._worker, args=(e,), daemon=True) for e in self._engines]
        for t in self._threads:
            t.start()

    def submit(self, rid, keys, t_arrival=None):
        req = Request(rid, np.ascontiguousarray(keys, dtype=np.uint64), time.perf_counter() if t_arrival is None else t_arrival)
        with self._cv:
            self._q.append(req)
            self._cv.notify()
        return req

    def _take(self):
        """Arrival-ordered prefix of the queue that fits one batch (at least one request)."""
        batch, total = [], 0
        while self._q:
            n = len(self._q[0].keys)
            if batch and total + n > self.batch_keys:
                break
            batch.append(self._q.popleft())
            total += n
        return batch

    def _worker(self, eng):
        while True:
            with self._cv:
                while not self._q and not self._stop:
                    self._cv.wait()
                if self._stop and not self._q:
                    return
                batch = self._take()
            t0 = time.perf_counter()
            for r in batch:
                r.t_start = t0
                r.batch_size = len(batch)
            try:
                results = eng.build_batch_u64(self.variant, self.leaf, [r.keys for r in batch], self.bucket)
                err = None
            except Exception as ex:  # reported per request
                results, err = [None] * len(batch), ex
            t1 = time.perf_counter()
            with self._cv:
                self.busy_s += t1 - t0
                self.batches.append((t0, t1, len(batch), sum(len(r.keys) for r in batch)))
            for r, res in zip(batch, results):
                try:
                    r.t_done = t1
                    r.error = err
                    if self.keep_results:
                        r.result = res
                    else:
                        if res is not None:
                            res.free()
                        r.keys = None
                except Exception as ex:  # never leave a waiter without an answer
                    r.error = ex
                finally:
                    r._event.set()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for e in self._engines:
            e.close()


def poisson_stream(n_requests, rate=200.0, seed=31, lo_exp=3.0, hi_exp=7.0):
    """(arrival offset s, size, key seed) per request: exponential inter-arrival times with mean
    1/rate, sizes round(10^(lo + (hi-lo) u)), per-request key sub-seeds; std::mt19937_64 draws."""
    draws = keys_mt19937_64(seed, 2 * n_requests).astype(np.float64) / 2.0**64
    gaps = -np.log1p(-draws[:n_requests]) / rate
    sizes = np.round(10 ** (lo_exp + (hi_exp - lo_exp) * draws[n_requests:])).astype(np.int64)
    arrivals = np.cumsum(gaps)
    return [(float(arrivals[i]), int(sizes[i]), seed * 1000003 + i) for i in range(n_requests)]


def run_stream(stream, workers=2, leaf=64, bucket=2000, mem_fraction=0.5, max_batch_keys=32_000_000):
    # every request's keys exist before the clock starts, as a client's would when it submits
    all_keys = [keys_mt19937_64(kseed, size) for _, size, kseed in stream]
    srv = BuildServer(leaf=leaf, bucket=bucket, workers=workers, mem_fraction=mem_fraction,
                      max_batch_keys=max_batch_keys, keep_results=False)
    reqs = []
    t0 = time.perf_counter()
    for i, (at, size, kseed) in enumerate(stream):
        keys = all_keys[i]
        all_keys[i] = None
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(srv.submit(i, keys, t_arrival=t0 + at))
    for r in reqs:
        r.wait()
    t_end = max(r.t_done for r in reqs)
    srv.close()
    lat = np.array([r.latency for r in reqs]) * 1e3
    total_keys = sum(s for _, s, _ in stream)
    span = t_end - t0
    return {
        "requests": len(reqs), "total_keys": int(total_keys), "workers": workers,
        "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "mean_ms": round(float(lat.mean()), 3), "max_ms": round(float(lat.max()), 3),
        "aggregate_keys_per_s": round(total_keys / span, 1), "wall_s": round(span, 3),
        "offered_keys_per_s": round(total_keys / max(stream[-1][0], 1e-9), 1),
        "device_busy_fraction": round(min(1.0, srv.busy_s / (span * workers)), 4),
        "batches": len(srv.batches), "mean_batch_requests": round(float(np.mean([b[2] for b in srv.batches])), 2),
        "batch_key_cap": srv.batch_keys,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--requests", type=int, default=400)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--workers", type=int, default=2)
    ap.add_argument("--seed", type=int, default=31)
    ap.add_argument("--leaf", type=int, default=64)
    ap.add_argument("--bucket", type=int, default=2000)
    ap.add_argument("--max-batch-keys", type=int, default=32_000_000)
    args = ap.parse_args()
    stream = poisson_stream(args.requests, args.rate, args.seed)
    out = run_stream(stream, workers=args.workers, leaf=args.leaf, bucket=args.bucket,
                     max_batch_keys=args.max_batch_keys)
    out.update({"metric": "ShockHash2 build service: p50/p99 build latency and aggregate keys/s",
                "config": {"variant": "ShockHash2", "leaf_size": args.leaf, "bucket_size": args.bucket,
                           "arrivals": f"Poisson, mean {args.rate}/s, seed {args.seed}",
                           "sizes": "round(10^(3+4u)) uint64 keys per request",
                           "sample": f"first {args.requests} requests of the 10,000-request stream"}})
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
