"""Continuous-batching construction service for ShockHash2 (and ShockHash) build requests.

A request is one independent key set (uint64 keys, each hashed as its 8-byte string) to be built
into its own minimal perfect hash function, e.g. ShockHash2<64> with bucket size 2000. The server
runs `workers` threads; each owns an Engine (its own CUDA stream and resident device buffers).
Whenever a worker is free it takes, in arrival order, as many queued requests as fit its batch
capacity and builds them in ONE batched call (shg_build_batch_u64): their buckets, split nodes and
leaves share the same kernel launches, one persistent leaf launch for the whole batch. Requests
that arrive while batches run wait for the next free worker; with two or more workers, the
batches of different workers overlap on the device.

Admission is by free device memory, read again whenever a batch is formed. At start the server
reads the free HBM, keeps `mem_fraction` of it, and gives every worker an equal share: its warm
capacity, share / bytes_per_key keys (at most `max_batch_keys`). Each worker builds one batch of
that size before serving, so that its device buffers and its pinned result block exist before the
first request arrives. When a worker forms a batch, it takes, in arrival order, requests up to its
warm capacity plus what the device's free memory at that moment allows beyond it (`mem_fraction`
of the free bytes, less what other workers have reserved for batches in flight, divided by
bytes_per_key); a batch beyond the warm capacity grows that worker's buffers once, and the new
size becomes its capacity. A request larger than every limit is built alone. Each result is
bit-identical to building that request alone.

With `chunk_keys` set, a request of more keys than that is split into bucket-range pieces by the
first worker that reaches it in the queue: its keys are hashed and partitioned by bucket range on
that worker's GPU (shg_partition_u64, the partition of a multi-GPU build) and the pieces go back to
the head of the queue as separate items, so they fit the batch limits, spread over the workers and
share batches with other requests; the last piece to finish joins them (shg_merge_shards), which
gives the same bits as building the request alone.

    python -m shockhash_b200.serve --requests 400
prints one JSON line with p50/p99 build latency, aggregate keys/s and device utilisation for a
Poisson stream (mean 200 requests/s) of log-uniform sizes between 10^3 and 10^7 keys. Each
request's keys are drawn when it is submitted (keys_mix of the request's sub-seed), so a stream of
any length runs in bounded host memory; the latency clock starts at submission.
"""
import argparse
import json
import math
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import SHOCKHASH2, Engine, _check, _ptr, device_memory, hash_u64_host, keys_mix, keys_mt19937_64, lib, merge_shards


class Request:
    __slots__ = ("rid", "keys", "t_arrival", "t_start", "t_done", "result", "error", "_event", "batch_size",
                 "parts", "remaining", "to_split")

    def __init__(self, rid, keys, t_arrival):
        self.rid, self.keys, self.t_arrival = rid, keys, t_arrival
        self.t_start = self.t_done = None
        self.result = self.error = None
        self.batch_size = 0
        self.parts, self.remaining = None, 0  # bucket-range pieces of a chunked request
        self.to_split = False  # queued whole, split into pieces by the first worker that reaches it
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


class Piece:
    """Buckets [b0, b1) of a chunked request's structure (nb_global buckets): the fingerprints of
    exactly its keys, built like a shard and joined with the request's other pieces at the end."""
    __slots__ = ("parent", "idx", "first", "second", "nb_global", "b0", "b1")

    def __init__(self, parent, idx, first, second, nb_global, b0, b1):
        self.parent, self.idx, self.first, self.second = parent, idx, first, second
        self.nb_global, self.b0, self.b1 = nb_global, b0, b1

    @property
    def keys(self):  # the size the admission counts
        return self.first


def split_request(keys, bucket, chunk_keys, engine=None, threads=8):
    """The bucket-range pieces of a request of more than `chunk_keys` keys: its fingerprints
    partitioned by range of their bucket remap128(first, nb) into ceil(n / chunk_keys) ranges (at most
    64), stable. With an engine the keys are hashed and partitioned on its GPU (shg_partition_u64),
    otherwise on the host (shg_hash_u64_host, shg_shard_partition); both give the same pieces.
    Returns [(first, second, nb_global, b0, b1)] in bucket order, empty ranges left out."""
    n = len(keys)
    nb = max(1, (n + bucket - 1) // bucket)
    parts = max(1, min(64, -(-n // chunk_keys), nb))
    if engine is not None:
        pairs, counts = engine.partition_u64(keys, nb, parts)
    else:
        first, second = hash_u64_host(keys, threads)
        pairs = np.empty((n, 2), dtype=np.uint64)
        counts = np.zeros(parts, dtype=np.uint64)
        _check(lib().shg_shard_partition(_ptr(first), _ptr(second), n, nb, parts, _ptr(pairs), _ptr(counts)))
    out, at = [], 0
    for g in range(parts):
        b0, b1 = nb * g // parts, nb * (g + 1) // parts
        c = int(counts[g])
        if b1 > b0:
            out.append((np.ascontiguousarray(pairs[at:at + c, 0]), np.ascontiguousarray(pairs[at:at + c, 1]), nb, b0, b1))
        at += c
    return out


class BuildServer:
    def __init__(self, variant=SHOCKHASH2, leaf=64, bucket=2000, workers=2, device=0, mem_fraction=0.5,
                 bytes_per_key=96, max_batch_keys=32_000_000, keep_results=True, warm=True, free_memory=None,
                 chunk_keys=0):
        self.variant, self.leaf, self.bucket = variant, leaf, bucket
        self.chunk_keys = chunk_keys  # requests above this size are built in bucket-range pieces
        self.keep_results = keep_results
        self.device, self.mem_fraction, self.bytes_per_key = device, mem_fraction, bytes_per_key
        self.max_batch_keys = max_batch_keys
        # free device bytes now (a callable; tests substitute their own)
        self._free_memory = free_memory or (lambda: device_memory(device)[0])
        share = self._free_memory() * mem_fraction / workers
        self.batch_keys = int(min(max_batch_keys or share // bytes_per_key, share // bytes_per_key))
        self._q = deque()
        self._cv = threading.Condition()
        self._stop = False
        self._reserved = 0  # bytes of growth admitted for batches in flight
        self.busy_s = 0.0
        self.batches = []
        self.grown = 0  # batches admitted beyond their worker's warm capacity
        self._engines = [Engine(device) for _ in range(workers)]
        self._cap = [self.batch_keys] * workers  # keys each worker's buffers fit
        if warm:  # size every worker's buffers for a full batch before serving
            sample = keys_mt19937_64(0x5EED, self.batch_keys)
            for e in self._engines:
                for r in e.build_batch_u64(variant, leaf, [sample], bucket):
                    r.free()
            del sample
        self._merger = ThreadPoolExecutor(max_workers=2) if chunk_keys else None
        self._threads = [threading.Thread(target=self._worker, args=(w, e), daemon=True)
                         for w, e in enumerate(self._engines)]
        for t in self._threads:
            t.start()

    def submit(self, rid, keys, t_arrival=None):
        req = Request(rid, np.ascontiguousarray(keys, dtype=np.uint64), time.perf_counter() if t_arrival is None else t_arrival)
        # a large request queues whole; the worker that reaches it splits it on its GPU and puts the
        # pieces back at the head of the queue (its latency clock runs from here, split included)
        req.to_split = bool(self.chunk_keys) and len(req.keys) > self.chunk_keys
        with self._cv:
            self._q.append(req)
            self._cv.notify()
        return req

    def _split(self, req, eng):
        """Replaces a large request at the head of the queue by its pieces (worker thread)."""
        try:
            pieces = split_request(req.keys, self.bucket, self.chunk_keys, engine=eng)
        except Exception as ex:
            req.error, req.t_done = ex, time.perf_counter()
            req._event.set()
            return
        req.parts, req.remaining = [None] * len(pieces), len(pieces)
        req.keys = None
        with self._cv:
            # pieces go first, in bucket order; other requests are admitted beside them
            self._q.extendleft(reversed([Piece(req, i, *pc) for i, pc in enumerate(pieces)]))
            self._cv.notify_all()

    def batch_limit(self, w):
        """Keys worker `w` may take now: its capacity plus the growth the free device memory allows
        (call with the lock held)."""
        extra = max(0, int(self._free_memory() * self.mem_fraction) - self._reserved) // self.bytes_per_key
        limit = self._cap[w] + extra
        return min(limit, self.max_batch_keys) if self.max_batch_keys else limit

    def _take(self, w):
        """Arrival-ordered prefix of the queue that fits worker w's limit (at least one request), and
        the bytes of growth it reserves."""
        limit = self.batch_limit(w)
        batch, total = [], 0
        while self._q:
            n = len(self._q[0].keys)
            if batch and total + n > limit:
                break
            batch.append(self._q.popleft())
            total += n
        grow = max(0, total - self._cap[w]) * self.bytes_per_key
        self._reserved += grow
        return batch, total, grow

    def _worker(self, w, eng):
        while True:
            with self._cv:
                while not self._q and not self._stop:
                    self._cv.wait()
                if self._stop and not self._q:
                    return
                head = self._q[0]
                if isinstance(head, Request) and head.to_split:
                    self._q.popleft()
                    head.to_split = False
                    if head.t_start is None:
                        head.t_start = time.perf_counter()
                    split = head
                else:
                    split = None
                    batch, total, grow = self._take(w)
            if split is not None:
                self._split(split, eng)
                continue
            t0 = time.perf_counter()
            for r in batch:
                owner = r.parent if isinstance(r, Piece) else r
                if owner.t_start is None:
                    owner.t_start = t0
                owner.batch_size = max(owner.batch_size, len(batch))
            try:
                if any(isinstance(r, Piece) for r in batch):
                    items = [dict(first=r.first, second=r.second, nb_global=r.nb_global, b0=r.b0, b1=r.b1)
                             if isinstance(r, Piece) else dict(keys=r.keys) for r in batch]
                    results = eng.build_batch_items(self.variant, self.leaf, items, self.bucket)
                else:
                    results = eng.build_batch_u64(self.variant, self.leaf, [r.keys for r in batch], self.bucket)
                err = None
            except Exception as ex:  # reported per request
                results, err = [None] * len(batch), ex
            t1 = time.perf_counter()
            with self._cv:
                self.busy_s += t1 - t0
                self.batches.append((t0, t1, len(batch), total))
                self._reserved -= grow
                if total > self._cap[w]:
                    self._cap[w] = total  # the engine's buffers now fit this batch
                    self.grown += 1
            for r, res in zip(batch, results):
                if isinstance(r, Piece):
                    self._piece_done(r, res, err)
                    continue
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

    def _piece_done(self, piece, res, err):
        """Keeps a finished piece's products; the last piece of a request joins them all
        (shg_merge_shards: accumulators offset, codes concatenated at bit granularity), which gives
        exactly the result of building the request alone."""
        req = piece.parent
        with self._cv:
            req.parts[piece.idx] = res
            if err is not None:
                req.error = err
            req.remaining -= 1
            last = req.remaining == 0
        if last:  # the join runs beside the workers, which go on building
            self._merger.submit(self._join, req)

    def _join(self, req):
        try:
            if req.error is None:
                merged = merge_shards(self.variant, self.leaf, req.parts, self.bucket)
                if self.keep_results:
                    req.result = merged
                else:
                    merged.free()
        except Exception as ex:
            req.error = ex
        finally:
            for x in req.parts:
                if x is not None:
                    x.free()
            req.parts = None
            req.t_done = time.perf_counter()
            req._event.set()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        if self._merger is not None:
            self._merger.shutdown(wait=True)
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


def run_stream(stream, workers=2, leaf=64, bucket=2000, mem_fraction=0.5, max_batch_keys=32_000_000, chunk_keys=0):
    """Replay `stream` against a fresh server. Each request's keys are drawn just before it is
    submitted (keys_mix of its sub-seed, on the host); it is submitted at its arrival time, or as
    soon as its keys exist if drawing them ran past that time, and its latency runs from submission
    to the end of its batch."""
    srv = BuildServer(leaf=leaf, bucket=bucket, workers=workers, mem_fraction=mem_fraction,
                      max_batch_keys=max_batch_keys, keep_results=False, chunk_keys=chunk_keys)
    reqs = []
    late = 0.0
    t0 = time.perf_counter()
    for i, (at, size, kseed) in enumerate(stream):
        keys = keys_mix(kseed, size)
        now = time.perf_counter()
        delay = t0 + at - now
        if delay > 0:
            time.sleep(delay)
        else:
            late = max(late, -delay)
        reqs.append(srv.submit(i, keys, t_arrival=max(t0 + at, now)))
        del keys
    for r in reqs:
        r.wait()
    t_end = max(r.t_done for r in reqs)
    srv.close()
    lat = np.array([r.latency for r in reqs]) * 1e3
    small = np.array([s <= 100_000 for _, s, _ in stream])
    total_keys = sum(s for _, s, _ in stream)
    span = t_end - t0
    return {
        "requests": len(reqs), "total_keys": int(total_keys), "workers": workers,
        "max_submit_lag_ms": round(late * 1e3, 3), "batches_grown": srv.grown,
        "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "mean_ms": round(float(lat.mean()), 3), "max_ms": round(float(lat.max()), 3),
        "p99_ms_small": round(float(np.percentile(lat[small], 99)), 3) if small.any() else None,
        "chunk_keys": chunk_keys,
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
    ap.add_argument("--chunk-keys", type=int, default=0, help="build requests above this size in bucket-range pieces")
    args = ap.parse_args()
    stream = poisson_stream(args.requests, args.rate, args.seed)
    out = run_stream(stream, workers=args.workers, leaf=args.leaf, bucket=args.bucket,
                     max_batch_keys=args.max_batch_keys, chunk_keys=args.chunk_keys)
    out.update({"metric": "ShockHash2 build service: p50/p99 build latency and aggregate keys/s",
                "config": {"variant": "ShockHash2", "leaf_size": args.leaf, "bucket_size": args.bucket,
                           "arrivals": f"Poisson, mean {args.rate}/s, seed {args.seed}",
                           "sizes": "round(10^(3+4u)) uint64 keys per request",
                           "keys": "remix(sub_seed ^ j * 0x9E3779B97F4A7C15), drawn at submission",
                           "sample": f"first {args.requests} requests of the 10,000-request stream"}})
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
