"""Benchmark: ShockHash2 construction (leaf size 64, bucket size 2000) of 10M uint64 keys
(std::mt19937_64 seed 7, each key hashed as its 8-byte string) on B200 GPUs.

One step = one full construction (hash, partition, split-seed search, bipartite leaf search,
Golomb-Rice encoding, copy-out of descriptors / accumulators / retrieval input to the host).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank builds its own 10M-key shard (seed 7 + rank): buckets are independent,
so shards need no data-path collective (weak scaling); the barrier and the max-over-ranks of the
device-timed steps use torch.distributed. Rank 0 prints one JSON line.

--impl reference times the reference's own CPU construction (oracle/_ref: the reference headers
compiled with the restated third-party stand-ins) on the same 10M keys, drawn by the oracle's own
generator, with all host threads; only the constructor call is timed, as the reference's benchmark
does. That process loads no library of this package.

Besides the headline line the GPU arm reports, on rank 0 at N=1:
  * cpu_baseline + parity: the reference CPU build of the same keys, its products compared word
    for word with the device build (descriptors, accumulators, retrieval input);
  * forms: the level schedule against the pipelined one and the per-leaf-launch form (1M keys),
    the SIMD format (SIMDShockHash<30>, 1M keys) against the reference's SIMD CPU build, the
    north-star size (100M keys), a Poisson serving stream, the device query of every key and the
    device retrieval structure;
  * forms.configs: the other configurations of the same path at stated sizes (ShockHash<30> over 1M
    printable strings, ShockHash<40> over 100M keys, ShockHash2Flat<100> over 50M Zipf-length
    strings), each with its leaf stage against its roofline and, on a bounded sample, the reference
    CPU build of the same keys and a word-for-word comparison.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_KEYS = 10_000_000
LEAF, BUCKET, VARIANT = 64, 2000, 2
SEED = 7
METRIC = "build ns/key on 1 B200, batched vs per-leaf GPU vs CPU, bit-exact; p99 latency"
CONFIG_NAME = "ShockHash2<64> b=2000, 10M uint64 keys (mt19937_64 seed 7) hashed to 128-bit"
MODES = ["default (work queue for ShockHash2 with leaves of up to 64 keys, else levels)", "levels", "per_leaf",
         "pipelined", "queue"]
# DRAM bytes (read + write) per key of one launch, from one ncu capture of the 1M-key case
# (profiles/k_tree_queue_sh2_l64.md, profiles/k_split_sh2_l64.md) scaled by keys: the work-queue
# kernel (the whole search: node keys read, retrieval bits and spilled leaf scratch written) and a
# quarter-split level launch of the level schedule (node keys read once; the partition's writes
# stay in L2).
QUEUE_DRAM_BYTES_PER_KEY = (13_114_880 + 81_113_856) / 1_000_000
SPLIT_DRAM_BYTES_PER_KEY = (6_560_256 + 512) / 1_000_000


def _workload(args):
    """--variant / --leaf / --seed / --n pick another configuration of the same path (e.g. the
    original ShockHash<40> with seed 11 for profiling); the defaults are the configuration above."""
    global VARIANT, LEAF, SEED, CONFIG_NAME
    VARIANT, LEAF, SEED = args.variant, args.leaf, args.seed
    if VARIANT == 4:
        CONFIG_NAME = (f"ShockHash2Flat<{LEAF}>, {args.n / 1e6:g}M uint64 keys (mt19937_64 seed {SEED}) as 8-byte "
                       "strings")
        return
    CONFIG_NAME = (f"{class_name(VARIANT, LEAF)} b={BUCKET}, {args.n / 1e6:g}M uint64 keys (mt19937_64 seed {SEED}) "
                   "hashed to 128-bit")


def class_name(variant, leaf):
    """The reference class a variant builds (shg_variant numbering)."""
    return {1: f"ShockHash<{leaf}>", 2: f"ShockHash2<{leaf}>", 3: f"ShockHash<{leaf}, true>",
            5: f"SIMDShockHash<{leaf}>", 6: f"SIMDShockHash<{leaf}, true>"}[variant]


def is_simd(variant):
    return variant in (5, 6)


def config_dict(args):
    """The workload, identical in both arms' JSON lines."""
    return {"workload": CONFIG_NAME, "keys_per_gpu": args.n, "leaf_size": LEAF, "bucket_size": BUCKET,
            "variant": class_name(VARIANT, LEAF).split("<")[0], "mode": MODES[args.mode],
            "key_encoding": "each uint64 key hashed as its 8-byte little-endian string (SpookyV2-128, seed 0)",
            "l2": "inputs (10M keys: 80 MB keys, 160 MB fingerprints, 240 MB partition buffers) exceed the 126 MB L2, "
                  "and a 256 MB buffer is written before every timed step, outside the timing",
            "parallelism": (f"one structure over {args.gpus} ranks: bucket-range shards after a device partition and "
                            "an NCCL all-to-all of 16-byte fingerprints" if getattr(args, "sharded", False) else
                            f"{args.gpus} independent bucket shards, no data-path collective")}


class _Summary:
    """What the report needs from one build, kept after its result block is released."""

    def __init__(self, r):
        self.stage_ms, self.work = dict(r.stage_ms), dict(r.work)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks + throttle reasons every 200 ms while running."""

    def __init__(self, device):
        self.device, self.samples, self._stop = device, [], threading.Event()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if "Active" in s[3 + i]
                          and "Not" not in s[3 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def u64_as_strings(keys):
    """uint64 keys as the reference's string keys: 8 little-endian bytes each, packed with offsets."""
    data = np.ascontiguousarray(keys, dtype="<u8").tobytes()
    offs = np.arange(0, 8 * (len(keys) + 1), 8, dtype=np.uint64)
    return data, offs


def cpu_reference(keys, threads, keep=False, variant=None, leaf=None, bucket=None):
    """The reference CPU construction of `keys` (uint64, given to the reference's string constructor
    as 8-byte strings): (constructor seconds, kind, threads used, products or None). Uses
    oracle/_ref (SIMDShockHash: its SIMD build); the C++ restatement oracle/_port (one thread) when
    that build is absent."""
    from oracle import bindings
    variant, leaf, bucket = variant or VARIANT, leaf or LEAF, bucket or BUCKET
    if bindings.ref_available():
        data, offs = u64_as_strings(keys)
        if is_simd(variant):
            b, secs = bindings.RefSimdLib().build_strings_packed_timed(variant == 6, leaf, data, offs, bucket, threads)
        else:
            b, secs = bindings.RefLib().build_strings_packed_timed(variant, leaf, data, offs, bucket, threads)
        if not keep:
            b.free()
            b = None
        return secs, "reference", threads, b
    lib = bindings.PortLib()
    data, offs = u64_as_strings(keys)
    first, second = lib.spooky128(bindings.split_strings(data, offs))
    t = time.perf_counter()
    b = lib.build_hash(variant, leaf, first, second, bucket)
    dt = time.perf_counter() - t
    if not keep:
        b.free()
        b = None
    return dt, "port", 1, b


def ref_phase_split(n):
    """The reference's own -DSTATS phase times for `n` keys of the same stream on one thread
    (oracle/ref_stats.py in a subprocess, since the STATS build prints to stdout), or None."""
    from oracle import bindings
    helper = os.path.join(ROOT, "oracle", "ref_stats.py")
    if not os.path.exists(bindings.STATS_SO) or VARIANT not in (1, 2):
        return None
    try:
        out = subprocess.run([sys.executable, helper, "--n", str(n), "--variant", str(VARIANT), "--leaf", str(LEAF),
                              "--bucket", str(BUCKET), "--seed", str(SEED)],
                             capture_output=True, text=True, timeout=180)
        if out.returncode != 0:
            return None
        return json.loads(out.stdout.strip().splitlines()[-1])
    except Exception:
        return None


def run_reference_arm(args):
    """The reference's CPU construction on the same keys and config as the GPU arm (rank 0 only)."""
    ws, rank, local = dist_env()
    if ws > 1 and rank != 0:
        return
    from oracle import bindings
    threads = os.cpu_count() or 1
    n = args.n
    if not bindings.ref_available():  # the one-thread restatement: a bounded sample of the stream
        n = min(n, int(os.environ.get("SHG_PORT_SAMPLE", "200000")))
    keys = bindings.keys_mt19937_64(SEED, n)
    for _ in range(args.warmup):
        cpu_reference(keys, threads)
    times, kind, used = [], None, threads
    for _ in range(args.steps):
        dt, kind, used, _ = cpu_reference(keys, threads)
        times.append(dt)
    ms = 1e3 * statistics.mean(times)
    v = ms * 1e6 / n
    sample = (f"all {n} keys of the mt19937_64 seed-{SEED} stream (oracle generator), reference string "
              "constructor, constructor call only" if n == args.n else
              f"first {n} keys of the mt19937_64 seed-{SEED} stream (bounded sample for the one-thread port)")
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ns/key", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config_dict(args),
            "cpu_baseline": {"value": round(v, 3), "unit": "ns/key", "cores": used, "kind": kind, "sample": sample,
                             "build": bindings.ref_build_info()},
            "e2e": {"value": round(v, 3), "unit": "ns/key", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def compare_products(r, b):
    """Word-for-word comparison of a device build with the reference's products."""
    checks = {
        "descriptors": np.array_equal(r.descriptors, b.desc),
        "bucket_size_acc": np.array_equal(r.bucket_size_acc, b.size_acc),
        "bucket_pos_acc": np.array_equal(r.bucket_pos_acc, b.pos_acc),
        "ribbon_keys": np.array_equal(r.ribbon_keys, b.ribbon_keys),
        "ribbon_bits": np.array_equal(r.ribbon_bits, b.ribbon_bits),
    }
    return {"bit_exact": all(checks.values()), "compared": sorted(checks), "mismatch": sorted(k for k, v in checks.items() if not v),
            "descriptor_words": int(len(b.desc)), "retrieval_keys": int(len(b.ribbon_keys))}


def search_roofline(queue_used, achieved, peak_eff, split_ms, split_ceil_s, leaf_ceil_s, n):
    """The dominant kernel against its ceiling. Level schedule: k_split, useful split evaluations per
    second against the evaluation-weighted peak of the node kinds' loops. Work-queue schedule:
    k_tree_queue, which runs both searches; its ceiling is the split ceiling plus the leaf ceiling
    (section 5 of the work model), expressed in split-evaluation equivalents so that `achieved` and
    `peak` keep the split kernel's unit."""
    if not queue_used:
        return {"kernel": "k_split (RecSplit split-seed search, level schedule)", "bound": "int",
                "achieved": round(achieved / 1e9, 3), "peak": round(peak_eff / 1e9, 3), "unit": "Gevals/s",
                "frac": round(achieved / peak_eff, 4), "traffic": round(SPLIT_DRAM_BYTES_PER_KEY * n),
                "traffic_note": "DRAM bytes of a quarter-split level launch (ncu, 1M keys, scaled by keys)",
                "note": "useful split evaluations (the reference's sequential count) / device time of the split "
                        "stage; peak = each node kind's evaluations at its inner loop's measured rate"}
    t = split_ms * 1e-3
    equiv = (split_ceil_s + leaf_ceil_s) * peak_eff  # split-evaluation equivalents of all the search work
    return {"kernel": "k_tree_queue (split nodes and leaves in one persistent launch)", "bound": "int",
            "achieved": round(equiv / t / 1e9, 3), "peak": round(peak_eff / 1e9, 3),
            "unit": "Gevals/s (split-evaluation equivalents)", "frac": round((split_ceil_s + leaf_ceil_s) / t, 4),
            "traffic": round(QUEUE_DRAM_BYTES_PER_KEY * n),
            "traffic_note": "DRAM bytes of the launch (ncu, 1M keys, scaled by keys)",
            "note": "frac = (split evaluations per node kind at that kind's measured loop peak + the bipartite leaf "
                    "work model's ceiling) / the launch's device time"}


def leaf_report(last, leaf_ms, leaf_peak, lpeaks, extra):
    """The leaf stage against its roofline. Original leaves: hash evaluations at the coverage loop's
    measured peak. Bipartite leaves: the stage's four operation kinds (hash evaluations, candidate-scan
    mask pairs, pair filters, pseudoforest edges) at their loops' measured peaks, summed into the
    time the stage's work takes with every lane busy; frac = that time / the measured stage time."""
    import shockhash_b200 as shg
    out = {"ms": round(leaf_ms, 3), "leaf_evals": last.work["leaf_evals"], "pairs": last.work["pairs"],
           "uf_edges": last.work["uf_edges"]}
    if lpeaks is None:
        rate = last.work["leaf_evals"] / (leaf_ms * 1e-3)
        out.update({"evals_per_s_g": round(rate / 1e9, 3), "peak_g": round(leaf_peak / 1e9, 3),
                    "frac": round(rate / leaf_peak, 4),
                    "note": "hash evaluations of the original leaf search per second vs the measured peak of its "
                            "coverage loop"})
        return out
    counts = {"hash_evals": last.work["leaf_evals"], "scan_tests": extra["leaf_scan_tests"],
              "pair_tests": last.work["pairs"], "uf_edges": last.work["uf_edges"]}
    ceil_s = shg.leaf_ceiling_s(counts, lpeaks)
    out.update({"counts": counts, "peaks_g_per_s": {k: round(v / 1e9, 3) for k, v in lpeaks.items()},
                "ceiling_ms": round(ceil_s * 1e3, 3),
                "ceiling_ms_by_op": {k: round(counts[k] / lpeaks[k] * 1e3, 3) for k in shg.LEAF_OPS},
                "frac": round(ceil_s * 1e3 / leaf_ms, 4),
                "note": "work model of the bipartite leaf search: each operation kind's count (as the sequential "
                        "reference performs them up to its answer, plus the candidates' cell rows) at the measured "
                        "peak of that loop run alone with every lane busy; frac = ceiling time / stage time"})
    return out


def run_flat(args):
    """ShockHash2Flat<k> (ShockHash2Flat.h:66-171) over n uint64 keys as 8-byte strings on one GPU:
    build time per key from host strings, and its leaf stage (k keys per bucket, one persistent leaf
    launch) against the bipartite work model's ceiling for leaves of its size."""
    import shockhash_b200 as shg
    n, k = args.n, LEAF
    keys = shg.keys_mt19937_64(SEED, n)
    strings = u64_as_strings(keys)
    eng = shg.Engine(0)
    lpeaks = shg.leaf_peaks(0, large=k > 64)
    for _ in range(args.warmup):
        eng.build_flat_strings(k, strings).free()
    totals, leaves = [], []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            f = eng.build_flat_strings(k, strings)
            totals.append(f.stage_ms[7])
            leaves.append(f.stage_ms[4])
            f.free()
    w = eng.last_work()["flat_leaves"]
    counts = {"hash_evals": w["hash_evals"], "scan_tests": w["scan_tests"], "pair_tests": w["pair_tests"],
              "uf_edges": w["uf_edges"]}
    leaf_ms = statistics.mean(leaves)
    ceil_s = shg.leaf_ceiling_s(counts, lpeaks)
    ms = statistics.mean(totals)
    line = {"metric": METRIC, "value": round(ms * 1e6 / n, 3), "unit": "ns/key", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": CONFIG_NAME, "keys": n, "k": k, "input": "host strings (8 bytes each)"},
            "leaf_stage": {"ms": round(leaf_ms, 3), "counts": counts,
                           "peaks_g_per_s": {x: round(v / 1e9, 3) for x, v in lpeaks.items()},
                           "ceiling_ms": round(ceil_s * 1e3, 3),
                           "ceiling_ms_by_op": {x: round(counts[x] / lpeaks[x] * 1e3, 3) for x in shg.LEAF_OPS},
                           "frac": round(ceil_s * 1e3 / leaf_ms, 4)},
            "clocks": clocks.summary(), "tuning": eng.get_tuning(shg.TUNING_FLAT, k)}
    eng.close()
    print(json.dumps(line), flush=True)


def timed_device_builds(eng, d_ptr, n, mode, flush, reps, warm=1):
    """Device-resident builds: `warm` untimed, then `reps` with the L2 flushed before each; returns
    (mean device ms, stage means, last result summary)."""
    import torch
    res = []
    for it in range(warm + reps):
        flush.zero_()
        torch.cuda.synchronize()
        rm = eng.build_u64_device(VARIANT, LEAF, d_ptr, n, BUCKET, mode)
        if it >= warm:
            res.append(_Summary(rm))
        rm.free()
    import shockhash_b200 as shg
    stages = {k: round(statistics.mean(x.stage_ms[k] for x in res), 3) for k in shg.STAGES}
    return statistics.mean(x.stage_ms["total"] for x in res), stages, res[-1]


def simd_format_form(eng, d_ptr, keys, n, flush):
    """SIMDShockHash<30> (the class the reference's SIMD benchmark builds as its ShockHash<30>; the leaf
    and bucket size of configuration 1) on the first n keys of the stream: the device build, the
    reference's SIMD CPU build of the same keys on all host threads, and a word-for-word comparison."""
    import torch
    import shockhash_b200 as shg
    leaf, ms = 30, []
    r = None
    for it in range(4):  # one warm-up, then three timed builds
        flush.zero_()
        torch.cuda.synchronize()
        if r is not None:
            r.free()
        r = eng.build_u64_device(shg.SIMDSHOCKHASH, leaf, d_ptr, n, BUCKET, shg.MODE_DEFAULT)
        if it:
            ms.append(r.stage_ms["total"])
    dev = statistics.mean(ms) * 1e6 / n
    dt, kind, cores, b = cpu_reference(keys[:n], os.cpu_count() or 1, keep=True, variant=shg.SIMDSHOCKHASH,
                                       leaf=leaf)
    out = {"class": f"SIMDShockHash<{leaf}> b={BUCKET}", "keys": n, "device_ns_per_key": round(dev, 3),
           "stage_ms": {k: round(v, 3) for k, v in r.stage_ms.items()},
           "cpu_reference_ns_per_key": round(dt * 1e9 / n, 3), "cpu_kind": kind, "cpu_cores": cores,
           "vs_cpu_reference": round(dt * 1e9 / n / dev, 1), "parity": compare_products(r, b)}
    b.free()
    r.free()
    return out


def synthetic_strings(kind, seed, n):
    """Seeded synthetic string keys of a configuration's shape (numpy's PCG64 stream, packed as
    (bytes, offsets[n+1])): "printable" = lengths uniform in 16..40, bytes uniform in 33..126;
    "zipf" = lengths l in 8..200 with P(l) proportional to (l - 7)^-1.1 (Zipf(1.1) on the clipped
    range, mean about 34 bytes), bytes uniform in 0..255."""
    rng = np.random.default_rng(seed)
    if kind == "printable":
        lengths = rng.integers(16, 41, size=n, dtype=np.uint64)
    else:
        w = np.arange(1, 194, dtype=np.float64) ** -1.1
        lengths = (8 + np.searchsorted(np.cumsum(w) / w.sum(), rng.random(n), side="right")).astype(np.uint64)
        np.minimum(lengths, 200, out=lengths)
    offs = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(lengths, out=offs[1:])
    total = int(offs[-1])
    if kind == "printable":
        data = rng.integers(33, 127, size=total, dtype=np.uint8).tobytes()
    else:
        data = rng.bytes(total)
    return data, offs


def config_forms(eng, dev, flush, with_cpu):
    """The other configurations of the same path at stated sizes: device stage times, the leaf stage
    against its roofline, and, where the reference's CPU build of the same keys finishes in seconds
    on the host cores, its time and a word-for-word comparison with the device build.
      c1: ShockHash<30, false>, b = 2000, 1M printable strings of 16..40 bytes (host strings in);
      c3: ShockHash<40, false>, b = 2000, 100M uint64 keys (mt19937_64 seed 11, device-resident),
          the CPU reference and the comparison on the first 200k keys;
      c4: ShockHash2Flat<100>, 50M strings of Zipf(1.1) lengths 8..200 (host strings in), the
          comparison on the first 20k keys."""
    import torch
    import shockhash_b200 as shg
    threads = os.cpu_count() or 1
    out = {}
    bindings = None
    if with_cpu:
        from oracle import bindings
        if not bindings.ref_available():
            bindings = None

    peak1, _ = shg.int_peak(dev.index or 0, 1 << 15, 1)  # the original leaf search's coverage loop

    def sh1_leaf_stage(stage_ms, work):
        rate = work["leaf_evals"] / (stage_ms["leaves"] * 1e-3)
        return {"evals_per_s_g": round(rate / 1e9, 3), "peak_g": round(peak1 / 1e9, 3), "frac": round(rate / peak1, 4),
                "note": "hash evaluations of the original leaf search per second vs the measured peak of its "
                        "coverage loop"}

    # c1
    n1 = int(os.environ.get("SHG_C1_N", "1000000"))
    data, offs = synthetic_strings("printable", 42, n1)
    r, dev_ms, wall_ms = None, [], []
    for it in range(4):  # one warm-up, then three timed builds
        if r is not None:
            r.free()
        t0 = time.perf_counter()
        r = eng.build_strings(shg.SHOCKHASH, 30, (data, offs), BUCKET)
        if it:
            wall_ms.append(1e3 * (time.perf_counter() - t0))
            dev_ms.append(r.stage_ms["total"])
    c1 = {"class": "ShockHash<30, false> b=2000", "keys": n1,
          "input": "host strings, 16-40 printable bytes (numpy seed 42)",
          "device_ns_per_key": round(statistics.mean(dev_ms) * 1e6 / n1, 3),
          "wall_ns_per_key": round(statistics.mean(wall_ms) * 1e6 / n1, 3),
          "stage_ms": {k: round(v, 3) for k, v in r.stage_ms.items()},
          "leaf_stage": sh1_leaf_stage(r.stage_ms, r.work)}
    if bindings:
        b, secs = bindings.RefLib().build_strings_packed_timed(shg.SHOCKHASH, 30, data, offs, BUCKET, threads)
        c1["cpu_reference_ns_per_key"] = round(secs * 1e9 / n1, 3)
        c1["cpu_cores"] = threads
        c1["vs_cpu_reference"] = round(secs * 1e9 / n1 / c1["device_ns_per_key"], 1)
        c1["parity"] = {"keys": n1, **compare_products(r, b)}
        b.free()
    r.free()
    out["c1_sh1_l30_strings"] = c1
    del data, offs

    # c3
    n3 = int(os.environ.get("SHG_C3_N", "100000000"))
    keys3 = shg.keys_mt19937_64(11, n3)
    d3 = torch.from_numpy(keys3.view(np.int64)).to(dev)
    res = []
    for it in range(2):  # one warm-up, then one timed build
        flush.zero_()
        torch.cuda.synchronize()
        rm = eng.build_u64_device(shg.SHOCKHASH, 40, d3.data_ptr(), n3, BUCKET)
        if it:
            res.append(_Summary(rm))
        rm.free()
    st = res[-1].stage_ms
    c3 = {"class": "ShockHash<40, false> b=2000", "keys": n3, "input": "device-resident uint64 keys (seed 11)",
          "device_ns_per_key": round(st["total"] * 1e6 / n3, 3), "stage_ms": {k: round(v, 3) for k, v in st.items()},
          "leaf_stage": sh1_leaf_stage(st, res[-1].work)}
    if bindings:
        ns = min(n3, int(os.environ.get("SHG_C3_CPU_SAMPLE", "200000")))
        dt, kind, cores, b = cpu_reference(keys3[:ns], threads, keep=True, variant=shg.SHOCKHASH, leaf=40)
        rs = eng.build_u64_device(shg.SHOCKHASH, 40, d3.data_ptr(), ns, BUCKET)
        c3["cpu_reference_ns_per_key"] = round(dt * 1e9 / ns, 3)
        c3["cpu_sample"] = f"first {ns} keys, all {cores} host threads"
        c3["vs_cpu_reference"] = round(dt * 1e9 / ns / c3["device_ns_per_key"], 1)
        c3["parity"] = {"keys": ns, **compare_products(rs, b)}
        rs.free()
        b.free()
    out["c3_sh1_l40_u64"] = c3
    del d3, keys3
    torch.cuda.empty_cache()

    # c4
    n4 = int(os.environ.get("SHG_C4_N", "50000000"))
    data, offs = synthetic_strings("zipf", 23, n4)
    lpeaks = shg.leaf_peaks(dev.index or 0, large=True)
    f, wall_ms = None, []
    for it in range(2):  # one warm-up, then one timed build
        if f is not None:
            f.free()
        t0 = time.perf_counter()
        f = eng.build_flat_strings(100, (data, offs))
        if it:
            wall_ms.append(1e3 * (time.perf_counter() - t0))
    w = eng.last_work()["flat_leaves"]
    counts = {"hash_evals": w["hash_evals"], "scan_tests": w["scan_tests"], "pair_tests": w["pair_tests"],
              "uf_edges": w["uf_edges"]}
    ceil_s = shg.leaf_ceiling_s(counts, lpeaks)
    names = ("hash", "layers", "fallback_build", "assign", "leaves", "copy_out", None, "total")  # shg_flat_result
    dq = f.device_query()
    q = dq.query_strings((data, offs))
    c4 = {"class": "ShockHash2Flat<100>", "keys": n4,
          "input": f"host strings, Zipf(1.1) lengths 8..200 (numpy seed 23, mean {len(data) / n4:.1f} bytes)",
          "wall_ns_per_key": round(statistics.mean(wall_ms) * 1e6 / n4, 3),
          "device_ns_per_key": round(f.stage_ms[7] * 1e6 / n4, 3),
          "stage_ms": {k: round(v, 3) for k, v in zip(names, f.stage_ms) if k},
          "leaf_stage": {"ms": round(f.stage_ms[4], 3), "counts": counts, "ceiling_ms": round(ceil_s * 1e3, 3),
                         "frac": round(ceil_s * 1e3 / f.stage_ms[4], 4)},
          "device_query_ns_per_key": round(dq.last_kernel_ms() * 1e6 / n4, 4),
          "device_query_is_permutation": bool(np.array_equal(np.sort(q), np.arange(n4, dtype=np.uint64)))}
    dq.close()
    f.free()
    del q
    if bindings:
        ns = min(n4, int(os.environ.get("SHG_C4_CPU_SAMPLE", "20000")))
        sd, so = data[:int(offs[ns])], offs[:ns + 1]
        ref = bindings.RefLib().flat_build_strings(100, [sd[int(so[i]):int(so[i + 1])] for i in range(ns)])
        fs = eng.build_flat_strings(100, (sd, so))
        checks = {"thresholds_and_seeds": np.array_equal(fs.thresholds_and_seeds, ref["thresholds_and_seeds"]),
                  "layer_bases": np.array_equal(fs.layer_bases, ref["layer_bases"]),
                  "fallback_seeds": np.array_equal(fs.fallback_seeds, ref["fallback_seeds"]),
                  "free_positions": np.array_equal(fs.free_positions, ref["free_positions"]),
                  "ribbon_keys": np.array_equal(fs.ribbon_keys, ref["ribbon_keys"]),
                  "ribbon_bits": np.array_equal(fs.ribbon_bits, ref["ribbon_bits"]),
                  "query": np.array_equal(fs.query_strings((sd, so)), ref["query"])}
        c4["parity"] = {"keys": ns, "against": "reference", "bit_exact": all(checks.values()),
                        "compared": sorted(checks), "mismatch": sorted(k for k, v in checks.items() if not v)}
        fs.free()
    out["c4_flat100_zipf_strings"] = c4
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_KEYS)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--variant", type=int, default=VARIANT, choices=[1, 2, 3, 4, 5, 6],
                    help="1 ShockHash, 2 ShockHash2, 3 ShockHash with rotation fitting, 4 ShockHash2Flat (leaf = k; "
                         "a profiling and C4 line), 5 SIMDShockHash, 6 SIMDShockHash with rotation fitting")
    ap.add_argument("--leaf", type=int, default=LEAF)
    ap.add_argument("--seed", type=int, default=SEED)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and parity leg")
    ap.add_argument("--no-forms", action="store_true", help="skip the comparison forms")
    ap.add_argument("--target-n", type=int, default=int(os.environ.get("SHG_TARGET_N", "100000000")),
                    help="keys of the north-star size leg (0 skips it)")
    ap.add_argument("--serve-requests", type=int, default=int(os.environ.get("SHG_SERVE_REQUESTS", "400")),
                    help="requests of the serving leg (0 skips it)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations' leg (ShockHash<30> strings, ShockHash<40> at 100M keys, "
                         "ShockHash2Flat<100> at 50M strings)")
    ap.add_argument("--sharded", action="store_true",
                    help="build ONE structure over all ranks: every step exchanges the ranks' keys by bucket range "
                         "(device partition + NCCL all-to-all) and builds each rank's buckets on its GPU")
    args = ap.parse_args()
    _workload(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    if VARIANT == 4:
        return run_flat(args)

    import torch
    import shockhash_b200 as shg
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = args.n

    keys = shg.keys_mt19937_64(SEED + rank, n)
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    h_keys = torch.from_numpy(keys.view(np.int64)).pin_memory()
    eng = shg.Engine(local)
    peak_forms = {}
    peaks = shg.split_peaks(local, detail=peak_forms, simd=is_simd(VARIANT))
    leaf_peak, _ = shg.int_peak(local, 1 << 15, 2 if VARIANT == 2 else 1)
    lpeaks = shg.leaf_peaks(local) if VARIANT == 2 else None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    args.sharded = args.sharded and ws > 1  # one rank: the sharded build is the plain build
    if args.sharded:  # fingerprints of this rank's keys, device-resident (the exchange moves 16 B per key)
        d_first = torch.empty(n, dtype=torch.int64, device=dev)
        d_second = torch.empty(n, dtype=torch.int64, device=dev)
        eng.hash_u64_device(d_keys.data_ptr(), n, d_first.data_ptr(), d_second.data_ptr())

    def step_device():
        if not args.sharded:
            return eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), n, BUCKET, args.mode)
        from shockhash_b200 import shard
        build = lambda f, s, nbg, b0, b1: eng.build_shard_hash128_device(VARIANT, LEAF, f.data_ptr(), s.data_ptr(),
                                                                        f.numel(), nbg, b0, b1, BUCKET, args.mode)
        part, _, _ = shard.build_sharded_tensors(build, d_first, d_second, BUCKET, engine=eng)
        return part

    for _ in range(args.warmup):
        step_device().free()
    # ---- device-resident timed steps (value)
    results, step_ms = [], []
    r = None
    barrier()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            if r is not None:
                r.free()  # the previous step's pinned result block is reused
            t0 = time.perf_counter()
            r = step_device()
            step_ms.append(1e3 * (time.perf_counter() - t0))
            results.append(_Summary(r))
        barrier()
    split_kinds = eng.last_work()
    tuning = {"table": os.path.relpath(eng.tuning_source(), ROOT) if eng.tuning_source() else None,
              "params": eng.get_tuning(VARIANT, LEAF)}
    dev_ms = [x.stage_ms["total"] for x in results]
    # ---- end to end through the public API, host (pinned) input, host outputs (e2e)
    e2e_ms = []
    r2 = None
    for _ in range(args.warmup):  # the host-input path has its own device and pinned buffers
        if r2 is not None:
            r2.free()
        r2 = eng.build_u64(VARIANT, LEAF, h_keys.numpy().view(np.uint64), BUCKET, args.mode)
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        if r2 is not None:
            r2.free()
        t0 = time.perf_counter()
        r2 = eng.build_u64(VARIANT, LEAF, h_keys.numpy().view(np.uint64), BUCKET, args.mode)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    barrier()
    r2.free()

    # the level schedule's stages, measured apart for the per-kernel fractions when the default build
    # runs both searches in the work-queue kernel
    lv = None
    if VARIANT == 2 and LEAF <= 64 and args.mode in (0, 4):
        t_lv, st_lv, last_lv = timed_device_builds(eng, d_keys.data_ptr(), n, shg.MODE_LEVELS, flush, reps=2)
        lv = (st_lv, last_lv, eng.last_work())

    def maxed(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    ms = maxed(statistics.mean(step_ms))
    ms_dev = maxed(statistics.mean(dev_ms))
    ms_e2e = maxed(statistics.mean(e2e_ms))
    p99 = maxed(float(np.percentile(e2e_ms, 99)))
    total_keys = n * ws
    split_ms = statistics.mean(x.stage_ms["splits"] for x in results)
    leaf_ms = statistics.mean(x.stage_ms["leaves"] for x in results)
    last = results[-1]
    achieved = last.work["split_evals"] / (split_ms * 1e-3)
    # denominator: each node kind's useful evaluations at that kind's measured loop peak
    peak_eff = shg.weighted_split_peak(split_kinds, peaks)
    # the default ShockHash2 build (leaves <= 64) runs both searches in the one work-queue kernel,
    # whose time is the split stage's: its ceiling is the split ceiling plus the leaf ceiling
    # (the library reports the whole launch as the split stage and no separate leaf stage then)
    queue_used = VARIANT == 2 and LEAF <= 64 and args.mode in (0, 4) and leaf_ms < 0.05 * split_ms
    split_ceil_s = sum(split_kinds[k] / peaks[k] for k in shg.SPLIT_KINDS if split_kinds[k])
    leaf_ceil_s = (shg.leaf_ceiling_s({"hash_evals": last.work["leaf_evals"], "scan_tests": split_kinds["leaf_scan_tests"],
                                       "pair_tests": last.work["pairs"], "uf_edges": last.work["uf_edges"]}, lpeaks)
                   if lpeaks else 0.0)
    bits_per_key = (r.descriptors.size * 64) / n

    line = None
    if rank == 0:
        cpu, parity = None, None
        if ws == 1 and not args.no_cpu:
            cpu_n = min(n, int(os.environ.get("SHG_CPU_SAMPLE", str(n))))
            dt, kind, cores, b = cpu_reference(keys[:cpu_n], os.cpu_count() or 1, keep=True)
            from oracle import bindings
            cpu = {"value": round(dt * 1e9 / cpu_n, 3), "unit": "ns/key", "cores": cores, "kind": kind,
                   "sample": (f"all {cpu_n} keys of the step's workload" if cpu_n == n else f"first {cpu_n} keys") +
                             ", reference string constructor, constructor call only, all host threads",
                   "build": bindings.ref_build_info()}
            if kind == "reference":  # the reference's split and leaf phases (its STATS timers, one thread)
                cpu["phases_1_thread"] = ref_phase_split(int(os.environ.get("SHG_CPU_PHASE_SAMPLE", "200000")))
            if cpu_n == n:
                parity = {"keys": n, "against": kind, **compare_products(r, b)}
            else:  # compare a device build of the same sample
                rs = eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), cpu_n, BUCKET, args.mode)
                parity = {"keys": cpu_n, "against": kind, **compare_products(rs, b)}
                rs.free()
            b.free()
        forms = {"default_ns_per_key": round(ms * 1e6 / n, 3)}
        if ws == 1 and not args.no_forms:
            for name, mode in (("levels", shg.MODE_LEVELS), ("pipelined", shg.MODE_PIPELINED), ("queue", shg.MODE_QUEUE)):
                t, _, _ = timed_device_builds(eng, d_keys.data_ptr(), n, mode, flush, reps=3)
                forms[f"{name}_device_ns_per_key"] = round(t * 1e6 / n, 3)
            # the per-leaf-launch comparison form on the first 1M keys of the same stream
            pl_n = min(n, int(os.environ.get("SHG_PER_LEAF_SAMPLE", "1000000")))
            t_pl, st_pl, _ = timed_device_builds(eng, d_keys.data_ptr(), pl_n, shg.MODE_PER_LEAF, flush, reps=1)
            t_b, st_b, _ = timed_device_builds(eng, d_keys.data_ptr(), pl_n, args.mode, flush, reps=3)
            rp = eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), pl_n, BUCKET, shg.MODE_PER_LEAF)
            rl = eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), pl_n, BUCKET, args.mode)
            forms["per_leaf"] = {"keys": pl_n, "per_leaf_launch_ns_per_key": round(t_pl * 1e6 / pl_n, 3),
                                 "batched_ns_per_key": round(t_b * 1e6 / pl_n, 3),
                                 "batched_speedup": round(t_pl / t_b, 2),
                                 "per_leaf_leaves_ms": st_pl["leaves"], "batched_leaves_ms": st_b["leaves"],
                                 "bit_exact_vs_batched": bool(np.array_equal(rp.descriptors, rl.descriptors)
                                                              and np.array_equal(rp.ribbon_bits, rl.ribbon_bits))}
            rp.free()
            rl.free()
            if VARIANT == 2:  # the SIMD format beside the headline configuration
                forms["simd_format"] = simd_format_form(eng, d_keys.data_ptr(), keys,
                                                        min(n, int(os.environ.get("SHG_SIMD_SAMPLE", "1000000"))), flush)
        if ws == 1 and not args.no_forms:
            # operator() for every key of the build on the device (keys resident, SpookyV2 fused)
            dq = shg.DeviceMphf(r, local)
            d_out = torch.empty(n, dtype=torch.int64, device=dev)
            for _ in range(3):
                dq.query_u64_device(d_keys.data_ptr(), n, d_out.data_ptr())
            q_ms = []
            for _ in range(5):
                flush.zero_()
                torch.cuda.synchronize()
                dq.query_u64_device(d_keys.data_ptr(), n, d_out.data_ptr())
                q_ms.append(dq.last_kernel_ms())
            forms["device_query_ns_per_key"] = round(statistics.mean(q_ms) * 1e6 / n, 4)
            forms["device_query_is_permutation"] = bool(
                torch.equal(torch.sort(d_out).values, torch.arange(n, device=dev, dtype=torch.int64)))
            dq.close()
            del d_out
            # compact retrieval structure from the build's retrieval input (device-resident input)
            d_rk = torch.from_numpy(r.ribbon_keys.view(np.int64)).to(dev)
            d_rb = torch.from_numpy(r.ribbon_bits).to(dev)
            rt_ms = []
            for it in range(3):  # one warm-up, then the mean of two
                rt = shg.Retrieval.build_device(eng, d_rk.data_ptr(), d_rb.data_ptr(), len(r.ribbon_keys))
                if it:
                    rt_ms.append(rt.build_ms())
                if it < 2:
                    rt.close()
            d_rout = torch.empty(len(r.ribbon_keys), dtype=torch.uint8, device=dev)
            rt.query_device(d_rk.data_ptr(), len(r.ribbon_keys), d_rout.data_ptr())
            forms["retrieval"] = {"keys": len(r.ribbon_keys), "build_ms": round(statistics.mean(rt_ms), 3),
                                  "bits_per_key": round(rt.bits() / max(1, len(r.ribbon_keys)), 4),
                                  "levels": rt.levels(), "all_bits_retrieved": bool(torch.equal(d_rout, d_rb))}
            rt.close()
            del d_rk, d_rb, d_rout
        d2h = (r.bucket_size_acc.nbytes + r.bucket_pos_acc.nbytes + r.descriptors.nbytes + r.ribbon_keys.nbytes
               + r.ribbon_bits.nbytes)
        if ws == 1 and not args.no_forms and args.target_n:
            # the north-star size: the first 100M keys of the same stream, device-resident
            tn = args.target_n
            t_keys = shg.keys_mt19937_64(SEED, tn)
            d_t = torch.from_numpy(t_keys.view(np.int64)).to(dev)
            del t_keys
            t, st, lw = timed_device_builds(eng, d_t.data_ptr(), tn, args.mode, flush, reps=2)
            sk = eng.last_work()
            t_split_ceil = sum(sk[k] / peaks[k] for k in shg.SPLIT_KINDS if sk[k])
            t_leaf_ceil = (shg.leaf_ceiling_s({"hash_evals": lw.work["leaf_evals"], "scan_tests": sk["leaf_scan_tests"],
                                               "pair_tests": lw.work["pairs"], "uf_edges": lw.work["uf_edges"]}, lpeaks)
                           if lpeaks else 0.0)
            searches_ms = st["splits"] + st["leaves"]  # one work-queue launch, or the split and leaf launches
            tgt = {"keys": tn, "device_ns_per_key": round(t * 1e6 / tn, 3), "stage_ms": st,
                   "search_frac": round((t_split_ceil + t_leaf_ceil) * 1e3 / searches_ms, 4)}
            if cpu:
                tgt["vs_cpu_reference"] = round(cpu["value"] / (t * 1e6 / tn), 1)
            if "per_leaf" in forms:
                tgt["vs_per_leaf_launch_form"] = round(forms["per_leaf"]["per_leaf_launch_ns_per_key"] / (t * 1e6 / tn), 1)
            forms["target"] = tgt
            del d_t
            torch.cuda.empty_cache()
        if ws == 1 and not args.no_forms and args.serve_requests:
            from shockhash_b200 import serve
            eng.close()  # the serving leg's workers hold their own engines
            eng = None
            torch.cuda.empty_cache()
            forms["serving"] = serve.run_stream(serve.poisson_stream(args.serve_requests, 200.0, 31), workers=2)
        if ws == 1 and not args.no_forms and not args.no_configs:  # after serving, whose host-side
            # request generation is sensitive to the host memory these large key sets take
            ceng = eng if eng is not None else shg.Engine(local)
            forms["configs"] = config_forms(ceng, dev, flush, not args.no_cpu)
            if ceng is not eng:
                ceng.close()
        line = {
            "metric": METRIC, "value": round(ms * 1e6 / total_keys, 3), "unit": "ns/key", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config_dict(args),
            "device_ms_per_step": round(ms_dev, 3),
            "stage_ms": {k: round(statistics.mean(x.stage_ms[k] for x in results), 3) for k in shg.STAGES},
            "e2e": {"value": round(ms_e2e * 1e6 / total_keys, 3), "unit": "ns/key", "p99_ms": round(p99, 3),
                    "h2d_bytes_per_step": int(n * 8), "d2h_bytes_per_step": int(d2h)},
            "roofline": search_roofline(queue_used, achieved, peak_eff, split_ms, split_ceil_s, leaf_ceil_s, n) | {
                         "peaks_by_kind_gevals": {k: round(v / 1e9, 3) for k, v in peaks.items()},
                         "peaks_by_form_gevals": {k: {f: round(x / 1e9, 3) for f, x in v.items()}
                                                  for k, v in peak_forms.items()},
                         "evals_by_kind": {k: split_kinds[k] for k in shg.SPLIT_KINDS},
                         "split_ceiling_ms": round(split_ceil_s * 1e3, 3), "leaf_ceiling_ms": round(leaf_ceil_s * 1e3, 3)},
            "leaf_stage": (leaf_report(last, leaf_ms, leaf_peak, lpeaks, split_kinds) if lv is None else
                           dict(leaf_report(lv[1], lv[0]["leaves"], leaf_peak, lpeaks, lv[2]),
                                schedule="level schedule, measured apart (2 builds)")),
            "split_stage": ({"ms": round(split_ms, 3), "frac": round(achieved / peak_eff, 4)} if lv is None else
                            {"ms": lv[0]["splits"], "schedule": "level schedule, measured apart (2 builds)",
                             "achieved_gevals": round(lv[1].work["split_evals"] / (lv[0]["splits"] * 1e-3) / 1e9, 3),
                             "peak_gevals": round(peak_eff / 1e9, 3),
                             "frac": round(lv[1].work["split_evals"] / (lv[0]["splits"] * 1e-3) / peak_eff, 4)}),
            "work": last.work, "bits_per_key_trees": round(bits_per_key, 4),
            "gpu_launches": int(last.work["launches"] * args.steps),
            "clocks": clocks.summary(),
            "cpu_baseline": cpu, "parity": parity, "forms": forms, "tuning": tuning,
        }
    r.free()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
