"""Benchmark: ShockHash2 construction (leaf size 64, bucket size 2000) of 10M uint64 keys
(std::mt19937_64 seed 7, each key hashed as its 8-byte string) on B200 GPUs.

One step = one full construction (hash, partition, split-seed search, bipartite leaf search,
Golomb-Rice encoding, copy-out of descriptors / accumulators / retrieval input to the host).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank builds its own 10M-key shard (seed 7 + rank): buckets are independent,
so shards need no data-path collective (weak scaling); the barrier and the max-over-ranks of the
device-timed steps use torch.distributed. Rank 0 prints one JSON line.

--impl reference times the reference's own CPU construction (oracle/_ref: the reference headers
compiled with the restated third-party stand-ins; the C++ restatement oracle/port when that build
is absent) on a bounded sample of the same key stream, with all host threads.
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


def _workload(args):
    """--variant / --leaf / --seed / --n pick another configuration of the same path (e.g. the
    original ShockHash<40> with seed 11 for profiling); the defaults are the configuration above."""
    global VARIANT, LEAF, SEED, CONFIG_NAME
    VARIANT, LEAF, SEED = args.variant, args.leaf, args.seed
    name = "ShockHash2" if VARIANT == 2 else "ShockHash"
    CONFIG_NAME = (f"{name}<{LEAF}> b={BUCKET}, {args.n / 1e6:g}M uint64 keys (mt19937_64 seed {SEED}) "
                   "hashed to 128-bit")


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


def cpu_reference(keys, threads):
    """Time the reference CPU construction (oracle/_ref, else oracle/port) on `keys`."""
    from oracle.bindings import PortLib, RefLib, ref_available
    import shockhash_b200 as shg
    eng = None
    # 128-bit fingerprints as the reference computes them (spooky over the 8-byte strings)
    from oracle import bindings
    data = keys.astype("<u8").tobytes()
    offs = np.arange(0, 8 * (len(keys) + 1), 8, dtype=np.uint64)
    first = np.zeros(len(keys), np.uint64)
    second = np.zeros(len(keys), np.uint64)
    if ref_available():
        lib = RefLib()
        import ctypes
        lib.lib.ref_spooky128.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                          ctypes.c_void_p]
        lib.lib.ref_spooky128(data, bindings._ptr(offs), len(keys), bindings._ptr(first), bindings._ptr(second))
        t = time.perf_counter()
        b = lib.build_hash(VARIANT, LEAF, first, second, BUCKET, threads)
        dt = time.perf_counter() - t
        b.free()
        return dt, "reference", threads
    lib = PortLib()
    first, second = lib.spooky128([keys[i:i + 1].tobytes() for i in range(len(keys))])
    t = time.perf_counter()
    b = lib.build_hash(VARIANT, LEAF, first, second, BUCKET)
    dt = time.perf_counter() - t
    b.free()
    return dt, "port", 1


def ref_phase_split(n):
    """The reference's own -DSTATS phase times for `n` keys of the same stream on one thread
    (oracle/ref_stats.py in a subprocess, since the STATS build prints to stdout), or None."""
    helper = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "ref_stats.py")
    if not os.path.exists(os.path.join(os.path.dirname(helper), "_ref", "libshref_stats.so")):
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
    ws, rank, local = dist_env()
    if ws > 1 and rank != 0:
        return
    import shockhash_b200 as shg
    threads = os.cpu_count() or 1
    sample = int(os.environ.get("SHG_REF_SAMPLE", "1000000"))
    keys = shg.keys_mt19937_64(SEED, sample)
    for _ in range(args.warmup):
        cpu_reference(keys, threads)
    times, kind = [], None
    for _ in range(args.steps):
        dt, kind, used = cpu_reference(keys, threads)
        times.append(dt)
    ms = 1e3 * statistics.mean(times)
    v = ms * 1e6 / sample
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ns/key", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": CONFIG_NAME, "sample_keys": sample, "threads": used},
            "cpu_baseline": {"value": round(v, 3), "unit": "ns/key", "cores": used, "kind": kind,
                             "sample": f"{sample} keys of the same mt19937_64 seed-7 stream, constructor only"},
            "e2e": {"value": round(v, 3), "unit": "ns/key", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_KEYS)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--variant", type=int, default=VARIANT, choices=[1, 2])
    ap.add_argument("--leaf", type=int, default=LEAF)
    ap.add_argument("--seed", type=int, default=SEED)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-forms", action="store_true", help="skip the per-leaf-launch comparison form")
    args = ap.parse_args()
    _workload(args)
    if args.impl == "reference":
        return run_reference_arm(args)

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
    peak_evals, _ = shg.int_peak(local, 1 << 15)
    leaf_peak, _ = shg.int_peak(local, 1 << 15, 1 if VARIANT == 1 else 2)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def step_device():
        return eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), n, BUCKET, args.mode)

    for _ in range(args.warmup):
        step_device()
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
    dev_ms = [r.stage_ms["total"] for r in results]
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
    bits_per_key = (r.descriptors.size * 64) / n

    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu:
            sample = int(os.environ.get("SHG_CPU_SAMPLE", "2000000"))
            dt, kind, cores = cpu_reference(keys[:sample], os.cpu_count() or 1)
            cpu = {"value": round(dt * 1e9 / sample, 3), "unit": "ns/key", "cores": cores, "kind": kind,
                   "sample": f"first {sample} keys of the same stream, constructor only, all host threads"}
            if kind == "reference":  # the reference's split and leaf phases (its STATS timers, one thread)
                cpu["phases_1_thread"] = ref_phase_split(int(os.environ.get("SHG_CPU_PHASE_SAMPLE", "200000")))
        forms = {"default_ns_per_key": round(ms * 1e6 / n, 3)}
        if ws == 1 and not args.no_forms:
            for name, mode in (("levels", shg.MODE_LEVELS), ("pipelined", shg.MODE_PIPELINED)):
                t = []
                for it in range(4):  # one warm-up, then the mean of three
                    flush.zero_()
                    torch.cuda.synchronize()
                    rm = eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), n, BUCKET, mode)
                    if it:
                        t.append(rm.stage_ms["total"])
                    rm.free()
                forms[f"{name}_device_ns_per_key"] = round(statistics.mean(t) * 1e6 / n, 3)
        if ws == 1 and not args.no_forms:
            pl_n = int(os.environ.get("SHG_PER_LEAF_SAMPLE", "100000"))
            for _ in range(2):  # the second of each is reported (the first grows buffers for the size)
                rp = eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), pl_n, BUCKET, shg.MODE_PER_LEAF)
                rl = eng.build_u64_device(VARIANT, LEAF, d_keys.data_ptr(), pl_n, BUCKET, shg.MODE_LEVELS)
            forms["per_leaf_launch_ns_per_key_at_%d" % pl_n] = round(rp.stage_ms["total"] * 1e6 / pl_n, 3)
            forms["batched_ns_per_key_at_%d" % pl_n] = round(rl.stage_ms["total"] * 1e6 / pl_n, 3)
            forms["per_leaf_bit_exact_vs_batched"] = bool(np.array_equal(rp.descriptors, rl.descriptors))
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
        line = {
            "metric": METRIC, "value": round(ms * 1e6 / total_keys, 3), "unit": "ns/key", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": CONFIG_NAME, "keys_per_gpu": n, "leaf_size": LEAF, "bucket_size": BUCKET,
                       "variant": "ShockHash2" if VARIANT == 2 else "ShockHash", "mode": ["default (levels)", "levels", "per_leaf", "pipelined"][args.mode],
                       "l2": "flushed (256 MB write) before every timed step, outside the timing",
                       "parallelism": f"{ws} independent bucket shards, no data-path collective"},
            "device_ms_per_step": round(ms_dev, 3),
            "stage_ms": {k: round(statistics.mean(x.stage_ms[k] for x in results), 3) for k in shg.STAGES},
            "e2e": {"value": round(ms_e2e * 1e6 / total_keys, 3), "unit": "ns/key", "p99_ms": round(p99, 3),
                    "h2d_bytes_per_step": int(n * 8), "d2h_bytes_per_step": int(d2h)},
            "roofline": {"kernel": "k_split (RecSplit split-seed search)", "bound": "int",
                         "achieved": round(achieved / 1e9, 3), "peak": round(peak_evals / 1e9, 3),
                         "unit": "Gevals/s", "frac": round(achieved / peak_evals, 4), "traffic": None,
                         "note": "useful split evaluations (the reference's sequential count) / device time of "
                                 "the split stage; peak = measured integer microbenchmark of the same "
                                 "arithmetic (no memory traffic)"},
            "leaf_stage": {"ms": round(leaf_ms, 3), "leaf_evals": last.work["leaf_evals"],
                           "evals_per_s_g": round(last.work["leaf_evals"] / (leaf_ms * 1e-3) / 1e9, 3),
                           "peak_g": round(leaf_peak / 1e9, 3),
                           "frac": round(last.work["leaf_evals"] / (leaf_ms * 1e-3) / leaf_peak, 4),
                           "note": "hash evaluations of the leaf search per second vs the measured peak of its "
                                   "inner loop (original leaves: coverage loop; bipartite leaves: raw-seed loop, "
                                   "which leaves out the candidate scans and pseudoforest tests)",
                           "pairs": last.work["pairs"], "uf_edges": last.work["uf_edges"]},
            "work": last.work, "bits_per_key_trees": round(bits_per_key, 4),
            "gpu_launches": int(last.work["launches"] * args.steps),
            "clocks": clocks.summary(),
            "cpu_baseline": cpu, "forms": forms,
        }
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
