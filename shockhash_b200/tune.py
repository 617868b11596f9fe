"""Autotuner of the search kernels' launch parameters (``python -m shockhash_b200.tune``).

The split-seed search and the leaf searches have launch parameters that change their speed and
never their results (shg_engine_set_tuning): seeds per lane, threads per split block and the size
of a split round relative to a node's expected trials, the leaf grid's blocks per SM, the register
bound of the bipartite leaf kernel, the original leaf kernel's seeds per lane, and which pipes the
split search's remix runs on. The best values
depend on the leaf size (the reference's own search loops are ShockHash.h:404-434 for the original
leaves, ShockHash2-internal.h:386-483 for the bipartite finder and ShockHash.h:451-547 /
ShockHash2.h:290-386 for the splits).

For each configuration this module builds one synthetic key set (uint64 keys of the benchmark
stream, hashed as 8-byte strings; ShockHash2Flat<k> gets the same keys as 8-byte strings) and
tunes by coordinate descent: the split parameters first, then the leaf parameters, one parameter
at a time over its candidate values, each candidate timed by the CUDA-event time of the two search
stages together (the best of `reps` builds after one warm-up; the default ShockHash2 schedule runs
both searches in one launch). A value replaces the incumbent only when it is
faster by more than `min_gain`. Every build's products are compared with the first build's: a
parameter that changed a result would be a bug, and the tuner stops with an error.

The chosen values go to a table (default: shockhash_b200/tuning.tsv next to this file, which every
engine loads at creation), one line per parameter, with a comment per configuration giving the
stage times of the defaults and of the chosen values.
"""
import argparse
import datetime
import json
import os
import sys

import numpy as np

from . import SHOCKHASH, SHOCKHASH2, SIMDSHOCKHASH, TUNING_FLAT, Engine, keys_mt19937_64

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.tsv")

SPLIT_CANDIDATES = {"split_arith": (0, 1), "split_seeds_per_lane": (1, 2, 4), "split_threads": (128, 256, 512),
                    "split_round_div": (2, 4, 8, 16, 32)}
LEAF_CANDIDATES = {
    SHOCKHASH2: {"leaf_blocks_per_sm": (3, 4, 5, 6, 7, 8), "leaf_min_blocks": (4, 6, 8)},
    SHOCKHASH: {"leaf_blocks_per_sm": (4, 6, 8, 12, 16), "sh1_seeds_per_lane": (1, 2)},
    SIMDSHOCKHASH: {"leaf_blocks_per_sm": (4, 6, 8, 12, 16), "sh1_seeds_per_lane": (1, 2)},
    TUNING_FLAT: {"leaf_blocks_per_sm": (1, 2, 3)},
}
# (variant, leaf size, keys): the benchmark configurations' searches
CONFIGS = [(SHOCKHASH2, 64, 10_000_000), (SHOCKHASH, 30, 2_000_000), (SHOCKHASH, 40, 2_000_000),
           (SIMDSHOCKHASH, 30, 2_000_000),
           (TUNING_FLAT, 100, 500_000)]
NAMES = {SHOCKHASH: "ShockHash<{}>", SHOCKHASH2: "ShockHash2<{}>", SIMDSHOCKHASH: "SIMDShockHash<{}>",
         TUNING_FLAT: "ShockHash2Flat<{}>"}


class Tuner:
    def __init__(self, eng, variant, leaf, n, seed=7, reps=3, bucket=2000):
        self.eng, self.variant, self.leaf, self.bucket, self.reps = eng, variant, leaf, bucket, reps
        keys = keys_mt19937_64(seed, n)
        if variant == TUNING_FLAT:
            self.strings = (np.ascontiguousarray(keys, dtype="<u8").tobytes(),
                            np.arange(0, 8 * (n + 1), 8, dtype=np.uint64))
        self.keys = keys
        self.reference = None
        self.builds = 0
        self.trials = []

    def _build(self):
        """One build: (split ms, leaf ms, fingerprint of the products)."""
        self.builds += 1
        if self.variant == TUNING_FLAT:
            f = self.eng.build_flat_strings(self.leaf, self.strings)
            out = (0.0, float(f.stage_ms[4]), (f.thresholds_and_seeds.tobytes(), f.ribbon_bits.tobytes()))
            f.free()
            return out
        r = self.eng.build_u64(self.variant, self.leaf, self.keys, self.bucket)
        out = (r.stage_ms["splits"], r.stage_ms["leaves"], (r.descriptors.tobytes(), r.ribbon_bits.tobytes()))
        r.free()
        return out

    def measure(self, params):
        """Best split and leaf stage times over `reps` builds with `params` applied."""
        self.eng.set_tuning(self.variant, self.leaf, **params)
        self._build()  # warm-up (and buffer growth)
        best_s = best_l = float("inf")
        for _ in range(self.reps):
            s, l, fp = self._build()
            if self.reference is None:
                self.reference = fp
            elif fp != self.reference:
                raise RuntimeError(f"launch parameters {params} changed a build product")
            best_s, best_l = min(best_s, s), min(best_l, l)
        return best_s, best_l

    def descend(self, params, candidates, stage, min_gain):
        """Coordinate descent over `candidates`, timing both search stages together (the default
        ShockHash2 schedule runs them in one launch, so its time is all in the split stage); `stage`
        names the parameter group in self.trials, which receives every candidate's time."""
        best = sum(self.measure(params))
        for name, values in candidates.items():
            for v in values:
                if v == params[name]:
                    continue
                trial = dict(params, **{name: v})
                t = sum(self.measure(trial))
                self.trials.append({"group": ("split", "leaf")[stage], name: v, "ms": round(t, 3),
                                    "incumbent_ms": round(best, 3)})
                if t < best * (1.0 - min_gain):
                    params, best = trial, t
            self.eng.set_tuning(self.variant, self.leaf, **params)
        return params, best


def tune_config(eng, variant, leaf, n, reps=3, min_gain=0.02, log=print):
    tu = Tuner(eng, variant, leaf, n, reps=reps)
    # start from the library's untuned defaults, whatever table the engine loaded
    base = {"split_seeds_per_lane": 2, "split_threads": 256, "split_round_div": 8, "split_arith": 0,
            "leaf_blocks_per_sm": 0, "leaf_min_blocks": 6, "sh1_seeds_per_lane": 2, "queue_lag_rounds": 8}
    t0_split, t0_leaf = tu.measure(base)
    params = dict(base)
    split_c, leaf_c = dict(SPLIT_CANDIDATES), dict(LEAF_CANDIDATES[variant])
    if variant == SHOCKHASH2 and leaf <= 64:
        # the work-queue schedule (the default here): 256-thread blocks, at most 3 per SM
        split_c.pop("split_threads", None)
        leaf_c = {"leaf_blocks_per_sm": (1, 2, 3), "queue_lag_rounds": (0, 2, 4, 16, 32)}
    if variant == SIMDSHOCKHASH:  # its split hash has one arithmetic form, chosen by the engine
        split_c.pop("split_arith", None)
    if variant != TUNING_FLAT:
        params, _ = tu.descend(params, split_c, 0, min_gain)
    params, _ = tu.descend(params, leaf_c, 1, min_gain)
    t1_split, t1_leaf = tu.measure(params)
    res = {"variant": variant, "leaf": leaf, "keys": n, "params": params,
           "default_ms": {"splits": round(t0_split, 3), "leaves": round(t0_leaf, 3)},
           "tuned_ms": {"splits": round(t1_split, 3), "leaves": round(t1_leaf, 3)}, "builds": tu.builds,
           "trials": tu.trials}
    log(json.dumps(res))
    return res


def write_table(results, path, device_name=""):
    lines = ["# Launch parameters of the search kernels per configuration, written by python -m shockhash_b200.tune",
             f"# on {device_name or 'a CUDA device'}, {datetime.date.today().isoformat()}. Columns: variant (1 ShockHash, "
             "2 ShockHash2, 4 ShockHash2Flat, 5 SIMDShockHash) leaf name value.",
             "# Parameters change speed only; every result is identical."]
    for r in results:
        name = NAMES[r["variant"]].format(r["leaf"])
        d, t = r["default_ms"], r["tuned_ms"]
        lines.append(f"# {name}, {r['keys']} keys: splits {d['splits']} -> {t['splits']} ms, leaves {d['leaves']} -> "
                     f"{t['leaves']} ms (default -> tuned, best of the timed builds)")
        for k, v in r["params"].items():
            if k.startswith("sh1_") and r["variant"] not in (SHOCKHASH, SIMDSHOCKHASH):
                continue
            if k == "split_arith" and r["variant"] == SIMDSHOCKHASH:
                continue
            if k == "leaf_min_blocks" and (r["variant"] != SHOCKHASH2 or r["leaf"] > 64):
                continue
            if k.startswith("split_") and r["variant"] == TUNING_FLAT:
                continue
            lines.append(f"{r['variant']} {r['leaf']} {k} {v}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--min-gain", type=float, default=0.02, help="relative gain a value must show to be kept")
    ap.add_argument("--only", default="", help="comma-separated variant:leaf pairs (default: all configurations)")
    a = ap.parse_args(argv)
    prev = os.environ.get("SHG_TUNING_TABLE")
    os.environ["SHG_TUNING_TABLE"] = ""  # tune from the defaults, whatever table exists
    try:
        eng = Engine(a.device)
    finally:
        if prev is None:
            del os.environ["SHG_TUNING_TABLE"]
        else:
            os.environ["SHG_TUNING_TABLE"] = prev
    todo = CONFIGS
    if a.only:
        want = {tuple(int(x) for x in p.split(":")) for p in a.only.split(",")}
        todo = [c for c in CONFIGS if (c[0], c[1]) in want]
    results = [tune_config(eng, v, l, n, a.reps, a.min_gain) for v, l, n in todo]
    try:
        import torch
        dev = torch.cuda.get_device_name(a.device)
    except Exception:
        dev = ""
    write_table(results, a.out, dev)
    eng.close()
    print(json.dumps({"table": a.out, "configs": len(results)}), flush=True)


if __name__ == "__main__":
    sys.exit(main())
