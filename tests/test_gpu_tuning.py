"""Launch-parameter tuning (shg_engine_*_tuning, shockhash_b200.tune): every parameter value gives
identical products, tables load and reject bad entries, and the tuner writes a table engines read."""
import os

import numpy as np
import pytest

import shockhash_b200 as shg
from shockhash_b200 import tune

pytestmark = pytest.mark.gpu


def products(r):
    return (r.descriptors.tobytes(), r.bucket_size_acc.tobytes(), r.bucket_pos_acc.tobytes(), r.ribbon_keys.tobytes(),
            r.ribbon_bits.tobytes())


@pytest.mark.parametrize("variant,leaf", [(shg.SHOCKHASH2, 64), (shg.SHOCKHASH, 30), (shg.SHOCKHASH, 40),
                                          (shg.SHOCKHASH2, 24)])
def test_every_parameter_value_gives_identical_products(variant, leaf):
    keys = shg.keys_mt19937_64(77, 150_000)
    eng = shg.Engine(0)
    base = products(eng.build_u64(variant, leaf, keys, 2000))
    settings = [dict(split_seeds_per_lane=s, split_threads=t, split_round_div=d, split_arith=a)
                for s, t, d, a in ((1, 128, 2, 0), (4, 512, 32, 1), (4, 128, 1, 0), (1, 512, 64, 1), (2, 256, 16, 1),
                                   (2, 256, 8, 1))]
    if variant == shg.SHOCKHASH2:
        settings += [dict(leaf_blocks_per_sm=b, leaf_min_blocks=mb) for b, mb in ((1, 4), (3, 8), (8, 6))]
        settings += [dict(leaf_blocks_per_sm=0, queue_lag_rounds=q) for q in (1, 3, 64, 0)]
    else:
        settings += [dict(leaf_blocks_per_sm=b, sh1_seeds_per_lane=sp) for b, sp in ((1, 1), (16, 1), (4, 2))]
    for st in settings:
        eng.set_tuning(variant, leaf, **st)
        got = eng.get_tuning(variant, leaf)
        assert all(got[k] == v for k, v in st.items())
        assert products(eng.build_u64(variant, leaf, keys, 2000)) == base, st
    eng.close()


def test_flat_leaf_grid_gives_identical_products():
    keys = [f"flat-{i}".encode() for i in range(30_000)]
    eng = shg.Engine(0)
    base = eng.build_flat_strings(100, keys)
    ref = (base.thresholds_and_seeds.copy(), base.ribbon_bits.copy())
    for b in (1, 2):
        eng.set_tuning(shg.TUNING_FLAT, 100, leaf_blocks_per_sm=b)
        f = eng.build_flat_strings(100, keys)
        assert np.array_equal(f.thresholds_and_seeds, ref[0]) and np.array_equal(f.ribbon_bits, ref[1])
    eng.close()


def test_table_is_loaded_at_creation_and_bad_tables_are_rejected(tmp_path, monkeypatch):
    good = tmp_path / "t.tsv"
    good.write_text("# comment\n2 64 split_seeds_per_lane 4  # trailing\n\n2 64 leaf_min_blocks 8\n1 40 sh1_seeds_per_lane 1\n"
                    "4 100 leaf_blocks_per_sm 2\n3 30 split_threads 512\n")
    monkeypatch.setenv("SHG_TUNING_TABLE", str(good))
    eng = shg.Engine(0)
    assert eng.tuning_source() == str(good)
    t = eng.get_tuning(2, 64)
    assert t["split_seeds_per_lane"] == 4 and t["leaf_min_blocks"] == 8 and t["split_threads"] == 256
    assert eng.get_tuning(1, 40)["sh1_seeds_per_lane"] == 1
    assert eng.get_tuning(shg.TUNING_FLAT, 100)["leaf_blocks_per_sm"] == 2
    assert eng.get_tuning(1, 30)["split_threads"] == 512  # rotation fitting shares ShockHash's entry
    assert eng.get_tuning(2, 32) == eng.get_tuning(2, 33)  # untuned configurations: defaults
    with pytest.raises(shg.ShgError):
        eng.set_tuning(2, 64, split_threads=384)
    with pytest.raises(shg.ShgError):
        eng.set_tuning(2, 64, no_such_parameter=1)
    eng.close()
    bad = tmp_path / "bad.tsv"
    bad.write_text("2 64 split_seeds_per_lane 3\n")
    monkeypatch.setenv("SHG_TUNING_TABLE", str(bad))
    with pytest.raises(shg.ShgError):
        shg.Engine(0)
    monkeypatch.setenv("SHG_TUNING_TABLE", "")
    eng = shg.Engine(0)
    assert eng.tuning_source() == ""
    with pytest.raises(shg.ShgError):
        eng.load_tuning(str(tmp_path / "missing.tsv"))
    eng.close()


def test_tuner_writes_a_table_engines_read(tmp_path, monkeypatch):
    out = tmp_path / "tuned.tsv"
    monkeypatch.setattr(tune, "CONFIGS", [(shg.SHOCKHASH2, 16, 100_000)])
    monkeypatch.setattr(tune, "SPLIT_CANDIDATES", {"split_seeds_per_lane": (1, 2), "split_round_div": (4, 8)})
    monkeypatch.setattr(tune, "LEAF_CANDIDATES", {shg.SHOCKHASH2: {"leaf_blocks_per_sm": (2, 4)}})
    tune.main(["--out", str(out), "--reps", "1"])
    lines = [ln for ln in out.read_text().splitlines() if ln and not ln.startswith("#")]
    assert lines and all(ln.split()[:2] == ["2", "16"] for ln in lines)
    monkeypatch.setenv("SHG_TUNING_TABLE", str(out))
    eng = shg.Engine(0)
    assert eng.tuning_source() == str(out)
    for ln in lines:
        _, _, name, v = ln.split()
        assert eng.get_tuning(2, 16)[name] == int(v)
    eng.close()
