"""Autotuner table logic (host only): persistence, size ranges, lookup and
how the table fills the launch-shape fields."""
import pytest

from cvrp_aco_ocl_b200 import MODE_PARITY, MODE_THROUGHPUT, default_params
from cvrp_aco_ocl_b200.tune import TuneEntry, TuneTable, size_ranges


def entry(mode=MODE_THROUGHPUT, lo=3, hi=300, ants=128, apc=4, wpa=0, lsw=8, stage=-1, ms=1.0):
    return TuneEntry(mode, lo, hi, ants, apc, wpa, lsw, stage, ms, 25)


def test_size_ranges_cover_and_split_geometrically():
    r = size_ranges([1001, 101, 201, 501])
    assert r[0][0] == 3 and r[-1][1] == 1 << 30
    for (lo0, hi0), (lo1, hi1) in zip(r, r[1:]):
        assert hi0 + 1 == lo1
    assert r[1] == (int((101 * 201) ** 0.5) + 1, int((201 * 501) ** 0.5))


def test_table_roundtrip(tmp_path):
    t = TuneTable([entry(), entry(lo=301, hi=1 << 30, apc=16, stage=0)], device="B200")
    path = tmp_path / "t.json"
    t.save(str(path))
    u = TuneTable.load(str(path))
    assert u.device == "B200" and u.entries == t.entries


def test_table_rejects_unknown_version(tmp_path):
    path = tmp_path / "t.json"
    path.write_text('{"version": 9, "entries": []}')
    with pytest.raises(ValueError):
        TuneTable.load(str(path))


def test_lookup_by_mode_range_and_nearest_ants():
    t = TuneTable([entry(ants=64, apc=2), entry(ants=256, apc=8), entry(mode=MODE_PARITY, apc=1, wpa=4),
                   entry(lo=301, hi=2000, apc=16)])
    assert t.lookup(200, MODE_THROUGHPUT, 70).ants_per_block == 2
    assert t.lookup(200, MODE_THROUGHPUT, 200).ants_per_block == 8
    assert t.lookup(200, MODE_PARITY, 200).warps_per_ant == 4
    assert t.lookup(1500, MODE_THROUGHPUT, 128).ants_per_block == 16
    assert t.lookup(3000, MODE_THROUGHPUT, 128) is None


def test_add_replaces_same_key():
    t = TuneTable([entry(apc=2)])
    t.add(entry(apc=8))
    assert len(t.entries) == 1 and t.entries[0].ants_per_block == 8


def test_apply_fills_only_unset_fields():
    t = TuneTable([entry(apc=4, lsw=8, stage=-1)])
    p = default_params(201)
    p.mode, p.n_ants = MODE_THROUGHPUT, 128
    p.ls_warps = 16  # set by the caller: kept
    t.apply(p, 201)
    assert (p.ants_per_block, p.ls_warps, p.stage_matrix) == (4, 16, -1)
    q = default_params(5000)
    q.mode = MODE_THROUGHPUT
    t.apply(q, 5000)  # no range holds n: unchanged
    assert (q.ants_per_block, q.ls_warps, q.stage_matrix) == (0, 0, 0)


def test_shipped_prior_weights_match_the_network():
    import numpy as np
    from cvrp_aco_ocl_b200 import prior as PR
    from cvrp_aco_ocl_b200._lib import lib
    d = np.load(PR.DEFAULT_WEIGHTS)
    assert int(d["layers"]) == PR.LAYERS
    assert d["params"].size == lib().aco_mpnn_param_count(PR.LAYERS)
    assert np.all(np.isfinite(d["params"]))


def test_table_without_newer_fields_loads_and_fills(tmp_path):
    # a table written before ls_ants existed: the field defaults to 0 (automatic)
    path = tmp_path / "old.json"
    path.write_text('{"version": 1, "device": "x", "entries": [{"mode": 1, "n_lo": 3, "n_hi": 500, "ants": 128, '
                    '"ants_per_block": 4, "warps_per_ant": 0, "ls_warps": 16, "stage_matrix": 0, '
                    '"ms_per_iter": 1.0}]}')
    t = TuneTable.load(str(path))
    assert t.entries[0].ls_ants == 0 and t.entries[0].nn_ants == 0
    p = default_params(200)
    p.mode, p.n_ants = MODE_THROUGHPUT, 128
    t.apply(p, 200)
    assert p.ants_per_block == 4 and p.ls_warps == 16 and p.ls_ants == 0


def test_committed_table_loads():
    import os
    from cvrp_aco_ocl_b200 import tune
    t = TuneTable.load(os.path.join(os.path.dirname(tune.__file__), "tune_b200.json"))
    assert t.entries and all(e.ls_ants == 0 for e in t.entries)


def test_batch_entries_serve_batches_only_and_fill_the_new_fields():
    single = entry(lo=3, hi=2000, apc=1)
    b = TuneEntry(MODE_THROUGHPUT, 101, 1001, 128, 16, 0, 0, 0, 20.0, 25, 0, -1, 1, batch=1)
    t = TuneTable([single, b])
    assert t.lookup(550, MODE_THROUGHPUT, 128).ants_per_block == 1
    assert t.lookup(550, MODE_THROUGHPUT, 128, batch=True).ants_per_block == 16
    assert t.lookup(50, MODE_THROUGHPUT, 128, batch=True) is None
    p = default_params(1001)
    p.mode, p.n_ants = MODE_THROUGHPUT, 128
    t.apply(p, 550, batch=True)
    assert (p.ants_per_block, p.draw_warps, p.route_ls) == (16, -1, 1)
    q = default_params(1001)
    q.mode, q.n_ants, q.route_ls = MODE_THROUGHPUT, 128, -1  # set by the caller: kept
    t.apply(q, 550, batch=True)
    assert q.route_ls == -1 and q.draw_warps == -1
