"""CPU tests of host-side logic: the roofline arithmetic of bench.py, the
tuner's cache, and workload shapes the bench relies on."""
import importlib
import json

import numpy as np

import bench
from wind_b200 import autotune, networks as W


def test_sie_flops_per_substep():
    """LU-equivalent count (2/3)N^3 + 4N^2 + F_f + F_J per SIE substep."""
    katz = W.workload_katz96(4)
    assert abs(bench.flops_per_substep(katz, "sie") - (2 / 3 * 125 + 100 + 40 + 20)) < 1e-9
    ma = W.workload_mixed(40, seed=3, sizes=(157,), fractions=(1.0,), dt=1e-5)[0]
    n, r = 157, ma.net.n_react
    assert r == 1570
    want = 2 / 3 * n ** 3 + 4 * n * n + 5 * r + 8 * r
    assert abs(bench.flops_per_substep(ma, "sie") - want) < 1e-6 * want
    # RK2: the RHS plus the state update only
    assert abs(bench.flops_per_substep(ma, "rk2") - (5 * r + 2 * n)) < 1e-9


def test_dense_term_counts_its_matvec():
    wl = W.workload_dense(8)
    n, r = 32, wl.net.n_react
    want = 2 / 3 * n ** 3 + 4 * n * n + (5 * r + 2 * n * n) + 8 * r
    assert abs(bench.flops_per_substep(wl, "sie") - want) < 1e-9


def test_tuner_key_buckets_batch_size():
    wl = W.workload_katz96(1000)
    k1000 = autotune._key(wl, "sie", "device", "B200")
    k1024 = autotune._key(W.workload_katz96(1024), "sie", "device", "B200")
    k1025 = autotune._key(W.workload_katz96(1025), "sie", "device", "B200")
    assert k1000 == k1024 and k1025 != k1024
    assert autotune._key(wl, "rk2", "device", "B200") != k1000
    assert autotune._key(wl, "sie", "gold", "B200") != k1000


def test_tuner_cache_roundtrip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tuned.json"
    monkeypatch.setattr(autotune, "CACHE", str(path))
    assert autotune._load() == {}
    db = {"k": {"solver": "lu_f64", "spec_width": 4, "table": []}}
    autotune._save(db)
    assert json.loads(path.read_text()) == db
    assert autotune._load() == db
    path.write_text("{not json")
    assert autotune._load() == {}


def test_tuner_cache_path_follows_environment(tmp_path, monkeypatch):
    monkeypatch.setenv("WIND_TUNE_CACHE", str(tmp_path / "t.json"))
    mod = importlib.reload(autotune)
    try:
        assert mod.CACHE == str(tmp_path / "t.json")
    finally:
        monkeypatch.delenv("WIND_TUNE_CACHE")
        importlib.reload(autotune)


def test_bench_workloads_have_the_named_shapes():
    wl, desc = bench.make_workload("katz96", 0, 0.0)
    assert wl.net.nsys == 65536 and wl.net.n_eq == 5 and wl.tend - wl.tnow == 1e13
    assert (wl.atol, wl.rtol) == (1e-8, 1e-6)
    wl, _ = bench.make_workload("ma64", 16, 1e-4)
    assert wl.net.n_eq == 64 and wl.net.n_react == 640 and wl.net.nsys == 16
    s = wl.net.species
    assert s.dtype == np.uint16 and int(s.max()) < 64


def test_bench_shards_cover_the_dense_job_once():
    # strong scaling: two ranks' shards are the two halves of the same job
    full, _ = bench.make_workload("dense", 64, 0.0)
    parts = [bench.make_workload("dense", 64, 0.0, r, 2)[0] for r in range(2)]
    assert [p.net.nsys for p in parts] == [32, 32]
    assert np.array_equal(np.concatenate([p.y0 for p in parts]), full.y0)
    assert np.array_equal(np.concatenate([p.net.rates for p in parts]), full.net.rates)
    assert np.array_equal(np.concatenate([p.net.linear for p in parts]), full.net.linear)
    k = [bench.make_workload("katz96", 10, 0.0, r, 3)[0].net.nsys for r in range(3)]
    assert k == [4, 3, 3]


def test_bench_error_stats_count_divergent_systems():
    ref = np.array([[1.0, 2.0], [np.nan, 1.0], [1.0, 1.0], [3.0, np.inf]])
    y = np.array([[1.0, 2.0 + 2e-6], [np.nan, np.nan], [np.nan, 1.0], [3.0, 1.0]])
    e = bench.error_stats(y, ref, 1e-8)
    assert abs(e["max_rel_err"] - 1e-6) < 1e-12
    assert e["finite_systems"] == 1 and e["nonfinite_both"] == 1 and e["finiteness_differs"] == 2
    assert bench.error_stats(y[1:2], ref[1:2], 1e-8)["max_rel_err"] is None


def test_bench_json_is_strict():
    import json
    line = bench.finite_json({"a": float("nan"), "b": [1.0, float("inf")], "c": {"d": 2}})
    assert line == {"a": None, "b": [1.0, None], "c": {"d": 2}}
    json.dumps(line, allow_nan=False)
